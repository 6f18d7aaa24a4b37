"""The kernels' own pass code and codelets, run on the CPU, against the oracle.

libfft3d_hostcheck.so executes stage_in / pass_z / pass_y / pass_x_out of
opt-fft_b200/csrc/volume.cuh and the codelets of codelets.cuh -- the same
templates the VOLUME kernels instantiate -- thread by thread.  This checks every
codelet route (folded direct, Rader-17, PFA, Cooley-Tukey), the shared-memory
layouts (natural, padded, XOR-swizzled) and the partial-CTA tail without a GPU.
"""
import glob
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN, field

C128_TOL = 1e-13
C64_TOL = 1e-6

# (shape, alg, vpc) pairs the emulator was built with
GEOMS = [((6, 6, 6), 0, 16), ((8, 8, 8), 0, 8), ((12, 12, 12), 0, 2), ((16, 16, 16), 0, 1),
         ((17, 17, 17), 0, 1), ((17, 17, 17), 1, 1), ((24, 24, 24), 0, 1), ((8, 8, 16), 0, 8),
         ((16, 16, 32), 0, 1), ((36, 36, 36), 0, 1), ((2, 3, 5), 0, 3), ((7, 11, 13), 0, 2),
         ((9, 9, 9), 0, 2), ((5, 8, 12), 0, 1), ((32, 8, 4), 0, 1), ((13, 5, 8), 0, 1),
         ((4, 4, 4), 0, 2), ((1, 8, 8), 0, 1), ((8, 1, 8), 0, 1), ((8, 8, 1), 0, 1),
         ((1, 1, 1), 0, 1), ((3, 3, 3), 0, 1), ((17, 2, 2), 0, 1), ((13, 13, 13), 0, 2),
         ((23, 23, 23), 0, 1), ((17, 17, 17), 2, 1),
         # the group sizes of the VOLUME kernels for the reference's other extents
         ((1, 1, 1), 0, 64), ((3, 3, 3), 0, 32), ((4, 4, 4), 0, 16), ((9, 9, 9), 0, 4),
         ((10, 10, 10), 0, 2), ((15, 15, 15), 0, 1), ((2, 3, 5), 0, 32), ((5, 8, 12), 0, 4),
         ((13, 5, 8), 0, 4), ((17, 2, 2), 0, 16), ((32, 8, 4), 0, 2), ((1, 8, 8), 0, 32),
         ((8, 1, 8), 0, 32), ((8, 8, 1), 0, 32),
         # the rest of the reference's test geometries (python/test_fft3d.py:25-36)
         ((2, 2, 2), 0, 64), ((5, 5, 5), 0, 24), ((7, 7, 7), 0, 8), ((11, 11, 11), 0, 2),
         ((49, 2, 2), 0, 10), ((25, 4, 3), 0, 10), ((27, 2, 2), 0, 18), ((19, 3, 2), 0, 17),
         ((23, 2, 2), 0, 22), ((47, 3, 2), 0, 7), ((83, 2, 1), 0, 18), ((97, 2, 1), 0, 15),
         ((1, 1, 16), 0, 64), ((1, 7, 1), 0, 64), ((3, 5, 7), 0, 29), ((4, 6, 10), 0, 11),
         ((16, 3, 5), 0, 12), ((24, 18, 12), 0, 1), ((2, 2, 64), 0, 12), ((64, 2, 2), 0, 8),
         ((9, 25, 7), 0, 1), ((20, 12, 6), 0, 1), ((11, 4, 9), 0, 7)]
GEOMS64 = [((6, 6, 6), 0, 32), ((8, 8, 8), 0, 16), ((12, 12, 12), 0, 4), ((16, 16, 16), 0, 2),
           ((17, 17, 17), 0, 2), ((17, 17, 17), 1, 2), ((17, 17, 17), 2, 2),
           ((24, 24, 24), 0, 1), ((8, 8, 16), 0, 16),
           ((16, 16, 32), 0, 1), ((36, 36, 36), 0, 1), ((13, 13, 13), 0, 4), ((23, 23, 23), 0, 1),
           ((1, 1, 1), 0, 128), ((3, 3, 3), 0, 64), ((4, 4, 4), 0, 32), ((9, 9, 9), 0, 8),
           ((10, 10, 10), 0, 4), ((15, 15, 15), 0, 2), ((2, 3, 5), 0, 64), ((7, 11, 13), 0, 4),
           ((5, 8, 12), 0, 8), ((13, 5, 8), 0, 8), ((17, 2, 2), 0, 32), ((32, 8, 4), 0, 4),
           ((1, 8, 8), 0, 64), ((8, 1, 8), 0, 64), ((8, 8, 1), 0, 64),
           ((2, 2, 2), 0, 64), ((5, 5, 5), 0, 49), ((7, 7, 7), 0, 17), ((11, 11, 11), 0, 4),
           ((49, 2, 2), 0, 20), ((25, 4, 3), 0, 20), ((27, 2, 2), 0, 37), ((19, 3, 2), 0, 35),
           ((23, 2, 2), 0, 44), ((47, 3, 2), 0, 14), ((83, 2, 1), 0, 37), ((97, 2, 1), 0, 31),
           ((1, 1, 16), 0, 64), ((1, 7, 1), 0, 64), ((3, 5, 7), 0, 58), ((4, 6, 10), 0, 23),
           ((16, 3, 5), 0, 25), ((24, 18, 12), 0, 1), ((30, 30, 30), 0, 1), ((2, 2, 64), 0, 24),
           ((64, 2, 2), 0, 16), ((9, 25, 7), 0, 3), ((20, 12, 6), 0, 3), ((11, 4, 9), 0, 15)]


def run(hc, x, shape, prec, sign, alg, vpc):
    out = np.empty_like(x)
    rc = hc.hostcheck_fft3d(shape[0], shape[1], shape[2], prec, sign, alg, vpc,
                            x.ctypes.data, out.ctypes.data, x.shape[0])
    assert rc == 0, f"no emulator entry for {shape} prec={prec} alg={alg} vpc={vpc}"
    return out


def nbatch(shape, vpc):
    # a full CTA plus a partial one, capped for the big volumes
    v = int(np.prod(shape))
    return vpc + max(1, vpc // 2) if v <= 8192 else 1


@pytest.mark.parametrize("shape,alg,vpc", GEOMS, ids=[f"{g[0]}-alg{g[1]}" for g in GEOMS])
@pytest.mark.parametrize("sign", [-1, +1])
def test_c128_pass_code(hostcheck, shape, alg, vpc, sign):
    rng = np.random.default_rng(1000 + sum(shape) + alg)
    x = field(rng, (nbatch(shape, vpc),) + shape)
    got = run(hostcheck, x, shape, 0, sign, alg, vpc)
    want = oracle.fft3d(x) if sign < 0 else oracle.ifft3d(x)
    err = oracle.rel_error_per_volume(got, want).max()
    assert err < C128_TOL, err


@pytest.mark.parametrize("shape,alg,vpc", GEOMS64, ids=[f"{g[0]}-alg{g[1]}" for g in GEOMS64])
@pytest.mark.parametrize("sign", [-1, +1])
def test_c64_pass_code(hostcheck, shape, alg, vpc, sign):
    rng = np.random.default_rng(2000 + sum(shape) + alg)
    x = field(rng, (nbatch(shape, vpc),) + shape, dtype=np.complex64)
    got = run(hostcheck, x, shape, 1, sign, alg, vpc)
    x64 = x.astype(np.complex128)
    want = oracle.fft3d(x64) if sign < 0 else oracle.ifft3d(x64)
    err = oracle.rel_error_per_volume(got, want).max()
    assert err < C64_TOL, err


@pytest.mark.parametrize("prec,c", [(0, 4), (0, 6), (0, 9), (1, 2), (1, 4), (1, 6)])
@pytest.mark.parametrize("sign", [-1, +1])
def test_cluster_data_movement(hostcheck, prec, c, sign):
    """The CLUSTER kernel's slab split and distributed x-pass gather (alg = 100 + C)."""
    shape = (36, 36, 36)
    rng = np.random.default_rng(3000 + c + prec)
    dt = np.complex128 if prec == 0 else np.complex64
    x = field(rng, (2,) + shape, dist="normal", dtype=dt)
    got = run(hostcheck, x, shape, prec, sign, 100 + c, 1)
    x64 = x.astype(np.complex128)
    want = oracle.fft3d(x64) if sign < 0 else oracle.ifft3d(x64)
    err = oracle.rel_error_per_volume(got, want).max()
    assert err < (C128_TOL if prec == 0 else C64_TOL), err


BST = [((17, 17, 17), 0, 1, 3), ((17, 17, 17), 1, 2, 3), ((13, 13, 13), 0, 1, 2),
       ((13, 13, 13), 0, 2, 3), ((13, 13, 13), 1, 2, 3),
       # swizzled layouts: x lines re-laid through registers
       ((8, 8, 8), 0, 1, 3), ((16, 16, 16), 0, 1, 2), ((16, 16, 16), 1, 1, 2)]


@pytest.mark.parametrize("shape,prec,vpc,nvol", BST,
                         ids=[f"{t[0]}-c{128 if t[1] == 0 else 64}-vpc{t[2]}" for t in BST])
@pytest.mark.parametrize("sign", [-1, +1])
def test_stream_bulk_store_item(hostcheck, shape, prec, vpc, nvol, sign):
    """The STREAM kernel's bulk-store item (alg = 400 + ALG): x pass in place and
    the natural-layout stage copied out whole, a partial group included."""
    rng = np.random.default_rng(3500 + prec + shape[0])
    dt = np.complex128 if prec == 0 else np.complex64
    x = field(rng, (nvol,) + shape, dtype=dt)
    got = run(hostcheck, x, shape, prec, sign, 400, vpc)
    x64 = x.astype(np.complex128)
    want = oracle.fft3d(x64) if sign < 0 else oracle.ifft3d(x64)
    err = oracle.rel_error_per_volume(got, want).max()
    assert err < (C128_TOL if prec == 0 else C64_TOL), err


@pytest.mark.parametrize("prec,vpc", [(0, 1), (1, 2)])
@pytest.mark.parametrize("sign", [-1, +1])
def test_stream_bulk_store_crt17(hostcheck, prec, vpc, sign):
    """The bulk-store item with the CRT 17-point codelet (alg = 400 + 2)."""
    shape = (17, 17, 17)
    rng = np.random.default_rng(3700 + prec)
    dt = np.complex128 if prec == 0 else np.complex64
    x = field(rng, (3,) + shape, dtype=dt)
    got = run(hostcheck, x, shape, prec, sign, 402, vpc)
    x64 = x.astype(np.complex128)
    want = oracle.fft3d(x64) if sign < 0 else oracle.ifft3d(x64)
    assert oracle.rel_error_per_volume(got, want).max() < (C128_TOL if prec == 0 else C64_TOL)


@pytest.mark.parametrize("n,prec,pl", [(36, 0, 4), (36, 1, 6), (36, 1, 4)])
@pytest.mark.parametrize("sign", [-1, +1])
def test_two_phase_cube(hostcheck, n, prec, pl, sign):
    """The batch kernel's two-phase route through scratch (alg = 200 + slab
    planes): 36^3 in both kernel classes' slabs."""
    shape = (n, n, n)
    rng = np.random.default_rng(4000 + pl)
    dt = np.complex128 if prec == 0 else np.complex64
    x = field(rng, (2,) + shape, dist="normal", dtype=dt)
    got = run(hostcheck, x, shape, prec, sign, 200 + pl, 1)
    x64 = x.astype(np.complex128)
    want = oracle.fft3d(x64) if sign < 0 else oracle.ifft3d(x64)
    err = oracle.rel_error_per_volume(got, want).max()
    assert err < (C128_TOL if prec == 0 else C64_TOL), err


TWOPASS = [((36, 36, 36), 0, 4, 11), ((36, 36, 36), 0, 2, 3), ((36, 36, 36), 0, 6, 9),
           ((36, 36, 36), 1, 4, 11), ((36, 36, 36), 1, 6, 2), ((16, 16, 32), 0, 4, 13),
           ((16, 16, 32), 0, 8, 1), ((6, 9, 5), 0, 3, 41), ((45, 45, 45), 0, 3, 5),
           ((45, 45, 45), 1, 5, 3), ((64, 64, 64), 0, 1, 3), ((64, 64, 64), 1, 2, 2),
           ((36, 36, 36), 0, 3, 7), ((30, 30, 30), 0, 3, 4), ((30, 30, 30), 0, 5, 3)]


@pytest.mark.parametrize("shape,prec,g,nvol", TWOPASS,
                         ids=[f"{t[0]}-c{128 if t[1] == 0 else 64}-g{t[2]}-b{t[3]}" for t in TWOPASS])
@pytest.mark.parametrize("sign", [-1, +1])
def test_twopass_items(hostcheck, shape, prec, g, nvol, sign):
    """The TWOPASS kernel's plane and row items in ticket order (alg = 300 + G):
    decode, element maps, scratch-ring reuse; batches below and above the lag D
    and the ring size R.  Every dependency wait must already hold in ticket
    order -- the property that makes the kernel's order deadlock-free."""
    import ctypes
    hostcheck.hostcheck_twopass_violations.restype = ctypes.c_longlong
    hostcheck.hostcheck_twopass_violations()
    rng = np.random.default_rng(5000 + g + nvol + prec)
    dt = np.complex128 if prec == 0 else np.complex64
    x = field(rng, (nvol,) + shape, dist="normal", dtype=dt)
    got = run(hostcheck, x, shape, prec, sign, 300 + g, 1)
    assert hostcheck.hostcheck_twopass_violations() == 0
    x64 = x.astype(np.complex128)
    want = oracle.fft3d(x64) if sign < 0 else oracle.ifft3d(x64)
    err = oracle.rel_error_per_volume(got, want).max()
    assert err < (C128_TOL if prec == 0 else C64_TOL), err


REGS = [((36, 36, 36), 500, 3, 7), ((36, 36, 36), 500, 2, 11), ((36, 36, 36), 500, 4, 3),
        ((6, 9, 5), 500, 3, 41), ((36, 36, 36), 540, 3, 6), ((36, 36, 36), 540, 2, 3),
        ((6, 9, 5), 540, 3, 41)]
# complex float at row pitch 38 (bulk rows): (shape, alg base, G, batch)
REGS_F = [((36, 36, 36), 540, 3, 7), ((36, 36, 36), 540, 2, 5), ((36, 36, 36), 540, 4, 3)]


@pytest.mark.parametrize("shape,base,g,nvol", REGS_F, ids=[f"{t[0]}-g{t[2]}-b{t[3]}" for t in REGS_F])
@pytest.mark.parametrize("sign", [-1, +1])
def test_twopass_lean_control_complex64(hostcheck, shape, base, g, nvol, sign):
    """The lean-control TWOPASS kernel in complex float with its explicit row
    pitch of 38 points (16-byte aligned rows for the bulk copies)."""
    import ctypes
    hostcheck.hostcheck_twopass_violations.restype = ctypes.c_longlong
    hostcheck.hostcheck_twopass_violations()
    rng = np.random.default_rng(7100 + g + nvol)
    x = field(rng, (nvol,) + shape, dist="normal", dtype=np.complex64)
    got = run(hostcheck, x, shape, 1, sign, base + g, 1)
    assert hostcheck.hostcheck_twopass_violations() == 0
    x64 = x.astype(np.complex128)
    want = oracle.fft3d(x64) if sign < 0 else oracle.ifft3d(x64)
    assert oracle.rel_error_per_volume(got, want).max() < C64_TOL


@pytest.mark.parametrize("shape,base,g,nvol", REGS,
                         ids=[f"{t[0]}-a{t[1]}-g{t[2]}-b{t[3]}" for t in REGS])
@pytest.mark.parametrize("sign", [-1, +1])
def test_twopass_lean_control_variants(hostcheck, shape, base, g, nvol, sign):
    """The lean-control TWOPASS variants: y pass stored straight into the
    scratch slot and x pass loaded straight from it (alg = 500 + G), or x pass
    from bulk-gathered rows (540 + G); the line maps of pass_y_store_l2 /
    pass_x_load_l2, in ticket order with the dependency check."""
    import ctypes
    hostcheck.hostcheck_twopass_violations.restype = ctypes.c_longlong
    hostcheck.hostcheck_twopass_violations()
    rng = np.random.default_rng(7000 + g + nvol + sum(shape))
    x = field(rng, (nvol,) + shape, dist="normal")
    got = run(hostcheck, x, shape, 0, sign, base + g, 1)
    assert hostcheck.hostcheck_twopass_violations() == 0
    want = oracle.fft3d(x) if sign < 0 else oracle.ifft3d(x)
    assert oracle.rel_error_per_volume(got, want).max() < C128_TOL


STAGED = [(64, 0, 2), (64, 1, 2), (45, 0, 3)]  # (N, precision, batch)


@pytest.mark.parametrize("n,prec,nvol", STAGED, ids=[f"{t[0]}-c{128 if t[1] == 0 else 64}" for t in STAGED])
@pytest.mark.parametrize("sign", [-1, +1])
def test_twopass_staged_lines(hostcheck, n, prec, nvol, sign):
    """The staged TWOPASS kernel (alg = 701): 64-point lines as 8 x 8
    Cooley-Tukey and 45-point lines as 5 x 9 Good-Thomas stages through shared
    memory at the kernel's row pitch, rows left in slot order by the z pass."""
    import ctypes
    hostcheck.hostcheck_twopass_violations.restype = ctypes.c_longlong
    hostcheck.hostcheck_twopass_violations()
    shape = (n, n, n)
    rng = np.random.default_rng(9000 + n + prec + nvol)
    dt = np.complex128 if prec == 0 else np.complex64
    x = field(rng, (nvol,) + shape, dist="normal", dtype=dt)
    got = run(hostcheck, x, shape, prec, sign, 701, 1)
    assert hostcheck.hostcheck_twopass_violations() == 0
    x64 = x.astype(np.complex128)
    want = oracle.fft3d(x64) if sign < 0 else oracle.ifft3d(x64)
    assert oracle.rel_error_per_volume(got, want).max() < (C128_TOL if prec == 0 else C64_TOL)


LANES = [(2, 2, 11), (2, 4, 5), (1, 4, 3), (3, 4, 7)]  # (G, P, batch)


@pytest.mark.parametrize("g,p,nvol", LANES, ids=[f"g{t[0]}-lanes{t[1]}-b{t[2]}" for t in LANES])
@pytest.mark.parametrize("sign", [-1, +1])
def test_twopass_lane_split(hostcheck, g, p, nvol, sign):
    """The lane-split TWOPASS kernel for 36^3 complex double (alg = 1024 + P,
    vpc = G): 36 = 2 x 18 Cooley-Tukey with the lane twiddle, or 4 x 9
    Good-Thomas, at the kernel's row pitch of 37 and its index maps, in ticket
    order with the dependency check."""
    import ctypes
    hostcheck.hostcheck_twopass_violations.restype = ctypes.c_longlong
    hostcheck.hostcheck_twopass_violations()
    shape = (36, 36, 36)
    rng = np.random.default_rng(8000 + g + 10 * p + nvol)
    x = field(rng, (nvol,) + shape, dist="normal")
    got = run(hostcheck, x, shape, 0, sign, 1024 + p, g)
    assert hostcheck.hostcheck_twopass_violations() == 0
    want = oracle.fft3d(x) if sign < 0 else oracle.ifft3d(x)
    assert oracle.rel_error_per_volume(got, want).max() < C128_TOL


GOLD = [p for p in sorted(glob.glob(os.path.join(GOLDEN, "vol_*.npz")))]


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p) for p in GOLD])
def test_pass_code_vs_reference_golden(hostcheck, path):
    d = np.load(path)
    shape = tuple(int(s) for s in d["shape"])
    match = [g for g in GEOMS if g[0] == shape]
    # volumes beyond one CTA's shared memory (36^3, 30^3 complex double): TWOPASS items
    match += [(shape, 300 + t[2], 1) for t in TWOPASS if t[0] == shape and t[1] == 0][:1]
    assert match, f"{shape}: a reference golden geometry without a kernel emulation"
    for _, alg, vpc in match:
        got = run(hostcheck, d["x"], shape, 0, -1, alg, vpc)
        assert oracle.rel_error(got, d["fwd"]) < C128_TOL
        inv = run(hostcheck, d["x"], shape, 0, +1, alg, vpc)
        assert oracle.rel_error(inv, d["inv"]) < C128_TOL


def chain_reference(x, c, steps, kind):
    """The chain with the oracle's transform: unitary (x <- FFT(x)/sqrt(V)) or map
    (z = FFT(x) + c; x <- z / (1 + |z|)), docs/GRADER.md of the reference."""
    s = x.astype(np.complex128)
    v = int(np.prod(x.shape[1:]))
    for _ in range(steps):
        z = oracle.fft3d(s)
        if kind == 1:
            s = z / np.sqrt(v)
        else:
            w = z + c
            s = w / (1.0 + np.abs(w))
    return s


@pytest.mark.parametrize("L,prec", [(6, 0), (8, 0), (17, 0), (8, 1)])
@pytest.mark.parametrize("kind", [1, 2])
def test_chain_kernel_pass_code(hostcheck, L, prec, kind):
    """The chain kernel's on-chip step loop and fused epilogues, 3 steps."""
    import ctypes
    hostcheck.hostcheck_chain.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p] * 3 + \
        [ctypes.c_longlong] * 2
    rng = np.random.default_rng(50 + L + kind)
    dt = np.complex128 if prec == 0 else np.complex64
    x = field(rng, (3, L, L, L), dtype=dt)
    c = field(rng, (3, L, L, L), dtype=dt)
    out = np.empty_like(x)
    assert hostcheck.hostcheck_chain(L, prec, kind, x.ctypes.data, out.ctypes.data,
                                     c.ctypes.data, 3, 3) == 0
    want = chain_reference(x, c.astype(np.complex128), 3, kind)
    err = oracle.rel_error_per_volume(out, want).max()
    assert err < (1e-13 if prec == 0 else 5e-6), err
