"""Parity of the CUDA path with the oracle, through the C ABI (needs a B200).

Every compiled kernel variant of every geometry, both directions and both
precisions, on seeded inputs, against the C oracle (a restatement of the
reference's python/fft3d.py pinned by tests/test_oracle.py) and against the
reference's own golden vectors.  Bars: complex128 within 1e-13 relative L2 per
volume (the reference gate is 1e-12, bench/geom/check.py:13); complex64 in FP32
within 1e-6 per volume of the FP64 oracle.  Every variant's worst error is
recorded (conftest.record_error).  At the full benchmark sizes the
checks are size-independent properties: forward->inverse round trip, Parseval,
linearity, bit-exact repeatability, input left untouched, and a seeded subset of
volumes against the oracle.
"""
import ctypes
import glob
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN, field, record_error

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import fft3d_b200 as fb  # noqa: E402

C128_TOL = 1e-13
C64_TOL = 1e-6

GEOMS = [(6, 6, 6), (8, 8, 8), (12, 12, 12), (16, 16, 16), (17, 17, 17), (24, 24, 24),
         (8, 8, 16), (16, 16, 32), (36, 36, 36), (13, 13, 13), (23, 23, 23), (45, 45, 45),
         (64, 64, 64),
         # the other extents of the reference's tests (python/test_fft3d.py:25-36)
         (1, 1, 1), (3, 3, 3), (4, 4, 4), (9, 9, 9), (10, 10, 10), (15, 15, 15), (2, 3, 5),
         (7, 11, 13), (5, 8, 12), (13, 5, 8), (17, 2, 2), (32, 8, 4), (1, 8, 8), (8, 1, 8),
         (8, 8, 1), (2, 2, 2), (5, 5, 5), (7, 7, 7), (11, 11, 11), (49, 2, 2), (25, 4, 3),
         (27, 2, 2), (19, 3, 2), (23, 2, 2), (47, 3, 2), (83, 2, 1), (97, 2, 1), (1, 1, 16),
         (1, 7, 1), (3, 5, 7), (4, 6, 10), (16, 3, 5), (24, 18, 12), (30, 30, 30), (2, 2, 64),
         (64, 2, 2), (9, 25, 7), (20, 12, 6), (11, 4, 9)]
TDT = {fb.C128: torch.complex128, fb.C64: torch.complex64}
NDT = {fb.C128: np.complex128, fb.C64: np.complex64}


def dev():
    return torch.device("cuda:0")


def to_dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).to(dev())


def run_plan(plan, x):
    xin = to_dev(x)
    out = torch.empty_like(xin)
    plan.execute(xin.data_ptr(), out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return out.cpu().numpy(), xin


def ref(x, direction):
    x64 = x.astype(np.complex128)
    return oracle.fft3d(x64) if direction == fb.FORWARD else oracle.ifft3d(x64)


def batch_for(shape, prec):
    v = int(np.prod(shape))
    return max(3, min(40, 600000 // v))


CASES = [(g, p, d) for g in GEOMS for p in (fb.C128, fb.C64) for d in (fb.FORWARD, fb.BACKWARD)
         if fb.supports(g, p)]


@pytest.mark.parametrize("shape,prec,direction", CASES,
                         ids=[f"{c[0]}-{'c128' if c[1] == 0 else 'c64'}-{'fwd' if c[2] < 0 else 'inv'}"
                              for c in CASES])
def test_every_variant_matches_oracle(shape, prec, direction):
    rng = np.random.default_rng(abs(hash((shape, prec, direction))) % 2**31)
    tol = C128_TOL if prec == fb.C128 else C64_TOL
    for v in fb.variants(shape, prec, direction):
        # the two-term split-BF16 tensor-core variant keeps 16 bits (bound of test_gpu_tensor.py)
        tol = 3e-5 if "split2" in v else (C128_TOL if prec == fb.C128 else C64_TOL)
        b = batch_for(shape, prec)
        if v.startswith("stream"):
            # persistent kernels: every CTA walks >= 2 groups and, for groups of
            # several volumes, the last group is partial (for complex64 17^3 and
            # 13^3 a group that is not 16-byte aligned: the threads' copy paths)
            vpc = int(v.split(" vpc")[1].split()[0])
            b = 2 * 148 * vpc + (vpc + 1) // 2
        elif v.startswith("volume"):
            # several CTAs and a partial group
            vpc = int(v.split(" vpc")[1].split()[0])
            b = max(b, 2 * vpc + (vpc + 1) // 2)
        elif v.startswith("twopass"):
            # beyond the scratch ring (about 40 volumes at a full grid): slots are reused
            b = 100
        x = field(rng, (b,) + shape, dtype=NDT[prec])
        want = ref(x, direction)
        plan = fb.Plan(shape, b, direction, prec, variant=v)
        got, xin = run_plan(plan, x)
        err = oracle.rel_error_per_volume(got, want)
        record_error(f"{shape} {'c128' if prec == fb.C128 else 'c64'} "
                     f"{'fwd' if direction == fb.FORWARD else 'inv'} x{b}", v, err.max(), tol)
        assert err.max() < tol, f"{v}: worst volume rel err {err.max():.3e}"
        assert np.array_equal(xin.cpu().numpy(), x), f"{v} modified its input"


GOLD = sorted(glob.glob(os.path.join(GOLDEN, "vol_*.npz")))


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p) for p in GOLD])
def test_reference_golden_vectors(path):
    d = np.load(path)
    shape = tuple(int(s) for s in d["shape"])
    assert fb.supports(shape, fb.C128), f"{shape}: a reference test geometry without a kernel"
    x = d["x"]
    for direction, key in ((fb.FORWARD, "fwd"), (fb.BACKWARD, "inv")):
        plan = fb.Plan(shape, x.shape[0], direction, fb.C128)
        got, _ = run_plan(plan, x)
        assert oracle.rel_error(got, d[key]) < C128_TOL


def test_complex64_golden():
    d = np.load(os.path.join(GOLDEN, "c64_8x8x8_b2.npz"))
    plan = fb.Plan((8, 8, 8), 2, fb.FORWARD, fb.C64)
    got, _ = run_plan(plan, d["x"])
    assert got.dtype == np.complex64
    assert oracle.rel_error(got.astype(np.complex128), d["fwd"].astype(np.complex128)) < C64_TOL


# ---------------------------------------------------------------- reference contracts

def test_reference_host_abi_drop_in():
    """fft3d_create / fft3d_execute / fft3d_destroy on pageable host buffers, as
    bench/geom/driver.c calls them (:136, :208, :231, :290)."""
    lib = fb.lib()
    for L, B in ((8, 37), (17, 5), (12, 9)):
        rng = np.random.default_rng(L * 100 + B)
        x = field(rng, (B, L, L, L))
        keep = x.copy()
        out = np.zeros_like(x)
        plan = lib.fft3d_create(L, B)
        assert plan, fb.lib().fft3d_b200_last_status()
        lib.fft3d_execute(plan, x.ctypes.data, out.ctypes.data)
        assert oracle.rel_error_per_volume(out, oracle.fft3d(x)).max() < C128_TOL
        assert np.array_equal(x, keep)
        again = np.zeros_like(x)
        lib.fft3d_execute(plan, x.ctypes.data, again.ctypes.data)
        assert np.array_equal(out, again), "execute is not bit-repeatable"
        # anti-memoization (bench/geom/driver.c:225-239)
        x[0, 0, 0, 0] += 1.0 - 2.0j
        poked = np.zeros_like(x)
        lib.fft3d_execute(plan, x.ctypes.data, poked.ctypes.data)
        assert not np.array_equal(poked, out)
        lib.fft3d_destroy(plan)


def test_reference_device_abi_drop_in():
    """fft3d_gpu_* on cudaMalloc'd buffers with legacy-stream ordering, as
    bench/gpu/driver.cu calls them (:150, :161, :194, :240, :306)."""
    lib = fb.lib()
    L, B = 17, 11
    rng = np.random.default_rng(7)
    x = field(rng, (B, L, L, L))
    din = to_dev(x)
    dout = torch.zeros_like(din)
    plan = lib.fft3d_gpu_create(L, B)
    assert plan
    lib.fft3d_gpu_execute(plan, din.data_ptr(), dout.data_ptr())
    torch.cuda.synchronize()
    assert oracle.rel_error_per_volume(dout.cpu().numpy(), oracle.fft3d(x)).max() < C128_TOL
    lib.fft3d_gpu_destroy(plan)
    assert not lib.fft3d_gpu_create(14, 1)  # unsupported -> NULL (bench/gpu/fft3d_gpu_api.h:46-50)


def test_host_chain_round_trip_and_pinned_path():
    shape, B = (17, 17, 17), 9
    rng = np.random.default_rng(3)
    x = field(rng, (B,) + shape)
    f = fb.Plan(shape, B, fb.FORWARD)
    i = fb.Plan(shape, B, fb.BACKWARD)
    back = fb.execute_host_chain([f, i], x)
    assert oracle.rel_error_per_volume(back, x).max() < C128_TOL
    fwd = fb.execute_host_chain([f], x)
    assert oracle.rel_error_per_volume(fwd, oracle.fft3d(x)).max() < C128_TOL
    # page-locked buffers take the direct-DMA path
    pin_in = torch.from_numpy(x).pin_memory()
    pin_out = torch.empty_like(pin_in).pin_memory()
    st = fb.lib().fft3d_b200_execute_host(f.handle, pin_in.data_ptr(), pin_out.data_ptr())
    assert st == 0
    assert np.array_equal(pin_out.numpy(), fwd)


def test_pinned_host_chain_with_scratch_kernels():
    """Page-locked buffers, several chunks: a TWOPASS plan's chunks alternate
    over two streams with a scratch workspace each.  Same bits as the device
    path, the input left untouched, repeated calls exact."""
    shape, B = (36, 36, 36), 20
    rng = np.random.default_rng(36)
    x = field(rng, (B,) + shape, dist="normal")
    f = fb.Plan(shape, B, fb.FORWARD)
    i = fb.Plan(shape, B, fb.BACKWARD)
    pin_in = torch.from_numpy(x).pin_memory()
    pin_out = torch.empty_like(pin_in).pin_memory()
    arr = (ctypes.c_void_p * 2)(f.handle.value, i.handle.value)
    for _ in range(2):  # repeated calls reuse the plan's streams and events
        assert fb.lib().fft3d_b200_execute_host_chain(arr, 2, pin_in.data_ptr(), pin_out.data_ptr()) == 0
        assert oracle.rel_error_per_volume(pin_out.numpy(), x).max() < C128_TOL
    assert fb.lib().fft3d_b200_execute_host_chain(arr, 1, pin_in.data_ptr(), pin_out.data_ptr()) == 0
    dev_out, _ = run_plan(f, x)
    assert np.array_equal(pin_out.numpy(), dev_out)
    assert np.array_equal(pin_in.numpy(), x)


@pytest.mark.parametrize("shape,prec,B", [((17, 17, 17), fb.C128, 61), ((13, 13, 13), fb.C64, 301)])
def test_pinned_host_chain_unaligned_chunks(monkeypatch, shape, prec, B):
    """Page-locked buffers cut into 1 MB chunks of whole volumes whose
    boundaries are not 64 KB multiples: the copies run between 64 KB
    boundaries (an upload may carry the head of the next chunk, a download
    stops short of the current chunk's end), so every byte still arrives
    once and after its transform.  One, two and three plans (the result
    alternates between the two device buffers) give the device path's bits."""
    monkeypatch.setenv("FFT3D_B200_HOST_CHUNK_MB", "1")  # read when a plan first stages
    rng = np.random.default_rng(B)
    x = field(rng, (B,) + shape, dtype=NDT[prec])
    f = fb.Plan(shape, B, fb.FORWARD, prec)
    i = fb.Plan(shape, B, fb.BACKWARD, prec)
    pin_in = torch.from_numpy(x).pin_memory()
    pin_out = torch.empty_like(pin_in).pin_memory()
    arr = (ctypes.c_void_p * 3)(f.handle.value, i.handle.value, f.handle.value)
    fwd, _ = run_plan(f, x)
    back, _ = run_plan(i, fwd)
    fwd2, _ = run_plan(f, back)
    for n, want in ((1, fwd), (2, back), (3, fwd2)):
        pin_out.zero_()
        assert fb.lib().fft3d_b200_execute_host_chain(arr, n, pin_in.data_ptr(), pin_out.data_ptr()) == 0
        assert np.array_equal(pin_out.numpy(), want), n
    assert np.array_equal(pin_in.numpy(), x)


# ---------------------------------------------------------------- edges and errors

def test_edges_and_errors():
    shape = (8, 8, 8)
    # batch of one, and a batch that leaves a partial CTA
    for b in (1, 13):
        rng = np.random.default_rng(b)
        x = field(rng, (b,) + shape)
        got, _ = run_plan(fb.Plan(shape, b), x)
        assert oracle.rel_error_per_volume(got, oracle.fft3d(x)).max() < C128_TOL
    # empty batch is a no-op
    p0 = fb.Plan(shape, 0)
    p0.execute(0, 0)
    # misaligned and overlapping buffers are refused, not computed
    p = fb.Plan(shape, 4)
    buf = torch.zeros(2 * 4 * 512 + 8, dtype=torch.complex128, device=dev())
    with pytest.raises(fb.Fft3dError) as e:
        p.execute(buf.data_ptr() + 8, buf.data_ptr() + 4 * 512 * 16 + 16)
    assert e.value.status == fb.ERR_ALIGN
    with pytest.raises(fb.Fft3dError) as e:
        p.execute(buf.data_ptr(), buf.data_ptr() + 16)
    assert e.value.status == fb.ERR_OVERLAP
    with pytest.raises(fb.Fft3dError) as e:
        p.execute(0, buf.data_ptr())
    assert e.value.status == fb.ERR_INVALID


def test_named_variant_and_tuner():
    shape = (17, 17, 17)
    names = fb.variants(shape)
    assert len(names) >= 2
    p = fb.Plan(shape, 64)
    assert p.describe() in names
    with pytest.raises(fb.Fft3dError):
        fb.Plan(shape, 64, variant="no such kernel")


# ---------------------------------------------------------------- full benchmark sizes

def _full_size_checks(shape, batch, dist, seed, subset=24):
    rng = np.random.default_rng(seed)
    x = field(rng, (batch,) + shape, dist=dist)
    f = fb.Plan(shape, batch, fb.FORWARD)
    i = fb.Plan(shape, batch, fb.BACKWARD)
    xin = to_dev(x)
    X = torch.empty_like(xin)
    back = torch.empty_like(xin)
    s = torch.cuda.current_stream().cuda_stream
    f.execute(xin.data_ptr(), X.data_ptr(), s)
    i.execute(X.data_ptr(), back.data_ptr(), s)
    X2 = torch.empty_like(xin)
    f.execute(xin.data_ptr(), X2.data_ptr(), s)
    torch.cuda.synchronize()
    assert torch.equal(X, X2), "forward not bit-repeatable"
    assert torch.equal(xin, to_dev(x)), "input modified"
    xb = back.cpu().numpy()
    rt = oracle.rel_error_per_volume(xb, x)
    assert rt.max() < C128_TOL, f"round trip {rt.max():.3e}"
    Xn = X.cpu().numpy()
    v = int(np.prod(shape))
    lhs = np.sum(np.abs(Xn.reshape(batch, -1)) ** 2, axis=1)
    rhs = v * np.sum(np.abs(x.reshape(batch, -1)) ** 2, axis=1)
    assert np.max(np.abs(lhs - rhs) / rhs) < C128_TOL
    idx = np.sort(rng.choice(batch, size=min(subset, batch), replace=False))
    err = oracle.rel_error_per_volume(Xn[idx], oracle.fft3d(x[idx]))
    assert err.max() < C128_TOL, f"subset {err.max():.3e}"
    return rt.max(), err.max()


def test_full_size_8cubed_4096():
    _full_size_checks((8, 8, 8), 4096, "uniform", 11, subset=4096)


def test_full_size_17cubed_2048_round_trip():
    _full_size_checks((17, 17, 17), 2048, "uniform", 12, subset=64)


def test_full_size_16x16x32_1024():
    _full_size_checks((16, 16, 32), 1024, "normal", 13, subset=32)


def test_full_size_36cubed_256():
    if not fb.supports((36, 36, 36), fb.C128):
        pytest.skip("36^3 not compiled")
    _full_size_checks((36, 36, 36), 256, "normal", 14, subset=8)


def test_linearity_full_batch_c64():
    shape, b = (16, 16, 16), 1024
    rng = np.random.default_rng(21)
    x = field(rng, (b,) + shape, dtype=np.complex64)
    y = field(rng, (b,) + shape, dtype=np.complex64)
    p = fb.Plan(shape, b, fb.FORWARD, fb.C64)
    fx, _ = run_plan(p, x)
    fy, _ = run_plan(p, y)
    fxy, _ = run_plan(p, (x + y).astype(np.complex64))
    assert oracle.rel_error(fxy.astype(np.complex128), (fx + fy).astype(np.complex128)) < 1e-6


@pytest.mark.parametrize("shape,batch", [((8, 8, 8), (1 << 22) + 3), ((36, 36, 36), 6000)])
def test_large_batches_64_bit_offsets(shape, batch):
    """Maximum sizes: 2^22 + 3 volumes of 8^3 put element offsets past 2^31
    (34 GB a buffer, about 100 GB on the device in all); 6000 volumes of 36^3
    put the TWOPASS kernel's byte offsets past 2^32.  The first, a middle and
    the last volumes against the oracle, and the forward -> inverse round trip
    of every volume on the device."""
    vol = int(np.prod(shape))
    assert batch * vol * 16 > (1 << 32)
    g = torch.Generator(device="cuda").manual_seed(77)
    x = torch.empty((batch,) + shape, dtype=torch.complex128, device="cuda")
    x.real.uniform_(-1.0, 1.0, generator=g)
    x.imag.uniform_(-1.0, 1.0, generator=g)
    y = torch.empty_like(x)
    f = fb.Plan(shape, batch, fb.FORWARD, fb.C128)
    f.execute(x.data_ptr(), y.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    f.check()
    for k in (0, batch // 2 + 1, batch - 1):
        xs = x[k:k + 1].cpu().numpy()
        assert oracle.rel_error(y[k:k + 1].cpu().numpy(), oracle.fft3d(xs)) < C128_TOL, k
    f.close()
    back = torch.empty_like(x)
    i = fb.Plan(shape, batch, fb.BACKWARD, fb.C128)
    i.execute(y.data_ptr(), back.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    i.check()
    i.close()
    del y
    # per-volume relative L2 of the round trip, every volume, in chunks
    worst = 0.0
    step = max(1, (1 << 28) // (vol * 16))
    for k0 in range(0, batch, step):
        xb = x[k0:k0 + step].reshape(-1, vol)
        d = (back[k0:k0 + step].reshape(-1, vol) - xb).abs().pow(2).sum(1).sqrt()
        n = xb.abs().pow(2).sum(1).sqrt()
        worst = max(worst, float((d / n).max()))
    assert worst < C128_TOL, worst
