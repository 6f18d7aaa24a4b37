"""Generate the golden vectors that pin the oracle and the CUDA path to the reference.

Run with the reference's Python oracle (python/fft3d.py and python/slow_dft.py of
wdetmold/opt-fft) in a checkout at PATH:

    python tests/golden/make_golden.py --ref-root PATH [--missing]

(--ref-root defaults to $REF_ROOT; one of them is required.  --missing writes
only the fixtures that are not there yet.)

It imports the reference's own code, transforms seeded inputs with it, and writes
small .npz fixtures next to this script.  The fixtures are committed; the tests
read them and never need the reference checkout.

Each fixture holds:
    x        input, shape (B, n0, n1, n2)
    fwd      fft3d.fftn(x)                        (python/fft3d.py:360-399, textbook route)
    inv      fft3d.ifftn(x)                       (python/fft3d.py:402-407)
    sep      slow_dft.dft3d_separable(x)          (python/slow_dft.py:93-106), small cases only
    shape, seed, dist                              provenance
and 1d.npz holds fft1d of every length 1..40 (python/fft3d.py:300-334).
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# (batch, shape, distribution, seed).  The target extents of the build (6, 8, 12,
# 16, 17, 24, 36 and the anisotropic 8x8x16 / 16x16x32) plus a spread of the
# reference's own test geometries (python/test_fft3d.py:25-36).
CASES = [
    (2, (8, 8, 8), "uniform", 101),
    (1, (17, 17, 17), "uniform", 102),
    (1, (36, 36, 36), "normal", 103),
    (1, (16, 16, 32), "normal", 104),
    (2, (8, 8, 16), "uniform", 105),
    (2, (6, 6, 6), "uniform", 106),
    (1, (12, 12, 12), "uniform", 107),
    (1, (16, 16, 16), "uniform", 108),
    (1, (24, 24, 24), "uniform", 109),
    (3, (4, 4, 4), "normal", 110),
    (2, (2, 3, 5), "normal", 111),
    (2, (7, 11, 13), "normal", 112),
    (1, (1, 8, 8), "normal", 113),
    (1, (8, 1, 8), "normal", 114),
    (1, (8, 8, 1), "normal", 115),
    (1, (1, 1, 1), "normal", 116),
    (2, (9, 9, 9), "normal", 117),
    (1, (5, 8, 12), "normal", 118),
    (1, (13, 5, 8), "normal", 119),
    (1, (17, 2, 2), "normal", 120),
    (1, (3, 3, 3), "normal", 121),
    (1, (32, 8, 4), "normal", 122),
    # the rest of python/test_fft3d.py:25-36
    (2, (2, 2, 2), "normal", 123),
    (1, (5, 5, 5), "normal", 124),
    (1, (7, 7, 7), "normal", 125),
    (1, (11, 11, 11), "normal", 126),
    (1, (49, 2, 2), "normal", 127),
    (1, (25, 4, 3), "normal", 128),
    (1, (27, 2, 2), "normal", 129),
    (1, (19, 3, 2), "normal", 130),
    (1, (23, 2, 2), "normal", 131),
    (1, (47, 3, 2), "normal", 132),
    (1, (83, 2, 1), "normal", 133),
    (1, (97, 2, 1), "normal", 134),
    (1, (1, 1, 16), "normal", 135),
    (1, (1, 7, 1), "normal", 136),
    (1, (3, 5, 7), "normal", 137),
    (1, (4, 6, 10), "normal", 138),
    (1, (16, 3, 5), "normal", 139),
    (1, (24, 18, 12), "normal", 140),
    (1, (30, 30, 30), "normal", 141),
    (1, (2, 2, 64), "normal", 142),
    (1, (64, 2, 2), "normal", 143),
    (1, (9, 25, 7), "normal", 144),
    (1, (20, 12, 6), "normal", 145),
    (1, (11, 4, 9), "normal", 146),
    (1, (10, 10, 10), "normal", 147),
    (1, (15, 15, 15), "normal", 148),
]


def field(rng, shape, dist):
    if dist == "uniform":
        return rng.uniform(-1.0, 1.0, shape) + 1j * rng.uniform(-1.0, 1.0, shape)
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=os.environ.get("REF_ROOT"))
    ap.add_argument("--missing", action="store_true", help="only write fixtures not present yet")
    a = ap.parse_args()
    if not a.ref_root:
        ap.error("--ref-root (or REF_ROOT) is required")
    sys.path.insert(0, os.path.join(a.ref_root, "python"))
    import fft3d  # noqa: E402  (the reference's textbook FFT)
    import slow_dft  # noqa: E402  (the reference's definitional DFT)

    for batch, shape, dist, seed in CASES:
        name = "vol_%dx%dx%d_b%d.npz" % (shape + (batch,))
        if a.missing and os.path.exists(os.path.join(HERE, name)):
            continue
        rng = np.random.default_rng(seed)
        x = field(rng, (batch,) + shape, dist).astype(np.complex128)
        t0 = time.perf_counter()
        fwd = fft3d.fftn(x)
        inv = fft3d.ifftn(x)
        extra = {}
        if int(np.prod(shape)) <= 13 * 13 * 13:
            extra["sep"] = slow_dft.dft3d_separable(x)
        np.savez_compressed(os.path.join(HERE, name), x=x, fwd=fwd, inv=inv,
                            shape=np.array(shape), seed=seed, dist=dist, **extra)
        print(f"{name}: {time.perf_counter() - t0:.2f}s")

    if a.missing:
        print("done")
        return
    # complex64 contract: computed in double, returned as complex64 (fft3d.py:368-371)
    rng = np.random.default_rng(201)
    x32 = field(rng, (2, 8, 8, 8), "uniform").astype(np.complex64)
    np.savez_compressed(os.path.join(HERE, "c64_8x8x8_b2.npz"), x=x32, fwd=fft3d.fftn(x32),
                        shape=np.array((8, 8, 8)), seed=201, dist="uniform")

    # every 1D length 1..40 (python/test_fft3d.py:49-59)
    lines = {}
    for n in range(1, 41):
        x = slow_dft.random_field((n,), seed=n)
        lines[f"x{n}"] = x
        lines[f"y{n}"] = fft3d.fft1d(x)
        lines[f"d{n}"] = slow_dft.dft1d_loops(x)
    np.savez_compressed(os.path.join(HERE, "lines_1_40.npz"), **lines)

    # primitive roots used by Rader (fft3d.py:119-133)
    primes = [p for p in range(2, 200) if fft3d.is_prime(p)]
    np.savez_compressed(os.path.join(HERE, "primitive_roots.npz"), p=np.array(primes),
                        g=np.array([fft3d.primitive_root(p) for p in primes]))
    print("done")


if __name__ == "__main__":
    main()
