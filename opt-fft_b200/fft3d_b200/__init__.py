"""Python binding of libfft3d_b200.so, the B200 batched 3D complex FFT.

A thin ctypes layer over the C ABI (include/fft3d_b200.h, fft3d_api.h,
fft3d_gpu_api.h).  The arithmetic is the CUDA library's; nothing here computes a
transform.  If the shared library is missing the import fails loudly -- there is
no CPU fallback.

    import fft3d_b200 as fb
    plan = fb.Plan((17, 17, 17), batch=2048, direction=fb.FORWARD, precision=fb.C128)
    plan.execute(d_in_ptr, d_out_ptr, stream_ptr)     # device pointers (ints)
    out = plan.execute_host(x)                        # numpy in, numpy out

Device buffers are plain integers (e.g. ``torch_tensor.data_ptr()``), so this
module needs neither torch nor numpy to import.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("FFT3D_B200_LIB",
                          os.path.join(os.path.dirname(_HERE), "libfft3d_b200.so"))

OK = 0
ERR_INVALID = -1
ERR_UNSUPPORTED = -2
ERR_ALIGN = -3
ERR_CUDA = -4
ERR_NOMEM = -5
ERR_TIMEOUT = -6
ERR_BUDGET = -7
ERR_OVERLAP = -8
ERR_BUSY = -9
ERR_PEER = -10

FORWARD = -1
BACKWARD = +1
C128 = 0
C64 = 1
FLAG_NO_TUNE = 0x1
FLAG_NO_GRAPH = 0x2
BATCH_PERSISTENT = 0x4
BATCH_SEGMENTS = 0x8

ELEMENT_BYTES = {C128: 16, C64: 8}


class Fft3dError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        msg = _lib.fft3d_b200_status_string(status).decode() if _lib else str(status)
        super().__init__(f"{what}: {msg} ({status})" if what else f"{msg} ({status})")


class Desc(ctypes.Structure):
    _fields_ = [("n0", ctypes.c_int), ("n1", ctypes.c_int), ("n2", ctypes.c_int),
                ("batch", ctypes.c_longlong), ("direction", ctypes.c_int),
                ("precision", ctypes.c_int), ("flags", ctypes.c_uint), ("device", ctypes.c_int)]


class Segment(ctypes.Structure):
    _fields_ = [("n0", ctypes.c_int), ("n1", ctypes.c_int), ("n2", ctypes.c_int),
                ("direction", ctypes.c_int), ("precision", ctypes.c_int),
                ("batch", ctypes.c_longlong), ("in_", ctypes.c_void_p), ("out", ctypes.c_void_p)]


def segment_dtype():
    """numpy record layout of Segment (for streams of many requests)."""
    import numpy as np
    return np.dtype({"names": ["n0", "n1", "n2", "direction", "precision", "batch", "in_", "out"],
                     "formats": ["i4", "i4", "i4", "i4", "i4", "i8", "u8", "u8"],
                     "offsets": [0, 4, 8, 12, 16, 24, 32, 40], "itemsize": 48})


class ServerStats(ctypes.Structure):
    _fields_ = [("requests", ctypes.c_longlong), ("volumes", ctypes.c_longlong),
                ("launches", ctypes.c_longlong), ("mean_requests_per_launch", ctypes.c_double),
                ("peak_admitted_bytes", ctypes.c_longlong), ("p50_s", ctypes.c_double),
                ("p99_s", ctypes.c_double), ("mean_s", ctypes.c_double), ("max_s", ctypes.c_double),
                ("volumes_per_s", ctypes.c_double), ("span_s", ctypes.c_double)]


SERVE_PLAIN = 0x1
CHAIN_UNITARY = 1
CHAIN_MAP = 2

# Every symbol the headers in include/ declare, by header.
EXPORTS = {
    "fft3d_api.h": ["fft3d_name", "fft3d_description", "fft3d_supports", "fft3d_create",
                    "fft3d_execute", "fft3d_destroy"],
    "fft3d_gpu_api.h": ["fft3d_gpu_name", "fft3d_gpu_description", "fft3d_gpu_supports",
                        "fft3d_gpu_create", "fft3d_gpu_execute", "fft3d_gpu_destroy"],
    "fft3d_mgpu_api.h": ["fft3d_mgpu_name", "fft3d_mgpu_description", "fft3d_mgpu_supports",
                         "fft3d_mgpu_create", "fft3d_mgpu_create_ex", "fft3d_mgpu_upload",
                         "fft3d_mgpu_execute", "fft3d_mgpu_download", "fft3d_mgpu_destroy"],
    "fft3d_b200.h": ["fft3d_b200_supports", "fft3d_b200_plan_create", "fft3d_b200_plan_destroy",
                     "fft3d_b200_variants", "fft3d_b200_plan_create_variant",
                     "fft3d_b200_execute", "fft3d_b200_execute_host",
                     "fft3d_b200_execute_host_chain", "fft3d_b200_plan_describe",
                     "fft3d_b200_plan_check", "fft3d_b200_debug_stall_next_execute",
                     "fft3d_b200_plan_launches", "fft3d_b200_last_status",
                     "fft3d_b200_status_string", "fft3d_b200_wisdom_export",
                     "fft3d_b200_wisdom_import", "fft3d_b200_wisdom_forget",
                     "fft3d_b200_plan4d_supports", "fft3d_b200_plan4d_create",
                     "fft3d_b200_plan4d_execute", "fft3d_b200_plan4d_destroy",
                     "fft3d_b200_plan4d_describe",
                     "fft3d_b200_batch_create",
                     "fft3d_b200_batch_execute", "fft3d_b200_batch_destroy",
                     "fft3d_b200_batch_describe", "fft3d_b200_batch_execute_noalloc",
                     "fft3d_b200_noalloc_check",
                     "fft3d_b200_chain_create", "fft3d_b200_chain_run",
                     "fft3d_b200_chain_destroy",
                     "fft3d_b200_server_create", "fft3d_b200_server_submit",
                     "fft3d_b200_server_submit_many",
                     "fft3d_b200_server_poll", "fft3d_b200_server_drain",
                     "fft3d_b200_server_get_stats", "fft3d_b200_server_latencies",
                     "fft3d_b200_server_destroy"],
}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python opt-fft_b200/build.py` "
                          "(there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    vp, i, ll = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong
    sig = {
        "fft3d_name": ([], ctypes.c_char_p),
        "fft3d_description": ([], ctypes.c_char_p),
        "fft3d_supports": ([i], i),
        "fft3d_create": ([i, i], vp),
        "fft3d_execute": ([vp, vp, vp], None),
        "fft3d_destroy": ([vp], None),
        "fft3d_gpu_name": ([], ctypes.c_char_p),
        "fft3d_gpu_description": ([], ctypes.c_char_p),
        "fft3d_gpu_supports": ([i], i),
        "fft3d_gpu_create": ([i, i], vp),
        "fft3d_gpu_execute": ([vp, vp, vp], None),
        "fft3d_gpu_destroy": ([vp], None),
        "fft3d_mgpu_name": ([], ctypes.c_char_p),
        "fft3d_mgpu_description": ([], ctypes.c_char_p),
        "fft3d_mgpu_supports": ([i, i], i),
        "fft3d_mgpu_create": ([i, i, i, ctypes.POINTER(i)], vp),
        "fft3d_mgpu_create_ex": ([i, i, i, ctypes.POINTER(i), i], vp),
        "fft3d_mgpu_upload": ([vp, vp], None),
        "fft3d_mgpu_execute": ([vp], None),
        "fft3d_mgpu_download": ([vp, vp], None),
        "fft3d_mgpu_destroy": ([vp], None),
        "fft3d_b200_supports": ([i, i, i, i], i),
        "fft3d_b200_plan_create": ([ctypes.POINTER(Desc), ctypes.POINTER(vp)], i),
        "fft3d_b200_plan_destroy": ([vp], None),
        "fft3d_b200_variants": ([i, i, i, i, i, ctypes.POINTER(ctypes.c_char_p), i], i),
        "fft3d_b200_plan_create_variant": ([ctypes.POINTER(Desc), ctypes.c_char_p,
                                            ctypes.POINTER(vp)], i),
        "fft3d_b200_execute": ([vp, vp, vp, vp], i),
        "fft3d_b200_execute_host": ([vp, vp, vp], i),
        "fft3d_b200_execute_host_chain": ([ctypes.POINTER(vp), i, vp, vp], i),
        "fft3d_b200_plan_describe": ([vp], ctypes.c_char_p),
        "fft3d_b200_plan_check": ([vp], i),
        "fft3d_b200_debug_stall_next_execute": ([vp], i),
        "fft3d_b200_plan_launches": ([vp], i),
        "fft3d_b200_last_status": ([], i),
        "fft3d_b200_status_string": ([i], ctypes.c_char_p),
        "fft3d_b200_wisdom_export": ([ctypes.c_char_p], i),
        "fft3d_b200_wisdom_import": ([ctypes.c_char_p], i),
        "fft3d_b200_wisdom_forget": ([], None),
        "fft3d_b200_plan4d_supports": ([i, i, i, i, i], i),
        "fft3d_b200_plan4d_create": ([i, ctypes.POINTER(Desc), ctypes.POINTER(vp)], i),
        "fft3d_b200_plan4d_execute": ([vp, vp, vp, vp], i),
        "fft3d_b200_plan4d_destroy": ([vp], None),
        "fft3d_b200_plan4d_describe": ([vp], ctypes.c_char_p),
        "fft3d_b200_batch_create": ([ctypes.POINTER(Segment), i, ctypes.c_uint, i,
                                     ctypes.POINTER(vp)], i),
        "fft3d_b200_batch_execute": ([vp, vp], i),
        "fft3d_b200_batch_destroy": ([vp], None),
        "fft3d_b200_batch_describe": ([vp], ctypes.c_char_p),
        "fft3d_b200_batch_execute_noalloc": ([ctypes.POINTER(Segment), i, vp], i),
        "fft3d_b200_noalloc_check": ([vp], i),
        "fft3d_b200_chain_create": ([i, i, i, ll, i, i, vp, i, ctypes.POINTER(vp)], i),
        "fft3d_b200_chain_run": ([vp, vp, vp, ll, vp], i),
        "fft3d_b200_chain_destroy": ([vp], None),
        "fft3d_b200_server_create": ([ctypes.c_size_t, i, ctypes.c_uint, i, ctypes.POINTER(vp)], i),
        "fft3d_b200_server_submit": ([vp, ctypes.POINTER(Segment),
                                      ctypes.POINTER(ctypes.c_ulonglong)], i),
        "fft3d_b200_server_submit_many": ([vp, ctypes.POINTER(Segment),
                                           ctypes.POINTER(ctypes.c_double), i,
                                           ctypes.POINTER(ctypes.c_ulonglong)], i),
        "fft3d_b200_server_poll": ([vp, ctypes.POINTER(ctypes.c_ulonglong), i], i),
        "fft3d_b200_server_drain": ([vp, ctypes.c_double], i),
        "fft3d_b200_server_get_stats": ([vp, ctypes.POINTER(ServerStats)], i),
        "fft3d_b200_server_latencies": ([vp, ctypes.POINTER(ctypes.c_ulonglong),
                                         ctypes.POINTER(ctypes.c_double), ll], ll),
        "fft3d_b200_server_destroy": ([vp], None),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _ = ll
    return lib


_lib = _load()


def lib():
    """The loaded ctypes library."""
    return _lib


def supports(shape, precision=C128) -> bool:
    n0, n1, n2 = shape
    return bool(_lib.fft3d_b200_supports(n0, n1, n2, precision))


def variants(shape, precision=C128, direction=FORWARD):
    """Names of the compiled kernel variants the autotuner chooses among."""
    n0, n1, n2 = shape
    n = _lib.fft3d_b200_variants(n0, n1, n2, precision, direction, None, 0)
    arr = (ctypes.c_char_p * max(n, 1))()
    _lib.fft3d_b200_variants(n0, n1, n2, precision, direction, arr, n)
    return [arr[k].decode() for k in range(n)]


def wisdom_export(path) -> int:
    """Write the autotuner's choices to `path`; returns the entries written."""
    n = _lib.fft3d_b200_wisdom_export(os.fsencode(path))
    if n < 0:
        raise Fft3dError(n, "wisdom_export")
    return n


def wisdom_import(path) -> int:
    """Merge a wisdom file into this process's choices; returns the entries taken."""
    n = _lib.fft3d_b200_wisdom_import(os.fsencode(path))
    if n < 0:
        raise Fft3dError(n, "wisdom_import")
    return n


def wisdom_forget():
    """Forget every autotuner choice of this process."""
    _lib.fft3d_b200_wisdom_forget()


class Plan4D:
    """4D DFT over (t, x, y, z) of `batch` lattices of nt x n0 x n1 x n2 (device
    pointers): the tuned 3D plan over every time slice, then the t pass."""

    def __init__(self, nt: int, shape, batch: int, direction: int = FORWARD,
                 precision: int = C128, device: int = -1):
        n0, n1, n2 = shape
        self.nt, self.shape, self.batch = nt, tuple(shape), batch
        d = Desc(n0, n1, n2, batch, direction, precision, 0, device)
        h = ctypes.c_void_p()
        _check(_lib.fft3d_b200_plan4d_create(nt, ctypes.byref(d), ctypes.byref(h)), "plan4d_create")
        self._h = h

    def execute(self, d_in: int, d_out: int, stream: int = 0):
        _check(_lib.fft3d_b200_plan4d_execute(self._h, d_in, d_out, stream or None), "plan4d_execute")

    def describe(self) -> str:
        return _lib.fft3d_b200_plan4d_describe(self._h).decode()

    def close(self):
        if self._h:
            _lib.fft3d_b200_plan4d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MgpuPlan:
    """One batch of L^3 complex128 cubes split over several GPUs of this process
    (include/fft3d_mgpu_api.h): x-slabs in, the all-to-all fused into the first
    kernel as peer stores, x pass on y-slabs.  `devices` may repeat a device."""

    def __init__(self, L: int, batch: int, devices, inverse: bool = False):
        self.L, self.batch, self.devices = L, batch, list(devices)
        arr = (ctypes.c_int * len(self.devices))(*self.devices)
        self._h = _lib.fft3d_mgpu_create_ex(L, batch, len(self.devices), arr, 1 if inverse else 0)
        if not self._h:
            raise Fft3dError(ERR_UNSUPPORTED, f"mgpu create L={L} batch={batch} devices={self.devices}")

    def upload(self, x):
        import numpy as np
        x = np.ascontiguousarray(x, dtype=np.complex128)
        if x.shape != (self.batch, self.L, self.L, self.L):
            raise ValueError(f"expected {(self.batch, self.L, self.L, self.L)}, got {x.shape}")
        _lib.fft3d_mgpu_upload(self._h, x.ctypes.data)

    def execute(self):
        _lib.fft3d_mgpu_execute(self._h)

    def download(self):
        import numpy as np
        out = np.empty((self.batch, self.L, self.L, self.L), dtype=np.complex128)
        _lib.fft3d_mgpu_download(self._h, out.ctypes.data)
        return out

    def close(self):
        if self._h:
            _lib.fft3d_mgpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _check(status, what):
    if status != OK:
        raise Fft3dError(status, what)


class Plan:
    """A plan for `batch` volumes of `shape` = (n0, n1, n2)."""

    def __init__(self, shape, batch, direction=FORWARD, precision=C128, flags=0, device=-1,
                 variant=None):
        n0, n1, n2 = (int(s) for s in shape)
        self.shape = (n0, n1, n2)
        self.batch = int(batch)
        self.direction = direction
        self.precision = precision
        self.elem_bytes = ELEMENT_BYTES.get(precision, 16)
        self.nbytes = self.batch * n0 * n1 * n2 * self.elem_bytes
        d = Desc(n0, n1, n2, self.batch, direction, precision, flags, device)
        h = ctypes.c_void_p()
        if variant is None:
            _check(_lib.fft3d_b200_plan_create(ctypes.byref(d), ctypes.byref(h)), "plan_create")
        else:
            _check(_lib.fft3d_b200_plan_create_variant(ctypes.byref(d), variant.encode(),
                                                       ctypes.byref(h)), "plan_create_variant")
        self._h = h

    @property
    def handle(self):
        return self._h

    def describe(self) -> str:
        return _lib.fft3d_b200_plan_describe(self._h).decode()

    def check(self):
        """Synchronise and raise if a bounded device-side wait ran out."""
        _check(_lib.fft3d_b200_plan_check(self._h), "plan_check")

    def launches(self) -> int:
        return _lib.fft3d_b200_plan_launches(self._h)

    def execute(self, d_in: int, d_out: int, stream: int = 0):
        """Enqueue on `stream` (a cudaStream_t as int; 0 = legacy default stream)."""
        _check(_lib.fft3d_b200_execute(self._h, d_in, d_out, stream or None), "execute")

    def execute_host(self, x, out=None):
        """numpy in (complex128 for C128, complex64 for C64), numpy out."""
        import numpy as np
        dt = np.complex128 if self.precision == C128 else np.complex64
        x = np.ascontiguousarray(x, dtype=dt)
        if x.nbytes != self.nbytes:
            raise ValueError(f"expected {self.nbytes} bytes, got {x.nbytes}")
        if out is None:
            out = np.empty_like(x)
        _check(_lib.fft3d_b200_execute_host(self._h, x.ctypes.data, out.ctypes.data),
               "execute_host")
        return out

    def close(self):
        if getattr(self, "_h", None):
            _lib.fft3d_b200_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def execute_host_chain(plans, x, out=None):
    """Upload x once, run plans back to back on the device, download once."""
    import numpy as np
    x = np.ascontiguousarray(x)
    if out is None:
        out = np.empty_like(x)
    arr = (ctypes.c_void_p * len(plans))(*[p.handle.value for p in plans])
    _check(_lib.fft3d_b200_execute_host_chain(arr, len(plans), x.ctypes.data, out.ctypes.data),
           "execute_host_chain")
    return out


def _segments(segments):
    arr = (Segment * max(1, len(segments)))()
    for k, s in enumerate(segments):
        arr[k] = Segment(s["shape"][0], s["shape"][1], s["shape"][2],
                         s.get("direction", FORWARD), s.get("precision", C128),
                         int(s["batch"]), s["in"], s["out"])
    return arr


def batch_execute_noalloc(segments, stream: int = 0):
    """One persistent batch launch with no device allocation (static scratch);
    see fft3d_b200_batch_execute_noalloc in include/fft3d_b200.h for the limits."""
    _check(_lib.fft3d_b200_batch_execute_noalloc(_segments(segments), len(segments),
                                                 stream or None), "batch_execute_noalloc")


def noalloc_check(stream: int = 0):
    """Synchronise `stream` and raise if an allocation-free launch on it failed."""
    _check(_lib.fft3d_b200_noalloc_check(stream or None), "noalloc_check")


class Batch:
    """Segments of uneven geometry (device pointers) in one graph launch: the
    persistent descriptor-list kernel or one tuned plan per segment, whichever
    batch creation measures faster (flags BATCH_PERSISTENT / BATCH_SEGMENTS pin one)."""

    def __init__(self, segments, flags=0, device=-1):
        arr = _segments(segments)
        h = ctypes.c_void_p()
        _check(_lib.fft3d_b200_batch_create(arr, len(segments), flags, device, ctypes.byref(h)),
               "batch_create")
        self._h = h

    def execute(self, stream: int = 0):
        _check(_lib.fft3d_b200_batch_execute(self._h, stream or None), "batch_execute")

    def describe(self) -> str:
        return _lib.fft3d_b200_batch_describe(self._h).decode()

    def close(self):
        if getattr(self, "_h", None):
            _lib.fft3d_b200_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Chain:
    """m forward transforms with a pointwise step each (CHAIN_UNITARY or CHAIN_MAP),
    one launch per run; volumes stay in shared memory for the whole chain."""

    def __init__(self, shape, batch, kind, precision=C128, d_c=0, device=-1):
        n0, n1, n2 = shape
        h = ctypes.c_void_p()
        _check(_lib.fft3d_b200_chain_create(n0, n1, n2, int(batch), precision, kind, d_c or None,
                                            device, ctypes.byref(h)), "chain_create")
        self._h = h

    def run(self, d_x0: int, d_out: int, steps: int, stream: int = 0):
        _check(_lib.fft3d_b200_chain_run(self._h, d_x0, d_out, int(steps), stream or None),
               "chain_run")

    def close(self):
        if getattr(self, "_h", None):
            _lib.fft3d_b200_chain_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching request server (fft3d_b200_server_*).

    Requests are segment dicts (shape, batch, direction, precision, device in/out
    pointers).  They are admitted against `budget_bytes` of in+out HBM, coalesced
    into persistent batch launches on up to `max_inflight` streams, and finish
    asynchronously; `stats()` gives p50/p99 latency and throughput."""

    def __init__(self, budget_bytes, max_inflight=4, flags=0, device=-1):
        h = ctypes.c_void_p()
        _check(_lib.fft3d_b200_server_create(int(budget_bytes), max_inflight, flags, device,
                                             ctypes.byref(h)), "server_create")
        self._h = h

    def submit(self, seg) -> int:
        arr = _segments([seg])
        t = ctypes.c_ulonglong()
        _check(_lib.fft3d_b200_server_submit(self._h, arr, ctypes.byref(t)), "server_submit")
        return t.value

    def submit_many(self, segs, arrival_s=None):
        """Submit segs[k] at arrival_s[k] seconds from now (C load generator)."""
        arr = _segments(segs)
        times = None
        if arrival_s is not None:
            times = (ctypes.c_double * len(segs))(*[float(t) for t in arrival_s])
        tk = (ctypes.c_ulonglong * max(1, len(segs)))()
        _check(_lib.fft3d_b200_server_submit_many(self._h, arr, times, len(segs), tk),
               "server_submit_many")
        return [tk[k] for k in range(len(segs))]

    def submit_array(self, segs, arrival_s=None):
        """submit_many for a numpy array of segment_dtype() records (large
        streams); returns the tickets as a numpy array."""
        import numpy as np
        segs = np.ascontiguousarray(segs, dtype=segment_dtype())
        n = len(segs)
        times = None
        if arrival_s is not None:
            arrival_s = np.ascontiguousarray(arrival_s, dtype=np.float64)
            times = arrival_s.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        tk = np.zeros(max(1, n), dtype=np.uint64)
        _check(_lib.fft3d_b200_server_submit_many(
            self._h, segs.ctypes.data_as(ctypes.POINTER(Segment)), times, n,
            tk.ctypes.data_as(ctypes.POINTER(ctypes.c_ulonglong))), "server_submit_many")
        return tk[:n]

    def latencies(self):
        """(tickets, latency_s) of every finished request, in completion order."""
        import numpy as np
        n = self.stats()["requests"]
        tk = np.zeros(max(1, n), dtype=np.uint64)
        lat = np.zeros(max(1, n), dtype=np.float64)
        got = _lib.fft3d_b200_server_latencies(
            self._h, tk.ctypes.data_as(ctypes.POINTER(ctypes.c_ulonglong)),
            lat.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n)
        if got < 0:
            raise Fft3dError(int(got), "server_latencies")
        return tk[:got], lat[:got]

    def poll(self, max_n=4096):
        buf = (ctypes.c_ulonglong * max_n)()
        n = _lib.fft3d_b200_server_poll(self._h, buf, max_n)
        if n < 0:
            raise Fft3dError(n, "server_poll")
        return [buf[k] for k in range(n)]

    def drain(self, timeout_s=120.0):
        _check(_lib.fft3d_b200_server_drain(self._h, float(timeout_s)), "server_drain")

    def stats(self) -> dict:
        st = ServerStats()
        _check(_lib.fft3d_b200_server_get_stats(self._h, ctypes.byref(st)), "server_stats")
        return {name: getattr(st, name) for name, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            _lib.fft3d_b200_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
