"""ctypes binding of the sm_100a tracking library (``_csl.so``).

The library is built in-tree by ``gpustreamlines_b200/build.py`` (or
``__graft_entry__.build()``).  There is no CPU fallback: loading fails loudly
when the shared object is missing, and every entry point raises on a non-zero
status with the library's own error message.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_csl.so")

CSL_OK = 0
CSL_E_INVALID = -1
CSL_E_CUDA = -2
CSL_E_NOMEM = -3
CSL_E_STATE = -4
CSL_E_KERNEL = -5

MODEL_OPDT, MODEL_CSA, MODEL_PROB, MODEL_PTT = 0, 1, 2, 3


class CslParams(C.Structure):
    _fields_ = [
        ("model", C.c_int),
        ("dimx", C.c_int), ("dimy", C.c_int), ("dimz", C.c_int), ("dimt", C.c_int),
        ("nvertices", C.c_int), ("nedges", C.c_int), ("samplm_nr", C.c_int),
        ("sphere_symm", C.c_int), ("max_sline_len", C.c_int), ("seed_order", C.c_int),
        ("step_size", C.c_double), ("max_angle", C.c_double), ("tc_threshold", C.c_double),
        ("relative_peak_thresh", C.c_double), ("min_separation_angle", C.c_double),
        ("pmf_threshold", C.c_double), ("rng_seed", C.c_ulonglong),
        ("min_signal", C.c_double), ("delta_nr", C.c_int), ("boot_fit", C.c_int),
        ("odf_lut_res", C.c_int), ("step_frac", C.c_int),
        ("probe_step_size", C.c_double), ("probe_quality", C.c_double),
        ("max_curvature", C.c_double),
        ("tile_log2_x", C.c_int), ("tile_log2_y", C.c_int),
        ("tile_nx", C.c_int), ("tile_ny", C.c_int), ("tile_nz", C.c_int), ("prob_sampler", C.c_int),
    ]


_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


class CslInputs(C.Structure):
    _fields_ = [
        ("dataf", _fp), ("stop_map", _fp), ("vertices", _fp), ("edges", _ip),
        ("H", _fp), ("R", _fp), ("delta_b", _fp), ("delta_q", _fp),
        ("sampling_matrix", _fp), ("b0s_mask", _ip),
        ("ptt_odf_tiled", _fp), ("ptt_lut", _fp),
    ]


_lib = None

# every symbol declared in include/gpustreamlines_b200.h
EXPORTS = (
    "csl_create", "csl_destroy", "csl_propagate", "csl_propagate_device", "csl_counts",
    "csl_fetch", "csl_device_results", "csl_seed_peaks", "csl_get_direction",
    "csl_device_constants", "csl_philox_stream", "csl_last_error", "csl_version",
    "csl_batch_timings", "csl_track_noalloc", "csl_boot_odf", "csl_odf_volume",
    "csl_compress", "csl_fetch_compressed",
    "csl_mlp_gemm", "csl_mlp_bias_act", "csl_mlp_act_bwd", "csl_mlp_colsum", "csl_mlp_vmf_nll",
    "csl_mlp_adam", "csl_mlp_param_count", "csl_mlp_infer", "csl_dti_fa", "csl_seeds_from_mask",
    "csl_multi_create", "csl_multi_launch", "csl_multi_wait", "csl_multi_info", "csl_multi_destroy",
    "csl_multi_set_concurrency",
    "csl_set_launch", "csl_get_launch", "csl_autotune", "csl_sampler_stats", "csl_env_step",
    "csl_device_count", "csl_dev_alloc", "csl_dev_free", "csl_dev_copy", "csl_dev_sync",
    "csl_ptt_layout", "csl_ptt_prepare", "csl_boot_step", "csl_boot_refit_stats",
)


def load(path: str | None = None):
    """Load the shared library (once) and declare argument types."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"gpustreamlines_b200: CUDA library not built ({p} missing); run "
            "`python -m gpustreamlines_b200.build` first (there is no CPU fallback)")
    lib = C.CDLL(p)
    vp = C.c_void_p
    ll = C.c_longlong
    ull_p = C.POINTER(C.c_ulonglong)
    lib.csl_create.argtypes = [C.POINTER(CslParams), C.POINTER(CslInputs), C.c_int, C.POINTER(vp)]
    lib.csl_destroy.argtypes = [vp]
    lib.csl_propagate.argtypes = [vp, _fp, ll, ll, vp]
    lib.csl_propagate_device.argtypes = [vp, vp, ll, ll, vp]
    lib.csl_counts.argtypes = [vp, C.POINTER(ll), C.POINTER(ll)]
    lib.csl_fetch.argtypes = [vp, _ip, _ip, _fp]
    lib.csl_device_results.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]
    lib.csl_seed_peaks.argtypes = [vp, _fp, ll, C.c_int, _ip, _ip, _fp]
    lib.csl_get_direction.argtypes = [vp, _fp, _fp, ull_p, ull_p, ll, _fp, _fp, _ip, _ip]
    lib.csl_device_constants.argtypes = [vp, _fp, _fp]
    lib.csl_batch_timings.argtypes = [vp, _fp, _ip]
    lib.csl_track_noalloc.argtypes = [vp, vp, ll, ll, C.c_int, vp, vp, vp, vp]
    lib.csl_boot_odf.argtypes = [vp, vp, vp, ll, C.c_int, vp, C.c_int, vp]
    lib.csl_compress.argtypes = [vp, C.POINTER(C.c_double), C.c_double, C.c_double, C.c_int, C.c_int,
                                 C.POINTER(ll)]
    lib.csl_fetch_compressed.argtypes = [vp, _ip, _fp]
    f32 = C.c_float
    lib.csl_mlp_gemm.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, vp, C.c_int, vp, C.c_int, vp,
                                 C.c_int, f32, vp]
    lib.csl_mlp_bias_act.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_int, vp]
    lib.csl_mlp_act_bwd.argtypes = [vp, vp, vp, ll, vp]
    lib.csl_mlp_colsum.argtypes = [vp, C.c_int, C.c_int, vp, vp]
    lib.csl_mlp_vmf_nll.argtypes = [vp, vp, C.c_int, f32, vp, vp, vp]
    lib.csl_mlp_adam.argtypes = [vp, vp, vp, vp, ll, f32, f32, f32, f32, C.c_int, vp]
    lib.csl_mlp_infer.argtypes = [vp, vp, C.c_int, vp, _fp, vp]
    dp = C.POINTER(C.c_double)
    lib.csl_dti_fa.argtypes = [vp, ll, C.c_int, dp, dp, vp, C.c_double, vp, vp]
    lib.csl_seeds_from_mask.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_float, ll, C.c_ulonglong, vp,
                                        C.POINTER(ll), vp]
    lib.csl_odf_volume.argtypes = [vp, ll, C.c_int, vp, C.c_int, C.c_int, vp, vp, ll, _fp, vp]
    lib.csl_philox_stream.argtypes = [C.c_ulonglong, C.c_ulonglong, C.c_ulonglong, ll,
                                      C.POINTER(C.c_uint)]
    llp = C.POINTER(ll)
    lib.csl_multi_create.argtypes = [C.POINTER(vp), C.POINTER(vp), llp, llp, C.c_int, C.c_int, C.POINTER(vp)]
    lib.csl_multi_launch.argtypes = [vp, vp]
    lib.csl_multi_wait.argtypes = [vp, llp, llp, _ip, _fp]
    lib.csl_multi_info.argtypes = [vp, _ip, _ip, llp]
    lib.csl_multi_destroy.argtypes = [vp]
    lib.csl_multi_set_concurrency.argtypes = [vp, C.c_int]
    lib.csl_set_launch.argtypes = [vp, C.c_int, C.c_int]
    lib.csl_get_launch.argtypes = [vp, _ip, _ip, _ip]
    lib.csl_autotune.argtypes = [vp, vp, ll, ll, C.c_int, _fp]
    lib.csl_boot_step.argtypes = [vp, vp, vp, vp, ll, vp, C.c_int, vp, vp]
    lib.csl_boot_refit_stats.argtypes = [vp, ull_p, C.c_int]
    lib.csl_ptt_layout.argtypes = [C.c_int, _ip, _ip, _ip, _ip, _ip]
    lib.csl_ptt_prepare.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, vp, C.c_int, C.c_int,
                                    C.c_int, vp, vp, vp]
    lib.csl_device_count.argtypes = [_ip]
    lib.csl_dev_alloc.argtypes = [C.c_int, C.c_ulonglong, C.POINTER(vp)]
    lib.csl_dev_free.argtypes = [C.c_int, vp]
    lib.csl_dev_copy.argtypes = [C.c_int, vp, vp, C.c_ulonglong, C.c_int]
    lib.csl_dev_sync.argtypes = [C.c_int]
    lib.csl_sampler_stats.argtypes = [vp, ull_p, C.c_int]
    lib.csl_env_step.argtypes = [vp, _fp, _ip, _ip, ull_p, ll, _ip, _ip]
    lib.csl_last_error.argtypes = [vp, C.c_char_p, C.c_int]
    lib.csl_version.restype = C.c_char_p
    for name in EXPORTS:
        if name != "csl_version":
            getattr(lib, name).restype = C.c_int
    if path is None:
        _lib = lib
    return lib


def last_error(handle=None) -> str:
    lib = load()
    buf = C.create_string_buffer(1024)
    lib.csl_last_error(handle, buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc: int, handle=None):
    if rc == CSL_OK:
        return
    msg = last_error(handle)
    if rc == CSL_E_INVALID:
        raise ValueError(msg)
    raise RuntimeError(f"gpustreamlines_b200 error {rc}: {msg}")


def fptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_fp)


def iptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_ip)


def any_fptr(a):
    """float pointer to a host numpy array or to a DeviceBuffer's device memory."""
    if isinstance(a, DeviceBuffer):
        return C.cast(C.c_void_p(a.ptr), _fp)
    return fptr(a)


def uptr(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_ulonglong))


def philox_stream(seed: int, subsequence: int, offset: int, n: int) -> np.ndarray:
    """This library's Philox4x32-10 words (curand_init(seed, subsequence, offset) layout)."""
    lib = load()
    out = np.empty(n, dtype=np.uint32)
    check(lib.csl_philox_stream(seed, subsequence, offset, n,
                                out.ctypes.data_as(C.POINTER(C.c_uint))))
    return out


def device_count() -> int:
    """CUDA devices visible to the library (0 without a driver or device)."""
    n = C.c_int()
    check(load().csl_device_count(C.byref(n)))
    return n.value


class DeviceBuffer:
    """Device memory owned by the library's allocator (no framework needed).

    ``DeviceBuffer(device, shape, dtype)`` allocates; ``from_array`` copies a
    host array in; ``numpy()`` copies back; ``ptr`` is the raw device address
    for the C ABI.  Freed on ``close()`` or garbage collection.
    """

    def __init__(self, device: int, shape, dtype=np.float32):
        self.lib = load()
        self.device = int(device)
        self.shape = tuple(int(x) for x in (shape if hasattr(shape, "__len__") else (shape,)))
        self.dtype = np.dtype(dtype)
        self.nbytes = int(np.prod(self.shape, dtype=np.int64)) * self.dtype.itemsize
        p = C.c_void_p()
        check(self.lib.csl_dev_alloc(self.device, max(self.nbytes, 1), C.byref(p)))
        self._p = p

    @classmethod
    def from_array(cls, a, device: int = 0, dtype=None):
        a = np.ascontiguousarray(a, dtype=dtype or np.asarray(a).dtype)
        b = cls(device, a.shape, a.dtype)
        b.upload(a)
        return b

    @property
    def ptr(self) -> int:
        return self._p.value or 0

    def upload(self, a):
        a = np.ascontiguousarray(a, dtype=self.dtype)
        if a.nbytes > self.nbytes:
            raise ValueError("array larger than the buffer")
        check(self.lib.csl_dev_copy(self.device, self._p, a.ctypes.data_as(C.c_void_p), a.nbytes, 1))

    def numpy(self) -> np.ndarray:
        out = np.empty(self.shape, dtype=self.dtype)
        check(self.lib.csl_dev_copy(self.device, out.ctypes.data_as(C.c_void_p), self._p, self.nbytes, 2))
        return out

    def reshape(self, *shape):
        shape = shape[0] if len(shape) == 1 and hasattr(shape[0], "__len__") else shape
        if int(np.prod(shape, dtype=np.int64)) * self.dtype.itemsize != self.nbytes:
            raise ValueError("reshape must keep the size")
        self.shape = tuple(int(x) for x in shape)
        return self

    def close(self):
        if getattr(self, "_p", None) is not None and self._p.value:
            self.lib.csl_dev_free(self.device, self._p)
        self._p = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def device_sync(device: int = 0):
    check(load().csl_dev_sync(int(device)))


class Handle:
    """Owns one ``csl_tracker`` (one device)."""

    def __init__(self, params: CslParams, inputs: CslInputs, device: int, keepalive=()):
        self.lib = load()
        self._keep = list(keepalive)
        h = C.c_void_p()
        check(self.lib.csl_create(C.byref(params), C.byref(inputs), int(device), C.byref(h)))
        self.h = h
        self.device = device
        self.model = params.model
        self._keep = []  # inputs were copied to the device

    def close(self):
        if getattr(self, "h", None):
            self.lib.csl_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc):
        check(rc, self.h)

    def propagate(self, seeds: np.ndarray, rng_index_base: int = 0, stream: int | None = None):
        seeds = np.ascontiguousarray(seeds, dtype=np.float32).reshape(-1, 3)
        self._chk(self.lib.csl_propagate(self.h, fptr(seeds), len(seeds), int(rng_index_base),
                                         stream))

    def propagate_device(self, seeds_ptr: int, n: int, rng_index_base: int = 0,
                         stream: int | None = None):
        self._chk(self.lib.csl_propagate_device(self.h, C.c_void_p(seeds_ptr), int(n),
                                                int(rng_index_base), stream))

    def counts(self):
        a, b = C.c_longlong(), C.c_longlong()
        self._chk(self.lib.csl_counts(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def fetch(self, lengths=True, seed_index=True, points=True):
        nsl, npts = self.counts()
        L = np.empty(nsl, dtype=np.int32) if lengths else None
        S = np.empty(nsl, dtype=np.int32) if seed_index else None
        Pt = np.empty((npts, 3), dtype=np.float32) if points else None
        self._chk(self.lib.csl_fetch(self.h, iptr(L), iptr(S), fptr(Pt)))
        return L, S, Pt

    def fetch_into(self, L, S, Pt):
        self._chk(self.lib.csl_fetch(self.h, iptr(L), iptr(S), fptr(Pt)))

    def device_results(self):
        ptrs = [C.c_void_p() for _ in range(4)]
        self._chk(self.lib.csl_device_results(self.h, *[C.byref(p) for p in ptrs]))
        return tuple(p.value for p in ptrs)

    def seed_peaks(self, seeds: np.ndarray, max_peaks: int = 32):
        seeds = np.ascontiguousarray(seeds, dtype=np.float32).reshape(-1, 3)
        n = len(seeds)
        counts = np.zeros(n, dtype=np.int32)
        pv = np.full((n, max_peaks), -1, dtype=np.int32)
        pd = np.zeros((n, max_peaks, 3), dtype=np.float32)
        self._chk(self.lib.csl_seed_peaks(self.h, fptr(seeds), n, max_peaks, iptr(counts),
                                          iptr(pv), fptr(pd)))
        return counts, pv, pd

    def get_direction(self, points, dirs, subsequence, offset, frames=None):
        pts = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
        ds = np.ascontiguousarray(dirs, dtype=np.float32).reshape(-1, 3)
        n = len(pts)
        sq = np.ascontiguousarray(subsequence, dtype=np.uint64).reshape(n)
        of = np.ascontiguousarray(offset, dtype=np.uint64).reshape(n)
        fr = None if frames is None else np.ascontiguousarray(frames, dtype=np.float32).reshape(n, 9)
        nd = np.zeros((n, 3), dtype=np.float32)
        ok = np.zeros(n, dtype=np.int32)
        dr = np.zeros(n, dtype=np.int32)
        self._chk(self.lib.csl_get_direction(self.h, fptr(pts), fptr(ds), uptr(sq), uptr(of), n,
                                             fptr(fr), fptr(nd), iptr(ok), iptr(dr)))
        return nd, ok, dr, fr

    def track_noalloc(self, seeds_ptr: int, n: int, rng_index_base: int, max_peaks: int,
                      counts_ptr: int, lens_ptr: int, points_ptr: int, stream: int | None = None):
        """Allocation-free tracking into caller-owned device buffers (see the C header)."""
        self._chk(self.lib.csl_track_noalloc(self.h, C.c_void_p(seeds_ptr), int(n),
                                             int(rng_index_base), int(max_peaks),
                                             C.c_void_p(counts_ptr), C.c_void_p(lens_ptr),
                                             C.c_void_p(points_ptr), stream))

    def boot_odf(self, points_ptr: int, resample_ptr: int, n: int, fit: int, odf_ptr: int, odf_stride: int,
                 stream: int | None = None):
        """ODF of one bootstrap fit per point with given resample indices, into
        a device buffer (fit 0: per-warp FP32, 1: batched BF16x3; see the C header)."""
        self._chk(self.lib.csl_boot_odf(self.h, C.c_void_p(points_ptr), C.c_void_p(resample_ptr), int(n),
                                        int(fit), C.c_void_p(odf_ptr), int(odf_stride), stream))

    def boot_step(self, points_ptr: int, resample_ptr: int, dirs_ptr: int, n: int, odf_ptr: int, odf_stride: int,
                  step_ptr: int, stream: int | None = None):
        """The batched fit's step at fixed state into device buffers (see the C header)."""
        self._chk(self.lib.csl_boot_step(self.h, C.c_void_p(points_ptr), C.c_void_p(resample_ptr),
                                         C.c_void_p(dirs_ptr), int(n), C.c_void_p(odf_ptr), int(odf_stride),
                                         C.c_void_p(step_ptr), stream))

    def boot_refit_stats(self, reset: bool = False):
        """{rows searched, rows fitted again in float64} of the batched fit."""
        out = np.zeros(2, dtype=np.uint64)
        self._chk(self.lib.csl_boot_refit_stats(self.h, uptr(out), int(bool(reset))))
        return {"rows": int(out[0]), "refit": int(out[1])}

    def compress(self, affine=None, tol_error=0.1, max_segment_length=10.0, minlen=0, maxlen=None):
        """Linearise the last batch on the device in world coordinates; returns
        (counts per streamline, 0 = dropped; kept points [n, 3] float32)."""
        aff = None
        if affine is not None:
            a = np.ascontiguousarray(np.asarray(affine, dtype=np.float64).reshape(4, 4))
            aff = a.ctypes.data_as(C.POINTER(C.c_double))
        mx = 2**31 - 1 if maxlen is None or not np.isfinite(maxlen) else int(min(maxlen, 2**31 - 1))
        npts = C.c_longlong()
        self._chk(self.lib.csl_compress(self.h, aff, float(tol_error), float(max_segment_length),
                                        int(max(0, minlen)), mx, C.byref(npts)))
        nsl, _ = self.counts()
        cnt = np.empty(nsl, dtype=np.int32)
        pts = np.empty((npts.value, 3), dtype=np.float32)
        self._chk(self.lib.csl_fetch_compressed(self.h, iptr(cnt), fptr(pts)))
        return cnt, pts

    def timings(self):
        """(pass1_ms, gap_ms, pass2_ms, compact_ms), pass-2 runs of the last batch."""
        ms = np.zeros(4, dtype=np.float32)
        runs = C.c_int()
        self._chk(self.lib.csl_batch_timings(self.h, fptr(ms), C.byref(runs)))
        return tuple(float(x) for x in ms), runs.value

    def set_launch(self, threads_per_block: int, seed_order: int):
        self._chk(self.lib.csl_set_launch(self.h, int(threads_per_block), int(seed_order)))

    def get_launch(self):
        """(threads per CTA, seed order, CTAs per SM) of the per-warp tracking path."""
        b, o, k = C.c_int(), C.c_int(), C.c_int()
        self._chk(self.lib.csl_get_launch(self.h, C.byref(b), C.byref(o), C.byref(k)))
        return b.value, o.value, k.value

    def autotune(self, seeds_ptr: int, n: int, rng_index_base: int = 0, repeats: int = 2):
        """Time the six launch shapes on a device seed sample and keep the fastest.

        Returns {(threads_per_block, seed_order): ms or None}."""
        ms = np.zeros(6, dtype=np.float32)
        self._chk(self.lib.csl_autotune(self.h, C.c_void_p(seeds_ptr), int(n), int(rng_index_base),
                                        int(repeats), fptr(ms)))
        shapes = [(256, 0), (256, 1), (128, 0), (128, 1), (64, 0), (64, 1)]
        return {sh: (float(v) if v >= 0 else None) for sh, v in zip(shapes, ms)}

    def sampler_stats(self, reset: bool = False):
        """Envelope-sampler counters since creation or the last reset:
        {steps, proposals, resolves, fallbacks}."""
        out = np.zeros(4, dtype=np.uint64)
        self._chk(self.lib.csl_sampler_stats(self.h, uptr(out), int(bool(reset))))
        return dict(zip(("steps", "proposals", "resolves", "fallbacks"), (int(x) for x in out)))

    def env_step(self, points, dir_vertex, dir_neg, subsequence):
        """One envelope-sampler direction per query; returns (vertex or -1, sign)."""
        pts = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
        n = len(pts)
        dv = np.ascontiguousarray(dir_vertex, dtype=np.int32).reshape(n)
        dn = np.ascontiguousarray(dir_neg, dtype=np.int32).reshape(n)
        sq = np.ascontiguousarray(subsequence, dtype=np.uint64).reshape(n)
        ov = np.zeros(n, dtype=np.int32)
        on = np.zeros(n, dtype=np.int32)
        self._chk(self.lib.csl_env_step(self.h, fptr(pts), iptr(dv), iptr(dn), uptr(sq), n, iptr(ov),
                                        iptr(on)))
        return ov, on

    def device_constants(self):
        a, b = C.c_float(), C.c_float()
        self._chk(self.lib.csl_device_constants(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value


class MultiPlan:
    """Owns one ``csl_multi``: the batches of several handles (subjects) as
    branches of one captured CUDA graph.  ``seeds`` are device pointers with
    their counts; the plan keeps the handles alive."""

    def __init__(self, handles, seeds_ptrs, counts, rng_index_base=None, points_per_streamline: int = 0):
        self.lib = load()
        n = len(handles)
        if not (len(seeds_ptrs) == len(counts) == n):
            raise ValueError("one seed batch per subject")
        self.handles = list(handles)
        self.n = n
        subs = (C.c_void_p * n)(*[h.h for h in handles])
        sp = (C.c_void_p * n)(*[int(p) for p in seeds_ptrs])
        cnt = (C.c_longlong * n)(*[int(c) for c in counts])
        rb = None if rng_index_base is None else (C.c_longlong * n)(*[int(r) for r in rng_index_base])
        p = C.c_void_p()
        check(self.lib.csl_multi_create(subs, sp, cnt, rb, n, int(points_per_streamline), C.byref(p)))
        self.p = p

    def launch(self, stream: int | None = None):
        check(self.lib.csl_multi_launch(self.p, C.c_void_p(stream) if stream else None))

    def wait(self):
        """(n_streamlines [n], n_points [n], replayed [n], graph ms)."""
        nsl = np.zeros(self.n, dtype=np.int64)
        npts = np.zeros(self.n, dtype=np.int64)
        rep = np.zeros(self.n, dtype=np.int32)
        ms = np.zeros(1, dtype=np.float32)
        llp = C.POINTER(C.c_longlong)
        check(self.lib.csl_multi_wait(self.p, nsl.ctypes.data_as(llp), npts.ctypes.data_as(llp), iptr(rep),
                                      fptr(ms)))
        return nsl, npts, rep, float(ms[0])

    def set_concurrency(self, max_concurrent: int):
        """At most this many tracking kernels in flight (0: no limit); next launch re-captures."""
        check(self.lib.csl_multi_set_concurrency(self.p, int(max_concurrent)))

    def info(self):
        """(graph captures so far, slot capacities [n], pool capacities in points [n])."""
        cap = C.c_int()
        sl = np.zeros(self.n, dtype=np.int32)
        pool = np.zeros(self.n, dtype=np.int64)
        check(self.lib.csl_multi_info(self.p, C.byref(cap), iptr(sl),
                                      pool.ctypes.data_as(C.POINTER(C.c_longlong))))
        return cap.value, sl, pool

    def close(self):
        if getattr(self, "p", None):
            self.lib.csl_multi_destroy(self.p)
            self.p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
