"""ctypes wrappers of the C oracle and of the compiled reference -- TEST INFRASTRUCTURE ONLY.

Used by tests/ (as the checker) and by bench.py's CPU-baseline leg.
"""

from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


class OrcParams(C.Structure):
    _fields_ = [
        ("model", C.c_int), ("dimx", C.c_int), ("dimy", C.c_int), ("dimz", C.c_int), ("dimt", C.c_int),
        ("nvert", C.c_int), ("nedges", C.c_int), ("samplm_nr", C.c_int),
        ("sphere_symm", C.c_int), ("max_sline_len", C.c_int),
        ("step_size", C.c_double), ("max_angle", C.c_double), ("tc_threshold", C.c_double),
        ("relative_peak_thresh", C.c_double), ("min_separation_angle", C.c_double),
        ("pmf_threshold", C.c_double), ("rng_seed", C.c_uint64),
        ("cos_max_angle", C.c_float), ("cos_min_sep", C.c_float), ("min_signal", C.c_float),
        ("delta_nr", C.c_int),
        ("dataf", _fp), ("stop_map", _fp), ("verts", _fp), ("edges", _ip),
        ("H", _fp), ("R", _fp), ("delta_b", _fp), ("delta_q", _fp), ("sampling", _fp),
        ("b0s_mask", _ip),
        ("ptt_odf", _fp), ("ptt_lut", _fp),
        ("lut_res", C.c_int), ("log2_x", C.c_int), ("log2_y", C.c_int), ("tile_nx", C.c_int),
        ("tile_ny", C.c_int), ("tile_nz", C.c_int), ("step_frac", C.c_int), ("ptt_pad", C.c_int),
        ("probe_step_size", C.c_float), ("probe_quality", C.c_float), ("max_curvature", C.c_double),
        ("rng_base", C.c_longlong),
    ]


def _f(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32).ctypes.data_as(_fp)


def _i(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32).ctypes.data_as(_ip)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            from oracle.build import build
            build()
        L = C.CDLL(LIB)
        u64 = C.c_uint64
        ll = C.c_longlong
        L.orc_philox_stream.argtypes = [u64, u64, u64, ll, C.POINTER(C.c_uint32)]
        L.orc_philox_uniform.argtypes = [u64, u64, u64, ll, _fp]
        L.orc_sort_partners.argtypes = [_ip]
        L.orc_sample_stop.argtypes = [C.POINTER(OrcParams), _fp, ll, _fp]
        L.orc_seed_peaks.argtypes = [C.POINTER(OrcParams), _fp, ll, _ip, _ip, C.c_int, C.c_int]
        L.orc_track.argtypes = [C.POINTER(OrcParams), _fp, ll, _ip, _ip, C.c_int, _ip, _ip, _fp, C.c_int]
        L.orc_track.restype = ll
        L.orc_get_direction.argtypes = [C.POINTER(OrcParams), _fp, _fp, C.POINTER(u64), C.POINTER(u64),
                                        ll, _fp, _ip, _ip, _fp]
        L.orc_dot3_forms.argtypes = [_fp, _fp, ll, _fp]
        u32p = C.POINTER(C.c_uint32)
        L.orc_philox_block.argtypes = [u32p, u32p, u32p]
        _lib = L
    return _lib


def dot3_forms(a, b):
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    out = np.zeros((len(a), 3), dtype=np.float32)
    lib().orc_dot3_forms(_f(a), _f(b), len(a), out.ctypes.data_as(_fp))
    return out


def philox_block(ctr, key):
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    p = C.POINTER(C.c_uint32)
    lib().orc_philox_block(c.ctypes.data_as(p), k.ctypes.data_as(p), o.ctypes.data_as(p))
    return o


def philox_stream(seed, subseq, offset, n):
    out = np.empty(n, dtype=np.uint32)
    lib().orc_philox_stream(seed, subseq, offset, n, out.ctypes.data_as(C.POINTER(C.c_uint32)))
    return out


def philox_uniform(seed, subseq, offset, n):
    out = np.empty(n, dtype=np.float32)
    lib().orc_philox_uniform(seed, subseq, offset, n, out.ctypes.data_as(_fp))
    return out


def sort_partners():
    out = np.zeros((15, 32), dtype=np.int32)
    lib().orc_sort_partners(out.ctypes.data_as(_ip))
    return out


class Oracle:
    """Oracle bound to one case's host inputs (see oracle/cases.py)."""

    def __init__(self, inp: dict, cos_max_angle=None, cos_min_sep=None, max_sline_len=501, ptt=None):
        c = inp["case"]
        self.inp = inp
        self._keep = []
        P = OrcParams()
        model = {"OPDT": 0, "CSA": 1, "PROB": 2, "PTT": 3}[c["model"]]
        d = np.ascontiguousarray(inp["dataf"], dtype=np.float32)
        P.model = model
        P.dimx, P.dimy, P.dimz, P.dimt = d.shape
        verts = np.ascontiguousarray(inp["vertices"], dtype=np.float32)
        edges = np.ascontiguousarray(inp["edges"], dtype=np.int32)
        P.nvert, P.nedges = len(verts), len(edges)
        P.samplm_nr = inp["sampling_matrix"].shape[0] if model < 2 else d.shape[3]
        P.sphere_symm = int(c.get("sphere_symm", 0))
        P.max_sline_len = max_sline_len
        P.step_size = float(np.float32(c["step"]))
        P.max_angle = float(np.float32(math.radians(c["max_angle"])))
        P.tc_threshold = float(np.float32(c["fa_thr"]))
        P.relative_peak_thresh = float(np.float32(c["rel"]))
        P.min_separation_angle = float(np.float32(math.radians(c["min_sep"])))
        P.pmf_threshold = 0.05
        P.rng_seed = int(c["rng_seed"])
        P.cos_max_angle = np.float32(np.cos(np.float32(P.max_angle))) if cos_max_angle is None \
            else cos_max_angle
        P.cos_min_sep = np.float32(np.cos(np.float32(P.min_separation_angle))) if cos_min_sep is None \
            else cos_min_sep
        stop = np.ascontiguousarray(inp["stop_map"], dtype=np.float32)
        arrs = [d, stop, verts, edges]
        P.dataf, P.stop_map, P.verts, P.edges = _f(d), _f(stop), _f(verts), _i(edges)
        if model < 2:
            mats = [np.ascontiguousarray(inp[k], dtype=np.float32)
                    for k in ("H", "R", "delta_b", "delta_q", "sampling_matrix")]
            arrs += mats
            P.H, P.R, P.delta_b, P.delta_q, P.sampling = (_f(m) for m in mats)
            b0 = np.ascontiguousarray(inp["b0s_mask"], dtype=np.int32)
            arrs.append(b0)
            P.b0s_mask = _i(b0)
            P.delta_nr = mats[2].shape[0]
            P.min_signal = float(inp.get("min_signal", 1.0))
        if model == 3:
            if ptt is None:
                raise ValueError("the PTT oracle needs the tiled texture layout (cases.ptt_layout)")
            tiled = np.ascontiguousarray(ptt["tiled"], dtype=np.float32)
            lut = np.ascontiguousarray(ptt["lut"], dtype=np.float32)
            arrs += [tiled, lut]
            P.ptt_odf, P.ptt_lut = _f(tiled), _f(lut)
            P.lut_res = int(ptt["res"])
            P.log2_x, P.log2_y = int(ptt["log2_x"]), int(ptt["log2_y"])
            P.tile_nx, P.tile_ny, P.tile_nz = int(ptt["nx"]), int(ptt["ny"]), int(ptt["nz"])
            P.step_frac = int(np.round(np.float32(c["step"]) / 0.025))
            P.probe_step_size = 0.25
            P.probe_quality = 8.0
            P.max_curvature = float(8.0 * np.sin(np.float32(math.radians(c["max_angle"])) / 2.0))
        self._keep = arrs
        self.P = P

    def seed_peaks(self, seeds, maxp=32, threads=0):
        seeds = np.ascontiguousarray(seeds, dtype=np.float32)
        n = len(seeds)
        counts = np.zeros(n, dtype=np.int32)
        peaks = np.full((n, maxp), -1, dtype=np.int32)
        lib().orc_seed_peaks(C.byref(self.P), _f(seeds), n, _i(counts), peaks.ctypes.data_as(_ip),
                             maxp, threads)
        return counts, peaks

    def track(self, seeds, threads=0, maxp=32, rng_index_base=0):
        """Full two-pass tracking -> (counts, lengths, seed index, compacted points).
        Seed s uses the Philox streams of index s + rng_index_base."""
        seeds = np.ascontiguousarray(seeds, dtype=np.float32)
        self.P.rng_base = int(rng_index_base)
        counts, peaks = self.seed_peaks(seeds, maxp, threads)
        if (counts > maxp).any():
            raise RuntimeError("oracle: raise maxp")
        nsl = int(counts.sum())
        lens = np.zeros(max(nsl, 1), dtype=np.int32)
        sidx = np.zeros(max(nsl, 1), dtype=np.int32)
        slot = 2 * self.P.max_sline_len * 3
        pts = np.zeros((max(nsl, 1), slot), dtype=np.float32)
        lib().orc_track(C.byref(self.P), _f(seeds), len(seeds), _i(counts), peaks.ctypes.data_as(_ip),
                        maxp, lens.ctypes.data_as(_ip), sidx.ctypes.data_as(_ip),
                        pts.ctypes.data_as(_fp), threads)
        lens, sidx = lens[:nsl], sidx[:nsl]
        flat = np.concatenate([pts[j, :3 * lens[j]].reshape(-1, 3) for j in range(nsl)]) if nsl else \
            np.zeros((0, 3), np.float32)
        return counts, lens, sidx, flat

    def get_direction(self, points, dirs, subseq, offs, frames=None):
        """One getter call per query.  PTT takes and updates ``frames`` [n, 9]
        (tangent, normal, binormal) and uses offset 0 of each lane's stream."""
        pts = np.ascontiguousarray(points, dtype=np.float32)
        ds = np.ascontiguousarray(dirs, dtype=np.float32)
        n = len(pts)
        sq = np.ascontiguousarray(subseq, dtype=np.uint64)
        of = np.ascontiguousarray(offs, dtype=np.uint64)
        nd = np.zeros((n, 3), dtype=np.float32)
        ok = np.zeros(n, dtype=np.int32)
        dr = np.zeros(n, dtype=np.int32)
        fr = None if frames is None else np.ascontiguousarray(frames, dtype=np.float32).reshape(n, 9).copy()
        lib().orc_get_direction(C.byref(self.P), _f(pts), _f(ds),
                                sq.ctypes.data_as(C.POINTER(C.c_uint64)),
                                of.ctypes.data_as(C.POINTER(C.c_uint64)), n, nd.ctypes.data_as(_fp),
                                ok.ctypes.data_as(_ip), dr.ctypes.data_as(_ip),
                                None if fr is None else fr.ctypes.data_as(_fp))
        return (nd, ok, dr) if fr is None else (nd, ok, dr, fr)

    def sample_stop(self, points):
        pts = np.ascontiguousarray(points, dtype=np.float32)
        out = np.zeros(len(pts), dtype=np.float32)
        lib().orc_sample_stop(C.byref(self.P), _f(pts), len(pts), out.ctypes.data_as(_fp))
        return out


class Reference:
    """The reference's own kernels (oracle/_ref/ref_<case>.so), GPU only."""

    def __init__(self, case_name: str):
        path = os.path.join(REF_DIR, f"ref_{case_name}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = C.CDLL(path)
        L.ref_config.restype = C.c_char_p
        L.ref_track.restype = C.c_longlong
        L.ref_track.argtypes = [_fp, C.c_int, _fp, _fp, _fp, _ip, _fp, _fp, _fp, _fp, _fp, _ip,
                                C.c_float, C.c_int, _fp, C.c_int, C.c_int, C.c_int, _fp, C.c_int, _ip,
                                _fp, C.c_int, _ip, _ip, _fp, _fp]
        self.L = L
        self.name = case_name

    def track(self, inp: dict, seeds, cap=None, ptt=None, points=True):
        seeds = np.ascontiguousarray(seeds, dtype=np.float32)
        n = len(seeds)
        counts = np.zeros(n, dtype=np.int32)
        cap = cap if cap is not None else 12 * n + 16
        sl_seed = np.zeros(cap, dtype=np.int32)
        sl_len = np.zeros(cap, dtype=np.int32)
        slines = np.zeros((cap if points else 1, 2 * 501 * 3), dtype=np.float32)
        boot = "H" in inp
        args = [_f(seeds), n, _f(inp["dataf"]) if ptt is None else None, _f(inp["stop_map"]),
                _f(inp["vertices"]), _i(inp["edges"])]
        if boot:
            args += [_f(inp["H"]), _f(inp["R"]), _f(inp["delta_b"]), _f(inp["delta_q"]),
                     _f(inp["sampling_matrix"]), _i(inp["b0s_mask"]), float(inp["min_signal"]),
                     int(inp["delta_b"].shape[0])]
        else:
            args += [None] * 6 + [0.0, 0]
        if ptt is not None:
            t = ptt["tiled"]
            args += [_f(t), t.shape[2], t.shape[1], t.shape[0], _f(ptt["lut"]), int(ptt["res"])]
        else:
            args += [None, 0, 0, 0, None, 0]
        ms = np.zeros(2, dtype=np.float32)
        args += [_i(counts), None, cap, _i(sl_seed), _i(sl_len),
                 slines.ctypes.data_as(_fp) if points else None, ms.ctypes.data_as(_fp)]
        nsl = self.L.ref_track(*args)
        self.last_ms = (float(ms[0]), float(ms[1]))
        if nsl < 0:
            raise RuntimeError(f"reference kernels failed ({nsl})")
        if boot:  # pass 1 only: the reference's bootstrap pass 2 is not launched
            return counts, None, None, None
        if nsl > cap:
            return self.track(inp, seeds, cap=int(nsl) + 16, ptt=ptt, points=points)
        sl_seed, sl_len = sl_seed[:nsl], sl_len[:nsl]
        if not points:
            return counts, sl_len, sl_seed, None
        flat = np.concatenate([slines[j, :3 * sl_len[j]].reshape(-1, 3) for j in range(nsl)]) if nsl \
            else np.zeros((0, 3), np.float32)
        return counts, sl_len, sl_seed, flat
