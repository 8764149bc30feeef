"""Streamline containers and the TRK / TRX writers used by the chunked seed loop.

The reference builds on nibabel (``ArraySequence``, ``Tractogram``, TRK via
``save_tractogram``), trx-python (memory-mapped ``TrxFile``) and DIPY
(``StatefulTractogram``, ``compress_streamlines``); see
``cuslines/generic_tracker.py:1-9``.  None of these packages is available
offline, so this module provides minimal, format-conformant equivalents:

* ``ArraySequence``: points ``_data [N,3]``, ``_offsets``, ``_lengths``;
* ``Tractogram`` / ``StatefulTractogram``: streamlines + affine (voxel -> RAS mm);
* ``TrxFile``: memory-mapped positions/offsets in a work directory, grown by
  doubling, saved as a TRX zip (``header.json``, ``positions.3.<dtype>``,
  ``offsets.uint64``) -- the TRX specification's layout;
* TRK (TrackVis v2): 1000-byte header, then per streamline an int32 point
  count and float32 points in voxel-mm coordinates (corner origin);
* ``compress_streamlines``: the linearisation of Presseau et al. 2015
  (drop points while the reconstructed polyline stays within ``tol_error``
  mm and segments stay shorter than ``max_segment_length`` mm).
"""

from __future__ import annotations

import json
import os
import shutil
import struct
import tempfile
import zipfile

import numpy as np

MEGABYTE = 1024 * 1024


class ArraySequence:
    def __init__(self, iterable=None, buffer_size=4):
        self._data = np.zeros((0, 3), dtype=np.float32)
        self._offsets = np.zeros(0, dtype=np.int64)
        self._lengths = np.zeros(0, dtype=np.int64)
        if iterable is None:
            return
        items = [np.asarray(x) for x in iterable]
        if items:
            self._lengths = np.array([len(x) for x in items], dtype=np.int64)
            self._offsets = np.concatenate([[0], np.cumsum(self._lengths)[:-1]]).astype(np.int64)
            self._data = np.concatenate(items, axis=0) if self._lengths.sum() else \
                np.zeros((0, 3), dtype=items[0].dtype)

    @classmethod
    def from_flat(cls, data, lengths, offsets=None):
        a = cls()
        a._data = data
        a._lengths = np.asarray(lengths, dtype=np.int64)
        if offsets is None:
            offsets = np.zeros(len(a._lengths), dtype=np.int64)
            if len(a._lengths):
                np.cumsum(a._lengths[:-1], out=offsets[1:])
        a._offsets = np.asarray(offsets, dtype=np.int64)
        return a

    def __len__(self):
        return len(self._lengths)

    def __getitem__(self, i):
        if isinstance(i, (int, np.integer)):
            o = self._offsets[i]
            return self._data[o:o + self._lengths[i]]
        raise TypeError("integer index expected")

    def __iter__(self):
        for i in range(len(self)):
            yield self[i]

    def copy(self):
        return ArraySequence.from_flat(self._data.copy(), self._lengths.copy(), self._offsets.copy())

    @property
    def total_nb_rows(self):
        return int(self._lengths.sum())


def apply_affine(aff, pts):
    aff = np.asarray(aff, dtype=np.float64)
    return (np.asarray(pts, dtype=np.float64) @ aff[:3, :3].T + aff[:3, 3])


class Tractogram:
    """Streamlines plus the affine that maps them to RAS mm."""

    def __init__(self, streamlines=None, affine_to_rasmm=None):
        self.streamlines = streamlines if streamlines is not None else ArraySequence()
        self.affine_to_rasmm = np.eye(4) if affine_to_rasmm is None else np.asarray(affine_to_rasmm)

    def __len__(self):
        return len(self.streamlines)

    def to_world(self):
        s = self.streamlines
        if len(s):
            s._data = apply_affine(self.affine_to_rasmm, s._data).astype(s._data.dtype)
        self.affine_to_rasmm = np.eye(4)
        return self


class Space:
    VOX = "vox"
    VOXMM = "voxmm"
    RASMM = "rasmm"


def _ref_affine_dims(ref_img):
    if hasattr(ref_img, "affine"):
        aff = np.asarray(ref_img.affine, dtype=np.float64)
        dims = tuple(int(d) for d in ref_img.shape[:3])
    else:
        aff, dims = ref_img
        aff = np.asarray(aff, dtype=np.float64)
        dims = tuple(int(d) for d in dims)
    return aff, dims


class StatefulTractogram:
    """Streamlines in a known space of a reference image (DIPY's role)."""

    def __init__(self, streamlines, reference, space=Space.VOX):
        self.streamlines = streamlines
        self.affine, self.dimensions = _ref_affine_dims(reference)
        self.space = space

    def __len__(self):
        return len(self.streamlines)


class RefImage:
    """Minimal stand-in for a nibabel image: ``affine`` and ``shape``."""

    def __init__(self, affine, shape):
        self.affine = np.asarray(affine, dtype=np.float64)
        self.shape = tuple(shape)


# ----------------------------------------------------------------------------- TRX


class TrxFile:
    """Memory-mapped TRX tractogram (positions in RAS mm)."""

    def __init__(self, nb_streamlines=0, nb_vertices=0, init_as=None, reference=None,
                 pos_dtype=np.float32):
        if init_as is not None:
            self.header = dict(init_as.header)
            pos_dtype = init_as.pos_dtype
        else:
            aff, dims = _ref_affine_dims(reference) if reference is not None else (np.eye(4), (1, 1, 1))
            self.header = {"DIMENSIONS": list(dims), "VOXEL_TO_RASMM": aff.tolist(),
                           "NB_VERTICES": 0, "NB_STREAMLINES": 0}
        self.pos_dtype = np.dtype(pos_dtype)
        self._dir = tempfile.mkdtemp(prefix="csl_trx_")
        self.header["NB_STREAMLINES"] = int(nb_streamlines)
        self.header["NB_VERTICES"] = int(nb_vertices)
        self.streamlines = ArraySequence()
        self._alloc(nb_streamlines, nb_vertices)

    def _mm(self, name, dtype, shape):
        path = os.path.join(self._dir, name)
        n = int(np.prod(shape))
        if n == 0:
            return np.zeros(shape, dtype=dtype)
        return np.memmap(path, dtype=dtype, mode="w+", shape=shape)

    def _alloc(self, nsl, nv, keep_sl=0, keep_v=0, old=None):
        data = self._mm(f"positions.{nv}.3.{self.pos_dtype.name}", self.pos_dtype, (nv, 3))
        offs = self._mm(f"offsets.{nsl}.uint64", np.uint64, (nsl,))
        lens = self._mm(f"lengths.{nsl}.uint32", np.uint32, (nsl,))
        if old is not None:
            data[:keep_v] = old._data[:keep_v]
            offs[:keep_sl] = old._offsets[:keep_sl]
            lens[:keep_sl] = old._lengths[:keep_sl]
        s = ArraySequence()
        s._data, s._offsets, s._lengths = data, offs, lens
        self.streamlines = s

    def resize(self, nb_streamlines=None, nb_vertices=None):
        """Grow (or, with no arguments, shrink to the used size)."""
        used_sl = self._used_sl
        used_v = self._used_v
        if nb_streamlines is None:
            nb_streamlines, nb_vertices = used_sl, used_v
        old = self.streamlines
        self._alloc(nb_streamlines, nb_vertices, min(used_sl, nb_streamlines),
                    min(used_v, nb_vertices), old)
        self.header["NB_STREAMLINES"] = int(nb_streamlines)
        self.header["NB_VERTICES"] = int(nb_vertices)

    _used_sl = 0
    _used_v = 0

    def append_block(self, data, lengths):
        """Append streamlines given as flat points + lengths (grows by doubling)."""
        n = len(lengths)
        nv = len(data)
        need_sl = self._used_sl + n
        need_v = self._used_v + nv
        if need_sl > self.header["NB_STREAMLINES"] or need_v > self.header["NB_VERTICES"]:
            self.resize(max(need_sl * 2, self.header["NB_STREAMLINES"]),
                        max(need_v * 2, self.header["NB_VERTICES"]))
        s = self.streamlines
        s._data[self._used_v:need_v] = data
        offs = np.zeros(n, dtype=np.uint64)
        if n:
            np.cumsum(np.asarray(lengths[:-1], dtype=np.uint64), out=offs[1:])
        s._offsets[self._used_sl:need_sl] = offs + np.uint64(self._used_v)
        s._lengths[self._used_sl:need_sl] = lengths
        self._used_sl, self._used_v = need_sl, need_v

    def __len__(self):
        return self._used_sl

    def close(self):
        shutil.rmtree(self._dir, ignore_errors=True)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def save_trx(trx: TrxFile, filename: str):
    """Write a TRX zip archive (uncompressed members)."""
    n = trx._used_sl
    nv = trx._used_v
    hdr = dict(trx.header)
    hdr["NB_STREAMLINES"] = int(n)
    hdr["NB_VERTICES"] = int(nv)
    s = trx.streamlines
    with zipfile.ZipFile(filename, "w", compression=zipfile.ZIP_STORED) as z:
        z.writestr("header.json", json.dumps(hdr))
        z.writestr(f"positions.3.{trx.pos_dtype.name}", np.ascontiguousarray(s._data[:nv]).tobytes())
        offs = np.concatenate([np.asarray(s._offsets[:n], dtype=np.uint64), [np.uint64(nv)]])
        z.writestr("offsets.uint64", offs.tobytes())


def load_trx(filename: str):
    """Read a TRX zip -> (header, ArraySequence in RAS mm)."""
    with zipfile.ZipFile(filename) as z:
        hdr = json.loads(z.read("header.json"))
        pos_name = [n for n in z.namelist() if n.startswith("positions.3.")][0]
        dt = np.dtype(pos_name.split(".")[-1])
        data = np.frombuffer(z.read(pos_name), dtype=dt).reshape(-1, 3)
        offs = np.frombuffer(z.read("offsets.uint64"), dtype=np.uint64).astype(np.int64)
    nv = hdr["NB_VERTICES"]
    offs = offs[:hdr["NB_STREAMLINES"]]  # drop the trailing NB_VERTICES sentinel
    lens = np.diff(np.concatenate([offs, [nv]]))
    return hdr, ArraySequence.from_flat(data, lens, offs)


# ----------------------------------------------------------------------------- TRK


def _aff2axcodes(aff):
    R = np.asarray(aff)[:3, :3]
    labels = (("L", "R"), ("P", "A"), ("I", "S"))
    codes = []
    for j in range(3):
        col = R[:, j]
        ax = int(np.argmax(np.abs(col)))
        codes.append(labels[ax][1] if col[ax] > 0 else labels[ax][0])
    return "".join(codes)


def save_trk(sft: StatefulTractogram, filename: str):
    """TrackVis v2 file from voxel-space streamlines (``save_tractogram`` for TRK)."""
    aff = sft.affine
    vox = np.sqrt((aff[:3, :3] ** 2).sum(0)).astype(np.float32)
    hdr = bytearray(1000)
    struct.pack_into("6s", hdr, 0, b"TRACK")
    struct.pack_into("<3h", hdr, 6, *[int(d) for d in sft.dimensions])
    struct.pack_into("<3f", hdr, 12, *vox)
    struct.pack_into("<16f", hdr, 440, *aff.astype(np.float32).ravel())
    struct.pack_into("4s", hdr, 948, _aff2axcodes(aff).encode())
    struct.pack_into("<i", hdr, 988, len(sft.streamlines))
    struct.pack_into("<i", hdr, 992, 2)
    struct.pack_into("<i", hdr, 996, 1000)
    s = sft.streamlines
    with open(filename, "wb") as f:
        f.write(hdr)
        for i in range(len(s)):
            pts = (np.asarray(s[i], dtype=np.float64) + 0.5) * vox
            f.write(struct.pack("<i", len(pts)))
            f.write(pts.astype("<f4").tobytes())


def load_trk(filename: str):
    """Read a TrackVis v2 file -> (header dict, ArraySequence in voxel coordinates)."""
    with open(filename, "rb") as f:
        raw = f.read()
    if raw[:5] != b"TRACK":
        raise ValueError("not a TRK file")
    dims = struct.unpack_from("<3h", raw, 6)
    vox = np.array(struct.unpack_from("<3f", raw, 12), dtype=np.float64)
    aff = np.array(struct.unpack_from("<16f", raw, 440), dtype=np.float64).reshape(4, 4)
    n = struct.unpack_from("<i", raw, 988)[0]
    pos = 1000
    items = []
    for _ in range(n):
        m = struct.unpack_from("<i", raw, pos)[0]
        pos += 4
        pts = np.frombuffer(raw, dtype="<f4", count=3 * m, offset=pos).reshape(m, 3)
        pos += 12 * m
        items.append((pts / vox - 0.5).astype(np.float32))
    return {"dimensions": dims, "voxel_sizes": vox, "vox_to_ras": aff, "n_count": n}, \
        ArraySequence(items)


def save_tractogram(sft: StatefulTractogram, filename: str):
    if filename.endswith(".trk"):
        return save_trk(sft, filename)
    raise ValueError("only .trk is supported by save_tractogram; use save_trx for .trx")


# ----------------------------------------------------------------------------- linearisation


def _compress_one(s, tol_error, max_segment_length):
    n = len(s)
    if n <= 2:
        return s.copy()
    keep = [0]
    start = 0
    i = 2
    tol2 = tol_error * tol_error
    while i < n:
        a = s[start]
        b = s[i]
        ab = b - a
        L = float(np.sqrt((ab * ab).sum()))
        ok = L <= max_segment_length
        if ok and i - start > 1:
            mid = s[start + 1:i] - a
            if L > 0:
                cr = np.cross(mid, ab / L)
                d2 = (cr * cr).sum(1)
            else:
                d2 = (mid * mid).sum(1)
            ok = bool((d2 <= tol2).all())
        if not ok:
            keep.append(i - 1)
            start = i - 1
        i += 1
    keep.append(n - 1)
    return s[keep]


def compress_streamlines(streamlines, tol_error=0.01, max_segment_length=10):
    """Linearise streamlines (Presseau et al. 2015): list of arrays in, list out."""
    return [_compress_one(np.asarray(s), tol_error, max_segment_length) for s in streamlines]
