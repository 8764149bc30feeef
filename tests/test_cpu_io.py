"""CPU tests of the writers and the chunk/propagator host logic."""

from __future__ import annotations

import numpy as np

from gpustreamlines_b200 import io


def _sls(rng, n=20):
    return [rng.normal(size=(int(rng.integers(1, 40)), 3)).astype(np.float32) * 5 + 20 for _ in range(n)]


def test_trx_roundtrip(tmp_path):
    rng = np.random.default_rng(0)
    aff = np.diag([2.0, 2.0, 2.0, 1.0])
    aff[:3, 3] = [-80, -100, -60]
    ref = io.RefImage(aff, (81, 106, 76))
    trx = io.TrxFile(nb_streamlines=4, nb_vertices=10, init_as=io.TrxFile(reference=ref))
    allsl = []
    for _ in range(3):  # several chunks -> exercises the doubling resize
        s = _sls(rng)
        allsl += s
        trx.append_block(np.concatenate(s), np.array([len(x) for x in s]))
    trx.resize()
    f = str(tmp_path / "a.trx")
    io.save_trx(trx, f)
    hdr, seq = io.load_trx(f)
    assert hdr["NB_STREAMLINES"] == len(allsl)
    assert hdr["NB_VERTICES"] == sum(len(x) for x in allsl)
    assert hdr["DIMENSIONS"] == [81, 106, 76]
    for a, b in zip(seq, allsl):
        assert np.array_equal(a, b)


def test_trk_roundtrip(tmp_path):
    rng = np.random.default_rng(1)
    s = _sls(rng)
    aff = np.diag([2.0, 2.0, 2.0, 1.0])
    sft = io.StatefulTractogram(io.ArraySequence(s), io.RefImage(aff, (30, 30, 30)), io.Space.VOX)
    f = str(tmp_path / "a.trk")
    io.save_tractogram(sft, f)
    hdr, seq = io.load_trk(f)
    assert hdr["n_count"] == len(s)
    for a, b in zip(seq, s):
        assert np.allclose(a, b, atol=1e-5)


def test_to_world_applies_affine():
    aff = np.array([[2, 0, 0, -10], [0, 3, 0, 5], [0, 0, 1, 1], [0, 0, 0, 1]], float)
    seq = io.ArraySequence([np.array([[1, 2, 3]], np.float32)])
    io.Tractogram(seq, affine_to_rasmm=aff).to_world()
    assert np.allclose(seq[0], [[-8, 11, 4]])


def test_compress_streamlines_properties():
    rng = np.random.default_rng(2)
    t = np.linspace(0, 1, 200)[:, None]
    line = np.hstack([t * 50, t * 10, t * 0]).astype(np.float64)
    c = io.compress_streamlines([line], tol_error=0.01, max_segment_length=100)[0]
    assert len(c) == 2 and np.array_equal(c[0], line[0]) and np.array_equal(c[-1], line[-1])
    wavy = np.hstack([t * 50, np.sin(t * 20), t * 0])
    c = io.compress_streamlines([wavy], tol_error=0.1, max_segment_length=10)[0]
    assert 2 < len(c) < len(wavy)
    assert np.all(np.linalg.norm(np.diff(c, axis=0), axis=1) <= 10 + 1e-9)
    # every dropped point lies within tol of the kept polyline
    for p in wavy:
        d = min(_seg_dist(p, a, b) for a, b in zip(c[:-1], c[1:]))
        assert d <= 0.1 + 1e-9


def _seg_dist(p, a, b):
    ab = b - a
    t = np.clip(np.dot(p - a, ab) / max(np.dot(ab, ab), 1e-12), 0, 1)
    return np.linalg.norm(p - (a + t * ab))


class _FakeHandle:
    """Host-side stand-in for one GPU's tracker handle (no GPU needed)."""

    def __init__(self, dev):
        self.dev = dev

    def propagate(self, seeds, rng_index_base=0):
        self.n = len(seeds)
        self.seeds = np.asarray(seeds)

    def fetch(self):
        L = np.array([2 + (i % 3) for i in range(2 * self.n)], np.int32)
        S = np.repeat(np.arange(self.n), 2).astype(np.int32)
        P = np.concatenate([np.full((l, 3), self.dev * 1000 + s, np.float32) for l, s in zip(L, S)]) \
            if len(L) else np.zeros((0, 3), np.float32)
        return L, S, P


class _FakeTracker:
    def __init__(self, ngpus):
        self.ngpus = ngpus
        self.handles = [_FakeHandle(i) for i in range(ngpus)]
        self._allocated = True
        self.rng_offset = 0
        self.chunk_size = 7


def test_propagator_shards_contiguously_and_filters():
    from gpustreamlines_b200.propagate import SeedBatchPropagator

    t = _FakeTracker(3)
    sp = SeedBatchPropagator(t, minlen=3, maxlen=3)
    seeds = np.arange(3 * 10, dtype=np.float32).reshape(10, 3)
    sp.propagate(seeds)
    # ceil(10/3) = 4 seeds per GPU: 4, 4, 2
    assert [h.n for h in t.handles] == [4, 4, 2]
    assert list(sp.nSlines) == [8, 8, 4]
    got = list(sp.as_generator())
    assert all(len(g) == 3 for g in got)
    a = sp.as_array_sequence()
    assert len(a) == len(got) and all(np.array_equal(x, y) for x, y in zip(a, got))
    assert t.rng_offset == 10


def test_generate_trx_chunks(tmp_path):
    from gpustreamlines_b200.generic_tracker import GenericTracker
    from gpustreamlines_b200.propagate import SeedBatchPropagator

    class T(GenericTracker):
        pass

    tr = T()
    ft = _FakeTracker(2)
    tr.ngpus, tr.chunk_size = 2, 3
    tr.seed_propagator = SeedBatchPropagator(ft)
    seeds = np.zeros((13, 3), np.float32)
    ref = io.RefImage(np.eye(4), (10, 10, 10))
    trx = tr.generate_trx(seeds, ref)
    assert len(trx) == 26  # two streamlines per seed
    f = str(tmp_path / "x.trx")
    io.save_trx(trx, f)
    hdr, seq = io.load_trx(f)
    assert hdr["NB_STREAMLINES"] == 26
    sft = tr.generate_sft(seeds, ref)
    assert len(sft) == 26
