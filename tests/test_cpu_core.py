"""CPU tests: oracle known answers, library loading/exports, host logic."""

from __future__ import annotations

import math
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden


# Philox4x32-10 known-answer vectors published with the Random123 library
# (Salmon et al., SC'11): (counter, key) -> output
PHILOX_KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


def test_oracle_philox_kat():
    from oracle import api

    for ctr, key, want in PHILOX_KAT:
        assert tuple(int(x) for x in api.philox_block(ctr, key)) == want
        # the same block through the stream layout: subsequence = high 64 counter
        # bits, offset = 4 x low 64 bits (when representable)
        lo = ctr[0] | (ctr[1] << 32)
        if 4 * lo < (1 << 64):
            got = api.philox_stream(key[0] | (key[1] << 32), ctr[2] | (ctr[3] << 32), 4 * lo, 4)
            assert tuple(int(x) for x in got) == want


def test_oracle_matches_curand_golden():
    from oracle import api

    for seed in (0, 1234):
        g = golden(f"curand_{seed}.npz")
        for q in range(len(g["subseq"])):
            s, o = int(g["subseq"][q]), int(g["offs"][q])
            assert np.array_equal(api.philox_stream(seed, s, o, 24), g["u32"][q])
            assert np.array_equal(api.philox_uniform(seed, s, o, 24), g["uniform"][q])


def test_sort_network_is_a_sorter():
    from oracle import api

    part = api.sort_partners()
    assert part.shape == (15, 32)
    for l in range(15):
        assert np.array_equal(part[l][part[l]], np.arange(32))  # involution
    rng = np.random.default_rng(0)
    for _ in range(200):
        k = rng.integers(0, 6, 32).astype(np.float32)
        v = np.arange(32)
        kk, vv = k.copy(), v.copy()
        for l in range(15):
            p = part[l]
            a, b = kk[p], vv[p]
            lower = np.arange(32) < p
            take = np.where(lower, a > kk, a < kk)
            kk = np.where(take, a, kk)
            vv = np.where(take, b, vv)
        assert np.all(np.diff(kk) <= 0)
        assert sorted(vv) == list(range(32))


def test_library_exports_every_header_symbol():
    from gpustreamlines_b200 import _lib

    hdr = open(os.path.join(ROOT, "include", "gpustreamlines_b200.h")).read()
    declared = set(re.findall(r"^\s*(?:int|const char \*)\s*(csl_\w+)\(", hdr, re.M))
    assert declared == set(_lib.EXPORTS)
    lib = _lib.load()
    for name in declared:
        assert hasattr(lib, name)
    assert b"sm_100a" in lib.csl_version()


def test_library_rejects_bad_arguments_without_gpu():
    from gpustreamlines_b200 import _lib

    lib = _lib.load()
    import ctypes as C

    h = C.c_void_p()
    rc = lib.csl_create(None, None, 0, C.byref(h))
    assert rc == _lib.CSL_E_INVALID
    assert "NULL" in _lib.last_error()
    assert lib.csl_counts(None, None, None) == _lib.CSL_E_INVALID
    # multi-subject plan and launch-shape calls validate before touching a device
    plan = C.c_void_p()
    assert lib.csl_multi_create(None, None, None, None, 0, 0, C.byref(plan)) == _lib.CSL_E_INVALID
    assert "subject" in _lib.last_error()
    assert lib.csl_multi_launch(None, None) == _lib.CSL_E_INVALID
    assert lib.csl_multi_wait(None, None, None, None, None) == _lib.CSL_E_INVALID
    assert lib.csl_multi_destroy(None) == _lib.CSL_OK
    assert lib.csl_set_launch(None, 128, 0) == _lib.CSL_E_INVALID
    assert lib.csl_autotune(None, None, 0, 0, 1, None) == _lib.CSL_E_INVALID


def test_tracker_validation_matches_reference_errors():
    from gpustreamlines_b200 import BootDirectionGetter, ProbDirectionGetter, Tracker
    from gpustreamlines_b200.sphere import get_sphere

    sph = get_sphere("repulsion724")
    data = np.zeros((4, 4, 4, 100), np.float32)
    with pytest.raises(ValueError, match="must match last dimension"):
        Tracker(ProbDirectionGetter(), data, np.zeros((4, 4, 4)), 0.1, sph.vertices, sph.edges)
    with pytest.raises(ValueError, match="Invalid model_type"):
        BootDirectionGetter("DTI", 1, *[np.zeros((2, 2))] * 5, np.zeros(3))


def test_shm_matrices_properties():
    from gpustreamlines_b200 import shm
    from gpustreamlines_b200.phantom import make_phantom
    from gpustreamlines_b200.sphere import get_sphere

    ph = make_phantom((8, 8, 8), seed=1, with_dwi=False)
    gt = ph.gtab
    sph = get_sphere("repulsion724")
    for order, ncoef in ((4, 15), (6, 28), (8, 45)):
        d = shm.prepare_csa(gt, sph, sh_order_max=order)
        H, R = d["H"], d["R"]
        assert H.shape == (150, 150) and d["delta_b"].shape == (ncoef, 150)
        assert d["sampling_matrix"].shape == (724, ncoef)
        assert np.allclose(H, H.T, atol=1e-10) and np.allclose(H @ H, H, atol=1e-8)
        assert np.allclose(np.trace(H), ncoef, atol=1e-6)
        assert np.allclose(R.mean(0), 0, atol=1e-12)
        o = shm.prepare_opdt(gt, sph, sh_order_max=order)
        assert o["delta_q"].shape == (ncoef, 150)
    assert d["b0s_mask"].sum() == 10


def test_sphere_is_antipodal_and_triangulated():
    from gpustreamlines_b200.sphere import get_sphere

    s = get_sphere("repulsion724")
    v = s.vertices
    assert v.shape == (724, 3) and s.edges.shape == (2166, 2)
    assert np.allclose(np.linalg.norm(v, axis=1), 1)
    assert np.allclose(v[:362], -v[362:])
    assert s.edges.min() >= 0 and s.edges.max() < 724


def test_phantom_is_deterministic():
    from gpustreamlines_b200.phantom import make_phantom, odf_volume, seeds_from_mask

    a = make_phantom((12, 14, 10), seed=3)
    b = make_phantom((12, 14, 10), seed=3)
    assert np.array_equal(a.dwi, b.dwi) and np.array_equal(a.fa, b.fa)
    o = odf_volume(a)
    assert o.shape == (12, 14, 10, 724) and o.min() >= 0
    s1 = seeds_from_mask(a.fa, 50, seed=2)
    s2 = seeds_from_mask(a.fa, 50, seed=2)
    assert np.array_equal(s1, s2)


def test_boot_fit_option_validation():
    """fit='bf16x3' is the batched tensor-core fit (CSA, OPDT); other names are rejected."""
    from gpustreamlines_b200 import BootDirectionGetter
    from oracle import cases

    inp = cases.inputs("csa_s")
    args = (inp["H"], inp["R"], inp["delta_b"], inp["delta_q"], inp["sampling_matrix"], inp["b0s_mask"])
    assert BootDirectionGetter("CSA", 1.0, *args, fit="bf16x3").fit == "bf16x3"
    assert BootDirectionGetter("CSA", 1.0, *args).fit == "fp32"
    assert BootDirectionGetter("OPDT", 1.0, *args, fit="bf16x3").fit == "bf16x3"
    with pytest.raises(ValueError):
        BootDirectionGetter("CSA", 1.0, *args, fit="tf32")


def test_mlp_oracle_gradient_matches_finite_differences():
    """The float64 restatement of the learned-proposal network (the checker of
    the CUDA training kernels) is itself pinned by central differences."""
    from oracle import mlp_ref

    rng = np.random.default_rng(0)
    n = sum(o * i + o for o, i in mlp_ref.SHAPES)
    p = rng.normal(size=n) * 0.1
    X = rng.normal(size=(8, 48))
    T = rng.normal(size=(8, 3))
    T /= np.linalg.norm(T, axis=1, keepdims=True)
    _, g = mlp_ref.grads(p, X, T)
    eps = 1e-6
    for k in rng.integers(0, n, 16):
        q = p.copy()
        q[k] += eps
        lp, _ = mlp_ref.grads(q, X, T)
        q[k] -= 2 * eps
        lm, _ = mlp_ref.grads(q, X, T)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-5 * abs(fd) + 1e-9
