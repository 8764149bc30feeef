"""Multi-subject CUDA-graph run (csl_multi_*) and launch-shape tuning
(csl_set_launch / csl_autotune) through the C ABI.

Bars, all bit-exact:
  * every subject's streamline lengths, seed indices and float32 points from
    the one-graph launch equal its own csl_propagate batch on the same seeds
    (mixed getters: probabilistic with two parameter sets, bootstrap CSA and
    OPDT with the per-warp FP32 fit and with the batched tensor-core fit, PTT;
    one empty subject);
  * the same on a second launch of the same graph, after seeds are rewritten
    in place, and when a pool far too small forces the plain-path re-run and
    a re-capture with grown capacities;
  * streamlines do not depend on the launch shape (threads per CTA, seed
    order), so every shape the tuner tries gives the same batch.
"""

from __future__ import annotations

import numpy as np
import pytest

from test_gpu_parity import _handle

pytestmark = pytest.mark.gpu

NAMES = ["prob_s", "csa_s", "ptt_s", "opdt_s", "prob_v", "prob_s", "csa_s", "opdt_s"]
COUNTS = [3000, 400, 300, 0, 1500, 700, 600, 500]
KW = [{}, {}, {}, {}, {}, {}, {"boot_fit": 1}, {"boot_fit": 1}]


def _handles():
    return [_handle(n, **kw) for n, kw in zip(NAMES, KW)]


def _dev(seeds):
    import torch

    t = torch.zeros((max(len(seeds), 1), 3), dtype=torch.float32, device="cuda")
    if len(seeds):
        t[: len(seeds)].copy_(torch.from_numpy(np.ascontiguousarray(seeds, np.float32)))
    return t


def _seeds(seed_base):
    from oracle import cases

    return [cases.seeds(n, max(c, 1), seed=seed_base + i)[:c] for i, (n, c) in enumerate(zip(NAMES, COUNTS))]


def _plain(handles, seeds):
    out = []
    for h, s in zip(handles, seeds):
        h.propagate(s)
        out.append(h.fetch())
    return out


def _check(plan, handles, ref):
    nsl, npts, rep, ms = plan.wait()
    assert ms > 0
    for i, h in enumerate(handles):
        got = h.fetch()
        assert nsl[i] == len(ref[i][0]) and npts[i] == len(ref[i][2]), i
        for a, b in zip(got, ref[i]):
            assert np.array_equal(a, b), i
    return rep


def test_multi_subject_graph_matches_plain_batches():
    import torch

    from gpustreamlines_b200 import _lib

    handles = _handles()
    try:
        seeds = _seeds(21)
        dev = [_dev(s) for s in seeds]
        torch.cuda.synchronize()
        plan = _lib.MultiPlan(handles, [d.data_ptr() for d in dev], COUNTS)
        try:
            # the plan's own launches come first: nothing has been tracked yet
            plan.launch()
            ref = None
            nsl, npts, rep, _ = plan.wait()
            got = [h.fetch() for h in handles]
            ref = _plain(handles, seeds)
            for i in range(len(handles)):
                for a, b in zip(got[i], ref[i]):
                    assert np.array_equal(a, b), i
            assert sum(len(r[0]) for r in ref) > 1000
            # second launch of the same graph (the plain batches above left the
            # buffers in place or grew them; either way the results must match)
            plan.launch()
            _check(plan, handles, ref)
            # seeds rewritten in place
            new = _seeds(77)
            for d, s in zip(dev, new):
                if len(s):
                    d[: len(s)].copy_(torch.from_numpy(s))
            torch.cuda.synchronize()
            ref2 = _plain(handles, new)
            plan.launch()
            rep = _check(plan, handles, ref2)
            plan.launch()
            rep = _check(plan, handles, ref2)
            assert not rep.any()
            # any limit on concurrent tracking kernels (0: none) gives the same batches
            for k in (0, 2, 5):
                plan.set_concurrency(k)
                plan.launch()
                _check(plan, handles, ref2)
        finally:
            plan.close()
    finally:
        for h in handles:
            h.close()


def test_multi_subject_pool_overflow_reruns_and_recaptures():
    import torch

    from gpustreamlines_b200 import _lib

    handles = _handles()
    try:
        seeds = _seeds(31)
        dev = [_dev(s) for s in seeds]
        torch.cuda.synchronize()
        ref = _plain(handles, seeds)
        # one point per streamline: every non-empty subject overflows its pool
        plan = _lib.MultiPlan(handles, [d.data_ptr() for d in dev], COUNTS, points_per_streamline=1)
        try:
            plan.launch()
            rep = _check(plan, handles, ref)
            assert all(rep[i] == (1 if COUNTS[i] else 0) for i in range(len(NAMES)))
            cap0, _, pool = plan.info()
            assert all(pool[i] >= len(ref[i][2]) for i in range(len(NAMES)) if COUNTS[i])
            plan.launch()
            rep = _check(plan, handles, ref)
            assert not rep.any()
            cap1, _, _ = plan.info()
            assert cap1 == cap0 + 1
        finally:
            plan.close()
    finally:
        for h in handles:
            h.close()


def test_multi_subject_validation():
    import torch

    from gpustreamlines_b200 import _lib

    h = _handle("prob_s")
    try:
        d = _dev(np.zeros((4, 3), np.float32) + 10)
        torch.cuda.synchronize()
        with pytest.raises(ValueError):
            _lib.MultiPlan([h, h], [d.data_ptr(), d.data_ptr()], [4, 4])
        with pytest.raises(ValueError):
            _lib.MultiPlan([h], [0], [4])
        plan = _lib.MultiPlan([h], [d.data_ptr()], [4])
        try:
            with pytest.raises(RuntimeError):
                plan.wait()
            plan.launch()
            with pytest.raises(RuntimeError):
                plan.launch()
            plan.wait()
        finally:
            plan.close()
    finally:
        h.close()


@pytest.mark.parametrize("name,n", [("prob_s", 2000), ("ptt_s", 300), ("csa_s", 200)])
def test_launch_shapes_do_not_change_streamlines(name, n):
    import torch

    from oracle import cases

    seeds = cases.seeds(name, n, seed=41)
    h = _handle(name)
    try:
        h.propagate(seeds)
        ref = h.fetch()
        for block in (256, 128, 64):
            for order in (0, 1):
                try:
                    h.set_launch(block, order)
                except ValueError:  # the CTA's shared memory does not fit at this size
                    assert block == 256
                    continue
                assert h.get_launch()[:2] == (block, order)
                h.propagate(seeds)
                for a, b in zip(h.fetch(), ref):
                    assert np.array_equal(a, b), (block, order)
        d = _dev(seeds)
        torch.cuda.synchronize()
        ms = h.autotune(d.data_ptr(), n, 0, repeats=1)
        assert len(ms) == 6 and any(v is not None for v in ms.values())
        best = h.get_launch()[:2]
        assert ms[best] is not None and ms[best] == min(v for v in ms.values() if v is not None)
        for a, b in zip(h.fetch(), ref):
            assert np.array_equal(a, b)
        with pytest.raises(ValueError):
            h.set_launch(96, 0)
    finally:
        h.close()


def test_tracker_autotune_then_multi_subject_run():
    """The reference-style API end to end: trackers tuned on their seeds, then
    a MultiSubjectRun whose streamlines equal each tracker's own batch."""
    import math

    from gpustreamlines_b200 import ProbDirectionGetter, Tracker
    from gpustreamlines_b200.multi import MultiSubjectRun
    from oracle import cases

    inp = cases.inputs("prob_s")
    c = inp["case"]
    trs, seeds = [], []
    for k, n in enumerate((1500, 400)):
        tr = Tracker(ProbDirectionGetter(), inp["dataf"], inp["stop_map"], c["fa_thr"], inp["vertices"],
                     inp["edges"], max_angle=math.radians(c["max_angle"]), step_size=c["step"])
        tr.__enter__()
        trs.append(tr)
        seeds.append(cases.seeds("prob_s", n, seed=50 + k))
    try:
        ref = []
        for tr, s in zip(trs, seeds):
            tr.handles[0].propagate(s)
            ref.append(tr.handles[0].fetch())
        (ms, shape), = trs[0].autotune(seeds[0], sample=1000, repeats=1)
        assert ms[shape] is not None
        with MultiSubjectRun(trs, seeds) as run:
            nsl, npts, rep, _ = run.run()
            for i in range(2):
                for a, b in zip(run.results(i), ref[i]):
                    assert np.array_equal(a, b)
                assert len(run.streamlines(i)) == len(ref[i][0])
    finally:
        for tr in trs:
            tr.__exit__(None, None, None)
