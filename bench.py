"""Benchmark: tracking steps/s of the probabilistic getter at 1M seeds on B200.

Workload (one "step" = one pass of the tracking path over one batch): the
probabilistic direction getter on the synthetic 81x106x76 phantom with its
float32 PMF volume of 724 sphere vertices (1.9 GB), 1,000,000 seeds per GPU
drawn from the FA > 0.3 mask, step 0.5 voxel, max angle 45 deg, stop at
FA < 0.1, at most 501 points per direction.  A tracking step is one accepted
direction + position update: steps = sum over streamlines of (length - 1).

  value   device-timed (CUDA events on the library's stream) pass 1 + scans +
          pass 2 + compaction with the seeds already resident in HBM
  e2e     the same work through the C ABI with host buffers: H2D of the
          seeds and D2H of lengths, seed ids and points inside the timed region
  reference arm (--impl reference): the CPU restatement of the reference
          algorithm on all host threads, on a bounded sample of the same seeds

Supplementary lines (not the headline): --getter (the other getters on the
same phantom), --odf-volume (ODF/PMF volume generation), --learned (learned
proposal), --multi (uneven subjects with mixed getters in one CUDA-graph
launch against the same batches tracked one after another), --autotune (the
launch-shape tuner's timings on the workload's seeds).

Multi-GPU (torchrun): one process per GPU; each rank tracks its own 1M seeds
(weak scaling, no data exchange); per-rank times are reduced with MAX and the
per-rank streamline/point counts are all-gathered (the offsets a global TRX
file needs).  Inputs (1.9 GB PMF) exceed the 126 MB L2, so no flush is needed.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "tracking steps/s on 1 B200, learned+BF16 form vs plain FP32 kernel, 1M seeds"
BYTES_PER_STEP = 8 * 724 * 4 + 8 * 4 + 12  # PMF corners + stop-map taps + point write
# DRAM bytes (read + write) per tracking step of track_kernel<PROB>, from one ncu
# capture of this workload at 20,000 seeds (27.25 GB over 6,372,721 steps, see
# profiles/track_kernel_prob_81x106x76x724.md); scaled to a full launch by steps.
TRAFFIC_BYTES_PER_STEP = 4277.0
# The same for track_kernel<PROB_ENV> (envelope sampler, four draws per round):
# 9.83 GB over 6,349,590 steps at 20,000 seeds
# (profiles/track_kernel_prob_env_81x106x76x724.md).
ENV_TRAFFIC_BYTES_PER_STEP = 1547.4


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seeds", type=int, default=1_000_000)
    ap.add_argument("--odf-volume", action="store_true",
                    help="time the GPU ODF/PMF volume generation (SH coefficients -> clipped ODF) instead")
    ap.add_argument("--multi", action="store_true",
                    help="multi-subject run: uneven subjects, mixed getters, one CUDA-graph launch")
    ap.add_argument("--subjects", type=int, default=12)
    ap.add_argument("--multi-boot-fit", choices=("fp32", "bf16x3"), default="fp32",
                    help="bootstrap subjects of --multi: per-warp FP32 fit or the batched tensor-core fit")
    ap.add_argument("--autotune", action="store_true",
                    help="print the launch-shape tuner's timings on this workload's seeds and exit")
    ap.add_argument("--learned", action="store_true",
                    help="train and evaluate the learned vMF-mixture proposal instead")
    ap.add_argument("--getter", default="prob_env", choices=sorted(GETTERS),
                    help="prob_env = the headline (envelope sampler, with the plain FP32 kernel timed "
                         "beside it); prob/csa/opdt/ptt/... print supplementary lines")
    ap.add_argument("--boot-compare", action="store_true",
                    help="bootstrap CSA sh 8 at --seeds: batched BF16x3 tensor-core fit and per-warp FP32 fit "
                         "timed in the same run (one JSON line)")
    ap.add_argument("--no-plain-arm", action="store_true",
                    help="headline only: skip timing the plain FP32 inverse-CDF kernel beside it")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--env-traffic-bytes-per-step", type=float, default=ENV_TRAFFIC_BYTES_PER_STEP,
                    help="DRAM bytes per step of the envelope-sampler kernel from an ncu capture (0 = unknown)")
    ap.add_argument("--traffic-bytes-per-step", type=float, default=TRAFFIC_BYTES_PER_STEP,
                    help="DRAM bytes per tracking step from an ncu capture (0 = unknown)")
    return ap.parse_args()


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


GETTERS = {
    # the headline workload: probabilistic getter with the bounded-envelope
    # proposal (bf16 cluster-maxima table, exact accept/reject against the FP32
    # PMF); the plain FP32 inverse-CDF kernel is timed beside it in the same run
    "prob_env": dict(model="PROB", max_angle=45.0, sampler="envelope",
                     label="prob getter, bounded-envelope proposal (bf16 cluster-maxima table) with exact FP32 "
                           "PMF accept/reject, vs the plain FP32 inverse-CDF kernel; 81x106x76 PMF x 724 "
                           "vertices (1.9 GB)"),
    # the plain FP32 kernel alone (the reference's sampler, bit-exact to it)
    "prob": dict(model="PROB", max_angle=45.0,
                 label="prob getter (plain FP32 inverse CDF), 81x106x76 PMF x 724 vertices (1.9 GB)"),
    # supplementary lines (not the headline): the other getters on the same phantom
    "csa": dict(model="CSA", max_angle=60.0, sh_order=8,
                label="bootstrap CSA getter (plain FP32), sh_order 8 (45 coeffs), 81x106x76x160 DWI"),
    "csa_bf16x3": dict(model="CSA", max_angle=60.0, sh_order=8, fit="bf16x3",
                       label="bootstrap CSA getter, batched tensor-core fit (BF16x3, FP32 accumulate), "
                             "sh_order 8 (45 coeffs), 81x106x76x160 DWI"),
    "opdt": dict(model="OPDT", max_angle=60.0, sh_order=6,
                 label="bootstrap OPDT getter (plain FP32), sh_order 6 (28 coeffs), 81x106x76x160 DWI"),
    "opdt_bf16x3": dict(model="OPDT", max_angle=60.0, sh_order=6, fit="bf16x3",
                        label="bootstrap OPDT getter, batched tensor-core fit (BF16x3, FP32 accumulate), "
                              "sh_order 6 (28 coeffs), 81x106x76x160 DWI"),
    "ptt": dict(model="PTT", max_angle=60.0,
                label="PTT getter, 81x106x76 ODF x 724 vertices (tiled texture), step 0.5 = 20 sub-steps"),
}


def build_workload(rank: int, nseeds: int, getter: str = "prob"):
    from gpustreamlines_b200.phantom import make_phantom, odf_volume, seeds_from_mask
    from gpustreamlines_b200.sphere import get_sphere

    ph = make_phantom((81, 106, 76), seed=1234)
    sph = get_sphere("repulsion724")
    if GETTERS[getter]["model"] in ("CSA", "OPDT"):
        data = np.ascontiguousarray(ph.dwi, dtype=np.float32)
    else:
        data = odf_volume(ph, sph)
    seeds = seeds_from_mask(ph.fa, nseeds, threshold=0.3, seed=1000 + rank).astype(np.float32)
    return ph, sph, data, seeds


def make_getter(getter: str, ph, sph):
    from gpustreamlines_b200 import BootDirectionGetter, ProbDirectionGetter, PttDirectionGetter

    g = GETTERS[getter]
    if g["model"] == "CSA":
        return BootDirectionGetter.from_dipy_csa(ph.gtab, sph, sh_order_max=g["sh_order"],
                                                 fit=g.get("fit", "fp32"))
    if g["model"] == "OPDT":
        return BootDirectionGetter.from_dipy_opdt(ph.gtab, sph, sh_order_max=g["sh_order"],
                                                  fit=g.get("fit", "fp32"))
    if g["model"] == "PTT":
        return PttDirectionGetter()
    return ProbDirectionGetter(sampler=g.get("sampler", "inverse_cdf"))


def plain_arm(args, data, ph, sph, gcfg, seeds_d, local, stream, barrier, dist, world):
    """The plain FP32 inverse-CDF kernel on the same PMF and seeds, timed the same
    way (device-resident seeds, pass 1 + pass 2 + compaction, max over ranks)."""
    import torch

    from gpustreamlines_b200 import ProbDirectionGetter, Tracker

    with Tracker(ProbDirectionGetter(), data, ph.fa, 0.1, sph.vertices, sph.edges,
                 max_angle=math.radians(gcfg["max_angle"]), step_size=0.5, ngpus=1, device_offset=local) as tr:
        hp = tr.handles[0]
        n = int(seeds_d.shape[0])
        for _ in range(max(1, min(args.warmup, 2))):
            hp.propagate_device(seeds_d.data_ptr(), n, 0, stream.cuda_stream)
        nsl, npts = hp.counts()
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        p2 = []
        e0.record(stream)
        for _ in range(args.steps):
            hp.propagate_device(seeds_d.data_ptr(), n, 0, stream.cuda_stream)
            p2.append(hp.timings()[0][2])
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        steps = float(npts - nsl)
        if dist is not None:
            t = torch.tensor([ms, steps], device=f"cuda:{local}", dtype=torch.float64)
            mx = t[:1].clone()
            dist.all_reduce(mx, op=dist.ReduceOp.MAX)
            sm = t[1:].clone()
            dist.all_reduce(sm)
            ms, steps = float(mx.item()), float(sm.item())
        return {"value": steps * args.steps / (ms / 1e3), "unit": "steps/s", "ms_per_step": ms / args.steps,
                "pass2_ms": float(np.mean(p2)), "streamlines_per_gpu": int(nsl), "steps_per_gpu": int(npts - nsl),
                "kernel": "track_kernel<PROB> (inverse CDF over the gathered PMF, the reference's sampler)"}


def run_boot_compare(args):
    """Bootstrap CSA (sh_order 8, 45 coefficients, 81x106x76x160 DWI) at --seeds,
    three pass-2 forms in one run: the batched BF16x3 tensor-core fit with the
    float64 re-fit of near-tie rows (boot_fit 1, the default batched form), the
    same without the re-fit (boot_fit 2), and the per-warp FP32 fit (the
    reference's arithmetic).  Each is timed device-resident (pass 1 + pass 2 +
    compaction) after one untimed batch of the same seeds (which sizes the point
    pool), with the tensor roofline of the batched fit and its re-fit counts."""
    from gpustreamlines_b200 import _lib, Tracker, BootDirectionGetter

    ph, sph, data, seeds = build_workload(0, args.seeds, "csa_bf16x3")
    d = _lib.DeviceBuffer.from_array(seeds, 0)
    out = {}
    for fit in ("bf16x3", "bf16x3_fp64", "fp32"):
        dg = BootDirectionGetter.from_dipy_csa(ph.gtab, sph, sh_order_max=8, fit=fit)
        with Tracker(dg, data, ph.fa, 0.1, sph.vertices, sph.edges, max_angle=math.radians(60), step_size=0.5) as tr:
            h = tr.handles[0]
            h.propagate_device(d.ptr, len(seeds), 0, None)
            if fit != "fp32":
                h.boot_refit_stats(reset=True)
            reps = args.steps if fit != "fp32" else 1
            with ClockSampler(0) as clk:
                t0 = time.perf_counter()
                ms = []
                for _ in range(reps):
                    h.propagate_device(d.ptr, len(seeds), 0, None)
                    (p1, gap, p2, cp), _ = h.timings()
                    ms.append((p1 + gap + p2 + cp, p2))
                wall = time.perf_counter() - t0
            nsl, npts = h.counts()
            tot = float(np.mean([m[0] for m in ms]))
            p2 = float(np.mean([m[1] for m in ms]))
            out[fit] = {"steps": int(npts - nsl), "streamlines": int(nsl), "batch_ms": tot, "pass2_ms": p2,
                        "steps_per_s": (npts - nsl) / (tot / 1e3), "batches": reps, "wall_s": wall,
                        "clocks": clk.summary()}
            if fit != "fp32":
                st = h.boot_refit_stats()
                out[fit]["rows_searched"] = st["rows"]
                out[fit]["rows_fitted_again_fp64"] = st["refit"]
                nc = dg.delta_nr
                hr = int((dg.b0s_mask == 0).sum())
                flop = 2 * 2 * hr * hr + 2 * nc * hr + 2 * nc * dg.sampling_matrix.shape[0]
                with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
                    tpeak = float(json.load(f)["bf16_tflops"])
                tach = (npts - nsl) * flop / (p2 / 1e3) / 1e12
                out[fit]["roofline"] = {"bound": "tensor", "achieved": tach, "peak": tpeak, "unit": "TFLOP/s",
                                        "frac": tach / tpeak, "algorithmic_flop_per_step": flop,
                                        "issued_bf16_flop_per_step": 3 * flop,
                                        "peak_source": "measured MEASURED_PEAKS bf16_tflops"}
    print(json.dumps({"workload": f"bootstrap CSA getter, sh_order 8 (45 coeffs), 81x106x76x160 DWI, {args.seeds} seeds, "
                                  "step 0.5, max angle 60", "batched_bf16x3": out["bf16x3"],
                      "batched_bf16x3_fp64_refit": out["bf16x3_fp64"], "per_warp_fp32": out["fp32"],
                      "speedup_bf16x3_vs_fp32": out["bf16x3"]["steps_per_s"] / out["fp32"]["steps_per_s"]}),
          flush=True)
    return 0


def measured_peaks():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


def cpu_baseline(ph, sph, data, seeds, seconds: float, threads: int | None = None,
                 getter: str = "prob", dg=None):
    """The oracle (CPU restatement of the reference) on a bounded seed sample."""
    import math as _m

    from oracle import api

    g = GETTERS[getter]
    threads = threads or os.cpu_count() or 1
    inp = dict(case=dict(model=g["model"], step=0.5, max_angle=g["max_angle"], fa_thr=0.1, rel=0.25,
                         min_sep=45.0, rng_seed=0),
               dataf=data, stop_map=np.ascontiguousarray(ph.fa, dtype=np.float32),
               vertices=np.ascontiguousarray(sph.vertices, dtype=np.float32),
               edges=np.ascontiguousarray(sph.edges, dtype=np.int32))
    if g["model"] in ("CSA", "OPDT"):
        for k in ("H", "R", "delta_b", "delta_q", "sampling_matrix", "b0s_mask", "min_signal"):
            inp[k] = getattr(dg, k)
    ptt = None
    if g["model"] == "PTT":
        from gpustreamlines_b200.direction_getters import PttDirectionGetter

        pg = PttDirectionGetter()
        tiled = pg.prepare_data_host(np.array(data, copy=True), inp["stop_map"], np.float32(0.1), inp["vertices"], False)
        ptt = dict(tiled=tiled, lut=pg.sphere_vertices_lut_h, log2_x=pg.log2_x, log2_y=pg.log2_y,
                   nx=pg.nx, ny=pg.ny, nz=pg.nz, res=pg.odf_lut_res)
    ang = np.float32(_m.radians(g["max_angle"]))
    o = api.Oracle(inp, cos_max_angle=np.float32(_m.cos(ang)), ptt=ptt)
    n = {"PROB": 256, "PTT": 16}.get(g["model"], 64)
    steps = 0
    elapsed = 0.0
    used = 0
    while True:
        batch = seeds[used:used + n]
        t0 = time.perf_counter()
        _, lens, _, _ = o.track(batch, threads=threads)
        dt = time.perf_counter() - t0
        steps += int((lens - 1).sum())
        elapsed += dt
        used += len(batch)
        if elapsed >= seconds or used >= len(seeds):
            break
        rate = used / max(elapsed, 1e-9)
        n = int(min(max(64, rate * (seconds - elapsed)), len(seeds) - used))
    return dict(value=steps / elapsed, unit="steps/s", cores=threads, kind="port",
                sample=f"{used} of the benchmark's seeds ({steps} steps, {elapsed:.1f} s)")


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    ph, sph, data, seeds = build_workload(0, args.seeds, args.getter)
    dg = make_getter(args.getter, ph, sph)
    threads = os.cpu_count() or 1
    per = args.cpu_seconds / max(args.steps + args.warmup, 1)
    vals = []
    for i in range(args.warmup + args.steps):
        sub = seeds[(i * 997) % max(len(seeds) - 50_000, 1):]
        r = cpu_baseline(ph, sph, data, sub, max(per, 2.0), threads, args.getter, dg)
        if i >= args.warmup:
            vals.append(r)
    v = float(np.mean([r["value"] for r in vals]))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic phantom (Stanford HARDI shapes)",
            "config": {"workload": f"{GETTERS[args.getter]['label']}, {args.seeds} seeds "
                                   "(bounded CPU sample per step)", "seeds": args.seeds},
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": threads, "kind": "port",
                             "sample": "; ".join(r["sample"] for r in vals)},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


class _DeviceArray:
    """A DeviceBuffer seen as a CUDA array argument (used in place, not copied)."""

    is_cuda = True

    def __init__(self, buf):
        self.buf = buf
        self.shape = buf.shape
        self.dtype = buf.dtype

    def data_ptr(self):
        return self.buf.ptr

    def is_contiguous(self):
        return True


def run_odf_volume(args):
    """GPU ODF/PMF volume generation on the benchmark phantom (81x106x76 voxels,
    sh_order 8 -> 724 vertices, 1.9 GB written) against the host evaluation."""
    from gpustreamlines_b200 import _lib, shm
    from gpustreamlines_b200.odf import odf_volume_gpu
    from gpustreamlines_b200.phantom import make_phantom
    from gpustreamlines_b200.sphere import get_sphere

    ph = make_phantom((81, 106, 76), seed=1234, with_dwi=False)
    sph = get_sphere("repulsion724")
    B, _, _ = shm.real_sh_descoteaux(ph.meta["sh_order"], sph.theta, sph.phi)
    B = np.ascontiguousarray(B, dtype=np.float32)
    coef = _lib.DeviceBuffer.from_array(np.ascontiguousarray(ph.sh_coef, dtype=np.float32), 0)
    dev_coef = _DeviceArray(coef)
    ms = []
    out = None
    for i in range(args.warmup + args.steps):
        if out is not None:
            out.close()
        out, m = odf_volume_gpu(dev_coef, B, return_ms=True)
        if i >= args.warmup:
            ms.append(m)
    nvox, V, C = int(np.prod(ph.shape)), B.shape[0], B.shape[1]
    t_kernel = float(np.median(ms)) / 1e3
    written = nvox * V * 4
    peak, kind = measured_peaks()
    t0 = time.perf_counter()
    c2 = ph.sh_coef.reshape(-1, C).astype(np.float32)
    host = np.maximum(c2[: nvox // 8] @ B.T, 0)
    t_host = (time.perf_counter() - t0) * 8
    rows = np.nonzero(np.abs(c2).max(axis=1) > 0)[0][:: max(1, nvox // 20000)][:20000]
    ref = np.maximum(c2[rows] @ B.T, 0)
    got = out.numpy().reshape(-1, V)[rows]
    err = float((np.abs(got - ref).max(axis=1) / np.maximum(np.abs(ref).max(axis=1), 1e-20)).max())
    print(json.dumps({"workload": "ODF/PMF volume from SH (81x106x76 voxels, 45 coeffs -> 724 vertices, clipped)",
                      "kernel_ms": t_kernel * 1e3, "voxels_per_s": nvox / t_kernel,
                      "roofline": {"bound": "hbm", "achieved": (written + nvox * C * 4) / t_kernel / 1e9,
                                   "peak": peak, "unit": "GB/s",
                                   "frac": (written + nvox * C * 4) / t_kernel / 1e9 / peak,
                                   "peak_source": f"{kind} MEASURED_PEAKS hbm_gbs"},
                      "host_numpy_s": t_host, "speedup_vs_host": t_host / t_kernel,
                      "max_rel_err_vs_host_f32": err, "rows_checked": int(len(rows)), "dtype": "bf16x3 -> f32"}), flush=True)
    del host
    return 0


def multi_subjects(nsub: int, seed: int = 5, boot_fit: str = "fp32"):
    """Uneven synthetic subjects for the multi-subject run: volumes log-uniform
    between 48^3 and 96x116x96 voxels (phantom shape scaled), two diffusion
    schemes (6 b0 + 64 dirs at b=1000, 2.5 mm; 10 b0 + 150 dirs at b=2000,
    2 mm), seeds log-uniform in [5k, 250k] (1/25 of that, at least 1000,
    for bootstrap and PTT subjects, whose steps cost 40-120x a probabilistic
    step), getters
    cycling probabilistic, bootstrap CSA, PTT, probabilistic, bootstrap OPDT,
    probabilistic.  boot_fit "bf16x3" gives the bootstrap subjects the batched
    tensor-core fit (same subjects and seeds)."""
    rng = np.random.default_rng(seed)
    b = "_bf16x3" if boot_fit == "bf16x3" else ""
    cycle = ["prob", "csa" + b, "ptt", "prob", "opdt" + b, "prob"]
    vox = np.exp(rng.uniform(np.log(48 ** 3), np.log(96 * 116 * 96), nsub))
    nseeds = np.exp(rng.uniform(np.log(5_000), np.log(250_000), nsub)).astype(int)
    out = []
    for i in range(nsub):
        scale = (vox[i] / (81 * 106 * 76)) ** (1 / 3)
        shape = tuple(max(24, int(round(d * scale))) for d in (81, 106, 76))
        n_b0, n_dirs, bval, mm = [(6, 64, 1000.0, 2.5), (10, 150, 2000.0, 2.0)][i % 2]
        getter = cycle[i % len(cycle)]
        n = int(nseeds[i]) if getter == "prob" else max(1000, int(nseeds[i]) // 25)
        out.append(dict(getter=getter, shape=shape, n_b0=n_b0, n_dirs=n_dirs, bval=bval,
                        voxel_mm=mm, seeds=n, seed=100 + i))
    return out


def run_multi(args):
    """All subjects' batches as one captured CUDA graph (MultiSubjectRun)
    against the same batches tracked one after another through the plain
    per-subject path (host round trips between pass 1, pass 2 and compaction)."""
    import torch

    from gpustreamlines_b200 import Tracker
    from gpustreamlines_b200.multi import MultiSubjectRun
    from gpustreamlines_b200.phantom import make_phantom, odf_volume, seeds_from_mask
    from gpustreamlines_b200.sphere import get_sphere

    sph = get_sphere("repulsion724")
    subs = multi_subjects(args.subjects, boot_fit=args.multi_boot_fit)
    trackers, seeds, vol_bytes = [], [], 0
    t_setup = time.perf_counter()
    for sd in subs:
        g = GETTERS[sd["getter"]]
        boot = g["model"] in ("CSA", "OPDT")
        ph = make_phantom(sd["shape"], seed=sd["seed"], n_b0=sd["n_b0"], n_dirs=sd["n_dirs"], bval=sd["bval"],
                          voxel_mm=sd["voxel_mm"], with_dwi=boot)
        data = np.ascontiguousarray(ph.dwi, dtype=np.float32) if boot else odf_volume(ph, sph)
        vol_bytes += data.nbytes
        dg = make_getter(sd["getter"], ph, sph)
        tr = Tracker(dg, data, ph.fa, 0.1, sph.vertices, sph.edges, max_angle=math.radians(g["max_angle"]),
                     step_size=0.5, ngpus=1, device_offset=0)
        tr.__enter__()
        trackers.append(tr)
        seeds.append(seeds_from_mask(ph.fa, sd["seeds"], threshold=0.3, seed=sd["seed"]).astype(np.float32))
        del data
    t_setup = time.perf_counter() - t_setup
    stream = torch.cuda.Stream()
    run = MultiSubjectRun(trackers, seeds)
    for _ in range(args.warmup):
        run.launch(stream.cuda_stream)
        run.wait()
    nsl, npts, rep, _ = run.last
    steps = int((npts - nsl).sum())
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed_graph(k):
        run.plan.set_concurrency(k)
        run.launch(stream.cuda_stream)  # re-capture, untimed
        run.wait()
        replays, graph_ms = 0, []
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            run.launch(stream.cuda_stream)
            _, _, rep, ms = run.wait()
            replays += int(rep.sum())
            graph_ms.append(ms)
        ev1.record(stream)
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1) / args.steps, replays, float(np.median(graph_ms))

    by_k = {}
    for k in (0, 1, 3):
        by_k[k] = timed_graph(k)
    with ClockSampler(0) as clk:
        by_k[2] = timed_graph(2)  # the library default, the reported value
    multi_ms, replays, graph_med = by_k[2]
    captures, _, _ = run.plan.info()

    # the same batches one after another through the plain path (the plan's
    # device seed buffers, viewed as tensors for the stream-ordered copies below)
    def tensor_view(buf):
        class _View:
            __cuda_array_interface__ = {"shape": buf.shape, "typestr": "<f4", "data": (buf.ptr, False),
                                        "version": 3, "strides": None}
        return torch.as_tensor(_View(), device="cuda")

    dev = [tensor_view(t) for t, _ in run._seeds]
    handles = [tr.handles[0] for tr in trackers]
    for h, d, s in zip(handles, dev, seeds):
        h.propagate_device(d.data_ptr(), len(s), 0, stream.cuda_stream)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        for h, d, s in zip(handles, dev, seeds):
            h.propagate_device(d.data_ptr(), len(s), 0, stream.cuda_stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    seq_ms = ev0.elapsed_time(ev1) / args.steps
    seq_steps = sum(h.counts()[1] - h.counts()[0] for h in handles)

    # end to end: seeds from pinned host memory, one graph launch, results to pinned host memory
    pinned = [torch.from_numpy(s).pin_memory() for s in seeds]
    outs = [(torch.empty(int(a), dtype=torch.int32).pin_memory().numpy(),
             torch.empty(int(a), dtype=torch.int32).pin_memory().numpy(),
             torch.empty((int(b), 3), dtype=torch.float32).pin_memory().numpy()) for a, b in zip(nsl, npts)]
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            for d, p in zip(dev, pinned):
                if len(p):
                    d[: len(p)].copy_(p, non_blocking=True)
        run.launch(stream.cuda_stream)
        _, np_, _, _ = run.wait()
        for h, (L, S, P), k in zip(handles, outs, np_):
            if len(L) and int(k) == len(P):
                h.fetch_into(L, S, P)
    ev1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = ev0.elapsed_time(ev1) / args.steps
    h2d = sum(s.nbytes for s in seeds)
    d2h = sum(L.nbytes + S.nbytes + P.nbytes for L, S, P in outs)
    run.close()
    for tr in trackers:
        tr.__exit__(None, None, None)
    nonempty = sum(1 for s in seeds if len(s))
    print(json.dumps({
        "metric": "tracking steps/s, multi-subject run in one CUDA-graph launch", "value": steps / (multi_ms / 1e3),
        "unit": "steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": multi_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic phantoms (seeded), random seeds in FA>0.3",
        "config": {"workload": f"{len(subs)} subjects of uneven size, mixed getters, one graph launch",
                   "subjects": [{k: sd[k] for k in ("getter", "shape", "n_dirs", "seeds")} for sd in subs],
                   "seeds_total": int(sum(len(s) for s in seeds)), "streamlines_total": int(nsl.sum()),
                   "steps_total": steps, "volume_bytes_total": vol_bytes,
                   "l2": "inputs (volumes) larger than L2; no flush", "setup_s": t_setup,
                   "graph_device_ms": graph_med, "graph_captures": captures,
                   "replays_in_timed_region": replays, "max_concurrent_tracking_kernels": 2,
                   "ms_per_step_by_max_concurrent": {str(k): v[0] for k, v in sorted(by_k.items())},
                   "bootstrap_fit": {"fp32": "per-warp FP32", "bf16x3": "batched tensor-core BF16x3"}[args.multi_boot_fit]},
        "sequential_plain": {"value": seq_steps / (seq_ms / 1e3), "ms_per_step": seq_ms,
                             "note": "same batches, one csl_propagate_device per subject in turn"},
        "speedup_vs_sequential": seq_ms / multi_ms,
        "e2e": {"value": steps / (e2e_ms / 1e3), "unit": "steps/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "roofline": None,
        "gpu_launches": 7 * nonempty * args.steps,
        "clocks": clk.summary(),
    }), flush=True)
    return 0


def run_learned(args):
    """Learned proposal: trained with the library's CUDA kernels on the plain
    tracker's steps on one phantom (seed 7), evaluated on the benchmark phantom
    (seed 1234): NLL, exact-rejection acceptance against the uniform-cone
    proposal, sampled-distribution check, training and inference throughput."""
    import torch
    from scipy.stats import ks_2samp

    from gpustreamlines_b200 import ProbDirectionGetter, Tracker, learned, shm
    from gpustreamlines_b200.odf import odf_volume_gpu
    from gpustreamlines_b200.phantom import make_phantom, seeds_from_mask
    from gpustreamlines_b200.sphere import get_sphere

    sph = get_sphere("repulsion724")
    cos_max = math.cos(math.radians(45.0))

    def track(seed, nseeds, sseed):
        ph = make_phantom((81, 106, 76), seed=seed, with_dwi=False)
        B, _, _ = shm.real_sh_descoteaux(ph.meta["sh_order"], sph.theta, sph.phi)
        pmf = odf_volume_gpu(ph.sh_coef, B).numpy()
        seeds = seeds_from_mask(ph.fa, nseeds, threshold=0.3, seed=sseed).astype(np.float32)
        with Tracker(ProbDirectionGetter(), pmf, ph.fa, 0.1, sph.vertices, sph.edges,
                     max_angle=math.radians(45), step_size=0.5) as tr:
            h = tr.handles[0]
            h.propagate(seeds)
            L, S, P = h.fetch()
        pos, din, dout = learned.steps_from_tracks(L, S, P, seeds)
        return ph, pmf, pos, din, dout

    t0 = time.time()
    ph_a, _, pos_a, din_a, dout_a = track(7, 4000, 70)
    ph_b, pmf_b, pos_b, din_b, dout_b = track(1234, 2000, 1000)
    prep_s = time.time() - t0
    net = learned.VmfProposalNet(seed=1)
    sh_a = learned.trilinear(ph_a.sh_coef, pos_a)
    f = np.concatenate([sh_a, din_a], axis=1)
    net.feat_mean = f.mean(0).astype(np.float32)
    net.feat_std = (f.std(0) + 1e-6).astype(np.float32)
    Xa = torch.from_numpy(net.features(sh_a, din_a)).cuda()
    Ta = torch.from_numpy(dout_a.astype(np.float32)).cuda()
    rng = np.random.default_rng(2)
    iters, batch = 3000, 1024
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(iters):
        idx = torch.from_numpy(rng.integers(0, len(pos_a), batch)).cuda()
        net.train_step(Xa[idx], Ta[idx], lr=2e-3)
    e1.record()
    torch.cuda.synchronize()
    train_ms = e0.elapsed_time(e1)
    sel = rng.choice(len(pos_b), size=min(3000, len(pos_b)), replace=False)
    sh_b = learned.trilinear(ph_b.sh_coef, pos_b[sel])
    Xb = torch.from_numpy(net.features(sh_b, din_b[sel])).cuda()
    Tb = torch.from_numpy(dout_b[sel].astype(np.float32)).cuda()
    nll = float(net.loss_and_grad(Xb, Tb).mean())
    mu, kap, lpi = learned.mixture(net.infer(Xb).cpu().numpy())
    p, x, cone = learned.target_pmf(pmf_b, sph.vertices, pos_b[sel], din_b[sel], cos_max)
    ok = p.sum(axis=1) > 0
    acc_l, acc_u, q = learned.acceptance(p[ok], x[ok], cone[ok], mu[ok], kap[ok], lpi[ok])
    acc_0, _, _ = learned.acceptance(p[ok], x[ok], cone[ok], mu[ok], kap[ok], lpi[ok], eps=0.0)
    r = np.random.default_rng(5)
    a_exact, a_rej, draws = [], [], 0
    dd = din_b[sel][ok]
    for b in range(min(2000, int(ok.sum()))):
        pb, qb, xb = p[ok][b], q[b], x[ok][b]
        a_exact.append(float(np.dot(xb[r.choice(len(pb), p=pb)], dd[b])))
        M = np.max(np.divide(pb, qb, out=np.zeros_like(pb), where=pb > 0))
        for _ in range(100000):
            v = r.choice(len(qb), p=qb)
            draws += 1
            if r.random() * M * qb[v] <= pb[v]:
                break
        a_rej.append(float(np.dot(xb[v], dd[b])))
    Xi = Xb.repeat(max(1, 1_000_000 // len(sel)), 1)
    net.infer(Xi)
    _, inf_ms = net.infer(Xi, return_ms=True)
    print(json.dumps({
        "workload": "learned vMF-mixture proposal: 48-128-128-128-40 SiLU MLP, trained on the plain prob "
                    "tracker's steps on phantom seed 7, evaluated on the benchmark phantom (seed 1234)",
        "train_steps": len(pos_a), "train_iters": iters, "batch": batch,
        "train_samples_per_s": iters * batch / (train_ms / 1e3),
        "nll_learned": nll, "nll_uniform_cone": math.log(2 * math.pi * (1 - cos_max)),
        "nll_uniform_sphere": math.log(4 * math.pi),
        "acceptance_learned_defensive30": float(acc_l.mean()), "acceptance_learned_bare": float(acc_0.mean()),
        "acceptance_uniform_cone": float(acc_u.mean()),
        "rejection_draws_per_step_learned": draws / max(1, len(a_rej)),
        "ks_turning_angle_exact_vs_rejection_p": float(ks_2samp(a_exact, a_rej).pvalue),
        "inference_samples_per_s": Xi.shape[0] / (inf_ms / 1e3), "inference_flop_per_sample": 88064,
        "prep_s": prep_s}), flush=True)
    return 0


def main():
    args = parse()
    rank, world, local = dist_info()
    if args.learned:
        return run_learned(args) if rank == 0 else 0
    if args.odf_volume:
        return run_odf_volume(args) if rank == 0 else 0
    if args.multi:
        return run_multi(args) if rank == 0 else 0
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.boot_compare:
        return run_boot_compare(args) if rank == 0 else 0

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    from gpustreamlines_b200 import Tracker

    gcfg = GETTERS[args.getter]
    ph, sph, data, seeds = build_workload(rank, args.seeds, args.getter)
    dg = make_getter(args.getter, ph, sph)
    tracker = Tracker(dg, data, ph.fa, 0.1, sph.vertices, sph.edges,
                      max_angle=math.radians(gcfg["max_angle"]), step_size=0.5, ngpus=1,
                      device_offset=local)
    tracker.__enter__()
    h = tracker.handles[0]
    if args.autotune:
        if rank == 0:
            t0 = time.perf_counter()
            ((ms, best),) = tracker.autotune(seeds, sample=len(seeds), repeats=2)
            print(json.dumps({"workload": f"{gcfg['label']}, {args.seeds} seeds", "tuner_s": time.perf_counter() - t0,
                              "batch_ms_by_shape": {f"{b} threads, {'Morton' if o else 'input'} order": v
                                                    for (b, o), v in ms.items()},
                              "chosen": {"threads_per_block": best[0], "seed_order": best[1]}}), flush=True)
        tracker.__exit__(None, None, None)
        return 0
    stream = torch.cuda.Stream(device=local)
    seeds_d = torch.from_numpy(seeds).to(f"cuda:{local}")
    seeds_pinned = torch.from_numpy(seeds).pin_memory()
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()

    def device_step():
        h.propagate_device(seeds_d.data_ptr(), len(seeds), 0, stream.cuda_stream)

    for _ in range(args.warmup):
        device_step()
    nsl, npts = h.counts()
    steps_per_batch = npts - nsl  # sum(len - 1)

    # ---- device-resident timed region
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    pass2_ms, pass1_ms, compact_ms = [], [], []
    envelope = gcfg.get("sampler") == "envelope"
    if envelope:
        h.sampler_stats(reset=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            device_step()
            (p1, gap, p2, cp), runs = h.timings()
            pass1_ms.append(p1)
            pass2_ms.append(p2)
            compact_ms.append(cp)
        ev1.record(stream)
        torch.cuda.synchronize()
    total_ms = ev0.elapsed_time(ev1)
    env_stats = h.sampler_stats() if envelope else None
    barrier()
    counts = torch.tensor([float(total_ms), float(nsl), float(npts)], device=f"cuda:{local}",
                          dtype=torch.float64)
    if dist is not None:
        t = counts[:1].clone()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        gathered = [torch.zeros_like(counts) for _ in range(world)]
        dist.all_gather(gathered, counts)
        total_ms_max = float(t.item())
        all_steps = sum(float(g[2].item() - g[1].item()) for g in gathered)
    else:
        total_ms_max = total_ms
        all_steps = float(steps_per_batch)
    ms_per_step = total_ms_max / args.steps
    value = all_steps * args.steps / (total_ms_max / 1e3)

    # ---- end-to-end through the C ABI with host buffers
    # pinned host buffers for the results, as for the seeds
    L = torch.empty(nsl, dtype=torch.int32).pin_memory().numpy()
    S = torch.empty(nsl, dtype=torch.int32).pin_memory().numpy()
    Pt = torch.empty((npts, 3), dtype=torch.float32).pin_memory().numpy()
    seeds_host = seeds_pinned.numpy()
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        h.propagate(seeds_host, 0, stream.cuda_stream)
        h.fetch_into(L, S, Pt)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if dist is not None:
        t = torch.tensor([e2e_ms], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = all_steps * args.steps / (e2e_ms / 1e3)
    h2d = seeds.nbytes
    d2h = L.nbytes + S.nbytes + Pt.nbytes

    peak, peak_kind = measured_peaks()
    p2 = float(np.mean(pass2_ms))
    model = gcfg["model"]
    if model == "PTT":
        # dependent texture fetches: reported as sub-steps/s, no byte roofline
        bytes_per_step = None
        achieved = None
    elif model in ("CSA", "OPDT"):
        bytes_per_step = 8 * data.shape[3] * 4 + 8 * 4 + 12  # DWI corners + stop taps + point
        achieved = steps_per_batch * bytes_per_step / (p2 / 1e3) / 1e9
    elif envelope:
        # the sampler's algorithmic bytes: 8 corner rows of the bf16 cluster-maxima
        # table (128 B each), the incoming direction's cone-bit row (256 B), 8 PMF
        # values per evaluated draw (4 per round), the stop-map taps and the point write
        props = env_stats["proposals"] / max(env_stats["steps"], 1)
        bytes_per_step = 8 * 128 + 256 + 8 * 4 * props + 8 * 4 + 12
        achieved = steps_per_batch * bytes_per_step / (p2 / 1e3) / 1e9
    else:
        bytes_per_step = BYTES_PER_STEP
        achieved = steps_per_batch * BYTES_PER_STEP / (p2 / 1e3) / 1e9
    traffic = None
    if envelope and args.env_traffic_bytes_per_step:
        traffic = args.env_traffic_bytes_per_step * steps_per_batch
    elif args.traffic_bytes_per_step and model == "PROB" and not envelope:
        traffic = args.traffic_bytes_per_step * steps_per_batch
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": None if achieved is None else achieved / peak, "traffic": traffic,
                "kernel": f"track_kernel<{model}> (pass 2)",
                "peak_source": f"{peak_kind} MEASURED_PEAKS hbm_gbs",
                "algorithmic_bytes_per_step": bytes_per_step}
    if model == "PROB" and traffic is not None:
        roofline["traffic_source"] = "ncu dram__bytes_read+write per step at 20k seeds x steps"
        # the HBM fraction the measured DRAM traffic implies (algorithmic bytes
        # above include L2 hits)
        roofline["dram_frac"] = traffic / (p2 / 1e3) / 1e9 / peak
    if envelope:
        roofline["kernel"] = "track_kernel<PROB_ENV> (pass 2, envelope sampler)"
        # the plain kernel's algorithmic bytes per step over the same time: the
        # rate the inverse-CDF path would need to match this kernel
        roofline["plain_equivalent_gbs"] = steps_per_batch * BYTES_PER_STEP / (p2 / 1e3) / 1e9
    if gcfg.get("fit") == "bf16x3":
        # tensor roofline of the batched fit: algorithmic FP32-equivalent FLOP per
        # attempt (each step takes >= 1 attempt) against the measured BF16 peak;
        # the BF16x3 split issues 3x these on the tensor pipe
        nc = dg.delta_nr
        hr = int((dg.b0s_mask == 0).sum())
        flop = 2 * 2 * hr * hr + 2 * nc * hr * (2 if model == "OPDT" else 1) + 2 * nc * dg.sampling_matrix.shape[0]
        tpeak = None
        path = os.path.join(HERE, "MEASURED_PEAKS.json")
        if os.path.exists(path):
            with open(path) as f:
                tpeak = float(json.load(f).get("bf16_tflops", 0) or 0) or None
        tach = steps_per_batch * flop / (p2 / 1e3) / 1e12
        roofline = {"bound": "tensor", "achieved": tach, "peak": tpeak or 1590.0, "unit": "TFLOP/s",
                    "frac": tach / (tpeak or 1590.0), "traffic": None,
                    "kernel": "boot_batch_kernel (pass 2, tcgen05 BF16x3)",
                    "peak_source": "measured MEASURED_PEAKS bf16_tflops" if tpeak else "fallback",
                    "algorithmic_flop_per_step": flop, "issued_bf16_flop_per_step": 3 * flop}
    extra = {}
    if envelope:
        st = env_stats
        extra["sampler"] = {"draws_evaluated_per_step": st["proposals"] / max(st["steps"], 1),
                            "rounds_of_4_draws_per_step": st["proposals"] / 4 / max(st["steps"], 1),
                            "exact_max_resolutions_per_step": st["resolves"] / max(st["steps"], 1),
                            "inverse_cdf_fallbacks_per_step": st["fallbacks"] / max(st["steps"], 1)}
    if envelope and not args.no_plain_arm:
        extra["plain_fp32"] = plain_arm(args, data, ph, sph, gcfg, seeds_d, local, stream, barrier, dist, world)
        extra["speedup_vs_plain_fp32"] = value / extra["plain_fp32"]["value"]
    if model == "PTT":
        frac = int(np.round(0.5 / dg.target_short_step))  # propagation sub-steps per point
        extra["sub_steps_per_s"] = value * frac
        extra["step_frac"] = frac
    if model in ("CSA", "OPDT"):
        nc = dg.delta_nr
        hr = int((dg.b0s_mask == 0).sum())
        k = 2 if model == "OPDT" else 1
        extra["flop_per_attempt"] = 2 * 2 * hr * hr + 2 * nc * hr * k + 2 * nc * dg.sampling_matrix.shape[0]

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(ph, sph, data, seeds, args.cpu_seconds, getter=args.getter, dg=dg)
        except Exception as e:  # the oracle is optional on the GPU box
            cpu = {"value": None, "unit": "steps/s", "cores": 0, "kind": "port",
                   "sample": f"unavailable: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic phantom with Stanford HARDI shapes (seeded), random seeds in FA>0.3",
            "config": {"workload": f"{gcfg['label']}, {args.seeds} seeds per GPU, step 0.5, "
                                   f"max angle {gcfg['max_angle']:g}",
                       "global_batch": args.seeds * world, "seeds_per_gpu": args.seeds,
                       "streamlines_per_gpu": nsl, "steps_per_gpu": int(steps_per_batch),
                       "parallelism": f"seed shards x{world}",
                       "l2": f"inputs ({data.nbytes / 1e9:.2f} GB volume) larger than L2; no flush",
                       "pass1_ms": float(np.mean(pass1_ms)), "pass2_ms": p2,
                       "compact_ms": float(np.mean(compact_ms)),
                       "streamlines_per_s": nsl * world * args.steps / (total_ms_max / 1e3), **extra},
            "roofline": roofline,
            "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": 3 * args.steps,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    tracker.__exit__(None, None, None)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
