"""Benchmark of the forward-model hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload production|small]

One step of the default ("production") workload is the hot path of the
pipeline at 64 slices of 2048^2: the USFFT Radon transform R of the volume
at 2058 angles on [0, 2 pi), then psi = exp(-p s/beta_r)(cos p s, sin p s),
Fresnel propagation D (30 keV, 0.12 m, 0.69 um pixels, 2x mirror padding)
and |.|^2 of all 2058 projections.  The metric is R/RT throughput in
Gvox*angle/s = slices * n^2 * ntheta / step time (whole job, all ranks); the
adjoint RT is timed on the same data and reported beside it.

Rank layout: one process per GPU (torchrun for N > 1); every rank runs its
own 64-slice slab (weak scaling, no collective on the data path; the ranks
only meet at barriers and in a max-reduce of their timings).

--impl reference times the reference's own kernels (processing/kernels.py,
compiled for the host into oracle/_ref by oracle/build_ref.py) with the
reference's host glue restated in NumPy/SciPy on all host cores, on a bounded
sample of the same workload (one slice of R plus 32 frames of D, scaled to a
full step).  Under torchrun only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # 64 slices of 2048^2, 2058 angles on [0, 2 pi), then D of all projections
    "production": dict(n=2048, nz=64, ntheta=2058, theta_max=2 * np.pi, energy_kev=30.0,
                       distance=0.12, voxelsize=0.69e-6),
    # 128 slices of 128^2, 180 angles on [0, pi)
    "small": dict(n=128, nz=128, ntheta=180, theta_max=np.pi, energy_kev=30.0,
                  distance=0.12, voxelsize=0.69e-6),
    # same kernels as "production" on a few GB of device memory (for ncu captures)
    "profile": dict(n=1024, nz=64, ntheta=512, theta_max=2 * np.pi, energy_kev=30.0,
                    distance=0.12, voxelsize=0.69e-6),
    # the production slice size (4096-point columns, 2048-point rows) on ~4.5 GB
    "profile2048": dict(n=2048, nz=32, ntheta=128, theta_max=2 * np.pi, energy_kev=30.0,
                        distance=0.12, voxelsize=0.69e-6),
    # the production layout (64 slices of 2048^2: the same column, gather and
    # D kernels, per-launch column traffic independent of the angle count) on
    # ~9.5 GB, few angles
    "profile64": dict(n=2048, nz=64, ntheta=64, theta_max=2 * np.pi, energy_kev=30.0,
                      distance=0.12, voxelsize=0.69e-6),
    # the adjoint scatter with a polar spectrum larger than L2 (1024 angles of
    # 513 x 64 complex: 269 MB) on ~3.5 GB, for ncu captures of the scatter
    "rtprofile": dict(n=1024, nz=64, ntheta=1024, theta_max=2 * np.pi, energy_kev=30.0,
                      distance=0.12, voxelsize=0.69e-6),
    # the 3 * 2^k kernels of the n = 3072 size (6144-point x-side and
    # column lines, 1536-point r-side lines, 3072-point D rows) on ~3 GB
    "profile3072": dict(n=3072, nz=8, ntheta=288, theta_max=np.pi, energy_kev=30.0,
                        distance=0.12, voxelsize=0.69e-6),
    # step8_fbp.py's default size (n = 3072, 3n/4 = 2304 angles on [0, pi)):
    # 6144-point columns and rows, 1536-point r-side lines (radix-3 passes)
    "n3072": dict(n=3072, nz=32, ntheta=2304, theta_max=np.pi, energy_kev=30.0,
                  distance=0.12, voxelsize=0.69e-6),
}
BETA_RATIO = 100.0
L2_BYTES = 126 * 2 ** 20


def workload_desc(w, name):
    return (f"{name}: R of {w['nz']} slices of {w['n']}^2 at {w['ntheta']} angles on "
            f"[0, {'2pi' if w['theta_max'] > 4 else 'pi'}), then psi -> Fresnel D ({w['energy_kev']:g} keV, "
            f"{w['distance']} m, {w['voxelsize'] * 1e6:.2f} um, 2x mirror pad) -> |.|^2 of all projections")


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(workload, kernel):
    """Per-launch DRAM bytes of `kernel` on `workload` from a committed ncu
    summary, if any: a line 'traffic_bytes_per_launch <workload> <kernel>
    <bytes>' in profiles/*.md."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for fn in sorted(os.listdir(pdir)):
        if not fn.endswith((".md", ".txt")):
            continue
        for line in open(os.path.join(pdir, fn)):
            parts = line.strip().strip("`").split()
            if (len(parts) == 4 and parts[0] == "traffic_bytes_per_launch" and parts[1] == workload
                    and parts[2] == kernel):
                return float(parts[3])
    return None


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons.  The sampler runs
    from before the warm-up to after the last timed loop (every 25 ms, with
    timestamps); the summary keeps the samples that fall inside the timed
    regions (``window`` marks each)."""
    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.windows = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "25"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def window(self, t0, t1):
        self.windows.append((t0, t1))

    def stop(self):
        if self.proc:
            time.sleep(0.1)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]
            self.proc = None

    def summary(self):
        import datetime
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                smv, mxv = float(f[2]), float(f[3])
            except ValueError:
                continue
            if not any(t0 - 0.03 <= ts <= t1 + 0.03 for t0, t1 in self.windows):
                continue
            sm.append(smv)
            mx.append(mxv)
            for nm, v in zip(names, f[6:10]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm), "sampled": "nvidia-smi every 25 ms inside the timed step, RT and e2e loops"}


# ---------------------------------------------------------------- our arm
def run_ours(args, w, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from model_mosaic_b200.processing.tomo import TomoReal
    from model_mosaic_b200.processing.propagation import Propagation
    from model_mosaic_b200.phantom import ellipsoid_volume_torch

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n, nz, T = w["n"], w["nz"], w["ntheta"]
    theta = np.linspace(0, w["theta_max"], T, endpoint=False).astype(np.float32)
    wavelength = 1.24e-9 / w["energy_kev"]
    inv_norm = float(np.float32(1.0 / np.sqrt(n / T)))       # step3_propagation.py:82,182
    inv_beta = float(np.float32(1.0 / BETA_RATIO))

    tomo = TomoReal(n, nz, theta)
    prop = Propagation(n, nz, T, 1, wavelength, w["voxelsize"], [w["distance"]])
    from model_mosaic_b200.pipeline import StreamedForward
    obj = ellipsoid_volume_torch(n, nz, seed=rank, device=dev)        # each rank: its own slab
    sino = torch.empty((T, nz, n), dtype=torch.float32, device=dev)
    inten = torch.empty((T, nz, n), dtype=torch.float32, device=dev)
    rec = torch.empty((nz, n, n), dtype=torch.float32, device=dev)
    if not args.no_rt:
        tomo.prepare_rt()

    def step():
        tomo.R_into(obj, sino)
        prop.intensity_into(sino, inten, inv_norm, inv_beta)

    clk = Clocks(local_rank).start()   # running before the warm-up, stopped after the last timed loop

    def barrier():
        if world > 1:
            dist.barrier()

    from model_mosaic_b200.dist import max_over_ranks

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # -- timed region: K steps, stage timers on the launching stream ----------
    tomo.set_timing(True)
    prop.set_timing(True)
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    t_w0 = time.time()
    torch.cuda.nvtx.range_push("timed_step")
    e0.record(st)
    for _ in range(args.steps):
        step()
    e1.record(st)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    clk.window(t_w0, time.time())
    barrier()
    ms_step = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    tstages, tk = tomo.timing()
    pstages, pk = prop.timing()
    tomo.set_timing(False)
    prop.set_timing(False)

    # -- adjoint RT on the same data (reported beside the step) --------------
    ms_rt, rtstages = None, {}
    if not args.no_rt:
        for _ in range(max(1, args.warmup // 2)):
            tomo.RT_into(sino, rec)
        tomo.set_timing(True)
        barrier()
        torch.cuda.synchronize()
        t_w0 = time.time()
        torch.cuda.nvtx.range_push("timed_rt")
        e0.record(st)
        for _ in range(args.steps):
            tomo.RT_into(sino, rec)
        e1.record(st)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        clk.window(t_w0, time.time())
        ms_rt = max_over_ranks(e0.elapsed_time(e1) / args.steps)
        rtstages, _ = tomo.timing()
        tomo.set_timing(False)

    # -- end to end through the public API: pinned host in, host out ---------
    # StreamedForward double-buffers the volumes: the copy-in of step i+1,
    # the compute of step i and the copy-out of step i-1 overlap.
    tomo.free()
    prop.free()
    fwd = StreamedForward(n, nz, theta, wavelength, w["voxelsize"], w["distance"], inv_norm, inv_beta)
    obj_h = obj.cpu().pin_memory()
    outs_h = [fwd.pinned_intensity() for _ in range(2)]
    for i in range(max(2, args.warmup)):
        fwd.submit(obj_h, outs_h[i % 2])
    fwd.synchronize()
    barrier()
    t_w0 = time.time()
    torch.cuda.nvtx.range_push("timed_e2e")
    e0.record(fwd.s_in)
    for i in range(args.steps):
        fwd.submit(obj_h, outs_h[i % 2])
    e1.record(fwd.s_out)
    torch.cuda.nvtx.range_pop()
    fwd.synchronize()
    clk.window(t_w0, time.time())
    clk.stop()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    fwd.free()

    V = nz * n * n
    units = world * V * T
    value = units / (ms_step * 1e-3) / 1e9
    K = args.steps
    r_ms = sum(v[0] for k, v in tstages.items() if v[1]) / K
    d_ms = sum(v[0] for v in pstages.values()) / K

    # roofline of the dominant own kernel in the step
    P = T * nz * n
    H = 2 * n * (n + 1) * nz
    Kh = n // 2 + 1
    alg = {  # algorithmic bytes per launch: each kernel's inputs read once, outputs written once
        "pad_phi": 4 * V + 8 * nz * n * (n + 1),               # k_xfwd: obj -> centre rows of Y
        "y_fft": 8 * nz * n * (n + 1) + 16 * nz * n * (n + 1),  # k_col_fft: centre rows -> 2n rows
        "gather": 8 * H + 8 * Kh * T * nz,                     # k_gather: half spectrum -> polar lines
        "r_c2r": 8 * Kh * T * nz + 4 * T * nz * n,             # k_rc2r: polar lines -> sinogram
        "y_pass": 4 * P + 8 * P,                               # k_ypass: p -> psi -> column pass
        "x_pass": 8 * P + 4 * P,                               # k_xpass: row pass -> |.|^2
    }
    own = {k: (tstages if k in tstages else pstages)[k] for k in alg if k in tstages or k in pstages}
    top = max(own, key=lambda k: own[k][0])
    t_launch = own[top][0] / max(1, own[top][1])
    peak, peak_kind = peaks()
    achieved = alg[top] / (t_launch * 1e-3) / 1e9
    col_kernel = "k_col_l2" if (n == 2048 and nz % 8 == 0) else "k_col_fft"   # tomo_col.cu covers 2n = 4096
    kname = {"gather": "k_gather", "pad_phi": "k_xfwd", "y_fft": col_kernel, "r_c2r": "k_rc2r",
             "y_pass": "k_ypass_pf" if (nz & (nz - 1)) == 0 and 64 <= nz <= 1024 else "k_ypass",
             "x_pass": "k_xpass"}[top]
    traffic = profile_traffic(args.workload, kname)
    # the step's algorithmic bytes as the hot-path scope defines them: R's
    # B_R = 4V + 16Hc + 16H + 4S and D's B_D = 24P (Hc = nz n (n+1))
    Hc = nz * n * (n + 1)
    step_bytes = (4 * V + 16 * Hc + 16 * H + 4 * T * nz * n) + 24 * P
    roof = {"bound": "hbm", "kernel": kname, "achieved": round(achieved, 1), "peak": peak,
            "peak_source": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "traffic": traffic, "alg_bytes_per_launch": alg[top], "ms_per_launch": round(t_launch, 4)}

    line = {
        "metric": "R/RT Gvox·angle/s", "value": round(value, 3), "unit": "Gvox·angle/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: 10 seeded random ellipsoids per slab (values in [1e-7, 1e-6], beta = delta/100)",
        "config": {"workload": workload_desc(w, args.workload), "n": n, "nz_per_rank": nz, "ntheta": T,
                   "l2": "inputs larger than L2 (volume %.2f GB, sinogram %.2f GB per rank); no flush"
                         % (4 * V / 1e9, 4 * P / 1e9),
                   "parallelism": f"{world} ranks x independent slabs"},
        "roofline": roof,
        "gpu_launches": int(tk + pk),
        "ops": {"R_ms": round(r_ms, 4), "D_ms": round(d_ms, 4), "RT_ms": round(ms_rt, 4) if ms_rt else None,
                "R_gvox_angle_s": round(V * T / (r_ms * 1e-3) / 1e9, 3) if r_ms else None,
                "RT_gvox_angle_s": round(world * V * T / (ms_rt * 1e-3) / 1e9, 3) if ms_rt else None,
                "D_gpix_s": round(P / (d_ms * 1e-3) / 1e9, 3) if d_ms else None,
                "step_frac_of_hbm": round(step_bytes / (ms_step * 1e-3) / 1e9 / peak, 4),
                "stages_ms": {k: round(v[0] / K, 4) for k, v in {**tstages, **pstages}.items() if v[1]},
                "rt_stages_ms": {k: round(v[0] / K, 4) for k, v in rtstages.items() if v[1] and k != "table_build"}},
        "e2e": {"value": round(units / (ms_e2e * 1e-3) / 1e9, 3), "unit": "Gvox·angle/s",
                "ms_per_step": round(ms_e2e, 4), "h2d_bytes_per_step": int(4 * V),
                "d2h_bytes_per_step": int(4 * P)},
        "clocks": clk.summary(),
    }
    return line


# ---------------------------------------------------------------- differentiable model
MODEL = dict(n=512, nz=512, ntheta=1024, theta_max=np.pi, chunk=128)


def run_model(args, local_rank):
    """fwd+grad ms/iter of the L2 misfit of |D(exp(i(R delta + i R beta)))|^2 at
    512^3 with 1024 angles, psi recomputed per 128-angle chunk: the fused
    kernels against the same gradient composed from the unfused operators."""
    import torch
    from model_mosaic_b200.model import ForwardModel
    from model_mosaic_b200.phantom import ellipsoid_volume_torch
    w = WORKLOADS["production"]
    n, nz, T = MODEL["n"], MODEL["nz"], MODEL["ntheta"]
    dev = torch.device("cuda", local_rank)
    theta = np.linspace(0, MODEL["theta_max"], T, endpoint=False).astype(np.float32)
    m = ForwardModel(n, nz, theta, 1.24e-9 / w["energy_kev"], w["voxelsize"], w["distance"],
                     angle_chunk=MODEL["chunk"])
    delta = ellipsoid_volume_torch(n, nz, seed=0, device=dev)
    data = m.forward(ellipsoid_volume_torch(n, nz, seed=1, device=dev))
    st = torch.cuda.current_stream()
    out = {}
    for name, fn in (("fused", m.loss_and_grad), ("plain", m.plain_loss_and_grad)):
        for _ in range(args.warmup):
            fn(delta, data)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.nvtx.range_push(f"timed_model_{name}")
        e0.record(st)
        for _ in range(args.steps):
            fn(delta, data)
        e1.record(st)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        out[name + "_ms"] = round(e0.elapsed_time(e1) / args.steps, 3)
    out["speedup_vs_plain"] = round(out["plain_ms"] / out["fused_ms"], 3)
    # baseline leg: the same step composed from the reference's own kernels
    # (oracle/refgpu.py: its R, D, psi, |.|^2 plus the exact adjoints)
    from oracle import refgpu
    if not args.no_ref_gpu and refgpu.available():
        inv_norm = m.s      # the model's phase scale s
        rt = refgpu.RefGpuTomoReal(n, nz, theta, device=dev)
        rp = refgpu.RefGpuPropagation(n, nz, MODEL["chunk"], 1, 1.24e-9 / w["energy_kev"], w["voxelsize"],
                                      [w["distance"]], device=dev)
        ref_step = lambda: refgpu.ref_loss_and_grad(rt, rp, delta, data, inv_norm, 1.0 / BETA_RATIO,  # noqa: E731
                                                    chunk=MODEL["chunk"])
        ref_step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = max(2, min(args.steps, 5))
        e0.record(st)
        for _ in range(reps):
            ref_step()
        e1.record(st)
        torch.cuda.synchronize()
        out["reference_ms"] = round(e0.elapsed_time(e1) / reps, 3)
        out["speedup_vs_reference"] = round(out["reference_ms"] / out["fused_ms"], 3)
        out["reference"] = ("the same loss and gradient composed from the reference's kernels "
                            "(processing/kernels.py for sm_100a) and its cupy glue on torch/cuFFT, with the "
                            "exact adjoint of its D; atomic scatter in RT")
        del rt, rp
        torch.cuda.empty_cache()
    out["config"] = f"{nz} slices of {n}^2, {T} angles on [0, pi), psi recomputed per {MODEL['chunk']}-angle chunk"
    return out


# ---------------------------------------------------------------- uneven tiles (CUDA graph)
def run_tiles(args, local_rank):
    """36 mosaic tiles, n drawn from {512, 768, 1024, 1536} and angle counts
    uniform in [360, 2058] (seeded), 16 slices each, seeded ellipsoid volumes:
    R, psi -> D -> |.|^2 and RT of every tile as one CUDA graph over 4 streams
    (TileBatch), against the same work launched eagerly tile after tile."""
    import torch
    from model_mosaic_b200.phantom import ellipsoid_volume_torch
    from model_mosaic_b200.tiles import TileBatch
    w = WORKLOADS["production"]
    rng = np.random.default_rng(5)
    specs = []
    for _ in range(36):
        n = int(rng.choice([512, 768, 1024, 1536]))
        T = int(rng.integers(360, 2059))
        specs.append(dict(n=n, nz=16, theta=np.linspace(0, np.pi, T, endpoint=False).astype(np.float32)))
    dev = torch.device("cuda", local_rank)
    wl = 1.24e-9 / w["energy_kev"]

    def fill(b):
        for i, t in enumerate(specs):
            b.obj(i).copy_(ellipsoid_volume_torch(t["n"], 16, seed=100 + i, device=dev))

    # per tile size the USFFT pair (eps, m) and for the batch the stream count,
    # chosen by the project's autotuner (outside the timed region; its cache
    # lives in a scratch file so every run tunes afresh)
    import tempfile
    from model_mosaic_b200.autotune import autotuned_batch
    with tempfile.TemporaryDirectory() as tmp:
        batch, tuned = autotuned_batch(specs, wl, w["voxelsize"], w["distance"], cache=os.path.join(tmp, "at.json"),
                                       fill=fill, device=local_rank)
    st = torch.cuda.current_stream(dev)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(args.steps):
            fn()
        e1.record(st)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / args.steps

    def eager_one_stream():
        for tl in batch.tiles:
            tl.step()

    ms_graph = timed(batch.run)            # the autotuner left the winning graph captured
    ms_eager = timed(eager_one_stream)
    units = batch.voxel_angles()
    out = {"metric": "R+D+RT Gvox·angle/s over a batch of uneven tiles", "workload": "tiles",
           "value": round(units / (ms_graph * 1e-3) / 1e9, 3), "unit": "Gvox·angle/s",
           "graph_ms": round(ms_graph, 3), "eager_ms": round(ms_eager, 3),
           "graph_speedup": round(ms_eager / ms_graph, 3), "steps": args.steps, "warmup": args.warmup,
           "config": {"tiles": len(specs), "n": [t["n"] for t in specs],
                      "ntheta": [len(t["theta"]) for t in specs], "slices_per_tile": 16,
                      "streams": tuned["streams"]["streams"], "step": "R, psi -> D -> |.|^2 and RT of every tile"},
           "autotune": {"per_size": {str(k): {"eps": v["choice"][0], "m": v["choice"][1],
                                              "err_vs_eps1e-5": v["errors"], "tile_ms": v["ms"]}
                                     for k, v in tuned["classes"].items()},
                        "streams_ms": tuned["streams"]["ms"],
                        "rule": "fastest (eps, m) with R error <= the reference setting's (eps 1e-3, m 4); "
                                "grid oversampling 2"}}
    batch.free()
    return out


# ---------------------------------------------------------------- filtered backprojection (step8)
def run_fbp(args, local_rank):
    """step8_fbp's compute (step8_fbp.py:203-205) on the sinogram of the
    --base workload (production: 2058 x 64 rows of 2048): the FBP filter
    ('shepp', 4x edge padding), then RT.  Reports the filter alone (rows/s, GB/s of its 8 bytes per sample and
    the FP32 rate of its two 8192-point transforms per row pair) and the
    filtered backprojection in Gvox*angle/s."""
    import torch
    from model_mosaic_b200.phantom import ellipsoid_volume_torch
    from model_mosaic_b200.processing.fbp_filter import FBPFilter
    from model_mosaic_b200.processing.tomo import TomoReal
    w = WORKLOADS[args.base]
    n, nz, T = w["n"], w["nz"], w["ntheta"]
    dev = torch.device("cuda", local_rank)
    theta = np.linspace(0, w["theta_max"], T, endpoint=False).astype(np.float32)
    tomo = TomoReal(n, nz, theta)
    tomo.prepare_rt()
    sino0 = tomo.R(ellipsoid_volume_torch(n, nz, seed=0, device=dev))
    sino = torch.empty_like(sino0)
    rec = torch.empty((nz, n, n), dtype=torch.float32, device=dev)
    f = FBPFilter(n)
    wts = f.calc_filter("shepp")
    st = torch.cuda.current_stream(dev)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(args.steps):
            fn()
        e1.record(st)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / args.steps

    ms_copy = timed(lambda: sino.copy_(sino0))
    ms_filter = timed(lambda: (sino.copy_(sino0), f.filter(sino, wts))) - ms_copy

    def fbp():
        sino.copy_(sino0)
        f.filter(sino, wts)
        tomo.RT_into(sino, rec)

    ms_fbp = timed(fbp) - ms_copy
    rows = T * nz
    flops = rows / 2 * 2 * 5 * (4 * n) * np.log2(4 * n)
    V = nz * n * n
    out = {"metric": "filtered backprojection Gvox·angle/s (FBP filter + RT)", "workload": "fbp",
           "value": round(V * T / (ms_fbp * 1e-3) / 1e9, 3), "unit": "Gvox·angle/s",
           "fbp_ms": round(ms_fbp, 3), "filter_ms": round(ms_filter, 3),
           "filter_rows_per_s": round(rows / (ms_filter * 1e-3), 1),
           "filter_gbs": round(8 * rows * n / (ms_filter * 1e-3) / 1e9, 1),
           "filter_fp32_tflops": round(flops / (ms_filter * 1e-3) / 1e12, 2),
           "steps": args.steps, "warmup": args.warmup,
           "config": {"n": n, "nz": nz, "ntheta": T, "filter": "shepp", "padding": "edge, 4n",
                      "note": "times exclude the untimed-equivalent sinogram refresh copy (measured and subtracted)"}}
    f.free()
    tomo.free()
    return out


# ---------------------------------------------------------------- Paganin retrieval (step7)
def run_paganin(args, local_rank):
    """step7_paganin's compute on the frames of the --base workload
    (production: 2058 intensity frames of 64 x 2048; 30 keV, 0.12 m, 0.69 um,
    alpha 1e-3), device-resident.  Three passes of 24 bytes per pixel of HBM traffic
    (4 in, 8 + 8 through the half spectrum, 4 out): the roofline is HBM."""
    import torch
    from model_mosaic_b200.processing.paganin import Paganin
    w = WORKLOADS[args.base]
    n, nz, T = w["n"], w["nz"], w["ntheta"]
    dev = torch.device("cuda", local_rank)
    pgn = Paganin(n, nz, T, 1.24e-9 / w["energy_kev"], w["voxelsize"], w["distance"], 1e-3)
    g = torch.Generator(device=dev).manual_seed(0)
    x = 0.5 + 0.5 * torch.rand((T, nz, n), device=dev, generator=g)
    y = torch.empty_like(x)
    st = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        pgn.retrieve_into(x, y)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(args.steps):
        pgn.retrieve_into(x, y)
    e1.record(st)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / args.steps
    P = T * nz * n
    peak, peak_kind = peaks()
    gbs = 24 * P / (ms * 1e-3) / 1e9
    pgn.free()
    return {"metric": "Paganin retrieval Gpix/s", "workload": "paganin", "value": round(P / (ms * 1e-3) / 1e9, 3),
            "unit": "Gpix/s", "ms_per_step": round(ms, 3), "steps": args.steps, "warmup": args.warmup,
            "roofline": {"bound": "hbm", "achieved": round(gbs, 1), "peak": peak, "peak_source": peak_kind,
                         "unit": "GB/s", "frac": round(gbs / peak, 4), "alg_bytes_per_pixel": 24},
            "config": {"frames": T, "nz": nz, "n": n, "alpha": 1e-3, "data": "synthetic 0.5 + 0.5 U[0, 1)"}}


# ---------------------------------------------------------------- mosaic tiles (step4 / step6)
def run_stitch(args, local_rank):
    """step6_stitch's blend (step6_stitch.py:206-262) for one vchunk of 64
    output angles (its default --nthetachunk) on the reference's ups = 2
    mosaic (6144 x 6144 projection, 11 x 4 tiles of 606 x 808, overlap 50),
    tiles device-resident; beside it step4_extract's crop (step4_extract.py:
    176-192) of the same 64 angles.  Algorithmic bytes: every tile frame read
    once plus the output written once (stitch); every tile pixel read from the
    projection and written once (extract).  Inputs are 10-11 GB, far above
    L2.  e2e: the same stitch for 8 angles with the tile frames copied in
    from pinned host memory and the result copied back inside the timed
    region.  cpu_baseline: the reference's NumPy blend (oracle/mosaic.py,
    one thread) on 2 angles of the same mosaic."""
    import torch
    from model_mosaic_b200 import mosaic as mo
    from oracle import mosaic as om
    dev = torch.device("cuda", local_rank)
    meta, rows = mo.mosaic_layout(args.ups)
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        mo.write_positions_file(os.path.join(d, "pos.txt"), meta, rows)
        meta, pl = mo.read_placements(os.path.join(d, "pos.txt"))
    nth = args.angles
    nz, n = meta["NZ"], meta["N"]
    mt = mo.MosaicTiles(dict(meta, N_HALF=nth, NTHETA=2 * nth), pl)
    g = torch.Generator(device=dev).manual_seed(0)
    proj = 0.5 + torch.rand((nth, nz, n), device=dev, generator=g)
    tiles = mt.extract(proj)  # (2 nth, h, w) per tile: direct then mirror frames
    for k, t in enumerate(tiles):  # one gain per tile: overlapping tiles disagree as after step5
        t.mul_(1.0 + 0.01 * k)
    out = torch.empty_like(proj)
    st = torch.cuda.current_stream(dev)
    direct = [t[:nth] for t in tiles]
    mirror = [t[nth:] for t in tiles]

    def timed(fn, steps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            fn()
        e1.record(st)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / steps

    ms_stitch = timed(lambda: mt.stitch_into(direct, mirror, out), args.steps)
    ms_extract = timed(lambda: mt.extract_into(proj, direct, mirror), args.steps)
    tile_px = sum(2 * nth * h * w for h, w in mt.shapes)
    out_px = nth * nz * n
    b_stitch = 4 * (tile_px + out_px)
    b_extract = 8 * tile_px
    peak, peak_kind = peaks()
    gbs = b_stitch / (ms_stitch * 1e-3) / 1e9
    gbs_x = b_extract / (ms_extract * 1e-3) / 1e9
    del proj
    # e2e: 8 angles through pinned host memory
    ne = 8
    mt8 = mo.MosaicTiles(dict(meta, N_HALF=ne, NTHETA=2 * ne), pl)
    host_tiles = [torch.cat([t[:ne], t[nth:nth + ne]]).cpu().pin_memory() for t in tiles]
    del tiles, direct, mirror, out
    dev_tiles = [torch.empty(t.shape, dtype=torch.float32, device=dev) for t in host_tiles]
    out8 = torch.empty((ne, nz, n), dtype=torch.float32, device=dev)
    host_out = torch.empty((ne, nz, n), dtype=torch.float32).pin_memory()

    def e2e():
        for hsrc, dd in zip(host_tiles, dev_tiles):
            dd.copy_(hsrc, non_blocking=True)
        mt8.stitch(dev_tiles, 0, ne, out=out8)
        host_out.copy_(out8, non_blocking=True)

    ms_e2e = timed(e2e, max(2, args.steps // 2))
    h2d = sum(t.numel() * 4 for t in host_tiles)
    # CPU: the reference's NumPy blend on 2 angles of the same mosaic
    import time
    s = 2
    tiles_np = [np.concatenate([t[:s].numpy(), t[ne:ne + s].numpy()]) for t in host_tiles]
    t0 = time.perf_counter()
    om.stitch(tiles_np, pl, nz, n, s, meta["OVERLAP"], 0, s)
    t_cpu = time.perf_counter() - t0
    mt.free()
    mt8.free()
    return {"metric": "mosaic stitch Gpix/s", "workload": "stitch",
            "value": round(out_px / (ms_stitch * 1e-3) / 1e9, 3), "unit": "Gpix/s",
            "ms_per_step": round(ms_stitch, 3), "steps": args.steps, "warmup": args.warmup,
            "roofline": {"bound": "hbm", "kernel": "k_stitch", "achieved": round(gbs, 1), "peak": peak,
                         "peak_source": peak_kind, "unit": "GB/s", "frac": round(gbs / peak, 4),
                         "traffic": profile_traffic("stitch", "k_stitch") if (args.ups, nth) == (2, 64) else None,
                         "alg_bytes_per_launch": b_stitch},
            "extract": {"ms": round(ms_extract, 3), "gbs": round(gbs_x, 1), "frac": round(gbs_x / peak, 4),
                        "alg_bytes_per_launch": b_extract, "kernel": "k_extract"},
            "e2e": {"value": round(ne * nz * n / (ms_e2e * 1e-3) / 1e9, 3), "unit": "Gpix/s",
                    "ms_per_step": round(ms_e2e, 3), "angles": ne, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": ne * nz * n * 4},
            "cpu_baseline": {"value": round(s * nz * n / t_cpu / 1e9, 5), "unit": "Gpix/s", "cores": 1,
                             "kind": "port", "sample": f"the reference's NumPy blend, {s} output angles"},
            "gpu_launches": args.steps,
            "config": {"mosaic": f"ups {args.ups}: {nz} x {n}, {meta['n_z']} x {meta['n_x']} tiles of "
                                 f"{meta['DET_H']} x {meta['DET_W']}, overlap {meta['OVERLAP']}", "angles": nth,
                       "tile_gb": round(4 * tile_px / 1e9, 2), "out_gb": round(4 * out_px / 1e9, 2),
                       "l2": "inputs far larger than L2; no flush",
                       "data": "synthetic 0.5 + U[0, 1) projection, per-tile gains 1 + 0.01 k"}}


# ---------------------------------------------------------------- precision report
def run_precision(args, local_rank):
    """Relative L2 error against the FP64 oracle, per precision variant: float32
    storage and arithmetic; bfloat16 storage of volume and sinogram with float32
    arithmetic; Kahan-compensated adjoint scatter.  R and RT on a 64-slice slab
    of the 1024^3 seeded volume at 1536 angles on [0, pi) (oracle on 2 of its
    slices), D on 8 of the slab's frames, the model gradient on 128^3 with 192
    angles (the FP64 oracle of the full 1024^3 model does not fit a host run)."""
    import torch
    from model_mosaic_b200.model import ForwardModel
    from model_mosaic_b200.phantom import ellipsoid_volume, ellipsoid_volume_torch
    from model_mosaic_b200.processing.propagation import Propagation
    from model_mosaic_b200.processing.tomo import TomoReal
    from oracle.fresnel import PropagationOracle, psi_from_proj
    from oracle.model import ModelOracle
    from oracle.usfft import TomoRealOracle

    def rl2(a, b):
        a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) else np.float64)
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    dev = torch.device("cuda", local_rank)
    w = WORKLOADS["production"]
    wl = 1.24e-9 / w["energy_kev"]
    n, T, z0, nzs = 1024, 1536, 480, 64
    theta = np.linspace(0, np.pi, T, endpoint=False).astype(np.float32)
    pick = [0, 42]
    x = ellipsoid_volume_torch(n, 1024, seed=0, device=dev)[z0:z0 + nzs].contiguous()
    tomo = TomoReal(n, nzs, theta)
    tomo_k = TomoReal(n, nzs, theta, compensated=True)
    ora = TomoRealOracle(n, len(pick), theta)
    xh = x[pick].cpu().numpy()
    ref_r = ora.R(xh)
    r32 = tomo.R(x)
    rbf = tomo.R(x.to(torch.bfloat16))
    rep = {"R": {"float32": rl2(r32[:, pick].cpu().numpy(), ref_r),
                 "bfloat16_storage": rl2(rbf[:, pick].float().cpu().numpy(), ref_r)}}
    y = r32
    ref_rt = ora.RT(y[:, pick].cpu().numpy())
    rep["RT"] = {"float32": rl2(tomo.RT(y)[pick].cpu().numpy(), ref_rt),
                 "bfloat16_storage": rl2(tomo.RT(y.to(torch.bfloat16))[pick].float().cpu().numpy(), ref_rt),
                 "kahan_scatter": rl2(tomo_k.RT(y)[pick].cpu().numpy(), ref_rt)}
    s, ib = float(np.float32(1.0 / np.sqrt(n / T))), 0.01
    p = (r32[:8] * (1.5 / float(r32.abs().max()))).cpu().numpy()          # phases up to 1.5 rad
    psi = psi_from_proj(p, s, ib)
    prop = Propagation(n, nzs, 8, 1, wl, w["voxelsize"], [w["distance"]])
    ref_d = PropagationOracle(n, nzs, 8, 1, wl, w["voxelsize"], [w["distance"]]).D(psi, 0)
    rep["D"] = {"float32": rl2(prop.D(torch.from_numpy(psi.astype(np.complex64)).to(dev), 0).cpu().numpy(), ref_d)}
    ng, tg = 128, 192
    thg = np.linspace(0, np.pi, tg, endpoint=False).astype(np.float32)
    dg = ellipsoid_volume(ng, ng, seed=0, vmin=0.2, vmax=1.0)
    dg2 = ellipsoid_volume(ng, ng, seed=1, vmin=0.2, vmax=1.0)
    sg = float(np.float32(1.5 / np.abs(ModelOracle(ng, ng, thg, wl, w["voxelsize"], w["distance"], s=1.0)
                                        .tomo.R(dg)).max()))
    mo = ModelOracle(ng, ng, thg, wl, w["voxelsize"], w["distance"], s=sg)
    data = mo.forward(dg2)
    gref = mo.grad(dg, data)
    rep["gradient"] = {}
    for name, comp in (("float32", False), ("kahan_scatter", True)):
        m = ForwardModel(ng, ng, thg, wl, w["voxelsize"], w["distance"], inv_norm=sg, angle_chunk=64,
                         compensated=comp)
        _, g = m.loss_and_grad(torch.from_numpy(dg).to(dev), torch.from_numpy(data.astype(np.float32)).to(dev))
        rep["gradient"][name] = rl2(g.cpu().numpy(), gref)
    rep = {k: {v: float(f"{e:.3e}") for v, e in d.items()} for k, d in rep.items()}
    return {"precision_report": rep,
            "config": {"R_RT": f"slices {z0}..{z0 + nzs - 1} of the seeded 1024^3 volume, {T} angles on [0, pi), "
                               f"oracle on slices {[z0 + q for q in pick]}",
                       "D": f"8 frames of {nzs}x{n} from those projections (phase scaled to 1.5 rad)",
                       "gradient": f"{ng}^3, {tg} angles, FP64 oracle",
                       "bfloat16_storage": "inputs and outputs stored as bfloat16, float32 arithmetic; "
                                           "D and the gradient kernels take float32 only"}}


# ---------------------------------------------------------------- GPU (reference kernels on this GPU)
def ref_gpu_ops(args, w, local_rank):
    """Baseline leg: the reference's own CUDA kernels (processing/kernels.py,
    compiled verbatim for sm_100a by oracle/build_ref.py) with its cupy host
    glue restated on torch/cuFFT (oracle/refgpu.py), timed on this GPU at the
    workload's size: R, RT and psi -> D -> |.|^2 of all projections."""
    import torch
    from oracle import refgpu
    if not refgpu.available():
        return {"unavailable": "oracle/_ref/libref_gpu.so not built (reference tree absent at build time)"}
    from model_mosaic_b200.phantom import ellipsoid_volume_torch
    torch.cuda.empty_cache()
    dev = torch.device("cuda", local_rank)
    n, nz, T = w["n"], w["nz"], w["ntheta"]
    theta = np.linspace(0, w["theta_max"], T, endpoint=False).astype(np.float32)
    inv_norm = float(np.float32(1.0 / np.sqrt(n / T)))
    inv_beta = float(np.float32(1.0 / BETA_RATIO))
    st = torch.cuda.current_stream()

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    obj = ellipsoid_volume_torch(n, nz, seed=0, device=dev)
    tomo = refgpu.RefGpuTomoReal(n, nz, theta, device=dev)
    sino = tomo.R(obj)
    r_ms = timed(lambda: tomo.R(obj))
    rt_ms = timed(lambda: tomo.RT(sino))
    del tomo
    torch.cuda.empty_cache()
    prop = refgpu.RefGpuPropagation(n, nz, T, 1, 1.24e-9 / w["energy_kev"], w["voxelsize"], [w["distance"]],
                                    device=dev)
    d_ms = timed(lambda: refgpu.abs2(prop.D(refgpu.psi_from_proj(sino, inv_norm, inv_beta), 0)))
    del prop, sino, obj
    torch.cuda.empty_cache()
    return {"R_ms": round(r_ms, 3), "RT_ms": round(rt_ms, 3), "D_ms": round(d_ms, 3),
            "step_ms": round(r_ms + d_ms, 3),
            "what": "the reference's kernels (processing/kernels.py) compiled for sm_100a with its host glue "
                    "(processing/tomo.py, propagation.py, step3 psi/|.|^2) on torch/cuFFT, CUDA events, "
                    "1 warm-up + 3 timed calls"}


# ---------------------------------------------------------------- CPU (reference kernels on the host)
def cpu_sample(w, slices=1, frames=32, cores=None):
    """Time the reference's kernels + restated glue on a bounded sample and
    scale to one full step.  Returns (seconds per full step, description)."""
    from oracle.refkernels import RefTomoReal, RefPropagation, available
    from model_mosaic_b200.phantom import ellipsoid_volume
    cores = cores or os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    n, nz, T = w["n"], w["nz"], w["ntheta"]
    theta = np.linspace(0, w["theta_max"], T, endpoint=False).astype(np.float32)
    x = ellipsoid_volume(n, nz, seed=0, z0=nz // 2, z1=nz // 2 + slices)
    tomo = RefTomoReal(n, slices, theta, workers=cores)
    wavelength = 1.24e-9 / w["energy_kev"]
    prop = RefPropagation(n, nz, frames, 1, wavelength, w["voxelsize"], [w["distance"]], workers=cores)
    frame = np.ascontiguousarray(
        np.broadcast_to(ellipsoid_volume(n, 1, seed=1)[0][:nz][None], (frames, nz, n)).astype(np.float32))
    t0 = time.perf_counter()
    tomo.R(x)
    t1 = time.perf_counter()
    inv_norm = np.float32(1.0 / np.sqrt(n / T))
    phase = frame * inv_norm
    psi = (np.exp(-phase / BETA_RATIO) * (np.cos(phase) + 1j * np.sin(phase))).astype(np.complex64)
    u = prop.D(psi, 0)
    _ = (u.real * u.real + u.imag * u.imag)
    t2 = time.perf_counter()
    t_step = (t1 - t0) * (nz / slices) + (t2 - t1) * (T / frames)
    kind = "reference" if available() else "port"
    desc = (f"R of {slices} of {nz} slices and psi/D/|.|^2 of {frames} of {T} frames, scaled linearly "
            f"to the full step; reference kernels (processing/kernels.py) built for the host with "
            f"OpenMP, SciPy FFT workers={cores}")
    return t_step, desc, kind, cores


def run_reference(args, w):
    n, nz, T = w["n"], w["nz"], w["ntheta"]
    V = nz * n * n
    for _ in range(args.warmup):
        cpu_sample(w)
    ts = []
    desc = kind = cores = None
    for _ in range(args.steps):
        t, desc, kind, cores = cpu_sample(w)
        ts.append(t)
    t = statistics.median(ts)
    value = V * T / t / 1e9
    return {"metric": "R/RT Gvox·angle/s", "value": round(value, 5), "unit": "Gvox·angle/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t * 1e3, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: 10 seeded random ellipsoids (values in [1e-7, 1e-6], beta = delta/100)",
            "config": {"workload": workload_desc(w, args.workload), "n": n, "nz_per_rank": nz, "ntheta": T},
            "cpu_baseline": {"value": round(value, 5), "unit": "Gvox·angle/s", "cores": cores, "kind": kind,
                             "sample": desc},
            "e2e": {"value": round(value, 5), "unit": "Gvox·angle/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["tiles", "fbp", "paganin", "stitch"], default="production")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-rt", action="store_true", help="skip the adjoint (no scatter table)")
    ap.add_argument("--no-model", action="store_true", help="skip the fwd+grad timing of the model")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="skip the baseline legs that time the reference's own kernels on the GPU")
    ap.add_argument("--base", choices=sorted(WORKLOADS), default="production",
                    help="sizes for the fbp and paganin workloads (frames / sinogram of this workload)")
    ap.add_argument("--ups", type=int, default=2, help="stitch workload: mosaic of this upsampling factor")
    ap.add_argument("--angles", type=int, default=64, help="stitch workload: output angles per step (>= 8)")
    ap.add_argument("--precision", action="store_true",
                    help="print the precision report (errors vs the FP64 oracle per variant) instead of timing")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    w = WORKLOADS.get(args.workload)
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))

    if args.impl == "reference":
        if rank == 0:
            if w is None:
                print(json.dumps({"impl": "reference", "unavailable": f"the {args.workload} workload is timed on "
                                                                      "the GPU arm only"}), flush=True)
            else:
                print(json.dumps(run_reference(args, w)), flush=True)
        return
    if args.precision:
        if rank == 0:
            print(json.dumps(run_precision(args, local_rank)), flush=True)
        return
    if args.workload == "tiles":
        if rank == 0:
            print(json.dumps(run_tiles(args, local_rank)), flush=True)
        return
    if args.workload == "fbp":
        if rank == 0:
            print(json.dumps(run_fbp(args, local_rank)), flush=True)
        return
    if args.workload == "paganin":
        if rank == 0:
            print(json.dumps(run_paganin(args, local_rank)), flush=True)
        return
    if args.workload == "stitch":
        if rank == 0:
            print(json.dumps(run_stitch(args, local_rank)), flush=True)
        return

    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    try:
        line = run_ours(args, w, rank, world, local_rank)
        if args.workload == "production" and not args.no_model:
            line["model_fwd_grad"] = run_model(args, local_rank)
        if rank == 0 and world == 1 and args.workload == "production" and not args.no_ref_gpu:
            ref = ref_gpu_ops(args, w, local_rank)
            if "R_ms" in ref:
                ops = line["ops"]
                ref["speedup"] = {"R": round(ref["R_ms"] / ops["R_ms"], 3),
                                  "RT": round(ref["RT_ms"] / ops["RT_ms"], 3) if ops["RT_ms"] else None,
                                  "D": round(ref["D_ms"] / ops["D_ms"], 3),
                                  "step": round(ref["step_ms"] / line["ms_per_step"], 3)}
            line["reference_gpu"] = ref
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            t, desc, kind, cores = cpu_sample(w)
            V = w["nz"] * w["n"] ** 2
            line["cpu_baseline"] = {"value": round(V * w["ntheta"] / t / 1e9, 5), "unit": "Gvox·angle/s",
                                    "cores": cores, "kind": kind, "sample": desc}
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
