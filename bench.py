"""Benchmark of the elastic staggered-grid time loop on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config config2|config1|config3]

One bench step is one complete forward modelling run of the configuration:
zero the state, nt time steps (velocity + stress passes, source injection,
receiver sampling), inputs already resident in HBM.  Default workload
(config2): 3D homogeneous SSG-CPML 200^3, dx=10 m, dt=1 ms, 1000 time steps,
20-cell CPML, double-couple (30/60/90) 15 Hz Ricker2 source, 50x50 receivers,
fp32.  The state (~0.56 GB) is larger than L2, so no L2 flush is needed.

Metric: Gcell-updates/s = cells * time steps / device time (max over ranks,
whole job).  Multi-GPU runs are independent replicas (one shot per GPU):
the forward loop of one model has no data-path exchange.

`e2e` is the same metric through the public drop-in API with host buffers:
each step copies the model (vp, vs, rho) from pinned host memory into the
solver, runs the nt steps and reads the seismogram back into pinned memory.

`--impl reference` times the reference's scheme on the host CPU: the
SeisWave_Taichi Taichi package is not installable here, so its CPU arm is the
C++/OpenMP restatement of the same kernels (oracle/), run on every host core
on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FALLBACK_HBM_GBS = 6650.0

# dram__bytes_read.sum + dram__bytes_write.sum of one k_segy_decode<1> launch
# at 8192 x 16000 IBM samples
SEGY_NCU_TRAFFIC = (525.916672 + 482.566656) * 1e6
# DRAM bytes per time step (velocity + stress launch pair at step 700, default
# path and exact numerics) from one ncu capture of the full workload (profiles/).
NCU_TRAFFIC_PER_STEP = {"3d-ssg-cpml-tensor-200^3-nt1000": (435.430144 + 125.214464 + 483.239680 + 209.421568) * 1e6}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """Samples nvidia-smi clocks/throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"),
                               parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def build_solver(cfg, torch, exact=True, dtype=None, coef64=False):
    if cfg.get("scheme") == "SPML":
        from seiswave_taichi_b200.Elastic3D_SSG_SPML import ElasticWAVE as SPML
        w = SPML(cfg["vs"], cfg["vp"], cfg["rho"], cfg["dx"], cfg["dy"], cfg["dz"], cfg["dt"], cfg["isx"],
                 cfg["isy"], cfg["isz"], cfg["rsx"], cfg["rsy"], cfg["rsz"], cfg["nt"], cfg["accuracy"], cfg["freq"],
                 cfg["src_scale"], dtype or torch.float32, exact=exact, coef64=coef64)
        w.SetADEPML3D(cfg["surface"], cfg["pml"])
        return w
    from seiswave_taichi_b200.Elastic3D_SSG_Tensor import ElasticWAVE
    w = ElasticWAVE(cfg["vs"], cfg["vp"], cfg["rho"], cfg["dx"], cfg["dy"], cfg["dz"], cfg["dt"],
                    cfg["isx"], cfg["isy"], cfg["isz"], cfg["rsx"], cfg["rsy"], cfg["rsz"], cfg["MT"],
                    cfg["src_scale"], cfg["nt"], cfg["accuracy"], cfg["freq"], dtype or torch.float32, exact=exact,
                    coef64=coef64)
    w.SetADEPML3D(cfg["surface"], cfg["pml"])
    return w


def build_solver2d(cfg, torch, dtype=None, coef64=False):
    from seiswave_taichi_b200.Elastic2D_CPML import ElasticWAVE
    w = ElasticWAVE(cfg["vs"], cfg["vp"], cfg["rho"], cfg["dx"], cfg["dz"], cfg["dt"], cfg["isx"],
                    cfg["isz"], cfg["rsx"], cfg["rsz"], cfg["nt"], cfg["accuracy"], cfg["freq"],
                    dtype or torch.float32, MT=cfg.get("MT"), src_scale=cfg.get("src_scale", 1.0), coef64=coef64)
    w.SetADEPML2D(cfg["surface"], cfg["pml"])
    return w


def fp64_error(cfg, w32, torch):
    """Relative L2 error of the f32 run's traces and final vx against float64
    runs of the same scheme: with the f32-rounded stencil coefficients (the
    reference's own f64 mode) and with float64 coefficients."""
    three_d = len(cfg["shape"]) == 3
    out = {}
    for tag, c64 in (("f64_run_f32_coef", False), ("f64_run_f64_coef", True)):
        w = (build_solver(cfg, torch, dtype=torch.float64, coef64=c64) if three_d
             else build_solver2d(cfg, torch, dtype=torch.float64, coef64=c64))
        w.run(cfg["nt"])
        torch.cuda.synchronize()
        d64, d32 = w.data.double(), w32.data.double()
        v64, v32 = w.vx.double(), w32.vx.double()
        out[tag] = {"traces_rel_l2": float(torch.linalg.norm(d32 - d64) / torch.linalg.norm(d64)),
                    "final_vx_rel_l2": float(torch.linalg.norm(v32 - v64) / torch.linalg.norm(v64))}
        del w
    return out


def spml_config():
    """The split-field PML scheme on config 2's grid: 200^3 homogeneous,
    dx = 10 m, dt = 1 ms, 1000 steps, N = 2, 20-cell PML, a 15 Hz point force
    (the scheme's source, Elastic3D_SSG_SPML.py:294) at the centre, one vx
    receiver (:393)."""
    from seiswave_taichi_b200 import synthetic as S
    c = dict(S.config2())
    n = c["shape"][0]
    c.update(name=f"3d-ssg-spml-{n}^3-nt{c['nt']}", scheme="SPML", rsx=n // 2 - 30, rsy=n // 2, rsz=c["accuracy"] + 5,
             src_scale=1.0e6, MT=None)
    return c


def algorithmic_bytes(cfg, npml=20):
    """Fused minimum bytes per time step: every wavefield read and written
    once, the material read once, and each CPML memory variable read and
    written once on its slabs: 3D 84*N + 48*(S_x+S_y+S_z), 2D 52*N + 32*(S_x+S_z),
    S_d = 2*npml*(product of the other two extents)."""
    shape = cfg["shape"]
    ncell = int(np.prod(shape))
    if cfg.get("scheme") == "SPML":
        # 84 B/cell + 24 split fields read and written on the PML cells
        nx, ny, nz = shape
        npml_cells = ncell - (nx - 2 * npml) * (ny - 2 * npml) * (nz - 2 * npml)
        return 84 * ncell + 8 * 24 * npml_cells
    if len(shape) == 3:
        nx, ny, nz = shape
        S = 2 * npml * (ny * nz + nx * nz + nx * ny)
        return 84 * ncell + 48 * S
    nx, nz = shape
    S = 2 * npml * (nz + nx)
    return 52 * ncell + 32 * S


def oracle_for(cfg):
    """The CPU oracle (C++/OpenMP restatement of the reference kernels) set up
    for workload cfg, and a function advancing it by n time steps from it."""
    from oracle import oracle as O
    if len(cfg["shape"]) == 3:
        o = O.Oracle3D(cfg.get("scheme", "TENSOR"), cfg["vs"], cfg["vp"], cfg["rho"], cfg["dx"], cfg["dy"],
                       cfg["dz"], cfg["dt"], cfg["isx"], cfg["isy"], cfg["isz"], cfg["rsx"], cfg["rsy"], cfg["rsz"],
                       cfg["nt"], cfg["accuracy"], cfg["freq"], cfg["surface"], cfg["pml"], MT=cfg["MT"],
                       src_scale=cfg["src_scale"])
        return lambda it, n: o.run(it, n)
    from seiswave_taichi_b200 import BaseFun
    from seiswave_taichi_b200.Elastic2D_CPML import moment_2d
    wav = BaseFun.series("ricker2", cfg["nt"], cfg["dt"], cfg["freq"], cfg.get("src_scale", 1.0),
                         t0=np.float32(1.5 / float(cfg["freq"])))
    table = cfg["rsx"].reshape(-1) * cfg["shape"][1] + cfg["rsz"].reshape(-1)
    o = O.Oracle2D(cfg["vs"], cfg["vp"], cfg["rho"], cfg["dx"], cfg["dz"], cfg["dt"], cfg["isx"], cfg["isz"],
                   int(cfg["rsx"].reshape(-1)[0]), int(cfg["rsz"].reshape(-1)[0]), cfg["nt"],
                   cfg["accuracy"], cfg["freq"], cfg["surface"], cfg["pml"], wavelet=wav,
                   MT=moment_2d(cfg["MT"]) if cfg.get("MT") is not None else None, rec_index=table)
    return lambda it, n: o.run("VS", it, n)


# above this many cell updates a whole CPU run would take too long for one
# bench invocation (config 3: 6.4e10); the sample is then the run's first steps
CPU_FULL_RUN_MAX_UPDATES = 2.0e10


def cpu_segments(cfg, nseg: int):
    """Time the oracle over the workload's time loop from rest, split into nseg
    consecutive segments: [(time steps, seconds)].  The whole loop of nt steps
    is run when it has at most CPU_FULL_RUN_MAX_UPDATES cell updates, else
    its first steps up to that many."""
    from oracle import oracle as O
    O.set_threads(os.cpu_count() or 1)
    ncell = int(np.prod(cfg["shape"]))
    total = min(cfg["nt"], max(1, int(CPU_FULL_RUN_MAX_UPDATES // ncell)))
    nseg = max(1, min(int(nseg), total))
    step = oracle_for(cfg)
    bounds = [round(total * q / nseg) for q in range(nseg + 1)]
    out = []
    for a, b in zip(bounds[:-1], bounds[1:]):
        t0 = time.perf_counter()
        step(a, b - a)
        out.append((b - a, time.perf_counter() - t0))
    return out, total


def cpu_sample_text(cfg, total, seconds):
    run = "all" if total == cfg["nt"] else "the first"
    return (f"{run} {total} of the {cfg['nt']} time steps of the full {'x'.join(map(str, cfg['shape']))} grid "
            f"from rest ({seconds:.1f} s; C++/OpenMP oracle restating the reference kernels, "
            f"bit-identical to them)")


def cpu_baseline(cfg):
    """The oracle on all host cores over the workload's time loop (one run,
    timed whole; see cpu_segments for the cap)."""
    segs, total = cpu_segments(cfg, 1)
    el = sum(t for _, t in segs)
    ncell = int(np.prod(cfg["shape"]))
    return {"value": ncell * total / el / 1e9, "unit": "Gcell-updates/s", "cores": os.cpu_count() or 1,
            "kind": "port", "sample": cpu_sample_text(cfg, total, el)}


def workload_config(cfg, world):
    """The `config` object of both arms' JSON lines (identical by construction)."""
    three_d = len(cfg["shape"]) == 3
    return {"workload": cfg["name"], "grid": list(cfg["shape"]), "time_steps": cfg["nt"],
            "accuracy": cfg["accuracy"], "parallelism": f"replicas{world}",
            "l2": "state larger than L2 (no flush needed)" if three_d else
                  "state fits in L2 (2D 400^2); %HBM not meaningful"}


def get_config(name):
    from seiswave_taichi_b200 import synthetic as S
    if name == "config2":
        return S.config2()
    if name == "config1":
        return S.config1()
    if name == "config3":
        return S.config3()
    if name == "spml":
        return spml_config()
    raise SystemExit(f"unknown config {name}")


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    if args.config == "segy":
        # segyio (the reference's decoder) is absent: the numpy oracle, one core
        sys.path.insert(0, str(ROOT))
        from oracle import segy_ref
        ntr, ns = 512, 16000
        rec = 240 + 4 * ns
        body = np.random.default_rng(0).integers(0, 256, ntr * rec, dtype=np.uint8)
        vals = []
        for s_ in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            segy_ref.decode(body, ntr, ns, 1)
            if s_ >= args.warmup:
                vals.append(ntr * rec / (time.perf_counter() - t0) / 1e9)
        v = float(np.mean(vals))
        print(json.dumps({
            "impl": "reference", "metric": "GB/s", "value": v, "unit": "GB/s (SEG-Y input decoded)",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ntr * rec / v / 1e6,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8->f32",
            "data": "synthetic", "config": {"workload": f"segy-ibm-{ntr}x{ns} (bounded sample)"},
            "cpu_baseline": {"value": v, "unit": "GB/s", "cores": 1, "kind": "port",
                             "sample": f"{ntr} traces of {ns} IBM samples per step, numpy oracle"},
            "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)
        return 0
    cfg = get_config(args.config)
    ncell = int(np.prod(cfg["shape"]))
    # warm-up: short runs from rest (caches, page faults, thread pool), untimed
    for _ in range(args.warmup):
        oracle_for(cfg)(0, 2)
    # timed: the time loop from rest split into `steps` consecutive segments,
    # so the timed region is one whole run (or its capped prefix)
    segs, total = cpu_segments(cfg, args.steps)
    el = sum(t for _, t in segs)
    v = ncell * total / el / 1e9
    line = {
        "impl": "reference", "metric": "Gcell-updates/s", "value": v, "unit": "Gcell-updates/s",
        "n_gpus": world, "steps": len(segs), "warmup": args.warmup, "ms_per_step": el / len(segs) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(cfg, world),
        "cpu_baseline": {"value": v, "unit": "Gcell-updates/s", "cores": os.cpu_count() or 1, "kind": "port",
                         "sample": cpu_sample_text(cfg, total, el) + f", timed as {len(segs)} segments"},
        "e2e": {"value": v, "unit": "Gcell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def max_over_ranks(ms: float, dist, device="cuda") -> float:
    """The slowest rank's device time: every rank takes part, in the same
    order, and gets the maximum (a no-op on one process)."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_value(world: int, ncell: int, nt: int, steps: int, ms: float) -> float:
    """Gcell-updates/s of the whole job: every rank runs its own replica of
    the workload (weak scaling), timed by the slowest rank."""
    return world * ncell * nt * steps / (ms * 1e-3) / 1e9


def run_batch(args, rank, world, local):
    """Batched ragged 2D workload (config4: 64 shots, 1500 steps): one step
    is one batched forward run of every shot from rest (value: whole-job
    Gcell-updates/s; shots/s beside it); then one FWI gradient step
    (batched forward with checkpoints every 100 steps + every shot's
    adjoint) is timed once."""
    import torch
    from seiswave_taichi_b200 import synthetic as S
    from seiswave_taichi_b200.Elastic2D_CPML import ElasticWAVE
    from seiswave_taichi_b200.fwi import FWIStep
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    shots = S.config4(seed=rank)
    waves = []
    for c in shots:
        w = ElasticWAVE(c["vs"], c["vp"], c["rho"], c["dx"], c["dz"], c["dt"], c["isx"], c["isz"], c["rsx"],
                        c["rsz"], c["nt"], c["accuracy"], c["freq"], torch.float32, MT=c["MT"],
                        src_scale=c["src_scale"])
        w.SetADEPML2D(c["surface"], c["pml"])
        waves.append(w)
    nt = shots[0]["nt"]
    cells = sum(w.gridsize[0] * w.gridsize[1] for w in waves)
    step = FWIStep(waves, checkpoint_every=100)
    b = step.batch
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        b.reset()
        b.run()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            b.reset()
            b.run()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), dist)
    value = whole_job_value(world, cells, nt, args.steps, ms)
    # the same shots one after the other, each through its own cached graph
    for w in waves:
        w.reset()
        w.run(nt)
    torch.cuda.synchronize()
    e0.record(stream)
    for w in waves:
        w.reset()
        w.run(nt)
    e1.record(stream)
    torch.cuda.synchronize()
    seq_ms = max_over_ranks(e0.elapsed_time(e1), dist)
    # error of the batched float32 forward against float64 runs of the same
    # scheme (the first four shots, one by one)
    err64 = None
    if rank == 0 and not args.no_fp64:
        tr, fv = [], []
        for c, w32 in list(zip(shots, waves))[:4]:
            w64 = ElasticWAVE(c["vs"], c["vp"], c["rho"], c["dx"], c["dz"], c["dt"], c["isx"], c["isz"],
                              c["rsx"], c["rsz"], c["nt"], c["accuracy"], c["freq"], torch.float64, MT=c["MT"],
                              src_scale=c["src_scale"])
            w64.SetADEPML2D(c["surface"], c["pml"])
            w64.run(nt)
            torch.cuda.synchronize()
            for dst, a32, a64 in ((tr, w32.data, w64.data), (fv, w32.vx, w64.vx)):
                dst.append(float(torch.linalg.norm(a32.double() - a64) / torch.linalg.norm(a64)))
            del w64
        err64 = {"shots": len(tr), "traces_rel_l2_max": max(tr), "final_vx_rel_l2_max": max(fv),
                 "against": "float64 runs of the same scheme (f32 stencil coefficients, as the reference's f64 mode)"}
    # end to end: observed traces from host memory in, misfit gradient out
    d_obs = [w.data.detach().cpu().pin_memory() for w in waves]
    h2d = sum(t.numel() * t.element_size() for t in d_obs)
    d2h = 3 * 4 * cells

    def fwi_once():
        obs = [t.to("cuda", non_blocking=True) * 1.01 for t in d_obs]
        _, grads = step(obs)
        return [tuple(g.to("cpu", non_blocking=True) for g in gs) for gs in grads]

    fwi_once()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0.record(stream)
    fwi_once()
    e1.record(stream)
    torch.cuda.synchronize()
    fwi_ms = max_over_ranks(e0.elapsed_time(e1), dist)
    if rank == 0:
        info = b.info()
        line = {
            "metric": "Gcell-updates/s", "value": value, "unit": "Gcell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"2d-batch-{len(waves)}shots-nt{nt}", "shots": len(waves), "cells": cells,
                       "time_steps": nt, "accuracy": 2, "parallelism": f"replicas{world}", "tile": info,
                       "l2": "batch state (~1.2 GB) larger than L2"},
            "shots_per_s": world * len(waves) * args.steps / (ms * 1e-3),
            "sequential": {"value": whole_job_value(world, cells, nt, 1, seq_ms), "unit": "Gcell-updates/s",
                           "shots_per_s": world * len(waves) / (seq_ms * 1e-3),
                           "what": "the same shots one after the other, each from its own cached CUDA graph"},
            "fwi_step": {"ms": fwi_ms, "checkpoint_every": 100,
                         "what": "batched forward with checkpoints + 64 per-shot adjoints + gradient chain, "
                                 "observed traces from pinned host memory, gradients back to the host"},
            "e2e": {"value": whole_job_value(world, cells, nt, 1, fwi_ms), "unit": "Gcell-updates/s (FWI step: "
                    "forward cell updates per second of the whole gradient step)", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": args.steps * (2 * nt + 1),
            "clocks": clk.summary(),
            "cpu_baseline": None,
            "fp64_error": err64,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_segy(args, rank, world, local):
    """SEG-Y ingestion (`--config segy`): a file of 8192 traces of 16000
    IBM-float samples (0.53 GB of seeded synthetic bytes: normal amplitudes
    over several orders of magnitude, SourceX in each trace header) decoded
    to float32 with sw_segy_decode, 20 decodes per step.  value: GB/s of
    SEG-Y input decoded with the bytes already in HBM; e2e: one file per
    step through pinned host memory (host-to-device copy of the bytes,
    decode, device-to-host read of the float samples)."""
    import ctypes as C
    import torch
    from seiswave_taichi_b200 import _native as N
    from seiswave_taichi_b200.ReadSegy import decode_traces
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    ntr, ns, fmt = 8192, 16000, 1
    rec = 240 + 4 * ns
    rng = np.random.default_rng(rank)
    body = np.empty((ntr, rec), np.uint8)
    # recorded amplitudes: normal values of a few orders of magnitude, as IBM
    # words (fraction truncated) written big-endian
    amp = rng.standard_normal((ntr, ns)) * np.exp(rng.uniform(-8.0, 8.0, (ntr, 1)))
    m, p2 = np.frexp(np.abs(amp))
    q = -((-p2) // 4)
    f = np.floor(np.ldexp(m, p2 - 4 * q + 24)).astype(np.uint32)
    w = (np.signbit(amp).astype(np.uint32) << 31) | ((q + 64).astype(np.uint32) << 24) | f
    w[amp == 0] = 0
    body[:, 240:] = w.astype(">u4").view(np.uint8).reshape(ntr, 4 * ns)
    del amp, m, p2, q, f, w
    body[:, :240] = 0
    body[:, 72:76] = np.arange(ntr, dtype=">i4").view(np.uint8).reshape(ntr, 4)
    host = torch.from_numpy(body.reshape(-1)).pin_memory()
    dev = host.to("cuda")
    nbytes = host.numel()
    out_host = torch.empty((ntr, ns), dtype=torch.float32).pin_memory()
    stream = torch.cuda.current_stream()
    # warm-up: at least the requested steps and 0.3 s of decoding, so that the
    # clocks have left their idle state before the timed region
    reps = 20  # decodes of the file per timed step
    t_end = time.perf_counter() + 0.3
    n_warm = 0
    while n_warm < max(3, args.warmup) * reps or time.perf_counter() < t_end:
        decode_traces(dev, ntr, ns, fmt)
        n_warm += 1
        if n_warm % reps == 0:
            torch.cuda.synchronize()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps * reps):
            out, _ = decode_traces(dev, ntr, ns, fmt)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), dist) / args.steps
    value = world * nbytes * reps / (ms * 1e-3) / 1e9
    # end to end: file bytes from pinned host memory in, float samples out
    e0.record(stream)
    for _ in range(args.steps):
        d = host.to("cuda", non_blocking=True)
        o, _ = decode_traces(d, ntr, ns, fmt)
        out_host.copy_(o, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1), dist) / args.steps
    peak, peak_kind = peaks()
    moved = nbytes + 4 * ntr * ns
    ms_launch = ms / reps
    line = None
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline:
            sys.path.insert(0, str(ROOT))
            from oracle import segy_ref
            k = 512
            t0 = time.perf_counter()
            reps = 0
            while time.perf_counter() - t0 < 10.0:
                segy_ref.decode(body[:k].reshape(-1), k, ns, fmt)
                reps += 1
            sec = time.perf_counter() - t0
            cpu = {"value": reps * k * rec / sec / 1e9, "unit": "GB/s", "cores": 1, "kind": "port",
                   "sample": f"{reps} decodes of {k} traces ({k * rec / 1e6:.0f} MB) with the numpy oracle"}
        line = {
            "metric": "GB/s", "value": value, "unit": "GB/s (SEG-Y input decoded)", "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8->f32", "data": "synthetic",
            "config": {"workload": f"segy-ibm-{ntr}x{ns}", "traces": ntr, "samples": ns, "format": "IBM float",
                       "file_bytes": nbytes, "decodes_per_step": reps, "l2": "input larger than L2"},
            "roofline": {"bound": "hbm", "achieved": moved / (ms_launch * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": moved / (ms_launch * 1e-3) / 1e9 / peak, "traffic": SEGY_NCU_TRAFFIC,
                         "kernel": "k_segy_decode<1> (file bytes in, float32 samples out)",
                         "algorithmic_bytes_per_launch": moved, "ms_per_launch": ms_launch,
                         "peak_source": f"{peak_kind} {peak:.0f} GB/s"},
            "e2e": {"value": world * nbytes / (ms_e2e * 1e-3) / 1e9, "unit": "GB/s", "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": 4 * ntr * ns},
            "gpu_launches": args.steps * reps, "clocks": clk.summary(), "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_thin_layer(args, rank, world, local):
    """Config 5's cost comparison on one GPU: forward runs of a 256^3
    interior (seeded layered vp 2000-5000 m/s, dx = 10 m, dt = 0.8 ms,
    moment-tensor 12 Hz Ricker2, 1500 steps) inside a 20-cell CPML (300^3
    grid) and inside the 6-cell thin layer with its network corrections
    (272^3 grid), shot after shot.  value: interior Gcell-updates/s of the
    learned-layer runs; the line reports both shots/s and their ratio.  The
    network's cost does not depend on its weights, so an untrained one is
    timed."""
    import torch
    from seiswave_taichi_b200 import learned_abc3d as LA
    from seiswave_taichi_b200.synthetic import layered
    torch.cuda.set_device(local)
    # SEISWAVE_CONFIG5_N / _STEPS shrink the case (profiling captures)
    n = int(os.environ.get("SEISWAVE_CONFIG5_N", "256"))
    nt, pad20, pad6 = int(os.environ.get("SEISWAVE_CONFIG5_STEPS", "1500")), 22, 8
    vp, vs, rho = layered((n, n, n), 2000.0, 5000.0, nlayers=8, seed=rank, anomaly=0.05)
    h, dt, f0 = 10.0, 8e-4, 12.0
    out = {}
    # thin6: the 6-cell layer without its network corrections, which bounds
    # what any correction kernel could reach (its cost taken as zero)
    for tag, P, npml in (("cpml20", pad20, 20), ("learned6", pad6, 6), ("thin6", pad6, 6)):
        m = [np.pad(a, P, mode="edge") for a in (vp, vs, rho)]
        c = m[0].shape[0] // 2
        w = LA.solver3d(*m, h, dt, c, c, c, nt, npml=npml, freq=f0)
        abc = LA.LearnedABC3D(scale=(1e-9,) * 3 + (1.0,) * 6, oscale=(1e-12,) * 9) if tag == "learned6" else None

        def shot():
            w.reset()
            if abc is None:
                w.run(nt)
            else:
                abc.run(w, nt)

        for _ in range(max(1, args.warmup // 3)):
            shot()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            shot()
        e1.record()
        torch.cuda.synchronize()
        out[tag] = e0.elapsed_time(e1) / args.steps
        if tag == "cpml20" and rank == 0 and not args.no_fp64:
            # the 20-cell CPML run (the last timed shot) against float64
            w64 = LA.solver3d(*m, h, dt, c, c, c, nt, npml=npml, freq=f0, dtype=torch.float64)
            w64.run(nt)
            torch.cuda.synchronize()
            out["fp64"] = {"traces_rel_l2": float(torch.linalg.norm(w.data.double() - w64.data)
                                                  / torch.linalg.norm(w64.data)),
                           "final_vx_rel_l2": float(torch.linalg.norm(w.vx.double() - w64.vx)
                                                    / torch.linalg.norm(w64.vx)),
                           "scheme": "20-cell CPML grid (300^3 at n = 256), float64 run of the same scheme"}
            del w64
        del w
    if rank == 0:
        cells = n ** 3
        line = {
            "metric": "Gcell-updates/s", "value": cells * nt / (out["learned6"] * 1e-3) / 1e9,
            "unit": "Gcell-updates/s (interior cells)", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": out["learned6"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"3d-thin-layer-vs-cpml20-{n}^3-nt{nt}", "interior": [n, n, n],
                       "grids": {"cpml20": n + 2 * pad20, "learned6": n + 2 * pad6}, "time_steps": nt},
            "shots_per_s": {"learned6": 1e3 / out["learned6"], "cpml20": 1e3 / out["cpml20"]},
            "learned_over_cpml20": out["cpml20"] / out["learned6"],
            "bound_free_correction": {"thin6_shots_per_s": 1e3 / out["thin6"],
                                      "cpml20_over_thin6": out["cpml20"] / out["thin6"],
                                      "what": "the 6-cell grid stepped without the network corrections"},
            "fp64_error": out.get("fp64"),
            "note": "shots run one after the other (no 3D shot batching); error gate measured on small grids "
                    "in tests/test_learned_abc3d.py",
            "gpu_launches": args.steps * (2 * nt + 2 * nt + 1 + 2 * nt),
        }
        print(json.dumps(line), flush=True)
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="config2", choices=["config2", "config1", "config3", "config4", "config5", "segy", "spml"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the float64 error runs")
    ap.add_argument("--path", default=None, choices=["staged", "fused", "two_pass"],
                    help="3D execution path of the timed solver (default: the plan's own)")
    args = ap.parse_args(argv)
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.config == "config4":
        return run_batch(args, rank, world, local)
    if args.config == "config5":
        return run_thin_layer(args, rank, world, local)
    if args.config == "segy":
        return run_segy(args, rank, world, local)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    cfg = get_config(args.config)
    three_d = len(cfg["shape"]) == 3
    w = build_solver(cfg, torch) if three_d else build_solver2d(cfg, torch)
    if three_d:
        if args.path:
            (w._plan or w._build_plan()).set_path(args.path)
        w.autotune()  # x planes per work unit, outside the timed region
    nt = cfg["nt"]
    ncell = int(np.prod(cfg["shape"]))
    stream = torch.cuda.current_stream()

    def one_run():
        w.reset()
        w.run(nt)

    for _ in range(args.warmup):
        one_run()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            one_run()
        e1.record(stream)
        torch.cuda.synchronize()
    ms_total = max_over_ranks(e0.elapsed_time(e1), dist)
    ms_step = ms_total / args.steps
    value = whole_job_value(world, ncell, nt, args.steps, ms_total)

    # roofline of one time step (velocity + stress pass)
    peak, peak_kind = peaks()
    alg = algorithmic_bytes(cfg)
    ms_per_tstep = ms_step / nt
    achieved = alg / (ms_per_tstep * 1e-3) / 1e9
    # the captured traffic belongs to the plan's default path (the staged passes)
    traffic = NCU_TRAFFIC_PER_STEP.get(cfg["name"]) if not args.path else None

    # end to end through the public API with host buffers
    pin = {k: torch.from_numpy(np.ascontiguousarray(cfg[k])).pin_memory() for k in ("vp", "vs", "rho")}
    out = torch.empty(tuple(w.data.shape), dtype=w.data.dtype).pin_memory()
    h2d = sum(t.numel() * t.element_size() for t in pin.values())
    d2h = out.numel() * out.element_size()

    def e2e_run():
        w.set_model(pin["vp"], pin["vs"], pin["rho"])
        w.reset()
        w.run(nt)
        out.copy_(w.data, non_blocking=True)

    for _ in range(2):
        e2e_run()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        e2e_run()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), dist)
    e2e_value = whole_job_value(world, ncell, nt, args.steps, e2e_ms)

    # the opt-in fast numeric mode (exact=False) on the same workload
    fast = None
    if three_d and cfg.get("scheme") != "SPML":  # the split-field PML runs exact numerics only
        wf = build_solver(cfg, torch, exact=False)
        wf.autotune()
        for _ in range(2):
            wf.reset()
            wf.run(nt)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            wf.reset()
            wf.run(nt)
        e1.record(stream)
        torch.cuda.synchronize()
        f_ms = max_over_ranks(e0.elapsed_time(e1), dist)
        f_tstep = f_ms / args.steps / nt
        fast = {"value": whole_job_value(world, ncell, nt, args.steps, f_ms), "unit": "Gcell-updates/s",
                "ms_per_step": f_ms / args.steps,
                "roofline_frac": alg / (f_tstep * 1e-3) / 1e9 / peak,
                "parity": "traces within 1e-5 rel. L2 of the oracle over 400 steps; fields within 1e-4"}
        del wf

    # error of the f32 result (the last timed run) against float64 runs
    err64 = fp64_error(cfg, w, torch) if rank == 0 and not args.no_fp64 else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(cfg)

    # per run: velocity + stress kernel per time step, plus the first step's
    # moment-tensor injection (receivers and next-step sources ride inside the
    # stress kernel); w.reset() zeroes the state with torch fills
    launches_per_run = 2 * nt + 1
    info = w._plan.info() if three_d else {"path": "two_pass"}
    kname = {"staged": "k3s_velocity + k3s_stress", "two_pass": "k3_velocity + k3_stress",
             "fused": "k3_fused"}.get(info["path"], info["path"]) if three_d else "k2_velocity + k2_stress"
    if rank == 0:
        line = {
            "metric": "Gcell-updates/s", "value": value, "unit": "Gcell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(cfg, world),
            "implementation": {"path": info, "numerics": "exact (bit-identical to the reference's own source "
                                                           "and to the CPU oracle)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": kname + " (one time step)",
                         "algorithmic_bytes_per_launch": alg, "ms_per_launch": ms_per_tstep,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                                        else "fallback 6650 GB/s"},
            "e2e": {"value": e2e_value, "unit": "Gcell-updates/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches_per_run * args.steps,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "fast_mode": fast,
            "fp64_error": err64,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
