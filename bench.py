#!/usr/bin/env python
"""Benchmark: K3DOM update frames/s on B200 at 2.1M voxels / 4.2M particles / 120k points.

Workload (one step = one steady-state frame of the K3DOM 10 Hz sequence): 256x256x32 grid at
0.1 m (2,097,152 voxels), 4,194,304 persistent + 1,048,576 new-born particles, 64-beam scans of
120,000 returns, ego motion 0-2 m/s, 20 static + 20 moving cuboids (k3dom_b200.scene.config1).
Seeded synthetic scans stand in for the reference's rosbags (not in its checkout).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference|reference-gpu]
                    [--variant k3dom|dsphdmib]

ours           the library through its C ABI: `value` is device-timed frames/s with the scans
               resident in HBM (graph-captured frames); `e2e` is frames/s through
               k3dom_update_grid with the scan in pinned host memory and the per-voxel occupancy
               read back to pinned host memory every frame (wall clock).
reference      the CPU baseline of the path: the reference has no CPU implementation, so its
               restatement (oracle/, FP64, OpenMP over all host threads) runs the same frames.
reference-gpu  the reference's own CUDA update (oracle/_ref, built from its sources), frames/s
               on this GPU (a second reference measurement, reported beside the CPU one).

Multi-GPU: the single-scene update does not shard (replicas only); with torchrun every rank
runs an independent scene (weak scaling), timed on the device, max over ranks.
"""
from __future__ import annotations

import argparse
import json
from typing import Optional
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "update frames/s @2.1M voxels,4M particles; batched vs plain; grad-step ms"
UNIT = "frames/s"
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0
NOMINAL_FP32_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # 74.4: no measured FP32 peak exists
FLOP_PER_EVAL = 20  # distance (8 + sqrt) + sparse kernel (2x/ls, cospi, sinpi, 7 arithmetic)
FLOP_PER_DS_NEIGHBOUR = 25  # window test (c.m, (c.m)^2/|m|^2, compare: 8) + pOcc (r^2, exp, scale: 17)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (clocks, power, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu = gpu_id
        self.proc = None
        self.lines: list[str] = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ distributed plumbing
def dist_setup(gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        return rank, world, local, dist
    return 0, 1, local, None


def barrier(dist):
    if dist is not None:
        dist.barrier()


def max_over_ranks(x: float, dist) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, dist) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def read_peaks() -> tuple[float, str]:
    try:
        d = json.loads(PEAKS_FILE.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def stage_bytes(P: int, B: int, C: int, N: int) -> dict:
    """Algorithmic HBM bytes per frame of each timed stage, minimal FP32 SoA: prediction 60P;
    assignment = key sort 52P + payload permute 56P + ranges 4P+8C + the per-cell moment sums
    fused into the gather 16P+12C; occupancy (evidence + cell update) 36C+4P+12N; persistent
    reweight 12P+4C; births 8C+36B; resampling = joint scan 12(P+B) + draw sort 32P + ancestor
    gather 60P. Sum: 1.486 GB at 2,097,152 cells, P=4,194,304, B=1,048,576, N=120,000."""
    return {
        "predict": 60 * P,
        "assign": 52 * P + 56 * P + 4 * P + 8 * C + 16 * P + 12 * C,
        "occupancy": 36 * C + 4 * P + 12 * N,
        "persistent": 12 * P + 4 * C,
        "births": 8 * C + 36 * B,
        "resample": 12 * (P + B) + 32 * P + 60 * P,
    }


PARTICLE_STAGES = ("predict", "assign", "persistent", "births", "resample")


def hbm_bytes_particle_stages(P: int, B: int, C: int, N: int) -> float:
    """Algorithmic bytes of the HBM-bound particle stages per frame (the occupancy stage, which
    is bound by SIMT issue, is left out)."""
    b = stage_bytes(P, B, C, N)
    return float(sum(b[k] for k in PARTICLE_STAGES))


def stage_roofline(stage: dict, P: int, B: int, C: int, N: int, hbm_peak: float) -> dict:
    """Each stage's algorithmic bytes / its CUDA-event time / the HBM peak."""
    out = {}
    for k, nbytes in stage_bytes(P, B, C, N).items():
        ms = stage.get(f"{k}_ms")
        if not ms:
            continue
        gbs = nbytes / (ms * 1e-3) / 1e9
        out[k] = {"algorithmic_bytes": int(nbytes), "ms": round(ms, 4), "gbs": round(gbs, 1),
                  "frac": round(gbs / hbm_peak, 4)}
    return out


def workload_name(cfg, variant: str) -> str:
    """The workload string both arms report (same scene, same frames)."""
    G = int(np.float32(cfg.params["size"]) / np.float32(cfg.params["resolution"]))
    Gz = int(np.float32(cfg.params["size_z"]) / np.float32(cfg.params["resolution"]))
    return (f"{cfg.name}: {variant} steady-state frame, {G}x{G}x{Gz} voxels @{cfg.params['resolution']:g} m, "
            f"P={cfg.params['particle_count']}, B={cfg.params['new_born_particle_count']}, "
            f"{cfg.n_points} points/scan, ego motion, 10 Hz")


# ------------------------------------------------------------------ frames
def make_frames(cfg, n_frames: int):
    frames = []
    for f in range(n_frames):
        t = 0.1 + f * cfg.dt
        s, pts = cfg.scene.scan(f, t, cfg.n_points)
        frames.append((t, s, np.ascontiguousarray(pts)))
    return frames


def cpu_oracle_frames(cfg, variant: str, frames, steps: int, warmup: int, budget_s: float,
                      warmup_budget_s: float = 90.0, done: Optional[dict] = None):
    """Time steady-state frames of the CPU oracle. Returns (frames/s, sample note, threads, frames
    timed); done["warmup"] receives the warm-up frames run (at most `warmup`, within
    warmup_budget_s)."""
    from oracle import binding as O
    from oracle.frame import OracleDOM
    dom = OracleDOM(_params_struct(variant, dict(cfg.params)), variant)
    t, s, pts = frames[0]
    dom.update_pose(*s)
    dom.update_grid(t, pts)
    idx = 1
    w_start = time.perf_counter()
    n_warm = 0
    for _ in range(warmup):
        t, s, pts = frames[idx]
        idx += 1
        dom.update_pose(*s)
        dom.update_grid(t, pts)
        n_warm += 1
        if time.perf_counter() - w_start > warmup_budget_s:
            break
    if done is not None:
        done["warmup"] = n_warm
    times = []
    t_start = time.perf_counter()
    for _ in range(steps):
        t, s, pts = frames[idx]
        idx += 1
        dom.update_pose(*s)
        t0 = time.perf_counter()
        dom.update_grid(t, pts)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start > budget_s:
            break
    fps = len(times) / sum(times)
    note = (f"{len(times)} full steady-state frame(s) of the {cfg.name} sequence on the CPU oracle "
            f"(FP64 continuous math, all stages), {O.oracle().orc_num_threads()} OpenMP threads")
    return fps, note, int(O.oracle().orc_num_threads()), len(times)


def _params_struct(variant, params):
    from k3dom_b200 import _native as N
    p = N.Params()
    # defaults without the library (the CPU arm must not need a GPU)
    for k, v in params.items():
        setattr(p, k, v)
    return p


def scene_cfg(variant: str, rank: int):
    from k3dom_b200 import scene
    cfg = scene.config1(seed=1000 + rank, variant=variant)
    cfg.params["seed"] = 20240 + rank
    return cfg


# ------------------------------------------------------------------ arms
def measure_plain(args, variant: str, cfg, rank: int, world: int, local: int, dist, sample_clocks: bool) -> dict:
    """One plain handle on this rank's scene: autotune, warm up, time K graph-replayed frames with
    the scans in HBM (CUDA events on the handle's stream), then per-stage times, then K frames end
    to end through k3dom_update_grid (pinned host scan in, occupancy out to pinned host memory)."""
    import torch

    import k3dom_b200 as K
    from k3dom_b200 import _native as N
    W, Kst = args.warmup, args.steps
    n_tune = 16  # evidence autotuner: one live frame per candidate (k3dom_autotune), at most 16
    n_e2e_warm = 3  # untimed end-to-end iterations (first-call costs: export buffer, host staging)
    n_frames = 1 + n_tune + W + Kst + 2 + Kst + 1 + n_e2e_warm + Kst
    log(f"[rank {rank}] {variant}: generating {n_frames} scans of {cfg.n_points} points")
    frames = make_frames(cfg, n_frames)
    p = K.make_params(variant, **cfg.params)
    dom = K.DOM(p, variant, device=local)
    try:
        # scans resident in HBM for the device-timed run
        dev_pts = [torch.from_numpy(f[2]).to(f"cuda:{local}") for f in frames]
        torch.cuda.synchronize()

        def step_device(i):
            t, s, _ = frames[i]
            dom.updatePose(*s)
            dom.updateGridAsync(t, dev_pts[i])

        # first frame (initialisation), the autotuner's frames, then warm-up; the graph is captured
        # on the first steady frame after tuning
        dom.set_graph_mode(True)
        dom.updatePose(*frames[0][1])
        dom.updateGrid(frames[0][0], dev_pts[0])
        idx = 1
        if args.tile_rule is None:
            dom.autotune(True)
            for _ in range(dom.tuning()["candidates"]):
                step_device(idx)
                idx += 1
        else:
            dom.set_tuning(args.tile_rule, args.chunk)
        dom.synchronize()
        tuning = dom.tuning()
        for _ in range(W):
            step_device(idx)
            idx += 1
        dom.synchronize()
        stream = torch.cuda.ExternalStream(dom.stream())
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        props = torch.cuda.get_device_properties(local)
        uuid = getattr(props, "uuid", None)
        gpu_id = f"GPU-{uuid}" if uuid is not None else str(local)
        sampler = ClockSampler(gpu_id) if (rank == 0 and sample_clocks) else None
        barrier(dist)
        torch.cuda.synchronize()
        if sampler:
            sampler.start()
            time.sleep(0.3)
        ev0.record(stream)
        for _ in range(Kst):
            step_device(idx)
            idx += 1
        ev1.record(stream)
        dom.synchronize()
        torch.cuda.synchronize()
        barrier(dist)
        clocks = sampler.stop() if sampler else None
        ms = ev0.elapsed_time(ev1) / Kst
        ms_max = max_over_ranks(ms, dist)
        launches = int(dom.diagnostics()["kernel_launches_per_frame"])

        # end to end on the frames right after the device-timed ones, so that the two rates see
        # the same stretch of the scene
        # (through the C ABI: pinned host scan in, per-voxel occupancy out, every frame)
        host_pts = [torch.from_numpy(f[2]).pin_memory() for f in frames]
        occ_out = torch.empty(dom.grid_cell_count, dtype=torch.float32).pin_memory()
        lib = dom._lib
        field = N.CELL_FIELDS["occ_mean" if variant == "k3dom" else "occ_prob"]
        # every frame writes its occupancy into the pinned host buffer (registered output): the
        # device->host copy is part of each frame, overlapped with the frame's last stages
        N.check(lib.k3dom_set_output(dom._h, field, occ_out.data_ptr(), N.MEM_HOST), "set_output")

        def e2e_frame(i):
            t, s, _ = frames[i]
            hp = host_pts[i].numpy()
            dom.updatePose(*s)
            N.check(lib.k3dom_update_grid(dom._h, float(t), hp.ctypes.data, None, None, hp.shape[0], N.MEM_HOST),
                    "update_grid")

        for _ in range(n_e2e_warm):
            e2e_frame(idx)
            idx += 1
        barrier(dist)
        t0 = time.perf_counter()
        n_e2e = 0
        while n_e2e < Kst and idx < len(frames):
            e2e_frame(idx)
            idx += 1
            n_e2e += 1
        e2e_s = max_over_ranks(time.perf_counter() - t0, dist)
        N.check(lib.k3dom_set_output(dom._h, 0, None, N.MEM_HOST), "set_output")

        # per-stage device times and the evidence kernel's work (events on the handle's stream)
        dom.set_timing(True)
        st_acc, evals = [], []
        for _ in range(2):
            step_device(idx)
            idx += 1
            dom.synchronize()
        for _ in range(min(Kst, 10)):
            step_device(idx)
            idx += 1
            dom.synchronize()
            st_acc.append(dom.stage_times())
            evals.append(dom.diagnostics()["kernel_evaluations"])
        dom.set_timing(False)
        diag_after = dom.diagnostics()
        stage = {k: float(np.mean([s[k] for s in st_acc])) for k in st_acc[0]}

        return {"ms": ms_max, "value": world * 1000.0 / ms_max, "e2e_fps": world * n_e2e / e2e_s,
                "launches": launches, "stage": stage, "evals": float(np.mean(evals)), "tuning": tuning,
                "diag": diag_after, "clocks": clocks, "frames": frames, "C": dom.grid_cell_count,
                "P": dom.particle_count, "B": dom.new_born_particle_count}
    finally:
        dom.close()


def evidence_roofline(m: dict, variant: str) -> dict:
    """The dominant kernel's line: in-support evaluations (K3DOM) or accepted neighbours (DS) x
    FLOP per unit / its CUDA-event time / the nominal FP32 issue peak."""
    ev_ms = m["stage"]["evidence_ms"]
    ds = variant != "k3dom"
    flop_per = FLOP_PER_DS_NEIGHBOUR if ds else FLOP_PER_EVAL
    achieved = m["evals"] * flop_per / (ev_ms * 1e-3) / 1e12
    traffic, issue = None, None
    tr_file = ROOT / "profiles" / ("dsgrid_traffic.json" if ds else "bgki_traffic.json")
    rule_name = ["by-size", "8x8x4", "16x16x4", "16x16x8"][m["tuning"]["tile_rule"]]
    if rule_name == "by-size":
        rule_name = "16x16x8"  # the rule's choice for grids of >= 2^20 cells
    if tr_file.exists():
        try:
            d = json.loads(tr_file.read_text())
            issue = d.get("issue")
            per = d["per_tiling"]
            hit = per.get(f"{rule_name}@{m['tuning']['chunk']}") or per.get(rule_name) or {}
            traffic = hit.get("dram_bytes_per_launch")
        except Exception:
            traffic = None
    return {
        "kernel": ("k_dsgrid (DS measurement grid + fused Dempster update)" if ds else
                   "k_bgki (sparse BGKI evidence + fused cell update)"),
        "bound": "fp32", "achieved": round(achieved, 3), "peak": round(NOMINAL_FP32_TFLOPS, 1),
        "unit": "TFLOP/s", "frac": round(achieved / NOMINAL_FP32_TFLOPS, 4), "traffic": traffic,
        "peak_source": "nominal FP32 (148 SMs x 128 lanes x 2 x 1.965 GHz); no measured FP32 peak",
        "work": (f"{m['evals']:.4g} accepted neighbours x {flop_per} FLOP per frame" if ds else
                 f"{m['evals']:.4g} in-support kernel evaluations x {flop_per} FLOP per frame"),
        "launch_ms": round(ev_ms, 4),
        "note": ("SIMT-issue bound: frac counts only in-support evaluations x FLOP; the lanes outside "
                 "a ray's support, the FP64 pair set-up and the fixed-point rounding are the rest"),
        "ncu_issue": issue,
    }


def run_ours(args):
    import torch

    rank, world, local, dist = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    cfg = scene_cfg(args.variant, rank)
    m = measure_plain(args, args.variant, cfg, rank, world, local, dist, sample_clocks=True)
    Kst, W = args.steps, args.warmup
    ds_m = None
    if args.variant == "k3dom" and not args.no_ds:
        ds_cfg = scene_cfg("dsphdmib", rank)
        ds_m = measure_plain(args, "dsphdmib", ds_cfg, rank, world, local, dist, sample_clocks=False)
    batch_res = None
    if not args.no_batch:
        batch_res = run_batch(args, local, rank, world, dist)
    out = None
    if rank == 0:
        hbm_peak, peak_src = read_peaks()
        C_, P, B = m["C"], m["P"], m["B"]
        stage = m["stage"]
        part_ms = sum(stage[f"{k}_ms"] for k in PARTICLE_STAGES)
        part_bytes = hbm_bytes_particle_stages(P, B, C_, cfg.n_points)
        tuning = m["tuning"]
        out = {
            "metric": METRIC, "value": round(m["value"], 3), "unit": UNIT, "n_gpus": world, "steps": Kst,
            "warmup": W, "ms_per_step": round(m["ms"], 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (f64 accumulation)", "data": "synthetic (seeded LiDAR scans)",
            "config": {
                "workload": workload_name(cfg, args.variant),
                "voxels": C_, "particles": P, "new_born": B, "points_per_frame": cfg.n_points,
                "parallelism": f"replicas x{world} (independent scenes)",
                "l2": "state > L2 (about 1 GB of particle/cell arrays touched per frame)",
                "graph": True, "evidence_tiling": ("autotuned (k3dom_autotune) during warm-up" if args.tile_rule is None
                                                else f"fixed (--tile-rule {args.tile_rule} --chunk {args.chunk})"),
            },
            "e2e": {"value": round(m["e2e_fps"], 3), "unit": UNIT, "h2d_bytes_per_step": int(cfg.n_points * 12),
                    "d2h_bytes_per_step": int(C_ * 4),
                    "path": "k3dom_update_grid (synchronous) with the (N, 3) scan in pinned host memory; the "
                            "frame's occupancy (one float per voxel) lands in pinned host memory "
                            "through k3dom_set_output; host clock around every frame"},
            "gpu_launches": m["launches"] * Kst,
            "clocks": m["clocks"],
            "roofline": evidence_roofline(m, args.variant),
            "roofline_hbm": {
                "kernels": "particle stages (predict, sort, gather+sums, reweight, births, resampling)",
                "bound": "hbm", "achieved": round(part_bytes / (part_ms * 1e-3) / 1e9, 1), "peak": hbm_peak,
                "unit": "GB/s", "frac": round(part_bytes / (part_ms * 1e-3) / 1e9 / hbm_peak, 4),
                "peak_source": peak_src, "algorithmic_bytes": int(part_bytes), "time_ms": round(part_ms, 4),
            },
            "stage_ms": {k: round(v, 4) for k, v in stage.items()},
            "stage_roofline": {"peak_gbs": hbm_peak, "peak_source": peak_src,
                               **stage_roofline(stage, P, B, C_, cfg.n_points, hbm_peak)},
            "evidence_lists": {k: m["diag"][k] for k in ("ray_list_entries", "ray_list_capacity", "work_items",
                                                          "kernel_evaluations")},
            "tuning": {"tile_rule": ["by-size", "8x8x4", "16x16x4", "16x16x8"][tuning["tile_rule"]],
                       "chunk": tuning["chunk"], "candidate_ms": [round(x, 3) for x in tuning["candidate_ms"]]},
        }
        if ds_m is not None:
            out["ds_frame"] = {
                "workload": workload_name(ds_cfg, "dsphdmib"), "unit": UNIT,
                "value": round(ds_m["value"], 3), "ms_per_step": round(ds_m["ms"], 4),
                "e2e": round(ds_m["e2e_fps"], 3), "gpu_launches_per_frame": ds_m["launches"],
                "stage_ms": {k: round(v, 4) for k, v in ds_m["stage"].items()},
                "roofline": evidence_roofline(ds_m, "dsphdmib"),
                "stage_roofline": stage_roofline(ds_m["stage"], ds_m["P"], ds_m["B"], ds_m["C"], ds_cfg.n_points,
                                                 hbm_peak),
                "tuning": {"tile_rule": ["by-size", "8x8x4", "16x16x4", "16x16x8"][ds_m["tuning"]["tile_rule"]],
                           "chunk": ds_m["tuning"]["chunk"]},
            }
        if batch_res is not None:
            out["batched"] = batch_res
        if world == 1 and not args.no_grad:
            out["grad_step"] = run_grad_step(args, local, frame_ms=m["ms"])
        if world == 1 and not args.no_cpu_baseline:
            fps, note, cores, n = cpu_oracle_frames(cfg, args.variant, m["frames"], 1, 0, budget_s=60.0)
            out["cpu_baseline"] = {"value": round(fps, 5), "unit": UNIT, "cores": cores, "kind": "port",
                                   "sample": note}
    if dist is not None:
        dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out), flush=True)


def run_reference_cpu(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg = scene_cfg(args.variant, 0)
    frames = make_frames(cfg, 1 + args.warmup + args.steps)
    done = {}
    fps, note, cores, n = cpu_oracle_frames(cfg, args.variant, frames, args.steps, args.warmup, budget_s=240.0,
                                            done=done)
    out = {
        "impl": "reference", "metric": METRIC, "value": round(fps, 5), "unit": UNIT, "n_gpus": args.gpus,
        "steps": n, "warmup": done.get("warmup", args.warmup), "ms_per_step": round(1000.0 / fps, 2),
        "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded LiDAR scans)",
        "config": {"workload": workload_name(cfg, args.variant), "parallelism": "CPU"},
        "cpu_baseline": {"value": round(fps, 5), "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": note + "; the reference has no CPU implementation of the update"},
        "e2e": {"value": round(fps, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def run_reference_gpu(args):
    """The reference's own CUDA update (unmodified sources behind oracle/ref_harness.cu)."""
    import torch

    import k3dom_b200 as K
    from oracle.binding import Reference
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg = scene_cfg(args.variant, 0)
    frames = make_frames(cfg, 1 + args.warmup + args.steps)
    p = K.make_params(args.variant, **cfg.params)
    ref = Reference(p, args.variant)
    t, s, pts = frames[0]
    ref.update_pose(*s)
    ref.update_grid(t, pts)
    for i in range(1, 1 + args.warmup):
        t, s, pts = frames[i]
        ref.update_pose(*s)
        ref.update_grid(t, pts)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(1 + args.warmup, len(frames)):
        t, s, pts = frames[i]
        ref.update_pose(*s)
        ref.update_grid(t, pts)  # ends with cudaDeviceSynchronize (src/k3dom/dom.cu:47)
    wall = time.perf_counter() - t0
    ref.close()
    fps = args.steps / wall
    print(json.dumps({"impl": "reference-gpu", "metric": METRIC, "value": round(fps, 4), "unit": UNIT,
                      "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                      "ms_per_step": round(1000 / fps, 3), "higher_is_better": True,
                      "config": {"workload": workload_name(cfg, args.variant),
                                 "path": "the reference's own CUDA updateGrid (host vectors in, synchronising)"}}),
          flush=True)


def run_batch(args, local: int = 0, rank: int = 0, world: int = 1, dist=None) -> dict:
    """Batched form: 16 independent scenes (k3dom_b200.scene.config3) updated together by one
    BatchDOM (one launch per stage, graph-replayed, evidence tiling autotuned on live frames)
    against the plain form looping over the same 16 scenes with one DOM each. Aggregate frames/s
    = scenes x frames / time. Both arms take the same host scans and run synchronous calls (the
    reference's updateGrid synchronises, src/k3dom/dom.cu:47); time = host clock around the
    timed frames. The device-resident rows feed the scans from HBM instead. With several ranks
    the scenes are partitioned by estimated cost (k3dom_b200.shard) and each rank runs its own
    share; time = max over ranks."""
    import torch

    import k3dom_b200 as K
    from k3dom_b200 import scene, shard
    all_cfgs = scene.config3(seed=args.batch_seed, n_scenes=args.scenes, variant=args.variant)
    mine = shard.my_scenes([shard.scene_cost(c.params, c.n_points) for c in all_cfgs], rank, world)
    cfgs = [all_cfgs[i] for i in mine]
    S = len(cfgs)
    W, Kst = 2, args.batch_steps
    n_frames = 1 + W + Kst
    log(f"[rank {rank}] batch: generating {S} x {n_frames} scans")
    frames = [make_frames(c, n_frames) for c in cfgs]  # frames[s][f] = (t, sensor, pts)
    params = [K.make_params(args.variant, **c.params) for c in cfgs]
    dev = f"cuda:{local}"
    dev_pts = [[torch.from_numpy(fr[2]).to(dev) for fr in frames[s]] for s in range(S)]
    torch.cuda.synchronize()

    def timed_region(run_frames) -> float:
        barrier(dist)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        run_frames()
        torch.cuda.synchronize()
        return max_over_ranks(time.perf_counter() - t0, dist)

    stage_keys = ("predict_ms", "assign_ms", "occupancy_ms", "binning_ms", "evidence_ms", "persistent_ms",
                  "births_ms", "resample_ms", "total_ms")
    breakdown = {}

    def plain_arm(device_resident: bool) -> float:
        doms = [K.DOM(p, args.variant, device=local) for p in params]
        try:
            def frame(f, t_shift=0.0):
                for s, d in enumerate(doms):
                    t, pose, pts = frames[s][f]
                    d.updatePose(*pose)
                    if device_resident:
                        d.updateGridAsync(t + t_shift, dev_pts[s][f])
                        d.synchronize()
                    else:
                        d.updateGrid(t + t_shift, pts)
            for f in range(1 + W):
                frame(f)

            def timed():
                for f in range(1 + W, n_frames):
                    frame(f)
            secs = timed_region(timed)
            if device_resident and S:
                # per-stage device time of one frame of every scene, summed over the 16 handles
                for d in doms:
                    d.set_timing(True)
                frame(n_frames - 1, t_shift=0.1)
                frame(n_frames - 1, t_shift=0.2)
                acc = {k: 0.0 for k in stage_keys}
                for d in doms:
                    st_ = d.stage_times()
                    for k in stage_keys:
                        acc[k] += st_[k]
                breakdown["plain_sum_of_scenes"] = {k: round(v, 4) for k, v in acc.items()}
            return secs
        finally:
            for d in doms:
                d.close()

    def batch_arm(device_resident: bool):
        if S == 0:
            return timed_region(lambda: None), None, 0
        b = K.BatchDOM(params, args.variant, device=local)
        try:
            for s in range(S):
                b.updatePose(s, *frames[s][0][1])
            b.update([frames[s][0][0] for s in range(S)], [frames[s][0][2] for s in range(S)])
            # autotune on live frames (replaying frame 1's scans as the clock advances)
            b.autotune(True)
            tune_frames = b.tuning()["candidates"]
            for k in range(tune_frames):
                for s in range(S):
                    b.updatePose(s, *frames[s][1][1])
                b.update([frames[s][1][0] + 0.1 * k for s in range(S)], [frames[s][1][2] for s in range(S)])
            tuning = b.tuning()
            t_shift = 0.1 * tune_frames

            def frame(f):
                for s in range(S):
                    b.updatePose(s, *frames[s][f][1])
                ts = [frames[s][f][0] + t_shift for s in range(S)]
                if device_resident:
                    b.update_async(ts, [dev_pts[s][f] for s in range(S)])
                    b.synchronize()
                else:
                    b.update(ts, [frames[s][f][2] for s in range(S)])
            for f in range(1, 1 + W):
                frame(f)

            def timed():
                for f in range(1 + W, n_frames):
                    frame(f)
            secs = timed_region(timed)
            launches = b.diagnostics()["kernel_launches_per_frame"]
            if device_resident:
                # per-stage device time of one batched frame (events on the batch's stream)
                b.set_timing(True)
                for k in (1, 2):
                    for s in range(S):
                        b.updatePose(s, *frames[s][n_frames - 1][1])
                    b.update_async([frames[s][n_frames - 1][0] + t_shift + 0.1 * k for s in range(S)],
                                   [dev_pts[s][n_frames - 1] for s in range(S)])
                    b.synchronize()
                st_ = b.stage_times()
                breakdown["batched"] = {k: round(st_[k], 4) for k in stage_keys}
                b.set_timing(False)
            return secs, tuning, launches
        finally:
            b.close()

    total = len(all_cfgs) * Kst
    plain_host = total / (plain_arm(False) if S else timed_region(lambda: None))
    plain_dev = total / (plain_arm(True) if S else timed_region(lambda: None))
    bh, tuning, launches = batch_arm(False)
    bd, _, _ = batch_arm(True)
    batch_host, batch_dev = total / bh, total / bd
    rules = ["by-size", "8x8x4", "16x16x4", "16x16x8"]
    return {
        "workload": f"config3: {len(all_cfgs)} independent {args.variant} scenes, G 64-256, Gz 16-32, "
                    f"P 2^18-2^22, B=P/4, 10k-200k points; {Kst} timed frames after {W} warm-up",
        "scenes": len(all_cfgs), "frames": Kst, "unit": "aggregate frames/s", "ranks": world,
        "scenes_per_rank": [len(p) for p in shard.partition(
            [shard.scene_cost(c.params, c.n_points) for c in all_cfgs], world)],
        "voxels_total": int(sum(int(np.float32(c.params["size"]) / np.float32(0.1)) ** 2 *
                                int(np.float32(c.params["size_z"]) / np.float32(0.1)) for c in all_cfgs)),
        "particles_total": int(sum(c.params["particle_count"] for c in all_cfgs)),
        "points_per_frame_total": int(sum(c.n_points for c in all_cfgs)),
        "plain_loop": round(plain_host, 2), "batched": round(batch_host, 2),
        "speedup": round(batch_host / plain_host, 3),
        "plain_loop_device_resident": round(plain_dev, 2), "batched_device_resident": round(batch_dev, 2),
        "speedup_device_resident": round(batch_dev / plain_dev, 3),
        "batched_launches_per_frame": int(launches),
        "stage_ms": breakdown,
        "tuning": None if tuning is None else {
            "tile_rule": rules[tuning["tile_rule"]], "chunk": tuning["chunk"],
            "candidate_ms": [round(x, 3) for x in tuning["candidate_ms"]]},
        "timing": "host clock around synchronous calls (both arms), max over ranks; host scans unless "
                  "device_resident",
    }


def run_grad_step(args, local: int = 0, frame_ms: float | None = None) -> dict:
    """Differentiable update (config4 scaled to config1's grid): one gradient step is
    k3dom_bgki_backward (kernel and derivative sums of both training frames, the mass recursion,
    the loss and its hand-written adjoint); the forward is k3dom_bgki_forward. The length-scale
    changes every call, so the sums are recomputed each time, as in a calibration loop. Device
    time between CUDA events on the problem's stream (the calls synchronise inside)."""
    import torch

    from k3dom_b200 import calib, scene
    cfg = scene.config4(seed=0, scale="config1")
    pr = calib.build_problem(cfg, device=local)
    try:
        stream = torch.cuda.ExternalStream(pr.calib.stream())
        th = np.array(pr.theta0, np.float64)

        def timed(fn, n):
            ms = []
            for i in range(n):
                t = th.copy()
                t[0] = th[0] * (1.0 + 1e-4 * (i % 7 + 1))
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                fn(t)
                e1.record(stream)
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
            return float(np.median(ms))
        for _ in range(3):
            pr.calib.loss_and_grad(th)
        fwd = timed(pr.calib.loss, 10)
        step = timed(pr.calib.loss_and_grad, 10)
        loss, g = pr.calib.loss_and_grad(th)
        n0, n1 = pr.calib.label_counts()
        out = {
            "workload": "config4 scaled to config1: 256x256x32 grid @0.1 m, 2 training frames of 120,000 points "
                        "(initialisation + one update with the particle filter's weights), 10 held-out scans "
                        "of 120,000 points; theta = (ls 0.3 m, sigma 1.0, gamma 0.1, occupied prior 0.01, free "
                        "prior 0.01)",
            "forward_ms": round(fwd, 3), "grad_step_ms": round(step, 3),
            "step_over_forward": round(step / fwd, 3),
            "label_instances": int(n0.sum() + n1.sum()), "loss": round(float(loss), 6),
            "grad": [float(f"{v:.6g}") for v in g],
            "timing": "CUDA events on the problem's stream, median of 10, ls perturbed every call",
        }
        if frame_ms:
            out["step_over_plain_frame"] = round(step / frame_ms, 3)
        return out
    finally:
        pr.close()


def run_profile_case(args):
    """Scenes for ncu captures, eager frames (no graph), the first frame plus `--steps` frames.
    medium: 128x128x32 voxels at 0.1 m, P=1,048,576, B=262,144, 60,000 points (state > L2, a few
    hundred MB on the device). config1: the benchmark's own scene (256x256x32, P=4,194,304,
    B=1,048,576, 120,000 points; about 1.5 GB on the device) with the tiling given by
    --profile-tile-rule/--chunk. batch: the 16 scenes of the batched measurement in one BatchDOM
    (a few GB on the device)."""
    import k3dom_b200 as K
    from k3dom_b200 import scene
    if args.profile_case == "batch":
        cfgs = scene.config3(seed=args.batch_seed, n_scenes=args.scenes, variant=args.variant)
        b = K.BatchDOM([K.make_params(args.variant, **c.params) for c in cfgs], args.variant)
        if args.profile_tile_rule is not None:
            b.set_tuning(args.profile_tile_rule, args.chunk)
        for f in range(1 + args.steps):
            ts, clouds = [], []
            for s, c in enumerate(cfgs):
                t = 0.1 + f * c.dt
                sensor, pts = c.scene.scan(f, t, c.n_points)
                b.updatePose(s, *sensor)
                ts.append(t)
                clouds.append(pts)
            b.update(ts, clouds)
        log("profile case done", b.diagnostics())
        b.close()
        return
    cfg = scene.config1(seed=5, variant=args.variant)
    if args.profile_case == "medium":
        cfg.params.update(size=12.8, particle_count=1 << 20, new_born_particle_count=1 << 18, max_points=60000)
        cfg.n_points = 60000
        cfg.scene.max_range = 12.8
    p = K.make_params(args.variant, **cfg.params)
    dom = K.DOM(p, args.variant)
    if args.profile_tile_rule is not None:
        dom.set_tuning(args.profile_tile_rule, args.chunk)
    for f in range(1 + args.steps):
        t = 0.1 + f * cfg.dt
        s, pts = cfg.scene.scan(f, t, cfg.n_points)
        dom.updatePose(*s)
        dom.updateGrid(t, pts)
    log("profile case done", dom.diagnostics())
    dom.close()


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference", "reference-gpu"], default="ours")
    ap.add_argument("--variant", choices=["k3dom", "dsphdmib"], default="k3dom")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-case", choices=["medium", "config1", "batch"], default=None,
                    help="run a mid-size scene for profiler captures instead of the benchmark")
    ap.add_argument("--workload", choices=["frame", "batch", "grad"], default="frame",
                    help="batch: only the batched-vs-plain line (16 scenes); grad: only the gradient step")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-vs-plain measurement")
    ap.add_argument("--no-grad", action="store_true", help="skip the gradient-step measurement")
    ap.add_argument("--no-ds", action="store_true", help="skip the DS-PHD/MIB frame measured beside K3DOM")
    ap.add_argument("--tile-rule", type=int, default=None,
                    help="fixed evidence tile rule instead of autotuning (0 by size, 1 8x8x4, 2 16x16x4, 3 16x16x8)")
    ap.add_argument("--chunk", type=int, default=1024,
                    help="rays per evidence work item with --tile-rule or --profile-tile-rule")
    ap.add_argument("--profile-tile-rule", type=int, default=None,
                    help="profile case: evidence tile rule (0 by size, 1 8x8x4, 2 16x16x4, 3 16x16x8)")
    ap.add_argument("--scenes", type=int, default=16)
    ap.add_argument("--batch-steps", type=int, default=5)
    ap.add_argument("--batch-seed", type=int, default=0)
    args = ap.parse_args(argv)
    if args.warmup < 3 and args.impl == "ours":
        log("warmup < 3 raised to 3")
        args.warmup = 3
    if args.profile_case:
        run_profile_case(args)
    elif args.workload == "batch":
        import torch
        torch.cuda.set_device(0)
        print(json.dumps({"metric": "batched vs plain aggregate frames/s", **run_batch(args)}), flush=True)
    elif args.workload == "grad":
        import torch
        torch.cuda.set_device(0)
        print(json.dumps({"metric": "gradient step ms", **run_grad_step(args)}), flush=True)
    elif args.impl == "ours":
        run_ours(args)
    elif args.impl == "reference":
        run_reference_cpu(args)
    else:
        run_reference_gpu(args)
    return 0


if __name__ == "__main__":
    sys.exit(main())
