"""Benchmark of the reionization grid step on B200.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config NAME] [--mode fused|plain]

One step = one snapshot of the configured workload on seeded synthetic grids
(inputs resident in HBM before the timed region).  The metric is ms per
snapshot (lower is better), whole-job: with N ranks each rank processes its own
snapshot per step (independent replicas: a snapshot does not shard), so the job
time per snapshot is the max-over-ranks step time divided by N.

Between timed steps the per-cell state is reset and a 512 MiB buffer is written
to flush L2; each step is timed with CUDA events on the stream the library
launches on.  ``e2e`` times the host-buffer entry point (pinned host inputs,
host<->device copies inside the timed region).  ``roofline`` comes from a
separate pass with the library's per-kernel CUDA-event timing switched on.
``--impl reference`` times the CPU restatement of the reference algorithm
(the reference itself cannot be built: FFTW/GSL/HDF5/MPI are absent).
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "meraxes-devs_qyxnew_b200")
sys.path.insert(0, PKG)

import numpy as np  # noqa: E402

import workloads as wl  # noqa: E402

METRIC = "ms/snapshot find_HII_bubbles+Ts at 256^3/512^3"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c1_256")
    ap.add_argument("--mode", default="fused", choices=["fused", "plain"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def config_params(cfg: wl.GridConfig, rg):
    return rg.make_params(cfg.n, cfg.box, Flag_EvolvingReionRBubbleMax=cfg.evolving_rmax,
                          ReionRBubbleMax=cfg.r_bubble_max, ReionRBubbleMin=cfg.r_bubble_min,
                          ReionDeltaRFactor=cfg.delta_r_factor, ReionFilterType=cfg.filter_type,
                          ReionEfficiency=cfg.efficiency, ReionUVBFlag=cfg.uvb_flag)


def workload_desc(cfg: wl.GridConfig, nr: int) -> dict:
    return {"workload": f"find_HII_bubbles {cfg.n}^3 float32, box {cfg.box:g} Mpc/h, z={cfg.z:g}, "
                        f"filter {cfg.filter_type}, {nr} radii, ReionEfficiency {cfg.efficiency:g}",
            "grid": cfg.n, "box_mpc_h": cfg.box, "redshift": cfg.z, "radii": nr,
            "filter_type": cfg.filter_type, "l2": "flushed (512 MiB write) before every timed step; inputs > L2"}


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower().startswith("active")})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def measured_peak():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_from_profiles(kernel: str, cfg_name: str):
    """Per-launch DRAM bytes recorded from an ncu capture, if a summary is committed."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for f in sorted(os.listdir(pdir)):
        if kernel in f and cfg_name in f and f.endswith(".md"):
            m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(os.path.join(pdir, f)).read())
            if m:
                return float(m.group(1))
    return None


# ---------------------------------------------------------------------------

def cpu_sample(cfg: wl.GridConfig, src, sample_radii: int = 4):
    """Time the CPU restatement (oracle, float32 pocketfft on all cores) on a bounded
    sample of one snapshot: the forward transforms, ``sample_radii`` filter radii and
    the closing pass, extrapolated to the full radius count."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import reion_oracle as ro
    import tables
    ro.set_recfast(tables.Recfast(tables.default_tables_dir()).T)
    p = ro.Params(ReionGridDim=cfg.n, BoxSize=cfg.box, Flag_EvolvingReionRBubbleMax=cfg.evolving_rmax,
                  ReionRBubbleMax=cfg.r_bubble_max, ReionRBubbleMin=cfg.r_bubble_min,
                  ReionDeltaRFactor=cfg.delta_r_factor, ReionFilterType=cfg.filter_type,
                  ReionEfficiency=cfg.efficiency, ReionUVBFlag=cfg.uvb_flag)
    st = ro.HIIState.fresh(cfg.n)
    t0 = time.perf_counter()
    _, _, _, diag = ro.find_hii_bubbles(p, cfg.z, src.deltax, src.stars, src.sfr, st, "fp32",
                                        radius_subset=sample_radii, with_dead_grids=True)
    wall = time.perf_counter() - t0
    nr = diag["n_radii"]
    t = diag["timing"]
    est = t["forward"] + t["per_radius"] * nr + t["final"]
    return est * 1e3, wall, nr, os.cpu_count()


def run_reference(args, cfg):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    src = wl.make_sources(cfg.n, cfg.box, cfg.seed, cfg.source_scale)
    vals = []
    nr = 0
    for i in range(args.warmup + args.steps):
        ms, wall, nr, cores = cpu_sample(cfg, src)
        if i >= args.warmup:
            vals.append(ms)
    v = statistics.mean(vals)
    sample = (f"1 snapshot of {cfg.n}^3: forward r2c + 4 of {nr} radii + closing pass per step, "
              f"extrapolated to {nr} radii")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "ms/snapshot", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": v, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators)",
            "config": workload_desc(cfg, nr),
            "cpu_baseline": {"value": v, "unit": "ms/snapshot", "cores": os.cpu_count(), "kind": "port",
                             "sample": sample + "; oracle restatement, scipy pocketfft float32, all host cores "
                                                "(the reference needs FFTW/GSL/MPI, absent here)"},
            "e2e": {"value": v, "unit": "ms/snapshot", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, cfg):
    import torch
    import rg_b200 as rg

    ws, rank, local = dist_env()
    if ws > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    n = cfg.n
    src = wl.make_sources(n, cfg.box, cfg.seed + rank, cfg.source_scale)
    p = config_params(cfg, rg)
    zz, snap = wl.snapshot_redshifts(cfg.z)
    s = rg.snapshot(zz, snap)
    ctx = rg.Context(n, device=local)
    ctx.call("rg_set_mode", rg.RG_MODE_PLAIN if args.mode == "plain" else rg.RG_MODE_FUSED)
    stream = torch.cuda.current_stream(dev)
    ctx.call("rg_set_stream", C.c_void_p(stream.cuda_stream))

    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32).ravel()).to(dev)
    nreal = n ** 3
    bufs = {"deltax": t(src.deltax), "stars": t(src.stars), "weighted_sfr": t(src.sfr)}
    for k in ("xH", "r_bubble", "z_at_ionization", "J_21_at_ionization", "temp_kinetic_all_gas"):
        bufs[k] = torch.zeros(nreal, device=dev)
    g = rg.rg_grids()
    for k, v in bufs.items():
        setattr(g, k, v.data_ptr())
    out = rg.rg_hii_scalars()
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def reset():
        bufs["z_at_ionization"].fill_(-1.0)
        bufs["J_21_at_ionization"].zero_()
        bufs["temp_kinetic_all_gas"].zero_()
        flush.zero_()

    def step():
        ctx.call("rg_find_HII_bubbles", C.byref(p), C.byref(s), C.byref(g), C.byref(out))

    for _ in range(args.warmup):
        reset()
        step()
    torch.cuda.synchronize(dev)
    if ws > 1:
        torch.distributed.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    times = []
    for _ in range(args.steps):
        reset()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    ms_step = statistics.mean(times)
    if ws > 1:
        tt = torch.tensor([ms_step], device=dev)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        ms_step = float(tt.item())
        torch.distributed.barrier()
    nr = out.n_radii
    value = ms_step / ws

    # e2e through the host-buffer entry point: pinned host inputs and outputs
    e2e = None
    if not args.no_e2e:
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32).ravel()).pin_memory()
        hb = {"deltax": pin(src.deltax), "stars": pin(src.stars), "weighted_sfr": pin(src.sfr)}
        for k in ("xH", "r_bubble", "J_21_at_ionization", "temp_kinetic_all_gas"):
            hb[k] = torch.zeros(nreal).pin_memory()
        hb["z_at_ionization"] = torch.full((nreal,), -1.0).pin_memory()
        hg = rg.rg_grids()
        for k, v in hb.items():
            setattr(hg, k, v.data_ptr())
        h2d = sum(hb[k].numel() * 4 for k in ("deltax", "stars", "weighted_sfr", "z_at_ionization",
                                              "J_21_at_ionization", "temp_kinetic_all_gas"))
        d2h = sum(hb[k].numel() * 4 for k in ("xH", "r_bubble", "z_at_ionization", "J_21_at_ionization",
                                              "temp_kinetic_all_gas"))
        o2 = rg.rg_hii_scalars()
        et = []
        for i in range(args.warmup + args.steps):
            hb["z_at_ionization"].fill_(-1.0)
            hb["J_21_at_ionization"].zero_()
            hb["temp_kinetic_all_gas"].zero_()
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.call("rg_find_HII_bubbles_host", C.byref(p), C.byref(s), C.byref(hg), C.byref(o2))
            e1.record(stream)
            e1.synchronize()
            if i >= args.warmup:
                et.append(e0.elapsed_time(e1))
        em = statistics.mean(et)
        if ws > 1:
            tt = torch.tensor([em], device=dev)
            torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
            em = float(tt.item())
        e2e = {"value": em / ws, "unit": "ms/snapshot", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}

    # roofline pass: per-kernel CUDA events inside the library
    ctx.profile(True)
    for _ in range(max(2, min(args.steps, 3))):
        reset()
        step()
    stats = ctx.kernel_stats()
    ctx.profile(False)
    launches = sum(k["launches"] for k in stats) // max(2, min(args.steps, 3))
    top = max(stats, key=lambda k: k["ms_total"])
    peak, peak_kind = measured_peak()
    ach = top["alg_bytes_total"] / (top["ms_total"] * 1e-3) / 1e9
    per_launch_bytes = top["alg_bytes_total"] / top["launches"]
    traffic = traffic_from_profiles(top["name"], cfg.name)
    total_ms = sum(k["ms_total"] for k in stats)
    roofline = {"bound": "hbm", "kernel": top["name"], "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": ach / peak, "peak_kind": peak_kind, "traffic": traffic,
                "alg_bytes_per_launch": per_launch_bytes,
                "share_of_step": top["ms_total"] / total_ms if total_ms > 0 else None,
                "kernels": {k["name"]: {"launches": k["launches"], "ms": k["ms_total"],
                                        "GBps": k["alg_bytes_total"] / max(k["ms_total"], 1e-9) / 1e6}
                            for k in stats}}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        ms_cpu, wall, nr_c, cores = cpu_sample(cfg, src)
        cpu = {"value": ms_cpu, "unit": "ms/snapshot", "cores": cores, "kind": "port",
               "sample": f"1 snapshot of {n}^3: forward r2c + 4 of {nr_c} radii + closing pass, extrapolated to "
                         f"{nr_c} radii; oracle restatement, scipy pocketfft float32 on all host cores "
                         f"({wall:.1f} s wall)"}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "ms/snapshot", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators, BASELINE shapes)",
                "config": dict(workload_desc(cfg, nr), mode=args.mode, parallelism=f"replicas x{ws}"),
                "e2e": e2e, "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu,
                "clocks": clk, "mean_xH": out.volume_weighted_global_xH}
        print(json.dumps(line), flush=True)
    ctx.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


def main():
    args = parse()
    cfg = wl.CONFIGS[args.config]
    if args.impl == "reference":
        run_reference(args, cfg)
    else:
        run_ours(args, cfg)


if __name__ == "__main__":
    main()
