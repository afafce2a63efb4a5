"""Benchmark of the reionization grid step on B200.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config NAME] [--mode fused|plain]

One step = one snapshot of the configured workload on seeded synthetic grids, with
the inputs resident in HBM before the timed region.  The default workload is the
full step at 512^3 (box 500 Mpc/h, z = 8): ComputeTs (40 shells) -> find_HII_bubbles
(61 radii) -> delta_T, in the reference's order (src/core/dracarys.c:383-391).
``--config c1_256`` times find_HII_bubbles alone at 256^3.

The metric is ms per snapshot (lower is better), whole job: with N ranks each rank
processes its own snapshot per step (independent replicas: a snapshot does not
shard), so the job time per snapshot is the max-over-ranks step time divided by N.

Between timed steps the per-cell state is restored and a 512 MiB buffer is written
to flush L2; each step is timed with CUDA events on the stream the library launches
on.  ``e2e`` times the combined host-buffer entry point rg_reion_step_host (pinned host
inputs, host<->device copies inside the timed region); the three separate host-buffer
calls are timed beside it (``e2e.three_calls``).  ``roofline`` comes from a separate pass with the
library's per-kernel CUDA-event timing switched on.  ``--impl reference`` times the
CPU restatement of the reference algorithm on bounded samples (the reference itself
cannot be built: FFTW/GSL/HDF5/MPI are absent).
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
DATA_DESC = "synthetic (seeded generators at the workload's shapes and sizes)"
DEFAULT_CONFIG = "c4_512"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default=DEFAULT_CONFIG)
    ap.add_argument("--mode", default="fused", choices=["fused", "plain"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the timings reported under extras")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--only-extra", choices=["dft_y_pass_256"],
                    help="run only this extra timing on one GPU and print it (for profiling)")
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
                          ReionEfficiency=cfg.efficiency, ReionUVBFlag=cfg.uvb_flag,
                          Flag_IncludeSpinTemp=cfg.spin_temp, TsHeatingFilterType=cfg.ts_filter_type,
                          TsNumFilterSteps=cfg.ts_steps)


def oracle_params(cfg: wl.GridConfig):
    import reion_oracle as ro
    return ro.Params(ReionGridDim=cfg.n, BoxSize=cfg.box, Flag_EvolvingReionRBubbleMax=cfg.evolving_rmax,
                     ReionRBubbleMax=cfg.r_bubble_max, ReionRBubbleMin=cfg.r_bubble_min,
                     ReionDeltaRFactor=cfg.delta_r_factor, ReionFilterType=cfg.filter_type,
                     ReionEfficiency=cfg.efficiency, ReionUVBFlag=cfg.uvb_flag, Flag_IncludeSpinTemp=cfg.spin_temp,
                     TsHeatingFilterType=cfg.ts_filter_type, TsNumFilterSteps=cfg.ts_steps)


def workload_desc(cfg: wl.GridConfig, nr: int) -> dict:
    what = "ComputeTs -> find_HII_bubbles -> delta_T" if cfg.spin_temp else "find_HII_bubbles"
    ts = f", {cfg.ts_steps} Ts shells (heating filter {cfg.ts_filter_type})" if cfg.spin_temp else ""
    return {"workload": f"{what}, {cfg.n}^3 float32, box {cfg.box:g} Mpc/h, z={cfg.z:g}, "
                        f"filter {cfg.filter_type}, {nr} radii{ts}, ReionEfficiency {cfg.efficiency:g}",
            "name": cfg.name, "grid": cfg.n, "box_mpc_h": cfg.box, "redshift": cfg.z, "radii": nr,
            "ts_shells": cfg.ts_steps if cfg.spin_temp else 0, "filter_type": cfg.filter_type,
            "l2": "flushed (512 MiB write) before every timed step; inputs > L2"}


def alg_bytes(cfg: wl.GridConfig, nr: int, live_grids: int) -> float:
    """Algorithmic HBM bytes per snapshot (B_HII + B_Ts + B_dT), Nc = N^2 (N/2 + 1)."""
    n = cfg.n
    n3 = float(n) ** 3
    nc = float(n) * n * (n // 2 + 1)
    b = live_grids * (4 * n3 + 8 * nc) + nr * (live_grids * 8 * nc + 8 * n3) + 24 * n3
    if cfg.spin_temp:
        b += cfg.ts_steps * (2 * (4 * n3 + 16 * nc) + 36 * n3) + 24 * n3
        b += 16 * n3
    return b


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
    pat = re.compile(r"traffic_bytes_per_launch\[" + re.escape(kernel) + "@" + re.escape(cfg_name) + r"\]:\s*([0-9.eE+]+)")
    for f in sorted(os.listdir(pdir)):
        if f.endswith(".md"):
            m = pat.search(open(os.path.join(pdir, f)).read())
            if m:
                return float(m.group(1))
    return None


# ---------------------------------------------------------------------------
# inputs

def history_slots(cfg, rg, zz, snap):
    """History slots the shells use (from the library's host coefficient engine, no device work)."""
    p = config_params(cfg, rg)
    _, _, coef = rg.ts_tables(p, zz, snap, snap + 1, 2e-4, 1e-3, np.zeros(len(zz)), with_freq=False)
    used = np.nonzero(np.any(coef != 0, axis=0))[0]
    return int(used.max()) if used.size else 0       # sources 1..k = history slots 0..k-1


def make_inputs(cfg, rank, zz, snap, n_hist):
    src = wl.make_sources(cfg.n, cfg.box, cfg.seed + rank, cfg.source_scale)
    ti = wl.make_config_ts_inputs(src, zz, snap, n_hist) if cfg.spin_temp else None
    return src, ti


# ---------------------------------------------------------------------------
# CPU restatement on bounded samples

def oracle_history_slots(cfg, zz, snap):
    """History slots the shells read, from the oracle's own shell schedule (no library call)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ts_oracle as to
    sh, _ = to.shells_and_sources(oracle_params(cfg), zz, snap, None, None, None, None, want_grids=False)
    return sh.max_slot + 1


class CpuSampler:
    """The oracle (float32 pocketfft on all host cores) timed on bounded samples of one snapshot.

    ``fixed()`` times, once, the parts that run once per snapshot: the forward r2c of every
    find_HII grid and the closing pass; ComputeTs' history re-weighting and per-cell update on a
    few x-planes (scaled by N / planes), the frequency tables of two shells (scaled by nS / 2),
    the x_e interpolation nodes; delta_T in full.  ``sample(i)`` times one radius of the
    excursion set (window, inverse FFTs, barrier test; successive radius samples walk the schedule
    in steps of 7) or, on odd i with ComputeTs, one Ts shell (r2c, filter, c2r, sums; shells in
    steps of 3).  A snapshot's estimate is fixed + nR x mean radius + nS x mean shell."""

    def __init__(self, cfg, src, ti, zz, snap):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import reion_oracle as ro
        import tables
        ro.set_recfast(tables.Recfast(tables.default_tables_dir()).T)
        self.ro = ro
        self.cfg, self.src, self.ti, self.zz, self.snap = cfg, src, ti, zz, snap
        self.p = oracle_params(cfg)
        self.n = cfg.n
        self.nr = len(ro.radius_schedule(self.p, cfg.z))
        self.nS = self.p.TsNumFilterSteps if cfg.spin_temp else 0
        self.spectra = None
        self.fixed_s = None
        self.desc = ""
        self.radius_s, self.shell_s = [], []

    def _hii(self, **kw):
        ro, src, ti, n = self.ro, self.src, self.ti, self.n
        st = ro.HIIState.fresh(n)
        xe = wl.from_padded(ti.x_e_box_prev) if ti is not None else None
        tk = ti.Tk_box if ti is not None else None
        return ro.find_hii_bubbles(self.p, self.cfg.z, src.deltax, src.stars, src.sfr, st, "fp32",
                                   x_e_box=xe, Tk_box=tk, with_dead_grids=True, **kw)

    def fixed(self, planes: int = 0, table_shells: int = 2):
        ro, src, ti, n, U = self.ro, self.src, self.ti, self.n, wl.from_padded
        parts = {}
        _, _, _, d = self._hii(radius_indices=(), skip_final=True)
        parts["hii_forward"] = d["timing"]["forward"]
        self.spectra = d["spectra"]
        t0 = time.perf_counter()
        self._hii(radius_indices=(), spectra_in=self.spectra)
        parts["hii_closing_pass"] = time.perf_counter() - t0
        desc = [f"find_HII_bubbles: forward r2c + closing pass once, 1 of {self.nr} radii per sample x {self.nr}"]
        if ti is not None:
            import ts_oracle as to
            self.to = to
            p, zz, snap = self.p, self.zz, self.snap
            self.T = to.TsTables()
            to.gk61_rule()                 # the quadrature rule is set up once, outside the timed parts
            cm = to.Cosmo(p)
            self.zp = zp = float(zz[snap])
            nS = self.nS
            planes = planes or max(1, n // 64)
            xprev = U(ti.x_e_box_prev)
            t0 = time.perf_counter()
            sh, _ = to.shells_and_sources(p, zz, snap, U(src.sfr)[:planes], U(src.xray)[:planes],
                                          [U(a)[:planes] for a in ti.sfr_histories],
                                          [U(a)[:planes] for a in ti.xray_histories])
            parts["ts_history_reweighting"] = (time.perf_counter() - t0) * n / planes
            self.sh = sh
            sub = to.Shells()
            for k in ("R", "zpp_edge", "zpp", "dzpp", "dt_dzpp"):
                setattr(sub, k, getattr(sh, k)[:table_shells])
            sub.final_weight = sh.final_weight
            t0 = time.perf_counter()
            heat, ion, lya, sum_lyn = to.freq_tables(p, self.T, sub, zp, float(np.mean(xprev)), 1e-3, zz,
                                                     ti.stored_fcoll, snap)
            parts["ts_frequency_tables"] = (time.perf_counter() - t0) * nS / table_shells
            self.tabs = tuple(np.repeat(a[:, :1], nS, axis=1) for a in (heat, ion, lya))
            self.lyn = np.repeat(sum_lyn[:1], nS)
            t0 = time.perf_counter()
            self.xi = to.xe_interp_index(self.T, xprev)
            parts["ts_xe_nodes"] = time.perf_counter() - t0
            sums = [np.zeros((planes, n, n)) for _ in range(4)]
            pf = to.prefactors(p, zp)
            d = U(src.deltax)[:planes]
            t0 = time.perf_counter()
            to.finish_sums(p, cm, pf, zp, d, sums)
            to.evolve_cells(p, cm, self.T, pf, zp, zp - float(zz[snap - 1]), d, xprev[:planes], ti.Tk_box[:planes],
                            sums)
            parts["ts_per_cell_update"] = (time.perf_counter() - t0) * n / planes
            t0 = time.perf_counter()
            ro.delta_T(p, self.cfg.z, np.full((n, n, n), 0.5, np.float32), U(src.deltax), ti.Tk_box)
            parts["delta_T"] = time.perf_counter() - t0
            self.sums = [np.zeros((n, n, n)) for _ in range(4)]
            desc.append(f"ComputeTs: history re-weighting and per-cell update on {planes} of {n} x-planes "
                        f"x {n / planes:g}, frequency tables of {table_shells} shells x {nS / table_shells:g}, "
                        f"1 of {nS} shells (r2c, filter, c2r, sums) per sample x {nS}; delta_T in full once")
        self.fixed_s = parts
        self.desc = "; ".join(desc)
        return parts

    def sample(self, i: int):
        """One radius (even i, or every i without ComputeTs) or one Ts shell (odd i).  Returns the
        wall seconds of the sample; ``estimate()`` combines the samples taken so far."""
        t0 = time.perf_counter()
        if not self.nS or i % 2 == 0:
            ir = ((i // 2 if self.nS else i) * 7) % self.nr
            _, _, _, d = self._hii(radius_indices=(ir,), spectra_in=self.spectra, skip_final=True)
            self.radius_s.append(d["timing"]["per_radius"])
        else:
            U = wl.from_padded
            r = 1 + ((i // 2) * 3) % (self.nS - 1) if self.nS > 1 else 0
            t1 = time.perf_counter()
            self.to.shell_accumulate(self.p, self.sh, r, U(self.src.sfr), U(self.src.xray), self.xi, self.tabs,
                                     self.lyn, self.zp, self.sums, "fp32")
            self.shell_s.append(time.perf_counter() - t1)
        return time.perf_counter() - t0

    def estimate(self):
        """ms per snapshot: fixed parts + nR x mean radius + nS x mean shell."""
        t_r = statistics.mean(self.radius_s)
        t_s = statistics.mean(self.shell_s) if self.nS else 0.0
        return (sum(self.fixed_s.values()) + self.nr * t_r + self.nS * t_s) * 1e3


def run_reference(args, cfg):
    """The reference arm: the CPU restatement of the reference algorithm (the oracle), rank 0 only.
    It loads nothing of the library."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    zz, snap = wl.snapshot_redshifts(cfg.z)
    n_hist = oracle_history_slots(cfg, zz, snap) if cfg.spin_temp else 0
    src, ti = make_inputs(cfg, 0, zz, snap, n_hist)
    cs = CpuSampler(cfg, src, ti, zz, snap)
    w0 = time.perf_counter()
    cs.fixed()
    fixed_wall = time.perf_counter() - w0
    walls = []
    for i in range(args.warmup):
        cs.sample(i)
    cs.radius_s, cs.shell_s = [], []
    for i in range(args.warmup, args.warmup + args.steps):
        walls.append(cs.sample(i))
    if not cs.radius_s or (cs.nS and not cs.shell_s):
        cs.sample(0 if not cs.radius_s else 1)        # fewer than two timed steps: one more sample
    v = cs.estimate()
    sample_ms = statistics.mean(walls) * 1e3
    desc = (cs.desc + f"; each timed step is one sample, a radius or a shell in turn ({sample_ms / 1e3:.2f} s "
            f"wall on average), the snapshot value is extrapolated from the samples and the once-per-snapshot "
            f"parts ({fixed_wall:.1f} s wall, timed before the warm-up); oracle restatement, scipy pocketfft "
            "float32, all host cores (the reference's path needs FFTW, GSL, MPI and HDF5, absent here; its "
            "C compiled over in-tree stand-ins pins the oracle but would time a plain stand-in FFT, not FFTW)")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "ms/snapshot", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sample_ms, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": DATA_DESC,
            "config": workload_desc(cfg, cs.nr), "extrapolated": True,
            "fixed_parts_s": cs.fixed_s, "radius_sample_s": statistics.mean(cs.radius_s),
            "shell_sample_s": statistics.mean(cs.shell_s) if cs.shell_s else None,
            "cpu_baseline": {"value": v, "unit": "ms/snapshot", "cores": os.cpu_count(), "kind": "port",
                             "sample": desc},
            "e2e": {"value": v, "unit": "ms/snapshot", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# the GPU arm

class Workload:
    """Device grids of one snapshot and the step through the library's device entry points."""

    def __init__(self, cfg, rg, torch, dev, ctx, src, ti, zz, snap, n_hist):
        self.cfg, self.rg, self.torch, self.dev, self.ctx = cfg, rg, torch, dev, ctx
        n = cfg.n
        self.n = n
        npad = n * n * 2 * (n // 2 + 1)
        nreal = n ** 3
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32).ravel()).to(dev)
        b = {"deltax": t(src.deltax), "stars": t(src.stars), "weighted_sfr": t(src.sfr)}
        for k in ("xH", "r_bubble", "z_at_ionization", "J_21_at_ionization", "temp_kinetic_all_gas", "delta_T"):
            b[k] = torch.zeros(nreal, device=dev)
        self.spin = bool(cfg.spin_temp)
        if self.spin:
            b["sfr"] = t(src.sfr)
            b["xray_luminosity"] = t(src.xray)
            b["x_e_box_prev"] = t(ti.x_e_box_prev)
            b["x_e_box"] = torch.zeros(npad, device=dev)
            b["Tk_box"] = t(ti.Tk_box)
            b["TS_box"] = torch.zeros(nreal, device=dev)
            self.xe0 = b["x_e_box_prev"].clone()
            self.tk0 = b["Tk_box"].clone()
            if n_hist:
                b["sfr_histories"] = torch.cat([t(a) for a in ti.sfr_histories])
                b["xray_luminosity_histories"] = torch.cat([t(a) for a in ti.xray_histories])
        self.b = b
        g = rg.rg_grids()
        for k, v in b.items():
            setattr(g, k, v.data_ptr())
        g.n_hist = n_hist
        self.g = g
        self.p = config_params(cfg, rg)
        self.sf0 = ti.stored_fcoll.copy() if ti is not None else np.zeros(len(zz))
        self.sf = self.sf0.copy()
        self.s = rg.snapshot(zz, snap, self.sf)
        self.hii = rg.rg_hii_scalars()
        self.ts = rg.rg_ts_scalars()
        self.tb = C.c_double()
        self.flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def reset(self):
        b = self.b
        b["z_at_ionization"].fill_(-1.0)
        b["J_21_at_ionization"].zero_()
        b["temp_kinetic_all_gas"].zero_()
        if self.spin:
            b["x_e_box_prev"].copy_(self.xe0)
            b["Tk_box"].copy_(self.tk0)
        self.sf[:] = self.sf0
        self.flush.zero_()

    def step(self):
        ctx, g, p, s = self.ctx, C.byref(self.g), C.byref(self.p), C.byref(self.s)
        if self.spin:
            ctx.call("rg_compute_Ts", p, s, g, C.byref(self.ts))
        ctx.call("rg_find_HII_bubbles", p, s, g, C.byref(self.hii))
        if self.spin:
            ctx.call("rg_delta_T", p, s, g, C.byref(self.tb))


class HostWorkload:
    """The same snapshot through the host-buffer entry points (pinned host arrays)."""

    def __init__(self, wk: Workload, src, ti, n_hist):
        torch, rg = wk.torch, wk.rg
        self.wk = wk
        n = wk.n
        nreal = n ** 3
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32).ravel()).pin_memory()
        h = {"deltax": pin(src.deltax), "stars": pin(src.stars), "weighted_sfr": pin(src.sfr)}
        for k in ("xH", "r_bubble", "J_21_at_ionization", "temp_kinetic_all_gas", "delta_T"):
            h[k] = torch.zeros(nreal).pin_memory()
        h["z_at_ionization"] = torch.full((nreal,), -1.0).pin_memory()
        if wk.spin:
            h["sfr"] = pin(src.sfr)
            h["xray_luminosity"] = pin(src.xray)
            h["x_e_box_prev"] = pin(ti.x_e_box_prev)
            h["x_e_box"] = torch.zeros_like(h["x_e_box_prev"]).pin_memory()
            h["Tk_box"] = pin(ti.Tk_box)
            h["TS_box"] = torch.zeros(nreal).pin_memory()
            self.xe0 = h["x_e_box_prev"].clone()
            self.tk0 = h["Tk_box"].clone()
            if n_hist:
                h["sfr_histories"] = torch.cat([pin(a) for a in ti.sfr_histories]).pin_memory()
                h["xray_luminosity_histories"] = torch.cat([pin(a) for a in ti.xray_histories]).pin_memory()
        self.h = h
        hg = rg.rg_grids()
        for k, v in h.items():
            setattr(hg, k, v.data_ptr())
        hg.n_hist = n_hist
        self.hg = hg
        bp = 4 * n * n * 2 * (n // 2 + 1)
        br = 4 * nreal
        # bytes each entry point copies (rg_api.cu / rg_dT.cu / rg_ts.cu host forms)
        h2d = 3 * bp + 3 * br                                   # find_HII: deltax, stars, weighted_sfr, 3 state
        d2h = 5 * br
        if wk.spin:
            h2d += bp + br                                      # find_HII: x_e_box, Tk_box
            used = history_slots(wk.cfg, rg, *self.zzsnap()) + 1   # source grids staged by rg_compute_Ts_host
            h2d += 3 * bp + br + 2 * used * bp                  # Ts: deltax, stars, x_e_box_prev, Tk_box, sources
            d2h += 2 * bp + 2 * br                              # Ts: x_e_box_prev, x_e_box, Tk_box, TS_box
            h2d += bp + 2 * br                                  # delta_T: deltax, xH, TS_box
            d2h += br                                           # delta_T: delta_T
        self.h2d, self.d2h = h2d, d2h
        # the combined call (rg_reion_step_host): each input once, each output once
        if wk.spin:
            self.h2d_step = 4 * bp + 4 * br + 2 * used * bp             # deltax stars x_e_prev wsfr; Tk z_in J21 temp
            self.d2h_step = 2 * bp + 8 * br                            # x_e_prev x_e; Tk TS xH r_bubble z_in J21 temp dT
        else:
            self.h2d_step, self.d2h_step = 3 * bp + 3 * br, 6 * br

    def zzsnap(self):
        s = self.wk.s
        return np.ctypeslib.as_array(s.ZZ, shape=(s.n_snapshots,)).copy(), s.snapshot

    def reset(self):
        h = self.h
        h["z_at_ionization"].fill_(-1.0)
        h["J_21_at_ionization"].zero_()
        h["temp_kinetic_all_gas"].zero_()
        if self.wk.spin:
            h["x_e_box_prev"].copy_(self.xe0)
            h["Tk_box"].copy_(self.tk0)
        self.wk.sf[:] = self.wk.sf0
        self.wk.flush.zero_()

    def step(self):
        """The snapshot through the three host-buffer entry points, one after another."""
        wk = self.wk
        ctx, g, p, s = wk.ctx, C.byref(self.hg), C.byref(wk.p), C.byref(wk.s)
        if wk.spin:
            ctx.call("rg_compute_Ts_host", p, s, g, C.byref(wk.ts))
        ctx.call("rg_find_HII_bubbles_host", p, s, g, C.byref(wk.hii))
        if wk.spin:
            ctx.call("rg_delta_T_host", p, s, g, C.byref(wk.tb))

    def step_combined(self):
        """The snapshot through the combined host-buffer entry point (the reference's per-snapshot
        block of ComputeTs, find_HII_bubbles and the brightness temperature)."""
        wk = self.wk
        hg = self.hg
        if not wk.spin:
            hg.delta_T = None
        wk.ctx.call("rg_reion_step_host", C.byref(wk.p), C.byref(wk.s), C.byref(hg), C.byref(wk.ts),
                    C.byref(wk.hii), C.byref(wk.tb))


def time_recombinations(wk, ctx, torch, stream, dev):
    rg = wk.rg
    n = wk.n
    npad, nreal = n * n * 2 * (n // 2 + 1), n ** 3
    ctx.set_recombination_tables(*wl.rec_stand_in_tables())
    # recombinations accumulated over earlier snapshots (N_rec up to 0.4 per baryon) and an
    # ionising background, so the barrier's 1 + N_rec term and the recombination closing pass see
    # non-zero state
    gen = torch.Generator(device=dev).manual_seed(7)
    extra = {"Gamma12": torch.rand(nreal, device=dev, generator=gen) * 0.5,
             "N_rec": torch.rand(npad, device=dev, generator=gen) * 0.4,
             "residual_xH": torch.zeros(nreal, device=dev), "clumping_factor": torch.zeros(nreal, device=dev),
             "t_resp": torch.full((nreal,), 1e30, device=dev)}
    gr = rg.rg_grids.from_buffer_copy(wk.g)
    for k, v in extra.items():
        setattr(gr, k, v.data_ptr())
    pr = rg.rg_params.from_buffer_copy(wk.p)
    pr.Flag_IncludeRecombinations = 1
    out = rg.rg_hii_scalars()
    res = {}
    for name, p in (("ms", pr), ("ms_without", wk.p)):
        call = lambda: ctx.call("rg_find_HII_bubbles", C.byref(p), C.byref(wk.s), C.byref(gr), C.byref(out))
        call()
        torch.cuda.synchronize(dev)
        t = []
        for _ in range(3):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            call()
            e1.record(stream)
            e1.synchronize()
            t.append(e0.elapsed_time(e1))
        res[name] = statistics.mean(t)
        if name == "ms":
            res["mean_N_rec"] = out.volume_weighted_global_N_rec
    wk.reset()
    res["what"] = ("rg_find_HII_bubbles at the workload's size with Flag_IncludeRecombinations (N_rec and "
                   "weighted_sfr filtered, the recombination closing pass) on stand-in MHR tables; ms_without "
                   "is the same call without recombinations")
    del extra
    return res


def time_dft_y_pass(rg, torch, dev, reps=5, ng=4):
    """The y pass of ng whole 256^3 spectra (ng x 135 MB, above L2) by the FP32 register transform
    and by the split-BF16 tensor-core form (rg_dft_y_pass), kernel times from the library's
    events, and each form's relative L2 error against numpy's FP64 transform of 8 kz planes."""
    import numpy as np
    n, nz = 256, 129
    ctx = rg.Context(n)
    g = torch.Generator(device=dev).manual_seed(5)
    base = torch.complex(torch.randn(ng * nz * n * n, device=dev, generator=g),
                         torch.randn(ng * nz * n * n, device=dev, generator=g))
    sample = base[: 8 * n * n].cpu().numpy().reshape(8, n, n).astype(np.complex128)
    want = np.fft.fft(sample, axis=-1)
    res = {}
    for name, impl in (("fp32", rg.RG_DFT_FP32), ("tc_bf16x3", rg.RG_DFT_TC_BF16X3)):
        work = base.clone()
        ctx.call("rg_dft_y_pass", work.data_ptr(), 1, 0, impl)
        got = work[: 8 * n * n].cpu().numpy().reshape(8, n, n)
        err = float(np.linalg.norm(got - want) / np.linalg.norm(want))
        ctx.profile(True)
        for _ in range(reps):
            ctx.call("rg_dft_y_pass", work.data_ptr(), ng, 0, impl)
        st = {k["name"]: k for k in ctx.kernel_stats()}
        ctx.profile(False)
        k = next(v for kname, v in st.items() if kname.startswith("dft_y"))
        ms = k["ms_total"] / reps
        res[name] = {"ms": ms, "GBps": k["alg_bytes_total"] / reps / (ms * 1e-3) / 1e9, "rel_l2_vs_fp64": err}
        del work
    ctx.close()
    res["speedup_tc_over_fp32"] = res["fp32"]["ms"] / res["tc_bf16x3"]["ms"]
    res["what"] = (f"one forward c2c pass along y over {ng} Hermitian 256^3 spectra (16 B per complex value "
                   "read and written): FP32 register Stockham transform vs split-BF16 tcgen05 matrix products "
                   "(256 = 16 x 16, three BF16 products per radix-16 stage, FP32 accumulation in tensor memory)")
    return res


def timed(torch, stream, fn, reset, warmup, steps):
    for _ in range(warmup):
        reset()
        fn()
    torch.cuda.synchronize()
    times = []
    for _ in range(steps):
        reset()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    return times


def run_ours(args, cfg):
    import torch
    import rg_b200 as rg

    ws, rank, local = dist_env()
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    zz, snap = wl.snapshot_redshifts(cfg.z)
    n_hist = history_slots(cfg, rg, zz, snap) if cfg.spin_temp else 0
    src, ti = make_inputs(cfg, rank, zz, snap, n_hist)
    ctx = rg.Context(cfg.n, device=local)
    ctx.call("rg_set_mode", rg.RG_MODE_PLAIN if args.mode == "plain" else rg.RG_MODE_FUSED)
    stream = torch.cuda.current_stream(dev)
    ctx.call("rg_set_stream", C.c_void_p(stream.cuda_stream))
    wk = Workload(cfg, rg, torch, dev, ctx, src, ti, zz, snap, n_hist)

    for _ in range(args.warmup):
        wk.reset()
        wk.step()
    torch.cuda.synchronize(dev)
    if ws > 1:
        torch.distributed.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    times = timed(torch, stream, wk.step, wk.reset, 0, args.steps)
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    ms_step = statistics.mean(times)
    if ws > 1:
        tt = torch.tensor([ms_step], device=dev)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        ms_step = float(tt.item())
        torch.distributed.barrier()
    nr = wk.hii.n_radii
    value = ms_step / ws
    results = {"mean_xH": wk.hii.volume_weighted_global_xH}
    if wk.spin:
        results.update(mean_TS=wk.ts.volume_ave_TS, mean_TK=wk.ts.volume_ave_TK, mean_xe=wk.ts.volume_ave_xe,
                       mean_Tb=wk.tb.value, collapse_fraction=wk.ts.collapse_fraction)

    # e2e through the host-buffer entry points
    e2e = None
    if not args.no_e2e:
        hw = HostWorkload(wk, src, ti, n_hist)
        et = timed(torch, stream, hw.step_combined, hw.reset, args.warmup, args.steps)
        e3 = timed(torch, stream, hw.step, hw.reset, max(1, args.warmup // 2), args.steps)
        em, em3 = statistics.mean(et), statistics.mean(e3)
        if ws > 1:
            tt = torch.tensor([em, em3], device=dev)
            torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
            em, em3 = float(tt[0].item()), float(tt[1].item())
        e2e = {"value": em / ws, "unit": "ms/snapshot", "h2d_bytes_per_step": hw.h2d_step,
               "d2h_bytes_per_step": hw.d2h_step, "entry": "rg_reion_step_host",
               "three_calls": {"value": em3 / ws, "h2d_bytes_per_step": hw.h2d, "d2h_bytes_per_step": hw.d2h,
                               "entry": "rg_compute_Ts_host, rg_find_HII_bubbles_host, rg_delta_T_host"}}
        del hw

    # roofline pass: per-kernel CUDA events inside the library
    nprof = max(2, min(args.steps, 3))
    ctx.profile(True)
    for _ in range(nprof):
        wk.reset()
        wk.step()
    stats = ctx.kernel_stats()
    ctx.profile(False)
    launches = sum(k["launches"] for k in stats) // nprof
    top = max(stats, key=lambda k: k["ms_total"])
    peak, peak_kind = measured_peak()
    ach = top["alg_bytes_total"] / (top["ms_total"] * 1e-3) / 1e9
    per_launch_bytes = top["alg_bytes_total"] / top["launches"]
    traffic = traffic_from_profiles(top["name"], cfg.name)
    total_ms = sum(k["ms_total"] for k in stats)
    live = 3 if cfg.spin_temp else 2       # filtered grids in fused mode: deltax, stars (+ x_e)
    step_bytes = alg_bytes(cfg, nr, live + (1 if args.mode == "plain" else 0))
    roofline = {"bound": "hbm", "kernel": top["name"], "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": ach / peak, "peak_kind": peak_kind, "traffic": traffic,
                "alg_bytes_per_launch": per_launch_bytes,
                "share_of_step": top["ms_total"] / total_ms if total_ms > 0 else None,
                "step_alg_bytes": step_bytes, "step_GBps": step_bytes / (ms_step * 1e-3) / 1e9,
                "step_frac": step_bytes / (ms_step * 1e-3) / 1e9 / peak,
                "kernels": {k["name"]: {"launches": k["launches"] // nprof, "ms": k["ms_total"] / nprof,
                                        "GBps": k["alg_bytes_total"] / max(k["ms_total"], 1e-9) / 1e6}
                            for k in stats}}

    # the same step in the plain mode (one FFT chain per grid per radius, the reference's pass
    # structure, every grid it filters): the baseline of the fused mode
    extras = {}
    if args.mode == "fused" and not args.no_extras:
        ctx.call("rg_set_mode", rg.RG_MODE_PLAIN)
        tp = timed(torch, stream, wk.step, wk.reset, 2, max(2, min(args.steps, 3)))
        ctx.call("rg_set_mode", rg.RG_MODE_FUSED)
        extras["plain_mode"] = {"ms_per_step": statistics.mean(tp),
                                "what": "the step with RG_MODE_PLAIN (unbatched radii, separate passes)"}
    # the 21-cm power spectrum of the step's delta_T (Compute_PS, run after the step by the
    # reference when Flag_ComputePS is set): not part of the metric, timed on its own
    if wk.spin and not args.no_extras:
        dptr = wk.b["delta_T"].data_ptr()
        ctx.power_spectrum(wk.p, dptr)
        torch.cuda.synchronize(dev)
        pst = []
        for _ in range(3):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ps_k, ps_d, _ = ctx.power_spectrum(wk.p, dptr)
            e1.record(stream)
            e1.synchronize()
            pst.append(e0.elapsed_time(e1))
        extras["power_spectrum"] = {"ms": statistics.mean(pst), "bins": int(len(ps_k)),
                                    "what": "Compute_PS of delta_T on the device, host outputs"}
        # delta_T with peculiar velocities and line-of-sight re-binning (flag 3) on a random
        # velocity grid; not part of the metric
        pv = rg.rg_params.from_buffer_copy(wk.p)
        pv.Flag_IncludePecVelsFor21cm = 3
        vel = torch.randn(wk.b["deltax"].numel(), device=dev) * 20.0
        gv = rg.rg_grids.from_buffer_copy(wk.g)
        gv.vel = vel.data_ptr()
        tbv = C.c_double()
        call = lambda: ctx.call("rg_delta_T", C.byref(pv), C.byref(wk.s), C.byref(gv), C.byref(tbv))
        call()
        torch.cuda.synchronize(dev)
        vt = []
        for _ in range(3):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            call()
            e1.record(stream)
            e1.synchronize()
            vt.append(e0.elapsed_time(e1))
        extras["delta_T_velocity_rsd"] = {"ms": statistics.mean(vt),
                                          "what": "rg_delta_T with Flag_IncludePecVelsFor21cm 3 (random velocities)"}
        del vel

    # find_HII_bubbles with inhomogeneous recombinations (stand-in MHR tables): the cost of the
    # recombination branch next to the same call without it; not part of the metric
    if not args.no_extras:
        extras["find_hii_recombinations"] = time_recombinations(wk, ctx, torch, stream, dev)
    # the tensor-core (split-BF16 tcgen05) form of a DFT pass against the FP32 form; not part of
    # the metric (the step uses the FP32 form)
    if not args.no_extras:
        extras["dft_y_pass_256"] = time_dft_y_pass(rg, torch, dev)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        w0 = time.perf_counter()
        cs = CpuSampler(cfg, src, ti, zz, snap)
        cs.fixed()
        for i in range(2):
            cs.sample(i)
        ms_cpu = cs.estimate()
        cpu = {"value": ms_cpu, "unit": "ms/snapshot", "cores": os.cpu_count(), "kind": "port",
               "sample": cs.desc + f"; two samples; oracle restatement, scipy pocketfft float32 on all host cores "
                                   f"({time.perf_counter() - w0:.1f} s wall)"}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "ms/snapshot", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": DATA_DESC,
                "config": workload_desc(cfg, nr), "mode": args.mode, "parallelism": f"replicas x{ws}",
                "e2e": e2e, "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu,
                "clocks": clk, "results": results, "extras": extras}
        print(json.dumps(line), flush=True)
    ctx.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


# ---------------------------------------------------------------------------
# the batched workload: 48 independent snapshots over boxes of uneven size

BATCH_METRIC = "snapshots/s find_HII_bubbles, 48 snapshots z=16->6 over 64^3/96^3/128^3/192^3 boxes"


def batch_params(rg, u):
    return rg.make_params(u.n, u.box, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMax=50.0,
                          ReionEfficiency=u.efficiency)


def run_batch(args):
    """Units are placed whole on ranks (no exchange).  On a rank, `plain` runs its units one
    after another on one stream, each call returning its scalars before the next starts;
    `batched` runs one host thread and one stream per box size, so the four sizes overlap on the
    GPU and no unit waits for another size's host round trip."""
    import threading
    import torch
    import autotune
    import rg_b200 as rg
    import sharding

    ws, rank, local = dist_env()
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    units = wl.batch_units()
    radii = {}
    for u in units:
        radii[u.index] = len(rg.radius_schedule(batch_params(rg, u), u.z))
    costs = [sharding.unit_cost(u.n, radii[u.index]) for u in units]
    mine = sharding.assign_units(costs, ws)[rank]
    sizes = sorted({units[i].n for i in mine})
    ctxs = {n: rg.Context(n, device=local) for n in sizes}
    streams = {n: torch.cuda.Stream(dev) for n in sizes}
    master = torch.cuda.current_stream(dev)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32).ravel()).to(dev)
    state = {}
    for i in mine:
        u = units[i]
        src = wl.make_sources(u.n, u.box, u.seed)
        b = {"deltax": t(src.deltax), "stars": t(src.stars), "weighted_sfr": t(src.sfr)}
        for k in ("xH", "r_bubble", "z_at_ionization", "J_21_at_ionization", "temp_kinetic_all_gas"):
            b[k] = torch.zeros(u.n ** 3, device=dev)
        g = rg.rg_grids()
        for k, v in b.items():
            setattr(g, k, v.data_ptr())
        zz, idx = wl.snapshot_redshifts(u.z)
        state[i] = dict(b=b, g=g, p=batch_params(rg, u), s=rg.snapshot(zz, idx), out=rg.rg_hii_scalars())
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def reset():
        for st in state.values():
            st["b"]["z_at_ionization"].fill_(-1.0)
            st["b"]["J_21_at_ionization"].zero_()
            st["b"]["temp_kinetic_all_gas"].zero_()
        flush.zero_()

    def run_unit(i):
        st = state[i]
        ctxs[units[i].n].call("rg_find_HII_bubbles", C.byref(st["p"]), C.byref(st["s"]), C.byref(st["g"]),
                              C.byref(st["out"]))

    def plain():
        for n in sizes:
            ctxs[n].call("rg_set_stream", C.c_void_p(master.cuda_stream))
        for i in mine:
            run_unit(i)

    def batched():
        ev0 = torch.cuda.Event()
        ev0.record(master)
        for n in sizes:
            streams[n].wait_event(ev0)
            ctxs[n].call("rg_set_stream", C.c_void_p(streams[n].cuda_stream))
        errs = []

        def worker(n):
            try:
                for i in mine:
                    if units[i].n == n:
                        run_unit(i)
            except Exception as e:      # surfaced after the join
                errs.append(e)
        ths = [threading.Thread(target=worker, args=(n,)) for n in sizes]
        for th in ths:
            th.start()
        for th in ths:
            th.join()
        if errs:
            raise errs[0]
        for n in sizes:
            ev = torch.cuda.Event()
            ev.record(streams[n])
            master.wait_event(ev)

    # the batch entry point: one rg_find_HII_bubbles_batch call per box size and group of
    # per_call snapshots, one host thread and stream per size; the radius batch and the group
    # size are tuned per size (autotune.py, cached per GPU model and workload shape)
    by_size = {n: [i for i in mine if units[i].n == n] for n in sizes}

    def reset_size(n):
        for i in by_size[n]:
            b = state[i]["b"]
            b["z_at_ionization"].fill_(-1.0)
            b["J_21_at_ionization"].zero_()
            b["temp_kinetic_all_gas"].zero_()

    def run_size(n, kb, per_call):
        ctx = ctxs[n]
        ctx.call("rg_set_radius_batch", kb)
        ids = by_size[n]
        for j in range(0, len(ids), per_call):
            grp = ids[j:j + per_call]
            outs = ctx.find_hii_batch([state[i]["p"] for i in grp], [state[i]["s"] for i in grp],
                                      [state[i]["g"] for i in grp])
            for i, o in zip(grp, outs):
                state[i]["out"] = o

    gpu = torch.cuda.get_device_name(dev)
    shape = {}
    for n in sizes:
        ctxs[n].call("rg_set_stream", C.c_void_p(master.cuda_stream))
        key = autotune.shape_key(gpu, n, 2, len(by_size[n]), radii[by_size[n][0]])
        shape[n] = autotune.tuned(key, lambda kb, pc, n=n: (reset_size(n), run_size(n, kb, pc)),
                                  lambda: torch.cuda.synchronize(dev), len(by_size[n]))

    def batch_api():
        ev0 = torch.cuda.Event()
        ev0.record(master)
        for n in sizes:
            streams[n].wait_event(ev0)
            ctxs[n].call("rg_set_stream", C.c_void_p(streams[n].cuda_stream))
        errs = []

        def worker(n):
            try:
                run_size(n, *shape[n])
            except Exception as e:      # surfaced after the join
                errs.append(e)
        ths = [threading.Thread(target=worker, args=(n,)) for n in sizes]
        for th in ths:
            th.start()
        for th in ths:
            th.join()
        if errs:
            raise errs[0]
        for n in sizes:
            ev = torch.cuda.Event()
            ev.record(streams[n])
            master.wait_event(ev)

    def timed_ms(fn):
        for _ in range(args.warmup):
            reset()
            fn()
        torch.cuda.synchronize(dev)
        out = []
        for _ in range(args.steps):
            reset()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(master)
            fn()
            e1.record(master)
            e1.synchronize()
            out.append(e0.elapsed_time(e1))
        return statistics.mean(out)

    if ws > 1:
        torch.distributed.barrier()
    ms_plain = sharding.max_over_ranks(timed_ms(plain))
    ms_threads = sharding.max_over_ranks(timed_ms(batched))
    clocks = ClockSampler(local)
    clocks.start()
    ms_batch = sharding.max_over_ranks(timed_ms(batch_api))
    clk = clocks.stop()
    xh = sharding.gather_scalars({i: [state[i]["out"].volume_weighted_global_xH] for i in mine}, len(units))
    # per-kernel timing of one pass through the batch entry point
    for c in ctxs.values():
        c.profile(True)
    reset()
    batch_api()
    torch.cuda.synchronize(dev)
    stats = {}
    for c in ctxs.values():
        for k in c.kernel_stats():
            a = stats.setdefault(k["name"], [0, 0.0, 0.0])
            a[0] += k["launches"]
            a[1] += k["ms_total"]
            a[2] += k["alg_bytes_total"]
        c.profile(False)
    top = max(stats.items(), key=lambda kv: kv[1][1])
    peak, peak_kind = measured_peak()
    ach = top[1][2] / (top[1][1] * 1e-3) / 1e9
    if rank == 0:
        value = len(units) / (ms_batch * 1e-3)
        line = {"metric": BATCH_METRIC, "value": value, "unit": "snapshots/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_batch, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators at the workload's shapes and sizes)",
                "config": {"workload": "48 independent find_HII_bubbles snapshots, z = 16 -> 6, boxes 64^3, 96^3, "
                                       "128^3, 192^3 (12 each, L = N Mpc/h), efficiency calibrated for <xH> 0.99 -> 0.1",
                           "name": "c2_batch", "parallelism": f"units placed whole on {ws} rank(s)",
                           "l2": "flushed (512 MiB write) before every timed step"},
                "what": "rg_find_HII_bubbles_batch: per box size, groups of snapshots in one call (shared "
                        "forward and x/y launches), one host thread and stream per size, launch shape tuned",
                "tuned": {str(n): {"radius_batch": shape[n][0], "per_call": shape[n][1]} for n in sizes},
                "plain": {"value": len(units) / (ms_plain * 1e-3), "ms_per_step": ms_plain,
                          "what": "rg_find_HII_bubbles per snapshot, one after another on one stream"},
                "per_snapshot_threads": {"value": len(units) / (ms_threads * 1e-3), "ms_per_step": ms_threads,
                                         "what": "rg_find_HII_bubbles per snapshot, one host thread and stream "
                                                 "per box size"},
                "gpu_launches": sum(v[0] for v in stats.values()),
                "roofline": {"bound": "hbm", "kernel": top[0], "achieved": ach, "peak": peak, "unit": "GB/s",
                             "frac": ach / peak, "peak_kind": peak_kind, "traffic": None},
                "clocks": clk, "results": {"mean_xH_first": xh[0][0], "mean_xH_last": xh[-1][0]}}
        print(json.dumps(line), flush=True)
    for c in ctxs.values():
        c.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


def main():
    args = parse()
    if args.only_extra == "dft_y_pass_256":
        import torch
        import rg_b200 as rg
        print(json.dumps({"extra": "dft_y_pass_256", **time_dft_y_pass(rg, torch, "cuda:0")}), flush=True)
        return
    if args.config == "c2_batch":
        if args.impl == "reference":
            ws, rank, _ = dist_env()
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the batched workload has no CPU arm here; "
                                  "the reference arm runs on the default workload"}), flush=True)
            return
        run_batch(args)
        return
    cfg = wl.CONFIGS[args.config]
    if args.impl == "reference":
        run_reference(args, cfg)
    else:
        run_ours(args, cfg)


if __name__ == "__main__":
    main()
