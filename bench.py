#!/usr/bin/env python3
"""Benchmark of the HARM3D step engine: zone-updates/s on B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

A step is one full RK2 step_ch() of the grid (predictor + corrector with
boundaries, fixups and the CFL reduction).  Rank 0 prints one JSON line.

Workloads (synthetic data of the configuration's shape; no dataset involved):
  torus192    (default) magnetised Fishbone-Moncrief torus around a Kerr
              black hole, a = 0.9, modified Kerr-Schild coordinates,
              192x192x128 zones (r from inside the horizon to 120 M, full
              2 pi in phi), r_in = 6 M, r_pmax = 12 M, Gamma = 5/3, one
              poloidal loop scaled to beta 100, seeded +-2% u perturbation,
              H/R = 0.1 cooling; PPM_MC + HLLE + para flux-CT, entropy fix,
              RESCALE_R, spherical outflow-3 boundaries; FP64.
  linwave256  3D periodic Minkowski linear wave, 256^3 zones, Gamma=4/3,
              rho=1, p=1, B=(1,1.5,0), plane-wave perturbation of amplitude
              1e-6 along the grid diagonal; PPM_MC + HLLE + para flux-CT, FP64.

Multi-GPU (torchrun): the path does not shard across GPUs in this engine
(one grid per GPU); every rank advances its own replica, time = max over
ranks, value = total zone-updates of all ranks / that time ("weak").

The reference arm (--impl reference) times the reference's own CPU build
(compiled on the host with gcc -O3 -march=native -fcommon from the sources
oracle/build_ref.py staged in oracle/_ref/<config>/src) on the host cores:
the workload's grid split into one block per core as the reference's MPI
runs split it (192x192x128 over 16 cores: 2x2x4 blocks of 96x96x32), every
block advanced by its own process for W untimed + K timed steps, without MPI
(no halo exchange, so an upper bound on the MPI build's rate), plus one
single-process step of the whole grid for the per-zone cost at full size.
"""
import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

PEAKS_FILE = os.path.join(HERE, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="torus192")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tune-steps", type=int, default=3,
                    help="steps per candidate of the launch-configuration autotuner (0: keep the defaults)")
    ap.add_argument("--mixed-steps", type=int, default=2000,
                    help="steps of the mixed-precision accuracy comparison (0: skip the mixed form)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp64_fma"],
                    help="form timed for `value`: fp64 (bit-identical to the reference) or fp64_fma "
                         "(fused multiply-adds)")
    ap.add_argument("--fma-steps", type=int, default=200,
                    help="steps of the FP64-with-FMA accuracy comparison beside the fp64 line (0: skip)")
    return ap.parse_args()


# the reference has no PN metric bodies: its arm for the binary-disk
# workloads runs the same setup on its dynamic path with the Minkowski test
# spacetime (geometry of the time levels and the connection rebuilt the same
# way, a cheaper metric function)
PN_REF_NOTE = "; the reference's Minkowski-spherical test spacetime in place of the PN metric it does not ship"

WORKLOADS = {
    "torus192": dict(kind="torus", n=(192, 192, 128), ref_cfg="torus",
                     label="Fishbone-Moncrief torus, Kerr-Schild a=0.9, MKS 192x192x128, r_in 6, r_pmax 12, "
                           "Gamma 5/3, beta 100 loop, H/R 0.1 cooling, PPM_MC+HLLE+para flux-CT, entropy fix, FP64"),
    "torus96": dict(kind="torus", n=(96, 96, 64), ref_cfg="torus",
                    label="Fishbone-Moncrief torus as torus192 on 96x96x64 zones"),
    "torus96dyn": dict(kind="torus_dyn", n=(96, 96, 64), ref_cfg="torus_dynmink",
                       label="torus192dyn on 96x96x64 zones"),
    "torus192dyn": dict(kind="torus_dyn", n=(192, 192, 128), ref_cfg="torus_dynmink",
                        label="torus192's initial state on the time-dependent metric path (metric_dim 3): the "
                              "Minkowski-spherical test spacetime, geometry of three time levels and the "
                              "finite-difference connection evaluated on the device every step, FP64"),
    "pnbbh300": dict(kind="pnbbh", n=(300, 160, 400), ref_cfg="pnbbh_dynmink", ref_note=PN_REF_NOTE, ref_nblocks=64,
                     label="circumbinary disk of an equal-mass black-hole binary (the post-Newtonian binary disk "
                           "setup: separation 20M, r 0.75a-13a, beta 10 loop, H/R 0.1 cooling, 1% seeded noise) in "
                           "the first post-Newtonian binary metric evaluated on the device every substep "
                           "(metric_dim 3: three time levels, finite-difference connection), COORD_DIAGONAL3 "
                           "300x160x400, PPM_MC+HLLE+para flux-CT, entropy fix, FP64"),
    "pnbbh150": dict(kind="pnbbh", n=(150, 80, 200), ref_cfg="pnbbh_dynmink", ref_note=PN_REF_NOTE,
                     label="pnbbh300 on 150x80x200 zones"),
    "pnbbh75": dict(kind="pnbbh", n=(75, 40, 100), ref_cfg="pnbbh_dynmink", ref_note=PN_REF_NOTE,
                    label="pnbbh300 on 75x40x100 zones (profiling size)"),
    "balsara1024": dict(kind="setup", setup="balsara1", n=(1024, 1, 1), ref_cfg="balsara1",
                        label="Balsara-1 shock tube, 1024 zones, MC + HLLE + para flux-CT, CFL 0.5, FP64"),
    "fieldloop512": dict(kind="setup", setup="field_loop", n=(512, 512, 1), ref_cfg="field_loop",
                         label="advected field loop 512^2, PPM_MC + HLLE + para flux-CT, FP64"),
    "linwave256": dict(kind="linwave", n=(256, 256, 256), gam=4.0 / 3.0, cour=0.4, recon=5, flux=1, bc=1, ref_cfg="linwave",
                       label="3D periodic Minkowski linear wave 256^3, PPM_MC+HLLE+para flux-CT, FP64"),
    "linwave128": dict(kind="linwave", n=(128, 128, 128), gam=4.0 / 3.0, cour=0.4, recon=5, flux=1, bc=1, ref_cfg="linwave",
                       label="3D periodic Minkowski linear wave 128^3, PPM_MC+HLLE+para flux-CT, FP64"),
}


def linwave_state(n, gam):
    """rho=1, p=1, B=(1,1.5,0) plus a diagonal plane wave of amplitude 1e-6."""
    import coolharm3d_b200 as hg
    shape = hg.ref_shape(n)
    dx = [1.0 / x for x in n]
    x = -3 * dx[0] + (np.arange(shape[0]) + 0.5) * dx[0]
    y = -3 * dx[1] + (np.arange(shape[1]) + 0.5) * dx[1]
    z = -3 * dx[2] + (np.arange(shape[2]) + 0.5) * dx[2]
    ph = np.cos(2 * np.pi * (x[:, None, None] + y[None, :, None] + z[None, None, :]))
    amp = 1e-6
    p = np.empty(shape + (8,))
    p[..., 0] = 1 + amp * ph
    p[..., 1] = 1.0 / (gam - 1.0) + amp * 3.0 * ph
    p[..., 2] = amp * 0.5 * ph
    p[..., 3] = amp * 0.5 * ph
    p[..., 4] = amp * -0.2 * ph
    p[..., 5] = 1.0 + amp * 0.3 * ph
    p[..., 6] = 1.5 - amp * 0.2 * ph
    p[..., 7] = amp * 0.7 * ph
    return p


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def peak_hbm():
    try:
        with open(PEAKS_FILE) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def algorithmic_bytes(kind, n):
    """Algorithmic HBM bytes of one launch of a kernel class (FP64 state).

    flux (one direction): every zone of the stencil box read once (8 prims)
    plus the 8 flux components written once per face.  update: p, p_h read,
    five non-induction flux components of the three face families, three
    EMFs and two floors read once per zone; p_f (8), p_gamma and pflag
    written once per zone."""
    N0, N1, N2 = n
    T = [x + 6 for x in n]
    if kind == "flux":
        faces = (N0 + 1) * T[1] * T[2]
        return 64.0 * T[0] * T[1] * T[2] + 64.0 * faces
    if kind == "update":
        return (64 + 64 + 3 * 40 + 24 + 16 + 64 + 8 + 4) * float(N0 * N1 * N2)
    if kind == "emf":
        return (6 * 8 + 3 * 8) * float((N0 + 1) * (N1 + 1) * (N2 + 1))
    return None


def setup(wl, device, precision=0, p_init=None):
    """Engine holding the workload's initial state, and that state on the host.
    precision 1 builds the mixed-precision engine; p_init, if given, is
    uploaded instead of a freshly built initial state."""
    import coolharm3d_b200 as hg
    n = wl["n"]
    if wl["kind"] == "torus_dyn":
        from coolharm3d_b200 import torus
        ks, p0 = setup(dict(wl, kind="torus"), device, precision, p_init)
        ks.close()
        desc = torus.torus_desc(n, device=device, precision=precision)
        t = torus.torus_tables(desc)
        desc.metric_dim = 3
        e = hg.Engine(desc)
        e.set_dynamic_metric(hg.dyn_metric())
        e.set_cell_data(t["cell6"], t["rface"])
        e.set_cooling_tables(t["cool_omega"], t["cool_temp"])
        e.upload(p0)
        e.set_time(desc.t, desc.dx[0])
        return e, p0
    if wl["kind"] == "pnbbh":
        from coolharm3d_b200 import pnbbh
        desc = pnbbh.pnbbh_desc(n, device=device, precision=precision)
        t = pnbbh.pnbbh_tables(desc)
        m = pnbbh.pnbbh_coords(spacetime=hg.DYN_PN_BINARY)
        e = hg.Engine(desc)
        e.set_dynamic_metric(m)
        e.set_cell_data(t["cell6"], t["rface"])
        e.set_cooling_tables(*pnbbh.pn_cooling_tables(t))
        if p_init is None:
            p0, _ = pnbbh.set_disk(e, desc, t, m)
        else:
            p0 = p_init
            e.upload(p0)
        e.set_time(0.0, desc.dx[0])
        return e, p0
    if wl["kind"] == "torus":
        from coolharm3d_b200 import torus
        desc = torus.torus_desc(n, device=device, precision=precision)
        t = torus.torus_tables(desc)
        e = hg.Engine(desc)
        e.set_geometry(t["geom"], t["conn"])
        e.set_cell_data(t["cell6"], t["rface"])
        e.set_cooling_tables(t["cool_omega"], t["cool_temp"])
        if p_init is None:
            p0 = torus.set_torus(e, desc, t, seed=2024)
        else:
            p0 = p_init
            e.upload(p0)
        e.set_time(desc.t, desc.dx[0])
        return e, p0
    if wl["kind"] == "setup":
        from coolharm3d_b200 import setups
        prob = setups.balsara1(n[0], precision=precision, device=device) if wl["setup"] == "balsara1" else \
            setups.field_loop(n, precision=precision, device=device)
        prob.desc.grid_length[0] = 1e9  # time the step, not the approach to t_final
        e = hg.Engine(prob.desc)
        if p_init is None:
            setups.start(e, prob)
            p0 = e.download()
        else:
            p0 = p_init
            e.set_geometry(prob.geom)
            e.set_cell_data(prob.cell6)
            e.upload(p0)
            e.set_time(0.0, prob.desc.dx[0])
        return e, p0
    dx = [1e-5] + [1.0 / x for x in n]
    startx = [0.0] + [-3 * d for d in dx[1:]]
    desc = hg.make_desc(n, wl["gam"], wl["cour"], dx, startx, [1e9, 1, 1, 1], recon=wl["recon"], flux=wl["flux"],
                        bc=wl["bc"], device=device, precision=precision)
    geom, cell6 = hg.minkowski_tables(desc)
    p0 = linwave_state(n, wl["gam"]) if p_init is None else p_init
    e = hg.Engine(desc)
    e.set_geometry(geom)
    e.set_cell_data(cell6)
    e.upload(p0)
    return e, p0


def max_over_ranks(values, world):
    """Element-wise maximum of `values` over all ranks (the slowest rank sets
    every time): one all_reduce on the process group's device (the GPU under
    NCCL, the host under gloo)."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    tt = torch.tensor([float(v) for v in values], dtype=torch.float64, device=dev)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return [float(v) for v in tt.tolist()]


def whole_job_rates(world, zones, steps, ms_max, e2e_s_max):
    """Zone-updates/s of the whole job: every rank advances its own replica
    of `zones` zones by `steps` steps, timed by the slowest rank (device
    milliseconds, end-to-end seconds)."""
    return world * zones * steps / (ms_max * 1e-3), world * zones * steps / e2e_s_max


PRECISIONS = {"fp64": 0, "fp64_fma": 2}


def run_ours(args, wl, rank, world, device):
    import coolharm3d_b200 as hg
    n = wl["n"]
    e, p0 = setup(wl, device, precision=PRECISIONS[args.precision])
    # launch configuration measured on this grid's own state (restored after)
    if args.tune_steps > 0:
        tuned, tune_before, tune_after = e.autotune(steps=args.tune_steps)
    else:
        tuned, tune_before, tune_after = e.launch_config(), None, None
    zones = n[0] * n[1] * n[2]
    barrier, sync = lambda: None, lambda: None
    try:
        import torch
        if torch.cuda.is_available():
            sync = torch.cuda.synchronize
        if world > 1:
            import torch.distributed as dist
            barrier = dist.barrier
    except ImportError:
        pass
    e.step(args.warmup)
    # timed region: K steps on the device, state resident, each step one
    # CUDA-graph launch (no per-kernel events)
    fails0 = e.fail_counts().astype(np.int64)
    clk = ClockSampler(device)
    clk.start()
    barrier()
    sync()
    e.step(args.steps)
    sync()
    barrier()
    clocks = clk.stop()
    ms = e.last_step_ms()
    # failure counters (nfailtot) of the timed steps, per step: how many
    # zones the inversion's fallback tree and the entropy fix took
    dfail = e.fail_counts().astype(np.int64) - fails0
    nfail_per_step = {nm: float(dfail[i]) / args.steps for i, nm in enumerate(hg.NFAIL_NAMES) if dfail[i]}
    # kernel classes: the same K steps again with an event before every kernel
    e.profile(True)
    e.step(args.steps)
    kt = e.kernel_times()
    e.profile(False)
    # end to end through the C ABI with host buffers: upload from host, K x
    # (hg_step + t/dt + nfailtot readback, what step_ch()'s caller needs every
    # step), download to host -- all inside the timed region
    # (the host buffers are page-locked, allocated before the timed region,
    # so both transfers are single DMAs of the caller's memory)
    host_p = hg.pinned_array(p0.shape)
    host_p[...] = p0
    back = hg.pinned_array(p0.shape)
    t0 = time.perf_counter()
    e.upload(host_p)
    e.set_time(e.desc.t, e.desc.dx[0])
    for _ in range(args.steps):
        e.step(1)
        e.fail_counts()
    e.download(out=back)
    e2e_s = time.perf_counter() - t0
    del back, host_p
    ms_max, e2e_max = max_over_ranks([ms, e2e_s], world)
    value, e2e_val = whole_job_rates(world, zones, args.steps, ms_max, e2e_max)
    state_bytes = 8 * 8 * np.prod(hg.ref_shape(n))
    out = dict(metric="zone-updates/s", value=value, unit="zone-updates/s", n_gpus=world, steps=args.steps,
               warmup=args.warmup, ms_per_step=ms_max / args.steps, higher_is_better=True, scaling="weak",
               vs_baseline=None, dtype="f64", data="synthetic",
               config={"workload": args.workload, "description": wl["label"], "grid": list(n),
                       "zones": zones, "parallelism": "replicas" if world > 1 else "single",
                       "precision": args.precision,
                       "l2": "inputs larger than L2 (state arrays of %.2f GB each)" % (
                           8 * 8 * np.prod(hg.ref_shape(n)) / 1e9),
                       "e2e": "upload from pinned host memory once + K x (hg_step(1) + nfailtot readback) + download to pinned host memory once",
                       "launch": dict(tuned.as_dict(), autotune_ms_per_step=[tune_before, tune_after])})
    # roofline of the dominant kernel class (live CUDA events on the engine stream)
    dom = max(("flux", "update", "emf"), key=lambda c: kt[c][0])
    avg_ms = kt[dom][0] / max(kt[dom][1], 1)
    alg = algorithmic_bytes(dom, n)
    peak, src = peak_hbm()
    ach = alg / (avg_ms * 1e-3) / 1e9
    traffic, fp64 = None, None
    tf = os.path.join(HERE, "profiles", "traffic.json")
    if os.path.exists(tf):
        try:
            rec = json.load(open(tf)).get(args.workload, {})
            traffic = rec.get(dom)
            fp64 = rec.get("fp64_pipe_active", {}).get(dom)
        except (OSError, ValueError):
            traffic = None
    out["roofline"] = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "peak_source": src,
                       "unit": "GB/s", "frac": ach / peak, "traffic": traffic,
                       "avg_launch_ms": avg_ms, "algorithmic_bytes_per_launch": alg,
                       "kernel_share": {c: kt[c][0] / max(sum(v[0] for v in kt.values()), 1e-30) for c in kt},
                       "fp64_pipe_active_ncu": fp64,
                       "note": "the step is FP64-issue bound; fp64_pipe_active_ncu is the FP64 pipe's active "
                               "fraction for this kernel from the committed ncu capture"}
    # FP64 roofline: FP64 operations per zone-update counted by ncu (fma = 2)
    # times the measured rate, over the FP64 peak measured now on this GPU
    ops = fp64_ops(args.workload)
    if ops is not None:
        peak64, _ = hg.fp64_peak(device)
        step_tf = ops["step"] * value / world / 1e12
        fl = ops["per_launch"].get(dom)
        blk = {"bound": "fp64", "unit": "TFLOP/s", "peak": peak64, "peak_source": "measured now (hg_fp64_peak)",
               "step": {"achieved": step_tf, "frac": step_tf / peak64,
                        "fp64_ops_per_zone_update": ops["step"]}, "source": ops["source"]}
        if fl is not None:
            k_tf = fl * ops["scale"] / (avg_ms * 1e-3) / 1e12
            blk["kernel"] = {"name": dom, "achieved": k_tf, "frac": k_tf / peak64,
                             "fp64_ops_per_launch": fl * ops["scale"]}
        out["roofline"]["fp64"] = blk
    out["e2e"] = {"value": e2e_val, "unit": "zone-updates/s",
                  "h2d_bytes_per_step": float(state_bytes) / args.steps,
                  "d2h_bytes_per_step": float(state_bytes) / args.steps + 16 + 120}
    total_launches = sum(v[1] for v in kt.values()) + 2 * args.steps  # k_begin launches are in "misc"
    out["gpu_launches"] = int(sum(v[1] for v in kt.values()))
    out["nfail_per_step"] = nfail_per_step
    if clocks:
        out["clocks"] = clocks
    if rank == 0 and args.mixed_steps > 0 and args.precision == "fp64":
        out["mixed"] = mixed_form(args, wl, device, e, p0, ms / args.steps)
    if rank == 0 and args.fma_steps > 0 and args.precision == "fp64":
        if e.h is None:  # released by the sequential mixed comparison (the grid fills the device)
            out["fp64_fma"] = {"skipped": "the FP64 engine was released to make room for the mixed one"}
        else:
            out["fp64_fma"] = fma_form(args, wl, device, e, p0, ms / args.steps)
    e.close()
    return out


def fp64_ops(workload):
    """FP64 operations (fma counted twice) per zone-update of the whole step
    and per launch of each kernel class, from the committed ncu count
    (profiles/fp64_ops.json); a count taken on a smaller grid of the same
    problem is scaled to this one by its zones per launch."""
    try:
        rec = json.load(open(os.path.join(HERE, "profiles", "fp64_ops.json")))
    except (OSError, ValueError):
        return None
    for name, r in rec.get("workloads", {}).items():
        if workload in r.get("applies_to", [name]):
            zones = float(np.prod(WORKLOADS[workload]["n"]))
            return {"step": r["per_zone_update"], "per_launch": r["per_launch"],
                    "scale": zones / float(np.prod(r["grid"])), "source": r["command"]}
    return None


VARS = ["rho", "u", "U1", "U2", "U3", "B1", "B2", "B3"]


def l1_rel(a, b):
    """Per variable: sum |a - b| / sum |b| over the physical zones."""
    a, b = a[3:-3, 3:-3, 3:-3], b[3:-3, 3:-3, 3:-3]
    return {nm: float(np.abs(a[..., l] - b[..., l]).sum() / max(np.abs(b[..., l]).sum(), 1e-300))
            for l, nm in enumerate(VARS)}


def mixed_form(args, wl, device, e64, p0, fp64_ms):
    """The mixed-precision form on the same workload: its device time per
    step, and after args.mixed_steps steps (and at a tenth of that) the
    per-variable relative L1 difference from the FP64 run, beside the
    difference a one-ulp change of u in the initial state makes to the FP64
    run itself (how far the flow amplifies rounding) and the difference the
    FP64 run shows when its initial state is rounded once to FP32."""
    import copy
    import coolharm3d_b200 as hg
    K = args.mixed_steps
    k1 = max(1, K // 10)
    pert = p0.copy()
    pert[..., 1] = np.nextafter(pert[..., 1], np.inf)
    # the state rounded once to FP32: what a single FP32 rounding of every
    # primitive (the floor of any form that reads FP32 states) grows into
    r32 = p0.astype(np.float32).astype(np.float64)
    snaps = {}

    def run(name, eng, start):
        eng.upload(start)
        eng.set_time(eng.desc.t, eng.desc.dx[0])
        eng.step(k1)
        a = eng.download()
        eng.step(K - k1)
        snaps[name] = (a, eng.download())

    # a grid too large for both engines at once (the 300x160x400 binary disk):
    # the FP64 runs first, then the FP64 engine makes room for the mixed one
    dm = copy.copy(e64.desc)
    dm.precision = 1
    sequential = hg.grid_bytes(dm) + (2 << 30) > hg.mem_info(device)[0]
    if sequential:
        for name, start in (("fp64", p0), ("fp64_ulp", pert), ("fp64_r32", r32)):
            run(name, e64, start)
        e64.close()
    em, _ = setup(wl, device, precision=1, p_init=p0)
    if args.tune_steps > 0:
        em.autotune(steps=args.tune_steps)
    # the FP64 form's protocol: from the initial state, W warm-up steps, then
    # K steps timed (the same states, so the same fallback and fixup work)
    em.upload(p0)
    em.set_time(em.desc.t, em.desc.dx[0])
    em.step(args.warmup)
    em.step(args.steps)
    mixed_ms = em.last_step_ms() / args.steps
    em.profile(True)
    em.step(args.steps)
    kt = em.kernel_times()
    em.profile(False)
    run("mixed", em, p0)
    if not sequential:
        for name, start in (("fp64", p0), ("fp64_ulp", pert), ("fp64_r32", r32)):
            run(name, e64, start)
    em.close()
    zones = float(np.prod(wl["n"]))
    res = {"value": zones / (mixed_ms * 1e-3), "unit": "zone-updates/s", "ms_per_step": mixed_ms,
           "speedup_vs_fp64": fp64_ms / mixed_ms, "dtype": "f32 reconstruction+flux, f64 elsewhere",
           "sequential": sequential,
           "kernel_ms_per_step": {c: v[0] / args.steps for c, v in kt.items() if v[1]}, "accuracy": {}}
    for idx, steps in ((0, k1), (1, K)):
        res["accuracy"]["steps_%d" % steps] = {
            "l1_rel_mixed_vs_fp64": l1_rel(snaps["mixed"][idx], snaps["fp64"][idx]),
            "l1_rel_fp64_one_ulp": l1_rel(snaps["fp64_ulp"][idx], snaps["fp64"][idx]),
            "l1_rel_fp64_from_fp32_rounded_state": l1_rel(snaps["fp64_r32"][idx], snaps["fp64"][idx])}
    return res


def fma_form(args, wl, device, e64, p0, fp64_ms):
    """The FP64 form with fused multiply-adds on the same workload: its device
    time per step, and after args.fma_steps steps the per-variable relative L1
    difference from the plain FP64 run (beside the difference a one-ulp
    change of u in the initial state makes to the plain run itself)."""
    ef, _ = setup(wl, device, precision=2, p_init=p0)
    if args.tune_steps > 0:
        ef.autotune(steps=args.tune_steps)
    ef.upload(p0)  # the FP64 form's protocol: W warm-up steps from p0, K timed
    ef.set_time(ef.desc.t, ef.desc.dx[0])
    ef.step(args.warmup)
    ef.step(args.steps)
    fma_ms = ef.last_step_ms() / args.steps
    K = args.fma_steps
    pert = p0.copy()
    pert[..., 1] = np.nextafter(pert[..., 1], np.inf)
    snaps = {}
    for name, eng, start in (("fp64", e64, p0), ("fma", ef, p0), ("fp64_ulp", e64, pert)):
        eng.upload(start)
        eng.set_time(eng.desc.t, eng.desc.dx[0])
        eng.step(1)
        one = eng.download()
        eng.step(K - 1)
        snaps[name] = (one, eng.download(), eng.fail_counts().tolist())
    ef.close()
    zones = float(np.prod(wl["n"]))
    a, b = snaps["fma"][0][3:-3, 3:-3, 3:-3], snaps["fp64"][0][3:-3, 3:-3, 3:-3]
    scale = np.abs(b).reshape(-1, 8).max(0)
    normwise = np.abs(a - b).reshape(-1, 8).max(0) / np.where(scale > 0, scale, 1.0)
    return {"value": zones / (fma_ms * 1e-3), "unit": "zone-updates/s", "ms_per_step": fma_ms,
            "speedup_vs_fp64": fp64_ms / fma_ms, "dtype": "f64 (fused multiply-adds)",
            "one_step_normwise_rel_vs_fp64": dict(zip(VARS, normwise.tolist())),
            "steps_%d" % K: {"l1_rel_fma_vs_fp64": l1_rel(snaps["fma"][1], snaps["fp64"][1]),
                             "l1_rel_fp64_one_ulp": l1_rel(snaps["fp64_ulp"][1], snaps["fp64"][1]),
                             "nfailtot_fma": snaps["fma"][2], "nfailtot_fp64": snaps["fp64"][2]}}


def reference_exe(cfg, native=True):
    """The reference's own CPU build of `cfg`: built on this machine with
    -O3 -march=native -fcommon from the staged sources (oracle/build_ref.py
    build_native), else the portable build that travels with the repository.
    Returns (path, how) or (None, why)."""
    if native:
        try:
            sys.path.insert(0, os.path.join(HERE, "oracle"))
            import build_ref
            return build_ref.build_native(cfg), "gcc -O3 -march=native -fcommon (built on this host)"
        except Exception as ex:  # the portable build still measures the reference
            why = str(ex)
        finally:
            sys.path.pop(0)
    exe = os.path.join(HERE, "oracle", "_ref", cfg, "harm3d")
    if os.path.exists(exe):
        return exe, "gcc -O3 -fcommon -ffp-contract=off (portable build)"
    return None, "reference build %s absent (run oracle/build_ref.py where the reference sources are)" % exe


def decompose(n, procs):
    """Block decomposition of grid n over at most `procs` processes, as the
    reference's MPI runs split it (harm_mpi.c: a x b x c ranks, each block
    n/a x n/b x n/c): the largest process count whose factors divide n, and
    among those the split with the least block surface.  Directions with one
    zone are not split.  Returns (counts, block)."""
    best = None
    for p in range(procs, 0, -1):
        for a in range(1, p + 1):
            if p % a or n[0] % a:
                continue
            for b in range(1, p // a + 1):
                if (p // a) % b or n[1] % b:
                    continue
                c = p // a // b
                if n[2] % c:
                    continue
                blk = (n[0] // a, n[1] // b, n[2] // c)
                if any(x == 1 and m > 1 for x, m in zip(blk, n)) and p > 1:
                    continue
                surf = sum(blk[x] * blk[y] for x, y in ((0, 1), (0, 2), (1, 2)))
                if best is None or surf < best[0]:
                    best = (surf, (a, b, c), blk)
        if best is not None:
            return best[1], best[2]
    return (1, 1, 1), tuple(n)


def run_reference_blocks(exe, block, procs, warmup, steps):
    """`procs` concurrent processes of the reference build, each advancing a
    `block` grid by warmup + steps steps; only the last `steps` are timed
    (the probe's own clock around step_ch()).  Returns (zone-updates/s of the
    whole ensemble, seconds of the slowest process for the timed steps) or
    (None, why)."""
    env = dict(os.environ, HARM_PROBE_MAXSTEPS=str(warmup + steps), HARM_PROBE_TIME="1",
               HARM_PROBE_TIME_SKIP=str(warmup))
    tds, ps = [], []
    for _ in range(procs):
        td = tempfile.mkdtemp()
        tds.append(td)
        ps.append(subprocess.Popen([exe, "1", "1", "1"] + [str(x) for x in block], cwd=td, env=env,
                                   stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True))
    secs, cells = [], None
    for p in ps:
        outp, _ = p.communicate(timeout=1800)
        m = re.search(r"probe_time steps=(\d+) seconds=([0-9.eE+-]+) cells=(\d+)", outp)
        if not m or int(m.group(1)) != steps:
            return None, "reference run produced no timing line for %d steps" % steps
        secs.append(float(m.group(2)))
        cells = int(m.group(3))
    slowest = max(secs)
    return procs * steps * cells / slowest, slowest


def reference_arm(wl, ncores, warmup, steps, full_grid=False):
    """The reference's CPU build on this host's cores, on the workload's own
    grid: split into one block per core (decompose), every block advanced by
    its own process (no halo exchange: an upper bound on the MPI build's
    rate, MPI being absent from the image).  1D/2D grids run one whole-grid
    replica per core instead.  full_grid adds one single-process step of the
    whole grid (after one warm-up step)."""
    exe, how = reference_exe(wl["ref_cfg"])
    if exe is None:
        return None, how
    n = wl["n"]
    procs = max(1, min(ncores, 64))
    if min(n) > 1 and wl.get("ref_nblocks"):
        # a bounded sample: the grid split into ref_nblocks equal blocks (the
        # reference's dynamic path holds ~6 KB per zone, too much for one
        # block per core of the whole grid in host memory), procs of them
        counts, block = decompose(n, wl["ref_nblocks"])
        layout = "%d of the %dx%dx%d blocks of %s" % ((procs,) + counts + ("x".join(map(str, block)),))
    elif min(n) > 1:
        counts, block = decompose(n, procs)
        procs = counts[0] * counts[1] * counts[2]
        layout = "%dx%dx%d blocks of %s" % (counts + ("x".join(map(str, block)),))
    else:
        block, layout = tuple(n), "%d replicas of the whole grid" % procs
    value, slowest = run_reference_blocks(exe, block, procs, warmup, steps)
    if value is None:
        return None, slowest
    zones_step = procs * int(np.prod(block))
    res = {"value": value, "ms_per_step": 1e3 * slowest / steps, "procs": procs, "block": list(block),
           "build": how, "cpu": _cpu_model(),
           "sample": "%s of the %s grid, one process per core, %d untimed + %d timed steps each "
                     "(reference CPU build, no MPI halo exchange); %d zones per step%s" % (
                         layout, "x".join(map(str, n)), warmup, steps, zones_step, wl.get("ref_note", ""))}
    if full_grid and min(n) > 1:
        v1, s1 = run_reference_blocks(exe, tuple(n), 1, 1, 1)
        if v1 is not None:
            res["single_process_full_grid"] = {"value": v1, "ms_per_step": 1e3 * s1, "steps": 1, "warmup": 1}
    return res, None


def _cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    wl = WORKLOADS[args.workload]
    ncores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    if args.impl == "reference":
        if rank != 0:
            return 0
        res, err = reference_arm(wl, ncores, max(1, args.warmup), args.steps, full_grid=True)
        if res is None:
            print(json.dumps({"impl": "reference", "unavailable": err}))
            return 0
        value = res["value"]
        out = dict(impl="reference", metric="zone-updates/s", value=value, unit="zone-updates/s", n_gpus=world,
                   steps=args.steps, warmup=max(1, args.warmup), ms_per_step=res["ms_per_step"],
                   higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f64", data="synthetic",
                   config={"workload": args.workload, "description": wl["label"], "grid": list(wl["n"]),
                           "reference": {k: v for k, v in res.items() if k not in ("value", "ms_per_step")}},
                   cpu_baseline={"value": value, "unit": "zone-updates/s", "cores": res["procs"],
                                 "kind": "reference", "sample": res["sample"]},
                   e2e={"value": value, "unit": "zone-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
        print(json.dumps(out))
        return 0
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    out = run_ours(args, wl, rank, world, local)
    if rank == 0 and not args.no_cpu_baseline:
        # a bounded sample of the same measurement: 1 untimed + 2 timed steps
        res, err = reference_arm(wl, ncores, 1, 2)
        if res is not None:
            out["cpu_baseline"] = {"value": res["value"], "unit": "zone-updates/s", "cores": res["procs"],
                                   "kind": "reference", "sample": res["sample"], "build": res["build"],
                                   "cpu": res["cpu"], "ms_per_step": res["ms_per_step"]}
        else:
            out["cpu_baseline"] = {"value": None, "unit": "zone-updates/s", "cores": 0, "kind": "reference",
                                   "sample": err}
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
