#!/usr/bin/env python
"""Benchmark of the MCV_SW explicit RK step on B200.

`python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]`

One step = one RK step (all stages + halo corrections) of the workload on every
GPU.  Default workload: MCV4, Nc=256, RK3_TVD, seeded balanced tilted zonal flow
+ spherical-harmonic height perturbation (degree <= 32, RMS 20 m) + a 2000 m
Gaussian mountain (the single-large-instance configuration).  The state stays
resident in HBM; `value` is simulated days per wall second over all GPUs
(replicas: every rank advances its own instance).  Each stage reads ~9 padded
FP64 fields (~260 MB) -- more than the 126 MB L2 -- so no L2 flush is needed.

`--impl reference` times the reference algorithm's CPU implementation (the
FP64 C restatement under oracle/, all host threads) on the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "sim-days/s MCV4 Nc=256 mixed vs FP64 on 1 B200 at stated L2 error; p99 latency"
UNIT = "sim-days/s"
DEFAULT_HBM_GBS = 6650.0


def strict_json(x):
    """x with every non-finite float replaced by None: the output line stays
    strict JSON (a forecast that blew up reports null, not NaN)."""
    if isinstance(x, float):
        return x if np.isfinite(x) else None
    if isinstance(x, dict):
        return {k: strict_json(v) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [strict_json(v) for v in x]
    return x


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=2000)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", choices=["large", "small", "stress"], default="large")
    p.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    p.add_argument("--error-days", type=float, default=5.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--e2e-steps", type=int, default=20)
    p.add_argument("--ensemble", type=int, default=1, help="run the 64-member ensemble block (1 GPU only)")
    p.add_argument("--serve-requests", type=int, default=200,
                   help="requests of the serving stream served by the native request loop (0: skip the block)")
    p.add_argument("--serve-python-requests", type=int, default=24,
                   help="first requests of the stream also served by the Python request loop")
    p.add_argument("--serve-baseline-requests", type=int, default=24,
                   help="first requests of the stream also run by the FP64 one-request-at-a-time loop")
    p.add_argument("--stress", type=int, default=1, help="run the Nc=1024 roofline-stress block (1 GPU only)")
    p.add_argument("--admission", type=int, default=1, help="run the device-admission timing block (1 GPU only)")
    p.add_argument("--paths", default="fp64,mixed",
                   help="precisions timed on the main workload (the headline precision must be one of them)")
    p.add_argument("--tiles", default=None,
                   help="pin the stage-kernel candidates of the main workload as 'fp64_index,mixed_index' "
                        "(default: each handle's autotuner chooses)")
    return p.parse_args()


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(x, dist, device="cuda"):
    """The largest x over the ranks: the job's time is its slowest rank's."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(world, steps, dt, ms):
    """Whole-job simulated days per second: each of `world` ranks advances its
    own replica by `steps` steps of dt seconds within the job's ms."""
    return world * steps * dt / 86400.0 / (ms / 1e3)


def build_workload(name):
    from mcv_sw_b200 import cases
    if name == "large":
        st, geom = cases.large(seed=2)
        desc = "MCV4 Nc=256 RK3_TVD, seeded balanced tilted zonal flow + harmonics (deg<=32, RMS 20 m) + 2000 m mountain"
    elif name == "small":
        st, geom = cases.small(seed=1)
        desc = "MCV3 Nc=32 RK4, seeded balanced tilted zonal flow + harmonics (deg 1-8, RMS 10 m)"
    else:
        st, geom = cases.stress(seed=5)
        desc = "MCV4 Nc=1024 RK4, balanced zonal flow + Rossby-Haurwitz waves R=4..12 (50-200 m)"
    return st, geom, desc


def stage_bytes(scheme, precision):
    """Algorithmic bytes per interior PV of each stage-kernel launch.

    FP64: 8-byte words of stage input (3), RK base where the stage reads it (3),
    6 metric scalars, stage output (3), RK4 accumulator read/write (3 each):
    RK3 12, 15, 15 words; RK4 15, 21, 21, 18.
    Split precision: FP64 state (24 B), FP32 input increment (12), FP32 phi_s
    (4; the metric is recomputed from 1-D tables), FP32 output increment (12) or
    FP64 new state (24), FP32 RK4 accumulator read/write (12 each)."""
    if precision == "fp64":
        words = [12, 15, 15] if scheme == "RK3_TVD" else [15, 21, 21, 18]
        return [8 * w for w in words]
    if scheme == "RK3_TVD":
        return [24 + 4 + 12, 24 + 12 + 4 + 12, 24 + 12 + 4 + 24]
    return [24 + 4 + 12 + 12, 24 + 12 + 4 + 12 + 24, 24 + 12 + 4 + 12 + 24, 24 + 12 + 4 + 12 + 24]


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device)], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return DEFAULT_HBM_GBS, "fallback"


def stage_traffic_per_pv():
    """DRAM bytes per interior PV per stage-kernel launch from the committed ncu
    summary (profiles/stage_kernel_traffic.txt: `<workload> <kind> <bytes_per_pv>`)."""
    path = os.path.join(ROOT, "profiles", "stage_kernel_traffic.txt")
    out = {}
    if os.path.exists(path):
        for line in open(path):
            parts = line.split()
            if len(parts) == 3 and not line.startswith("#"):
                out[(parts[0], parts[1])] = float(parts[2])
    return out


def cpu_baseline(st, budget_s=20.0):
    """The oracle (FP64 C restatement, all host threads) on a bounded sample of
    the same workload: as many RK steps as fit in ~budget_s."""
    from oracle import oracle as orc
    o = orc.Oracle(st.order, st.nc, st.dt, st.scheme, 6.371e6)
    o.set_phi_s(st.phi_s)
    o.init_state(st.zonal, st.merid, st.phi)
    t0 = time.perf_counter()
    o.step(1)
    t1 = time.perf_counter() - t0
    nsteps = max(1, min(200, int(budget_s / max(t1, 1e-6))))
    t0 = time.perf_counter()
    o.step(nsteps)
    el = time.perf_counter() - t0
    return {"value": nsteps * st.dt / 86400.0 / el, "unit": UNIT, "cores": orc.num_threads(), "kind": "port",
            "sample": f"{nsteps} RK steps of the same workload after 1 warm-up step ({el:.1f} s)"}


def mapped_libraries():
    """Shared objects mapped into this process (from /proc/self/maps)."""
    try:
        with open("/proc/self/maps") as f:
            return sorted({line.split()[-1] for line in f if line.rstrip().endswith(".so") or ".so." in line})
    except OSError:
        return []


def run_reference(args):
    """The reference algorithm's CPU implementation (the FP64 oracle, all host
    threads) on the same workload, built from the oracle's own mesh and IC
    routines: this arm maps no GPU library of the product."""
    world, rank, local = dist_setup()
    if rank != 0:
        return
    from oracle import oracle as orc
    from oracle import workloads
    w, desc = workloads.build(args.workload)
    if any("libmcv_gpu" in m for m in mapped_libraries()):
        raise RuntimeError("the reference arm must not load the GPU library")
    o = w.o
    o.step(min(args.warmup, 2))
    # bounded sample: at most args.steps RK steps or ~90 s of CPU time
    done, t0 = 0, time.perf_counter()
    while done < args.steps and (time.perf_counter() - t0) < 90.0:
        o.step(1)
        done += 1
    el = time.perf_counter() - t0
    value = done * w.dt / 86400.0 / el
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": done, "warmup": min(args.warmup, 2), "ms_per_step": 1e3 * el / done,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": desc, "order": w.order, "nc": w.nc, "scheme": w.scheme,
                                            "precision": "fp64", "dt_s": w.dt},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": orc.num_threads(), "kind": "port",
                             "sample": f"{done} RK steps (of {args.steps} asked; capped at ~90 s) after "
                                       f"{min(args.warmup, 2)} warm-up steps; inputs built by the oracle "
                                       f"(oracle/workloads.py), no GPU library mapped"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "libraries": [m for m in mapped_libraries() if "oracle" in m or "mcv" in m]}
    print(json.dumps(strict_json(line), allow_nan=False), flush=True)


def time_path(args, st, geom, precision, world, barrier, dist, local):
    """Device time of args.steps RK steps of one precision (state resident)."""
    import torch
    from mcv_sw_b200 import api
    n_pv = 6 * geom.n * geom.n
    s = api.Stepper(st.order, st.nc, st.dt, st.scheme, members=1, precision=precision, radius=6.371e6)
    s.set_geometry(geom)
    if args.tiles:
        s.select_tile(int(args.tiles.split(",")[0 if precision == "fp64" else 1]))
    s.set_member(0, st.phi_s, st.u, st.v, st.phi)
    s.time_steps(max(args.warmup, 3))
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    ms = s.time_steps(args.steps)
    barrier()
    clk = clocks.stop()
    ms = max_over_ranks(ms, dist)
    value = replica_value(world, args.steps, st.dt, ms)
    stage_ms, halo_ms = s.profile_step(3)
    per_pv = stage_bytes(st.scheme, precision)
    achieved = sum(b * n_pv for b in per_pv) / (sum(stage_ms) * 1e-3) / 1e9
    cands, chosen = s.tuning()
    out = {"value": value, "ms_per_step": ms / args.steps, "stage_ms": stage_ms, "halo_ms": halo_ms,
           "achieved_gbs": achieved, "bytes_per_pv_step": sum(per_pv), "clocks": clk,
           "tile": {"shape_fields": ["cells_x", "cells_y", "threads", "walk_cells", "ctas_per_sm", "tma"],
                    "chosen": list(cands[chosen][0]),
                    "candidates": [{"shape": list(c), "ms": round(t, 5)} for c, t in cands]}}
    return s, out


def ensemble_block(steps=40, days=2.0, members=64):
    """Batched ensemble: `members` MCV3 Nc=128 RK4 states (per-member tilt,
    u0 and harmonic RMS) advanced together, each stage one launch over all
    members.  Throughput in member-days per second; per-member normalized L2
    height error of split precision against the FP64 path after `days`."""
    from mcv_sw_b200 import api, cases, diag
    geom = api.Geometry(3, 128, cases.EARTH_RADIUS)
    sts = [cases.ensemble_member(geom, 1000 + m, days=days) for m in range(members)]
    dt = min(st.dt for st in sts)  # one dt for the batch: CFL 0.5 for every member
    nsteps = int(np.ceil(days * 86400.0 / dt))
    dt = days * 86400.0 / nsteps
    out = {"config": f"{members} members, MCV3 Nc=128 RK4, dt {dt:.2f} s, {days} days ({nsteps} steps)"}
    finals = {}
    for precision in ("fp64", "mixed"):
        with api.Stepper(3, 128, dt, "RK4", members=members, precision=precision, radius=cases.EARTH_RADIUS) as s:
            s.set_geometry(geom)
            for m, st in enumerate(sts):
                s.set_member(m, st.phi_s, st.u, st.v, st.phi)
            m0 = [s.mass_energy(m)[0] for m in range(members)]
            s.time_steps(3)
            ms = s.time_steps(steps)
            cands, chosen = s.tuning()
            s.step(nsteps - 3 - steps)
            finals[precision] = [s.get_state(m)["phi"] / cases.GRAVITY for m in range(members)]
            drift = [abs(s.mass_energy(m)[0] - m0[m]) / m0[m] for m in range(members)]
        out[precision] = {"member_days_per_s": members * steps * dt / 86400.0 / (ms / 1e3),
                          "ms_per_step": ms / steps, "tile_chosen": list(cands[chosen][0]),
                          "tile_candidates": [{"shape": list(c), "ms": round(t, 5)} for c, t in cands],
                          "max_abs_mass_drift": max(drift)}
    errs = [diag.norms(geom, finals["mixed"][m], finals["fp64"][m]) for m in range(members)]
    l2 = np.array([e[1] for e in errs])
    out["mixed_height_error_vs_fp64"] = {"L2_median": float(np.median(l2)), "L2_max": float(l2.max()),
                                         "L1_max": float(max(e[0] for e in errs)),
                                         "Linf_max": float(max(e[2] for e in errs)),
                                         "L2_per_member": [float(x) for x in l2]}
    out["speedup_mixed_vs_fp64"] = out["mixed"]["member_days_per_s"] / out["fp64"]["member_days_per_s"]
    return out


def serving_block(count, python_count, baseline_count):
    """The serving stream through the continuous-batching loops in split
    precision -- its first `count` requests through the native request loop
    behind the C ABI (mcv_server_*, what a C or Fortran driver calls), its
    first `python_count` through the Python loop over the per-handle calls --
    and its first `baseline_count` through the plain FP64
    one-request-at-a-time loop.  The stream (Poisson arrivals at 20 req/s)
    asks for far more simulated days per second than one GPU delivers, so
    latencies include the backlog that builds up over the stream; forecasts
    that become non-finite are reported (the reference scheme has no
    dissipation: some MCV4 forecasts with a mountain blow up in FP64 too)."""
    from mcv_sw_b200 import serving
    n = max(count, python_count, baseline_count)
    reqs, geoms = serving.make_requests(n, specs=True)
    out = {"stream": "Poisson 20 req/s (seed 4), MCV3/MCV4 50/50, Nc 48/96/192/384 (.4/.3/.2/.1), 6-120 h, half "
                     "with mountains; RK3_TVD, CFL 0.45; geometry and initial states generated on the device at "
                     "admission"}
    if count > 0:
        # grouping: idle pools of one order whose grids lie in one factor-8
        # size class advance together in one batched launch per stage
        stats = {}
        res, busy = serving.run_native(reqs[:count], precision="mixed", geoms=geoms, grouping=(4, 8.0),
                                       stats_out=stats)
        out["native_server_mixed"] = dict(serving.summarize(res), max_concurrent_pools=busy,
                                          chunks=stats.get("chunks"), grouped_chunks=stats.get("grouped_chunks"),
                                          pools_created=stats.get("pools_created"),
                                          loop="mcv_server_submit_balanced_flow / mcv_server_poll / "
                                               "mcv_server_result, grouping (4 grids, size class x8)")
    if python_count > 0:
        sub = reqs[:python_count]
        srv = serving.ForecastServer(precision="mixed", geoms=geoms, device_setup=True)
        srv.prepare(sorted({r.key for r in sub}))
        res = srv.run(sub)
        out["python_server_mixed"] = dict(serving.summarize(res), **srv.stats)
        srv.close()
    if baseline_count > 0:
        base = serving.run_one_at_a_time(reqs[:baseline_count], precision="fp64", geoms=geoms, device_setup=True)
        out["one_at_a_time_fp64"] = serving.summarize(base)
    return out


def stress_block(steps=200):
    """Roofline stress: MCV4 Nc=1024 RK4; per-stage-kernel achieved GB/s and the
    halo kernel's share of the step, FP64 and split precision."""
    from mcv_sw_b200 import api
    st, geom = build_workload("stress")[:2]
    n_pv = 6 * geom.n * geom.n
    out = {"config": f"MCV4 Nc=1024 RK4, {n_pv} PVs per field, {steps} steps"}
    for precision in ("fp64", "mixed"):
        with api.Stepper(st.order, st.nc, st.dt, st.scheme, precision=precision, radius=6.371e6) as s:
            s.set_geometry(geom)
            s.set_member(0, st.phi_s, st.u, st.v, st.phi)
            s.time_steps(3)
            ms = s.time_steps(steps)
            stage_ms, halo_ms = s.profile_step(3)
            per_pv = stage_bytes(st.scheme, precision)
            out[precision] = {"ms_per_step": ms / steps,
                              "stage_gbs": [b * n_pv / (t * 1e-3) / 1e9 for b, t in zip(per_pv, stage_ms)],
                              "stage_ms": stage_ms, "halo_ms": halo_ms,
                              "halo_share_of_step": len(stage_ms) * halo_ms / (ms / steps),
                              "tile_chosen": list(s.tuning()[0][s.tuning()[1]][0])}
    return out


def admission_block(order=4, nc=384, repeats=3):
    """Admission of one new grid and request (the largest serving grid): the host
    init chain (geometry build and upload, initial state on the host and
    upload) vs geometry and initial state generated on the device.  Wall-clock
    ms of the blocking API calls, best of `repeats`, handle creation excluded."""
    import numpy as np
    from mcv_sw_b200 import api, cases
    times = {"host_chain": [], "device": []}
    for _ in range(repeats):
        for how in ("host_chain", "device"):
            with api.Stepper(order, nc, 30.0, "RK3_TVD", precision="mixed", radius=cases.EARTH_RADIUS) as s:
                t0 = time.perf_counter()
                if how == "host_chain":
                    geom = api.Geometry(order, nc, cases.EARTH_RADIUS)
                    s.set_geometry(geom)
                    spec = cases.balanced_flow_spec(geom, np.random.default_rng(17), lmax=8, rms=10.0, mountain=True)
                    zw, mw, phi, phis = cases.balanced_flow_from_spec(geom, spec)
                    u, v = api.sphere_to_cov(geom, zw, mw)
                    s.set_member(0, phis, u, v, phi)
                else:
                    s.set_geometry_equiangular()
                    spec = cases.balanced_flow_spec(s, np.random.default_rng(17), lmax=8, rms=10.0, mountain=True)
                    s.set_member_balanced_flow(0, spec)
                times[how].append(1e3 * (time.perf_counter() - t0))
    return {"config": f"MCV{order} Nc={nc} split precision, balanced flow + degree<=8 harmonics + mountain",
            "host_chain_ms": min(times["host_chain"]), "device_ms": min(times["device"]),
            "speedup": min(times["host_chain"]) / min(times["device"])}


def run_ours(args):
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from mcv_sw_b200 import api, diag
    st, geom, desc = build_workload(args.workload)
    n_pv = 6 * geom.n * geom.n

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    paths = {}
    timed = [x for x in ("fp64", "mixed") if x in args.paths.split(",")]
    if args.precision not in timed:
        raise SystemExit("--paths must include the headline --precision")
    for precision in timed:
        s, paths[precision] = time_path(args, st, geom, precision, world, barrier, dist, local)
        if precision != args.precision:
            s.close()
        else:
            main = s
    head = paths[args.precision]
    peak, peak_kind = measured_peak()
    traffic_pv = stage_traffic_per_pv()
    key = (args.workload, f"{st.scheme}-{args.precision}")
    traffic = traffic_pv[key] * n_pv if key in traffic_pv else None
    nst = len(head["stage_ms"])
    roofline = {"bound": "hbm", "achieved": head["achieved_gbs"], "peak": peak, "unit": "GB/s",
                "frac": head["achieved_gbs"] / peak, "traffic": traffic, "peak_source": peak_kind,
                "kernel": f"stage_kernel ({args.precision})",
                "algorithmic_bytes_per_launch": head["bytes_per_pv_step"] * n_pv / nst,
                "stage_ms": head["stage_ms"], "halo_ms": head["halo_ms"],
                "halo_share_of_step": nst * head["halo_ms"] / head["ms_per_step"]}

    # end to end through the C ABI with pinned host buffers: per step upload the
    # state (u, v, phi), advance one RK step, download the state
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    hp = {k: pin(getattr(st, k)) for k in ("phi_s", "u", "v", "phi")}
    ho = {k: torch.empty(geom.shape, dtype=torch.float64).pin_memory().numpy() for k in ("u", "v", "phi")}
    e2e = None
    if args.e2e_steps > 0:
        main.set_member(0, hp["phi_s"], hp["u"], hp["v"], hp["phi"])
        main.step(1)
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            main.set_state(0, hp["u"], hp["v"], hp["phi"])
            main.step(1)
            main.get_state(0, out=ho)
        barrier()
        e2e_s = time.perf_counter() - t0
        e2e_s = max_over_ranks(e2e_s, dist)
        field_bytes = 8 * 6 * geom.npx * geom.npx
        e2e = {"value": world * args.e2e_steps * st.dt / 86400.0 / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": 3 * field_bytes, "d2h_bytes_per_step": 3 * field_bytes,
               "how": "per step: mcv_set_state (u, v, phi from pinned host) + mcv_step(1) + "
                      "mcv_get_state (u, v, phi to pinned host); host wall clock around synchronous calls"}
    main.close()

    # accuracy of split precision against the FP64 path over the full forecast,
    # as a daily curve, beside an FP64 "twin" whose initial phi differs by 1e-12
    # (relative, pointwise): the twin shows how far the flow itself amplifies a
    # perturbation of that size
    accuracy = None
    # (one GPU only: at N > 1 the other ranks would wait for it at the final barrier)
    if rank == 0 and world == 1 and args.error_days > 0:
        nsteps = int(round(args.error_days * 86400.0 / st.dt))
        twin_phi = st.phi * (1.0 + 1e-12 * np.random.default_rng(0).standard_normal(st.phi.shape))
        runs = {"fp64": ("fp64", st.phi), "fp64_twin": ("fp64", twin_phi), "mixed": ("mixed", st.phi)}
        ncheck = max(1, int(round(args.error_days)))
        curves, drift, finite_days = {k: [] for k in runs}, {}, {}
        H, n = geom.H, geom.n
        for name, (precision, phi0) in runs.items():
            with api.Stepper(st.order, st.nc, st.dt, st.scheme, precision=precision, radius=6.371e6) as s:
                s.set_geometry(geom)
                s.set_member(0, st.phi_s, st.u, st.v, phi0)
                m0, _ = s.mass_energy(0)
                done = 0
                finite_days[name] = 0.0
                for c in range(ncheck):
                    k = (nsteps * (c + 1)) // ncheck - done
                    s.step(k)
                    done += k
                    phi = s.get_state(0)["phi"] / 9.80616
                    curves[name].append(phi)
                    if np.isfinite(phi[:, H:H + n, H:H + n]).all() and finite_days[name] == done - k:
                        finite_days[name] = done
                m1, _ = s.mass_energy(0)
                drift[name] = (m1 - m0) / m0
                finite_days[name] *= st.dt / 86400.0

        def norms(a, b):
            if not np.isfinite(a[:, H:H + n, H:H + n]).all():
                return (float("nan"),) * 3
            return diag.norms(geom, a, b)

        days = [nsteps * (c + 1) // ncheck * st.dt / 86400.0 for c in range(ncheck)]
        mixed_curve = [norms(curves["mixed"][c], curves["fp64"][c]) for c in range(ncheck)]
        twin_curve = [norms(curves["fp64_twin"][c], curves["fp64"][c]) for c in range(ncheck)]
        l1, l2, linf = mixed_curve[-1]
        accuracy = {"sim_days": nsteps * st.dt / 86400.0, "steps": nsteps,
                    "height_error_vs_fp64": {"L1": l1, "L2": l2, "Linf": linf},
                    "curve_days": days, "mixed_L2_curve": [c[1] for c in mixed_curve],
                    "fp64_twin_L2_curve": [c[1] for c in twin_curve],
                    "mass_drift": {"fp64": drift["fp64"], "mixed": drift["mixed"]},
                    # the last check (in simulated days) up to which each run stayed finite
                    "finite_through_days": finite_days,
                    "reference": "FP64 GPU path (oracle-validated by the parity tests); fp64_twin: the FP64 "
                                 "path from phi*(1+1e-12*N(0,1))"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(st)
    # the other configurations (one GPU: the multi-rank run only measures the main workload)
    extra = {}
    if rank == 0 and world == 1:
        if args.ensemble:
            extra["ensemble"] = ensemble_block()
        if max(args.serve_requests, args.serve_python_requests, args.serve_baseline_requests) > 0:
            extra["serving"] = serving_block(args.serve_requests, args.serve_python_requests,
                                             args.serve_baseline_requests)
        if args.stress:
            extra["stress"] = stress_block()
        if args.admission:
            extra["admission"] = admission_block()
    if rank == 0:
        other = "fp64" if args.precision == "mixed" else "mixed"
        line = {"metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "f32+f64", "data": "synthetic",
                "config": {"workload": desc, "order": st.order, "nc": st.nc, "scheme": st.scheme,
                           "precision": args.precision, "dt_s": st.dt, "interior_pvs": n_pv,
                           "parallelism": f"replicas{world}",
                           "l2": "no flush: each stage reads > 126 MB (inputs larger than L2)"},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": args.steps * 2 * nst, "clocks": head["clocks"],
                "paths": paths,
                f"speedup_{args.precision}_vs_{other}": (head["value"] / paths[other]["value"]
                                                         if other in paths else None),
                # like for like: the FP64 GPU path against the FP64 CPU oracle on the same box
                "fp64_gpu_vs_cpu_baseline": (paths["fp64"]["value"] / cpu["value"]
                                             if cpu and "fp64" in paths else None),
                "accuracy": accuracy, **extra}
        print(json.dumps(strict_json(line), allow_nan=False), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
