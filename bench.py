"""Benchmark: coupled heat simulation on the standard-tissue cube (the C0 geometry), plus the
plain MC transport of that cube, on B200 through the library's C ABI.

Workload ("coupled heat on config-0 geometry"):
  * geometry: 100^3 voxels over a 0.1 cm cube (air / epidermis / dermis / vessel);
  * heat source: absorbed power of a 1 W pencil beam from a 1e6-packet MC run (seed 1);
  * thermal: VHC 3.9, TC 0.0037 (tissue), VHC 0.0012, TC 0.00026 (air); T0 = 37 degC;
    damage in the vessel (E = 4.48e5 J/mol, A = 7.6e66 /s); insulating faces;
  * dt = 0.9 x the explicit stability limit (calcdtmax);
  * one bench step = one call of the stepper over `--nt` DG-ADI time steps with the light on
    (the illumination phase of the schedule; a full update call of that phase is ~1.45e5 steps).
Metric: heat voxel-updates/s (voxels x time steps / s), whole job. The MC transport of the
same cube (photon packets/s) is reported in the same line under "mc" (with N GPUs: N x 1e6
packets sharded over the ranks, tallies merged by one NCCL all-reduce). On 1 GPU the line also
carries the batched sweep ("mc_batched": batched launch vs per-instance launches), the
perturbation-MC gradients ("mc_grad": gradient run vs plain forward on the 256^3 8-medium cube)
and the heat adjoint ("heat_adjoint": adjoint vs forward on 300x300x200, 2000 steps).

Timing: `value` = device time (CUDA events recorded by the library on its own stream) of the
stepping loop with all grids resident in HBM; L2 is flushed (256 MB write) between timed steps
because the 100^3 working set (~30 MB) is smaller than L2. `e2e` = the same metric through
mcb_heat_forward with host buffers (H2D of the inputs and D2H of T, Omega, sensors and maxima
inside the timed region), wall clock per call.

`--impl reference` times the reference's own C heat stepper (finiteElementHeatPropagator.c,
compiled from source with the reference's flags into oracle/_ref) on all host cores, on a
bounded sample of steps of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import tempfile
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from mcmatlab_b200 import configs, mexargs, prep  # noqa: E402

METRIC = "photon packets/s, heat voxel-updates/s on 1 B200; batched+adjoint vs plain"
HEAT_STEP_DRAM_BYTES = 27.4e6
N_GRID = 100
MC_PACKETS = 1_000_000


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def build_heat_inputs(NA_sum, m):
    G = m.G
    media = G.mediaPropertiesFunc([])
    th = prep.thermal_media_properties(media, G.M_raw)
    c, Q = prep.calc_dTdt_arrays(th["VHC"], th["TC"], G.dx, G.dy, G.dz, NA_sum, 1.0, th["M"])
    dtmax = prep.calc_dtmax(th["M"], th["TC"], th["VHC"], G.dx, G.dy, G.dz)
    dt = 0.9 * dtmax
    return th, c, Q, dt


class ClockSampler:
    """nvidia-smi clocks sampled every 200 ms during the timed region."""

    def __init__(self, gpu_index=0):
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), "mcb_bench_clocks_%d.csv" % os.getpid())
        self.gpu = gpu_index

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
            sm = [float(r[1]) for r in rows]
            mx = float(rows[0][2])
            reasons = set()
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for r in rows:
                for k, nme in enumerate(names):
                    if r[5 + k].strip().lower().startswith("active"):
                        reasons.add(nme)
            return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}
        except Exception:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, None
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    return rank, ws, dist


def run_ours(args):
    import torch
    from mcmatlab_b200 import native
    rank, ws, dist = dist_init()
    dev = torch.cuda.current_device() if torch.cuda.is_available() else 0
    m = configs.standard_tissue_cube(n=N_GRID, nPhotons=MC_PACKETS * ws, seed=1)
    mc_in = mexargs.prepare_mc(m)
    # warm the transport once, then time it (packets/s on the cube). With N ranks the N x 1e6
    # packets of one seed are sharded over the ranks (packet r, r + N, ...) and the tallies are
    # merged by one all-reduce (NCCL); the time is the max over ranks of transport + merge.
    mc_small = dict(mc_in)
    mc_small["nPhotonsRequested"] = 1e5
    native.mc_run(mc_small, device=dev)
    # the launch-parameter autotuner on this workload's size class (1e6 packets per candidate);
    # the timed run below uses its choice
    tune = native.mc_autotune(mc_in, 1e6, device=dev)
    if dist:
        from mcmatlab_b200 import shard
        dist.barrier()
    t0 = time.perf_counter()
    if dist:
        out = native.mc_run(shard.shard_model(mc_in, rank, ws), device=dev)
        mc_ms = out["kernelMs"]
        steps_mc = out["propagationSteps"]
        tm = time.perf_counter()
        out = shard.merge(out, mc_in, rank, ws, shard.torch_allreduce())
        merge_ms = (time.perf_counter() - tm) * 1e3
        t = torch.tensor([mc_ms + merge_ms, time.perf_counter() - t0, float(steps_mc)], dtype=torch.float64, device="cuda")
        dist.all_reduce(t[:2], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[2:], op=dist.ReduceOp.SUM)
        mc_ms, mc_wall, steps_mc = float(t[0]), float(t[1]), int(t[2])
    else:
        out = native.mc_run(mc_in, device=dev)
        mc_wall = time.perf_counter() - t0
        mc_ms = out["kernelMs"]
        steps_mc = out["propagationSteps"]
    NFR = out["NFR"][..., 0]
    mua = mc_in["mua"][:, 0]
    NA = mua[mc_in["M"].astype(np.int64) - 1].astype(np.float32) * NFR
    th, c, Q, dt = build_heat_inputs(NA, m)
    hp = mexargs.heat_mex_params(th["M"], th["A"], th["E"], c, Q, True, 0, None, None, True, args.nt, dt)
    T0 = np.full((N_GRID,) * 3, 37.0, np.float32, order="F")
    O0 = np.zeros((N_GRID,) * 3, np.float32, order="F")
    L = N_GRID ** 3
    state = native.HeatState(T0, O0, hp, N_GRID, N_GRID, N_GRID, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2
    for _ in range(args.warmup):
        state.step(hp)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    times = []
    with ClockSampler(dev) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            state.step(hp)
            times.append(native.last_kernel_ms(dev))
    torch.cuda.synchronize()
    # the light-off phase of the schedule (no source term) on the same resident state
    hp_off = dict(hp, lightsOn=False)
    state.step(dict(hp_off, steps=float(min(args.nt, 1000))))
    off_times = []
    for _ in range(max(1, args.steps // 2)):
        flush.zero_()
        torch.cuda.synchronize()
        state.step(hp_off)
        off_times.append(native.last_kernel_ms(dev))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    dev_ms = float(sum(times))
    # e2e through the host-buffer entry point
    e2e_times = []
    Tn, On = T0.copy(order="F"), O0.copy(order="F")
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        Tn, On, _, _ = native.heat_forward(Tn, On, hp, N_GRID, N_GRID, N_GRID, device=dev)
        if k >= args.warmup:
            e2e_times.append(time.perf_counter() - t0)
    e2e_s = float(sum(e2e_times))
    if dist:
        t = torch.tensor([dev_ms, e2e_s], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_ms, e2e_s = float(t[0]), float(t[1])
    updates = float(L) * args.nt * args.steps * ws
    value = updates / (dev_ms / 1e3)
    e2e_value = updates / e2e_s
    ms_per_step = dev_ms / args.steps
    # roofline: algorithmic bytes per voxel-update with the light on: T read + write (8), M (1),
    # source (4), plus Omega read + write (8) in the voxels that accumulate damage
    frac_dmg = float(np.mean(th["E"][th["M"].astype(np.int64) - 1] != 0))
    bytes_per_update = 9.0 + 4.0 + 8.0 * frac_dmg
    hbm, src = peaks()
    achieved = bytes_per_update * L * args.nt / (ms_per_step / 1e3) / 1e9
    # light off: no source read (T read + write, M, and Omega where damage accumulates)
    off_ms = float(np.mean(off_times))
    off_bytes = 9.0 + 8.0 * frac_dmg
    off_achieved = off_bytes * L * args.nt / (off_ms / 1e3) / 1e9
    # one bench step: 3 passes per time step + the maxima decode
    launches = args.steps * (3 * args.nt + 1)
    res = {
        "metric": METRIC, "value": value, "unit": "voxel-updates/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (tallies f64)", "data": "synthetic",
        "config": {"workload": "coupled heat on the 100^3 standard-tissue cube (config-0 geometry), light on, "
                               "DG-ADI + Arrhenius, dt = 0.9 x stability limit",
                   "grid": [N_GRID] * 3, "time_steps_per_bench_step": args.nt, "dt_s": dt,
                   "heat_source": "absorbed power of a 1e6-packet pencil-beam MC run at 1 W",
                   "l2": "flushed (256 MB write) between timed steps", "parallelism": "replicas" if ws > 1 else "1 GPU"},
        "e2e": {"value": e2e_value, "unit": "voxel-updates/s",
                "h2d_bytes_per_step": int(L * (4 + 4 + 1 + 4) + 12 * len(th["VHC"]) ** 2 + 16 * len(th["VHC"])),
                "d2h_bytes_per_step": int(L * 8 + 4 * len(th["VHC"])),
                "timing": "wall clock around mcb_heat_forward (host buffers)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_source": src,
                     # DRAM bytes of one DG-ADI step (X + Y + Z pass) from a cold-cache ncu capture of
                     # this workload (reads; the writes stay in L2); in the timed loop the grid is
                     # L2-resident
                     "traffic": HEAT_STEP_DRAM_BYTES, "traffic_note": "ncu cold-cache capture, bytes per DG-ADI step",
                     "algorithmic_bytes_per_voxel_update": bytes_per_update,
                     "kernel": "DG-ADI step (sx_kernel + scol_kernel<y> + scol_kernel<z>)"},
        "light_off": {"workload": "same state and dt, light off (the cooling phase of the schedule)",
                      "value": float(L) * args.nt / (off_ms / 1e3), "unit": "voxel-updates/s", "ms_per_step": off_ms,
                      "steps": len(off_times),
                      "roofline": {"bound": "hbm", "achieved": off_achieved, "peak": hbm, "unit": "GB/s",
                                   "frac": off_achieved / hbm, "peak_source": src,
                                   "algorithmic_bytes_per_voxel_update": off_bytes}},
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "mc": {"metric": "photon packets/s", "workload": "standard-tissue cube 100^3, pencil beam, %d x 1e6 packets" % ws,
               "value": MC_PACKETS * ws / (mc_ms / 1e3), "e2e_value": MC_PACKETS * ws / mc_wall,
               "kernel_ms": mc_ms, "propagation_steps": steps_mc,
               "free_step_cuts": out.get("freeStepCuts"), "free_step_cut_weight_fraction":
                   (out.get("freeStepCutWeight", 0.0) / out["nPhotons"]) if out.get("nPhotons") else None,
               "steps_per_s": steps_mc / (mc_ms / 1e3),
               "autotune": {"refillMin": tune["refillMin"], "scatterMin": tune["scatterMin"],
                            "candidate_ms_min": float(tune["table"][:, 2].min()),
                            "candidate_ms_max": float(tune["table"][:, 2].max())},
               "parallelism": "packets sharded over %d ranks, one NCCL all-reduce of the tallies" % ws if ws > 1 else "1 GPU"},
    }
    # transport roofline: propagation sub-steps/s against the measured scattered FP64 atomicAdd
    # rate (one deposit per sub-step is the algorithmic work; runs in one voxel share one atomic)
    atom = native.probe_atomics(1 << 20, device=dev)
    res["mc"]["roofline"] = {"bound": "fp64 atomics", "achieved": steps_mc / (mc_ms / 1e3), "peak": atom,
                             "unit": "sub-steps/s vs FP64 atomicAdd/s", "frac": steps_mc / (mc_ms / 1e3) / atom,
                             "peak_source": "measured in this run: mcb_probe_atomics, 2^20 scattered slots"}
    # the remaining measurements are single-GPU ones (run on 1-GPU invocations only)
    if args.c2 and ws == 1:
        res["mc_batched"] = batched_sweep_measure(dev, args.c2_instances, args.c2_scale)
    if args.c3 and ws == 1:
        res["mc_grad"] = grad_measure(dev, args.c3_packets, args.c3_grid)
    if args.c4 and ws == 1:
        res["heat_adjoint"] = adjoint_measure(dev, args.c4_steps)
    if args.lbfgs and ws == 1:
        res["lbfgs"] = lbfgs_measure(dev, args.c3_packets, args.c3_grid)
    if rank == 0:
        if args.cpu_baseline:
            res["cpu_baseline"] = cpu_baseline(args, sample_steps=args.ref_nt)
            res["mc"]["cpu_baseline"] = res["cpu_baseline"].pop("mc")
            c4 = res["cpu_baseline"].pop("heat_c4")
            if "heat_adjoint" in res:
                res["heat_adjoint"]["cpu_forward"] = c4
            c2 = res["cpu_baseline"].pop("mc_batched")
            if "mc_batched" in res and c2:
                res["mc_batched"]["cpu_baseline"] = c2
        print(json.dumps(res), flush=True)
    state.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


_SWEEP = {}


def sweep_inputs(n_inst, scale):
    """MEX-level inputs of the batched sweep's instances (prepared once per process)."""
    key = (n_inst, scale)
    if key not in _SWEEP:
        models = configs.batched_sweep(n_instances=n_inst, seed=7, photons=(1e5 * scale, 1e7 * scale))
        _SWEEP[key] = [mexargs.prepare_mc(x) for x in models]
    return _SWEEP[key]


def batched_sweep_measure(dev, n_inst, scale):
    """Batched sweep (64 seeded instances, grids 64^3..200x200x150, 450-900 nm, 1e5-1e7 packets
    log-uniform, Gaussian beams, half with 64 time bins and cyclic x/y boundaries): one batched
    launch vs the plain kernel launched once per instance."""
    from mcmatlab_b200 import native
    ins = sweep_inputs(n_inst, scale)
    total = float(sum(x["nPhotonsRequested"] for x in ins))
    native.mc_run(dict(ins[0], nPhotonsRequested=1e4), device=dev)
    # warm-up over every instance, so the batch's device buffers are sized before the timed calls
    native.mc_run_batch([dict(x, nPhotonsRequested=1e3) for x in ins], device=dev)
    plain_ms = plain_wall = 0.0
    per_inst = []
    for x in ins:
        t0 = time.perf_counter()
        o = native.mc_run(x, device=dev)
        plain_wall += time.perf_counter() - t0
        plain_ms += o["kernelMs"]
        per_inst.append([float(x["nPhotonsRequested"]), int(np.asarray(x["M"]).size), round(float(o["kernelMs"]), 3)])
    t0 = time.perf_counter()
    outs = native.mc_run_batch(ins, device=dev)
    batch_wall = time.perf_counter() - t0
    batch_ms = outs[0]["kernelMs"]
    return {"workload": "%d-instance batched sweep (grids 64^3..200x200x150, 450-900 nm, %.0e-%.0e packets)"
                        % (n_inst, 1e5 * scale, 1e7 * scale),
            "packets": total,
            "batched_packets_per_s": total / (batch_ms / 1e3), "plain_per_instance_packets_per_s": total / (plain_ms / 1e3),
            "ratio_device": plain_ms / batch_ms,
            "batched_e2e_packets_per_s": total / batch_wall, "plain_e2e_packets_per_s": total / plain_wall,
            "ratio_e2e": plain_wall / batch_wall,
            "free_step_cuts": float(sum(o["freeStepCuts"] for o in outs)),
            "free_step_cut_weight_fraction": float(sum(o["freeStepCutWeight"] for o in outs) / sum(o["nPhotons"] for o in outs)),
            "plain_instances": {"columns": ["packets", "voxels", "plain_kernel_ms"], "rows": per_inst}}


def grad_measure(dev, packets, n):
    """Perturbation-MC gradients on the 0.5 cm, 8-medium cube (n^3 voxels): 32 radial reflectance
    bins and the mean fluence of a 16^3 box, d/dmua and d/dmus of every medium, against one plain
    forward run of the same packets."""
    from mcmatlab_b200 import native
    mc_in = mexargs.prepare_mc(configs.perturbation_cube(n=n, nPhotons=packets))
    z0 = n // 6
    box = [n // 2 - 8, n // 2 + 8, n // 2 - 8, n // 2 + 8, z0, z0 + 16]
    obj = dict(nRadialBins=32, radialBinWidth=0.25 / 32, box=box)
    native.mc_run(dict(mc_in, nPhotonsRequested=1e5), device=dev)
    native.mc_grad(dict(mc_in, nPhotonsRequested=1e5), device=dev, **obj)
    fwd = native.mc_run(mc_in, device=dev)
    o, g = native.mc_grad(mc_in, device=dev, **obj)
    return {"workload": "perturbation MC, %d^3 voxels over a 0.5 cm cube, 8 tissue media + air, %.0e packets, "
                        "32 radial reflectance bins + 16^3-box fluence, d/dmua and d/dmus of 9 media" % (n, packets),
            "forward_packets_per_s": packets / (fwd["kernelMs"] / 1e3),
            "grad_packets_per_s": packets / (o["kernelMs"] / 1e3),
            "forward_ms": fwd["kernelMs"], "grad_ms": o["kernelMs"],
            "grad_over_forward": o["kernelMs"] / fwd["kernelMs"], "target_grad_over_forward": 1.5}


def adjoint_measure(dev, nt):
    """Heat adjoint on 300x300x200 voxels (4 seeded media, Gaussian source, damage and peak
    objectives) with ceil(sqrt(nt)) checkpoints, against the plain forward of the same steps."""
    from mcmatlab_b200 import native
    case = configs.heat_adjoint_case(nt=nt)
    nx, ny, nz = case["n"]
    native.heat_forward(case["T0"], None, dict(case["hp"], steps=4.0), nx, ny, nz, device=dev)
    native.heat_forward(case["T0"], None, case["hp"], nx, ny, nz, device=dev)
    fwd_ms = native.last_kernel_ms(dev)
    g = native.heat_adjoint(case["T0"], case["hp"], nx, ny, nz, case["wd"], case["wp"], device=dev)
    L = nx * ny * nz
    res = {"workload": "heat adjoint, 300x300x200 voxels, 4 media, %d steps, %d checkpoints, damage + peak objectives"
                       % (nt, math.ceil(math.sqrt(nt))),
           "forward_voxel_updates_per_s": L * nt / (fwd_ms / 1e3), "forward_ms": fwd_ms,
           "adjoint_forward_sweep_ms": g["forwardMs"], "adjoint_reverse_sweep_ms": g["adjointMs"],
           "adjoint_over_forward": (g["forwardMs"] + g["adjointMs"]) / fwd_ms}
    # every state stored (nCheckpoints = steps) where HBM holds them: no recomputation
    import torch
    need = 4 * L * (nt + 16) + (8 << 30)
    if torch.cuda.is_available() and torch.cuda.mem_get_info(dev)[0] > need:
        ga = native.heat_adjoint(case["T0"], case["hp"], nx, ny, nz, case["wd"], case["wp"], nCheckpoints=nt, device=dev)
        res["all_states"] = {"stored_GB": 4 * L * (nt + 1) / 1e9, "adjoint_forward_sweep_ms": ga["forwardMs"],
                             "adjoint_reverse_sweep_ms": ga["adjointMs"],
                             "adjoint_over_forward": (ga["forwardMs"] + ga["adjointMs"]) / fwd_ms,
                             "max_rel_diff_dJ_dT0": float(np.max(np.abs(ga["dJ_dT0"] - g["dJ_dT0"])) /
                                                          np.max(np.abs(g["dJ_dT0"])))}
    return res


def lbfgs_measure(dev, packets, n):
    """Recovery of the top two tissue layers' mua and mus of the n^3 8-medium cube from its 32-bin
    radial reflectance map (generated at the seeded ground truth with an independent seed and 2x
    the packets) by L-BFGS over perturbation-MC gradients, from mua x 1.5, mus x 0.7."""
    from mcmatlab_b200 import grad, native
    mc_in = mexargs.prepare_mc(configs.perturbation_cube(n=n, nPhotons=packets))
    obj = dict(nRadialBins=32, radialBinWidth=0.25 / 32, box=None)
    ta = np.asarray(mc_in["mua"])[:, 0].copy()
    ts = np.asarray(mc_in["mus"])[:, 0].copy()
    media = [1, 2]
    t0 = time.perf_counter()
    _, g = native.mc_grad(dict(mc_in, seed=1001, nPhotonsRequested=2 * packets), device=dev, **obj)
    r = grad.recover_optical_properties(mc_in, g["R"], media, obj, mua0=ta[media] * 1.5, mus0=ts[media] * 0.7,
                                        max_evals=45)
    return {"workload": "L-BFGS recovery of 2 layers' mua, mus on the %d^3 8-medium cube, %.0e packets per evaluation"
                        % (n, packets), "evaluations": r["evals"], "seconds": time.perf_counter() - t0,
            "relative_errors": {"mua": [float(r["mua"][m] / ta[m] - 1) for m in media],
                                "mus": [float(r["mus"][m] / ts[m] - 1) for m in media]},
            "final_loss": r["loss"]}


REF_MC_PACKETS = 1e6


def reference_setup(timings=None):
    from oracle import ref
    m = configs.standard_tissue_cube(n=N_GRID, nPhotons=REF_MC_PACKETS, seed=1)
    mc_in = mexargs.prepare_mc(m)
    tree = mexargs.mex_model_tree(mc_in)
    t0 = time.perf_counter()
    out = ref.RefMC().run(tree, seed=None)  # reference MC, all cores, for the heat source
    if timings is not None:
        timings["mc_s"] = time.perf_counter() - t0
        timings["mc_packets"] = float(np.asarray(out["nPhotons"]).ravel()[0])
    NFR = out["NFR"]
    NFR = NFR[..., 0] if NFR.ndim == 4 else NFR
    mua = mc_in["mua"][:, 0]
    NA = mua[mc_in["M"].astype(np.int64) - 1].astype(np.float32) * NFR
    return m, NA


def cpu_baseline(args, sample_steps):
    """The reference's own heat stepper on all host cores, bounded sample of `sample_steps` steps."""
    from oracle import ref
    tm = {}
    m, NA = reference_setup(tm)
    th, c, Q, dt = build_heat_inputs(NA, m)
    hp = mexargs.heat_mex_params(th["M"], th["A"], th["E"], c, Q, True, 0, None, None, True, sample_steps, dt)
    T0 = np.full((N_GRID,) * 3, 37.0, np.float32, order="F")
    O0 = np.zeros((N_GRID,) * 3, np.float32, order="F")
    R = ref.RefHeat()
    cores = os.cpu_count()
    R.run(T0, O0, dict(hp, steps=2.0), nthreads=cores)
    t0 = time.perf_counter()
    R.run(T0, O0, hp, nthreads=cores)
    dtw = time.perf_counter() - t0
    # the heat-adjoint workload's grid (300x300x200), forward steps only
    case = configs.heat_adjoint_case(nt=args.c4_cpu_steps)
    nx4, ny4, nz4 = case["n"]
    R.run(case["T0"], np.float32(np.nan), dict(case["hp"], steps=1.0), nthreads=cores)
    t0 = time.perf_counter()
    R.run(case["T0"], np.float32(np.nan), case["hp"], nthreads=cores)
    dt4 = time.perf_counter() - t0
    c4 = {"value": nx4 * ny4 * nz4 * args.c4_cpu_steps / dt4, "unit": "voxel-updates/s", "cores": cores, "kind": "reference",
          "sample": "%d DG-ADI steps of the 300x300x200 heat-adjoint workload (forward only, no damage), reference MEX C "
                    "code (-Ofast -fopenmp) on %d host threads" % (args.c4_cpu_steps, cores)}
    # the batched sweep's instances one after another on the reference MC, each with 0.5% of its packets
    # (at least 1e3): packets/s of the sweep's instance mix on the host cores
    c2 = None
    if args.c2:
        R2 = ref.RefMC()
        tp = ts = 0.0
        for x in sweep_inputs(args.c2_instances, args.c2_scale):
            mc_in = dict(x)
            mc_in["nPhotonsRequested"] = max(1e3, round(0.005 * mc_in["nPhotonsRequested"]))
            tree = mexargs.mex_model_tree(mc_in)
            t0 = time.perf_counter()
            out = R2.run(tree, seed=None)
            ts += time.perf_counter() - t0
            tp += float(np.asarray(out["nPhotons"]).ravel()[0])
        c2 = {"value": tp / ts, "unit": "photon packets/s", "cores": cores, "kind": "reference",
              "sample": "the %d instances of the batched sweep one after another, 0.5%% of each one's packets "
                        "(%.2e in all), reference MEX C code (-Ofast -fopenmp) on %d host threads"
                        % (args.c2_instances, tp, cores)}
    return {"value": N_GRID ** 3 * sample_steps / dtw, "unit": "voxel-updates/s", "cores": cores, "kind": "reference",
            "heat_c4": c4, "mc_batched": c2,
            "sample": "%d DG-ADI steps of the same 100^3 workload (light on, damage), reference MEX C code "
                      "(-Ofast -fopenmp) on %d host threads" % (sample_steps, cores),
            "mc": {"value": tm["mc_packets"] / tm["mc_s"], "unit": "photon packets/s", "cores": cores, "kind": "reference",
                   "sample": "%.0e packets of the 100^3 standard-tissue cube (MCmatlab.c, -Ofast -fopenmp, %d threads)"
                             % (tm["mc_packets"], cores)}}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import ref
    m, NA = reference_setup()
    th, c, Q, dt = build_heat_inputs(NA, m)
    hp = mexargs.heat_mex_params(th["M"], th["A"], th["E"], c, Q, True, 0, None, None, True, args.ref_nt, dt)
    T0 = np.full((N_GRID,) * 3, 37.0, np.float32, order="F")
    O0 = np.zeros((N_GRID,) * 3, np.float32, order="F")
    R = ref.RefHeat()
    cores = os.cpu_count()
    T, O = T0, O0
    for _ in range(args.warmup):
        T, O, _, _ = R.run(T, O, hp, nthreads=cores)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        T, O, _, _ = R.run(T, O, hp, nthreads=cores)
        times.append(time.perf_counter() - t0)
    tot = float(sum(times))
    value = N_GRID ** 3 * args.ref_nt * args.steps / tot
    res = {"metric": METRIC, "value": value, "unit": "voxel-updates/s", "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot / args.steps * 1e3, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
           "config": {"workload": "coupled heat on the 100^3 standard-tissue cube (config-0 geometry), light on, "
                                  "DG-ADI + Arrhenius, dt = 0.9 x stability limit",
                      "grid": [N_GRID] * 3, "time_steps_per_bench_step": args.ref_nt, "dt_s": dt},
           "cpu_baseline": {"value": value, "unit": "voxel-updates/s", "cores": cores, "kind": "reference",
                            "sample": "%d DG-ADI steps per bench step" % args.ref_nt},
           "e2e": {"value": value, "unit": "voxel-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(res), flush=True)


def run_profile(args):
    """Short runs of one workload for profiler captures (no JSON line; times printed for reference):
    heat-c1: the heat state of the 100^3 cube stepped args.nt steps (source from a 1e5-packet run);
    heat-c4: the 300x300x200 heat-adjoint grid stepped args.nt steps forward; mc-c0: the transport of
    the 100^3 cube at args.packets packets; each args.steps times."""
    from mcmatlab_b200 import native
    if args.profile == "mc-c0":
        mc_in = mexargs.prepare_mc(configs.standard_tissue_cube(n=N_GRID, nPhotons=args.packets, seed=1))
        for _ in range(args.steps):
            o = native.mc_run(mc_in)
            print("mc-c0: %.0f packets in %.3f ms" % (args.packets, o["kernelMs"]), flush=True)
        return
    if args.profile == "heat-c1":
        m = configs.standard_tissue_cube(n=N_GRID, nPhotons=1e5, seed=1)
        mc_in = mexargs.prepare_mc(m)
        out = native.mc_run(mc_in)
        NA = mc_in["mua"][:, 0][mc_in["M"].astype(np.int64) - 1].astype(np.float32) * out["NFR"][..., 0]
        th, c, Q, dt = build_heat_inputs(NA, m)
        hp = mexargs.heat_mex_params(th["M"], th["A"], th["E"], c, Q, True, 0, None, None, True, args.nt, dt)
        n = (N_GRID,) * 3
        T0, O0 = np.full(n, 37.0, np.float32, order="F"), np.zeros(n, np.float32, order="F")
    else:
        case = configs.heat_adjoint_case(nt=args.nt)
        n, hp, T0, O0 = case["n"], case["hp"], case["T0"], None
    st = native.HeatState(T0, O0, hp, *n)
    for _ in range(args.steps):
        st.step(hp)
        print("%s: %d steps in %.3f ms" % (args.profile, args.nt, native.last_kernel_ms(0)), flush=True)
    st.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nt", type=int, default=20000, help="DG-ADI time steps per bench step")
    ap.add_argument("--ref-nt", type=int, default=50, help="time steps per bench step of the CPU reference")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-c2", dest="c2", action="store_false", help="skip the batched-sweep measurement")
    ap.add_argument("--c2-instances", type=int, default=64)
    ap.add_argument("--c2-scale", type=float, default=1.0, help="photon-count scale of the batched sweep")
    ap.add_argument("--no-c3", dest="c3", action="store_false", help="skip the perturbation-MC gradient measurement")
    ap.add_argument("--c3-packets", type=float, default=1e8)
    ap.add_argument("--c3-grid", type=int, default=256)
    ap.add_argument("--no-c4", dest="c4", action="store_false", help="skip the heat-adjoint measurement")
    ap.add_argument("--c4-steps", type=int, default=2000)
    ap.add_argument("--lbfgs", action="store_true", help="also run the L-BFGS recovery (about 80 s at 256^3, 1e8 packets)")
    ap.add_argument("--c4-cpu-steps", type=int, default=10, help="time steps of the CPU reference on the 300x300x200 grid")
    ap.add_argument("--profile", choices=["heat-c1", "heat-c4", "mc-c0"], default=None,
                    help="run one workload briefly for a profiler capture instead of the benchmark")
    ap.add_argument("--packets", type=float, default=1e5, help="packets of the mc-c0 profile run")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.profile:
        run_profile(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
