#!/usr/bin/env python
"""Benchmark of the B200 DIVA velocity solver.

Metric: DIVA solves/s at 321 x 561 x 15 to rel-res 1e-6, learned + FP32 vs plain FP64 GPU:
cold-start DIVA + SIA solves of synthetic ice caps (1600 x 2800 km at 5 km, 15 layers), each
run to a relative nonlinear residual of 1e-6.  Before the timed region the warm-start network
is trained on plain FP64 solutions of --members seeded caps (seeds 0..) by the library's own
tcgen05 kernels; timed step k solves held-out cap HELD_OUT_SEEDS[k] (seeds from 10000 on).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload ...]

One process per GPU (torchrun for N > 1).  A single solve does not shard: each rank runs an
independent replica of the workload, so per-GPU work is fixed as N grows ("scaling": "weak")
and there is no data-path collective; the only collectives are the timing barrier and the
max over ranks.

value : learned-path solves/s of the whole job -- network warm start (prediction plus 10
        state-completion sweeps), FP32 finest-level smoother inside the FP64 BiCGStab,
        Anderson mixing of the viscosity iteration -- device-timed with CUDA events on the
        solve's stream around predict + solve + SIA, inputs resident in HBM.  The plain FP64
        path (the reference's relaxed Picard update) on the same geometries is reported in
        config as the denominator of the learned + FP32 vs plain FP64 ratio.
e2e   : the learned path through the public API with host buffers: every step uploads the
        geometry's inputs and the cold-start state from pinned host memory, prepares them on
        the GPU (update_general_ice_model_data, rheology), predicts, solves, computes the SIA
        velocities and downloads the velocity fields.
--impl reference : the CPU port of the reference path on the host threads, one full cold
        solve of the same geometries per step.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))


def load_package():
    import importlib.util
    if "imau_ice_b200" in sys.modules:
        return sys.modules["imau_ice_b200"]
    d = os.path.join(ROOT, "imau-ice_b200")
    spec = importlib.util.spec_from_file_location("imau_ice_b200", os.path.join(d, "__init__.py"),
                                                  submodule_search_locations=[d])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["imau_ice_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


METRIC = "DIVA solves/s at 321x561x15 to rel-res 1e-6"
UNIT = "solves/s"
INPUT_FIELDS = ["Hi_a", "Hb_a", "SL_a", "dHb_dt_a", "Ti_a", "beta_sq_a"]
STATE_FIELDS = ["u_vav_cx", "v_vav_cy", "visc_eff_3D_a", "taub_cx", "taub_cy", "u_3D_a", "v_3D_a"]
OUTPUT_FIELDS = ["u_vav_cx", "v_vav_cy", "u_3D_cx", "v_3D_cy", "w_3D_a", "u_3D_SIA_cx", "v_3D_SIA_cy"]
KERNEL_NAMES = {0: "K1 column coefficients (all launches of one viscosity iteration)",
                1: "k_smooth_down+k_smooth_up (fine level)", 2: "k_matvec",
                3: "V-cycle (all levels)", 4: "k_subcycle (coarse levels, one block)",
                5: "K1 column launches (without the b-grid faces)"}
# committed ncu summaries holding the DRAM bytes of one launch of each part
TRAFFIC_KEYS = {0: "k1_icecap321x561", 3: "vcycle_icecap321x561"}


def workload(seed=2, precision="fp64", anderson=0, eta=None, dx=None):
    """The ice cap, solved cold to rel-res 1e-6.  anderson = 0: the reference's relaxed
    Picard update with the adaptive linear tolerance 0.5 min(1, rel-res); anderson = m > 0:
    Anderson mixing of depth m, linear tolerance factor 0.1 unless eta is given."""
    from imau_ice_b200 import synth
    g, cfg, fields = synth.ice_cap(seed=seed, **({"dx": dx} if dx else {}))
    cfg = dict(cfg)
    cfg.update(picard_stop="relres", picard_relres_tol=1e-6, DIVA_visc_it_nit=500, lin_adaptive=1, lin_rtol=1e-10,
               precision=precision, picard_anderson_m=anderson,
               lin_adaptive_eta=eta if eta is not None else (0.1 if anderson else 0.5))
    return g, cfg, fields


def nonlinear_json(cfg):
    m = cfg.get("picard_anderson_m", 0)
    it = (f"Anderson mixing of depth {m} on the unrelaxed Picard map" if m else
          f"the reference's relaxed Picard update (relax {cfg.get('DIVA_visc_it_relax', 0.4)})")
    return {"nonlinear_iteration": it,
            "linear_solver": "BiCGStab + geometric multigrid V(2,2), adaptive tolerance "
                             f"{cfg['lin_adaptive_eta']:g} min(1, rel-res)"}


def config_json(g, extra=None):
    c = {"workload": "DIVA+SIA cold-start solve, synthetic ice cap 1600x2800 km @5 km",
         "nx": g["nx"], "ny": g["ny"], "nz": len(g["zeta"]), "stop": "nonlinear rel-res <= 1e-6",
         "l2": "inputs larger than L2: each step is a whole solve over ~0.6 GB of device state; the 3D "
               "fields (21.6 MB each) stream from HBM every viscosity iteration, the 2D multigrid "
               "levels (~17 MB at level 0) stay L2-resident within a solve; no flush"}
    c.update(extra or {})
    return c


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def read_traffic(kernel_key):
    """dram bytes per launch of a kernel from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", f"{kernel_key}.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.strip().startswith("dram_bytes_per_launch_scaled:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_baseline(threads=None, seed=2, dx=None):
    """The oracle (a CPU port of the reference path) on the same workload: one full cold
    solve to rel-res 1e-6 plus the SIA velocities, timed.  Linear solves: GMRES(30) +
    ILU(0) from the current iterate, right-preconditioned so that it tests the true
    residual, with the same adaptive tolerance rule as the GPU path; with T > 1 host
    threads the ILU(0) is block-Jacobi over T row blocks (what PETSc uses on T ranks)
    and the viscosity columns are split over the threads."""
    threads = min(threads or host_threads(), 64)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_backend
    from imau_ice_b200 import diva
    orc = oracle_backend.oracle_backend()
    g, cfg, fields = workload(seed=seed, dx=dx)
    grid = diva.Grid(**g)
    ctx = diva.Context(grid, cfg, orc)
    oracle_backend.set_linear_solver(ctx, oracle_backend.LIN_GMRES_WARM, rtol=1e-10, abstol=0.0)
    oracle_backend.set_threads(ctx, threads)
    ctx.upload(fields)
    ctx.update_general_ice_model_data()
    ctx.calc_pressure_melting_point()
    ctx.calc_ice_rheology()
    ctx.update_general_ice_model_data()
    t0 = time.perf_counter()
    rep = ctx.solve_DIVA()
    ctx.calc_sia_3d_velocities()
    t = time.perf_counter() - t0
    ctx.close()
    return {"value": 1.0 / t, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": (f"one full cold solve of ice cap seed {seed} at 321x561x15 to rel-res {rep['relres']:.2e} "
                       f"({rep['picard_iterations']} viscosity iterations, {rep['linear_iterations']} GMRES "
                       f"iterations) plus SIA, {t:.1f} s on {threads} threads")}


def run_cpu_variants(args):
    """The CPU port's variants of the linear solve on the ice cap (321 x 561 x 15), each one
    full cold solve_DIVA plus SIA on the host threads: (i) the reference's defaults (Picard
    step-norm tolerance 1e-2, at most 50 viscosity iterations, PETSc KSP rtol 1e-2 / abstol
    2.5, petsc_module.F90:49-69), (ii) the configuration's tolerances (step norm 1e-3, linear
    1e-8), (iii) SOR as utilities_module.f90:644-718 (omega 1.3, max |res/diag| <= 2.5,
    sweep cap 10000; one thread, it is sequential) at the configuration's step-norm tolerance,
    and (iv) the bench's rel-res 1e-6 stop with the adaptive tolerance (the cpu_baseline leg).
    Reported only: one JSON line with each variant's time, iterations and final rel-res."""
    load_package()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_backend as ob
    from imau_ice_b200 import diva
    threads = min(host_threads(), 64)
    orc = ob.oracle_backend()
    g, base, fields = workload()
    grid = diva.Grid(**g)
    ref_stop = dict(base, picard_stop="resid_UV", lin_adaptive=0)
    variants = {
        "reference_defaults_gmres": (dict(ref_stop, DIVA_visc_it_norm_dUV_tol=1e-2, DIVA_visc_it_nit=50),
                                     (ob.LIN_GMRES_WARM, 1e-2, 2.5), threads),
        "config_tolerances_gmres": (dict(ref_stop, DIVA_visc_it_norm_dUV_tol=1e-3, DIVA_visc_it_nit=200,
                                         lin_rtol=1e-8), (ob.LIN_GMRES_WARM, 1e-8, 0.0), threads),
        "config_tolerances_sor": (dict(ref_stop, DIVA_visc_it_norm_dUV_tol=1e-3, DIVA_visc_it_nit=200),
                                  (ob.LIN_SOR, 0.0, 0.0), 1),
        "relres_1e-6_adaptive_gmres": (base, (ob.LIN_GMRES_WARM, 1e-10, 0.0), threads),
    }
    out = {}
    for name, (cfg, solver, thr) in variants.items():
        ctx = diva.Context(grid, cfg, orc)
        if solver[0] == ob.LIN_SOR:
            ob.set_linear_solver(ctx, ob.LIN_SOR, sor_nit=10000, sor_tol=2.5, sor_omega=1.3)
        else:
            ob.set_linear_solver(ctx, solver[0], rtol=solver[1], abstol=solver[2])
        ob.set_threads(ctx, thr)
        ctx.upload(fields)
        ctx.update_general_ice_model_data()
        ctx.calc_pressure_melting_point()
        ctx.calc_ice_rheology()
        ctx.update_general_ice_model_data()
        t0 = time.perf_counter()
        rep = ctx.solve_DIVA()
        ctx.calc_sia_3d_velocities()
        t = time.perf_counter() - t0
        rr = ctx.nonlinear_residual()
        ctx.close()
        out[name] = {"seconds": round(t, 3), "solves_per_s": 1.0 / t, "threads": thr,
                     "viscosity_iterations": rep["picard_iterations"], "linear_iterations": rep["linear_iterations"],
                     "status": rep["status"], "final_relres": rr}
        print(name, out[name], file=sys.stderr, flush=True)
    print(json.dumps({"workload": "CPU port variants, synthetic ice cap 321x561x15, one cold solve_DIVA + SIA each",
                      "host_threads": threads, "variants": out}))
    return 0


def run_cnn(args):
    """The warm-start network's tensor-core kernels alone at the headline grid: one forward
    pass (inference) and one training step (forward, dgrad, wgrad, Adam) on a batch of 8
    321 x 561 samples, device-synchronised wall clock per call (each call synchronises).
    FLOPs: 2 x 9 x Cin x Cout per pixel of each 3x3 convolution at its level's resolution
    (175 kFLOP per pixel of the padded grid forward; a training step counts three times
    the forward's convolution FLOPs); the tensor roofline is the measured dense BF16 GEMM
    rate (MEASURED_PEAKS.json)."""
    import numpy as np
    import torch
    load_package()
    from imau_ice_b200 import build, diva, learned
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    build.build()
    g = headline_case(0, True)[0]
    grid = diva.Grid(**g)
    batch = 8
    net = learned.WarmStartNet(grid, batch=batch, capacity=0, seed=0)
    Hp, Wp = net.padded_shape
    rng = np.random.default_rng(0)
    feat = torch.as_tensor(rng.normal(0, 1, (batch, Hp, Wp, learned.IN_C)).astype(np.float32)).to(torch.bfloat16).cuda()
    tgt = torch.as_tensor(rng.normal(0, 1, (batch, Hp, Wp, learned.N_OUT)).astype(np.float32)).cuda()
    out = torch.zeros(batch, Hp, Wp, learned.N_OUT, device="cuda")
    level_px = [Hp * Wp, (Hp // 2) * (Wp // 2), (Hp // 4) * (Wp // 4)]
    lvl = {"e1a": 0, "e1b": 0, "e2a": 1, "e2b": 1, "ba": 2, "bb": 2, "d2a": 1, "d2b": 1, "d1a": 0, "d1b": 0}
    flop_fwd = batch * sum(2.0 * 9 * ci * co * level_px[lvl[name]] for name, ci, co in learned.LAYERS)

    def timed(fn, reps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / reps

    t_fwd = timed(lambda: net.forward(feat.data_ptr(), out.data_ptr(), batch), args.steps)
    t_train = timed(lambda: net.train_step(feat.data_ptr(), tgt.data_ptr(), batch, 1e-4), args.steps)
    try:
        peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops"]
        src = "measured (MEASURED_PEAKS.json bf16_tflops)"
    except Exception:
        peak, src = 1590.0, "fallback 1590 TFLOP/s"
    fwd_tf = flop_fwd / t_fwd / 1e12
    train_tf = 3 * flop_fwd / t_train / 1e12
    print(json.dumps({
        "metric": "warm-start network forward passes/s (batch of 8 samples of 321x561)", "value": 1.0 / t_fwd,
        "unit": "passes/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * t_fwd,
        "higher_is_better": True, "dtype": "bf16 (fp32 accumulation)", "data": "synthetic (random features)",
        "config": {"workload": "U-Net of 10 3x3 convolutions (16-128 channels) on the padded a-grid "
                               f"{Hp}x{Wp}, batch {batch}", "training_step_ms": 1000 * t_train,
                   "training_steps_per_s": 1.0 / t_train,
                   "timing": "device-synchronised wall clock per call"},
        "roofline": {"bound": "tensor", "kernel": "k_conv3x3 (all convolutions of one pass)",
                     "achieved": fwd_tf, "peak": peak, "unit": "TFLOP/s", "frac": fwd_tf / peak,
                     "flop_per_pass": flop_fwd, "peak_source": src,
                     "training_step": {"achieved": train_tf, "frac": train_tf / peak}}}))
    net.close()
    return 0


def run_reference(args):
    """The reference arm: the CPU port of the reference path (relaxed Picard update, GMRES +
    ILU(0)) on all host threads, one full cold solve per step of the same workload as the
    default line (the headline: held-out ice-cap seed 10000 + k at step k; --workload icecap:
    the fixed seed-2 cap).  Warm-up steps solve the 40 km ice cap (81 x 141) so they stay
    short.  Rank 0 alone runs and prints."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    load_package()
    headline = args.workload == "headline"
    g, _, _ = workload()
    secs = []
    threads = min(host_threads(), 64)
    for _ in range(args.warmup):
        cpu_baseline(threads, seed=2, dx=40e3)
    last = None
    for k in range(args.steps):
        last = cpu_baseline(threads, seed=held_out_seed(k) if headline else 2)
        secs.append(1.0 / last["value"])
    v = args.steps / sum(secs)
    out = {"metric": HEADLINE_METRIC if headline else METRIC, "value": v, "unit": UNIT, "impl": "reference",
           "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / v, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded ice cap)",
           "config": config_json(g, {**({"workload": "DIVA+SIA cold-start solves of held-out synthetic ice caps "
                                                     "1600x2800 km @5 km, one geometry per step",
                                         "seeds": [held_out_seed(k) for k in range(args.steps)]} if headline else {}),
                                     "parallelism": f"CPU oracle port on {threads} host threads (block-Jacobi "
                                                     f"ILU(0) over {threads} row blocks, column loops split)",
                                     "nonlinear_iteration": "the reference's relaxed Picard update (relax 0.4)",
                                     "linear_solver": "GMRES(30) + ILU(0) from the current iterate, adaptive "
                                                      "tolerance 0.5 min(1, rel-res)"}),
           "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                            "sample": ("each step one full cold solve of the step's geometry (the first "
                                       f"{args.steps} held-out ice-cap seeds of the list)" if headline else "each step " +
                                       last["sample"])},
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def run_b200(args):
    import numpy as np
    import torch
    import torch.distributed as dist
    load_package()
    from imau_ice_b200 import build, diva

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    build.build()

    g, cfg, fields = workload(precision=args.precision, anderson=args.anderson, eta=args.eta)
    grid = diva.Grid(**g)
    ctx = diva.Context(grid, cfg)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    ctx.upload(fields)
    ctx.update_general_ice_model_data()
    ctx.calc_pressure_melting_point()
    ctx.calc_ice_rheology()
    ctx.update_general_ice_model_data()
    ctx.state_save()

    def step():
        ctx.state_restore()          # cold start: the initial state of the solve, a device copy
        r = ctx.solve_DIVA()
        ctx.calc_sia_3d_velocities()
        return r

    for _ in range(args.warmup):
        step()
    clocks = ClockSampler(local)
    if not args.quick:            # no NVML polling while a profiler owns the counters
        clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = ctx.kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    reps = [step() for _ in range(args.steps)]
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop() if not args.quick else {}
    launches = ctx.kernel_launches() - l0
    ms = e0.elapsed_time(e1)
    if args.quick:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": world * args.steps / (ms / 1000.0), "unit": UNIT,
                              "quick": True, "gpu_launches": int(launches), "reports": reps}))
        ctx.close()
        if world > 1:
            dist.destroy_process_group()
        return 0
    t = torch.tensor([ms], device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * args.steps / (ms_max / 1000.0)
    picard = [r["picard_iterations"] for r in reps]
    mg = [r["mg_cycles"] for r in reps]

    # roofline of the dominant part of the solve, by device time per solve = time per launch
    # (CUDA events on the solve's stream, the part run alone on the converged state) x launches
    # per solve.  Candidates: the column coefficients K1 (four launches per viscosity iteration,
    # 480 B per column: (3 nz + 15) x 8) and one multigrid V-cycle (all levels; per level the
    # smoothing sweeps, residual and transfers, weighted by its points); sub-parts of the
    # V-cycle ride along in other_kernels.
    prof = {}
    for which in (0, 1, 2, 3, 4, 5):
        prof[which] = ctx.profile_kernel(which, reps=30 if which else 10)
    per_solve = {0: prof[0][0] * statistics.mean(picard), 3: prof[3][0] * statistics.mean(mg)}
    dom = max(per_solve, key=per_solve.get)
    ms_l, bytes_l = prof[dom]
    hbm_peak = None
    peak_src = "fallback 6650 GB/s"
    try:
        hbm_peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
        peak_src = "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        hbm_peak = 6650.0
    achieved = bytes_l / (ms_l * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": KERNEL_NAMES[dom], "achieved": achieved, "peak": hbm_peak,
                "unit": "GB/s", "frac": achieved / hbm_peak, "traffic": read_traffic(TRAFFIC_KEYS[dom]),
                "peak_source": peak_src, "algorithmic_bytes_per_launch": bytes_l, "ms_per_launch": ms_l,
                "launches_per_solve": statistics.mean(picard) if dom == 0 else statistics.mean(mg),
                "other_kernels": {KERNEL_NAMES[w]: {"ms_per_launch": prof[w][0], "algorithmic_bytes": prof[w][1],
                                                    "GB/s": prof[w][1] / (prof[w][0] * 1e-3) / 1e9}
                                  for w in prof},
                "ms_per_solve": {KERNEL_NAMES[w]: per_solve[w] for w in per_solve}}

    # end to end through the public API with pinned host buffers
    def pinned(a):
        t_ = torch.empty(a.shape[::-1], dtype=torch.float64 if a.dtype == np.float64 else torch.int32,
                         pin_memory=True)
        h = t_.numpy().T            # Fortran-ordered view of the pinned buffer
        h[...] = a
        return h, t_

    keep = []
    host_in = {}
    for n in INPUT_FIELDS:
        h, t_ = pinned(np.asarray(fields[n]))
        host_in[n] = h
        keep.append(t_)
    for n in STATE_FIELDS:
        h, t_ = pinned(ctx.empty(n))
        host_in[n] = h
        keep.append(t_)
    h2d = sum(a.nbytes for a in host_in.values())
    host_out = {}
    for n in OUTPUT_FIELDS:
        h, t_ = pinned(ctx.empty(n))
        host_out[n] = h
        keep.append(t_)
    e2e_steps = args.steps

    def e2e_step():
        ctx.upload(host_in)
        ctx.update_general_ice_model_data()
        ctx.calc_pressure_melting_point()
        ctx.calc_ice_rheology()
        ctx.update_general_ice_model_data()
        ctx.solve_DIVA()
        ctx.calc_sia_3d_velocities()
        return ctx.download(OUTPUT_FIELDS, out=host_out)

    out = e2e_step()
    d2h = sum(a.nbytes for a in out.values())
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    torch.cuda.synchronize()
    te = torch.tensor([time.perf_counter() - t0], device="cuda")
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
        dist.barrier()
    e2e_val = world * e2e_steps / float(te.item())

    if rank == 0:
        res = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded ice cap)",
               "config": config_json(g, {"parallelism": f"replicas x{world} (a single solve does not shard)",
                                         "precision": args.precision, **nonlinear_json(cfg),
                                         "picard_iterations": picard, "mg_cycles": mg,
                                         "relres": [r["relres"] for r in reps]}),
               "roofline": roofline, "clocks": clk,
               "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                       "timing": "host wall clock with device synchronisation, max over ranks"},
               "gpu_launches": int(launches)}
        if not args.no_cpu_baseline:
            try:
                res["cpu_baseline"] = cpu_baseline()
            except Exception as ex:   # the baseline is reported, never required
                res["cpu_baseline"] = {"value": None, "unit": UNIT, "error": str(ex)[:200]}
        print(json.dumps(res))
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


HEADLINE_METRIC = "DIVA solves/s at 321x561x15 to rel-res 1e-6: learned+FP32 vs plain FP64 GPU"


# Held-out ice caps of the headline line: the seeds from 10000 on whose plain FP64 solve
# reaches rel-res 1e-6 within 500 viscosity iterations.  Of seeds 10000-10099, 29 do not:
# their fastest ice runs into the reference's 5000 m/yr velocity limit (apply_velocity_limits,
# ice_velocity_module.f90:1432-1498), and the fixed point of the limited iteration does not
# solve the unlimited equations, so no method reaches rel-res 1e-6 there.  The list was taken
# from one scan of those 100 seeds with the plain FP64 path on a B200 (76-267 iterations for
# the 71 that converge) and is fixed here, so both arms of the bench time the same geometries.
HELD_OUT_SEEDS = [
    10000, 10001, 10002, 10003, 10004, 10005, 10010, 10011, 10012, 10014, 10015, 10016, 10017, 10018,
    10019, 10021, 10023, 10024, 10026, 10027, 10028, 10029, 10031, 10034, 10036, 10038, 10040, 10041,
    10042, 10043, 10049, 10050, 10051, 10052, 10053, 10054, 10056, 10057, 10058, 10059, 10060, 10061,
    10062, 10063, 10064, 10065, 10066, 10067, 10068, 10069, 10070, 10071, 10073, 10074, 10079, 10080,
    10081, 10083, 10084, 10085, 10086, 10088, 10089, 10090, 10091, 10093, 10094, 10096, 10097, 10098,
    10099]


def held_out_seed(k):
    """Geometry of timed step k: held-out ice caps, never in the training set (seeds 0..)."""
    return HELD_OUT_SEEDS[k % len(HELD_OUT_SEEDS)]


def headline_case(seed, learned_path, anderson=3, eta=0.1):
    """The seeded ice cap and its solve settings: the learned path (FP32 smoother, Anderson
    mixing, tighter adaptive linear tolerance) or the plain FP64 path (the reference's
    relaxed Picard update)."""
    from imau_ice_b200 import synth
    g, cfg, f = synth.ice_cap(seed=seed)
    cfg = dict(cfg, picard_stop="relres", picard_relres_tol=1e-6, DIVA_visc_it_nit=500, lin_adaptive=1,
               lin_rtol=1e-10)
    if learned_path:
        cfg.update(precision="mixed", picard_anderson_m=anderson, lin_adaptive_eta=eta)
    else:
        cfg.update(precision="fp64", picard_anderson_m=0, lin_adaptive_eta=0.5)
    return g, cfg, f


def train_warm_start(grid, members, epochs):
    """The warm-start network trained on `members` plain FP64 solutions (seeds 0..) by the
    library's own tcgen05 forward and backward kernels; returns (net, loss, seconds)."""
    from imau_ice_b200 import diva, learned
    net = learned.WarmStartNet(grid, batch=8, capacity=members, seed=0)
    net.velocities_only()                  # predict completes the rest of the state
    t0 = time.perf_counter()
    seed = 0
    while net.num_samples < members and seed < 4 * members:
        g, cfg, f = headline_case(seed, False)
        ctx = diva.Context(diva.Grid(**g), cfg)
        ctx.upload(f)
        ctx.update_general_ice_model_data()
        ctx.calc_pressure_melting_point()
        ctx.calc_ice_rheology()
        ctx.update_general_ice_model_data()
        if ctx.solve_DIVA()["status"] == 0:
            net.add_sample(ctx)
        ctx.close()
        seed += 1
    t_data = time.perf_counter() - t0
    t0 = time.perf_counter()
    loss = net.train(epochs, lr=1e-3, seed=1)
    return net, loss, t_data, time.perf_counter() - t0


def train_member_net(kind, samples, epochs):
    """A warm-start network for the ensemble's members of one size: trained, by the library's
    tcgen05 kernels, on plain FP64 solutions of that size's generator at seeds 0.. (the
    ensemble's members use seeds 1000 and up), with friction and flow factors drawn from
    the ensemble's distributions.  Returns (net, loss, data seconds, training seconds)."""
    import numpy as np
    from imau_ice_b200 import diva, learned, synth
    gen = {"channel": synth.marine_channel, "icecap": synth.ice_cap}[kind]
    grid = diva.Grid(**gen(seed=0)[0])
    net = learned.WarmStartNet(grid, batch=8, capacity=samples, seed=0)
    net.velocities_only()
    rng = np.random.default_rng(7)
    t0 = time.perf_counter()
    seed = 0
    while net.num_samples < samples and seed < 4 * samples:
        g, cfg, f = gen(seed=seed)
        fb = float(np.exp(rng.uniform(np.log(0.3), np.log(3.0))))
        fa = float(np.exp(rng.uniform(np.log(0.5), np.log(2.0))))
        f = dict(f)
        if "beta_sq_a" in f:
            f["beta_sq_a"] = np.asfortranarray(f["beta_sq_a"] * fb)
        cfg = dict(cfg, m_enh_sheet=fa, m_enh_shelf=fa, picard_stop="relres", picard_relres_tol=1e-6,
                   DIVA_visc_it_nit=500, lin_adaptive=1, lin_rtol=1e-10, lin_adaptive_eta=0.5)
        ctx = diva.Context(diva.Grid(**g), cfg)
        ctx.upload(f)
        ctx.update_general_ice_model_data()
        ctx.calc_pressure_melting_point()
        ctx.calc_ice_rheology()
        ctx.update_general_ice_model_data()
        try:
            if ctx.solve_DIVA()["status"] == 0:
                net.add_sample(ctx)
        except diva.DivaError:
            pass
        ctx.close()
        seed += 1
    t_data = time.perf_counter() - t0
    t0 = time.perf_counter()
    loss = net.train(epochs, lr=1e-3, seed=1)
    return net, loss, t_data, time.perf_counter() - t0


def run_headline(args):
    """The headline line: DIVA + SIA solves of held-out 321 x 561 x 15 ice caps to rel-res
    1e-6 through the learned path (network warm start, FP32 finest-level smoother, Anderson
    mixing), with the plain FP64 GPU path on the same geometries as its denominator.
    value: learned-path solves/s, device-timed with CUDA events around predict + solve +
    SIA on the solve's stream (inputs resident); e2e: the same through the public API with
    host buffers (upload, data-model update, predict, solve, SIA, download)."""
    import numpy as np
    import torch
    import torch.distributed as dist
    load_package()
    from imau_ice_b200 import build, diva

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    build.build()
    g0 = headline_case(0, True)[0]
    grid = diva.Grid(**g0)
    net, loss, t_data, t_train = train_warm_start(grid, args.members, args.epochs)
    stream = torch.cuda.Stream()

    def prepared(seed, learned_path):
        g, cfg, f = headline_case(seed, learned_path, args.anderson or 3, args.eta or 0.1)
        ctx = diva.Context(grid, cfg)
        ctx.set_stream(stream.cuda_stream)
        ctx.upload(f)
        ctx.update_general_ice_model_data()
        ctx.calc_pressure_melting_point()
        ctx.calc_ice_rheology()
        ctx.update_general_ice_model_data()
        return ctx

    def device_solve(seed, learned_path, keep=False):
        ctx = prepared(seed, learned_path)
        torch.cuda.synchronize()
        l0 = ctx.kernel_launches()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        if learned_path:
            net.predict(ctx, complete_sweeps=10)
        try:
            rep = ctx.solve_DIVA()
        except diva.DivaError as e:
            rep = {"status": e.status, "picard_iterations": -1, "mg_cycles": -1, "relres": -1.0}
        ctx.calc_sia_3d_velocities()
        e1.record(stream)
        torch.cuda.synchronize()
        launches = ctx.kernel_launches() - l0
        if keep:
            return e0.elapsed_time(e1), rep, launches, ctx
        ctx.close()
        return e0.elapsed_time(e1), rep, launches

    for k in range(args.warmup):
        device_solve(20000 + k, True)
        device_solve(20000 + k, False)
    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    learned_runs = [device_solve(held_out_seed(k), True) for k in range(args.steps)]
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    plain_runs = [device_solve(held_out_seed(k), False) for k in range(args.steps)]
    t = torch.tensor([sum(r[0] for r in learned_runs), sum(r[0] for r in plain_runs)], device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_learned, ms_plain = float(t[0]), float(t[1])
    value = world * args.steps / (ms_learned / 1000.0)
    plain_value = world * args.steps / (ms_plain / 1000.0)

    # roofline: the dominant part of a learned-path solve, timed alone on its converged state
    _, rep_k, _, ctx = device_solve(held_out_seed(0), True, keep=True)
    prof = {w: ctx.profile_kernel(w, reps=30 if w else 10) for w in (0, 1, 2, 3, 4, 5)}
    ctx.close()
    its = statistics.mean(r[1]["picard_iterations"] for r in learned_runs)
    cyc = statistics.mean(r[1]["mg_cycles"] for r in learned_runs)
    per_solve = {0: prof[0][0] * its, 3: prof[3][0] * cyc}
    dom = max(per_solve, key=per_solve.get)
    ms_l, bytes_l = prof[dom]
    try:
        hbm_peak, peak_src = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"], \
            "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        hbm_peak, peak_src = 6650.0, "fallback 6650 GB/s"
    achieved = bytes_l / (ms_l * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": KERNEL_NAMES[dom], "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved / hbm_peak, "traffic": read_traffic(TRAFFIC_KEYS[dom]), "peak_source": peak_src,
                "algorithmic_bytes_per_launch": bytes_l, "ms_per_launch": ms_l,
                "launches_per_solve": its if dom == 0 else cyc,
                "other_kernels": {KERNEL_NAMES[w]: {"ms_per_launch": prof[w][0], "algorithmic_bytes": prof[w][1],
                                                    "GB/s": prof[w][1] / (prof[w][0] * 1e-3) / 1e9} for w in prof},
                "ms_per_solve": {KERNEL_NAMES[w]: per_solve[w] for w in per_solve}}

    # end to end through the public API: pinned host inputs of every step's geometry, the
    # cold-start state, and pinned outputs
    def pinned(a):
        t_ = torch.empty(a.shape[::-1], dtype=torch.float64 if a.dtype == np.float64 else torch.int32,
                         pin_memory=True)
        h = t_.numpy().T
        h[...] = a
        return h, t_

    keep = []
    host_inputs = []
    for k in range(args.steps):
        f = headline_case(held_out_seed(k), True)[2]
        hk = {}
        for n in INPUT_FIELDS:
            h, t_ = pinned(np.asarray(f[n]))
            hk[n] = h
            keep.append(t_)
        host_inputs.append(hk)
    ectx = prepared(held_out_seed(0), True)
    host_state, host_out = {}, {}
    for n in STATE_FIELDS:
        h, t_ = pinned(np.zeros_like(ectx.empty(n)))
        host_state[n] = h
        keep.append(t_)
    for n in OUTPUT_FIELDS:
        h, t_ = pinned(ectx.empty(n))
        host_out[n] = h
        keep.append(t_)
    h2d = sum(a.nbytes for a in host_inputs[0].values()) + sum(a.nbytes for a in host_state.values())
    d2h = sum(a.nbytes for a in host_out.values())

    def e2e_step(k):
        ectx.upload(host_inputs[k])
        ectx.upload(host_state)
        ectx.update_general_ice_model_data()
        ectx.calc_pressure_melting_point()
        ectx.calc_ice_rheology()
        ectx.update_general_ice_model_data()
        net.predict(ectx, complete_sweeps=10)
        try:
            ectx.solve_DIVA()
        except diva.DivaError:
            pass
        ectx.calc_sia_3d_velocities()
        return ectx.download(OUTPUT_FIELDS, out=host_out)

    e2e_step(0)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(args.steps):
        e2e_step(k)
    torch.cuda.synchronize()
    te = torch.tensor([time.perf_counter() - t0], device="cuda")
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
        dist.barrier()
    e2e_val = world * args.steps / float(te.item())
    ectx.close()

    if rank == 0:
        res = {"metric": HEADLINE_METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms_learned / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
               "data": "synthetic (seeded ice caps; network trained on seeds 0.., timed on held-out seeds 10000..)",
               "config": {
                   "workload": "DIVA+SIA cold-start solves of held-out synthetic ice caps 1600x2800 km @5 km, "
                               "one geometry per step",
                   "nx": grid.nx, "ny": grid.ny, "nz": grid.nz, "stop": "nonlinear rel-res <= 1e-6",
                   "learned_path": "warm start by the trained network (10 state-completion sweeps), FP32 "
                                   "finest-level smoother in the FP64 BiCGStab, Anderson mixing of depth "
                                   f"{args.anderson or 3}, adaptive linear tolerance {args.eta or 0.1:g} min(1, rel-res)",
                   "plain_path": "FP64 throughout, the reference's relaxed Picard update (relax 0.4), adaptive "
                                 "linear tolerance 0.5 min(1, rel-res)",
                   "plain_fp64_solves_per_s": plain_value,
                   "ratio_learned_vs_plain_fp64": value / plain_value,
                   "seeds": [held_out_seed(k) for k in range(args.steps)],
                   "iterations_learned": [r[1]["picard_iterations"] for r in learned_runs],
                   "iterations_plain": [r[1]["picard_iterations"] for r in plain_runs],
                   "mg_cycles_learned": [r[1]["mg_cycles"] for r in learned_runs],
                   "mg_cycles_plain": [r[1]["mg_cycles"] for r in plain_runs],
                   "status_learned": [r[1]["status"] for r in learned_runs],
                   "relres_learned": [r[1]["relres"] for r in learned_runs],
                   "training": {"samples": net.num_samples, "epochs": args.epochs, "final_loss": loss,
                                "data_generation_s": round(t_data, 2), "training_s": round(t_train, 2)},
                   "parallelism": f"replicas x{world} (a single solve does not shard)",
                   "l2": "inputs larger than L2: each step is a whole solve over ~0.6 GB of device state; the 3D "
                         "fields (21.6 MB each) stream from HBM every viscosity iteration, the 2D multigrid "
                         "levels (~17 MB at level 0) stay L2-resident within a solve; no flush"},
               "roofline": roofline, "clocks": clk,
               "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                       "timing": "host wall clock with device synchronisation, max over ranks"},
               "gpu_launches": int(sum(r[2] for r in learned_runs))}
        if not args.no_cpu_baseline:
            try:
                res["cpu_baseline"] = cpu_baseline(seed=held_out_seed(0))
            except Exception as ex:   # the baseline is reported, never required
                res["cpu_baseline"] = {"value": None, "unit": UNIT, "error": str(ex)[:200]}
        print(json.dumps(res))
    net.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_ensemble(args):
    """Ensemble workload: ``--members`` seeded members (sizes from ``--ensemble-sizes``,
    friction and flow factor perturbed), partitioned over the ranks by expected cost.  Each
    rank splits its share into groups that fit in device memory; per group the contexts are
    prepared (untimed), then warm-up and timed batched solves run, each from the prepared
    cold state.  Solves/s of the whole ensemble: members x steps over the max over ranks of
    the per-rank sum of the groups' device-synchronised wall times."""
    import numpy as np
    import torch
    import torch.distributed as dist
    load_package()
    from imau_ice_b200 import build, diva, ensemble, synth
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    build.build()
    sizes = tuple(args.ensemble_sizes.split(","))
    members = synth.ensemble(n=args.members, seed=0, sizes=sizes)
    parts = ensemble.partition([ensemble.member_cost(m) for m in members], world)
    budget = 0.7 * torch.cuda.mem_get_info()[0]
    clocks = ClockSampler(local)
    clocks.start()
    t_total, launches, last, group_seconds = 0.0, 0, {}, []
    fp64_err = {}
    nets, net_info = {}, {}
    if args.learned:
        # one network per member size; the 1501 x 1501 sheet has none (one training sample
        # of it is ~250 MB of device memory), its members start cold
        for kind in sizes:
            if kind == "sheet":
                net_info[kind] = "none: members start cold"
                continue
            net, loss, t_data, t_train = train_member_net(kind, args.learned_samples, args.epochs)
            nets[kind] = net
            net_info[kind] = {"samples": net.num_samples, "epochs": args.epochs, "final_loss": loss,
                              "data_generation_s": round(t_data, 2), "training_s": round(t_train, 2)}

    def member_cfg(cfg, accelerated=True, kind=None):
        cfg = dict(cfg, picard_stop="relres", picard_relres_tol=1e-6, DIVA_visc_it_nit=500, lin_adaptive=1,
                   lin_rtol=1e-10, picard_stall_its=args.stall_its, lin_maxit=args.lin_maxit)
        if accelerated:
            m = args.anderson_sheet if (kind == "sheet" and args.anderson_sheet is not None) else args.anderson
            cfg.update(picard_anderson_m=m, precision=args.precision,
                       lin_adaptive_eta=args.eta if args.eta is not None else (0.1 if m else 0.5))
        return cfg

    for grp in ensemble.groups(members, parts[rank], budget):
        ctxs = []
        for k in grp:
            name, g, cfg, f = members[k]
            cfg = member_cfg(cfg, kind=name.split("-")[0])
            c = diva.Context(diva.Grid(**g) if isinstance(g, dict) else g, cfg)
            c.upload(f)
            c.update_general_ice_model_data()
            c.calc_pressure_melting_point()
            c.calc_ice_rheology()
            c.update_general_ice_model_data()
            c.state_save()
            ctxs.append(c)

        batch = diva.Batch(ctxs)   # every member's viscosity loop in one graph, captured once
        kinds_grp = [members[k][0].split("-")[0] for k in grp]

        def step():
            for c, kind in zip(ctxs, kinds_grp):
                c.state_restore()
                if kind in nets:   # the warm start is part of the timed solve
                    nets[kind].predict(c, complete_sweeps=10)
            return batch.solve_DIVA(raise_on_error=False)

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        l0 = sum(c.kernel_launches() for c in ctxs)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            reps = step()
        torch.cuda.synchronize()
        group_seconds.append((time.perf_counter() - t0) / args.steps)
        t_total += time.perf_counter() - t0
        launches += sum(c.kernel_launches() for c in ctxs) - l0
        last.update({k: r for k, r in zip(grp, reps)})
        batch.close()
        if args.anderson or args.precision != "fp64":
            # each member's error against the plain FP64 path (untimed): the same member
            # solved again from its cold state with the reference's relaxation in FP64
            for k, c in zip(grp, ctxs):
                a = c.download(["u_vav_cx", "v_vav_cy"])
                c.set_config(member_cfg(members[k][2], accelerated=False))
                c.state_restore()
                try:
                    r64 = c.solve_DIVA()
                except diva.DivaError:
                    r64 = {"status": -1}
                b = c.download(["u_vav_cx", "v_vav_cy"])
                x = np.concatenate([a["u_vav_cx"].ravel(), a["v_vav_cy"].ravel()])
                y = np.concatenate([b["u_vav_cx"].ravel(), b["v_vav_cy"].ravel()])
                den = float(np.linalg.norm(y))
                fp64_err[k] = (float(np.linalg.norm(x - y)) / den if den > 0 else 0.0,
                               float(np.abs(x - y).max()), r64["status"])
        for c in ctxs:
            c.close()
    for net in nets.values():
        net.close()
    clk = clocks.stop()
    dt = torch.tensor([t_total], device="cuda")
    if world > 1:
        dist.all_reduce(dt, op=dist.ReduceOp.MAX)
    t_max = float(dt.item())
    its = [last[k]["picard_iterations"] for k in sorted(last)]
    cycles = [last[k]["mg_cycles"] for k in sorted(last)]
    member_ms = [round(last[k]["elapsed_ms"], 3) for k in sorted(last)]
    converged = sum(1 for k in last if last[k]["status"] == 0)
    stalled = sum(1 for k in last if last[k].get("stalled"))
    failed = {k: last[k]["status"] for k in sorted(last) if last[k]["status"] not in (0, 1)}
    # members that reached rel-res 1e-6 on both paths: the error the accelerated path leaves
    both = [fp64_err[k][0] for k in sorted(fp64_err) if last[k]["status"] == 0 and fp64_err[k][2] == 0]
    kinds = [members[k][0] for k in sorted(last)]
    if rank == 0:
        print(json.dumps({
            "metric": f"DIVA ensemble solves/s ({args.members} members) to rel-res 1e-6", "value":
            args.members * args.steps / t_max, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * t_max / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded ensemble)",
            "config": {"workload": f"{args.members}-member ensemble, sizes {'/'.join(sizes)}, beta_sq x "
                                   "U_log[0.3,3], flow factor x U_log[0.5,2]",
                       "members_per_rank": [len(p) for p in parts],
                       "member_kinds_rank0": kinds,
                       "picard_iterations_rank0": its,
                       "mg_cycles_rank0": cycles,
                       "member_stream_span_ms_rank0": member_ms,
                       "group_seconds_rank0": [round(x, 4) for x in group_seconds],
                       "rank0_members_converged": converged,
                       "rank0_members_stalled": stalled,
                       "rank0_members_at_iteration_cap": len(last) - converged - stalled - len(failed),
                       "rank0_members_failed": failed,
                       "solver": (f"Anderson({args.anderson}) " if args.anderson else "relaxed Picard ") +
                                 (f"(sheets: Anderson({args.anderson_sheet})) " if args.anderson_sheet else
                                  "(sheets: relaxed) " if args.anderson_sheet == 0 else "") +
                                 f"precision {args.precision}, stall window {args.stall_its} iterations" +
                                 (", learned warm start" if args.learned else ""),
                       "warm_start": net_info or None,
                       "error_vs_plain_fp64_summary": ({"members_both_converged": len(both),
                                                        "rel_l2_median": float(np.median(both)) if both else None,
                                                        "rel_l2_max": float(np.max(both)) if both else None}
                                                       if fp64_err else None),
                       "error_vs_plain_fp64_rank0": {"rel_l2": [round(fp64_err[k][0], 9) for k in sorted(fp64_err)],
                                                     "max_abs_m_per_yr": [round(fp64_err[k][1], 6)
                                                                          for k in sorted(fp64_err)],
                                                     "fp64_status": [fp64_err[k][2] for k in sorted(fp64_err)]}
                       if fp64_err else None,
                       "note": "members with low friction reach the 5000 m/yr velocity limit of the reference's "
                               "Picard update: the limited iteration settles on or cycles around states above "
                               "rel-res 1e-6; with a stall window they stop once rel-res has not fallen by 10 % "
                               "for that many iterations (status MAX_PICARD), without one at the cap",
                       "timing": "device-synchronised wall clock of the batched solves (per memory-bounded group "
                                 "one persistent graph holding every member's viscosity loop, one launch per "
                                 "solve), summed over the groups, max over ranks; a member's stream span is its "
                                 "events' span while it shares the GPU with the group's others",
                       "parallelism": f"members partitioned over {world} GPU(s), no data-path collective"},
            "clocks": clk, "gpu_launches": int(launches)}))
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_timestep(args):
    """Time-step workload: the ice cap (321 x 561 x 15) advanced by predictor/corrector
    steps with DIVA velocities, the explicit thickness update and the 3D heat equation,
    all resident on the device (host arithmetic only for the step control).  Each step
    is a warm-started solve from the previous step's state.  Metric: time steps/s,
    device-synchronised wall clock (the step control reads scalars on the host)."""
    import numpy as np
    import torch
    load_package()
    from imau_ice_b200 import build, diva, dynamics
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    build.build()
    g, cfg, fields = workload()
    cfg = dict(cfg, dt_thermo=0.05)
    grid = diva.Grid(**g)
    ctx = diva.Context(grid, cfg)
    ny, nx = fields["Hi_a"].shape
    f = dict(fields)
    f["SMB_a"] = np.asfortranarray(np.full((ny, nx), 0.2))
    f["T_surf_annual_a"] = np.asfortranarray(np.asarray(fields["Ti_a"])[0])
    f["GHF_a"] = np.asfortranarray(np.full((ny, nx), 1.7e6))
    ctx.upload(f)
    ctx.update_general_ice_model_data()
    ctx.calc_pressure_melting_point()
    ctx.calc_ice_rheology()
    ctx.update_general_ice_model_data()
    ctx.upload({"mask_ice_a_prev": ctx.download(["mask_ice_a"])["mask_ice_a"]})
    ctx.determine_floating_margin_fraction()
    pc = dynamics.PCTimeStepper(ctx, 0.0, 1e5, thermo=True)
    for _ in range(args.warmup):
        pc.step()
    n0, t_model0 = len(pc.reports), pc.time
    clocks = ClockSampler(0)
    clocks.start()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        pc.step()
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    clk = clocks.stop()
    its = [r["picard_iterations"] for r in pc.reports[n0:]]
    print(json.dumps({
        "metric": "ice-dynamics time steps/s at 321x561x15 (PC + DIVA + thickness + heat equation)",
        "value": args.steps / dt, "unit": "steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * dt / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded ice cap, SMB 0.2 m/yr, GHF 1.7e6 J/m2/yr)",
        "config": {"workload": "predictor/corrector time steps of the synthetic ice cap 1600x2800 km @5 km",
                   "viscosity_iterations_per_solve": its, "model_years": pc.time - t_model0,
                   "thermo_solves": pc.thermo_solves,
                   "timing": "device-synchronised wall clock around the host-controlled steps"},
        "clocks": clk}))
    ctx.close()
    return 0


def run_learned(args):
    """Learned warm start workload (the ice cap 321 x 561 x 15, seeded geometries):
    solve --members training caps (seeds 0..) with the plain FP64 path and keep them
    on the device, train the warm-start network on them, then time --steps held-out
    caps (seeds 10000..) both ways -- cold FP64, and network prediction + 10 state-
    completion sweeps + solve at --precision -- each to rel-res 1e-6.  value = learned
    solves/s; the cold FP64 rate and the iteration counts ride along.  Device-
    synchronised wall clock around each whole solve call (inputs already resident)."""
    import numpy as np
    import torch
    load_package()
    from imau_ice_b200 import build, diva, learned, synth
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    build.build()

    def case(seed, precision, anderson=0):
        g, cfg, f = synth.ice_cap(seed=seed)
        cfg = dict(cfg, picard_stop="relres", picard_relres_tol=1e-6, DIVA_visc_it_nit=500, lin_adaptive=1,
                   lin_rtol=1e-10, precision=precision, picard_anderson_m=anderson,
                   lin_adaptive_eta=args.eta if args.eta is not None else (0.1 if anderson else 0.5))
        return diva.Grid(**g), cfg, f

    def prepared(seed, precision, anderson=0):
        grid, cfg, f = case(seed, precision, anderson)
        ctx = diva.Context(grid, cfg)
        ctx.upload(f)
        ctx.update_general_ice_model_data()
        ctx.calc_pressure_melting_point()
        ctx.calc_ice_rheology()
        ctx.update_general_ice_model_data()
        return ctx

    grid = case(0, "fp64")[0]
    net = learned.WarmStartNet(grid, batch=8, capacity=args.members, seed=0)
    net.velocities_only()                  # predict below completes the rest of the state
    t0 = time.perf_counter()
    seed = 0
    while net.num_samples < args.members and seed < 4 * args.members:
        ctx = prepared(seed, "fp64")
        if ctx.solve_DIVA()["status"] == 0:
            net.add_sample(ctx)
        ctx.close()
        seed += 1
    t_data = time.perf_counter() - t0
    t0 = time.perf_counter()
    loss = net.train(args.epochs, lr=1e-3, seed=1)
    t_train = time.perf_counter() - t0

    def timed(seed, use_net, precision="fp64", anderson=0):
        ctx = prepared(seed, precision, anderson)
        torch.cuda.synchronize()
        t = time.perf_counter()
        if use_net:
            net.predict(ctx, complete_sweeps=10)
        try:
            rep = ctx.solve_DIVA()
        except diva.DivaError as e:     # reported in the line, not fatal to the run
            rep = {"status": e.status, "picard_iterations": -1, "mg_cycles": -1, "relres": -1.0, "error": str(e)}
        torch.cuda.synchronize()
        dt = time.perf_counter() - t
        ctx.close()
        return dt, rep

    arms = {"plain": (False, "fp64", 0), "learned": (True, args.precision, args.anderson),
            "accelerated_cold": (False, args.precision, args.anderson)}
    for k in range(args.warmup):
        for a in arms.values():
            timed(20000 + k, *a)
    clocks = ClockSampler(0)
    clocks.start()
    res = {name: [timed(10000 + k, *a) for k in range(args.steps)] for name, a in arms.items()}
    clk = clocks.stop()
    cold, warm = res["plain"], res["learned"]
    t_cold, t_warm = sum(d for d, _ in cold), sum(d for d, _ in warm)
    t_acc = sum(d for d, _ in res["accelerated_cold"])
    parts = ["learned warm start"] + (["FP32 smoother"] if args.precision == "mixed" else []) + \
            ([f"Anderson({args.anderson})"] if args.anderson else [])
    print(json.dumps({
        "metric": "DIVA solves/s at 321x561x15 to rel-res 1e-6: " + " + ".join(parts) + " vs plain FP64 GPU",
        "value": args.steps / t_warm, "unit": "solves/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * t_warm / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f64+f32",
        "data": "synthetic (seeded ice caps; training seeds 0.., held-out seeds 10000..)",
        "config": {"workload": "held-out ice caps 1600x2800 km @5 km, network warm start + 10 completion sweeps",
                   "plain_fp64_solves_per_s": args.steps / t_cold,
                   "ratio_vs_plain_fp64": t_cold / t_warm,
                   "same_method_cold_solves_per_s": args.steps / t_acc,
                   "iterations_cold": [r["picard_iterations"] for _, r in cold],
                   "iterations_learned": [r["picard_iterations"] for _, r in warm],
                   "iterations_same_method_cold": [r["picard_iterations"] for _, r in res["accelerated_cold"]],
                   "mg_cycles_cold": [r["mg_cycles"] for _, r in cold],
                   "mg_cycles_learned": [r["mg_cycles"] for _, r in warm],
                   "status_learned": [r["status"] for _, r in warm],
                   "status_same_method_cold": [r["status"] for _, r in res["accelerated_cold"]],
                   "relres_learned": [r["relres"] for _, r in warm],
                   "training_samples": net.num_samples, "epochs": args.epochs, "final_loss": loss,
                   "data_generation_s": t_data, "training_s": t_train,
                   "timing": "device-synchronised wall clock around predict + solve (inputs resident)"},
        "clocks": clk}))
    net.close()
    return 0


def main():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--quick", action="store_true",
                   help="timed solves only (no roofline, e2e or CPU legs): the command profiled with ncu")
    p.add_argument("--workload", choices=["headline", "icecap", "ensemble", "timestep", "learned", "cpu-variants",
                                          "cnn"],
                   default="headline",
                   help="headline (default): held-out ice caps through the learned path (trained network, "
                        "FP32 smoother, Anderson mixing) against the plain FP64 path; icecap: the plain FP64 solve "
                        "of one fixed ice cap; ensemble: --members perturbed members; "
                        "timestep: predictor/corrector steps with thickness and heat equation; "
                        "learned: --members training caps, then held-out solves cold vs warm-started")
    p.add_argument("--epochs", type=int, default=60, help="training epochs of the learned workload")
    p.add_argument("--members", type=int, default=64)
    p.add_argument("--anderson-sheet", type=int, default=None,
                   help="ensemble: Anderson depth for the 1501 x 1501 members (default: --anderson)")
    p.add_argument("--learned", action="store_true",
                   help="ensemble: warm-start the channel and ice-cap members with a trained network each")
    p.add_argument("--learned-samples", type=int, default=64, help="training solutions per network (ensemble)")
    p.add_argument("--ensemble-sizes", default="channel,icecap",
                   help="member kinds drawn from: channel (129x17), icecap (321x561), sheet (1501x1501)")
    p.add_argument("--precision", choices=["fp64", "mixed"], default="fp64",
                   help="mixed: FP32 finest-level smoother inside the FP64 Krylov solve (not the default line)")
    p.add_argument("--anderson", type=int, default=0,
                   help="Anderson mixing depth of the viscosity iteration (0: the reference's relaxation)")
    p.add_argument("--eta", type=float, default=None,
                   help="adaptive linear tolerance factor (default 0.5, or 0.1 with --anderson)")
    p.add_argument("--lin-maxit", type=int, default=500,
                   help="ensemble: Krylov iteration cap of each linear solve")
    p.add_argument("--stall-its", type=int, default=0,
                   help="ensemble: stop a member whose rel-res has not fallen by 10 %% for this many viscosity "
                        "iterations (a velocity-limited member that cannot reach the tolerance); 0 = off")
    args = p.parse_args()
    if args.impl == "b200" and args.workload == "ensemble":
        return run_ensemble(args)
    if args.impl == "b200" and args.workload == "timestep":
        return run_timestep(args)
    if args.impl == "b200" and args.workload == "learned":
        return run_learned(args)
    if args.workload == "cpu-variants":
        return run_cpu_variants(args)
    if args.impl == "b200" and args.workload == "cnn":
        return run_cnn(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "headline":
        return run_headline(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
