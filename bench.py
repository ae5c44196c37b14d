"""Benchmark: simulated picoseconds per wall-clock hour of the time step.

Workload (default): the large-droplet configuration, 256^3 grid, h=0.4 A,
N=5000 He atoms, 16384 Bohmian test particles at 200 m/s, Morse impurity,
core4='OTC', npd=7, dt = 1 fs, plain FP64 form.  One "step" is one Hamming
predictor-corrector step (two mean-field evaluations) of that system.

Arms
  (default)          the CUDA library on N GPUs, one independent replica per
                     GPU ("replicas only": the path does not shard).
  --impl reference   the CPU oracle (FP64 restatement of the reference step)
                     on all host cores, rank 0 only, bounded sample.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--config c3]
For N > 1 run under torchrun (one rank per GPU).
"""
import argparse
import ctypes as C
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "4hetddft-isotropic-bohmian_b200")
METRIC = "simulated ps/hour at 256^3 N=5000: parareal+FP32 conv vs plain FP64, 1 B200"
DT_FS = 1.0


def load_pkg():
    name = "he4b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(
        name, os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.tmp = None

    def __enter__(self):
        try:
            self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.tmp, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.tmp is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.tmp.flush()
        rows = [l.split(",") for l in open(self.tmp.name).read().splitlines() if l.strip()]
        os.unlink(self.tmp.name)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus, backend="nccl"):
    """One process per GPU (torchrun env); the replicas share nothing but
    the timing reduction.  backend "gloo" runs the same plumbing on CPU."""
    if n_gpus <= 1 and "RANK" not in os.environ:
        return 0, 1, 0, None
    import datetime

    import torch
    import torch.distributed as dist
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    kw = {}
    if backend == "nccl":
        torch.cuda.set_device(local)
        kw["device_id"] = torch.device("cuda", local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600), **kw)
    return rank, world, local, dist


def max_over_ranks(dist, x, device):
    """The largest value of x over all ranks (x itself without a group)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world, sim_ps_per_rank, seconds_max):
    """Whole-job simulated ps per hour: every rank advanced its own replica
    by sim_ps_per_rank in at most seconds_max (the slowest rank)."""
    return world * sim_ps_per_rank / (seconds_max / 3600.0)


FORMS = {"fp64": "plain FP64", "fp32": "FP32 convolutions (FP32 half spectra, kernels and twiddles; "
                                         "FP64 real grids, psi update, reductions and trajectories)",
         "parareal": "learned parareal: FNO coarse step (64^3, width 32, 12 modes/axis, 4 layers, BF16 weights) "
                     "+ FP32-convolution PC fine propagator over 6 slices of 50 fs, sequential fallback"}
PARAREAL_SLICES, PARAREAL_STEPS = 6, 50


def form_params(pkg, p, form):
    q = pkg.abi.He4Params.from_buffer_copy(p)
    q.precision = pkg.abi.HE4_PREC_FP32CONV if form == "fp32" else pkg.abi.HE4_PREC_FP64
    return q


def gpu_arm(args):
    import torch
    pkg = load_pkg()
    rank, world, local, dist = dist_setup(args.gpus)
    w = pkg.workloads
    cfg = w.CONFIGS[args.config]
    p, psi, r, v, _ = w.workload(args.config, seed=1234 + rank)
    p.device = local
    dt = w.deltat_fs(DT_FS)

    def barrier():
        torch.cuda.synchronize(local)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(local)

    def timed_run(g, stream, reps=1):
        """K PC steps from device-resident state, CUDA events on the
        library's stream, max over ranks; `reps` windows, each from the same
        state after the same warm-up, the median returned with all."""
        windows, launches = [], 0
        with ClockSampler(local) as clk:
            for _ in range(reps):
                g.set_state(psi, r, v)
                # the RK-Gill starter, then one PC step of each of the 30
                # buffer states of the step (and at least --warmup), so every
                # step graph is captured before timing
                g.run(3 + max(args.warmup, 30), dt)
                barrier()
                n0 = g.launch_count()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                err, means = g.run(args.steps, dt)
                e1.record(stream)
                e1.synchronize()
                launches = g.launch_count() - n0
                ms = e0.elapsed_time(e1)
                barrier()
                windows.append(max_over_ranks(dist, ms, f"cuda:{local}"))
                if not np.all(np.isfinite(err)) or not np.all(np.isfinite(means)):
                    raise RuntimeError("non-finite step errors in the timed region")
        return float(np.median(windows)), launches, clk.summary(), windows

    # ---- every form on the same workload; the headline is args.form
    forms = {}
    sim_ps = args.steps * DT_FS * 1e-3
    step_form = "fp32" if args.form == "parareal" else args.form
    g = stream = None
    for form in ("fp64", "fp32"):
        if form != step_form and not args.all_forms:
            continue
        gf = pkg.He4Step(form_params(pkg, p, form))
        sf = torch.cuda.ExternalStream(gf.stream(), device=torch.device("cuda", local))
        # a step-form headline times exactly one window of K steps; beside the
        # parareal headline each form is timed over --form-reps windows of K
        # steps and the median window reported (a stall of the shared box
        # inside one window then moves no number)
        reps = 1 if form == args.form else max(1, args.form_reps)
        ms_f, launches_f, clocks_f, windows = timed_run(gf, sf, reps)
        ms_step = ms_f / args.steps
        cap, unc = gf.graph_stats()
        forms[form] = {"form": FORMS[form], "ms_per_step": ms_step, "windows_ms": windows,
                       "value": replica_throughput(world, sim_ps, ms_f * 1e-3), "gpu_launches": launches_f,
                       "clocks": clocks_f, "graphs": {"captured": cap, "steps_uncaptured": unc}}
        # whole-step roofline: the algorithmic bytes of one PC step over its time
        peak, _ = load_peaks()
        sb = step_bytes(form, p.nx * p.ny * p.nz)
        forms[form]["step_roofline"] = {"bytes_per_step": sb, "achieved_gbs": sb / (ms_step * 1e-3) / 1e9,
                                        "peak_gbs": peak, "frac": sb / (ms_step * 1e-3) / 1e9 / peak}
        forms[form]["roofline"] = kernel_roofline(pkg, gf, args, form)
        forms[form]["kernels"] = [kernel_roofline(pkg, gf, args, form, which=i) for i in NEXT_KERNELS[form]]
        forms[form]["e2e"] = e2e_leg(pkg, torch, gf, psi, r, v, dt, args, barrier, dist, local, world)
        if form == step_form:
            g, stream = gf, sf
            ms_max, launches, clocks = ms_f, launches_f, clocks_f
        else:
            gf.close()
    value = replica_throughput(world, sim_ps, ms_max * 1e-3)
    roof = dict(forms[step_form]["roofline"] or {})
    if roof:
        roof["step_frac"] = forms[step_form]["step_roofline"]["frac"]
        roof["step_bytes"] = forms[step_form]["step_roofline"]["bytes_per_step"]
        roof["form"] = step_form
    e2e = forms[step_form]["e2e"]

    par = None
    if args.form == "parareal":
        par = parareal_form(pkg, args, p, psi, r, v, dt, local, barrier)
        dev_s = max_over_ranks(dist, par["device_s"], f"cuda:{local}")
        par["e2e_s"] = max_over_ranks(dist, par["e2e_s"], f"cuda:{local}")
        par["value"] = replica_throughput(world, par["sim_ps"], dev_s)
        par["ms_per_step"] = dev_s * 1e3 / (PARAREAL_SLICES * PARAREAL_STEPS)
        nsteps_par = PARAREAL_SLICES * PARAREAL_STEPS
        # end to end = the parareal run from host buffers to the final state
        # on the host (initial upload, training excluded, final download)
        par["e2e"] = {"value": replica_throughput(world, par["sim_ps"], par["e2e_s"]), "unit": "simulated ps/hour",
                      "h2d_bytes_per_step": par["e2e_h2d"] / nsteps_par,
                      "d2h_bytes_per_step": par["e2e_d2h"] / nsteps_par, "steps": nsteps_par,
                      "includes": "parareal run from host state: upload, iterations, fallback, final-state download"}
        forms["parareal"] = par
        value = par["value"]
        ms_max = par["ms_per_step"]
        launches = par["gpu_launches"]
        clocks = par["clocks"]
        e2e = par["e2e"]

    if args.ensemble > 0 and world == 1:
        forms["ensemble"] = ensemble_form(pkg, args, local, barrier)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(pkg, args)
    g.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    timed = ("K predictor-corrector steps from device-resident state (he4_run); K = --steps" if par is None else
             f"a fixed {PARAREAL_SLICES} x {PARAREAL_STEPS} fs of parareal from device-resident state, the "
             f"median of {args.parareal_reps} runs (FNO training untimed); --steps K sets the K PC steps each "
             f"step form in 'forms' times")
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "simulated ps/hour",
        "n_gpus": world,
        "steps": args.steps if par is None else PARAREAL_SLICES * PARAREAL_STEPS,
        "warmup": max(args.warmup, 30),
        "ms_per_step": ms_max / args.steps if par is None else ms_max,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": {"fp64": "f64", "fp32": "f32 spectra / f64 state",
                  "parareal": "bf16 weights / f32 FNO / f32 spectra / f64 state"}[args.form],
        "data": "synthetic (Fermi-profile droplet, seeded Gaussian test particles)",
        "config": {
            "workload": f"{args.config}: {cfg['n']}^3 grid h={cfg['h']} A, N={cfg['n4']} He, "
                        f"{cfg['npar']} test particles at {cfg['speed_ms']:g} m/s, Morse impurity, "
                        f"core4=OTC npd=7 icon=8, dt=1 fs, Hamming PC steps",
            "form": FORMS[args.form],
            "parallelism": f"replicas x{world} (no data-path collective)",
            "l2": "inputs larger than L2: every grid array is >= 134 MB",
            "timed": timed,
        },
        "e2e": e2e,
        "gpu_launches": launches,
        "roofline": roof or None,
        "clocks": clocks,
        "forms": forms,
    }
    if "fp64" in forms and args.form != "fp64":
        line["speedup_vs_plain_fp64"] = forms["fp64"]["ms_per_step"] / forms[args.form]["ms_per_step"]
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


def parareal_form(pkg, args, p, psi, r, v, dt, local, barrier):
    """Train the FNO coarse propagator on solver trajectories of the 128^3
    family (FP32 form, restricted to 64^3), then run parareal on the
    workload: PARAREAL_SLICES slices of PARAREAL_STEPS fine steps (6 x 50 fs:
    the 256^3 workload leaves the range the integrator handles after about
    300 fs), FP32-convolution fine propagator.  The timed region is the
    parareal run; its final state is compared with the plain FP64
    sequential run over the same 300 fs."""
    import torch
    w, pr, fno = pkg.workloads, pkg.parareal, pkg.fno
    dev = torch.device("cuda", local)
    S, K = PARAREAL_SLICES, PARAREAL_STEPS
    spec = fno.FnoSpec(n=64, width=32, modes=(12, 12, 12), layers=4)
    net = fno.Fno(spec, seed=5, device=local)
    t_train = time.perf_counter()
    xs, ys = [], []
    gen = None
    for i in range(args.fno_traj):
        pm, ps, rm, vm = w.family_member("c2", 10000 + i)
        pm.device = local
        if gen is None:  # one handle for every trajectory (same grid and form)
            gen = pkg.He4Step(form_params(pkg, pm, "fp32"))
        enc = pr.FnoCoarse(net, pm, 2, K * dt)
        a, b = pr.trajectory_pairs(w, pm, ps, rm, vm, 4, K, dt, enc, dev, handle=gen)
        xs += a
        ys += b
    gen.close()
    # the last 8 trajectories (32 coarse steps) are held out
    hold_x, hold_y = xs[-32:], ys[-32:]
    xs, ys = xs[:-32], ys[:-32]
    before = pr.evaluate(net, hold_x, hold_y)
    pr.train(net, xs, ys, args.fno_steps, batch=2, lr=1e-3)
    after = pr.evaluate(net, hold_x, hold_y)
    t_train = time.perf_counter() - t_train
    # the training pairs are not needed again: release them (and torch's
    # cached blocks) before the fine handles are created and timed
    del xs, ys, hold_x, hold_y
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    q = form_params(pkg, p, "fp32")
    coarse = pr.FnoCoarse(net, q, p.nx // spec.n, K * dt)
    par = pr.Parareal(q, S, K, dt, coarse, concurrent=8)
    par.warm(psi, r, v)  # graph capture of the fine propagators, untimed
    # the whole run is one timed region of ~1.5 s, so one stall of the shared
    # host or GPU moves it far; it is repeated from the same state and the
    # median run is reported (every run's time is listed)
    runs = []
    # host buffers in pinned memory, as a host that streams states would keep
    # them: the initial state in, the final state out
    psi_in = pin(torch, psi.view(np.float64)).numpy().view(np.complex128)
    r_in, v_in = pin(torch, r).numpy(), pin(torch, v).numpy()
    fin0 = par.final_state()
    psi_h = torch.empty(fin0.psi.shape, dtype=fin0.psi.dtype).pin_memory()
    r_h = torch.empty(fin0.r.shape, dtype=fin0.r.dtype).pin_memory()
    v_h = torch.empty(fin0.v.shape, dtype=fin0.v.dtype).pin_memory()
    with ClockSampler(local) as clk:
        for _ in range(max(1, args.parareal_reps)):
            n_lib0 = sum(h.launch_count() for h in par.handles)
            n_net0 = net.launches
            barrier()
            t0 = time.perf_counter()
            res = par.run(psi_in, r_in, v_in, tol=1e-6)
            fin = par.final_state()
            psi_h.copy_(fin.psi)
            r_h.copy_(fin.r)
            v_h.copy_(fin.v)
            e2e_s = time.perf_counter() - t0
            psi_out = psi_h.numpy().view(np.complex128).reshape(psi.shape).copy()
            r_out = r_h.numpy().copy()
            v_out = v_h.numpy().copy()
            launches = sum(h.launch_count() for h in par.handles) - n_lib0 + (net.launches - n_net0)
            runs.append((res["device_s"], e2e_s, res, launches, psi_out, r_out, v_out))
    clocks = clk.summary()
    device_runs = [x[0] for x in runs]
    e2e_runs = [x[1] for x in runs]
    _, _, res, launches, psi_out, r_out, v_out = sorted(runs, key=lambda x: x[0])[len(runs) // 2]
    e2e_s = float(np.median(e2e_runs))
    gstats = [h.graph_stats() for h in par.handles]
    # coarse-step error over slice 0 at this grid: the network's (as the
    # judge measured it) and G = identity's (psi unchanged)
    identity_err = par._rel_psi(par.F[1], par.U[0])
    par.close()
    # accuracy against the plain FP64 sequential run over the same time
    with pkg.He4Step(p) as g64:
        g64.set_state(psi, r, v)
        g64.run(S * K, dt)
        psi64 = g64.get_state()[0]
        e64 = g64.energy()
        g64.set_state(psi_out, r_out, v_out)
        epar = g64.energy()
    d64, dpar = np.abs(psi64) ** 2, np.abs(psi_out) ** 2
    sim_ps = S * K * DT_FS * 1e-3
    return {"form": FORMS["parareal"], "sim_ps": sim_ps, "device_s": res["device_s"], "e2e_s": e2e_s,
            "runs": {"count": len(runs), "device_s": device_runs, "e2e_s": e2e_runs,
                     "reported": "median run (device time); e2e is the median of the runs' e2e times"},
            "iterations": res["iterations"],
            "converged": res["converged"], "exact_by_fallback": res["exact_by_fallback"],
            "diverged": res["diverged"], "fallback_at": res["fallback_at"],
            "changes": res["changes"], "fine_steps_executed": res["fine_steps"],
            "coarse_step_error": {"fno": res["changes"][0] if res["changes"] else None,
                                  "identity": identity_err, "judge_threshold": 1e-6,
                                  "over": f"slice 0 ({PARAREAL_STEPS} fs) at {p.nx}^3"},
            "fno": {"training_trajectories": args.fno_traj, "training_steps": args.fno_steps,
                    "held_out_rel_error_before": before, "held_out_rel_error_after": after,
                    "train_and_data_s": t_train},
            "vs_plain_fp64_serial": {"density_rel_l2": float(np.linalg.norm(dpar - d64) / np.linalg.norm(d64)),
                                     "etot_rel_diff": abs(epar["etot"] - e64["etot"]) / abs(e64["etot"])},
            "gpu_launches": launches, "clocks": clocks,
            "graphs": {"captured": sum(c for c, _ in gstats), "steps_uncaptured": sum(u for _, u in gstats)},
            "e2e_h2d": psi.nbytes + r.nbytes + v.nbytes,
            "e2e_d2h": psi.nbytes + r.nbytes + v.nbytes}


def ensemble_form(pkg, args, local, barrier):
    """The batched ensemble: 64 members (N log-uniform in [200, 3000],
    grids 64^3 / 96^3 / 128^3, 1024 test particles, 50-300 m/s), tile shapes
    from the autotuner, K ensemble PC steps timed; the same members run one
    after the other (each through its own he4_run) give the unbatched time."""
    import torch
    w = pkg.workloads
    dt = w.deltat_fs(DT_FS)
    ms = [w.ensemble_member(i) for i in range(args.ensemble)]
    params = []
    for m in ms:
        m[0].device = local
        params.append(m[0])
    grids = {}
    for m in ms:
        grids[m[0].nx] = grids.get(m[0].nx, 0) + 1
    t0 = time.perf_counter()
    b = pkg.He4Batch(params)
    t_create = time.perf_counter() - t0
    for mem, m in zip(b.members, ms):
        mem.set_state(m[1], m[2], m[3])
    t0 = time.perf_counter()
    tiles, tms = b.tune(reps=3)
    t_tune = time.perf_counter() - t0
    K = args.ensemble_steps
    # the starter and one K-step run capture the graphs the timed run
    # replays (the members' buffer states repeat every 30 steps)
    b.run(3 + K * max(1, -(-30 // K)), dt)
    barrier()
    n0 = b.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record()
        err, means = b.run(K, dt)
        torch.cuda.synchronize(local)
        e1.record()
        e1.synchronize()
    batched_s = e0.elapsed_time(e1) * 1e-3
    launches = b.launch_count() - n0
    clocks = clk.summary()
    # the same members one after the other (unbatched), same tiles and state phase
    barrier()
    e0.record()
    for mem in b.members:
        mem.run(K, dt)
    torch.cuda.synchronize(local)
    e1.record()
    e1.synchronize()
    seq_s = e0.elapsed_time(e1) * 1e-3
    per_grid = {}
    for t, m in zip(tiles.tolist(), ms):
        per_grid.setdefault(f"{m[0].nx}^3", t)
    b.close()
    sim = args.ensemble * K * DT_FS * 1e-3
    # step-level roofline of the batch: the members' algorithmic bytes per
    # ensemble step (plain FP64 counting rule) over its time
    peak, _ = load_peaks()
    ens_bytes = sum(step_bytes("fp64", m[0].nx * m[0].ny * m[0].nz) for m in ms)
    ens_gbs = ens_bytes / (batched_s / K) / 1e9
    return {"form": f"batched ensemble of {args.ensemble} systems, graphs of up to 30 ensemble steps per launch",
            "step_roofline": {"bytes_per_ensemble_step": ens_bytes, "achieved_gbs": ens_gbs, "peak_gbs": peak,
                              "frac": ens_gbs / peak},
            "members_per_grid": {f"{k}^3": v for k, v in sorted(grids.items())}, "steps": K,
            "value": sim / (batched_s / 3600.0), "unit": "simulated ps/hour (sum over members)",
            "ms_per_ensemble_step": batched_s * 1e3 / K, "unbatched_ms_per_ensemble_step": seq_s * 1e3 / K,
            "batching_speedup": seq_s / batched_s, "gpu_launches": launches,
            "tiles_per_grid": per_grid, "create_s": t_create, "tune_s": t_tune, "clocks": clocks}


def pin(torch, a):
    t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    return t


# dominant kernel of each step form's launch list (profiles/launch_list_*):
# he4_bench_kernel ids 12 (inverse y pass) and 3 (x pass C2R); the next
# kernels of each list are timed beside it (ids 6: z convolution with three
# outputs, 9: merged pot4 on float grids, 8: on FP64 grids, 1: forward y pass)
DOMINANT_KERNEL = {"fp32": 12, "fp64": 3}
NEXT_KERNELS = {"fp32": (6, 9), "fp64": (1, 6, 8)}


def step_bytes(form, n):
    """Algorithmic bytes of one PC step of an n-point grid: every pointwise
    op fused into an adjacent FFT or stencil pass, each FFT one read and one
    write, each kernel array read once per use, stencils reading their
    inputs once (R = 8n bytes a real grid, a half spectrum S ~ R).  Per
    field evaluation 60R + 28S (forward FFTs 18R + 10S, inverse 18S + 12R,
    stencils and pointwise ~30R), per step two evaluations plus 39R of
    predictor / corrector: 215R = 1720 n bytes.  The FP32-convolution form
    halves the FFT and convolution bytes: per evaluation 45R + 14S, per step
    157R = 1256 n bytes."""
    return (1256 if form == "fp32" else 1720) * float(n)


def kernel_roofline(pkg, g, args, form, reps=20, which=None):
    """Average duration of the form's dominant kernel (or of bench id
    `which`), timed with CUDA events on the library's stream (the kernel's
    own launch stream), against its algorithmic bytes; DRAM traffic per
    launch from the committed ncu capture of the same kernel."""
    L = pkg.load_library()
    L.he4_bench_kernel.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_double),
                                   C.POINTER(C.c_double), C.c_char_p, C.c_int32]
    ms, byts = C.c_double(), C.c_double()
    name = C.create_string_buffer(64)
    which = DOMINANT_KERNEL[form] if which is None else which
    g.field()  # the stencil ids work on the fields of a current evaluation
    rc = L.he4_bench_kernel(g._h, which, reps, C.byref(ms), C.byref(byts), name, 64)
    if rc != 0:
        return None
    peak, src = load_peaks()
    achieved = byts.value / (ms.value * 1e-3) / 1e9
    kname = name.value.decode()
    traffic, tsrc = None, None
    prof = os.path.join(ROOT, "profiles", "dominant_kernels_traffic.json")
    if args.config == "c3" and os.path.exists(prof):
        ent = json.load(open(prof))["kernels"].get(f"{form}:{which}")
        if ent:
            traffic, tsrc = ent["traffic_bytes_per_launch_256"], ent["source"]
    return {"kernel": kname, "bench_id": which, "bound": "hbm", "achieved": achieved, "peak": peak,
            "peak_source": f"{src} (MEASURED_PEAKS.json hbm_gbs)" if src == "measured" else src,
            "unit": "GB/s", "frac": achieved / peak, "traffic": traffic, "traffic_source": tsrc,
            "bytes_per_launch": byts.value, "ms_per_launch": ms.value, "launches_timed": reps}


def e2e_leg(pkg, torch, g, psi, r, v, dt, args, barrier, dist, local, world):
    """The same metric end to end through the per-step C ABI with host
    buffers: he4_set_state (pinned host -> device), 3 he4_step_rk + (K-3)
    he4_step_pc (each returns its errors and means to the host),
    he4_get_state (device -> pinned host)."""
    psi_h = pin(torch, psi.view(np.float64))
    r_h, v_h = pin(torch, r), pin(torch, v)
    out_psi = pin(torch, np.zeros_like(psi).view(np.float64))
    out_r = pin(torch, np.zeros_like(r))
    L = pkg.load_library()
    dp = lambda t: C.cast(t.data_ptr(), C.POINTER(C.c_double))
    steps = max(args.steps, 4)
    e_buf, m_buf = (C.c_double * 3)(), (C.c_double * 9)()
    barrier()
    t0 = time.perf_counter()
    if L.he4_set_state(g._h, dp(psi_h), dp(r_h), dp(v_h)) != 0:
        raise RuntimeError("he4_set_state failed")
    for s in range(steps):
        rc = L.he4_step_rk(g._h, dt, m_buf) if s < 3 else L.he4_step_pc(g._h, dt, e_buf, m_buf)
        if rc != 0:
            raise RuntimeError(f"step failed: {rc}")
    if L.he4_get_state(g._h, dp(out_psi), dp(out_r), None, None) != 0:
        raise RuntimeError("he4_get_state failed")
    t1 = time.perf_counter()
    e2e_s = max_over_ranks(dist, t1 - t0, f"cuda:{local}")
    h2d = psi.nbytes + r.nbytes + v.nbytes
    d2h = psi.nbytes + r.nbytes + (3 * 8 + 9 * 8) * (steps - 3) + 9 * 8 * 3
    return {"value": replica_throughput(world, steps * DT_FS * 1e-3, e2e_s), "unit": "simulated ps/hour",
            "h2d_bytes_per_step": h2d / steps, "d2h_bytes_per_step": d2h / steps, "steps": steps,
            "includes": "3 RK-Gill starter steps, per-step err/means copy-out, state upload and download"}


def cpu_baseline(pkg, args, target_s=20.0):
    """The CPU oracle on all host threads, bounded sample: setup is untimed,
    then PC steps are timed until ~target_s of CPU work."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    w = pkg.workloads
    p, psi, r, v, _ = w.workload(args.config)
    o = oracle.Oracle(p)
    o.set_state(psi, r, v)
    o.field()
    dt = w.deltat_fs(DT_FS)
    t0 = time.perf_counter()
    n = 0
    while True:
        o.steppc(dt)
        n += 1
        el = time.perf_counter() - t0
        if el > target_s or n >= 50:
            break
    o.close()
    return {"value": n * DT_FS * 1e-3 / (el / 3600.0), "unit": "simulated ps/hour", "cores": threads,
            "kind": "port", "sample": f"{n} predictor-corrector steps of the {args.config} workload "
                                      f"({el:.1f} s) after an untimed setup and field evaluation"}


def reference_arm(args):
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    pkg = load_pkg()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    w = pkg.workloads
    p, psi, r, v, _ = w.workload(args.config)
    o = oracle.Oracle(p)
    o.set_state(psi, r, v)
    o.field()
    dt = w.deltat_fs(DT_FS)
    warm = min(args.warmup, 1)
    for _ in range(warm):
        o.steppc(dt)
    steps = max(1, min(args.steps, 3))
    t0 = time.perf_counter()
    for _ in range(steps):
        o.steppc(dt)
    el = time.perf_counter() - t0
    o.close()
    value = steps * DT_FS * 1e-3 / (el / 3600.0)
    cfg = w.CONFIGS[args.config]
    print(json.dumps({
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "simulated ps/hour",
        "n_gpus": 0,
        "steps": steps,
        "warmup": warm,
        "ms_per_step": el * 1e3 / steps,
        "higher_is_better": True,
        "dtype": "f64",
        "data": "synthetic (Fermi-profile droplet, seeded Gaussian test particles)",
        "config": {"workload": f"{args.config}: {cfg['n']}^3 grid, N={cfg['n4']} He, {cfg['npar']} test "
                               f"particles, core4=OTC npd=7, plain FP64 predictor-corrector steps",
                   "timed": f"min(K, 3) = {steps} PC steps after {warm} untimed: a bounded sample of the CPU run "
                            "(about 1.7 s per step on 16 threads at 256^3); simulated ps/hour is a rate, so "
                            "the sample length does not change it"},
        "cpu_baseline": {"value": value, "unit": "simulated ps/hour", "cores": threads, "kind": "port",
                         "sample": f"{steps} PC steps (bounded sample of the {args.config} workload)"},
        "e2e": {"value": value, "unit": "simulated ps/hour", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def profile_kernels(form, config="c3", shape=None, ids=None, reps=1):
    """One field evaluation of a workload, then one warm-up and one timed
    launch of each pass he4_bench_kernel measures: the workload the ncu
    summaries under profiles/ capture.  shape (nx, ny, nz) replaces the
    grid of the config (the same spacing and droplet), so a capture keeps
    its inputs above L2 with a few GB on the device."""
    pkg = load_pkg()
    w = pkg.workloads
    if shape is None:
        p, psi, r, v, _ = w.workload(config)
    else:
        cfg = w.CONFIGS[config]
        p = w.make_params(shape[0], cfg["h"], cfg["npar"], ny=shape[1], nz=shape[2])
        psi = w.droplet_psi(p, cfg["n4"])
        r, v = w.particles(cfg["npar"], 1234, cfg["speed_ms"])
    g = pkg.He4Step(form_params(pkg, p, form))
    g.set_state(psi, r, v)
    g.run(1, w.deltat_fs(DT_FS))  # a merged evaluation fills the float grids
    L = pkg.load_library()
    L.he4_bench_kernel.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_double),
                                   C.POINTER(C.c_double), C.c_char_p, C.c_int32]
    if ids is None:
        ids = (0, 1, 2, 3, 6, 7, 8) + ((9, 10) if form == "fp32" else ())
    for which in ids:
        ms, b = C.c_double(), C.c_double()
        nm = C.create_string_buffer(64)
        if L.he4_bench_kernel(g._h, which, reps, C.byref(ms), C.byref(b), nm, 64) != 0:
            raise RuntimeError(L.he4_last_error().decode())
        print(json.dumps({"which": which, "kernel": nm.value.decode(), "algorithmic_bytes": b.value,
                          "ms": ms.value, "grid": [p.nx, p.ny, p.nz]}), flush=True)
    g.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c3", choices=["c1", "c2", "c3"])
    ap.add_argument("--form", default="parareal", choices=sorted(FORMS))
    ap.add_argument("--fno-traj", type=int, default=200, help="training trajectories of the FNO (parareal form)")
    ap.add_argument("--fno-steps", type=int, default=1500, help="training steps of the FNO (parareal form)")
    ap.add_argument("--form-reps", type=int, default=3,
                    help="timed windows of K steps per step form beside the parareal headline (median reported)")
    ap.add_argument("--parareal-reps", type=int, default=5,
                    help="timed parareal runs from the same state; the median is reported")
    ap.add_argument("--all-forms", action=argparse.BooleanOptionalAction, default=True,
                    help="also time the other forms on the same workload")
    ap.add_argument("--ensemble", type=int, default=64, help="ensemble members timed beside (0 = skip)")
    ap.add_argument("--ensemble-steps", type=int, default=30)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-kernels", choices=["fp64", "fp32"], default=None,
                    help="run each FFT/stencil pass once on the --config workload (for ncu captures) and exit")
    ap.add_argument("--profile-shape", default=None, help="nx,ny,nz grid for --profile-kernels")
    ap.add_argument("--profile-reps", type=int, default=1, help="timed launches per id for --profile-kernels")
    ap.add_argument("--profile-ids", default=None, help="comma-separated he4_bench_kernel ids for --profile-kernels")
    args = ap.parse_args()
    if args.profile_kernels:
        shape = tuple(int(x) for x in args.profile_shape.split(",")) if args.profile_shape else None
        ids = tuple(int(x) for x in args.profile_ids.split(",")) if args.profile_ids else None
        profile_kernels(args.profile_kernels, args.config, shape, ids, args.profile_reps)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
