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


def dist_setup(n_gpus):
    if n_gpus <= 1 and "RANK" not in os.environ:
        return 0, 1, 0, None
    import torch
    import torch.distributed as dist
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    import datetime
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                            device_id=torch.device("cuda", local))
    return rank, world, local, dist


FORMS = {"fp64": "plain FP64", "fp32": "FP32 convolutions (FP32 half spectra, kernels and twiddles; "
                                         "FP64 real grids, psi update, reductions and trajectories)"}


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

    def timed_run(g, stream):
        """K PC steps from device-resident state, CUDA events on the
        library's stream, max over ranks."""
        g.set_state(psi, r, v)
        g.run(3 + args.warmup, dt)
        barrier()
        n0 = g.launch_count()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            e0.record(stream)
            err, means = g.run(args.steps, dt)
            e1.record(stream)
            e1.synchronize()
        launches = g.launch_count() - n0
        ms = e0.elapsed_time(e1)
        barrier()
        if dist is not None:
            t = torch.tensor([ms], device=f"cuda:{local}", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        if not np.all(np.isfinite(err)) or not np.all(np.isfinite(means)):
            raise RuntimeError("non-finite step errors in the timed region")
        return ms, launches, clk.summary()

    # ---- every form on the same workload; the headline is args.form
    forms = {}
    sim_ps = args.steps * DT_FS * 1e-3
    for form in ("fp64", "fp32"):
        if form != args.form and not args.all_forms:
            continue
        gf = pkg.He4Step(form_params(pkg, p, form))
        sf = torch.cuda.ExternalStream(gf.stream(), device=torch.device("cuda", local))
        ms_f, launches_f, clocks_f = timed_run(gf, sf)
        forms[form] = {"form": FORMS[form], "ms_per_step": ms_f / args.steps,
                       "value": world * sim_ps / (ms_f / 3.6e6), "gpu_launches": launches_f, "clocks": clocks_f}
        if form == args.form:
            g, stream = gf, sf
            ms_max, launches, clocks = ms_f, launches_f, clocks_f
        else:
            gf.close()
    value = world * sim_ps / (ms_max / 3.6e6)

    # ---- dominant-kernel roofline, measured live with CUDA events
    roof = kernel_roofline(pkg, g, stream, args)

    # ---- end to end through the per-step C ABI with host buffers:
    # he4_set_state (pinned host -> device), 3 he4_step_rk + (K-3)
    # he4_step_pc (each returns err/means to the host), he4_get_state.
    psi_h = pin(torch, psi.view(np.float64))
    r_h, v_h = pin(torch, r), pin(torch, v)
    out_psi = pin(torch, np.zeros_like(psi).view(np.float64))
    out_r = pin(torch, np.zeros_like(r))
    L = pkg.load_library()
    dp = lambda t: C.cast(t.data_ptr(), C.POINTER(C.c_double))
    e2e_steps = max(args.steps, 4)
    e_buf, m_buf = (C.c_double * 3)(), (C.c_double * 9)()
    barrier()
    t0 = time.perf_counter()
    assert L.he4_set_state(g._h, dp(psi_h), dp(r_h), dp(v_h)) == 0
    for s in range(e2e_steps):
        if s < 3:
            rc = L.he4_step_rk(g._h, dt, m_buf)
        else:
            rc = L.he4_step_pc(g._h, dt, e_buf, m_buf)
        if rc != 0:
            raise RuntimeError(f"step failed: {rc}")
    assert L.he4_get_state(g._h, dp(out_psi), dp(out_r), None, None) == 0
    t1 = time.perf_counter()
    e2e_s = t1 - t0
    if dist is not None:
        t = torch.tensor([e2e_s], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    h2d = psi.nbytes + r.nbytes + v.nbytes
    d2h = psi.nbytes + r.nbytes + (3 * 8 + 9 * 8) * (e2e_steps - 3) + 9 * 8 * 3
    e2e_value = world * e2e_steps * DT_FS * 1e-3 / (e2e_s / 3600.0)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(pkg, args)
    g.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "simulated ps/hour",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if args.form == "fp64" else "f32 spectra / f64 state",
        "data": "synthetic (Fermi-profile droplet, seeded Gaussian test particles)",
        "config": {
            "workload": f"{args.config}: {cfg['n']}^3 grid h={cfg['h']} A, N={cfg['n4']} He, "
                        f"{cfg['npar']} test particles at {cfg['speed_ms']:g} m/s, Morse impurity, "
                        f"core4=OTC npd=7 icon=8, dt=1 fs, Hamming PC steps",
            "form": FORMS[args.form],
            "parallelism": f"replicas x{world} (no data-path collective)",
            "l2": "inputs larger than L2: every grid array is >= 134 MB",
            "timed": "K predictor-corrector steps from device-resident state (he4_run)",
        },
        "e2e": {"value": e2e_value, "unit": "simulated ps/hour", "h2d_bytes_per_step": h2d / e2e_steps,
                "d2h_bytes_per_step": d2h / e2e_steps, "steps": e2e_steps,
                "includes": "3 RK-Gill starter steps, per-step err/means copy-out, state upload and download"},
        "gpu_launches": launches,
        "roofline": roof,
        "clocks": clocks,
        "forms": forms,
    }
    if "fp64" in forms and args.form != "fp64":
        line["speedup_vs_plain_fp64"] = forms["fp64"]["ms_per_step"] / forms[args.form]["ms_per_step"]
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


def pin(torch, a):
    t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    return t


def kernel_roofline(pkg, g, stream, args):
    """Average duration of the dominant kernel, timed with CUDA events on the
    library's stream, against its algorithmic bytes."""
    L = pkg.load_library()
    if not hasattr(L, "he4_bench_kernel"):
        return None
    L.he4_bench_kernel.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_double),
                                   C.POINTER(C.c_double), C.c_char_p, C.c_int32]
    ms, byts = C.c_double(), C.c_double()
    name = C.create_string_buffer(64)
    rc = L.he4_bench_kernel(g._h, 0, 20, C.byref(ms), C.byref(byts), name, 64)
    if rc != 0:
        return None
    peak, src = load_peaks()
    achieved = byts.value / (ms.value * 1e-3) / 1e9
    kname = name.value.decode()
    # DRAM bytes per launch of this kernel from the committed ncu capture of
    # the same launch at 256^3 (profiles/fft_passes_c3.md)
    traffic = None
    prof = os.path.join(ROOT, "profiles", "fft_passes_c3.json")
    if args.config == "c3" and os.path.exists(prof):
        key = kname if args.form == "fp64" else f"{kname}:{args.form}"
        traffic = json.load(open(prof))["traffic_bytes_per_launch"].get(key)
    return {"kernel": kname, "bound": "hbm", "achieved": achieved, "peak": peak,
            "peak_source": f"{src} (MEASURED_PEAKS.json hbm_gbs)" if src == "measured" else src,
            "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
            "traffic_source": "ncu dram__bytes, profiles/fft_passes_c3.md" if traffic else None,
            "bytes_per_launch": byts.value, "ms_per_launch": ms.value}


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
                               f"particles, core4=OTC npd=7, plain FP64 predictor-corrector steps"},
        "cpu_baseline": {"value": value, "unit": "simulated ps/hour", "cores": threads, "kind": "port",
                         "sample": f"{steps} PC steps (bounded sample of the {args.config} workload)"},
        "e2e": {"value": value, "unit": "simulated ps/hour", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c3", choices=["c1", "c2", "c3"])
    ap.add_argument("--form", default="fp32", choices=sorted(FORMS))
    ap.add_argument("--all-forms", action=argparse.BooleanOptionalAction, default=True,
                    help="also time the other forms on the same workload")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
