"""Benchmark: RK45 (Cash-Karp, NR step control) steps/s and simulated years per
hour of the 3-D quasi-dynamic boundary-integral model at N = 20,000
Nikkhoo-Walter triangles (curved megathrust, oblique rake, full reference
layout: K is 60,000 x 40,000, 19.2 GB in FP64).

One "step" is one accepted main-loop iteration of the reference
(fortran/3d/src/ratestate.f90:307-326): f(y), yscal, RKQSm attempts until one
is accepted.

Default workload (--workload all): the parsed line is the plain FP64 path --
the reference's algorithm and precision on one instance (ucg_run, state
resident in HBM) -- so that the reference arm (the same main loop on the host
cores) measures the same quantity; `e2e` is the same metric through the
host-array ABI call (ucg_step: state host->device, state and rate back, every
step).  `chosen_forms` holds the forms measured against it on the same model:
split-BF16 K (single instance), 64 frictional parameter sets in one ensemble
(tensor-core K V contraction), the learned step-size proposal, the
hierarchical K and the ensemble on it, each with its speed-up over the plain
FP64 path.  --workload ensemble makes the ensemble the parsed line instead;
--workload plain / split time one single-instance path alone; --workload hens
the ensemble on the hierarchical K alone (no dense K; --nx 200 --nz 200 is
N = 80k), --workload hmatrix the single instance on it; --workload cfg4 the
batched configuration of 4 faults x 64 sets; --workload coupled the
fault + strain-volume assembly.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--workload ...]
Multi-GPU: replicas only (the path runs on one GPU; no inter-GPU collective).
"""
import argparse
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "RK45 steps/s at N=20k (plain FP64, full layout)"
METRIC_ENS = "RK45 steps/s at N=20k, 64-instance ensemble (aggregate)"
N_SETS = 64
YEAR = 3.15576e7


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=60)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--nx", type=int, default=100, help="along-strike cells (2 triangles each per row)")
    p.add_argument("--nz", type=int, default=100, help="down-dip rows")
    p.add_argument("--precision", default="fp64", choices=["fp64", "split_bf16"])
    p.add_argument("--workload", default="all",
                   choices=["all", "ensemble", "plain", "split", "coupled", "cfg1", "cfg3", "cfg4", "hmatrix", "hens"])
    p.add_argument("--cfg3-size", default="64,64,32,16,16",
                   help="cfg3 workload: fault nx,nz and volume nx,ny,nz (full size: 4,096 + 8,192)")
    p.add_argument("--cfg3-steps", type=int, default=2000, help="cfg3 workload: accepted steps per precision")
    p.add_argument("--coupled-size", default="64,64,16,8,8",
                   help="coupled assembly leg: fault nx,nz and volume nx,ny,nz")
    p.add_argument("--sets", type=int, default=N_SETS, help="instances in the ensemble workload")
    p.add_argument("--ens-eager", action="store_true",
                   help="launch the ensemble's attempt kernels from the host instead of one graph launch "
                        "(for ncu, which does not follow conditional graph nodes)")
    p.add_argument("--no-learned", action="store_true", help="skip the learned step-size leg")
    p.add_argument("--no-split", action="store_true", help="skip the single-instance split-BF16 leg")
    p.add_argument("--ens-terms", type=int, default=3, choices=[2, 3],
                   help="ensemble stage increments: 3 (the anchor form, histories within 1e-6 of FP64) or 2 "
                        "(K hi only, half the bytes)")
    p.add_argument("--no-hmatrix", action="store_true", help="skip the hierarchical-matrix leg")
    p.add_argument("--hm-eta", type=float, default=2.0, help="hierarchical matrix: admissibility parameter")
    p.add_argument("--hm-eps", type=float, default=1e-6, help="hierarchical matrix: ACA relative accuracy")
    p.add_argument("--hm-leaf", type=int, default=32, help="hierarchical matrix: patches per cluster leaf")
    p.add_argument("--hm-ens-leaf", type=int, default=40,
                   help="hierarchical ensemble: patches per cluster leaf (at most 42: a row leaf is one 128-row tile)")
    p.add_argument("--no-hier-ensemble", action="store_true", help="skip the hierarchical-ensemble leg")
    p.add_argument("--hier-planes", type=int, default=3, choices=[2, 3],
                   help="hierarchical ensemble: bf16 planes of the operand images, 3 (24 bits, histories within "
                        "1e-6 of FP64) or 2 (16 bits, two thirds of the bytes)")
    p.add_argument("--trace-runs", type=int, default=64, help="seeded cfg1 runs that record training traces")
    p.add_argument("--trace-attempts", type=int, default=16000, help="attempts of the trace-recording runs")
    p.add_argument("--learned-eval-years", type=float, default=15.0,
                   help="simulated years of the held-out comparison (0: train only, no comparison)")
    p.add_argument("--spinup", type=int, default=200,
                   help="untimed accepted steps (plain) / attempts (ensemble) before warm-up, past the start-up "
                        "transient of the step size (from dt0 = 1 ms the step grows at most 5x per step and "
                        "settles after about 100 steps at N = 20k)")
    p.add_argument("--e2e-steps", type=int, default=None)
    p.add_argument("--cpu-seconds", type=float, default=20.0, help="target CPU sample length")
    return p.parse_args()


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(name):
    """DRAM bytes per launch from a committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d.get(name)
    return None


class Clocks:
    """SM clock and throttle reasons sampled through NVML every 20 ms during the
    timed region (nvidia-smi's own loop is too coarse for sub-second regions)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, index):
        self.index = index
        self.sm, self.mx, self.reasons = [], None, set()
        self.stop = threading.Event()
        self.t = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.mx = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))

            def loop():
                while not self.stop.is_set():
                    try:
                        self.sm.append(float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)))
                        r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                        for nm, bit in self.REASONS.items():
                            if r & bit:
                                self.reasons.add(nm)
                    except Exception:
                        pass
                    self.stop.wait(0.02)
            self.t = threading.Thread(target=loop, daemon=True)
            self.t.start()
        except Exception:
            self.t = None
        return self

    def __exit__(self, *a):
        self.stop.set()
        if self.t:
            self.t.join(timeout=2)

    def summary(self):
        return {"sm_mhz": statistics.median(self.sm) if self.sm else None, "sm_max_mhz": self.mx,
                "reasons": sorted(self.reasons), "samples": len(self.sm), "source": "nvml, 20 ms"}


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def reduce_max(x, world, args):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if args.impl == "ours" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---- CPU leg: the oracle restatement on a bounded row-block sample ----------------

def cpu_step_rate(cfg, K_rows, threads, target_s):
    """Steps/s of the oracle's main loop at full size, from a timed row-block
    sample of its matrix-vector product (the step's dominant cost; the reference
    distributes exactly these rows over MPI ranks) plus the O(N) remainder
    timed on the full state."""
    import oracle
    n = K_rows.shape[1]
    m_full = 3 * cfg["n_patch"]
    v = np.random.default_rng(0).standard_normal(n)
    # the sample must stream from DRAM like the full matrix: tile it past 256 MB
    reps_rows = max(1, int(np.ceil(256e6 / K_rows.nbytes)))
    if reps_rows > 1:
        K_rows = np.tile(K_rows, (reps_rows, 1))
    # time the sample matvec with the oracle's OpenMP row-block DGEMV
    reps, t_mv = 0, 0.0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < target_s * 0.8 or reps < 2:
        t1 = time.perf_counter()
        oracle.dgemv_t(K_rows, v, threads)
        t_mv += time.perf_counter() - t1
        reps += 1
    t_mv /= reps
    rows = K_rows.shape[0]
    t_full_mv = t_mv * m_full / rows
    # O(N) remainder: the odefun elementwise parts, RK combinations, error norm
    # and control, timed on the full state without the products
    t_rest = oracle.rk_overhead_seconds(cfg)
    step_s = 6.0 * t_full_mv + t_rest
    sample = (f"{rows} of {m_full} receiver rows x {n} sources (row-block DGEMV, {reps} reps), "
              f"extrapolated x{m_full / rows:.0f}; O(N) remainder timed in full")
    return 1.0 / step_s, sample, t_full_mv


# ---- arms ------------------------------------------------------------------------

def run_reference(args, world, rank):
    """The reference path on the host cores: the oracle restatement (the Fortran
    drivers cannot be compiled here), all threads, same workload and metric."""
    import oracle
    from unicycle_b200 import configs
    if rank != 0:
        return None
    cfg = configs.cfg2(nx=args.nx, nz=args.nz)
    threads = os.cpu_count() or 1
    oracle.build(ref=False)
    i1, i2, i3, v = cfg["mesh"]["tri"]
    M = oracle.Mesh(cfg["mu"], cfg["lam"], tri=(v, i1, i2, i3))
    m_full = 3 * cfg["n_patch"]
    rows = min(m_full, 3 * max(8, min(128, 4 * threads)))
    t0 = time.perf_counter()
    G = oracle.build_g_omp(M, 0, rows, threads)
    t_asm = time.perf_counter() - t0
    rate, sample, _ = cpu_step_rate(cfg, G, threads, args.cpu_seconds)
    n = cfg["n_patch"]
    if args.workload == "ensemble":
        # the reference has no batching: the parameter sets are separate runs,
        # each bound by the same matrix traffic, so the per-run rate is the aggregate
        return {"metric": METRIC_ENS, "value": rate, "unit": "steps/s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 / rate, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded cfg2 curved megathrust; Dc redrawn per parameter set)",
                "impl": "reference",
                "config": {"workload": f"megathrust {n} Nikkhoo-Walter triangles x {args.sets} frictional "
                                       "parameter sets, one ensemble", "n_triangles": n, "instances": args.sets,
                           "K_shape": [3 * n, 2 * n]},
                "cpu_baseline": {"value": rate, "unit": "steps/s", "cores": threads, "kind": "port",
                                 "sample": sample + f"; assembly sample {rows} rows in {t_asm:.1f} s; "
                                 f"{args.sets} separate runs (no batching in the reference) share the same "
                                 "per-step matrix traffic, so the per-run rate is their aggregate"},
                "assembly": {"mentries_per_s": rows * 2 * n / t_asm / 1e6, "sample_rows": rows},
                "e2e": {"value": rate, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return {"metric": METRIC, "value": rate, "unit": "steps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 / rate, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded cfg2 curved megathrust; random Dc)",
            "impl": "reference",
            "config": {"workload": f"megathrust {n} Nikkhoo-Walter triangles, full FP64 layout",
                       "n_triangles": n, "K_shape": [3 * n, 2 * n], "precision": "fp64"},
            "cpu_baseline": {"value": rate, "unit": "steps/s", "cores": threads, "kind": "port",
                             "sample": sample + f"; assembly sample {rows} rows in {t_asm:.1f} s"},
            "assembly": {"mentries_per_s": rows * 2 * n / t_asm / 1e6, "sample_rows": rows},
            "e2e": {"value": rate, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_ours(args, world, rank, local, keep_sim=False, plain_steps=None):
    import torch
    import unicycle_b200
    from unicycle_b200 import configs

    torch.cuda.set_device(local)
    cfg = configs.cfg2(nx=args.nx, nz=args.nz)
    n = cfg["n_patch"]
    sim = unicycle_b200.Simulation(cfg["mu"], cfg["lam"], device=local)
    i1, i2, i3, v = cfg["mesh"]["tri"]
    sim.set_triangles(i1, i2, i3, v)
    fr = cfg["friction"]
    sim.set_friction(fr["Vpl"], fr["rake"], fr["mu0"], fr["sig"], fr["a"], fr["b"], fr["L"], fr["Vo"],
                     fr["damping"])
    sim.set_tolerance(cfg["epsilon"])
    stream = torch.cuda.ExternalStream(sim.stream, device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    sim.buildG()
    e1.record(stream)
    torch.cuda.synchronize()
    t_asm = e0.elapsed_time(e1) / 1e3
    mn = 6 * n * n
    if args.precision != "fp64":
        sim.set_precision(args.precision)
    steps_req = plain_steps or args.steps
    # spin-up past the start-up transient, then warm-up
    sim.set_state(cfg["y0"], 0.0, cfg["dt0"])
    sim.run(1e300, args.spinup + args.warmup)
    y_w, t_w, dt_w, acc_w, rej_w = sim.get_state()
    launches0 = sim.launch_count
    barrier(world)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        e0.record(stream)
        steps = sim.run(1e300, steps_req)
        e1.record(stream)
        torch.cuda.synchronize()
    elapsed = e0.elapsed_time(e1) / 1e3
    launches = sim.launch_count - launches0
    y_t, t_t, dt_t, acc_t, rej_t = sim.get_state()
    elapsed_max = reduce_max(elapsed, world, args)
    # roofline of the dominant kernel (traction product), timed live
    ms_mv = sim.profile_traction(reps=10)
    # the profiled launch is stage 2: FP64 K, or (split) the hi plane of the anchored increments
    K_bytes = 8.0 * (3 * n) * (2 * n) if args.precision == "fp64" else 2.0 * (3 * n) * (2 * n) + 4.0 * 3 * n
    alg_bytes = K_bytes + 8.0 * (2 * n + 3 * n)
    peak, peak_kind = load_peaks()
    achieved = alg_bytes / (ms_mv / 1e3) / 1e9
    # end to end through the host-array ABI call
    e2e_steps = args.e2e_steps or max(10, steps_req // 3)
    y_h, t_h, dt_h = y_t.copy(), t_t, dt_t
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(e2e_steps):
        t_h, y_h, dydt_h, dt_h, _, _ = sim.step(t_h, y_h, dt_h)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_elapsed = reduce_max(e0.elapsed_time(e1) / 1e3, world, args)
    out = None
    if rank == 0:
        value = world * steps / elapsed_max
        cpu = None
        if world == 1:
            K_rows = sim.copy_G(0, 3 * 128) if args.precision == "fp64" else None
            if K_rows is not None:
                rate, sample, _ = cpu_step_rate(cfg, K_rows, os.cpu_count() or 1, args.cpu_seconds)
                cpu = {"value": rate, "unit": "steps/s", "cores": os.cpu_count() or 1, "kind": "port",
                       "sample": sample}
        out = {
            "metric": METRIC if args.precision == "fp64" else "RK45 steps/s at N=20k (split K: fp16 increment plane)",
            "value": value, "unit": "steps/s", "n_gpus": world, "steps": steps_req,
            "warmup": args.warmup, "ms_per_step": 1e3 * elapsed_max / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f16 K increments x f32 / f64 sums",
            "data": "synthetic (seeded cfg2 curved megathrust; random Dc)",
            "config": {"workload": f"megathrust {n} Nikkhoo-Walter triangles, full FP64 layout",
                       "n_triangles": n, "K_shape": [3 * n, 2 * n], "precision": args.precision,
                       "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (K %.1f GB)" % (K_bytes / 1e9),
                       "rtol": cfg["epsilon"]},
            "sim_years_per_hour": (t_t - t_w) / YEAR / (elapsed / 3600.0),
            "rejected_attempts": rej_t - rej_w,
            "assembly": {"seconds": t_asm, "mentries_per_s": mn / t_asm / 1e6, "entries": mn},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": load_traffic("k_traction"),
                         "kernel": "k_traction (FP64 K.v + rate-state epilogue)" if args.precision == "fp64"
                         else "k_traction<S,bf16> (hi plane x velocity increments + rate-state epilogue)",
                         "ms_per_launch": ms_mv, "peak_source": peak_kind,
                         "bytes_per_launch": alg_bytes},
            "e2e": {"value": world * e2e_steps / e2e_elapsed, "unit": "steps/s",
                    "h2d_bytes_per_step": 8 * 7 * n, "d2h_bytes_per_step": 2 * 8 * 7 * n},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
    if keep_sim:
        out = dict(out or {})
        out["_sim"] = sim
        return out
    sim.close()
    return out


def load_tensor_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    return 1590.0, "fallback"


def fp64_peak_tflops(local):
    """Measured FP64 throughput of this GPU: the best of three cuBLAS DGEMMs of
    8,192^3 (2 n^3 flops), the denominator of the assembly kernels' FP64 fraction."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=f"cuda:{local}")
    b = torch.randn(n, n, dtype=torch.float64, device=f"cuda:{local}")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 1e300
    torch.matmul(a, b)
    for _ in range(3):
        torch.cuda.synchronize()
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def load_flops(name):
    """FP64 flops per (receiver, source) pair of an assembly kernel family by
    receiver kind, counted by ncu (dadd + dmul + 2 dfma thread instructions),
    or None."""
    path = os.path.join(ROOT, "profiles", "ncu_flops.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f).get(name)
    return None


def family_fp64(entry, family, peak_tf):
    """flops per entry and FP64 fraction of one assembly family entry (its
    `pairs` by receiver kind times the counted flops per pair)."""
    per_pair = load_flops(family)
    pairs = entry.get("pairs", {})
    if per_pair and pairs and all(k in per_pair for k in pairs):
        flops = sum(per_pair[k] * v for k, v in pairs.items())
        tf = flops / (entry["ms"] * 1e-3) / 1e12
        entry.update({"flops_per_entry": flops / entry["entries"], "fp64_tflops": tf, "fp64_frac": tf / peak_tf})
    else:
        entry["flops_per_entry"] = None
    return entry


def add_fp64_fractions(fam, peak_tf, names=None):
    """flops per entry and FP64 fraction of each assembly family."""
    names = names or {"okada_rect": "okada_rect", "bml17_vol": "bml17_vol", "nikkhoo_tri": "nikkhoo_tri"}
    for key, family in names.items():
        if key in fam and isinstance(fam[key], dict):
            family_fp64(fam[key], family, peak_tf)
    fam["fp64_peak_tflops"] = peak_tf
    fam["fp64_peak_source"] = "measured: cuBLAS DGEMM 8192^3, best of 3 (torch.matmul float64)"
    fam["flops_source"] = "ncu-counted FP64 flops per pair, profiles/ncu_flops.json"
    return fam


def assembly_leg(args, local):
    """Green's-function assembly per source family on a coupled fault + volume
    model (cfg3 geometry, reduced wedge): device time of the rectangle and the
    cuboid columns, in Mentries/s."""
    import unicycle_b200
    from unicycle_b200 import configs
    nxf, nzf, nxv, nyv, nzv = (int(v) for v in args.coupled_size.split(","))
    c = configs.cfg3(nxf=nxf, nzf=nzf, nxv=nxv, nyv=nyv, nzv=nzv)
    sim = unicycle_b200.Simulation(c["mu"], c["lam"], driver="viscouscycles", device=local)
    configs.build_coupled(sim, c)
    rect_ms, _, vol_ms = sim.assembly_times()
    n, m = sim.dims
    nf, nv = c["n_patch"], c["n_vol"]
    sim.close()
    return {"model": f"{nf} rectangles + {nv} cuboids (K {m} x {n})",
            "okada_rect": {"entries": m * 2 * nf, "ms": rect_ms, "mentries_per_s": m * 2 * nf / rect_ms / 1e3,
                           "pairs": {"fault_receiver": nf * nf, "volume_receiver": nv * nf}},
            "bml17_vol": {"entries": m * 6 * nv, "ms": vol_ms, "mentries_per_s": m * 6 * nv / vol_ms / 1e3,
                          "pairs": {"fault_receiver": nf * nv, "volume_receiver": nv * nv}}}


def run_cfg1(args, world, rank, local):
    """The reference's own small configuration run in full: 512 Okada rectangles
    on a vertical strike-slip fault, 300 simulated years, plain FP64 on the
    device (ucg_run, the state resident), with accepted / rejected counts."""
    import torch
    import unicycle_b200
    from unicycle_b200 import configs
    torch.cuda.set_device(local)
    c = configs.cfg1()
    sim = unicycle_b200.Simulation(c["mu"], c["lam"], device=local)
    configs.build(sim, c)
    sim.set_tolerance(c["epsilon"])
    sim.set_state(c["y0"], 0.0, c["dt0"])
    stream = torch.cuda.ExternalStream(sim.stream, device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        e0.record(stream)
        steps = 0
        while True:
            k = sim.run(c["t_end"], 1 << 20)
            steps += k
            _, t, _, acc, rej = sim.get_state()
            if t >= c["t_end"] or k == 0:
                break
        e1.record(stream)
        torch.cuda.synchronize()
    el = reduce_max(e0.elapsed_time(e1) / 1e3, world, args)
    sim.close()
    if rank != 0:
        return None
    return {"metric": "RK45 steps/s, cfg1 full run (512 rectangles, 300 yr, plain FP64)", "value": world * acc / el,
            "unit": "steps/s", "n_gpus": world, "steps": int(acc), "warmup": 0, "ms_per_step": 1e3 * el / acc,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded cfg1: lognormal initial slip rate, seed 1)",
            "config": {"workload": "cfg1 vertical strike-slip fault, 32 x 16 Okada rectangles, rtol 1e-8, 300 yr, "
                                   "full run", "rtol": c["epsilon"]},
            "sim_years": t / YEAR, "sim_years_per_hour": t / YEAR / (el / 3600.0), "accepted": int(acc),
            "rejected": int(rej), "seconds": el, "clocks": clk.summary()}


def run_reference_cfg1(args):
    """cfg1 in full on the host cores: the oracle restatement of the reference
    main loop (ratestate.f90:307-326 with RKQSm), its DGEMV over all threads."""
    import oracle
    from unicycle_b200 import configs
    c = configs.cfg1()
    threads = os.cpu_count() or 1
    oracle.build(ref=False)
    t0 = time.perf_counter()
    G = oracle.build_g_omp(oracle.Mesh(c["mu"], c["lam"], rect=c["mesh"]["rect"]), 0, 3 * c["n_patch"], threads)
    t_asm = time.perf_counter() - t0
    oracle.set_dgemv_threads(threads)
    md = oracle.Model(G, c["friction"])
    y, t, dt = c["y0"].copy(), 0.0, c["dt0"]
    acc = rej = 0
    limit = args.cpu_seconds if args.cpu_seconds > 0 else float("inf")
    t0 = time.perf_counter()
    while t < c["t_end"] and time.perf_counter() - t0 < limit:
        rc, t, y, _, dt, _, nr = md.step(t, y, dt, c["epsilon"])
        if rc:
            break
        acc += 1
        rej += nr
    el = time.perf_counter() - t0
    oracle.set_dgemv_threads(0)
    full = t >= c["t_end"]
    rate = acc / el
    sample = ("full run: 300 simulated years" if full else f"first {t / YEAR:.2f} of 300 simulated years "
              f"({el:.0f} s cap)") + f", {acc} accepted / {rej} rejected steps; assembly {t_asm:.2f} s"
    return {"metric": "RK45 steps/s, cfg1 full run (512 rectangles, 300 yr, plain FP64)", "value": rate,
            "unit": "steps/s", "n_gpus": args.gpus, "steps": acc, "warmup": 0, "ms_per_step": 1e3 / rate,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded cfg1: lognormal initial slip rate, seed 1)", "impl": "reference",
            "config": {"workload": "cfg1 vertical strike-slip fault, 32 x 16 Okada rectangles, rtol 1e-8, 300 yr, "
                                   "full run", "rtol": c["epsilon"]},
            "sim_years": t / YEAR, "sim_years_per_hour": t / YEAR / (el / 3600.0), "accepted": acc, "rejected": rej,
            "seconds": el,
            "cpu_baseline": {"value": rate, "unit": "steps/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": rate, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_cfg3(args, world, rank, local):
    """The coupled configuration at full size: 4,096 rectangular fault patches and
    8,192 cuboids (K 61,440 x 57,344, 28 GB in FP64), linear Maxwell volumes,
    a 5 m uniform coseismic strike slip applied on the device at t = 0 (K u), then
    postseismic relaxation towards 50 years with the plain FP64 path and with
    the split-BF16 K (anchored stages).  Assembly is timed per source family
    (fault columns: fault-fault and fault-volume blocks; volume columns:
    volume-fault and volume-volume blocks)."""
    import torch
    import unicycle_b200
    from unicycle_b200 import configs
    torch.cuda.set_device(local)
    nxf, nzf, nxv, nyv, nzv = (int(v) for v in args.cfg3_size.split(","))
    c = configs.cfg3(nxf=nxf, nzf=nzf, nxv=nxv, nyv=nyv, nzv=nzv)
    nf, nv = c["n_patch"], c["n_vol"]
    sim = unicycle_b200.Simulation(c["mu"], c["lam"], driver="viscouscycles", device=local)
    t0 = time.perf_counter()
    configs.build_coupled(sim, c)
    torch.cuda.synchronize()
    t_build = time.perf_counter() - t0
    rect_ms, _, vol_ms = sim.assembly_times()
    n, m = sim.dims
    fam = {"okada_rect_columns": {"entries": m * 2 * nf, "ms": rect_ms, "mentries_per_s": m * 2 * nf / rect_ms / 1e3,
                                  "blocks": "fault-fault + fault-volume",
                                  "pairs": {"fault_receiver": nf * nf, "volume_receiver": nv * nf}},
           "bml17_vol_columns": {"entries": m * 6 * nv, "ms": vol_ms, "mentries_per_s": m * 6 * nv / vol_ms / 1e3,
                                 "blocks": "volume-fault + volume-volume",
                                 "pairs": {"fault_receiver": nf * nv, "volume_receiver": nv * nv}},
           "total_seconds_incl_host": t_build}
    fam = add_fp64_fractions(fam, fp64_peak_tflops(local),
                             {"okada_rect_columns": "okada_rect", "bml17_vol_columns": "bml17_vol"})
    slip = np.zeros((nf, 2))
    slip[:, 0] = c["coseismic_slip"]
    sim.set_state(c["y0"], 0.0, c["dt0"])
    sim.apply_perturbation(slip=slip)
    y_pre = sim.get_state()[0]
    stream = torch.cuda.ExternalStream(sim.stream, device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    peak, peak_kind = load_peaks()
    t_end = c["t_end"]
    legs = {}
    for prec in ("fp64", "split_bf16"):
        sim.set_precision(prec)
        sim.set_state(y_pre, 0.0, c["dt0"])
        sim.run(t_end, args.warmup)
        _, tw, _, aw, rw = sim.get_state()
        torch.cuda.synchronize()
        with Clocks(local) as clk:
            e0.record(stream)
            steps = sim.run(t_end, args.cfg3_steps)
            e1.record(stream)
            torch.cuda.synchronize()
        el = e0.elapsed_time(e1) / 1e3
        y, tt, _, at, rt = sim.get_state()
        ms_mv = sim.profile_traction(reps=5)
        if prec == "fp64":
            alg = 8.0 * m * n + 8.0 * (n + m)
        else:
            alg = 2.0 * m * n + 4.0 * m + 8.0 * (n + m)
        legs[prec] = {"steps": steps, "steps_per_s": steps / el, "ms_per_step": 1e3 * el / max(1, steps),
                      "sim_years": (tt - tw) / YEAR, "reached_years": tt / YEAR,
                      "sim_years_per_hour": (tt - tw) / YEAR / (el / 3600.0), "rejected_attempts": rt - rw,
                      "roofline": {"bound": "hbm", "ms_per_launch": ms_mv, "bytes_per_launch": alg,
                                   "achieved": alg / (ms_mv / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                                   "frac": alg / (ms_mv / 1e3) / 1e9 / peak, "peak_source": peak_kind,
                                   "kernel": "k_traction<S,double>" if prec == "fp64" else
                                   "k_traction<S,bf16> (hi plane x increments)"},
                      "clocks": clk.summary(), "final_state_finite": bool(np.all(np.isfinite(y)))}
    # split product error against FP64 on the preloaded state
    sim.set_precision("fp64")
    d64, _ = sim.odefun(y_pre)
    sim.set_precision("split_bf16")
    dsp, _ = sim.odefun(y_pre)
    sim.set_precision("fp64")
    idx_f = np.concatenate([np.arange(q, 7 * nf, 7) for q in (2, 3, 4)])
    vol = np.arange(7 * nf, len(y_pre)).reshape(-1, 12)[:, 6:].ravel()
    legs["split_bf16"]["rhs_max_rel_error_vs_fp64"] = {
        "fault_traction_rates": float(np.max(np.abs(dsp[idx_f] - d64[idx_f])) / np.max(np.abs(d64[idx_f]))),
        "volume_stress_rates": float(np.max(np.abs(dsp[vol] - d64[vol])) / np.max(np.abs(d64[vol])))}
    sim.close()
    if rank != 0:
        return None
    p64 = legs["fp64"]
    return {"metric": "simulated years/hour, coupled fault + strain volumes (plain FP64)",
            "value": world * p64["sim_years_per_hour"], "unit": "sim-yr/hr", "n_gpus": world,
            "steps": p64["steps"], "warmup": args.warmup, "ms_per_step": p64["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded cfg3: viscosity log-uniform 1e18-1e20 Pa s)",
            "config": {"workload": f"{nf} Okada rectangles + {nv} cuboids, linear Maxwell, 5 m coseismic preload, "
                                   f"relaxation towards {t_end / YEAR:.0f} yr", "K_shape": [m, n],
                       "K_gb_fp64": 8.0 * m * n / 1e9, "rtol": c["epsilon"],
                       "l2": "inputs larger than L2 (K %.1f GB)" % (8.0 * m * n / 1e9)},
            "assembly": fam, "plain_fp64": p64, "split_bf16": legs["split_bf16"],
            "speedup_split_vs_fp64": {"steps_per_s": legs["split_bf16"]["steps_per_s"] / p64["steps_per_s"],
                                      "sim_years_per_hour": legs["split_bf16"]["sim_years_per_hour"] /
                                      max(1e-300, p64["sim_years_per_hour"])},
            "roofline": p64["roofline"], "clocks": p64["clocks"], "gpu_launches": None}


def run_cfg4(args, world, rank, local):
    """The batched-ensemble configuration: 4 fault geometries of 1,024 to 4,096
    rectangles x 64 frictional parameter sets in one ensemble (256 instances),
    against the plain FP64 single-instance path run over the same instances one
    after another (estimated from one instance per geometry)."""
    import torch
    import unicycle_b200
    from unicycle_b200 import configs
    torch.cuda.set_device(local)
    cfg = configs.cfg4()
    ens = unicycle_b200.Ensemble(device=local)
    configs.build_ensemble(ens, cfg, lambda mu, lam: unicycle_b200.Simulation(mu, lam, device=local))
    report = ens.tune(reps=3)
    stream = torch.cuda.ExternalStream(ens.stream, device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    spin = max(args.spinup, 300)   # past the start-up transient of the step size (dt0 = 1 ms)
    ens.run(cfg["t_end"], spin + args.warmup)
    i0 = ens.info()
    barrier(world)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        e0.record(stream)
        attempts = ens.run(cfg["t_end"], args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
    elapsed = reduce_max(e0.elapsed_time(e1) / 1e3, world, args)
    i1 = ens.info()
    ens.close()
    acc, rej = i1["accepted"] - i0["accepted"], i1["rejected"] - i0["rejected"]
    syh = (i1["time_sum"] - i0["time_sum"]) / YEAR / (elapsed / 3600.0)
    # plain FP64: one instance per geometry, same spin-up, same number of steps
    plain = []
    for g in cfg["geoms"]:
        sim = unicycle_b200.Simulation(g["mu"], g["lam"], device=local)
        configs.build(sim, g)
        sim.set_state(g["y0s"][0], 0.0, cfg["dt0"])
        sim.run(cfg["t_end"], spin + args.warmup)
        _, t0, _, a0, _ = sim.get_state()
        st = torch.cuda.ExternalStream(sim.stream, device=local)
        torch.cuda.synchronize()
        e0.record(st)
        n = sim.run(cfg["t_end"], max(5, args.steps // 2))
        e1.record(st)
        torch.cuda.synchronize()
        sec = e0.elapsed_time(e1) / 1e3
        _, t1, _, a1, _ = sim.get_state()
        plain.append({"patches": g["n_patch"], "steps_per_s": n / sec, "sim_years_per_hour": (t1 - t0) / YEAR / (sec / 3600)})
        sim.close()
    # the 256 instances one after another on the plain path
    per_step = sum(64.0 / p["steps_per_s"] for p in plain) / 256.0
    plain_agg = 1.0 / per_step
    plain_syh = sum(p["sim_years_per_hour"] for p in plain) / 4.0
    if rank != 0:
        return None
    return {"metric": "RK45 steps/s, cfg4 batched ensemble (aggregate over 256 instances)", "value": world * acc / elapsed,
            "unit": "steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * elapsed / attempts, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16x3/f32 product, f64 state", "data": "synthetic (seeded cfg4: 4 faults x 64 parameter sets)",
            "config": {"workload": "4 rectangle faults (1,024 / 2,048 / 3,072 / 4,096 patches) x 64 frictional "
                                   "parameter sets, one ensemble", "plan": i1["plan"], "rtol": cfg["epsilon"],
                       "step": "one attempt of every instance"},
            "sim_years_per_hour": world * syh, "accepted_steps": acc, "rejected_fraction": rej / max(1, acc + rej),
            "plain_fp64": {"per_geometry": plain, "aggregate_steps_per_s": plain_agg,
                           "sim_years_per_hour_per_instance": plain_syh},
            "speedup_vs_plain_fp64": {"steps_per_s": acc / elapsed / plain_agg,
                                      "sim_years_per_hour": syh / plain_syh if plain_syh > 0 else None},
            "autotune": report.strip().splitlines(), "clocks": clk.summary(), "gpu_launches": int(attempts * 20 + 3)}


def learned_leg(args, local, sim20, sets, y0s, plain_window):
    """The learned step-size proposal: traces from seeded cfg1 runs train the
    perceptron on the device; it is then compared with the plain controller on
    held-out cfg1 seeds (to 15 simulated years) and on the N = 20k ensemble
    over the same attempt window as the headline run."""
    import torch
    import unicycle_b200
    from unicycle_b200 import configs
    from unicycle_b200.stepmodel import training_set

    def cuda_time(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        return r, time.perf_counter() - t0

    c1, y_train = configs.cfg1_instances(range(100, 100 + args.trace_runs))
    _, y_test = configs.cfg1_instances(range(200, 216))
    sim1 = unicycle_b200.Simulation(c1["mu"], c1["lam"], device=local)
    configs.build(sim1, c1)
    f1 = c1["friction"]

    def ens1(y0s_, model):
        e = unicycle_b200.Ensemble(device=local)
        e.add_geometry(sim1, len(y0s_))
        for i, y0 in enumerate(y0s_):
            e.set_friction(0, i, f1["Vpl"], f1["rake"], f1["mu0"], f1["sig"], f1["a"], f1["b"], f1["L"], f1["Vo"],
                           f1["damping"])
        e.set_states(0, np.stack(y0s_), 0.0, c1["dt0"])
        e.set_tolerance(c1["epsilon"])
        e.set_step_model(model)
        return e

    tr = ens1(y_train, None)
    tr.record_traces(int(1.1 * args.trace_runs * args.trace_attempts))
    _, t_traces = cuda_time(lambda: tr.run(300 * YEAR, args.trace_attempts))
    traces = tr.traces()
    tr.close()
    x, y = training_set(traces)
    model = unicycle_b200.StepModel(device=local, seed=1)
    model.set_data(x, y)
    losses, t_train = cuda_time(lambda: model.train(epochs=20, batch=4096, lr=1e-3))
    out = {"traces": int(len(traces)), "trace_runs": args.trace_runs, "trace_seconds": t_traces,
           "train_epochs": 20, "train_seconds": t_train, "loss_first_last": [float(losses[0]), float(losses[-1])]}
    if args.learned_eval_years <= 0:
        sim1.close()
        model.close()
        return out
    # held-out cfg1 runs
    t_end = args.learned_eval_years * YEAR
    held = {}
    for name, mdl in (("plain", None), ("learned", model)):
        e = ens1(y_test, mdl)
        _, secs = cuda_time(lambda: e.run(t_end, 400000))
        _, t, _, acc, rej, st = e.get_states(0)
        onsets = np.array([e.events(0, i)[1] for i in range(len(y_test))])
        held[name] = dict(attempts=int(np.sum(acc + rej)), rejected_fraction=float(np.sum(rej) / np.sum(acc + rej)),
                          seconds=secs, seconds_per_sim_year=secs / (args.learned_eval_years * len(y_test)),
                          onsets=onsets)
        e.close()
    ok = (held["plain"]["onsets"] > 0) & (held["learned"]["onsets"] > 0)
    rel = np.abs(held["learned"]["onsets"] - held["plain"]["onsets"])[ok] / held["plain"]["onsets"][ok]
    for h in held.values():
        h.pop("onsets")
    out["held_out_cfg1"] = {"runs": len(y_test), "t_end_years": args.learned_eval_years, **held,
                            "attempt_ratio_plain_over_learned": held["plain"]["attempts"] / held["learned"]["attempts"],
                            "wallclock_gain_per_sim_year": held["plain"]["seconds"] / held["learned"]["seconds"],
                            "max_onset_rel_diff": float(rel.max()) if len(rel) else None}
    sim1.close()
    # the N = 20k ensemble over the headline's attempt window, same start
    e = unicycle_b200.Ensemble(device=local)
    e.add_geometry(sim20, len(sets))
    for i, fr in enumerate(sets):
        e.set_friction(0, i, fr["Vpl"], fr["rake"], fr["mu0"], fr["sig"], fr["a"], fr["b"], fr["L"], fr["Vo"],
                       fr["damping"])
    e.set_states(0, np.stack(y0s), 0.0, configs.cfg2(nx=args.nx, nz=args.nz)["dt0"])
    e.set_tolerance(1.0e-8)
    e.set_step_model(model)
    e.run(1e300, plain_window["before"])
    i0 = e.info()
    _, secs = cuda_time(lambda: e.run(1e300, plain_window["attempts"]))
    i1 = e.info()
    acc, rej = i1["accepted"] - i0["accepted"], i1["rejected"] - i0["rejected"]
    syh = (i1["time_sum"] - i0["time_sum"]) / YEAR / (secs / 3600.0)
    out["megathrust_20k_ensemble"] = {
        "attempts": plain_window["attempts"], "learned": {"accepted": acc, "rejected_fraction": rej / max(1, acc + rej),
                                                          "sim_years_per_hour": syh},
        "plain": {"accepted": plain_window["accepted"],
                  "rejected_fraction": plain_window["rejected"] / max(1, plain_window["accepted"] +
                                                                     plain_window["rejected"]),
                  "sim_years_per_hour": plain_window["sim_years_per_hour"]}}
    e.close()
    model.close()
    return out


def hmatrix_leg(args, local, sim, cfg, plain):
    """The same N = 20k model with its K replaced by the hierarchical
    approximation (ucg_build_hmatrix): build, storage, accuracy on a row block
    of the dense K, the product's bandwidth and the plain integrator's steps/s
    against the dense FP64 path."""
    import torch
    import unicycle_b200
    n = cfg["n_patch"]
    m, nn = 3 * n, 2 * n
    t0 = time.perf_counter()
    sim.build_hmatrix(eta=args.hm_eta, eps=args.hm_eps, leaf=args.hm_leaf)
    build_s = time.perf_counter() - t0
    info = sim.hmatrix_info()
    x = np.random.default_rng(3).standard_normal(nn)
    Kr = sim.copy_G(0, 3 * 256)
    y = sim.hmatrix_matvec(x)[:3 * 256]
    ref = Kr @ x
    err = float(np.linalg.norm(y - ref) / np.linalg.norm(ref))
    ms = sim.hmatrix_profile(20)
    alg = info["bytes"] + 8.0 * (nn + m)
    peak, peak_kind = load_peaks()
    sim.set_precision(unicycle_b200.UCG_PREC_HMATRIX)
    stream = torch.cuda.ExternalStream(sim.stream, device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sim.set_state(cfg["y0"], 0.0, cfg["dt0"])
    sim.run(1e300, args.spinup + args.warmup)
    _, t_w, *_ = sim.get_state()
    steps_req = max(10, args.steps // 2)
    torch.cuda.synchronize()
    e0.record(stream)
    steps = sim.run(1e300, steps_req)
    e1.record(stream)
    torch.cuda.synchronize()
    el = e0.elapsed_time(e1) / 1e3
    _, t_t, *_ = sim.get_state()
    # the same on the split (bf16 hi + lo) copy with anchored stages
    sim.set_precision(unicycle_b200.UCG_PREC_HMATRIX_SPLIT)
    sim.set_state(cfg["y0"], 0.0, cfg["dt0"])
    sim.run(1e300, args.spinup + args.warmup)
    _, ts_w, *_ = sim.get_state()
    torch.cuda.synchronize()
    e0.record(stream)
    steps_s = sim.run(1e300, steps_req)
    e1.record(stream)
    torch.cuda.synchronize()
    el_s = e0.elapsed_time(e1) / 1e3
    _, ts_t, *_ = sim.get_state()
    sim.set_precision(unicycle_b200.UCG_PREC_FP64)
    split = {"steps_per_s": steps_s / el_s, "ms_per_step": 1e3 * el_s / steps_s,
             "speedup_vs_plain_fp64_steps": steps_s / el_s / plain["value"],
             "sim_years_per_hour": (ts_t - ts_w) / YEAR / (el_s / 3600.0),
             "bytes_per_stage": info["bytes"] / 2,
             "note": "the FP32 value of every stored entry in two 16-bit planes (bf16 hi bits + 16-bit lo "
                     "extension), read by every stage (anchored stages, FP64 sums)"}
    return {"eta": args.hm_eta, "eps": args.hm_eps, "leaf": args.hm_leaf, "build_seconds": build_s,
            "blocks_dense": info["n_dense"], "blocks_lowrank": info["n_lowrank"], "max_rank": info["max_rank"],
            "bytes": info["bytes"], "compression_vs_dense_fp64": info["compression"],
            "product_rel_error_rows_0_767": err,
            "steps_per_s": steps / el, "ms_per_step": 1e3 * el / steps,
            "speedup_vs_plain_fp64_steps": steps / el / plain["value"],
            "sim_years_per_hour": (t_t - t_w) / YEAR / (el / 3600.0),
            "split": split,
            "roofline": {"bound": "hbm", "kernel": "hierarchical product (k_hm_gather, k_hm_z, k_hm_rows, "
                                                   "k_hm_reduce)", "ms_per_launch": ms, "bytes_per_launch": alg,
                         "achieved": alg / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / (ms / 1e3) / 1e9 / peak, "peak_source": peak_kind}}


def split_leg(args, local, sim, cfg, plain):
    """The single-instance split forms on the same N = 20k model, K = diag(s) k:
    split_bf16 anchors every step on the FP32 pair plane of k and contracts the
    stage increments against an fp16 plane (a quarter of the FP64 bytes at
    stages 2-6); split_pair uses the pair plane for every stage (half of the FP64
    bytes; histories within 1e-6 of FP64).  Steps/s and simulated years per hour
    over the same window as the plain FP64 leg, the traction launch against the
    HBM roofline, and the right-hand side's error against FP64."""
    import torch
    import unicycle_b200
    n = cfg["n_patch"]
    y_probe = sim.get_state()[0]
    d64, _ = sim.odefun(y_probe)
    idx = np.concatenate([np.arange(q, len(y_probe), 7) for q in (2, 3, 4)])
    stream = torch.cuda.ExternalStream(sim.stream, device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    peak, peak_kind = load_peaks()
    out = {}
    for form in ("split_bf16", "split_pair"):
        sim.set_precision(form)
        dsp, _ = sim.odefun(y_probe)
        rhs_err = float(np.max(np.abs(dsp[idx] - d64[idx])) / np.max(np.abs(d64[idx])))
        sim.set_state(cfg["y0"], 0.0, cfg["dt0"])
        sim.run(1e300, args.spinup + args.warmup)
        _, t_w, _, _, rej_w = sim.get_state()
        steps_req = plain["steps"]
        torch.cuda.synchronize()
        e0.record(stream)
        steps = sim.run(1e300, steps_req)
        e1.record(stream)
        torch.cuda.synchronize()
        el = e0.elapsed_time(e1) / 1e3
        _, t_t, _, _, rej_t = sim.get_state()
        ms_mv = sim.profile_traction(reps=10)   # a stage-2 launch: the increment plane (bf16) or the pair plane
        if form == "split_bf16":
            alg = 2.0 * (3 * n) * (2 * n) + 4.0 * 3 * n + 8.0 * (2 * n + 3 * n)
            kern = "k_traction<S,__half> (fp16 increment plane x FP32 velocity increments, 8-term FP32 sums added in FP64)"
        else:
            alg = 4.0 * (3 * n) * (2 * n) + 4.0 * 3 * n + 8.0 * (2 * n + 3 * n)
            kern = "k_traction<S,float> (FP32 pair plane, FP64 sums)"
        syh = (t_t - t_w) / YEAR / (el / 3600.0)
        out[form] = {"steps_per_s": steps / el, "ms_per_step": 1e3 * el / steps, "steps": steps,
                     "sim_years_per_hour": syh, "rejected_attempts": rej_t - rej_w,
                     "speedup_vs_plain_fp64": {"steps_per_s": steps / el / plain["value"],
                                               "sim_years_per_hour": syh / plain["sim_years_per_hour"]
                                               if plain["sim_years_per_hour"] > 0 else None},
                     "rhs_traction_rate_max_rel_error_vs_fp64": rhs_err,
                     "roofline": {"bound": "hbm", "kernel": kern, "ms_per_launch": ms_mv, "bytes_per_launch": alg,
                                  "achieved": alg / (ms_mv / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                                  "frac": alg / (ms_mv / 1e3) / 1e9 / peak, "peak_source": peak_kind}}
    sim.set_precision(unicycle_b200.UCG_PREC_FP64)
    out["split_bf16"]["dtype"] = "FP32 pair anchor, fp16 increments, FP64 sums, f64 state"
    out["split_pair"]["dtype"] = "FP32 pair every stage, FP64 sums, f64 state"
    return out


def hier_ensemble_leg(args, local, cfg, sets, y0s, dense, Kr):
    """The headline ensemble with K replaced by its hierarchical approximation
    (a context that never assembles the dense K): the two-pass tcgen05
    contraction over the hierarchical operand images, timed the same way as
    the dense ensemble, its contraction's bandwidth, and its accuracy against
    the FP64 hierarchical product and the dense K's first rows."""
    import torch
    import unicycle_b200
    n = cfg["n_patch"]
    nn = 2 * n
    sim = unicycle_b200.Simulation(cfg["mu"], cfg["lam"], device=local)
    i1, i2, i3, v = cfg["mesh"]["tri"]
    sim.set_triangles(i1, i2, i3, v)
    t0 = time.perf_counter()
    sim.build_hmatrix(eta=args.hm_eta, eps=args.hm_eps, leaf=args.hm_ens_leaf)
    build_s = time.perf_counter() - t0
    info = sim.hmatrix_info()
    sim.set_precision(unicycle_b200.UCG_PREC_HMATRIX)
    ens = unicycle_b200.Ensemble(device=local)
    ens.set_hier_planes(args.hier_planes)
    t0 = time.perf_counter()
    ens.add_geometry(sim, args.sets)
    images_s = time.perf_counter() - t0
    for i, (fr, y0) in enumerate(zip(sets, y0s)):
        ens.set_friction(0, i, fr["Vpl"], fr["rake"], fr["mu0"], fr["sig"], fr["a"], fr["b"], fr["L"], fr["Vo"],
                         fr["damping"])
        ens.set_state(0, i, y0, 0.0, cfg["dt0"])
    ens.set_tolerance(cfg["epsilon"])
    ens.set_increment_terms(args.ens_terms)
    stream = torch.cuda.ExternalStream(ens.stream, device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ens.run(1e300, args.spinup + args.warmup)
    i0 = ens.info()
    torch.cuda.synchronize()
    e0.record(stream)
    attempts = ens.run(1e300, args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    el = e0.elapsed_time(e1) / 1e3
    i1 = ens.info()
    acc = i1["accepted"] - i0["accepted"]
    rej = i1["rejected"] - i0["rejected"]
    ms_a, ms_c = ens.profile_contract(10)
    plan = i1["plan"]
    img = float(plan.split("images ")[1].split(" GB")[0]) * 1e9 if "images " in plan else None
    peak, peak_kind = load_peaks()
    # accuracy: instances 0-2 against the FP64 hierarchical product, and the
    # first 768 rows against the dense K (the approximation's error included)
    V = np.random.default_rng(7).standard_normal((args.sets, nn)) * 1e-9
    T = ens.matvec(0, V)
    T2 = ens.matvec(0, V, terms=2)
    ref = np.stack([sim.hmatrix_matvec(V[i]) for i in range(3)])
    e_h = float(max(np.linalg.norm(T[i] - ref[i]) / np.linalg.norm(ref[i]) for i in range(3)))
    e_h2 = float(max(np.linalg.norm(T2[i] - ref[i]) / np.linalg.norm(ref[i]) for i in range(3)))
    mag = np.abs(V) @ np.abs(Kr).T
    e_k = float(np.max(np.abs(T[:, :Kr.shape[0]] - V @ Kr.T) / mag))
    ens.close()
    sim.close()
    out = {"leaf": args.hm_ens_leaf, "eta": args.hm_eta, "eps": args.hm_eps, "planes": args.hier_planes,
           "hmatrix_build_seconds": build_s,
           "images_seconds": images_s, "hmatrix_fp64_bytes": info["bytes"], "image_bytes": img,
           "steps_per_s": acc / el, "ms_per_attempt": 1e3 * el / attempts, "accepted_steps": acc,
           "rejected_attempts": rej,
           "speedup_vs_dense_ensemble_ms_per_attempt": dense["ms_per_step"] / (1e3 * el / attempts),
           "speedup_vs_plain_fp64_steps": acc / el / dense["plain_value"],
           "plan": plan,
           "contraction_ms": {"anchor": ms_a, "increment": ms_c},
           "rel_l2_error_vs_fp64_hmatrix": {"anchor": e_h, "increment_form": e_h2},
           "max_rel_to_abs_product_vs_dense_K_rows_0_767": e_k}
    if img:
        out["roofline"] = hier_roofline(args, img, ms_a, ms_c, peak, peak_kind)
    return out


def hier_roofline(args, img, ms_a, ms_c, peak, peak_kind):
    """The hierarchical contraction in the form every stage of the run takes:
    all planes of the operand images (three planes, or two with the anchor's
    form at every stage), else the hi planes of the two-term increments."""
    full = args.hier_planes == 3 or args.ens_terms == 3
    byt, ms = (img, ms_a) if full else (img / 2, ms_c)
    kern = (f"k_hm_contract<64,true,{args.hier_planes}> x2 + k_hm_zconv (every operand plane)" if full else
            "k_hm_contract<64,false,2> x2 + k_hm_zconv (increment form; operand hi planes)")
    return {"bound": "hbm", "kernel": kern, "ms_per_launch": ms, "bytes_per_launch": byt,
            "achieved": byt / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
            "frac": byt / (ms / 1e3) / 1e9 / peak, "peak_source": peak_kind,
            "traffic": load_traffic("k_hm_contract_3planes") if args.hier_planes == 3 and args.nx * args.nz == 10000
            else None}


def run_hier_ensemble(args, world, rank, local):
    """--workload hens: args.sets frictional parameter sets of the cfg2
    megathrust at --nx x --nz cells in one ensemble on the hierarchical K alone
    (no dense K is assembled; at 200 x 200 = 80,000 triangles the dense FP64 K
    would be 307 GB).  value = accepted steps/s summed over the instances."""
    import torch
    import unicycle_b200
    from unicycle_b200 import configs
    torch.cuda.set_device(local)
    cfg = configs.cfg2(nx=args.nx, nz=args.nz)
    n = cfg["n_patch"]
    m, nn = 3 * n, 2 * n
    sets, y0s = configs.parameter_sets(cfg, args.sets)
    sim = unicycle_b200.Simulation(cfg["mu"], cfg["lam"], device=local)
    i1, i2, i3, v = cfg["mesh"]["tri"]
    sim.set_triangles(i1, i2, i3, v)
    t0 = time.perf_counter()
    sim.build_hmatrix(eta=args.hm_eta, eps=args.hm_eps, leaf=args.hm_ens_leaf)
    build_s = time.perf_counter() - t0
    info = sim.hmatrix_info()
    sim.set_precision(unicycle_b200.UCG_PREC_HMATRIX)
    ens = unicycle_b200.Ensemble(device=local)
    ens.set_hier_planes(args.hier_planes)
    t0 = time.perf_counter()
    ens.add_geometry(sim, args.sets)
    images_s = time.perf_counter() - t0
    for i, (fr, y0) in enumerate(zip(sets, y0s)):
        ens.set_friction(0, i, fr["Vpl"], fr["rake"], fr["mu0"], fr["sig"], fr["a"], fr["b"], fr["L"], fr["Vo"],
                         fr["damping"])
        ens.set_state(0, i, y0, 0.0, cfg["dt0"])
    ens.set_tolerance(cfg["epsilon"])
    ens.set_increment_terms(args.ens_terms)
    if args.ens_eager:
        ens.use_graph(False)
    stream = torch.cuda.ExternalStream(ens.stream, device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ens.run(1e300, args.spinup + args.warmup)
    i0 = ens.info()
    barrier(world)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        e0.record(stream)
        attempts = ens.run(1e300, args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
    el = e0.elapsed_time(e1) / 1e3
    el_max = reduce_max(el, world, args)
    i1 = ens.info()
    acc = i1["accepted"] - i0["accepted"]
    rej = i1["rejected"] - i0["rejected"]
    sim_years = (i1["time_sum"] - i0["time_sum"]) / YEAR
    ms_a, ms_c = ens.profile_contract(10)
    plan = i1["plan"]
    img = float(plan.split("images ")[1].split(" GB")[0]) * 1e9
    peak, peak_kind = load_peaks()
    # accuracy against the FP64 hierarchical product (instances 0-2)
    V = np.random.default_rng(7).standard_normal((args.sets, nn)) * 1e-9
    T = ens.matvec(0, V)
    ref = np.stack([sim.hmatrix_matvec(V[i]) for i in range(3)])
    err = float(max(np.linalg.norm(T[i] - ref[i]) / np.linalg.norm(ref[i]) for i in range(3)))
    # end to end: every attempt, all instances' states host->device (pinned) and back
    e2e_att = args.e2e_steps or max(10, args.steps // 3)
    pin = torch.empty((args.sets, 7 * n), dtype=torch.float64, pin_memory=True).numpy()
    y_h, t_h, dt_h, acc0, *_r = ens.get_states(0, out=pin)
    acc0 = int(acc0.sum())
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_att):
        ens.put_states(0, y_h)
        ens.run(1e300, 1)
        y_h, t_h, dt_h, acc_h, rej_h, st_h = ens.get_states(0, out=pin)
    torch.cuda.synchronize()
    acc_e2e = int(acc_h.sum()) - acc0
    e2e_el = reduce_max(time.perf_counter() - t0, world, args)
    ens.close()
    sim.close()
    if rank != 0:
        return None
    return {"metric": f"RK45 steps/s at N={n}, {args.sets}-instance ensemble on the hierarchical K (aggregate)",
            "value": world * acc / el_max, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * el_max / attempts, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": f"bf16 x {args.hier_planes} planes / f32 product, f64 state",
            "data": "synthetic (seeded cfg2 curved megathrust; Dc redrawn per parameter set)",
            "config": {"workload": f"megathrust {n} Nikkhoo-Walter triangles x {args.sets} frictional parameter "
                                   "sets, one ensemble, hierarchical K only", "n_triangles": n,
                       "planes": args.hier_planes,
                       "instances": args.sets, "K_shape": [m, nn], "dense_fp64_bytes": 8.0 * m * nn,
                       "step": "one attempt of every instance (timed steps = attempts)",
                       "parallelism": f"replicas x{world}", "rtol": cfg["epsilon"],
                       "l2": "inputs larger than L2 (operand images %.2f GB)" % (img / 1e9), "plan": plan},
            "sim_years_per_hour": world * sim_years / (el_max / 3600.0),
            "accepted_steps": acc, "rejected_attempts": rej,
            "hmatrix": {"build_seconds": build_s, "images_seconds": images_s, "eta": args.hm_eta,
                        "eps": args.hm_eps, "leaf": args.hm_ens_leaf,
                        **{k: info[k] for k in ("n_dense", "n_lowrank", "max_rank", "bytes", "compression")}},
            "rel_l2_error_vs_fp64_hmatrix": err,
            "roofline": hier_roofline(args, img, ms_a, ms_c, peak, peak_kind),
            "e2e": {"value": world * acc_e2e / e2e_el, "unit": "steps/s",
                    "h2d_bytes_per_step": 8 * 7 * n * args.sets, "d2h_bytes_per_step": 8 * 7 * n * args.sets},
            "gpu_launches": int(attempts * 32 + 3), "clocks": clk.summary(), "cpu_baseline": None}


def run_hmatrix(args, world, rank, local):
    """--workload hmatrix: the cfg2 megathrust at --nx x --nz cells held only as
    its hierarchical approximation (no dense K; at 200 x 200 = 80,000 triangles
    the dense FP64 K would be 307 GB, beyond the B200's HBM)."""
    import torch
    import unicycle_b200
    from unicycle_b200 import configs
    torch.cuda.set_device(local)
    cfg = configs.cfg2(nx=args.nx, nz=args.nz)
    n = cfg["n_patch"]
    m, nn = 3 * n, 2 * n
    sim = unicycle_b200.Simulation(cfg["mu"], cfg["lam"], device=local)
    i1, i2, i3, v = cfg["mesh"]["tri"]
    sim.set_triangles(i1, i2, i3, v)
    fr = cfg["friction"]
    sim.set_friction(fr["Vpl"], fr["rake"], fr["mu0"], fr["sig"], fr["a"], fr["b"], fr["L"], fr["Vo"],
                     fr["damping"])
    sim.set_tolerance(cfg["epsilon"])
    t0 = time.perf_counter()
    sim.build_hmatrix(eta=args.hm_eta, eps=args.hm_eps, leaf=args.hm_leaf)
    build_s = time.perf_counter() - t0
    info = sim.hmatrix_info()
    split = args.precision == "split_bf16"
    sim.set_precision(unicycle_b200.UCG_PREC_HMATRIX_SPLIT if split else unicycle_b200.UCG_PREC_HMATRIX)
    stream = torch.cuda.ExternalStream(sim.stream, device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sim.set_state(cfg["y0"], 0.0, cfg["dt0"])
    sim.run(1e300, args.spinup + args.warmup)
    _, t_w, *_ = sim.get_state()
    launches0 = sim.launch_count
    barrier(world)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        e0.record(stream)
        steps = sim.run(1e300, args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
    el = e0.elapsed_time(e1) / 1e3
    launches = sim.launch_count - launches0
    el_max = reduce_max(el, world, args)
    y_t, t_t, dt_t, *_ = sim.get_state()
    ms = sim.hmatrix_profile(10)
    alg = info["bytes"] + 8.0 * (nn + m)
    peak, peak_kind = load_peaks()
    e2e_steps = max(3, args.steps // 6)
    y_h, t_h, dt_h = y_t.copy(), t_t, dt_t
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(e2e_steps):
        t_h, y_h, _, dt_h, _, _ = sim.step(t_h, y_h, dt_h)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_el = reduce_max(e0.elapsed_time(e1) / 1e3, world, args)
    sim.close()
    if rank != 0:
        return None
    return {"metric": METRIC, "value": world * steps / el_max, "unit": "steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el_max / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16x2/f64 sums" if split else "f64",
            "data": "synthetic (seeded cfg2 curved megathrust; random Dc)",
            "config": {"workload": f"megathrust {n} Nikkhoo-Walter triangles, hierarchical K only"
                                   + (" (bf16 hi + lo, anchored stages)" if split else ""),
                       "n_triangles": n, "K_shape": [m, nn], "dense_fp64_bytes": 8.0 * m * nn,
                       "parallelism": f"replicas x{world}", "rtol": cfg["epsilon"],
                       "l2": "inputs larger than L2 (H %.1f GB)" % (info["bytes"] / 1e9)},
            "sim_years_per_hour": (t_t - t_w) / YEAR / (el / 3600.0),
            "hmatrix": {"build_seconds": build_s, "eta": args.hm_eta, "eps": args.hm_eps, "leaf": args.hm_leaf,
                        **{k: info[k] for k in ("n_dense", "n_lowrank", "max_rank", "bytes", "compression")}},
            "roofline": {"bound": "hbm", "kernel": "hierarchical product (k_hm_gather, k_hm_z, k_hm_rows, "
                                                   "k_hm_reduce)", "ms_per_launch": ms, "bytes_per_launch": alg,
                         "achieved": alg / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / (ms / 1e3) / 1e9 / peak, "peak_source": peak_kind, "traffic": None},
            "e2e": {"value": world * e2e_steps / e2e_el, "unit": "steps/s", "h2d_bytes_per_step": 8 * 7 * n,
                    "d2h_bytes_per_step": 2 * 8 * 7 * n},
            "gpu_launches": int(launches), "clocks": clk.summary(), "cpu_baseline": None}


def ens_roofline(args, ms_a, ms_c, a_bytes, a_flops, c_bytes, c_flops, peak, peak_kind, tpeak, tpeak_kind):
    """Roofline of the ensemble's dominant kernel: the three-term contraction,
    which runs every stage with the default increment form, or the two-term
    increment contraction (5 of 6 stages) with --ens-terms 2; the other form
    beside it."""
    full = {"kernel": "k_bf16x3_contract<64,true,1> (tcgen05 Khi Vhi + 2^-11 (Khi Vlo + Klo Vhi), per-k-block "
                      "drains; every stage)" if args.ens_terms == 3 else
                      "k_bf16x3_contract<64,true,1> (stage 1)",
            "ms_per_launch": ms_a, "bytes_per_launch": a_bytes, "achieved": a_bytes / (ms_a / 1e3) / 1e9,
            "frac": a_bytes / (ms_a / 1e3) / 1e9 / peak, "tensor_tflops": a_flops / (ms_a / 1e3) / 1e12,
            "traffic": load_traffic("k_bf16x3_contract")}
    two = {"kernel": "k_bf16x3_contract<64,false,2> (tcgen05 Khi (Vhi + 2^-11 Vlo); stages 2-6 with --ens-terms 2)",
           "ms_per_launch": ms_c, "bytes_per_launch": c_bytes, "achieved": c_bytes / (ms_c / 1e3) / 1e9,
           "frac": c_bytes / (ms_c / 1e3) / 1e9 / peak, "tensor_tflops": c_flops / (ms_c / 1e3) / 1e12,
           "traffic": load_traffic("k_bf16x3_contract_increment")}
    main, other = (full, two) if args.ens_terms == 3 else (two, full)
    flops = a_flops if args.ens_terms == 3 else c_flops
    ms = main["ms_per_launch"]
    return {"bound": "hbm", "achieved": main["achieved"], "peak": peak, "unit": "GB/s", "frac": main["frac"],
            "traffic": main["traffic"], "kernel": main["kernel"], "ms_per_launch": ms, "peak_source": peak_kind,
            "bytes_per_launch": main["bytes_per_launch"], "tensor_tflops": flops / (ms / 1e3) / 1e12,
            "tensor_peak_tflops": tpeak, "tensor_frac": flops / (ms / 1e3) / 1e12 / tpeak,
            "tensor_peak_source": tpeak_kind, "other_form": other}


def run_ensemble(args, world, rank, local):
    """Headline: args.sets frictional parameter sets of the N = 20k model in one
    ensemble, beside the same model as one plain FP64 instance."""
    import torch
    import unicycle_b200
    from unicycle_b200 import configs

    torch.cuda.set_device(local)
    headline_plain = args.workload == "all"
    plain = run_ours(args, world, rank, local, keep_sim=True,
                     plain_steps=args.steps if headline_plain else max(10, args.steps // 2))
    sim, plain = plain["_sim"], {k: v for k, v in plain.items() if k != "_sim"}
    split = split_leg(args, local, sim, configs.cfg2(nx=args.nx, nz=args.nz), plain) \
        if rank == 0 and not args.no_split else None
    cfg = configs.cfg2(nx=args.nx, nz=args.nz)
    n = cfg["n_patch"]
    sets, y0s = configs.parameter_sets(cfg, args.sets)
    ens = unicycle_b200.Ensemble(device=local)
    ens.add_geometry(sim, args.sets)
    for i, (fr, y0) in enumerate(zip(sets, y0s)):
        ens.set_friction(0, i, fr["Vpl"], fr["rake"], fr["mu0"], fr["sig"], fr["a"], fr["b"], fr["L"], fr["Vo"],
                         fr["damping"])
        ens.set_state(0, i, y0, 0.0, cfg["dt0"])
    ens.set_tolerance(cfg["epsilon"])
    if args.ens_eager:
        ens.use_graph(False)
    tune_report = ens.tune(reps=3)
    stream = torch.cuda.ExternalStream(ens.stream, device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ens.run(1e300, args.spinup + args.warmup)
    i0 = ens.info()
    barrier(world)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        e0.record(stream)
        attempts = ens.run(1e300, args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
    elapsed = e0.elapsed_time(e1) / 1e3
    i1 = ens.info()
    elapsed_max = reduce_max(elapsed, world, args)
    accepted = i1["accepted"] - i0["accepted"]
    rejected = i1["rejected"] - i0["rejected"]
    sim_years = (i1["time_sum"] - i0["time_sum"]) / YEAR
    # roofline of the dominant kernel, the tensor-core contraction in its
    # increment form (5 of the 6 launches of an attempt), timed live; the
    # anchor form beside it
    ms_a, ms_c = ens.profile_contract(10)
    m, nn = 3 * n, 2 * n
    c_bytes = 2.0 * m * nn + 4.0 * args.sets * (nn + m)
    c_flops = 2.0 * m * nn * args.sets * 2
    a_bytes = 4.0 * m * nn + 4.0 * args.sets * (nn + m)
    a_flops = 2.0 * m * nn * args.sets * 3
    peak, peak_kind = load_peaks()
    tpeak, tpeak_kind = load_tensor_peak()
    achieved = c_bytes / (ms_c / 1e3) / 1e9
    # the contraction against FP64 on a row block of the full-size matrix
    V = np.random.default_rng(7).standard_normal((args.sets, nn)) * 1e-9
    Kr = sim.copy_G(0, 3 * 256)
    mag = np.abs(V) @ np.abs(Kr).T
    check = float(np.max(np.abs(ens.matvec(0, V)[:, :3 * 256] - V @ Kr.T) / mag))
    check2 = float(np.max(np.abs(ens.matvec(0, V, terms=2)[:, :3 * 256] - V @ Kr.T) / mag))
    # end to end: every attempt, all instances' states host->device (pinned host
    # arrays) and back
    e2e_att = args.e2e_steps or max(10, args.steps // 3)
    pin = torch.empty((args.sets, 7 * n), dtype=torch.float64, pin_memory=True).numpy()
    y_h, t_h, dt_h, acc0, *_r = ens.get_states(0, out=pin)
    acc0 = int(acc0.sum())
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_att):
        ens.put_states(0, y_h)
        ens.run(1e300, 1)
        y_h, t_h, dt_h, acc_h, rej_h, st_h = ens.get_states(0, out=pin)
    torch.cuda.synchronize()
    acc_e2e = int(acc_h.sum()) - acc0
    e2e_elapsed = reduce_max(time.perf_counter() - t0, world, args)
    ens.close()
    tri_ms = sim.assembly_times()[1]
    families = assembly_leg(args, local) if rank == 0 else None
    if families:
        families["nikkhoo_tri"] = {"entries": 6 * n * n, "ms": tri_ms, "mentries_per_s": 6 * n * n / tri_ms / 1e3,
                                   "pairs": {"fault_receiver": n * n}}
        families = add_fp64_fractions(families, fp64_peak_tflops(local))
    hens = None
    if rank == 0 and not args.no_hier_ensemble:
        hens = hier_ensemble_leg(args, local, cfg, sets, y0s,
                                 {"ms_per_step": 1e3 * elapsed / attempts, "plain_value": plain["value"]}, Kr)
    hmat = hmatrix_leg(args, local, sim, cfg, plain) if rank == 0 and not args.no_hmatrix else None
    learned = None
    if not args.no_learned and rank == 0:
        learned = learned_leg(args, local, sim, sets, y0s,
                              {"before": args.spinup + args.warmup, "attempts": args.steps, "accepted": accepted,
                               "rejected": rejected, "sim_years_per_hour": sim_years / (elapsed / 3600.0)})
    out = None
    if rank == 0:
        value = world * accepted / elapsed_max
        syh = world * sim_years / (elapsed_max / 3600.0)
        cpu = plain.get("cpu_baseline")
        if cpu:
            cpu = dict(cpu)
            cpu["sample"] += ("; the reference has no batching: the instances of the ensemble are separate runs, "
                              "each bound by the same matrix traffic, so this per-run rate is also their aggregate")
        out = {
            "metric": METRIC_ENS, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * elapsed_max / attempts, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16x3/f32 product, f64 state",
            "data": "synthetic (seeded cfg2 curved megathrust; Dc redrawn per parameter set)",
            "config": {"workload": f"megathrust {n} Nikkhoo-Walter triangles x {args.sets} frictional parameter "
                                   "sets, one ensemble", "n_triangles": n, "instances": args.sets,
                       "K_shape": [m, nn], "step": "one attempt of every instance (timed steps = attempts)",
                       "parallelism": f"replicas x{world}", "rtol": cfg["epsilon"],
                       "l2": "inputs larger than L2 (K images %.1f GB)" % (4.0 * m * nn / 1e9),
                       "plan": i1["plan"]},
            "sim_years_per_hour": syh,
            "accepted_steps": accepted, "rejected_attempts": rejected,
            "speedup_vs_plain_fp64": {"steps_per_s": value / plain["value"],
                                      "sim_years_per_hour": syh / plain["sim_years_per_hour"]
                                      if plain["sim_years_per_hour"] > 0 else None},
            "plain_fp64": {k: plain[k] for k in ("value", "unit", "ms_per_step", "sim_years_per_hour",
                                                 "rejected_attempts", "roofline", "e2e", "gpu_launches")},
            "assembly": plain["assembly"],
            "roofline": ens_roofline(args, ms_a, ms_c, a_bytes, a_flops, c_bytes, c_flops, peak, peak_kind, tpeak,
                                     tpeak_kind),
            "autotune": tune_report.strip().splitlines(),
            "e2e": {"value": world * acc_e2e / e2e_elapsed, "unit": "steps/s",
                    "h2d_bytes_per_step": 8 * 7 * n * args.sets, "d2h_bytes_per_step": 8 * 7 * n * args.sets,
                    "attempts": e2e_att,
                    "note": "per attempt: ucg_ens_put_states of all instances from pinned host arrays (controller "
                            "state kept), one attempt (one graph launch), ucg_ens_get_states back; wall clock"},
            "contraction_check": {"anchor_max_rel_to_abs_product": check, "anchor_bound": 1e-4,
                                  "increment_max_rel_to_abs_product": check2, "increment_bound": 5e-3,
                                  "rows": 3 * 256},
            "gpu_launches": int(attempts * 20 + 3),
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "assembly_families": families,
            "learned_step": learned,
            "hmatrix": hmat,
            "hierarchical_ensemble": hens,
            "split_bf16": split,
        }
        if headline_plain:
            out = headline_line(out, plain)
    sim.close()
    return out


def headline_line(ens_line, plain):
    """The parsed line: the plain FP64 path (the reference's own precision and
    algorithm, so its arm measures the same thing), with the chosen forms beside
    it as extras, each with its speed-up over this plain FP64 path."""
    ens = {k: v for k, v in ens_line.items() if k not in (
        "n_gpus", "warmup", "higher_is_better", "scaling", "vs_baseline", "data", "cpu_baseline", "plain_fp64",
        "assembly", "assembly_families", "learned_step", "hmatrix", "hierarchical_ensemble", "split_bf16")}
    learned = ens_line.get("learned_step") or {}
    comb = None
    l20 = learned.get("megathrust_20k_ensemble")
    if l20 and plain.get("sim_years_per_hour"):
        comb = {"sim_years_per_hour": l20["learned"]["sim_years_per_hour"],
                "speedup_vs_plain_fp64": l20["learned"]["sim_years_per_hour"] / plain["sim_years_per_hour"],
                "target": 10.0,
                "what": "split-BF16 K (tensor-core contraction) x 64-instance batching x learned step proposal, "
                        "simulated years per hour summed over the instances, over the plain FP64 single instance"}
    out = dict(plain)
    out.pop("_sim", None)
    out["chosen_forms"] = {
        "combined": comb,
        "ensemble": ens,
        "split_bf16": ens_line.get("split_bf16"),
        "learned_step": learned,
        "hmatrix": ens_line.get("hmatrix"),
        "hierarchical_ensemble": ens_line.get("hierarchical_ensemble"),
    }
    out["assembly_families"] = ens_line.get("assembly_families")
    return out


def main():
    args = parse()
    world, rank, local = dist_init(args)
    if args.impl == "reference" and args.workload == "cfg1":
        out = run_reference_cfg1(args) if rank == 0 else None
    elif args.impl == "reference":
        out = run_reference(args, world, rank)
    elif args.workload in ("all", "ensemble"):
        out = run_ensemble(args, world, rank, local)
    elif args.workload == "cfg4":
        out = run_cfg4(args, world, rank, local)
    elif args.workload == "cfg3":
        out = run_cfg3(args, world, rank, local)
    elif args.workload == "cfg1":
        out = run_cfg1(args, world, rank, local)
    elif args.workload == "hmatrix":
        out = run_hmatrix(args, world, rank, local)
    elif args.workload == "hens":
        out = run_hier_ensemble(args, world, rank, local)
    elif args.workload == "coupled":
        import torch
        torch.cuda.set_device(local)
        fam = assembly_leg(args, local) if rank == 0 else None
        out = None
        if rank == 0:
            fam = add_fp64_fractions(fam, fp64_peak_tflops(local))
            tot_e = fam["okada_rect"]["entries"] + fam["bml17_vol"]["entries"]
            tot_ms = fam["okada_rect"]["ms"] + fam["bml17_vol"]["ms"]
            out = {"metric": "GF assembly Mentries/s (coupled fault + volume)", "value": tot_e / tot_ms / 1e3,
                   "unit": "Mentries/s", "n_gpus": world, "steps": 1, "warmup": 0, "ms_per_step": tot_ms,
                   "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                   "data": "synthetic (seeded cfg3 geometry)", "config": {"workload": fam["model"]},
                   "assembly_families": fam}
    else:
        if args.workload == "split":
            args.precision = "split_bf16"
        out = run_ours(args, world, rank, local)
    if out is not None and rank == 0:
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
