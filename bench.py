"""Benchmark of the PME reciprocal path: evals/s on one B200 (or N independent replicas).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload water8k_64_p4|water1k_32|water8k_64_p6|water336k_216_p6]

One step = one full reciprocal evaluation (spread, R2C, solve with energy+virial, C2R, gather,
self energy) of the workload.  The default workload is 8,000 TIP3P-geometry waters (24,000
atoms) in a 62.1 A cube, 64^3 grid, spline order 4, kappa 0.32 (seeded synthetic data).

value: device-timed evals/s with inputs resident in HBM, L2 flushed (256 MiB write) before every
step outside the per-step CUDA-event pair; each step is the one fused launch, which also delivers
its energy/virial record to pinned host memory (the record mirror).  e2e: the same through the C
ABI with host buffers (pme_eval_host): the evaluation reads the pinned xyzq over the bus while it
bins the atoms, the forces come back D2H by one copy, and the energy/virial record reaches pinned
host memory from the kernel (the record mirror), all inside the timed region.
roofline: the dominant stage of the staged C-ABI calls, timed with CUDA events on the
operator's stream, algorithmic bytes per launch against the measured HBM copy bandwidth.
--impl reference: the CPU oracle (multithreaded FP64 restatement of the reference algorithm;
the reference itself has no CPU path and its GPU code does not build for sm_100a unmodified).
"""
from __future__ import annotations

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

METRIC = "PME recip evals/s at 24k atoms/64^3; batched evals/s + p50/p99 latency, same GPU"

UNIT = "evals/s"
# DRAM bytes (read + write) per launch of each workload's dominant kernel, from ncu captures kept
# beside their summaries (each entry names its command); null where a workload was not captured.
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "dram_traffic.json")
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="water8k_64_p4")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="time budget of the cpu_baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch", type=int, default=256, help="systems in the batched measurement (0: skip)")
    ap.add_argument("--batch-steps", type=int, default=200)
    ap.add_argument("--large-steps", type=int, default=20, help="timed evaluations of the 216^3 system (0: skip)")
    ap.add_argument("--triclinic-steps", type=int, default=200,
                    help="timed evaluations of the 24,000-atom rhombic dodecahedron (0: skip)")
    ap.add_argument("--direct-steps", type=int, default=200,
                    help="timed direct-space evaluations of the reference's 23,558-atom system (0: skip)")
    ap.add_argument("--reference-gpu-steps", type=int, default=200,
                    help="timed evaluations of the reference's own CUDA operator on this GPU (0: skip)")
    ap.add_argument("--serve-requests", type=int, default=600, help="requests of the serving run (0: skip)")
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="Poisson arrival rate (requests/s)")
    ap.add_argument("--also", nargs="*", default=["water1k_32", "water8k_64_p6"],
                    help="further single-system workloads timed beside the main one")
    ap.add_argument("--also-steps", type=int, default=200)
    ap.add_argument("--no-fft-comparator", dest="fft_comparator", action="store_false")
    ap.add_argument("--fft-schedule", default="auto", choices=list(SCHEDULES),
                    help="auto: the autotuner picks the launch shape; otherwise that y/z schedule with default "
                         "tiles and no autotuning (profilers that cannot launch thread-block clusters)")
    return ap.parse_args()


SCHEDULES = {"auto": 0, "planes": 1, "passes": 2, "cluster": 3}


def new_handle(args, nfft, order, stream=None):
    """A CudaPMERecip with the y/z schedule pinned from its first evaluation when --fft-schedule
    asks for one."""
    from gpu_recip_b200 import CudaPMERecip
    pme = CudaPMERecip(*nfft, order, stream=stream)
    if args.fft_schedule != "auto":
        pme.set_fft_schedule(SCHEDULES[args.fft_schedule])
    return pme


def tune_single(pme, args, inv_box, x, n, kappa, reps):
    """The autotuner's launch shape, or (--fft-schedule) the pinned y/z schedule with default tiles."""
    if args.fft_schedule == "auto":
        return pme.autotune(inv_box, x, n, kappa, reps=reps)
    return dict(pme.get_tune_config(), schedule=SCHEDULES[args.fft_schedule], pinned=True)


def make_workload(name: str, rank: int = 0):
    from gpu_recip_b200 import systems as S
    if name == "water8k_64_p4":
        s = S.config_production(4, seed=2 + 1000 * rank)
    elif name == "water8k_64_p6":
        s = S.config_production(6, seed=2 + 1000 * rank)
    elif name == "water1k_32":
        s = S.config_small(seed=1 + 1000 * rank)
    elif name == "water336k_216_p6":
        s = S.config_large(seed=3 + 1000 * rank)
    else:
        raise SystemExit(f"unknown workload {name}")
    return s


def workload_config(s, extra=None):
    cfg = {"workload": f"{s.name}: {s.natom} atoms TIP3P-geometry water, box {s.box[0]:.2f} A, "
                       f"grid {s.nfft[0]}x{s.nfft[1]}x{s.nfft[2]}, order {s.order}, kappa {s.kappa}",
           "natom": s.natom, "nfft": list(s.nfft), "order": s.order, "kappa": s.kappa,
           "alg_bytes_per_eval": s.alg_bytes(), "l2": "flushed (256 MiB write) before every step"}
    if extra:
        cfg.update(extra)
    return cfg


def measured_traffic(workload: str):
    """(bytes per launch, source) of a workload's dominant kernel from the ncu capture record."""
    try:
        with open(TRAFFIC_FILE) as fh:
            rec = json.load(fh).get(workload)
        if rec:
            return int(rec["dram_bytes_per_launch"]), rec.get("command")
    except Exception:
        pass
    return None, None


def replica_plan(gpus: int, env=None):
    """What `--gpus N` means for this process: ("spawn", N) when N > 1 and no launcher started the
    ranks (bench.py then starts N rank processes itself), ("run", world) under a launcher whose
    world size is N (or N == 1 alone).  A launcher world size other than N is an error."""
    env = os.environ if env is None else env
    world = int(env.get("WORLD_SIZE", "0") or 0)
    if world == 0:
        return ("spawn", gpus) if gpus > 1 else ("run", 1)
    if world != gpus:
        raise SystemExit(f"bench.py: --gpus {gpus} but the launcher started {world} ranks")
    return ("run", world)


def torchrun_command(argv, nproc: int, port: int):
    """The command that runs this benchmark as nproc rank processes on this node."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={nproc}",
            "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + list(argv)


def spawn_replicas(nproc: int) -> int:
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    return subprocess.call(["timeout", "-k", "60", "3600"] + torchrun_command(sys.argv[1:], nproc, port))


def rank_summary(per_rank_ms: float, units: int, world: int, device=None):
    """Whole-job figures of a timed region: the slowest rank's time (ms) and the rate of all
    ranks' units over it (units per rank are equal: every replica runs the same workload)."""
    from gpu_recip_b200 import replicas as R
    total_ms = R.max_over_ranks(float(per_rank_ms), device)
    return total_ms, R.aggregate_rate([units] * world, total_ms / 1000.0)


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.tmp = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=self.tmp,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        self.tmp.flush()
        rows = []
        try:
            with open(self.tmp.name) as fh:
                for line in fh:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        finally:
            try:
                os.unlink(self.tmp.name)
            except OSError:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def workload_parity(pme, s, x_dev, f_dev, stride, inv_box, stream):
    """One fused evaluation of the workload against the FP64 oracle on the same inputs: force
    relative RMS, energy and virial errors, and whether the int64 charge grid is bit-exact
    against the oracle's FP32 mirror (tolerances: force 1e-5, energy 1e-6)."""
    import torch
    from oracle import oracle as O
    O.build()
    n = s.natom
    with torch.cuda.stream(stream):
        pme.energy_virial.clear()
        pme.eval_ortho(inv_box, x_dev, n, s.kappa, True, True, f_dev, stride)
    stream.synchronize()
    ev = pme.energy_virial
    ev.copyToHost()
    f = f_dev.view(3, stride)[:, :n].T.cpu().numpy().astype(np.float64)
    ref = O.evaluate(s.xyzq.astype(np.float64), s.recip3, s.nfft, s.order, s.kappa)
    pme.spread_charge(x_dev, n, [inv_box[0], 0, 0, 0, inv_box[1], 0, 0, 0, inv_box[2]])
    grid_exact = bool(np.array_equal(pme.charge_grid_fixed(), O.spread_fixed(s.xyzq, s.recip3, s.nfft, s.order)))
    return {"vs": "FP64 oracle (CPU) on the same inputs",
            "force_rel_rms": float(np.sqrt(((f - ref["force"]) ** 2).sum() / (ref["force"] ** 2).sum())),
            "energy_rel": float(abs(ev.getEnergy("recip") - ref["energy"]) / abs(ref["energy"])),
            "self_energy_rel": float(abs(ev.getEnergy("self") - ref["energy_self"]) / abs(ref["energy_self"])),
            "virial_rel": float(np.abs(ev.getVirial() - ref["virial"]).max() / np.abs(ref["virial"]).max()),
            "charge_grid_bit_exact": grid_exact,
            "tolerances": {"force_rel_rms": 1e-5, "energy_rel": 1e-6}}


def cpu_oracle_rate(s, seconds: float, nthreads: int = 0):
    from oracle import oracle as O
    O.build()
    x = s.xyzq.astype(np.float64)
    O.evaluate(x, s.recip3, s.nfft, s.order, s.kappa, nthreads)  # warm-up
    n = 0
    t0 = time.perf_counter()
    while True:
        O.evaluate(x, s.recip3, s.nfft, s.order, s.kappa, nthreads)
        n += 1
        dt = time.perf_counter() - t0
        if dt >= seconds or n >= 1000:
            break
    cores = nthreads if nthreads > 0 else O.hardware_threads()
    return n / dt, n, dt, cores


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    s = make_workload(args.workload)
    from oracle import oracle as O
    O.build()
    x = s.xyzq.astype(np.float64)
    for _ in range(max(1, args.warmup)):
        O.evaluate(x, s.recip3, s.nfft, s.order, s.kappa)
    # each step is one full evaluation, capped so the run stays within a few minutes
    steps = args.steps
    t0 = time.perf_counter()
    done = 0
    budget = 150.0
    while done < steps:
        O.evaluate(x, s.recip3, s.nfft, s.order, s.kappa)
        done += 1
        if time.perf_counter() - t0 > budget:
            break
    dt = time.perf_counter() - t0
    rate = done / dt
    cores = O.hardware_threads()
    sample = f"{done} full FP64 evaluations of the workload on {cores} host threads"
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
            "steps": done, "warmup": args.warmup, "ms_per_step": 1000.0 * dt / done,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded TIP3P-geometry water)",
            "config": workload_config(s, {"parallelism": "cpu threads", "l2": "n/a (CPU)"}),
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference has no CPU implementation of the path; this is the oracle port of its algorithm"}
    print(json.dumps(line), flush=True)


def run_b200(args):
    import torch
    from gpu_recip_b200 import replicas as R
    rank, world, local = R.rank_world()
    torch.cuda.set_device(local if world > 1 else 0)
    R.init("nccl")
    dev = torch.device("cuda", torch.cuda.current_device())

    from gpu_recip_b200 import CudaPMERecip, force_stride, load_library
    from gpu_recip_b200 import build as B
    if rank == 0 or world == 1:
        B.build()
    R.barrier()
    load_library()

    s = make_workload(args.workload, rank)
    n = s.natom
    stride = force_stride(n)
    stream = torch.cuda.Stream(device=dev)
    pme = new_handle(args, s.nfft, s.order, stream)
    inv_box = [1.0 / b for b in s.box]
    recip = [inv_box[0], 0, 0, 0, inv_box[1], 0, 0, 0, inv_box[2]]
    x_dev = torch.from_numpy(s.xyzq).to(dev)
    f_dev = torch.zeros(3 * stride, dtype=torch.float32, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    # each evaluation delivers its own energy/virial record to pinned host memory (the record
    # mirror), so a step is the one fused launch with no record clear
    ev_step = torch.zeros(11, dtype=torch.float64).pin_memory()
    pme.set_energy_virial_mirror(ev_step)

    def one_eval():
        pme.eval_ortho(inv_box, x_dev, n, s.kappa, True, True, f_dev, stride)

    kernels_per_eval = 1   # the fused cooperative kernel

    with torch.cuda.stream(stream):
        for _ in range(max(3, args.warmup)):
            flush.fill_(0.0)
            one_eval()
    stream.synchronize()
    # launch shape of the fused kernel from the autotuner (results are the same for every shape)
    tune = tune_single(pme, args, inv_box, x_dev, n, s.kappa, 10)
    with torch.cuda.stream(stream):
        for _ in range(3):
            flush.fill_(0.0)
            one_eval()
    stream.synchronize()

    K = args.steps
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    clocks = ClockSampler(dev.index)
    R.barrier()
    torch.cuda.synchronize()
    with clocks:
        with torch.cuda.stream(stream):
            for i in range(K):
                flush.fill_(float(i & 7))
                starts[i].record(stream)
                one_eval()
                ends[i].record(stream)
        stream.synchronize()
    torch.cuda.synchronize()
    per = np.array([starts[i].elapsed_time(ends[i]) for i in range(K)])  # ms
    pme.set_energy_virial_mirror(None)
    if not np.isfinite(ev_step.numpy()).all() or ev_step[0].item() == 0.0:
        raise RuntimeError("value: the energy record did not reach the host")
    total_ms, value = rank_summary(float(per.sum()), K, world, dev)     # slowest replica
    R.barrier()

    # ---- e2e through the C ABI with host buffers -------------------------------------------------
    x_host = torch.from_numpy(s.xyzq).pin_memory()
    f_host = torch.empty(3 * stride, dtype=torch.float32).pin_memory()
    ev_host = torch.empty(11, dtype=torch.float64).pin_memory()
    Ke = max(10, K // 4)
    e_starts = [torch.cuda.Event(enable_timing=True) for _ in range(Ke)]
    e_ends = [torch.cuda.Event(enable_timing=True) for _ in range(Ke)]
    # one call per step, pme_eval_host: the evaluation reads the pinned coordinates over the bus
    # while it bins them, the forces come back by one copy, and the step's energy and virial
    # reach pinned host memory from the kernel itself (the record mirror)
    pme.set_energy_virial_mirror(ev_host)
    with torch.cuda.stream(stream):
        for i in range(Ke + 3):
            flush.fill_(0.0)
            if i >= 3:
                e_starts[i - 3].record(stream)
            pme.eval_host(recip, x_host, n, s.kappa, True, True, f_host, stride)
            if i >= 3:
                e_ends[i - 3].record(stream)
    stream.synchronize()
    pme.set_energy_virial_mirror(None)
    if not np.isfinite(ev_host.numpy()).all() or ev_host[0].item() == 0.0:
        raise RuntimeError("e2e: the energy record did not reach the host")
    e_total, e2e_value = rank_summary(float(sum(e_starts[i].elapsed_time(e_ends[i]) for i in range(Ke))), Ke,
                                      world, dev)

    # ---- staged C-ABI calls, per reference stage (informational) -----------------------------------
    stages = stage_times(pme, s, x_dev, f_dev, stride, recip, stream, flush)
    sequence_ms = sequence_time(pme, s, x_dev, f_dev, stride, recip, stream, flush)

    # ---- roofline of the dominant kernel: the fused evaluation is one launch -------------------------
    peak, peak_kind = measured_peak()
    eval_ms = total_ms / K
    achieved = s.alg_bytes() / (eval_ms * 1e-3) / 1e9
    traffic, traffic_cmd = measured_traffic(args.workload)
    roofline = {"bound": "hbm", "kernel": "k_fused (whole evaluation, one cooperative launch)",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": peak_kind, "traffic": traffic, "traffic_source": traffic_cmd,
                "alg_bytes_per_launch": s.alg_bytes(),
                "staged_stage_us": {k: v * 1000 for k, v in stages.items()},
                "staged_total_us": 1000 * sum(stages.values()),
                "staged_sequence_us": 1000 * sequence_ms,
                "staged_note": ("staged_total_us sums per-call event intervals (an event between every two "
                                "calls); staged_sequence_us times the record clear and the six calls between "
                                "two events, as the reference's own operator is timed in reference_gpu")}

    fft_cmp = fft_comparator(s, dev, flush) if args.fft_comparator else None

    # ---- the other single-system workloads: 3,000 atoms at 32^3 and the production size at order 6
    others = {}
    for wname in args.also:
        others[wname] = run_single(wname, args, dev, stream, flush, rank, world)


    # ---- batched: uneven systems in one persistent launch --------------------------------------------
    batched = None
    if args.batch > 0:
        batched = run_batched(args, dev, stream, flush, rank, world)

    # ---- large system: 1,008,000 atoms, 216^3, order 6 -------------------------------------------
    large = None
    if args.large_steps > 0:
        large = run_large(args, dev, stream, flush, rank, world)

    # ---- triclinic box: the same atom count and grid in a rhombic dodecahedron --------------------
    triclinic = None
    if args.triclinic_steps > 0:
        triclinic = run_triclinic(args, dev, stream, flush, rank, world)

    # ---- direct space: the reference's direct-test system, and a whole Ewald step ------------------
    direct = None
    if args.direct_steps > 0:
        direct = run_direct(args, dev, stream, flush, rank, world)

    # ---- serving: Poisson request stream, continuous batching vs the plain path ------------------
    serving = None
    if args.serve_requests > 0:
        serving = run_serving(args, dev, rank, world)

    # ---- the reference's own CUDA operator on this GPU (timing comparator, single GPU only) --------
    reference_gpu = None
    if rank == 0 and world == 1 and args.reference_gpu_steps > 0:
        head = min(n, 4096)
        f_head = f_dev.view(3, stride)[:, :head].T.cpu().numpy().astype(np.float64)
        from oracle import oracle as O
        O.build()
        ref = O.evaluate(s.xyzq.astype(np.float64), s.recip3, s.nfft, s.order, s.kappa)
        reference_gpu = run_reference_gpu(s, args, float(np.percentile(per, 50)) * 1000.0, float(ev_step[0].item()),
                                          f_head, {"energy": float(ref["energy"]), "force_head": ref["force"][:head]})

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        rate, cnt, dt, cores = cpu_oracle_rate(s, args.cpu_seconds)
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{cnt} full FP64 evaluations of the workload ({dt:.1f} s)",
               # the same FP64 evaluation checks the GPU's result on these inputs
               "gpu_parity": workload_parity(pme, s, x_dev, f_dev, stride, inv_box, stream)}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
                "warmup": args.warmup, "ms_per_step": total_ms / K, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32+i64 fixed-point grid",
                "data": "synthetic (seeded TIP3P-geometry water)",
                "config": workload_config(s, {"parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                                              "launch_shape": {k: tune[k] for k in ("schedule", "x_lines", "y_lines",
                                                                                     "z_columns", "grid_ctas")}}),
                "latency_ms": {"p50": float(np.percentile(per, 50)), "p99": float(np.percentile(per, 99))},
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 16 * n,
                        "d2h_bytes_per_step": 4 * 3 * n + 8 * 11},
                "gpu_launches": kernels_per_eval * K,
                "roofline": roofline, "batched": batched, "serving": serving, "large": large,
                "triclinic": triclinic, "direct": direct, "other_workloads": others,
                "fft_comparator": fft_cmp, "reference_gpu": reference_gpu,
                "clocks": clocks.summary(), "cpu_baseline": cpu}
        print(json.dumps(line), flush=True)
    R.barrier()
    R.shutdown()


def run_single(name, args, dev, stream, flush, rank, world):
    """One more single-system workload timed like the main one (fused evaluations, launch shape
    from the autotuner, L2 flushed before every step), with its roofline and its parity against
    the FP64 oracle on the same inputs."""
    import torch
    from gpu_recip_b200 import CudaPMERecip, force_stride
    s = make_workload(name, rank)
    n = s.natom
    stride = force_stride(n)
    pme = new_handle(args, s.nfft, s.order, stream)
    inv_box = [1.0 / b for b in s.box]
    x = torch.from_numpy(s.xyzq).to(dev)
    f = torch.zeros(3 * stride, dtype=torch.float32, device=dev)
    tune = tune_single(pme, args, inv_box, x, n, s.kappa, 10)
    K = args.also_steps
    W = max(3, args.warmup)
    e0 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    e1 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    with torch.cuda.stream(stream):
        for i in range(K + W):
            flush.fill_(float(i & 7))
            if i >= W:
                e0[i - W].record(stream)
            pme.eval_ortho(inv_box, x, n, s.kappa, True, True, f, stride)
            if i >= W:
                e1[i - W].record(stream)
    stream.synchronize()
    per = np.array([e0[i].elapsed_time(e1[i]) for i in range(K)])
    total_ms, rate = rank_summary(float(per.sum()), K, world, dev)
    peak, peak_kind = measured_peak()
    ms = total_ms / K
    traffic, traffic_cmd = measured_traffic(name)
    out = {"workload": workload_config(s)["workload"], "steps": K, "ms_per_eval": ms, "evals_per_s": rate,
           "p50_ms": float(np.percentile(per, 50)), "p99_ms": float(np.percentile(per, 99)),
           "alg_bytes_per_eval": s.alg_bytes(),
           "roofline": {"achieved": s.alg_bytes() / (ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": s.alg_bytes() / (ms * 1e-3) / 1e9 / peak, "peak_source": peak_kind,
                        "traffic": traffic, "traffic_source": traffic_cmd},
           "launch_shape": {k: tune[k] for k in ("schedule", "x_lines", "y_lines", "z_columns", "grid_ctas")}}
    if rank == 0:
        out["gpu_parity"] = workload_parity(pme, s, x, f, stride, inv_box, stream)
    pme.close()
    return out


def run_batched(args, dev, stream, flush, rank, world):
    """256 independent water boxes of 648-24,000 atoms, 24^3-64^3 grids, order 4, kappa 0.32, all
    evaluated by one persistent launch per step, launch shape picked by the batch autotuner and the
    step replayed from a CUDA graph (L2 flushed before every step, outside the timed events)."""
    import torch
    from gpu_recip_b200 import PmeBatch, force_stride
    from gpu_recip_b200 import replicas as R
    from gpu_recip_b200 import systems as S
    systems = S.batch_systems(args.batch, seed=R.replica_seed(4, rank))
    specs = []
    for sy in systems:
        x = torch.from_numpy(sy.xyzq).to(dev)
        st = force_stride(sy.natom)
        f = torch.zeros(3 * st, dtype=torch.float32, device=dev)
        specs.append(dict(nfft=sy.nfft, order=sy.order, box=sy.box, kappa=sy.kappa, xyzq=x, force=f, stride=st))
    forces = [(sp["force"], sp["stride"]) for sp in specs]
    b = PmeBatch(specs, stream=stream)
    tune = b.autotune(reps=5)
    with torch.cuda.stream(stream):
        for _ in range(3):
            flush.fill_(0.0)
            b.clear_energy_virial()
            b.eval()
    stream.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        b.clear_energy_virial()
        b.eval()
    K = args.batch_steps
    st_ev = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    en_ev = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    R.barrier()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for i in range(K):
            flush.fill_(float(i & 7))
            st_ev[i].record(stream)
            graph.replay()
            en_ev[i].record(stream)
    stream.synchronize()
    per = np.array([st_ev[i].elapsed_time(en_ev[i]) for i in range(K)])
    total = R.max_over_ranks(float(per.sum()), dev)
    del graph
    parity = batch_parity(systems, forces, b.energy_virial()) if rank == 0 else None
    peak, _ = measured_peak()
    alg = sum(sy.alg_bytes() for sy in systems)
    ms = total / K
    info = b.info()
    return {"systems": len(systems), "atoms": int(sum(sy.natom for sy in systems)),
            "evals_per_s": R.aggregate_rate([len(systems) * K] * world, total / 1000.0), "ms_per_batch": ms,
            "p50_ms": float(np.percentile(per, 50)), "p99_ms": float(np.percentile(per, 99)),
            "launches_per_batch": 1, "cuda_graph": True, "grid_ctas": info["grid_ctas"],
            "autotune": {"schedule": ["auto", "planes", "passes", "cluster"][tune["schedule"]], "grid_ctas": tune["grid_ctas"],
                         "line_scale": tune["x_lines"], "candidates": tune["candidates"]},
            "device_bytes": info["device_bytes"], "alg_bytes_per_batch": alg,
            "roofline_frac": alg / (ms * 1e-3) / 1e9 / peak,
            "traffic": measured_traffic("batch256")[0], "gpu_parity": parity}


def parity_subset(systems, count=32, seed=41):
    """A seeded subset of a batch that includes the smallest and largest atom counts and grids."""
    natom = np.array([sy.natom for sy in systems])
    grid = np.array([int(np.prod(sy.nfft)) for sy in systems])
    keep = {int(natom.argmin()), int(natom.argmax()), int(grid.argmin()), int(grid.argmax())}
    rest = [i for i in range(len(systems)) if i not in keep]
    rng = np.random.default_rng(seed)
    keep.update(int(i) for i in rng.choice(rest, size=min(len(rest), count - len(keep)), replace=False))
    return sorted(keep)


def batch_parity(systems, forces, ev):
    """The last timed batch evaluation of a subset of systems against the FP64 oracle on the same
    inputs: worst force relative RMS, energy and virial errors (tolerances 1e-5 / 1e-6 / 1e-5)."""
    from oracle import oracle as O
    O.build()
    worst = {"force_rel_rms": 0.0, "energy_rel": 0.0, "self_energy_rel": 0.0, "virial_rel": 0.0}
    idx = parity_subset(systems)
    for i in idx:
        sy = systems[i]
        f, st = forces[i]
        F = f.view(3, st)[:, :sy.natom].T.cpu().numpy().astype(np.float64)
        ref = O.evaluate(sy.xyzq.astype(np.float64), sy.recip3, sy.nfft, sy.order, sy.kappa)
        err = {"force_rel_rms": float(np.sqrt(((F - ref["force"]) ** 2).sum() / (ref["force"] ** 2).sum())),
               "energy_rel": float(abs(ev[i, 0] - ref["energy"]) / abs(ref["energy"])),
               "self_energy_rel": float(abs(ev[i, 1] - ref["energy_self"]) / abs(ref["energy_self"])),
               "virial_rel": float(np.abs(ev[i, 2:].reshape(3, 3) - ref["virial"]).max()
                                   / np.abs(ref["virial"]).max())}
        for k in worst:
            worst[k] = max(worst[k], err[k])
    return {"vs": "FP64 oracle (CPU) on the same inputs", "systems_checked": len(idx),
            "natom_range": [min(systems[i].natom for i in idx), max(systems[i].natom for i in idx)],
            "worst": worst, "tolerances": {"force_rel_rms": 1e-5, "energy_rel": 1e-6, "virial_rel": 1e-5},
            "within_tolerance": bool(worst["force_rel_rms"] <= 1e-5 and worst["energy_rel"] <= 1e-6
                                     and worst["virial_rel"] <= 1e-5)}


def stage_alg_bytes(s):
    """Algorithmic bytes of each staged call: each stage reads its input and writes its output
    once (FP32 real grid, FP32 complex)."""
    N, (nx, ny, nz) = s.natom, s.nfft
    G, H = nx * ny * nz, (nx // 2 + 1) * ny * nz
    return {"spread": 16 * N + 4 * G, "r2c_fft": 4 * G + 8 * H, "scalar_sum": 16 * H,
            "c2r_fft": 8 * H + 4 * G, "gather": 28 * N + 4 * G, "self_energy": 16 * N}


def run_large(args, dev, stream, flush, rank, world):
    """The 216^3 configuration (1,008,000 atoms, order 6, kappa 0.30): fused evaluations with L2
    flushed between steps, plus each staged stage against its algorithmic bytes."""
    import torch
    from gpu_recip_b200 import CudaPMERecip, force_stride
    from gpu_recip_b200 import replicas as R
    from gpu_recip_b200 import systems as S
    s = S.config_large(seed=R.replica_seed(3, rank))
    n = s.natom
    st = force_stride(n)
    pme = new_handle(args, s.nfft, s.order, stream)
    inv_box = [1.0 / b for b in s.box]
    recip = [inv_box[0], 0, 0, 0, inv_box[1], 0, 0, 0, inv_box[2]]
    x = torch.from_numpy(s.xyzq).to(dev)
    f = torch.zeros(3 * st, dtype=torch.float32, device=dev)
    tune = tune_single(pme, args, inv_box, x, n, s.kappa, 3)
    K = args.large_steps
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    with torch.cuda.stream(stream):
        for i in range(K + 2):
            flush.fill_(float(i & 7))
            if i >= 2:
                ev0[i - 2].record(stream)
            pme.energy_virial.clear()
            pme.eval_ortho(inv_box, x, n, s.kappa, True, True, f, st)
            if i >= 2:
                ev1[i - 2].record(stream)
    stream.synchronize()
    total = R.max_over_ranks(float(sum(ev0[i].elapsed_time(ev1[i]) for i in range(K))), dev)
    ms = total / K
    peak, _ = measured_peak()
    stages = stage_times(pme, s, x, f, st, recip, stream, flush, reps=5)
    alg = stage_alg_bytes(s)
    per_stage = {k: {"us": 1000 * stages[k], "alg_bytes": alg[k],
                     "GBps": alg[k] / (stages[k] * 1e-3) / 1e9,
                     "roofline_frac": alg[k] / (stages[k] * 1e-3) / 1e9 / peak} for k in stages}
    return {"workload": f"{s.name}: {n} atoms, box {s.box[0]:.1f} A, grid {s.nfft[0]}^3, order {s.order}, "
                        f"kappa {s.kappa}", "steps": K, "ms_per_eval": ms,
            "evals_per_s": R.aggregate_rate([K] * world, total / 1000.0),
            "alg_bytes_per_eval": s.alg_bytes(),
            "roofline_frac": s.alg_bytes() / (ms * 1e-3) / 1e9 / peak,
            "launch_shape": {k: tune[k] for k in ("schedule", "x_lines", "y_lines", "z_columns", "grid_ctas")},
            "staged_stages": per_stage}


REF_GPU_BIN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "baseline", "_ref", "ref_gpu_bench")


def run_reference_gpu(s, args, b200_us_p50: float, b200_energy: float, b200_force, fp64):
    """Times the reference's own operator, CudaPMERecip<float, float, float2> built from its
    unmodified sources (baseline/ref_gpu), on this GPU and workload: per evaluation the sequence of
    its test driver (record clear, spread, R2C, solve with energy and virial, C2R, gather, self
    energy) with L2 flushed in between, BOX (3-D cuFFT) and COLUMN (1-D cuFFTs and transposes)
    modes.  It runs as a child process: the reference exits the process on a CUDA error.  Its
    in-place real<->complex transforms run out of place through a scratch copy (the compatibility
    header's bridge for cuFFT's removed native layout), which adds one grid copy per transform to
    its time.  Its result is checked against the FP64 oracle on the same inputs (fp64: energy and
    the forces of the first atoms), with the reference driver's own tolerances: forces within
    1e-3 kcal/mol/A (gpu_recip.cu:286-287), energy within 2e-3 kcal/mol (gpu_recip.cu:146) of an
    energy of 594 kcal/mol (gpu_recip.cu:81), i.e. 3.4e-6 relative, scaled to this workload's
    energy; this engine's differences from the same values are beside them.  The same binary also
    runs the reference's own test system (the 23,558-atom fixture, order 4), checked against the
    energy, virial and forces its driver hard-codes, with that driver's absolute tolerances.  In COLUMN mode the reference applies its
    x-mirror energy doubling to the z axis (CudaPMERecip.cu:708-742 run with nfft1 = nfftz,
    :1977-1988), so its COLUMN energy differs by design of that code path; its own test drives
    BOX only (gpu_recip.cu:80), and COLUMN is judged by its forces."""
    import struct
    import subprocess
    if not os.path.exists(REF_GPU_BIN):
        return {"unavailable": "baseline/_ref/ref_gpu_bench not built (needs the reference's sources at build time)"}
    out = {"operator": "reference CudaPMERecip<float, float, float2> (gpu_recip), unmodified sources, "
                       "compiled for sm_100a with compatibility shims", "l2": "flushed (256 MiB memset) before every evaluation",
           "fft_bridge": "in-place R2C/C2R run out of place from a scratch copy (one extra grid copy per transform)"}
    nforce = int(b200_force.shape[0])
    for ft, name in ((2, "box"), (0, "column")):
        hdr = struct.pack("<9i4x4d", s.natom, *s.nfft, s.order, ft, 3, args.reference_gpu_steps, nforce, s.kappa,
                          *s.box)
        try:
            p = subprocess.run([REF_GPU_BIN], input=hdr + np.ascontiguousarray(s.xyzq, dtype=np.float32).tobytes(),
                               capture_output=True, timeout=300)
        except subprocess.TimeoutExpired:
            out[name] = {"unavailable": "timed out"}
            continue
        if p.returncode != 0:
            out[name] = {"unavailable": f"exit {p.returncode}: {p.stderr.decode(errors='replace')[-300:]}"}
            continue
        r = json.loads(p.stdout.decode().strip().splitlines()[-1])
        e = r["energy_recip"]
        fh = r.get("force_head") or []
        f_max = f_rms = None
        ff = fp64["force_head"]
        if len(fh) == 3 * nforce and all(v is not None for v in fh):
            fr = np.array(fh, dtype=np.float64).reshape(nforce, 3)
            f_max = float(np.abs(fr - ff).max())
            f_rms = float(np.sqrt(((fr - ff) ** 2).sum() / (ff ** 2).sum()))
        e_tol = 2e-3 * abs(fp64["energy"]) / 593.973027
        e_ok = e is not None and abs(e - fp64["energy"]) <= e_tol
        f_ok = f_max is not None and f_max <= 1e-3
        out[name] = {"us_per_eval_p50": r["us_p50"], "us_per_eval_mean": r["us_mean"], "steps": r["steps"],
                     "evals_per_s": 1e6 / r["us_mean"],
                     "energy_recip": e, "energy_fp64": fp64["energy"], "energy_b200": b200_energy,
                     "energy_abs_diff_vs_fp64": None if e is None else abs(e - fp64["energy"]),
                     "b200_energy_abs_diff_vs_fp64": abs(b200_energy - fp64["energy"]),
                     "force_max_abs_diff_vs_fp64": f_max, "force_rel_rms_vs_fp64": f_rms,
                     "b200_force_max_abs_diff_vs_fp64": float(np.abs(b200_force - ff).max()),
                     "b200_force_rel_rms_vs_fp64": float(np.sqrt(((b200_force - ff) ** 2).sum() / (ff ** 2).sum())),
                     "forces_compared": nforce, "energy_tolerance": e_tol, "energy_valid": bool(e_ok),
                     "forces_valid": bool(f_ok),
                     "result_valid": bool(f_ok and (e_ok or name == "column")),
                     "b200_speedup_p50": r["us_p50"] / b200_us_p50}
    out["own_test_system"] = reference_own_fixture(args)
    return out


def reference_own_fixture(args):
    """The reference operator (BOX) on its own test system, tests/golden/ref_recip_23558.npz (the
    reference's test_data: 23,558 atoms, 62.23 A, 64^3, order 4, kappa 0.32), against the energy,
    virial and forces its test driver hard-codes, with that driver's tolerances
    (gpu_recip.cu:81-84, :146-174, :286-287)."""
    import struct
    import subprocess
    fx = dict(np.load(os.path.join(ROOT, "tests", "golden", "ref_recip_23558.npz")))
    n = fx["xyzq"].shape[0]
    hdr = struct.pack("<9i4x4d", n, *[int(v) for v in fx["nfft"]], 4, 2, 3, 20, n, float(fx["kappa"]),
                      *[float(v) for v in fx["box"]])
    try:
        p = subprocess.run([REF_GPU_BIN], input=hdr + np.ascontiguousarray(fx["xyzq"], dtype=np.float32).tobytes(),
                           capture_output=True, timeout=300)
    except subprocess.TimeoutExpired:
        return {"unavailable": "timed out"}
    if p.returncode != 0:
        return {"unavailable": f"exit {p.returncode}: {p.stderr.decode(errors='replace')[-300:]}"}
    r = json.loads(p.stdout.decode().strip().splitlines()[-1])
    e = r["energy_recip"]
    vir = np.array([np.nan if v is None else v for v in r["virial"]]).reshape(3, 3)
    fr = np.array([np.nan if v is None else v for v in r["force_head"]], dtype=np.float64).reshape(n, 3)
    de = None if e is None else abs(e - float(fx["energy4"]))
    dv = float(np.abs(vir - fx["virial4"]).max())
    df = float(np.abs(fr - fx["force4"]).max())
    ok = de is not None and de <= float(fx["tol_energy4"]) and dv <= float(fx["tol_virial4"]) and \
        df <= float(fx["tol_force4"])
    return {"system": "reference test_data: 23,558 atoms, 62.23 A, 64^3, order 4, kappa 0.32",
            "energy": e, "energy_expected": float(fx["energy4"]), "energy_abs_diff": de,
            "virial_max_abs_diff": dv, "force_max_abs_diff": df,
            "tolerances": {"energy": float(fx["tol_energy4"]), "virial": float(fx["tol_virial4"]),
                           "force": float(fx["tol_force4"])},
            "passes_its_own_test": bool(ok), "us_per_eval_p50": r["us_p50"]}


def run_triclinic(args, dev, stream, flush, rank, world):
    """8,000 waters in a rhombic dodecahedron (the volume of the 62.1 A cube), 64^3, order 4, through
    pme_eval with the full reciprocal matrix: fused evaluations with L2 flushed between steps."""
    import torch
    from gpu_recip_b200 import CudaPMERecip, force_stride
    from gpu_recip_b200 import replicas as R
    from gpu_recip_b200 import systems as S
    s = S.config_triclinic(4, seed=R.replica_seed(6, rank))
    n = s.natom
    st = force_stride(n)
    pme = new_handle(args, s.nfft, s.order, stream)
    x = torch.from_numpy(s.xyzq).to(dev)
    f = torch.zeros(3 * st, dtype=torch.float32, device=dev)
    r9 = s.recip9
    K = args.triclinic_steps
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    W = max(3, args.warmup)
    with torch.cuda.stream(stream):
        for i in range(K + W):
            flush.fill_(float(i & 7))
            if i >= W:
                ev0[i - W].record(stream)
            pme.energy_virial.clear()
            pme.eval(r9, x, n, s.kappa, True, True, f, st)
            if i >= W:
                ev1[i - W].record(stream)
    stream.synchronize()
    total = R.max_over_ranks(float(sum(ev0[i].elapsed_time(ev1[i]) for i in range(K))), dev)
    ms = total / K
    peak, _ = measured_peak()
    pme.close()
    return {"workload": f"{s.name}: {n} atoms, rhombic dodecahedron a=b={s.vectors[0][0]:.2f} A, "
                        f"grid {s.nfft[0]}^3, order {s.order}, kappa {s.kappa}",
            "steps": K, "ms_per_eval": ms, "evals_per_s": R.aggregate_rate([K] * world, total / 1000.0),
            "alg_bytes_per_eval": s.alg_bytes(),
            "roofline_frac": s.alg_bytes() / (ms * 1e-3) / 1e9 / peak}


def run_direct(args, dev, stream, flush, rank, world):
    """Direct-space PME on the reference's direct test system (tests/golden/ref_direct_23558.npz:
    23,558 atoms, 62.23 A box, roff 9 A, kappa 0.32, 35 vdW types, CHARMM exclusions, 6,556 1-4
    and 28,153 excluded pairs): the main pair list, main + 1-4 lists, and a whole Ewald step
    (direct + 1-4 + reciprocal 64^3 order 4) on the same coordinates, L2 flushed between steps.
    The FP64 oracle's main list on all host threads beside it."""
    import torch
    from gpu_recip_b200 import CudaPMERecip, force_stride
    from gpu_recip_b200 import replicas as R
    from gpu_recip_b200.direct import CudaPMEDirectForce
    d = dict(np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden",
                                  "ref_direct_23558.npz")))
    n = d["xyzq"].shape[0]
    dr = CudaPMEDirectForce(stream=stream)
    dr.setup(*d["box"], float(d["kappa"]), float(d["roff"]), float(d["ron"]), float(d["e14fac"]))
    dr.set_vdwparam(d["vdwparam"])
    dr.set_vdwparam14(d["vdwparam14"])
    dr.set_vdwtype(d["vdwtype"])
    dr.set_exclusions(d["iblo14"], d["inb14"], d["loc2glo"])
    dr.set_14_list(d["in14"], d["ex14"])
    x = torch.from_numpy(np.ascontiguousarray(d["xyzq"], dtype=np.float32)).to(dev)
    stride = force_stride(n, 8)
    fi = torch.zeros(3 * stride, dtype=torch.int64, device=dev)
    pme = new_handle(args, (64, 64, 64), 4, stream)
    inv = [1.0 / float(b) for b in d["box"]]
    K = args.direct_steps
    W = max(3, args.warmup)

    def timed(body):
        e0 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
        e1 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
        with torch.cuda.stream(stream):
            for i in range(K + W):
                flush.fill_(float(i & 7))
                if i >= W:
                    e0[i - W].record(stream)
                body()
                if i >= W:
                    e1[i - W].record(stream)
        stream.synchronize()
        return R.max_over_ranks(float(sum(e0[i].elapsed_time(e1[i]) for i in range(K))), dev) / K

    def main_only():
        dr.energy_virial.clear()
        dr.calc_force(x, n, True, True, stride, fi)

    def with14():
        main_only()
        dr.calc_14_force(x, True, True, stride, fi)

    def ewald():
        with14()
        pme.energy_virial.clear()
        pme.eval_ortho(inv, x, n, float(d["kappa"]), True, True, fi, stride)

    ms_main = timed(main_only)
    ms_14 = timed(with14)
    ms_ewald = timed(ewald)
    dr.close()
    pme.close()
    out = {"workload": "ref_direct_23558: the reference's direct-space test system, 23,558 atoms, box 62.23 A, "
                       "roff 9 A, kappa 0.32, VDW_VSH + EWALD, 35 vdW types, CHARMM exclusions, 1-4 lists",
           "steps": K, "ms_main_list": ms_main, "ms_with_14_lists": ms_14,
           "direct_evals_per_s": R.aggregate_rate([K] * world, ms_14 * K / 1000.0),
           "ewald_step_ms": ms_ewald, "ewald_steps_per_s": R.aggregate_rate([K] * world, ms_ewald * K / 1000.0),
           "ewald_step": "direct main + 1-4 lists + reciprocal (64^3, order 4), one int64 force array",
           "launches_per_direct_eval": 6}
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as O
        ptr, idx = O.exclusions_csr(d["iblo14"], d["inb14"], n, d["loc2glo"])
        t0 = time.perf_counter()
        O.direct_force(d["xyzq"].astype(np.float64), d["box"], float(d["kappa"]), float(d["roff"]), d["vdwparam"],
                       d["vdwtype"], ptr, idx)
        out["cpu_oracle_ms_main_list"] = (time.perf_counter() - t0) * 1000.0
        out["cpu_oracle_cores"] = O.hardware_threads()
    return out


def serving_stream(n: int, rate: float, seed: int):
    """Poisson arrivals (s), system indices into a pool of batch-distribution systems, evaluation
    counts 1-100 and jitter seeds."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n)) if rate > 0 else np.zeros(n)
    return arrivals, rng.integers(0, 64, size=n), rng.integers(1, 101, size=n), rng.integers(1, 2 ** 62, size=n)


def run_serving(args, dev, rank, world):
    """Requests drawn from the batch distribution (648-24,000 atoms, 24^3-64^3 grids), 1-100
    evaluations each with 0.05 A Gaussian coordinate jitter.  Two arrival patterns over the same
    request mix: every request queued at once (capacity: the server saturated, against the plain
    single-system path saturated), and a Poisson stream at --serve-rate (latency under load).  The
    server is the continuous-batching pme_server_*; the plain path runs one request at a time in
    arrival order through pme_eval_ortho on one stream, each evaluation's jittered coordinates made
    on the device and its energy/virial record delivered to pinned host memory by the evaluation
    itself, with one synchronisation per request (after its last evaluation and the copy of its
    forces).  Latency = completion - arrival; evals/s = all evaluations / (last completion - first
    arrival)."""
    import threading
    import torch
    from gpu_recip_b200 import CudaPMERecip, PmeServer
    from gpu_recip_b200 import replicas as R
    from gpu_recip_b200 import systems as S
    pool = S.batch_systems(64, seed=R.replica_seed(11, rank))
    n = args.serve_requests
    arrivals, idx, nev, seeds = serving_stream(n, args.serve_rate, R.replica_seed(23, rank))
    sigma = 0.05
    total_evals = float(nev.sum())

    def serve(rate_arrivals):
        srv = PmeServer(24 << 30, max_active=256)
        srv.wait(srv.submit(pool[0], n_evals=2, sigma=sigma, seed=1))       # warm-up
        ids = [None] * n
        t0 = time.perf_counter()

        def submitter():
            for i in range(n):
                dt = t0 + rate_arrivals[i] - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
                ids[i] = srv.submit(pool[idx[i]], n_evals=int(nev[i]), sigma=sigma, seed=int(seeds[i]))

        th = threading.Thread(target=submitter)
        th.start()
        th.join()
        res = [srv.wait(rid, timeout=600) for rid in ids]
        st = srv.stats()
        srv.close()
        lat = np.array([r["latency"] for r in res]) * 1000.0
        span = max(r["t_done"] for r in res) - min(r["t_submit"] for r in res)
        return {"evals_per_s": total_evals / span, "p50_ms": float(np.percentile(lat, 50)),
                "p99_ms": float(np.percentile(lat, 99)), "steps": st["steps"], "seconds": span}

    stream = torch.cuda.Stream(device=dev)
    handles = {}
    xs = [torch.from_numpy(sy.xyzq).to(dev) for sy in pool]
    cur = [torch.empty_like(x) for x in xs]
    noise = [torch.empty((sy.natom, 3), dtype=torch.float32, device=dev) for sy in pool]
    fdev = [torch.empty((sy.natom, 3), dtype=torch.float32, device=dev) for sy in pool]
    fhost = [torch.empty((sy.natom, 3), dtype=torch.float32).pin_memory() for sy in pool]
    evh = torch.zeros((int(nev.max()) if n else 1, 11), dtype=torch.float64).pin_memory()
    gen = torch.Generator(device=dev)
    for sy in pool:
        key = (tuple(sy.nfft), sy.order)
        if key not in handles:
            handles[key] = new_handle(args, sy.nfft, sy.order, stream)

    def plain(rate_arrivals):
        lat = []
        count = len(rate_arrivals)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with torch.cuda.stream(stream):
            for i in range(count):
                wait = t0 + rate_arrivals[i] - time.perf_counter()
                if wait > 0:
                    time.sleep(wait)
                j = int(idx[i])
                sy = pool[j]
                pme = handles[(tuple(sy.nfft), sy.order)]
                gen.manual_seed(int(seeds[i]) & 0x7FFFFFFF)
                for k in range(int(nev[i])):
                    torch.randn((sy.natom, 3), generator=gen, device=dev, out=noise[j])
                    cur[j].copy_(xs[j])
                    cur[j][:, :3].add_(noise[j], alpha=sigma)
                    pme.set_energy_virial_mirror(evh[k])
                    pme.eval_ortho([1.0 / b for b in sy.box], cur[j], sy.natom, sy.kappa, True, True, fdev[j], 1)
                fhost[j].copy_(fdev[j], non_blocking=True)
                stream.synchronize()
                lat.append((time.perf_counter() - t0 - rate_arrivals[i]) * 1000.0)
        span = time.perf_counter() - t0
        for pme in handles.values():
            pme.set_energy_virial_mirror(None)
        return {"evals_per_s": float(nev[:count].sum()) / span, "p50_ms": float(np.percentile(lat, 50)),
                "p99_ms": float(np.percentile(lat, 99)), "seconds": span}

    plain(np.zeros(min(n, 4)))                      # warm-up of the plain path's handles
    # capacity: every request queued at once, on the same mix
    server_cap = serve(np.zeros(n))
    plain_cap = plain(np.zeros(n))
    # latency under load: Poisson arrivals at the stated rate
    server_rate = serve(arrivals)
    plain_rate = plain(arrivals)
    arrival_span = float(arrivals[-1]) if n else 0.0
    total = R.sum_over_ranks(total_evals, dev)
    for pme in handles.values():
        pme.close()

    def bound(r):   # the run lasted about as long as the arrivals: its rate is the arrival rate
        return dict(r, arrival_bound=bool(r["seconds"] < 1.1 * arrival_span + 0.05))

    return {"requests": n, "evals": int(total_evals), "sigma_A": sigma, "pool_systems": len(pool),
            "evals_per_request": "uniform 1-100",
            "capacity": {"arrivals": "all requests queued at t = 0", "server": server_cap, "plain_path": plain_cap,
                         "server_over_plain": server_cap["evals_per_s"] / plain_cap["evals_per_s"]},
            "at_rate": {"rate_per_s": args.serve_rate, "arrival_span_s": arrival_span,
                        "server": bound(server_rate), "plain_path": bound(plain_rate)},
            "all_ranks_evals": total}


def fft_comparator(s, dev, flush, reps: int = 30):
    """cuFFT (torch.fft) 3-D R2C and C2R beside this engine's staged pme_r2c_fft and pme_c2r_fft
    (which also convert the fixed-point grid, or write the real grid), each timed with CUDA events
    and L2 flushed before every transform, on the workload's grid, the 216^3 grid and the
    smallest, median and largest grids of the 256-system batch.  Timing only: cuFFT is never on
    the product path."""
    import torch
    from gpu_recip_b200 import CudaPMERecip
    from gpu_recip_b200 import systems as S
    grids = [tuple(s.nfft), (216, 216, 216)]
    batch = sorted({tuple(sy.nfft) for sy in S.batch_systems(256, seed=4)}, key=lambda g: g[0] * g[1] * g[2])
    for g in (batch[0], batch[len(batch) // 2], batch[-1]):
        if g not in grids:
            grids.append(g)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        tot = 0.0
        for r in range(reps + 3):
            flush.fill_(float(r & 7))
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            if r >= 3:
                tot += e0.elapsed_time(e1)
        return 1000.0 * tot / reps

    out = []
    for (nx, ny, nz) in grids:
        g = torch.randn((nz, ny, nx), dtype=torch.float32, device=dev)
        h = torch.fft.rfftn(g)
        pme = CudaPMERecip(nx, ny, nz, 4)
        row = {"grid": [nx, ny, nz],
               "cufft_r2c_us": timed(lambda: torch.fft.rfftn(g)),
               "cufft_c2r_us": timed(lambda: torch.fft.irfftn(h, s=(nz, ny, nx))),
               "b200_r2c_fft_us": timed(pme.r2c_fft),
               "b200_c2r_fft_us": timed(pme.c2r_fft)}
        pme.close()
        out.append(row)
    return {"grids": out, "l2": "flushed (256 MiB write) before every transform, both arms",
            "note": "cuFFT timed as a comparator only (torch.fft)"}


def stage_times(pme, s, x, f, stride, recip, stream, flush, reps: int = 50):
    import torch
    names = ["spread", "r2c_fft", "scalar_sum", "c2r_fft", "gather", "self_energy"]
    acc = {k: 0.0 for k in names}
    n = s.natom
    with torch.cuda.stream(stream):
        for r in range(reps + 3):
            flush.fill_(0.0)
            # the GPU spins while the host enqueues the six calls, so that the events time the
            # device work of each call, not the host's submission rate
            torch.cuda._sleep(400000)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(len(names) + 1)]
            ev[0].record(stream)
            pme.spread_charge(x, n, recip); ev[1].record(stream)
            pme.r2c_fft(); ev[2].record(stream)
            pme.scalar_sum(recip, s.kappa, True, True); ev[3].record(stream)
            pme.c2r_fft(); ev[4].record(stream)
            pme.gather_force(x, n, recip, stride, f); ev[5].record(stream)
            pme.calc_self_energy(x, n, s.kappa); ev[6].record(stream)
            stream.synchronize()
            if r >= 3:
                for i, k in enumerate(names):
                    acc[k] += ev[i].elapsed_time(ev[i + 1])
    return {k: v / reps for k, v in acc.items()}


def sequence_time(pme, s, x, f, stride, recip, stream, flush, reps: int = 50):
    """The six reference-interface calls and the record clear timed as one sequence, as the
    reference's own driver loop is timed (events around the whole sequence, L2 flushed before it;
    the GPU held while the host enqueues it).  Mean ms."""
    import torch
    n = s.natom
    tot = 0.0
    with torch.cuda.stream(stream):
        for r in range(reps + 3):
            torch.cuda._sleep(400000)
            flush.fill_(0.0)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            pme.energy_virial.clear()
            pme.spread_charge(x, n, recip)
            pme.r2c_fft()
            pme.scalar_sum(recip, s.kappa, True, True)
            pme.c2r_fft()
            pme.gather_force(x, n, recip, stride, f)
            pme.calc_self_energy(x, n, s.kappa)
            b.record(stream)
            stream.synchronize()
            if r >= 3:
                tot += a.elapsed_time(b)
    return tot / reps


def main():
    args = parse()
    mode, n = replica_plan(args.gpus)
    if mode == "spawn":
        sys.exit(spawn_replicas(n))
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
