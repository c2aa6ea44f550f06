#!/usr/bin/env python3
"""Benchmark: restricted CCSD(T) at o=45, v=477 (the 522-basis-function
9 H2O / cc-pVTZ shape) on B200, FP64 DMMA path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one pass of the triples engine over a fixed, evenly strided sample
of the workload's triples queue (every 211th of its 58,740 triples: 68
same-spin + 211 mixed-spin triples, ~1.1e14 flops), with every operand
resident in HBM (74 GB of pt.h inputs; the engine's padded copies).  The
metric is TFLOP/s of the reference's own contraction flops (twice the
multiply-adds of its dgemm_ calls for those triples); the projected full-solve
time is the queue's flops over that rate.

Lines printed (rank 0, one JSON line):
  value      whole-job TFLOP/s, device-resident operands, CUDA-event timed
  e2e        libpt_rpt (host arrays, the reference-facing C ABI) on a full
             solve of o=4, v=477 with the host->device copies inside the
             timed region
  roofline   the contraction kernel (gemm_dmma_kernel): achieved FP64 TFLOP/s
             from CUDA events around each launch over the measured FP64
             tensor peak (cuBLAS DGEMM measured here, MEASURED_PEAKS.json
             having no FP64 figure)
  cpu_baseline  the reference library (oracle/_ref, OpenMP + OpenBLAS) timed
             on the host cores on a full solve of o=2, v=477 (rank 0, N=1),
             with the o=45 solve's time extrapolated from that rate
  precision_table  |dE| of every precision form: restricted o=8, v=64
             against the reference run with one thread (plus the
             reference's own 1-vs-all-threads spread), then unrestricted (T)
             and (fT) against the FP64 path
--impl reference prints the reference's own CPU implementation on the same
sample workload (o=2, v=477 full solves), with all host threads.

Multi-GPU (torchrun): the ranks shard one solve the way the reference's MPI
build does (src/pt.c:213, 474-477): identical inputs on every GPU, a sample
N times denser whose entry q runs on rank q % N, and per step one sum
all-reduce of the per-triple energy slots (NCCL); scaling "weak" (fixed
triples per GPU), time = max over ranks.  The e2e figure stays one host-API
solve per rank.
"""
import argparse
import csv
import io
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

O_FULL, V_FULL = 45, 477      # the workload (restricted, all-electron)
STRIDE = 211                  # triples-queue sampling stride of one step
O_E2E = 4                     # full solves through the host API
O_CPU = 2                     # full solves of the reference on the host


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--o", type=int, default=O_FULL)
    ap.add_argument("--v", type=int, default=V_FULL)
    ap.add_argument("--stride", type=int, default=STRIDE)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-worker", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--cpu-o", type=int, default=O_CPU)
    ap.add_argument("--cpu-reps", type=int, default=1)
    ap.add_argument("--precision", default="fp64,emu64",
                    help="comma list of fp64, emu64, tf32x3; the first is "
                         "the headline value")
    ap.add_argument("--serve-slices", type=int, default=6,
                    help="digit slices of the served stream's emulated half")
    ap.add_argument("--slices", type=int, default=0,
                    help="emulated FP64 digit slices (4..7; 0: chosen by the "
                         "plan for LIBPT_EMU_TOL, default 1e-6 Eh)")
    ap.add_argument("--serve-requests", type=int, default=40,
                    help="requests of the served stream (0: skip)")
    ap.add_argument("--serve-rate", type=float, default=20.0,
                    help="Poisson arrival rate of the served stream (req/s)")
    ap.add_argument("--serve-budget-gb", type=float, default=150.0)
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the precision table (unrestricted (T) and (fT))")
    ap.add_argument("--accuracy-rft", action="store_true",
                    help="add restricted (fT) o=30 v=300 to the table (~2 min)")
    return ap.parse_args()


PRECISIONS = {"fp64": 0, "tf32x3": 1, "emu64": 2}

# DRAM bytes (read + write) per reference flop of the contraction kernels,
# from one ncu capture each of restricted (T) o=2, v=477 (two mixed-spin
# triples, 9.26e11 flops; profiles/gemm_dmma_rpt_o2_v477_fp64_full.txt and
# profiles/gemm_i8_rpt_o2_v477_emu64s5_full.txt).  A launch's traffic grows
# with its triples (each reads its own operand slices and writes its own
# outputs), so the bench scales these by the flops of its launches.
DRAM_BYTES_PER_FLOP = {"gemm_dmma_kernel": (7.141e9 + 4.338e9) / 9.26e11,
                       "gemm_i8_kernel": (11.637e9 + 4.342e9) / 9.26e11}


# ------------------------------------------------------------------ helpers


def rpt_flops(o, v):
    """Reference dgemm_ flops of libpt_rpt (src/pt.c:49,65,81,97,110,126,
    142,158): C(o,3)[3v^3(v-1)+6ov^3] + C(o,2)o[6v^4+2v^3(v-1)+10ov^3]."""
    c3 = o * (o - 1) * (o - 2) / 6.0
    c2o = o * (o - 1) / 2.0 * o
    v = float(v)
    return (c3 * (3 * v**3 * (v - 1) + 6 * o * v**3)
            + c2o * (6 * v**4 + 2 * v**3 * (v - 1) + 10 * o * v**3))


class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None

    def init(self, backend):
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group(backend,
                                    timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x):
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x):
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        self.pg.all_reduce(t)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during a region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.out = None

    def start(self):
        try:
            self.out = open(os.path.join("/tmp", f"clocks_{os.getpid()}.csv"),
                            "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.gpu_id, "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.close()
        rows = []
        with open(self.out.name) as fp:
            for r in csv.reader(fp):
                if len(r) >= 8:
                    rows.append([x.strip() for x in r])
        os.unlink(self.out.name)
        if not rows:
            return None
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = max(float(r[1]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if r[4 + i].lower() == "active"})
        load = [s for s in sm if s > 0.5 * mx] or sm
        return dict(sm_mhz=float(np.median(load)), sm_max_mhz=mx,
                    reasons=reasons, samples=len(rows),
                    power_w_max=max(float(r[2]) for r in rows
                                    if r[2].replace(".", "").isdigit()))


def fp64_peak_tflops(torch):
    """Burst FP64 tensor-core throughput of cuBLAS DGEMM (n=8192), best of 5."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(True), torch.cuda.Event(True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2.0 * n**3 / (s.elapsed_time(e) / 1e3) / 1e12)
    del a, b
    return best


def cpu_worker(args):
    """Time the reference library (oracle/_ref) on full rpt solves of
    (cpu-o, v); prints one JSON line.  Run in a subprocess so that the
    OpenMP/OpenBLAS thread counts apply from library load."""
    from libpt_b200 import synth
    from oracle import oracle
    case = synth.rpt_case(args.cpu_o, args.v, seed=7)
    ref = oracle.reference()
    oracle.solve(ref, synth.rpt_case(2, 24, seed=1))   # load + thread spin-up
    t0 = time.perf_counter()
    for _ in range(args.cpu_reps):
        e = oracle.solve(ref, case)
    dt = (time.perf_counter() - t0) / args.cpu_reps
    print(json.dumps(dict(seconds=dt, flops=rpt_flops(args.cpu_o, args.v),
                          energy=e)))


def run_cpu(o, v, reps, threads_mode="blas"):
    n = os.cpu_count() or 1
    env = dict(os.environ)
    if threads_mode == "blas":    # few triples: give the cores to BLAS
        env.update(OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS=str(n))
    elif threads_mode == "single":  # one thread: a fixed summation order
        n = 1
        env.update(OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1")
    else:                         # OpenMP over triples (src/pt.c:227-230)
        env.update(OMP_NUM_THREADS=str(n), OPENBLAS_NUM_THREADS="1")
    r = subprocess.run([sys.executable, os.path.abspath(__file__),
                        "--cpu-worker", "--cpu-o", str(o), "--v", str(v),
                        "--cpu-reps", str(reps)],
                       env=env, capture_output=True, text=True, timeout=1800)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-2000:])
    out = json.loads(r.stdout.strip().splitlines()[-1])
    out["cores"] = n
    out["threads"] = threads_mode
    return out


def extrapolation(args, tflops):
    """The full o, v solve on the host cores, extrapolated from the measured
    sample rate (the workload's queue flops over that rate: a solve too large
    for the host's memory and hours of CPU time is not run in full)."""
    return dict(
        extrapolated_solve_seconds=rpt_flops(args.o, args.v) / (tflops * 1e12),
        extrapolation=f"extrapolated: rpt o={args.o} v={args.v} reference "
                      f"flops ({rpt_flops(args.o, args.v):.4g}) over the rate "
                      f"measured on the o={args.cpu_o} v={args.v} sample")


# ------------------------------------------------------------------ arms


def workload_config(args, world):
    """The `config` both arms report: the sampled o, v workload of one step
    (restricted queue: C(o,3) same-spin then C(o,2)*o mixed-spin triples;
    per-triple flops of src/pt.c's dgemm_ calls, as rpt_flops)."""
    o, v = args.o, float(args.v)
    naaa = o * (o - 1) * (o - 2) // 6
    n = naaa + o * (o - 1) // 2 * o
    stride = max(1, args.stride // world)
    sample = np.arange(0, n, stride, dtype=np.int64)
    nsame = int((sample < naaa).sum())
    f_aaa = 3 * v**3 * (v - 1) + 6 * o * v**3
    f_aab = 6 * v**4 + 2 * v**3 * (v - 1) + 10 * o * v**3
    return dict(
        workload=f"rpt o={args.o} v={args.v}: every {stride}th triple of the "
                 f"{n}-entry queue per step ({len(sample)} triples, {nsame} "
                 "same-spin)",
        precision=args.precision.split(",")[0],
        parallelism="1 GPU" if world == 1 else
        f"triples sharded x{world} (entry q on rank q % {world}), one "
        "energy-slot all-reduce per step",
        l2="inputs (74 GB) larger than L2; no flush needed",
        flops_per_step=nsame * f_aaa + (len(sample) - nsame) * f_aab)


def run_reference(args, d):
    """Reference arm: the reference's own CPU implementation (oracle/_ref:
    src/pt.c + OpenBLAS, OpenMP) on full solves of o=2, v=477."""
    if d.rank != 0:
        return
    from oracle import oracle
    if not os.path.exists(oracle.reference_path()):
        print(json.dumps(dict(impl="reference", unavailable=(
            "oracle/_ref/libpt_ref.so was not built (needs the reference "
            "source tree at build time)"))))
        return
    if args.warmup > 0:
        run_cpu(args.cpu_o, args.v, 1)
    t0 = time.perf_counter()
    res = run_cpu(args.cpu_o, args.v, max(args.steps, 1))
    wall = time.perf_counter() - t0
    val = res["flops"] / res["seconds"] / 1e12
    line = dict(
        metric="(T) TFLOP/s, restricted o=45 v=477 workload (reference "
               "dgemm flops per second)",
        value=val, unit="TFLOP/s", n_gpus=args.gpus, steps=args.steps,
        warmup=args.warmup, ms_per_step=res["seconds"] * 1e3,
        higher_is_better=True, scaling="weak", vs_baseline=None,
        dtype="f64", data="synthetic", impl="reference",
        config=workload_config(args, args.gpus),
        cpu_baseline=dict(value=val, unit="TFLOP/s", cores=res["cores"],
                          kind="reference",
                          sample=f"bounded sample of the workload: full "
                                 f"libpt_rpt solves of o={args.cpu_o} "
                                 f"v={args.v} (the same virtual space; "
                                 f"OpenMP 1 thread, OpenBLAS "
                                 f"{res['cores']} threads)",
                          **extrapolation(args, val)),
        e2e=dict(value=val, unit="TFLOP/s", h2d_bytes_per_step=0,
                 d2h_bytes_per_step=0),
        wall_seconds=wall)
    print(json.dumps(line))


def run_ours(args, d):
    import torch
    from libpt_b200 import ffi, synth

    torch.cuda.set_device(d.local)
    d.init("nccl")
    dev = torch.device("cuda", d.local)
    props = torch.cuda.get_device_properties(dev)
    gpu_id = "GPU-" + str(props.uuid) if getattr(props, "uuid", None) else "0"

    peak64 = fp64_peak_tflops(torch)

    # ---- operands: generated on the device, then planned (resident) -------
    t_gen = time.perf_counter()
    # the same inputs on every rank (a sharded solve needs identical copies)
    meta, tens = synth.rpt_case_device(args.o, args.v, seed=1000, device=dev)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t_gen
    naaa = args.o * (args.o - 1) * (args.o - 2) // 6

    def measure(prec_name):
        prec = PRECISIONS[prec_name]
        if prec == 2:
            prec |= args.slices << 8
        t0 = time.perf_counter()
        mp = prec_name == "tf32x3"
        src = {k: x.float() for k, x in tens.items()} if mp else tens
        plan = ffi.Plan(meta, src, mp=mp, precision=prec)
        del src
        torch.cuda.synchronize()
        t_plan = time.perf_counter() - t0
        # N ranks: a sample N times denser, entry q of it on rank q % N
        gsample = np.arange(0, plan.n, max(1, args.stride // d.world),
                            dtype=np.int64)
        sample = gsample[d.rank::d.world]
        flops_step = sum(plan.flops(int(q), 1) for q in sample)
        flops_all = d.sum(flops_step)
        flops_full = plan.flops()
        slots = exch = None
        if d.world > 1:
            # the ranks' energies meet in one slot all-reduce per step; the
            # plan's own slots keep only this rank's entries
            slots = plan.energy_slots()
            exch = torch.empty_like(slots)

        def step():
            plan.run(sample)
            if exch is not None:
                exch.copy_(slots)
                d.pg.all_reduce(exch)

        for _ in range(args.warmup):
            step()
            plan.energy(sample)
        plan.timing(True)
        plan.kernel_stats()
        clocks = Clocks(gpu_id)
        clocks.start()
        d.barrier()
        torch.cuda.synchronize()
        s_ev, e_ev = torch.cuda.Event(True), torch.cuda.Event(True)
        s_ev.record()
        for _ in range(args.steps):
            step()
        e_ev.record()
        torch.cuda.synchronize()
        d.barrier()
        clk = clocks.stop()
        secs = s_ev.elapsed_time(e_ev) / 1e3
        secs_max = d.max(secs)
        stats = plan.kernel_stats()
        if exch is not None:    # the whole sample's energy, from the exchange
            energy = 2.0 * ffi.energy_sum(exch.cpu().numpy()[gsample])
            del slots
        else:
            energy = plan.energy(sample)
        n = plan.n
        chosen = plan.slices
        plan.close()
        torch.cuda.empty_cache()
        return dict(sample=sample, flops_step=flops_step, flops_full=flops_full,
                    secs=secs, secs_max=secs_max, stats=stats, clk=clk,
                    energy=energy, n=n, plan_seconds=t_plan, slices=chosen,
                    flops_all=flops_all, nsample=len(gsample),
                    nsame=int((gsample < naaa).sum()),
                    value=args.steps * flops_all / secs_max / 1e12,
                    gemm=stats["gemm_flops"] / (stats["gemm_ms"] / 1e3) / 1e12)

    runs = {}
    for name in args.precision.split(","):
        runs[name] = measure(name)
    del tens
    torch.cuda.empty_cache()
    head = args.precision.split(",")[0]
    R0 = runs[head]
    sample, flops_step, flops_full = R0["sample"], R0["flops_step"], R0["flops_full"]
    secs, secs_max, stats, clk = R0["secs"], R0["secs_max"], R0["stats"], R0["clk"]
    energy_sample = R0["energy"]
    value = R0["value"]
    ach = R0["gemm"]
    plan_n = R0["n"]

    # ---- e2e: reference-facing host API, copies inside the timed region ---
    e2e = None
    if not args.no_e2e:
        case = synth.rpt_case(O_E2E, args.v, seed=77 + d.rank)
        arrs = {n: np.ascontiguousarray(case[n]) for n in ffi.PT_ARGS}
        case.update(arrs)
        h2d = sum(a.nbytes for a in arrs.values())
        ffi.solve_host(case)                       # warm-up
        reps = 2
        d.barrier()
        t0 = time.perf_counter()
        for _ in range(reps):
            ffi.solve_host(case)
        t_e2e = (time.perf_counter() - t0) / reps
        t_e2e = d.max(t_e2e)
        nq = O_E2E * (O_E2E - 1) * (O_E2E - 2) // 6 + \
            O_E2E * (O_E2E - 1) // 2 * O_E2E
        e2e = dict(value=d.world * rpt_flops(O_E2E, args.v) / t_e2e / 1e12,
                   unit="TFLOP/s", h2d_bytes_per_step=h2d,
                   d2h_bytes_per_step=8 * (nq + 1) + 4,
                   seconds_per_solve=t_e2e,
                   workload=f"libpt_rpt(o={O_E2E}, v={args.v}) host arrays, "
                            "full solve")

    serving = None
    if args.serve_requests > 0:
        serving = run_serving(args, torch, gpu_id)
    accuracy = None
    if not args.no_accuracy:
        accuracy = run_accuracy(args, torch)
        if d.rank == 0:
            try:
                accuracy.insert(0, run_accuracy_reference(torch))
            except Exception as ex:   # report, do not fail the bench
                accuracy.insert(0, dict(kind="rpt", sizes=[8, 64],
                                        failed=f"{ex}"[:300]))

    cpu = None
    if not args.no_cpu and d.world == 1 and d.rank == 0:
        try:
            r = run_cpu(args.cpu_o, args.v, 1)
            rate = r["flops"] / r["seconds"] / 1e12
            cpu = dict(value=rate, unit="TFLOP/s",
                       cores=r["cores"], kind="reference",
                       sample=f"reference libpt_rpt (oracle/_ref) full solve "
                              f"o={args.cpu_o} v={args.v}, "
                              f"{r['seconds']:.1f} s; OpenMP 1 thread, "
                              f"OpenBLAS {r['cores']} threads",
                       **extrapolation(args, rate))
        except Exception as ex:   # report, do not fail the bench
            cpu = dict(value=None, unit="TFLOP/s", cores=os.cpu_count(),
                       kind="reference", sample=f"failed: {ex}"[:300])

    if d.rank == 0:
        line = dict(
            metric="(T) TFLOP/s, restricted o=45 v=477 workload (reference "
                   "dgemm flops per second)",
            value=value, unit="TFLOP/s", n_gpus=d.world, steps=args.steps,
            warmup=args.warmup, ms_per_step=secs_max / args.steps * 1e3,
            higher_is_better=True, scaling="weak", vs_baseline=None,
            dtype="f64", data="synthetic",
            config=workload_config(args, d.world),
            projected_solve_seconds=flops_full / (value * 1e12),
            roofline=dict(bound="tensor", achieved=ach, peak=peak64,
                          unit="TFLOP/s", frac=ach / peak64,
                          traffic=DRAM_BYTES_PER_FLOP["gemm_dmma_kernel"] *
                          stats["gemm_flops"] / max(stats["gemm_launches"], 1),
                          traffic_note="bytes per launch, scaled from the "
                                       "o=2 v=477 ncu capture by flops",
                          kernel="gemm_dmma_kernel",
                          peak_source="cuBLAS DGEMM n=8192 burst, measured "
                                      "in this run (FP64 tensor)",
                          launches=stats["gemm_launches"],
                          epilogue_ms_share=stats["epi_ms"] /
                          max(secs * 1e3, 1e-9)),
            cpu_baseline=cpu, e2e=e2e, clocks=clk, serving=serving,
            precision_table=accuracy,
            gpu_launches=stats["launches"],
            energy_sample=energy_sample, setup_seconds=t_gen)
        for name, Rr in runs.items():
            if name == head:
                continue
            line[name] = dict(
                value=Rr["value"], unit="TFLOP/s",
                ratio_to_head=Rr["value"] / value,
                ms_per_step=Rr["secs_max"] / args.steps * 1e3,
                projected_solve_seconds=Rr["flops_full"] / (Rr["value"] * 1e12),
                gemm_tflops=Rr["gemm"],
                gemm_traffic_per_launch=(
                    DRAM_BYTES_PER_FLOP["gemm_i8_kernel"] *
                    Rr["stats"]["gemm_flops"] /
                    max(Rr["stats"]["gemm_launches"], 1))
                if name == "emu64" else None,
                energy_sample=Rr["energy"],
                energy_sample_delta=Rr["energy"] - energy_sample,
                slices=Rr["slices"] if name == "emu64" else None,
                slice_choice=("chosen by the plan for |dE| <= "
                              f"{os.environ.get('LIBPT_EMU_TOL', '1e-6')} Eh "
                              "(sampled error estimate)")
                if name == "emu64" and args.slices == 0 else
                (f"fixed at {args.slices}" if name == "emu64" else None),
                epilogue_ms_share=Rr["stats"]["epi_ms"] / max(Rr["secs"] * 1e3, 1e-9),
                plan_seconds=Rr["plan_seconds"], clocks=Rr["clk"])
        print(json.dumps(line))
    d.close()


def serve_stream(n, rate, seed):
    """The served workload: restricted (T) requests with o ~ U{4..24},
    v = round(o * U[6, 12]), Poisson arrivals at `rate` per second, half
    FP64 and half emulated FP64, one input seed per request."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    reqs = []
    for i in range(n):
        o = int(rng.integers(4, 25))
        v = int(round(o * rng.uniform(6.0, 12.0)))
        reqs.append(dict(o=o, v=v, seed=10_000 + i, emu=bool(i % 2),
                         arrival=float(t[i] - t[0])))
    return reqs


def percentile(x, q):
    return float(np.percentile(np.asarray(x), q)) if len(x) else None


def run_serving(args, torch, gpu_id):
    """Served stream through the continuous-batching server (pt_serve.h):
    each request's inputs are generated on the device when it arrives and
    submitted; latency runs from submission to its energy.  Beside it, the
    same requests as one-at-a-time FP64 solves (libpt plan per request,
    FIFO at the same arrival times, queueing computed from the measured
    service times)."""
    from libpt_b200 import ffi, synth
    reqs = serve_stream(args.serve_requests, args.serve_rate, seed=4)
    emu = ffi.PREC_EMU64 | (args.serve_slices << 8)
    budget = int(args.serve_budget_gb * (1 << 30))
    free = torch.cuda.mem_get_info()[0]
    # room beside the pool for arriving requests' inputs until admission
    budget = min(budget, int(free - (24 << 30)))
    flops = 0.0
    srv = ffi.Server(mem_budget=budget)
    clocks = Clocks(gpu_id)
    clocks.start()
    t0 = time.perf_counter()
    tickets = []
    for r in reqs:
        while time.perf_counter() - t0 < r["arrival"]:
            time.sleep(0.0005)
        srv.release_inputs()            # inputs already resident in the pool
        meta, tens = synth.rpt_case_device(r["o"], r["v"], seed=r["seed"])
        torch.cuda.synchronize()
        tickets.append(srv.submit(meta, tensors=tens,
                                  precision=emu if r["emu"] else 0))
        del tens
        flops += rpt_flops(r["o"], r["v"])
    lat, energies = [], []
    for tk in tickets:
        e, l = srv.wait(tk)
        lat.append(l)
        energies.append(e)
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    st = srv.stats()
    srv.close()
    torch.cuda.empty_cache()
    # one-at-a-time FP64 solves of the same requests
    service = []
    for r in reqs:
        meta, tens = synth.rpt_case_device(r["o"], r["v"], seed=r["seed"])
        torch.cuda.synchronize()
        a = time.perf_counter()
        p = ffi.Plan(meta, tens)
        p.run()
        p.energy()
        p.close()
        service.append(time.perf_counter() - a)
        del tens
    torch.cuda.empty_cache()
    done, blat = 0.0, []
    for r, sv in zip(reqs, service):
        done = max(done, r["arrival"]) + sv
        blat.append(done - r["arrival"])
    return dict(
        workload=f"{len(reqs)} restricted (T) requests, o~U{{4..24}}, "
                 f"v=round(o*U[6,12]), Poisson {args.serve_rate:g} req/s, "
                 f"half FP64 / half emulated FP64 ({args.serve_slices} slices), "
                 "inputs generated on the device at arrival",
        solves_per_s=len(reqs) / wall, p50_s=percentile(lat, 50),
        p99_s=percentile(lat, 99), tflops=flops / wall / 1e12,
        rounds=st["rounds"], graph_rounds=st["graph_rounds"],
        max_resident=st["max_resident"],
        peak_pool_gb=st["peak_bytes_in_use"] / 2**30,
        pool_gb=st["pool_bytes"] / 2**30, clocks=clk,
        one_at_a_time_fp64=dict(
            solves_per_s=len(reqs) / done, p50_s=percentile(blat, 50),
            p99_s=percentile(blat, 99),
            note="sequential FP64 plan per request, FIFO queue at the same "
                 "arrivals (service times measured)"))


def precision_forms(ffi):
    """(name, precision word, FP32 inputs) of every form the tables report."""
    forms = [("fp64", ffi.PREC_FP64, False)]
    forms += [(f"emu64_s{s}", ffi.PREC_EMU64 | (s << 8), False)
              for s in (4, 5, 6, 7)]
    forms += [("emu64_auto", ffi.PREC_EMU64, False)]   # S chosen for 1 uEh
    forms += [("tf32x3", ffi.PREC_TF32X3, True)]
    return forms


def run_accuracy_reference(torch, o=8, v=64, seed=7):
    """Restricted (T) o=8, v=64 (host inputs, seed 7) in every precision form
    against the reference build run with one OpenMP and one BLAS thread (a
    fixed summation order), plus the reference's own spread between that
    run and one with OpenMP over triples on all host cores (src/pt.c:227-230,
    a dynamic schedule whose summation order varies)."""
    from libpt_b200 import ffi, synth
    from oracle import oracle
    row = dict(kind="rpt", sizes=[o, v], seed=seed)
    if not os.path.exists(oracle.reference_path()):
        row["unavailable"] = "oracle/_ref/libpt_ref.so was not built"
        return row
    r1 = run_cpu(o, v, 1, "single")
    rn = run_cpu(o, v, 1, "omp")
    e_ref = r1["energy"]
    row.update(reference_energy=e_ref,
               reference="oracle/_ref, OpenMP 1 thread, OpenBLAS 1 thread",
               reference_thread_spread_Eh=abs(rn["energy"] - e_ref),
               reference_threads=rn["cores"])
    case = synth.rpt_case(o, v, seed=seed)
    dev = {n: torch.as_tensor(case[n]).to(device="cuda", dtype=torch.float64)
           for n in ffi.PT_ARGS}
    res = {}
    for name, prec, mp in precision_forms(ffi):
        src = {k: x.float() for k, x in dev.items()} if mp else dev
        p = ffi.Plan(case, src, mp=mp, precision=prec)
        try:
            p.run()
            e = p.energy()
            sl = p.slices or None
        finally:
            p.close()
        res[name] = dict(energy=e, slices=sl, dE_uEh=abs(e - e_ref) * 1e6,
                         dE_rel=abs(e - e_ref) / abs(e_ref) if e_ref else None)
    row["forms"] = res
    return row


def run_accuracy(args, torch):
    """Full solves of unrestricted (T) oa=20 va=180 ob=18 vb=182 and
    unrestricted (fT) o=15 v=150 (spin blocks 15/150 each), inputs generated
    on the device, in every precision form: FP64 (DMMA), emulated FP64 with
    4-7 INT8 slices, and 3xTF32 on the FP32 inputs.  |dE| against the FP64
    path (the FP64 path matches the reference FP64 build to <= 1e-12 |E| in
    the parity tests; the CPU reference itself would need ~10 min here).
    Seconds exclude plan creation (reported apart)."""
    from libpt_b200 import ffi, synth
    cases = [("upt", (20, 180, 18, 182)), ("uft", (15, 150, 15, 150))]
    if args.accuracy_rft:
        cases.append(("rft", (30, 300)))
    forms = precision_forms(ffi)
    rows = []
    for kind, sz in cases:
        meta, tens = synth.case_device(kind, *sz, seed=7)
        res = {}
        for name, prec, mp in forms:
            src = {k: x.float() for k, x in tens.items()} if mp else tens
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            p = ffi.Plan(meta, src, mp=mp, precision=prec)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            p.run()
            e = p.energy()
            t2 = time.perf_counter()
            fl = p.flops()
            sl = p.slices or None
            p.close()
            del src
            res[name] = dict(seconds=t2 - t1, plan_seconds=t1 - t0,
                             tflops=fl / (t2 - t1) / 1e12, energy=e,
                             slices=sl)
        e64 = res["fp64"]["energy"]
        for name, r in res.items():
            r["dE_uEh"] = abs(r["energy"] - e64) * 1e6
            r["dE_rel"] = abs(r["energy"] - e64) / abs(e64) if e64 else None
            r["speedup_vs_fp64"] = res["fp64"]["seconds"] / r["seconds"]
        rows.append(dict(kind=kind, sizes=list(sz), flops=fl, forms=res))
        del tens
        torch.cuda.empty_cache()
    return rows


def main():
    args = parse()
    if args.cpu_worker:
        cpu_worker(args)
        return
    d = Dist()
    if args.impl == "reference":
        run_reference(args, d)
        return
    run_ours(args, d)


if __name__ == "__main__":
    main()
