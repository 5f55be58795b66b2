#!/usr/bin/env python
"""Benchmark: 30-qubit complex128 circuit (H on all qubits, RZ(theta_q), full
QFT = 540 gates) executed through the fused planner, then sample(1,000,000)
and measure() -- one "step".  Prints ONE JSON line (rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value      gates/s of the whole step with the circuit, draws and results in
           device memory (CUDA events on the library's stream, max over ranks).
e2e        the same step through the public Python API (Circuit): op list
           host->device, indices device->host, inside the timed region.
roofline   the fused pass kernel: algorithmic bytes (32 B per amplitude per
           pass) / its mean per-launch device time, against the measured HBM
           copy bandwidth.
cpu_baseline / --impl reference
           the reference's own AVX2/OpenMP backend (compiled from its sources
           into oracle/_ref) on the host cores, on a bounded prefix of the same
           circuit plus the full sample(1e6) and measure(), extrapolated to
           the 540-gate step.
qaoa       adjoint gradients/s (24-qubit 3-regular Max-Cut, p=8, 16 params)
           vs the parameter-shift rule with one kernel per gate, and the max
           difference between the two gradients.
batch      512 parameterised circuits (widths 10..22): forward <O> and the full
           adjoint gradient of each, one persistent kernel per run replayed as
           a CUDA graph, against parameter shift with one kernel per gate.
           --batch-only runs just this section (--batch-circuits/-wmin/-wmax
           set a smaller case, --no-autotune keeps the default configuration).
Multi-GPU: the state does not shard here; every rank runs its own replica
(weak scaling), value = sum over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_QUBITS = 30
SHOTS = 1_000_000
METRIC = "30q gates/s + HBM GB/s vs peak; QAOA grads/s adjoint vs param-shift @1e-10"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--qubits", type=int, default=N_QUBITS)
    ap.add_argument("--shots", type=int, default=SHOTS)
    ap.add_argument("--no-qaoa", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--batch-only", action="store_true", help="only the batched forward+adjoint section")
    ap.add_argument("--batch-circuits", type=int, default=512)
    ap.add_argument("--batch-wmin", type=int, default=10)
    ap.add_argument("--batch-wmax", type=int, default=22)
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-gates", type=int, default=0, help="gates in the CPU sample (0 = auto)")
    ap.add_argument("--tile", type=int, default=0, help="tile qubits of the fused passes (0 = library default)")
    ap.add_argument("--playground", default=None,
                    help="comma-separated playground workloads (or 'all'): the paper's construct -> execute -> "
                         "sample wall-clock timings, one JSON line instead of the step")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"qse_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
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
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    smax = float(p[2])
                except ValueError:
                    continue
                for nm, v in zip(names, p[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- CPU reference
def cpu_reference_step(n, ops, shots, max_gates, threads):
    """The reference's own Circuit on its AVX2 backend, bounded: the first
    `g` gates timed and extrapolated; sample(shots) and measure() timed in full.
    Returns (gates_per_s, seconds_of_cpu_work, description, kind)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import numpy as np

    import oracle_ffi as O
    ref = O.load_reference(gpu=False)
    if ref is None:
        return None
    ref.ref_set_quiet(1)
    assert ref.ref_set_backend(1) == 0  # CircuitUnitaryOperationAVX
    h = ref.ref_circuit_new(n, 0)
    g = max(1, min(max_gates, len(ops)))
    sub = np.ascontiguousarray(ops[:g])
    ref.ref_circuit_add_many(h, sub.ctypes.data_as(C.c_void_p), g)
    t0 = time.perf_counter()
    ref.ref_circuit_execute(h, 0)
    t_gates = time.perf_counter() - t0
    out = np.empty(shots, dtype=np.uint64)
    t0 = time.perf_counter()
    ref.ref_circuit_sample(h, shots, out.ctypes.data_as(C.POINTER(C.c_uint64)))
    t_sample = time.perf_counter() - t0
    t0 = time.perf_counter()
    ref.ref_circuit_measure(h)
    t_measure = time.perf_counter() - t0
    ref.ref_circuit_free(h)
    ref.ref_set_backend(0)
    step = t_gates / g * len(ops) + t_sample + t_measure
    desc = (f"reference Circuit on CircuitUnitaryOperationAVX, OMP_NUM_THREADS={threads}: first {g} of "
            f"{len(ops)} gates timed ({t_gates:.2f} s) and scaled to {len(ops)}, + sample({shots}) "
            f"{t_sample:.2f} s + measure() {t_measure:.2f} s at {n} qubits")
    return len(ops) / step, t_gates + t_sample + t_measure, desc, "reference"


def run_reference_arm(args, rank):
    import numpy as np  # noqa: F401

    from quantumsimevo_b200 import workloads as W
    if rank != 0:
        return
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    ops = W.hrz_qft(args.qubits, seed=2)
    gates = args.cpu_gates or 4
    vals, work = [], 0.0
    desc, kind = "", "reference"
    for i in range(args.warmup + args.steps):
        r = cpu_reference_step(args.qubits, ops, args.shots, gates, threads)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libqse_ref_cpu.so not built"}))
            return
        v, w, desc, kind = r
        if i >= args.warmup:
            vals.append(v)
            work += w
    v = statistics.median(vals)
    line = {
        "metric": METRIC, "value": v, "unit": "gates/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * len(ops) / v, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"H+RZ+QFT {args.qubits}q complex128 ({len(ops)} gates) + sample({args.shots}) + "
                               f"measure()", "qubits": args.qubits, "gates": len(ops), "shots": args.shots},
        "cpu_baseline": {"value": v, "unit": "gates/s", "cores": threads, "kind": kind, "sample": desc},
        "e2e": {"value": v, "unit": "gates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------- our arm
def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    os.environ.setdefault("OMP_PROC_BIND", "close")

    if args.impl == "reference":
        run_reference_arm(args, rank)
        return

    import numpy as np

    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist

    from quantumsimevo_b200 import _lib as L
    from quantumsimevo_b200 import workloads as W
    from quantumsimevo_b200.circuit import Circuit, Device, StateVector

    if args.playground:
        if rank == 0:
            print(json.dumps(bench_playground(Device(local), args.playground)))
        if dist:
            dist.destroy_process_group()
        return

    if args.batch_only:
        r = bench_batch(Device(local), L, W, np, steps=args.steps, warmup=args.warmup,
                        autotune=not args.no_autotune, count=args.batch_circuits, wmin=args.batch_wmin,
                        wmax=args.batch_wmax, dist=dist)
        if rank == 0:
            print(json.dumps(r))
        if dist:
            dist.destroy_process_group()
        return

    n = args.qubits
    ops = W.hrz_qft(n, seed=2)
    ngates = len(ops)
    dev = Device(local)
    if args.tile:
        dev.set_fusion(True, args.tile, 0)
    lib = L.lib
    st = StateVector(n, dev)
    d_out = C.c_void_p()
    cudart = None
    # device buffer for the sample outcomes (value arm: results stay in HBM)
    import torch
    out_t = torch.empty(args.shots, dtype=torch.int64, device=f"cuda:{local}")
    d_out = C.c_void_p(out_t.data_ptr())
    meas = L.C.c_uint64()

    def device_step(i):
        L.check(lib.qse_state_reset(st.handle))
        L.check(lib.qse_execute(st.handle, L.dptr(ops), ngates, None, 0, None, None, 0, None))
        L.check(lib.qse_sample_device(st.handle, None, args.shots, 1000 + i, d_out))
        L.check(lib.qse_measure(st.handle, 0.5, C.byref(meas)))

    def barrier():
        if dist:
            dist.barrier()

    def max_over_ranks(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    for i in range(args.warmup):
        device_step(i)
    dev.synchronize()

    # ---- timed: device-resident step ----
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    dev.synchronize()
    launches0 = dev.kernel_launches
    L.check(lib.qse_ctx_time_passes(dev.handle, 1))
    ptimes = (L.C.c_uint64(), L.C.c_double())
    L.check(lib.qse_ctx_pass_times(dev.handle, C.byref(ptimes[0]), C.byref(ptimes[1])))  # clear
    L.check(lib.qse_ctx_record(dev.handle, 0))
    for i in range(args.steps):
        device_step(args.warmup + i)
    L.check(lib.qse_ctx_record(dev.handle, 1))
    ms = C.c_float()
    L.check(lib.qse_ctx_elapsed(dev.handle, 0, 1, C.byref(ms)))
    dev.synchronize()
    barrier()
    clk = clocks.stop()
    launches = dev.kernel_launches - launches0
    plist = np.zeros(4096)
    pcount = C.c_size_t()
    L.check(lib.qse_ctx_pass_time_list(dev.handle, plist.ctypes.data_as(L._pd), plist.size, C.byref(pcount)))
    L.check(lib.qse_ctx_time_passes(dev.handle, 0))
    plist = plist[:min(int(pcount.value), plist.size)]
    pass_launches, pass_ms = len(plist), float(plist.sum())
    step_ms = max_over_ranks(ms.value / args.steps)
    value = world * ngates / (step_ms / 1e3)
    passes_per_exec = pass_launches / args.steps

    # phase breakdown of one step (device events on the library stream)
    phases = {}
    L.check(lib.qse_ctx_record(dev.handle, 4))
    L.check(lib.qse_state_reset(st.handle))
    L.check(lib.qse_execute(st.handle, L.dptr(ops), ngates, None, 0, None, None, 0, None))
    L.check(lib.qse_ctx_record(dev.handle, 5))
    L.check(lib.qse_sample_device(st.handle, None, args.shots, 77, d_out))
    L.check(lib.qse_ctx_record(dev.handle, 6))
    L.check(lib.qse_measure(st.handle, 0.5, C.byref(meas)))
    L.check(lib.qse_ctx_record(dev.handle, 7))
    for name, a, b in (("execute_ms", 4, 5), ("sample_ms", 5, 6), ("measure_ms", 6, 7)):
        L.check(lib.qse_ctx_elapsed(dev.handle, a, b, C.byref(ms)))
        phases[name] = ms.value

    # HBM roofline of the pass kernel.  Each step resets the state, so the first
    # pass of every execute starts from |0..0> generated in registers and only
    # writes (16 B per amplitude); the others read and write (32 B per
    # amplitude).  The roofline is taken on the read+write launches; the
    # execute's algorithmic bytes count both kinds.
    hbm_peak, peak_kind = peaks()
    bytes_per_pass = 32.0 * (1 << n)
    ppe = max(1, int(round(passes_per_exec)))
    idx = np.arange(len(plist))
    rw = plist[(idx % ppe) != 0] if ppe > 1 else plist
    zs = plist[(idx % ppe) == 0] if ppe > 1 else plist[:0]
    avg_pass_ms = float(rw.mean()) if rw.size else float(plist.mean())
    achieved = bytes_per_pass / (avg_pass_ms / 1e3) / 1e9
    exec_bytes = bytes_per_pass * passes_per_exec - (16.0 * (1 << n) if ppe > 1 else 0.0)
    # DRAM bytes per launch from the committed ncu summary (26-qubit capture
    # scaled by the amplitudes per launch), for the 30-qubit workload only
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "qse_pass_hrz_qft_26q.md")) as f:
            for line in f:
                if f"traffic_bytes_per_launch_{n}q:" in line:
                    traffic = float(line.split(":")[-1])
    except OSError:
        pass

    # ---- timed: end to end through the public API (host buffers) ----
    c = Circuit(n, device=dev, seed=7)
    for i in range(args.warmup):
        c.reset()
        c.add_ops(ops)
        c.execute()
        c.sample(args.shots)
        c.measure()
    barrier()
    dev.synchronize()
    L.check(lib.qse_ctx_record(dev.handle, 2))
    t0 = time.perf_counter()
    for i in range(args.steps):
        c.reset()
        c.add_ops(ops)
        c.execute()
        res = c.sample(args.shots)
        m = c.measure()
    L.check(lib.qse_ctx_record(dev.handle, 3))
    e2e_wall = (time.perf_counter() - t0) / args.steps
    L.check(lib.qse_ctx_elapsed(dev.handle, 2, 3, C.byref(ms)))
    e2e_ms = max_over_ranks(max(ms.value / args.steps, e2e_wall * 1e3))
    e2e_value = world * ngates / (e2e_ms / 1e3)
    del res, m, c

    # ---- reference CPU baseline (rank 0, N == 1) ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = int(os.environ.get("OMP_NUM_THREADS", "1"))
        r = cpu_reference_step(n, ops, args.shots, args.cpu_gates or 4, threads)
        if r is not None:
            v, w, desc, kind = r
            cpu = {"value": v, "unit": "gates/s", "cores": threads, "kind": kind, "sample": desc}

    # ---- QAOA gradients (rank 0) ----
    qaoa = None
    if rank == 0 and world == 1 and not args.no_qaoa:   # a single-GPU figure, reported at N = 1
        qaoa = bench_qaoa(dev, L, W, np)
    batch = None
    if not args.no_batch and (dist or rank == 0):
        # N ranks: the batch's circuits are split across the GPUs (no collective
        # on the data path; one gather of the results at the end)
        batch = bench_batch(dev, L, W, np, steps=args.steps, warmup=args.warmup, autotune=not args.no_autotune,
                            count=args.batch_circuits, wmin=args.batch_wmin, wmax=args.batch_wmax, dist=dist)

    barrier()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "gates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"H+RZ+QFT {n}q complex128 ({ngates} gates) + sample({args.shots}) + measure()",
                       "qubits": n, "gates": ngates, "shots": args.shots,
                       "parallelism": f"replicas{world}" if world > 1 else "single",
                       "l2": "state (16 GiB at 30 qubits) far larger than L2; no flush needed"},
            "passes_per_execute": passes_per_exec,
            "phases": phases,
            "execute_ms": pass_ms / args.steps,
            "hbm_gbs_execute": exec_bytes / (pass_ms / args.steps / 1e3) / 1e9,
            "zero_start_pass_ms": float(zs.mean()) if zs.size else None,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "qse_pass (fused pass, NVRTC-specialised)", "bytes_per_launch": bytes_per_pass,
                         "avg_launch_ms": avg_pass_ms,
                         "launches": "read+write passes (2nd and 3rd of each execute)"},
            "e2e": {"value": e2e_value, "unit": "gates/s", "h2d_bytes_per_step": int(ops.nbytes),
                    "d2h_bytes_per_step": int(8 * args.shots + 8)},
            "gpu_launches": int(launches),
            "clocks": clk,
            "cpu_baseline": cpu,
            "qaoa": qaoa,
            "batch": batch,
        }
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def bench_playground(dev, names):
    """The reference playground's workloads (GHZ, QFT, IQFT, Grover, QAOA Max-Cut) timed as
    its paper times them: wall clock from constructing the Circuit to the sampled indices
    on the host.  The first run includes compiling the pass kernels; "ms" is the best of
    the two runs after it."""
    from quantumsimevo_b200 import playground as P
    from quantumsimevo_b200.circuit import Circuit
    table = {w.name: w for w in P.workloads()}
    sel = list(table) if names == "all" else [x for x in names.split(",") if x]
    out = {}
    for name in sel:
        w = table[name]
        t0 = time.perf_counter()
        ops = w.build()
        build_ms = (time.perf_counter() - t0) * 1e3
        runs = []
        for rep in range(3):
            t0 = time.perf_counter()
            c = Circuit(w.qubits, device=dev, seed=rep)
            c.add_ops(ops)
            c.execute()
            c.sample(w.shots)
            runs.append((time.perf_counter() - t0) * 1e3)
            del c
        best = min(runs[1:])
        out[name] = {"qubits": w.qubits, "gates": int(len(ops)), "shots": w.shots, "ms": round(best, 3),
                     "ms_first_run": round(runs[0], 3), "op_list_build_ms": round(build_ms, 3),
                     "paper_ms": w.paper_ms, "paper_backend": w.paper_what,
                     "speedup_vs_paper": round(w.paper_ms / best, 1) if w.paper_ms else None}
    return {"metric": "playground wall clock: construct -> execute -> sample", "unit": "ms",
            "higher_is_better": False, "n_gpus": 1, "data": "the reference playground's circuits",
            "playground": out}


def bench_qaoa(dev, L, W, np):
    """24-qubit Max-Cut QAOA, p = 8: adjoint vs parameter-shift (plain kernels)."""
    from quantumsimevo_b200.circuit import StateVector
    n, p = 24, 8
    ops, params, edges, obs_t = W.qaoa_maxcut(n, p, seed=4)
    obs, keep = L.observable(*obs_t)
    st = StateVector(n, dev)
    pp = np.ascontiguousarray(params)
    g = np.zeros(pp.size)
    v = C.c_double()

    def adjoint():
        L.check(L.lib.qse_adjoint(st.handle, L.dptr(ops), len(ops), pp.ctypes.data_as(L._pd), pp.size,
                                  C.byref(obs), C.byref(v), g.ctypes.data_as(L._pd)))

    for _ in range(2):
        adjoint()
    reps = 5
    t0 = time.perf_counter()
    for _ in range(reps):
        adjoint()
    t_adj = (time.perf_counter() - t0) / reps
    g_adj = g.copy()

    # parameter shift: 2 executes per parameterised occurrence
    occ = [i for i in range(len(ops)) if int(ops[i]["param"]) >= 0]
    bound = ops.copy()
    for i in occ:
        bound[i]["theta"] = ops[i]["theta"] + ops[i]["coeff"] * pp[int(ops[i]["param"])]
        bound[i]["param"] = -1
        bound[i]["coeff"] = 1.0

    def f_at(arr):
        L.check(L.lib.qse_state_reset(st.handle))
        L.check(L.lib.qse_execute(st.handle, L.dptr(arr), len(arr), None, 0, None, None, 0, None))
        L.check(L.lib.qse_expectation(st.handle, C.byref(obs), C.byref(v)))
        return v.value

    # plain method: one kernel per gate
    dev.set_fusion(False)
    f_at(bound)
    t0 = time.perf_counter()
    for _ in range(3):
        f_at(bound)
    t_plain = (time.perf_counter() - t0) / 3
    dev.set_fusion(True, 12, 0)
    # full parameter-shift gradient on the fused path, for the accuracy check
    t0 = time.perf_counter()
    g_ps = np.zeros(pp.size)
    work = bound.copy()
    for i in occ:
        th = bound[i]["theta"]
        work[i]["theta"] = th + math.pi / 2
        fp = f_at(work)
        work[i]["theta"] = th - math.pi / 2
        fm = f_at(work)
        work[i]["theta"] = th
        g_ps[int(ops[i]["param"])] += ops[i]["coeff"] * (fp - fm) / 2
    t_ps_fused = time.perf_counter() - t0
    evals = 2 * len(occ)
    return {
        "workload": f"Max-Cut QAOA, random 3-regular graph, {n} qubits, p={p}, {pp.size} params, "
                    f"{len(ops)} gates, {len(occ)} parameterised occurrences",
        "adjoint_grads_per_s": 1.0 / t_adj,
        "param_shift_plain_grads_per_s": 1.0 / (evals * t_plain),
        "param_shift_fused_grads_per_s": 1.0 / t_ps_fused,
        "adjoint_vs_plain_param_shift": (evals * t_plain) / t_adj,
        "max_abs_grad_diff_vs_param_shift": float(np.max(np.abs(g_adj - g_ps))),
        "plain_execute_ms": t_plain * 1e3,
        "param_shift_evals_per_grad": evals,
        "timing": "host wall clock around synchronous C-ABI calls; plain param-shift extrapolated from 3 executes",
    }


def bench_batch(dev, L, W, np, steps=5, warmup=3, autotune=True, count=512, wmin=10, wmax=22, dist=None):
    """512 hardware-efficient-ansatz circuits (width U{10..22}, depth U{4..12}
    layers of RY+RZ per qubit and a CNOT ring, observable sum_i Z_i): forward
    <O> and the full adjoint gradient of every circuit per run, one persistent
    kernel replayed as a CUDA graph.  Baseline: the parameter-shift rule with
    one kernel per gate (2 executes per parameterised occurrence), timed on a
    width-stratified sample of the same circuits and summed over the batch.
    With dist (N ranks): each rank runs its balanced share of the circuits,
    timings are the slowest rank's, results are gathered once; rank 0 returns
    the report, the others None."""
    import torch

    from quantumsimevo_b200 import distributed as D
    from quantumsimevo_b200.batch import Batch
    from quantumsimevo_b200.circuit import StateVector
    hb = W.hea_batch(count, wmin, wmax, 4, 12, seed=5)
    circs = [(w, ops, len(p), obs) for (w, ops, p, obs) in hb]
    params = np.concatenate([p for (_, _, p, _) in hb])
    rank, world = (dist.get_rank(), dist.get_world_size()) if dist else (0, 1)
    idx = D.shard_for_rank(circs, rank, world) if dist else list(range(len(circs)))
    mine = [circs[i] for i in idx]
    my_params = D.local_params(circs, params, idx)
    local = dev.index
    t0 = time.perf_counter()
    b = Batch(mine, dev)
    cfg = None
    if autotune:
        cache = os.path.join(tempfile.gettempdir(), f"qse_batch_autotune_r{rank}.json")
        b.run(my_params)
        cfg = b.autotune(cache)
    t_setup = time.perf_counter() - t0
    p_t = torch.tensor(my_params, dtype=torch.float64, device=f"cuda:{local}")
    v_t = torch.zeros(len(mine), dtype=torch.float64, device=f"cuda:{local}")
    g_t = torch.zeros(max(1, my_params.size), dtype=torch.float64, device=f"cuda:{local}")
    torch.cuda.synchronize()
    for _ in range(warmup):
        b.run_device(p_t.data_ptr(), v_t.data_ptr(), g_t.data_ptr())
    dev.synchronize()
    if dist:
        dist.barrier()
    ms = C.c_float()
    L.check(L.lib.qse_ctx_record(dev.handle, 8))
    for _ in range(steps):
        b.run_device(p_t.data_ptr(), v_t.data_ptr(), g_t.data_ptr())
    L.check(L.lib.qse_ctx_record(dev.handle, 9))
    L.check(L.lib.qse_ctx_elapsed(dev.handle, 8, 9, C.byref(ms)))
    run_ms = ms.value / steps
    if dist:
        run_ms = D.max_over_ranks(run_ms, dist, device=f"cuda:{local}")
    st = b.stats()
    # end to end: host parameters in, host values + gradients out
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        vals, grads = b.run(my_params)
    e2e_ms = (time.perf_counter() - t0) / steps * 1e3
    if dist:
        e2e_ms = D.max_over_ranks(e2e_ms, dist, device=f"cuda:{local}")
        vals, grads = D.gather_results(circs, idx, vals, grads, dist)
        if rank != 0:
            return None

    # accuracy: the single-state adjoint path on a few circuits of the batch
    off = np.concatenate([[0], np.cumsum([c[2] for c in circs])])
    diffs = []
    for i in range(0, len(circs), max(1, len(circs) // 8)):
        w, ops, npar, obs_t = circs[i]
        obs, keep = L.observable(*obs_t)
        sv = StateVector(w, dev)
        pp = np.ascontiguousarray(params[off[i]:off[i + 1]])
        g = np.zeros(npar)
        v = C.c_double()
        L.check(L.lib.qse_adjoint(sv.handle, L.dptr(ops), len(ops), pp.ctypes.data_as(L._pd), npar, C.byref(obs),
                                  C.byref(v), g.ctypes.data_as(L._pd)))
        diffs.append(max(abs(v.value - vals[i]), float(np.max(np.abs(g - grads[off[i]:off[i + 1]])))))
        del sv

    # plain-kernel parameter shift: per width, one circuit's execute + <O>, scaled by depth
    dev.set_fusion(False)
    per_width = {}
    v = C.c_double()
    for i, (w, ops, npar, obs_t) in enumerate(circs):
        if w in per_width:
            continue
        obs, keep = L.observable(*obs_t)
        sv = StateVector(w, dev)
        bound = ops.copy()
        pp = params[off[i]:off[i + 1]]
        for j in range(len(bound)):
            if int(bound[j]["param"]) >= 0:
                bound[j]["theta"] = bound[j]["theta"] + bound[j]["coeff"] * pp[int(bound[j]["param"])]
                bound[j]["param"] = -1

        def f_at():
            L.check(L.lib.qse_state_reset(sv.handle))
            L.check(L.lib.qse_execute(sv.handle, L.dptr(bound), len(bound), None, 0, None, None, 0, None))
            L.check(L.lib.qse_expectation(sv.handle, C.byref(obs), C.byref(v)))

        f_at()
        t0 = time.perf_counter()
        for _ in range(3):
            f_at()
        per_width[w] = ((time.perf_counter() - t0) / 3, len(ops))
        del sv
    dev.set_fusion(True, 12, 0)
    ps_total = 0.0
    occ_total = 0
    for (w, ops, npar, obs_t) in circs:
        t, g0 = per_width[w]
        occ = int(np.sum(ops["param"] >= 0))
        occ_total += occ
        ps_total += 2 * occ * t * len(ops) / g0
    hbm_peak, peak_kind = peaks()
    hbm_gbs = st["hbm_bytes"] / (run_ms / 1e3) / 1e9
    return {
        "workload": f"{count} HEA circuits, width U{{{wmin}..{wmax}}}, depth U{{4..12}} (RY+RZ per qubit + CNOT ring), "
                    f"sum_i Z_i; {params.size} parameters, {occ_total} parameterised occurrences",
        "circuits_per_s": len(circs) / (run_ms / 1e3),
        "gradient_entries_per_s": params.size / (run_ms / 1e3),
        "run_ms": run_ms,
        "e2e_ms": e2e_ms,
        "e2e_circuits_per_s": len(circs) / (e2e_ms / 1e3),
        "param_shift_plain_ms_est": ps_total * 1e3,
        "adjoint_batch_vs_plain_param_shift": ps_total / (run_ms / 1e3),
        "max_abs_diff_vs_single_state_adjoint": max(diffs),
        "config": None if cfg is None else cfg.__dict__,
        "stats": {k: st[k] for k in ("passes", "items", "tile_visits", "hbm_bytes", "grid", "smem_bytes", "plan_ms")},
        "hbm_gbs_multi_tile": hbm_gbs,
        "hbm_frac_multi_tile": hbm_gbs / hbm_peak,
        "setup_s": t_setup,
        "ranks": world,
        "rank0_circuits": len(mine),
        "timing": "device: CUDA events on the library stream around `steps` graph replays (device params); "
                  "e2e: host wall clock of qse_batch_run (params H2D, values+grads D2H); plain param-shift: "
                  "host wall clock of plain-kernel execute+<O> per width, scaled by depth and occurrences",
    }


if __name__ == "__main__":
    main()
