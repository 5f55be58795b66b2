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
cpu_baseline
           the reference's own AVX2/OpenMP backend (compiled from its sources
           into oracle/_ref) on the host cores: a stratified sample of the
           circuit (one gate per gate kind x qubit class) timed and charged to
           every gate of its class, plus the full sample(1e6) and measure().
--impl reference
           the same reference code for the whole workload with no
           extrapolation: the K timed steps apply the 540 gates once, in
           order, and the last one also samples and measures.  This arm maps
           no library of this project.
qaoa       adjoint gradients/s (24-qubit 3-regular Max-Cut, p=8, 16 params)
           vs the parameter-shift rule on the reference's own CUDA kernels
           (CircuitUnitaryOperationGPU rebuilt for sm_100a), every execute of
           one parameter's entry timed on the device and checked against the
           adjoint.
adjoint_30q
           the adjoint at 30 qubits (two 16 GiB states): gradients/s and the
           HBM fraction of its reverse passes (64 B per amplitude).
gates_30q  every apply* through this project's drop-in adapter against the
           reference's CUDA kernels on the same GPU, at low/middle/high qubits.
batch      512 parameterised circuits (widths 10..22): forward <O> and the full
           adjoint gradient of each, one persistent kernel per run replayed as
           a CUDA graph, against parameter shift on the reference's CUDA
           kernels.  --batch-only runs just this section (--batch-circuits/
           -wmin/-wmax set a smaller case, --no-autotune keeps the default
           configuration).
Multi-GPU: the step's state does not shard; every rank runs its own replica
(weak scaling), value = sum over ranks.  --sharded QUBITS instead runs one
state of QUBITS qubits sharded over the N ranks (strong scaling, execute only,
NCCL half-shard exchanges) and prints that line.
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
L2_BYTES = 126 * 1000 * 1000
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
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="skip the baselines on the reference's CUDA kernels (gradients, per-gate section)")
    ap.add_argument("--no-gates", action="store_true", help="skip the per-gate drop-in comparison")
    ap.add_argument("--no-adjoint30", action="store_true", help="skip the 30-qubit adjoint section")
    ap.add_argument("--tile", type=int, default=0, help="tile qubits of the fused passes (0 = library default)")
    ap.add_argument("--pass-kernel", type=int, default=-1, choices=[-1, 0, 1, 2],
                    help="pass kernels (qse_ctx_set_jit): 0 interpreter, 1 one CTA per tile, 2 streamed; "
                         "-1 = library default")
    ap.add_argument("--adjoint", type=int, default=0, metavar="QUBITS",
                    help="instead of the step: only the adjoint section (Max-Cut QAOA, p = 2) at QUBITS qubits")
    ap.add_argument("--sharded", type=int, default=0, metavar="QUBITS",
                    help="instead of the step: one H+RZ+QFT state of QUBITS qubits sharded over the N ranks "
                         "(2^g = N, the top g qubits global; NCCL half-shard exchanges), execute only")
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
    """nvidia-smi clocks and throttle reasons sampled every 100 ms.  start()
    returns once the first sample is written, so that sampling runs through the
    whole timed region; stop() reads the samples written after start() returned
    (the last earlier one when the region was shorter than the interval)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.offset = 0
        self.path = os.path.join(tempfile.gettempdir(), f"qse_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        t0 = time.time()
        while os.path.getsize(self.path) == 0 and time.time() - t0 < 5.0 and self.proc.poll() is None:
            time.sleep(0.01)
        self.offset = os.path.getsize(self.path)

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
            text = f.read()
        lines = text[self.offset:].splitlines()
        in_region = len(lines)
        if not lines:
            lines = text[:self.offset].splitlines()[-1:]
        for line in lines:
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
                "samples": len(sm), "samples_in_region": in_region}


# ---------------------------------------------------------------- reference code (oracle/_ref)
# Everything in this section drives the reference's own sources compiled into
# oracle/_ref (libqse_ref_cpu.so: AVX2/OpenMP backend; libqse_ref_gpu.so: its
# CUDA backend rebuilt for sm_100a) as baselines.  None of it is in a timed
# region of this project's arm.

def _oracle_ffi():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_ffi as O
    return O


def _chunks(nitems, k):
    """k contiguous index ranges covering range(nitems), sizes differing by at most one."""
    b = [nitems * s // k for s in range(k + 1)]
    return [(b[s], b[s + 1]) for s in range(k)]


def _qclass(q, n):
    """Qubit classes of the stratified sample: qubit 0 (the AVX2 backend special-cases it),
    then the low, middle and high thirds of the qubit range."""
    if q == 0:
        return "q0"
    return ("low", "mid", "high")[min(2, 3 * q // n)]


def _gate_key(op, n):
    t = int(op["type"])
    if t in (9, 10, 12):   # CNOT, CPHASE, SWAP: both qubits matter for the access pattern
        return (t, _qclass(int(op["target"]), n), _qclass(int(op["control"]), n))
    return (t, _qclass(int(op["target"]), n))


def cpu_reference_estimate(n, ops, shots, threads):
    """cpu_baseline leg: the reference's AVX2 backend (CircuitUnitaryOperationAVX
    behind ICircuitUnitaryOperation, as Circuit::execute calls it) on a stratified
    sample of the circuit -- one gate of every (gate kind, qubit class) the circuit
    contains, qubit classes = qubit 0 and the low / middle / high thirds (both
    qubits for two-qubit gates) -- each timed once; every gate of the circuit is
    charged the time of its class's sample.  StateVector::sample(shots) and
    StateVector::measure() are timed in full.  Returns (gates/s, description)."""
    import numpy as np
    O = _oracle_ffi()
    ref = O.load_reference(gpu=False)
    if ref is None:
        return None
    ref.ref_set_quiet(1)
    be = ref.ref_backend_new(1)
    sv = ref.ref_statevector_new(n)
    try:
        reps = {}
        for i in range(len(ops)):
            reps.setdefault(_gate_key(ops[i], n), i)
        per_key = {}
        for key, i in reps.items():
            one = np.ascontiguousarray(ops[i:i + 1])
            t0 = time.perf_counter()
            assert ref.ref_backend_apply(be, sv, one.ctypes.data_as(C.c_void_p), 1) == 0
            per_key[key] = time.perf_counter() - t0
        t_gates = sum(per_key[_gate_key(ops[i], n)] for i in range(len(ops)))
        out = np.empty(shots, dtype=np.uint64)
        t0 = time.perf_counter()
        ref.ref_statevector_sample(sv, shots, out.ctypes.data_as(C.POINTER(C.c_uint64)))
        t_sample = time.perf_counter() - t0
        t0 = time.perf_counter()
        ref.ref_statevector_measure(sv)
        t_measure = time.perf_counter() - t0
    finally:
        ref.ref_statevector_free(sv)
        ref.ref_backend_free(be)
    step = t_gates + t_sample + t_measure
    desc = (f"reference CircuitUnitaryOperationAVX, OMP_NUM_THREADS={threads}, {n} qubits: {len(per_key)} sampled "
            f"gates (one per gate kind x qubit class: qubit 0 / low / middle / high third), {sum(per_key.values()):.2f} s, "
            f"each circuit gate charged its class's time -> {t_gates:.1f} s for {len(ops)} gates; StateVector::sample("
            f"{shots}) {t_sample:.2f} s and measure() {t_measure:.2f} s timed in full")
    return len(ops) / step, desc


def run_reference_arm(args, rank):
    """--impl reference: the reference's own AVX2/OpenMP code on the host cores for
    the whole workload, no extrapolation.  The K timed steps together apply the
    540 gates once, in order (step s applies the s-th contiguous share through
    ICircuitUnitaryOperation on CircuitUnitaryOperationAVX, as Circuit::execute
    does), and the last step also runs StateVector::sample(shots) and
    StateVector::measure() on the final state.  value = gates / total time, so it
    is the gates/s of one full step of this project's arm.  Warm-up: the first W
    shares on the same state, which is then reset to |0..0>.  Rank 0 only."""
    if rank != 0:
        return
    import numpy as np
    from quantumsimevo_b200 import workloads as W   # plain data: libqse_b200.so is not mapped
    O = _oracle_ffi()
    ref = O.load_reference(gpu=False)
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libqse_ref_cpu.so not built"}))
        return
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    n = args.qubits
    ops = W.hrz_qft(n, seed=2)
    ref.ref_set_quiet(1)
    be = ref.ref_backend_new(1)
    sv = ref.ref_statevector_new(n)
    parts = _chunks(len(ops), args.steps)
    out = np.empty(args.shots, dtype=np.uint64)

    def apply(lo, hi):
        if hi > lo:
            a = np.ascontiguousarray(ops[lo:hi])
            assert ref.ref_backend_apply(be, sv, a.ctypes.data_as(C.c_void_p), hi - lo) == 0

    for i in range(args.warmup):
        apply(*parts[i % len(parts)])
    ref.ref_statevector_reset(sv)
    times = []
    for s, (lo, hi) in enumerate(parts):
        t0 = time.perf_counter()
        apply(lo, hi)
        if s == len(parts) - 1:
            ref.ref_statevector_sample(sv, args.shots, out.ctypes.data_as(C.POINTER(C.c_uint64)))
            ref.ref_statevector_measure(sv)
        times.append(time.perf_counter() - t0)
    ref.ref_statevector_free(sv)
    ref.ref_backend_free(be)
    total = sum(times)
    v = len(ops) / total
    sample = (f"reference CircuitUnitaryOperationAVX + StateVector, OMP_NUM_THREADS={threads}: the full {len(ops)}-gate "
              f"circuit applied once across the {args.steps} timed steps ({len(ops) // args.steps}-"
              f"{-(-len(ops) // args.steps)} gates each, in order), sample({args.shots}) + measure() in the last step; "
              f"{total:.1f} s in all")
    line = {
        "metric": METRIC, "value": v, "unit": "gates/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(n, len(ops), args.shots),
        "cpu_baseline": {"value": v, "unit": "gates/s", "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": "gates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "step_seconds": [round(t, 3) for t in times],
    }
    print(json.dumps(line))


class RefGpu:
    """The reference's CUDA backend (CircuitUnitaryOperationGPU.cu, one kernel per
    gate on its private stream) rebuilt for sm_100a, on a reference StateVector:
    the "plain GPU kernels" of the gradient baselines."""

    def __init__(self, n):
        O = _oracle_ffi()
        self.ref = O.load_reference(gpu=True)
        if self.ref is None:
            raise RuntimeError("oracle/_ref/libqse_ref_gpu.so not built")
        self.ref.ref_set_quiet(1)
        self.n = n
        self.be = self.ref.ref_backend_new(2)
        self.sv = self.ref.ref_statevector_new(n)
        self._ident = None

    def run(self, ops):
        """|0..0>, then ops on the device.  Returns the device time of the ops'
        kernels (host clock between two device synchronisations).  The state's
        upload (the backend's ensureOnDevice after reset) happens before the
        timed part, triggered by an identity pair Z(0) Z(0)."""
        import numpy as np
        from quantumsimevo_b200 import workloads as W
        if self._ident is None:
            self._ident = W.to_array([W._op(3, 0), W._op(3, 0)])
        r = self.ref
        r.ref_statevector_reset(self.sv)
        r.ref_backend_mark_host_dirty(self.be)
        assert r.ref_backend_apply(self.be, self.sv, self._ident.ctypes.data_as(C.c_void_p), 2) == 0
        assert r.ref_device_synchronize() == 0
        a = np.ascontiguousarray(ops)
        t0 = time.perf_counter()
        assert r.ref_backend_apply(self.be, self.sv, a.ctypes.data_as(C.c_void_p), len(a)) == 0
        assert r.ref_device_synchronize() == 0
        return time.perf_counter() - t0

    def probabilities(self):
        import numpy as np
        self.ref.ref_backend_flush(self.be)
        st = np.empty(1 << self.n, dtype=np.complex128)
        self.ref.ref_statevector_get(self.sv, st.ctypes.data_as(C.c_void_p))
        return st.real * st.real + st.imag * st.imag

    def close(self):
        self.ref.ref_statevector_free(self.sv)
        self.ref.ref_backend_free(self.be)


def observable_vector(n, zmasks, weights, constant):
    """O(x) for every basis index x (host, for the baselines' own expectation values)."""
    import numpy as np
    x = np.arange(1 << n, dtype=np.uint64)
    o = np.full(1 << n, float(constant))
    for z, w in zip(zmasks, weights):
        par = np.zeros(1 << n, dtype=np.uint8)
        m = int(z)
        while m:
            b = (m & -m).bit_length() - 1
            par ^= ((x >> np.uint64(b)) & np.uint64(1)).astype(np.uint8)
            m &= m - 1
        o += np.where(par == 1, -float(w), float(w))
    return o


def bind(ops, params):
    """ops with every parameterised angle bound (theta + coeff * params[param])."""
    b = ops.copy()
    for i in range(len(b)):
        if int(b[i]["param"]) >= 0:
            b[i]["theta"] = b[i]["theta"] + b[i]["coeff"] * params[int(b[i]["param"])]
            b[i]["param"] = -1
            b[i]["coeff"] = 1.0
    return b


def plain_param_shift_entries(gpu, ops, params, obs_vec, pick):
    """Gradient entries `pick` by the parameter-shift rule, every occurrence of each
    picked parameter evaluated with the reference's CUDA kernels (2 executes per
    occurrence; <O> from the state on the host, untimed).  Returns
    ({param: value}, kernel seconds per execute, executes timed)."""
    import numpy as np
    bound = bind(ops, params)
    work = bound.copy()
    out, t, evals = {}, 0.0, 0
    for p in pick:
        acc = 0.0
        for i in np.nonzero(ops["param"] == p)[0]:
            th = bound[i]["theta"]
            f = []
            for sgn in (1.0, -1.0):
                work[i]["theta"] = th + sgn * math.pi / 2
                t += gpu.run(work)
                evals += 1
                f.append(float(np.dot(gpu.probabilities(), obs_vec)))
            work[i]["theta"] = th
            acc += ops[i]["coeff"] * (f[0] - f[1]) / 2
        out[p] = acc
    return out, t / max(1, evals), evals


def device_expectation_ms(dev, L, n, obs, reps=5):
    """Device time of one <O> evaluation (qse_expectation) on an n-qubit state: the
    cost added to every plain execute of the parameter-shift baselines."""
    from quantumsimevo_b200.circuit import StateVector
    st = StateVector(n, dev)
    v = C.c_double()
    L.check(L.lib.qse_expectation(st.handle, C.byref(obs), C.byref(v)))
    dev.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        L.check(L.lib.qse_expectation(st.handle, C.byref(obs), C.byref(v)))
    dev.synchronize()
    return (time.perf_counter() - t0) / reps * 1e3


# ---------------------------------------------------------------- our arm
def workload_config(n, ngates, shots):
    """The `config` of both arms (identical keys and values)."""
    state = 16 << n
    if state > L2_BYTES:
        l2 = (f"state ({state / 2**30:g} GiB at {n} qubits) larger than the 126 MB L2: every pass streams it "
              f"from HBM, no flush needed")
    else:
        l2 = f"state ({state / 2**20:g} MiB at {n} qubits) fits in L2: a small-case run, not the benchmark"
    return {"workload": f"H+RZ+QFT {n}q complex128 ({ngates} gates) + sample({shots}) + measure()",
            "qubits": n, "gates": ngates, "shots": shots, "l2": l2}


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

    if args.adjoint:
        if rank == 0:
            print(json.dumps(bench_adjoint_30q(Device(local), L, W, np, n=args.adjoint)))
        if dist:
            dist.destroy_process_group()
        return

    if args.sharded:
        r = bench_sharded(args, dist, rank, world, local, L, W, np)
        if rank == 0:
            print(json.dumps(r))
        if dist:
            dist.destroy_process_group()
        return

    if args.batch_only:
        r = bench_batch(Device(local), L, W, np, steps=args.steps, warmup=args.warmup,
                        autotune=not args.no_autotune, count=args.batch_circuits, wmin=args.batch_wmin,
                        wmax=args.batch_wmax, dist=dist, plain=not args.no_ref_gpu)
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
    if args.pass_kernel >= 0:
        L.check(L.lib.qse_ctx_set_jit(dev.handle, args.pass_kernel))
    lib = L.lib
    st = StateVector(n, dev)
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
    # the exact scan's path statistics on the executed state (untimed)
    L.check(lib.qse_state_reset(st.handle))
    L.check(lib.qse_execute(st.handle, L.dptr(ops), ngates, None, 0, None, None, 0, None))
    sst = (C.c_uint32 * 4)()
    L.check(lib.qse_sampler_stats(st.handle, sst))
    phases["sampler_scan"] = {"spans": int(sst[0]), "single_blocks": int(sst[1]), "exact_blocks": int(sst[2]),
                              "blocks": int(sst[3])}

    # HBM roofline of the pass kernel.  Each step resets the state, so the first
    # pass of every execute starts from |0..0> generated in registers and only
    # writes (16 B per amplitude); the others read and write (32 B per
    # amplitude).  The roofline is taken on the read+write launches; the
    # execute's algorithmic bytes count both kinds.
    # The pass timings list the passes over the full state only (passes that
    # run on a compact state of the first touched qubits are not timed).  Every
    # step resets, so the first full-state pass of an execute reads no full
    # state: it generates its input (from |0..0>, or from the compact state of
    # at most 2^22 amplitudes, under 0.5 % of its bytes at 30 qubits) and writes
    # 16 B per amplitude; any later one reads and writes 32 B per amplitude.
    hbm_peak, peak_kind = peaks()
    ppe = max(1, int(round(passes_per_exec)))
    idx = np.arange(len(plist))
    rw = plist[(idx % ppe) != 0]
    zs = plist[(idx % ppe) == 0]
    if rw.size:
        bytes_per_pass, avg_pass_ms = 32.0 * (1 << n), float(rw.mean())
        kernel = "qse_pass"
        launches_desc = "read+write full-state passes (all but the first of each execute)"
    else:
        # the steps sample, so the pass also writes each probability (8 B per
        # amplitude) for the next sample
        bytes_per_pass, avg_pass_ms = 24.0 * (1 << n), float(zs.mean())
        kernel = "qse_pass_compact_in"
        launches_desc = ("the one full-state pass of each execute (input generated from the compact state of the "
                         "leading passes; writes 16 B per amplitude and 8 B per probability for the sampler)")
    achieved = bytes_per_pass / (avg_pass_ms / 1e3) / 1e9
    exec_bytes = 24.0 * (1 << n) + 32.0 * (1 << n) * (ppe - 1)
    # DRAM bytes per launch from the committed ncu summary (26-qubit capture
    # scaled by the amplitudes per launch), for the 30-qubit workload only
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", f"{kernel}_hrz_qft_26q.md")) as f:
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
    del st, out_t
    torch.cuda.empty_cache()

    single = rank == 0 and world == 1   # single-GPU figures, reported at N = 1
    # ---- reference CPU baseline (rank 0, N == 1) ----
    cpu = None
    if single and not args.no_cpu_baseline:
        threads = int(os.environ.get("OMP_NUM_THREADS", "1"))
        r = cpu_reference_estimate(n, ops, args.shots, threads)
        if r is not None:
            cpu = {"value": r[0], "unit": "gates/s", "cores": threads, "kind": "reference", "sample": r[1]}

    # ---- gradients and the per-gate drop-in comparison (rank 0, N == 1) ----
    qaoa = bench_qaoa(dev, L, W, np, plain=not args.no_ref_gpu) if single and not args.no_qaoa else None
    adjoint30 = bench_adjoint_30q(dev, L, W, np) if single and not args.no_adjoint30 and n >= 30 else None
    gates = bench_gates(dev, L, W, np, n) if single and not args.no_gates and not args.no_ref_gpu else None
    batch = None
    if not args.no_batch and (dist or rank == 0):
        # N ranks: the batch's circuits are split across the GPUs (no collective
        # on the data path; one gather of the results at the end)
        batch = bench_batch(dev, L, W, np, steps=args.steps, warmup=args.warmup, autotune=not args.no_autotune,
                            count=args.batch_circuits, wmin=args.batch_wmin, wmax=args.batch_wmax, dist=dist,
                            plain=not args.no_ref_gpu and single)

    barrier()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "gates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(n, ngates, args.shots),
            "parallelism": f"replicas{world}" if world > 1 else "single",
            "passes_per_execute": passes_per_exec,
            "passes_per_execute_meaning": "passes over the full state (leading passes on a compact state not counted)",
            "phases": phases,
            "execute_ms": pass_ms / args.steps,
            "execute_ms_meaning": "device time of the full-state passes of one execute (phases.execute_ms: the whole "
                                  "execute)",
            "hbm_gbs_execute": exec_bytes / (pass_ms / args.steps / 1e3) / 1e9,
            "first_pass_ms": float(zs.mean()) if zs.size else None,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": f"{kernel} (fused pass, NVRTC-specialised)", "bytes_per_launch": bytes_per_pass,
                         "avg_launch_ms": avg_pass_ms,
                         "launches": launches_desc},
            "e2e": {"value": e2e_value, "unit": "gates/s", "h2d_bytes_per_step": int(ops.nbytes),
                    "d2h_bytes_per_step": int(8 * args.shots + 8)},
            "gpu_launches": int(launches),
            "clocks": clk,
            "cpu_baseline": cpu,
            "qaoa": qaoa,
            "adjoint_30q": adjoint30,
            "gates_30q": gates,
            "batch": batch,
        }
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def bench_sharded(args, dist, rank, world, local, L, W, np):
    """One n-qubit H+RZ+QFT state over the N ranks (quantumsimevo_b200.sharded):
    each step resets the shards and executes the 540-gate circuit (at 30
    qubits; 18n gates in general), local segments as fused passes on each
    rank's engine, global-qubit gates through pipelined half-shard exchanges
    with the partner rank.  Total work is fixed as N grows (strong scaling).
    Timed from a barrier to a barrier with the host clock (the exchanges
    synchronise the host with both the engine stream and NCCL), max over ranks."""
    import torch

    from quantumsimevo_b200 import sharded as S
    from quantumsimevo_b200.circuit import Device
    n = args.sharded
    g = world.bit_length() - 1
    if (1 << g) != world or n - g < 12:
        raise SystemExit("--sharded needs a power-of-two rank count and at least 12 local qubits")
    ops = W.hrz_qft(n, seed=2)
    dev = Device(local)
    shard = S.DeviceShard(n - g, rank, dev)
    stats = {}

    def step(st):
        shard.reset()
        S.execute_rank(ops, n, g, rank, shard, dist, stats=st)

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize(local)

    for _ in range(args.warmup):
        step(None)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step(stats)
    barrier()
    sec = (time.perf_counter() - t0) / args.steps
    if dist:
        t = torch.tensor([sec, stats.get("exchange_s", 0.0) / args.steps], dtype=torch.float64,
                         device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        sec, exch = float(t[0]), float(t[1])
    else:
        exch = stats.get("exchange_s", 0.0) / args.steps
    nex = stats.get("exchanges", 0) / args.steps
    xbytes = stats.get("exchange_bytes", 0) / args.steps
    del shard
    return {
        "metric": f"sharded {n}q H+RZ+QFT execute gates/s", "value": len(ops) / sec, "unit": "gates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"H+RZ+QFT {n}q complex128 ({len(ops)} gates), one state over {world} ranks",
                   "qubits": n, "gates": len(ops), "global_qubits": g,
                   "l2": f"shard ({16 << (n - g) >> 20} MiB per rank) streamed from HBM by every pass"},
        "parallelism": f"sharded{world}",
        "exchanges_per_execute": nex,
        "exchange_ms": exch * 1e3,
        "exchange_bytes_sent_per_rank": xbytes,
        "exchange_gbs_per_rank": (xbytes / exch / 1e9) if exch > 0 else None,
        "nvlink_peer_copy_gbs": 770.0,
        "timing": "host clock between barriers (every exchange synchronises the host with the engine stream "
                  "and NCCL), max over ranks; exchange_ms: host time inside the exchanges",
    }


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


def bench_qaoa(dev, L, W, np, plain=True):
    """24-qubit Max-Cut QAOA, p = 8 (16 parameters, 1080 gates): adjoint gradients/s
    against the parameter-shift rule with the plain per-gate GPU kernels -- the
    reference's own CircuitUnitaryOperationGPU kernels rebuilt for sm_100a.  The
    plain baseline is run in full for a sample: every occurrence of parameter
    beta_0 (24 RX gates, 48 executes), each execute timed on the device, plus one
    device <O> evaluation per execute; a full gradient is 2 executes per
    parameterised occurrence (2112).  The sampled entry is checked against the
    adjoint's."""
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
    occ = int(np.sum(ops["param"] >= 0))
    evals = 2 * occ
    out = {
        "workload": f"Max-Cut QAOA, random 3-regular graph, {n} qubits, p={p}, {pp.size} params, "
                    f"{len(ops)} gates, {occ} parameterised occurrences",
        "adjoint_grads_per_s": 1.0 / t_adj,
        "adjoint_ms": t_adj * 1e3,
        "param_shift_evals_per_grad": evals,
    }
    if not plain:
        return out
    del st
    obs_ms = device_expectation_ms(dev, L, n, obs)
    gpu = RefGpu(n)
    try:
        ovec = observable_vector(n, *obs_t)
        beta0 = p   # params[p + l] = beta_l
        entries, exec_s, timed = plain_param_shift_entries(gpu, ops, params, ovec, [beta0])
    finally:
        gpu.close()
    eval_s = exec_s + obs_ms / 1e3
    out.update({
        "param_shift_plain_grads_per_s": 1.0 / (evals * eval_s),
        "adjoint_vs_plain_param_shift": (evals * eval_s) / t_adj,
        "plain_execute_ms": exec_s * 1e3,
        "plain_expectation_ms": obs_ms,
        "plain_executes_timed": timed,
        "sampled_entry": {"param": f"beta_0 (index {beta0})", "plain_param_shift": entries[beta0],
                          "adjoint": float(g_adj[beta0]), "abs_diff": abs(entries[beta0] - float(g_adj[beta0]))},
        "timing": "adjoint: host wall clock around synchronous qse_adjoint (5 runs); plain: the reference's "
                  "CircuitUnitaryOperationGPU kernels (sm_100a), device time of each full execute (host clock "
                  "between device synchronisations, state upload excluded), every execute of the sampled "
                  "parameter, plus one qse_expectation per execute",
    })
    return out


def bench_adjoint_30q(dev, L, W, np, n=30):
    """Adjoint at n qubits (30 by default: two 16 GiB states on one GPU): Max-Cut QAOA
    on a random 3-regular graph with n nodes, p = 2 (4 parameters).  Reports
    gradients/s, the device time of every pass (forward, then reverse) and the HBM
    fraction of the reverse passes (64 B per amplitude: psi and lambda read and
    written, the <lambda|dG|psi> reductions fused)."""
    import torch
    from quantumsimevo_b200.circuit import StateVector
    if torch.cuda.mem_get_info(dev.index)[0] < 40 * (1 << n):   # two states of 16 B per amplitude, and slack
        return {"skipped": "not enough free device memory for two states"}
    p = 2
    ops, params, edges, obs_t = W.qaoa_maxcut(n, p, seed=30)
    obs, keep = L.observable(*obs_t)
    st = StateVector(n, dev)
    pp = np.ascontiguousarray(params)
    g = np.zeros(pp.size)
    v = C.c_double()
    # timed forward passes of the same execute (passes on a compact state are not timed)
    L.check(L.lib.qse_ctx_time_passes(dev.handle, 1))
    fl = np.zeros(256)
    fc = C.c_size_t()
    L.check(L.lib.qse_ctx_pass_time_list(dev.handle, fl.ctypes.data_as(L._pd), fl.size, C.byref(fc)))
    L.check(L.lib.qse_execute(st.handle, L.dptr(ops), len(ops), pp.ctypes.data_as(L._pd), pp.size, None, None, 0,
                              None))
    dev.synchronize()
    L.check(L.lib.qse_ctx_pass_time_list(dev.handle, fl.ctypes.data_as(L._pd), fl.size, C.byref(fc)))
    L.check(L.lib.qse_ctx_time_passes(dev.handle, 0))
    fwd = int(fc.value)

    def adjoint():
        L.check(L.lib.qse_adjoint(st.handle, L.dptr(ops), len(ops), pp.ctypes.data_as(L._pd), pp.size,
                                  C.byref(obs), C.byref(v), g.ctypes.data_as(L._pd)))

    adjoint()
    dev.synchronize()
    L.check(L.lib.qse_ctx_time_passes(dev.handle, 1))
    L.check(L.lib.qse_ctx_record(dev.handle, 10))
    adjoint()
    L.check(L.lib.qse_ctx_record(dev.handle, 11))
    ms = C.c_float()
    L.check(L.lib.qse_ctx_elapsed(dev.handle, 10, 11, C.byref(ms)))
    plist = np.zeros(1024)
    cnt = C.c_size_t()
    L.check(L.lib.qse_ctx_pass_time_list(dev.handle, plist.ctypes.data_as(L._pd), plist.size, C.byref(cnt)))
    L.check(L.lib.qse_ctx_time_passes(dev.handle, 0))
    plist = plist[:int(cnt.value)]
    rev = plist[fwd:]
    hbm_peak, peak_kind = peaks()
    rev_gbs = 64.0 * (1 << n) / (rev.mean() / 1e3) / 1e9 if rev.size else None
    return {
        "workload": f"Max-Cut QAOA, random 3-regular graph, {n} qubits, p={p}, {pp.size} params, {len(ops)} gates",
        "grads_per_s": 1e3 / ms.value,
        "adjoint_ms": ms.value,
        "forward_passes": fwd,
        "reverse_passes": int(rev.size),
        "reverse_pass_ms": float(rev.mean()) if rev.size else None,
        "reverse_pass_gbs": rev_gbs,
        "reverse_pass_hbm_frac": rev_gbs / hbm_peak if rev_gbs else None,
        "pass_ms": [round(float(x), 4) for x in plist],
        "peak_kind": peak_kind,
        "value": v.value,
        "timing": "CUDA events on the library stream around one qse_adjoint; pass times from per-launch events",
    }


GATE_NAMES_BENCH = {4: "H", 1: "X", 2: "Y", 3: "Z", 5: "PHASE", 6: "RX", 7: "RY", 8: "RZ", 9: "CNOT",
                    10: "CPHASE", 11: "MCPHASE", 12: "SWAP", 15: "GATE2X2"}


def bench_gates(dev, L, W, np, n, reps=4):
    """Per-gate drop-in comparison at n qubits: every ICircuitUnitaryOperation::apply*
    through this project's adapter (CircuitUnitaryOperationB200, one kernel per gate
    over the C ABI) against the reference's CircuitUnitaryOperationGPU kernels
    rebuilt for sm_100a, on the same B200, at low, middle and high qubits.  Device
    time per gate (host clock between device synchronisations, `reps` gates)."""
    O = _oracle_ffi()
    ref = O.load_reference(gpu=True)
    if ref is None:
        return {"skipped": "oracle/_ref/libqse_ref_gpu.so not built"}
    ref.ref_set_quiet(1)
    rng = W.SplitMix64(77)
    cases = []
    for q in (0, 3, 5, n // 2, n - 1):
        q2 = n - 2 if q >= n - 2 else n - 1
        for t in (4, 1, 2, 3, 5, 6, 7, 8, 9, 10, 11, 12, 15):
            theta = rng.uniform() * 6.283185307179586
            m = W.gate2x2_unitary(rng) if t == 15 else (0.0,) * 8
            ctl = (1 << (q2 - 1)) | (1 << q2) if t == 11 else 0
            cases.append((GATE_NAMES_BENCH[t], q, W.to_array([(t, q, q2, -1, ctl, theta, 1.0, m)] * reps)))
    res = {}
    for backend, name in ((2, "reference_cuda"), (3, "adapter")):
        be = ref.ref_backend_new(backend)
        sv = ref.ref_statevector_new(n)
        try:
            warm = cases[0][2]
            assert ref.ref_backend_apply(be, sv, warm.ctypes.data_as(C.c_void_p), len(warm)) == 0
            assert ref.ref_device_synchronize() == 0
            for gname, q, arr in cases:
                assert ref.ref_backend_apply(be, sv, arr.ctypes.data_as(C.c_void_p), 1) == 0
                assert ref.ref_device_synchronize() == 0
                t0 = time.perf_counter()
                assert ref.ref_backend_apply(be, sv, arr.ctypes.data_as(C.c_void_p), len(arr)) == 0
                assert ref.ref_device_synchronize() == 0
                res.setdefault(f"{gname}@q{q}", {})[name] = (time.perf_counter() - t0) / len(arr) * 1e3
        finally:
            ref.ref_statevector_free(sv)
            ref.ref_backend_free(be)
    wins = sum(1 for r in res.values() if r["adapter"] <= r["reference_cuda"])
    for r in res.values():
        r["speedup"] = r["reference_cuda"] / r["adapter"] if r["adapter"] > 0 else None
    return {"qubits": n, "ms_per_gate": res, "adapter_not_slower": f"{wins} of {len(res)}",
            "timing": f"host clock between device synchronisations around {reps} applications of each gate, "
                      "after one untimed application"}


def bench_batch(dev, L, W, np, steps=5, warmup=3, autotune=True, count=512, wmin=10, wmax=22, dist=None, plain=True):
    """512 hardware-efficient-ansatz circuits (width U{10..22}, depth U{4..12}
    layers of RY+RZ per qubit and a CNOT ring, observable sum_i Z_i): forward
    <O> and the full adjoint gradient of every circuit per run, one persistent
    kernel replayed as a CUDA graph.  Baseline: the parameter-shift rule on the
    reference's per-gate CUDA kernels (2 executes per parameterised occurrence),
    run in full for sampled gradient entries of one circuit per width and
    charged per gate to every circuit of the batch.
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

    # plain parameter shift on the reference's CUDA kernels: for one circuit of each
    # width, 4 of its parameters' gradient entries computed in full (2 executes per
    # occurrence, each execute timed on the device plus one device <O>), checked
    # against the batch's adjoint; every circuit of the batch is then charged
    # 2 x occurrences x (that width's per-gate execute time x its gate count)
    occ_total = int(sum(int(np.sum(c[1]["param"] >= 0)) for c in circs))
    plain_est = None
    if plain:
        per_width = {}
        check_diff = 0.0
        for i, (w, ops, npar, obs_t) in enumerate(circs):
            if w in per_width:
                continue
            obs, keep = L.observable(*obs_t)
            obs_ms = device_expectation_ms(dev, L, w, obs, reps=3)
            gpu = RefGpu(w)
            try:
                pp = params[off[i]:off[i + 1]]
                pick = [int(x) for x in np.linspace(0, npar - 1, 4).astype(int)]
                entries, exec_s, timed = plain_param_shift_entries(gpu, ops, pp, observable_vector(w, *obs_t), pick)
            finally:
                gpu.close()
            for k, val in entries.items():
                check_diff = max(check_diff, abs(val - grads[off[i] + k]))
            per_width[w] = (exec_s / len(ops), obs_ms / 1e3, timed)
        ps_total = 0.0
        for (w, ops, npar, obs_t) in circs:
            occ = int(np.sum(ops["param"] >= 0))
            ps_total += 2 * occ * (per_width[w][0] * len(ops) + per_width[w][1])
        plain_est = {"param_shift_plain_s": ps_total,
                     "adjoint_batch_vs_plain_param_shift": ps_total / (run_ms / 1e3),
                     "plain_executes_timed": int(sum(t for _, _, t in per_width.values())),
                     "sampled_entries_max_abs_diff_vs_adjoint": check_diff,
                     "method": "the reference's CircuitUnitaryOperationGPU kernels (sm_100a): per width one circuit, "
                               "4 gradient entries in full by parameter shift (device time per execute + one "
                               "qse_expectation), the per-gate execute time of that width charged to every "
                               "circuit's 2 x occurrences executes"}
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
        "plain_param_shift": plain_est,
        "max_abs_diff_vs_single_state_adjoint": max(diffs),
        "config": None if cfg is None else cfg.__dict__,
        "stats": {k: st[k] for k in ("passes", "items", "tile_visits", "hbm_bytes", "grid", "smem_bytes", "plan_ms")},
        "hbm_gbs_multi_tile": hbm_gbs,
        "hbm_frac_multi_tile": hbm_gbs / hbm_peak,
        "setup_s": t_setup,
        "ranks": world,
        "rank0_circuits": len(mine),
        "timing": "device: CUDA events on the library stream around `steps` graph replays (device params); "
                  "e2e: host wall clock of qse_batch_run (params H2D, values+grads D2H)",
    }


if __name__ == "__main__":
    main()
