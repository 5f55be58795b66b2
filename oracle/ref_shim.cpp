// ref_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Linked with the reference's own sources (compiled from the reference tree
// by oracle/Makefile into oracle/_ref/, never copied into this repository).
// It replaces CircuitUnitaryOperationFactory.cpp, whose backend choice is
// MSVC-only on the CPU side (CircuitUnitaryOperationFactory.cpp:95-108), with
// an explicit choice, and exposes the reference Circuit through extern "C"
// so Python tests and bench.py's reference arm can drive it.
//
// Built three ways: libqse_ref_cpu.so (CPU backends), libqse_ref_gpu.so (+ the
// reference CUDA backend and the B200 adapter), libqse_ref_patched.so (the GPU
// build over a copy of the reference tree whose interface and Circuit carry the
// optional executeProgram / sample / measure hooks, oracle/patch_reference.py;
// QSE_REF_PATCHED).
//
// Backends: 0 = scalar CircuitUnitaryOperation (the FP64 oracle of record),
//           1 = CircuitUnitaryOperationAVX (the timed CPU baseline),
//           2 = CircuitUnitaryOperationGPU rebuilt for sm_100a (only in libqse_ref_gpu.so),
//           3 = CircuitUnitaryOperationB200, this project's drop-in adapter
//               (only in libqse_ref_gpu.so).
#include "Circuit.h"
#include "CircuitUnitaryOperation.h"
#include "CircuitUnitaryOperationAVX.h"
#include "CircuitUnitaryOperationFactory.h"
#include "Noise.h"
#include "StateVector.h"
#include "../include/qse_b200.h"

#include <cstdint>
#include <cstring>
#include <iostream>
#include <memory>
#include <random>
#include <sstream>
#include <vector>

#ifdef QSE_REF_WITH_GPU
#include "CircuitUnitaryOperationGPU.h"
#include "CircuitUnitaryOperationB200.h"
#endif

#ifdef QSE_REF_WITH_PLAYGROUND
#include "QFT.h"
// Grover::createGroverCircuit is a private static member; the test shim
// calls it directly (it builds the circuit without running or printing)
#define private public
#include "Grover.h"
#undef private
#include "TVS.h"
#endif

static int g_backend = 0;
#ifdef QSE_REF_WITH_GPU
static CircuitUnitaryOperationB200* g_last_b200 = nullptr;   // the newest adapter the factory made
#endif

std::unique_ptr<ICircuitUnitaryOperation> CircuitUnitaryOperationFactory::create(size_t numQubits)
{
    (void)numQubits;
    switch (g_backend) {
    case 1: return std::make_unique<CircuitUnitaryOperationAVX>();
#ifdef QSE_REF_WITH_GPU
    case 2: return std::make_unique<CircuitUnitaryOperationGPU>();
    case 3: {
        auto p = std::make_unique<CircuitUnitaryOperationB200>();
        g_last_b200 = p.get();
        return p;
    }
#endif
    default: return std::make_unique<CircuitUnitaryOperation>();
    }
}

namespace {
// Silences the reference's unconditional std::cout timing prints while in scope.
struct Quiet {
    std::streambuf* old;
    std::ostringstream sink;
    bool on;
    explicit Quiet(bool enable) : old(nullptr), on(enable) { if (on) old = std::cout.rdbuf(sink.rdbuf()); }
    ~Quiet() { if (on) std::cout.rdbuf(old); }
};
bool g_quiet = true;

struct RefCircuit {
    std::unique_ptr<Circuit> c;
    unsigned n;
};
}  // namespace

extern "C" {

int ref_has_gpu(void)
{
#ifdef QSE_REF_WITH_GPU
    return 1;
#else
    return 0;
#endif
}

void ref_set_quiet(int q) { g_quiet = q != 0; }

int ref_set_backend(int b)
{
#ifndef QSE_REF_WITH_GPU
    if (b >= 2) return -1;
#endif
    g_backend = b;
    return 0;
}

void* ref_circuit_new(unsigned n, int noise)
{
    Quiet q(g_quiet);
    auto* rc = new RefCircuit;
    rc->c = std::make_unique<Circuit>(n, noise != 0);
    rc->n = n;
    return rc;
}

void ref_circuit_free(void* h) { Quiet q(g_quiet); delete static_cast<RefCircuit*>(h); }

// Queue one op through Circuit's public gate builders (Circuit.cpp:9-62).
int ref_circuit_add(void* h, const qse_op* op)
{
    Circuit& c = *static_cast<RefCircuit*>(h)->c;
    switch (op->type) {
    case QSE_GATE_H: c.hadamard(op->target); return 0;
    case QSE_GATE_X: c.pauliX(op->target); return 0;
    case QSE_GATE_Y: c.pauliY(op->target); return 0;
    case QSE_GATE_Z: c.pauliZ(op->target); return 0;
    case QSE_GATE_PHASE: c.phase(op->theta, op->target); return 0;
    case QSE_GATE_RX: c.rotateX(op->theta, op->target); return 0;
    case QSE_GATE_RY: c.rotateY(op->theta, op->target); return 0;
    case QSE_GATE_RZ: c.rotateZ(op->theta, op->target); return 0;
    case QSE_GATE_CNOT: c.cnot(op->control, op->target); return 0;
    case QSE_GATE_CPHASE: c.cphase(op->theta, op->control, op->target); return 0;
    case QSE_GATE_MCPHASE: {
        std::vector<size_t> ctl;
        for (unsigned b = 0; b < 64; ++b)
            if ((op->controls >> b) & 1u) ctl.push_back(b);
        c.mcphase(op->theta, ctl, op->target);
        return 0;
    }
    case QSE_GATE_SWAP: c.swap(op->target, op->control); return 0;
    default: return -1;
    }
}

int ref_circuit_add_many(void* h, const qse_op* ops, size_t n)
{
    for (size_t i = 0; i < n; ++i)
        if (ref_circuit_add(h, &ops[i]) != 0) return -1;
    return 0;
}

void ref_circuit_execute(void* h, int print_steps)
{
    Quiet q(g_quiet);
    static_cast<RefCircuit*>(h)->c->execute(print_steps != 0);
}

void ref_circuit_reset(void* h)
{
    Quiet q(g_quiet);
    static_cast<RefCircuit*>(h)->c->reset();
}

// Host copy of the state.  Circuit::printState() is the public call that
// flushes a device backend (Circuit.cpp:135-138); its print is silenced.
void ref_circuit_state(void* h, double* out)
{
    auto* rc = static_cast<RefCircuit*>(h);
    {
        Quiet q(true);
        rc->c->printState();
    }
    auto& v = rc->c->getStateVector().data();
    std::memcpy(out, v.data(), v.size() * sizeof(std::complex<double>));
}

// The reference playground's circuit builders queueing onto a reference
// Circuit, with the preamble of the run* function that calls them:
// which 0 = QFT::runQFT (QFT.cpp:39-71: X(0), createQFT over 0..n-1),
// 1 = QFT::runIQFT (QFT.cpp:73-105: X(0), createIQFT), 2 =
// Grover::createGroverCircuit(n, target, iterations) (Grover.cpp:65-75).
// Returns -1 when built without the playground sources or for an unknown which.
int ref_playground_build(void* h, int which, int target, int iterations)
{
#ifdef QSE_REF_WITH_PLAYGROUND
    auto* rc = static_cast<RefCircuit*>(h);
    Circuit& c = *rc->c;
    std::vector<size_t> qs;
    for (unsigned i = 0; i < rc->n; ++i) qs.push_back(i);
    switch (which) {
    case 0: c.pauliX(0); QFT::createQFT(c, qs); return 0;
    case 1: c.pauliX(0); QFT::createIQFT(c, qs); return 0;
    case 2: Grover::createGroverCircuit(c, int(rc->n), target, iterations); return 0;
    default: return -1;
    }
#else
    (void)h; (void)which; (void)target; (void)iterations;
    return -1;
#endif
}

// TVS::buildIsing (TVS.cpp:31-99) on an n x n distance matrix (row-major):
// fields into h (n*n), couplings into pairs (2 per coupling, i < j) and coeffs
// in the reference's hash-map order; *npairs receives their count (at most cap).
// Returns -1 without the playground sources or when cap is too small.
int ref_tsp_ising(const double* dist, unsigned n, double penalty, double weight, int row_constraint,
                  int col_constraint, double* h, unsigned* pairs, double* coeffs, unsigned cap, unsigned* npairs)
{
#ifdef QSE_REF_WITH_PLAYGROUND
    std::vector<std::vector<double>> d(n, std::vector<double>(n));
    for (unsigned a = 0; a < n; ++a)
        for (unsigned b = 0; b < n; ++b) d[a][b] = dist[a * n + b];
    std::vector<std::pair<size_t, size_t>> zz;
    std::vector<double> c;
    std::vector<double> hv = TVS::buildIsing(n, penalty, weight, d, zz, c, row_constraint != 0, col_constraint != 0);
    if (zz.size() > cap) return -1;
    for (size_t i = 0; i < hv.size(); ++i) h[i] = hv[i];
    for (size_t k = 0; k < zz.size(); ++k) {
        pairs[2 * k] = unsigned(zz[k].first);
        pairs[2 * k + 1] = unsigned(zz[k].second);
        coeffs[k] = c[k];
    }
    *npairs = unsigned(zz.size());
    return 0;
#else
    (void)dist; (void)n; (void)penalty; (void)weight; (void)row_constraint; (void)col_constraint;
    (void)h; (void)pairs; (void)coeffs; (void)cap; (void)npairs;
    return -1;
#endif
}

uint64_t ref_circuit_measure(void* h)
{
    Quiet q(g_quiet);
    return static_cast<RefCircuit*>(h)->c->measure();
}

void ref_circuit_sample(void* h, int shots, uint64_t* out)
{
    Quiet q(g_quiet);
    auto r = static_cast<RefCircuit*>(h)->c->sample(shots);
    for (size_t i = 0; i < r.size(); ++i) out[i] = r[i];
}

// Noise (Noise.cpp) driven directly: accumulate over a sequence of gate types
// and targets, then applyPauliNoise onto a caller-given state through the
// scalar backend.  Returns total bit flips / phase flips.
void ref_noise_run(unsigned n, unsigned seed, double mult, const int* types, const unsigned* targets,
                   size_t ngates, double* state, uint64_t* bit_total, uint64_t* phase_total)
{
    Quiet q(true);
    Noise nz(n, seed, mult);
    for (size_t i = 0; i < ngates; ++i) nz.accumulateError(static_cast<GateType>(types[i]), targets[i]);
    StateVector sv(n);
    std::memcpy(sv.data().data(), state, (size_t(1) << n) * sizeof(std::complex<double>));
    CircuitUnitaryOperation op;
    nz.applyPauliNoise(sv, op);
    std::memcpy(state, sv.data().data(), (size_t(1) << n) * sizeof(std::complex<double>));
    *bit_total = nz.getTotalBitFlips();
    *phase_total = nz.getTotalPhaseFlips();
}

// std::uniform_real_distribution<double>(0,1) over std::mt19937(seed): the
// draw sequence Noise.cpp consumes (checks the oracle's mt19937 restatement).
void ref_std_uniforms(unsigned seed, size_t count, double* out)
{
    std::mt19937 gen(seed);
    std::uniform_real_distribution<double> dist(0.0, 1.0);
    for (size_t i = 0; i < count; ++i) out[i] = dist(gen);
}

// Per-gate timing through one backend object directly (bench reference arm):
// applies ops [0, nops) to the state held by the circuit's StateVector.
void* ref_backend_new(int b)
{
    int saved = g_backend;
    g_backend = b;
    auto p = CircuitUnitaryOperationFactory::create(0);
    g_backend = saved;
    return p.release();
}

void ref_backend_free(void* be) { delete static_cast<ICircuitUnitaryOperation*>(be); }

// CircuitUnitaryOperationB200's sample / measure extensions on a backend made
// by ref_backend_new(3) (only in libqse_ref_gpu.so); -1 for another backend.
int ref_b200_sample(void* be, void* svp, const double* u, size_t shots, uint64_t* out)
{
#ifdef QSE_REF_WITH_GPU
    auto* b = dynamic_cast<CircuitUnitaryOperationB200*>(static_cast<ICircuitUnitaryOperation*>(be));
    if (!b) return -1;
    std::vector<size_t> r;
    b->sample(*static_cast<StateVector*>(svp), u, shots, r);
    for (size_t i = 0; i < r.size(); ++i) out[i] = r[i];
    return 0;
#else
    (void)be; (void)svp; (void)u; (void)shots; (void)out;
    return -1;
#endif
}

// Kernels launched so far by the newest adapter the factory made (tells the
// fused path, a few passes, from one kernel per gate); 0 without one.
uint64_t ref_b200_kernel_launches(void)
{
#ifdef QSE_REF_WITH_GPU
    return g_last_b200 ? qse_ctx_kernel_launches(g_last_b200->context()) : 0;
#else
    return 0;
#endif
}

int ref_b200_measure(void* be, void* svp, double u, uint64_t* out)
{
#ifdef QSE_REF_WITH_GPU
    auto* b = dynamic_cast<CircuitUnitaryOperationB200*>(static_cast<ICircuitUnitaryOperation*>(be));
    if (!b) return -1;
    size_t r = 0;
    b->measure(*static_cast<StateVector*>(svp), u, r);
    *out = r;
    return 0;
#else
    (void)be; (void)svp; (void)u; (void)out;
    return -1;
#endif
}

void* ref_statevector_new(unsigned n) { Quiet q(true); return new StateVector(n); }
void ref_statevector_free(void* sv) { delete static_cast<StateVector*>(sv); }

int ref_backend_apply(void* be, void* svp, const qse_op* ops, size_t nops)
{
    auto& op = *static_cast<ICircuitUnitaryOperation*>(be);
    auto& sv = *static_cast<StateVector*>(svp);
    for (size_t i = 0; i < nops; ++i) {
        const qse_op& o = ops[i];
        switch (o.type) {
        case QSE_GATE_H: op.applyHadamard(sv, o.target); break;
        case QSE_GATE_X: op.applyPauliX(sv, o.target); break;
        case QSE_GATE_Y: op.applyPauliY(sv, o.target); break;
        case QSE_GATE_Z: op.applyPauliZ(sv, o.target); break;
        case QSE_GATE_PHASE: op.applyPhase(sv, o.target, o.theta); break;
        case QSE_GATE_RX: op.applyRotateX(sv, o.target, o.theta); break;
        case QSE_GATE_RY: op.applyRotateY(sv, o.target, o.theta); break;
        case QSE_GATE_RZ: op.applyRotateZ(sv, o.target, o.theta); break;
        case QSE_GATE_CNOT: op.applyCNOT(sv, o.control, o.target); break;
        case QSE_GATE_CPHASE: op.applyCPhase(sv, o.control, o.target, o.theta); break;
        case QSE_GATE_MCPHASE: {
            std::vector<size_t> ctl;
            for (unsigned b = 0; b < 64; ++b)
                if ((o.controls >> b) & 1u) ctl.push_back(b);
            op.applyMCPhase(sv, ctl, o.target, o.theta);
            break;
        }
        case QSE_GATE_SWAP: op.applySwap(sv, o.target, o.control); break;
        case QSE_GATE_2X2: {
            Gate2x2 g(Complex(o.m[0], o.m[1]), Complex(o.m[2], o.m[3]),
                      Complex(o.m[4], o.m[5]), Complex(o.m[6], o.m[7]));
            op.applyGate(sv, g, o.target);
            break;
        }
        default: return -1;
        }
    }
    return 0;
}

void ref_backend_flush(void* be) { static_cast<ICircuitUnitaryOperation*>(be)->flush(); }
void ref_backend_mark_host_dirty(void* be) { static_cast<ICircuitUnitaryOperation*>(be)->markHostDirty(); }

void ref_statevector_get(void* svp, double* out)
{
    auto& v = static_cast<StateVector*>(svp)->data();
    std::memcpy(out, v.data(), v.size() * sizeof(std::complex<double>));
}

void ref_statevector_set(void* svp, const double* in)
{
    auto& v = static_cast<StateVector*>(svp)->data();
    std::memcpy(v.data(), in, v.size() * sizeof(std::complex<double>));
}

uint64_t ref_statevector_measure(void* svp) { Quiet q(g_quiet); return static_cast<StateVector*>(svp)->measure(); }
int ref_statevector_measure_qubit(void* svp, unsigned qubit)
{
    Quiet q(g_quiet);
    return static_cast<StateVector*>(svp)->measureQubit(qubit);
}
void ref_statevector_reset_qubit(void* svp, unsigned qubit)
{
    Quiet q(true);
    static_cast<StateVector*>(svp)->resetQubit(qubit);
}

#ifdef QSE_REF_PATCHED
// Draw source of the patched Circuit::sample / Circuit::measure
// (oracle/patch_reference.py): injected uniforms first, then a generator seeded
// from std::random_device like the reference's own draws.
namespace {
std::vector<double> g_injected;
size_t g_injected_next = 0;
}  // namespace
}  // extern "C"
double qse_patch_next_uniform()
{
    if (g_injected_next < g_injected.size()) return g_injected[g_injected_next++];
    static std::mt19937 gen{std::random_device{}()};
    return std::uniform_real_distribution<double>(0.0, 1.0)(gen);
}
extern "C" {
void ref_inject_uniforms(const double* u, size_t n)
{
    g_injected.assign(u, u + n);
    g_injected_next = 0;
}
#endif

// StateVector::reset (StateVector.cpp:34-46): |0..0> on the host copy.
void ref_statevector_reset(void* svp)
{
    Quiet q(true);
    static_cast<StateVector*>(svp)->reset();
}

// Waits for every kernel the reference CUDA backend has queued (it launches
// on a private stream and synchronises only in flush or print_steps timing);
// lets the bench time its kernels without a state copy.  0 on success.
int ref_device_synchronize(void)
{
#ifdef QSE_REF_WITH_GPU
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
#else
    return -1;
#endif
}

void ref_statevector_sample(void* svp, int shots, uint64_t* out)
{
    Quiet q(g_quiet);
    auto r = static_cast<StateVector*>(svp)->sample(shots);
    for (size_t i = 0; i < r.size(); ++i) out[i] = r[i];
}

}  // extern "C"
