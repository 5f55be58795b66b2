// planner.h -- gate-fusion planner: turns the queued gate list of
// Circuit::execute (Circuit.cpp:64-120) into full-state passes, each applied by
// one launch of the tile kernel (tile.cu).
//
// A pass owns a set T of k "tile" qubits.  Every CTA loads the 2^k amplitudes
// that differ only in T (the other, "outer" bits are fixed per CTA), applies a
// run of gates in registers, and writes them back: one HBM read + write per
// pass instead of one per gate.  A non-diagonal gate (H, X, Y, RX, RY, 2x2,
// CNOT target) needs its target in T; diagonal gates (Z, PHASE, RZ, CPHASE,
// MCPHASE) and CNOT controls can sit on any qubit, because each amplitude's
// full index is known inside the kernel.  SWAP costs nothing: it relabels the
// logical->physical qubit map.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace qse {
namespace plan {

// ---- device program records (layout shared with tile.cu) ----
enum KKind : uint8_t {
    K_NOP = 0,
    K_H,           // unscaled Hadamard on register bit p (the pass scale carries 1/sqrt2 per H)
    K_X,           // X on p, controls: register mask f, thread mask tcond, outer mask ocond
    K_Y,           // Y on p, same controls
    K_RX,          // [[c,-is],[-is,c]] on p, (a,b) = (c,s)
    K_RY,          // [[c,-s],[s,c]] on p
    K_U,           // generic 2x2 on p, matrix index g, controls as K_X
    K_ACC_THR,     // if thread cond: acc_thr += group value g  (acc_mul: acc_thr *= (cos, sin) g)
    K_ACC_REG,     // if thread cond: acc[p] += group value g   (acc_mul: acc[p] *= (cos, sin) g)
    K_PHD,         // if thread cond: amplitudes with (j & f) == f *= group (cos, sin) g
    K_FLUSH_REG,   // amplitudes with bit p *= e^{i acc[p]}; acc[p] = 0
    K_FLUSH_ALL,   // flush acc[p] for p in f, then all amplitudes *= e^{i acc_thr} * (a + ib)
    K_TRANSPOSE,   // exchange through shared memory into layout g
    K_GRAD_X,      // slot g += sum_pairs Im(conj(l0) s1 + conj(l1) s0)         (RX generator)
    K_GRAD_Y,      // slot g += sum_pairs Re(conj(l1) s0) - Re(conj(l0) s1)     (RY generator)
    K_GRAD_Z,      // slot g += sum sign * Im(conj(l) s): sign flips on reg bit p (p<8), thread mask tcond, outer mask ocond
    K_GRAD_P,      // if conds: slot g += sum_{(j&f)==f} Im(conj(l) s)          (phase-type generator, scaled on host)
    K_KIND_COUNT
};

struct KOp {
    uint8_t kind;
    uint8_t p;
    uint8_t q;
    uint8_t f;
    uint16_t tcond;
    uint16_t g;
    uint64_t ocond;
    double a;
    double b;
};
static_assert(sizeof(KOp) == 32, "KOp layout");

struct LayoutRec {
    uint8_t reg[5];    // tile-local bits held in registers (register index bit i <-> reg[i]; rb <= 5)
    uint8_t nthr;      // number of thread-index bits
    uint8_t pad[2];
    uint16_t L[16];    // shared-memory slot image of every tile-local bit (XOR-linear map)
    uint8_t thr[16];   // tile-local bit of thread-index bit t (ascending), t < nthr
};
static_assert(sizeof(LayoutRec) == 56, "LayoutRec layout");

struct TermRec {       // one diagonal term: angle theta if all outer bits of ocond are set
    uint64_t ocond;
    double theta;
};

struct GroupRec {      // terms [first, first+count) summed per CTA; direct groups get (cos, sin)
    uint32_t first;
    uint32_t count;
    uint32_t direct;
    uint32_t pad;
};

// An angle-carrying record of a pass and the source gate it came from: a
// K_RX / K_RY op (a, b) = (cos, sin)(theta/2), or a diagonal term's theta.
// Lets a caller rebind angles on the device without planning again.
struct AngleRef {
    uint32_t index;   // into PassProgram::ops or PassProgram::terms
    uint32_t src;     // source-gate index in the planner input
};

struct PassProgram {
    uint32_t k = 0;                 // tile qubits
    uint32_t rb = 4;                // register bits per thread
    bool acc_mul = false;           // accumulators carry complex factors (Options::acc_mul)
    uint64_t outer_mask = 0;        // physical qubits not in the tile
    uint8_t tile_phys[16] = {0};    // physical qubit of tile-local bit b (ascending)
    uint32_t layout0 = 0;           // layout at load time (index into layouts)
    std::vector<KOp> ops;
    std::vector<LayoutRec> layouts;
    std::vector<TermRec> terms;
    std::vector<GroupRec> groups;
    std::vector<double> mats;       // 8 doubles per K_U matrix
    std::vector<int32_t> slot_src;  // gradient slot (local) -> gradient occurrence id
    std::vector<AngleRef> op_angles;    // K_RX / K_RY ops
    std::vector<AngleRef> term_angles;  // terms of PHASE / RZ / CPHASE / MCPHASE gates
    std::vector<uint32_t> order;    // source-gate indices absorbed, in execution order
    // debug view, per entry of `order`: physical target, physical control
    // (CNOT / CPHASE) and physical support (diagonal gates); SWAPs come first
    // with zeros (they only relabel)
    std::vector<uint32_t> phys_target;
    std::vector<uint32_t> phys_control;
    std::vector<uint64_t> phys_support;
    uint32_t ngates = 0;            // source gates absorbed
    uint32_t n_nondiag = 0;
};

// ---- planner input ----
struct Gate {
    int type = 0;          // qse_gate_type
    uint32_t t = 0;        // target (SWAP: q0)
    uint32_t c = 0;        // control (CNOT, CPHASE; SWAP: q1)
    uint64_t cmask = 0;    // MCPHASE controls (logical)
    double theta = 0.0;    // bound angle
    double m[8] = {0};     // QSE_GATE_2X2
    int32_t grad = -1;     // gradient occurrence id (adjoint reverse sweep), -1 = none
};

// Non-diagonal gates per pass when the passes are compiled into specialised
// kernels: NVRTC's compile time grows faster than linearly with the length of
// the straight-line kernel (a 12-qubit pass of 2400 gates takes over a minute),
// while an extra pass costs one sweep of the state.
constexpr uint32_t kJitMaxGates = 256;

struct Options {
    uint32_t k = 12;             // tile qubits (clamped to n)
    uint32_t rb = 4;             // register bits per thread (at most 5; the interpreter kernel takes 3 or 4)
    uint32_t max_gates = 0;      // 0 = no cap on non-diagonal gates per pass
    uint32_t max_terms = 1024;   // diagonal terms per pass (shared-memory group table)
    bool grads = false;          // emit K_GRAD_* for gates with grad >= 0
    uint32_t max_slots = 0;      // gradient slots per pass, 0 = no cap
    bool direct_phases = false;  // single-register-bit phase terms without a thread
                                 // condition as direct (cos, sin) groups
    bool acc_mul = false;        // accumulator groups (K_ACC_THR / K_ACC_REG) are direct too:
                                 // kernels multiply their (cos, sin) into per-thread complex
                                 // factors instead of summing angles and calling sincos per flush
    bool zz_fuse = false;        // rewrite CNOT(c,t) RZ(th,t) CNOT(c,t) as the diagonal
                                 // RZ(th,c) PHASE(th,t) CPHASE(-2th,c,t) (same three slots;
                                 // only for plans whose angles are never rebound)
    bool keep_gphase = true;     // false: drop RZ's global phase (expectations and gradients
                                 // do not see it; the pass programs then depend on angles
                                 // only through op_angles / term_angles)
};

struct Plan {
    std::vector<PassProgram> passes;
    uint32_t perm_final[64];
    double gphase = 0.0;         // global phase (RZ's e^{-i theta/2}), folded into the last pass
    uint64_t gates = 0;
};

// The rewrite of Options::zz_fuse on its own: out = gates with every
// CNOT(c,t) RZ(th,t) CNOT(c,t) (no gradient ids) replaced by RZ(th,c)
// PHASE(th,t) CPHASE(-2th,c,t) in the same three slots; false (out untouched)
// when there is none.
bool fuse_zz(const std::vector<Gate>& gates, std::vector<Gate>& out);

// Plans gates (logical qubits) for an n-qubit state whose logical->physical
// map is perm_in.  Throws qse::Error on invalid gates.
Plan build(const std::vector<Gate>& gates, uint32_t n, const uint32_t* perm_in, const Options& opt);

// Planner-only debug view used by the CPU tests: for each pass, the tile
// (physical qubits) and the source-gate indices in execution order.
std::string describe(const Plan& p);

}  // namespace plan
}  // namespace qse
