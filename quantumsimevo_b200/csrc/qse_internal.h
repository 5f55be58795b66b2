// qse_internal.h -- host-side structures shared by the CUDA and C++ sources of
// libqse_b200.so.  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/qse_b200.h"

namespace qse {

// Exception carrying a C-ABI status; caught at the extern "C" boundary.
struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

[[noreturn]] void fail(int status, const std::string& msg);
void set_last_error(const std::string& msg);   // qse_last_error() text of the calling thread
void cuda_check(cudaError_t e, const char* what, const char* file, int line);
#define QSE_CUDA(call) ::qse::cuda_check((call), #call, __FILE__, __LINE__)

// Growable device buffer owned by a context.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    void reserve(size_t n);
    void release();
    ~DevBuf() { release(); }
};

struct PlanCache;   // engine.cu: plans of recent executes, reused when a program runs again

// Pinned host staging buffer.
struct HostBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    void reserve(size_t n);
    void release();
    ~HostBuf() { release(); }
};

}  // namespace qse

struct qse_ctx {
    int device = 0;
    int num_sms = 148;
    size_t smem_optin = 0;
    cudaStream_t stream = nullptr;
    // planner knobs
    int fusion = 1;
    int jit = 1;             // specialised NVRTC pass kernels (0: generic interpreter kernel,
                             // 2: specialised, with the streamed persistent kernel where it applies)
    int tile_qubits = 12;
    int max_gates_per_pass = 0;
    int sample_mode = 0;
    uint64_t launches = 0;
    // device error word of the kernels with bounded waits (streamed passes, the sampling scan):
    // mapped pinned host memory, read on the host after a synchronisation
    unsigned* status_host = nullptr;
    unsigned* status_dev = nullptr;
    // scratch shared by the calls on this context (single host thread, like the reference backend)
    qse::DevBuf plan_buf;    // uploaded pass programs
    qse::HostBuf plan_host;  // pinned staging for the pass programs
    qse::DevBuf scratch;     // reductions, sampling, noise decisions
    qse::DevBuf scratch2;
    qse::DevBuf gv_buf;      // per-tile group values of the pass being launched (precomputed)
    qse::HostBuf host_small; // pinned small results
    qse::HostBuf host_small2;
    cudaEvent_t plan_event = nullptr;  // last H2D copy out of plan_host
    cudaEvent_t slots[64] = {};        // qse_ctx_record / qse_ctx_elapsed
    // qse_ctx_time_passes: event pairs around every fused-pass launch
    bool time_passes = false;
    std::vector<cudaEvent_t> pass_events;  // pool, pairs (start, stop)
    size_t pass_events_used = 0;
    // state of at most kCompactMaxQubits qubits on which an execute runs the
    // leading passes of a circuit that leave the other qubits in their basis
    // state (engine.cu, compact_prefix); allocated on first use
    qse_state* compact = nullptr;
    qse::PlanCache* plan_cache = nullptr;   // allocated on first use
};

struct qse_state {
    qse_ctx* ctx = nullptr;
    uint32_t n = 0;
    double* amp = nullptr;       // 2^n complex128 (interleaved), physical qubit order
    double* aux = nullptr;       // second state (adjoint |lambda>), allocated on first use
    uint32_t perm[64];           // logical qubit -> physical bit
    uint64_t version = 0;        // bumped by every call that writes the amplitudes
    bool lazy_basis = false;     // the state is the basis state |lazy_index> (a physical index)
    uint64_t lazy_index = 0;     // but the array has not been written: the next fused execute
                                 // generates it in its first pass, every other reader calls
                                 // materialize() first (reset: |0..0>; measure: the outcome)
    // with lazy_basis, inside one execute: the state is a compact state on the
    // physical qubits of lazy_umask (lazy_src, indexed by those bits in
    // ascending order) times, on the qubits of lazy_pmask, one single-qubit
    // state each (product qubits: the 2 amplitudes of the i-th lowest at
    // lazy_src[2^popcount(lazy_umask) + 2i + bit]) times the basis bits of
    // lazy_index on the other qubits
    uint64_t lazy_umask = 0;
    uint64_t lazy_pmask = 0;
    const void* lazy_src = nullptr;
    // probabilities written by the last pass of an execute (cdf buffer, see
    // prob_buffer_bytes) are current while prob_version == version.  prob_hint:
    // the state has been sampled, so executes write them; prob_pending: they
    // were written and no sampling has read them yet (an execute that finds
    // them unread stops writing them)
    bool prob_hint = false;
    bool prob_pending = false;
    bool prob_bsum = false;      // the block sums were written with them
    uint64_t prob_version = ~uint64_t(0);
    // exact cumulative probabilities (sample.cu), valid while cdf_version == version
    qse::DevBuf cdf;
    uint64_t cdf_version = ~uint64_t(0);
    double* cdf_values = nullptr;
    double* cdf_block_start = nullptr;
    uint32_t cdf_nb = 0;
    uint32_t cdf_bs = 0;
    void touch() { ++version; }
    bool identity_perm() const {
        for (uint32_t q = 0; q < n; ++q)
            if (perm[q] != q) return false;
        return true;
    }
    size_t size() const { return size_t(1) << n; }
};

struct qse_noise {
    qse_ctx* ctx = nullptr;
    uint32_t n = 0;
    qse_noise_config cfg{};
    uint64_t draws = 0;          // noisy gates so far (Philox counter)
    int32_t* d_counts = nullptr; // device: bit[64], phase[64], then rates double[16]
    // QSE_RNG_MT19937: the generator and distribution of Noise.cpp:7-8
    std::mt19937 gen;
    std::uniform_real_distribution<double> dist{0.0, 1.0};
};

namespace qse {

// Launch bookkeeping.
inline void count_launch(qse_ctx* ctx, uint64_t n = 1) { ctx->launches += n; }

// After a synchronisation of the context's stream: the error word the pass
// kernels set when one of their bounded waits gave up (then cleared).
inline void check_device_status(qse_ctx* ctx)
{
    if (!ctx->status_host) return;
    volatile unsigned* s = ctx->status_host;
    const unsigned v = *s;
    if (v == 0u) return;
    *s = 0u;
    fail(QSE_ERR_TIMEOUT, "a kernel's bounded wait gave up (status " + std::to_string(v) +
                              ": 1-2 a streamed pass, 4 the sampling scan, 8 a pass kernel's index check in "
                              "QSE_DEBUG_BOUNDS mode); its results are invalid");
}

// ---- per-gate ("plain method") kernels: gates.cu ----
void launch_gate2x2(qse_state* st, uint32_t q, const double m[8], uint64_t ctrl_mask);
void launch_h(qse_state* st, uint32_t q);
void launch_x(qse_state* st, uint32_t q);
void launch_y(qse_state* st, uint32_t q);
void launch_z(qse_state* st, uint32_t q);
void launch_phase_mask(qse_state* st, uint64_t all_mask, double c, double s);  // phase/cphase/mcphase
void launch_cphase(qse_state* st, uint32_t c, uint32_t t, double co, double si);
void launch_rx(qse_state* st, uint32_t q, double c, double s);
void launch_ry(qse_state* st, uint32_t q, double c, double s);
void launch_rz(qse_state* st, uint32_t q, double c0, double s0, double c1, double s1);
void launch_cnot(qse_state* st, uint32_t c, uint32_t t);
void launch_swap(qse_state* st, uint32_t q0, uint32_t q1);
void launch_init_zero_state(qse_state* st);                          // write |0..0> now
void mark_basis(qse_state* st, uint64_t phys_index);                 // lazy |phys_index>
void mark_zero(qse_state* st);       // reset without writing: lazy |0..0>
// StateVector::measureQubit (reset = false) / resetQubit (reset = true), draw u injected
int measure_or_reset_qubit(qse_state* st, uint32_t qubit, double u, bool reset, double* prob1);
void materialize(qse_state* st);     // write a lazy basis (or compact) state into the array (no-op otherwise)
void destroy_compact_state(qse_ctx* ctx);
void destroy_plan_cache(qse_ctx* ctx);
void launch_pauli_frame(qse_state* st, const int32_t* d_counts);      // Noise::applyPauliNoise
void permute_to_logical(qse_state* st, double* dst_device);           // gather into logical order
void scale_state(qse_state* st, double s);

// ---- fused execution (engine.cu / planner.cpp / tile.cu) ----
void execute_program(qse_state* st, const qse_op* ops, size_t nops, const double* params, size_t nparams,
                     qse_noise* noise, const double* inj, size_t ninj, qse_exec_stats* stats);
void canonicalize(qse_state* st);

// ---- sampling (sample.cu) ----
size_t prob_buffer_bytes(uint64_t size);
void sample(qse_state* st, const double* u_host, size_t nshots, uint64_t seed, uint64_t* out_host);
void sample_device(qse_state* st, const double* d_u, size_t nshots, uint64_t seed, uint64_t* d_out);
uint64_t measure(qse_state* st, double u);
double total_probability(qse_state* st);
void sampler_stats(qse_state* st, uint32_t out[4]);

// ---- noise (noise.cu) ----
void noise_decide(qse_noise* nz, const int32_t* d_types, const uint32_t* d_targets, size_t ngates,
                  const double* d_uniforms);
// ---- observables / adjoint (adjoint.cu) ----
double expectation(qse_state* st, const qse_observable* obs);
double expectation_noalloc(qse_state* st, const qse_observable* obs);
double adjoint(qse_state* st, const qse_op* ops, size_t nops, const double* params, size_t nparams,
               const qse_observable* obs, double* grad);

// helpers
uint64_t logical_to_physical_index(const qse_state* st, uint64_t logical);
uint64_t physical_to_logical_index(const qse_state* st, uint64_t physical);
double bound_angle(const qse_op& op, const double* params, size_t nparams);

}  // namespace qse
