/*
 * qse_b200.h -- C ABI of the B200 (sm_100a) state-vector backend.
 *
 * Plain C: opaque handles, pointers and sizes, int status codes, no C++ or
 * torch types.  Every entry point returns QSE_OK (0) or a QSE_ERR_* code and
 * never aborts the process; qse_last_error() gives the message of the last
 * failure on the calling thread.
 *
 * Conventions (identical to the reference engine, QuantumSimEvo):
 *   - a state of n qubits is 2^n complex128 amplitudes, interleaved (re, im),
 *     basis index little-endian: qubit 0 is the least significant bit
 *     (QSETests/QSETests.cpp:131-132);
 *   - gate matrices and semantics follow QuantumSimEvo/CircuitUnitaryOperation.cpp
 *     (the scalar FP64 backend) and QuantumSimEvo/QubitUnitaryOperation.cpp;
 *   - the gate-type numbering follows GateType (QuantumSimEvo/Structurs.h:10).
 *
 * Each entry point names the reference interface it stands in for.
 */
#ifndef QSE_B200_H
#define QSE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define QSE_API __attribute__((visibility("default")))
#else
#define QSE_API
#endif

/* ---- status codes ---------------------------------------------------- */
enum qse_status {
    QSE_OK = 0,
    QSE_ERR_INVALID = 1,      /* bad argument (null pointer, bad enum, ...)   */
    QSE_ERR_QUBIT = 2,        /* qubit index out of range / duplicated        */
    QSE_ERR_OOM = 3,          /* device or host allocation failed             */
    QSE_ERR_CUDA = 4,         /* CUDA runtime error (message has details)     */
    QSE_ERR_SIZE = 5,         /* qubit count / size beyond supported limits   */
    QSE_ERR_UNSUPPORTED = 6,  /* gate type not handled on this path           */
    QSE_ERR_TIMEOUT = 7,      /* a bounded device wait gave up                */
    QSE_ERR_STATE = 8         /* call not valid in the handle's current state */
};

/* ---- gate types: same numbering as GateType (Structurs.h:10) ---------- */
enum qse_gate_type {
    QSE_GATE_IDENTITY = 0,
    QSE_GATE_X = 1,
    QSE_GATE_Y = 2,
    QSE_GATE_Z = 3,
    QSE_GATE_H = 4,
    QSE_GATE_PHASE = 5,
    QSE_GATE_RX = 6,
    QSE_GATE_RY = 7,
    QSE_GATE_RZ = 8,
    QSE_GATE_CNOT = 9,
    QSE_GATE_CPHASE = 10,
    QSE_GATE_MCPHASE = 11,
    QSE_GATE_SWAP = 12,
    QSE_GATE_MEASURE = 13,      /* not executable on this path (reference has no executor for it) */
    QSE_GATE_RESET_QUBIT = 14,  /* not executable on this path */
    QSE_GATE_2X2 = 15           /* ICircuitUnitaryOperation::applyGate (no GateType in the reference) */
};

/*
 * One queued gate: the fields of GateCommand (Structurs.h:12-20) as plain data.
 *   target   GateCommand::target  (SWAP: q0)
 *   control  GateCommand::control (CNOT / CPHASE control; SWAP: q1)
 *   controls MCPHASE: bit mask of GateCommand::controls_list (duplicates are
 *            harmless, as in applyMCPhase's allMask, CircuitUnitaryOperation.cpp:296-297)
 *   theta    rotation / phase angle
 *   param    -1: the angle is theta.  >= 0: the angle is theta + coeff*params[param]
 *            (parameter binding for the adjoint and batched entry points)
 *   m        QSE_GATE_2X2 only: Gate2x2::data row-major, (re, im) pairs:
 *            m = {d00.re, d00.im, d01.re, d01.im, d10.re, d10.im, d11.re, d11.im}
 */
typedef struct qse_op {
    int32_t  type;
    uint32_t target;
    uint32_t control;
    int32_t  param;
    uint64_t controls;
    double   theta;
    double   coeff;
    double   m[8];
} qse_op;

/* Diagonal observable O(x) = constant + sum_t weight[t] * (-1)^popcount(x & zmask[t]):
 * sums of Z-strings, e.g. sum_i Z_i or the Max-Cut cost sum_edges (1 - Z_u Z_v)/2. */
typedef struct qse_observable {
    size_t          nterms;
    const uint64_t* zmask;
    const double*   weight;
    double          constant;
} qse_observable;

/* Noise model of QuantumSimEvo/Noise.cpp: per-gate error rates indexed by
 * gate type (Noise.cpp:10-18 defaults: X,Y,Z,PHASE,RX,RY,RZ 1e-3, H 2e-3,
 * CNOT 5e-3, every other type 0 = never draws) times a multiplier. */
enum qse_rng_mode {
    QSE_RNG_PHILOX = 0,     /* device Philox4x32-10, counter = draw index   */
    QSE_RNG_MT19937 = 1,    /* host mt19937(seed) + libstdc++ generate_canonical, as Noise.cpp */
    QSE_RNG_INJECTED = 2    /* caller-supplied uniforms, two per noisy gate */
};

typedef struct qse_noise_config {
    int32_t  enabled;
    int32_t  rng_mode;      /* qse_rng_mode */
    uint64_t seed;          /* Noise(N, seed=42, ...) */
    double   multiplier;    /* errorRateMultiplier */
    double   rates[16];     /* per qse_gate_type; rates of types outside the map must be 0 */
} qse_noise_config;

typedef struct qse_exec_stats {
    uint64_t gates;          /* gates executed                               */
    uint64_t passes;         /* full-state HBM passes launched               */
    uint64_t kernels;        /* kernel launches issued                       */
    uint64_t noisy_gates;    /* gates that drew noise uniforms               */
} qse_exec_stats;

/* ---- library / context ---------------------------------------------- */
typedef struct qse_ctx qse_ctx;
typedef struct qse_state qse_state;

QSE_API const char* qse_last_error(void);
QSE_API const char* qse_version(void);

/* CircuitUnitaryOperationGPU::CircuitUnitaryOperationGPU (CircuitUnitaryOperationGPU.cu:140-149):
 * binds `device`, creates the private stream. */
QSE_API int qse_ctx_create(int device, qse_ctx** out);
QSE_API int qse_ctx_destroy(qse_ctx* ctx);
QSE_API int qse_ctx_synchronize(qse_ctx* ctx);
/* fused-planner knobs: tile qubits (10..12), cap on non-diagonal gates per pass
 * (0 = none; with specialised pass kernels at most 256, which bounds their
 * compile time), fusion on/off (off = one kernel per gate, the plain method). */
QSE_API int qse_ctx_set_fusion(qse_ctx* ctx, int enabled, int tile_qubits, int max_gates_per_pass);
/* 0 = sequential-rounding-exact CDF (default), 1 = plain parallel scan */
QSE_API int qse_ctx_set_sample_mode(qse_ctx* ctx, int mode);
/* number of kernels this context has launched so far */
QSE_API uint64_t qse_ctx_kernel_launches(const qse_ctx* ctx);
/* Timing on the context's stream (print_steps / benchmarks, like
 * CircuitUnitaryOperationGPU::timedLaunchStart/End, CircuitUnitaryOperationGPU.cu:194-207):
 * record event `slot` (0..63); elapsed milliseconds between two recorded slots. */
QSE_API int qse_ctx_record(qse_ctx* ctx, int slot);
QSE_API int qse_ctx_elapsed(qse_ctx* ctx, int slot_a, int slot_b, float* ms);
/* Per-launch device time of the fused pass kernel: when enabled, every pass
 * launch is bracketed by events on the launching stream; qse_ctx_pass_times
 * returns (and clears) the count and summed milliseconds. */
QSE_API int qse_ctx_time_passes(qse_ctx* ctx, int enabled);
QSE_API int qse_ctx_pass_times(qse_ctx* ctx, uint64_t* launches, double* total_ms);
/* the same, one duration per launch in launch order (up to cap of them);
 * *count receives the number recorded; the record is cleared */
QSE_API int qse_ctx_pass_time_list(qse_ctx* ctx, double* ms, size_t cap, size_t* count);

/* ---- state vector ---------------------------------------------------- */
/* StateVector::StateVector (StateVector.cpp:14-32): 2^n amplitudes, |0..0>. Device-resident. */
QSE_API int qse_state_create(qse_ctx* ctx, uint32_t nqubits, qse_state** out);
QSE_API int qse_state_destroy(qse_state* st);
QSE_API uint32_t qse_state_qubits(const qse_state* st);
/* StateVector::reset (StateVector.cpp:34-46) + Circuit::reset's markHostDirty (Circuit.cpp:127-133) */
QSE_API int qse_state_reset(qse_state* st);
/* ensureOnDevice's H2D copy (CircuitUnitaryOperationGPU.cu:158-180): host = 2^n interleaved complex128 */
QSE_API int qse_state_upload(qse_state* st, const double* host);
/* flush()'s D2H copy (CircuitUnitaryOperationGPU.cu:182-188), in logical qubit order */
QSE_API int qse_state_download(qse_state* st, double* host);
/* logical amplitudes [first, first+count) only (StateVector::printState reads 32) */
QSE_API int qse_state_download_range(qse_state* st, uint64_t first, uint64_t count, double* host);
/* device pointer of the physical amplitude array (valid until the next call on st) */
QSE_API int qse_state_device_ptr(qse_state* st, void** dptr);
/* current logical->physical qubit map (SWAP relabelling); map has nqubits entries */
QSE_API int qse_state_qubit_map(const qse_state* st, uint32_t* map);
/* apply the pending qubit relabelling physically so logical == physical */
QSE_API int qse_state_canonicalize(qse_state* st);

/* ---- one kernel per gate: ICircuitUnitaryOperation::apply* (ICircuitUnitaryOperation.h:19-31) ---- */
QSE_API int qse_apply_gate2x2(qse_state* st, const double m[8], uint32_t q);                /* applyGate     :19 */
QSE_API int qse_apply_cnot(qse_state* st, uint32_t control, uint32_t target);                /* applyCNOT     :20 */
QSE_API int qse_apply_x(qse_state* st, uint32_t q);                                          /* applyPauliX   :21 */
QSE_API int qse_apply_y(qse_state* st, uint32_t q);                                          /* applyPauliY   :22 */
QSE_API int qse_apply_z(qse_state* st, uint32_t q);                                          /* applyPauliZ   :23 */
QSE_API int qse_apply_phase(qse_state* st, uint32_t q, double theta);                        /* applyPhase    :24 */
QSE_API int qse_apply_rx(qse_state* st, uint32_t q, double theta);                           /* applyRotateX  :25 */
QSE_API int qse_apply_ry(qse_state* st, uint32_t q, double theta);                           /* applyRotateY  :26 */
QSE_API int qse_apply_rz(qse_state* st, uint32_t q, double theta);                           /* applyRotateZ  :27 */
QSE_API int qse_apply_h(qse_state* st, uint32_t q);                                          /* applyHadamard :28 */
QSE_API int qse_apply_cphase(qse_state* st, uint32_t control, uint32_t target, double theta);/* applyCPhase   :29 */
QSE_API int qse_apply_mcphase(qse_state* st, const uint32_t* controls, size_t ncontrols,
                              uint32_t target, double theta);                                /* applyMCPhase  :30 */
QSE_API int qse_apply_swap(qse_state* st, uint32_t q0, uint32_t q1);                         /* applySwap     :31 */

/* ---- Circuit::execute (Circuit.cpp:64-120) through the fusion planner ----
 * Replays ops in order (parameters bound from params when op.param >= 0).
 * With noise->enabled, draws the Noise::accumulateError decisions for every
 * gate in order and applies the odd-count X/Z at the end (Noise.cpp:21-44).
 * injected_uniforms: QSE_RNG_INJECTED only, 2 per noisy gate (host memory). */
typedef struct qse_noise qse_noise;
QSE_API int qse_noise_create(qse_ctx* ctx, uint32_t nqubits, const qse_noise_config* cfg, qse_noise** out);
QSE_API int qse_noise_destroy(qse_noise* nz);
/* Noise::resetStats (Noise.cpp:46-50): counts to zero; the draw stream continues */
QSE_API int qse_noise_reset_stats(qse_noise* nz);
/* bit- and phase-flip counts per qubit (Noise::bitFlipCounts / phaseFlipCounts) */
QSE_API int qse_noise_counts(qse_noise* nz, int32_t* bit_counts, int32_t* phase_counts);

QSE_API int qse_execute(qse_state* st, const qse_op* ops, size_t nops,
                        const double* params, size_t nparams,
                        qse_noise* noise, const double* injected_uniforms, size_t n_uniforms,
                        qse_exec_stats* stats);
/* Circuit::execute over a gate list that also holds mid-circuit QSE_GATE_MEASURE
 * and QSE_GATE_RESET_QUBIT gates (GateType::MEASURE / RESET_QUBIT, Structurs.h:10,
 * which the reference's execute loop does not run): the gates between two such
 * gates run fused as in qse_execute; a MEASURE on `target` writes its outcome to
 * results[control] (GateCommand::resultIdx, Structurs.h:18); RESET_QUBIT resets
 * `target`.  uniforms: one draw per MEASURE / RESET_QUBIT gate, in program order. */
QSE_API int qse_execute_mid(qse_state* st, const qse_op* ops, size_t nops, const double* params, size_t nparams,
                            const double* uniforms, size_t n_uniforms, int32_t* results, size_t n_results);

/* Planner introspection (no device work, no GPU needed): JSON description of
 * the passes the fusion planner forms for ops on an n-qubit state with
 * tile_qubits (0 = default 12) and max_gates_per_pass (0 = none) -- per pass
 * the tile qubits and the source-gate order, each gate as given.  qse_execute
 * plans the same way, and in addition caps specialised passes at 256
 * non-diagonal gates and plans each CNOT(c,t) RZ(t) CNOT(c,t) as one diagonal
 * phase, so its pass count can differ.  Writes at most buflen bytes
 * (NUL-terminated); *needed receives the full length + 1. */
QSE_API int qse_plan_describe(uint32_t nqubits, const qse_op* ops, size_t nops, const double* params,
                              size_t nparams, uint32_t tile_qubits, uint32_t max_gates_per_pass,
                              char* buf, size_t buflen, size_t* needed);

/* Pass kernels: 1 (default) = each planned pass is specialised into its own
 * kernel and compiled for sm_100a at run time (cached by source); 0 = one
 * generic kernel interprets the pass program; 2 = specialised, and forward
 * read+write passes over at least 2^10 tiles run as a persistent streamed
 * kernel (one CTA per SM, tiles arriving in shared memory by bulk async copies
 * while two thread groups compute). */
QSE_API int qse_ctx_set_jit(qse_ctx* ctx, int enabled);
/* Generates and compiles (no GPU needed, nothing loaded) every distinct pass
 * kernel the planner makes for ops: nstates 1 = forward passes, 2 = adjoint
 * reverse passes, 3 = forward passes as streamed kernels where a pass allows
 * it (qse_ctx_set_jit mode 2).  *source_bytes receives the total generated
 * source size. */
QSE_API int qse_plan_compile(uint32_t nqubits, const qse_op* ops, size_t nops, const double* params,
                             size_t nparams, uint32_t tile_qubits, int nstates, size_t* source_bytes);

/* ---- StateVector::sample / measure (StateVector.cpp:77-156), on the device ----
 * Outcome = first index i whose inclusive cumulative probability (summed in
 * index order with FP64 rounding after every addition, exactly as the
 * reference's sequential loop) is >= u*total.  uniforms: host array of
 * nshots values in [0,1), or NULL to draw them from Philox(seed).
 * Results are logical basis indices. */
QSE_API int qse_sample(qse_state* st, const double* uniforms, size_t nshots, uint64_t seed,
                       uint64_t* out_indices);
/* Device-resident variant: d_uniforms (or NULL for Philox(seed)) and d_out are
 * device pointers; enqueued on the context stream, no host synchronisation. */
QSE_API int qse_sample_device(qse_state* st, const double* d_uniforms, size_t nshots, uint64_t seed,
                              uint64_t* d_out);
/* measure(): outcome for uniform u, then collapse to |outcome> (amplitude 1, all others 0) */
QSE_API int qse_measure(qse_state* st, double u, uint64_t* out_index);
/* StateVector::measureQubit (StateVector.cpp:158-185): prob1 = sum of |a_i|^2 over
 * the basis states with the qubit set; outcome = (u < prob1); amplitudes of the
 * other outcome become 0 and the rest are divided by sqrt(its probability).
 * u in [0,1) stands in for the reference's random_device draw.  prob1 may be NULL. */
QSE_API int qse_measure_qubit(qse_state* st, uint32_t qubit, double u, int32_t* outcome, double* prob1);
/* StateVector::resetQubit (StateVector.cpp:187-221): the same draw, then the
 * outcome's amplitudes (renormalised) move to the qubit-0 half and the qubit is
 * left in |0>.  outcome and prob1 may be NULL. */
QSE_API int qse_reset_qubit(qse_state* st, uint32_t qubit, double u, int32_t* outcome, double* prob1);
/* Diagnostics of the exact cumulative scan on the current state: out = {spans
 * of blocks composed in parallel, blocks handled on their own (no fold on the
 * running sum's binade, or the sum leaves it inside the block), blocks folded
 * element by element, blocks}.  Reruns the scan. */
QSE_API int qse_sampler_stats(qse_state* st, uint32_t out[4]);
/* total probability as the reference's sequential loop rounds it */
QSE_API int qse_total_probability(qse_state* st, double* total);

/* ---- differentiation (no reference counterpart) ---- */
/* <psi|O|psi> for the current state */
QSE_API int qse_expectation(qse_state* st, const qse_observable* obs, double* value);
/* <psi|O|psi> like qse_expectation, for callers that cannot allocate memory at
 * the point of the call (a locked or exhausted allocator, an embedding that
 * forbids allocation after start-up).  It allocates nothing, device or host:
 * its scratch is a fixed 64 KiB device array inside the library, so it takes
 * at most 2048 observable terms (more: QSE_ERR_SIZE).  All calls on a device
 * share that array, so calls that run at the same time race: calls from
 * several host threads (on one context or several) and calls whose GPU work
 * overlaps.  The call is synchronous (it returns once the value is on the
 * host), so it cannot be made during a stream capture.  No counterpart in the
 * reference (it has no observables). */
QSE_API int qse_expectation_noalloc(qse_state* st, const qse_observable* obs, double* value);
/* Runs ops from |0..0> into st, then the adjoint sweep: grad[p] = d<O>/d params[p].
 * Parameterised types: RX, RY, RZ, PHASE, CPHASE, MCPHASE. */
QSE_API int qse_adjoint(qse_state* st, const qse_op* ops, size_t nops,
                        const double* params, size_t nparams,
                        const qse_observable* obs, double* value, double* grad);

/* ---- batched forward + adjoint of many small circuits (no reference counterpart) ---- */
typedef struct qse_batch qse_batch;
typedef struct qse_batch_circuit {
    uint32_t      nqubits;      /* 4..26 */
    size_t        nops;
    const qse_op* ops;          /* param indices are local to the circuit */
    size_t        nparams;
    qse_observable obs;
} qse_batch_circuit;
QSE_API int qse_batch_create(qse_ctx* ctx, const qse_batch_circuit* circuits, size_t ncircuits,
                             qse_batch** out);
QSE_API int qse_batch_destroy(qse_batch* b);
/* params: concatenation of every circuit's params; values[c], grads: concatenated like params */
QSE_API int qse_batch_run(qse_batch* b, const double* params, double* values, double* grads);
/* device-resident variant: d_params / d_values / d_grads are device pointers; no host copies, no sync */
QSE_API int qse_batch_run_device(qse_batch* b, const double* d_params, double* d_values, double* d_grads);
QSE_API int qse_batch_total_params(const qse_batch* b, size_t* n);
/* Times candidate configurations on this batch (block shape / tile qubits, gates
 * fused per pass, how many tiles a circuit may have and still run start to end
 * in one CTA) with the parameters of the last run (zeros before the first) and
 * keeps the fastest.  cache_path (may be NULL): a JSON file of earlier results,
 * keyed by the batch's structure and the device; read first, updated after. */
QSE_API int qse_batch_autotune(qse_batch* b, const char* cache_path);
/* 1 (default): every run replays one CUDA graph [reset counters, bind angles,
 * persistent kernel, reductions]; 0: the same launches issued one by one. */
QSE_API int qse_batch_use_graph(qse_batch* b, int enabled);

typedef struct qse_batch_config {
    uint32_t threads;       /* CTA size, a power of two in 32..512                       */
    uint32_t reg_bits;      /* 2^reg_bits amplitudes per thread: 2 or 3                   */
                            /* tile qubits k = log2(threads) + reg_bits                   */
    uint32_t max_gates;     /* non-diagonal gates per pass, 0 = no cap                    */
    uint32_t chain_tiles;   /* circuits with at most this many tiles per pass run as one
                               work item (one CTA, start to end); >= 1                    */
    uint32_t ctas_per_sm;   /* persistent CTAs per SM, 0 = as many as fit                 */
    uint32_t grad_slots;    /* gradient slots per pass, 0 = no cap                        */
    uint32_t wide_regs;     /* 1: up to 255 registers per thread (threads <= 256, one CTA
                               per SM); 0: 128 registers (two CTAs of 256 per SM)         */
} qse_batch_config;
QSE_API int qse_batch_set_config(qse_batch* b, const qse_batch_config* cfg);
/* Bound of the persistent kernel's dependency waits: a work item polls the
 * completion counter of the pass it depends on at most `polls` times (with
 * back-off) before it gives up; then every CTA stops claiming work and the run
 * returns QSE_ERR_TIMEOUT (results invalid, the batch stays usable).
 * 0 restores the default (2^21 polls, about a second).  No reference
 * counterpart (failure detection of the batched kernel). */
QSE_API int qse_batch_set_wait_limit(qse_batch* b, uint32_t polls);
QSE_API int qse_batch_get_config(const qse_batch* b, qse_batch_config* cfg);

typedef struct qse_batch_stats {
    uint64_t passes;        /* planned passes, forward + reverse, all circuits            */
    uint64_t items;         /* work-queue entries of one run                              */
    uint64_t tile_visits;   /* (pass, tile) pairs processed per run                       */
    uint64_t hbm_bytes;     /* algorithmic HBM bytes of one run: 32 B per amplitude per
                               forward pass and 64 B per reverse pass of circuits that
                               span several tiles (single-tile circuits stay on chip)     */
    uint64_t occurrences;   /* parameterised gate occurrences (gradient slots)            */
    uint32_t grid;          /* persistent CTAs                                            */
    uint32_t smem_bytes;    /* dynamic shared memory per CTA                              */
    double   last_ms;       /* device time of the last run (0 if none)                    */
    double   plan_ms;       /* host time of the last planning                             */
} qse_batch_stats;
QSE_API int qse_batch_get_stats(qse_batch* b, qse_batch_stats* out);

#ifdef __cplusplus
}
#endif
#endif /* QSE_B200_H */
