// capi.cpp -- the extern "C" surface of libqse_b200.so (include/qse_b200.h).
// Every entry point converts exceptions to status codes; none aborts.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <set>
#include <string>

#include "jit.h"
#include "planner.h"
#include "qse_internal.h"

namespace qse {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string& msg) { g_last_error = msg; }

[[noreturn]] void fail(int status, const std::string& msg) { throw Error(status, msg); }

void cuda_check(cudaError_t e, const char* what, const char* file, int line)
{
    if (e == cudaSuccess) return;
    cudaGetLastError();  // clear a sticky-free error so later calls are not poisoned
    char buf[512];
    std::snprintf(buf, sizeof(buf), "CUDA error %s (%d) in %s at %s:%d", cudaGetErrorString(e), int(e), what, file, line);
    if (e == cudaErrorMemoryAllocation) throw Error(QSE_ERR_OOM, buf);
    throw Error(QSE_ERR_CUDA, buf);
}

void DevBuf::reserve(size_t n)
{
    if (n <= bytes) return;
    release();
    size_t want = n + n / 4 + 256;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        e = cudaMalloc(&p, n);
        if (e != cudaSuccess) cuda_check(e, "cudaMalloc(scratch)", __FILE__, __LINE__);
        want = n;
    }
    ptr = p;
    bytes = want;
}

void DevBuf::release()
{
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

void HostBuf::reserve(size_t n)
{
    if (n <= bytes) return;
    release();
    size_t want = n + n / 4 + 256;
    void* p = nullptr;
    QSE_CUDA(cudaMallocHost(&p, want));
    ptr = p;
    bytes = want;
}

void HostBuf::release()
{
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
}

void apply_single(qse_state* st, const qse_op& op);
void download_logical(qse_state* st, double* host);
void download_range(qse_state* st, uint64_t first, uint64_t count, double* host);

}  // namespace qse

using qse::Error;

#define QSE_GUARD_BEGIN try {
#define QSE_GUARD_END                                   \
    }                                                   \
    catch (const qse::Error& e)                         \
    {                                                   \
        qse::g_last_error = e.what();                   \
        return e.status;                                \
    }                                                   \
    catch (const std::bad_alloc&)                       \
    {                                                   \
        qse::g_last_error = "host allocation failed";   \
        return QSE_ERR_OOM;                             \
    }                                                   \
    catch (const std::exception& e)                     \
    {                                                   \
        qse::g_last_error = e.what();                   \
        return QSE_ERR_INVALID;                         \
    }                                                   \
    return QSE_OK;

namespace {

void need(bool cond, int status, const char* msg)
{
    if (!cond) qse::fail(status, msg);
}

void bind_device(const qse_ctx* ctx) { QSE_CUDA(cudaSetDevice(ctx->device)); }

qse_op make_op(int type, uint32_t t, uint32_t c, double theta)
{
    qse_op op{};
    op.type = type;
    op.target = t;
    op.control = c;
    op.param = -1;
    op.theta = theta;
    return op;
}

int apply_one(qse_state* st, const qse_op& op)
{
    QSE_GUARD_BEGIN
    need(st != nullptr, QSE_ERR_INVALID, "null state");
    bind_device(st->ctx);
    qse::apply_single(st, op);
    QSE_GUARD_END
}

}  // namespace

extern "C" {

const char* qse_last_error(void) { return qse::g_last_error.c_str(); }
const char* qse_version(void) { return "qse_b200 0.1 (sm_100a)"; }

int qse_ctx_create(int device, qse_ctx** out)
{
    QSE_GUARD_BEGIN
    need(out != nullptr, QSE_ERR_INVALID, "null output pointer");
    int count = 0;
    QSE_CUDA(cudaGetDeviceCount(&count));
    need(device >= 0 && device < count, QSE_ERR_INVALID, "no such CUDA device");
    QSE_CUDA(cudaSetDevice(device));
    auto* ctx = new qse_ctx;
    ctx->device = device;
    QSE_CUDA(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device));
    int optin = 0;
    QSE_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    ctx->smem_optin = size_t(optin);
    QSE_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    QSE_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&ctx->status_host), 16, cudaHostAllocMapped));
    *reinterpret_cast<volatile unsigned*>(ctx->status_host) = 0u;
    QSE_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void**>(&ctx->status_dev), ctx->status_host, 0));
    QSE_CUDA(cudaEventCreateWithFlags(&ctx->plan_event, cudaEventDisableTiming));
    QSE_CUDA(cudaEventRecord(ctx->plan_event, ctx->stream));
    *out = ctx;
    QSE_GUARD_END
}

int qse_ctx_destroy(qse_ctx* ctx)
{
    QSE_GUARD_BEGIN
    if (!ctx) return QSE_OK;
    bind_device(ctx);
    cudaStreamSynchronize(ctx->stream);
    qse::destroy_compact_state(ctx);
    qse::destroy_plan_cache(ctx);
    ctx->plan_buf.release();
    ctx->scratch.release();
    ctx->scratch2.release();
    ctx->gv_buf.release();
    ctx->plan_host.release();
    ctx->host_small.release();
    ctx->host_small2.release();
    if (ctx->plan_event) cudaEventDestroy(ctx->plan_event);
    for (cudaEvent_t e : ctx->slots)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->pass_events) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->status_host) cudaFreeHost(ctx->status_host);
    delete ctx;
    QSE_GUARD_END
}

int qse_ctx_synchronize(qse_ctx* ctx)
{
    QSE_GUARD_BEGIN
    need(ctx != nullptr, QSE_ERR_INVALID, "null context");
    bind_device(ctx);
    QSE_CUDA(cudaStreamSynchronize(ctx->stream));
    qse::check_device_status(ctx);
    QSE_GUARD_END
}

int qse_ctx_set_fusion(qse_ctx* ctx, int enabled, int tile_qubits, int max_gates_per_pass)
{
    QSE_GUARD_BEGIN
    need(ctx != nullptr, QSE_ERR_INVALID, "null context");
    need(tile_qubits == 0 || (tile_qubits >= 4 && tile_qubits <= 12), QSE_ERR_INVALID, "tile_qubits must be 4..12");
    need(max_gates_per_pass >= 0, QSE_ERR_INVALID, "max_gates_per_pass must be >= 0");
    ctx->fusion = enabled ? 1 : 0;
    if (tile_qubits) ctx->tile_qubits = tile_qubits;
    ctx->max_gates_per_pass = max_gates_per_pass;
    QSE_GUARD_END
}

int qse_ctx_set_sample_mode(qse_ctx* ctx, int mode)
{
    QSE_GUARD_BEGIN
    need(ctx != nullptr, QSE_ERR_INVALID, "null context");
    need(mode == 0, QSE_ERR_UNSUPPORTED, "only the sequential-rounding-exact sampler (mode 0) is built");
    ctx->sample_mode = mode;
    QSE_GUARD_END
}

uint64_t qse_ctx_kernel_launches(const qse_ctx* ctx) { return ctx ? ctx->launches : 0; }

int qse_ctx_record(qse_ctx* ctx, int slot)
{
    QSE_GUARD_BEGIN
    need(ctx != nullptr && slot >= 0 && slot < 64, QSE_ERR_INVALID, "bad context or slot");
    bind_device(ctx);
    if (!ctx->slots[slot]) QSE_CUDA(cudaEventCreate(&ctx->slots[slot]));
    QSE_CUDA(cudaEventRecord(ctx->slots[slot], ctx->stream));
    QSE_GUARD_END
}

int qse_ctx_elapsed(qse_ctx* ctx, int a, int b, float* ms)
{
    QSE_GUARD_BEGIN
    need(ctx && ms && a >= 0 && a < 64 && b >= 0 && b < 64, QSE_ERR_INVALID, "bad argument");
    need(ctx->slots[a] && ctx->slots[b], QSE_ERR_STATE, "slot never recorded");
    bind_device(ctx);
    QSE_CUDA(cudaEventSynchronize(ctx->slots[b]));
    QSE_CUDA(cudaEventElapsedTime(ms, ctx->slots[a], ctx->slots[b]));
    QSE_GUARD_END
}

int qse_ctx_time_passes(qse_ctx* ctx, int enabled)
{
    QSE_GUARD_BEGIN
    need(ctx != nullptr, QSE_ERR_INVALID, "null context");
    ctx->time_passes = enabled != 0;
    QSE_GUARD_END
}

int qse_ctx_pass_times(qse_ctx* ctx, uint64_t* launches, double* total_ms)
{
    QSE_GUARD_BEGIN
    need(ctx && launches && total_ms, QSE_ERR_INVALID, "null argument");
    bind_device(ctx);
    QSE_CUDA(cudaStreamSynchronize(ctx->stream));
    double t = 0.0;
    for (size_t i = 0; i + 1 < ctx->pass_events_used; i += 2) {
        float ms = 0.f;
        QSE_CUDA(cudaEventElapsedTime(&ms, ctx->pass_events[i], ctx->pass_events[i + 1]));
        t += ms;
    }
    *launches = ctx->pass_events_used / 2;
    *total_ms = t;
    ctx->pass_events_used = 0;
    QSE_GUARD_END
}

int qse_ctx_pass_time_list(qse_ctx* ctx, double* ms, size_t cap, size_t* count)
{
    QSE_GUARD_BEGIN
    need(ctx && count && (cap == 0 || ms), QSE_ERR_INVALID, "null argument");
    bind_device(ctx);
    QSE_CUDA(cudaStreamSynchronize(ctx->stream));
    const size_t n = ctx->pass_events_used / 2;
    *count = n;
    for (size_t i = 0; i < n && i < cap; ++i) {
        float t = 0.f;
        QSE_CUDA(cudaEventElapsedTime(&t, ctx->pass_events[2 * i], ctx->pass_events[2 * i + 1]));
        ms[i] = t;
    }
    ctx->pass_events_used = 0;
    QSE_GUARD_END
}

int qse_state_create(qse_ctx* ctx, uint32_t nqubits, qse_state** out)
{
    QSE_GUARD_BEGIN
    need(ctx != nullptr && out != nullptr, QSE_ERR_INVALID, "null argument");
    need(nqubits >= 1 && nqubits <= 36, QSE_ERR_SIZE, "qubit count must be 1..36");
    bind_device(ctx);
    auto* st = new qse_state;
    st->ctx = ctx;
    st->n = nqubits;
    for (uint32_t q = 0; q < 64; ++q) st->perm[q] = q;
    cudaError_t e = cudaMalloc(&st->amp, st->size() * 16);
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete st;
        qse::fail(QSE_ERR_OOM, "device allocation of the state vector failed (" + std::to_string(nqubits) + " qubits)");
    }
    // |0..0> recorded, not written: the first execute's first pass generates
    // it, every other reader writes it first (materialize)
    qse::mark_zero(st);
    *out = st;
    QSE_GUARD_END
}

int qse_state_destroy(qse_state* st)
{
    QSE_GUARD_BEGIN
    if (!st) return QSE_OK;
    bind_device(st->ctx);
    cudaStreamSynchronize(st->ctx->stream);
    if (st->amp) cudaFree(st->amp);
    if (st->aux) cudaFree(st->aux);
    delete st;
    QSE_GUARD_END
}

uint32_t qse_state_qubits(const qse_state* st) { return st ? st->n : 0; }

int qse_state_reset(qse_state* st)
{
    QSE_GUARD_BEGIN
    need(st != nullptr, QSE_ERR_INVALID, "null state");
    bind_device(st->ctx);
    // |0..0> without writing 16 B per amplitude: the next fused execute's first
    // pass generates it; any other reader writes it first (materialize)
    qse::mark_zero(st);
    QSE_GUARD_END
}

int qse_state_upload(qse_state* st, const double* host)
{
    QSE_GUARD_BEGIN
    need(st != nullptr && host != nullptr, QSE_ERR_INVALID, "null argument");
    bind_device(st->ctx);
    for (uint32_t q = 0; q < 64; ++q) st->perm[q] = q;
    st->lazy_basis = false;
    st->touch();
    QSE_CUDA(cudaMemcpyAsync(st->amp, host, st->size() * 16, cudaMemcpyHostToDevice, st->ctx->stream));
    QSE_CUDA(cudaStreamSynchronize(st->ctx->stream));
    QSE_GUARD_END
}

int qse_state_download(qse_state* st, double* host)
{
    QSE_GUARD_BEGIN
    need(st != nullptr && host != nullptr, QSE_ERR_INVALID, "null argument");
    bind_device(st->ctx);
    qse::download_logical(st, host);
    qse::check_device_status(st->ctx);
    QSE_GUARD_END
}

int qse_state_download_range(qse_state* st, uint64_t first, uint64_t count, double* host)
{
    QSE_GUARD_BEGIN
    need(st != nullptr && (host != nullptr || count == 0), QSE_ERR_INVALID, "null argument");
    need(first <= st->size() && count <= st->size() - first, QSE_ERR_INVALID, "range outside the state");
    bind_device(st->ctx);
    qse::download_range(st, first, count, host);
    qse::check_device_status(st->ctx);
    QSE_GUARD_END
}

int qse_state_device_ptr(qse_state* st, void** dptr)
{
    QSE_GUARD_BEGIN
    need(st != nullptr && dptr != nullptr, QSE_ERR_INVALID, "null argument");
    qse::materialize(st);
    *dptr = st->amp;
    QSE_GUARD_END
}

int qse_state_qubit_map(const qse_state* st, uint32_t* map)
{
    QSE_GUARD_BEGIN
    need(st != nullptr && map != nullptr, QSE_ERR_INVALID, "null argument");
    for (uint32_t q = 0; q < st->n; ++q) map[q] = st->perm[q];
    QSE_GUARD_END
}

int qse_state_canonicalize(qse_state* st)
{
    QSE_GUARD_BEGIN
    need(st != nullptr, QSE_ERR_INVALID, "null state");
    bind_device(st->ctx);
    qse::canonicalize(st);
    QSE_GUARD_END
}

int qse_apply_gate2x2(qse_state* st, const double m[8], uint32_t q)
{
    if (!m) { qse::g_last_error = "null matrix"; return QSE_ERR_INVALID; }
    qse_op op = make_op(QSE_GATE_2X2, q, 0, 0.0);
    std::memcpy(op.m, m, 8 * sizeof(double));
    return apply_one(st, op);
}
int qse_apply_cnot(qse_state* st, uint32_t control, uint32_t target) { return apply_one(st, make_op(QSE_GATE_CNOT, target, control, 0.0)); }
int qse_apply_x(qse_state* st, uint32_t q) { return apply_one(st, make_op(QSE_GATE_X, q, 0, 0.0)); }
int qse_apply_y(qse_state* st, uint32_t q) { return apply_one(st, make_op(QSE_GATE_Y, q, 0, 0.0)); }
int qse_apply_z(qse_state* st, uint32_t q) { return apply_one(st, make_op(QSE_GATE_Z, q, 0, 0.0)); }
int qse_apply_phase(qse_state* st, uint32_t q, double theta) { return apply_one(st, make_op(QSE_GATE_PHASE, q, 0, theta)); }
int qse_apply_rx(qse_state* st, uint32_t q, double theta) { return apply_one(st, make_op(QSE_GATE_RX, q, 0, theta)); }
int qse_apply_ry(qse_state* st, uint32_t q, double theta) { return apply_one(st, make_op(QSE_GATE_RY, q, 0, theta)); }
int qse_apply_rz(qse_state* st, uint32_t q, double theta) { return apply_one(st, make_op(QSE_GATE_RZ, q, 0, theta)); }
int qse_apply_h(qse_state* st, uint32_t q) { return apply_one(st, make_op(QSE_GATE_H, q, 0, 0.0)); }
int qse_apply_cphase(qse_state* st, uint32_t control, uint32_t target, double theta)
{
    return apply_one(st, make_op(QSE_GATE_CPHASE, target, control, theta));
}
int qse_apply_mcphase(qse_state* st, const uint32_t* controls, size_t ncontrols, uint32_t target, double theta)
{
    if (ncontrols && !controls) { qse::g_last_error = "null controls"; return QSE_ERR_INVALID; }
    qse_op op = make_op(QSE_GATE_MCPHASE, target, 0, theta);
    for (size_t i = 0; i < ncontrols; ++i) {
        if (controls[i] >= 64) { qse::g_last_error = "control qubit out of range"; return QSE_ERR_QUBIT; }
        op.controls |= uint64_t(1) << controls[i];
    }
    return apply_one(st, op);
}
int qse_apply_swap(qse_state* st, uint32_t q0, uint32_t q1) { return apply_one(st, make_op(QSE_GATE_SWAP, q0, q1, 0.0)); }

int qse_noise_create(qse_ctx* ctx, uint32_t nqubits, const qse_noise_config* cfg, qse_noise** out)
{
    QSE_GUARD_BEGIN
    need(ctx && cfg && out, QSE_ERR_INVALID, "null argument");
    need(nqubits >= 1 && nqubits <= 64, QSE_ERR_SIZE, "qubit count out of range");
    need(cfg->rng_mode >= 0 && cfg->rng_mode <= 2, QSE_ERR_INVALID, "bad rng mode");
    bind_device(ctx);
    auto* nz = new qse_noise;
    nz->ctx = ctx;
    nz->n = nqubits;
    nz->cfg = *cfg;
    nz->gen.seed(static_cast<std::mt19937::result_type>(static_cast<unsigned int>(cfg->seed)));
    cudaError_t e = cudaMalloc(&nz->d_counts, 128 * 4 + 16 * 8);
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete nz;
        qse::fail(QSE_ERR_OOM, "noise counters allocation failed");
    }
    QSE_CUDA(cudaMemsetAsync(nz->d_counts, 0, 128 * 4, ctx->stream));
    QSE_CUDA(cudaMemcpyAsync(nz->d_counts + 128, cfg->rates, 16 * 8, cudaMemcpyHostToDevice, ctx->stream));
    QSE_CUDA(cudaStreamSynchronize(ctx->stream));
    *out = nz;
    QSE_GUARD_END
}

int qse_noise_destroy(qse_noise* nz)
{
    QSE_GUARD_BEGIN
    if (!nz) return QSE_OK;
    bind_device(nz->ctx);
    cudaStreamSynchronize(nz->ctx->stream);
    if (nz->d_counts) cudaFree(nz->d_counts);
    delete nz;
    QSE_GUARD_END
}

int qse_noise_reset_stats(qse_noise* nz)
{
    QSE_GUARD_BEGIN
    need(nz != nullptr, QSE_ERR_INVALID, "null noise");
    bind_device(nz->ctx);
    QSE_CUDA(cudaMemsetAsync(nz->d_counts, 0, 128 * 4, nz->ctx->stream));
    QSE_CUDA(cudaStreamSynchronize(nz->ctx->stream));
    QSE_GUARD_END
}

int qse_noise_counts(qse_noise* nz, int32_t* bit_counts, int32_t* phase_counts)
{
    QSE_GUARD_BEGIN
    need(nz != nullptr, QSE_ERR_INVALID, "null noise");
    bind_device(nz->ctx);
    int32_t h[128];
    QSE_CUDA(cudaMemcpyAsync(h, nz->d_counts, sizeof(h), cudaMemcpyDeviceToHost, nz->ctx->stream));
    QSE_CUDA(cudaStreamSynchronize(nz->ctx->stream));
    if (bit_counts) std::memcpy(bit_counts, h, nz->n * 4);
    if (phase_counts) std::memcpy(phase_counts, h + 64, nz->n * 4);
    QSE_GUARD_END
}

int qse_execute(qse_state* st, const qse_op* ops, size_t nops, const double* params, size_t nparams,
                qse_noise* noise, const double* injected_uniforms, size_t n_uniforms, qse_exec_stats* stats)
{
    QSE_GUARD_BEGIN
    need(st != nullptr, QSE_ERR_INVALID, "null state");
    need(nops == 0 || ops != nullptr, QSE_ERR_INVALID, "null ops");
    bind_device(st->ctx);
    qse::execute_program(st, ops, nops, params, nparams, noise, injected_uniforms, n_uniforms, stats);
    QSE_GUARD_END
}

int qse_execute_mid(qse_state* st, const qse_op* ops, size_t nops, const double* params, size_t nparams,
                    const double* uniforms, size_t n_uniforms, int32_t* results, size_t n_results)
{
    QSE_GUARD_BEGIN
    need(st != nullptr, QSE_ERR_INVALID, "null state");
    need(nops == 0 || ops != nullptr, QSE_ERR_INVALID, "null ops");
    // validate the measurement layout before anything runs
    size_t nmr = 0;
    for (size_t i = 0; i < nops; ++i) {
        const int t = ops[i].type;
        if (t != QSE_GATE_MEASURE && t != QSE_GATE_RESET_QUBIT) continue;
        need(ops[i].target < st->n, QSE_ERR_QUBIT, "measured qubit out of range");
        if (t == QSE_GATE_MEASURE)
            need(results != nullptr && ops[i].control < n_results, QSE_ERR_INVALID, "result index out of range");
        ++nmr;
    }
    need(nmr <= n_uniforms && (nmr == 0 || uniforms != nullptr), QSE_ERR_INVALID,
         "one uniform per MEASURE / RESET_QUBIT gate is needed");
    for (size_t k = 0; k < nmr; ++k)
        need(uniforms[k] >= 0.0 && uniforms[k] < 1.0, QSE_ERR_INVALID, "uniforms must lie in [0,1)");
    bind_device(st->ctx);
    size_t start = 0, k = 0;
    for (size_t i = 0; i <= nops; ++i) {
        const bool mr = i < nops && (ops[i].type == QSE_GATE_MEASURE || ops[i].type == QSE_GATE_RESET_QUBIT);
        if (!mr && i < nops) continue;
        if (i > start) qse::execute_program(st, ops + start, i - start, params, nparams, nullptr, nullptr, 0, nullptr);
        if (mr) {
            const bool reset = ops[i].type == QSE_GATE_RESET_QUBIT;
            const int outcome = qse::measure_or_reset_qubit(st, ops[i].target, uniforms[k++], reset, nullptr);
            if (!reset) results[ops[i].control] = outcome;
        }
        start = i + 1;
    }
    QSE_GUARD_END
}

int qse_plan_describe(uint32_t nqubits, const qse_op* ops, size_t nops, const double* params, size_t nparams,
                      uint32_t tile_qubits, uint32_t max_gates_per_pass, char* buf, size_t buflen, size_t* needed)
{
    QSE_GUARD_BEGIN
    need(nqubits >= 1 && nqubits <= 40, QSE_ERR_SIZE, "qubit count out of range");
    need(nops == 0 || ops != nullptr, QSE_ERR_INVALID, "null ops");
    std::vector<qse::plan::Gate> gates;
    for (size_t i = 0; i < nops; ++i) {
        qse::plan::Gate g;
        g.type = ops[i].type;
        g.t = ops[i].target;
        g.c = ops[i].control;
        g.cmask = ops[i].controls;
        g.theta = qse::bound_angle(ops[i], params, nparams);
        std::memcpy(g.m, ops[i].m, sizeof(g.m));
        gates.push_back(g);
    }
    uint32_t perm[64];
    for (uint32_t q = 0; q < 64; ++q) perm[q] = q;
    qse::plan::Options opt;
    opt.k = tile_qubits ? tile_qubits : 12;
    opt.max_gates = max_gates_per_pass;
    qse::plan::Plan pl = qse::plan::build(gates, nqubits, perm, opt);
    std::string s = qse::plan::describe(pl);
    if (needed) *needed = s.size() + 1;
    if (buf && buflen) {
        size_t n = std::min(buflen - 1, s.size());
        std::memcpy(buf, s.data(), n);
        buf[n] = '\0';
    }
    QSE_GUARD_END
}

int qse_ctx_set_jit(qse_ctx* ctx, int enabled)
{
    QSE_GUARD_BEGIN
    need(ctx != nullptr, QSE_ERR_INVALID, "null context");
    need(enabled >= 0 && enabled <= 2, QSE_ERR_INVALID, "pass kernel mode must be 0, 1 or 2");
    ctx->jit = enabled;
    QSE_GUARD_END
}

int qse_plan_compile(uint32_t nqubits, const qse_op* ops, size_t nops, const double* params, size_t nparams,
                     uint32_t tile_qubits, int nstates, size_t* source_bytes)
{
    QSE_GUARD_BEGIN
    need(nqubits >= 3 && nqubits <= 40, QSE_ERR_SIZE, "qubit count out of range");
    need(nops == 0 || ops != nullptr, QSE_ERR_INVALID, "null ops");
    need(nstates >= 1 && nstates <= 3, QSE_ERR_INVALID, "nstates must be 1, 2 or 3");
    const bool streamed = nstates == 3;
    if (streamed) nstates = 1;
    std::vector<qse::plan::Gate> gates;
    for (size_t i = 0; i < nops; ++i) {
        size_t k = nstates == 2 ? nops - 1 - i : i;
        qse::plan::Gate g;
        g.type = ops[k].type;
        g.t = ops[k].target;
        g.c = ops[k].control;
        g.cmask = ops[k].controls;
        g.theta = qse::bound_angle(ops[k], params, nparams);
        std::memcpy(g.m, ops[k].m, sizeof(g.m));
        if (nstates == 2 && ops[k].param >= 0) g.grad = int32_t(k);
        gates.push_back(g);
    }
    uint32_t perm[64];
    for (uint32_t q = 0; q < 64; ++q) perm[q] = q;
    qse::plan::Options opt;
    opt.k = std::min<uint32_t>(tile_qubits ? tile_qubits : (nstates == 2 ? 11 : 12), nqubits);
    opt.rb = nstates == 2 ? 3 : (!streamed && opt.k == 12) ? 5 : 4;   // as the engine plans them
    opt.grads = nstates == 2;
    opt.acc_mul = true;
    opt.max_gates = qse::plan::kJitMaxGates;
    if (nstates == 2) opt.max_terms = 512;
    qse::plan::Plan pl = qse::plan::build(gates, nqubits, perm, opt);
    size_t total = 0;
    std::set<std::string> done;   // identical passes share one kernel, as in execution
    for (const auto& p : pl.passes) {
        qse::jit::Source s = qse::jit::generate(p, nstates, false, streamed, nqubits >= qse::jit::kPreGroupQubits);
        total += s.code.size();
        if (done.insert(s.code).second) qse::jit::compile_only(s);
    }
    if (source_bytes) *source_bytes = total;
    QSE_GUARD_END
}

int qse_sample(qse_state* st, const double* uniforms, size_t nshots, uint64_t seed, uint64_t* out_indices)
{
    QSE_GUARD_BEGIN
    need(st != nullptr, QSE_ERR_INVALID, "null state");
    need(nshots == 0 || out_indices != nullptr, QSE_ERR_INVALID, "null output");
    if (uniforms)
        for (size_t i = 0; i < nshots; ++i)
            need(uniforms[i] >= 0.0 && uniforms[i] < 1.0, QSE_ERR_INVALID, "uniforms must lie in [0,1)");
    bind_device(st->ctx);
    qse::sample(st, uniforms, nshots, seed, out_indices);
    qse::check_device_status(st->ctx);
    QSE_GUARD_END
}

int qse_sample_device(qse_state* st, const double* d_uniforms, size_t nshots, uint64_t seed, uint64_t* d_out)
{
    QSE_GUARD_BEGIN
    need(st != nullptr, QSE_ERR_INVALID, "null state");
    need(nshots == 0 || d_out != nullptr, QSE_ERR_INVALID, "null output");
    bind_device(st->ctx);
    qse::sample_device(st, d_uniforms, nshots, seed, d_out);
    QSE_GUARD_END
}

int qse_measure(qse_state* st, double u, uint64_t* out_index)
{
    QSE_GUARD_BEGIN
    need(st != nullptr && out_index != nullptr, QSE_ERR_INVALID, "null argument");
    need(u >= 0.0 && u < 1.0, QSE_ERR_INVALID, "u must lie in [0,1)");
    bind_device(st->ctx);
    *out_index = qse::measure(st, u);
    qse::check_device_status(st->ctx);
    QSE_GUARD_END
}

int qse_measure_qubit(qse_state* st, uint32_t qubit, double u, int32_t* outcome, double* prob1)
{
    QSE_GUARD_BEGIN
    need(st != nullptr && outcome != nullptr, QSE_ERR_INVALID, "null argument");
    need(u >= 0.0 && u < 1.0, QSE_ERR_INVALID, "u must lie in [0,1)");
    bind_device(st->ctx);
    *outcome = qse::measure_or_reset_qubit(st, qubit, u, false, prob1);
    QSE_GUARD_END
}

int qse_reset_qubit(qse_state* st, uint32_t qubit, double u, int32_t* outcome, double* prob1)
{
    QSE_GUARD_BEGIN
    need(st != nullptr, QSE_ERR_INVALID, "null argument");
    need(u >= 0.0 && u < 1.0, QSE_ERR_INVALID, "u must lie in [0,1)");
    bind_device(st->ctx);
    const int o = qse::measure_or_reset_qubit(st, qubit, u, true, prob1);
    if (outcome) *outcome = o;
    QSE_GUARD_END
}

int qse_sampler_stats(qse_state* st, uint32_t out[4])
{
    QSE_GUARD_BEGIN
    need(st != nullptr && out != nullptr, QSE_ERR_INVALID, "null argument");
    bind_device(st->ctx);
    qse::sampler_stats(st, out);
    QSE_GUARD_END
}

int qse_total_probability(qse_state* st, double* total)
{
    QSE_GUARD_BEGIN
    need(st != nullptr && total != nullptr, QSE_ERR_INVALID, "null argument");
    bind_device(st->ctx);
    *total = qse::total_probability(st);
    qse::check_device_status(st->ctx);
    QSE_GUARD_END
}

int qse_expectation(qse_state* st, const qse_observable* obs, double* value)
{
    QSE_GUARD_BEGIN
    need(st && obs && value, QSE_ERR_INVALID, "null argument");
    need(obs->nterms == 0 || (obs->zmask && obs->weight), QSE_ERR_INVALID, "null observable terms");
    bind_device(st->ctx);
    *value = qse::expectation(st, obs);
    qse::check_device_status(st->ctx);
    QSE_GUARD_END
}

int qse_expectation_noalloc(qse_state* st, const qse_observable* obs, double* value)
{
    QSE_GUARD_BEGIN
    need(st && obs && value, QSE_ERR_INVALID, "null argument");
    need(obs->nterms == 0 || (obs->zmask && obs->weight), QSE_ERR_INVALID, "null observable terms");
    bind_device(st->ctx);
    *value = qse::expectation_noalloc(st, obs);
    QSE_GUARD_END
}

int qse_adjoint(qse_state* st, const qse_op* ops, size_t nops, const double* params, size_t nparams,
                const qse_observable* obs, double* value, double* grad)
{
    QSE_GUARD_BEGIN
    need(st && obs && value, QSE_ERR_INVALID, "null argument");
    need(nops == 0 || ops, QSE_ERR_INVALID, "null ops");
    need(nparams == 0 || (params && grad), QSE_ERR_INVALID, "null params / grad");
    need(obs->nterms == 0 || (obs->zmask && obs->weight), QSE_ERR_INVALID, "null observable terms");
    bind_device(st->ctx);
    *value = qse::adjoint(st, ops, nops, params, nparams, obs, grad);
    QSE_GUARD_END
}

}  // extern "C"
