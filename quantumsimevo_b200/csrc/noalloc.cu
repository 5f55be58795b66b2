// noalloc.cu -- <psi|O|psi> without any allocation.
//
// qse_expectation reserves its scratch (the observable's term table and the
// per-block partial sums) in context buffers that grow with cudaMalloc, and
// stages results through pinned host memory (cudaMallocHost).  Some callers
// cannot allocate at that point: code running while a memory pool or
// allocator is locked or exhausted, a caller that has handed all device
// memory to its own allocator, or an embedding that forbids allocation after
// initialisation.  qse_expectation_noalloc gives them the same value with the
// scratch in a fixed file-scope device array instead.
//
// Limits and sharing:
//   - kNoAllocBytes = 64 KiB per device, held from library load until exit;
//     at most kMaxTerms (2048) observable terms and kMaxBlocks (4096) partial
//     sums fit, larger observables are rejected with QSE_ERR_SIZE;
//   - every call on a device shares the array: a call writes all the partial
//     sums it reads and the term table it uses, so nothing has to start at
//     zero, but any two calls on one device that run at the same time race on
//     it: calls from several host threads (on one context or several), and
//     calls whose GPU work overlaps (other streams, other contexts);
//   - the call is synchronous: it returns after its result has reached the
//     host (it waits on the context's stream), so it cannot be made while the
//     context's stream is being captured into a graph;
//   - the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (the host-side name of a __device__ array is not a
//     device address).
#include <cuda_runtime.h>

#include <mutex>

#include "qse_internal.h"

namespace qse {
namespace {

constexpr size_t kNoAllocBytes = 64 * 1024;
constexpr uint32_t kMaxTerms = 2048;   // 2048 x (8 B mask + 8 B weight) = 32 KiB
constexpr uint32_t kMaxBlocks = 4096;  // 4096 x 8 B partial sums = 32 KiB, the last slot also holds the total
constexpr int kThreads = 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_mu;
void* g_scratch_dev[64] = {nullptr};

// device address of g_noalloc_scratch on the current device (looked up once per device)
char* scratch_address(int device)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (device < 0 || device >= 64) fail(QSE_ERR_INVALID, "device index out of range");
    if (!g_scratch_dev[device]) {
        void* p = nullptr;
        QSE_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_scratch_dev[device] = p;
    }
    return static_cast<char*>(g_scratch_dev[device]);
}

// partial[b] = sum over the block's amplitudes of O(x)|psi_x|^2; the term
// table (at most kMaxTerms entries, 32 KiB) is staged in static shared memory
// once per block, as qse_expectation's kernel does, so the inner loop over
// the terms reads shared memory instead of global memory
__global__ void __launch_bounds__(kThreads) k_expect_noalloc(const double2* __restrict__ psi, uint64_t size,
                                                             const uint64_t* __restrict__ z,
                                                             const double* __restrict__ w, uint32_t nt, double c,
                                                             double* __restrict__ partial)
{
    __shared__ double sh[kThreads / 32];
    __shared__ uint64_t sz[kMaxTerms];
    __shared__ double sw[kMaxTerms];
    for (uint32_t t = threadIdx.x; t < nt; t += blockDim.x) { sz[t] = z[t]; sw[t] = w[t]; }
    __syncthreads();
    double acc = 0.0;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < size; i += uint64_t(gridDim.x) * blockDim.x) {
        const double2 v = psi[i];
        double o = c;
        for (uint32_t t = 0; t < nt; ++t) o += (__popcll(i & sz[t]) & 1) ? -sw[t] : sw[t];
        acc += o * (v.x * v.x + v.y * v.y);
    }
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < kThreads / 32; ++k) t += sh[k];
        partial[blockIdx.x] = t;
    }
}

// out = sum of n partial sums, in a fixed order (one block)
__global__ void __launch_bounds__(kThreads) k_sum_noalloc(const double* __restrict__ partial, uint32_t n,
                                                          double* __restrict__ out)
{
    __shared__ double sh[kThreads];
    double acc = 0.0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) acc += partial[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if (int(threadIdx.x) < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

}  // namespace

double expectation_noalloc(qse_state* st, const qse_observable* obs)
{
    materialize(st);
    qse_ctx* ctx = st->ctx;
    if (obs->nterms > kMaxTerms)
        fail(QSE_ERR_SIZE, "qse_expectation_noalloc: at most " + std::to_string(kMaxTerms) + " observable terms");
    char* base = scratch_address(ctx->device);
    uint64_t* d_z = reinterpret_cast<uint64_t*>(base);
    double* d_w = reinterpret_cast<double*>(base + 8 * kMaxTerms);
    double* d_part = reinterpret_cast<double*>(base + 16 * kMaxTerms);
    double* d_total = d_part + (kMaxBlocks - 1);

    // terms in physical qubits, copied in fixed-size pieces from a stack buffer
    constexpr uint32_t kChunk = 128;
    uint64_t hz[kChunk];
    double hw[kChunk];
    for (uint32_t t0 = 0; t0 < obs->nterms; t0 += kChunk) {
        const uint32_t cnt = std::min<uint32_t>(kChunk, uint32_t(obs->nterms) - t0);
        for (uint32_t i = 0; i < cnt; ++i) {
            uint64_t m = obs->zmask[t0 + i], pm = 0;
            if (st->n < 64 && (m >> st->n) != 0) fail(QSE_ERR_QUBIT, "observable acts on a qubit out of range");
            for (; m; m &= m - 1) pm |= uint64_t(1) << st->perm[__builtin_ctzll(m)];
            hz[i] = pm;
            hw[i] = obs->weight[t0 + i];
        }
        QSE_CUDA(cudaMemcpyAsync(d_z + t0, hz, cnt * 8, cudaMemcpyHostToDevice, ctx->stream));
        QSE_CUDA(cudaMemcpyAsync(d_w + t0, hw, cnt * 8, cudaMemcpyHostToDevice, ctx->stream));
        QSE_CUDA(cudaStreamSynchronize(ctx->stream));  // hz / hw are reused for the next piece
    }
    const uint64_t size = st->size();
    const uint32_t blocks = uint32_t(std::min<uint64_t>(
        std::min<uint64_t>((size + kThreads - 1) / kThreads, uint64_t(ctx->num_sms) * 8), kMaxBlocks - 1));
    k_expect_noalloc<<<blocks, kThreads, 0, ctx->stream>>>(reinterpret_cast<const double2*>(st->amp), size, d_z, d_w,
                                                          uint32_t(obs->nterms), obs->constant, d_part);
    QSE_CUDA(cudaGetLastError());
    k_sum_noalloc<<<1, kThreads, 0, ctx->stream>>>(d_part, blocks, d_total);
    QSE_CUDA(cudaGetLastError());
    count_launch(ctx, 2);
    double value = 0.0;
    QSE_CUDA(cudaMemcpyAsync(&value, d_total, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    QSE_CUDA(cudaStreamSynchronize(ctx->stream));
    return value;
}

}  // namespace qse
