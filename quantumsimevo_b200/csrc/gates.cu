// gates.cu -- one kernel per gate (the "plain method"), state management kernels.
//
// These are the kernels behind ICircuitUnitaryOperation's per-gate entry
// points (ICircuitUnitaryOperation.h:19-31) when the caller drives the backend
// gate by gate, and behind qse_execute when fusion is switched off.  Each is a
// grid-stride loop over the amplitudes a gate touches; the single-qubit pair
// kernels move two adjacent amplitudes per 32-byte load and store, the others
// use 16-byte complex128 accesses; a pair kernel visits only the 2^(n-1) pairs, a diagonal
// kernel only the amplitudes whose mask bits are all set (the reference
// launches 2^n threads and lets most of them idle, CircuitUnitaryOperationGPU.cu:74-117).
#include "qse_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

namespace qse {
namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ uint64_t insert0(uint64_t i, uint32_t q)
{
    return ((i >> q) << (q + 1)) | (i & ((uint64_t(1) << q) - 1));
}

// insert a 1 bit at every set position of `mask` (ascending), expanding i
__device__ __forceinline__ uint64_t insert_ones(uint64_t i, uint64_t mask)
{
    while (mask) {
        uint32_t b = __ffsll((long long)mask) - 1;
        mask &= mask - 1;
        i = insert0(i, b) | (uint64_t(1) << b);
    }
    return i;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Streaming element-wise kernels: one work item per thread over a full grid.
// Blocks are dispatched in index order, so the amplitudes in flight form a
// sliding window through the state; a grid capped at a few blocks per SM with
// a grid-stride loop measured 5-45 % slower on B200 for the same bytes.
unsigned grid_full(uint64_t work)
{
    uint64_t blocks = (work + kBlock - 1) / kBlock;
    if (blocks > 0x7fffffffull) blocks = 0x7fffffffull;
    if (blocks == 0) blocks = 1;
    return unsigned(blocks);
}

unsigned grid_for(const qse_ctx* ctx, uint64_t work)
{
    uint64_t blocks = (work + kBlock - 1) / kBlock;
    uint64_t cap = uint64_t(ctx->num_sms) * 32;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    return unsigned(blocks);
}

// ---- pair kernels: (a[i0], a[i1]) with i1 = i0 | 2^q ----
struct FH {
    __device__ void operator()(double2& v0, double2& v1) const
    {
        const double s = 0.7071067811865475244;
        double2 a = v0, b = v1;
        v0 = make_double2((a.x + b.x) * s, (a.y + b.y) * s);
        v1 = make_double2((a.x - b.x) * s, (a.y - b.y) * s);
    }
};
struct FX {
    __device__ void operator()(double2& v0, double2& v1) const { double2 t = v0; v0 = v1; v1 = t; }
};
struct FY {  // (-i v1, i v0)
    __device__ void operator()(double2& v0, double2& v1) const
    {
        double2 a = v0, b = v1;
        v0 = make_double2(b.y, -b.x);
        v1 = make_double2(-a.y, a.x);
    }
};
struct FRX {  // [[c, -is], [-is, c]]
    double c, s;
    __device__ void operator()(double2& v0, double2& v1) const
    {
        double2 a = v0, b = v1;
        v0 = make_double2(c * a.x + s * b.y, c * a.y - s * b.x);
        v1 = make_double2(s * a.y + c * b.x, -s * a.x + c * b.y);
    }
};
struct FRY {  // [[c, -s], [s, c]]
    double c, s;
    __device__ void operator()(double2& v0, double2& v1) const
    {
        double2 a = v0, b = v1;
        v0 = make_double2(c * a.x - s * b.x, c * a.y - s * b.y);
        v1 = make_double2(s * a.x + c * b.x, s * a.y + c * b.y);
    }
};
struct FRZ {  // diag(p0, p1)
    double2 p0, p1;
    __device__ void operator()(double2& v0, double2& v1) const { v0 = cmul(v0, p0); v1 = cmul(v1, p1); }
};
struct F2x2 {
    double2 g00, g01, g10, g11;
    __device__ void operator()(double2& v0, double2& v1) const
    {
        double2 a = v0, b = v1;
        double2 x = cmul(g00, a), y = cmul(g01, b);
        double2 z = cmul(g10, a), w = cmul(g11, b);
        v0 = make_double2(x.x + y.x, x.y + y.y);
        v1 = make_double2(z.x + w.x, z.y + w.y);
    }
};

template <class F>
__global__ void __launch_bounds__(kBlock) k_pairs(double2* __restrict__ a, uint64_t npairs, uint32_t q, F f)
{
    const uint64_t step = uint64_t(1) << q;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < npairs;
         i += uint64_t(gridDim.x) * blockDim.x) {
        uint64_t i0 = insert0(i, q);
        double2 v0 = a[i0], v1 = a[i0 | step];
        f(v0, v1);
        a[i0] = v0;
        a[i0 | step] = v1;
    }
}

// 32-byte vector access to two adjacent amplitudes (index even: 32-byte aligned)
__device__ __forceinline__ void ld2(const double2* p, double2& x, double2& y)
{
    asm volatile("ld.global.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(x.x), "=d"(x.y), "=d"(y.x), "=d"(y.y) : "l"(p));
}
__device__ __forceinline__ void st2(double2* p, const double2& x, const double2& y)
{
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(x.x), "d"(x.y), "d"(y.x), "d"(y.y)
                 : "memory");
}

// The same pairs, two per thread with 32-byte loads and stores (npairs even):
// thread t takes pair indices 2t and 2t+1.  q = 0: the four amplitudes 4t..4t+3
// are the pairs (4t, 4t+1), (4t+2, 4t+3); q >= 1: i0 = insert0(2t, q) is even,
// so (i0, i0+1) and (i0|2^q, i0|2^q + 1) are two aligned 32-byte halves.  A
// warp still reads and writes contiguous 1 KiB spans; half the memory
// instructions of k_pairs, the same arithmetic.
template <class F>
__global__ void __launch_bounds__(kBlock) k_pairs2(double2* __restrict__ a, uint64_t nquads, uint32_t q, F f)
{
    const uint64_t step = uint64_t(1) << q;
    for (uint64_t t = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; t < nquads;
         t += uint64_t(gridDim.x) * blockDim.x) {
        double2 v0, v1, w0, w1;
        if (q == 0) {
            double2* p = a + 4 * t;
            ld2(p, v0, v1);
            ld2(p + 2, w0, w1);
            f(v0, v1);
            f(w0, w1);
            st2(p, v0, v1);
            st2(p + 2, w0, w1);
        } else {
            const uint64_t i0 = insert0(2 * t, q);
            ld2(a + i0, v0, w0);
            ld2(a + (i0 | step), v1, w1);
            f(v0, v1);
            f(w0, w1);
            st2(a + i0, v0, w0);
            st2(a + (i0 | step), v1, w1);
        }
    }
}

// Pairs on target t restricted to control bit c = 1 (CNOT): 2^(n-2) pairs.
template <class F>
__global__ void __launch_bounds__(kBlock) k_cpairs(double2* __restrict__ a, uint64_t npairs, uint32_t c,
                                                   uint32_t t, F f)
{
    const uint32_t lo = c < t ? c : t, hi = c < t ? t : c;
    const uint64_t cm = uint64_t(1) << c, tm = uint64_t(1) << t;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < npairs;
         i += uint64_t(gridDim.x) * blockDim.x) {
        uint64_t i0 = insert0(insert0(i, lo), hi) | cm;
        double2 v0 = a[i0], v1 = a[i0 | tm];
        f(v0, v1);
        a[i0] = v0;
        a[i0 | tm] = v1;
    }
}

// Multiply every amplitude whose `mask` bits are all 1 by (c, s).
__global__ void __launch_bounds__(kBlock) k_phase_mask(double2* __restrict__ a, uint64_t count, uint64_t mask,
                                                       double c, double s)
{
    const double2 ph = make_double2(c, s);
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < count;
         i += uint64_t(gridDim.x) * blockDim.x) {
        uint64_t idx = insert_ones(i, mask);
        a[idx] = cmul(a[idx], ph);
    }
}

__global__ void __launch_bounds__(kBlock) k_negate_mask(double2* __restrict__ a, uint64_t count, uint32_t q)
{
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < count;
         i += uint64_t(gridDim.x) * blockDim.x) {
        uint64_t idx = insert0(i, q) | (uint64_t(1) << q);
        double2 v = a[idx];
        a[idx] = make_double2(-v.x, -v.y);
    }
}

// Swap |..1_q0..0_q1..> <-> |..0_q0..1_q1..>: 2^(n-2) pairs.
__global__ void __launch_bounds__(kBlock) k_swap(double2* __restrict__ a, uint64_t count, uint32_t q0, uint32_t q1)
{
    const uint32_t lo = q0 < q1 ? q0 : q1, hi = q0 < q1 ? q1 : q0;
    const uint64_t m0 = uint64_t(1) << q0, m1 = uint64_t(1) << q1;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < count;
         i += uint64_t(gridDim.x) * blockDim.x) {
        uint64_t base = insert0(insert0(i, lo), hi);
        double2 x = a[base | m0], y = a[base | m1];
        a[base | m0] = y;
        a[base | m1] = x;
    }
}

__global__ void k_set_one(double2* a, uint64_t i) { a[i] = make_double2(1.0, 0.0); }

// index of the j-th amplitude with physical bit b equal to v (j < 2^(n-1))
__device__ __forceinline__ uint64_t with_bit(uint64_t j, uint32_t b, uint64_t v)
{
    const uint64_t lo = j & ((uint64_t(1) << b) - 1);
    return ((j >> b) << (b + 1)) | (v << b) | lo;
}

// partial[block] = sum of |a_i|^2 (std::norm's two roundings, no FMA) over the
// amplitudes with bit b set; grid-stride per thread, then a fixed-order tree
__global__ void __launch_bounds__(kBlock) k_prob_bit(const double2* __restrict__ a, uint64_t half, uint32_t b,
                                                     double* __restrict__ partial)
{
    __shared__ double sh[kBlock / 32];
    double s = 0.0;
    for (uint64_t j = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; j < half; j += uint64_t(gridDim.x) * blockDim.x) {
        const double2 v = a[with_bit(j, b, 1)];
        s += __dadd_rn(__dmul_rn(v.x, v.x), __dmul_rn(v.y, v.y));
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kBlock / 32; ++w) t += sh[w];
        partial[blockIdx.x] = t;
    }
}

// StateVector::measureQubit's collapse (StateVector.cpp:173-182): amplitudes whose
// bit differs from the outcome become 0, the others are divided by norm
__global__ void __launch_bounds__(kBlock) k_collapse_bit(double2* __restrict__ a, uint64_t half, uint32_t b,
                                                         uint64_t outcome, double norm)
{
    for (uint64_t j = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; j < half; j += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t keep = with_bit(j, b, outcome), drop = with_bit(j, b, outcome ^ 1);
        const double2 v = a[keep];
        a[keep] = make_double2(v.x / norm, v.y / norm);
        a[drop] = make_double2(0.0, 0.0);
    }
}

// StateVector::resetQubit's move (StateVector.cpp:203-215): the outcome's
// amplitudes, divided by nf, land on the bit-0 half; the bit-1 half becomes 0
__global__ void __launch_bounds__(kBlock) k_reset_bit(double2* __restrict__ a, uint64_t half, uint32_t b,
                                                      uint64_t outcome, double nf)
{
    for (uint64_t j = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; j < half; j += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t i0 = with_bit(j, b, 0), i1 = with_bit(j, b, 1);
        const double2 v = a[outcome ? i1 : i0];
        a[i0] = make_double2(v.x / nf, v.y / nf);
        a[i1] = make_double2(0.0, 0.0);
    }
}

__global__ void __launch_bounds__(kBlock) k_scale(double2* __restrict__ a, uint64_t count, double s)
{
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < count;
         i += uint64_t(gridDim.x) * blockDim.x) {
        double2 v = a[i];
        a[i] = make_double2(v.x * s, v.y * s);
    }
}

// Noise::applyPauliNoise (Noise.cpp:34-44) as one pass: X on every qubit
// with an odd bit-flip count, then Z on every qubit with an odd phase-flip
// count.  Product of those operators: out[i] = (-1)^popc(i & z) * in[i ^ x].
__global__ void k_pauli_masks(const int32_t* __restrict__ counts, uint32_t n, uint64_t* masks)
{
    uint64_t x = 0, z = 0;
    for (uint32_t q = 0; q < n; ++q) {
        if (counts[q] % 2 != 0) x |= uint64_t(1) << q;
        if (counts[64 + q] % 2 != 0) z |= uint64_t(1) << q;
    }
    masks[0] = x;
    masks[1] = z;
}

__global__ void __launch_bounds__(kBlock) k_pauli_frame(double2* __restrict__ a, uint64_t npairs,
                                                        const uint64_t* __restrict__ masks, const uint32_t* perm)
{
    // masks are in logical qubits; map them to physical bits
    __shared__ uint64_t sx, sz;
    if (threadIdx.x == 0) {
        uint64_t lx = masks[0], lz = masks[1], px = 0, pz = 0;
        for (uint32_t q = 0; q < 64; ++q) {
            if ((lx >> q) & 1) px |= uint64_t(1) << perm[q];
            if ((lz >> q) & 1) pz |= uint64_t(1) << perm[q];
        }
        sx = px;
        sz = pz;
    }
    __syncthreads();
    const uint64_t x = sx, z = sz;
    if (x == 0 && z == 0) return;
    const uint32_t hb = x ? 63 - __clzll((long long)x) : 0;
    for (uint64_t k = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; k < npairs;
         k += uint64_t(gridDim.x) * blockDim.x) {
        uint64_t i = insert0(k, hb);
        uint64_t j = x ? (i ^ x) : (i | 1);
        double2 vi = a[i], vj = a[j];
        double si = (__popcll(i & z) & 1) ? -1.0 : 1.0;
        double sj = (__popcll(j & z) & 1) ? -1.0 : 1.0;
        if (x) {
            a[i] = make_double2(si * vj.x, si * vj.y);
            a[j] = make_double2(sj * vi.x, sj * vi.y);
        } else {
            a[i] = make_double2(si * vi.x, si * vi.y);
            a[j] = make_double2(sj * vj.x, sj * vj.y);
        }
    }
}

// out[logical L] = amp[physical(L)] for L in [base, base + count)
__global__ void __launch_bounds__(kBlock) k_gather_logical(const double2* __restrict__ a, double2* __restrict__ out,
                                                           uint64_t base, uint64_t count, const uint32_t* perm,
                                                           uint32_t n)
{
    __shared__ uint32_t sp[64];
    if (threadIdx.x < 64) sp[threadIdx.x] = threadIdx.x < n ? perm[threadIdx.x] : 0;
    __syncthreads();
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < count;
         i += uint64_t(gridDim.x) * blockDim.x) {
        uint64_t L = base + i, P = 0;
        for (uint32_t q = 0; q < n; ++q) P |= ((L >> q) & 1) << sp[q];
        out[i] = a[P];
    }
}

template <class F>
void launch_pairs(qse_state* st, uint32_t q, F f)
{
    uint64_t np = st->size() >> 1;
    if (np >= 2)
        k_pairs2<<<grid_full(np / 2), kBlock, 0, st->ctx->stream>>>(reinterpret_cast<double2*>(st->amp), np / 2,
                                                                            q, f);
    else
        k_pairs<<<grid_full(np), kBlock, 0, st->ctx->stream>>>(reinterpret_cast<double2*>(st->amp), np, q, f);
    QSE_CUDA(cudaGetLastError());
    count_launch(st->ctx);
}

}  // namespace

void launch_h(qse_state* st, uint32_t q) { launch_pairs(st, q, FH{}); }
void launch_x(qse_state* st, uint32_t q) { launch_pairs(st, q, FX{}); }
void launch_y(qse_state* st, uint32_t q) { launch_pairs(st, q, FY{}); }
void launch_rx(qse_state* st, uint32_t q, double c, double s) { launch_pairs(st, q, FRX{c, s}); }
void launch_ry(qse_state* st, uint32_t q, double c, double s) { launch_pairs(st, q, FRY{c, s}); }
void launch_rz(qse_state* st, uint32_t q, double c0, double s0, double c1, double s1)
{
    launch_pairs(st, q, FRZ{make_double2(c0, s0), make_double2(c1, s1)});
}

void launch_gate2x2(qse_state* st, uint32_t q, const double m[8], uint64_t ctrl_mask)
{
    (void)ctrl_mask;
    launch_pairs(st, q, F2x2{make_double2(m[0], m[1]), make_double2(m[2], m[3]), make_double2(m[4], m[5]),
                             make_double2(m[6], m[7])});
}

void launch_z(qse_state* st, uint32_t q)
{
    uint64_t cnt = st->size() >> 1;
    k_negate_mask<<<grid_full(cnt), kBlock, 0, st->ctx->stream>>>(reinterpret_cast<double2*>(st->amp), cnt, q);
    QSE_CUDA(cudaGetLastError());
    count_launch(st->ctx);
}

void launch_phase_mask(qse_state* st, uint64_t all_mask, double c, double s)
{
    uint64_t cnt = st->size() >> __builtin_popcountll(all_mask);
    k_phase_mask<<<grid_full(cnt), kBlock, 0, st->ctx->stream>>>(reinterpret_cast<double2*>(st->amp), cnt,
                                                                        all_mask, c, s);
    QSE_CUDA(cudaGetLastError());
    count_launch(st->ctx);
}

void launch_cphase(qse_state* st, uint32_t c, uint32_t t, double co, double si)
{
    launch_phase_mask(st, (uint64_t(1) << c) | (uint64_t(1) << t), co, si);
}

void launch_cnot(qse_state* st, uint32_t c, uint32_t t)
{
    uint64_t np = st->size() >> 2;
    k_cpairs<<<grid_full(np), kBlock, 0, st->ctx->stream>>>(reinterpret_cast<double2*>(st->amp), np, c, t,
                                                                   FX{});
    QSE_CUDA(cudaGetLastError());
    count_launch(st->ctx);
}

void launch_swap(qse_state* st, uint32_t q0, uint32_t q1)
{
    uint64_t cnt = st->size() >> 2;
    k_swap<<<grid_full(cnt), kBlock, 0, st->ctx->stream>>>(reinterpret_cast<double2*>(st->amp), cnt, q0, q1);
    QSE_CUDA(cudaGetLastError());
    count_launch(st->ctx);
}

void mark_zero(qse_state* st)
{
    for (uint32_t q = 0; q < 64; ++q) st->perm[q] = q;
    mark_basis(st, 0);
}

void mark_basis(qse_state* st, uint64_t phys_index)
{
    st->lazy_basis = true;
    st->lazy_index = phys_index;
    st->lazy_umask = 0;
    st->lazy_pmask = 0;
    st->lazy_src = nullptr;
    st->touch();
}

namespace {
void write_basis_state(qse_state* st, uint64_t phys_index)
{
    st->lazy_basis = false;
    st->lazy_umask = 0;
    st->lazy_pmask = 0;
    st->lazy_src = nullptr;
    st->touch();
    QSE_CUDA(cudaMemsetAsync(st->amp, 0, st->size() * 16, st->ctx->stream));
    k_set_one<<<1, 1, 0, st->ctx->stream>>>(reinterpret_cast<double2*>(st->amp), phys_index);
    QSE_CUDA(cudaGetLastError());
    count_launch(st->ctx);
}

// out[pdep(i, umask) | fixed] = src[i] for i < count (count = 2^popcount(umask);
// every other amplitude was zeroed before)
__global__ void __launch_bounds__(kBlock) k_expand_compact(double2* __restrict__ out, const double2* __restrict__ src,
                                                          uint64_t count, uint64_t umask, uint64_t fixed)
{
    for (uint64_t i = blockIdx.x * uint64_t(kBlock) + threadIdx.x; i < count; i += uint64_t(gridDim.x) * kBlock) {
        uint64_t x = fixed, r = i;
        for (uint64_t m = umask; m; m &= m - 1, r >>= 1)
            if (r & 1) x |= m & (~m + 1);
        out[x] = src[i];
    }
}

// out[x] for every x < size: 0 unless x's bits outside umask | pmask equal
// fixed's, else src[pext(x, umask)] times, for the i-th qubit of pmask
// (ascending), src[count + 2i + its bit of x]
__global__ void __launch_bounds__(kBlock) k_expand_product(double2* __restrict__ out, const double2* __restrict__ src,
                                                          uint64_t size, uint64_t count, uint64_t umask,
                                                          uint64_t pmask, uint64_t fixed)
{
    const uint64_t zmask = (size - 1) & ~(umask | pmask);
    for (uint64_t x = blockIdx.x * uint64_t(kBlock) + threadIdx.x; x < size; x += uint64_t(gridDim.x) * kBlock) {
        if ((x ^ fixed) & zmask) {
            out[x] = make_double2(0.0, 0.0);
            continue;
        }
        uint64_t c = 0, r = 0;
        for (uint64_t m = umask; m; m &= m - 1, ++r) c |= ((x >> (__ffsll(static_cast<long long>(m)) - 1)) & 1) << r;
        double2 v = src[c];
        uint64_t i = 0;
        for (uint64_t m = pmask; m; m &= m - 1, ++i)
            v = cmul(v, src[count + 2 * i + ((x >> (__ffsll(static_cast<long long>(m)) - 1)) & 1)]);
        out[x] = v;
    }
}

// the compact form of a lazy state written out: zeros, then the compact
// amplitudes at their places (with product qubits: every amplitude)
void write_compact_state(qse_state* st)
{
    const uint64_t umask = st->lazy_umask, pmask = st->lazy_pmask, fixed = st->lazy_index & ~umask;
    const double2* src = static_cast<const double2*>(st->lazy_src);
    st->lazy_basis = false;
    st->lazy_umask = 0;
    st->lazy_pmask = 0;
    st->lazy_src = nullptr;
    st->touch();
    const uint64_t count = uint64_t(1) << __builtin_popcountll(umask);
    if (pmask) {
        k_expand_product<<<grid_full(st->size()), kBlock, 0, st->ctx->stream>>>(
            reinterpret_cast<double2*>(st->amp), src, st->size(), count, umask, pmask, fixed);
    } else {
        QSE_CUDA(cudaMemsetAsync(st->amp, 0, st->size() * 16, st->ctx->stream));
        k_expand_compact<<<grid_full(count), kBlock, 0, st->ctx->stream>>>(reinterpret_cast<double2*>(st->amp), src,
                                                                           count, umask, fixed);
    }
    QSE_CUDA(cudaGetLastError());
    count_launch(st->ctx);
}
}  // namespace

void materialize(qse_state* st)
{
    if (!st->lazy_basis) return;
    if (st->lazy_umask) write_compact_state(st);
    else write_basis_state(st, st->lazy_index);
}

// StateVector::measureQubit / resetQubit (StateVector.cpp:158-221) with the
// draw u injected: prob1 = sum of |a_i|^2 over the qubit's 1 half (fixed-order
// reduction), outcome = u < prob1, then the collapse (or the reset move).
int measure_or_reset_qubit(qse_state* st, uint32_t q, double u, bool reset, double* prob1)
{
    if (q >= st->n) fail(QSE_ERR_QUBIT, "qubit index out of range");
    materialize(st);
    qse_ctx* ctx = st->ctx;
    const uint32_t b = st->perm[q];
    const uint64_t half = st->size() / 2;
    const unsigned grid = unsigned(std::min<uint64_t>((half + kBlock - 1) / kBlock, uint64_t(ctx->num_sms) * 8));
    ctx->scratch.reserve(size_t(grid) * 8 + 16);
    ctx->host_small.reserve(size_t(grid) * 8 + 16);
    QSE_CUDA(cudaStreamSynchronize(ctx->stream));  // host_small may still feed an earlier copy
    double* part = static_cast<double*>(ctx->scratch.ptr);
    k_prob_bit<<<grid, kBlock, 0, ctx->stream>>>(reinterpret_cast<const double2*>(st->amp), half, b, part);
    QSE_CUDA(cudaGetLastError());
    count_launch(ctx);
    double* hp = static_cast<double*>(ctx->host_small.ptr);
    QSE_CUDA(cudaMemcpyAsync(hp, part, size_t(grid) * 8, cudaMemcpyDeviceToHost, ctx->stream));
    QSE_CUDA(cudaStreamSynchronize(ctx->stream));
    double p1 = 0.0;
    for (unsigned i = 0; i < grid; ++i) p1 += hp[i];
    const int outcome = (u < p1) ? 1 : 0;
    const double norm = std::sqrt(outcome ? p1 : 1.0 - p1);
    st->touch();
    if (reset)
        k_reset_bit<<<grid, kBlock, 0, ctx->stream>>>(reinterpret_cast<double2*>(st->amp), half, b, uint64_t(outcome),
                                                      norm);
    else
        k_collapse_bit<<<grid, kBlock, 0, ctx->stream>>>(reinterpret_cast<double2*>(st->amp), half, b,
                                                         uint64_t(outcome), norm);
    QSE_CUDA(cudaGetLastError());
    count_launch(ctx);
    if (prob1) *prob1 = p1;
    return outcome;
}

void launch_init_zero_state(qse_state* st) { write_basis_state(st, 0); }

void scale_state(qse_state* st, double s)
{
    uint64_t cnt = st->size();
    k_scale<<<grid_full(cnt), kBlock, 0, st->ctx->stream>>>(reinterpret_cast<double2*>(st->amp), cnt, s);
    QSE_CUDA(cudaGetLastError());
    count_launch(st->ctx);
}

void launch_pauli_frame(qse_state* st, const int32_t* d_counts)
{
    materialize(st);
    qse_ctx* ctx = st->ctx;
    ctx->scratch.reserve(64 * sizeof(uint32_t) + 2 * sizeof(uint64_t));
    uint64_t* d_masks = static_cast<uint64_t*>(ctx->scratch.ptr);
    uint32_t* d_perm = reinterpret_cast<uint32_t*>(d_masks + 2);
    uint32_t perm[64];
    for (uint32_t q = 0; q < 64; ++q) perm[q] = q < st->n ? st->perm[q] : 0;
    ctx->host_small.reserve(sizeof(perm));
    std::memcpy(ctx->host_small.ptr, perm, sizeof(perm));
    QSE_CUDA(cudaMemcpyAsync(d_perm, ctx->host_small.ptr, sizeof(perm), cudaMemcpyHostToDevice, ctx->stream));
    k_pauli_masks<<<1, 1, 0, ctx->stream>>>(d_counts, st->n, d_masks);
    QSE_CUDA(cudaGetLastError());
    uint64_t np = st->size() >> 1;
    k_pauli_frame<<<grid_full(np), kBlock, 0, ctx->stream>>>(reinterpret_cast<double2*>(st->amp), np, d_masks,
                                                                d_perm);
    QSE_CUDA(cudaGetLastError());
    count_launch(ctx, 2);
    // the host buffer is reused by the next call only after this stream work
    QSE_CUDA(cudaStreamSynchronize(ctx->stream));
}

// flush(): device -> host in logical qubit order, logical indices
// [first, first + count).  With the identity map a plain copy; otherwise
// gathered chunk by chunk through device scratch.
void download_range(qse_state* st, uint64_t first, uint64_t count, double* host)
{
    materialize(st);
    qse_ctx* ctx = st->ctx;
    if (count == 0) return;
    if (st->identity_perm()) {
        QSE_CUDA(cudaMemcpyAsync(host, st->amp + 2 * first, count * 16, cudaMemcpyDeviceToHost, ctx->stream));
        QSE_CUDA(cudaStreamSynchronize(ctx->stream));
        return;
    }
    const uint64_t chunk = std::min<uint64_t>(count, uint64_t(1) << 24);
    ctx->scratch.reserve(chunk * 16 + 64 * 4 + 256);
    uint32_t perm[64] = {0};
    for (uint32_t q = 0; q < st->n; ++q) perm[q] = st->perm[q];
    char* d = static_cast<char*>(ctx->scratch.ptr);
    uint32_t* d_perm = reinterpret_cast<uint32_t*>(d + chunk * 16);
    ctx->host_small.reserve(sizeof(perm));
    QSE_CUDA(cudaStreamSynchronize(ctx->stream));
    std::memcpy(ctx->host_small.ptr, perm, sizeof(perm));
    QSE_CUDA(cudaMemcpyAsync(d_perm, ctx->host_small.ptr, sizeof(perm), cudaMemcpyHostToDevice, ctx->stream));
    for (uint64_t off = 0; off < count; off += chunk) {
        uint64_t cnt = std::min(chunk, count - off);
        k_gather_logical<<<grid_for(ctx, cnt), kBlock, 0, ctx->stream>>>(
            reinterpret_cast<const double2*>(st->amp), reinterpret_cast<double2*>(d), first + off, cnt, d_perm, st->n);
        QSE_CUDA(cudaGetLastError());
        count_launch(ctx);
        QSE_CUDA(cudaMemcpyAsync(host + 2 * off, d, cnt * 16, cudaMemcpyDeviceToHost, ctx->stream));
        QSE_CUDA(cudaStreamSynchronize(ctx->stream));
    }
}

void download_logical(qse_state* st, double* host) { download_range(st, 0, st->size(), host); }

void permute_to_logical(qse_state* st, double* dst_device)
{
    materialize(st);
    qse_ctx* ctx = st->ctx;
    ctx->scratch.reserve(64 * sizeof(uint32_t));
    uint32_t perm[64] = {0};
    for (uint32_t q = 0; q < st->n; ++q) perm[q] = st->perm[q];
    ctx->host_small.reserve(sizeof(perm));
    std::memcpy(ctx->host_small.ptr, perm, sizeof(perm));
    QSE_CUDA(cudaMemcpyAsync(ctx->scratch.ptr, ctx->host_small.ptr, sizeof(perm), cudaMemcpyHostToDevice,
                             ctx->stream));
    uint64_t cnt = st->size();
    k_gather_logical<<<grid_for(ctx, cnt), kBlock, 0, ctx->stream>>>(
        reinterpret_cast<const double2*>(st->amp), reinterpret_cast<double2*>(dst_device), 0, cnt,
        static_cast<const uint32_t*>(ctx->scratch.ptr), st->n);
    QSE_CUDA(cudaGetLastError());
    count_launch(ctx);
    QSE_CUDA(cudaStreamSynchronize(ctx->stream));
}

}  // namespace qse
