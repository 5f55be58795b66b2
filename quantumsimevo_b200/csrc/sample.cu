// sample.cu -- device StateVector::sample / measure (StateVector.cpp:77-156).
//
// The reference computes cum[i] = fl(cum[i-1] + p_i), p_i = fl(re^2 + im^2),
// sequentially in index order, then answers each shot with the first i such
// that cum[i] >= u * total (std::lower_bound).  A plain parallel scan rounds
// differently, and at 30 qubits the sequential chain's own rounding (up to
// ~1e-7 of the total) exceeds the probability of a typical basis state, so
// the outcome index would differ for many shots.  This file reproduces the
// sequential chain bit for bit with a parallel algorithm:
//
//   While the running sum c stays inside one binade [2^e, 2^(e+1)), every
//   addition rounds to the fixed grid G = 2^(e-52), so with C = c/G an integer
//   the step is C += round(p_i / G), where a tie (p_i/G exactly k + 1/2)
//   rounds so that C stays even.  A step is therefore the map
//   x -> x + d[x mod 2] (two offsets, one per parity of the incoming sum), and
//   such maps compose associatively: a block of elements folds into one
//   (d_even, d_odd) pair, and a block-wide scan gives every prefix.  When the
//   sum leaves the binade (C reaches 2^53) that single step is redone with a
//   real FP64 addition and the scan restarts on the new grid; c only grows, so
//   there are at most a few dozen such restarts in the whole vector.
//
// Passes: (1) per-block approximate sums, (2) a scan of those to guess each
// block's binade, (3) per-block (d_even, d_odd) on the guessed grid,
// (4) one CTA walks the blocks in order with the exact running sum (blocks
// whose guess fails are redone exactly), (5) every block writes its exact
// cumulative values.  Shots then binary-search the block starts and the
// block's values.
#include <cuda_runtime.h>

#include <algorithm>

#include "philox.cuh"
#include "qse_internal.h"

namespace qse {
namespace {

constexpr int kBT = 256;            // threads per block
constexpr int kEPT = 16;            // elements per thread
constexpr int kBS = kBT * kEPT;     // elements per block (4096)
constexpr uint64_t kTwo53 = uint64_t(1) << 53;
constexpr int kPad = kEPT + 1;      // staging-buffer row stride (doubles)

// staging-buffer position of block element i (row i / kEPT, column i % kEPT)
__device__ __forceinline__ uint32_t stage_slot(uint32_t i) { return (i / kEPT) * kPad + (i % kEPT); }

// Block folds on the grids of two adjacent binades, e and e+1: the running sum
// at the block is known only approximately, and near a binade boundary (for a
// normalised state the sum ends just below 1.0 = 2^0 for many blocks) either
// can hold.  The chain picks the fold of the binade the exact sum is in.
struct Summ {
    uint64_t d[2][2];               // d[k] = offsets (even, odd incoming sum) on the grid of binade e+k
    int32_t e;                      // lower binade guessed (INT32_MIN: no guess)
    int32_t ok;                     // bit k: no single step leaves binade e+k
};

// the fold of s that applies to a running sum in binade e0, if any
__device__ __forceinline__ bool summ_pick(const Summ& s, int e0, uint64_t& d0, uint64_t& d1)
{
    if (s.e == INT32_MIN) return false;
    const int k = e0 - s.e;
    if (k < 0 || k > 1 || !((s.ok >> k) & 1)) return false;
    d0 = s.d[k][0];
    d1 = s.d[k][1];
    return true;
}

__device__ __forceinline__ double norm2(double2 a)
{
    // std::norm(complex<double>) = re*re + im*im, two roundings, no FMA
    return __dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y));
}

struct PermMap {
    uint32_t n;
    uint32_t identity;
    uint8_t p[64];
};

__device__ __forceinline__ uint64_t phys_index(uint64_t L, const PermMap& pm)
{
    if (pm.identity) return L;
    uint64_t P = 0;
    for (uint32_t q = 0; q < pm.n; ++q) P |= ((L >> q) & 1) << pm.p[q];
    return P;
}

// epoch of a running sum: exponent of its binade (subnormals and 0 share -1022)
__device__ __forceinline__ int epoch_of(double c)
{
    if (c < 2.2250738585072014e-308) return -1022;
    return ilogb(c);
}

// element map x -> x + d[x&1] on grid 2^(e-52); returns false if p alone leaves the binade
__device__ __forceinline__ bool elem_map(double p, int e, uint64_t& d0, uint64_t& d1)
{
    if (p >= ldexp(1.0, e + 1)) { d0 = d1 = kTwo53; return false; }
    double q = ldexp(p, 52 - e);
    double f = floor(q);
    double fr = q - f;
    uint64_t fi = uint64_t(f);
    if (fr > 0.5) { d0 = d1 = fi + 1; }
    else if (fr < 0.5) { d0 = d1 = fi; }
    else if (fi & 1) { d0 = fi + 1; d1 = fi; }       // tie: result must be even
    else { d0 = fi; d1 = fi + 1; }
    return true;
}

// The grid of binade e as a multiplier: q = p * 2^(52-e) is exact (a power-of-two
// scaling whose result stays below 2^53), so one multiply, one rint and one
// exact difference give the element map.  Binades whose multiplier is not a
// finite double (a running sum that is still zero or subnormal) keep elem_map.
struct Grid {
    double scale;   // 2^(52-e)
    double limit;   // 2^(e+1): an element this large leaves the binade by itself
    int e;
    int fast;
};

__device__ __forceinline__ Grid grid_of(int e)
{
    Grid g;
    g.e = e;
    g.fast = (52 - e) <= 1000 ? 1 : 0;
    g.scale = g.fast ? ldexp(1.0, 52 - e) : 0.0;
    g.limit = ldexp(1.0, e + 1);
    return g;
}

// elem_map on grid g: d0 == d1 unless p / G ends in exactly one half (a tie)
__device__ __forceinline__ bool elem_map_g(double p, const Grid& g, uint64_t& d0, uint64_t& d1)
{
    if (!g.fast) return elem_map(p, g.e, d0, d1);
    if (!(p < g.limit)) { d0 = d1 = kTwo53; return false; }
    const double q = p * g.scale;
    const double r = rint(q);
    const double df = q - r;               // exact (Sterbenz)
    if (df == 0.5 || df == -0.5) {         // tie: the sum must come out even
        const uint64_t k = uint64_t(floor(q));
        if (k & 1) { d0 = k + 1; d1 = k; }
        else { d0 = k; d1 = k + 1; }
    } else {
        d0 = d1 = uint64_t(r);
    }
    return true;
}

// block-wide exclusive prefix of 64-bit integers (warp shuffles, then the
// warp totals); returns the block total.  sh: >= 2 * (kBT / 32) + 1 words.
__device__ uint64_t block_scan_add(uint64_t v, uint64_t& excl, uint64_t* sh)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nw = blockDim.x >> 5;
    uint64_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) sh[warp] = inc;
    __syncthreads();
    if (tid == 0) {
        uint64_t run = 0;
        for (int w = 0; w < nw; ++w) {
            const uint64_t t = sh[w];
            sh[32 + w] = run;
            run += t;
        }
        sh[64] = run;
    }
    __syncthreads();
    excl = sh[32 + warp] + inc - v;
    const uint64_t total = sh[64];
    __syncthreads();
    return total;
}

// block_scan_add on integer-valued doubles; exact while the sums stay below 2^53
__device__ double block_scan_addd(double v, double& excl, double* sh)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nw = blockDim.x >> 5;
    double inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) sh[warp] = inc;
    __syncthreads();
    if (tid == 0) {
        double run = 0.0;
        for (int w = 0; w < nw; ++w) {
            const double t = sh[w];
            sh[32 + w] = run;
            run += t;
        }
        sh[64] = run;
    }
    __syncthreads();
    excl = sh[32 + warp] + (inc - v);
    const double total = sh[64];
    __syncthreads();
    return total;
}

__device__ __forceinline__ void compose(uint64_t a0, uint64_t a1, uint64_t b0, uint64_t b1, uint64_t& r0, uint64_t& r1)
{
    // first a, then b
    r0 = a0 + ((a0 & 1) ? b1 : b0);
    r1 = a1 + (((1 + a1) & 1) ? b1 : b0);
}

// block-wide inclusive scan of parity maps; returns the inclusive prefix of
// this thread's last element and fills excl (exclusive prefix of the thread)
__device__ void block_scan_maps(uint64_t t0, uint64_t t1, uint64_t& ex0, uint64_t& ex1, uint64_t* sh)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint64_t i0 = t0, i1 = t1;
    // warp inclusive scan
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t u0 = __shfl_up_sync(0xffffffffu, i0, o);
        uint64_t u1 = __shfl_up_sync(0xffffffffu, i1, o);
        if (lane >= o) {
            uint64_t r0, r1;
            compose(u0, u1, i0, i1, r0, r1);
            i0 = r0;
            i1 = r1;
        }
    }
    if (lane == 31) { sh[2 * warp] = i0; sh[2 * warp + 1] = i1; }
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        uint64_t w0 = lane < nw ? sh[2 * lane] : 0, w1 = lane < nw ? sh[2 * lane + 1] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t u0 = __shfl_up_sync(0xffffffffu, w0, o);
            uint64_t u1 = __shfl_up_sync(0xffffffffu, w1, o);
            if (lane >= o) {
                uint64_t r0, r1;
                compose(u0, u1, w0, w1, r0, r1);
                w0 = r0;
                w1 = r1;
            }
        }
        if (lane < nw) { sh[64 + 2 * lane] = w0; sh[64 + 2 * lane + 1] = w1; }
    }
    __syncthreads();
    // exclusive prefix for this thread = (warp prefix before this warp) then (lanes before)
    uint64_t w0 = 0, w1 = 0;
    if (warp > 0) { w0 = sh[64 + 2 * (warp - 1)]; w1 = sh[64 + 2 * (warp - 1) + 1]; }
    uint64_t l0 = __shfl_up_sync(0xffffffffu, i0, 1), l1 = __shfl_up_sync(0xffffffffu, i1, 1);
    if (lane == 0) { l0 = 0; l1 = 0; }
    compose(w0, w1, l0, l1, ex0, ex1);
    __syncthreads();
}

// Exact sequential cumulative sums of one block of `cnt` (<= kBS) values held
// in stage (element i at stage_slot(i), so thread tid's elements tid*kEPT + j
// sit in row tid), starting from the exact running sum c_in.  The values go
// to out (if non-null), staged in the same buffer.  Returns the block's final
// sum.  Must be called by all threads of the block.
__device__ __forceinline__ double block_exact(uint32_t cnt, double c_in, double* out, uint64_t* sh, double* stage)
{
    __shared__ double s_c;
    __shared__ int s_t;
    const uint32_t tid = threadIdx.x;
    uint32_t pos = 0;
    double c = c_in;
    // Fast path (nearly every block): a full block on a fast grid with no tie
    // and a running sum that stays below 2^53 grid units.  The grid integers
    // and all their partial sums are then exact in FP64, so the scan runs on
    // doubles with no integer conversion; otherwise fall through.
    if (cnt == uint32_t(kBS) && c > 0.0) {
        const int e = epoch_of(c);
        const Grid g = grid_of(e);
        if (g.fast) {
            double q[kEPT];
            double tsum = 0.0;
            bool ok = true;
#pragma unroll
            for (int j = 0; j < kEPT; ++j) {
                const double pj = stage[tid * kPad + j];
                const double x = pj * g.scale;
                const double r = rint(x);
                const double df = x - r;
                ok = ok && pj < g.limit && df != 0.5 && df != -0.5;
                q[j] = r;
                tsum += r;
            }
            if (__syncthreads_and(ok)) {
                double ex;
                block_scan_addd(tsum, ex, reinterpret_cast<double*>(sh));
                double run = c * g.scale + ex;
#pragma unroll
                for (int j = 0; j < kEPT; ++j) {
                    run += q[j];
                    q[j] = run;
                }
                if (!__syncthreads_or(run >= 0x1p53)) {   // sums only grow: the last is the largest
                    const double G = ldexp(1.0, e - 52);
                    if (out) {
#pragma unroll
                        for (int j = 0; j < kEPT; ++j) stage[tid * kPad + j] = q[j] * G;
                    }
                    if (tid == blockDim.x - 1) s_c = run * G;
                    __syncthreads();
                    if (out) {
#pragma unroll
                        for (int j = 0; j < kEPT; ++j) {
                            const uint32_t i = j * kBT + tid;
                            out[i] = stage[stage_slot(i)];
                        }
                    }
                    const double cf = s_c;
                    __syncthreads();
                    return cf;
                }
            }
        }
    }
    // general path (the fast path writes stage only when it returns)
    double p[kEPT];
#pragma unroll
    for (int j = 0; j < kEPT; ++j) p[j] = stage[tid * kPad + j];
    while (pos < cnt) {
        const int e = epoch_of(c);
        const double G = ldexp(1.0, e - 52);
        const uint64_t C = uint64_t(ldexp(c, 52 - e));
        const Grid g = grid_of(e);
        // this thread's element maps over its elements >= pos (even-parity
        // offsets kept; a tie anywhere sends the block to the general path,
        // which recomputes both offsets)
        uint64_t Ci[kEPT];
        int bad = kBS;
        bool pure = true;
        uint64_t tsum = 0;
#pragma unroll
        for (int j = 0; j < kEPT; ++j) {
            uint32_t i = tid * kEPT + j;
            uint64_t a0 = 0, a1 = 0;
            if (i >= pos && i < cnt) {
                if (!elem_map_g(p[j], g, a0, a1) && bad == kBS) bad = int(i);
            }
            Ci[j] = a0;
            pure = pure && a0 == a1;
            tsum += a0;
        }
        int first = bad;
        if (__syncthreads_and(pure)) {
            // no ties anywhere: every map is a translation and prefixes are sums
            uint64_t ex;
            block_scan_add(tsum, ex, sh);
            uint64_t run = C + ex;
#pragma unroll
            for (int j = 0; j < kEPT; ++j) {
                run += Ci[j];
                Ci[j] = run;
                uint32_t i = tid * kEPT + j;
                if (i >= pos && i < cnt && run >= kTwo53 && int(i) < first) first = int(i);
            }
        } else {
            uint64_t t0 = 0, t1 = 0;
#pragma unroll
            for (int j = 0; j < kEPT; ++j) {
                uint64_t a0 = 0, a1 = 0, r0, r1;
                const uint32_t i = tid * kEPT + j;
                if (i >= pos && i < cnt) elem_map_g(p[j], g, a0, a1);
                compose(t0, t1, a0, a1, r0, r1);
                t0 = r0;
                t1 = r1;
            }
            uint64_t ex0, ex1;
            block_scan_maps(t0, t1, ex0, ex1, sh);
            // running values; first index that reaches 2^53 or is flagged
            uint64_t run0 = ex0, run1 = ex1;
#pragma unroll
            for (int j = 0; j < kEPT; ++j) {
                uint64_t a0 = 0, a1 = 0, r0, r1;
                const uint32_t i = tid * kEPT + j;
                if (i >= pos && i < cnt) elem_map_g(p[j], g, a0, a1);
                compose(run0, run1, a0, a1, r0, r1);
                run0 = r0;
                run1 = r1;
                uint64_t v = C + ((C & 1) ? run1 : run0);
                Ci[j] = v;
                if (i >= pos && i < cnt && v >= kTwo53 && int(i) < first) first = int(i);
            }
        }
        if (tid == 0) s_t = int(cnt);
        __syncthreads();
        if (first < int(cnt)) atomicMin(&s_t, first);
        __syncthreads();
        const uint32_t t = uint32_t(s_t);
        // values before t are exact on this grid
#pragma unroll
        for (int j = 0; j < kEPT; ++j) {
            uint32_t i = tid * kEPT + j;
            if (i >= pos && i < t && out) stage[tid * kPad + j] = double(Ci[j]) * G;
            if (t < cnt && i >= pos && i + 1 == t) s_c = double(Ci[j]) * G;   // c_{t-1}
            if (t == cnt && i + 1 == cnt) s_c = double(Ci[j]) * G;
        }
        if (tid == 0 && t == pos) s_c = c;                           // no element on this grid
        __syncthreads();
        if (t >= cnt) { c = s_c; __syncthreads(); break; }
        // step t with a real FP64 addition (the reference's own rounding)
        if (tid == t / kEPT) {
            double prev = s_c;
            // element t from the staging buffer: slots >= t are still the
            // probabilities (indexing p[] here would put it in local memory)
            const double pt = stage[stage_slot(t)];
            double ct = __dadd_rn(prev, pt);
            if (out) stage[stage_slot(t)] = ct;
            s_c = ct;
        }
        __syncthreads();
        c = s_c;
        pos = t + 1;
        __syncthreads();
    }
    if (out) {
        // coalesced copy of the staged cumulative values
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kEPT; ++j) {
            const uint32_t i = j * kBT + tid;
            if (i < cnt) out[i] = stage[stage_slot(i)];
        }
    }
    return c;
}

// Probabilities of block elements [base, base + kBS) of the logical-order
// probability array: element i belongs to thread i / kEPT, slot i % kEPT.  The
// array is read coalesced into the padded staging buffer and each thread then
// picks up its kEPT consecutive values (row stride kPad keeps the 8-byte
// reads free of bank conflicts).
__device__ __forceinline__ void load_block_prob(const double* prob, uint64_t base, double (&p)[kEPT], double* stage)
{
    __syncthreads();  // earlier readers of the staging buffer are done
#pragma unroll
    for (int j = 0; j < kEPT; ++j) {
        const uint32_t i = j * kBT + threadIdx.x;
        stage[stage_slot(i)] = prob[base + i];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kEPT; ++j) p[j] = stage[threadIdx.x * kPad + j];
}

__device__ __forceinline__ void block_sum_store(double s, double* out)
{
    __shared__ double sh[kBT / 32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kBT / 32; ++w) t += sh[w];
        *out = t;
    }
}

// Block sums of a probability array written without them (coalesced reads).
__global__ void __launch_bounds__(kBT) k_block_sums(const double* __restrict__ prob, double* __restrict__ bsum)
{
    const double* src = prob + uint64_t(blockIdx.x) * kBS + threadIdx.x;
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < kEPT; ++j) s += src[j * kBT];
    block_sum_store(s, bsum + blockIdx.x);
}

// Identity qubit map: prob[i] = |amp[i]|^2 (coalesced), block sums on the way.
__global__ void __launch_bounds__(kBT) k_prob_identity(const double2* __restrict__ amp, double* __restrict__ prob,
                                                       double* __restrict__ bsum)
{
    const uint64_t base = uint64_t(blockIdx.x) * kBS;
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < kEPT; ++j) {
        const uint64_t i = base + j * kBT + threadIdx.x;
        const double v = norm2(amp[i]);
        prob[i] = v;
        s += v;
    }
    block_sum_store(s, bsum + blockIdx.x);
}

// Relabelled qubits (after SWAPs): the logical-order probability array is a
// bit permutation of the physical amplitudes.  Each CTA takes the 4096
// amplitudes spanned by 12 physical bits S that contain physical bits 0..4
// (contiguous 512-byte reads) and the physical images of logical bits 0..6
// (contiguous 1 KiB writes of probabilities), and transposes through shared
// memory.  Slot of read-order index r: XOR of img[b] over the set bits b of r,
// img[b] = 2^b with a host-chosen low nibble for b >= 4, so that both the
// write side (lanes vary r's bits 0..4) and the read side (lanes vary the
// read-order images of logical bits 0..4) touch 16 distinct 8-byte bank pairs
// per half-warp.  Each warp's 32 written probabilities of one j share one
// 4096-block of the logical array; their sum goes to that block's approximate
// sum (atomic: only the binade guess reads it).
struct GatherPlan {
    uint64_t outer_mask;      // physical bits outside S
    uint8_t sphys[12];        // S ascending (tile order for the reads)
    uint8_t slog[12];         // logical images of S, ascending (tile order for the writes)
    uint8_t wsrc[12];         // write-order bit b' -> read-order bit
    uint8_t pad[4];
    uint16_t img[12];         // shared-memory slot image of read-order bit b
    uint8_t inv[64];          // physical bit -> logical bit
};

__global__ void __launch_bounds__(kBT) k_prob_gather(const double2* __restrict__ amp, double* __restrict__ prob,
                                                     double* __restrict__ bsum, const __grid_constant__ GatherPlan g)
{
    __shared__ double sm[kBS];
    const uint32_t t = threadIdx.x;
    uint64_t ob = 0, lb = 0;
    {
        uint64_t c = blockIdx.x, m = g.outer_mask;
        while (m) {
            const uint32_t b = __ffsll((long long)m) - 1;
            m &= m - 1;
            if (c & 1) {
                ob |= uint64_t(1) << b;
                lb |= uint64_t(1) << g.inv[b];
            }
            c >>= 1;
        }
    }
    uint64_t tr = ob, tw = lb;
    uint32_t sw = 0, sr = 0;
    for (int b = 0; b < 8; ++b)
        if ((t >> b) & 1) {
            tr |= uint64_t(1) << g.sphys[b];
            tw |= uint64_t(1) << g.slog[b];
            sw ^= g.img[b];
            sr ^= g.img[g.wsrc[b]];
        }
#pragma unroll
    for (int j = 0; j < kEPT; ++j) {
        uint64_t off = 0;
        uint32_t so = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b)
            if ((j >> b) & 1) {
                off |= uint64_t(1) << g.sphys[8 + b];
                so ^= g.img[8 + b];
            }
        sm[sw ^ so] = norm2(amp[tr | off]);
    }
    __syncthreads();
    double ws[kEPT];
#pragma unroll
    for (int j = 0; j < kEPT; ++j) {
        uint64_t off = 0;
        uint32_t so = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b)
            if ((j >> b) & 1) {
                off |= uint64_t(1) << g.slog[8 + b];
                so ^= g.img[g.wsrc[8 + b]];
            }
        const double v = sm[sr ^ so];
        prob[tw | off] = v;
        ws[j] = v;
    }
    // Warp sums of the 16 values (one 4096-block per j): a transpose-reduce
    // butterfly.  Each step trades half of a lane's remaining partial sums with
    // the partner lane and keeps the half its lane bit selects, so after four
    // steps lane l holds the 16-lane sum for j = (l >> 1) & 15 and the last
    // exchange completes it (32 shuffles per lane instead of 160).
    const uint32_t lane = t & 31;
#pragma unroll
    for (int h = 8, lb = 16; h >= 1; h >>= 1, lb >>= 1) {
        const bool up = (lane & uint32_t(lb)) != 0;
#pragma unroll
        for (int k = 0; k < h; ++k) {
            const double lo = ws[k], hi = ws[k + h];
            const double give = up ? lo : hi;
            ws[k] = (up ? hi : lo) + __shfl_xor_sync(0xffffffffu, give, lb);
        }
    }
    ws[0] += __shfl_xor_sync(0xffffffffu, ws[0], 1);
    if ((lane & 1) == 0) {
        const uint32_t j = (lane >> 1) & 15;
        uint64_t off = 0;
        for (int b = 0; b < 4; ++b)
            if ((j >> b) & 1) off |= uint64_t(1) << g.slog[8 + b];
        atomicAdd(bsum + ((tw | off) >> 12), ws[0]);
    }
}

// Grid guess per block from approximate prefix sums of the block sums, in
// groups of kGT blocks: k_guess_part sums each group, k_guess_fin adds the
// groups before its own and scans its group.  The guess only selects the
// binades k_cdf_summ folds on; a block whose exact running sum turns out to
// lie elsewhere is folded exactly by the chain, so the summation order here
// affects speed, never results.
constexpr int kGT = 1024;

__device__ __forceinline__ double block_sum_all(double v, double* sh)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) t += sh[w];
    return t;
}

__global__ void __launch_bounds__(kGT) k_guess_part(const double* __restrict__ bsum, uint32_t nb,
                                                    double* __restrict__ gtot)
{
    __shared__ double sh[32];
    const uint32_t b = blockIdx.x * kGT + threadIdx.x;
    const double t = block_sum_all(b < nb ? bsum[b] : 0.0, sh);
    if (threadIdx.x == 0) gtot[blockIdx.x] = t;
}

__global__ void __launch_bounds__(kGT) k_guess_fin(const double* __restrict__ bsum, uint32_t nb,
                                                   const double* __restrict__ gtot, int32_t* __restrict__ guess)
{
    __shared__ double sh[32];
    __shared__ double wsc[32];
    double o = 0.0;
    for (uint32_t g = threadIdx.x; g < blockIdx.x; g += kGT) o += gtot[g];
    o = block_sum_all(o, sh);
    const uint32_t b = blockIdx.x * kGT + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double v = b < nb ? bsum[b] : 0.0;
    double inc = v;
    for (int d = 1; d < 32; d <<= 1) {
        const double u = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= uint32_t(d)) inc += u;
    }
    if (lane == 31) wsc[warp] = inc;
    __syncthreads();
    double wo = 0.0;
    for (uint32_t w = 0; w < warp; ++w) wo += wsc[w];
    if (b >= nb) return;
    const double lo_c = o + wo + (inc - v), hi_c = o + wo + inc;
    // conservative slack for the difference between this sum and the sequential
    // one (relative: sums of the same non-negative terms in another order; a
    // zero sum is exact, so leading zero blocks get binade -1022)
    const double slack = hi_c * 0x1.0p-20;
    const int e1 = lo_c - slack > 2.2250738585072014e-308 ? ilogb(lo_c - slack) : -1022;
    const int e2 = hi_c + slack > 2.2250738585072014e-308 ? ilogb(hi_c + slack) : -1022;
    // 2 e1 + 1 when the block may reach binade e1 + 1, 2 e1 when it stays in e1
    guess[b] = (e2 - e1 <= 1) ? 2 * e1 + (e2 - e1) : INT32_MIN;
}

// Block b's probabilities into the padded staging buffer with asynchronous
// 8-byte copies (same slots as load_block_prob), committed as one group; the
// persistent k_cdf_write fetches the next block while it works on this one.
__device__ __forceinline__ void stage_async(double* stage, const double* prob, uint64_t base)
{
#pragma unroll
    for (int j = 0; j < kEPT; ++j) {
        const uint32_t i = j * kBT + threadIdx.x;
        const uint32_t sa = uint32_t(__cvta_generic_to_shared(stage + stage_slot(i)));
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(prob + base + i) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void stage_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
// shared memory of k_cdf_write: two staging buffers
constexpr size_t kStage2 = size_t(2) * kBT * kPad * sizeof(double);
// resident CTAs per SM of k_cdf_write (its register budget: 128 per thread);
// the persistent grid is exactly that many per SM
constexpr int kWriteCTAs = 2;

// Fold of one block on the one or two binades its guess allows.  p holds the
// block coalesced (p[j] = element j * kBT + tid).  Per binade, three facts are
// independent of the element order: whether an element leaves the binade by
// itself (no fold there), whether any element lands on a tie of the grid, and
// the integer sum of the rounded elements.  Without ties every element's map
// is a translation, so the fold is that sum (exact below 2^53, and a sum at or
// above 2^53 stays there under rounding: the block then leaves the binade).
// Only a binade with a tie composes the maps in element order, after the block
// is restaged so that thread tid holds elements tid * kEPT .. + kEPT - 1.
__device__ __forceinline__ Summ block_summ(double (&p)[kEPT], int32_t gs, uint64_t* sh, double* stage)
{
    const int32_t e = gs >> 1;          // arithmetic shift: floor(gs / 2)
    const int nbin = 1 + (gs & 1);      // binades the block may run in
    Summ out{{{0, 0}, {0, 0}}, e, 0};
    unsigned flags = 0;                 // bit 2k: every element stays in binade e+k; bit 2k+1: no tie there
    double tsum[2] = {0.0, 0.0};
    for (int k = 0; k < nbin; ++k) {
        const Grid g = grid_of(e + k);
        int ok = 1;
        bool pure = true;
        double t = 0.0;
        if (g.fast) {
            // grid integers as doubles (exact below 2^53; a larger total
            // means the block leaves the binade, whatever its exact value)
#pragma unroll
            for (int j = 0; j < kEPT; ++j) {
                const double x = p[j] * g.scale;
                const double r = rint(x);
                const double df = x - r;
                if (!(p[j] < g.limit)) ok = 0;
                pure = pure && df != 0.5 && df != -0.5;
                t += r;
            }
        } else {
#pragma unroll
            for (int j = 0; j < kEPT; ++j) {
                uint64_t a0, a1;
                if (!elem_map_g(p[j], g, a0, a1)) ok = 0;
                pure = pure && a0 == a1;
                t += double(a0);
            }
        }
        flags |= unsigned(ok) << (2 * k) | unsigned(pure) << (2 * k + 1);
        tsum[k] = t;
    }
    // one barrier for the flags of both binades and both sums
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    flags = __reduce_and_sync(0xffffffffu, flags);
    for (int o = 16; o > 0; o >>= 1) {
        tsum[0] += __shfl_xor_sync(0xffffffffu, tsum[0], o);
        tsum[1] += __shfl_xor_sync(0xffffffffu, tsum[1], o);
    }
    double* shd = reinterpret_cast<double*>(sh);
    if (lane == 0) {
        shd[warp] = tsum[0];
        shd[kBT / 32 + warp] = tsum[1];
        sh[2 * (kBT / 32) + warp] = flags;
    }
    __syncthreads();
    double total[2] = {0.0, 0.0};
    unsigned all = ~0u;
    for (int w = 0; w < kBT / 32; ++w) {
        total[0] += shd[w];
        total[1] += shd[kBT / 32 + w];
        all &= unsigned(sh[2 * (kBT / 32) + w]);
    }
    __syncthreads();   // sh is reused below
    bool staged = false;    // p restaged in element order (each binade's sums are already taken)
    for (int k = 0; k < nbin; ++k) {
        if (!((all >> (2 * k)) & 1)) continue;  // an element leaves binade e+k by itself: no fold there
        if ((all >> (2 * k + 1)) & 1) {
            const uint64_t d = total[k] >= 0x1p53 ? kTwo53 : uint64_t(total[k]);
            out.d[k][0] = out.d[k][1] = d;
        } else {
            if (!staged) {
#pragma unroll
                for (int j = 0; j < kEPT; ++j) stage[stage_slot(j * kBT + threadIdx.x)] = p[j];
                __syncthreads();
#pragma unroll
                for (int j = 0; j < kEPT; ++j) p[j] = stage[threadIdx.x * kPad + j];
                staged = true;
            }
            const Grid g = grid_of(e + k);
            uint64_t t0 = 0, t1 = 0;
#pragma unroll
            for (int j = 0; j < kEPT; ++j) {
                uint64_t a0, a1, r0, r1;
                elem_map_g(p[j], g, a0, a1);
                compose(t0, t1, a0, a1, r0, r1);
                t0 = r0;
                t1 = r1;
            }
            uint64_t ex0, ex1;
            block_scan_maps(t0, t1, ex0, ex1, sh);
            uint64_t r0, r1;
            compose(ex0, ex1, t0, t1, r0, r1);
            out.d[k][0] = r0;
            out.d[k][1] = r1;
        }
        out.ok |= 1 << k;
    }
    return out;
}

// One CTA per block: the block's probabilities straight into registers
// (coalesced, no staging unless a binade has a tie), then its fold.  Four
// CTAs per SM (64 registers) keep 128 KiB of loads in flight per SM.
__global__ void __launch_bounds__(kBT, 4) k_cdf_summ(const double* __restrict__ prob,
                                                  const int32_t* __restrict__ guess, Summ* __restrict__ summ)
{
    __shared__ uint64_t sh[160];
    const int32_t gs = guess[blockIdx.x];
    if (gs == INT32_MIN) {
        if (threadIdx.x == 0) summ[blockIdx.x] = Summ{{{0, 0}, {0, 0}}, gs, 0};
        return;
    }
    __shared__ double stage[kBT * kPad];
    const double* src = prob + uint64_t(blockIdx.x) * kBS + threadIdx.x;
    double p[kEPT];
#pragma unroll
    for (int j = 0; j < kEPT; ++j) p[j] = src[j * kBT];
    const Summ out = block_summ(p, gs, sh, stage);
    if (threadIdx.x == blockDim.x - 1) summ[blockIdx.x] = out;
}

// blocks composed per thread in one step of the chain (9: a thread's records
// start 45 8-byte words apart, so 16 threads hit 16 distinct bank pairs)
constexpr int kChainPer = 9;
constexpr uint32_t kSpan = uint32_t(kChainPer) * kBT;
// one buffer of k_cdf_chain: a span of fold records copied from a 16-byte
// aligned start (the records start 0 or 8 bytes in), rounded up to 16 bytes
constexpr uint32_t kSpanBuf = uint32_t((size_t(kSpan) * sizeof(Summ) + 32) & ~size_t(15));
constexpr size_t kChainSmem = 2 * size_t(kSpanBuf);
// bytes after the fold records that a rounded-up copy may read (the
// scratch that holds them reserves that much beyond them)
constexpr size_t kSummSlack = 32;
// polls of a bounded wait in k_cdf_chain before it gives up (status 4)
constexpr uint32_t kChainWaitLimit = 1u << 22;
static_assert(sizeof(Summ) % 8 == 0, "fold records are 8-byte aligned");

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

// The fold records summ[base, base + cnt) into buffer buf by bulk copies
// (thread 0; completion counted on bar).  Returns the records' offset in buf.
__device__ __forceinline__ uint32_t summ_fetch(char* buf, const Summ* summ, uint32_t base, uint32_t cnt, uint64_t* bar)
{
    const uint64_t s0 = uint64_t(base) * sizeof(Summ);
    const uint64_t a0 = s0 & ~uint64_t(15);
    const uint32_t skew = uint32_t(s0 - a0);
    const uint32_t bytes = (cnt * uint32_t(sizeof(Summ)) + skew + 15u) & ~15u;
    const char* src = reinterpret_cast<const char*>(summ) + a0;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // earlier reads of buf before the copy's writes
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes) : "memory");
    constexpr uint32_t kPiece = 32768;
    for (uint32_t o = 0; o < bytes; o += kPiece) {
        const uint32_t nbytes = min(kPiece, bytes - o);
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         smem_addr(buf + o)),
                     "l"(src + o), "r"(nbytes), "r"(smem_addr(bar)) : "memory");
    }
    return skew;
}

// waits (every thread) for the phase of bar with the given parity; false
// after kChainWaitLimit polls
__device__ __forceinline__ bool chain_wait(uint64_t* bar, uint32_t parity)
{
    const uint32_t a = smem_addr(bar);
    for (uint32_t i = 0; i < kChainWaitLimit; ++i) {
        uint32_t done;
        asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                     : "=r"(done) : "r"(a), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

// Shared memory of the chain (one CTA) besides the two record buffers.
struct ChainShm {
    uint64_t sh[160];
    double stage[kBT * kPad];
    double c;          // the exact running sum
    int slow;
    uint32_t end;
    __align__(8) uint64_t bar[2];
    uint32_t skew[2];
};

// The record buffers and their copies.  Every thread holds the same copy of
// this state and calls fetch/drain together.
struct ChainIO {
    ChainShm& S;
    char* raw;
    const Summ* summ;
    uint32_t pend[2] = {0, 0};             // copy in flight, per buffer
    uint32_t ph[2] = {0, 0};               // parity of its mbarrier phase
    uint32_t loaded[2] = {~0u, ~0u};       // first block the buffer holds (or will)
    __device__ ChainIO(ChainShm& s, char* r, const Summ* sm) : S(s), raw(r), summ(sm) {}
    __device__ void fetch(uint32_t b, uint32_t from, uint32_t cnt)
    {
        if (threadIdx.x == 0) S.skew[b] = summ_fetch(raw + b * kSpanBuf, summ, from, cnt, &S.bar[b]);
        pend[b] = 1;
        loaded[b] = from;
    }
    // waits for buffer b's copy; uniform result (a copy not seen done stays pending)
    __device__ bool drain(uint32_t b)
    {
        bool ok = true;
        if (pend[b]) ok = chain_wait(&S.bar[b], ph[b]);
        ok = __syncthreads_and(ok) != 0;
        if (pend[b] && ok) {
            ph[b] ^= 1u;
            pend[b] = 0;
        }
        return ok;
    }
    __device__ const Summ* rec(uint32_t b) const { return reinterpret_cast<const Summ*>(raw + b * kSpanBuf + S.skew[b]); }
};

// The exact running sum over blocks [b_begin, b_end), starting from S.c (the
// exact sum before b_begin) and leaving the sum after b_end there; writes
// cin[b_begin, b_end).  Each step takes the next span of up to kSpan blocks
// (kChainPer consecutive per thread): every block up to the first one without
// a fold on the running sum's binade composes with one block-wide scan, and
// the step commits the blocks up to the first one whose sum would leave the
// binade (or the one without a fold).  That block is handled on its own (its
// fold on the binade it actually starts in, else an exact element-by-element
// fold) and the next span starts after it.  The fold records of a span arrive
// in shared memory by bulk copies while the previous span is composed (two
// buffers; a span that stopped early reloads its successor's records; records
// already in buffer 0 for b_begin are used as they are).  A running sum of
// zero is on the grid of binade -1022 (spacing 2^-1074, shared by the
// subnormals), where zero and subnormal blocks fold exactly.  False when a
// bounded wait gave up.
__device__ bool chain_range(ChainIO& io, const double* __restrict__ prob, uint32_t b_begin, uint32_t b_end,
                            double* __restrict__ cin, uint32_t& n_span, uint32_t& n_single, uint32_t& n_exact)
{
    ChainShm& S = io.S;
    const uint32_t t = threadIdx.x;
    uint32_t base = b_begin, cur = 0;
    while (base < b_end) {
        const uint32_t span = min(kSpan, b_end - base);
        if (io.loaded[cur] != base) {   // the first span, or the previous span stopped early
            if (!io.drain(0) || !io.drain(1)) return false;
            io.fetch(cur, base, span);
        }
        const uint32_t next = base + span;
        if (next < b_end) io.fetch(cur ^ 1, next, min(kSpan, b_end - next));
        if (!io.drain(cur)) return false;
        const Summ* rec = io.rec(cur);
        const double c = S.c;
        const int e0 = epoch_of(c);
        const uint32_t p0 = t * kChainPer;           // this thread's first position in the span
        uint64_t d0[kChainPer], d1[kChainPer];
        uint32_t my_bad = span;
#pragma unroll
        for (int k = 0; k < kChainPer; ++k) {
            d0[k] = d1[k] = 0;
            const uint32_t pos = p0 + k;
            if (pos < span && !summ_pick(rec[pos], e0, d0[k], d1[k]) && my_bad == span) my_bad = pos;
        }
        if (t == 0) S.end = span;
        __syncthreads();
        if (my_bad < span) atomicMin(&S.end, my_bad);
        __syncthreads();
        const uint32_t bad = S.end;
        uint64_t m0 = 0, m1 = 0;
#pragma unroll
        for (int k = 0; k < kChainPer; ++k) {
            if (p0 + k >= bad) d0[k] = d1[k] = 0;     // identity from the first block without a fold on
            uint64_t r0, r1;
            compose(m0, m1, d0[k], d1[k], r0, r1);
            m0 = r0;
            m1 = r1;
        }
        uint64_t ex0, ex1;
        if (__syncthreads_and(m0 == m1)) {
            block_scan_add(m0, ex0, S.sh);    // translations only: the prefix is a sum
            ex1 = ex0;
        } else {
            block_scan_maps(m0, m1, ex0, ex1, S.sh);
        }
        const uint64_t C = c > 0.0 ? uint64_t(ldexp(c, 52 - e0)) : 0;
        uint64_t x = C + ((C & 1) ? ex1 : ex0);
        uint64_t xin[kChainPer];
        uint32_t my_over = bad;
#pragma unroll
        for (int k = 0; k < kChainPer; ++k) {
            xin[k] = x;
            x += (x & 1) ? d1[k] : d0[k];
            if (x >= kTwo53 && my_over == bad && p0 + k < bad) my_over = p0 + k;   // the sum leaves the binade here
        }
        if (t == 0) S.end = bad;
        __syncthreads();
        if (my_over < bad) atomicMin(&S.end, my_over);
        __syncthreads();
        const uint32_t end = S.end;
#pragma unroll
        for (int k = 0; k < kChainPer; ++k) {
            const uint32_t pos = p0 + k;
            if (pos < end) cin[base + pos] = ldexp(double(xin[k]), e0 - 52);
            if (pos + 1 == end) S.c = ldexp(double(xin[k] + ((xin[k] & 1) ? d1[k] : d0[k])), e0 - 52);
        }
        if (t == 0 && end > 0) ++n_span;
        __syncthreads();   // every thread is done with rec and S.c before either changes
        if (end >= span) {
            base = next;
            cur ^= 1;   // loaded[cur] == next: fetched above
            continue;
        }
        // block b starts in the running sum's binade but has no fold there or leaves it
        ++n_single;
        const uint32_t b = base + end;
        if (t == 0) {
            double cc = S.c;
            cin[b] = cc;
            const int eb = epoch_of(cc);
            uint64_t b0, b1;
            int slow = 1;
            if (summ_pick(rec[end], eb, b0, b1)) {
                uint64_t Cb = cc > 0.0 ? uint64_t(ldexp(cc, 52 - eb)) : 0;
                uint64_t Co = Cb + ((Cb & 1) ? b1 : b0);
                if (Co < kTwo53 && Co >= Cb) {
                    S.c = ldexp(double(Co), eb - 52);
                    slow = 0;
                }
            }
            S.slow = slow;
        }
        __syncthreads();
        if (S.slow) {
            ++n_exact;
            double p[kEPT];
            load_block_prob(prob, uint64_t(b) * kBS, p, S.stage);
            double cc = block_exact(kBS, S.c, nullptr, S.sh, S.stage);
            if (t == 0) S.c = cc;
        }
        __syncthreads();
        base = b + 1;
    }
    return true;
}

// hand-off between consecutive segments of the chain: the exact sum after a
// segment, valid once flag is 1
struct ChainLink {
    double value;
    uint32_t flag;
    uint32_t pad;
};
// polls of the wait for the previous segment's sum (with a short sleep each)
constexpr uint32_t kLinkWaitLimit = 1u << 24;

// The chain in segments of kSpan blocks, one CTA each, taken in order through
// a ticket (so a segment's predecessor always runs earlier or at the same
// time).  Ahead of knowing its exact incoming sum, a CTA composes its
// segment's folds on the one or two binades its first block's guess allows.
// When the predecessor publishes the exact sum before the segment (link[j -
// 1]), the CTA applies the composed fold of that sum's binade if the whole
// segment stays in it and publishes the sum after the segment at once, so
// the hand-off along the segments costs one fold application each; only
// segments where the sum changes binade (a few dozen in a 2^30-element
// vector) pass their sum on after the sequential range routine.  Every CTA
// then writes its segment's exact block starts with chain_range from the
// exact incoming sum.  Waits are bounded: a CTA that gives up writes 4 to
// *status and publishes nothing, so the ones after it give up too.
// stats (zeroed before the launch): spans, single blocks, exact blocks, blocks.
__global__ void __launch_bounds__(kBT, 1) k_cdf_chain(const double* __restrict__ prob,
                                                   const Summ* __restrict__ summ, uint32_t nb, double* __restrict__ cin,
                                                   uint32_t* __restrict__ stats, unsigned* __restrict__ status,
                                                   ChainLink* __restrict__ link, uint32_t* __restrict__ ticket)
{
    extern __shared__ __align__(16) char sraw[];
    __shared__ ChainShm S;
    __shared__ uint32_t s_seg;
    __shared__ uint64_t s_map[2][2];
    __shared__ int s_mapok[2];
    __shared__ int s_done;
    __shared__ int s_fail;
    const uint32_t t = threadIdx.x;
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&S.bar[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&S.bar[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_seg = atomicAdd(ticket, 1u);
        s_done = 0;
        s_fail = 0;
    }
    __syncthreads();
    const uint32_t j = s_seg;
    const uint32_t b0 = j * kSpan, b1 = min(nb, b0 + kSpan), cnt = b1 - b0;
    ChainIO io(S, sraw, summ);
    uint32_t n_span = 0, n_single = 0, n_exact = 0;
    io.fetch(0, b0, cnt);
    bool ok = io.drain(0);
    if (ok && j > 0) {
        // the segment's fold on each binade its first block may start in
        const Summ* rec = io.rec(0);
        const int32_t eg = rec[0].e;
        for (int kb = 0; kb < 2; ++kb) {
            const int e = eg + kb;
            const uint32_t p0 = t * kChainPer;
            bool valid = eg != INT32_MIN;
            uint64_t m0 = 0, m1 = 0;
#pragma unroll
            for (int k = 0; k < kChainPer; ++k) {
                uint64_t d0 = 0, d1 = 0;
                if (p0 + k < cnt && !summ_pick(rec[p0 + k], e, d0, d1)) valid = false;
                uint64_t r0, r1;
                compose(m0, m1, d0, d1, r0, r1);
                m0 = r0;
                m1 = r1;
            }
            // each thread's fold below 2^53 keeps the block total below 2^61 (no wrap)
            valid = valid && m0 < kTwo53 && m1 < kTwo53;
            if (!__syncthreads_and(valid)) {
                if (t == 0) s_mapok[kb] = 0;
                continue;
            }
            uint64_t ex0, ex1;
            block_scan_maps(m0, m1, ex0, ex1, S.sh);
            if (t == kBT - 1) {
                uint64_t r0, r1;
                compose(ex0, ex1, m0, m1, r0, r1);
                s_map[kb][0] = r0;
                s_map[kb][1] = r1;
                s_mapok[kb] = 1;
            }
        }
        __syncthreads();   // s_map / s_mapok written above
        // the exact sum before the segment, then at once the one after it if
        // the segment's fold on that sum's binade applies
        if (t == 0) {
            volatile uint32_t* f = &link[j - 1].flag;
            uint32_t i = 0;
            while (*f == 0u && i < kLinkWaitLimit) {
                __nanosleep(64);
                ++i;
            }
            if (*f == 0u) {
                s_fail = 1;
            } else {
                __threadfence();
                const double c = *(volatile double*)&link[j - 1].value;
                S.c = c;
                const int e = epoch_of(c);
                const int kb = e - eg;
                if (eg != INT32_MIN && (kb == 0 || kb == 1) && s_mapok[kb]) {
                    const uint64_t C = c > 0.0 ? uint64_t(ldexp(c, 52 - e)) : 0;
                    const uint64_t x = C + ((C & 1) ? s_map[kb][1] : s_map[kb][0]);
                    if (x < kTwo53) {
                        link[j].value = ldexp(double(x), e - 52);
                        __threadfence();
                        *(volatile uint32_t*)&link[j].flag = 1u;
                        s_done = 1;
                    }
                }
            }
        }
        __syncthreads();
        ok = !s_fail;
    } else if (t == 0) {
        S.c = 0.0;
    }
    __syncthreads();
    // the segment's own block starts from the exact incoming sum
    if (ok) ok = chain_range(io, prob, b0, b1, cin, n_span, n_single, n_exact);
    if (ok && t == 0 && !s_done) {
        link[j].value = S.c;
        __threadfence();
        *(volatile uint32_t*)&link[j].flag = 1u;
    }
    // no copy may still be writing shared memory when the CTA leaves
    const bool dr0 = io.drain(0), dr1 = io.drain(1);
    if (!ok || !dr0 || !dr1) {
        if (t == 0) *(volatile unsigned*)status = 4u;
        return;
    }
    if (t == 0) {
        if (b1 == nb) cin[nb] = S.c;
        if (stats) {
            atomicAdd(stats + 0, n_span);
            atomicAdd(stats + 1, n_single);
            atomicAdd(stats + 2, n_exact);
            if (j == 0) stats[3] = nb;
        }
    }
}

__device__ __forceinline__ uint64_t lower_bound_dev(const double* a, uint64_t n, double target)
{
    uint64_t lo = 0, len = n;
    while (len > 0) {
        uint64_t half = len >> 1, mid = lo + half;
        if (a[mid] < target) { lo = mid + 1; len = len - half - 1; }
        else len = half;
    }
    return lo;
}

// ---- shots against the exact block starts, without a cumulative array ----
// The cumulative values are never written to memory: each shot's block is
// found by binary search over the exact block starts cin (a few MB, L2
// resident), the shots are bucketed by block, and every block that holds a
// shot rebuilds its exact cumulative values in shared memory (block_exact,
// the reference's sequential rounding) and answers its shots there.

// target = u * total (StateVector.cpp:100-107's uniform_real_distribution(0, total)),
// block = first b with cin[b + 1] >= target; targets beyond the total answer size
__global__ void k_shot_block(const double* __restrict__ cin, uint32_t nb, const double* __restrict__ u,
                             uint64_t nshots, uint64_t seed, uint64_t size, double* __restrict__ target,
                             uint32_t* __restrict__ blk, uint32_t* __restrict__ count, uint64_t* __restrict__ out)
{
    const double total = cin[nb];
    for (uint64_t s = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; s < nshots;
         s += uint64_t(gridDim.x) * blockDim.x) {
        double us;
        if (u) us = u[s];
        else {
            double u2;
            philox_uniform_pair(seed, s, kTagSample, us, u2);
        }
        const double t = __dadd_rn(__dmul_rn(us, total), 0.0);
        uint64_t lo = 0, len = nb;
        while (len > 0) {
            uint64_t half = len >> 1, mid = lo + half;
            if (cin[mid + 1] < t) { lo = mid + 1; len = len - half - 1; }
            else len = half;
        }
        target[s] = t;
        if (lo >= nb) {
            blk[s] = nb;
            out[s] = size;   // beyond the end: lower_bound returns size
        } else {
            blk[s] = uint32_t(lo);
            atomicAdd(count + lo, 1u);
        }
    }
}

// offset[b] = shots in blocks < b (offset[nb] = all) and the list of blocks
// holding at least one shot, by a three-kernel scan over chunks of kOT blocks:
// chunk sums, an exclusive scan of the chunk sums (one CTA), then each chunk's
// own exclusive scan plus its base
constexpr int kOT = 1024;

// exclusive block-wide scan of two counters (kOT threads)
__device__ __forceinline__ void block_scan2(uint32_t a, uint32_t b, uint32_t& ea, uint32_t& eb, uint32_t& ta,
                                            uint32_t& tb)
{
    __shared__ uint32_t wa[kOT / 32], wb[kOT / 32];
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    uint32_t ia = a, ib = b;   // inclusive within the warp
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t xa = __shfl_up_sync(0xffffffffu, ia, o), xb = __shfl_up_sync(0xffffffffu, ib, o);
        if (lane >= uint32_t(o)) { ia += xa; ib += xb; }
    }
    if (lane == 31u) { wa[w] = ia; wb[w] = ib; }
    __syncthreads();
    if (w == 0) {
        uint32_t va = wa[lane], vb = wb[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t xa = __shfl_up_sync(0xffffffffu, va, o), xb = __shfl_up_sync(0xffffffffu, vb, o);
            if (lane >= uint32_t(o)) { va += xa; vb += xb; }
        }
        wa[lane] = va;   // inclusive over warps
        wb[lane] = vb;
    }
    __syncthreads();
    const uint32_t ba = w ? wa[w - 1] : 0u, bb = w ? wb[w - 1] : 0u;
    ea = ba + ia - a;
    eb = bb + ib - b;
    ta = wa[kOT / 32 - 1];
    tb = wb[kOT / 32 - 1];
    __syncthreads();   // wa / wb are reused by the next call
}

__global__ void __launch_bounds__(kOT) k_scan_part(const uint32_t* __restrict__ count, uint32_t nb,
                                                   uint32_t* __restrict__ psum, uint32_t* __restrict__ pnz)
{
    const uint32_t i = blockIdx.x * kOT + threadIdx.x;
    const uint32_t c = i < nb ? count[i] : 0u;
    uint32_t ea, eb, ta, tb;
    block_scan2(c, c != 0u, ea, eb, ta, tb);
    if (threadIdx.x == 0) {
        psum[blockIdx.x] = ta;
        pnz[blockIdx.x] = tb;
    }
}

// one CTA: the chunk sums become exclusive prefixes (in place); totals to offset[nb] and *nne
__global__ void __launch_bounds__(kOT) k_scan_top(uint32_t* __restrict__ psum, uint32_t* __restrict__ pnz,
                                                  uint32_t nchunks, uint32_t* __restrict__ offset_end,
                                                  uint32_t* __restrict__ nne)
{
    uint32_t carry_a = 0, carry_b = 0;
    for (uint32_t base = 0; base < nchunks; base += kOT) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t a = i < nchunks ? psum[i] : 0u, b = i < nchunks ? pnz[i] : 0u;
        uint32_t ea, eb, ta, tb;
        block_scan2(a, b, ea, eb, ta, tb);
        if (i < nchunks) {
            psum[i] = carry_a + ea;
            pnz[i] = carry_b + eb;
        }
        carry_a += ta;
        carry_b += tb;
    }
    if (threadIdx.x == 0) {
        *offset_end = carry_a;
        *nne = carry_b;
    }
}

__global__ void __launch_bounds__(kOT) k_scan_final(const uint32_t* __restrict__ count, uint32_t nb,
                                                    const uint32_t* __restrict__ psum, const uint32_t* __restrict__ pnz,
                                                    uint32_t* __restrict__ offset, uint32_t* __restrict__ nonempty)
{
    const uint32_t i = blockIdx.x * kOT + threadIdx.x;
    const uint32_t c = i < nb ? count[i] : 0u;
    uint32_t ea, eb, ta, tb;
    block_scan2(c, c != 0u, ea, eb, ta, tb);
    if (i < nb) {
        offset[i] = psum[blockIdx.x] + ea;
        if (c) nonempty[pnz[blockIdx.x] + eb] = i;
    }
}

__global__ void k_shot_scatter(const uint32_t* __restrict__ blk, uint64_t nshots, uint32_t nb,
                               const uint32_t* __restrict__ offset, uint32_t* __restrict__ cursor,
                               uint32_t* __restrict__ order)
{
    for (uint64_t s = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; s < nshots;
         s += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t b = blk[s];
        if (b < nb) order[offset[b] + atomicAdd(cursor + b, 1u)] = uint32_t(s);
    }
}

// A few shots (a measure(), a short sample): one CTA per shot finds the shot's
// block, rebuilds that block's exact cumulative values in shared memory and
// answers the shot -- no bucketing pass over every block.
__global__ void __launch_bounds__(kBT) k_search_each(const double* __restrict__ cin, const double* __restrict__ prob,
                                                     uint32_t nb, const double* __restrict__ u, uint64_t seed,
                                                     uint64_t size, uint64_t* __restrict__ out)
{
    __shared__ uint64_t sh[160];
    __shared__ double s_t;
    __shared__ uint32_t s_b;
    extern __shared__ double stg[];
    double* const cum = stg + kBT * kPad;
    const uint64_t s = blockIdx.x;
    if (threadIdx.x == 0) {
        double us;
        if (u) us = u[s];
        else {
            double u2;
            philox_uniform_pair(seed, s, kTagSample, us, u2);
        }
        const double t = __dadd_rn(__dmul_rn(us, cin[nb]), 0.0);
        uint64_t lo = 0, len = nb;
        while (len > 0) {
            uint64_t half = len >> 1, mid = lo + half;
            if (cin[mid + 1] < t) { lo = mid + 1; len = len - half - 1; }
            else len = half;
        }
        s_t = t;
        s_b = uint32_t(lo);
    }
    __syncthreads();
    const uint32_t b = s_b;
    if (b >= nb) {
        if (threadIdx.x == 0) out[s] = size;   // beyond the end: lower_bound returns size
        return;
    }
    stage_async(stg, prob, uint64_t(b) * kBS);
    stage_wait<0>();
    __syncthreads();
    block_exact(kBS, cin[b], cum, sh, stg);
    __syncthreads();
    if (threadIdx.x == 0) out[s] = uint64_t(b) * kBS + lower_bound_dev(cum, kBS, s_t);
}
constexpr size_t kEachSmem = (size_t(kBT) * kPad + kBS) * sizeof(double);
constexpr size_t kFewShots = 64;

// shared memory of k_block_search: two staging buffers + one block's cumulative values
constexpr size_t kSearchSmem = kStage2 + size_t(kBS) * sizeof(double);

// Persistent over the blocks that hold shots (blockIdx.x, +gridDim.x, ... of
// the non-empty list): the next block's probabilities stream into the other
// staging buffer while this block's exact cumulative values are built in
// shared memory and its shots answered by lower_bound there.
__global__ void __launch_bounds__(kBT, kWriteCTAs) k_block_search(const double* __restrict__ cin,
                                                                  const double* __restrict__ prob,
                                                                  const uint32_t* __restrict__ nonempty,
                                                                  const uint32_t* __restrict__ nne,
                                                                  const uint32_t* __restrict__ offset,
                                                                  const uint32_t* __restrict__ order,
                                                                  const double* __restrict__ target,
                                                                  uint64_t* __restrict__ out)
{
    __shared__ uint64_t sh[160];
    extern __shared__ double stg[];
    double* const cum = stg + 2 * (kBT * kPad);
    const uint32_t n = *nne;
    uint32_t k = blockIdx.x;
    if (k >= n) return;
    stage_async(stg, prob, uint64_t(nonempty[k]) * kBS);
    for (uint32_t it = 0; k < n; k += gridDim.x, ++it) {
        double* cur = stg + (it & 1) * (kBT * kPad);
        const uint32_t kn = k + gridDim.x;
        if (kn < n) {
            stage_async(stg + ((it + 1) & 1) * (kBT * kPad), prob, uint64_t(nonempty[kn]) * kBS);
            stage_wait<1>();
        } else {
            stage_wait<0>();
        }
        __syncthreads();
        const uint32_t b = nonempty[k];
        block_exact(kBS, cin[b], cum, sh, cur);
        __syncthreads();
        for (uint32_t i = offset[b] + threadIdx.x; i < offset[b + 1]; i += kBT) {
            const uint32_t s = order[i];
            out[s] = uint64_t(b) * kBS + lower_bound_dev(cum, kBS, target[s]);
        }
        __syncthreads();  // cur is refilled by the next iteration's prefetch, cum by the next block
    }
}

// small states (< one block): the sequential chain itself
__global__ void k_cdf_small(const double2* __restrict__ amp, uint64_t size, PermMap pm, double* cdf, double* cin)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double c = 0.0;
    for (uint64_t i = 0; i < size; ++i) {
        c = __dadd_rn(c, norm2(amp[phys_index(i, pm)]));
        cdf[i] = c;
    }
    cin[0] = 0.0;
    cin[1] = c;
}

// shots: target = u * total; block by binary search over block starts, then inside the block
__global__ void k_sample(const double* __restrict__ cdf, uint64_t size, const double* __restrict__ cin, uint32_t nb,
                         uint32_t bs, const double* __restrict__ u, uint64_t nshots, uint64_t seed,
                         uint64_t* __restrict__ out, PermMap pm)
{
    const double total = cin[nb];
    for (uint64_t s = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; s < nshots;
         s += uint64_t(gridDim.x) * blockDim.x) {
        double us;
        if (u) us = u[s];
        else {
            double u2;
            philox_uniform_pair(seed, s, kTagSample, us, u2);
        }
        double target = __dadd_rn(__dmul_rn(us, total), 0.0);
        // last block whose first value could be >= target: search on block ends
        // block b's last value is cin[b+1]; find first b with cin[b+1] >= target
        uint64_t lo = 0, len = nb;
        while (len > 0) {
            uint64_t half = len >> 1, mid = lo + half;
            if (cin[mid + 1] < target) { lo = mid + 1; len = len - half - 1; }
            else len = half;
        }
        uint64_t idx;
        if (lo >= nb) idx = size;  // beyond the end: lower_bound returns size
        else {
            uint64_t base = lo * bs;
            uint64_t cnt = min(uint64_t(bs), size - base);
            idx = base + lower_bound_dev(cdf + base, cnt, target);
        }
        out[s] = idx;
    }
    (void)pm;
}

PermMap make_perm(const qse_state* st)
{
    PermMap pm{};
    pm.n = st->n;
    pm.identity = st->identity_perm() ? 1 : 0;
    for (uint32_t q = 0; q < st->n; ++q) pm.p[q] = uint8_t(st->perm[q]);
    return pm;
}

// The exact sampling tables of a state: states of at least one block (4096
// amplitudes) keep the probabilities in logical order (cdf) and the exact
// cumulative value before every block (cin, nb + 1 values); smaller states
// keep the whole cumulative array (cdf) with cin = {0, total}.
struct CdfView {
    double* cdf;
    double* cin;
    uint32_t nb;
    uint32_t bs;
};

// Tile of the gather: physical bits 0..4 and the physical images of logical
// bits 0..6, padded with the lowest remaining physical bits to 12 (n >= 12).
GatherPlan make_gather(const qse_state* st)
{
    GatherPlan g{};
    uint64_t S = 0x1Full;
    for (uint32_t q = 0; q < 7; ++q) S |= uint64_t(1) << st->perm[q];
    for (uint32_t q = 0; q < st->n && __builtin_popcountll(S) < 12; ++q) S |= uint64_t(1) << q;
    for (uint32_t q = 0; q < st->n; ++q) g.inv[st->perm[q]] = uint8_t(q);
    int b = 0;
    for (uint32_t q = 0; q < st->n; ++q)
        if ((S >> q) & 1) g.sphys[b++] = uint8_t(q);
    uint64_t Slog = 0;
    for (int i = 0; i < 12; ++i) Slog |= uint64_t(1) << g.inv[g.sphys[i]];
    b = 0;
    for (uint32_t q = 0; q < st->n; ++q)
        if ((Slog >> q) & 1) g.slog[b++] = uint8_t(q);
    for (int i = 0; i < 12; ++i) {
        const uint32_t phys = st->perm[g.slog[i]];
        for (int r = 0; r < 12; ++r)
            if (g.sphys[r] == phys) g.wsrc[i] = uint8_t(r);
    }
    // slot images: read-order bits 0..3 keep their place; bits >= 4 get a low
    // nibble chosen so that the read side's half-warp bits (the read-order
    // images of write-order bits 0..3) span all 16 low-nibble values
    uint32_t low[12] = {0};
    uint64_t rng = 0x2545F4914F6CDD1Dull;
    for (int attempt = 0; attempt < 4096; ++attempt) {
        uint32_t cand[12] = {0};
        for (int r = 4; r < 12; ++r) {
            rng ^= rng << 13; rng ^= rng >> 7; rng ^= rng << 17;
            cand[r] = attempt ? uint32_t(rng >> 60) : 0u;
        }
        // rank over GF(2) of the 4 read-side images
        uint32_t basis[4] = {0, 0, 0, 0};
        int rank = 0;
        for (int i = 0; i < 4; ++i) {
            const int r = g.wsrc[i];
            uint32_t v = r < 4 ? (1u << r) : cand[r];
            for (int k = 3; k >= 0 && v; --k)
                if ((v >> k) & 1) {
                    if (basis[k]) v ^= basis[k];
                    else { basis[k] = v; ++rank; v = 0; }
                }
        }
        if (rank == 4) {
            std::copy(cand, cand + 12, low);
            break;
        }
    }
    for (int r = 0; r < 12; ++r) g.img[r] = uint16_t((1u << r) ^ low[r]);
    const uint64_t all = st->n >= 64 ? ~uint64_t(0) : ((uint64_t(1) << st->n) - 1);
    g.outer_mask = all & ~S;
    return g;
}

// Exact sampling tables of the current amplitudes, cached per state until the
// amplitudes change (sample() followed by measure() builds them once).
CdfView build_cdf(qse_state* st)
{
    materialize(st);
    qse_ctx* ctx = st->ctx;
    const uint64_t size = st->size();
    // this state is sampled: its next executes also write the probabilities
    // (the last pass's side output), which this call consumes if they are current
    st->prob_hint = true;
    st->prob_pending = false;
    if (st->cdf_version == st->version)
        return CdfView{st->cdf_values, st->cdf_block_start, st->cdf_nb, st->cdf_bs};
    PermMap pm = make_perm(st);
    CdfView v{};
    const double2* amp = reinterpret_cast<const double2*>(st->amp);
    if (size < uint64_t(kBS)) {
        st->cdf.reserve(size * 8 + 4 * 8);
        v.cdf = static_cast<double*>(st->cdf.ptr);
        v.cin = v.cdf + size;
        v.nb = 1;
        v.bs = uint32_t(size);
        k_cdf_small<<<1, 32, 0, ctx->stream>>>(amp, size, pm, v.cdf, v.cin);
        QSE_CUDA(cudaGetLastError());
        count_launch(ctx);
    } else {
        const uint32_t nb = uint32_t(size / kBS);
        // state-owned: probabilities [size] | bsum [nb] | cin [nb+1] | stats;
        // context scratch: guess [nb] | summ [nb] | group sums
        st->cdf.reserve(prob_buffer_bytes(size));
        v.cdf = static_cast<double*>(st->cdf.ptr);
        double* bsum = v.cdf + size;
        v.cin = bsum + nb;
        size_t off_summ = (size_t(nb) * 4 + 15) & ~size_t(15);
        size_t off_gtot = off_summ + size_t(nb) * sizeof(Summ);
        size_t off_link = (off_gtot + (size_t(nb) / kGT + 1) * 8 + 15) & ~size_t(15);
        size_t off_ticket = off_link + size_t((nb + kSpan - 1) / kSpan) * sizeof(ChainLink);
        ctx->scratch2.reserve(off_ticket + 16 + kSummSlack);
        char* base = static_cast<char*>(ctx->scratch2.ptr);
        int32_t* guess = reinterpret_cast<int32_t*>(base);
        Summ* summ = reinterpret_cast<Summ*>(base + off_summ);
        double* gtot = reinterpret_cast<double*>(base + off_gtot);
        v.nb = nb;
        v.bs = kBS;
        // probabilities in logical order and the block sums: written by the
        // execute's last pass when current (prob_version), else gathered here
        if (st->prob_version == st->version) {
            if (!st->prob_bsum) {
                k_block_sums<<<nb, kBT, 0, ctx->stream>>>(v.cdf, bsum);
                count_launch(ctx);
            }
        } else if (pm.identity) {
            k_prob_identity<<<nb, kBT, 0, ctx->stream>>>(amp, v.cdf, bsum);
            count_launch(ctx);
        } else {
            GatherPlan g = make_gather(st);
            QSE_CUDA(cudaMemsetAsync(bsum, 0, size_t(nb) * 8, ctx->stream));
            k_prob_gather<<<unsigned(size / kBS), kBT, 0, ctx->stream>>>(amp, v.cdf, bsum, g);
            count_launch(ctx);
        }
        const uint32_t ng = (nb + kGT - 1) / kGT;
        const uint32_t nseg = (nb + kSpan - 1) / kSpan;
        k_guess_part<<<ng, kGT, 0, ctx->stream>>>(bsum, nb, gtot);
        k_guess_fin<<<ng, kGT, 0, ctx->stream>>>(bsum, nb, gtot, guess);
        k_cdf_summ<<<nb, kBT, 0, ctx->stream>>>(v.cdf, guess, summ);
        ChainLink* link = reinterpret_cast<ChainLink*>(base + off_link);
        uint32_t* ticket = reinterpret_cast<uint32_t*>(base + off_ticket);
        uint32_t* stats = reinterpret_cast<uint32_t*>(v.cin + nb + 1);
        QSE_CUDA(cudaMemsetAsync(link, 0, off_ticket + 16 - off_link, ctx->stream));
        QSE_CUDA(cudaMemsetAsync(stats, 0, 16, ctx->stream));
        QSE_CUDA(cudaFuncSetAttribute(k_cdf_chain, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kChainSmem)));
        k_cdf_chain<<<nseg, kBT, kChainSmem, ctx->stream>>>(v.cdf, summ, nb, v.cin, stats, ctx->status_dev, link,
                                                           ticket);
        QSE_CUDA(cudaGetLastError());
        count_launch(ctx, 4);
        // the array keeps the probabilities: shots rebuild the cumulative values
        // of their blocks in shared memory (sample_blocks)
    }
    st->cdf_values = v.cdf;
    st->cdf_block_start = v.cin;
    st->cdf_nb = v.nb;
    st->cdf_bs = v.bs;
    st->cdf_version = st->version;
    return v;
}

}  // namespace

namespace {
size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

// Outcomes of nshots draws (device uniforms d_u, or Philox(seed) when null)
// into d_out.  `scratch` must hold sample_scratch_bytes(nb, nshots) bytes.
size_t sample_scratch_bytes(uint32_t nb, size_t nshots)
{
    const size_t nchunks = (size_t(nb) + kOT - 1) / kOT;
    return align16(nshots * 8) + 2 * align16(nshots * 4) + 2 * align16((size_t(nb) + 1) * 4) +
           align16((size_t(nb) + 2) * 4) + align16(size_t(nb) * 4 + 4) + align16(4) + 2 * align16(nchunks * 4) + 16;
}

void sample_on(qse_state* st, const CdfView& v, const double* d_u, size_t nshots, uint64_t seed, uint64_t* d_out,
               char* scratch)
{
    qse_ctx* ctx = st->ctx;
    const unsigned grid = unsigned(std::min<uint64_t>((nshots + 255) / 256, uint64_t(ctx->num_sms) * 8));
    if (st->size() < uint64_t(kBS)) {   // small state: the whole cumulative array
        k_sample<<<grid, 256, 0, ctx->stream>>>(v.cdf, st->size(), v.cin, v.nb, v.bs, d_u, nshots, seed, d_out,
                                                make_perm(st));
        QSE_CUDA(cudaGetLastError());
        count_launch(ctx);
        return;
    }
    const uint32_t nb = v.nb;
    if (nshots <= kFewShots) {
        QSE_CUDA(cudaFuncSetAttribute(k_search_each, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kEachSmem)));
        k_search_each<<<unsigned(nshots), kBT, kEachSmem, ctx->stream>>>(v.cin, v.cdf, nb, d_u, seed, st->size(), d_out);
        QSE_CUDA(cudaGetLastError());
        count_launch(ctx);
        return;
    }
    const uint32_t nchunks = (nb + kOT - 1) / kOT;
    char* p = scratch;
    auto take = [&](size_t bytes) { char* q = p; p += align16(bytes); return q; };
    double* target = reinterpret_cast<double*>(take(nshots * 8));
    uint32_t* blk = reinterpret_cast<uint32_t*>(take(nshots * 4));
    uint32_t* order = reinterpret_cast<uint32_t*>(take(nshots * 4));
    uint32_t* count = reinterpret_cast<uint32_t*>(take((size_t(nb) + 1) * 4));
    uint32_t* cursor = reinterpret_cast<uint32_t*>(take((size_t(nb) + 1) * 4));
    uint32_t* offset = reinterpret_cast<uint32_t*>(take((size_t(nb) + 2) * 4));
    uint32_t* nonempty = reinterpret_cast<uint32_t*>(take(size_t(nb) * 4 + 4));
    uint32_t* nne = reinterpret_cast<uint32_t*>(take(4));
    uint32_t* psum = reinterpret_cast<uint32_t*>(take(size_t(nchunks) * 4));
    uint32_t* pnz = reinterpret_cast<uint32_t*>(take(size_t(nchunks) * 4));
    // count and cursor are adjacent: one clear
    QSE_CUDA(cudaMemsetAsync(count, 0, reinterpret_cast<char*>(offset) - reinterpret_cast<char*>(count), ctx->stream));
    k_shot_block<<<grid, 256, 0, ctx->stream>>>(v.cin, nb, d_u, nshots, seed, st->size(), target, blk, count, d_out);
    k_scan_part<<<nchunks, kOT, 0, ctx->stream>>>(count, nb, psum, pnz);
    k_scan_top<<<1, kOT, 0, ctx->stream>>>(psum, pnz, nchunks, offset + nb, nne);
    k_scan_final<<<nchunks, kOT, 0, ctx->stream>>>(count, nb, psum, pnz, offset, nonempty);
    k_shot_scatter<<<grid, 256, 0, ctx->stream>>>(blk, nshots, nb, offset, cursor, order);
    // the attribute belongs to the current device: set on every call
    QSE_CUDA(cudaFuncSetAttribute(k_block_search, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSearchSmem)));
    const unsigned pgrid = unsigned(std::min<uint64_t>(std::min<uint64_t>(nb, nshots), uint64_t(ctx->num_sms) * kWriteCTAs));
    k_block_search<<<pgrid, kBT, kSearchSmem, ctx->stream>>>(v.cin, v.cdf, nonempty, nne, offset, order, target, d_out);
    QSE_CUDA(cudaGetLastError());
    count_launch(ctx, 6);
}
}  // namespace

void sample(qse_state* st, const double* u_host, size_t nshots, uint64_t seed, uint64_t* out_host)
{
    qse_ctx* ctx = st->ctx;
    if (nshots == 0) return;
    CdfView v = build_cdf(st);
    // scratch: u [nshots] | out [nshots] | the bucketing tables
    const size_t ubytes = u_host ? align16(nshots * 8) : 0;
    const size_t obytes = align16(nshots * 8);
    ctx->scratch.reserve(ubytes + obytes + sample_scratch_bytes(v.nb, nshots));
    char* base = static_cast<char*>(ctx->scratch.ptr);
    double* d_u = u_host ? reinterpret_cast<double*>(base) : nullptr;
    uint64_t* d_out = reinterpret_cast<uint64_t*>(base + ubytes);
    if (u_host) QSE_CUDA(cudaMemcpyAsync(d_u, u_host, nshots * 8, cudaMemcpyHostToDevice, ctx->stream));
    sample_on(st, v, d_u, nshots, seed, d_out, base + ubytes + obytes);
    QSE_CUDA(cudaMemcpyAsync(out_host, d_out, nshots * 8, cudaMemcpyDeviceToHost, ctx->stream));
    QSE_CUDA(cudaStreamSynchronize(ctx->stream));
}

void sample_device(qse_state* st, const double* d_u, size_t nshots, uint64_t seed, uint64_t* d_out)
{
    qse_ctx* ctx = st->ctx;
    if (nshots == 0) return;
    CdfView v = build_cdf(st);
    ctx->scratch.reserve(sample_scratch_bytes(v.nb, nshots));
    sample_on(st, v, d_u, nshots, seed, d_out, static_cast<char*>(ctx->scratch.ptr));
}

uint64_t measure(qse_state* st, double u)
{
    uint64_t idx = 0;
    sample(st, &u, 1, 0, &idx);
    // StateVector.cpp:142-149: every amplitude 0, the outcome 1 (no phase kept).
    // Recorded, not written: the next fused execute generates the basis state in
    // its first pass, a reset discards it, any other reader writes it first.
    uint64_t L = idx < st->size() ? idx : 0;
    mark_basis(st, logical_to_physical_index(st, L));
    return L;
}

double total_probability(qse_state* st)
{
    CdfView v = build_cdf(st);
    double t = 0.0;
    QSE_CUDA(cudaMemcpyAsync(&t, v.cin + v.nb, 8, cudaMemcpyDeviceToHost, st->ctx->stream));
    QSE_CUDA(cudaStreamSynchronize(st->ctx->stream));
    return t;
}

}  // namespace qse

namespace qse {
// the state's sampling buffer: probabilities [size] | block sums [size/4096] |
// exact block starts [size/4096 + 1] | scan statistics (16 B)
size_t prob_buffer_bytes(uint64_t size)
{
    const size_t nb = size_t(size / kBS);
    return size_t(size) * 8 + nb * 8 + (nb + 1) * 8 + 16;
}
}  // namespace qse

namespace qse {
// chain statistics of the last exact scan of st: spans, single blocks,
// blocks folded exactly, blocks (zeros for states below one block)
void sampler_stats(qse_state* st, uint32_t out[4])
{
    st->cdf_version = ~uint64_t(0);
    CdfView v = build_cdf(st);
    std::memset(out, 0, 16);
    if (v.nb > 1 || st->size() >= uint64_t(kBS))
        QSE_CUDA(cudaMemcpyAsync(out, v.cin + v.nb + 1, 16, cudaMemcpyDeviceToHost, st->ctx->stream));
    QSE_CUDA(cudaStreamSynchronize(st->ctx->stream));
}
}  // namespace qse
