// tile_dev.cuh -- device side of the tile-program interpreter, shared by the
// per-pass kernel (tile.cu) and the batched persistent kernel (batch.cu).
//
// A thread holds R = 2^RB amplitudes of each of NS states in registers: the RB
// "register" tile bits of the current layout select the register, the other
// tile bits are the thread index.  run_ops() executes one pass program (the
// KOp list of planner.h) on them; K_TRANSPOSE exchanges the tile through
// shared memory with an XOR-swizzled slot map.
#pragma once

#include <cuda_runtime.h>

#include "planner.h"

namespace qse {
namespace tile {
namespace dev {

using plan::KOp;

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// Im(conj(l) * s), Re(conj(l) * s)
__device__ __forceinline__ double im_ls(double2 l, double2 s) { return l.x * s.y - l.y * s.x; }
__device__ __forceinline__ double re_ls(double2 l, double2 s) { return l.x * s.x + l.y * s.y; }

template <int R, int P, class F>
__device__ __forceinline__ void pairs_at(double2 (&a)[R], F& f)
{
#pragma unroll
    for (int j = 0; j < R; ++j)
        if (!(j & (1 << P))) f(a[j], a[j | (1 << P)], j);
}

template <int RB, class F>
__device__ __forceinline__ void pairs(int p, double2 (&a)[1 << RB], F& f)
{
    constexpr int R = 1 << RB;
    switch (p) {
    case 0: pairs_at<R, 0>(a, f); break;
    case 1: pairs_at<R, 1>(a, f); break;
    case 2: pairs_at<R, 2>(a, f); break;
    default:
        if constexpr (RB > 3) pairs_at<R, 3>(a, f);
        break;
    }
}

template <int R, int P, class F>
__device__ __forceinline__ void pairs2_at(const double2 (&s)[R], const double2 (&l)[R], F& f)
{
#pragma unroll
    for (int j = 0; j < R; ++j)
        if (!(j & (1 << P))) f(s[j], s[j | (1 << P)], l[j], l[j | (1 << P)]);
}

template <int RB, class F>
__device__ __forceinline__ void pairs2(int p, const double2 (&s)[1 << RB], const double2 (&l)[1 << RB], F& f)
{
    constexpr int R = 1 << RB;
    switch (p) {
    case 0: pairs2_at<R, 0>(s, l, f); break;
    case 1: pairs2_at<R, 1>(s, l, f); break;
    case 2: pairs2_at<R, 2>(s, l, f); break;
    default:
        if constexpr (RB > 3) pairs2_at<R, 3>(s, l, f);
        break;
    }
}

struct OpH {
    __device__ void operator()(double2& v0, double2& v1, int) const
    {
        double2 a = v0, b = v1;
        v0 = make_double2(a.x + b.x, a.y + b.y);
        v1 = make_double2(a.x - b.x, a.y - b.y);
    }
};
struct OpX {
    int f;
    __device__ void operator()(double2& v0, double2& v1, int j) const
    {
        if ((j & f) == f) { double2 t = v0; v0 = v1; v1 = t; }
    }
};
struct OpY {
    int f;
    __device__ void operator()(double2& v0, double2& v1, int j) const
    {
        if ((j & f) == f) {
            double2 a = v0, b = v1;
            v0 = make_double2(b.y, -b.x);
            v1 = make_double2(-a.y, a.x);
        }
    }
};
struct OpRX {
    double c, s;
    __device__ void operator()(double2& v0, double2& v1, int) const
    {
        double2 a = v0, b = v1;
        v0 = make_double2(c * a.x + s * b.y, c * a.y - s * b.x);
        v1 = make_double2(s * a.y + c * b.x, c * b.y - s * a.x);
    }
};
struct OpRY {
    double c, s;
    __device__ void operator()(double2& v0, double2& v1, int) const
    {
        double2 a = v0, b = v1;
        v0 = make_double2(c * a.x - s * b.x, c * a.y - s * b.y);
        v1 = make_double2(s * a.x + c * b.x, s * a.y + c * b.y);
    }
};
struct OpU {
    double2 g00, g01, g10, g11;
    int f;
    __device__ void operator()(double2& v0, double2& v1, int j) const
    {
        if ((j & f) == f) {
            double2 a = v0, b = v1;
            double2 x = cmul(g00, a), y = cmul(g01, b), z = cmul(g10, a), w = cmul(g11, b);
            v0 = make_double2(x.x + y.x, x.y + y.y);
            v1 = make_double2(z.x + w.x, z.y + w.y);
        }
    }
};
// multiply the bit-p-set half by e
struct OpPhase1 {
    double2 e;
    __device__ void operator()(double2&, double2& v1, int) const { v1 = cmul(v1, e); }
};

template <int R, int F>
__device__ __forceinline__ void phase_pattern(double2 (&a)[R], double2 e)
{
#pragma unroll
    for (int j = 0; j < R; ++j)
        if ((j & F) == F) a[j] = cmul(a[j], e);
}

template <int RB>
__device__ __forceinline__ void phase_masked(int f, double2 (&a)[1 << RB], double2 e)
{
    constexpr int R = 1 << RB;
    switch (f) {
    case 1: phase_pattern<R, 1>(a, e); break;
    case 2: phase_pattern<R, 2>(a, e); break;
    case 4: phase_pattern<R, 4>(a, e); break;
    case 3: phase_pattern<R, 3>(a, e); break;
    case 5: phase_pattern<R, 5>(a, e); break;
    case 6: phase_pattern<R, 6>(a, e); break;
    case 7: phase_pattern<R, 7>(a, e); break;
    default:
        if constexpr (RB > 3) {
            switch (f) {
            case 8: phase_pattern<R, 8>(a, e); break;
            case 9: phase_pattern<R, 9>(a, e); break;
            case 10: phase_pattern<R, 10>(a, e); break;
            case 11: phase_pattern<R, 11>(a, e); break;
            case 12: phase_pattern<R, 12>(a, e); break;
            case 13: phase_pattern<R, 13>(a, e); break;
            case 14: phase_pattern<R, 14>(a, e); break;
            case 15: phase_pattern<R, 15>(a, e); break;
            default:
#pragma unroll
                for (int j = 0; j < R; ++j)
                    if ((j & f) == f) a[j] = cmul(a[j], e);
            }
        } else {
#pragma unroll
            for (int j = 0; j < R; ++j)
                if ((j & f) == f) a[j] = cmul(a[j], e);
        }
    }
}

// sum over the lanes of a warp; blocks smaller than a warp (tiny states) use
// only their own lanes in the mask and only partner offsets inside the block
__device__ __forceinline__ double warp_sum(double v)
{
    const uint32_t nb = blockDim.x;
    const unsigned mask = nb >= 32 ? 0xffffffffu : ((1u << nb) - 1u);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        if (uint32_t(o) < nb) v += __shfl_xor_sync(mask, v, o);
    return v;
}

template <int RB>
struct LayoutState {
    int reg[RB];                     // tile-local bits in registers
    uint64_t rg[RB];                 // their physical masks
    uint64_t gbase;                  // physical index of register 0 of this thread
    const plan::LayoutRec* rec;      // thread-bit list of the layout
};

template <int RB>
__device__ __forceinline__ void load_layout(LayoutState<RB>& L, const plan::LayoutRec* rec, const uint8_t* tphys,
                                            uint32_t /*k*/, uint64_t obase, uint32_t tid)
{
    L.rec = rec;
#pragma unroll
    for (int i = 0; i < RB; ++i) {
        L.reg[i] = rec->reg[i];
        L.rg[i] = uint64_t(1) << tphys[L.reg[i]];
    }
    uint64_t g = obase;
    const uint32_t nthr = rec->nthr;
    for (uint32_t t = 0; t < nthr; ++t)
        if ((tid >> t) & 1u) g |= uint64_t(1) << tphys[rec->thr[t]];
    L.gbase = g;
}

// shared-memory slot of register 0 and per-register-bit slot images under map Lm
template <int RB>
__device__ __forceinline__ uint32_t slot_base(const LayoutState<RB>& L, const uint16_t* Lm, uint32_t /*k*/,
                                              uint32_t tid, uint32_t (&sreg)[RB])
{
    uint32_t sb = 0;
    const plan::LayoutRec* r = L.rec;
    const uint32_t nthr = r->nthr;
    for (uint32_t t = 0; t < nthr; ++t)
        if ((tid >> t) & 1u) sb ^= Lm[r->thr[t]];
#pragma unroll
    for (int i = 0; i < RB; ++i) sreg[i] = Lm[L.reg[i]];
    return sb;
}

template <int RB>
__device__ __forceinline__ uint64_t gidx(const LayoutState<RB>& L, int j)
{
    uint64_t idx = L.gbase;
#pragma unroll
    for (int i = 0; i < RB; ++i)
        if ((j >> i) & 1) idx |= L.rg[i];
    return idx;
}

template <int RB>
__device__ __forceinline__ uint32_t sidx(uint32_t sb, const uint32_t (&sreg)[RB], int j)
{
    uint32_t s = sb;
#pragma unroll
    for (int i = 0; i < RB; ++i)
        if ((j >> i) & 1) s ^= sreg[i];
    return s;
}

template <int RB, int NS>
__device__ __forceinline__ void flush_reg(int p, double (&acc)[RB], double2 (&a)[NS][1 << RB], int nact)
{
    double v = 0.0;
#pragma unroll
    for (int i = 0; i < RB; ++i)
        if (i == p) { v = acc[i]; acc[i] = 0.0; }
    if (v != 0.0) {
        double s, c;
        sincos(v, &s, &c);
        OpPhase1 ph{make_double2(c, s)};
#pragma unroll
        for (int st = 0; st < NS; ++st)
            if (st < nact) pairs<RB>(p, a[st], ph);
    }
}

// Outer bits of tile `c` (the bits of c spread over the set bits of outer_mask).
__device__ __forceinline__ uint64_t tile_base(uint64_t c, uint64_t outer_mask)
{
    uint64_t obase = 0, m = outer_mask;
    while (m && c) {
        uint32_t b = __ffsll((long long)m) - 1;
        m &= m - 1;
        if (c & 1) obase |= uint64_t(1) << b;
        c >>= 1;
    }
    return obase;
}

// Per-CTA value of every diagonal group of a pass: the sum of the angles of
// its terms whose outer condition holds for this tile, in term order; direct
// groups store (cos, sin) of the sum, accumulator groups the sum itself.
__device__ __forceinline__ void group_values(const plan::GroupRec* __restrict__ groups, uint32_t ngroups,
                                             const plan::TermRec* __restrict__ terms, uint64_t obase, double2* gval)
{
    for (uint32_t g = threadIdx.x; g < ngroups; g += blockDim.x) {
        const plan::GroupRec gr = groups[g];
        double th = 0.0;
        for (uint32_t i = 0; i < gr.count; ++i) {
            const plan::TermRec t = terms[gr.first + i];
            if ((obase & t.ocond) == t.ocond) th += t.theta;
        }
        if (gr.direct) {
            double s, c;
            sincos(th, &s, &c);
            gval[g] = make_double2(c, s);
        } else {
            gval[g] = make_double2(th, 0.0);
        }
    }
}

// Everything run_ops needs besides the registers.
struct OpsEnv {
    const KOp* ops;
    uint32_t nops;
    const plan::LayoutRec* layouts;   // layout indices of the program are relative to this
    const double* mats;               // K_U matrix indices are relative to this
    const uint8_t* tile_phys;         // shared-memory copy of the pass's tile qubits
    uint32_t k;
    uint64_t obase;
    double2* xbuf;                    // 2^k slots
    const double2* gval;              // group values of this CTA
    double* wpart;                    // [slot][warp] gradient partials (NS == 2)
    uint32_t nwarps;
};

// Executes a pass program on the registers a[NS][R].  nact states take part
// (1: only |psi>, forward; NS: the adjoint sweep on |psi> and |lambda>).
// Threads with active == false hold zeros, never touch the exchange buffer
// and add nothing to the gradient partials; they only join the barriers
// (a CTA wider than the tile of a small state).
template <int RB, int NS>
__device__ __forceinline__ void run_ops(const OpsEnv& E, LayoutState<RB>& L, double2 (&a)[NS][1 << RB], int nact,
                                        bool active)
{
    constexpr int R = 1 << RB;
    const uint32_t tid = threadIdx.x;
    const uint32_t warp = tid >> 5, lane = tid & 31;
    double acc_thr = 0.0;
    double acc[RB];
#pragma unroll
    for (int i = 0; i < RB; ++i) acc[i] = 0.0;

    KOp nxt = E.nops ? E.ops[0] : KOp{};
    for (uint32_t i = 0; i < E.nops; ++i) {
        const KOp op = nxt;
        if (i + 1 < E.nops) nxt = E.ops[i + 1];  // in flight while this op executes
        const bool tc = (tid & op.tcond) == op.tcond;
        switch (op.kind) {
        case plan::K_H: {
            OpH f;
#pragma unroll
            for (int st = 0; st < NS; ++st)
                if (st < nact) pairs<RB>(op.p, a[st], f);
            break;
        }
        case plan::K_X: {
            if (tc && (E.obase & op.ocond) == op.ocond) {
                OpX f{op.f};
#pragma unroll
                for (int st = 0; st < NS; ++st)
                    if (st < nact) pairs<RB>(op.p, a[st], f);
            }
            break;
        }
        case plan::K_Y: {
            if (tc && (E.obase & op.ocond) == op.ocond) {
                OpY f{op.f};
#pragma unroll
                for (int st = 0; st < NS; ++st)
                    if (st < nact) pairs<RB>(op.p, a[st], f);
            }
            break;
        }
        case plan::K_RX: {
            OpRX f{op.a, op.b};
#pragma unroll
            for (int st = 0; st < NS; ++st)
                if (st < nact) pairs<RB>(op.p, a[st], f);
            break;
        }
        case plan::K_RY: {
            OpRY f{op.a, op.b};
#pragma unroll
            for (int st = 0; st < NS; ++st)
                if (st < nact) pairs<RB>(op.p, a[st], f);
            break;
        }
        case plan::K_U: {
            if (tc && (E.obase & op.ocond) == op.ocond) {
                const double* m = E.mats + 8 * op.g;
                OpU f{make_double2(m[0], m[1]), make_double2(m[2], m[3]), make_double2(m[4], m[5]),
                      make_double2(m[6], m[7]), op.f};
#pragma unroll
                for (int st = 0; st < NS; ++st)
                    if (st < nact) pairs<RB>(op.p, a[st], f);
            }
            break;
        }
        case plan::K_ACC_THR:
            if (tc) acc_thr += E.gval[op.g].x;
            break;
        case plan::K_ACC_REG: {
            if (tc) {
                double v = E.gval[op.g].x;
#pragma unroll
                for (int r = 0; r < RB; ++r)
                    if (r == op.p) acc[r] += v;
            }
            break;
        }
        case plan::K_PHD: {
            if (tc) {
                double2 e = E.gval[op.g];
#pragma unroll
                for (int st = 0; st < NS; ++st)
                    if (st < nact) phase_masked<RB>(op.f, a[st], e);
            }
            break;
        }
        case plan::K_FLUSH_REG:
            flush_reg<RB, NS>(op.p, acc, a, nact);
            break;
        case plan::K_FLUSH_ALL: {
#pragma unroll
            for (int r = 0; r < RB; ++r)
                if ((op.f >> r) & 1) flush_reg<RB, NS>(r, acc, a, nact);
            double2 e = make_double2(op.a, op.b);
            if (acc_thr != 0.0) {
                double s, c;
                sincos(acc_thr, &s, &c);
                e = cmul(e, make_double2(c, s));
                acc_thr = 0.0;
            }
            if (e.x != 1.0 || e.y != 0.0) {
#pragma unroll
                for (int st = 0; st < NS; ++st)
                    if (st < nact)
#pragma unroll
                        for (int j = 0; j < R; ++j) a[st][j] = cmul(a[st][j], e);
            }
            break;
        }
        case plan::K_TRANSPOSE: {
            const plan::LayoutRec* nrec = E.layouts + op.g;
            const uint16_t* Lm = nrec->L;
            uint32_t sreg_w[RB], sreg_r[RB];
            uint32_t sbw = slot_base<RB>(L, Lm, E.k, tid, sreg_w);
            LayoutState<RB> N;
            load_layout<RB>(N, nrec, E.tile_phys, E.k, E.obase, tid);
            uint32_t sbr = slot_base<RB>(N, Lm, E.k, tid, sreg_r);
#pragma unroll
            for (int st = 0; st < NS; ++st) {
                if (st < nact) {
                    __syncthreads();
                    if (active)
#pragma unroll
                        for (int j = 0; j < R; ++j) E.xbuf[sidx<RB>(sbw, sreg_w, j)] = a[st][j];
                    __syncthreads();
                    if (active)
#pragma unroll
                        for (int j = 0; j < R; ++j) a[st][j] = E.xbuf[sidx<RB>(sbr, sreg_r, j)];
                }
            }
            L = N;
            break;
        }
        case plan::K_GRAD_X:
        case plan::K_GRAD_Y:
        case plan::K_GRAD_Z:
        case plan::K_GRAD_P: {
            if constexpr (NS == 2) {
                double part = 0.0;
                if (op.kind == plan::K_GRAD_X || op.kind == plan::K_GRAD_Y) {
                    const bool isx = op.kind == plan::K_GRAD_X;
                    auto f = [&](const double2& s0, const double2& s1, const double2& l0, const double2& l1) {
                        part += isx ? (im_ls(l0, s1) + im_ls(l1, s0)) : (re_ls(l1, s0) - re_ls(l0, s1));
                    };
                    pairs2<RB>(op.p, a[0], a[NS - 1], f);
                } else if (op.kind == plan::K_GRAD_Z) {
                    double sg = ((tid & op.tcond) != 0) != ((E.obase & op.ocond) != 0) ? -1.0 : 1.0;
#pragma unroll
                    for (int j = 0; j < R; ++j) {
                        double v = im_ls(a[1][j], a[0][j]);
                        part += (op.p < RB && ((j >> op.p) & 1)) ? -v : v;
                    }
                    part *= sg;
                } else {
                    if (tc && (E.obase & op.ocond) == op.ocond) {
#pragma unroll
                        for (int j = 0; j < R; ++j)
                            if ((j & op.f) == op.f) part += im_ls(a[1][j], a[0][j]);
                    }
                }
                part = warp_sum(part * op.a);
                if (lane == 0) E.wpart[op.g * E.nwarps + warp] += part;
            }
            break;
        }
        default:
            break;
        }
    }
}

}  // namespace dev
}  // namespace tile
}  // namespace qse
