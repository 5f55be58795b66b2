// batch.cu -- forward expectation and adjoint gradient of many independent
// parameterised circuits of uneven width and depth in ONE persistent kernel,
// replayed as a CUDA graph.  No reference counterpart: the reference evaluates
// one Circuit at a time (Circuit.cpp:64-120).
//
// Planning (host, once per configuration).  Every circuit is planned twice by
// the fusion planner, with tile qubits k = min(log2(threads) + reg_bits, width):
// its gates (forward, from |0..0>) and its inverse gates in reverse order with
// gradient slots (the adjoint sweep, starting from the forward's final qubit
// map).  Angles enter the pass programs only through the records the planner
// lists in op_angles / term_angles, so a run rebinds parameters by patching
// those records on the device (k_bind) instead of planning again.  RZ's global
// phase is dropped: <O> and the gradients do not see it.
//
// Work queue.  A circuit whose passes have at most chain_tiles tiles is ONE
// item: a single CTA runs all its passes, forward and reverse, tile after tile
// (the state stays in L2).  Wider circuits give one item per (pass, tile),
// queued level-major (every circuit's pass 0, then every circuit's pass 1, ...),
// so a tile's dependencies (all tiles of the circuit's previous pass) sit
// earlier in the queue.  CTAs claim items in queue order with one atomic, and
// wait (bounded) on the previous pass's completion counter.  Because claims go
// in order, the lowest unfinished claimed item always has its inputs complete:
// the queue cannot deadlock, whatever the number of resident CTAs.
//
// Per tile: the first forward pass starts from |0..0> without reading memory;
// the first reverse pass loads |psi> only, forms |lambda> = O|psi> in registers
// and the tile's share of <psi|O|psi>; the last reverse pass stores nothing.
// Reductions are deterministic: per-tile partials, summed in a fixed order by
// k_fin_slots / k_fin_out.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "planner.h"
#include "qse_internal.h"
#include "tile_dev.cuh"

namespace qse {
namespace batch {

enum : uint32_t { F_ZERO = 1, F_LAMBDA = 2, F_REV = 4, F_NOSTORE = 8 };

struct BPass {
    uint64_t outer_mask;
    uint32_t op0, nops;
    uint32_t lay0, layout0;
    uint32_t term0, grp0;
    uint32_t ngroups, mat0;      // mat0: first 2x2 matrix (8 doubles each)
    uint32_t part0, nslots;      // gradient partials part[part0 + tile * nslots + s]
    uint32_t k, ntiles;
    uint32_t flags, circ;
    int32_t wait;                // pass whose counter must reach its ntiles first, -1 none
    uint32_t pad;
    uint8_t tile_phys[16];
};

struct BCirc {
    uint64_t psi, lam;           // element offsets in the state pool
    uint32_t obs0, nobs;         // observable terms (physical masks after the forward pass)
    double obs_c;
    uint32_t vpart0, nvpart;     // value partials (one per tile of the first reverse pass)
    double value0;               // <O> when the circuit has no gates (|0..0>)
};

struct BItem {
    uint32_t pass, npass;        // consecutive passes [pass, pass + npass)
    uint32_t tile, ntile;        // tiles [tile, tile + ntile) of each
};

struct BPatch {                  // angle = theta0 + coeff * params[param]
    uint32_t dst, kind;          // kind 0: ops[dst].(a, b) = (cos, sin)(angle / 2); 1: terms[dst].theta = angle
    int32_t param, pad;
    double theta0, coeff;
};

struct FinPass {                 // occ[slot_occ[slot0 + s]] = sum over tiles of part[part0 + t * nslots + s]
    uint32_t part0, nslots, ntiles, slot0;
};

struct BCtl {
    uint32_t next;               // next queue entry to claim
    uint32_t error;              // 1: a bounded wait gave up
    uint32_t err_pass;
    uint32_t pad;
};

struct BatchArgs {
    const BItem* items;
    const BPass* passes;
    const plan::KOp* ops;
    const plan::LayoutRec* layouts;
    const plan::TermRec* terms;
    const plan::GroupRec* groups;
    const double* mats;
    const BCirc* circs;
    const uint64_t* obs_z;
    const double* obs_w;
    double2* pool;
    double* vpart;
    double* part;
    uint32_t* done;
    BCtl* ctl;
    uint32_t nitems;
    uint32_t kmax;
    uint32_t max_groups;
    uint32_t max_slots;
    uint32_t spin_limit;
    uint32_t pad;
};

constexpr uint32_t kMaxThreads = 512;
// polls (with back-off up to 2 us each) before a work item's dependency wait
// gives up: about a second, far beyond any pass of a circuit that fits
constexpr uint32_t kDefaultWaitPolls = 1u << 21;

// exchange buffer | group values | per-warp gradient partials | warp sums
size_t smem_bytes(uint32_t kmax, uint32_t max_groups, uint32_t max_slots, uint32_t threads)
{
    const size_t nwarps = threads / 32;
    return (size_t(1) << kmax) * 16 + size_t(max_groups) * 16 + size_t(max_slots) * nwarps * 8 + nwarps * 8;
}

// ------------------------------------------------------------------ device
using namespace tile::dev;

__device__ __forceinline__ uint32_t claim(BCtl* ctl)
{
    if (*reinterpret_cast<volatile uint32_t*>(&ctl->error)) return ~0u;
    return atomicAdd(&ctl->next, 1u);
}

// Spins until *ctr >= target; gives up after `limit` polls (or when another
// CTA has given up), sets the error flag and returns false.
__device__ bool wait_count(const uint32_t* ctr, uint32_t target, BCtl* ctl, uint32_t pass, uint32_t limit)
{
    uint32_t ns = 32;
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(ctr) : "memory");
        if (v >= target) return true;
        if (*reinterpret_cast<volatile uint32_t*>(&ctl->error)) return false;
        __nanosleep(ns);
        if (ns < 2048) ns <<= 1;
    }
    if (atomicCAS(&ctl->error, 0u, 1u) == 0u) ctl->err_pass = pass;
    return false;
}

__device__ __forceinline__ double obs_value(uint64_t x, const uint64_t* z, const double* w, uint32_t nt, double c)
{
    double v = c;
    for (uint32_t t = 0; t < nt; ++t) v += (__popcll(x & __ldg(z + t)) & 1) ? -__ldg(w + t) : __ldg(w + t);
    return v;
}

// CTA-wide sum in a fixed order (warp trees, then warps in index order); thread 0 gets it.
__device__ __forceinline__ double block_sum(double v, double* red, uint32_t nwarps)
{
    v = warp_sum(v);
    const uint32_t tid = threadIdx.x;
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (tid == 0)
        for (uint32_t w = 0; w < nwarps; ++w) t += red[w];
    return t;
}

template <int RB>
__device__ __forceinline__ void run_tile(const BatchArgs& A, uint32_t pid, uint32_t tile, double2* xbuf, double2* gval,
                                         double* wpart, double* red, uint8_t* s_tile, uint32_t nwarps)
{
    constexpr int R = 1 << RB;
    const uint32_t tid = threadIdx.x;
    const BPass& P = A.passes[pid];
    const uint32_t flags = P.flags, k = P.k, nslots = P.nslots;
    const BCirc& C = A.circs[P.circ];
    const uint64_t obase = tile_base(tile, P.outer_mask);
    const bool rev = flags & F_REV;

    __syncthreads();  // the previous tile's users of the shared tables are done
    if (tid < 16) s_tile[tid] = P.tile_phys[tid];
    group_values(A.groups + P.grp0, P.ngroups, A.terms + P.term0, obase, gval);
    if (rev)
        for (uint32_t i = tid; i < nslots * nwarps; i += blockDim.x) wpart[i] = 0.0;
    __syncthreads();

    const bool active = tid < (1u << (k - RB));
    LayoutState<RB> L;
    load_layout<RB>(L, A.layouts + P.lay0 + P.layout0, s_tile, k, obase, tid);
    double2* psi = A.pool + C.psi;
    double2* lam = A.pool + C.lam;

    double2 a[2][R];
    double vsum = 0.0;
#pragma unroll
    for (int j = 0; j < R; ++j) {
        a[0][j] = make_double2(0.0, 0.0);
        a[1][j] = make_double2(0.0, 0.0);
        if (!active) continue;
        const uint64_t idx = gidx<RB>(L, j);
        if (flags & F_ZERO) a[0][j] = make_double2(idx == 0 ? 1.0 : 0.0, 0.0);
        else a[0][j] = __ldcg(psi + idx);
        if (flags & F_LAMBDA) {
            const double o = obs_value(idx, A.obs_z + C.obs0, A.obs_w + C.obs0, C.nobs, C.obs_c);
            a[1][j] = make_double2(o * a[0][j].x, o * a[0][j].y);
            vsum += o * (a[0][j].x * a[0][j].x + a[0][j].y * a[0][j].y);
        } else if (rev) {
            a[1][j] = __ldcg(lam + idx);
        }
    }

    const OpsEnv E{A.ops + P.op0, P.nops, A.layouts + P.lay0, A.mats + 8 * size_t(P.mat0), s_tile, k, obase,
                   xbuf, gval, wpart, nwarps};
    run_ops<RB, 2>(E, L, a, rev ? 2 : 1, active);

    if (!(flags & F_NOSTORE) && active) {
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const uint64_t idx = gidx<RB>(L, j);
            __stcg(psi + idx, a[0][j]);
            if (rev) __stcg(lam + idx, a[1][j]);
        }
    }
    if (flags & F_LAMBDA) {
        const double t = block_sum(vsum, red, nwarps);
        if (tid == 0) A.vpart[C.vpart0 + tile] = t;
    }
    if (rev && nslots) {
        __syncthreads();
        double* out = A.part + P.part0 + uint64_t(tile) * nslots;
        for (uint32_t s = tid; s < nslots; s += blockDim.x) {
            double v = 0.0;
            for (uint32_t w = 0; w < nwarps; ++w) v += wpart[s * nwarps + w];
            out[s] = v;
        }
    }
}

// Register budget: WIDE = 0 caps the kernel at 128 registers per thread (two
// CTAs of 256 threads per SM, a few spills); WIDE = 1 lets it use up to 255
// (CTAs of at most 256 threads, one per SM).  The autotuner picks by measurement.
template <int RB, int WIDE>
__global__ void __launch_bounds__(WIDE ? 256 : kMaxThreads, 1) k_batch(const __grid_constant__ BatchArgs A)
{
    extern __shared__ double2 smem[];
    const uint32_t tid = threadIdx.x;
    const uint32_t nwarps = blockDim.x >> 5;
    double2* xbuf = smem;
    double2* gval = smem + (size_t(1) << A.kmax);
    double* wpart = reinterpret_cast<double*>(gval + A.max_groups);
    double* red = wpart + size_t(A.max_slots) * nwarps;
    __shared__ uint8_t s_tile[16];
    __shared__ uint32_t s_cur, s_next;
    __shared__ int s_ok;

    if (tid == 0) s_cur = claim(A.ctl);
    for (;;) {
        __syncthreads();
        const uint32_t it = s_cur;
        if (it >= A.nitems) break;
        const BItem item = A.items[it];
        if (tid == 0) {
            const int32_t w = A.passes[item.pass].wait;
            bool ok = true;
            if (w >= 0) ok = wait_count(A.done + w, A.passes[w].ntiles, A.ctl, item.pass, A.spin_limit);
            s_ok = ok ? 1 : 0;
            s_next = ok ? claim(A.ctl) : ~0u;  // claim ahead: the queue order keeps this deadlock-free
        }
        __syncthreads();
        if (!s_ok) break;
        for (uint32_t p = 0; p < item.npass; ++p)
            for (uint32_t t = 0; t < item.ntile; ++t)
                run_tile<RB>(A, item.pass + p, item.tile + t, xbuf, gval, wpart, red, s_tile, nwarps);
        // publish: every thread's stores are visible GPU-wide before the counter moves
        __threadfence();
        __syncthreads();
        if (tid == 0) {
            if (item.npass == 1) {
                uint32_t* ctr = A.done + item.pass;
                asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(ctr), "r"(item.ntile) : "memory");
            }
            s_cur = s_next;
        }
    }
}

// angle binding: the records the planner listed as angle-carrying
__global__ void k_bind(const BPatch* __restrict__ pt, uint32_t n, const double* __restrict__ params, plan::KOp* ops,
                       plan::TermRec* terms)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const BPatch p = pt[i];
        const double ang = p.theta0 + p.coeff * params[p.param];
        if (p.kind == 0) {
            double s, c;
            sincos(ang / 2.0, &s, &c);
            ops[p.dst].a = c;
            ops[p.dst].b = s;
        } else {
            terms[p.dst].theta = ang;
        }
    }
}

// occurrence sums: one CTA per reverse pass, thread per slot, tiles in order
__global__ void k_fin_slots(const FinPass* __restrict__ fp, const double* __restrict__ part,
                            const uint32_t* __restrict__ slot_occ, double* __restrict__ occ)
{
    const FinPass f = fp[blockIdx.x];
    for (uint32_t s = threadIdx.x; s < f.nslots; s += blockDim.x) {
        double v = 0.0;
        const double* p = part + f.part0 + s;
        for (uint32_t t = 0; t < f.ntiles; ++t) v += p[uint64_t(t) * f.nslots];
        occ[slot_occ[f.slot0 + s]] = v;
    }
}

// grads[p] = sum of factor * occurrence over the occurrences of parameter p (fixed order);
// values[c] = sum of the circuit's value partials in tile order
__global__ void k_fin_out(const uint32_t* __restrict__ csr, const uint32_t* __restrict__ csr_occ,
                          const double* __restrict__ csr_fac, const double* __restrict__ occ, uint32_t nparams,
                          const BCirc* __restrict__ circs, uint32_t ncirc, const double* __restrict__ vpart,
                          double* __restrict__ grads, double* __restrict__ values)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nparams) {
        double g = 0.0;
        for (uint32_t e = csr[i]; e < csr[i + 1]; ++e) g += csr_fac[e] * occ[csr_occ[e]];
        grads[i] = g;
    } else if (i < nparams + ncirc) {
        const BCirc& c = circs[i - nparams];
        double v = c.value0;
        if (c.nvpart) {
            v = 0.0;
            for (uint32_t t = 0; t < c.nvpart; ++t) v += vpart[c.vpart0 + t];
        }
        values[i - nparams] = v;
    }
}

// ------------------------------------------------------------------ host
struct Config {
    uint32_t threads = 256, rb = 3, max_gates = 0, chain_tiles = 1, ctas_per_sm = 0;
    uint32_t grad_slots = 0;   // gradient slots per pass, 0 = no cap
    uint32_t wide = 0;         // 1: up to 255 registers per thread (threads <= 256); 0: 128
};

const void* kernel_of(const Config& c)
{
    if (c.rb == 3) return c.wide ? reinterpret_cast<const void*>(k_batch<3, 1>) : reinterpret_cast<const void*>(k_batch<3, 0>);
    return c.wide ? reinterpret_cast<const void*>(k_batch<2, 1>) : reinterpret_cast<const void*>(k_batch<2, 0>);
}

struct CircuitHost {
    uint32_t w = 0;
    std::vector<qse_op> ops;
    size_t nparams = 0, param0 = 0, occ0 = 0;
    std::vector<uint64_t> z;
    std::vector<double> wt;
    double c = 0.0;
};

bool parameterised(int type)
{
    return type == QSE_GATE_RX || type == QSE_GATE_RY || type == QSE_GATE_RZ || type == QSE_GATE_PHASE ||
           type == QSE_GATE_CPHASE || type == QSE_GATE_MCPHASE;
}

bool phase_type(int type)
{
    return type == QSE_GATE_PHASE || type == QSE_GATE_CPHASE || type == QSE_GATE_MCPHASE;
}

plan::Gate gate_of(const qse_op& op, double theta)
{
    plan::Gate g;
    g.type = op.type;
    g.t = op.target;
    g.c = op.control;
    g.cmask = op.controls;
    g.theta = theta;
    for (int i = 0; i < 8; ++i) g.m[i] = op.m[i];
    return g;
}

plan::Gate inverse_of(const qse_op& op, int32_t grad)
{
    plan::Gate g = gate_of(op, -op.theta);
    if (op.type == QSE_GATE_2X2) {
        g.m[0] = op.m[0]; g.m[1] = -op.m[1];
        g.m[2] = op.m[4]; g.m[3] = -op.m[5];
        g.m[4] = op.m[2]; g.m[5] = -op.m[3];
        g.m[6] = op.m[6]; g.m[7] = -op.m[7];
    }
    g.grad = grad;
    return g;
}

uint32_t log2u(uint32_t x)
{
    uint32_t r = 0;
    while ((1u << (r + 1)) <= x) ++r;
    return r;
}

template <class T>
size_t push_bytes(std::vector<char>& blob, const T* p, size_t n)
{
    size_t off = (blob.size() + 255) & ~size_t(255);
    blob.resize(off + n * sizeof(T));
    if (n) std::memcpy(blob.data() + off, p, n * sizeof(T));
    return off;
}

}  // namespace batch
}  // namespace qse

using namespace qse::batch;

struct qse_batch {
    qse_ctx* ctx = nullptr;
    std::vector<CircuitHost> circs;
    size_t total_params = 0, total_occ = 0;
    Config cfg;
    bool use_graph = true;
    bool built = false;
    uint32_t wait_limit = 0;      // polls before a dependency wait gives up, 0 = kDefaultWaitPolls
    std::vector<double> last_params;

    qse::DevBuf prog, work, pool;
    qse::HostBuf host;
    // device pointers into prog / work
    BatchArgs args{};
    const BPatch* patches = nullptr;
    uint32_t npatches = 0;
    const FinPass* fins = nullptr;
    uint32_t nfins = 0;
    const uint32_t* slot_occ = nullptr;
    const uint32_t* csr = nullptr;
    const uint32_t* csr_occ = nullptr;
    const double* csr_fac = nullptr;
    qse::plan::KOp* d_ops = nullptr;
    qse::plan::TermRec* d_terms = nullptr;
    double* occ = nullptr;
    double* params = nullptr;
    double* values = nullptr;
    double* grads = nullptr;
    size_t zero_bytes = 0;        // ctl + done + occ, cleared every run
    unsigned grid = 0;
    size_t smem = 0;
    cudaGraphExec_t gexec = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool timed = false;
    qse_batch_stats stats{};

    ~qse_batch()
    {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
    }
};

namespace qse {
namespace batch {
namespace {

void drop_graph(qse_batch* b)
{
    if (b->gexec) {
        cudaGraphExecDestroy(b->gexec);
        b->gexec = nullptr;
    }
}

// Plans every circuit under b->cfg and uploads programs, queue and reduction maps.
void build(qse_batch* b)
{
    auto t0 = std::chrono::steady_clock::now();
    qse_ctx* ctx = b->ctx;
    const Config& cf = b->cfg;
    const uint32_t kcfg = log2u(cf.threads) + cf.rb;
    drop_graph(b);
    b->built = false;

    std::vector<plan::KOp> ops;
    std::vector<plan::LayoutRec> layouts;
    std::vector<plan::TermRec> terms;
    std::vector<plan::GroupRec> groups;
    std::vector<double> mats;
    std::vector<BPass> passes;
    std::vector<BCirc> bc(b->circs.size());
    std::vector<uint64_t> obs_z;
    std::vector<double> obs_w;
    std::vector<BPatch> patches;
    std::vector<FinPass> fins;
    std::vector<uint32_t> slot_occ;
    std::vector<uint32_t> first_pass(b->circs.size()), npass(b->circs.size()), ntiles(b->circs.size());
    uint64_t part_total = 0, vpart_total = 0, pool_total = 0;
    uint32_t max_groups = 1, max_slots = 1, kmax = 1;
    uint64_t hbm = 0, visits = 0, occurrences = 0;

    for (size_t ci = 0; ci < b->circs.size(); ++ci) {
        const CircuitHost& ch = b->circs[ci];
        const uint32_t w = ch.w;
        plan::Options opt;
        opt.rb = cf.rb;
        opt.k = std::min(kcfg, w);
        opt.max_gates = cf.max_gates;
        opt.max_terms = 512;
        opt.keep_gphase = false;
        opt.direct_phases = true;
        opt.max_slots = cf.grad_slots;
        uint32_t perm0[64];
        for (uint32_t q = 0; q < 64; ++q) perm0[q] = q;

        std::vector<plan::Gate> fw;
        fw.reserve(ch.ops.size());
        for (const qse_op& op : ch.ops) fw.push_back(gate_of(op, op.theta));
        plan::Plan pf = plan::build(fw, w, perm0, opt);

        std::vector<plan::Gate> rv;
        rv.reserve(ch.ops.size());
        for (size_t i = ch.ops.size(); i-- > 0;) {
            const qse_op& op = ch.ops[i];
            rv.push_back(inverse_of(op, (op.param >= 0 && parameterised(op.type)) ? int32_t(i) : -1));
        }
        plan::Options optr = opt;
        optr.grads = true;
        plan::Plan pr = plan::build(rv, w, pf.perm_final, optr);

        const uint32_t k = opt.k;
        const uint32_t nt = 1u << (w - k);
        kmax = std::max(kmax, k);
        ntiles[ci] = nt;
        first_pass[ci] = uint32_t(passes.size());
        npass[ci] = uint32_t(pf.passes.size() + pr.passes.size());

        // state buffers (|lambda> only when the reverse sweep spans several passes)
        BCirc& c = bc[ci];
        const uint64_t amps = uint64_t(1) << w;
        c.psi = pool_total;
        pool_total += (amps + 15) & ~uint64_t(15);
        c.lam = pool_total;
        if (pr.passes.size() > 1) pool_total += (amps + 15) & ~uint64_t(15);
        // observable on the physical qubits of the forward's final map
        c.obs0 = uint32_t(obs_z.size());
        c.nobs = uint32_t(ch.z.size());
        c.obs_c = ch.c;
        c.value0 = ch.c;
        for (size_t t = 0; t < ch.z.size(); ++t) {
            uint64_t pm = 0;
            for (uint64_t m = ch.z[t]; m; m &= m - 1) pm |= uint64_t(1) << pf.perm_final[__builtin_ctzll(m)];
            obs_z.push_back(pm);
            obs_w.push_back(ch.wt[t]);
            c.value0 += ch.wt[t];
        }
        c.vpart0 = uint32_t(vpart_total);
        c.nvpart = pr.passes.empty() ? 0u : nt;
        vpart_total += c.nvpart;

        const size_t nf = pf.passes.size(), nall = nf + pr.passes.size();
        const bool multi = nt > cf.chain_tiles;
        for (size_t j = 0; j < nall; ++j) {
            const bool isrev = j >= nf;
            const plan::PassProgram& P = isrev ? pr.passes[j - nf] : pf.passes[j];
            BPass bp{};
            bp.outer_mask = P.outer_mask;
            bp.op0 = uint32_t(ops.size());
            bp.nops = uint32_t(P.ops.size());
            bp.lay0 = uint32_t(layouts.size());
            bp.layout0 = P.layout0;
            bp.term0 = uint32_t(terms.size());
            bp.grp0 = uint32_t(groups.size());
            bp.ngroups = uint32_t(P.groups.size());
            bp.mat0 = uint32_t(mats.size() / 8);
            bp.k = P.k;
            bp.ntiles = nt;
            bp.circ = uint32_t(ci);
            bp.wait = (j > 0 && multi) ? int32_t(passes.size() - 1) : -1;
            std::memcpy(bp.tile_phys, P.tile_phys, 16);
            if (j == 0) bp.flags |= F_ZERO;
            if (isrev) {
                bp.flags |= F_REV;
                if (j == nf) bp.flags |= F_LAMBDA;
                if (j + 1 == nall) bp.flags |= F_NOSTORE;
            }
            bp.nslots = uint32_t(P.slot_src.size());
            if (bp.nslots) {
                bp.part0 = uint32_t(part_total);
                fins.push_back(FinPass{uint32_t(part_total), bp.nslots, nt, uint32_t(slot_occ.size())});
                for (int32_t s : P.slot_src) slot_occ.push_back(uint32_t(ch.occ0 + uint32_t(s)));
                part_total += uint64_t(nt) * bp.nslots;
                if (part_total > 0xffffffffull) fail(QSE_ERR_SIZE, "batch: too many gradient partials");
            }
            max_groups = std::max(max_groups, bp.ngroups);
            max_slots = std::max(max_slots, bp.nslots);
            // angle records -> patches
            for (const plan::AngleRef& r : P.op_angles) {
                const size_t src = isrev ? ch.ops.size() - 1 - r.src : r.src;
                const qse_op& op = ch.ops[src];
                if (op.param < 0) continue;
                const double sg = isrev ? -1.0 : 1.0;
                patches.push_back(BPatch{bp.op0 + r.index, 0u, int32_t(ch.param0 + op.param), 0, sg * op.theta,
                                         sg * op.coeff});
            }
            for (const plan::AngleRef& r : P.term_angles) {
                const size_t src = isrev ? ch.ops.size() - 1 - r.src : r.src;
                const qse_op& op = ch.ops[src];
                if (op.param < 0) continue;
                const double sg = isrev ? -1.0 : 1.0;
                patches.push_back(BPatch{bp.term0 + r.index, 1u, int32_t(ch.param0 + op.param), 0, sg * op.theta,
                                         sg * op.coeff});
            }
            ops.insert(ops.end(), P.ops.begin(), P.ops.end());
            layouts.insert(layouts.end(), P.layouts.begin(), P.layouts.end());
            terms.insert(terms.end(), P.terms.begin(), P.terms.end());
            groups.insert(groups.end(), P.groups.begin(), P.groups.end());
            mats.insert(mats.end(), P.mats.begin(), P.mats.end());
            passes.push_back(bp);
            visits += nt;
            if (multi) hbm += amps * (isrev ? 64u : 32u);
        }
        // a reverse-only circuit (no forward pass) starts its reverse sweep from |0..0>
        if (nf == 0 && nall > 0) passes[first_pass[ci]].flags |= F_ZERO;
        for (const qse_op& op : ch.ops) occurrences += (op.param >= 0 && parameterised(op.type)) ? 1 : 0;
    }

    // parameter -> occurrence map (CSR, occurrences in program order)
    std::vector<uint32_t> csr(b->total_params + 1, 0), csr_occ;
    std::vector<double> csr_fac;
    {
        std::vector<std::vector<std::pair<uint32_t, double>>> per(b->total_params);
        for (const CircuitHost& ch : b->circs)
            for (size_t i = 0; i < ch.ops.size(); ++i) {
                const qse_op& op = ch.ops[i];
                if (op.param < 0 || !parameterised(op.type)) continue;
                per[ch.param0 + op.param].emplace_back(uint32_t(ch.occ0 + i),
                                                       op.coeff * (phase_type(op.type) ? -2.0 : 1.0));
            }
        for (size_t p = 0; p < per.size(); ++p) {
            csr[p + 1] = csr[p] + uint32_t(per[p].size());
            for (auto& e : per[p]) {
                csr_occ.push_back(e.first);
                csr_fac.push_back(e.second);
            }
        }
    }

    // work queue: single-CTA circuits first (longest first), then level-major tiles
    std::vector<BItem> items;
    {
        std::vector<size_t> chains, multis;
        for (size_t ci = 0; ci < b->circs.size(); ++ci) {
            if (npass[ci] == 0) continue;
            (ntiles[ci] <= cf.chain_tiles ? chains : multis).push_back(ci);
        }
        std::stable_sort(chains.begin(), chains.end(), [&](size_t x, size_t y) {
            return uint64_t(npass[x]) * ntiles[x] * (uint64_t(1) << b->circs[x].w) >
                   uint64_t(npass[y]) * ntiles[y] * (uint64_t(1) << b->circs[y].w);
        });
        for (size_t ci : chains) items.push_back(BItem{first_pass[ci], npass[ci], 0, ntiles[ci]});
        uint32_t maxlev = 0;
        for (size_t ci : multis) maxlev = std::max(maxlev, npass[ci]);
        for (uint32_t lev = 0; lev < maxlev; ++lev)
            for (size_t ci : multis) {
                if (lev >= npass[ci]) continue;
                for (uint32_t t = 0; t < ntiles[ci]; ++t) items.push_back(BItem{first_pass[ci] + lev, 1, t, 1});
            }
        if (items.size() > 0xffffff00ull) fail(QSE_ERR_SIZE, "batch: work queue too long");
    }

    // shared memory and grid
    const size_t smem = smem_bytes(kmax, max_groups, max_slots, cf.threads);
    if (smem + 64 > ctx->smem_optin)
        fail(QSE_ERR_SIZE, "batch: a pass needs " + std::to_string(smem) +
                               " B of shared memory; lower max_gates or the tile size");
    const void* kfn = kernel_of(cf);
    {
        cudaFuncAttributes fa{};
        QSE_CUDA(cudaFuncGetAttributes(&fa, kfn));
        QSE_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(ctx->smem_optin - fa.sharedSizeBytes)));
    }
    int occ_blocks = 0;
    QSE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_blocks, kfn, int(cf.threads), smem));
    if (occ_blocks < 1) fail(QSE_ERR_SIZE, "batch: kernel configuration does not fit on an SM");
    uint32_t per_sm = uint32_t(occ_blocks);
    if (cf.ctas_per_sm) per_sm = std::min(per_sm, cf.ctas_per_sm);
    b->grid = unsigned(std::min<uint64_t>(uint64_t(ctx->num_sms) * per_sm, std::max<size_t>(items.size(), 1)));
    b->smem = smem;

    // one blob for everything read-only (plus the patched ops / terms)
    std::vector<char> blob;
    size_t o_ops = push_bytes(blob, ops.data(), ops.size());
    size_t o_lay = push_bytes(blob, layouts.data(), layouts.size());
    size_t o_terms = push_bytes(blob, terms.data(), terms.size());
    size_t o_groups = push_bytes(blob, groups.data(), groups.size());
    size_t o_mats = push_bytes(blob, mats.data(), mats.size());
    size_t o_passes = push_bytes(blob, passes.data(), passes.size());
    size_t o_items = push_bytes(blob, items.data(), items.size());
    size_t o_circs = push_bytes(blob, bc.data(), bc.size());
    size_t o_oz = push_bytes(blob, obs_z.data(), obs_z.size());
    size_t o_ow = push_bytes(blob, obs_w.data(), obs_w.size());
    size_t o_pt = push_bytes(blob, patches.data(), patches.size());
    size_t o_fin = push_bytes(blob, fins.data(), fins.size());
    size_t o_so = push_bytes(blob, slot_occ.data(), slot_occ.size());
    size_t o_csr = push_bytes(blob, csr.data(), csr.size());
    size_t o_cocc = push_bytes(blob, csr_occ.data(), csr_occ.size());
    size_t o_cfac = push_bytes(blob, csr_fac.data(), csr_fac.size());
    blob.resize(blob.size() + 256);
    b->prog.reserve(blob.size());
    char* pd = static_cast<char*>(b->prog.ptr);
    // every copy and clear goes on the library stream: the legacy-stream forms
    // do not order against a non-blocking stream
    QSE_CUDA(cudaMemcpyAsync(pd, blob.data(), blob.size(), cudaMemcpyHostToDevice, ctx->stream));

    // work: ctl | done | occ | vpart | part | params | values | grads
    const size_t npasses = passes.size();
    size_t w_ctl = 0;
    size_t w_done = 256;
    size_t w_occ = (w_done + npasses * 4 + 255) & ~size_t(255);
    size_t zero_end = w_occ + std::max<size_t>(b->total_occ, 1) * 8;
    size_t w_vp = (zero_end + 255) & ~size_t(255);
    size_t w_part = (w_vp + std::max<uint64_t>(vpart_total, 1) * 8 + 255) & ~size_t(255);
    size_t w_par = (w_part + std::max<uint64_t>(part_total, 1) * 8 + 255) & ~size_t(255);
    size_t w_val = (w_par + std::max<size_t>(b->total_params, 1) * 8 + 255) & ~size_t(255);
    size_t w_grad = (w_val + std::max<size_t>(b->circs.size(), 1) * 8 + 255) & ~size_t(255);
    size_t w_end = w_grad + std::max<size_t>(b->total_params, 1) * 8 + 256;
    b->work.reserve(w_end);
    char* wd = static_cast<char*>(b->work.ptr);
    QSE_CUDA(cudaMemsetAsync(wd, 0, w_end, ctx->stream));
    b->pool.reserve(std::max<uint64_t>(pool_total, 1) * 16);

    BatchArgs& A = b->args;
    A.items = reinterpret_cast<const BItem*>(pd + o_items);
    A.passes = reinterpret_cast<const BPass*>(pd + o_passes);
    A.ops = reinterpret_cast<const plan::KOp*>(pd + o_ops);
    A.layouts = reinterpret_cast<const plan::LayoutRec*>(pd + o_lay);
    A.terms = reinterpret_cast<const plan::TermRec*>(pd + o_terms);
    A.groups = reinterpret_cast<const plan::GroupRec*>(pd + o_groups);
    A.mats = reinterpret_cast<const double*>(pd + o_mats);
    A.circs = reinterpret_cast<const BCirc*>(pd + o_circs);
    A.obs_z = reinterpret_cast<const uint64_t*>(pd + o_oz);
    A.obs_w = reinterpret_cast<const double*>(pd + o_ow);
    A.pool = static_cast<double2*>(b->pool.ptr);
    A.vpart = reinterpret_cast<double*>(wd + w_vp);
    A.part = reinterpret_cast<double*>(wd + w_part);
    A.done = reinterpret_cast<uint32_t*>(wd + w_done);
    A.ctl = reinterpret_cast<BCtl*>(wd + w_ctl);
    A.nitems = uint32_t(items.size());
    A.kmax = kmax;
    A.max_groups = max_groups;
    A.max_slots = max_slots;
    A.spin_limit = b->wait_limit ? b->wait_limit : kDefaultWaitPolls;
    b->d_ops = reinterpret_cast<plan::KOp*>(pd + o_ops);
    b->d_terms = reinterpret_cast<plan::TermRec*>(pd + o_terms);
    b->patches = reinterpret_cast<const BPatch*>(pd + o_pt);
    b->npatches = uint32_t(patches.size());
    b->fins = reinterpret_cast<const FinPass*>(pd + o_fin);
    b->nfins = uint32_t(fins.size());
    b->slot_occ = reinterpret_cast<const uint32_t*>(pd + o_so);
    b->csr = reinterpret_cast<const uint32_t*>(pd + o_csr);
    b->csr_occ = reinterpret_cast<const uint32_t*>(pd + o_cocc);
    b->csr_fac = reinterpret_cast<const double*>(pd + o_cfac);
    b->occ = reinterpret_cast<double*>(wd + w_occ);
    b->params = reinterpret_cast<double*>(wd + w_par);
    b->values = reinterpret_cast<double*>(wd + w_val);
    b->grads = reinterpret_cast<double*>(wd + w_grad);
    b->zero_bytes = zero_end;

    b->stats = qse_batch_stats{};
    b->stats.passes = npasses;
    b->stats.items = items.size();
    b->stats.tile_visits = visits;
    b->stats.hbm_bytes = hbm;
    b->stats.occurrences = occurrences;
    b->stats.grid = b->grid;
    b->stats.smem_bytes = uint32_t(smem);
    b->stats.plan_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    b->timed = false;
    QSE_CUDA(cudaStreamSynchronize(ctx->stream));  // blob is pageable and goes out of scope
    b->built = true;
}

// The launches of one run on ctx->stream (captured into the graph, or issued directly).
void enqueue(qse_batch* b)
{
    qse_ctx* ctx = b->ctx;
    cudaStream_t s = ctx->stream;
    QSE_CUDA(cudaMemsetAsync(b->work.ptr, 0, b->zero_bytes, s));
    if (b->npatches) {
        unsigned g = unsigned(std::min<uint64_t>((b->npatches + 255) / 256, uint64_t(ctx->num_sms) * 8));
        k_bind<<<g, 256, 0, s>>>(b->patches, b->npatches, b->params, b->d_ops, b->d_terms);
        QSE_CUDA(cudaGetLastError());
    }
    if (b->args.nitems) {
        const Config& c = b->cfg;
        if (c.rb == 3 && c.wide) k_batch<3, 1><<<b->grid, c.threads, b->smem, s>>>(b->args);
        else if (c.rb == 3) k_batch<3, 0><<<b->grid, c.threads, b->smem, s>>>(b->args);
        else if (c.wide) k_batch<2, 1><<<b->grid, c.threads, b->smem, s>>>(b->args);
        else k_batch<2, 0><<<b->grid, c.threads, b->smem, s>>>(b->args);
        QSE_CUDA(cudaGetLastError());
    }
    if (b->nfins) {
        k_fin_slots<<<b->nfins, 128, 0, s>>>(b->fins, b->args.part, b->slot_occ, b->occ);
        QSE_CUDA(cudaGetLastError());
    }
    const uint32_t nout = uint32_t(b->total_params + b->circs.size());
    if (nout) {
        k_fin_out<<<(nout + 255) / 256, 256, 0, s>>>(b->csr, b->csr_occ, b->csr_fac, b->occ, uint32_t(b->total_params),
                                                     b->args.circs, uint32_t(b->circs.size()), b->args.vpart, b->grads,
                                                     b->values);
        QSE_CUDA(cudaGetLastError());
    }
}

void launch_run(qse_batch* b)
{
    qse_ctx* ctx = b->ctx;
    if (!b->built) build(b);
    if (!b->ev0) {
        QSE_CUDA(cudaEventCreate(&b->ev0));
        QSE_CUDA(cudaEventCreate(&b->ev1));
    }
    QSE_CUDA(cudaEventRecord(b->ev0, ctx->stream));
    if (b->use_graph) {
        if (!b->gexec) {
            cudaGraph_t g = nullptr;
            QSE_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
            try {
                enqueue(b);
            } catch (...) {
                cudaStreamEndCapture(ctx->stream, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            QSE_CUDA(cudaStreamEndCapture(ctx->stream, &g));
            cudaError_t e = cudaGraphInstantiate(&b->gexec, g, 0);
            cudaGraphDestroy(g);
            QSE_CUDA(e);
        }
        QSE_CUDA(cudaGraphLaunch(b->gexec, ctx->stream));
        count_launch(ctx, 4);
    } else {
        enqueue(b);
        count_launch(ctx, 4);
    }
    QSE_CUDA(cudaEventRecord(b->ev1, ctx->stream));
    b->timed = true;
}

// after a synchronised run: the device error word
void check_ctl(qse_batch* b)
{
    BCtl c{};
    QSE_CUDA(cudaMemcpyAsync(&c, b->args.ctl, sizeof(c), cudaMemcpyDeviceToHost, b->ctx->stream));
    QSE_CUDA(cudaStreamSynchronize(b->ctx->stream));
    if (c.error)
        fail(QSE_ERR_TIMEOUT, "batch: a work item waited too long for pass " + std::to_string(c.err_pass) +
                                  " (bounded wait gave up; results are invalid)");
}

std::string signature(const qse_batch* b)
{
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint64_t v) {
        for (int i = 0; i < 8; ++i) {
            h ^= (v >> (8 * i)) & 0xff;
            h *= 1099511628211ull;
        }
    };
    mix(b->circs.size());
    for (const CircuitHost& c : b->circs) {
        mix(c.w);
        mix(c.ops.size());
        for (const qse_op& op : c.ops) {
            mix(uint64_t(uint32_t(op.type)) | (uint64_t(op.target) << 32));
            mix(uint64_t(op.control) | (uint64_t(op.param >= 0) << 32));
            mix(op.controls);
        }
        mix(c.z.size());
    }
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, b->ctx->device);
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%016llx", (unsigned long long)h);
    std::string name(prop.name);
    for (char& ch : name)
        if (ch == '"' || ch == '\\') ch = '_';
    return name + "/" + buf;
}

std::string config_json(const Config& c)
{
    std::ostringstream os;
    os << "{\"threads\":" << c.threads << ",\"reg_bits\":" << c.rb << ",\"max_gates\":" << c.max_gates
       << ",\"chain_tiles\":" << c.chain_tiles << ",\"ctas_per_sm\":" << c.ctas_per_sm
       << ",\"grad_slots\":" << c.grad_slots << ",\"wide_regs\":" << c.wide << "}";
    return os.str();
}

// minimal reader for the cache file written by save_cache: one "key": {config} per line
std::map<std::string, std::string> load_cache(const char* path)
{
    std::map<std::string, std::string> m;
    if (!path) return m;
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
        size_t a = line.find('"');
        if (a == std::string::npos) continue;
        size_t bq = line.find('"', a + 1);
        size_t l = line.find('{', bq);
        size_t r = line.find('}', l);
        if (bq == std::string::npos || l == std::string::npos || r == std::string::npos) continue;
        m[line.substr(a + 1, bq - a - 1)] = line.substr(l, r - l + 1);
    }
    return m;
}

void save_cache(const char* path, const std::map<std::string, std::string>& m)
{
    if (!path) return;
    std::ofstream f(path, std::ios::trunc);
    f << "{\n";
    size_t i = 0;
    for (auto& kv : m) f << "  \"" << kv.first << "\": " << kv.second << (++i < m.size() ? ",\n" : "\n");
    f << "}\n";
}

bool parse_config(const std::string& s, Config& c)
{
    auto get = [&](const char* key, uint32_t& out) {
        std::string k = std::string("\"") + key + "\":";
        size_t p = s.find(k);
        if (p == std::string::npos) return false;
        out = uint32_t(std::strtoul(s.c_str() + p + k.size(), nullptr, 10));
        return true;
    };
    Config t;
    bool ok = get("threads", t.threads) && get("reg_bits", t.rb) && get("max_gates", t.max_gates) &&
              get("chain_tiles", t.chain_tiles) && get("ctas_per_sm", t.ctas_per_sm) &&
              get("grad_slots", t.grad_slots) && get("wide_regs", t.wide);
    if (ok) c = t;
    return ok;
}

void validate(const qse_batch* b, const Config& c)
{
    if (c.threads < 32 || c.threads > kMaxThreads || (c.threads & (c.threads - 1)))
        fail(QSE_ERR_INVALID, "batch: threads must be a power of two in 32..512");
    if (c.wide > 1 || (c.wide && c.threads > 256))
        fail(QSE_ERR_INVALID, "batch: wide_regs needs threads <= 256");
    if (c.grad_slots > 4096) fail(QSE_ERR_INVALID, "batch: grad_slots too large");
    if (c.rb != 2 && c.rb != 3) fail(QSE_ERR_INVALID, "batch: reg_bits must be 2 or 3");
    if (c.chain_tiles < 1) fail(QSE_ERR_INVALID, "batch: chain_tiles must be >= 1");
    for (const CircuitHost& ch : b->circs)
        if (ch.w < c.rb + 1) fail(QSE_ERR_SIZE, "batch: circuit narrower than reg_bits + 1 qubits");
}

double time_config(qse_batch* b, int reps)
{
    launch_run(b);  // warm-up (and graph instantiation)
    QSE_CUDA(cudaStreamSynchronize(b->ctx->stream));
    check_ctl(b);
    double best = 1e30;
    for (int r = 0; r < reps; ++r) {
        launch_run(b);
        QSE_CUDA(cudaEventSynchronize(b->ev1));
        check_ctl(b);
        float ms = 0.f;
        QSE_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
        best = std::min(best, double(ms));
    }
    return best;
}

void upload_params(qse_batch* b, const double* params_host)
{
    const size_t n = b->total_params;
    b->last_params.assign(params_host, params_host + n);
    if (n) QSE_CUDA(cudaMemcpyAsync(b->params, b->last_params.data(), n * 8, cudaMemcpyHostToDevice, b->ctx->stream));
}

}  // namespace
}  // namespace batch
}  // namespace qse

// ------------------------------------------------------------------ C ABI

#define QSE_BATCH_GUARD_BEGIN try {
#define QSE_BATCH_GUARD_END                            \
    }                                                  \
    catch (const qse::Error& e)                        \
    {                                                  \
        qse::set_last_error(e.what());                 \
        return e.status;                               \
    }                                                  \
    catch (const std::bad_alloc&)                      \
    {                                                  \
        qse::set_last_error("host allocation failed"); \
        return QSE_ERR_OOM;                            \
    }                                                  \
    catch (const std::exception& e)                    \
    {                                                  \
        qse::set_last_error(e.what());                 \
        return QSE_ERR_INVALID;                        \
    }                                                  \
    return QSE_OK;

extern "C" {

int qse_batch_create(qse_ctx* ctx, const qse_batch_circuit* circuits, size_t ncircuits, qse_batch** out)
{
    QSE_BATCH_GUARD_BEGIN
    if (!ctx || !out || (ncircuits && !circuits)) qse::fail(QSE_ERR_INVALID, "null argument");
    *out = nullptr;
    QSE_CUDA(cudaSetDevice(ctx->device));
    auto b = std::make_unique<qse_batch>();
    b->ctx = ctx;
    size_t p0 = 0, o0 = 0;
    for (size_t i = 0; i < ncircuits; ++i) {
        const qse_batch_circuit& c = circuits[i];
        if (c.nqubits < 3 || c.nqubits > 30) qse::fail(QSE_ERR_SIZE, "batch: circuit width must be 3..30 qubits");
        if (c.nops && !c.ops) qse::fail(QSE_ERR_INVALID, "batch: null ops");
        if (c.obs.nterms && (!c.obs.zmask || !c.obs.weight)) qse::fail(QSE_ERR_INVALID, "batch: null observable");
        CircuitHost ch;
        ch.w = c.nqubits;
        ch.ops.assign(c.ops, c.ops + c.nops);
        ch.nparams = c.nparams;
        ch.param0 = p0;
        ch.occ0 = o0;
        for (const qse_op& op : ch.ops)
            if (op.param >= 0 && size_t(op.param) >= c.nparams)
                qse::fail(QSE_ERR_INVALID, "batch: op parameter index out of range");
        for (size_t t = 0; t < c.obs.nterms; ++t) {
            if (c.nqubits < 64 && (c.obs.zmask[t] >> c.nqubits) != 0)
                qse::fail(QSE_ERR_QUBIT, "batch: observable acts on a qubit out of range");
            ch.z.push_back(c.obs.zmask[t]);
            ch.wt.push_back(c.obs.weight[t]);
        }
        ch.c = c.obs.constant;
        p0 += c.nparams;
        o0 += c.nops;
        b->circs.push_back(std::move(ch));
    }
    b->total_params = p0;
    b->total_occ = o0;
    if (o0 > 0xffffffffull || p0 > 0xffffffffull) qse::fail(QSE_ERR_SIZE, "batch: too many ops");
    b->cfg.threads = 256;
    b->cfg.rb = 3;
    validate(b.get(), b->cfg);
    b->last_params.assign(p0, 0.0);
    *out = b.release();
    QSE_BATCH_GUARD_END
}

int qse_batch_destroy(qse_batch* b)
{
    if (!b) return QSE_OK;
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    delete b;
    return QSE_OK;
}

int qse_batch_run(qse_batch* b, const double* params, double* values, double* grads)
{
    QSE_BATCH_GUARD_BEGIN
    if (!b) qse::fail(QSE_ERR_INVALID, "null batch");
    if (b->total_params && (!params || !grads)) qse::fail(QSE_ERR_INVALID, "null params / grads");
    if (!values && !b->circs.empty()) qse::fail(QSE_ERR_INVALID, "null values");
    QSE_CUDA(cudaSetDevice(b->ctx->device));
    if (!b->built) build(b);
    upload_params(b, params);
    launch_run(b);
    const size_t np = b->total_params, nc = b->circs.size();
    check_ctl(b);
    if (nc) QSE_CUDA(cudaMemcpyAsync(values, b->values, nc * 8, cudaMemcpyDeviceToHost, b->ctx->stream));
    if (np) QSE_CUDA(cudaMemcpyAsync(grads, b->grads, np * 8, cudaMemcpyDeviceToHost, b->ctx->stream));
    QSE_CUDA(cudaStreamSynchronize(b->ctx->stream));
    QSE_BATCH_GUARD_END
}

int qse_batch_run_device(qse_batch* b, const double* d_params, double* d_values, double* d_grads)
{
    QSE_BATCH_GUARD_BEGIN
    if (!b) qse::fail(QSE_ERR_INVALID, "null batch");
    if (b->total_params && (!d_params || !d_grads)) qse::fail(QSE_ERR_INVALID, "null params / grads");
    if (!d_values && !b->circs.empty()) qse::fail(QSE_ERR_INVALID, "null values");
    QSE_CUDA(cudaSetDevice(b->ctx->device));
    if (!b->built) build(b);
    cudaStream_t s = b->ctx->stream;
    const size_t np = b->total_params, nc = b->circs.size();
    if (np) QSE_CUDA(cudaMemcpyAsync(b->params, d_params, np * 8, cudaMemcpyDeviceToDevice, s));
    launch_run(b);
    if (nc) QSE_CUDA(cudaMemcpyAsync(d_values, b->values, nc * 8, cudaMemcpyDeviceToDevice, s));
    if (np) QSE_CUDA(cudaMemcpyAsync(d_grads, b->grads, np * 8, cudaMemcpyDeviceToDevice, s));
    QSE_BATCH_GUARD_END
}

int qse_batch_total_params(const qse_batch* b, size_t* n)
{
    QSE_BATCH_GUARD_BEGIN
    if (!b || !n) qse::fail(QSE_ERR_INVALID, "null argument");
    *n = b->total_params;
    QSE_BATCH_GUARD_END
}

int qse_batch_use_graph(qse_batch* b, int enabled)
{
    QSE_BATCH_GUARD_BEGIN
    if (!b) qse::fail(QSE_ERR_INVALID, "null batch");
    b->use_graph = enabled != 0;
    drop_graph(b);
    QSE_BATCH_GUARD_END
}

int qse_batch_set_wait_limit(qse_batch* b, uint32_t polls)
{
    QSE_BATCH_GUARD_BEGIN
    if (!b) qse::fail(QSE_ERR_INVALID, "null batch");
    QSE_CUDA(cudaSetDevice(b->ctx->device));
    QSE_CUDA(cudaStreamSynchronize(b->ctx->stream));
    b->wait_limit = polls;
    b->args.spin_limit = polls ? polls : kDefaultWaitPolls;
    drop_graph(b);   // the graph holds the kernel's arguments by value
    QSE_BATCH_GUARD_END
}

int qse_batch_set_config(qse_batch* b, const qse_batch_config* cfg)
{
    QSE_BATCH_GUARD_BEGIN
    if (!b || !cfg) qse::fail(QSE_ERR_INVALID, "null argument");
    Config c;
    c.threads = cfg->threads;
    c.rb = cfg->reg_bits;
    c.max_gates = cfg->max_gates;
    c.chain_tiles = cfg->chain_tiles;
    c.ctas_per_sm = cfg->ctas_per_sm;
    c.grad_slots = cfg->grad_slots;
    c.wide = cfg->wide_regs;
    validate(b, c);
    QSE_CUDA(cudaSetDevice(b->ctx->device));
    QSE_CUDA(cudaStreamSynchronize(b->ctx->stream));
    b->cfg = c;
    b->built = false;
    drop_graph(b);
    QSE_BATCH_GUARD_END
}

int qse_batch_get_config(const qse_batch* b, qse_batch_config* cfg)
{
    QSE_BATCH_GUARD_BEGIN
    if (!b || !cfg) qse::fail(QSE_ERR_INVALID, "null argument");
    cfg->threads = b->cfg.threads;
    cfg->reg_bits = b->cfg.rb;
    cfg->max_gates = b->cfg.max_gates;
    cfg->chain_tiles = b->cfg.chain_tiles;
    cfg->ctas_per_sm = b->cfg.ctas_per_sm;
    cfg->grad_slots = b->cfg.grad_slots;
    cfg->wide_regs = b->cfg.wide;
    QSE_BATCH_GUARD_END
}

int qse_batch_get_stats(qse_batch* b, qse_batch_stats* out)
{
    QSE_BATCH_GUARD_BEGIN
    if (!b || !out) qse::fail(QSE_ERR_INVALID, "null argument");
    QSE_CUDA(cudaSetDevice(b->ctx->device));
    if (!b->built) build(b);
    b->stats.last_ms = 0.0;
    if (b->timed) {
        QSE_CUDA(cudaEventSynchronize(b->ev1));
        float ms = 0.f;
        QSE_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
        b->stats.last_ms = ms;
    }
    *out = b->stats;
    QSE_BATCH_GUARD_END
}

int qse_batch_autotune(qse_batch* b, const char* cache_path)
{
    QSE_BATCH_GUARD_BEGIN
    if (!b) qse::fail(QSE_ERR_INVALID, "null batch");
    QSE_CUDA(cudaSetDevice(b->ctx->device));
    const std::string key = signature(b);
    auto cache = load_cache(cache_path);
    auto hit = cache.find(key);
    Config c;
    if (hit != cache.end() && parse_config(hit->second, c)) {
        validate(b, c);
        b->cfg = c;
        b->built = false;
        drop_graph(b);
        build(b);
        return QSE_OK;
    }
    uint32_t wmin = 64;
    for (const CircuitHost& ch : b->circs) wmin = std::min(wmin, ch.w);
    // block shape x tile qubits x register budget, then gates fused per pass, then
    // the single-CTA threshold
    std::vector<Config> shapes;
    const uint32_t shape_list[][3] = {{128, 3, 0}, {256, 3, 0}, {512, 3, 0}, {256, 2, 0}, {512, 2, 0},
                                      {256, 3, 1}};
    for (auto& sh : shape_list) {
        Config t;
        t.threads = sh[0];
        t.rb = sh[1];
        t.wide = sh[2];
        if (wmin < t.rb + 1) continue;
        shapes.push_back(t);
    }
    Config best_c = b->cfg;
    double best = 1e30;
    auto trial = [&](const Config& t) {
        b->cfg = t;
        b->built = false;
        try {
            build(b);
            upload_params(b, b->last_params.data());
            double ms = time_config(b, 2);
            if (ms < best) {
                best = ms;
                best_c = t;
            }
        } catch (const qse::Error& e) {
            if (e.status != QSE_ERR_SIZE) throw;  // a configuration that does not fit is skipped
        }
    };
    for (const Config& t : shapes) trial(t);
    {
        const Config base = best_c;
        for (uint32_t mg : {24u, 48u}) {
            Config t = base;
            t.max_gates = mg;
            trial(t);
        }
    }
    {
        const Config base = best_c;
        for (uint32_t ct : {4u, 16u}) {
            Config t = base;
            t.chain_tiles = ct;
            trial(t);
        }
    }
    if (best >= 1e30) qse::fail(QSE_ERR_SIZE, "batch autotune: no configuration fits");
    b->cfg = best_c;
    b->built = false;
    drop_graph(b);
    build(b);
    if (cache_path) {
        cache[key] = config_json(best_c);
        save_cache(cache_path, cache);
    }
    QSE_BATCH_GUARD_END
}

}  // extern "C"
