// engine.cu -- Circuit::execute (Circuit.cpp:64-120) on the device: gate
// list -> planner -> one tile-kernel launch per pass; noise decisions and the
// end-of-execute Pauli frame; expectation values and the adjoint sweep.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>

#include "jit.h"
#include "planner.h"
#include "qse_internal.h"
#include "tile.cuh"

namespace qse {

double bound_angle(const qse_op& op, const double* params, size_t nparams)
{
    if (op.param < 0) return op.theta;
    if (!params || size_t(op.param) >= nparams) fail(QSE_ERR_INVALID, "op parameter index out of range");
    return op.theta + op.coeff * params[op.param];
}

uint64_t logical_to_physical_index(const qse_state* st, uint64_t L)
{
    uint64_t P = 0;
    for (uint32_t q = 0; q < st->n; ++q) P |= ((L >> q) & 1) << st->perm[q];
    return P;
}

uint64_t physical_to_logical_index(const qse_state* st, uint64_t P)
{
    uint64_t L = 0;
    for (uint32_t q = 0; q < st->n; ++q) L |= ((P >> st->perm[q]) & 1) << q;
    return L;
}

// ---- plan cache ----
// An execute of a program that ran before on a state in the same layout (a
// sampling loop that runs one circuit from |0..0> again and again, a repeated
// adjoint sweep at fixed parameters) reuses that plan: its pass programs, its
// kernels' sources and the compiled kernels.  Planning a 500-gate circuit and
// generating its kernels' sources takes close to a millisecond of host time,
// during which the device has nothing queued.  An entry's key holds every input
// the plan depends on, written field by field (plan::Gate has padding).
struct PlanEntry {
    std::string key;
    size_t hash = 0;
    uint64_t used = 0;
    plan::Plan pl;
    bool use_jit = false;
    std::vector<jit::Source> srcs;
    std::vector<std::shared_ptr<jit::Kernel>> ks;   // filled by the first run
};

struct PlanCache {
    std::vector<std::shared_ptr<PlanEntry>> entries;
    uint64_t tick = 0;
};

void destroy_plan_cache(qse_ctx* ctx)
{
    delete ctx->plan_cache;
    ctx->plan_cache = nullptr;
}

namespace {

constexpr size_t kPlanCacheEntries = 16;

struct KeyWriter {
    std::string s;
    template <class T>
    void put(const T& v)
    {
        s.append(reinterpret_cast<const char*>(&v), sizeof(T));
    }
    void put_options(const plan::Options& o)
    {
        put(o.k); put(o.rb); put(o.max_gates); put(o.max_terms); put(o.grads); put(o.max_slots);
        put(o.direct_phases); put(o.acc_mul); put(o.zz_fuse); put(o.keep_gphase);
    }
    void put_gates(const std::vector<plan::Gate>& gates)
    {
        put(uint64_t(gates.size()));
        s.reserve(s.size() + gates.size() * 96);
        for (const plan::Gate& g : gates) {
            put(g.type); put(g.t); put(g.c); put(g.cmask); put(g.theta); put(g.grad);
            s.append(reinterpret_cast<const char*>(g.m), sizeof g.m);
        }
    }
    // the state's layout: qubit count and logical -> physical map
    void put_state(const qse_state* st)
    {
        put(st->n);
        s.append(reinterpret_cast<const char*>(st->perm), st->n * sizeof(uint32_t));
    }
};

std::shared_ptr<PlanEntry> plan_cache_find(qse_ctx* ctx, const std::string& key, size_t hash)
{
    if (!ctx->plan_cache) return nullptr;
    for (auto& e : ctx->plan_cache->entries)
        if (e->hash == hash && e->key == key) {
            e->used = ++ctx->plan_cache->tick;
            return e;
        }
    return nullptr;
}

void plan_cache_insert(qse_ctx* ctx, std::shared_ptr<PlanEntry> e)
{
    if (!ctx->plan_cache) ctx->plan_cache = new PlanCache;
    PlanCache& c = *ctx->plan_cache;
    e->used = ++c.tick;
    if (c.entries.size() < kPlanCacheEntries) {
        c.entries.push_back(std::move(e));
        return;
    }
    auto lru = std::min_element(c.entries.begin(), c.entries.end(),
                                [](const auto& a, const auto& b) { return a->used < b->used; });
    *lru = std::move(e);   // an entry still in use by a caller stays alive through its shared_ptr
}

plan::Gate to_gate(const qse_op& op, double theta)
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

void check_qubits(const plan::Gate& g, uint32_t n)
{
    auto bad = [&](uint32_t q) { return q >= n; };
    switch (g.type) {
    case QSE_GATE_IDENTITY: return;
    case QSE_GATE_CNOT: case QSE_GATE_CPHASE: case QSE_GATE_SWAP:
        if (bad(g.t) || bad(g.c)) fail(QSE_ERR_QUBIT, "qubit index out of range");
        return;
    case QSE_GATE_MCPHASE:
        if (bad(g.t) || (n < 64 && (g.cmask >> n) != 0)) fail(QSE_ERR_QUBIT, "qubit index out of range");
        return;
    case QSE_GATE_H: case QSE_GATE_X: case QSE_GATE_Y: case QSE_GATE_Z: case QSE_GATE_PHASE:
    case QSE_GATE_RX: case QSE_GATE_RY: case QSE_GATE_RZ: case QSE_GATE_2X2:
        if (bad(g.t)) fail(QSE_ERR_QUBIT, "qubit index out of range");
        return;
    default: fail(QSE_ERR_UNSUPPORTED, "gate type " + std::to_string(g.type) + " is not executable");
    }
}

// One kernel per gate, in program order, on physical qubits (perm[logical]).
void apply_plain(qse_state* st, const plan::Gate& g)
{
    const uint32_t* P = st->perm;
    switch (g.type) {
    case QSE_GATE_IDENTITY: return;
    case QSE_GATE_H: launch_h(st, P[g.t]); return;
    case QSE_GATE_X: launch_x(st, P[g.t]); return;
    case QSE_GATE_Y: launch_y(st, P[g.t]); return;
    case QSE_GATE_Z: launch_z(st, P[g.t]); return;
    case QSE_GATE_PHASE: launch_phase_mask(st, uint64_t(1) << P[g.t], std::cos(g.theta), std::sin(g.theta)); return;
    case QSE_GATE_RX: launch_rx(st, P[g.t], std::cos(g.theta / 2.0), std::sin(g.theta / 2.0)); return;
    case QSE_GATE_RY: launch_ry(st, P[g.t], std::cos(g.theta / 2.0), std::sin(g.theta / 2.0)); return;
    case QSE_GATE_RZ:
        launch_rz(st, P[g.t], std::cos(-g.theta / 2.0), std::sin(-g.theta / 2.0), std::cos(g.theta / 2.0),
                  std::sin(g.theta / 2.0));
        return;
    case QSE_GATE_CNOT:
        if (g.c == g.t) return;
        launch_cnot(st, P[g.c], P[g.t]);
        return;
    case QSE_GATE_CPHASE:
        launch_phase_mask(st, (uint64_t(1) << P[g.c]) | (uint64_t(1) << P[g.t]), std::cos(g.theta), std::sin(g.theta));
        return;
    case QSE_GATE_MCPHASE: {
        uint64_t m = uint64_t(1) << P[g.t];
        for (uint64_t s = g.cmask; s; s &= s - 1) m |= uint64_t(1) << P[__builtin_ctzll(s)];
        launch_phase_mask(st, m, std::cos(g.theta), std::sin(g.theta));
        return;
    }
    case QSE_GATE_SWAP:
        // a relabelling of the logical -> physical map: no amplitude moves
        // (downloads, samples and later gates read through the map)
        if (g.t != g.c) std::swap(st->perm[g.t], st->perm[g.c]);
        return;
    case QSE_GATE_2X2: launch_gate2x2(st, P[g.t], g.m, 0); return;
    default: fail(QSE_ERR_UNSUPPORTED, "gate type not executable");
    }
}

size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

struct Uploaded {
    std::vector<tile::PassArgs> args;
    std::vector<const double2*> texp;   // per pass: (cos, sin) of each term's angle
};

// Packs every pass program into one pinned buffer and one H2D copy.  With
// term_phases, each pass also gets the (cos, sin) of its terms' angles (for
// k_group_values; only passes whose kernels read precomputed group values).
Uploaded upload_plan(qse_ctx* ctx, const plan::Plan& pl, bool term_phases = false)
{
    constexpr size_t kArr = 6;
    std::vector<size_t> off(pl.passes.size() * kArr);
    size_t total = 0;
    for (size_t i = 0; i < pl.passes.size(); ++i) {
        const plan::PassProgram& p = pl.passes[i];
        size_t* o = &off[kArr * i];
        o[0] = total; total = align16(total + p.ops.size() * sizeof(plan::KOp));
        o[1] = total; total = align16(total + p.layouts.size() * sizeof(plan::LayoutRec));
        o[2] = total; total = align16(total + p.terms.size() * sizeof(plan::TermRec));
        o[3] = total; total = align16(total + p.groups.size() * sizeof(plan::GroupRec));
        o[4] = total; total = align16(total + p.mats.size() * sizeof(double));
        o[5] = total; total = align16(total + (term_phases ? p.terms.size() * sizeof(double2) : 0));
    }
    total = std::max<size_t>(total, 16);
    QSE_CUDA(cudaEventSynchronize(ctx->plan_event));
    ctx->plan_host.reserve(total);
    ctx->plan_buf.reserve(total);
    char* h = static_cast<char*>(ctx->plan_host.ptr);
    for (size_t i = 0; i < pl.passes.size(); ++i) {
        const plan::PassProgram& p = pl.passes[i];
        const size_t* o = &off[kArr * i];
        std::memcpy(h + o[0], p.ops.data(), p.ops.size() * sizeof(plan::KOp));
        std::memcpy(h + o[1], p.layouts.data(), p.layouts.size() * sizeof(plan::LayoutRec));
        std::memcpy(h + o[2], p.terms.data(), p.terms.size() * sizeof(plan::TermRec));
        std::memcpy(h + o[3], p.groups.data(), p.groups.size() * sizeof(plan::GroupRec));
        std::memcpy(h + o[4], p.mats.data(), p.mats.size() * sizeof(double));
        double2* e = reinterpret_cast<double2*>(h + o[5]);
        if (term_phases)
            for (size_t t = 0; t < p.terms.size(); ++t)
                e[t] = make_double2(std::cos(p.terms[t].theta), std::sin(p.terms[t].theta));
    }
    QSE_CUDA(cudaMemcpyAsync(ctx->plan_buf.ptr, h, total, cudaMemcpyHostToDevice, ctx->stream));
    QSE_CUDA(cudaEventRecord(ctx->plan_event, ctx->stream));
    char* d = static_cast<char*>(ctx->plan_buf.ptr);
    Uploaded up;
    for (size_t i = 0; i < pl.passes.size(); ++i) {
        const plan::PassProgram& p = pl.passes[i];
        const size_t* o = &off[kArr * i];
        tile::PassArgs a{};
        a.ops = reinterpret_cast<const plan::KOp*>(d + o[0]);
        a.layouts = reinterpret_cast<const plan::LayoutRec*>(d + o[1]);
        a.terms = reinterpret_cast<const plan::TermRec*>(d + o[2]);
        a.groups = reinterpret_cast<const plan::GroupRec*>(d + o[3]);
        a.mats = reinterpret_cast<const double*>(d + o[4]);
        up.texp.push_back(reinterpret_cast<const double2*>(d + o[5]));
        a.outer_mask = p.outer_mask;
        a.nops = uint32_t(p.ops.size());
        a.ngroups = uint32_t(p.groups.size());
        a.nslots = uint32_t(p.slot_src.size());
        a.layout0 = p.layout0;
        a.k = p.k;
        std::memcpy(a.tile_phys, p.tile_phys, 16);
        up.args.push_back(a);
    }
    return up;
}

// The per-CTA values of a pass's diagonal groups, one row per tile (out[t * ng
// + g], the row CTA t of the pass copies).  The value of a direct group is the
// product of the unit phases (cos, sin) of its terms whose outer-qubit
// conditions hold for t's outer bits (t's bits deposited on the outer positions
// in ascending order, as the pass kernel numbers its CTAs); each term's phase
// is computed once on the host, so this kernel multiplies and never takes a
// sincos.  Other groups keep the plain sum of their angles.  A CTA handles
// kGvTiles consecutive tiles: their outer bits once into shared memory, then
// its threads walk the rows' elements in address order (coalesced stores).
// For the two tables of a split pass (jit::Source::gv_lo) the "tiles" are the
// values of one part of the outer qubits (outer_mask = that part); a term
// conditioned on the other part never holds there, and skip_unconditioned
// leaves the terms without a condition to the other table.
constexpr uint32_t kGvTiles = 32;

__global__ void __launch_bounds__(256) k_group_values(const plan::TermRec* __restrict__ terms,
                                                      const double2* __restrict__ texp,
                                                      const plan::GroupRec* __restrict__ groups, uint32_t ng,
                                                      uint64_t outer_mask, uint64_t ntiles, double2* __restrict__ out,
                                                      bool skip_unconditioned)
{
    __shared__ uint64_t s_ob[kGvTiles];
    const uint64_t t0 = uint64_t(blockIdx.x) * kGvTiles;
    if (threadIdx.x < kGvTiles) {
        uint64_t ob = 0, c = t0 + threadIdx.x;
        for (uint64_t m = outer_mask; m; m &= m - 1) {
            ob |= (c & 1ull) << (__ffsll((long long)m) - 1);
            c >>= 1;
        }
        s_ob[threadIdx.x] = ob;
    }
    __syncthreads();
    const uint32_t nt = uint32_t(min(uint64_t(kGvTiles), ntiles - t0));
    const uint32_t cnt = nt * ng;
    double2* row = out + t0 * ng;
    for (uint32_t e = threadIdx.x; e < cnt; e += blockDim.x) {
        const uint32_t tl = e / ng, g = e - tl * ng;
        const uint64_t ob = s_ob[tl];
        const plan::GroupRec gr = groups[g];
        double2 v;
        if (gr.direct) {
            v = make_double2(1.0, 0.0);
            for (uint32_t k = 0; k < gr.count; ++k) {
                const uint64_t oc = terms[gr.first + k].ocond;
                if ((ob & oc) == oc && (oc || !skip_unconditioned)) {
                    const double2 f = texp[gr.first + k];
                    v = make_double2(v.x * f.x - v.y * f.y, v.x * f.y + v.y * f.x);
                }
            }
        } else {
            double th = 0.0;
            for (uint32_t k = 0; k < gr.count; ++k) {
                const plan::TermRec t = terms[gr.first + k];
                if ((ob & t.ocond) == t.ocond && (t.ocond || !skip_unconditioned)) th += t.theta;
            }
            v = make_double2(th, 0.0);
        }
        row[e] = v;
    }
}

// Specialised pass kernels repay their compile time (NVRTC: about a second or
// more per distinct kernel) when a pass is expensive, i.e. on large states, or
// when few of a plan's kernels are new.  A deep circuit on a small state can
// need hundreds of distinct kernels; its plan runs on the interpreter instead.
constexpr uint32_t kJitAlwaysQubits = 22;
constexpr size_t kJitMaxNewKernels = 32;

// Plans gates for the specialised kernels (their sources generated into srcs,
// use_jit = true) or, when the context disables them or they are not worth
// compiling, for the interpreter (angle accumulators, use_jit = false).
// Specialised plans are kept in the context's plan cache.
std::shared_ptr<PlanEntry> plan_for(qse_state* st, const std::vector<plan::Gate>& gates, plan::Options opt, int ns,
                                    bool prob_out = false)
{
    qse_ctx* ctx = st->ctx;
    auto e = std::make_shared<PlanEntry>();
    e->use_jit = ctx->jit != 0;
    opt.acc_mul = e->use_jit;
    if (e->use_jit) {
        KeyWriter w;
        w.put('F');
        w.put(ctx->jit);
        w.put(ns);
        w.put(prob_out);
        w.put(st->lazy_basis);
        w.put(st->lazy_basis ? st->lazy_umask : 0);
        w.put(st->lazy_basis ? st->lazy_pmask : 0);
        const char* dbg = std::getenv("QSE_DEBUG_BOUNDS");   // read by jit::generate
        w.s.append(dbg ? dbg : "");
        w.put('\0');
        w.put_options(opt);
        w.put_state(st);
        w.put_gates(gates);
        e->key = std::move(w.s);
        e->hash = std::hash<std::string>{}(e->key);
        if (auto hit = plan_cache_find(ctx, e->key, e->hash)) return hit;
    }
    e->pl = plan::build(gates, st->n, st->perm, opt);
    if (!e->use_jit) return e;
    const plan::Plan& pl = e->pl;
    e->srcs.reserve(pl.passes.size());
    // the last pass may also write the probabilities in logical order
    uint8_t lpos[64] = {0};
    for (uint32_t q = 0; q < st->n; ++q) lpos[pl.perm_final[q]] = uint8_t(q);
    for (size_t i = 0; i < pl.passes.size(); ++i) {
        const bool basis_in = i == 0 && ns == 1 && st->lazy_basis;
        const bool prob = prob_out && ns == 1 && i + 1 == pl.passes.size();
        e->srcs.push_back(jit::generate(pl.passes[i], ns, basis_in, ctx->jit == 2, st->n >= jit::kPreGroupQubits,
                                        basis_in ? st->lazy_umask : 0, prob ? lpos : nullptr,
                                        basis_in ? st->lazy_pmask : 0));
    }
    if (st->n >= kJitAlwaysQubits || jit::count_uncached(e->srcs) <= kJitMaxNewKernels) {
        plan_cache_insert(ctx, e);
        return e;
    }
    e->use_jit = false;
    e->srcs.clear();
    e->key.clear();
    opt.acc_mul = false;
    opt.rb = std::min(opt.rb, 4u);   // the interpreter kernel holds at most 16 amplitudes per thread
    e->pl = plan::build(gates, st->n, st->perm, opt);
    return e;
}

// Runs the passes of a plan: specialised NVRTC kernels (jit.cpp, sources from
// plan_for) or the generic tile-program interpreter (tile.cu).
struct PassRunner {
    qse_ctx* ctx;
    qse_state* st;
    Uploaded& up;
    int ns;
    uint32_t rb;
    bool jit;
    const std::vector<jit::Source>& srcs;
    const std::vector<std::shared_ptr<jit::Kernel>>& ks;
    std::vector<uint32_t> kq;

    PassRunner(qse_state* s, PlanEntry& e, Uploaded& u, int nstates, uint32_t regbits)
        : ctx(s->ctx), st(s), up(u), ns(nstates), rb(regbits), jit(e.use_jit), srcs(e.srcs), ks(e.ks)
    {
        for (const auto& p : e.pl.passes) kq.push_back(p.k);
        if (!jit || e.ks.size() == e.srcs.size()) return;
        std::vector<const jit::Source*> ptrs;
        for (const auto& s2 : e.srcs) ptrs.push_back(&s2);
        e.ks = jit::get_kernels(ptrs);
    }

    void run(size_t i, double2* lam, double* part)
    {
        // the first pass of a compact-input plan reads the compact state
        if (jit && i == 0 && ns == 1 && st->lazy_basis && st->lazy_umask)
            lam = const_cast<double2*>(static_cast<const double2*>(st->lazy_src));
        tile::PassArgs a = up.args[i];
        a.psi = reinterpret_cast<double2*>(st->amp);
        a.lam = lam;
        a.slot_partial = part;
        // one NVTX range per planned pass (host side, around the launch; free
        // unless a profiler injects an NVTX handler)
        char name[64];
        std::snprintf(name, sizeof(name), "qse pass %zu/%zu %s%s", i + 1, up.args.size(),
                      ns == 2 ? "adjoint " : "", !jit ? "interpreter" : srcs[i].streamed ? "streamed" : "tile");
        nvtxRangePushA(name);
        if (!jit) {
            tile::launch_pass(ctx, a, st->n, rb, ns);
            nvtxRangePop();
            return;
        }
        const void* gvt = nullptr;
        if (srcs[i].pre_gv) {
            // one table of every tile's row, or (gv_lo) a table for each part of the outer qubits
            const uint32_t nob = st->n - kq[i], lo = srcs[i].gv_lo;
            uint64_t lomask = 0, m = a.outer_mask;
            for (uint32_t b = 0; b < lo; ++b, m &= m - 1) lomask |= m & (~m + 1);
            struct Part { uint64_t mask, ntiles; bool skip; };
            const Part parts[2] = {{lo ? lomask : a.outer_mask, uint64_t(1) << (lo ? lo : nob), false},
                                   {a.outer_mask & ~lomask, uint64_t(1) << (nob - lo), true}};
            const int nparts = lo ? 2 : 1;
            const uint64_t ng = srcs[i].ngroups;
            ctx->gv_buf.reserve((parts[0].ntiles + (lo ? parts[1].ntiles : 0)) * ng * sizeof(double2));
            double2* out = static_cast<double2*>(ctx->gv_buf.ptr);
            for (int p = 0; p < nparts; ++p) {
                const uint64_t blocks = (parts[p].ntiles + kGvTiles - 1) / kGvTiles;
                k_group_values<<<unsigned(blocks), 256, 0, ctx->stream>>>(a.terms, up.texp[i], a.groups, uint32_t(ng),
                                                                         parts[p].mask, parts[p].ntiles, out,
                                                                         parts[p].skip);
                QSE_CUDA(cudaGetLastError());
                count_launch(ctx);
                out += parts[p].ntiles * ng;
            }
            gvt = ctx->gv_buf.ptr;
        }
        cudaEvent_t stop = tile::pass_timer_begin(ctx);
        jit::launch(ctx, *ks[i], srcs[i], st->n, kq[i], a.psi, lam, a.terms, a.groups, part, st->lazy_index, gvt);
        tile::pass_timer_end(ctx, stop);
        count_launch(ctx);
        nvtxRangePop();
    }
};

uint32_t tile_qubits_for(const qse_ctx* ctx, uint32_t n, uint32_t rb, uint32_t kmax)
{
    uint32_t k = std::min<uint32_t>(std::max(ctx->tile_qubits, int(rb) + 1), kmax);
    return std::min(k, n);
}

// noisy gates of the list in program order (types in the rate map)
void run_noise(qse_state* st, qse_noise* nz, const qse_op* ops, size_t nops, const double* inj, size_t ninj,
               qse_exec_stats* stats)
{
    qse_ctx* ctx = st->ctx;
    std::vector<int32_t> types;
    std::vector<uint32_t> targets;
    for (size_t i = 0; i < nops; ++i) {
        int t = ops[i].type;
        if (t >= 0 && t < 16 && nz->cfg.rates[t] >= 0.0) {
            types.push_back(t);
            targets.push_back(ops[i].target);
        }
    }
    const size_t ng = types.size();
    if (stats) stats->noisy_gates = ng;
    if (ng == 0) return;
    std::vector<double> uni;
    if (nz->cfg.rng_mode == QSE_RNG_MT19937) {
        uni.resize(2 * ng);
        for (size_t i = 0; i < 2 * ng; ++i) uni[i] = nz->dist(nz->gen);
    } else if (nz->cfg.rng_mode == QSE_RNG_INJECTED) {
        if (!inj || ninj < 2 * ng) fail(QSE_ERR_INVALID, "injected noise needs 2 uniforms per noisy gate");
        uni.assign(inj, inj + 2 * ng);
    }
    size_t bytes = ng * 4 + ng * 4 + uni.size() * 8 + 64;
    ctx->host_small2.reserve(bytes);
    ctx->scratch.reserve(bytes);
    char* h = static_cast<char*>(ctx->host_small2.ptr);
    size_t o_t = 0, o_g = align16(ng * 4), o_u = align16(o_g + ng * 4);
    std::memcpy(h + o_t, types.data(), ng * 4);
    std::memcpy(h + o_g, targets.data(), ng * 4);
    if (!uni.empty()) std::memcpy(h + o_u, uni.data(), uni.size() * 8);
    char* d = static_cast<char*>(ctx->scratch.ptr);
    QSE_CUDA(cudaMemcpyAsync(d, h, o_u + uni.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
    noise_decide(nz, reinterpret_cast<const int32_t*>(d + o_t), reinterpret_cast<const uint32_t*>(d + o_g), ng,
                 uni.empty() ? nullptr : reinterpret_cast<const double*>(d + o_u));
    QSE_CUDA(cudaStreamSynchronize(ctx->stream));
}

plan::Options fused_options(const qse_ctx* ctx, uint32_t n)
{
    plan::Options opt;
    opt.rb = 4;
    opt.k = tile_qubits_for(ctx, n, 4, 12);
    // specialised tile kernels on 4096-amplitude tiles hold 32 amplitudes per
    // thread (128 threads, three CTAs per SM): twice the independent FP64 work
    // per thread and one layout exchange per five register qubits instead of four
    if (ctx->jit == 1 && opt.k == 12) opt.rb = 5;
    opt.max_gates = uint32_t(std::max(0, ctx->max_gates_per_pass));
    if (ctx->jit && (opt.max_gates == 0 || opt.max_gates > plan::kJitMaxGates)) opt.max_gates = plan::kJitMaxGates;
    opt.zz_fuse = true;
    return opt;
}

// Forward passes of gates on st through the planner; returns the pass count.
// prob_out: the last pass also writes the probabilities in logical order and
// their block sums into the state's sampling buffer (specialised kernels,
// states of at least one 4096-block).
uint64_t run_fused(qse_state* st, const std::vector<plan::Gate>& gates, bool prob_out = false)
{
    qse_ctx* ctx = st->ctx;
    prob_out = prob_out && st->size() >= 4096 && ctx->jit != 0;
    const std::shared_ptr<PlanEntry> e = plan_for(st, gates, fused_options(ctx, st->n), 1, prob_out);
    const plan::Plan& pl = e->pl;
    const bool use_jit = e->use_jit;
    const std::vector<jit::Source>& srcs = e->srcs;
    if (!use_jit) materialize(st);  // interpreter passes read the state
    double* prob = nullptr;
    const bool with_bsum = !srcs.empty() && srcs.back().prob_bsum;
    if (prob_out && use_jit && !srcs.empty() && srcs.back().prob) {
        st->cdf.reserve(prob_buffer_bytes(st->size()));
        prob = static_cast<double*>(st->cdf.ptr);
        QSE_CUDA(cudaMemsetAsync(prob + st->size(), 0, (st->size() / 4096) * 8, ctx->stream));
        st->cdf_version = ~uint64_t(0);   // the buffer's cumulative values are overwritten
    }
    Uploaded up = upload_plan(ctx, pl, use_jit && st->n >= jit::kPreGroupQubits);
    PassRunner runner(st, *e, up, 1, 4);
    for (size_t i = 0; i < up.args.size(); ++i) runner.run(i, nullptr, i + 1 == up.args.size() ? prob : nullptr);
    if (!up.args.empty()) {   // the first pass wrote every amplitude
        st->lazy_basis = false;
        st->lazy_umask = 0;
        st->lazy_pmask = 0;
        st->lazy_src = nullptr;
    }
    for (uint32_t q = 0; q < st->n; ++q) st->perm[q] = pl.perm_final[q];
    if (prob) {
        st->prob_version = st->version;
        st->prob_pending = true;
        st->prob_bsum = with_bsum;
    }
    return pl.passes.size();
}

// ---- compact prefix ----
// A circuit started from a basis state touches its qubits progressively (a
// QFT's first passes act on its low qubits while the others are still |0>).
// While the qubits touched so far are few, the state is that of those qubits
// times the untouched qubits' basis bits, so the leading passes can run on a
// state of only the touched qubits: 2^m amplitudes (at most 64 MiB, resident
// in L2) instead of 2^n.  The first pass over the full state then reads its
// input from that compact state (jit.cpp, compact input) instead of from HBM.
// Touched means acted on non-diagonally (a target other than of a phase, or a
// SWAP); an untouched qubit keeps its basis bit through the prefix, so in the
// prefix's diagonal gates and CNOT controls it is a known 0 or 1: those gates
// drop, lose that qubit, or become a factor of the whole state (compact_gate).
constexpr uint32_t kCompactMinQubits = 24;   // full states this large (smaller ones gain little)
constexpr uint32_t kCompactMaxQubits = 22;   // compact states up to this size

// qubits a gate acts on non-diagonally
uint64_t gate_nondiag(const plan::Gate& g)
{
    auto b = [](uint32_t q) { return uint64_t(1) << q; };
    switch (g.type) {
    case QSE_GATE_H: case QSE_GATE_X: case QSE_GATE_Y: case QSE_GATE_RX: case QSE_GATE_RY: case QSE_GATE_2X2:
        return b(g.t);
    case QSE_GATE_CNOT: return g.c == g.t ? 0 : b(g.t);   // control == target: a no-op
    case QSE_GATE_SWAP: return g.c == g.t ? 0 : b(g.t) | b(g.c);
    default: return 0;   // identity and the phase gates
    }
}

// Gate g of the prefix on the compact state: qubits in `touched` renumbered by
// rank, the others replaced by their basis bit (bit); a gate that becomes a
// factor of the whole state multiplies glob instead.  Appends to out.
void compact_gate(const plan::Gate& g, uint64_t touched, const uint32_t* rank, uint64_t bits,
                  std::vector<plan::Gate>& out, double& gre, double& gim)
{
    auto in = [&](uint32_t q) { return (touched >> q) & 1; };
    auto bit = [&](uint32_t q) { return (bits >> q) & 1; };
    auto mul = [&](double c, double s) {
        const double r = gre * c - gim * s, i = gre * s + gim * c;
        gre = r;
        gim = i;
    };
    plan::Gate x = g;
    switch (g.type) {
    case QSE_GATE_IDENTITY: return;
    case QSE_GATE_Z: case QSE_GATE_PHASE: case QSE_GATE_RZ:
        if (in(g.t)) break;
        if (g.type == QSE_GATE_RZ) mul(std::cos(g.theta / 2), bit(g.t) ? std::sin(g.theta / 2) : -std::sin(g.theta / 2));
        else if (bit(g.t)) {
            if (g.type == QSE_GATE_Z) mul(-1.0, 0.0);
            else mul(std::cos(g.theta), std::sin(g.theta));
        }
        return;
    case QSE_GATE_CNOT:
        if (g.c == g.t) return;
        if (!in(g.c)) {   // a classical control: X on the target or nothing
            if (!bit(g.c)) return;
            x.type = QSE_GATE_X;
        }
        break;
    case QSE_GATE_CPHASE: case QSE_GATE_MCPHASE: {
        // phase theta on the amplitudes whose bits of `all` are all 1
        uint64_t all = g.type == QSE_GATE_CPHASE ? ((uint64_t(1) << g.t) | (uint64_t(1) << g.c))
                                                 : (g.cmask | (uint64_t(1) << g.t));
        const uint64_t fixed = all & ~touched;
        if (!fixed) break;                      // every qubit touched: the gate as it is
        if ((fixed & bits) != fixed) return;   // a classical qubit at 0: never applies
        all &= touched;
        if (!all) {
            mul(std::cos(g.theta), std::sin(g.theta));
            return;
        }
        x.type = QSE_GATE_MCPHASE;
        x.t = uint32_t(__builtin_ctzll(all));
        x.cmask = all & (all - 1);
        x.c = 0;
        break;
    }
    default: break;
    }
    x.t = rank[x.t];
    if (x.type == QSE_GATE_CNOT || x.type == QSE_GATE_CPHASE || x.type == QSE_GATE_SWAP) x.c = rank[x.c];
    if (x.type == QSE_GATE_MCPHASE) {
        uint64_t cm = 0;
        for (uint64_t b = x.cmask; b; b &= b - 1) cm |= uint64_t(1) << rank[__builtin_ctzll(b)];
        x.cmask = cm;
    }
    out.push_back(x);
}

qse_state* compact_state(qse_ctx* ctx, uint32_t m)
{
    if (!ctx->compact) {
        auto* cs = new qse_state;
        cs->ctx = ctx;
        cs->n = kCompactMaxQubits;
        if (cudaMalloc(&cs->amp, (cs->size() + 128) * 16) != cudaSuccess) {   // + the product qubits' table
            cudaGetLastError();
            delete cs;
            fail(QSE_ERR_OOM, "device allocation of the compact state failed");
        }
        ctx->compact = cs;
    }
    qse_state* cs = ctx->compact;
    cs->n = m;
    for (uint32_t q = 0; q < 64; ++q) cs->perm[q] = q;
    cs->touch();
    return cs;
}

// logical qubits a gate involves
uint64_t gate_support(const plan::Gate& g)
{
    auto b = [](uint32_t q) { return uint64_t(1) << q; };
    switch (g.type) {
    case QSE_GATE_IDENTITY: return 0;
    case QSE_GATE_CNOT: case QSE_GATE_CPHASE: case QSE_GATE_SWAP: return b(g.t) | b(g.c);
    case QSE_GATE_MCPHASE: return b(g.t) | g.cmask;
    default: return b(g.t);
    }
}

bool one_qubit_gate(int type)
{
    switch (type) {
    case QSE_GATE_H: case QSE_GATE_X: case QSE_GATE_Y: case QSE_GATE_Z: case QSE_GATE_PHASE:
    case QSE_GATE_RX: case QSE_GATE_RY: case QSE_GATE_RZ: case QSE_GATE_2X2:
        return true;
    default: return false;
    }
}

// v <- (matrix of g) v for a one-qubit gate; v = (re, im) of the qubit's |0>
// and |1> amplitudes (the matrices of the pass kernels' ops and of apply_plain)
void apply_one_qubit(const plan::Gate& g, double* v)
{
    const double a0 = v[0], b0 = v[1], a1 = v[2], b1 = v[3];
    auto set = [&](double r0, double i0, double r1, double i1) {
        v[0] = r0;
        v[1] = i0;
        v[2] = r1;
        v[3] = i1;
    };
    const double c = std::cos(g.theta / 2.0), s = std::sin(g.theta / 2.0);
    switch (g.type) {
    case QSE_GATE_H: {
        const double h = 0.70710678118654752440;   // 1/sqrt(2)
        set(h * (a0 + a1), h * (b0 + b1), h * (a0 - a1), h * (b0 - b1));
        return;
    }
    case QSE_GATE_X: set(a1, b1, a0, b0); return;
    case QSE_GATE_Y: set(b1, -a1, -b0, a0); return;   // [[0, -i], [i, 0]]
    case QSE_GATE_Z: set(a0, b0, -a1, -b1); return;
    case QSE_GATE_PHASE: {
        const double pc = std::cos(g.theta), ps = std::sin(g.theta);
        set(a0, b0, a1 * pc - b1 * ps, a1 * ps + b1 * pc);
        return;
    }
    case QSE_GATE_RX: set(c * a0 + s * b1, c * b0 - s * a1, s * b0 + c * a1, c * b1 - s * a0); return;   // [[c, -is], [-is, c]]
    case QSE_GATE_RY: set(c * a0 - s * a1, c * b0 - s * b1, s * a0 + c * a1, s * b0 + c * b1); return;   // [[c, -s], [s, c]]
    case QSE_GATE_RZ: set(a0 * c + b0 * s, b0 * c - a0 * s, a1 * c - b1 * s, a1 * s + b1 * c); return;   // diag(e^-i/2, e^i/2)
    case QSE_GATE_2X2: {
        const double* m = g.m;
        set(m[0] * a0 - m[1] * b0 + m[2] * a1 - m[3] * b1, m[0] * b0 + m[1] * a0 + m[2] * b1 + m[3] * a1,
            m[4] * a0 - m[5] * b0 + m[6] * a1 - m[7] * b1, m[4] * b0 + m[5] * a0 + m[6] * b1 + m[7] * a1);
        return;
    }
    default: fail(QSE_ERR_INVALID, "internal: not a one-qubit gate");
    }
}

// Product qubits: a qubit outside the compact state (mask `compact`) whose
// first gates after the prefix act on it alone stays in a single-qubit state
// through them (its basis bit from lbits, then those gates).  For every such
// qubit whose leading gates include a non-diagonal one, the gates leave `rest`
// and its two amplitudes go to phi[q] (re0, im0, re1, im1); returns the mask of
// those qubits.  The first pass over the full state multiplies them into its
// input, instead of applying the gates to every amplitude.
uint64_t absorb_product_qubits(std::vector<plan::Gate>& rest, uint64_t compact, uint64_t lbits, double (*phi)[4])
{
    uint64_t blocked = compact, nondiag = 0;
    std::vector<char> lead(rest.size(), 0);
    for (size_t i = 0; i < rest.size(); ++i) {
        const plan::Gate& g = rest[i];
        if (one_qubit_gate(g.type) && !((blocked >> g.t) & 1)) {
            lead[i] = 1;
            nondiag |= gate_nondiag(g);
            continue;
        }
        blocked |= gate_support(g);
    }
    const uint64_t pq = nondiag;   // a run of phases alone stays a basis qubit with its phases in the plan
    if (!pq) return 0;
    for (uint64_t s = pq; s; s &= s - 1) {
        const uint32_t q = uint32_t(__builtin_ctzll(s));
        const bool one = (lbits >> q) & 1;
        phi[q][0] = one ? 0.0 : 1.0;
        phi[q][1] = 0.0;
        phi[q][2] = one ? 1.0 : 0.0;
        phi[q][3] = 0.0;
    }
    std::vector<plan::Gate> kept;
    kept.reserve(rest.size());
    for (size_t i = 0; i < rest.size(); ++i) {
        if (lead[i] && ((pq >> rest[i].t) & 1)) apply_one_qubit(rest[i], phi[rest[i].t]);
        else kept.push_back(rest[i]);
    }
    rest.swap(kept);
    return pq;
}

// Runs the longest prefix of the plan's passes (at least two) whose gates
// touch at most kCompactMaxQubits qubits on the compact state and leaves st
// in the lazy compact form; rest = the other gates in program order (a valid
// order: every gate of the prefix passes runs before every other gate in the
// plan, and both parts keep their program order, which the plan's order only
// changes between gates that commute).  False (nothing done) when no such prefix exists.  A CPHASE or
// MCPHASE that keeps only touched qubits becomes an MCPHASE on them (the same
// phase on the same amplitudes).
bool compact_prefix(qse_state* st, const std::vector<plan::Gate>& gates_in, std::vector<plan::Gate>& rest,
                    uint64_t& passes)
{
    qse_ctx* ctx = st->ctx;
    if (!ctx->jit || !st->lazy_basis || st->lazy_umask || st->n < kCompactMinQubits) return false;
    // the zz rewrite moves gates between slots: apply it first so that the
    // plan's source indices name the gates that run
    plan::Options opt = fused_options(ctx, st->n);
    std::vector<plan::Gate> fused;
    const std::vector<plan::Gate>& gates = plan::fuse_zz(gates_in, fused) ? fused : gates_in;
    opt.zz_fuse = false;
    opt.acc_mul = true;
    KeyWriter w;
    w.put('C');
    w.put_options(opt);
    w.put_state(st);
    w.put_gates(gates);
    const size_t hash = std::hash<std::string>{}(w.s);
    std::shared_ptr<PlanEntry> e = plan_cache_find(ctx, w.s, hash);
    if (!e) {
        e = std::make_shared<PlanEntry>();
        e->pl = plan::build(gates, st->n, st->perm, opt);
        e->key = std::move(w.s);
        e->hash = hash;
        plan_cache_insert(ctx, e);
    }
    const plan::Plan& pl = e->pl;
    size_t K = 0;
    uint64_t u = 0, uK = 0;
    for (size_t i = 0; i < pl.passes.size(); ++i) {
        for (uint32_t g : pl.passes[i].order) u |= gate_nondiag(gates[g]);
        if (uint32_t(__builtin_popcountll(u)) > kCompactMaxQubits) break;
        K = i + 1;
        uK = u;
    }
    if (K < 2 || uK == 0) return false;
    // compact qubit r = the touched qubit with the r-th lowest physical position
    std::vector<uint32_t> qs;
    for (uint32_t q = 0; q < st->n; ++q)
        if ((uK >> q) & 1) qs.push_back(q);
    std::sort(qs.begin(), qs.end(), [&](uint32_t a, uint32_t b) { return st->perm[a] < st->perm[b]; });
    const uint32_t m = uint32_t(qs.size());
    uint32_t rank[64] = {0};
    uint64_t umask = 0, cbasis = 0, lbits = 0;   // lbits: basis bit of every logical qubit
    for (uint32_t q = 0; q < st->n; ++q) lbits |= ((st->lazy_index >> st->perm[q]) & 1) << q;
    for (uint32_t r = 0; r < m; ++r) {
        rank[qs[r]] = r;
        umask |= uint64_t(1) << st->perm[qs[r]];
        cbasis |= ((lbits >> qs[r]) & 1) << r;
    }
    std::vector<char> in_prefix(gates.size(), 0);
    std::vector<plan::Gate> sub;
    double gre = 1.0, gim = 0.0;
    for (size_t i = 0; i < K; ++i)
        for (uint32_t g : pl.passes[i].order) in_prefix[g] = 1;
    // the prefix's gates in program order (a pass lists its SWAPs first: they
    // only relabel there, but on the compact state they run where they stand)
    for (size_t g = 0; g < gates.size(); ++g)
        if (in_prefix[g]) compact_gate(gates[g], uK, rank, lbits, sub, gre, gim);
    if (gre != 1.0 || gim != 0.0) {   // the factors of the classical qubits' phases
        plan::Gate f{};
        f.type = QSE_GATE_2X2;
        f.t = 0;
        f.m[0] = gre;
        f.m[1] = gim;
        f.m[6] = gre;
        f.m[7] = gim;
        sub.push_back(f);
    }
    rest.clear();
    for (size_t g = 0; g < gates.size(); ++g)
        if (!in_prefix[g]) rest.push_back(gates[g]);
    double phi[64][4];
    const uint64_t pq = absorb_product_qubits(rest, uK, lbits, phi);
    // the prefix on the compact state (its passes are not the full state's:
    // they stay out of the pass timings)
    qse_state* cs = compact_state(ctx, m);
    mark_basis(cs, cbasis);
    const bool timing = ctx->time_passes;
    ctx->time_passes = false;
    try {
        if (m < 4) {   // as execute_program runs states this small: gate by gate
            materialize(cs);
            for (const plan::Gate& g : sub) apply_plain(cs, g);
            passes = sub.size();
        } else {
            passes = run_fused(cs, sub);
        }
        materialize(cs);
        canonicalize(cs);
    } catch (...) {
        ctx->time_passes = timing;
        throw;
    }
    ctx->time_passes = timing;
    // the product qubits' amplitudes after the compact ones, in ascending
    // physical position
    uint64_t pmask = 0;
    for (uint32_t q = 0; q < st->n; ++q)
        if ((pq >> q) & 1) pmask |= uint64_t(1) << st->perm[q];
    if (pmask) {
        std::vector<double> tab;
        for (uint64_t s = pmask; s; s &= s - 1) {
            const uint32_t p = uint32_t(__builtin_ctzll(s));
            uint32_t q = 0;
            while (st->perm[q] != p) ++q;
            tab.insert(tab.end(), phi[q], phi[q] + 4);
        }
        QSE_CUDA(cudaMemcpyAsync(cs->amp + 2 * (size_t(1) << m), tab.data(), tab.size() * 8, cudaMemcpyHostToDevice,
                                 ctx->stream));
    }
    st->lazy_umask = umask;
    st->lazy_pmask = pmask;
    st->lazy_src = cs->amp;
    return true;
}

}  // namespace

void destroy_compact_state(qse_ctx* ctx)
{
    if (!ctx->compact) return;
    cudaFree(ctx->compact->amp);
    if (ctx->compact->aux) cudaFree(ctx->compact->aux);
    delete ctx->compact;
    ctx->compact = nullptr;
}

void execute_program(qse_state* st, const qse_op* ops, size_t nops, const double* params, size_t nparams,
                     qse_noise* noise, const double* inj, size_t ninj, qse_exec_stats* stats)
{
    qse_ctx* ctx = st->ctx;
    const uint64_t launches0 = ctx->launches;
    if (stats) *stats = qse_exec_stats{};
    st->touch();
    std::vector<plan::Gate> gates;
    gates.reserve(nops);
    for (size_t i = 0; i < nops; ++i) {
        gates.push_back(to_gate(ops[i], bound_angle(ops[i], params, nparams)));
        check_qubits(gates.back(), st->n);
    }
    if (noise && noise->cfg.enabled) {
        if (noise->n != st->n) fail(QSE_ERR_INVALID, "noise object was created for a different qubit count");
        run_noise(st, noise, ops, nops, inj, ninj, stats);
    }
    uint64_t passes = 0;
    if (!ctx->fusion || st->n < 4 || !ctx->jit) materialize(st);  // only JIT passes start from a lazy basis state
    if (!ctx->fusion || st->n < 4) {
        for (const plan::Gate& g : gates) apply_plain(st, g);
        passes = gates.size();
    } else {
        // probabilities for the sampler from the last pass: only while the
        // state is being sampled (the last ones written were read) and no
        // Pauli frame follows
        if (st->prob_pending) st->prob_hint = st->prob_pending = false;
        const bool prob_out = st->prob_hint && !(noise && noise->cfg.enabled);
        std::vector<plan::Gate> rest;
        uint64_t compact_passes = 0;
        if (compact_prefix(st, gates, rest, compact_passes)) {
            passes = compact_passes + run_fused(st, rest, prob_out);
            materialize(st);   // no pass consumed the compact form (nothing after the prefix)
        } else {
            passes = run_fused(st, gates, prob_out);
        }
    }
    if (noise && noise->cfg.enabled) launch_pauli_frame(st, noise->d_counts);
    if (stats) {
        stats->gates = nops;
        stats->passes = passes;
        stats->kernels = ctx->launches - launches0;
    }
}

void apply_single(qse_state* st, const qse_op& op)
{
    materialize(st);
    plan::Gate g = to_gate(op, op.theta);
    check_qubits(g, st->n);
    st->touch();
    apply_plain(st, g);
}

void canonicalize(qse_state* st)
{
    materialize(st);
    st->touch();
    // restore logical == physical with physical qubit swaps (each a half sweep)
    for (uint32_t q = 0; q < st->n; ++q) {
        if (st->perm[q] == q) continue;
        // find the logical qubit r currently sitting on physical q
        uint32_t r = q;
        for (uint32_t s = 0; s < st->n; ++s)
            if (st->perm[s] == q) r = s;
        launch_swap(st, q, st->perm[q]);
        std::swap(st->perm[q], st->perm[r]);
    }
}

// ---------------------------------------------------------------- observables
namespace {

constexpr int kRB = 256;

__device__ __forceinline__ double obs_value(uint64_t x, const uint64_t* z, const double* w, uint32_t nt, double c)
{
    double v = c;
    for (uint32_t t = 0; t < nt; ++t) v += (__popcll(x & z[t]) & 1) ? -w[t] : w[t];
    return v;
}

// partial[b] = sum O(x)|psi_x|^2 over the block's range; lam = O psi if lam != nullptr
__global__ void __launch_bounds__(kRB) k_obs(const double2* __restrict__ psi, double2* __restrict__ lam, uint64_t size,
                                             const uint64_t* __restrict__ z, const double* __restrict__ w, uint32_t nt,
                                             double c, double* __restrict__ partial)
{
    __shared__ double sh[kRB / 32];
    extern __shared__ uint64_t sz[];
    double* sw = reinterpret_cast<double*>(sz + nt);
    for (uint32_t t = threadIdx.x; t < nt; t += blockDim.x) { sz[t] = z[t]; sw[t] = w[t]; }
    __syncthreads();
    double acc = 0.0;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < size; i += uint64_t(gridDim.x) * blockDim.x) {
        double2 v = psi[i];
        double o = obs_value(i, sz, sw, nt, c);
        acc += o * (v.x * v.x + v.y * v.y);
        if (lam) lam[i] = make_double2(o * v.x, o * v.y);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < kRB / 32; ++i) t += sh[i];
        partial[blockIdx.x] = t;
    }
}

// out[src[s]] = sum_b partial[s][b]
__global__ void __launch_bounds__(kRB) k_reduce_slots(const double* __restrict__ partial, uint32_t nslots, uint64_t nb,
                                                      const int32_t* __restrict__ src, double* __restrict__ out)
{
    __shared__ double sh[kRB / 32];
    for (uint32_t s = blockIdx.x; s < nslots; s += gridDim.x) {
        double acc = 0.0;
        for (uint64_t b = threadIdx.x; b < nb; b += blockDim.x) acc += partial[uint64_t(s) * nb + b];
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int i = 0; i < kRB / 32; ++i) t += sh[i];
            out[src[s]] += t;
        }
        __syncthreads();
    }
}

struct ObsDev {
    const uint64_t* z;
    const double* w;
    uint32_t nt;
    double c;
};

// Physical-qubit copy of the observable in device scratch (after `reserve_extra` bytes).
ObsDev upload_obs(qse_state* st, const qse_observable* obs, char* dbase, char* hbase)
{
    ObsDev o{};
    o.nt = uint32_t(obs->nterms);
    o.c = obs->constant;
    uint64_t* hz = reinterpret_cast<uint64_t*>(hbase);
    double* hw = reinterpret_cast<double*>(hbase + 8 * obs->nterms);
    for (size_t t = 0; t < obs->nterms; ++t) {
        uint64_t m = obs->zmask[t], pm = 0;
        if (st->n < 64 && (m >> st->n) != 0) fail(QSE_ERR_QUBIT, "observable acts on a qubit out of range");
        for (; m; m &= m - 1) pm |= uint64_t(1) << st->perm[__builtin_ctzll(m)];
        hz[t] = pm;
        hw[t] = obs->weight[t];
    }
    QSE_CUDA(cudaMemcpyAsync(dbase, hbase, 16 * obs->nterms, cudaMemcpyHostToDevice, st->ctx->stream));
    o.z = reinterpret_cast<const uint64_t*>(dbase);
    o.w = reinterpret_cast<const double*>(dbase + 8 * obs->nterms);
    return o;
}

double run_obs(qse_state* st, const qse_observable* obs, double2* lam)
{
    materialize(st);
    qse_ctx* ctx = st->ctx;
    if (obs->nterms > 4096) fail(QSE_ERR_SIZE, "observable has too many terms");
    const uint64_t size = st->size();
    const unsigned grid = unsigned(std::min<uint64_t>((size + kRB - 1) / kRB, uint64_t(ctx->num_sms) * 8));
    size_t obytes = align16(16 * obs->nterms);
    ctx->scratch.reserve(obytes + size_t(grid) * 8 + 16);
    ctx->host_small.reserve(obytes + size_t(grid) * 8 + 16);
    QSE_CUDA(cudaStreamSynchronize(ctx->stream));  // host_small may still feed an earlier copy
    char* d = static_cast<char*>(ctx->scratch.ptr);
    char* h = static_cast<char*>(ctx->host_small.ptr);
    ObsDev o = upload_obs(st, obs, d, h);
    double* partial = reinterpret_cast<double*>(d + obytes);
    k_obs<<<grid, kRB, 16 * obs->nterms, ctx->stream>>>(reinterpret_cast<const double2*>(st->amp), lam, size, o.z, o.w,
                                                        o.nt, o.c, partial);
    QSE_CUDA(cudaGetLastError());
    count_launch(ctx);
    double* hp = reinterpret_cast<double*>(h + obytes);
    QSE_CUDA(cudaMemcpyAsync(hp, partial, size_t(grid) * 8, cudaMemcpyDeviceToHost, ctx->stream));
    QSE_CUDA(cudaStreamSynchronize(ctx->stream));
    double acc = 0.0;
    for (unsigned b = 0; b < grid; ++b) acc += hp[b];
    return acc;
}

plan::Gate inverse_gate(const qse_op& op, double theta, int32_t grad)
{
    plan::Gate g = to_gate(op, theta);
    switch (op.type) {
    case QSE_GATE_PHASE: case QSE_GATE_RX: case QSE_GATE_RY: case QSE_GATE_RZ:
    case QSE_GATE_CPHASE: case QSE_GATE_MCPHASE:
        g.theta = -theta;
        break;
    case QSE_GATE_2X2:
        g.m[0] = op.m[0]; g.m[1] = -op.m[1];
        g.m[2] = op.m[4]; g.m[3] = -op.m[5];
        g.m[4] = op.m[2]; g.m[5] = -op.m[3];
        g.m[6] = op.m[6]; g.m[7] = -op.m[7];
        break;
    default: break;
    }
    g.grad = grad;
    return g;
}

bool parameterised(int type)
{
    return type == QSE_GATE_RX || type == QSE_GATE_RY || type == QSE_GATE_RZ || type == QSE_GATE_PHASE ||
           type == QSE_GATE_CPHASE || type == QSE_GATE_MCPHASE;
}

}  // namespace

double expectation(qse_state* st, const qse_observable* obs) { return run_obs(st, obs, nullptr); }

double adjoint(qse_state* st, const qse_op* ops, size_t nops, const double* params, size_t nparams,
               const qse_observable* obs, double* grad)
{
    qse_ctx* ctx = st->ctx;
    if (st->n < 3) fail(QSE_ERR_SIZE, "adjoint needs at least 3 qubits");
    // forward from |0..0> (recorded: the first pass generates it)
    mark_zero(st);
    execute_program(st, ops, nops, params, nparams, nullptr, nullptr, 0, nullptr);
    if (!st->aux) QSE_CUDA(cudaMalloc(&st->aux, st->size() * 16));
    double value = run_obs(st, obs, reinterpret_cast<double2*>(st->aux));

    // reverse sweep over the inverse gates, gradient slots on parameterised ones.
    // Slot sums give 2 Im<l|G|s> for X/Y/Z generators and -2 Im<l|P|s> must be
    // applied for phase types (factor f); occurrences of one parameter with the
    // same coeff * f add into one bucket, reduced once per pass
    std::vector<plan::Gate> rev;
    rev.reserve(nops);
    std::map<std::pair<int32_t, double>, int32_t> bucket_of;
    std::vector<std::pair<int32_t, double>> buckets;
    // bucket of an occurrence of `param` whose angle moves by dtheta per unit
    // of the parameter, on a gate of the given type
    auto bucket = [&](int type, int32_t param, double dtheta) {
        const double f = (type == QSE_GATE_PHASE || type == QSE_GATE_CPHASE || type == QSE_GATE_MCPHASE) ? -2.0 : 1.0;
        const std::pair<int32_t, double> key{param, dtheta * f};
        auto it = bucket_of.find(key);
        if (it == bucket_of.end()) {
            it = bucket_of.emplace(key, int32_t(buckets.size())).first;
            buckets.push_back(key);
        }
        return it->second;
    };
    for (size_t i = nops; i-- > 0;) {
        // CNOT(c,t) RZ(th,t) CNOT(c,t) = exp(-i th/2 Z_c Z_t) = RZ(th,c) PHASE(th,t)
        // CPHASE(-2th,c,t), exactly (global phase included): the reverse sweep
        // undoes the three commuting phase gates, each an occurrence of the
        // RZ's parameter (angle derivatives coeff, coeff, -2 coeff), instead of
        // two CNOTs that each need their target in registers
        if (i >= 2 && ops[i].type == QSE_GATE_CNOT && ops[i - 1].type == QSE_GATE_RZ &&
            ops[i - 2].type == QSE_GATE_CNOT && ops[i].control == ops[i - 2].control &&
            ops[i].target == ops[i - 2].target && ops[i - 1].target == ops[i].target &&
            ops[i].control != ops[i].target) {
            const qse_op& rz = ops[i - 1];
            const double th = bound_angle(rz, params, nparams);
            const bool p = rz.param >= 0;
            qse_op a = rz;
            a.target = ops[i].control;
            qse_op b = rz;
            b.type = QSE_GATE_PHASE;
            qse_op c = rz;
            c.type = QSE_GATE_CPHASE;
            c.control = ops[i].control;
            rev.push_back(inverse_gate(a, th, p ? bucket(QSE_GATE_RZ, rz.param, rz.coeff) : -1));
            rev.push_back(inverse_gate(b, th, p ? bucket(QSE_GATE_PHASE, rz.param, rz.coeff) : -1));
            rev.push_back(inverse_gate(c, -2.0 * th, p ? bucket(QSE_GATE_CPHASE, rz.param, -2.0 * rz.coeff) : -1));
            i -= 2;
            continue;
        }
        double th = bound_angle(ops[i], params, nparams);
        int32_t gid = -1;
        if (ops[i].param >= 0 && parameterised(ops[i].type)) gid = bucket(ops[i].type, ops[i].param, ops[i].coeff);
        rev.push_back(inverse_gate(ops[i], th, gid));
    }
    plan::Options opt;
    opt.rb = 3;
    opt.k = tile_qubits_for(ctx, st->n, 3, 11);
    opt.grads = true;
    opt.max_terms = 512;
    opt.max_gates = plan::kJitMaxGates;
    const std::shared_ptr<PlanEntry> e = plan_for(st, rev, opt, 2);
    const plan::Plan& pl = e->pl;
    Uploaded up = upload_plan(ctx, pl, e->use_jit && st->n >= jit::kPreGroupQubits);

    // occurrence gradients accumulate in scratch2: [nops] | slot partials
    size_t max_part = 0;
    for (size_t i = 0; i < pl.passes.size(); ++i)
        max_part = std::max(max_part, pl.passes[i].slot_src.size() * (size_t(1) << (st->n - pl.passes[i].k)));
    size_t srcmax = 0;
    for (auto& p : pl.passes) srcmax = std::max(srcmax, p.slot_src.size());
    size_t b_occ = align16(nops * 8 + 8), b_part = align16(max_part * 8 + 8), b_src = align16(srcmax * 4 + 4);
    ctx->scratch2.reserve(b_occ + b_part + b_src * pl.passes.size() + 16);
    char* base = static_cast<char*>(ctx->scratch2.ptr);
    double* occ = reinterpret_cast<double*>(base);
    double* part = reinterpret_cast<double*>(base + b_occ);
    char* srcbase = base + b_occ + b_part;
    QSE_CUDA(cudaMemsetAsync(occ, 0, nops * 8 + 8, ctx->stream));
    // slot -> occurrence maps, one upload
    {
        size_t hb = b_src * pl.passes.size() + 16;
        ctx->host_small2.reserve(hb);
        char* h = static_cast<char*>(ctx->host_small2.ptr);
        for (size_t i = 0; i < pl.passes.size(); ++i)
            std::memcpy(h + i * b_src, pl.passes[i].slot_src.data(), pl.passes[i].slot_src.size() * 4);
        QSE_CUDA(cudaMemcpyAsync(srcbase, h, b_src * pl.passes.size(), cudaMemcpyHostToDevice, ctx->stream));
    }
    PassRunner runner(st, *e, up, 2, 3);
    for (size_t i = 0; i < up.args.size(); ++i) {
        const tile::PassArgs& a = up.args[i];
        runner.run(i, reinterpret_cast<double2*>(st->aux), part);
        if (a.nslots) {
            uint64_t nb = uint64_t(1) << (st->n - a.k);
            unsigned g = std::min<unsigned>(a.nslots, unsigned(ctx->num_sms) * 4);
            k_reduce_slots<<<g, kRB, 0, ctx->stream>>>(part, a.nslots, nb,
                                                        reinterpret_cast<const int32_t*>(srcbase + i * b_src), occ);
            QSE_CUDA(cudaGetLastError());
            count_launch(ctx);
        }
    }
    for (uint32_t q = 0; q < st->n; ++q) st->perm[q] = pl.perm_final[q];
    st->touch();
    std::vector<double> hocc(nops);
    QSE_CUDA(cudaMemcpyAsync(hocc.data(), occ, nops * 8, cudaMemcpyDeviceToHost, ctx->stream));
    QSE_CUDA(cudaStreamSynchronize(ctx->stream));
    for (size_t p = 0; p < nparams; ++p) grad[p] = 0.0;
    for (size_t b = 0; b < buckets.size(); ++b)
        if (size_t(buckets[b].first) < nparams) grad[buckets[b].first] += buckets[b].second * hocc[b];
    return value;
}

}  // namespace qse
