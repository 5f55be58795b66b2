// planner.cpp -- gate-fusion planner and tile-program lowering.  Host only.
//
// Semantics preserved: gates are replayed as Circuit::execute does
// (Circuit.cpp:64-120), in program order, except that a gate may run before
// an earlier gate it commutes with.  Two gates commute here when, on every
// qubit they share, both act diagonally (Z/PHASE/RZ/CPHASE/MCPHASE, and the
// control of a CNOT).  SWAP (Circuit.cpp:59-62, applySwap) is a relabelling of
// the logical->physical qubit map, applied with zero memory traffic.
#include "planner.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <set>
#include <sstream>
#include <tuple>

#include "qse_internal.h"

namespace qse {
namespace plan {
namespace {

constexpr double kInvSqrt2 = 0.7071067811865475244;  // CircuitUnitaryOperation.cpp:87
// smallest pending scale (unscaled Hadamards, deferred pass constants) before it
// is applied: stored values stay below 2^200 times the state's own, and a pass
// adds at most another 2^200, far from the 2^1024 overflow
constexpr double kFlushScale = 0x1p-200;

enum Cls { C_DROP, C_N1, C_CX, C_DIAG, C_SWAP };

struct Info {
    Cls cls = C_DROP;
    uint64_t nset = 0;  // logical qubits acted on non-diagonally
    uint64_t dset = 0;  // logical qubits acted on diagonally (incl. controls)
};

inline uint64_t bit(uint32_t q) { return uint64_t(1) << q; }

Info classify(const Gate& g, uint32_t n)
{
    auto chk = [&](uint32_t q) {
        if (q >= n) fail(QSE_ERR_QUBIT, "qubit index " + std::to_string(q) + " out of range for " +
                                            std::to_string(n) + " qubits");
    };
    Info r;
    switch (g.type) {
    case QSE_GATE_IDENTITY: return r;
    case QSE_GATE_H: case QSE_GATE_X: case QSE_GATE_Y: case QSE_GATE_RX: case QSE_GATE_RY: case QSE_GATE_2X2:
        chk(g.t);
        r.cls = C_N1;
        r.nset = bit(g.t);
        return r;
    case QSE_GATE_CNOT:
        chk(g.t);
        chk(g.c);
        // control == target: the reference's condition (i & c) && (i < (i ^ t)) is never true
        // (CircuitUnitaryOperation.cpp:47-51): a no-op.
        if (g.c == g.t) return r;
        r.cls = C_CX;
        r.nset = bit(g.t);
        r.dset = bit(g.c);
        return r;
    case QSE_GATE_Z: case QSE_GATE_PHASE: case QSE_GATE_RZ:
        chk(g.t);
        r.cls = C_DIAG;
        r.dset = bit(g.t);
        return r;
    case QSE_GATE_CPHASE:
        chk(g.t);
        chk(g.c);
        r.cls = C_DIAG;
        r.dset = bit(g.t) | bit(g.c);
        return r;
    case QSE_GATE_MCPHASE:
        chk(g.t);
        if (n < 64 && (g.cmask >> n) != 0) fail(QSE_ERR_QUBIT, "mcphase control out of range");
        r.cls = C_DIAG;
        r.dset = bit(g.t) | g.cmask;
        return r;
    case QSE_GATE_SWAP:
        chk(g.t);
        chk(g.c);
        if (g.t == g.c) return r;  // applySwap with q0 == q1 is a no-op (CircuitUnitaryOperationGPU.cu:338)
        r.cls = C_SWAP;
        r.nset = bit(g.t) | bit(g.c);
        return r;
    default:
        fail(QSE_ERR_UNSUPPORTED, "gate type " + std::to_string(g.type) + " is not executable");
    }
}

int popc(uint64_t x) { return __builtin_popcountll(x); }

// One absorbed gate with its physical qubits resolved.
struct Absorbed {
    size_t src;
    const Gate* g;
    Cls cls;
    uint32_t pt;     // physical target
    uint32_t pc;     // physical control (CNOT)
    uint64_t psup;   // physical support (diagonal)
};

// ---------- lowering of one pass ----------
class Lowering {
public:
    Lowering(PassProgram& prog, uint32_t n, const Options& opt) : P(prog), n_(n), opt_(opt)
    {
        for (int i = 0; i < 64; ++i) loc_[i] = -1;
        for (uint32_t b = 0; b < P.k; ++b) loc_[P.tile_phys[b]] = int(b);
    }

    // Gates of the pass are emitted in a topological order of their
    // dependency graph (b depends on an earlier a when they share a qubit on
    // which either acts non-diagonally; SWAPs are already folded into the
    // physical qubits).  Ready diagonal gates go first; then ready gates on
    // the current register bits; only when none is left does the pass change
    // register layout, to the bits with the most ready gates.  For the QFT
    // this halves the layouts of program order (one per block of register bits).
    // carry: constant factor deferred by the previous passes of the plan
    // (the unscaled Hadamards' 1/sqrt2 and RZ's global phase); the pass
    // applies carry times its own factor when it is the last pass (apply),
    // else it applies nothing and returns the product for the next pass
    std::pair<double, double> run(const std::vector<Absorbed>& abs, double gphase, std::pair<double, double> carry,
                                  bool apply)
    {
        const int m = int(abs.size());
        std::vector<std::vector<int>> succ(m);
        std::vector<int> indeg(m, 0);
        {
            std::vector<int> last_n(64, -1);
            std::vector<std::vector<int>> dl(64);
            auto edge = [&](int a, int b) {
                succ[a].push_back(b);
                ++indeg[b];
            };
            for (int i = 0; i < m; ++i) {
                const Absorbed& a = abs[i];
                if (a.cls == C_SWAP) continue;
                uint64_t nq = 0, dq = 0;
                if (a.cls == C_N1) nq = bit(a.pt);
                else if (a.cls == C_CX) { nq = bit(a.pt); dq = bit(a.pc); }
                else dq = a.psup;
                for (uint64_t s = nq; s; s &= s - 1) {
                    int q = __builtin_ctzll(s);
                    if (last_n[q] >= 0) edge(last_n[q], i);
                    for (int d : dl[q]) edge(d, i);
                    last_n[q] = i;
                    dl[q].clear();
                }
                for (uint64_t s = dq; s; s &= s - 1) {
                    int q = __builtin_ctzll(s);
                    if (last_n[q] >= 0) edge(last_n[q], i);
                    dl[q].push_back(i);
                }
            }
        }
        std::set<int> ready_d, ready_n;
        auto make_ready = [&](int i) {
            if (abs[i].cls == C_DIAG) ready_d.insert(i);
            else ready_n.insert(i);
        };
        int total = 0;
        for (int i = 0; i < m; ++i) {
            if (abs[i].cls == C_SWAP) continue;
            ++total;
            if (indeg[i] == 0) make_ready(i);
        }
        auto release = [&](int i) {
            for (int s : succ[i])
                if (--indeg[s] == 0) make_ready(s);
        };
        // register bits for a new layout: most ready gates, then most gates in the lookahead, then earliest
        auto pick_regs = [&](const int* prev) {
            std::vector<long long> score(P.k, 0);
            std::vector<int> first(P.k, 1 << 30);
            for (int i : ready_n) {
                int b = loc_[abs[i].pt];
                score[b] += 1000000;
                first[b] = std::min(first[b], i);
            }
            int seen = 0;
            for (int i = 0; i < m && seen < 64; ++i) {
                if (abs[i].cls != C_N1 && abs[i].cls != C_CX) continue;
                if (indeg[i] < 0) continue;  // already emitted
                int b = loc_[abs[i].pt];
                score[b] += 64 - seen;
                first[b] = std::min(first[b], i);
                ++seen;
            }
            std::vector<int> bits(P.k);
            for (uint32_t b = 0; b < P.k; ++b) bits[b] = int(b);
            std::stable_sort(bits.begin(), bits.end(), [&](int x, int y) {
                if (score[x] != score[y]) return score[x] > score[y];
                bool px = false, py = false;
                if (prev)
                    for (uint32_t r = 0; r < P.rb; ++r) { px |= prev[r] == x; py |= prev[r] == y; }
                if (px != py) return px;
                return first[x] < first[y];
            });
            std::vector<int> r(bits.begin(), bits.begin() + P.rb);
            std::sort(r.begin(), r.end());
            for (uint32_t i = 0; i < P.rb; ++i) reg_[i] = r[i];
            nthr_ = 0;
            for (uint32_t b = 0; b < P.k; ++b)
                if (reg_pos(int(b)) < 0) thr_[nthr_++] = int(b);
        };
        pick_regs(nullptr);
        P.layout0 = add_layout(nullptr);
        scale_ = 1.0;
        P.order.clear();
        P.phys_target.clear();
        for (int i = 0; i < m; ++i)
            if (abs[i].cls == C_SWAP) {
                P.order.push_back(uint32_t(abs[i].src));
                P.phys_target.push_back(0);
                P.phys_control.push_back(0);
                P.phys_support.push_back(0);
            }
        int emitted = 0;
        while (emitted < total) {
            int pick = -1;
            if (!ready_d.empty()) {
                pick = *ready_d.begin();
                ready_d.erase(ready_d.begin());
            } else {
                for (int i : ready_n)
                    if (reg_pos(loc_[abs[i].pt]) >= 0) { pick = i; break; }
                if (pick < 0) {
                    if (ready_n.empty()) fail(QSE_ERR_INVALID, "internal: pass schedule stalled");
                    close_all(false, 1.0, 0.0);
                    std::vector<int> prev(reg_, reg_ + P.rb);
                    pick_regs(prev.data());
                    KOp t{};
                    t.kind = K_TRANSPOSE;
                    t.g = uint16_t(add_layout(prev.data()));
                    P.ops.push_back(t);
                    continue;
                }
                ready_n.erase(pick);
            }
            indeg[pick] = -1;
            ++emitted;
            release(pick);
            const Absorbed& a = abs[pick];
            P.order.push_back(uint32_t(a.src));
            P.phys_target.push_back(a.pt);
            P.phys_control.push_back(a.pc);
            P.phys_support.push_back(a.psup);
            const Gate& g = *a.g;
            if (a.cls == C_DIAG) {
                if (opt_.grads && g.grad >= 0) emit_grad_diag(a);
                add_diag_terms(a, gphase);
                continue;
            }
            const int p = reg_pos(loc_[a.pt]);
            close_reg(p);
            if (opt_.grads && g.grad >= 0) emit_grad_pair(a, p);
            KOp op{};
            op.p = uint8_t(p);
            if (a.cls == C_CX) {
                op.kind = K_X;
                set_control(op, a.pc);
            } else {
                switch (g.type) {
                case QSE_GATE_H: op.kind = K_H; scale_ *= kInvSqrt2; break;
                case QSE_GATE_X: op.kind = K_X; break;
                case QSE_GATE_Y: op.kind = K_Y; break;
                case QSE_GATE_RX: case QSE_GATE_RY:
                    op.kind = g.type == QSE_GATE_RX ? K_RX : K_RY;
                    op.a = std::cos(g.theta / 2.0);
                    op.b = std::sin(g.theta / 2.0);
                    P.op_angles.push_back(AngleRef{uint32_t(P.ops.size()), uint32_t(a.src)});
                    break;
                case QSE_GATE_2X2:
                    op.kind = K_U;
                    op.g = uint16_t(P.mats.size() / 8);
                    P.mats.insert(P.mats.end(), g.m, g.m + 8);
                    break;
                default: fail(QSE_ERR_UNSUPPORTED, "internal: unexpected non-diagonal type");
                }
            }
            P.ops.push_back(op);
            P.n_nondiag++;
            // each unscaled Hadamard grows the stored values by sqrt2: apply the
            // pending 1/sqrt2 factors before they fall below kFlushScale
            if (scale_ < kFlushScale) {
                close_all(true, scale_, 0.0);
                scale_ = 1.0;
            }
        }
        const double ga = opt_.keep_gphase ? scale_ * std::cos(gphase_) : scale_;
        const double gb = opt_.keep_gphase ? scale_ * std::sin(gphase_) : 0.0;
        const std::pair<double, double> c{carry.first * ga - carry.second * gb, carry.first * gb + carry.second * ga};
        // the deferred constant stays above kFlushScale in magnitude, so the
        // stored amplitudes stay below 1 / kFlushScale times their true size
        if (apply || std::hypot(c.first, c.second) < kFlushScale) {
            close_all(true, c.first, c.second);
            return {1.0, 0.0};
        }
        close_all(true, 1.0, 0.0);
        return c;
    }

private:
    PassProgram& P;
    uint32_t n_;
    const Options& opt_;
    int loc_[64];
    int reg_[5] = {0, 0, 0, 0, 0};
    int thr_[16];
    int nthr_ = 0;
    double gphase_ = 0.0;
    double scale_ = 1.0;   // product of the 1/sqrt2 factors of the unscaled K_H applied so far

    struct OG {
        uint8_t kind, p, f;
        uint16_t tcond;
        std::vector<TermRec> terms;
        std::vector<int32_t> src;   // source gate of each term (-1: constant angle)
    };
    std::map<std::tuple<int, int, int>, OG> open_;

    int reg_pos(int tb) const
    {
        for (uint32_t i = 0; i < P.rb; ++i)
            if (reg_[i] == tb) return int(i);
        return -1;
    }
    int thr_pos(int tb) const
    {
        for (int i = 0; i < nthr_; ++i)
            if (thr_[i] == tb) return i;
        return -1;
    }

    // Slot images for the shared-memory exchange from layout `prev` to the
    // current one: L(e_b) = e_b ^ s_b (s_b in the low 3 bits, b >= 3), chosen so
    // that the 8 lanes of each quarter-warp hit 8 distinct 16-byte bank groups
    // both when writing (prev layout) and reading (new layout).
    uint32_t add_layout(const int* prev)
    {
        LayoutRec rec{};
        for (uint32_t i = 0; i < P.rb; ++i) rec.reg[i] = uint8_t(reg_[i]);
        rec.nthr = uint8_t(nthr_);
        for (int t = 0; t < nthr_; ++t) rec.thr[t] = uint8_t(thr_[t]);
        uint32_t s[16] = {0};
        if (prev && nthr_ >= 3) {
            int pl[3], nl[3], np = 0;
            for (uint32_t b = 0; b < P.k && np < 3; ++b) {
                bool in_prev = false;
                for (uint32_t i = 0; i < P.rb; ++i) in_prev |= prev[i] == int(b);
                if (!in_prev) pl[np++] = int(b);
            }
            for (int i = 0; i < 3; ++i) nl[i] = thr_[i];
            auto low3 = [&](int b, const uint32_t* sv) -> uint32_t { return b < 3 ? (1u << b) : sv[b]; };
            auto rank_ok = [&](const int* lb, const uint32_t* sv) {
                uint32_t v0 = low3(lb[0], sv), v1 = low3(lb[1], sv), v2 = low3(lb[2], sv);
                if (!v0 || !v1 || !v2 || v0 == v1 || v0 == v2 || v1 == v2) return false;
                return (v0 ^ v1) != v2;
            };
            uint64_t rng = 0x9E3779B97F4A7C15ull ^ (uint64_t(P.layouts.size()) * 0xBF58476D1CE4E5B9ull);
            bool found = false;
            for (int attempt = 0; attempt < 4096 && !found; ++attempt) {
                uint32_t sv[16] = {0};
                if (attempt > 0)
                    for (uint32_t b = 3; b < P.k; ++b) {
                        rng ^= rng << 13; rng ^= rng >> 7; rng ^= rng << 17;
                        sv[b] = uint32_t(rng >> 61);
                    }
                if (rank_ok(pl, sv) && rank_ok(nl, sv)) {
                    std::copy(sv, sv + 16, s);
                    found = true;
                }
            }
        }
        for (uint32_t b = 0; b < 16; ++b) rec.L[b] = uint16_t((1u << b) ^ (b >= 3 ? s[b] : 0u));
        P.layouts.push_back(rec);
        return uint32_t(P.layouts.size() - 1);
    }

    void set_control(KOp& op, uint32_t pc)
    {
        int tb = loc_[pc];
        if (tb < 0) {
            op.ocond = bit(pc);
            return;
        }
        int rp = reg_pos(tb);
        if (rp >= 0) {
            op.f = uint8_t(1u << rp);
            return;
        }
        op.tcond = uint16_t(1u << thr_pos(tb));
    }

    // split a physical support into (register mask, thread mask, outer mask)
    void split(uint64_t sup, uint8_t& f, uint16_t& tcond, uint64_t& ocond) const
    {
        f = 0;
        tcond = 0;
        ocond = 0;
        for (uint64_t s = sup; s; s &= s - 1) {
            uint32_t q = uint32_t(__builtin_ctzll(s));
            int tb = loc_[q];
            if (tb < 0) { ocond |= bit(q); continue; }
            int rp = reg_pos(tb);
            if (rp >= 0) f |= uint8_t(1u << rp);
            else tcond |= uint16_t(1u << thr_pos(tb));
        }
    }

    void add_term(uint64_t sup, double theta, int32_t src)
    {
        if (sup == 0) { gphase_ += theta; return; }
        uint8_t f;
        uint16_t tc;
        uint64_t oc;
        split(sup, f, tc, oc);
        int nreg = popc(f);
        // direct_phases: terms on register bits whose angle does not depend on
        // the thread (no thread condition) are direct, their group's sum turned
        // into (cos, sin) once per CTA; otherwise single-bit terms accumulate
        // angles per thread, one sincos per flush.
        const bool direct1 = opt_.direct_phases && tc == 0;
        int kind = nreg == 0 ? K_ACC_THR : ((nreg == 1 && !direct1) ? K_ACC_REG : K_PHD);
        int key2 = kind == K_ACC_REG ? __builtin_ctz(f) : (kind == K_PHD ? f : 0);
        auto key = std::make_tuple(kind, key2, int(tc));
        auto it = open_.find(key);
        if (it == open_.end()) {
            OG og{uint8_t(kind), uint8_t(kind == K_ACC_REG ? __builtin_ctz(f) : 0), f, tc, {}, {}};
            it = open_.emplace(key, std::move(og)).first;
        }
        it->second.terms.push_back(TermRec{oc, theta});
        it->second.src.push_back(src);
    }

    void add_diag_terms(const Absorbed& a, double& /*unused*/)
    {
        const Gate& g = *a.g;
        switch (g.type) {
        case QSE_GATE_Z: add_term(a.psup, M_PI, -1); break;
        case QSE_GATE_PHASE: case QSE_GATE_CPHASE: case QSE_GATE_MCPHASE: add_term(a.psup, g.theta, int32_t(a.src)); break;
        case QSE_GATE_RZ:  // diag(e^{-it/2}, e^{it/2}) = e^{-it/2} diag(1, e^{it})
            add_term(a.psup, g.theta, int32_t(a.src));
            gphase_ += -g.theta / 2.0;
            break;
        default: fail(QSE_ERR_UNSUPPORTED, "internal: unexpected diagonal type");
        }
    }

    uint16_t emit_group(OG& og)
    {
        GroupRec gr{};
        gr.first = uint32_t(P.terms.size());
        gr.count = uint32_t(og.terms.size());
        gr.direct = (og.kind == K_PHD || opt_.acc_mul) ? 1u : 0u;
        for (size_t i = 0; i < og.src.size(); ++i)
            if (og.src[i] >= 0) P.term_angles.push_back(AngleRef{uint32_t(P.terms.size() + i), uint32_t(og.src[i])});
        P.terms.insert(P.terms.end(), og.terms.begin(), og.terms.end());
        P.groups.push_back(gr);
        return uint16_t(P.groups.size() - 1);
    }

    void close_reg(int p)
    {
        bool acc = false;
        for (auto it = open_.begin(); it != open_.end();) {
            OG& og = it->second;
            bool hit = (og.kind == K_ACC_REG && og.p == p) || (og.kind == K_PHD && ((og.f >> p) & 1));
            if (!hit) { ++it; continue; }
            KOp op{};
            op.kind = og.kind;
            op.p = og.p;
            op.f = og.f;
            op.tcond = og.tcond;
            op.g = emit_group(og);
            P.ops.push_back(op);
            acc |= og.kind == K_ACC_REG;
            it = open_.erase(it);
        }
        if (acc) {
            KOp fl{};
            fl.kind = K_FLUSH_REG;
            fl.p = uint8_t(p);
            P.ops.push_back(fl);
        }
    }

    void close_all(bool final, double ca, double cb)
    {
        uint8_t fmask = 0;
        bool thr = false;
        for (auto& kv : open_) {
            OG& og = kv.second;
            KOp op{};
            op.kind = og.kind;
            op.p = og.p;
            op.f = og.f;
            op.tcond = og.tcond;
            op.g = emit_group(og);
            P.ops.push_back(op);
            if (og.kind == K_ACC_REG) fmask |= uint8_t(1u << og.p);
            if (og.kind == K_ACC_THR) thr = true;
        }
        open_.clear();
        if (final || fmask || thr) {
            KOp fl{};
            fl.kind = K_FLUSH_ALL;
            fl.f = fmask;
            fl.a = final ? ca : 1.0;
            fl.b = final ? cb : 0.0;
            P.ops.push_back(fl);
        }
    }

    // one slot per gradient source within a pass: occurrences that share a
    // source (the adjoint gives occurrences of one parameter with one factor the
    // same source) add into one slot
    uint16_t new_slot(int32_t src)
    {
        for (size_t s = 0; s < P.slot_src.size(); ++s)
            if (P.slot_src[s] == src) return uint16_t(s);
        P.slot_src.push_back(src);
        return uint16_t(P.slot_src.size() - 1);
    }

    void emit_grad_pair(const Absorbed& a, int p)
    {
        const Gate& g = *a.g;
        KOp op{};
        op.p = uint8_t(p);
        if (g.type == QSE_GATE_RX) op.kind = K_GRAD_X;
        else if (g.type == QSE_GATE_RY) op.kind = K_GRAD_Y;
        else return;
        op.g = new_slot(g.grad);
        op.a = scale_ * scale_;   // both states still lack the pass's pending H scale
        P.ops.push_back(op);
    }

    void emit_grad_diag(const Absorbed& a)
    {
        const Gate& g = *a.g;
        KOp op{};
        if (g.type == QSE_GATE_RZ) {
            op.kind = K_GRAD_Z;
            uint8_t f;
            split(a.psup, f, op.tcond, op.ocond);
            op.p = f ? uint8_t(__builtin_ctz(f)) : uint8_t(255);
        } else if (g.type == QSE_GATE_PHASE || g.type == QSE_GATE_CPHASE || g.type == QSE_GATE_MCPHASE) {
            op.kind = K_GRAD_P;
            split(a.psup, op.f, op.tcond, op.ocond);
        } else {
            return;
        }
        op.g = new_slot(g.grad);
        op.a = scale_ * scale_;   // both states still lack the pass's pending H scale
        P.ops.push_back(op);
    }
};

}  // namespace

// CNOT(c,t) RZ(th,t) CNOT(c,t) multiplies |c t> by e^{-i th/2} e^{i th (c XOR t)}, and
// c XOR t = c + t - 2ct: the diagonal RZ(th,c) PHASE(th,t) CPHASE(-2th,c,t), global
// phase included.  QAOA cost layers written with CNOTs (QSEplayground/QAOA.cpp:128-133)
// then need no pass of their own.  Returns false when nothing matched.
bool fuse_zz(const std::vector<Gate>& gates, std::vector<Gate>& out)
{
    bool any = false;
    for (size_t i = 0; i + 2 < gates.size(); ++i) {
        const Gate& a = gates[i];
        const Gate& b = gates[i + 1];
        const Gate& c = gates[i + 2];
        if (a.type != QSE_GATE_CNOT || b.type != QSE_GATE_RZ || c.type != QSE_GATE_CNOT) continue;
        if (a.c != c.c || a.t != c.t || b.t != a.t || a.c == a.t) continue;
        if (a.grad >= 0 || b.grad >= 0 || c.grad >= 0) continue;
        if (!any) out = gates;
        any = true;
        Gate rz = b;
        rz.t = a.c;
        Gate ph{};
        ph.type = QSE_GATE_PHASE;
        ph.t = a.t;
        ph.theta = b.theta;
        Gate cp{};
        cp.type = QSE_GATE_CPHASE;
        cp.t = a.t;
        cp.c = a.c;
        cp.theta = -2.0 * b.theta;
        out[i] = rz;
        out[i + 1] = ph;
        out[i + 2] = cp;
        i += 2;
    }
    return any;
}

Plan build(const std::vector<Gate>& gates_in, uint32_t n, const uint32_t* perm_in, const Options& opt)
{
    if (n == 0 || n > 40) fail(QSE_ERR_SIZE, "planner: unsupported qubit count");
    std::vector<Gate> fused;
    const std::vector<Gate>& gates = (opt.zz_fuse && fuse_zz(gates_in, fused)) ? fused : gates_in;
    Plan plan;
    uint32_t perm[64];
    for (uint32_t q = 0; q < 64; ++q) perm[q] = q < n ? perm_in[q] : q;
    std::vector<Info> info(gates.size());
    std::vector<size_t> remaining;
    for (size_t i = 0; i < gates.size(); ++i) {
        info[i] = classify(gates[i], n);
        if (info[i].cls != C_DROP) remaining.push_back(i);
    }
    plan.gates = gates.size();
    const uint32_t k = std::min<uint32_t>(opt.k, n);
    const uint32_t seed_bits = std::min<uint32_t>(3, k);
    // forward plans defer every pass's constant factor to the last pass (no
    // caller reads the state between the passes of one plan); gradient plans
    // scale each pass, their K_GRAD_* weights assume it
    std::pair<double, double> carry{1.0, 0.0};

    // remaining[head..) are the gates still to plan, in order
    size_t head = 0;
    while (head < remaining.size()) {
        uint64_t T = 0;
        for (uint32_t q = 0; q < seed_bits; ++q) T |= bit(q);
        uint64_t bN = 0, bD = 0;
        std::vector<Absorbed> abs;
        std::vector<size_t> deferred;
        uint32_t nN = 0, nterms = 0, nslots = 0;
        double gph = 0.0;
        const uint64_t allq = n >= 64 ? ~uint64_t(0) : (bit(n) - 1);
        size_t stop = remaining.size();   // first gate this pass did not look at
        for (size_t r = head; r < remaining.size(); ++r) {
            const size_t idx = remaining[r];
            const Info& in = info[idx];
            const Gate& g = gates[idx];
            bool blocked = ((in.nset | in.dset) & bN) || (in.nset & bD);
            const bool slot = opt.grads && g.grad >= 0 && in.cls != C_SWAP;
            if (slot && opt.max_slots && nslots >= opt.max_slots) blocked = true;
            if (!blocked) {
                if (in.cls == C_SWAP) {
                    std::swap(perm[g.t], perm[g.c]);
                    abs.push_back(Absorbed{idx, &g, C_SWAP, 0, 0, 0});
                    continue;
                }
                if (in.cls == C_DIAG) {
                    if (nterms < opt.max_terms) {
                        uint64_t ps = 0;
                        for (uint64_t s = in.dset; s; s &= s - 1) ps |= bit(perm[__builtin_ctzll(s)]);
                        abs.push_back(Absorbed{idx, &g, C_DIAG, perm[g.t],
                                               g.type == QSE_GATE_CPHASE ? perm[g.c] : 0u, ps});
                        ++nterms;
                        nslots += slot ? 1 : 0;
                        continue;
                    }
                } else {
                    uint64_t pt = bit(perm[g.t]);
                    bool fits = (T & pt) || uint32_t(popc(T)) < k;
                    bool capped = opt.max_gates && nN >= opt.max_gates;
                    if (fits && !capped) {
                        T |= pt;
                        abs.push_back(Absorbed{idx, &g, in.cls, perm[g.t], in.cls == C_CX ? perm[g.c] : 0, 0});
                        ++nN;
                        nslots += slot ? 1 : 0;
                        continue;
                    }
                }
            }
            deferred.push_back(idx);
            bN |= in.nset;
            bD |= in.dset;
            if ((bN & allq) == allq) {
                // every later gate shares a qubit with a deferred non-diagonal one:
                // none can join this pass (keeps planning linear in the gate count)
                stop = r + 1;
                break;
            }
        }
        // fill the tile with the lowest unused physical qubits
        for (uint32_t q = 0; q < n && uint32_t(popc(T)) < k; ++q) T |= bit(q);
        PassProgram prog;
        prog.k = k;
        prog.rb = opt.rb;
        prog.acc_mul = opt.acc_mul;
        uint32_t b = 0;
        for (uint32_t q = 0; q < n; ++q)
            if ((T >> q) & 1) prog.tile_phys[b++] = uint8_t(q);
        uint64_t all = n >= 64 ? ~uint64_t(0) : (bit(n) - 1);
        prog.outer_mask = all & ~T;
        prog.ngates = uint32_t(abs.size());
        Lowering low(prog, n, opt);
        const bool last = deferred.empty() && stop == remaining.size();
        carry = low.run(abs, gph, carry, opt.grads || last);
        plan.passes.push_back(std::move(prog));
        // next: this pass's deferred gates, then the ones it did not look at
        // (written in place just before those, no copy of the unscanned rest)
        head = stop - deferred.size();
        std::copy(deferred.begin(), deferred.end(), remaining.begin() + std::ptrdiff_t(head));
    }
    for (uint32_t q = 0; q < 64; ++q) plan.perm_final[q] = perm[q];
    return plan;
}

std::string describe(const Plan& p)
{
    std::ostringstream os;
    os << "{\"passes\":[";
    for (size_t i = 0; i < p.passes.size(); ++i) {
        const PassProgram& pp = p.passes[i];
        if (i) os << ",";
        os << "{\"k\":" << pp.k << ",\"tile\":[";
        for (uint32_t b = 0; b < pp.k; ++b) os << (b ? "," : "") << int(pp.tile_phys[b]);
        os << "],\"ops\":" << pp.ops.size() << ",\"groups\":" << pp.groups.size() << ",\"terms\":" << pp.terms.size()
           << ",\"layouts\":" << pp.layouts.size() << ",\"gates\":" << pp.ngates
           << ",\"nondiag\":" << pp.n_nondiag << ",\"order\":[";
        for (size_t j = 0; j < pp.order.size(); ++j)
            os << (j ? "," : "") << "[" << pp.order[j] << "," << pp.phys_target[j] << "," << pp.phys_control[j]
               << "," << pp.phys_support[j] << "]";
        os << "],\"kinds\":[";
        for (size_t j = 0; j < pp.ops.size(); ++j) os << (j ? "," : "") << int(pp.ops[j].kind);
        os << "]}";
    }
    os << "],\"perm\":[";
    for (uint32_t q = 0; q < 64; ++q) os << (q ? "," : "") << p.perm_final[q];
    os << "]}";
    return os.str();
}

}  // namespace plan
}  // namespace qse
