// jit.cpp -- per-pass kernel specialisation.
//
// The planner lowers a pass into a short program (planner.h: KOp list,
// register layouts, diagonal groups).  Interpreting that program per thread
// costs more instructions than the arithmetic it drives.  Here each pass is
// turned into straight-line CUDA C++ -- register positions, bit masks,
// layouts, index offsets and conditions as compile-time constants; angles,
// matrices and the pass scale as a __grid_constant__ parameter block -- and
// compiled for sm_100a with NVRTC.  Kernels are cached by their source text,
// so a circuit re-executed with new angles (parameter sweeps, gradients)
// reuses them.  NVRTC is loaded with dlopen and the cubin through
// cudaLibraryLoadData, so the library has no link-time dependency on either.
#include "jit.h"

#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvrtc.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string_view>
#include <thread>
#include <unordered_set>

namespace qse {
namespace jit {
namespace {

const char* kPrelude =
#include "jit_prelude.inc"
    ;

// ---- NVRTC entry points (dlopen) ----
struct Nvrtc {
    decltype(&nvrtcCreateProgram) create = nullptr;
    decltype(&nvrtcCompileProgram) compile = nullptr;
    decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
    decltype(&nvrtcGetProgramLog) log = nullptr;
    decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
    decltype(&nvrtcGetCUBIN) cubin = nullptr;
    decltype(&nvrtcDestroyProgram) destroy = nullptr;
    decltype(&nvrtcGetErrorString) err = nullptr;
    bool ok = false;
    std::string why;
};

Nvrtc& nvrtc()
{
    static Nvrtc n;
    static std::once_flag once;
    std::call_once(once, [] {
        const char* names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12",
                               "/usr/local/cuda/lib64/libnvrtc.so"};
        void* h = nullptr;
        for (const char* nm : names)
            if ((h = dlopen(nm, RTLD_NOW | RTLD_LOCAL))) break;
        if (!h) {
            n.why = "libnvrtc.so.12 not found";
            return;
        }
#define QSE_SYM(field, name)                                                  \
    n.field = reinterpret_cast<decltype(n.field)>(dlsym(h, name));            \
    if (!n.field) {                                                           \
        n.why = std::string("missing ") + name;                               \
        return;                                                               \
    }
        QSE_SYM(create, "nvrtcCreateProgram");
        QSE_SYM(compile, "nvrtcCompileProgram");
        QSE_SYM(log_size, "nvrtcGetProgramLogSize");
        QSE_SYM(log, "nvrtcGetProgramLog");
        QSE_SYM(cubin_size, "nvrtcGetCUBINSize");
        QSE_SYM(cubin, "nvrtcGetCUBIN");
        QSE_SYM(destroy, "nvrtcDestroyProgram");
        QSE_SYM(err, "nvrtcGetErrorString");
#undef QSE_SYM
        n.ok = true;
    });
    return n;
}

// ---- code generation ----
struct Gen {
    const plan::PassProgram& P;
    int ns;
    std::ostringstream o;
    std::vector<double> prm;
    uint32_t R, T, NW;
    int reg[5];
    int thr[16];
    int nthr;

    bool zero_in = false;   // generate the basis state |bi> instead of loading (ns == 1)
    int basis_slot = -1;    // prm slot of bi (set per launch)
    // with zero_in: physical qubits whose input comes from a compact state
    // (lam, 2^popcount(umask) amplitudes indexed by those bits in ascending
    // order); the other qubits hold the bits of bi.  0: the plain basis state
    uint64_t umask = 0;
    // with umask: product qubits (their amplitude pairs after the compact
    // state's) and whether any of them sits on a register bit (the pass then
    // builds the registers' factors in shared memory, pfs)
    uint64_t pmask = 0;
    bool preg = false;
    // probability side output (forward passes): logical position of every
    // physical qubit after this pass; empty = none (emit_prob)
    std::vector<uint8_t> lpos;
    bool prob_bsum = false;   // the side output includes the block sums
    // debug mode (QSE_DEBUG_BOUNDS set in the environment when the kernel is
    // generated): every global access of the kernel checks its index against
    // the array's size; one outside records 8 in *status and is skipped
    bool dbg = false;
    std::string nstr() const { return hex(uint64_t(1) << (P.k + uint32_t(__builtin_popcountll(P.outer_mask)))); }
    // index in lam of product qubit q's |0> amplitude, and the size of lam with the product table
    std::string ph_index(uint32_t q) const
    {
        const uint64_t below = uint64_t(__builtin_popcountll(pmask & ((uint64_t(1) << q) - 1)));
        return hex((uint64_t(1) << __builtin_popcountll(umask)) + 2 * below);
    }
    std::string ph_size() const
    {
        return hex((uint64_t(1) << __builtin_popcountll(umask)) + 2 * uint64_t(__builtin_popcountll(pmask)));
    }
    // array[idx] as an operand (a zero amplitude when out of range in debug mode)
    std::string ld(const std::string& arr, const std::string& idx, const std::string& size) const
    {
        if (!dbg) return arr + "[" + idx + "]";
        return "(qse_idx_ok(" + idx + ", " + size + ", status) ? " + arr + "[" + idx + "] : make_double2(0.0, 0.0))";
    }
    // prefix of a statement that writes at idx (skipped when out of range in debug mode)
    std::string guard(const std::string& idx, const std::string& size) const
    {
        return dbg ? "if (qse_idx_ok(" + idx + ", " + size + ", status)) " : std::string();
    }
    // kernel names tell the input kinds apart in profiles
    std::string kernel_name() const
    {
        if (ns == 2) return "qse_pass_adjoint";
        return !zero_in ? "qse_pass" : umask ? "qse_pass_compact_in" : "qse_pass_basis_in";
    }
    bool xb_used = false;   // the exchange buffer holds data some thread may still read
    std::string SYNC = "__syncthreads();";   // barrier of the threads that share xb
    // gradient slots accumulated per thread (slot -> accumulator index)
    static constexpr uint32_t kRegSlots = 4;
    bool qv = false;   // qz holds Im(conj(l) s) of the registers as they are
    std::map<uint16_t, uint32_t> gacc;
    // the per-CTA group values come precomputed from global memory (gvt, one row
    // of ng values per tile): the prologue copies them instead of summing terms
    // and calling sincos per group
    bool pre_gv = false;
    uint32_t gv_lo = 0;   // pre_gv from two tables split at this many low CTA-index bits (Source::gv_lo)

    Gen(const plan::PassProgram& p, int nstates, bool zero_input, bool precomputed_groups = false,
        uint64_t compact_mask = 0)
        : P(p), ns(nstates), zero_in(zero_input && nstates == 1), umask(zero_in ? compact_mask : 0),
          pre_gv(precomputed_groups && (!zero_in || umask != 0) && !p.groups.empty())
    {
        R = 1u << P.rb;
        T = 1u << (P.k - P.rb);
        NW = std::max(1u, T / 32);
        const uint32_t nob = uint32_t(__builtin_popcountll(P.outer_mask));
        if (pre_gv && nob >= 2) {
            uint64_t lo = 0, m = P.outer_mask;
            for (uint32_t i = 0; i < nob / 2; ++i, m &= m - 1) lo |= m & (~m + 1);
            bool split = true;
            for (const plan::TermRec& t : P.terms) split = split && ((t.ocond & lo) == 0 || (t.ocond & ~lo) == 0);
            if (split) gv_lo = nob / 2;
        }
    }

    void set_layout(const plan::LayoutRec& L)
    {
        for (uint32_t i = 0; i < P.rb; ++i) reg[i] = L.reg[i];
        nthr = 0;
        for (uint32_t b = 0; b < P.k; ++b) {
            bool isreg = false;
            for (uint32_t i = 0; i < P.rb; ++i) isreg |= reg[i] == int(b);
            if (!isreg) thr[nthr++] = int(b);
        }
    }

    static std::string hex(uint64_t v)
    {
        char b[32];
        std::snprintf(b, sizeof(b), "0x%llxull", (unsigned long long)v);
        return b;
    }

    // physical index of register 0 of this thread: outer base | thread bits deposited
    std::string gbase_expr() const
    {
        std::string e = "ob";
        for (int t = 0; t < nthr; ++t)
            e += " | ((u64)((tid >> " + std::to_string(t) + ") & 1u) << " + std::to_string(P.tile_phys[thr[t]]) + ")";
        return e;
    }
    uint64_t reg_off(uint32_t j) const
    {
        uint64_t off = 0;
        for (uint32_t i = 0; i < P.rb; ++i)
            if ((j >> i) & 1) off |= uint64_t(1) << P.tile_phys[reg[i]];
        return off;
    }
    std::string slot_expr(const plan::LayoutRec& Lm) const
    {
        std::string e = "0u";
        for (int t = 0; t < nthr; ++t)
            e += " ^ (((tid >> " + std::to_string(t) + ") & 1u) * " + std::to_string(Lm.L[thr[t]]) + "u)";
        return e;
    }
    uint32_t slot_off(const plan::LayoutRec& Lm, uint32_t j) const
    {
        uint32_t s = 0;
        for (uint32_t i = 0; i < P.rb; ++i)
            if ((j >> i) & 1) s ^= Lm.L[reg[i]];
        return s;
    }

    uint32_t push(double v)
    {
        prm.push_back(v);
        return uint32_t(prm.size() - 1);
    }

    std::string cond(uint16_t tcond, uint64_t ocond) const
    {
        std::string c;
        if (tcond) c = "((tid & " + std::to_string(tcond) + "u) == " + std::to_string(tcond) + "u)";
        if (ocond) {
            if (!c.empty()) c += " && ";
            c += "((ob & " + hex(ocond) + ") == " + hex(ocond) + ")";
        }
        return c;
    }

    void each_state(const std::string& stmt_with_A)
    {
        // stmt_with_A contains "A" for the register array of one state
        for (int s = 0; s < ns; ++s) {
            std::string st = stmt_with_A;
            std::string name = s == 0 ? "a0" : "a1";
            size_t pos = 0;
            while ((pos = st.find("@A", pos)) != std::string::npos) {
                st.replace(pos, 2, name);
                pos += name.size();
            }
            o << "  " << st << "\n";
        }
    }

    void emit_flush_reg(int p)
    {
        if (P.acc_mul) {
            o << "  if (notOne(ar" << p << ")) { const double2 e = ar" << p << "; ar" << p
              << " = make_double2(1.0, 0.0);";
        } else {
            o << "  if (ar" << p << " != 0.0) { const double2 e = expi(ar" << p << "); ar" << p << " = 0.0;";
        }
        for (int s = 0; s < ns; ++s) o << " phD<" << (1 << p) << ">(" << (s ? "a1" : "a0") << ", e);";
        o << " }\n";
    }

    // per-thread accumulators: angles (sincos at each flush) or, with acc_mul,
    // complex factors multiplied by the groups' per-CTA (cos, sin)
    void emit_acc_decls()
    {
        const char* ty = P.acc_mul ? "double2" : "double";
        const char* one = P.acc_mul ? "make_double2(1.0, 0.0)" : "0.0";
        o << "  " << ty << " at = " << one;
        for (uint32_t i = 0; i < P.rb; ++i) o << ", ar" << i << " = " << one;
        o << ";\n";
        for (uint32_t i = P.rb; i < 5; ++i) o << "  " << ty << " ar" << i << " = " << one << "; (void)ar" << i << ";\n";
    }

    // ---- acc_mul: merged diagonal runs ----
    // Diagonal ops between two non-diagonal ones commute.  Each run becomes
    // one factor per register mask M (the product of its K_PHD groups, its
    // flushed accumulator chain, or, for M = 0, the K_ACC_THR chain times the
    // pass constant); the registers then take the products of the factors
    // whose masks they contain, built through a prefix trie when that needs
    // fewer complex multiplies than one multiply per (factor, register).
    // Factors with two or more lane-conditioned groups read a per-CTA table
    // over the 32 lanes, built once in the prologue; groups conditioned on
    // warp bits stay per-thread multiplies (uniform within a warp).
    struct Item { uint16_t tcond; uint16_t g; };
    struct Fac { std::vector<Item> items; bool hc = false; double ca = 1.0, cb = 0.0; };
    static constexpr uint32_t kMaxTables = 32;
    static constexpr int kThrChain = 5;   // chain index of the thread accumulator (after ar0..ar4)
    uint32_t max_tables = kMaxTables;   // 0 with precomputed group values (no prologue)
    std::vector<plan::KOp> run_ops;
    std::vector<Item> chain[kThrChain + 1];   // pending accumulator groups: ar0..ar4, at
    std::ostringstream tabs;      // prologue code building the lane tables
    uint32_t ntab = 0;
    uint32_t nvar = 0;

    static bool diag_kind(uint8_t k)
    {
        using namespace plan;
        return k == K_ACC_THR || k == K_ACC_REG || k == K_PHD || k == K_FLUSH_REG || k == K_FLUSH_ALL;
    }

    void emit_op(const plan::KOp& op)
    {
        if (P.acc_mul) {
            if (diag_kind(op.kind)) { run_ops.push_back(op); return; }
            // A phase generator's gradient sums sign * Im(conj(l) s) per
            // amplitude, which the diagonal phases still pending for both
            // states leave unchanged (unless a pending constant is not of unit
            // modulus): it is taken without applying them, from one cached
            // Im(conj(l) s) per register shared by every such occurrence of the
            // run, and the run of phases stays open.
            if (ns == 2 && (op.kind == plan::K_GRAD_Z || op.kind == plan::K_GRAD_P) && run_unimodular()) {
                if (!qv) {
                    for (uint32_t j = 0; j < R; ++j) o << "  qz[" << j << "] = im_ls(a1[" << j << "], a0[" << j << "]);";
                    o << "\n";
                    qv = true;
                }
                emit_grad(op, true);
                return;
            }
            flush_run();
        }
        emit(op);
    }

    // no pending constant of the open run scales the amplitudes
    bool run_unimodular() const
    {
        for (const plan::KOp& k : run_ops)
            if (k.kind == plan::K_FLUSH_ALL && std::fabs(k.a * k.a + k.b * k.b - 1.0) > 1e-12) return false;
        return true;
    }

    static std::string cond_t(const char* v, uint16_t tc)
    {
        return std::string("((") + v + " & " + std::to_string(tc) + "u) == " + std::to_string(tc) + "u)";
    }

    std::string emit_factor(const Fac& F)
    {
        std::vector<Item> L, W;
        for (const Item& it : F.items) ((it.tcond & ~31u) == 0 ? L : W).push_back(it);
        const std::string v = "f" + std::to_string(nvar++);
        std::string cst;
        if (F.hc) {
            const uint32_t ci = push(F.ca);
            push(F.cb);
            cst = "make_double2(P.v[" + std::to_string(ci) + "], P.v[" + std::to_string(ci + 1) + "])";
        }
        if (ntab < max_tables && (L.size() >= 2 || (L.size() == 1 && F.hc))) {
            const uint32_t t = ntab++;
            tabs << "  if ((tid >> 5) == " << (t % NW) << "u) { const u32 l = tid & 31u; double2 v = "
                 << (F.hc ? cst : std::string("make_double2(1.0, 0.0)")) << ";";
            for (const Item& it : L) {
                if (it.tcond) tabs << " if (" << cond_t("l", it.tcond) << ")";
                tabs << " v = cmul(v, gv[" << it.g << "]);";
            }
            tabs << " tb[" << t * 32 << "u + l] = v; }\n";
            o << "    double2 " << v << " = tb[" << t * 32 << "u + (tid & 31u)];\n";
        } else {
            size_t i = 0;
            o << "    double2 " << v << " = ";
            if (F.hc) o << cst;
            else if (!L.empty()) {
                const Item& it = L[i++];
                if (it.tcond) o << cond_t("tid", it.tcond) << " ? gv[" << it.g << "] : make_double2(1.0, 0.0)";
                else o << "gv[" << it.g << "]";
            } else o << "make_double2(1.0, 0.0)";
            o << ";\n";
            for (; i < L.size(); ++i) {
                o << "    ";
                if (L[i].tcond) o << "if (" << cond_t("tid", L[i].tcond) << ") ";
                o << v << " = cmul(" << v << ", gv[" << L[i].g << "]);\n";
            }
        }
        for (const Item& it : W)
            o << "    if (" << cond_t("tid", it.tcond) << ") " << v << " = cmul(" << v << ", gv[" << it.g << "]);\n";
        return v;
    }

    void flush_run()
    {
        using namespace plan;
        if (run_ops.empty()) return;
        std::map<int, Fac> fac;
        auto take = [&](int c, int mask) {
            std::vector<Item>& d = fac[mask].items;
            d.insert(d.end(), chain[c].begin(), chain[c].end());
            chain[c].clear();
        };
        for (const KOp& op : run_ops) {
            switch (op.kind) {
            case K_ACC_REG: chain[op.p].push_back(Item{op.tcond, op.g}); break;
            case K_ACC_THR: chain[kThrChain].push_back(Item{op.tcond, op.g}); break;
            case K_PHD: fac[op.f].items.push_back(Item{op.tcond, op.g}); break;
            case K_FLUSH_REG: take(op.p, 1 << op.p); break;
            case K_FLUSH_ALL: {
                for (uint32_t r = 0; r < P.rb; ++r)
                    if ((op.f >> r) & 1) take(int(r), 1 << r);
                take(kThrChain, 0);
                if (!(op.a == 1.0 && op.b == 0.0)) {
                    Fac& f = fac[0];
                    const double a = f.ca * op.a - f.cb * op.b, b = f.ca * op.b + f.cb * op.a;
                    f.ca = a;
                    f.cb = b;
                    f.hc = true;
                }
                break;
            }
            default: break;
            }
        }
        run_ops.clear();
        for (auto it = fac.begin(); it != fac.end();)
            it = (it->second.items.empty() && !it->second.hc) ? fac.erase(it) : std::next(it);
        if (fac.empty()) return;
        qv = false;   // the phases change the registers
        o << "  {\n";
        std::vector<int> masks;
        std::map<int, std::string> val;
        for (auto& kv : fac) {
            masks.push_back(kv.first);
            val[kv.first] = emit_factor(kv.second);
        }
        std::stable_sort(masks.begin(), masks.end(),
                         [](int a, int b) { return __builtin_popcount(a) < __builtin_popcount(b); });
        // per register: the masks it contains, in the sorted order
        std::vector<std::vector<int>> key(R);
        size_t direct = 0;
        for (uint32_t j = 0; j < R; ++j)
            for (int m : masks)
                if ((int(j) & m) == m) { key[j].push_back(m); ++direct; }
        std::map<std::vector<int>, std::string> node;
        size_t trie = 0;
        for (uint32_t j = 0; j < R; ++j) {
            if (key[j].empty()) continue;
            ++trie;
            for (size_t len = 2; len <= key[j].size(); ++len)
                if (node.emplace(std::vector<int>(key[j].begin(), key[j].begin() + len), std::string()).second) ++trie;
        }
        auto apply = [&](uint32_t j, const std::string& e) {
            for (int s = 0; s < ns; ++s) {
                const char* A = s ? "a1" : "a0";
                o << "    " << A << "[" << j << "] = cmul(" << A << "[" << j << "], " << e << ");\n";
            }
        };
        if (trie < direct) {
            for (auto& kv : node) {   // map order: every prefix precedes its extensions
                const std::vector<int>& k = kv.first;
                const std::vector<int> parent(k.begin(), k.end() - 1);
                const std::string pv = parent.size() == 1 ? val[parent[0]] : node[parent];
                kv.second = "t" + std::to_string(nvar++);
                o << "    const double2 " << kv.second << " = cmul(" << pv << ", " << val[k.back()] << ");\n";
            }
            for (uint32_t j = 0; j < R; ++j)
                if (!key[j].empty()) apply(j, key[j].size() == 1 ? val[key[j][0]] : node[key[j]]);
        } else {
            for (int m : masks)
                for (int s = 0; s < ns; ++s) {
                    const char* A = s ? "a1" : "a0";
                    if (m == 0) o << "    scaleAll(" << A << ", " << val[m] << ");\n";
                    else o << "    phD<" << m << ">(" << A << ", " << val[m] << ");\n";
                }
        }
        o << "  }\n";
    }

    std::string run()
    {
        const uint32_t tsize = 1u << P.k;
        const uint32_t ng = uint32_t(P.groups.size());
        const uint32_t nslots = uint32_t(P.slot_src.size());

        // the pass body first (it decides the lane tables the prologue builds)
        set_layout(P.layouts[P.layout0]);
        std::ostringstream body;
        std::swap(o, body);
        if (!P.acc_mul) emit_acc_decls();
        for (const plan::KOp& op : P.ops) emit_op(op);
        flush_run();
        // store (final layout)
        for (uint32_t j = 0; j < R; ++j) {
            const std::string ix = "gb + " + hex(reg_off(j));
            o << "  " << guard(ix, nstr()) << "psi[" << ix << "] = a0[" << j << "];";
            if (ns == 2) o << " " << guard(ix, nstr()) << "lam[" << ix << "] = a1[" << j << "];";
            o << "\n";
        }
        if (!lpos.empty()) emit_prob();
        for (const auto& kv : gacc)
            o << "  { const double v = warpSum<" << T << ">(gs" << kv.second << ");"
              << " if ((tid & 31u) == 0u) wp[" << kv.first << "u * " << NW << "u + (tid >> 5)] += v; }\n";
        if (ns == 2 && nslots) {
            o << "  __syncthreads();\n"
              << "  for (u32 s = tid; s < " << nslots << "u; s += " << T << "u) { double v = 0.0;"
              << " for (u32 w = 0; w < " << NW << "u; ++w) v += wp[s * " << NW << "u + w];"
              << " slot_partial[(u64)s * gridDim.x + blockIdx.x] = v; }\n";
        }
        std::swap(o, body);
        const std::string ops_txt = body.str();
        set_layout(P.layouts[P.layout0]);

        std::ostringstream head;
        std::swap(o, head);
        o << "  const u32 tid = threadIdx.x;\n";
        for (const auto& kv : gacc) o << "  double gs" << kv.second << " = 0.0;\n";
        if (ns == 2) o << "  double qz[" << R << "]; (void)qz;\n";
        o << "  extern __shared__ double2 sm[];\n";
        o << "  double2* xb = sm; (void)xb;\n";
        o << "  double2* gv = sm + " << tsize << "; (void)gv;\n";
        o << "  double2* tb = gv + " << ng << "; (void)tb;\n";
        if (ns == 2) o << "  double* wp = reinterpret_cast<double*>(tb + " << 32 * ntab << ");\n";
        // outer base
        o << "  u64 ob = 0;\n  { u64 c = blockIdx.x;";
        for (uint32_t q = 0; q < 64; ++q)
            if ((P.outer_mask >> q) & 1) o << " ob |= (c & 1ull) << " << q << "; c >>= 1;";
        o << " (void)c; }\n";
        if (zero_in) {
            // basis-state input |bi> (bi: physical index, from the parameter block so
            // one kernel serves every index): only the tile holding bi has a nonzero
            // amplitude; every gate is linear, so every other tile's output is zero,
            // stored in tile-local order m = tid + j*T (the tile always holds physical
            // qubits 0..2, so consecutive threads write consecutive amplitudes).
            // Compact input (umask): the input is zero unless the bits outside umask
            // equal bi's, so a tile whose outer bits outside umask differ stores zeros
            basis_slot = int(push(0.0));
            o << "  const u64 bi = (u64)P.v[" << basis_slot << "]; (void)bi;\n";
            const uint32_t lt = uint32_t(__builtin_ctz(T));
            const uint64_t zmask = P.outer_mask & ~umask & ~pmask;
            if (zmask) {
                o << "  if (((ob ^ bi) & " << hex(zmask) << ") != 0ull) {\n    const u64 gz = ob";
                for (uint32_t b = 0; b < lt; ++b)
                    o << " | ((u64)((tid >> " << b << ") & 1u) << " << int(P.tile_phys[b]) << ")";
                o << ";\n";
                for (uint32_t j = 0; j < R; ++j) {
                    uint64_t cj = 0;
                    const uint64_t m = uint64_t(j) * T;
                    for (uint32_t b = lt; b < P.k; ++b)
                        if ((m >> b) & 1) cj |= uint64_t(1) << P.tile_phys[b];
                    o << "    " << guard("gz + " + hex(cj), nstr()) << "psi[gz + " << hex(cj)
                      << "] = make_double2(0.0, 0.0);\n";
                }
                o << "    return;\n  }\n";
            }
        }
        // load first (gb holds only thread and outer bits, the offsets only
        // register bits: gb + off == gb | off, and the constant folds into the
        // address); the prologue below then runs while the loads are in flight
        o << "  u64 gb = " << gbase_expr() << ";\n";
        for (int s = 0; s < ns; ++s) o << "  double2 a" << s << "[" << R << "];\n";
        if (!zero_in) {
            for (uint32_t j = 0; j < R; ++j) {
                const std::string ix = "gb + " + hex(reg_off(j));
                o << "  a0[" << j << "] = " << ld("psi", ix, nstr()) << ";";
                if (ns == 2) o << " a1[" << j << "] = " << ld("lam", ix, nstr()) << ";";
                o << "\n";
            }
        } else if (umask) {
            // compact input: amplitude x = lam[pext(x, umask)] where x's other tile
            // bits equal bi's, else 0 (pext of gb and of each register offset add:
            // their bits are disjoint)
            auto rank = [&](uint32_t q) { return __builtin_popcountll(umask & ((uint64_t(1) << q) - 1)); };
            o << "  u64 cb = 0;\n  { u64 c = blockIdx.x;";
            for (uint32_t q = 0; q < 64; ++q)
                if ((P.outer_mask >> q) & 1) {
                    if ((umask >> q) & 1) o << " cb |= (c & 1ull) << " << rank(q) << ";";
                    o << " c >>= 1;";
                }
            o << " (void)c; }\n";
            for (int t = 0; t < nthr; ++t) {
                const uint32_t q = P.tile_phys[thr[t]];
                if ((umask >> q) & 1) o << "  cb |= (u64)((tid >> " << t << ") & 1u) << " << rank(q) << ";\n";
            }
            uint64_t tmask = 0;
            for (uint32_t b = 0; b < P.k; ++b) tmask |= uint64_t(1) << P.tile_phys[b];
            const uint64_t tz = tmask & ~umask & ~pmask;
            for (uint32_t j = 0; j < R; ++j) {
                uint64_t coff = 0;
                for (uint32_t i = 0; i < P.rb; ++i)
                    if ((j >> i) & 1) {
                        const uint32_t q = P.tile_phys[reg[i]];
                        if ((umask >> q) & 1) coff |= uint64_t(1) << rank(q);
                    }
                o << "  a0[" << j << "] = ";
                if (tz) o << "((((gb | " << hex(reg_off(j)) << ") ^ bi) & " << hex(tz) << ") == 0ull) ? ";
                o << ld("lam", "cb + " + hex(coff), hex(uint64_t(1) << __builtin_popcountll(umask)));
                if (tz) o << " : make_double2(0.0, 0.0)";
                o << ";\n";
            }
            if (pmask) {
                // product qubits on outer and thread bits: one factor per thread
                o << "  double2 pf = make_double2(1.0, 0.0);\n";
                for (uint32_t q = 0; q < 64; ++q)
                    if ((P.outer_mask >> q) & (pmask >> q) & 1)
                        o << "  pf = cmul(pf, " << ld("lam", ph_index(q) + " + ((ob >> " + std::to_string(q) + ") & 1ull)", ph_size())
                          << ");\n";
                for (int t = 0; t < nthr; ++t) {
                    const uint32_t q = P.tile_phys[thr[t]];
                    if ((pmask >> q) & 1)
                        o << "  pf = cmul(pf, "
                          << ld("lam", ph_index(q) + " + (u64)((tid >> " + std::to_string(t) + ") & 1u)", ph_size()) << ");\n";
                }
                for (uint32_t i = 0; i < P.rb; ++i) preg |= ((pmask >> P.tile_phys[reg[i]]) & 1) != 0;
            }
        }
        // prologue: per-CTA diagonal group values, then the lane tables
        if (ng && pre_gv && gv_lo) {
            const uint32_t nob = uint32_t(__builtin_popcountll(P.outer_mask));
            const uint64_t rows_lo = uint64_t(1) << gv_lo;
            const std::string total = hex((rows_lo + (uint64_t(1) << (nob - gv_lo))) * ng);
            o << "  for (u32 g = tid; g < " << ng << "u; g += " << T << "u) {\n"
              << "    const double2 l = "
              << ld("gvt", "(u64)(blockIdx.x & " + hex(rows_lo - 1) + ") * " + std::to_string(ng) + "u + g", total) << ";\n"
              << "    const double2 h = "
              << ld("gvt", hex(rows_lo * ng) + " + (u64)(blockIdx.x >> " + std::to_string(gv_lo) + ") * " +
                               std::to_string(ng) + "u + g", total)
              << ";\n";
            // the groups' kinds are known here: no load of the group records.  The
            // product's roundings are written out (no contraction left to the
            // compiler), so the debug mode's kernel gives the same bits
            bool all_direct = true, none_direct = true;
            for (const plan::GroupRec& gr : P.groups) {
                all_direct = all_direct && gr.direct;
                none_direct = none_direct && !gr.direct;
            }
            const std::string prod = "make_double2(__fma_rn(l.x, h.x, -__dmul_rn(l.y, h.y)), __fma_rn(l.x, h.y, __dmul_rn(l.y, h.x)))";
            const std::string sum = "make_double2(__dadd_rn(l.x, h.x), 0.0)";
            if (all_direct) o << "    gv[g] = " << prod << ";\n  }\n";
            else if (none_direct) o << "    gv[g] = " << sum << ";\n  }\n";
            else o << "    gv[g] = groups[g].direct ? " << prod << " : " << sum << ";\n  }\n";
        } else if (ng && pre_gv) {
            o << "  for (u32 g = tid; g < " << ng << "u; g += " << T << "u) gv[g] = "
              << ld("gvt", "(u64)blockIdx.x * " + std::to_string(ng) + "u + g", "(u64)gridDim.x * " + std::to_string(ng) + "u")
              << ";\n";
        } else if (ng) {
            // the pass's terms are first copied into the exchange buffer (unused until
            // the first layout exchange, which follows the prologue's barrier) by every
            // thread at once, so the per-group sums read shared memory instead of
            // issuing one dependent global load per term
            const size_t nterms = P.terms.size();
            const bool stage = nterms > 0 && nterms <= tsize;
            if (stage)
                o << "  TermRec* ts = reinterpret_cast<TermRec*>(xb);\n"
                  << "  for (u32 i = tid; i < " << nterms << "u; i += " << T << "u) ts[i] = terms[i];\n"
                  << "  __syncthreads();\n";
            o << "  for (u32 g = tid; g < " << ng << "u; g += " << T << "u) {\n"
              << "    const GroupRec gr = groups[g]; double th = 0.0;\n"
              << "    for (u32 i = 0; i < gr.count; ++i) { const TermRec t = " << (stage ? "ts" : "terms")
              << "[gr.first + i]; if ((ob & t.ocond) == t.ocond) th += t.theta; }\n"
              << "    gv[g] = gr.direct ? expi(th) : make_double2(th, 0.0);\n  }\n";
        }
        if (ntab) o << "  __syncthreads();\n" << tabs.str();
        if (ns == 2 && nslots) o << "  for (u32 i = tid; i < " << nslots * NW << "u; i += " << T << "u) wp[i] = 0.0;\n";
        if (preg) {
            // product qubits on register bits: the factor of every register index
            o << "  double2* pfs = tb + " << 32 * ntab << ";\n"
              << "  for (u32 j = tid; j < " << R << "u; j += " << T << "u) {\n    double2 f = make_double2(1.0, 0.0);\n";
            for (uint32_t i = 0; i < P.rb; ++i) {
                const uint32_t q = P.tile_phys[reg[i]];
                if ((pmask >> q) & 1)
                    o << "    f = cmul(f, " << ld("lam", ph_index(q) + " + (u64)((j >> " + std::to_string(i) + ") & 1u)", ph_size())
                      << ");\n";
            }
            o << "    pfs[j] = f;\n  }\n";
        }
        o << "  __syncthreads();\n";
        if (zero_in && !umask)
            for (uint32_t j = 0; j < R; ++j)
                o << "  a0[" << j << "] = make_double2((gb | " << hex(reg_off(j)) << ") == bi ? 1.0 : 0.0, 0.0);\n";
        if (pmask && !preg) {
            for (uint32_t j = 0; j < R; ++j) o << "  a0[" << j << "] = cmul(a0[" << j << "], pf);\n";
        } else if (preg) {
            bool all = true;   // every register bit a product qubit: one input value per thread
            for (uint32_t i = 0; i < P.rb; ++i) all = all && ((pmask >> P.tile_phys[reg[i]]) & 1);
            if (all) {
                o << "  { const double2 pv = cmul(a0[0], pf);";
                for (uint32_t j = 0; j < R; ++j) o << " a0[" << j << "] = cmul(pv, pfs[" << j << "]);";
                o << " }\n";
            } else {
                for (uint32_t j = 0; j < R; ++j)
                    o << "  a0[" << j << "] = cmul(a0[" << j << "], cmul(pf, pfs[" << j << "]));\n";
            }
        }
        std::swap(o, head);

        std::ostringstream src;
        src << kPrelude << "\n";
        src << "struct Prm { double v[" << std::max<size_t>(1, prm.size()) << "]; };\n";
        // resident CTAs per SM the register budget allows: 128 registers per
        // thread, 168 for 32 amplitudes per thread (their 128 registers and the
        // rest; three CTAs of 128 threads per SM)
        const uint32_t budget = R >= 32 ? 168u : 128u;
        const uint32_t min_blocks = std::max(1u, std::min(8u, 65536u / (T * budget)));
        src << "extern \"C\" __global__ void __launch_bounds__(" << T << ", " << min_blocks << ") " << kernel_name() << "("
            << "double2* __restrict__ psi, double2* __restrict__ lam, const TermRec* __restrict__ terms, "
            << "const GroupRec* __restrict__ groups, double* __restrict__ slot_partial, u32* __restrict__ status, "
            << "const double2* __restrict__ gvt, const __grid_constant__ Prm P)\n{\n"
            << "  (void)lam; (void)terms; (void)groups; (void)slot_partial; (void)status; (void)gvt;\n"
            << head.str() << ops_txt << "}\n";
        return src.str();
    }

    // Probability side output of the last pass of an execute: |a|^2 of every
    // stored amplitude (re*re + im*im, two roundings, as the sampler computes
    // it) into prob[logical index], and the sums of its logical 4096-blocks
    // into bsum = prob + 2^n (zeroed before the pass; atomic adds, so their
    // order varies, which only the sampler's binade guess sees).  The tile's
    // values go through shared memory in "local" order (tile bits sorted by
    // logical position) so that consecutive threads store consecutive logical
    // indices.  An XOR of the lane bits that sit at local positions >= 4 into
    // the free low positions keeps the scattered writes to shared memory at
    // most two-way conflicted; the linear reads stay conflict-free.
    void emit_prob()
    {
        const uint32_t n = P.k + uint32_t(__builtin_popcountll(P.outer_mask));
        // local rank of every tile bit
        std::vector<std::pair<int, uint32_t>> lp;
        for (uint32_t b = 0; b < P.k; ++b) lp.push_back({lpos[P.tile_phys[b]], b});
        std::sort(lp.begin(), lp.end());
        uint32_t lr[16] = {0};
        std::vector<int> lsorted(P.k);
        for (uint32_t i = 0; i < P.k; ++i) {
            lr[lp[i].second] = i;
            lsorted[i] = lp[i].first;
        }
        // swizzle: lane bits at local positions >= 4 into the free low positions
        const uint32_t nl = std::min<uint32_t>(5, uint32_t(nthr));
        uint32_t lowused = 0;
        std::vector<uint32_t> highlane;
        for (uint32_t t = 0; t < nl; ++t) {
            const uint32_t l = lr[thr[t]];
            if (l < 4) lowused |= 1u << l;
            else highlane.push_back(l);
        }
        std::string swz;
        {
            uint32_t slot = 0;
            for (uint32_t l : highlane) {
                while (slot < 4 && ((lowused >> slot) & 1)) ++slot;
                if (slot >= 4) break;
                swz += " ^ (((x >> " + std::to_string(l) + ") & 1u) << " + std::to_string(slot) + ")";
                ++slot;
            }
        }
        o << "  {\n    // probabilities in logical order and their 4096-block sums\n"
          << "    double* const prob = slot_partial;\n"
          << "    double* const bsum = prob + " << hex(uint64_t(1) << n) << ";\n"
          << "    double* const pb = reinterpret_cast<double*>(xb);\n"
          << "    auto sw = [](u32 x) { return x" << swz << "; };\n"
          << "    __syncthreads();\n";
        std::string ls = "0u";
        for (int t = 0; t < nthr; ++t)
            ls += " | (((tid >> " + std::to_string(t) + ") & 1u) << " + std::to_string(lr[thr[t]]) + ")";
        o << "    const u32 ls = " << ls << ";\n";
        for (uint32_t j = 0; j < R; ++j) {
            uint32_t off = 0;
            for (uint32_t i = 0; i < P.rb; ++i)
                if ((j >> i) & 1) off |= 1u << lr[reg[i]];
            o << "    pb[sw(ls | " << off << "u)] = __dadd_rn(__dmul_rn(a0[" << j << "].x, a0[" << j << "].x), __dmul_rn(a0["
              << j << "].y, a0[" << j << "].y));\n";
        }
        o << "    __syncthreads();\n";
        // logical base of the tile and of this thread's store index (tid + k*T)
        o << "    u64 lb = 0;\n    { u64 c = blockIdx.x;";
        for (uint32_t q = 0; q < 64; ++q)
            if ((P.outer_mask >> q) & 1) o << " lb |= (c & 1ull) << " << int(lpos[q]) << "; c >>= 1;";
        o << " (void)c; }\n";
        const uint32_t lt = uint32_t(__builtin_ctz(T));
        std::string lt_expr = "lb";
        for (uint32_t i = 0; i < lt; ++i)
            lt_expr += " | ((u64)((tid >> " + std::to_string(i) + ") & 1u) << " + std::to_string(lsorted[i]) + ")";
        o << "    const u64 lbt = " << lt_expr << ";\n";
        // block key of each k: the logical bits >= 12 of its local bits; the
        // thread bits must all map below 12 for a per-CTA reduction
        uint32_t i0 = P.k;
        for (uint32_t i = 0; i < P.k; ++i)
            if (lsorted[i] >= 12) { i0 = i; break; }
        std::map<uint64_t, std::vector<uint32_t>> keys;
        for (uint32_t kk = 0; kk < R; ++kk) {
            uint64_t lk = 0;
            for (uint32_t i = lt; i < P.k; ++i)
                if (((uint64_t(kk) * T) >> i) & 1) lk |= uint64_t(1) << lsorted[i];
            o << "    const double p" << kk << " = pb[sw(tid + " << kk * T << "u)]; "
              << guard("lbt | " + hex(lk), hex(uint64_t(1) << n)) << "prob[lbt | " << hex(lk) << "] = p" << kk << ";\n";
            keys[lk >> 12].push_back(kk);
        }
        prob_bsum = i0 >= 5;
        if (i0 >= lt && T >= 32) {
            // one sum per block key: per thread, then across the warp by a
            // transpose-reduce butterfly (each exchange halves the values a lane
            // holds: 2K - 1 + 5 - log2 K shuffles for K keys instead of 5K), then
            // per CTA in shared memory
            o << "    double* const bs = pb + " << (1u << P.k) << ";\n";
            uint32_t K = 1;
            while (K < keys.size()) K <<= 1;
            o << "    {\n";
            uint32_t ki = 0;
            for (const auto& kv : keys) {
                o << "      double v" << ki << " = 0.0;";
                for (uint32_t kk : kv.second) o << " v" << ki << " += p" << kk << ";";
                o << "\n";
                ++ki;
            }
            for (; ki < K; ++ki) o << "      double v" << ki << " = 0.0;\n";
            uint32_t c = K, keymask = 0;
            std::vector<std::pair<uint32_t, uint32_t>> keybits;   // (lane bit, key bit value)
            for (uint32_t off = 16; off >= 1; off >>= 1) {
                if (c > 1) {
                    const uint32_t h = c / 2;
                    o << "      { const bool hi = (tid & " << off << "u) != 0u;";
                    for (uint32_t i = 0; i < h; ++i)
                        o << " { const double s = hi ? v" << i << " : v" << i + h << "; const double k = hi ? v" << i + h
                          << " : v" << i << "; v" << i << " = k + __shfl_xor_sync(0xffffffffu, s, " << off << "); }";
                    o << " }\n";
                    keybits.push_back({off, h});
                    c = h;
                } else {
                    o << "      v0 += __shfl_xor_sync(0xffffffffu, v0, " << off << ");\n";
                    keymask |= off;
                }
            }
            std::string key = "0u";
            for (const auto& kb : keybits) key += " + (((tid & " + std::to_string(kb.first) + "u) != 0u) ? " +
                                                  std::to_string(kb.second) + "u : 0u)";
            o << "      const u32 key = " << key << ";\n"
              << "      if ((tid & " << keymask << "u) == 0u && key < " << keys.size() << "u) bs[key * " << NW
              << "u + (tid >> 5)] = v0;\n    }\n";
            o << "    __syncthreads();\n";
            ki = 0;
            for (const auto& kv : keys) {
                o << "    if (tid == " << ki << "u) { double v = 0.0; for (u32 w = 0; w < " << NW << "u; ++w) v += bs["
                  << ki * NW << "u + w]; " << guard("((lb >> 12) | " + hex(kv.first) + ")", hex(uint64_t(1) << n >> 12))
                  << "atomicAdd(bsum + ((lb >> 12) | " << hex(kv.first) << "), v); }\n";
                ++ki;
            }
        } else if (prob_bsum) {
            // warp bits at logical positions >= 12: one sum per warp and k
            for (uint32_t kk = 0; kk < R; ++kk) {
                uint64_t lk = 0;
                for (uint32_t i = lt; i < P.k; ++i)
                    if (((uint64_t(kk) * T) >> i) & 1) lk |= uint64_t(1) << lsorted[i];
                const std::string bix = "((lbt | " + hex(lk) + ") >> 12)";
                o << "    { const double v = warpSum<" << T << ">(p" << kk << "); if ((tid & 31u) == 0u) { "
                  << guard(bix, hex(uint64_t(1) << n >> 12)) << "atomicAdd(bsum + " << bix << ", v); } }\n";
            }
        }
        // else: lane bits at logical positions >= 12 (a warp's 32 values span
        // several blocks); the sampler sums the blocks from prob instead
        o << "  }\n";
    }

    // ---- streamed pass (forward passes on large states) ----
    // One persistent CTA per SM with two compute groups of T threads that take
    // alternate tiles.  Tiles arrive in a ring of three shared-memory slots by
    // bulk async copies (one per contiguous piece of 2^c amplitudes, completion
    // counted on the slot's mbarrier).  A group waits for its slot, loads its
    // registers from it, runs the pass with the slot as its exchange buffer
    // (group-local named barriers), stores straight to global memory, and then
    // itself issues the copies of the tile three ahead into the slot it just
    // freed -- a tile the other group takes next -- so the loads of upcoming
    // tiles run while both groups compute.  Every wait is bounded: a wait that
    // gives up writes a nonzero code to *status (mapped host memory, plain stores) and the group leaves its loop (group-
    // uniformly); before the CTA exits, thread 0 waits (bounded) for every copy
    // it knows was issued.
    static constexpr uint32_t kWaitLimit = 1u << 24;

    static uint32_t contiguous_low_bits(const plan::PassProgram& p)
    {
        uint32_t c = 0;
        while (c < p.k && p.tile_phys[c] == c) ++c;
        return c;
    }

    size_t streamed_smem() const
    {
        const size_t tsize = size_t(1) << P.k;
        return 3 * tsize * 16 + 64 + P.terms.size() * 16 + 2 * (P.groups.size() + 32 * size_t(ntab)) * 16;
    }

    std::string run_streamed()
    {
        const uint32_t tsize = 1u << P.k;
        const uint32_t ng = uint32_t(P.groups.size());
        const uint32_t nt = uint32_t(P.terms.size());
        const uint32_t c = contiguous_low_bits(P);
        const uint32_t npieces = 1u << (P.k - c), piece = 1u << c;
        const uint32_t nth = 2 * T;
        const uint32_t lt = uint32_t(__builtin_ctz(T));
        SYNC = "group_sync(1u + grp, " + std::to_string(T) + "u);";
        xb_used = true;   // the registers are loaded from the slot the first exchange writes

        set_layout(P.layouts[P.layout0]);
        std::ostringstream body;
        std::swap(o, body);
        if (!P.acc_mul) emit_acc_decls();
        for (const plan::KOp& op : P.ops) emit_op(op);
        flush_run();
        for (uint32_t j = 0; j < R; ++j) o << "      psi[gb + " << hex(reg_off(j)) << "] = a0[" << j << "];\n";
        std::swap(o, body);
        const std::string ops_txt = body.str();
        set_layout(P.layouts[P.layout0]);
        const uint32_t gstride = ng + 32 * ntab;

        std::string deposit = "u64 ob = 0; { u64 cc = tile;";
        for (uint32_t q = 0; q < 64; ++q)
            if ((P.outer_mask >> q) & 1) deposit += " ob |= (cc & 1ull) << " + std::to_string(q) + "; cc >>= 1;";
        deposit += " (void)cc; }";
        std::string scatter = "0ull";
        for (uint32_t b = c; b < P.k; ++b)
            scatter += " | ((u64)((p >> " + std::to_string(b - c) + ") & 1u) << " + std::to_string(P.tile_phys[b]) + ")";
        std::string lbase = "0u";
        for (int t = 0; t < nthr; ++t)
            lbase += " | (((tid >> " + std::to_string(t) + ") & 1u) << " + std::to_string(thr[t]) + ")";
        const uint64_t ntiles = uint64_t(1) << __builtin_popcountll(P.outer_mask);
        const std::string NT = std::to_string(ntiles) + "ull";
        const std::string LIM = std::to_string(kWaitLimit) + "u";

        std::ostringstream s;
        s << kPrelude << "\n";
        s << "struct Prm { double v[" << std::max<size_t>(1, prm.size()) << "]; };\n";
        // the copies of one tile: lane 0 announces the bytes, the warp's lanes issue the pieces
        s << "__device__ __forceinline__ void fill(double2* __restrict__ psi, double2* sm, u64* bar, u32* nfill, u64 tile, "
             "u32 s, u32 lane)\n{\n"
          << "  if (lane == 0u) { mbar_expect_tx(bar + s, " << tsize * 16 << "u); nfill[s] += 1u; }\n"
          << "  __syncwarp();\n"
          << "  " << deposit << "\n"
          << "  double2* const dst = sm + s * " << tsize << "u;\n"
          << "  for (u32 p = lane; p < " << npieces << "u; p += 32u)\n"
          << "    bulk_g2s(dst + p * " << piece << "u, psi + (ob | " << scatter << "), " << piece * 16 << "u, bar + s);\n"
          << "}\n";
        s << "extern \"C\" __global__ void __launch_bounds__(" << nth << ", 1) qse_pass("
          << "double2* __restrict__ psi, double2* __restrict__ lam, const TermRec* __restrict__ terms, "
          << "const GroupRec* __restrict__ groups, double* __restrict__ slot_partial, u32* __restrict__ status, "
          << "const double2* __restrict__ gvt, const __grid_constant__ Prm P)\n{\n"
          << "  (void)lam; (void)slot_partial; (void)gvt;\n"
          << "  extern __shared__ __align__(128) double2 sm[];\n"
          << "  u64* const bar = reinterpret_cast<u64*>(sm + " << 3 * tsize << ");   // one per slot\n"
          << "  u32* const nfill = reinterpret_cast<u32*>(bar + 4);                   // copies issued per slot\n"
          << "  TermRec* const ts = reinterpret_cast<TermRec*>(bar + 8);\n"
          << "  double2* const gscr = reinterpret_cast<double2*>(ts + " << nt << ");\n"
          << "  const u32 tx = threadIdx.x, grp = tx >> " << lt << ", tid = tx & " << (T - 1) << "u;\n"
          << "  if (tx == 0u) {\n"
          << "    for (u32 i = 0; i < 3u; ++i) { mbar_init(bar + i, 1u); nfill[i] = 0u; }\n"
          << "    mbar_fence_init();\n"
          << "  }\n"
          << "  __syncthreads();\n"
          << "  if (tx < 32u)\n"
          << "    for (u32 i = 0; i < 3u; ++i)\n"
          << "      if (blockIdx.x + (u64)i * gridDim.x < " << NT << ") fill(psi, sm, bar, nfill, blockIdx.x + (u64)i * gridDim.x, i, tx);\n"
          << "  for (u32 i = tx; i < " << nt << "u; i += " << nth << "u) ts[i] = terms[i];\n"
          << "  __syncthreads();\n"
          << "  double2* const gv = gscr + grp * " << gstride << "u; (void)gv;\n"
          << "  double2* const tb = gv + " << ng << "; (void)tb;\n"
          << "  u32 it = grp;\n"
          << "  for (u64 tile = blockIdx.x + (u64)grp * gridDim.x; tile < " << NT << "; tile += 2ull * gridDim.x, it += 2u) {\n"
          << "    const u32 s = it % 3u, use = it / 3u;\n"
          << "    double2* const xb = sm + s * " << tsize << "u;\n"
          << "    " << deposit << "\n";
        if (ng) {
            s << "    for (u32 g = tid; g < " << ng << "u; g += " << T << "u) {\n"
              << "      const GroupRec gr = groups[g]; double th = 0.0;\n"
              << "      for (u32 i = 0; i < gr.count; ++i) { const TermRec t = ts[gr.first + i];"
                 " if ((ob & t.ocond) == t.ocond) th += t.theta; }\n"
              << "      gv[g] = gr.direct ? expi(th) : make_double2(th, 0.0);\n    }\n";
            s << "    " << SYNC << "\n";
            if (ntab) s << tabs.str() << "    " << SYNC << "\n";
        }
        s << "    if (!group_all(1u + grp, " << T << "u, mbar_wait(bar + s, use & 1u, " << LIM << "))) {"
             " if (tid == 0u) *(volatile u32*)status = 1u; break; }\n"
          << "    {\n"
          << "      u64 gb = " << gbase_expr() << ";\n"
          << "      const u32 lb = " << lbase << ";\n"
          << "      double2 a0[" << R << "];\n";
        for (uint32_t j = 0; j < R; ++j) {
            uint32_t loc = 0;
            for (uint32_t i = 0; i < P.rb; ++i)
                if ((j >> i) & 1) loc |= 1u << reg[i];
            s << "      a0[" << j << "] = xb[lb + " << loc << "u];\n";
        }
        s << ops_txt
          << "    }\n"
          << "    fence_proxy_async();   // this group's shared-memory writes before the copies that reuse the slot\n"
          << "    " << SYNC << "\n"
          << "    const u64 next = tile + 3ull * gridDim.x;\n"
          << "    if (tid < 32u && next < " << NT << ") fill(psi, sm, bar, nfill, next, s, tid);\n"
          << "  }\n"
          << "  __syncthreads();\n"
          << "  // copies a group that gave up did not consume complete before the CTA leaves\n"
          << "  if (tx == 0u)\n"
          << "    for (u32 i = 0; i < 3u; ++i)\n"
          << "      if (nfill[i] != 0u && !mbar_wait(bar + i, (nfill[i] - 1u) & 1u, " << LIM << ")) *(volatile u32*)status = 2u;\n"
          << "}\n";
        return s.str();
    }

    void emit(const plan::KOp& op)
    {
        using namespace plan;
        if (op.kind < K_GRAD_X || op.kind > K_GRAD_P) qv = false;   // the registers may change
        const int p = op.p;
        const std::string c = cond(op.tcond, op.ocond);
        auto guarded = [&](const std::string& stmt) {
            if (c.empty()) each_state(stmt);
            else {
                o << "  if (" << c << ") {\n";
                each_state("  " + stmt);
                o << "  }\n";
            }
        };
        switch (op.kind) {
        case K_H: each_state("opH<" + std::to_string(p) + ">(@A);"); break;
        case K_X: guarded("opX<" + std::to_string(p) + ", " + std::to_string(op.f) + ">(@A);"); break;
        case K_Y: guarded("opY<" + std::to_string(p) + ", " + std::to_string(op.f) + ">(@A);"); break;
        case K_RX: case K_RY: {
            uint32_t i = push(op.a);
            push(op.b);
            each_state(std::string(op.kind == K_RX ? "opRX<" : "opRY<") + std::to_string(p) + ">(@A, P.v[" +
                       std::to_string(i) + "], P.v[" + std::to_string(i + 1) + "]);");
            break;
        }
        case K_U: {
            uint32_t i = uint32_t(prm.size());
            for (int t = 0; t < 8; ++t) push(P.mats[8 * op.g + t]);
            guarded("opU<" + std::to_string(p) + ", " + std::to_string(op.f) + ">(@A, &P.v[" + std::to_string(i) + "]);");
            break;
        }
        case K_ACC_THR:
            o << "  " << (op.tcond ? "if (" + cond(op.tcond, 0) + ") " : std::string());
            if (P.acc_mul) o << "at = cmul(at, gv[" << op.g << "]);\n";
            else o << "at += gv[" << op.g << "].x;\n";
            break;
        case K_ACC_REG:
            o << "  " << (op.tcond ? "if (" + cond(op.tcond, 0) + ") " : std::string());
            if (P.acc_mul) o << "ar" << p << " = cmul(ar" << p << ", gv[" << op.g << "]);\n";
            else o << "ar" << p << " += gv[" << op.g << "].x;\n";
            break;
        case K_PHD: {
            std::string t = op.tcond ? "if (" + cond(op.tcond, 0) + ") " : std::string();
            o << "  " << t << "{ const double2 e = gv[" << op.g << "];";
            for (int s = 0; s < ns; ++s) o << " phD<" << int(op.f) << ">(" << (s ? "a1" : "a0") << ", e);";
            o << " }\n";
            break;
        }
        case K_FLUSH_REG: emit_flush_reg(p); break;
        case K_FLUSH_ALL: {
            for (uint32_t r = 0; r < P.rb; ++r)
                if ((op.f >> r) & 1) emit_flush_reg(int(r));
            const bool unit = op.a == 1.0 && op.b == 0.0;
            if (P.acc_mul) {
                if (unit) {
                    o << "  if (notOne(at)) { const double2 e = at; at = make_double2(1.0, 0.0);";
                } else {
                    uint32_t i = push(op.a);
                    push(op.b);
                    o << "  { const double2 e = cmul(make_double2(P.v[" << i << "], P.v[" << i + 1
                      << "]), at); at = make_double2(1.0, 0.0);";
                }
            } else if (unit) {
                o << "  if (at != 0.0) { const double2 e = expi(at); at = 0.0;";
            } else {
                uint32_t i = push(op.a);
                push(op.b);
                o << "  { double2 e = make_double2(P.v[" << i << "], P.v[" << i + 1 << "]);"
                  << " if (at != 0.0) { e = cmul(e, expi(at)); at = 0.0; }";
            }
            for (int s = 0; s < ns; ++s) o << " scaleAll(" << (s ? "a1" : "a0") << ", e);";
            o << " }\n";
            break;
        }
        case K_TRANSPOSE: {
            const LayoutRec& nl = P.layouts[op.g];
            o << "  {\n    const u32 sw = " << slot_expr(nl) << ";\n";
            uint32_t woff[32];
            for (uint32_t j = 0; j < R; ++j) woff[j] = slot_off(nl, j);
            set_layout(nl);
            o << "    const u32 sr = " << slot_expr(nl) << ";\n";
            for (int s = 0; s < ns; ++s) {
                const char* A = s ? "a1" : "a0";
                // the first exchange of a pass follows the prologue's barrier: nobody reads xb yet
                if (xb_used) o << "    " << SYNC << "\n";
                xb_used = true;
                for (uint32_t j = 0; j < R; ++j) o << "    xb[sw ^ " << woff[j] << "u] = " << A << "[" << j << "];\n";
                o << "    " << SYNC << "\n";
                for (uint32_t j = 0; j < R; ++j)
                    o << "    " << A << "[" << j << "] = xb[sr ^ " << slot_off(nl, j) << "u];\n";
            }
            o << "    gb = " << gbase_expr() << ";\n  }\n";
            break;
        }
        case K_GRAD_X: case K_GRAD_Y: case K_GRAD_Z: case K_GRAD_P: emit_grad(op, false); break;
        default: break;
        }
    }

    // One gradient occurrence.  cached: phase generators read the per-register
    // Im(conj(l) s) in qz (taken while diagonal phases are still pending).
    void emit_grad(const plan::KOp& op, bool cached)
    {
        using namespace plan;
        if (ns != 2) return;
        const int p = op.p;
        const std::string c = cond(op.tcond, op.ocond);
        {
            std::string expr;
            if (op.kind == K_GRAD_X) expr = "gradX<" + std::to_string(p) + ">(a0, a1)";
            else if (op.kind == K_GRAD_Y) expr = "gradY<" + std::to_string(p) + ">(a0, a1)";
            else if (op.kind == K_GRAD_Z) {
                expr = std::string(cached ? "gradZq<" : "gradZ<") + std::to_string(p < int(P.rb) ? p : -1) +
                       (cached ? ">(qz)" : ">(a0, a1)");
                std::string sg;
                if (op.tcond) sg += "((tid & " + std::to_string(op.tcond) + "u) != 0u)";
                if (op.ocond) sg += std::string(sg.empty() ? "" : " != ") + "((ob & " + hex(op.ocond) + ") != 0ull)";
                if (!sg.empty()) expr = "((" + sg + ") ? -" + expr + " : " + expr + ")";
            } else {
                expr = std::string(cached ? "gradPq<" : "gradP<") + std::to_string(int(op.f)) +
                       (cached ? ">(qz)" : ">(a0, a1)");
                if (!c.empty()) expr = "((" + c + ") ? " + expr + " : 0.0)";
            }
            const uint32_t si = push(op.a);
            // the first kRegSlots slots of a pass accumulate in registers (one
            // warp reduction per slot at the end of the pass instead of one per
            // gate occurrence); further slots reduce immediately
            auto it = gacc.find(op.g);
            if (it == gacc.end() && gacc.size() < kRegSlots) it = gacc.emplace(op.g, uint32_t(gacc.size())).first;
            if (it != gacc.end())
                o << "  gs" << it->second << " += " << expr << " * P.v[" << si << "];\n";
            else
                o << "  { const double v = warpSum<" << T << ">(" << expr << " * P.v[" << si << "]);"
                  << " if ((tid & 31u) == 0u) wp[" << op.g << "u * " << NW << "u + (tid >> 5)] += v; }\n";
        }
    }
};

std::mutex g_mu;
std::map<std::string, std::shared_ptr<Kernel>> g_cache;

std::string compile_to_cubin(const std::string& src, std::string& err)
{
    Nvrtc& nv = nvrtc();
    nvrtcProgram prog;
    if (nv.create(&prog, src.c_str(), "qse_pass.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS) {
        err = "nvrtcCreateProgram failed";
        return {};
    }
    const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "-default-device", "--restrict"};
    nvrtcResult r = nv.compile(prog, 4, opts);
    if (r != NVRTC_SUCCESS) {
        size_t n = 0;
        nv.log_size(prog, &n);
        std::string log(n, '\0');
        if (n) nv.log(prog, &log[0]);
        err = std::string("NVRTC: ") + nv.err(r) + "\n" + log;
        nv.destroy(&prog);
        return {};
    }
    size_t n = 0;
    nv.cubin_size(prog, &n);
    std::string bin(n, '\0');
    nv.cubin(prog, &bin[0]);
    nv.destroy(&prog);
    return bin;
}

}  // namespace

size_t compile_only(const Source& s)
{
    if (!available(nullptr)) fail(QSE_ERR_UNSUPPORTED, "NVRTC unavailable: " + nvrtc().why);
    std::string err;
    std::string bin = compile_to_cubin(s.code, err);
    if (bin.empty()) fail(QSE_ERR_CUDA, "pass kernel compilation failed: " + err);
    return bin.size();
}

bool available(std::string* why)
{
    Nvrtc& nv = nvrtc();
    if (!nv.ok && why) *why = nv.why;
    return nv.ok;
}

static bool streamable(const plan::PassProgram& p, int nstates, bool basis_input)
{
    // forward read+write passes over many tiles whose pieces are at least 128 bytes
    return nstates == 1 && !basis_input && p.k == 12 && p.rb == 4 && Gen::contiguous_low_bits(p) >= 3 &&
           __builtin_popcountll(p.outer_mask) >= 10;
}

Source generate(const plan::PassProgram& p, int nstates, bool basis_input, bool streamed, bool precomputed_groups,
                uint64_t compact_mask, const uint8_t* prob_lpos, uint64_t product_mask)
{
    const char* dbg_env = std::getenv("QSE_DEBUG_BOUNDS");
    const bool dbg = dbg_env && *dbg_env && std::strcmp(dbg_env, "0") != 0;
    if (streamed && !dbg && !prob_lpos && streamable(p, nstates, basis_input)) {
        Gen g(p, nstates, false);
        Source s;
        s.code = g.run_streamed();
        if (g.streamed_smem() <= kStreamedSmemMax) {
            s.prm = std::move(g.prm);
            s.threads = 2 * g.T;
            s.smem = g.streamed_smem();
            s.streamed = true;
            return s;
        }
    }
    Gen g(p, nstates, basis_input, precomputed_groups, compact_mask);
    g.pmask = g.umask ? product_mask : 0;
    g.dbg = dbg;
    // (not with a tile that stores zeros and returns early: a basis input with outer bits)
    if (prob_lpos && nstates == 1 && !(g.zero_in && (p.outer_mask & ~g.umask & ~g.pmask) != 0))
        g.lpos.assign(prob_lpos, prob_lpos + 64);
    Source s;
    s.code = g.run();
    s.prm = std::move(g.prm);
    s.basis_slot = g.basis_slot;
    s.pre_gv = g.pre_gv;
    s.gv_lo = g.gv_lo;
    s.name = g.kernel_name();
    s.prob = !g.lpos.empty();
    s.prob_bsum = g.prob_bsum;
    s.ngroups = uint32_t(p.groups.size());
    s.threads = g.T;
    s.smem = (size_t(1) << p.k) * 16 + p.groups.size() * 16 + size_t(g.ntab) * 32 * 16 +
             (nstates == 2 ? p.slot_src.size() * g.NW * 8 : 0) + (g.preg ? size_t(g.R) * 16 : 0);
    return s;
}

size_t count_uncached(const std::vector<Source>& srcs)
{
    std::lock_guard<std::mutex> lk(g_mu);
    std::unordered_set<std::string_view> seen;
    size_t n = 0;
    for (const Source& s : srcs)
        if (g_cache.find(s.code) == g_cache.end() && seen.insert(s.code).second) ++n;
    return n;
}

std::vector<std::shared_ptr<Kernel>> get_kernels(const std::vector<const Source*>& srcs)
{
    std::vector<std::shared_ptr<Kernel>> out(srcs.size());
    std::vector<size_t> missing;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        for (size_t i = 0; i < srcs.size(); ++i) {
            auto it = g_cache.find(srcs[i]->code);
            if (it != g_cache.end()) out[i] = it->second;
            else missing.push_back(i);
        }
    }
    if (missing.empty()) return out;
    if (!available(nullptr)) fail(QSE_ERR_UNSUPPORTED, "NVRTC unavailable: " + nvrtc().why);
    // distinct sources only, compiled in parallel
    std::map<std::string, size_t> uniq;
    std::vector<size_t> todo;
    for (size_t i : missing)
        if (uniq.emplace(srcs[i]->code, i).second) todo.push_back(i);
    std::vector<std::string> bins(todo.size()), errs(todo.size());
    const size_t nth = std::min<size_t>(todo.size(), std::max(1u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    std::atomic<size_t> next{0};
    for (size_t t = 0; t < nth; ++t)
        pool.emplace_back([&] {
            for (size_t w; (w = next.fetch_add(1)) < todo.size();) bins[w] = compile_to_cubin(srcs[todo[w]]->code, errs[w]);
        });
    for (auto& th : pool) th.join();
    // QSE_JIT_DUMP=<directory>: every source compiled is also written there
    // (<entry point>_<hash of the source>.cu), for reading the generated kernels
    if (const char* dir = std::getenv("QSE_JIT_DUMP"); dir && *dir)
        for (size_t i : todo) {
            char name[64];
            std::snprintf(name, sizeof(name), "_%016zx.cu", std::hash<std::string>{}(srcs[i]->code));
            if (FILE* f = std::fopen((std::string(dir) + "/" + srcs[i]->name + name).c_str(), "w")) {
                std::fwrite(srcs[i]->code.data(), 1, srcs[i]->code.size(), f);
                std::fclose(f);
            }
        }
    std::lock_guard<std::mutex> lk(g_mu);
    for (size_t w = 0; w < todo.size(); ++w) {
        if (bins[w].empty()) fail(QSE_ERR_CUDA, "pass kernel compilation failed: " + errs[w]);
        auto k = std::make_shared<Kernel>();
        QSE_CUDA(cudaLibraryLoadData(&k->lib, bins[w].data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
        QSE_CUDA(cudaLibraryGetKernel(&k->kern, k->lib, srcs[todo[w]]->name.c_str()));
        k->threads = srcs[todo[w]]->threads;
        g_cache[srcs[todo[w]]->code] = k;
    }
    for (size_t i : missing) out[i] = g_cache[srcs[i]->code];
    return out;
}

void launch(qse_ctx* ctx, Kernel& k, const Source& s, uint32_t n, uint32_t kq, void* psi, void* lam,
            const void* terms, const void* groups, double* slot_partial, uint64_t basis_index, const void* gvt)
{
    unsigned* status = ctx->status_dev;
    if (s.smem > ctx->smem_optin) fail(QSE_ERR_SIZE, "pass needs more shared memory than the device offers");
    if (s.smem > k.smem_set) {
        QSE_CUDA(cudaFuncSetAttribute(reinterpret_cast<const void*>(k.kern), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(s.smem)));
        k.smem_set = s.smem;
    }
    std::vector<double> prm = s.prm;
    if (s.basis_slot >= 0) prm[size_t(s.basis_slot)] = double(basis_index);   // exact below 2^53
    if (prm.empty()) prm.push_back(0.0);
    void* args[] = {&psi, &lam, const_cast<const void**>(&terms), const_cast<const void**>(&groups), &slot_partial,
                    &status, const_cast<const void**>(&gvt), prm.data()};
    // streamed passes: one persistent CTA per SM; otherwise one CTA per tile
    const uint64_t tiles = uint64_t(1) << (n - kq);
    const uint64_t grid = s.streamed ? std::min<uint64_t>(tiles, uint64_t(ctx->num_sms)) : tiles;
    QSE_CUDA(cudaLaunchKernel(reinterpret_cast<const void*>(k.kern), dim3(unsigned(grid)), dim3(k.threads), args,
                              s.smem, ctx->stream));
}

}  // namespace jit
}  // namespace qse
