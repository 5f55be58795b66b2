// jit.h -- per-pass kernel specialisation with NVRTC (jit.cpp).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <memory>
#include <string>
#include <vector>

#include "planner.h"
#include "qse_internal.h"

namespace qse {
namespace jit {

struct Source {
    std::string code;         // CUDA C++ of the pass kernel (angles not included)
    std::string name = "qse_pass";   // its entry point (qse_pass, qse_pass_basis_in, qse_pass_compact_in, qse_pass_adjoint)
    bool prob = false;               // writes the probability side output (prob_lpos)
    bool prob_bsum = false;          // ... with its 4096-block sums
    std::vector<double> prm;  // the kernel's parameter block (angles, matrices, scales)
    uint32_t threads = 0;
    size_t smem = 0;
    int basis_slot = -1;      // basis-input passes: the prm slot that takes the basis index
    bool streamed = false;    // persistent streamed kernel (grid = SM count) instead of one CTA per tile
    bool pre_gv = false;      // the per-CTA group values are read from a precomputed table (gvt)
    uint32_t ngroups = 0;     // diagonal groups of the pass (the table's row length)
    // pre_gv with gv_lo > 0: every term's outer condition lies in the lowest
    // gv_lo outer qubits or in the others, so the table is two tables: one row
    // per value of the low gv_lo CTA-index bits, then one per value of the
    // other bits (terms without a condition in the first only); a CTA's value
    // is the product (direct groups) or the sum (angle groups) of its two rows'
    uint32_t gv_lo = 0;
};

// States of at least this many qubits run their passes with the group values
// precomputed per tile (the table costs one small kernel and 16 B per group and
// tile; on small states the in-kernel prologue is cheaper than a launch)
constexpr uint32_t kPreGroupQubits = 22;

// dynamic shared memory a streamed pass may use (227 KiB per CTA on sm_100)
constexpr size_t kStreamedSmemMax = 227 * 1024;

struct Kernel {
    cudaLibrary_t lib = nullptr;
    cudaKernel_t kern = nullptr;
    uint32_t threads = 0;
    size_t smem_set = 48 * 1024;
};

bool available(std::string* why);
// compiles one source without loading it (no GPU needed); returns the cubin size
size_t compile_only(const Source& s);
// basis_input: the state is a basis state |i> that is not in memory; the pass
// generates its input amplitudes instead of loading them (forward passes only;
// i is set per launch, so one kernel serves every i)
// streamed: use the persistent streamed kernel when the pass allows it (forward
// read+write passes of 12 tile qubits over at least 2^10 tiles, pieces of at
// least 8 contiguous amplitudes); otherwise one CTA per tile
// precomputed_groups: the pass reads its per-CTA diagonal group values from a
// table computed beforehand (k_group_values: one row of ngroups values per
// tile) instead of computing them in a prologue; not for plain basis-input
// passes (their tiles but one store zeros)
// compact_mask (with basis_input): the input is a compact state on the
// physical qubits of the mask (passed as `lam` at launch, indexed by those
// bits in ascending order) times the basis bits of i on the other qubits
// prob_lpos (forward passes): the pass also writes the probabilities of the
// amplitudes it stores in logical order and their 4096-block sums (passed as
// `slot_partial` at launch: 2^n doubles, then 2^n / 4096 sums, zeroed before);
// prob_lpos[q] = logical position of physical qubit q after the pass
// product_mask (with compact_mask): physical qubits outside the compact state
// that hold a single-qubit state each, whose two amplitudes (the i-th lowest
// qubit's at lam[2^popcount(compact_mask) + 2i + bit]) multiply the input
Source generate(const plan::PassProgram& p, int nstates, bool basis_input = false, bool streamed = false,
                bool precomputed_groups = false, uint64_t compact_mask = 0, const uint8_t* prob_lpos = nullptr,
                uint64_t product_mask = 0);
// distinct sources among srcs that are not compiled yet
size_t count_uncached(const std::vector<Source>& srcs);
// compiled kernels for every source (cached by source text; missing ones are compiled in parallel)
std::vector<std::shared_ptr<Kernel>> get_kernels(const std::vector<const Source*>& srcs);
// basis_index: the physical index of a basis-input pass's input state (ignored otherwise)
void launch(qse_ctx* ctx, Kernel& k, const Source& s, uint32_t n, uint32_t kq, void* psi, void* lam,
            const void* terms, const void* groups, double* slot_partial, uint64_t basis_index = 0,
            const void* gvt = nullptr);

}  // namespace jit
}  // namespace qse
