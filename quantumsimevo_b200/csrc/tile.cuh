// tile.cuh -- launch interface of the fused tile kernel (tile.cu).
#pragma once

#include <cuda_runtime.h>

#include "planner.h"
#include "qse_internal.h"

namespace qse {
namespace tile {

struct PassArgs {
    double2* psi;                        // state (physical order)
    double2* lam;                        // second state for the adjoint sweep (NS == 2)
    const plan::KOp* ops;
    const plan::LayoutRec* layouts;
    const plan::TermRec* terms;
    const plan::GroupRec* groups;
    const double* mats;
    double* slot_partial;                // [nslots][grid] gradient partial sums (NS == 2)
    uint64_t outer_mask;
    uint32_t nops;
    uint32_t ngroups;
    uint32_t nslots;
    uint32_t layout0;
    uint32_t k;
    uint32_t pad;
    uint8_t tile_phys[16];
};

// Launch one pass: grid = 2^(n-k) CTAs of 2^(k-rb) threads.
void launch_pass(qse_ctx* ctx, const PassArgs& a, uint32_t n, uint32_t rb, int nstates);
size_t pass_smem_bytes(uint32_t k, uint32_t ngroups, uint32_t nslots, uint32_t rb, int nstates);
// events bracketing one pass launch when qse_ctx_time_passes is on (else no-ops)
cudaEvent_t pass_timer_begin(qse_ctx* ctx);
void pass_timer_end(qse_ctx* ctx, cudaEvent_t stop);

}  // namespace tile
}  // namespace qse
