// tile.cu -- the fused tile kernel: one launch applies one planned pass
// (planner.cpp) to the whole state with one HBM read and one write per
// amplitude.
//
// CTA c owns the 2^k amplitudes whose outer (non-tile) bits spell c.  Each
// thread holds R = 2^RB of them in registers: the RB "register" tile bits of
// the current layout select the register, the other k-RB tile bits are the
// thread index.  A gate on a register bit is pure register arithmetic; to
// reach other tile bits the CTA exchanges the tile through shared memory
// (K_TRANSPOSE) with an XOR-swizzled slot map that keeps every quarter-warp of
// 16-byte accesses on distinct bank groups.
//
// Diagonal gates never move data.  Their phase terms are summed per CTA in a
// prologue (terms whose outer bits are not all set drop out) and applied per
// thread as accumulated angles (one sincos per flush) or, for terms on two or
// more register bits, as a direct multiply.
//
// NS == 2 runs the adjoint sweep: the same gates are applied to |psi> and
// |lambda>, and K_GRAD_* ops reduce 2 Im<lambda|G|psi> for the generator G of
// the gate about to be undone.
#include "tile.cuh"
#include "tile_dev.cuh"

namespace qse {
namespace tile {
namespace {

using namespace dev;

template <int RB, int NS>
__global__ void __launch_bounds__(256, 2) k_tile(const PassArgs A)
{
    constexpr int R = 1 << RB;
    extern __shared__ double2 smem[];
    const uint32_t tid = threadIdx.x;
    const uint32_t tsize = 1u << A.k;
    double2* xbuf = smem;
    double2* gval = smem + tsize;
    double* wpart = reinterpret_cast<double*>(gval + A.ngroups);
    const uint32_t nwarps = (blockDim.x + 31) >> 5;

    __shared__ uint8_t s_tile[16];
    for (uint32_t i = tid; i < 16; i += blockDim.x) s_tile[i] = A.tile_phys[i];

    const uint64_t obase = tile_base(blockIdx.x, A.outer_mask);
    group_values(A.groups, A.ngroups, A.terms, obase, gval);
    if (NS == 2)
        for (uint32_t i = tid; i < A.nslots * nwarps; i += blockDim.x) wpart[i] = 0.0;
    __syncthreads();

    LayoutState<RB> L;
    load_layout<RB>(L, A.layouts + A.layout0, s_tile, A.k, obase, tid);

    double2 a[NS][R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
        uint64_t idx = gidx<RB>(L, j);
        a[0][j] = A.psi[idx];
        if (NS == 2) a[NS - 1][j] = A.lam[idx];
    }

    OpsEnv E{A.ops, A.nops, A.layouts, A.mats, s_tile, A.k, obase, xbuf, gval, wpart, nwarps};
    run_ops<RB, NS>(E, L, a, NS, true);

#pragma unroll
    for (int j = 0; j < R; ++j) {
        uint64_t idx = gidx<RB>(L, j);
        A.psi[idx] = a[0][j];
        if (NS == 2) A.lam[idx] = a[NS - 1][j];
    }
    if (NS == 2) {
        __syncthreads();
        for (uint32_t s = tid; s < A.nslots; s += blockDim.x) {
            double v = 0.0;
            for (uint32_t w = 0; w < nwarps; ++w) v += wpart[s * nwarps + w];
            A.slot_partial[uint64_t(s) * gridDim.x + blockIdx.x] = v;
        }
    }
}

template <int RB, int NS>
void launch_t(qse_ctx* ctx, const PassArgs& a, uint32_t n, size_t smem)
{
    static bool configured[64] = {false};
    int dev = ctx->device;
    if (!configured[dev & 63]) {
        cudaFuncAttributes fa{};
        QSE_CUDA(cudaFuncGetAttributes(&fa, k_tile<RB, NS>));
        QSE_CUDA(cudaFuncSetAttribute(k_tile<RB, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(ctx->smem_optin - fa.sharedSizeBytes)));
        configured[dev & 63] = true;
    }
    uint32_t threads = 1u << (a.k - RB);
    uint64_t grid = uint64_t(1) << (n - a.k);
    cudaEvent_t ev_stop = pass_timer_begin(ctx);
    k_tile<RB, NS><<<unsigned(grid), threads, smem, ctx->stream>>>(a);
    QSE_CUDA(cudaGetLastError());
    pass_timer_end(ctx, ev_stop);
    count_launch(ctx);
}

}  // namespace

cudaEvent_t pass_timer_begin(qse_ctx* ctx)
{
    if (!ctx->time_passes) return nullptr;
    if (ctx->pass_events_used + 2 > ctx->pass_events.size()) {
        for (int i = 0; i < 64; ++i) {
            cudaEvent_t e;
            QSE_CUDA(cudaEventCreate(&e));
            ctx->pass_events.push_back(e);
        }
    }
    QSE_CUDA(cudaEventRecord(ctx->pass_events[ctx->pass_events_used], ctx->stream));
    cudaEvent_t stop = ctx->pass_events[ctx->pass_events_used + 1];
    ctx->pass_events_used += 2;
    return stop;
}

void pass_timer_end(qse_ctx* ctx, cudaEvent_t stop)
{
    if (stop) QSE_CUDA(cudaEventRecord(stop, ctx->stream));
}

size_t pass_smem_bytes(uint32_t k, uint32_t ngroups, uint32_t nslots, uint32_t rb, int nstates)
{
    size_t threads = size_t(1) << (k - rb);
    size_t b = (size_t(1) << k) * 16 + size_t(ngroups) * 16;
    if (nstates == 2) b += size_t(nslots) * ((threads + 31) / 32) * 8;
    return b;
}

void launch_pass(qse_ctx* ctx, const PassArgs& a, uint32_t n, uint32_t rb, int nstates)
{
    size_t smem = pass_smem_bytes(a.k, a.ngroups, a.nslots, rb, nstates);
    if (smem > ctx->smem_optin) fail(QSE_ERR_SIZE, "tile pass needs more shared memory than the device offers");
    if (n - a.k > 31) fail(QSE_ERR_SIZE, "too many tiles for one launch");
    if (rb == 4 && nstates == 1) launch_t<4, 1>(ctx, a, n, smem);
    else if (rb == 3 && nstates == 2) launch_t<3, 2>(ctx, a, n, smem);
    else if (rb == 3 && nstates == 1) launch_t<3, 1>(ctx, a, n, smem);
    else fail(QSE_ERR_INVALID, "unsupported tile configuration");
}

}  // namespace tile
}  // namespace qse
