// noise.cu -- device Pauli noise (Noise.cpp).
//
// Noise::accumulateError (Noise.cpp:21-32) draws two uniforms for every gate
// whose type is in the error-rate map, in program order, before the gate:
// u1 < p adds a bit flip to the gate's target, u2 < p a phase flip.  The
// decisions depend only on the gate list and the draws, never on the state, so
// all of them are taken at once: one thread per noisy gate, counts summed
// with atomics.  The draws come from Philox4x32-10 keyed by the seed with the
// noisy-gate index as counter (so the stream continues across executes like
// the reference's mt19937), or from the host (mt19937 or caller-injected).
// Noise::applyPauliNoise (Noise.cpp:34-44) is the one-pass Pauli frame kernel
// in gates.cu.
#include <cuda_runtime.h>

#include "philox.cuh"
#include "qse_internal.h"

namespace qse {
namespace {

__global__ void k_noise_decide(const int32_t* __restrict__ types, const uint32_t* __restrict__ targets,
                               uint64_t ngates, const double* __restrict__ rates, double mult, int mode,
                               uint64_t seed, uint64_t draw0, const double* __restrict__ u, int32_t* counts)
{
    for (uint64_t g = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; g < ngates;
         g += uint64_t(gridDim.x) * blockDim.x) {
        const double p = rates[types[g]] * mult;
        double u1, u2;
        if (mode == QSE_RNG_PHILOX) {
            philox_uniform_pair(seed, draw0 + g, kTagNoise, u1, u2);
        } else {
            u1 = u[2 * g];
            u2 = u[2 * g + 1];
        }
        const uint32_t t = targets[g];
        if (u1 < p) atomicAdd(&counts[t], 1);
        if (u2 < p) atomicAdd(&counts[64 + t], 1);
    }
}

}  // namespace

void noise_decide(qse_noise* nz, const int32_t* d_types, const uint32_t* d_targets, size_t ngates,
                  const double* d_uniforms)
{
    if (ngates == 0) return;
    qse_ctx* ctx = nz->ctx;
    unsigned grid = unsigned(std::min<uint64_t>((ngates + 255) / 256, uint64_t(ctx->num_sms) * 4));
    const double* d_rates = reinterpret_cast<const double*>(nz->d_counts + 128);
    k_noise_decide<<<grid, 256, 0, ctx->stream>>>(d_types, d_targets, ngates, d_rates, nz->cfg.multiplier,
                                                  nz->cfg.rng_mode, nz->cfg.seed, nz->draws, d_uniforms,
                                                  nz->d_counts);
    QSE_CUDA(cudaGetLastError());
    count_launch(ctx);
    nz->draws += ngates;
}

}  // namespace qse
