// philox.cuh -- Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC'11), written from the published round
// function: two 32x32->64 multiplies per round with M0 = 0xD2511F53,
// M1 = 0xCD9E8D57, Weyl key bumps W0 = 0x9E3779B9, W1 = 0xBB67AE85, 10 rounds.
#pragma once
#include <cstdint>

namespace qse {

struct Philox4 {
    uint32_t w[4];
};

__host__ __device__ __forceinline__ Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                          uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint64_t p0 = uint64_t(0xD2511F53u) * c0;
        uint64_t p1 = uint64_t(0xCD9E8D57u) * c2;
        uint32_t n0 = uint32_t(p1 >> 32) ^ c1 ^ k0;
        uint32_t n2 = uint32_t(p0 >> 32) ^ c3 ^ k1;
        c1 = uint32_t(p1);
        c3 = uint32_t(p0);
        c0 = n0;
        c2 = n2;
    }
    return Philox4{{c0, c1, c2, c3}};
}

// Stream tags in counter word 2 keep the noise and sampling streams apart.
constexpr uint32_t kTagNoise = 0x4E4F4953u;   // "NOIS"
constexpr uint32_t kTagSample = 0x53414D50u;  // "SAMP"

// Two 53-bit uniforms in [0,1) from one block: (w1:w0) >> 11 and (w3:w2) >> 11.
__host__ __device__ __forceinline__ void philox_uniform_pair(uint64_t seed, uint64_t counter, uint32_t tag, double& u1,
                                                             double& u2)
{
    Philox4 r = philox4x32_10(uint32_t(counter), uint32_t(counter >> 32), tag, 0u, uint32_t(seed),
                              uint32_t(seed >> 32));
    uint64_t a = (uint64_t(r.w[1]) << 32) | r.w[0];
    uint64_t b = (uint64_t(r.w[3]) << 32) | r.w[2];
    u1 = double(a >> 11) * 0x1.0p-53;
    u2 = double(b >> 11) * 0x1.0p-53;
}

}  // namespace qse
