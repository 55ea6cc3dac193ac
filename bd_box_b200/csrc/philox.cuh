// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) and the Box-Muller
// transform: the device Gaussian stream of the engine, keyed by the seed,
// counter = (pair index, stream index). Shared by k_noise (noise.cu) and the
// stored-matrix product that draws its noise itself (matvec.cu), so that both
// produce the same bits.
#pragma once
#include <cstdint>

namespace bdb {

__device__ __forceinline__ void philox_round(uint32_t* c, const uint32_t* k)
{
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t hi0 = __umulhi(M0, c[0]), lo0 = M0 * c[0];
    const uint32_t hi1 = __umulhi(M1, c[2]), lo1 = M1 * c[2];
    const uint32_t n0 = hi1 ^ c[1] ^ k[0];
    const uint32_t n2 = hi0 ^ c[3] ^ k[1];
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
}

__device__ __forceinline__ void philox4x32_10(uint32_t* c, uint32_t k0, uint32_t k1)
{
    uint32_t k[2] = {k0, k1};
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        philox_round(c, k);
        k[0] += 0x9E3779B9u;
        k[1] += 0xBB67AE85u;
    }
}

// two unit Gaussians for (stream, index)
__device__ __forceinline__ void gauss2(uint64_t seed, uint64_t stream, uint32_t idx, double& z0, double& z1)
{
    uint32_t c[4] = {idx, (uint32_t)stream, (uint32_t)(stream >> 32), 0x42444242u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const double two53 = 9007199254740992.0;
    const double u0 = ((double)(c[0] >> 5) * 67108864.0 + (double)(c[1] >> 6) + 0.5) / two53;   // (0,1)
    const double u1 = ((double)(c[2] >> 5) * 67108864.0 + (double)(c[3] >> 6)) / two53;         // [0,1)
    const double r = sqrt(-2.0 * log(u0));
    double sn, cs;
    sincospi(2.0 * u1, &sn, &cs);
    z0 = r * cs;
    z1 = r * sn;
}

}  // namespace bdb
