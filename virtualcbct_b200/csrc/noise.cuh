// noise.cuh -- counter-based Gaussian detector noise.
//
// Random numbers come from Philox-4x32-10 (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC 2011), keyed by a
// 64-bit seed and counted by the pixel's global index, so a pixel's draw
// does not depend on the launch shape or on the other pixels; normals by
// the Box-Muller transform.
#pragma once
#include <cstdint>

namespace vcbct {

__host__ __device__ __forceinline__ void philox_round(uint32_t (&c)[4], uint32_t k0, uint32_t k1)
{
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
}

// Philox-4x32 with 10 rounds: counter c (4 words), key (k0, k1).
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t (&c)[4], uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; r++) {
        philox_round(c, k0, k1);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// Four 32-bit random words for counter (ctr_lo, ctr_hi, stream_id, 0) under
// key `seed`.
__host__ __device__ __forceinline__ void philox4x32(uint64_t ctr, uint32_t stream_id, uint64_t seed,
                                                    uint32_t (&out)[4])
{
    uint32_t c[4] = {(uint32_t)ctr, (uint32_t)(ctr >> 32), stream_id, 0u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    out[0] = c[0];
    out[1] = c[1];
    out[2] = c[2];
    out[3] = c[3];
}

// A standard normal draw for pixel `index` (double precision Box-Muller on
// two 32-bit uniforms in (0, 1)).
__device__ __forceinline__ double normal_draw(uint64_t index, uint32_t stream_id, uint64_t seed)
{
    uint32_t w[4];
    philox4x32(index, stream_id, seed, w);
    const double u1 = ((double)w[0] + 0.5) * 2.3283064365386963e-10;  // 2^-32
    const double u2 = ((double)w[1] + 0.5) * 2.3283064365386963e-10;
    return sqrt(-2.0 * log(u1)) * sinpi(2.0 * u2);
}

// Detector counts of an intensity, with Gaussian noise of the count's
// square-root width (the reference's model, prior_weight_production.cpp:24-38,
// in count units): n = i0 * I, n' = n + sqrt(n) z, clamped to [0, max_counts];
// returns n' / i0.
__device__ __forceinline__ float noisy_intensity(float I, double i0, double max_counts, uint64_t index,
                                                 uint64_t seed)
{
    const double n = i0 * (double)I;
    double m = n + sqrt(n > 0.0 ? n : 0.0) * normal_draw(index, 0u, seed);
    if (m < 0.0) m = 0.0;
    if (m > max_counts) m = max_counts;
    return (float)(m / i0);
}

}  // namespace vcbct
