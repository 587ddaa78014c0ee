// noise.cuh -- counter-based Gaussian detector noise.
//
// Random numbers come from Philox-4x32-10 (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC 2011), keyed by a
// 64-bit seed and counted by the pixel's global index, so a pixel's draw
// does not depend on the launch shape or on the other pixels; normals by
// the Box-Muller transform in single precision (noise of a count n has width
// sqrt(n), so float's 1e-7 relative rounding is far below it).
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

// Box-Muller on two 32-bit random words, in single precision with the fast
// hardware logarithm and sine/cosine: two independent standard normals.  The
// uniforms take the words' top 23 bits (u1 in (0, 1], so the radius is
// finite; u2's angle centred on zero, where the fast sine/cosine are
// accurate to ~1e-6 absolute, far below what noise statistics can see).
__device__ __forceinline__ float2 box_muller(uint32_t a, uint32_t b)
{
    const float u1 = 2.0f - __uint_as_float(0x3f800000u | (a >> 9));        // (0, 1]
    const float u2 = __uint_as_float(0x3f800000u | (b >> 9)) - 1.5f;        // [-0.5, 0.5)
    const float r = sqrtf(-2.0f * __logf(u1));
    float s, c;
    __sincosf(6.283185307179586f * u2, &s, &c);
    return make_float2(r * c, r * s);
}

// Four standard normals for pixels 4q .. 4q + 3 from one counter draw:
// words 0, 1 give pixels 4q (cosine) and 4q + 1 (sine), words 2, 3 pixels
// 4q + 2 and 4q + 3.
__device__ __forceinline__ float4 normal_quad(uint64_t q, uint32_t stream_id, uint64_t seed)
{
    uint32_t w[4];
    philox4x32(q, stream_id, seed, w);
    const float2 a = box_muller(w[0], w[1]), b = box_muller(w[2], w[3]);
    return make_float4(a.x, a.y, b.x, b.y);
}

// The standard normal of pixel `index` (its part of its quad's draw, with
// only its own Box-Muller pair evaluated).
__device__ __forceinline__ float normal_draw(uint64_t index, uint32_t stream_id, uint64_t seed)
{
    uint32_t w[4];
    philox4x32(index >> 2, stream_id, seed, w);
    const bool hi = (index & 2) != 0;
    const float2 z = box_muller(hi ? w[2] : w[0], hi ? w[3] : w[1]);
    return (index & 1) ? z.y : z.x;
}

// Detector counts of an intensity, with Gaussian noise of the count's
// square-root width (the reference's model, prior_weight_production.cpp:24-38,
// in count units): n = i0 * I, n' = n + sqrt(n) z, clamped to [0, max_counts];
// returns n' / i0.
__device__ __forceinline__ float noisy_intensity(float I, float i0, float max_counts, uint64_t index,
                                                 uint64_t seed)
{
    const float n = i0 * I;
    float m = n + sqrtf(n > 0.0f ? n : 0.0f) * normal_draw(index, 0u, seed);
    if (m < 0.0f) m = 0.0f;
    if (m > max_counts) m = max_counts;
    return m / i0;
}

// Counter draw for the Poisson sampler: word 3 of the counter numbers the
// draws a pixel consumes.
__device__ __forceinline__ void philox4x32_nth(uint64_t ctr, uint32_t stream_id, uint32_t nth, uint64_t seed,
                                               uint32_t (&out)[4])
{
    uint32_t c[4] = {(uint32_t)ctr, (uint32_t)(ctr >> 32), stream_id, nth};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    out[0] = c[0];
    out[1] = c[1];
    out[2] = c[2];
    out[3] = c[3];
}

__device__ __forceinline__ double unit_open(uint32_t w)  // (0, 1)
{
    return ((double)w + 0.5) * 2.3283064365386963e-10;
}

// A Poisson(lam) count for pixel `index`.  lam < 10: multiplication of
// uniforms until the product falls below exp(-lam) (Knuth); lam >= 10: the
// transformed rejection method PTRS (W. Hormann, "The transformed rejection
// method for generating Poisson random variables", Insurance: Mathematics
// and Economics 12, 1993), two trials per counter draw.  Both loops are
// bounded (128 uniforms; 64 trials, acceptance ~0.9 each); past the bound,
// which no realistic draw reaches, the normal approximation is returned.
__device__ __forceinline__ double poisson_count(double lam, uint64_t index, uint64_t seed)
{
    if (!(lam > 0.0)) return 0.0;
    uint32_t w[4];
    if (lam < 10.0) {
        const double lim = exp(-lam);
        double prod = 1.0;
        for (int n = 0; n < 128; n++) {
            if ((n & 3) == 0) philox4x32_nth(index, 2u, (uint32_t)(n >> 2), seed, w);
            prod *= unit_open(w[n & 3]);
            if (prod <= lim) return (double)n;
        }
    } else {
        const double sl = sqrt(lam), ll = log(lam);
        const double b = 0.931 + 2.53 * sl, a = -0.059 + 0.02483 * b;
        const double log_inv_alpha = log(1.1239 + 1.1328 / (b - 3.4)), vr = 0.9277 - 3.6224 / (b - 2.0);
        for (int t = 0; t < 64; t++) {
            if ((t & 1) == 0) philox4x32_nth(index, 2u, (uint32_t)(t >> 1), seed, w);
            const double u = unit_open(w[2 * (t & 1)]) - 0.5, v = unit_open(w[2 * (t & 1) + 1]);
            const double us = 0.5 - fabs(u);
            const double k = floor((2.0 * a / us + b) * u + lam + 0.43);
            if (us >= 0.07 && v <= vr) return k;
            if (k < 0.0 || (us < 0.013 && v > us)) continue;
            if (log(v) + log_inv_alpha - log(a / (us * us) + b) <= -lam + k * ll - lgamma(k + 1.0)) return k;
        }
    }
    return fmax(0.0, rint(lam + sqrt(lam) * (double)normal_draw(index, 3u, seed)));
}

// Poisson detector counts of an intensity: n = i0 * I expected counts, a
// Poisson(n) draw clamped to [0, max_counts]; returns it / i0.
__device__ __forceinline__ float poisson_intensity(float I, double i0, double max_counts, uint64_t index,
                                                   uint64_t seed)
{
    const double m = fmin(poisson_count(i0 * (double)I, index, seed), max_counts);
    return (float)(m / i0);
}

}  // namespace vcbct
