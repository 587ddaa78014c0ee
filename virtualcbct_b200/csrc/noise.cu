// noise.cu -- the reference's Gaussian detector noise (gaussiannoise,
// Release_CBCT_Projection_CM/prior_weight_production.cpp:24-38) on device
// projections in its units (value = MAX_PIXVALUE - counts): per pixel,
// n = max - p, n += N(0, sqrt(n)), p = max - n clamped to [0, max].  The
// reference draws its normals from one rand() stream in pixel order; here
// each pixel has its own counter-based draw (noise.cuh), so the result is
// the same distribution, reproducible for a seed and independent of the
// launch shape.  Computed in single precision: the noise of a count n has
// width sqrt(n), far above float's rounding of values up to 65535.
#include "internal.h"
#include "noise.cuh"

namespace vcbct {
namespace {

__device__ __forceinline__ float ref_unit_noise(float p, float maxv, float z)
{
    float nstar = maxv - p;
    // sqrt(n) from the reciprocal square root (within 2 ulp; NaN for n < 0
    // as the reference's sqrt gives)
    const float sigma = nstar == 0.0f ? 0.0f : nstar * rsqrtf(nstar);
    nstar = nstar + sigma * z;
    float v = maxv - nstar;
    if (maxv - nstar < 0.0f) v = 0.0f;
    if (maxv - nstar > maxv) v = maxv;
    return v;
}

// One thread per four pixels (one counter draw, four normals); VEC when
// the stack is 16-byte aligned.
template <bool VEC>
__global__ void gaussian_noise_kernel(float* __restrict__ p, size_t n, float maxv, unsigned long long seed)
{
    const size_t nq = (n + 3) / 4;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += (size_t)gridDim.x * blockDim.x) {
        const float4 z = normal_quad(q, 1u, seed);
        const size_t i = 4 * q;
        if (VEC && i + 4 <= n) {  // one 16-byte load and store per quad
            float4 v = *reinterpret_cast<const float4*>(p + i);
            v.x = ref_unit_noise(v.x, maxv, z.x);
            v.y = ref_unit_noise(v.y, maxv, z.y);
            v.z = ref_unit_noise(v.z, maxv, z.z);
            v.w = ref_unit_noise(v.w, maxv, z.w);
            *reinterpret_cast<float4*>(p + i) = v;
        } else {
            const float zz[4] = {z.x, z.y, z.z, z.w};
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (i + k < n) p[i + k] = ref_unit_noise(p[i + k], maxv, zz[k]);
        }
    }
}

}  // namespace

cudaError_t launch_gaussian_noise(float* proj, size_t n, double max_pixvalue, unsigned long long seed,
                                  cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const size_t want = ((n + 3) / 4 + 255) / 256;
    const unsigned blocks = (unsigned)(want < (size_t)sms * 16 ? want : (size_t)sms * 16);
    if ((reinterpret_cast<uintptr_t>(proj) & 15) == 0)
        gaussian_noise_kernel<true><<<blocks, 256, 0, st>>>(proj, n, (float)max_pixvalue, seed);
    else
        gaussian_noise_kernel<false><<<blocks, 256, 0, st>>>(proj, n, (float)max_pixvalue, seed);
    return cudaGetLastError();
}

}  // namespace vcbct

extern "C" void vcbct_philox4x32_10(const uint32_t* ctr, const uint32_t* key, uint32_t* out)
{
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    vcbct::philox4x32_10(c, key[0], key[1]);
    for (int i = 0; i < 4; i++) out[i] = c[i];
}
