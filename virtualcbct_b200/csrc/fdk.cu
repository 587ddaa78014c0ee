// fdk.cu -- FDK ramp filter (direct FP32 path) and voxel-driven cone-beam
// backprojection on sm_100a.
//
// Reference: Release_recon_from_forward_pro_float_CM/filterSinogram.cpp:67-131
// and reconstructImage.cpp:10-184 (OpenMP CPU code).
#include "internal.h"

#include <climits>

namespace vcbct {
namespace {

// ------------------------------------------------------------------ filter --
// out[r][m] = Cm(v, n, m) * sum_k hT[k][m] * g[r][k],  g = -logf(p),  r = v*H + n,
// where hT already holds the diagonal coefficient (filterSinogram.cpp:103) and
// the ramp kernel (:106-110).  A 64x64 output tile per block, K tiles of 32;
// each thread computes 4x4 outputs.  -logf is applied while staging the A tile
// (the reference's log of a float is the float overload, :103/:108).
constexpr int FT_M = 64, FT_N = 64, FT_K = 32;

__global__ void __launch_bounds__(256) filter_direct_kernel(
    const float* __restrict__ proj, float* __restrict__ out, const float* __restrict__ hT,
    const FilterView* __restrict__ views, const float* __restrict__ wts, float pitch, float sad,
    int V, int H, int W)
{
    __shared__ float As[FT_K][FT_M + 4];
    __shared__ float Bs[FT_K][FT_N + 4];
    const int M = V * H;
    const int r0 = blockIdx.y * FT_M, c0 = blockIdx.x * FT_N;
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < W; k0 += FT_K) {
        // stage A: 64 rows x 32 k  (g = -logf(p))
        for (int i = threadIdx.x; i < FT_M * FT_K; i += 256) {
            const int rr = i / FT_K, kk = i % FT_K;
            const int r = r0 + rr, k = k0 + kk;
            float g = 0.0f;
            if (r < M && k < W) {
                g = -logf(__ldg(proj + (size_t)r * W + k));
                if (wts) g *= __ldg(wts + (size_t)(r / H) * W + k);
            }
            As[kk][rr] = g;
        }
        // stage B: 32 k x 64 cols of hT
        for (int i = threadIdx.x; i < FT_K * FT_N; i += 256) {
            const int kk = i / FT_N, cc = i % FT_N;
            const int k = k0 + kk, c = c0 + cc;
            Bs[kk][cc] = (k < W && c < W) ? __ldg(hT + (size_t)k * W + c) : 0.0f;
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < FT_K; kk++) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int i = 0; i < 4; i++) b[i] = Bs[kk][tx * 4 + i];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int jn = 0; jn < 4; jn++) acc[i][jn] = fmaf(a[i], b[jn], acc[i][jn]);
        }
        __syncthreads();
    }
    // epilogue: cosine factor Cm = D / sqrt(D^2 + pos1^2 + pos2^2) (:92-99)
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int r = r0 + ty * 4 + i;
        if (r >= M) continue;
        const int v = r / H, n = r - v * H;
        const FilterView sh = views[v];
        const float pos2 = fabsf(sh.ycs + (float)n) * pitch;
#pragma unroll
        for (int jn = 0; jn < 4; jn++) {
            const int m = c0 + tx * 4 + jn;
            if (m >= W) continue;
            const float pos1 = fabsf(sh.xcs + (float)m) * pitch;
            const float cm = sad / sqrtf(sad * sad + pos1 * pos1 + pos2 * pos2);
            out[(size_t)r * W + m] = acc[i][jn] * cm;
        }
    }
}

// ----------------------------------------------------------- backprojection --
// One thread per (x, y) voxel column and a chunk of ZB slices (register
// accumulators).  Per (x, y, view) the detector column coordinate U, its
// interpolation weight and the magnification are formed in FP64 (the floor
// of U decides which two detector columns are read and must agree with the
// reference); per slice the row coordinate ZETA is an exact integer base plus
// an FP32 fractional offset.  Bilinear interpolation is manual FP32 with the
// reference's edge rules and its weight quirk (the column weight is frac(U),
// not frac(UUU), reconstructImage.cpp:80-83).
// Register cap (minimum resident 256-thread blocks per SM) and slices per
// thread.  The gathers are latency-bound, so occupancy pays: with 4 x 8 warp
// tiles, 8 slices at 6 blocks (40 registers, 48 warps per SM) measured on
// B200 as fast as 16 slices at 5 blocks on 270x270x200 from 360 half-fan
// views (3.39 vs 3.37 ms) and 10-19 % faster where more of the volume lies in
// the cone (512x512x400 / x100 from 720 views of 800x800: 55 vs 61 ms, 22 vs
// 27 ms); 12, 20 slices and 16 at 4 blocks were slower.
#ifndef VCBCT_BP_MIN_BLOCKS
#define VCBCT_BP_MIN_BLOCKS 6
#endif
#ifndef VCBCT_BP_TILE
#define VCBCT_BP_TILE 4  // warp tile width in voxel columns (4, 8, 16 or 32)
#endif
#ifndef VCBCT_BP_ZB
#define VCBCT_BP_ZB 8
#endif
template <int ZB>
__global__ void __launch_bounds__(256, VCBCT_BP_MIN_BLOCKS) backproject_kernel(
    FdkParams f, const BpView* __restrict__ views, const float* __restrict__ filt,
    float* __restrict__ vol_f32, short* __restrict__ vol_i16)
{
    // each warp takes a TW x (32 / TW) tile of the block's 32 x 8 columns:
    // the detector's column-edge and cone-edge lines split fewer warps than
    // with 32 x 1 rows, and a warp's taps fall in fewer cache lines (B200,
    // 270x270x200 from 360 half-fan views: 3.35 ms with 4 x 8 tiles, 3.44
    // with 8 x 4, 3.59 with 16 x 2, 3.96 with 32 x 1; the volume is the same)
    constexpr int TW = VCBCT_BP_TILE, TH = 32 / TW, WX = 32 / TW;
    const int x = blockIdx.x * 32 + (threadIdx.y % WX) * TW + (threadIdx.x % TW);
    const int y = blockIdx.y * 8 + (threadIdx.y / WX) * TH + (threadIdx.x / TW);
    const int z0 = blockIdx.z * ZB;
    if (x >= f.N || y >= f.N) return;
    const double R = (double)(f.N - 1) / 2.0;
    const bool inmask = ((double)y - R) * ((double)y - R) + ((double)x - R) * ((double)x - R) <= R * R;
    float acc[ZB];
#pragma unroll
    for (int i = 0; i < ZB; i++) acc[i] = 0.0f;
    const double pitch = f.piso * f.mpn / f.W;
    const double zz0 = f.zstart + z0 * f.step;
    const int W = f.W, H = f.H;
    // Slices of this block that no column of the mask sees in any view (the
    // cone's height is exceeded: |Y| <= rm over the mask, so the detector
    // row coordinate H/2 + z g lies between the bounds of g below) are left
    // at zero without looping over the views; block-uniform.
    bool seen = true;
    {
        const double rm = (f.N * 0.5 + 1.0) * f.scale;
        const double gmin = 1.0 / ((1.0 + rm / f.sad) * pitch), gmax = 1.0 / ((1.0 - rm / f.sad) * pitch);
        const double zzb = zz0 + (double)(min(ZB, f.Z - z0) - 1) * f.step;
        const double a = zz0 * gmin, b = zz0 * gmax, c = zzb * gmin, d = zzb * gmax;
        const double lo = (double)(H / 2) + fmin(fmin(a, b), fmin(c, d));
        const double hi = (double)(H / 2) + fmax(fmax(a, b), fmax(c, d));
        if (rm < f.sad && (hi < -1.0 || lo > (double)H + 1.0)) seen = false;
    }
    const bool full = z0 + ZB <= f.Z;  // every slice of the block exists
    if (inmask && seen) {
        const double cp = (double)f.N / 2.0 - 0.5;
        const double xx = (x - cp) * f.scale;
        const double yy = -(y - cp) * f.scale;
        const double inv_sad = 1.0 / f.sad;
        for (int th = 0; th < f.V; th++) {
            const BpView bv = views[th];
            const double cs = bv.cs, sn = bv.sn;
            // FP64 detector coordinates of this column (:76-83)
            const double X = xx * cs + yy * sn;
            const double Y = -xx * sn + yy * cs;
            const double L2 = 1.0 - Y * inv_sad;
            const double g = 1.0 / (L2 * pitch);
            const double U = X * g;
            const double Uf = floor(U);
            const float wu = (float)(U - Uf);
            const double UUU = bv.ushift + U;
            const int UU = (int)floor(UUU);
            if (UU < 0 || UU > W - 1) continue;
            const double zeta0 = (double)(H / 2) + zz0 * g;
            // every slice of the block projects above or below the detector
            if (zeta0 + (double)(ZB - 1) * f.step * g < -1.0 || zeta0 > (double)H + 1.0) continue;
            const double zf = floor(zeta0);
            const int Zi = (int)zf;
            const float Zf = (float)(zeta0 - zf);
            const float dz = (float)(f.step * g);
            const float iL = (float)(g * pitch);  // 1 / L2
            const float w2 = iL * iL * bv.dbeta * (float)f.xfactor;
            const bool lastc = (UU == W - 1);
            const float cw0 = lastc ? 1.0f : 1.0f - wu;
            const float cw1 = lastc ? 0.0f : wu;
            const int UU1 = lastc ? UU : UU + 1;
            const float* pv = filt + (size_t)th * H * W;
            if (!lastc && full && zeta0 >= 0.0 && zeta0 + (double)(ZB - 1) * f.step * g < (double)H - 2.5) {
                // every slice of the block projects between detector rows 0
                // and H - 2: no bounds or last-row tests
                const float* pc = pv + UU;
#pragma unroll
                for (int i = 0; i < ZB; i++) {
                    const float zfrac = fmaf((float)i, dz, Zf);
                    const float tq = __fadd_rd(zfrac, 12582912.0f);
                    const float fl = tq - 12582912.0f;
                    const int NZ = Zi + (__float_as_int(tq) - 0x4B400000);
                    const float wz = zfrac - fl;
                    const float* r0p = pc + NZ * W;
                    const float* r1p = r0p + W;
                    const float s0 = fmaf(cw1, __ldg(r0p + 1), cw0 * __ldg(r0p));
                    const float s1 = fmaf(cw1, __ldg(r1p + 1), cw0 * __ldg(r1p));
                    acc[i] = fmaf(fmaf(wz, s1, (1.0f - wz) * s0), w2, acc[i]);
                }
                continue;
            }
            if (!lastc && full) {
                // columns UU, UU + 1 of rows NZ, NZ1: one address per row and
                // the second column at +4 bytes; all slices of the block exist
                const float* pc = pv + UU;
#pragma unroll
                for (int i = 0; i < ZB; i++) {
                    const float zfrac = fmaf((float)i, dz, Zf);
                    const float tq = __fadd_rd(zfrac, 12582912.0f);
                    const float fl = tq - 12582912.0f;
                    const int NZ = Zi + (__float_as_int(tq) - 0x4B400000);
                    const float wz = zfrac - fl;
                    if ((unsigned)NZ > (unsigned)(H - 1)) continue;
                    const bool lastr = (NZ == H - 1);
                    const float rw0 = lastr ? 1.0f : 1.0f - wz;
                    const float rw1 = lastr ? 0.0f : wz;
                    const float* r0p = pc + NZ * W;
                    const float* r1p = lastr ? r0p : r0p + W;
                    const float s0 = fmaf(cw1, __ldg(r0p + 1), cw0 * __ldg(r0p));
                    const float s1 = fmaf(cw1, __ldg(r1p + 1), cw0 * __ldg(r1p));
                    acc[i] = fmaf(fmaf(rw1, s1, rw0 * s0), w2, acc[i]);
                }
                continue;
            }
#pragma unroll
            for (int i = 0; i < ZB; i++) {
                const float zfrac = fmaf((float)i, dz, Zf);
                // floor through the adder instead of the conversion unit: the
                // round-down add of 1.5 * 2^23 leaves floor(zfrac) in the low
                // mantissa bits (|zfrac| < 2^22 here); bitwise the same as
                // floorf and (int), 3.5 % faster on B200
                const float tq = __fadd_rd(zfrac, 12582912.0f);
                const float fl = tq - 12582912.0f;
                const int NZ = Zi + (__float_as_int(tq) - 0x4B400000);
                const float wz = zfrac - fl;
                if (NZ < 0 || NZ > H - 1 || z0 + i >= f.Z) continue;
                const bool lastr = (NZ == H - 1);
                const float rw0 = lastr ? 1.0f : 1.0f - wz;
                const float rw1 = lastr ? 0.0f : wz;
                const int NZ1 = lastr ? NZ : NZ + 1;
                const float* r0p = pv + (size_t)NZ * W;
                const float* r1p = pv + (size_t)NZ1 * W;
                const float s0 = fmaf(cw1, __ldg(r0p + UU1), cw0 * __ldg(r0p + UU));
                const float s1 = fmaf(cw1, __ldg(r1p + UU1), cw0 * __ldg(r1p + UU));
                acc[i] = fmaf(fmaf(rw1, s1, rw0 * s0), w2, acc[i]);
            }
        }
    }
#pragma unroll
    for (int i = 0; i < ZB; i++) {
        const int z = z0 + i;
        if (z >= f.Z) break;
        const size_t o = ((size_t)z * f.N + y) * f.N + x;
        if (vol_f32) vol_f32[o] = acc[i];
        if (vol_i16) {
            // (short) of the reconstructed value: truncation toward zero
            // (R/main.cpp:184), saturated to the short range.
            float a = fminf(fmaxf(acc[i], -32768.0f), 32767.0f);
            vol_i16[o] = (short)__float2int_rz(a);
        }
    }
}

}  // namespace

}  // namespace vcbct

namespace vcbct {

cudaError_t launch_filter_direct(const float* proj, float* out, const float* hT,
                                 const FilterView* views, const float* wts, float pitch,
                                 float sad, int V, int H, int W, cudaStream_t st)
{
    const int M = V * H;
    dim3 grid((W + FT_N - 1) / FT_N, (M + FT_M - 1) / FT_M);
    filter_direct_kernel<<<grid, 256, 0, st>>>(proj, out, hT, views, wts, pitch, sad, V, H, W);
    return cudaGetLastError();
}

cudaError_t launch_backproject(const FdkParams& f, const BpView* d_views, const float* filt,
                               float* vol_f32, short* vol_i16, cudaStream_t st)
{
    constexpr int ZB = VCBCT_BP_ZB;
    dim3 block(32, 8);
    dim3 grid((f.N + 31) / 32, (f.N + 7) / 8, (f.Z + ZB - 1) / ZB);
    backproject_kernel<ZB><<<grid, block, 0, st>>>(f, d_views, filt, vol_f32, vol_i16);
    return cudaGetLastError();
}

}  // namespace vcbct
