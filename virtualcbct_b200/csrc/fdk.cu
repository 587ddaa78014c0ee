// fdk.cu -- FDK ramp filter (direct FP32 path) and voxel-driven cone-beam
// backprojection on sm_100a.
//
// Reference: Release_recon_from_forward_pro_float_CM/filterSinogram.cpp:67-131
// and reconstructImage.cpp:10-184 (OpenMP CPU code).
#include "internal.h"

#include <climits>
#include <cstdlib>

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

// Packed pairs of floats for Blackwell's f32x2 arithmetic: one instruction
// for two elements, each rounded exactly as the scalar instruction would
// round it.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 f2pack(float a, float b)
{
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void f2unpack(f32x2 r, float& a, float& b)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r));
}
__device__ __forceinline__ f32x2 ffma2(f32x2 a, f32x2 b, f32x2 c)
{
    f32x2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}
__device__ __forceinline__ f32x2 fmul2(f32x2 a, f32x2 b)
{
    f32x2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 fsub2(f32x2 a, f32x2 b)
{
    f32x2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 fadd2_rd(f32x2 a, f32x2 b)  // rounded toward -inf, as __fadd_rd
{
    f32x2 r;
    asm("add.rm.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
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
// thread.  The packed f32x2 slice loop needs register pairs: with the launch
// constants in the parameter bank, 5 blocks (48 registers) and 6 (40) both
// run without spills on 270x270x200 from 360 half-fan views, and 5 is faster
// on B200 (3.05 vs 3.21 ms, the volume bitwise the same).  16 slices per
// thread at 4 or 3 blocks measured slower (3.55 / 3.49 vs 3.30 ms): more
// columns leave the interior loop at the cone's edges.
#ifndef VCBCT_BP_MIN_BLOCKS
#define VCBCT_BP_MIN_BLOCKS 5
#endif
#ifndef VCBCT_BP_TILE
#define VCBCT_BP_TILE 4  // warp tile width in voxel columns (4, 8, 16 or 32)
#endif
#ifndef VCBCT_BP_ZB
#define VCBCT_BP_ZB 8
#endif
// Per (backprojection block, view): may any column of the block's 32 x 8
// tile take the view in backproject_kernel?  U, g = 1 / (L2 pitch) and the
// row coordinate H/2 + z g are linear-fractional in (x, y) with a positive
// denominator, so over the tile's rectangle they take their extremes at its
// four corners.  A view whose corner values put every column left of column
// 0 or right of column W - 1 (the column test UU < 0 || UU > W - 1), or every
// slice of the block above or below the detector (the row test), is
// dropped; the margin is far above FP64 rounding, so a dropped view is one
// every column of the tile would have skipped.  One warp per (block, 32
// views): bit th & 31 of word th >> 5 of the block's mask.
template <int ZB>
__global__ void __launch_bounds__(256) bp_cull_kernel(FdkParams f, const BpView* __restrict__ views,
                                                      int gx, int gy, int nblocks, unsigned* __restrict__ keep)
{
    constexpr double kMargin = 1e-3;  // detector pixels
    const int nwords = (f.V + 31) >> 5;
    const long wid = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (wid >= (long)nblocks * nwords) return;
    const int lane = threadIdx.x & 31;
    const int blk = (int)(wid / nwords), word = (int)(wid % nwords);
    const int bx = blk % gx, by = (blk / gx) % gy, bz = blk / (gx * gy);
    const int th = word * 32 + lane;
    bool keep_it = false;
    if (th < f.V) {
        const double pitch = f.piso * f.mpn / f.W;
        const double cp = (double)f.N / 2.0 - 0.5;
        const double inv_sad = 1.0 / f.sad;
        const int xa = bx * 32, xb = min(xa + 31, f.N - 1);
        const int ya = by * 8, yb = min(ya + 7, f.N - 1);
        const double zza = f.zstart + (double)(bz * ZB) * f.step;
        const double zzl = zza + (double)(ZB - 1) * f.step;
        const BpView bv = views[th];
        double umin = 1e300, umax = -1e300, gmin = 1e300, gmax = -1e300;
        bool ok = true;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const double xx = (((c & 1) ? xb : xa) - cp) * f.scale;
            const double yy = -(((c & 2) ? yb : ya) - cp) * f.scale;
            const double X = xx * bv.cs + yy * bv.sn;
            const double L2 = 1.0 - (-xx * bv.sn + yy * bv.cs) * inv_sad;
            ok = ok && L2 > 1e-3;
            const double g = 1.0 / (L2 * pitch);
            const double u = bv.ushift + X * g;
            umin = fmin(umin, u);
            umax = fmax(umax, u);
            gmin = fmin(gmin, g);
            gmax = fmax(gmax, g);
        }
        keep_it = true;
        if (ok) {
            const bool left = umax < -kMargin, right = umin >= (double)f.W + kMargin;
            const double last_max = (double)(f.H / 2) + fmax(zzl * gmin, zzl * gmax);
            const double first_min = (double)(f.H / 2) + fmin(zza * gmin, zza * gmax);
            const bool below = last_max < -1.0 - kMargin, above = first_min > (double)f.H + 1.0 + kMargin;
            keep_it = !(left || right || below || above);
        }
    }
    const unsigned m = __ballot_sync(0xffffffffu, keep_it);
    if (lane == 0) keep[wid] = m;
}

// Launch constants of the backprojection, formed on the host in the same
// IEEE double operations as the device would (kernel parameters, so they
// are read from the constant bank instead of occupying registers).
struct BpConst {
    double pitch;    // piso * mpn / W: detector pitch at the isocentre
    double inv_sad;  // 1 / sad
    double cp;       // N / 2 - 0.5: the volume centre in voxels
};

static_assert(sizeof(BpView) == 32, "BpView is staged as four 8-byte words");

// Slice block of launch index i of n, from the middle of the volume out
// (c, c + 1, c - 1, c + 2, ... with c = (n - 1) / 2): the blocks near the
// slab's centre, seen by every view, are the longest and start first, the
// short ones at the cone's edges fill the last wave.
__device__ __forceinline__ int bp_zblock(int i, int n)
{
    const int c = (n - 1) / 2, off = (i + 1) >> 1;
    return (i & 1) ? c + off : c - off;
}

// SV: the view table is copied to shared memory at block start (the
// per-view loads at the head of each set-up chain then come from shared
// memory instead of through L1).
template <int ZB, int MINB, bool SV>
__global__ void __launch_bounds__(256, MINB) backproject_kernel(
    FdkParams f, BpConst k, const BpView* __restrict__ views, const float* __restrict__ filt,
    float* __restrict__ vol_f32, short* __restrict__ vol_i16, const unsigned* __restrict__ keep)
{
    // each warp takes a TW x (32 / TW) tile of the block's 32 x 8 columns:
    // the detector's column-edge and cone-edge lines split fewer warps than
    // with 32 x 1 rows, and a warp's taps fall in fewer cache lines (B200,
    // 270x270x200 from 360 half-fan views: 3.35 ms with 4 x 8 tiles, 3.44
    // with 8 x 4, 3.59 with 16 x 2, 3.96 with 32 x 1; the volume is the same)
    constexpr int TW = VCBCT_BP_TILE, TH = 32 / TW, WX = 32 / TW;
    const int x = blockIdx.x * 32 + (threadIdx.y % WX) * TW + (threadIdx.x % TW);
    const int y = blockIdx.y * 8 + (threadIdx.y / WX) * TH + (threadIdx.x / TW);
    const int bz = bp_zblock(blockIdx.z, gridDim.z);
    const int z0 = bz * ZB;
    const bool valid = x < f.N && y < f.N;
    const double R = (double)(f.N - 1) / 2.0;
    const bool inmask = valid && ((double)y - R) * ((double)y - R) + ((double)x - R) * ((double)x - R) <= R * R;
    float acc[ZB];
#pragma unroll
    for (int i = 0; i < ZB; i++) acc[i] = 0.0f;
    const double pitch = k.pitch;
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
    // Views this block's tile of columns can see (bp_cull_kernel): a view
    // that contributes nothing to any column of the tile is dropped for the
    // whole block.  The kept views are visited in order, so the accumulation
    // order and the volume are those of visiting every view.
    extern __shared__ __align__(16) unsigned char s_raw[];
    const BpView* s_bv = reinterpret_cast<const BpView*>(s_raw);  // SV: [V]
    unsigned* s_views = reinterpret_cast<unsigned*>(s_raw + (SV ? (size_t)f.V * sizeof(BpView) : 0));
    {
        const int tid = threadIdx.y * 32 + threadIdx.x;
        const int nwords = (f.V + 31) >> 5;
        const int blk = (bz * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
        for (int i = tid; i < nwords; i += 256) s_views[i] = __ldg(keep + (size_t)blk * nwords + i);
        if (SV) {
            const unsigned long long* src = reinterpret_cast<const unsigned long long*>(views);
            unsigned long long* dst = reinterpret_cast<unsigned long long*>(s_raw);
            for (int i = tid; i < f.V * 4; i += 256) dst[i] = __ldg(src + i);
        }
    }
    const double cp = k.cp;
    const double inv_sad = k.inv_sad;
    __syncthreads();
    if (!valid) return;
    const bool full = z0 + ZB <= f.Z;  // every slice of the block exists
    if (inmask && seen) {
        const double xx = (x - cp) * f.scale;
        const double yy = -(y - cp) * f.scale;
        // the kept views in order, one mask word at a time (the culled ones
        // cost nothing)
        const int nwords = (f.V + 31) >> 5;
        for (int wi = 0; wi < nwords; wi++)
        for (unsigned wd = s_views[wi]; wd != 0u;) {
            const int th = wi * 32 + __ffs(wd) - 1;
            wd &= wd - 1u;
            const BpView bv = SV ? s_bv[th] : views[th];
            const double cs = bv.cs, sn = bv.sn;
            // FP64 detector coordinates of this column (:76-83)
            const double X = xx * cs + yy * sn;
            const double Y = -xx * sn + yy * cs;
            const double L2 = 1.0 - Y * inv_sad;
            // the correctly rounded reciprocal: 1.0 / (L2 pitch) to the bit
            const double g = __drcp_rn(L2 * pitch);
            const double U = X * g;
            const double Uf = floor(U);
            const float wu = (float)(U - Uf);
            const double UUU = bv.ushift + U;
            // floor and conversion in one (round-down conversion; out of
            // range or NaN gives INT_MIN or INT_MAX, both rejected below)
            const int UU = __double2int_rd(UUU);
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
                // and H - 2: no bounds or last-row tests.  Two slices per
                // step in packed f32x2 arithmetic (each element rounded as
                // the scalar operation would round it: the same volume, half
                // the floating-point instructions)
                const float* pc = pv + UU;
                const f32x2 dz2 = f2pack(dz, dz), zf2b = f2pack(Zf, Zf);
                const f32x2 cw0_2 = f2pack(cw0, cw0), cw1_2 = f2pack(cw1, cw1), w2_2 = f2pack(w2, w2);
                const f32x2 big2 = f2pack(12582912.0f, 12582912.0f), one2 = f2pack(1.0f, 1.0f);
#pragma unroll
                for (int i = 0; i < ZB; i += 2) {
                    const f32x2 zfrac = ffma2(f2pack((float)i, (float)(i + 1)), dz2, zf2b);
                    const f32x2 tq = fadd2_rd(zfrac, big2);
                    const f32x2 wz = fsub2(zfrac, fsub2(tq, big2));
                    float tqa, tqb;
                    f2unpack(tq, tqa, tqb);
                    const float* ra = pc + (Zi + (__float_as_int(tqa) - 0x4B400000)) * W;
                    const float* rb = pc + (Zi + (__float_as_int(tqb) - 0x4B400000)) * W;
                    const f32x2 s0 = ffma2(cw1_2, f2pack(__ldg(ra + 1), __ldg(rb + 1)),
                                           fmul2(cw0_2, f2pack(__ldg(ra), __ldg(rb))));
                    const f32x2 s1 = ffma2(cw1_2, f2pack(__ldg(ra + W + 1), __ldg(rb + W + 1)),
                                           fmul2(cw0_2, f2pack(__ldg(ra + W), __ldg(rb + W))));
                    const f32x2 v = ffma2(wz, s1, fmul2(fsub2(one2, wz), s0));
                    f32x2 a2 = f2pack(acc[i], acc[i + 1]);
                    a2 = ffma2(v, w2_2, a2);
                    f2unpack(a2, acc[i], acc[i + 1]);
                }
                continue;
            }
            if (!lastc && full) {
                // some slices of the block project outside rows 0 .. H - 2:
                // the same packed pairs, a slice off the detector (NZ outside
                // 0 .. H - 1) adding an exact zero (its rows clamped, its
                // weight 0; the sums are never -0, so acc + 0 = acc), the last
                // row taking row weights (1, 0) as the scalar rule does
                const float* pc = pv + UU;
                const f32x2 dz2 = f2pack(dz, dz), zf2b = f2pack(Zf, Zf);
                const f32x2 cw0_2 = f2pack(cw0, cw0), cw1_2 = f2pack(cw1, cw1);
                const f32x2 big2 = f2pack(12582912.0f, 12582912.0f), one2 = f2pack(1.0f, 1.0f);
#pragma unroll
                for (int i = 0; i < ZB; i += 2) {
                    const f32x2 zfrac = ffma2(f2pack((float)i, (float)(i + 1)), dz2, zf2b);
                    const f32x2 tq = fadd2_rd(zfrac, big2);
                    float wza, wzb, tqa, tqb;
                    f2unpack(fsub2(zfrac, fsub2(tq, big2)), wza, wzb);
                    f2unpack(tq, tqa, tqb);
                    const int NZa = Zi + (__float_as_int(tqa) - 0x4B400000);
                    const int NZb = Zi + (__float_as_int(tqb) - 0x4B400000);
                    const bool ina = (unsigned)NZa <= (unsigned)(H - 1), inb = (unsigned)NZb <= (unsigned)(H - 1);
                    const bool la = NZa == H - 1, lb = NZb == H - 1;
                    const int ra = min(max(NZa, 0), H - 1), rb = min(max(NZb, 0), H - 1);
                    const float* r0a = pc + ra * W;
                    const float* r0b = pc + rb * W;
                    const float* r1a = la || !ina ? r0a : r0a + W;
                    const float* r1b = lb || !inb ? r0b : r0b + W;
                    const f32x2 wz = f2pack(la ? 0.0f : wza, lb ? 0.0f : wzb);
                    const f32x2 s0 = ffma2(cw1_2, f2pack(__ldg(r0a + 1), __ldg(r0b + 1)),
                                           fmul2(cw0_2, f2pack(__ldg(r0a), __ldg(r0b))));
                    const f32x2 s1 = ffma2(cw1_2, f2pack(__ldg(r1a + 1), __ldg(r1b + 1)),
                                           fmul2(cw0_2, f2pack(__ldg(r1a), __ldg(r1b))));
                    const f32x2 v = ffma2(wz, s1, fmul2(fsub2(one2, wz), s0));
                    f32x2 a2 = f2pack(acc[i], acc[i + 1]);
                    a2 = ffma2(v, f2pack(ina ? w2 : 0.0f, inb ? w2 : 0.0f), a2);
                    f2unpack(a2, acc[i], acc[i + 1]);
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

size_t backproject_workspace_bytes(const FdkParams& f)
{
    constexpr int ZB = VCBCT_BP_ZB;
    const size_t nblocks = (size_t)((f.N + 31) / 32) * ((f.N + 7) / 8) * ((f.Z + ZB - 1) / ZB);
    return nblocks * (size_t)((f.V + 31) / 32) * sizeof(unsigned);
}

cudaError_t launch_backproject(const FdkParams& f, const BpView* d_views, const float* filt,
                               float* vol_f32, short* vol_i16, unsigned* keep, int* keep_ready,
                               cudaStream_t st)
{
    constexpr int ZB = VCBCT_BP_ZB;
    dim3 block(32, 8);
    dim3 grid((f.N + 31) / 32, (f.N + 7) / 8, (f.Z + ZB - 1) / ZB);
    BpConst k;
    k.pitch = f.piso * f.mpn / f.W;
    k.inv_sad = 1.0 / f.sad;
    k.cp = (double)f.N / 2.0 - 0.5;
    const int nblocks = (int)(grid.x * grid.y * grid.z);
    const long nwarps = (long)nblocks * ((f.V + 31) / 32);
    if (!keep_ready || !*keep_ready) {
        // the view masks follow the geometry and the views only: made once
        bp_cull_kernel<ZB><<<(unsigned)((nwarps * 32 + 255) / 256), 256, 0, st>>>(f, d_views, (int)grid.x,
                                                                                   (int)grid.y, nblocks, keep);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (keep_ready) *keep_ready = 1;
    }
    // the view table goes to shared memory where it fits the default 48 KB
    // with the view mask
    const size_t mask_bytes = (size_t)((f.V + 31) / 32) * sizeof(unsigned);
    const size_t table_bytes = (size_t)f.V * sizeof(BpView);
    const bool sv = table_bytes + mask_bytes <= 48 * 1024;
    const size_t smem = mask_bytes + (sv ? table_bytes : 0);
    // resident blocks per SM (the register cap): VCBCT_BP_MIN_BLOCKS by
    // default, 5 or 6 through the environment variable of the same name
    int minb = VCBCT_BP_MIN_BLOCKS;
    if (const char* e = std::getenv("VCBCT_BP_MIN_BLOCKS")) minb = std::atoi(e) == 6 ? 6 : 5;
    if (minb == 5 && sv)
        backproject_kernel<ZB, 5, true><<<grid, block, smem, st>>>(f, k, d_views, filt, vol_f32, vol_i16, keep);
    else if (minb == 5)
        backproject_kernel<ZB, 5, false><<<grid, block, smem, st>>>(f, k, d_views, filt, vol_f32, vol_i16, keep);
    else if (sv)
        backproject_kernel<ZB, 6, true><<<grid, block, smem, st>>>(f, k, d_views, filt, vol_f32, vol_i16, keep);
    else
        backproject_kernel<ZB, 6, false><<<grid, block, smem, st>>>(f, k, d_views, filt, vol_f32, vol_i16, keep);
    return cudaGetLastError();
}

}  // namespace vcbct
