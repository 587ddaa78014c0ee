// mbfpa.cu -- material-based polychromatic forward projection (MBFPA) on sm_100a.
//
// Reference: Release_CBCT_Projection_CM/reprojectionOnGPU.cu (reprojectionKernel,
// :56-690, launched once per energy bin from :1004-1056).  This file keeps its
// per-ray semantics -- the Siddon-style march with its discrete rules -- and
// changes how the work maps to the GPU:
//
//  * one launch marches every ray once and accumulates the six per-element
//    path integrals L_k; the spectral sum  leng * sum_E pdf_E exp(-sum_k
//    mu_k(E) L_k / xfactor)  is formed in the same kernel (the reference
//    re-marches every ray for each of ~100 bins and copies the whole stack to
//    the host after each);
//  * a warp is 32 consecutive detector rows of one column: those rays share
//    their xy trajectory, so trip counts and x/y plane crossings are
//    warp-uniform and only z crossings diverge;
//  * the volume is re-laid out once into z-fastest 16-byte voxel records
//    (all elements of a voxel in one vector load); the warp's loads at a step
//    fall in one contiguous run of a z column;
//  * FP64 is used only for the per-ray source/detector geometry, the
//    entry/exit and loop-bound computation, and the parametric positions
//    (Siddon alphas) of plane crossings.  The march itself is FP32, with
//    voxel cells carried as integers plus a small fractional offset so that no
//    FP32 value has to resolve a large coordinate near a plane.
//
// Also here: the band footprints of the host-to-host pipelined projection,
// the batch kernels (persistent work queue, flat tile list), the adjoint
// (per-ray spectral derivative, then the same segments scattered into one
// z-fastest plane per element, optionally restricted to a strip of volume
// rows), and the volume / gradient re-layout kernels.
#include "internal.h"
#include "noise.cuh"

#include <cfloat>
#include <climits>
#include <type_traits>

namespace vcbct {

size_t packed_u16_bytes(int N, int Z) { return (size_t)N * N * Z * sizeof(uint4); }
size_t packed_f32_bytes(int N, int Z) { return (size_t)N * N * Z * 2 * sizeof(float4); }

namespace {

// ---------------------------------------------------------------- FP64 ops --
// Explicitly rounded double operations: nvcc may not contract these into
// FMAs, so the setup reproduces the reference's double arithmetic bitwise.
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// (a - a0)/(a1 - a0)*(b1 - b0) + b0, the reference's line evaluation (:159).
__device__ __forceinline__ double line_at(double a, double a0, double a1, double b0, double b1)
{
    return dadd(dmul(ddiv(dsub(a, a0), dsub(a1, a0)), dsub(b1, b0)), b0);
}

// (int) cast of a double made total (non-finite / out of range -> INT_MIN).
__device__ __forceinline__ int d2i(double v)
{
    if (!(v > -2147483648.0 && v < 2147483647.0)) return INT_MIN;
    return __double2int_rz(v);
}

constexpr float kInf = 3.0e38f;

// One axis of the march: value(t) = I + F + slope * (t - ta), in voxel (or
// slice) units.  I is an integer cell base, F a small fraction.
struct Axis {
    int I;
    float F;
    float slope;
    float ta;
};

__device__ __forceinline__ float axis_frac(const Axis& a, float t)
{
    return fmaf(a.slope, t - a.ta, a.F);
}

// Everything the FP32 march needs about one ray, produced by ray_setup().
struct RayPlan {
    int active;      // emits at least one segment
    int d;           // dominant axis (0: x, 1: y)
    int pha;         // +1 / -1 along the dominant axis
    int kstar;       // last iteration index (iterations 0..kstar)
    int klo, khi;    // iterations k >= 1 that can contribute (inclusive)
    int first_idx;   // packed voxel of the first segment, or -1
    float first_len; // its length [cm]
    float Lt;        // cm per unit of t
    float leng;      // cos^3 factor (reprojectionOnGPU.cu:141-150)
    double D0;       // dominant coordinate / s at t = 0
    double O0, O1;   // other in-plane coordinate / s:  O0 + O1 t
    double Z0, Z1;   // z / step:                        Z0 + Z1 t
    double invO1, invZ1;  // 1 / O1, 1 / Z1 (0 when the slope is 0)
    double tc0, tc1; // chord of the cylindrical mask in t
};

// Per-ray FP64 setup: reprojectionOnGPU.cu:128-212, mirrored operation for
// operation.  Rays that hit the xy square fewer than twice are defined to miss
// (the reference reads uninitialised entries there).  Written with scalars and
// selects instead of small arrays indexed by the ray's axes, and inlined, so
// the plan stays in registers (no per-ray stack traffic).
__device__ __forceinline__ void ray_setup(const ProjParams& P, const ViewGeom& vg, int j, int jj, RayPlan& R)
{
    const double s = P.s, step = P.step;
    const int nxm = (int)(P.N * 0.5), nym = (int)(P.N * 0.5), nzm = (int)(P.Z * 0.5);
    const double S0 = dadd(dmul(-P.sad, vg.sn), P.xr);
    const double S1 = dadd(dmul(P.sad, vg.cs), P.yr);
    const double S2 = P.zr;
    const double bin = ddiv(P.dpn, (double)P.H);
    const double P2 = dadd(dmul(dmul(-dadd(vg.yc, (double)j), P.piso), bin), ddiv(dmul(P.zr, P.piso), P.pdet));
    const double pr = dmul(dmul(P.piso, dadd(vg.xc, (double)jj)), bin);
    const double P0 = dadd(dmul(pr, vg.cs), ddiv(dmul(P.xr, P.piso), P.pdet));
    const double P1 = dadd(dmul(pr, vg.sn), ddiv(dmul(P.yr, P.piso), P.pdet));
    {
        const double d2 = dmul(P.sad, P.sad);
        double l = ddiv(d2, dadd(d2, dadd(dmul(pr, pr), dmul(P2, P2))));
        R.leng = (float)dmul(l, __dsqrt_rn(l));
    }
    R.active = 0;
    R.klo = INT_MAX;
    R.khi = -1;
    R.first_idx = -1;
    R.first_len = 0.0f;

    // entry / exit against the four side planes (:154-183); only the first
    // two hits are used, so only they are kept
    const double hx = dmul((double)nxm, s), hy = dmul((double)nym, s);
    double hx0 = 0.0, hy0 = 0.0, hz0 = 0.0, hx1 = 0.0, hy1 = 0.0, hz1 = 0.0;
    int m = 0;
    auto hit = [&](double x, double y, double z) {
        if (m == 0) { hx0 = x; hy0 = y; hz0 = z; }
        else if (m == 1) { hx1 = x; hy1 = y; hz1 = z; }
        m++;
    };
    if (fabs(line_at(hy, S1, P1, S0, P0)) < hx) hit(line_at(hy, S1, P1, S0, P0), hy, line_at(hy, S1, P1, S2, P2));
    if (fabs(line_at(-hy, S1, P1, S0, P0)) < hx) hit(line_at(-hy, S1, P1, S0, P0), -hy, line_at(-hy, S1, P1, S2, P2));
    if (fabs(line_at(hx, S0, P0, S1, P1)) < hy) hit(hx, line_at(hx, S0, P0, S1, P1), line_at(hx, S0, P0, S2, P2));
    if (fabs(line_at(-hx, S0, P0, S1, P1)) < hy) hit(-hx, line_at(-hx, S0, P0, S1, P1), line_at(-hx, S0, P0, S2, P2));
    if (m < 2) return;

    // entry I = the hit nearer the source, exit F = the other
    double I0, I1, I2, F0, F1;
    {
        const double e0 = dadd(dadd(dmul(dsub(hx0, S0), dsub(hx0, S0)), dmul(dsub(hy0, S1), dsub(hy0, S1))),
                               dmul(dsub(hz0, S2), dsub(hz0, S2)));
        const double e1 = dadd(dadd(dmul(dsub(hx1, S0), dsub(hx1, S0)), dmul(dsub(hy1, S1), dsub(hy1, S1))),
                               dmul(dsub(hz1, S2), dsub(hz1, S2)));
        const bool f0 = e0 < e1;
        I0 = f0 ? hx0 : hx1; I1 = f0 ? hy0 : hy1; I2 = f0 ? hz0 : hz1;
        F0 = f0 ? hx1 : hx0; F1 = f0 ? hy1 : hy0;
    }
    // dominant axis, GPU twin rule (:198); _d / _o name the dominant and the
    // other in-plane axis
    const int d = (fabs(dsub(I0, F0)) > fabs(dsub(I1, F1))) ? 0 : 1;
    const double Id = d ? I1 : I0, Fd = d ? F1 : F0;
    const double Sd = d ? S1 : S0, So = d ? S0 : S1;
    const double Pd = d ? P1 : P0, Po = d ? P0 : P1;
    const double dF = dsub(Fd, Id);
    const double pha = ddiv(dF, fabs(dsub(Id, Fd)));
    if (!(pha == 1.0 || pha == -1.0)) return;
    int ain;
    if ((Id < 0 && dF < 0) || (Id > 0 && dF > 0))
        ain = d2i(dadd((double)d2i(Id), ddiv(dF, fabs(dF))));
    else
        ain = d2i(Id);
    if (ain == INT_MIN) return;

    const double h = hx;  // hx == hy (both from reconSize)
    auto inb = [&](double k) {
        double a = dadd((double)ain, dmul(dmul(pha, k), s));
        double ov = line_at(a, Sd, Pd, So, Po);
        return a <= h && a >= -h && ov <= h && ov >= -h;
    };
    if (!inb(0.0)) return;

    // first iteration whose step point leaves the box; the loop of the
    // reference (:212) executes it and stops.
    const double go = ddiv(dsub(Po, So), dsub(Pd, Sd));
    const double gz = ddiv(dsub(P2, S2), dsub(Pd, Sd));
    const double o0 = line_at((double)ain, Sd, Pd, So, Po);
    const double z0 = line_at((double)ain, Sd, Pd, S2, P2);
    double kd = floor((h - pha * ain) / s) + 1.0;
    double ko = 1e30;
    const double vo = go * pha * s;
    if (vo > 0) ko = floor((h - o0) / vo) + 1.0;
    else if (vo < 0) ko = floor((-h - o0) / vo) + 1.0;
    double ke = fmin(kd, ko);
    const int kcap = 4 * (P.N + 4) + (int)(8.0 / s) + 64;
    if (!(ke >= 1.0)) ke = 1.0;
    if (ke > kcap) ke = kcap;
    int ks = (int)ke;
    while (ks > 1 && !inb((double)(ks - 1))) ks--;
    int guard = 0;
    while (inb((double)ks) && guard < kcap) { ks++; guard++; }
    R.kstar = ks;

    R.d = d;
    R.pha = (int)pha;
    R.D0 = (double)ain / s;
    R.O0 = o0 / s;
    R.O1 = go * pha;
    R.Z0 = z0 / step;
    R.Z1 = gz * pha * s / step;
    R.Lt = (float)(s * sqrt(1.0 + go * go + gz * gz));
    R.invO1 = (R.O1 != 0.0) ? 1.0 / R.O1 : 0.0;
    R.invZ1 = (R.Z1 != 0.0) ? 1.0 / R.Z1 : 0.0;
    R.tc0 = 1.0;
    R.tc1 = 0.0;
    R.active = 1;

    // Iteration 0 emits one unsplit segment from the entry point to the first
    // step point (:405-427 with ik == 0).  It can span many voxels and its
    // midpoint often lies exactly on a voxel plane (entry through a face), so
    // its voxel, length and mask are evaluated in FP64 exactly as the
    // reference does.
    {
        const double b10 = d ? o0 : (double)ain;
        const double b11 = d ? (double)ain : o0;
        const double b12 = z0;
        const double rr = __dsqrt_rn(dadd(dadd(dmul(dsub(I0, b10), dsub(I0, b10)),
                                               dmul(dsub(I1, b11), dsub(I1, b11))),
                                          dmul(dsub(I2, b12), dsub(I2, b12))));
        const int xmc = d2i(dadd(ddiv(dmul(dadd(I0, b10), 0.5), s), (double)nxm));
        const int ymc = d2i(dadd(ddiv(dmul(dsub(-I1, b11), 0.5), s), (double)nym));
        const int zmc = d2i(dadd(ddiv(dmul(dsub(-I2, b12), 0.5), step), (double)nzm));
        if (xmc >= 0 && ymc >= 0 && zmc >= 0 && xmc <= P.N - 1 && ymc <= P.N - 1 && zmc <= P.Z - 1) {
            const double r = dmul(__dsqrt_rn(dadd(dmul(dadd(I0, b10), dadd(I0, b10)),
                                                  dmul(dsub(-I1, b11), dsub(-I1, b11)))), 0.5);
            if (!(r >= dmul(dmul((double)P.N, 0.5), s))) {
                R.first_idx = (ymc * P.N + xmc) * P.Z + zmc;
                R.first_len = (float)rr;
            }
        }
    }

    // iterations whose segments can pass the cylinder mask and the z bounds
    const double Rv = P.N * 0.5;
    double A = 1.0 + R.O1 * R.O1;
    double B = 2.0 * (R.D0 * pha + R.O0 * R.O1);
    double C = R.D0 * R.D0 + R.O0 * R.O0 - Rv * Rv;
    double disc = B * B - 4.0 * A * C;
    if (!(disc > 0.0)) return;
    double sq = sqrt(disc);
    double tl = (-B - sq) / (2.0 * A), th = (-B + sq) / (2.0 * A);
    R.tc0 = tl;
    R.tc1 = th;
    const double zlo = (double)(nzm - P.Z), zhi = (double)(nzm + 1);  // (int) of zmc in [0, Z-1]
    if (R.Z1 > 0) {
        tl = fmax(tl, (zlo - R.Z0) / R.Z1);
        th = fmin(th, (zhi - R.Z0) / R.Z1);
    } else if (R.Z1 < 0) {
        tl = fmax(tl, (zhi - R.Z0) / R.Z1);
        th = fmin(th, (zlo - R.Z0) / R.Z1);
    } else if (!(R.Z0 > zlo && R.Z0 < zhi)) {
        return;
    }
    if (!(th > tl)) return;
    // iteration k >= 1 covers t in [k-1, k]; one step of margin each side
    int klo = (int)fmax(1.0, floor(tl) - 1.0);
    int khi = (int)fmin((double)ks, floor(th) + 2.0);
    if (khi < klo) return;
    R.klo = klo;
    R.khi = khi;
}

// Map a cell index to the reference's (int)-truncated voxel index: the value
// lies in (q, q+1); q >= 0 -> q, q == -1 -> 0 (truncation toward zero), else
// out of range.  Returns -1 when out of [0, size).
__device__ __forceinline__ int trunc_index(int q, int size)
{
    return ((unsigned)(q + 1) <= (unsigned)size) ? max(q, 0) : -1;
}

// Slice index of a ray with Z1 == 0 (it stays in the plane z = Z0 * step;
// with z_reg = 0 the central detector row does).  The reference's rule
// (int)(nzm - z/step) differs from the cell rule when Z0 is an integer (the
// midpoints then lie exactly on a slice boundary), so it is applied as is.
__device__ __forceinline__ int flat_z_index(const ProjParams& P, double Z0)
{
    const double q = (double)(int)(P.Z * 0.5) - Z0;
    return (q > -1.0 && q < (double)P.Z) ? (int)q : -1;
}

// Anchor of an axis at parameter t (FP64 value v = c0 + c1 t).
__device__ __forceinline__ Axis make_axis(double c0, double c1, double t)
{
    double v = c0 + c1 * t;
    double fl = floor(v);
    Axis a;
    a.I = (int)fl;
    a.F = (float)(v - fl);
    a.slope = (float)c1;
    a.ta = (float)t;
    return a;
}

// Parameter of the crossing of plane `m` (FP64 Siddon alpha, as float).
__device__ __forceinline__ float cross_t(double c0, double inv1, int m)
{
    return (float)(((double)m - c0) * inv1);
}

// The FP32 march of iterations k in [Klo, Khi] (k >= 1) of one ray
// (reprojectionOnGPU.cu:200-429 and its y-dominant mirror :441-666).
// `visit(idx, len)` is called with the packed voxel index of every segment
// that passes the voxel-bounds test and the cylinder mask.
template <class Visit>
__device__ __forceinline__ void march(const ProjParams& P, const RayPlan& R, int Klo, int Khi,
                                      Visit& visit)
{
    const int nxm = (int)(P.N * 0.5), nym = (int)(P.N * 0.5), nzm = (int)(P.Z * 0.5);
    const float R2 = (float)(P.N * 0.5) * (float)(P.N * 0.5);
    const int d = R.d;
    const float fpha = (float)R.pha;
    const double Dfl = floor(R.D0);
    const int Id0 = (int)Dfl;
    const float Fd = (float)(R.D0 - Dfl);

    // o / z crossing bookkeeping (FP64 alphas)
    const int diro = (R.O1 > 0) ? 1 : ((R.O1 < 0) ? -1 : 0);
    const int dirz = (R.Z1 > 0) ? 1 : ((R.Z1 < 0) ? -1 : 0);
    const double invO1 = diro ? 1.0 / R.O1 : 0.0;
    const double invZ1 = dirz ? 1.0 / R.Z1 : 0.0;

    const int ks = Klo;
    const double t0s = (double)(ks - 1);
    Axis ao = make_axis(R.O0, R.O1, t0s);
    Axis az = make_axis(R.Z0, R.Z1, t0s);
    int mo = 0, mz = 0;
    float to_next = kInf, tz_next = kInf;
    if (diro) {
        double v = R.O0 + R.O1 * t0s;
        mo = (diro > 0) ? (int)floor(v) + 1 : (int)ceil(v) - 1;
        to_next = cross_t(R.O0, invO1, mo);
    }
    if (dirz) {
        double v = R.Z0 + R.Z1 * t0s;
        mz = (dirz > 0) ? (int)floor(v) + 1 : (int)ceil(v) - 1;
        if (mz == 0) mz += dirz;  // z = 0 is never a split plane (:237-238)
        tz_next = cross_t(R.Z0, invZ1, mz);
    }

    const int izflat = dirz ? -1 : flat_z_index(P, R.Z0);

    // One segment [ta, tb] within the step whose start is t = tbase, where the
    // dominant cell base is Idk.
    auto segment = [&](float ta, float tb, float tbase, int Idk) {
        const float tm = 0.5f * (ta + tb);
        const float ud = fmaf(fpha, tm - tbase, Fd);
        const float uo = axis_frac(ao, tm);
        const float uz = axis_frac(az, tm);
        const int cd = Idk + __float2int_rd(ud);
        const int co = ao.I + __float2int_rd(uo);
        const int cz = az.I + __float2int_rd(uz);
        const float vd = (float)Idk + ud;
        const float vo = (float)ao.I + uo;
        const int cx = d ? co : cd;
        const int cy = d ? cd : co;
        const int ix = trunc_index(nxm + cx, P.N);
        const int iy = trunc_index(nym - 1 - cy, P.N);
        const int iz = dirz ? trunc_index(nzm - 1 - cz, P.Z) : izflat;
        if ((ix | iy | iz) < 0) return;
        if (!(fmaf(vd, vd, vo * vo) < R2)) return;
        visit((iy * P.N + ix) * P.Z + iz, fabsf(tb - ta));
    };

    const int kcap = Khi;
    for (int k = ks; k <= kcap; k++) {
        const float tk = (float)k;
        const float t0 = tk - 1.0f;
        const int Idk = Id0 + R.pha * (k - 1);
        const bool eo = to_next <= tk;
        const bool ez = tz_next <= tk;
        float tY = 0.0f, tZ = 0.0f;
        if (eo) {
            tY = to_next;
            ao.I = mo; ao.F = 0.0f; ao.ta = tY;
            mo += diro;
            to_next = cross_t(R.O0, invO1, mo);
        }
        if (ez) {
            // the reference splits only at the last z plane crossed in a step
            int guard = 0;
            do {
                tZ = tz_next;
                az.I = mz; az.F = 0.0f; az.ta = tZ;
                mz += dirz;
                if (mz == 0) mz += dirz;
                tz_next = cross_t(R.Z0, invZ1, mz);
            } while (tz_next <= tk && ++guard < 64);
        }
        // order of the split points: the one farther from the step point first
        // (chz > chy, :249-404)
        int ns = 0;
        float a1 = tk, a2 = tk;
        if (eo && ez) {
            const float dY = tk - tY, dZ = tk - tZ;
            if (dZ > dY) { a1 = tZ; a2 = tY; ns = 2; }
            else if (dZ < dY) { a1 = tY; a2 = tZ; ns = 2; }
        } else if (eo) {
            if (tY != tk) { a1 = tY; ns = 1; }
        } else if (ez) {
            if (tZ != tk) { a1 = tZ; ns = 1; }
        }
        segment(t0, ns > 0 ? a1 : tk, t0, Idk);
        if (ns > 0) segment(a1, ns > 1 ? a2 : tk, t0, Idk);
        if (ns > 1) segment(a2, tk, t0, Idk);
    }
}

// -------------------------------------------------------------- visitors --
// Partial sums are kept as pairs of floats and updated with Blackwell's
// packed f32x2 add / fma (one instruction for two elements, each element
// rounded exactly as the scalar fmaf / fadd would round it).
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
__device__ __forceinline__ f32x2 fadd2(f32x2 a, f32x2 b)
{
    f32x2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 ffma2(f32x2 a, f32x2 b, f32x2 c)
{
    f32x2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}

// Both uint16 halves of a packed word as exact floats {low, high} without
// the conversion unit: each half is placed in the mantissa of 2^23
// (0x4B000000 | u, a byte permute) and 2^23 is subtracted (exact).
__device__ __forceinline__ f32x2 u16pair(unsigned w)
{
    const float lo = __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7410));
    const float hi = __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7432));
    return fadd2(f2pack(lo, hi), 0xCB000000CB000000ull);  // {-2^23, -2^23}
}

// Two-level sums: segments accumulate into the pairs P2 (element 2i in the
// low half, 2i+1 in the high half); fold() adds them into L every 32
// iterations, which bounds the FP32 error growth.  The marches pass each
// segment's length in units of the ray parameter (dt); fold() scales the
// pair sums by the ray's cm per unit (lt): one multiply per 32 steps instead
// of one per segment.  first() adds a segment of absolute length to L.
template <int M>
struct PairSums {
    static constexpr int NP = (M + 1) / 2;
    float L[M];
    f32x2 P2[NP];
    float lt = 1.0f;  // cm per unit of the ray parameter: the pair sums hold sum v dt
    __device__ __forceinline__ void clear()
    {
#pragma unroll
        for (int i = 0; i < M; i++) L[i] = 0.0f;
#pragma unroll
        for (int i = 0; i < NP; i++) P2[i] = 0ull;
    }
    __device__ __forceinline__ void fold()
    {
#pragma unroll
        for (int i = 0; i < NP; i++) {
            float a, b;
            f2unpack(P2[i], a, b);
            L[2 * i] = fmaf(a, lt, L[2 * i]);
            if (2 * i + 1 < M) L[2 * i + 1] = fmaf(b, lt, L[2 * i + 1]);
            P2[i] = 0ull;
        }
    }
    __device__ __forceinline__ void zero_L()
    {
#pragma unroll
        for (int i = 0; i < M; i++) L[i] = 0.0f;
    }
};

// The same with L in shared memory (this thread's column of an [M][threads
// of the block] array): L is touched once per 32 steps, and its registers are
// free for the walk and the interval production.  Sized by the block (not by
// the largest block) so that the shared memory the resident blocks leave to
// L1 is as large as it can be.
__device__ __forceinline__ int ls_stride() { return (int)(blockDim.x * blockDim.y); }
template <int M>
struct PairSumsS {
    static constexpr int NP = (M + 1) / 2;
    float* Ls;
    f32x2 P2[NP];
    float lt = 1.0f;
    __device__ __forceinline__ float Lget(int i) const { return Ls[i * ls_stride()]; }
    __device__ __forceinline__ void clear()
    {
#pragma unroll
        for (int i = 0; i < M; i++) Ls[i * ls_stride()] = 0.0f;
#pragma unroll
        for (int i = 0; i < NP; i++) P2[i] = 0ull;
    }
    __device__ __forceinline__ void fold()
    {
#pragma unroll
        for (int i = 0; i < NP; i++) {
            float a, b;
            f2unpack(P2[i], a, b);
            Ls[2 * i * ls_stride()] = fmaf(a, lt, Ls[2 * i * ls_stride()]);
            if (2 * i + 1 < M) Ls[(2 * i + 1) * ls_stride()] = fmaf(b, lt, Ls[(2 * i + 1) * ls_stride()]);
            P2[i] = 0ull;
        }
    }
    __device__ __forceinline__ void zero_L()
    {
#pragma unroll
        for (int i = 0; i < M; i++) Ls[i * ls_stride()] = 0.0f;
    }
};

template <int M>
struct AccumU16 : PairSumsS<M> {
    const uint4* __restrict__ vol;
    unsigned nseg;
    __device__ __forceinline__ AccumU16(const uint4* v, float* ls) : vol(v), nseg(0u)
    {
        this->Ls = ls;
        this->clear();
    }
    // called by all 32 lanes together; p: this lane has a segment
    __device__ __forceinline__ void lanes(bool p, int idx, float len)
    {
        if (p) (*this)(idx, len);
    }
    __device__ __forceinline__ void operator()(int idx, float len)
    {
        const uint4 v = __ldg(vol + idx);
        const f32x2 l2 = f2pack(len, len);
        this->P2[0] = ffma2(u16pair(v.x), l2, this->P2[0]);
        this->P2[1] = ffma2(u16pair(v.y), l2, this->P2[1]);
        this->P2[2] = ffma2(u16pair(v.z), l2, this->P2[2]);
        if (M > 6) this->P2[3 % PairSumsS<M>::NP] = ffma2(u16pair(v.w), l2, this->P2[3 % PairSumsS<M>::NP]);
        nseg++;
    }
    // a segment of absolute length len (cm), straight into L
    __device__ __forceinline__ void first(int idx, float len)
    {
        const uint4 v = __ldg(vol + idx);
        const unsigned w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int i = 0; i < M; i++) {
            float a, b;
            f2unpack(u16pair(w[i / 2]), a, b);
            this->Ls[i * ls_stride()] = fmaf((i & 1) ? b : a, len, this->Ls[i * ls_stride()]);
        }
        nseg++;
    }
};

template <int M, bool SL = false>
struct AccumF32 : std::conditional_t<SL, PairSumsS<M>, PairSums<M>> {
    using Base = std::conditional_t<SL, PairSumsS<M>, PairSums<M>>;
    const float4* __restrict__ vol;
    unsigned nseg;
    __device__ __forceinline__ AccumF32(const float4* v, float* ls = nullptr) : vol(v), nseg(0u)
    {
        if constexpr (SL) this->Ls = ls;
        this->clear();
    }
    __device__ __forceinline__ void lanes(bool p, int idx, float len)
    {
        if (p) (*this)(idx, len);
    }
    __device__ __forceinline__ void operator()(int idx, float len)
    {
        const ulonglong2* p = reinterpret_cast<const ulonglong2*>(vol + 2 * (size_t)idx);
        const ulonglong2 a = __ldg(p), b = __ldg(p + 1);
        const f32x2 l2 = f2pack(len, len);
        this->P2[0] = ffma2(a.x, l2, this->P2[0]);
        this->P2[1] = ffma2(a.y, l2, this->P2[1]);
        this->P2[2] = ffma2(b.x, l2, this->P2[2]);
        if (M > 6) this->P2[3 % Base::NP] = ffma2(b.y, l2, this->P2[3 % Base::NP]);
        nseg++;
    }
    // a segment of absolute length len (cm), straight into L
    __device__ __forceinline__ void first(int idx, float len)
    {
        const float* p = reinterpret_cast<const float*>(vol + 2 * (size_t)idx);
#pragma unroll
        for (int i = 0; i < M; i++) {
            if constexpr (SL) this->Ls[i * ls_stride()] = fmaf(__ldg(p + i), len, this->Ls[i * ls_stride()]);
            else this->L[i] = fmaf(__ldg(p + i), len, this->L[i]);
        }
        nseg++;
    }
};

// Scatter of one segment's gradient into element planes: plane k holds
// element k of every voxel at the packed record index (y*N + x)*Z + z, so
// the 32 lanes of a warp -- adjacent detector rows, adjacent z cells of one
// xy cell -- reduce into a few consecutive sectors of each plane (one
// reduction per element and lane; the L2 applies them per sector).
template <int M>
struct Scatter {
    float* __restrict__ grad;   // element groups: quads [N*N*Z][4] (elements 4q .. 4q+3), the last
                                // group a pair [N*N*Z][2] when it holds one or two elements
    size_t plane;               // N*N*Z
    int nmat;
    float g[8];                 // zero beyond nmat
    unsigned lo, span;          // packed indices [lo, lo + span) of the strip scattered into
    float lt;                   // cm per unit of the ray parameter (the march passes dt)
    __device__ __forceinline__ void operator()(int idx, float dt) { first(idx, dt * lt); }
    // a segment of absolute length len (cm)
    __device__ __forceinline__ void first(int idx, float len)
    {
        if ((unsigned)idx - lo >= span) return;
        // one 16-byte vector reduction per group of four elements (8 bytes
        // for a last group of one or two): a third fewer reduction requests
        // than per element pair for six elements, the same sectors
#pragma unroll
        for (int q = 0; q < (M + 3) / 4; q++) {
            const int e0 = 4 * q;
            if (e0 >= nmat) break;
            float* base = grad + (size_t)e0 * plane;  // earlier groups are full quads
            if (nmat - e0 > 2)
                atomicAdd(reinterpret_cast<float4*>(base) + idx,
                          make_float4(g[e0] * len, g[e0 + 1] * len, g[(e0 + 2) % 8] * len, g[(e0 + 3) % 8] * len));
            else
                atomicAdd(reinterpret_cast<float2*>(base) + idx, make_float2(g[e0] * len, g[e0 + 1] * len));
        }
    }
    __device__ __forceinline__ void lanes(bool p, int idx, float len)
    {
        if (p) (*this)(idx, len);
    }
};

// ------------------------------------------------- interval march (fast) --
// The xy part of a ray's segments is the same for the 32 rays of a warp (one
// detector column): the dominant-axis steps cut by the crossings of the other
// in-plane axis.  Every 32 steps the lanes compute those xy intervals in
// parallel (lane l takes step k0 + l: its o-plane crossing, each piece's xy
// cell and cylinder test, all in FP64), a warp scan packs them into shared
// memory, and then every lane walks the list with only its own z work: a
// cached slice index, and an exact slow path at the rare z-plane crossings.
// The segments are those of the per-step march whenever at most one z plane
// is crossed per step (|Z1| < 1); warps with steeper rays use the per-step
// march, which reproduces the reference's last-plane-only split.
struct IvRec {
    float ta, tb;  // parameter range of the xy interval
    int base;      // (iy*N + ix)*Z of its midpoint, or -1 (outside mask / bounds)
    float lim;     // ta if every sub-segment has the same xy cell and mask result, else tb:
                   // a z crossing at or before lim needs the exact path
};

constexpr int kIvPerWarp = 64;

// The xy part of the ray plan: identical for the 32 rays of a warp (one
// detector column), so it is kept once per warp in shared memory after the
// interval buffer instead of in every lane's registers.  The interval
// producer and the slow path read it from there.
struct XyPlan {
    double D0, O0, O1, invO1, tc0, tc1;
    int pha, d;
};
constexpr int kIvSlots = kIvPerWarp + (int)((sizeof(XyPlan) + sizeof(IvRec) - 1) / sizeof(IvRec));

__device__ __forceinline__ const XyPlan& publish_plan(const RayPlan& R, IvRec* wbuf)
{
    XyPlan* xp = reinterpret_cast<XyPlan*>(wbuf + kIvPerWarp);
    if (threadIdx.x == 0 && R.active) {
        xp->D0 = R.D0;
        xp->O0 = R.O0;
        xp->O1 = R.O1;
        xp->invO1 = R.invO1;
        xp->tc0 = R.tc0;
        xp->tc1 = R.tc1;
        xp->pha = R.pha;
        xp->d = R.d;
    }
    __syncwarp();
    return *xp;
}

// xy cell of the point at parameter t (FP64), as the reference's midpoint
// rule: -1 when outside the cylindrical mask or the volume.
__device__ __forceinline__ int xy_base_at(const ProjParams& P, const XyPlan& R, double t)
{
    const int nxm = (int)(P.N * 0.5), nym = (int)(P.N * 0.5);
    const double Rv = P.N * 0.5;
    const double Dm = R.D0 + R.pha * t, Om = R.O0 + R.O1 * t;
    if (!(Dm * Dm + Om * Om < Rv * Rv)) return -1;
    const int cd = (int)floor(Dm), co = (int)floor(Om);
    const int cx = R.d ? co : cd, cy = R.d ? cd : co;
    const int ix = trunc_index(nxm + cx, P.N), iy = trunc_index(nym - 1 - cy, P.N);
    if (ix < 0 || iy < 0) return -1;
    return (iy * P.N + ix) * P.Z;
}

__device__ __forceinline__ bool make_rec(const ProjParams& P, const XyPlan& R, double ta,
                                         double tb, IvRec& rec)
{
    // keep every interval that meets the mask chord: a z split can move a
    // sub-segment's midpoint inside even when the interval's is outside
    if (!(tb > R.tc0 - 1e-9 && ta < R.tc1 + 1e-9)) return false;
    rec.ta = (float)ta;
    rec.tb = (float)tb;
    if (!(rec.tb > rec.ta)) return false;  // zero-length (a crossing exactly at a step)
    rec.base = xy_base_at(P, R, 0.5 * (ta + tb));
    // a dominant-axis plane strictly inside (only when 1/s is not an integer)
    // or the mask boundary inside makes sub-segments' cells differ
    const double da = R.D0 + R.pha * ta, db = R.D0 + R.pha * tb;
    const double lo = fmin(da, db), hi = fmax(da, db);
    double m = floor(hi);
    if (m == hi) m -= 1.0;
    const bool dplane = m > lo;
    const bool edge = (R.tc0 > ta && R.tc0 < tb) || (R.tc1 > ta && R.tc1 < tb);
    rec.lim = (dplane || edge) ? rec.tb : rec.ta;
    return true;
}

// Intervals of steps [k0, min(k0 + 31, Khi)] into buf; returns their number.
__device__ __forceinline__ int produce_intervals(const ProjParams& P, const XyPlan& R, int k0,
                                                 int Khi, IvRec* buf)
{
    const int lane = threadIdx.x;
    const int k = k0 + lane;
    IvRec r0, r1;
    bool v0 = false, v1 = false;
    if (k <= Khi) {
        const double tk = (double)k, tkm = tk - 1.0;
        double tsplit = tk;
        bool ev = false;
        if (R.O1 != 0.0) {
            // a plane m of the other axis is crossed in (k-1, k]: floor changes
            // (all integers, the zero plane included: reprojectionOnGPU.cu:226)
            const double fk = floor(R.O0 + R.O1 * tk), fkm = floor(R.O0 + R.O1 * tkm);
            if (fk != fkm) {
                const double m = (R.O1 > 0.0) ? fk : fkm;
                const double t = (m - R.O0) * R.invO1;
                if (t > tkm && t < tk) {
                    ev = true;
                    tsplit = t;
                }
            }
        }
        v0 = make_rec(P, R, tkm, tsplit, r0);
        if (ev) v1 = make_rec(P, R, tsplit, tk, r1);
    }
    const int n = (int)v0 + (int)v1;
    int incl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    const int off = incl - n;
    if (v0) buf[off] = r0;
    if (v1) buf[off + (int)v0] = r1;
    __syncwarp();
    return total;
}

// Per-lane z state of the interval march.
struct ZState {
    int cz;        // floor(z / step) of the current position's cell
    int iz;        // its slice index (trunc rule), or -1
    int mz;        // next z plane that splits (never 0: :237-238)
    int dirz;
    float tz_next; // parameter of that crossing
    float tz0;     // parameter of the (non-splitting) z = 0 crossing ahead, or inf
};

__device__ __forceinline__ float zcross(const RayPlan& R, int m)
{
    return (float)(((double)m - R.Z0) * R.invZ1);
}

__device__ __forceinline__ void zstate_init(const ProjParams& P, const RayPlan& R, double t0, ZState& z)
{
    const int nzm = (int)(P.Z * 0.5);
    const double v = R.Z0 + R.Z1 * t0;
    const double fl = floor(v);
    z.cz = (int)fl;
    z.dirz = (R.Z1 > 0.0) ? 1 : ((R.Z1 < 0.0) ? -1 : 0);
    z.tz_next = kInf;
    z.tz0 = kInf;
    if (z.dirz) {
        z.mz = (z.dirz > 0) ? z.cz + 1 : ((v == fl) ? z.cz - 1 : z.cz);
        if (z.mz == 0) z.mz += z.dirz;
        z.tz_next = zcross(R, z.mz);
        if ((z.dirz > 0 && v < 0.0) || (z.dirz < 0 && v > 0.0)) z.tz0 = zcross(R, 0);
        z.iz = trunc_index(nzm - 1 - z.cz, P.Z);
    } else {
        z.iz = flat_z_index(P, R.Z0);
    }
}

// One interval, exact: split it at the z planes inside it (and apply the
// midpoint rule across the z = 0 plane, which does not split).
template <class Visit>
__device__ __forceinline__ void consume_slow(const ProjParams& P, const RayPlan& R, const XyPlan& xp,
                                             const IvRec& rc,
                                             ZState& z, Visit& visit)
{
    const int nzm = (int)(P.Z * 0.5);
    float cur = rc.ta;
    const float tb = rc.tb;
    // crossings in intervals that were not produced (outside the mask chord)
    // only move the state
    for (int guard = 0; z.tz_next <= cur && guard < 64; guard++) {
        z.cz = (z.dirz > 0) ? z.mz : z.mz - 1;
        z.mz += z.dirz;
        if (z.mz == 0) z.mz += z.dirz;
        z.tz_next = zcross(R, z.mz);
    }
    if (z.tz0 <= cur) {
        z.cz = (z.dirz > 0) ? 0 : -1;
        z.tz0 = kInf;
    }
    for (int guard = 0; guard < 8; guard++) {
        const bool split = z.tz_next <= tb;
        const float end = split ? z.tz_next : tb;
        int cseg = z.cz;
        if (z.tz0 <= end) {
            const int after = (z.dirz > 0) ? 0 : -1;
            if (0.5f * (cur + end) >= z.tz0) cseg = after;
            z.cz = after;
            z.tz0 = kInf;
        }
        if (end > cur) {
            const bool whole = (cur == rc.ta) && (end == tb);
            const int base = whole ? rc.base : xy_base_at(P, xp, 0.5 * ((double)cur + (double)end));
            const int iz = trunc_index(nzm - 1 - cseg, P.Z);
            if (base >= 0 && iz >= 0) visit(base + iz, end - cur);
        }
        if (!split) break;
        z.cz = (z.dirz > 0) ? z.mz : z.mz - 1;
        cur = end;
        z.mz += z.dirz;
        if (z.mz == 0) z.mz += z.dirz;
        z.tz_next = zcross(R, z.mz);
    }
    z.iz = trunc_index(nzm - 1 - z.cz, P.Z);
}

template <class Visit>
__device__ __forceinline__ void consume_one(const ProjParams& P, const RayPlan& R, const XyPlan& xp,
                                            const IvRec& rc,
                                            ZState& z, Visit& visit)
{
    if (z.tz_next <= rc.tb || z.tz0 <= rc.tb) {
        consume_slow(P, R, xp, rc, z, visit);
    } else if (rc.base >= 0 && z.iz >= 0) {
        visit(rc.base + z.iz, rc.tb - rc.ta);
    }
}

// Iterations [Klo, Khi] of one ray by intervals; `flush` folds partial sums.
// Per interval the common case is one vector load in the lane's current z
// cell; a z crossing inside an exact interval splits it inline (second load
// in the new cell).  Everything else -- the non-splitting z = 0 plane, a
// crossing in an interval whose sub-segments may change xy cell or mask
// result, and crossings passed in intervals that were not produced -- goes
// through consume_slow.  Both branches are taken warp-uniformly.
template <class Visit, class Flush>
__device__ __forceinline__ void march_intervals(const ProjParams& P, const RayPlan& R, const XyPlan& xp, bool act,
                                                int Klo, int Khi, IvRec* buf, Visit& visit,
                                                Flush flush)
{
    const int nzm = (int)(P.Z * 0.5);
    ZState z;
    zstate_init(P, R, (double)(Klo - 1), z);
    if (!act) {  // inactive lanes follow the warp without contributing
        z.iz = -1;
        z.tz_next = kInf;
        z.tz0 = kInf;
    }
    for (int k0 = Klo; k0 <= Khi; k0 += 32) {
        const int total = produce_intervals(P, xp, k0, Khi, buf);
        // two intervals per loop trip: 2 % fewer cycles on B200 (512x512x200,
        // 360 views) than one, while four lose to register pressure
#pragma unroll 2
        for (int i = 0; i < total; i++) {
            const IvRec rc = buf[i];
            const bool rare = (z.tz0 <= rc.tb) || (z.tz_next <= rc.lim);
            if (__any_sync(0xffffffffu, rare)) {
                consume_one(P, R, xp, rc, z, visit);
                continue;
            }
            const bool ev = z.tz_next <= rc.tb;
            const float tz = ev ? z.tz_next : rc.tb;
            visit.lanes(rc.base >= 0 && z.iz >= 0, rc.base + z.iz, tz - rc.ta);
            if (__any_sync(0xffffffffu, ev)) {
                if (ev) {
                    z.cz = (z.dirz > 0) ? z.mz : z.mz - 1;
                    z.iz = trunc_index(nzm - 1 - z.cz, P.Z);
                    z.mz += z.dirz;
                    if (z.mz == 0) z.mz += z.dirz;
                    z.tz_next = zcross(R, z.mz);
                }
                visit.lanes(ev && rc.base >= 0 && z.iz >= 0 && rc.tb > tz, rc.base + z.iz, rc.tb - tz);
            }
        }
        __syncwarp();
        flush();
    }
}

// Two-level summation: the visitor accumulates into its pair sums; every 32 iterations
// the partials are folded into L (bounds the FP32 error growth).
template <class Acc, int M>
__device__ __forceinline__ void march_accumulate(const ProjParams& P, const RayPlan& R, int Klo,
                                                 int Khi, Acc& acc)
{
    acc.clear();
    acc.lt = R.Lt;
    if (R.first_idx >= 0) acc.first(R.first_idx, R.first_len);
    for (int k0 = Klo; k0 <= Khi; k0 += 32) {
        const int k1 = min(Khi, k0 + 31);
        march(P, R, k0, k1, acc);
        acc.fold();
    }
}

__device__ __forceinline__ void load_spectrum(const SpectrumDev& sp, float4* s_mu, float* s_pdf)
{
    for (int e = threadIdx.x + threadIdx.y * blockDim.x; e < sp.NE; e += blockDim.x * blockDim.y) {
        s_mu[2 * e] = sp.mu8[2 * e];
        s_mu[2 * e + 1] = sp.mu8[2 * e + 1];
        s_pdf[e] = sp.pdf[e];
    }
}

template <int M>
__device__ __forceinline__ float spectral_sum(const float4* s_mu, const float* s_pdf, int NE,
                                              const float* L)
{
    float acc = 0.0f;
    for (int e = 0; e < NE; e++) {
        const float4 a = s_mu[2 * e], b = s_mu[2 * e + 1];
        float T = a.x * L[0];
        T = fmaf(a.y, L[1], T);
        T = fmaf(a.z, L[2], T);
        T = fmaf(a.w, L[3], T);
        T = fmaf(b.x, L[4], T);
        T = fmaf(b.y, L[5], T);
        if (M > 6) {
            T = fmaf(b.z, L[6 % M], T);
            T = fmaf(b.w, L[7 % M], T);
        }
        acc = fmaf(s_pdf[e], expf(-T), acc);
    }
    return acc;
}

// Warp-uniform iteration range: the union over the warp's lanes.
__device__ __forceinline__ void warp_range(const RayPlan& R, bool valid, int& Klo, int& Khi)
{
    const int lo = (valid && R.active) ? R.klo : INT_MAX;
    const int hi = (valid && R.active) ? R.khi : -1;
    Klo = __reduce_min_sync(0xffffffffu, lo);
    Khi = __reduce_max_sync(0xffffffffu, hi);
}

// Iterations [klo, khi] narrowed to those whose segments can lie in volume
// rows iy in [y0, y1): the ray's y cell cy = floor(D or O) is linear in t
// (iy = nym - 1 - cy), two cells of margin each way; the interval march
// computes every step's cells from t alone, so a narrowed range gives the
// same segments as the whole ray.
__device__ __forceinline__ void strip_iterations(const ProjParams& P, const RayPlan& R, int y0, int y1, int& klo,
                                                 int& khi)
{
    const int nym = (int)(P.N * 0.5);
    const double ca = (double)(nym - y1 - 2), cb = (double)(nym - y0 + 2);  // cy range, with margin
    double ta, tb;
    if (R.d) {                       // y dominant: cy = floor(D0 + pha t)
        ta = (ca - R.D0) * R.pha;
        tb = (cb - R.D0) * R.pha;
    } else if (R.O1 != 0.0) {        // cy = floor(O0 + O1 t)
        ta = (ca - R.O0) * R.invO1;
        tb = (cb - R.O0) * R.invO1;
    } else {                         // constant y
        if (!(R.O0 >= ca && R.O0 <= cb)) khi = klo - 1;
        return;
    }
    if (ta > tb) {
        const double t = ta;
        ta = tb;
        tb = t;
    }
    if (!(tb >= (double)(klo - 1)) || !(ta <= (double)khi)) {
        khi = klo - 1;
        return;
    }
    klo = max(klo, (int)floor(ta));
    khi = min(khi, (int)ceil(tb) + 1);
}

__device__ __forceinline__ void warp_range_k(int klo, int khi, bool use, int& Klo, int& Khi)
{
    Klo = __reduce_min_sync(0xffffffffu, use && klo <= khi ? klo : INT_MAX);
    Khi = __reduce_max_sync(0xffffffffu, use && klo <= khi ? khi : -1);
}

// grid: (ceil(W / cols_per_block), ceil(H / 32), V); block: (32, cols_per_block).
// Per-element path integrals of one ray (first segment + iterations
// [Klo, Khi]).  The interval march is used unless a lane of the warp has
// |Z1| >= 1 (more than one z plane per step), where the per-step march keeps
// the reference's last-plane-only split.  R.active is warp-uniform.
template <class Acc, int M>
__device__ __forceinline__ void ray_integrals(const ProjParams& P, const RayPlan& R, bool act,
                                              int Klo, int Khi, IvRec* wbuf, Acc& acc)
{
    acc.clear();
    if (!R.active) return;
    const bool steep = __any_sync(0xffffffffu, fabs(R.Z1) >= 1.0);
    if (steep) {
        march_accumulate<Acc, M>(P, R, Klo, Khi, acc);
        if (!act) acc.zero_L();
        return;
    }
    acc.lt = R.Lt;
    if (act && R.first_idx >= 0) acc.first(R.first_idx, R.first_len);
    auto fold = [&]() { acc.fold(); };
    const XyPlan& xp = publish_plan(R, wbuf);
    if (Klo <= Khi) march_intervals(P, R, xp, act, Klo, Khi, wbuf, acc, fold);
    fold();
}

// One work tile of the forward projection: detector columns
// [colb*cpb, colb*cpb + cpb) (one per warp), rows [rowt*32, rowt*32 + 32) (one
// per lane) of view v.  The spectrum table must already be in shared memory.
template <int M, bool F32VOL, bool COUNT>
__device__ __forceinline__ void forward_tile(const ForwardArgs& a, const float4* s_mu, const float* s_pdf,
                                             IvRec* s_iv, int v, int rowt, int colb)
{
    const ProjParams& P = a.p;
    const int lane = threadIdx.x;
    const int jj = colb * blockDim.y + threadIdx.y;  // detector column
    if (jj >= P.W) return;                           // whole warp exits together
    const int j = rowt * 32 + lane;                  // detector row
    const bool valid = j < P.H;
    IvRec* wbuf = s_iv + threadIdx.y * kIvSlots;

    const ViewGeom vg = a.views[v];
    RayPlan R;
    ray_setup(P, vg, j, jj, R);
    int Klo, Khi;
    warp_range(R, valid, Klo, Khi);

    float L[M];
    unsigned nseg = 0;
    float* s_L = reinterpret_cast<float*>(s_iv + blockDim.y * kIvSlots) + threadIdx.y * 32 + lane;
    if (F32VOL) {
        AccumF32<M, true> acc(a.vol_f32, s_L);
        ray_integrals<AccumF32<M, true>, M>(P, R, valid, Klo, Khi, wbuf, acc);
#pragma unroll
        for (int i = 0; i < M; i++) L[i] = acc.Lget(i);
        nseg = acc.nseg;
    } else {
        AccumU16<M> acc(a.vol_u16, s_L);
        ray_integrals<AccumU16<M>, M>(P, R, valid, Klo, Khi, wbuf, acc);
#pragma unroll
        for (int i = 0; i < M; i++) L[i] = acc.Lget(i);
        nseg = acc.nseg;
    }
    if (COUNT) {
        unsigned tot = __reduce_add_sync(0xffffffffu, valid ? nseg : 0u);
        if (lane == 0 && tot) atomicAdd(a.seg_count, (unsigned long long)tot);
    }
    if (!valid) return;
    const size_t o = ((size_t)v * P.H + (P.H - 1 - j)) * P.W + jj;
    if (a.L_out) {
#pragma unroll
        for (int i = 0; i < M; i++)
            if (i < P.nmat) a.L_out[o * P.nmat + i] = L[i];
    }
    if (a.out) {
        float I = spectral_sum<M>(s_mu, s_pdf, a.spec.NE, L) * R.leng;
        if (a.noise_kind != 0) {
            const uint64_t gidx = ((uint64_t)(v + a.view_offset) * P.H + (P.H - 1 - j)) * P.W + jj;
            I = (a.noise_kind == 1) ? noisy_intensity(I, a.noise_i0, a.noise_max, gidx, a.noise_seed)
                                    : poisson_intensity(I, a.noise_i0, a.noise_max, gidx, a.noise_seed);
        }
        a.out[o] = I;
    }
}

__device__ __forceinline__ IvRec* iv_buffer(float4* smem, int NEmax)
{
    return reinterpret_cast<IvRec*>(smem + 2 * NEmax + (NEmax + 3) / 4);
}

// grid: (ceil(W / cols_per_block), V, ceil(H / 32)); block: (32, cols_per_block).
// Blocks are dispatched view-fastest within a band of 32 detector rows, so
// the blocks resident at a time share one z band of the volume (L2 reuse
// across views).
// Register cap of the forward kernel: minimum resident 256-thread blocks per
// SM (0 leaves the choice to the compiler).  The march is bound by the
// latency of its L2 gathers, so occupancy pays more than registers: 5 blocks
// (48 registers, 40 warps per SM) measured 26 % faster on B200 than the
// compiler's own choice (80 registers, 24 warps), although the rarely taken
// paths then spill; with the long-term sums L in shared memory (six
// registers freed), 6 blocks (40 registers, 48 warps) run the 512x512x200 /
// 360-view projection in 45.7 ms against 48.6 ms at 5 (7 blocks: 50.5 ms),
// and its FP32-volume form in 45.0 ms against 48.1 ms.
#ifndef VCBCT_FWD_MIN_BLOCKS
#define VCBCT_FWD_MIN_BLOCKS 6
#endif
#if VCBCT_FWD_MIN_BLOCKS > 0
#define VCBCT_FWD_BOUNDS __launch_bounds__(256, VCBCT_FWD_MIN_BLOCKS)
#else
#define VCBCT_FWD_BOUNDS __launch_bounds__(256)
#endif
template <int M, bool F32VOL, bool COUNT>
__global__ void __launch_bounds__(256, VCBCT_FWD_MIN_BLOCKS)
    forward_kernel(ForwardArgs a)
{
    extern __shared__ float4 smem[];
    float4* s_mu = smem;
    float* s_pdf = reinterpret_cast<float*>(smem + 2 * a.spec.NE);
    load_spectrum(a.spec, s_mu, s_pdf);
    __syncthreads();
    forward_tile<M, F32VOL, COUNT>(a, s_mu, s_pdf, iv_buffer(smem, a.spec.NE), blockIdx.y, a.band0 + blockIdx.z,
                                   blockIdx.x);
}

// Slices each detector row band can read, reduced over the band's rays of
// every view.  Conservative: the z cells of the ray's line over the
// iterations [klo - 1, khi] it marches (the warp-wide march reads nothing
// outside them), one cell of margin each way, and the first segment's slice.
// grid: (ceil(W / 8), V, ceil(H / 32)); block: (32, 8).
__global__ void __launch_bounds__(256) band_footprint_kernel(ProjParams P, const ViewGeom* __restrict__ views,
                                                             int* __restrict__ span)
{
    const int jj = blockIdx.x * 8 + threadIdx.y, j = blockIdx.z * 32 + threadIdx.x;
    int lo = INT_MAX, hi = -1;
    if (jj < P.W && j < P.H) {
        RayPlan R;
        ray_setup(P, views[blockIdx.y], j, jj, R);
        if (R.active) {
            if (R.first_idx >= 0) {
                const int z = R.first_idx % P.Z;
                lo = min(lo, z);
                hi = max(hi, z);
            }
            if (R.klo <= R.khi) {
                const int nzm = (int)(P.Z * 0.5);
                const double za = R.Z0 + R.Z1 * (double)(R.klo - 1), zb = R.Z0 + R.Z1 * (double)R.khi;
                const double zmin = fmin(za, zb), zmax = fmax(za, zb);
                // slice q = nzm - 1 - floor(z) (q = -1 reads slice 0)
                const double qlo = (double)(nzm - 2) - floor(zmax), qhi = (double)nzm - floor(zmin);
                if (qhi >= -1.0 && qlo <= (double)(P.Z - 1)) {
                    lo = min(lo, (int)fmax(0.0, qlo));
                    hi = max(hi, (int)fmax(0.0, fmin(qhi, (double)(P.Z - 1))));
                }
            }
        }
    }
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    if (threadIdx.x == 0 && hi >= 0) {
        atomicMin(span + 2 * blockIdx.z, lo);
        atomicMax(span + 2 * blockIdx.z + 1, hi);
    }
}

// Single-launch batched forward projection: one block per work tile of every
// item, the items' arguments in the launch's parameter block.  A block finds
// its item by a binary search over the items' first tiles; the index only
// depends on blockIdx, so the item's arguments are read from the parameter
// bank like forward_kernel's and cost no registers per thread.
template <int M>
__global__ void VCBCT_FWD_BOUNDS flat_batch_kernel(const __grid_constant__ FlatBatch b)
{
    extern __shared__ float4 smem[];
    const long long u = blockIdx.x;
    int lo = 0, hi = b.nitems - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (b.begin[mid] <= u) lo = mid;
        else hi = mid - 1;
    }
    const ForwardArgs& fa = b.fa[lo];
    float4* s_mu = smem;
    float* s_pdf = reinterpret_cast<float*>(smem + 2 * fa.spec.NE);
    load_spectrum(fa.spec, s_mu, s_pdf);
    __syncthreads();
    const long long w = u - b.begin[lo];
    const int colb = (int)(w % b.ncolb[lo]);
    const long long rest = w / b.ncolb[lo];
    const int v = (int)(rest % fa.p.V);
    const int rowt = (int)(rest / fa.p.V);
    forward_tile<M, true, false>(fa, s_mu, s_pdf, iv_buffer(smem, fa.spec.NE), v, rowt, colb);
}

// Persistent batched forward projection: a grid of as many blocks as fit on
// the GPU at once, every block repeatedly taking the next work tile from a
// global counter.  Tiles are numbered item by item, and within an item by
// row band, then view, then column block (the order of forward_kernel's
// grid), so the items' uneven view and slice counts load-balance across the
// whole GPU in one launch.  The items' arguments sit in the launch's
// parameter block as for flat_batch_kernel: the march reads them from the
// parameter bank (a block-uniform index found by a binary search), so they
// hold no registers; a block reloads the spectrum table only when its next
// tile belongs to another item.
template <int M>
__global__ void VCBCT_FWD_BOUNDS persistent_batch_kernel(const __grid_constant__ FlatBatch b,
                                                         unsigned long long* counter, int NEmax)
{
    extern __shared__ float4 smem[];
    __shared__ long long s_unit;
    float4* s_mu = smem;
    float* s_pdf = reinterpret_cast<float*>(smem + 2 * NEmax);
    IvRec* s_iv = iv_buffer(smem, NEmax);
    const long long total = b.begin[b.nitems];
    int cur = -1;
    for (;;) {
        if (threadIdx.x == 0 && threadIdx.y == 0) s_unit = (long long)atomicAdd(counter, 1ull);
        __syncthreads();
        const long long u = s_unit;
        if (u >= total) break;  // block-uniform
        int lo = 0, hi = b.nitems - 1;  // last item with begin <= u
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (b.begin[mid] <= u) lo = mid;
            else hi = mid - 1;
        }
        if (lo != cur) {  // block-uniform
            load_spectrum(b.fa[lo].spec, s_mu, s_pdf);
            cur = lo;
        }
        __syncthreads();
        const long long w = u - b.begin[lo];
        const int colb = (int)(w % b.ncolb[lo]);
        const long long rest = w / b.ncolb[lo];
        const int v = (int)(rest % b.fa[lo].p.V);
        const int rowt = (int)(rest / b.fa[lo].p.V);
        forward_tile<M, true, false>(b.fa[lo], s_mu, s_pdf, s_iv, v, rowt, colb);
        __syncthreads();
    }
}

// Register cap of the adjoint (minimum resident 256-thread blocks per SM):
// 3 (80 registers) and 4 (64) measured within 1.5 % on B200, 5 (48) 15 %
// slower; 3 is kept.
#ifndef VCBCT_ADJ_MIN_BLOCKS
#define VCBCT_ADJ_MIN_BLOCKS 3
#endif
template <int M>
__global__ void __launch_bounds__(256, VCBCT_ADJ_MIN_BLOCKS) adjoint_kernel(AdjointArgs a)
{
    extern __shared__ float4 smem[];
    float4* s_mu = smem;
    float* s_pdf = reinterpret_cast<float*>(smem + 2 * a.spec.NE);
    IvRec* s_iv = reinterpret_cast<IvRec*>(smem + 2 * a.spec.NE + (a.spec.NE + 3) / 4);
    load_spectrum(a.spec, s_mu, s_pdf);
    __syncthreads();

    const ProjParams& P = a.p;
    const int lane = threadIdx.x;
    const int colb = blockIdx.x, v = blockIdx.y, rowt = blockIdx.z;
    const int jj = colb * blockDim.y + threadIdx.y;
    if (jj >= P.W) return;
    const int j = rowt * 32 + lane;
    const bool valid = j < P.H;
    IvRec* wbuf = s_iv + threadIdx.y * kIvSlots;
    const ViewGeom vg = a.views[v];
    RayPlan R;
    ray_setup(P, vg, j, jj, R);
    float r = 0.0f;
    if (valid) r = a.grad_out[((size_t)v * P.H + (P.H - 1 - j)) * P.W + jj];
    const bool act = valid && r != 0.0f;
    int Klo, Khi;
    // rays with a zero residual do not scatter
    warp_range(R, act, Klo, Khi);
    if (!__any_sync(0xffffffffu, act && R.active)) return;
    // a warp none of whose segments can lie in the strip stops here (before
    // recomputing or reading its path integrals)
    const bool strip = a.y1 > a.y0;
    const bool steep = R.active && __any_sync(0xffffffffu, fabs(R.Z1) >= 1.0);
    int Klo2 = Klo, Khi2 = Khi;
    if (strip && R.active && !steep) {
        int klo = R.klo, khi = R.khi;
        strip_iterations(P, R, a.y0, a.y1, klo, khi);
        warp_range_k(klo, khi, act, Klo2, Khi2);
        const unsigned NZ = (unsigned)P.N * (unsigned)P.Z;
        const bool first_in = act && R.first_idx >= 0 &&
                              (unsigned)R.first_idx - (unsigned)a.y0 * NZ < (unsigned)(a.y1 - a.y0) * NZ;
        if (Klo2 > Khi2 && !__any_sync(0xffffffffu, first_in)) return;
    }

    // pass 1: the per-element path integrals of this ray, recomputed by a
    // first march or read from the forward projection that made them
    AccumF32<M> acc(a.vol_f32);
    if (a.L_in) {
        if (act) {
            const float* Lr = a.L_in + (((size_t)v * P.H + (P.H - 1 - j)) * P.W + jj) * P.nmat;
#pragma unroll
            for (int i = 0; i < M; i++)
                if (i < P.nmat) acc.L[i] = Lr[i];
        }
    } else {
        ray_integrals<AccumF32<M>, M>(P, R, act, Klo, Khi, wbuf, acc);
    }

    // d I / d L_k = -leng * sum_E pdf_E mu'_k(E) exp(-sum_k mu'_k(E) L_k)
    float g[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int e = 0; e < a.spec.NE; e++) {
        const float4 m0 = s_mu[2 * e], m1 = s_mu[2 * e + 1];
        float T = m0.x * acc.L[0];
        T = fmaf(m0.y, acc.L[1], T);
        T = fmaf(m0.z, acc.L[2], T);
        T = fmaf(m0.w, acc.L[3], T);
        T = fmaf(m1.x, acc.L[4], T);
        T = fmaf(m1.y, acc.L[5], T);
        if (M > 6) {
            T = fmaf(m1.z, acc.L[6 % M], T);
            T = fmaf(m1.w, acc.L[7 % M], T);
        }
        // the hardware exponential (relative error ~1e-6, far inside the
        // gradient's 1e-5 bar): this loop runs once per ray and strip
        const float w = s_pdf[e] * __expf(-T);
        g[0] = fmaf(w, m0.x, g[0]); g[1] = fmaf(w, m0.y, g[1]);
        g[2] = fmaf(w, m0.z, g[2]); g[3] = fmaf(w, m0.w, g[3]);
        g[4] = fmaf(w, m1.x, g[4]); g[5] = fmaf(w, m1.y, g[5]);
        g[6] = fmaf(w, m1.z, g[6]); g[7] = fmaf(w, m1.w, g[7]);
    }
    const float scale = -R.leng * r;
    const unsigned NZ = (unsigned)P.N * (unsigned)P.Z;
    Scatter<M> sc{a.grad_planes, (size_t)P.N * P.N * P.Z, P.nmat, {},
                  strip ? (unsigned)a.y0 * NZ : 0u, strip ? (unsigned)(a.y1 - a.y0) * NZ : 0xffffffffu, R.Lt};
#pragma unroll
    for (int i = 0; i < 8; i++) sc.g[i] = g[i] * scale;
    // pass 2: scatter along the same segments
    if (!R.active) return;
    if (steep) {  // the whole ray (its per-step state depends on where it starts), filtered
        if (act) {
            if (R.first_idx >= 0) sc.first(R.first_idx, R.first_len);
            if (Klo <= Khi) march(P, R, Klo, Khi, sc);
        }
        return;
    }
    if (act && R.first_idx >= 0) sc.first(R.first_idx, R.first_len);
    // only the iterations whose segments can lie in the strip's rows
    const XyPlan& xp = publish_plan(R, wbuf);
    if (Klo2 <= Khi2) march_intervals(P, R, xp, act, Klo2, Khi2, wbuf, sc, []() {});
}

// ------------------------------------------------------- layout kernels --
// Reference layout [Z][nmat][N][N] -> packed z-fastest records.
// grid (ceil(N/32), N, ceil(Z/32)), block (32, 8).
// A slab of nz slices [zoff, zoff + nz) of a Z-slice volume: src holds the
// slab [nz][nmat][N][N], dst the whole packed volume.  F32REC: the values as
// floats (exact for uint16) in two 16-byte records per voxel, the layout of
// pack_f32_kernel; otherwise one 16-byte record of eight uint16.
template <bool F32REC>
__global__ void pack_u16_kernel(const uint16_t* __restrict__ src, int N, int nz, int zoff, int Z, int nmat,
                                void* __restrict__ dst)
{
    __shared__ uint16_t tile[32][8][33];
    const int x0 = blockIdx.x * 32, y = blockIdx.y, z0 = blockIdx.z * 32;
    const size_t NN = (size_t)N * N;
    for (int zz = threadIdx.y; zz < 32; zz += 8) {
        const int z = z0 + zz, x = x0 + threadIdx.x;
        for (int m = 0; m < 8; m++) {
            uint16_t v = 0;
            if (m < nmat && z < nz && x < N) v = src[((size_t)z * nmat + m) * NN + (size_t)y * N + x];
            tile[zz][m][threadIdx.x] = v;
        }
    }
    __syncthreads();
    for (int xx = threadIdx.y; xx < 32; xx += 8) {
        const int x = x0 + xx, z = z0 + threadIdx.x;
        if (x >= N || z >= nz) continue;
        const int zz = threadIdx.x;
        const size_t o = ((size_t)y * N + x) * Z + zoff + z;
        if (F32REC) {
            float4* p = static_cast<float4*>(dst) + 2 * o;
            p[0] = make_float4(tile[zz][0][xx], tile[zz][1][xx], tile[zz][2][xx], tile[zz][3][xx]);
            p[1] = make_float4(tile[zz][4][xx], tile[zz][5][xx], tile[zz][6][xx], tile[zz][7][xx]);
        } else {
            uint4 r;
            r.x = (uint32_t)tile[zz][0][xx] | ((uint32_t)tile[zz][1][xx] << 16);
            r.y = (uint32_t)tile[zz][2][xx] | ((uint32_t)tile[zz][3][xx] << 16);
            r.z = (uint32_t)tile[zz][4][xx] | ((uint32_t)tile[zz][5][xx] << 16);
            r.w = (uint32_t)tile[zz][6][xx] | ((uint32_t)tile[zz][7][xx] << 16);
            static_cast<uint4*>(dst)[o] = r;
        }
    }
}

// A thin slab (nz <= 8 slices) of uint16 -> float records: thread t of a
// 256-thread block makes record (y, x0 + t / 8, zoff + t % 8), so a warp
// writes four runs of 8 consecutive records (256 bytes each) and every lane
// has work; the tiled kernel above gives a slab of 8 slices a quarter of its
// lanes.  Reads go straight to global memory (the block's 32 x 8 values of
// an element row share their sectors in L1).  grid (ceil(N/32), N).
__global__ void __launch_bounds__(256) pack_u16_f32_thin_kernel(const uint16_t* __restrict__ src, int N, int nz,
                                                                int zoff, int Z, int nmat, float4* __restrict__ dst)
{
    const int t = threadIdx.x;
    const int z = t & 7, x = blockIdx.x * 32 + (t >> 3), y = blockIdx.y;
    if (z >= nz || x >= N) return;
    const size_t NN = (size_t)N * N;
    const uint16_t* s = src + (size_t)z * nmat * NN + (size_t)y * N + x;
    float e[8];
#pragma unroll
    for (int m = 0; m < 8; m++) e[m] = m < nmat ? (float)__ldg(s + (size_t)m * NN) : 0.0f;
    float4* p = dst + 2 * (((size_t)y * N + x) * Z + zoff + z);
    p[0] = make_float4(e[0], e[1], e[2], e[3]);
    p[1] = make_float4(e[4], e[5], e[6], e[7]);
}

__global__ void pack_f32_kernel(const float* __restrict__ src, int N, int Z, int nmat,
                                float4* __restrict__ dst)
{
    __shared__ float tile[32][8][33];
    const int x0 = blockIdx.x * 32, y = blockIdx.y, z0 = blockIdx.z * 32;
    const size_t NN = (size_t)N * N;
    for (int zz = threadIdx.y; zz < 32; zz += 8) {
        const int z = z0 + zz, x = x0 + threadIdx.x;
        for (int m = 0; m < 8; m++) {
            float v = 0.0f;
            if (m < nmat && z < Z && x < N) v = src[((size_t)z * nmat + m) * NN + (size_t)y * N + x];
            tile[zz][m][threadIdx.x] = v;
        }
    }
    __syncthreads();
    for (int xx = threadIdx.y; xx < 32; xx += 8) {
        const int x = x0 + xx, z = z0 + threadIdx.x;
        if (x >= N || z >= Z) continue;
        const int zz = threadIdx.x;
        float4* p = dst + 2 * (((size_t)y * N + x) * Z + z);
        p[0] = make_float4(tile[zz][0][xx], tile[zz][1][xx], tile[zz][2][xx], tile[zz][3][xx]);
        p[1] = make_float4(tile[zz][4][xx], tile[zz][5][xx], tile[zz][6][xx], tile[zz][7][xx]);
    }
}

// packed float records -> [Z][nmat][N][N], accumulated (+=).
// element planes [nmat][(y*N + x)*Z + z] -> [Z][nmat][N][N], accumulated (+=).
// grid (ceil(N/32), N, ceil(Z/32) * nmat), block (32, 8): a 32 x 32 (x, z)
// tile of one plane through shared memory.
__global__ void unpack_grad_kernel(const float* __restrict__ src, int N, int Z, int nmat,
                                   float* __restrict__ dst)
{
    __shared__ float tile[32][33];
    const int zt = (Z + 31) / 32;
    const int m = blockIdx.z / zt;
    const int x0 = blockIdx.x * 32, y = blockIdx.y, z0 = (blockIdx.z % zt) * 32;
    const size_t NN = (size_t)N * N;
    // element m is slot m % 4 of the group starting at element 4 (m / 4),
    // four wide, or two for a last group of one or two elements (see Scatter)
    const int e0 = (m / 4) * 4, wdt = nmat - e0 > 2 ? 4 : 2;
    const float* plane = src + (size_t)e0 * NN * Z + (m % 4);
    for (int xx = threadIdx.y; xx < 32; xx += 8) {
        const int x = x0 + xx, z = z0 + threadIdx.x;
        tile[threadIdx.x][xx] = (x < N && z < Z) ? plane[(((size_t)y * N + x) * Z + z) * wdt] : 0.0f;
    }
    __syncthreads();
    for (int zz = threadIdx.y; zz < 32; zz += 8) {
        const int z = z0 + zz, x = x0 + threadIdx.x;
        if (z >= Z || x >= N) continue;
        dst[((size_t)z * nmat + m) * NN + (size_t)y * N + x] += tile[zz][threadIdx.x];
    }
}

}  // namespace

cudaError_t launch_pack_u16(const uint16_t* src, int N, int Z, int nmat, uint4* dst, cudaStream_t st)
{
    dim3 grid((N + 31) / 32, N, (Z + 31) / 32), block(32, 8);
    pack_u16_kernel<false><<<grid, block, 0, st>>>(src, N, Z, 0, Z, nmat, dst);
    return cudaGetLastError();
}

cudaError_t launch_pack_u16_f32_slab(const uint16_t* src, int N, int nz, int zoff, int Z, int nmat, float4* dst,
                                     cudaStream_t st)
{
    if (nz <= 8) {
        pack_u16_f32_thin_kernel<<<dim3((N + 31) / 32, N), 256, 0, st>>>(src, N, nz, zoff, Z, nmat, dst);
        return cudaGetLastError();
    }
    dim3 grid((N + 31) / 32, N, (nz + 31) / 32), block(32, 8);
    pack_u16_kernel<true><<<grid, block, 0, st>>>(src, N, nz, zoff, Z, nmat, dst);
    return cudaGetLastError();
}

cudaError_t launch_pack_f32(const float* src, int N, int Z, int nmat, float4* dst, cudaStream_t st)
{
    dim3 grid((N + 31) / 32, N, (Z + 31) / 32), block(32, 8);
    pack_f32_kernel<<<grid, block, 0, st>>>(src, N, Z, nmat, dst);
    return cudaGetLastError();
}

cudaError_t launch_unpack_grad(const float* planes, int N, int Z, int nmat, float* dst, cudaStream_t st)
{
    dim3 grid((N + 31) / 32, N, ((Z + 31) / 32) * nmat), block(32, 8);
    unpack_grad_kernel<<<grid, block, 0, st>>>(planes, N, Z, nmat, dst);
    return cudaGetLastError();
}

template <int M, bool F32VOL, bool COUNT>
static cudaError_t launch_fwd_t(const ForwardArgs& a, cudaStream_t st)
{
    const int cpb = a.cols_per_block;
    dim3 block(32, cpb);
    dim3 grid((a.p.W + cpb - 1) / cpb, a.p.V, a.nbands > 0 ? a.nbands : (a.p.H + 31) / 32);
    size_t shm = ((size_t)2 * a.spec.NE + (a.spec.NE + 3) / 4) * sizeof(float4) +
                 (size_t)cpb * kIvSlots * sizeof(IvRec) + (size_t)M * 32 * cpb * sizeof(float);
    auto k = forward_kernel<M, F32VOL, COUNT>;
    if (shm > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
        if (e != cudaSuccess) return e;
    }
    k<<<grid, block, shm, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_persistent_batch(const FlatBatch& b, int NEmax, int nmat_max, int cols_per_block, int blocks,
                                   unsigned long long* counter, cudaStream_t st)
{
    if (b.begin[b.nitems] <= 0) return cudaSuccess;
    dim3 block(32, cols_per_block);
    size_t shm = ((size_t)2 * NEmax + (NEmax + 3) / 4) * sizeof(float4) +
                 (size_t)cols_per_block * kIvSlots * sizeof(IvRec) + (size_t)8 * 32 * cols_per_block * sizeof(float);
    // (the shared-memory attribute is set by batch_blocks_per_sm, before any
    // stream capture)
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    auto k = (nmat_max <= 6) ? persistent_batch_kernel<6> : persistent_batch_kernel<8>;
    k<<<blocks, block, shm, st>>>(b, counter, NEmax);
    return cudaGetLastError();
}

cudaError_t launch_flat_batch(const FlatBatch& b, int NEmax, int nmat_max, int cols_per_block, cudaStream_t st)
{
    const long long total = b.begin[b.nitems];
    if (total <= 0) return cudaSuccess;
    if (total > 0x7fffffffLL) return cudaErrorInvalidValue;
    dim3 block(32, cols_per_block);
    size_t shm = ((size_t)2 * NEmax + (NEmax + 3) / 4) * sizeof(float4) +
                 (size_t)cols_per_block * kIvSlots * sizeof(IvRec) + (size_t)8 * 32 * cols_per_block * sizeof(float);
    auto k = (nmat_max <= 6) ? flat_batch_kernel<6> : flat_batch_kernel<8>;
    // (the shared-memory attribute is set by batch_blocks_per_sm, before any
    // stream capture)
    k<<<(unsigned)total, block, shm, st>>>(b);
    return cudaGetLastError();
}

int batch_blocks_per_sm(int nmat_max, int cols_per_block, int NEmax)
{
    size_t shm = ((size_t)2 * NEmax + (NEmax + 3) / 4) * sizeof(float4) +
                 (size_t)cols_per_block * kIvSlots * sizeof(IvRec) + (size_t)8 * 32 * cols_per_block * sizeof(float);
    int n = 0;
    auto k = (nmat_max <= 6) ? persistent_batch_kernel<6> : persistent_batch_kernel<8>;
    if (shm > 48 * 1024 && cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm) != cudaSuccess)
        return 0;
    auto kf = (nmat_max <= 6) ? flat_batch_kernel<6> : flat_batch_kernel<8>;
    if (shm > 48 * 1024 && cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm) != cudaSuccess)
        return 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, 32 * cols_per_block, shm);
    return n;
}

cudaError_t launch_band_footprint(const ProjParams& P, const ViewGeom* d_views, int* d_span, cudaStream_t st)
{
    dim3 grid((P.W + 7) / 8, P.V, (P.H + 31) / 32), block(32, 8);
    band_footprint_kernel<<<grid, block, 0, st>>>(P, d_views, d_span);
    return cudaGetLastError();
}

cudaError_t launch_forward(const ForwardArgs& a, cudaStream_t st)
{
    const bool f32 = a.vol_f32 != nullptr;
    const bool cnt = a.seg_count != nullptr;
    if (a.p.nmat <= 6) {
        if (f32) return cnt ? launch_fwd_t<6, true, true>(a, st) : launch_fwd_t<6, true, false>(a, st);
        return cnt ? launch_fwd_t<6, false, true>(a, st) : launch_fwd_t<6, false, false>(a, st);
    }
    if (f32) return cnt ? launch_fwd_t<8, true, true>(a, st) : launch_fwd_t<8, true, false>(a, st);
    return cnt ? launch_fwd_t<8, false, true>(a, st) : launch_fwd_t<8, false, false>(a, st);
}

template <int M>
static cudaError_t launch_adj_t(const AdjointArgs& a, cudaStream_t st)
{
    const int cpb = a.cols_per_block;
    dim3 block(32, cpb);
    // the forward's block order; (columns, row bands, views) and (views,
    // columns, row bands) measured within 3 % on B200
    dim3 grid((a.p.W + cpb - 1) / cpb, a.p.V, (a.p.H + 31) / 32);
    size_t shm = ((size_t)2 * a.spec.NE + (a.spec.NE + 3) / 4) * sizeof(float4) +
                 (size_t)cpb * kIvSlots * sizeof(IvRec);
    auto k = adjoint_kernel<M>;
    if (shm > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
        if (e != cudaSuccess) return e;
    }
    k<<<grid, block, shm, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_adjoint(const AdjointArgs& a, cudaStream_t st)
{
    return a.p.nmat <= 6 ? launch_adj_t<6>(a, st) : launch_adj_t<8>(a, st);
}

}  // namespace vcbct
