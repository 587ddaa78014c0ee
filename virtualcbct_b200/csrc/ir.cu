// ir.cu -- the building blocks of the reference's iterative reconstruction on
// sm_100a:
//   lengthproj_kernel  voxel-driven sensitivity backprojection of uint16
//                      projections weighted by each voxel's chord length
//                      (Release_CBCT_Projection_CM/lengthproj.cpp:10-131)
//   ir_update_kernel   the MLEM-type multiplicative update with a total
//                      variation penalty (IR_ImageCBCT.cpp:19-93)
//
// Both follow the reference's double arithmetic operation by operation; this
// file is compiled with -fmad=false so that nvcc does not contract products
// and sums into FMAs, and the results are bitwise those of the reference's
// g++ build.  One thread per voxel; lengthproj walks the views in order and
// accumulates in float as the reference does, so the per-voxel sums have the
// same order too.
#include "internal.h"

namespace vcbct {
namespace {

constexpr double kMaxPixValue = 65535.0;  // MAX_PIXVALUE, P/physParams.h:63

// Per-view constants of lengthproj (independent of the voxel).
struct LpView {
    double sx, sy, ox, oy, sn, cs, xshift, yshift, go;  // go = (oy-sy)/(ox-sx)
};

__global__ void lengthproj_views_kernel(const ViewGeom* __restrict__ views, int v0, int nv, LpParams q,
                                        LpView* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv) return;
    const ViewGeom g = views[v0 + i];
    LpView w;
    w.sn = g.sn;
    w.cs = g.cs;
    w.sx = -q.sad * g.sn + q.xr;
    w.sy = q.sad * g.cs + q.yr;
    w.ox = w.sx + q.pdet / q.piso * g.sn * q.sad;
    w.oy = w.sy - q.pdet / q.piso * g.cs * q.sad;
    w.go = (w.oy - w.sy) / (w.ox - w.sx);
    const double bin = q.pdet * (q.dpn / q.H);
    w.xshift = -(g.xc + q.H / 2.0) * bin;
    w.yshift = -(g.yc + q.H / 2.0) * bin;
    out[i] = w;
}

// grid (ceil(N / 32), ceil(N / 8), Z), block (32, 8)
__global__ void __launch_bounds__(256) lengthproj_kernel(LpParams q, const LpView* __restrict__ vw, int v0, int nv,
                                                         const uint16_t* __restrict__ proj, float* __restrict__ npf)
{
    const int jx = blockIdx.x * 32 + threadIdx.x, jy = blockIdx.y * 8 + threadIdx.y, jz = blockIdx.z;
    if (jx >= q.N || jy >= q.N) return;
    const double s = q.s, step = q.step;
    const double rz = q.Z * step * 0.5 - (jz + 0.5) * step;
    const double ry = q.N * s * 0.5 - (jy + 0.5) * s;
    const double rx = -q.N * s * 0.5 + (jx + 0.5) * s;
    const double sz = q.zr;
    const double bin = q.pdet * (q.dpn / q.H);
    const int W = q.W, H = q.H;
    const double wh = (double)((W - H) / 2) * bin;
    float acc = 0.0f;
    for (int t = 0; t < nv; t++) {
        const LpView w = vw[t];
        const double sx = w.sx, sy = w.sy;
        const double yslope = fabs(ry - sy), xslope = fabs(rx - sx);
        double rr;
        if (xslope > yslope) {
            const double xx0 = rx - 0.5 * s;
            const double yy0 = (xx0 - sx) / (rx - sx) * (ry - sy) + sy;
            const double zz0 = (xx0 - sx) / (rx - sx) * (rz - sz) + sz;
            const double xx1 = rx + 0.5 * s;
            const double yy1 = (xx1 - sx) / (rx - sx) * (ry - sy) + sy;
            const double zz1 = (xx1 - sx) / (rx - sx) * (rz - sz) + sz;
            rr = sqrt((xx0 - xx1) * (xx0 - xx1) + (yy0 - yy1) * (yy0 - yy1) + (zz0 - zz1) * (zz0 - zz1));
        } else {
            const double yy0 = ry - 0.5 * s;
            const double xx0 = (yy0 - sy) / (ry - sy) * (rx - sx) + sx;
            const double zz0 = (yy0 - sy) / (ry - sy) * (rz - sz) + sz;
            const double yy1 = ry + 0.5 * s;
            const double xx1 = (yy1 - sy) / (ry - sy) * (rx - sx) + sx;
            const double zz1 = (yy1 - sy) / (ry - sy) * (rz - sz) + sz;
            rr = sqrt((xx0 - xx1) * (xx0 - xx1) + (yy0 - yy1) * (yy0 - yy1) + (zz0 - zz1) * (zz0 - zz1));
        }
        // the voxel centre's projection on the detector line (lengthproj.cpp:76-94)
        const double py = (w.ox - rx + (sx - rx) / (sy - ry) * ry + w.go * w.oy) / ((sx - rx) / (sy - ry) + w.go);
        const double px = ((sx - rx) / (sy - ry) * (py - ry) + rx);
        const double pz = ((sz - rz) / (sy - ry) * (py - ry) + rz);
        const double vv = -(pz - q.zr - w.yshift);
        const double uu = (px - q.xr) * w.cs + (py - q.xr) * w.sn + w.xshift - wh;
        // non-finite or out-of-int-range positions: the reference's (int)
        // conversion yields INT_MIN there and its bounds test drops the view
        if (!(fabs(vv / bin) < 1.0e9) || !(fabs(uu / bin) < 1.0e9)) continue;
        const double vfac = vv < 0 ? -0.5 : 0.5;
        const double ufac = uu < 0 ? -0.5 : 0.5;
        const int v1 = __double2int_rz(vv / bin + vfac);
        const int u1 = __double2int_rz(uu / bin + ufac);
        const double dv1 = vv / bin - v1;
        const double du1 = uu / bin - u1;
        // (vv - v1) mixes cm and pixels as the reference does; only its sign
        // is used, and an exact zero keeps the first pixel
        int v2 = v1, u2 = u1;
        if (!(fabs(vv - v1) < 0.000000001)) v2 = v1 + ((vv - v1) > 0 ? 1 : -1);
        if (!(fabs(uu - u1) < 0.000000001)) u2 = u1 + ((uu - u1) > 0 ? 1 : -1);
        const int r1 = v1 + H / 2, r2 = v2 + H / 2, c1 = u1 + W / 2, c2 = u2 + W / 2;
        if (r1 >= 0 && r1 < H && r2 >= 0 && r2 < H && c1 >= 0 && c1 < W && c2 >= 0 && c2 < W) {
            const uint16_t* pv = proj + (size_t)(v0 + t) * W * H;
            const double p11 = pv[r1 * W + c1], p12 = pv[r2 * W + c1];
            const double p21 = pv[r1 * W + c2], p22 = pv[r2 * W + c2];
            // the reference weights the column neighbours with dv1 and the
            // row pair with du1 (lengthproj.cpp:114-116)
            const double np1 = ((1 - dv1) * p11 + dv1 * p21);
            const double np2 = ((1 - dv1) * p12 + dv1 * p22);
            const double np3 = ((1 - du1) * np1 + du1 * np2);
            const double np = (kMaxPixValue - np3);
            acc += (float)(np * rr);
        }
    }
    npf[((size_t)jz * q.N + jy) * q.N + jx] = acc;
}

__device__ __forceinline__ double tv_term(short a, short ax, short ay, short az, short ax1, short ay1, short az1,
                                          short ayx1, short azx1, short axy1, short azy1, short axz1, short ayz1)
{
    // IR_ImageCBCT.cpp:10-17: integer differences, double norms
    const double dist1 = sqrt(double((a - ax) * (a - ax) + (a - ay) * (a - ay) + (a - az) * (a - az))) + 0.00000001;
    const double dist2 =
        sqrt(double((a - ax1) * (a - ax1) + (ax1 - ayx1) * (ax1 - ayx1) + (ax1 - azx1) * (ax1 - azx1))) + 0.00000001;
    const double dist3 =
        sqrt(double((ay1 - axy1) * (ay1 - axy1) + (a - ay1) * (a - ay1) + (ay1 - azy1) * (ay1 - azy1))) + 0.00000001;
    const double dist4 =
        sqrt(double((az1 - axz1) * (az1 - axz1) + (az1 - ayz1) * (az1 - ayz1) + (a - az1) * (a - az1))) + 0.00000001;
    return ((a - ax) + (a - ay) + (a - az)) / dist1 + (a - ax1) / dist2 + (a - ay1) / dist3 + (a - az1) / dist4;
}

// grid (ceil(N / 32), ceil(N / 8), Z), block (32, 8)
__global__ void __launch_bounds__(256) ir_update_kernel(int N, int Z, double scale, const short* __restrict__ before,
                                                        float* __restrict__ out, const float* __restrict__ npf,
                                                        const float* __restrict__ npf_re, double wbefore,
                                                        double weight_tv, double weight_prior)
{
    const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    if (x >= N || y >= N) return;
    const size_t NN = (size_t)N * N;
    const size_t kk = (size_t)z * NN + (size_t)y * N + x;
    double cost_tv = 0.0;
    const double cost_prior = 0.0;
    if (z < Z - 1 && y < N - 1 && x < N - 1 && x > 0 && y > 0 && z > 0) {
        auto at = [&](int dz, int dy, int dx) { return before[kk + (long long)dz * (long long)NN + (long long)dy * N + dx]; };
        cost_tv = tv_term(at(0, 0, 0), at(0, 0, 1), at(0, 1, 0), at(1, 0, 0), at(0, 0, -1), at(0, -1, 0), at(-1, 0, 0),
                          at(0, 1, -1), at(1, 0, -1), at(0, -1, 1), at(1, -1, 0), at(-1, 0, 1), at(-1, 1, 0));
    }
    const double lambda = weight_tv * cost_tv + weight_prior * cost_prior + 0.000001;
    float v = (float)(before[kk] * (wbefore + (1 - wbefore) * npf_re[kk] / (npf[kk] + lambda)));
    if (v < 0.0) v = 0.0f;
    else if (v > 65535 / 2) v = 5000.0f;
    // the mask compares a radius in cm with half the size in voxels
    // (IR_ImageCBCT.cpp:22,85-88), as the reference does
    const double rmax = N * 0.5 * 1.0;
    const double xx = -N * scale * 0.5 + (x + 0.5) * scale;
    const double yy = N * scale * 0.5 - (y + 0.5) * scale;
    const double r = sqrt((xx) * (xx) + (yy) * (yy));
    if (r >= rmax) v = 0.0f;
    out[kk] = v;
}

}  // namespace

cudaError_t launch_lengthproj(const LpParams& q, const ViewGeom* d_views, int v0, int v1, const uint16_t* d_proj,
                              float* d_npf, void* d_scratch, cudaStream_t st)
{
    const int nv = v1 - v0;
    if (nv <= 0) return cudaSuccess;
    LpView* vw = static_cast<LpView*>(d_scratch);
    lengthproj_views_kernel<<<(nv + 127) / 128, 128, 0, st>>>(d_views, v0, nv, q, vw);
    dim3 grid((q.N + 31) / 32, (q.N + 7) / 8, q.Z), block(32, 8);
    lengthproj_kernel<<<grid, block, 0, st>>>(q, vw, v0, nv, d_proj, d_npf);
    return cudaGetLastError();
}

size_t lengthproj_scratch_bytes(int n_views) { return (size_t)n_views * sizeof(LpView); }

cudaError_t launch_ir_update(int N, int Z, double scale, const short* d_before, float* d_out, const float* d_npf,
                             const float* d_npf_re, double wbefore, double weight_tv, double weight_prior,
                             cudaStream_t st)
{
    dim3 grid((N + 31) / 32, (N + 7) / 8, Z), block(32, 8);
    ir_update_kernel<<<grid, block, 0, st>>>(N, Z, scale, d_before, d_out, d_npf, d_npf_re, wbefore, weight_tv,
                                             weight_prior);
    return cudaGetLastError();
}

}  // namespace vcbct
