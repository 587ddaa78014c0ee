/*
 * vcbct_oracle.c -- TEST INFRASTRUCTURE ONLY (see vcbct_oracle.h).
 *
 * Double-precision CPU restatement of the reference's hot paths, used by the
 * tests and the bench's CPU-baseline leg as the checker.  It is never linked
 * into, or called by, the product library.
 *
 * Reference files (paths within hagaakihiro/VirtualCBCT):
 *   P = Release_CBCT_Projection_CM, R = Release_recon_from_forward_pro_float_CM
 *   P/reprojectionOnGPU.cu:56-690   reprojectionKernel (GPU twin)
 *   P/reprojection.cpp:10-710       reprojection       (CPU twin)
 *   P/misc.cpp:10-37                prepareTrigonometricTable
 *   R/filterSinogram.cpp:10-131     prepareConstMap / filterSinogram
 *   R/reconstructImage.cpp:10-184   reconstructImage
 *   R/misc.cpp:9-37                 prepareMaskData
 *
 * Arithmetic is written in the same operation order as the reference so that
 * the double results are bitwise reproducible (x86-64, no FMA contraction).
 */
#include "vcbct_oracle.h"

#include <math.h>
#include <limits.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI 3.141592653589793238462643383279

/* (a - a0)/(a1 - a0)*(b1 - b0) + b0: coordinate b on the source-detector line
 * where coordinate a equals `a`.  Same form as reprojectionOnGPU.cu:159 etc. */
static inline double line_at(double a, double a0, double a1, double b0, double b1)
{
    return (a - a0) / (a1 - a0) * (b1 - b0) + b0;
}

/* C cast to int, made total: non-finite or out-of-range values map to
 * INT_MIN (what x86 cvttsd2si yields), which every bounds test rejects. */
static inline int to_int(double v)
{
    if (!(v > -2147483648.0 && v < 2147483647.0)) return INT_MIN;
    return (int)v;
}

typedef struct {
    const orc_proj_geom* g;
    int nxm, nym, nzm;
    double rmax;
    const uint16_t* vol;
    const float* volf;
    const float* mu;
    int NE;
    int exact;
    double* transp;   /* [NE] (exact mode) */
    double L[16];     /* per-element path integrals (fast mode) */
    int64_t nb, nm;
    double* grad;     /* adjoint scatter target, or NULL */
    const double* gk; /* adjoint per-element weights */
} seg_ctx;

static inline double voxel_value(const seg_ctx* c, int64_t vnum)
{
    return c->volf ? (double)c->volf[vnum] : (double)c->vol[vnum];
}

/* One segment b0 -> b1: reprojectionOnGPU.cu:255-271 (and its 6 copies). */
static void emit_segment(seg_ctx* c, const double* b0, const double* b1)
{
    const orc_proj_geom* g = c->g;
    double rr = sqrt((b0[0] - b1[0]) * (b0[0] - b1[0]) +
                     (b0[1] - b1[1]) * (b0[1] - b1[1]) +
                     (b0[2] - b1[2]) * (b0[2] - b1[2]));
    int xmc = to_int((b0[0] + b1[0]) * 0.5 / g->s + c->nxm);
    int ymc = to_int((-b0[1] - b1[1]) * 0.5 / g->s + c->nym);
    int zmc = to_int((-b0[2] - b1[2]) * 0.5 / g->step + c->nzm);
    if (!(xmc >= 0 && ymc >= 0 && zmc >= 0 && xmc <= g->N - 1 &&
          ymc <= g->N - 1 && zmc <= g->Z - 1))
        return;
    c->nb++;
    double r = sqrt((b0[0] + b1[0]) * (b0[0] + b1[0]) +
                    (-b0[1] - b1[1]) * (-b0[1] - b1[1])) * 0.5;
    double ph = (r >= c->rmax) ? 0.0 : 1.0;
    /* the throughput unit: a segment that reads voxel data and contributes
     * (zero-length segments, emitted at exact plane ties, are not counted) */
    if (ph != 0.0 && rr > 0.0) c->nm++;
    const int64_t NN = (int64_t)g->N * g->N;
    for (int mat = 0; mat < g->nmat; mat++) {
        int64_t vnum = xmc + (int64_t)ymc * g->N + ((int64_t)zmc * g->nmat + mat) * NN;
        if (c->grad) {
            c->grad[vnum] += c->gk[mat] * rr * ph;
            continue;
        }
        if (c->exact) {
            /* uint16 * float is a float product in the reference (:268). */
            float v = c->volf ? c->volf[vnum] : (float)c->vol[vnum];
            for (int ke = 0; ke < c->NE; ke++)
                c->transp[ke] += (double)(v * c->mu[mat * c->NE + ke]) * rr * ph;
        } else {
            c->L[mat] += voxel_value(c, vnum) * rr * ph;
        }
    }
}

/*
 * The per-ray march of reprojectionKernel (reprojectionOnGPU.cu:154-429 for
 * the x-dominant branch, :441-666 for its y-dominant mirror), written once for
 * a dominant axis d in {x, y}.  Returns 0 if the ray misses the xy square.
 */
static int march_ray(seg_ctx* c, int ties, const double S[3], const double P[3])
{
    const orc_proj_geom* g = c->g;
    const int nxm = c->nxm, nym = c->nym;
    double xx[4], yy[4], zz[4];
    int m = 0;

    /* entry/exit against the four side planes (:154-183) */
    yy[m] = (double)nym * g->s;
    if (fabs(line_at(yy[m], S[1], P[1], S[0], P[0])) < (double)nxm * g->s) {
        xx[m] = line_at(yy[m], S[1], P[1], S[0], P[0]);
        zz[m] = line_at(yy[m], S[1], P[1], S[2], P[2]);
        m++;
    }
    yy[m] = -(double)nym * g->s;
    if (fabs(line_at(yy[m], S[1], P[1], S[0], P[0])) < (double)nxm * g->s) {
        xx[m] = line_at(yy[m], S[1], P[1], S[0], P[0]);
        zz[m] = line_at(yy[m], S[1], P[1], S[2], P[2]);
        m++;
    }
    if (m < 4) {
        xx[m] = (double)nxm * g->s;
        if (fabs(line_at(xx[m], S[0], P[0], S[1], P[1])) < (double)nym * g->s) {
            yy[m] = line_at(xx[m], S[0], P[0], S[1], P[1]);
            zz[m] = line_at(xx[m], S[0], P[0], S[2], P[2]);
            m++;
        }
    }
    if (m < 4) {
        xx[m] = -(double)nxm * g->s;
        if (fabs(line_at(xx[m], S[0], P[0], S[1], P[1])) < (double)nym * g->s) {
            yy[m] = line_at(xx[m], S[0], P[0], S[1], P[1]);
            zz[m] = line_at(xx[m], S[0], P[0], S[2], P[2]);
            m++;
        }
    }
    /* Fewer than two hits: the reference reads uninitialised entries here
     * (undefined behaviour); the ray is defined to miss the volume. */
    if (m < 2) return 0;

    double I[3], F[3];
    double d0 = (xx[0] - S[0]) * (xx[0] - S[0]) + (yy[0] - S[1]) * (yy[0] - S[1]) +
                (zz[0] - S[2]) * (zz[0] - S[2]);
    double d1 = (xx[1] - S[0]) * (xx[1] - S[0]) + (yy[1] - S[1]) * (yy[1] - S[1]) +
                (zz[1] - S[2]) * (zz[1] - S[2]);
    if (d0 < d1) {
        I[0] = xx[0]; I[1] = yy[0]; I[2] = zz[0];
        F[0] = xx[1]; F[1] = yy[1]; F[2] = zz[1];
    } else {
        I[0] = xx[1]; I[1] = yy[1]; I[2] = zz[1];
        F[0] = xx[0]; F[1] = yy[0]; F[2] = zz[0];
    }

    /* dominant axis: ">" on the GPU twin (:198), ">=" on the CPU twin (:123) */
    int xdom = (ties == ORC_TIES_GPU) ? (fabs(I[0] - F[0]) > fabs(I[1] - F[1]))
                                      : (fabs(I[0] - F[0]) >= fabs(I[1] - F[1]));
    const int d = xdom ? 0 : 1, o = 1 - d;
    const double s = g->s, step = g->step;
    const double hx = (double)nxm * s, hy = (double)nym * s;

    double pha = (F[d] - I[d]) / fabs(I[d] - F[d]);
    int ain;
    if ((I[d] < 0 && (F[d] - I[d]) < 0) || (I[d] > 0 && (F[d] - I[d]) > 0))
        ain = to_int((int)I[d] + (F[d] - I[d]) / fabs(F[d] - I[d]));
    else
        ain = to_int(I[d]);

    double cur[3];
    cur[d] = ain;
    cur[o] = line_at(cur[d], S[d], P[d], S[o], P[o]);
    cur[2] = line_at(cur[d], S[d], P[d], S[2], P[2]);

    double b0[3] = {I[0], I[1], I[2]};
    int om = 0, zm = 0;
    const long kmax = 8L * (g->N + g->Z) + (long)(8.0 * (hx + hy + 4.0) / s) + 64;
    for (long k = 0; k < kmax; k++) {
        if (!(cur[0] <= hx && cur[0] >= -hx && cur[1] <= hy && cur[1] >= -hy)) break;
        cur[d] = ain + pha * (double)k * s;
        int om_prev = om;
        double oj = cur[o];
        cur[o] = line_at(cur[d], S[d], P[d], S[o], P[o]);
        om = to_int(cur[o] / s);
        int zm_prev = zm;
        cur[2] = line_at(cur[d], S[d], P[d], S[2], P[2]);
        zm = to_int(cur[2] / step);

        int icheck = 0;
        double chy = 0.0, chz = 0.0;
        double Yp[3] = {0, 0, 0}, Zp[3] = {0, 0, 0};
        /* crossing of a plane of the non-dominant axis, or of its zero plane
         * (:226-236 / :469-479) */
        if ((k != 0 && om != om_prev) || (k != 0 && (cur[o] / fabs(cur[o]) != oj / fabs(oj)))) {
            double dir = F[o] - I[o];
            int at_plane = (ties == ORC_TIES_GPU)
                               ? ((cur[o] <= 0 && dir < 0) || (cur[o] >= 0 && dir > 0))
                               : ((cur[o] < 0 && dir < 0) || (cur[o] > 0 && dir > 0));
            if (at_plane) Yp[o] = (double)(om * s);
            else Yp[o] = (double)(om * s) - dir / fabs(dir) * s;
            Yp[d] = line_at(Yp[o], S[o], P[o], S[d], P[d]);
            Yp[2] = line_at(Yp[o], S[o], P[o], S[2], P[2]);
            chy = (cur[0] - Yp[0]) * (cur[0] - Yp[0]) + (cur[1] - Yp[1]) * (cur[1] - Yp[1]) +
                  (cur[2] - Yp[2]) * (cur[2] - Yp[2]);
            icheck++;
        }
        /* z crossing; the z = 0 plane is not tested (:237-247) */
        if (k != 0 && zm != zm_prev) {
            double dir = F[2] - I[2];
            if ((cur[2] < 0 && dir < 0) || (cur[2] > 0 && dir > 0)) Zp[2] = (double)(zm * step);
            else Zp[2] = (double)(zm * step) - dir / fabs(dir) * step;
            Zp[0] = line_at(Zp[2], S[2], P[2], S[0], P[0]);
            Zp[1] = line_at(Zp[2], S[2], P[2], S[1], P[1]);
            chz = (cur[0] - Zp[0]) * (cur[0] - Zp[0]) + (cur[1] - Zp[1]) * (cur[1] - Zp[1]) +
                  (cur[2] - Zp[2]) * (cur[2] - Zp[2]);
            icheck++;
        }
        /* segment emission order (:249-404) */
        if (icheck == 2 && chz > chy) {
            emit_segment(c, b0, Zp); memcpy(b0, Zp, sizeof b0);
            emit_segment(c, b0, Yp); memcpy(b0, Yp, sizeof b0);
        } else if (icheck == 2 && chz < chy) {
            emit_segment(c, b0, Yp); memcpy(b0, Yp, sizeof b0);
            emit_segment(c, b0, Zp); memcpy(b0, Zp, sizeof b0);
        } else if (icheck == 1 && chz != 0) {
            emit_segment(c, b0, Zp); memcpy(b0, Zp, sizeof b0);
        } else if (icheck == 1 && chy != 0) {
            emit_segment(c, b0, Yp); memcpy(b0, Yp, sizeof b0);
        }
        emit_segment(c, b0, cur);
        memcpy(b0, cur, sizeof b0);
    }
    return 1;
}

static void ray_endpoints(const orc_proj_geom* g, const double* cosT, const double* sinT,
                          const double* Xc, const double* Yc, int v, int j, int jj,
                          double S[3], double P[3], double* leng)
{
    /* reprojectionOnGPU.cu:128-150 */
    S[0] = -g->sad * sinT[v] + g->x_reg;
    S[1] = g->sad * cosT[v] + g->y_reg;
    S[2] = g->z_reg;
    P[2] = -(Yc[v] + j) * g->piso * (g->dpn / g->H) + g->z_reg * g->piso / g->pdet;
    double pr = g->piso * (Xc[v] + jj) * (g->dpn / g->H);
    P[0] = pr * cosT[v] + g->x_reg * g->piso / g->pdet;
    P[1] = pr * sinT[v] + g->y_reg * g->piso / g->pdet;
    double l = g->sad * g->sad / (g->sad * g->sad + (pr * pr + P[2] * P[2]));
    *leng = l * sqrt(l);
}

static void ctx_init(seg_ctx* c, const orc_proj_geom* g)
{
    memset(c, 0, sizeof *c);
    c->g = g;
    c->nxm = (int)(g->N * 0.5);
    c->nym = (int)(g->N * 0.5);
    c->nzm = (int)(g->Z * 0.5);
    c->rmax = g->N * 0.5 * g->s;
}

int orc_mbfpa_forward(const orc_proj_geom* g,
                      const double* cosT, const double* sinT,
                      const double* Xc, const double* Yc,
                      const uint16_t* vol, const float* volf,
                      const float* mu, const float* pdf, int NE,
                      double xfactor,
                      const int* views, int nviews,
                      int j0, int j1, int c0, int c1,
                      int ties, int with_leng, int flip, int exact,
                      float* out_f, double* out_d, double* L_out,
                      int64_t* nseg_bounds, int64_t* nseg_mask)
{
    if (!g || NE <= 0 || NE > 4096 || g->nmat <= 0 || g->nmat > 16) return 1;
    if (j0 < 0 || j1 > g->H || c0 < 0 || c1 > g->W || j0 >= j1 || c0 >= c1) return 1;
    const int nrow = j1 - j0, ncol = c1 - c0;
    const long nrays = (long)nviews * nrow * ncol;

#pragma omp parallel
    {
        double* transp = (double*)malloc(sizeof(double) * NE);
#pragma omp for schedule(dynamic, 16)
        for (long r = 0; r < nrays; r++) {
            int v = views[r / ((long)nrow * ncol)];
            int j = j0 + (int)((r / ncol) % nrow);
            int jj = c0 + (int)(r % ncol);
            double S[3], P[3], leng;
            ray_endpoints(g, cosT, sinT, Xc, Yc, v, j, jj, S, P, &leng);
            seg_ctx c;
            ctx_init(&c, g);
            c.vol = vol; c.volf = volf; c.mu = mu; c.NE = NE; c.exact = exact;
            c.transp = transp;
            for (int ke = 0; ke < NE; ke++) transp[ke] = 0.0;
            march_ray(&c, ties, S, P);

            if (!exact) {
                for (int ke = 0; ke < NE; ke++) {
                    double t = 0.0;
                    for (int mat = 0; mat < g->nmat; mat++)
                        t += (double)mu[mat * NE + ke] * c.L[mat];
                    transp[ke] = t;
                }
            }
            double lf = with_leng ? leng : 1.0;
            float accf = 0.0f;
            double accd = 0.0;
            for (int ke = 0; ke < NE; ke++) {
                double intens = pdf[ke] * exp(-transp[ke] / xfactor) * lf;
                accf += (float)intens;
                accd += intens;
            }
            long row = flip ? (g->H - 1 - j) : j;
            long idx = ((long)v * g->H + row) * g->W + jj;
            if (out_f) out_f[idx] = accf;
            if (out_d) out_d[idx] = accd;
            if (L_out)
                for (int mat = 0; mat < g->nmat; mat++) L_out[idx * g->nmat + mat] = c.L[mat];
            if (nseg_bounds) nseg_bounds[idx] = c.nb;
            if (nseg_mask) nseg_mask[idx] = c.nm;
        }
        free(transp);
    }
    return 0;
}

int orc_mbfpa_adjoint(const orc_proj_geom* g,
                      const double* cosT, const double* sinT,
                      const double* Xc, const double* Yc,
                      const float* volf, const float* mu, const float* pdf,
                      int NE, double xfactor, const double* resid,
                      double* grad)
{
    if (!g || !volf || NE <= 0 || g->nmat > 16) return 1;
    for (int v = 0; v < g->V; v++)
        for (int j = 0; j < g->H; j++)
            for (int jj = 0; jj < g->W; jj++) {
                long idx = ((long)v * g->H + (g->H - 1 - j)) * g->W + jj;
                double r = resid[idx];
                if (r == 0.0) continue;
                double S[3], P[3], leng;
                ray_endpoints(g, cosT, sinT, Xc, Yc, v, j, jj, S, P, &leng);
                seg_ctx c;
                ctx_init(&c, g);
                c.volf = volf; c.mu = mu; c.NE = NE; c.exact = 0;
                if (!march_ray(&c, ORC_TIES_GPU, S, P)) continue;
                double gk[16] = {0};
                for (int ke = 0; ke < NE; ke++) {
                    double t = 0.0;
                    for (int mat = 0; mat < g->nmat; mat++) t += (double)mu[mat * NE + ke] * c.L[mat];
                    double e = (double)pdf[ke] * exp(-t / xfactor);
                    for (int mat = 0; mat < g->nmat; mat++)
                        gk[mat] -= leng / xfactor * e * (double)mu[mat * NE + ke];
                }
                for (int mat = 0; mat < g->nmat; mat++) gk[mat] *= r;
                seg_ctx c2;
                ctx_init(&c2, g);
                c2.volf = volf; c2.grad = grad; c2.gk = gk;
                march_ray(&c2, ORC_TIES_GPU, S, P);
            }
    return 0;
}

void orc_trig_tables(int W, int H, int V, const double* angles_rad,
                     const double* xshift, const double* yshift,
                     double pdet, double dpn,
                     double* cosT, double* sinT, double* Xc, double* Yc)
{
    (void)W;
    /* P/misc.cpp:10-37: the height is used for both shifts. */
    for (int i = 0; i < V; i++) {
        cosT[i] = cos(angles_rad[i]);
        sinT[i] = sin(angles_rad[i]);
        Xc[i] = -H / 2.0 - xshift[i] * 10.0 / (pdet * (dpn / H));
        Yc[i] = -H / 2.0 - yshift[i] * 10.0 / (pdet * (dpn / H));
    }
}

/* ------------------------------------------------------------------ FDK -- */

void orc_const_map(int W, const orc_fdk_consts* c, double* h)
{
    /* R/filterSinogram.cpp:21-62 */
    double theConst = 1.0 / (8.0 * ORC_PI * ORC_PI * c->piso * c->mpn / W);
    double gxc = c->gamma_ * c->cutoff;
    double pxc = ORC_PI * c->cutoff;
    double oma = 1.0 - c->alpha;
    double omega = ORC_PI / c->gamma_;
    double co = cos(omega), so = sin(omega);
    for (int m = 0; m < W; m++)
        for (int n = 0; n < W; n++) {
            if (m == n) {
                h[(long)m * W + n] = 0.0;
                continue;
            }
            double MN = (double)(m - n);
            double th = pxc * MN;
            double de = gxc * MN;
            double eta = 1.0 / (1.0 - 1.0 / de);
            double xi = 1.0 / (1.0 + 1.0 / de);
            double ct = cos(th), st = sin(th);
            h[(long)m * W + n] = theConst / MN / MN *
                (2.0 * c->alpha * th * st
                 + 2.0 * c->alpha * (ct - 1.0)
                 + xi * oma * th * (st * co + ct * so)
                 + eta * oma * th * (st * co - ct * so)
                 + xi * xi * oma * (ct * co - st * so - 1.0)
                 + eta * eta * oma * (ct * co + st * so - 1.0));
        }
}

double orc_filter_coeff(int W, const orc_fdk_consts* c)
{
    double omega = ORC_PI / c->gamma_;
    return c->cutoff * c->cutoff / 4.0 / (c->piso * c->mpn / W) *
           (c->alpha * 0.5 + (1.0 - c->alpha) * (1.0 / omega * sin(omega) +
                                                1.0 / omega / omega * (cos(omega) - 1.0)));
}

void orc_filter(int V, int H, int W, const float* proj, const double* h,
                const double* xshift, const double* yshift,
                const orc_fdk_consts* c, int mode, float* out_f,
                double* out_d)
{
    double coeff = orc_filter_coeff(W, c);
    double pitch = c->piso * c->mpn / W;
#pragma omp parallel for
    for (int th = 0; th < V; th++) {
        /* R/filterSinogram.cpp:86-113 */
        double XcS = -W / 2.0 - xshift[th] / (c->pdet * c->mpn / W) - 1;
        double YcS = -W / 2.0 - yshift[th] / (c->pdet * c->mpn / W) - 1;
        for (int n = 0; n < H; n++) {
            double pos2 = fabs((YcS + n)) * pitch;
            const float* p = proj + ((long)th * H + n) * W;
            for (int m = 0; m < W; m++) {
                double pos1 = fabs((XcS + m)) * pitch;
                double Cm = c->sad / sqrt(c->sad * c->sad + pos1 * pos1 + pos2 * pos2);
                long o = ((long)th * H + n) * W + m;
                /* log() of a float argument is the C++ float overload in the
                 * reference (:103, :108), i.e. logf, widened to double. */
                if (mode == 0) {
                    float acc = (float)(-(double)logf(p[m]) * Cm * coeff);
                    for (int k = 0; k < W; k++)
                        acc = (float)(acc + h[(long)m * W + k] * (-(double)logf(p[k])) * Cm);
                    out_f[o] = acc;
                } else {
                    double acc = -log((double)p[m]) * Cm * coeff;
                    for (int k = 0; k < W; k++) acc += h[(long)m * W + k] * (-log((double)p[k])) * Cm;
                    out_d[o] = acc;
                }
            }
        }
    }
}

void orc_mask(int N, char* mask)
{
    /* R/misc.cpp:20-36 */
    double R = (double)(N - 1) / 2.0;
    double R2 = R * R;
    for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++)
            mask[(long)j * N + i] = (((double)j - R) * ((double)j - R) + ((double)i - R) * ((double)i - R) <= R2) ? 1 : 0;
}

void orc_backproject(int N, int Z, int zstart, double step, double scale,
                     double* vol, const char* mask, int H, int W, int V,
                     const float* filt, const double* filt_d, int xfactor,
                     const double* angles, const double* cosT,
                     const double* sinT, const double* xshift,
                     const orc_fdk_consts* c)
{
    double centerPos = (double)N / 2.0 - 0.5;
    double pitch = c->piso * c->mpn / W;
#define FV(th, r, col) (filt_d ? filt_d[((long)(th) * H + (r)) * W + (col)] \
                               : (double)filt[((long)(th) * H + (r)) * W + (col)])
#pragma omp parallel for
    for (int z = 0; z < Z; z++) {
        double zz = zstart + z * step;
        for (int y = 0; y < N; y++)
            for (int x = 0; x < N; x++) {
                if (mask[(long)y * N + x] == 0) continue;
                double xx = (x - centerPos) * scale;
                double yy = -(y - centerPos) * scale;
                double acc = vol[((long)z * N + y) * N + x];
                for (int th = 0; th < V; th++) {
                    /* R/reconstructImage.cpp:37-72: half the neighbouring gap */
                    double dbeta;
                    if (th == 0) dbeta = fabs(angles[1] - angles[0]) / 2;
                    else if (th == V - 1) dbeta = fabs(angles[th] - angles[th - 1]) / 2;
                    else {
                        double t0 = angles[th - 1], t2 = angles[th + 1];
                        double t1 = angles[th + 1] - 2 * ORC_PI;
                        if (t2 < 0) t1 = angles[th + 1] + 2 * ORC_PI;
                        dbeta = fabs(t2 - t0) / 2;
                        if (dbeta > ORC_PI / 2) dbeta = fabs(t1 - t0) / 2;
                    }
                    double X = xx * cosT[th] + yy * sinT[th];
                    double Y = -xx * sinT[th] + yy * cosT[th];
                    double L2 = 1.0 - Y / c->sad;
                    double U = X / L2 / pitch;
                    double wu = fabs(fabs(U) - fabs(floor(U)));
                    double UUU = (double)(W / 2 + U + xshift[th] / (c->pdet * c->mpn / W) - 0.5);
                    int UU = (int)floor(UUU);
                    double ZETA = (double)(H / 2) + zz / L2 / pitch;
                    int NZ = (int)floor(ZETA);
                    double wz = fabs(fabs(ZETA) - fabs(floor(ZETA)));
                    double sum;
                    int ok = 1;
                    if ((UU >= 0 && UU < W - 1) && (NZ >= 0 && NZ < H - 1))
                        sum = FV(th, NZ, UU) * (1.0 - wu) * (1.0 - wz) + FV(th, NZ, UU + 1) * wu * (1.0 - wz) +
                              FV(th, NZ + 1, UU) * (1.0 - wu) * wz + FV(th, NZ + 1, UU + 1) * wu * wz;
                    else if ((UU == W - 1) && (NZ >= 0 && NZ < H - 1))
                        sum = FV(th, NZ, UU) * (1.0 - wz) + FV(th, NZ + 1, UU) * wz;
                    else if ((UU >= 0 && UU < W - 1) && (NZ == H - 1))
                        sum = FV(th, NZ, UU) * (1.0 - wu) + FV(th, NZ, UU + 1) * wu;
                    else if ((UU == W - 1) && (NZ == H - 1))
                        sum = FV(th, NZ, UU);
                    else
                        ok = 0;
                    if (ok) acc += (1.0 / L2 / L2 * sum * dbeta * xfactor);
                }
                vol[((long)z * N + y) * N + x] = acc;
            }
    }
#undef FV
}


/* ------------------------------------------------------ iterative recon --
 * Sensitivity backprojection, restating lengthproj (P/lengthproj.cpp:10-131)
 * operation by operation: per voxel, the views [v0, v1) in order, float
 * accumulation of (65535 - bilinear projection) x chord length.  npf
 * [Z][N][N] is overwritten.  Registration shifts are zeroed for ite != 0
 * (:18-23). */
void orc_lengthproj(int ite, int N, int Z, const unsigned short* proj, float* npf, double s, double step,
                    int W, int H, int v0, int v1, const double* cosT, const double* sinT,
                    const double* Xc, const double* Yc, double pdet, double piso, double sad,
                    double dpn, double xr, double yr, double zr)
{
    if (ite != 0) { xr = 0.0; yr = 0.0; zr = 0.0; }
    const double maxpix = 65535.0; /* P/physParams.h:63 */
#pragma omp parallel for
    for (int jz = 0; jz < Z; jz++) {
        double rz = Z * step * 0.5 - (jz + 0.5) * step;
        for (int jy = 0; jy < N; jy++) {
            double ry = N * s * 0.5 - (jy + 0.5) * s;
            for (int jx = 0; jx < N; jx++) {
                double rx = -N * s * 0.5 + (jx + 0.5) * s;
                float acc = 0.0f;
                for (int v = v0; v < v1; v++) {
                    double sx = -sad * sinT[v] + xr;
                    double sy = sad * cosT[v] + yr;
                    double sz = zr;
                    double yslope = fabs(ry - sy), xslope = fabs(rx - sx);
                    double rr;
                    if (xslope > yslope) {
                        double xx0 = rx - 0.5 * s;
                        double yy0 = (xx0 - sx) / (rx - sx) * (ry - sy) + sy;
                        double zz0 = (xx0 - sx) / (rx - sx) * (rz - sz) + sz;
                        double xx1 = rx + 0.5 * s;
                        double yy1 = (xx1 - sx) / (rx - sx) * (ry - sy) + sy;
                        double zz1 = (xx1 - sx) / (rx - sx) * (rz - sz) + sz;
                        rr = sqrt((xx0 - xx1) * (xx0 - xx1) + (yy0 - yy1) * (yy0 - yy1) + (zz0 - zz1) * (zz0 - zz1));
                    } else {
                        double yy0 = ry - 0.5 * s;
                        double xx0 = (yy0 - sy) / (ry - sy) * (rx - sx) + sx;
                        double zz0 = (yy0 - sy) / (ry - sy) * (rz - sz) + sz;
                        double yy1 = ry + 0.5 * s;
                        double xx1 = (yy1 - sy) / (ry - sy) * (rx - sx) + sx;
                        double zz1 = (yy1 - sy) / (ry - sy) * (rz - sz) + sz;
                        rr = sqrt((xx0 - xx1) * (xx0 - xx1) + (yy0 - yy1) * (yy0 - yy1) + (zz0 - zz1) * (zz0 - zz1));
                    }
                    double ox = sx + pdet / piso * sinT[v] * sad;
                    double oy = sy - pdet / piso * cosT[v] * sad;
                    double py = (ox - rx + (sx - rx) / (sy - ry) * ry + (oy - sy) / (ox - sx) * oy) /
                                ((sx - rx) / (sy - ry) + (oy - sy) / (ox - sx));
                    double px = ((sx - rx) / (sy - ry) * (py - ry) + rx);
                    double pz = ((sz - rz) / (sy - ry) * (py - ry) + rz);
                    double bin = pdet * (dpn / H);
                    double xshift = -(Xc[v] + H / 2.0) * bin;
                    double yshift = -(Yc[v] + H / 2.0) * bin;
                    double vv = -(pz - zr - yshift);
                    double uu = (px - xr) * cosT[v] + (py - xr) * sinT[v] + xshift - (W - H) / 2 * bin;
                    /* the reference's (int) of a non-finite or huge value
                     * drops the view through its bounds test */
                    if (!(fabs(vv / bin) < 1.0e9) || !(fabs(uu / bin) < 1.0e9)) continue;
                    double vfac = vv < 0 ? -0.5 : 0.5;
                    double ufac = uu < 0 ? -0.5 : 0.5;
                    int vi1 = (int)(vv / bin + vfac);
                    int ui1 = (int)(uu / bin + ufac);
                    double dv1 = vv / bin - vi1;
                    double du1 = uu / bin - ui1;
                    int vi2 = vi1, ui2 = ui1;
                    if (!(fabs(vv - vi1) < 0.000000001)) vi2 = vi1 + ((vv - vi1) > 0 ? 1 : -1);
                    if (!(fabs(uu - ui1) < 0.000000001)) ui2 = ui1 + ((uu - ui1) > 0 ? 1 : -1);
                    int r1 = vi1 + H / 2, r2 = vi2 + H / 2, c1 = ui1 + W / 2, c2 = ui2 + W / 2;
                    if (r1 >= 0 && r1 < H && r2 >= 0 && r2 < H && c1 >= 0 && c1 < W && c2 >= 0 && c2 < W) {
                        const unsigned short* pv = proj + (size_t)v * W * H;
                        double np1 = ((1 - dv1) * pv[r1 * W + c1] + dv1 * pv[r1 * W + c2]);
                        double np2 = ((1 - dv1) * pv[r2 * W + c1] + dv1 * pv[r2 * W + c2]);
                        double np3 = ((1 - du1) * np1 + du1 * np2);
                        acc += (float)((maxpix - np3) * rr);
                    }
                }
                npf[((size_t)jz * N + jy) * N + jx] = acc;
            }
        }
    }
}

/* IR_ImageCBCT (P/IR_ImageCBCT.cpp:10-93) restated. */
static double orc_tv(int a, int ax, int ay, int az, int ax1, int ay1, int az1, int ayx1, int azx1, int axy1,
                     int azy1, int axz1, int ayz1)
{
    double d1 = sqrt((double)((a - ax) * (a - ax) + (a - ay) * (a - ay) + (a - az) * (a - az))) + 0.00000001;
    double d2 = sqrt((double)((a - ax1) * (a - ax1) + (ax1 - ayx1) * (ax1 - ayx1) + (ax1 - azx1) * (ax1 - azx1))) +
                0.00000001;
    double d3 = sqrt((double)((ay1 - axy1) * (ay1 - axy1) + (a - ay1) * (a - ay1) + (ay1 - azy1) * (ay1 - azy1))) +
                0.00000001;
    double d4 = sqrt((double)((az1 - axz1) * (az1 - axz1) + (az1 - ayz1) * (az1 - ayz1) + (a - az1) * (a - az1))) +
                0.00000001;
    return ((a - ax) + (a - ay) + (a - az)) / d1 + (a - ax1) / d2 + (a - ay1) / d3 + (a - az1) / d4;
}

void orc_ir_update(int N, int Z, double scale, const short* before, float* out, const float* npf,
                   const float* npf_re, double wbefore, double wtv, double wprior)
{
    const double rmax = N * 0.5 * 1.0;
    const size_t NN = (size_t)N * N;
#pragma omp parallel for
    for (int z = 0; z < Z; z++)
        for (int y = 0; y < N; y++)
            for (int x = 0; x < N; x++) {
                size_t kk = (size_t)z * NN + (size_t)y * N + x;
                double cost_tv = 0.0, cost_prior = 0.0;
                if (z < Z - 1 && y < N - 1 && x < N - 1 && x > 0 && y > 0 && z > 0) {
#define B(dz, dy, dx) before[kk + (long)(dz) * (long)NN + (long)(dy) * N + (dx)]
                    cost_tv = orc_tv(B(0, 0, 0), B(0, 0, 1), B(0, 1, 0), B(1, 0, 0), B(0, 0, -1), B(0, -1, 0),
                                     B(-1, 0, 0), B(0, 1, -1), B(1, 0, -1), B(0, -1, 1), B(1, -1, 0), B(-1, 0, 1),
                                     B(-1, 1, 0));
#undef B
                }
                double lambda = wtv * cost_tv + wprior * cost_prior + 0.000001;
                float v = (float)(before[kk] * (wbefore + (1 - wbefore) * npf_re[kk] / (npf[kk] + lambda)));
                if (v < 0.0) v = 0.0f;
                else if (v > 65535 / 2) v = 5000.0f;
                double xx = -N * scale * 0.5 + (x + 0.5) * scale;
                double yy = N * scale * 0.5 - (y + 0.5) * scale;
                double r = sqrt((xx) * (xx) + (yy) * (yy));
                if (r >= rmax) v = 0.0f;
                out[kk] = v;
            }
}
