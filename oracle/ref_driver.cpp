/*
 * ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Thin extern "C" drivers around the reference's own CPU code, which
 * oracle/Makefile compiles straight from the reference sources into
 * oracle/_ref/ (the sources are never copied into this repository).  Built
 * twice: with -DREF_PROJ against the projector sources
 * (Release_CBCT_Projection_CM) and with -DREF_FDK against the FDK sources
 * (Release_recon_from_forward_pro_float_CM); both define their own
 * PROJECTION_DATA/loadData, so they live in separate shared objects.
 *
 * Used by the tests (to pin the oracle and the CUDA path against the
 * reference itself) and by bench.py's reference / cpu_baseline arm.
 */
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <unistd.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "mallocMD.h"

#ifdef REF_PROJ
#include "projectionData.h"
#include "reprojection.h"
#include "misc.h"
#include "lengthproj.h"
#include "IR_ImageCBCT.h"
int gaussiannoise(float* ProjImagefloat, int NN);  // prior_weight_production.cpp:24 (no header)
void attenuation_coefficient(char* spectrum_data_name, int num_material, float* Attenuation,
                             float* pdf_pe, int* NE, int nthin, char* mat_type);

extern "C" {

/*
 * The CPU twin reprojection() (reprojection.cpp:10) only computes view 0
 * (:45, jjj is hard-wired to 0) for one energy bin.  Drive it once per
 * (view, bin) with the per-view tables offset to that view, over all host
 * threads, and sum the bins of a view in bin order in float, as the
 * reference's CPU main loop does (main.cpp:128-142).
 *   out: float [V][H][W], rows NOT flipped, no cos^3 factor (CPU twin).
 * Returns the wall time in seconds of the reprojection() calls.
 */
double ref_mbfpa_views(int N, int Z, const unsigned short* vol, double s, double step,
                       int W, int H, const double* cosT, const double* sinT,
                       const double* Xc, const double* Yc, double xfactor, double pdet,
                       double piso, double sad, double dpn, double xr, double yr, double zr,
                       const float* mu, const float* pdf, int nmat, int NE,
                       const int* views, int nviews, const int* bins, int nbins,
                       int nthreads, float* out)
{
    const long HW = (long)H * W;
    const long npairs = (long)nviews * nbins;
    std::vector<float> part((size_t)npairs * HW, 0.0f);
    std::vector<float> dummy((size_t)HW, 0.0f);   /* projVolume: read, unused */
    double xalpha[1] = {0.0};
    auto t0 = std::chrono::steady_clock::now();
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 1)
    for (long p = 0; p < npairs; p++) {
        int v = views[p / nbins];
        int ke = bins[p % nbins];
        reprojection(0, N, Z, const_cast<unsigned short*>(vol), part.data() + p * HW, nullptr,
                     dummy.data(), s, step, W, H, 0, 1, nullptr,
                     const_cast<double*>(cosT + v), const_cast<double*>(sinT + v),
                     const_cast<double*>(Xc + v), const_cast<double*>(Yc + v), xfactor, xalpha,
                     pdet, piso, sad, dpn, xr, yr, zr, const_cast<float*>(mu),
                     const_cast<float*>(pdf), nmat, NE, ke);
    }
    auto t1 = std::chrono::steady_clock::now();
    for (int iv = 0; iv < nviews; iv++) {
        float* o = out + (long)views[iv] * HW;
        for (long i = 0; i < HW; i++) o[i] = 0.0f;
        for (int b = 0; b < nbins; b++) {
            const float* q = part.data() + ((long)iv * nbins + b) * HW;
            for (long i = 0; i < HW; i++) o[i] += q[i];
        }
    }
    return std::chrono::duration<double>(t1 - t0).count();
}

/* misc.cpp:10 prepareTrigonometricTable, copied out into caller buffers. */
int ref_proj_trig(int W, int H, int V, const double* angles, const double* xs, const double* ys,
                  double pdet, double dpn, double* c, double* s, double* xc, double* yc)
{
    double *a, *b, *e, *f;
    int r = prepareTrigonometricTable(W, H, V, const_cast<double*>(angles), const_cast<double*>(xs),
                                      const_cast<double*>(ys), pdet, dpn, &a, &b, &e, &f);
    std::memcpy(c, a, sizeof(double) * V);
    std::memcpy(s, b, sizeof(double) * V);
    std::memcpy(xc, e, sizeof(double) * V);
    std::memcpy(yc, f, sizeof(double) * V);
    delete1DArray(a); delete1DArray(b); delete1DArray(e); delete1DArray(f);
    return r;
}

/*
 * prior_weight_production.cpp:200 attenuation_coefficient.  It opens
 * "attenuation_xraydb/..." relative to the working directory, so the call is
 * made from `workdir` (the projector directory) and the directory restored.
 */
int ref_attenuation(const char* workdir, const char* spectrum, int nmat, const char* mat_type,
                    float* mu /* 1024*nmat */, float* pdf /* 1024 */)
{
    char old[4096];
    if (!getcwd(old, sizeof old)) return -1;
    if (chdir(workdir) != 0) return -1;
    int NE = 0;
    char sp[1024], mt[64];
    std::snprintf(sp, sizeof sp, "%s", spectrum);
    std::snprintf(mt, sizeof mt, "%s", mat_type);
    attenuation_coefficient(sp, nmat, mu, pdf, &NE, 1, mt);
    if (chdir(old) != 0) return -1;
    return NE;
}

/* projectionData.cpp:64 loadData: parsed fields and the assembled volume. */
int ref_proj_load(const char* txt, int* ints /* 8 */, double* dbls /* 12 */,
                  char* spectrum, char* outname, char* mattype,
                  unsigned short** vol_out, double** angles_out, double** xs_out, double** ys_out)
{
    PROJECTION_DATA* p = newProjectionData();
    int r = loadData(const_cast<char*>(txt), p);
    if (r == 0) return 0;
    ints[0] = p->totalProjNumber; ints[1] = p->projImgWidth; ints[2] = p->projImgHeight;
    ints[3] = p->zICposition; ints[4] = p->reconSize; ints[5] = p->reconSlices;
    ints[6] = p->mat_num; ints[7] = p->usedZNumber;
    dbls[0] = p->x_scale; dbls[1] = p->y_scale; dbls[2] = p->z_scale; dbls[3] = p->xfactor;
    dbls[4] = p->x_reg; dbls[5] = p->y_reg; dbls[6] = p->z_reg;
    dbls[7] = p->DETECTOR_PITCH_CM; dbls[8] = p->DETECTOR_PITCH_CM_AT_ISO_CENT;
    dbls[9] = p->DIST_BTWN_SRC_AND_ISOCENT_CM; dbls[10] = p->DETECTOR_PIXEL_NUM;
    dbls[11] = p->DIST_BTWN_DETECTOR_AND_ISOCENT_CM;
    std::strcpy(spectrum, p->SpectrumString);
    std::strcpy(outname, p->outputname);
    std::strcpy(mattype, p->mat_type);
    *vol_out = p->matVolume;
    *angles_out = p->anglesRad;
    *xs_out = p->xshift;
    *ys_out = p->yshift;
    return r;
}

void ref_free(void* p) { std::free(p); }

/* lengthproj (lengthproj.cpp:10) and IR_ImageCBCT (IR_ImageCBCT.cpp:19) as
 * they are: arguments the reference ignores are passed as NULL / 0. */
void ref_lengthproj(int ite, int N, int Z, unsigned short* proj, float* npf, double s, double step, int W, int H,
                    int v0, int v1, double* cosT, double* sinT, double* Xc, double* Yc, double pdet, double piso,
                    double sad, double dpn, double xr, double yr, double zr)
{
    lengthproj(ite, N, Z, nullptr, nullptr, npf, proj, s, step, W, H, v0, v1, nullptr, cosT, sinT, Xc, Yc, 0.0,
               nullptr, pdet, piso, sad, dpn, xr, yr, zr);
}

void ref_ir_update(int N, int Z, double scale, short* before, float* out, float* npf, float* npf_re, double wbefore,
                   double wtv, double wprior)
{
    IR_ImageCBCT(0, N, Z, scale, before, out, npf, npf_re, wbefore, wtv, wprior, 1);
}

/* gaussiannoise (prior_weight_production.cpp:24-38) after srand(seed). */
void ref_gaussiannoise(float* proj, int n, unsigned seed)
{
    srand(seed);
    gaussiannoise(proj, n);
}

}  // extern "C"
#endif  /* REF_PROJ */

#ifdef REF_FDK
#include "projectionDataMVkV.h"
#include "filterSinogram.h"
#include "reconstructImage.h"
#include "misc.h"

template <class T>
static T*** view3d(T* base, int W, int H, int D)
{
    T*** t = (T***)std::malloc(sizeof(T**) * D);
    for (int k = 0; k < D; k++) {
        t[k] = (T**)std::malloc(sizeof(T*) * H);
        for (int j = 0; j < H; j++) t[k][j] = base + ((long)k * H + j) * W;
    }
    return t;
}
template <class T>
static void free3d(T*** t, int D)
{
    for (int k = 0; k < D; k++) std::free(t[k]);
    std::free(t);
}

extern "C" {

/* filterSinogram.cpp:10 prepareConstMap, row-major copy. */
void ref_const_map(int W, double piso, double* out)
{
    double** h = prepareConstMap(W, piso);
    std::memcpy(out, h[0], sizeof(double) * W * W);
    delete2DArray((void**)h, W, W, UNIT_FLOAT64);
}

/* filterSinogram.cpp:67 on flat [V][H][W] buffers; returns wall seconds. */
double ref_filter(int V, int H, int W, const float* proj, float* out, const double* xs,
                  const double* ys, double piso, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    double** h = prepareConstMap(W, piso);
    float*** pin = view3d(const_cast<float*>(proj), W, H, V);
    float*** pout = view3d(out, W, H, V);
    auto t0 = std::chrono::steady_clock::now();
    filterSinogram(H, W, V, pin, pout, h, const_cast<double*>(xs), const_cast<double*>(ys), piso);
    auto t1 = std::chrono::steady_clock::now();
    free3d(pin, V);
    free3d(pout, V);
    delete2DArray((void**)h, W, W, UNIT_FLOAT64);
    return std::chrono::duration<double>(t1 - t0).count();
}

/* reconstructImage.cpp:10 on flat buffers (vol is accumulated); wall seconds. */
double ref_backproject(int N, int Z, int zstart, double step, double scale, double* vol,
                       int H, int W, int V, const float* filt, int xfactor, const double* angles,
                       const double* xs, double piso, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    char** mask = prepareMaskData(N);
    double *c, *s;
    prepareTrigonometricTable(V, const_cast<double*>(angles), &c, &s);
    double*** pv = view3d(vol, N, N, Z);
    float*** pf = view3d(const_cast<float*>(filt), W, H, V);
    auto t0 = std::chrono::steady_clock::now();
    reconstructImage(N, Z, zstart, step, scale, pv, mask, H, W, V, pf, xfactor,
                     const_cast<double*>(angles), c, s, const_cast<double*>(xs), piso);
    auto t1 = std::chrono::steady_clock::now();
    free3d(pv, Z);
    free3d(pf, V);
    delete2DArray((void**)mask, N, N, UNIT_UINT8);
    delete1DArray(c);
    delete1DArray(s);
    return std::chrono::duration<double>(t1 - t0).count();
}

/* misc.cpp:9 prepareMaskData, row-major copy. */
void ref_mask(int N, char* out)
{
    char** m = prepareMaskData(N);
    std::memcpy(out, m[0], (size_t)N * N);
    delete2DArray((void**)m, N, N, UNIT_UINT8);
}

/* projectionDataMVkV.cpp:52 loadData: parsed fields and the view tables. */
int ref_fdk_load(const char* txt, int* ints /* 8 */, double* dbls /* 3 */, char* projdir,
                 char* ext, char* outname, char* sml, double* angles, double* xs, double* ys)
{
    PROJECTION_DATA* p = newProjectionData();
    int r = loadData(const_cast<char*>(txt), p);
    if (r == 0) return 0;
    ints[0] = p->totalProjNumber; ints[1] = p->usedProjNumber; ints[2] = p->projImgWidth;
    ints[3] = p->projImgHeight; ints[4] = p->reconSize; ints[5] = p->reconOffset;
    ints[6] = p->reconSlices; ints[7] = p->xfactor;
    dbls[0] = p->reconStep; dbls[1] = p->reconScale; dbls[2] = p->DETECTOR_PITCH_CM_AT_ISO_CENT;
    std::strcpy(projdir, p->projImgFileDirname);
    std::strcpy(ext, p->projImgFileExt);
    std::strcpy(outname, p->reconDataFilename);
    std::strcpy(sml, p->SMLClassString);
    for (int i = 0; i < p->usedProjNumber; i++) {
        angles[i] = p->anglesRad[i];
        xs[i] = p->xshift[i];
        ys[i] = p->yshift[i];
    }
    return r;
}

}  // extern "C"
#endif  /* REF_FDK */
