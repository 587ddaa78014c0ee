/*
 * vcbct_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU oracle for the two VirtualCBCT hot paths (MBFPA forward projection and
 * FDK filter + backprojection).  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it, and only as the checker.  The
 * product library (virtualcbct_b200/csrc) never links or calls it.
 *
 * Every function restates, in double precision, the arithmetic of the
 * reference file/line given in its comment.  The restatement is pinned
 * against the reference's own CPU code compiled from its sources
 * (oracle/_ref, see oracle/Makefile) by tests/test_oracle_pin.py.
 */
#ifndef VCBCT_ORACLE_H
#define VCBCT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Projection geometry: the arguments of initializeGPU
 * (Release_CBCT_Projection_CM/reprojectionOnGPU.h:2-8). */
typedef struct {
    int N;          /* reconSize: voxels along x and y */
    int Z;          /* reconSlices: slices along z */
    double s;       /* reconScale: voxel pitch in x/y [cm] */
    double step;    /* reconStep: slice pitch [cm] */
    int W, H, V;    /* projImgWidth, projImgHeight, number of views */
    double pdet;    /* DETECTOR_PITCH_CM */
    double piso;    /* DETECTOR_PITCH_CM_AT_ISO_CENT */
    double sad;     /* DIST_BTWN_SRC_AND_ISOCENT_CM */
    double dpn;     /* DETECTOR_PIXEL_NUM */
    double x_reg, y_reg, z_reg;
    int nmat;       /* num_material */
} orc_proj_geom;

/* Tie rules of the two reference twins. */
enum {
    ORC_TIES_GPU = 0, /* reprojectionOnGPU.cu:198 (">"), :230/:473 ("<=", ">=") */
    ORC_TIES_CPU = 1  /* reprojection.cpp:123 (">="), :153/:448 ("<", ">")       */
};

/* Output modes of orc_mbfpa_forward. */
enum {
    ORC_OUT_REFERENCE = 0, /* per-bin (float) cast, float sum over bins, as
                              reprojectionOnGPU.cu:432,1038-1044 */
    ORC_OUT_FP64 = 1       /* no intermediate rounding; double sum */
};

/*
 * Forward-project a rectangular subset of rays of the given views.
 *   vol      uint16 [Z][nmat][N][N]        (reference matVolume layout)
 *   volf     float  [Z][nmat][N][N]        (used instead of vol when non-NULL)
 *   mu       float  [nmat][NE]             (Attenuation, cm^2/g)
 *   pdf      float  [NE]
 *   views    list of nviews view indices
 *   rows     [j0, j1), cols [c0, c1)       (detector row j, column jj)
 *   ties     ORC_TIES_GPU / ORC_TIES_CPU
 *   with_leng  1: multiply by the cos^3 factor (GPU twin), 0: not (CPU twin)
 *   flip     1: store at row H-1-j (GPU twin), 0: at row j (CPU twin)
 *   exact    1: accumulate transp per bin in the reference's order (bitwise
 *            reproduction), 0: accumulate per-element path integrals L_k once
 *            and form transp = sum_k mu_k L_k (reassociated, ~1e-16 rel.)
 *   out_f    float  [V][H][W] (ORC_OUT_REFERENCE result), may be NULL
 *   out_d    double [V][H][W] (ORC_OUT_FP64 result), may be NULL
 *   L_out    double [V][H][W][nmat] per-element path integrals, may be NULL
 *   nseg_bounds / nseg_mask  int64 per ray [V][H][W] (GPU layout index) of
 *            segments that passed the voxel-bounds test / also the cylinder
 *            mask and have non-zero length (the throughput unit), may be NULL
 * Returns 0 on success.
 */
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
                      int64_t* nseg_bounds, int64_t* nseg_mask);

/*
 * Adjoint of the polychromatic projection with respect to float element
 * volumes (no reference counterpart; the derivative of the FP64 forward).
 *   resid  double [V][H][W] weights r per ray (GPU layout index)
 *   grad   double [Z][nmat][N][N] accumulated += sum_rays r dI/dvol
 */
int orc_mbfpa_adjoint(const orc_proj_geom* g,
                      const double* cosT, const double* sinT,
                      const double* Xc, const double* Yc,
                      const float* volf, const float* mu, const float* pdf,
                      int NE, double xfactor, const double* resid,
                      double* grad);

/* misc.cpp:10-37 (projector): cos/sin and detector centre shifts. */
void orc_trig_tables(int W, int H, int V, const double* angles_rad,
                     const double* xshift, const double* yshift,
                     double pdet, double dpn,
                     double* cosT, double* sinT, double* Xc, double* Yc);

/* FDK geometry constants (Release_recon_from_forward_pro_float_CM/physParams.h). */
typedef struct {
    double mpn;   /* MAX_PIC_NUM */
    double pdet;  /* DETECTOR_PITCH_CM */
    double sad;   /* DIST_BTWN_SRC_AND_ISOCENT_CM */
    double piso;  /* DETECTOR_PITCH_CM_AT_ISO_CENT */
    double cutoff, gamma_, alpha; /* CUTOFF_FREQ, GAMMA, ALPHA */
} orc_fdk_consts;

/* filterSinogram.cpp:10-65: ramp kernel h[m][n], row-major W*W. */
void orc_const_map(int W, const orc_fdk_consts* c, double* h);

/* filterSinogram.cpp:79-80: the diagonal coefficient. */
double orc_filter_coeff(int W, const orc_fdk_consts* c);

/*
 * filterSinogram.cpp:67-131.  proj/out float [V][H][W].
 *   mode 0: float accumulator, each term formed in double (reference)
 *   mode 1: double accumulator (FP64 oracle) written to out_d
 */
void orc_filter(int V, int H, int W, const float* proj, const double* h,
                const double* xshift, const double* yshift,
                const orc_fdk_consts* c, int mode, float* out_f,
                double* out_d);

/* misc.cpp:9-37 (FDK): circular mask, char [N][N]. */
void orc_mask(int N, char* mask);

/*
 * reconstructImage.cpp:10-184.  vol double [Z][N][N] is accumulated (+=).
 * filt float [V][H][W] (filt_d double, used instead when non-NULL).
 */
void orc_backproject(int N, int Z, int zstart, double step, double scale,
                     double* vol, const char* mask, int H, int W, int V,
                     const float* filt, const double* filt_d, int xfactor,
                     const double* angles, const double* cosT,
                     const double* sinT, const double* xshift,
                     const orc_fdk_consts* c);

/* Iterative reconstruction helpers (P/lengthproj.cpp:10-131,
 * P/IR_ImageCBCT.cpp:10-93). */
void orc_lengthproj(int ite, int N, int Z, const unsigned short* proj, float* npf, double s, double step,
                    int W, int H, int v0, int v1, const double* cosT, const double* sinT,
                    const double* Xc, const double* Yc, double pdet, double piso, double sad,
                    double dpn, double xr, double yr, double zr);
void orc_ir_update(int N, int Z, double scale, const short* before, float* out, const float* npf,
                   const float* npf_re, double wbefore, double wtv, double wprior);

#ifdef __cplusplus
}
#endif
#endif
