/*
 * vcbct.h -- C ABI of libvcbct, the B200 (sm_100a) implementation of
 * VirtualCBCT's two hot paths:
 *
 *   MBFPA  material-based polychromatic ray-driven forward projection
 *   FDK    cosine weighting + ramp filter + voxel-driven cone-beam
 *          backprojection
 *
 * Two layers are exported.
 *
 *  1. Reference-named entry points with the reference's exact signatures, so
 *     that a main.cpp-style driver of hagaakihiro/VirtualCBCT links unchanged
 *     against -lvcbct.  Each cites the declaration it replaces.
 *  2. vcbct_* entry points: explicit geometry structs, host or device
 *     buffers, a CUDA stream (passed as void*, 0 = legacy default stream) and
 *     an int status (VCBCT_OK = 0).  vcbct_last_error() gives the message of
 *     the last failure on the calling thread.  Nothing here calls exit().
 *
 * All arrays are dense, C order.  Layouts follow the reference:
 *   element volume   uint16 [Z][nmat][N][N]   (projectionData.cpp:192-215)
 *   projections      float  [V][H][W]          (reprojectionOnGPU.cu:106)
 *   reconstruction   short / float / double [Z][N][N] (R/main.cpp:47-49)
 *   attenuation      float  [nmat][NE] (cm^2/g), pdf float [NE]
 */
#ifndef VCBCT_H
#define VCBCT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
enum {
    VCBCT_OK = 0,
    VCBCT_ERR_ARG = 1,     /* invalid argument (size, NULL, range) */
    VCBCT_ERR_CUDA = 2,    /* a CUDA runtime call failed */
    VCBCT_ERR_LIMIT = 3,   /* a size exceeds a documented limit */
    VCBCT_ERR_STATE = 4,   /* object not ready (e.g. no volume loaded) */
    VCBCT_ERR_IO = 5,      /* file could not be read or written */
    VCBCT_ERR_DEVICE = 6   /* a kernel reported a runtime fault flag */
};

/* Compile-time limits of the library. */
#define VCBCT_MAX_MATERIALS 8   /* element planes per voxel */
#define VCBCT_MAX_BINS 1024     /* energy bins (reference arrays are 1024) */

const char* vcbct_last_error(void);
const char* vcbct_version(void);

/* ------------------------------------------------------------------ MBFPA */

/* Projection geometry = the arguments of initializeGPU
 * (Release_CBCT_Projection_CM/reprojectionOnGPU.h:2-8). */
typedef struct {
    int recon_size;          /* N: voxels along x and y */
    int recon_slices;        /* Z */
    double recon_scale;      /* voxel pitch in x/y [cm] */
    double recon_step;       /* slice pitch [cm] */
    int proj_width;          /* W */
    int proj_height;         /* H */
    int n_views;             /* V */
    double det_pitch_cm;     /* DETECTOR_PITCH_CM */
    double det_pitch_iso_cm; /* DETECTOR_PITCH_CM_AT_ISO_CENT */
    double sad_cm;           /* DIST_BTWN_SRC_AND_ISOCENT_CM */
    double det_pixel_num;    /* DETECTOR_PIXEL_NUM */
    double x_reg, y_reg, z_reg;
    int num_material;        /* <= VCBCT_MAX_MATERIALS */
} vcbct_proj_geometry;

typedef struct vcbct_projector vcbct_projector;

/* Replaces initializeGPU (reprojectionOnGPU.h:2-8): per-view tables are the
 * outputs of prepareTrigonometricTable (misc.cpp:10-37), n_views entries. */
int vcbct_projector_create(const vcbct_proj_geometry* g, const double* cos_table,
                           const double* sin_table, const double* xcenter_shift,
                           const double* ycenter_shift, vcbct_projector** out);
/* Replaces terminateGPU (reprojectionOnGPU.h:10). */
int vcbct_projector_destroy(vcbct_projector* p);

/* Spectrum: Attenuation float [nmat][NE] and pdf_pe float [NE] as produced by
 * attenuation_coefficient (prior_weight_production.cpp:200-523); xfactor is
 * the density factor of the input txt (projectionData.cpp:164). */
int vcbct_projector_set_spectrum(vcbct_projector* p, const float* attenuation,
                                 const float* pdf, int n_bins, double xfactor);

/* Element volume uint16 [Z][nmat][N][N] (the matVolume of projectionData.cpp),
 * from host memory (on_device = 0) or device memory (on_device = 1).  The
 * values are kept unaltered; the device copy is re-laid out once into the
 * z-fastest packed form the projector reads (the values as floats, which
 * represent every uint16 exactly). */
int vcbct_projector_load_volume(vcbct_projector* p, const uint16_t* volume, int on_device,
                                void* stream);

/* Same, from float element volumes [Z][nmat][N][N] (densities x1000, the
 * differentiable path; no reference counterpart).  Both loaders give the same
 * packed form: a float volume holding integer values projects bit for bit as
 * the uint16 volume of those values. */
int vcbct_projector_load_volume_f32(vcbct_projector* p, const float* volume, int on_device,
                                    void* stream);

/* The spectral projection of reprojectionOnGPU (reprojectionOnGPU.cu:838-1056):
 * out float [V][H][W] (row H-1-j holds detector row j, as :106), host or
 * device.  One fused launch marches every ray once and forms the spectral sum
 * in-kernel instead of one launch + D2H copy per energy bin. */
int vcbct_projector_forward(vcbct_projector* p, float* out, int out_on_device, void* stream);

/* vcbct_projector_load_volume + vcbct_projector_forward from host memory to
 * host memory in one call, the work of one reprojectionOnGPU call
 * (reprojectionOnGPU.cu:838-1056 with its volume upload, :867): the
 * volume [Z][nmat][N][N] goes up in slabs of slices while the detector is
 * projected in bands of 32 rows, each band as soon as the slices it reads are
 * in, and each band's rows come back while later bands are projected (the
 * download overlaps only into page-locked `out`).  Returns when `out` is
 * written; the volume stays loaded.  Results are bitwise those of the
 * two-call form. */
int vcbct_projector_project(vcbct_projector* p, const uint16_t* volume, float* out, void* stream);

/* Detector noise of the projections the projector writes (no reference
 * counterpart in the projector; the model is the reference's gaussiannoise,
 * prior_weight_production.cpp:24-38, in count units): kind 1 turns every
 * intensity I into n' / i0 with n = i0 * I and n' = n + sqrt(n) z (z standard
 * normal from a counter-based generator keyed by `seed` and the pixel's
 * index, so reproducible and independent of launch shape), clamped to
 * [0, max_counts]; kind 2 draws n' from Poisson(n) instead (exact counting
 * statistics for low counts: multiplication of uniforms below n = 10, the
 * transformed rejection method PTRS above; no reference counterpart); kind 0
 * turns it off (default).  Applied in the forward kernel's epilogue. */
int vcbct_projector_set_noise(vcbct_projector* p, int kind, double i0, double max_counts,
                              unsigned long long seed);
/* The counter-based generator of the noise options: Philox-4x32-10 (Salmon
 * et al., SC 2011) of counter ctr[4] under key[2] (host function, for
 * reproducing the draws). */
void vcbct_philox4x32_10(const uint32_t* ctr, const uint32_t* key, uint32_t* out);
/* The reference's gaussiannoise on projections in its own units (value =
 * max_pixvalue - counts), float [n]; host or device; synchronous for host. */
int vcbct_gaussian_noise(float* proj, size_t n, double max_pixvalue, unsigned long long seed,
                         int on_device, void* stream);

/* Per-ray element path integrals L[V][H][W][nmat] (float, cm x density
 * units) -- the decomposition state; device pointer. */
int vcbct_projector_path_integrals(vcbct_projector* p, float* d_L, void* stream);

/* Segment counter (diagnostics and the Gseg/s metric): number of in-volume,
 * in-cylinder segments of every ray, summed; device-side count. */
int vcbct_projector_count_segments(vcbct_projector* p, unsigned long long* total, void* stream);

/* Adjoint (no reference counterpart; nearest analogue lengthproj.cpp:10-131):
 * given d(loss)/d(out) as float [V][H][W] on the device, accumulate
 * d(loss)/d(volume) into d_grad float [Z][nmat][N][N] (+=).  Requires a
 * loaded volume (either loader).  Per-ray spectral state is recomputed, not
 * stored. */
int vcbct_projector_adjoint(vcbct_projector* p, const float* d_grad_out, float* d_grad,
                            void* stream);
/* The same pair with the per-ray element path integrals L[V][H][W][nmat]
 * (device, float) kept between them: vcbct_projector_forward_state writes
 * the projection d_out [V][H][W] and L in one launch, and
 * vcbct_projector_adjoint_state reads L instead of re-marching each ray to
 * recompute it; the per-ray spectral derivatives are still recomputed from L.
 * Results are bitwise those of vcbct_projector_forward / _adjoint. */
int vcbct_projector_forward_state(vcbct_projector* p, float* d_out, float* d_L, void* stream);
int vcbct_projector_adjoint_state(vcbct_projector* p, const float* d_L, const float* d_grad_out,
                                  float* d_grad, void* stream);

/* Batched projection (no reference counterpart; the reference projects one
 * phantom per process run).  Items are projector objects holding a volume
 * and a spectrum, each with its own device output [V][H][W]; the items
 * may differ in volume size, view count and detector.  vcbct_batch_forward
 * projects all of them either in one persistent launch that balances the
 * uneven work through a global tile counter (the default), as per-item
 * launches on two branches forked from `stream`, or in one flat launch with a
 * block per tile of every item (vcbct_batch_autotune picks the fastest);
 * with use_graph != 0 the launch sequence
 * is captured into a CUDA graph on the first call and replayed on later calls
 * (the items must not change in between; adding an item rebuilds it). */
typedef struct vcbct_batch vcbct_batch;
int vcbct_batch_create(vcbct_batch** out);
int vcbct_batch_add(vcbct_batch* b, vcbct_projector* p, float* d_out);
int vcbct_batch_forward(vcbct_batch* b, int use_graph, void* stream);
int vcbct_batch_destroy(vcbct_batch* b);
/* Fix the launch strategy (0: persistent launch, 1: per-item launches on two
 * branches, 2: one flat launch with a block per tile of every item) and the
 * columns per block (1, 2, 4 or 8) instead of the defaults (0, 4). */
int vcbct_batch_configure(vcbct_batch* b, int strategy, int cols_per_block);

/* Autotuner: time the launch-shape candidates (columns of the detector per
 * thread block: 2, 4, 8; for a batch also the two launch strategies) on the
 * object's own data and keep the fastest, per geometry signature; with the
 * environment variable VCBCT_TUNE_CACHE naming a file the choices persist
 * across processes.  *chosen = columns per block + 100 x the batch strategy.
 * d_out receives a projection. */
int vcbct_projector_autotune(vcbct_projector* p, float* d_out, void* stream, int* chosen);
int vcbct_batch_autotune(vcbct_batch* b, void* stream, int* chosen);

/* C-linkage twins of the reference-named projector entry points
 * (Release_CBCT_Projection_CM/reprojectionOnGPU.h).  The reference names
 * themselves, with the C++ linkage of the reference headers, are declared in
 * vcbct_reference.h and forward here; these twins serve C and ctypes callers.
 * Same argument lists and meaning, including the ignored ones (ite,
 * reprojection_float, npf_double, projVolume, anglesRad, xalpha,
 * startProjNumber).  vcbct_reprojectionOnGPU writes "<outputname>.raw" as
 * the reference does.  Errors are printed to stderr and leave the state
 * unchanged (the reference exits with status 0 instead). */
void vcbct_initializeGPU(int reconSize, double reconScale, int reconSlices, double reconStep,
                   int projImgHeight, int projImgWidth, int totalProjNumber, double* cosTable,
                   double* sinTable, double* XcenterShift, double* YcenterShift, double x_reg,
                   double y_reg, double z_reg, double DETECTOR_PITCH_CM,
                   double DETECTOR_PITCH_CM_AT_ISO_CENT, double DIST_BTWN_SRC_AND_ISOCENT_CM,
                   double DETECTOR_PIXEL_NUM, int num_material);
void vcbct_terminateGPU(void);
void vcbct_reprojectionOnGPU(int ite, int reconSize, int reconSlices, unsigned short* reconImageshort,
                       float* reprojection_float, float* npf_double, float* projVolume,
                       double reconScale, double reconStep, int projImgWidth,
                       int projImgHeight, int startProjNumber, int endProjNumber,
                       double* anglesRad, double* cosTable, double* sinTable,
                       double* XcenterShift, double* YcenterShift, double xfactor,
                       double* xalpha, double DETECTOR_PITCH_CM,
                       double DETECTOR_PITCH_CM_AT_ISO_CENT,
                       double DIST_BTWN_SRC_AND_ISOCENT_CM, double DETECTOR_PIXEL_NUM,
                       double x_reg, double y_reg, double z_reg, float* Attenuation,
                       float* pdf_pe, int num_material, int NE, char* outputname);

/* Iterative-reconstruction helpers of the projector program.
 *
 * Sensitivity backprojection (replaces lengthproj, lengthproj.h:1-9 /
 * lengthproj.cpp:10-131): for every voxel of the projector's geometry, the
 * sum over views [start_view, end_view) of (65535 - bilinear uint16
 * projection value) x the voxel's chord length, in the reference's float
 * accumulation order; npf float [Z][N][N] is overwritten.  proj uint16
 * [n_views][H][W].  With ite != 0 the registration shifts are ignored, as in
 * the reference.  Host or device buffers; host calls are synchronous. */
int vcbct_projector_lengthproj(vcbct_projector* p, int ite, int start_view, int end_view,
                               const uint16_t* proj, int proj_on_device, float* npf, int npf_on_device,
                               void* stream);
/* MLEM-type update with a total-variation penalty (replaces IR_ImageCBCT,
 * IR_ImageCBCT.h:1-4 / IR_ImageCBCT.cpp:19-93): out = before * (wbefore +
 * (1 - wbefore) * npf_re / (npf + weight_tv * TV(before) + 1e-6)), clamped
 * and masked as the reference does.  Arrays [Z][N][N]; all host or all device
 * (on_device). */
int vcbct_ir_update(int N, int Z, double scale, const short* before, float* out, const float* npf,
                    const float* npf_re, double wbefore, double weight_tv, double weight_prior,
                    int on_device, void* stream);
/* C-linkage twins of lengthproj / IR_ImageCBCT (the reference names are in
 * vcbct_reference.h): host arrays, same argument lists (the unused ones are
 * ignored as in the reference). */
void vcbct_lengthproj(int ite, int reconSize, int reconSlices, short* reconImageshort,
                unsigned short* ProjImageshort, float* npf_float, unsigned short* projVolume,
                double reconScale, double reconStep, int projImgWidth, int projImgHeight,
                int startProjNumber, int endProjNumber, double* ProjAngle, double* cosTable,
                double* sinTable, double* XcenterShift, double* YcenterShift, double xfactor,
                double* xalpha, double DETECTOR_PITCH_CM, double DETECTOR_PITCH_CM_AT_ISO_CENT,
                double DIST_BTWN_SRC_AND_ISOCENT_CM, double DETECTOR_PIXEL_NUM, double x_reg,
                double y_reg, double z_reg);
void vcbct_IR_ImageCBCT(const int ite, int reconSize, int reconSlices, double reconScale,
                  short* reconImageshort_before, float* reconImagefloat, float* npf_float,
                  float* npf_float_re, double wbefore, double weight_tv, double weight_prior,
                  const int thinout);

/* Forward projection that allocates no memory (no counterpart in the
 * reference).  For callers that cannot let a library call cudaMalloc: hosts
 * that own all device memory in their own fixed arena, latency-critical
 * pipelines that cannot accept cudaMalloc's implicit synchronisation or a late
 * out-of-memory failure, deployments that forbid device allocation after
 * start-up.  Same result as vcbct_projector_create + set_spectrum +
 * load_volume (device) + forward (device), in one call.
 *   d_volume  device uint16 [Z][nmat][N][N];  d_out  device float [V][H][W]
 *   tables / attenuation / pdf are host arrays as for the object API; they
 *   are copied before the call returns, so the caller may free or reuse them
 *   at once (page-locked or not).  The device work is asynchronous on
 *   `stream`: d_volume must stay valid, and d_out is written, when the stream
 *   reaches the call.
 * Scratch: one file-scope device array of VCBCT_NOALLOC_SCRATCH_BYTES, held by
 * every GPU that loads the library until the process exits.  Limits:
 * recon_size^2 * recon_slices <= 4177920 voxels (16 B each), n_views <= 1024,
 * n_bins <= 1024; larger requests return VCBCT_ERR_LIMIT, non-finite geometry
 * or xfactor VCBCT_ERR_ARG, before any device work.  Each call looks up the
 * array's device address (cudaGetSymbolAddress) with the caller's device
 * current; the first call on a device also loads the library's kernels
 * there, so make that first call before any stream capture.  Calls share the
 * array: calls that overlap on the GPU (different streams or threads, not
 * ordered) race and corrupt each other. */
#define VCBCT_NOALLOC_SCRATCH_BYTES (64u * 1024u * 1024u)
int vcbct_mbfpa_forward_noalloc(const vcbct_proj_geometry* g, const double* cos_table,
                                const double* sin_table, const double* xcenter_shift,
                                const double* ycenter_shift, const uint16_t* d_volume,
                                const float* attenuation, const float* pdf, int n_bins,
                                double xfactor, float* d_out, void* stream);

/* Host helpers of the projector's input preparation. */
/* misc.cpp:10-37 prepareTrigonometricTable (outputs caller-allocated). */
int vcbct_proj_trig_tables(int proj_width, int proj_height, int n_views,
                           const double* angles_rad, const double* xshift,
                           const double* yshift, double det_pitch_cm, double det_pixel_num,
                           double* cos_table, double* sin_table, double* xcenter_shift,
                           double* ycenter_shift);
/* prior_weight_production.cpp:200-523 attenuation_coefficient: parse the
 * spectrum CSV and look up photo+Compton+Rayleigh (cm^2/g) per element at
 * each bin midpoint in the x-ray DB directory (photo_/comp_/rayl_5keVto150keV
 * .csv).  mu: nmat*VCBCT_MAX_BINS floats, pdf: VCBCT_MAX_BINS floats. */
int vcbct_attenuation_table(const char* spectrum_csv, const char* xraydb_dir, int num_material,
                            int nthin, float* mu, float* pdf, int* n_bins);

/* ------------------------------------------------ projector input deck */

/* The projector's info file (txt), read as loadData does
 * (Release_CBCT_Projection_CM/projectionData.cpp:63-102; fields of
 * projectionData.h:2-63): six header lines, then per field two skipped lines
 * and one value line parsed with the reference's scanf formats.  Relative
 * paths inside are relative to the current directory, as in the reference.
 * The derived members are computed exactly as projectionData.cpp:173-218 and
 * main.cpp:101-103 do; the volume itself is read by
 * vcbct_proj_deck_load_volume. */
typedef struct {
    char spectrum[256];      /* SpectrumString: spectrum CSV path */
    int total_proj;          /* totalProjNumber: views (flexmap entries) */
    int proj_width;          /* projImgWidth */
    int proj_height;         /* projImgHeight */
    char angle_file[256];    /* angleDataFilename: flexmap path */
    char mat_prefix[256];    /* matImgFileDirname: slices "<prefix>_%03d.raw" */
    int z_ic;                /* zICposition as written (isocentre slice) */
    char output_name[256];   /* outputname: projections go to "<name>.raw" */
    double x_scale, y_scale, z_scale;  /* voxel pitch [cm] */
    int recon_size;          /* reconSize: N */
    int recon_slices;        /* reconSlices: slices on disk */
    int mat_num;             /* element planes per slice */
    char mat_type[16];       /* human / watercylinder / ...: no effect on mu */
    double xfactor;          /* density factor */
    double x_reg, y_reg, z_reg_file;   /* registration shift as written */
    /* physParams.h:47-51 ("CM" block) */
    double det_pitch_cm, det_pitch_iso_cm, sad_cm, det_pixel_num, det_iso_cm;
    /* derived */
    int slice_first;         /* linemin: first slice read */
    int used_slices;         /* usedZNumber: slices in the volume */
    int z_ic_local;          /* zICposition - linemin */
    double z_reg;            /* (used_slices/2 - z_ic_local) * z_scale (main.cpp:103) */
} vcbct_proj_deck;

int vcbct_proj_deck_read(const char* txt_path, vcbct_proj_deck* deck);
/* Reads the used_slices slice files into volume uint16
 * [used_slices][mat_num][N][N].  A missing or short slice file leaves that
 * slice holding the previous slice's values (zeros for the first), as the
 * reference's reused read buffer does (projectionData.cpp:187-215); their
 * number goes to *n_incomplete (may be NULL) and a warning to stderr. */
int vcbct_proj_deck_load_volume(const vcbct_proj_deck* deck, uint16_t* volume,
                                int* n_incomplete);
/* The deck's slice files streamed straight into a projector's device volume
 * (the projector's geometry must have the deck's N, used_slices and mat_num):
 * slabs of slices are read into pinned memory while the previous slab is
 * copied and re-laid out on the device.  Same values and missing-file rule as
 * vcbct_proj_deck_load_volume; synchronous. */
int vcbct_projector_load_deck(vcbct_projector* p, const vcbct_proj_deck* deck, int* n_incomplete,
                              void* stream);
/* Flexmap "angle[deg] xshift yshift class" lines (projectionData.cpp:
 * 164-171): angles_rad = angle * pi / 180.  Entries beyond `capacity` return
 * VCBCT_ERR_LIMIT (the reference writes past its arrays); a malformed line
 * returns VCBCT_ERR_IO.  Unfilled entries are left as they are. */
int vcbct_flexmap_read(const char* path, int capacity, double* angles_rad, double* xshift,
                       double* yshift, int* n_entries);

/* ---------------------------------------------------- phantom generator */

/* Element volumes from organ-labelled voxel phantoms, as
 * ICRPphantoms_2mmslice/To_material_distribution_for512_random.cpp does:
 * vcbct_phantom_tables_read parses the media CSV ("id,H,C,N,O,Na,Mg,P,S,Cl,
 * K,Ca,Fe,I" mass percentages) and the organ CSV ("organ,medium,density"),
 * jitters H, C, N (and P, Ca above 0.09 %) of every medium but 53 with
 * N(mu, 0.1 mu) draws and closes the sum with O (renormalising when O < 0),
 * draws (and, as the reference does, does not use) a jittered density per
 * organ, all from the C library's rand() sequence for `seed` (the reference
 * runs with the default seed 1) in the reference's order, and fills
 * table[v] = (short)(percent x density x 10) for H, C, N, O, P, Ca of the
 * last organ row numbered v (0 for numbers without a row; the reference
 * leaves those voxels uninitialised).  vcbct_organs_to_elements maps an
 * organ-number volume uint8 [Z][slice_voxels] to uint16
 * [Z][6][slice_voxels], the projector's input layout; host buffers
 * (on_device 0: synchronous) or device buffers (on_device 1: asynchronous on
 * `stream`, no allocation). */
#define VCBCT_MAX_MEDIA 100
#define VCBCT_MAX_ORGANS 150
typedef struct {
    int n_media, n_organs;
    int media_id[VCBCT_MAX_MEDIA];
    float media[VCBCT_MAX_MEDIA][6];          /* jittered H, C, N, O, P, Ca [%] */
    int organ[VCBCT_MAX_ORGANS];
    int organ_medium[VCBCT_MAX_ORGANS];
    float organ_density[VCBCT_MAX_ORGANS];    /* g/cm3 */
    uint16_t table[256][6];
} vcbct_phantom_tables;
int vcbct_phantom_tables_read(const char* media_csv, const char* organs_csv, unsigned seed,
                              vcbct_phantom_tables* t);
int vcbct_organs_to_elements(const uint8_t* ids, long long slice_voxels, int Z,
                             const vcbct_phantom_tables* t, uint16_t* out, int on_device, void* stream);

/* -------------------------------------------------------------------- FDK */

/* Geometry of filterSinogram / reconstructImage.  The reference fixes
 * MAX_PIC_NUM, DETECTOR_PITCH_CM, DIST_BTWN_SRC_AND_ISOCENT_CM and the filter
 * shape at compile time (R/physParams.h:22-41); here they are fields, and
 * vcbct_fdk_default_geometry() fills the reference's values. */
typedef struct {
    int proj_width;          /* W */
    int proj_height;         /* H */
    int n_views;             /* V (usedProjNumber) */
    int recon_size;          /* N */
    int recon_slices;        /* Z */
    int zstart;              /* reconOffset [cm], an int in the reference */
    double recon_step;       /* [cm] */
    double recon_scale;      /* [cm] */
    int xfactor;             /* CT-value factor (int, R/projectionDataMVkV.h:26) */
    double det_pitch_iso_cm; /* DETECTOR_PITCH_CM_AT_ISO_CENT */
    double det_pitch_cm;     /* DETECTOR_PITCH_CM */
    double max_pic_num;      /* MAX_PIC_NUM */
    double sad_cm;           /* DIST_BTWN_SRC_AND_ISOCENT_CM */
    double cutoff;           /* CUTOFF_FREQ */
    double gamma;            /* GAMMA */
    double alpha;            /* ALPHA */
    int redundancy;          /* 0: none (reference); 1: Parker/half-fan weights */
} vcbct_fdk_geometry;

void vcbct_fdk_default_geometry(vcbct_fdk_geometry* g);

/* VCBCT_FILTER_BF16X3 splits -log p inside the GEMM and stores through TMA
 * when the rows of the projections and of the output are 16-byte aligned
 * (proj_width % 4 == 0 and 16-byte-aligned buffers; always so for the host
 * path, which uses the object's own device buffers); otherwise it splits in
 * a separate pass into a larger workspace.  The results agree within the
 * filter's 1e-5 tolerance either way.  Detectors narrower than 16 or wider
 * than 4096 columns are filtered by the direct path. */
enum {
    VCBCT_FILTER_DIRECT_F32 = 0, /* FP32 direct Toeplitz product (parity path) */
    VCBCT_FILTER_BF16X3 = 1      /* tcgen05 BF16 3-term split GEMM, FP32 accumulate */
};

typedef struct vcbct_fdk vcbct_fdk;

/* angles_rad / xshift / yshift: per view, in the order the projections are
 * stored (the caller applies the reference's CW reversal,
 * projectionDataMVkV.cpp:184-197, as loadData does). */
int vcbct_fdk_create(const vcbct_fdk_geometry* g, const double* angles_rad,
                     const double* xshift, const double* yshift, vcbct_fdk** out);
int vcbct_fdk_destroy(vcbct_fdk* f);
/* The redundancy weights the filter applies to -log p with redundancy = 1,
 * float [n_views][proj_width] into w (host only, no device call): for an
 * offset (half-fan) detector, 2 sin^2(pi/4 (1 + u/u0)) across the band
 * |u| < u0 seen from both sides of the rotation axis, 2 beyond it on the long
 * side, 0 beyond the short edge (u: column position at the isocentre), so
 * that a ray and its conjugate weigh 2 together.  No reference counterpart
 * (the reference has only the offset terms of filterSinogram.cpp:86-87). */
int vcbct_fdk_redundancy_weights(const vcbct_fdk_geometry* g, const double* xshift, float* w);
/* Optional: replace the ramp kernel h[W][W] (prepareConstMap layout). */
int vcbct_fdk_set_kernel(vcbct_fdk* f, const double* h);
/* filterSinogram (R/filterSinogram.cpp:67-131): proj, filtered float [V][H][W]. */
int vcbct_fdk_filter(vcbct_fdk* f, const float* proj, float* filtered, int on_device,
                     int method, void* stream);
/* reconstructImage (R/reconstructImage.cpp:10-184) over filtered [V][H][W]:
 * vol_f32 float [Z][N][N] (may be NULL) and vol_i16 short [Z][N][N] (the
 * (short) cast of R/main.cpp:179-185; may be NULL).  Overwrites. */
int vcbct_fdk_backproject(vcbct_fdk* f, const float* filtered, float* vol_f32, short* vol_i16,
                          int on_device, void* stream);

/* The FDK info file, read as loadData + loadProjectionData do
 * (R/projectionDataMVkV.cpp:51-321; fields of projectionDataMVkV.h:2-42):
 *  - the "first file number" field is read in hex for "kV", in decimal for
 *    "MV"; any other energy class returns VCBCT_ERR_ARG (the reference then
 *    skips the field and leaves the isocentre pitch unset); kV and MV use
 *    the same pitch at the isocentre (R/physParams.h:24-25);
 *  - flexmap entries whose class matches target_class ("*" = all) are kept;
 *    the list is reversed when the 1st angle minus the 30th is negative
 *    (:156-211); with fewer than 30 entries the reference reads an
 *    uninitialised value, and here the list is kept in file order;
 *  - recon_slices is corrected when recon_offset + recon_step *
 *    (recon_slices - 1) reaches proj_height (:283-302);
 *  - panel_class is S / M / L from the mean xshift (:276-281).
 * The per-view arrays hold total_proj entries (the views in the projection
 * file); entries beyond n_target stay zero.  More than VCBCT_FDK_MAX_VIEWS
 * flexmap lines, or more matching lines than total_proj, return
 * VCBCT_ERR_LIMIT (the reference overruns its arrays). */
#define VCBCT_FDK_MAX_VIEWS 1080   /* MAX_Proj_Num, R/physParams.h:47 */
typedef struct {
    char energy_class[16];   /* kVMVClassString */
    int total_proj;          /* totalProjNumber as written = usedProjNumber */
    int proj_width;
    int proj_height;
    int proj_header_bytes;   /* projImgFileOffset (unused by the float path) */
    char proj_prefix[256];   /* projImgFileDirname: the file is "<prefix>.<ext>" */
    int proj_num_digits;     /* projImgFileNumDigits (unused) */
    int proj_first_number;   /* projImgFile1stNumber (unused; 0 if unparsed) */
    char proj_ext[8];        /* projImgFileExt */
    char angle_file[256];
    int recon_size;
    char target_class[16];   /* reconTgtClassString */
    int recon_offset;        /* zstart [cm] (an int) */
    double recon_step;
    int recon_slices;        /* after the slice-count correction */
    double recon_scale;
    int xfactor;
    char recon_file[256];    /* reconDataFilename: short volume output */
    double det_pitch_iso_cm;
    int n_lines;             /* flexmap entries */
    int n_target;            /* entries matching target_class */
    int reversed;            /* 1 when the list was reversed */
    char panel_class[8];     /* SMLClassString */
    double angles_rad[VCBCT_FDK_MAX_VIEWS];
    double xshift[VCBCT_FDK_MAX_VIEWS];
    double yshift[VCBCT_FDK_MAX_VIEWS];
} vcbct_fdk_deck;

int vcbct_fdk_deck_read(const char* txt_path, vcbct_fdk_deck* deck);

/* C-linkage twins of the reference-named FDK entry points
 * (R/filterSinogram.h:2-6, R/reconstructImage.h:2-5; the reference names are
 * in vcbct_reference.h).  Arrays are VOLUME-ONE style pointer tables over
 * contiguous storage (mallocMD.cpp:69-109).  vcbct_prepareConstMap returns a
 * pointer table laid out as new2DArray's (one calloc'd block, one malloc'd
 * row table), which the caller frees with vcbct_free_const_map or the
 * reference's delete2DArray. */
double** vcbct_prepareConstMap(int projWidth, double DETECTOR_PITCH_CM_AT_ISO_CENT);
void vcbct_free_const_map(double** constMap, int projWidth);
void vcbct_filterSinogram(int projHeight, int projWidth, int sngrmHeight, float*** projVolume,
                    float*** fltdVoxData, double** constMap, double* xshift, double* yshift,
                    double DETECTOR_PITCH_CM_AT_ISO_CENT);
void vcbct_reconstructImage(int reconSize, int reconSlices, int zstart, double reconStep,
                      double reconScale, double*** reconVoxData, char** maskData,
                      int projHeight, int projWidth, int sngrmHeight, float*** sngrmVoxData,
                      int xfactor, double* anglesRad, double* cosTable, double* sinTable,
                      double* xshift, double DETECTOR_PITCH_CM_AT_ISO_CENT);

#ifdef __cplusplus
}
#endif
#endif /* VCBCT_H */
