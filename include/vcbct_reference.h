/*
 * vcbct_reference.h -- the reference program's own entry points, exported by
 * libvcbct with the reference's C++ linkage, so that the reference's drivers
 * (Release_CBCT_Projection_CM/main.cpp, Release_recon_from_forward_pro_float_CM
 * /main.cpp), compiled unchanged against the reference's own headers, link
 * against -lvcbct in place of reprojectionOnGPU.o, lengthproj.o,
 * IR_ImageCBCT.o, filterSinogram.o and reconstructImage.o.
 *
 * The reference headers declare these without extern "C", so the linker
 * looks for their C++ (mangled) names; the prototypes below are the
 * reference's, parameter type for parameter type.  Each forwards to the
 * C-linkage twin of the same name with a vcbct_ prefix in vcbct.h, which
 * documents the behaviour (host arrays, synchronous, errors printed to
 * stderr instead of exit(0)).
 *
 * C++ only: a C caller uses the vcbct_ twins.
 */
#ifndef VCBCT_REFERENCE_H
#define VCBCT_REFERENCE_H

#ifndef __cplusplus
#error "vcbct_reference.h declares C++-linkage functions; C callers use the vcbct_ twins in vcbct.h"
#endif

/* Release_CBCT_Projection_CM/reprojectionOnGPU.h:2-8 */
void initializeGPU(int reconSize, double reconScale, int reconSlices, double reconStep,
                   int projImgHeight, int projImgWidth, int totalProjNumber, double* cosTable,
                   double* sinTable, double* XcenterShift, double* YcenterShift, double x_reg,
                   double y_reg, double z_reg, double DETECTOR_PITCH_CM,
                   double DETECTOR_PITCH_CM_AT_ISO_CENT, double DIST_BTWN_SRC_AND_ISOCENT_CM,
                   double DETECTOR_PIXEL_NUM, int num_material);

/* Release_CBCT_Projection_CM/reprojectionOnGPU.h:10 */
void terminateGPU();

/* Release_CBCT_Projection_CM/reprojectionOnGPU.h:12-19; writes
 * "<outputname>.raw" as the reference does. */
void reprojectionOnGPU(int ite, int reconSize, int reconSlices, unsigned short* reconImageshort,
                       float* reprojection_float, float* npf_double, float* projVolume,
                       double reconScale, double reconStep, int projImgWidth, int projImgHeight,
                       int startProjNumber, int endProjNumber, double* anglesRad, double* cosTable,
                       double* sinTable, double* XcenterShift, double* YcenterShift, double xfactor,
                       double* xalpha, double DETECTOR_PITCH_CM, double DETECTOR_PITCH_CM_AT_ISO_CENT,
                       double DIST_BTWN_SRC_AND_ISOCENT_CM, double DETECTOR_PIXEL_NUM, double x_reg,
                       double y_reg, double z_reg, float* Attenuation, float* pdf_pe, int num_material,
                       int NE, char* outputname);

/* Release_CBCT_Projection_CM/lengthproj.h:1-9 */
void lengthproj(int ite, int reconSize, int reconSlices, short* reconImageshort,
                unsigned short* ProjImageshort, float* npf_double, unsigned short* projVolume,
                double reconScale, double reconStep, int projImgWidth, int projImgHeight,
                int startProjNumber, int endProjNumber, double* anglesRad, double* cosTable,
                double* sinTable, double* XcenterShift, double* YcenterShift, double xfactor,
                double* xalpha, double DETECTOR_PITCH_CM, double DETECTOR_PITCH_CM_AT_ISO_CENT,
                double DIST_BTWN_SRC_AND_ISOCENT_CM, double DETECTOR_PIXEL_NUM, double x_reg,
                double y_reg, double z_reg);

/* Release_CBCT_Projection_CM/IR_ImageCBCT.h:1-4 */
void IR_ImageCBCT(const int ite, int reconSize, int reconSlices, double reconScale,
                  short* reconImageshort_before, float* reconImagefloat, float* npf_float,
                  float* npf_float_re, double wbefore, double weight_tv, double weight_prior,
                  const int thinout);

/* Release_recon_from_forward_pro_float_CM/filterSinogram.h:2; the returned
 * table is laid out as the reference's new2DArray (one data block, one row
 * table), so the reference's delete2DArray frees it. */
double** prepareConstMap(int projWidth, double DETECTOR_PITCH_CM_AT_ISO_CENT);

/* Release_recon_from_forward_pro_float_CM/filterSinogram.h:4-6; filters with
 * the tensor-core BF16x3 GEMM (VCBCT_FILTER=direct: the FP32 direct
 * filter), both within 1e-5 of the FP64 filter's output scale. */
void filterSinogram(int projHeight, int projWidth, int sngrmHeight, float*** projVolume,
                    float*** fltdVoxData, double** constMap, double* xshift, double* yshift,
                    double DETECTOR_PITCH_CM_AT_ISO_CENT);

/* Release_recon_from_forward_pro_float_CM/reconstructImage.h:2-5; accumulates
 * into reconVoxData as the reference does. */
void reconstructImage(int reconSize, int reconSlices, int zstart, double reconStep, double reconScale,
                      double*** reconVoxData, char** maskData, int projHeight, int sngrmWidth,
                      int sngrmHeight, float*** sngrmVoxData, int xfactor, double* anglesRad,
                      double* cosTable, double* sinTable, double* xshift,
                      double DETECTOR_PITCH_CM_AT_ISO_CENT);

#endif /* VCBCT_REFERENCE_H */
