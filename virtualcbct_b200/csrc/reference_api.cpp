// reference_api.cpp -- the reference's entry points with C++ linkage
// (include/vcbct_reference.h), each forwarding to its vcbct_ C twin.
//
// The reference's drivers include the reference's own headers, which declare
// these functions without extern "C"; defining them here in a C++
// translation unit gives them the same mangled names, so those drivers link
// against -lvcbct unchanged.
#include "vcbct.h"
#include "vcbct_reference.h"

void initializeGPU(int reconSize, double reconScale, int reconSlices, double reconStep, int projImgHeight,
                   int projImgWidth, int totalProjNumber, double* cosTable, double* sinTable, double* XcenterShift,
                   double* YcenterShift, double x_reg, double y_reg, double z_reg, double DETECTOR_PITCH_CM,
                   double DETECTOR_PITCH_CM_AT_ISO_CENT, double DIST_BTWN_SRC_AND_ISOCENT_CM,
                   double DETECTOR_PIXEL_NUM, int num_material)
{
    vcbct_initializeGPU(reconSize, reconScale, reconSlices, reconStep, projImgHeight, projImgWidth, totalProjNumber,
                        cosTable, sinTable, XcenterShift, YcenterShift, x_reg, y_reg, z_reg, DETECTOR_PITCH_CM,
                        DETECTOR_PITCH_CM_AT_ISO_CENT, DIST_BTWN_SRC_AND_ISOCENT_CM, DETECTOR_PIXEL_NUM,
                        num_material);
}

void terminateGPU() { vcbct_terminateGPU(); }

void reprojectionOnGPU(int ite, int reconSize, int reconSlices, unsigned short* reconImageshort,
                       float* reprojection_float, float* npf_double, float* projVolume, double reconScale,
                       double reconStep, int projImgWidth, int projImgHeight, int startProjNumber,
                       int endProjNumber, double* anglesRad, double* cosTable, double* sinTable,
                       double* XcenterShift, double* YcenterShift, double xfactor, double* xalpha,
                       double DETECTOR_PITCH_CM, double DETECTOR_PITCH_CM_AT_ISO_CENT,
                       double DIST_BTWN_SRC_AND_ISOCENT_CM, double DETECTOR_PIXEL_NUM, double x_reg, double y_reg,
                       double z_reg, float* Attenuation, float* pdf_pe, int num_material, int NE, char* outputname)
{
    vcbct_reprojectionOnGPU(ite, reconSize, reconSlices, reconImageshort, reprojection_float, npf_double,
                            projVolume, reconScale, reconStep, projImgWidth, projImgHeight, startProjNumber,
                            endProjNumber, anglesRad, cosTable, sinTable, XcenterShift, YcenterShift, xfactor,
                            xalpha, DETECTOR_PITCH_CM, DETECTOR_PITCH_CM_AT_ISO_CENT, DIST_BTWN_SRC_AND_ISOCENT_CM,
                            DETECTOR_PIXEL_NUM, x_reg, y_reg, z_reg, Attenuation, pdf_pe, num_material, NE,
                            outputname);
}

void lengthproj(int ite, int reconSize, int reconSlices, short* reconImageshort, unsigned short* ProjImageshort,
                float* npf_double, unsigned short* projVolume, double reconScale, double reconStep,
                int projImgWidth, int projImgHeight, int startProjNumber, int endProjNumber, double* anglesRad,
                double* cosTable, double* sinTable, double* XcenterShift, double* YcenterShift, double xfactor,
                double* xalpha, double DETECTOR_PITCH_CM, double DETECTOR_PITCH_CM_AT_ISO_CENT,
                double DIST_BTWN_SRC_AND_ISOCENT_CM, double DETECTOR_PIXEL_NUM, double x_reg, double y_reg,
                double z_reg)
{
    vcbct_lengthproj(ite, reconSize, reconSlices, reconImageshort, ProjImageshort, npf_double, projVolume,
                     reconScale, reconStep, projImgWidth, projImgHeight, startProjNumber, endProjNumber, anglesRad,
                     cosTable, sinTable, XcenterShift, YcenterShift, xfactor, xalpha, DETECTOR_PITCH_CM,
                     DETECTOR_PITCH_CM_AT_ISO_CENT, DIST_BTWN_SRC_AND_ISOCENT_CM, DETECTOR_PIXEL_NUM, x_reg, y_reg,
                     z_reg);
}

void IR_ImageCBCT(const int ite, int reconSize, int reconSlices, double reconScale, short* reconImageshort_before,
                  float* reconImagefloat, float* npf_float, float* npf_float_re, double wbefore, double weight_tv,
                  double weight_prior, const int thinout)
{
    vcbct_IR_ImageCBCT(ite, reconSize, reconSlices, reconScale, reconImageshort_before, reconImagefloat, npf_float,
                       npf_float_re, wbefore, weight_tv, weight_prior, thinout);
}

double** prepareConstMap(int projWidth, double DETECTOR_PITCH_CM_AT_ISO_CENT)
{
    return vcbct_prepareConstMap(projWidth, DETECTOR_PITCH_CM_AT_ISO_CENT);
}

void filterSinogram(int projHeight, int projWidth, int sngrmHeight, float*** projVolume, float*** fltdVoxData,
                    double** constMap, double* xshift, double* yshift, double DETECTOR_PITCH_CM_AT_ISO_CENT)
{
    vcbct_filterSinogram(projHeight, projWidth, sngrmHeight, projVolume, fltdVoxData, constMap, xshift, yshift,
                         DETECTOR_PITCH_CM_AT_ISO_CENT);
}

void reconstructImage(int reconSize, int reconSlices, int zstart, double reconStep, double reconScale,
                      double*** reconVoxData, char** maskData, int projHeight, int sngrmWidth, int sngrmHeight,
                      float*** sngrmVoxData, int xfactor, double* anglesRad, double* cosTable, double* sinTable,
                      double* xshift, double DETECTOR_PITCH_CM_AT_ISO_CENT)
{
    vcbct_reconstructImage(reconSize, reconSlices, zstart, reconStep, reconScale, reconVoxData, maskData,
                           projHeight, sngrmWidth, sngrmHeight, sngrmVoxData, xfactor, anglesRad, cosTable, sinTable,
                           xshift, DETECTOR_PITCH_CM_AT_ISO_CENT);
}
