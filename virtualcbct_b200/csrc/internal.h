// internal.h -- shared declarations of libvcbct's CUDA translation units.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>

#include "vcbct.h"

namespace vcbct {

// Thread-local error message behind vcbct_last_error().
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define VCBCT_CUDA_TRY(call)                                  \
    do {                                                      \
        cudaError_t e__ = (call);                             \
        if (e__ != cudaSuccess) return ::vcbct::cuda_fail(e__, #call); \
    } while (0)

// Per-view geometry the projector kernels read (double, from the host
// tables of prepareTrigonometricTable, misc.cpp:10-37).
struct ViewGeom {
    double cs, sn, xc, yc;
};

// Scalar projection geometry passed by value to the kernels.
struct ProjParams {
    int N, Z, W, H, V, nmat;
    double s, step, pdet, piso, sad, dpn, xr, yr, zr;
};

// ---------------------------------------------------------------- MBFPA --
// Packed volume: voxel (x, y, z) at index (y*N + x)*Z + z, one 16-byte record
// of 8 uint16 element values (u16 form) or two 16-byte records of 8 floats
// (f32 form).  Elements beyond nmat are zero.  The projector object keeps
// every volume in the f32 form (uint16 values convert exactly): the march
// then gathers without converting, 1.8 % faster on B200 than the u16 form
// (512x512x200 x 6, 360 views) with the same projections bit for bit.  The
// u16 form serves the scratch-free entry point, whose fixed scratch holds
// half as many voxels in the f32 form.
size_t packed_u16_bytes(int N, int Z);
size_t packed_f32_bytes(int N, int Z);

// uint16 slab [nz][nmat][N][N] -> slices [zoff, zoff + nz) of an f32-form volume
cudaError_t launch_pack_u16_f32_slab(const uint16_t* src, int N, int nz, int zoff, int Z, int nmat, float4* dst,
                                     cudaStream_t st);
cudaError_t launch_pack_u16(const uint16_t* src, int N, int Z, int nmat, uint4* dst,
                            cudaStream_t st);
cudaError_t launch_pack_f32(const float* src, int N, int Z, int nmat, float4* dst,
                            cudaStream_t st);
cudaError_t launch_unpack_grad(const float* planes, int N, int Z, int nmat, float* dst, cudaStream_t st);

// Spectral table: per bin 8 floats mu_k(E)/xfactor (zero padded) + pdf.
struct SpectrumDev {
    const float4* mu8;  // [NE][2] float4
    const float* pdf;   // [NE]
    int NE;
};

struct ForwardArgs {
    ProjParams p;
    const ViewGeom* views;   // device [V]
    SpectrumDev spec;
    const uint4* vol_u16;    // packed (or nullptr)
    const float4* vol_f32;   // packed (or nullptr)
    float* out;              // [V][H][W] intensities (or nullptr)
    float* L_out;            // [V][H][W][nmat] path integrals (or nullptr)
    unsigned long long* seg_count;  // (or nullptr)
    int* err_flag;           // device fault flag
    int cols_per_block;
    // detector noise on `out` (kind 0: none, 1: Gaussian counts)
    int noise_kind;
    int view_offset;         // global index of view 0 of this launch (noise counters)
    int band0, nbands;       // detector row bands [band0, band0 + nbands) of 32 rows (nbands 0: all)
    double noise_i0, noise_max;
    unsigned long long noise_seed;
};
cudaError_t launch_forward(const ForwardArgs& a, cudaStream_t st);
// Slice range [span[2b], span[2b+1]] the forward projection of detector row
// band b (rows 32b..32b+31, all views) can read; span must hold (Z, -1) per
// band on entry (bands that read nothing keep it).
cudaError_t launch_band_footprint(const ProjParams& P, const ViewGeom* d_views, int* d_span, cudaStream_t st);
cudaError_t launch_gaussian_noise(float* proj, size_t n, double max_pixvalue, unsigned long long seed,
                                  cudaStream_t st);

// Items of one single-launch batch, passed in the kernel's parameter block.
constexpr int kFlatItems = 40;
struct FlatBatch {
    int nitems;
    int ncolb[kFlatItems];
    long long begin[kFlatItems + 1];  // first tile of each item; begin[nitems] = total
    ForwardArgs fa[kFlatItems];
};
cudaError_t launch_flat_batch(const FlatBatch& b, int NEmax, int nmat_max, int cols_per_block, cudaStream_t st);

// The same items in one persistent launch of `blocks` blocks that take work
// tiles from `counter` (zeroed by the launch).
cudaError_t launch_persistent_batch(const FlatBatch& b, int NEmax, int nmat_max, int cols_per_block, int blocks,
                                   unsigned long long* counter, cudaStream_t st);
int batch_blocks_per_sm(int nmat_max, int cols_per_block, int NEmax);

struct AdjointArgs {
    ProjParams p;
    const ViewGeom* views;
    SpectrumDev spec;
    const float4* vol_f32;   // packed float volume
    const float* grad_out;   // [V][H][W] d loss / d intensity
    const float* L_in;       // [V][H][W][nmat] path integrals of the forward, or
                             // nullptr: recompute them (first march)
    float* grad_planes;      // float accumulator, z fastest, ceil(nmat/2) x 2 floats per voxel: groups of
                             // four elements [N*N*Z][4], the last a pair [N*N*Z][2] if it holds one or two
    int* err_flag;
    int cols_per_block;
    int y0, y1;              // scatter only into volume rows iy in [y0, y1) (y1 <= y0: all)
};
cudaError_t launch_adjoint(const AdjointArgs& a, cudaStream_t st);

// ------------------------------------------------------ iterative recon --
// Geometry of lengthproj (the projector's, with the registration shifts the
// call uses).
struct LpParams {
    int N, Z, W, H;
    double s, step, pdet, piso, sad, dpn, xr, yr, zr;
};
size_t lengthproj_scratch_bytes(int n_views);
cudaError_t launch_lengthproj(const LpParams& q, const ViewGeom* d_views, int v0, int v1, const uint16_t* d_proj,
                              float* d_npf, void* d_scratch, cudaStream_t st);
cudaError_t launch_ir_update(int N, int Z, double scale, const short* d_before, float* d_out, const float* d_npf,
                             const float* d_npf_re, double wbefore, double weight_tv, double weight_prior,
                             cudaStream_t st);

// ------------------------------------------------------------------ FDK --
struct FdkParams {
    int W, H, V, N, Z, zstart, xfactor, redundancy;
    double step, scale, piso, pdet, mpn, sad;
};

// Per-view filter constants: detector centre shifts of filterSinogram.cpp:86-87.
struct FilterView {
    float xcs, ycs;
};
// Direct FP32 ramp filter.  hT: [W][W] float, hT[k][m] = h[m][k] + coeff*(m==k).
// wts: optional [V][W] redundancy weights applied to -log(p) before filtering.
cudaError_t launch_filter_direct(const float* proj, float* out, const float* hT,
                                 const FilterView* views, const float* wts, float pitch,
                                 float sad, int V, int H, int W, cudaStream_t st);

struct BpView {
    double cs, sn;   // cos / sin of the view angle
    double ushift;   // W/2 - 0.5 + xshift in pixels (reconstructImage.cpp:83)
    float dbeta;     // half the neighbouring angular gap (:45-71)
    float pad;
};
// keep: backproject_workspace_bytes(f) of device scratch holding the
// per-block view masks, a function of the geometry and the views only: with
// *keep_ready set they are taken as made and not redone; the launch sets it
// once it has queued them (keep_ready may be null: made every call).
size_t backproject_workspace_bytes(const FdkParams& f);
cudaError_t launch_backproject(const FdkParams& f, const BpView* d_views, const float* filt,
                               float* vol_f32, short* vol_i16, unsigned* keep, int* keep_ready,
                               cudaStream_t st);

// BF16 3-term split tensor-core ramp filter (tcgen05).  The workspace holds
// the split Toeplitz planes: with *b_ready set they are taken as already
// split from hT into this workspace and are not redone; the launch sets it
// once it has queued the split (b_ready may be null: split every call).
// The fused form (rows of `proj` and `out` 16-byte aligned: W % 4 == 0 and
// aligned bases, ramp_gemm_fused) splits -ln p inside the GEMM and stores
// through TMA; the other needs room for the split A planes as well: size the
// workspace with the same flag.
bool ramp_gemm_fused(const float* proj, const float* out, int W);
size_t ramp_gemm_workspace_bytes(int V, int H, int W, bool fused);
cudaError_t launch_ramp_gemm_bf16x3(const float* proj, float* out, const float* hT,
                                    const FilterView* views, const float* wts, float pitch,
                                    float sad, int V, int H, int W, void* workspace,
                                    int* b_ready, cudaStream_t st);
// The kernel's fault flag (1 after a bounded wait ran out; its output is then
// invalid), read synchronously on `st`; -1 if it cannot be read.
int ramp_gemm_error_flag(void* workspace, int V, int H, int W, cudaStream_t st);

}  // namespace vcbct
