// noalloc.cu -- a forward-projection entry point that allocates no memory.
//
// Some callers cannot let a library call cudaMalloc: hosts that own all device
// memory through their own fixed arena (a plugin framework that budgets
// memory at start-up), latency-critical pipelines for which cudaMalloc's
// implicit device synchronisation or a late out-of-memory failure is not
// acceptable, and deployments that forbid dynamic device allocation after
// initialisation.  vcbct_mbfpa_forward_noalloc serves them: the caller passes
// every input and the output; the only device memory it touches besides those
// is the fixed array below, which every GPU that loads the library holds
// until the process exits.
#include <cmath>
#include <cstring>
#include <mutex>

#include "internal.h"

namespace vcbct {
namespace {

constexpr size_t kScratchBytes = VCBCT_NOALLOC_SCRATCH_BYTES;
// [0, 256 KiB): raw caller tables and the rebuilt view / spectrum tables;
// [256 KiB, end): the packed volume.
constexpr size_t kTableRegion = 256 * 1024;
constexpr size_t kMaxViews = 1024;
constexpr size_t kOffRaw = 0;                 // caller's cos/sin/Xc/Yc: 4 x V doubles (<= 32 KiB)
constexpr size_t kOffViews = 128 * 1024;      // ViewGeom[V] built from them (<= 32 KiB)
constexpr size_t kOffMuRaw = 160 * 1024;      // caller's mu [nmat][NE] floats (<= 32 KiB)
constexpr size_t kOffMu8 = 192 * 1024;        // [NE][8] floats mu / xfactor (<= 32 KiB)
constexpr size_t kOffPdf = 224 * 1024;        // [NE] floats (<= 4 KiB)

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Host staging of the caller's tables, laid out as the device table region.
// It is ordinary pageable memory: a cudaMemcpyAsync from pageable host memory
// to the device has consumed its source by the time it returns (the runtime
// stages it), so once this entry point returns the caller may free or reuse
// its host tables, whether or not they are page-locked.  The mutex keeps two
// host threads from filling it at once.
std::mutex g_stage_mu;
unsigned char g_host_stage[kTableRegion];

// ViewGeom records from the four caller tables (copied raw into scratch).
__global__ void build_views_kernel(const double* raw, int V, ViewGeom* out)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < V) out[v] = ViewGeom{raw[v], raw[V + v], raw[2 * V + v], raw[3 * V + v]};
}

// [NE][8] table of mu_k(E) / xfactor (zero padded) from mu [nmat][NE].
__global__ void build_mu8_kernel(const float* mu, int nmat, int NE, double xfactor, float* mu8)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NE * 8) return;
    const int e = i / 8, k = i % 8;
    mu8[i] = (k < nmat) ? (float)((double)mu[(size_t)k * NE + e] / xfactor) : 0.0f;
}

}  // namespace
}  // namespace vcbct

using namespace vcbct;

extern "C" int vcbct_mbfpa_forward_noalloc(const vcbct_proj_geometry* g, const double* cos_table,
                                           const double* sin_table, const double* xcenter_shift,
                                           const double* ycenter_shift, const uint16_t* d_volume,
                                           const float* attenuation, const float* pdf,
                                           int n_bins, double xfactor, float* d_out, void* stream)
{
    // all size checks come first: nothing reaches the device on a rejection
    if (!g || !cos_table || !sin_table || !xcenter_shift || !ycenter_shift || !d_volume ||
        !attenuation || !pdf || !d_out)
        return fail(VCBCT_ERR_ARG, "vcbct_mbfpa_forward_noalloc: NULL argument");
    if (g->recon_size <= 0 || g->recon_slices <= 0 || g->proj_width <= 0 || g->proj_height <= 0 ||
        g->n_views <= 0 || g->num_material <= 0 || g->num_material > VCBCT_MAX_MATERIALS)
        return fail(VCBCT_ERR_ARG, "vcbct_mbfpa_forward_noalloc: invalid geometry");
    if (!(g->recon_scale > 0) || !(g->recon_step > 0) || !(g->sad_cm > 0) || !(g->det_pitch_cm > 0) ||
        !(g->det_pitch_iso_cm > 0) || !(g->det_pixel_num > 0))
        return fail(VCBCT_ERR_ARG, "vcbct_mbfpa_forward_noalloc: pitches and distances must be positive");
    if (!std::isfinite(g->recon_scale) || !std::isfinite(g->recon_step) || !std::isfinite(g->sad_cm) ||
        !std::isfinite(g->det_pitch_cm) || !std::isfinite(g->det_pitch_iso_cm) || !std::isfinite(g->det_pixel_num) ||
        !std::isfinite(g->x_reg) || !std::isfinite(g->y_reg) || !std::isfinite(g->z_reg))
        return fail(VCBCT_ERR_ARG, "vcbct_mbfpa_forward_noalloc: geometry values must be finite");
    if (n_bins <= 0 || n_bins > VCBCT_MAX_BINS || !(xfactor != 0.0) || !std::isfinite(xfactor))
        return fail(VCBCT_ERR_ARG,
                    "vcbct_mbfpa_forward_noalloc: n_bins must be in [1, 1024], xfactor finite and non-zero");
    if ((size_t)g->n_views > kMaxViews)
        return fail(VCBCT_ERR_LIMIT, "vcbct_mbfpa_forward_noalloc: at most 1024 views");
    const double vol_bytes = (double)g->recon_size * g->recon_size * g->recon_slices * sizeof(uint4);
    if (vol_bytes > (double)(kScratchBytes - kTableRegion))
        return fail(VCBCT_ERR_LIMIT,
                    "vcbct_mbfpa_forward_noalloc: volume exceeds the fixed scratch (recon_size^2 * "
                    "recon_slices must be <= 4177920 voxels; use vcbct_projector_* for larger volumes)");

    // The device address of the scratch array, looked up on every call with
    // the caller's device current (the host-side name of g_noalloc_scratch is
    // not a device address).  The lookup is a runtime table read; doing it per
    // call keeps the address right after a cudaDeviceReset.  The first call on
    // a device also loads this library's kernels there, which is why that
    // first call belongs outside any stream capture.
    void* sym = nullptr;
    VCBCT_CUDA_TRY(cudaGetSymbolAddress(&sym, g_noalloc_scratch));
    unsigned char* base = static_cast<unsigned char*>(sym);
    cudaStream_t st = (cudaStream_t)stream;
    const int V = g->n_views, NE = n_bins, nmat = g->num_material;
    double* raw = reinterpret_cast<double*>(base + kOffRaw);
    ViewGeom* views = reinterpret_cast<ViewGeom*>(base + kOffViews);
    float* mu_raw = reinterpret_cast<float*>(base + kOffMuRaw);
    float* mu8 = reinterpret_cast<float*>(base + kOffMu8);
    float* dpdf = reinterpret_cast<float*>(base + kOffPdf);
    uint4* vol = reinterpret_cast<uint4*>(base + kTableRegion);

    // Every region read below is fully rewritten by this call, so the
    // contents left by a previous call need no clearing.
    {
        std::lock_guard<std::mutex> lk(g_stage_mu);
        double* hraw = reinterpret_cast<double*>(g_host_stage + kOffRaw);
        std::memcpy(hraw, cos_table, sizeof(double) * V);
        std::memcpy(hraw + V, sin_table, sizeof(double) * V);
        std::memcpy(hraw + 2 * V, xcenter_shift, sizeof(double) * V);
        std::memcpy(hraw + 3 * V, ycenter_shift, sizeof(double) * V);
        std::memcpy(g_host_stage + kOffMuRaw, attenuation, sizeof(float) * nmat * NE);
        std::memcpy(g_host_stage + kOffPdf, pdf, sizeof(float) * NE);
        VCBCT_CUDA_TRY(cudaMemcpyAsync(raw, hraw, sizeof(double) * 4 * V, cudaMemcpyHostToDevice, st));
        VCBCT_CUDA_TRY(cudaMemcpyAsync(mu_raw, g_host_stage + kOffMuRaw, sizeof(float) * nmat * NE,
                                       cudaMemcpyHostToDevice, st));
        VCBCT_CUDA_TRY(cudaMemcpyAsync(dpdf, g_host_stage + kOffPdf, sizeof(float) * NE, cudaMemcpyHostToDevice,
                                       st));
    }
    build_views_kernel<<<(V + 127) / 128, 128, 0, st>>>(raw, V, views);
    VCBCT_CUDA_TRY(cudaGetLastError());
    build_mu8_kernel<<<(NE * 8 + 255) / 256, 256, 0, st>>>(mu_raw, nmat, NE, xfactor, mu8);
    VCBCT_CUDA_TRY(cudaGetLastError());
    VCBCT_CUDA_TRY(launch_pack_u16(d_volume, g->recon_size, g->recon_slices, nmat, vol, st));

    ForwardArgs a{};
    a.p = ProjParams{g->recon_size, g->recon_slices, g->proj_width, g->proj_height, V, nmat,
                     g->recon_scale, g->recon_step, g->det_pitch_cm, g->det_pitch_iso_cm, g->sad_cm,
                     g->det_pixel_num, g->x_reg, g->y_reg, g->z_reg};
    a.views = views;
    a.spec = SpectrumDev{reinterpret_cast<const float4*>(mu8), dpdf, NE};
    a.vol_u16 = vol;
    a.out = d_out;
    a.cols_per_block = 4;
    VCBCT_CUDA_TRY(launch_forward(a, st));
    return VCBCT_OK;
}
