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

std::mutex g_mu;
constexpr int kMaxDevices = 64;
unsigned char* g_addr[kMaxDevices] = {};

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
    if (n_bins <= 0 || n_bins > VCBCT_MAX_BINS || !(xfactor != 0.0))
        return fail(VCBCT_ERR_ARG, "vcbct_mbfpa_forward_noalloc: n_bins must be in [1, 1024], xfactor non-zero");
    if ((size_t)g->n_views > kMaxViews)
        return fail(VCBCT_ERR_LIMIT, "vcbct_mbfpa_forward_noalloc: at most 1024 views");
    const double vol_bytes = (double)g->recon_size * g->recon_size * g->recon_slices * sizeof(uint4);
    if (vol_bytes > (double)(kScratchBytes - kTableRegion))
        return fail(VCBCT_ERR_LIMIT,
                    "vcbct_mbfpa_forward_noalloc: volume exceeds the fixed scratch (recon_size^2 * "
                    "recon_slices must be <= 4177920 voxels; use vcbct_projector_* for larger volumes)");

    int dev = 0;
    VCBCT_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(VCBCT_ERR_LIMIT, "device ordinal out of range");
    unsigned char* base = nullptr;
    {
        // once per device, with that device current: the host-side name of
        // g_noalloc_scratch is not a device address
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_addr[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
            g_addr[dev] = static_cast<unsigned char*>(p);
        }
        base = g_addr[dev];
    }
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
    VCBCT_CUDA_TRY(cudaMemcpyAsync(raw, cos_table, sizeof(double) * V, cudaMemcpyHostToDevice, st));
    VCBCT_CUDA_TRY(cudaMemcpyAsync(raw + V, sin_table, sizeof(double) * V, cudaMemcpyHostToDevice, st));
    VCBCT_CUDA_TRY(cudaMemcpyAsync(raw + 2 * V, xcenter_shift, sizeof(double) * V, cudaMemcpyHostToDevice, st));
    VCBCT_CUDA_TRY(cudaMemcpyAsync(raw + 3 * V, ycenter_shift, sizeof(double) * V, cudaMemcpyHostToDevice, st));
    VCBCT_CUDA_TRY(cudaMemcpyAsync(mu_raw, attenuation, sizeof(float) * nmat * NE, cudaMemcpyHostToDevice, st));
    VCBCT_CUDA_TRY(cudaMemcpyAsync(dpdf, pdf, sizeof(float) * NE, cudaMemcpyHostToDevice, st));
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
