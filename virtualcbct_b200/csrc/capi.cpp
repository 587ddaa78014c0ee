// capi.cpp -- the C ABI of libvcbct (declared in include/vcbct.h): projector
// and FDK objects, the reference-named entry points, and host-side input
// preparation.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <sys/stat.h>

#include "internal.h"

namespace vcbct {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg)
{
    set_error(msg);
    return code;
}

int cuda_fail(cudaError_t e, const char* what)
{
    return fail(VCBCT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Grow-only device buffer.
struct DevBuf {
    void* p = nullptr;
    size_t n = 0;
    cudaError_t ensure(size_t bytes)
    {
        if (bytes <= n) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e == cudaSuccess) n = bytes;
        return e;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

static const double kPi = 3.141592653589793238462643383279;

}  // namespace vcbct

using namespace vcbct;

// ===================================================================== MBFPA

// Host-bound projections are computed in this many view chunks, each
// downloaded while the next is computed.
constexpr int kForwardChunks = 8;
// view chunks of the last row band of a host-to-host projection
constexpr int kTailChunks = 4;
static_assert(kTailChunks <= kForwardChunks, "the tail chunks use the chunk events");

struct vcbct_projector {
    vcbct_proj_geometry g;
    ProjParams pp;
    DevBuf views;      // ViewGeom[V]
    DevBuf vol_f32;    // packed, f32 form (uint16 volumes converted exactly)
    DevBuf stage;      // staging for host inputs / outputs
    DevBuf spec_mu;    // float4 [NE][2]
    DevBuf spec_pdf;   // float [NE]
    DevBuf grad_pk;    // packed float gradient accumulator
    DevBuf counter;    // unsigned long long + int err flag
    int NE = 0;
    int have_u16 = 0, have_f32 = 0;
    int cols_per_block = 4;
    int noise_kind = 0;
    double noise_i0 = 0.0, noise_max = 0.0;
    unsigned long long noise_seed = 0;
    // streaming deck loader: pinned slab buffers and their copy events
    uint16_t* pin = nullptr;
    size_t pin_bytes = 0;
    cudaEvent_t slab_copied[2] = {};
    // download of host-bound projections, overlapped with the later views
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t chunk_done[kForwardChunks] = {};
    cudaEvent_t copies_done = nullptr;
    // host-to-host projection (vcbct_projector_project): upload stream, an
    // event per uploaded slab and per projected row band, and the slices each
    // row band reads (computed once per view set)
    cudaStream_t up_stream = nullptr;
    cudaStream_t band_stream = nullptr;  // every other row band, so one band's tail overlaps the next
    cudaStream_t pack_stream = nullptr;  // re-layout of uploaded slabs, at the highest priority
    std::vector<cudaEvent_t> slab_copied_ev;
    cudaEvent_t up_start = nullptr, up_done = nullptr, bands_done = nullptr;
    std::vector<cudaEvent_t> slab_ready, band_done;
    std::vector<int> band_span;  // [2 * bands]: first and last slice (Z, -1: reads none)
    int band_V = -1;
    DevBuf band_dev;
};

extern "C" const char* vcbct_last_error(void) { return g_last_error.c_str(); }
extern "C" const char* vcbct_version(void) { return "vcbct-b200 0.1 (sm_100a)"; }

static int check_geom(const vcbct_proj_geometry* g)
{
    if (!g) return fail(VCBCT_ERR_ARG, "geometry is NULL");
    if (g->recon_size <= 0 || g->recon_slices <= 0 || g->proj_width <= 0 || g->proj_height <= 0 ||
        g->n_views <= 0)
        return fail(VCBCT_ERR_ARG, "geometry sizes must be positive");
    if (g->num_material <= 0 || g->num_material > VCBCT_MAX_MATERIALS)
        return fail(VCBCT_ERR_LIMIT, "num_material must be in [1, 8]");
    if (!(g->recon_scale > 0) || !(g->recon_step > 0) || !(g->sad_cm > 0) ||
        !(g->det_pitch_cm > 0) || !(g->det_pitch_iso_cm > 0) || !(g->det_pixel_num > 0))
        return fail(VCBCT_ERR_ARG, "geometry pitches and distances must be positive");
    if ((double)g->recon_size * g->recon_size * g->recon_slices > 2.0e9)
        return fail(VCBCT_ERR_LIMIT, "volume exceeds 2e9 voxels");
    if ((double)g->proj_width * g->proj_height * g->n_views > 2.0e9)
        return fail(VCBCT_ERR_LIMIT, "projection stack exceeds 2e9 pixels");
    return VCBCT_OK;
}

extern "C" int vcbct_projector_create(const vcbct_proj_geometry* g, const double* cos_table,
                                      const double* sin_table, const double* xcs,
                                      const double* ycs, vcbct_projector** out)
{
    if (!out) return fail(VCBCT_ERR_ARG, "out is NULL");
    *out = nullptr;
    int rc = check_geom(g);
    if (rc) return rc;
    if (!cos_table || !sin_table || !xcs || !ycs) return fail(VCBCT_ERR_ARG, "view tables are NULL");
    auto* p = new vcbct_projector();
    p->g = *g;
    p->pp = ProjParams{g->recon_size, g->recon_slices, g->proj_width, g->proj_height, g->n_views,
                       g->num_material, g->recon_scale, g->recon_step, g->det_pitch_cm,
                       g->det_pitch_iso_cm, g->sad_cm, g->det_pixel_num, g->x_reg, g->y_reg,
                       g->z_reg};
    std::vector<ViewGeom> vg(g->n_views);
    for (int i = 0; i < g->n_views; i++) vg[i] = ViewGeom{cos_table[i], sin_table[i], xcs[i], ycs[i]};
    cudaError_t e = p->views.ensure(sizeof(ViewGeom) * vg.size());
    if (e == cudaSuccess) e = cudaMemcpy(p->views.p, vg.data(), sizeof(ViewGeom) * vg.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = p->counter.ensure(64);
    if (e == cudaSuccess) e = cudaMemset(p->counter.p, 0, 64);
    if (e != cudaSuccess) {
        vcbct_projector_destroy(p);  // frees what was allocated
        return cuda_fail(e, "vcbct_projector_create");
    }
    if (const char* c = std::getenv("VCBCT_COLS_PER_BLOCK")) {
        int v = std::atoi(c);
        if (v == 1 || v == 2 || v == 4 || v == 8) p->cols_per_block = v;
    }
    *out = p;
    return VCBCT_OK;
}

extern "C" int vcbct_projector_destroy(vcbct_projector* p)
{
    if (!p) return VCBCT_OK;
    if (p->up_stream) cudaStreamSynchronize(p->up_stream);
    if (p->band_stream) cudaStreamSynchronize(p->band_stream);
    if (p->pack_stream) cudaStreamSynchronize(p->pack_stream);
    p->views.release();
    p->vol_f32.release();
    p->stage.release();
    p->spec_mu.release();
    p->spec_pdf.release();
    p->grad_pk.release();
    p->counter.release();
    if (p->pin) cudaFreeHost(p->pin);
    for (cudaEvent_t e : p->slab_copied)
        if (e) cudaEventDestroy(e);
    if (p->copy_stream) cudaStreamDestroy(p->copy_stream);
    for (cudaEvent_t e : p->chunk_done)
        if (e) cudaEventDestroy(e);
    if (p->copies_done) cudaEventDestroy(p->copies_done);
    if (p->up_stream) cudaStreamDestroy(p->up_stream);
    if (p->band_stream) cudaStreamDestroy(p->band_stream);
    if (p->pack_stream) cudaStreamDestroy(p->pack_stream);
    for (cudaEvent_t e : p->slab_copied_ev) cudaEventDestroy(e);
    for (cudaEvent_t e : {p->up_start, p->up_done, p->bands_done})
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : p->slab_ready) cudaEventDestroy(e);
    for (cudaEvent_t e : p->band_done) cudaEventDestroy(e);
    p->band_dev.release();
    delete p;
    return VCBCT_OK;
}

extern "C" int vcbct_projector_set_spectrum(vcbct_projector* p, const float* mu, const float* pdf,
                                            int NE, double xfactor)
{
    if (!p || !mu || !pdf) return fail(VCBCT_ERR_ARG, "NULL argument");
    if (NE <= 0 || NE > VCBCT_MAX_BINS) return fail(VCBCT_ERR_LIMIT, "n_bins must be in [1, 1024]");
    if (!(xfactor != 0.0) || !std::isfinite(xfactor)) return fail(VCBCT_ERR_ARG, "xfactor must be finite and non-zero");
    std::vector<float> tab((size_t)NE * 8, 0.0f);
    for (int e = 0; e < NE; e++)
        for (int k = 0; k < p->g.num_material; k++)
            tab[(size_t)e * 8 + k] = (float)((double)mu[(size_t)k * NE + e] / xfactor);
    VCBCT_CUDA_TRY(p->spec_mu.ensure(tab.size() * sizeof(float)));
    VCBCT_CUDA_TRY(p->spec_pdf.ensure((size_t)NE * sizeof(float)));
    VCBCT_CUDA_TRY(cudaMemcpy(p->spec_mu.p, tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice));
    VCBCT_CUDA_TRY(cudaMemcpy(p->spec_pdf.p, pdf, (size_t)NE * sizeof(float), cudaMemcpyHostToDevice));
    p->NE = NE;
    return VCBCT_OK;
}

static size_t vol_elems(const vcbct_proj_geometry& g)
{
    return (size_t)g.recon_slices * g.num_material * g.recon_size * g.recon_size;
}

extern "C" int vcbct_projector_load_volume(vcbct_projector* p, const uint16_t* vol, int on_device,
                                           void* stream)
{
    if (!p || !vol) return fail(VCBCT_ERR_ARG, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    const auto& g = p->g;
    const uint16_t* src = vol;
    if (!on_device) {
        VCBCT_CUDA_TRY(p->stage.ensure(vol_elems(g) * sizeof(uint16_t)));
        VCBCT_CUDA_TRY(cudaMemcpyAsync(p->stage.p, vol, vol_elems(g) * sizeof(uint16_t), cudaMemcpyHostToDevice, st));
        src = p->stage.as<uint16_t>();
    }
    VCBCT_CUDA_TRY(p->vol_f32.ensure(packed_f32_bytes(g.recon_size, g.recon_slices)));
    VCBCT_CUDA_TRY(launch_pack_u16_f32_slab(src, g.recon_size, g.recon_slices, 0, g.recon_slices, g.num_material,
                                            p->vol_f32.as<float4>(), st));
    p->have_u16 = 1;
    p->have_f32 = 0;
    return VCBCT_OK;
}

extern "C" int vcbct_projector_load_volume_f32(vcbct_projector* p, const float* vol, int on_device,
                                               void* stream)
{
    if (!p || !vol) return fail(VCBCT_ERR_ARG, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    const auto& g = p->g;
    const float* src = vol;
    if (!on_device) {
        VCBCT_CUDA_TRY(p->stage.ensure(vol_elems(g) * sizeof(float)));
        VCBCT_CUDA_TRY(cudaMemcpyAsync(p->stage.p, vol, vol_elems(g) * sizeof(float), cudaMemcpyHostToDevice, st));
        src = p->stage.as<float>();
    }
    VCBCT_CUDA_TRY(p->vol_f32.ensure(packed_f32_bytes(g.recon_size, g.recon_slices)));
    VCBCT_CUDA_TRY(launch_pack_f32(src, g.recon_size, g.recon_slices, g.num_material, p->vol_f32.as<float4>(), st));
    p->have_f32 = 1;
    p->have_u16 = 0;
    return VCBCT_OK;
}

// Slice files of a projector deck streamed into the packed volume: slabs of
// kDeckSlab slices are read into one of two pinned buffers while the other is
// copied to the device and re-laid out there, so disk reads, the copy and the
// re-layout overlap.  Missing or short files keep the previous slice's values
// (zeros for the first), as the reference's reused read buffer does
// (projectionData.cpp:187-215).
constexpr int kDeckSlab = 8;

extern "C" int vcbct_projector_load_deck(vcbct_projector* p, const vcbct_proj_deck* d, int* n_incomplete,
                                         void* stream)
{
    if (!p || !d) return fail(VCBCT_ERR_ARG, "NULL argument");
    const auto& g = p->g;
    if (d->recon_size != g.recon_size || d->used_slices != g.recon_slices || d->mat_num != g.num_material)
        return fail(VCBCT_ERR_ARG, "deck volume (N, used slices, mat_num) differs from the projector's geometry");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t slice = (size_t)g.recon_size * g.recon_size * g.num_material;
    const size_t slab = (size_t)kDeckSlab * slice;
    if (p->pin_bytes < 2 * slab * sizeof(uint16_t)) {
        if (p->pin) cudaFreeHost(p->pin);
        p->pin = nullptr;
        p->pin_bytes = 0;
        VCBCT_CUDA_TRY(cudaHostAlloc((void**)&p->pin, 2 * slab * sizeof(uint16_t), cudaHostAllocDefault));
        p->pin_bytes = 2 * slab * sizeof(uint16_t);
    }
    for (cudaEvent_t& e : p->slab_copied)
        if (!e) VCBCT_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    VCBCT_CUDA_TRY(p->stage.ensure(2 * slab * sizeof(uint16_t)));
    VCBCT_CUDA_TRY(p->vol_f32.ensure(packed_f32_bytes(g.recon_size, g.recon_slices)));
    std::vector<uint16_t> zeros(slice, 0);
    const uint16_t* prev = zeros.data();
    int bad = 0;
    char name[600];
    const int Z = g.recon_slices;
    for (int z0 = 0, b = 0; z0 < Z; z0 += kDeckSlab, b++) {
        const int k = b & 1, nz = std::min(kDeckSlab, Z - z0);
        uint16_t* host = p->pin + (size_t)k * slab;
        if (b >= 2) VCBCT_CUDA_TRY(cudaEventSynchronize(p->slab_copied[k]));  // buffer k copied out
        for (int t = 0; t < nz; t++) {
            uint16_t* dst = host + (size_t)t * slice;
            std::snprintf(name, sizeof name, "%s_%03d.raw", d->mat_prefix, d->slice_first + z0 + t);
            size_t got = 0;
            FILE* fp = std::fopen(name, "rb");
            if (fp) {
                got = std::fread(dst, 1, slice * sizeof(uint16_t), fp) / sizeof(uint16_t);
                std::fclose(fp);
            }
            if (got < slice) {
                std::fprintf(stderr, fp ? "WARNING: pixel data size unmatch (%s)\n" : "data file: %s not found\n", name);
                std::memcpy(dst + got, prev + got, (slice - got) * sizeof(uint16_t));
                bad++;
            }
            prev = dst;
        }
        uint16_t* dev = p->stage.as<uint16_t>() + (size_t)k * slab;
        VCBCT_CUDA_TRY(cudaMemcpyAsync(dev, host, (size_t)nz * slice * sizeof(uint16_t), cudaMemcpyHostToDevice, st));
        VCBCT_CUDA_TRY(cudaEventRecord(p->slab_copied[k], st));
        VCBCT_CUDA_TRY(
            launch_pack_u16_f32_slab(dev, g.recon_size, nz, z0, Z, g.num_material, p->vol_f32.as<float4>(), st));
    }
    VCBCT_CUDA_TRY(cudaStreamSynchronize(st));
    p->have_u16 = 1;
    p->have_f32 = 0;
    if (n_incomplete) *n_incomplete = bad;
    return VCBCT_OK;
}

static int make_fwd_args(vcbct_projector* p, ForwardArgs& a)
{
    if (!p->have_u16 && !p->have_f32) return fail(VCBCT_ERR_STATE, "no volume loaded");
    if (p->NE <= 0) return fail(VCBCT_ERR_STATE, "no spectrum set");
    a = ForwardArgs{};
    a.p = p->pp;
    a.views = p->views.as<ViewGeom>();
    a.spec = SpectrumDev{p->spec_mu.as<float4>(), p->spec_pdf.as<float>(), p->NE};
    a.vol_u16 = nullptr;
    a.vol_f32 = p->vol_f32.as<float4>();
    a.err_flag = reinterpret_cast<int*>(p->counter.as<char>() + 8);
    a.cols_per_block = p->cols_per_block;
    a.noise_kind = p->noise_kind;
    a.noise_i0 = p->noise_i0;
    a.noise_max = p->noise_max;
    a.noise_seed = p->noise_seed;
    a.view_offset = 0;
    return VCBCT_OK;
}

extern "C" int vcbct_projector_set_noise(vcbct_projector* p, int kind, double i0, double max_counts,
                                         unsigned long long seed)
{
    if (!p) return fail(VCBCT_ERR_ARG, "NULL projector");
    if (kind < 0 || kind > 2)
        return fail(VCBCT_ERR_ARG, "noise kind must be 0 (none), 1 (Gaussian counts) or 2 (Poisson counts)");
    if (kind != 0 && (!(i0 > 0.0) || !(max_counts > 0.0)))
        return fail(VCBCT_ERR_ARG, "i0 and max_counts must be positive");
    p->noise_kind = kind;
    p->noise_i0 = i0;
    p->noise_max = max_counts;
    p->noise_seed = seed;
    return VCBCT_OK;
}

extern "C" int vcbct_gaussian_noise(float* proj, size_t n, double max_pixvalue, unsigned long long seed,
                                    int on_device, void* stream)
{
    if (!proj) return fail(VCBCT_ERR_ARG, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    if (on_device) {
        VCBCT_CUDA_TRY(launch_gaussian_noise(proj, n, max_pixvalue, seed, st));
        return VCBCT_OK;
    }
    float* d = nullptr;
    VCBCT_CUDA_TRY(cudaMalloc(&d, std::max<size_t>(n, 1) * sizeof(float)));
    cudaError_t e = cudaMemcpyAsync(d, proj, n * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = launch_gaussian_noise(d, n, max_pixvalue, seed, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(proj, d, n * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(e, "gaussian noise");
    return VCBCT_OK;
}

extern "C" int vcbct_projector_forward(vcbct_projector* p, float* out, int out_on_device, void* stream)
{
    if (!p || !out) return fail(VCBCT_ERR_ARG, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    ForwardArgs a;
    int rc = make_fwd_args(p, a);
    if (rc) return rc;
    const size_t nout = (size_t)p->g.n_views * p->g.proj_height * p->g.proj_width;
    if (out_on_device) {
        a.out = out;
        VCBCT_CUDA_TRY(launch_forward(a, st));
        return VCBCT_OK;
    }
    // Host output: project in view chunks on `st` and download each chunk on
    // a second stream while the next one is projected.
    VCBCT_CUDA_TRY(p->grad_pk.ensure(nout * sizeof(float)));
    float* dout = p->grad_pk.as<float>();
    if (!p->copy_stream) {
        VCBCT_CUDA_TRY(cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking));
        for (cudaEvent_t& e : p->chunk_done) VCBCT_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        VCBCT_CUDA_TRY(cudaEventCreateWithFlags(&p->copies_done, cudaEventDisableTiming));
    }
    const int V = p->g.n_views;
    const size_t per_view = (size_t)p->g.proj_height * p->g.proj_width;
    const int nch = std::min(kForwardChunks, V);
    const ViewGeom* views = a.views;
    for (int c = 0; c < nch; c++) {
        const int v0 = (int)((long long)V * c / nch), v1 = (int)((long long)V * (c + 1) / nch);
        ForwardArgs ac = a;
        ac.views = views + v0;
        ac.view_offset = v0;
        ac.p.V = v1 - v0;
        ac.out = dout + (size_t)v0 * per_view;
        VCBCT_CUDA_TRY(launch_forward(ac, st));
        VCBCT_CUDA_TRY(cudaEventRecord(p->chunk_done[c], st));
        VCBCT_CUDA_TRY(cudaStreamWaitEvent(p->copy_stream, p->chunk_done[c], 0));
        VCBCT_CUDA_TRY(cudaMemcpyAsync(out + (size_t)v0 * per_view, dout + (size_t)v0 * per_view,
                                       (size_t)(v1 - v0) * per_view * sizeof(float), cudaMemcpyDeviceToHost,
                                       p->copy_stream));
    }
    VCBCT_CUDA_TRY(cudaEventRecord(p->copies_done, p->copy_stream));
    VCBCT_CUDA_TRY(cudaStreamWaitEvent(st, p->copies_done, 0));
    VCBCT_CUDA_TRY(cudaStreamSynchronize(st));
    return VCBCT_OK;
}

// Slices each detector row band of 32 rows reads, over all views (once per
// view set; a small launch and a synchronisation of `st`).
static int band_footprints(vcbct_projector* p, cudaStream_t st)
{
    const int nb = (p->pp.H + 31) / 32;
    if (p->band_V == p->pp.V && (int)p->band_span.size() == 2 * nb) return VCBCT_OK;
    std::vector<int> span(2 * (size_t)nb);
    for (int b = 0; b < nb; b++) {
        span[2 * b] = p->pp.Z;
        span[2 * b + 1] = -1;
    }
    VCBCT_CUDA_TRY(p->band_dev.ensure(span.size() * sizeof(int)));
    VCBCT_CUDA_TRY(cudaMemcpyAsync(p->band_dev.p, span.data(), span.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    VCBCT_CUDA_TRY(launch_band_footprint(p->pp, p->views.as<ViewGeom>(), p->band_dev.as<int>(), st));
    VCBCT_CUDA_TRY(cudaMemcpyAsync(span.data(), p->band_dev.p, span.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
    VCBCT_CUDA_TRY(cudaStreamSynchronize(st));
    p->band_span = span;
    p->band_V = p->pp.V;
    return VCBCT_OK;
}

static int grow_events(std::vector<cudaEvent_t>& ev, size_t n)
{
    while (ev.size() < n) {
        cudaEvent_t e;
        VCBCT_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ev.push_back(e);
    }
    return VCBCT_OK;
}

// Host volume in, host projections out (the whole of reprojectionOnGPU's
// work), with the volume's upload overlapped with the projection: the volume
// goes up in slabs of kDeckSlab slices on one stream, each slab re-laid out
// as it lands on another of the highest priority (so that its blocks take the
// first free slots among the projection's, and the copies never wait for
// them); the detector is projected in row bands of 32 rows (all
// views per launch), each band launched as soon as the slabs it reads are in
// (its slice footprint is computed once per view set; bands alternate between
// two streams so that one band's last blocks overlap the next band's first),
// and each band's rows are downloaded on another stream while later bands are
// projected.  Bands
// are taken greedily, the one that needs the fewest slabs not yet requested
// first, and slabs are uploaded in the order the bands request them.  The
// result is bitwise that of vcbct_projector_load_volume + _forward.
static int project_host(vcbct_projector* p, const uint16_t* vol, float* out, cudaStream_t st)
{
    const auto& g = p->g;
    if (p->NE <= 0) return fail(VCBCT_ERR_STATE, "no spectrum set");
    ForwardArgs a;
    p->have_u16 = 1;  // the volume is (re)written below
    p->have_f32 = 0;
    int rc = make_fwd_args(p, a);
    if (rc) return rc;
    if (!p->copy_stream) {
        VCBCT_CUDA_TRY(cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking));
        for (cudaEvent_t& e : p->chunk_done) VCBCT_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        VCBCT_CUDA_TRY(cudaEventCreateWithFlags(&p->copies_done, cudaEventDisableTiming));
    }
    if (!p->up_stream) {
        VCBCT_CUDA_TRY(cudaStreamCreateWithFlags(&p->up_stream, cudaStreamNonBlocking));
        VCBCT_CUDA_TRY(cudaEventCreateWithFlags(&p->up_start, cudaEventDisableTiming));
        VCBCT_CUDA_TRY(cudaEventCreateWithFlags(&p->up_done, cudaEventDisableTiming));
        VCBCT_CUDA_TRY(cudaStreamCreateWithFlags(&p->band_stream, cudaStreamNonBlocking));
        VCBCT_CUDA_TRY(cudaEventCreateWithFlags(&p->bands_done, cudaEventDisableTiming));
        int least = 0, greatest = 0;
        VCBCT_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        VCBCT_CUDA_TRY(cudaStreamCreateWithPriority(&p->pack_stream, cudaStreamNonBlocking, greatest));
    }
    rc = band_footprints(p, st);
    if (rc) return rc;
    const int Z = g.recon_slices, H = g.proj_height, W = g.proj_width, V = g.n_views;
    const int nb = (H + 31) / 32, nslab = (Z + kDeckSlab - 1) / kDeckSlab;
    const size_t slice = (size_t)g.recon_size * g.recon_size * g.num_material;
    const size_t nout = (size_t)V * H * W;
    VCBCT_CUDA_TRY(p->stage.ensure(vol_elems(g) * sizeof(uint16_t)));
    VCBCT_CUDA_TRY(p->vol_f32.ensure(packed_f32_bytes(g.recon_size, Z)));
    VCBCT_CUDA_TRY(p->grad_pk.ensure(nout * sizeof(float)));
    rc = grow_events(p->slab_ready, nslab);
    if (!rc) rc = grow_events(p->slab_copied_ev, nslab);
    if (!rc) rc = grow_events(p->band_done, nb);
    if (rc) return rc;
    a.vol_f32 = p->vol_f32.as<float4>();
    uint16_t* stage = p->stage.as<uint16_t>();
    float* dout = p->grad_pk.as<float>();
    // downloads per band overlap only into page-locked memory (a copy into
    // pageable memory holds the calling thread); otherwise they follow the
    // last band
    cudaPointerAttributes at{};
    const bool out_locked = cudaPointerGetAttributes(&at, out) == cudaSuccess && at.type == cudaMemoryTypeHost;
    cudaGetLastError();
    // the upload overwrites buffers earlier work on `st` may still read
    VCBCT_CUDA_TRY(cudaEventRecord(p->up_start, st));
    VCBCT_CUDA_TRY(cudaStreamWaitEvent(p->up_stream, p->up_start, 0));
    VCBCT_CUDA_TRY(cudaStreamWaitEvent(p->copy_stream, p->up_start, 0));
    VCBCT_CUDA_TRY(cudaStreamWaitEvent(p->band_stream, p->up_start, 0));
    const cudaStream_t cs[2] = {st, p->band_stream};

    std::vector<int> pos(nslab, -1);  // upload position of each slab
    int issued = 0;
    auto upload = [&](int s) -> int {
        const int z0 = s * kDeckSlab, nz = std::min(kDeckSlab, Z - z0);
        uint16_t* dev = stage + (size_t)z0 * slice;
        VCBCT_CUDA_TRY(cudaMemcpyAsync(dev, vol + (size_t)z0 * slice, (size_t)nz * slice * sizeof(uint16_t),
                                       cudaMemcpyHostToDevice, p->up_stream));
        VCBCT_CUDA_TRY(cudaEventRecord(p->slab_copied_ev[issued], p->up_stream));
        VCBCT_CUDA_TRY(cudaStreamWaitEvent(p->pack_stream, p->slab_copied_ev[issued], 0));
        VCBCT_CUDA_TRY(launch_pack_u16_f32_slab(dev, g.recon_size, nz, z0, Z, g.num_material,
                                                p->vol_f32.as<float4>(), p->pack_stream));
        VCBCT_CUDA_TRY(cudaEventRecord(p->slab_ready[issued], p->pack_stream));
        pos[s] = issued++;
        return VCBCT_OK;
    };
    // band b's rows of views [v0, v1), once `done` has been reached
    auto download_views = [&](int b, int v0, int v1, cudaEvent_t done) -> int {
        const int j1 = std::min(H, 32 * b + 32), r0 = H - j1, nr = j1 - 32 * b;  // rows H-1-j
        const size_t pitch = (size_t)H * W * sizeof(float);
        const size_t o = (size_t)v0 * H * W + (size_t)r0 * W;
        VCBCT_CUDA_TRY(cudaStreamWaitEvent(p->copy_stream, done, 0));
        VCBCT_CUDA_TRY(cudaMemcpy2DAsync(out + o, pitch, dout + o, pitch, (size_t)nr * W * sizeof(float), v1 - v0,
                                         cudaMemcpyDeviceToHost, p->copy_stream));
        return VCBCT_OK;
    };
    auto download = [&](int b) -> int { return download_views(b, 0, V, p->band_done[b]); };
    std::vector<char> done(nb, 0);
    std::vector<int> order;
    for (int step = 0; step < nb; step++) {
        int best = -1, best_new = INT_MAX;
        for (int b = 0; b < nb; b++) {
            if (done[b]) continue;
            int need = 0;
            if (p->band_span[2 * b + 1] >= 0)
                for (int s = p->band_span[2 * b] / kDeckSlab; s <= p->band_span[2 * b + 1] / kDeckSlab; s++)
                    need += pos[s] < 0;
            if (need < best_new) {
                best = b;
                best_new = need;
            }
        }
        done[best] = 1;
        int wait = -1;
        if (p->band_span[2 * best + 1] >= 0) {
            for (int s = p->band_span[2 * best] / kDeckSlab; s <= p->band_span[2 * best + 1] / kDeckSlab; s++) {
                if (pos[s] < 0) {
                    rc = upload(s);
                    if (rc) return rc;
                }
                wait = std::max(wait, pos[s]);
            }
        }
        order.push_back(best);
        // The last band goes in view chunks on alternating streams, each
        // downloaded as soon as it is done: only the last chunk's rows are
        // left to copy after the last launch.
        const int nch = (step == nb - 1 && out_locked) ? std::min(kTailChunks, V) : 1;
        for (int c = 0; c < nch; c++) {
            const cudaStream_t bs = cs[(step + c) & 1];
            if (wait >= 0) VCBCT_CUDA_TRY(cudaStreamWaitEvent(bs, p->slab_ready[wait], 0));
            const int v0 = (int)((long long)V * c / nch), v1 = (int)((long long)V * (c + 1) / nch);
            ForwardArgs ab = a;
            ab.views = a.views + v0;
            ab.view_offset = v0;
            ab.p.V = v1 - v0;
            ab.out = dout + (size_t)v0 * H * W;
            ab.band0 = best;
            ab.nbands = 1;
            VCBCT_CUDA_TRY(launch_forward(ab, bs));
            cudaEvent_t done = nch == 1 ? p->band_done[best] : p->chunk_done[c];
            VCBCT_CUDA_TRY(cudaEventRecord(done, bs));
            if (out_locked) {
                rc = download_views(best, v0, v1, done);
                if (rc) return rc;
            }
        }
    }
    for (int s = 0; s < nslab; s++)  // slices no band reads still form the loaded volume
        if (pos[s] < 0) {
            rc = upload(s);
            if (rc) return rc;
        }
    if (!out_locked)
        for (int b : order) {
            rc = download(b);
            if (rc) return rc;
        }
    VCBCT_CUDA_TRY(cudaEventRecord(p->up_done, p->pack_stream));  // after every copy and re-layout
    VCBCT_CUDA_TRY(cudaEventRecord(p->bands_done, p->band_stream));
    VCBCT_CUDA_TRY(cudaEventRecord(p->copies_done, p->copy_stream));
    VCBCT_CUDA_TRY(cudaStreamWaitEvent(st, p->up_done, 0));
    VCBCT_CUDA_TRY(cudaStreamWaitEvent(st, p->bands_done, 0));
    VCBCT_CUDA_TRY(cudaStreamWaitEvent(st, p->copies_done, 0));
    VCBCT_CUDA_TRY(cudaStreamSynchronize(st));
    return VCBCT_OK;
}

extern "C" int vcbct_projector_project(vcbct_projector* p, const uint16_t* vol, float* out, void* stream)
{
    if (!p || !vol || !out) return fail(VCBCT_ERR_ARG, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    const int rc = project_host(p, vol, out, st);
    if (rc) {  // nothing may still read `vol` or write `out` after a failed call
        cudaStreamSynchronize(st);
        if (p->up_stream) cudaStreamSynchronize(p->up_stream);
        if (p->pack_stream) cudaStreamSynchronize(p->pack_stream);
        if (p->band_stream) cudaStreamSynchronize(p->band_stream);
        if (p->copy_stream) cudaStreamSynchronize(p->copy_stream);
        p->have_u16 = 0;
    }
    return rc;
}

extern "C" int vcbct_projector_path_integrals(vcbct_projector* p, float* d_L, void* stream)
{
    if (!p || !d_L) return fail(VCBCT_ERR_ARG, "NULL argument");
    ForwardArgs a;
    int rc = make_fwd_args(p, a);
    if (rc) return rc;
    a.L_out = d_L;
    VCBCT_CUDA_TRY(launch_forward(a, (cudaStream_t)stream));
    return VCBCT_OK;
}

extern "C" int vcbct_projector_count_segments(vcbct_projector* p, unsigned long long* total, void* stream)
{
    if (!p || !total) return fail(VCBCT_ERR_ARG, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    ForwardArgs a;
    int rc = make_fwd_args(p, a);
    if (rc) return rc;
    unsigned long long* cnt = p->counter.as<unsigned long long>();
    VCBCT_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), st));
    a.seg_count = cnt;
    VCBCT_CUDA_TRY(launch_forward(a, st));
    VCBCT_CUDA_TRY(cudaMemcpyAsync(total, cnt, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    VCBCT_CUDA_TRY(cudaStreamSynchronize(st));
    return VCBCT_OK;
}

static int projector_adjoint(vcbct_projector* p, const float* d_L, const float* d_grad_out, float* d_grad,
                             void* stream);

extern "C" int vcbct_projector_adjoint(vcbct_projector* p, const float* d_grad_out, float* d_grad,
                                       void* stream)
{
    return projector_adjoint(p, nullptr, d_grad_out, d_grad, stream);
}

extern "C" int vcbct_projector_forward_state(vcbct_projector* p, float* d_out, float* d_L, void* stream)
{
    if (!p || !d_out || !d_L) return fail(VCBCT_ERR_ARG, "NULL argument");
    ForwardArgs a;
    int rc = make_fwd_args(p, a);
    if (rc) return rc;
    a.out = d_out;
    a.L_out = d_L;
    VCBCT_CUDA_TRY(launch_forward(a, (cudaStream_t)stream));
    return VCBCT_OK;
}

extern "C" int vcbct_projector_adjoint_state(vcbct_projector* p, const float* d_L, const float* d_grad_out,
                                             float* d_grad, void* stream)
{
    if (!d_L) return fail(VCBCT_ERR_ARG, "NULL argument");
    return projector_adjoint(p, d_L, d_grad_out, d_grad, stream);
}

static int projector_adjoint(vcbct_projector* p, const float* d_L, const float* d_grad_out, float* d_grad,
                             void* stream)
{
    if (!p || !d_grad_out || !d_grad) return fail(VCBCT_ERR_ARG, "NULL argument");
    if (!p->have_u16 && !p->have_f32) return fail(VCBCT_ERR_STATE, "no volume loaded");
    if (p->NE <= 0) return fail(VCBCT_ERR_STATE, "no spectrum set");
    cudaStream_t st = (cudaStream_t)stream;
    const auto& g = p->g;
    // gradient planes (ceil(nmat / 2) x 2 floats per voxel: element quads, then a
    // pair for a last group of one or two elements)
    const size_t pk = (size_t)((g.num_material + 1) / 2) * 2 * g.recon_size * g.recon_size * g.recon_slices *
                      sizeof(float);
    VCBCT_CUDA_TRY(p->grad_pk.ensure(pk));
    VCBCT_CUDA_TRY(cudaMemsetAsync(p->grad_pk.p, 0, pk, st));
    AdjointArgs a{};
    a.p = p->pp;
    a.views = p->views.as<ViewGeom>();
    a.spec = SpectrumDev{p->spec_mu.as<float4>(), p->spec_pdf.as<float>(), p->NE};
    a.vol_f32 = p->vol_f32.as<float4>();
    a.grad_out = d_grad_out;
    a.L_in = d_L;
    a.grad_planes = p->grad_pk.as<float>();
    a.err_flag = reinterpret_cast<int*>(p->counter.as<char>() + 8);
    a.cols_per_block = p->cols_per_block;
    // Volumes whose gradient planes far exceed L2 are scattered in strips of
    // volume rows, one launch each (every launch marches only the part of
    // each ray that crosses its strip), so that more of the reductions of the
    // blocks resident at one time hit L2.  Only with kept path integrals:
    // re-marching them would repeat per strip.
    // (measured on B200: 2 strips -18 % at 0.8 GB of planes, 3 strips -20 %
    // at 2.5 GB; more strips repeat the rays' set-up for no further gain)
    int ns = !d_L ? 1 : (pk > ((size_t)2 << 30) ? 3 : (pk > ((size_t)512 << 20) ? 2 : 1));
    if (const char* e = std::getenv("VCBCT_ADJ_STRIPS")) ns = std::max(1, std::min(64, std::atoi(e)));
    ns = std::min(ns, g.recon_size);
    for (int s = 0; s < ns; s++) {
        a.y0 = ns > 1 ? (int)((long long)g.recon_size * s / ns) : 0;
        a.y1 = ns > 1 ? (int)((long long)g.recon_size * (s + 1) / ns) : 0;
        VCBCT_CUDA_TRY(launch_adjoint(a, st));
    }
    VCBCT_CUDA_TRY(launch_unpack_grad(p->grad_pk.as<float>(), g.recon_size, g.recon_slices, g.num_material, d_grad, st));
    return VCBCT_OK;
}

// ----------------------------------------------------- iterative recon --

extern "C" int vcbct_projector_lengthproj(vcbct_projector* p, int ite, int start_view, int end_view,
                                          const uint16_t* proj, int proj_on_device, float* npf,
                                          int npf_on_device, void* stream)
{
    if (!p || !proj || !npf) return fail(VCBCT_ERR_ARG, "NULL argument");
    const auto& g = p->g;
    if (start_view < 0 || end_view > g.n_views || start_view > end_view)
        return fail(VCBCT_ERR_ARG, "view range outside [0, n_views]");
    cudaStream_t st = (cudaStream_t)stream;
    LpParams q{g.recon_size, g.recon_slices, g.proj_width, g.proj_height, g.recon_scale, g.recon_step,
               g.det_pitch_cm, g.det_pitch_iso_cm, g.sad_cm, g.det_pixel_num, g.x_reg, g.y_reg, g.z_reg};
    if (ite != 0) q.xr = q.yr = q.zr = 0.0;  // lengthproj.cpp:18-23
    const size_t nproj = (size_t)g.n_views * g.proj_height * g.proj_width;
    const size_t nvox = (size_t)g.recon_size * g.recon_size * g.recon_slices;
    const size_t nscr = lengthproj_scratch_bytes(end_view - start_view);
    // scratch: per-view constants, then (host inputs / outputs) the staged arrays
    const size_t o_proj = (nscr + 255) / 256 * 256;
    const size_t o_npf = o_proj + (proj_on_device ? 0 : (nproj * sizeof(uint16_t) + 255) / 256 * 256);
    const size_t total = o_npf + (npf_on_device ? 0 : nvox * sizeof(float));
    VCBCT_CUDA_TRY(p->stage.ensure(std::max<size_t>(total, 256)));
    char* base = p->stage.as<char>();
    const uint16_t* d_proj = proj;
    float* d_npf = npf;
    if (!proj_on_device) {
        VCBCT_CUDA_TRY(cudaMemcpyAsync(base + o_proj, proj, nproj * sizeof(uint16_t), cudaMemcpyHostToDevice, st));
        d_proj = reinterpret_cast<const uint16_t*>(base + o_proj);
    }
    if (!npf_on_device) d_npf = reinterpret_cast<float*>(base + o_npf);
    VCBCT_CUDA_TRY(launch_lengthproj(q, p->views.as<ViewGeom>(), start_view, end_view, d_proj, d_npf, base, st));
    if (start_view == end_view) VCBCT_CUDA_TRY(cudaMemsetAsync(d_npf, 0, nvox * sizeof(float), st));
    if (!npf_on_device) {
        VCBCT_CUDA_TRY(cudaMemcpyAsync(npf, d_npf, nvox * sizeof(float), cudaMemcpyDeviceToHost, st));
        VCBCT_CUDA_TRY(cudaStreamSynchronize(st));
    }
    return VCBCT_OK;
}

namespace {
struct IrScratch {
    std::mutex mu;
    DevBuf buf;
};
IrScratch& ir_scratch()
{
    static IrScratch s;
    return s;
}
}  // namespace

extern "C" int vcbct_ir_update(int N, int Z, double scale, const short* before, float* out, const float* npf,
                               const float* npf_re, double wbefore, double weight_tv, double weight_prior,
                               int on_device, void* stream)
{
    if (!before || !out || !npf || !npf_re) return fail(VCBCT_ERR_ARG, "NULL argument");
    if (N <= 0 || Z <= 0) return fail(VCBCT_ERR_ARG, "sizes must be positive");
    cudaStream_t st = (cudaStream_t)stream;
    if (on_device) {
        VCBCT_CUDA_TRY(launch_ir_update(N, Z, scale, before, out, npf, npf_re, wbefore, weight_tv, weight_prior, st));
        return VCBCT_OK;
    }
    const size_t n = (size_t)N * N * Z;
    const size_t ob = 0, oo = (n * sizeof(short) + 255) / 256 * 256, on = oo + n * sizeof(float),
                 or_ = on + n * sizeof(float);
    IrScratch& sc = ir_scratch();
    std::lock_guard<std::mutex> lk(sc.mu);
    VCBCT_CUDA_TRY(sc.buf.ensure(or_ + n * sizeof(float)));
    char* b = sc.buf.as<char>();
    VCBCT_CUDA_TRY(cudaMemcpyAsync(b + ob, before, n * sizeof(short), cudaMemcpyHostToDevice, st));
    VCBCT_CUDA_TRY(cudaMemcpyAsync(b + on, npf, n * sizeof(float), cudaMemcpyHostToDevice, st));
    VCBCT_CUDA_TRY(cudaMemcpyAsync(b + or_, npf_re, n * sizeof(float), cudaMemcpyHostToDevice, st));
    VCBCT_CUDA_TRY(launch_ir_update(N, Z, scale, reinterpret_cast<short*>(b + ob), reinterpret_cast<float*>(b + oo),
                                    reinterpret_cast<float*>(b + on), reinterpret_cast<float*>(b + or_), wbefore,
                                    weight_tv, weight_prior, st));
    VCBCT_CUDA_TRY(cudaMemcpyAsync(out, b + oo, n * sizeof(float), cudaMemcpyDeviceToHost, st));
    VCBCT_CUDA_TRY(cudaStreamSynchronize(st));
    return VCBCT_OK;
}

// Reference-named entry points of the iterative reconstruction helpers.
extern "C" void vcbct_lengthproj(int ite, int reconSize, int reconSlices, short* reconImageshort,
                           unsigned short* ProjImageshort, float* npf_float, unsigned short* projVolume,
                           double reconScale, double reconStep, int projImgWidth, int projImgHeight,
                           int startProjNumber, int endProjNumber, double* ProjAngle, double* cosTable,
                           double* sinTable, double* XcenterShift, double* YcenterShift, double xfactor,
                           double* xalpha, double DETECTOR_PITCH_CM, double DETECTOR_PITCH_CM_AT_ISO_CENT,
                           double DIST_BTWN_SRC_AND_ISOCENT_CM, double DETECTOR_PIXEL_NUM, double x_reg,
                           double y_reg, double z_reg)
{
    (void)reconImageshort;
    (void)ProjImageshort;
    (void)ProjAngle;
    (void)xfactor;
    (void)xalpha;
    vcbct_proj_geometry g{reconSize, reconSlices, reconScale, reconStep, projImgWidth, projImgHeight, endProjNumber,
                          DETECTOR_PITCH_CM, DETECTOR_PITCH_CM_AT_ISO_CENT, DIST_BTWN_SRC_AND_ISOCENT_CM,
                          DETECTOR_PIXEL_NUM, x_reg, y_reg, z_reg, 1};
    vcbct_projector* p = nullptr;
    int rc = vcbct_projector_create(&g, cosTable, sinTable, XcenterShift, YcenterShift, &p);
    if (!rc) rc = vcbct_projector_lengthproj(p, ite, startProjNumber, endProjNumber, projVolume, 0, npf_float, 0,
                                             nullptr);
    if (rc) std::fprintf(stderr, "lengthproj: %s\n", vcbct_last_error());
    if (p) vcbct_projector_destroy(p);
}

extern "C" void vcbct_IR_ImageCBCT(const int ite, int reconSize, int reconSlices, double reconScale,
                             short* reconImageshort_before, float* reconImagefloat, float* npf_float,
                             float* npf_float_re, double wbefore, double weight_tv, double weight_prior,
                             const int thinout)
{
    (void)ite;
    (void)thinout;
    int rc = vcbct_ir_update(reconSize, reconSlices, reconScale, reconImageshort_before, reconImagefloat, npf_float,
                             npf_float_re, wbefore, weight_tv, weight_prior, 0, nullptr);
    if (rc) std::fprintf(stderr, "IR_ImageCBCT: %s\n", vcbct_last_error());
}

// ------------------------------------------------------------------ batching --
//
// A batch is a list of (projector, device output) items.  Three launch
// strategies, picked by vcbct_batch_autotune:
//  - persistent: one launch of persistent_batch_kernel per kFlatItems items,
//    a GPU-filling grid whose blocks take every item's tiles from a counter
//    (counter reset + kernel);
//  - per-item: each item's own forward_kernel launch, spread over two
//    branches that fork from and join to the caller's stream, so one item's
//    tail overlaps the next item's start;
//  - flat: one launch of flat_batch_kernel with a block per tile of every
//    item (up to kFlatItems items per launch, their arguments in the
//    launch's parameter block).
// Either launch sequence is captured once into a CUDA graph and replayed.

constexpr int kBatchBranches = 2;
static_assert(sizeof(FlatBatch) <= 32000, "the flat batch parameter block exceeds the kernel parameter limit");

struct vcbct_batch {
    std::vector<vcbct_projector*> proj;
    std::vector<float*> outs;
    DevBuf counter;
    long long total = 0;
    int NEmax = 0, nmat_max = 0;
    int cols_per_block = 4, blocks = 0;
    int strategy = 0;   // 0: persistent launch, 1: per-item launches, 2: single flat launch
    std::vector<FlatBatch> flat;  // strategies 0 and 2: the launches' parameter blocks
    bool dirty = true;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t graph_stream = nullptr;
    cudaStream_t branch[kBatchBranches] = {};
    cudaEvent_t fork = nullptr, join[kBatchBranches] = {};
};

static void batch_drop_graph(vcbct_batch* b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

extern "C" int vcbct_batch_create(vcbct_batch** out)
{
    if (!out) return fail(VCBCT_ERR_ARG, "out is NULL");
    *out = new vcbct_batch();
    return VCBCT_OK;
}

extern "C" int vcbct_batch_destroy(vcbct_batch* b)
{
    if (!b) return VCBCT_OK;
    batch_drop_graph(b);
    b->counter.release();
    for (int k = 0; k < kBatchBranches; k++) {
        if (b->branch[k]) cudaStreamDestroy(b->branch[k]);
        if (b->join[k]) cudaEventDestroy(b->join[k]);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    delete b;
    return VCBCT_OK;
}

extern "C" int vcbct_batch_add(vcbct_batch* b, vcbct_projector* p, float* d_out)
{
    if (!b || !p || !d_out) return fail(VCBCT_ERR_ARG, "NULL argument");
    if (!p->have_u16 && !p->have_f32) return fail(VCBCT_ERR_STATE, "no volume loaded");
    if (p->NE <= 0) return fail(VCBCT_ERR_STATE, "no spectrum set");
    b->proj.push_back(p);
    b->outs.push_back(d_out);
    b->dirty = true;
    return VCBCT_OK;
}

extern "C" int vcbct_batch_configure(vcbct_batch* b, int strategy, int cols_per_block)
{
    if (!b) return fail(VCBCT_ERR_ARG, "NULL batch");
    if ((strategy < 0 || strategy > 2) ||
        !(cols_per_block == 1 || cols_per_block == 2 || cols_per_block == 4 || cols_per_block == 8))
        return fail(VCBCT_ERR_ARG, "strategy must be 0, 1 or 2 and cols_per_block 1, 2, 4 or 8");
    b->strategy = strategy;
    b->cols_per_block = cols_per_block;
    b->dirty = true;
    return VCBCT_OK;
}

static int batch_build(vcbct_batch* b)
{
    if (b->proj.empty()) return fail(VCBCT_ERR_STATE, "empty batch");
    b->NEmax = 0;
    b->nmat_max = 0;
    b->total = 0;
    const int cpb = b->cols_per_block;
    // parameter blocks of the single-launch strategies, kFlatItems items each
    b->flat.clear();
    for (size_t i0 = 0; i0 < b->proj.size(); i0 += kFlatItems) {
        FlatBatch fb{};
        const size_t n = std::min<size_t>(kFlatItems, b->proj.size() - i0);
        fb.nitems = (int)n;
        long long t = 0;
        for (size_t i = 0; i < n; i++) {
            vcbct_projector* p = b->proj[i0 + i];
            ForwardArgs a;
            int rc = make_fwd_args(p, a);
            if (rc) return rc;
            a.out = b->outs[i0 + i];
            a.cols_per_block = cpb;
            fb.fa[i] = a;
            fb.ncolb[i] = (p->g.proj_width + cpb - 1) / cpb;
            fb.begin[i] = t;
            t += (long long)fb.ncolb[i] * p->g.n_views * ((p->g.proj_height + 31) / 32);
            b->NEmax = std::max(b->NEmax, p->NE);
            b->nmat_max = std::max(b->nmat_max, p->g.num_material);
        }
        fb.begin[n] = t;
        b->total += t;
        b->flat.push_back(fb);
    }
    VCBCT_CUDA_TRY(b->counter.ensure(64));
    int dev = 0, sms = 0;
    VCBCT_CUDA_TRY(cudaGetDevice(&dev));
    VCBCT_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int per_sm = batch_blocks_per_sm(b->nmat_max, cpb, b->NEmax);
    b->blocks = std::max(1, per_sm) * sms;
    batch_drop_graph(b);
    b->dirty = false;
    return VCBCT_OK;
}

static int batch_launch(vcbct_batch* b, cudaStream_t st)
{
    if (b->strategy == 2) {
        for (const FlatBatch& fb : b->flat)
            VCBCT_CUDA_TRY(launch_flat_batch(fb, b->NEmax, b->nmat_max, b->cols_per_block, st));
        return VCBCT_OK;
    }
    if (b->strategy == 0) {
        for (const FlatBatch& fb : b->flat)
            VCBCT_CUDA_TRY(launch_persistent_batch(fb, b->NEmax, b->nmat_max, b->cols_per_block, b->blocks,
                                                   b->counter.as<unsigned long long>(), st));
        return VCBCT_OK;
    }
    if (!b->fork) {
        VCBCT_CUDA_TRY(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
        for (int k = 0; k < kBatchBranches; k++) {
            VCBCT_CUDA_TRY(cudaStreamCreateWithFlags(&b->branch[k], cudaStreamNonBlocking));
            VCBCT_CUDA_TRY(cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming));
        }
    }
    VCBCT_CUDA_TRY(cudaEventRecord(b->fork, st));
    for (int k = 0; k < kBatchBranches; k++) VCBCT_CUDA_TRY(cudaStreamWaitEvent(b->branch[k], b->fork, 0));
    for (size_t i = 0; i < b->proj.size(); i++) {
        ForwardArgs a;
        int rc = make_fwd_args(b->proj[i], a);
        if (rc) return rc;
        a.out = b->outs[i];
        a.cols_per_block = b->cols_per_block;
        VCBCT_CUDA_TRY(launch_forward(a, b->branch[i % kBatchBranches]));
    }
    for (int k = 0; k < kBatchBranches; k++) {
        VCBCT_CUDA_TRY(cudaEventRecord(b->join[k], b->branch[k]));
        VCBCT_CUDA_TRY(cudaStreamWaitEvent(st, b->join[k], 0));
    }
    return VCBCT_OK;
}

extern "C" int vcbct_batch_forward(vcbct_batch* b, int use_graph, void* stream)
{
    if (!b) return fail(VCBCT_ERR_ARG, "NULL batch");
    cudaStream_t st = (cudaStream_t)stream;
    if (b->dirty) {
        int rc = batch_build(b);
        if (rc) return rc;
    }
    if (!use_graph) return batch_launch(b, st);
    if (!b->exec || b->graph_stream != st) {
        batch_drop_graph(b);
        cudaStream_t cap = st;
        bool own = false;
        if (cap == nullptr) {  // the legacy stream cannot be captured
            VCBCT_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
            own = true;
        }
        VCBCT_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        int rc = batch_launch(b, cap);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(cap, &g);
        if (own) cudaStreamDestroy(cap);
        if (rc) return rc;
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        b->graph = g;
        VCBCT_CUDA_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
        b->graph_stream = st;
    }
    VCBCT_CUDA_TRY(cudaGraphLaunch(b->exec, st));
    return VCBCT_OK;
}

// ----------------------------------------------------------------- autotuner --
//
// Launch shapes are picked by timing the candidates on the caller's data:
// columns per block (warps per block) for the plain and the batched forward
// projection.  Results are kept per geometry signature in memory and, when
// VCBCT_TUNE_CACHE names a file, in that file ("signature value" lines).

namespace {
std::mutex g_tune_mu;
std::map<std::string, int> g_tune;
bool g_tune_loaded = false;

void tune_load()
{
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char* f = std::getenv("VCBCT_TUNE_CACHE");
    if (!f) return;
    std::ifstream in(f);
    std::string key;
    int v;
    while (in >> key >> v) g_tune[key] = v;
}

void tune_store(const std::string& key, int v)
{
    g_tune[key] = v;
    const char* f = std::getenv("VCBCT_TUNE_CACHE");
    if (!f) return;
    std::ofstream out(f, std::ios::app);
    out << key << " " << v << "\n";
}

std::string device_tag()
{
    int dev = 0;
    cudaDeviceProp prop;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return "dev?";
    std::string n = prop.name;
    for (auto& c : n)
        if (c == ' ') c = '_';
    return n;
}

template <class F>
float time_ms(F f, cudaStream_t st, int reps)
{
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    f();
    cudaEventRecord(a, st);
    for (int i = 0; i < reps; i++) f();
    cudaEventRecord(b, st);
    cudaEventSynchronize(b);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms / reps;
}
}  // namespace

extern "C" int vcbct_projector_autotune(vcbct_projector* p, float* d_out, void* stream, int* chosen)
{
    if (!p || !d_out) return fail(VCBCT_ERR_ARG, "NULL argument");
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_load();
    const auto& g = p->g;
    std::ostringstream key;
    key << "fwd:" << device_tag() << ":" << g.recon_size << "x" << g.recon_slices << ":" << g.proj_width << "x"
        << g.proj_height << "x" << g.n_views << ":" << g.num_material << ":" << p->NE;
    auto it = g_tune.find(key.str());
    if (it == g_tune.end()) {
        cudaStream_t st = (cudaStream_t)stream;
        float best = 1e30f;
        int bestc = p->cols_per_block;
        for (int c : {2, 4, 8}) {
            p->cols_per_block = c;
            float ms = time_ms([&]() { vcbct_projector_forward(p, d_out, 1, stream); }, st, 2);
            if (ms < best) {
                best = ms;
                bestc = c;
            }
        }
        tune_store(key.str(), bestc);
        p->cols_per_block = bestc;
    } else {
        p->cols_per_block = it->second;
    }
    if (chosen) *chosen = p->cols_per_block;
    return VCBCT_OK;
}

extern "C" int vcbct_batch_autotune(vcbct_batch* b, void* stream, int* chosen)
{
    if (!b || b->proj.empty()) return fail(VCBCT_ERR_ARG, "empty batch");
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_load();
    std::ostringstream key;
    key << "batch:" << device_tag() << ":" << b->proj.size();
    for (auto* p : b->proj)
        key << ":" << p->g.recon_size << "x" << p->g.recon_slices << "x" << p->g.n_views << "x" << p->g.proj_width
            << "x" << p->g.proj_height;
    auto it = g_tune.find(key.str());
    int bestc = b->cols_per_block + 100 * b->strategy;
    if (it == g_tune.end()) {
        cudaStream_t st = (cudaStream_t)stream;
        float best = 1e30f;
        for (int mode : {0, 1, 2}) {
            for (int c : {2, 4, 8}) {
                b->strategy = mode;
                b->cols_per_block = c;
                b->dirty = true;
                float ms = time_ms([&]() { vcbct_batch_forward(b, 0, stream); }, st, 1);
                if (ms < best) {
                    best = ms;
                    bestc = c + 100 * mode;
                }
            }
        }
        tune_store(key.str(), bestc);
    } else {
        bestc = it->second;
    }
    b->strategy = bestc / 100;
    b->cols_per_block = bestc % 100;
    b->dirty = true;
    if (chosen) *chosen = bestc;
    return VCBCT_OK;
}

// ------------------------------------------------------------ host helpers --

extern "C" int vcbct_proj_trig_tables(int W, int H, int V, const double* angles, const double* xs,
                                      const double* ys, double pdet, double dpn, double* c,
                                      double* s, double* xc, double* yc)
{
    (void)W;
    if (V <= 0 || H <= 0 || !angles || !xs || !ys || !c || !s || !xc || !yc)
        return fail(VCBCT_ERR_ARG, "invalid argument");
    // misc.cpp:22-32: the projector's shifts are scaled by 10 and use the
    // detector height for both axes.
    for (int i = 0; i < V; i++) {
        c[i] = std::cos(angles[i]);
        s[i] = std::sin(angles[i]);
        xc[i] = -H / 2.0 - xs[i] * 10.0 / (pdet * (dpn / H));
        yc[i] = -H / 2.0 - ys[i] * 10.0 / (pdet * (dpn / H));
    }
    return VCBCT_OK;
}

// The x-ray DB tables (photo / Compton / Rayleigh, 6 elements + energy per
// row) parsed once per directory and kept for later calls; a change of a
// file's size or modification time re-reads them.
struct XrayDb {
    std::vector<double> e;     // MeV
    std::vector<double> t[3];  // [row][6]
    std::string stamp;
};

static int xray_db(const char* dbdir, std::shared_ptr<const XrayDb>* out)
{
    static std::mutex mu;
    static std::map<std::string, std::shared_ptr<const XrayDb>> cache;
    const char* names[3] = {"photo_5keVto150keV.csv", "comp_5keVto150keV.csv", "rayl_5keVto150keV.csv"};
    std::string stamp;
    for (int t = 0; t < 3; t++) {
        struct stat sb;
        const std::string path = std::string(dbdir) + "/" + names[t];
        if (stat(path.c_str(), &sb) != 0) return fail(VCBCT_ERR_IO, "cannot open " + path);
        stamp += std::to_string((long long)sb.st_size) + ":" + std::to_string((long long)sb.st_mtime) + ";";
    }
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(dbdir);
    if (it != cache.end() && it->second->stamp == stamp) {
        *out = it->second;
        return VCBCT_OK;
    }
    auto dbp = std::make_shared<XrayDb>();
    XrayDb& db = *dbp;
    db.stamp = stamp;
    for (int t = 0; t < 3; t++) {
        std::string path = std::string(dbdir) + "/" + names[t];
        FILE* f = std::fopen(path.c_str(), "r");
        if (!f) return fail(VCBCT_ERR_IO, "cannot open " + path);
        char line[512];
        if (!std::fgets(line, sizeof line, f)) {
            std::fclose(f);
            return fail(VCBCT_ERR_IO, "empty " + path);
        }
        while (std::fgets(line, sizeof line, f)) {
            double v[7];
            if (std::sscanf(line, "%lf,%lf,%lf,%lf,%lf,%lf,%lf", &v[0], &v[1], &v[2], &v[3], &v[4], &v[5], &v[6]) != 7) continue;
            for (int k = 0; k < 6; k++) db.t[t].push_back(v[k]);
            if (t == 0) db.e.push_back(v[6] / 1000 / 1000);
        }
        std::fclose(f);
    }
    const size_t nrow = db.e.size();
    if (nrow == 0 || db.t[1].size() != 6 * nrow || db.t[2].size() != 6 * nrow)
        return fail(VCBCT_ERR_IO, "x-ray DB tables are inconsistent");
    cache[dbdir] = dbp;
    *out = dbp;
    return VCBCT_OK;
}

// Spectrum + x-ray DB lookup, following attenuation_coefficient
// (prior_weight_production.cpp:200-523): bin midpoints in MeV (float sum of
// the CSV's lo/hi), optional merging of nthin bins, pdf normalised in float,
// and for each element the photo + Compton + Rayleigh mass attenuation of the
// DB row whose energy matches the midpoint within 0.03 eV.
extern "C" int vcbct_attenuation_table(const char* spectrum_csv, const char* dbdir, int nmat,
                                       int nthin, float* mu, float* pdf, int* n_bins)
{
    if (!spectrum_csv || !dbdir || !mu || !pdf || !n_bins) return fail(VCBCT_ERR_ARG, "NULL argument");
    if (nmat <= 0 || nmat > 6) return fail(VCBCT_ERR_LIMIT, "the x-ray DB holds 6 elements (H,C,N,O,P,Ca)");
    if (nthin <= 0) return fail(VCBCT_ERR_ARG, "nthin must be positive");
    FILE* fp = std::fopen(spectrum_csv, "r");
    if (!fp) return fail(VCBCT_ERR_IO, std::string("cannot open spectrum ") + spectrum_csv);
    char row[1024];
    std::vector<double> energy;
    std::vector<float> frac;
    if (!std::fgets(row, sizeof row, fp)) {
        std::fclose(fp);
        return fail(VCBCT_ERR_IO, "empty spectrum file");
    }
    while (std::fgets(row, sizeof row, fp)) {
        float lo, hi, fr;
        if (std::sscanf(row, "%f,%f,%f", &lo, &hi, &fr) != 3) continue;
        energy.push_back((hi + lo) * 0.5);
        frac.push_back(fr);
        if (energy.size() > 1024) break;
    }
    std::fclose(fp);
    // merge nthin consecutive bins (:231-248)
    std::vector<float> pdf_t, e_t;
    double psum = 0.0, esum = 0.0, sum_t = 0.0;
    for (size_t i = 0; i < energy.size(); i++) {
        psum += frac[i];
        esum += energy[i];
        const long q = (long)i - nthin + 1;
        if (q >= 0 && q % nthin == 0) {
            pdf_t.push_back((float)psum);
            e_t.push_back((float)(esum / nthin));
            sum_t += psum;
            psum = 0.0;
            esum = 0.0;
        }
    }
    const int NE = (int)pdf_t.size();
    if (NE <= 0 || NE > VCBCT_MAX_BINS) return fail(VCBCT_ERR_LIMIT, "spectrum has no bins or more than 1024");
    const float sum = (float)sum_t;
    for (int i = 0; i < NE; i++) pdf[i] = pdf_t[i] / sum;

    std::shared_ptr<const XrayDb> dbp;
    {
        int rc = xray_db(dbdir, &dbp);
        if (rc) return rc;
    }
    const std::vector<double>& db_e = dbp->e;
    const std::vector<double>* db = dbp->t;
    const size_t nrow = db_e.size();
    for (int k = 0; k < nmat; k++) {
        for (int i = 0; i < NE; i++) {
            const double E = (double)e_t[i];
            long hit = -1;
            for (size_t r = 0; r < nrow; r++) {
                const double aaa = db_e[r] * 1000 * 1000 * 1000 - E * 1000 * 1000 * 1000;
                if (-30 < aaa && aaa < 30) hit = (long)r;  // the last match wins, as :471-501
            }
            if (hit < 0) return fail(VCBCT_ERR_ARG, "spectrum bin midpoint not on the 5 eV DB grid");
            mu[(size_t)k * NE + i] = (float)(db[0][hit * 6 + k] + db[1][hit * 6 + k] + db[2][hit * 6 + k] + 0.0);
        }
    }
    *n_bins = NE;
    return VCBCT_OK;
}

// ------------------------------------------------ reference-named MBFPA API --

namespace {
std::mutex g_ref_mu;
vcbct_projector* g_ref_proj = nullptr;
}  // namespace

extern "C" void vcbct_initializeGPU(int reconSize, double reconScale, int reconSlices, double reconStep,
                              int projImgHeight, int projImgWidth, int totalProjNumber,
                              double* cosTable, double* sinTable, double* XcenterShift,
                              double* YcenterShift, double x_reg, double y_reg, double z_reg,
                              double DETECTOR_PITCH_CM, double DETECTOR_PITCH_CM_AT_ISO_CENT,
                              double DIST_BTWN_SRC_AND_ISOCENT_CM, double DETECTOR_PIXEL_NUM,
                              int num_material)
{
    std::lock_guard<std::mutex> lk(g_ref_mu);
    vcbct_proj_geometry g{reconSize, reconSlices, reconScale, reconStep, projImgWidth,
                          projImgHeight, totalProjNumber, DETECTOR_PITCH_CM,
                          DETECTOR_PITCH_CM_AT_ISO_CENT, DIST_BTWN_SRC_AND_ISOCENT_CM,
                          DETECTOR_PIXEL_NUM, x_reg, y_reg, z_reg, num_material};
    vcbct_projector* p = nullptr;
    int rc = vcbct_projector_create(&g, cosTable, sinTable, XcenterShift, YcenterShift, &p);
    if (rc) {
        std::fprintf(stderr, "initializeGPU: %s\n", vcbct_last_error());
        return;
    }
    if (g_ref_proj) vcbct_projector_destroy(g_ref_proj);
    g_ref_proj = p;
}

extern "C" void vcbct_terminateGPU(void)
{
    std::lock_guard<std::mutex> lk(g_ref_mu);
    vcbct_projector_destroy(g_ref_proj);
    g_ref_proj = nullptr;
}

extern "C" void vcbct_reprojectionOnGPU(int ite, int reconSize, int reconSlices, unsigned short* reconImageshort,
                                  float* reprojection_float, float* npf_double, float* projVolume,
                                  double reconScale, double reconStep, int projImgWidth,
                                  int projImgHeight, int startProjNumber, int endProjNumber,
                                  double* anglesRad, double* cosTable, double* sinTable,
                                  double* XcenterShift, double* YcenterShift, double xfactor,
                                  double* xalpha, double DETECTOR_PITCH_CM,
                                  double DETECTOR_PITCH_CM_AT_ISO_CENT,
                                  double DIST_BTWN_SRC_AND_ISOCENT_CM, double DETECTOR_PIXEL_NUM,
                                  double x_reg, double y_reg, double z_reg, float* Attenuation,
                                  float* pdf_pe, int num_material, int NE, char* outputname)
{
    (void)ite; (void)reprojection_float; (void)npf_double; (void)projVolume; (void)startProjNumber;
    (void)anglesRad; (void)xalpha; (void)reconScale; (void)reconStep; (void)cosTable;
    (void)sinTable; (void)XcenterShift; (void)YcenterShift; (void)DETECTOR_PITCH_CM;
    (void)DETECTOR_PITCH_CM_AT_ISO_CENT; (void)DIST_BTWN_SRC_AND_ISOCENT_CM;
    (void)DETECTOR_PIXEL_NUM; (void)x_reg; (void)y_reg; (void)z_reg;
    std::lock_guard<std::mutex> lk(g_ref_mu);
    vcbct_projector* p = g_ref_proj;
    if (!p) {
        std::fprintf(stderr, "reprojectionOnGPU: initializeGPU was not called\n");
        return;
    }
    // the geometry set by initializeGPU is the one used (as the reference's
    // __constant__ memory); the counts here must agree with it
    if (reconSize != p->g.recon_size || reconSlices != p->g.recon_slices ||
        projImgWidth != p->g.proj_width || projImgHeight != p->g.proj_height ||
        num_material != p->g.num_material || endProjNumber <= 0 || endProjNumber > p->g.n_views) {
        std::fprintf(stderr, "reprojectionOnGPU: arguments disagree with initializeGPU\n");
        return;
    }
    const int V = endProjNumber;  // views 0..endProjNumber-1, as the launch grid (:976)
    const int saveV = p->g.n_views;
    p->g.n_views = V;
    p->pp.V = V;
    int rc = vcbct_projector_set_spectrum(p, Attenuation, pdf_pe, NE, xfactor);
    std::vector<float> out((size_t)V * projImgHeight * projImgWidth);
    if (!rc) rc = vcbct_projector_project(p, reconImageshort, out.data(), nullptr);
    p->g.n_views = saveV;
    p->pp.V = saveV;
    if (rc) {
        std::fprintf(stderr, "reprojectionOnGPU: %s\n", vcbct_last_error());
        return;
    }
    char fname[512];
    std::snprintf(fname, sizeof fname, "%s.raw", outputname ? outputname : "reprojection");
    FILE* f = std::fopen(fname, "wb");
    if (!f) {
        std::fprintf(stderr, "reprojectionOnGPU: cannot write %s\n", fname);
        return;
    }
    std::fwrite(out.data(), sizeof(float), out.size(), f);
    std::fclose(f);
}

// ======================================================================= FDK

struct vcbct_fdk {
    vcbct_fdk_geometry g;
    FdkParams fp;
    std::vector<double> angles, xs, ys, h;  // host copies
    DevBuf hT;        // float [W][W]
    DevBuf fviews;    // FilterView[V]
    DevBuf bviews;    // BpView[V]
    DevBuf wts;       // float [V][W] redundancy weights (optional)
    DevBuf in, mid, outv, outs, work;
    DevBuf bpkeep;    // per-block view masks of the backprojection
    int bp_keep_ready = 0;    // the masks in `bpkeep` are made (they follow the geometry only) ...
    void* bp_keep_at = nullptr;  // ... at this address
    int have_wts = 0;
    int b_ready = 0;          // the tensor-core filter's Toeplitz planes are split in `work`
    void* b_at = nullptr;     // ... at this address
};

extern "C" void vcbct_fdk_default_geometry(vcbct_fdk_geometry* g)
{
    if (!g) return;
    std::memset(g, 0, sizeof *g);
    // R/physParams.h:22-41 and the shipped FDK txt (FDK_36pro_water20cm.txt)
    g->proj_width = 400;
    g->proj_height = 400;
    g->n_views = 36;
    g->recon_size = 270;
    g->recon_slices = 50;
    g->zstart = -5;
    g->recon_step = 0.2;
    g->recon_scale = 0.1;
    g->xfactor = 1000;
    g->det_pitch_iso_cm = 0.032509752;
    g->det_pitch_cm = 0.05;
    g->max_pic_num = 800;
    g->sad_cm = 100.0;
    g->cutoff = 1.60;
    g->gamma = 1.00;
    g->alpha = 0.50;
    g->redundancy = 0;
}

// Ramp kernel h[m][n] of prepareConstMap (filterSinogram.cpp:21-62): a
// band-limited Ram-Lak/Hamming-type kernel with cutoff CUTOFF_FREQ and
// window ALPHA, GAMMA; zero on the diagonal.
static void ramp_kernel(int W, double piso, double mpn, double cutoff, double gam, double alpha,
                        double* h)
{
    const double c0 = 1.0 / (8.0 * kPi * kPi * piso * mpn / W);
    const double gc = gam * cutoff, pc = kPi * cutoff, oma = 1.0 - alpha;
    const double om = kPi / gam, co = std::cos(om), so = std::sin(om);
    for (int m = 0; m < W; m++)
        for (int n = 0; n < W; n++) {
            if (m == n) {
                h[(size_t)m * W + n] = 0.0;
                continue;
            }
            const double d = (double)(m - n);
            const double th = pc * d, de = gc * d;
            const double eta = 1.0 / (1.0 - 1.0 / de), xi = 1.0 / (1.0 + 1.0 / de);
            const double ct = std::cos(th), st = std::sin(th);
            h[(size_t)m * W + n] = c0 / d / d *
                (2.0 * alpha * th * st + 2.0 * alpha * (ct - 1.0) +
                 xi * oma * th * (st * co + ct * so) + eta * oma * th * (st * co - ct * so) +
                 xi * xi * oma * (ct * co - st * so - 1.0) +
                 eta * eta * oma * (ct * co + st * so - 1.0));
        }
}

static double filter_coeff(const vcbct_fdk_geometry& g)
{
    // filterSinogram.cpp:79-80
    const double om = kPi / g.gamma;
    return g.cutoff * g.cutoff / 4.0 / (g.det_pitch_iso_cm * g.max_pic_num / g.proj_width) *
           (g.alpha * 0.5 + (1.0 - g.alpha) * (1.0 / om * std::sin(om) + 1.0 / om / om * (std::cos(om) - 1.0)));
}

static int upload_kernel(vcbct_fdk* f)
{
    const int W = f->g.proj_width;
    const double coeff = filter_coeff(f->g);
    std::vector<float> hT((size_t)W * W);
    for (int k = 0; k < W; k++)
        for (int m = 0; m < W; m++)
            hT[(size_t)k * W + m] = (float)(f->h[(size_t)m * W + k] + (m == k ? coeff : 0.0));
    VCBCT_CUDA_TRY(f->hT.ensure(hT.size() * sizeof(float)));
    VCBCT_CUDA_TRY(cudaMemcpy(f->hT.p, hT.data(), hT.size() * sizeof(float), cudaMemcpyHostToDevice));
    f->b_ready = 0;  // the split Toeplitz planes follow the kernel
    return VCBCT_OK;
}

// Redundancy weights for an offset (half-fan) detector over a full rotation
// (Wang, Med. Phys. 29 (2002) 1464): with u the lateral column position at
// the isocentre and u0 the half-width of the band seen from both sides of the
// rotation axis, w = 2 sin^2(pi/4 (1 + u/u0)) inside the band, 2 on the long
// side beyond it and 0 beyond the short edge, so conjugate rays sum to 2 and
// the 2*pi angular integral stays normalised.  Not in the reference, which
// has only the offset terms of Cm and UUU.
static void halffan_weights(const vcbct_fdk& f, std::vector<float>& w)
{
    const int W = f.g.proj_width, V = f.g.n_views;
    const double pitch = f.g.det_pitch_iso_cm * f.g.max_pic_num / W;
    const double px = f.g.det_pitch_cm * f.g.max_pic_num / W;
    w.assign((size_t)V * W, 1.0f);
    for (int v = 0; v < V; v++) {
        const double xcs = -W / 2.0 - f.xs[v] / px - 1;
        const double umin = xcs * pitch, umax = (xcs + W - 1) * pitch;
        const double u0 = std::fmin(-umin, umax);
        if (!(u0 > 0)) continue;
        const double side = (umax >= -umin) ? 1.0 : -1.0;  // +1: long side at +u
        for (int m = 0; m < W; m++) {
            const double x = side * (xcs + m) * pitch / u0;
            double wt;
            if (x >= 1.0) wt = 2.0;
            else if (x <= -1.0) wt = 0.0;
            else {
                const double sn = std::sin(kPi / 4.0 * (1.0 + x));
                wt = 2.0 * sn * sn;
            }
            w[(size_t)v * W + m] = (float)wt;
        }
    }
}

extern "C" int vcbct_fdk_redundancy_weights(const vcbct_fdk_geometry* g, const double* xshift, float* w)
{
    if (!g || !xshift || !w) return fail(VCBCT_ERR_ARG, "NULL argument");
    if (g->proj_width <= 1 || g->n_views <= 0 || !(g->det_pitch_iso_cm > 0) || !(g->det_pitch_cm > 0) ||
        !(g->max_pic_num > 0))
        return fail(VCBCT_ERR_ARG, "FDK sizes and pitches must be positive");
    vcbct_fdk f;  // host fields only: the weights read the geometry and the shifts
    f.g = *g;
    f.xs.assign(xshift, xshift + g->n_views);
    std::vector<float> wv;
    halffan_weights(f, wv);
    std::copy(wv.begin(), wv.end(), w);
    return VCBCT_OK;
}

extern "C" int vcbct_fdk_create(const vcbct_fdk_geometry* g, const double* angles,
                                const double* xshift, const double* yshift, vcbct_fdk** out)
{
    if (!out) return fail(VCBCT_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!g || !angles || !xshift || !yshift) return fail(VCBCT_ERR_ARG, "NULL argument");
    if (g->proj_width <= 1 || g->proj_height <= 1 || g->n_views < 2 || g->recon_size <= 0 ||
        g->recon_slices <= 0)
        return fail(VCBCT_ERR_ARG, "FDK sizes must be positive (at least 2 views)");
    if (!(g->det_pitch_iso_cm > 0) || !(g->det_pitch_cm > 0) || !(g->max_pic_num > 0) || !(g->sad_cm > 0))
        return fail(VCBCT_ERR_ARG, "FDK pitches and distances must be positive");
    auto* f = new vcbct_fdk();
    f->g = *g;
    const int V = g->n_views, W = g->proj_width;
    f->angles.assign(angles, angles + V);
    f->xs.assign(xshift, xshift + V);
    f->ys.assign(yshift, yshift + V);
    f->fp = FdkParams{g->proj_width, g->proj_height, V, g->recon_size, g->recon_slices, g->zstart,
                      g->xfactor, g->redundancy, g->recon_step, g->recon_scale, g->det_pitch_iso_cm,
                      g->det_pitch_cm, g->max_pic_num, g->sad_cm};
    f->h.resize((size_t)W * W);
    ramp_kernel(W, g->det_pitch_iso_cm, g->max_pic_num, g->cutoff, g->gamma, g->alpha, f->h.data());
    int rc = upload_kernel(f);
    if (rc) {
        vcbct_fdk_destroy(f);  // frees what was allocated
        return rc;
    }
    std::vector<FilterView> fv(V);
    std::vector<BpView> bv(V);
    const double px = g->det_pitch_cm * g->max_pic_num / W;
    for (int th = 0; th < V; th++) {
        // filterSinogram.cpp:86-87 (the height shift also uses the width)
        fv[th].xcs = (float)(-W / 2.0 - f->xs[th] / px - 1);
        fv[th].ycs = (float)(-W / 2.0 - f->ys[th] / px - 1);
        // reconstructImage.cpp:37-72
        double dbeta;
        if (th == 0) dbeta = std::fabs(angles[1] - angles[0]) / 2;
        else if (th == V - 1) dbeta = std::fabs(angles[th] - angles[th - 1]) / 2;
        else {
            const double t0 = angles[th - 1], t2 = angles[th + 1];
            double t1 = angles[th + 1] - 2 * kPi;
            if (t2 < 0) t1 = angles[th + 1] + 2 * kPi;
            dbeta = std::fabs(t2 - t0) / 2;
            if (dbeta > kPi / 2) dbeta = std::fabs(t1 - t0) / 2;
        }
        bv[th].cs = std::cos(angles[th]);
        bv[th].sn = std::sin(angles[th]);
        bv[th].ushift = (double)(W / 2) + f->xs[th] / px - 0.5;
        bv[th].dbeta = (float)dbeta;
        bv[th].pad = 0.0f;
    }
    cudaError_t e = f->fviews.ensure(sizeof(FilterView) * V);
    if (e == cudaSuccess) e = cudaMemcpy(f->fviews.p, fv.data(), sizeof(FilterView) * V, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = f->bviews.ensure(sizeof(BpView) * V);
    if (e == cudaSuccess) e = cudaMemcpy(f->bviews.p, bv.data(), sizeof(BpView) * V, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && g->redundancy == 1) {
        std::vector<float> w;
        halffan_weights(*f, w);
        e = f->wts.ensure(w.size() * sizeof(float));
        if (e == cudaSuccess) e = cudaMemcpy(f->wts.p, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice);
        f->have_wts = 1;
    }
    if (e != cudaSuccess) {
        vcbct_fdk_destroy(f);  // frees what was allocated
        return cuda_fail(e, "vcbct_fdk_create");
    }
    *out = f;
    return VCBCT_OK;
}

extern "C" int vcbct_fdk_destroy(vcbct_fdk* f)
{
    if (!f) return VCBCT_OK;
    f->hT.release(); f->fviews.release(); f->bviews.release(); f->wts.release();
    f->in.release(); f->mid.release(); f->outv.release(); f->outs.release(); f->work.release();
    delete f;
    return VCBCT_OK;
}

extern "C" int vcbct_fdk_set_kernel(vcbct_fdk* f, const double* h)
{
    if (!f || !h) return fail(VCBCT_ERR_ARG, "NULL argument");
    f->h.assign(h, h + (size_t)f->g.proj_width * f->g.proj_width);
    return upload_kernel(f);
}

extern "C" int vcbct_fdk_filter(vcbct_fdk* f, const float* proj, float* filtered, int on_device,
                                int method, void* stream)
{
    if (!f || !proj || !filtered) return fail(VCBCT_ERR_ARG, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    const auto& g = f->g;
    const size_t n = (size_t)g.n_views * g.proj_height * g.proj_width;
    const float* din = proj;
    float* dout = filtered;
    if (!on_device) {
        VCBCT_CUDA_TRY(f->in.ensure(n * sizeof(float)));
        VCBCT_CUDA_TRY(f->mid.ensure(n * sizeof(float)));
        VCBCT_CUDA_TRY(cudaMemcpyAsync(f->in.p, proj, n * sizeof(float), cudaMemcpyHostToDevice, st));
        din = f->in.as<float>();
        dout = f->mid.as<float>();
    }
    const float pitch = (float)(g.det_pitch_iso_cm * g.max_pic_num / g.proj_width);
    const float* w = f->have_wts ? f->wts.as<float>() : nullptr;
    // the tensor-core tiles take 16 to 4096 detector columns; outside that
    // the direct filter runs (the same result within the 1e-5 tolerance)
    if (method == VCBCT_FILTER_BF16X3 && (g.proj_width < 16 || g.proj_width > 4096)) method = VCBCT_FILTER_DIRECT_F32;
    if (method == VCBCT_FILTER_DIRECT_F32) {
        VCBCT_CUDA_TRY(launch_filter_direct(din, dout, f->hT.as<float>(), f->fviews.as<FilterView>(), w,
                                            pitch, (float)g.sad_cm, g.n_views, g.proj_height,
                                            g.proj_width, st));
    } else if (method == VCBCT_FILTER_BF16X3) {
        VCBCT_CUDA_TRY(f->work.ensure(ramp_gemm_workspace_bytes(g.n_views, g.proj_height, g.proj_width,
                                                                 ramp_gemm_fused(din, dout, g.proj_width))));
        if (f->work.p != f->b_at) {
            f->b_ready = 0;
            f->b_at = f->work.p;
        }
        VCBCT_CUDA_TRY(launch_ramp_gemm_bf16x3(din, dout, f->hT.as<float>(), f->fviews.as<FilterView>(), w,
                                               pitch, (float)g.sad_cm, g.n_views, g.proj_height,
                                               g.proj_width, f->work.p, &f->b_ready, st));
    } else {
        return fail(VCBCT_ERR_ARG, "unknown filter method");
    }
    if (!on_device) {
        VCBCT_CUDA_TRY(cudaMemcpyAsync(filtered, dout, n * sizeof(float), cudaMemcpyDeviceToHost, st));
        VCBCT_CUDA_TRY(cudaStreamSynchronize(st));
        if (method == VCBCT_FILTER_BF16X3 &&
            ramp_gemm_error_flag(f->work.p, g.n_views, g.proj_height, g.proj_width, st) != 0)
            return fail(VCBCT_ERR_DEVICE, "tensor-core filter: a bounded wait ran out (output invalid)");
    }
    return VCBCT_OK;
}

extern "C" int vcbct_fdk_backproject(vcbct_fdk* f, const float* filtered, float* vol_f32,
                                     short* vol_i16, int on_device, void* stream)
{
    if (!f || !filtered || (!vol_f32 && !vol_i16)) return fail(VCBCT_ERR_ARG, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    const auto& g = f->g;
    const size_t np = (size_t)g.n_views * g.proj_height * g.proj_width;
    const size_t nv = (size_t)g.recon_slices * g.recon_size * g.recon_size;
    const float* din = filtered;
    float* df = vol_f32;
    short* di = vol_i16;
    if (!on_device) {
        VCBCT_CUDA_TRY(f->in.ensure(np * sizeof(float)));
        VCBCT_CUDA_TRY(cudaMemcpyAsync(f->in.p, filtered, np * sizeof(float), cudaMemcpyHostToDevice, st));
        din = f->in.as<float>();
        if (vol_f32) {
            VCBCT_CUDA_TRY(f->outv.ensure(nv * sizeof(float)));
            df = f->outv.as<float>();
        }
        if (vol_i16) {
            VCBCT_CUDA_TRY(f->outs.ensure(nv * sizeof(short)));
            di = f->outs.as<short>();
        }
    }
    VCBCT_CUDA_TRY(f->bpkeep.ensure(backproject_workspace_bytes(f->fp)));
    if (f->bpkeep.p != f->bp_keep_at) {
        f->bp_keep_ready = 0;
        f->bp_keep_at = f->bpkeep.p;
    }
    VCBCT_CUDA_TRY(launch_backproject(f->fp, f->bviews.as<BpView>(), din, df, di, f->bpkeep.as<unsigned>(),
                                      &f->bp_keep_ready, st));
    if (!on_device) {
        if (vol_f32) VCBCT_CUDA_TRY(cudaMemcpyAsync(vol_f32, df, nv * sizeof(float), cudaMemcpyDeviceToHost, st));
        if (vol_i16) VCBCT_CUDA_TRY(cudaMemcpyAsync(vol_i16, di, nv * sizeof(short), cudaMemcpyDeviceToHost, st));
        VCBCT_CUDA_TRY(cudaStreamSynchronize(st));
    }
    return VCBCT_OK;
}

// ------------------------------------------------- reference-named FDK API --

extern "C" double** vcbct_prepareConstMap(int projWidth, double piso)
{
    if (projWidth <= 0) {
        std::fprintf(stderr, "ERROR: invalid projWidth for prepareConstMap\n");
        return nullptr;
    }
    // VOLUME-ONE 2D layout (mallocMD.cpp:47-67): contiguous data + row table
    double* data = (double*)std::calloc((size_t)projWidth * projWidth, sizeof(double));
    double** rows = (double**)std::malloc(sizeof(double*) * projWidth);
    if (!data || !rows) {
        std::free(data);
        std::free(rows);
        std::fprintf(stderr, "ERROR: not enough memory for prepareConstMap\n");
        return nullptr;
    }
    for (int j = 0; j < projWidth; j++) rows[j] = data + (size_t)j * projWidth;
    vcbct_fdk_geometry g;
    vcbct_fdk_default_geometry(&g);
    ramp_kernel(projWidth, piso, g.max_pic_num, g.cutoff, g.gamma, g.alpha, data);
    return rows;
}

extern "C" void vcbct_free_const_map(double** m, int projWidth)
{
    (void)projWidth;
    if (!m) return;
    std::free(m[0]);
    std::free(m);
}

extern "C" void vcbct_filterSinogram(int projHeight, int projWidth, int sngrmHeight, float*** projVolume,
                               float*** fltdVoxData, double** constMap, double* xshift,
                               double* yshift, double piso)
{
    if (!fltdVoxData || !projVolume || !constMap) {
        std::fprintf(stderr, "ERROR: fltdVoxData is NULL\n");
        return;
    }
    vcbct_fdk_geometry g;
    vcbct_fdk_default_geometry(&g);
    g.proj_width = projWidth;
    g.proj_height = projHeight;
    g.n_views = sngrmHeight;
    g.det_pitch_iso_cm = piso;
    std::vector<double> ang(sngrmHeight > 1 ? sngrmHeight : 2, 0.0);
    for (size_t i = 0; i < ang.size(); i++) ang[i] = (double)i;  // unused by the filter
    std::vector<double> ys(yshift, yshift + sngrmHeight), xs(xshift, xshift + sngrmHeight);
    if (sngrmHeight < 2) { xs.resize(2, 0.0); ys.resize(2, 0.0); g.n_views = 2; }
    vcbct_fdk* f = nullptr;
    int rc = vcbct_fdk_create(&g, ang.data(), xs.data(), ys.data(), &f);
    if (!rc) rc = vcbct_fdk_set_kernel(f, constMap[0]);
    if (!rc) {
        f->g.n_views = sngrmHeight;
        f->fp.V = sngrmHeight;
        // the tensor-core filter unless VCBCT_FILTER=direct asks for the FP32
        // direct one (both within 1e-5 of the FP64 filter's scale)
        const char* fm = std::getenv("VCBCT_FILTER");
        const int method =
            (fm && std::strcmp(fm, "direct") == 0) ? VCBCT_FILTER_DIRECT_F32 : VCBCT_FILTER_BF16X3;
        rc = vcbct_fdk_filter(f, &projVolume[0][0][0], &fltdVoxData[0][0][0], 0, method, nullptr);
    }
    if (rc) std::fprintf(stderr, "filterSinogram: %s\n", vcbct_last_error());
    vcbct_fdk_destroy(f);
}

extern "C" void vcbct_reconstructImage(int reconSize, int reconSlices, int zstart, double reconStep,
                                 double reconScale, double*** reconVoxData, char** maskData,
                                 int projHeight, int projWidth, int sngrmHeight,
                                 float*** sngrmVoxData, int xfactor, double* anglesRad,
                                 double* cosTable, double* sinTable, double* xshift, double piso)
{
    (void)cosTable; (void)sinTable;
    if (!reconVoxData) {
        std::fprintf(stderr, "ERROR: reconVoxData is NULL\n");
        return;
    }
    vcbct_fdk_geometry g;
    vcbct_fdk_default_geometry(&g);
    g.proj_width = projWidth;
    g.proj_height = projHeight;
    g.n_views = sngrmHeight;
    g.recon_size = reconSize;
    g.recon_slices = reconSlices;
    g.zstart = zstart;
    g.recon_step = reconStep;
    g.recon_scale = reconScale;
    g.xfactor = xfactor;
    g.det_pitch_iso_cm = piso;
    std::vector<double> ys(sngrmHeight, 0.0);
    vcbct_fdk* f = nullptr;
    int rc = vcbct_fdk_create(&g, anglesRad, xshift, ys.data(), &f);
    const size_t nv = (size_t)reconSlices * reconSize * reconSize;
    std::vector<float> vol(nv);
    if (!rc) rc = vcbct_fdk_backproject(f, &sngrmVoxData[0][0][0], vol.data(), nullptr, 0, nullptr);
    vcbct_fdk_destroy(f);
    if (rc) {
        std::fprintf(stderr, "reconstructImage: %s\n", vcbct_last_error());
        return;
    }
    double* dst = &reconVoxData[0][0][0];
    for (int z = 0; z < reconSlices; z++)
        for (int y = 0; y < reconSize; y++)
            for (int x = 0; x < reconSize; x++) {
                if (maskData && maskData[y][x] == 0) continue;
                const size_t o = ((size_t)z * reconSize + y) * reconSize + x;
                dst[o] += (double)vol[o];
            }
}
