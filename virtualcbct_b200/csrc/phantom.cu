// phantom.cu -- element volumes from organ-labelled voxel phantoms, the
// conversion of ICRPphantoms_2mmslice/To_material_distribution_for512_random.cpp:
//
//  - host: the media table (mass percentages of H, C, N, O, P, Ca per medium)
//    and the organ table (organ number -> medium, density) are read from the
//    reference's CSV files and jittered with the reference's Gaussian draws
//    (:14-24, :117-165, :178-198), consuming the C library's rand() sequence
//    for the given seed in the reference's order, through a private
//    random_r state so the process's rand() is untouched;
//  - device: each voxel's organ number is mapped to its six element values
//    (short)(percent x density x 10) (:212-226) by a table lookup, writing the
//    projector's [Z][6][rows][cols] uint16 layout (HBM-bound: 1 byte read and
//    12 written per voxel).
#include "internal.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

namespace vcbct {
namespace {

// Uniform0 / rand_gauss0 of the reference (:14-24) on a private state.
struct RefRng {
    struct random_data data;
    char state[128];
    explicit RefRng(unsigned seed)
    {
        std::memset(&data, 0, sizeof data);
        std::memset(state, 0, sizeof state);
        initstate_r(seed, state, sizeof state, &data);
    }
    double uniform()
    {
        int32_t r = 0;
        random_r(&data, &r);
        return ((double)r + 1.0) / ((double)RAND_MAX + 2.0);
    }
    double gauss(double mu, double sigma)
    {
        const double PI = 3.14159265;
        const double u1 = uniform();  // the operand order g++ evaluates
        const double u2 = uniform();
        const double z = std::sqrt(-2.0 * std::log(u1)) * std::sin(2.0 * PI * u2);
        return mu + sigma * z;
    }
};

// The element table travels in the launch's parameter block (4 KB), so the
// device path needs no allocation: one 16-byte row per organ number (six
// uint16 elements and two pads), copied to shared memory, where each voxel's
// data-dependent lookup is one 16-byte read.
struct OrganTable {
    uint4 row[256];
};

__device__ __forceinline__ uint32_t elem_word(const uint4& r, int w)
{
    return w == 0 ? r.x : (w == 1 ? r.y : r.z);
}

// grid: (ceil(slice / (256 * PER)), Z); block 256.  PER voxels per thread:
// 8 when slice % 8 == 0 (8-byte id loads, 16-byte stores per element plane),
// else 1.
template <int PER>
__global__ void __launch_bounds__(256) organs_to_elements_kernel(const uint8_t* __restrict__ ids, long long slice,
                                                                 const __grid_constant__ OrganTable tab,
                                                                 uint16_t* __restrict__ out)
{
    __shared__ uint4 t[256];
    t[threadIdx.x] = tab.row[threadIdx.x];
    __syncthreads();
    const long long n = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * PER;
    const int z = blockIdx.y;
    if (n >= slice) return;
    const uint8_t* src = ids + (long long)z * slice + n;
    uint16_t* o = out + (long long)z * 6 * slice + n;
    if constexpr (PER == 8) {
        const uint2 v = *reinterpret_cast<const uint2*>(src);
        uint4 r[8];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            r[k] = t[(v.x >> (8 * k)) & 255];
            r[4 + k] = t[(v.y >> (8 * k)) & 255];
        }
#pragma unroll
        for (int m = 0; m < 6; m++) {
            const uint32_t sel = (m & 1) ? 0x7632u : 0x5410u;  // high or low halves of the two words
            uint4 w;
            w.x = __byte_perm(elem_word(r[0], m >> 1), elem_word(r[1], m >> 1), sel);
            w.y = __byte_perm(elem_word(r[2], m >> 1), elem_word(r[3], m >> 1), sel);
            w.z = __byte_perm(elem_word(r[4], m >> 1), elem_word(r[5], m >> 1), sel);
            w.w = __byte_perm(elem_word(r[6], m >> 1), elem_word(r[7], m >> 1), sel);
            *reinterpret_cast<uint4*>(o + (long long)m * slice) = w;
        }
    } else {
        const uint4 r = t[*src];
#pragma unroll
        for (int m = 0; m < 6; m++) o[(long long)m * slice] = (uint16_t)(elem_word(r, m >> 1) >> (16 * (m & 1)));
    }
}

static cudaError_t launch_organs(const uint8_t* ids, long long slice, int Z, const OrganTable& tab, uint16_t* out,
                                 cudaStream_t st)
{
    const bool vec = slice % 8 == 0 && (reinterpret_cast<uintptr_t>(ids) & 7) == 0 &&
                     (reinterpret_cast<uintptr_t>(out) & 15) == 0;
    if (vec) {
        dim3 grid((unsigned)((slice / 8 + 255) / 256), (unsigned)Z);
        organs_to_elements_kernel<8><<<grid, 256, 0, st>>>(ids, slice, tab, out);
    } else {
        dim3 grid((unsigned)((slice + 255) / 256), (unsigned)Z);
        organs_to_elements_kernel<1><<<grid, 256, 0, st>>>(ids, slice, tab, out);
    }
    return cudaGetLastError();
}

}  // namespace
}  // namespace vcbct

using namespace vcbct;

extern "C" int vcbct_phantom_tables_read(const char* media_csv, const char* organs_csv, unsigned seed,
                                         vcbct_phantom_tables* t)
{
    if (!media_csv || !organs_csv || !t) return fail(VCBCT_ERR_ARG, "NULL argument");
    std::memset(t, 0, sizeof *t);
    RefRng rng(seed);
    FILE* fp = std::fopen(media_csv, "r");
    if (!fp) return fail(VCBCT_ERR_IO, std::string("cannot open ") + media_csv);
    int n = 0;
    for (;;) {
        int id;
        float w[13];
        const int r = std::fscanf(fp, "%d,%f,%f,%f,%f,%f,%f,%f,%f,%f,%f,%f,%f,%f", &id, &w[0], &w[1], &w[2], &w[3],
                                  &w[4], &w[5], &w[6], &w[7], &w[8], &w[9], &w[10], &w[11], &w[12]);
        if (r == EOF) break;
        if (r != 14) {
            std::fclose(fp);
            return fail(VCBCT_ERR_IO, std::string(media_csv) + ": malformed row " + std::to_string(n + 1));
        }
        if (n >= VCBCT_MAX_MEDIA) {
            std::fclose(fp);
            return fail(VCBCT_ERR_LIMIT, "more media than VCBCT_MAX_MEDIA");
        }
        // columns H C N O Na Mg P S Cl K Ca Fe I; keep H C N O P Ca
        float H = w[0], Cc = w[1], Nn = w[2], O = w[3], P = w[6], Ca = w[10];
        if (id != 53) {  // medium 53 (air) is not jittered (:119)
            double sigma = double(H * 0.1), mu = double(H);
            H = (float)(rng.gauss(mu, sigma));
            if (H < 0.0) H = 0.0;
            sigma = double(Cc * 0.1);
            mu = double(Cc);
            Cc = (float)(rng.gauss(mu, sigma));
            if (Cc < 0.0) Cc = 0.0;
            sigma = double(Nn * 0.1);
            mu = double(Nn);
            Nn = (float)(rng.gauss(mu, sigma));
            if (Nn < 0.0) Nn = 0.0;
            if (P > 0.09) {
                sigma = double(P * 0.1);
                mu = double(P);
                P = (float)(rng.gauss(mu, sigma));
                if (P < 0.0) P = 0.0;
            }
            if (Ca > 0.09) {
                sigma = double(Ca * 0.1);
                mu = double(Ca);
                Ca = (float)(rng.gauss(mu, sigma));
                if (Ca < 0.0) Ca = 0.0;
            }
        }
        O = 100 - H - Cc - Nn - P - Ca;  // oxygen closes the sum (:151-162)
        if (O < 0.0) {
            const double s = (H + Cc + Nn + P + Ca) * 0.01;
            O = 0.0;
            H = H / s;
            Cc = Cc / s;
            Nn = Nn / s;
            P = P / s;
            Ca = Ca / s;
        }
        t->media_id[n] = id;
        float* m = t->media[n];
        m[0] = H;
        m[1] = Cc;
        m[2] = Nn;
        m[3] = O;
        m[4] = P;
        m[5] = Ca;
        n++;
    }
    std::fclose(fp);
    t->n_media = n;

    fp = std::fopen(organs_csv, "r");
    if (!fp) return fail(VCBCT_ERR_IO, std::string("cannot open ") + organs_csv);
    int k = 0;
    for (;;) {
        int organ, medium;
        float dens;
        const int r = std::fscanf(fp, "%d,%d,%f", &organ, &medium, &dens);
        if (r == EOF) break;
        if (r != 3) {
            std::fclose(fp);
            return fail(VCBCT_ERR_IO, std::string(organs_csv) + ": malformed row " + std::to_string(k + 1));
        }
        if (k >= VCBCT_MAX_ORGANS) {
            std::fclose(fp);
            return fail(VCBCT_ERR_LIMIT, "more organs than VCBCT_MAX_ORGANS");
        }
        // the reference draws a jittered density here (:180-195) but writes
        // the tabulated one (:218-223); the draws still advance the sequence
        if (medium != 53) {
            if (medium <= 2) (void)rng.gauss(double(dens * 0.9), double(dens * 0.05));
            else (void)rng.gauss(double(dens), double(dens * 0.05));
        }
        t->organ[k] = organ;
        t->organ_medium[k] = medium;
        t->organ_density[k] = dens;
        k++;
    }
    std::fclose(fp);
    t->n_organs = k;

    // voxel value -> six element values; the last organ row with that number
    // wins (:214-225); numbers without a row stay 0
    for (int j = 0; j < k; j++) {
        const int v = t->organ[j];
        const int mi = t->organ_medium[j] - 1;  // media are indexed by id - 1 (:218)
        if (v < 0 || v > 255) continue;
        if (mi < 0 || mi >= t->n_media) return fail(VCBCT_ERR_ARG, "organ row names a medium that is not listed");
        for (int e = 0; e < 6; e++) t->table[v][e] = (uint16_t)(short)(t->media[mi][e] * t->organ_density[j] * 10);
    }
    return VCBCT_OK;
}

extern "C" int vcbct_organs_to_elements(const uint8_t* ids, long long slice_voxels, int Z,
                                        const vcbct_phantom_tables* t, uint16_t* out, int on_device, void* stream)
{
    if (!ids || !t || !out) return fail(VCBCT_ERR_ARG, "NULL argument");
    if (slice_voxels <= 0 || Z <= 0) return fail(VCBCT_ERR_ARG, "sizes must be positive");
    if (Z > 65535) return fail(VCBCT_ERR_LIMIT, "more than 65535 slices");
    cudaStream_t st = (cudaStream_t)stream;
    OrganTable tab;
    std::memset(&tab, 0, sizeof tab);
    for (int v = 0; v < 256; v++) {
        const uint16_t* e = t->table[v];
        tab.row[v] = make_uint4((uint32_t)e[0] | ((uint32_t)e[1] << 16), (uint32_t)e[2] | ((uint32_t)e[3] << 16),
                                (uint32_t)e[4] | ((uint32_t)e[5] << 16), 0u);
    }
    if (on_device) {  // asynchronous on `stream`, no allocation
        VCBCT_CUDA_TRY(launch_organs(ids, slice_voxels, Z, tab, out, st));
        return VCBCT_OK;
    }
    const size_t nid = (size_t)slice_voxels * Z, nout = nid * 6;
    void* buf = nullptr;
    const size_t o_out = (nid + 255) / 256 * 256;
    VCBCT_CUDA_TRY(cudaMalloc(&buf, o_out + nout * sizeof(uint16_t)));
    char* b = static_cast<char*>(buf);
    uint8_t* d_ids = reinterpret_cast<uint8_t*>(b);
    uint16_t* d_out = reinterpret_cast<uint16_t*>(b + o_out);
    cudaError_t e = cudaMemcpyAsync(d_ids, ids, nid, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = launch_organs(d_ids, slice_voxels, Z, tab, d_out, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, nout * sizeof(uint16_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(buf);
    if (e != cudaSuccess) return cuda_fail(e, "organs_to_elements");
    return VCBCT_OK;
}
