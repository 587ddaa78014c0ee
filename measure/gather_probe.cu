// gather_probe.cu -- measured gather rooflines of the two gather-bound kernels.
//
// Measurement code only: built into measure/libgather_probe.so for bench.py,
// not part of libvcbct.so.
//
// The forward projector and the backprojector are bound by how fast the SMs
// can gather small records, not by DRAM streaming (their working sets sit in
// L2 / L1).  These probes replay each kernel's access pattern with no
// arithmetic around it, on the same device, so a kernel's rate divided by the
// probe's rate is its fraction of the achievable gather bandwidth.
//
//  kind 0, ray-front gather (the MBFPA pattern): a z-fastest volume of 16-byte
//    records, 512 x 512 x 200 (839 MB, larger than L2).  A warp is 32 adjacent
//    detector rows of one column: at each dominant-axis step its lanes read a
//    run of 11 consecutive records (the z extent of 32 rows at 2 mm slices),
//    and the next step moves one voxel along x (stride Z records).  Each warp
//    marches 512 steps from a random (y, z) start, then restarts.  Rate unit:
//    lane-records per second (one per lane and step = one segment).
//  kind 1, detector-tile gather from shared memory (the BP pattern): a block
//    stages a 64 x 96 float tile of one filtered view once; each thread reads the
//    four bilinear taps of one voxel per slice, neighbouring threads 1.5
//    columns apart, successive slices 3.1 rows apart.  Rate unit: voxel
//    updates (4 taps) per second.
//  kind 2, the same BP pattern read from global memory through L1.
//  kind 3, kind 0 with 32-byte records (8 floats, two 16-byte loads per lane
//    and step; 1.68 GB): the float records the projector object keeps.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>

namespace {

constexpr int kProbeN = 512, kProbeZ = 200, kRun = 11, kSteps = 512;

__device__ __forceinline__ uint32_t hash32(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

// HALVES: 16-byte loads per record (1: uint16 records, 2: float records)
template <int HALVES>
__global__ void __launch_bounds__(128) ray_front_probe(const uint4* __restrict__ vol, int rounds,
                                                       unsigned* __restrict__ sink)
{
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    unsigned acc = 0;
    const int off = (lane * kRun) >> 5;
    for (int r = 0; r < rounds; r++) {
        const uint32_t h = hash32(warp * 7919u + (uint32_t)r * 104729u);
        const int y = (int)(h % kProbeN);
        const int z0 = (int)((h >> 9) % (kProbeZ - kRun));
        // record index <= (N - 1) N Z + (Z - 2) + (kSteps - 1) Z < N N Z
        const uint4* p = vol + ((size_t)y * kProbeN * kProbeZ + z0 + off) * HALVES;
#pragma unroll 4
        for (int k = 0; k < kSteps; k++) {
            const uint4* q = p + (size_t)k * kProbeZ * HALVES;
            const uint4 v = __ldg(q);
            acc += v.x ^ v.y ^ v.z;
            if (HALVES == 2) {
                const uint4 w = __ldg(q + 1);
                acc += w.x ^ w.y;
            }
        }
    }
    if (acc == 0x9e3779b9u) sink[0] = acc;  // keeps the loads; never true for zeroed data
}

constexpr int kTileR = 64, kTileC = 96, kSlices = 16;

template <bool SHARED>
__global__ void __launch_bounds__(256) bp_tile_probe(const float* __restrict__ tiles, int rounds,
                                                     float* __restrict__ sink)
{
    __shared__ float tile[kTileR * kTileC];
    const int t = threadIdx.x;
    float acc = 0.0f;
    const float* g = tiles + (size_t)(blockIdx.x % 64) * kTileR * kTileC;
    if (SHARED) {
        for (int i = t; i < kTileR * kTileC; i += 256) tile[i] = __ldg(g + i);
        __syncthreads();
    }
    const float* src = SHARED ? tile : g;
    for (int r = 0; r < rounds; r++) {
        // voxel column t of the block: column 1.5 t mod the tile, rows 3.1 per slice
        const float u = fmodf(1.5f * (float)(t & 31) + 0.37f * (float)r, (float)(kTileC - 2));
        const int c = (int)u;
        const float wu = u - (float)c;
        const float zr0 = (float)(t >> 5) * 0.7f;
#pragma unroll
        for (int i = 0; i < kSlices; i++) {
            const float zr = zr0 + 3.1f * (float)i;
            const int rr = (int)zr;
            const float wz = zr - (float)rr;
            const float* p = src + rr * kTileC + c;
            const float s0 = fmaf(wu, p[1], (1.0f - wu) * p[0]);
            const float s1 = fmaf(wu, p[kTileC + 1], (1.0f - wu) * p[kTileC]);
            acc = fmaf(wz, s1 - s0, acc + s0);
        }
    }
    if (acc == 1.2345e-30f) sink[0] = acc;
}

char g_msg[256];

int cuda_err(cudaError_t e, const char* what)
{
    std::snprintf(g_msg, sizeof g_msg, "%s: %s", what, cudaGetErrorString(e));
    return 2;
}

}  // namespace

// Message of the last failure (empty after a success).
extern "C" const char* gather_probe_error(void) { return g_msg; }

// Rate of probe `kind` (0 .. 3; units above) on the current device, written
// to *rate.  Returns 0, 1 for a bad argument, 2 for a CUDA failure.
// Synchronous on `stream`; allocates and frees its own buffers.
extern "C" int gather_probe_run(int kind, double* rate, void* stream)
{
    g_msg[0] = 0;
    if (!rate || kind < 0 || kind > 3) {
        std::snprintf(g_msg, sizeof g_msg, "kind must be 0, 1, 2 or 3");
        return 1;
    }
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_err(e, "device query");
    cudaEvent_t e0, e1;
    if ((e = cudaEventCreate(&e0)) != cudaSuccess) return cuda_err(e, "event");
    if ((e = cudaEventCreate(&e1)) != cudaSuccess) {
        cudaEventDestroy(e0);
        return cuda_err(e, "event");
    }
    void* buf = nullptr;
    void* sink = nullptr;
    cudaError_t err = cudaSuccess;
    double units = 0.0;
    float ms = 0.0f;
    if (kind == 0 || kind == 3) {
        const int halves = kind == 3 ? 2 : 1;
        const size_t bytes = (size_t)kProbeN * kProbeN * kProbeZ * sizeof(uint4) * halves;
        err = cudaMalloc(&buf, bytes);
        if (err == cudaSuccess) err = cudaMalloc(&sink, 64);
        if (err == cudaSuccess) err = cudaMemsetAsync(buf, 0, bytes, st);
        const int blocks = sms * 6, rounds = 32;  // 24 warps per SM, as the projector
        if (err == cudaSuccess) {
            auto k = halves == 2 ? ray_front_probe<2> : ray_front_probe<1>;
            k<<<blocks, 128, 0, st>>>((const uint4*)buf, 1, (unsigned*)sink);
            cudaEventRecord(e0, st);
            k<<<blocks, 128, 0, st>>>((const uint4*)buf, rounds, (unsigned*)sink);
            cudaEventRecord(e1, st);
            err = cudaEventSynchronize(e1);
        }
        units = (double)blocks * 128 * rounds * kSteps;
    } else {
        const size_t bytes = (size_t)64 * kTileR * kTileC * sizeof(float);
        err = cudaMalloc(&buf, bytes);
        if (err == cudaSuccess) err = cudaMalloc(&sink, 64);
        if (err == cudaSuccess) err = cudaMemsetAsync(buf, 0, bytes, st);
        const int blocks = sms * 3, rounds = 2000;
        if (err == cudaSuccess) {
            auto k = kind == 1 ? bp_tile_probe<true> : bp_tile_probe<false>;
            k<<<blocks, 256, 0, st>>>((const float*)buf, 1, (float*)sink);
            cudaEventRecord(e0, st);
            k<<<blocks, 256, 0, st>>>((const float*)buf, rounds, (float*)sink);
            cudaEventRecord(e1, st);
            err = cudaEventSynchronize(e1);
        }
        units = (double)blocks * 256 * rounds * kSlices;
    }
    if (err == cudaSuccess) err = cudaGetLastError();
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (buf) cudaFree(buf);
    if (sink) cudaFree(sink);
    if (err != cudaSuccess) return cuda_err(err, "gather probe");
    *rate = units / (ms * 1e-3);
    return 0;
}
