// ramp_gemm.cu -- the FDK ramp filter as a tensor-core GEMM on sm_100a
// (tcgen05 + TMA + TMEM), with a BF16 three-term split for FP32-level accuracy.
//
// filterSinogram (R/filterSinogram.cpp:67-131) is, per view and detector row,
//     out[m] = Cm(m) * sum_k h'[m][k] g[k],   g = -log p,  h' = h + coeff*I,
// i.e. one GEMM  Out[V*H][W] = G[V*H][K] x B[W][K]^T  followed by the cosine
// factor.  Each operand is split x = x0 + x1 + x2 into bfloat16 parts
// (x0 = bf16(x), x1 = bf16(x - x0), x2 = bf16(x - x0 - x1)); the six products
// with i + j <= 2 (G0B0 G0B1 G1B0 G0B2 G1B1 G2B0) are accumulated in FP32 in
// tensor memory, which keeps about 24 significant bits.
//
// One CTA computes a 128-row x NT-column output tile (NT <= 512; wider
// detectors take several column tiles): warp 0 issues
// TMA loads into a 3-stage shared-memory ring (128B swizzle, K-major), warp 1
// issues tcgen05.mma from a single thread into a 128 x NT FP32 accumulator in
// tensor memory, warps 2-5 read the accumulator back (tcgen05.ld), apply the
// cosine factor and store.  No cluster multicast is used.  Every mbarrier
// wait is bounded; on timeout the kernel raises a device flag and returns.
#include <cuda.h>
#include <cuda_bf16.h>

#include "internal.h"

namespace vcbct {
namespace {

constexpr int BM = 128;           // rows per CTA tile (UMMA M)
constexpr int BK = 64;            // K per stage: 64 bf16 = one 128-byte swizzle row
constexpr int kThreads = 192;     // 6 warps
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 1.9 GHz

// (a-plane, b-plane) of the six split products, smallest terms first
__constant__ int c_terms[6][2] = {{2, 0}, {1, 1}, {0, 2}, {1, 0}, {0, 1}, {0, 0}};

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// Bounded wait on an mbarrier phase; false (and the error flag) on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, int* err)
{
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, phase)) {
        if (clock64() - t0 > kWaitCycles) {
            atomicExch(err, 1);
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0,
                                            int c1, int c2)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

// Shared-memory matrix descriptor of a K-major tile with 128-byte swizzle:
// rows of 128 B, 8-row atoms 1024 B apart (stride byte offset), start address
// advanced by 32 B per K=16 slice inside the atom.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);  // start address [0,14)
    d |= (uint64_t)1 << 16;                   // leading byte offset (unused, swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;         // stride byte offset [32,46)
    d |= (uint64_t)1 << 46;                   // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;                   // layout: 128-byte swizzle
    return d;
}

// Instruction descriptor, kind::f16: BF16 x BF16 -> F32, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v)
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

struct GemmArgs {
    float* out;
    const FilterView* views;
    float pitch, sad;
    int M, H, W, NT, Kp, ktiles, stages;  // NT: output columns per CTA (blockIdx.y selects the column tile)
    int vec;                              // rows of `out` 16-byte aligned (W % 4 == 0, aligned base)
    int* err;
};

__global__ void __launch_bounds__(kThreads, 1)
ramp_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, GemmArgs g)
{
    extern __shared__ uint8_t smem_raw[];
    // 1024-byte alignment for the 128-byte swizzle atoms
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int S = g.stages;
    const uint32_t a_bytes = BM * BK * 2;
    const uint32_t b_bytes = (uint32_t)g.NT * BK * 2;
    uint8_t* stage_base = smem;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + (size_t)S * (a_bytes + b_bytes));
    uint64_t* full = bars;
    uint64_t* empty = bars + S;
    uint64_t* accum = bars + 2 * S;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * S + 1);

    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int m0 = blockIdx.x * BM;
    const int n0 = blockIdx.y * g.NT;
    const int N1 = g.NT < 256 ? g.NT : 256;
    const int N2 = g.NT - N1;
    const int nk = 6 * g.ktiles;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(accum, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t taddr = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // TMA producer
        for (int kb = 0; kb < nk; kb++) {
            const int s = kb % S;
            if (kb >= S && !mbar_wait(&empty[s], ((kb / S) - 1) & 1, g.err)) break;
            const int term = kb / g.ktiles, kt = kb % g.ktiles;
            uint8_t* sa = stage_base + (size_t)s * (a_bytes + b_bytes);
            uint8_t* sb = sa + a_bytes;
            mbar_expect_tx(&full[s], a_bytes + b_bytes);
            tma_load_3d(sa, &tmA, &full[s], kt * BK, m0, c_terms[term][0]);
            tma_load_3d(sb, &tmB, &full[s], kt * BK, n0, c_terms[term][1]);
            tma_load_3d(sb + (size_t)(g.NT / 2) * BK * 2, &tmB, &full[s], kt * BK, n0 + g.NT / 2, c_terms[term][1]);
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer
        const uint32_t id1 = idesc_bf16(BM, N1);
        const uint32_t id2 = idesc_bf16(BM, N2 > 0 ? N2 : 16);
        bool ok = true;
        for (int kb = 0; kb < nk && ok; kb++) {
            const int s = kb % S;
            ok = mbar_wait(&full[s], (kb / S) & 1, g.err);
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t sa = smem_u32(stage_base + (size_t)s * (a_bytes + b_bytes));
            const uint32_t sb = sa + a_bytes;
#pragma unroll
            for (int kk = 0; kk < BK / 16; kk++) {
                const uint64_t ad = sw128_desc(sa + kk * 32);
                const uint32_t acc = (kb > 0 || kk > 0) ? 1u : 0u;
                umma_bf16(taddr, ad, sw128_desc(sb + kk * 32), id1, acc);
                if (N2 > 0) umma_bf16(taddr + (uint32_t)N1, ad, sw128_desc(sb + N1 * 128 + kk * 32), id2, acc);
            }
            umma_commit(&empty[s]);
        }
        umma_commit(accum);
    } else if (warp >= 2) {
        // epilogue: TMEM -> registers -> cosine factor -> global
        const int q = warp % 4;  // TMEM lane quarter this warp may access
        const int row = m0 + 32 * q + lane;
        // warp-uniform outcome: tcgen05.ld needs the whole warp converged
        const bool ready = __all_sync(0xffffffffu, mbar_wait(accum, 0, g.err));
        if (ready) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            float pos2 = 0.0f, xcs = 0.0f;
            if (row < g.M) {
                const int v = row / g.H, n = row - v * g.H;
                const FilterView fv = g.views[v];
                pos2 = fabsf(fv.ycs + (float)n) * g.pitch;
                xcs = fv.xcs;
            }
            // cosine factor sad / sqrt(sad^2 + pos1^2 + pos2^2) from the
            // reciprocal square root (2 ulp), stored 16 bytes at a time
            const float sad = g.sad, base2 = fmaf(pos2, pos2, sad * sad);
            for (int c = 0; c < g.NT; c += 32) {
                float v32[32];
                tmem_ld32(taddr + ((uint32_t)(32 * q) << 16) + (uint32_t)c, v32);
                const int mb = n0 + c;
                if (row < g.M && mb < g.W) {
                    float* o = g.out + (size_t)row * g.W + mb;
#pragma unroll
                    for (int i = 0; i < 32; i++) {
                        const float pos1 = fabsf(xcs + (float)(mb + i)) * g.pitch;
                        v32[i] *= sad * rsqrtf(fmaf(pos1, pos1, base2));
                    }
                    // columns of this tile only (the last 32-column chunk may
                    // run past NT into unwritten accumulator columns)
                    const int lim = min(g.W - mb, g.NT - c);
                    if (g.vec && lim >= 32) {
#pragma unroll
                        for (int i = 0; i < 32; i += 4)
                            *reinterpret_cast<float4*>(o + i) = make_float4(v32[i], v32[i + 1], v32[i + 2], v32[i + 3]);
                    } else {
#pragma unroll
                        for (int i = 0; i < 32; i++)
                            if (i < lim) o[i] = v32[i];
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(512));
    }
}

// x = x0 + x1 + x2 in bfloat16 (round to nearest even at each step).
__device__ __forceinline__ void split3(float x, __nv_bfloat16& a, __nv_bfloat16& b, __nv_bfloat16& c)
{
    a = __float2bfloat16_rn(x);
    const float r1 = x - __bfloat162float(a);
    b = __float2bfloat16_rn(r1);
    const float r2 = r1 - __bfloat162float(b);
    c = __float2bfloat16_rn(r2);
}

// A planes [3][M][Kp]: split of g = -logf(p) (times the redundancy weight).
// grid (M, ceil(Kp / 512)), block 128: one detector row per block, four
// consecutive columns per thread, written as 8-byte groups (Kp is a multiple
// of 64, so every group is aligned).
__global__ void split_a_kernel(const float* __restrict__ proj, const float* __restrict__ wts, int M, int H, int W,
                               int Kp, __nv_bfloat16* __restrict__ planes)
{
    const int r = blockIdx.x;
    const int k0 = 4 * (blockIdx.y * blockDim.x + threadIdx.x);
    if (k0 >= Kp) return;
    const float* pr = proj + (size_t)r * W;
    const float* wr = wts ? wts + (size_t)(r / H) * W : nullptr;
    __align__(8) __nv_bfloat16 a[4], b[4], c[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int k = k0 + q;
        float g = 0.0f;
        if (k < W) {
            g = -logf(__ldg(pr + k));
            if (wr) g *= __ldg(wr + k);
        }
        split3(g, a[q], b[q], c[q]);
    }
    const size_t plane = (size_t)M * Kp, o = (size_t)r * Kp + k0;
    *reinterpret_cast<uint2*>(planes + o) = *reinterpret_cast<const uint2*>(a);
    *reinterpret_cast<uint2*>(planes + plane + o) = *reinterpret_cast<const uint2*>(b);
    *reinterpret_cast<uint2*>(planes + 2 * plane + o) = *reinterpret_cast<const uint2*>(c);
}

// B planes [3][Np][Kp]: B[m][k] = hT[k][m] (ramp kernel + diagonal coefficient).
__global__ void split_b_kernel(const float* __restrict__ hT, int W, int Np, int Kp, __nv_bfloat16* __restrict__ planes)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)Np * Kp) return;
    const int m = (int)(i / Kp), k = (int)(i % Kp);
    const float x = (m < W && k < W) ? hT[(size_t)k * W + m] : 0.0f;
    __nv_bfloat16 a, b, c;
    split3(x, a, b, c);
    const size_t plane = (size_t)Np * Kp;
    planes[i] = a;
    planes[plane + i] = b;
    planes[2 * plane + i] = c;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// 3D bf16 tensor [planes][rows][Kp] with box {64, box_rows, 1}, 128-byte swizzle.
bool make_map(CUtensorMap* map, void* base, int rows, int Kp, int box_rows)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[3] = {(cuuint64_t)Kp, (cuuint64_t)rows, 3};
    cuuint64_t strides[2] = {(cuuint64_t)Kp * 2, (cuuint64_t)rows * Kp * 2};
    cuuint32_t box[3] = {(cuuint32_t)BK, (cuuint32_t)box_rows, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, base, dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Output columns are split into ntiles tiles of NT <= 512 columns (one
// tensor-memory accumulator of 128 x NT FP32 each); B is padded to
// Np = ntiles * NT rows.
struct Layout {
    int M, Np, NT, ntiles, Kp, stages;
    size_t a_off, b_off, err_off, total, smem;
};

Layout layout_for(int V, int H, int W)
{
    Layout L{};
    L.M = V * H;
    const int n16 = (W + 15) / 16 * 16;
    L.ntiles = (n16 + 511) / 512;
    L.NT = ((n16 + L.ntiles - 1) / L.ntiles + 15) / 16 * 16;
    L.Np = L.ntiles * L.NT;
    L.Kp = (W + BK - 1) / BK * BK;
    const size_t stage = (size_t)BM * BK * 2 + (size_t)L.NT * BK * 2;
    L.stages = (int)((225 * 1024 - 1024 - 128) / stage);
    if (L.stages > 3) L.stages = 3;
    L.smem = 1024 + (size_t)L.stages * stage + 8 * (2 * L.stages + 1) + 16;
    L.a_off = 0;
    L.b_off = (3 * (size_t)L.M * L.Kp * 2 + 1023) / 1024 * 1024;
    L.err_off = L.b_off + (3 * (size_t)L.Np * L.Kp * 2 + 1023) / 1024 * 1024;
    L.total = L.err_off + 256;
    return L;
}

}  // namespace

size_t ramp_gemm_workspace_bytes(int V, int H, int W) { return layout_for(V, H, W).total; }

cudaError_t launch_ramp_gemm_bf16x3(const float* proj, float* out, const float* hT, const FilterView* views,
                                    const float* wts, float pitch, float sad, int V, int H, int W, void* workspace,
                                    cudaStream_t st)
{
    if (W < 16 || W > 4096) return cudaErrorInvalidValue;
    const Layout L = layout_for(V, H, W);
    if (L.stages < 2) return cudaErrorInvalidValue;
    uint8_t* ws = static_cast<uint8_t*>(workspace);
    __nv_bfloat16* ap = reinterpret_cast<__nv_bfloat16*>(ws + L.a_off);
    __nv_bfloat16* bp = reinterpret_cast<__nv_bfloat16*>(ws + L.b_off);
    int* err = reinterpret_cast<int*>(ws + L.err_off);
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    {
        split_a_kernel<<<dim3((unsigned)L.M, (unsigned)((L.Kp + 511) / 512)), 128, 0, st>>>(proj, wts, L.M, H, W,
                                                                                         L.Kp, ap);
        const size_t nb = (size_t)L.Np * L.Kp;
        split_b_kernel<<<(unsigned)((nb + 255) / 256), 256, 0, st>>>(hT, W, L.Np, L.Kp, bp);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    CUtensorMap tmA, tmB;
    if (!make_map(&tmA, ap, L.M, L.Kp, BM) || !make_map(&tmB, bp, L.Np, L.Kp, L.NT / 2))
        return cudaErrorInvalidValue;
    const int vec = (W % 4 == 0 && (reinterpret_cast<uintptr_t>(out) & 15) == 0) ? 1 : 0;
    GemmArgs g{out, views, pitch, sad, L.M, H, W, L.NT, L.Kp, L.Kp / BK, L.stages, vec, err};
    e = cudaFuncSetAttribute(ramp_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem);
    if (e != cudaSuccess) return e;
    ramp_gemm_kernel<<<dim3((L.M + BM - 1) / BM, L.ntiles), kThreads, L.smem, st>>>(tmA, tmB, g);
    return cudaGetLastError();
}

int ramp_gemm_error_flag(void* workspace, int V, int H, int W, cudaStream_t st)
{
    const Layout L = layout_for(V, H, W);
    int h = 0;
    if (cudaMemcpyAsync(&h, static_cast<uint8_t*>(workspace) + L.err_off, sizeof(int), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return -1;
    return h;
}

}  // namespace vcbct
