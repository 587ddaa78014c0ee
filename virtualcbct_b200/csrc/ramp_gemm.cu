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
// One CTA computes a 128-row x NT-column output tile (NT <= 512, a multiple
// of 32; wider detectors take several column tiles), K tile by K tile.  The
// split Toeplitz planes (B) are made once per kernel.  In the GEMM, warp 0
// streams by TMA, per K tile, the A operand and then B planes 2, 1, 0, each
// as two column halves (a ring of 3 or 4 stages), so each B plane of a K tile
// is loaded once and multiplied by every A plane it pairs with; warp 1 issues
// tcgen05.mma from a single thread into two 128 x NT/2 FP32 accumulators in
// tensor memory (columns 0 and 256); warps 2-17 read them back (tcgen05.ld),
// apply the cosine factor and store.  Each K tile is multiplied column half 0
// first, so after the last one the warps of half 0 start their epilogue while
// half 1's MMAs still run.
//
// The A operand, fused form (rows of p 16-byte aligned): warp 0 stages the
// 128 x 64 FP32 tile of p in shared memory and warps 2-17, idle until the
// epilogue, turn it into the three swizzled bf16 planes of -ln p in a
// 2-stage ring -- p is read from HBM once and no split copy is written.
// Unfused form (other widths): split_a_kernel first writes the three A planes
// to global memory and warp 0 loads them by TMA.
//
// No cluster multicast is used.  Every mbarrier wait is bounded; on timeout
// the kernel raises a device flag, stops issuing, waits (bounded) for its
// loads in flight and returns; its output is then invalid.
#include <cuda.h>
#include <cuda_bf16.h>

#include "async_copy.cuh"
#include "internal.h"

namespace vcbct {
namespace {

using namespace async_copy;

constexpr int BM = 128;           // rows per CTA tile (UMMA M)
constexpr int BK = 64;            // K per stage: 64 bf16 = one 128-byte swizzle row
constexpr int kThreads = 576;     // 18 warps

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

// x = x0 + x1 + x2 in bfloat16 (round to nearest even at each step).
__device__ __forceinline__ void split3(float x, __nv_bfloat16& a, __nv_bfloat16& b, __nv_bfloat16& c)
{
    a = __float2bfloat16_rn(x);
    const float r1 = x - __bfloat162float(a);
    b = __float2bfloat16_rn(r1);
    const float r2 = r1 - __bfloat162float(b);
    c = __float2bfloat16_rn(r2);
}

// The same split of two values at once, each plane packed as bf16x2 (low
// half = first value): one cvt.rn.bf16x2.f32 per plane and a packed f32x2
// subtraction per residual, each element rounded exactly as split3 rounds it.
__device__ __forceinline__ uint32_t bf16x2_rn(float lo, float hi)
{
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}
__device__ __forceinline__ unsigned long long bf16x2_widen(uint32_t v)  // -> {lo, hi} as f32x2
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "r"(v << 16), "r"(v & 0xffff0000u));
    return r;
}
__device__ __forceinline__ unsigned long long fsub2(unsigned long long a, unsigned long long b)
{
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ void split3x2(float x, float y, uint32_t& p0, uint32_t& p1, uint32_t& p2)
{
    unsigned long long v;
    asm("mov.b64 %0, {%1, %2};" : "=l"(v) : "f"(x), "f"(y));
    p0 = bf16x2_rn(x, y);
    const unsigned long long r1 = fsub2(v, bf16x2_widen(p0));
    float r1x, r1y;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r1x), "=f"(r1y) : "l"(r1));
    p1 = bf16x2_rn(r1x, r1y);
    const unsigned long long r2 = fsub2(r1, bf16x2_widen(p1));
    float r2x, r2y;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r2x), "=f"(r2y) : "l"(r2));
    p2 = bf16x2_rn(r2x, r2y);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// The same load without its wait, and the wait as a use of the registers it
// fills (so that no read of them is scheduled before it): the next chunk's
// load overlaps the current chunk's arithmetic.
__device__ __forceinline__ void tmem_ld16_async(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld(uint32_t (&r)[16])
{
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])
                 :
                 : "memory");
}

struct GemmArgs {
    float* out;
    const FilterView* views;
    const float* wts;             // fused form: optional redundancy weights [V][W] (multiply -ln p)
    float pitch, sad;
    int M, H, W, NT, Kp, ktiles;  // NT: output columns per CTA (blockIdx.y selects the column tile)
    int vec;                      // rows of `out` 16-byte aligned (W % 4 == 0, aligned base)
    int* err;
};

constexpr int kEpiWarps = 16;                   // warps 2-17: A planes (fused form), then the epilogue
static_assert(kThreads == 64 + 32 * kEpiWarps, "warp 0 TMA, warp 1 MMA, the rest A planes / epilogue");
constexpr uint32_t kHalfCol = 256;              // TMEM column of the second column half
constexpr int kAStages = 2;                     // A ring: the three planes of one K tile each
constexpr uint32_t kAPlaneBytes = BM * BK * 2;  // one 128 x 64 bf16 plane, 16 KiB
constexpr uint32_t kAStageBytes = 3 * kAPlaneBytes;
// the fused epilogue stages 8 warps x 2 x 2 KB per column half in one A stage
static_assert(kAStages == 2 && 8 * 4096 <= kAStageBytes, "epilogue staging in the A ring");
constexpr uint32_t kPTileBytes = BM * BK * 4;   // fused form: one 128 x 64 FP32 tile of p, 32 KiB

// B ring stages (one column half of one plane of one K tile each): the fused
// form gives up one to hold the FP32 tile of p.
__host__ __device__ constexpr int b_stages(bool fused) { return fused ? 3 : 4; }

// Shared-memory footprint of a CTA with NT output columns (before 1 KiB
// alignment slack): [p tile], A ring, B ring of NT/2-row halves, mbarriers,
// TMEM slot.
__host__ __device__ constexpr size_t gemm_smem_bytes(int NT, bool fused)
{
    return (fused ? (size_t)kPTileBytes : 0) + (size_t)kAStages * kAStageBytes +
           (size_t)b_stages(fused) * (NT / 2) * BK * 2 + 8 * (2 + 2 * kAStages + 2 * b_stages(fused) + 2) + 16;
}

// Shared -> global tensor store of one box (clipped at the tensor's edges),
// tracked as a bulk group of the issuing thread.
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, const void* src, int c0, int c1)
{
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(map),
                 "r"(smem_u32(src)), "r"(c0), "r"(c1)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// this thread's bulk groups but the newest one have finished reading shared memory
__device__ __forceinline__ void bulk_wait_read_all_but_one()
{
    asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
}
// all of this thread's bulk groups are complete
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void st_shared_v4(uint32_t addr, float a, float b, float c, float d)
{
    asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(a), "f"(b), "f"(c), "f"(d) : "memory");
}

__device__ __forceinline__ void st_shared_u32(uint32_t addr, uint32_t v)
{
    asm volatile("st.shared.b32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}

__device__ __forceinline__ float2 ld_shared_f2(uint32_t addr)
{
    float2 v;
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr) : "memory");
    return v;
}

// Fused form: one K tile of the A operand made in shared memory from the
// FP32 tile of p the TMA thread has staged (row r at r * 256 bytes; rows
// beyond M and columns beyond W read as 0 and are skipped): g = -ln(p)
// (times the redundancy weight), split into three bf16 planes, each stored as
// the 128-byte-swizzled K-major tile a TMA load with
// CU_TENSOR_MAP_SWIZZLE_128B would write (row r at r * 128 bytes, the 16-byte
// chunk index XOR r % 8; buffers 1024-byte aligned).  Producer warp w makes
// rows R w .. R w + R - 1 (R = BM / kEpiWarps = 8), lane l the columns
// kt * 64 + 2 l, + 1 of each: one 8-byte shared load and one 4-byte store per
// plane, conflict-free.  Redundancy weights: with wfast (H >= R) the warp's
// rows hold at most two views, whose weights the caller has loaded (wa before
// CTA row rsplit, wb from it on); otherwise each row loads its own.
__device__ __forceinline__ void convert_a_tile(const GemmArgs& g, int m0, int kt, int pw, int lane,
                                               uint32_t ptile, uint32_t abuf, bool wfast, int rsplit, float2 wa,
                                               float2 wb)
{
    const int k = kt * BK + 2 * lane;
    const bool in0 = k < g.W, in1 = k + 1 < g.W;
#pragma unroll 4
    for (int rr = 0; rr < BM / kEpiWarps; rr++) {
        const int r = pw * (BM / kEpiWarps) + rr;
        const int row = m0 + r;
        const float2 pv = ld_shared_f2(ptile + (uint32_t)r * (BK * 4) + (uint32_t)lane * 8u);
        float x = 0.0f, y = 0.0f;
        if (row < g.M) {
            // -ln p from the hardware base-2 logarithm (relative error ~2^-22;
            // the split keeps ~24 bits, the filter's bar is 1e-5 of its scale)
            if (in0) x = __log2f(pv.x) * -0.693147180559945309f;
            if (in1) y = __log2f(pv.y) * -0.693147180559945309f;
            if (g.wts && in0) {
                float2 w = r < rsplit ? wa : wb;
                if (!wfast) {
                    const float* wr = g.wts + (size_t)(row / g.H) * g.W + k;
                    w = make_float2(__ldg(wr), in1 ? __ldg(wr + 1) : 1.0f);
                }
                x *= w.x;
                y *= w.y;
            }
        }
        uint32_t q0, q1, q2;
        split3x2(x, y, q0, q1, q2);
        const uint32_t off = (uint32_t)r * 128u + (uint32_t)lane * 4u;
        const uint32_t sw = off ^ (((off >> 7) & 7u) << 4);
        st_shared_u32(abuf + sw, q0);
        st_shared_u32(abuf + kAPlaneBytes + sw, q1);
        st_shared_u32(abuf + 2 * kAPlaneBytes + sw, q2);
    }
}

// Warp-uniform bounded wait (tcgen05.ld needs converged warps).
__device__ __forceinline__ bool warp_wait(uint64_t* bar, uint32_t phase, int* err)
{
    return __all_sync(0xffffffffu, mbar_wait(bar, phase, err));
}

template <bool FUSED>
__global__ void __launch_bounds__(kThreads, 1)
ramp_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                 const __grid_constant__ CUtensorMap tmO, GemmArgs g)
{
    constexpr int SB = b_stages(FUSED);
    extern __shared__ uint8_t smem_raw[];
    // 1024-byte alignment for the 128-byte swizzle atoms
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int NH = g.NT / 2;                      // columns of one B half (a multiple of 16)
    const uint32_t bh_bytes = (uint32_t)NH * BK * 2;
    uint8_t* ptile = smem;                        // fused form: the FP32 tile of p
    uint8_t* abuf = smem + (FUSED ? kPTileBytes : 0);   // kAStages x 3 planes
    uint8_t* bbuf = abuf + kAStages * kAStageBytes;    // SB x one B half
    uint64_t* bars = reinterpret_cast<uint64_t*>(bbuf + (size_t)SB * bh_bytes);
    uint64_t* p_full = bars;                      // fused form: TMA bytes of the p tile
    uint64_t* p_empty = bars + 1;                 // fused form: the converter warps are done reading it
    uint64_t* a_full = bars + 2;
    uint64_t* a_empty = bars + 2 + kAStages;
    uint64_t* b_full = bars + 2 + 2 * kAStages;
    uint64_t* b_empty = bars + 2 + 2 * kAStages + SB;
    uint64_t* accum = bars + 2 + 2 * kAStages + 2 * SB;  // every MMA of the tile done
    uint64_t* accum0 = accum + 1;                        // those of column half 0 done
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accum0 + 1);

    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int m0 = blockIdx.x * BM;
    const int n0 = blockIdx.y * g.NT;

    if (threadIdx.x == 0) {
        mbar_init(p_full, 1);
        mbar_init(p_empty, kEpiWarps);
        for (int s = 0; s < kAStages; s++) {
            mbar_init(&a_full[s], FUSED ? kEpiWarps : 1);
            mbar_init(&a_empty[s], 1);
        }
        for (int s = 0; s < SB; s++) {
            mbar_init(&b_full[s], 1);
            mbar_init(&b_empty[s], 1);
        }
        mbar_init(accum, 1);
        mbar_init(accum0, 1);
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
        // TMA producer.  Per K tile: the A operand (fused form: the FP32 tile
        // of p; otherwise the three split A planes, one A stage), then column
        // half 0 of B planes 2, 1, 0 and half 1 of the same (six B stages) --
        // the order the consumers take them in.  Fused form: p tile n + 1 is
        // requested as soon as the converters have released tile n, polled
        // while the thread waits for B ring stages.
        int na = 0, nb = 0;  // stages (fused form: p tiles) issued
        bool ok = true;
        auto issue_p = [&]() {
            mbar_expect_tx(p_full, kPTileBytes);
            tma_load_2d(ptile, &tmA, p_full, na * BK, m0);
            na++;
        };
        if (FUSED) issue_p();
        for (int kt = 0; kt < g.ktiles && ok; kt++) {
            if (!FUSED) {
                const int sa = kt % kAStages;
                if (kt >= kAStages && !(ok = mbar_wait(&a_empty[sa], ((kt / kAStages) - 1) & 1, g.err))) break;
                uint8_t* da = abuf + (size_t)sa * kAStageBytes;
                mbar_expect_tx(&a_full[sa], kAStageBytes);
                for (int i = 0; i < 3; i++) tma_load_3d(da + i * kAPlaneBytes, &tmA, &a_full[sa], kt * BK, m0, i);
                na = kt + 1;
            }
            for (int q = 0; q < 6 && ok; q++) {
                const int kb = kt * 6 + q, s = kb % SB;
                if (kb >= SB) {
                    // bounded wait for the stage, serving the p tiles meanwhile
                    const uint32_t ph = ((kb / SB) - 1) & 1;
                    const long long t0 = clock64();
                    while (!mbar_try_wait(&b_empty[s], ph)) {
                        if (FUSED && na < g.ktiles && mbar_try_wait(p_empty, (na - 1) & 1)) issue_p();
                        if (clock64() - t0 > kWaitCycles) {
                            atomicExch(g.err, 1);
                            ok = false;
                            break;
                        }
                    }
                    if (!ok) break;
                }
                if (FUSED && na < g.ktiles && mbar_try_wait(p_empty, (na - 1) & 1)) issue_p();
                const int plane = 2 - q % 3, h = q / 3;
                mbar_expect_tx(&b_full[s], bh_bytes);
                tma_load_3d(bbuf + (size_t)s * bh_bytes, &tmB, &b_full[s], kt * BK, n0 + h * NH, plane);
                nb = kb + 1;
            }
        }
        // p tiles not yet requested when the last B stage went out
        while (FUSED && ok && na < g.ktiles) {
            if (!(ok = mbar_wait(p_empty, (na - 1) & 1, g.err))) break;
            issue_p();
        }
        // no load may still be in flight into this CTA's shared memory when it
        // exits: wait (bounded) for the last stages issued
        if (FUSED) {
            if (na > 0) mbar_wait(p_full, (na - 1) & 1, g.err);
        } else {
            for (int k = na - kAStages; k < na; k++)
                if (k >= 0) mbar_wait(&a_full[k % kAStages], (k / kAStages) & 1, g.err);
        }
        for (int k = nb - SB; k < nb; k++)
            if (k >= 0) mbar_wait(&b_full[k % SB], (k / SB) & 1, g.err);
    } else if (warp == 1 && lane == 0) {
        // MMA issuer: per K tile, column half 0 then 1, and per half B plane
        // j against A planes 2 - j .. 0, so the products (2,0) (1,1) (0,2)
        // (1,0) (0,1) (0,0) are all formed, smaller terms of a tile before
        // larger ones.  Half 0 of the last K tile is committed on its own, so
        // its epilogue starts while half 1's last MMAs run.
        const uint32_t idesc = idesc_bf16(BM, NH);
        bool ok = true, fresh[2] = {true, true}, half0 = false;
        for (int kt = 0; kt < g.ktiles && ok; kt++) {
            const int sa = kt % kAStages;
            if (!(ok = mbar_wait(&a_full[sa], (kt / kAStages) & 1, g.err))) break;
            const uint32_t abase = smem_u32(abuf + (size_t)sa * kAStageBytes);
            for (int q = 0; q < 6 && ok; q++) {
                const int kb = kt * 6 + q, s = kb % SB;
                if (!(ok = mbar_wait(&b_full[s], (kb / SB) & 1, g.err))) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const int j = 2 - q % 3, h = q / 3;
                const uint32_t sb = smem_u32(bbuf + (size_t)s * bh_bytes);
                const uint32_t dcol = taddr + (uint32_t)h * kHalfCol;
                for (int i = 2 - j; i >= 0; i--) {
                    const uint32_t sai = abase + (uint32_t)i * kAPlaneBytes;
#pragma unroll
                    for (int kk = 0; kk < BK / 16; kk++) {
                        umma_bf16(dcol, sw128_desc(sai + kk * 32), sw128_desc(sb + kk * 32), idesc, fresh[h] ? 0u : 1u);
                        fresh[h] = false;
                    }
                }
                umma_commit(&b_empty[s]);
                if (q == 2 && kt == g.ktiles - 1) {
                    umma_commit(accum0);
                    half0 = true;
                }
            }
            umma_commit(&a_empty[sa]);
        }
        if (!half0) umma_commit(accum0);  // (an error path: the waiters see the flag)
        umma_commit(accum);
    } else if (warp >= 2) {
        bool ok = true;
        if (FUSED) {
            // the A planes of every K tile from the staged p tile,
            // double-buffered against the MMAs
            const int pw = warp - 2;
            // the warp's rows m0 + 8 pw .. + 7 lie in views va and (from CTA
            // row rsplit on) va + 1 when H >= 8
            const int rw = m0 + pw * (BM / kEpiWarps);
            const bool wfast = g.wts != nullptr && g.H >= BM / kEpiWarps;
            const int va = rw / g.H;
            const int rsplit = (va + 1) * g.H - m0;
            const bool has_a = rw < g.M;
            const bool has_b = rsplit < pw * (BM / kEpiWarps) + BM / kEpiWarps && m0 + rsplit < g.M;
            for (int kt = 0; kt < g.ktiles; kt++) {
                const int sa = kt % kAStages;
                // this tile's weights, loaded before the waits so that their
                // latency passes while the p tile arrives
                float2 wa = make_float2(1.0f, 1.0f), wb = wa;
                const int k = kt * BK + 2 * lane;
                if (wfast && k < g.W) {
                    const bool in1 = k + 1 < g.W;
                    if (has_a) {
                        const float* wr = g.wts + (size_t)va * g.W + k;
                        wa = make_float2(__ldg(wr), in1 ? __ldg(wr + 1) : 1.0f);
                    }
                    if (has_b) {
                        const float* wr = g.wts + (size_t)(va + 1) * g.W + k;
                        wb = make_float2(__ldg(wr), in1 ? __ldg(wr + 1) : 1.0f);
                    }
                }
                if (!(ok = warp_wait(p_full, kt & 1, g.err))) break;
                if (kt >= kAStages && !(ok = warp_wait(&a_empty[sa], ((kt / kAStages) - 1) & 1, g.err))) break;
                convert_a_tile(g, m0, kt, pw, lane, smem_u32(ptile), smem_u32(abuf + (size_t)sa * kAStageBytes),
                               wfast, rsplit, wa, wb);
                // generic-proxy stores -> visible to the tensor core (async proxy)
                fence_proxy_async();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(p_empty);
                    mbar_arrive(&a_full[sa]);
                }
            }
        }
        // epilogue: TMEM -> registers -> cosine factor -> global; four warps
        // per TMEM lane quarter (a warp may access lanes 32 (warp % 4) ..),
        // grp = (warp - 2) / 4 choosing the column half (grp / 2) and every
        // other 16-column chunk of it (grp % 2); logical column c lies at
        // TMEM column c (first half) or kHalfCol + c - NT/2 (second half)
        const int q = warp % 4;
        const int grp = (warp - 2) / 4;
        const int half = grp >> 1, part = grp & 1;
        const int row = m0 + 32 * q + lane;
        if (ok && warp_wait(half ? accum : accum0, 0, g.err)) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            float pos2 = 0.0f, xcs = 0.0f;
            if (row < g.M) {
                const int v = row / g.H, n = row - v * g.H;
                const FilterView fv = g.views[v];
                pos2 = fabsf(fv.ycs + (float)n) * g.pitch;
                xcs = fv.xcs;
            }
            // cosine factor sad / sqrt(sad^2 + pos1^2 + pos2^2) from the
            // reciprocal square root (2 ulp)
            const float sad = g.sad, base2 = fmaf(pos2, pos2, sad * sad);
            if (FUSED) {
                // Warp (q, half, part) drains TMEM lane quarter q of column
                // half `half` (the logical columns half NH .. half NH + NH -
                // 1), the 16-column chunks part, part + 2, ..., the next
                // chunk's load in flight while this one is scaled and stored.
                // Each 32-row x 16-column chunk goes through a 2 KB staging
                // buffer (two per warp, in the A ring) in the layout of a
                // CU_TENSOR_MAP_SWIZZLE_64B box (row r at 64 r bytes, 16-byte
                // chunk j at j ^ ((r >> 1) & 3): conflict-free vector stores),
                // and one TMA store writes it whole: full sectors, rows and
                // columns past the detector clipped, instead of 32 rows
                // touched by every warp store.
                // half 0 drains while half 1's last MMAs still read the A
                // stage of the last K tile: its warps stage in the other A
                // stage (its K tile's MMAs have completed), half 1's in that
                // last stage once every MMA is done; 8 warps x 4 KB each
                const int last_sa = (g.ktiles - 1) % kAStages;
                const int ssel = half ? last_sa : kAStages - 1 - last_sa;
                uint8_t* stage = abuf + (size_t)ssel * kAStageBytes + (size_t)((warp - 2) % 8) * 4096;
                const int r0 = m0 + 32 * q;
                const uint32_t tq = taddr + ((uint32_t)(32 * q) << 16) + (uint32_t)half * kHalfCol;
                const int nch = NH / 16;
                int nst = 0;
                uint32_t cur[16], nxt[16];
                if (part < nch) {
                    tmem_ld16_async(tq + 16u * (uint32_t)part, cur);
                    tmem_wait_ld(cur);
                }
                for (int i = part; i < nch; i += 2) {
                    if (i + 2 < nch) tmem_ld16_async(tq + 16u * (uint32_t)(i + 2), nxt);
                    const int mb = n0 + half * NH + 16 * i;
                    if (mb < g.W && r0 < g.M) {  // else the whole box lies past the detector
                        float v16[16];
                        const float fmb = (float)mb;  // + j exactly: column indices are far below 2^24
#pragma unroll
                        for (int j = 0; j < 16; j++) {
                            const float pos1 = fabsf(xcs + (fmb + (float)j)) * g.pitch;
                            v16[j] = __uint_as_float(cur[j]) * (sad * rsqrtf(fmaf(pos1, pos1, base2)));
                        }
                        uint8_t* buf = stage + (nst & 1) * 2048;
                        if (nst >= 2) {
                            // the store issued from this buffer two chunks ago has read it
                            if (lane == 0) bulk_wait_read_all_but_one();
                            __syncwarp();
                        }
                        const uint32_t rb = smem_u32(buf) + (uint32_t)lane * 64u;
                        const uint32_t sw = ((uint32_t)lane >> 1) & 3u;
#pragma unroll
                        for (int j = 0; j < 4; j++)
                            st_shared_v4(rb + ((j ^ sw) << 4), v16[4 * j], v16[4 * j + 1], v16[4 * j + 2],
                                         v16[4 * j + 3]);
                        fence_proxy_async();
                        __syncwarp();
                        if (lane == 0) {
                            tma_store_2d(&tmO, buf, mb, r0);
                            bulk_commit();
                        }
                        nst++;
                    }
                    if (i + 2 < nch) {
                        tmem_wait_ld(nxt);
#pragma unroll
                        for (int j = 0; j < 16; j++) cur[j] = nxt[j];
                    }
                }
                // the stores are complete (and their buffers read) before exit
                if (lane == 0) bulk_wait_all();
            } else {
                // stored 16 bytes at a time
                for (int c = 16 * grp; c < g.NT; c += 64) {
                    float v16[16];
                    const uint32_t col = c < NH ? (uint32_t)c : kHalfCol + (uint32_t)(c - NH);
                    tmem_ld16(taddr + ((uint32_t)(32 * q) << 16) + col, v16);
                    const int mb = n0 + c;
                    if (row < g.M && mb < g.W) {
                        float* o = g.out + (size_t)row * g.W + mb;
#pragma unroll
                        for (int i = 0; i < 16; i++) {
                            const float pos1 = fabsf(xcs + (float)(mb + i)) * g.pitch;
                            v16[i] *= sad * rsqrtf(fmaf(pos1, pos1, base2));
                        }
                        // columns of this tile and of the detector only
                        const int lim = min(g.W - mb, g.NT - c);
                        if (g.vec && lim >= 16) {
#pragma unroll
                            for (int i = 0; i < 16; i += 4)
                                *reinterpret_cast<float4*>(o + i) =
                                    make_float4(v16[i], v16[i + 1], v16[i + 2], v16[i + 3]);
                        } else {
#pragma unroll
                            for (int i = 0; i < 16; i++)
                                if (i < lim) o[i] = v16[i];
                        }
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        // every MMA this CTA issued has completed before its accumulator is
        // released (the commit above arrives on `accum` once they have)
        warp_wait(accum, 0, g.err);
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(512));
    }
}

// Unfused form, rows of p not 16-byte aligned: A planes [3][M][Kp], the
// split of g = -logf(p) (times the redundancy weight).  grid (M, ceil(Kp /
// 1024)), block 128: one detector row per block, eight consecutive columns
// per thread, each plane written as one 16-byte group (Kp is a multiple of 64).
__global__ void __launch_bounds__(128) split_a_kernel(const float* __restrict__ proj, const float* __restrict__ wts,
                                                      int M, int H, int W, int Kp, __nv_bfloat16* __restrict__ planes)
{
    const int r = blockIdx.x;
    const int k0 = 8 * (blockIdx.y * blockDim.x + threadIdx.x);
    if (k0 >= Kp) return;
    const float* pr = proj + (size_t)r * W;
    const float* wr = wts ? wts + (size_t)(r / H) * W : nullptr;
    float x[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
        x[q] = 0.0f;
        if (k0 + q < W) {
            x[q] = -logf(__ldg(pr + k0 + q));
            if (wr) x[q] *= __ldg(wr + k0 + q);
        }
    }
    uint4 p0, p1, p2;
    split3x2(x[0], x[1], p0.x, p1.x, p2.x);
    split3x2(x[2], x[3], p0.y, p1.y, p2.y);
    split3x2(x[4], x[5], p0.z, p1.z, p2.z);
    split3x2(x[6], x[7], p0.w, p1.w, p2.w);
    const size_t plane = (size_t)M * Kp, o = (size_t)r * Kp + k0;
    *reinterpret_cast<uint4*>(planes + o) = p0;
    *reinterpret_cast<uint4*>(planes + plane + o) = p1;
    *reinterpret_cast<uint4*>(planes + 2 * plane + o) = p2;
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

// 2D FP32 tensor [M][W] (the projections) with box {64, 128}, no swizzle;
// columns beyond W and rows beyond M read as zero.
bool make_p_map(CUtensorMap* map, const float* proj, int M, int W)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)W, (cuuint64_t)M};
    cuuint64_t strides[1] = {(cuuint64_t)W * 4};
    cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)BM};
    cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(proj), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// 2D FP32 tensor [M][W] (the filtered output) with box {16, 32} in the
// 64-byte swizzle layout; stores are clipped at W and M.
bool make_out_map(CUtensorMap* map, float* out, int M, int W)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)W, (cuuint64_t)M};
    cuuint64_t strides[1] = {(cuuint64_t)W * 4};
    cuuint32_t box[2] = {16, 32};
    cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, out, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Output columns are split into ntiles tiles of NT <= 512 columns (one
// tensor-memory accumulator of 128 x NT FP32 each; NT a multiple of 32, so a
// column half is a legal MMA width); B is padded to Np = ntiles * NT rows.
// The workspace holds the split Toeplitz planes (a function of the kernel
// and W only, split once per kernel), the error flag and, for the unfused
// form only, the split A planes.
struct Layout {
    int M, Np, NT, ntiles, Kp;
    size_t a_off, b_off, err_off, total, smem;
};

Layout layout_for(int V, int H, int W, bool fused)
{
    Layout L{};
    L.M = V * H;
    const int n16 = (W + 15) / 16 * 16;
    L.ntiles = (n16 + 511) / 512;
    L.NT = ((n16 + L.ntiles - 1) / L.ntiles + 31) / 32 * 32;
    L.Np = L.ntiles * L.NT;
    L.Kp = (W + BK - 1) / BK * BK;
    L.smem = 1024 + gemm_smem_bytes(L.NT, fused);
    L.b_off = 0;
    L.err_off = (3 * (size_t)L.Np * L.Kp * 2 + 1023) / 1024 * 1024;
    L.a_off = L.err_off + 1024;
    L.total = L.a_off + (fused ? 0 : (3 * (size_t)L.M * L.Kp * 2 + 1023) / 1024 * 1024);
    return L;
}

}  // namespace

bool ramp_gemm_fused(const float* proj, const float* out, int W)
{
    return W % 4 == 0 && (reinterpret_cast<uintptr_t>(proj) & 15) == 0 && (reinterpret_cast<uintptr_t>(out) & 15) == 0;
}

size_t ramp_gemm_workspace_bytes(int V, int H, int W, bool fused) { return layout_for(V, H, W, fused).total; }

cudaError_t launch_ramp_gemm_bf16x3(const float* proj, float* out, const float* hT, const FilterView* views,
                                    const float* wts, float pitch, float sad, int V, int H, int W, void* workspace,
                                    int* b_ready, cudaStream_t st)
{
    if (W < 16 || W > 4096) return cudaErrorInvalidValue;
    const bool fused = ramp_gemm_fused(proj, out, W);
    const Layout L = layout_for(V, H, W, fused);
    if (L.smem > 227 * 1024) return cudaErrorInvalidValue;
    uint8_t* ws = static_cast<uint8_t*>(workspace);
    __nv_bfloat16* bp = reinterpret_cast<__nv_bfloat16*>(ws + L.b_off);
    int* err = reinterpret_cast<int*>(ws + L.err_off);
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    if (!b_ready || !*b_ready) {
        // the Toeplitz planes change only with the kernel: split once
        const size_t nb = (size_t)L.Np * L.Kp;
        split_b_kernel<<<(unsigned)((nb + 255) / 256), 256, 0, st>>>(hT, W, L.Np, L.Kp, bp);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if (b_ready) *b_ready = 1;
    }
    CUtensorMap tmA, tmB, tmO;
    if (!make_map(&tmB, bp, L.Np, L.Kp, L.NT / 2)) return cudaErrorInvalidValue;
    tmO = tmB;  // the unfused form stores without TMA
    if (fused) {
        if (!make_p_map(&tmA, proj, L.M, W) || !make_out_map(&tmO, out, L.M, W)) return cudaErrorInvalidValue;
    } else {
        // rows not 16-byte aligned: split A into the workspace first
        __nv_bfloat16* ap = reinterpret_cast<__nv_bfloat16*>(ws + L.a_off);
        split_a_kernel<<<dim3((unsigned)L.M, (unsigned)((L.Kp + 1023) / 1024)), 128, 0, st>>>(proj, wts, L.M, H, W,
                                                                                          L.Kp, ap);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if (!make_map(&tmA, ap, L.M, L.Kp, BM)) return cudaErrorInvalidValue;
    }
    const int vec = (W % 4 == 0 && (reinterpret_cast<uintptr_t>(out) & 15) == 0) ? 1 : 0;
    GemmArgs g{out, views, fused ? wts : nullptr, pitch, sad, L.M, H, W, L.NT, L.Kp, L.Kp / BK, vec, err};
    const dim3 grid((L.M + BM - 1) / BM, L.ntiles);
    if (fused) {
        e = cudaFuncSetAttribute(ramp_gemm_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem);
        if (e != cudaSuccess) return e;
        ramp_gemm_kernel<true><<<grid, kThreads, L.smem, st>>>(tmA, tmB, tmO, g);
    } else {
        e = cudaFuncSetAttribute(ramp_gemm_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem);
        if (e != cudaSuccess) return e;
        ramp_gemm_kernel<false><<<grid, kThreads, L.smem, st>>>(tmA, tmB, tmO, g);
    }
    return cudaGetLastError();
}

int ramp_gemm_error_flag(void* workspace, int V, int H, int W, cudaStream_t st)
{
    const Layout L = layout_for(V, H, W, true);  // the flag's place is the same in both layouts
    int h = 0;
    if (cudaMemcpyAsync(&h, static_cast<uint8_t*>(workspace) + L.err_off, sizeof(int), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return -1;
    return h;
}

}  // namespace vcbct
