// mlp_tc.cuh -- the learned Kepler heads (MLP 2 -> 64 -> 64 -> 64 -> 1, ReLU) evaluated on
// the 5th-generation tensor cores: BF16 operands in shared memory, FP32 accumulators in
// tensor memory (TMEM), one thread issuing tcgen05.mma for the CTA.
//
// A CTA of kMlpThreads = 256 threads evaluates 256 rows (one per thread) per call: two
// M = 128 tiles, N = 64, K = 16 for layer 1 (2 inputs padded with zeros) and K = 64 for
// layers 2 and 3; layer 4 (64 -> 1) is a per-thread FP32 dot product.  Between layers each
// thread reads its own accumulator row back with tcgen05.ld (warp w owns TMEM lanes
// 32 (w mod 4) .. + 31 of tile w / 4), adds the bias, applies ReLU, rounds to BF16 and
// writes the row as the next layer's A operand.
//
// The two tiles are two independent pipelines: warpgroup g (warps 4g .. 4g + 3, rows
// 128 g .. + 127) has its own A tile, TMEM columns, issuing thread and mbarrier and
// synchronises on its own named barrier, so one warpgroup's epilogue runs while the other
// waits for its MMAs.
//
// Operand layout: K-major, no swizzle, the canonical arrangement of 8-row x 16-byte core
// matrices: element (row, k) of a [rows][K] BF16 matrix sits at byte
//     ((row / 8) * (K / 8) + k / 8) * 128 + (row % 8) * 16 + (k % 8) * 2,
// so core matrices adjacent in K are 128 bytes apart (leading byte offset) and 8-row groups
// are K * 16 bytes apart (stride byte offset).  One MMA covers K = 16 (two core matrices):
// the descriptor start advances 256 bytes per K step.
//
// Completion: tcgen05.commit arrives on an mbarrier; every wait is bounded and a timeout
// sets the CTA's abort flag (no further MMA is issued; the caller treats the guesses as
// missing and reports BIA_ERR_DEVICE_TIMEOUT).
#pragma once
#include <cuda_bf16.h>

#include <cstddef>
#include <cstdint>
#include <cstring>

namespace bia {

constexpr int kMlpHidden = 64;
constexpr int kMlpK1 = 16;
constexpr int kMlpThreads = 256;

// One head as stored in learned_heads.bin (after its 16-byte header): BF16 weights
// output-major W[n][k], FP32 biases and the last layer.
struct MlpHead {
    uint16_t w1[kMlpHidden * kMlpK1];
    uint16_t w2[kMlpHidden * kMlpHidden];
    uint16_t w3[kMlpHidden * kMlpHidden];
    float b1[kMlpHidden], b2[kMlpHidden], b3[kMlpHidden], w4[kMlpHidden], b4[4];
};
static_assert(sizeof(MlpHead) == 19472, "learned_heads.bin head record");
constexpr int kMlpHeads = 2;  // 0 elliptic, 1 hyperbolic

// A head as the kernels keep it in device memory: the weights already in the shared-memory
// operand layout (kmajor_off below; W1 at byte 0, W2 at 2048, W3 at 10240, as in MlpSmem),
// then the FP32 vectors in MlpSmem's order, so that loading a head is a straight copy.
constexpr int kMlpWeightBytes = (kMlpHidden * kMlpK1 + 2 * kMlpHidden * kMlpHidden) * 2;  // 18432
struct MlpImage {
    alignas(16) uint8_t w[kMlpWeightBytes];
    float b1[kMlpHidden], b2[kMlpHidden], b3[kMlpHidden], w4[kMlpHidden], b4[4];
};
static_assert(sizeof(MlpImage) == 19472, "head image");

// Shared-memory image of one head and the activation tile (1024-aligned parts).  Each
// warpgroup's layer-1 rows (K = 16, 4 KB) live at the start of its own 16 KB half of the
// layer-2/3 tile: its layer-1 MMA has completed before its first epilogue overwrites them.
constexpr uint32_t kMlpTileBytes = 128u * kMlpHidden * 2;  // one warpgroup's A tile
struct MlpSmem {
    alignas(1024) uint8_t w1[kMlpHidden * kMlpK1 * 2];        // 2 KB
    alignas(1024) uint8_t w2[kMlpHidden * kMlpHidden * 2];    // 8 KB
    alignas(1024) uint8_t w3[kMlpHidden * kMlpHidden * 2];    // 8 KB
    alignas(1024) uint8_t a2[kMlpThreads * kMlpHidden * 2];   // 32 KB; a1 = a2
    float b1[kMlpHidden], b2[kMlpHidden], b3[kMlpHidden], w4[kMlpHidden], b4;
    alignas(8) uint64_t mbar[2];  // one per warpgroup
    uint32_t tmem_base;
    int abort[2];
    int turns;  // scratch for CTA-wide counts of the callers
    int head;   // the head whose weights are loaded (-1: none)
    int wsum[2][kMlpThreads / 32];  // per-warp totals of the callers' row scans
};

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__host__ __device__ __forceinline__ uint32_t kmajor_off(int row, int k, int K)
{
    return (uint32_t)((((row >> 3) * (K >> 3)) + (k >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// tcgen05 shared-memory matrix descriptor: start, leading and stride byte offsets (>> 4),
// descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t mma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// kind::f16 instruction descriptor: D F32, A and B BF16, both K-major, N = 64, M = 128.
constexpr uint32_t kIdescBf16M128N64 =
    (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(kIdescBf16M128N64), "r"(accumulate));
}

__device__ __forceinline__ void tc_commit(uint64_t *mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr(mbar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Bounded wait for the mbarrier phase with parity `phase` to complete; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t phase)
{
    const uint32_t a = smem_addr(mbar);
    for (int it = 0; it < (1 << 22); it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

// max(a, 0), max(b, 0) rounded to BF16 (nearest even), a in the low half: one paired
// conversion with the ReLU built in (rounding is monotone and keeps 0, so this equals
// rounding the ReLU's FP32 output)
__device__ __forceinline__ uint32_t pack_bf16_relu(float a, float b)
{
    uint32_t d;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(b), "f"(a));
    return d;
}

// 32 consecutive FP32 accumulator columns of this thread's TMEM lane (one load, one wait)
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float v[32])
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
    for (int j = 0; j < 32; j++) v[j] = __uint_as_float(r[j]);
}

// (a, b) rounded to BF16 (nearest even), a in the low half: one paired conversion
__device__ __forceinline__ uint32_t pack_bf16(float a, float b)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t *>(&v);
}

// The device image of a head from its file record (host side, once per set of heads).
inline void mlp_image_from_head(const MlpHead &H, MlpImage &I)
{
    for (int e = 0; e < kMlpHidden * kMlpK1; e++)
        memcpy(I.w + kmajor_off(e / kMlpK1, e % kMlpK1, kMlpK1), &H.w1[e], 2);
    for (int e = 0; e < kMlpHidden * kMlpHidden; e++) {
        const int n = e / kMlpHidden, k = e % kMlpHidden;
        memcpy(I.w + 2048 + kmajor_off(n, k, kMlpHidden), &H.w2[e], 2);
        memcpy(I.w + 10240 + kmajor_off(n, k, kMlpHidden), &H.w3[e], 2);
    }
    memcpy(I.b1, H.b1, sizeof(I.b1));
    memcpy(I.b2, H.b2, sizeof(I.b2));
    memcpy(I.b3, H.b3, sizeof(I.b3));
    memcpy(I.w4, H.w4, sizeof(I.w4));
    memcpy(I.b4, H.b4, sizeof(I.b4));
}

// One head from its device image into shared memory (all threads, 16-byte copies, with a
// CTA barrier at the end: the two warpgroups' MMAs read every weight).  The caller makes
// sure that no MMA on the old weights is in flight.
__device__ __forceinline__ void mlp_load_head(MlpSmem &S, const MlpImage *heads, int h)
{
    static_assert(offsetof(MlpSmem, w2) == 2048 && offsetof(MlpSmem, w3) == 10240, "weight image layout");
    static_assert(offsetof(MlpSmem, b2) == offsetof(MlpSmem, b1) + 256 && offsetof(MlpSmem, w4) == offsetof(MlpSmem, b1) + 768,
                  "vector layout");
    const int tid = threadIdx.x;
    const MlpImage &I = heads[h];
    const uint4 *src = reinterpret_cast<const uint4 *>(I.w);
    uint4 *dst = reinterpret_cast<uint4 *>(S.w1);
    for (int e = tid; e < kMlpWeightBytes / 16; e += blockDim.x) dst[e] = src[e];
    const float4 *vs = reinterpret_cast<const float4 *>(I.b1);
    float4 *vd = reinterpret_cast<float4 *>(S.b1);
    for (int e = tid; e < 4 * kMlpHidden / 4; e += blockDim.x) vd[e] = vs[e];
    if (tid == 0) {
        S.b4 = I.b4[0];
        S.head = h;
    }
    fence_async_smem();
    __syncthreads();
}

// Once per CTA (all threads): the mbarrier and the TMEM allocation (warp 0, 128 columns:
// two 128 x 64 FP32 accumulator tiles).  No head is loaded yet.
__device__ __forceinline__ void mlp_setup(MlpSmem &S)
{
    const int tid = threadIdx.x;
    if (tid == 0) {
        S.abort[0] = S.abort[1] = 0;
        S.head = -1;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&S.mbar[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&S.mbar[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();  // the .sync.aligned TMEM instructions need the whole warp converged
    if ((tid >> 5) == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;" ::"r"(
                         smem_addr(&S.tmem_base))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}

// Once per CTA at the end (all threads): free the TMEM columns.  After a timeout the
// warpgroup's MMA group in flight is waited for once more (bounded) before the columns are
// released.
__device__ __forceinline__ void mlp_teardown(MlpSmem &S, uint32_t phase)
{
    const int wg = threadIdx.x >> 7;
    tc_fence_before();
    __syncthreads();
    if (S.abort[wg]) mbar_wait(&S.mbar[wg], phase);
    __syncthreads();
    tc_fence_after();
    __syncwarp();
    if ((threadIdx.x >> 5) == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;" ::"r"(S.tmem_base) : "memory");
}

// Barrier of this thread's warpgroup (named barriers 1 and 2; 0 is __syncthreads).
__device__ __forceinline__ void wg_sync(int wg)
{
    asm volatile("bar.sync %0, 128;" ::"r"(1 + wg) : "memory");
}

// One layer of this warpgroup's 128-row tile: the MMAs issued by the warpgroup's first
// thread (A rows at a + wg * kMlpTileBytes, K-major with K columns), then the bounded wait
// of every thread of the warpgroup.  Returns false (and sets S.abort[wg]) on a timeout;
// the answer is the same on every thread of the warpgroup.
__device__ __forceinline__ bool mlp_layer(MlpSmem &S, const uint8_t *a, const uint8_t *w, int K, uint32_t &phase)
{
    const int wg = threadIdx.x >> 7;
    fence_async_smem();
    tc_fence_before();
    wg_sync(wg);
    tc_fence_after();
    if (S.abort[wg]) return false;  // uniform in the warpgroup: read after its barrier
    if ((threadIdx.x & 127) == 0) {
        const uint32_t sbo = (uint32_t)K * 16;
        for (int ks = 0; ks < K / 16; ks++) {
            const uint64_t ad = mma_desc(smem_addr(a) + wg * kMlpTileBytes + ks * 256, 128, sbo);
            const uint64_t bd = mma_desc(smem_addr(w) + ks * 256, 128, sbo);
            tc_mma(S.tmem_base + (uint32_t)(wg * 64), ad, bd, ks > 0 ? 1u : 0u);
        }
        tc_commit(&S.mbar[wg]);
    }
    const bool ok = mbar_wait(&S.mbar[wg], phase);
    // a timeout on any thread aborts the warpgroup's MLP work
    if (!ok) S.abort[wg] = 1;
    wg_sync(wg);
    if (S.abort[wg]) return false;  // the phase stays: teardown waits for it once more
    phase ^= 1u;
    tc_fence_after();
    return true;
}

// This thread's accumulator row of the last layer: + bias, ReLU; either written as BF16
// into the next A tile (dst != nullptr) or dotted with w4 (returned).
__device__ __forceinline__ float mlp_epilogue(MlpSmem &S, const float *bias, uint8_t *dst)
{
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const uint32_t taddr = S.tmem_base + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)((warp >> 2) * 64);
    float dot = 0.0f;
    __syncwarp();
#pragma unroll
    for (int c = 0; c < kMlpHidden; c += 32) {
        float v[32];
        tc_ld32(taddr + (uint32_t)c, v);
#pragma unroll
        for (int j = 0; j < 32; j++) v[j] += bias[c + j];
        if (dst) {
#pragma unroll
            for (int q = 0; q < 32; q += 8) {
                uint4 o;
                o.x = pack_bf16_relu(v[q + 0], v[q + 1]); o.y = pack_bf16_relu(v[q + 2], v[q + 3]);
                o.z = pack_bf16_relu(v[q + 4], v[q + 5]); o.w = pack_bf16_relu(v[q + 6], v[q + 7]);
                *(uint4 *)(dst + kmajor_off(tid, c + q, kMlpHidden)) = o;
            }
        } else {
#pragma unroll
            for (int j = 0; j < 32; j++) dot = fmaf(fmaxf(v[j], 0.0f), S.w4[c + j], dot);
        }
    }
    return dot + S.b4;
}

// The loaded head's output for this thread's input row, given as packed BF16 (x0 in the
// low half); every thread of the CTA calls it.  ok (the same on every thread of a
// warpgroup) is false when the warpgroup's tensor-core pipeline timed out; it then issues
// no more MMAs.
__device__ __forceinline__ float mlp_eval_cta(MlpSmem &S, uint32_t x01_bf16, uint32_t &phase, bool &ok)
{
    const int tid = threadIdx.x;
    // layer-1 rows at the start of the warpgroup's own half of the layer-2 tile
    uint8_t *a1 = S.a2 + (tid >> 7) * kMlpTileBytes;
    *(uint4 *)(a1 + kmajor_off(tid & 127, 0, kMlpK1)) = make_uint4(x01_bf16, 0u, 0u, 0u);
    *(uint4 *)(a1 + kmajor_off(tid & 127, 8, kMlpK1)) = make_uint4(0u, 0u, 0u, 0u);
    ok = false;
    if (!mlp_layer(S, S.a2, S.w1, kMlpK1, phase)) return 0.0f;
    mlp_epilogue(S, S.b1, S.a2);
    if (!mlp_layer(S, S.a2, S.w2, kMlpHidden, phase)) return 0.0f;
    mlp_epilogue(S, S.b2, S.a2);
    if (!mlp_layer(S, S.a2, S.w3, kMlpHidden, phase)) return 0.0f;
    ok = true;
    return mlp_epilogue(S, S.b3, nullptr);
}

}  // namespace bia
