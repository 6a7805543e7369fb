// mlp_train.cu -- training of the learned Kepler heads on the device: samples from the FP64
// Kepler solver, forward and backward passes on the 5th-generation tensor cores (BF16
// operands in shared memory, FP32 accumulators in tensor memory), Adam on FP32 master
// weights.
//
// Network (one head): x (2) -> ReLU(W1 x + b1) (64) -> ReLU(W2 . + b2) (64) ->
// ReLU(W3 . + b3) (64) -> w4 . + b4, mean squared error against the target anomaly.
//
// One CTA of 128 threads trains on 128 rows per launch, one row per thread and per TMEM
// lane.  Every GEMM is a tcgen05.mma of M = 128 issued by thread 0:
//   forward          Z1 = X W1^T (K = 16), Z2 = H1 W2^T, Z3 = H2 W3^T (K = 64, N = 64)
//   data gradients   dH2 = dZ3 W3, dH1 = dZ2 W2 (K = 64, N = 64; B = the transposed images)
//   weight gradients over the 128 rows (K = 128), two MMAs with stacked operands:
//     [dZ3^T ; dZ2^T] x [H2^T ; H1^T ; 1]            (M = 128, N = 144): dW3, db3 and dW2, db2
//     [dZ1^T ; dy ; 0] x [x0 ; x1 ; 1 ; 0 ; H3^T]   (M = 128, N = 80):  dW1, db1 and dw4, db4
//   (the products of the off-diagonal blocks are computed and not read).
// The activations and gradients are rounded to BF16 as MMA operands (the inference kernels
// round the activations the same way); the loss, dy, the biases and the output layer are FP32.
// Each CTA writes its gradient sums; the Adam kernel adds the CTAs' sums in CTA order (the
// training is deterministic for a seed), updates the FP32 master parameters and rewrites
// the BF16 operand images the next step's CTAs load.
//
// Operand layout: the K-major canonical layout of mlp_tc.cuh (kmajor_off), for K = 16, 64
// and 128.  Every mbarrier wait is bounded; a timeout stops the CTA's MMAs and is reported
// (BIA_ERR_DEVICE_TIMEOUT) without a fault.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "bia_internal.cuh"
#include "bia_learned.cuh"
#include "mlp_tc.cuh"

namespace bia {

constexpr int kTrainRows = 128;
constexpr int kTrainThreads = 128;
constexpr int kHid = kMlpHidden;  // 64

// FP32 parameters of one head, in this order (the host API's layout as well)
constexpr int kPW1 = 0;                       // W1 [64][2]
constexpr int kPB1 = kPW1 + kHid * 2;         // b1 [64]
constexpr int kPW2 = kPB1 + kHid;             // W2 [64][64] (output-major)
constexpr int kPB2 = kPW2 + kHid * kHid;
constexpr int kPW3 = kPB2 + kHid;             // W3 [64][64]
constexpr int kPB3 = kPW3 + kHid * kHid;
constexpr int kPW4 = kPB3 + kHid;             // w4 [64]
constexpr int kPB4 = kPW4 + kHid;             // b4
constexpr int kParams = kPB4 + 1;             // 8577
static_assert(kParams == 8577, "parameter count");

// BF16 operand images the training CTAs load (written by the Adam kernel): the forward
// weights as in MlpImage (W1 [64][16] padded, W2, W3 [64][64], K-major) and the transposed
// W2^T, W3^T (element (i, o) holds W[o][i]) for the data gradients.
constexpr int kImgW1 = 0, kImgW2 = 2048, kImgW3 = 10240, kImgW2T = 18432, kImgW3T = 26624;
constexpr int kImgBytes = 34816;

struct TrainSmem {
    alignas(1024) uint8_t w[kImgBytes];      // the five weight images
    alignas(1024) uint8_t a1[kTrainRows * 16 * 2];       // X rows, K = 16
    alignas(1024) uint8_t p[kTrainRows * kHid * 2];      // H1, then dZ3 (K = 64)
    alignas(1024) uint8_t q[kTrainRows * kHid * 2];      // H2, then dZ2
    alignas(1024) uint8_t awg[128 * 128 * 2];            // [dZ3^T ; dZ2^T], K = 128
    alignas(1024) uint8_t bwg[144 * 128 * 2];            // [H2^T ; H1^T ; 1 ; 0]
    alignas(1024) uint8_t awg1[128 * 128 * 2];           // [dZ1^T ; dy ; 0]
    alignas(1024) uint8_t bwg1[80 * 128 * 2];            // [x0 ; x1 ; 1 ; 0 ; H3^T]
    float b1[kHid], b2[kHid], b3[kHid], w4[kHid];
    float b4;
    float loss[kTrainThreads / 32];
    alignas(8) uint64_t mbar;
    uint32_t tmem_base;
    int abort;
};
constexpr size_t kTrainSmemBytes = sizeof(TrainSmem) + 1024;

// kind::f16 instruction descriptor: D F32, A and B BF16, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t M, uint32_t N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void tc_mma_id(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// Issues D = A B^T over K (A: 128 rows at a, B: N rows at b, both K-major with K columns)
// into TMEM column dcol (thread 0 only; no commit).
__device__ __forceinline__ void issue_gemm(uint32_t tmem, uint32_t dcol, const uint8_t *a, const uint8_t *b, int K,
                                           uint32_t N)
{
    const uint32_t sbo = (uint32_t)K * 16;
    const uint32_t id = idesc_bf16(128, N);
    for (int ks = 0; ks < K / 16; ks++) {
        const uint64_t ad = mma_desc(smem_addr(a) + ks * 256, 128, sbo);
        const uint64_t bd = mma_desc(smem_addr(b) + ks * 256, 128, sbo);
        tc_mma_id(tmem + dcol, ad, bd, id, ks > 0 ? 1u : 0u);
    }
}

// Makes the threads' shared-memory writes visible to the tensor cores, issues (thread 0)
// what `issue` launches, commits, and waits (bounded) on every thread.  false: timed out
// (S.abort set; no further MMA is issued by the caller).
template <typename F>
__device__ __forceinline__ bool run_mma(TrainSmem &S, uint32_t &phase, F issue)
{
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (S.abort) return false;
    if (threadIdx.x == 0) {
        issue();
        tc_commit(&S.mbar);
    }
    const bool ok = mbar_wait(&S.mbar, phase);
    if (!ok) S.abort = 1;
    __syncthreads();
    if (S.abort) return false;
    phase ^= 1u;
    tc_fence_after();
    return true;
}

__device__ __forceinline__ uint16_t bf16_bits(float v) { return __bfloat16_as_ushort(__float2bfloat16_rn(v)); }

__device__ __forceinline__ void st_bf16(uint8_t *base, uint32_t off, float v)
{
    *reinterpret_cast<uint16_t *>(base + off) = bf16_bits(v);
}

// 8 consecutive values of one row into a K-major tile (one 16-byte store)
__device__ __forceinline__ void st_row8(uint8_t *base, int row, int k, int K, const float v[8])
{
    uint4 o;
    o.x = pack_bf16(v[0], v[1]);
    o.y = pack_bf16(v[2], v[3]);
    o.z = pack_bf16(v[4], v[5]);
    o.w = pack_bf16(v[6], v[7]);
    *reinterpret_cast<uint4 *>(base + kmajor_off(row, k, K)) = o;
}

// n consecutive FP32 columns of this thread's TMEM lane (n = 1 .. 4: an x4 load)
__device__ __forceinline__ void tc_ld4(uint32_t taddr, float v[4])
{
    uint32_t r[4];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 4; j++) v[j] = __uint_as_float(r[j]);
}

struct TrainArgs {
    const float *x;          // samples [n][2]
    const float *y;          // targets [n]
    long long n;             // samples (a power of two when perm_mul != 0)
    long long row0;          // first row of this launch in the epoch's order
    unsigned long long perm_mul, perm_add;  // sample index = (perm_mul * row + perm_add) mod n; mul 0: row itself
    float dy_scale;          // 2 / (rows of the batch): d(mean squared error)/dy
    const uint8_t *img;      // the BF16 weight images (kImgBytes)
    const float *vec;        // FP32 master parameters (biases and w4, b4 are read from here)
    float *grad;             // [gridDim.x][kParams] gradient sums of each CTA
    float *loss;             // [gridDim.x] squared-error sums
    int *status;             // set to 1 on a timed-out tensor-core wait
};

__global__ void __launch_bounds__(kTrainThreads, 1) mlp_train_kernel(const TrainArgs A)
{
    extern __shared__ uint8_t train_smem_raw[];
    TrainSmem &S = *reinterpret_cast<TrainSmem *>(((uintptr_t)train_smem_raw + 1023) & ~(uintptr_t)1023);
    const int r = threadIdx.x;
    const int warp = r >> 5;
    // ---- set-up: weights and vectors, constant rows, mbarrier, tensor memory
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(A.img);
        uint4 *dst = reinterpret_cast<uint4 *>(S.w);
        for (int e = r; e < kImgBytes / 16; e += kTrainThreads) dst[e] = src[e];
        if (r < kHid) {
            S.b1[r] = A.vec[kPB1 + r];
            S.b2[r] = A.vec[kPB2 + r];
            S.b3[r] = A.vec[kPB3 + r];
            S.w4[r] = A.vec[kPW4 + r];
        }
        if (r == 0) {
            S.b4 = A.vec[kPB4];
            S.abort = 0;
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&S.mbar)) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        // this thread's column r of the constant rows: the ones rows of the bias gradients,
        // zero padding rows
        st_bf16(S.bwg, kmajor_off(128, r, 128), 1.0f);
        for (int row = 129; row < 144; row++) st_bf16(S.bwg, kmajor_off(row, r, 128), 0.0f);
        st_bf16(S.bwg1, kmajor_off(2, r, 128), 1.0f);
        for (int row = 3; row < 16; row++) st_bf16(S.bwg1, kmajor_off(row, r, 128), 0.0f);
        for (int row = 65; row < 128; row++) st_bf16(S.awg1, kmajor_off(row, r, 128), 0.0f);
        __syncwarp();
        if (warp == 0) {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(
                             smem_addr(&S.tmem_base))
                         : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        }
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    }
    const uint32_t tmem = S.tmem_base;
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);  // this thread's TMEM lane
    uint32_t phase = 0;

    // ---- this thread's sample
    const long long row = A.row0 + (long long)blockIdx.x * kTrainRows + r;
    const long long idx = A.perm_mul ? (long long)((A.perm_mul * (unsigned long long)row + A.perm_add) &
                                                   (unsigned long long)(A.n - 1))
                                     : row;
    const bool valid = idx < A.n;
    const float x0 = valid ? A.x[2 * idx] : 0.0f, x1 = valid ? A.x[2 * idx + 1] : 0.0f;
    const float yt = valid ? A.y[idx] : 0.0f;
    {
        const float v[8] = {x0, x1, 0, 0, 0, 0, 0, 0}, z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        st_row8(S.a1, r, 0, 16, v);
        st_row8(S.a1, r, 8, 16, z);
        st_bf16(S.bwg1, kmajor_off(0, r, 128), x0);
        st_bf16(S.bwg1, kmajor_off(1, r, 128), x1);
    }
    uint64_t m1 = 0, m2 = 0;  // ReLU masks of layers 1 and 2
    float dy = 0.0f, err = 0.0f;
    const uint8_t *W1 = S.w + kImgW1, *W2 = S.w + kImgW2, *W3 = S.w + kImgW3;
    const uint8_t *W2T = S.w + kImgW2T, *W3T = S.w + kImgW3T;
    bool ok = true;

    // ---- forward
    ok = ok && run_mma(S, phase, [&] { issue_gemm(tmem, 0, S.a1, W1, 16, 64); });
    if (ok) {  // H1 = ReLU(Z1 + b1): A of layer 2 and rows 64..127 of bwg (H1^T)
        __syncwarp();
#pragma unroll
        for (int c = 0; c < kHid; c += 32) {
            float v[32];
            tc_ld32(lane_addr + c, v);
#pragma unroll
            for (int j = 0; j < 32; j++) {
                v[j] += S.b1[c + j];
                if (v[j] > 0.0f) m1 |= 1ull << (c + j);
                v[j] = fmaxf(v[j], 0.0f);
                st_bf16(S.bwg, kmajor_off(64 + c + j, r, 128), v[j]);
            }
#pragma unroll
            for (int q8 = 0; q8 < 32; q8 += 8) st_row8(S.p, r, c + q8, kHid, v + q8);
        }
    }
    ok = ok && run_mma(S, phase, [&] { issue_gemm(tmem, 0, S.p, W2, kHid, 64); });
    if (ok) {  // H2: A of layer 3 and rows 0..63 of bwg (H2^T)
        __syncwarp();
#pragma unroll
        for (int c = 0; c < kHid; c += 32) {
            float v[32];
            tc_ld32(lane_addr + c, v);
#pragma unroll
            for (int j = 0; j < 32; j++) {
                v[j] += S.b2[c + j];
                if (v[j] > 0.0f) m2 |= 1ull << (c + j);
                v[j] = fmaxf(v[j], 0.0f);
                st_bf16(S.bwg, kmajor_off(c + j, r, 128), v[j]);
            }
#pragma unroll
            for (int q8 = 0; q8 < 32; q8 += 8) st_row8(S.q, r, c + q8, kHid, v + q8);
        }
    }
    ok = ok && run_mma(S, phase, [&] { issue_gemm(tmem, 0, S.q, W3, kHid, 64); });
    if (ok) {  // y = w4 . ReLU(Z3 + b3) + b4 in FP32; dy; dZ3 = dy w4 (Z3 > 0)
        __syncwarp();
        float z3[kHid];
        tc_ld32(lane_addr, z3);
        tc_ld32(lane_addr + 32, z3 + 32);
        float yv = S.b4;
#pragma unroll
        for (int j = 0; j < kHid; j++) {
            z3[j] += S.b3[j];
            yv = fmaf(fmaxf(z3[j], 0.0f), S.w4[j], yv);
        }
        err = valid ? yv - yt : 0.0f;
        dy = err * A.dy_scale;
        st_bf16(S.awg1, kmajor_off(64, r, 128), dy);
#pragma unroll
        for (int c = 0; c < kHid; c += 8) {
            float g[8];
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const float h3 = fmaxf(z3[c + j], 0.0f);
                st_bf16(S.bwg1, kmajor_off(16 + c + j, r, 128), h3);
                g[j] = z3[c + j] > 0.0f ? dy * S.w4[c + j] : 0.0f;
                st_bf16(S.awg, kmajor_off(c + j, r, 128), g[j]);
            }
            st_row8(S.p, r, c, kHid, g);
        }
    }
    // ---- backward: data gradients
    ok = ok && run_mma(S, phase, [&] { issue_gemm(tmem, 0, S.p, W3T, kHid, 64); });
    if (ok) {  // dZ2 = dH2 (Z2 > 0): A of the next MMA and rows 64..127 of awg
        __syncwarp();
#pragma unroll
        for (int c = 0; c < kHid; c += 32) {
            float v[32];
            tc_ld32(lane_addr + c, v);
#pragma unroll
            for (int j = 0; j < 32; j++) {
                v[j] = ((m2 >> (c + j)) & 1ull) ? v[j] : 0.0f;
                st_bf16(S.awg, kmajor_off(64 + c + j, r, 128), v[j]);
            }
#pragma unroll
            for (int q8 = 0; q8 < 32; q8 += 8) st_row8(S.q, r, c + q8, kHid, v + q8);
        }
    }
    ok = ok && run_mma(S, phase, [&] { issue_gemm(tmem, 0, S.q, W2T, kHid, 64); });
    if (ok) {  // dZ1 = dH1 (Z1 > 0): rows 0..63 of awg1
        __syncwarp();
#pragma unroll
        for (int c = 0; c < kHid; c += 32) {
            float v[32];
            tc_ld32(lane_addr + c, v);
#pragma unroll
            for (int j = 0; j < 32; j++)
                st_bf16(S.awg1, kmajor_off(c + j, r, 128), ((m1 >> (c + j)) & 1ull) ? v[j] : 0.0f);
        }
    }
    // ---- weight gradients over the 128 rows (both stacked products in one commit)
    ok = ok && run_mma(S, phase, [&] {
        issue_gemm(tmem, 64, S.awg, S.bwg, 128, 144);
        issue_gemm(tmem, 256, S.awg1, S.bwg1, 128, 80);
    });
    float *G = A.grad + (size_t)blockIdx.x * kParams;
    if (ok) {
        __syncwarp();
        if (warp < 2) {  // lane r = output o of layer 3 (columns 64.. 127: dW3 row, 192: db3)
            float v[32], t4[4];
            tc_ld32(lane_addr + 64, v);
#pragma unroll
            for (int j = 0; j < 32; j++) G[kPW3 + r * kHid + j] = v[j];
            tc_ld32(lane_addr + 96, v);
#pragma unroll
            for (int j = 0; j < 32; j++) G[kPW3 + r * kHid + 32 + j] = v[j];
            tc_ld4(lane_addr + 192, t4);
            G[kPB3 + r] = t4[0];
            // dW1 row o = r (columns 256, 257), db1 (column 258)
            tc_ld4(lane_addr + 256, t4);
            G[kPW1 + 2 * r] = t4[0];
            G[kPW1 + 2 * r + 1] = t4[1];
            G[kPB1 + r] = t4[2];
        } else {  // lane r = 64 + output o of layer 2 (columns 128 .. 191: dW2 row, 192: db2)
            const int o = r - 64;
            float v[32], t4[4];
            tc_ld32(lane_addr + 128, v);
#pragma unroll
            for (int j = 0; j < 32; j++) G[kPW2 + o * kHid + j] = v[j];
            tc_ld32(lane_addr + 160, v);
#pragma unroll
            for (int j = 0; j < 32; j++) G[kPW2 + o * kHid + 32 + j] = v[j];
            tc_ld4(lane_addr + 192, t4);
            G[kPB2 + o] = t4[0];
            if (warp == 2) {  // lane 64 holds dy: dw4 (columns 272 .. 335), db4 (column 258)
                tc_ld4(lane_addr + 256, t4);
                float u[32], w[32];
                tc_ld32(lane_addr + 272, u);
                tc_ld32(lane_addr + 304, w);
                if (r == 64) {
                    G[kPB4] = t4[2];
#pragma unroll
                    for (int j = 0; j < 32; j++) {
                        G[kPW4 + j] = u[j];
                        G[kPW4 + 32 + j] = w[j];
                    }
                }
            }
        }
    }
    // squared-error sum of the CTA
    float e2 = err * err;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) e2 += __shfl_xor_sync(0xffffffffu, e2, d);
    if ((r & 31) == 0) S.loss[warp] = e2;
    tc_fence_before();
    __syncthreads();
    if (r == 0) {
        A.loss[blockIdx.x] = S.loss[0] + S.loss[1] + S.loss[2] + S.loss[3];
        if (S.abort) atomicExch(A.status, 1);
    }
    if (S.abort) mbar_wait(&S.mbar, phase);  // the group in flight, once more (bounded)
    __syncthreads();
    tc_fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

// ---------------------------------------------------------------------------------------
// Adam on the FP32 master parameters from the CTAs' gradient sums (added in CTA order), and
// the BF16 operand images for the next step.  One thread per parameter.
struct AdamArgs {
    float *param, *m, *v;
    const float *grad;
    int nparts;
    float lr, beta1, beta2, eps, bc1, bc2;  // bc = 1 - beta^t
    uint8_t *img;
};

__device__ __forceinline__ void write_images(uint8_t *img, int p, float w)
{
    const uint16_t b = bf16_bits(w);
    if (p < kPB1) {
        const int o = (p - kPW1) >> 1, i = (p - kPW1) & 1;
        *reinterpret_cast<uint16_t *>(img + kImgW1 + kmajor_off(o, i, 16)) = b;
    } else if (p >= kPW2 && p < kPB2) {
        const int o = (p - kPW2) / kHid, i = (p - kPW2) % kHid;
        *reinterpret_cast<uint16_t *>(img + kImgW2 + kmajor_off(o, i, kHid)) = b;
        *reinterpret_cast<uint16_t *>(img + kImgW2T + kmajor_off(i, o, kHid)) = b;
    } else if (p >= kPW3 && p < kPB3) {
        const int o = (p - kPW3) / kHid, i = (p - kPW3) % kHid;
        *reinterpret_cast<uint16_t *>(img + kImgW3 + kmajor_off(o, i, kHid)) = b;
        *reinterpret_cast<uint16_t *>(img + kImgW3T + kmajor_off(i, o, kHid)) = b;
    }
}

__global__ void mlp_adam_kernel(const AdamArgs A)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    float g = 0.0f;
    for (int c = 0; c < A.nparts; c++) g += A.grad[(size_t)c * kParams + p];
    const float m = A.beta1 * A.m[p] + (1.0f - A.beta1) * g;
    const float v = A.beta2 * A.v[p] + (1.0f - A.beta2) * g * g;
    A.m[p] = m;
    A.v[p] = v;
    const float w = A.param[p] - A.lr * (m / A.bc1) / (sqrtf(v / A.bc2) + A.eps);
    A.param[p] = w;
    write_images(A.img, p, w);
}

// the images from the parameters (no update): after set_params and at creation
__global__ void mlp_images_kernel(const float *param, uint8_t *img)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < kParams) write_images(img, p, param[p]);
}

// the gradient of one batch (no update): the CTAs' sums added in CTA order
__global__ void mlp_grad_sum_kernel(const float *grad, int nparts, float *out)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    float g = 0.0f;
    for (int c = 0; c < nparts; c++) g += grad[(size_t)c * kParams + p];
    out[p] = g;
}

// ---------------------------------------------------------------------------------------
// Samples: (e, M) uniform over the head's domain from a counter-based generator, the anomaly
// from a bracketed Newton iteration in FP64 (the plain solver's equations), the network's
// inputs and target scaled as the learned step scales them (bia_learned.cuh).
__device__ __forceinline__ unsigned long long mix64(unsigned long long z)
{
    z += 0x9E3779B97F4A7C15ull;  // splitmix64 (Steele, Lea and Flood 2014)
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ double unit_double(unsigned long long seed, unsigned long long k)
{
    return (double)(mix64(seed ^ mix64(k)) >> 11) * (1.0 / 9007199254740992.0);  // [0, 1)
}

// E - e sin E = M on [M, min(M + e, pi)] for M in [0, pi]
__device__ double kepler_elliptic(double e, double M)
{
    double lo = M, hi = fmin(M + e, kPi);
    double x = fmin(fmax(M + e * sin(M), lo), hi);
    for (int it = 0; it < 100; it++) {
        double s, c;
        sincos(x, &s, &c);
        const double f = x - e * s - M;
        if (f == 0.0) break;
        if (f < 0.0) lo = x; else hi = x;
        double xn = x - f / (1.0 - e * c);
        if (!(xn > lo && xn < hi)) xn = 0.5 * (lo + hi);
        if (xn == x) break;
        x = xn;
    }
    return x;
}

// e sinh H - H = M on [0, max(asinh((M + 10)/e) + 1, cbrt(6 M) + 1)] for M >= 0
__device__ double kepler_hyperbolic(double e, double M)
{
    double lo = 0.0, hi = fmax(asinh((M + 10.0) / e) + 1.0, cbrt(6.0 * M) + 1.0);
    double x = fmin(fmax(asinh(M / e), lo), hi);
    for (int it = 0; it < 200; it++) {
        const double f = e * sinh(x) - x - M;
        if (f == 0.0) break;
        if (f < 0.0) lo = x; else hi = x;
        double xn = x - f / (e * cosh(x) - 1.0);
        if (!(xn > lo && xn < hi)) xn = 0.5 * (lo + hi);
        if (xn == x) break;
        x = xn;
    }
    return x;
}

__global__ void mlp_samples_kernel(int head, long long n, unsigned long long seed, float *x, float *y)
{
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double u1 = unit_double(seed, 2ull * (unsigned long long)k);
    const double u2 = unit_double(seed, 2ull * (unsigned long long)k + 1ull);
    if (head == kHeadEll) {
        const double e = (double)kEllEMax * u1, M = kPi * u2;
        const double E = kepler_elliptic(e, M);
        x[2 * k] = (float)(2.0 * e / (double)kEllEMax - 1.0);
        x[2 * k + 1] = (float)(2.0 * M / kPi - 1.0);
        y[k] = (float)(E / kPi);
    } else {
        const double e = (double)kHypEMin + ((double)kHypEMax - (double)kHypEMin) * u1;
        const double M = (double)kHypMMax * u2;
        const double H = kepler_hyperbolic(e, M);
        x[2 * k] = (float)(2.0 * log(e) / log((double)kHypEMax) - 1.0);
        x[2 * k + 1] = (float)(2.0 * log1p(M) / log1p((double)kHypMMax) - 1.0);
        y[k] = (float)(H / (double)kHypOut);
    }
}

// torch.nn.Linear's default initialisation: weights and biases uniform in
// [-1/sqrt(fan_in), 1/sqrt(fan_in)]
__global__ void mlp_init_kernel(unsigned long long seed, float *param)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    const double fan_in = (p < kPW2) ? 2.0 : 64.0;
    const double bound = 1.0 / sqrt(fan_in);
    param[p] = (float)(bound * (2.0 * unit_double(seed ^ 0x5EEDull, (unsigned long long)p) - 1.0));
}

}  // namespace bia

// ---------------------------------------------------------------------------------------
using namespace bia;

struct bia_trainer {
    int device = 0;
    cudaStream_t stream = nullptr;
    int head = 0;
    long long n = 0;
    unsigned long long seed = 0;
    float *x = nullptr, *y = nullptr;             // samples
    float *param = nullptr, *m = nullptr, *v = nullptr;
    uint8_t *img = nullptr;
    float *grad = nullptr;                        // [max_ctas][kParams]
    float *gsum = nullptr;                        // [kParams]
    float *loss = nullptr;                        // [loss_cap]
    int *status = nullptr;
    int max_ctas = 0;
    long long loss_cap = 0;
    long long t = 0;                              // Adam steps taken
};

namespace {

// Once per device (the current one): the training kernel's dynamic shared-memory opt-in.
int trainer_setup_kernel()
{
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static bool done_of[kMaxDevices] = {};
    static bool ok_of[kMaxDevices] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 0;
    std::lock_guard<std::mutex> lk(mu);
    if (!done_of[dev]) {
        ok_of[dev] = cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)kTrainSmemBytes) == cudaSuccess;
        if (!ok_of[dev]) cudaGetLastError();
        done_of[dev] = true;
    }
    return ok_of[dev] ? 1 : 0;
}

void trainer_free(bia_trainer *t)
{
    void *ptrs[] = {t->x, t->y, t->param, t->m, t->v, t->img, t->grad, t->gsum, t->loss, t->status};
    for (void *p : ptrs)
        if (p) cudaFree(p);
}

// grows the gradient and loss buffers for `ctas` CTAs per launch and `slots` loss entries
cudaError_t trainer_reserve(bia_trainer *t, int ctas, long long slots)
{
    cudaError_t e = cudaSuccess;
    if (ctas > t->max_ctas) {
        if (t->grad) cudaFree(t->grad);
        t->grad = nullptr;
        e = cudaMalloc(&t->grad, (size_t)ctas * kParams * sizeof(float));
        if (e != cudaSuccess) return e;
        t->max_ctas = ctas;
    }
    if (slots > t->loss_cap) {
        if (t->loss) cudaFree(t->loss);
        t->loss = nullptr;
        e = cudaMalloc(&t->loss, (size_t)slots * sizeof(float));
        if (e != cudaSuccess) return e;
        t->loss_cap = slots;
    }
    return e;
}

uint16_t host_bf16(float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    const uint32_t r = ((u >> 16) & 1u) + 0x7FFFu;
    return (uint16_t)((u + r) >> 16);
}

unsigned long long host_mix64(unsigned long long z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

int launch_train(bia_trainer *t, const float *x, const float *y, long long n, long long row0, int ctas,
                 unsigned long long mul, unsigned long long add, float dy_scale, float *loss)
{
    TrainArgs A;
    A.x = x; A.y = y; A.n = n; A.row0 = row0;
    A.perm_mul = mul; A.perm_add = add;
    A.dy_scale = dy_scale;
    A.img = t->img; A.vec = t->param;
    A.grad = t->grad; A.loss = loss; A.status = t->status;
    mlp_train_kernel<<<ctas, kTrainThreads, kTrainSmemBytes, t->stream>>>(A);
    return cuda_status(cudaGetLastError());
}

int read_status(bia_trainer *t)
{
    int h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, t->status, sizeof(int), cudaMemcpyDeviceToHost, t->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
    if (e != cudaSuccess) return cuda_status(e);
    return h ? BIA_ERR_DEVICE_TIMEOUT : BIA_OK;
}

}  // namespace

extern "C" {

int bia_trainer_create(bia_context *ctx, int head, long long nsamples, unsigned long long seed, bia_trainer **out)
{
    if (!ctx || !out || (head != kHeadEll && head != kHeadHyp) || nsamples < 1) return BIA_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_status(e);
    if (!trainer_setup_kernel()) return BIA_ERR_CUDA;
    bia_trainer *t = new bia_trainer();
    t->device = ctx->device;
    t->stream = ctx->stream;
    t->head = head;
    t->n = nsamples;
    t->seed = seed;
    e = cudaMalloc(&t->x, (size_t)nsamples * 2 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&t->y, (size_t)nsamples * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&t->param, kParams * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&t->m, kParams * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&t->v, kParams * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&t->img, kImgBytes);
    if (e == cudaSuccess) e = cudaMalloc(&t->gsum, kParams * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&t->status, sizeof(int));
    if (e == cudaSuccess) e = cudaMemsetAsync(t->m, 0, kParams * sizeof(float), t->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(t->v, 0, kParams * sizeof(float), t->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(t->img, 0, kImgBytes, t->stream);  // W1 padding stays 0
    if (e == cudaSuccess) e = cudaMemsetAsync(t->status, 0, sizeof(int), t->stream);
    if (e != cudaSuccess) {
        trainer_free(t);
        delete t;
        return cuda_status(e);
    }
    const unsigned sb = (unsigned)((nsamples + 255) / 256);
    mlp_samples_kernel<<<sb, 256, 0, t->stream>>>(head, nsamples, seed, t->x, t->y);
    mlp_init_kernel<<<(kParams + 255) / 256, 256, 0, t->stream>>>(seed, t->param);
    mlp_images_kernel<<<(kParams + 255) / 256, 256, 0, t->stream>>>(t->param, t->img);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
    if (e != cudaSuccess) {
        trainer_free(t);
        delete t;
        return cuda_status(e);
    }
    *out = t;
    return BIA_OK;
}

int bia_trainer_destroy(bia_trainer *t)
{
    if (!t) return BIA_OK;
    cudaSetDevice(t->device);
    cudaStreamSynchronize(t->stream);
    trainer_free(t);
    delete t;
    return BIA_OK;
}

int bia_trainer_get_params(bia_trainer *t, float *params)
{
    if (!t || !params) return BIA_ERR_INVALID_ARGUMENT;
    cudaSetDevice(t->device);
    cudaError_t e = cudaMemcpyAsync(params, t->param, kParams * sizeof(float), cudaMemcpyDeviceToHost, t->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
    return cuda_status(e);
}

int bia_trainer_set_params(bia_trainer *t, const float *params)
{
    if (!t || !params) return BIA_ERR_INVALID_ARGUMENT;
    cudaSetDevice(t->device);
    cudaError_t e = cudaMemcpyAsync(t->param, params, kParams * sizeof(float), cudaMemcpyHostToDevice, t->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(t->m, 0, kParams * sizeof(float), t->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(t->v, 0, kParams * sizeof(float), t->stream);
    if (e != cudaSuccess) return cuda_status(e);
    t->t = 0;
    mlp_images_kernel<<<(kParams + 255) / 256, 256, 0, t->stream>>>(t->param, t->img);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
    return cuda_status(e);
}

int bia_trainer_gradient(bia_trainer *t, const float *x, const float *y, int rows, float *grad, float *loss)
{
    if (!t || !x || !y || !grad || rows < 1) return BIA_ERR_INVALID_ARGUMENT;
    cudaSetDevice(t->device);
    const int ctas = (rows + kTrainRows - 1) / kTrainRows;
    cudaError_t e = trainer_reserve(t, ctas, ctas);
    if (e == cudaSuccess) e = cudaMemsetAsync(t->status, 0, sizeof(int), t->stream);
    if (e != cudaSuccess) return cuda_status(e);
    int st = launch_train(t, x, y, rows, 0, ctas, 0ull, 0ull, 2.0f / (float)rows, t->loss);
    if (st != BIA_OK) return st;
    mlp_grad_sum_kernel<<<(kParams + 255) / 256, 256, 0, t->stream>>>(t->grad, ctas, t->gsum);
    e = cudaGetLastError();
    std::vector<float> l(ctas);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(grad, t->gsum, kParams * sizeof(float), cudaMemcpyDeviceToHost, t->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(l.data(), t->loss, ctas * sizeof(float), cudaMemcpyDeviceToHost, t->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
    if (e != cudaSuccess) return cuda_status(e);
    if (loss) {
        double s = 0.0;
        for (int c = 0; c < ctas; c++) s += l[c];
        *loss = (float)(s / rows);
    }
    return read_status(t);
}

int bia_trainer_train(bia_trainer *t, int epochs, int batch, float lr, float *loss_per_epoch)
{
    if (!t || epochs < 1 || batch < kTrainRows || batch % kTrainRows != 0 || !(lr > 0.0f))
        return BIA_ERR_INVALID_ARGUMENT;
    // a power-of-two sample count split into whole batches: the epoch's order is an affine
    // permutation of the indices modulo n
    if ((t->n & (t->n - 1)) != 0 || t->n % batch != 0) return BIA_ERR_INVALID_ARGUMENT;
    cudaSetDevice(t->device);
    const int ctas = batch / kTrainRows;
    const long long steps = t->n / batch;
    cudaError_t e = trainer_reserve(t, ctas, steps * ctas);
    if (e == cudaSuccess) e = cudaMemsetAsync(t->status, 0, sizeof(int), t->stream);
    if (e != cudaSuccess) return cuda_status(e);
    std::vector<float> l((size_t)(steps * ctas));
    const float beta1 = 0.9f, beta2 = 0.999f;
    for (int ep = 0; ep < epochs; ep++) {
        // cosine annealing over the epochs (the learning rate of epoch ep)
        const float lr_ep = (float)(0.5 * lr * (1.0 + cos(kPi * (double)ep / (double)epochs)));
        const unsigned long long h = host_mix64(t->seed * 0x100000001B3ull + (unsigned long long)ep + 1ull);
        const unsigned long long mul = (h | 1ull) & (unsigned long long)(t->n - 1);
        const unsigned long long add = host_mix64(h) & (unsigned long long)(t->n - 1);
        for (long long s = 0; s < steps; s++) {
            int st = launch_train(t, t->x, t->y, t->n, s * batch, ctas, mul | 1ull, add, 2.0f / (float)batch,
                                  t->loss + s * ctas);
            if (st != BIA_OK) return st;
            t->t++;
            AdamArgs A;
            A.param = t->param; A.m = t->m; A.v = t->v;
            A.grad = t->grad; A.nparts = ctas;
            A.lr = lr_ep; A.beta1 = beta1; A.beta2 = beta2; A.eps = 1e-8f;
            A.bc1 = (float)(1.0 - pow((double)beta1, (double)t->t));
            A.bc2 = (float)(1.0 - pow((double)beta2, (double)t->t));
            A.img = t->img;
            mlp_adam_kernel<<<(kParams + 255) / 256, 256, 0, t->stream>>>(A);
            e = cudaGetLastError();
            if (e != cudaSuccess) return cuda_status(e);
        }
        e = cudaMemcpyAsync(l.data(), t->loss, l.size() * sizeof(float), cudaMemcpyDeviceToHost, t->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
        if (e != cudaSuccess) return cuda_status(e);
        const int st = read_status(t);
        if (st != BIA_OK) return st;
        if (loss_per_epoch) {
            double sum = 0.0;
            for (float v : l) sum += v;
            loss_per_epoch[ep] = (float)(sum / (double)t->n);
        }
    }
    return BIA_OK;
}

int bia_trainer_export(bia_trainer *t, void *record)
{
    if (!t || !record) return BIA_ERR_INVALID_ARGUMENT;
    std::vector<float> p(kParams);
    const int st = bia_trainer_get_params(t, p.data());
    if (st != BIA_OK) return st;
    MlpHead H;
    memset(&H, 0, sizeof(H));
    for (int o = 0; o < kHid; o++) {
        H.w1[o * kMlpK1 + 0] = host_bf16(p[kPW1 + 2 * o]);
        H.w1[o * kMlpK1 + 1] = host_bf16(p[kPW1 + 2 * o + 1]);
        for (int i = 0; i < kHid; i++) {
            H.w2[o * kHid + i] = host_bf16(p[kPW2 + o * kHid + i]);
            H.w3[o * kHid + i] = host_bf16(p[kPW3 + o * kHid + i]);
        }
        H.b1[o] = p[kPB1 + o];
        H.b2[o] = p[kPB2 + o];
        H.b3[o] = p[kPB3 + o];
        H.w4[o] = p[kPW4 + o];
    }
    H.b4[0] = p[kPB4];
    memcpy(record, &H, sizeof(H));
    return BIA_OK;
}

int bia_trainer_samples(bia_trainer *t, const float **x, const float **y, long long *n)
{
    if (!t || !x || !y || !n) return BIA_ERR_INVALID_ARGUMENT;
    *x = t->x;
    *y = t->y;
    *n = t->n;
    return BIA_OK;
}

int bia_trainer_copy_samples(bia_trainer *t, long long first, long long count, float *x, float *y)
{
    if (!t || !x || !y || first < 0 || count < 0 || first + count > t->n) return BIA_ERR_INVALID_ARGUMENT;
    cudaSetDevice(t->device);
    cudaError_t e = cudaMemcpyAsync(x, t->x + 2 * first, (size_t)count * 2 * sizeof(float), cudaMemcpyDeviceToHost,
                                    t->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(y, t->y + first, (size_t)count * sizeof(float), cudaMemcpyDeviceToHost, t->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
    return cuda_status(e);
}

int bia_trainer_param_count(void) { return kParams; }

}  // extern "C"
