// invariance.cu -- conserved quantities of an N-body state on the device, FP64.
//
// Replaces invariance_gpu_ / inv_device / sum_device (bia/invariance.cu:15-110):
// sum x, sum v, sum L = x cross v, KE = sum |v|^2 (no 1/2) and
// PE = eps_th * sum_{i<j} 1/r_ij (bia/Invariance_CPU.f90:8-19), with optional charges
// (q_i q_j / r_ij).  The reference's inv_device gives thread i the whole row j > i
// (triangular imbalance, uncoalesced) and sum_device runs 11 serial sums on one thread
// each.  Here the pair sum uses the step kernel's 32 x 32 warp-blocks over the upper
// triangle with shuffled column data, each warp's partial goes to a fixed slot, and all
// partials are reduced by a tree in fixed order, so the result is reproducible and the
// rounding error grows with log(n) instead of n.
#include <cuda_runtime.h>

#include "bia_internal.cuh"

namespace bia {

constexpr int kInvThreads = 256;
constexpr int kInvWarps = kInvThreads / 32;

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    return v;
}

// per-block partials of the ten one-body sums, order {KE, -, Lx, Ly, Lz, Ua, Va, Wa, Xa, Ya, Za}
__global__ void __launch_bounds__(kInvThreads) inv_onebody_kernel(int n, const double *x, const double *y,
                                                                  const double *z, const double *u,
                                                                  const double *v, const double *w,
                                                                  double *part /* [blocks][11] */)
{
    __shared__ double sh[kInvWarps][11];
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    double s[11];
#pragma unroll
    for (int k = 0; k < 11; k++) s[k] = 0.0;
    if (p < n) {
        const double X = x[p], Y = y[p], Z = z[p], U = u[p], V = v[p], W = w[p];
        s[0] = U * U + V * V + W * W;
        s[2] = Y * W - Z * V;
        s[3] = Z * U - X * W;
        s[4] = X * V - Y * U;
        s[5] = U; s[6] = V; s[7] = W;
        s[8] = X; s[9] = Y; s[10] = Z;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 11; k++) {
        double t = warp_sum(s[k]);
        if (lane == 0) sh[wid][k] = t;
    }
    __syncthreads();
    if (threadIdx.x < 11) {
        double t = 0.0;
        for (int k = 0; k < kInvWarps; k++) t += sh[k][threadIdx.x];
        part[(size_t)blockIdx.x * 11 + threadIdx.x] = t;
    }
}

__device__ __forceinline__ void inv_block_coords(long long t, int &bi, int &bj)
{
    long long c = (long long)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while (c * (c + 1) / 2 > t) c--;
    while ((c + 1) * (c + 2) / 2 <= t) c++;
    bj = (int)c;
    bi = (int)(t - c * (c + 1) / 2);
}

// sum over i<j of (q_i q_j) / r_ij; one warp per 32 x 32 block, one partial per CTA
__global__ void __launch_bounds__(kInvThreads) inv_pairs_kernel(int n, long long nwb, const double *x,
                                                                const double *y, const double *z,
                                                                const double *q, double *part)
{
    __shared__ double sh[kInvWarps];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const long long t = (long long)blockIdx.x * kInvWarps + wid;
    double acc = 0.0;
    if (t < nwb) {
        int bi, bj;
        inv_block_coords(t, bi, bj);
        const int i = bi * 32 + lane, jo = bj * 32 + lane;
        const bool iv = i < n, jv = jo < n;
        const double xi = iv ? x[i] : 0.0, yi = iv ? y[i] : 0.0, zi = iv ? z[i] : 0.0;
        const double qi = (iv && q) ? q[i] : 1.0;
        const double xj = jv ? x[jo] : 0.0, yj = jv ? y[jo] : 0.0, zj = jv ? z[jo] : 0.0;
        const double qj = (jv && q) ? q[jo] : 1.0;
        const bool diag = bi == bj;
        const int k0 = diag ? 1 : 0, k1 = diag ? 16 : 31;
        for (int k = k0; k <= k1; k++) {
            const int src = (lane + k) & 31;
            const double cx = __shfl_sync(full, xj, src);
            const double cy = __shfl_sync(full, yj, src);
            const double cz = __shfl_sync(full, zj, src);
            const double cq = __shfl_sync(full, qj, src);
            const int j = bj * 32 + src;
            if ((!diag || k < 16 || lane < 16) && iv && j < n) {
                const double dx = xi - cx, dy = yi - cy, dz = zi - cz;
                const double w = 1.0 / sqrt(dx * dx + dy * dy + dz * dz);
                acc += q ? qi * cq * w : w;
            }
        }
    }
    acc = warp_sum(acc);
    if (lane == 0) sh[wid] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < kInvWarps; k++) s += sh[k];
        part[blockIdx.x] = s;
    }
}

// fixed-order tree reduction of `count` groups of `width` values: out[k] = sum_g in[g*width+k]
__global__ void __launch_bounds__(1024) inv_final_kernel(const double *in, long long count, int width,
                                                         double *out)
{
    __shared__ double sh[32];
    for (int k = 0; k < width; k++) {
        double s = 0.0;
        for (long long g = threadIdx.x; g < count; g += blockDim.x) s += in[g * width + k];
        s = warp_sum(s);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x < 32) {
            double t = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
            t = warp_sum(t);
            if (threadIdx.x == 0) out[k] = t;
        }
        __syncthreads();
    }
}

// Enqueue the invariants of device SoA state into out_dev[12] (11 values, slot 1 = raw
// pair sum before the eps_th factor).  scratch must hold inv_scratch_doubles(n).
size_t inv_scratch_doubles(int n)
{
    const long long nb = (n + 31) / 32;
    const long long nwb = nb * (nb + 1) / 2;
    const long long pair_blocks = (nwb + kInvWarps - 1) / kInvWarps;
    const long long one_blocks = (n + kInvThreads - 1) / kInvThreads;
    return (size_t)(one_blocks * 11 + pair_blocks + 16);
}

cudaError_t enqueue_invariance(cudaStream_t st, int n, const double *x, const double *y, const double *z,
                               const double *u, const double *v, const double *w, const double *q,
                               double *scratch, double *out_dev)
{
    const long long nb = (n + 31) / 32;
    const long long nwb = nb * (nb + 1) / 2;
    const long long pair_blocks = (nwb + kInvWarps - 1) / kInvWarps;
    const int one_blocks = (n + kInvThreads - 1) / kInvThreads;
    double *p1 = scratch;
    double *p2 = scratch + (size_t)one_blocks * 11;
    inv_onebody_kernel<<<one_blocks, kInvThreads, 0, st>>>(n, x, y, z, u, v, w, p1);
    inv_pairs_kernel<<<(unsigned)pair_blocks, kInvThreads, 0, st>>>(n, nwb, x, y, z, q, p2);
    inv_final_kernel<<<1, 1024, 0, st>>>(p1, one_blocks, 11, out_dev);
    inv_final_kernel<<<1, 1024, 0, st>>>(p2, pair_blocks, 1, out_dev + 11);
    return cudaGetLastError();
}

struct InvDropInState {
    int ready = 0;
    DeviceBuffer state, scratch;
    double *h_out = nullptr;
};
static thread_local InvDropInState g_inv;

}  // namespace bia

using namespace bia;

extern "C" int bia_invariance(bia_context *ctx, int n, double eps_th, const double *x, const double *y,
                              const double *z, const double *u, const double *v, const double *w,
                              const double *q, double out[11])
{
    if (!ctx || n < 1 || !x || !y || !z || !u || !v || !w || !out) return BIA_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    const size_t need = inv_scratch_doubles(n) + 12;
    cudaError_t e = ctx->inv.reserve(need * sizeof(double));
    if (e != cudaSuccess) return cuda_status(e);
    double *scratch = (double *)ctx->inv.ptr;
    double *res = scratch + inv_scratch_doubles(n);
    e = enqueue_invariance(ctx->stream, n, x, y, z, u, v, w, q, scratch, res);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ctx->h_inv, res, 12 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_status(e);
    for (int k = 0; k < 11; k++) out[k] = ctx->h_inv[k];
    out[1] = eps_th * ctx->h_inv[11];
    return BIA_OK;
}

extern "C" void invariance_gpu_(const int N, const double eps_th, double *X, double *Y, double *Z, double *U,
                                double *V, double *W, double *KE, double *PE, double *Lx, double *Ly,
                                double *Lz, double *Ua, double *Va, double *Wa, double *Xa, double *Ya,
                                double *Za)
{
    if (N < 1 || !X || !Y || !Z || !U || !V || !W || !KE || !PE || !Lx || !Ly || !Lz || !Ua || !Va || !Wa ||
        !Xa || !Ya || !Za) {
        set_last_error(BIA_ERR_INVALID_ARGUMENT);
        return;
    }
    InvDropInState &S = g_inv;
    cudaError_t e = cudaSuccess;
    if (!S.ready) {
        e = cudaMallocHost((void **)&S.h_out, 12 * sizeof(double));
        if (e != cudaSuccess) {
            set_last_error(cuda_status(e));
            return;
        }
        S.ready = 1;
    }
    const size_t need = inv_scratch_doubles(N) + 12;
    if ((e = S.state.reserve((size_t)6 * N * sizeof(double))) != cudaSuccess ||
        (e = S.scratch.reserve(need * sizeof(double))) != cudaSuccess) {
        set_last_error(cuda_status(e));
        return;
    }
    double *d = (double *)S.state.ptr;
    double *host[6] = {X, Y, Z, U, V, W};
    for (int k = 0; k < 6 && e == cudaSuccess; k++)
        e = cudaMemcpy(d + (size_t)k * N, host[k], N * sizeof(double), cudaMemcpyHostToDevice);
    double *scratch = (double *)S.scratch.ptr;
    double *res = scratch + inv_scratch_doubles(N);
    if (e == cudaSuccess)
        e = enqueue_invariance(0, N, d, d + N, d + 2 * (size_t)N, d + 3 * (size_t)N, d + 4 * (size_t)N,
                               d + 5 * (size_t)N, nullptr, scratch, res);
    if (e == cudaSuccess) e = cudaMemcpy(S.h_out, res, 12 * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        set_last_error(cuda_status(e));
        return;
    }
    const double *o = S.h_out;
    *KE = o[0];
    *PE = eps_th * o[11];
    *Lx = o[2]; *Ly = o[3]; *Lz = o[4];
    *Ua = o[5]; *Va = o[6]; *Wa = o[7];
    *Xa = o[8]; *Ya = o[9]; *Za = o[10];
    set_last_error(BIA_OK);
}
