// bia_row.cu -- drop-in replacement of the reference's per-particle entry
// find_dxyuv_kernel_ (bia/find_dXYUV_kernel.cu:526-561), called once per particle i
// by bia/bia.f90:135,138.
//
// Semantics kept: for the fixed 1-based particle I and every j > I the pair given by
// the host AoS array RXYZUVW (x_i-x_j, ..., w_i-w_j) is solved, dXYZUVW[6j+k] receives
// the half-displacement and the host arrays dX..dW are accumulated in place
// (dX[i] += h_j, dX[j] -= h_j).  Unlike the reference, device buffers are kept across
// calls (one set per host thread) instead of a cudaMalloc/cudaFree pair per call, the
// row sum for i is reduced on the device, and entries j <= i of dXYZUVW are zero.
#include <cuda_runtime.h>

#include "bia_internal.cuh"
#include "bia_pair.cuh"

namespace bia {

struct RowArgs {
    const double *rel;  // AoS [6n]
    double *out;        // AoS [6n]
    double *rowsum;     // [6]: sum over j of h_j
    unsigned long long *stats;
    int n, i;
    double eps_th;
    PairParams P;
};

template <int M>
__global__ void __launch_bounds__(128) bia_row_kernel(const RowArgs A)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    PairCounters cnt;
    counters_zero(cnt);
    double h[6] = {0, 0, 0, 0, 0, 0};
    if (j > A.i && j < A.n) {
        const double *s = A.rel + (size_t)6 * j;
        const double r[3] = {s[0], s[1], s[2]};
        const double g[3] = {s[3], s[4], s[5]};
        pair_halfdisp<M>(A.P, A.eps_th, r, g, h, cnt);
    }
    if (j < A.n) {
#pragma unroll
        for (int c = 0; c < 6; c++) A.out[(size_t)6 * j + c] = h[c];
    }
    const unsigned full = 0xffffffffu;
#pragma unroll
    for (int c = 0; c < 6; c++) {
        double v = h[c];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(full, v, off);
        if (lane == 0 && v != 0.0) atomicAdd(&A.rowsum[c], v);
    }
    int vals[kNumStats] = {cnt.cls[0], cnt.cls[1], cnt.cls[2], cnt.cls[3], cnt.cls[4], cnt.cls[5],
                           cnt.it_hyp, cnt.it_ell, cnt.it_par, cnt.it_uv, cnt.rkf_steps,
                           cnt.nonconverged, cnt.bracket_exits, cnt.fallbacks, cnt.nonfinite,
                           cnt.learned, cnt.learned_fallbacks, cnt.learned_coarse, cnt.timeouts, cnt.learned_fp32};
#pragma unroll
    for (int k = 0; k < kNumStats; k++) {
        int s = __reduce_add_sync(full, vals[k]);
        if (lane == 0 && s != 0) atomicAdd(&A.stats[k], (unsigned long long)s);
    }
}

// Per-host-thread device buffers of the drop-in entry (grown on demand).
struct RowState {
    int device = -1;
    DeviceBuffer rel, out, scratch;
    double *h_rowsum = nullptr;
    unsigned long long *h_stats = nullptr;
    ~RowState()
    {
        // buffers die with the process; freeing here could run after the CUDA
        // runtime has shut down
    }
};
static thread_local RowState g_row;

}  // namespace bia

using namespace bia;

extern "C" void find_dxyuv_kernel_(const int METHOD, const int N, const int I, const double EPS,
                                   const double DT, const int ITR, double *dX, double *dY, double *dZ,
                                   double *dU, double *dV, double *dW, double *RXYZUVW,
                                   double *dXYZUVW)
{
    const int i = I - 1;
    if (N < 1 || i < 0 || i >= N || !RXYZUVW || !dXYZUVW || !dX || !dY || !dZ || !dU || !dV || !dW ||
        (METHOD != 0 && METHOD != 1) || ITR < 1 || ITR > 62) {
        set_last_error(BIA_ERR_INVALID_ARGUMENT);
        return;
    }
    RowState &S = g_row;
    cudaError_t e = cudaSuccess;
    if (S.device < 0) {
        e = cudaGetDevice(&S.device);
        if (e == cudaSuccess) e = cudaMallocHost((void **)&S.h_rowsum, 6 * sizeof(double));
        if (e == cudaSuccess) e = cudaMallocHost((void **)&S.h_stats, kNumStats * sizeof(unsigned long long));
        if (e != cudaSuccess) {
            S.device = -1;
            set_last_error(cuda_status(e));
            return;
        }
    }
    const size_t bytes = (size_t)6 * N * sizeof(double);
    if ((e = S.rel.reserve(bytes)) != cudaSuccess || (e = S.out.reserve(bytes)) != cudaSuccess ||
        (e = S.scratch.reserve(6 * sizeof(double) + kNumStats * sizeof(unsigned long long))) != cudaSuccess) {
        set_last_error(cuda_status(e));
        return;
    }
    double *d_rowsum = (double *)S.scratch.ptr;
    unsigned long long *d_stats = (unsigned long long *)(d_rowsum + 6);
    e = cudaMemcpy(S.rel.ptr, RXYZUVW, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(S.scratch.ptr, 0, 6 * sizeof(double) + kNumStats * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        set_last_error(cuda_status(e));
        return;
    }
    RowArgs A;
    A.rel = (const double *)S.rel.ptr;
    A.out = (double *)S.out.ptr;
    A.rowsum = d_rowsum;
    A.stats = d_stats;
    A.n = N;
    A.i = i;
    A.eps_th = EPS;
    A.P.dt = DT;
    A.P.err = 1e-12;
    A.P.relerr = 0.0;
    A.P.abserr = 1e-16;
    A.P.itr = ITR;
    A.P.method = METHOD;
    if (METHOD == 0)
        bia_row_kernel<kMethodRkf><<<(N + 127) / 128, 128>>>(A);
    else
        bia_row_kernel<kMethodAlg><<<(N + 127) / 128, 128>>>(A);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(dXYZUVW, S.out.ptr, bytes, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(S.h_rowsum, d_rowsum, 6 * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpy(S.h_stats, d_stats, kNumStats * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        set_last_error(cuda_status(e));
        return;
    }
    double *acc[6] = {dX, dY, dZ, dU, dV, dW};
    for (int c = 0; c < 6; c++) acc[c][i] += S.h_rowsum[c];
    for (int j = i + 1; j < N; j++) {
        const double *h = dXYZUVW + (size_t)6 * j;
        for (int c = 0; c < 6; c++) acc[c][j] -= h[c];
    }
    set_last_error(S.h_stats[kStatNonfinite] ? BIA_ERR_NONFINITE : BIA_OK);
}
