// dim_rkf.cu -- the direct-integration (DIM) FP64 reference solver on the device.
//
// Rebuilds dim/rkf_kernel.cu: all 6n equations y' = (v, a) with the direct-sum
// acceleration a_i = eps sum_j (r_i - r_j) / (|r_ij|^2 + 1e-99)^{3/2}
// (dim/rkf_kernel.cu:29-53) integrated from x0 to xe by the Fehlberg 4(5) pair with
// step doubling and the reference's adaptive control (dim/rkf_kernel.cu:194-495):
// the "low" track advances by one step h with the embedded error estimate, the "high"
// track by two steps h/2; a step is accepted when max_i |er_i| / et_i <= 1.
//
// Differences from the reference, none of which changes the scheme:
//  * the state stays on the device for the whole integration; per attempted step the
//    host reads one double (the error norm) instead of copying the 11*6n work array
//    both ways (dim/rkf_kernel.cu:290-292,485-489);
//  * the acceleration sum over j is split into 8 fixed chunks whose partial sums are
//    added in order (deterministic; the association differs from the reference's single
//    running sum by rounding only);
//  * errors set IER (10000 too many steps, 20000 zero tolerance, 30000 step underflow)
//    and return instead of calling exit(0) (dim/rkf_kernel.cu:298-315,491-494).
// Layout: SoA, component-major, 6 arrays of n (x, y, z, u, v, w).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "bia_internal.cuh"

namespace bia {

constexpr int kDimChunks = 8;
constexpr int kDimParticlesPerBlock = 32;

// Fehlberg coefficients (dim/rkf_kernel.cu:161-168); stage s (1..5) forms
// w_s = y0 + h * sum_m B[s][m] k_m, the 6th line forms yn with GA, the 7th er with DA.
__constant__ double c_fehl[7][6] = {
    {1.0 / 4, 0, 0, 0, 0, 0},
    {3.0 / 32, 9.0 / 32, 0, 0, 0, 0},
    {1932.0 / 2197, -7200.0 / 2197, 7296.0 / 2197, 0, 0, 0},
    {439.0 / 216, -8.0, 3680.0 / 513, -845.0 / 4104, 0, 0},
    {-8.0 / 27, 2.0, -3544.0 / 2565, 1859.0 / 4104, -11.0 / 40, 0},
    {16.0 / 135, 0, 6656.0 / 12825, 28561.0 / 56430, -9.0 / 50, 2.0 / 55},
    {1.0 / 360, 0, -128.0 / 4275, -2197.0 / 75240, 1.0 / 50, 2.0 / 55},
};

// k_out = (v, a)(y_in).  Block: 32 particles x 8 j-chunks; the chunk partial sums are
// added in chunk order.
__global__ void __launch_bounds__(kDimParticlesPerBlock * kDimChunks) dim_accel_kernel(
    int n, double eps, const double *__restrict__ yin, double *__restrict__ kout)
{
    __shared__ double part[kDimChunks][3][kDimParticlesPerBlock];
    const int lane = threadIdx.x % kDimParticlesPerBlock;
    const int chunk = threadIdx.x / kDimParticlesPerBlock;
    const int i = blockIdx.x * kDimParticlesPerBlock + lane;
    const double *X = yin, *Y = yin + n, *Z = yin + 2 * (size_t)n;
    double ax = 0.0, ay = 0.0, az = 0.0;
    if (i < n) {
        const double xi = X[i], yi = Y[i], zi = Z[i];
        const int per = (n + kDimChunks - 1) / kDimChunks;
        const int j0 = chunk * per;
        const int j1 = min(n, j0 + per);
        for (int j = j0; j < j1; j++) {
            const double xij = xi - X[j], yij = yi - Y[j], zij = zi - Z[j];
            const double rsq = xij * xij + yij * yij + zij * zij + 1e-99;
            const double eee = eps / (rsq * sqrt(rsq));
            ax += xij * eee;
            ay += yij * eee;
            az += zij * eee;
        }
    }
    part[chunk][0][lane] = ax;
    part[chunk][1][lane] = ay;
    part[chunk][2][lane] = az;
    __syncthreads();
    if (chunk == 0 && i < n) {
        double s[3] = {0.0, 0.0, 0.0};
        for (int c = 0; c < kDimChunks; c++)
            for (int d = 0; d < 3; d++) s[d] += part[c][d][lane];
        kout[i] = yin[3 * (size_t)n + i];
        kout[(size_t)n + i] = yin[4 * (size_t)n + i];
        kout[2 * (size_t)n + i] = yin[5 * (size_t)n + i];
        kout[3 * (size_t)n + i] = s[0];
        kout[4 * (size_t)n + i] = s[1];
        kout[5 * (size_t)n + i] = s[2];
    }
}

// out = y0 + h * sum_{m < nk} c_fehl[row][m] k_m  (row 0..5), or er = h * sum (row 6)
__global__ void __launch_bounds__(256) dim_combine_kernel(int len, int row, int nk, bool add_y0,
                                                          const double *__restrict__ hdev,
                                                          const double *__restrict__ y0,
                                                          const double *__restrict__ k, double *__restrict__ out)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= len) return;
    const double h = *hdev;
    double acc;
    if (row == 0) {
        acc = h * c_fehl[0][0] * k[e];  // (h * B21) * k1, dim/rkf_kernel.cu:82
    } else {
        acc = 0.0;
        for (int m = 0; m < nk; m++) acc += c_fehl[row][m] * k[(size_t)m * len + e];
        acc = h * acc;
    }
    out[e] = add_y0 ? y0[e] + acc : acc;
}

// per-block max of |er| / et with et = relerr (|yl0| + |yln|) / 2 + abserr; a zero et
// is flagged by a negative result
__global__ void __launch_bounds__(256) dim_errnorm_kernel(int len, double relerr, double abserr,
                                                          const double *__restrict__ yl0,
                                                          const double *__restrict__ yln,
                                                          const double *__restrict__ er, double *__restrict__ blockmax)
{
    __shared__ double sh[256];
    double m = 0.0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < len; e += gridDim.x * blockDim.x) {
        const double et = relerr * (fabs(yl0[e]) + fabs(yln[e])) / 2 + abserr;
        if (et == 0.0) m = -1.0e300;
        else if (m >= 0.0) m = fmax(m, fabs(er[e]) / et);
    }
    sh[threadIdx.x] = m;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            const double a = sh[threadIdx.x], b = sh[threadIdx.x + s];
            sh[threadIdx.x] = (a < 0.0 || b < 0.0) ? -1.0e300 : fmax(a, b);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) blockmax[blockIdx.x] = sh[0];
}

// min over i with |k1_i| > 0 of |(relerr |y_i| + abserr) / k1_i| (initial step size,
// dim/rkf_kernel.cu:248-261); +inf when no k1_i is nonzero
__global__ void __launch_bounds__(256) dim_toldy_kernel(int len, double relerr, double abserr,
                                                        const double *__restrict__ y, const double *__restrict__ k1,
                                                        double *__restrict__ blockmin)
{
    __shared__ double sh[256];
    double m = INFINITY;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < len; e += gridDim.x * blockDim.x) {
        if (fabs(k1[e]) > 0.0) m = fmin(m, fabs((relerr * fabs(y[e]) + abserr) / k1[e]));
    }
    sh[threadIdx.x] = m;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] = fmin(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) blockmin[blockIdx.x] = sh[0];
}

__global__ void dim_final_reduce_kernel(int count, bool take_max, const double *__restrict__ in, double *out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double m = take_max ? 0.0 : INFINITY;
    for (int b = 0; b < count; b++) {
        const double v = in[b];
        if (take_max) m = (m < 0.0 || v < 0.0) ? -1.0e300 : fmax(m, v);
        else m = fmin(m, v);
    }
    *out = m;
}

__global__ void __launch_bounds__(256) dim_esterr_kernel(int len, const double *__restrict__ yln,
                                                         const double *__restrict__ yhn, double *__restrict__ ese)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < len) ese[e] = (yln[e] - yhn[e]) / 31;
}

constexpr int kDimReduceBlocks = 148;
constexpr int kDimCoopMaxBlocks = 1024;  // partials of the cooperative solver's reductions

// Device buffers of one integration: 6n doubles each for yl0, yln, yh0, yhm, yhn, er, w
// and 6 x 6n for k1..k6; plus reduction scratch and the step size.
struct DimBuffers {
    double *yl0, *yln, *yh0, *yhm, *yhn, *er, *w, *wb, *k, *red, *h, *scal, *io;
};

struct DimRun {
    int n, len;
    bool fast_inv = false;  // the cooperative solver's rsqrt-based inverse cube
    double eps, relerr, abserr;
    cudaStream_t st;
    DimBuffers B;
    double *h_pinned;  // [0] h to upload, [1] reduction result read back
};

static unsigned grid_of(int len) { return (unsigned)((len + 255) / 256); }

// One Fehlberg step of size *hdev from y0: yn and (want_er) er (dim/rkf_kernel.cu fehl).
static cudaError_t dim_fehl(const DimRun &R, const double *y0, double *yn, bool want_er)
{
    const int n = R.n, len = R.len;
    const unsigned ga = (unsigned)((n + kDimParticlesPerBlock - 1) / kDimParticlesPerBlock);
    const unsigned threads = kDimParticlesPerBlock * kDimChunks;
    double *k = R.B.k;
    dim_accel_kernel<<<ga, threads, 0, R.st>>>(n, R.eps, y0, k);
    for (int s = 0; s < 5; s++) {
        dim_combine_kernel<<<grid_of(len), 256, 0, R.st>>>(len, s, s + 1, true, R.B.h, y0, k, R.B.w);
        dim_accel_kernel<<<ga, threads, 0, R.st>>>(n, R.eps, R.B.w, k + (size_t)(s + 1) * len);
    }
    dim_combine_kernel<<<grid_of(len), 256, 0, R.st>>>(len, 5, 6, true, R.B.h, y0, k, yn);
    if (want_er) dim_combine_kernel<<<grid_of(len), 256, 0, R.st>>>(len, 6, 6, false, R.B.h, y0, k, R.B.er);
    return cudaGetLastError();
}

static cudaError_t set_h(const DimRun &R, double h)
{
    R.h_pinned[0] = h;
    return cudaMemcpyAsync(R.B.h, R.h_pinned, sizeof(double), cudaMemcpyHostToDevice, R.st);
}

static cudaError_t read_scalar(const DimRun &R, double *out)
{
    cudaError_t e = cudaMemcpyAsync(R.h_pinned + 1, R.B.scal, sizeof(double), cudaMemcpyDeviceToHost, R.st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(R.st);
    if (e == cudaSuccess) *out = R.h_pinned[1];
    return e;
}

// The adaptive loop of dim/rkf_kernel.cu:194-495 (INIT = 1 computes the first step).
// y (device SoA 6n) holds the state at *x0 on entry and the high track at xe on exit;
// ese (optional device 6n) the final (yln - yhn)/31.  Returns ier.
static int dim_integrate(DimRun &R, double *y, double *x0, double xe, int init, double *H, int *nde,
                         long long *accepted, long long *rejected, double *ese, int *status)
{
    const double EPSMIN = 1e-15;
    const int ITEMAX = 10000;
    const size_t bytes = (size_t)R.len * sizeof(double);
    cudaError_t e;
    *status = BIA_OK;
#define DIM_CHECK(x)                          \
    do {                                      \
        e = (x);                              \
        if (e != cudaSuccess) {               \
            *status = cuda_status(e);         \
            return 0;                         \
        }                                     \
    } while (0)
    DIM_CHECK(cudaMemcpyAsync(R.B.yh0, y, bytes, cudaMemcpyDeviceToDevice, R.st));
    DIM_CHECK(cudaMemcpyAsync(R.B.yl0, y, bytes, cudaMemcpyDeviceToDevice, R.st));
    *nde = 0;
    if (init == 1) {
        const unsigned ga = (unsigned)((R.n + kDimParticlesPerBlock - 1) / kDimParticlesPerBlock);
        dim_accel_kernel<<<ga, kDimParticlesPerBlock * kDimChunks, 0, R.st>>>(R.n, R.eps, R.B.yl0, R.B.k);
        dim_toldy_kernel<<<kDimReduceBlocks, 256, 0, R.st>>>(R.len, R.relerr, R.abserr, R.B.yl0, R.B.k, R.B.red);
        dim_final_reduce_kernel<<<1, 32, 0, R.st>>>(kDimReduceBlocks, false, R.B.red, R.B.scal);
        double toldy = 0.0;
        DIM_CHECK(read_scalar(R, &toldy));
        *H = std::isinf(toldy) ? EPSMIN * (xe - *x0) : fmin((xe - *x0) / 100e0, pow(toldy, 0.2));
        *nde = 1;
    }
    double X = *x0;
    int ier = 10000;
    for (int iter = 0; iter < ITEMAX; iter++) {
        DIM_CHECK(set_h(R, *H));
        DIM_CHECK(dim_fehl(R, R.B.yl0, R.B.yln, true));
        *nde += 6;
        dim_errnorm_kernel<<<kDimReduceBlocks, 256, 0, R.st>>>(R.len, R.relerr, R.abserr, R.B.yl0, R.B.yln,
                                                                 R.B.er, R.B.red);
        dim_final_reduce_kernel<<<1, 32, 0, R.st>>>(kDimReduceBlocks, true, R.B.red, R.B.scal);
        double erret = 0.0;
        DIM_CHECK(read_scalar(R, &erret));
        if (erret < 0.0) {
            ier = 20000;
            break;
        }
        if (erret > 1) {
            (*rejected)++;
            if (erret >= 59049) *H *= 0.1;
            else *H *= 0.9 / pow(erret, 0.2);
            if (*H <= EPSMIN) {
                ier = 30000;
                break;
            }
        } else if (X + *H < xe) {
            // two half steps on the high track (fhstep, dim/rkf_kernel.cu:318-362)
            DIM_CHECK(set_h(R, *H / 2));
            DIM_CHECK(dim_fehl(R, R.B.yh0, R.B.yhm, false));
            DIM_CHECK(dim_fehl(R, R.B.yhm, R.B.yhn, false));
            *nde += 12;
            X += *H;
            *x0 = X;
            DIM_CHECK(cudaMemcpyAsync(R.B.yl0, R.B.yln, bytes, cudaMemcpyDeviceToDevice, R.st));
            DIM_CHECK(cudaMemcpyAsync(R.B.yh0, R.B.yhn, bytes, cudaMemcpyDeviceToDevice, R.st));
            (*accepted)++;
            if (erret <= 1.889568e-4) *H *= 5.0;
            else *H *= 0.9 / pow(erret, 0.2);
        } else {
            // last step to xe (dim/rkf_kernel.cu:386-483)
            *H = xe - X;
            DIM_CHECK(set_h(R, *H));
            DIM_CHECK(dim_fehl(R, R.B.yl0, R.B.yln, true));
            DIM_CHECK(set_h(R, *H / 2));
            DIM_CHECK(dim_fehl(R, R.B.yh0, R.B.yhm, false));
            DIM_CHECK(dim_fehl(R, R.B.yhm, R.B.yhn, false));
            *nde += 18;
            if (ese) dim_esterr_kernel<<<grid_of(R.len), 256, 0, R.st>>>(R.len, R.B.yln, R.B.yhn, ese);
            DIM_CHECK(cudaMemcpyAsync(y, R.B.yhn, bytes, cudaMemcpyDeviceToDevice, R.st));
            DIM_CHECK(cudaMemcpyAsync(R.B.yl0, R.B.yln, bytes, cudaMemcpyDeviceToDevice, R.st));
            *x0 = xe;
            (*accepted)++;
            ier = 0;
            break;
        }
    }
    if (ier != 0) {  // leave the last accepted high-track state in y
        DIM_CHECK(cudaMemcpyAsync(y, R.B.yh0, bytes, cudaMemcpyDeviceToDevice, R.st));
    }
    DIM_CHECK(cudaStreamSynchronize(R.st));
#undef DIM_CHECK
    return ier;
}

static size_t dim_buffer_doubles(int n)
{
    const size_t len = (size_t)6 * n;
    return 8 * len + 6 * len + kDimCoopMaxBlocks + 16;
}

static void dim_carve(double *base, int n, DimBuffers &B)
{
    const size_t len = (size_t)6 * n;
    B.yl0 = base;
    B.yln = base + len;
    B.yh0 = base + 2 * len;
    B.yhm = base + 3 * len;
    B.yhn = base + 4 * len;
    B.er = base + 5 * len;
    B.w = base + 6 * len;
    B.k = base + 7 * len;
    B.wb = base + 13 * len;
    B.red = base + 14 * len;
    B.h = B.red + kDimCoopMaxBlocks;
    B.scal = B.h + 1;
    B.io = B.scal + 2;  // 6 doubles of the cooperative solver's inputs and outputs
}



// ---------------------------------------------------------------------------------------
// The whole adaptive integration in one cooperative kernel: the same stages, arithmetic
// and acceptance rule as dim_integrate below, with the step control on the device.  Every
// block computes the decisions from the same grid-wide reductions (bitwise the same
// values), so all blocks take the same path and meet at the same grid-wide barriers; the
// loop is bounded by ITEMAX attempted steps.  Tracks are swapped, not copied.
namespace cg = cooperative_groups;

struct DimCoopArgs {
    int n, len, init, itemax;
    double eps, relerr, abserr, xe;
    DimBuffers B;   // B.red holds >= gridDim.x doubles
    double *y;      // state in (at io[0]) and out
    double *ese;    // optional (yln - yhn) / 31 of the last step
    double *io;     // in: [0] x0, [1] H; out: [0] x reached, [1] H, [2] nde, [3] accepted,
                    // [4] rejected, [5] ier
};

// Fused stage of the cooperative solver: k_s = (v, a)(win) for a group of P particles, and
// right away, by the thread that owns particle i, the next stage's input for particle i:
// w = y0 + h sum_m c_fehl[s][m] k_m (s < 5), or yn (row 5) and er (row 6) after the last
// stage.  The combination is per particle, so only the next stage needs a grid-wide
// barrier.
//
// j-tiles: the block's 256 threads load the positions of 256 particles j at a time into
// shared memory (coalesced structure-of-arrays loads, one element per thread and
// component); thread (particle lane, chunk c) of the block's P x C threads (C = 256 / P)
// adds the tile's entries c, c + C, ..., and the C chunk sums of a particle are added in
// chunk order at the end (deterministic).  P = 8 below n = 4096 (more groups than SMs at
// small n), 32 above (each tile then serves 32 particles, 32 entries per thread).
//
// Inverse cube: kFastInv (bia_dim_integrate) eps r^-3 from one rsqrt (r^-1, then its cube;
// rsqrt is within 1 ulp, the product within ~4 ulp of eps / r^3); otherwise the
// reference's eps / (rsq sqrt(rsq)) (dim/rkf_kernel.cu:44-46), the form rkf_c_ keeps.
constexpr int kCoopTile = 256;
template <int P>
struct CoopShared {
    double part[256 / P][3][P];
    double tile[3][kCoopTile];
};

template <int P, bool kFastInv>
__device__ void coop_stage(const DimCoopArgs &A, int s, double h, const double *__restrict__ y0,
                           const double *__restrict__ win, double *__restrict__ wout, double *__restrict__ yn,
                           bool want_er, CoopShared<P> &sh)
{
    constexpr int C = 256 / P;
    const int n = A.n;
    const size_t len = (size_t)A.len;
    const int lane = threadIdx.x % P;
    const int chunk = threadIdx.x / P;
    const int ngroups = (n + P - 1) / P;
    const double *X = win, *Y = win + n, *Z = win + 2 * (size_t)n;
    double *k = A.B.k;
    for (int grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
        const int i = grp * P + lane;
        const bool live = i < n;
        const double xi = live ? X[i] : 0.0, yi = live ? Y[i] : 0.0, zi = live ? Z[i] : 0.0;
        double ax = 0.0, ay = 0.0, az = 0.0;
        for (int jt = 0; jt < n; jt += kCoopTile) {
            __syncthreads();  // the previous tile (or group) is consumed
            const int jl = jt + (int)threadIdx.x;
            if (jl < n) {
                sh.tile[0][threadIdx.x] = X[jl];
                sh.tile[1][threadIdx.x] = Y[jl];
                sh.tile[2][threadIdx.x] = Z[jl];
            }
            __syncthreads();
            const int cnt = min(kCoopTile, n - jt);
            if (live) {
                for (int q = chunk; q < cnt; q += C) {
                    const double xij = xi - sh.tile[0][q], yij = yi - sh.tile[1][q], zij = zi - sh.tile[2][q];
                    const double rsq = xij * xij + yij * yij + zij * zij + 1e-99;
                    double eee;
                    if (kFastInv) {
                        const double ir = rsqrt(rsq);
                        eee = A.eps * (ir * ir * ir);
                    } else {
                        eee = A.eps / (rsq * sqrt(rsq));
                    }
                    ax += xij * eee;
                    ay += yij * eee;
                    az += zij * eee;
                }
            }
        }
        sh.part[chunk][0][lane] = ax;
        sh.part[chunk][1][lane] = ay;
        sh.part[chunk][2][lane] = az;
        __syncthreads();
        if (chunk == 0 && live) {
            double a3[3] = {0.0, 0.0, 0.0};
            for (int c = 0; c < C; c++)
                for (int d = 0; d < 3; d++) a3[d] += sh.part[c][d][lane];
            double *ks = k + (size_t)s * len;
            for (int c = 0; c < 3; c++) {
                ks[(size_t)c * n + i] = win[(size_t)(3 + c) * n + i];
                ks[(size_t)(3 + c) * n + i] = a3[c];
            }
            for (int c = 0; c < 6; c++) {
                const size_t e = (size_t)c * n + i;
                if (s < 5) {
                    double acc;
                    if (s == 0) {
                        acc = h * c_fehl[0][0] * k[e];
                    } else {
                        acc = 0.0;
                        for (int m = 0; m <= s; m++) acc += c_fehl[s][m] * k[(size_t)m * len + e];
                        acc = h * acc;
                    }
                    wout[e] = y0[e] + acc;
                } else {
                    double acc = 0.0;
                    for (int m = 0; m < 6; m++) acc += c_fehl[5][m] * k[(size_t)m * len + e];
                    yn[e] = y0[e] + h * acc;
                    if (want_er) {
                        double ae = 0.0;
                        for (int m = 0; m < 6; m++) ae += c_fehl[6][m] * k[(size_t)m * len + e];
                        A.B.er[e] = h * ae;
                    }
                }
            }
        }
    }
    __syncthreads();
}

// One Fehlberg step of size h: six fused stages, one grid-wide barrier after each.
template <int P, bool kFastInv>
__device__ void coop_fehl(const DimCoopArgs &A, cg::grid_group &grid, double h, const double *y0, double *yn,
                          bool want_er, CoopShared<P> &part)
{
    // stage inputs alternate between two scratch vectors so a stage never overwrites the
    // input other blocks are still reading: w_a for even stages' output, w_b for odd
    double *wa = A.B.w, *wb = A.B.wb;
    const double *win = y0;
    for (int st = 0; st < 6; st++) {
        double *wout = (st % 2 == 0) ? wa : wb;
        coop_stage<P, kFastInv>(A, st, h, y0, win, wout, yn, want_er, part);
        grid.sync();
        win = wout;
    }
}

// grid-wide max of |er| / et (negative when an et is zero), the same on every block
__device__ double coop_errnorm(const DimCoopArgs &A, cg::grid_group &grid, const double *yl0, const double *yln,
                               double *sh)
{
    double m = 0.0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < A.len; e += gridDim.x * blockDim.x) {
        const double et = A.relerr * (fabs(yl0[e]) + fabs(yln[e])) / 2 + A.abserr;
        if (et == 0.0) m = -1.0e300;
        else if (m >= 0.0) m = fmax(m, fabs(A.B.er[e]) / et);
    }
    sh[threadIdx.x] = m;
    __syncthreads();
    for (int s2 = 128; s2 > 0; s2 >>= 1) {
        if (threadIdx.x < s2) {
            const double a = sh[threadIdx.x], b = sh[threadIdx.x + s2];
            sh[threadIdx.x] = (a < 0.0 || b < 0.0) ? -1.0e300 : fmax(a, b);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) A.B.red[blockIdx.x] = sh[0];
    grid.sync();
    __shared__ double total;
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int b = 0; b < (int)gridDim.x; b++) {
            const double v = A.B.red[b];
            t = (t < 0.0 || v < 0.0) ? -1.0e300 : fmax(t, v);
        }
        total = t;
    }
    __syncthreads();
    const double r = total;
    __syncthreads();
    return r;
}

template <int P, bool kFastInv>
__global__ void __launch_bounds__(256) dim_coop_kernel(const DimCoopArgs A)
{
    cg::grid_group grid = cg::this_grid();
    __shared__ CoopShared<P> part;
    __shared__ double sh[256];
    __shared__ double total;
    const double EPSMIN = 1e-15;
    const int len = A.len;
    const int gid = blockIdx.x * blockDim.x + threadIdx.x, gsz = gridDim.x * blockDim.x;
    double *yl0 = A.B.yl0, *yln = A.B.yln, *yh0 = A.B.yh0, *yhn = A.B.yhn;
    for (int e = gid; e < len; e += gsz) {
        yh0[e] = A.y[e];
        yl0[e] = A.y[e];
    }
    double X = A.io[0], H = A.io[1];
    int nde = 0;
    grid.sync();
    if (A.init == 1) {
        coop_stage<P, kFastInv>(A, 0, 0.0, yl0, yl0, A.B.wb, nullptr, false, part);  // k1 only (w unused)
        grid.sync();
        double m = INFINITY;
        for (int e = gid; e < len; e += gsz)
            if (fabs(A.B.k[e]) > 0.0) m = fmin(m, fabs((A.relerr * fabs(yl0[e]) + A.abserr) / A.B.k[e]));
        sh[threadIdx.x] = m;
        __syncthreads();
        for (int s2 = 128; s2 > 0; s2 >>= 1) {
            if (threadIdx.x < s2) sh[threadIdx.x] = fmin(sh[threadIdx.x], sh[threadIdx.x + s2]);
            __syncthreads();
        }
        if (threadIdx.x == 0) A.B.red[blockIdx.x] = sh[0];
        grid.sync();
        if (threadIdx.x == 0) {
            double t = INFINITY;
            for (int b = 0; b < (int)gridDim.x; b++) t = fmin(t, A.B.red[b]);
            total = t;
        }
        __syncthreads();
        const double toldy = total;
        H = isinf(toldy) ? EPSMIN * (A.xe - X) : fmin((A.xe - X) / 100e0, pow(toldy, 0.2));
        nde = 1;
        grid.sync();  // the reduction scratch is reused below
    }
    long long acc = 0, rej = 0;
    int ier = 10000;
    for (int iter = 0; iter < A.itemax; iter++) {
        coop_fehl<P, kFastInv>(A, grid, H, yl0, yln, true, part);
        nde += 6;
        const double erret = coop_errnorm(A, grid, yl0, yln, sh);
        if (erret < 0.0) {
            ier = 20000;
            break;
        }
        if (erret > 1) {
            rej++;
            if (erret >= 59049) H *= 0.1;
            else H *= 0.9 / pow(erret, 0.2);
            if (H <= EPSMIN) {
                ier = 30000;
                break;
            }
        } else if (X + H < A.xe) {
            coop_fehl<P, kFastInv>(A, grid, H / 2, yh0, A.B.yhm, false, part);
            coop_fehl<P, kFastInv>(A, grid, H / 2, A.B.yhm, yhn, false, part);
            nde += 12;
            X += H;
            double *t1 = yl0; yl0 = yln; yln = t1;  // accepted: the new tracks become the old ones
            double *t2 = yh0; yh0 = yhn; yhn = t2;
            acc++;
            if (erret <= 1.889568e-4) H *= 5.0;
            else H *= 0.9 / pow(erret, 0.2);
        } else {
            H = A.xe - X;
            coop_fehl<P, kFastInv>(A, grid, H, yl0, yln, true, part);
            coop_fehl<P, kFastInv>(A, grid, H / 2, yh0, A.B.yhm, false, part);
            coop_fehl<P, kFastInv>(A, grid, H / 2, A.B.yhm, yhn, false, part);
            nde += 18;
            X = A.xe;
            acc++;
            ier = 0;
            break;
        }
    }
    // outputs: the state (the high track at xe, or the last accepted one), the low track
    // in B.yl0, (yln - yhn) / 31
    const double *yout = (ier == 0) ? yhn : yh0;
    const double *lout = (ier == 0) ? yln : yl0;
    for (int e = gid; e < len; e += gsz) {
        if (A.ese && ier == 0) A.ese[e] = (yln[e] - yhn[e]) / 31;
        A.y[e] = yout[e];
    }
    grid.sync();
    if (lout != A.B.yl0)
        for (int e = gid; e < len; e += gsz) A.B.yl0[e] = lout[e];
    if (gid == 0) {
        A.io[0] = X;
        A.io[1] = H;
        A.io[2] = nde;
        A.io[3] = (double)acc;
        A.io[4] = (double)rej;
        A.io[5] = ier;
    }
}

// The cooperative solver (dim_coop_kernel); *ran = false when the device cannot run it
// (no cooperative launch), and the caller takes the host-controlled loop instead.
static int dim_integrate_coop(DimRun &R, double *y, double *x0, double xe, int init, double *H, int *nde,
                              long long *accepted, long long *rejected, double *ese, int *status, bool *ran)
{
    *ran = false;
    *status = BIA_OK;
    const char *force_host = getenv("BIA_DIM_HOST_CONTROL");
    if (force_host && force_host[0] == '1') return 0;
    int dev = 0, coop = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    // groups of 8 particles below n = 4096, of 32 above; the inverse-cube form of the run
    const bool wide = R.n >= 4096;
    const void *kern = wide ? (R.fast_inv ? (const void *)dim_coop_kernel<32, true> : (const void *)dim_coop_kernel<32, false>)
                            : (R.fast_inv ? (const void *)dim_coop_kernel<8, true> : (const void *)dim_coop_kernel<8, false>);
    const int P = wide ? 32 : 8;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        return 0;
    }
    const int ngroups = (R.n + P - 1) / P;
    int G = ngroups;
    if (G > sms * per_sm) G = sms * per_sm;
    if (G > kDimCoopMaxBlocks) G = kDimCoopMaxBlocks;  // B.red holds kDimCoopMaxBlocks partials
    const char *gcap = getenv("BIA_DIM_COOP_BLOCKS");
    if (gcap && atoi(gcap) > 0 && atoi(gcap) < G) G = atoi(gcap);
    if (G < 1) G = 1;
    DimCoopArgs A;
    A.n = R.n;
    A.len = R.len;
    A.init = init;
    A.itemax = 10000;
    A.eps = R.eps;
    A.relerr = R.relerr;
    A.abserr = R.abserr;
    A.xe = xe;
    A.B = R.B;
    A.y = y;
    A.ese = ese;
    A.io = R.B.io;
    R.h_pinned[0] = *x0;
    R.h_pinned[1] = *H;
    cudaError_t e = cudaMemcpyAsync(R.B.io, R.h_pinned, 2 * sizeof(double), cudaMemcpyHostToDevice, R.st);
    void *args[] = {(void *)&A};
    if (e == cudaSuccess)
        e = cudaLaunchCooperativeKernel(kern, dim3(G), dim3(256), args, 0, R.st);
    double out[6] = {0, 0, 0, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(R.h_pinned, R.B.io, 6 * sizeof(double), cudaMemcpyDeviceToHost, R.st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(R.st);
    if (e != cudaSuccess) {
        *status = cuda_status(e);
        *ran = true;
        return 0;
    }
    for (int k = 0; k < 6; k++) out[k] = R.h_pinned[k];
    *x0 = out[0];
    *H = out[1];
    *nde = (int)out[2];
    *accepted += (long long)out[3];
    *rejected += (long long)out[4];
    *ran = true;
    return (int)out[5];
}

struct DimDropIn {
    bool ready = false;
    DeviceBuffer buf, state;
    double *h_pinned = nullptr;
};
static thread_local DimDropIn g_dim;

}  // namespace bia

using namespace bia;

extern "C" int bia_dim_integrate(bia_context *ctx, int n, double eps_th, double *y, double x0, double xe,
                                 double relerr, double abserr, bia_dim_stats *stats)
{
    if (!ctx || n < 1 || !y || !(xe > x0)) return BIA_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    cudaError_t e = ctx->dim.reserve(dim_buffer_doubles(n) * sizeof(double));
    if (e != cudaSuccess) return cuda_status(e);
    if (!ctx->h_dim) {
        e = cudaMallocHost((void **)&ctx->h_dim, 8 * sizeof(double));
        if (e != cudaSuccess) return cuda_status(e);
    }
    DimRun R;
    R.n = n;
    R.len = 6 * n;
    R.eps = eps_th;
    R.relerr = relerr;
    R.abserr = abserr;
    R.st = ctx->stream;
    R.h_pinned = ctx->h_dim;
    R.fast_inv = true;
    dim_carve((double *)ctx->dim.ptr, n, R.B);
    double X = x0, H = 0.0;
    int nde = 0, status = BIA_OK;
    long long acc = 0, rej = 0;
    bool ran = false;
    int ier = dim_integrate_coop(R, y, &X, xe, 1, &H, &nde, &acc, &rej, nullptr, &status, &ran);
    if (!ran) ier = dim_integrate(R, y, &X, xe, 1, &H, &nde, &acc, &rej, nullptr, &status);
    if (stats) {
        stats->accepted = acc;
        stats->rejected = rej;
        stats->nde = nde;
        stats->ier = ier;
        stats->h_last = H;
        stats->x_reached = X;
    }
    if (status != BIA_OK) return status;
    return ier == 0 ? BIA_OK : BIA_ERR_NOT_CONVERGED;
}

// Drop-in for rkf_c_ (dim/rkf_kernel.cu:194-495), called from dim/dim_3D.f90:30 as
// RKF_C(%VAL(NEQ), %VAL(eps_th), X0, XE, Y0, INIT, RELERR, ABSERR, YN, ESTERR, NDE, IER,
// WK0, WK1, WK2, WK3, WK4).  Host arrays are AoS (x, y, z, u, v, w per particle).
extern "C" void rkf_c_(const int neq, const double eps_th, double *X0, double *XE, double *YH0, int *INIT,
                       const double *RELERR, const double *ABSERR, double *YHN, double *ESE, int *NDE, int *IER,
                       double *H, double *YL0, double *YLN, double *ERR, double *WRK)
{
    (void)WRK;
    if (neq < 6 || neq % 6 || !X0 || !XE || !YH0 || !INIT || !RELERR || !ABSERR || !YHN || !ESE || !NDE ||
        !IER || !H || !YL0 || !YLN || !ERR || !(*XE > *X0)) {
        set_last_error(BIA_ERR_INVALID_ARGUMENT);
        return;
    }
    const int n = neq / 6;
    DimDropIn &S = g_dim;
    cudaError_t e = cudaSuccess;
    if (!S.ready) {
        e = cudaMallocHost((void **)&S.h_pinned, 8 * sizeof(double));
        if (e != cudaSuccess) {
            set_last_error(cuda_status(e));
            return;
        }
        S.ready = true;
    }
    if ((e = S.buf.reserve(dim_buffer_doubles(n) * sizeof(double))) != cudaSuccess ||
        (e = S.state.reserve((size_t)2 * neq * sizeof(double))) != cudaSuccess) {
        set_last_error(cuda_status(e));
        return;
    }
    double *dy = (double *)S.state.ptr;       // SoA state
    double *dese = dy + neq;                  // SoA esterr
    // AoS host -> SoA device
    double *tmp = (double *)malloc(sizeof(double) * neq);
    if (!tmp) {
        set_last_error(BIA_ERR_OUT_OF_MEMORY);
        return;
    }
    for (int i = 0; i < n; i++)
        for (int c = 0; c < 6; c++) tmp[(size_t)c * n + i] = YH0[6 * (size_t)i + c];
    e = cudaMemcpy(dy, tmp, sizeof(double) * neq, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        free(tmp);
        set_last_error(cuda_status(e));
        return;
    }
    DimRun R;
    R.n = n;
    R.len = neq;
    R.eps = eps_th;
    R.relerr = *RELERR;
    R.abserr = *ABSERR;
    R.st = 0;
    R.h_pinned = S.h_pinned;
    dim_carve((double *)S.buf.ptr, n, R.B);
    int nde = 0, status = BIA_OK;
    long long acc = 0, rej = 0;
    const int init = *INIT;
    bool ran = false;
    int ier = dim_integrate_coop(R, dy, X0, *XE, init, H, &nde, &acc, &rej, dese, &status, &ran);
    if (!ran) ier = dim_integrate(R, dy, X0, *XE, init, H, &nde, &acc, &rej, dese, &status);
    if (init == 1) *INIT = 2;
    *NDE = nde;
    *IER = ier;
    if (status == BIA_OK) {
        // SoA device -> AoS host: YHN (high track), YL0 / YLN (low track), ESE, ERR
        double *outs[4] = {YHN, YLN, ESE, ERR};
        const double *srcs[4] = {dy, R.B.yl0, dese, R.B.er};
        for (int o = 0; o < 4 && e == cudaSuccess; o++) {
            if (ier != 0 && o == 2) continue;
            e = cudaMemcpy(tmp, srcs[o], sizeof(double) * neq, cudaMemcpyDeviceToHost);
            if (e == cudaSuccess)
                for (int i = 0; i < n; i++)
                    for (int c = 0; c < 6; c++) outs[o][6 * (size_t)i + c] = tmp[(size_t)c * n + i];
        }
        if (e == cudaSuccess) {
            memcpy(YL0, YLN, sizeof(double) * neq);  // after the last step YL0 = YLN
            if (ier == 0) memcpy(YH0, YHN, sizeof(double) * neq);
        }
        status = cuda_status(e);
    }
    free(tmp);
    set_last_error(status != BIA_OK ? status : (ier == 0 ? BIA_OK : BIA_ERR_NOT_CONVERGED));
}
