// bia_ensemble.cu -- many independent BIA systems of uneven size in one launch per step.
//
// The systems are stored back to back in one set of SoA arrays: system s owns particles
// [off[s], off[s] + n_s) and has pair coupling eps[s] (gravity: -2/n_s for G = 1 and
// masses 1/n_s).  At creation the host lists every 32 x 32 warp-block of every system's
// upper triangle as one work item (system, bi, bj); a step is then one launch of the pair
// kernel over the whole item table -- the same per-warp-block code as the single-system
// step (bia_tiles.cuh), so each system's result is identical to a bia_step of that system
// alone -- plus one reduction launch over all particles.  bia_ensemble_run captures the
// step sequence in a CUDA graph.  Per-system partial sums use the single-system layout at
// offset part_off[s]: [nb_s][6][32 nb_s] doubles.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "bia_internal.cuh"
#include "bia_learned_block.cuh"
#include "bia_pair.cuh"
#include "bia_tiles.cuh"

struct bia_ensemble {
    int nsys = 0;
    long long nparticles = 0, nitems = 0;
    int *d_off = nullptr;              // [nsys + 1] particle offsets
    int *d_psys = nullptr;             // [nparticles] system of each particle
    long long *d_part_off = nullptr;   // [nsys] partial-buffer offsets (doubles)
    long long *d_item_off = nullptr;   // [nsys + 1] first item of each system
    double *d_eps = nullptr;           // [nsys]
    uint2 *d_items = nullptr;          // [nitems] (system, bi | bj << 16)
    double *d_part = nullptr;          // partial sums
    double *d_scratch = nullptr;       // [nitems + nparticles] energy scratch
    double *d_energy = nullptr;        // [2 nsys] KE, PE per system
    // learned step: the deferred pairs' rows and the list of items holding them
    // (bia_learned_block.cuh), one buffer
    uint8_t *d_split = nullptr;
    unsigned int rows_cap = 0;
    size_t part_doubles = 0;
    // launch shape chosen by bia_ensemble_autotune per method (index BIA_METHOD_*), -1: the
    // built-in rule
    int tuned[4] = {-1, -1, -1, -1};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    bia::GraphKey graph_key;
};

namespace bia {

constexpr int kEnsWarps = 8;
constexpr int kEnsThreads = kEnsWarps * 32;

struct EnsArgs {
    const double *x, *y, *z, *u, *v, *w, *q;
    const int *off;
    const long long *part_off;
    const double *eps;
    const uint2 *items;
    long long nitems;
    double *part;
    unsigned long long *stats;
    PairParams P;
    const MlpImage *heads;  // BIA_METHOD_LEARNED
    LearnedRows R;          // learned step: the deferred pairs' rows and the listed items
};

// Each warp takes items t = (its global warp index) + k * (warps in the grid), as
// bia_pair_tiles_kernel (a persistent grid for the universal-variable method, the counters
// flushed per warp every kFlushBlocks items).
template <int M>
__global__ void __launch_bounds__(kEnsThreads, TileOccupancy<M>::kMinBlocks) ens_pair_tiles_kernel(const EnsArgs A)
{
    const int lane = threadIdx.x & 31;
    PairCounters tot;
    counters_zero(tot);
    int nblk = 0;
    for (long long t = (long long)blockIdx.x * kEnsWarps + (threadIdx.x >> 5); t < A.nitems;
         t += (long long)gridDim.x * kEnsWarps) {  // warp-uniform
        const uint2 it = A.items[t];
        const int s = (int)it.x;
        const int bi = (int)(it.y & 0xffffu), bj = (int)(it.y >> 16);
        const int base = A.off[s];
        const int n = A.off[s + 1] - base;
        const double *q = A.q ? A.q + base : nullptr;
        double racc[6], cacc[6];
        PairCounters cnt;
        warp_block_solve<M>(A.x + base, A.y + base, A.z + base, A.u + base, A.v + base, A.w + base, q, n,
                            A.eps[s], A.P, bi, bj, lane, racc, cacc, cnt);
        counters_add(tot, cnt);
        if (++nblk == kFlushBlocks) {
            flush_counters(tot, A.stats, lane);
            counters_zero(tot);
            nblk = 0;
        }
        const int nb = (n + 31) / 32;
        write_partials(A.part + A.part_off[s], (size_t)nb * 32, bi, bj, lane, racc, cacc);
    }
    if (nblk > 0) flush_counters(tot, A.stats, lane);
}

// Phase-locked ALG variant of ens_pair_tiles_kernel (see phase_block_solve): CTAs of kW
// warps, kMinB of them per SM, each warp on one item, the counters flushed once per CTA as in
// bia_pair_phase_kernel; bitwise the same results.
template <int kW, int kMinB, bool kBalanced = true>
__global__ void __launch_bounds__(kW * 32, kMinB) ens_pair_phase_kernel(const EnsArgs A)
{
    extern __shared__ double phase_smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    unsigned long long *slots = reinterpret_cast<unsigned long long *>(phase_smem + kW * phase_slice_doubles<kBalanced>());
    unsigned long long *wtot = slots + warp * kNumStats;
    if (lane < kNumStats) wtot[lane] = 0ull;
    __syncwarp();
    const long long t = (long long)blockIdx.x * kW + warp;
    const bool live = t < A.nitems;
    int s = 0, bi = 0, bj = 0;
    if (live) {
        const uint2 it = A.items[t];
        s = (int)it.x;
        bi = (int)(it.y & 0xffffu);
        bj = (int)(it.y >> 16);
    }
    const int base = A.off[s];
    const int n = A.off[s + 1] - base;
    const double *q = A.q ? A.q + base : nullptr;
    double racc[6], cacc[6];
    PairCounters cnt;
    phase_block_solve<kBalanced>(A.x + base, A.y + base, A.z + base, A.u + base, A.v + base, A.w + base, q, n,
                                 A.eps[s],
                      A.P, bi, bj, lane, live, phase_smem + warp * phase_slice_doubles<kBalanced>(), racc, cacc, cnt);
    if (live) {  // warp-uniform
        counters_to_slot(cnt, wtot, lane);
        const int nb = (n + 31) / 32;
        write_partials(A.part + A.part_off[s], (size_t)nb * 32, bi, bj, lane, racc, cacc);
    }
    __syncthreads();
    if (warp == 0) flush_slots(slots, kW, A.stats, lane);
}

// Once per device (the current one): dynamic shared memory opt-in of the phase-locked
// ensemble kernel and the SM count; 0 when the set-up failed (8-warp kernel used).
static int ens_phase_setup()
{
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static int sms_of[kMaxDevices] = {};
    static bool done_of[kMaxDevices] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 0;
    std::lock_guard<std::mutex> lk(mu);
    if (!done_of[dev]) {
        int sms = 0;
        bool ok = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess;
        ok = ok && cudaFuncSetAttribute(ens_pair_phase_kernel<32, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        32 * (kPhaseSliceDoubles + kNumStats) * (int)sizeof(double)) == cudaSuccess;
        ok = ok && cudaFuncSetAttribute(ens_pair_phase_kernel<32, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        32 * (kTileSmemDoubles + kNumStats) * (int)sizeof(double)) == cudaSuccess;
        if (!ok) cudaGetLastError();
        sms_of[dev] = ok ? sms : 0;
        done_of[dev] = true;
    }
    return sms_of[dev];
}

// Learned step over the item table, first kernel: each item's pairs except the deferred ones
// (rest_block_solve, rest_block_defer, as bia_pair_rest_kernel), the items holding deferred
// pairs listed with their rows; the head kernel of the single-system step then evaluates the
// rows and ens_pair_learned_finish_kernel solves the listed items' deferred pairs.
__global__ void __launch_bounds__(kEnsThreads, 2) ens_pair_rest_kernel(const EnsArgs A)
{
    extern __shared__ __align__(16) uint8_t ens_rest_smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    double *ws = reinterpret_cast<double *>(ens_rest_smem + warp * kRestWarpBytes);
    uint32_t *wslots = reinterpret_cast<uint32_t *>(ens_rest_smem + warp * kRestWarpBytes +
                                                    kTileSmemDoubles * sizeof(double));
    PairCounters tot;
    counters_zero(tot);
    int nblk = 0;
    for (long long t = (long long)blockIdx.x * kEnsWarps + warp; t < A.nitems;
         t += (long long)gridDim.x * kEnsWarps) {  // warp-uniform
        const uint2 it = A.items[t];
        const int s = (int)it.x;
        const int bi = (int)(it.y & 0xffffu), bj = (int)(it.y >> 16);
        const int base = A.off[s];
        const int n = A.off[s + 1] - base;
        double racc[6], cacc[6];
        uint32_t mask[kMlpHeads];
        PairCounters cnt;
        rest_block_solve(A.x + base, A.y + base, A.z + base, A.u + base, A.v + base, A.w + base,
                         A.q ? A.q + base : nullptr, n, A.eps[s], A.P.dt, bi, bj, lane, ws, wslots, racc, cacc,
                         mask, cnt);
        counters_add(tot, cnt);
        if (++nblk == kFlushBlocks) {
            flush_counters(tot, A.stats, lane);
            counters_zero(tot);
            nblk = 0;
        }
        const int nb = (n + 31) / 32;
        write_partials(A.part + A.part_off[s], (size_t)nb * 32, bi, bj, lane, racc, cacc);
        rest_block_defer(A.R, (unsigned int)t, mask, wslots, lane);
    }
    if (nblk > 0) flush_counters(tot, A.stats, lane);
}

// Learned step over the item table, third kernel (persistent 8-warp CTAs): a dense or
// diagonal item finished by one warp, then the sparse ones in chunks of 32 list entries and
// batches of 32 pairs, as bia_pair_learned_finish_kernel (each system bitwise its own step).
__global__ void __launch_bounds__(kEnsThreads, 2) ens_pair_learned_finish_kernel(const EnsArgs A)
{
    __shared__ double s_fin[kTileWarps][kTileSmemDoubles];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const long long count = (long long)*A.R.nlist;
    PairCounters tot;
    counters_zero(tot);
    int nchunk = 0;
    // the system, block and partials of list entry e
    auto resolve_entry = [&](long long e) {
        const uint2 it = A.items[A.R.entries[e].x];
        const int s = (int)it.x;
        const int base = A.off[s];
        const int n = A.off[s + 1] - base;
        FinishBlock F;
        F.B = {A.x + base, A.y + base, A.z + base, A.u + base, A.v + base, A.w + base,
               A.q ? A.q + base : nullptr, n, A.eps[s], A.P.dt, A.heads};
        F.bi = (int)(it.y & 0xffffu);
        F.bj = (int)(it.y >> 16);
        F.part = A.part + A.part_off[s];
        F.plane = (size_t)((n + 31) / 32) * 32;
        return F;
    };
    // 1. the dense and diagonal items, the list entries spread over the warps one at a time,
    // read 32 at a time with one load per lane
    const long long gw = (long long)blockIdx.x * kEnsWarps + warp;
    const long long stride = (long long)gridDim.x * kEnsWarps;
    for (long long k0 = 0; gw + k0 * stride < count; k0 += 32) {  // warp-uniform
        const long long el = gw + (k0 + lane) * stride;
        bool dense = false;
        if (el < count) {
            const uint4 ent = A.R.entries[el];
            const uint2 it = A.items[ent.x];
            dense = !((it.y & 0xffffu) != (it.y >> 16) && ent.w <= (unsigned)kBatchPairs);
        }
        for (unsigned dm = __ballot_sync(full, dense); dm; dm &= dm - 1u) {
            const long long e = gw + (k0 + (__ffs(dm) - 1)) * stride;
            const FinishBlock F = resolve_entry(e);
            double racc[6], cacc[6];
            PairCounters cnt;
            bool row_hit, col_hit;
            finish_block_solve(A.R, e, F.B, F.bi, F.bj, lane, s_fin[warp], racc, cacc, cnt, row_hit, col_hit);
            counters_add(tot, cnt);
            if (++nchunk == kFlushBlocks) {
                flush_counters(tot, A.stats, lane);
                counters_zero(tot);
                nchunk = 0;
            }
            add_partials(F.part, F.plane, F.bi, F.bj, lane, racc, cacc, row_hit, col_hit);
        }
    }
    // 2. the sparse ones, batched per chunk of list entries (up to 32 per warp, fewer when the
    // list is short)
    const long long nwarps = (long long)gridDim.x * kEnsWarps;
    const long long chunk = count >= 32 * nwarps ? 32 : (count + nwarps - 1) / nwarps;
    for (long long c0 = ((long long)blockIdx.x * kEnsWarps + warp) * chunk; c0 < count;
         c0 += nwarps * chunk) {  // warp-uniform
        const long long e = c0 + lane;
        const bool valid = lane < chunk && e < count;
        unsigned int npairs = 0u;
        bool sparse = false;
        if (valid) {
            npairs = A.R.entries[e].w;
            const uint2 it = A.items[A.R.entries[e].x];
            sparse = (it.y & 0xffffu) != (it.y >> 16) && npairs <= (unsigned)kBatchPairs;
        }
        if (__ballot_sync(full, sparse) == 0u) continue;
        auto resolve = [&](int l) { return resolve_entry(c0 + l); };
        PairCounters cnt;
        counters_zero(cnt);
        finish_batches<true>(A.R, c0, sparse, npairs, lane, resolve, cnt);
        counters_add(tot, cnt);
        if (++nchunk == kFlushBlocks) {
            flush_counters(tot, A.stats, lane);
            counters_zero(tot);
            nchunk = 0;
        }
    }
    if (nchunk > 0) flush_counters(tot, A.stats, lane);
}

// Once per device: shared-memory opt-in of the ensemble's rest kernel (the head kernel is the
// single-system step's, set up by bia_learned_head_grid); returns the head kernel's grid
// (resident CTAs), 0 on failure.
static int ens_learned_setup()
{
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static bool done_of[kMaxDevices] = {};
    static bool ok_of[kMaxDevices] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 0;
    const int hgrid = learned_head_grid();
    std::lock_guard<std::mutex> lk(mu);
    if (!done_of[dev]) {
        ok_of[dev] = cudaFuncSetAttribute(ens_pair_rest_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)kRestSmemBytes) == cudaSuccess;
        if (!ok_of[dev]) cudaGetLastError();
        done_of[dev] = true;
    }
    return ok_of[dev] ? hgrid : 0;
}

struct EnsUpdateArgs {
    double *x, *y, *z, *u, *v, *w;
    const int *off, *psys;
    const long long *part_off;
    const double *part;
    long long nparticles;
    double dt;
};

// fixed-order partial sums, drift and update (bia/bia.f90:194-204), all systems at once
__global__ void __launch_bounds__(256) ens_reduce_update_kernel(const EnsUpdateArgs A)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.nparticles) return;
    const int s = A.psys[p];
    const int base = A.off[s];
    const int n = A.off[s + 1] - base;
    const int nb = (n + 31) / 32;
    const size_t plane = (size_t)nb * 32;
    const double *src = A.part + A.part_off[s] + (p - base);
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int m = 0; m < nb; m++) {
#pragma unroll
        for (int c = 0; c < 6; c++) acc[c] += src[((size_t)m * 6 + c) * plane];
    }
    const double u = A.u[p], v = A.v[p], w = A.w[p];
    A.x[p] = A.x[p] + (acc[0] + u * A.dt);
    A.y[p] = A.y[p] + (acc[1] + v * A.dt);
    A.z[p] = A.z[p] + (acc[2] + w * A.dt);
    A.u[p] = u + acc[3];
    A.v[p] = v + acc[4];
    A.w[p] = w + acc[5];
}

// per-item pair sums sum (q_i q_j) / r_ij of each system (energy)
__global__ void __launch_bounds__(kEnsThreads) ens_pe_items_kernel(const double *x, const double *y, const double *z,
                                                                    const double *q, const int *off,
                                                                    const uint2 *items, long long nitems,
                                                                    double *out)
{
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const long long t = (long long)blockIdx.x * kEnsWarps + (threadIdx.x >> 5);
    if (t >= nitems) return;
    const uint2 it = items[t];
    const int s = (int)it.x;
    const int bi = (int)(it.y & 0xffffu), bj = (int)(it.y >> 16);
    const int base = off[s];
    const int n = off[s + 1] - base;
    const int i = bi * 32 + lane, jo = bj * 32 + lane;
    const bool iv = i < n, jv = jo < n;
    const double xi = iv ? x[base + i] : 0.0, yi = iv ? y[base + i] : 0.0, zi = iv ? z[base + i] : 0.0;
    const double qi = (iv && q) ? q[base + i] : 1.0;
    const double xj = jv ? x[base + jo] : 0.0, yj = jv ? y[base + jo] : 0.0, zj = jv ? z[base + jo] : 0.0;
    const double qj = (jv && q) ? q[base + jo] : 1.0;
    const bool diag = bi == bj;
    double acc = 0.0;
    for (int k = diag ? 1 : 0; k <= (diag ? 16 : 31); k++) {
        const int src = (lane + k) & 31;
        const double cx = __shfl_sync(full, xj, src), cy = __shfl_sync(full, yj, src);
        const double cz = __shfl_sync(full, zj, src), cq = __shfl_sync(full, qj, src);
        if ((!diag || k < 16 || lane < 16) && iv && bj * 32 + src < n) {
            const double dx = xi - cx, dy = yi - cy, dz = zi - cz;
            const double wgt = 1.0 / sqrt(dx * dx + dy * dy + dz * dz);
            acc += q ? qi * cq * wgt : wgt;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(full, acc, o);
    if (lane == 0) out[t] = acc;
}

// one block per system: KE = sum |v|^2 over its particles, PE = eps_s * (ordered sum of
// its items' pair sums)
__global__ void __launch_bounds__(256) ens_energy_kernel(const double *u, const double *v, const double *w,
                                                         const int *off, const long long *item_off,
                                                         const double *eps, const double *item_pe, double *energy)
{
    __shared__ double sh[2][256];
    const int s = blockIdx.x;
    double ke = 0.0, pe = 0.0;
    for (int p = off[s] + threadIdx.x; p < off[s + 1]; p += blockDim.x) ke += u[p] * u[p] + v[p] * v[p] + w[p] * w[p];
    for (long long t = item_off[s] + threadIdx.x; t < item_off[s + 1]; t += blockDim.x) pe += item_pe[t];
    sh[0][threadIdx.x] = ke;
    sh[1][threadIdx.x] = pe;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if (threadIdx.x < k) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + k];
            sh[1][threadIdx.x] += sh[1][threadIdx.x + k];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        energy[2 * s] = sh[0][0];
        energy[2 * s + 1] = eps[s] * sh[1][0];
    }
}

// Launch shapes of the ensemble's pair kernels (bia_ensemble_autotune chooses among them):
//   ALG          0: 8-warp CTAs (ens_pair_tiles_kernel), 1: phase-locked 32-warp CTAs (1 per
//                SM) with per-lane class loops, 2: the same with the balanced class loops;
//                built-in rule: 2 from two of its CTAs per SM up, else 0
//   universal    0: one item per warp, 1: a persistent grid of 2 CTAs per SM (built-in)
//   learned      the persistent head kernel with 0: 1 CTA per SM, 1: 2 CTAs per SM (built-in)
// Every shape runs the same per-item arithmetic in the same order: the results are bitwise
// the same.
constexpr int kEnsShapes = 3;

static int ens_pair_launch(bia_context *ctx, bia_ensemble *E, EnsArgs &A, int method, int shape)
{
    const unsigned grid = (unsigned)((E->nitems + kEnsWarps - 1) / kEnsWarps);
    cudaStream_t st = ctx->stream;
    if (method == BIA_METHOD_LEARNED) {
        // the split step of bia_step: the rest, head and finish kernels (the same
        // per-warp-block arithmetic, so each system equals its own learned bia_step)
        const int lsetup = ens_learned_setup();
        if (!ctx->heads_loaded) return BIA_ERR_INVALID_ARGUMENT;
        if (lsetup <= 0) return BIA_ERR_CUDA;
        uint8_t *b = E->d_split;
        A.R.counts = (unsigned long long *)b;
        A.R.nlist = (unsigned int *)(b + 16);
        A.R.entries = (uint4 *)(b + kSplitHeader);
        A.R.masks = (uint32_t *)(b + kSplitHeader + (size_t)E->nitems * 16);
        A.R.pairs = (uint2 *)(b + kSplitHeader + (size_t)E->nitems * (16 + 64 * sizeof(uint32_t)));
        uint32_t *rows = (uint32_t *)(b + kSplitHeader + (size_t)E->nitems * kListBytesPerBlock);
        A.R.rows_cap = E->rows_cap;
        A.R.rows[kHeadEll] = rows;
        A.R.rows[kHeadHyp] = rows + E->rows_cap;
        cudaError_t e = cudaMemsetAsync(A.R.counts, 0, kSplitHeader, st);
        if (e != cudaSuccess) return cuda_status(e);
        const unsigned rgrid = (unsigned)persistent_grid(grid);
        ens_pair_rest_kernel<<<rgrid, kEnsThreads, kRestSmemBytes, st>>>(A);
        long long hcap = lsetup;
        if (shape == 0 || shape == 1) hcap = (long long)device_sm_count() * (shape + 1);
        launch_learned_head(A.R, A.heads, A.stats, (int)hcap, st);
        ens_pair_learned_finish_kernel<<<rgrid, kEnsThreads, 0, st>>>(A);
        return cuda_status(cudaGetLastError());
    }
    switch (method) {
    case BIA_METHOD_RKF: ens_pair_tiles_kernel<kMethodRkf><<<grid, kEnsThreads, 0, st>>>(A); break;
    case BIA_METHOD_UNIVERSAL:
        ens_pair_tiles_kernel<kMethodUniversal>
            <<<shape == 0 ? grid : (unsigned)persistent_grid(grid), kEnsThreads, 0, st>>>(A);
        break;
    default: {
        const int sms = BIA_PHASE_WARPS > 0 ? ens_phase_setup() : 0;
        int var = shape;
        if (var < 0 || var >= kEnsShapes) var = (sms > 0 && (E->nitems + 31) / 32 >= 2LL * sms) ? 2 : 0;
        if (sms <= 0) var = 0;
        if (var == 2) {
            ens_pair_phase_kernel<32, 1><<<(unsigned)((E->nitems + 31) / 32), 32 * 32,
                                            32 * (kPhaseSliceDoubles + kNumStats) * sizeof(double), st>>>(A);
        } else if (var == 1) {
            ens_pair_phase_kernel<32, 1, false><<<(unsigned)((E->nitems + 31) / 32), 32 * 32,
                                                   32 * (kTileSmemDoubles + kNumStats) * sizeof(double), st>>>(A);
        } else {
            ens_pair_tiles_kernel<kMethodAlg><<<grid, kEnsThreads, 0, st>>>(A);
        }
        break;
    }
    }
    return cuda_status(cudaGetLastError());
}

static int ens_enqueue_step(bia_context *ctx, bia_ensemble *E, const bia_config *cfg, double *x, double *y,
                            double *z, double *u, double *v, double *w, const double *q)
{
    EnsArgs A{};
    A.x = x; A.y = y; A.z = z; A.u = u; A.v = v; A.w = w; A.q = q;
    A.off = E->d_off;
    A.part_off = E->d_part_off;
    A.eps = E->d_eps;
    A.items = E->d_items;
    A.nitems = E->nitems;
    A.part = E->d_part;
    A.stats = (unsigned long long *)ctx->stats.ptr;
    A.P.dt = cfg->dt;
    A.P.err = cfg->err;
    A.P.relerr = cfg->rkf_relerr;
    A.P.abserr = cfg->rkf_abserr;
    A.P.itr = cfg->itr;
    A.P.method = cfg->method;
    A.heads = (const MlpImage *)ctx->heads.ptr;
    const int st = ens_pair_launch(ctx, E, A, cfg->method, E->tuned[cfg->method & 3]);
    if (st != BIA_OK) return st;
    EnsUpdateArgs U;
    U.x = x; U.y = y; U.z = z; U.u = u; U.v = v; U.w = w;
    U.off = E->d_off;
    U.psys = E->d_psys;
    U.part_off = E->d_part_off;
    U.part = E->d_part;
    U.nparticles = E->nparticles;
    U.dt = cfg->dt;
    ens_reduce_update_kernel<<<(unsigned)((E->nparticles + 255) / 256), 256, 0, ctx->stream>>>(U);
    return cuda_status(cudaGetLastError());
}

static void ens_free(bia_ensemble *E)
{
    if (!E) return;
    if (E->graph_exec) cudaGraphExecDestroy(E->graph_exec);
    if (E->graph) cudaGraphDestroy(E->graph);
    cudaFree(E->d_off);
    cudaFree(E->d_psys);
    cudaFree(E->d_part_off);
    cudaFree(E->d_item_off);
    cudaFree(E->d_eps);
    cudaFree(E->d_items);
    cudaFree(E->d_part);
    cudaFree(E->d_scratch);
    cudaFree(E->d_energy);
    cudaFree(E->d_split);
    delete E;
}

}  // namespace bia

using namespace bia;

extern "C" int bia_ensemble_create(bia_context *ctx, int nsys, const int *sizes, const double *eps,
                                   bia_ensemble **out)
{
    if (!ctx || !out || nsys < 1 || !sizes || !eps) return BIA_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    cudaSetDevice(ctx->device);
    std::vector<int> off(nsys + 1, 0);
    std::vector<long long> part_off(nsys), item_off(nsys + 1, 0);
    size_t part = 0;
    for (int s = 0; s < nsys; s++) {
        if (sizes[s] < 1 || sizes[s] > 32 * 65535) return BIA_ERR_INVALID_ARGUMENT;
        if ((long long)off[s] + sizes[s] > (1LL << 30)) return BIA_ERR_INVALID_ARGUMENT;
        off[s + 1] = off[s] + sizes[s];
        const long long nb = (sizes[s] + 31) / 32;
        part_off[s] = (long long)part;
        part += (size_t)nb * 6 * nb * 32;
        item_off[s + 1] = item_off[s] + nb * (nb + 1) / 2;
    }
    const long long np = off[nsys], nitems = item_off[nsys];
    std::vector<uint2> items((size_t)nitems);
    for (int s = 0; s < nsys; s++) {
        const int nb = (sizes[s] + 31) / 32;
        long long t = item_off[s];
        for (int bj = 0; bj < nb; bj++)
            for (int bi = 0; bi <= bj; bi++) items[(size_t)t++] = make_uint2((unsigned)s, (unsigned)bi | ((unsigned)bj << 16));
    }
    std::vector<int> psys((size_t)np);
    for (int s = 0; s < nsys; s++)
        for (int p = off[s]; p < off[s + 1]; p++) psys[(size_t)p] = s;
    bia_ensemble *E = new bia_ensemble();
    E->nsys = nsys;
    E->nparticles = np;
    E->nitems = nitems;
    E->part_doubles = part;
    cudaError_t e = cudaSuccess;
#define ENS_ALLOC(ptr, count)                                                        \
    if (e == cudaSuccess) e = cudaMalloc((void **)&(ptr), sizeof(*(ptr)) * (size_t)(count))
    ENS_ALLOC(E->d_off, nsys + 1);
    ENS_ALLOC(E->d_psys, np);
    ENS_ALLOC(E->d_part_off, nsys);
    ENS_ALLOC(E->d_item_off, nsys + 1);
    ENS_ALLOC(E->d_eps, nsys);
    ENS_ALLOC(E->d_items, nitems);
    ENS_ALLOC(E->d_part, part);
    ENS_ALLOC(E->d_scratch, nitems);
    ENS_ALLOC(E->d_energy, 2 * nsys);
    {
        // rows: up to every pair of the ensemble per head, capped as in the single-system step
        unsigned long long pairs = 0;
        for (int s2 = 0; s2 < nsys; s2++) pairs += (unsigned long long)sizes[s2] * (sizes[s2] - 1) / 2;
        E->rows_cap = (unsigned int)(pairs < (1ull << 27) ? (pairs > 0 ? pairs : 1) : (1ull << 27));
        ENS_ALLOC(E->d_split, kSplitHeader + (size_t)nitems * kListBytesPerBlock +
                                  (size_t)kMlpHeads * E->rows_cap * sizeof(uint32_t));
    }
#undef ENS_ALLOC
    if (e == cudaSuccess) e = cudaMemcpy(E->d_off, off.data(), sizeof(int) * (nsys + 1), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(E->d_psys, psys.data(), sizeof(int) * np, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(E->d_part_off, part_off.data(), sizeof(long long) * nsys, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(E->d_item_off, item_off.data(), sizeof(long long) * (nsys + 1), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(E->d_eps, eps, sizeof(double) * nsys, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(E->d_items, items.data(), sizeof(uint2) * nitems, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = ctx->stats.reserve(kNumStats * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        ens_free(E);
        return cuda_status(e);
    }
    *out = E;
    return BIA_OK;
}

extern "C" int bia_ensemble_destroy(bia_ensemble *ens)
{
    ens_free(ens);
    return BIA_OK;
}

extern "C" long long bia_ensemble_particles(const bia_ensemble *ens) { return ens ? ens->nparticles : 0; }

extern "C" int bia_ensemble_run(bia_context *ctx, bia_ensemble *E, const bia_config *cfg, double *x, double *y,
                                double *z, double *u, double *v, double *w, const double *q, int nsteps,
                                int use_graph, bia_stats *stats)
{
    if (!ctx || !E || !cfg || !x || !y || !z || !u || !v || !w || nsteps < 0) return BIA_ERR_INVALID_ARGUMENT;
    const bool learned_ok = cfg->method == BIA_METHOD_LEARNED && ctx->heads_loaded;
    if (cfg->method != BIA_METHOD_ALG && cfg->method != BIA_METHOD_RKF && cfg->method != BIA_METHOD_UNIVERSAL &&
        !learned_ok)
        return BIA_ERR_INVALID_ARGUMENT;
    if (cfg->itr < 1 || cfg->itr > 62) return BIA_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    if (learned_ok && !ens_learned_setup()) return BIA_ERR_CUDA;  // before any stream capture
    cudaError_t e = cudaSuccess;
    if (stats) {
        e = cudaMemsetAsync(ctx->stats.ptr, 0, kNumStats * sizeof(unsigned long long), ctx->stream);
        if (e != cudaSuccess) return cuda_status(e);
    }
    if (use_graph && ctx->stream && nsteps > 0) {
        GraphKey key;
        key.n = (int)E->nparticles; key.nsteps = nsteps; key.method = cfg->method; key.itr = cfg->itr;
        key.deterministic = 1; key.eps = 0.0; key.dt = cfg->dt; key.err = cfg->err;
        key.relerr = cfg->rkf_relerr; key.abserr = cfg->rkf_abserr;
        const void *p[7] = {x, y, z, u, v, w, q};
        for (int k = 0; k < 7; k++) key.ptrs[k] = p[k];
        if (!E->graph_exec || !(key == E->graph_key)) {
            if (E->graph_exec) cudaGraphExecDestroy(E->graph_exec);
            if (E->graph) cudaGraphDestroy(E->graph);
            E->graph_exec = nullptr;
            E->graph = nullptr;
            e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) return cuda_status(e);
            int st = BIA_OK;
            for (int s = 0; s < nsteps && st == BIA_OK; s++) st = ens_enqueue_step(ctx, E, cfg, x, y, z, u, v, w, q);
            e = cudaStreamEndCapture(ctx->stream, &E->graph);
            if (st != BIA_OK) return st;
            if (e != cudaSuccess) return cuda_status(e);
            e = cudaGraphInstantiate(&E->graph_exec, E->graph, 0);
            if (e != cudaSuccess) return cuda_status(e);
            E->graph_key = key;
        }
        e = cudaGraphLaunch(E->graph_exec, ctx->stream);
        if (e != cudaSuccess) return cuda_status(e);
    } else {
        for (int s = 0; s < nsteps; s++) {
            int st = ens_enqueue_step(ctx, E, cfg, x, y, z, u, v, w, q);
            if (st != BIA_OK) return st;
        }
    }
    if (stats) return bia_context_stats(ctx, stats, 0);
    return cuda_status(cudaGetLastError());
}

extern "C" int bia_ensemble_energy(bia_context *ctx, bia_ensemble *E, const double *x, const double *y,
                                   const double *z, const double *u, const double *v, const double *w,
                                   const double *q, double *energy)
{
    if (!ctx || !E || !x || !y || !z || !u || !v || !w || !energy) return BIA_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    const unsigned grid = (unsigned)((E->nitems + kEnsWarps - 1) / kEnsWarps);
    ens_pe_items_kernel<<<grid, kEnsThreads, 0, ctx->stream>>>(x, y, z, q, E->d_off, E->d_items, E->nitems,
                                                               E->d_scratch);
    ens_energy_kernel<<<E->nsys, 256, 0, ctx->stream>>>(u, v, w, E->d_off, E->d_item_off, E->d_eps, E->d_scratch,
                                                        E->d_energy);
    cudaError_t e = cudaMemcpyAsync(energy, E->d_energy, sizeof(double) * 2 * E->nsys, cudaMemcpyDeviceToHost,
                                    ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    return cuda_status(e);
}

extern "C" int bia_ensemble_autotune(bia_context *ctx, bia_ensemble *E, const bia_config *cfg, double *x, double *y,
                                     double *z, double *u, double *v, double *w, const double *q, int *variant,
                                     float *ms)
{
    if (!ctx || !E || !cfg || !x || !y || !z || !u || !v || !w) return BIA_ERR_INVALID_ARGUMENT;
    if (variant) *variant = -1;
    if (ms)
        for (int k = 0; k < kEnsShapes; k++) ms[k] = -1.0f;
    const int method = cfg->method;
    if (method == BIA_METHOD_LEARNED && !ctx->heads_loaded) return BIA_ERR_INVALID_ARGUMENT;
    const int nshapes = method == BIA_METHOD_ALG ? 3 : (method == BIA_METHOD_UNIVERSAL || method == BIA_METHOD_LEARNED) ? 2 : 0;
    if (nshapes == 0) return BIA_OK;  // one shape only
    cudaError_t e = cudaSetDevice(ctx->device);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (e == cudaSuccess && ctx->stream) e = cudaStreamIsCapturing(ctx->stream, &cap);
    if (e != cudaSuccess) return cuda_status(e);
    if (cap != cudaStreamCaptureStatusNone) return BIA_ERR_INVALID_ARGUMENT;
    if (method == BIA_METHOD_LEARNED && !ens_learned_setup()) return BIA_ERR_CUDA;
    EnsArgs A{};
    A.x = x; A.y = y; A.z = z; A.u = u; A.v = v; A.w = w; A.q = q;
    A.off = E->d_off;
    A.part_off = E->d_part_off;
    A.eps = E->d_eps;
    A.items = E->d_items;
    A.nitems = E->nitems;
    A.part = E->d_part;
    A.stats = (unsigned long long *)ctx->stats.ptr;
    A.P.dt = cfg->dt; A.P.err = cfg->err; A.P.relerr = cfg->rkf_relerr; A.P.abserr = cfg->rkf_abserr;
    A.P.itr = cfg->itr; A.P.method = method;
    A.heads = (const MlpImage *)ctx->heads.ptr;
    cudaEvent_t ev[2];
    e = cudaEventCreate(&ev[0]);
    if (e == cudaSuccess) e = cudaEventCreate(&ev[1]);
    if (e != cudaSuccess) return cuda_status(e);
    int best = -1;
    float best_ms = 0.0f;
    int st = BIA_OK;
    for (int var = 0; var < nshapes && st == BIA_OK && e == cudaSuccess; var++) {
        float t_min = 0.0f;
        for (int rep = 0; rep < 4 && st == BIA_OK && e == cudaSuccess; rep++) {  // the first is a warm-up
            e = cudaEventRecord(ev[0], ctx->stream);
            if (e == cudaSuccess) st = ens_pair_launch(ctx, E, A, method, var);
            if (e == cudaSuccess && st == BIA_OK) e = cudaEventRecord(ev[1], ctx->stream);
            if (e == cudaSuccess && st == BIA_OK) e = cudaEventSynchronize(ev[1]);
            float t = 0.0f;
            if (e == cudaSuccess && st == BIA_OK) e = cudaEventElapsedTime(&t, ev[0], ev[1]);
            if (rep == 1 || (rep > 1 && t < t_min)) t_min = t;
        }
        if (e != cudaSuccess || st != BIA_OK) break;
        if (ms) ms[var] = t_min;
        if (best < 0 || t_min < best_ms) {
            best = var;
            best_ms = t_min;
        }
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    if (st != BIA_OK) return st;
    // the timing launches counted pairs: clear the counters
    if (e == cudaSuccess) e = cudaMemsetAsync(ctx->stats.ptr, 0, kNumStats * sizeof(unsigned long long), ctx->stream);
    if (e == cudaSuccess) e = ctx->stream ? cudaStreamSynchronize(ctx->stream) : cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_status(e);
    if (E->tuned[method] != best && E->graph_exec) {  // a captured step sequence has the old shape
        cudaGraphExecDestroy(E->graph_exec);
        cudaGraphDestroy(E->graph);
        E->graph_exec = nullptr;
        E->graph = nullptr;
    }
    E->tuned[method] = best;
    if (variant) *variant = best;
    return BIA_OK;
}
