// bia_step.cu -- the BIA pair step on B200: tile kernel, reduction, context and API.
//
// Work decomposition.  The pairs i<j form the upper triangle of an n x n matrix.  It
// is cut into 32 x 32 warp-blocks (bi <= bj, 32-particle row and column blocks); one
// warp owns one warp-block.  Lane l keeps its row particle i = 32*bi + l and its
// column particle j = 32*bj + l in registers.  At rotation step k lane l pairs its
// row with column slot (l + k) mod 32, fetched from that lane with a shuffle, so
// every lane solves a different pair and the column slot's accumulator can be
// handed back by a second shuffle from lane (l - k) mod 32.  Off-diagonal blocks take
// 32 rotation steps (1024 pairs), diagonal blocks 16 (k = 1..15 on all lanes, k = 16
// on lanes 0..15: the 496 pairs of the block once each; orientation does not matter
// because the half-displacement is exactly antisymmetric under i <-> j).
//
// Reduction.  Each warp-block leaves 32 row sums and 32 column sums of the six
// half-displacement components.  Deterministic mode writes them to a partial buffer
// part[m][c][p] in which every (m, p) slot is written exactly once per step (row sums
// of block (bi, bj) at m = bj, column sums at m = bi, the diagonal block's combined
// sums at m = bi), and a second kernel adds the nb partials of each particle in a fixed
// order, adds the drift u*dt and updates the state: the result is bitwise
// reproducible.  Atomic mode adds the sums straight into an accumulator with FP64
// atomics (no partial buffer; summation order varies between runs).
//
// Layout in HBM: state is SoA (x, y, z, u, v, w, optional q), FP64, n entries each;
// partials are [nb][6][nb*32] FP64 (1.5 n^2 bytes); accumulators [6][nb*32].
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "bia_internal.cuh"
#include "bia_learned_block.cuh"
#include "bia_pair.cuh"
#include "bia_tiles.cuh"
#include "mlp_tc.cuh"

namespace bia {

constexpr int kWarpsPerBlock = 8;
constexpr int kThreads = kWarpsPerBlock * 32;

struct StepArgs {
    const double *x, *y, *z, *u, *v, *w, *q;
    double *part;   // deterministic partials, or atomic accumulators
    unsigned long long *stats;
    long long nwb;  // warp-blocks of the launch: t0 .. t0 + nwb - 1 (all: nb*(nb+1)/2)
    long long t0;   // first warp-block (a shard of a multi-GPU step; 0 otherwise)
    int n, nb, npad;
    double eps_th;
    PairParams P;
    const MlpImage *heads;  // BIA_METHOD_LEARNED
    // split learned step (split = true): the deferred pairs' rows and the list of warp-blocks
    // holding them (bia_learned_block.cuh)
    bool split;
    LearnedRows R;
};

// Each warp solves warp-blocks t = (its global warp index) + k * (warps in the grid): one
// block per warp when the grid covers every block, several in a persistent grid (the
// universal-variable and split-step rest kernels launch one resident grid, kPersistentCtas
// CTAs per SM).  The counters are summed per warp in registers and flushed every
// kFlushBlocks blocks: one set of atomics per warp instead of one per block.
template <bool kDeterministic, int M>
__global__ void __launch_bounds__(kThreads, TileOccupancy<M>::kMinBlocks) bia_pair_tiles_kernel(const StepArgs A)
{
    const int lane = threadIdx.x & 31;
    PairCounters tot;
    counters_zero(tot);
    int nblk = 0;
    for (long long tl = (long long)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5); tl < A.nwb;
         tl += (long long)gridDim.x * kWarpsPerBlock) {  // warp-uniform
        int bi, bj;
        warp_block_coords(A.t0 + tl, bi, bj);
        const int i = bi * 32 + lane;
        const int jown = bj * 32 + lane;
        const bool diag = (bi == bj);
        double racc[6], cacc[6];
        PairCounters cnt;
        warp_block_solve<M>(A.x, A.y, A.z, A.u, A.v, A.w, A.q, A.n, A.eps_th, A.P, bi, bj, lane, racc, cacc, cnt);
        counters_add(tot, cnt);
        if (++nblk == kFlushBlocks) {
            flush_counters(tot, A.stats, lane);
            counters_zero(tot);
            nblk = 0;
        }
        const size_t plane = (size_t)A.npad;
        if (kDeterministic) {
            write_partials(A.part, plane, bi, bj, lane, racc, cacc);
        } else {
            if (diag) {
#pragma unroll
                for (int c = 0; c < 6; c++)
                    if (i < A.n) atomicAdd(&A.part[c * plane + i], racc[c] - cacc[c]);
            } else {
#pragma unroll
                for (int c = 0; c < 6; c++) {
                    if (i < A.n) atomicAdd(&A.part[c * plane + i], racc[c]);
                    if (jown < A.n) atomicAdd(&A.part[c * plane + jown], -cacc[c]);
                }
            }
        }
    }
    if (nblk > 0) flush_counters(tot, A.stats, lane);
}

// Phase-locked ALG step kernel (see phase_block_solve): CTAs of kW warps, kMinB of them
// per SM, each warp on one warp-block.  The counters of the CTA's warps are summed in shared
// memory and flushed with one set of atomics per CTA: flushing per warp-block put ~10 atomics
// per block on the same 20 addresses from all kW warps at once (the same kernel without
// counters ran 13 % faster on the Coulomb cube).  (A persistent grid of one CTA per SM, each
// taking groups in a fixed stride, was slower again: the groups' costs differ, and the
// hardware's block scheduler balances them better.)
template <bool kDeterministic, int kW, int kMinB, bool kBalanced = true>
__global__ void __launch_bounds__(kW * 32, kMinB) bia_pair_phase_kernel(const StepArgs A)
{
    extern __shared__ double phase_smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    unsigned long long *slots = reinterpret_cast<unsigned long long *>(phase_smem + kW * phase_slice_doubles<kBalanced>());
    unsigned long long *wtot = slots + warp * kNumStats;
    if (lane < kNumStats) wtot[lane] = 0ull;
    __syncwarp();
    const long long tl = (long long)blockIdx.x * kW + warp;
    const bool live = tl < A.nwb;
    int bi = 0, bj = 0;
    if (live) warp_block_coords(A.t0 + tl, bi, bj);
    double racc[6], cacc[6];
    PairCounters cnt;
    phase_block_solve<kBalanced>(A.x, A.y, A.z, A.u, A.v, A.w, A.q, A.n, A.eps_th, A.P, bi, bj, lane, live,
                      phase_smem + warp * phase_slice_doubles<kBalanced>(), racc, cacc, cnt);
    if (live) {  // warp-uniform
        counters_to_slot(cnt, wtot, lane);
        const int i = bi * 32 + lane;
        const int jown = bj * 32 + lane;
        const size_t plane = (size_t)A.npad;
        if (kDeterministic) {
            write_partials(A.part, plane, bi, bj, lane, racc, cacc);
        } else if (bi == bj) {
#pragma unroll
            for (int c = 0; c < 6; c++)
                if (i < A.n) atomicAdd(&A.part[c * plane + i], racc[c] - cacc[c]);
        } else {
#pragma unroll
            for (int c = 0; c < 6; c++) {
                if (i < A.n) atomicAdd(&A.part[c * plane + i], racc[c]);
                if (jown < A.n) atomicAdd(&A.part[c * plane + jown], -cacc[c]);
            }
        }
    }
    __syncthreads();
    if (warp == 0) flush_slots(slots, kW, A.stats, lane);
}

// ALG pair-kernel shapes the autotuner chooses from (bia_context_autotune):
//   kVarTiles8    8-warp CTAs, per-warp class phases (bia_pair_tiles_kernel)
//   kVarPhase32Lane phase-locked CTAs of 32 warps, 1 per SM, per-lane class loops (rows in
//                 registers: all-hyperbolic systems, where packing saves no turn)
//   kVarPhase32   phase-locked CTAs of 32 warps, 1 per SM (64 registers), balanced class
//                 loops (mixed classes)
// (CTAs of 16 warps, 2 per SM, were never the fastest: Plummer 72.6, Coulomb 111 ms against
// 70.9 and 82.7 ms for kVarPhase32 at n = 32768.)  All shapes give bitwise the same step.
// Without a tuned entry the step takes kVarPhase32 when it gives at least two CTAs per SM,
// else kVarTiles8.
enum AlgVariant { kVarTiles8 = 0, kVarPhase32Lane = 1, kVarPhase32 = 2, kVarCount = 3 };

// the warps' slices, then one counter slot of kNumStats u64 per warp
template <int kW, bool kBalanced = true>
constexpr int phase_smem_bytes()
{
    return kW * (phase_slice_doubles<kBalanced>() + kNumStats) * (int)sizeof(double);
}

// Once per device (the current one): opt the phase-locked kernels in to their dynamic
// shared memory and read the SM count.  Returns the SM count, 0 when the set-up failed
// (the caller then launches the 8-warp kernel).
static int phase_kernel_setup()
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
        ok = ok && cudaFuncSetAttribute(bia_pair_phase_kernel<true, 32, 1>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, phase_smem_bytes<32>()) == cudaSuccess;
        ok = ok && cudaFuncSetAttribute(bia_pair_phase_kernel<false, 32, 1>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, phase_smem_bytes<32>()) == cudaSuccess;
        ok = ok && cudaFuncSetAttribute(bia_pair_phase_kernel<true, 32, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        phase_smem_bytes<32, false>()) == cudaSuccess;
        ok = ok && cudaFuncSetAttribute(bia_pair_phase_kernel<false, 32, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        phase_smem_bytes<32, false>()) == cudaSuccess;
        if (!ok) cudaGetLastError();  // clear; the 8-warp kernel is used instead
        sms_of[dev] = ok ? sms : 0;
        done_of[dev] = true;
    }
    return sms_of[dev];
}

// The variant the step uses for this launch: the tuned one when given (>= 0), else the
// default rule above.
static int alg_variant_for(long long nwb, int tuned)
{
    const int sms = phase_kernel_setup();
    if (sms <= 0 || BIA_PHASE_WARPS == 0) return kVarTiles8;
    if (tuned >= 0 && tuned < kVarCount) return tuned;
    return ((nwb + 31) / 32 >= 2LL * sms) ? kVarPhase32 : kVarTiles8;
}

// CTAs per SM of the persistent universal-variable and rest kernels (their launch bound)
constexpr int kPersistentCtas = 2;

// SM count of the current device (cached per device); 0 when the query fails
int device_sm_count()
{
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static int sms_of[kMaxDevices] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 0;
    std::lock_guard<std::mutex> lk(mu);
    if (sms_of[dev] == 0) {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        sms_of[dev] = sms;
    }
    return sms_of[dev];
}

// the grid of a persistent warp-block kernel: every block covered, at most one resident wave
long long persistent_grid(long long blocks_needed)
{
    const long long cap = (long long)device_sm_count() * kPersistentCtas;
    return (cap > 0 && blocks_needed > cap) ? cap : blocks_needed;
}

static int ilog2_bucket(int n)
{
    int b = 0;
    while ((n >> (b + 1)) > 0 && b < 31) b++;
    return b;
}

template <bool kDeterministic>
static void launch_pair_tiles(const StepArgs &A, long long grid, cudaStream_t st, int tuned = -1)
{
    if (A.P.method == kMethodAlg) {
        const int var = alg_variant_for(A.nwb, tuned);
        if (var == kVarPhase32) {
            bia_pair_phase_kernel<kDeterministic, 32, 1>
                <<<(unsigned)((A.nwb + 31) / 32), 32 * 32, phase_smem_bytes<32>(), st>>>(A);
            return;
        }
        if (var == kVarPhase32Lane) {
            bia_pair_phase_kernel<kDeterministic, 32, 1, false>
                <<<(unsigned)((A.nwb + 31) / 32), 32 * 32, phase_smem_bytes<32, false>(), st>>>(A);
            return;
        }
    }
    switch (A.P.method) {
    case kMethodRkf:
        bia_pair_tiles_kernel<kDeterministic, kMethodRkf><<<(unsigned)grid, kThreads, 0, st>>>(A);
        break;
    case kMethodUniversal:
        bia_pair_tiles_kernel<kDeterministic, kMethodUniversal>
            <<<(unsigned)persistent_grid(grid), kThreads, 0, st>>>(A);
        break;
    default:
        bia_pair_tiles_kernel<kDeterministic, kMethodAlg><<<(unsigned)grid, kThreads, 0, st>>>(A);
        break;
    }
}

// Adds a learned warp-block's sums onto the partials (deterministic: the rest kernel wrote
// every slot first) or into the accumulators; assign: write the slots instead.  With
// assign == false only the slots the added sums touch are read and written: row_hit (this
// lane's row has a pair among them) and col_hit (this lane's column does); the others would
// add zero, so the sums are bitwise the same.
template <bool kDeterministic>
__device__ __forceinline__ void add_learned_sums(const StepArgs &A, int bi, int bj, int lane, const double racc[6],
                                                 const double cacc[6], bool assign, bool row_hit = true,
                                                 bool col_hit = true)
{
    const int i = bi * 32 + lane;
    const int jown = bj * 32 + lane;
    const size_t plane = (size_t)A.npad;
    if (kDeterministic) {
        if (assign) write_partials(A.part, plane, bi, bj, lane, racc, cacc);
        else add_partials(A.part, plane, bi, bj, lane, racc, cacc, row_hit, col_hit);
    } else if (bi == bj) {
        if (row_hit || col_hit) {
#pragma unroll
            for (int c = 0; c < 6; c++)
                if (i < A.n) atomicAdd(&A.part[c * plane + i], racc[c] - cacc[c]);
        }
    } else {
#pragma unroll
        for (int c = 0; c < 6; c++) {
            if (row_hit && i < A.n) atomicAdd(&A.part[c * plane + i], racc[c]);
            if (col_hit && jown < A.n) atomicAdd(&A.part[c * plane + jown], -cacc[c]);
        }
    }
}

// Learned mixed-precision step kernel (BIA_METHOD_LEARNED) in one launch: every pair of
// every warp-block, the learned ones from a head's guess (bia_learned_block.cuh).
template <bool kDeterministic>
__global__ void __launch_bounds__(kMlpThreads, 2) bia_pair_learned_kernel(const StepArgs A)
{
    extern __shared__ uint8_t learned_smem_raw[];
    const LearnedSmem M = learned_smem(learned_smem_raw);
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const long long tl = (long long)blockIdx.x * kLearnedWarps + warp;
    const bool live = tl < A.nwb;
    int bi = 0, bj = 0;
    if (live) warp_block_coords(A.t0 + tl, bi, bj);
    const LearnedBlockIn B = {A.x, A.y, A.z, A.u, A.v, A.w, A.q, A.n, A.eps_th, A.P.dt, A.heads};
    double racc[6], cacc[6];
    PairCounters cnt;
    mlp_setup(*M.mlp);
    uint32_t phase = 0;
    const bool timed_out = learned_block_solve(M, B, bi, bj, lane, live, racc, cacc, cnt, phase);
    mlp_teardown(*M.mlp, phase);
    if (timed_out && threadIdx.x == 0 && !live) atomicAdd(&A.stats[kStatTimeouts], 1ull);
    if (!live) return;  // warp-uniform; no barrier follows
    flush_counters(cnt, A.stats, lane);
    add_learned_sums<kDeterministic>(A, bi, bj, lane, racc, cacc, true);
}

// Split learned step, first kernel (rest_block_solve, rest_block_defer): every warp-block's
// pairs except the deferred ones, whose head inputs go to the rows and whose warp-blocks are
// listed.  Deterministic mode writes every partial slot here; the finish kernel adds onto
// them.  Two CTAs per SM (kPersistentCtas): at three the filter spills registers inside the
// rotation loop.  A persistent grid with the counters flushed per warp, as
// bia_pair_tiles_kernel; dynamic shared memory: each warp's column slice and row slots.
// Warps per CTA of the rest kernel.  At 112 registers the register file would hold 18 warps
// per SM, but CTAs of 9 (96 registers, small spills) or 10 warps (92 registers) are slower:
// 6.45 and 6.50 against 5.61 ms for the learned pair kernels on plummer_32768.
#ifndef BIA_REST_WARPS
#define BIA_REST_WARPS 8
#endif
constexpr int kRestWarps = BIA_REST_WARPS;
constexpr size_t kRestKernelSmemBytes = kRestWarps * kRestWarpBytes;

template <bool kDeterministic>
__global__ void __launch_bounds__(kRestWarps * 32, kPersistentCtas) bia_pair_rest_kernel(const StepArgs A)
{
    extern __shared__ __align__(16) uint8_t rest_smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    double *ws = reinterpret_cast<double *>(rest_smem + warp * kRestWarpBytes);
    uint32_t *wslots = reinterpret_cast<uint32_t *>(rest_smem + warp * kRestWarpBytes +
                                                    kTileSmemDoubles * sizeof(double));
    PairCounters tot;
    counters_zero(tot);
    int nblk = 0;
    for (long long tl = (long long)blockIdx.x * kRestWarps + warp; tl < A.nwb;
         tl += (long long)gridDim.x * kRestWarps) {  // warp-uniform
        const long long t = A.t0 + tl;
        int bi, bj;
        warp_block_coords(t, bi, bj);
        double racc[6], cacc[6];
        uint32_t mask[kMlpHeads];
        PairCounters cnt;
        rest_block_solve(A.x, A.y, A.z, A.u, A.v, A.w, A.q, A.n, A.eps_th, A.P.dt, bi, bj, lane, ws, wslots, racc,
                         cacc, mask, cnt);
        counters_add(tot, cnt);
        if (++nblk == kFlushBlocks) {
            flush_counters(tot, A.stats, lane);
            counters_zero(tot);
            nblk = 0;
        }
        add_learned_sums<kDeterministic>(A, bi, bj, lane, racc, cacc, true);
        rest_block_defer(A.R, (unsigned int)t, mask, wslots, lane);
    }
    if (nblk > 0) flush_counters(tot, A.stats, lane);
}

// Split learned step, second kernel: the rows of both heads on the tensor cores (persistent
// CTAs of kMlpThreads, TMEM allocated once per CTA).  A timed-out pipeline is counted; its
// rows keep their inputs, which the finish kernel's FP64 step rejects (the plain solver
// takes those pairs).
__global__ void __launch_bounds__(kMlpThreads, 2) bia_pair_learned_head_kernel(const LearnedRows R,
                                                                                 const MlpImage *heads,
                                                                                 unsigned long long *stats)
{
    extern __shared__ uint8_t head_rows_smem[];
    MlpSmem &S = *reinterpret_cast<MlpSmem *>(((uintptr_t)head_rows_smem + 1023) & ~(uintptr_t)1023);
    mlp_setup(S);
    uint32_t phase = 0;
    bool ok = head_rows_pass(S, R, heads, kHeadHyp, phase);
    if (ok) ok = head_rows_pass(S, R, heads, kHeadEll, phase);
    mlp_teardown(S, phase);
    if (!ok && threadIdx.x == 0) atomicAdd(&stats[kStatTimeouts], 1ull);
}

// Split learned step, third kernel (persistent 8-warp CTAs, no CTA barrier).  A warp-block
// with many deferred pairs (or on the diagonal) is finished by one warp, one lane per row, the
// list entries spread over the warps one at a time; the others, with at most kBatchPairs
// pairs, are then taken in chunks of 32 list entries, laid end to end and finished 32 pairs
// at a time (finish_batches).  Whether a block is batched depends on the block alone, so
// the step stays deterministic.  (With one warp per warp-block, the Coulomb cube's ~3e5
// listed blocks of one or two pairs each kept a warp for a whole solve per block: 1.0 ms per
// step.)

template <bool kDeterministic>
__global__ void __launch_bounds__(kThreads, 2) bia_pair_learned_finish_kernel(const StepArgs A)
{
    __shared__ double s_fin[kTileWarps][kTileSmemDoubles];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const long long count = (long long)*A.R.nlist;
    const LearnedBlockIn B = {A.x, A.y, A.z, A.u, A.v, A.w, A.q, A.n, A.eps_th, A.P.dt, A.heads};
    PairCounters tot;
    counters_zero(tot);
    int nflush = 0;
    // 1. the dense and diagonal warp-blocks, the list entries spread over the warps one at a
    // time; a warp reads its next 32 entries with one load per lane (not one dependent load
    // per entry) and finishes the dense ones among them in order
    const long long gw = (long long)blockIdx.x * kWarpsPerBlock + warp;
    const long long stride = (long long)gridDim.x * kWarpsPerBlock;
    for (long long k0 = 0; gw + k0 * stride < count; k0 += 32) {  // warp-uniform
        const long long el = gw + (k0 + lane) * stride;
        bool dense = false;
        int lbi = 0, lbj = 0;
        if (el < count) {
            const uint4 ent = A.R.entries[el];
            warp_block_coords((long long)ent.x, lbi, lbj);
            dense = !(lbi != lbj && ent.w <= (unsigned)kBatchPairs);  // else batched below
        }
        for (unsigned dm = __ballot_sync(full, dense); dm; dm &= dm - 1u) {
            const int src = __ffs(dm) - 1;
            const long long e = gw + (k0 + src) * stride;
            const int bi = __shfl_sync(full, lbi, src), bj = __shfl_sync(full, lbj, src);
            double racc[6], cacc[6];
            PairCounters cnt;
            bool row_hit, col_hit;
            finish_block_solve(A.R, e, B, bi, bj, lane, s_fin[warp], racc, cacc, cnt, row_hit, col_hit);
            counters_add(tot, cnt);
            if (++nflush == kFlushBlocks) {
                flush_counters(tot, A.stats, lane);
                counters_zero(tot);
                nflush = 0;
            }
            add_learned_sums<kDeterministic>(A, bi, bj, lane, racc, cacc, false, row_hit, col_hit);
        }
    }
    // 2. the sparse ones, batched per chunk of list entries: up to 32 per warp, fewer when the
    // list is short, so that every warp has a chunk (a block's sums do not depend on the blocks
    // batched with it)
    const long long nwarps = (long long)gridDim.x * kWarpsPerBlock;
    const long long chunk = count >= 32 * nwarps ? 32 : (count + nwarps - 1) / nwarps;
    for (long long c0 = ((long long)blockIdx.x * kWarpsPerBlock + warp) * chunk; c0 < count;
         c0 += nwarps * chunk) {  // warp-uniform
        const long long e = c0 + lane;
        const bool valid = lane < chunk && e < count;
        const uint4 ent = valid ? A.R.entries[e] : make_uint4(0u, 0u, 0u, 0u);
        int bi = 0, bj = 0;
        if (valid) warp_block_coords((long long)ent.x, bi, bj);
        const bool sparse = valid && bi != bj && ent.w <= (unsigned)kBatchPairs;
        if (__ballot_sync(full, sparse) == 0u) continue;
        auto resolve = [&](int l) {
            FinishBlock F;
            F.B = B;
            warp_block_coords((long long)A.R.entries[c0 + l].x, F.bi, F.bj);
            F.part = A.part;
            F.plane = (size_t)A.npad;
            return F;
        };
        PairCounters cnt;
        counters_zero(cnt);
        finish_batches<kDeterministic>(A.R, c0, sparse, ent.w, lane, resolve, cnt);
        counters_add(tot, cnt);
        if (++nflush == kFlushBlocks) {
            flush_counters(tot, A.stats, lane);
            counters_zero(tot);
            nflush = 0;
        }
    }
    if (nflush > 0) flush_counters(tot, A.stats, lane);
}

// Once per device: dynamic shared memory opt-in of the learned kernels; returns the grid of
// the persistent head kernel (resident CTAs on the device), 0 on failure.
static int learned_kernel_setup()
{
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static int grid_of[kMaxDevices] = {};
    static bool done_of[kMaxDevices] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 0;
    std::lock_guard<std::mutex> lk(mu);
    if (!done_of[dev]) {
        const int bytes = (int)kLearnedSmemBytes;
        const int hbytes = (int)(1024 + sizeof(MlpSmem));
        int sms = 0, occ = 0;
        bool ok = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess;
        ok = ok && cudaFuncSetAttribute(bia_pair_learned_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        bytes) == cudaSuccess;
        ok = ok && cudaFuncSetAttribute(bia_pair_learned_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        bytes) == cudaSuccess;
        ok = ok && cudaFuncSetAttribute(bia_pair_rest_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)kRestKernelSmemBytes) == cudaSuccess;
        ok = ok && cudaFuncSetAttribute(bia_pair_rest_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)kRestKernelSmemBytes) == cudaSuccess;
        ok = ok && cudaFuncSetAttribute(bia_pair_learned_head_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        hbytes) == cudaSuccess;
        // the largest shared-memory carveout, so that the occupancy query sees what the
        // launch gets (without it the query assumes the default split: 1 CTA per SM)
        ok = ok && cudaFuncSetAttribute((const void *)bia_pair_learned_head_kernel,
                                        cudaFuncAttributePreferredSharedMemoryCarveout,
                                        (int)cudaSharedmemCarveoutMaxShared) == cudaSuccess;
        ok = ok && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, bia_pair_learned_head_kernel, kMlpThreads,
                                                                 (size_t)hbytes) == cudaSuccess;
        if (!ok) cudaGetLastError();
        // at least the launch bound's two CTAs per SM: CTAs beyond the resident ones wait
        // for a slot, so a low answer costs nothing but a short queue
        grid_of[dev] = ok ? sms * (occ > 2 ? occ : 2) : 0;
        done_of[dev] = true;
    }
    return grid_of[dev];
}

int learned_head_grid() { return learned_kernel_setup(); }

void launch_learned_head(const LearnedRows &R, const MlpImage *heads, unsigned long long *stats, int grid,
                         cudaStream_t st)
{
    bia_pair_learned_head_kernel<<<grid, kMlpThreads, 1024 + sizeof(MlpSmem), st>>>(R, heads, stats);
}

// The learned step's pair launches: one kernel, or (A.split) the rest, head and finish
// kernels.
template <bool kDeterministic>
static int launch_pair_learned(const StepArgs &A, cudaStream_t st)
{
    const int lgrid = learned_kernel_setup();
    if (lgrid <= 0) return BIA_ERR_CUDA;
    if (!A.split) {
        const long long grid = (A.nwb + kLearnedWarps - 1) / kLearnedWarps;
        bia_pair_learned_kernel<kDeterministic><<<(unsigned)grid, kMlpThreads, kLearnedSmemBytes, st>>>(A);
        return BIA_OK;
    }
    // the row counts of both heads and the list length start at zero
    if (cudaMemsetAsync(A.R.counts, 0, kSplitHeader, st) != cudaSuccess) return BIA_ERR_CUDA;
    const long long rgrid = persistent_grid((A.nwb + kRestWarps - 1) / kRestWarps);
    bia_pair_rest_kernel<kDeterministic><<<(unsigned)rgrid, kRestWarps * 32, kRestKernelSmemBytes, st>>>(A);
    launch_learned_head(A.R, A.heads, A.stats, lgrid, st);
    const long long fgrid = persistent_grid((A.nwb + kWarpsPerBlock - 1) / kWarpsPerBlock);
    bia_pair_learned_finish_kernel<kDeterministic><<<(unsigned)fgrid, kThreads, 0, st>>>(A);
    return BIA_OK;
}

// The split learned step's buffer: the row counts and list length (kSplitHeader bytes), the
// list entries (16 bytes per warp-block), the pair masks (2 x 32 words per warp-block) and the
// rows of both heads (4 bytes each, up to kRowsCap per head: 1 GB in all at the cap).
constexpr unsigned int kRowsCap = 1u << 27;
static unsigned int rows_cap(long long nwb)
{
    const unsigned long long pairs = (unsigned long long)nwb * 1024ull;
    return pairs < kRowsCap ? (unsigned int)pairs : kRowsCap;
}
static size_t split_buffer_bytes(long long nwb)
{
    return kSplitHeader + (size_t)nwb * kListBytesPerBlock + (size_t)kMlpHeads * rows_cap(nwb) * sizeof(uint32_t);
}

static void split_buffer_carve(void *base, long long nwb, StepArgs &A)
{
    uint8_t *b = (uint8_t *)base;
    A.split = true;
    A.R.counts = (unsigned long long *)b;
    A.R.nlist = (unsigned int *)(b + 16);
    A.R.entries = (uint4 *)(b + kSplitHeader);
    A.R.masks = (uint32_t *)(b + kSplitHeader + (size_t)nwb * 16);
    A.R.pairs = (uint2 *)(b + kSplitHeader + (size_t)nwb * (16 + 64 * sizeof(uint32_t)));
    uint32_t *rows = (uint32_t *)(b + kSplitHeader + (size_t)nwb * kListBytesPerBlock);
    A.R.rows_cap = rows_cap(nwb);
    A.R.rows[kHeadEll] = rows;
    A.R.rows[kHeadHyp] = rows + A.R.rows_cap;
}

// The learned step splits (plain pairs in the rest kernel, learned pairs in the list
// kernel) at every size unless the autotuner chose the one-kernel layout: the ensemble takes
// the same split, so each of its systems equals its own bia_step bit for bit.
static bool learned_split(long long nwb) { return nwb > 0; }

struct UpdateArgs {
    double *x, *y, *z, *u, *v, *w;
    const double *part;
    double *disp;  // optional [6][n]
    int n, nb, npad, nparts;  // nparts = nb (deterministic) or 1 (atomic)
    double dt;
};

// Sum of the partials in fixed order, drift and state update (bia/bia.f90:194-204).  A CTA
// covers 32 particles with one warp per component: warp c sums component c of its 32
// particles over the nparts planes in plane order (each load is 256 contiguous bytes, and
// six warps per 32 particles keep enough loads in flight to stream the 1.5 n^2 bytes of
// partials), then warp 0 applies the drift and the update.
constexpr int kReduceThreads = 6 * 32;

__global__ void __launch_bounds__(kReduceThreads) bia_reduce_update_kernel(const UpdateArgs A)
{
    __shared__ double s_sum[6][32];
    const int lane = threadIdx.x & 31;
    const int c = threadIdx.x >> 5;
    const int p = blockIdx.x * 32 + lane;
    const size_t plane = (size_t)A.npad;
    if (p < A.n) {
        const double *src = A.part + (size_t)c * plane + p;
        const size_t step = 6 * plane;
        double sum = 0.0;
        int m = 0;
        for (; m + 8 <= A.nparts; m += 8) {
            double t[8];
#pragma unroll
            for (int k = 0; k < 8; k++) t[k] = src[(size_t)(m + k) * step];
#pragma unroll
            for (int k = 0; k < 8; k++) sum += t[k];
        }
        for (; m < A.nparts; m++) sum += src[(size_t)m * step];
        s_sum[c][lane] = sum;
    }
    __syncthreads();
    if (c != 0 || p >= A.n) return;
    const double s[6] = {s_sum[0][lane], s_sum[1][lane], s_sum[2][lane],
                         s_sum[3][lane], s_sum[4][lane], s_sum[5][lane]};
    const double u = A.u[p], v = A.v[p], w = A.w[p];
    const double d[6] = {s[0] + u * A.dt, s[1] + v * A.dt, s[2] + w * A.dt, s[3], s[4], s[5]};
    A.x[p] = A.x[p] + d[0];
    A.y[p] = A.y[p] + d[1];
    A.z[p] = A.z[p] + d[2];
    A.u[p] = u + d[3];
    A.v[p] = v + d[4];
    A.w[p] = w + d[5];
    if (A.disp) {
#pragma unroll
        for (int k = 0; k < 6; k++) A.disp[(size_t)k * A.n + p] = d[k];
    }
}

// ----------------------------------------------------------------------------------
static thread_local int g_last_error = BIA_OK;

int set_last_error(int status)
{
    g_last_error = status;
    return status;
}

int cuda_status(cudaError_t e)
{
    if (e == cudaSuccess) return BIA_OK;
    if (e == cudaErrorMemoryAllocation) return BIA_ERR_OUT_OF_MEMORY;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return BIA_ERR_NO_DEVICE;
    return BIA_ERR_CUDA;
}

static int num_blocks32(int n) { return (n + 31) / 32; }

int ensure_step_buffers(bia_context *ctx, const bia_config *cfg, int n)
{
    const int nb = num_blocks32(n);
    const size_t npad = (size_t)nb * 32;
    cudaError_t e;
    if (cfg->method == BIA_METHOD_LEARNED) {
        const long long nwb = (long long)nb * (nb + 1) / 2;
        if (learned_split(nwb) || ctx->learned_tuned[cfg->deterministic ? 1 : 0][ilog2_bucket(n)] == 1) {
            e = ctx->lmask.reserve(split_buffer_bytes(nwb));
            if (e != cudaSuccess) return cuda_status(e);
        }
    }
    if (cfg->deterministic) {
        e = ctx->part.reserve((size_t)nb * 6 * npad * sizeof(double));
    } else {
        e = ctx->acc.reserve(6 * npad * sizeof(double));
    }
    if (e != cudaSuccess) return cuda_status(e);
    e = ctx->stats.reserve(kNumStats * sizeof(unsigned long long));
    return cuda_status(e);
}

static int validate(const bia_config *cfg, int n, const void *x, const void *y, const void *z,
                    const void *u, const void *v, const void *w, const bia_context *ctx = nullptr)
{
    if (!cfg || n < 1 || !x || !y || !z || !u || !v || !w) return BIA_ERR_INVALID_ARGUMENT;
    const bool learned_ok = cfg->method == BIA_METHOD_LEARNED && ctx && ctx->heads_loaded;
    if (cfg->method != BIA_METHOD_ALG && cfg->method != BIA_METHOD_RKF && cfg->method != BIA_METHOD_UNIVERSAL &&
        !learned_ok)
        return BIA_ERR_INVALID_ARGUMENT;
    if (cfg->itr < 1 || cfg->itr > 62) return BIA_ERR_INVALID_ARGUMENT;
    // 32-bit particle indices and a warp-block count that fits the grid
    if (n > (1 << 30)) return BIA_ERR_INVALID_ARGUMENT;
    return BIA_OK;
}

static void record_event(bia_context *ctx)
{
    if (!ctx->timing) return;
    if (ctx->ev_used == ctx->ev_cap) {
        int cap = ctx->ev_cap ? ctx->ev_cap * 2 : 64;
        cudaEvent_t *ev = (cudaEvent_t *)realloc(ctx->ev, sizeof(cudaEvent_t) * cap);
        if (!ev) return;
        for (int k = ctx->ev_cap; k < cap; k++) cudaEventCreate(&ev[k]);
        ctx->ev = ev;
        ctx->ev_cap = cap;
    }
    cudaEventRecord(ctx->ev[ctx->ev_used++], ctx->stream);
}

// The pair launches of a step over warp-blocks t0 .. t0 + nwb - 1 (all of them: t0 = 0,
// nwb = -1), into the deterministic partials or the atomic accumulators of the context.
static int enqueue_pairs(bia_context *ctx, const bia_config *cfg, int n, double *x, double *y, double *z,
                         double *u, double *v, double *w, const double *q, long long t0, long long nwb)
{
    const int nb = num_blocks32(n);
    StepArgs A{};
    A.x = x; A.y = y; A.z = z; A.u = u; A.v = v; A.w = w; A.q = q;
    A.stats = (unsigned long long *)ctx->stats.ptr;
    A.n = n;
    A.nb = nb;
    A.npad = nb * 32;
    const long long all = (long long)nb * (nb + 1) / 2;
    A.t0 = t0;
    A.nwb = nwb < 0 ? all : nwb;
    A.eps_th = cfg->eps_th;
    A.P.dt = cfg->dt;
    A.P.err = cfg->err;
    A.P.relerr = cfg->rkf_relerr;
    A.P.abserr = cfg->rkf_abserr;
    A.P.itr = cfg->itr;
    A.P.method = cfg->method;
    const long long grid = (A.nwb + kWarpsPerBlock - 1) / kWarpsPerBlock;
    A.heads = (const MlpImage *)ctx->heads.ptr;
    const bool learned = cfg->method == BIA_METHOD_LEARNED;
    bool split = false;
    if (learned) {
        const int lt = ctx->learned_tuned[cfg->deterministic ? 1 : 0][ilog2_bucket(n)];
        split = (lt >= 0) ? (lt == 1 && ctx->lmask.ptr) : learned_split(all);
    }
    if (split) split_buffer_carve(ctx->lmask.ptr, all, A);
    else A.split = false;
    if (learned && !ctx->heads_loaded) return BIA_ERR_INVALID_ARGUMENT;
    if (A.nwb == 0) {  // an empty shard: nothing to launch (the accumulators are cleared)
        if (!cfg->deterministic)
            return cuda_status(cudaMemsetAsync(ctx->acc.ptr, 0, 6 * (size_t)A.npad * sizeof(double), ctx->stream));
        return BIA_OK;
    }
    int st = BIA_OK;
    if (cfg->deterministic) {
        A.part = (double *)ctx->part.ptr;
        record_event(ctx);
        if (learned) st = launch_pair_learned<true>(A, ctx->stream);
        else launch_pair_tiles<true>(A, grid, ctx->stream, ctx->alg_tuned[1][ilog2_bucket(n)]);
        record_event(ctx);
    } else {
        A.part = (double *)ctx->acc.ptr;
        cudaMemsetAsync(A.part, 0, 6 * (size_t)A.npad * sizeof(double), ctx->stream);
        record_event(ctx);
        if (learned) st = launch_pair_learned<false>(A, ctx->stream);
        else launch_pair_tiles<false>(A, grid, ctx->stream, ctx->alg_tuned[0][ilog2_bucket(n)]);
        record_event(ctx);
    }
    return st;
}

int enqueue_step(bia_context *ctx, const bia_config *cfg, int n, double *x, double *y, double *z,
                 double *u, double *v, double *w, const double *q, double *disp)
{
    const int st = enqueue_pairs(ctx, cfg, n, x, y, z, u, v, w, q, 0, -1);
    if (st != BIA_OK) return st;
    const int nb = num_blocks32(n);
    UpdateArgs U;
    U.x = x; U.y = y; U.z = z; U.u = u; U.v = v; U.w = w;
    U.disp = disp;
    U.n = n;
    U.nb = nb;
    U.npad = nb * 32;
    U.dt = cfg->dt;
    U.part = cfg->deterministic ? (double *)ctx->part.ptr : (double *)ctx->acc.ptr;
    U.nparts = cfg->deterministic ? nb : 1;
    bia_reduce_update_kernel<<<(n + 31) / 32, kReduceThreads, 0, ctx->stream>>>(U);
    return cuda_status(cudaGetLastError());
}

// ----------------------------------------------------------------------------------
// Multi-GPU shards.  Shard s of S owns the warp-blocks of the triangle's columns
// [c0, c1) (column bj holds bj + 1 blocks; the boundaries split the blocks, so the pairs, as
// evenly as whole columns allow).  Those blocks are one contiguous range of the linear order
// t = bj (bj + 1) / 2 + bi, and they write these partial planes of particle p (block b):
// rows, m = bj for bj in [max(c0, b + 1), c1), and, when b is one of the shard's columns,
// columns and diagonal, m = 0 .. b.  The shard's reduction sums exactly those planes in
// ascending m, the order of the whole step's reduction.
void shard_columns(int nb, int shard, int nshards, int *c0, int *c1)
{
    const long long all = (long long)nb * (nb + 1) / 2;
    auto boundary = [&](int r) {
        if (r <= 0) return 0;
        if (r >= nshards) return nb;
        const long long target = (all * r + nshards - 1) / nshards;  // ceil(all r / S) blocks
        long long c = (long long)((sqrt(8.0 * (double)target + 1.0) - 1.0) * 0.5);
        while (c > 0 && c * (c + 1) / 2 >= target) c--;
        while (c * (c + 1) / 2 < target) c++;
        return (int)(c < nb ? c : nb);
    };
    *c0 = boundary(shard);
    *c1 = boundary(shard + 1);
}

struct ShardReduceArgs {
    const double *part;
    double *out;  // [6][n]
    int n, npad, c0, c1;
    bool atomic;  // part is the atomic-mode accumulator (one plane, the shard's sums only)
};

// out[c][p] = the shard's partial planes of particle p summed in ascending plane order
// (deterministic), or the atomic accumulator: one warp per component per 32 particles, as
// bia_reduce_update_kernel.
__global__ void __launch_bounds__(kReduceThreads) bia_shard_reduce_kernel(const ShardReduceArgs A)
{
    const int lane = threadIdx.x & 31;
    const int c = threadIdx.x >> 5;
    const int p = blockIdx.x * 32 + lane;
    if (p >= A.n) return;
    const size_t plane = (size_t)A.npad;
    const double *src = A.part + (size_t)c * plane + p;
    const size_t step = 6 * plane;
    double sum = 0.0;
    if (A.atomic) {
        sum = src[0];
    } else {
        const int b = p / 32;
        if (b >= A.c0 && b < A.c1)
            for (int m = 0; m <= b; m++) sum += src[(size_t)m * step];
        for (int m = max(A.c0, b + 1); m < A.c1; m++) sum += src[(size_t)m * step];
    }
    A.out[(size_t)c * A.n + p] = sum;
}

// x += sums[0..2] + u dt, u += sums[3..5] (bia/bia.f90:194-204)
__global__ void __launch_bounds__(256) bia_apply_update_kernel(int n, double dt, double *x, double *y, double *z,
                                                                 double *u, double *v, double *w, const double *sums)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const double uu = u[p], vv = v[p], ww = w[p];
    x[p] = x[p] + (sums[p] + uu * dt);
    y[p] = y[p] + (sums[(size_t)n + p] + vv * dt);
    z[p] = z[p] + (sums[2 * (size_t)n + p] + ww * dt);
    u[p] = uu + sums[3 * (size_t)n + p];
    v[p] = vv + sums[4 * (size_t)n + p];
    w[p] = ww + sums[5 * (size_t)n + p];
}

static void copy_stats(const unsigned long long *h, bia_stats *s)
{
    s->hyperbola = (long long)h[0];
    s->parabola = (long long)h[1];
    s->ellipse = (long long)h[2];
    s->degenerate = (long long)h[3];
    s->rkf = (long long)h[4];
    s->universal = (long long)h[5];
    s->iter_hyperbola = (long long)h[6];
    s->iter_ellipse = (long long)h[7];
    s->iter_parabola = (long long)h[8];
    s->iter_universal = (long long)h[9];
    s->iterations = s->iter_hyperbola + s->iter_ellipse + s->iter_parabola;
    s->rkf_steps = (long long)h[10];
    s->nonconverged = (long long)h[11];
    s->bracket_exits = (long long)h[12];
    s->fallbacks = (long long)h[13];
    s->nonfinite = (long long)h[14];
    s->learned = (long long)h[15];
    s->learned_fallbacks = (long long)h[16];
    s->learned_coarse = (long long)h[17];
    s->timeouts = (long long)h[18];
    s->learned_fp32_steps = (long long)h[19];
}

static int fetch_stats(bia_context *ctx, bia_stats *stats)
{
    cudaError_t e = cudaMemcpyAsync(ctx->h_stats, ctx->stats.ptr, kNumStats * sizeof(unsigned long long),
                                    cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_status(e);
    copy_stats(ctx->h_stats, stats);
    if (stats->timeouts) return BIA_ERR_DEVICE_TIMEOUT;
    return stats->nonfinite ? BIA_ERR_NONFINITE : BIA_OK;
}

}  // namespace bia

using namespace bia;

extern "C" {

void bia_config_default(bia_config *cfg)
{
    if (!cfg) return;
    cfg->method = BIA_METHOD_ALG;
    cfg->itr = 18;
    cfg->eps_th = -6e-7;
    cfg->dt = 1.0;
    cfg->err = 1e-12;
    cfg->rkf_relerr = 0.0;
    cfg->rkf_abserr = 1e-16;
    cfg->deterministic = 1;
}

const char *bia_status_string(int status)
{
    switch (status) {
    case BIA_OK: return "ok";
    case BIA_ERR_INVALID_ARGUMENT: return "invalid argument";
    case BIA_ERR_NONFINITE: return "a pair produced a non-finite displacement";
    case BIA_ERR_NOT_CONVERGED: return "solver did not converge";
    case BIA_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
    case BIA_ERR_CUDA: return "CUDA runtime error";
    case BIA_ERR_OUT_OF_MEMORY: return "out of device memory";
    case BIA_ERR_NO_DEVICE: return "no CUDA device";
    default: return "unknown status";
    }
}

int bia_last_error(void) { return g_last_error; }

int bia_context_create(bia_context **out, int device, void *stream)
{
    if (!out) return BIA_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return BIA_ERR_NO_DEVICE;
    if (device < 0 || device >= count) return BIA_ERR_INVALID_ARGUMENT;
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_status(e);
    bia_context *ctx = new bia_context();
    ctx->device = device;
    for (int d = 0; d < 2; d++)
        for (int b = 0; b < 32; b++) ctx->alg_tuned[d][b] = ctx->learned_tuned[d][b] = -1;
    ctx->stream = (cudaStream_t)stream;
    e = cudaMallocHost((void **)&ctx->h_stats, kNumStats * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&ctx->h_inv, 64 * sizeof(double));
    if (e == cudaSuccess) e = ctx->stats.reserve(kNumStats * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(ctx->stats.ptr, 0, kNumStats * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        bia_context_destroy(ctx);
        return cuda_status(e);
    }
    *out = ctx;
    return BIA_OK;
}

int bia_context_set_heads(bia_context *ctx, const void *blob, size_t bytes)
{
    if (!ctx || !blob) return BIA_ERR_INVALID_ARGUMENT;
    const size_t want = 16 + (size_t)kMlpHeads * sizeof(MlpHead);
    if (bytes != want) return BIA_ERR_INVALID_ARGUMENT;
    const unsigned char *b = (const unsigned char *)blob;
    uint32_t version = 0, nheads = 0;
    memcpy(&version, b + 8, 4);
    memcpy(&nheads, b + 12, 4);
    if (memcmp(b, "BIAHEAD1", 8) != 0 || version != 1 || nheads != (uint32_t)kMlpHeads)
        return BIA_ERR_INVALID_ARGUMENT;
    // the kernels' image of each head (weights in the shared-memory operand layout)
    MlpImage img[kMlpHeads];
    for (int h = 0; h < kMlpHeads; h++) {
        MlpHead H;
        memcpy(&H, b + 16 + (size_t)h * sizeof(MlpHead), sizeof(MlpHead));
        memset(&img[h], 0, sizeof(MlpImage));
        mlp_image_from_head(H, img[h]);
    }
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess) e = ctx->heads.reserve(kMlpHeads * sizeof(MlpImage));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ctx->heads.ptr, img, kMlpHeads * sizeof(MlpImage), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = ctx->stream ? cudaStreamSynchronize(ctx->stream) : cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_status(e);
    ctx->heads_loaded = true;
    return BIA_OK;
}

int bia_context_autotune(bia_context *ctx, const bia_config *cfg, int n, double *x, double *y, double *z,
                         double *u, double *v, double *w, const double *q, int *variant, float *ms)
{
    int st = validate(cfg, n, x, y, z, u, v, w, ctx);
    if (!ctx) return set_last_error(BIA_ERR_INVALID_ARGUMENT);
    if (st != BIA_OK) return set_last_error(st);
    if (variant) *variant = -1;
    if (ms)
        for (int k = 0; k < kVarCount; k++) ms[k] = -1.0f;
    if (cfg->method != BIA_METHOD_ALG && cfg->method != BIA_METHOD_LEARNED)
        return set_last_error(BIA_OK);  // one shape only
    cudaError_t e = cudaSetDevice(ctx->device);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (e == cudaSuccess && ctx->stream) e = cudaStreamIsCapturing(ctx->stream, &cap);
    if (e != cudaSuccess) return set_last_error(cuda_status(e));
    if (cap != cudaStreamCaptureStatusNone) return set_last_error(BIA_ERR_INVALID_ARGUMENT);
    st = ensure_step_buffers(ctx, cfg, n);
    if (st != BIA_OK) return set_last_error(st);
    const int nb = num_blocks32(n);
    StepArgs A{};
    A.x = x; A.y = y; A.z = z; A.u = u; A.v = v; A.w = w; A.q = q;
    A.stats = (unsigned long long *)ctx->stats.ptr;
    A.n = n; A.nb = nb; A.npad = nb * 32;
    A.nwb = (long long)nb * (nb + 1) / 2;
    A.eps_th = cfg->eps_th;
    A.P.dt = cfg->dt; A.P.err = cfg->err; A.P.relerr = cfg->rkf_relerr; A.P.abserr = cfg->rkf_abserr;
    A.P.itr = cfg->itr; A.P.method = cfg->method;
    A.heads = (const MlpImage *)ctx->heads.ptr;
    A.split = false;
    const int det = cfg->deterministic ? 1 : 0;
    A.part = det ? (double *)ctx->part.ptr : (double *)ctx->acc.ptr;
    const bool learned = cfg->method == BIA_METHOD_LEARNED;
    if (learned) {  // layouts: 0 one kernel, 1 split (the rest, head and finish kernels)
        e = ctx->lmask.reserve(split_buffer_bytes(A.nwb));
        if (e != cudaSuccess) return set_last_error(cuda_status(e));
    }
    const int nvar = learned ? 2 : kVarCount;
    const long long grid = (A.nwb + kWarpsPerBlock - 1) / kWarpsPerBlock;
    const int sms = phase_kernel_setup();
    cudaEvent_t ev[2];
    e = cudaEventCreate(&ev[0]);
    if (e == cudaSuccess) e = cudaEventCreate(&ev[1]);
    if (e != cudaSuccess) return set_last_error(cuda_status(e));
    int best = -1;
    float best_ms = 0.0f;
    for (int var = 0; var < nvar && e == cudaSuccess; var++) {
        if (!learned && var != kVarTiles8 && sms <= 0) continue;
        float t_min = 0.0f;
        for (int rep = 0; rep < 4 && e == cudaSuccess; rep++) {  // the first launch is a warm-up
            if (!det) e = cudaMemsetAsync(A.part, 0, 6 * (size_t)A.npad * sizeof(double), ctx->stream);
            if (e == cudaSuccess) e = cudaEventRecord(ev[0], ctx->stream);
            int lst = BIA_OK;
            if (learned) {
                A.split = false;
                if (var == 1) split_buffer_carve(ctx->lmask.ptr, A.nwb, A);
                lst = det ? launch_pair_learned<true>(A, ctx->stream) : launch_pair_learned<false>(A, ctx->stream);
            } else if (det) {
                launch_pair_tiles<true>(A, grid, ctx->stream, var);
            } else {
                launch_pair_tiles<false>(A, grid, ctx->stream, var);
            }
            if (lst != BIA_OK) e = cudaErrorUnknown;
            if (e == cudaSuccess) e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaEventRecord(ev[1], ctx->stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(ev[1]);
            float t = 0.0f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&t, ev[0], ev[1]);
            if (rep == 1 || (rep > 1 && t < t_min)) t_min = t;
        }
        if (e != cudaSuccess) break;
        if (ms) ms[var] = t_min;
        if (best < 0 || t_min < best_ms) {
            best = var;
            best_ms = t_min;
        }
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    // the timing launches counted pairs: clear the counters
    if (e == cudaSuccess) e = cudaMemsetAsync(ctx->stats.ptr, 0, kNumStats * sizeof(unsigned long long), ctx->stream);
    if (e == cudaSuccess) e = ctx->stream ? cudaStreamSynchronize(ctx->stream) : cudaDeviceSynchronize();
    if (e != cudaSuccess) return set_last_error(cuda_status(e));
    if (learned) ctx->learned_tuned[det][ilog2_bucket(n)] = best;
    else ctx->alg_tuned[det][ilog2_bucket(n)] = best;
    if (variant) *variant = best;
    return set_last_error(BIA_OK);
}

int bia_context_set_shape(bia_context *ctx, int method, int deterministic, int n, int variant)
{
    if (!ctx || n < 1) return set_last_error(BIA_ERR_INVALID_ARGUMENT);
    const int det = deterministic ? 1 : 0;
    if (method == BIA_METHOD_ALG) {
        if (variant < -1 || variant >= kVarCount) return set_last_error(BIA_ERR_INVALID_ARGUMENT);
        ctx->alg_tuned[det][ilog2_bucket(n)] = variant;
    } else if (method == BIA_METHOD_LEARNED) {
        if (variant < -1 || variant > 1) return set_last_error(BIA_ERR_INVALID_ARGUMENT);
        ctx->learned_tuned[det][ilog2_bucket(n)] = variant;
    } else {
        return set_last_error(BIA_ERR_INVALID_ARGUMENT);  // one shape only
    }
    return set_last_error(BIA_OK);
}

int bia_context_destroy(bia_context *ctx)
{
    if (!ctx) return BIA_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    else cudaDeviceSynchronize();
    if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
    if (ctx->graph) cudaGraphDestroy(ctx->graph);
    for (int k = 0; k < ctx->ev_cap; k++) cudaEventDestroy(ctx->ev[k]);
    free(ctx->ev);
    ctx->part.release();
    ctx->acc.release();
    ctx->heads.release();
    ctx->lmask.release();
    ctx->stats.release();
    ctx->state.release();
    ctx->inv.release();
    ctx->dim.release();
    if (ctx->h_dim) cudaFreeHost(ctx->h_dim);
    if (ctx->h_stats) cudaFreeHost(ctx->h_stats);
    if (ctx->h_inv) cudaFreeHost(ctx->h_inv);
    delete ctx;
    return BIA_OK;
}

int bia_context_set_stream(bia_context *ctx, void *stream)
{
    if (!ctx) return BIA_ERR_INVALID_ARGUMENT;
    ctx->stream = (cudaStream_t)stream;
    return BIA_OK;
}

int bia_context_set_timing(bia_context *ctx, int on)
{
    if (!ctx) return BIA_ERR_INVALID_ARGUMENT;
    ctx->timing = on != 0;
    ctx->ev_used = 0;
    return BIA_OK;
}

int bia_context_stats(bia_context *ctx, bia_stats *stats, int reset)
{
    if (!ctx || !stats) return BIA_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    int st = fetch_stats(ctx, stats);
    if (st != BIA_OK && st != BIA_ERR_NONFINITE) return st;
    if (reset) {
        cudaError_t e = cudaMemsetAsync(ctx->stats.ptr, 0, kNumStats * sizeof(unsigned long long), ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) return cuda_status(e);
    }
    return st;
}

int bia_context_kernel_ms(bia_context *ctx, double *ms, long long *launches)
{
    if (!ctx || !ms) return BIA_ERR_INVALID_ARGUMENT;
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_status(e);
    double total = 0.0;
    long long cnt = 0;
    for (int k = 0; k + 1 < ctx->ev_used; k += 2) {
        float t = 0.f;
        if (cudaEventElapsedTime(&t, ctx->ev[k], ctx->ev[k + 1]) == cudaSuccess) {
            total += t;
            cnt++;
        }
    }
    *ms = total;
    if (launches) *launches = cnt;
    ctx->ev_used = 0;
    return BIA_OK;
}

int bia_step(bia_context *ctx, const bia_config *cfg, int n, double *x, double *y, double *z,
             double *u, double *v, double *w, const double *q, double *disp, bia_stats *stats)
{
    if (!ctx) return BIA_ERR_INVALID_ARGUMENT;
    int st = validate(cfg, n, x, y, z, u, v, w, ctx);
    if (st != BIA_OK) return st;
    cudaSetDevice(ctx->device);
    st = ensure_step_buffers(ctx, cfg, n);
    if (st != BIA_OK) return st;
    if (stats) {
        cudaError_t e = cudaMemsetAsync(ctx->stats.ptr, 0, kNumStats * sizeof(unsigned long long), ctx->stream);
        if (e != cudaSuccess) return cuda_status(e);
    }
    st = enqueue_step(ctx, cfg, n, x, y, z, u, v, w, q, disp);
    if (st != BIA_OK) return st;
    if (stats) return fetch_stats(ctx, stats);
    return BIA_OK;
}

int bia_run(bia_context *ctx, const bia_config *cfg, int n, double *x, double *y, double *z,
            double *u, double *v, double *w, const double *q, int nsteps, int use_graph,
            bia_stats *stats)
{
    if (!ctx || nsteps < 0) return BIA_ERR_INVALID_ARGUMENT;
    int st = validate(cfg, n, x, y, z, u, v, w, ctx);
    if (st != BIA_OK) return st;
    cudaSetDevice(ctx->device);
    st = ensure_step_buffers(ctx, cfg, n);
    if (st != BIA_OK) return st;
    cudaError_t e = cudaSuccess;
    if (stats) {
        e = cudaMemsetAsync(ctx->stats.ptr, 0, kNumStats * sizeof(unsigned long long), ctx->stream);
        if (e != cudaSuccess) return cuda_status(e);
    }
    // a capturing stream needs a non-default stream; timing events are per launch, so
    // graph replay is only used with timing off
    if (use_graph && ctx->stream && !ctx->timing && nsteps > 0) {
        // one-time kernel attribute set-up happens before the capture begins
        if (cfg->method == BIA_METHOD_LEARNED && !learned_kernel_setup()) return BIA_ERR_CUDA;
        if (cfg->method == BIA_METHOD_ALG) phase_kernel_setup();
        GraphKey key;
        key.n = n; key.nsteps = nsteps; key.method = cfg->method; key.itr = cfg->itr;
        key.deterministic = cfg->deterministic; key.eps = cfg->eps_th; key.dt = cfg->dt;
        key.err = cfg->err; key.relerr = cfg->rkf_relerr; key.abserr = cfg->rkf_abserr;
        const void *p[7] = {x, y, z, u, v, w, q};
        for (int k = 0; k < 7; k++) key.ptrs[k] = p[k];
        if (!ctx->graph_exec || !(key == ctx->graph_key)) {
            if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
            if (ctx->graph) cudaGraphDestroy(ctx->graph);
            ctx->graph_exec = nullptr;
            ctx->graph = nullptr;
            e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) return cuda_status(e);
            int est = BIA_OK;
            for (int s = 0; s < nsteps && est == BIA_OK; s++)
                est = enqueue_step(ctx, cfg, n, x, y, z, u, v, w, q, nullptr);
            e = cudaStreamEndCapture(ctx->stream, &ctx->graph);
            if (est != BIA_OK) return est;
            if (e != cudaSuccess) return cuda_status(e);
            e = cudaGraphInstantiate(&ctx->graph_exec, ctx->graph, 0);
            if (e != cudaSuccess) return cuda_status(e);
            ctx->graph_key = key;
        }
        e = cudaGraphLaunch(ctx->graph_exec, ctx->stream);
        if (e != cudaSuccess) return cuda_status(e);
    } else {
        for (int s = 0; s < nsteps; s++) {
            st = enqueue_step(ctx, cfg, n, x, y, z, u, v, w, q, nullptr);
            if (st != BIA_OK) return st;
        }
    }
    if (stats) return fetch_stats(ctx, stats);
    return cuda_status(cudaGetLastError());
}

int bia_run_host(bia_context *ctx, const bia_config *cfg, int n, double *x, double *y, double *z,
                 double *u, double *v, double *w, const double *q, int nsteps, bia_stats *stats)
{
    if (!ctx) return BIA_ERR_INVALID_ARGUMENT;
    int st = validate(cfg, n, x, y, z, u, v, w, ctx);
    if (st != BIA_OK) return st;
    cudaSetDevice(ctx->device);
    cudaError_t e = ctx->state.reserve((size_t)7 * n * sizeof(double));
    if (e != cudaSuccess) return cuda_status(e);
    double *d = (double *)ctx->state.ptr;
    double *host[6] = {x, y, z, u, v, w};
    // six arrays back to back in host memory (a [6][n] state) move in one copy each way
    bool packed = true;
    for (int k = 1; k < 6; k++) packed = packed && host[k] == x + (size_t)k * n;
    const int ncopies = packed ? 1 : 6;
    const size_t copy_bytes = (packed ? 6 : 1) * (size_t)n * sizeof(double);
    for (int k = 0; k < ncopies; k++) {
        e = cudaMemcpyAsync(d + (size_t)k * n, host[k], copy_bytes, cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) return cuda_status(e);
    }
    const double *dq = nullptr;
    if (q) {
        e = cudaMemcpyAsync(d + (size_t)6 * n, q, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) return cuda_status(e);
        dq = d + (size_t)6 * n;
    }
    st = bia_run(ctx, cfg, n, d, d + n, d + 2 * (size_t)n, d + 3 * (size_t)n, d + 4 * (size_t)n,
                 d + 5 * (size_t)n, dq, nsteps, 1, stats);
    if (st != BIA_OK && st != BIA_ERR_NONFINITE) return st;
    int st2 = st;
    for (int k = 0; k < ncopies; k++) {
        e = cudaMemcpyAsync(host[k], d + (size_t)k * n, copy_bytes, cudaMemcpyDeviceToHost, ctx->stream);
        if (e != cudaSuccess) return cuda_status(e);
    }
    e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_status(e);
    return st2;
}

int bia_shard_columns(int n, int shard, int nshards, int *c0, int *c1)
{
    if (n < 1 || nshards < 1 || shard < 0 || shard >= nshards || !c0 || !c1) return BIA_ERR_INVALID_ARGUMENT;
    shard_columns(num_blocks32(n), shard, nshards, c0, c1);
    return BIA_OK;
}

int bia_step_shard(bia_context *ctx, const bia_config *cfg, int n, double *x, double *y, double *z, double *u,
                   double *v, double *w, const double *q, int shard, int nshards, double *sums, bia_stats *stats)
{
    if (!ctx || !sums || nshards < 1 || shard < 0 || shard >= nshards) return BIA_ERR_INVALID_ARGUMENT;
    int st = validate(cfg, n, x, y, z, u, v, w, ctx);
    if (st != BIA_OK) return st;
    cudaSetDevice(ctx->device);
    st = ensure_step_buffers(ctx, cfg, n);
    if (st != BIA_OK) return st;
    if (stats) {
        cudaError_t e = cudaMemsetAsync(ctx->stats.ptr, 0, kNumStats * sizeof(unsigned long long), ctx->stream);
        if (e != cudaSuccess) return cuda_status(e);
    }
    const int nb = num_blocks32(n);
    int c0 = 0, c1 = 0;
    shard_columns(nb, shard, nshards, &c0, &c1);
    const long long t0 = (long long)c0 * (c0 + 1) / 2, t1 = (long long)c1 * (c1 + 1) / 2;
    st = enqueue_pairs(ctx, cfg, n, x, y, z, u, v, w, q, t0, t1 - t0);
    if (st != BIA_OK) return st;
    ShardReduceArgs R;
    R.part = cfg->deterministic ? (const double *)ctx->part.ptr : (const double *)ctx->acc.ptr;
    R.out = sums;
    R.n = n;
    R.npad = nb * 32;
    R.atomic = !cfg->deterministic;
    R.c0 = c0;
    R.c1 = c1;
    bia_shard_reduce_kernel<<<(n + 31) / 32, kReduceThreads, 0, ctx->stream>>>(R);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e);
    if (stats) return fetch_stats(ctx, stats);
    return BIA_OK;
}

int bia_apply_update(bia_context *ctx, int n, double dt, double *x, double *y, double *z, double *u, double *v,
                     double *w, const double *sums)
{
    if (!ctx || n < 1 || !x || !y || !z || !u || !v || !w || !sums) return BIA_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    bia_apply_update_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(n, dt, x, y, z, u, v, w, sums);
    return cuda_status(cudaGetLastError());
}

}  // extern "C"

// ----------------------------------------------------------------------------------
// Allocation-free BIA step.
//
// Some callers cannot allocate device memory once they are running: a host process
// whose GPU memory is handed out by another framework's pool up front, a real-time
// loop that must not touch the CUDA allocator, or code that enqueues work where a
// cudaMalloc would synchronise or fail.  For them the step's scratch (the
// deterministic per-block partial sums and the step counters) lives in a file-scope
// __device__ array of fixed size instead of a context's buffers, so one call only
// enqueues kernels and a memset on the caller's stream.
//
// Limit: n <= kNoAllocMaxN = 2048 particles (partials nb x 6 x 2048 doubles with
// nb = 64: 6 MiB, plus 256 bytes of counters).  Every GPU that loads this library
// holds the array until the process exits.
namespace bia {

constexpr int kNoAllocMaxN = 2048;
constexpr int kNoAllocNb = kNoAllocMaxN / 32;
constexpr size_t kNoAllocPartDoubles = (size_t)kNoAllocNb * 6 * kNoAllocMaxN;
constexpr int kNoAllocMaxDevices = 64;

// Partials first, then the counters (32 doubles of room for kNumStats u64).
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocPartDoubles + 32];

// Device address of g_noalloc_scratch per device ordinal.  The host-side name of the
// array is only a stand-in: it must be resolved with cudaGetSymbolAddress while the
// device is current.  It is resolved again on every call made outside stream capture (a
// cheap query that allocates nothing), so a device reset or a recreated primary context,
// which loads the module again at a new address, is picked up; during a capture the
// address of the last call outside capture is used.
static double *g_noalloc_addr[kNoAllocMaxDevices] = {};
static std::mutex g_noalloc_mutex;

static int noalloc_scratch(cudaStream_t s, double **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e);
    if (dev < 0 || dev >= kNoAllocMaxDevices) return BIA_ERR_INVALID_ARGUMENT;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(s, &cap);
    if (e != cudaSuccess) return cuda_status(e);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (cap == cudaStreamCaptureStatusNone || !g_noalloc_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_status(e);
        g_noalloc_addr[dev] = (double *)p;
    }
    *out = g_noalloc_addr[dev];
    return BIA_OK;
}

}  // namespace bia

extern "C" int bia_step_noalloc(const bia_config *cfg, int n, double *x, double *y, double *z, double *u,
                                double *v, double *w, const double *q, double *disp, void *stream)
{
    int st = validate(cfg, n, x, y, z, u, v, w);
    if (st != BIA_OK) return set_last_error(st);
    if (n > kNoAllocMaxN) return set_last_error(BIA_ERR_INVALID_ARGUMENT);  // beyond the fixed scratch
    cudaStream_t s = (cudaStream_t)stream;
    double *part = nullptr;
    st = noalloc_scratch(s, &part);
    if (st != BIA_OK) return set_last_error(st);
    unsigned long long *counters = (unsigned long long *)(part + kNoAllocPartDoubles);
    // the partials are fully rewritten by every step; only the counters start at zero
    cudaError_t e = cudaMemsetAsync(counters, 0, kNumStats * sizeof(unsigned long long), s);
    if (e != cudaSuccess) return set_last_error(cuda_status(e));
    const int nb = (n + 31) / 32;
    StepArgs A{};
    A.x = x; A.y = y; A.z = z; A.u = u; A.v = v; A.w = w; A.q = q;
    A.part = part;
    A.stats = counters;
    A.n = n;
    A.nb = nb;
    A.npad = nb * 32;
    A.nwb = (long long)nb * (nb + 1) / 2;
    A.eps_th = cfg->eps_th;
    A.P.dt = cfg->dt;
    A.P.err = cfg->err;
    A.P.relerr = cfg->rkf_relerr;
    A.P.abserr = cfg->rkf_abserr;
    A.P.itr = cfg->itr;
    A.P.method = cfg->method;
    const long long grid = (A.nwb + kWarpsPerBlock - 1) / kWarpsPerBlock;
    launch_pair_tiles<true>(A, grid, s);
    UpdateArgs U;
    U.x = x; U.y = y; U.z = z; U.u = u; U.v = v; U.w = w;
    U.part = part;
    U.disp = disp;
    U.n = n;
    U.nb = nb;
    U.npad = nb * 32;
    U.nparts = nb;
    U.dt = cfg->dt;
    bia_reduce_update_kernel<<<(n + 31) / 32, kReduceThreads, 0, s>>>(U);
    return set_last_error(cuda_status(cudaGetLastError()));
}

// ---------------------------------------------------------------------------------------
// Head evaluation on its own (tests of the tensor-core network path).
namespace bia {
__global__ void __launch_bounds__(kMlpThreads, 1) bia_head_eval_kernel(const MlpImage *heads, int head, int n,
                                                                      const float *in, float *out,
                                                                      unsigned long long *timeouts)
{
    extern __shared__ uint8_t head_smem_raw[];
    uint8_t *base = (uint8_t *)(((uintptr_t)head_smem_raw + 1023) & ~(uintptr_t)1023);
    MlpSmem &S = *reinterpret_cast<MlpSmem *>(base);
    mlp_setup(S);
    mlp_load_head(S, heads, head);
    uint32_t phase = 0;
    bool ok = true;
    // the same number of rounds on every thread of a warpgroup (the MLP synchronises the
    // warpgroup)
    for (long long row0 = (long long)blockIdx.x * kMlpThreads; row0 < n && ok;
         row0 += (long long)gridDim.x * kMlpThreads) {
        const long long row = row0 + threadIdx.x;
        const float x0 = row < n ? in[2 * row] : 0.0f;
        const float x1 = row < n ? in[2 * row + 1] : 0.0f;
        const float y = mlp_eval_cta(S, pack_bf16(x0, x1), phase, ok);
        if (row < n) out[row] = ok ? y : __int_as_float(0x7fc00000);
    }
    mlp_teardown(S, phase);
    if (__syncthreads_or(ok ? 0 : 1) && threadIdx.x == 0) atomicAdd(timeouts, 1ull);
}
}  // namespace bia

int bia_learned_head_eval(bia_context *ctx, int head, int n, const float *in, float *out)
{
    if (!ctx || !in || !out || n < 1 || head < 0 || head >= kMlpHeads || !ctx->heads_loaded)
        return set_last_error(BIA_ERR_INVALID_ARGUMENT);
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess) e = ctx->stats.reserve(kNumStats * sizeof(unsigned long long));
    unsigned long long *timeouts = (unsigned long long *)ctx->stats.ptr + kStatTimeouts;
    if (e == cudaSuccess) e = cudaMemsetAsync(timeouts, 0, sizeof(unsigned long long), ctx->stream);
    if (e == cudaSuccess &&
        cudaFuncSetAttribute(bia_head_eval_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(1024 + sizeof(MlpSmem))) != cudaSuccess)
        e = cudaGetLastError();
    if (e != cudaSuccess) return set_last_error(cuda_status(e));
    int blocks = (n + kMlpThreads - 1) / kMlpThreads;
    if (blocks > 4096) blocks = 4096;
    bia_head_eval_kernel<<<blocks, kMlpThreads, 1024 + sizeof(MlpSmem), ctx->stream>>>(
        (const MlpImage *)ctx->heads.ptr, head, n, in, out, timeouts);
    e = cudaGetLastError();
    unsigned long long h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, timeouts, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = ctx->stream ? cudaStreamSynchronize(ctx->stream) : cudaDeviceSynchronize();
    if (e != cudaSuccess) return set_last_error(cuda_status(e));
    return set_last_error(h ? BIA_ERR_DEVICE_TIMEOUT : BIA_OK);
}

// ---------------------------------------------------------------------------------------
// Self-test of the bounded-wait path: one thread waits on an mbarrier that nothing
// arrives at, with the same bounded try_wait loop the tensor-core pipeline uses (a short
// limit here), and records that the wait gave up.  No fault, trap or endless loop.
namespace bia {
__global__ void bia_wait_selftest_kernel(int limit, int *gave_up)
{
    __shared__ alignas(8) uint64_t mbar;
    if (threadIdx.x != 0) return;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&mbar)) : "memory");
    const uint32_t a = smem_addr(&mbar);
    int done = 0;
    for (int it = 0; it < limit && !done; it++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(a), "r"(0u)
            : "memory");
        done = (int)ok;
    }
    *gave_up = done ? 0 : 1;
}
}  // namespace bia

int bia_selftest_wait_timeout(bia_context *ctx)
{
    if (!ctx) return set_last_error(BIA_ERR_INVALID_ARGUMENT);
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess) e = ctx->stats.reserve(kNumStats * sizeof(unsigned long long));
    int *flag = (int *)((unsigned long long *)ctx->stats.ptr + kStatTimeouts);
    if (e == cudaSuccess) e = cudaMemsetAsync(flag, 0, sizeof(int), ctx->stream);
    if (e != cudaSuccess) return set_last_error(cuda_status(e));
    bia_wait_selftest_kernel<<<1, 32, 0, ctx->stream>>>(1 << 14, flag);
    int h = 0;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = ctx->stream ? cudaStreamSynchronize(ctx->stream) : cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemsetAsync(ctx->stats.ptr, 0, kNumStats * sizeof(unsigned long long), ctx->stream);
    if (e == cudaSuccess) e = ctx->stream ? cudaStreamSynchronize(ctx->stream) : cudaDeviceSynchronize();
    if (e != cudaSuccess) return set_last_error(cuda_status(e));
    return set_last_error(h ? BIA_ERR_DEVICE_TIMEOUT : BIA_OK);
}
