// bia_tiles.cuh -- one 32 x 32 warp-block of pairs, shared by the single-system step
// (bia_step.cu) and the ensemble step (bia_ensemble.cu).
//
// Lane l keeps row particle 32*bi + l and column particle 32*bj + l in registers.  At
// rotation step k it solves the pair (row l, column (l + k) mod 32), the column state
// arriving by shuffle, and the column's half-displacement goes back by a second shuffle
// from lane (l - k) mod 32, so every lane works on a different pair and both sums stay in
// registers.  Off-diagonal blocks take 32 steps (1024 pairs); diagonal blocks 16 (k =
// 1..15 on all lanes, k = 16 on lanes 0..15: each of the 496 pairs once; orientation does
// not matter because the half-displacement is exactly antisymmetric under i <-> j).
#pragma once
#include <mutex>

#include "bia_internal.cuh"
#include "bia_pair.cuh"

namespace bia {

// Resident CTAs per SM each method's 8-warp kernel is compiled for (register budget
// 65536 / (256 threads * blocks)): ALG 3 (<= 85 registers, measured fastest on the
// mixed-class Coulomb workload), universal variables 2 and RKF45 2 (<= 128).
#ifndef BIA_ALG_MIN_BLOCKS
#define BIA_ALG_MIN_BLOCKS 3
#endif
#ifndef BIA_UV_MIN_BLOCKS
#define BIA_UV_MIN_BLOCKS 2  // 3 spills in the rotation loop: 9.4 ms vs 8.6 ms at n = 32768
#endif
// RKF45: the shared-memory column walk at two CTAs per SM (128 registers; 600 B of spills
// around the out-of-line pair integrator) measured 184 ms per Coulomb step at n = 32768
// against 245 ms for the shuffle walk at one CTA per SM (222 registers) and 194 ms for the
// shuffle walk at two; bitwise the same sums.
#ifndef BIA_RKF_MIN_BLOCKS
#define BIA_RKF_MIN_BLOCKS 2
#endif
#ifndef BIA_RKF_SMEM
#define BIA_RKF_SMEM 1  // RKF walks with the column slice in shared memory
#endif
template <int M> struct TileOccupancy { static constexpr int kMinBlocks = 1; };
template <> struct TileOccupancy<kMethodRkf> { static constexpr int kMinBlocks = BIA_RKF_MIN_BLOCKS; };
template <> struct TileOccupancy<kMethodAlg> { static constexpr int kMinBlocks = BIA_ALG_MIN_BLOCKS; };
template <> struct TileOccupancy<kMethodUniversal> { static constexpr int kMinBlocks = BIA_UV_MIN_BLOCKS; };

__device__ __forceinline__ void warp_block_coords(long long t, int &bi, int &bj)
{
    // t = bj*(bj+1)/2 + bi with 0 <= bi <= bj
    long long c = (long long)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while (c * (c + 1) / 2 > t) c--;
    while ((c + 1) * (c + 2) / 2 <= t) c++;
    bj = (int)c;
    bi = (int)(t - c * (c + 1) / 2);
}

__device__ __forceinline__ void load_particle(const double *x, const double *y, const double *z,
                                              const double *u, const double *v, const double *w,
                                              const double *q, int n, int p, double s[7])
{
    if (p < n) {
        s[0] = x[p]; s[1] = y[p]; s[2] = z[p];
        s[3] = u[p]; s[4] = v[p]; s[5] = w[p];
        s[6] = q ? q[p] : 1.0;
    } else {
#pragma unroll
        for (int k = 0; k < 7; k++) s[k] = 0.0;
    }
}

__device__ __forceinline__ void flush_counters(const PairCounters &c, unsigned long long *stats, int lane)
{
    const unsigned full = 0xffffffffu;
    int vals[kNumStats] = {c.cls[0], c.cls[1], c.cls[2], c.cls[3], c.cls[4], c.cls[5],
                           c.it_hyp, c.it_ell, c.it_par, c.it_uv, c.rkf_steps,
                           c.nonconverged, c.bracket_exits, c.fallbacks, c.nonfinite,
                           c.learned, c.learned_fallbacks, c.learned_coarse, c.timeouts, c.learned_fp32};
#pragma unroll
    for (int k = 0; k < kNumStats; k++) {
        int s = __reduce_add_sync(full, vals[k]);
        if (lane == 0 && s != 0) atomicAdd(&stats[k], (unsigned long long)s);
    }
}

// Class-compacted ALG warp-block.  A warp that walks the 32 rotation steps together runs
// the hyperbola, ellipse and universal-variable code at nearly every step, because almost
// every step has lanes of each class.  Here each lane first classifies its own pairs (one
// bit per rotation offset k in a mask per class), then the warp runs the hyperbola
// pairs, the ellipse pairs and the rare classes as three loops, each lane taking its next
// pair of that class: every loop turn is one class on all busy lanes, and the number of
// turns is the largest per-lane count of that class instead of 32.  Column states and
// column sums live in this warp's slice of shared memory; lanes that hit the same column
// in one turn add their h in lane order (__match_any_sync groups), so the column sums
// have a fixed order for given inputs and the step stays bitwise reproducible.
#ifndef BIA_ALG_COMPACT
#define BIA_ALG_COMPACT 1
#endif
constexpr int kTileWarps = 8;              // warps per CTA of every kernel using warp-blocks
constexpr int kTileSmemDoubles = 13 * 32;  // per warp: column state [7][32], sums [6][32]

template <int C>
__device__ __forceinline__ void compact_class_loop(unsigned m, const double si[7], const double *ws,
                                                   double *wacc, int lane, bool has_q, double eps_th,
                                                   const PairParams &P, double racc[6], PairCounters &cnt)
{
    const unsigned full = 0xffffffffu;
    const unsigned lt = (1u << lane) - 1u;
    for (;;) {
        const bool busy = (m != 0u);
        const unsigned bm = __ballot_sync(full, busy);
        if (bm == 0u) break;
        if (busy) {
            const int k = __ffs(m) - 1;
            m &= m - 1u;
            const int j = (lane + k) & 31;
            double sc[7];
#pragma unroll
            for (int c = 0; c < 7; c++) sc[c] = ws[c * 32 + j];
            const double r[3] = {si[0] - sc[0], si[1] - sc[1], si[2] - sc[2]};
            const double g[3] = {si[3] - sc[3], si[4] - sc[4], si[5] - sc[5]};
            const double eps_ij = has_q ? eps_th * si[6] * sc[6] : eps_th;
            double h[6];
            if (C == kClsUv) {
                alg_rare_pair(P, eps_ij, r, g, h, cnt, alg_classify(eps_ij, r, g));
            } else {
                alg_conic_pair<C>(P, eps_ij, r, g, h, cnt);
            }
#pragma unroll
            for (int c = 0; c < 6; c++) racc[c] += h[c];
            const unsigned grp = __match_any_sync(bm, j);
            const int rank = __popc(grp & lt);
            const int turns = (int)__reduce_max_sync(bm, (unsigned)__popc(grp));
            for (int t = 0; t < turns; t++) {
                if (rank == t) {
#pragma unroll
                    for (int c = 0; c < 6; c++) wacc[c * 32 + j] += h[c];
                }
                __syncwarp(bm);
            }
        }
    }
}

// Balanced class loop of the phase-locked kernels.  The class's pairs of the warp-block are
// enumerated round by round: round r holds the r-th pair (in bit order) of every lane that
// has more than r of them, lanes in order.  Turn t takes entries 32 t .. 32 t + 31 of that
// enumeration, one per lane.  Full rounds are exactly the compact loop's turns (lane l solves
// its own pair); the tail rounds, in which only some lanes still have pairs, are packed
// together, so the loop takes ceil(pairs / 32) turns instead of the largest per-lane count
// (on the mixed-class Coulomb cube the compact loop's turns cost about 1.5x the balanced
// ones).  The solving lane is no longer the row's lane, so the row states rs and the row
// sums racs live in the warp's shared slice, and lanes that hit the same row or the same
// column in one turn add in lane order.  Every row then takes its pairs in rank order and
// every column in (round, lane) order: the compact loop's orders, so the sums are bitwise the
// compact loop's.
template <int C>
__device__ __forceinline__ void balanced_class_loop(unsigned m, const double *rs, double *racs, const double *ws,
                                                    double *wacc, int lane, bool has_q, double eps_th,
                                                    const PairParams &P, PairCounters &cnt)
{
    const unsigned full = 0xffffffffu;
    const unsigned lt = (1u << lane) - 1u;
    const int total = (int)__reduce_add_sync(full, (unsigned)__popc(m));
    const int most = (int)__reduce_max_sync(full, (unsigned)__popc(m));
    // packing saves turns only when the busiest lane has more than ceil(total / 32) pairs;
    // otherwise (every round full, as on an all-hyperbolic system) each lane solves its own
    // pairs in order and adds its own row directly: the same schedule and sums.  (The
    // per-lane loop with rows in registers as a second copy of the solver here spilled more
    // and was slower on the mixed classes.)
    const bool packed = most * 32 > total + 31;  // warp-uniform
    const int nturns = packed ? (total + 31) / 32 : most;
    int rbase = 0;                          // enumeration index of the current round's first pair
    unsigned cur = m;                       // this lane's pairs not in a finished round
    unsigned rm = __ballot_sync(full, cur != 0u);  // lanes of the current round
    for (int turn = 0; turn < nturns; turn++) {
        int o = -1, k = 0;
        if (!packed) {
            if (cur) {
                o = lane;
                k = __ffs(cur) - 1;
                cur &= cur - 1u;
            }
        } else {
            const int base = turn * 32;
            const int q = base + lane;
            while (rm != 0u) {  // the rounds this turn covers (warp-uniform)
                const int nr = __popc(rm);
                const int idx = q - rbase;
                const bool here = idx >= 0 && idx < nr;
                const int src = here ? (int)__fns(rm, 0, idx + 1) : 0;
                const int kk = __shfl_sync(full, __ffs(cur) - 1, src);  // the owner's pair of this round
                if (here) {
                    o = src;
                    k = kk;
                }
                if (rbase + nr > base + 32) break;  // the round goes on in the next turn
                rbase += nr;
                if ((rm >> lane) & 1u) cur &= cur - 1u;
                rm = __ballot_sync(full, cur != 0u);
            }
        }
        const bool busy = o >= 0;
        const unsigned bm = __ballot_sync(full, busy);
        if (busy) {
            const int j = (o + k) & 31;
            double si[7], sc[7];
#pragma unroll
            for (int c = 0; c < 7; c++) {
                si[c] = rs[c * 32 + o];
                sc[c] = ws[c * 32 + j];
            }
            const double r[3] = {si[0] - sc[0], si[1] - sc[1], si[2] - sc[2]};
            const double g[3] = {si[3] - sc[3], si[4] - sc[4], si[5] - sc[5]};
            const double eps_ij = has_q ? eps_th * si[6] * sc[6] : eps_th;
            double h[6];
            if (C == kClsUv) {
                alg_rare_pair(P, eps_ij, r, g, h, cnt, alg_classify(eps_ij, r, g));
            } else {
                alg_conic_pair<C>(P, eps_ij, r, g, h, cnt);
            }
            if (!packed) {  // the lane's own row
#pragma unroll
                for (int c = 0; c < 6; c++) racs[c * 32 + o] += h[c];
            } else {
                const unsigned grp = __match_any_sync(bm, o);
                const int rank = __popc(grp & lt);
                const int turns = (int)__reduce_max_sync(bm, (unsigned)__popc(grp));
                for (int t = 0; t < turns; t++) {
                    if (rank == t) {
#pragma unroll
                        for (int c = 0; c < 6; c++) racs[c * 32 + o] += h[c];
                    }
                    __syncwarp(bm);
                }
            }
            {
                const unsigned grp = __match_any_sync(bm, j);
                const int rank = __popc(grp & lt);
                const int turns = (int)__reduce_max_sync(bm, (unsigned)__popc(grp));
                for (int t = 0; t < turns; t++) {
                    if (rank == t) {
#pragma unroll
                        for (int c = 0; c < 6; c++) wacc[c * 32 + j] += h[c];
                    }
                    __syncwarp(bm);
                }
            }
        }
    }
}

// Loads of a compacted warp-block and classification of its pairs: the column states go
// to the warp's shared slice ws (sums zeroed), si receives the row particle, and the class
// masks (bit k: the pair with column (lane + k) mod 32) are returned in mh, me, mr.
// live == false leaves every mask empty (a warp without a block that still joins the
// barriers of a phase-locked CTA).
__device__ __forceinline__ void compact_prepare(const double *x, const double *y, const double *z,
                                                const double *u, const double *v, const double *w,
                                                const double *q, int n, double eps_th, int bi, int bj,
                                                int lane, bool live, double *ws, double si[7],
                                                unsigned &mh, unsigned &me, unsigned &mr)
{
    double *wacc = ws + 7 * 32;
    const int i = bi * 32 + lane;
    double sj[7];
    load_particle(x, y, z, u, v, w, q, n, i, si);
    load_particle(x, y, z, u, v, w, q, n, bj * 32 + lane, sj);
#pragma unroll
    for (int c = 0; c < 7; c++) ws[c * 32 + lane] = sj[c];
#pragma unroll
    for (int c = 0; c < 6; c++) wacc[c * 32 + lane] = 0.0;
    __syncwarp();
    mh = me = mr = 0u;
    if (!live) return;
    const bool diag = (bi == bj);
    const int k0 = diag ? 1 : 0;
    const int k1 = diag ? 16 : 31;
    for (int k = k0; k <= k1; k++) {
        const int src = (lane + k) & 31;
        const int j = bj * 32 + src;
        if ((!diag || k < 16 || lane < 16) && i < n && j < n) {
            const double r[3] = {si[0] - ws[0 * 32 + src], si[1] - ws[1 * 32 + src], si[2] - ws[2 * 32 + src]};
            const double g[3] = {si[3] - ws[3 * 32 + src], si[4] - ws[4 * 32 + src], si[5] - ws[5 * 32 + src]};
            const double eps_ij = q ? eps_th * si[6] * ws[6 * 32 + src] : eps_th;
            const int c = alg_classify(eps_ij, r, g);
            const unsigned bit = 1u << k;
            if (c == kClsHyp) mh |= bit;
            else if (c == kClsEll) me |= bit;
            else mr |= bit;
        }
    }
}

__device__ __forceinline__ void warp_block_solve_compact(const double *x, const double *y, const double *z,
                                                         const double *u, const double *v, const double *w,
                                                         const double *q, int n, double eps_th,
                                                         const PairParams &P, int bi, int bj, int lane,
                                                         double racc[6], double cacc[6], PairCounters &cnt)
{
    __shared__ double s_tile[kTileWarps][kTileSmemDoubles];
    double *ws = s_tile[(threadIdx.x >> 5) % kTileWarps];
    double si[7];
    unsigned mh, me, mr;
    compact_prepare(x, y, z, u, v, w, q, n, eps_th, bi, bj, lane, true, ws, si, mh, me, mr);
#pragma unroll
    for (int c = 0; c < 6; c++) racc[c] = 0.0;
    counters_zero(cnt);
    compact_class_loop<kClsHyp>(mh, si, ws, ws + 7 * 32, lane, q != nullptr, eps_th, P, racc, cnt);
    compact_class_loop<kClsEll>(me, si, ws, ws + 7 * 32, lane, q != nullptr, eps_th, P, racc, cnt);
    compact_class_loop<kClsUv>(mr, si, ws, ws + 7 * 32, lane, q != nullptr, eps_th, P, racc, cnt);
    __syncwarp();
#pragma unroll
    for (int c = 0; c < 6; c++) cacc[c] = ws[(7 + c) * 32 + lane];
    __syncwarp();  // the slice is reused by this warp's next block
}

// Phase-locked CTAs (32 warps, one warp-block each).  After the classification
// every warp of the CTA runs the hyperbola loop, then (barrier) the ellipse loop, then
// (barrier) the rare classes, so the SM fetches one solver's instructions at a time: the
// mixed-class ALG step is bound by instruction fetch when the warps of one SM sit in
// different solvers (measured on B200, Coulomb N = 32768: 218 ms per step with 8-warp
// CTAs, 122 ms phase-locked with 32 warps).  kBalanced: the balanced class loops
// (balanced_class_loop; mixed classes), else the per-lane loops of warp_block_solve_compact
// with the row in registers (all-hyperbolic systems); both have the per-block arithmetic and
// order of warp_block_solve_compact, so the results are bitwise equal.  Every thread of the
// CTA must call it (warps without a block pass live = false); ws is the warp's slice of
// phase_slice_doubles<kBalanced>() doubles: column states [7][32], column sums [6][32], and
// for the balanced loops row states [7][32] and row sums [6][32].
#ifndef BIA_PHASE_WARPS
#define BIA_PHASE_WARPS 32  // 0: never use the phase-locked kernels
#endif
constexpr int kPhaseSliceDoubles = kTileSmemDoubles + 13 * 32;
// a phase-locked warp's slice: the balanced loops add the rows to the column slice; the
// per-lane loops keep the rows in registers and leave the rest of the SM's on-chip memory to
// L1, which caches their register spills
template <bool kBalanced>
__host__ __device__ constexpr int phase_slice_doubles() { return kBalanced ? kPhaseSliceDoubles : kTileSmemDoubles; }

template <bool kBalanced = true>
__device__ __forceinline__ void phase_block_solve(const double *x, const double *y, const double *z,
                                                  const double *u, const double *v, const double *w,
                                                  const double *q, int n, double eps_th, const PairParams &P,
                                                  int bi, int bj, int lane, bool live, double *ws,
                                                  double racc[6], double cacc[6], PairCounters &cnt)
{
    unsigned mh, me, mr;
    counters_zero(cnt);
    const bool hq = q != nullptr;
    if (!kBalanced) {  // the per-lane class loops, row state and row sums in registers
        double si[7];
#pragma unroll
        for (int c = 0; c < 6; c++) racc[c] = 0.0;
        compact_prepare(x, y, z, u, v, w, q, n, eps_th, bi, bj, lane, live, ws, si, mh, me, mr);
        __syncthreads();
        compact_class_loop<kClsHyp>(mh, si, ws, ws + 7 * 32, lane, hq, eps_th, P, racc, cnt);
        __syncthreads();
        compact_class_loop<kClsEll>(me, si, ws, ws + 7 * 32, lane, hq, eps_th, P, racc, cnt);
        __syncthreads();
        compact_class_loop<kClsUv>(mr, si, ws, ws + 7 * 32, lane, hq, eps_th, P, racc, cnt);
        __syncwarp();
#pragma unroll
        for (int c = 0; c < 6; c++) cacc[c] = ws[(7 + c) * 32 + lane];
        return;
    }
    double *rs = ws + kTileSmemDoubles;
    double *racs = rs + 7 * 32;
    {
        double si[7];
        compact_prepare(x, y, z, u, v, w, q, n, eps_th, bi, bj, lane, live, ws, si, mh, me, mr);
#pragma unroll
        for (int c = 0; c < 7; c++) rs[c * 32 + lane] = si[c];
#pragma unroll
        for (int c = 0; c < 6; c++) racs[c * 32 + lane] = 0.0;
    }
    __syncthreads();
    balanced_class_loop<kClsHyp>(mh, rs, racs, ws, ws + 7 * 32, lane, hq, eps_th, P, cnt);
    __syncthreads();
    balanced_class_loop<kClsEll>(me, rs, racs, ws, ws + 7 * 32, lane, hq, eps_th, P, cnt);
    __syncthreads();
    balanced_class_loop<kClsUv>(mr, rs, racs, ws, ws + 7 * 32, lane, hq, eps_th, P, cnt);
    __syncwarp();
#pragma unroll
    for (int c = 0; c < 6; c++) {
        racc[c] = racs[c * 32 + lane];
        cacc[c] = ws[(7 + c) * 32 + lane];
    }
}

// Universal-variable warp-block: lanes walk the rotation offsets as in warp_block_solve,
// with the column states and the column sums in the warp's shared slice instead of
// registers and shuffles.  Lane l adds its pair at offset k into column slot (l + k) mod 32,
// a different slot on every lane, so the slots take their pairs in ascending k, the order
// of the shuffle walk: the sums are bitwise the same.  Measured at n = 32768: 6.48 ms
// against 6.79 ms for the shuffle walk (100 instead of 118 registers, no shuffles).
// The non-finite pairs of a warp-block whose sums came out non-finite (rare): this lane's
// pairs solved again, counted one by one.  Out of line, so that the walk carries no copy.
template <int M>
static __device__ __noinline__ int uv_block_recount(const PairParams &P, const double *si, const double *ws,
                                                    bool hq, double eps_th, int i, int n, int bj, int lane)
{
    const bool diag = (i / 32 == bj);
    const int k0 = diag ? 1 : 0, k1 = diag ? 16 : 31;
    int bad = 0;
    for (int k = k0; k <= k1; k++) {
        const int src = (lane + k) & 31;
        if ((!diag || k < 16 || lane < 16) && i < n && bj * 32 + src < n) {
            const double r[3] = {si[0] - ws[0 * 32 + src], si[1] - ws[1 * 32 + src], si[2] - ws[2 * 32 + src]};
            const double g[3] = {si[3] - ws[3 * 32 + src], si[4] - ws[4 * 32 + src], si[5] - ws[5 * 32 + src]};
            const double eps_ij = hq ? eps_th * si[6] * ws[6 * 32 + src] : eps_th;
            double h[6];
            PairCounters scratch;
            counters_zero(scratch);
            pair_halfdisp<M, true>(P, eps_ij, r, g, h, scratch);
            bad += scratch.nonfinite;
        }
    }
    return bad;
}

template <int M = kMethodUniversal>
__device__ __forceinline__ void warp_block_solve_uv(const double *x, const double *y, const double *z,
                                                    const double *u, const double *v, const double *w,
                                                    const double *q, int n, double eps_th, const PairParams &P,
                                                    int bi, int bj, int lane, double racc[6], double cacc[6],
                                                    PairCounters &cnt)
{
    // universal variables: the non-finite pairs counted from the block's sums (one test per
    // block instead of six per pair); RKF45 pairs are costly enough to keep the per-pair count
    constexpr bool kBlockCheck = (M == kMethodUniversal);
    __shared__ double s_uv[kTileWarps][kTileSmemDoubles];
    double *ws = s_uv[(threadIdx.x >> 5) % kTileWarps];
    double *wacc = ws + 7 * 32;
    const int i = bi * 32 + lane;
    double si[7];
    {
        double sj[7];
        load_particle(x, y, z, u, v, w, q, n, i, si);
        load_particle(x, y, z, u, v, w, q, n, bj * 32 + lane, sj);
#pragma unroll
        for (int c = 0; c < 7; c++) ws[c * 32 + lane] = sj[c];
#pragma unroll
        for (int c = 0; c < 6; c++) wacc[c * 32 + lane] = 0.0;
    }
    __syncwarp();
#pragma unroll
    for (int c = 0; c < 6; c++) racc[c] = 0.0;
    counters_zero(cnt);
    const bool diag = (bi == bj);
    const int k0 = diag ? 1 : 0;
    const int k1 = diag ? 16 : 31;
    for (int k = k0; k <= k1; k++) {
        const int src = (lane + k) & 31;
        const bool active = (!diag || k < 16 || lane < 16) && i < n && bj * 32 + src < n;
        double h[6] = {0, 0, 0, 0, 0, 0};
        if (active) {
            const double r[3] = {si[0] - ws[0 * 32 + src], si[1] - ws[1 * 32 + src], si[2] - ws[2 * 32 + src]};
            const double g[3] = {si[3] - ws[3 * 32 + src], si[4] - ws[4 * 32 + src], si[5] - ws[5 * 32 + src]};
            const double eps_ij = q ? eps_th * si[6] * ws[6 * 32 + src] : eps_th;
            pair_halfdisp<M, !kBlockCheck>(P, eps_ij, r, g, h, cnt);
        }
#pragma unroll
        for (int c = 0; c < 6; c++) {
            racc[c] += h[c];
            wacc[c * 32 + src] += h[c];
        }
        __syncwarp();  // slot src is the next offset's slot of lane - 1
    }
#pragma unroll
    for (int c = 0; c < 6; c++) cacc[c] = wacc[c * 32 + lane];
    if (kBlockCheck && __any_sync(0xffffffffu, !sums_finite(racc, cacc))) {
        double sic[7];  // a copy: passing si itself would keep it in memory for the whole walk
#pragma unroll
        for (int c = 0; c < 7; c++) sic[c] = si[c];
        cnt.nonfinite += uv_block_recount<M>(P, sic, ws, q != nullptr, eps_th, i, n, bj, lane);
    }
    __syncwarp();  // the slice is reused by this warp's next block
}

// The phase-locked kernels' counters: a warp-block's counters summed over the warp into the
// warp's slot wtot[kNumStats] in shared memory (lane 0); after a CTA barrier one warp adds
// the CTA's slots up and flushes them with one set of atomics (flush_slots).
__device__ __forceinline__ void counters_to_slot(const PairCounters &c, unsigned long long *wtot, int lane)
{
    const unsigned full = 0xffffffffu;
    int vals[kNumStats] = {c.cls[0], c.cls[1], c.cls[2], c.cls[3], c.cls[4], c.cls[5],
                           c.it_hyp, c.it_ell, c.it_par, c.it_uv, c.rkf_steps,
                           c.nonconverged, c.bracket_exits, c.fallbacks, c.nonfinite,
                           c.learned, c.learned_fallbacks, c.learned_coarse, c.timeouts, c.learned_fp32};
#pragma unroll
    for (int k = 0; k < kNumStats; k++) {
        const int s = __reduce_add_sync(full, vals[k]);
        if (lane == 0 && s != 0) wtot[k] += (unsigned long long)s;
    }
}
__device__ __forceinline__ void flush_slots(const unsigned long long *slots, int nwarps, unsigned long long *stats,
                                            int lane)
{
    if (lane >= kNumStats) return;
    unsigned long long sum = 0ull;
    for (int w = 0; w < nwarps; w++) sum += slots[w * kNumStats + lane];
    if (sum != 0ull) atomicAdd(&stats[lane], sum);
}

// Running sums of a warp's counters over the blocks it solves (persistent kernels flush
// them every kFlushBlocks blocks instead of once per block: one set of atomics per warp).
constexpr int kFlushBlocks = 64;
__device__ __forceinline__ void counters_add(PairCounters &a, const PairCounters &b)
{
#pragma unroll
    for (int k = 0; k < 6; k++) a.cls[k] += b.cls[k];
    a.it_hyp += b.it_hyp; a.it_ell += b.it_ell; a.it_par += b.it_par; a.it_uv += b.it_uv;
    a.rkf_steps += b.rkf_steps; a.nonconverged += b.nonconverged; a.bracket_exits += b.bracket_exits;
    a.fallbacks += b.fallbacks; a.nonfinite += b.nonfinite; a.learned += b.learned;
    a.learned_fallbacks += b.learned_fallbacks; a.learned_coarse += b.learned_coarse;
    a.timeouts += b.timeouts; a.learned_fp32 += b.learned_fp32;
}

// Pairs of warp-block (bi, bj) of the system whose particles are x[0..n) etc.: row sums
// racc (particle 32 bi + lane) and column sums cacc (particle 32 bj + lane) of the pair
// half-displacements h (row receives +h, column -h: the caller writes -cacc).
template <int M>
__device__ __forceinline__ void warp_block_solve(const double *x, const double *y, const double *z,
                                                 const double *u, const double *v, const double *w,
                                                 const double *q, int n, double eps_th, const PairParams &P,
                                                 int bi, int bj, int lane, double racc[6], double cacc[6],
                                                 PairCounters &cnt)
{
    if (M == kMethodAlg && BIA_ALG_COMPACT) {
        warp_block_solve_compact(x, y, z, u, v, w, q, n, eps_th, P, bi, bj, lane, racc, cacc, cnt);
        return;
    }
    if (M == kMethodUniversal || (M == kMethodRkf && BIA_RKF_SMEM)) {
        warp_block_solve_uv<M>(x, y, z, u, v, w, q, n, eps_th, P, bi, bj, lane, racc, cacc, cnt);
        return;
    }
    const unsigned full = 0xffffffffu;
    const int i = bi * 32 + lane;
    double si[7], sj[7];
    load_particle(x, y, z, u, v, w, q, n, i, si);
    load_particle(x, y, z, u, v, w, q, n, bj * 32 + lane, sj);
#pragma unroll
    for (int c = 0; c < 6; c++) racc[c] = cacc[c] = 0.0;
    counters_zero(cnt);
    const bool diag = (bi == bj);
    const int k0 = diag ? 1 : 0;
    const int k1 = diag ? 16 : 31;
    for (int k = k0; k <= k1; k++) {
        const int src = (lane + k) & 31;
        double sc[7];
#pragma unroll
        for (int c = 0; c < 7; c++) sc[c] = __shfl_sync(full, sj[c], src);
        const int j = bj * 32 + src;
        const bool active = (!diag || k < 16 || lane < 16) && i < n && j < n;
        double h[6] = {0, 0, 0, 0, 0, 0};
        if (active) {
            const double r[3] = {si[0] - sc[0], si[1] - sc[1], si[2] - sc[2]};
            const double g[3] = {si[3] - sc[3], si[4] - sc[4], si[5] - sc[5]};
            const double eps_ij = q ? eps_th * si[6] * sc[6] : eps_th;
            pair_halfdisp<M>(P, eps_ij, r, g, h, cnt);
        }
        const int back = (lane - k) & 31;
#pragma unroll
        for (int c = 0; c < 6; c++) {
            racc[c] += h[c];
            cacc[c] += __shfl_sync(full, h[c], back);
        }
    }
}

// Deterministic partial layout part[m][c][p] (plane = padded particle count): row sums
// of block (bi, bj) at m = bj, column sums at m = bi, the diagonal block's combined sums
// at m = bi; each (m, p) slot is written once per step.
__device__ __forceinline__ void write_partials(double *part, size_t plane, int bi, int bj, int lane,
                                               const double racc[6], const double cacc[6])
{
    const int i = bi * 32 + lane;
    const int j = bj * 32 + lane;
    if (bi == bj) {
        double *dst = part + (size_t)bi * 6 * plane;
#pragma unroll
        for (int c = 0; c < 6; c++) dst[c * plane + i] = racc[c] - cacc[c];
    } else {
        double *drow = part + (size_t)bj * 6 * plane;
        double *dcol = part + (size_t)bi * 6 * plane;
#pragma unroll
        for (int c = 0; c < 6; c++) {
            drow[c * plane + i] = racc[c];
            dcol[c * plane + j] = -cacc[c];
        }
    }
}

// The same slots as write_partials, added onto instead of written (a second kernel's share
// of the same warp-block).  row_hit / col_hit false: this lane's row / column sum is zero
// and its slot is left alone (adding zero would not change it).
__device__ __forceinline__ void add_partials(double *part, size_t plane, int bi, int bj, int lane,
                                             const double racc[6], const double cacc[6], bool row_hit = true,
                                             bool col_hit = true)
{
    const int i = bi * 32 + lane;
    const int j = bj * 32 + lane;
    if (bi == bj) {
        if (!row_hit && !col_hit) return;
        double *dst = part + (size_t)bi * 6 * plane;
#pragma unroll
        for (int c = 0; c < 6; c++) dst[c * plane + i] += racc[c] - cacc[c];
    } else {
        double *drow = part + (size_t)bj * 6 * plane;
        double *dcol = part + (size_t)bi * 6 * plane;
        if (row_hit) {
#pragma unroll
            for (int c = 0; c < 6; c++) drow[c * plane + i] += racc[c];
        }
        if (col_hit) {
#pragma unroll
            for (int c = 0; c < 6; c++) dcol[c * plane + j] -= cacc[c];
        }
    }
}

}  // namespace bia
