// bia_learned_block.cuh -- one warp-block of the learned mixed-precision form
// (BIA_METHOD_LEARNED) for a CTA of kLearnedWarps warps, shared by the single-system step
// (bia_step.cu) and the ensemble (bia_ensemble.cu).
#pragma once
#include "bia_learned.cuh"
#include "bia_pair.cuh"
#include "bia_tiles.cuh"
#include "mlp_tc.cuh"

namespace bia {

// The one-kernel learned form: a CTA of 8 warps, one warp-block each, two CTAs per SM, in
// three phases (the split step below spreads the same work over three kernels).
//  1. Each lane classifies its pairs (hyperbolic head, elliptic head, plain) and writes the
//     head input of each learned pair (packed BF16) into the pair's own row slot
//     (warp, lane, k) in shared memory.
//  2. A CTA scan of the per-lane counts numbers the learned pairs of each head in thread
//     and bit order; the CTA evaluates each head on its pairs in full 256-row blocks on
//     the tensor cores (mlp_tc.cuh), each thread finding its row's slot from the scan, and
//     writes each row's output over its input.
//  3. Each warp finishes its learned pairs from the stored guesses (FP32 correction, FP64
//     Halley step, composition; the plain solver where the FP64 step does not settle),
//     then its plain pairs with the universal-variable solver, with no CTA barrier.
// Column sums in the warp's shared slice, added in lane order per turn (deterministic).
constexpr int kLearnedWarps = kMlpThreads / 32;
constexpr int kLearnedMaxRows = kLearnedWarps * 1024;
constexpr size_t kLearnedTileBytes = (size_t)kLearnedWarps * kTileSmemDoubles * sizeof(double);
constexpr size_t kLearnedSmemBytes = 1024 + sizeof(MlpSmem) + kLearnedTileBytes + kLearnedMaxRows * sizeof(uint32_t);

__device__ __forceinline__ void add_column(double *wacc, int j, const double h[6], unsigned bm, int lane)
{
    const unsigned grp = __match_any_sync(bm, j);
    const int rank = __popc(grp & ((1u << lane) - 1u));
    const int turns = (int)__reduce_max_sync(bm, (unsigned)__popc(grp));
    for (int t = 0; t < turns; t++) {
        if (rank == t) {
#pragma unroll
            for (int c = 0; c < 6; c++) wacc[c * 32 + j] += h[c];
        }
        __syncwarp(bm);
    }
}

// exclusive CTA-wide prefix sums of (a, b) over threads in thread order; totals returned
__device__ __forceinline__ void cta_scan2(MlpSmem &S, int a, int b, int &oa, int &ob, int &ta, int &tb)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int ia = a, ib = b;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int xa = __shfl_up_sync(0xffffffffu, ia, d);
        const int xb = __shfl_up_sync(0xffffffffu, ib, d);
        if (lane >= d) { ia += xa; ib += xb; }
    }
    if (lane == 31) { S.wsum[0][warp] = ia; S.wsum[1][warp] = ib; }
    __syncthreads();
    int ba = 0, bb = 0;
    ta = tb = 0;
    for (int w = 0; w < kLearnedWarps; w++) {
        if (w < warp) { ba += S.wsum[0][w]; bb += S.wsum[1][w]; }
        ta += S.wsum[0][w];
        tb += S.wsum[1][w];
    }
    oa = ba + ia - a;
    ob = bb + ib - b;
}


// The split learned step in three kernels, shared by the single-system step and the ensemble:
//  rest    every pair gets the universal-variable prepare and the fifth-order start; a pair
//          whose start is exact is composed right there.  A pair whose start is not exact and
//          that lies inside a head's domain (learned_filter, then learned_prepare) is deferred:
//          its head input goes to the warp's row slot (lane, k) in shared memory.  The other
//          non-exact pairs run the safeguarded Newton iteration.  After the walk the warp
//          allocates rows for its deferred pairs in the global row buffer of each head (one
//          atomic per head and warp-block), writes their inputs there (per lane in ascending
//          k, lanes in order) and lists the warp-block with its row bases and pair masks.
//  head    the rows of each head in full 256-row tiles on the tensor cores (mlp_tc.cuh), each
//          row's guess written over its input.
//  finish  the deferred pairs from their guesses (FP32 correction, FP64 Halley step,
//          composition; the plain solver where the FP64 step does not settle), their sums
//          added onto the rest kernel's partials: a listed warp-block with many pairs (or on
//          the diagonal) by one warp, the others batched 32 pairs at a time from the pair
//          descriptors the rest kernel wrote for them (finish_batches).
// A pair's row holds only that pair's input and guess, and every partial slot is written by
// the rest kernel and added to by at most one listed warp-block, so neither the order of the
// rows nor that of the list changes the results.  The rows of a head are capped (rows_cap);
// a warp-block whose rows do not fit is listed without rows and the finish kernel solves its
// pairs with the plain solver: only then do the results depend on the order in which
// warp-blocks took rows.
struct LearnedRows {
    uint32_t *rows[kMlpHeads];   // per head (kHeadEll, kHeadHyp): packed BF16 inputs, then FP32 guesses
    unsigned long long *counts;  // [kMlpHeads] rows taken this step (may run past rows_cap)
    unsigned int *nlist;         // listed warp-blocks
    uint4 *entries;              // per listed warp-block: (item, row base ell, row base hyp, pairs)
    uint32_t *masks;             // per listed warp-block: [kMlpHeads][32] lane masks
    uint2 *pairs;                // per listed warp-block with at most kBatchPairs pairs: [kBatchPairs]
                                 // (row or kNoRows, lane | k << 5 | head << 10) in solve order
    unsigned int rows_cap;
};
constexpr unsigned int kNoRows = 0xffffffffu;
// A listed warp-block with at most this many deferred pairs (and off the diagonal) is
// finished in a batch with other such blocks, one pair per lane.
constexpr int kBatchPairs = 32;
// list bytes per warp-block: the entry, the masks, the pair descriptors
constexpr size_t kListBytesPerBlock = 16 + 64 * sizeof(uint32_t) + kBatchPairs * sizeof(uint2);
// the buffer's header: the two row counts (u64) and the list length (u32), 32 bytes
constexpr size_t kSplitHeader = 32;

// Shared memory of a rest-kernel warp: its column slice (kTileSmemDoubles doubles) and 1024
// row slots (slot lane * 32 + k: the packed head input of the lane's pair at offset k).
constexpr size_t kRestWarpBytes = kTileSmemDoubles * sizeof(double) + 1024 * sizeof(uint32_t);
constexpr size_t kRestSmemBytes = kTileWarps * kRestWarpBytes;

// One pair of the rest kernel's walk: the universal-variable prepare and series; a non-exact
// pair inside a head's domain is deferred (returns its head, L holds its head input), any
// other is solved here (returns kLearnedPlain, h and its Newton iterations in it).
__device__ __forceinline__ int rest_pair(double eps_ij, double dt, const double r[3], const double g[3],
                                         double h[6], LearnedPair &L, int &it)
{
    it = 0;
    const UvPair p = uv_prepare(eps_ij, r, g);
    if (dt == 0.0) return kLearnedPlain;  // h stays zero
    const UvSeries sq = uv_series(p, dt);
    if (!sq.exact && learned_filter(p, dt)) {
        learned_prepare(eps_ij, dt, r, g, L);
        if (L.kind != kLearnedPlain) return L.kind;
    }
    if (sq.exact) {
        uv_compose_series(p, sq, dt, r, g, h);
    } else {
        double s = uv_series_start(sq);
        double ifp = 0.0;
        it = uv_iterate(p, dt, s, &ifp);
        uv_compose<true>(p, s, r, g, h, ifp);
    }
    return kLearnedPlain;
}

// The non-finite pairs solved in a rest-kernel warp-block whose sums came out non-finite
// (rare): this lane's pairs solved again, the plain ones counted one by one (the deferred
// ones are counted where they are finished).  Out of line, so that the walk carries no copy.
static __device__ __noinline__ int rest_block_recount(const double *si, const double *ws, bool hq, double eps_th,
                                                      double dt, int i, int n, int bj, int lane)
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
            double h[6] = {0, 0, 0, 0, 0, 0};
            LearnedPair L;
            int it;
            if (rest_pair(eps_ij, dt, r, g, h, L, it) == kLearnedPlain) {
                PairCounters scratch;
                counters_zero(scratch);
                count_nonfinite(h, scratch);
                bad += scratch.nonfinite;
            }
        }
    }
    return bad;
}

// The rest kernel's walk over warp-block (bi, bj) of the system x..w[0, n) (charges q,
// coupling eps_th), with the column states and sums in the warp's slice ws and the row slots
// wslots.  Returns the row sums racc, column sums cacc of the pairs solved here, and the
// lane's masks of deferred pairs per head (bit k: column (lane + k) mod 32).  The pairs
// solved here are counted as universal-variable pairs, degenerate ones included, as
// BIA_METHOD_UNIVERSAL counts them.
__device__ __forceinline__ void rest_block_solve(const double *x, const double *y, const double *z,
                                                 const double *u, const double *v, const double *w,
                                                 const double *q, int n, double eps_th, double dt, int bi, int bj,
                                                 int lane, double *ws, uint32_t *wslots, double racc[6],
                                                 double cacc[6], uint32_t mask[kMlpHeads], PairCounters &cnt)
{
    double *wacc = ws + 7 * 32;
    const int i = bi * 32 + lane;
    const bool diag = (bi == bj);
    mask[kHeadEll] = mask[kHeadHyp] = 0u;
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
    const int k0 = diag ? 1 : 0, k1 = diag ? 16 : 31;
    for (int k = k0; k <= k1; k++) {
        const int src = (lane + k) & 31;
        const bool active = (!diag || k < 16 || lane < 16) && i < n && bj * 32 + src < n;
        double h[6] = {0, 0, 0, 0, 0, 0};
        if (active) {
            const double r[3] = {si[0] - ws[0 * 32 + src], si[1] - ws[1 * 32 + src], si[2] - ws[2 * 32 + src]};
            const double g[3] = {si[3] - ws[3 * 32 + src], si[4] - ws[4 * 32 + src], si[5] - ws[5 * 32 + src]};
            const double eps_ij = q ? eps_th * si[6] * ws[6 * 32 + src] : eps_th;
            LearnedPair L;
            int it;
            const int kind = rest_pair(eps_ij, dt, r, g, h, L, it);
            if (kind != kLearnedPlain) {
                mask[kind == kLearnedHyp ? kHeadHyp : kHeadEll] |= 1u << k;
                wslots[lane * 32 + k] = pack_bf16(L.x0, L.x1);
            } else {
                cnt.it_uv += it;
                if (it > kUvItMax) cnt.nonconverged++;
                cnt.cls[kUniversal]++;
            }
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
    if (__any_sync(0xffffffffu, !sums_finite(racc, cacc))) {
        double sic[7];  // a copy: passing si itself would keep it in memory for the whole walk
#pragma unroll
        for (int c = 0; c < 7; c++) sic[c] = si[c];
        cnt.nonfinite += rest_block_recount(sic, ws, q != nullptr, eps_th, dt, i, n, bj, lane);
    }
    __syncwarp();  // the slice is reused by this warp's next block
}

// After rest_block_solve: rows for the warp-block's deferred pairs and its list entry (item:
// the warp-block's index for the finish kernel).  Every lane of the warp calls it.
__device__ __forceinline__ void rest_block_defer(const LearnedRows &R, unsigned int item,
                                                 const uint32_t mask[kMlpHeads], const uint32_t *wslots, int lane)
{
    const unsigned full = 0xffffffffu;
    unsigned int base[kMlpHeads], pre[kMlpHeads], tot[kMlpHeads];
#pragma unroll
    for (int hd = 0; hd < kMlpHeads; hd++) {
        // exclusive prefix of the lanes' counts
        const unsigned c = (unsigned)__popc(mask[hd]);
        unsigned inc = c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned o = __shfl_up_sync(full, inc, d);
            if (lane >= d) inc += o;
        }
        pre[hd] = inc - c;
        tot[hd] = __shfl_sync(full, inc, 31);
    }
    if (tot[kHeadEll] + tot[kHeadHyp] == 0u) return;  // warp-uniform
    bool fits = true;
#pragma unroll
    for (int hd = 0; hd < kMlpHeads; hd++) {
        unsigned long long b = 0ull;
        if (lane == 0 && tot[hd] != 0u) b = atomicAdd(&R.counts[hd], (unsigned long long)tot[hd]);
        b = __shfl_sync(full, b, 0);
        if (tot[hd] != 0u && b + tot[hd] > (unsigned long long)R.rows_cap) fits = false;
        base[hd] = (unsigned int)(b < R.rows_cap ? b : 0ull);
    }
    if (fits) {
#pragma unroll
        for (int hd = 0; hd < kMlpHeads; hd++) {
            uint32_t m = mask[hd];
            unsigned int row = base[hd] + pre[hd];
            while (m) {
                const int k = __ffs(m) - 1;
                m &= m - 1u;
                R.rows[hd][row++] = wslots[lane * 32 + k];
            }
        }
    }
    unsigned int e = 0u;
    if (lane == 0) e = atomicAdd(R.nlist, 1u);
    e = __shfl_sync(full, e, 0);
    const unsigned int npairs = tot[kHeadEll] + tot[kHeadHyp];
    if (lane == 0)
        R.entries[e] = make_uint4(item, fits ? base[kHeadEll] : kNoRows, fits ? base[kHeadHyp] : kNoRows, npairs);
    R.masks[(size_t)e * 64 + lane] = mask[kHeadEll];
    R.masks[(size_t)e * 64 + 32 + lane] = mask[kHeadHyp];
    if (npairs <= (unsigned)kBatchPairs) {
        // the pairs in the order the per-block finish solves them: round r holds the r-th pair
        // (in k order) of every lane with more than r, lanes in order
        const uint32_t both = mask[kHeadEll] | mask[kHeadHyp];
        uint32_t left = both;
        unsigned int at = 0u;
        for (;;) {
            const unsigned rm = __ballot_sync(full, left != 0u);
            if (rm == 0u) break;
            if (left) {
                const int k = __ffs(left) - 1;
                left &= left - 1u;
                const int hd = ((mask[kHeadHyp] >> k) & 1u) ? kHeadHyp : kHeadEll;
                const unsigned int row =
                    fits ? base[hd] + pre[hd] + (unsigned)__popc(mask[hd] & ((1u << k) - 1u)) : kNoRows;
                const unsigned int pos = at + (unsigned)__popc(rm & ((1u << lane) - 1u));
                R.pairs[(size_t)e * kBatchPairs + pos] = make_uint2(row, (unsigned)lane | ((unsigned)k << 5) |
                                                                              ((unsigned)hd << 10));
            }
            at += (unsigned)__popc(rm);
        }
    }
}

// The system a warp-block belongs to: particles x..w[0, n) (and charges q), coupling eps_th.
struct LearnedBlockIn {
    const double *x, *y, *z, *u, *v, *w, *q;
    int n;
    double eps_th, dt;
    const MlpImage *heads;
};

// Dynamic shared memory of a learned CTA: the MLP image, the warps' column tiles (the
// column particles of all warps, then their column sums: the first 4 KB of the sums hold
// the row numbering of phase 2), the row slots; base aligned to 1024 bytes.
struct LearnedSmem {
    MlpSmem *mlp;
    double *tiles;
    uint32_t *rows;
};
__device__ __forceinline__ LearnedSmem learned_smem(uint8_t *raw)
{
    uint8_t *base = (uint8_t *)(((uintptr_t)raw + 1023) & ~(uintptr_t)1023);
    LearnedSmem L;
    L.mlp = reinterpret_cast<MlpSmem *>(base);
    L.tiles = reinterpret_cast<double *>(base + sizeof(MlpSmem));
    L.rows = reinterpret_cast<uint32_t *>(base + sizeof(MlpSmem) + kLearnedTileBytes);
    return L;
}

// Every thread of the CTA calls it (warps without a block pass live = false), between the
// CTA's mlp_setup and mlp_teardown; phase is the MMA barrier's phase, carried across
// calls.  Returns the row sums racc (particle 32 bi + lane), the column sums cacc (particle
// 32 bj + lane; the caller writes -cacc) and the counters; true when the tensor-core
// pipeline timed out.
__device__ __forceinline__ bool learned_block_solve(const LearnedSmem &M, const LearnedBlockIn &B, int bi, int bj,
                                                    int lane, bool live, double racc[6], double cacc[6],
                                                    PairCounters &cnt, uint32_t &phase)
{
    MlpSmem &S = *M.mlp;
    const int warp = threadIdx.x >> 5;
    double *ws = M.tiles + warp * 7 * 32;
    double *wacc = M.tiles + kLearnedWarps * 7 * 32 + warp * 6 * 32;
    uint32_t *dec = reinterpret_cast<uint32_t *>(M.tiles + kLearnedWarps * 7 * 32);  // phase 2 only
    uint32_t *rows = M.rows;
    uint32_t *myrows = rows + warp * 1024 + lane * 32;  // slot k: the pair with column (lane + k) mod 32
    counters_zero(cnt);
    double si[7];
#pragma unroll
    for (int c = 0; c < 6; c++) racc[c] = 0.0;
    const double dt = B.dt;
    const int n = B.n;
    const bool hq = B.q != nullptr;
    {
        double sj[7];
        load_particle(B.x, B.y, B.z, B.u, B.v, B.w, B.q, n, bi * 32 + lane, si);
        load_particle(B.x, B.y, B.z, B.u, B.v, B.w, B.q, n, bj * 32 + lane, sj);
#pragma unroll
        for (int c = 0; c < 7; c++) ws[c * 32 + lane] = sj[c];
        __syncwarp();
    }
    const int i = bi * 32 + lane;
    const bool diag = (bi == bj);

    // 1. classification and the head inputs
    unsigned mh = 0u, me = 0u, mr = 0u;
    if (live) {
        const int k0 = diag ? 1 : 0, k1 = diag ? 16 : 31;
        for (int k = k0; k <= k1; k++) {
            const int src = (lane + k) & 31;
            if ((!diag || k < 16 || lane < 16) && i < n && bj * 32 + src < n) {
                const double r[3] = {si[0] - ws[0 * 32 + src], si[1] - ws[1 * 32 + src], si[2] - ws[2 * 32 + src]};
                const double g[3] = {si[3] - ws[3 * 32 + src], si[4] - ws[4 * 32 + src], si[5] - ws[5 * 32 + src]};
                const double eps_ij = hq ? B.eps_th * si[6] * ws[6 * 32 + src] : B.eps_th;
                const unsigned bit = 1u << k;
                int kind = kLearnedPlain;
                if (learned_candidate(eps_ij, dt, r, g)) {
                    // the split step's routing: a pair whose fifth-order start is exact stays plain
                    if (!uv_series(uv_prepare(eps_ij, r, g), dt).exact) {
                        LearnedPair L;
                        learned_prepare(eps_ij, dt, r, g, L);
                        kind = L.kind;
                        if (kind != kLearnedPlain) myrows[k] = pack_bf16(L.x0, L.x1);
                    }
                }
                if (kind == kLearnedHyp) mh |= bit;
                else if (kind == kLearnedEll) me |= bit;
                else mr |= bit;
            }
        }
    }
    // each thread's first row number per head (thread order, then bit order) and its masks
    int oh, oe, rh, re;
    cta_scan2(S, __popc(mh), __popc(me), oh, oe, rh, re);
    dec[threadIdx.x] = (uint32_t)oh;
    dec[kMlpThreads + threadIdx.x] = (uint32_t)oe;
    dec[2 * kMlpThreads + threadIdx.x] = mh;
    dec[3 * kMlpThreads + threadIdx.x] = me;
    __syncthreads();

    // 2. the heads on the tensor cores, 256 rows per evaluation; the head already in shared
    // memory first (S.head is uniform here: written before the last barrier)
    bool timed_out = false;
    const bool ell_first = S.head == kHeadEll;
    for (int pass = 0; pass < 2; pass++) {
        const bool hyp = (pass == 0) != ell_first;
        const int head = hyp ? kHeadHyp : kHeadEll;
        const uint32_t *first = dec + (hyp ? 0 : kMlpThreads);
        const uint32_t *bits = dec + (hyp ? 2 : 3) * kMlpThreads;
        const int nr = hyp ? rh : re;
        if (nr == 0) continue;  // uniform
        if (S.head != head) {
            __syncthreads();  // every thread has read S.head
            mlp_load_head(S, B.heads, head);
        }
        for (int b = 0; b < nr; b += kMlpThreads) {
            const int row = b + (int)threadIdx.x;
            const bool valid = row < nr;
            int slot = 0;
            if (valid) {
                // the row's owner: the last thread whose first row is <= row (first[] does not
                // decrease), then the (row - first)-th set bit of its mask
                int o = 0;
#pragma unroll
                for (int step = kMlpThreads / 2; step > 0; step >>= 1)
                    if (first[o + step] <= (uint32_t)row) o += step;
                const int k = (int)__fns(bits[o], 0, row - (int)first[o] + 1);
                slot = (o >> 5) * 1024 + (o & 31) * 32 + k;
            }
            const uint32_t x01 = valid ? rows[slot] : 0u;
            bool ok;
            const float y = mlp_eval_cta(S, x01, phase, ok);
            if (!ok) timed_out = true;
            if (valid) rows[slot] = __float_as_uint(ok ? y : __int_as_float(0x7fc00000));
        }
    }
    __syncthreads();
    // the row numbering is read: the column sums start from zero
#pragma unroll
    for (int c = 0; c < 6; c++) wacc[c * 32 + lane] = 0.0;
    __syncwarp();

    // 3. learned pairs from their guesses, per warp.  A warp without learned pairs walks the
    // rotation offsets instead (all its pairs plain; column sums by shuffle, no shared adds)
    const bool warp_learned = __any_sync(0xffffffffu, (mh | me) != 0u);
    if (!warp_learned) {
        const unsigned full = 0xffffffffu;
#pragma unroll
        for (int c = 0; c < 6; c++) cacc[c] = 0.0;
        const int k0 = diag ? 1 : 0, k1 = diag ? 16 : 31;
        for (int k = k0; k <= k1; k++) {
            const int src = (lane + k) & 31;
            double h[6] = {0, 0, 0, 0, 0, 0};
            if ((mr >> k) & 1u) {
                double r[3], g[3];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    r[c] = si[c] - ws[c * 32 + src];
                    g[c] = si[3 + c] - ws[(3 + c) * 32 + src];
                }
                const double eps_ij = hq ? B.eps_th * si[6] * ws[6 * 32 + src] : B.eps_th;
                const int it = uv_halfdisp_fast(eps_ij, dt, r, g, h);
                cnt.it_uv += it;
                if (it > kUvItMax) cnt.nonconverged++;
                cnt.cls[pair_degenerate(r, g) ? kDegenerate : kUniversal]++;
                count_nonfinite(h, cnt);
            }
            const int back = (lane - k) & 31;
#pragma unroll
            for (int c = 0; c < 6; c++) {
                racc[c] += h[c];
                cacc[c] += __shfl_sync(full, h[c], back);
            }
        }
        mr = 0u;
    } else {
        unsigned m = mh | me;
        for (;;) {
            const bool busy = (m != 0u);
            const unsigned bm = __ballot_sync(0xffffffffu, busy);
            if (bm == 0u) break;
            if (busy) {
                const int k = __ffs(m) - 1;
                m &= m - 1u;
                const bool is_h = (mh >> k) & 1u;
                const float y = __uint_as_float(myrows[k]);
                const int j = (lane + k) & 31;
                double r[3], g[3], h[6];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    r[c] = si[c] - ws[c * 32 + j];
                    g[c] = si[3 + c] - ws[(3 + c) * 32 + j];
                }
                const double eps_ij = hq ? B.eps_th * si[6] * ws[6 * 32 + j] : B.eps_th;
                LearnedPair L;
                learned_prepare(eps_ij, dt, r, g, L, is_h ? kLearnedHyp : kLearnedEll);
                bool coarse = true;
                int fp32_steps = 0;
                const bool done = learned_finish(L, dt, y, r, g, h, coarse, fp32_steps);
                cnt.learned++;
                cnt.learned_fp32 += fp32_steps;
                if (coarse) cnt.learned_coarse++;
                if (!done) {
                    cnt.learned_fallbacks++;
                    const int it = uv_halfdisp(eps_ij, dt, r, g, h);
                    cnt.it_uv += it;
                    if (it > kUvItMax) cnt.nonconverged++;
                }
                cnt.cls[is_h ? kHyperbola : kEllipse]++;
                count_nonfinite(h, cnt);
#pragma unroll
                for (int c = 0; c < 6; c++) racc[c] += h[c];
                add_column(wacc, j, h, bm, lane);
            }
        }
    }
    // plain pairs: the universal-variable solver, per warp (mr is empty on rotation warps)
    for (;;) {
        const bool busy = (mr != 0u);
        const unsigned bm = __ballot_sync(0xffffffffu, busy);
        if (bm == 0u) break;
        if (busy) {
            const int k = __ffs(mr) - 1;
            mr &= mr - 1u;
            const int j = (lane + k) & 31;
            double r[3], g[3], h[6];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                r[c] = si[c] - ws[c * 32 + j];
                g[c] = si[3 + c] - ws[(3 + c) * 32 + j];
            }
            const double eps_ij = hq ? B.eps_th * si[6] * ws[6 * 32 + j] : B.eps_th;
            const int it = uv_halfdisp(eps_ij, dt, r, g, h);
            cnt.it_uv += it;
            if (it > kUvItMax) cnt.nonconverged++;
            cnt.cls[pair_degenerate(r, g) ? kDegenerate : kUniversal]++;
            count_nonfinite(h, cnt);
#pragma unroll
            for (int c = 0; c < 6; c++) racc[c] += h[c];
            add_column(wacc, j, h, bm, lane);
        }
    }
    if (warp_learned) {
        __syncwarp();
#pragma unroll
        for (int c = 0; c < 6; c++) cacc[c] = wacc[c * 32 + lane];
    }
    // the row list and the tiles are free for the CTA's next call; a timeout of either
    // warpgroup's tensor-core pipeline counts once
    timed_out = __syncthreads_or(timed_out ? 1 : 0) != 0;
    if (timed_out && threadIdx.x == 0) cnt.timeouts++;
    return timed_out;
}

// One deferred pair (row state si, column state sc) from its head's guess in row `row` of
// head is_h (kNoRows: no row, the plain solver): the FP32 correction and FP64 step, or the
// plain universal-variable solver where the guess does not settle; counted in cnt.
__device__ __forceinline__ void finish_pair(const LearnedRows &R, const LearnedBlockIn &B, const double si[7],
                                            const double sc[7], bool is_h, unsigned int row, double h[6],
                                            PairCounters &cnt)
{
    double r[3], g[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        r[c] = si[c] - sc[c];
        g[c] = si[3 + c] - sc[3 + c];
    }
    const double eps_ij = B.q ? B.eps_th * si[6] * sc[6] : B.eps_th;
    bool done = false;
    if (row != kNoRows) {
        const float yg = __uint_as_float(R.rows[is_h ? kHeadHyp : kHeadEll][row]);
        LearnedPair L;
        learned_prepare(eps_ij, B.dt, r, g, L, is_h ? kLearnedHyp : kLearnedEll);
        bool coarse = true;
        int fp32_steps = 0;
        done = learned_finish(L, B.dt, yg, r, g, h, coarse, fp32_steps);
        cnt.learned++;
        cnt.learned_fp32 += fp32_steps;
        if (coarse) cnt.learned_coarse++;
        if (!done) cnt.learned_fallbacks++;
    }
    if (!done) {
        const int it = uv_halfdisp(eps_ij, B.dt, r, g, h);
        cnt.it_uv += it;
        if (it > kUvItMax) cnt.nonconverged++;
    }
    cnt.cls[is_h ? kHyperbola : kEllipse]++;
    count_nonfinite(h, cnt);
}

// finish_pair for the batched path, compiled once per file: the per-block path inlines
// finish_pair into its own loop, and the compiler may contract the FP64 expressions of an
// inlined copy differently in different places (so the single-system and the ensemble
// kernels, whose batched paths differ around the call, would not give the same bits); one
// out-of-line body gives every kernel the same bits for a batched pair.  Batched pairs are
// few (at most kBatchPairs per warp-block), so the call costs little.
static __device__ __noinline__ void finish_pair_batched(const LearnedRows &R, const LearnedBlockIn &B,
                                                        const double si[7], const double sc[7], bool is_h,
                                                        unsigned int row, double h[6], PairCounters &cnt)
{
    finish_pair(R, B, si, sc, is_h, row, h, cnt);
}

// The finish kernel's work on listed warp-block e (item resolved by the caller to the system
// B and the block (bi, bj)): every deferred pair from its head's guess, with the column
// states and sums in the warp's slice ws.  Returns the row sums racc and column sums cacc of
// those pairs only (the caller adds them onto the rest kernel's partials).  Every lane of the
// warp calls it.
__device__ __forceinline__ void finish_block_solve(const LearnedRows &R, long long e, const LearnedBlockIn &B,
                                                   int bi, int bj, int lane, double *ws, double racc[6],
                                                   double cacc[6], PairCounters &cnt, bool &row_hit,
                                                   bool &col_hit)
{
    const unsigned full = 0xffffffffu;
    double *wacc = ws + 7 * 32;
    const uint4 ent = R.entries[e];
    const uint32_t me = R.masks[(size_t)e * 64 + lane], mh = R.masks[(size_t)e * 64 + 32 + lane];
    // the rows and columns this block's listed pairs touch (bit k of a lane's mask: column
    // (lane + k) mod 32, so the mask rotated left by the lane is the lane's column set)
    row_hit = (me | mh) != 0u;
    col_hit = (__reduce_or_sync(full, __funnelshift_l(me | mh, me | mh, lane)) >> lane) & 1u;
    double si[7];
    {
        double sj[7];
        load_particle(B.x, B.y, B.z, B.u, B.v, B.w, B.q, B.n, bi * 32 + lane, si);
        load_particle(B.x, B.y, B.z, B.u, B.v, B.w, B.q, B.n, bj * 32 + lane, sj);
#pragma unroll
        for (int c = 0; c < 7; c++) ws[c * 32 + lane] = sj[c];
#pragma unroll
        for (int c = 0; c < 6; c++) wacc[c * 32 + lane] = 0.0;
    }
    __syncwarp();
    // the lane's first row of each head: the exclusive prefix of the lanes' counts, as the
    // rest kernel numbered them
    unsigned int pre[kMlpHeads];
#pragma unroll
    for (int hd = 0; hd < kMlpHeads; hd++) {
        const unsigned c = (unsigned)__popc(hd == kHeadEll ? me : mh);
        unsigned inc = c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned o = __shfl_up_sync(full, inc, d);
            if (lane >= d) inc += o;
        }
        pre[hd] = inc - c;
    }
    const bool have_rows = ent.y != kNoRows;
#pragma unroll
    for (int c = 0; c < 6; c++) racc[c] = 0.0;
    counters_zero(cnt);
    uint32_t m = mh | me;
    for (;;) {
        const bool busy = (m != 0u);
        const unsigned bm = __ballot_sync(full, busy);
        if (bm == 0u) break;
        if (busy) {
            const int k = __ffs(m) - 1;
            m &= m - 1u;
            const bool is_h = (mh >> k) & 1u;
            const int j = (lane + k) & 31;
            unsigned int row = kNoRows;
            if (have_rows) {
                const uint32_t below = (1u << k) - 1u;
                row = is_h ? ent.z + pre[kHeadHyp] + (unsigned)__popc(mh & below)
                           : ent.y + pre[kHeadEll] + (unsigned)__popc(me & below);
            }
            double sc[7], h[6];
#pragma unroll
            for (int c = 0; c < 7; c++) sc[c] = ws[c * 32 + j];
            finish_pair(R, B, si, sc, is_h, row, h, cnt);
#pragma unroll
            for (int c = 0; c < 6; c++) racc[c] += h[c];
            add_column(wacc, j, h, bm, lane);
        }
    }
    __syncwarp();
#pragma unroll
    for (int c = 0; c < 6; c++) cacc[c] = wacc[c * 32 + lane];
    __syncwarp();  // the slice is reused by this warp's next block
}

// A listed warp-block as the batched finish sees it: its system, its block and where its
// partial slots live (deterministic: part[m][6][plane]; atomic: one accumulator plane).
struct FinishBlock {
    LearnedBlockIn B;
    int bi, bj;
    double *part;
    size_t plane;
};

// Batched finish of the sparse listed warp-blocks among the 32 list entries of a chunk (lane
// l holds entry l: sparse says whether it is one of them, npairs its deferred pairs).  The
// sparse blocks' pairs are laid end to end and taken 32 at a time, one per lane, each block
// whole within one batch.  A block's pairs sit in the per-block finish's solve order (its
// descriptors), and its row and column sums are added in lane order from zero and then onto
// the slots once, as the per-block finish adds them; which blocks share a batch does not
// change any block's sums, so the step stays deterministic.  resolve(l) gives the
// FinishBlock of the chunk's entry l.  Every lane of the warp calls it.
template <bool kDeterministic, class Resolve>
__device__ __forceinline__ void finish_batches(const LearnedRows &R, long long first_entry, bool sparse,
                                               unsigned int npairs, int lane, const Resolve &resolve,
                                               PairCounters &cnt)
{
    const unsigned full = 0xffffffffu;
    const int c = sparse ? (int)npairs : 0;
    int incl = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int o = __shfl_up_sync(full, incl, d);
        if (lane >= d) incl += o;
    }
    const int total = __shfl_sync(full, incl, 31);
    int done = 0;
    while (done < total) {  // warp-uniform
        // this batch: the blocks whose pairs end within done + 32
        const unsigned bm = __ballot_sync(full, c > 0 && incl > done && incl <= done + kBatchPairs);
        if (bm == 0u) break;  // not reached: the next block's pairs always fit a batch
        const int upto = __shfl_sync(full, incl, 31 - __clz(bm));
        const int qp = done + lane;
        const bool act = qp < upto;
        // the block of pair qp: the first lane whose prefix passes it
        int lo = 0, hi = 31;
#pragma unroll
        for (int it = 0; it < 5; it++) {
            const int mid = (lo + hi) >> 1;
            if (__shfl_sync(full, incl, mid) > qp) hi = mid;
            else lo = mid + 1;
        }
        const int own = lo;
        const int own_start = __shfl_sync(full, incl - c, own);
        double h[6] = {0, 0, 0, 0, 0, 0};
        unsigned int row_key = 0u, col_key = 0u;
        int l = 0, j = 0;
        FinishBlock F{};
        if (act) {
            F = resolve(own);
            const uint2 d = R.pairs[(size_t)(first_entry + own) * kBatchPairs + (qp - own_start)];
            l = (int)(d.y & 31u);
            const int k = (int)((d.y >> 5) & 31u);
            const bool is_h = ((d.y >> 10) & 1u) == (unsigned)kHeadHyp;
            j = (l + k) & 31;
            double si[7], sc[7];
            load_particle(F.B.x, F.B.y, F.B.z, F.B.u, F.B.v, F.B.w, F.B.q, F.B.n, F.bi * 32 + l, si);
            load_particle(F.B.x, F.B.y, F.B.z, F.B.u, F.B.v, F.B.w, F.B.q, F.B.n, F.bj * 32 + j, sc);
            finish_pair_batched(R, F.B, si, sc, is_h, d.x, h, cnt);
            row_key = ((unsigned)own << 6) | (unsigned)l;
            col_key = ((unsigned)own << 6) | 32u | (unsigned)j;
        }
        const unsigned am = __ballot_sync(full, act);
        if (act) {
#pragma unroll
            for (int pass = 0; pass < 2; pass++) {
                const unsigned grp = __match_any_sync(am, pass == 0 ? row_key : col_key);
                double sum[6] = {0, 0, 0, 0, 0, 0};
                for (unsigned m = grp; m; m &= m - 1u) {  // members in lane order (grp-uniform)
                    const int src = __ffs(m) - 1;
#pragma unroll
                    for (int cc = 0; cc < 6; cc++) sum[cc] += __shfl_sync(grp, h[cc], src);
                }
                if (lane == 31 - __clz(grp)) {  // the group's last lane adds the sum once
                    const int p = pass == 0 ? F.bi * 32 + l : F.bj * 32 + j;
                    const size_t m0 = kDeterministic ? (size_t)(pass == 0 ? F.bj : F.bi) * 6 * F.plane : 0;
#pragma unroll
                    for (int cc = 0; cc < 6; cc++) {
                        double *slot = F.part + m0 + (size_t)cc * F.plane + p;
                        const double v = pass == 0 ? sum[cc] : -sum[cc];
                        if (kDeterministic) *slot += v;
                        else atomicAdd(slot, v);
                    }
                }
            }
        }
        done = upto;
    }
}

// The head kernel's pass over the rows of head hd (every thread of the CTA calls it, between
// mlp_setup and mlp_teardown): 256-row tiles t = blockIdx.x + k gridDim.x of the rows taken
// (up to rows_cap), each guess written over its row.  Returns false when the tensor-core
// pipeline timed out (the remaining rows keep their inputs; the step reports the timeout).
__device__ __forceinline__ bool head_rows_pass(MlpSmem &S, const LearnedRows &R, const MlpImage *heads, int hd,
                                               uint32_t &phase)
{
    const unsigned long long taken = *(volatile unsigned long long *)&R.counts[hd];
    const unsigned int nrows = taken < R.rows_cap ? (unsigned int)taken : R.rows_cap;
    const unsigned int ntiles = (nrows + kMlpThreads - 1) / kMlpThreads;
    if ((unsigned int)blockIdx.x >= ntiles) return true;  // CTA-uniform
    if (S.head != hd) {
        __syncthreads();  // every thread has read S.head
        mlp_load_head(S, heads, hd);
    }
    bool ok_all = true;
    for (unsigned int t = blockIdx.x; t < ntiles && ok_all; t += gridDim.x) {
        const unsigned int row = t * kMlpThreads + threadIdx.x;
        const bool valid = row < nrows;
        const uint32_t x01 = valid ? R.rows[hd][row] : 0u;
        bool ok;
        const float y = mlp_eval_cta(S, x01, phase, ok);
        if (!ok) ok_all = false;
        if (valid) R.rows[hd][row] = __float_as_uint(ok ? y : __int_as_float(0x7fc00000));
        ok_all = __syncthreads_and(ok_all ? 1 : 0) != 0;
    }
    return ok_all;
}

// The head kernel of the split learned step (bia_step.cu), shared with the ensemble: its
// once-per-device set-up (returns the resident grid, 0 on failure) and its launch over the
// rows of R with `grid` CTAs.
int learned_head_grid();
void launch_learned_head(const LearnedRows &R, const MlpImage *heads, unsigned long long *stats, int grid,
                         cudaStream_t st);

}  // namespace bia
