// bia_internal.cuh -- shared host-side definitions of libbia_b200.so.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "../../include/bia_capi.h"

namespace bia {

// device counters in the stats buffer: hyperbola, parabola, ellipse, degenerate, rkf,
// universal, iter_hyperbola, iter_ellipse, iter_parabola, iter_universal, rkf_steps,
// nonconverged, bracket_exits, fallbacks, nonfinite
constexpr int kNumStats = 20;
constexpr int kStatNonfinite = 14;
constexpr int kStatTimeouts = 18;  // tensor-core waits that gave up

struct DeviceBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    // grow-only; returns cudaSuccess or the allocation error
    cudaError_t reserve(size_t want)
    {
        if (want <= bytes) return cudaSuccess;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&ptr, want);
        if (e == cudaSuccess) bytes = want;
        return e;
    }
    void release()
    {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

struct GraphKey {
    int n = -1, nsteps = -1, method = -1, itr = -1, deterministic = -1;
    double eps = 0, dt = 0, err = 0, relerr = 0, abserr = 0;
    const void *ptrs[7] = {};
    bool operator==(const GraphKey &o) const
    {
        if (n != o.n || nsteps != o.nsteps || method != o.method || itr != o.itr ||
            deterministic != o.deterministic)
            return false;
        if (eps != o.eps || dt != o.dt || err != o.err || relerr != o.relerr || abserr != o.abserr)
            return false;
        for (int k = 0; k < 7; k++)
            if (ptrs[k] != o.ptrs[k]) return false;
        return true;
    }
};

}  // namespace bia

struct bia_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    bia::DeviceBuffer part;     // deterministic per-block partial sums
    bia::DeviceBuffer acc;      // atomic-mode accumulators
    bia::DeviceBuffer stats;    // kNumStats unsigned long long
    bia::DeviceBuffer state;    // host-path staging: 7 arrays of n
    bia::DeviceBuffer inv;      // invariance partials
    bia::DeviceBuffer dim;      // DIM integrator work arrays
    double *h_dim = nullptr;    // pinned scalars of the DIM control loop
    unsigned long long *h_stats = nullptr;  // pinned
    double *h_inv = nullptr;                // pinned
    // kernel timing
    bool timing = false;
    cudaEvent_t *ev = nullptr;
    int ev_cap = 0, ev_used = 0;
    // autotuned ALG pair-kernel shape per reduction mode and floor(log2 n); -1: default rule
    int alg_tuned[2][32];
    // autotuned learned-step layout (0 one kernel, 1 split), same indexing; -1: default rule
    int learned_tuned[2][32];
    // learned heads (BIA_METHOD_LEARNED), 2 records of learned_heads.bin
    bia::DeviceBuffer heads;
    bool heads_loaded = false;
    bia::DeviceBuffer lmask;    // learned-pair masks of a split learned step
    // graph cache
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    bia::GraphKey graph_key;
};

namespace bia {
int set_last_error(int status);
int cuda_status(cudaError_t e);
// stream-ordered launches of one step (no synchronisation); used by bia_step and graphs
int enqueue_step(bia_context *ctx, const bia_config *cfg, int n, double *x, double *y, double *z,
                 double *u, double *v, double *w, const double *q, double *disp);
int ensure_step_buffers(bia_context *ctx, const bia_config *cfg, int n);
// SM count of the current device (cached); the grid of a persistent warp-block kernel
int device_sm_count();
long long persistent_grid(long long blocks_needed);
}  // namespace bia
