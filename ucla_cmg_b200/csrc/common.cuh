// common.cuh -- shared helpers of the sm_100a monodomain library.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/ep_gpu.h"

// cell-model code is host+device so the same source can be exercised on
// the host (tests, debugging) and compiled into the sm_100a kernels
#define EP_HD __host__ __device__ __forceinline__

namespace ep {

// ---- error reporting (thread-local message behind ep_last_error) ----
void set_error(const char *fmt, ...);
const char *last_error();

#define EP_CUDA(call)                                                          \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) {                                               \
            ::ep::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,         \
                            cudaGetErrorString(e_));                           \
            return EP_ERR_CUDA;                                                \
        }                                                                      \
    } while (0)

#define EP_CHECK_ARG(cond, msg)                                                \
    do {                                                                       \
        if (!(cond)) { ::ep::set_error("%s", msg); return EP_ERR_ARG; }        \
    } while (0)

constexpr int kMaxTypes = 256;     // parameter sets per handle (uint8 node types)
constexpr int kMaxSub = 64;        // ionic sub-steps per global step
constexpr int kSlice = 32;         // SELL slice height (one warp)

// Device status word shared by all kernels of a handle.
struct DevStatus {
    unsigned long long newton_iters;
    unsigned int newton_cap_hits;
    unsigned int timeouts;
    unsigned int nonfinite;
    unsigned int cg_fail;
    unsigned long long fallback;
    unsigned int pad[8];
};

// Bounded sense-reversing grid barrier for cooperative (co-resident) grids.
// Returns false when the wait gave up; the caller must then leave the kernel
// (every block reaches the same conclusion through *err).  `limit` caps the
// polls of one wait (0: kGridPolls, a few seconds); a wait that runs out
// sets err, which the host reads as EP_ERR_TIMEOUT and then clears.
constexpr unsigned int kGridPolls = 1u << 24;
struct GridBarrier {
    unsigned int count;
    unsigned int gen;
    unsigned int err;
    unsigned int limit;
};

__device__ __forceinline__ bool grid_sync(GridBarrier *b, unsigned int nblocks) {
    __shared__ int s_ok;
    // the CTA barrier orders every thread's writes before thread 0's
    // gpu-scope fence and arrival (fences are cumulative), as a cooperative
    // grid sync does: one fence per CTA, not one per thread
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        volatile unsigned int *vgen = &b->gen;
        volatile unsigned int *verr = &b->err;
        const unsigned int lim = *(volatile unsigned int *)&b->limit;
        const unsigned int max_polls = lim ? lim : kGridPolls;
        const unsigned int g = *vgen;
        __threadfence();
        // the last arrival wraps the count back to 0 in the same atomic (no
        // separate reset store for the release fence to wait on)
        const unsigned int arrived = atomicInc(&b->count, nblocks - 1u);
        if (arrived == nblocks - 1) {
            __threadfence();
            atomicAdd(&b->gen, 1u);
        } else {
            // at most max_polls polls with a short sleep, then give up
            unsigned int polls = 0;
            while (*vgen == g) {
                if (*verr) { ok = 0; break; }
                if (++polls > max_polls) { atomicExch(&b->err, 1u); ok = 0; break; }
                __nanosleep(64);
            }
        }
        __threadfence();
        if (*verr) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

template <typename T> struct RealName;
template <> struct RealName<float> { static constexpr const char *s = "f32"; };
template <> struct RealName<double> { static constexpr const char *s = "f64"; };

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace ep
