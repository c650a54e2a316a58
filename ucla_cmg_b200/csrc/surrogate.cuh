// surrogate.cuh -- the learned ionic step: BF16 tcgen05 inference kernel
// interface and the packed parameter block it reads.
#pragma once
#include "kernels.cuh"

namespace ep {

constexpr int SG_M = 128;        // nodes per tile = MMA M = TMEM lanes
constexpr int SG_THREADS = 256;  // threads per CTA of the network kernel
constexpr int SG_H = 128;        // hidden width
constexpr int SG_KIN = 32;       // padded input width
constexpr int SG_NOUT = 32;      // padded output width
constexpr int SG_NF = 23;        // features used: V, 18 states, I_stim, G_Ks, G_to, s-gate variant
constexpr int SG_NY = 19;        // outputs used: dV, 18 state changes
// BF16 weight images, laid out as the UMMA no-swizzle K-major core matrices
constexpr int SG_W1 = SG_H * SG_KIN;       // elements
constexpr int SG_W2 = SG_H * SG_H;
constexpr int SG_W3 = SG_H * SG_H;
constexpr int SG_W4 = SG_NOUT * SG_H;
constexpr int SG_WTOT = SG_W1 + SG_W2 + SG_W3 + SG_W4;   // 40960 bf16 = 80 KB

// FP32 side parameters (device, global memory)
struct SurrogateAux {
    float b1[SG_H], b2[SG_H], b3[SG_H], b4[SG_NOUT];
    float in_mean[SG_KIN], in_rstd[SG_KIN];
    float out_mean[SG_NOUT], out_std[SG_NOUT];
    float out_scale[SG_NOUT];   // > 0: output j is asinh(delta / out_scale[j])
    float out_lo[SG_NOUT], out_hi[SG_NOUT];   // accepted range of the de-normalised outputs
    unsigned int out_mask;      // outputs the state update uses
    int hyb_sub;                // v_update 2: sub-steps per global step (0: the handle's)
    float env_lo[SG_KIN], env_hi[SG_KIN];   // in the transformed (log) space
    float nah_max;
    unsigned int log_mask;      // bit k: feature k (and state output k) is log-scaled
    int v_update;               // 0: every quantity from the network;
                                // 2: network concentrations, reference gates and V
};

// element offset of (row r, column k) of an R x K bf16 matrix in the core
// matrix layout: 8x8 blocks of 128 bytes, k-blocks contiguous, then row blocks
__host__ __device__ inline int core_offset(int r, int k, int K) {
    return ((r >> 3) * (K >> 3) + (k >> 3)) * 64 + (r & 7) * 8 + (k & 7);
}

struct SurrogateArgs {
    int n, pitch;
    float *V, *S;                       // FP32 state (SoA), updated for in-envelope nodes
    const uint8_t *type;
    const float *gks;
    const float *consts;                // TT parameter sets (FP32)
    int nconst;
    // stimulus (the same windows as the plain kernel)
    const int *stim_head, *stim_next;
    const long long *stim_on, *stim_off;
    const float *stim_amp;
    const long long *step_ptr;
    int nsub;                           // ionic sub-steps of one global step
    float sub_dt[kMaxSub];
    double t_per_step;
    float Cm, Xi, act_thr;
    Track *track;
    const unsigned short *wimg;         // SG_WTOT bf16 (core-matrix images W1|W2|W3|W4)
    const SurrogateAux *aux;
    int *fallback_list, *fallback_count;
    DevStatus *status;
    unsigned int *err;                  // set when an in-kernel wait gave up
    unsigned int mbar_polls;            // polls of one completion wait (0: kMbarPolls)
    // raw mode (tests): X [n x 32] normalised inputs -> Y [n x 32] raw outputs
    const float *rawX;
    float *rawY;
    // hybrid form: the network's new concentrations [6][pitch] and which
    // nodes it took (1) or handed to the plain model (0)
    float *pred;
    uint8_t *take;
};

int launch_surrogate(const SurrogateArgs &a, cudaStream_t s, int variant = 0);
int launch_hybrid(const SurrogateArgs &a, cudaStream_t s);
size_t surrogate_smem_bytes();

}  // namespace ep
