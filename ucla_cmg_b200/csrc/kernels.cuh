// kernels.cuh -- launch interfaces of the device kernels (host side).
#pragma once
#include "common.cuh"
#include "tt.cuh"
#include "mahajan.cuh"
#include "lr.cuh"
#include "purkinje.cuh"

namespace ep {

// Per-node activation record {t_act, t_rep, v_peak, v_rest}; -1 = not yet.
struct Track { float t_act, t_rep, v_peak, v_rest; };

// Update the record over one interval [t0, t0 + h] in which V goes v0 -> v1
// (an ionic sub-step, or a whole learned step).  A crossing inside the
// interval is interpolated linearly; a node already past the threshold at
// the interval's start crossed during the preceding diffusion half step and
// is stamped t0 (at most dt/2 late).  Activation: upward crossing of thr;
// repolarisation (APD90): downward crossing of v_peak - 0.9 (v_peak - v_rest)
// later than 5 ms after activation, v_rest = the node's voltage at its first
// tracked interval (the diastolic level the run starts from).  Not the
// minimum before activation: ahead of a steep front the consistent-mass
// Crank-Nicolson step undershoots rest by several mV for a few tenths of a
// ms, and a level taken from that dip falls into the slow end of
// repolarisation (< 0.01 mV/ms), where 1 mV moves the crossing by ~100 ms.
__device__ __forceinline__ void track_interval(Track &tr, bool &dirty, float v0, float v1, double t0, float h,
                                               float thr) {
    if (tr.t_act < 0.f) {
        if (tr.v_rest > 1e29f) { tr.v_rest = v0; dirty = true; }
        if (v0 >= thr) {
            tr.t_act = (float)t0;
            tr.v_peak = fmaxf(v0, v1);
            dirty = true;
        } else if (v1 >= thr) {
            tr.t_act = (float)(t0 + (double)((thr - v0) / (v1 - v0) * h));
            tr.v_peak = v1;
            dirty = true;
        }
    } else if (tr.t_rep < 0.f) {
        if (v1 > tr.v_peak) { tr.v_peak = v1; dirty = true; }
        const float v90 = tr.v_peak - 0.9f * (tr.v_peak - tr.v_rest);
        if ((float)t0 > tr.t_act + 5.f) {
            if (v0 < v90) {
                tr.t_rep = (float)t0;
                dirty = true;
            } else if (v1 < v90) {
                tr.t_rep = (float)(t0 + (double)((v0 - v90) / (v0 - v1) * h));
                dirty = true;
            }
        }
    }
}

// Ionic phase of one global step for all nodes: the reference loop of
// EP_CrankNicholson::Solve (Solvers/EP_CrankNicholson.cc:114-143) with
// CardiacBody::getIonicCurrent (Body/CardiacBody.cc:405-435) inside.
template <typename R> struct IonicArgs {
    int n, pitch;
    R *V;                        // in/out
    R *S;                        // SoA states: S[k * pitch + i]
    const uint8_t *type;         // nullable
    const R *gks;                // nullable (TT)
    // stimulus windows, chained per node (head[i] = -1: none)
    const int *stim_head, *stim_next;
    const long long *stim_on, *stim_off;
    const R *stim_amp;
    const long long *step_ptr;   // device step counter (read)
    double t_per_step;           // dt
    R Cm, Xi;                    // Xi: the model's or the user's
    int nsub;
    R sub_dt[kMaxSub];
    R act_thr;
    Track *track;                // nullable
    DevStatus *status;
    const R *consts;             // ntypes * nconst, device memory
    int nconst;
    R *dvdt_out;                 // non-null: plugin mode -- write the returned
                                 // dV/dt, leave V unchanged (one sub-step)
    const int *node_list;        // non-null: run only these nodes (count on the device)
    const int *list_count;
    int list_warp_max;           // > 0 (ten Tusscher lists): a list of at most this many
                                 // nodes runs one warp per node (k_ionic_warp), a longer
                                 // one one thread per node
    const uint8_t *skip;         // non-null: nodes with skip[i] != 0 are left alone (mixed
                                 // tissues: the Purkinje nodes in the tissue model's launch)
    // model options
    TTOpts tt;
    int mh_abs;
    const R *lr_table;           // nullable
    // stride: the per-node adaptive sub-steps of the backward-Euler and
    // explicit schemes (CardiacBody::getVoltageFromIonicCurrent) with base
    // sub-step stride_dt, instead of the fixed sub_dt sequence
    int stride;
    R stride_dt;
};

template <typename R>
int launch_ionic(int model, const IonicArgs<R> &a, cudaStream_t s, int block = 128, int min_ctas = 0);

// Crank-Nicolson half diffusion step: x <- A^-1 (B x) by Jacobi-PCG in one
// persistent cooperative launch (Solvers/EP_CrankNicholson.cc:99-104).
template <typename R> struct CGArgs {
    int n, nslices;
    const int *slice_ptr;        // nslices + 1
    const int *col;
    const R *Aval, *Bval, *dinv;
    R *x, *r, *q, *p0;           // p0: the direction p (two-reduction: p' of the own rows)
    R *zp;                       // two-reduction variant: 2 * pitch, (z_i, p_i) pairs with
                                 // z = dinv r, gathered by the neighbours (16-byte aligned)
    double *partial;             // 12 * grid: consecutive phases use disjoint slots
    GridBarrier *bar;
    double tol;
    double floor_rel;            // stop also when ||r|| <= floor_rel ||B x||
    int maxit;
    unsigned long long *iters_total;
    unsigned int *iters_max, *fails;
    double *last;                // per instance: [2k] iterations, [2k+1] ||r||/||r0||
    // independent instances (block-diagonal operator): instance k owns rows
    // [inst_row[k], inst_row[k+1]) and CTAs [inst_blk[k], inst_blk[k+1]),
    // solves on its own (own dots, stop test and barrier bar[k]).  ninst <= 1:
    // one instance owning every row and CTA.
    int ninst;
    const int *inst_row, *inst_blk;
    // single-reduction variant only: second r buffer, w = A z and s = A p
    // (two buffers each); p lives in p0
    R *r1, *w0, *w1, *s0, *s1;
    // predictor (two-reduction variant only; nullable): delta = the previous
    // solve's x - V for this half step, updated in place; dext (nullable) the
    // linear extrapolation 2 delta - delta_prev of the last two, which the
    // previous solve stores for the next one's start (one vector gathered in
    // the prologue, not two); vin scratch of n
    R *delta, *dext, *vin;
    // two-reduction variant: each warp asks L2 for the indices and values of
    // the slice it reads `prefetch` slices ahead (0: no prefetch)
    int prefetch;
    // arrivals the grid barrier waits for beyond the CTAs that exist (0;
    // > 0 only from ep_test_hold_barrier, to make the bounded wait run out)
    unsigned int bar_extra;
    // staged variant (cg_batch kStagedBatch): units of 8 slice columns each
    // warp keeps in flight in its shared-memory ring (1 .. kStageMaxDepth)
    int depth;
};

// cg_batch value of the staged kernel (asynchronous copies of each warp's
// next units of SELL columns into shared memory), its deepest ring and the
// depth it runs at when none is asked for
constexpr int kStagedBatch = 32;
// the learned step's fallback list runs one warp per node up to this many
// nodes (its time is then one node's serial Newton chain), one thread per
// node beyond (throughput)
constexpr int kFallbackWarpMax = 4096;
constexpr int kStageMaxDepth = 4;
constexpr int kStageDepthDefault = 2;

// batch: SELL columns gathered per group (4 or 8; two register budgets);
// variant 0: the two-reduction CG of the reference, 1: Chronopoulos-Gear
// (one reduction per iteration; needs r1, w0, w1, s0, s1)
template <typename R>
int launch_cg(const CGArgs<R> &a, int grid, int block, cudaStream_t s, int batch = 4, int variant = 0);
// CTAs of the persistent launch: per_sm (0 = as many as fit) x SM count
template <typename R>
int cg_grid_size(int block, int *grid, int per_sm = 0, int batch = 4, int variant = 0, int depth = 0);
template <typename R>
int cg_max_per_sm(int block, int *per, int batch = 4, int variant = 0, int depth = 0);

// ECG_k = sum_i W[k n + i] V[i] (ComputeECG.h:172-189 in per-node form),
// deterministic two-level reduction, written to out[k].
template <typename R>
int launch_ecg(int n, int ne, const R *W, int wpitch, const R *V, double *partial,
               unsigned int *counter, double *out, int grid, cudaStream_t s,
               unsigned int *slot = nullptr, int cap = 0);

void launch_step_inc(long long *step, cudaStream_t s);
// explicit scheme: V <- V + h (D V) / C_L over the SELL operator D = -K
// (tmp: a scratch vector of n)
template <typename R>
int launch_explicit(int n, int nslices, const int *slice_ptr, const int *col, const R *Dval, const R *cl, R *V,
                    R *tmp, double h, cudaStream_t s);

}  // namespace ep
