// ionic.cu -- the ionic phase of one split step, one thread per node.
//
// Each thread loads its node's state once (SoA, coalesced), runs all ionic
// sub-steps of the global step in registers -- Compute_Ion followed by the
// lumped-capacitance update V <- V + h dV/dt of EP_CrankNicholson.cc:124-133
// -- applies its stimulus window, tracks activation/repolarisation, and
// writes the state back once.
#include <algorithm>

#include "kernels.cuh"

namespace ep {

template <typename R>
__device__ __forceinline__ R node_istim(const IonicArgs<R> &a, int i, long long step) {
    if (a.stim_head == nullptr) return R(0);
    int k = a.stim_head[i];
    long long best_on = -1;
    R amp = R(0);
    while (k >= 0) {
        const long long on = a.stim_on[k], off = a.stim_off[k];
        if (step >= on && step < off && on > best_on) { best_on = on; amp = a.stim_amp[k]; }
        k = a.stim_next[k];
    }
    return amp;
}

template <typename R>
__device__ __forceinline__ void track_update(Track &tr, bool &dirty, R v0, R v1, double t0, R h, R thr) {
    track_interval(tr, dirty, (float)v0, (float)v1, t0, (float)h, (float)thr);
}

// one node's ionic phase (all sub-steps), counters accumulated by the caller;
// WARP: the whole warp advances node i (ten Tusscher; every lane computes the
// same values, lane 0 counts and stores)
template <typename R, int MODEL, int NS, bool WARP = false>
__device__ __forceinline__ void ionic_node(const IonicArgs<R> &a, const int i, unsigned int &my_newton,
                                           unsigned int &my_caps, unsigned int &my_bad, int lane = 0) {
    const long long step = *a.step_ptr;
    const double t_start = (double)step * a.t_per_step;
    R V = a.V[i];
    R s[NS + 1];
#pragma unroll
    for (int k = 0; k < NS; k++) s[k + 1] = a.S[(size_t)k * a.pitch + i];
    const int ty = a.type ? a.type[i] : 0;
    const R istim = node_istim(a, i, step);
    Track tr = {-1.f, -1.f, -1.f, 1e30f};
    bool dirty = false;
    if (a.track) tr = a.track[i];
    const bool do_track = a.track != nullptr && tr.t_rep < 0.f;
    double tsub = t_start;
    R last = R(0);
    // The sub-step lengths: the fixed sequence sub_dt, or (stride) the
    // per-node sequence of CardiacBody::getVoltageFromIonicCurrent
    // (Body/CardiacBody.cc:819-904): one sub-step of stride_dt; when its rate
    // truncates to the integer 0 the stride grows fivefold; sub-steps then
    // fill the global step, the last one shortened to end on it.  One loop
    // with one Compute_Ion call site, so the model code is inlined once.
    const R dT = (R)a.t_per_step;
    const bool multi = a.stride && dT / a.stride_dt > R(1);
    const int kmax = a.stride ? (multi ? (int)(dT / a.stride_dt) + 3 : 1) : a.nsub;
    R h = a.stride ? a.stride_dt : a.sub_dt[0];
    R totT = R(0), hs = a.stride_dt;
    bool more = true;
    for (int k = 0; k < kmax && more; k++) {
        if (!a.stride) {
            h = a.sub_dt[k];
            more = k + 1 < a.nsub;
        } else if (k == 0) {
            h = a.stride_dt;
            more = multi;
        } else {
            more = !(totT + hs > dT);
            h = more ? hs : dT - totT;
        }
        R dvdt;
        if constexpr (MODEL == EP_TUSSCHER) {
            const R *__restrict__ c = a.consts + (size_t)ty * a.nconst;
            const R gks = a.gks ? a.gks[i] : R(1);
            int it = 0;
            if constexpr (WARP) dvdt = tt_compute_ion_warp<R>(s + 1, V, -istim / (a.Cm * a.Xi), h, c, gks, a.tt, it, lane);
            else dvdt = tt_compute_ion<R>(s + 1, V, -istim / (a.Cm * a.Xi), h, c, gks, a.tt, it);
            if (!WARP || lane == 0) {
                my_newton += it;
                if (it >= a.tt.newton_cap) my_caps++;
            }
        } else if constexpr (MODEL == EP_MAHAJAN || MODEL == EP_MAHAJAN_FAIL) {
            const R *__restrict__ c = a.consts + (size_t)ty * a.nconst;
            int sub = 0;
            dvdt = mh_compute_ion<R>(s, V, istim / (a.Cm * a.Xi), h, c, a.mh_abs, sub);
            my_newton += sub;
        } else if constexpr (MODEL == EP_PURKINJE) {
            // the stimulus in uA/cm^3 and the model's (or the user's) Xi;
            // C_m does not enter (Purkinje.cc:183-213)
            const R *__restrict__ c = a.consts + (size_t)ty * a.nconst;
            int sub = 0;
            dvdt = pk_compute_ion<R>(s, V, istim, a.Xi, h, c, sub);
            my_newton += sub;
        } else {
            dvdt = lr_compute_ion<R>(s + 1, V, istim, a.Cm, h, a.lr_table);
        }
        last = dvdt;
        const R v1 = V + h * dvdt;
        if (do_track) track_update(tr, dirty, V, v1, tsub, h, a.act_thr);
        V = v1;
        tsub += (double)h;
        if (a.stride) {
            totT += h;
            if (k == 0) {
                const int slope = (fabs((double)dvdt) < 2.0e9) ? (int)dvdt : 1;
                if (!slope) hs *= R(5);
            }
        }
    }
    if (WARP && lane != 0) return;
    if (!isfinite((double)V)) my_bad = 1;
    if (a.dvdt_out) a.dvdt_out[i] = last;
    else a.V[i] = V;
#pragma unroll
    for (int k = 0; k < NS; k++) a.S[(size_t)k * a.pitch + i] = s[k + 1];
    if (dirty) a.track[i] = tr;
}

// MINB > 1 asks the compiler for MINB resident CTAs of 128 threads per SM
// (fewer registers, some spilled to L1); the autotuner picks it per workload
template <typename R, int MODEL, int NS, int MINB>
__global__ void __launch_bounds__(128, MINB) k_ionic(const IonicArgs<R> a) {
    __shared__ unsigned long long s_newton;
    __shared__ unsigned int s_caps, s_bad;
    if (threadIdx.x == 0) { s_newton = 0; s_caps = 0; s_bad = 0; }
    __syncthreads();
    unsigned int my_newton = 0, my_caps = 0, my_bad = 0;
    // every node or the fallback list of the learned step (the nodes it
    // could not take).  One call site, so both modes run the same machine
    // code and a node's result does not depend on which mode advanced it
    // (k_ionic_warp, which takes the short lists, reproduces those bits).
    int cnt = a.node_list ? *a.list_count : a.n;
    if (a.node_list && a.list_warp_max > 0 && cnt <= a.list_warp_max) cnt = 0;   // k_ionic_warp takes it
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x) {
        const int node = a.node_list ? a.node_list[k] : k;
        if (a.skip && a.skip[node]) continue;
        ionic_node<R, MODEL, NS>(a, node, my_newton, my_caps, my_bad);
    }
    // block-level status reduction, one atomic per block
    for (int o = 16; o > 0; o >>= 1) {
        my_newton += __shfl_xor_sync(0xffffffffu, my_newton, o);
        my_caps += __shfl_xor_sync(0xffffffffu, my_caps, o);
        my_bad += __shfl_xor_sync(0xffffffffu, my_bad, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (my_newton) atomicAdd(&s_newton, (unsigned long long)my_newton);
        if (my_caps) atomicAdd(&s_caps, my_caps);
        if (my_bad) atomicAdd(&s_bad, my_bad);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (s_newton) atomicAdd(&a.status->newton_iters, s_newton);
        if (s_caps) atomicAdd(&a.status->newton_cap_hits, s_caps);
        if (s_bad) atomicAdd(&a.status->nonfinite, s_bad);
    }
}

// A short ten Tusscher node list (at most list_warp_max nodes: the learned
// step's fallback nodes, mostly upstrokes) one warp per node.  Its cost is the
// serial chain of one node's Newton iterations, not throughput, and the warp
// runs the Jacobian's 12 rate evaluations side by side
// (tt_compute_ion_warp: the same bits as one thread per node).
template <typename R>
__global__ void __launch_bounds__(128) k_ionic_warp(const IonicArgs<R> a) {
    __shared__ unsigned long long s_newton;
    __shared__ unsigned int s_caps, s_bad;
    if (threadIdx.x == 0) { s_newton = 0; s_caps = 0; s_bad = 0; }
    __syncthreads();
    unsigned int my_newton = 0, my_caps = 0, my_bad = 0;
    const int cnt = *a.list_count;
    if (cnt <= a.list_warp_max) {            // else k_ionic takes the list
        const int lane = threadIdx.x & 31;
        const int nw = (int)(gridDim.x * blockDim.x) >> 5;
        for (int k = (int)(blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < cnt; k += nw) {
            const int node = a.node_list[k];
            if (a.skip && a.skip[node]) continue;
            ionic_node<R, EP_TUSSCHER, TT_NS, true>(a, node, my_newton, my_caps, my_bad, lane);
        }
    }
    if ((threadIdx.x & 31) == 0) {           // lane 0 holds each warp's counts
        if (my_newton) atomicAdd(&s_newton, (unsigned long long)my_newton);
        if (my_caps) atomicAdd(&s_caps, my_caps);
        if (my_bad) atomicAdd(&s_bad, my_bad);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (s_newton) atomicAdd(&a.status->newton_iters, s_newton);
        if (s_caps) atomicAdd(&a.status->newton_cap_hits, s_caps);
        if (s_bad) atomicAdd(&a.status->nonfinite, s_bad);
    }
}

template <typename R, int MINB>
static void dispatch_ionic(int model, const IonicArgs<R> &a, int grid, int block, cudaStream_t st) {
    switch (model) {
    case EP_TUSSCHER:
        k_ionic<R, EP_TUSSCHER, TT_NS, MINB><<<grid, block, 0, st>>>(a);
        break;
    case EP_MAHAJAN:
    case EP_MAHAJAN_FAIL:
        k_ionic<R, EP_MAHAJAN, MH_NS, MINB><<<grid, block, 0, st>>>(a);
        break;
    case EP_PURKINJE:
        k_ionic<R, EP_PURKINJE, PK_NS, MINB><<<grid, block, 0, st>>>(a);
        break;
    default:
        k_ionic<R, EP_LUORUDY, LR_NS, 1><<<grid, block, 0, st>>>(a);
        break;
    }
}

template <typename R>
int launch_ionic(int model, const IonicArgs<R> &a, cudaStream_t st, int block, int min_ctas) {
    if (block != 64 && block != 128) { set_error("ionic block must be 64 or 128"); return EP_ERR_ARG; }
    if (min_ctas != 0 && min_ctas != 3 && min_ctas != 4) { set_error("ionic min_ctas must be 0, 3 or 4"); return EP_ERR_ARG; }
    if (model != EP_TUSSCHER && model != EP_MAHAJAN && model != EP_MAHAJAN_FAIL && model != EP_LUORUDY &&
        model != EP_LUORUDYWITHGATE && model != EP_PURKINJE) {
        set_error("unknown model %d", model);
        return EP_ERR_ARG;
    }
    int grid = div_up(a.n, block);
    if (a.n == 0) return EP_OK;
    if (a.node_list) {
        // the list length is only known on the device: a fixed grid strides over it
        int dev = 0, nsm = 148;
        EP_CUDA(cudaGetDevice(&dev));
        EP_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        grid = std::min(grid, 16 * nsm);   // one node per thread up to ~300K listed nodes
    }
    if (a.node_list && a.list_warp_max > 0) {
        if constexpr (sizeof(R) == 4) {
            if (model != EP_TUSSCHER) { set_error("one warp per node is built for ten Tusscher lists"); return EP_ERR_ARG; }
            int dev = 0, nsm = 148;
            EP_CUDA(cudaGetDevice(&dev));
            EP_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
            const int wgrid = std::min(div_up((long long)a.list_warp_max * 32, 128), 8 * nsm);
            k_ionic_warp<R><<<wgrid, 128, 0, st>>>(a);
            EP_CUDA(cudaGetLastError());
        } else {
            set_error("one warp per node is built for FP32 lists (the learned step's fallback)");
            return EP_ERR_ARG;
        }
    }
    if constexpr (sizeof(R) == 8) {
        dispatch_ionic<R, 1>(model, a, grid, block, st);       // FP64: the compiler's register choice
    } else {
        if (min_ctas == 0) dispatch_ionic<R, 1>(model, a, grid, block, st);
        else if (min_ctas == 3) dispatch_ionic<R, 3>(model, a, grid, block, st);
        else dispatch_ionic<R, 4>(model, a, grid, block, st);
    }
    EP_CUDA(cudaGetLastError());
    return EP_OK;
}

template int launch_ionic<float>(int, const IonicArgs<float> &, cudaStream_t, int, int);
template int launch_ionic<double>(int, const IonicArgs<double> &, cudaStream_t, int, int);

}  // namespace ep
