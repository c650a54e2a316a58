// cg.cu -- one Crank-Nicolson half diffusion step as a single persistent
// cooperative launch.
//
// Reference: EP_CrankNicholson::Solve (Solvers/EP_CrankNicholson.cc:99-104,
// 146-150): b = B V (B = C_m M - dt/4 K), then AztecOO CG with a Jacobi
// preconditioner on A = C_m M + dt/4 K from x0 = V, stopped when
// ||r_k||_2 <= tol ||r_0||_2.
//
// Layout: SELL-32 (slices of 32 consecutive rows, column-major inside the
// slice, one warp per slice, one lane per row) so every value/column load is
// a coalesced 128-byte transaction.  A and B share the column array.
//
// Per iteration two grid barriers:
//   phase A  p' = z + beta p (recomputed on the fly for each column, z =
//            dinv r), q = A p', partial p'.q          -> barrier
//   phase B  x += alpha p', r -= alpha q, partial r.z, r.r -> barrier
// The same thread owns a row in every phase, so x, r, q need no cross-block
// visibility; only r and p are read across blocks (through L2, ld.cg).
// Dot products accumulate in FP64 whatever the vector type.  Reductions
// sum the per-block partials in block order, so results are deterministic.
#include "kernels.cuh"

namespace ep {

__device__ __forceinline__ float ldcg(const float *p) { return __ldcg(p); }
__device__ __forceinline__ double ldcg(const double *p) { return __ldcg(p); }

// p' = z + beta p with z = dinv r, written as one explicit fma so the owner
// row and every neighbour that recomputes it round identically
template <typename R>
__device__ __forceinline__ R pdir(R dinv, R r, R beta, R p) { return fma(beta, p, dinv * r); }

template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&v)[NV], double *out, int stride) {
    __shared__ double sh[NV][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; k++) sh[k][warp] = v[k];
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double t = lane < nw ? sh[k][lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            if (lane == 0) out[k * stride + blockIdx.x] = t;
        }
    }
    __syncthreads();
}

// every block of a group sums the group's partials in the same order
template <int NV>
__device__ __forceinline__ void grid_total(const double *partial, int stride, int b0, int nblk, double (&tot)[NV]) {
    __shared__ double sh[NV];
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double t = 0.0;
            for (int b = lane; b < nblk; b += 32) t += __ldcg(partial + k * stride + b0 + b);
            for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            if (lane == 0) sh[k] = t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++) tot[k] = sh[k];
    __syncthreads();
}

// Row sums of one SELL slice, NB slice columns at a time: the column and
// value loads of a group are issued together, then the gathers, so each lane
// has 3 NB independent loads in flight (at one lane per row the kernel is
// bound by memory latency, not bandwidth).  The products are still added in
// column order, so the sums are those of the plain loop whatever NB is.
template <int NB, typename R, typename F>
__device__ __forceinline__ R slice_row_sum(const int *__restrict__ col, const R *__restrict__ val, int beg, int w,
                                           int lane, F gather) {
    R acc = R(0);
    int k = 0;
    for (; k + NB <= w; k += NB) {
        int c[NB];
        R v[NB], g[NB];
#pragma unroll
        for (int u = 0; u < NB; u++) {
            const int idx = beg + (k + u) * kSlice + lane;
            c[u] = __ldg(col + idx);
            v[u] = __ldg(val + idx);
        }
#pragma unroll
        for (int u = 0; u < NB; u++) g[u] = gather(c[u]);
#pragma unroll
        for (int u = 0; u < NB; u++) acc += v[u] * g[u];
    }
    for (; k < w; k++) {
        const int idx = beg + k * kSlice + lane;
        acc += __ldg(val + idx) * gather(__ldg(col + idx));
    }
    return acc;
}

// register budget: NB = 4 takes 42 (six 256-thread CTAs, or two of 768, per
// SM); NB = 8 takes 64 (four 256-thread CTAs) for twice the loads in flight
template <typename R, int NB>
__global__ void __launch_bounds__(NB == 4 ? 768 : 256, NB == 4 ? 2 : 4) k_cn_half(const CGArgs<R> a) {
    const int lane = threadIdx.x & 31;
    const int G = gridDim.x;                 // partial-array stride
    // this CTA's instance: its rows, its CTA group and its barrier
    int inst = 0, b0 = 0, nb = G, rb = 0, re = a.n;
    if (a.ninst > 1) {
        int lo = 0, hi = a.ninst - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.inst_blk[mid] <= (int)blockIdx.x) lo = mid; else hi = mid - 1;
        }
        inst = lo;
        b0 = a.inst_blk[inst]; nb = a.inst_blk[inst + 1] - b0;
        rb = a.inst_row[inst]; re = a.inst_row[inst + 1];
    }
    GridBarrier *bar = a.bar + inst;
    const unsigned int nblk = nb;
    const int s_lo = rb / kSlice, s_hi = (re + kSlice - 1) / kSlice;
    const int gwarp = s_lo + (((int)blockIdx.x - b0) * (int)blockDim.x + (int)threadIdx.x) / 32;
    const int nwarps = (nb * (int)blockDim.x) >> 5;

    // ---- prologue: r = B x - A x, z = dinv r, p = 0 ----
    {
        double v[3] = {0.0, 0.0, 0.0};
        for (int s = gwarp; s < s_hi; s += nwarps) {
            const int row = s * kSlice + lane;
            const int beg = a.slice_ptr[s], w = (a.slice_ptr[s + 1] - beg) / kSlice;
            R ax = R(0), bx = R(0);
            for (int k = 0; k < w; k++) {
                const int idx = beg + k * kSlice + lane;
                const int c = __ldg(a.col + idx);
                const R xv = a.x[c];
                ax += __ldg(a.Aval + idx) * xv;
                bx += __ldg(a.Bval + idx) * xv;
            }
            if (row >= rb && row < re) {
                const R r = bx - ax;
                const R z = __ldg(a.dinv + row) * r;
                a.r[row] = r;
                a.p0[row] = R(0);
                v[0] += (double)r * (double)z;
                v[1] += (double)r * (double)r;
                v[2] += (double)bx * (double)bx;
            }
        }
        block_reduce_store<3>(v, a.partial, G);
    }
    if (!grid_sync(bar, nblk)) return;
    double rz, rr0, bb;
    {
        double t[3];
        grid_total<3>(a.partial, G, b0, nb, t);
        rz = t[0]; rr0 = t[1]; bb = t[2];
    }
    // ||r|| <= tol ||r0||, or the residual is at the resolution of b in the
    // vector type (FP32 cannot resolve a 1e-7 reduction of an r0 that is
    // itself rounding noise of B x - A x; in FP64 the floor is ~1e-16 ||b||)
    const double floor2 = a.floor_rel * a.floor_rel * bb;
    const double stop2 = fmax(a.tol * a.tol * rr0, floor2);
    double beta = 0.0;
    int it = 0;
    bool converged = (rr0 <= stop2);
    double rr_last = rr0;
    R *pc = a.p0, *pn = a.p1;
    while (!converged && it < a.maxit) {
        // ---- phase A: p' = z + beta p; q = A p' ----
        {
            double v[1] = {0.0};
            const R bR = (R)beta;
            for (int s = gwarp; s < s_hi; s += nwarps) {
                const int row = s * kSlice + lane;
                const int beg = a.slice_ptr[s], w = (a.slice_ptr[s + 1] - beg) / kSlice;
                const R *pcc = pc;
                const R q = slice_row_sum<NB>(a.col, a.Aval, beg, w, lane, [&](int c) {
                    return pdir(__ldg(a.dinv + c), ldcg(a.r + c), bR, ldcg(pcc + c));
                });
                if (row >= rb && row < re) {
                    const R pi = pdir(__ldg(a.dinv + row), a.r[row], bR, ldcg(pc + row));
                    pn[row] = pi;
                    a.q[row] = q;
                    v[0] += (double)pi * (double)q;
                }
            }
            block_reduce_store<1>(v, a.partial + 3 * G, G);   // disjoint from the neighbours' slots
        }
        if (!grid_sync(bar, nblk)) return;
        double pq;
        {
            double t[1];
            grid_total<1>(a.partial + 3 * G, G, b0, nb, t);
            pq = t[0];
        }
        const double alpha = rz / pq;
        // ---- phase B: x += alpha p', r -= alpha q ----
        {
            double v[2] = {0.0, 0.0};
            const R aR = (R)alpha;
            for (int s = gwarp; s < s_hi; s += nwarps) {
                const int row = s * kSlice + lane;
                if (row >= rb && row < re) {
                    const R pi = pn[row];
                    a.x[row] += aR * pi;
                    const R r = a.r[row] - aR * a.q[row];
                    a.r[row] = r;
                    const R z = __ldg(a.dinv + row) * r;
                    v[0] += (double)r * (double)z;
                    v[1] += (double)r * (double)r;
                }
            }
            block_reduce_store<2>(v, a.partial, G);
        }
        if (!grid_sync(bar, nblk)) return;
        double t[2];
        grid_total<2>(a.partial, G, b0, nb, t);
        it++;
        rr_last = t[1];
        converged = (t[1] <= stop2);
        beta = t[0] / rz;
        rz = t[0];
        R *tmp = pc; pc = pn; pn = tmp;
    }
    if ((int)blockIdx.x == b0 && threadIdx.x == 0) {
        atomicAdd(a.iters_total, (unsigned long long)it);
        atomicMax(a.iters_max, (unsigned int)it);
        if (!converged) atomicAdd(a.fails, 1u);
        if (a.last) {
            a.last[2 * inst] = (double)it;
            a.last[2 * inst + 1] = rr0 > 0.0 ? sqrt(rr_last / rr0) : 0.0;
        }
    }
}

template <typename R>
int cg_max_per_sm(int block, int *per, int batch) {
    if (batch == 8) EP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per, k_cn_half<R, 8>, block, 0));
    else EP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per, k_cn_half<R, 4>, block, 0));
    if (*per < 1) { set_error("CG kernel cannot be resident with %d threads per CTA", block); return EP_ERR_CUDA; }
    return EP_OK;
}

template <typename R>
int cg_grid_size(int block, int *grid, int per_sm, int batch) {
    int dev = 0, nsm = 0, per = 0;
    EP_CUDA(cudaGetDevice(&dev));
    EP_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    int rc = cg_max_per_sm<R>(block, &per, batch);
    if (rc) return rc;
    if (per_sm > 0 && per_sm < per) per = per_sm;
    *grid = nsm * per;
    return EP_OK;
}

template <typename R>
int launch_cg(const CGArgs<R> &a, int grid, int block, cudaStream_t s, int batch) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (batch == 8) EP_CUDA(cudaLaunchKernelEx(&cfg, k_cn_half<R, 8>, a));
    else EP_CUDA(cudaLaunchKernelEx(&cfg, k_cn_half<R, 4>, a));
    return EP_OK;
}

template int launch_cg<float>(const CGArgs<float> &, int, int, cudaStream_t, int);
template int launch_cg<double>(const CGArgs<double> &, int, int, cudaStream_t, int);
template int cg_grid_size<float>(int, int *, int, int);
template int cg_grid_size<double>(int, int *, int, int);
template int cg_max_per_sm<float>(int, int *, int);
template int cg_max_per_sm<double>(int, int *, int);

// ---------------------------------------------------------------------------
// pseudo-ECG: out[k] = sum_i W[k * wpitch + i] V[i], FP64 accumulation.
// Block partials, then the last block to finish sums them in block order.
template <typename R>
__global__ void __launch_bounds__(256) k_ecg(int n, int ne, const R *__restrict__ W, int wpitch,
                                             const R *__restrict__ V, double *partial,
                                             unsigned int *counter, double *out, unsigned int *slot, int cap) {
    constexpr int MAXE = 16;
    double acc[MAXE];
#pragma unroll
    for (int k = 0; k < MAXE; k++) acc[k] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double v = (double)V[i];
#pragma unroll
        for (int k = 0; k < MAXE; k++)
            if (k < ne) acc[k] += (double)__ldg(W + (size_t)k * wpitch + i) * v;
    }
    __shared__ double sh[MAXE][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < MAXE; k++) {
        double t = acc[k];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (lane == 0) sh[k][warp] = t;
    }
    __syncthreads();
    __shared__ bool last;
    if (threadIdx.x < ne) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[threadIdx.x][w];
        partial[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = t;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (last) {
        __threadfence();
        // with a slot counter the sample goes to row *slot of out (the
        // counter lives on the device so that replayed graphs advance it)
        const unsigned int row = slot ? *(volatile unsigned int *)slot : 0u;
        if (threadIdx.x < ne && (int)row < cap) {
            double t = 0.0;
            for (int b = 0; b < (int)gridDim.x; b++) t += __ldcg(partial + (size_t)threadIdx.x * gridDim.x + b);
            out[(size_t)row * ne + threadIdx.x] = t;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            *counter = 0;
            if (slot) *slot = row + 1u;
        }
    }
}

template <typename R>
int launch_ecg(int n, int ne, const R *W, int wpitch, const R *V, double *partial,
               unsigned int *counter, double *out, int grid, cudaStream_t s, unsigned int *slot, int cap) {
    if (ne <= 0) return EP_OK;
    if (ne > 16) { set_error("at most 16 electrodes"); return EP_ERR_ARG; }
    k_ecg<R><<<grid, 256, 0, s>>>(n, ne, W, wpitch, V, partial, counter, out, slot, slot ? cap : 1);
    EP_CUDA(cudaGetLastError());
    return EP_OK;
}

template int launch_ecg<float>(int, int, const float *, int, const float *, double *, unsigned int *,
                               double *, int, cudaStream_t, unsigned int *, int);
template int launch_ecg<double>(int, int, const double *, int, const double *, double *,
                                unsigned int *, double *, int, cudaStream_t, unsigned int *, int);

__global__ void k_step_inc(long long *step) { *step += 1; }
void launch_step_inc(long long *step, cudaStream_t s) { k_step_inc<<<1, 1, 0, s>>>(step); }

}  // namespace ep
