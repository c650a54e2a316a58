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
// visibility; z and p are read across blocks, interleaved as (z_i, p_i) pairs
// so that one load brings a neighbour's both (phase B writes the pair: the
// new z and the p' it used).  Phase A gathers them with
// plain (L1-allocating) loads: neither changes during the phase, and the grid
// barrier before it (a gpu-scope fence after the arrival wait, then the CTA
// barrier, as a cooperative grid sync) orders every block's writes of the
// previous phase before them, so the neighbouring rows of a slice, which
// gather many of the same nodes, hit L1 (2 % faster than L2-only loads on
// the 2M-node shell, same bits).
// Dot products accumulate in FP64 whatever the vector type.  Reductions
// sum the per-block partials in block order, so results are deterministic.
#include <algorithm>

#include "kernels.cuh"

namespace ep {

__device__ __forceinline__ float ldcg(const float *p) { return __ldcg(p); }
__device__ __forceinline__ double ldcg(const double *p) { return __ldcg(p); }

// p' = z + beta p with z = dinv r, written as one explicit fma so the owner
// row and every neighbour that recomputes it round identically
template <typename R>
__device__ __forceinline__ R pdir(R dinv, R r, R beta, R p) { return fma(beta, p, dinv * r); }
// the same with z = dinv r already rounded and stored
template <typename R>
__device__ __forceinline__ R pdir_z(R z, R beta, R p) { return fma(beta, p, z); }

// the gathered pair (z_i, p_i) of the two-reduction kernels, interleaved so a
// neighbour's two values come in one load (zp[2i] = z_i, zp[2i+1] = p_i)
template <typename R> struct ZP;
template <> struct ZP<float> { using T = float2; };
template <> struct ZP<double> { using T = double2; };
template <typename R> using zp_t = typename ZP<R>::T;

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

// Ask L2 for the column indices and values (and the B values when Bv is
// given) of slice sn, which this warp reads next: one lane issues bulk L2
// prefetches, so the warp's next index loads hit L2 instead of waiting on
// DRAM.  A hint only: nothing waits on it.  Every slice starts on a 128-byte
// boundary of the arrays and spans a multiple of 128 bytes.
__device__ __forceinline__ void l2_prefetch(const void *p, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}
template <typename R>
__device__ __forceinline__ void prefetch_slice(const int *__restrict__ slice_ptr, const int *col, const R *Av,
                                               const R *Bv, int sn, int s_hi, int lane) {
    if (lane == 0 && sn < s_hi) {
        const int b = slice_ptr[sn], e = slice_ptr[sn + 1];
        if (e > b) {
            l2_prefetch(col + b, (unsigned)(e - b) * 4u);
            l2_prefetch(Av + b, (unsigned)(e - b) * (unsigned)sizeof(R));
            if (Bv) l2_prefetch(Bv + b, (unsigned)(e - b) * (unsigned)sizeof(R));
        }
    }
}

// The columns k .. w-1 (fewer than NB) of a slice as one group: loads of the
// columns that exist (the test is the same for the whole warp), then their
// gathers, then the products added in column order.
template <int NB, typename R, typename F>
__device__ __forceinline__ R slice_tail(const int *__restrict__ col, const R *__restrict__ val, int beg, int k, int w,
                                        int lane, F gather, R acc) {
    int c[NB];
    R v[NB], g[NB];
#pragma unroll
    for (int u = 0; u < NB; u++) {
        if (k + u < w) {
            const int idx = beg + (k + u) * kSlice + lane;
            c[u] = __ldg(col + idx);
            v[u] = __ldg(val + idx);
        }
    }
#pragma unroll
    for (int u = 0; u < NB; u++)
        if (k + u < w) g[u] = gather(c[u]);
#pragma unroll
    for (int u = 0; u < NB; u++)
        if (k + u < w) acc += v[u] * g[u];
    return acc;
}

// G columns k .. k+G-1 of a slice as one group: their column and value loads,
// then their gathers, then the products added in column order
template <int G, typename R, typename F>
__device__ __forceinline__ R slice_group(const int *__restrict__ col, const R *__restrict__ val, int beg, int k,
                                         int lane, F gather, R acc) {
    int c[G];
    R v[G], g[G];
#pragma unroll
    for (int u = 0; u < G; u++) {
        const int idx = beg + (k + u) * kSlice + lane;
        c[u] = __ldg(col + idx);
        v[u] = __ldg(val + idx);
    }
#pragma unroll
    for (int u = 0; u < G; u++) g[u] = gather(c[u]);
#pragma unroll
    for (int u = 0; u < G; u++) acc += v[u] * g[u];
    return acc;
}

// Row sums of one SELL slice, NB slice columns at a time: the column and
// value loads of a group are issued together, then the gathers, so each lane
// has 3 NB independent loads in flight (at one lane per row the kernel is
// bound by memory latency, not bandwidth); the w mod NB columns left over
// form one more, partial group -- except a single one, which joins the last
// full group (a 17-wide slice gathers in 2 rounds of 8 + 9, not 3 of
// 8 + 8 + 1: on the shell's meshes this is what evens out the warps' loads).
// The products are still added in column order, so the sums are those of
// the plain loop whatever the grouping.
template <int NB, typename R, typename F>
__device__ __forceinline__ R slice_row_sum(const int *__restrict__ col, const R *__restrict__ val, int beg, int w,
                                           int lane, F gather) {
    R acc = R(0);
    int k = 0;
    for (; k + NB <= w && w - k != NB + 1; k += NB) acc = slice_group<NB>(col, val, beg, k, lane, gather, acc);
    if (w - k == NB + 1) acc = slice_group<NB + 1>(col, val, beg, k, lane, gather, acc);
    else if (k < w) acc = slice_tail<NB>(col, val, beg, k, w, lane, gather, acc);
    return acc;
}

// Prologue sums of one slice row: A x and B x, and A d when pred (d = the
// predictor's start correction, dget(c) its value at column c), NB columns
// a group like slice_row_sum; each sum is added in column order.
template <int NB, typename R, typename FD>
__device__ __forceinline__ void slice_ab_sums(const int *__restrict__ col, const R *__restrict__ Av,
                                              const R *__restrict__ Bv, const R *x, int beg, int w, int lane,
                                              bool pred, FD dget, R &ax, R &bx, R &ad) {
    for (int k = 0; k < w; k += NB) {
        int c[NB];
        R av[NB], bv[NB], xv[NB], dv[NB];
#pragma unroll
        for (int u = 0; u < NB; u++) {
            if (k + u < w) {
                const int idx = beg + (k + u) * kSlice + lane;
                c[u] = __ldg(col + idx);
                av[u] = __ldg(Av + idx);
                bv[u] = __ldg(Bv + idx);
            }
        }
#pragma unroll
        for (int u = 0; u < NB; u++) {
            if (k + u < w) {
                xv[u] = x[c[u]];
                if (pred) dv[u] = dget(c[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < NB; u++) {
            if (k + u < w) {
                ax += av[u] * xv[u];
                bx += bv[u] * xv[u];
                if (pred) ad += av[u] * dv[u];
            }
        }
    }
}

// The same sum with the next group's column and value loads issued before
// the current group's gathers (software pipelining: the index loads of
// group k + 1 overlap the gathers of group k).  Same order of additions.
template <int NB, typename R, typename F>
__device__ __forceinline__ R slice_row_sum_pipe(const int *__restrict__ col, const R *__restrict__ val, int beg, int w,
                                                int lane, F gather) {
    R acc = R(0);
    const int full = w / NB;
    int c[NB], cn[NB];
    R v[NB], vn[NB];
    if (full > 0) {
#pragma unroll
        for (int u = 0; u < NB; u++) {
            const int idx = beg + u * kSlice + lane;
            c[u] = __ldg(col + idx);
            v[u] = __ldg(val + idx);
        }
    }
    for (int b = 0; b < full; b++) {
        const bool more = b + 1 < full;
#pragma unroll
        for (int u = 0; u < NB; u++) {
            const int idx = beg + ((b + 1) * NB + u) * kSlice + lane;
            cn[u] = more ? __ldg(col + idx) : 0;
            vn[u] = more ? __ldg(val + idx) : R(0);
        }
        R g[NB];
#pragma unroll
        for (int u = 0; u < NB; u++) g[u] = gather(c[u]);
#pragma unroll
        for (int u = 0; u < NB; u++) acc += v[u] * g[u];
#pragma unroll
        for (int u = 0; u < NB; u++) { c[u] = cn[u]; v[u] = vn[u]; }
    }
    if (full * NB < w) acc = slice_tail<NB>(col, val, beg, full * NB, w, lane, gather, acc);
    return acc;
}

// register budget: NB = 4 takes 42 (six 256-thread CTAs, or two of 768, per
// SM); NB = 8 takes 64 (four 256-thread CTAs) for twice the loads in flight;
// NB = 16 is NB = 8 software-pipelined (64 registers)
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
    const unsigned int nblk = nb + a.bar_extra;
    const int s_lo = rb / kSlice, s_hi = (re + kSlice - 1) / kSlice;
    const int gwarp = s_lo + (((int)blockIdx.x - b0) * (int)blockDim.x + (int)threadIdx.x) / 32;
    const int nwarps = (nb * (int)blockDim.x) >> 5;

    // ---- prologue: r = B x - A x, z = dinv r, p = 0 ----
    // With a predictor (delta: the previous solve's correction x - V of
    // this half step; with dext its linear extrapolation 2 delta - delta_prev,
    // stored by the previous solve) the iteration starts from x + pred
    // instead, r = B x - A (x + pred), while the stop test keeps the
    // reference's r0 = B x - A x; x itself is not touched before the barrier
    // (neighbours read it here).
    const bool pred = a.delta != nullptr;
    const bool lin = a.dext != nullptr;
    {
        double v[4] = {0.0, 0.0, 0.0, 0.0};
        for (int s = gwarp; s < s_hi; s += nwarps) {
            if (a.prefetch) prefetch_slice(a.slice_ptr, a.col, a.Aval, a.Bval, s + a.prefetch * nwarps, s_hi, lane);
            const int row = s * kSlice + lane;
            const int beg = a.slice_ptr[s], w = (a.slice_ptr[s + 1] - beg) / kSlice;
            R ax = R(0), bx = R(0), ad = R(0);
            slice_ab_sums<NB == 4 ? 2 : 4>(a.col, a.Aval, a.Bval, a.x, beg, w, lane, pred, [&](int c) {
                return lin ? a.dext[c] : a.delta[c];
            }, ax, bx, ad);
            if (row >= rb && row < re) {
                const R rref = bx - ax;
                const R r = pred ? rref - ad : rref;
                const R z = __ldg(a.dinv + row) * r;
                a.r[row] = r;
                reinterpret_cast<zp_t<R> *>(a.zp)[row] = zp_t<R>{z, R(0)};
                if (pred) a.vin[row] = a.x[row];
                v[0] += (double)r * (double)z;
                v[1] += (double)r * (double)r;
                v[2] += (double)bx * (double)bx;
                v[3] += (double)rref * (double)rref;
            }
        }
        block_reduce_store<4>(v, a.partial + 6 * G, G);      // slots [6G, 10G): the iterations use [0, 4G)
    }
    if (!grid_sync(bar, nblk)) return;
    double rz, rr_start, bb, rr0;
    {
        double t[4];
        grid_total<4>(a.partial + 6 * G, G, b0, nb, t);
        rz = t[0]; rr_start = t[1]; bb = t[2]; rr0 = t[3];
    }
    // ||r|| <= tol ||r0||, or the residual is at the resolution of b in the
    // vector type (FP32 cannot resolve a 1e-7 reduction of an r0 that is
    // itself rounding noise of B x - A x; in FP64 the floor is ~1e-16 ||b||)
    const double floor2 = a.floor_rel * a.floor_rel * bb;
    const double stop2 = fmax(a.tol * a.tol * rr0, floor2);
    double beta = 0.0;
    int it = 0;
    bool converged = (rr_start <= stop2);
    double rr_last = rr_start;
    zp_t<R> *zp = reinterpret_cast<zp_t<R> *>(a.zp);
    R *pn = a.p0;                             // p' of the own rows, phase A -> phase B
    while (!converged && it < a.maxit) {
        // ---- phase A: p' = z + beta p; q = A p' ----
        {
            double v[1] = {0.0};
            const R bR = (R)beta;
            for (int s = gwarp; s < s_hi; s += nwarps) {
                if (a.prefetch)
                    prefetch_slice<R>(a.slice_ptr, a.col, a.Aval, nullptr, s + a.prefetch * nwarps, s_hi, lane);
                const int row = s * kSlice + lane;
                const int beg = a.slice_ptr[s], w = (a.slice_ptr[s + 1] - beg) / kSlice;
                auto gat = [&](int c) { const zp_t<R> t = zp[c]; return pdir_z(t.x, bR, t.y); };
                R q;
                if constexpr (NB == 16) q = slice_row_sum_pipe<8>(a.col, a.Aval, beg, w, lane, gat);
                else q = slice_row_sum<NB>(a.col, a.Aval, beg, w, lane, gat);
                if (row >= rb && row < re) {
                    const zp_t<R> t = zp[row];
                    const R pi = pdir_z(t.x, bR, t.y);
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
        // ---- phase B: x += alpha p', r -= alpha q, z = dinv r ----
        // two of the warp's slices a pass: both slices' loads are issued
        // before either is updated (the rows are added to the dots in the
        // same order as one slice at a time)
        {
            double v[2] = {0.0, 0.0};
            const R aR = (R)alpha;
            for (int s = gwarp; s < s_hi; s += 2 * nwarps) {
                const int row = s * kSlice + lane, row2 = row + nwarps * kSlice;
                const bool on = row >= rb && row < re;
                const bool on2 = s + nwarps < s_hi && row2 >= rb && row2 < re;
                R pi = R(0), xi = R(0), ri = R(0), qi = R(0), di = R(0);
                R pi2 = R(0), xi2 = R(0), ri2 = R(0), qi2 = R(0), di2 = R(0);
                if (on) { pi = pn[row]; xi = a.x[row]; ri = a.r[row]; qi = a.q[row]; di = __ldg(a.dinv + row); }
                if (on2) { pi2 = pn[row2]; xi2 = a.x[row2]; ri2 = a.r[row2]; qi2 = a.q[row2]; di2 = __ldg(a.dinv + row2); }
                if (on) {
                    a.x[row] = xi + aR * pi;
                    const R r = ri - aR * qi;
                    a.r[row] = r;
                    const R z = di * r;
                    zp[row] = zp_t<R>{z, pi};
                    v[0] += (double)r * (double)z;
                    v[1] += (double)r * (double)r;
                }
                if (on2) {
                    a.x[row2] = xi2 + aR * pi2;
                    const R r = ri2 - aR * qi2;
                    a.r[row2] = r;
                    const R z = di2 * r;
                    zp[row2] = zp_t<R>{z, pi2};
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
        // a non-finite residual (a NaN or inf voltage upstream) cannot
        // recover: stop now, counted as a failed solve (every block sees the
        // same total and leaves at the same iteration)
        if (!isfinite(t[1])) break;
        beta = t[0] / rz;
        rz = t[0];
    }
    if (pred) {
        // the solution x + delta, and the correction this solve made, for the
        // next solve of this half step (own rows; every block is past the
        // prologue's reads of delta)
        for (int s = gwarp; s < s_hi; s += nwarps) {
            const int row = s * kSlice + lane;
            if (row >= rb && row < re) {
                const R d = a.delta[row];
                const R xf = a.x[row] + (lin ? a.dext[row] : d);
                a.x[row] = xf;
                const R dn = xf - a.vin[row];
                a.delta[row] = dn;
                if (lin) a.dext[row] = R(2) * dn - d;     // the next solve's start: 2 delta - delta_prev
            }
        }
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

// ---------------------------------------------------------------------------
// The same solve by the Chronopoulos-Gear recurrences: one grid barrier per
// iteration instead of two.  With z = dinv r and w = A z,
//   gamma = (r, z), delta = (z, w)                 (one reduction)
//   beta = gamma / gamma_old, alpha = gamma / (delta - beta gamma / alpha_old)
//   p = z + beta p, s = w + beta s, x += alpha p, r -= alpha s
// and the next w = A z is formed in the same pass: each neighbour's new z is
// recomputed from its old r, w, s (read from the other half of r, w, s's
// double buffers), with the owner's explicit fma sequence so both round alike.
// In exact arithmetic the iterates are those of k_cn_half; in floating point
// they differ at the rounding level (an option of the autotuner, not the
// default).
template <typename R>
__device__ __forceinline__ R cg1_snew(R w, R beta, R s) { return fma(beta, s, w); }
template <typename R>
__device__ __forceinline__ R cg1_rnew(R r, R alpha, R snew) { return fma(-alpha, snew, r); }

template <typename R, int NB>
__global__ void __launch_bounds__(NB == 4 ? 768 : 256, NB == 4 ? 2 : 4) k_cn_half_cg1(const CGArgs<R> a) {
    const int lane = threadIdx.x & 31;
    const int G = gridDim.x;
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
    const unsigned int nblk = nb + a.bar_extra;
    const int s_lo = rb / kSlice, s_hi = (re + kSlice - 1) / kSlice;
    const int gwarp = s_lo + (((int)blockIdx.x - b0) * (int)blockDim.x + (int)threadIdx.x) / 32;
    const int nwarps = (nb * (int)blockDim.x) >> 5;

    // ---- P1: r0 = B x - A x; p = 0, s_{-1} = 0 ----
    {
        double v[2] = {0.0, 0.0};
        for (int s = gwarp; s < s_hi; s += nwarps) {
            const int row = s * kSlice + lane;
            const int beg = a.slice_ptr[s], w = (a.slice_ptr[s + 1] - beg) / kSlice;
            R ax = R(0), bx = R(0), ad = R(0);
            slice_ab_sums<NB == 4 ? 2 : 4>(a.col, a.Aval, a.Bval, a.x, beg, w, lane, false, [](int) { return R(0); },
                                           ax, bx, ad);
            if (row >= rb && row < re) {
                const R r = bx - ax;
                a.r[row] = r;
                a.p0[row] = R(0);
                a.s1[row] = R(0);
                v[0] += (double)r * (double)r;
                v[1] += (double)bx * (double)bx;
            }
        }
        block_reduce_store<2>(v, a.partial, G);
    }
    if (!grid_sync(bar, nblk)) return;
    double rr0, bb;
    {
        double t[2];
        grid_total<2>(a.partial, G, b0, nb, t);
        rr0 = t[0]; bb = t[1];
    }
    const double stop2 = fmax(a.tol * a.tol * rr0, a.floor_rel * a.floor_rel * bb);
    bool converged = (rr0 <= stop2);
    double rr_last = rr0;
    int it = 0;
    double gamma = 0.0, delta = 0.0;
    // ---- P2: w0 = A z0, gamma0 = (r0, z0), delta0 = (z0, w0) ----
    if (!converged) {
        double v[2] = {0.0, 0.0};
        for (int s = gwarp; s < s_hi; s += nwarps) {
            const int row = s * kSlice + lane;
            const int beg = a.slice_ptr[s], w = (a.slice_ptr[s + 1] - beg) / kSlice;
            const R wv = slice_row_sum<NB>(a.col, a.Aval, beg, w, lane,
                                           [&](int c) { return __ldg(a.dinv + c) * ldcg(a.r + c); });
            if (row >= rb && row < re) {
                const R z = __ldg(a.dinv + row) * a.r[row];
                a.w0[row] = wv;
                v[0] += (double)a.r[row] * (double)z;
                v[1] += (double)z * (double)wv;
            }
        }
        // partial slots: P1 [0, 2G), P2 [9G, 11G), iterations alternate
        // [3G, 6G) and [6G, 9G): consecutive phases never share a slot
        block_reduce_store<2>(v, a.partial + 9 * G, G);
        if (!grid_sync(bar, nblk)) return;
        double t[2];
        grid_total<2>(a.partial + 9 * G, G, b0, nb, t);
        gamma = t[0]; delta = t[1];
    }
    double alpha = (delta > 0.0) ? gamma / delta : 0.0, beta = 0.0;
    if (!(delta > 0.0)) converged = true;       // A z0 = 0: nothing left to solve
    int cur = 0;
    while (!converged && it < a.maxit) {
        const R aR = (R)alpha, bR = (R)beta;
        // the double buffers by selects (no local-memory pointer arrays)
        const R *rc = cur ? a.r1 : a.r, *wc = cur ? a.w1 : a.w0, *sp = cur ? a.s0 : a.s1;
        R *rn = cur ? a.r : a.r1, *wn = cur ? a.w0 : a.w1, *sc = cur ? a.s1 : a.s0;
        double v[3] = {0.0, 0.0, 0.0};
        for (int s = gwarp; s < s_hi; s += nwarps) {
            const int row = s * kSlice + lane;
            const int beg = a.slice_ptr[s], w = (a.slice_ptr[s + 1] - beg) / kSlice;
            // w_{k+1} = A z_{k+1}, z_{k+1} of the neighbours rebuilt from old r, w, s
            const R wv = slice_row_sum<NB>(a.col, a.Aval, beg, w, lane, [&](int c) {
                const R snew = cg1_snew(ldcg(wc + c), bR, ldcg(sp + c));
                return __ldg(a.dinv + c) * cg1_rnew(ldcg(rc + c), aR, snew);
            });
            if (row >= rb && row < re) {
                const R d = __ldg(a.dinv + row);
                const R rk = rc[row];
                const R p = fma(bR, a.p0[row], d * rk);
                const R snew = cg1_snew(wc[row], bR, sp[row]);
                const R rnew = cg1_rnew(rk, aR, snew);
                const R znew = d * rnew;
                a.p0[row] = p;
                sc[row] = snew;
                a.x[row] += aR * p;
                rn[row] = rnew;
                wn[row] = wv;
                v[0] += (double)rnew * (double)znew;
                v[1] += (double)znew * (double)wv;
                v[2] += (double)rnew * (double)rnew;
            }
        }
        block_reduce_store<3>(v, a.partial + 3 * (cur + 1) * G, G);   // alternate slots
        if (!grid_sync(bar, nblk)) return;
        double t[3];
        grid_total<3>(a.partial + 3 * (cur + 1) * G, G, b0, nb, t);
        it++;
        rr_last = t[2];
        converged = (t[2] <= stop2);
        if (!isfinite(t[2])) { converged = false; break; }   // as in k_cn_half
        const double gnew = t[0];
        beta = gnew / gamma;
        const double den = t[1] - beta * gnew / alpha;
        if (!(den > 0.0)) converged = true;        // breakdown at the rounding floor
        alpha = gnew / den;
        gamma = gnew;
        cur = 1 - cur;
    }
    // the solution is in x; r's current buffer is left wherever it is
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

// ---------------------------------------------------------------------------
// k_cn_half_staged: the two-reduction solve of k_cn_half (same recurrences,
// same order of additions, so the same bits on the same grid) with the matrix
// stream of phase A taken off the warps' critical path.  A warp's slices are
// cut into units of kUnitCols slice columns: the column indices and A values
// of one slice's columns k .. k+7 (8 x 128 bytes of indices, 8 x 32 x
// sizeof(R) bytes of values).  The warp copies the units into a ring of
// shared memory with per-thread asynchronous copies (cp.async.cg: 16 bytes
// each, L2 only, evict-first, so the matrix streams through L2 while the
// gathered vectors stay there), `depth` units ahead of the one it gathers
// for.  The DRAM latency of the index -> gather chain is then hidden behind
// the gathers of the units before it, and the loads in flight occupy ring
// slots instead of registers.  The stream runs on past the end of a sweep
// into the next iteration's first units (the matrix does not change), under
// phase B and the grid barriers.  No wait in this kernel spins:
// cp.async.wait_group is the hardware's wait for the thread's own copies, and
// every exit path waits for all of them before the CTA leaves.
constexpr int kUnitCols = 8;

__host__ __device__ inline size_t unit_bytes(int rsize) { return (size_t)kUnitCols * kSlice * (4 + (size_t)rsize); }
// dynamic shared memory of a CTA of `block` threads, `depth` units in flight per warp
__host__ __device__ inline size_t stage_smem_bytes(int block, int depth, int rsize) {
    return (size_t)(block / 32) * (size_t)(depth + 1) * unit_bytes(rsize);
}

__device__ __forceinline__ uint32_t cg_smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t l2_evict_first_policy() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

// one 16-byte global -> shared copy, cached in L2 only (both addresses
// 16-byte aligned: every unit starts on a 128-byte boundary of the SELL
// arrays and of the ring)
__device__ __forceinline__ void cp16(void *dst, const void *src, uint64_t pol) {
    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(cg_smem_u32(dst)), "l"(src),
                 "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// this thread's copies of every unit but the newest depth - 1 have landed
__device__ __forceinline__ void unit_wait(int depth) {
    switch (depth) {
        case 1: cp_wait<0>(); break;
        case 2: cp_wait<1>(); break;
        case 3: cp_wait<2>(); break;
        default: cp_wait<3>(); break;
    }
}

template <typename R>
struct UnitRing {
    int *idx;          // slot k's indices at idx + k * kUnitCols * kSlice
    R *val;            // slot k's values at val + k * kUnitCols * kSlice
    int slots, depth;  // slots = depth + 1
    int L;             // this warp's slices per sweep (0: nothing to stage)
    int j, k, beg, w;  // producer cursor: slice j of the warp, its column k, start, width
    int issued;        // units issued so far
    uint64_t pol;
};

// issue the unit under the cursor into the ring slot of its position and
// advance the cursor (the next unit of the slice, or the next slice,
// wrapping to the warp's first slice: the next sweep).  Every lane commits
// one copy group per call, empty or not, so the group counts stay uniform.
template <typename R>
__device__ __forceinline__ void unit_issue(UnitRing<R> &q, const CGArgs<R> &a, int gwarp, int nwarps, int lane) {
    if (q.L > 0) {
        const int slot = q.issued % q.slots;
        const int nc = min(kUnitCols, q.w - q.k);
        int *di = q.idx + slot * (kUnitCols * kSlice);
        R *dv = q.val + slot * (kUnitCols * kSlice);
        const int *si = a.col + q.beg + q.k * kSlice;
        const R *sv = a.Aval + q.beg + q.k * kSlice;
        // indices: column u, 16-byte piece p is chunk c = 8 u + p
#pragma unroll
        for (int t = 0; t < 2; t++) {
            const int c = lane + 32 * t;
            if ((c >> 3) < nc) cp16(di + 4 * c, si + 4 * c, q.pol);
        }
        // values: VPC chunks of VE values per column
        constexpr int VPC = kSlice * (int)sizeof(R) / 16, VE = 16 / (int)sizeof(R);
#pragma unroll
        for (int t = 0; t < VPC * kUnitCols / 32; t++) {
            const int c = lane + 32 * t;
            if (c / VPC < nc) cp16(dv + VE * c, sv + VE * c, q.pol);
        }
        q.k += kUnitCols;
        while (q.k >= q.w) {               // ends: some slice of the warp has columns (q.L > 0)
            q.j = q.j + 1 == q.L ? 0 : q.j + 1;
            const int s = gwarp + q.j * nwarps;
            q.beg = __ldg(a.slice_ptr + s);
            q.w = (__ldg(a.slice_ptr + s + 1) - q.beg) / kSlice;
            q.k = 0;
        }
    }
    q.issued++;
    cp_commit();
}

template <typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 8 ? 3 : 4) k_cn_half_staged(const CGArgs<R> a) {
    extern __shared__ __align__(128) unsigned char cg_sm[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int G = gridDim.x;
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
    const unsigned int nblk = nb + a.bar_extra;
    const int s_lo = rb / kSlice, s_hi = (re + kSlice - 1) / kSlice;
    const int gwarp = s_lo + (((int)blockIdx.x - b0) * (int)blockDim.x + (int)threadIdx.x) / 32;
    const int nwarps = (nb * (int)blockDim.x) >> 5;

    // this warp's ring: slots x unit of indices, then slots x unit of values
    UnitRing<R> q;
    {
        q.depth = a.depth;
        q.slots = a.depth + 1;
        unsigned char *base = cg_sm + (size_t)wib * q.slots * unit_bytes((int)sizeof(R));
        q.idx = reinterpret_cast<int *>(base);
        q.val = reinterpret_cast<R *>(base + (size_t)q.slots * kUnitCols * kSlice * 4);
        q.L = gwarp < s_hi ? (s_hi - gwarp + nwarps - 1) / nwarps : 0;
        int cols = 0;
        for (int j = 0; j < q.L; j++) {
            const int s = gwarp + j * nwarps;
            cols += __ldg(a.slice_ptr + s + 1) - __ldg(a.slice_ptr + s);
        }
        if (cols == 0) q.L = 0;
        q.j = 0;
        q.k = 0;
        q.beg = q.L > 0 ? __ldg(a.slice_ptr + gwarp) : 0;
        q.w = q.L > 0 ? (__ldg(a.slice_ptr + gwarp + 1) - q.beg) / kSlice : 0;
        while (q.L > 0 && q.w == 0) {      // ends: some slice has columns
            q.j++;
            const int s = gwarp + q.j * nwarps;
            q.beg = __ldg(a.slice_ptr + s);
            q.w = (__ldg(a.slice_ptr + s + 1) - q.beg) / kSlice;
        }
        q.issued = 0;
        q.pol = l2_evict_first_policy();
    }
    // the first units start streaming under the prologue
    for (int d = 0; d < q.depth; d++) unit_issue(q, a, gwarp, nwarps, lane);
    int cons = 0;                             // units consumed so far

    // ---- prologue: as k_cn_half ----
    const bool pred = a.delta != nullptr;
    const bool lin = a.dext != nullptr;
    {
        double v[4] = {0.0, 0.0, 0.0, 0.0};
        for (int s = gwarp; s < s_hi; s += nwarps) {
            const int row = s * kSlice + lane;
            const int beg = a.slice_ptr[s], w = (a.slice_ptr[s + 1] - beg) / kSlice;
            R ax = R(0), bx = R(0), ad = R(0);
            slice_ab_sums<4>(a.col, a.Aval, a.Bval, a.x, beg, w, lane, pred, [&](int c) {
                return lin ? a.dext[c] : a.delta[c];
            }, ax, bx, ad);
            if (row >= rb && row < re) {
                const R rref = bx - ax;
                const R r = pred ? rref - ad : rref;
                const R z = __ldg(a.dinv + row) * r;
                a.r[row] = r;
                reinterpret_cast<zp_t<R> *>(a.zp)[row] = zp_t<R>{z, R(0)};
                if (pred) a.vin[row] = a.x[row];
                v[0] += (double)r * (double)z;
                v[1] += (double)r * (double)r;
                v[2] += (double)bx * (double)bx;
                v[3] += (double)rref * (double)rref;
            }
        }
        block_reduce_store<4>(v, a.partial + 6 * G, G);
    }
    if (!grid_sync(bar, nblk)) { cp_wait_all(); return; }
    double rz, rr_start, bb, rr0;
    {
        double t[4];
        grid_total<4>(a.partial + 6 * G, G, b0, nb, t);
        rz = t[0]; rr_start = t[1]; bb = t[2]; rr0 = t[3];
    }
    const double floor2 = a.floor_rel * a.floor_rel * bb;
    const double stop2 = fmax(a.tol * a.tol * rr0, floor2);
    double beta = 0.0;
    int it = 0;
    bool converged = (rr_start <= stop2);
    double rr_last = rr_start;
    zp_t<R> *zp = reinterpret_cast<zp_t<R> *>(a.zp);
    R *pn = a.p0;                             // p' of the own rows, phase A -> phase B
    while (!converged && it < a.maxit) {
        // ---- phase A: q = A p', p' = z + beta p, the units from the ring ----
        {
            double v[1] = {0.0};
            const R bR = (R)beta;
            for (int s = gwarp; s < s_hi; s += nwarps) {
                const int row = s * kSlice + lane;
                const int beg = __ldg(a.slice_ptr + s), w = (__ldg(a.slice_ptr + s + 1) - beg) / kSlice;
                R qv = R(0);
                for (int k = 0; k < w; k += kUnitCols, cons++) {
                    unit_wait(q.depth);
                    __syncwarp();                 // the unit is visible to every lane, and every
                                                  // lane is done with the slot refilled next
                    unit_issue(q, a, gwarp, nwarps, lane);
                    const int off = (cons % q.slots) * (kUnitCols * kSlice) + lane;
                    const int *ci = q.idx + off;
                    const R *cv = q.val + off;
                    const int nc = min(kUnitCols, w - k);
                    int c[kUnitCols];
                    R g[kUnitCols];
#pragma unroll
                    for (int u = 0; u < kUnitCols; u++)
                        if (u < nc) c[u] = ci[u * kSlice];
#pragma unroll
                    for (int u = 0; u < kUnitCols; u++)
                        if (u < nc) {
                            const zp_t<R> t = zp[c[u]];
                            g[u] = pdir_z(t.x, bR, t.y);
                        }
#pragma unroll
                    for (int u = 0; u < kUnitCols; u++)
                        if (u < nc) qv += cv[u * kSlice] * g[u];
                }
                if (row >= rb && row < re) {
                    const zp_t<R> t = zp[row];
                    const R pi = pdir_z(t.x, bR, t.y);
                    pn[row] = pi;
                    a.q[row] = qv;
                    v[0] += (double)pi * (double)qv;
                }
            }
            block_reduce_store<1>(v, a.partial + 3 * G, G);
        }
        if (!grid_sync(bar, nblk)) { cp_wait_all(); return; }
        double pq;
        {
            double t[1];
            grid_total<1>(a.partial + 3 * G, G, b0, nb, t);
            pq = t[0];
        }
        const double alpha = rz / pq;
        // ---- phase B: as k_cn_half ----
        {
            double v[2] = {0.0, 0.0};
            const R aR = (R)alpha;
            for (int s = gwarp; s < s_hi; s += 2 * nwarps) {
                const int row = s * kSlice + lane, row2 = row + nwarps * kSlice;
                const bool on = row >= rb && row < re;
                const bool on2 = s + nwarps < s_hi && row2 >= rb && row2 < re;
                R pi = R(0), xi = R(0), ri = R(0), qi = R(0), di = R(0);
                R pi2 = R(0), xi2 = R(0), ri2 = R(0), qi2 = R(0), di2 = R(0);
                if (on) { pi = pn[row]; xi = a.x[row]; ri = a.r[row]; qi = a.q[row]; di = __ldg(a.dinv + row); }
                if (on2) { pi2 = pn[row2]; xi2 = a.x[row2]; ri2 = a.r[row2]; qi2 = a.q[row2]; di2 = __ldg(a.dinv + row2); }
                if (on) {
                    a.x[row] = xi + aR * pi;
                    const R r = ri - aR * qi;
                    a.r[row] = r;
                    const R z = di * r;
                    zp[row] = zp_t<R>{z, pi};
                    v[0] += (double)r * (double)z;
                    v[1] += (double)r * (double)r;
                }
                if (on2) {
                    a.x[row2] = xi2 + aR * pi2;
                    const R r = ri2 - aR * qi2;
                    a.r[row2] = r;
                    const R z = di2 * r;
                    zp[row2] = zp_t<R>{z, pi2};
                    v[0] += (double)r * (double)z;
                    v[1] += (double)r * (double)r;
                }
            }
            block_reduce_store<2>(v, a.partial, G);
        }
        if (!grid_sync(bar, nblk)) { cp_wait_all(); return; }
        double t[2];
        grid_total<2>(a.partial, G, b0, nb, t);
        it++;
        rr_last = t[1];
        converged = (t[1] <= stop2);
        if (!isfinite(t[1])) break;
        beta = t[0] / rz;
        rz = t[0];
    }
    cp_wait_all();                            // the units that ran ahead into the next sweep
    if (pred) {
        for (int s = gwarp; s < s_hi; s += nwarps) {
            const int row = s * kSlice + lane;
            if (row >= rb && row < re) {
                const R d = a.delta[row];
                const R xf = a.x[row] + (lin ? a.dext[row] : d);
                a.x[row] = xf;
                const R dn = xf - a.vin[row];
                a.delta[row] = dn;
                if (lin) a.dext[row] = R(2) * dn - d;     // the next solve's start: 2 delta - delta_prev
            }
        }
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

// the kernel of a (gather width, variant) choice and its dynamic shared
// memory; cg_batch kStagedBatch selects k_cn_half_staged with `depth` units
// in flight per warp (1 .. kStageMaxDepth)
// (set_attr: allow the staged kernel the largest ring any handle can ask
// for -- 256 threads, kStageMaxDepth units -- once, from the planning path,
// never during a stream capture; the attribute only caps the request)
template <typename R>
static int cg_kernel(int block, int batch, int variant, int depth, const void **fn, size_t *smem,
                     bool set_attr) {
    *smem = 0;
    if (batch == kStagedBatch) {
        if (variant != 0) { set_error("the staged CG runs the two-reduction recurrences only"); return EP_ERR_ARG; }
        if (depth < 1 || depth > kStageMaxDepth) {
            set_error("staged CG: %d units in flight, not 1..%d", depth, kStageMaxDepth);
            return EP_ERR_ARG;
        }
        *fn = (const void *)k_cn_half_staged<R>;
        *smem = stage_smem_bytes(block, depth, (int)sizeof(R));
        if (set_attr)
            EP_CUDA(cudaFuncSetAttribute(*fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)stage_smem_bytes(256, kStageMaxDepth, (int)sizeof(R))));
        return EP_OK;
    }
    *fn = variant == 1 ? (batch >= 8 ? (const void *)k_cn_half_cg1<R, 8> : (const void *)k_cn_half_cg1<R, 4>)
          : batch == 8 ? (const void *)k_cn_half<R, 8>
          : batch == 16 ? (const void *)k_cn_half<R, 16>
                        : (const void *)k_cn_half<R, 4>;
    return EP_OK;
}

template <typename R>
int cg_max_per_sm(int block, int *per, int batch, int variant, int depth) {
    const void *fn = nullptr;
    size_t smem = 0;
    int rc = cg_kernel<R>(block, batch, variant, depth, &fn, &smem, true);
    if (rc) return rc;
    cudaFuncAttributes fa;
    EP_CUDA(cudaFuncGetAttributes(&fa, fn));
    if (block > fa.maxThreadsPerBlock) {
        set_error("CG gather width %d takes at most %d threads per CTA (asked %d)", batch, fa.maxThreadsPerBlock, block);
        return EP_ERR_ARG;
    }
    EP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per, fn, block, smem));
    if (*per < 1) { set_error("CG kernel cannot be resident with %d threads per CTA", block); return EP_ERR_CUDA; }
    return EP_OK;
}

template <typename R>
int cg_grid_size(int block, int *grid, int per_sm, int batch, int variant, int depth) {
    int dev = 0, nsm = 0, per = 0;
    EP_CUDA(cudaGetDevice(&dev));
    EP_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    int rc = cg_max_per_sm<R>(block, &per, batch, variant, depth);
    if (rc) return rc;
    if (per_sm > 0 && per_sm < per) per = per_sm;
    *grid = nsm * per;
    return EP_OK;
}

template <typename R>
int launch_cg(const CGArgs<R> &a, int grid, int block, cudaStream_t s, int batch, int variant) {
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
    if (batch == kStagedBatch) {
        const void *fn = nullptr;
        size_t smem = 0;
        int rc = cg_kernel<R>(block, batch, variant, a.depth, &fn, &smem, false);
        if (rc) return rc;
        cfg.dynamicSmemBytes = smem;
        EP_CUDA(cudaLaunchKernelEx(&cfg, k_cn_half_staged<R>, a));
    } else if (variant == 1) {
        if (!a.r1 || !a.w0 || !a.w1 || !a.s0 || !a.s1) { set_error("single-reduction CG needs its vectors"); return EP_ERR_ARG; }
        if (batch >= 8) EP_CUDA(cudaLaunchKernelEx(&cfg, k_cn_half_cg1<R, 8>, a));
        else EP_CUDA(cudaLaunchKernelEx(&cfg, k_cn_half_cg1<R, 4>, a));
    } else if (batch == 8) {
        EP_CUDA(cudaLaunchKernelEx(&cfg, k_cn_half<R, 8>, a));
    } else if (batch == 16) {
        EP_CUDA(cudaLaunchKernelEx(&cfg, k_cn_half<R, 16>, a));
    } else {
        EP_CUDA(cudaLaunchKernelEx(&cfg, k_cn_half<R, 4>, a));
    }
    return EP_OK;
}

template int launch_cg<float>(const CGArgs<float> &, int, int, cudaStream_t, int, int);
template int launch_cg<double>(const CGArgs<double> &, int, int, cudaStream_t, int, int);
template int cg_grid_size<float>(int, int *, int, int, int, int);
template int cg_grid_size<double>(int, int *, int, int, int, int);
template int cg_max_per_sm<float>(int, int *, int, int, int);
template int cg_max_per_sm<double>(int, int *, int, int, int);

// ---------------------------------------------------------------------------
// One forward-Euler diffusion sub-step of the explicit scheme
// (EP_ExplicitSolver::Solve, Solvers/EP_ExplicitSolver.cc:54-83):
// out_i = V_i + h (D V)_i / C_L,i with D = -K in the SELL operator.
template <typename R>
__global__ void __launch_bounds__(256) k_explicit(int n, int nslices, const int *__restrict__ slice_ptr,
                                                  const int *__restrict__ col, const R *__restrict__ Dval,
                                                  const R *__restrict__ cl, const R *__restrict__ V, R *out, R h) {
    const int lane = threadIdx.x & 31;
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int s = gwarp; s < nslices; s += nwarps) {
        const int row = s * kSlice + lane;
        const int beg = slice_ptr[s], w = (slice_ptr[s + 1] - beg) / kSlice;
        const R d = slice_row_sum<4>(col, Dval, beg, w, lane, [&](int c) { return __ldg(V + c); });
        if (row < n) out[row] = V[row] + h * d / cl[row];
    }
}

template <typename R>
int launch_explicit(int n, int nslices, const int *slice_ptr, const int *col, const R *Dval, const R *cl, R *V,
                    R *tmp, double h, cudaStream_t s) {
    int dev = 0, nsm = 148;
    EP_CUDA(cudaGetDevice(&dev));
    EP_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int grid = std::max(1, std::min(8 * nsm, (nslices + 7) / 8));
    k_explicit<R><<<grid, 256, 0, s>>>(n, nslices, slice_ptr, col, Dval, cl, V, tmp, (R)h);
    EP_CUDA(cudaGetLastError());
    EP_CUDA(cudaMemcpyAsync(V, tmp, sizeof(R) * (size_t)n, cudaMemcpyDeviceToDevice, s));
    return EP_OK;
}

template int launch_explicit<float>(int, int, const int *, const int *, const float *, const float *, float *,
                                     float *, double, cudaStream_t);
template int launch_explicit<double>(int, int, const int *, const int *, const double *, const double *, double *,
                                      double *, double, cudaStream_t);

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
