// surrogate.cu -- BF16 tensor-core (tcgen05) inference of the learned ionic
// step, one persistent CTA per half SM.
//
// Per tile of 128 nodes (one node per thread = one TMEM lane):
//   1. features of the node (V, 18 states, I_stim, G_Ks, G_to, s-gate) ->
//      normalised -> BF16 row of the A operand in shared memory;
//   2. four layers: one elected thread issues tcgen05.mma (kind::f16, BF16 x
//      BF16 -> FP32 in TMEM, M = 128, N = 128 or 32, K = 16 per instruction)
//      with A = activations and B = the layer's weights, both resident in
//      shared memory as no-swizzle K-major core matrices, then
//      tcgen05.commit arrives on an mbarrier;
//   3. every warp reads its 32 TMEM lanes back (tcgen05.ld 32x32b), adds the
//      bias, applies tanh.approx and writes the next BF16 A operand;
//   4. the output layer's 19 values are de-normalised and added to the
//      node's state; nodes outside the training envelope (input box, fast
//      Na-gate product m^3 h, an active stimulus) are appended to a fallback
//      list that the plain FP32 kernel then runs.
// The weights (80 KB) are loaded once per CTA.  Shared memory 112 KB and
// 256 TMEM columns per CTA, so two CTAs share an SM and one's epilogue
// overlaps the other's MMAs.  Every mbarrier wait is bounded; on timeout the
// CTA records the error, frees its TMEM and leaves.
#include <cuda_bf16.h>

#include "surrogate.cuh"
#include "tt.cuh"

namespace ep {

constexpr int OFF_W1 = 0;
constexpr int OFF_W2 = OFF_W1 + SG_W1 * 2;
constexpr int OFF_W3 = OFF_W2 + SG_W2 * 2;
constexpr int OFF_W4 = OFF_W3 + SG_W3 * 2;
constexpr int OFF_A = OFF_W4 + SG_W4 * 2;                 // 128 x 128 bf16
constexpr int OFF_MISC = OFF_A + SG_M * SG_H * 2;
constexpr int OFF_FLAGS = OFF_MISC + 64;                 // 2 x 128 envelope flags
constexpr int SG_SMEM = OFF_FLAGS + 2 * SG_M;
constexpr uint32_t SG_TMEM_COLS = 256;

size_t surrogate_smem_bytes() { return SG_SMEM; }

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// UMMA shared-memory descriptor: no swizzle, K-major; lbo/sbo in bytes
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: BF16 x BF16 -> F32, both K-major
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t *holder, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(holder)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void umma_bf16(uint32_t d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]),
          "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
          "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float tanh_fast(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t *>(&v);
}

// issue one layer: D[128 x N] = A[128 x K] W^T, W = [N x K]; thread 0 only
__device__ __forceinline__ void issue_layer(uint32_t d, uint32_t sA, uint32_t sW, int K, int N, uint64_t *bar) {
    const uint32_t sbo = (uint32_t)(K / 8) * 128u;
    const uint32_t id = idesc_bf16(SG_M, N);
    for (int kk = 0; kk < K / 16; kk++) {
        const uint32_t off = (uint32_t)kk * 256u;          // two 128-byte core matrices along K
        umma_bf16(d, umma_desc(sA + off, 128u, sbo), umma_desc(sW + off, 128u, sbo), id, kk > 0 ? 1u : 0u);
    }
    umma_commit(bar);
}

// block-uniform bounded wait for the next commit of this CTA: at most
// `polls` try-waits (0: kMbarPolls)
constexpr unsigned int kMbarPolls = 1u << 22;
__device__ __forceinline__ bool wait_commit(uint64_t *bar, uint32_t &phase, unsigned int *err, unsigned int polls) {
    bool ok = false;
    const unsigned int lim = polls ? polls : kMbarPolls;
    for (unsigned int it = 0; it < lim; it++)
        if (mbar_try_wait(bar, phase)) { ok = true; break; }
    phase ^= 1u;
    const int bad = __syncthreads_or(ok ? 0 : 1);
    if (bad) {
        if (threadIdx.x == 0) atomicExch(err, 1u);
        return false;
    }
    tc_fence_after();
    return true;
}

// hidden-layer epilogue: TMEM -> +bias -> tanh -> BF16 A row (K = 128
// layout).  Row r's 128 columns are split between the two warps that share
// its TMEM lane quarter: half h takes columns [64 h, 64 h + 64).
__device__ __forceinline__ void hidden_epilogue(uint32_t tmem_row, const float *__restrict__ bias, unsigned char *A,
                                                int r, int half) {
#pragma unroll 1
    for (int qq = 0; qq < 2; qq++) {
        const int q = 2 * half + qq;
        uint32_t v[32];
        tmem_ld32(tmem_row + 32u * q, v);
        uint32_t w[16];
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const float a0 = tanh_fast(__uint_as_float(v[2 * j]) + __ldg(bias + 32 * q + 2 * j));
            const float a1 = tanh_fast(__uint_as_float(v[2 * j + 1]) + __ldg(bias + 32 * q + 2 * j + 1));
            w[j] = pack_bf16(a0, a1);
        }
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int chunk = 4 * q + c;
            uint4 *dst = (uint4 *)(A + ((r >> 3) * (SG_H / 8) + chunk) * 128 + (r & 7) * 16);
            *dst = make_uint4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]);
        }
    }
}

// Ask L2 for the 128-byte lines that build_row will read for tile nt (V,
// the 18 stored states, G_Ks scale, stimulus heads, node types), one line
// per thread t of the CTA's second half, so the row build at the end of the
// current tile finds them in L2.  A hint only; every address is below n.
__device__ __forceinline__ void prefetch_rows(const SurrogateArgs &a, int nt, int t) {
    const int base = nt * SG_M;
    const void *p = nullptr;
    if (t < 80) {
        const int arr = t >> 2, off = base + 32 * (t & 3);
        if (off < a.n) {
            if (arr == 0) p = a.V + off;
            else if (arr <= 18) p = a.S + (size_t)(arr - 1) * a.pitch + off;
            else if (a.gks) p = a.gks + off;
        }
    } else if (t < 84) {
        const int off = base + 32 * (t - 80);
        if (a.stim_head && off < a.n) p = a.stim_head + off;
    } else if (t == 84) {
        if (a.type && base < a.n) p = a.type + base;
    }
    if (p) asm volatile("prefetch.L2 [%0];" ::"l"(p));
}

// One node's input row: features (V, 18 states, I_stim, G_Ks, G_to, s-gate),
// logarithms of the wide-range ones, normalisation, BF16 row of A (K = 32
// layout); returns whether the node is inside the training envelope.
__device__ __forceinline__ bool build_row(const SurrogateArgs &a, const SurrogateAux *aux, long long step, bool raw,
                                          int i, bool valid, int row, unsigned char *A) {
    float xn[SG_KIN];
#pragma unroll
    for (int k = 0; k < SG_KIN; k++) xn[k] = 0.f;
    bool inside = false;
    if (valid && raw) {
#pragma unroll
        for (int k = 0; k < SG_KIN; k++) xn[k] = a.rawX[(size_t)i * SG_KIN + k];
    } else if (valid) {
        float x[SG_NF];
        x[0] = a.V[i];
#pragma unroll
        for (int k = 0; k < 18; k++) x[k + 1] = a.S[(size_t)k * a.pitch + i];
        const int ty = a.type ? a.type[i] : 0;
        const float *c = a.consts + (size_t)ty * a.nconst;
        float istim = 0.f;
        if (a.stim_head) {
            int k = a.stim_head[i];
            long long best = -1;
            while (k >= 0) {
                const long long on = a.stim_on[k], off = a.stim_off[k];
                if (step >= on && step < off && on > best) { best = on; istim = a.stim_amp[k]; }
                k = a.stim_next[k];
            }
        }
        x[19] = istim / (a.Cm * a.Xi);
        x[20] = c[15] * (a.gks ? a.gks[i] : 1.f);
        x[21] = c[20];
        x[22] = c[53];
        inside = (istim == 0.f);
        const float m = x[7], h = x[8];
        inside = inside && (m * m * m * h <= aux->nah_max);
        const unsigned int lm = aux->log_mask;
#pragma unroll
        for (int k = 0; k < SG_NF; k++) {
            // quantities spanning decades enter as logarithms
            const float xt = ((lm >> k) & 1u) ? __logf(fmaxf(x[k], 1e-30f)) : x[k];
            inside = inside && (xt >= aux->env_lo[k]) && (xt <= aux->env_hi[k]);
            xn[k] = (xt - aux->in_mean[k]) * aux->in_rstd[k];
        }
    }
    uint32_t w[16];
#pragma unroll
    for (int j = 0; j < 16; j++) w[j] = pack_bf16(xn[2 * j], xn[2 * j + 1]);
#pragma unroll
    for (int cch = 0; cch < 4; cch++) {
        uint4 *dst = (uint4 *)(A + ((row >> 3) * (SG_KIN / 8) + cch) * 128 + (row & 7) * 16);
        *dst = make_uint4(w[4 * cch], w[4 * cch + 1], w[4 * cch + 2], w[4 * cch + 3]);
    }
    return inside;
}

// One node's share of the output stage: the network's de-normalised
// changes applied (or, in the hybrid form, its six concentrations handed to
// k_hybrid), and the nodes outside the envelope or with an output outside
// its training range appended to the fallback list.  yv: the node's 32
// output-layer accumulators (bias not yet added).
__device__ __forceinline__ void output_node(const SurrogateArgs &a, const SurrogateAux *aux, int i, bool valid,
                                            bool raw, bool inside, const uint32_t (&yv)[32], double t0,
                                            unsigned int &my_fb) {
    if (valid && raw) {
#pragma unroll
        for (int j = 0; j < SG_NOUT; j++) a.rawY[(size_t)i * SG_NOUT + j] = __uint_as_float(yv[j]) + aux->b4[j];
    } else if (valid) {
        // the six concentrations the hybrid form replaces, loaded before
        // any store of this node (the stores below could alias them for
        // the compiler, which would otherwise serialise load and store)
        const int cslot[6] = {0, 1, 2, 9, 16, 17};
        float xs[6];
        if (aux->v_update == 2) {
#pragma unroll
            for (int j = 0; j < 6; j++) xs[j] = a.S[(size_t)cslot[j] * a.pitch + i];
        }
        // de-normalise; a used output outside the range seen in training
        // sends the node to the plain model as well
        float d[SG_NY];
        bool out_ok = inside;
#pragma unroll
        for (int j = 0; j < SG_NY; j++) {
            // only the outputs the update reads (out_mask: the six concentrations
            // in the hybrid form, every output otherwise) are range-checked and
            // mapped back; the others are never read
            d[j] = 0.f;
            if ((aux->out_mask >> j) & 1u) {
                const float u = (__uint_as_float(yv[j]) + aux->b4[j]) * aux->out_std[j] + aux->out_mean[j];
                out_ok = out_ok && (u >= aux->out_lo[j]) && (u <= aux->out_hi[j]);
                const float sc = aux->out_scale[j];
                d[j] = sc > 0.f ? sc * sinhf(fminf(fmaxf(u, -80.f), 80.f)) : u;
            }
        }
        const unsigned int lm = aux->log_mask;
        if (aux->v_update == 2) a.take[i] = out_ok ? 1 : 0;
        if (!out_ok) {
            const int slot = atomicAdd(a.fallback_count, 1);
            a.fallback_list[slot] = i;
            my_fb++;
        } else if (aux->v_update == 2) {
            // the new concentrations; k_hybrid advances gates and V
#pragma unroll
            for (int j = 0; j < 6; j++) {
                const int q = cslot[j];
                a.pred[(size_t)j * a.pitch + i] =
                    ((lm >> (q + 1)) & 1u) ? xs[j] * __expf(d[q + 1]) : xs[j] + d[q + 1];
            }
        } else {
            // every quantity from the network (all loads before the stores)
            float xk[18];
#pragma unroll
            for (int k = 0; k < 18; k++) xk[k] = a.S[(size_t)k * a.pitch + i];
#pragma unroll
            for (int k = 0; k < 18; k++) {
                // log-scaled states are updated multiplicatively: x' = x exp(d)
                a.S[(size_t)k * a.pitch + i] = ((lm >> (k + 1)) & 1u) ? xk[k] * __expf(d[k + 1]) : xk[k] + d[k + 1];
            }
            const float V0 = a.V[i], V1 = V0 + d[0];
            a.V[i] = V1;
            if (a.track) {
                Track tr = a.track[i];
                if (tr.t_rep < 0.f) {
                    bool dirty = false;
                    track_interval(tr, dirty, V0, V1, t0, (float)a.t_per_step, a.act_thr);
                    if (dirty) a.track[i] = tr;
                }
            }
        }
    }
}

// The network over tiles of 128 nodes, 256 threads per CTA.  Threads
// 0..127 own one node each (features, the output layer, the envelope
// decision); all eight warps share the hidden-layer epilogues (warp w reads
// TMEM lane quarter w % 4, column half w / 4).
__global__ void __launch_bounds__(SG_THREADS, 2) k_surrogate(const SurrogateArgs a) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5;
    const int row = tid & (SG_M - 1), half = tid >> 7;
    const bool owner = half == 0;                 // warp-uniform
    uint64_t *bar = (uint64_t *)(smem + OFF_MISC);
    uint32_t *holder = (uint32_t *)(smem + OFF_MISC + 16);
    unsigned char *A = smem + OFF_A;
    const SurrogateAux *aux = a.aux;

    // weights: global image -> shared (already in core-matrix order)
    {
        const uint4 *src = (const uint4 *)a.wimg;
        uint4 *dst = (uint4 *)smem;
        for (int i = tid; i < SG_WTOT * 2 / 16; i += blockDim.x) dst[i] = __ldg(src + i);
    }
    if (tid == 0) mbar_init(bar, 1);
    if (warp == 0) tmem_alloc(holder, SG_TMEM_COLS);
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *holder;
    const uint32_t lane_off = (uint32_t)(32 * (warp & 3)) << 16;
    const uint32_t d_hid = tmem, d_out = tmem + 128u;
    const uint32_t sW1 = smem_u32(smem + OFF_W1), sW2 = smem_u32(smem + OFF_W2);
    const uint32_t sW3 = smem_u32(smem + OFF_W3), sW4 = smem_u32(smem + OFF_W4);
    const uint32_t sA = smem_u32(A);
    uint32_t phase = 0;
    unsigned int my_fb = 0;
    const bool raw = a.rawX != nullptr;
    const long long step = raw ? 0 : *a.step_ptr;
    const double t0 = (double)step * a.t_per_step;
    const int ntiles = (a.n + SG_M - 1) / SG_M;

    // The rows of a tile are built by the owner threads for the first tile,
    // then by the other half of the CTA while the owners finish the previous
    // tile's output (A is free once the output layer's MMA has completed).
    uint8_t *flags = smem + OFF_FLAGS;            // [2][SG_M]: inside the envelope
    int buf = 0;
    if (owner && (int)blockIdx.x < ntiles) {
        const int i0 = (int)blockIdx.x * SG_M + row;
        flags[row] = build_row(a, aux, step, raw, i0, i0 < a.n, row, A) ? 1 : 0;
    }
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int i = tile * SG_M + row;
        const bool valid = owner && i < a.n;
        if (!owner && !raw && tile + (int)gridDim.x < ntiles) prefetch_rows(a, tile + (int)gridDim.x, row);
        // layer 1 (K = 32), 2, 3 (K = 128): hidden, tanh
        const uint32_t sW[3] = {sW1, sW2, sW3};
        const float *bias[3] = {aux->b1, aux->b2, aux->b3};
        bool ok = true;
#pragma unroll 1
        for (int l = 0; l < 3 && ok; l++) {
            fence_proxy_async();
            tc_fence_before();
            __syncthreads();
            if (tid == 0) {
                tc_fence_after();
                issue_layer(d_hid, sA, sW[l], l == 0 ? SG_KIN : SG_H, SG_H, bar);
            }
            ok = wait_commit(bar, phase, a.err, a.mbar_polls);
            if (ok) hidden_epilogue(d_hid + lane_off, bias[l], A, row, half);
        }
        if (!ok) break;
        // output layer (K = 128, N = 32)
        fence_proxy_async();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            issue_layer(d_out, sA, sW4, SG_H, SG_NOUT, bar);
        }
        if (!wait_commit(bar, phase, a.err, a.mbar_polls)) break;
        if (!owner) {
            // the next tile's rows (its layer-1 MMA waits for the barrier at
            // the top of the next iteration)
            const int nt = tile + (int)gridDim.x;
            if (nt < ntiles) {
                const int i1 = nt * SG_M + row;
                flags[(buf ^ 1) * SG_M + row] = build_row(a, aux, step, raw, i1, i1 < a.n, row, A) ? 1 : 0;
            }
            buf ^= 1;
            continue;
        }
        const bool inside = flags[buf * SG_M + row] != 0;
        buf ^= 1;
        uint32_t yv[32];
        tmem_ld32(d_out + lane_off, yv);
        tc_fence_before();
        output_node(a, aux, i, valid, raw, inside, yv, t0, my_fb);
    }
    // count fallback node-steps
    for (int o = 16; o > 0; o >>= 1) my_fb += __shfl_xor_sync(0xffffffffu, my_fb, o);
    if ((tid & 31) == 0 && my_fb && a.status) atomicAdd(&a.status->fallback, (unsigned long long)my_fb);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, SG_TMEM_COLS);
}

// ---------------------------------------------------------------------------
// The same network with four tile pipelines in one CTA per SM (512 threads =
// four warpgroups).  Warpgroup g owns slot g: an A buffer of its own, TMEM
// columns [128 g, 128 g + 128) (the output layer reuses the first 32 once the
// last hidden epilogue has read them), an mbarrier and a named barrier; it
// runs its tiles start to end -- row build, four MMA layers, output --
// while the other three do the same, so four tiles are in flight per SM
// against two with k_surrogate, with one copy of the weights (80 KB) instead
// of two.  Each thread owns one node of its slot's tile and its whole row in
// the hidden epilogues.  Same instructions per tile, same results.
constexpr int SG4_SLOTS = 4;
constexpr int SG4_THREADS = SG4_SLOTS * SG_M;
constexpr int OFF4_A = OFF_W4 + SG_W4 * 2;
constexpr int OFF4_MISC = OFF4_A + SG4_SLOTS * SG_M * SG_H * 2;
constexpr int SG4_SMEM = OFF4_MISC + 128;
constexpr uint32_t SG4_TMEM_COLS = 512;

// named barrier `id` over the 128 threads of one warpgroup
__device__ __forceinline__ void wg_sync(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }
__device__ __forceinline__ bool wg_any(bool pred, int id) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, %2, 128, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(id)
        : "memory");
    return r != 0;
}

// wait_commit for one warpgroup (bounded, warpgroup-uniform)
__device__ __forceinline__ bool wait_commit_wg(uint64_t *bar, uint32_t &phase, unsigned int *err, unsigned int polls,
                                               int id) {
    bool ok = false;
    const unsigned int lim = polls ? polls : kMbarPolls;
    for (unsigned int it = 0; it < lim; it++)
        if (mbar_try_wait(bar, phase)) { ok = true; break; }
    phase ^= 1u;
    if (wg_any(!ok, id)) {
        if ((threadIdx.x & (SG_M - 1)) == 0) atomicExch(err, 1u);
        return false;
    }
    tc_fence_after();
    return true;
}

__global__ void __launch_bounds__(SG4_THREADS, 1) k_surrogate4(const SurrogateArgs a) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5;
    const int g = tid >> 7, row = tid & (SG_M - 1);
    const int bid = 1 + g;                        // named barrier of this warpgroup
    uint64_t *bars = (uint64_t *)(smem + OFF4_MISC);
    uint32_t *holder = (uint32_t *)(smem + OFF4_MISC + 64);
    unsigned char *A = smem + OFF4_A + (size_t)g * SG_M * SG_H * 2;
    const SurrogateAux *aux = a.aux;
    {
        const uint4 *src = (const uint4 *)a.wimg;
        uint4 *dst = (uint4 *)smem;
        for (int k = tid; k < SG_WTOT * 2 / 16; k += blockDim.x) dst[k] = __ldg(src + k);
    }
    if (tid == 0)
        for (int k = 0; k < SG4_SLOTS; k++) mbar_init(bars + k, 1);
    if (warp == 0) tmem_alloc(holder, SG4_TMEM_COLS);
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *holder;
    const uint32_t lane_off = (uint32_t)(32 * (warp & 3)) << 16;
    const uint32_t d_acc = tmem + 128u * (uint32_t)g;
    const uint32_t sW[4] = {smem_u32(smem + OFF_W1), smem_u32(smem + OFF_W2), smem_u32(smem + OFF_W3),
                            smem_u32(smem + OFF_W4)};
    const float *bias[3] = {aux->b1, aux->b2, aux->b3};
    const uint32_t sA = smem_u32(A);
    uint64_t *bar = bars + g;
    uint32_t phase = 0;
    unsigned int my_fb = 0;
    const bool raw = a.rawX != nullptr;
    const long long step = raw ? 0 : *a.step_ptr;
    const double t0 = (double)step * a.t_per_step;
    const int ntiles = (a.n + SG_M - 1) / SG_M;
    for (int tile = (int)blockIdx.x * SG4_SLOTS + g; tile < ntiles; tile += (int)gridDim.x * SG4_SLOTS) {
        const int i = tile * SG_M + row;
        const bool valid = i < a.n;
        const bool inside = build_row(a, aux, step, raw, i, valid, row, A);
        bool ok = true;
#pragma unroll 1
        for (int l = 0; l < 4 && ok; l++) {
            fence_proxy_async();
            tc_fence_before();
            wg_sync(bid);
            if (row == 0) {
                tc_fence_after();
                issue_layer(d_acc, sA, sW[l], l == 0 ? SG_KIN : SG_H, l == 3 ? SG_NOUT : SG_H, bar);
            }
            ok = wait_commit_wg(bar, phase, a.err, a.mbar_polls, bid);
            if (ok && l < 3) {
                hidden_epilogue(d_acc + lane_off, bias[l], A, row, 0);
                hidden_epilogue(d_acc + lane_off, bias[l], A, row, 1);
            }
        }
        if (!ok) break;
        uint32_t yv[32];
        tmem_ld32(d_acc + lane_off, yv);
        tc_fence_before();
        output_node(a, aux, i, valid, raw, inside, yv, t0, my_fb);
        // the next tile's row build overwrites A: every thread of the slot
        // is past its last read of this tile's TMEM and A above
        wg_sync(bid);
    }
    for (int o = 16; o > 0; o >>= 1) my_fb += __shfl_xor_sync(0xffffffffu, my_fb, o);
    if ((tid & 31) == 0 && my_fb && a.status) atomicAdd(&a.status->fallback, (unsigned long long)my_fb);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, SG4_TMEM_COLS);
}

// The hybrid form's physics for the nodes the network took: the reference's
// gate update and current balance over the sub-steps, with the six
// concentrations moving from their start to the network's end values
// (geometrically for the log-scaled Cai and Cass).  One thread per node.
__global__ void __launch_bounds__(128, 4) k_hybrid(const SurrogateArgs a) {
    const SurrogateAux *aux = a.aux;
    const long long step = *a.step_ptr;
    const double t0 = (double)step * a.t_per_step;
    const unsigned int lm = aux->log_mask;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        if (!a.take[i]) continue;
        float s[18], c0[6], c1[6];
#pragma unroll
        for (int k = 0; k < 18; k++) s[k] = a.S[(size_t)k * a.pitch + i];
        const int cslot[6] = {0, 1, 2, 9, 16, 17};
#pragma unroll
        for (int j = 0; j < 6; j++) {
            c0[j] = s[cslot[j]];
            c1[j] = a.pred[(size_t)j * a.pitch + i];
        }
        const int ty = a.type ? a.type[i] : 0;
        const float *c = a.consts + (size_t)ty * a.nconst;
        const float gks_i = a.gks ? a.gks[i] : 1.f;
        Track tr = {-1.f, -1.f, -1.f, 1e30f};
        bool dirty = false;
        const bool trk = a.track != nullptr;
        if (trk) tr = a.track[i];
        const int ns = aux->hyb_sub > 0 ? aux->hyb_sub : a.nsub;
        const float hu = (float)a.t_per_step / (float)ns;
        const float rdt = 1.f / (float)a.t_per_step;
        float V = a.V[i], tsum = 0.f;
        double tsub = t0;
        for (int k = 0; k < ns; k++) {
            const float h = aux->hyb_sub > 0 ? hu : a.sub_dt[k];
            tt_gate_step(s, V, h, c);
            tsum += h;
            const float w = fminf(tsum * rdt, 1.f);
#pragma unroll
            for (int j = 0; j < 6; j++) {
                const int q = cslot[j];
                s[q] = ((lm >> (q + 1)) & 1u) ? c0[j] * __powf(c1[j] / c0[j], w) : c0[j] + w * (c1[j] - c0[j]);
            }
            const float v1 = V + h * tt_dvdt<float>(V, s, c, 0.f, gks_i);
            if (trk && tr.t_rep < 0.f) track_interval(tr, dirty, V, v1, tsub, h, a.act_thr);
            V = v1;
            tsub += (double)h;
        }
#pragma unroll
        for (int k = 0; k < 18; k++) a.S[(size_t)k * a.pitch + i] = s[k];
        a.V[i] = V;
        if (dirty) a.track[i] = tr;
    }
}

// variant 0: k_surrogate, two CTAs of one tile pipeline per SM; 1:
// k_surrogate4, one CTA of four tile pipelines per SM
int launch_surrogate(const SurrogateArgs &a, cudaStream_t s, int variant) {
    // the shared-memory limit is per kernel and per device; setting it again
    // is cheap and keeps a second device right
    if (variant == 1)
        EP_CUDA(cudaFuncSetAttribute(k_surrogate4, cudaFuncAttributeMaxDynamicSharedMemorySize, SG4_SMEM));
    else
        EP_CUDA(cudaFuncSetAttribute(k_surrogate, cudaFuncAttributeMaxDynamicSharedMemorySize, SG_SMEM));
    int dev = 0, nsm = 148;
    EP_CUDA(cudaGetDevice(&dev));
    EP_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int ntiles = (a.n + SG_M - 1) / SG_M;
    if (ntiles <= 0) return EP_OK;
    if (variant == 1) {
        const int want = (ntiles + SG4_SLOTS - 1) / SG4_SLOTS;
        k_surrogate4<<<want < nsm ? want : nsm, SG4_THREADS, SG4_SMEM, s>>>(a);
    } else {
        k_surrogate<<<ntiles < 2 * nsm ? ntiles : 2 * nsm, SG_THREADS, SG_SMEM, s>>>(a);
    }
    EP_CUDA(cudaGetLastError());
    return EP_OK;
}

int launch_hybrid(const SurrogateArgs &a, cudaStream_t s) {
    if (a.n <= 0) return EP_OK;
    k_hybrid<<<(a.n + 127) / 128, 128, 0, s>>>(a);
    EP_CUDA(cudaGetLastError());
    return EP_OK;
}

}  // namespace ep
