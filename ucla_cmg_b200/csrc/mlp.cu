// mlp.cu -- trainer for the learned ionic step: a tanh MLP with FP32 master
// weights, trained on the GPU by the kernels in this file (tiled SGEMM for
// the forward and backward products, fused bias/tanh epilogues, loss and
// Adam kernels).  Inference in the time loop uses the BF16 tensor-core
// kernel in surrogate.cu; these kernels are for training only.
#include <cstring>
#include <vector>
#include <random>
#include <cmath>

#include "kernels.cuh"

namespace ep {

constexpr int GT = 64, GK = 16;   // 64x64 output tile, 16-deep k slices, 4x4 per thread

// C = op(A) op(B) (+ beta C) (+ bias) (tanh); A: M x K (TA: K x M), B: K x N (TB: N x K)
template <bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(256) k_sgemm(int M, int N, int K, const float *__restrict__ A, int lda,
                                               const float *__restrict__ B, int ldb, float *C, int ldc,
                                               const float *__restrict__ bias, float beta) {
    __shared__ float As[GK][GT + 4];
    __shared__ float Bs[GK][GT + 4];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.y * GT, n0 = blockIdx.x * GT;
    float acc[4][4] = {{0.f}};
    for (int k0 = 0; k0 < K; k0 += GK) {
        for (int e = threadIdx.x; e < GT * GK; e += 256) {
            const int mm = e / GK, kk = e % GK;     // A tile element (m, k)
            const int gm = m0 + mm, gk = k0 + kk;
            float v = 0.f;
            if (gm < M && gk < K) v = TA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk];
            As[kk][mm] = v;
            const int nn = e / GK, kb = e % GK;     // B tile element (k, n)
            const int gn = n0 + nn, gkb = k0 + kb;
            float w = 0.f;
            if (gn < N && gkb < K) w = TB ? B[(size_t)gn * ldb + gkb] : B[(size_t)gkb * ldb + gn];
            Bs[kb][nn] = w;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GK; kk++) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int gm = m0 + ty * 4 + i;
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int gn = n0 + tx * 4 + j;
            if (gn >= N) continue;
            float v = acc[i][j];
            if (beta != 0.f) v += beta * C[(size_t)gm * ldc + gn];
            if (EPI >= 1) v += bias[gn];
            if (EPI == 2) v = tanhf(v);
            C[(size_t)gm * ldc + gn] = v;
        }
    }
}

template <bool TA, bool TB, int EPI>
static void sgemm(int M, int N, int K, const float *A, int lda, const float *B, int ldb, float *C, int ldc,
                  const float *bias, float beta, cudaStream_t s) {
    dim3 grid((N + GT - 1) / GT, (M + GT - 1) / GT);
    k_sgemm<TA, TB, EPI><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, beta);
}

// delta <- delta * (1 - h^2)
__global__ void k_tanh_back(int n, float *d, const float *h) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) d[i] *= (1.f - h[i] * h[i]);
}

// column sums: out[j] (+)= sum_i D[i, j]
__global__ void k_colsum(int rows, int cols, const float *D, float *out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= cols) return;
    float s = 0.f;
    for (int i = 0; i < rows; i++) s += D[(size_t)i * cols + j];
    out[j] = s;
}

// delta = 2 w (P - Y) / batch ; loss += sum w (P - Y)^2 / batch
__global__ void k_mse(int rows, int cols, const float *P, const float *Y, const float *w, float *delta,
                      double *loss) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.0;
    if (i < rows * cols) {
        const int j = i % cols;
        const float d = P[i] - Y[i];
        const float wj = w ? w[j] : 1.f;
        delta[i] = 2.f * wj * d / (float)rows;
        l = (double)wj * (double)d * (double)d / (double)rows;
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && l != 0.0) atomicAdd(loss, l);
}

__global__ void k_adam(int n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

}  // namespace ep

using namespace ep;

struct ep_mlp {
    int device = 0;
    int L = 0;                       // number of weight layers
    std::vector<int> dims;           // L + 1
    std::vector<size_t> woff, boff;  // offsets into the flat parameter vector
    size_t np = 0;
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    float *act = nullptr;            // activations of the largest batch (layers 1..L)
    float *dlt = nullptr, *dlt2 = nullptr;
    float *w_out = nullptr;
    double *loss = nullptr;
    int cap = 0;                     // batch capacity of act/dlt
    long long t = 0;                 // Adam step
    int maxw = 0;
};

static int mlp_reserve(ep_mlp *m, int batch) {
    if (batch <= m->cap) return EP_OK;
    size_t tot = 0;
    for (int l = 1; l <= m->L; l++) tot += (size_t)m->dims[l];
    cudaFree(m->act); cudaFree(m->dlt); cudaFree(m->dlt2);
    m->act = m->dlt = m->dlt2 = nullptr;
    if (cudaMalloc(&m->act, sizeof(float) * tot * batch) != cudaSuccess ||
        cudaMalloc(&m->dlt, sizeof(float) * (size_t)m->maxw * batch) != cudaSuccess ||
        cudaMalloc(&m->dlt2, sizeof(float) * (size_t)m->maxw * batch) != cudaSuccess) {
        cudaGetLastError();
        set_error("MLP workspace allocation failed (batch %d)", batch);
        return EP_ERR_NOMEM;
    }
    m->cap = batch;
    return EP_OK;
}

// activation of layer l (1..L) for a batch of `cap` rows
static float *act_of(ep_mlp *m, int l) {
    size_t off = 0;
    for (int k = 1; k < l; k++) off += (size_t)m->dims[k] * m->cap;
    return m->act + off;
}

static void forward(ep_mlp *m, const float *X, int B, cudaStream_t s) {
    const float *h = X;
    for (int l = 1; l <= m->L; l++) {
        float *z = act_of(m, l);
        const float *W = m->p + m->woff[l - 1], *b = m->p + m->boff[l - 1];
        if (l < m->L) sgemm<false, true, 2>(B, m->dims[l], m->dims[l - 1], h, m->dims[l - 1], W, m->dims[l - 1], z,
                                             m->dims[l], b, 0.f, s);
        else sgemm<false, true, 1>(B, m->dims[l], m->dims[l - 1], h, m->dims[l - 1], W, m->dims[l - 1], z,
                                    m->dims[l], b, 0.f, s);
        h = z;
    }
}

extern "C" {

int ep_mlp_create(int32_t n_layers, const int32_t *dims, uint64_t seed, int device, ep_mlp **out) {
    EP_CHECK_ARG(out && dims && n_layers >= 1 && n_layers <= 8, "bad MLP shape");
    for (int l = 0; l <= n_layers; l++) EP_CHECK_ARG(dims[l] > 0 && dims[l] <= 4096, "bad MLP width");
    EP_CUDA(cudaSetDevice(device));
    ep_mlp *m = new ep_mlp();
    m->device = device;
    m->L = n_layers;
    m->dims.assign(dims, dims + n_layers + 1);
    for (int l = 0; l < n_layers; l++) {
        m->woff.push_back(m->np);
        m->np += (size_t)dims[l + 1] * dims[l];
        m->boff.push_back(m->np);
        m->np += (size_t)dims[l + 1];
        m->maxw = std::max(m->maxw, std::max(dims[l], dims[l + 1]));
    }
    // Xavier-uniform weights, zero biases
    std::vector<float> h(m->np, 0.f);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < n_layers; l++) {
        const float a = std::sqrt(6.f / (float)(dims[l] + dims[l + 1]));
        std::uniform_real_distribution<float> U(-a, a);
        for (size_t k = 0; k < (size_t)dims[l + 1] * dims[l]; k++) h[m->woff[l] + k] = U(rng);
    }
    if (cudaMalloc(&m->p, sizeof(float) * m->np) != cudaSuccess ||
        cudaMalloc(&m->g, sizeof(float) * m->np) != cudaSuccess ||
        cudaMalloc(&m->m, sizeof(float) * m->np) != cudaSuccess ||
        cudaMalloc(&m->v, sizeof(float) * m->np) != cudaSuccess ||
        cudaMalloc(&m->w_out, sizeof(float) * dims[n_layers]) != cudaSuccess ||
        cudaMalloc(&m->loss, sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        ep_mlp_destroy(m);
        set_error("MLP allocation failed");
        return EP_ERR_NOMEM;
    }
    cudaMemcpy(m->p, h.data(), sizeof(float) * m->np, cudaMemcpyHostToDevice);
    cudaMemset(m->g, 0, sizeof(float) * m->np);
    cudaMemset(m->m, 0, sizeof(float) * m->np);
    cudaMemset(m->v, 0, sizeof(float) * m->np);
    *out = m;
    return EP_OK;
}

void ep_mlp_destroy(ep_mlp *m) {
    if (!m) return;
    cudaFree(m->p); cudaFree(m->g); cudaFree(m->m); cudaFree(m->v);
    cudaFree(m->act); cudaFree(m->dlt); cudaFree(m->dlt2); cudaFree(m->w_out); cudaFree(m->loss);
    delete m;
}

int ep_mlp_num_params(const ep_mlp *m) { return m ? (int)m->np : EP_ERR_ARG; }

int ep_mlp_get_params(ep_mlp *m, float *out) {
    EP_CHECK_ARG(m && out, "null argument");
    EP_CUDA(cudaMemcpy(out, m->p, sizeof(float) * m->np, cudaMemcpyDeviceToHost));
    return EP_OK;
}

int ep_mlp_set_params(ep_mlp *m, const float *in) {
    EP_CHECK_ARG(m && in, "null argument");
    EP_CUDA(cudaMemcpy(m->p, in, sizeof(float) * m->np, cudaMemcpyHostToDevice));
    EP_CUDA(cudaMemset(m->m, 0, sizeof(float) * m->np));
    EP_CUDA(cudaMemset(m->v, 0, sizeof(float) * m->np));
    m->t = 0;
    return EP_OK;
}

int ep_mlp_forward(ep_mlp *m, const float *X, float *Y, int32_t B, void *stream) {
    EP_CHECK_ARG(m && X && Y && B > 0, "bad arguments");
    int rc = mlp_reserve(m, B);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    forward(m, X, B, s);
    EP_CUDA(cudaMemcpyAsync(Y, act_of(m, m->L), sizeof(float) * (size_t)B * m->dims[m->L],
                            cudaMemcpyDeviceToDevice, s));
    EP_CUDA(cudaGetLastError());
    return EP_OK;
}

int ep_mlp_loss_grad(ep_mlp *m, const float *X, const float *Y, const float *w_out_host, int32_t B,
                     double *loss, float *grad_host, void *stream) {
    EP_CHECK_ARG(m && X && Y && B > 0, "bad arguments");
    int rc = mlp_reserve(m, B);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const int L = m->L, dout = m->dims[L];
    if (w_out_host) EP_CUDA(cudaMemcpyAsync(m->w_out, w_out_host, sizeof(float) * dout, cudaMemcpyHostToDevice, s));
    forward(m, X, B, s);
    EP_CUDA(cudaMemsetAsync(m->loss, 0, sizeof(double), s));
    const int ne = B * dout;
    k_mse<<<(ne + 255) / 256, 256, 0, s>>>(B, dout, act_of(m, L), Y, w_out_host ? m->w_out : nullptr, m->dlt,
                                           m->loss);
    float *d = m->dlt, *d2 = m->dlt2;
    for (int l = L; l >= 1; l--) {
        const float *hprev = l > 1 ? act_of(m, l - 1) : X;
        const int nout = m->dims[l], nin = m->dims[l - 1];
        // dW_l = delta^T hprev  (nout x nin), db_l = colsum(delta)
        sgemm<true, false, 0>(nout, nin, B, d, nout, hprev, nin, m->g + m->woff[l - 1], nin, nullptr, 0.f, s);
        k_colsum<<<(nout + 127) / 128, 128, 0, s>>>(B, nout, d, m->g + m->boff[l - 1]);
        if (l > 1) {
            // delta_{l-1} = (delta W_l) * (1 - h_{l-1}^2)
            sgemm<false, false, 0>(B, nin, nout, d, nout, m->p + m->woff[l - 1], nin, d2, nin, nullptr, 0.f, s);
            k_tanh_back<<<(B * nin + 255) / 256, 256, 0, s>>>(B * nin, d2, act_of(m, l - 1));
            std::swap(d, d2);
        }
    }
    EP_CUDA(cudaGetLastError());
    if (loss) {
        EP_CUDA(cudaMemcpyAsync(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    if (grad_host) EP_CUDA(cudaMemcpyAsync(grad_host, m->g, sizeof(float) * m->np, cudaMemcpyDeviceToHost, s));
    if (loss || grad_host) EP_CUDA(cudaStreamSynchronize(s));
    return EP_OK;
}

int ep_mlp_adam_step(ep_mlp *m, float lr, float beta1, float beta2, float eps) {
    EP_CHECK_ARG(m, "null trainer");
    m->t++;
    const float c1 = 1.f - std::pow(beta1, (float)m->t), c2 = 1.f - std::pow(beta2, (float)m->t);
    k_adam<<<(int)((m->np + 255) / 256), 256>>>((int)m->np, m->p, m->g, m->m, m->v, lr, beta1, beta2, eps, c1, c2);
    EP_CUDA(cudaGetLastError());
    return EP_OK;
}

}  // extern "C"
