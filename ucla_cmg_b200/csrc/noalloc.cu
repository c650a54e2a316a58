// noalloc.cu -- the Crank-Nicolson half diffusion step for callers that
// cannot allocate device memory.
//
// Some hosts of this solver own every device allocation themselves: a code
// that runs inside a larger simulator's memory pool, a driver that must not
// call cudaMalloc once its time loop has started (allocation synchronises the
// device and can fail late in a long run), or a C/Fortran caller that only
// hands over buffers it manages.  ep_cn_half_step_noalloc gives them the
// persistent Jacobi-PCG kernel with its working vectors (r, q and the two
// search-direction buffers), the reduction partials and the grid barrier
// placed in one statically sized device array defined in this file, so a
// call performs no device allocation at all.  The caller passes the matrix
// (SELL-32 layout) and the voltage vector, both in its own device memory.
//
// Limits and rules (repeated in include/ep_gpu.h):
// * at most kNoAllocMaxRows rows; larger systems are rejected with
//   EP_ERR_ARG;
// * the array (about 8.2 MB) is part of the module: every GPU that loads the
//   library holds it until the process exits;
// * every call shares the one array, so calls that overlap on the GPU (two
//   streams, two host threads) race -- serialise them;
// * each call looks up the array's device address on the current device
//   (cudaGetSymbolAddress): host code only holds a stand-in for the symbol,
//   and an address kept from an earlier call would be stale after a
//   cudaDeviceReset;
// * the call waits on `stream` for its own results before it returns; on a
//   stream in capture mode it returns EP_ERR_ARG before touching the stream,
//   so the caller's capture stays intact.
#include "kernels.cuh"

namespace ep {

constexpr int kNoAllocMaxRows = 262144;                 // 2^18 rows
constexpr int kNoAllocMaxGrid = 2048;                   // >= 148 SMs x 8 blocks
constexpr size_t kVecBytes = sizeof(double) * (size_t)kNoAllocMaxRows;   // one vector, FP64
constexpr size_t kScratchBytes = 5 * kVecBytes                            // r, q, p0, (z, p) pairs (2)
                               + sizeof(double) * 12 * kNoAllocMaxGrid    // reduction partials (12 slots)
                               + 256;                                     // barrier, stats, result

// the only storage a call uses beyond the caller's buffers
static __device__ __align__(256) unsigned char g_cg_scratch[kScratchBytes];

namespace {

// the device address of g_cg_scratch on the current device, looked up anew
// on every call (cheap next to a persistent CG launch, and never stale)
int scratch_address(void **out) {
    int dev = 0;
    EP_CUDA(cudaGetDevice(&dev));
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_cg_scratch);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("cudaGetSymbolAddress(scratch) on device %d: %s", dev, cudaGetErrorString(e));
        return EP_ERR_CUDA;
    }
    *out = p;
    return EP_OK;
}

template <typename R>
int run(unsigned char *base, int n, int nslices, const int *slice_ptr, const int *col, const R *A,
        const R *B, const R *dinv, R *x, double tol, int maxit, cudaStream_t s, int *iters,
        double *relres) {
    CGArgs<R> a{};
    a.n = n; a.nslices = nslices;
    a.slice_ptr = slice_ptr; a.col = col;
    a.Aval = A; a.Bval = B; a.dinv = dinv; a.x = x;
    a.r = (R *)(base + 0 * kVecBytes);
    a.q = (R *)(base + 1 * kVecBytes);
    a.p0 = (R *)(base + 2 * kVecBytes);
    a.zp = (R *)(base + 3 * kVecBytes);                            // two vectors: (z, p) pairs
    a.partial = (double *)(base + 5 * kVecBytes);
    unsigned char *tail = base + 5 * kVecBytes + sizeof(double) * 12 * kNoAllocMaxGrid;
    a.bar = (GridBarrier *)tail;                                   // 16 B
    unsigned long long *st = (unsigned long long *)(tail + 64);   // 32 B of counters
    a.iters_total = st;
    a.iters_max = (unsigned int *)(st + 1);
    a.fails = (unsigned int *)(st + 1) + 1;
    a.last = (double *)(tail + 128);                               // 16 B result
    a.tol = tol > 0 ? tol : 1e-7;
    a.floor_rel = sizeof(R) == 4 ? 1.2e-7 : 2.2e-16;
    a.maxit = maxit > 0 ? maxit : 1000;
    // the barrier and the counters must start at zero; the kernel writes the
    // vectors and partials before it reads them
    EP_CUDA(cudaMemsetAsync(tail, 0, 256, s));
    int grid = 0;
    int rc = cg_grid_size<R>(256, &grid);
    if (rc) return rc;
    grid = grid < kNoAllocMaxGrid ? grid : kNoAllocMaxGrid;
    if ((rc = launch_cg<R>(a, grid, 256, s))) return rc;
    double last[2] = {0.0, 0.0};
    GridBarrier bar{};
    EP_CUDA(cudaMemcpyAsync(last, a.last, sizeof last, cudaMemcpyDeviceToHost, s));
    EP_CUDA(cudaMemcpyAsync(&bar, a.bar, sizeof bar, cudaMemcpyDeviceToHost, s));
    EP_CUDA(cudaStreamSynchronize(s));
    if (iters) *iters = (int)last[0];
    if (relres) *relres = last[1];
    if (bar.err) { set_error("a grid barrier wait gave up"); return EP_ERR_TIMEOUT; }
    return EP_OK;
}

}  // namespace
}  // namespace ep

extern "C" int ep_cn_half_step_noalloc(int32_t precision, int32_t n, int32_t nslices,
                                       const int32_t *slice_ptr, const int32_t *col,
                                       const void *Aval, const void *Bval, const void *dinv,
                                       void *x, double cg_tol, int32_t cg_maxit, void *stream,
                                       int32_t *iters, double *relres) {
    using namespace ep;
    EP_CHECK_ARG(precision == EP_FP64 || precision == EP_FP32, "precision must be EP_FP64 or EP_FP32");
    EP_CHECK_ARG(n > 0, "n must be positive");
    if (n > kNoAllocMaxRows) {
        set_error("ep_cn_half_step_noalloc: %d rows exceed the static scratch limit of %d rows",
                  n, kNoAllocMaxRows);
        return EP_ERR_ARG;
    }
    EP_CHECK_ARG(nslices == (n + kSlice - 1) / kSlice, "nslices must be ceil(n / 32)");
    EP_CHECK_ARG(slice_ptr && col && Aval && Bval && dinv && x, "null device pointer");
    cudaStream_t s = (cudaStream_t)stream;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    EP_CUDA(cudaStreamIsCapturing(s, &cap));
    if (cap != cudaStreamCaptureStatusNone) {
        set_error("ep_cn_half_step_noalloc: the stream is being captured; the call waits for its "
                  "results on the stream and would invalidate the capture");
        return EP_ERR_ARG;
    }
    void *base = nullptr;
    int rc = scratch_address(&base);
    if (rc) return rc;
    if (precision == EP_FP64)
        return run<double>((unsigned char *)base, n, nslices, slice_ptr, col, (const double *)Aval,
                           (const double *)Bval, (const double *)dinv, (double *)x, cg_tol, cg_maxit, s,
                           iters, relres);
    return run<float>((unsigned char *)base, n, nslices, slice_ptr, col, (const float *)Aval,
                      (const float *)Bval, (const float *)dinv, (float *)x, cg_tol, cg_maxit, s, iters,
                      relres);
}
