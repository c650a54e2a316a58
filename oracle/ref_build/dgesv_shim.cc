// dgesv_shim.cc -- LAPACK's dgesv_ for the reference's ten Tusscher model
// (voomEP/src/IonicModel/Tusscher.cc:181), which calls it for its 6x6 Newton
// step.  LAPACK is not installed here.  TEST INFRASTRUCTURE ONLY, linked into
// both oracle libraries built from the reference's sources.
#include <cmath>
#include <utility>

// ---- LAPACK dgesv_.  Column-major, partial
// pivoting, the textbook getf2 elimination + getrs triangular solves. ----
extern "C" void dgesv_(int *N, int *NRHS, double *A, int *LDA, int *IPIV,
                       double *B, int *LDB, int *INFO)
{
    const int n = *N, lda = *LDA, ldb = *LDB, nrhs = *NRHS;
    *INFO = 0;
    for (int k = 0; k < n; k++) {
        int p = k; double amax = std::fabs(A[k + k * lda]);
        for (int i = k + 1; i < n; i++) {
            double v = std::fabs(A[i + k * lda]);
            if (v > amax) { amax = v; p = i; }
        }
        IPIV[k] = p + 1;
        if (A[p + k * lda] != 0.0) {
            if (p != k)
                for (int j = 0; j < n; j++) std::swap(A[k + j * lda], A[p + j * lda]);
            const double r = 1.0 / A[k + k * lda];
            for (int i = k + 1; i < n; i++) A[i + k * lda] *= r;
        } else if (*INFO == 0) {
            *INFO = k + 1;
        }
        for (int j = k + 1; j < n; j++) {
            const double ukj = A[k + j * lda];
            if (ukj != 0.0)
                for (int i = k + 1; i < n; i++) A[i + j * lda] -= A[i + k * lda] * ukj;
        }
    }
    if (*INFO) return;
    for (int c = 0; c < nrhs; c++) {
        double *b = B + c * ldb;
        for (int k = 0; k < n; k++)
            if (IPIV[k] - 1 != k) std::swap(b[k], b[IPIV[k] - 1]);
        for (int j = 0; j < n; j++)
            if (b[j] != 0.0)
                for (int i = j + 1; i < n; i++) b[i] -= b[j] * A[i + j * lda];
        for (int j = n - 1; j >= 0; j--)
            if (b[j] != 0.0) {
                b[j] /= A[j + j * lda];
                for (int i = 0; i < j; i++) b[i] -= b[j] * A[i + j * lda];
            }
    }
}
