// cells_host.cu -- TEST HARNESS: the library's cell-model source
// (ucla_cmg_b200/csrc/{tt,mahajan,purkinje}.cuh, host+device code) compiled
// for the host, so its formulas can be checked against the oracle and the
// reference's golden vectors without a GPU.  Not part of the library.
#include <cstdint>
#include <cstring>

#include "../../ucla_cmg_b200/csrc/tt.cuh"
#include "../../ucla_cmg_b200/csrc/mahajan.cuh"
#include "../../ucla_cmg_b200/csrc/purkinje.cuh"

using namespace ep;

// One Compute_Ion call per node in FP64 (fp32 = 0) or FP32 (fp32 = 1, the
// precision of the FP32 kernels).  model: EP_TUSSCHER, EP_MAHAJAN /
// EP_MAHAJAN_FAIL, or 5 (the Purkinje cell).  states: node-major reference
// state vectors (TT 19, Mahajan 26, Purkinje 22; [0] = V), advanced in place.
// consts: ntypes x nconst, type[i] picks the set (NULL: 0).  Returns 0, or -1
// for an unknown model.
// one node in precision R (states and results in double at the interface)
template <typename R>
static int node(int model, double dt, double Cm, double Xi, const double *cd, int nconst, double gks, int jac_true,
                int newton_cap, double newton_tol, int mh_abs, double V, double ist, double *st, double *dvdt,
                long long &w) {
    R c[64], s[26];
    const int ns = model == EP_TUSSCHER ? 19 : (model == 5 ? 22 : 26);
    for (int k = 0; k < nconst && k < 64; k++) c[k] = (R)cd[k];
    for (int k = 0; k < ns; k++) s[k] = (R)st[k];
    R d;
    if (model == EP_TUSSCHER) {
        TTOpts o;
        o.newton_cap = newton_cap > 0 ? newton_cap : 100;
        o.jac_true = jac_true;
        o.fp32_scaled_tol = sizeof(R) == 4 ? 1 : 0;
        o.newton_tol = newton_tol > 0 ? newton_tol : 1e-6;
        int it = 0;
        d = tt_compute_ion<R>(s + 1, (R)V, (R)(-ist / (Cm * Xi)), (R)dt, c, (R)gks, o, it);
        s[0] = (R)V;
        w += it;
    } else if (model == EP_MAHAJAN || model == EP_MAHAJAN_FAIL) {
        int sub = 0;
        d = mh_compute_ion<R>(s, (R)V, (R)(ist / (Cm * Xi)), (R)dt, c, mh_abs, sub);
        w += sub;
    } else if (model == 5) {
        int sub = 0;
        d = pk_compute_ion<R>(s, (R)V, (R)ist, (R)Xi, (R)dt, c, sub);
        w += sub;
    } else {
        return -1;
    }
    for (int k = 0; k < ns; k++) st[k] = (double)s[k];
    *dvdt = (double)d;
    return 0;
}

extern "C" int cells_host_compute_ion(int model, int n, double dt, double Cm, double Xi, const double *consts,
                                      int nconst, const uint8_t *type, const double *gks, int jac_true,
                                      int newton_cap, double newton_tol, int mh_abs, const double *V,
                                      const double *istim, double *states, double *dvdt, long long *work,
                                      int fp32) {
    if (nconst > 64) return -1;
    long long w = 0;
    const int ns = model == EP_TUSSCHER ? 19 : (model == 5 ? 22 : 26);
    for (int i = 0; i < n; i++) {
        const double *c = consts + (size_t)(type ? type[i] : 0) * nconst;
        const double ist = istim ? istim[i] : 0.0;
        const double g = gks ? gks[i] : 1.0;
        double *st = states + (size_t)i * ns;
        const int rc = fp32 ? node<float>(model, dt, Cm, Xi, c, nconst, g, jac_true, newton_cap, newton_tol, mh_abs,
                                          V[i], ist, st, dvdt + i, w)
                            : node<double>(model, dt, Cm, Xi, c, nconst, g, jac_true, newton_cap, newton_tol, mh_abs,
                                           V[i], ist, st, dvdt + i, w);
        if (rc) return rc;
    }
    if (work) *work = w;
    return 0;
}
