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

// One Compute_Ion call per node in FP64.  model: EP_TUSSCHER, EP_MAHAJAN /
// EP_MAHAJAN_FAIL, or 5 (the Purkinje cell).  states: node-major reference
// state vectors (TT 19, Mahajan 26, Purkinje 22; [0] = V), advanced in place.
// consts: ntypes x nconst, type[i] picks the set (NULL: 0).  Returns 0, or -1
// for an unknown model.
extern "C" int cells_host_compute_ion(int model, int n, double dt, double Cm, double Xi, const double *consts,
                                      int nconst, const uint8_t *type, const double *gks, int jac_true,
                                      int newton_cap, double newton_tol, int mh_abs, const double *V,
                                      const double *istim, double *states, double *dvdt, long long *work) {
    long long w = 0;
    for (int i = 0; i < n; i++) {
        const double *c = consts + (size_t)(type ? type[i] : 0) * nconst;
        const double ist = istim ? istim[i] : 0.0;
        if (model == EP_TUSSCHER) {
            double *s = states + (size_t)i * 19;
            TTOpts o;
            o.newton_cap = newton_cap > 0 ? newton_cap : 100;
            o.jac_true = jac_true;
            o.fp32_scaled_tol = 0;
            o.newton_tol = newton_tol > 0 ? newton_tol : 1e-6;
            int it = 0;
            dvdt[i] = tt_compute_ion<double>(s + 1, V[i], -ist / (Cm * Xi), dt, c, gks ? gks[i] : 1.0, o, it);
            s[0] = V[i];
            w += it;
        } else if (model == EP_MAHAJAN || model == EP_MAHAJAN_FAIL) {
            int sub = 0;
            dvdt[i] = mh_compute_ion<double>(states + (size_t)i * 26, V[i], ist / (Cm * Xi), dt, c, mh_abs, sub);
            w += sub;
        } else if (model == 5) {
            int sub = 0;
            dvdt[i] = pk_compute_ion<double>(states + (size_t)i * 22, V[i], ist, Xi, dt, c, sub);
            w += sub;
        } else {
            return -1;
        }
    }
    if (work) *work = w;
    return 0;
}
