/*
 * ep_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY, see ep_oracle.h).
 *
 * A plain-C FP64 restatement of the reference voomEP monodomain path.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 */
#include "ep_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

void epo_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
int epo_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ====================================================================== */
/* ten Tusscher 2006 -- Tusscher.cc / Tusscher.h / SetUpIonicConstants.h   */
/* ====================================================================== */

/* SetUpIonicConstants.h:88-147 (epicardial set).  [53] selects the s-gate
 * kinetics: 0 = the reference's (epi/M) form, 1 = TT2006 endocardial form
 * (not in the reference; used only for the transmural shell workload). */
void epo_tt_constants(double *c) {
    static const double k[53] = {
        8314.472, 310, 96485.3415, 0.185, 0.016404, 10, 1000, 1, 52, 0.03,
        5.4, 140, 2, 5.405, 0.153, 0.392, 14.838, 0.00029, 0.0000398, 0.000592,
        0.294, 2.724, 1, 40, 1000, 0.1, 2.5, 0.35, 1.38, 87.5,
        0.1238, 0.0005, 0.0146, 0.15, 0.045, 0.06, 0.005, 1.5, 2.5, 1,
        0.102, 0.0038, 0.00025, 0.00036, 0.006375, 0.2, 0.001, 10, 0.3, 0.4,
        0.00025, 0.001094, 0.00005468 };
    memcpy(c, k, sizeof k);
    c[53] = 0.0;
}

/* Tusscher.h:51-69, the "KCL" resting state */
void epo_tt_initial_state(double *s) {
    static const double k[19] = {
        -85.423, 136.89, 8.604, 0.000126, 0.00621, 0.4712, 0.0095, 0.00172,
        0.7444, 0.7045, 0.00036, 3.373e-5, 0.7888, 0.9755, 0.9953, 0.999998,
        2.42e-8, 3.64, 0.9073 };
    memcpy(s, k, sizeof k);
}

/* Gate states updated semi-implicitly, in the reference order
 * (Tusscher.cc:122-143). */
static const int TT_GATE[12] = {4, 5, 6, 7, 8, 9, 11, 12, 13, 14, 15, 16};
/* States solved by Newton (Tusscher.cc:126). */
static const int TT_NR[6] = {1, 2, 3, 10, 17, 18};

/* Tusscher::ComputeRates (Tusscher.cc:4-96).  ginf/gtau receive the
 * steady state and time constant of the 12 gates in TT_GATE order; rate
 * receives dV/dt in [0] and the Newton-state rates at their state index.
 * ist is Algebraic[12] = -istim/(Cm*Xi). */
static void tt_rates(const double *s, const double *c, double ist,
                     double *ginf, double *gtau, double *rate)
{
    const double V = s[0], Ki = s[1], Nai = s[2], Cai = s[3];
    const double xr1 = s[4], xr2 = s[5], xs = s[6], m = s[7], h = s[8], j = s[9];
    const double Cass = s[10], d = s[11], f = s[12], f2 = s[13], fcass = s[14];
    const double sg = s[15], rg = s[16], Casr = s[17], Rp = s[18];
    const double R = c[0], T = c[1], F = c[2];
    const double RT = R * T;

    /* ---- gates ---- */
    double t;
    /* f (12) */
    ginf[7] = 1.0 / (1.0 + exp((V + 20.0) / 7.0));
    t = V + 27.0;
    gtau[7] = 1102.5 * exp((-(t * t)) / 225.0) + 200.0 / (1.0 + exp((13.0 - V) / 10.0))
            + 180.0 / (1.0 + exp((V + 30.0) / 10.0)) + 20.0;
    /* f2 (13) */
    ginf[8] = 0.67 / (1.0 + exp((V + 35.0) / 7.0)) + 0.33;
    gtau[8] = 562.0 * exp((-(t * t)) / 240.0) + 31.0 / (1.0 + exp((25.0 - V) / 10.0))
            + 80.0 / (1.0 + exp((V + 30.0) / 10.0));
    /* fCass (14) */
    t = Cass / 0.05;
    ginf[9] = 0.6 / (1.0 + t * t) + 0.4;
    gtau[9] = 80.0 / (1.0 + t * t) + 2.0;
    /* s (15) */
    if (c[53] == 0.0) {
        ginf[10] = 1.0 / (1.0 + exp((V + 20.0) / 5.0));
        t = V + 45.0;
        gtau[10] = 85.0 * exp((-(t * t)) / 320.0) + 5.0 / (1.0 + exp((V - 20.0) / 5.0)) + 3.0;
    } else {
        ginf[10] = 1.0 / (1.0 + exp((V + 28.0) / 5.0));
        t = V + 67.0;
        gtau[10] = 1000.0 * exp((-(t * t)) / 1000.0) + 8.0;
    }
    /* r (16) */
    ginf[11] = 1.0 / (1.0 + exp((20.0 - V) / 6.0));
    t = V + 40.0;
    gtau[11] = 9.5 * exp((-(t * t)) / 1800.0) + 0.8;
    /* Xr1 (4) */
    ginf[0] = 1.0 / (1.0 + exp((-26.0 - V) / 7.0));
    gtau[0] = (450.0 / (1.0 + exp((-45.0 - V) / 10.0))) * (6.0 / (1.0 + exp((V + 30.0) / 11.5)));
    /* Xr2 (5) */
    ginf[1] = 1.0 / (1.0 + exp((V + 88.0) / 24.0));
    gtau[1] = (3.0 / (1.0 + exp((-60.0 - V) / 20.0))) * (1.12 / (1.0 + exp((V - 60.0) / 20.0)));
    /* Xs (6) */
    ginf[2] = 1.0 / (1.0 + exp((-5.0 - V) / 14.0));
    gtau[2] = (1400.0 / sqrt(1.0 + exp((5.0 - V) / 6.0))) * (1.0 / (1.0 + exp((V - 35.0) / 15.0))) + 80.0;
    /* m (7) */
    t = 1.0 + exp((-56.86 - V) / 9.03);
    ginf[3] = 1.0 / (t * t);
    gtau[3] = (1.0 / (1.0 + exp((-60.0 - V) / 5.0)))
            * (0.1 / (1.0 + exp((V + 35.0) / 5.0)) + 0.1 / (1.0 + exp((V - 50.0) / 200.0)));
    /* h (8), j (9) */
    t = 1.0 + exp((V + 71.55) / 7.43);
    ginf[4] = 1.0 / (t * t);
    ginf[5] = ginf[4];
    {
        double ah, bh, aj, bj;
        if (V < -40.0) {
            ah = 0.057 * exp((-(V + 80.0)) / 6.8);
            bh = 2.7 * exp(0.079 * V) + 310000.0 * exp(0.3485 * V);
            aj = ((-25428.0 * exp(0.2444 * V) - 6.948e-06 * exp(-0.04391 * V)) * (V + 37.78))
               / (1.0 + exp(0.311 * (V + 79.23)));
            bj = (0.02424 * exp(-0.01052 * V)) / (1.0 + exp(-0.1378 * (V + 40.14)));
        } else {
            ah = 0.0;
            bh = 0.77 / (0.13 * (1.0 + exp((V + 10.66) / -11.1)));
            aj = 0.0;
            bj = (0.6 * exp(0.057 * V)) / (1.0 + exp(-0.1 * (V + 32.0)));
        }
        gtau[4] = 1.0 / (ah + bh);
        gtau[5] = 1.0 / (aj + bj);
    }
    /* d (11) */
    ginf[6] = 1.0 / (1.0 + exp((-8.0 - V) / 7.5));
    gtau[6] = (1.4 / (1.0 + exp((-35.0 - V) / 13.0)) + 0.25) * (1.4 / (1.0 + exp((V + 5.0) / 5.0)))
            + 1.0 / (1.0 + exp((50.0 - V) / 20.0));

    /* ---- currents ---- */
    const double i_nak = (((c[21] * c[10]) / (c[10] + c[22])) * Nai) / (Nai + c[23])
        / (1.0 + 0.1245 * exp((-0.1 * V * F) / RT) + 0.0353 * exp((-V * F) / RT));
    const double E_Na = (RT / F) * log(c[11] / Nai);
    const double i_na = c[16] * (m * m * m) * h * j * (V - E_Na);
    const double i_bna = c[17] * (V - E_Na);
    const double e_g = exp((c[27] * V * F) / RT);
    const double e_g1 = exp(((c[27] - 1.0) * V * F) / RT);
    const double i_naca = (c[24] * (e_g * (Nai * Nai * Nai) * c[12]
                                    - e_g1 * (c[11] * c[11] * c[11]) * Cai * c[26]))
        / (((c[29] * c[29] * c[29]) + (c[11] * c[11] * c[11])) * (c[28] + c[12])
           * (1.0 + c[25] * e_g1));
    rate[2] = ((-(i_na + i_bna + 3.0 * i_nak + 3.0 * i_naca)) / (c[4] * F)) * c[3];

    const double E_K = (RT / F) * log(c[10] / Ki);
    const double vk = V - E_K;
    const double a_k1 = 0.1 / (1.0 + exp(0.06 * (vk - 200.0)));
    const double b_k1 = (3.0 * exp(0.0002 * (vk + 100.0)) + exp(0.1 * (vk - 10.0)))
                      / (1.0 + exp(-0.5 * vk));
    const double xk1 = a_k1 / (a_k1 + b_k1);
    const double sq_ko = sqrt(c[10] / 5.4);
    const double i_k1 = c[13] * xk1 * sq_ko * vk;
    const double i_to = c[20] * rg * sg * vk;
    const double i_kr = c[14] * sq_ko * xr1 * xr2 * vk;
    const double E_Ks = (RT / F) * log((c[10] + c[9] * c[11]) / (Ki + c[9] * Nai));
    const double i_ks = c[15] * (xs * xs) * (V - E_Ks);
    const double e_ca = exp((2.0 * (V - 15.0) * F) / RT);
    const double i_cal = (((c[18] * d * f * f2 * fcass * 4.0 * (V - 15.0) * (F * F)) / RT)
                          * (0.25 * Cass * e_ca - c[12])) / (e_ca - 1.0);
    const double E_Ca = ((0.5 * R * T) / F) * log(c[12] / Cai);
    const double i_bca = c[19] * (V - E_Ca);
    const double i_pk = (c[32] * vk) / (1.0 + exp((25.0 - V) / 5.98));
    const double i_pca = (c[30] * Cai) / (Cai + c[31]);

    rate[0] = -(i_k1 + i_to + i_kr + i_ks + i_cal + i_nak + i_na + i_bna + i_naca
                + i_bca + i_pk + i_pca + ist);
    rate[1] = ((-((i_k1 + i_to + i_kr + i_ks + i_pk + ist) - 2.0 * i_nak)) / (c[4] * F)) * c[3];

    const double j_up = c[44] / (1.0 + (c[42] * c[42]) / (Cai * Cai));
    const double j_leak = c[43] * (Casr - Cai);
    const double j_xfer = c[41] * (Cass - Cai);
    const double bufc = 1.0 / (1.0 + (c[45] * c[46]) / ((Cai + c[46]) * (Cai + c[46])));
    rate[3] = bufc * ((((j_leak - j_up) * c[51]) / c[4] + j_xfer)
                      - (((i_bca + i_pca) - 2.0 * i_naca) * c[3]) / (2.0 * c[4] * F));
    t = c[37] / Casr;
    const double kcasr = c[38] - (c[38] - c[39]) / (1.0 + t * t);
    const double k2 = c[34] * kcasr;
    rate[18] = -k2 * Cass * Rp + c[36] * (1.0 - Rp);
    const double k1 = c[33] / kcasr;
    const double O = (k1 * (Cass * Cass) * Rp) / (c[35] + k1 * (Cass * Cass));
    const double j_rel = c[40] * O * (Casr - Cass);
    const double bufsr = 1.0 / (1.0 + (c[47] * c[48]) / ((Casr + c[48]) * (Casr + c[48])));
    rate[17] = bufsr * (j_up - (j_rel + j_leak));
    const double bufss = 1.0 / (1.0 + (c[49] * c[50]) / ((Cass + c[50]) * (Cass + c[50])));
    rate[10] = bufss * (((-i_cal * c[3]) / (2.0 * c[52] * F) + (j_rel * c[51]) / c[52])
                        - (j_xfer * c[4]) / c[52]);
}

/* LAPACK-convention dense solve (column-major, partial pivoting, the
 * textbook getf2 elimination followed by the two triangular solves).  The
 * reference calls dgesv_ on its Jacobian stored as J[j*6+i] = df_j/dx_i,
 * which column-major reads as the TRANSPOSE; callers keep that layout. */
static int lu_solve6(double *a, double *b)
{
    const int n = 6;
    int piv[6], info = 0;
    for (int k = 0; k < n; k++) {
        int p = k; double amax = fabs(a[k + k * n]);
        for (int i = k + 1; i < n; i++) {
            double v = fabs(a[i + k * n]);
            if (v > amax) { amax = v; p = i; }
        }
        piv[k] = p;
        if (a[p + k * n] != 0.0) {
            if (p != k)
                for (int jj = 0; jj < n; jj++) {
                    double tmp = a[k + jj * n]; a[k + jj * n] = a[p + jj * n]; a[p + jj * n] = tmp;
                }
            double r = 1.0 / a[k + k * n];
            for (int i = k + 1; i < n; i++) a[i + k * n] *= r;
        } else if (info == 0) {
            info = k + 1;
        }
        for (int jj = k + 1; jj < n; jj++) {
            double ukj = a[k + jj * n];
            if (ukj != 0.0)
                for (int i = k + 1; i < n; i++) a[i + jj * n] -= a[i + k * n] * ukj;
        }
    }
    if (info) return info;
    for (int k = 0; k < n; k++)
        if (piv[k] != k) { double tmp = b[k]; b[k] = b[piv[k]]; b[piv[k]] = tmp; }
    for (int jj = 0; jj < n; jj++)            /* L y = b (unit lower) */
        if (b[jj] != 0.0)
            for (int i = jj + 1; i < n; i++) b[i] -= b[jj] * a[i + jj * n];
    for (int jj = n - 1; jj >= 0; jj--) {     /* U x = y */
        if (b[jj] != 0.0) {
            b[jj] /= a[jj + jj * n];
            for (int i = 0; i < jj; i++) b[i] -= b[jj] * a[i + jj * n];
        }
    }
    return 0;
}

/* Tusscher::UpdateStateVariables + Compute_Ion (Tusscher.cc:116-213). */
double epo_tt_compute_ion(double *s, const double *c, double Xi, double Cm,
                          double dt, double V, double istim, int newton_cap,
                          int jac_true, int *iters)
{
    double ginf[12], gtau[12], rate[19];
    double xn[6], old[6], fp[6], fm[6], J[36], B[6];
    const double ist = -istim / (Cm * Xi);
    s[0] = V;
    for (int i = 0; i < 6; i++) xn[i] = s[TT_NR[i]];

    tt_rates(s, c, ist, ginf, gtau, rate);
    for (int g = 0; g < 12; g++) {
        const double b = -1.0 / gtau[g];
        const double a = ginf[g] / gtau[g];
        s[TT_GATE[g]] = (s[TT_GATE[g]] + dt * a) / (1.0 - dt * b);
    }
    tt_rates(s, c, ist, ginf, gtau, rate);
    for (int i = 0; i < 6; i++) old[i] = rate[TT_NR[i]];

    double resid = 100.0;
    int it = 0;
    while (resid > 1e-6) {
        if (newton_cap > 0 && it >= newton_cap) break;
        for (int i = 0; i < 6; i++) {
            const int si = TT_NR[i];
            const double eps = 1e-3 * s[si];
            const double twoeps = 2.0 * eps;
            s[si] += eps;
            tt_rates(s, c, ist, ginf, gtau, rate);
            for (int k = 0; k < 6; k++) fp[k] = s[TT_NR[k]] - xn[k] - dt * rate[TT_NR[k]];
            s[si] -= 2.0 * eps;
            tt_rates(s, c, ist, ginf, gtau, rate);
            for (int k = 0; k < 6; k++) fm[k] = s[TT_NR[k]] - xn[k] - dt * rate[TT_NR[k]];
            s[si] += eps;
            for (int k = 0; k < 6; k++) {
                const double v = (fp[k] - fm[k]) / twoeps;
                if (jac_true) J[i * 6 + k] = v;   /* column-major J(k,i) */
                else J[k * 6 + i] = v;            /* the reference's layout */
            }
        }
        for (int i = 0; i < 6; i++) B[i] = s[TT_NR[i]] - xn[i] - dt * old[i];
        lu_solve6(J, B);
        for (int i = 0; i < 6; i++) s[TT_NR[i]] -= B[i];
        tt_rates(s, c, ist, ginf, gtau, rate);
        for (int i = 0; i < 6; i++) old[i] = rate[TT_NR[i]];
        resid = 0.0;
        for (int i = 0; i < 6; i++) resid += B[i] * B[i];
        resid = sqrt(resid);
        it++;
    }
    if (iters) *iters = it;
    return rate[0];
}

/* ====================================================================== */
/* Mahajan 2008 UCLA rabbit -- Mahajan.cc, SetUpIonicConstants.h:159-315   */
/* ====================================================================== */

void epo_mh_constants(double *c, int pos, int failing)
{
    if (!failing) {
        c[0] = 136.0; c[1] = 140.0; c[2] = 5.4; c[3] = 1.8; c[4] = 182.0; c[5] = 1.0; c[6] = 0.04;
        switch (pos) {
        case 0: c[7] = 0.11; c[10] = 1.9 * 0.32; break;
        case 1: c[7] = 0.11; c[10] = 1.4 * 0.32; break;
        case 2: c[7] = 0.11; c[10] = 1.0 * 0.32; break;
        case 3: c[7] = 0.11; c[10] = 0.74 * 0.32; break;
        case 4: c[7] = 0.11; c[10] = 0.52 * 0.32; break;
        case 5: c[7] = 0.11; c[10] = 0.35 * 0.32; break;
        case 6: c[7] = 0.11 * .85; c[10] = 0.98 * 0.32; break;
        case 7: c[7] = 0.11 * .85; c[10] = 0.7 * 0.32; break;
        case 8: c[7] = 0.11 * .85; c[10] = 0.5 * 0.32; break;
        default: c[7] = 0.11; c[10] = 0.32;
        }
        c[8] = 0.84; c[9] = 0.0125; c[11] = 0.3; c[12] = 1.5; c[13] = 0.4; c[14] = 4.0;
        c[15] = 12.0; c[16] = 30.0; c[17] = 100.0; c[18] = 11.3; c[19] = 90.0;
        c[20] = 308.; c[21] = -80.; c[22] = 8.314; c[23] = 96.485;
        c[24] = c[23] / (c[22] * c[20]);
        c[25] = 153; c[26] = 50; c[27] = 1.0; c[28] = 1.0; c[29] = 1.0; c[30] = 1.0;
        c[31] = 0.0; c[32] = 0.0; c[33] = 0.0; c[34] = 1.0;
    } else {
        c[0] = 136.0; c[1] = 140.0; c[2] = 5.4; c[3] = 1.8; c[4] = 182.0; c[5] = 1.0;
        c[6] = 0.04 * 0.65;
        switch (pos) {
        case 0: c[7] = 0.12; c[10] = 1.5 * 0.1386; break;
        case 1: c[7] = 0.12; c[10] = 1.3 * 0.1386; break;
        case 2: c[7] = 0.12; c[10] = 1.1 * 0.1386; break;
        case 3: c[7] = 0.12; c[10] = 1.0 * 0.1386; break;
        case 4: c[7] = 0.12; c[10] = 0.9 * 0.1386; break;
        case 5: c[7] = 0.12; c[10] = 0.8 * 0.1386; break;
        case 6: c[7] = 0.12 * 0.77; c[10] = 1.1 * 0.1386; break;
        case 7: c[7] = 0.12 * 0.77; c[10] = 1.0 * 0.1386; break;
        case 8: c[7] = 0.12 * 0.77; c[10] = 0.9 * 0.1386; break;
        default: c[7] = 0.12; c[10] = 0.1386;
        }
        c[7] *= 0.67; c[8] = 0.84 * 2.0; c[9] = 0.0125; c[10] *= 0.6; c[11] = 0.3 * 0.5;
        c[12] = 1.5; c[13] = 0.27; c[14] = 6.0; c[15] = 12.0; c[16] = 30.0; c[17] = 200.0;
        c[18] = 22.5; c[19] = 50.0; c[20] = 308.; c[21] = -80.; c[22] = 8.314; c[23] = 96.485;
        c[24] = c[23] / (c[22] * c[20]);
        c[25] = 153; c[26] = 10; c[27] = 1.0; c[28] = 1.0; c[29] = 1.0; c[30] = 1.0;
        c[31] = 0.01; c[32] = 0.01; c[33] = 0.01; c[34] = 1.0;
    }
}

void epo_mh_initial_state(double *s, int pos)
{
    static const double init[9][26] = {
        {-81.4359, 0.002789, 0.96679, 0.97859, 0.014994, 0.044487, 0.091992, 2.1933, 0.23277,
         0.24868, 101.6418, 95.4278, 0.009495, 3.7e-005, 0.96094, 0.003718, 6.7e-005, 0.010571,
         0.024659, 11.5909, 0.00533, 0.99047, 0.005333, 0.17488, 21.5955, 20.0206},
        {-81.3846, 0.002813, 0.96642, 0.97829, 0.015109, 0.04988, 0.10153, 2.3513, 0.23616,
         0.2529, 102.5325, 96.0961, 0.010394, 3.7e-005, 0.95815, 0.004448, 6.7e-005, 0.01261,
         0.024683, 11.442, 0.005349, 0.99012, 0.005352, 0.17323, 21.8749, 20.2219},
        {-81.3238, 0.002841, 0.96596, 0.97791, 0.015254, 0.056799, 0.11328, 2.5207, 0.23954,
         0.25736, 103.4612, 96.8014, 0.011385, 3.7e-005, 0.95449, 0.005413, 6.7e-005, 0.015284,
         0.024706, 11.2566, 0.00537, 0.98962, 0.005373, 0.17158, 22.1689, 20.4268},
        {-81.2657, 0.002868, 0.96553, 0.97752, 0.015406, 0.064019, 0.12504, 2.6684, 0.24235,
         0.26131, 104.2505, 97.4054, 0.01227, 3.7e-005, 0.95055, 0.006458, 6.8e-005, 0.018158,
         0.024723, 11.0791, 0.005391, 0.98902, 0.005394, 0.17018, 22.4276, 20.6034},
        {-81.1929, 0.002903, 0.96497, 0.97694, 0.015625, 0.073994, 0.14059, 2.8407, 0.2456,
         0.26605, 105.1459, 98.097, 0.013328, 3.7e-005, 0.94486, 0.00798, 6.8e-005, 0.022313,
         0.024742, 10.8644, 0.005417, 0.98806, 0.005421, 0.16859, 22.7359, 20.8156},
        {-81.1078, 0.002944, 0.96431, 0.97609, 0.01595, 0.087401, 0.1603, 3.0189, 0.24905,
         0.27153, 106.0478, 98.7911, 0.014455, 3.8e-005, 0.93663, 0.010192, 6.8e-005, 0.028302,
         0.024766, 10.6216, 0.005448, 0.98648, 0.005452, 0.16682, 23.0895, 21.0607},
        {-81.2626, 0.00287, 0.9655, 0.97756, 0.015387, 0.061634, 0.12278, 2.7185, 0.24183,
         0.2588, 104.2029, 97.6338, 0.01267, 3.7e-005, 0.95198, 0.006047, 6.8e-005, 0.017057,
         0.024804, 11.0783, 0.005392, 0.98941, 0.005395, 0.16991, 22.2542, 20.5438},
        {-81.1873, 0.002905, 0.96493, 0.97701, 0.015593, 0.071141, 0.13799, 2.9031, 0.24508,
         0.26334, 105.1225, 98.3761, 0.013821, 3.7e-005, 0.94672, 0.007447, 6.8e-005, 0.020885,
         0.024838, 10.8496, 0.005419, 0.9886, 0.005422, 0.16858, 22.5504, 20.7522},
        {-81.1085, 0.002943, 0.96432, 0.97631, 0.015852, 0.082505, 0.15518, 3.0765, 0.2482,
         0.26807, 105.9653, 99.0544, 0.01493, 3.8e-005, 0.94008, 0.009226, 6.8e-005, 0.025709,
         0.024873, 10.6197, 0.005448, 0.98743, 0.005451, 0.16728, 22.8568, 20.9674}};
    const int p = (pos >= 0 && pos < 9) ? pos : 2;   /* default case == pos 2 */
    memcpy(s, init[p], sizeof init[p]);
}

/* ucla_rhsfun and its current routines (Mahajan.cc:168-603). */
static void mh_rhs(const double *s, const double *c, double h, double istim, double *r)
{
    const double V = s[0], frt = c[24];
    /* ---- I_K1 (comp_ik1) ---- */
    const double ek1 = (1.0 / frt) * log((100.0 * c[2] + 1.0 * c[0]) / (100.0 * c[1] + 1.0 * s[19]));
    const double gki = sqrt(c[2] / 5.4);
    const double aki = 1.02 / (1.0 + exp(0.2385 * (V - ek1 - 59.215)));
    const double bki = (0.49124 * exp(0.08032 * (V - ek1 + 5.476)) + exp(0.061750 * (V - ek1 - 594.31)))
                     / (1.0 + exp(-0.5143 * (V - ek1 + 4.753)));
    const double xik1 = c[11] * gki * (aki / (aki + bki)) * (V - ek1);
    /* ---- I_to slow + fast (comp_ito) ---- */
    const double ek = 1.0 / frt * log(c[2] / c[1]);
    const double rt1 = -(V + 3.0) / 15.0, rt2 = (V + 33.5) / 10.0, rt3 = (V + 60.0) / 10.0;
    const double xtos_inf = 1.0 / (1.0 + exp(rt1));
    const double ytos_inf = 1.0 / (1.0 + exp(rt2));
    const double rs_inf = 1.0 / (1.0 + exp(rt2));
    const double txs = 9.0 / (1.0 + exp(-rt1)) + 0.5;
    const double tys = 3000.0 / (1.0 + exp(rt3)) + 30.0;
    const double xitos = c[6] * s[22] * (s[23] + 0.5 * rs_inf) * (V - ek);
    r[22] = (xtos_inf - (xtos_inf - s[22]) * exp(-h / txs) - s[22]) / h;
    r[23] = (ytos_inf - (ytos_inf - s[23]) * exp(-h / tys) - s[23]) / h;
    const double rt4 = -(V / 30.0) * (V / 30.0), rt5 = (V + 33.5) / 10.0;
    const double txf = 3.5 * exp(rt4) + 1.5;
    const double tyf = 20.0 / (1.0 + exp(rt5)) + 20.0;
    const double xitof = c[7] * s[20] * s[21] * (V - ek);
    r[20] = (xtos_inf - (xtos_inf - s[20]) * exp(-h / txf) - s[20]) / h;
    r[21] = (ytos_inf - (ytos_inf - s[21]) * exp(-h / tyf) - s[21]) / h;
    const double xito = xitos + xitof;
    /* ---- I_NaK (comp_inak) ---- */
    const double sigma = (exp(c[0] / 67.3) - 1.0) / 7.0;
    const double fnak = 1.0 / (1 + 0.1245 * exp(-0.1 * V * frt) + 0.0365 * sigma * exp(-V * frt));
    const double xinak = c[12] * fnak * (1. / (1. + (12.0 / s[19]))) * c[2] / (c[2] + 1.5);
    /* ---- I_NaCa flux (comp_inaca) ---- */
    double jnaca;
    {
        const double csm = s[8] / 1000.0;
        const double na3 = pow(s[19], 3), nao3 = pow(c[0], 3);
        const double zw3 = na3 * c[3] * exp(V * 0.35 * frt) - nao3 * csm * exp(V * (0.35 - 1.) * frt);
        const double zw4 = 1.0 + 0.2 * exp(V * (0.35 - 1.0) * frt);
        const double aloss = 1.0 / (1.0 + pow((0.3 / s[8]), 3));
        const double yz1 = 1.3 * na3 + pow(87.5, 3) * csm;
        const double yz2 = pow(12.3, 3) * c[3] * (1.0 + csm / 0.0036);
        const double yz3 = 0.0036 * nao3 * (1.0 + pow((s[19] / 12.3), 3));
        const double yz4 = na3 * c[3] + nao3 * csm;
        jnaca = c[8] * aloss * zw3 / (zw4 * (yz1 + yz2 + yz3 + yz4));
    }
    /* ---- Ca cycling ---- */
    const double jd = c[28] * (s[8] - s[9]) / c[14];
    r[24] = c[29] * (0.0327 * s[9] * (70.0 - s[24]) - 0.0196 * s[24]);
    r[25] = 0.0327 * s[8] * (70.0 - s[25]) - 0.0196 * s[25];
    const double jup = c[30] * (c[13] * s[9] * s[9] / (s[9] * s[9] + 0.5 * 0.5));
    const double jleak = c[27] * (0.00002069 * s[10] * s[10] / (s[10] * s[10] + 50.0 * 50.0)
                                  * (s[10] * 16.667 - s[9]));
    /* ---- Markov L-type Ca channel (comp_icalpo) ---- */
    double po;
    {
        const double poinf = 1.0 / (1.0 + exp(-(V - 0.0) / 8.0));
        const double alpha = poinf / 1.0, beta = (1.0 - poinf) / 1.0;
        const double r1 = 0.30, r2 = 3.0;
        const double fca = 1.0 / (1.0 + pow((double)(3.0 / s[7]), 3));
        const double s1 = 0.0182688 * fca;
        const double s1t = 0.00195;
        const double k1 = 0.024168 * fca;
        const double k2 = 1.03615e-4, k1t = 0.00413, k2t = 0.00224;
        const double s2 = s1 * (r1 / r2) * (k2 / k1);
        const double s2t = s1t * (r1 / r2) * (k2t / k1t);
        const double poi = 1.0 / (1.0 + exp(-(V - -40) / 3.0));
        const double k3 = (1.0 - poi) / 3.0, k3t = k3;
        const double Pr = 1.0 - 1.0 / (1.0 + exp(-(V - -40.0) / 4.0));
        const double recov = 10.0 + 4954.0 * exp(V / 15.6);
        const double tau_ca = 78.0329 / (1.0 + pow((s[7] / 6.09365), 4)) + 0.1;
        const double tauca = (recov - tau_ca) * Pr + tau_ca;
        const double tauba = (recov - 450.0) * Pr + 450.0;
        const double Ps = 1.0 / (1.0 + exp(-(V - -40.0) / 11.32));
        const double k6 = fca * Ps / tauca, k5 = (1.0 - Ps) / tauca;
        const double k6t = Ps / tauba, k5t = (1.0 - Ps) / tauba;
        const double k4 = k3 * (alpha / beta) * (k1 / k2) * (k5 / k6);
        const double k4t = k3t * (alpha / beta) * (k1t / k2t) * (k5t / k6t);
        po = 1.0 - s[15] - s[17] - s[16] - s[18] - s[13] - s[14];
        r[14] = beta * s[13] + k5 * s[17] + k5t * s[18] - (k6 + k6t + alpha) * s[14];
        r[13] = alpha * s[14] + k2 * s[15] + k2t * s[16] + r2 * po - (beta + r1 + k1t + k1) * s[13];
        r[15] = k1 * s[13] + k4 * s[17] + s1 * po - (k3 + k2 + s2) * s[15];
        r[17] = k3 * s[15] + k6 * s[14] - (k5 + k4) * s[17];
        r[16] = k1t * s[13] + k4t * s[18] + s1t * po - (k3t + k2t + s2t) * s[16];
        r[18] = k3t * s[16] + k6t * s[14] - (k5t + k4t) * s[18];
    }
    /* ---- driving force (comp_rxa) ---- */
    double rxa;
    {
        const double csm = s[8] / 1000.0;
        const double za = V * 2.0 * frt;
        const double factor1 = 4.0 * 0.00054 * c[23] * c[23] / (c[22] * c[20]);
        const double factor = V * factor1;
        if (fabs(za) < 0.001)
            rxa = factor1 * (csm * exp(za) - 0.341 * (c[3])) / (2.0 * frt);
        else
            rxa = factor * (csm * exp(za) - 0.341 * (c[3])) / (exp(za) - 1.0);
    }
    const double jca = c[4] * po * rxa;
    /* instantaneous buffers (comp_inst_buffer) */
#define MH_BUF(cv) (1.0 / (1.0 + 24.0 * 7.0 / ((7.0 + (cv)) * (7.0 + (cv))) \
                              + 47.0 * 0.6 / ((0.6 + (cv)) * (0.6 + (cv)))   \
                              + 15.0 * 0.3 / ((0.3 + (cv)) * (0.3 + (cv)))   \
                              + 42.0 * 13.0 / ((13.0 + (cv)) * (13.0 + (cv)))))
    r[8] = MH_BUF(s[8]) * (50.0 * (s[12] - jd - jca + jnaca) - r[25]);
    r[9] = MH_BUF(s[9]) * (jd - jup + jleak - r[24]);
#undef MH_BUF
    r[10] = -s[12] + jup - jleak;
    r[11] = (s[10] - s[11]) / c[17];
    /* release-load dependence (comp_Q) */
    double Qr;
    {
        const double bv = (c[19] - c[26]) - c[18] * c[19];
        double q = 0;
        if (s[11] > c[26] && s[11] < c[19]) q = s[11] - c[26];
        else if (s[11] >= c[19]) q = c[18] * s[11] + bv;
        if (q >= c[25]) q = c[25];
        Qr = s[10] * q / c[19];
    }
    /* comp_dir */
    {
        const double sparkV = exp(-0.05 * (V + 30)) / (1. + exp(-0.05 * (V + 30)));
        const double spark_rate = 2.58079 * po * fabs(rxa) * sparkV;
        r[12] = spark_rate * Qr - s[12] * (1 - c[16] * r[10] / s[10]) / c[16];
    }
    /* comp_dcp */
    {
        const double gsr = 26841.8 * exp(-0.3576 * (V + 30)) / (1.0 + exp(-0.3576 * (V + 30)));
        const double xirp = po * Qr * fabs(rxa) * gsr;
        const double xicap = po * 9000.0 * fabs(rxa);
        r[7] = xirp + xicap - (s[7] - s[8]) / 0.5;
    }
    /* ---- I_Na (comp_ina) ---- */
    double xina;
    {
        const double ena = (1.0 / frt) * log(c[0] / s[19]);
        double am = 3.2;
        if (fabs(V + 47.13) > 0.001) am = 0.32 * (V + 47.13) / (1.0 - exp(-0.1 * (V + 47.13)));
        const double bm = 0.08 * exp(-V / 11.0);
        const double a = 1.0 - 1.0 / (1.0 + exp(-(V + 40.0) / 0.24));
        const double ah = a * 0.135 * exp((80.0 + V) / (-6.8));
        const double bh = (1.0 - a) / (0.13 * (1 + exp((V + 10.66) / (-11.1))))
                        + a * (3.56 * exp(0.079 * V) + 3.1 * 1.0e5 * exp(0.35 * V));
        const double aj = a * (-1.2714e5 * exp(0.2444 * V) - 3.474e-5 * exp(-0.04391 * V)) * (V + 37.78)
                        / (1.0 + exp(0.311 * (V + 79.23)));
        const double bj = (1.0 - a) * (0.3 * exp(-2.535e-7 * V) / (1 + exp(-0.1 * (V + 32))))
                        + a * (0.1212 * exp(-0.01052 * V) / (1 + exp(-0.1378 * (V + 40.14))));
        const double tauh = 1.0 / (ah + bh);
        const double tauj = c[34] * 1.0 / (aj + bj);
        const double taum = 1.0 / (am + bm);
        xina = c[15] * (s[2] + c[32]) / (1 + c[32]) * (s[3] + c[33]) / (1 + c[33])
             * (s[1] + c[31]) / (1 + c[31]) * (s[1] + c[31]) / (1 + c[31])
             * (s[1] + c[31]) / (1 + c[31]) * (V - ena);
        r[2] = (ah * tauh - (ah * tauh - s[2]) * exp(-h / tauh) - s[2]) / h;
        r[3] = (aj * tauj - (aj * tauj - s[3]) * exp(-h / tauj) - s[3]) / h;
        r[1] = (am * taum - (am * taum - s[1]) * exp(-h / taum) - s[1]) / h;
    }
    /* ---- I_Kr (comp_ikr) ---- */
    double xikr;
    {
        const double ekr = (1.0 / frt) * log(c[2] / c[1]);
        const double gss = sqrt(c[2] / 5.4);
        double v1 = 0.00138 / 0.123;
        if (fabs(V + 7.0) > 0.001) v1 = 0.00138 * (V + 7.0) / (1. - exp(-0.123 * (V + 7.0)));
        double v2 = 0.00061 / 0.145;
        if (fabs(V + 10.0) > 0.001) v2 = 0.00061 * (V + 10.0) / (exp(0.145 * (V + 10.0)) - 1.0);
        const double taukr = 1.0 / (v1 + v2);
        const double xkrinf = 1.0 / (1.0 + exp(-(V + 50.0) / 7.5));
        const double rg = 1.0 / (1.0 + exp((V + 33.0) / 22.4));
        xikr = c[9] * gss * s[4] * rg * (V - ekr);
        r[4] = (xkrinf - (xkrinf - s[4]) * exp(-h / taukr) - s[4]) / h;
    }
    /* ---- I_Ks (comp_iks) ---- */
    double xiks;
    {
        const double prnak = 0.018330;
        const double eks = (1.0 / frt) * log((c[2] + prnak * c[0]) / (c[1] + prnak * s[19]));
        const double xs1ss = 1.0 / (1.0 + exp(-(V - 1.50) / 16.70));
        double tauxs1;
        if (fabs(V + 30.0) < 0.001 / 0.0687)
            tauxs1 = 1 / (0.0000719 / 0.148 + 0.000131 / 0.0687);
        else
            tauxs1 = 1.0 / (0.0000719 * (V + 30.0) / (1.0 - exp(-0.148 * (V + 30.0)))
                            + 0.000131 * (V + 30.0) / (exp(0.0687 * (V + 30.0)) - 1.0));
        const double tauxs2 = 4 * tauxs1;
        const double gksx = (1 + 0.8 / (1 + pow((0.5 / s[9]), 3)));
        xiks = c[10] * gksx * s[5] * s[6] * (V - eks);
        r[5] = (xs1ss - (xs1ss - s[5]) * exp(-h / tauxs1) - s[5]) / h;
        r[6] = (xs1ss - (xs1ss - s[6]) * exp(-h / tauxs2) - s[6]) / h;
    }
    const double wca = 8.0313;
    const double xinaca = wca * jnaca;
    const double xica = 2.0 * wca * jca;
    const double xrr = (1.0 / wca) / 1000.0;
    r[19] = (-xrr * (xina + 3.0 * xinak + 3.0 * xinaca));
    r[0] = (-(xina + xik1 + xikr + xiks + xito + xinaca + xica + xinak) + istim);
}

/* Mahajan::UpdateStateVariables + Compute_Ion (Mahajan.cc:607-645). */
double epo_mh_compute_ion(double *s, const double *c, double Xi, double Cm,
                          double dt, double V, double istim, int abs_mode,
                          int *substepped)
{
    double r[26];
    const double ist = istim / (Cm * Xi);
    s[0] = V;
    mh_rhs(s, c, dt, ist, r);
    const double mag = abs_mode ? fabs(r[0]) : (double)abs((int)r[0]);
    if (mag > 20.0) {
        for (int k = 0; k < 10; k++) {
            mh_rhs(s, c, dt / 10, ist, r);
            for (int j = 0; j < 26; j++) s[j] += r[j] * dt / 10;
        }
        if (substepped) *substepped = 1;
    } else {
        for (int j = 0; j < 26; j++) s[j] += r[j] * dt;
        if (substepped) *substepped = 0;
    }
    return r[0];
}

/* ====================================================================== */
/* Luo-Rudy -- LR.cc, LRGateTable.h                                        */
/* ====================================================================== */

#define LR_RT_F 26.73
static double lr_ek1(void) { return LR_RT_F * log(5.4 / 145.0); }

void epo_lr_initial_state(double *s)
{
    s[0] = .001; s[1] = 0.0001; s[2] = 0.99; s[3] = .001; s[4] = 0.9; s[5] = .001;
    s[6] = 0.0000001; s[7] = 0;
}

/* LuoRudy::make_parameter1 (LR.cc:102-183) */
void epo_lr_params(double v, double *tab)
{
    double am, bm, ah, bh, aj, bj, x1;
    const double E_K1 = lr_ek1();
    const double G_K1 = .6047 * sqrt(5.4 / 5.4);
    if (fabs(v + 47.13) < 0.001) am = 3.2;
    else am = 0.32 * (v + 47.13) / (1.0 - exp(-0.1 * (v + 47.13)));
    bm = 0.08 * exp(-v / 11.);
    if (v > -40.) {
        ah = 0; aj = 0;
        bh = 1. / (0.13 * (1 + exp(-(v + 10.66) / 11.1)));
        bj = 0.3 * exp(-2.535e-7 * v) / (1 + exp(-0.1 * (v + 32)));
    } else {
        ah = 0.135 * exp(-(80 + v) / 6.8);
        aj = (-1.2714e5 * exp(0.2444 * v) - 3.474e-5 * exp(-0.04391 * v)) * (v + 37.78)
           / (1 + exp(0.311 * (v + 79.23)));
        bh = 3.56 * exp(0.079 * v) + 3.1e5 * exp(0.35 * v);
        bj = 0.1212 * exp(-0.01052 * v) / (1 + exp(-0.1378 * (v + 40.14)));
    }
    const double ad = .095 * exp(-.01 * (v - 5)) / (1 + exp(-.072 * (v - 5)));
    const double bd = .07 * exp(-.017 * (v + 44)) / (1 + exp(.05 * (v + 44)));
    const double af = .012 * exp(-.008 * (v + 28)) / (1 + exp(.15 * (v + 28)));
    const double bf = .0065 * exp(-.02 * (v + 30)) / (1 + exp(-.2 * (v + 30)));
    const double ax = .0005 * exp(.083 * (v + 50)) / (1 + exp(.057 * (v + 50)));
    const double bx = .0013 * exp(-.06 * (v + 20)) / (1 + exp(-.04 * (v + 20)));
    const double tm = am + bm, th = ah + bh, tj = aj + bj;
    const double td = ad + bd, tf = af + bf, tx = ax + bx;
    if (v > -100) {
        if (fabs(v + 77.) < 0.001) x1 = 0.608889;
        else x1 = 2.837 * (exp(0.04 * (v + 77)) - 1) / ((v + 77) * exp(0.04 * (v + 35)));
    } else x1 = 1.;
    const double ak1 = 1.02 / (1 + exp(0.2385 * (v - E_K1 - 59.215)));
    const double b1 = 0.49124 * exp(0.08032 * (v - E_K1 + 5.476));
    const double b2 = exp(0.06175 * (v - E_K1 - 594.31));
    const double b3 = 1 + exp(-0.5143 * (v - E_K1 + 4.753));
    const double bk1 = (b1 + b2) / b3;
    const double k1_inf = ak1 / (ak1 + bk1);
    const double I_k1 = G_K1 * k1_inf * (v - E_K1);
    const double kp = 1. / (1 + exp((7.488 - v) / 5.98));
    const double I_kp = 0.0183 * kp * (v - E_K1);
    const double I_b = 0.0392 * (v + 59.87);
    tab[0] = am / tm; tab[1] = tm; tab[2] = ah / th; tab[3] = th; tab[4] = aj / tj; tab[5] = tj;
    tab[6] = ad / (ad + bd); tab[7] = td; tab[8] = af / (af + bf); tab[9] = tf;
    tab[10] = ax / (ax + bx); tab[11] = tx; tab[12] = x1; tab[13] = I_k1 + I_kp + I_b;
}

double *epo_lr_gate_table(void)
{
    double *t = (double *)malloc(sizeof(double) * 290001 * 14);
    if (!t) return NULL;
    for (int i = 0; i < 290001; i++) epo_lr_params(-90 + 0.001 * i, t + 14 * (size_t)i);
    return t;
}

/* LuoRudy::Compute_Ion (LR.cc:65-100); table != NULL selects the gate
 * table path (LRGateTable.h:96-110, linear interpolation). */
double epo_lr_compute_ion(double *s, const double *table, double Xi_unused,
                          double Cm, double dt, double V, double istim)
{
    (void)Xi_unused;
    double tab[14];
    const double Xi = 2. * (11e-4 + 100E-4) / (11e-4 * 100E-4);
    const double GK = 0.705 * sqrt(5.4 / 5.4);
    s[7] = V;
    if (table && V > -90 && V < 200) {
        const int idx = (int)((V + 90) * 1000);
        const double w = 1000 * (V - (-90 + 0.001 * idx));
        const double *t0 = table + 14 * (size_t)idx, *t1 = t0 + 14;
        for (int i = 0; i < 14; i++) tab[i] = (t1[i] - t0[i]) * w + t0[i];
    } else {
        epo_lr_params(V, tab);
    }
    for (int i = 0; i < 6; i++) s[i] = tab[2 * i] - (tab[2 * i] - s[i]) * exp(-dt * tab[2 * i + 1]);
    const double Es = 7.7 - 13.0287 * log(s[6]);
    const double i_na = 12.00 * s[0] * s[0] * s[0] * s[1] * s[2] * (s[7] - 54.4);
    const double i_si = 0.07 * s[3] * s[4] * (s[7] - Es);
    const double i_k = GK * tab[12] * s[5] * (s[7] + 77.0);
    s[6] = s[6] + (-.0001 * i_si + 0.07 * (0.0001 - s[6])) * dt;
    const double i_tot = -(tab[13] + i_k + i_na + i_si);
    return (i_tot + istim / (Xi * Cm));
}

/* ====================================================================== */
/* Corrias 2011 rabbit Purkinje -- Purkinje.h/.cc, SetUpIonicConstants.h:16-85 */
/* ====================================================================== */

/* the 63-entry parameter set of SetUpPurkinjeParameters (SetUpIonicConstants.h:16-85);
 * [11..15] are the model's own pacing stimulus, unused on this path */
void epo_pk_constants(double *c)
{
    static const double base[57] = {
        310.0, 96485.3415, 8314.472, 2.0, 140, 5.4, 69.0, 13266.5, 0.6, 0.2,
        0.06, 700, 9000000, 500, 0.5, -4320.0, 1.0, 0.9, 0.7, 5.4,
        5.0, 350.0, 10.0, 3.0, 0.005, 2.0, 1140.0, 15.0, 2.0, 20.0,
        1.5, 3.0, 3, 0.001, 0.001, 0.5, 442.2, 0.01, 0.01, 0.0001,
        5.0, 0.0001, 1.5, 0.188709677, 0.045290323, 2500.0, 0.001, 120.0, 0.000246, 1.7,
        1.6, 120.0, 0.000246, 1.7, 1.6, 10.0, 5000.0};
    for (int k = 0; k < 57; k++) c[k] = base[k];
    c[57] = c[1] / (c[2] * c[0]);          /* F/RT */
    c[58] = (c[2] * c[0]) / c[1];          /* RT/F */
    c[59] = c[9] * c[7];                   /* the three compartment volumes */
    c[60] = c[8] * c[7];
    c[61] = (c[8] + c[9]) * c[7];
    c[62] = c[10] * c[7];
}

/* Purkinje.h:43-51 */
void epo_pk_initial_state(double *s)
{
    static const double s0[EPO_PK_NSTATE] = {
        -88.34, 0.00001, 0.000032, 0.17, 6.7, 140, 0.001337, 0.01, 0.000003, 0.1,
        0.7, 0.0, 0.7, 0.000007, 0.978861, 0.000012, 0.864489, 0.25, 1.0, 0.0,
        0.011099, 0.011099};
    for (int k = 0; k < EPO_PK_NSTATE; k++) s[k] = s0[k];
}

/* Purkinje::ComputeRates (Purkinje.cc:5-103): r[0] = dV/dt, the gates relax
 * to their steady states, the ion concentrations follow the currents.
 * istim_pA enters the balances as the reference's Algebraic[0]. */
static void pk_rates(const double *s, const double *c, double istim_pA, double *r)
{
    const double V = s[0];
    /* gates: steady state and time constant */
    const double ss6 = 1.0 / (1.0 + exp((V + 47.8) / -5.5));
    const double ss8 = 1.0 / (1.0 + exp((V + 14.6) / -5.5));
    const double ss11 = 1.0 / (1.0 + exp((V + -7.0) / -9.0));
    const double ss12 = 1.0 / (1.0 + exp((V + 27.5) / 8.0));
    const double ss13 = 1.0 / (1.0 + exp((V + 25.0) / -5.0));
    const double ss14 = 1.0 / (1.0 + exp((V + 69.0) / 3.96));
    const double ss15 = 1.0 / (1.0 + exp((V + 30.0) / -5.0));
    const double ss7 = 1.0 / (1.0 + exp((V + 67.9) / 3.87));
    const double tau7 = 1.42271 * exp(-0.05119 * V);
    const double ss9 = 1.0 / (1.0 + exp((V + 31.0) / 5.54));
    const double tau9 = 25.1 / (0.04 + 0.7 * exp(-1.0 * pow(0.028 * (V + 14.5), 2.0)));
    const double cai_f = 1.0 + pow(s[1] / 0.0001, 2.0);
    const double ss10 = 0.4 + 0.6 / cai_f;
    const double tau10 = 2.0 + 80.0 / cai_f;
    const double ss16 = 0.1 + 0.9 / (1.0 + exp((V + 75.6) / 6.3));
    const double tau16 = 120.0 + 1.0 * exp((V + 100.0) / 25.0);
    const double ss18 = 1.0 / (1.0 + exp((V - 1.5) / -16.7));
    const double v30 = V + 30.0;
    const double tau18 = fabs(v30) < 0.0145 ? 417.946
        : 1.0 / ((7.19e-05 * v30) / (1.0 - exp(-0.148 * v30)) + (0.000131 * v30) / (exp(0.0687 * v30) - 1.0));
    const double ss_f = 1.0 / (1.0 + exp((V + 109.0) / 10.0));       /* s20 and s21 */
    const double tau_f = 6000.0 / (exp(-1.0 * (2.9 + 0.04 * V)) + exp(1.0 * (3.6 + 0.11 * V)));
    const double ss17 = 1.0 / (1.0 + exp((V + 50.0) / -7.5));
    const double v7 = V + 7.0, v10 = V + 10.0;
    const double al17 = fabs(v7) > 0.001 ? (0.00138 * 1.0 * v7) / (1.0 - exp(-0.123 * v7)) : 0.00138 / 0.123;
    const double be17 = fabs(v10) > 0.001 ? (6.1e-05 * 1.0 * v10) / (exp(0.145 * v10) - 1.0) : 0.00061 / 0.145;
    const double tau17 = 1.0 / (al17 + be17);
    r[6] = (ss6 - s[6]) / c[16];
    r[8] = (ss8 - s[8]) / c[18];
    r[11] = (ss11 - s[11]) / c[20];
    r[12] = (ss12 - s[12]) / c[21];
    r[13] = (ss13 - s[13]) / c[24];
    r[14] = (ss14 - s[14]) / c[25];
    r[15] = (ss15 - s[15]) / c[27];
    r[7] = (ss7 - s[7]) / tau7;
    r[9] = (ss9 - s[9]) / tau9;
    r[10] = (ss10 - s[10]) / tau10;
    r[16] = (ss16 - s[16]) / tau16;
    r[18] = (ss18 - s[18]) / tau18;
    r[20] = (ss_f - s[20]) / tau_f;
    r[21] = (ss_f - s[21]) / tau_f;
    r[17] = (ss17 - s[17]) / tau17;
    r[19] = (ss18 - s[19]) / (4.0 * tau18);
    /* reversal potentials */
    const double RTF = c[58];
    const double EK = RTF * log(c[5] / s[5]);
    const double ENa = RTF * log(c[4] / s[4]);
    const double ECa = 0.5 * RTF * log(c[3] / s[1]);
    /* potassium currents */
    const double iK1 = c[29] * pow(c[5] / 5.4, 0.8) * (1.0 / (1.0 + exp((92.0 + V) / 10.0))) * (V - EK);
    const double ito = c[22] * s[11] * s[12] * (V - EK);
    const double iKp = c[23] * (1.0 / (1.0 + exp((5.0 - V) / 17.0))) * (V - EK);
    const double iKr = c[30] * pow(c[5] / 5.4, 1.0) * (1.0 / (1.0 + exp((33.0 + V) / 22.4))) * s[17] * (V - EK);
    const double iKs = c[31] * s[18] * s[19] * (V - EK);
    const double iKb = c[37] * (V - EK);
    const double iNaK = c[36] * (1.0 / (1.0 + exp((V + 80.0) / -45.0))) * (1.0 / (1.0 + exp((V + 0.0) / 125.0))) *
                        (1.0 / (1.0 + pow(1.9 / c[5], 1.45))) * (1.0 / (1.0 + pow(31.98 / s[4], 1.0)));
    const double ifK = c[43] * s[20] * (V - EK);
    /* calcium and sodium currents */
    const double iCaL = c[19] * s[8] * s[9] * s[10] * (V - ECa);
    const double iCaT = c[17] * s[6] * s[7] * (V - ECa);
    const double iNa = c[26] * s[13] * s[14] * (V - ENa);
    const double iNaL = c[28] * s[15] * s[16] * (V - ENa);
    const double ipCa = c[40] * (1.0 / (1.0 + pow(c[41] / s[1], c[42])));
    const double iCab = c[39] * (V - ECa);
    const double ifNa = c[44] * s[21] * (V - ENa);
    const double iNaCa = (512.009 * c[33] *
                          (exp((c[35] * (c[32] - 2.0) * V) / RTF) * pow(s[4], c[32]) * c[3] -
                           s[1] * exp(((c[35] - 1.0) * (c[32] - 2.0) * V) / RTF) * pow(c[4], c[32]))) /
                         ((1.0 + c[34] * (s[1] * pow(c[4], c[32]) + c[3] * pow(s[4], c[32]))) * (1.0 + s[1] / 0.0069));
    const double iNab = c[38] * (V - ENa);
    r[5] = ((-ito - iKp - iKr - iKs - iK1 - iKb - ifK - istim_pA + 2.0 * iNaK) * 1000.0) / (c[1] * c[61]);
    r[0] = ((-1.0 * 1.0) / c[6]) * (iK1 + ito + iKp + iKr + iKs + iKb + iNaK + iCaL + iCaT + iNa + iNaL + ipCa +
                                     iCab + ifNa + ifK + iNaCa + iNab + istim_pA);
    /* calcium handling: release, two uptakes, transfer */
    const double jrel = c[45] * (s[3] / (1.0 + pow(c[46] / s[1], 2.0)));
    const double jup1 = c[47] * ((pow(s[1] / c[48], c[50]) - pow(s[3] / c[49], c[50])) /
                                 (1.0 + pow(s[1] / c[48], c[50]) + pow(s[3] / c[49], c[50])));
    const double jup2 = c[51] * ((pow(s[2] / c[52], c[54]) - pow(s[3] / c[53], c[54])) /
                                 (1.0 + pow(s[2] / c[52], c[54]) + pow(s[3] / c[53], c[54])));
    const double jtr = c[55] * (s[3] - s[2]);
    const double jdiff = c[56] * (s[1] - s[2]);
    r[3] = ((-jrel - jtr + jup2 + jup1) * 1000.0) / (2.0 * c[1] * c[62]);
    r[4] = ((-iNa - iNaL - 3.0 * iNaK - 3.0 * iNaCa - ifNa - iNab) * 1000.0) / (c[1] * c[61]);
    r[1] = ((-iCaL - iCaT - iCab + 1.0 * jrel - jup1 - jdiff + 2.0 * iNaCa - ipCa) * 1000.0) / (2.0 * c[1] * c[59]);
    r[2] = ((-jup2 + jdiff + jtr) * 1000.0) / (2.0 * c[1] * c[60]);
}

/* Purkinje::Compute_Ion + UpdateStateVariables (Purkinje.cc:183-213,
 * 157-173): V into State[0], the stimulus [uA/cm^3] as pA through the cell's
 * surface area (4.612e-5 cm^2) and Xi, then one forward-Euler step of dt --
 * or ten of dt/10 when |dV/dt| > 1.5 mV/ms at the start.  Every state,
 * V included, is advanced; the returned dV/dt is the last evaluated rate.
 * C_m is not used by the model. */
double epo_pk_compute_ion(double *s, const double *c, double Xi, double dt, double V, double istim,
                          int *substepped)
{
    double r[EPO_PK_NSTATE];
    s[0] = V;
    const double istim_pA = -1e6 * istim * 4.612e-5 / Xi;
    pk_rates(s, c, istim_pA, r);
    if (fabs(r[0]) > 1.5) {
        for (int k = 0; k < 10; k++) {
            pk_rates(s, c, istim_pA, r);
            for (int j = 0; j < EPO_PK_NSTATE; j++) s[j] += r[j] * dt / 10;
        }
        if (substepped) *substepped = 1;
    } else {
        for (int j = 0; j < EPO_PK_NSTATE; j++) s[j] += r[j] * dt;
        if (substepped) *substepped = 0;
    }
    return r[0];
}

/* ====================================================================== */
/* population                                                              */
/* ====================================================================== */

epo_cells *epo_cells_create(int model, int n, const uint8_t *type, int ntypes,
                            const double *type_consts)
{
    epo_cells *c = (epo_cells *)calloc(1, sizeof(epo_cells));
    c->model = model; c->n = n; c->type = type; c->ntypes = ntypes > 0 ? ntypes : 1;
    c->newton_cap = 0; c->mh_abs_mode = 0;
    switch (model) {
    case EPO_TUSSCHER: c->nstate = EPO_TT_NSTATE; c->nconst = EPO_TT_NCONST; c->Xi = 2000.; break;
    case EPO_MAHAJAN: case EPO_MAHAJAN_FAIL:
        c->nstate = EPO_MH_NSTATE; c->nconst = EPO_MH_NCONST; c->Xi = 1.55E-4 / 2.58E-8; break;
    case EPO_PURKINJE: c->nstate = EPO_PK_NSTATE; c->nconst = EPO_PK_NCONST; c->Xi = 2500.; break;
    default: c->nstate = EPO_LR_NSTATE; c->nconst = 1;
        c->Xi = 2. * (11e-4 + 100E-4) / (11e-4 * 100E-4); break;
    }
    c->state = (double *)malloc(sizeof(double) * (size_t)n * c->nstate);
    c->consts = (double *)calloc((size_t)c->ntypes * c->nconst, sizeof(double));
    if (type_consts) memcpy(c->consts, type_consts, sizeof(double) * c->ntypes * c->nconst);
    else {
        for (int t = 0; t < c->ntypes; t++) {
            double *k = c->consts + (size_t)t * c->nconst;
            if (model == EPO_TUSSCHER) epo_tt_constants(k);
            else if (model == EPO_MAHAJAN) epo_mh_constants(k, t, 0);
            else if (model == EPO_MAHAJAN_FAIL) epo_mh_constants(k, t, 1);
            else if (model == EPO_PURKINJE) epo_pk_constants(k);
        }
    }
    if (model == EPO_TUSSCHER) c->alg12 = (double *)calloc((size_t)n, sizeof(double));
    if (model == EPO_LUORUDYWITHGATE) c->lr_table = epo_lr_gate_table();
    for (int i = 0; i < n; i++) {
        double *s = c->state + (size_t)i * c->nstate;
        int t = type ? type[i] : 0;
        if (model == EPO_TUSSCHER) epo_tt_initial_state(s);
        else if (model == EPO_MAHAJAN || model == EPO_MAHAJAN_FAIL) epo_mh_initial_state(s, t);
        else if (model == EPO_PURKINJE) epo_pk_initial_state(s);
        else epo_lr_initial_state(s);
    }
    return c;
}

void epo_cells_destroy(epo_cells *c)
{
    if (!c) return;
    free(c->state); free(c->consts); free(c->alg12); free(c->lr_table); free(c->gks_scale);
    free(c);
}

void epo_cells_initial_voltage(const epo_cells *c, double *V)
{
    for (int i = 0; i < c->n; i++) {
        const double *s = c->state + (size_t)i * c->nstate;
        V[i] = (c->model == EPO_LUORUDY || c->model == EPO_LUORUDYWITHGATE) ? s[7] : s[0];
    }
}

void epo_cells_compute_ion(epo_cells *c, double Cm, double dt, const double *V,
                           const double *istim, double *dvdt)
{
    const int n = c->n;
    long long ntot = 0, nmax = 0, nsub = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+:ntot, nsub) reduction(max:nmax)
    for (int i = 0; i < n; i++) {
        double *s = c->state + (size_t)i * c->nstate;
        const int t = c->type ? c->type[i] : 0;
        const double *k = c->consts + (size_t)t * c->nconst;
        const double Xi = c->user_xi ? c->user_Xi : c->Xi;
        if (c->model == EPO_TUSSCHER) {
            int it = 0;
            double kk[EPO_TT_NCONST];
            const double *kp = k;
            if (c->gks_scale) {
                memcpy(kk, k, sizeof kk);
                kk[15] *= c->gks_scale[i];
                kp = kk;
            }
            dvdt[i] = epo_tt_compute_ion(s, kp, Xi, Cm, dt, V[i], istim[i], c->newton_cap,
                                         c->tt_jac_true, &it);
            ntot += it; if (it > nmax) nmax = it;
        } else if (c->model == EPO_MAHAJAN || c->model == EPO_MAHAJAN_FAIL) {
            int sub = 0;
            dvdt[i] = epo_mh_compute_ion(s, k, Xi, Cm, dt, V[i], istim[i], c->mh_abs_mode, &sub);
            nsub += sub;
        } else if (c->model == EPO_PURKINJE) {
            int sub = 0;
            dvdt[i] = epo_pk_compute_ion(s, k, Xi, dt, V[i], istim[i], &sub);
            nsub += sub;
        } else {
            dvdt[i] = epo_lr_compute_ion(s, c->lr_table, Xi, Cm, dt, V[i], istim[i]);
        }
    }
    c->newton_total += ntot;
    if (nmax > c->newton_max) c->newton_max = nmax;
    c->substep_count += nsub;
}

void epo_cells_ionic_cb(void *ctx, double Cm, double dt, const double *V,
                        const double *istim, double *dvdt)
{
    epo_cells_compute_ion((epo_cells *)ctx, Cm, dt, V, istim, dvdt);
}

void epo_mixed_init(epo_mixed *m, int n, const uint8_t *is_purk, epo_ionic_fn tfn, void *tctx,
                    epo_ionic_fn pfn, void *pctx)
{
    memset(m, 0, sizeof *m);
    m->n = n;
    m->tmap = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    m->pmap = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; i++) {
        if (is_purk && is_purk[i]) m->pmap[m->np++] = i;
        else m->tmap[m->nt++] = i;
    }
    m->tfn = tfn; m->tctx = tctx; m->pfn = pfn; m->pctx = pctx;
    m->buf = (double *)malloc(sizeof(double) * 3 * (size_t)(n > 0 ? n : 1));
}

void epo_mixed_free(epo_mixed *m)
{
    free(m->tmap); free(m->pmap); free(m->buf);
    memset(m, 0, sizeof *m);
}

/* one population: gather, Compute_Ion, scatter */
static void mixed_part(const epo_mixed *m, const int *map, int cnt, epo_ionic_fn fn, void *ctx, double Cm,
                       double dt, const double *V, const double *istim, double *dvdt)
{
    if (cnt == 0) return;
    double *v = m->buf, *ist = m->buf + m->n, *d = m->buf + 2 * (size_t)m->n;
    for (int k = 0; k < cnt; k++) { v[k] = V[map[k]]; ist[k] = istim[map[k]]; }
    fn(ctx, Cm, dt, v, ist, d);
    for (int k = 0; k < cnt; k++) dvdt[map[k]] = d[k];
}

void epo_mixed_ionic_cb(void *ctx, double Cm, double dt, const double *V, const double *istim, double *dvdt)
{
    const epo_mixed *m = (const epo_mixed *)ctx;
    mixed_part(m, m->tmap, m->nt, m->tfn, m->tctx, Cm, dt, V, istim, dvdt);
    mixed_part(m, m->pmap, m->np, m->pfn, m->pctx, Cm, dt, V, istim, dvdt);
}

/* ====================================================================== */
/* P1 tetrahedra -- TetMesh.cc, CardiacBody.cc                             */
/* ====================================================================== */

/* TetQuadrature order 2 (TetQuadrature.cc:16-30), truncated coordinates */
static const double QA = 0.58541020, QB = 0.13819660;

/* Shape functions / spatial gradients / w*J of one tet at its 4 points.
 * Returns J (the reference keeps its sign). */
static double tet_geometry(const double *x0, const double *x1, const double *x2,
                           const double *x3, double N[4][4], double dN[4][3], double *wJ)
{
    const double *X[4] = {x0, x1, x2, x3};
    static const double DN[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    double a[3][3], b[3][3];
    for (int r = 0; r < 3; r++)
        for (int cc = 0; cc < 3; cc++) {
            double v = 0.0;
            for (int k = 0; k < 4; k++) v += DN[k][cc] * X[k][r];
            a[r][cc] = v;
        }
    const double det = a[0][0] * a[1][1] * a[2][2] + a[1][0] * a[2][1] * a[0][2]
                     + a[0][1] * a[1][2] * a[2][0] - a[0][2] * a[1][1] * a[2][0]
                     - a[0][1] * a[1][0] * a[2][2] - a[1][2] * a[2][1] * a[0][0];
    b[0][0] = (a[1][1] * a[2][2] - a[2][1] * a[1][2]) / det;
    b[1][0] = (a[2][0] * a[1][2] - a[1][0] * a[2][2]) / det;
    b[2][0] = (a[1][0] * a[2][1] - a[1][1] * a[2][0]) / det;
    b[0][1] = (a[2][1] * a[0][2] - a[0][1] * a[2][2]) / det;
    b[1][1] = (a[0][0] * a[2][2] - a[2][0] * a[0][2]) / det;
    b[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) / det;
    b[0][2] = (a[0][1] * a[1][2] - a[1][1] * a[0][2]) / det;
    b[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) / det;
    b[2][2] = (a[0][0] * a[1][1] - a[1][0] * a[0][1]) / det;
    for (int k = 0; k < 4; k++)
        for (int cc = 0; cc < 3; cc++) {
            double v = 0.0;
            for (int al = 0; al < 3; al++) v += DN[k][al] * b[al][cc];
            dN[k][cc] = v;
        }
    const double qc[4][3] = {{QA, QB, QB}, {QB, QA, QB}, {QB, QB, QA}, {QB, QB, QB}};
    for (int q = 0; q < 4; q++) {
        N[q][0] = 1.0 - qc[q][0] - qc[q][1] - qc[q][2];
        N[q][1] = qc[q][0]; N[q][2] = qc[q][1]; N[q][3] = qc[q][2];
    }
    *wJ = (1.0 / 4.0 / 6.0) * det;
    return det;
}

/* D_e = sum_p D[p] f_p f_p^T  (CardiacBody.cc:138-160) */
static void elem_tensor(const double *fib, const double D[3], double De[3][3])
{
    for (int m = 0; m < 3; m++) for (int n = 0; n < 3; n++) De[m][n] = 0.0;
    if (!fib) { for (int p = 0; p < 3; p++) De[p][p] = D[0]; return; }
    for (int p = 0; p < 3; p++) {
        const double *f = fib + 3 * p;
        for (int m = 0; m < 3; m++) for (int n = 0; n < 3; n++) De[m][n] += D[p] * f[m] * f[n];
    }
}

typedef struct { int r, c; double k, m; } trip_t;

#define EPO_PI 3.14159265358979323846      /* M_PI */

/* the 16 entries of every tet, in element order (TetMesh::Compute +
 * CardiacBody::Compute), and their lumped capacitance */
static int tet_triplets(const double *xyz, int m, const int *tets, const double *fibers, const double D[3],
                        double Cm, trip_t *t, double *CL)
{
    int bad = 0;
    for (int e = 0; e < m; e++) {
        const int *v = tets + 4 * (size_t)e;
        double N[4][4], dN[4][3], wJ, De[3][3];
        tet_geometry(xyz + 3 * v[0], xyz + 3 * v[1], xyz + 3 * v[2], xyz + 3 * v[3], N, dN, &wJ);
        if (!(wJ > 0.0)) bad = 1;
        elem_tensor(fibers ? fibers + 9 * (size_t)e : NULL, D, De);
        double Ke[4][4] = {{0}}, Me[4][4] = {{0}};
        for (int q = 0; q < 4; q++)
            for (int a = 0; a < 4; a++)
                for (int b = 0; b < 4; b++) {
                    Me[a][b] += N[q][a] * N[q][b] * wJ;
                    for (int mm = 0; mm < 3; mm++)
                        for (int nn = 0; nn < 3; nn++)
                            Ke[a][b] += De[mm][nn] * dN[a][mm] * dN[b][nn] * wJ * Cm;
                }
        for (int q = 0; q < 4; q++)
            for (int a = 0; a < 4; a++) CL[v[a]] += N[q][a] * Cm * wJ;
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) {
                trip_t *p = t + 16 * (size_t)e + 4 * a + b;
                p->r = v[a]; p->c = v[b]; p->k = Ke[a][b]; p->m = Me[a][b];
            }
    }
    return bad;
}

/* 2-node cable elements of a mixed mesh (MixedMesh3D.cc:62-108 for the
 * geometry and quadrature, CardiacBody.cc:100-187 for D, K, M and
 * CardiacBody.cc:32-67 for the capacitance): the 4 entries of every bar in
 * element order after the tets' entries. */
/* Direction (unit) and length of every cable in order, with the .angle
 * overrides of MixedMesh3D::Compute (MixedMesh3D.cc:30-34, 78-87): per cable
 * from bar_orient_node when the caller resolved them over the whole element
 * order, else the cables-only rule (sticky or not).  ang[3 nb], mag[nb]. */
static void bar_frames(const double *xyz, const epo_cables *cb, double *ang_out, double *mag_out)
{
    int pmj = 0;
    double pmj_data[4] = {0., 0., 0., 0.};
    for (int e = 0; e < cb->nb; e++) {
        const int *v = cb->bars + 2 * (size_t)e;
        if (cb->orient_has && cb->orient_has[v[0]]) {
            pmj = 1;
            for (int k = 0; k < 4; k++) pmj_data[k] = cb->orient[4 * (size_t)v[0] + k];
        }
        double ang[3], mag;
        for (int k = 0; k < 3; k++) ang[k] = xyz[3 * v[1] + k] - xyz[3 * v[0] + k];
        mag = sqrt(ang[0] * ang[0] + ang[1] * ang[1] + ang[2] * ang[2]);
        for (int k = 0; k < 3; k++) ang[k] /= mag;
        if (cb->bar_orient_node) {
            const int o = cb->bar_orient_node[e];
            if (o >= 0) {
                for (int k = 0; k < 3; k++) ang[k] = cb->orient[4 * (size_t)o + k];
                mag = cb->orient[4 * (size_t)o + 3];
            }
        } else if (pmj && cb->orient_sticky) {
            for (int k = 0; k < 3; k++) ang[k] = pmj_data[k];
            mag = pmj_data[3];
        } else if (cb->orient_has && cb->orient_has[v[0]]) {
            for (int k = 0; k < 3; k++) ang[k] = pmj_data[k];
            mag = pmj_data[3];
        }
        for (int k = 0; k < 3; k++) ang_out[3 * (size_t)e + k] = ang[k];
        mag_out[e] = mag;
    }
}

/* LineQuadrature of order 2 q - 1 on [-1, 1] (LineQuadrature.cc); -1 for
 * an order the reference does not have */
static int bar_quadrature(int quad_order, double *qx, double *qw)
{
    const int qord = 2 * (quad_order > 0 ? quad_order : 2) - 1;
    if (qord == 1) { qx[0] = 0.0; qw[0] = 2.0; return 1; }
    if (qord == 3) { qx[0] = -0.577350269189626; qx[1] = 0.577350269189626; qw[0] = qw[1] = 1.0; return 2; }
    if (qord == 5) {
        qx[0] = -0.774596669241483; qx[1] = 0.0; qx[2] = 0.774596669241483;
        qw[0] = qw[2] = 5.0 / 9.0; qw[1] = 8.0 / 9.0;
        return 3;
    }
    return -1;
}

static int bar_triplets(const double *xyz, const epo_cables *cb, double Cm, trip_t *t, double *CL)
{
    /* LineQuadrature of order 2 q - 1 on [-1, 1] (LineQuadrature.cc) */
    double qx[3], qw[3];
    int nq;
    const int qord = 2 * (cb->quad_order > 0 ? cb->quad_order : 2) - 1;
    if (qord == 1) { nq = 1; qx[0] = 0.0; qw[0] = 2.0; }
    else if (qord == 3) { nq = 2; qx[0] = -0.577350269189626; qx[1] = 0.577350269189626; qw[0] = qw[1] = 1.0; }
    else if (qord == 5) {
        nq = 3; qx[0] = -0.774596669241483; qx[1] = 0.0; qx[2] = 0.774596669241483;
        qw[0] = qw[2] = 5.0 / 9.0; qw[1] = 8.0 / 9.0;
    } else return -2;
    int bad = 0;
    int pmj = 0;                    /* once set, stays set: see the note in ep_oracle.h */
    double pmj_data[4] = {0., 0., 0., 0.};
    for (int e = 0; e < cb->nb; e++) {
        const int *v = cb->bars + 2 * (size_t)e;
        if (cb->orient_has && cb->orient_has[v[0]]) {
            pmj = 1;
            for (int k = 0; k < 4; k++) pmj_data[k] = cb->orient[4 * (size_t)v[0] + k];
        }
        double ang[3], mag;
        for (int k = 0; k < 3; k++) ang[k] = xyz[3 * v[1] + k] - xyz[3 * v[0] + k];
        mag = sqrt(ang[0] * ang[0] + ang[1] * ang[1] + ang[2] * ang[2]);
        for (int k = 0; k < 3; k++) ang[k] /= mag;
        if (cb->bar_orient_node) {
            const int o = cb->bar_orient_node[e];
            if (o >= 0) {
                for (int k = 0; k < 3; k++) ang[k] = cb->orient[4 * (size_t)o + k];
                mag = cb->orient[4 * (size_t)o + 3];
            }
        } else if (pmj && cb->orient_sticky) {
            for (int k = 0; k < 3; k++) ang[k] = pmj_data[k];
            mag = pmj_data[3];
        } else if (cb->orient_has && cb->orient_has[v[0]]) {
            for (int k = 0; k < 3; k++) ang[k] = pmj_data[k];
            mag = pmj_data[3];
        }
        if (!(mag > 0.0)) bad = 1;
        /* conductivity: LV cables (a node of tissue type 11) take DpLeft */
        const int lv = cb->lv ? cb->lv[e] : 0;
        double Dc[3];
        for (int k = 0; k < 3; k++) Dc[k] = lv ? cb->DpLeft[k] : cb->Dp[k];
        double De[3][3];
        elem_tensor(cb->fibers ? cb->fibers + 9 * (size_t)e : NULL, Dc, De);
        const double fac = 2. / mag;
        const double dN[2] = {-0.5, 0.5};
        double dx[2][3];
        for (int a = 0; a < 2; a++)
            for (int k = 0; k < 3; k++) dx[a][k] = dN[a] * ang[k] * fac;
        double Ke[2][2] = {{0}}, Me[2][2] = {{0}};
        for (int q = 0; q < nq; q++) {
            const double N[2] = {0.5 * (1. - qx[q]), 0.5 * (1. + qx[q])};
            const double w = qw[q] * EPO_PI * (cb->radius * cb->radius) * mag;
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++) {
                    Me[a][b] += N[a] * N[b] * w;
                    for (int mm = 0; mm < 3; mm++)
                        for (int nn = 0; nn < 3; nn++)
                            Ke[a][b] += De[mm][nn] * dx[a][mm] * dx[b][nn] * w * Cm;
                }
            for (int a = 0; a < 2; a++) CL[v[a]] += N[a] * Cm * w;
        }
        for (int a = 0; a < 2; a++)
            for (int b = 0; b < 2; b++) {
                trip_t *p = t + 4 * (size_t)e + 2 * a + b;
                p->r = v[a]; p->c = v[b]; p->k = Ke[a][b]; p->m = Me[a][b];
            }
    }
    return bad;
}

static void csr_from_triplets(int n, trip_t *t, size_t nt, double *CL, double Cm, double dt_diff,
                              double smoothing_alpha, epo_csr *out)
{
    /* group the element entries by (row, col) keeping element order inside
     * each run, so duplicates are summed in insertion order */
    {
        trip_t *tmp = (trip_t *)malloc(sizeof(trip_t) * nt);
        /* counting sort by row, then insertion by column inside a row keeps order */
        int *cnt = (int *)calloc((size_t)n + 1, sizeof(int));
        for (size_t i = 0; i < nt; i++) cnt[t[i].r + 1]++;
        for (int i = 0; i < n; i++) cnt[i + 1] += cnt[i];
        int *pos = (int *)malloc(sizeof(int) * ((size_t)n + 1));
        memcpy(pos, cnt, sizeof(int) * ((size_t)n + 1));
        for (size_t i = 0; i < nt; i++) tmp[pos[t[i].r]++] = t[i];
        /* inside each row: stable sort by column (insertion sort, rows are short) */
        for (int r = 0; r < n; r++) {
            for (int i = cnt[r] + 1; i < cnt[r + 1]; i++) {
                trip_t key = tmp[i]; int j = i - 1;
                while (j >= cnt[r] && tmp[j].c > key.c) { tmp[j + 1] = tmp[j]; j--; }
                tmp[j + 1] = key;
            }
        }
        /* count unique */
        int *rowptr = (int *)calloc((size_t)n + 1, sizeof(int));
        size_t nnz = 0;
        for (int r = 0; r < n; r++) {
            int last = -1;
            for (int i = cnt[r]; i < cnt[r + 1]; i++)
                if (tmp[i].c != last) { nnz++; last = tmp[i].c; }
            rowptr[r + 1] = (int)nnz;
        }
        int *col = (int *)malloc(sizeof(int) * nnz);
        double *K = (double *)calloc(nnz, sizeof(double)), *M = (double *)calloc(nnz, sizeof(double));
        double *A = (double *)calloc(nnz, sizeof(double)), *B = (double *)calloc(nnz, sizeof(double));
        const double s = dt_diff / 4.0;
        const double sm = smoothing_alpha > 0 ? smoothing_alpha * 4. / dt_diff : 0.0;
        for (int r = 0; r < n; r++) {
            int k = rowptr[r] - 1, last = -1;
            for (int i = cnt[r]; i < cnt[r + 1]; i++) {
                if (tmp[i].c != last) { k++; col[k] = tmp[i].c; last = tmp[i].c; }
                K[k] += tmp[i].k; M[k] += tmp[i].m;
            }
        }
        /* A/B: the diffusion contributions are inserted first (all elements,
         * scaled by +-dt/4), then the capacitance (EP_CrankNicholson.cc:22-29) */
        for (int r = 0; r < n; r++) {
            int k = rowptr[r] - 1, last = -1;
            for (int i = cnt[r]; i < cnt[r + 1]; i++) {
                if (tmp[i].c != last) { k++; last = tmp[i].c; }
                A[k] += tmp[i].k * s; B[k] += tmp[i].k * (-s);
            }
            k = rowptr[r] - 1; last = -1;
            for (int i = cnt[r]; i < cnt[r + 1]; i++) {
                if (tmp[i].c != last) { k++; last = tmp[i].c; }
                A[k] += tmp[i].m * Cm; B[k] += tmp[i].m * Cm;
            }
            if (sm > 0) {
                k = rowptr[r] - 1; last = -1;
                for (int i = cnt[r]; i < cnt[r + 1]; i++) {
                    if (tmp[i].c != last) { k++; last = tmp[i].c; }
                    A[k] += tmp[i].k * sm; B[k] += tmp[i].k * (-sm);
                }
            }
        }
        out->n = n; out->nnz = (int)nnz; out->rowptr = rowptr; out->col = col;
        out->A = A; out->B = B; out->K = K; out->M = M; out->CL = CL;
        free(tmp); free(cnt); free(pos);
    }
}

int epo_assemble(int n, const double *xyz, int m, const int *tets,
                 const double *fibers, const double D[3], double Cm,
                 double dt_diff, double smoothing_alpha, epo_csr *out)
{
    return epo_assemble_mixed(n, xyz, m, tets, fibers, D, NULL, Cm, dt_diff, smoothing_alpha, out);
}

int epo_assemble_mixed(int n, const double *xyz, int m, const int *tets,
                       const double *fibers, const double D[3], const epo_cables *cables,
                       double Cm, double dt_diff, double smoothing_alpha, epo_csr *out)
{
    memset(out, 0, sizeof *out);
    const size_t nb = cables ? (size_t)cables->nb : 0;
    const size_t nt = (size_t)m * 16 + nb * 4;
    trip_t *t = (trip_t *)malloc(sizeof(trip_t) * (nt ? nt : 1));
    double *CL = (double *)calloc((size_t)n, sizeof(double));
    int bad = tet_triplets(xyz, m, tets, fibers, D, Cm, t, CL);
    if (nb) {
        const int rb = bar_triplets(xyz, cables, Cm, t + (size_t)m * 16, CL);
        if (rb == -2) { free(t); free(CL); return -2; }
        bad |= rb;
    }
    csr_from_triplets(n, t, nt, CL, Cm, dt_diff, smoothing_alpha, out);
    free(t);
    return bad ? -1 : 0;
}

void epo_csr_free(epo_csr *a)
{
    free(a->rowptr); free(a->col); free(a->A); free(a->B); free(a->K); free(a->M); free(a->CL);
    memset(a, 0, sizeof *a);
}

void epo_spmv(const epo_csr *a, const double *vals, const double *x, double *y)
{
#pragma omp parallel for schedule(static)
    for (int r = 0; r < a->n; r++) {
        double s = 0.0;
        for (int k = a->rowptr[r]; k < a->rowptr[r + 1]; k++) s += vals[k] * x[a->col[k]];
        y[r] = s;
    }
}

/* sums of fixed blocks of 4096 entries, then the block sums in order: the
 * same bits whatever the thread count (an OpenMP reduction combines thread
 * partials in arrival order) */
static double dotp(int n, const double *x, const double *y)
{
    enum { BLK = 4096 };
    const int nb = (n + BLK - 1) / BLK;
    double stackbuf[256];
    double *part = nb <= 256 ? stackbuf : (double *)malloc(sizeof(double) * (size_t)nb);
#pragma omp parallel for schedule(static)
    for (int b = 0; b < nb; b++) {
        const int lo = b * BLK, hi = lo + BLK < n ? lo + BLK : n;
        double s = 0.0;
        for (int i = lo; i < hi; i++) s += x[i] * y[i];
        part[b] = s;
    }
    double s = 0.0;
    for (int b = 0; b < nb; b++) s += part[b];
    if (part != stackbuf) free(part);
    return s;
}

/* k-step Jacobi: z_0 = 0, z_{m+1} = z_m + D^-1 (r - A z_m) */
static void jacobi_apply(const epo_csr *a, const double *vals, const double *dinv,
                         int steps, const double *r, double *z, double *w)
{
    const int n = a->n;
    for (int i = 0; i < n; i++) z[i] = dinv[i] * r[i];
    for (int s = 1; s < steps; s++) {
        epo_spmv(a, vals, z, w);
        for (int i = 0; i < n; i++) z[i] += dinv[i] * (r[i] - w[i]);
    }
}

int epo_pcg(const epo_csr *a, const double *vals, const double *b, double *x,
            double tol, int maxit, int jacobi_steps, double *relres)
{
    const int n = a->n;
    double *r = (double *)malloc(sizeof(double) * n), *z = (double *)malloc(sizeof(double) * n);
    double *p = (double *)malloc(sizeof(double) * n), *q = (double *)malloc(sizeof(double) * n);
    double *w = (double *)malloc(sizeof(double) * n), *dinv = (double *)malloc(sizeof(double) * n);
    for (int i = 0; i < n; i++) {
        double d = 0;
        for (int k = a->rowptr[i]; k < a->rowptr[i + 1]; k++) if (a->col[k] == i) d = vals[k];
        dinv[i] = 1.0 / d;
    }
    epo_spmv(a, vals, x, q);
    for (int i = 0; i < n; i++) r[i] = b[i] - q[i];
    const double r0 = sqrt(dotp(n, r, r));
    int it = 0, ok = 1;
    double rn = r0;
    if (r0 > 0.0) {
        jacobi_apply(a, vals, dinv, jacobi_steps < 1 ? 1 : jacobi_steps, r, z, w);
        double rz = dotp(n, r, z);
        for (int i = 0; i < n; i++) p[i] = z[i];
        ok = 0;
        while (it < maxit) {
            epo_spmv(a, vals, p, q);
            const double alpha = rz / dotp(n, p, q);
            for (int i = 0; i < n; i++) { x[i] += alpha * p[i]; r[i] -= alpha * q[i]; }
            it++;
            rn = sqrt(dotp(n, r, r));
            if (rn <= tol * r0) { ok = 1; break; }
            jacobi_apply(a, vals, dinv, jacobi_steps < 1 ? 1 : jacobi_steps, r, z, w);
            const double rz1 = dotp(n, r, z);
            const double beta = rz1 / rz;
            rz = rz1;
            for (int i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
        }
    }
    if (relres) *relres = r0 > 0 ? rn / r0 : 0.0;
    free(r); free(z); free(p); free(q); free(w); free(dinv);
    return ok ? it : -1;
}

/* ====================================================================== */
/* pseudo-ECG -- ComputeECG.h                                              */
/* ====================================================================== */

static void qp_positions(const double *X[4], double N[4][4], double pos[4][3])
{
    for (int q = 0; q < 4; q++)
        for (int d = 0; d < 3; d++) {
            double v = 0.0;
            for (int a = 0; a < 4; a++) v += N[q][a] * X[a][d];
            pos[q][d] = v;
        }
}

static void grad_one_by_r(const double *x, const double *e, double *g)
{
    double dist = 0.0;
    for (int d = 0; d < 3; d++) dist += (x[d] - e[d]) * (x[d] - e[d]);
    dist = sqrt(dist);
    if (dist < 1e-6) { g[0] = g[1] = g[2] = 0.0; return; }
    const double d3 = dist * dist * dist;
    for (int d = 0; d < 3; d++) g[d] = -(x[d] - e[d]) / d3;
}

void epo_ecg_elementwise(int n, const double *xyz, int m, const int *tets,
                         const double *fibers, const double D[3], int ne,
                         const double *electrodes, const double *V, double *ecg)
{
    (void)n;
    for (int k = 0; k < ne; k++) ecg[k] = 0.0;
    for (int e = 0; e < m; e++) {
        const int *v = tets + 4 * (size_t)e;
        const double *X[4] = {xyz + 3 * v[0], xyz + 3 * v[1], xyz + 3 * v[2], xyz + 3 * v[3]};
        double N[4][4], dN[4][3], wJ, De[3][3], pos[4][3], gv[3];
        tet_geometry(X[0], X[1], X[2], X[3], N, dN, &wJ);
        elem_tensor(fibers ? fibers + 9 * (size_t)e : NULL, D, De);
        qp_positions(X, N, pos);
        for (int d = 0; d < 3; d++) {
            double s = 0.0;
            for (int a = 0; a < 4; a++) s += dN[a][d] * V[v[a]];
            gv[d] = s;
        }
        for (int k = 0; k < ne; k++)
            for (int q = 0; q < 4; q++) {
                double g[3];
                grad_one_by_r(pos[q], electrodes + 3 * k, g);
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) ecg[k] += De[a][b] * gv[a] * g[b] * wJ;
            }
    }
}

void epo_ecg_weights(int n, const double *xyz, int m, const int *tets,
                     const double *fibers, const double D[3], int ne,
                     const double *electrodes, double *W)
{
    memset(W, 0, sizeof(double) * (size_t)ne * n);
    for (int e = 0; e < m; e++) {
        const int *v = tets + 4 * (size_t)e;
        const double *X[4] = {xyz + 3 * v[0], xyz + 3 * v[1], xyz + 3 * v[2], xyz + 3 * v[3]};
        double N[4][4], dN[4][3], wJ, De[3][3], pos[4][3];
        tet_geometry(X[0], X[1], X[2], X[3], N, dN, &wJ);
        elem_tensor(fibers ? fibers + 9 * (size_t)e : NULL, D, De);
        qp_positions(X, N, pos);
        for (int k = 0; k < ne; k++) {
            double G[3] = {0, 0, 0};
            for (int q = 0; q < 4; q++) {
                double g[3];
                grad_one_by_r(pos[q], electrodes + 3 * k, g);
                for (int d = 0; d < 3; d++) G[d] += g[d] * wJ;
            }
            double DG[3];
            for (int a = 0; a < 3; a++) DG[a] = De[a][0] * G[0] + De[a][1] * G[1] + De[a][2] * G[2];
            for (int a = 0; a < 4; a++)
                W[(size_t)k * n + v[a]] += dN[a][0] * DG[0] + dN[a][1] * DG[1] + dN[a][2] * DG[2];
        }
    }
}

/* The cables' share of the per-node ECG weights, added to W: ComputeECG.h's
 * sums over the 2-node elements of a MIX3D mesh (they are not skipped there,
 * ComputeECG.h:47-50, 107-110): quadrature points of MixedMesh3D::Compute
 * placed by the shape functions on the cable's own nodes (ComputeECG.h:
 * 65-70), grad N = -+ ang / length, weight w_q pi r^2 length, and the tissue
 * D along the cable's fibre frame, or D[0] I without fibres
 * (computeDiffusionTensor applies Diff to every element, ComputeECG.h:
 * 92-136; cables->Dp is not used here).  ComputeECG fixes the radius at
 * 0.0275 cm (ComputeECG.cc:75); the caller passes it in cables->radius. */
int epo_ecg_weights_cables(int n, const double *xyz, const epo_cables *cb, const double D[3], int ne,
                           const double *electrodes, double *W)
{
    double qx[3], qw[3];
    const int nq = bar_quadrature(cb->quad_order, qx, qw);
    if (nq < 0) return -2;
    double *ang = (double *)malloc(sizeof(double) * 3 * (size_t)(cb->nb > 0 ? cb->nb : 1));
    double *mag = (double *)malloc(sizeof(double) * (size_t)(cb->nb > 0 ? cb->nb : 1));
    bar_frames(xyz, cb, ang, mag);
    for (int e = 0; e < cb->nb; e++) {
        const int *v = cb->bars + 2 * (size_t)e;
        double De[3][3];
        elem_tensor(cb->fibers ? cb->fibers + 9 * (size_t)e : NULL, D, De);
        const double *a = ang + 3 * (size_t)e;
        const double dx[2][3] = {{-a[0] / mag[e], -a[1] / mag[e], -a[2] / mag[e]},
                                 {a[0] / mag[e], a[1] / mag[e], a[2] / mag[e]}};
        for (int k = 0; k < ne; k++) {
            double G[3] = {0, 0, 0};
            for (int q = 0; q < nq; q++) {
                const double N0 = 0.5 * (1. - qx[q]), N1 = 0.5 * (1. + qx[q]);
                double pos[3], g[3];
                for (int d = 0; d < 3; d++) pos[d] = N0 * xyz[3 * v[0] + d] + N1 * xyz[3 * v[1] + d];
                grad_one_by_r(pos, electrodes + 3 * k, g);
                const double w = qw[q] * EPO_PI * (cb->radius * cb->radius) * mag[e];
                for (int d = 0; d < 3; d++) G[d] += g[d] * w;
            }
            double DG[3];
            for (int r = 0; r < 3; r++) DG[r] = De[r][0] * G[0] + De[r][1] * G[1] + De[r][2] * G[2];
            for (int b = 0; b < 2; b++)
                W[(size_t)k * n + v[b]] += dx[b][0] * DG[0] + dx[b][1] * DG[1] + dx[b][2] * DG[2];
        }
    }
    free(ang);
    free(mag);
    return 0;
}

/* ====================================================================== */
/* time stepping -- EP_CrankNicholson.cc, EPSimulator.cc                   */
/* ====================================================================== */

void epo_sim_init(epo_sim *s, epo_csr *csr, double dt, double ionic_dt,
                  double Cm, double cg_tol, int cg_maxit, int jacobi_steps,
                  epo_ionic_fn fn, void *ctx)
{
    memset(s, 0, sizeof *s);
    s->csr = csr; s->n = csr->n; s->dt = dt; s->ionic_dt = ionic_dt; s->Cm = Cm;
    s->cg_tol = cg_tol; s->cg_maxit = cg_maxit; s->jacobi_steps = jacobi_steps;
    s->ionic = fn; s->ionic_ctx = ctx;
    const size_t n = (size_t)s->n;
    s->V = (double *)calloc(n, sizeof(double)); s->istim = (double *)calloc(n, sizeof(double));
    s->dvdt = (double *)calloc(n, sizeof(double)); s->b = (double *)calloc(n, sizeof(double));
    s->ici = (double *)calloc(n, sizeof(double));
    /* EP_CrankNicholson.cc:114-143: the sub-step sequence of one ionic phase */
    double total = 0.0, h = (ionic_dt < dt) ? ionic_dt : dt;
    s->nsub = 0;
    while (total < dt && s->nsub < 64) {
        s->sub_dt[s->nsub++] = h;
        total += h;
        h = (total + h < dt) ? h : dt - total;
    }
}

void epo_sim_free(epo_sim *s)
{
    free(s->V); free(s->istim); free(s->dvdt); free(s->b); free(s->ici);
    free(s->A_be); free(s->B_be);
}

double epo_cells_ionic_node_cb(void *ctx, int i, double Cm, double dt, double V, double istim)
{
    epo_cells *c = (epo_cells *)ctx;
    double *st = c->state + (size_t)i * c->nstate;
    const int t = c->type ? c->type[i] : 0;
    const double *k = c->consts + (size_t)t * c->nconst;
    const double Xi = c->user_xi ? c->user_Xi : c->Xi;
    if (c->model == EPO_TUSSCHER) {
        int it = 0;
        double kk[EPO_TT_NCONST];
        const double *kp = k;
        if (c->gks_scale) {
            memcpy(kk, k, sizeof kk);
            kk[15] *= c->gks_scale[i];
            kp = kk;
        }
        return epo_tt_compute_ion(st, kp, Xi, Cm, dt, V, istim, c->newton_cap, c->tt_jac_true, &it);
    }
    if (c->model == EPO_MAHAJAN || c->model == EPO_MAHAJAN_FAIL) {
        int sub = 0;
        return epo_mh_compute_ion(st, k, Xi, Cm, dt, V, istim, c->mh_abs_mode, &sub);
    }
    return epo_lr_compute_ion(st, c->lr_table, Xi, Cm, dt, V, istim);
}

void epo_sim_set_scheme(epo_sim *s, int scheme, double dt_diff, epo_ionic_node_fn fn, void *ctx)
{
    const epo_csr *a = s->csr;
    s->scheme = scheme;
    s->ionic_node = fn;
    s->ionic_ctx = ctx;
    free(s->A_be); free(s->B_be);
    s->A_be = s->B_be = NULL;
    if (scheme == EPO_SCHEME_BE) {
        /* the stiffness times dt/2 plus the lumped capacitance on the diagonal
         * (EP_BackwardEuler.cc:13-30); the right side C_L V */
        s->A_be = (double *)calloc((size_t)a->nnz, sizeof(double));
        s->B_be = (double *)calloc((size_t)a->nnz, sizeof(double));
        for (int i = 0; i < a->n; i++)
            for (int k = a->rowptr[i]; k < a->rowptr[i + 1]; k++) {
                s->A_be[k] = a->K[k] * (s->dt / 2.0);
                if (a->col[k] == i) { s->A_be[k] += a->CL[i]; s->B_be[k] = a->CL[i]; }
            }
    } else if (scheme == EPO_SCHEME_EXPLICIT) {
        /* EP_ExplicitSolver::Solve: steps of min(dtDiff, dt/2) while more
         * than 1e-6 of the half step is left */
        double solve = 0.5 * s->dt, st = dt_diff < 0.5 * s->dt ? dt_diff : 0.5 * s->dt;
        s->nex = 0;
        while (solve > 1e-6 && s->nex < 4096) {
            s->ex_h[s->nex++] = st;
            solve -= st;
            st = st < solve ? st : solve;
        }
    }
}

/* CardiacBody::getVoltageFromIonicCurrent (CardiacBody.cc:819-904), per node:
 * a first sub-step of dt_ion; when its rate, stored in an int, is 0 the
 * stride becomes 5 dt_ion; then strides until dT, the last one shortened. */
static void ionic_strides(epo_sim *s)
{
    const double dT = s->dt;
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < s->n; i++) {
        double dt = s->ionic_dt;
        double V = s->V[i];
        const double ist = s->istim[i];
        if (dT / dt > 1.0) {
            double iion = s->ionic_node(s->ionic_ctx, i, s->Cm, dt, V, ist);
            V += dt * iion;
            double totT = dt, delT;
            const int slope = (int)iion;
            if (!slope) dt *= 5;
            int flag = 1;
            while (flag) {
                if (totT + dt > dT) { delT = dT - totT; flag = 0; }
                else delT = dt;
                iion = s->ionic_node(s->ionic_ctx, i, s->Cm, delT, V, ist);
                V += delT * iion;
                totT += delT;
            }
        } else {
            const double iion = s->ionic_node(s->ionic_ctx, i, s->Cm, dt, V, ist);
            V += dt * iion;
        }
        s->V[i] = V;
    }
}

static void half_be(epo_sim *s)
{
    double rr;
    epo_spmv(s->csr, s->B_be, s->V, s->b);
    const int it = epo_pcg(s->csr, s->A_be, s->b, s->V, s->cg_tol, s->cg_maxit, s->jacobi_steps, &rr);
    if (it < 0) { s->cg_fail++; s->cg_iters_total += s->cg_maxit; }
    else s->cg_iters_total += it;
}

static void half_explicit(epo_sim *s)
{
    const int n = s->n;
    for (int k = 0; k < s->nex; k++) {
        const double h = s->ex_h[k];
        epo_spmv(s->csr, s->csr->K, s->V, s->b);          /* K V; D = -K */
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) s->V[i] += h * (-s->b[i]) / s->csr->CL[i];
    }
}

static void half_step(epo_sim *s)
{
    double rr;
    epo_spmv(s->csr, s->csr->B, s->V, s->b);
    const int it = epo_pcg(s->csr, s->csr->A, s->b, s->V, s->cg_tol, s->cg_maxit, s->jacobi_steps, &rr);
    if (it < 0) { s->cg_fail++; s->cg_iters_total += s->cg_maxit; }
    else s->cg_iters_total += it;
}

void epo_sim_step(epo_sim *s)
{
    const int n = s->n;
    const double *CL = s->csr->CL;
    if (s->scheme == EPO_SCHEME_BE || s->scheme == EPO_SCHEME_EXPLICIT) {
        if (s->scheme == EPO_SCHEME_BE) half_be(s); else half_explicit(s);
        ionic_strides(s);
        if (s->scheme == EPO_SCHEME_BE) half_be(s); else half_explicit(s);
        s->step++;
        return;
    }
    half_step(s);
    for (int k = 0; k < s->nsub; k++) {
        const double h = s->sub_dt[k];
        s->ionic(s->ionic_ctx, s->Cm, h, s->V, s->istim, s->dvdt);
        /* C_L V' = C_L V + h C_L I: the diagonal solve (EP_CrankNicholson.cc:124-133) */
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) {
            const double ici = CL[i] * s->dvdt[i];
            const double rhs = CL[i] * s->V[i] + h * ici;
            s->V[i] = rhs / CL[i];
        }
    }
    half_step(s);
    s->step++;
}

void epo_stim_schedule(int nstim, const double *t_start, const double *t_stop,
                       double dt, long nsteps, long *start_step, long *stop_step)
{
    for (int i = 0; i < nstim; i++) { start_step[i] = -1; stop_step[i] = -1; }
    if (nstim <= 0) return;
    long pulse_start = (long)(t_start[0] / dt), pulse_stop = (long)(t_stop[0] / dt);
    int sc = 0, pc = 0;
    for (long count = 0; count < nsteps; count++) {
        if (count == pulse_start) {
            start_step[sc] = count;
            sc++;
            if (sc == nstim) sc--;
            pulse_start = (int)(t_start[sc] / dt);
        }
        if (count == pulse_stop) {
            stop_step[pc] = count;
            pc++;
            if (pc == nstim) pc--;
            pulse_stop = (int)(t_stop[pc] / dt);
        }
    }
}

long epo_num_steps(double dt, double T)
{
    double t = 0.0; long k = 0;
    while (t < T) { t += dt; k++; }
    return k;
}
