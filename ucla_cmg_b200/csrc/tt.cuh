// tt.cuh -- ten Tusscher 2006 cell model, device side.
//
// Follows voomEP/src/IonicModel/Tusscher.cc (ComputeRates 4-96,
// UpdateStateVariables 116-195, Compute_Ion 201-213): 12 gates by the
// semi-implicit update (s + dt*inf/tau)/(1 + dt/tau), then Newton on
// (Ki, Nai, Cai, Cass, CaSR, R') for x - x^n - dt f(x) = 0 with a central
// finite-difference Jacobian (eps = 1e-3 x) and a partially pivoted 6x6 LU.
//
// The voltage is frozen during a Compute_Ion call, so every voltage-only
// term (all gate kinetics, the exponentials of I_NaK, I_NaCa, I_CaL, I_pK)
// is evaluated once per call instead of in each of the 2 + 13k rate
// evaluations of the reference, and the reversal potentials (and the I_K1
// rectifier) are re-evaluated only when the Newton perturbation touches
// their concentration.  Each evaluation still sees exactly the same inputs
// as the reference's, so the arithmetic of every rate is unchanged.
#pragma once
#include "common.cuh"

namespace ep {

constexpr int TT_NS = 18;      // stored states besides V: reference State[1..18]
constexpr int TT_NC = 54;      // 53 reference constants + [53] s-gate variant

// Newton-state slots (reference State index): 0 Ki(1) 1 Nai(2) 2 Cai(3)
// 3 Cass(10) 4 CaSR(17) 5 R'(18)
template <typename R> struct TTFixed {          // voltage/gate-only terms
    R V, F, rtf, rtf_half, ist;
    R nak_fac, nak_den, g_na, e_g, e_g1, naca_den, nao3, sq_ko;
    R g_to, g_kr, g_ks, cal_pre, e_ca, cal_den, pk_den, eks_num;
};

template <typename R> struct TTRev {            // concentration-dependent terms
    R ENa, EK, EKs, ECa, xk1;
};

// Gate kinetics (Tusscher.cc:5-55) in the reference update order
// 4,5,6,7,8,9,11,12,13,14,15,16.
template <typename R>
EP_HD void tt_gates(R V, R Cass, const R *c, R ginf[12], R gtau[12]) {
    R t;
    ginf[0] = R(1) / (R(1) + exp((R(-26) - V) / R(7)));
    gtau[0] = (R(450) / (R(1) + exp((R(-45) - V) / R(10)))) * (R(6) / (R(1) + exp((V + R(30)) / R(11.5))));
    ginf[1] = R(1) / (R(1) + exp((V + R(88)) / R(24)));
    gtau[1] = (R(3) / (R(1) + exp((R(-60) - V) / R(20)))) * (R(1.12) / (R(1) + exp((V - R(60)) / R(20))));
    ginf[2] = R(1) / (R(1) + exp((R(-5) - V) / R(14)));
    gtau[2] = (R(1400) / sqrt(R(1) + exp((R(5) - V) / R(6)))) * (R(1) / (R(1) + exp((V - R(35)) / R(15)))) + R(80);
    t = R(1) + exp((R(-56.86) - V) / R(9.03));
    ginf[3] = R(1) / (t * t);
    gtau[3] = (R(1) / (R(1) + exp((R(-60) - V) / R(5))))
            * (R(0.1) / (R(1) + exp((V + R(35)) / R(5))) + R(0.1) / (R(1) + exp((V - R(50)) / R(200))));
    t = R(1) + exp((V + R(71.55)) / R(7.43));
    ginf[4] = R(1) / (t * t);
    ginf[5] = ginf[4];
    R ah, bh, aj, bj;
    if (V < R(-40)) {
        ah = R(0.057) * exp((-(V + R(80))) / R(6.8));
        bh = R(2.7) * exp(R(0.079) * V) + R(310000) * exp(R(0.3485) * V);
        aj = ((R(-25428) * exp(R(0.2444) * V) - R(6.948e-06) * exp(R(-0.04391) * V)) * (V + R(37.78)))
           / (R(1) + exp(R(0.311) * (V + R(79.23))));
        bj = (R(0.02424) * exp(R(-0.01052) * V)) / (R(1) + exp(R(-0.1378) * (V + R(40.14))));
    } else {
        ah = R(0);
        bh = R(0.77) / (R(0.13) * (R(1) + exp((V + R(10.66)) / R(-11.1))));
        aj = R(0);
        bj = (R(0.6) * exp(R(0.057) * V)) / (R(1) + exp(R(-0.1) * (V + R(32))));
    }
    gtau[4] = R(1) / (ah + bh);
    gtau[5] = R(1) / (aj + bj);
    ginf[6] = R(1) / (R(1) + exp((R(-8) - V) / R(7.5)));
    gtau[6] = (R(1.4) / (R(1) + exp((R(-35) - V) / R(13))) + R(0.25)) * (R(1.4) / (R(1) + exp((V + R(5)) / R(5))))
            + R(1) / (R(1) + exp((R(50) - V) / R(20)));
    ginf[7] = R(1) / (R(1) + exp((V + R(20)) / R(7)));
    t = V + R(27);
    gtau[7] = R(1102.5) * exp((-(t * t)) / R(225)) + R(200) / (R(1) + exp((R(13) - V) / R(10)))
            + R(180) / (R(1) + exp((V + R(30)) / R(10))) + R(20);
    ginf[8] = R(0.67) / (R(1) + exp((V + R(35)) / R(7))) + R(0.33);
    gtau[8] = R(562) * exp((-(t * t)) / R(240)) + R(31) / (R(1) + exp((R(25) - V) / R(10)))
            + R(80) / (R(1) + exp((V + R(30)) / R(10)));
    t = Cass / R(0.05);
    ginf[9] = R(0.6) / (R(1) + t * t) + R(0.4);
    gtau[9] = R(80) / (R(1) + t * t) + R(2);
    if (c[53] == R(0)) {
        ginf[10] = R(1) / (R(1) + exp((V + R(20)) / R(5)));
        t = V + R(45);
        gtau[10] = R(85) * exp((-(t * t)) / R(320)) + R(5) / (R(1) + exp((V - R(20)) / R(5))) + R(3);
    } else {  // TT2006 endocardial s gate (not in the reference)
        ginf[10] = R(1) / (R(1) + exp((V + R(28)) / R(5)));
        t = V + R(67);
        gtau[10] = R(1000) * exp((-(t * t)) / R(1000)) + R(8);
    }
    ginf[11] = R(1) / (R(1) + exp((R(20) - V) / R(6)));
    t = V + R(40);
    gtau[11] = R(9.5) * exp((-(t * t)) / R(1800)) + R(0.8);
}

// s: the 18 stored states (s[k-1] = reference State[k]), after the gate update
template <typename R>
EP_HD TTFixed<R> tt_fixed(R V, const R *s, const R *__restrict__ c, R ist, R gks) {
    TTFixed<R> f;
    const R Rg = c[0], T = c[1], F = c[2];
    const R RT = Rg * T;
    f.V = V; f.F = F; f.ist = ist;
    f.rtf = RT / F;
    f.rtf_half = (R(0.5) * Rg * T) / F;
    f.nak_fac = (c[21] * c[10]) / (c[10] + c[22]);
    f.nak_den = R(1) + R(0.1245) * exp((R(-0.1) * V * F) / RT) + R(0.0353) * exp((-V * F) / RT);
    const R m = s[6], h = s[7], j = s[8];
    f.g_na = c[16] * (m * m * m) * h * j;
    f.e_g = exp((c[27] * V * F) / RT);
    f.e_g1 = exp(((c[27] - R(1)) * V * F) / RT);
    f.nao3 = c[11] * c[11] * c[11];
    f.naca_den = ((c[29] * c[29] * c[29]) + f.nao3) * (c[28] + c[12]) * (R(1) + c[25] * f.e_g1);
    f.sq_ko = sqrt(c[10] / R(5.4));
    f.g_to = c[20] * s[15] * s[14];                 // r (16), s (15)
    f.g_kr = c[14] * f.sq_ko * s[3] * s[4];         // Xr1, Xr2
    f.g_ks = (c[15] * gks) * (s[5] * s[5]);         // Xs (per-node G_Ks multiplier)
    const R xca = (R(2) * (V - R(15)) * F) / RT;
    f.e_ca = exp(xca);
    // I_CaL's GHK factor (V-15)/(exp(x)-1) is 0/0 at V = 15 mV; FP32 lands
    // on it (V within an ulp of 15) often enough over millions of
    // node-steps, so the removable singularity takes its series
    // x/(e^x - 1) = 1 - x/2 + x^2/12 (next term x^4/720) inside a band where
    // that series is exact to the type's precision and e^x - 1 would lose
    // most of its digits to cancellation.
    const R band = sizeof(R) == 4 ? R(1e-2) : R(1e-6);
    if (fabs(xca) < band) {
        f.cal_pre = (c[18] * s[10] * s[11] * s[12] * s[13] * R(4) * (F * F)) / RT
                  * (RT / (R(2) * F)) * (R(1) - xca * R(0.5) + xca * xca / R(12));
        f.cal_den = R(1);
    } else {
        f.cal_pre = (c[18] * s[10] * s[11] * s[12] * s[13] * R(4) * (V - R(15)) * (F * F)) / RT;
        f.cal_den = f.e_ca - R(1);
    }
    f.pk_den = R(1) + exp((R(25) - V) / R(5.98));
    f.eks_num = c[10] + c[9] * c[11];
    return f;
}

template <typename R>
EP_HD void tt_rev_na(TTRev<R> &e, R Nai, const R *c, const TTFixed<R> &f) {
    e.ENa = f.rtf * log(c[11] / Nai);
}
template <typename R>
EP_HD void tt_rev_k(TTRev<R> &e, R Ki, const R *c, const TTFixed<R> &f) {
    e.EK = f.rtf * log(c[10] / Ki);
    const R vk = f.V - e.EK;
    const R a = R(0.1) / (R(1) + exp(R(0.06) * (vk - R(200))));
    const R b = (R(3) * exp(R(0.0002) * (vk + R(100))) + exp(R(0.1) * (vk - R(10))))
              / (R(1) + exp(R(-0.5) * vk));
    e.xk1 = a / (a + b);
}
template <typename R>
EP_HD void tt_rev_ks(TTRev<R> &e, R Ki, R Nai, const R *c, const TTFixed<R> &f) {
    e.EKs = f.rtf * log(f.eks_num / (Ki + c[9] * Nai));
}
template <typename R>
EP_HD void tt_rev_ca(TTRev<R> &e, R Cai, const R *c, const TTFixed<R> &f) {
    e.ECa = f.rtf_half * log(c[12] / Cai);
}

// Rates of the 6 Newton states and dV/dt (Tusscher.cc:56-95) at
// x = (Ki, Nai, Cai, Cass, CaSR, R').
template <typename R>
EP_HD void tt_nr_rates(const R x[6], const TTRev<R> &e, const TTFixed<R> &f,
                                            const R *c, R r[6], R &dvdt) {
    const R V = f.V, F = f.F;
    const R Ki = x[0], Nai = x[1], Cai = x[2], Cass = x[3], Casr = x[4], Rp = x[5];
    (void)Ki;
    const R i_nak = (f.nak_fac * Nai) / (Nai + c[23]) / f.nak_den;
    const R i_na = f.g_na * (V - e.ENa);
    const R i_bna = c[17] * (V - e.ENa);
    const R i_naca = (c[24] * (f.e_g * (Nai * Nai * Nai) * c[12] - f.e_g1 * f.nao3 * Cai * c[26])) / f.naca_den;
    const R vk = V - e.EK;
    const R i_k1 = c[13] * e.xk1 * f.sq_ko * vk;
    const R i_to = f.g_to * vk;
    const R i_kr = f.g_kr * vk;
    const R i_ks = f.g_ks * (V - e.EKs);
    const R i_cal = (f.cal_pre * (R(0.25) * Cass * f.e_ca - c[12])) / f.cal_den;
    const R i_bca = c[19] * (V - e.ECa);
    const R i_pk = (c[32] * vk) / f.pk_den;
    const R i_pca = (c[30] * Cai) / (Cai + c[31]);
    const R c4F = c[4] * F;
    dvdt = -(i_k1 + i_to + i_kr + i_ks + i_cal + i_nak + i_na + i_bna + i_naca + i_bca + i_pk + i_pca + f.ist);
    r[0] = ((-((i_k1 + i_to + i_kr + i_ks + i_pk + f.ist) - R(2) * i_nak)) / c4F) * c[3];
    r[1] = ((-(i_na + i_bna + R(3) * i_nak + R(3) * i_naca)) / c4F) * c[3];
    const R j_up = c[44] / (R(1) + (c[42] * c[42]) / (Cai * Cai));
    const R j_leak = c[43] * (Casr - Cai);
    const R j_xfer = c[41] * (Cass - Cai);
    const R bufc = R(1) / (R(1) + (c[45] * c[46]) / ((Cai + c[46]) * (Cai + c[46])));
    r[2] = bufc * ((((j_leak - j_up) * c[51]) / c[4] + j_xfer)
                   - (((i_bca + i_pca) - R(2) * i_naca) * c[3]) / (R(2) * c[4] * F));
    const R t = c[37] / Casr;
    const R kcasr = c[38] - (c[38] - c[39]) / (R(1) + t * t);
    const R k2 = c[34] * kcasr;
    r[5] = -k2 * Cass * Rp + c[36] * (R(1) - Rp);
    const R k1 = c[33] / kcasr;
    const R O = (k1 * (Cass * Cass) * Rp) / (c[35] + k1 * (Cass * Cass));
    const R j_rel = c[40] * O * (Casr - Cass);
    const R bufsr = R(1) / (R(1) + (c[47] * c[48]) / ((Casr + c[48]) * (Casr + c[48])));
    r[4] = bufsr * (j_up - (j_rel + j_leak));
    const R bufss = R(1) / (R(1) + (c[49] * c[50]) / ((Cass + c[50]) * (Cass + c[50])));
    r[3] = bufss * (((-i_cal * c[3]) / (R(2) * c[52] * F) + (j_rel * c[51]) / c[52])
                    - (j_xfer * c[4]) / c[52]);
}

// dV/dt of the model at an arbitrary state (the current balance of
// ComputeRates, Tusscher.cc:56-78), s = the 18 stored states
template <typename R>
EP_HD R tt_dvdt(R V, const R *s, const R *__restrict__ c, R ist, R gks) {
    const TTFixed<R> f = tt_fixed<R>(V, s, c, ist, gks);
    TTRev<R> e;
    tt_rev_na(e, s[1], c, f);
    tt_rev_k(e, s[0], c, f);
    tt_rev_ks(e, s[0], s[1], c, f);
    tt_rev_ca(e, s[2], c, f);
    const R x[6] = {s[0], s[1], s[2], s[9], s[16], s[17]};
    R r[6], dvdt;
    tt_nr_rates(x, e, f, c, r, dvdt);
    return dvdt;
}

// In-register 6x6 solve A x = b, A column-major (LAPACK convention),
// partial pivoting in the getf2 order; b is overwritten with x.
template <typename R>
EP_HD void lu6_solve(R a[36], R b[6]) {
#pragma unroll
    for (int k = 0; k < 6; k++) {
        int p = k;
        R amax = fabs(a[k + k * 6]);
#pragma unroll
        for (int i = k + 1; i < 6; i++) {
            const R v = fabs(a[i + k * 6]);
            if (v > amax) { amax = v; p = i; }
        }
        // swap rows k and p (p >= k) with selects so the arrays stay in registers
#pragma unroll
        for (int i = k + 1; i < 6; i++) {
            const bool sw = (p == i);
#pragma unroll
            for (int jj = 0; jj < 6; jj++) {
                const R ak = a[k + jj * 6], ai = a[i + jj * 6];
                a[k + jj * 6] = sw ? ai : ak;
                a[i + jj * 6] = sw ? ak : ai;
            }
            const R bk = b[k], bi = b[i];
            b[k] = sw ? bi : bk;
            b[i] = sw ? bk : bi;
        }
        const R piv = a[k + k * 6];
        const R rp = (piv != R(0)) ? R(1) / piv : R(0);
#pragma unroll
        for (int i = k + 1; i < 6; i++) a[i + k * 6] *= rp;
#pragma unroll
        for (int jj = k + 1; jj < 6; jj++) {
            const R ukj = a[k + jj * 6];
#pragma unroll
            for (int i = k + 1; i < 6; i++) a[i + jj * 6] -= a[i + k * 6] * ukj;
        }
    }
    // The row interchanges were applied to b while eliminating, which is the
    // same permutation getrs applies before the forward solve.
#pragma unroll
    for (int jj = 0; jj < 6; jj++)
#pragma unroll
        for (int i = jj + 1; i < 6; i++) b[i] -= b[jj] * a[i + jj * 6];
#pragma unroll
    for (int jj = 5; jj >= 0; jj--) {
        b[jj] /= a[jj + jj * 6];
#pragma unroll
        for (int i = 0; i < jj; i++) b[i] -= b[jj] * a[i + jj * 6];
    }
}

// the 12 gates of one Compute_Ion call: semi-implicit (s + dt inf/tau) /
// (1 + dt/tau) at voltage V (UpdateStateVariables, Tusscher.cc:116-195)
template <typename R>
EP_HD void tt_gate_step(R s[TT_NS], R V, R dt, const R *__restrict__ c) {
    R ginf[12], gtau[12];
    tt_gates(V, s[9], c, ginf, gtau);
    const int gidx[12] = {3, 4, 5, 6, 7, 8, 10, 11, 12, 13, 14, 15};
#pragma unroll
    for (int g = 0; g < 12; g++) {
        const R b = R(-1) / gtau[g];
        const R a = ginf[g] / gtau[g];
        s[gidx[g]] = (s[gidx[g]] + dt * a) / (R(1) - dt * b);
    }
}

struct TTOpts {
    int newton_cap;
    int jac_true;
    int fp32_scaled_tol;
    double newton_tol;
};

// One Compute_Ion call: s (18 stored states) advanced in place by dt at
// frozen voltage V; returns dV/dt at the final Newton iterate.  *iters
// receives the Newton iteration count (capped by opt.newton_cap).
template <typename R>
EP_HD R tt_compute_ion(R s[TT_NS], R V, R ist, R dt, const R *__restrict__ c,
                                            R gks, const TTOpts &opt, int &iters) {
    tt_gate_step(s, V, dt, c);
    const TTFixed<R> f = tt_fixed<R>(V, s, c, ist, gks);
    // Newton slots: Ki s0, Nai s1, Cai s2, Cass s9, CaSR s16, R' s17
    R x[6] = {s[0], s[1], s[2], s[9], s[16], s[17]};
    R xn[6];
#pragma unroll
    for (int i = 0; i < 6; i++) xn[i] = x[i];
    TTRev<R> e;
    tt_rev_na(e, x[1], c, f);
    tt_rev_k(e, x[0], c, f);
    tt_rev_ks(e, x[0], x[1], c, f);
    tt_rev_ca(e, x[2], c, f);
    R old[6], dvdt;
    tt_nr_rates(x, e, f, c, old, dvdt);

    const R tol = R(opt.newton_tol);
    R resid = R(100);
    int it = 0;
    while (resid > tol) {
        if (it >= opt.newton_cap) break;
        R J[36];
#pragma unroll
        for (int i = 0; i < 6; i++) {
            const R eps = R(1e-3) * x[i];
            const R twoeps = R(2) * eps;
            R fp[6], fm[6], rr[6], dd;
            const R xi = x[i];
            TTRev<R> ep = e;
            x[i] = xi + eps;
            if (i == 0) { tt_rev_k(ep, x[0], c, f); tt_rev_ks(ep, x[0], x[1], c, f); }
            if (i == 1) { tt_rev_na(ep, x[1], c, f); tt_rev_ks(ep, x[0], x[1], c, f); }
            if (i == 2) { tt_rev_ca(ep, x[2], c, f); }
            tt_nr_rates(x, ep, f, c, rr, dd);
#pragma unroll
            for (int k = 0; k < 6; k++) fp[k] = x[k] - xn[k] - dt * rr[k];
            x[i] = x[i] - R(2) * eps;
            if (i == 0) { tt_rev_k(ep, x[0], c, f); tt_rev_ks(ep, x[0], x[1], c, f); }
            if (i == 1) { tt_rev_na(ep, x[1], c, f); tt_rev_ks(ep, x[0], x[1], c, f); }
            if (i == 2) { tt_rev_ca(ep, x[2], c, f); }
            tt_nr_rates(x, ep, f, c, rr, dd);
#pragma unroll
            for (int k = 0; k < 6; k++) fm[k] = x[k] - xn[k] - dt * rr[k];
            x[i] = x[i] + eps;
#pragma unroll
            for (int k = 0; k < 6; k++) {
                const R v = (fp[k] - fm[k]) / twoeps;
                if (opt.jac_true) J[i * 6 + k] = v;   // column-major J(k, i)
                else J[k * 6 + i] = v;                // the reference's layout
            }
        }
        R B[6];
#pragma unroll
        for (int i = 0; i < 6; i++) B[i] = x[i] - xn[i] - dt * old[i];
        lu6_solve(J, B);
#pragma unroll
        for (int i = 0; i < 6; i++) x[i] -= B[i];
        tt_rev_na(e, x[1], c, f);
        tt_rev_k(e, x[0], c, f);
        tt_rev_ks(e, x[0], x[1], c, f);
        tt_rev_ca(e, x[2], c, f);
        tt_nr_rates(x, e, f, c, old, dvdt);
        R acc = R(0);
        if (opt.fp32_scaled_tol) {
#pragma unroll
            for (int i = 0; i < 6; i++) {
                const R sc = fmax(fabs(x[i]), R(1));
                const R q = B[i] / sc;
                acc += q * q;
            }
        } else {
#pragma unroll
            for (int i = 0; i < 6; i++) acc += B[i] * B[i];
        }
        resid = sqrt(acc);
        it++;
    }
    s[0] = x[0]; s[1] = x[1]; s[2] = x[2]; s[9] = x[3]; s[16] = x[4]; s[17] = x[5];
    iters = it;
    return dvdt;
}

#ifdef __CUDACC__
// tt_compute_ion with one node per warp, for short node lists (a single
// upstroke node's Newton is a long serial chain).  Every lane holds the node's
// state and runs the gate step, the fixed terms, the LU solve and the update
// (the same bits on every lane); the 12 perturbed rate evaluations of the
// finite-difference Jacobian run one per lane (lane 2i: column i plus side,
// lane 2i + 1: minus side; lanes 12..31 repeat lane 0's) and their residuals
// are gathered by shuffles.  Each lane rebuilds the state the sequential loop
// has when it reaches its evaluation -- x_i + eps and (x_i + eps) - 2 eps for
// column i, and the earlier columns' entries after their round trip
// ((x_j + eps) - 2 eps) + eps -- and the update continues from those
// round-tripped entries, as the sequential loop does, so the result is
// tt_compute_ion's to the bit.
template <typename R>
__device__ __forceinline__ R tt_compute_ion_warp(R s[TT_NS], R V, R ist, R dt, const R *__restrict__ c, R gks,
                                                 const TTOpts &opt, int &iters, int lane) {
    tt_gate_step(s, V, dt, c);
    const TTFixed<R> f = tt_fixed<R>(V, s, c, ist, gks);
    R x[6] = {s[0], s[1], s[2], s[9], s[16], s[17]};
    R xn[6];
#pragma unroll
    for (int i = 0; i < 6; i++) xn[i] = x[i];
    TTRev<R> e;
    tt_rev_na(e, x[1], c, f);
    tt_rev_k(e, x[0], c, f);
    tt_rev_ks(e, x[0], x[1], c, f);
    tt_rev_ca(e, x[2], c, f);
    R old[6], dvdt;
    tt_nr_rates(x, e, f, c, old, dvdt);

    const int col = (lane >> 1) < 6 ? (lane >> 1) : 0;
    const bool minus = (lane & 1) && (lane >> 1) < 6;
    const R tol = R(opt.newton_tol);
    R resid = R(100);
    int it = 0;
    while (resid > tol) {
        if (it >= opt.newton_cap) break;
        R eps[6], xd[6];
#pragma unroll
        for (int i = 0; i < 6; i++) {
            eps[i] = R(1e-3) * x[i];
            const R up = x[i] + eps[i];
            xd[i] = (up - R(2) * eps[i]) + eps[i];
        }
        // this lane's evaluation: column col's entry perturbed, the columns
        // before it round-tripped, the ones after it as they are
        R xp[6];
#pragma unroll
        for (int k = 0; k < 6; k++) {
            const R up = x[k] + eps[k];
            xp[k] = k < col ? xd[k] : k == col ? (minus ? up - R(2) * eps[k] : up) : x[k];
        }
        TTRev<R> ep = e;
        if (col == 0) { tt_rev_k(ep, xp[0], c, f); tt_rev_ks(ep, xp[0], xp[1], c, f); }
        if (col == 1) { tt_rev_na(ep, xp[1], c, f); tt_rev_ks(ep, xp[0], xp[1], c, f); }
        if (col == 2) { tt_rev_ca(ep, xp[2], c, f); }
        R rr[6], dd, F[6];
        tt_nr_rates(xp, ep, f, c, rr, dd);
#pragma unroll
        for (int k = 0; k < 6; k++) F[k] = xp[k] - xn[k] - dt * rr[k];
        R J[36];
#pragma unroll
        for (int i = 0; i < 6; i++) {
            const R twoeps = R(2) * eps[i];
#pragma unroll
            for (int k = 0; k < 6; k++) {
                const R fp = __shfl_sync(0xffffffffu, F[k], 2 * i);
                const R fm = __shfl_sync(0xffffffffu, F[k], 2 * i + 1);
                const R v = (fp - fm) / twoeps;
                if (opt.jac_true) J[i * 6 + k] = v;
                else J[k * 6 + i] = v;
            }
        }
#pragma unroll
        for (int i = 0; i < 6; i++) x[i] = xd[i];
        R B[6];
#pragma unroll
        for (int i = 0; i < 6; i++) B[i] = x[i] - xn[i] - dt * old[i];
        lu6_solve(J, B);
#pragma unroll
        for (int i = 0; i < 6; i++) x[i] -= B[i];
        tt_rev_na(e, x[1], c, f);
        tt_rev_k(e, x[0], c, f);
        tt_rev_ks(e, x[0], x[1], c, f);
        tt_rev_ca(e, x[2], c, f);
        tt_nr_rates(x, e, f, c, old, dvdt);
        R acc = R(0);
        if (opt.fp32_scaled_tol) {
#pragma unroll
            for (int i = 0; i < 6; i++) {
                const R sc = fmax(fabs(x[i]), R(1));
                const R q = B[i] / sc;
                acc += q * q;
            }
        } else {
#pragma unroll
            for (int i = 0; i < 6; i++) acc += B[i] * B[i];
        }
        resid = sqrt(acc);
        it++;
    }
    s[0] = x[0]; s[1] = x[1]; s[2] = x[2]; s[9] = x[3]; s[16] = x[4]; s[17] = x[5];
    iters = it;
    return dvdt;
}
#endif

}  // namespace ep
