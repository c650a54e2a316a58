// mahajan.cuh -- Mahajan 2008 UCLA rabbit ventricular model, device side.
//
// Follows voomEP/src/IonicModel/Mahajan.cc: ucla_rhsfun (168-219) with the
// current routines (227-603), forward Euler with Rush-Larsen-type gate
// rates, and the adaptive update of UpdateStateVariables (607-621): if
// |dV/dt| > 20 the step is redone as 10 sub-steps of dt/10, and
// Compute_Ion (624-645) returns the rate of the LAST sub-step.
// Mahajan_fail.cc is the same code with other constants.
#pragma once
#include "common.cuh"

namespace ep {

constexpr int MH_NS = 25;   // stored states besides V: reference State[1..25]
constexpr int MH_NC = 35;

// r[k] receives the rate of reference state k (k = 0..25); s[k] holds
// reference state k (s[0] = V).
template <typename R>
EP_HD void mh_rhs(const R s[26], const R *__restrict__ c, R h, R istim, R r[26]) {
    const R V = s[0], frt = c[24];
    const R inv_frt = R(1) / frt;
    // I_K1
    const R ek1 = inv_frt * log((R(100) * c[2] + R(1) * c[0]) / (R(100) * c[1] + R(1) * s[19]));
    const R gki = sqrt(c[2] / R(5.4));
    const R aki = R(1.02) / (R(1) + exp(R(0.2385) * (V - ek1 - R(59.215))));
    const R bki = (R(0.49124) * exp(R(0.08032) * (V - ek1 + R(5.476))) + exp(R(0.061750) * (V - ek1 - R(594.31))))
                / (R(1) + exp(R(-0.5143) * (V - ek1 + R(4.753))));
    const R xik1 = c[11] * gki * (aki / (aki + bki)) * (V - ek1);
    // I_to (slow + fast)
    const R ek = inv_frt * log(c[2] / c[1]);
    const R rt1 = -(V + R(3)) / R(15), rt2 = (V + R(33.5)) / R(10), rt3 = (V + R(60)) / R(10);
    const R xtos_inf = R(1) / (R(1) + exp(rt1));
    const R ytos_inf = R(1) / (R(1) + exp(rt2));
    const R txs = R(9) / (R(1) + exp(-rt1)) + R(0.5);
    const R tys = R(3000) / (R(1) + exp(rt3)) + R(30);
    const R xitos = c[6] * s[22] * (s[23] + R(0.5) * ytos_inf) * (V - ek);
    r[22] = (xtos_inf - (xtos_inf - s[22]) * exp(-h / txs) - s[22]) / h;
    r[23] = (ytos_inf - (ytos_inf - s[23]) * exp(-h / tys) - s[23]) / h;
    const R rt4 = -(V / R(30)) * (V / R(30));
    const R txf = R(3.5) * exp(rt4) + R(1.5);
    const R tyf = R(20) / (R(1) + exp(rt2)) + R(20);
    const R xitof = c[7] * s[20] * s[21] * (V - ek);
    r[20] = (xtos_inf - (xtos_inf - s[20]) * exp(-h / txf) - s[20]) / h;
    r[21] = (ytos_inf - (ytos_inf - s[21]) * exp(-h / tyf) - s[21]) / h;
    const R xito = xitos + xitof;
    // I_NaK
    const R sigma = (exp(c[0] / R(67.3)) - R(1)) / R(7);
    const R fnak = R(1) / (R(1) + R(0.1245) * exp(R(-0.1) * V * frt) + R(0.0365) * sigma * exp(-V * frt));
    const R xinak = c[12] * fnak * (R(1) / (R(1) + (R(12) / s[19]))) * c[2] / (c[2] + R(1.5));
    // Na-Ca exchange flux
    const R csm = s[8] / R(1000);
    const R na3 = s[19] * s[19] * s[19], nao3 = c[0] * c[0] * c[0];
    const R ez = exp(V * (R(0.35) - R(1)) * frt);
    R jnaca;
    {
        const R zw3 = na3 * c[3] * exp(V * R(0.35) * frt) - nao3 * csm * ez;
        const R zw4 = R(1) + R(0.2) * ez;
        const R q = R(0.3) / s[8];
        const R aloss = R(1) / (R(1) + q * q * q);
        const R yz1 = R(1.3) * na3 + R(669921.875) * csm;               // 87.5^3
        const R yz2 = R(1860.867) * c[3] * (R(1) + csm / R(0.0036));    // 12.3^3
        const R qn = s[19] / R(12.3);
        const R yz3 = R(0.0036) * nao3 * (R(1) + qn * qn * qn);
        const R yz4 = na3 * c[3] + nao3 * csm;
        jnaca = c[8] * aloss * zw3 / (zw4 * (yz1 + yz2 + yz3 + yz4));
    }
    // Ca cycling
    const R jd = c[28] * (s[8] - s[9]) / c[14];
    r[24] = c[29] * (R(0.0327) * s[9] * (R(70) - s[24]) - R(0.0196) * s[24]);
    r[25] = R(0.0327) * s[8] * (R(70) - s[25]) - R(0.0196) * s[25];
    const R jup = c[30] * (c[13] * s[9] * s[9] / (s[9] * s[9] + R(0.25)));
    const R jleak = c[27] * (R(0.00002069) * s[10] * s[10] / (s[10] * s[10] + R(2500)) * (s[10] * R(16.667) - s[9]));
    // Markov L-type Ca channel
    R po;
    {
        const R poinf = R(1) / (R(1) + exp(-V / R(8)));
        const R alpha = poinf, beta = R(1) - poinf;
        const R r1 = R(0.30), r2 = R(3);
        const R q = R(3) / s[7];
        const R fca = R(1) / (R(1) + q * q * q);
        const R s1 = R(0.0182688) * fca, s1t = R(0.00195);
        const R k1 = R(0.024168) * fca;
        const R k2 = R(1.03615e-4), k1t = R(0.00413), k2t = R(0.00224);
        const R s2 = s1 * (r1 / r2) * (k2 / k1);
        const R s2t = s1t * (r1 / r2) * (k2t / k1t);
        const R poi = R(1) / (R(1) + exp(-(V + R(40)) / R(3)));
        const R k3 = (R(1) - poi) / R(3), k3t = k3;
        const R Pr = R(1) - R(1) / (R(1) + exp(-(V + R(40)) / R(4)));
        const R recov = R(10) + R(4954) * exp(V / R(15.6));
        const R qc = s[7] / R(6.09365);
        const R qc2 = qc * qc;
        const R tau_ca = R(78.0329) / (R(1) + qc2 * qc2) + R(0.1);
        const R tauca = (recov - tau_ca) * Pr + tau_ca;
        const R tauba = (recov - R(450)) * Pr + R(450);
        const R Ps = R(1) / (R(1) + exp(-(V + R(40)) / R(11.32)));
        const R k6 = fca * Ps / tauca, k5 = (R(1) - Ps) / tauca;
        const R k6t = Ps / tauba, k5t = (R(1) - Ps) / tauba;
        const R k4 = k3 * (alpha / beta) * (k1 / k2) * (k5 / k6);
        const R k4t = k3t * (alpha / beta) * (k1t / k2t) * (k5t / k6t);
        po = R(1) - s[15] - s[17] - s[16] - s[18] - s[13] - s[14];
        r[14] = beta * s[13] + k5 * s[17] + k5t * s[18] - (k6 + k6t + alpha) * s[14];
        r[13] = alpha * s[14] + k2 * s[15] + k2t * s[16] + r2 * po - (beta + r1 + k1t + k1) * s[13];
        r[15] = k1 * s[13] + k4 * s[17] + s1 * po - (k3 + k2 + s2) * s[15];
        r[17] = k3 * s[15] + k6 * s[14] - (k5 + k4) * s[17];
        r[16] = k1t * s[13] + k4t * s[18] + s1t * po - (k3t + k2t + s2t) * s[16];
        r[18] = k3t * s[16] + k6t * s[14] - (k5t + k4t) * s[18];
    }
    // driving force of I_Ca
    R rxa;
    {
        const R za = V * R(2) * frt;
        const R factor1 = R(4) * R(0.00054) * c[23] * c[23] / (c[22] * c[20]);
        const R ez2 = exp(za);
        if (fabs(za) < R(0.001))
            rxa = factor1 * (csm * ez2 - R(0.341) * c[3]) / (R(2) * frt);
        else
            rxa = V * factor1 * (csm * ez2 - R(0.341) * c[3]) / (ez2 - R(1));
    }
    const R jca = c[4] * po * rxa;
    auto buf = [](R cv) {
        return R(1) / (R(1) + R(168) / ((R(7) + cv) * (R(7) + cv)) + R(28.2) / ((R(0.6) + cv) * (R(0.6) + cv))
                       + R(4.5) / ((R(0.3) + cv) * (R(0.3) + cv)) + R(546) / ((R(13) + cv) * (R(13) + cv)));
    };
    r[8] = buf(s[8]) * (R(50) * (s[12] - jd - jca + jnaca) - r[25]);
    r[9] = buf(s[9]) * (jd - jup + jleak - r[24]);
    r[10] = -s[12] + jup - jleak;
    r[11] = (s[10] - s[11]) / c[17];
    R Qr;
    {
        const R bv = (c[19] - c[26]) - c[18] * c[19];
        R q = R(0);
        if (s[11] > c[26] && s[11] < c[19]) q = s[11] - c[26];
        else if (s[11] >= c[19]) q = c[18] * s[11] + bv;
        if (q >= c[25]) q = c[25];
        Qr = s[10] * q / c[19];
    }
    const R arxa = fabs(rxa);
    {
        const R e = exp(R(-0.05) * (V + R(30)));
        const R sparkV = e / (R(1) + e);
        const R spark_rate = R(2.58079) * po * arxa * sparkV;
        r[12] = spark_rate * Qr - s[12] * (R(1) - c[16] * r[10] / s[10]) / c[16];
    }
    {
        const R e = exp(R(-0.3576) * (V + R(30)));
        const R gsr = R(26841.8) * e / (R(1) + e);
        r[7] = po * Qr * arxa * gsr + po * R(9000) * arxa - (s[7] - s[8]) / R(0.5);
    }
    // I_Na
    R xina;
    {
        const R ena = inv_frt * log(c[0] / s[19]);
        R am = R(3.2);
        if (fabs(V + R(47.13)) > R(0.001)) am = R(0.32) * (V + R(47.13)) / (R(1) - exp(R(-0.1) * (V + R(47.13))));
        const R bm = R(0.08) * exp(-V / R(11));
        const R a = R(1) - R(1) / (R(1) + exp(-(V + R(40)) / R(0.24)));
        const R ah = a * R(0.135) * exp((R(80) + V) / R(-6.8));
        const R bh = (R(1) - a) / (R(0.13) * (R(1) + exp((V + R(10.66)) / R(-11.1))))
                   + a * (R(3.56) * exp(R(0.079) * V) + R(3.1e5) * exp(R(0.35) * V));
        const R aj = a * (R(-1.2714e5) * exp(R(0.2444) * V) - R(3.474e-5) * exp(R(-0.04391) * V)) * (V + R(37.78))
                   / (R(1) + exp(R(0.311) * (V + R(79.23))));
        const R bj = (R(1) - a) * (R(0.3) * exp(R(-2.535e-7) * V) / (R(1) + exp(R(-0.1) * (V + R(32)))))
                   + a * (R(0.1212) * exp(R(-0.01052) * V) / (R(1) + exp(R(-0.1378) * (V + R(40.14)))));
        const R tauh = R(1) / (ah + bh);
        const R tauj = c[34] * (R(1) / (aj + bj));
        const R taum = R(1) / (am + bm);
        const R gm = (s[1] + c[31]) / (R(1) + c[31]);
        xina = c[15] * ((s[2] + c[32]) / (R(1) + c[32])) * ((s[3] + c[33]) / (R(1) + c[33])) * (gm * gm * gm) * (V - ena);
        r[2] = (ah * tauh - (ah * tauh - s[2]) * exp(-h / tauh) - s[2]) / h;
        r[3] = (aj * tauj - (aj * tauj - s[3]) * exp(-h / tauj) - s[3]) / h;
        r[1] = (am * taum - (am * taum - s[1]) * exp(-h / taum) - s[1]) / h;
    }
    // I_Kr
    R xikr;
    {
        const R gss = sqrt(c[2] / R(5.4));
        R v1 = R(0.00138) / R(0.123);
        if (fabs(V + R(7)) > R(0.001)) v1 = R(0.00138) * (V + R(7)) / (R(1) - exp(R(-0.123) * (V + R(7))));
        R v2 = R(0.00061) / R(0.145);
        if (fabs(V + R(10)) > R(0.001)) v2 = R(0.00061) * (V + R(10)) / (exp(R(0.145) * (V + R(10))) - R(1));
        const R taukr = R(1) / (v1 + v2);
        const R xkrinf = R(1) / (R(1) + exp(-(V + R(50)) / R(7.5)));
        const R rg = R(1) / (R(1) + exp((V + R(33)) / R(22.4)));
        xikr = c[9] * gss * s[4] * rg * (V - ek);
        r[4] = (xkrinf - (xkrinf - s[4]) * exp(-h / taukr) - s[4]) / h;
    }
    // I_Ks
    R xiks;
    {
        const R eks = inv_frt * log((c[2] + R(0.018330) * c[0]) / (c[1] + R(0.018330) * s[19]));
        const R xs1ss = R(1) / (R(1) + exp(-(V - R(1.5)) / R(16.7)));
        R tauxs1;
        if (fabs(V + R(30)) < R(0.001) / R(0.0687))
            tauxs1 = R(1) / (R(0.0000719) / R(0.148) + R(0.000131) / R(0.0687));
        else
            tauxs1 = R(1) / (R(0.0000719) * (V + R(30)) / (R(1) - exp(R(-0.148) * (V + R(30))))
                             + R(0.000131) * (V + R(30)) / (exp(R(0.0687) * (V + R(30))) - R(1)));
        const R tauxs2 = R(4) * tauxs1;
        const R q = R(0.5) / s[9];
        const R gksx = R(1) + R(0.8) / (R(1) + q * q * q);
        xiks = c[10] * gksx * s[5] * s[6] * (V - eks);
        r[5] = (xs1ss - (xs1ss - s[5]) * exp(-h / tauxs1) - s[5]) / h;
        r[6] = (xs1ss - (xs1ss - s[6]) * exp(-h / tauxs2) - s[6]) / h;
    }
    const R wca = R(8.0313);
    r[19] = -(R(1) / wca / R(1000)) * (xina + R(3) * xinak + R(3) * wca * jnaca);
    r[0] = -(xina + xik1 + xikr + xiks + xito + wca * jnaca + R(2) * wca * jca + xinak) + istim;
}

// Compute_Ion; s[0..25] = reference State (s[0] overwritten with V).
template <typename R>
EP_HD R mh_compute_ion(R s[26], R V, R istim_pApF, R dt, const R *__restrict__ c,
                                            int abs_mode, int &substepped) {
    R r[26];
    s[0] = V;
    mh_rhs(s, c, dt, istim_pApF, r);
    const R mag = abs_mode ? fabs(r[0]) : R(abs((int)r[0]));
    if (mag > R(20)) {
        const R h = dt / R(10);
#pragma unroll 1
        for (int k = 0; k < 10; k++) {
            mh_rhs(s, c, h, istim_pApF, r);
#pragma unroll
            for (int j = 0; j < 26; j++) s[j] += r[j] * dt / R(10);
        }
        substepped = 1;
    } else {
#pragma unroll
        for (int j = 0; j < 26; j++) s[j] += r[j] * dt;
        substepped = 0;
    }
    return r[0];
}

}  // namespace ep
