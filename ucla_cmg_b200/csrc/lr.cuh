// lr.cuh -- Luo-Rudy cell model as voomEP implements it, device side.
//
// Follows voomEP/src/IonicModel/LR.cc (Compute_Ion 65-100,
// make_parameter1 102-183): six Rush-Larsen gates x = inf - (inf - x)
// exp(-dt (alpha+beta)), forward Euler for Ca_i, and the optional voltage
// lookup table of LRGateTable.h (290001 rows over [-90, 200] mV, linear
// interpolation, 96-110).  The stimulus always uses the model's own Xi
// (LR.cc:99).
#pragma once
#include "common.cuh"

namespace ep {

constexpr int LR_NS = 7;   // stored states besides V: _in[0..6] (the reference keeps V in _in[7])
constexpr int LR_TAB = 14;

template <typename R>
__host__ __device__ __forceinline__ void lr_params(R v, R tab[LR_TAB]) {
    const R E_K1 = R(26.73) * log(R(5.4) / R(145.0));
    const R G_K1 = R(0.6047);
    R am, ah, aj, bh, bj, x1;
    if (fabs(v + R(47.13)) < R(0.001)) am = R(3.2);
    else am = R(0.32) * (v + R(47.13)) / (R(1) - exp(R(-0.1) * (v + R(47.13))));
    const R bm = R(0.08) * exp(-v / R(11));
    if (v > R(-40)) {
        ah = R(0); aj = R(0);
        bh = R(1) / (R(0.13) * (R(1) + exp(-(v + R(10.66)) / R(11.1))));
        bj = R(0.3) * exp(R(-2.535e-7) * v) / (R(1) + exp(R(-0.1) * (v + R(32))));
    } else {
        ah = R(0.135) * exp(-(R(80) + v) / R(6.8));
        aj = (R(-1.2714e5) * exp(R(0.2444) * v) - R(3.474e-5) * exp(R(-0.04391) * v)) * (v + R(37.78))
           / (R(1) + exp(R(0.311) * (v + R(79.23))));
        bh = R(3.56) * exp(R(0.079) * v) + R(3.1e5) * exp(R(0.35) * v);
        bj = R(0.1212) * exp(R(-0.01052) * v) / (R(1) + exp(R(-0.1378) * (v + R(40.14))));
    }
    const R ad = R(0.095) * exp(R(-0.01) * (v - R(5))) / (R(1) + exp(R(-0.072) * (v - R(5))));
    const R bd = R(0.07) * exp(R(-0.017) * (v + R(44))) / (R(1) + exp(R(0.05) * (v + R(44))));
    const R af = R(0.012) * exp(R(-0.008) * (v + R(28))) / (R(1) + exp(R(0.15) * (v + R(28))));
    const R bf = R(0.0065) * exp(R(-0.02) * (v + R(30))) / (R(1) + exp(R(-0.2) * (v + R(30))));
    const R ax = R(0.0005) * exp(R(0.083) * (v + R(50))) / (R(1) + exp(R(0.057) * (v + R(50))));
    const R bx = R(0.0013) * exp(R(-0.06) * (v + R(20))) / (R(1) + exp(R(-0.04) * (v + R(20))));
    if (v > R(-100)) {
        if (fabs(v + R(77)) < R(0.001)) x1 = R(0.608889);
        else x1 = R(2.837) * (exp(R(0.04) * (v + R(77))) - R(1)) / ((v + R(77)) * exp(R(0.04) * (v + R(35))));
    } else {
        x1 = R(1);
    }
    const R ak1 = R(1.02) / (R(1) + exp(R(0.2385) * (v - E_K1 - R(59.215))));
    const R b1 = R(0.49124) * exp(R(0.08032) * (v - E_K1 + R(5.476)));
    const R b2 = exp(R(0.06175) * (v - E_K1 - R(594.31)));
    const R b3 = R(1) + exp(R(-0.5143) * (v - E_K1 + R(4.753)));
    const R bk1 = (b1 + b2) / b3;
    const R I_k1 = G_K1 * (ak1 / (ak1 + bk1)) * (v - E_K1);
    const R kp = R(1) / (R(1) + exp((R(7.488) - v) / R(5.98)));
    const R I_kp = R(0.0183) * kp * (v - E_K1);
    const R I_b = R(0.0392) * (v + R(59.87));
    tab[0] = am / (am + bm); tab[1] = am + bm;
    tab[2] = ah / (ah + bh); tab[3] = ah + bh;
    tab[4] = aj / (aj + bj); tab[5] = aj + bj;
    tab[6] = ad / (ad + bd); tab[7] = ad + bd;
    tab[8] = af / (af + bf); tab[9] = af + bf;
    tab[10] = ax / (ax + bx); tab[11] = ax + bx;
    tab[12] = x1;
    tab[13] = I_k1 + I_kp + I_b;
}

// s: _in[0..6]; returns dV/dt (LR.cc:99)
template <typename R>
__device__ __forceinline__ R lr_compute_ion(R s[LR_NS], R V, R istim, R Cm, R dt, const R *table) {
    R tab[LR_TAB];
    if (table != nullptr && V > R(-90) && V < R(200)) {
        const int idx = (int)((V + R(90)) * R(1000));
        const R w = R(1000) * (V - (R(-90) + R(0.001) * R(idx)));
        const R *t0 = table + (size_t)idx * LR_TAB;
#pragma unroll
        for (int i = 0; i < LR_TAB; i++) {
            const R a = __ldg(t0 + i), b = __ldg(t0 + LR_TAB + i);
            tab[i] = (b - a) * w + a;
        }
    } else {
        lr_params(V, tab);
    }
#pragma unroll
    for (int i = 0; i < 6; i++) s[i] = tab[2 * i] - (tab[2 * i] - s[i]) * exp(-dt * tab[2 * i + 1]);
    const R Xi = R(2) * (R(11e-4) + R(100e-4)) / (R(11e-4) * R(100e-4));
    const R Es = R(7.7) - R(13.0287) * log(s[6]);
    const R i_na = R(12) * s[0] * s[0] * s[0] * s[1] * s[2] * (V - R(54.4));
    const R i_si = R(0.07) * s[3] * s[4] * (V - Es);
    const R i_k = R(0.705) * tab[12] * s[5] * (V + R(77));
    s[6] = s[6] + (R(-0.0001) * i_si + R(0.07) * (R(0.0001) - s[6])) * dt;
    const R i_tot = -(tab[13] + i_k + i_na + i_si);
    return i_tot + istim / (Xi * Cm);
}

}  // namespace ep
