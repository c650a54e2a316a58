// purkinje.cuh -- Corrias 2011 rabbit Purkinje cell, host+device source.
//
// Follows voomEP/src/IonicModel/Purkinje.cc: ComputeRates (5-103), the
// adaptive forward Euler of UpdateStateVariables (157-173: one step of dt,
// or ten of dt/10 when |dV/dt| > 1.5 mV/ms at the start, every state V
// included) and Compute_Ion (183-213: V into State[0], the stimulus in pA
// through the cell's surface area and Xi, the LAST evaluated dV/dt
// returned).  Parameters: SetUpPurkinjeParameters (SetUpIonicConstants.h:
// 16-85), 63 entries.  CardiacBody::New gives this cell to every node of a
// .purk list (Body/CardiacBody.cc:982-1101).
#pragma once
#include "common.cuh"

namespace ep {

constexpr int PK_NS = 21;      // stored states besides V: reference State[1..21]
constexpr int PK_NC = 63;
constexpr double PK_AREA = 4.612e-5;   // cell surface area, cm^2 (Purkinje.h:56)

// r[k] = rate of reference state k (r[0] = dV/dt); s[k] = reference state k
// (s[0] = V); istim_pA enters the balances as the reference's Algebraic[0]
template <typename R>
EP_HD void pk_rates(const R s[22], const R *__restrict__ c, R istim_pA, R r[22]) {
    const R V = s[0];
    // gates relax to their steady states
    const R v30 = V + R(30), v7 = V + R(7), v10 = V + R(10);
    const R cai_f = R(1) + pow(s[1] / R(0.0001), R(2));
    const R tau18 = fabs(v30) < R(0.0145)
                        ? R(417.946)
                        : R(1) / ((R(7.19e-05) * v30) / (R(1) - exp(R(-0.148) * v30)) +
                                  (R(0.000131) * v30) / (exp(R(0.0687) * v30) - R(1)));
    const R ss18 = R(1) / (R(1) + exp((V - R(1.5)) / R(-16.7)));
    const R ssf = R(1) / (R(1) + exp((V + R(109)) / R(10)));
    const R tauf = R(6000) / (exp(R(-1) * (R(2.9) + R(0.04) * V)) + exp(R(1) * (R(3.6) + R(0.11) * V)));
    const R a17 = fabs(v7) > R(0.001) ? (R(0.00138) * R(1) * v7) / (R(1) - exp(R(-0.123) * v7)) : R(0.00138) / R(0.123);
    const R b17 = fabs(v10) > R(0.001) ? (R(6.1e-05) * R(1) * v10) / (exp(R(0.145) * v10) - R(1)) : R(0.00061) / R(0.145);
    r[6] = (R(1) / (R(1) + exp((V + R(47.8)) / R(-5.5))) - s[6]) / c[16];
    r[8] = (R(1) / (R(1) + exp((V + R(14.6)) / R(-5.5))) - s[8]) / c[18];
    r[11] = (R(1) / (R(1) + exp((V + R(-7)) / R(-9))) - s[11]) / c[20];
    r[12] = (R(1) / (R(1) + exp((V + R(27.5)) / R(8))) - s[12]) / c[21];
    r[13] = (R(1) / (R(1) + exp((V + R(25)) / R(-5))) - s[13]) / c[24];
    r[14] = (R(1) / (R(1) + exp((V + R(69)) / R(3.96))) - s[14]) / c[25];
    r[15] = (R(1) / (R(1) + exp((V + R(30)) / R(-5))) - s[15]) / c[27];
    r[7] = (R(1) / (R(1) + exp((V + R(67.9)) / R(3.87))) - s[7]) / (R(1.42271) * exp(R(-0.05119) * V));
    r[9] = (R(1) / (R(1) + exp((V + R(31)) / R(5.54))) - s[9]) /
           (R(25.1) / (R(0.04) + R(0.7) * exp(R(-1) * pow(R(0.028) * (V + R(14.5)), R(2)))));
    r[10] = (R(0.4) + R(0.6) / cai_f - s[10]) / (R(2) + R(80) / cai_f);
    r[16] = (R(0.1) + R(0.9) / (R(1) + exp((V + R(75.6)) / R(6.3))) - s[16]) /
            (R(120) + R(1) * exp((V + R(100)) / R(25)));
    r[18] = (ss18 - s[18]) / tau18;
    r[20] = (ssf - s[20]) / tauf;
    r[21] = (ssf - s[21]) / tauf;
    r[17] = (R(1) / (R(1) + exp((V + R(50)) / R(-7.5))) - s[17]) / (R(1) / (a17 + b17));
    r[19] = (ss18 - s[19]) / (R(4) * tau18);
    // reversal potentials (c[58] = RT/F)
    const R rtf = c[58];
    const R ek = rtf * log(c[5] / s[5]);
    const R ena = rtf * log(c[4] / s[4]);
    const R eca = R(0.5) * rtf * log(c[3] / s[1]);
    // membrane currents, pA
    const R ik1 = c[29] * pow(c[5] / R(5.4), R(0.8)) * (R(1) / (R(1) + exp((R(92) + V) / R(10)))) * (V - ek);
    const R ito = c[22] * s[11] * s[12] * (V - ek);
    const R ikp = c[23] * (R(1) / (R(1) + exp((R(5) - V) / R(17)))) * (V - ek);
    const R ikr = c[30] * pow(c[5] / R(5.4), R(1)) * (R(1) / (R(1) + exp((R(33) + V) / R(22.4)))) * s[17] * (V - ek);
    const R iks = c[31] * s[18] * s[19] * (V - ek);
    const R ikb = c[37] * (V - ek);
    const R inak = c[36] * (R(1) / (R(1) + exp((V + R(80)) / R(-45)))) * (R(1) / (R(1) + exp((V + R(0)) / R(125)))) *
                   (R(1) / (R(1) + pow(R(1.9) / c[5], R(1.45)))) * (R(1) / (R(1) + pow(R(31.98) / s[4], R(1))));
    const R ifk = c[43] * s[20] * (V - ek);
    const R ical = c[19] * s[8] * s[9] * s[10] * (V - eca);
    const R icat = c[17] * s[6] * s[7] * (V - eca);
    const R ina = c[26] * s[13] * s[14] * (V - ena);
    const R inal = c[28] * s[15] * s[16] * (V - ena);
    const R ipca = c[40] * (R(1) / (R(1) + pow(c[41] / s[1], c[42])));
    const R icab = c[39] * (V - eca);
    const R ifna = c[44] * s[21] * (V - ena);
    const R na_n = pow(s[4], c[32]), nao_n = pow(c[4], c[32]);
    const R inaca = (R(512.009) * c[33] *
                     (exp((c[35] * (c[32] - R(2)) * V) / rtf) * na_n * c[3] -
                      s[1] * exp(((c[35] - R(1)) * (c[32] - R(2)) * V) / rtf) * nao_n)) /
                    ((R(1) + c[34] * (s[1] * nao_n + c[3] * na_n)) * (R(1) + s[1] / R(0.0069)));
    const R inab = c[38] * (V - ena);
    r[0] = ((R(-1) * R(1)) / c[6]) * (ik1 + ito + ikp + ikr + iks + ikb + inak + ical + icat + ina + inal + ipca +
                                      icab + ifna + ifk + inaca + inab + istim_pA);
    r[5] = ((-ito - ikp - ikr - iks - ik1 - ikb - ifk - istim_pA + R(2) * inak) * R(1000)) / (c[1] * c[61]);
    r[4] = ((-ina - inal - R(3) * inak - R(3) * inaca - ifna - inab) * R(1000)) / (c[1] * c[61]);
    // calcium handling: release, the two uptakes, transfer, diffusion
    const R jrel = c[45] * (s[3] / (R(1) + pow(c[46] / s[1], R(2))));
    const R u1a = pow(s[1] / c[48], c[50]), u1b = pow(s[3] / c[49], c[50]);
    const R jup1 = c[47] * ((u1a - u1b) / (R(1) + u1a + u1b));
    const R u2a = pow(s[2] / c[52], c[54]), u2b = pow(s[3] / c[53], c[54]);
    const R jup2 = c[51] * ((u2a - u2b) / (R(1) + u2a + u2b));
    const R jtr = c[55] * (s[3] - s[2]);
    const R jdiff = c[56] * (s[1] - s[2]);
    r[3] = ((-jrel - jtr + jup2 + jup1) * R(1000)) / (R(2) * c[1] * c[62]);
    r[1] = ((-ical - icat - icab + R(1) * jrel - jup1 - jdiff + R(2) * inaca - ipca) * R(1000)) / (R(2) * c[1] * c[59]);
    r[2] = ((-jup2 + jdiff + jtr) * R(1000)) / (R(2) * c[1] * c[60]);
}

// One Compute_Ion call: s (22 reference states, s[0] overwritten by V) is
// advanced in place by dt; returns the last evaluated dV/dt.  istim in the
// reference's uA/cm^3, Xi the model's (2500 cm^-1) or the user's.
template <typename R>
EP_HD R pk_compute_ion(R s[22], R V, R istim, R Xi, R dt, const R *__restrict__ c, int &substepped) {
    R r[22];
    s[0] = V;
    const R istim_pA = R(-1e6) * istim * R(PK_AREA) / Xi;
    pk_rates(s, c, istim_pA, r);
    if (fabs(r[0]) > R(1.5)) {
        for (int k = 0; k < 10; k++) {
            pk_rates(s, c, istim_pA, r);
#pragma unroll
            for (int j = 0; j < 22; j++) s[j] += r[j] * dt / R(10);
        }
        substepped = 1;
    } else {
#pragma unroll
        for (int j = 0; j < 22; j++) s[j] += r[j] * dt;
        substepped = 0;
    }
    return r[0];
}

}  // namespace ep
