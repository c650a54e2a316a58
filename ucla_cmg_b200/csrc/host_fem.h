// host_fem.h -- host-side (FP64) P1-tet assembly of the Crank-Nicolson
// operators, the lumped capacitance and the per-node pseudo-ECG weights.
#pragma once
#include <cstdint>
#include <vector>

namespace ep {

struct HostCSR {
    int n = 0;
    std::vector<int> rowptr, col;   // sorted columns
    std::vector<double> A, B;       // A = Cm M + s K, B = Cm M - s K
    std::vector<double> CL;         // lumped capacitance (row sums of Cm M)
};

// Returns 0, or -1 if an element has a non-positive Jacobian.
// tets are zero-based.  s = dt/4 (+ smoothing 4 alpha / dt).
// scheme 0: Crank-Nicolson (A = Cm M + s K, B = Cm M - s K); 1: backward
// Euler (A = C_L + dt/2 K, B = diag C_L); 2: explicit (A = -K, B zero).
int assemble_cn(int n, const double *xyz, int m, const int *tets, const double *fibers,
                const double D[3], double Cm, double dt, double smoothing_alpha, HostCSR &out,
                int scheme = 0);

// W[k * n + i] with ECG_k = sum_i W V_i (ComputeECG.h:30-189 with grad V
// constant on a P1 tet).
void ecg_weights(int n, const double *xyz, int m, const int *tets, const double *fibers,
                 const double D[3], int ne, const double *electrodes, std::vector<double> &W);

// SELL-32 packing of a CSR pattern: slice_ptr (element offsets, multiples of
// 32), col, and the values of one or more value arrays.
struct Sell {
    int n = 0, nslices = 0;
    std::vector<int> slice_ptr, col;
    std::vector<std::vector<double>> vals;
};
void pack_sell(const HostCSR &a, const std::vector<const std::vector<double> *> &vals, Sell &out);

}  // namespace ep
