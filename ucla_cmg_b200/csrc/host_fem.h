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

// 2-node Purkinje cables of a mixed mesh (MixedMesh3D.cc:62-108,
// CardiacBody.cc:100-187): zero-based bars, optional per-bar fibres (else
// isotropic Dp[0]) and LV flags (DpLeft), cable radius, the mesh's
// quadrature order (2: two Gauss points), and the .angle overrides of
// direction and length for cables starting at a listed node (sticky: the
// reference's never-reset flag keeps the last override for every later cable).
struct HostCables {
    int nb = 0;
    const int *bars = nullptr;
    const double *fibers = nullptr;
    const uint8_t *lv = nullptr;
    double Dp[3] = {0.0016, 0.0016, 0.0016}, DpLeft[3] = {0.0016, 0.0016, 0.0016};
    double radius = 0.0275;
    int quad_order = 2;
    const uint8_t *orient_has = nullptr;    // n
    const double *orient = nullptr;         // n * 4
    int orient_sticky = 1;
    // nb or null: per cable the node whose orient row overrides it (-1:
    // none), resolved over the whole element order; replaces the rule above
    const int *bar_orient_node = nullptr;
};

// Returns 0, -1 if an element has a non-positive Jacobian (or a cable a
// non-positive length), -2 for an unsupported cable quadrature order.
// tets are zero-based.  s = dt/4 (+ smoothing 4 alpha / dt).
// scheme 0: Crank-Nicolson (A = Cm M + s K, B = Cm M - s K); 1: backward
// Euler (A = C_L + dt/2 K, B = diag C_L); 2: explicit (A = -K, B zero).
// Cables (optional) are summed after the tets of the same entry.
int assemble_cn(int n, const double *xyz, int m, const int *tets, const double *fibers,
                const double D[3], double Cm, double dt, double smoothing_alpha, HostCSR &out,
                int scheme = 0, const HostCables *cables = nullptr);

// W[k * n + i] with ECG_k = sum_i W V_i (ComputeECG.h:30-189 with grad V
// constant on a P1 tet); the cables of a MIX3D mesh add their share (with
// the tissue D and cables->radius, which ComputeECG fixes at 0.0275 cm).
void ecg_weights(int n, const double *xyz, int m, const int *tets, const double *fibers,
                 const double D[3], int ne, const double *electrodes, std::vector<double> &W,
                 const HostCables *cables = nullptr);

// SELL-32 packing of a CSR pattern: slice_ptr (element offsets, multiples of
// 32), col, and the values of one or more value arrays.
struct Sell {
    int n = 0, nslices = 0;
    std::vector<int> slice_ptr, col;
    std::vector<std::vector<double>> vals;
};
void pack_sell(const HostCSR &a, const std::vector<const std::vector<double> *> &vals, Sell &out);

}  // namespace ep
