// host_fem.cpp -- P1-tet assembly on the host in FP64, node-parallel and
// deterministic.
//
// Geometry of one tet follows voomEP/src/Mesh/TetMesh.cc:9-71 (Jacobian
// dx/dxi from the constant shape gradients of ShapeTet4CP.cc:4-16, 3x3
// inverse and determinant of VoomMath.cc:17-52, weight w*J with the 4-point
// rule of TetQuadrature.cc:16-30 -- its truncated alpha/beta included).
// Element matrices follow CardiacBody::Compute (Body/CardiacBody.cc:78-187):
// K_e = sum_q C_m dN^T D_e dN w J with D_e = sum_p D[p] f_p f_p^T,
// M_e = sum_q N N^T w J; C_L = row sums of C_m M (CardiacBody.cc:32-67).
// The CN operators follow EP_CrankNicholson::Initialize (Solvers/
// EP_CrankNicholson.cc:15-44): per matrix entry, all diffusion terms (scaled
// by +-dt/4) are summed first in element order, then the mass terms.
//
// Each row is owned by one thread, which walks its node's elements in
// increasing element order; that reproduces the element-order summation of
// a sequential assembly without atomics.
#include "host_fem.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace ep {

namespace {

constexpr double QA = 0.58541020, QB = 0.13819660;   // truncated as in the reference
const double QN[4][4] = {{1.0 - QA - QB - QB, QA, QB, QB},
                         {1.0 - QB - QA - QB, QB, QA, QB},
                         {1.0 - QB - QB - QA, QB, QB, QA},
                         {1.0 - QB - QB - QB, QB, QB, QB}};

struct Geo {
    double dN[4][3];
    double wJ;
    double De[3][3];
};

// returns the Jacobian determinant
double tet_geo(const double *xyz, const int *v, const double *fib, const double D[3], Geo &g) {
    static const double DN[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    double a[3][3], b[3][3];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) {
            double s = 0.0;
            for (int k = 0; k < 4; k++) s += DN[k][c] * xyz[3 * (size_t)v[k] + r];
            a[r][c] = s;
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
        for (int c = 0; c < 3; c++) {
            double s = 0.0;
            for (int al = 0; al < 3; al++) s += DN[k][al] * b[al][c];
            g.dN[k][c] = s;
        }
    g.wJ = (1.0 / 4.0 / 6.0) * det;
    for (int m = 0; m < 3; m++)
        for (int n = 0; n < 3; n++) g.De[m][n] = 0.0;
    if (!fib) {
        for (int p = 0; p < 3; p++) g.De[p][p] = D[0];
    } else {
        for (int p = 0; p < 3; p++) {
            const double *f = fib + 3 * p;
            for (int m = 0; m < 3; m++)
                for (int n = 0; n < 3; n++) g.De[m][n] += D[p] * f[m] * f[n];
        }
    }
    return det;
}

// K_e row a (the 4-point loop of CardiacBody::Compute, identical terms per point)
void k_row(const Geo &g, int a, double Cm, double out[4]) {
    for (int b = 0; b < 4; b++) out[b] = 0.0;
    for (int q = 0; q < 4; q++)
        for (int b = 0; b < 4; b++)
            for (int m = 0; m < 3; m++)
                for (int n = 0; n < 3; n++) out[b] += g.De[m][n] * g.dN[a][m] * g.dN[b][n] * g.wJ * Cm;
}

void m_row(const Geo &g, int a, double out[4]) {
    for (int b = 0; b < 4; b++) out[b] = 0.0;
    for (int q = 0; q < 4; q++)
        for (int b = 0; b < 4; b++) out[b] += QN[q][a] * QN[q][b] * g.wJ;
}

void incidence(int n, int m, const int *tets, std::vector<int> &ptr, std::vector<int> &elem) {
    ptr.assign((size_t)n + 1, 0);
    for (size_t k = 0; k < (size_t)m * 4; k++) ptr[tets[k] + 1]++;
    for (int i = 0; i < n; i++) ptr[i + 1] += ptr[i];
    elem.resize((size_t)m * 4);
    std::vector<int> pos(ptr.begin(), ptr.end() - 1);
    for (int e = 0; e < m; e++)
        for (int a = 0; a < 4; a++) elem[pos[tets[4 * (size_t)e + a]]++] = e;
}

}  // namespace

int assemble_cn(int n, const double *xyz, int m, const int *tets, const double *fibers,
                const double D[3], double Cm, double dt, double smoothing_alpha, HostCSR &out, int scheme) {
    std::vector<int> eptr, elem;
    incidence(n, m, tets, eptr, elem);
    out.n = n;
    out.rowptr.assign((size_t)n + 1, 0);
    // pattern: union of the vertices of each node's elements
    std::vector<std::vector<int>> rows(n);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int i = 0; i < n; i++) {
        std::vector<int> &r = rows[i];
        for (int k = eptr[i]; k < eptr[i + 1]; k++)
            for (int a = 0; a < 4; a++) r.push_back(tets[4 * (size_t)elem[k] + a]);
        std::sort(r.begin(), r.end());
        r.erase(std::unique(r.begin(), r.end()), r.end());
    }
    for (int i = 0; i < n; i++) out.rowptr[i + 1] = out.rowptr[i] + (int)rows[i].size();
    const size_t nnz = out.rowptr[n];
    out.col.resize(nnz);
    out.A.assign(nnz, 0.0);
    out.B.assign(nnz, 0.0);
    out.CL.assign(n, 0.0);
    // CN: A = Cm M + s K, B = Cm M - s K with s = dt/4 (EP_CrankNicholson.cc:5-76);
    // BE: A = C_L + (dt/2) K, B = C_L (EP_BackwardEuler.cc:5-40);
    // explicit: A = -K (EP_ExplicitSolver.cc:4-12), B unused
    const double s = scheme == 1 ? dt / 2.0 : scheme == 2 ? -1.0 : dt / 4.0;
    const bool mass = scheme == 0;
    const double sm = (scheme == 0 && smoothing_alpha > 0.0) ? smoothing_alpha * 4.0 / dt : 0.0;
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(| : bad)
    for (int i = 0; i < n; i++) {
        const int beg = out.rowptr[i];
        const int len = out.rowptr[i + 1] - beg;
        std::memcpy(&out.col[beg], rows[i].data(), sizeof(int) * len);
        double *A = &out.A[beg], *B = &out.B[beg];
        auto find = [&](int c) {
            int lo = 0, hi = len - 1;
            while (lo < hi) { const int mid = (lo + hi) >> 1; if (rows[i][mid] < c) lo = mid + 1; else hi = mid; }
            return lo;
        };
        double cl = 0.0;
        // pass 1: diffusion terms (+-s), pass 2: mass terms, pass 3: smoothing
        for (int pass = 0; pass < 3; pass++) {
            if (pass == 2 && sm == 0.0) break;
            for (int k = eptr[i]; k < eptr[i + 1]; k++) {
                const int e = elem[k];
                const int *v = tets + 4 * (size_t)e;
                Geo g;
                const double det = tet_geo(xyz, v, fibers ? fibers + 9 * (size_t)e : nullptr, D, g);
                if (!(det > 0.0)) bad = 1;
                int a = 0;
                while (v[a] != i) a++;
                double row[4];
                if (pass == 1) {
                    if (mass) {
                        m_row(g, a, row);
                        for (int b = 0; b < 4; b++) {
                            const int p = find(v[b]);
                            A[p] += row[b] * Cm;
                            B[p] += row[b] * Cm;
                        }
                    }
                    for (int q = 0; q < 4; q++) cl += QN[q][a] * Cm * g.wJ;
                } else {
                    k_row(g, a, Cm, row);
                    const double f = pass == 0 ? s : sm;
                    for (int b = 0; b < 4; b++) {
                        const int p = find(v[b]);
                        A[p] += row[b] * f;
                        if (mass) B[p] += row[b] * (-f);
                    }
                }
            }
        }
        out.CL[i] = cl;
        if (scheme == 1) {                       // lumped capacitance on the diagonal
            const int p = find(i);
            A[p] += cl;
            B[p] = cl;
        }
        std::vector<int>().swap(rows[i]);
    }
    return bad ? -1 : 0;
}

void ecg_weights(int n, const double *xyz, int m, const int *tets, const double *fibers,
                 const double D[3], int ne, const double *el, std::vector<double> &W) {
    std::vector<int> eptr, elem;
    incidence(n, m, tets, eptr, elem);
    W.assign((size_t)ne * n, 0.0);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int i = 0; i < n; i++) {
        for (int k = eptr[i]; k < eptr[i + 1]; k++) {
            const int e = elem[k];
            const int *v = tets + 4 * (size_t)e;
            Geo g;
            tet_geo(xyz, v, fibers ? fibers + 9 * (size_t)e : nullptr, D, g);
            int a = 0;
            while (v[a] != i) a++;
            double pos[4][3];
            for (int q = 0; q < 4; q++)
                for (int d = 0; d < 3; d++) {
                    double sacc = 0.0;
                    for (int b = 0; b < 4; b++) sacc += QN[q][b] * xyz[3 * (size_t)v[b] + d];
                    pos[q][d] = sacc;
                }
            for (int kk = 0; kk < ne; kk++) {
                const double *x = el + 3 * kk;
                double G[3] = {0, 0, 0};
                for (int q = 0; q < 4; q++) {
                    double d2 = 0.0;
                    for (int d = 0; d < 3; d++) d2 += (pos[q][d] - x[d]) * (pos[q][d] - x[d]);
                    const double dist = std::sqrt(d2);
                    if (dist < 1e-6) continue;       // ComputeECG.h:77-79
                    const double d3 = dist * dist * dist;
                    for (int d = 0; d < 3; d++) G[d] += (-(pos[q][d] - x[d]) / d3) * g.wJ;
                }
                double acc = 0.0;
                for (int r = 0; r < 3; r++)
                    acc += g.dN[a][r] * (g.De[r][0] * G[0] + g.De[r][1] * G[1] + g.De[r][2] * G[2]);
                W[(size_t)kk * n + i] += acc;
            }
        }
    }
}

void pack_sell(const HostCSR &a, const std::vector<const std::vector<double> *> &vals, Sell &out) {
    const int n = a.n, S = 32;
    out.n = n;
    out.nslices = (n + S - 1) / S;
    out.slice_ptr.assign((size_t)out.nslices + 1, 0);
    for (int s = 0; s < out.nslices; s++) {
        int w = 0;
        for (int r = s * S; r < std::min(n, (s + 1) * S); r++) w = std::max(w, a.rowptr[r + 1] - a.rowptr[r]);
        out.slice_ptr[s + 1] = out.slice_ptr[s] + w * S;
    }
    const size_t tot = out.slice_ptr[out.nslices];
    out.col.assign(tot, 0);
    out.vals.assign(vals.size(), std::vector<double>(tot, 0.0));
#pragma omp parallel for schedule(static)
    for (int s = 0; s < out.nslices; s++) {
        const int beg = out.slice_ptr[s], w = (out.slice_ptr[s + 1] - beg) / S;
        for (int l = 0; l < S; l++) {
            const int r = s * S + l;
            const int rr = r < n ? r : n - 1;
            const int len = r < n ? a.rowptr[r + 1] - a.rowptr[r] : 0;
            for (int k = 0; k < w; k++) {
                const size_t idx = beg + (size_t)k * S + l;
                if (k < len) {
                    out.col[idx] = a.col[a.rowptr[r] + k];
                    for (size_t v = 0; v < vals.size(); v++) out.vals[v][idx] = (*vals[v])[a.rowptr[r] + k];
                } else {
                    out.col[idx] = rr;     // padding: a valid column, value 0
                }
            }
        }
    }
}

}  // namespace ep
