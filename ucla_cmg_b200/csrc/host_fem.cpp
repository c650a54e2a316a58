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

// element matrices of the cables, in element order (the .angle override
// can carry over from one cable to the next)
struct BarMat {
    int nq = 0;
    double K[2][2] = {{0, 0}, {0, 0}}, M[2][2] = {{0, 0}, {0, 0}};
    double CL[3][2] = {{0, 0}, {0, 0}, {0, 0}};   // per quadrature point, for the element-order sums
};

// LineQuadrature of order 2 q - 1 on [-1, 1] (LineQuadrature.cc), weights
// summing to 2; -1 for an order the reference does not have
int bar_quadrature(int quad_order, double *qx, double *qw) {
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

// unit direction and length of every cable in order, with the .angle
// overrides of MixedMesh3D::Compute (MixedMesh3D.cc:30-34, 78-87): per cable
// from bar_orient_node when resolved over the whole element order, else the
// cables-only rule (the override carried on when orient_sticky)
void bar_frames(const double *xyz, const HostCables &cb, std::vector<double> &ang_out, std::vector<double> &len_out) {
    ang_out.assign(3 * (size_t)cb.nb, 0.0);
    len_out.assign(cb.nb, 0.0);
    bool carried = false;
    double carry[4] = {0, 0, 0, 0};
    for (int e = 0; e < cb.nb; e++) {
        const int *v = cb.bars + 2 * (size_t)e;
        const bool listed = cb.orient_has && cb.orient_has[v[0]];
        if (listed) {
            carried = true;
            for (int k = 0; k < 4; k++) carry[k] = cb.orient[4 * (size_t)v[0] + k];
        }
        double ang[3], len;
        for (int k = 0; k < 3; k++) ang[k] = xyz[3 * (size_t)v[1] + k] - xyz[3 * (size_t)v[0] + k];
        len = std::sqrt(ang[0] * ang[0] + ang[1] * ang[1] + ang[2] * ang[2]);
        for (int k = 0; k < 3; k++) ang[k] /= len;
        if (cb.bar_orient_node) {
            const int o = cb.bar_orient_node[e];
            if (o >= 0) {
                for (int k = 0; k < 3; k++) ang[k] = cb.orient[4 * (size_t)o + k];
                len = cb.orient[4 * (size_t)o + 3];
            }
        } else if (listed || (carried && cb.orient_sticky)) {
            for (int k = 0; k < 3; k++) ang[k] = carry[k];
            len = carry[3];
        }
        for (int k = 0; k < 3; k++) ang_out[3 * (size_t)e + k] = ang[k];
        len_out[e] = len;
    }
}

int bar_mats(const double *xyz, const HostCables &cb, double Cm, std::vector<BarMat> &out) {
    double qx[3], qw[3];
    const int nq = bar_quadrature(cb.quad_order, qx, qw);
    if (nq < 0) return -2;
    out.assign(cb.nb, BarMat());
    std::vector<double> angs, lens;
    bar_frames(xyz, cb, angs, lens);
    int bad = 0;
    for (int e = 0; e < cb.nb; e++) {
        const double *ang = &angs[3 * (size_t)e];
        const double len = lens[e];
        if (!(len > 0.0)) bad = 1;
        const bool lv = cb.lv && cb.lv[e];
        const double *Dc = lv ? cb.DpLeft : cb.Dp;
        double De[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        if (!cb.fibers) {
            for (int p = 0; p < 3; p++) De[p][p] = Dc[0];
        } else {
            const double *fib = cb.fibers + 9 * (size_t)e;
            for (int p = 0; p < 3; p++)
                for (int m = 0; m < 3; m++)
                    for (int q = 0; q < 3; q++) De[m][q] += Dc[p] * fib[3 * p + m] * fib[3 * p + q];
        }
        const double fac = 2. / len;
        const double dshape[2] = {-0.5, 0.5};
        double dx[2][3];
        for (int a = 0; a < 2; a++)
            for (int k = 0; k < 3; k++) dx[a][k] = dshape[a] * ang[k] * fac;
        BarMat &bm = out[e];
        bm.nq = nq;
        for (int q = 0; q < nq; q++) {
            const double N[2] = {0.5 * (1. - qx[q]), 0.5 * (1. + qx[q])};
            const double w = qw[q] * M_PI * (cb.radius * cb.radius) * len;
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++) {
                    bm.M[a][b] += N[a] * N[b] * w;
                    for (int m = 0; m < 3; m++)
                        for (int r = 0; r < 3; r++) bm.K[a][b] += De[m][r] * dx[a][m] * dx[b][r] * w * Cm;
                }
            for (int a = 0; a < 2; a++) bm.CL[q][a] = N[a] * Cm * w;
        }
    }
    return bad;
}

void bar_incidence(int n, const HostCables *cb, std::vector<int> &ptr, std::vector<int> &elem) {
    ptr.assign((size_t)n + 1, 0);
    const int nb = cb ? cb->nb : 0;
    for (size_t k = 0; k < (size_t)nb * 2; k++) ptr[cb->bars[k] + 1]++;
    for (int i = 0; i < n; i++) ptr[i + 1] += ptr[i];
    elem.resize((size_t)nb * 2);
    std::vector<int> pos(ptr.begin(), ptr.end() - 1);
    for (int e = 0; e < nb; e++)
        for (int a = 0; a < 2; a++) elem[pos[cb->bars[2 * (size_t)e + a]]++] = e;
}

}  // namespace

int assemble_cn(int n, const double *xyz, int m, const int *tets, const double *fibers,
                const double D[3], double Cm, double dt, double smoothing_alpha, HostCSR &out, int scheme,
                const HostCables *cables) {
    std::vector<int> eptr, elem, bptr, belem;
    incidence(n, m, tets, eptr, elem);
    bar_incidence(n, cables, bptr, belem);
    std::vector<BarMat> bars;
    int bad_bar = 0;
    if (cables && cables->nb > 0) {
        bad_bar = bar_mats(xyz, *cables, Cm, bars);
        if (bad_bar == -2) return -2;
    }
    out.n = n;
    out.rowptr.assign((size_t)n + 1, 0);
    // pattern: union of the vertices of each node's elements
    std::vector<std::vector<int>> rows(n);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int i = 0; i < n; i++) {
        std::vector<int> &r = rows[i];
        for (int k = eptr[i]; k < eptr[i + 1]; k++)
            for (int a = 0; a < 4; a++) r.push_back(tets[4 * (size_t)elem[k] + a]);
        for (int k = bptr[i]; k < bptr[i + 1]; k++)
            for (int a = 0; a < 2; a++) r.push_back(cables->bars[2 * (size_t)belem[k] + a]);
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
            // the cables at this node, after its tets
            for (int k = bptr[i]; k < bptr[i + 1]; k++) {
                const int e = belem[k];
                const int *v = cables->bars + 2 * (size_t)e;
                const BarMat &bm = bars[e];
                const int a = v[0] == i ? 0 : 1;
                if (pass == 1) {
                    if (mass)
                        for (int b = 0; b < 2; b++) {
                            const int p = find(v[b]);
                            A[p] += bm.M[a][b] * Cm;
                            B[p] += bm.M[a][b] * Cm;
                        }
                    for (int q = 0; q < bm.nq; q++) cl += bm.CL[q][a];
                } else {
                    const double f = pass == 0 ? s : sm;
                    for (int b = 0; b < 2; b++) {
                        const int p = find(v[b]);
                        A[p] += bm.K[a][b] * f;
                        if (mass) B[p] += bm.K[a][b] * (-f);
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
    return (bad || bad_bar) ? -1 : 0;
}

void ecg_weights(int n, const double *xyz, int m, const int *tets, const double *fibers,
                 const double D[3], int ne, const double *el, std::vector<double> &W,
                 const HostCables *cables) {
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
    // the cables of a MIX3D mesh: ComputeECG integrates over them too
    // (ComputeECG.h:47-50, 107-110) with the tissue D along each cable's
    // fibre frame (computeDiffusionTensor, ComputeECG.h:92-136), shape
    // derivatives -+ ang / length and weights w_q pi r^2 length of
    // MixedMesh3D::Compute; the radius is the caller's (ComputeECG fixes
    // 0.0275 cm, ComputeECG.cc:75)
    if (cables && cables->nb > 0) {
        double qx[3], qw[3];
        const int nq = bar_quadrature(cables->quad_order, qx, qw);
        std::vector<double> angs, lens;
        bar_frames(xyz, *cables, angs, lens);
        for (int e = 0; e < cables->nb && nq > 0; e++) {
            const int *v = cables->bars + 2 * (size_t)e;
            double De[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            if (!cables->fibers) {
                for (int p = 0; p < 3; p++) De[p][p] = D[0];
            } else {
                const double *fib = cables->fibers + 9 * (size_t)e;
                for (int p = 0; p < 3; p++)
                    for (int a = 0; a < 3; a++)
                        for (int b = 0; b < 3; b++) De[a][b] += D[p] * fib[3 * p + a] * fib[3 * p + b];
            }
            const double *ang = &angs[3 * (size_t)e];
            const double len = lens[e];
            const double dx[2][3] = {{-ang[0] / len, -ang[1] / len, -ang[2] / len},
                                     {ang[0] / len, ang[1] / len, ang[2] / len}};
            for (int kk = 0; kk < ne; kk++) {
                const double *x = el + 3 * kk;
                double G[3] = {0, 0, 0};
                for (int q = 0; q < nq; q++) {
                    const double N0 = 0.5 * (1. - qx[q]), N1 = 0.5 * (1. + qx[q]);
                    double pos[3], d2 = 0.0;
                    for (int d = 0; d < 3; d++) {
                        pos[d] = N0 * xyz[3 * (size_t)v[0] + d] + N1 * xyz[3 * (size_t)v[1] + d];
                        d2 += (pos[d] - x[d]) * (pos[d] - x[d]);
                    }
                    const double dist = std::sqrt(d2);
                    if (dist < 1e-6) continue;       // ComputeECG.h:77-79
                    const double d3 = dist * dist * dist;
                    const double w = qw[q] * M_PI * (cables->radius * cables->radius) * len;
                    for (int d = 0; d < 3; d++) G[d] += (-(pos[d] - x[d]) / d3) * w;
                }
                double DG[3];
                for (int r = 0; r < 3; r++) DG[r] = De[r][0] * G[0] + De[r][1] * G[1] + De[r][2] * G[2];
                for (int b = 0; b < 2; b++)
                    W[(size_t)kk * n + v[b]] += dx[b][0] * DG[0] + dx[b][1] * DG[1] + dx[b][2] * DG[2];
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
