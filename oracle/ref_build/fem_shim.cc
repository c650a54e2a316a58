// fem_shim.cc -- C entry points around the reference's UNMODIFIED finite-
// element sources, compiled from their sources in place against the
// stand-in headers of stub_fem/.  TEST INFRASTRUCTURE ONLY: it pins the
// oracle's restatement of the diffusion operators and of the pseudo-ECG to
// the reference's own arithmetic.
//
// Compiled from the reference (voomEP/src/...):
//   Mesh/Mesh.cc            Mesh::New (the .node/.ele/.fibers/.metis/.purk/
//                           .cell/.angle readers, Mesh.cc:142-483), the Mesh
//                           constructor and getIndices;
//   Mesh/TetMesh.cc         TetMesh::Compute (N, dN/dx, w*J per quadrature
//                           point, TetMesh.cc:9-71), with Shape/ShapeTet4CP.cc,
//                           Quadrature/TetQuadrature.cc, VoomMath/VoomMath.cc;
//   Mesh/MixedMesh3D.cc     the mixed tet + 2-node cable mesh (MixedMesh3D.cc:
//                           10-158) with Shape/ShapeBar.cc and
//                           Quadrature/LineQuadrature.cc;
//   Body/CardiacBody.cc     CardiacBody::New, Compute (element K and M,
//                           CardiacBody.cc:78-187), computeLumpedCapacitance
//                           (:32-67), getDiffusionMatrix / getCapacitanceMatrix
//                           (:348-391) -- the matrices come back as the
//                           (row, col, value) triplets the reference inserts;
//   Applications/CardiacEP/ComputeECG.h
//                           computeGradOneByR, computeDiffusionTensor,
//                           computeVoltageAtQuadPoints, computeECG
//                           (ComputeECG.h:30-189), chained as ComputeECG.cc's
//                           main does per output frame (ComputeECG.cc:96-156);
// plus the other mesh types, shapes and quadratures Mesh.cc names, and the
// cell models CardiacBody::New constructs.
#include "Mesh.h"
#include "TetMesh.h"
#include "MixedMesh3D.h"
#include "CardiacBody.h"
#include "ComputeECG.h"

#include <cstring>
#include <string>
#include <vector>

using namespace voom;

namespace {

struct FemMesh {
    Mesh *mesh = nullptr;
};

struct FemBody {
    CardiacBody *body = nullptr;
    FemMesh *m = nullptr;
};

long copy_triplets(const Epetra_CrsMatrix &A, int *rows, int *cols, double *vals) {
    const long n = (long)A.val.size();
    if (rows) std::memcpy(rows, A.row.data(), sizeof(int) * n);
    if (cols) std::memcpy(cols, A.col.data(), sizeof(int) * n);
    if (vals) std::memcpy(vals, A.val.data(), sizeof(double) * n);
    return n;
}

}  // namespace

extern "C" {

// Mesh::New(comm, base, quad_order, TETMESH or MIXEDMESH3D) with one rank
// and setRadius(radius), as EPSimulator does (EPSimulator.cc:373-374).  The
// files <base>.node/.ele[/.fibers] and <base>.metis.npart.1 / .metis.epart.1
// must exist (the reference reads the partition files even for one rank).
// The quadrature data come from fem_mesh_compute (ComputeECG.cc's order) or
// from the CardiacBody constructor (fem_body_new; CardiacBody.cc:17) -- use
// one or the other on a mesh, since Compute() appends to the point list.
void *fem_mesh_new(const char *base, int quad_order, int mixed, double radius) {
    Epetra_MpiComm comm;
    FemMesh *fm = new FemMesh;
    fm->mesh = Mesh::New(&comm, std::string(base), quad_order, mixed ? MIXEDMESH3D : TETMESH);
    fm->mesh->setRadius(radius);
    return fm;
}

void fem_mesh_compute(void *p) { ((FemMesh *)p)->mesh->Compute(); }

void fem_mesh_free(void *p) {
    FemMesh *fm = (FemMesh *)p;
    if (!fm) return;
    delete fm->mesh;
    delete fm;
}

int fem_mesh_num_points(void *p) { return ((FemMesh *)p)->mesh->QuadSize(); }
int fem_mesh_num_elements(void *p) { return ((FemMesh *)p)->mesh->getIDTableSize(); }
int fem_mesh_num_local_nodes(void *p) { return ((FemMesh *)p)->mesh->getNumLocalNodes(); }

// quadrature points of the elements, in element order: per point the
// element's node count k, then k shape values, k x 3 derivatives dN/dx and
// the weight w*J, packed into N[4], dN[12], w[1] per point (unused slots 0)
int fem_mesh_points(void *p, int *k_out, double *N, double *dN, double *w) {
    Mesh *m = ((FemMesh *)p)->mesh;
    const Mesh::QuadPoints &q = m->getPoints();
    for (size_t i = 0; i < q.size(); i++) {
        const int k = (int)q[i].shapeFunctions.size();
        k_out[i] = k;
        for (int a = 0; a < 4; a++) {
            N[4 * i + a] = a < k ? q[i].shapeFunctions[a] : 0.0;
            for (int d = 0; d < 3; d++)
                dN[12 * i + 3 * a + d] =
                    (a < k && d < (int)q[i].shapeDerivatives[a].size()) ? q[i].shapeDerivatives[a][d] : 0.0;
        }
        w[i] = q[i].weight;
    }
    return (int)q.size();
}

// CardiacBody::New(mesh, model) (every .purk node a Purkinje cell), the
// diffusion, Purkinje diffusion and capacitance set as EPSimulator does,
// then CardiacBody::Compute().
void *fem_body_new(void *mesh, int model, const double *D, double Cm, const double *Dp, const double *DpLeft) {
    FemMesh *fm = (FemMesh *)mesh;
    FemBody *fb = new FemBody;
    fb->m = fm;
    fb->body = CardiacBody::New(fm->mesh, (CellModelType)model);
    Real d[3] = {D[0], D[1], D[2]};
    fb->body->setDiffusion(d);
    if (Dp) {
        Real dp[3] = {Dp[0], Dp[1], Dp[2]};
        fb->body->setPurkinjeDiffusion(dp);
    }
    if (DpLeft) {
        Real dl[3] = {DpLeft[0], DpLeft[1], DpLeft[2]};
        fb->body->setPurkinjeDiffusionInLV(dl);
    }
    fb->body->setNodalCapacitance(Cm);
    fb->body->Compute();
    return fb;
}

void fem_body_free(void *p) {
    FemBody *fb = (FemBody *)p;
    if (!fb) return;
    delete fb->body;
    delete fb;
}

// CardiacBody::getDiffusionMatrix(M, scale): the triplets it inserts (call
// with NULL outputs for the count)
long fem_body_diffusion(void *p, double scale, int *rows, int *cols, double *vals) {
    Epetra_FECrsMatrix A;
    ((FemBody *)p)->body->getDiffusionMatrix(&A, scale);
    return copy_triplets(A, rows, cols, vals);
}

// CardiacBody::getCapacitanceMatrix(M, isCap)
long fem_body_capacitance(void *p, int is_cap, int *rows, int *cols, double *vals) {
    Epetra_FECrsMatrix A;
    ((FemBody *)p)->body->getCapacitanceMatrix(&A, is_cap != 0);
    return copy_triplets(A, rows, cols, vals);
}

// CardiacBody::computeLumpedCapacitance (one rank: no ghost nodes), local
// node order = global order
int fem_body_lumped(void *p, double *out) {
    FemBody *fb = (FemBody *)p;
    const int n = fb->m->mesh->getNumLocalNodes();
    Epetra_Vector cap(n), ghost(fb->m->mesh->getNumGhostNodes());
    fb->body->computeLumpedCapacitance(&cap, &ghost);
    for (int i = 0; i < n; i++) out[i] = cap[i];
    return n;
}

// ComputeECG.cc's per-frame chain on the mesh (ComputeECG.h:30-189): the
// diffusion tensor per quadrature point from D (the reference hard-codes
// D = {1e-3, 5e-4, 2.5e-4} in ComputeECG.cc:88; here it is an argument),
// grad(1/r) at each point for each electrode, grad V at each point from the
// nodal voltage (global node order), and the quadrature sum per electrode.
int fem_ecg(void *mesh, const double *D, int n_points, const double *xyz, const double *V, double *out) {
    Mesh *m = ((FemMesh *)mesh)->mesh;
    std::vector<std::vector<Real> > points(n_points, std::vector<Real>(3));
    for (int k = 0; k < n_points; k++)
        for (int d = 0; d < 3; d++) points[k][d] = xyz[3 * k + d];
    Real Diff[3] = {D[0], D[1], D[2]};
    Real Dp[3] = {D[0], D[1], D[2]};
    std::vector<Diffusion> diff;
    computeDiffusionTensor(m, Diff, Dp, diff);
    std::vector<GradVals> grad;
    computeGradOneByR(m, points, grad);
    std::vector<Real> volt(V, V + m->numberOfNodes());
    std::vector<GradVoltage> gv;
    computeVoltageAtQuadPoints(m, volt.data(), gv);
    Real *ecg = computeECG(diff, gv, grad, m->getDimension());
    for (int k = 0; k < n_points; k++) out[k] = ecg[k];
    delete[] ecg;
    return 0;
}

}  // extern "C"
