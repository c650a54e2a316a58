// ref_shim.cc -- C entry points around the reference's UNMODIFIED cell-model
// classes (voomEP/src/IonicModel/{Tusscher,Mahajan,Mahajan_fail,LR,Purkinje}.cc),
// compiled from their sources in place.  TEST INFRASTRUCTURE ONLY: it backs
// the oracle checks and the reference arm of the CPU baseline.
//
// Per node it keeps one heap object behind the IonicModel virtual ABI, the
// way CardiacBody::New builds them (voomEP/src/Body/CardiacBody.cc:975-1101),
// and calls Compute_Ion node by node like CardiacBody::getIonicCurrent
// (CardiacBody.cc:405-435).
#include "Tusscher.h"
#include "Mahajan.h"
#include "Mahajan_fail.h"
#include "LR.h"
#include "Purkinje.h"
#include "SetUpIonicConstants.h"
#include "../ep_oracle.h"
#include <cstring>
#include <cstdlib>
#include <cmath>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace voom;

// LAPACK dgesv_ (Tusscher.cc:181) comes from dgesv_shim.cc.

struct RefCells {
    int model, n, nstate;
    std::vector<IonicModel *> cells;
    std::vector<Real *> consts;
    LuoRudyGateTable *gate = nullptr;
    Real userXi = 0.0;
    bool userXiSet = false;
};

extern "C" {

// model: 0 LUORUDY, 1 LUORUDYWITHGATE, 2 TUSSCHER, 3 MAHAJAN, 4 MAHAJAN_FAIL,
// 5 the Purkinje cell CardiacBody::New puts on .purk nodes
void *ref_cells_create(int model, int n, const unsigned char *type)
{
    RefCells *r = new RefCells();
    r->model = model; r->n = n;
    switch (model) {
    case 0: case 1:
        r->nstate = 8;
        if (model == 1) r->gate = new LuoRudyGateTable();
        for (int i = 0; i < n; i++) r->cells.push_back(new LuoRudy(model == 1, r->gate));
        break;
    case 2: {
        r->nstate = 19;
        Real *c; SetUpTusscherParameters(&c); r->consts.push_back(c);
        for (int i = 0; i < n; i++) r->cells.push_back(new Tusscher(c));
        break; }
    case 3: case 4: {
        r->nstate = 26;
        for (int t = 0; t < 9; t++) {
            Real *c;
            if (model == 3) SetUpMahajanParameters(&c, t); else SetUpMahajan_failParameters(&c, t);
            r->consts.push_back(c);
        }
        for (int i = 0; i < n; i++) {
            int t = type ? type[i] : 0;
            if (model == 3) r->cells.push_back(new Mahajan(r->consts[t], t));
            else r->cells.push_back(new Mahajan_fail(r->consts[t], t));
        }
        break; }
    case 5: {
        r->nstate = 22;
        Real *c; SetUpPurkinjeParameters(&c); r->consts.push_back(c);
        for (int i = 0; i < n; i++) r->cells.push_back(new Purkinje(c));
        break; }
    default:
        delete r; return nullptr;
    }
    return r;
}

void ref_cells_destroy(void *h)
{
    RefCells *r = (RefCells *)h;
    if (!r) return;
    // IonicModel has a non-virtual destructor: delete through the real type
    for (IonicModel *c : r->cells) {
        switch (r->model) {
        case 0: case 1: delete (LuoRudy *)c; break;
        case 2: delete (Tusscher *)c; break;
        case 3: delete (Mahajan *)c; break;
        case 5: delete (Purkinje *)c; break;
        default: delete (Mahajan_fail *)c; break;
        }
    }
    for (Real *c : r->consts) delete[] c;
    if (r->gate) {
        for (int i = 0; i < 290001; i++) delete[] r->gate->_gateTable[i];
        delete[] r->gate->_gateTable;
        delete r->gate;
    }
    delete r;
}

int ref_cells_nstate(void *h) { return ((RefCells *)h)->nstate; }

void ref_cells_set_user_xi(void *h, double Xi)
{
    RefCells *r = (RefCells *)h; r->userXi = Xi; r->userXiSet = true;
}

// ic[i] = Compute_Ion(...) for every node (CardiacBody::getIonicCurrent)
void ref_cells_compute_ion(void *h, double Cm, double dt, const double *V,
                           const double *istim, double *dvdt)
{
    RefCells *r = (RefCells *)h;
    const int n = r->n;
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; i++)
        dvdt[i] = r->cells[i]->Compute_Ion(r->userXi, r->userXiSet, Cm, dt, V[i], istim[i]);
}

// one node's Compute_Ion, for the per-node strides of the non-CN schemes
double ref_cells_ionic_node_cb(void *h, int i, double Cm, double dt, double V, double istim)
{
    RefCells *r = (RefCells *)h;
    return r->cells[i]->Compute_Ion(r->userXi, r->userXiSet, Cm, dt, V, istim);
}

// adapter for the oracle's split-step driver
void ref_cells_ionic_cb(void *h, double Cm, double dt, const double *V,
                        const double *istim, double *dvdt)
{
    ref_cells_compute_ion(h, Cm, dt, V, istim, dvdt);
}

void ref_cells_get_states(void *h, double *out)
{
    RefCells *r = (RefCells *)h;
    for (int i = 0; i < r->n; i++) {
        int nd = 0;
        const std::vector<Real> &s = r->cells[i]->getInternalParameters(nd);
        for (int k = 0; k < nd; k++) out[(size_t)i * r->nstate + k] = s[k];
    }
}

void ref_cells_set_states(void *h, const double *in)
{
    RefCells *r = (RefCells *)h;
    std::vector<Real> s(r->nstate);
    for (int i = 0; i < r->n; i++) {
        for (int k = 0; k < r->nstate; k++) s[k] = in[(size_t)i * r->nstate + k];
        r->cells[i]->setInternalParameters(s);
    }
}

// IonicModel::getVoltage() per node (0 for TT and LR: hazard H1)
void ref_cells_get_voltage(void *h, double *out)
{
    RefCells *r = (RefCells *)h;
    for (int i = 0; i < r->n; i++) out[i] = r->cells[i]->getVoltage();
}

// the split time step with the reference cells in the ionic phase
void *ref_sim_create(void *cells, epo_csr *csr, double dt, double ionic_dt, double Cm,
                     double cg_tol, int cg_maxit, int jacobi_steps)
{
    epo_sim *s = (epo_sim *)calloc(1, sizeof(epo_sim));
    epo_sim_init(s, csr, dt, ionic_dt, Cm, cg_tol, cg_maxit, jacobi_steps,
                 ref_cells_ionic_cb, cells);
    return s;
}

}  // extern "C"
