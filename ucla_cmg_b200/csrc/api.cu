// api.cu -- the C ABI (include/ep_gpu.h): handle life cycle, the split
// time-step driver, I/O in the reference formats.
#include <cstdarg>
#include <cstring>
#include <cmath>
#include <vector>
#include <string>
#include <memory>
#include <algorithm>

#include "kernels.cuh"
#include "host_fem.h"
#include "model_defaults.h"
#include "surrogate.cuh"

namespace ep {

static thread_local char g_err[512] = "";

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}
const char *last_error() { return g_err; }

// owning device buffer
struct DBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() { if (p) cudaFree(p); }
    int alloc(size_t b) {
        if (p) { cudaFree(p); p = nullptr; bytes = 0; }
        if (b == 0) return EP_OK;
        if (cudaMalloc(&p, b) != cudaSuccess) {
            cudaGetLastError();
            set_error("cudaMalloc(%zu) failed", b);
            return EP_ERR_NOMEM;
        }
        bytes = b;
        return EP_OK;
    }
    template <typename T> T *as() const { return (T *)p; }
};

}  // namespace ep

using namespace ep;

struct ep_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t io_ev[16] = {};          // chunked host <-> device copies (created on first use)
    // learned step: the fallback list runs on a second, higher-priority
    // stream beside the physics of the nodes the network took
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int n = 0, pitch = 0, model = 0, precision = 0, nstate = 0, ns = 0, ntypes = 1;
    size_t rsize = 8;                    // bytes per real
    double dt = 0.1, ionic_dt = 0.1, Cm = 1.0, Xi = 0.0;
    int nsub = 1;
    double sub_dt[kMaxSub];
    double cg_tol = 1e-7;
    int scheme = 0;                      // EP_SCHEME_*
    std::vector<double> ex_h;            // explicit scheme: diffusion sub-steps of one half
    DBuf cl;                             // explicit scheme: lumped capacitance C_L
    int cg_maxit = 1000;
    int cg_grid = 0, cg_block = 256;
    int ecg_every = 0;
    double act_thr = -40.0;
    TTOpts tt{};
    int mh_abs = 0;
    long long step = 0;
    int nslices = 0;
    // device memory
    DBuf V, S, Aval, Bval, dinv, r, q, p0, zv, consts, gks, lr_table, type, slice_ptr, col;
    DBuf r1, w0, w1, s0, s1;             // single-reduction CG only (allocated on first use)
    DBuf pd0, pd1, pvin;                 // CG predictor: x - V of the first / second half step, scratch
    DBuf pq0, pq1;                       // linear CG predictor: each half step's next start, 2 delta - delta_prev
    DBuf partial, bar, status, cg_stats, cg_last, d_step, track;
    DBuf stim_head, stim_next, stim_on, stim_off, stim_amp;
    int nstim = 0;
    DBuf W, ecg_buf, ecg_partial, ecg_counter;
    int ne = 0, ecg_cap = 0, ecg_count = 0, ecg_grid = 0;
    std::vector<double> ecg_t;
    std::vector<double> model_V0;        // IonicModel::getVoltage() per node
    // mesh kept for the ECG weights
    std::vector<double> xyz, fibers;
    std::vector<int> tets;
    double D[3] = {0, 0, 0};
    // per-kernel timing
    int profile = 0;
    std::vector<cudaEvent_t> pev;
    std::vector<int> pkind;              // kernel class started at each event
    long long launches = 0;
    // learned ionic step (EP_SURROGATE)
    DBuf sg_wimg, sg_aux, sg_list, sg_count, sg_err, sg_pred, sg_take;
    int has_surrogate = 0, sg_vupdate = 0;
    // independent instances sharing the launches (ep_batch_create)
    int ninst = 1;
    std::vector<int> inst_row;           // ninst + 1 node offsets
    std::vector<int> inst_blk;           // ninst + 1 CTA offsets of the CG groups
    DBuf d_inst_row, d_inst_blk;
    // launch shape (ep_set_launch_config / ep_autotune)
    int sg_variant = 0;                  // learned step: 0 two CTAs/SM, 1 four pipelines in one CTA/SM
    int cg_per_sm = 0, cg_batch = 4, cg_variant = 0, cg_predict = 0, cg_prefetch = 0, ionic_block = 128,
        ionic_min = 0, graph_steps = 0;
    cudaGraphExec_t gexec = nullptr;
    int g_steps = 0;                     // steps in the instantiated graph
    long long g_launches = 0;            // kernel launches per graph replay
    DBuf ecg_slot;                       // next ECG sample slot (device counter)
    void *pin = nullptr;                 // pinned host staging for state transfers
    size_t pin_bytes = 0;
    // bounded in-kernel waits (ep_set_wait_limits; 0 = the built-in limits)
    // and the test hook that makes the CG barrier wait for arrivals that
    // never come (ep_test_hold_barrier)
    unsigned int wait_grid = 0, wait_mbar = 0, bar_extra = 0;
    // mixed tissues (ep_create_mixed): the Purkinje cell on the .purk nodes
    // (a second SoA population indexed by node id, 21 states + the shared
    // V), the tissue model everywhere else
    int mixed = 0, n_pk = 0, nstate_api = 0;   // nstate_api: row width of ep_get/set_states
    double pk_Xi = 0.0;
    DBuf Spk, pk_consts, pk_list, pk_count, is_purk_d;
    std::vector<uint8_t> is_purk;
    // the cables, kept for the pseudo-ECG weights (zero-based, per-cable
    // .angle overrides resolved)
    std::vector<int> cab_bars, cab_bon;
    std::vector<uint8_t> cab_ohas;
    std::vector<double> cab_orient, cab_fib;
    int cab_quad = 2, cab_sticky = 1;
};

// the radius ComputeECG gives cables (ComputeECG.cc:75), so an in-run ECG
// of a mixed tissue is the one the reference's post-processor computes
constexpr double kEcgCableRadius = 0.0275;

namespace {

template <typename R>
int upload(DBuf &b, const std::vector<double> &h, size_t count = 0) {
    const size_t n = count ? count : h.size();
    int rc = b.alloc(n * sizeof(R));
    if (rc) return rc;
    std::vector<R> tmp(n, R(0));
    for (size_t i = 0; i < std::min(n, h.size()); i++) tmp[i] = (R)h[i];
    EP_CUDA(cudaMemcpy(b.p, tmp.data(), n * sizeof(R), cudaMemcpyHostToDevice));
    return EP_OK;
}

template <typename T>
int upload_raw(DBuf &b, const T *h, size_t n) {
    int rc = b.alloc(n * sizeof(T));
    if (rc) return rc;
    if (n) EP_CUDA(cudaMemcpy(b.p, h, n * sizeof(T), cudaMemcpyHostToDevice));
    return EP_OK;
}

template <typename R>
int download(const DBuf &b, std::vector<double> &h, size_t n, cudaStream_t s) {
    std::vector<R> tmp(n);
    EP_CUDA(cudaMemcpyAsync(tmp.data(), b.p, n * sizeof(R), cudaMemcpyDeviceToHost, s));
    EP_CUDA(cudaStreamSynchronize(s));
    h.resize(n);
    for (size_t i = 0; i < n; i++) h[i] = (double)tmp[i];
    return EP_OK;
}

bool is_mh(int m) { return m == EP_MAHAJAN || m == EP_MAHAJAN_FAIL; }
bool is_lr(int m) { return m == EP_LUORUDY || m == EP_LUORUDYWITHGATE; }

// sub-step sequence of one ionic phase (EP_CrankNicholson.cc:114-143),
// computed with the reference's own double arithmetic
int substeps(double dt, double idt, double *out) {
    double total = 0.0, h = (idt < dt) ? idt : dt;
    int k = 0;
    while (total < dt) {
        if (k >= kMaxSub) return -1;
        out[k++] = h;
        total += h;
        h = (total + h < dt) ? h : dt - total;
    }
    return k;
}

template <typename R>
void fill_ionic_args(ep_handle *h, IonicArgs<R> &a) {
    std::memset(&a, 0, sizeof a);
    a.n = h->n; a.pitch = h->pitch;
    a.V = h->V.as<R>(); a.S = h->S.as<R>();
    a.type = h->type.as<uint8_t>();
    a.gks = h->gks.as<R>();
    a.stim_head = h->nstim ? h->stim_head.as<int>() : nullptr;
    a.stim_next = h->stim_next.as<int>();
    a.stim_on = h->stim_on.as<long long>();
    a.stim_off = h->stim_off.as<long long>();
    a.stim_amp = h->stim_amp.as<R>();
    a.step_ptr = h->d_step.as<long long>();
    a.t_per_step = h->dt;
    a.Cm = (R)h->Cm; a.Xi = (R)h->Xi;
    a.nsub = h->nsub;
    for (int k = 0; k < h->nsub; k++) a.sub_dt[k] = (R)h->sub_dt[k];
    a.act_thr = (R)h->act_thr;
    a.track = h->track.as<Track>();
    a.status = h->status.as<DevStatus>();
    a.consts = h->consts.as<R>();
    a.nconst = ep_model_nconst(h->model);
    a.dvdt_out = nullptr;
    a.tt = h->tt;
    a.mh_abs = h->mh_abs;
    a.lr_table = h->lr_table.as<R>();
    a.stride = h->scheme != EP_SCHEME_CN ? 1 : 0;
    a.stride_dt = (R)h->ionic_dt;
}

// units in flight per warp of the staged CG (cg_batch kStagedBatch): its
// cg_prefetch, or the default depth
static int stage_depth(const ep_handle *h) { return h->cg_prefetch > 0 ? h->cg_prefetch : kStageDepthDefault; }

template <typename R>
void fill_cg_args(ep_handle *h, CGArgs<R> &a) {
    a.n = h->n; a.nslices = h->nslices;
    a.slice_ptr = h->slice_ptr.as<int>(); a.col = h->col.as<int>();
    a.Aval = h->Aval.as<R>(); a.Bval = h->Bval.as<R>(); a.dinv = h->dinv.as<R>();
    a.x = h->V.as<R>(); a.r = h->r.as<R>(); a.q = h->q.as<R>(); a.zp = h->zv.as<R>();
    a.p0 = h->p0.as<R>();
    a.partial = h->partial.as<double>();
    a.bar = h->bar.as<GridBarrier>();
    a.tol = h->cg_tol; a.maxit = h->cg_maxit;
    a.floor_rel = sizeof(R) == 4 ? 1.2e-7 : 2.2e-16;   // unit roundoff of R
    unsigned long long *st = h->cg_stats.as<unsigned long long>();
    a.iters_total = st;
    a.iters_max = (unsigned int *)(st + 1);
    a.fails = (unsigned int *)(st + 1) + 1;
    a.last = h->cg_last.as<double>();
    a.ninst = h->ninst;
    a.inst_row = h->d_inst_row.as<int>();
    a.inst_blk = h->d_inst_blk.as<int>();
    a.r1 = h->r1.as<R>(); a.w0 = h->w0.as<R>(); a.w1 = h->w1.as<R>();
    a.s0 = h->s0.as<R>(); a.s1 = h->s1.as<R>();
    a.delta = nullptr; a.dext = nullptr; a.vin = nullptr;   // the time step sets the predictor
    a.prefetch = h->cg_batch == kStagedBatch ? 0 : h->cg_prefetch;   // the staged kernel's is its ring depth
    a.bar_extra = h->bar_extra;
    a.depth = stage_depth(h);
}

// start the CG predictor from x0 = V again (after a state upload or when it
// is switched on)
static int reset_predictor(ep_handle *h) {
    for (DBuf *b : {&h->pd0, &h->pd1, &h->pq0, &h->pq1})
        if (b->p) EP_CUDA(cudaMemsetAsync(b->p, 0, b->bytes, h->stream));
    return EP_OK;
}

template <typename R>
int create_typed(ep_handle *h, const HostCSR &csr, const std::vector<double> &states_nm,
                 const std::vector<double> &consts, const std::vector<double> &gks) {
    const int n = h->n;
    int rc;
    // operators
    Sell sell;
    pack_sell(csr, {&csr.A, &csr.B}, sell);
    h->nslices = sell.nslices;
    if ((rc = upload_raw(h->slice_ptr, sell.slice_ptr.data(), sell.slice_ptr.size()))) return rc;
    if ((rc = upload_raw(h->col, sell.col.data(), sell.col.size()))) return rc;
    if ((rc = upload<R>(h->Aval, sell.vals[0]))) return rc;
    if ((rc = upload<R>(h->Bval, sell.vals[1]))) return rc;
    std::vector<double> dinv(h->pitch, 1.0);
    for (int i = 0; i < n; i++) {
        double d = 0.0;
        for (int k = csr.rowptr[i]; k < csr.rowptr[i + 1]; k++) if (csr.col[k] == i) d = csr.A[k];
        dinv[i] = 1.0 / d;
    }
    if ((rc = upload<R>(h->dinv, dinv))) return rc;
    const size_t vb = (size_t)h->pitch * sizeof(R);
    if ((rc = h->r.alloc(vb)) || (rc = h->q.alloc(vb)) || (rc = h->p0.alloc(vb)) || (rc = h->zv.alloc(2 * vb)))
        return rc;
    EP_CUDA(cudaMemset(h->r.p, 0, vb)); EP_CUDA(cudaMemset(h->q.p, 0, vb)); EP_CUDA(cudaMemset(h->zv.p, 0, 2 * vb));
    EP_CUDA(cudaMemset(h->p0.p, 0, vb));
    // cell states (SoA) and voltage
    std::vector<double> V(h->pitch, 0.0), S((size_t)h->ns * h->pitch, 0.0);
    const int off = is_lr(h->model) ? 0 : 1;       // LR keeps V in slot 7
    for (int i = 0; i < n; i++) {
        const double *s = &states_nm[(size_t)i * h->nstate];
        if (is_lr(h->model)) {
            V[i] = s[7];
            for (int k = 0; k < 7; k++) S[(size_t)k * h->pitch + i] = s[k];
        } else {
            V[i] = s[0];
            for (int k = 0; k < h->ns; k++) S[(size_t)k * h->pitch + i] = s[k + off];
        }
    }
    if ((rc = upload<R>(h->V, V))) return rc;
    if ((rc = upload<R>(h->S, S))) return rc;
    if ((rc = upload<R>(h->consts, consts))) return rc;
    if (!gks.empty()) {
        if ((rc = upload<R>(h->gks, gks))) return rc;
    }
    if (h->model == EP_LUORUDYWITHGATE) {
        std::vector<double> tab;
        lr_gate_table(tab);
        if ((rc = upload<R>(h->lr_table, tab))) return rc;
    }
    return EP_OK;
}

}  // namespace

// CTA groups of the persistent CG launch: every instance gets at least one
// CTA, the rest in proportion to its SELL slices (largest remainder).
// Returns -1 if there are more instances than CTAs.
// ep_cables_desc -> HostCables (zero-based ids, .angle rows per node, the
// per-cable overrides), with the arrays kept in cs
struct CableStore {
    std::vector<int> bl, bon;
    std::vector<uint8_t> ohas;
    std::vector<double> orient;
};
static int host_cables(const ep_cables_desc *cables, int n, HostCables &hc, CableStore &cs) {
    if (!cables || cables->n_bars <= 0) return EP_OK;
    EP_CHECK_ARG(cables->bars, "null cable list");
    EP_CHECK_ARG(cables->radius > 0.0, "cable radius must be positive");
    const int off = cables->one_based ? 1 : 0;
    cs.bl.resize((size_t)cables->n_bars * 2);
    for (size_t k = 0; k < cs.bl.size(); k++) {
        cs.bl[k] = cables->bars[k] - off;
        EP_CHECK_ARG(cs.bl[k] >= 0 && cs.bl[k] < n, "cable node id out of range");
    }
    hc.nb = cables->n_bars;
    hc.bars = cs.bl.data();
    hc.fibers = cables->fibers;
    hc.lv = cables->lv;
    for (int k = 0; k < 3; k++) { hc.Dp[k] = cables->Dp[k]; hc.DpLeft[k] = cables->DpLeft[k]; }
    hc.radius = cables->radius;
    hc.quad_order = cables->quad_order > 0 ? cables->quad_order : 2;
    EP_CHECK_ARG(hc.quad_order >= 1 && hc.quad_order <= 3, "cable quadrature order must be 1, 2 or 3");
    hc.orient_sticky = cables->angle_sticky ? 1 : 0;
    if (cables->n_angle > 0) {
        EP_CHECK_ARG(cables->angle_nodes && cables->angle, "null .angle data");
        cs.ohas.assign(n, 0);
        cs.orient.assign((size_t)n * 4, 0.0);
        for (int k = 0; k < cables->n_angle; k++) {
            const int v = cables->angle_nodes[k] - off;
            EP_CHECK_ARG(v >= 0 && v < n, ".angle node id out of range");
            cs.ohas[v] = 1;
            for (int c = 0; c < 4; c++) cs.orient[4 * (size_t)v + c] = cables->angle[4 * (size_t)k + c];
        }
        hc.orient_has = cs.ohas.data();
        hc.orient = cs.orient.data();
        if (cables->bar_angle) {
            cs.bon.resize(cables->n_bars);
            for (int e = 0; e < cables->n_bars; e++) {
                const int k = cables->bar_angle[e];
                EP_CHECK_ARG(k >= -1 && k < cables->n_angle, "bar_angle entry out of range");
                cs.bon[e] = k < 0 ? -1 : cables->angle_nodes[k] - off;
            }
            hc.bar_orient_node = cs.bon.data();
        }
    }
    return EP_OK;
}

// host only: the operators ep_create would build (tests and inspection)
extern "C" int ep_assemble_operators(const ep_mesh_desc *mesh, const ep_cables_desc *cables,
                                     const ep_solver_desc *sd, int64_t *nnz, int32_t *rowptr, int32_t *col,
                                     double *A, double *B, double *CL) {
    EP_CHECK_ARG(mesh && sd && nnz, "null argument");
    EP_CHECK_ARG(mesh->n_nodes > 0 && mesh->xyz && (mesh->n_tets == 0 || mesh->tets), "bad mesh");
    EP_CHECK_ARG(sd->scheme >= EP_SCHEME_CN && sd->scheme <= EP_SCHEME_EXPLICIT, "unknown scheme");
    EP_CHECK_ARG(sd->dt > 0.0, "dt must be positive");
    const int n = mesh->n_nodes;
    std::vector<int> tl((size_t)mesh->n_tets * 4);
    for (size_t e = 0; e < tl.size(); e++) {
        const int v = mesh->tets[e] - (mesh->one_based ? 1 : 0);
        EP_CHECK_ARG(v >= 0 && v < n, "tet node id out of range");
        tl[e] = v;
    }
    HostCables hc;
    CableStore cs;
    int rc0 = host_cables(cables, n, hc, cs);
    if (rc0) return rc0;
    const double Cm = mesh->Cm > 0.0 ? mesh->Cm : 1.0;
    HostCSR csr;
    const int rc = assemble_cn(n, mesh->xyz, mesh->n_tets, tl.data(), mesh->fibers, mesh->D, Cm, sd->dt,
                               sd->smoothing_alpha, csr, sd->scheme, hc.nb ? &hc : nullptr);
    if (rc) {
        set_error(rc == -2 ? "unsupported cable quadrature order" : "an element has non-positive volume or length");
        return EP_ERR_MESH;
    }
    *nnz = (int64_t)csr.col.size();
    if (!rowptr) return EP_OK;
    EP_CHECK_ARG(col && A && B && CL, "null output array");
    std::memcpy(rowptr, csr.rowptr.data(), sizeof(int32_t) * ((size_t)n + 1));
    std::memcpy(col, csr.col.data(), sizeof(int32_t) * csr.col.size());
    std::memcpy(A, csr.A.data(), sizeof(double) * csr.A.size());
    std::memcpy(B, csr.B.data(), sizeof(double) * csr.B.size());
    std::memcpy(CL, csr.CL.data(), sizeof(double) * (size_t)n);
    return EP_OK;
}

extern "C" int ep_batch_plan(int32_t ninst, const int32_t *inst_row, int32_t grid, int32_t *inst_blk) {
    if (ninst <= 0 || !inst_row || !inst_blk || grid < ninst) return EP_ERR_ARG;
    std::vector<long long> sl(ninst);
    long long tot = 0;
    for (int k = 0; k < ninst; k++) {
        if (inst_row[k + 1] < inst_row[k]) return EP_ERR_ARG;
        sl[k] = (inst_row[k + 1] + kSlice - 1) / kSlice - inst_row[k] / kSlice;
        tot += sl[k];
    }
    const int spare = grid - ninst;
    std::vector<int> cnt(ninst, 1);
    std::vector<std::pair<double, int>> rem(ninst);
    int used = 0;
    for (int k = 0; k < ninst; k++) {
        const double share = tot > 0 ? (double)spare * (double)sl[k] / (double)tot : 0.0;
        const int whole = (int)share;
        cnt[k] += whole;
        used += whole;
        rem[k] = {share - whole, k};
    }
    std::stable_sort(rem.begin(), rem.end(), [](const std::pair<double, int> &x, const std::pair<double, int> &y) {
        return x.first > y.first;
    });
    for (int k = 0; used < spare; k = (k + 1) % ninst, used++) cnt[rem[k].second]++;
    inst_blk[0] = 0;
    for (int k = 0; k < ninst; k++) inst_blk[k + 1] = inst_blk[k] + cnt[k];
    return EP_OK;
}

// (re)size the CG launch for the handle's launch shape: grid, CTA groups,
// partials, barriers and per-instance results
// every instance's grid barrier back to its initial state (count, generation
// and error word 0) with the handle's poll limit: at creation, and after a
// wait gave up (the blocks that left early leave count and err behind)
static int reset_barriers(ep_handle *h) {
    std::vector<GridBarrier> b(h->ninst);
    for (GridBarrier &x : b) x = GridBarrier{0u, 0u, 0u, h->wait_grid};
    EP_CUDA(cudaMemcpy(h->bar.p, b.data(), sizeof(GridBarrier) * b.size(), cudaMemcpyHostToDevice));
    return EP_OK;
}

static int plan_cg(ep_handle *h) {
    const int ws = stage_depth(h);
    int rc = h->precision == EP_FP64
                 ? cg_grid_size<double>(h->cg_block, &h->cg_grid, h->cg_per_sm, h->cg_batch, h->cg_variant, ws)
                 : cg_grid_size<float>(h->cg_block, &h->cg_grid, h->cg_per_sm, h->cg_batch, h->cg_variant, ws);
    if (rc) return rc;
    if (h->cg_variant == 1 && !h->w0.p) {
        const size_t vb = (size_t)h->pitch * h->rsize;
        for (DBuf *b : {&h->r1, &h->w0, &h->w1, &h->s0, &h->s1}) {
            if ((rc = b->alloc(vb))) return rc;
            EP_CUDA(cudaMemset(b->p, 0, vb));
        }
    }
    if (h->ninst > h->cg_grid) {
        set_error("%d instances but only %d CTAs in the persistent launch", h->ninst, h->cg_grid);
        return EP_ERR_ARG;
    }
    h->inst_blk.assign(h->ninst + 1, 0);
    if ((rc = ep_batch_plan(h->ninst, h->inst_row.data(), h->cg_grid, h->inst_blk.data()))) {
        set_error("bad instance layout");
        return rc;
    }
    if ((rc = upload_raw(h->d_inst_row, h->inst_row.data(), h->inst_row.size()))) return rc;
    if ((rc = upload_raw(h->d_inst_blk, h->inst_blk.data(), h->inst_blk.size()))) return rc;
    if ((rc = h->partial.alloc(sizeof(double) * 12 * (size_t)h->cg_grid))) return rc;
    if (h->bar.bytes != sizeof(GridBarrier) * (size_t)h->ninst) {
        if ((rc = h->bar.alloc(sizeof(GridBarrier) * (size_t)h->ninst))) return rc;
        if ((rc = reset_barriers(h))) return rc;
    }
    if (h->cg_last.bytes != 2 * sizeof(double) * (size_t)h->ninst) {
        if ((rc = h->cg_last.alloc(2 * sizeof(double) * (size_t)h->ninst))) return rc;
        EP_CUDA(cudaMemset(h->cg_last.p, 0, 2 * sizeof(double) * (size_t)h->ninst));
    }
    return EP_OK;
}

static void drop_graph(ep_handle *h) {
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    h->gexec = nullptr;
    h->g_steps = 0;
}

static int ensure_ecg_cap(ep_handle *h, int need) {
    if (need <= h->ecg_cap) return EP_OK;
    int cap = std::max(need, std::max(64, 2 * h->ecg_cap));
    DBuf nb;
    int rc = nb.alloc(sizeof(double) * (size_t)cap * std::max(1, h->ne));
    if (rc) return rc;
    if (h->ecg_count)
        EP_CUDA(cudaMemcpyAsync(nb.p, h->ecg_buf.p, sizeof(double) * (size_t)h->ecg_count * h->ne,
                                cudaMemcpyDeviceToDevice, h->stream));
    EP_CUDA(cudaStreamSynchronize(h->stream));
    std::swap(h->ecg_buf.p, nb.p);
    std::swap(h->ecg_buf.bytes, nb.bytes);
    h->ecg_cap = cap;
    drop_graph(h);
    return EP_OK;
}

static void fill_surrogate_args(ep_handle *h, const IonicArgs<float> &ia, SurrogateArgs &sa) {
    std::memset(&sa, 0, sizeof sa);
    sa.n = h->n; sa.pitch = h->pitch;
    sa.V = ia.V; sa.S = ia.S; sa.type = ia.type; sa.gks = ia.gks;
    sa.consts = ia.consts; sa.nconst = ia.nconst;
    sa.stim_head = ia.stim_head; sa.stim_next = ia.stim_next;
    sa.stim_on = ia.stim_on; sa.stim_off = ia.stim_off; sa.stim_amp = ia.stim_amp;
    sa.step_ptr = ia.step_ptr; sa.t_per_step = h->dt;
    sa.nsub = ia.nsub;
    for (int k = 0; k < ia.nsub; k++) sa.sub_dt[k] = ia.sub_dt[k];
    sa.Cm = ia.Cm; sa.Xi = ia.Xi; sa.act_thr = ia.act_thr;
    sa.track = ia.track;
    sa.wimg = h->sg_wimg.as<unsigned short>();
    sa.aux = h->sg_aux.as<SurrogateAux>();
    sa.fallback_list = h->sg_list.as<int>();
    sa.fallback_count = h->sg_count.as<int>();
    sa.status = h->status.as<DevStatus>();
    sa.err = h->sg_err.as<unsigned int>();
    sa.mbar_polls = h->wait_mbar;
    sa.pred = h->sg_pred.as<float>();
    sa.take = h->sg_take.as<uint8_t>();
}

// the learned ionic phase: tensor-core MLP for the nodes inside the training
// envelope, then the plain FP32 kernel over the compacted fallback list
static int launch_learned_phase(ep_handle *h, const IonicArgs<float> &ia) {
    if (!h->has_surrogate) {
        set_error("EP_SURROGATE handle stepped before ep_set_surrogate");
        return EP_ERR_ARG;
    }
    EP_CUDA(cudaMemsetAsync(h->sg_count.p, 0, sizeof(int), h->stream));
    SurrogateArgs sa;
    fill_surrogate_args(h, ia, sa);
    int rc = launch_surrogate(sa, h->stream, h->sg_variant);
    if (rc) return rc;
    // the fallback list (the nodes the network did not take) on the side
    // stream, submitted first and at higher priority, beside the physics of
    // the taken nodes: disjoint nodes; a short list's time is one node's
    // Newton chain, which then hides under k_hybrid
    IonicArgs<float> fb = ia;
    fb.node_list = h->sg_list.as<int>();
    fb.list_count = h->sg_count.as<int>();
    fb.list_warp_max = kFallbackWarpMax;    // a short list: one warp per node
    EP_CUDA(cudaEventRecord(h->ev_fork, h->stream));
    EP_CUDA(cudaStreamWaitEvent(h->side, h->ev_fork, 0));
    if ((rc = launch_ionic<float>(EP_TUSSCHER, fb, h->side, h->ionic_block, h->ionic_min))) return rc;
    EP_CUDA(cudaEventRecord(h->ev_join, h->side));
    if (h->sg_vupdate == 2 && (rc = launch_hybrid(sa, h->stream))) return rc;
    EP_CUDA(cudaStreamWaitEvent(h->stream, h->ev_join, 0));
    return EP_OK;
}

enum { K_CG = 0, K_IONIC = 1, K_ECG = 2, K_OTHER = 3 };

// event before each kernel when profiling (the class of the kernel it starts)
static int mark(ep_handle *h, size_t &ne, int kind) {
    if (!h->profile) return EP_OK;
    if (ne == h->pev.size()) {
        cudaEvent_t e;
        EP_CUDA(cudaEventCreate(&e));
        h->pev.push_back(e);
        h->pkind.push_back(kind);
    }
    h->pkind[ne] = kind;
    EP_CUDA(cudaEventRecord(h->pev[ne], h->stream));
    ne++;
    return EP_OK;
}

// one half diffusion step of the handle's scheme
template <typename R>
static int half_diffusion(ep_handle *h, const CGArgs<R> &ca) {
    if (h->scheme == EP_SCHEME_EXPLICIT) {
        for (double hh : h->ex_h) {
            int rc = launch_explicit<R>(h->n, h->nslices, h->slice_ptr.as<int>(), h->col.as<int>(), h->Aval.as<R>(),
                                        h->cl.as<R>(), h->V.as<R>(), h->q.as<R>(), hh, h->stream);
            if (rc) return rc;
        }
        h->launches += (long long)h->ex_h.size() - 1;
        return EP_OK;
    }
    return launch_cg<R>(ca, h->cg_grid, h->cg_block, h->stream, h->cg_batch, h->cg_variant);
}

// The plain ionic phase: the tissue model over every node, and in a mixed
// tissue the Purkinje cell over the .purk nodes (which the tissue launch
// skips), each with its own states, constants and Xi (CardiacBody::
// getIonicCurrent calls each node's own model, Body/CardiacBody.cc:405-435)
template <typename R>
static int ionic_phase(ep_handle *h, const IonicArgs<R> &ia) {
    if (!h->mixed) return launch_ionic<R>(h->model, ia, h->stream, h->ionic_block, h->ionic_min);
    IonicArgs<R> t = ia;
    t.skip = h->is_purk_d.as<uint8_t>();
    int rc = launch_ionic<R>(h->model, t, h->stream, h->ionic_block, h->ionic_min);
    if (rc || h->n_pk == 0) return rc;
    IonicArgs<R> p = ia;
    p.n = h->n_pk;                       // grid size; the list holds the nodes
    p.S = h->Spk.as<R>();
    p.type = nullptr;
    p.gks = nullptr;
    p.consts = h->pk_consts.as<R>();
    p.nconst = ep_model_nconst(EP_PURKINJE);
    p.Xi = (R)h->pk_Xi;
    p.lr_table = nullptr;
    p.node_list = h->pk_list.as<int>();
    p.list_count = h->pk_count.as<int>();
    h->launches += 1;
    return launch_ionic<R>(EP_PURKINJE, p, h->stream, h->ionic_block, h->ionic_min);
}

template <typename R>
static int step_typed(ep_handle *h, int nsteps, size_t &ne) {
    IonicArgs<R> ia;
    fill_ionic_args<R>(h, ia);
    CGArgs<R> ca, ca2;
    fill_cg_args<R>(h, ca);
    ca2 = ca;
    if (h->cg_predict) {
        ca.delta = h->pd0.as<R>(); ca2.delta = h->pd1.as<R>();
        ca.vin = ca2.vin = h->pvin.as<R>();
        if (h->cg_predict == 2) { ca.dext = h->pq0.as<R>(); ca2.dext = h->pq1.as<R>(); }
    }
    int rc;
    for (int s = 0; s < nsteps; s++) {
        if ((rc = mark(h, ne, K_CG))) return rc;
        if ((rc = half_diffusion<R>(h, ca))) return rc;
        if ((rc = mark(h, ne, K_IONIC))) return rc;
        if constexpr (sizeof(R) == 4) {
            if (h->precision == EP_SURROGATE) {
                if ((rc = launch_learned_phase(h, ia))) return rc;
                h->launches += h->sg_vupdate == 2 ? 4 : 3;   // network, [physics,] fallback by warps and by threads
            } else if ((rc = ionic_phase<R>(h, ia))) {
                return rc;
            }
        } else {
            if ((rc = ionic_phase<R>(h, ia))) return rc;
        }
        if ((rc = mark(h, ne, K_CG))) return rc;
        if ((rc = half_diffusion<R>(h, ca2))) return rc;
        if ((rc = mark(h, ne, K_OTHER))) return rc;
        launch_step_inc(h->d_step.as<long long>(), h->stream);
        h->launches += 4;
        h->step++;
        if (h->ecg_every && h->ne > 0 && h->step % h->ecg_every == 0) {
            if ((rc = mark(h, ne, K_ECG))) return rc;
            rc = launch_ecg<R>(h->n, h->ne, h->W.as<R>(), h->pitch, h->V.as<R>(), h->ecg_partial.as<double>(),
                               h->ecg_counter.as<unsigned int>(), h->ecg_buf.as<double>(), h->ecg_grid, h->stream,
                               h->ecg_slot.as<unsigned int>(), h->ecg_cap);
            if (rc) return rc;
            h->launches += 1;
            h->ecg_count++;
            h->ecg_t.push_back((double)h->step * h->dt);
        }
    }
    return mark(h, ne, K_OTHER);
}

// Steps replayed from one instantiated CUDA graph of g_steps steps.  The
// graph is captured from the same launch sequence as the direct path; it is
// only valid while every buffer it names stays in place, so the entry points
// that reallocate drop it.  A graph that contains ECG samples is captured and
// replayed only at step counts that are multiples of ecg_every.
template <typename R>
static int step_graph(ep_handle *h, int &nsteps) {
    int k = h->graph_steps;
    const bool ecg = h->ecg_every && h->ne > 0;
    if (ecg) k = div_up(k, h->ecg_every) * h->ecg_every;
    if (ecg && h->step % h->ecg_every != 0) return EP_OK;     // not aligned: direct steps
    if (nsteps < k) return EP_OK;
    if (!h->gexec || h->g_steps != k) {
        drop_graph(h);
        const long long step0 = h->step, launches0 = h->launches;
        const int ecg_count0 = h->ecg_count;
        const size_t ecg_t0 = h->ecg_t.size();
        size_t ne = 0;
        EP_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeRelaxed));
        int rc = step_typed<R>(h, k, ne);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(h->stream, &g);
        h->step = step0;
        h->ecg_count = ecg_count0;
        h->ecg_t.resize(ecg_t0);
        h->g_launches = h->launches - launches0;
        h->launches = launches0;
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        if (ce != cudaSuccess) {
            cudaGetLastError();
            set_error("CUDA graph capture failed: %s", cudaGetErrorString(ce));
            return EP_ERR_CUDA;
        }
        const cudaError_t ie = cudaGraphInstantiate(&h->gexec, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) {
            cudaGetLastError();
            h->gexec = nullptr;
            set_error("CUDA graph instantiation failed: %s", cudaGetErrorString(ie));
            return EP_ERR_CUDA;
        }
        h->g_steps = k;
    }
    while (nsteps >= k) {
        EP_CUDA(cudaGraphLaunch(h->gexec, h->stream));
        for (int s = 0; s < k; s++) {
            h->step++;
            if (ecg && h->step % h->ecg_every == 0) {
                h->ecg_count++;
                h->ecg_t.push_back((double)h->step * h->dt);
            }
        }
        h->launches += h->g_launches;
        nsteps -= k;
    }
    return EP_OK;
}


static std::string out_name(const char *dir, const char *stem, double t) {
    char buf[1024];
    snprintf(buf, sizeof buf, "%s/%s_time_%08.2f.%02.0f", dir, stem, t, 0.0);
    return buf;
}


extern "C" {

int ep_version(void) { return EP_ABI_VERSION; }
const char *ep_last_error(void) { return ep::last_error(); }

int ep_model_nstate(int model) {
    switch (model) {
    case EP_TUSSCHER: return 19;
    case EP_MAHAJAN: case EP_MAHAJAN_FAIL: return 26;
    case EP_LUORUDY: case EP_LUORUDYWITHGATE: return 8;
    case EP_PURKINJE: return 22;
    default: return EP_ERR_ARG;
    }
}

int ep_model_nconst(int model) {
    switch (model) {
    case EP_TUSSCHER: return TT_NC;
    case EP_MAHAJAN: case EP_MAHAJAN_FAIL: return MH_NC;
    case EP_LUORUDY: case EP_LUORUDYWITHGATE: return 1;
    case EP_PURKINJE: return PK_NC;
    default: return EP_ERR_ARG;
    }
}

int ep_model_default_consts(int model, int type, double *out) {
    EP_CHECK_ARG(out != nullptr, "null output");
    return default_consts(model, type, out);
}

void ep_destroy(ep_handle *h) {
    if (!h) return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    drop_graph(h);
    for (cudaEvent_t e : h->pev) cudaEventDestroy(e);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    for (cudaEvent_t e : h->io_ev)
        if (e) cudaEventDestroy(e);
    if (h->side) cudaStreamSynchronize(h->side);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    if (h->side) cudaStreamDestroy(h->side);
    if (h->stream) cudaStreamDestroy(h->stream);
    if (h->pin) cudaFreeHost(h->pin);
    delete h;
    cudaSetDevice(cur);
}

}  // extern "C"

// One handle over ninst independent meshes (ninst = 1: ep_create).  The
// instances are concatenated node-wise into one block-diagonal operator;
// their parameter sets are concatenated into one type table.
// ninst meshes concatenated (block-diagonal operators); with cables and
// Purkinje nodes (ninst 1 only) a mixed tissue: the cables join the tets in
// the operators and the listed nodes carry the Purkinje cell
static int create_multi(int ninst, const ep_mesh_desc *meshes, const ep_model_desc *models,
                        const ep_solver_desc *sd, int device, ep_handle **out,
                        const ep_cables_desc *cables = nullptr, int32_t n_purk = 0,
                        const int32_t *purk_nodes = nullptr) {
    EP_CHECK_ARG(meshes && models && sd && out, "null descriptor");
    *out = nullptr;
    EP_CHECK_ARG(ninst >= 1, "no instances");
    const bool mixed = n_purk > 0 || (cables && cables->n_bars > 0);
    EP_CHECK_ARG(!mixed || ninst == 1, "cables and Purkinje nodes belong to a single mesh");
    EP_CHECK_ARG(n_purk >= 0 && (n_purk == 0 || purk_nodes), "bad Purkinje node list");
    EP_CHECK_ARG(!mixed || sd->precision != EP_SURROGATE, "the learned ionic step is not built for mixed tissues");
    const ep_model_desc *md = &models[0];
    const int nst = ep_model_nstate(md->model);
    EP_CHECK_ARG(nst > 0, "unknown cell model");
    EP_CHECK_ARG(md->model != EP_PURKINJE,
                 "the Purkinje cell is not a tissue model: list its nodes in ep_create_mixed");
    EP_CHECK_ARG(sd->precision == EP_FP64 || sd->precision == EP_FP32 ||
                     (sd->precision == EP_SURROGATE && md->model == EP_TUSSCHER),
                 "unsupported precision (EP_SURROGATE needs the ten Tusscher model)");
    EP_CHECK_ARG(sd->dt > 0 && sd->ionic_dt > 0, "dt and ionic_dt must be positive");
    EP_CHECK_ARG(sd->scheme >= EP_SCHEME_CN && sd->scheme <= EP_SCHEME_EXPLICIT, "unknown scheme");
    if (sd->scheme != EP_SCHEME_CN && sd->smoothing_alpha > 0.0) {
        set_error("diffusive smoothing is defined for the Crank-Nicolson scheme only");
        return EP_ERR_UNSUPPORTED;
    }
    EP_CHECK_ARG(sd->scheme == EP_SCHEME_CN || sd->precision != EP_SURROGATE,
                 "the learned ionic step is trained for the Crank-Nicolson sub-steps");
    long long ntot = 0, mtot = 0;
    int ntypes = 0;
    bool any_type = false, any_gks = false, all_fib = true;
    for (int k = 0; k < ninst; k++) {
        const ep_mesh_desc *mesh = &meshes[k];
        EP_CHECK_ARG(mesh->n_nodes > 0 && mesh->n_tets > 0 && mesh->xyz && mesh->tets, "empty mesh");
        EP_CHECK_ARG(models[k].model == md->model, "all instances must use the same cell model");
        EP_CHECK_ARG((mesh->Cm > 0 ? mesh->Cm : 1.0) == (meshes[0].Cm > 0 ? meshes[0].Cm : 1.0),
                     "all instances must have the same C_m");
        ntot += mesh->n_nodes;
        mtot += mesh->n_tets;
        ntypes += models[k].n_types > 0 ? models[k].n_types : 1;
        any_type |= models[k].node_type != nullptr;
        any_gks |= models[k].node_gks_scale != nullptr;
        all_fib &= mesh->fibers != nullptr;
    }
    EP_CHECK_ARG(ntot < (1ll << 31) - 64 && 4 * mtot < (1ll << 31), "mesh too large");
    EP_CHECK_ARG(ntypes <= kMaxTypes, "too many parameter sets");
    std::unique_ptr<ep_handle> h(new ep_handle());
    h->device = device;
    EP_CUDA(cudaSetDevice(device));
    const int n = (int)ntot;
    h->n = n;
    h->ninst = ninst;
    h->pitch = (n + 31) / 32 * 32;
    h->model = md->model;
    h->precision = sd->precision;
    h->rsize = sd->precision == EP_FP64 ? 8 : 4;
    h->nstate = nst;
    h->ns = is_lr(md->model) ? 7 : nst - 1;
    h->ntypes = ntypes;
    h->dt = sd->dt; h->ionic_dt = sd->ionic_dt;
    h->nsub = substeps(sd->dt, sd->ionic_dt, h->sub_dt);
    EP_CHECK_ARG(h->nsub > 0, "more than 64 ionic sub-steps per step");
    h->Cm = meshes[0].Cm > 0 ? meshes[0].Cm : 1.0;
    h->scheme = sd->scheme;
    // the reference's fixed tolerances: CN 1e-7 (EP_CrankNicholson.cc:104),
    // BE 1e-10 (EP_BackwardEuler.cc:67)
    h->cg_tol = sd->cg_tol > 0 ? sd->cg_tol : (sd->scheme == EP_SCHEME_BE ? 1e-10 : 1e-7);
    if (sd->scheme == EP_SCHEME_EXPLICIT) {
        // EP_ExplicitSolver::Solve: sub-steps of min(dtDiff, dt/2) until less
        // than 1e-6 of the half step is left, the last one shortened
        const double dtd = sd->diffusion_dt > 0 ? sd->diffusion_dt : 0.05;
        double solve = 0.5 * sd->dt, stepT = dtd < 0.5 * sd->dt ? dtd : 0.5 * sd->dt;
        while (solve > 1e-6) {
            h->ex_h.push_back(stepT);
            solve -= stepT;
            stepT = stepT < solve ? stepT : solve;
            EP_CHECK_ARG(h->ex_h.size() <= 100000, "too many explicit diffusion sub-steps");
        }
    }
    h->cg_maxit = sd->cg_maxit > 0 ? sd->cg_maxit : 1000;
    h->ecg_every = sd->ecg_every > 0 ? sd->ecg_every : 0;
    h->act_thr = sd->act_threshold != 0.0 ? sd->act_threshold : -40.0;
    h->Xi = md->user_xi > 0 ? md->user_xi : model_xi(md->model);
    h->tt.newton_cap = md->newton_cap > 0 ? md->newton_cap : 100;
    h->tt.jac_true = md->tt_jacobian == EP_TT_JAC_TRUE ? 1 : 0;
    h->tt.fp32_scaled_tol = sd->precision == EP_FP64 ? 0 : 1;
    h->tt.newton_tol = sd->newton_tol > 0 ? sd->newton_tol : 1e-6;
    h->mh_abs = md->mh_abs_mode ? 1 : 0;
    for (int k = 0; k < 3; k++) h->D[k] = meshes[0].D[k];
    const int nc = ep_model_nconst(md->model);
    std::vector<double> consts((size_t)ntypes * nc);
    std::vector<double> st((size_t)n * nst);
    std::vector<uint8_t> node_type(any_type || ninst > 1 ? n : 0, 0);
    std::vector<double> gks(any_gks ? n : 0, 1.0);
    h->xyz.resize(3 * (size_t)n);
    h->tets.resize(4 * (size_t)mtot);
    if (all_fib) h->fibers.resize(9 * (size_t)mtot);
    h->inst_row.assign(ninst + 1, 0);
    HostCSR csr;
    csr.n = n;
    csr.rowptr.assign(1, 0);
    int noff = 0, toff = 0;
    long long eoff = 0;
    for (int k = 0; k < ninst; k++) {
        const ep_mesh_desc *mesh = &meshes[k];
        const ep_model_desc *mk = &models[k];
        const int ni = mesh->n_nodes, mi = mesh->n_tets;
        const int nti = mk->n_types > 0 ? mk->n_types : 1;
        std::vector<int> tl((size_t)mi * 4);
        for (size_t e = 0; e < (size_t)mi * 4; e++) {
            const int v = mesh->tets[e] - (mesh->one_based ? 1 : 0);
            EP_CHECK_ARG(v >= 0 && v < ni, "tet node id out of range");
            tl[e] = v;
            h->tets[(size_t)eoff * 4 + e] = v + noff;
        }
        std::memcpy(&h->xyz[3 * (size_t)noff], mesh->xyz, sizeof(double) * 3 * ni);
        if (all_fib) std::memcpy(&h->fibers[9 * (size_t)eoff], mesh->fibers, sizeof(double) * 9 * mi);
        // FEM operators of this instance in FP64 (with the cables of a mixed
        // tissue after the tets), appended block-diagonally
        HostCSR ci;
        HostCables hc;
        CableStore cs;
        if (mixed) {
            int rc1 = host_cables(cables, ni, hc, cs);
            if (rc1) return rc1;
            h->cab_bars = cs.bl;
            h->cab_bon = cs.bon;
            h->cab_ohas = cs.ohas;
            h->cab_orient = cs.orient;
            if (hc.fibers) h->cab_fib.assign(hc.fibers, hc.fibers + 9 * (size_t)hc.nb);
            h->cab_quad = hc.quad_order;
            h->cab_sticky = hc.orient_sticky;
        }
        const int arc = assemble_cn(ni, mesh->xyz, mi, tl.data(), mesh->fibers, mesh->D, h->Cm, h->dt,
                                    sd->smoothing_alpha, ci, sd->scheme, hc.nb ? &hc : nullptr);
        if (arc != 0) {
            set_error(arc == -2 ? "unsupported cable quadrature order"
                                : "mesh %d has an element with non-positive volume or length", k);
            return EP_ERR_MESH;
        }
        const int base = csr.rowptr.back();
        for (int i = 0; i < ni; i++) csr.rowptr.push_back(base + ci.rowptr[i + 1]);
        for (int c : ci.col) csr.col.push_back(c + noff);
        csr.A.insert(csr.A.end(), ci.A.begin(), ci.A.end());
        csr.B.insert(csr.B.end(), ci.B.begin(), ci.B.end());
        csr.CL.insert(csr.CL.end(), ci.CL.begin(), ci.CL.end());
        // parameter sets
        for (int t = 0; t < nti; t++) {
            double *dst = &consts[(size_t)(toff + t) * nc];
            if (mk->type_consts) std::memcpy(dst, mk->type_consts + (size_t)t * nc, sizeof(double) * nc);
            else default_consts(md->model, t, dst);
        }
        // initial states, node-major like InterVariables
        for (int i = 0; i < ni; i++) {
            const int t = mk->node_type ? mk->node_type[i] : 0;
            if (mk->node_type) EP_CHECK_ARG(t < nti, "node type beyond n_types");
            double *dst = &st[(size_t)(noff + i) * nst];
            if (mk->initial_states) std::memcpy(dst, mk->initial_states + (size_t)i * nst, sizeof(double) * nst);
            else default_state(md->model, t, dst);
            if (!node_type.empty()) node_type[noff + i] = (uint8_t)(toff + t);
            if (mk->node_gks_scale) gks[noff + i] = mk->node_gks_scale[i];
        }
        noff += ni;
        toff += nti;
        eoff += mi;
        h->inst_row[k + 1] = noff;
    }
    h->model_V0.assign(n, 0.0);
    if (is_mh(md->model))
        for (int i = 0; i < n; i++) h->model_V0[i] = st[(size_t)i * nst];
    // mixed tissue: the Purkinje population (CardiacBody::New gives every
    // .purk node a Purkinje cell, Body/CardiacBody.cc:1025-1040)
    std::vector<double> pk_st;
    std::vector<int> pk_list;
    h->nstate_api = nst;
    if (mixed) {
        const int pns = ep_model_nstate(EP_PURKINJE);
        h->mixed = 1;
        h->nstate_api = std::max(nst, pns);
        h->is_purk.assign(n, 0);
        const int off = meshes[0].one_based ? 1 : 0;
        for (int k = 0; k < n_purk; k++) {
            const int v = purk_nodes[k] - off;
            EP_CHECK_ARG(v >= 0 && v < n, "Purkinje node id out of range");
            h->is_purk[v] = 1;
        }
        pk_st.assign((size_t)n * pns, 0.0);
        for (int i = 0; i < n; i++) {
            if (!h->is_purk[i]) continue;
            pk_list.push_back(i);
            double *ps = &pk_st[(size_t)i * pns];
            default_state(EP_PURKINJE, 0, ps);
            // the shared V starts from the cell's own voltage, which is also
            // what Purkinje::getVoltage reports (IonicModel.h:42, Purkinje.h:79)
            st[(size_t)i * nst + (is_lr(md->model) ? 7 : 0)] = ps[0];
            h->model_V0[i] = ps[0];
        }
        h->n_pk = (int)pk_list.size();
        h->pk_Xi = md->user_xi > 0 ? md->user_xi : model_xi(EP_PURKINJE);
    }
    int rc = EP_OK;
    EP_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    EP_CUDA(cudaEventCreate(&h->ev0));
    EP_CUDA(cudaEventCreate(&h->ev1));
    if (!node_type.empty()) {
        if ((rc = upload_raw(h->type, node_type.data(), node_type.size()))) return rc;
    }
    if (h->precision == EP_FP64) rc = create_typed<double>(h.get(), csr, st, consts, gks);
    else rc = create_typed<float>(h.get(), csr, st, consts, gks);
    if (rc) return rc;
    if (mixed) {
        const int pns = ep_model_nstate(EP_PURKINJE);     // V + the stored states
        std::vector<double> S((size_t)(pns - 1) * h->pitch, 0.0);
        for (int i = 0; i < n; i++)
            if (h->is_purk[i])
                for (int k = 0; k < pns - 1; k++) S[(size_t)k * h->pitch + i] = pk_st[(size_t)i * pns + k + 1];
        std::vector<double> pc(ep_model_nconst(EP_PURKINJE));
        default_consts(EP_PURKINJE, 0, pc.data());
        rc = h->precision == EP_FP64 ? upload<double>(h->Spk, S) : upload<float>(h->Spk, S);
        if (!rc) rc = h->precision == EP_FP64 ? upload<double>(h->pk_consts, pc) : upload<float>(h->pk_consts, pc);
        if (rc) return rc;
        if (pk_list.empty()) pk_list.push_back(0);           // never read: the count is 0
        if ((rc = upload_raw(h->pk_list, pk_list.data(), pk_list.size()))) return rc;
        if ((rc = upload_raw(h->pk_count, &h->n_pk, 1))) return rc;
        if ((rc = upload_raw(h->is_purk_d, h->is_purk.data(), h->is_purk.size()))) return rc;
    }
    if (h->scheme == EP_SCHEME_EXPLICIT) {
        std::vector<double> cl(csr.CL);
        cl.resize(h->pitch, 1.0);
        rc = h->precision == EP_FP64 ? upload<double>(h->cl, cl) : upload<float>(h->cl, cl);
        if (rc) return rc;
    }
    // solver scratch and status
    if ((rc = plan_cg(h.get()))) return rc;
    if ((rc = h->status.alloc(sizeof(DevStatus)))) return rc;
    if ((rc = h->cg_stats.alloc(32))) return rc;
    if ((rc = h->d_step.alloc(sizeof(long long)))) return rc;
    if ((rc = h->ecg_slot.alloc(sizeof(unsigned int)))) return rc;
    EP_CUDA(cudaMemset(h->status.p, 0, sizeof(DevStatus)));
    EP_CUDA(cudaMemset(h->cg_stats.p, 0, 32));
    EP_CUDA(cudaMemset(h->d_step.p, 0, sizeof(long long)));
    EP_CUDA(cudaMemset(h->ecg_slot.p, 0, sizeof(unsigned int)));
    std::vector<Track> tr(n, Track{-1.f, -1.f, -1.f, 1e30f});
    if ((rc = upload_raw(h->track, tr.data(), tr.size()))) return rc;
    EP_CUDA(cudaDeviceSynchronize());
    *out = h.release();
    return EP_OK;
}

extern "C" {

int ep_create(const ep_mesh_desc *mesh, const ep_model_desc *md, const ep_solver_desc *sd,
              int device, ep_handle **out) {
    return create_multi(1, mesh, md, sd, device, out);
}

int ep_create_mixed(const ep_mesh_desc *mesh, const ep_cables_desc *cables, int32_t n_purk,
                    const int32_t *purk_nodes, const ep_model_desc *tissue, const ep_solver_desc *sd,
                    int device, ep_handle **out) {
    return create_multi(1, mesh, tissue, sd, device, out, cables, n_purk, purk_nodes);
}

int ep_batch_create(int32_t n_inst, const ep_mesh_desc *meshes, const ep_model_desc *models,
                    const ep_solver_desc *sd, int device, ep_handle **out) {
    return create_multi(n_inst, meshes, models, sd, device, out);
}

int ep_batch_layout(const ep_handle *h, int32_t *n_inst, int32_t *node_offset, int32_t *cta_offset) {
    EP_CHECK_ARG(h, "null handle");
    if (n_inst) *n_inst = h->ninst;
    for (int k = 0; k <= h->ninst; k++) {
        if (node_offset) node_offset[k] = h->inst_row[k];
        if (cta_offset) cta_offset[k] = h->inst_blk[k];
    }
    return EP_OK;
}

int ep_batch_cg_last(ep_handle *h, int32_t *iters, double *relres) {
    EP_CHECK_ARG(h, "null handle");
    EP_CUDA(cudaSetDevice(h->device));
    std::vector<double> last(2 * (size_t)h->ninst);
    EP_CUDA(cudaMemcpyAsync(last.data(), h->cg_last.p, sizeof(double) * last.size(), cudaMemcpyDeviceToHost,
                            h->stream));
    EP_CUDA(cudaStreamSynchronize(h->stream));
    for (int k = 0; k < h->ninst; k++) {
        if (iters) iters[k] = (int32_t)last[2 * k];
        if (relres) relres[k] = last[2 * k + 1];
    }
    return EP_OK;
}

int ep_num_nodes(const ep_handle *h) { return h ? h->n : EP_ERR_ARG; }
int ep_num_states(const ep_handle *h) { return h ? h->nstate_api : EP_ERR_ARG; }

}  // extern "C"

// Host <-> device state transfers go through one pinned staging buffer of
// the handle (grown on demand) and copy into the existing device buffers:
// the buffers never move after ep_create, which captured graphs rely on.
static void *stage(ep_handle *h, size_t bytes) {
    if (bytes > h->pin_bytes) {
        if (h->pin) cudaFreeHost(h->pin);
        h->pin = nullptr;
        h->pin_bytes = 0;
        if (cudaMallocHost(&h->pin, bytes) != cudaSuccess) {
            cudaGetLastError();
            set_error("cudaMallocHost(%zu) failed", bytes);
            return nullptr;
        }
        h->pin_bytes = bytes;
    }
    return h->pin;
}

// Host <-> device transfers of the per-node arrays in chunks, so that the
// host-side conversion (FP64 node-major <-> the device's R / SoA layout) of
// one chunk overlaps the copy engine's transfer of the next: the copies of a
// chunk are issued as soon as it is converted (uploads), or all at once with
// an event after each chunk and each chunk converted once its event has
// completed (downloads).  Arrays under 64K nodes go in one piece.
constexpr int kIoChunks = 16;
static_assert(kIoChunks <= (int)(sizeof(((ep_handle *)nullptr)->io_ev) / sizeof(cudaEvent_t)), "io_ev too small");

static int io_chunks(ep_handle *h, int count) {
    if (count < (1 << 16)) return 1;
    for (cudaEvent_t &e : h->io_ev)
        if (!e) EP_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return kIoChunks;
}
// chunk k of K over [0, total), boundaries on multiples of 32 elements
static void io_range(int total, int k, int K, int &b, int &e) {
    const long long step = ((long long)total + K - 1) / K;
    const long long st = (step + 31) / 32 * 32;
    b = (int)std::min<long long>(total, st * k);
    e = (int)std::min<long long>(total, st * (k + 1));
}

template <typename R>
static int put_voltage(ep_handle *h, const double *V) {
    R *st = (R *)stage(h, sizeof(R) * h->n);
    if (!st) return EP_ERR_NOMEM;
    const int K = h->n >= (1 << 16) ? kIoChunks : 1;
    for (int k = 0; k < K; k++) {
        int b, e;
        io_range(h->n, k, K, b, e);
        if (e <= b) continue;
#pragma omp parallel for schedule(static)
        for (int i = b; i < e; i++) st[i] = (R)V[i];
        EP_CUDA(cudaMemcpyAsync(h->V.as<R>() + b, st + b, sizeof(R) * (e - b), cudaMemcpyHostToDevice, h->stream));
    }
    int rc = reset_predictor(h);
    if (rc) return rc;
    EP_CUDA(cudaStreamSynchronize(h->stream));
    return EP_OK;
}

template <typename R>
static int get_voltage(ep_handle *h, double *V) {
    R *st = (R *)stage(h, sizeof(R) * h->n);
    if (!st) return EP_ERR_NOMEM;
    const int K = io_chunks(h, h->n);
    if (K < 0) return K;
    if (K == 1) {
        EP_CUDA(cudaMemcpyAsync(st, h->V.p, sizeof(R) * h->n, cudaMemcpyDeviceToHost, h->stream));
        EP_CUDA(cudaStreamSynchronize(h->stream));
#pragma omp parallel for schedule(static)
        for (int i = 0; i < h->n; i++) V[i] = (double)st[i];
        return EP_OK;
    }
    for (int k = 0; k < K; k++) {
        int b, e;
        io_range(h->n, k, K, b, e);
        if (e > b)
            EP_CUDA(cudaMemcpyAsync(st + b, h->V.as<R>() + b, sizeof(R) * (e - b), cudaMemcpyDeviceToHost, h->stream));
        EP_CUDA(cudaEventRecord(h->io_ev[k], h->stream));
    }
    for (int k = 0; k < K; k++) {
        int b, e;
        io_range(h->n, k, K, b, e);
        EP_CUDA(cudaEventSynchronize(h->io_ev[k]));
#pragma omp parallel for schedule(static)
        for (int i = b; i < e; i++) V[i] = (double)st[i];
    }
    return EP_OK;
}

// stored states <-> node-major rows (State[0] = V except LR, which keeps V
// in slot 7); the staging buffer has the device's SoA layout, so a chunk of
// nodes is one 2-D copy per population
template <typename R>
static int put_states(ep_handle *h, const double *in) {
    const size_t tot = (size_t)h->ns * h->pitch;
    const int pns1 = h->mixed ? ep_model_nstate(EP_PURKINJE) - 1 : 0;
    const size_t ptot = (size_t)pns1 * h->pitch;
    R *st = (R *)stage(h, sizeof(R) * (tot + ptot));
    if (!st) return EP_ERR_NOMEM;
    R *sp = st + tot;
    const int off = is_lr(h->model) ? 0 : 1;
    const int w = h->nstate_api;
    const size_t rp = sizeof(R) * (size_t)h->pitch;
    const int K = h->pitch >= (1 << 16) ? kIoChunks : 1;
    for (int c = 0; c < K; c++) {
        int b, e;
        io_range(h->pitch, c, K, b, e);
        if (e <= b) continue;
#pragma omp parallel for schedule(static)
        for (int i = b; i < e; i++) {
            const bool pk = h->mixed && i < h->n && h->is_purk[i];
            if (i < h->n && !pk) {
                const double *s = in + (size_t)i * w;
                for (int k = 0; k < h->ns; k++) st[(size_t)k * h->pitch + i] = (R)s[k + off];
            } else {
                for (int k = 0; k < h->ns; k++) st[(size_t)k * h->pitch + i] = R(0);
            }
            // a Purkinje node's row: V, then its stored states (Purkinje.h)
            for (int k = 0; k < pns1; k++) sp[(size_t)k * h->pitch + i] = pk ? (R)in[(size_t)i * w + 1 + k] : R(0);
        }
        const size_t wb = sizeof(R) * (size_t)(e - b);
        if (h->ns)
            EP_CUDA(cudaMemcpy2DAsync(h->S.as<R>() + b, rp, st + b, rp, wb, h->ns, cudaMemcpyHostToDevice, h->stream));
        if (ptot)
            EP_CUDA(cudaMemcpy2DAsync(h->Spk.as<R>() + b, rp, sp + b, rp, wb, pns1, cudaMemcpyHostToDevice, h->stream));
    }
    EP_CUDA(cudaStreamSynchronize(h->stream));
    return EP_OK;
}

template <typename R>
static int get_states(ep_handle *h, double *out) {
    const size_t tot = (size_t)h->ns * h->pitch;
    const int pns1 = h->mixed ? ep_model_nstate(EP_PURKINJE) - 1 : 0;
    const size_t ptot = (size_t)pns1 * h->pitch;
    R *st = (R *)stage(h, sizeof(R) * (tot + h->pitch + ptot));
    if (!st) return EP_ERR_NOMEM;
    R *sv = st + tot;
    R *sp = sv + h->pitch;
    const size_t rp = sizeof(R) * (size_t)h->pitch;
    const int K = io_chunks(h, h->n);
    if (K < 0) return K;
    for (int c = 0; c < K; c++) {
        int b, e;
        io_range(h->n, c, K, b, e);
        if (e > b) {
            const size_t wb = sizeof(R) * (size_t)(e - b);
            if (h->ns)
                EP_CUDA(cudaMemcpy2DAsync(st + b, rp, h->S.as<R>() + b, rp, wb, h->ns, cudaMemcpyDeviceToHost, h->stream));
            EP_CUDA(cudaMemcpyAsync(sv + b, h->V.as<R>() + b, wb, cudaMemcpyDeviceToHost, h->stream));
            if (ptot)
                EP_CUDA(cudaMemcpy2DAsync(sp + b, rp, h->Spk.as<R>() + b, rp, wb, pns1, cudaMemcpyDeviceToHost, h->stream));
        }
        if (K > 1) EP_CUDA(cudaEventRecord(h->io_ev[c], h->stream));
    }
    if (K == 1) EP_CUDA(cudaStreamSynchronize(h->stream));
    const bool lr = is_lr(h->model);
    const int w = h->nstate_api;
    for (int c = 0; c < K; c++) {
        int b, e;
        io_range(h->n, c, K, b, e);
        if (K > 1) EP_CUDA(cudaEventSynchronize(h->io_ev[c]));
#pragma omp parallel for schedule(static)
        for (int i = b; i < e; i++) {
            double *o = out + (size_t)i * w;
            for (int k = h->nstate; k < w; k++) o[k] = 0.0;
            if (h->mixed && h->is_purk[i]) {
                // the Purkinje cell's row (its nVar is ep_model_nstate(EP_PURKINJE))
                o[0] = (double)sv[i];
                for (int k = 0; k < pns1; k++) o[k + 1] = (double)sp[(size_t)k * h->pitch + i];
                for (int k = pns1 + 1; k < w; k++) o[k] = 0.0;
            } else if (lr) {
                for (int k = 0; k < 7; k++) o[k] = (double)st[(size_t)k * h->pitch + i];
                o[7] = (double)sv[i];
            } else {
                o[0] = (double)sv[i];
                for (int k = 0; k < h->ns; k++) o[k + 1] = (double)st[(size_t)k * h->pitch + i];
            }
        }
    }
    return EP_OK;
}

extern "C" {

int ep_set_voltage(ep_handle *h, const double *V) {
    EP_CHECK_ARG(h && V, "null argument");
    EP_CUDA(cudaSetDevice(h->device));
    return h->precision == EP_FP64 ? put_voltage<double>(h, V) : put_voltage<float>(h, V);
}

int ep_get_voltage(ep_handle *h, double *V) {
    EP_CHECK_ARG(h && V, "null argument");
    EP_CUDA(cudaSetDevice(h->device));
    return h->precision == EP_FP64 ? get_voltage<double>(h, V) : get_voltage<float>(h, V);
}

int ep_get_model_voltage(ep_handle *h, double *V) {
    EP_CHECK_ARG(h && V, "null argument");
    std::memcpy(V, h->model_V0.data(), sizeof(double) * h->n);
    return EP_OK;
}

int ep_get_states(ep_handle *h, double *out) {
    EP_CHECK_ARG(h && out, "null argument");
    EP_CUDA(cudaSetDevice(h->device));
    return h->precision == EP_FP64 ? get_states<double>(h, out) : get_states<float>(h, out);
}

int ep_set_states(ep_handle *h, const double *in) {
    EP_CHECK_ARG(h && in, "null argument");
    EP_CUDA(cudaSetDevice(h->device));
    return h->precision == EP_FP64 ? put_states<double>(h, in) : put_states<float>(h, in);
}

int ep_set_stimulus(ep_handle *h, int32_t n, const int32_t *ids, const double *t_on,
                    const double *t_off, const double *amp) {
    EP_CHECK_ARG(h, "null handle");
    EP_CHECK_ARG(n >= 0 && (n == 0 || (ids && t_on && t_off && amp)), "bad stimulus table");
    EP_CUDA(cudaSetDevice(h->device));
    EP_CUDA(cudaStreamSynchronize(h->stream));
    drop_graph(h);
    std::vector<int> head(h->n, -1), next(n, -1);
    std::vector<long long> on(n), off(n);
    std::vector<double> a(n);
    for (int k = 0; k < n; k++) {
        EP_CHECK_ARG(ids[k] >= 0 && ids[k] < h->n, "stimulus node id out of range");
        next[k] = head[ids[k]];
        head[ids[k]] = k;
        on[k] = (long long)(t_on[k] / h->dt);      // long(t/dt) as EPSimulator.cc:487-488
        off[k] = (long long)(t_off[k] / h->dt);
        a[k] = amp[k];
    }
    int rc;
    if ((rc = upload_raw(h->stim_head, head.data(), head.size()))) return rc;
    if ((rc = upload_raw(h->stim_next, next.data(), next.size()))) return rc;
    if ((rc = upload_raw(h->stim_on, on.data(), on.size()))) return rc;
    if ((rc = upload_raw(h->stim_off, off.data(), off.size()))) return rc;
    rc = h->precision == EP_FP64 ? upload<double>(h->stim_amp, a) : upload<float>(h->stim_amp, a);
    h->nstim = n;
    return rc;
}

int ep_set_electrodes(ep_handle *h, int32_t ne, const double *xyz, const double *D_ecg) {
    EP_CHECK_ARG(h, "null handle");
    EP_CHECK_ARG(ne >= 0 && ne <= 16 && (ne == 0 || xyz), "1..16 electrodes");
    if (h->ninst > 1) {
        set_error("pseudo-ECG electrodes are per mesh; not available on a batch handle");
        return EP_ERR_UNSUPPORTED;
    }
    EP_CUDA(cudaSetDevice(h->device));
    EP_CUDA(cudaStreamSynchronize(h->stream));
    drop_graph(h);
    const double *D = D_ecg ? D_ecg : h->D;
    std::vector<double> W;
    HostCables hc;
    if (!h->cab_bars.empty()) {
        hc.nb = (int)(h->cab_bars.size() / 2);
        hc.bars = h->cab_bars.data();
        hc.fibers = h->cab_fib.empty() ? nullptr : h->cab_fib.data();
        hc.radius = kEcgCableRadius;
        hc.quad_order = h->cab_quad;
        hc.orient_sticky = h->cab_sticky;
        hc.orient_has = h->cab_ohas.empty() ? nullptr : h->cab_ohas.data();
        hc.orient = h->cab_orient.empty() ? nullptr : h->cab_orient.data();
        hc.bar_orient_node = h->cab_bon.empty() ? nullptr : h->cab_bon.data();
    }
    ecg_weights(h->n, h->xyz.data(), (int)(h->tets.size() / 4), h->tets.data(),
                h->fibers.empty() ? nullptr : h->fibers.data(), D, ne, xyz, W, hc.nb ? &hc : nullptr);
    // pad each electrode row to the pitch
    std::vector<double> Wp((size_t)ne * h->pitch, 0.0);
    for (int k = 0; k < ne; k++)
        std::memcpy(&Wp[(size_t)k * h->pitch], &W[(size_t)k * h->n], sizeof(double) * h->n);
    int rc = h->precision == EP_FP64 ? upload<double>(h->W, Wp) : upload<float>(h->W, Wp);
    if (rc) return rc;
    h->ne = ne;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    h->ecg_grid = std::max(1, std::min(nsm * 4, div_up(h->n, 256)));
    if ((rc = h->ecg_partial.alloc(sizeof(double) * 16 * (size_t)h->ecg_grid))) return rc;
    if ((rc = h->ecg_counter.alloc(sizeof(unsigned int)))) return rc;
    EP_CUDA(cudaMemset(h->ecg_counter.p, 0, sizeof(unsigned int)));
    EP_CUDA(cudaMemset(h->ecg_slot.p, 0, sizeof(unsigned int)));
    h->ecg_cap = 0; h->ecg_count = 0; h->ecg_t.clear();
    h->ecg_buf.alloc(0);
    return EP_OK;
}

int ep_step(ep_handle *h, int32_t nsteps, ep_step_stats *stats) {
    EP_CHECK_ARG(h && nsteps >= 0, "bad arguments");
    EP_CUDA(cudaSetDevice(h->device));
    if (h->ecg_every && h->ne > 0) {
        int rc = ensure_ecg_cap(h, h->ecg_count + nsteps / h->ecg_every + 1);
        if (rc) return rc;
    }
    EP_CUDA(cudaMemsetAsync(h->status.p, 0, sizeof(DevStatus), h->stream));
    EP_CUDA(cudaMemsetAsync(h->cg_stats.p, 0, 32, h->stream));
    EP_CUDA(cudaEventRecord(h->ev0, h->stream));
    // the clock at entry: a call whose waits gave up did not take its steps
    const long long step0 = h->step;
    const int ecg_count0 = h->ecg_count;
    const size_t ecg_t0 = h->ecg_t.size();
    size_t ne = 0;
    h->launches = 0;
    int rc = EP_OK;
    int left = nsteps;
    if (h->graph_steps > 0 && !h->profile) {
        // direct steps up to the ECG sampling phase, then whole graphs
        if (h->ecg_every && h->ne > 0) {
            const int lead = (int)((h->ecg_every - h->step % h->ecg_every) % h->ecg_every);
            const int d = std::min(lead, left);
            rc = h->precision == EP_FP64 ? step_typed<double>(h, d, ne) : step_typed<float>(h, d, ne);
            if (rc) return rc;
            left -= d;
        }
        rc = h->precision == EP_FP64 ? step_graph<double>(h, left) : step_graph<float>(h, left);
        if (rc) return rc;
    }
    rc = h->precision == EP_FP64 ? step_typed<double>(h, left, ne) : step_typed<float>(h, left, ne);
    if (rc) return rc;
    EP_CUDA(cudaEventRecord(h->ev1, h->stream));
    EP_CUDA(cudaEventSynchronize(h->ev1));
    double kms[4] = {0, 0, 0, 0};
    for (size_t k = 0; k + 1 < ne; k++) {
        float e = 0.f;
        EP_CUDA(cudaEventElapsedTime(&e, h->pev[k], h->pev[k + 1]));
        kms[h->pkind[k]] += e;
    }
    DevStatus st;
    unsigned long long cgs[4];
    GridBarrier bar;
    EP_CUDA(cudaMemcpy(&st, h->status.p, sizeof st, cudaMemcpyDeviceToHost));
    EP_CUDA(cudaMemcpy(cgs, h->cg_stats.p, 32, cudaMemcpyDeviceToHost));
    {
        std::vector<GridBarrier> bars(h->ninst);
        EP_CUDA(cudaMemcpy(bars.data(), h->bar.p, sizeof(GridBarrier) * bars.size(), cudaMemcpyDeviceToHost));
        bar = bars[0];
        for (const GridBarrier &b : bars) bar.err |= b.err;
    }
    float ms = 0.f;
    EP_CUDA(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        stats->steps = nsteps;
        stats->cg_iters = (int64_t)cgs[0];
        stats->cg_max_iters = (int32_t)((unsigned int *)(cgs + 1))[0];
        stats->cg_failures = (int32_t)((unsigned int *)(cgs + 1))[1];
        stats->newton_iters = (int64_t)st.newton_iters;
        stats->newton_cap_hits = (int32_t)st.newton_cap_hits;
        stats->nonfinite = (int32_t)st.nonfinite;
        stats->fallback_nodes = (int64_t)st.fallback;
        stats->device_ms = ms;
        stats->timeouts = (int32_t)bar.err;
        stats->cg_ms = kms[K_CG];
        stats->ionic_ms = kms[K_IONIC];
        stats->ecg_ms = kms[K_ECG];
        stats->launches = h->launches;
    }
    unsigned int sg_err = 0;
    if (h->has_surrogate) EP_CUDA(cudaMemcpy(&sg_err, h->sg_err.p, sizeof sg_err, cudaMemcpyDeviceToHost));
    if (stats) stats->timeouts += (int32_t)sg_err;
    if (bar.err || sg_err) {
        // the kernels left early; put the wait state back so the handle can
        // step again, and the clock (host and device step counters, ECG
        // samples) back to the call's start: the voltage and states are not
        // to be trusted and are put back by the caller (ep_set_voltage,
        // ep_set_states or ep_read_restart) before stepping on
        int rc2 = reset_barriers(h);
        if (rc2) return rc2;
        if (sg_err) EP_CUDA(cudaMemset(h->sg_err.p, 0, sizeof(unsigned int)));
        h->step = step0;
        h->ecg_count = ecg_count0;
        h->ecg_t.resize(ecg_t0);
        EP_CUDA(cudaMemcpy(h->d_step.p, &h->step, sizeof(long long), cudaMemcpyHostToDevice));
        if (h->ecg_slot.p) {
            const unsigned int slot = (unsigned int)ecg_count0;
            EP_CUDA(cudaMemcpy(h->ecg_slot.p, &slot, sizeof slot, cudaMemcpyHostToDevice));
        }
        set_error(bar.err ? "a grid barrier wait gave up" : "a tensor-core completion wait gave up");
        return EP_ERR_TIMEOUT;
    }
    if (st.nonfinite) {
        set_error("%u node(s) with a non-finite voltage after the step", st.nonfinite);
        return EP_ERR_NAN;
    }
    return EP_OK;
}

int ep_diffusion_half_step(ep_handle *h, int32_t *iters, double *relres) {
    EP_CHECK_ARG(h, "null handle");
    EP_CUDA(cudaSetDevice(h->device));
    int rc;
    if (h->precision == EP_FP64) {
        CGArgs<double> ca;
        fill_cg_args<double>(h, ca);
        rc = half_diffusion<double>(h, ca);
    } else {
        CGArgs<float> ca;
        fill_cg_args<float>(h, ca);
        rc = half_diffusion<float>(h, ca);
    }
    if (rc) return rc;
    double last[2];
    EP_CUDA(cudaMemcpyAsync(last, h->cg_last.p, sizeof last, cudaMemcpyDeviceToHost, h->stream));
    EP_CUDA(cudaStreamSynchronize(h->stream));
    GridBarrier bar;
    EP_CUDA(cudaMemcpy(&bar, h->bar.p, sizeof bar, cudaMemcpyDeviceToHost));
    if (iters) *iters = (int32_t)last[0];
    if (relres) *relres = last[1];
    if (bar.err) {
        int rc2 = reset_barriers(h);
        if (rc2) return rc2;
        set_error("a grid barrier wait gave up");
        return EP_ERR_TIMEOUT;
    }
    return EP_OK;
}

// IEEE float -> bfloat16, round to nearest even (NaN kept quiet)
static unsigned short to_bf16(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7fffffffu) > 0x7f800000u) return (unsigned short)((u >> 16) | 0x40u);
    const uint32_t r = 0x7fffu + ((u >> 16) & 1u);
    return (unsigned short)((u + r) >> 16);
}

// BF16 weight images + FP32 side block for the tensor-core kernel
static int pack_surrogate(const ep_surrogate_desc *d, std::vector<unsigned short> &img, SurrogateAux &aux) {
    EP_CHECK_ARG(d && d->params, "null surrogate descriptor");
    if (d->n_in != SG_NF || d->n_hidden != SG_H || d->n_hidden_layers != 3 || d->n_out != SG_NY) {
        set_error("surrogate shape %d-%dx%d-%d unsupported (the kernel is %d-%dx3-%d)", d->n_in, d->n_hidden,
                  d->n_hidden_layers, d->n_out, SG_NF, SG_H, SG_NY);
        return EP_ERR_UNSUPPORTED;
    }
    EP_CHECK_ARG(d->in_mean && d->in_std && d->out_mean && d->out_std && d->env_lo && d->env_hi,
                 "normalisation and envelope arrays are required");
    img.assign(SG_WTOT, 0);
    std::memset(&aux, 0, sizeof aux);
    const float *p = d->params;
    const int dims[5] = {SG_NF, SG_H, SG_H, SG_H, SG_NY};
    const int Kpad[4] = {SG_KIN, SG_H, SG_H, SG_H};
    const int base[4] = {0, SG_W1, SG_W1 + SG_W2, SG_W1 + SG_W2 + SG_W3};
    float *bias[4] = {aux.b1, aux.b2, aux.b3, aux.b4};
    size_t off = 0;
    for (int l = 0; l < 4; l++) {
        const int nout = dims[l + 1], nin = dims[l];
        for (int r = 0; r < nout; r++)
            for (int k = 0; k < nin; k++)
                img[base[l] + core_offset(r, k, Kpad[l])] = to_bf16(p[off + (size_t)r * nin + k]);
        off += (size_t)nout * nin;
        for (int r = 0; r < nout; r++) bias[l][r] = p[off + r];
        off += nout;
    }
    for (int k = 0; k < SG_KIN; k++) {
        const bool used = k < SG_NF;
        aux.in_mean[k] = used ? d->in_mean[k] : 0.f;
        aux.in_rstd[k] = used && d->in_std[k] > 0.f ? 1.f / d->in_std[k] : 0.f;
        aux.env_lo[k] = used ? d->env_lo[k] : -3.0e38f;
        aux.env_hi[k] = used ? d->env_hi[k] : 3.0e38f;
    }
    for (int j = 0; j < SG_NOUT; j++) {
        aux.out_mean[j] = j < SG_NY ? d->out_mean[j] : 0.f;
        aux.out_std[j] = j < SG_NY ? d->out_std[j] : 0.f;
        aux.out_scale[j] = (j < SG_NY && d->out_scale) ? d->out_scale[j] : 0.f;
        aux.out_lo[j] = (j < SG_NY && d->out_lo) ? d->out_lo[j] : -3.0e38f;
        aux.out_hi[j] = (j < SG_NY && d->out_hi) ? d->out_hi[j] : 3.0e38f;
        EP_CHECK_ARG(aux.out_scale[j] >= 0.f, "out_scale must be >= 0");
    }
    aux.nah_max = d->nah_max;
    aux.log_mask = d->log_mask & ((1u << SG_NF) - 1u) & ~1u;   // V stays linear
    EP_CHECK_ARG(d->v_update == 0 || d->v_update == 2, "v_update must be 0 or 2");
    aux.v_update = d->v_update;
    // outputs the update reads: the six Newton concentrations (stored states
    // Ki 1, Nai 2, Cai 3, Cass 10, CaSR 17, R' 18) in the hybrid form
    aux.out_mask = d->v_update == 2 ? ((1u << 1) | (1u << 2) | (1u << 3) | (1u << 10) | (1u << 17) | (1u << 18))
                                    : ((1u << SG_NY) - 1u);
    EP_CHECK_ARG(d->hybrid_substeps >= 0 && d->hybrid_substeps <= kMaxSub, "hybrid_substeps out of range");
    aux.hyb_sub = d->hybrid_substeps;
    return EP_OK;
}

int ep_set_surrogate(ep_handle *h, const ep_surrogate_desc *d) {
    EP_CHECK_ARG(h, "null handle");
    EP_CHECK_ARG(h->precision == EP_SURROGATE, "the handle was not created with EP_SURROGATE");
    EP_CUDA(cudaSetDevice(h->device));
    drop_graph(h);
    std::vector<unsigned short> img;
    SurrogateAux aux;
    int rc = pack_surrogate(d, img, aux);
    if (rc) return rc;
    EP_CUDA(cudaStreamSynchronize(h->stream));
    if ((rc = upload_raw(h->sg_wimg, img.data(), img.size()))) return rc;
    if ((rc = upload_raw(h->sg_aux, &aux, 1))) return rc;
    if (!h->sg_list.p) {
        if ((rc = h->sg_list.alloc(sizeof(int) * (size_t)h->pitch))) return rc;
        if ((rc = h->sg_count.alloc(sizeof(int)))) return rc;
        if ((rc = h->sg_err.alloc(sizeof(unsigned int)))) return rc;
    }
    if (aux.v_update == 2 && !h->sg_pred.p) {
        if ((rc = h->sg_pred.alloc(sizeof(float) * 6 * (size_t)h->pitch))) return rc;
        if ((rc = h->sg_take.alloc((size_t)h->pitch))) return rc;
    }
    if (!h->side) {
        int lo = 0, hi = 0;
        EP_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        EP_CUDA(cudaStreamCreateWithPriority(&h->side, cudaStreamNonBlocking, hi));
        EP_CUDA(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
        EP_CUDA(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
    }
    EP_CUDA(cudaMemset(h->sg_err.p, 0, sizeof(unsigned int)));
    h->has_surrogate = 1;
    h->sg_vupdate = aux.v_update;
    return EP_OK;
}

int ep_surrogate_forward(const ep_surrogate_desc *d, int32_t n, const float *X, float *Y) {
    EP_CHECK_ARG(d && X && Y && n > 0, "bad arguments");
    std::vector<unsigned short> img;
    SurrogateAux aux;
    int rc = pack_surrogate(d, img, aux);
    if (rc) return rc;
    DBuf dimg, daux, dx, dy, derr, dstat;
    if ((rc = upload_raw(dimg, img.data(), img.size())) || (rc = upload_raw(daux, &aux, 1)) ||
        (rc = upload_raw(dx, X, (size_t)n * SG_KIN)) || (rc = dy.alloc(sizeof(float) * (size_t)n * SG_NOUT)) ||
        (rc = derr.alloc(sizeof(unsigned int))) || (rc = dstat.alloc(sizeof(DevStatus))))
        return rc;
    EP_CUDA(cudaMemset(derr.p, 0, sizeof(unsigned int)));
    EP_CUDA(cudaMemset(dstat.p, 0, sizeof(DevStatus)));
    SurrogateArgs sa;
    std::memset(&sa, 0, sizeof sa);
    sa.n = n;
    sa.wimg = dimg.as<unsigned short>();
    sa.aux = daux.as<SurrogateAux>();
    sa.rawX = dx.as<float>();
    sa.rawY = dy.as<float>();
    sa.err = derr.as<unsigned int>();
    sa.status = dstat.as<DevStatus>();
    if ((rc = launch_surrogate(sa, 0))) return rc;
    EP_CUDA(cudaDeviceSynchronize());
    unsigned int err = 0;
    EP_CUDA(cudaMemcpy(&err, derr.p, sizeof err, cudaMemcpyDeviceToHost));
    EP_CUDA(cudaMemcpy(Y, dy.p, sizeof(float) * (size_t)n * SG_NOUT, cudaMemcpyDeviceToHost));
    if (err) { set_error("a tensor-core completion wait gave up"); return EP_ERR_TIMEOUT; }
    return EP_OK;
}

int ep_set_profiling(ep_handle *h, int on) {
    EP_CHECK_ARG(h, "null handle");
    h->profile = on ? 1 : 0;
    return EP_OK;
}

int ep_get_launch_config(const ep_handle *h, ep_launch_config *cfg) {
    EP_CHECK_ARG(h && cfg, "null argument");
    cfg->cg_block = h->cg_block;
    cfg->cg_batch = h->cg_batch;
    cfg->cg_variant = h->cg_variant;
    cfg->cg_predict = h->cg_predict;
    cfg->cg_prefetch = h->cg_prefetch;
    cfg->sg_variant = h->sg_variant;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cfg->cg_per_sm = h->cg_grid / std::max(1, nsm);
    cfg->ionic_block = h->ionic_block;
    cfg->ionic_min_ctas = h->ionic_min;
    cfg->graph_steps = h->graph_steps;
    return EP_OK;
}

int ep_set_wait_limits(ep_handle *h, uint32_t grid_polls, uint32_t mbar_polls) {
    EP_CHECK_ARG(h, "null handle");
    EP_CUDA(cudaSetDevice(h->device));
    EP_CUDA(cudaStreamSynchronize(h->stream));
    drop_graph(h);
    h->wait_grid = grid_polls;
    h->wait_mbar = mbar_polls;
    return reset_barriers(h);
}

int ep_test_hold_barrier(ep_handle *h, int32_t extra_arrivals) {
    EP_CHECK_ARG(h, "null handle");
    EP_CHECK_ARG(extra_arrivals >= 0 && extra_arrivals <= 1024, "extra_arrivals must be 0..1024");
    EP_CUDA(cudaSetDevice(h->device));
    EP_CUDA(cudaStreamSynchronize(h->stream));
    drop_graph(h);
    h->bar_extra = (unsigned int)extra_arrivals;
    return EP_OK;
}

int ep_set_launch_config(ep_handle *h, const ep_launch_config *cfg) {
    EP_CHECK_ARG(h && cfg, "null argument");
    EP_CHECK_ARG(cfg->cg_block == 128 || cfg->cg_block == 256 || cfg->cg_block == 512 || cfg->cg_block == 768,
                 "cg_block must be 128, 256, 512 or 768");
    EP_CHECK_ARG(cfg->cg_batch == 4 || cfg->cg_batch == 8 || cfg->cg_batch == 16 || cfg->cg_batch == kStagedBatch,
                 "cg_batch must be 4, 8, 16 or 32 (staged)");
    EP_CHECK_ARG(!(cfg->cg_batch == kStagedBatch && cfg->cg_variant), "cg_batch 32 (staged) needs cg_variant 0");
    EP_CHECK_ARG(cfg->cg_variant == 0 || cfg->cg_variant == 1, "cg_variant must be 0 or 1");
    EP_CHECK_ARG(cfg->cg_predict >= 0 && cfg->cg_predict <= 2, "cg_predict must be 0, 1 or 2");
    EP_CHECK_ARG(!(cfg->cg_predict && cfg->cg_variant), "cg_predict needs cg_variant 0");
    EP_CHECK_ARG(cfg->cg_prefetch >= 0 && cfg->cg_prefetch <= 4, "cg_prefetch must be 0..4");
    EP_CHECK_ARG(cfg->sg_variant == 0 || cfg->sg_variant == 1, "sg_variant must be 0 or 1");
    EP_CHECK_ARG(!(cfg->cg_prefetch && cfg->cg_variant), "cg_prefetch needs cg_variant 0");
    EP_CHECK_ARG(cfg->cg_per_sm >= 0 && cfg->cg_per_sm <= 32, "cg_per_sm out of range");
    EP_CHECK_ARG(cfg->ionic_block == 64 || cfg->ionic_block == 128, "ionic_block must be 64 or 128");
    EP_CHECK_ARG(cfg->ionic_min_ctas == 0 || cfg->ionic_min_ctas == 3 || cfg->ionic_min_ctas == 4,
                 "ionic_min_ctas must be 0, 3 or 4");
    EP_CHECK_ARG(cfg->graph_steps >= 0 && cfg->graph_steps <= 100000, "graph_steps out of range");
    EP_CUDA(cudaSetDevice(h->device));
    EP_CUDA(cudaStreamSynchronize(h->stream));
    drop_graph(h);
    const int ob = h->cg_block, op = h->cg_per_sm, obt = h->cg_batch, ov = h->cg_variant, opf = h->cg_prefetch;
    h->cg_block = cfg->cg_block;
    h->cg_per_sm = cfg->cg_per_sm;
    h->cg_batch = cfg->cg_batch;
    h->cg_variant = cfg->cg_variant;
    h->cg_prefetch = cfg->cg_prefetch;      // the staged kernel's ring depth sizes its launch
    int rc = plan_cg(h);
    if (rc) {
        h->cg_block = ob; h->cg_per_sm = op; h->cg_batch = obt; h->cg_variant = ov; h->cg_prefetch = opf;
        plan_cg(h);
        return rc;
    }
    const size_t vb = (size_t)h->pitch * h->rsize;
    if (cfg->cg_predict && !h->pd0.p) {
        for (DBuf *b : {&h->pd0, &h->pd1, &h->pvin}) {
            if ((rc = b->alloc(vb))) return rc;
            EP_CUDA(cudaMemset(b->p, 0, vb));
        }
    }
    if (cfg->cg_predict == 2 && !h->pq0.p) {
        for (DBuf *b : {&h->pq0, &h->pq1}) {
            if ((rc = b->alloc(vb))) return rc;
            EP_CUDA(cudaMemset(b->p, 0, vb));
        }
    }
    if (cfg->cg_predict != h->cg_predict) {
        if ((rc = reset_predictor(h))) return rc;
        EP_CUDA(cudaStreamSynchronize(h->stream));
    }
    h->cg_predict = cfg->cg_predict;
    h->sg_variant = cfg->sg_variant;
    h->ionic_block = cfg->ionic_block;
    h->ionic_min = cfg->ionic_min_ctas;
    h->graph_steps = cfg->graph_steps;
    return EP_OK;
}

namespace {
// device state that stepping changes, saved and put back around tuning trials
struct Snapshot {
    DBuf V, S, Spk, track, d_step, slot, pd0, pd1, pq0, pq1;
    long long step = 0;
    int ecg_count = 0;
    std::vector<double> ecg_t;
};

int snap_copy(DBuf &dst, const DBuf &src, cudaStream_t s, bool to_snapshot) {
    if (!src.p) return EP_OK;
    if (to_snapshot) {
        int rc = dst.alloc(src.bytes);
        if (rc) return rc;
        EP_CUDA(cudaMemcpyAsync(dst.p, src.p, src.bytes, cudaMemcpyDeviceToDevice, s));
    } else if (dst.p) {
        EP_CUDA(cudaMemcpyAsync((void *)src.p, dst.p, src.bytes, cudaMemcpyDeviceToDevice, s));
    } else {
        EP_CUDA(cudaMemsetAsync((void *)src.p, 0, src.bytes, s));   // allocated after the save: from zero
    }
    return EP_OK;
}

int snapshot(ep_handle *h, Snapshot &sn, bool save) {
    int rc;
    if ((rc = snap_copy(sn.V, h->V, h->stream, save))) return rc;
    if ((rc = snap_copy(sn.S, h->S, h->stream, save))) return rc;
    if ((rc = snap_copy(sn.Spk, h->Spk, h->stream, save))) return rc;
    if ((rc = snap_copy(sn.track, h->track, h->stream, save))) return rc;
    if ((rc = snap_copy(sn.d_step, h->d_step, h->stream, save))) return rc;
    if ((rc = snap_copy(sn.slot, h->ecg_slot, h->stream, save))) return rc;
    if ((rc = snap_copy(sn.pd0, h->pd0, h->stream, save))) return rc;
    if ((rc = snap_copy(sn.pd1, h->pd1, h->stream, save))) return rc;
    if ((rc = snap_copy(sn.pq0, h->pq0, h->stream, save))) return rc;
    if ((rc = snap_copy(sn.pq1, h->pq1, h->stream, save))) return rc;
    if (save) {
        sn.step = h->step; sn.ecg_count = h->ecg_count; sn.ecg_t = h->ecg_t;
    } else {
        h->step = sn.step; h->ecg_count = sn.ecg_count; h->ecg_t = sn.ecg_t;
    }
    EP_CUDA(cudaStreamSynchronize(h->stream));
    return EP_OK;
}
}  // namespace

int ep_autotune(ep_handle *h, int32_t trial_steps, ep_launch_config *best, double *best_ms,
                double *start_ms, int32_t *n_tried) {
    EP_CHECK_ARG(h && trial_steps > 0, "bad arguments");
    EP_CUDA(cudaSetDevice(h->device));
    EP_CUDA(cudaStreamSynchronize(h->stream));
    Snapshot sn;
    int rc = snapshot(h, sn, true);
    if (rc) return rc;
    const int prof = h->profile;
    h->profile = 0;
    int dev = 0, nsm = 148;
    EP_CUDA(cudaGetDevice(&dev));
    EP_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    ep_launch_config cur;
    cur.cg_block = h->cg_block;
    cur.cg_batch = h->cg_batch;
    cur.cg_variant = h->cg_variant;
    cur.cg_predict = h->cg_predict;
    cur.cg_prefetch = h->cg_prefetch;
    cur.sg_variant = h->sg_variant;
    cur.cg_per_sm = h->cg_grid / std::max(1, nsm);
    cur.ionic_block = h->ionic_block;
    cur.ionic_min_ctas = h->ionic_min;
    cur.graph_steps = h->graph_steps;
    int tried = 0;
    // ms per step of one configuration (negative: it could not run)
    auto trial = [&](const ep_launch_config &c) -> double {
        if (ep_set_launch_config(h, &c) != EP_OK) return -1.0;
        ep_step_stats st;
        for (int pass = 0; pass < 2; pass++) {      // the first pass warms up (and captures)
            if (snapshot(h, sn, false) != EP_OK) return -1.0;
            if (ep_step(h, trial_steps, &st) != EP_OK) return -1.0;
        }
        tried++;
        return st.device_ms / trial_steps;
    };
    double t_best = trial(cur);
    const double t_start = t_best;
    ep_launch_config b = cur;
    if (t_best < 0) {
        h->profile = prof;
        snapshot(h, sn, false);
        return EP_ERR_CUDA;
    }
    // coordinate descent: CG shape, then ionic block, then graphs
    // CG: gather width x CTA size x CTAs per SM (all that fit, or half:
    // fewer CTAs make the grid barrier cheaper)
    const ep_launch_config cg0 = b;
    // (the staged kernel: 256 threads, ring depths 1..3 in cg_prefetch)
    for (int nb : {4, 8, 16, kStagedBatch}) {
        for (int blk : {128, 256, 512, 768}) {
            for (int dp : {1, 2, 3}) {
                if (nb != kStagedBatch && dp > 1) break;
                if (nb == kStagedBatch && (blk != 256 || cg0.cg_variant != 0)) break;
                const int pf = nb == kStagedBatch ? dp : cg0.cg_prefetch;
                int maxper = 0;
                if ((h->precision == EP_FP64 ? cg_max_per_sm<double>(blk, &maxper, nb, cg0.cg_variant, dp)
                                             : cg_max_per_sm<float>(blk, &maxper, nb, cg0.cg_variant, dp)))
                    continue;
                maxper = std::min(maxper, 8);
                for (int per : {maxper, maxper / 2}) {
                    if (per < 1 || per * nsm < h->ninst) continue;
                    ep_launch_config c = cg0;
                    c.cg_block = blk; c.cg_per_sm = per; c.cg_batch = nb; c.cg_prefetch = pf;
                    if (c.cg_block == cg0.cg_block && c.cg_per_sm == cg0.cg_per_sm && c.cg_batch == cg0.cg_batch &&
                        c.cg_prefetch == cg0.cg_prefetch)
                        continue;
                    const double t = trial(c);
                    if (t >= 0 && t < t_best) { t_best = t; b = c; }
                }
            }
        }
    }
    {
        ep_launch_config c = b;
        c.cg_variant = 1 - b.cg_variant;
        c.cg_predict = 0;
        c.cg_prefetch = 0;
        const double t = trial(c);
        if (t >= 0 && t < t_best) { t_best = t; b = c; }
    }
    if (b.cg_variant == 0 && h->scheme != EP_SCHEME_EXPLICIT) {
        const ep_launch_config b0 = b;
        for (int pr : {0, 1, 2}) {
            if (pr == b0.cg_predict) continue;
            ep_launch_config c = b0;
            c.cg_predict = pr;
            const double t = trial(c);
            if (t >= 0 && t < t_best) { t_best = t; b = c; }
        }
        const ep_launch_config b1 = b;
        for (int pf : {0, 2}) {
            if (pf == b1.cg_prefetch || b1.cg_batch == kStagedBatch) continue;   // the staged kernel's depth is tuned above
            ep_launch_config c = b1;
            c.cg_prefetch = pf;
            const double t = trial(c);
            if (t >= 0 && t < t_best) { t_best = t; b = c; }
        }
    }
    if (h->has_surrogate) {
        ep_launch_config c = b;
        c.sg_variant = 1 - b.sg_variant;
        const double t = trial(c);
        if (t >= 0 && t < t_best) { t_best = t; b = c; }
    }
    for (int ib : {64, 128}) {
        if (ib == b.ionic_block) continue;
        ep_launch_config c = b;
        c.ionic_block = ib;
        const double t = trial(c);
        if (t >= 0 && t < t_best) { t_best = t; b = c; }
    }
    if (h->precision != EP_FP64) {
        for (int mc : {0, 3, 4}) {
            if (mc == b.ionic_min_ctas) continue;
            ep_launch_config c = b;
            c.ionic_min_ctas = mc;
            const double t = trial(c);
            if (t >= 0 && t < t_best) { t_best = t; b = c; }
        }
    }
    for (int gs : {0, trial_steps}) {
        if (gs == b.graph_steps) continue;
        ep_launch_config c = b;
        c.graph_steps = gs;
        const double t = trial(c);
        if (t >= 0 && t < t_best) { t_best = t; b = c; }
    }
    rc = ep_set_launch_config(h, &b);
    h->profile = prof;
    const int rc2 = snapshot(h, sn, false);
    if (best) *best = b;
    if (best_ms) *best_ms = t_best;
    if (start_ms) *start_ms = t_start;
    if (n_tried) *n_tried = tried;
    return rc ? rc : rc2;
}

int ep_get_time(ep_handle *h, double *t, int64_t *step) {
    EP_CHECK_ARG(h, "null handle");
    if (t) *t = (double)h->step * h->dt;
    if (step) *step = h->step;
    return EP_OK;
}

int ep_get_ecg(ep_handle *h, double *out, int32_t max_samples, int32_t *n_samples, double *t_samples) {
    EP_CHECK_ARG(h && n_samples, "null argument");
    EP_CUDA(cudaSetDevice(h->device));
    EP_CUDA(cudaStreamSynchronize(h->stream));
    const int cnt = std::min(h->ecg_count, std::max(0, max_samples));
    *n_samples = h->ecg_count;
    if (out && cnt > 0 && h->ne > 0)
        EP_CUDA(cudaMemcpy(out, h->ecg_buf.p, sizeof(double) * (size_t)cnt * h->ne, cudaMemcpyDeviceToHost));
    if (t_samples) for (int s = 0; s < cnt; s++) t_samples[s] = h->ecg_t[s];
    return EP_OK;
}

int ep_compute_ecg(ep_handle *h, double *out) {
    EP_CHECK_ARG(h && out, "null argument");
    EP_CHECK_ARG(h->ne > 0, "no electrodes set");
    EP_CUDA(cudaSetDevice(h->device));
    DBuf tmp;
    int rc = tmp.alloc(sizeof(double) * h->ne);
    if (rc) return rc;
    if (h->precision == EP_FP64)
        rc = launch_ecg<double>(h->n, h->ne, h->W.as<double>(), h->pitch, h->V.as<double>(),
                                h->ecg_partial.as<double>(), h->ecg_counter.as<unsigned int>(),
                                tmp.as<double>(), h->ecg_grid, h->stream);
    else
        rc = launch_ecg<float>(h->n, h->ne, h->W.as<float>(), h->pitch, h->V.as<float>(),
                               h->ecg_partial.as<double>(), h->ecg_counter.as<unsigned int>(),
                               tmp.as<double>(), h->ecg_grid, h->stream);
    if (rc) return rc;
    EP_CUDA(cudaMemcpyAsync(out, tmp.p, sizeof(double) * h->ne, cudaMemcpyDeviceToHost, h->stream));
    EP_CUDA(cudaStreamSynchronize(h->stream));
    return EP_OK;
}

// ---- offline pseudo-ECG (ComputeECG) ----
struct ep_ecg {
    int device = 0, n = 0, ne = 0, grid = 1;
    cudaStream_t stream = nullptr;
    DBuf W, V, out, partial, counter;
    int cap_frames = 0;
    ~ep_ecg() { if (stream) cudaStreamDestroy(stream); }
};

int ep_ecg_create(const ep_mesh_desc *mesh, const ep_cables_desc *cables, int32_t ne, const double *xyz,
                  const double *D_ecg, int device, ep_ecg **out) {
    EP_CHECK_ARG(mesh && out, "null argument");
    *out = nullptr;
    EP_CHECK_ARG(mesh->n_nodes > 0 && mesh->xyz && (mesh->n_tets == 0 || mesh->tets), "bad mesh");
    EP_CHECK_ARG(ne >= 1 && ne <= 16 && xyz, "1..16 electrodes");
    const int n = mesh->n_nodes;
    std::vector<int> tl((size_t)mesh->n_tets * 4);
    for (size_t e = 0; e < tl.size(); e++) {
        const int v = mesh->tets[e] - (mesh->one_based ? 1 : 0);
        EP_CHECK_ARG(v >= 0 && v < n, "tet node id out of range");
        tl[e] = v;
    }
    HostCables hc;
    CableStore cs;
    int rc = host_cables(cables, n, hc, cs);
    if (rc) return rc;
    hc.radius = kEcgCableRadius;                 // ComputeECG.cc:75, whatever the run's radius
    // ComputeECG.cc:88 hard-codes D; NULL keeps it
    const double Dref[3] = {1e-3, 5e-4, 2.5e-4};
    const double *D = D_ecg ? D_ecg : Dref;
    std::vector<double> Wh;
    ecg_weights(n, mesh->xyz, mesh->n_tets, tl.data(), mesh->fibers, D, ne, xyz, Wh, hc.nb ? &hc : nullptr);
    std::unique_ptr<ep_ecg> e(new ep_ecg());
    e->device = device;
    EP_CUDA(cudaSetDevice(device));
    EP_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    e->n = n;
    e->ne = ne;
    if ((rc = e->W.alloc(sizeof(double) * Wh.size()))) return rc;
    EP_CUDA(cudaMemcpy(e->W.p, Wh.data(), sizeof(double) * Wh.size(), cudaMemcpyHostToDevice));
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    e->grid = std::max(1, std::min(nsm * 4, div_up(n, 256)));
    if ((rc = e->partial.alloc(sizeof(double) * 16 * (size_t)e->grid))) return rc;
    if ((rc = e->counter.alloc(sizeof(unsigned int)))) return rc;
    EP_CUDA(cudaMemset(e->counter.p, 0, sizeof(unsigned int)));
    *out = e.release();
    return EP_OK;
}

int ep_ecg_eval(ep_ecg *e, int32_t n_frames, const double *V, double *out) {
    EP_CHECK_ARG(e && n_frames >= 0 && (n_frames == 0 || (V && out)), "bad arguments");
    EP_CUDA(cudaSetDevice(e->device));
    // frames go up in chunks of at most ~256 MB
    const int chunk = std::max(1, (int)std::min<long long>(n_frames, (256ll << 20) / (8ll * e->n)));
    int rc;
    if (chunk > e->cap_frames) {
        if ((rc = e->V.alloc(sizeof(double) * (size_t)chunk * e->n))) return rc;
        if ((rc = e->out.alloc(sizeof(double) * (size_t)chunk * e->ne))) return rc;
        e->cap_frames = chunk;
    }
    for (int f0 = 0; f0 < n_frames; f0 += chunk) {
        const int nf = std::min(chunk, n_frames - f0);
        EP_CUDA(cudaMemcpyAsync(e->V.p, V + (size_t)f0 * e->n, sizeof(double) * (size_t)nf * e->n,
                                cudaMemcpyHostToDevice, e->stream));
        for (int f = 0; f < nf; f++) {
            rc = launch_ecg<double>(e->n, e->ne, e->W.as<double>(), e->n, e->V.as<double>() + (size_t)f * e->n,
                                    e->partial.as<double>(), e->counter.as<unsigned int>(),
                                    e->out.as<double>() + (size_t)f * e->ne, e->grid, e->stream);
            if (rc) return rc;
        }
        EP_CUDA(cudaMemcpyAsync(out + (size_t)f0 * e->ne, e->out.p, sizeof(double) * (size_t)nf * e->ne,
                                cudaMemcpyDeviceToHost, e->stream));
        EP_CUDA(cudaStreamSynchronize(e->stream));
    }
    return EP_OK;
}

void ep_ecg_destroy(ep_ecg *e) {
    if (!e) return;
    cudaSetDevice(e->device);
    delete e;
}

int ep_get_activation(ep_handle *h, double *t_act, double *apd90) {
    EP_CHECK_ARG(h, "null handle");
    EP_CUDA(cudaSetDevice(h->device));
    EP_CUDA(cudaStreamSynchronize(h->stream));
    std::vector<Track> tr(h->n);
    EP_CUDA(cudaMemcpy(tr.data(), h->track.p, sizeof(Track) * h->n, cudaMemcpyDeviceToHost));
    for (int i = 0; i < h->n; i++) {
        if (t_act) t_act[i] = tr[i].t_act;
        if (apd90) apd90[i] = (tr[i].t_act >= 0.f && tr[i].t_rep >= 0.f) ? (double)tr[i].t_rep - tr[i].t_act : -1.0;
    }
    return EP_OK;
}

int ep_write_output(ep_handle *h, double t, const char *dir) {
    EP_CHECK_ARG(h && dir, "null argument");
    std::vector<double> v(h->n);
    int rc = ep_get_voltage(h, v.data());
    if (rc) return rc;
    const std::string name = out_name(dir, "Voltage", t);
    FILE *f = fopen(name.c_str(), "wb");
    if (!f) { set_error("cannot create %s", name.c_str()); return EP_ERR_IO; }
    const size_t w = fwrite(v.data(), sizeof(double), v.size(), f);
    fclose(f);
    if (w != v.size()) { set_error("short write %s", name.c_str()); return EP_ERR_IO; }
    return EP_OK;
}

// nVar of node i in the restart file: its own model's state count
static int node_nvar(const ep_handle *h, int i) {
    return (h->mixed && h->is_purk[i]) ? ep_model_nstate(EP_PURKINJE) : h->nstate;
}

int ep_write_restart(ep_handle *h, double t, const char *dir) {
    EP_CHECK_ARG(h && dir, "null argument");
    const int w = h->nstate_api;
    std::vector<double> s((size_t)h->n * w);
    int rc = ep_get_states(h, s.data());
    if (rc) return rc;
    const std::string name = out_name(dir, "InterVariables", t);
    FILE *f = fopen(name.c_str(), "wb");
    if (!f) { set_error("cannot create %s", name.c_str()); return EP_ERR_IO; }
    bool ok = true;
    for (int i = 0; i < h->n && ok; i++) {
        const int nv = node_nvar(h, i);
        ok = fwrite(&nv, sizeof(int), 1, f) == 1 &&
             fwrite(&s[(size_t)i * w], sizeof(double), nv, f) == (size_t)nv;
    }
    fclose(f);
    if (!ok) { set_error("short write %s", name.c_str()); return EP_ERR_IO; }
    return EP_OK;
}

int ep_read_restart(ep_handle *h, double t, const char *dir) {
    EP_CHECK_ARG(h && dir, "null argument");
    const std::string vn = out_name(dir, "Voltage", t), sn = out_name(dir, "InterVariables", t);
    FILE *fv = fopen(vn.c_str(), "rb");
    if (!fv) { set_error("cannot open %s", vn.c_str()); return EP_ERR_IO; }
    std::vector<double> v(h->n);
    const size_t got = fread(v.data(), sizeof(double), h->n, fv);
    fclose(fv);
    if (got != (size_t)h->n) { set_error("truncated %s", vn.c_str()); return EP_ERR_IO; }
    FILE *fs = fopen(sn.c_str(), "rb");
    if (!fs) { set_error("cannot open %s", sn.c_str()); return EP_ERR_IO; }
    const int w = h->nstate_api;
    std::vector<double> s((size_t)h->n * w, 0.0);
    for (int i = 0; i < h->n; i++) {
        int nv = 0;
        if (fread(&nv, sizeof(int), 1, fs) != 1 || nv != node_nvar(h, i) ||
            fread(&s[(size_t)i * w], sizeof(double), nv, fs) != (size_t)nv) {
            fclose(fs);
            set_error("truncated or mismatched %s at node %d", sn.c_str(), i);
            return EP_ERR_IO;
        }
    }
    fclose(fs);
    int rc = ep_set_states(h, s.data());
    if (rc) return rc;
    rc = ep_set_voltage(h, v.data());
    if (rc) return rc;
    h->step = (long long)(t / h->dt);   // count = long(simtime/dt), EPSimulator.cc:499
    EP_CUDA(cudaMemcpy(h->d_step.p, &h->step, sizeof(long long), cudaMemcpyHostToDevice));
    return EP_OK;
}

// Independent cells through the ionic kernel: one Compute_Ion call per cell
// returning dV/dt (dvdt != NULL, V unchanged), or a whole ionic phase of
// sub-steps with the V update (dvdt == NULL, V advanced in place).
static int ionic_batch(const ep_model_desc *md, int32_t precision, int32_t n, double dt,
                       double ionic_dt, double Cm, double *V, const double *istim, double *states,
                       double *dvdt) {
    EP_CHECK_ARG(md && V && states && n > 0, "bad arguments");
    EP_CHECK_ARG(precision == EP_FP64 || precision == EP_FP32, "unsupported precision");
    const int nst = ep_model_nstate(md->model);
    EP_CHECK_ARG(nst > 0, "unknown model");
    const int ntypes = md->n_types > 0 ? md->n_types : 1;
    EP_CHECK_ARG(ntypes <= kMaxTypes, "too many parameter sets");
    ep_handle h;
    cudaGetDevice(&h.device);
    h.n = n; h.pitch = (n + 31) / 32 * 32; h.model = md->model; h.precision = precision;
    h.nstate = nst; h.ns = is_lr(md->model) ? 7 : nst - 1; h.ntypes = ntypes;
    h.dt = dt; h.nsub = 1; h.sub_dt[0] = dt; h.Cm = Cm;
    if (!dvdt) {
        h.nsub = substeps(dt, ionic_dt > 0 ? ionic_dt : dt, h.sub_dt);
        EP_CHECK_ARG(h.nsub > 0, "more than 64 ionic sub-steps");
    }
    h.Xi = md->user_xi > 0 ? md->user_xi : model_xi(md->model);
    h.tt.newton_cap = md->newton_cap > 0 ? md->newton_cap : 100;
    h.tt.jac_true = md->tt_jacobian == EP_TT_JAC_TRUE ? 1 : 0;
    h.tt.fp32_scaled_tol = precision == EP_FP64 ? 0 : 1;
    h.tt.newton_tol = md->newton_tol > 0 ? md->newton_tol : 1e-6;
    h.mh_abs = md->mh_abs_mode ? 1 : 0;
    const int nc = ep_model_nconst(md->model);
    std::vector<double> consts((size_t)ntypes * nc);
    for (int t = 0; t < ntypes; t++) {
        if (md->type_consts) std::memcpy(&consts[(size_t)t * nc], md->type_consts + (size_t)t * nc, sizeof(double) * nc);
        else default_consts(md->model, t, &consts[(size_t)t * nc]);
    }
    std::vector<double> S((size_t)h.ns * h.pitch, 0.0), Vv(h.pitch, 0.0), ist(h.pitch, 0.0);
    for (int i = 0; i < n; i++) {
        const double *s = states + (size_t)i * nst;
        if (is_lr(md->model)) for (int k = 0; k < 7; k++) S[(size_t)k * h.pitch + i] = s[k];
        else for (int k = 0; k < h.ns; k++) S[(size_t)k * h.pitch + i] = s[k + 1];
        Vv[i] = V[i];
        ist[i] = istim ? istim[i] : 0.0;
    }
    // the stimulus enters as one window per node covering step 0
    std::vector<int> head(n), next(n, -1);
    std::vector<long long> on(n, 0), off(n, 1);
    for (int i = 0; i < n; i++) head[i] = i;
    DBuf dvd;
    int rc;
    EP_CUDA(cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking));
    auto run = [&](auto tag) -> int {
        using R = decltype(tag);
        int r2;
        if ((r2 = upload<R>(h.S, S)) || (r2 = upload<R>(h.V, Vv)) || (r2 = upload<R>(h.consts, consts)) ||
            (r2 = upload<R>(h.stim_amp, ist)))
            return r2;
        if ((r2 = upload_raw(h.stim_head, head.data(), n)) || (r2 = upload_raw(h.stim_next, next.data(), n)) ||
            (r2 = upload_raw(h.stim_on, on.data(), n)) || (r2 = upload_raw(h.stim_off, off.data(), n)))
            return r2;
        h.nstim = n;
        if (md->node_type && (r2 = upload_raw(h.type, md->node_type, (size_t)n))) return r2;
        if (md->node_gks_scale) {
            std::vector<double> g(md->node_gks_scale, md->node_gks_scale + n);
            if ((r2 = upload<R>(h.gks, g))) return r2;
        }
        if (md->model == EP_LUORUDYWITHGATE) {
            std::vector<double> tab;
            lr_gate_table(tab);
            if ((r2 = upload<R>(h.lr_table, tab))) return r2;
        }
        if ((r2 = h.status.alloc(sizeof(DevStatus))) || (r2 = h.d_step.alloc(sizeof(long long))) ||
            (r2 = dvd.alloc(sizeof(R) * h.pitch)))
            return r2;
        EP_CUDA(cudaMemset(h.status.p, 0, sizeof(DevStatus)));
        EP_CUDA(cudaMemset(h.d_step.p, 0, sizeof(long long)));
        IonicArgs<R> a;
        fill_ionic_args<R>(&h, a);
        a.track = nullptr;
        a.dvdt_out = dvdt ? dvd.as<R>() : nullptr;
        if ((r2 = launch_ionic<R>(h.model, a, h.stream))) return r2;
        EP_CUDA(cudaStreamSynchronize(h.stream));
        std::vector<double> o, so;
        if ((r2 = download<R>(dvdt ? dvd : h.V, o, n, h.stream))) return r2;
        if ((r2 = download<R>(h.S, so, (size_t)h.ns * h.pitch, h.stream))) return r2;
        for (int i = 0; i < n; i++) {
            if (dvdt) dvdt[i] = o[i];
            else V[i] = o[i];
            double *s = states + (size_t)i * nst;
            if (is_lr(md->model)) {
                for (int k = 0; k < 7; k++) s[k] = so[(size_t)k * h.pitch + i];
                s[7] = V[i];
            } else {
                s[0] = V[i];
                for (int k = 0; k < h.ns; k++) s[k + 1] = so[(size_t)k * h.pitch + i];
            }
        }
        return EP_OK;
    };
    rc = precision == EP_FP64 ? run(double(0)) : run(float(0));
    cudaStreamDestroy(h.stream);
    h.stream = nullptr;
    return rc;
}

int ep_ionic_step(const ep_model_desc *md, int32_t precision, int32_t n, double dt, double Cm,
                  const double *V, const double *istim, double *states, double *dvdt) {
    EP_CHECK_ARG(V && dvdt, "null V or dvdt");
    std::vector<double> v(V, V + (n > 0 ? n : 0));
    return ionic_batch(md, precision, n, dt, 0.0, Cm, v.data(), istim, states, dvdt);
}

int ep_ionic_phase(const ep_model_desc *md, int32_t precision, int32_t n, double dt,
                   double ionic_dt, double Cm, double *V, const double *istim, double *states) {
    return ionic_batch(md, precision, n, dt, ionic_dt, Cm, V, istim, states, nullptr);
}

}  // extern "C"
