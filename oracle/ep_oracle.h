/*
 * ep_oracle.h -- CPU oracle for the voomEP monodomain time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C, FP64 restatement of the
 * reference algorithm used as the checker for the CUDA path and as the timed
 * CPU baseline.  The product (ucla_cmg_b200/) never links, loads or calls it.
 *
 * Reference files followed (paths inside wsklug/UCLA_CMG):
 *   ten Tusscher 2006  voomEP/src/IonicModel/Tusscher.{h,cc}
 *   Mahajan 2008       voomEP/src/IonicModel/Mahajan.{h,cc}, Mahajan_fail.cc
 *   Luo-Rudy           voomEP/src/IonicModel/LR.{h,cc}, LRGateTable.h
 *   constants          voomEP/src/IonicModel/SetUpIonicConstants.h
 *   P1 tet geometry    voomEP/src/Mesh/TetMesh.cc:9-71, Shape/ShapeTet4CP.cc:4-16,
 *                      Quadrature/TetQuadrature.cc:16-30, VoomMath/VoomMath.cc:17-52
 *   K_e, M_e, C_L      voomEP/src/Body/CardiacBody.cc:32-187, 348-391
 *   CN split step      voomEP/src/Solvers/EP_CrankNicholson.cc:5-156
 *   stimulus schedule  voomEP/src/Applications/CardiacEP/EPSimulator.cc:483-596
 *   pseudo-ECG         voomEP/src/Applications/CardiacEP/ComputeECG.h:30-189
 */
#ifndef EP_ORACLE_H
#define EP_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* model ids follow the reference enum CellModelType (Body/CardiacBody.h:57) */
enum { EPO_LUORUDY = 0, EPO_LUORUDYWITHGATE = 1, EPO_TUSSCHER = 2,
       EPO_MAHAJAN = 3, EPO_MAHAJAN_FAIL = 4,
       /* not in CellModelType: CardiacBody::New gives every .purk node a
        * Purkinje cell (CardiacBody.cc:982-1101) */
       EPO_PURKINJE = 5 };

#define EPO_TT_NSTATE 19
#define EPO_TT_NCONST 54   /* 53 reference constants + [53] s-gate variant (0 epi, 1 endo) */
#define EPO_MH_NSTATE 26
#define EPO_MH_NCONST 35
#define EPO_LR_NSTATE 8
#define EPO_PK_NSTATE 22
#define EPO_PK_NCONST 63

/* ---------------- cell models (single cell, in place) ---------------- */
void   epo_tt_constants(double *c);                  /* SetUpTusscherParameters */
void   epo_tt_initial_state(double *s);              /* Tusscher.h:51-69 */
/* One Compute_Ion call.  newton_cap <= 0 means "no cap" like the
 * reference.  jac_true = 0 solves with the finite-difference Jacobian laid
 * out the way the reference hands it to the column-major dgesv_ (i.e. with
 * its transpose, Tusscher.cc:173,181); jac_true = 1 solves with J itself.
 * Returns dV/dt; *iters receives the Newton iteration count. */
double epo_tt_compute_ion(double *s, const double *c, double Xi, double Cm,
                          double dt, double V, double istim, int newton_cap,
                          int jac_true, int *iters);

void   epo_mh_constants(double *c, int pos, int failing);   /* SetUpMahajan[_fail]Parameters */
void   epo_mh_initial_state(double *s, int pos);            /* Mahajan.cc:25-160 */
/* abs_mode 0: the substep trigger uses int-truncated |dV/dt| (the reference
 * as compiled without <math.h>'s double abs), 1: double fabs. */
double epo_mh_compute_ion(double *s, const double *c, double Xi, double Cm,
                          double dt, double V, double istim, int abs_mode,
                          int *substepped);

void   epo_lr_initial_state(double *s);              /* LR.cc:18-59 */
void   epo_lr_params(double v, double *tab);         /* LR.cc:102-183 (14 entries) */
/* gate table: 290001 x 14 doubles (LRGateTable.h:66-108); caller frees */
double *epo_lr_gate_table(void);
double epo_lr_compute_ion(double *s, const double *table, double Xi_unused,
                          double Cm, double dt, double V, double istim);

void   epo_pk_constants(double *c);                  /* SetUpPurkinjeParameters */
void   epo_pk_initial_state(double *s);              /* Purkinje.h:43-51 */
/* One Compute_Ion call of the Purkinje cell (Xi: the model's 2500 or the
 * user's); *substepped = 1 when the ten dt/10 forward-Euler steps ran. */
double epo_pk_compute_ion(double *s, const double *c, double Xi, double dt,
                          double V, double istim, int *substepped);

/* ---------------- a population of cells ---------------- */
typedef struct epo_cells {
    int model, n, nstate, nconst;
    double *state;        /* n * nstate, row-major (node-major) */
    double *consts;       /* ntypes * nconst */
    int ntypes;
    const uint8_t *type;  /* n or NULL (type 0) -- not owned */
    double *gks_scale;    /* n or NULL: per-node G_Ks multiplier (TT) */
    double *alg12;        /* n (TT only) */
    double *lr_table;     /* LUORUDYWITHGATE */
    double Xi;            /* the model's own surface-to-volume ratio */
    double user_Xi;       /* CardiacBody::setSurfaceToVolumeRatio value ... */
    int user_xi;          /* ... used when non-zero (LR ignores it, LR.cc:98) */
    int newton_cap;       /* TT */
    int tt_jac_true;      /* TT: 0 reference (transposed) Jacobian, 1 true J */
    int mh_abs_mode;      /* Mahajan */
    long long newton_total, newton_max, substep_count;
} epo_cells;

epo_cells *epo_cells_create(int model, int n, const uint8_t *type, int ntypes,
                            const double *type_consts);
void epo_cells_destroy(epo_cells *c);
/* dvdt[i] = Compute_Ion(...) for every node (OpenMP over nodes) */
void epo_cells_compute_ion(epo_cells *c, double Cm, double dt, const double *V,
                           const double *istim, double *dvdt);
/* resting / initial V as the cells report it: Mahajan State[0]; TT and LR
 * State[0] resp. -85.423 / initial  (see the H1 note in epo_initial_voltage) */
void epo_cells_initial_voltage(const epo_cells *c, double *V);

/* ---------------- FEM (P1 tets, 4-point rule) ---------------- */
typedef struct epo_csr {
    int n, nnz;
    int *rowptr, *col;      /* sorted columns */
    double *A, *B;          /* A = Cm*M + s*K, B = Cm*M - s*K; s = dt/4 (+smoothing) */
    double *M;              /* consistent mass (no Cm), same pattern */
    double *K;              /* stiffness (includes Cm), same pattern */
    double *CL;             /* lumped capacitance, n */
} epo_csr;

/* tets: m*4 zero-based node ids.  fibers: m*9 (f,s,n) or NULL (isotropic
 * D[0]).  Returns 0 on success, <0 on a degenerate element. */
int  epo_assemble(int n, const double *xyz, int m, const int *tets,
                  const double *fibers, const double D[3], double Cm,
                  double dt_diff, double smoothing_alpha, epo_csr *out);
/* 2-node Purkinje cables of a mixed (MIX3D) mesh, MixedMesh3D.cc:62-108 and
 * CardiacBody.cc:100-187.  The quadrature weight is w_q * pi r^2 * length
 * with Gauss weights summing to 2 on [-1, 1], as in the reference: a cable's
 * mass and stiffness are twice those of a cylinder of that radius.  A node
 * listed in the .angle file overrides the direction and length of a cable
 * starting there; in the reference the override, once met, stays on for
 * every later cable (a flag that is never reset, MixedMesh3D.cc:14-34):
 * orient_sticky = 1 keeps that, 0 applies it to its own cable only. */
typedef struct epo_cables {
    int nb;
    const int *bars;             /* nb * 2 zero-based node ids */
    const double *fibers;        /* nb * 9 (f, s, n) or NULL: isotropic Dp[0] */
    const uint8_t *lv;           /* nb or NULL: 1 = a node of tissue type 11 (DpLeft) */
    double Dp[3], DpLeft[3];     /* setPurkinjeDiffusion / ...InLV */
    double radius;               /* Mesh::setRadius (TWODRADIUS, 0.0275 cm) */
    int quad_order;              /* the mesh's order; 2 -> two Gauss points */
    const uint8_t *orient_has;   /* n or NULL */
    const double *orient;        /* n * 4: direction, length */
    int orient_sticky;
    /* nb or NULL: per cable, the node whose .angle row overrides it (-1:
     * none), resolved by the caller over the whole element order (the
     * reference also lets a tet whose first node is listed switch the
     * override on, MixedMesh3D.cc:30-34); when given, orient_has and
     * orient_sticky are not consulted */
    const int *bar_orient_node;
} epo_cables;

/* tets then cables, summed in that element order; tets alone == epo_assemble */
int  epo_assemble_mixed(int n, const double *xyz, int m, const int *tets,
                        const double *fibers, const double D[3], const epo_cables *cables,
                        double Cm, double dt_diff, double smoothing_alpha, epo_csr *out);
void epo_csr_free(epo_csr *a);
/* y = A x for one of the value arrays */
void epo_spmv(const epo_csr *a, const double *vals, const double *x, double *y);
/* Jacobi-PCG (k Jacobi sweeps as preconditioner), x holds x0 on entry.
 * Stops when ||r_k||_2 <= tol * ||r_0||_2 (recursive residual).  Returns
 * the iteration count, or -1 when maxit was reached. */
int  epo_pcg(const epo_csr *a, const double *vals, const double *b, double *x,
             double tol, int maxit, int jacobi_steps, double *relres);

/* ---------------- pseudo-ECG ---------------- */
/* Reference element form (ComputeECG.h:30-189): ECG_k for one V field. */
void epo_ecg_elementwise(int n, const double *xyz, int m, const int *tets,
                         const double *fibers, const double D[3], int ne,
                         const double *electrodes, const double *V, double *ecg);
/* Per-node weights W (ne * n) with ECG_k = sum_i W[k*n+i] V[i]. */
/* the 2-node cables' share of the weights, added to W (ComputeECG on a MIX3D
 * mesh; radius from cables->radius, ComputeECG uses 0.0275) */
int  epo_ecg_weights_cables(int n, const double *xyz, const epo_cables *cables, const double D[3], int ne,
                            const double *electrodes, double *W);
void epo_ecg_weights(int n, const double *xyz, int m, const int *tets,
                     const double *fibers, const double D[3], int ne,
                     const double *electrodes, double *W);

/* ---------------- the split time step ---------------- */
/* ionic phase callback: dvdt = Compute_Ion(V, istim) for all nodes */
typedef void (*epo_ionic_fn)(void *ctx, double Cm, double dt, const double *V,
                             const double *istim, double *dvdt);

/* one node's Compute_Ion (returns dV/dt, advances that node's state) */
typedef double (*epo_ionic_node_fn)(void *ctx, int i, double Cm, double dt, double V, double istim);

#define EPO_SCHEME_CN 0
#define EPO_SCHEME_BE 1
#define EPO_SCHEME_EXPLICIT 2

typedef struct epo_sim {
    epo_csr *csr;
    int n;
    double dt, ionic_dt, Cm;
    double cg_tol; int cg_maxit, jacobi_steps;
    double *V, *istim, *dvdt, *b, *ici;
    epo_ionic_fn ionic; void *ionic_ctx;
    /* sub-step schedule of one ionic phase (EP_CrankNicholson.cc:115-143) */
    int nsub; double sub_dt[64];
    long long cg_iters_total; int cg_fail;
    long step;
    /* scheme (EPSolver Method) and what the non-CN schemes need */
    int scheme;
    epo_ionic_node_fn ionic_node;
    double *A_be, *B_be;    /* BE: C_L + dt/2 K and diag C_L on the csr pattern */
    int nex; double ex_h[4096];   /* explicit: diffusion sub-steps of one half */
} epo_sim;

void epo_sim_init(epo_sim *s, epo_csr *csr, double dt, double ionic_dt,
                  double Cm, double cg_tol, int cg_maxit, int jacobi_steps,
                  epo_ionic_fn fn, void *ctx);
void epo_sim_free(epo_sim *s);
/* EP_CrankNicholson::Solve: D/2 - ionic sub-steps - D/2 (or the scheme set
 * below) */
void epo_sim_step(epo_sim *s);
/* switch to EP_BackwardEuler (EP_BackwardEuler.cc:5-91) or EP_ExplicitSolver
 * (EP_ExplicitSolver.cc:4-118, diffusion sub-step dt_diff); both advance the
 * cells by CardiacBody::getVoltageFromIonicCurrent (CardiacBody.cc:819-904)
 * through the per-node callback */
void epo_sim_set_scheme(epo_sim *s, int scheme, double dt_diff, epo_ionic_node_fn fn, void *ctx);
double epo_cells_ionic_node_cb(void *ctx, int i, double Cm, double dt, double V, double istim);
void epo_cells_ionic_cb(void *ctx, double Cm, double dt, const double *V,
                        const double *istim, double *dvdt);

/* Two cell populations in one tissue (CardiacBody::New, CardiacBody.cc:982-1101:
 * the .purk nodes carry the Purkinje cell, every other node the tissue model):
 * each population is a compact set of cells behind its own callback (the
 * restatement's epo_cells_ionic_cb or the reference objects'), the mixed
 * callback gathers V and istim per population, calls both and scatters
 * dV/dt back. */
typedef struct epo_mixed {
    int n, nt, np;
    int *tmap, *pmap;                 /* compact index -> node */
    epo_ionic_fn tfn, pfn;
    void *tctx, *pctx;
    double *buf;                      /* 3 * n scratch */
} epo_mixed;
/* is_purk[n]: 1 on Purkinje nodes.  The populations must hold nt and np
 * cells in increasing node order. */
void epo_mixed_init(epo_mixed *m, int n, const uint8_t *is_purk, epo_ionic_fn tfn, void *tctx,
                    epo_ionic_fn pfn, void *pctx);
void epo_mixed_free(epo_mixed *m);
void epo_mixed_ionic_cb(void *ctx, double Cm, double dt, const double *V, const double *istim, double *dvdt);

/* Stimulus schedule of EPSimulator.cc:483-570 for nodal stimuli: given
 * stimuli (t_start, t_stop) in list order, the step indices at which each
 * one starts/stops under the reference's single-pointer logic.  A value of
 * -1 means "never".  */
void epo_stim_schedule(int nstim, const double *t_start, const double *t_stop,
                       double dt, long nsteps, long *start_step, long *stop_step);
/* Number of steps the reference time loop runs: while (t < T) t += dt. */
long epo_num_steps(double dt, double T);

void epo_set_threads(int n);
int  epo_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
