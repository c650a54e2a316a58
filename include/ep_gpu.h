/*
 * ep_gpu.h -- C ABI of the B200-native voomEP monodomain time step.
 *
 * One handle = one tissue instance resident on one GPU (device memory owned
 * by the handle, one CUDA stream per handle, not thread-safe per handle).
 * The caller owns every host buffer.  Every entry point returns EP_OK (0)
 * or a negative EP_ERR_* code; nothing calls exit().  ep_last_error()
 * returns a thread-local message for the last failure.
 *
 * Each entry point names the reference interface it replaces (paths inside
 * wsklug/UCLA_CMG, voomEP/src/...).
 */
#ifndef EP_GPU_H
#define EP_GPU_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define EP_ABI_VERSION 3

/* ---- status codes ---- */
#define EP_OK               0
#define EP_ERR_ARG         -1   /* bad argument / size */
#define EP_ERR_CUDA        -2   /* CUDA runtime error */
#define EP_ERR_NOMEM       -3
#define EP_ERR_MESH        -4   /* degenerate or inverted element */
#define EP_ERR_CG          -5   /* a CG solve reached cg_maxit */
#define EP_ERR_NEWTON      -6   /* a Newton solve reached its cap */
#define EP_ERR_NAN         -7   /* non-finite voltage after a step (ep_step; the
                                   step's stats are filled, stats->nonfinite > 0) */
#define EP_ERR_TIMEOUT     -8   /* an in-kernel wait gave up */
#define EP_ERR_UNSUPPORTED -9
#define EP_ERR_IO          -10

/* ---- cell models: the reference enum CellModelType
 *      (Body/CardiacBody.h:57) ---- */
#define EP_LUORUDY          0
#define EP_LUORUDYWITHGATE  1
#define EP_TUSSCHER         2
#define EP_MAHAJAN          3
#define EP_MAHAJAN_FAIL     4
/* not in CellModelType: the Purkinje cell CardiacBody::New gives every .purk
 * node (Body/CardiacBody.cc:982-1101; IonicModel/Purkinje.cc): at plugin
 * level (ep_ionic_step, ep_ionic_phase) and on the .purk nodes of mixed
 * tissues (ep_create_mixed); ep_create rejects it as a tissue model. */
#define EP_PURKINJE         5

/* ---- arithmetic of the ionic update and the SpMV ---- */
#define EP_FP64       0   /* everything FP64 */
#define EP_FP32       1   /* ionic + SpMV FP32; CG dots, residual, ECG sums FP64 */
#define EP_SURROGATE  2   /* EP_FP32 with the learned ionic step (ep_set_surrogate) */

/* ---- ten Tusscher Newton Jacobian layout ---- */
#define EP_TT_JAC_REFERENCE 0  /* the reference hands J[j*6+i]=df_j/dx_i to the
                                  column-major dgesv_ (Tusscher.cc:173,181) and so
                                  solves with J^T; kept for parity */
#define EP_TT_JAC_TRUE      1  /* Newton with J itself */

typedef struct ep_handle ep_handle;

/* Geometry: Mesh::New + TetMesh::Compute (Mesh/Mesh.cc:142-483,
 * Mesh/TetMesh.cc:9-71) and CardiacBody::setDiffusion / setNodalCapacitance
 * (Body/CardiacBody.h:252-260). */
typedef struct ep_mesh_desc {
    int32_t n_nodes;
    const double *xyz;          /* 3 * n_nodes, cm */
    int32_t n_tets;
    const int32_t *tets;        /* 4 * n_tets */
    int32_t one_based;          /* 1: ids as in the reference .ele files */
    const double *fibers;       /* 9 * n_tets (f, s, n) or NULL: isotropic D[0] */
    double D[3];                /* cm^2/ms along f, s, n */
    double Cm;                  /* uF/cm^2 (the reference uses 1.0) */
} ep_mesh_desc;

/* Cell models: CardiacBody::New + SetUp*Parameters
 * (Body/CardiacBody.cc:975-1101, IonicModel/SetUpIonicConstants.h). */
typedef struct ep_model_desc {
    int32_t model;              /* EP_TUSSCHER, ... */
    int32_t n_types;            /* parameter sets (<= 256) */
    const double *type_consts;  /* n_types * ep_model_nconst(model), or NULL:
                                   the reference constants for type 0..n_types-1 */
    const uint8_t *node_type;   /* n_nodes or NULL (all type 0) */
    const double *node_gks_scale; /* n_nodes or NULL: G_Ks multiplier (TT) */
    double user_xi;             /* > 0: CardiacBody user Xi; else the model's own */
    int32_t newton_cap;         /* TT Newton cap (0: 100) */
    int32_t tt_jacobian;        /* EP_TT_JAC_* */
    int32_t mh_abs_mode;        /* Mahajan sub-step trigger: 0 int |dV/dt| (as
                                   compiled), 1 double fabs (Mahajan.cc:611) */
    const double *initial_states; /* n_nodes * nstate node-major, or NULL */
    double newton_tol;          /* TT, batch entry points only (0: 1e-6, the
                                   reference's); handles take it from the solver */
} ep_model_desc;

/* Time stepping: EPSolver::New/setSolveTime/setIonicTimeStep
 * (Solvers/EPSolver.h:190-223) and EP_CrankNicholson (Solvers/
 * EP_CrankNicholson.cc:5-156). */
typedef struct ep_solver_desc {
    double dt;                  /* global step (ms) */
    double ionic_dt;            /* ionic sub-step (ms) */
    double cg_tol;              /* relative to ||r0|| (reference 1e-7) */
    int32_t cg_maxit;           /* reference 1000 */
    double smoothing_alpha;     /* SMOOTHING key, 0 = off */
    int32_t precision;          /* EP_FP64 / EP_FP32 / EP_SURROGATE */
    double newton_tol;          /* TT, 0: 1e-6 (the reference's absolute
                                   tolerance; FP32 scales it by max(|x|,1)) */
    int32_t ecg_every;          /* steps between pseudo-ECG samples (0 off) */
    double act_threshold;       /* mV; activation = upward crossing (0: -40) */
    int32_t scheme;             /* EP_SCHEME_*: the EPSolver Method (EPSolver.h:
                                   Method; the reference driver always takes
                                   CRANKNICKOLSON) */
    double diffusion_dt;        /* explicit scheme: diffusion sub-step (0: 0.05,
                                   EP_ExplicitSolver.h:68) */
} ep_solver_desc;

/* ---- operator-splitting schemes (EPSolver::New, Solvers/EPSolver.cc) ---- */
#define EP_SCHEME_CN        0  /* EP_CrankNicholson: D/2 by CN (CG to 1e-7),
                                  ionic sub-steps of IONICDT */
#define EP_SCHEME_BE        1  /* EP_BackwardEuler: (C_L + dt/2 K) V' = C_L V
                                  (CG to 1e-10), adaptive ionic strides, again */
#define EP_SCHEME_EXPLICIT  2  /* EP_ExplicitSolver: forward-Euler diffusion
                                  sub-steps V += h (-K V) / C_L over dt/2,
                                  adaptive ionic strides, again */

typedef struct ep_step_stats {
    int64_t steps;              /* steps done by this call */
    int64_t cg_iters;           /* CG iterations, both half-steps, all steps */
    int32_t cg_max_iters;       /* most iterations one solve took */
    int32_t cg_failures;        /* solves that hit cg_maxit */
    int64_t newton_iters;       /* TT Newton iterations, all nodes and sub-steps */
    int32_t newton_cap_hits;
    int32_t nonfinite;          /* nodes with a non-finite V after the call */
    int64_t fallback_nodes;     /* surrogate: node-steps run on the plain model */
    double device_ms;           /* CUDA-event time of the call's GPU work */
    int32_t timeouts;
    /* per-kernel CUDA-event times, filled when profiling is on */
    double cg_ms;               /* both CN half diffusion steps */
    double ionic_ms;            /* ionic phase */
    double ecg_ms;              /* pseudo-ECG samples */
    int64_t launches;           /* kernels launched by the call */
} ep_step_stats;

/* ---- life cycle ---- */
int  ep_version(void);
const char *ep_last_error(void);
/* stored-state count of a model (the reference getInternalParameters nData:
 * TT 19, Mahajan 26, LR 8) and its constant count */
int  ep_model_nstate(int model);
int  ep_model_nconst(int model);
/* reference default constants of parameter set `type` (SetUp*Parameters) */
int  ep_model_default_consts(int model, int type, double *out);

/* EPSolver::New(..., CRANKNICKOLSON) with CardiacBody::New and Compute()
 * (Solvers/EPSolver.cc:339-362, Body/CardiacBody.cc:78-187,975-1101):
 * assembles K, M and C_L in FP64 on the host, uploads the CN operators. */
int  ep_create(const ep_mesh_desc *mesh, const ep_model_desc *model,
               const ep_solver_desc *solver, int device, ep_handle **out);
void ep_destroy(ep_handle *h);
int  ep_num_nodes(const ep_handle *h);
int  ep_num_states(const ep_handle *h);

/* EPSolver::InitializeVoltage (Solvers/EPSolver.h:214-223) */
int  ep_set_voltage(ep_handle *h, const double *V);
/* the voltage field EPSolver::WriteOutput writes (Solvers/EPSolver.cc:116-152) */
int  ep_get_voltage(ep_handle *h, double *V);
/* CardiacBody::getStateVariables / setStateVariables
 * (Body/CardiacBody.cc:438-463): n_nodes * nstate, node-major */
int  ep_get_states(ep_handle *h, double *out);
int  ep_set_states(ep_handle *h, const double *in);
/* the resting voltage the cell models report (CardiacBody::getInitialVoltage,
 * Body/CardiacBody.h:299-307): Mahajan State[0]; TT and LR report 0 there
 * (IonicModel.h:42), which is what this returns for them too. */
int  ep_get_model_voltage(ep_handle *h, double *V);

/* Nodal stimuli: CardiacBody::setStimulusCurrent(nodeSet, istim) switched
 * on/off by the EPSimulator schedule (Body/CardiacBody.cc:315-324,
 * EPSimulator.cc:483-570).  Entry k stimulates node_ids[k] with amp[k]
 * [uA/cm^3] for steps long(t_on/dt) <= step < long(t_off/dt).  Replaces
 * the previous table.  A node may appear in several entries; at a given
 * step the entry whose window covers the step and starts latest wins. */
int  ep_set_stimulus(ep_handle *h, int32_t n, const int32_t *node_ids,
                     const double *t_on, const double *t_off, const double *amp);

/* Pseudo-ECG electrodes (ComputeECG.h:30-189 with the D of the run, or
 * D_ecg[3] when non-NULL -- the reference post-processor hard-codes
 * {1e-3, 5e-4, 2.5e-4}, ComputeECG.cc:88). */
int  ep_set_electrodes(ep_handle *h, int32_t n, const double *xyz, const double *D_ecg);
/* samples taken so far: out[s * n_electrodes + k], s < *n_samples */
int  ep_get_ecg(ep_handle *h, double *out, int32_t max_samples, int32_t *n_samples,
                double *t_samples);
/* ECG of the current voltage field, computed now */
int  ep_compute_ecg(ep_handle *h, double *out);

/* Advance n_steps global steps: EP_CrankNicholson::Solve per step
 * (half diffusion step, ionic sub-steps, half diffusion step), stimulus
 * windows, ECG sampling and activation tracking on the device. */
int  ep_step(ep_handle *h, int32_t n_steps, ep_step_stats *stats);
/* Record CUDA events around every kernel of ep_step (per-kernel times in
 * ep_step_stats); adds a few microseconds per step.  No reference
 * counterpart (the reference has no timers). */
int  ep_set_profiling(ep_handle *h, int on);
/* One Crank-Nicolson half diffusion step on the current voltage, nothing
 * else: V <- A^-1 (B V) (EP_CrankNicholson.cc:99-104).  *iters receives the
 * CG iteration count, *relres the final ||r||/||r0||. */
int  ep_diffusion_half_step(ep_handle *h, int32_t *iters, double *relres);
/* Allocation-free Crank-Nicolson half diffusion step.  No counterpart in
 * the reference: it exists for callers that own all device memory and may
 * not allocate any (solvers embedded in another code's memory pool, time
 * loops that must not call cudaMalloc after start-up, C/Fortran hosts that
 * pass only their own buffers).  The caller passes, in device memory, the
 * SELL-32 operators (slice_ptr: nslices+1 element offsets, col, Aval = A,
 * Bval = B, dinv = 1/diag(A); values FP64 or FP32 per `precision`) and x,
 * which holds V on entry and A^-1 B V on return; stream may be NULL.  The
 * working vectors live in one static device array of this library sized for
 * at most 262144 rows (about 8.2 MB, held by every GPU that loads the
 * library until exit); larger n returns EP_ERR_ARG.  Every call shares that
 * array, so calls that overlap on the GPU race: serialise them.  Each call
 * looks up the array's address on the current device.  The call waits on
 * `stream` for its results before it returns; on a stream in capture mode
 * it returns EP_ERR_ARG without touching the stream. */
int  ep_cn_half_step_noalloc(int32_t precision, int32_t n, int32_t nslices,
                             const int32_t *slice_ptr, const int32_t *col,
                             const void *Aval, const void *Bval, const void *dinv,
                             void *x, double cg_tol, int32_t cg_maxit, void *stream,
                             int32_t *iters, double *relres);
/* simulated time (ms) and step count */
int  ep_get_time(ep_handle *h, double *t, int64_t *step);

/* Batches of independent tissue instances.  No counterpart in the
 * reference (one EPSimulator per mesh).  n_inst meshes of any sizes, each
 * with its own parameter sets, stimuli, activation trackers and CG stop
 * test, advanced together: every kernel of a step covers all instances at
 * once, and the persistent CG launch gives each instance its own group of
 * CTAs (in proportion to its rows) with its own grid barrier, so the
 * instances never wait for one another inside a solve.  Nodes (and every
 * per-node array of the API) are the instances' nodes concatenated in
 * order; node_offset[k] is where instance k starts.  All instances share
 * the cell model, C_m and the solver settings; the type tables are
 * concatenated (at most 256 parameter sets in all).  The pseudo-ECG is not
 * available on a batch handle. */
int  ep_batch_create(int32_t n_inst, const ep_mesh_desc *meshes, const ep_model_desc *models,
                     const ep_solver_desc *solver, int device, ep_handle **out);
/* n_inst, node_offset[n_inst + 1] and cta_offset[n_inst + 1] (CG groups);
 * any pointer may be NULL */
int  ep_batch_layout(const ep_handle *h, int32_t *n_inst, int32_t *node_offset, int32_t *cta_offset);
/* per instance: CG iterations and ||r||/||r0|| of the latest solve */
int  ep_batch_cg_last(ep_handle *h, int32_t *iters, double *relres);
/* The CTA-group split itself (host only, for tests): every instance at
 * least one CTA, the remaining grid - n_inst in proportion to its SELL-32
 * slices by largest remainder.  inst_blk[n_inst + 1]. */
int  ep_batch_plan(int32_t n_inst, const int32_t *inst_row, int32_t grid, int32_t *inst_blk);

/* 2-node Purkinje cables of a mixed (MIX3D) mesh: the beam elements of
 * MixedMesh3D::Compute (Mesh/MixedMesh3D.cc:62-108) with the Purkinje
 * diffusion of CardiacBody::Compute (Body/CardiacBody.cc:100-187).  The
 * reference scales Gauss weights that sum to 2 by the cable length, so a
 * cable carries twice the mass and stiffness of a cylinder of that radius;
 * kept.  A node listed in the .angle file (Mesh.cc:403-416) overrides the
 * direction and length of the cable that starts there, and in the reference
 * the override, once met, stays on for every later cable (angle_sticky = 1;
 * 0 applies it to its own cable only). */
typedef struct ep_cables_desc {
    int32_t n_bars;
    const int32_t *bars;        /* 2 * n_bars node ids, in .ele order */
    int32_t one_based;          /* 1: ids as in the .ele / .angle files */
    const double *fibers;       /* 9 * n_bars (f, s, n) or NULL: isotropic Dp[0] */
    const uint8_t *lv;          /* n_bars or NULL: 1 = a node of tissue type 11 (DpLeft) */
    double Dp[3], DpLeft[3];    /* PURKINJEDIFFUSION / LVPURKINJEDIFFUSION, cm^2/ms */
    double radius;              /* TWODRADIUS, cm (the driver's default 0.0275) */
    int32_t quad_order;         /* the mesh's quadrature order (0: 2 = two Gauss points) */
    int32_t n_angle;            /* .angle entries */
    const int32_t *angle_nodes; /* n_angle node ids */
    const double *angle;        /* 4 * n_angle: direction (3), length */
    int32_t angle_sticky;
    /* n_bars or NULL: per cable, the index into angle_nodes/angle of the
     * row that overrides it (-1: none), resolved by the caller over the
     * whole .ele order.  The reference switches the override on for ANY
     * element whose first node is listed -- tets included -- and keeps it
     * on (MixedMesh3D.cc:30-34, 78-87), which a bars-only list cannot show;
     * given, angle_sticky is not consulted. */
    const int32_t *bar_angle;
} ep_cables_desc;

/* Mixed tissues: CardiacBody::New on a MIX3D mesh (Body/CardiacBody.cc:
 * 982-1101).  The 2-node cables join the tets in the operators
 * (MixedMesh3D.cc:62-108, CardiacBody.cc:100-187); every node of purk_nodes
 * (the .purk file; ids as mesh->one_based says) carries the Purkinje cell
 * (IonicModel/Purkinje.cc, defaults of SetUpPurkinjeParameters) with its own
 * 21 stored states, constants and Xi, every other node the tissue model of
 * `tissue`, and the shared V starts from each cell's own voltage.  States
 * (ep_get/set_states) come in rows of ep_num_states(h) = max(tissue nstate,
 * 22) values: a Purkinje node's row holds its 22 (V first), a tissue node's
 * its model's, zero-padded; restart files keep each node's own nVar, as the
 * reference writes them (EPSolver.cc:155-176).  The pseudo-ECG integrates
 * over the cables too, as ComputeECG does on a MIX3D mesh (tissue D along
 * each cable's fibres, radius 0.0275 cm).  FP64 and FP32 only. */
int  ep_create_mixed(const ep_mesh_desc *mesh, const struct ep_cables_desc *cables, int32_t n_purk,
                     const int32_t *purk_nodes, const ep_model_desc *tissue, const ep_solver_desc *solver,
                     int device, ep_handle **out);

/* Offline pseudo-ECG of stored voltage fields: the post-processor ComputeECG
 * (Applications/CardiacEP/ComputeECG.cc:26-162 over ComputeECG.h:30-189).
 * ep_ecg_create builds the per-node weights of the mesh once in FP64 on the
 * host -- the tets and, for a MIX3D mesh, the 2-node cables with the radius
 * ComputeECG fixes (0.0275 cm, ComputeECG.cc:75; cables->radius is not
 * used here) and the tissue D along each cable's fibres -- and keeps them on
 * the GPU; D_ecg NULL takes ComputeECG's hard-coded {1e-3, 5e-4, 2.5e-4}
 * (ComputeECG.cc:88).  ep_ecg_eval reduces n_frames voltage fields (host,
 * frame-major, n_nodes each) to out[f * n_electrodes + k], FP64 sums on the
 * device.  At most 16 electrodes. */
typedef struct ep_ecg ep_ecg;
int  ep_ecg_create(const ep_mesh_desc *mesh, const struct ep_cables_desc *cables, int32_t n_electrodes,
                   const double *xyz, const double *D_ecg, int device, ep_ecg **out);
int  ep_ecg_eval(ep_ecg *e, int32_t n_frames, const double *V, double *out);
void ep_ecg_destroy(ep_ecg *e);

/* The FP64 operators ep_create assembles for the solver's scheme, on the
 * host only (no GPU, no device memory): CSR of n_nodes rows, zero-based
 * sorted columns, A and B (CN: C_m M +- dt/4 K; BE: C_L + dt/2 K and C_L;
 * explicit: -K) and the lumped capacitance C_L, with the tets of `mesh`
 * followed by the optional cables (EP_CrankNicholson::Initialize,
 * Solvers/EP_CrankNicholson.cc:5-76, over CardiacBody::Compute).  Call with
 * rowptr == NULL for *nnz, then with rowptr[n+1], col/A/B[nnz], CL[n]. */
int  ep_assemble_operators(const ep_mesh_desc *mesh, const ep_cables_desc *cables,
                           const ep_solver_desc *solver, int64_t *nnz, int32_t *rowptr,
                           int32_t *col, double *A, double *B, double *CL);

/* Launch shape of ep_step (no reference counterpart).  cg_block: threads
 * per CTA of the persistent CG launch (128, 256, 512 or 768); cg_per_sm: its CTAs per
 * SM (0 = as many as are co-resident); ionic_block: threads per CTA of the
 * ionic kernel (64 or 128); graph_steps: 0 launches every kernel from the
 * host, k > 0 replays the steps from an instantiated CUDA graph of k steps
 * (rounded up to a multiple of the ECG interval); ionic_min_ctas: FP32
 * ionic kernel compiled for at least 3 or 4 resident 128-thread CTAs per SM
 * (fewer registers per thread), 0 = the compiler's register choice;
 * cg_batch: SELL columns whose gathers the CG kernel issues together (4 or
 * 8; 8 keeps more loads in flight at a larger register budget; 16: groups of
 * 8 with the next group's index loads issued before the current gathers;
 * 32: staged -- each warp copies its next units of 8 slice columns (column
 * indices and values) into a ring of shared memory with asynchronous copies
 * while it gathers the current one, cg_prefetch units ahead (1..4; 0 = 2),
 * 256 threads per CTA, cg_variant 0 only);
 * cg_variant: 0 the CG recurrences of the reference (two reductions per
 * iteration), 1 the Chronopoulos-Gear recurrences (one reduction per
 * iteration; same iterates in exact arithmetic, rounding-level differences;
 * five more vectors on the device). */
typedef struct ep_launch_config {
    int32_t cg_block, cg_per_sm, ionic_block, graph_steps, ionic_min_ctas, cg_batch, cg_variant;
    int32_t cg_predict;   /* 1: each CG solve starts from V + the previous solve's
                             correction of the same half step; 2: from V + the
                             linear extrapolation of the last two corrections
                             (cg_variant 0 only); the stop test stays relative
                             to B V - A V */
    int32_t cg_prefetch;  /* 0..4: each warp of the CG launch asks L2 for the
                             SELL indices and values of the slice it reads that
                             many slices ahead (cg_variant 0; 0 = off); with
                             cg_batch 32 the units the ring holds in flight
                             (0 = 2) */
    int32_t sg_variant;   /* learned ionic step (EP_SURROGATE): 0 two CTAs per SM,
                             each one tile of 128 nodes at a time; 1 one CTA per SM
                             running four tiles at once in four warpgroups (one
                             copy of the weights); same results */
} ep_launch_config;
/* Bounded in-kernel waits (no reference counterpart: the reference has no
 * device code; its Newton loop has no cap, Tusscher.cc:150).  Every wait of
 * the persistent kernels polls a bounded number of times and then gives up:
 * grid_polls caps one CG grid-barrier wait (polls of ~64 ns sleeps; 0 = the
 * built-in 2^24, seconds), mbar_polls one tensor-core completion wait of
 * the learned step (0 = 2^22).  A wait that runs out makes ep_step return
 * EP_ERR_TIMEOUT (stats->timeouts > 0); the handle's wait state is then
 * reset so it can step again and its clock (step count, ECG samples) is put
 * back to the call's start, but V and the states of that call are not to
 * be trusted (restore them with ep_set_voltage / ep_set_states). */
int  ep_set_wait_limits(ep_handle *h, uint32_t grid_polls, uint32_t mbar_polls);
/* Test hook for the timeout path (no reference counterpart): the CG grid
 * barrier waits for extra_arrivals more CTAs than the launch has, so every
 * wait runs out after its poll limit; 0 restores normal operation. */
int  ep_test_hold_barrier(ep_handle *h, int32_t extra_arrivals);
int  ep_get_launch_config(const ep_handle *h, ep_launch_config *cfg);
int  ep_set_launch_config(ep_handle *h, const ep_launch_config *cfg);
/* Autotuner: times trial_steps steps (after one untimed pass) for the
 * current shape, then by coordinate descent over the CG gather width, block
 * size and CTAs per SM, the CG variant, predictor and L2 prefetch, the ionic
 * block size and register budget, and graph replay, keeps the fastest and
 * sets it.  The simulation state (V, states, trackers, step, ECG samples) is put
 * back afterwards.  best_ms / start_ms: device ms per step of the chosen and
 * of the starting shape; any output may be NULL. */
int  ep_autotune(ep_handle *h, int32_t trial_steps, ep_launch_config *best, double *best_ms,
                 double *start_ms, int32_t *n_tried);

/* Activation time (first upward crossing of act_threshold, ms, -1 if none)
 * and APD90 (ms, -1 if not repolarised) per node. */
int  ep_get_activation(ep_handle *h, double *t_act, double *apd90);

/* Reference output formats (Solvers/EPSolver.cc:116-211), rank 00:
 * Voltage_time_%08.2f.00 (raw FP64 V) and InterVariables_time_%08.2f.00
 * (per node int nVar + nVar FP64). */
int  ep_write_output(ep_handle *h, double t, const char *dir);
int  ep_write_restart(ep_handle *h, double t, const char *dir);
int  ep_read_restart(ep_handle *h, double t, const char *dir);

/* Plugin-level entry: IonicModel::Compute_Ion for a batch of independent
 * cells (IonicModel/IonicModel.h:34-35, Body/CardiacBody.cc:405-435).
 * states: n * nstate node-major, updated in place; dvdt[i] receives the
 * return value.  Host buffers; runs on the current CUDA device. */
int  ep_ionic_step(const ep_model_desc *model, int32_t precision, int32_t n,
                   double dt, double Cm, const double *V, const double *istim,
                   double *states, double *dvdt);

/* The ionic phase of one global step for independent cells: the sub-step
 * loop of EP_CrankNicholson::Solve (Solvers/EP_CrankNicholson.cc:114-143)
 * with Compute_Ion and V += h dV/dt per sub-step, no diffusion.  V and
 * states (node-major) are advanced in place.  This is the map the learned
 * ionic step replaces; it also produces its training targets. */
int  ep_ionic_phase(const ep_model_desc *model, int32_t precision, int32_t n, double dt,
                    double ionic_dt, double Cm, double *V, const double *istim, double *states);

/* ---------------- learned ionic step (no reference counterpart) ----------
 * A tanh MLP trained on the plain model's ionic phase.  Training runs on
 * the GPU through ep_mlp_* (FP32 master weights, the project's own forward,
 * backward and Adam kernels); deployment (ep_set_surrogate) converts the
 * weights to BF16 for the tcgen05 tensor-core inference kernel. */
typedef struct ep_mlp ep_mlp;
/* dims[0..n_layers]: input, hidden..., output widths; hidden layers use tanh */
int  ep_mlp_create(int32_t n_layers, const int32_t *dims, uint64_t seed, int device, ep_mlp **out);
void ep_mlp_destroy(ep_mlp *m);
int  ep_mlp_num_params(const ep_mlp *m);
/* parameters flattened as W1 (dims[1] x dims[0], row-major), b1, W2, b2, ... */
int  ep_mlp_get_params(ep_mlp *m, float *out);
int  ep_mlp_set_params(ep_mlp *m, const float *in);
/* device pointers, row-major FP32: X [batch x dims[0]], Y [batch x dims[L]] */
int  ep_mlp_forward(ep_mlp *m, const float *X, float *Y, int32_t batch, void *stream);
/* loss = mean_i sum_j w_j (f(X_i)_j - Y_ij)^2 (w = 1 when NULL); gradients
 * are accumulated into the trainer and optionally copied to grad_host */
int  ep_mlp_loss_grad(ep_mlp *m, const float *X, const float *Y, const float *w_out_host,
                      int32_t batch, double *loss, float *grad_host, void *stream);
int  ep_mlp_adam_step(ep_mlp *m, float lr, float beta1, float beta2, float eps);

/* Deployment of a trained network as the ionic phase of EP_SURROGATE
 * handles (ten Tusscher only).  Inputs per node, in this order: V, the 18
 * stored states, I_stim [uA/uF], G_Ks (with the node scale), G_to, the
 * s-gate variant; outputs: the changes of V and the 18 states over one
 * global step.  A node whose inputs leave the box [env_lo, env_hi], whose
 * fast sodium gate product m^3 h exceeds nah_max, or which is being
 * stimulated, runs the plain FP32 model for that step instead. */
typedef struct ep_surrogate_desc {
    int32_t n_in, n_hidden, n_hidden_layers, n_out;
    const float *params;         /* ep_mlp flattening (FP32; converted to BF16) */
    const float *in_mean, *in_std, *out_mean, *out_std;
    const float *env_lo, *env_hi;   /* box in the transformed feature space */
    float nah_max;
    uint32_t log_mask;              /* bit k: feature k enters as log(x); for the
                                       states (k < 19) the output is then the
                                       change of log(x) and x' = x exp(out) */
    const float *out_scale;         /* NULL, or per output s_j > 0: the network
                                       predicts asinh(delta_j / s_j) (0: delta_j) */
    const float *out_lo, *out_hi;   /* NULL, or the accepted range of each
                                       de-normalised output (before the asinh
                                       inverse); a node whose used outputs leave
                                       it runs the plain model */
    int32_t hybrid_substeps;        /* v_update 2: gate/V sub-steps per global
                                       step (0: the handle's ionic sub-steps) */
    int32_t v_update;               /* 0: V and every state from the network;
                                       2: only the six Newton concentrations
                                       (Ki, Nai, Cai, Cass, CaSR, R') come from
                                       the network (interpolated over the
                                       sub-steps); the gates and V follow the
                                       reference sub-step scheme */
} ep_surrogate_desc;
int  ep_set_surrogate(ep_handle *h, const ep_surrogate_desc *d);
/* The deployed network alone on host buffers (tests): X [n x 32] already
 * normalised inputs (23 used), Y [n x 32] raw outputs before
 * de-normalisation (19 used); runs the same tensor-core kernel. */
int  ep_surrogate_forward(const ep_surrogate_desc *d, int32_t n, const float *X, float *Y);

#ifdef __cplusplus
}
#endif
#endif
