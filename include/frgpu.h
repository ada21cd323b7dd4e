/* frgpu.h -- C ABI of the B200 flux-reconstruction residual + Runge-Kutta path.
 *
 * Drop-in boundary for FlurryPP's solver entry points (include/solver.hpp:137-153
 * of the reference):
 *
 *   solver::calcResidual(int step)              -> frg_calc_residual
 *   solver::timeStepA(int step, double RKval)   -> frg_time_step_a
 *   solver::timeStepB(int step)                 -> frg_time_step_b
 *   solver::copyUspts_U0 / copyU0_Uspts         -> frg_copy_u_to_u0 / frg_copy_u0_to_u
 *   solver::calcDt()                            -> frg_calc_dt
 *   solver::update()  (+ the main loop's iter++,
 *                      src/flurry.cpp:50-53)     -> frg_update
 *   ele::getNormResidual summed as writeResidual
 *     does (src/ele.cpp:1882, src/output.cpp:846) -> frg_residual_norm
 *   oper::setupOperators(eType, order, ...)      -> built inside frg_create;
 *     (src/operators.cpp:13)                        frg_get_operator returns the
 *                                                   dense matrices for checking
 *   ele::setInitialCondition (src/ele.cpp:683)   -> frg_set_initial_condition
 *
 * Conventions
 *   - Plain pointers and sizes only.  Every function returns an frg_status.
 *   - Host arrays use the reference's layouts: solution [point][element][field]
 *     (src/solver.cpp:65-107).  Device arrays are [field][point][element].
 *   - Host buffers are caller-owned; device buffers are owned by the handle.
 *   - A handle is not thread-safe: one CUDA stream, calls serialised by the
 *     caller.  The reference is single-threaded too (makefile:14).
 *   - Errors replace the reference's fatalError()+exit(1) (include/error.hpp:10):
 *     the call returns a code and frg_last_error() gives the message.
 *   - There is no CPU fallback: without a usable CUDA device frg_create fails.
 */
#ifndef FRGPU_H
#define FRGPU_H
#ifdef __cplusplus
extern "C" {
#endif

typedef enum frg_status {
  FRG_OK = 0,
  FRG_ERR_ARG = 1,         /* invalid argument or unsupported configuration */
  FRG_ERR_CUDA = 2,        /* CUDA runtime error, or no device */
  FRG_ERR_NAN = 3,         /* NaN in the solution (src/output.cpp:833-841) */
  FRG_ERR_NEG_JAC = 4,     /* negative Jacobian (src/solver.cpp:1283) */
  FRG_ERR_DT = 5,          /* dt < 1e-13 (src/output.cpp:823-824) */
  FRG_ERR_TIMEOUT = 6,     /* a bounded device wait gave up */
  FRG_ERR_MESH = 7         /* unmatched face, self-neighbour, bad element */
} frg_status;

typedef enum frg_precision {
  FRG_FP64 = 0,  /* everything in FP64 */
  FRG_MIXED = 1  /* FP32 operators/fluxes/traces/metrics; FP64 Riemann pressure,
                    RK accumulation and norms */
} frg_precision;

/* Input parameters, same names and meaning as the reference's `input`
 * (include/input.hpp:63-234, src/input.cpp:214-554). Viscous runs take the
 * already non-dimensionalised values (input::nonDimensionalize). */
typedef struct frg_params {
  int nDims;       /* 2 or 3 */
  int order;       /* P: 1..5 in 2D, 1..4 in 3D */
  int equation;    /* 0 advection, 1 Euler / Navier-Stokes */
  int viscous;     /* 0 / 1 */
  int riemannType; /* 0 Rusanov, 1 Roe (2D) */
  int vcjhScheme;  /* 0 DG, 1 SD, 2 HU, 3 C+ */
  int timeType;    /* 0 FE, 2 RK2, 4 RK44, 5 RK44 (Jameson form) */
  int dtType;      /* 0 fixed, 1 global CFL, 2 local CFL */
  double dt, CFL;
  double gamma;
  double advectVx, advectVy, advectVz, lambda, diffD;
  double rhoBound, uBound, vBound, wBound, pBound;
  double mu_inf, prandtl, c_sth, rt_inf;
  int fixVis;
  double penFact, tau;
  double TWall, RGas, uWall, vWall, wWall;
  int precision; /* frg_precision */
} frg_params;

/* Mesh: element node coordinates and the vertex ids used to pair faces.
 * xv  [nEles][nNodes][nDims], node order of the reference's shape functions
 *     (src/funcs.cpp:126, :183): quads of any Lagrange order (4, 9, 16, ...
 *     nodes), 8-node hexahedra.
 * c2v [nEles][nCorners] (4 or 8); periodic images share one id.
 * bc  [nEles][nFacesPerEle] (4 or 6): reference BC_TYPE of a face on a
 *     boundary (include/global.hpp:63-78), -1 for faces paired by c2v. */
typedef struct frg_mesh {
  int nEles;
  int nNodes;
  const double *xv;
  const int *c2v;
  const int *bc;
} frg_mesh;

typedef struct frg_solver frg_solver;

/* which arrays frg_download / frg_upload address */
typedef enum frg_array {
  FRG_U_SPTS = 0,   /* [nSpts][nEles][nFields] current solution (solver::U_spts) */
  FRG_U0 = 1,       /* [nSpts][nEles][nFields] (solver::U0) */
  FRG_DIVF = 2,     /* [nSpts][nEles][nFields] divF_spts[stage] (reference space) */
  FRG_U_FPTS = 3,   /* [nFpts][nEles][nFields] traces of the current solution */
  FRG_POS_SPTS = 4, /* [nSpts][nEles][nDims] physical solution-point positions */
  FRG_WAVESP = 5,   /* [nEles][nFpts] wave speeds kept for calcDt */
  FRG_DETJAC = 6,   /* [nSpts][nEles] */
  FRG_ELE_DT = 7    /* [nEles] per-element CFL dt of the last calcDt */
} frg_array;

const char *frg_last_error(void);
const char *frg_version(void);

/* Creates a solver on the current CUDA device: connectivity, metrics,
 * operators (setup work, host side), device buffers.  Rejects configurations
 * the reference rejects (3D Roe: src/face.cpp:362; negative Jacobian). */
frg_status frg_create(const frg_params *params, const frg_mesh *mesh, frg_solver **out);

/* Host-only inspection of the set-up (no device needed): the metrics and
 * connectivity frg_create would build, in the reference's layouts.
 * which: 0 pos_spts [nS][nE][d], 1 JGinv_spts [d][nS][nE][d], 2 detJac_spts
 * [nS][nE], 3 norm_fpts [nF][nE][d], 4 dA_fpts [nF][nE], 5 face table
 * [nFaces][6] (eL, locF_L, eR, locF_R, relRot, bc) written as doubles.
 * With out == NULL only *count is set. */
frg_status frg_inspect_geometry(const frg_params *params, const frg_mesh *mesh, int which, double *out,
                                long *count);
frg_status frg_destroy(frg_solver *s);

/* Recomputes the element metrics on the device for new node coordinates of
 * the same mesh (same elements, node count, connectivity and boundary
 * conditions): solver::updateTransforms -> calcTransforms
 * (src/solver.cpp:1358-1363, :1227-1356) and the solution-point positions
 * of setPosSptsFpts (:904-951), for a mesh whose nodes moved.  xv is a host
 * array [nEles][nNodes][nDims] as in frg_mesh.  The metrics are bitwise the
 * ones frg_create builds on the host for those nodes.  The next CFL dt
 * recomputes the wave speeds with the new normals.  Grid-velocity (ALE)
 * flux terms are not part of this path.  FRG_ERR_NEG_JAC, with the solver's
 * metrics unchanged, when a solution point has a negative Jacobian.
 * Synchronises the solver's stream. */
frg_status frg_update_geometry(frg_solver *s, const double *xv);

/* The reference's ParaView file, which is also its restart file
 * (writeParaview, src/output.cpp:103-391): <dataFileName>_<iter, 9 digits>.vtu
 * with "<!-- TIME t -->" / "<!-- ITER n -->" header comments and per element
 * one piece of (P+3)^d plot points (the 1D points {-1, solution points, +1}
 * in a tensor grid, x fastest) carrying Density, Velocity and Pressure (the
 * primitives interpolated from the solution points; Density alone for
 * advection), their coordinates and the linear sub-cells, in ASCII with 16
 * significant digits.  The reference writes 3D only; 2D files use the layout
 * its restart reader expects, with a zero third velocity component.
 * frg_write_paraview writes the solver's state at its iteration and time. */
frg_status frg_write_paraview(frg_solver *s, const char *dataFileName);
/* solver::readRestartFile / ele::restart (src/solver.cpp:1420-1482,
 * src/ele.cpp:1451-1880): reads <dataFileName>_<restartIter, 9 digits>.vtu,
 * takes the solution points' primitives (the interior plot points), converts
 * them to conservative variables, interpolates from the file's order when it
 * differs, and sets the state, the time (TIME comment) and iter = initIter =
 * restartIter.  As in ele::restart (src/ele.cpp:1469-1478), an element the
 * file has no piece for is reported on stdout and set to 100 in every field. */
frg_status frg_read_restart(frg_solver *s, const char *dataFileName, int restartIter);
/* Host-only forms (no device): U is [nSpts][nEles][nFields] as frg_download. */
frg_status frg_write_paraview_host(const frg_params *params, const frg_mesh *mesh, const double *U, double time,
                                   int iter, const char *dataFileName);
frg_status frg_read_restart_host(const frg_params *params, int nEles, const char *dataFileName, int restartIter,
                                 double *U, double *time);

/* geo::readGmsh (src/geo.cpp:448-769) with the boundary matching of
 * geo::processConn3D (src/geo.cpp:169-193): a Gmsh v2 ASCII file into the
 * frg_mesh arrays.  meshBounds maps the file's physical names to boundary
 * conditions as the reference's "mesh_bound <name> <bc>" input lines do:
 * "<name> <bc>" pairs separated by ';' or newlines (case-insensitive), one of
 * them "<volume name> fluid".  Volumes: 8-node hexahedra (Gmsh type 5) in 3D,
 * 4-, 9- or 16-node quads (types 3, 10, 36) in 2D.  A face no other element
 * shares takes the condition of the first boundary (in $PhysicalNames order)
 * whose boundary elements hold all its corners.  With xv, c2v and bc all NULL
 * only the sizes are returned; else xv [nEles][nNodes][nDims], c2v
 * [nEles][4 or 8] (0-based vertex ids) and bc [nEles][4 or 6] are filled. */
frg_status frg_read_gmsh(const char *fileName, const char *meshBounds, int *nDims, int *nEles, int *nNodes,
                         double *xv, int *c2v, int *bc);

frg_status frg_info(const frg_solver *s, int *nSpts, int *nFpts, int *nFields, int *nEles);

/* Dense operator matrices, row-major, as oper::setupOperators builds them:
 * which 0 opp_spts_to_fpts [nF][nS], 1 opp_grad_spts[dim] [nS][nS],
 * 2 opp_extrapolateFn[dim] [nF][nS], 3 opp_correction [nS][nF],
 * 4 opp_correctU[dim] [nS][nF]. */
frg_status frg_get_operator(const frg_solver *s, int which, int dim, double *out);

/* The reference's operator matrices for the device path:
 * oper::setupOperators (src/operators.cpp:13-76) builds them per order; a
 * shim passes them here after frg_create.  E = opp_spts_to_fpts [nF][nS],
 * D = opp_grad_spts [nDims][nS][nS], C = opp_correction [nS][nF], Efn =
 * opp_extrapolateFn [nDims][nF][nS] (may be NULL), row-major.  The device
 * path applies these operators as tensor products of 1D tables (sum
 * factorisation), so the call identifies the matrices: they must be the FR
 * operators, within 1e-13 relative, of one VCJH correction scheme (DG, SD,
 * HU, C+) at the solver's order on the reference's Gauss points; the solver
 * then uses that scheme (a change takes effect from the next call).
 * FRG_ERR_ARG when they are not, or when the order differs. */
frg_status frg_set_operators(frg_solver *s, int order, const double *E, const double *D, const double *C,
                             const double *Efn);

/* The operator applications of the `oper` object -- applySptsFpts (which 0),
 * applyGradSpts (1, one dim), applyExtrapolateFn (2, one dim),
 * applyCorrectDivF (3), applyCorrectGradU's parent-space product (4, one
 * dim); src/operators.cpp:1191-1450 -- as batched dense GEMMs on the tensor
 * cores: Y = Op X + beta Y for every field and element.  X and Y are FP32
 * DEVICE arrays [nFields][K or M points][ld] (element index fastest, ld >=
 * nEles a multiple of 4, 16-byte aligned), K/M the operator's input/output
 * point counts as frg_get_operator shapes them; they must be ready on the
 * handle's stream (frg_set_stream).  The products are 3xTF32 split precision
 * with FP32 accumulation (about 1e-6 relative).  The kernel is enqueued on
 * the handle's stream and the call returns without waiting; frg_sync waits
 * and reports a kernel's expired bounded wait (FRG_ERR_TIMEOUT).  Operators
 * wider than 256 points, or needing more than 227 KB of shared memory (3D
 * order 4), are rejected with FRG_ERR_ARG. */
frg_status frg_apply_operator(frg_solver *s, int which, int dim, const float *X, float *Y, int ld, float beta);

frg_status frg_upload(frg_solver *s, int array, const double *host);
frg_status frg_download(frg_solver *s, int array, int stage, double *host);

/* ele::setInitialCondition: icType 0 freestream / Gaussian, 1 isentropic
 * vortex (eps 5) / sine, 2 Liang vortex; 10 Taylor-Green vortex (a0 = Mach);
 * 11 isentropic vortex of strength a0 (eps generalised). */
frg_status frg_set_initial_condition(frg_solver *s, int icType, double a0);

/* solver::calcResidual(step): divF_spts[step] of the current solution. */
frg_status frg_calc_residual(frg_solver *s, int step);
frg_status frg_time_step_a(frg_solver *s, int step, double rkval);
frg_status frg_time_step_b(frg_solver *s, int step);
frg_status frg_copy_u_to_u0(frg_solver *s);
frg_status frg_copy_u0_to_u(frg_solver *s);
/* solver::calcDt: on the first iteration recomputes the wave speeds
 * (ele::calcWaveSpFpts), then dt = min over elements (warp-shuffle reduction). */
frg_status frg_calc_dt(frg_solver *s, double *dt_out);

/* Allocation-free residual.  This entry point has no counterpart in the
 * reference.  It is for callers that must not allocate device memory when
 * they evaluate a residual: code running under a memory manager that owns
 * every device allocation, a real-time loop where cudaMalloc's implicit
 * synchronisation is not allowed, or a host application that pre-plans its
 * whole memory footprint.  It computes divF_spts (solver::calcResidual's
 * result, without touching the handle's wave speeds) of the caller's state
 * `U_dev` into the caller's `divF_dev`, both device arrays laid out
 * [nFields][nSpts][nEles] (element index fastest), on `stream` (NULL: the
 * handle's stream).  The handle only supplies the geometry and operators
 * built by frg_create.
 *
 * The flux-point traces it needs go to a fixed scratch array of 16 MiB in
 * device memory that the library declares statically: every GPU that loads
 * the library keeps it until the process exits.  Meshes whose traces
 * (nFields * nFpts * nEles values, 8 bytes each in FP64 mode, 4 in mixed
 * mode; viscous runs add one or two more arrays of that size for the
 * projected viscous fluxes) exceed 16 MiB are rejected with FRG_ERR_ARG.
 * frg_create does the set-up on its device: it looks up the scratch array's
 * device address (cudaGetSymbolAddress) and loads the kernels this call
 * launches, so the call itself only launches kernels.  On a stream other
 * than the handle's, the call first makes that stream wait (an event the
 * handle owns) for the work pending on the handle's stream, such as an
 * upload or a frg_update_geometry.  All calls share the one scratch array
 * and it keeps the last call's contents; every value a call reads is
 * written by the same call first, so nothing needs clearing.  Calls that
 * overlap on the GPU (different streams, or several handles at once) race on
 * the scratch array: serialise them. */
frg_status frg_calc_residual_noalloc(frg_solver *s, const double *U_dev, double *divF_dev, void *stream);

/* nsteps iterations of the reference main loop body (iter++; update()), as
 * one fused kernel per RK stage replayed from a CUDA graph.  Device-resident:
 * no host transfer.  Checks the NaN / dt flags after the last step. */
frg_status frg_update(frg_solver *s, int nsteps);
/* Same, with the solution in host memory ([spt][ele][field]): upload,
 * nsteps iterations, download, all on the handle's stream with one host
 * synchronisation at the end (pinned U_host keeps both copies asynchronous).
 * U_host receives the state after the last step even when the NaN / dt check
 * fails, as the reference's solution array does. */
frg_status frg_update_host(frg_solver *s, double *U_host, int nsteps);

/* writeResidual's norm of divF_spts[0] (normType 1, 2 or 3) of the last
 * calcResidual(0) or, after frg_set_monitor(s, 1), of the last update. */
frg_status frg_residual_norm(frg_solver *s, int normType, double *out /*[nFields]*/);
frg_status frg_set_monitor(frg_solver *s, int enable);

frg_status frg_get_time(const frg_solver *s, double *time, double *dt, int *iter);
frg_status frg_set_iter(frg_solver *s, int iter, int initIter);
/* Synchronise the handle's stream (all work finished). */
frg_status frg_sync(frg_solver *s);
/* Run subsequent work on `stream` (a cudaStream_t; NULL restores the
 * handle's own stream).  Pending work on the previous stream is finished first. */
frg_status frg_set_stream(frg_solver *s, void *stream);
/* Measurement hook: nsteps fused steps launched one kernel at a time (no
 * graph) with CUDA events around every launch.  If flush != NULL, flushBytes
 * of it are overwritten before each step (evicts L2).  ms_out[0] = mean time
 * of the per-step dt / wave-speed kernels, ms_out[1 + k] = mean time of RK
 * stage k's kernel, all in milliseconds ([1 + nRK] entries). */
frg_status frg_time_stages(frg_solver *s, int nsteps, void *flush, unsigned long long flushBytes, double *ms_out);
/* Picks the fastest tile shape (elements x threads per block) of the fused
 * TMA stage kernel for this mesh and configuration by timing `nsteps` steps
 * of each candidate, then restores the solution, time, dt and iteration the
 * handle had.  Results do not depend on the choice.  `variant_out` receives
 * the chosen index; `ms_out` (may be NULL) one time per step per candidate
 * (frg_tile_variant_count entries, at most FRG_MAX_TILE_VARIANTS).  A no-op
 * where the TMA kernel is not used.  No counterpart in the reference, which
 * has a single CPU code path. */
#define FRG_MAX_TILE_VARIANTS 16
frg_status frg_autotune(frg_solver *s, int nsteps, int *variant_out, double *ms_out);
/* Number of tile shapes the handle's configuration offers (1 without TMA). */
frg_status frg_tile_variant_count(const frg_solver *s, int *count);
/* Selects a tile shape of the TMA stage kernel by index (0 = default). */
frg_status frg_set_tile_variant(frg_solver *s, int variant);
/* ---- Ensemble mode (no counterpart in the reference) ---------------------
 * Many independent cases of one order in one handle: the mesh is the union
 * of the cases' meshes (no face joins two cases) and groupOfElement gives
 * each element's case.  Each case keeps its own CFL dt (the minimum over its
 * own elements, dtType 1) or the fixed dt given per case (dtType 0,
 * fixedDt[nGroups]), and its own time; everything else is shared, so one
 * launch per RK stage advances every case.  frg_calc_dt / frg_time_step_a/b
 * are not available in this mode (frg_update only); frg_get_time reports
 * group 0. */
frg_status frg_set_groups(frg_solver *s, const int *groupOfElement, int nGroups, const double *fixedDt);
/* Per-group time and the dt of the last step (nGroups doubles each). */
frg_status frg_get_group_times(frg_solver *s, double *time, double *dt);

/* Handles advanced together, e.g. one per order of a batch of cases: each
 * step is one CUDA graph launch whose parallel branches are the handles' own
 * captured fused steps.  frg_ensemble_update returns after the steps
 * finished and each handle's error flags were checked. */
typedef struct frg_ensemble frg_ensemble;
frg_status frg_ensemble_create(frg_solver *const *solvers, int n, frg_ensemble **out);
frg_status frg_ensemble_set_stream(frg_ensemble *e, void *stream);
frg_status frg_ensemble_update(frg_ensemble *e, int nsteps);
frg_status frg_ensemble_destroy(frg_ensemble *e);

/* ---- Discrete adjoint (no counterpart in the reference) ----------------
 * FP64, inviscid (Euler or advection), fixed dt (dtType 0), RK tables of
 * timeType 0/2/4.  The adjoint kernels transpose the residual operation by
 * operation (operators, flux Jacobians, Rusanov / Roe / Lax-Friedrichs and
 * the boundary ghost states through dual numbers). */

/* Objectives of the current state.  FRG_OBJ_ENTROPY: sum over solution
 * points of w detJ (p rhoBound^gamma / (rho^gamma pBound) - 1)
 * (integrateError's entropy error, src/solver.cpp:1507-1531).
 * FRG_OBJ_WALL_PRESSURE: pressure integrated over the slip-wall faces with
 * computeWallForce's face quadrature (src/boundFace.cpp:330-378), from the
 * elements' traces.  J receives the value; grad_host (may be NULL) dJ/dU at
 * the solution points, [spt][ele][field].  The gradient is kept as the
 * default seed of frg_adjoint_backward. */
enum { FRG_OBJ_ENTROPY = 1, FRG_OBJ_WALL_PRESSURE = 2 };
frg_status frg_objective(frg_solver *s, int kind, double *J, double *grad_host);

/* Vector-Jacobian product of calcResidual at the current state: given
 * gbar = dJ/d(divF) ([spt][ele][field]), ubar = (d divF / dU)^T gbar.
 * thetaDir (5 doubles, may be NULL) is the derivative of the boundary state
 * (rhoBound, uBound, vBound, wBound, pBound) with respect to a scalar
 * parameter theta; thetaBar receives gbar . d(divF)/d(theta). */
frg_status frg_residual_vjp(frg_solver *s, const double *gbar_host, const double *thetaDir, double *ubar_host,
                            double *thetaBar);

/* Forward run of nsteps frg_update steps keeping a checkpoint of U every
 * checkpointEvery steps (device memory: nsteps/checkpointEvery + 2 states,
 * plus checkpointEvery x nRK stage states for the reverse sweep, twice when
 * the recomputation overlaps the reversal).  checkpointEvery 0 keeps every
 * RK stage state of the run instead (nsteps x nRK states), so the reverse
 * sweep recomputes nothing.  checkpointEvery < 0 (FRG_CHECKPOINT_AUTO) keeps
 * every stage state when they take at most half of the device memory free
 * at the call, else checkpoints every 25 steps; frg_adjoint_mode reports the
 * choice. */
#define FRG_CHECKPOINT_AUTO (-1)
frg_status frg_adjoint_forward(frg_solver *s, int nsteps, int checkpointEvery);
/* The last frg_adjoint_forward run's checkpoint interval (0: every stage
 * state kept). */
frg_status frg_adjoint_mode(const frg_solver *s, int *checkpointEvery);
/* Reverse sweep of the last frg_adjoint_forward run: from lamN = dJ/dU_N
 * ([spt][ele][field]; NULL = the gradient of the last frg_objective call)
 * to lam0 = dJ/dU_0 and thetaBar = dJ/dtheta through the boundary state
 * (the initial state's own dependence on theta is lam0 . dU_0/dtheta).
 * Each segment between checkpoints is recomputed with its RK stage states,
 * then reversed stage by stage.  The solution is left at U_N. */
frg_status frg_adjoint_backward(frg_solver *s, const double *lamN_host, const double *thetaDir, double *lam0_host,
                                double *thetaBar);

/* ---- Output integrals of the current solution ---------------------------
 * Evaluated on the device from the current state's traces (and, for viscous
 * runs, its corrected gradient), i.e. on the face data a calcResidual(0) of
 * the current state would leave. */

/* solver::computeWallForce (src/solver.cpp:1367-1378) summing
 * boundFace::computeWallForce (src/boundFace.cpp:330-378) over the slip,
 * adiabatic and isothermal wall faces: force[0..2] the pressure force
 * (sum of p n dA w), force[3..5] the viscous force (minus the stress tensor
 * viscousStressTensor, src/flux.cpp:228-358, times n dA w); zeros for
 * advection. */
frg_status frg_wall_force(frg_solver *s, double *force /*[6]*/);
/* solver::computeMassFlux (src/solver.cpp:1380-1391) summing
 * boundFace::computeMassFlux (src/boundFace.cpp:380-418) over the
 * characteristic, supersonic and subsonic in- and outflow faces: the
 * faces' common normal flux Fn (Rusanov on the ghost state, plus the
 * viscous part) times dA w (errorNorm 0), |Fn| dA w n_x (1) or
 * (Fn dA)^2 w n_x (2). */
frg_status frg_mass_flux(frg_solver *s, int errorNorm, double *flux /*[nFields]*/);
/* solver::integrateError (src/solver.cpp:1507-1574) with calcError
 * (src/funcs.cpp:1875-1979) for testCase 1.  icType selects the analytic
 * solution: Navier-Stokes 0 (entropy error of the freestream rhoBound /
 * pBound) or 1 (isentropic vortex of strength eps, 5 in the reference);
 * advection 0 (Gaussian), 1 (sine wave), 2 (cosine product).  box =
 * {xmin, xmax, ymin, ymax}, the period of the convected solution (the
 * reference's mesh box, or +-5 for a mesh it reads).  errorNorm 0: the
 * integral of state minus solution and of the state at the solution points,
 * returned as |difference|; 1 / 2: the state and detJ interpolated to the
 * Gauss points of quadOrder and |error| / error^2 integrated (2: the square
 * root of the sum). */
frg_status frg_integrate_error(frg_solver *s, int icType, double eps, int errorNorm, int quadOrder,
                               const double *box, double *err /*[nFields]*/);

/* Device-side launch counter: kernels launched by this handle so far. */
frg_status frg_launch_count(const frg_solver *s, long long *count);

#ifdef __cplusplus
}
#endif
#endif
