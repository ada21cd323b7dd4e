/* fr_oracle.h -- TEST INFRASTRUCTURE: the CPU restatement ("oracle") of the
 * FlurryPP flux-reconstruction residual + Runge-Kutta path, in FP64.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library, and only as the checker / CPU timing baseline.  The
 * product (fr_learn_b200/, libfrgpu.so) never links or calls it.
 *
 * Pinning: the restatement is checked against the FlurryPP reference itself
 * (oracle/ref_harness.cpp built from the reference sources by oracle/Makefile):
 * operator matrices (QUAD and HEX, P=1..5), pointwise flux / Riemann / BC
 * known-answer vectors in 2D and 3D, and whole 3D hex cases (residual and
 * multi-step update).  Fixtures live in tests/golden/ with the script that
 * made them.  2D meshes and periodic pairing cannot run in the reference
 * (src/geo.cpp:35-37, src/boundFace.cpp:264-267); for those the oracle
 * re-enables the reference's own 2D branches and adds periodic face pairing.
 *
 * Layout follows the reference: every solution array is row-major
 * [point][element][field] (src/solver.cpp:65-107).
 */
#ifndef FR_ORACLE_H
#define FR_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_params {
  int nDims;       /* 2 or 3 */
  int order;       /* polynomial order P */
  int equation;    /* 0 advection(-diffusion), 1 Euler / Navier-Stokes */
  int viscous;     /* 0 / 1 */
  int riemannType; /* 0 Rusanov, 1 Roe (2D only, src/face.cpp:362) */
  int vcjhScheme;  /* 0 DG, 1 SD, 2 HU, 3 C+ */
  int timeType;    /* 0 FE, 2 RK2, 4 RK44, 5 RK44 Jameson form */
  int dtType;      /* 0 fixed dt, 1 global CFL, 2 local CFL */
  double dt, CFL;
  double gamma;
  double advectVx, advectVy, advectVz, lambda, diffD;
  double rhoBound, uBound, vBound, wBound, pBound;
  double mu_inf, prandtl, c_sth, rt_inf;
  int fixVis;
  double penFact, tau;
  double TWall, RGas, uWall, vWall, wWall;
} orc_params;

typedef struct orc_solver orc_solver;

/* xv: [nEles][nNodes][nDims] element node coordinates, reference shape-node
 *     order (Gmsh order; quads of any Lagrange order, 8-node hexes).
 * c2v: [nEles][nCorners] vertex ids used for face matching; periodic images
 *      share one id.
 * bc:  [nEles][nFacesPerEle] boundary condition (reference BC_TYPE) of an
 *      element face that has no neighbour, -1 otherwise.
 * Returns NULL and prints the reason on invalid input. */
orc_solver *orc_create(const orc_params *p, int nEles, int nNodes,
                       const double *xv, const int *c2v, const int *bc);
void orc_destroy(orc_solver *s);

int orc_nspts(const orc_solver *s);
int orc_nfpts(const orc_solver *s);
int orc_nfields(const orc_solver *s);
int orc_nfaces(const orc_solver *s);

/* Named array access ([point][element][field] layouts as in the reference):
 * U_spts U0 U_fpts F_spts Fn_fpts disFn_fpts dU_spts dU_fpts dUc_fpts
 * divF_spts0..3 pos_spts JGinv_spts detJac_spts norm_fpts dA_fpts waveSp
 * opp_spts_to_fpts opp_grad_spts0..2 opp_extrapolateFn0..2 opp_correction
 * opp_correctU0..2.  Returns the element count copied, -1 if unknown. */
long orc_get(const orc_solver *s, const char *name, double *out);
long orc_set(orc_solver *s, const char *name, const double *in);
/* faces: [nFaces][6] = eL, locF_L, eR, locF_R, relRot, bcType (-1 if none) */
void orc_get_faces(const orc_solver *s, int *out);

/* Initial conditions of ele::setInitialCondition (src/ele.cpp:683-790).
 * icType as in the reference; 10 = Taylor-Green vortex (not in the
 * reference): rho0=1, V0=1, p0 = 1/(gamma*Ma^2), parameter a0 = Ma. */
void orc_set_ic(orc_solver *s, int icType, double a0);

void orc_extrapolate_u(orc_solver *s);
void orc_calc_residual(orc_solver *s, int step);
void orc_time_step_a(orc_solver *s, int step, double rkval);
void orc_time_step_b(orc_solver *s, int step);
void orc_calc_dt(orc_solver *s);
/* One iteration of the reference main loop: iter++, solver::update(). */
void orc_update(orc_solver *s);
double orc_get_dt(const orc_solver *s);
double orc_get_time(const orc_solver *s);
int orc_get_iter(const orc_solver *s);
/* ele::getNormResidual summed as writeResidual does (src/output.cpp:846) */
void orc_residual_norm(const orc_solver *s, int normType, double *out);
void orc_set_threads(int n);
/* Integrals of the output path (computeWallForce, computeMassFlux,
 * integrateError); the first two use the face data of the last
 * orc_calc_residual. */
void orc_wall_force(const orc_solver *s, double *force /*[6]*/);
void orc_mass_flux(const orc_solver *s, int errorNorm, double *flux /*[nFields]*/);
void orc_integrate_error(const orc_solver *s, int icType, double eps, int errorNorm, int quadOrder,
                         const double *box /*xmin, xmax, ymin, ymax*/, double *out /*[nFields]*/);

/* Pointwise routines, exposed for known-answer tests against the reference.
 * Fluxes are [nDims][nFields]; gradU is [nDims][nFields]. */
void orc_point_flux(const orc_params *p, const double *U, const double *gradU, double *Finv, double *Fvis);
double orc_point_rusanov(const orc_params *p, const double *UL, const double *UR, const double *n, double *Fn);
void orc_point_roe(const orc_params *p, const double *UL, const double *UR, const double *n, double *Fn);
double orc_point_lf(const orc_params *p, double uL, double uR, const double *n, double *Fn);
void orc_point_ldg_uc(const orc_params *p, const double *UL, const double *UR, const double *n, double *UC);
void orc_point_bc(const orc_params *p, int bcType, const double *UL, const double *n, double *UR);

#ifdef __cplusplus
}
#endif
#endif
