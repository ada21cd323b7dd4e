/* ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Links the unmodified FlurryPP reference objects (compiled from their own
 * sources by oracle/Makefile into oracle/_ref/) and dumps what the reference
 * computes, so that the CPU restatement in oracle/fr_oracle.cpp and the CUDA
 * path can be checked against the reference itself.  Nothing in the product
 * links or runs this program.
 *
 * Modes
 *   ops   <nDims> <order> <vcjh> <outdir>  operator matrices built by
 *         oper::setupOperators (src/operators.cpp:13-76) for QUAD (nDims 2) or
 *         HEX (nDims 3) -- the QUAD branch is callable directly although the
 *         solver hard-codes HEX (src/solver.cpp:1395).
 *   kat   <outdir>                          pointwise known-answer vectors:
 *         inviscidFlux / viscousFlux (src/flux.cpp:37-226), face::rusanovFlux,
 *         face::roeFlux, face::laxFriedrichsFlux (src/face.cpp:289-514),
 *         face::ldgSolution (:582), boundFace::applyBCs (src/boundFace.cpp:33)
 *         on seeded states, in 2D and 3D, by driving stand-alone face objects.
 *   case  <input> <outdir> <nsteps>         solver::setup + initializeSolution,
 *         the metrics and face table, one calcResidual(0) with every
 *         intermediate array, then <nsteps> solver::update() calls as in
 *         src/flurry.cpp:49-66, with dt and the L2 residual norm per step.
 *   time  <input> <nsteps>                  seconds per update() (setup and
 *         one warm-up step excluded), printed as one JSON line.
 *   vtu   <input> <outdir> <nsteps>         <nsteps> update() calls, then
 *         writeParaview (src/output.cpp:103) into <outdir>/ref_<iter>.vtu with
 *         the state, nodes and time it wrote from; then a second solver
 *         restarted from that file (readRestartFile, src/solver.cpp:1420) and
 *         the state and time it read.
 *
 * Arrays are written as raw little-endian float64 / int32 files plus a
 * manifest (name dtype dims...) so numpy can read them.
 */
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "boundFace.hpp"
#include "ele.hpp"
#include "face.hpp"
#include "flux.hpp"
#include "geo.hpp"
#include "input.hpp"
#include "intFace.hpp"
#include "operators.hpp"
#include "output.hpp"
#include "solver.hpp"

static FILE *g_manifest = nullptr;
static std::string g_out;

static void dump(const std::string &name, const double *p, size_t n,
                 std::vector<int> dims) {
  std::string fn = g_out + "/" + name + ".f64";
  FILE *f = fopen(fn.c_str(), "wb");
  if (!f) { perror(fn.c_str()); exit(2); }
  fwrite(p, sizeof(double), n, f);
  fclose(f);
  fprintf(g_manifest, "%s f64", name.c_str());
  for (int d : dims) fprintf(g_manifest, " %d", d);
  fprintf(g_manifest, "\n");
}

static void dumpi(const std::string &name, const int *p, size_t n,
                  std::vector<int> dims) {
  std::string fn = g_out + "/" + name + ".i32";
  FILE *f = fopen(fn.c_str(), "wb");
  if (!f) { perror(fn.c_str()); exit(2); }
  fwrite(p, sizeof(int), n, f);
  fclose(f);
  fprintf(g_manifest, "%s i32", name.c_str());
  for (int d : dims) fprintf(g_manifest, " %d", d);
  fprintf(g_manifest, "\n");
}

template <typename A> static void dumpArr(const std::string &name, A &arr, std::vector<int> dims) {
  dump(name, arr.getData(), arr.getSize(), dims);
}

static void openOut(const std::string &dir) {
  g_out = dir;
  std::string cmd = "mkdir -p '" + dir + "'";
  if (system(cmd.c_str()) != 0) { fprintf(stderr, "mkdir failed\n"); exit(2); }
  g_manifest = fopen((dir + "/manifest.txt").c_str(), "w");
}

/* ---------------------------------------------------------------- ops */
static int modeOps(int nDims, int order, int vcjh, const char *out) {
  openOut(out);
  input params;
  params.nDims = nDims;
  params.nFields = 1;
  params.equation = 1;
  params.viscous = 1; /* builds opp_correctU too */
  params.sptsTypeQuad = "Legendre";
  params.vcjhSchemeQuad = vcjh;
  params.quadOrder = order;
  params.scFlag = 0;
  params.PMG = 0;
  params.motion = 0;
  geo g;
  g.nDims = nDims;
  oper op;
  op.setupOperators(nDims == 2 ? QUAD : HEX, order, &g, &params);
  int nS = op.nSpts, nF = op.nFpts;
  dumpArr("spts_to_fpts", op.opp_spts_to_fpts, {nF, nS});
  for (int d = 0; d < nDims; d++) {
    dumpArr("grad_spts_" + std::to_string(d), op.opp_grad_spts[d], {nS, nS});
    dumpArr("extrapolateFn_" + std::to_string(d), op.opp_extrapolateFn[d], {nF, nS});
    dumpArr("correctU_" + std::to_string(d), op.opp_correctU[d], {nS, nF});
  }
  dumpArr("correction", op.opp_correction, {nS, nF});
  std::vector<double> ls, lf;
  for (auto &p : op.loc_spts) for (int d = 0; d < nDims; d++) ls.push_back(p[d]);
  for (auto &p : op.loc_fpts) for (int d = 0; d < nDims; d++) lf.push_back(p[d]);
  dump("loc_spts", ls.data(), ls.size(), {nS, nDims});
  dump("loc_fpts", lf.data(), lf.size(), {nF, nDims});
  fclose(g_manifest);
  return 0;
}

/* ---------------------------------------------------------------- kat */
static unsigned long long g_lcg = 0x2545F4914F6CDD1DULL;
static double urand() { /* uniform [0,1) */
  g_lcg = g_lcg * 6364136223846793005ULL + 1442695040888963407ULL;
  return (double)(g_lcg >> 11) * (1.0 / 9007199254740992.0);
}
static double urange(double a, double b) { return a + (b - a) * urand(); }

/* A conservative state with rho in [0.5,1.5], |v| up to vmax, p in [0.5,1.5]. */
static void randState(int nDims, double gamma, double vmax, double *U) {
  double rho = urange(0.5, 1.5), p = urange(0.5, 1.5), v2 = 0;
  U[0] = rho;
  for (int d = 0; d < nDims; d++) {
    double v = urange(-vmax, vmax);
    U[1 + d] = rho * v;
    v2 += v * v;
  }
  U[nDims + 1] = p / (gamma - 1) + 0.5 * rho * v2;
}
static void randNormal(int nDims, double *n) {
  double s = 0;
  for (int d = 0; d < nDims; d++) { n[d] = urange(-1, 1); s += n[d] * n[d]; }
  s = sqrt(s);
  for (int d = 0; d < nDims; d++) n[d] /= s;
}

static void setupGas(input &p, int nDims, int viscous) {
  p.nDims = nDims;
  p.nFields = nDims + 2;
  p.equation = NAVIER_STOKES;
  p.gamma = 1.4;
  p.motion = 0;
  p.viscous = viscous;
  p.rhoBound = 1.0;
  p.uBound = 0.5 * sqrt(1.4);
  p.vBound = 0.1;
  p.wBound = nDims == 3 ? -0.05 : 0.0;
  p.pBound = 1.0;
  p.mu_inf = 1.0 / 1600.0;
  p.prandtl = 0.71;
  p.fixVis = 1;
  p.c_sth = 0.41;
  p.rt_inf = 2.5;
  p.penFact = 0.3;
  p.tau = 1.0;
}

static void faceArrays(face &f, input *p, int n) {
  f.params = p;
  f.nDims = p->nDims;
  f.nFields = p->nFields;
  f.nFptsL = n;
  f.UL.setup(n, p->nFields);
  f.UR.setup(n, p->nFields);
  f.UC.setup(n, p->nFields);
  f.Fn.setup(n, p->nFields);
  f.normL.setup(n, p->nDims);
  f.waveSp.resize(n);
}

static int modeKat(const char *out) {
  openOut(out);
  const int N = 64;
  for (int nDims = 2; nDims <= 3; nDims++) {
    std::string sfx = "_" + std::to_string(nDims) + "d";
    int nV = nDims + 2;
    /* -- pointwise inviscid + viscous flux, Sutherland off and on -- */
    for (int fix = 0; fix <= 1; fix++) {
      input p;
      setupGas(p, nDims, 1);
      p.fixVis = fix;
      std::vector<double> U(N * nV), G(N * nDims * nV), Fi(N * nDims * nV), Fv(N * nDims * nV);
      for (int i = 0; i < N; i++) {
        randState(nDims, p.gamma, 0.8, &U[i * nV]);
        for (int k = 0; k < nDims * nV; k++) G[i * nDims * nV + k] = urange(-1, 1);
        double F[3][5], FV[3][5];
        inviscidFlux(&U[i * nV], F, &p);
        matrix<double> gradU(nDims, nV);
        for (int d = 0; d < nDims; d++)
          for (int k = 0; k < nV; k++) gradU(d, k) = G[i * nDims * nV + d * nV + k];
        viscousFlux(&U[i * nV], gradU, FV, &p);
        for (int d = 0; d < nDims; d++)
          for (int k = 0; k < nV; k++) {
            Fi[i * nDims * nV + d * nV + k] = F[d][k];
            Fv[i * nDims * nV + d * nV + k] = FV[d][k];
          }
      }
      std::string s2 = sfx + "_fix" + std::to_string(fix);
      dump("flux_U" + s2, U.data(), U.size(), {N, nV});
      dump("flux_gradU" + s2, G.data(), G.size(), {N, nDims, nV});
      dump("flux_inv" + s2, Fi.data(), Fi.size(), {N, nDims, nV});
      dump("flux_vis" + s2, Fv.data(), Fv.size(), {N, nDims, nV});
    }
    /* -- common inviscid fluxes on one face of N points -- */
    {
      input p;
      setupGas(p, nDims, 1);
      intFace f;
      faceArrays(f, &p, N);
      std::vector<double> ws(N);
      for (int i = 0; i < N; i++) f.waveSp[i] = &ws[i];
      std::vector<double> UL(N * nV), UR(N * nV), nrm(N * nDims), Fr(N * nV), Fro(N * nV), W(N), UC(N * nV);
      for (int i = 0; i < N; i++) {
        randState(nDims, p.gamma, 0.8, &UL[i * nV]);
        randState(nDims, p.gamma, 0.8, &UR[i * nV]);
        randNormal(nDims, &nrm[i * nDims]);
        for (int k = 0; k < nV; k++) { f.UL(i, k) = UL[i * nV + k]; f.UR(i, k) = UR[i * nV + k]; }
        for (int d = 0; d < nDims; d++) f.normL(i, d) = nrm[i * nDims + d];
      }
      f.rusanovFlux();
      for (int i = 0; i < N; i++) { for (int k = 0; k < nV; k++) Fr[i * nV + k] = f.Fn(i, k); W[i] = ws[i]; }
      f.isBnd = 0;
      f.ldgSolution();
      for (int i = 0; i < N; i++) for (int k = 0; k < nV; k++) UC[i * nV + k] = f.UC(i, k);
      dump("face_UL" + sfx, UL.data(), UL.size(), {N, nV});
      dump("face_UR" + sfx, UR.data(), UR.size(), {N, nV});
      dump("face_norm" + sfx, nrm.data(), nrm.size(), {N, nDims});
      dump("face_rusanov" + sfx, Fr.data(), Fr.size(), {N, nV});
      dump("face_rusanov_wavesp" + sfx, W.data(), W.size(), {N});
      dump("face_ldgUC" + sfx, UC.data(), UC.size(), {N, nV});
      if (nDims == 2) {
        f.roeFlux();
        for (int i = 0; i < N; i++) for (int k = 0; k < nV; k++) Fro[i * nV + k] = f.Fn(i, k);
        dump("face_roe" + sfx, Fro.data(), Fro.size(), {N, nV});
      }
    }
    /* -- boundary ghost states for the BCs the path needs -- */
    {
      const int bcs[4] = {CHAR_INOUT, SLIP_WALL, SUP_IN, SUP_OUT};
      const char *names[4] = {"char", "slip_wall", "sup_in", "sup_out"};
      for (int b = 0; b < 4; b++) {
        for (int sub = 0; sub < 2; sub++) { /* subsonic and supersonic freestream */
          input p;
          setupGas(p, nDims, 0);
          if (sub) p.uBound = 2.0 * sqrt(1.4);
          boundFace f;
          faceArrays(f, &p, N);
          f.bcType = bcs[b];
          std::vector<double> UL(N * nV), nrm(N * nDims), UR(N * nV);
          for (int i = 0; i < N; i++) {
            randState(nDims, p.gamma, sub ? 3.0 : 0.8, &UL[i * nV]);
            randNormal(nDims, &nrm[i * nDims]);
            for (int k = 0; k < nV; k++) f.UL(i, k) = UL[i * nV + k];
            for (int d = 0; d < nDims; d++) f.normL(i, d) = nrm[i * nDims + d];
          }
          f.applyBCs();
          for (int i = 0; i < N; i++) for (int k = 0; k < nV; k++) UR[i * nV + k] = f.UR(i, k);
          std::string s2 = sfx + "_" + names[b] + (sub ? "_sup" : "_sub");
          dump("bc_UL" + s2, UL.data(), UL.size(), {N, nV});
          dump("bc_norm" + s2, nrm.data(), nrm.size(), {N, nDims});
          dump("bc_UR" + s2, UR.data(), UR.size(), {N, nV});
          double bnd[4] = {p.rhoBound, p.uBound, p.vBound, p.pBound};
          dump("bc_bound" + s2, bnd, 4, {4});
        }
      }
    }
    /* -- scalar advection Lax-Friedrichs -- */
    {
      input p;
      p.nDims = nDims; p.nFields = 1; p.equation = ADVECTION_DIFFUSION; p.motion = 0;
      p.advectVx = 1.0; p.advectVy = 1.0; p.advectVz = nDims == 3 ? 0.5 : 0.0; p.lambda = 1.0;
      intFace f;
      faceArrays(f, &p, N);
      std::vector<double> ws(N);
      for (int i = 0; i < N; i++) f.waveSp[i] = &ws[i];
      std::vector<double> uL(N), uR(N), nrm(N * nDims), Fn(N), W(N);
      for (int i = 0; i < N; i++) {
        uL[i] = urange(-1, 1); uR[i] = urange(-1, 1);
        randNormal(nDims, &nrm[i * nDims]);
        f.UL(i, 0) = uL[i]; f.UR(i, 0) = uR[i];
        for (int d = 0; d < nDims; d++) f.normL(i, d) = nrm[i * nDims + d];
      }
      f.laxFriedrichsFlux();
      for (int i = 0; i < N; i++) { Fn[i] = f.Fn(i, 0); W[i] = ws[i]; }
      dump("lf_uL" + sfx, uL.data(), N, {N});
      dump("lf_uR" + sfx, uR.data(), N, {N});
      dump("lf_norm" + sfx, nrm.data(), nrm.size(), {N, nDims});
      dump("lf_Fn" + sfx, Fn.data(), N, {N});
      dump("lf_wavesp" + sfx, W.data(), N, {N});
    }
  }
  fclose(g_manifest);
  return 0;
}

/* ---------------------------------------------------------------- case */
static void dumpResidualArrays(solver &S, input &params, const std::string &pre) {
  int nS = S.nSpts, nF = S.nFpts, nE = S.nEles, nV = S.nFields, nD = S.nDims;
  dumpArr(pre + "U_spts", S.U_spts, {nS, nE, nV});
  dumpArr(pre + "U_fpts", S.U_fpts, {nF, nE, nV});
  dumpArr(pre + "F_spts", S.F_spts, {nD, nS, nE, nV});
  dumpArr(pre + "Fn_fpts", S.Fn_fpts, {nF, nE, nV});
  dumpArr(pre + "disFn_fpts", S.disFn_fpts, {nF, nE, nV});
  dumpArr(pre + "divF_spts", S.divF_spts[0], {nS, nE, nV});
  if (params.viscous) {
    dumpArr(pre + "dU_spts", S.dU_spts, {nD, nS, nE, nV});
    dumpArr(pre + "dU_fpts", S.dU_fpts, {nD, nF, nE, nV});
    dumpArr(pre + "dUc_fpts", S.dUc_fpts, {nF, nE, nV});
  }
}

static int modeCase(char *inputFile, const char *out, int nsteps) {
  openOut(out);
  input params;
  params.rank = 0;
  params.nproc = 1;
  params.readInputFile(inputFile);
  solver S;
  S.setup(&params, params.order);
  S.initializeSolution();
  int nS = S.nSpts, nF = S.nFpts, nE = S.nEles, nD = S.nDims;
  /* effective (non-dimensionalised) parameters, src/input.cpp:483-554 */
  double prm[] = {params.gamma, params.rhoBound, params.uBound, params.vBound, params.wBound,
                  params.pBound, params.mu_inf, params.prandtl, params.c_sth, params.rt_inf,
                  (double)params.fixVis, params.penFact, params.tau, params.TWall, params.RGas,
                  params.uWall, params.vWall, params.wWall, params.dt, params.CFL};
  dump("params", prm, sizeof(prm) / sizeof(double), {(int)(sizeof(prm) / sizeof(double))});
  /* geometry and the face table */
  dumpArr("pos_spts", S.pos_spts, {nS, nE, nD});
  dumpArr("JGinv_spts", S.JGinv_spts, {nD, nS, nE, nD});
  dumpArr("detJac_spts", S.detJac_spts, {nS, nE});
  dumpArr("norm_fpts", S.norm_fpts, {nF, nE, nD});
  dumpArr("dA_fpts", S.dA_fpts, {nF, nE});
  dumpArr("nodes", S.nodes, {(int)S.nNodes, nE, nD});
  std::vector<int> ftab;
  for (auto &f : S.faces) {
    ftab.push_back(f->eL->ID);
    ftab.push_back(f->locF_L);
    ftab.push_back(f->isBnd ? -1 : f->eR->ID);
    ftab.push_back(f->isBnd ? -1 : f->myInfo.IDR);
    ftab.push_back(f->isBnd ? -1 : f->myInfo.relRot);
    ftab.push_back(f->isBnd ? f->bcType : -1);
  }
  dumpi("faces", ftab.data(), ftab.size(), {(int)S.faces.size(), 6});
  /* one residual evaluation, as the first RK stage sees it */
  params.iter = params.initIter + 1;
  S.calcResidual(0);
  dumpResidualArrays(S, params, "r0_");
  /* the time loop of src/flurry.cpp:49-66 */
  params.iter = params.initIter;
  std::vector<double> dts, res;
  for (int n = 0; n < nsteps; n++) {
    params.iter++;
    S.update();
    dts.push_back(params.dt);
    std::vector<double> r(params.nFields, 0.0);
    for (auto &e : S.eles) {
      auto rt = e->getNormResidual(2);
      for (int k = 0; k < params.nFields; k++) r[k] += rt[k];
    }
    for (double v : r) res.push_back(v);
  }
  if (nsteps > 0) {
    dumpArr("final_U_spts", S.U_spts, {nS, nE, (int)params.nFields});
    dump("dt_hist", dts.data(), dts.size(), {nsteps});
    dump("res_hist", res.data(), res.size(), {nsteps, (int)params.nFields});
    std::vector<double> ws;
    for (auto &e : S.eles) for (int f = 0; f < nF; f++) ws.push_back(e->waveSp_fpts[f]);
    dump("final_waveSp", ws.data(), ws.size(), {nE, nF});
  }
  double t = params.time;
  dump("final_time", &t, 1, {1});
  fclose(g_manifest);
  return 0;
}

static int modeVtu(char *inputFile, const char *out, int nsteps) {
  openOut(out);
  input params;
  params.rank = 0;
  params.nproc = 1;
  params.readInputFile(inputFile);
  solver S;
  S.setup(&params, params.order);
  S.initializeSolution();
  params.iter = params.initIter;
  for (int n = 0; n < nsteps; n++) {
    params.iter++;
    S.update();
  }
  const int nS = S.nSpts, nE = S.nEles, nD = S.nDims;
  dumpArr("U_spts", S.U_spts, {nS, nE, (int)params.nFields});
  dumpArr("nodes", S.nodes, {(int)S.nNodes, nE, nD});
  double t = params.time;
  dump("time", &t, 1, {1});
  int it = params.iter;
  dumpi("iter", &it, 1, {1});
  params.dataFileName = std::string(out) + "/ref";
  writeParaview(&S, &params);
  /* restart a second solver from the file (input::readInputFile with
     restart = 1 sets initIter = restartIter, src/input.cpp:417-421) */
  input p2;
  p2.rank = 0;
  p2.nproc = 1;
  p2.readInputFile(inputFile);
  p2.restart = 1;
  p2.restartIter = it;
  p2.initIter = it;
  p2.iter = it;
  p2.dataFileName = params.dataFileName;
  solver S2;
  S2.setup(&p2, p2.order);
  S2.initializeSolution();
  dumpArr("restart_U_spts", S2.U_spts, {nS, nE, (int)p2.nFields});
  double t2 = p2.time;
  dump("restart_time", &t2, 1, {1});
  fclose(g_manifest);
  return 0;
}

/* The output integrals after nsteps updates and one calcResidual(0):
 * solver::computeWallForce, computeMassFlux (errorNorm 0, 1, 2) and, with
 * testCase 1, integrateError (errorNorm 0, 1, 2; quadOrder from the input). */
static int modeIntegrals(char *inputFile, const char *out, int nsteps) {
  openOut(out);
  input params;
  params.rank = 0;
  params.nproc = 1;
  params.readInputFile(inputFile);
  solver S;
  S.setup(&params, params.order);
  S.initializeSolution();
  double prm[] = {params.gamma, params.rhoBound, params.uBound, params.vBound, params.wBound,
                  params.pBound, params.mu_inf, params.prandtl, params.c_sth, params.rt_inf,
                  (double)params.fixVis, params.penFact, params.tau, params.TWall, params.RGas,
                  params.uWall, params.vWall, params.wWall, params.dt, params.CFL};
  dump("params", prm, sizeof(prm) / sizeof(double), {(int)(sizeof(prm) / sizeof(double))});
  params.iter = params.initIter;
  for (int n = 0; n < nsteps; n++) {
    params.iter++;
    S.update();
  }
  const int nS = S.nSpts, nE = S.nEles;
  dumpArr("U_spts", S.U_spts, {nS, nE, (int)params.nFields});
  double t = params.time;
  dump("time", &t, 1, {1});
  S.calcResidual(0);
  std::vector<double> f = S.computeWallForce();
  dump("wall_force", f.data(), f.size(), {(int)f.size()});
  for (int en = 0; en < 3; en++) {
    params.errorNorm = en;
    std::vector<double> m = S.computeMassFlux();
    dump("mass_flux_" + std::to_string(en), m.data(), m.size(), {(int)m.size()});
  }
  params.testCase = 1;
  for (int en = 0; en < 3; en++) {
    params.errorNorm = en;
    std::vector<double> e = S.integrateError();
    dump("error_" + std::to_string(en), e.data(), e.size(), {(int)e.size()});
  }
  fclose(g_manifest);
  return 0;
}

static int modeTime(char *inputFile, int nsteps) {
  input params;
  params.rank = 0;
  params.nproc = 1;
  params.readInputFile(inputFile);
  solver S;
  auto t0 = std::chrono::steady_clock::now();
  S.setup(&params, params.order);
  S.initializeSolution();
  auto t1 = std::chrono::steady_clock::now();
  params.iter = params.initIter;
  params.iter++;
  S.update(); /* warm-up: first iteration also runs calcWaveSpFpts */
  auto t2 = std::chrono::steady_clock::now();
  for (int n = 0; n < nsteps; n++) {
    params.iter++;
    S.update();
  }
  auto t3 = std::chrono::steady_clock::now();
  double secs = std::chrono::duration<double>(t3 - t2).count();
  double dof = (double)S.nEles * S.nSpts * S.nFields;
  printf("{\"s_per_step\": %.9g, \"steps\": %d, \"dof\": %.0f, \"setup_s\": %.3f, "
         "\"dof_updates_per_s\": %.6g, \"checksum\": %.17g}\n",
         secs / nsteps, nsteps, dof, std::chrono::duration<double>(t1 - t0).count(),
         dof * nsteps / secs, S.U_spts.getData()[0]);
  (void)t2;
  return 0;
}

int main(int argc, char **argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: refharness ops|kat|case|time ...\n");
    return 2;
  }
  std::string mode = argv[1];
  if (mode == "ops" && argc == 6) return modeOps(atoi(argv[2]), atoi(argv[3]), atoi(argv[4]), argv[5]);
  if (mode == "kat" && argc == 3) return modeKat(argv[2]);
  if (mode == "case" && argc == 5) return modeCase(argv[2], argv[3], atoi(argv[4]));
  if (mode == "time" && argc == 4) return modeTime(argv[2], atoi(argv[3]));
  if (mode == "vtu" && argc == 5) return modeVtu(argv[2], argv[3], atoi(argv[4]));
  if (mode == "integrals" && argc == 5) return modeIntegrals(argv[2], argv[3], atoi(argv[4]));
  fprintf(stderr, "bad arguments\n");
  return 2;
}
