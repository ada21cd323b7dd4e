// solver_gpu.cpp -- the reference-side binding of libfrgpu: the code a
// maintainer adds to FlurryPP (compiled with the reference's include/ and
// this repository's include/frgpu.h, linked with libfrgpu.so) so that the
// main loop's solver::update() and solver::calcResidual() run on the B200
// path.  It uses only the reference's public members; solver.hpp needs no
// change.  The set-up (input file, mesh reading, operators, metrics on the
// host) stays the reference's own.
//
//   solver S;  S.setup(&params, params.order);  S.initializeSolution();
//   frg_solver *gpu = frgpu_setup(S, &params);          // once
//   for (...) { params.iter++; frgpu_update(gpu, &params); }   // solver::update
//   frgpu_download_state(gpu, S);                       // before output
#include <vector>

#include "ele.hpp"
#include "error.hpp"
#include "face.hpp"
#include "frgpu.h"
#include "geo.hpp"
#include "input.hpp"
#include "solver.hpp"

// input (include/input.hpp) -> frg_params
frg_params frgpu_params(const input *p) {
  frg_params q{};
  q.nDims = p->nDims;
  q.order = p->order;
  q.equation = p->equation;
  q.viscous = p->viscous;
  q.riemannType = p->riemannType;
  q.vcjhScheme = p->vcjhSchemeQuad;
  q.timeType = p->timeType;
  q.dtType = p->dtType;
  q.dt = p->dt;
  q.CFL = p->CFL;
  q.gamma = p->gamma;
  q.advectVx = p->advectVx;
  q.advectVy = p->advectVy;
  q.advectVz = p->advectVz;
  q.lambda = p->lambda;
  q.diffD = p->diffD;
  q.rhoBound = p->rhoBound;
  q.uBound = p->uBound;
  q.vBound = p->vBound;
  q.wBound = p->wBound;
  q.pBound = p->pBound;
  q.mu_inf = p->mu_inf;
  q.prandtl = p->prandtl;
  q.c_sth = p->c_sth;
  q.rt_inf = p->rt_inf;
  q.fixVis = p->fixVis;
  q.penFact = p->penFact;
  q.tau = p->tau;
  q.TWall = p->TWall;
  q.RGas = p->RGas;
  q.uWall = p->uWall;
  q.vWall = p->vWall;
  q.wWall = p->wWall;
  q.precision = FRG_FP64;
  return q;
}

// After solver::setup and initializeSolution: the element nodes, corner
// vertex ids and per-face boundary conditions of the reference's geometry
// become the device path's mesh, and U_spts its initial state.
frg_solver *frgpu_setup(solver &S, input *params) {
  const int nE = (int)S.nEles, nN = (int)S.nNodes, d = params->nDims;
  const int nC = d == 2 ? 4 : 8, nFc = d == 2 ? 4 : 6;
  std::vector<double> xv((size_t)nE * nN * d);
  for (int e = 0; e < nE; e++)
    for (int n = 0; n < nN; n++)
      for (int k = 0; k < d; k++) xv[((size_t)e * nN + n) * d + k] = S.nodes(n, e, k);
  std::vector<int> c2v((size_t)nE * nC), bc((size_t)nE * nFc, -1);
  for (int e = 0; e < nE; e++)
    for (int k = 0; k < nC; k++) c2v[(size_t)e * nC + k] = S.Geo->c2v(e, k);
  for (auto &f : S.faces)
    if (f->isBnd) bc[(size_t)f->eL->ID * nFc + f->locF_L] = f->bcType;
  frg_params q = frgpu_params(params);
  frg_mesh m{nE, nN, xv.data(), c2v.data(), bc.data()};
  frg_solver *gpu = nullptr;
  if (frg_create(&q, &m, &gpu) != FRG_OK) fatalError(frg_last_error());
  if (frg_upload(gpu, FRG_U_SPTS, S.U_spts.getData()) != FRG_OK) fatalError(frg_last_error());
  frg_set_iter(gpu, params->iter, params->initIter);
  return gpu;
}

// solver::update (src/solver.cpp:212-250), called after the main loop's
// iter++ (src/flurry.cpp:50-53): one step on the device; time and dt back
// into the input object as the reference keeps them.
void frgpu_update(frg_solver *gpu, input *params) {
  frg_set_iter(gpu, params->iter - 1, params->initIter);
  if (frg_update(gpu, 1) != FRG_OK) fatalError(frg_last_error());
  double t = 0, dt = 0;
  int it = 0;
  frg_get_time(gpu, &t, &dt, &it);
  params->time = t;
  params->rkTime = t;
  params->dt = dt;
}

// solver::calcResidual (src/solver.cpp:252-291) of the device state, with
// divF_spts[step] copied back for host code that reads it.
void frgpu_calc_residual(frg_solver *gpu, solver &S, int step) {
  if (frg_calc_residual(gpu, step) != FRG_OK) fatalError(frg_last_error());
  if (frg_download(gpu, FRG_DIVF, step, S.divF_spts[step].getData()) != FRG_OK) fatalError(frg_last_error());
}

// The device state into U_spts (before writeData / writeResidual).
void frgpu_download_state(frg_solver *gpu, solver &S) {
  if (frg_download(gpu, FRG_U_SPTS, 0, S.U_spts.getData()) != FRG_OK) fatalError(frg_last_error());
}
