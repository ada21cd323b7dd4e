// physics.cuh -- pointwise physics of the FR path as device functions:
// inviscid fluxes, the Rusanov / Roe / Lax-Friedrichs common fluxes, boundary
// ghost states and the viscous flux.  Each keeps the operation order of the
// reference routine it restates (cited per function), so the FP64 build agrees
// with the reference to rounding (FMA contraction aside).
//
// Template parameter R is the arithmetic type (double, or float in the mixed
// mode); PR is the type of the Riemann solvers' pressure recovery
// p = (gamma-1)(E - rho|v|^2/2), which is always double: at low Mach number E
// and the kinetic energy nearly cancel.
#pragma once
#include <cuda_runtime.h>

namespace frg {

// Parameters of the physics, as `input` holds them (include/input.hpp).
struct Phys {
  double gamma;
  double adv[3];  // advectVx, advectVy, advectVz
  double lambda;  // Lax-Friedrichs upwinding factor
  double diffD;   // advection-diffusion coefficient
  double rhoB, vB[3], pB;
  double mu, prandtl, c_sth, rt_inf;
  double penFact, tau;
  double TWall, RGas, vWall[3];
  int fixVis;
  int riemann;  // 0 Rusanov, 1 Roe
};

// BC_TYPE values (include/global.hpp:63-78)
enum : int {
  BC_CHAR = 1, BC_SUP_IN = 2, BC_SUP_OUT = 3, BC_SUB_IN = 4, BC_SUB_OUT = 5,
  BC_SLIP = 8, BC_ISO_NOSLIP = 9, BC_ADI_NOSLIP = 10, BC_SYMMETRY = 12, BC_ISO_NOSLIP_MOVING = 13
};

// inviscidFlux (src/flux.cpp:37-88).  F[d][k]: flux of field k along x_d.
template <int DIM, int NV, typename R>
__device__ __forceinline__ void inviscid_flux(const R *U, R F[DIM][NV], const Phys &ph) {
  if constexpr (NV == 1) {
    F[0][0] = (R)ph.adv[0] * U[0];
    F[1][0] = (R)ph.adv[1] * U[0];
    if constexpr (DIM == 3) F[2][0] = (R)ph.adv[2] * U[0];
  } else if constexpr (DIM == 2) {
    const R g = (R)ph.gamma;
    const R rho = U[0], ir = (R)1 / rho, u = U[1] * ir, v = U[2] * ir, E = U[3];
    R p = (g - (R)1.0) * (E - (R)0.5 * rho * (u * u + v * v));
    F[0][0] = rho * u; F[1][0] = rho * v;
    F[0][1] = rho * u * u + p; F[1][1] = rho * u * v;
    F[0][2] = rho * v * u; F[1][2] = rho * v * v + p;
    F[0][3] = (E + p) * u; F[1][3] = (E + p) * v;
  } else {
    const R g = (R)ph.gamma;
    const R rho = U[0], ir = (R)1 / rho, u = U[1] * ir, v = U[2] * ir, w = U[3] * ir, E = U[4];
    R p = (g - (R)1.0) * (E - (R)0.5 * rho * (u * u + v * v + w * w));
    F[0][0] = rho * u; F[1][0] = rho * v; F[2][0] = rho * w;
    F[0][1] = rho * u * u + p; F[1][1] = rho * u * v; F[2][1] = rho * u * w;
    F[0][2] = rho * v * u; F[1][2] = rho * v * v + p; F[2][2] = rho * v * w;
    F[0][3] = rho * w * u; F[1][3] = rho * w * v; F[2][3] = rho * w * w + p;
    F[0][4] = (E + p) * u; F[1][4] = (E + p) * v; F[2][4] = (E + p) * w;
  }
}

// face::rusanovFlux, one flux point (src/face.cpp:289-356).  Returns the wave
// speed max(|vn_L|+c_L, |vn_R|+c_R) that the reference stores for calcDt.
template <int DIM, int NV, typename R, typename PR>
__device__ __forceinline__ R rusanov(const R *UL, const R *UR, const R *n, R *Fn, const Phys &ph) {
  R FL[DIM][NV], FR[DIM][NV];
  inviscid_flux<DIM, NV, R>(UL, FL, ph);
  inviscid_flux<DIM, NV, R>(UR, FR, ph);
  R FnL[NV], FnR[NV];
#pragma unroll
  for (int i = 0; i < NV; i++) { FnL[i] = 0; FnR[i] = 0; }
  const PR g = (PR)ph.gamma;
  const PR rhoL = UL[0], rhoR = UR[0], irL = (PR)1 / rhoL, irR = (PR)1 / rhoR;
  PR uL = (PR)UL[1] * irL, uR = (PR)UR[1] * irR, vL = (PR)UL[2] * irL, vR = (PR)UR[2] * irR;
  PR pL, pR;
  if constexpr (DIM == 2) {
    pL = (g - (PR)1.0) * ((PR)UL[3] - (PR)0.5 * rhoL * (uL * uL + vL * vL));
    pR = (g - (PR)1.0) * ((PR)UR[3] - (PR)0.5 * rhoR * (uR * uR + vR * vR));
  } else {
    PR wL = (PR)UL[3] * irL, wR = (PR)UR[3] * irR;
    pL = (g - (PR)1.0) * ((PR)UL[4] - (PR)0.5 * rhoL * (uL * uL + vL * vL + wL * wL));
    pR = (g - (PR)1.0) * ((PR)UR[4] - (PR)0.5 * rhoR * (uR * uR + vR * vR + wR * wR));
  }
  const R irLr = (R)irL, irRr = (R)irR;
  R vnL = 0, vnR = 0;
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    vnL += n[d] * UL[d + 1] * irLr;
    vnR += n[d] * UR[d + 1] * irRr;
#pragma unroll
    for (int i = 0; i < NV; i++) { FnL[i] += n[d] * FL[d][i]; FnR[i] += n[d] * FR[d][i]; }
  }
  R csqL = (R)fmax(g * pL * irL, (PR)0.0), csqR = (R)fmax(g * pR * irR, (PR)0.0);
  R eigL = fabs(vnL) + sqrt(csqL), eigR = fabs(vnR) + sqrt(csqR);
  R eig = eigL > eigR ? eigL : eigR;
#pragma unroll
  for (int i = 0; i < NV; i++) Fn[i] = (R)0.5 * (FnL[i] + FnR[i] - eig * (UR[i] - UL[i]));
  return eig;
}

// face::roeFlux with the entropy fix, 2D (src/face.cpp:358-484).
template <typename R, typename PR>
__device__ __forceinline__ void roe2d(const R *UL, const R *UR, const R *n, R *Fn, const Phys &ph) {
  const R g = (R)ph.gamma;
  R vL[2], vR[2], um[2], du[4];
  const R irL = (R)1 / UL[0], irR = (R)1 / UR[0];
  for (int i = 0; i < 2; i++) { vL[i] = UL[i + 1] * irL; vR[i] = UR[i + 1] * irR; }
  const PR gp = (PR)ph.gamma;
  R pL = (R)((gp - (PR)1.0) * ((PR)UL[3] - ((PR)0.5 * (PR)UL[0] * ((PR)vL[0] * (PR)vL[0] + (PR)vL[1] * (PR)vL[1]))));
  R pR = (R)((gp - (PR)1.0) * ((PR)UR[3] - ((PR)0.5 * (PR)UR[0] * ((PR)vR[0] * (PR)vR[0] + (PR)vR[1] * (PR)vR[1]))));
  R hL = (UL[3] + pL) * irL, hR = (UR[3] + pR) * irR;
  R sq_rho = sqrt(UR[0] * irL);
  R rrho = (R)1. / (sq_rho + (R)1.);
  R usq = 0, unm = 0;
  for (int i = 0; i < 2; i++) {
    um[i] = rrho * (vL[i] + sq_rho * vR[i]);
    usq += (R)0.5 * um[i] * um[i];
    unm += um[i] * n[i];
  }
  R hm = rrho * (hL + sq_rho * hR);
  R am_sq = (g - (R)1.) * (hm - usq);
  R am = sqrt(am_sq), iam = (R)1 / am;
  R rhoUnL = 0, rhoUnR = 0;
  for (int i = 0; i < 2; i++) { rhoUnL += UL[i + 1] * n[i]; rhoUnR += UR[i + 1] * n[i]; }
  Fn[0] = rhoUnL + rhoUnR;
  Fn[1] = rhoUnL * vL[0] + rhoUnR * vR[0] + (pL + pR) * n[0];
  Fn[2] = rhoUnL * vL[1] + rhoUnR * vR[1] + (pL + pR) * n[1];
  Fn[3] = rhoUnL * hL + rhoUnR * hR;
  for (int i = 0; i < 4; i++) du[i] = UR[i] - UL[i];
  R lambda0 = fabs(unm), lambdaP = fabs(unm + am), lambdaM = fabs(unm - am);
  R eps = (R)0.5 * (fabs(rhoUnL * irL - rhoUnR * irR) + fabs(sqrt(g * pL * irL) - sqrt(g * pR * irR)));
  // the entropy fix is taken only when eps > lambda/2 >= 0, so 1/eps is finite there
  const R qe = (R)0.25 / eps;
  if (lambda0 < (R)2. * eps) lambda0 = qe * lambda0 * lambda0 + eps;
  if (lambdaP < (R)2. * eps) lambdaP = qe * lambdaP * lambdaP + eps;
  if (lambdaM < (R)2. * eps) lambdaM = qe * lambdaM * lambdaM + eps;
  R a2 = (R)0.5 * (lambdaP + lambdaM) - lambda0;
  R a3 = (R)0.5 * (lambdaP - lambdaM) * iam;
  R a1 = a2 * (g - (R)1.) * (iam * iam);
  R a4 = a3 * (g - (R)1.);
  R a5 = usq * du[0] - um[0] * du[1] - um[1] * du[2] + du[3];
  R a6 = unm * du[0] - n[0] * du[1] - n[1] * du[2];
  R aL1 = a1 * a5 - a3 * a6, bL1 = a4 * a5 - a2 * a6;
  Fn[0] -= lambda0 * du[0] + aL1;
  Fn[1] -= lambda0 * du[1] + aL1 * um[0] + bL1 * n[0];
  Fn[2] -= lambda0 * du[2] + aL1 * um[1] + bL1 * n[1];
  Fn[3] -= lambda0 * du[3] + aL1 * hm + bL1 * unm;
  for (int i = 0; i < 4; i++) Fn[i] *= (R)0.5;
}

// face::laxFriedrichsFlux for scalar advection (src/face.cpp:486-514).
template <int DIM, typename R>
__device__ __forceinline__ R lax_friedrichs(R uL, R uR, const R *n, R *Fn, const Phys &ph) {
  R uAvg = (R)0.5 * (uL + uR), uDiff = uL - uR;
  R vN = (R)ph.adv[0] * n[0] + (R)ph.adv[1] * n[1];
  if constexpr (DIM == 3) vN += (R)ph.adv[2] * n[2];
  Fn[0] = vN * uAvg + (R)0.5 * (R)ph.lambda * fabs(vN) * uDiff;
  return fabs(vN);
}

// viscousFlux (src/flux.cpp:90-226), Navier-Stokes, with the reference's
// index slips kept: tauxz = mu(du/dz + dv/dx), tauyz = mu(du/dz + dv/dy)
// (:197-198) and Fvis[0][3] = -tauzz, Fvis[1][3] = -tauyz (:216-217).
// g is the physical gradient [DIM][NV].
template <int DIM, typename R>
__device__ __forceinline__ void viscous_flux(const R *U, const R *g, R Fv[DIM][DIM + 2], const Phys &ph) {
  constexpr int NV = DIM + 2;
  auto G = [&](int a, int b) { return g[a * NV + b]; };
  R rho = U[0], u = U[1] / rho, v = U[2] / rho;
  R e = U[DIM + 1] / rho - (R)0.5 * (u * u + v * v);
  R w = 0;
  if constexpr (DIM == 3) {
    w = U[3] / rho;
    e -= (R)0.5 * (w * w);
  }
  R dRho_dx = G(0, 0), dRhoU_dx = G(0, 1), dRhoV_dx = G(0, 2), dE_dx = G(0, DIM + 1);
  R dRho_dy = G(1, 0), dRhoU_dy = G(1, 1), dRhoV_dy = G(1, 2), dE_dy = G(1, DIM + 1);
  R dRho_dz = 0, dRhoU_dz = 0, dRhoW_dx = 0, dRhoW_dy = 0, dRhoW_dz = 0, dE_dz = 0;
  if constexpr (DIM == 3) {
    dRho_dz = G(2, 0); dRhoU_dz = G(2, 1);
    dRhoW_dx = G(0, 3); dRhoW_dy = G(1, 3); dRhoW_dz = G(2, 3); dE_dz = G(2, 4);
  }
  R mu = (R)ph.mu;
  if (!ph.fixVis) {  // Sutherland's law
    R rt = ((R)ph.gamma - (R)1.0) * e / (R)ph.rt_inf;
    mu *= pow(rt, (R)1.5) * ((R)1. + (R)ph.c_sth) / (rt + (R)ph.c_sth);
  }
  R du_dx = (dRhoU_dx - dRho_dx * u) / rho, du_dy = (dRhoU_dy - dRho_dy * u) / rho;
  R dv_dx = (dRhoV_dx - dRho_dx * v) / rho, dv_dy = (dRhoV_dy - dRho_dy * v) / rho;
  R du_dz = 0, dw_dx = 0, dw_dy = 0, dw_dz = 0;
  if constexpr (DIM == 3) {
    du_dz = (dRhoU_dz - dRho_dz * u) / rho;
    dw_dx = (dRhoW_dx - dRho_dx * w) / rho;
    dw_dy = (dRhoW_dy - dRho_dy * w) / rho;
    dw_dz = (dRhoW_dz - dRho_dz * w) / rho;
  }
  R dK_dx, dK_dy, dK_dz = 0;
  if constexpr (DIM == 2) {
    dK_dx = (R)0.5 * (u * u + v * v) * dRho_dx + rho * (u * du_dx + v * dv_dx);
    dK_dy = (R)0.5 * (u * u + v * v) * dRho_dy + rho * (u * du_dy + v * dv_dy);
  } else {
    // the reference also forms dv/dz here; it only enters dK_dz
    R dv_dz = (G(2, 2) - dRho_dz * v) / rho;
    dK_dx = (R)0.5 * (u * u + v * v + w * w) * dRho_dx + rho * (u * du_dx + v * dv_dx + w * dw_dx);
    dK_dy = (R)0.5 * (u * u + v * v + w * w) * dRho_dy + rho * (u * du_dy + v * dv_dy + w * dw_dy);
    dK_dz = (R)0.5 * (u * u + v * v + w * w) * dRho_dz + rho * (u * du_dz + v * dv_dz + w * dw_dz);
  }
  R de_dx = (dE_dx - dK_dx - dRho_dx * e) / rho;
  R de_dy = (dE_dy - dK_dy - dRho_dy * e) / rho;
  R de_dz = 0;
  if constexpr (DIM == 3) de_dz = (dE_dz - dK_dz - dRho_dz * e) / rho;
  R diag = (du_dx + dv_dy + dw_dz) / (R)3.0;
  R tauxx = (R)2.0 * mu * (du_dx - diag), tauyy = (R)2.0 * mu * (dv_dy - diag);
  R tauxy = mu * (du_dy + dv_dx);
  R tauxz = 0, tauyz = 0, tauzz = 0;
  if constexpr (DIM == 3) {
    tauxz = mu * (du_dz + dv_dx);
    tauyz = mu * (du_dz + dv_dy);
    tauzz = (R)2.0 * mu * (dw_dz - diag);
  }
  const R kap = (mu / (R)ph.prandtl) * (R)ph.gamma;
  Fv[0][0] = 0; Fv[0][1] = -tauxx; Fv[0][2] = -tauxy;
  Fv[0][DIM + 1] = -(u * tauxx + v * tauxy + w * tauxz + kap * de_dx);
  Fv[1][0] = 0; Fv[1][1] = -tauxy; Fv[1][2] = -tauyy;
  Fv[1][DIM + 1] = -(u * tauxy + v * tauyy + w * tauyz + kap * de_dy);
  if constexpr (DIM == 3) {
    Fv[0][3] = -tauzz; Fv[1][3] = -tauyz;
    Fv[2][0] = 0; Fv[2][1] = -tauxz; Fv[2][2] = -tauyz; Fv[2][3] = -tauzz;
    Fv[2][4] = -(u * tauxz + v * tauyz + w * tauzz + kap * de_dz);
  }
}

// viscousFluxAD (src/flux.cpp:361-366): -D grad u.
template <int DIM, typename R>
__device__ __forceinline__ void viscous_flux_ad(const R *g, R Fv[DIM][1], const Phys &ph) {
#pragma unroll
  for (int d = 0; d < DIM; d++) Fv[d][0] = -(R)ph.diffD * g[d];
}

// boundFace::applyViscousBCs, adiabatic no-slip wall (src/boundFace.cpp:279-320):
// the ghost gradient is the interior one with its energy row rebuilt so the
// temperature gradient vanishes.  gL, gR are [DIM][NV].
template <int DIM, typename R>
__device__ __forceinline__ void adiabatic_gradient(const R *UL, const R *UR, const R *gL, R *gR, const Phys &ph) {
  constexpr int NV = DIM + 2;
  for (int i = 0; i < DIM * NV; i++) gR[i] = gL[i];
  R rhovSq = 0;
  for (int d = 0; d < DIM; d++) rhovSq += UL[d + 1] * UL[d + 1];
  R pL = ((R)ph.gamma - (R)1.) * (UL[DIM + 1] - (R)0.5 * rhovSq / UL[0]);
  R e = pL / (((R)ph.gamma - (R)1.) * UR[0]);
  R gv[DIM][DIM];
  for (int a = 0; a < DIM; a++)
    for (int b = 0; b < DIM; b++) gv[a][b] = (gR[a * NV + b + 1] - gR[a * NV] * UR[b + 1] / UR[0]) / UR[0];
  R vSq = 0;
  for (int d = 0; d < DIM; d++) vSq += UR[d + 1] * UR[d + 1] / (UR[0] * UR[0]);
  for (int a = 0; a < DIM; a++) {
    gR[a * NV + DIM + 1] = (e + (R)0.5 * vSq) * gR[a * NV];
    for (int b = 0; b < DIM; b++) gR[a * NV + DIM + 1] += UR[b + 1] * gv[b][a];
  }
}

// boundFace::applyBCs for Euler/Navier-Stokes (src/boundFace.cpp:33-277).
// T is double in the solver, a dual number in the adjoint (which also carries
// the derivative of the boundary state rhoB / vB / pB with respect to a
// freestream parameter).  Returns false for an unknown BC.
template <int DIM, typename T>
__device__ __forceinline__ bool bc_ghost_t(int bc, const T *UL, const double *n, T *UR, const Phys &ph,
                                           const T &rhoB, const T *vB, const T &pB) {
  T rhoR = 0, pR = 0, ER = 0;
  T vL[3] = {0, 0, 0}, vR[3] = {0, 0, 0};
  const double gamma = ph.gamma, gmo = gamma - 1.;
  T rhoL = UL[0], eL = UL[DIM + 1];
  for (int i = 0; i < DIM; i++) vL[i] = UL[i + 1] / UL[0];
  T vSq = 0;
  for (int i = 0; i < DIM; i++) vSq += (vL[i] * vL[i]);
  T pL = (gamma - 1.0) * (eL - 0.5 * rhoL * vSq);
  switch (bc) {
    case BC_SUB_IN:
      rhoR = rhoB;
      for (int i = 0; i < DIM; i++) vR[i] = vB[i];
      pR = pL;
      vSq = 0;
      for (int i = 0; i < DIM; i++) vSq += (vR[i] * vR[i]);
      ER = (pR / (gamma - 1.0)) + 0.5 * rhoR * vSq;
      break;
    case BC_SUB_OUT:
      rhoR = rhoL;
      for (int i = 0; i < DIM; i++) vR[i] = vL[i];
      pR = pB;
      vSq = 0.;
      for (int i = 0; i < DIM; i++) vSq += (vR[i] * vR[i]);
      ER = (pR / (gamma - 1.0)) + 0.5 * rhoR * vSq;
      break;
    case BC_SUP_IN:
      rhoR = rhoB;
      vR[0] = vB[0]; vR[1] = vB[1]; vR[2] = vB[2];
      pR = pB;
      vSq = 0.;
      for (int i = 0; i < DIM; i++) vSq += (vR[i] * vR[i]);
      ER = (pR / (gamma - 1.0)) + 0.5 * rhoR * vSq;
      break;
    case BC_SUP_OUT:
      rhoR = rhoL;
      for (int i = 0; i < DIM; i++) vR[i] = vL[i];
      ER = eL;
      break;
    case BC_SLIP:
    case BC_SYMMETRY: {
      rhoR = rhoL;
      T vnL = 0.;
      for (int i = 0; i < DIM; i++) vnL += (vL[i] - 0.0) * n[i];
      for (int i = 0; i < DIM; i++) vR[i] = vL[i] - (2.0) * vnL * n[i];
      ER = eL;
      break;
    }
    case BC_ISO_NOSLIP_MOVING:
    case BC_ISO_NOSLIP: {
      pR = pL;
      rhoR = pR / (ph.RGas * ph.TWall);
      for (int i = 0; i < DIM; i++) vR[i] = bc == BC_ISO_NOSLIP_MOVING ? 0.0 + ph.vWall[i] : 0.0;
      vSq = 0.;
      for (int i = 0; i < DIM; i++) vSq += (vR[i] * vR[i]);
      ER = (pR / (gamma - 1.0)) + 0.5 * rhoR * vSq;
      break;
    }
    case BC_ADI_NOSLIP:
      rhoR = rhoL;
      pR = pL;
      for (int i = 0; i < DIM; i++) vR[i] = 0.0;
      vSq = 0.;
      for (int i = 0; i < DIM; i++) vSq += (vR[i] * vR[i]);
      ER = (pR / (gamma - 1.0)) + 0.5 * rhoR * vSq;
      break;
    case BC_CHAR: {
      T vnL = 0., vnB = 0.;
      for (int i = 0; i < DIM; i++) vnL += vL[i] * n[i];
      for (int i = 0; i < DIM; i++) vnB += vB[i] * n[i];
      T cL = sqrt(gamma * pL / rhoL);
      T cB = sqrt(gamma * pB / rhoB);
      T R_L, R_B;
      if (fabs(vnB) >= cB && vnL >= 0) R_L = vnB + 2. / gmo * cB;
      else R_L = vnL + 2. / gmo * cL;
      if (fabs(vnB) >= cB && vnL < 0) R_B = vnL - 2. / gmo * cL;
      else R_B = vnB - 2. / gmo * cB;
      T rhoFac = .25 * (gamma - 1.) * (R_L - R_B);
      T rhoBG = rhoFac * rhoFac / gamma;
      if (vnL < 0) rhoBG *= pow(rhoB, gamma) / pB;
      else rhoBG *= pow(rhoL, gamma) / pL;
      rhoR = pow(rhoBG, 1. / gmo);
      pR = rhoFac * rhoFac * rhoR / gamma;
      T VB = 0.5 * (R_L + R_B);
      for (int i = 0; i < DIM; i++) {
        if (vnL < 0) vR[i] = vB[i] + (VB - vnB) * n[i];
        else vR[i] = vL[i] + (VB - vnL) * n[i];
      }
      T vMag2 = 0;
      for (int i = 0; i < DIM; i++) vMag2 += vR[i] * vR[i];
      ER = pR / gmo + .5 * rhoR * vMag2;
      break;
    }
    default:
      return false;
  }
  UR[0] = rhoR;
  for (int i = 0; i < DIM; i++) UR[i + 1] = rhoR * vR[i];
  UR[DIM + 1] = ER;
  return true;
}

template <int DIM>
__device__ bool bc_ghost(int bc, const double *UL, const double *n, double *UR, const Phys &ph) {
  const double vB[3] = {ph.vB[0], ph.vB[1], ph.vB[2]};
  return bc_ghost_t<DIM, double>(bc, UL, n, UR, ph, ph.rhoB, vB, ph.pB);
}

}  // namespace frg
