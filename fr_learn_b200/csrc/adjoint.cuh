// adjoint.cuh -- discrete adjoint (vector-Jacobian products) of one FR
// residual evaluation, and its fusion into the reverse sweep of the explicit
// RK update.  FP64 throughout.  There is no adjoint in the reference; these
// kernels transpose, operation by operation, the forward residual that the
// stage kernels compute (calcResidual, src/solver.cpp:252-291):
//
//   traces   U_f   = sum_j lag[side][j] U[line pt j]              (extrapolateU)
//   fluxes   Fs_d1 = sum_d2 JGinv[d1][d2] F_d2(U)                 (calcInviscidFlux_spts)
//   normal   dis   = +-sum_j lag[side][j] Fs_dir[line pt j]       (extrapolateNormalFlux)
//   common   Fn    = Riemann(U_L, U_R, n); jump J = +-Fn dA - dis (face::calcInviscidFlux)
//   residual divF  = sum_d sum_q dlag[i_d][q] Fs_d[line pt q] + sum_c g_c J[f_c]
//                                                                 (calcDivF_spts, correctDivFlux)
//
// Given gbar = dJ/d(divF) at the solution points, the transposed chain is
//   Jbar[f]      = sum_j g(side, j) gbar[line pt j]               (correction^T)
//   fbar[f]      = +-dA Jbar[f] from this element's copy of the common flux
//                  plus the neighbour's copy (both elements evaluate the same
//                  face flux), gathered from the face-seed pass
//   Ubar_f       = (dFn/dU_own)^T fbar   (dual numbers; on boundaries the
//                  ghost state is differentiated with the interior state, and
//                  the freestream-parameter column gives dJ/dtheta)
//   Fsbar_d[s]   = sum_i dlag[i][c_d(s)] gbar[line pt i] - sum_f (+-) lag Jbar[f]
//   Ubar[s]      = sum_d (dF_d/dU)^T (sum_d1 JGinv[d1][d] Fsbar_d1) + sum_f lag Ubar_f
//
// Two launches per residual: fr_adj_face_kernel (per flux point: the trace of
// the stage state and this element's share of the common-flux adjoint) and
// fr_adj_elem_kernel (per element tile: everything else).  In the reverse RK
// sweep the element kernel also forms the next stage's seed and accumulates
// the adjoint of the step's initial state, so a reverse step is 2 x nRK
// launches.
#pragma once
#include "dual.cuh"
#include "kernels.cuh"

namespace frg {

// Scratch of the viscous adjoint (adjoint_visc.cuh), FP64 [..][point][element].
struct AdjViscBufs {
  double *g;      // forward corrected gradient at the solution points [DIM][NV][NS][L]
  double *fvn;    // each side's projected viscous flux [NV][NF][L] (interior flux points)
  double *fvn2;   // 3D LDG penalty: the left side's projection [NV][NF][L]
  double *ub;     // state adjoint at the solution points [NV][NS][L]
  double *ufb;    // trace adjoint at the flux points [NV][NF][L]
  double *dcb;    // adjoint of the LDG correction Dc = Uc - U_f [NV][NF][L]
  int visc2;
};

struct AdjArgs {
  int nE, nEle;           // element stride (padded) and real element count
  const double *Y;        // stage state [NV][NS][nE]
  const double *gbar;     // seed dJ/d(divF) [NV][NS][nE]
  double *trY;            // traces of Y [NV][NF][nE] (face kernel out)
  double *fnbar;          // this element's common-flux adjoint [NV][NF][nE] (face kernel out)
  const int *nbr;         // [NF][nE]
  const double *nrm, *dA, *JG, *detJ;
  int vcjh;
  unsigned *err;
  // outputs of the element kernel
  double *ybar;           // (ADJ_PLAIN) Ybar = (d divF / dY)^T gbar
  const double *lam;      // (RK) adjoint of the step's final state
  double *lamNew;         // (RK) adjoint of the step's initial state, accumulated
  double *seedOut;        // (RK) seed of the stage before
  double cLam, cY;        // seedOut = -(cLam * base + cY * ybar) * dt / detJ
  double dt;
  int mode;               // ADJ_* flags
  const double *thetaDir; // d(rhoB, vB[0..2], pB) / d(theta) of the boundary state (device, 5)
  const int *grp;         // ensemble mode: group of each element, else null
  const double *dtGrp;    // ensemble mode: fixed dt per group (replaces dt)
  double *thetaBar;       // += fbar . dFn/dtheta over boundary flux points
  AdjViscBufs v;          // viscous runs only
  Phys ph;
};

enum : int {
  ADJ_PLAIN = 1,      // write ybar only
  ADJ_RK_FIRST = 2,   // the last RK stage, the first reversed: lamNew = lam + ybar
  ADJ_RK_LAST = 4,    // RK stage 0, the last reversed: seedOut from the finished lamNew
  ADJ_RK = 8          // fused reverse-RK outputs
};

template <class C, typename T>
__device__ __forceinline__ void adj_common(const T *UL, const T *UR, const T *n, int code, T *Fn, const Phys &ph,
                                           int rs) {
  constexpr int NV = C::NV, DIM = C::DIM;
  if constexpr (NV == 1) {
    lax_friedrichs<DIM, T>(UL[0], UR[0], n, Fn, ph);
  } else if constexpr (DIM == 3) {
    rusanov<DIM, NV, T, T>(UL, UR, n, Fn, ph);
  } else {
    // boundary faces always use Rusanov (src/face.cpp:142-145)
    if (rs == 0 || code < 0) rusanov<DIM, NV, T, T>(UL, UR, n, Fn, ph);
    else roe2d<T, T>(UL, UR, n, Fn, ph);
  }
}

// Face-seed pass: one thread per (flux point, element).
template <class C>
__global__ void __launch_bounds__(256) fr_adj_face_kernel(const AdjArgs a) {
  constexpr int NV = C::NV, NF = C::NF, NS = C::NS, N1 = C::N1;
  const OpTab<double> &op = optab<double>(a.vcjh, C::P);
  const long n = (long)NF * a.nE;
  for (long it = blockIdx.x * (long)blockDim.x + threadIdx.x; it < n; it += (long)gridDim.x * blockDim.x) {
    const int f = (int)(it / a.nE), eg = (int)(it - (long)f * a.nE);
    if (eg >= a.nEle) continue;
    int dir, side, s0, st;
    fpt_line<C>(f, dir, side, s0, st);
    const int code = a.nbr[(size_t)f * a.nE + eg];
    const bool right = code >= 0 && (code & 1);
    const double dA = a.dA[(size_t)f * a.nE + eg];
#pragma unroll
    for (int v = 0; v < NV; v++) {
      double t = 0, jb = 0;
#pragma unroll
      for (int j = 0; j < N1; j++) {
        const size_t gi = ((size_t)v * NS + s0 + j * st) * a.nE + eg;
        t += op.lag[side][j] * a.Y[gi];
        jb += (side ? op.gR[j] : -op.gL[j]) * a.gbar[gi];
      }
      a.trY[((size_t)v * NF + f) * a.nE + eg] = t;
      a.fnbar[((size_t)v * NF + f) * a.nE + eg] = (right ? -dA : dA) * jb;
    }
  }
}

template <class C>
struct AdjTile {
  static constexpr int PER_ELE = (2 * C::NV * C::NS + 2 * C::NV * C::NF) * 8;
  // at most 8 elements per block: the dual-number Jacobians need many
  // registers, so small tiles keep every SM busy on meshes of a few
  // thousand elements
  static constexpr int TE = (8 * PER_ELE <= 64 * 1024) ? 8 : (4 * PER_ELE <= 64 * 1024) ? 4
                            : (2 * PER_ELE <= 64 * 1024) ? 2 : 1;
  static constexpr int NT = 128;
  static constexpr int SMEM = TE * PER_ELE;
};

// Element pass: one block per tile of TE elements.  Registers are capped for
// four blocks per SM on periodic meshes; the boundary variants, which also
// carry the ghost states' Jacobians, spill about 2 KB a thread at that cap
// (1.2 KB at three) and run faster capped for three.
template <class C, bool BC, int RS>
__global__ void __launch_bounds__(128, BC ? 3 : 4) fr_adj_elem_kernel(const AdjArgs a) {
  using T = AdjTile<C>;
  constexpr int TE = T::TE, NT = T::NT, NS = C::NS, NF = C::NF, NV = C::NV, DIM = C::DIM, N1 = C::N1;
  // own trace, and with boundaries the freestream parameter the ghost states take
  using D1 = ad::Dual<BC ? NV + 1 : NV>;
  using D0 = ad::Dual<NV>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *sY = reinterpret_cast<double *>(smem_raw);
  double *sG = sY + NV * NS * TE;
  double *sUf = sG + NV * NS * TE;
  double *sDis = sUf + NV * NF * TE;
  __shared__ double red[NT / 32];

  const OpTab<double> &op = optab<double>(a.vcjh, C::P);
  const int tid = threadIdx.x, e0 = blockIdx.x * TE, L = a.nE;
  const Phys &ph = a.ph;
  for (int it = tid; it < NS * TE; it += NT) {
    const int s = it / TE, e = it - s * TE, eg = e0 + e;
#pragma unroll
    for (int v = 0; v < NV; v++) {
      const size_t gi = ((size_t)v * NS + s) * L + eg;
      sY[(v * NS + s) * TE + e] = eg < a.nEle ? a.Y[gi] : 1.0;
      sG[(v * NS + s) * TE + e] = eg < a.nEle ? a.gbar[gi] : 0.0;
    }
  }
  __syncthreads();

  // ---- phase 1: per flux point, the adjoint of the own trace
  double thetaLocal = 0;
  for (int it = tid; it < NF * TE; it += NT) {
    const int f = it / TE, e = it - f * TE, eg = e0 + e;
    if (eg >= a.nEle) continue;
    int dir, side, s0, st;
    fpt_line<C>(f, dir, side, s0, st);
    const int code = a.nbr[(size_t)f * L + eg];
    const bool right = code >= 0 && (code & 1);
    const double dA = a.dA[(size_t)f * L + eg];
    double own[NV], jb[NV], fb[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) {
      double t = 0, q = 0;
#pragma unroll
      for (int j = 0; j < N1; j++) {
        t += op.lag[side][j] * sY[(v * NS + s0 + j * st) * TE + e];
        q += (side ? op.gR[j] : -op.gL[j]) * sG[(v * NS + s0 + j * st) * TE + e];
      }
      own[v] = t;
      jb[v] = q;
      fb[v] = (right ? -dA : dA) * q;
    }
    double nd[DIM];
    D1 nT[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      nd[d] = a.nrm[((size_t)d * NF + f) * L + eg];
      nT[d] = D1(nd[d]);
    }
    D1 Uo[NV], Ot[NV], Fn[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) {
      Uo[v] = D1(own[v]);
      Uo[v].d[v] = 1.0;
    }
    if (code >= 0) {
      const size_t t = (size_t)(code >> 1);
#pragma unroll
      for (int v = 0; v < NV; v++) {
        Ot[v] = D1(a.trY[(size_t)v * NF * L + t]);
        fb[v] += a.fnbar[(size_t)v * NF * L + t];
      }
      adj_common<C, D1>(right ? Ot : Uo, right ? Uo : Ot, nT, code, Fn, ph, RS);
    } else {
      if constexpr (NV == 1 || !BC) {
#pragma unroll
        for (int v = 0; v < NV; v++) Ot[v] = D1(0.0);  // advection ghost state stays zero
        if constexpr (!BC) atomicOr(a.err, ERRF_BC);
      } else {
        D1 rhoB(ph.rhoB), pB(ph.pB), vB[3] = {D1(ph.vB[0]), D1(ph.vB[1]), D1(ph.vB[2])};
        rhoB.d[NV] = a.thetaDir[0];
        vB[0].d[NV] = a.thetaDir[1];
        vB[1].d[NV] = a.thetaDir[2];
        vB[2].d[NV] = a.thetaDir[3];
        pB.d[NV] = a.thetaDir[4];
        if (!bc_ghost_t<DIM, D1>(-1 - code, Uo, nd, Ot, ph, rhoB, vB, pB)) atomicOr(a.err, ERRF_BC);
      }
      adj_common<C, D1>(Uo, Ot, nT, code, Fn, ph, RS);
    }
#pragma unroll
    for (int w = 0; w < NV; w++) {
      double ub = 0;
#pragma unroll
      for (int v = 0; v < NV; v++) ub += fb[v] * Fn[v].d[w];
      sUf[(w * NF + f) * TE + e] = ub;
      sDis[(w * NF + f) * TE + e] = -jb[w];
    }
    if constexpr (BC) {
      if (code < 0)
#pragma unroll
        for (int v = 0; v < NV; v++) thetaLocal += fb[v] * Fn[v].d[NV];
    }
  }
  if constexpr (BC) {
    if (a.thetaBar) {
      for (int o = 16; o > 0; o >>= 1) thetaLocal += __shfl_xor_sync(0xffffffffu, thetaLocal, o);
      if ((tid & 31) == 0) red[tid >> 5] = thetaLocal;
    }
  }
  __syncthreads();
  if constexpr (BC) {
    if (a.thetaBar && tid == 0) {
      double t = 0;
      for (int w = 0; w < NT / 32; w++) t += red[w];
      if (t != 0) atomicAdd(a.thetaBar, t);
    }
  }

  // ---- phase 2: per solution point
  for (int it = tid; it < NS * TE; it += NT) {
    const int s = it / TE, e = it - s * TE, eg = e0 + e;
    if (eg >= a.nEle) continue;
    const int i = s % N1, j = (s / N1) % N1, k = DIM == 3 ? s / (N1 * N1) : 0;
    const int ijk[3] = {i, j, k};
    int cf[2 * DIM], cs[2 * DIM], ca[2 * DIM], cd[2 * DIM];
    corr_fpts<C>(i, j, k, cf, cs, ca);
#pragma unroll
    for (int c = 0; c < 2 * DIM; c++) {
      int dir, side, s0, st;
      fpt_line<C>(cf[c], dir, side, s0, st);
      cd[c] = dir;
    }
    double Fsb[DIM][NV];
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      const int sd = d == 0 ? 1 : d == 1 ? N1 : N1 * N1;
      const int sb = s - ijk[d] * sd;
#pragma unroll
      for (int v = 0; v < NV; v++) {
        double t = 0;
#pragma unroll
        for (int q = 0; q < N1; q++) t += op.dlag[q][ijk[d]] * sG[(v * NS + sb + q * sd) * TE + e];
#pragma unroll
        for (int c = 0; c < 2 * DIM; c++)
          if (cd[c] == d) t += (cs[c] ? 1.0 : -1.0) * op.lag[cs[c]][ca[c]] * sDis[(v * NF + cf[c]) * TE + e];
        Fsb[d][v] = t;
      }
    }
    // physical-flux adjoint, then through the flux Jacobians
    double Fb[DIM][NV];
#pragma unroll
    for (int d2 = 0; d2 < DIM; d2++)
#pragma unroll
      for (int v = 0; v < NV; v++) {
        double t = 0;
#pragma unroll
        for (int d1 = 0; d1 < DIM; d1++) t += a.JG[((size_t)(d1 * DIM + d2) * NS + s) * L + eg] * Fsb[d1][v];
        Fb[d2][v] = t;
      }
    D0 u[NV], F[DIM][NV];
#pragma unroll
    for (int v = 0; v < NV; v++) {
      u[v] = D0(sY[(v * NS + s) * TE + e]);
      u[v].d[v] = 1.0;
    }
    inviscid_flux<DIM, NV, D0>(u, F, ph);
    const double idet = 1.0 / a.detJ[(size_t)s * L + eg];
#pragma unroll
    for (int w = 0; w < NV; w++) {
      double yb = 0;
#pragma unroll
      for (int d = 0; d < DIM; d++)
#pragma unroll
        for (int v = 0; v < NV; v++) yb += Fb[d][v] * F[d][v].d[w];
#pragma unroll
      for (int c = 0; c < 2 * DIM; c++) yb += op.lag[cs[c]][ca[c]] * sUf[(w * NF + cf[c]) * TE + e];
      const size_t gi = ((size_t)w * NS + s) * L + eg;
      if (a.mode & ADJ_PLAIN) a.ybar[gi] = yb;
      if (a.mode & ADJ_RK) {
        // the adjoint of the step's initial state collects every stage's ybar
        const double base = (a.mode & ADJ_RK_FIRST) ? a.lam[gi] : a.lamNew[gi];
        const double ln = base + yb;
        a.lamNew[gi] = ln;
        const double D = (a.grp ? a.dtGrp[a.grp[eg]] : a.dt) * idet;
        if (a.mode & ADJ_RK_LAST) a.seedOut[gi] = -a.cLam * ln * D;
        else a.seedOut[gi] = -(a.cLam * a.lam[gi] + a.cY * yb) * D;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Objectives and their gradients with respect to the solution-point state.
// ---------------------------------------------------------------------------

// Entropy error integral, sum_e sum_s w_s detJ (p rhoB^gamma / (rho^gamma pB) - 1)
// (integrateError with the freestream entropy error, src/solver.cpp:1507-1531;
// src/funcs.cpp:1891-1901).  Per-block partial sums in `part`.
template <int DIM, int NV>
__global__ void __launch_bounds__(256) fr_obj_entropy_kernel(const double *U, const double *detJ,
                                                             const double *wvol, int NS, int nE, int L,
                                                             Phys ph, double *grad, double *part) {
  using D0 = ad::Dual<NV>;
  __shared__ double red[8];
  double acc = 0;
  const long n = (long)NS * L;
  const double rfg = pow(ph.rhoB, ph.gamma);
  for (long it = blockIdx.x * (long)blockDim.x + threadIdx.x; it < n; it += (long)gridDim.x * blockDim.x) {
    const int s = (int)(it / L), e = (int)(it - (long)s * L);
    if (e >= nE) {
      for (int v = 0; v < NV; v++) grad[(size_t)v * NS * L + it] = 0;
      continue;
    }
    D0 u[NV];
    for (int v = 0; v < NV; v++) {
      u[v] = D0(U[(size_t)v * NS * L + it]);
      u[v].d[v] = 1.0;
    }
    D0 ke = 0;
    for (int d = 0; d < DIM; d++) ke += u[d + 1] * u[d + 1];
    const D0 p = (ph.gamma - 1.) * (u[DIM + 1] - .5 * ke / u[0]);
    const D0 err = p * rfg / (ad::pow(u[0], ph.gamma) * ph.pB) - 1.;
    const double wj = wvol[s] * detJ[it];
    acc += err.v * wj;
    for (int v = 0; v < NV; v++) grad[(size_t)v * NS * L + it] = err.d[v] * wj;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    part[blockIdx.x] = t;
  }
}

// Pressure integrated over the slip-wall faces with the face quadrature of
// boundFace::computeWallForce (src/boundFace.cpp:330-378): sum w_f p(U_f) dA_f
// over wall flux points, U_f the element's trace.  One thread per element;
// `grad` must be zero on entry (only wall elements write).
template <class C>
__global__ void __launch_bounds__(128) fr_obj_wallp_kernel(const double *U, const int *nbr, const double *dA,
                                                           const double *wsurf, int vcjh, int nE, int L, int bcWall,
                                                           Phys ph, double *grad, double *part) {
  constexpr int NV = C::NV, NS = C::NS, NF = C::NF, N1 = C::N1, DIM = C::DIM;
  using D0 = ad::Dual<NV>;
  const OpTab<double> &op = optab<double>(vcjh, C::P);
  __shared__ double red[4];
  double acc = 0;
  const int eg = blockIdx.x * blockDim.x + threadIdx.x;
  if (eg < nE) {
    for (int f = 0; f < NF; f++) {
      const int code = nbr[(size_t)f * L + eg];
      if (code >= 0 || -1 - code != bcWall) continue;
      int dir, side, s0, st;
      fpt_line<C>(f, dir, side, s0, st);
      D0 u[NV];
      for (int v = 0; v < NV; v++) {
        double t = 0;
        for (int j = 0; j < N1; j++) t += op.lag[side][j] * U[((size_t)v * NS + s0 + j * st) * L + eg];
        u[v] = D0(t);
        u[v].d[v] = 1.0;
      }
      D0 ke = 0;
      for (int d = 0; d < DIM; d++) ke += u[d + 1] * u[d + 1] / (u[0] * u[0]);
      const D0 p = (ph.gamma - 1) * (u[DIM + 1] - 0.5 * u[0] * ke);
      const double wd = wsurf[f % C::NFF] * dA[(size_t)f * L + eg];
      acc += p.v * wd;
      for (int v = 0; v < NV; v++)
        for (int j = 0; j < N1; j++) grad[((size_t)v * NS + s0 + j * st) * L + eg] += op.lag[side][j] * p.d[v] * wd;
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    part[blockIdx.x] = t;
  }
}

}  // namespace frg
