// adjoint_visc.cuh -- vector-Jacobian product of a VISCOUS (LDG) residual
// evaluation, FP64.  The forward residual (the generic viscous kernels,
// kernels.cuh) is, per element, with U the stage state:
//
//   traces     U_f  = sum_j lag[side][j] U[line pt j]
//   LDG        Dc_f = Uc(U_L, U_R, n) - U_f         (face::ldgSolution)
//   gradient   gr_d = sum_q dlag U[line_d pt q] + sum_{f on d} gcorr Dc_f
//              g_d1 = (1/detJ) sum_d2 gr_d2 JGinv[d2][d1]  (calcGradU_spts,
//                                                   correctGradU)
//   fluxes     Fs_d1 = sum_d2 JGinv[d1][d2] (F_inv + F_vis)(U, g)
//   grad trace g_f  = sum_j lag[side][j] g[line pt j]   (extrapolateGradU)
//   common     Fn   = Riemann(U_L, U_R) + LDG viscous flux of both sides'
//                     projected viscous fluxes, or the boundary's
//   residual   divF = sum_d D_d Fs_d + C (+-Fn dA - disFn)
//
// The transposed chain runs in three element passes after the face-seed
// pass of the inviscid adjoint (traces of the stage state and this side's
// share +-dA C^T gbar of the common-flux adjoint):
//   pass 1  the forward gradient and each side's projected viscous flux (the
//           generic gradient kernel, fr_visc_grad_kernel), which the
//           neighbours' face fluxes read as constants;
//   pass 2  per flux point, the own-side Jacobian of the common flux
//           (both elements evaluate the same face flux, each differentiates
//           with respect to its own trace and gradient trace); per solution
//           point, the Jacobian of the point flux with respect to the state
//           and the gradient; the gradient's adjoint taken back through the
//           metric transform, the derivative operator (into Ubar) and the
//           correction (into the adjoint of the common solution, Dcbar);
//   pass 3  the common solution's adjoint of both sides (this side's Dcbar
//           plus the neighbour's, gathered) through Uc's dependence on this
//           side's trace, then every trace adjoint back to the solution
//           points, and the outputs (ybar, or the reverse-RK update).
// Pointwise Jacobians come from dual numbers, a few tangent directions at a
// time (vjp_chunked) to bound the register use.
#pragma once
#include <type_traits>

#include "adjoint.cuh"

namespace frg {

// xbar += J(x)^T ybar for y = f(x), NI inputs and NO outputs, with K tangent
// directions per evaluation of f (templated on the dual type).
template <int NI, int NO, int K, int C0 = 0, class F>
__device__ __forceinline__ void vjp_chunked(const double *x, const double *ybar, double *xbar, F &f) {
  if constexpr (C0 < NI) {
    using D = ad::Dual<K>;
    D X[NI], Y[NO];
#pragma unroll
    for (int i = 0; i < NI; i++) {
      X[i] = D(x[i]);
      if (i >= C0 && i < C0 + K) X[i].d[i - C0] = 1.0;
    }
    f(X, Y);
#pragma unroll
    for (int k = 0; k < K; k++) {
      if (C0 + k < NI) {
        double t = 0;
#pragma unroll
        for (int o = 0; o < NO; o++) t += ybar[o] * Y[o].d[k];
        xbar[C0 + k] += t;
      }
    }
    vjp_chunked<NI, NO, K, C0 + K>(x, ybar, xbar, f);
  }
}

template <class C>
struct AdjViscTile {
  static constexpr int NV = C::NV, NS = C::NS, NF = C::NF, D = C::DIM;
  // elements per block of pass 2: Y, gbar, g, Ubar (spts); dis, Ufbar,
  // gfbar (fpts) in FP64 within ~64 KB
  static constexpr int PER_ELE = (2 * NV * NS + D * NV * NS + NV * NS + 2 * NV * NF + D * NV * NF) * 8;
  static constexpr int TE = (4 * PER_ELE <= 64 * 1024) ? 4 : (2 * PER_ELE <= 64 * 1024) ? 2 : 1;
  static constexpr int NT = 128;
  static constexpr int SMEM = TE * PER_ELE;
};

// The ghost state of a boundary flux point in dual numbers, with the
// freestream parameter as the last input (value 0, direction thetaDir).
template <class C, typename T>
__device__ __forceinline__ void adjv_ghost(const AdjArgs &a, int code, const T *own, const double *nd, const T &th,
                                           T *oth) {
  constexpr int NV = C::NV, DIM = C::DIM;
  if constexpr (NV == 1) {
#pragma unroll
    for (int v = 0; v < NV; v++) oth[v] = T(0.0);  // advection ghost state stays zero
  } else {
    const Phys &ph = a.ph;
    T rhoB = T(ph.rhoB) + T(a.thetaDir[0]) * th, pB = T(ph.pB) + T(a.thetaDir[4]) * th;
    T vB[3] = {T(ph.vB[0]) + T(a.thetaDir[1]) * th, T(ph.vB[1]) + T(a.thetaDir[2]) * th,
               T(ph.vB[2]) + T(a.thetaDir[3]) * th};
    if (!bc_ghost_t<DIM, T>(-1 - code, own, nd, oth, ph, rhoB, vB, pB)) atomicOr(a.err, ERRF_BC);
  }
}

// Pass 2: the flux Jacobians and the gradient chain, per element tile.
template <class C, bool BC, int RS>
__global__ void __launch_bounds__(128) fr_adjv_elem_kernel(const AdjArgs a) {
  const AdjViscBufs &b = a.v;
  using T = AdjViscTile<C>;
  constexpr int TE = T::TE, NT = T::NT, NS = C::NS, NF = C::NF, NV = C::NV, DIM = C::DIM, N1 = C::N1;
  constexpr int NG = DIM * NV;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *sY = reinterpret_cast<double *>(smem_raw);  // [NV][NS][TE]
  double *sGb = sY + NV * NS * TE;                    // gbar [NV][NS][TE]
  double *sG = sGb + NV * NS * TE;                    // g, then the reference-gradient adjoint [NG][NS][TE]
  double *sUb = sG + NG * NS * TE;                    // [NV][NS][TE]
  double *sDis = sUb + NV * NS * TE;                  // -Jbar [NV][NF][TE]
  double *sUf = sDis + NV * NF * TE;                  // trace adjoint [NV][NF][TE]
  double *sGf = sUf + NV * NF * TE;                   // gradient-trace adjoint [NG][NF][TE]
  __shared__ double red[NT / 32];
  const OpTab<double> &op = optab<double>(a.vcjh, C::P);
  const int tid = threadIdx.x, e0 = blockIdx.x * TE, L = a.nE;
  const Phys &ph = a.ph;
  for (int it = tid; it < NS * TE; it += NT) {
    const int s = it / TE, e = it - s * TE, eg = e0 + e;
    const bool in = eg < a.nEle;
#pragma unroll
    for (int v = 0; v < NV; v++) {
      const size_t gi = ((size_t)v * NS + s) * L + eg;
      sY[(v * NS + s) * TE + e] = in ? a.Y[gi] : 1.0;
      sGb[(v * NS + s) * TE + e] = in ? a.gbar[gi] : 0.0;
    }
#pragma unroll
    for (int q = 0; q < NG; q++) sG[(q * NS + s) * TE + e] = in ? b.g[((size_t)q * NS + s) * L + eg] : 0.0;
  }
  __syncthreads();

  // ---- per flux point: the own-side Jacobian of the face flux
  double thetaLocal = 0;
  for (int it = tid; it < NF * TE; it += NT) {
    const int f = it / TE, e = it - f * TE, eg = e0 + e;
    if (eg >= a.nEle) continue;
    int dir, side, s0, st;
    fpt_line<C>(f, dir, side, s0, st);
    const int code = a.nbr[(size_t)f * L + eg];
    const bool right = code >= 0 && (code & 1);
    const size_t me = (size_t)f * L + eg;
    const double dA = a.dA[me];
    double x[NV + NG + 1], fb[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) {
      double t = 0, q = 0;
#pragma unroll
      for (int j = 0; j < N1; j++) {
        t += op.lag[side][j] * sY[(v * NS + s0 + j * st) * TE + e];
        q += (side ? op.gR[j] : -op.gL[j]) * sGb[(v * NS + s0 + j * st) * TE + e];
      }
      x[v] = t;
      fb[v] = (right ? -dA : dA) * q;
      sDis[(v * NF + f) * TE + e] = -q;
    }
#pragma unroll
    for (int qg = 0; qg < NG; qg++) {
      double t = 0;
#pragma unroll
      for (int j = 0; j < N1; j++) t += op.lag[side][j] * sG[(qg * NS + s0 + j * st) * TE + e];
      x[NV + qg] = t;
    }
    x[NV + NG] = 0.0;  // the freestream parameter
    double nd[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) nd[d] = a.nrm[((size_t)d * NF + f) * L + eg];
    double nn = 0;
#pragma unroll
    for (int d = 0; d < DIM; d++) nn += nd[d] * nd[d];
    double Un[NV] = {}, xn[NV] = {}, x2[NV] = {};
    if (code >= 0) {
      const size_t t = (size_t)(code >> 1);
#pragma unroll
      for (int v = 0; v < NV; v++) {
        Un[v] = a.trY[(size_t)v * NF * L + t];
        xn[v] = b.fvn[(size_t)v * NF * L + t];
        if constexpr (DIM == 3)
          if (b.visc2 && right) x2[v] = b.fvn2[(size_t)v * NF * L + t];
        fb[v] += a.fnbar[(size_t)v * NF * L + t];
      }
    }
    // Fn(own trace, own gradient trace, theta): the forward's face flux with
    // the neighbour's trace and projected fluxes as constants
    auto face_flux = [&](const auto *X, auto *Fo) {
      using TT = typename std::remove_cv<typename std::remove_reference<decltype(X[0])>::type>::type;
      TT n[DIM], own[NV], oth[NV], g[NG];
#pragma unroll
      for (int d = 0; d < DIM; d++) n[d] = TT(nd[d]);
#pragma unroll
      for (int v = 0; v < NV; v++) own[v] = X[v];
#pragma unroll
      for (int q = 0; q < NG; q++) g[q] = X[NV + q];
      if (code >= 0) {
#pragma unroll
        for (int v = 0; v < NV; v++) oth[v] = TT(Un[v]);
      } else {
        adjv_ghost<C, TT>(a, code, own, nd, X[NV + NG], oth);
      }
      const TT *UL = right ? oth : own;
      const TT *UR = right ? own : oth;
      adj_common<C, TT>(UL, UR, n, code, Fo, ph, RS);
      TT Fv[DIM][NV];
      visc_flux<C, TT>(own, g, Fv, ph);
      const TT tau = TT(ph.tau), tnn = TT(nn);
      if (code >= 0) {
        const TT pf = TT(ldg_pen<DIM, double>(nd, ph.penFact));
#pragma unroll
        for (int v = 0; v < NV; v++) {
          TT on = TT(0.0);
#pragma unroll
          for (int d = 0; d < DIM; d++) on = on + Fv[d][v] * n[d];
          const TT FLn = right ? TT(xn[v]) : on, FRn = right ? on : TT(xn[v]);
          if constexpr (NV == 1) {
            Fo[v] = Fo[v] + TT(0.5) * (FLn + FRn);
          } else {
            TT al = FLn;
            if constexpr (DIM == 3)
              if (b.visc2) al = right ? TT(x2[v]) : n[0] * Fv[0][v] + n[1] * Fv[1][v] + n[2] * Fv[1][v];
            Fo[v] = Fo[v] + (TT(0.5) * (FLn + FRn) + pf * tnn * (al - FRn) + tau * tnn * (UL[v] - UR[v]));
          }
        }
      } else {
        if constexpr (NV == 1) {
#pragma unroll
          for (int d = 0; d < DIM; d++) Fo[0] = Fo[0] + TT(0.5) * Fv[d][0] * n[d];
        } else if constexpr (BC) {
          TT Fb[DIM][NV];
          if (-1 - code == BC_ADI_NOSLIP) {
            TT gR[NG];
            adiabatic_gradient<DIM, TT>(UL, UR, g, gR, ph);
            visc_flux<C, TT>(UR, gR, Fb, ph);
          } else {
#pragma unroll
            for (int d = 0; d < DIM; d++)
#pragma unroll
              for (int v = 0; v < NV; v++) Fb[d][v] = Fv[d][v];
          }
#pragma unroll
          for (int v = 0; v < NV; v++) {
            TT bn = TT(0.0);
#pragma unroll
            for (int d = 0; d < DIM; d++) bn = bn + Fb[d][v] * n[d];
            Fo[v] = Fo[v] + (bn + tau * tnn * (UL[v] - UR[v]));
          }
        }
      }
    };
    double xb[NV + NG + 1] = {};
    vjp_chunked<NV + NG + 1, NV, 4>(x, fb, xb, face_flux);
#pragma unroll
    for (int v = 0; v < NV; v++) sUf[(v * NF + f) * TE + e] = xb[v];
#pragma unroll
    for (int q = 0; q < NG; q++) sGf[(q * NF + f) * TE + e] = xb[NV + q];
    if (code < 0) thetaLocal += xb[NV + NG];
  }
  if (a.thetaBar) {
    for (int o = 16; o > 0; o >>= 1) thetaLocal += __shfl_xor_sync(0xffffffffu, thetaLocal, o);
    if ((tid & 31) == 0) red[tid >> 5] = thetaLocal;
  }
  __syncthreads();
  if (a.thetaBar && tid == 0) {
    double t = 0;
    for (int w = 0; w < NT / 32; w++) t += red[w];
    if (t != 0) atomicAdd(a.thetaBar, t);
  }

  // ---- per solution point: point-flux Jacobians, gradient adjoint
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
        for (int q = 0; q < N1; q++) t += op.dlag[q][ijk[d]] * sGb[(v * NS + sb + q * sd) * TE + e];
#pragma unroll
        for (int c = 0; c < 2 * DIM; c++)
          if (cd[c] == d) t += (cs[c] ? 1.0 : -1.0) * op.lag[cs[c]][ca[c]] * sDis[(v * NF + cf[c]) * TE + e];
        Fsb[d][v] = t;
      }
    }
    double G[DIM][DIM];
#pragma unroll
    for (int d1 = 0; d1 < DIM; d1++)
#pragma unroll
      for (int d2 = 0; d2 < DIM; d2++) G[d1][d2] = a.JG[((size_t)(d1 * DIM + d2) * NS + s) * L + eg];
    double Fb[DIM * NV];
#pragma unroll
    for (int d2 = 0; d2 < DIM; d2++)
#pragma unroll
      for (int v = 0; v < NV; v++) {
        double t = 0;
#pragma unroll
        for (int d1 = 0; d1 < DIM; d1++) t += G[d1][d2] * Fsb[d1][v];
        Fb[d2 * NV + v] = t;
      }
    double x[NV + NG], xb[NV + NG] = {};
#pragma unroll
    for (int v = 0; v < NV; v++) x[v] = sY[(v * NS + s) * TE + e];
#pragma unroll
    for (int q = 0; q < NG; q++) x[NV + q] = sG[(q * NS + s) * TE + e];
    auto point_flux = [&](const auto *X, auto *Fo) {
      using TT = typename std::remove_cv<typename std::remove_reference<decltype(X[0])>::type>::type;
      TT u[NV], g[NG], Fi[DIM][NV], Fv[DIM][NV];
#pragma unroll
      for (int v = 0; v < NV; v++) u[v] = X[v];
#pragma unroll
      for (int q = 0; q < NG; q++) g[q] = X[NV + q];
      inviscid_flux<DIM, NV, TT>(u, Fi, ph);
      visc_flux<C, TT>(u, g, Fv, ph);
#pragma unroll
      for (int d = 0; d < DIM; d++)
#pragma unroll
        for (int v = 0; v < NV; v++) Fo[d * NV + v] = Fi[d][v] + Fv[d][v];
    };
    vjp_chunked<NV + NG, DIM * NV, 4>(x, Fb, xb, point_flux);
    // the gradient-trace adjoint back to this point (extrapolateGradU^T)
    double gb[NG];
#pragma unroll
    for (int q = 0; q < NG; q++) {
      double t = xb[NV + q];
#pragma unroll
      for (int c = 0; c < 2 * DIM; c++) t += op.lag[cs[c]][ca[c]] * sGf[(q * NF + cf[c]) * TE + e];
      gb[q] = t;
    }
    // physical gradient g_d1 = (1/detJ) sum_d2 gr_d2 G[d2][d1]: its adjoint on
    // the reference gradient, kept in sG (this point's slot only)
    const double invDet = 1.0 / a.detJ[(size_t)s * L + eg];
#pragma unroll
    for (int v = 0; v < NV; v++)
#pragma unroll
      for (int d2 = 0; d2 < DIM; d2++) {
        double t = 0;
#pragma unroll
        for (int d1 = 0; d1 < DIM; d1++) t += G[d2][d1] * gb[d1 * NV + v];
        sG[((d2 * NV + v) * NS + s) * TE + e] = invDet * t;
      }
#pragma unroll
    for (int v = 0; v < NV; v++) sUb[(v * NS + s) * TE + e] = xb[v];
  }
  __syncthreads();

  // ---- the reference gradient's adjoint through the derivative operators
  for (int it = tid; it < NS * TE; it += NT) {
    const int s = it / TE, e = it - s * TE, eg = e0 + e;
    if (eg >= a.nEle) continue;
    const int i = s % N1, j = (s / N1) % N1, k = DIM == 3 ? s / (N1 * N1) : 0;
    const int ijk[3] = {i, j, k};
#pragma unroll
    for (int v = 0; v < NV; v++) {
      double t = sUb[(v * NS + s) * TE + e];
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        const int sd = d == 0 ? 1 : d == 1 ? N1 : N1 * N1;
        const int sb = s - ijk[d] * sd;
#pragma unroll
        for (int q = 0; q < N1; q++) t += op.dlag[q][ijk[d]] * sG[((d * NV + v) * NS + sb + q * sd) * TE + e];
      }
      b.ub[((size_t)v * NS + s) * L + eg] = t;
    }
  }
  // ... and through the gradient corrections into the common solution
  for (int it = tid; it < NF * TE; it += NT) {
    const int f = it / TE, e = it - f * TE, eg = e0 + e;
    if (eg >= a.nEle) continue;
    int dir, side, s0, st;
    fpt_line<C>(f, dir, side, s0, st);
#pragma unroll
    for (int v = 0; v < NV; v++) {
      double t = 0;
#pragma unroll
      for (int jj = 0; jj < N1; jj++)
        t += (side ? op.gR[jj] : op.gL[jj]) * sG[((dir * NV + v) * NS + s0 + jj * st) * TE + e];
      const size_t gi = ((size_t)v * NF + f) * L + eg;
      b.dcb[gi] = t;
      b.ufb[gi] = sUf[(v * NF + f) * TE + e];
    }
  }
}

// Pass 3: the common solution's adjoint (both sides') into this side's
// trace, the traces back to the solution points, and the outputs.
template <class C, bool BC>
__global__ void __launch_bounds__(128) fr_adjv_out_kernel(const AdjArgs a) {
  const AdjViscBufs &b = a.v;
  constexpr int NS = C::NS, NF = C::NF, NV = C::NV, DIM = C::DIM, N1 = C::N1;
  constexpr int TE = 4, NT = 128;
  __shared__ double sUf[NV * NF * TE];
  __shared__ double red[NT / 32];
  const OpTab<double> &op = optab<double>(a.vcjh, C::P);
  const int tid = threadIdx.x, e0 = blockIdx.x * TE, L = a.nE;
  const Phys &ph = a.ph;
  double thetaLocal = 0;
  for (int it = tid; it < NF * TE; it += NT) {
    const int f = it / TE, e = it - f * TE, eg = e0 + e;
    if (eg >= a.nEle) continue;
    int dir, side, s0, st;
    fpt_line<C>(f, dir, side, s0, st);
    const int code = a.nbr[(size_t)f * L + eg];
    const size_t me = (size_t)f * L + eg;
    double ucb[NV], uf[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) {
      const double own = b.dcb[(size_t)v * NF * L + me];
      ucb[v] = own + (code >= 0 ? b.dcb[(size_t)v * NF * L + (size_t)(code >> 1)] : 0.0);
      uf[v] = b.ufb[(size_t)v * NF * L + me] - own;  // Dc = Uc - U_f
    }
    if (code >= 0) {
      // Uc = (1/2)(U_L + U_R) - pf (U_L - U_R): this side's coefficient
      double nd[DIM];
#pragma unroll
      for (int d = 0; d < DIM; d++) nd[d] = a.nrm[((size_t)d * NF + f) * L + eg];
      const double pf = ldg_pen<DIM, double>(nd, ph.penFact);
      const double c = (code & 1) ? 0.5 + pf : 0.5 - pf;
#pragma unroll
      for (int v = 0; v < NV; v++) uf[v] += c * ucb[v];
    } else {
      // Uc = (1/2)(U_f + ghost(U_f)), the ghost state in dual numbers
      double x[NV + 1], xb[NV + 1] = {}, nd[DIM];
#pragma unroll
      for (int d = 0; d < DIM; d++) nd[d] = a.nrm[((size_t)d * NF + f) * L + eg];
#pragma unroll
      for (int v = 0; v < NV; v++) {
        double t = 0;
#pragma unroll
        for (int jj = 0; jj < N1; jj++) t += op.lag[side][jj] * a.Y[((size_t)v * NS + s0 + jj * st) * L + eg];
        x[v] = t;
      }
      x[NV] = 0.0;
      auto uc = [&](const auto *X, auto *Uc) {
        using TT = typename std::remove_cv<typename std::remove_reference<decltype(X[0])>::type>::type;
        TT own[NV], oth[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) own[v] = X[v];
        if constexpr (BC || NV == 1) adjv_ghost<C, TT>(a, code, own, nd, X[NV], oth);
        else {
#pragma unroll
          for (int v = 0; v < NV; v++) oth[v] = TT(0.0);
        }
#pragma unroll
        for (int v = 0; v < NV; v++) Uc[v] = TT(0.5) * (own[v] + oth[v]);
      };
      vjp_chunked<NV + 1, NV, 3>(x, ucb, xb, uc);
#pragma unroll
      for (int v = 0; v < NV; v++) uf[v] += xb[v];
      thetaLocal += xb[NV];
    }
#pragma unroll
    for (int v = 0; v < NV; v++) sUf[(v * NF + f) * TE + e] = uf[v];
  }
  if (a.thetaBar) {
    for (int o = 16; o > 0; o >>= 1) thetaLocal += __shfl_xor_sync(0xffffffffu, thetaLocal, o);
    if ((tid & 31) == 0) red[tid >> 5] = thetaLocal;
  }
  __syncthreads();
  if (a.thetaBar && tid == 0) {
    double t = 0;
    for (int w = 0; w < NT / 32; w++) t += red[w];
    if (t != 0) atomicAdd(a.thetaBar, t);
  }
  for (int it = tid; it < NS * TE; it += NT) {
    const int s = it / TE, e = it - s * TE, eg = e0 + e;
    if (eg >= a.nEle) continue;
    const int i = s % N1, j = (s / N1) % N1, k = DIM == 3 ? s / (N1 * N1) : 0;
    int cf[2 * DIM], cs[2 * DIM], ca[2 * DIM];
    corr_fpts<C>(i, j, k, cf, cs, ca);
    const double idet = 1.0 / a.detJ[(size_t)s * L + eg];
#pragma unroll
    for (int w = 0; w < NV; w++) {
      const size_t gi = ((size_t)w * NS + s) * L + eg;
      double yb = b.ub[gi];
#pragma unroll
      for (int c = 0; c < 2 * DIM; c++) yb += op.lag[cs[c]][ca[c]] * sUf[(w * NF + cf[c]) * TE + e];
      if (a.mode & ADJ_PLAIN) a.ybar[gi] = yb;
      if (a.mode & ADJ_RK) {
        const double base = (a.mode & ADJ_RK_FIRST) ? a.lam[gi] : a.lamNew[gi];
        const double ln = base + yb;
        a.lamNew[gi] = ln;
        const double Dt = (a.grp ? a.dtGrp[a.grp[eg]] : a.dt) * idet;
        if (a.mode & ADJ_RK_LAST) a.seedOut[gi] = -a.cLam * ln * Dt;
        else a.seedOut[gi] = -(a.cLam * a.lam[gi] + a.cY * yb) * Dt;
      }
    }
  }
}

}  // namespace frg
