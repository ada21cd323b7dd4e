// kernels.cuh -- the FR residual + RK stage kernels for sm_100a.
//
// Data layout in HBM: every per-point array is [field][point][element] with
// the element index fastest, so a warp's 32 lanes (32 consecutive elements at
// one point) issue one coalesced 128/256-byte access.
//
// One thread block owns a tile of TE elements and keeps, in shared memory,
// the tile's solution at the solution points, its contravariant fluxes and
// its flux-point jumps.  One launch does a whole RK stage for the tile:
//
//   A  load stage state, pointwise inviscid flux + metric transform
//        (solver::calcInviscidFlux_spts, src/solver.cpp:514-539)
//   B  per flux point: own trace (extrapolateU, :401-412), neighbour trace
//        (gathered from the previous launch's trace buffer), common flux
//        (face::calcInviscidFlux, src/face.cpp:132-175), the extrapolated
//        normal flux (extrapolateNormalFlux, :729-787) and the jump
//        Fn*dA - disFn (correctDivFlux, :789-806)
//   C  divergence + correction (calcDivF_spts :707-727, correctDivFlux), then
//        the RK stage update (timeStepA/B, :307-385) in FP64
//   D  traces of the new state for the next launch
//
// The spts->fpts, gradient and correction operators are Kronecker products
// of 1D tables, so they are applied by sum factorisation along one
// coordinate line: (P+1) terms per output instead of nSpts or nFpts, summed
// in the order of the reference's dense GEMM rows.  Each face's common flux
// is evaluated by both elements that share it, in the reference's left/right
// order with the left element's normal, so both get the reference's values;
// this removes the separate face pass and its flux round trip through HBM.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "physics.cuh"

namespace frg {

constexpr int KMAXP = 5;

// 1D operator tables (see setup.h Ops1D), per VCJH scheme and order.
template <typename R>
struct OpTab {
  R lag[2][KMAXP + 1];
  R dlag[KMAXP + 1][KMAXP + 1];
  R gL[KMAXP + 1], gR[KMAXP + 1];
  R w[KMAXP + 1];
};
// Each CUDA translation unit that includes this header holds its own copy of
// the tables (internal linkage) and uploads it through its own entry point.
static __constant__ OpTab<double> c_opd[4][KMAXP + 1];
static __constant__ OpTab<float> c_opf[4][KMAXP + 1];

template <typename R>
__device__ __forceinline__ const OpTab<R> &optab(int vcjh, int P);
template <>
__device__ __forceinline__ const OpTab<double> &optab<double>(int vcjh, int P) { return c_opd[vcjh][P]; }
template <>
__device__ __forceinline__ const OpTab<float> &optab<float>(int vcjh, int P) { return c_opf[vcjh][P]; }

// Error flag bits written by kernels; the host reads the word after a step.
enum : unsigned { ERRF_NAN = 1u, ERRF_DT = 2u, ERRF_BC = 4u };

// Compile-time sizes of one (dimension, order, fields) configuration.
template <int DIM_, int P_, int NV_>
struct Cfg {
  static constexpr int DIM = DIM_, P = P_, NV = NV_, N1 = P_ + 1;
  static constexpr int NS = DIM == 2 ? N1 * N1 : N1 * N1 * N1;
  static constexpr int NFF = DIM == 2 ? N1 : N1 * N1;
  static constexpr int NF = 2 * DIM * NFF;
  static constexpr int NT = 256;  // threads per block
};

// Elements per block: as many as fit ~100 KB of shared memory (two blocks per
// SM), capped at 32 so a warp spans 32 elements of one point.
template <class C, typename R>
struct Tile {
  static constexpr int PER_ELE = (C::NV * C::NS + C::DIM * C::NV * C::NS + C::NV * C::NF) * (int)sizeof(R);
  static constexpr int TE = (32 * PER_ELE <= 100 * 1024) ? 32 : (16 * PER_ELE <= 100 * 1024) ? 16
                            : (8 * PER_ELE <= 110 * 1024) ? 8 : 4;
  static constexpr int SMEM = TE * PER_ELE;
};

// Geometry of flux point f: normal direction, side (0: -1 face, 1: +1 face),
// first solution point of the coordinate line through it and that line's stride.
template <class C>
__device__ __forceinline__ void fpt_line(int f, int &dir, int &side, int &s0, int &stride) {
  constexpr int P = C::P, N1 = C::N1;
  if constexpr (C::DIM == 2) {
    int face = f / N1, k = f - face * N1;
    switch (face) {
      case 0: dir = 1; side = 0; s0 = k; stride = N1; break;
      case 1: dir = 0; side = 1; s0 = k * N1; stride = 1; break;
      case 2: dir = 1; side = 1; s0 = P - k; stride = N1; break;
      default: dir = 0; side = 0; s0 = (P - k) * N1; stride = 1; break;
    }
  } else {
    constexpr int P12 = N1 * N1;
    int face = f / P12, k = f - face * P12, a = k % N1, b = k / N1;
    switch (face) {
      case 0: dir = 2; side = 0; s0 = a + N1 * b; stride = P12; break;
      case 1: dir = 2; side = 1; s0 = (P - a) + N1 * b; stride = P12; break;
      case 2: dir = 0; side = 0; s0 = N1 * a + P12 * b; stride = 1; break;
      case 3: dir = 0; side = 1; s0 = N1 * (P - a) + P12 * b; stride = 1; break;
      case 4: dir = 1; side = 0; s0 = (P - a) + P12 * b; stride = N1; break;
      default: dir = 1; side = 1; s0 = a + P12 * b; stride = N1; break;
    }
  }
}

// Flux points whose correction reaches solution point (i,j[,k]), in face
// order, with the sign of the correction-function derivative they carry
// (divVCJH_quad / divVCJH_hex, src/operators.cpp:1544-1619).
template <class C>
__device__ __forceinline__ void corr_fpts(int i, int j, int k, int fp[2 * C::DIM], int side[2 * C::DIM],
                                          int at[2 * C::DIM]) {
  constexpr int P = C::P, N1 = C::N1;
  if constexpr (C::DIM == 2) {
    fp[0] = i;                  side[0] = 0; at[0] = j;
    fp[1] = N1 + j;             side[1] = 1; at[1] = i;
    fp[2] = 2 * N1 + (P - i);   side[2] = 1; at[2] = j;
    fp[3] = 3 * N1 + (P - j);   side[3] = 0; at[3] = i;
  } else {
    constexpr int P12 = N1 * N1;
    fp[0] = i + N1 * j;                 side[0] = 0; at[0] = k;
    fp[1] = P12 + (P - i) + N1 * j;     side[1] = 1; at[1] = k;
    fp[2] = 2 * P12 + j + N1 * k;       side[2] = 0; at[2] = i;
    fp[3] = 3 * P12 + (P - j) + N1 * k; side[3] = 1; at[3] = i;
    fp[4] = 4 * P12 + (P - i) + N1 * k; side[4] = 0; at[4] = j;
    fp[5] = 5 * P12 + i + N1 * k;       side[5] = 1; at[5] = j;
  }
}

// Stage modes
enum : int {
  SF_WAVESP = 1,    // store Rusanov / LF wave speeds of left-side flux points
  SF_FIRST = 2,     // first RK stage: accumulator = U0 - b t
  SF_LAST = 4,      // last RK stage: U = accumulator - b t
  SF_RESIDUAL = 8,  // solver::calcResidual only: write divF, no update
  SF_JAMESON = 16,  // timeType 5: every stage U = U0 - a t
  SF_TIME = 32,     // advance the device time by dt (block 0)
  SF_DIVF = 64      // also store divF (residual monitoring) during an update
};

// Arguments of one stage launch.  Arrays of the stored type S (double, or
// float in the mixed mode) are passed untyped and cast in the kernel.
struct StageArgs {
  int nE;
  const double *Uin_d;  // stage input when stored in double (else null)
  const void *Uin_s;    // stage input in the stored type
  const double *U0;     // state at the start of the step
  double *Acc;          // running final combination U0 - sum_s b_s t_s
  double *Uout;         // final state (last stage); may alias U0
  void *Wout;           // next stage state (S)
  const void *trIn;     // traces of the input state (S), [NV][NF][nE]
  void *trOut;          // traces of the output state (S)
  double *divF;         // residual, [NV][NS][nE] (SF_RESIDUAL / SF_DIVF)
  const int *nbr;       // [NF][nE]
  const void *nrm;      // (S) [DIM][NF][nE] normal of the face's left element
  const void *dA;       // (S) [NF][nE]
  const void *JG;       // (S) [DIM][DIM][NS][nE]
  const void *detJ;     // (S) [NS][nE]
  double *waveSp;       // [NF][nE]
  const double *dt;     // scalar, or [nE] when dtLocal
  double *time;         // device time (SF_TIME)
  unsigned *err;
  double aNext, bCur;
  int dtLocal, flags, vcjh;
  Phys ph;
};

// ----------------------------------------------------------------------------
// The fused stage kernel (inviscid Euler or scalar advection).
// R: arithmetic type; S: stored type of stage states, traces and metrics.
// BC: the mesh has boundary faces (else the ghost-state code is not built);
// RS: interior Riemann solver, 0 Rusanov, 1 Roe (boundaries always Rusanov,
// src/face.cpp:142-145).  Two resident blocks per SM cap registers at 128.
// ----------------------------------------------------------------------------
template <class C, typename R, typename S, bool BC, int RS>
__global__ void __launch_bounds__(C::NT, 2) fr_stage_kernel(const StageArgs a) {
  using T = Tile<C, R>;
  constexpr int TE = T::TE, NS = C::NS, NF = C::NF, NV = C::NV, DIM = C::DIM, N1 = C::N1, NT = C::NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R *Us = reinterpret_cast<R *>(smem_raw);  // [NV][NS][TE]
  R *Fs = Us + NV * NS * TE;                // [DIM][NV][NS][TE]
  R *Js = Fs + DIM * NV * NS * TE;          // [NV][NF][TE]
  const OpTab<R> &op = optab<R>(a.vcjh, C::P);
  const int nE = a.nE, tid = threadIdx.x, e0 = blockIdx.x * TE;
  const Phys &ph = a.ph;
  const S *Uin_s = static_cast<const S *>(a.Uin_s);
  const S *trIn = static_cast<const S *>(a.trIn);
  const S *nrmG = static_cast<const S *>(a.nrm);
  const S *dAG = static_cast<const S *>(a.dA);
  const S *JGG = static_cast<const S *>(a.JG);
  const S *detJG = static_cast<const S *>(a.detJ);
  S *Wout = static_cast<S *>(a.Wout);
  S *trOut = static_cast<S *>(a.trOut);

  // ---- A: stage state and contravariant inviscid flux at solution points
  for (int it = tid; it < NS * TE; it += NT) {
    const int s = it / TE, e = it - s * TE, eg = e0 + e;
    if (eg >= nE) continue;
    R u[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) {
      size_t gi = ((size_t)v * NS + s) * nE + eg;
      u[v] = a.Uin_d ? (R)a.Uin_d[gi] : (R)Uin_s[gi];
      Us[(v * NS + s) * TE + e] = u[v];
    }
    R F[DIM][NV];
    inviscid_flux<DIM, NV, R>(u, F, ph);
    R G[DIM][DIM];
#pragma unroll
    for (int d1 = 0; d1 < DIM; d1++)
#pragma unroll
      for (int d2 = 0; d2 < DIM; d2++) G[d1][d2] = (R)JGG[(((size_t)d1 * DIM + d2) * NS + s) * nE + eg];
#pragma unroll
    for (int d1 = 0; d1 < DIM; d1++)
#pragma unroll
      for (int v = 0; v < NV; v++) {
        R t = 0;
#pragma unroll
        for (int d2 = 0; d2 < DIM; d2++) t += G[d1][d2] * F[d2][v];
        Fs[((d1 * NV + v) * NS + s) * TE + e] = t;
      }
  }
  __syncthreads();

  // ---- B: common flux and jump at flux points
  for (int it = tid; it < NF * TE; it += NT) {
    const int f = it / TE, e = it - f * TE, eg = e0 + e;
    if (eg >= nE) continue;
    int dir, side, s0, st;
    fpt_line<C>(f, dir, side, s0, st);
    R own[NV], dis[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) {
      R t = 0, q = 0;
#pragma unroll
      for (int j = 0; j < N1; j++) {
        const R l = op.lag[side][j];
        t += l * Us[(v * NS + s0 + j * st) * TE + e];
        q += l * Fs[((dir * NV + v) * NS + s0 + j * st) * TE + e];
      }
      own[v] = t;
      dis[v] = side ? q : -q;
    }
    R n[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) n[d] = (R)nrmG[((size_t)d * NF + f) * nE + eg];
    const R dA = (R)dAG[(size_t)f * nE + eg];
    const int code = a.nbr[(size_t)f * nE + eg];
    R oth[NV];
    bool right = false;
    int bc = 0;
    if (code >= 0) {
      right = code & 1;
      const size_t t = (size_t)(code >> 1);
#pragma unroll
      for (int v = 0; v < NV; v++) oth[v] = (R)trIn[(size_t)v * NF * nE + t];
    } else {
      bc = -1 - code;
      if constexpr (NV == 1 || !BC) {
        // advection boundaries keep a zero ghost state (src/boundFace.cpp:274)
#pragma unroll
        for (int v = 0; v < NV; v++) oth[v] = 0;
        if constexpr (!BC) atomicOr(a.err, ERRF_BC);
      } else {
        double ul[NV], ur[NV], nd[DIM];
#pragma unroll
        for (int v = 0; v < NV; v++) ul[v] = own[v];
#pragma unroll
        for (int d = 0; d < DIM; d++) nd[d] = n[d];
        if (!bc_ghost<DIM>(bc, ul, nd, ur, ph)) atomicOr(a.err, ERRF_BC);
#pragma unroll
        for (int v = 0; v < NV; v++) oth[v] = (R)ur[v];
      }
    }
    const R *UL = right ? oth : own;
    const R *UR = right ? own : oth;
    R Fn[NV];
    R ws = -1;
    if constexpr (NV == 1) {
      ws = lax_friedrichs<DIM, R>(UL[0], UR[0], n, Fn, ph);
    } else if constexpr (RS == 0 || DIM == 3) {
      ws = rusanov<DIM, NV, R, double>(UL, UR, n, Fn, ph);
    } else if constexpr (BC) {
      if (code < 0) ws = rusanov<DIM, NV, R, double>(UL, UR, n, Fn, ph);
      else roe2d<R, double>(UL, UR, n, Fn, ph);
    } else {
      roe2d<R, double>(UL, UR, n, Fn, ph);
    }
    if ((a.flags & SF_WAVESP) && !right && ws >= 0) a.waveSp[(size_t)f * nE + eg] = (double)ws;
#pragma unroll
    for (int v = 0; v < NV; v++) {
      const R fo = right ? -Fn[v] * dA : Fn[v] * dA;
      Js[(v * NF + f) * TE + e] = fo - dis[v];
    }
  }
  __syncthreads();

  // ---- C: divergence + correction, RK update
  const bool resid = a.flags & SF_RESIDUAL;
  for (int it = tid; it < NS * TE; it += NT) {
    const int s = it / TE, e = it - s * TE, eg = e0 + e;
    if (eg >= nE) continue;
    const int i = s % N1, j = (s / N1) % N1, k = DIM == 3 ? s / (N1 * N1) : 0;
    const int ijk[3] = {i, j, k};
    int cf[2 * DIM], cs[2 * DIM], ca[2 * DIM];
    corr_fpts<C>(i, j, k, cf, cs, ca);
    double det = 0, dtl = 0;
    if (!resid) {
      det = (double)detJG[(size_t)s * nE + eg];
      dtl = a.dtLocal ? a.dt[eg] : a.dt[0];
    }
#pragma unroll
    for (int v = 0; v < NV; v++) {
      R acc = 0;
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        const int sd = d == 0 ? 1 : d == 1 ? N1 : N1 * N1;
        const int sb = s - ijk[d] * sd;
#pragma unroll
        for (int q = 0; q < N1; q++) acc += op.dlag[ijk[d]][q] * Fs[((d * NV + v) * NS + sb + q * sd) * TE + e];
      }
#pragma unroll
      for (int c = 0; c < 2 * DIM; c++) {
        const R g = cs[c] ? op.gR[ca[c]] : -op.gL[ca[c]];
        acc += g * Js[(v * NF + cf[c]) * TE + e];
      }
      const size_t gi = ((size_t)v * NS + s) * nE + eg;
      const double div = (double)acc;
      if (a.flags & (SF_RESIDUAL | SF_DIVF)) a.divF[gi] = div;
      if (resid) continue;
      const bool last = a.flags & SF_LAST;
      double unew;
      if (a.flags & SF_JAMESON) {
        unew = a.U0[gi] - a.aNext * div / det * dtl;
        if (last) a.Uout[gi] = unew;
        else Wout[gi] = (S)unew;
      } else {
        const double t = a.bCur * div / det * dtl;
        const double base = (a.flags & SF_FIRST) ? a.U0[gi] : a.Acc[gi];
        if (last) {
          unew = base - t;
          a.Uout[gi] = unew;
        } else {
          a.Acc[gi] = base - t;
          const double u0 = (a.flags & SF_FIRST) ? base : a.U0[gi];
          unew = u0 - a.aNext * div / det * dtl;
          Wout[gi] = (S)unew;
        }
      }
      if (last && (v == 0 || v == NV - 1) && isnan(unew)) atomicOr(a.err, ERRF_NAN);
      Us[(v * NS + s) * TE + e] = (R)((a.flags & SF_LAST) ? unew : (double)(S)unew);
    }
  }
  if (resid) return;
  if ((a.flags & SF_TIME) && blockIdx.x == 0 && tid == 0) *a.time += a.dt[0];
  __syncthreads();

  // ---- D: traces of the new state
  for (int it = tid; it < NF * TE; it += NT) {
    const int f = it / TE, e = it - f * TE, eg = e0 + e;
    if (eg >= nE) continue;
    int dir, side, s0, st;
    fpt_line<C>(f, dir, side, s0, st);
#pragma unroll
    for (int v = 0; v < NV; v++) {
      R t = 0;
#pragma unroll
      for (int j = 0; j < N1; j++) t += op.lag[side][j] * Us[(v * NS + s0 + j * st) * TE + e];
      trOut[((size_t)v * NF + f) * nE + eg] = (S)t;
    }
  }
}

// ----------------------------------------------------------------------------
// Traces of a double state (solver::extrapolateU), one thread per
// (flux point, element).
// ----------------------------------------------------------------------------
template <class C, typename R, typename S>
__global__ void fr_trace_kernel(const double *__restrict__ U, S *__restrict__ tr, int nE, int vcjh) {
  constexpr int NS = C::NS, NF = C::NF, NV = C::NV, N1 = C::N1;
  const OpTab<R> &op = optab<R>(vcjh, C::P);
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)NF * nE) return;
  const int f = (int)(idx / nE), eg = (int)(idx - (long)f * nE);
  int dir, side, s0, st;
  fpt_line<C>(f, dir, side, s0, st);
#pragma unroll
  for (int v = 0; v < NV; v++) {
    R t = 0;
#pragma unroll
    for (int j = 0; j < N1; j++) t += op.lag[side][j] * (R)U[((size_t)v * NS + s0 + j * st) * nE + eg];
    tr[((size_t)v * NF + f) * nE + eg] = (S)t;
  }
}

// ele::calcWaveSpFpts (src/ele.cpp:1031-1084) for every flux point.
template <int DIM, int NV, typename S>
__global__ void fr_wavesp_kernel(const S *__restrict__ tr, const double *__restrict__ nrmOwn, double *waveSp,
                                 int NF, int nE, Phys ph) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)NF * nE) return;
  const int f = (int)(idx / nE), e = (int)(idx - (long)f * nE);
  double n[DIM];
  for (int d = 0; d < DIM; d++) n[d] = nrmOwn[((size_t)d * NF + f) * nE + e];
  double ws;
  if constexpr (NV == 1) {
    double vN = ph.adv[0] * n[0] + ph.adv[1] * n[1];
    if constexpr (DIM == 3) vN += ph.adv[2] * n[2];
    double vTot = fabs(vN - 0.0);
    vN = fabs(vN);
    ws = fmax(vTot, fmax(vN, 0.0));
  } else {
    double U[NV];
    for (int v = 0; v < NV; v++) U[v] = (double)tr[((size_t)v * NF + f) * nE + e];
    double rho = U[0], u = U[1] / rho, v = U[2] / rho, w = 0;
    if constexpr (DIM == 3) w = U[3] / rho;
    double rhoVSq = rho * (u * u + v * v + w * w);
    double p = (ph.gamma - 1) * (U[DIM + 1] - 0.5 * rhoVSq);
    double vN = u * n[0] + v * n[1];
    if constexpr (DIM == 3) vN += w * n[2];
    double csq = fmax(ph.gamma * p / rho, 0.0);
    ws = (fabs(vN - 0.0) + sqrt(csq));
  }
  waveSp[(size_t)f * nE + e] = ws;
}

}  // namespace frg
