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
  // Shared-memory slot of solution point s in the per-point tile arrays.  In
  // 3D one empty slot follows every PADG points -- by default every
  // coordinate line along xi, so the points that start the lines of a face
  // (4 apart at P = 3) fall on different shared-memory banks instead of one
  // (2D: no padding).
  static constexpr int PADG = N1;
  static constexpr int NSP = DIM == 3 ? NS + NS / PADG : NS;
};
template <class C>
__device__ __forceinline__ constexpr int sx(int s) {
  if constexpr (C::DIM == 3) return s + s / C::PADG;
  else return s;
}
// The 3D tiles of 4 FP32 (2 FP64) elements of the TMA viscous kernels: a
// warp spans 8 consecutive points, which one empty slot per 8 points keeps
// on distinct banks in the point-wise and coordinate-line passes (one per xi
// line would put points 0 and 7 on one bank); orders whose point count 8
// does not divide keep the per-line padding.
template <class C>
struct CfgV : C {
  static constexpr int PADG = C::NS % 8 == 0 ? 8 : C::N1;
  static constexpr int NSP = C::NS + C::NS / PADG;
};

// Elements per block: as many as fit ~100 KB of shared memory (two blocks per
// SM), capped at 32 so a warp spans 32 elements of one point.
template <class C, typename R>
struct Tile {
  static constexpr int PER_ELE = (C::NV * C::NSP + C::DIM * C::NV * C::NSP + C::NV * C::NF) * (int)sizeof(R);
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
  SF_DIVF = 64,     // also store divF (residual monitoring) during an update
  SF_DTNEXT = 128,  // last stage: compute the next step's CFL dt (TMA kernel)
  SF_PDL = 256      // launch as a programmatic dependent of the previous kernel (host side)
};

// Arguments of one stage launch.  Arrays of the stored type S (double, or
// float in the mixed mode) are passed untyped and cast in the kernel.
struct StageArgs {
  int nE;    // element stride of the mesh arrays (geometry, traces), a multiple of 32
  int nEle;  // number of real elements
  int ldU;   // element stride of the state arrays (U, U0, Acc, W, divF)
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
  const double *dt;     // scalar, [nE] when dtLocal, or one per group when grp is set
  const int *grp;       // ensemble mode: group (independent case) of each element, else null
  double *time;         // device time (SF_TIME)
  unsigned *err;
  double aNext, bCur;
  int dtLocal, flags, vcjh;
  // viscous path: this side's projected viscous flux per flux point (S),
  // [NV][NF][nE]; the second array only for the 3D LDG penalty term
  void *fvnOut, *fvn2Out;
  const void *fvnIn, *fvn2In;
  int visc2;
  // viscous path, optional: the corrected physical gradient at the solution
  // points (S), [DIM][NV][NS][nE], written by the gradient kernel and read by
  // the stage kernel instead of recomputing it (null: recompute)
  void *dUg;
  // SF_DTNEXT: the next step's dt (ele::calcDt + the global minimum)
  const double *vol, *dAd, *wsurf;
  double *blockMin, *dtNext, *eleDt;
  // first stage of a step with the fused dt (TMA kernels): the next step's dt
  // slot, set here to a huge value before the last stage minimises into it
  double *dtReset;
  unsigned *ticket;
  double cflFac;
  int nff;
  Phys ph;
  // the run's 1D operator tables (order, VCJH scheme), in the launch
  // parameters so the kernels' unrolled loops read them as constant-bank
  // operands rather than by indexed loads
  OpTab<float> opf;
  OpTab<double> opd;
};

template <typename R>
__device__ __forceinline__ const OpTab<R> &stage_op(const StageArgs &a);
template <>
__device__ __forceinline__ const OpTab<double> &stage_op<double>(const StageArgs &a) { return a.opd; }
template <>
__device__ __forceinline__ const OpTab<float> &stage_op<float>(const StageArgs &a) { return a.opf; }
// Host: fill a launch's tables from the 1D operators (setup.h Ops1D), cast
// as the constant-memory copies are.
template <class Ops>
inline void set_stage_ops(StageArgs &a, const Ops &o) {
  for (int i = 0; i <= KMAXP; i++) {
    for (int h = 0; h < 2; h++) {
      a.opd.lag[h][i] = o.lag[h][i];
      a.opf.lag[h][i] = (float)o.lag[h][i];
    }
    a.opd.gL[i] = o.gL[i];
    a.opd.gR[i] = o.gR[i];
    a.opd.w[i] = o.w[i];
    a.opf.gL[i] = (float)o.gL[i];
    a.opf.gR[i] = (float)o.gR[i];
    a.opf.w[i] = (float)o.w[i];
    for (int j = 0; j <= KMAXP; j++) {
      a.opd.dlag[i][j] = o.dlag[i][j];
      a.opf.dlag[i][j] = (float)o.dlag[i][j];
    }
  }
}

// ----------------------------------------------------------------------------
// The fused stage kernels and the block-level phases they share.
// R: arithmetic type; S: stored type of stage states, traces and metrics.
// BC: the mesh has boundary faces (else the ghost-state code is not built);
// RS: interior Riemann solver, 0 Rusanov, 1 Roe (boundaries always Rusanov,
// src/face.cpp:142-145).
// ----------------------------------------------------------------------------

// The state on the other side of flux point f: the neighbour's trace from the
// previous launch's trace buffer, or the boundary ghost state.
template <class C, typename R, typename S, bool BC>
__device__ __forceinline__ void other_side(const StageArgs &a, int code, const R *own, const R *n, R *oth,
                                           bool &right) {
  constexpr int NV = C::NV, NF = C::NF, DIM = C::DIM;
  right = false;
  if (code >= 0) {
    right = code & 1;
    const size_t t = (size_t)(code >> 1);
    const S *trIn = static_cast<const S *>(a.trIn);
#pragma unroll
    for (int v = 0; v < NV; v++) oth[v] = (R)trIn[(size_t)v * NF * a.nE + t];
    return;
  }
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
    if (!bc_ghost<DIM>(-1 - code, ul, nd, ur, a.ph)) atomicOr(a.err, ERRF_BC);
#pragma unroll
    for (int v = 0; v < NV; v++) oth[v] = (R)ur[v];
  }
}

// Common inviscid flux of face::calcInviscidFlux (src/face.cpp:132-175).
// Returns the wave speed the reference stores (negative for Roe).
template <class C, typename R, bool BC, int RS>
__device__ __forceinline__ R inviscid_common(const R *UL, const R *UR, const R *n, int code, R *Fn,
                                             const Phys &ph) {
  constexpr int NV = C::NV, DIM = C::DIM;
  if constexpr (NV == 1) {
    return lax_friedrichs<DIM, R>(UL[0], UR[0], n, Fn, ph);
  } else if constexpr (RS == 0 || DIM == 3) {
    return rusanov<DIM, NV, R, double>(UL, UR, n, Fn, ph);
  } else if constexpr (BC) {
    if (code < 0) return rusanov<DIM, NV, R, double>(UL, UR, n, Fn, ph);
    roe2d<R, double>(UL, UR, n, Fn, ph);
    return -1;
  } else {
    roe2d<R, double>(UL, UR, n, Fn, ph);
    return -1;
  }
}

// Phase A0: the tile's stage state into shared memory.
template <class C, typename R, typename S, int TE>
__device__ __forceinline__ void load_state(const StageArgs &a, R *Us, int e0) {
  constexpr int NS = C::NS, NSP = C::NSP, NV = C::NV, NT = C::NT;
  const S *Uin_s = static_cast<const S *>(a.Uin_s);
  for (int it = threadIdx.x; it < NS * TE; it += NT) {
    const int s = it / TE, e = it - s * TE, eg = e0 + e;
    if (eg >= a.nEle) continue;
#pragma unroll
    for (int v = 0; v < NV; v++) {
      const size_t gi = ((size_t)v * NS + s) * a.ldU + eg;
      Us[(v * NSP + sx<C>(s)) * TE + e] = a.Uin_d ? (R)a.Uin_d[gi] : (R)Uin_s[gi];
    }
  }
}

// Phase C: divergence + correction (calcDivF_spts, correctDivFlux), then the
// RK stage update in FP64 (timeStepA/B); the new state goes to Us.
template <class C, typename R, typename S, int TE>
__device__ __forceinline__ void update_phase(const StageArgs &a, const OpTab<R> &op, const R *Fs, const R *Js, R *Us,
                                             int e0) {
  constexpr int NS = C::NS, NSP = C::NSP, NF = C::NF, NV = C::NV, DIM = C::DIM, N1 = C::N1, NT = C::NT;
  const S *detJG = static_cast<const S *>(a.detJ);
  S *Wout = static_cast<S *>(a.Wout);
  const int nE = a.nE;
  const bool resid = a.flags & SF_RESIDUAL;
  const double dtG = (resid || a.dtLocal || a.grp) ? 0.0 : __ldg(a.dt);
  for (int it = threadIdx.x; it < NS * TE; it += NT) {
    const int s = it / TE, e = it - s * TE, eg = e0 + e;
    if (eg >= a.nEle) continue;
    const int i = s % N1, j = (s / N1) % N1, k = DIM == 3 ? s / (N1 * N1) : 0;
    const int ijk[3] = {i, j, k};
    int cf[2 * DIM], cs[2 * DIM], ca[2 * DIM];
    corr_fpts<C>(i, j, k, cf, cs, ca);
    double det = 0, dtl = 0;
    if (!resid) {
      det = (double)detJG[(size_t)s * nE + eg];
      dtl = a.grp ? a.dt[a.grp[eg]] : a.dtLocal ? a.dt[eg] : dtG;
    }
#pragma unroll
    for (int v = 0; v < NV; v++) {
      R acc = 0;
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        const int sd = d == 0 ? 1 : d == 1 ? N1 : N1 * N1;
        const int sb = s - ijk[d] * sd;
#pragma unroll
        for (int q = 0; q < N1; q++) acc += op.dlag[ijk[d]][q] * Fs[((d * NV + v) * NSP + sx<C>(sb + q * sd)) * TE + e];
      }
#pragma unroll
      for (int c = 0; c < 2 * DIM; c++) {
        const R g = cs[c] ? op.gR[ca[c]] : -op.gL[ca[c]];
        acc += g * Js[(v * NF + cf[c]) * TE + e];
      }
      const size_t gi = ((size_t)v * NS + s) * a.ldU + eg;
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
      Us[(v * NSP + sx<C>(s)) * TE + e] = (R)(last ? unew : (double)(S)unew);
    }
  }
  if (!resid && !a.grp && (a.flags & SF_TIME) && blockIdx.x == 0 && threadIdx.x == 0) *a.time += a.dt[0];
}

// Phase D: traces of the new state for the next launch.
template <class C, typename R, typename S, int TE>
__device__ __forceinline__ void trace_phase(const StageArgs &a, const OpTab<R> &op, const R *Us, int e0) {
  constexpr int NS = C::NS, NSP = C::NSP, NF = C::NF, NV = C::NV, N1 = C::N1, NT = C::NT;
  S *trOut = static_cast<S *>(a.trOut);
  for (int it = threadIdx.x; it < NF * TE; it += NT) {
    const int f = it / TE, e = it - f * TE, eg = e0 + e;
    if (eg >= a.nEle) continue;
    int dir, side, s0, st;
    fpt_line<C>(f, dir, side, s0, st);
#pragma unroll
    for (int v = 0; v < NV; v++) {
      R t = 0;
#pragma unroll
      for (int j = 0; j < N1; j++) t += op.lag[side][j] * Us[(v * NSP + sx<C>(s0 + j * st)) * TE + e];
      trOut[((size_t)v * NF + f) * a.nE + eg] = (S)t;
    }
  }
}

// Own trace of every field at flux point f: sum over the coordinate line.
template <class C, typename R, int TE>
__device__ __forceinline__ void own_trace(const OpTab<R> &op, const R *Us, int f, int e, R *out) {
  int dir, side, s0, st;
  fpt_line<C>(f, dir, side, s0, st);
#pragma unroll
  for (int v = 0; v < C::NV; v++) {
    R t = 0;
#pragma unroll
    for (int j = 0; j < C::N1; j++) t += op.lag[side][j] * Us[(v * C::NSP + sx<C>(s0 + j * st)) * TE + e];
    out[v] = t;
  }
}

// ----------------------------------------------------------------------------
// Inviscid stage kernel (Euler or scalar advection).  Two resident blocks
// per SM cap registers at 128.
// ----------------------------------------------------------------------------
template <class C, typename R, typename S, bool BC, int RS>
__global__ void __launch_bounds__(C::NT, 2) fr_stage_kernel(const StageArgs a) {
  using T = Tile<C, R>;
  constexpr int TE = T::TE, NS = C::NS, NSP = C::NSP, NF = C::NF, NV = C::NV, DIM = C::DIM, N1 = C::N1, NT = C::NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R *Us = reinterpret_cast<R *>(smem_raw);  // [NV][NSP][TE]
  R *Fs = Us + NV * NSP * TE;               // [DIM][NV][NSP][TE]
  R *Js = Fs + DIM * NV * NSP * TE;         // [NV][NF][TE]
  const OpTab<R> &op = stage_op<R>(a);
  const int nE = a.nE, tid = threadIdx.x, e0 = blockIdx.x * TE;
  const Phys &ph = a.ph;
  const S *nrmG = static_cast<const S *>(a.nrm);
  const S *dAG = static_cast<const S *>(a.dA);
  const S *JGG = static_cast<const S *>(a.JG);

  // ---- A: stage state and contravariant inviscid flux at solution points
  load_state<C, R, S, TE>(a, Us, e0);
  __syncthreads();
  for (int it = tid; it < NS * TE; it += NT) {
    const int s = it / TE, e = it - s * TE, eg = e0 + e;
    if (eg >= a.nEle) continue;
    R u[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) u[v] = Us[(v * NSP + sx<C>(s)) * TE + e];
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
        Fs[((d1 * NV + v) * NSP + sx<C>(s)) * TE + e] = t;
      }
  }
  __syncthreads();

  // ---- B: common flux and jump at flux points
  for (int it = tid; it < NF * TE; it += NT) {
    const int f = it / TE, e = it - f * TE, eg = e0 + e;
    if (eg >= a.nEle) continue;
    int dir, side, s0, st;
    fpt_line<C>(f, dir, side, s0, st);
    R own[NV], dis[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) {
      R t = 0, q = 0;
#pragma unroll
      for (int j = 0; j < N1; j++) {
        const R l = op.lag[side][j];
        t += l * Us[(v * NSP + sx<C>(s0 + j * st)) * TE + e];
        q += l * Fs[((dir * NV + v) * NSP + sx<C>(s0 + j * st)) * TE + e];
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
    bool right;
    other_side<C, R, S, BC>(a, code, own, n, oth, right);
    const R *UL = right ? oth : own;
    const R *UR = right ? own : oth;
    R Fn[NV];
    const R ws = inviscid_common<C, R, BC, RS>(UL, UR, n, code, Fn, ph);
    if ((a.flags & SF_WAVESP) && !right && ws >= 0) a.waveSp[(size_t)f * nE + eg] = (double)ws;
#pragma unroll
    for (int v = 0; v < NV; v++) {
      const R fo = right ? -Fn[v] * dA : Fn[v] * dA;
      Js[(v * NF + f) * TE + e] = fo - dis[v];
    }
  }
  __syncthreads();

  // ---- C: divergence + correction, RK update
  update_phase<C, R, S, TE>(a, op, Fs, Js, Us, e0);
  if (a.flags & SF_RESIDUAL) return;
  __syncthreads();

  // ---- D: traces of the new state
  trace_phase<C, R, S, TE>(a, op, Us, e0);
}

// ----------------------------------------------------------------------------
// Viscous path (solver::calcResidual with viscous = 1, src/solver.cpp:252-291):
// two launches per RK stage.
//   fr_visc_grad_kernel   LDG common solution, corrected physical gradient,
//                         and, per flux point, the viscous flux of this side
//                         projected on the face normal (what the other side
//                         of the face needs from it);
//   fr_stage_visc_kernel  recomputes the gradient locally (cheaper than a
//                         round trip through HBM), then fluxes, common
//                         inviscid + LDG viscous flux, divergence,
//                         correction, RK update and traces.
// ----------------------------------------------------------------------------

// L2 prefetch of a block's tile of a [rows][ld] array: one prefetch per
// row segment (the TE elements of the tile), spread over the block's threads,
// so the per-thread loads of the phases that follow hit L2.
template <int TE, int NT>
__device__ __forceinline__ void prefetch_tile(const void *base, int rows, int ld, int esz, int e0) {
  const char *p = static_cast<const char *>(base) + (size_t)e0 * esz;
  for (int r = threadIdx.x; r < rows; r += NT)
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p + (size_t)r * ld * esz));
}

// Prefetch of what a viscous kernel of one RK stage reads for its tile:
// state, metrics, face data and, for the stage kernel, the gradient, the
// projected viscous fluxes and the FP64 step-start arrays.
template <class C, typename S, int TE, int NT>
__device__ __forceinline__ void prefetch_visc(const StageArgs &a, int e0, bool stage) {
  constexpr int NS = C::NS, NSP = C::NSP, NF = C::NF, NV = C::NV, DIM = C::DIM;
  const int L = a.nE;
  if (a.Uin_d) prefetch_tile<TE, NT>(a.Uin_d, NV * NS, a.ldU, 8, e0);
  else prefetch_tile<TE, NT>(a.Uin_s, NV * NS, a.ldU, (int)sizeof(S), e0);
  prefetch_tile<TE, NT>(a.JG, DIM * DIM * NS, L, (int)sizeof(S), e0);
  prefetch_tile<TE, NT>(a.nrm, DIM * NF, L, (int)sizeof(S), e0);
  prefetch_tile<TE, NT>(a.nbr, NF, L, 4, e0);
  if (!stage) {
    prefetch_tile<TE, NT>(a.detJ, NS, L, (int)sizeof(S), e0);
    return;
  }
  prefetch_tile<TE, NT>(a.dA, NF, L, (int)sizeof(S), e0);
  if (a.dUg) prefetch_tile<TE, NT>(a.dUg, DIM * NV * NS, L, (int)sizeof(S), e0);
  prefetch_tile<TE, NT>(a.fvnIn, NV * NF, L, (int)sizeof(S), e0);
  if (!(a.flags & SF_RESIDUAL)) {
    prefetch_tile<TE, NT>(a.detJ, NS, L, (int)sizeof(S), e0);
    prefetch_tile<TE, NT>(a.U0, NV * NS, a.ldU, 8, e0);
    if (!(a.flags & (SF_FIRST | SF_JAMESON))) prefetch_tile<TE, NT>(a.Acc, NV * NS, a.ldU, 8, e0);
  }
}

// Elements per block for the viscous kernels (state, jumps, gradient, flux).
template <class C, typename R>
struct TileV {
  static constexpr int PER_ELE = (C::NV * C::NSP + C::NV * C::NF + 2 * C::DIM * C::NV * C::NSP) * (int)sizeof(R);
  static constexpr int TE = (32 * PER_ELE <= 100 * 1024) ? 32 : (16 * PER_ELE <= 100 * 1024) ? 16
                            : (8 * PER_ELE <= 110 * 1024) ? 8 : 4;
  static constexpr int SMEM = TE * PER_ELE;
};

// Normal direction of the c-th face (faces in reference order).
template <class C>
__device__ __forceinline__ int face_dir(int c) {
  if constexpr (C::DIM == 2) return (c & 1) ? 0 : 1;
  else return c < 2 ? 2 : (c < 4 ? 0 : 1);
}

// LDG penalty sign: face::ldgSolution (src/face.cpp:590-598).
template <int DIM, typename R>
__device__ __forceinline__ R ldg_pen(const R *n, double penFact) {
  if constexpr (DIM == 2) return (n[0] + n[1] < (R)0) ? (R)-penFact : (R)penFact;
  else return (n[0] + n[1] + (R)1.4142135623730951 * n[2] < (R)0) ? (R)-penFact : (R)penFact;
}

// B1: common solution minus own trace at every flux point (ldgSolution, and
// dUc = UC - U of face::calcInviscidFlux / intFace::setRightStateSolution).
template <class C, typename R, typename S, bool BC, int TE>
__device__ __forceinline__ void ldg_phase(const StageArgs &a, const OpTab<R> &op, const R *Us, R *Dc, int e0) {
  constexpr int NF = C::NF, NV = C::NV, DIM = C::DIM, NT = C::NT;
  const S *nrmG = static_cast<const S *>(a.nrm);
  for (int it = threadIdx.x; it < NF * TE; it += NT) {
    const int f = it / TE, e = it - f * TE, eg = e0 + e;
    if (eg >= a.nEle) continue;
    R own[NV], oth[NV], n[DIM];
    own_trace<C, R, TE>(op, Us, f, e, own);
#pragma unroll
    for (int d = 0; d < DIM; d++) n[d] = (R)nrmG[((size_t)d * NF + f) * a.nE + eg];
    const int code = a.nbr[(size_t)f * a.nE + eg];
    bool right;
    other_side<C, R, S, BC>(a, code, own, n, oth, right);
    const R *UL = right ? oth : own;
    const R *UR = right ? own : oth;
    const R pf = code < 0 ? (R)0 : ldg_pen<DIM, R>(n, a.ph.penFact);
#pragma unroll
    for (int v = 0; v < NV; v++) {
      const R uc = code < 0 ? (R)0.5 * (UL[v] + UR[v]) : (R)0.5 * (UL[v] + UR[v]) - pf * (UL[v] - UR[v]);
      Dc[(v * NF + f) * TE + e] = uc - own[v];
    }
  }
}

// C1: physical gradient at solution points: D U + correction by the common
// solution (calcGradU_spts, correctGradU src/solver.cpp:808-879), then
// JGinv^T / detJ.  dUs is [DIM][NV][NSP][TE] (point slots sx<C>(s)).
template <class C, typename R, typename S, int TE>
__device__ __forceinline__ void gradient_phase(const StageArgs &a, const OpTab<R> &op, const R *Us, const R *Dc,
                                               R *dUs, int e0) {
  constexpr int NS = C::NS, NSP = C::NSP, NF = C::NF, NV = C::NV, DIM = C::DIM, N1 = C::N1, NT = C::NT;
  const S *JGG = static_cast<const S *>(a.JG);
  const S *detJG = static_cast<const S *>(a.detJ);
  for (int it = threadIdx.x; it < NS * TE; it += NT) {
    const int s = it / TE, e = it - s * TE, eg = e0 + e;
    if (eg >= a.nEle) continue;
    const int i = s % N1, j = (s / N1) % N1, k = DIM == 3 ? s / (N1 * N1) : 0;
    const int ijk[3] = {i, j, k};
    int cf[2 * DIM], cs[2 * DIM], ca[2 * DIM];
    corr_fpts<C>(i, j, k, cf, cs, ca);
    R G[DIM][DIM];
#pragma unroll
    for (int d1 = 0; d1 < DIM; d1++)
#pragma unroll
      for (int d2 = 0; d2 < DIM; d2++) G[d1][d2] = (R)JGG[(((size_t)d1 * DIM + d2) * NS + s) * a.nE + eg];
    const R invDet = (R)1. / (R)detJG[(size_t)s * a.nE + eg];
#pragma unroll
    for (int v = 0; v < NV; v++) {
      R gr[DIM];
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        const int sd = d == 0 ? 1 : d == 1 ? N1 : N1 * N1;
        const int sb = s - ijk[d] * sd;
        R acc = 0;
#pragma unroll
        for (int q = 0; q < N1; q++) acc += op.dlag[ijk[d]][q] * Us[(v * NSP + sx<C>(sb + q * sd)) * TE + e];
#pragma unroll
        for (int c = 0; c < 2 * DIM; c++)
          if (face_dir<C>(c) == d) acc += (cs[c] ? op.gR[ca[c]] : op.gL[ca[c]]) * Dc[(v * NF + cf[c]) * TE + e];
        gr[d] = acc;
      }
#pragma unroll
      for (int d1 = 0; d1 < DIM; d1++) {
        R t = 0;
#pragma unroll
        for (int d2 = 0; d2 < DIM; d2++) t += gr[d2] * G[d2][d1];
        dUs[((d1 * NV + v) * NSP + sx<C>(s)) * TE + e] = invDet * t;
      }
    }
  }
}

// Gradient trace [DIM][NV] at own flux point f (extrapolateGradU, :881-895).
template <class C, typename R, int TE>
__device__ __forceinline__ void own_grad_trace(const OpTab<R> &op, const R *dUs, int f, int e, R *g) {
  int dir, side, s0, st;
  fpt_line<C>(f, dir, side, s0, st);
#pragma unroll
  for (int q = 0; q < C::DIM * C::NV; q++) {
    R t = 0;
#pragma unroll
    for (int j = 0; j < C::N1; j++) t += op.lag[side][j] * dUs[(q * C::NSP + sx<C>(s0 + j * st)) * TE + e];
    g[q] = t;
  }
}

// Viscous flux [DIM][NV] of a state and its physical gradient.
template <class C, typename R>
__device__ __forceinline__ void visc_flux(const R *u, const R *g, R Fv[C::DIM][C::NV], const Phys &ph) {
  if constexpr (C::NV == 1) {
    R t[C::DIM][1];
    viscous_flux_ad<C::DIM, R>(g, t, ph);
#pragma unroll
    for (int d = 0; d < C::DIM; d++) Fv[d][0] = t[d][0];
  } else {
    viscous_flux<C::DIM, R>(u, g, Fv, ph);
  }
}

template <class C, typename R, typename S, bool BC>
__global__ void __launch_bounds__(C::NT, 2) fr_visc_grad_kernel(const StageArgs a) {
  using T = TileV<C, R>;
  constexpr int TE = T::TE, NS = C::NS, NSP = C::NSP, NF = C::NF, NV = C::NV, DIM = C::DIM, NT = C::NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R *Us = reinterpret_cast<R *>(smem_raw);  // [NV][NSP][TE]
  R *Dc = Us + NV * NSP * TE;               // [NV][NF][TE]
  R *dUs = Dc + NV * NF * TE;               // [DIM][NV][NSP][TE]
  const OpTab<R> &op = stage_op<R>(a);
  const int e0 = blockIdx.x * TE;
  const S *nrmG = static_cast<const S *>(a.nrm);
  S *fvnOut = static_cast<S *>(a.fvnOut);
  S *fvn2Out = static_cast<S *>(a.fvn2Out);
  prefetch_visc<C, S, TE, NT>(a, e0, false);
  load_state<C, R, S, TE>(a, Us, e0);
  __syncthreads();
  ldg_phase<C, R, S, BC, TE>(a, op, Us, Dc, e0);
  __syncthreads();
  gradient_phase<C, R, S, TE>(a, op, Us, Dc, dUs, e0);
  __syncthreads();
  if (a.dUg) {  // the gradient for the stage kernel
    S *dUg = static_cast<S *>(a.dUg);
    for (int it = threadIdx.x; it < DIM * NV * NS * TE; it += NT) {
      const int q = it / TE, e = it - q * TE, eg = e0 + e;
      if (eg < a.nEle) dUg[(size_t)q * a.nE + eg] = (S)dUs[((q / NS) * NSP + sx<C>(q % NS)) * TE + e];
    }
  }
  // this side's viscous flux, projected, at every interior flux point
  for (int it = threadIdx.x; it < NF * TE; it += NT) {
    const int f = it / TE, e = it - f * TE, eg = e0 + e;
    if (eg >= a.nEle || a.nbr[(size_t)f * a.nE + eg] < 0) continue;
    R u[NV], g[DIM * NV], n[DIM], Fv[DIM][NV];
    own_trace<C, R, TE>(op, Us, f, e, u);
    own_grad_trace<C, R, TE>(op, dUs, f, e, g);
#pragma unroll
    for (int d = 0; d < DIM; d++) n[d] = (R)nrmG[((size_t)d * NF + f) * a.nE + eg];
    visc_flux<C, R>(u, g, Fv, a.ph);
#pragma unroll
    for (int v = 0; v < NV; v++) {
      R fn = 0;
#pragma unroll
      for (int d = 0; d < DIM; d++) fn += Fv[d][v] * n[d];
      fvnOut[((size_t)v * NF + f) * a.nE + eg] = (S)fn;
      if constexpr (DIM == 3) {
        // the LDG penalty term of the reference reads FL[1] where FL[2] is
        // meant (src/face.cpp:245): the left side contributes n0 F0 + n1 F1 + n2 F1
        if (a.visc2) fvn2Out[((size_t)v * NF + f) * a.nE + eg] = (S)(n[0] * Fv[0][v] + n[1] * Fv[1][v] + n[2] * Fv[1][v]);
      }
    }
  }
}

template <class C, typename R, typename S, bool BC, int RS>
__global__ void __launch_bounds__(C::NT, 2) fr_stage_visc_kernel(const StageArgs a) {
  using T = TileV<C, R>;
  constexpr int TE = T::TE, NS = C::NS, NSP = C::NSP, NF = C::NF, NV = C::NV, DIM = C::DIM, N1 = C::N1, NT = C::NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R *Us = reinterpret_cast<R *>(smem_raw);  // [NV][NSP][TE]
  R *Js = Us + NV * NSP * TE;               // [NV][NF][TE]: dUc, then the jumps
  R *dUs = Js + NV * NF * TE;               // [DIM][NV][NSP][TE]
  R *Fs = dUs + DIM * NV * NSP * TE;        // [DIM][NV][NSP][TE]
  const OpTab<R> &op = stage_op<R>(a);
  const int nE = a.nE, tid = threadIdx.x, e0 = blockIdx.x * TE;
  const Phys &ph = a.ph;
  const S *nrmG = static_cast<const S *>(a.nrm);
  const S *dAG = static_cast<const S *>(a.dA);
  const S *JGG = static_cast<const S *>(a.JG);
  const S *fvnIn = static_cast<const S *>(a.fvnIn);
  const S *fvn2In = static_cast<const S *>(a.fvn2In);

  prefetch_visc<C, S, TE, NT>(a, e0, true);
  load_state<C, R, S, TE>(a, Us, e0);
  if (a.dUg) {
    // the gradient kernel's corrected gradient (the same values this block
    // would compute: same inputs, same arithmetic)
    const S *dUg = static_cast<const S *>(a.dUg);
    for (int it = tid; it < DIM * NV * NS * TE; it += NT) {
      const int q = it / TE, e = it - q * TE, eg = e0 + e;
      if (eg < a.nEle) dUs[((q / NS) * NSP + sx<C>(q % NS)) * TE + e] = (R)dUg[(size_t)q * nE + eg];
    }
    __syncthreads();
  } else {
    __syncthreads();
    ldg_phase<C, R, S, BC, TE>(a, op, Us, Js, e0);
    __syncthreads();
    gradient_phase<C, R, S, TE>(a, op, Us, Js, dUs, e0);
    __syncthreads();
  }

  // ---- A: inviscid + viscous flux at solution points, transformed
  // (calcInviscidFlux_spts keeps the physical flux, calcViscousFlux_spts
  //  src/solver.cpp:562-596 adds the viscous flux and applies JGinv)
  for (int it = tid; it < NS * TE; it += NT) {
    const int s = it / TE, e = it - s * TE, eg = e0 + e;
    if (eg >= a.nEle) continue;
    R u[NV], g[DIM * NV];
#pragma unroll
    for (int v = 0; v < NV; v++) u[v] = Us[(v * NSP + sx<C>(s)) * TE + e];
#pragma unroll
    for (int q = 0; q < DIM * NV; q++) g[q] = dUs[(q * NSP + sx<C>(s)) * TE + e];
    R Fi[DIM][NV], Fv[DIM][NV];
    inviscid_flux<DIM, NV, R>(u, Fi, ph);
    visc_flux<C, R>(u, g, Fv, ph);
#pragma unroll
    for (int d = 0; d < DIM; d++)
#pragma unroll
      for (int v = 0; v < NV; v++) Fv[d][v] += Fi[d][v];
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
        for (int d2 = 0; d2 < DIM; d2++) t += G[d1][d2] * Fv[d2][v];
        Fs[((d1 * NV + v) * NSP + sx<C>(s)) * TE + e] = t;
      }
  }
  __syncthreads();

  // ---- B: common inviscid + LDG viscous flux (face::calcInviscidFlux and
  // face::calcViscousFlux, src/face.cpp:132-287) and the jumps
  for (int it = tid; it < NF * TE; it += NT) {
    const int f = it / TE, e = it - f * TE, eg = e0 + e;
    if (eg >= a.nEle) continue;
    int dir, side, s0, st;
    fpt_line<C>(f, dir, side, s0, st);
    R own[NV], dis[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) {
      R t = 0, q = 0;
#pragma unroll
      for (int j = 0; j < N1; j++) {
        const R l = op.lag[side][j];
        t += l * Us[(v * NSP + sx<C>(s0 + j * st)) * TE + e];
        q += l * Fs[((dir * NV + v) * NSP + sx<C>(s0 + j * st)) * TE + e];
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
    bool right;
    other_side<C, R, S, BC>(a, code, own, n, oth, right);
    const R *UL = right ? oth : own;
    const R *UR = right ? own : oth;
    R Fn[NV];
    const R ws = inviscid_common<C, R, BC, RS>(UL, UR, n, code, Fn, ph);
    if ((a.flags & SF_WAVESP) && !right && ws >= 0) a.waveSp[(size_t)f * nE + eg] = (double)ws;
    R nn = 0;
#pragma unroll
    for (int d = 0; d < DIM; d++) nn += n[d] * n[d];
    const R tau = (R)ph.tau;
    if (code >= 0) {
      // this side's projected viscous flux: the value the gradient kernel
      // stored for this flux point (its own trace, gradient trace and
      // viscousFlux, projected in the same order)
      const size_t t = (size_t)(code >> 1), me = (size_t)f * nE + eg;
      const R pf = ldg_pen<DIM, R>(n, ph.penFact);
#pragma unroll
      for (int v = 0; v < NV; v++) {
        const R on = (R)fvnIn[(size_t)v * NF * nE + me];
        const R xn = (R)fvnIn[(size_t)v * NF * nE + t];
        const R FLn = right ? xn : on, FRn = right ? on : xn;
        if constexpr (NV == 1) {
          Fn[v] += (R)0.5 * (FLn + FRn);  // centralFlux (src/flux.cpp:379-387)
        } else {
          R jumpF = FLn - FRn;
          if constexpr (DIM == 3) {
            // the left side's n0 F0 + n1 F1 + n2 F1 (src/face.cpp:245); it
            // only enters multiplied by the penalty factor, so without one
            // (no second array) any finite value gives the same sum
            const R al = a.visc2 ? (R)fvn2In[(size_t)v * NF * nE + (right ? t : me)] : (right ? xn : on);
            jumpF = al - FRn;
          }
          Fn[v] += (R)0.5 * (FLn + FRn) + pf * nn * jumpF + tau * nn * (UL[v] - UR[v]);
        }
      }
    } else {
      // boundary: this side's viscous flux from its gradient trace
      R g[DIM * NV], Fo[DIM][NV];
      own_grad_trace<C, R, TE>(op, dUs, f, e, g);
      visc_flux<C, R>(own, g, Fo, ph);
      if constexpr (NV == 1) {
#pragma unroll
        for (int d = 0; d < DIM; d++) Fn[0] += (R)0.5 * Fo[d][0] * n[d];  // ghost gradient is zero
      } else {
        if constexpr (BC) {
          R Fb[DIM][NV];
          if (-1 - code == BC_ADI_NOSLIP) {
            R gR[DIM * NV];
            adiabatic_gradient<DIM, R>(UL, UR, g, gR, ph);
            visc_flux<C, R>(UR, gR, Fb, ph);
          } else {
#pragma unroll
            for (int d = 0; d < DIM; d++)
#pragma unroll
              for (int v = 0; v < NV; v++) Fb[d][v] = Fo[d][v];
          }
#pragma unroll
          for (int v = 0; v < NV; v++) {
            R bn = 0;
#pragma unroll
            for (int d = 0; d < DIM; d++) bn += Fb[d][v] * n[d];
            Fn[v] += bn + tau * nn * (UL[v] - UR[v]);
          }
        }
      }
    }
#pragma unroll
    for (int v = 0; v < NV; v++) {
      const R fo = right ? -Fn[v] * dA : Fn[v] * dA;
      Js[(v * NF + f) * TE + e] = fo - dis[v];
    }
  }
  __syncthreads();

  update_phase<C, R, S, TE>(a, op, Fs, Js, Us, e0);
  if (a.flags & SF_RESIDUAL) return;
  __syncthreads();
  trace_phase<C, R, S, TE>(a, op, Us, e0);
}

// ----------------------------------------------------------------------------
// Traces of a double state (solver::extrapolateU), one thread per
// (flux point, element).
// ----------------------------------------------------------------------------
template <class C, typename R, typename S>
__global__ void fr_trace_kernel(const double *__restrict__ U, S *__restrict__ tr, int nE, int nEle, int ldU,
                                int vcjh) {
  constexpr int NS = C::NS, NSP = C::NSP, NF = C::NF, NV = C::NV, N1 = C::N1;
  const OpTab<R> &op = optab<R>(vcjh, C::P);
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)NF * nE) return;
  const int f = (int)(idx / nE), eg = (int)(idx - (long)f * nE);
  if (eg >= nEle) return;
  int dir, side, s0, st;
  fpt_line<C>(f, dir, side, s0, st);
#pragma unroll
  for (int v = 0; v < NV; v++) {
    R t = 0;
#pragma unroll
    for (int j = 0; j < N1; j++) t += op.lag[side][j] * (R)U[((size_t)v * NS + s0 + j * st) * ldU + eg];
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
