// kernels_tma.cuh -- the RK stage kernel of the fused update path with its
// tiles moved by the Tensor Memory Accelerator.
//
// The generic stage kernel (kernels.cuh) loads its inputs with per-thread
// loads, so each phase waits on a few loads in flight per thread.  Here one
// thread issues, at block start, every tile the block will need as 2D bulk
// tensor copies (cp.async.bulk.tensor) into shared memory, in three groups
// completing on three mbarriers:
//   group 0  stage state, JGinv, neighbour codes       (phase A, gathers)
//   group 1  face normals, dA, own traces               (phase B)
//   group 2  detJ, U0, RK accumulator                   (phase C)
// so the block's whole input is in flight at once while the earlier phases
// compute.  Neighbour traces, which are a gather, go to shared memory with
// cp.async as soon as the codes arrive.  Results (next stage state, RK
// accumulator or final state, traces) are staged in shared memory and written
// back with bulk tensor stores.  No multicast is used.
//
// Every mbarrier wait is bounded: on time-out the block records
// ERRF_TIMEOUT, waits (bounded again) for its copies, and returns.
#pragma once
#include <cuda.h>

#include "kernels.cuh"

namespace frg {

enum : unsigned { ERRF_TIMEOUT = 8u, ERRF_ALIGN = 16u };

// Tensor maps of one stage launch (all 2D: [rows][element stride]).
struct TmaMaps {
  CUtensorMap U;      // double [NV*NS]: stage-0 input, U0, final state
  CUtensorMap Acc;    // double [NV*NS]: RK accumulator
  CUtensorMap Win;    // S [NV*NS]: stage input (stages >= 1)
  CUtensorMap Wout;   // S [NV*NS]: next stage state
  CUtensorMap trOut;  // S [NV*NF]: traces of the new state
  CUtensorMap trIn;   // S [NV*NF]: traces of the stage input (own tile)
  CUtensorMap JG;     // S [DIM*DIM*NS]
  CUtensorMap det;    // S [NS]: 1 / detJ
  CUtensorMap nrm;    // S [DIM*NF]
  CUtensorMap dA;     // S [NF]
  CUtensorMap nbr;    // int32 [NF]
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t cnt) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(cnt) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: false after ~2^22 polls (each poll itself blocks for a
// hardware-defined interval), never an unbounded spin.
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity) {
  for (int i = 0; i < (1 << 22); i++)
    if (mbar_try_wait(b, parity)) return true;
  return false;
}
__device__ __forceinline__ void tma_load2d(void *dst, const CUtensorMap *m, int x, int y, uint64_t *b) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(smem_u32(dst)), "l"(m), "r"(x), "r"(y), "r"(smem_u32(b))
      : "memory");
}
__device__ __forceinline__ void tma_store2d(const CUtensorMap *m, int x, int y, const void *src) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(m), "r"(x),
               "r"(y), "r"(smem_u32(src))
               : "memory");
}
__device__ __forceinline__ void tma_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void tma_wait_reads() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
template <int BYTES>
__device__ __forceinline__ void cp_async_small(void *dst, const void *src) {
  static_assert(BYTES == 4 || BYTES == 8, "cp.async size");
  if constexpr (BYTES == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// Programmatic dependent launch.  Launched with the programmatic-
// serialization attribute, a stage kernel's blocks may start while the
// previous stage's last blocks still run; they issue the loads of the
// read-only metric tiles, then wait (pdl_wait) until the previous grid has
// finished and its writes are visible before touching anything a stage
// writes.  Each block signals at its start that the next stage may be
// scheduled (it is, once every block of this grid has signalled or exited).
// Launched without the attribute, both are no-ops.
__device__ __forceinline__ void pdl_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// First stage of a step with the fused dt: the slot the last stage will
// minimise the next dt into starts at a huge value (the bytes 0x7F, as a
// memset before the step would leave it); the stages in between do not read it.
__device__ __forceinline__ void stage_dt_reset(const StageArgs &a) {
  if (a.dtReset && blockIdx.x == 0 && threadIdx.x == 0) *a.dtReset = __longlong_as_double(0x7F7F7F7F7F7F7F7FLL);
}

// Tile of the TMA kernel: TE elements (box inner extent TE * sizeof >= 16 B),
// NT threads.  TE_ = 0 picks the widest of 16/8/4 elements whose shared
// memory stays within 72 KB (three blocks per SM); TE_ = -1 half of that,
// -2 a quarter (at least 4 elements: the 16-byte TMA box minimum).
template <class C, typename R, typename S, int TE_ = 0, int NT_ = 128>
struct TileT {
  static constexpr int NS = C::NS, NF = C::NF, NV = C::NV, D = C::DIM;
  static constexpr int per_ele(int te) {
    (void)te;
    return NV * NS * 8 * 2 + NV * NS * (int)sizeof(R) + D * D * NS * (int)sizeof(S) + NS * (int)sizeof(S) +
           D * NF * (int)sizeof(S) + NF * (int)sizeof(S) + NF * 4 + D * NV * NS * (int)sizeof(R) +
           NV * NF * (int)sizeof(R) + NF * 8 + NV * NF * (int)sizeof(S);
  }
  static constexpr int PER_ELE = per_ele(0);
  static constexpr int TE_AUTO = (16 * PER_ELE <= 72 * 1024) ? 16 : (8 * PER_ELE <= 72 * 1024) ? 8 : 4;
  static constexpr int TE = TE_ > 0 ? TE_ : TE_ == 0 ? TE_AUTO : TE_ == -1 ? (TE_AUTO > 4 ? TE_AUTO / 2 : 4)
                                                              : (TE_AUTO > 8 ? TE_AUTO / 4 : 4);
  static constexpr int NT = NT_;
  // blocks per SM the register budget is sized for
  static constexpr int MINB = NT_ >= 192 ? 2 : NT_ <= 64 ? 4 : 1;
  static constexpr int al(int b) { return (b + 127) & ~127; }
  // byte offsets of the shared-memory regions (each 128-byte aligned)
  static constexpr int oU0 = 0;
  static constexpr int oAcc = oU0 + al(NV * NS * TE * 8);
  static constexpr int oUs = oAcc + al(NV * NS * TE * 8);
  static constexpr int oJG = oUs + al(NV * NS * TE * (int)sizeof(R));
  static constexpr int oDet = oJG + al(D * D * NS * TE * (int)sizeof(S));
  static constexpr int oNrm = oDet + al(NS * TE * (int)sizeof(S));
  static constexpr int oDA = oNrm + al(D * NF * TE * (int)sizeof(S));
  static constexpr int oNbr = oDA + al(NF * TE * (int)sizeof(S));
  static constexpr int oTw = oNbr + al(NF * TE * 4);
  static constexpr int oFs = oTw + al(NV * NF * TE * (int)sizeof(S));
  static constexpr int oJs = oFs + al(D * NV * NS * TE * (int)sizeof(R));
  static constexpr int oWs = oJs + al(NV * NF * TE * (int)sizeof(R));
  static constexpr int oBar = oWs + al(NF * TE * 8);
  static constexpr int SMEM = oBar + 64 + 128;  // + room to align the base
};

// Shared-memory regions of one tile: what the bulk tensor loads fill (and
// the results leave from) and the block's working arrays.
template <typename R, typename S>
struct TmaBufs {
  double *U0, *Acc;  // [NV][NS][TE] FP64 step-start state and RK accumulator
  R *Us;             // [NV][NS][TE] stage state, then the new state
  S *JG, *Det, *Nrm, *DA;
  int *Nbr;
  S *Tw;       // [NV][NF][TE] traces of the stage input (the previous launch's phase D)
  R *Fs;       // [DIM][NV][NS][TE] contravariant flux
  R *Js;       // [NV][NF][TE] neighbour traces, then the jumps
  S *TrO;      // [NV][NF][TE] traces of the new state (may alias Js)
  double *Ws;  // [NF][TE] terms of ele::calcDt's surface integral
  double *Wd;  // [2][NF][TE] stored wave speeds and dA, then [TE] element volumes (SF_DTNEXT), or null
};

// Which inputs a stage reads, from its flags.
struct TmaNeeds {
  bool inU, needU0, needAcc;
  __device__ __forceinline__ explicit TmaNeeds(const StageArgs &a) {
    const bool last = a.flags & SF_LAST, first = a.flags & SF_FIRST, jam = a.flags & SF_JAMESON;
    inU = a.Uin_d != nullptr;  // stage input is the double state U
    needU0 = !inU && (jam || !last);
    needAcc = !first && !jam;
  }
};

// One thread: the bulk tensor loads of the tile starting at element e0, in
// three groups on bar[0..2] (see the file comment).  part 1: every group's
// expected byte count and the read-only metric tiles; part 2: the tiles a
// previous stage writes (state, traces, U0, accumulator); both parts when
// part is 0.
template <class C, typename R, typename S, int TE>
__device__ __forceinline__ void tma_issue_tile(const TmaMaps &m, const TmaNeeds &nd, const TmaBufs<R, S> &b, int e0,
                                               uint64_t *bar, int part = 0) {
  constexpr int NS = C::NS, NF = C::NF, NV = C::NV, DIM = C::DIM;
  if (part != 2) {
    const uint32_t b0 = (nd.inU ? NV * NS * TE * 8 : NV * NS * TE * (int)sizeof(S)) +
                        DIM * DIM * NS * TE * sizeof(S) + NF * TE * 4;
    mbar_expect_tx(&bar[0], b0);
    mbar_expect_tx(&bar[1], (DIM * NF * TE + NF * TE + NV * NF * TE) * sizeof(S));
    const uint32_t b2 =
        NS * TE * sizeof(S) + (nd.needU0 ? NV * NS * TE * 8 : 0) + (nd.needAcc ? NV * NS * TE * 8 : 0);
    mbar_expect_tx(&bar[2], b2);
    tma_load2d(b.JG, &m.JG, e0, 0, &bar[0]);
    tma_load2d(b.Nbr, &m.nbr, e0, 0, &bar[0]);
    tma_load2d(b.Nrm, &m.nrm, e0, 0, &bar[1]);
    tma_load2d(b.DA, &m.dA, e0, 0, &bar[1]);
    tma_load2d(b.Det, &m.det, e0, 0, &bar[2]);
  }
  if (part == 1) return;
  if (nd.inU) tma_load2d(b.U0, &m.U, e0, 0, &bar[0]);
  else tma_load2d(b.Us, &m.Win, e0, 0, &bar[0]);
  tma_load2d(b.Tw, &m.trIn, e0, 0, &bar[1]);
  if (nd.needU0) tma_load2d(b.U0, &m.U, e0, 0, &bar[2]);
  if (nd.needAcc) tma_load2d(b.Acc, &m.Acc, e0, 0, &bar[2]);
}

// Neighbour traces of the tile's interior flux points into Js, and with
// SF_DTNEXT the stored wave speeds and dA into Wd (cp.async; the caller waits
// with cp_async_wait_all before phase B).
template <class C, typename S, int TE, int NT, typename R>
__device__ __forceinline__ void tma_gather(const StageArgs &a, const int *sNbr, R *Js, double *Wd, int e0) {
  constexpr int NF = C::NF, NV = C::NV;
  const S *trIn = static_cast<const S *>(a.trIn);
  const int L = a.nE;
  const bool dtn = (a.flags & SF_DTNEXT) && Wd;
  for (int it = threadIdx.x; it < NF * TE; it += NT) {
    const int f = it / TE, e = it - f * TE;
    if (e0 + e >= a.nEle) continue;
    if (dtn) {
      cp_async_small<8>(&Wd[it], &a.waveSp[(size_t)f * L + e0 + e]);
      cp_async_small<8>(&Wd[NF * TE + it], &a.dAd[(size_t)f * L + e0 + e]);
    }
    const int code = sNbr[f * TE + e];
    if (code < 0) continue;
    const size_t t = (size_t)(code >> 1);
#pragma unroll
    for (int v = 0; v < NV; v++) cp_async_small<sizeof(S)>(&Js[(v * NF + f) * TE + e], &trIn[(size_t)v * NF * L + t]);
  }
}

// Phase A: contravariant inviscid flux at the solution points
// (calcInviscidFlux_spts, src/solver.cpp:514-539); with a double stage
// input, also its conversion into Us.
template <class C, typename R, typename S, int TE, int NT>
__device__ __forceinline__ void tma_phase_a(const StageArgs &a, bool inU, const TmaBufs<R, S> &b, int e0) {
  constexpr int NS = C::NS, NV = C::NV, DIM = C::DIM;
  for (int it = threadIdx.x; it < NS * TE; it += NT) {
    const int s = it / TE, e = it - s * TE;
    if (e0 + e >= a.nEle) continue;
    R u[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) {
      const int o = (v * NS + s) * TE + e;
      u[v] = inU ? (R)b.U0[o] : b.Us[o];
      if (inU) b.Us[o] = u[v];
    }
    R F[DIM][NV];
    inviscid_flux<DIM, NV, R>(u, F, a.ph);
#pragma unroll
    for (int d1 = 0; d1 < DIM; d1++)
#pragma unroll
      for (int v = 0; v < NV; v++) {
        R t = 0;
#pragma unroll
        for (int d2 = 0; d2 < DIM; d2++) t += (R)b.JG[((d1 * DIM + d2) * NS + s) * TE + e] * F[d2][v];
        b.Fs[((d1 * NV + v) * NS + s) * TE + e] = t;
      }
  }
}

// Phase B: own trace, neighbour trace (already in Js) or ghost state, common
// flux and the jump Fn*dA - disFn into Js (face::calcInviscidFlux,
// extrapolateNormalFlux, correctDivFlux's jump).  The own trace is the one the
// previous launch's phase D (or the trace kernel) left in the trace buffer:
// the same sum over the same line in the same order, so the same value.
template <class C, typename R, typename S, bool BC, int RS, int TE, int NT>
__device__ __forceinline__ void tma_phase_b(const StageArgs &a, const OpTab<R> &op, const TmaBufs<R, S> &b, int e0) {
  constexpr int NS = C::NS, NF = C::NF, NV = C::NV, DIM = C::DIM, N1 = C::N1;
  const int L = a.nE, flags = a.flags;
  for (int it = threadIdx.x; it < NF * TE; it += NT) {
    const int f = it / TE, e = it - f * TE, eg = e0 + e;
    if (eg >= a.nEle) continue;
    int dir, side, s0, st;
    fpt_line<C>(f, dir, side, s0, st);
    R own[NV], dis[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) {
      R q = 0;
#pragma unroll
      for (int j = 0; j < N1; j++) q += op.lag[side][j] * b.Fs[((dir * NV + v) * NS + s0 + j * st) * TE + e];
      own[v] = (R)b.Tw[(v * NF + f) * TE + e];
      dis[v] = side ? q : -q;
    }
    R n[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) n[d] = (R)b.Nrm[(d * NF + f) * TE + e];
    const R dA = (R)b.DA[f * TE + e];
    const int code = b.Nbr[f * TE + e];
    R oth[NV];
    bool right = false;
    if (code >= 0) {
      right = code & 1;
#pragma unroll
      for (int v = 0; v < NV; v++) oth[v] = b.Js[(v * NF + f) * TE + e];
    } else {
      if constexpr (NV == 1 || !BC) {
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
    const R *UL = right ? oth : own;
    const R *UR = right ? own : oth;
    R Fn[NV];
    const R ws = inviscid_common<C, R, BC, RS>(UL, UR, n, code, Fn, a.ph);
    const bool upd = !right && ws >= 0;
    if ((flags & SF_WAVESP) && upd) a.waveSp[(size_t)f * L + eg] = (double)ws;
    if (flags & SF_DTNEXT)  // this flux point's term of ele::calcDt's surface integral
      b.Ws[f * TE + e] = b.Wd ? (upd ? (double)ws : b.Wd[f * TE + e]) * a.wsurf[f % C::NFF] * b.Wd[NF * TE + f * TE + e]
                              : (upd ? (double)ws : a.waveSp[(size_t)f * L + eg]) * a.wsurf[f % C::NFF] *
                                    a.dAd[(size_t)f * L + eg];
#pragma unroll
    for (int v = 0; v < NV; v++) {
      const R fo = right ? -Fn[v] * dA : Fn[v] * dA;
      b.Js[(v * NF + f) * TE + e] = fo - dis[v];
    }
  }
}

// Phase C: divergence + correction and the FP64 RK update into the staging
// tiles, along coordinate lines.  Pass C1 takes the xi-derivative of the
// xi-flux along each row j plus the correction from the row's left/right
// flux points, for all N1 points of the row at once, into Us (free since
// phase B); pass C2 adds the eta part along each column i and does the RK
// update of the column's points.  One item = (line, field, element): the
// line's N1 values are loaded once and N1 results formed.  Items run
// element-fastest, then line, then field, so the lane groups of a warp
// fall on different shared-memory banks (the field stride of the flux-point
// arrays is a multiple of 32 words).  Contains a block barrier between the
// passes.  The RK update scales the divergence by 1/detJ in the arithmetic
// type, then by the stage's coefficient x dt in FP64.  COLTR: pass C2, which
// holds each column of the new state, also writes the column's bottom and
// top traces into TrO (phase D then does the rows): the sums phase D would
// form, in the same order over the same values.
template <class C, typename R, typename S, int TE, int NT, bool COLTR = false>
__device__ __forceinline__ void tma_phase_c(const StageArgs &a, const OpTab<R> &op, const TmaBufs<R, S> &b, int e0,
                                            double dtG) {
  constexpr int NS = C::NS, NF = C::NF, NV = C::NV, N1 = C::N1;
  static_assert(C::DIM == 2, "the TMA stage kernel is two-dimensional");
  const int flags = a.flags;
  const bool first = flags & SF_FIRST, last = flags & SF_LAST, jam = flags & SF_JAMESON;
  for (int it = threadIdx.x; it < N1 * NV * TE; it += NT) {
    const int e = it % TE, r = it / TE, j = r % N1, v = r / N1;
    if (e0 + e >= a.nEle) continue;
    R F[N1];
#pragma unroll
    for (int q = 0; q < N1; q++) F[q] = b.Fs[((0 * NV + v) * NS + j * N1 + q) * TE + e];
    const R JL = b.Js[(v * NF + 3 * N1 + C::P - j) * TE + e], JR = b.Js[(v * NF + N1 + j) * TE + e];
#pragma unroll
    for (int i = 0; i < N1; i++) {
      R acc = 0;
#pragma unroll
      for (int q = 0; q < N1; q++) acc += op.dlag[i][q] * F[q];
      acc += -op.gL[i] * JL;
      acc += op.gR[i] * JR;
      b.Us[(v * NS + j * N1 + i) * TE + e] = acc;
    }
  }
  __syncthreads();
  for (int it = threadIdx.x; it < N1 * NV * TE; it += NT) {
    const int e = it % TE, r = it / TE, i = r % N1, v = r / N1, eg = e0 + e;
    if (eg >= a.nEle) continue;
    const double dtl = a.grp ? a.dt[a.grp[eg]] : a.dtLocal ? a.dt[eg] : dtG;
    const double cb = a.bCur * dtl, ca = a.aNext * dtl;
    R F[N1];
#pragma unroll
    for (int q = 0; q < N1; q++) F[q] = b.Fs[((1 * NV + v) * NS + q * N1 + i) * TE + e];
    const R JB = b.Js[(v * NF + i) * TE + e], JT = b.Js[(v * NF + 2 * N1 + C::P - i) * TE + e];
    R t0 = 0, t1 = 0;  // COLTR: the column's bottom / top traces
#pragma unroll
    for (int j = 0; j < N1; j++) {
      const int s = j * N1 + i, o = (v * NS + s) * TE + e;
      R acc = b.Us[o];
#pragma unroll
      for (int q = 0; q < N1; q++) acc += op.dlag[j][q] * F[q];
      acc += -op.gL[j] * JB;
      acc += op.gR[j] * JT;
      if (flags & SF_DIVF) a.divF[((size_t)v * NS + s) * a.ldU + eg] = (double)acc;
      const double dj = (double)(acc * (R)b.Det[s * TE + e]);  // divF / detJ
      double unew;
      if (jam) {
        unew = b.U0[o] - ca * dj;
        if (last) b.U0[o] = unew;
      } else {
        const double t = cb * dj;
        const double base = first ? b.U0[o] : b.Acc[o];
        if (last) {
          unew = base - t;
          b.U0[o] = unew;
        } else {
          b.Acc[o] = base - t;
          const double u0 = first ? base : b.U0[o];
          unew = u0 - ca * dj;
        }
      }
      if (last && (v == 0 || v == NV - 1) && isnan(unew)) atomicOr(a.err, ERRF_NAN);
      const R un = (R)(last ? unew : (double)(S)unew);
      b.Us[o] = un;
      if (COLTR) {
        t0 += op.lag[0][j] * un;
        t1 += op.lag[1][j] * un;
      }
    }
    if (COLTR) {
      b.TrO[(v * NF + i) * TE + e] = (S)t0;
      b.TrO[(v * NF + 2 * N1 + C::P - i) * TE + e] = (S)t1;
    }
  }
}

// Phase D: traces of the new state into TrO; one item per (line, field,
// element) gives the traces at both ends of the line (rows: left face 3 /
// right face 1; columns: bottom face 0 / top face 2).  ROWS: the rows only
// (phase C wrote the columns').
template <class C, typename R, typename S, int TE, int NT, bool ROWS = false>
__device__ __forceinline__ void tma_phase_d(const OpTab<R> &op, const R *Us, S *TrO) {
  constexpr int NS = C::NS, NF = C::NF, NV = C::NV, N1 = C::N1, NL = ROWS ? N1 : 2 * N1;
  for (int it = threadIdx.x; it < NL * NV * TE; it += NT) {
    const int e = it % TE, r = it / TE, ln = r % NL, v = r / NL;
    const bool row = ln < N1;
    const int k = row ? ln : ln - N1;
    const int s0 = row ? k * N1 : k, st = row ? 1 : N1;
    R t0 = 0, t1 = 0;
#pragma unroll
    for (int q = 0; q < N1; q++) {
      const R u = Us[(v * NS + s0 + q * st) * TE + e];
      t0 += op.lag[0][q] * u;
      t1 += op.lag[1][q] * u;
    }
    const int f0 = row ? 3 * N1 + C::P - k : k, f1 = row ? N1 + k : 2 * N1 + C::P - k;
    TrO[(v * NF + f0) * TE + e] = (S)t0;
    TrO[(v * NF + f1) * TE + e] = (S)t1;
  }
}

// ele::calcDt for element e0 + ln (lane ln < TE) with the wave speeds this stage
// left (src/ele.cpp:1086-1105; flux points summed in order).  Returns the
// element's dt (INFINITY for other threads); in ensemble mode also reduces
// into the element's group minimum.
template <int NF, int TE>
__device__ __forceinline__ double tma_tile_dt(const StageArgs &a, const double *Ws, int e0, int ln,
                                              const double *volS = nullptr) {
  const int eg = e0 + ln;
  if (ln >= TE || eg >= a.nEle) return INFINITY;
  double iw = 0;
#pragma unroll
  for (int f = 0; f < NF; f++) iw += Ws[f * TE + ln];
  const double dte = a.cflFac * (volS ? volS[ln] : a.vol[eg]) / iw;
  a.eleDt[eg] = dte;
  if (a.grp) {  // ensemble mode: each element into its own group's minimum
    if (!(dte > 1e-13)) atomicOr(a.err, ERRF_DT);
    if (dte > 0)  // a tiny dt is still used, as the reference does before its check
      atomicMin(reinterpret_cast<unsigned long long *>(a.dtNext + a.grp[eg]),
                (unsigned long long)__double_as_longlong(dte));
  }
  return dte;
}

// Warp 0: minimum of the lanes' dt, then the global minimum by a 64-bit
// atomicMin on the bit pattern (positive doubles order like their bit
// patterns) into the next step's dt slot, which the host set to a huge value.
__device__ __forceinline__ void tma_dt_reduce(const StageArgs &a, double my) {
  for (int o = 16; o > 0; o >>= 1) {
    const double t = __shfl_xor_sync(0xffffffffu, my, o);
    my = (isnan(t) || t < my) ? t : my;
  }
  if ((threadIdx.x & 31) == 0 && !a.grp) {
    if (!(my > 1e-13)) atomicOr(a.err, ERRF_DT);  // also catches NaN
    if (my > 0)  // a tiny dt is still used, as the reference does before its check
      atomicMin(reinterpret_cast<unsigned long long *>(a.dtNext), (unsigned long long)__double_as_longlong(my));
  }
}

template <class C, typename R, typename S, bool BC, int RS, int TEV, int NTV>
__global__ void __launch_bounds__(NTV, (TileT<C, R, S, TEV, NTV>::MINB))
    fr_stage_tma_kernel(const StageArgs a, const __grid_constant__ TmaMaps m) {
  static_assert(sizeof(R) == sizeof(S), "stage state is loaded straight into the compute buffer");
  using T = TileT<C, R, S, TEV, NTV>;
  constexpr int TE = T::TE, NT = T::NT, NF = C::NF;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // bulk-tensor destinations start on 128-byte boundaries
  unsigned char *const sb = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  TmaBufs<R, S> b;
  b.U0 = reinterpret_cast<double *>(sb + T::oU0);
  b.Acc = reinterpret_cast<double *>(sb + T::oAcc);
  b.Us = reinterpret_cast<R *>(sb + T::oUs);
  b.JG = reinterpret_cast<S *>(sb + T::oJG);
  b.Det = reinterpret_cast<S *>(sb + T::oDet);
  b.Nrm = reinterpret_cast<S *>(sb + T::oNrm);
  b.DA = reinterpret_cast<S *>(sb + T::oDA);
  b.Nbr = reinterpret_cast<int *>(sb + T::oNbr);
  b.Tw = reinterpret_cast<S *>(sb + T::oTw);
  b.Fs = reinterpret_cast<R *>(sb + T::oFs);
  b.Js = reinterpret_cast<R *>(sb + T::oJs);
  b.TrO = reinterpret_cast<S *>(b.Js);  // the new traces replace the jumps
  b.Ws = reinterpret_cast<double *>(sb + T::oWs);
  b.Wd = nullptr;  // wave speeds and dA read from global memory in phase B
  uint64_t *bar = reinterpret_cast<uint64_t *>(sb + T::oBar);

  const OpTab<R> &op = stage_op<R>(a);
  const int tid = threadIdx.x, e0 = blockIdx.x * TE;
  const int flags = a.flags;
  const bool last = flags & SF_LAST, jam = flags & SF_JAMESON;
  const TmaNeeds nd(a);

  if (tid == 0) {
    for (int i = 0; i < 3; i++) mbar_init(&bar[i], 1);
    fence_mbar_init();
  }
  __syncthreads();
  pdl_launch_dependents();
  if (tid == 0) tma_issue_tile<C, R, S, TE>(m, nd, b, e0, bar, 1);
  pdl_wait();  // the previous stage has finished: its outputs are visible
  stage_dt_reset(a);
  if (tid == 0) tma_issue_tile<C, R, S, TE>(m, nd, b, e0, bar, 2);

  // the global dt, fetched while the tiles are in flight
  const double dtG = (a.dtLocal || a.grp) ? 0.0 : __ldg(a.dt);

  // ---- group 0: gathers of neighbour traces, then phase A
  bool ok = mbar_wait(&bar[0], 0);
  if (__syncthreads_or(!ok)) goto timeout;
  tma_gather<C, S, TE, NT>(a, b.Nbr, b.Js, b.Wd, e0);
  tma_phase_a<C, R, S, TE, NT>(a, nd.inU, b, e0);
  cp_async_wait_all();
  ok = mbar_wait(&bar[1], 0);
  if (__syncthreads_or(!ok)) goto timeout;

  // ---- phase B: common flux and jumps (neighbour traces already in Js)
  tma_phase_b<C, R, S, BC, RS, TE, NT>(a, op, b, e0);
  ok = mbar_wait(&bar[2], 0);
  if (__syncthreads_or(!ok)) goto timeout;

  // ---- phase C: divergence + correction, RK update into the staging tiles
  tma_phase_c<C, R, S, TE, NT>(a, op, b, e0, dtG);
  if ((flags & SF_TIME) && !a.grp && blockIdx.x == 0 && tid == 0) *a.time += dtG;
  fence_proxy_async();
  __syncthreads();
  if (tid == 0) {
    if (last) tma_store2d(&m.U, e0, 0, b.U0);
    else {
      tma_store2d(&m.Wout, e0, 0, b.Us);
      if (!jam) tma_store2d(&m.Acc, e0, 0, b.Acc);
    }
    tma_commit();
  }

  // ---- phase D: traces of the new state, staged in Js
  tma_phase_d<C, R, S, TE, NT>(op, b.Us, b.TrO);
  fence_proxy_async();
  __syncthreads();
  if (tid == 0) {
    tma_store2d(&m.trOut, e0, 0, b.TrO);
    tma_commit();
  }
  if ((flags & SF_DTNEXT) && tid < 32) tma_dt_reduce(a, tma_tile_dt<NF, TE>(a, b.Ws, e0, tid));
  if (tid == 0) tma_wait_reads();
  return;

timeout:
  if (tid == 0) {
    atomicOr(a.err, ERRF_TIMEOUT);
    for (int i = 0; i < 3; i++) mbar_wait(&bar[i], 0);  // bounded: let copies in flight land
  }
  cp_async_wait_all();
  __syncthreads();
}

// ----------------------------------------------------------------------------
// Persistent variant: a grid of (SMs x resident blocks) blocks, each walking
// the tiles blockIdx.x, blockIdx.x + gridDim.x, ...  The tiles' loads go to
// a ring of NB buffers, and the loads of the block's next tile are issued
// while the current tile computes (at its start with NB = 3, after phase A
// with NB = 2, when the buffer's previous stores have been read), so the
// memory system has the next tile's bytes in flight during every phase.
// The traces of the new state have their own ring slot, so the single
// working arrays (Fs, Js, Ws) are free as soon as a tile's phase D ends.
// Same per-element arithmetic as fr_stage_tma_kernel, hence bit-identical.
// ----------------------------------------------------------------------------
template <class C, typename R, typename S, int TEV, int NT_, int NB_>
struct PipeT {
  static constexpr int NS = C::NS, NF = C::NF, NV = C::NV, D = C::DIM;
  static constexpr int NT = NT_, NB = NB_;
  static constexpr int al(int b) { return (b + 127) & ~127; }
  static constexpr int slot_bytes(int te) {
    return al(NV * NS * te * 8) * 2 + al(NV * NS * te * (int)sizeof(R)) + al(D * D * NS * te * (int)sizeof(S)) +
           al(NS * te * (int)sizeof(S)) + al(D * NF * te * (int)sizeof(S)) + al(NF * te * (int)sizeof(S)) +
           al(NF * te * 4) + 2 * al(NV * NF * te * (int)sizeof(S));
  }
  static constexpr int smem_bytes(int te) {
    return NB * slot_bytes(te) + al(D * NV * NS * te * (int)sizeof(R)) + al(NV * NF * te * (int)sizeof(R)) +
           al(NF * te * 8) + al((2 * NF + 1) * te * 8) + NB * 3 * 8 + 128;
  }
  // TEV = 0: the widest of 16/8/4 elements within 100 KB (two blocks per
  // SM); -1: half of that (at least 4, the 16-byte TMA box minimum)
  static constexpr int TE_AUTO = smem_bytes(16) <= 100 * 1024 ? 16 : smem_bytes(8) <= 100 * 1024 ? 8 : 4;
  static constexpr int TE = TEV > 0 ? TEV : TEV == 0 ? TE_AUTO : (TE_AUTO > 4 ? TE_AUTO / 2 : 4);
  // one ring slot
  static constexpr int oU0 = 0;
  static constexpr int oAcc = oU0 + al(NV * NS * TE * 8);
  static constexpr int oUs = oAcc + al(NV * NS * TE * 8);
  static constexpr int oJG = oUs + al(NV * NS * TE * (int)sizeof(R));
  static constexpr int oDet = oJG + al(D * D * NS * TE * (int)sizeof(S));
  static constexpr int oNrm = oDet + al(NS * TE * (int)sizeof(S));
  static constexpr int oDA = oNrm + al(D * NF * TE * (int)sizeof(S));
  static constexpr int oNbr = oDA + al(NF * TE * (int)sizeof(S));
  static constexpr int oTw = oNbr + al(NF * TE * 4);
  static constexpr int oTr = oTw + al(NV * NF * TE * (int)sizeof(S));
  static constexpr int SLOT = oTr + al(NV * NF * TE * (int)sizeof(S));
  // working arrays after the ring
  static constexpr int oFs = NB * SLOT;
  static constexpr int oJs = oFs + al(D * NV * NS * TE * (int)sizeof(R));
  static constexpr int oWs = oJs + al(NV * NF * TE * (int)sizeof(R));
  static constexpr int oWd = oWs + al(NF * TE * 8);
  static constexpr int oBar = oWd + al((2 * NF + 1) * TE * 8);
  static constexpr int SMEM = oBar + NB * 3 * 8 + 128;
  static_assert(SMEM == smem_bytes(TE), "layout");
  // resident blocks per SM the register budget is sized for
  static constexpr int MINB = SMEM <= 75 * 1024 && NT <= 192 ? 3 : SMEM <= 113 * 1024 ? 2 : 1;
};

template <class C, typename R, typename S, bool BC, int RS, int TEV, int NT, int NB>
__global__ void __launch_bounds__(NT, (PipeT<C, R, S, TEV, NT, NB>::MINB))
    fr_stage_tma_pipe_kernel(const StageArgs a, const __grid_constant__ TmaMaps m) {
  static_assert(sizeof(R) == sizeof(S), "stage state is loaded straight into the compute buffer");
  static_assert(NB == 2 || NB == 3, "ring depth");
  using T = PipeT<C, R, S, TEV, NT, NB>;
  constexpr int NF = C::NF, TE = T::TE;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char *const sb = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  auto slot = [&](int k) {
    unsigned char *p = sb + k * T::SLOT;
    TmaBufs<R, S> b;
    b.U0 = reinterpret_cast<double *>(p + T::oU0);
    b.Acc = reinterpret_cast<double *>(p + T::oAcc);
    b.Us = reinterpret_cast<R *>(p + T::oUs);
    b.JG = reinterpret_cast<S *>(p + T::oJG);
    b.Det = reinterpret_cast<S *>(p + T::oDet);
    b.Nrm = reinterpret_cast<S *>(p + T::oNrm);
    b.DA = reinterpret_cast<S *>(p + T::oDA);
    b.Nbr = reinterpret_cast<int *>(p + T::oNbr);
    b.Tw = reinterpret_cast<S *>(p + T::oTw);
    b.TrO = reinterpret_cast<S *>(p + T::oTr);
    b.Fs = reinterpret_cast<R *>(sb + T::oFs);
    b.Js = reinterpret_cast<R *>(sb + T::oJs);
    b.Ws = reinterpret_cast<double *>(sb + T::oWs);
    b.Wd = reinterpret_cast<double *>(sb + T::oWd);
    return b;
  };
  uint64_t *bar = reinterpret_cast<uint64_t *>(sb + T::oBar);  // [NB][3]

  const OpTab<R> &op = stage_op<R>(a);
  const int tid = threadIdx.x;
  const int nTiles = (a.nEle + TE - 1) / TE;
  const int flags = a.flags;
  const bool last = flags & SF_LAST, jam = flags & SF_JAMESON;
  const TmaNeeds nd(a);
  if ((int)blockIdx.x >= nTiles) return;

  if (tid == 0) {
    for (int i = 0; i < 3 * NB; i++) mbar_init(&bar[i], 1);
    fence_mbar_init();
  }
  __syncthreads();
  pdl_launch_dependents();
  if (tid == 0) tma_issue_tile<C, R, S, TE>(m, nd, slot(0), blockIdx.x * TE, &bar[0], 1);
  pdl_wait();  // the previous stage has finished: its outputs are visible
  stage_dt_reset(a);
  if (tid == 0) tma_issue_tile<C, R, S, TE>(m, nd, slot(0), blockIdx.x * TE, &bar[0], 2);
  const double dtG = (a.dtLocal || a.grp) ? 0.0 : __ldg(a.dt);
  double dtMin = INFINITY;
  const bool dtn = flags & SF_DTNEXT;
  int prevE0 = -1;  // the previous tile's first element, for its deferred dt
  int issued = 1;  // tiles whose loads have been issued (thread 0's count)
  bool ok = true;
  int j = 0;
  // Thread 0: the next tile's loads into its ring slot, once the stores that
  // last read that slot have been read out (wait_group.read N leaves the N
  // most recent store groups, two per tile, pending).
  auto prefetch = [&](int jn, int pending) {
    const int tn = blockIdx.x + jn * gridDim.x;
    if (tn >= nTiles) return;
    if (pending == 2) asm volatile("cp.async.bulk.wait_group.read 2;" ::: "memory");
    else asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
    tma_issue_tile<C, R, S, TE>(m, nd, slot(jn % NB), tn * TE, &bar[3 * (jn % NB)]);
    issued++;
  };
  for (;; j++) {
    const int t = blockIdx.x + j * gridDim.x;
    if (t >= nTiles) break;
    const int k = j % NB;
    const uint32_t par = (uint32_t)((j / NB) & 1);
    const TmaBufs<R, S> b = slot(k);
    uint64_t *bk = &bar[3 * k];
    const int e0 = t * TE;
    if (NB == 3 && tid == 0) prefetch(j + 1, 2);
    ok = mbar_wait(&bk[0], par);
    if (__syncthreads_or(!ok)) break;
    tma_gather<C, S, TE, NT>(a, b.Nbr, b.Js, b.Wd, e0);
    tma_phase_a<C, R, S, TE, NT>(a, nd.inU, b, e0);
    // the previous tile's ele::calcDt, by the last warp, which phase A's
    // second round leaves idle; Ws is rewritten only in this tile's phase B
    if (dtn && prevE0 >= 0 && (tid >> 5) == NT / 32 - 1)
      dtMin = fmin(dtMin, tma_tile_dt<NF, TE>(a, b.Ws, prevE0, tid & 31));
    if (NB == 2 && tid == 0) prefetch(j + 1, 0);
    if (dtn) {
      // the next tile's stored wave speeds and dA into L2, so its gathers
      // (at its start) do not wait on DRAM
      const int tn = blockIdx.x + (j + 1) * gridDim.x;
      if (tn < nTiles)
        for (int r = tid; r < 2 * NF; r += NT) {
          const double *src = r < NF ? a.waveSp : a.dAd;
          asm volatile("prefetch.global.L2 [%0];" ::"l"(src + (size_t)(r % NF) * a.nE + (size_t)tn * TE));
        }
    }
    cp_async_wait_all();
    ok = mbar_wait(&bk[1], par);
    if (__syncthreads_or(!ok)) break;
    tma_phase_b<C, R, S, BC, RS, TE, NT>(a, op, b, e0);
    ok = mbar_wait(&bk[2], par);
    if (__syncthreads_or(!ok)) break;
    tma_phase_c<C, R, S, TE, NT, true>(a, op, b, e0, dtG);
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      if (last) tma_store2d(&m.U, e0, 0, b.U0);
      else {
        tma_store2d(&m.Wout, e0, 0, b.Us);
        if (!jam) tma_store2d(&m.Acc, e0, 0, b.Acc);
      }
      tma_commit();
    }
    tma_phase_d<C, R, S, TE, NT, true>(op, b.Us, b.TrO);
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      tma_store2d(&m.trOut, e0, 0, b.TrO);
      tma_commit();
    }
    prevE0 = e0;
    // the next tile's phase B rewrites Ws only after the barrier at its start
  }
  if (!ok) {
    // a bounded wait gave up: flag it, let every issued load land (bounded
    // again) so no copy targets shared memory after the block exits
    if (tid == 0) {
      atomicOr(a.err, ERRF_TIMEOUT);
      for (int q = j; q < j + NB && q < issued; q++)
        for (int g = 0; g < 3; g++) mbar_wait(&bar[3 * (q % NB) + g], (uint32_t)((q / NB) & 1));
    }
    cp_async_wait_all();
    __syncthreads();
    if (tid == 0) tma_wait_reads();
    return;
  }
  if ((flags & SF_TIME) && !a.grp && blockIdx.x == 0 && tid == 0) *a.time += dtG;
  if (dtn && (tid >> 5) == NT / 32 - 1) {
    if (prevE0 >= 0) dtMin = fmin(dtMin, tma_tile_dt<NF, TE>(a, slot(0).Ws, prevE0, tid & 31));
    tma_dt_reduce(a, dtMin);
  }
  if (tid == 0) tma_wait_reads();
}

// ----------------------------------------------------------------------------
// Split variant: the persistent ring of fr_stage_tma_pipe_kernel with the
// FP64 step-start state and RK accumulator kept OUT of the ring, in one
// buffer each per block.  The next tile's U0 (or, in the first stage, its
// double stage input) is loaded into its buffer as soon as the current
// tile's phase C has read it; the accumulator, which is a store source, at
// the start of the next tile once the stores have been read out.  The ring
// slots shrink by two thirds, so four blocks fit per SM instead of three
// (and registers are capped to match).  Same per-element arithmetic, hence
// bit-identical.
// ----------------------------------------------------------------------------
template <class C, typename R, typename S, int TEV, int NT_>
struct SplitT {
  static constexpr int NS = C::NS, NF = C::NF, NV = C::NV, D = C::DIM;
  static constexpr int NT = NT_;
  static constexpr int al(int b) { return (b + 127) & ~127; }
  static constexpr int slot_bytes(int te) {
    return al(NV * NS * te * (int)sizeof(R)) + al(D * D * NS * te * (int)sizeof(S)) + al(NS * te * (int)sizeof(S)) +
           al(D * NF * te * (int)sizeof(S)) + al(NF * te * (int)sizeof(S)) + al(NF * te * 4) +
           2 * al(NV * NF * te * (int)sizeof(S));
  }
  static constexpr int smem_bytes(int te) {
    return 2 * slot_bytes(te) + 2 * al(NV * NS * te * 8) + al(D * NV * NS * te * (int)sizeof(R)) +
           al(NV * NF * te * (int)sizeof(R)) + al(NF * te * 8) + al((2 * NF + 1) * te * 8) + al(2 * te * 8) + 8 * 8 +
           128;
  }
  // the widest of 16/8/4 elements within 56 KB (four blocks per SM)
  static constexpr int TE_AUTO = smem_bytes(16) <= 56 * 1024 ? 16 : smem_bytes(8) <= 56 * 1024 ? 8 : 4;
  static constexpr int TE = TEV > 0 ? TEV : TE_AUTO;
  static constexpr int oUs = 0;
  static constexpr int oJG = oUs + al(NV * NS * TE * (int)sizeof(R));
  static constexpr int oDet = oJG + al(D * D * NS * TE * (int)sizeof(S));
  static constexpr int oNrm = oDet + al(NS * TE * (int)sizeof(S));
  static constexpr int oDA = oNrm + al(D * NF * TE * (int)sizeof(S));
  static constexpr int oNbr = oDA + al(NF * TE * (int)sizeof(S));
  static constexpr int oTw = oNbr + al(NF * TE * 4);
  static constexpr int oTr = oTw + al(NV * NF * TE * (int)sizeof(S));
  static constexpr int SLOT = oTr + al(NV * NF * TE * (int)sizeof(S));
  static constexpr int oU0 = 2 * SLOT;
  static constexpr int oAcc = oU0 + al(NV * NS * TE * 8);
  static constexpr int oFs = oAcc + al(NV * NS * TE * 8);
  static constexpr int oJs = oFs + al(D * NV * NS * TE * (int)sizeof(R));
  static constexpr int oWs = oJs + al(NV * NF * TE * (int)sizeof(R));
  static constexpr int oWd = oWs + al(NF * TE * 8);
  static constexpr int oVol = oWd + al((2 * NF + 1) * TE * 8);  // double [2][TE] element volumes, by tile parity
  static constexpr int oBar = oVol + al(2 * TE * 8);
  static constexpr int SMEM = oBar + 8 * 8 + 128;
  static_assert(SMEM == smem_bytes(TE), "layout");
  static constexpr int MINB = SMEM <= 56 * 1024 && NT <= 160 ? 4 : SMEM <= 75 * 1024 && NT <= 192 ? 3 : 2;
};

template <class C, typename R, typename S, bool BC, int RS, int TEV, int NT>
__global__ void __launch_bounds__(NT, (SplitT<C, R, S, TEV, NT>::MINB))
    fr_stage_tma_split_kernel(const StageArgs a, const __grid_constant__ TmaMaps m) {
  static_assert(sizeof(R) == sizeof(S), "stage state is loaded straight into the compute buffer");
  using T = SplitT<C, R, S, TEV, NT>;
  constexpr int NS = C::NS, NF = C::NF, NV = C::NV, DIM = C::DIM, TE = T::TE;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char *const sb = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  auto slot = [&](int k) {
    unsigned char *p = sb + k * T::SLOT;
    TmaBufs<R, S> b;
    b.U0 = reinterpret_cast<double *>(sb + T::oU0);
    b.Acc = reinterpret_cast<double *>(sb + T::oAcc);
    b.Us = reinterpret_cast<R *>(p + T::oUs);
    b.JG = reinterpret_cast<S *>(p + T::oJG);
    b.Det = reinterpret_cast<S *>(p + T::oDet);
    b.Nrm = reinterpret_cast<S *>(p + T::oNrm);
    b.DA = reinterpret_cast<S *>(p + T::oDA);
    b.Nbr = reinterpret_cast<int *>(p + T::oNbr);
    b.Tw = reinterpret_cast<S *>(p + T::oTw);
    b.TrO = reinterpret_cast<S *>(p + T::oTr);
    b.Fs = reinterpret_cast<R *>(sb + T::oFs);
    b.Js = reinterpret_cast<R *>(sb + T::oJs);
    b.Ws = reinterpret_cast<double *>(sb + T::oWs);
    b.Wd = reinterpret_cast<double *>(sb + T::oWd);
    return b;
  };
  uint64_t *bar = reinterpret_cast<uint64_t *>(sb + T::oBar);  // [2][3] ring groups, then U and Acc
  uint64_t *barU = bar + 6, *barA = bar + 7;
  double *volB = reinterpret_cast<double *>(sb + T::oVol);

  const OpTab<R> &op = stage_op<R>(a);
  const int tid = threadIdx.x;
  const int nTiles = (a.nEle + TE - 1) / TE;
  const int flags = a.flags;
  const bool last = flags & SF_LAST, jam = flags & SF_JAMESON;
  const TmaNeeds nd(a);
  if ((int)blockIdx.x >= nTiles) return;

  // thread 0: a tile's ring groups (0: stage input W, JGinv, codes; 1:
  // normals, dA, own traces; 2: 1/detJ) into slot k
  // (part 1: the byte counts and the read-only metric tiles; part 2: the
  // stage input and traces a previous stage writes; 0: both)
  auto issue_slot = [&](const TmaBufs<R, S> &b, int e0, uint64_t *bk, int part) {
    if (part != 2) {
      mbar_expect_tx(&bk[0], (nd.inU ? 0u : (uint32_t)(NV * NS * TE * sizeof(S))) +
                                 (uint32_t)(DIM * DIM * NS * TE * sizeof(S)) + (uint32_t)(NF * TE * 4));
      mbar_expect_tx(&bk[1], (uint32_t)((DIM * NF * TE + NF * TE + NV * NF * TE) * sizeof(S)));
      mbar_expect_tx(&bk[2], (uint32_t)(NS * TE * sizeof(S)));
      tma_load2d(b.JG, &m.JG, e0, 0, &bk[0]);
      tma_load2d(b.Nbr, &m.nbr, e0, 0, &bk[0]);
      tma_load2d(b.Nrm, &m.nrm, e0, 0, &bk[1]);
      tma_load2d(b.DA, &m.dA, e0, 0, &bk[1]);
      tma_load2d(b.Det, &m.det, e0, 0, &bk[2]);
    }
    if (part == 1) return;
    if (!nd.inU) tma_load2d(b.Us, &m.Win, e0, 0, &bk[0]);
    tma_load2d(b.Tw, &m.trIn, e0, 0, &bk[1]);
  };
  // thread 0: the tile's double stage input or U0 (barU), and its RK
  // accumulator (barA), into the block's FP64 buffers
  const bool needUg = nd.inU || nd.needU0;
  auto issue_u = [&](const TmaBufs<R, S> &b, int e0) {
    mbar_expect_tx(barU, (uint32_t)(NV * NS * TE * 8));
    tma_load2d(b.U0, &m.U, e0, 0, barU);
  };
  auto issue_acc = [&](const TmaBufs<R, S> &b, int e0) {
    mbar_expect_tx(barA, (uint32_t)(NV * NS * TE * 8));
    tma_load2d(b.Acc, &m.Acc, e0, 0, barA);
  };

  if (tid == 0) {
    for (int i = 0; i < 8; i++) mbar_init(&bar[i], 1);
    fence_mbar_init();
  }
  __syncthreads();
  pdl_launch_dependents();
  if (tid == 0) issue_slot(slot(0), blockIdx.x * TE, &bar[0], 1);
  pdl_wait();  // the previous stage has finished: its outputs are visible
  stage_dt_reset(a);
  if (tid == 0) {
    issue_slot(slot(0), blockIdx.x * TE, &bar[0], 2);
    if (needUg) issue_u(slot(0), blockIdx.x * TE);
  }
  const double dtG = (a.dtLocal || a.grp) ? 0.0 : __ldg(a.dt);
  double dtMin = INFINITY;
  const bool dtn = flags & SF_DTNEXT;
  int prevE0 = -1;  // the previous tile's first element, for its deferred dt
  bool ok = true;
  // thread 0's counts of issued and completed phases, for the error path
  int uIss = needUg ? 1 : 0, uDone = 0, aIss = 0, aDone = 0, sIss = 1;
  int j = 0;
  for (;; j++) {
    const int t = blockIdx.x + j * gridDim.x;
    if (t >= nTiles) break;
    const int k = j & 1;
    const uint32_t par = (uint32_t)((j >> 1) & 1), parF = (uint32_t)(j & 1);
    const TmaBufs<R, S> b = slot(k);
    uint64_t *bk = &bar[3 * k];
    const int e0 = t * TE;
    if (tid == 0) {
      // the previous tile's state / accumulator stores have been read out
      // before the FP64 buffers and the other slot are reused; its trace
      // store (the most recent group) reads only that slot's trace buffer,
      // next written by the tile after this one, after its own wait
      asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
      if (nd.needAcc) {
        issue_acc(b, e0);
        aIss++;
      }
      if (needUg && last && j > 0) {  // the buffer was a store source: load only now
        issue_u(b, e0);
        uIss++;
      }
    }
    ok = mbar_wait(&bk[0], par);
    if (nd.inU && ok) {
      ok = mbar_wait(barU, parF);
      uDone += ok;
    }
    if (__syncthreads_or(!ok)) break;
    tma_gather<C, S, TE, NT>(a, b.Nbr, b.Js, b.Wd, e0);
    // the tile's element volumes for its ele::calcDt (one slot per tile
    // parity: the dt is formed during the next tile)
    if (dtn && tid < TE && e0 + tid < a.nEle) cp_async_small<8>(&volB[(j & 1) * TE + tid], &a.vol[e0 + tid]);
    tma_phase_a<C, R, S, TE, NT>(a, nd.inU, b, e0);
    // the previous tile's ele::calcDt, by the last warp, which phase A's
    // second round leaves idle; Ws is rewritten only in this tile's phase B
    if (dtn && prevE0 >= 0 && (tid >> 5) == NT / 32 - 1)
      dtMin = fmin(dtMin, tma_tile_dt<NF, TE>(a, b.Ws, prevE0, tid & 31, &volB[((j - 1) & 1) * TE]));
    // the next tile's loads, issued by the last thread, which has one phase-A
    // item where thread 0 has two (thread 0 keeps the counts)
    if (tid == NT - 1) {
      const int tn = t + gridDim.x;
      if (tn < nTiles) issue_slot(slot(k ^ 1), tn * TE, &bar[3 * (k ^ 1)], 0);
    }
    if (tid == 0 && t + gridDim.x < nTiles) sIss++;
    if (dtn) {
      // the next tile's stored wave speeds and dA into L2, so its gathers
      // (at its start) do not wait on DRAM
      const int tn = t + gridDim.x;
      if (tn < nTiles)
        for (int r = tid; r < 2 * NF; r += NT) {
          const double *src = r < NF ? a.waveSp : a.dAd;
          asm volatile("prefetch.global.L2 [%0];" ::"l"(src + (size_t)(r % NF) * a.nE + (size_t)tn * TE));
        }
    }
    if (nd.inU) {
      // first stage: likewise the next tile's double input, whose bulk load
      // is issued only once this tile's phase C has freed the buffer (the
      // later stages gain nothing from it: measured)
      const int tn = t + gridDim.x;
      if (tn < nTiles)
        for (int r = tid; r < NV * NS; r += NT)
          asm volatile("prefetch.global.L2 [%0];" ::"l"(a.Uin_d + (size_t)r * a.ldU + (size_t)tn * TE));
    }
    cp_async_wait_all();
    ok = mbar_wait(&bk[1], par);
    if (__syncthreads_or(!ok)) break;
    tma_phase_b<C, R, S, BC, RS, TE, NT>(a, op, b, e0);
    ok = mbar_wait(&bk[2], par);
    if (nd.needU0 && !nd.inU && ok) {
      ok = mbar_wait(barU, parF);
      uDone += ok;
    }
    if (nd.needAcc && ok) {
      ok = mbar_wait(barA, parF);
      aDone += ok;
    }
    if (__syncthreads_or(!ok)) break;
    tma_phase_c<C, R, S, TE, NT, true>(a, op, b, e0, dtG);
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      if (last) tma_store2d(&m.U, e0, 0, b.U0);
      else {
        tma_store2d(&m.Wout, e0, 0, b.Us);
        if (!jam) tma_store2d(&m.Acc, e0, 0, b.Acc);
      }
      tma_commit();
      // the U0 buffer is no longer read (and, outside the last stage, not a
      // store source): the next tile's double input or U0 can land now
      const int tn = t + gridDim.x;
      if (needUg && !last && tn < nTiles) {
        issue_u(b, tn * TE);
        uIss++;
      }
    }
    tma_phase_d<C, R, S, TE, NT, true>(op, b.Us, b.TrO);
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      tma_store2d(&m.trOut, e0, 0, b.TrO);
      tma_commit();
    }
    prevE0 = e0;
  }
  if (!ok) {
    // a bounded wait gave up: flag it and let every issued load land
    // (bounded again) before the block's shared memory is released
    if (tid == 0) {
      atomicOr(a.err, ERRF_TIMEOUT);
      for (int q = j; q < sIss; q++)
        for (int g = 0; g < 3; g++) mbar_wait(&bar[3 * (q & 1) + g], (uint32_t)((q >> 1) & 1));
      for (int q = uDone; q < uIss; q++) mbar_wait(barU, (uint32_t)(q & 1));
      for (int q = aDone; q < aIss; q++) mbar_wait(barA, (uint32_t)(q & 1));
    }
    cp_async_wait_all();
    __syncthreads();
    if (tid == 0) tma_wait_reads();
    return;
  }
  if ((flags & SF_TIME) && !a.grp && blockIdx.x == 0 && tid == 0) *a.time += dtG;
  if (dtn && (tid >> 5) == NT / 32 - 1) {
    if (prevE0 >= 0)
      dtMin = fmin(dtMin, tma_tile_dt<NF, TE>(a, slot(0).Ws, prevE0, tid & 31, &volB[((j - 1) & 1) * TE]));
    tma_dt_reduce(a, dtMin);
  }
  if (tid == 0) tma_wait_reads();
}

}  // namespace frg
