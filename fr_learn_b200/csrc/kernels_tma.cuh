// kernels_tma.cuh -- the RK stage kernel of the fused update path with its
// tiles moved by the Tensor Memory Accelerator.
//
// The generic stage kernel (kernels.cuh) loads its inputs with per-thread
// loads, so each phase waits on a few loads in flight per thread.  Here one
// thread issues, at block start, every tile the block will need as 2D bulk
// tensor copies (cp.async.bulk.tensor) into shared memory, in three groups
// completing on three mbarriers:
//   group 0  stage state, JGinv, neighbour codes       (phase A, gathers)
//   group 1  face normals, dA                           (phase B)
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

enum : unsigned { ERRF_TIMEOUT = 8u };

// Tensor maps of one stage launch (all 2D: [rows][element stride]).
struct TmaMaps {
  CUtensorMap U;      // double [NV*NS]: stage-0 input, U0, final state
  CUtensorMap Acc;    // double [NV*NS]: RK accumulator
  CUtensorMap Win;    // S [NV*NS]: stage input (stages >= 1)
  CUtensorMap Wout;   // S [NV*NS]: next stage state
  CUtensorMap trOut;  // S [NV*NF]: traces of the new state
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
           NV * NF * (int)sizeof(R) + NF * 8;
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
  static constexpr int oFs = oNbr + al(NF * TE * 4);
  static constexpr int oJs = oFs + al(D * NV * NS * TE * (int)sizeof(R));
  static constexpr int oWs = oJs + al(NV * NF * TE * (int)sizeof(R));
  static constexpr int oBar = oWs + al(NF * TE * 8);
  static constexpr int SMEM = oBar + 64 + 128;  // + room to align the base
};

template <class C, typename R, typename S, bool BC, int RS, int TEV, int NTV>
__global__ void __launch_bounds__(NTV, (TileT<C, R, S, TEV, NTV>::MINB))
    fr_stage_tma_kernel(const StageArgs a, const __grid_constant__ TmaMaps m) {
  static_assert(sizeof(R) == sizeof(S), "stage state is loaded straight into the compute buffer");
  using T = TileT<C, R, S, TEV, NTV>;
  constexpr int TE = T::TE, NT = T::NT, NS = C::NS, NF = C::NF, NV = C::NV, DIM = C::DIM, N1 = C::N1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // bulk-tensor destinations start on 128-byte boundaries
  unsigned char *const sbase = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
#define smem_raw sbase
  double *sU0 = reinterpret_cast<double *>(smem_raw + T::oU0);
  double *sAcc = reinterpret_cast<double *>(smem_raw + T::oAcc);
  R *Us = reinterpret_cast<R *>(smem_raw + T::oUs);
  S *sJG = reinterpret_cast<S *>(smem_raw + T::oJG);
  S *sDet = reinterpret_cast<S *>(smem_raw + T::oDet);
  S *sNrm = reinterpret_cast<S *>(smem_raw + T::oNrm);
  S *sDA = reinterpret_cast<S *>(smem_raw + T::oDA);
  int *sNbr = reinterpret_cast<int *>(smem_raw + T::oNbr);
  R *Fs = reinterpret_cast<R *>(smem_raw + T::oFs);
  R *Js = reinterpret_cast<R *>(smem_raw + T::oJs);
  double *sWs = reinterpret_cast<double *>(smem_raw + T::oWs);
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw + T::oBar);
#undef smem_raw

  const OpTab<R> &op = optab<R>(a.vcjh, C::P);
  const int tid = threadIdx.x, e0 = blockIdx.x * TE, L = a.nE;
  const Phys &ph = a.ph;
  const int flags = a.flags;
  const bool first = flags & SF_FIRST, last = flags & SF_LAST, jam = flags & SF_JAMESON;
  const bool inU = a.Uin_d != nullptr;                      // stage input is the double state U
  const bool needU0 = !inU && (jam || !last);               // U0 for the next stage state
  const bool needAcc = !first && !jam;

  if (tid == 0) {
    for (int i = 0; i < 3; i++) mbar_init(&bar[i], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tid == 0) {
    const uint32_t b0 = (inU ? NV * NS * TE * 8 : NV * NS * TE * (int)sizeof(S)) + DIM * DIM * NS * TE * sizeof(S) +
                        NF * TE * 4;
    mbar_expect_tx(&bar[0], b0);
    if (inU) tma_load2d(sU0, &m.U, e0, 0, &bar[0]);
    else tma_load2d(Us, &m.Win, e0, 0, &bar[0]);
    tma_load2d(sJG, &m.JG, e0, 0, &bar[0]);
    tma_load2d(sNbr, &m.nbr, e0, 0, &bar[0]);
    mbar_expect_tx(&bar[1], (DIM * NF * TE + NF * TE) * sizeof(S));
    tma_load2d(sNrm, &m.nrm, e0, 0, &bar[1]);
    tma_load2d(sDA, &m.dA, e0, 0, &bar[1]);
    const uint32_t b2 = NS * TE * sizeof(S) + (needU0 ? NV * NS * TE * 8 : 0) + (needAcc ? NV * NS * TE * 8 : 0);
    mbar_expect_tx(&bar[2], b2);
    tma_load2d(sDet, &m.det, e0, 0, &bar[2]);
    if (needU0) tma_load2d(sU0, &m.U, e0, 0, &bar[2]);
    if (needAcc) tma_load2d(sAcc, &m.Acc, e0, 0, &bar[2]);
  }

  // the global dt, fetched while the tiles are in flight
  const double dtG = (a.dtLocal || a.grp) ? 0.0 : __ldg(a.dt);

  // ---- group 0: gathers of neighbour traces, then phase A
  bool ok = mbar_wait(&bar[0], 0);
  if (__syncthreads_or(!ok)) goto timeout;
  {
    const S *trIn = static_cast<const S *>(a.trIn);
    for (int it = tid; it < NF * TE; it += NT) {
      const int f = it / TE, e = it - f * TE;
      if (e0 + e >= a.nEle) continue;
      const int code = sNbr[f * TE + e];
      if (code < 0) continue;
      const size_t t = (size_t)(code >> 1);
#pragma unroll
      for (int v = 0; v < NV; v++) cp_async_small<sizeof(S)>(&Js[(v * NF + f) * TE + e], &trIn[(size_t)v * NF * L + t]);
    }
  }
  for (int it = tid; it < NS * TE; it += NT) {
    const int s = it / TE, e = it - s * TE;
    if (e0 + e >= a.nEle) continue;
    R u[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) {
      const int o = (v * NS + s) * TE + e;
      u[v] = inU ? (R)sU0[o] : Us[o];
      if (inU) Us[o] = u[v];
    }
    R F[DIM][NV];
    inviscid_flux<DIM, NV, R>(u, F, ph);
#pragma unroll
    for (int d1 = 0; d1 < DIM; d1++)
#pragma unroll
      for (int v = 0; v < NV; v++) {
        R t = 0;
#pragma unroll
        for (int d2 = 0; d2 < DIM; d2++) t += (R)sJG[((d1 * DIM + d2) * NS + s) * TE + e] * F[d2][v];
        Fs[((d1 * NV + v) * NS + s) * TE + e] = t;
      }
  }
  cp_async_wait_all();
  ok = mbar_wait(&bar[1], 0);
  if (__syncthreads_or(!ok)) goto timeout;

  // ---- phase B: common flux and jumps (neighbour traces already in Js)
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
        t += l * Us[(v * NS + s0 + j * st) * TE + e];
        q += l * Fs[((dir * NV + v) * NS + s0 + j * st) * TE + e];
      }
      own[v] = t;
      dis[v] = side ? q : -q;
    }
    R n[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) n[d] = (R)sNrm[(d * NF + f) * TE + e];
    const R dA = (R)sDA[f * TE + e];
    const int code = sNbr[f * TE + e];
    R oth[NV];
    bool right = false;
    if (code >= 0) {
      right = code & 1;
#pragma unroll
      for (int v = 0; v < NV; v++) oth[v] = Js[(v * NF + f) * TE + e];
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
        if (!bc_ghost<DIM>(-1 - code, ul, nd, ur, ph)) atomicOr(a.err, ERRF_BC);
#pragma unroll
        for (int v = 0; v < NV; v++) oth[v] = (R)ur[v];
      }
    }
    const R *UL = right ? oth : own;
    const R *UR = right ? own : oth;
    R Fn[NV];
    const R ws = inviscid_common<C, R, BC, RS>(UL, UR, n, code, Fn, ph);
    const bool upd = !right && ws >= 0;
    if ((flags & SF_WAVESP) && upd) a.waveSp[(size_t)f * L + eg] = (double)ws;
    if (flags & SF_DTNEXT)  // this flux point's term of ele::calcDt's surface integral
      sWs[f * TE + e] = (upd ? (double)ws : a.waveSp[(size_t)f * L + eg]) * a.wsurf[f % a.nff] * a.dAd[(size_t)f * L + eg];
#pragma unroll
    for (int v = 0; v < NV; v++) {
      const R fo = right ? -Fn[v] * dA : Fn[v] * dA;
      Js[(v * NF + f) * TE + e] = fo - dis[v];
    }
  }
  ok = mbar_wait(&bar[2], 0);
  if (__syncthreads_or(!ok)) goto timeout;

  // ---- phase C: divergence + correction, RK update into the staging tiles.
  // Along coordinate lines: pass C1 takes the xi-derivative of the xi-flux
  // along each row j plus the correction from the row's left/right flux
  // points, for all N1 points of the row at once, into Us (free since phase
  // B); pass C2 adds the eta part along each column i and does the RK
  // update of the column's points.  One item = (line, field, element): the
  // line's N1 values are loaded once and N1 results formed.
  static_assert(DIM == 2, "the TMA stage kernel is two-dimensional");
  for (int it = tid; it < N1 * NV * TE; it += NT) {
    const int e = it % TE, r = it / TE, v = r % NV, j = r / NV;
    if (e0 + e >= a.nEle) continue;
    R F[N1];
#pragma unroll
    for (int q = 0; q < N1; q++) F[q] = Fs[((0 * NV + v) * NS + j * N1 + q) * TE + e];
    const R JL = Js[(v * NF + 3 * N1 + C::P - j) * TE + e], JR = Js[(v * NF + N1 + j) * TE + e];
#pragma unroll
    for (int i = 0; i < N1; i++) {
      R acc = 0;
#pragma unroll
      for (int q = 0; q < N1; q++) acc += op.dlag[i][q] * F[q];
      acc += -op.gL[i] * JL;
      acc += op.gR[i] * JR;
      Us[(v * NS + j * N1 + i) * TE + e] = acc;
    }
  }
  __syncthreads();
  for (int it = tid; it < N1 * NV * TE; it += NT) {
    const int e = it % TE, r = it / TE, v = r % NV, i = r / NV, eg = e0 + e;
    if (eg >= a.nEle) continue;
    const double dtl = a.grp ? a.dt[a.grp[eg]] : a.dtLocal ? a.dt[eg] : dtG;
    R F[N1];
#pragma unroll
    for (int q = 0; q < N1; q++) F[q] = Fs[((1 * NV + v) * NS + q * N1 + i) * TE + e];
    const R JB = Js[(v * NF + i) * TE + e], JT = Js[(v * NF + 2 * N1 + C::P - i) * TE + e];
#pragma unroll
    for (int j = 0; j < N1; j++) {
      const int s = j * N1 + i, o = (v * NS + s) * TE + e;
      R acc = Us[o];
#pragma unroll
      for (int q = 0; q < N1; q++) acc += op.dlag[j][q] * F[q];
      acc += -op.gL[j] * JB;
      acc += op.gR[j] * JT;
      const double idet = (double)sDet[s * TE + e];  // 1 / detJ
      const double div = (double)acc;
      if (flags & SF_DIVF) a.divF[((size_t)v * NS + s) * a.ldU + eg] = div;
      double unew;
      if (jam) {
        unew = sU0[o] - a.aNext * div * idet * dtl;
        if (last) sU0[o] = unew;
      } else {
        const double t = a.bCur * div * idet * dtl;
        const double base = first ? sU0[o] : sAcc[o];
        if (last) {
          unew = base - t;
          sU0[o] = unew;
        } else {
          sAcc[o] = base - t;
          const double u0 = first ? base : sU0[o];
          unew = u0 - a.aNext * div * idet * dtl;
        }
      }
      if (last && (v == 0 || v == NV - 1) && isnan(unew)) atomicOr(a.err, ERRF_NAN);
      Us[o] = (R)(last ? unew : (double)(S)unew);
    }
  }
  if ((flags & SF_TIME) && !a.grp && blockIdx.x == 0 && tid == 0) *a.time += dtG;
  fence_proxy_async();
  __syncthreads();
  if (tid == 0) {
    if (last) tma_store2d(&m.U, e0, 0, sU0);
    else {
      tma_store2d(&m.Wout, e0, 0, Us);
      if (!jam) tma_store2d(&m.Acc, e0, 0, sAcc);
    }
    tma_commit();
  }

  // ---- phase D: traces of the new state, staged in Js; one item per
  // (line, field, element) gives the traces at both ends of the line
  // (rows: left face 3 / right face 1; columns: bottom face 0 / top face 2)
  for (int it = tid; it < 2 * N1 * NV * TE; it += NT) {
    const int e = it % TE, r = it / TE, v = r % NV, ln = r / NV;
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
    reinterpret_cast<S *>(Js)[(v * NF + f0) * TE + e] = (S)t0;
    reinterpret_cast<S *>(Js)[(v * NF + f1) * TE + e] = (S)t1;
  }
  fence_proxy_async();
  __syncthreads();
  if (tid == 0) {
    tma_store2d(&m.trOut, e0, 0, Js);
    tma_commit();
  }
  if (flags & SF_DTNEXT) {
    // ele::calcDt for this block's elements with the wave speeds this stage
    // left (src/ele.cpp:1086-1105; flux points summed in order), then the
    // global minimum by a 64-bit atomicMin on the bit pattern (positive
    // doubles order like their bit patterns) into the next step's dt slot,
    // which the host set to a huge value before the step.
    if (tid < 32) {
      double my = INFINITY;
      const int eg = e0 + tid;
      if (tid < TE && eg < a.nEle) {
        double iw = 0;
#pragma unroll
        for (int f = 0; f < NF; f++) iw += sWs[f * TE + tid];
        const double dte = a.cflFac * a.vol[eg] / iw;
        a.eleDt[eg] = dte;
        my = dte;
        if (a.grp) {  // ensemble mode: each element into its own group's minimum
          if (!(dte > 1e-13)) atomicOr(a.err, ERRF_DT);
          else atomicMin(reinterpret_cast<unsigned long long *>(a.dtNext + a.grp[eg]),
                         (unsigned long long)__double_as_longlong(dte));
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double t = __shfl_xor_sync(0xffffffffu, my, o);
        my = (isnan(t) || t < my) ? t : my;
      }
      if (tid == 0 && !a.grp) {
        if (!(my > 1e-13)) atomicOr(a.err, ERRF_DT);  // also catches NaN
        else atomicMin(reinterpret_cast<unsigned long long *>(a.dtNext), (unsigned long long)__double_as_longlong(my));
      }
    }
  }
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

}  // namespace frg
