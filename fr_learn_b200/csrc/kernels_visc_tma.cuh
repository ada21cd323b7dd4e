// kernels_visc_tma.cuh -- the 3D viscous (LDG) RK stage of the fused update
// path with its tiles moved by the Tensor Memory Accelerator.
//
// A viscous stage needs two launches: the LDG common viscous flux at a face
// combines the viscous fluxes of both elements, and each of those needs its
// element's corrected gradient, which needs the neighbours' traces.
//
//   fr_visc3_grad_tma_kernel   per tile: LDG common solution, corrected
//       gradient, and at every flux point this side's viscous flux projected
//       on the face normal (at boundary faces: the whole viscous part of the
//       boundary flux), stored as one [field][fpt][element] array;
//   fr_visc3_stage_tma_kernel  per tile: the corrected gradient again
//       (recomputed: cheaper than a round trip through HBM), inviscid +
//       viscous flux at the solution points, common inviscid flux and LDG
//       viscous flux from the two sides' projected fluxes, divergence,
//       correction, the RK stage update and the traces of the new state.
//
// One thread issues, at block start, every tile the block reads as bulk
// tensor copies into shared memory (3D / 4D tensor maps with boxes of TE
// elements x all points x all fields), in groups on mbarriers so the later
// groups land while the earlier phases compute; neighbour traces and
// neighbour projected fluxes (a gather) go to shared memory with cp.async.
// The tile's own flux-point traces are loaded too (the previous launch's
// phase D stored them with the same sums), not recomputed.
// Results leave through bulk tensor stores.  The stage input lands in the
// padded point layout of the generic kernels (one empty slot after every xi
// line, Cfg::NSP): its tensor map walks the xi line with a box one point
// wider than the line, and the point outside the tensor is zero-filled.
// Every mbarrier wait is bounded; no multicast.
//
// The per-element arithmetic is the generic kernels' (kernels.cuh), value for
// value, except that the RK update multiplies by a stored 1/detJ.
#pragma once
#include "kernels_tma.cuh"

namespace frg {

// Tensor maps of one 3D viscous launch (see the host's set-up for shapes).
struct ViscMaps {
  CUtensorMap Uin;    // stage input: S 4D {L, N1, NS/N1, NV} box {TE, N1+1, NS/N1, NV},
                      // or (first stage) double 3D {L, NS, NV} box {TE, NS, NV}
  CUtensorMap U;      // double 3D {L, NS, NV}: U0, the final state
  CUtensorMap Acc;    // double 3D {L, NS, NV}: RK accumulator
  CUtensorMap Wout;   // S 3D {L, NS, NV}: next stage state
  CUtensorMap trOut;  // S 3D {L, NF, NV}: traces of the new state
  CUtensorMap trIn;   // S 3D {L, NF, NV}: traces of the stage input (own tile; the previous launch's phase D)
  CUtensorMap JG;     // S 3D {L, NS, DIM*DIM}
  CUtensorMap det;    // S 2D {L, NS}: 1 / detJ
  CUtensorMap nrm;    // S 3D {L, NF, DIM}
  CUtensorMap dA;     // S 2D {L, NF}
  CUtensorMap nbr;    // int32 2D {L, NF}
  CUtensorMap fvn;    // S 3D {L, NF, NV}: projected viscous flux (pass-1 store, pass-2 load)
  CUtensorMap fvn2;   // S 3D {L, NF, NV}: the left side's penalty-term projection (3D LDG penalty)
};

__device__ __forceinline__ void tma_load3d(void *dst, const CUtensorMap *m, int x, int y, int z, uint64_t *b) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(m), "r"(x), "r"(y), "r"(z), "r"(smem_u32(b))
      : "memory");
}
__device__ __forceinline__ void tma_load4d(void *dst, const CUtensorMap *m, int x, int y, int z, int w, uint64_t *b) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(m), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(b))
      : "memory");
}
// L2 prefetch of a tensor tile (no shared memory involved)
__device__ __forceinline__ void tma_prefetch2d(const CUtensorMap *m, int x, int y) {
  asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];" ::"l"(m), "r"(x), "r"(y) : "memory");
}
__device__ __forceinline__ void tma_prefetch3d(const CUtensorMap *m, int x, int y, int z) {
  asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];" ::"l"(m), "r"(x), "r"(y), "r"(z)
               : "memory");
}
__device__ __forceinline__ void tma_prefetch4d(const CUtensorMap *m, int x, int y, int z, int w) {
  asm volatile("cp.async.bulk.prefetch.tensor.4d.L2.global.tile [%0, {%1, %2, %3, %4}];" ::"l"(m), "r"(x), "r"(y),
               "r"(z), "r"(w)
               : "memory");
}
__device__ __forceinline__ void tma_store3d(const CUtensorMap *m, int x, int y, int z, const void *src) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(m),
               "r"(x), "r"(y), "r"(z), "r"(smem_u32(src))
               : "memory");
}

// Neighbour codes come by TMA when a tile row of them (TE int32) is at least
// the 16-byte TMA minimum, else by plain loads.
template <int TE>
constexpr bool nbr_by_tma() { return TE * 4 >= 16; }
template <class C, int TE, int NT>
__device__ __forceinline__ void load_nbr_plain(const StageArgs &a, int *Nbr, int e0) {
  for (int it = threadIdx.x; it < C::NF * TE; it += NT) {
    const int f = it / TE, e = it - f * TE;
    Nbr[it] = a.nbr[(size_t)f * a.nE + e0 + e];
  }
}

// Shared-memory layouts (byte offsets, 128-byte aligned regions).
template <class C, typename R, typename S, int TE_, int NT_>
struct VGradT {
  static constexpr int NS = C::NS, NSP = C::NSP, NF = C::NF, NV = C::NV, D = C::DIM, TE = TE_, NT = NT_;
  static constexpr int al(int b) { return (b + 127) & ~127; }
  static constexpr int mx(int a, int b) { return a > b ? a : b; }
  static constexpr int oUs = 0;                                    // R [NV][NSP][TE]
  static constexpr int odU = oUs + al(NV * NSP * TE * (int)sizeof(R));  // R [D][NV][NSP][TE]; first: double input
  static constexpr int oNtr = odU + al(mx(D * NV * NSP * TE * (int)sizeof(R), NV * NS * TE * 8));  // R [NV][NF][TE]
  static constexpr int oDc = oNtr + al(NV * NF * TE * (int)sizeof(R));  // R [NV][NF][TE], then the output (S)
  static constexpr int oJG = oDc + al(NV * NF * TE * (int)sizeof(R));   // S [D*D][NS][TE]
  static constexpr int oDet = oJG + al(D * D * NS * TE * (int)sizeof(S));
  static constexpr int oNrm = oDet + al(NS * TE * (int)sizeof(S));  // S [D][NF][TE]
  static constexpr int oNbr = oNrm + al(D * NF * TE * (int)sizeof(S));
  static constexpr int oTw = oNbr + al(NF * TE * 4);  // S [NV][NF][TE] own traces of the stage input
  static constexpr int oBar = oTw + al(NV * NF * TE * (int)sizeof(S));
  static constexpr int SMEM = oBar + 2 * 8 + 128;
  // resident blocks per SM the register budget is sized for (meshes with
  // boundary faces carry the ghost-state and wall code: two blocks)
  static constexpr int minb(bool bc) {
    return SMEM * 3 <= 227 * 1024 && (NT <= 128 || !bc) ? 3 : SMEM * 2 <= 227 * 1024 ? 2 : 1;
  }
};

template <class C, typename R, typename S, int TE_, int NT_>
struct VStageT {
  static constexpr int NS = C::NS, NSP = C::NSP, NF = C::NF, NV = C::NV, D = C::DIM, TE = TE_, NT = NT_;
  static constexpr int al(int b) { return (b + 127) & ~127; }
  static constexpr int oUs = 0;                                         // R [NV][NSP][TE]
  static constexpr int oFs = oUs + al(NV * NSP * TE * (int)sizeof(R));  // R [D][NV][NSP][TE]
  static constexpr int oNtr = oFs + al(D * NV * NSP * TE * (int)sizeof(R));  // R [NV][NF][TE]; then new traces (S)
  static constexpr int oDc = oNtr + al(NV * NF * TE * (int)sizeof(R));       // R [NV][NF][TE]; then the jumps
  static constexpr int oJG = oDc + al(NV * NF * TE * (int)sizeof(R));        // S [D*D][NS][TE]; then W (S)
  static constexpr int oDet = oJG + al(D * D * NS * TE * (int)sizeof(S));
  static constexpr int oNrm = oDet + al(NS * TE * (int)sizeof(S));
  static constexpr int oDA = oNrm + al(D * NF * TE * (int)sizeof(S));
  static constexpr int oNbr = oDA + al(NF * TE * (int)sizeof(S));
  static constexpr int oFo = oNbr + al(NF * TE * 4);                   // S [NV][NF][TE] own projected flux
  static constexpr int oFn = oFo + al(NV * NF * TE * (int)sizeof(S));  // R neighbour's projected flux
  static constexpr int oF2 = oFn + al(NV * NF * TE * (int)sizeof(R));  // R left side's penalty projection
  static constexpr int oU0 = oF2 + al(NV * NF * TE * (int)sizeof(R));  // double [NV][NS][TE]
  static constexpr int oAcc = oU0 + al(NV * NS * TE * 8);
  static constexpr int oTw = oAcc + al(NV * NS * TE * 8);  // S [NV][NF][TE] own traces of the stage input
  static constexpr int oNbrB = oTw + al(NV * NF * TE * (int)sizeof(S));  // int [NF][TE]: codes of odd tiles
  static constexpr int oBar = oNbrB + al(NF * TE * 4);
  static constexpr int SMEM = oBar + 4 * 8 + 128;
  static constexpr int MINB = SMEM * 2 <= 227 * 1024 ? 2 : 1;
};

// cp.async gather of one [field][fpt][element] array at the neighbour's flux
// points (by neighbour code) into dst [field][fpt][TE].
template <class C, typename S, int TE, int NT, typename R>
__device__ __forceinline__ void visc_gather(const StageArgs &a, const void *src_, const int *sNbr, R *dst, int e0) {
  static_assert(sizeof(R) == sizeof(S), "gathered straight into the compute type");
  constexpr int NF = C::NF, NV = C::NV;
  const S *src = static_cast<const S *>(src_);
  const size_t fl = (size_t)NF * a.nE;
  for (int it = threadIdx.x; it < NF * TE; it += NT) {
    const int f = it / TE, e = it - f * TE;
    if (e0 + e >= a.nEle) continue;
    const int code = sNbr[f * TE + e];
    if (code < 0) continue;
    const size_t t = (size_t)(code >> 1);
#pragma unroll
    for (int v = 0; v < NV; v++) cp_async_small<sizeof(S)>(&dst[(v * NF + f) * TE + e], &src[v * fl + t]);
  }
}

// The left side's penalty-term projection at every interior flux point
// (3D LDG penalty, src/face.cpp:245): the neighbour's value when this side is
// the right one, this side's own otherwise.
template <class C, typename S, int TE, int NT, typename R>
__device__ __forceinline__ void visc_gather_left(const StageArgs &a, const int *sNbr, R *dst, int e0) {
  constexpr int NF = C::NF, NV = C::NV;
  const S *src = static_cast<const S *>(a.fvn2In);
  const size_t fl = (size_t)NF * a.nE;
  for (int it = threadIdx.x; it < NF * TE; it += NT) {
    const int f = it / TE, e = it - f * TE;
    if (e0 + e >= a.nEle) continue;
    const int code = sNbr[f * TE + e];
    if (code < 0) continue;
    const size_t t = (code & 1) ? (size_t)(code >> 1) : (size_t)f * a.nE + e0 + e;
#pragma unroll
    for (int v = 0; v < NV; v++) cp_async_small<sizeof(S)>(&dst[(v * NF + f) * TE + e], &src[v * fl + t]);
  }
}

// The double stage input (first stage) into the padded compute tile.
template <class C, typename R, int TE, int NT>
__device__ __forceinline__ void visc_convert_input(const double *Ud, R *Us) {
  constexpr int NS = C::NS, NSP = C::NSP, NV = C::NV;
  for (int it = threadIdx.x; it < NS * TE; it += NT) {
    const int s = it / TE, e = it - s * TE;
#pragma unroll
    for (int v = 0; v < NV; v++) Us[(v * NSP + sx<C>(s)) * TE + e] = (R)Ud[(v * NS + s) * TE + e];
  }
}

// Ghost state of a boundary flux point (other_side's boundary branch).
template <class C, typename R, bool BC>
__device__ __forceinline__ void visc_ghost(const StageArgs &a, int code, const R *own, const R *n, R *oth) {
  constexpr int NV = C::NV, DIM = C::DIM;
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

// LDG common solution minus own trace at every flux point (ldg_phase with
// the tile's normals, codes, own traces and neighbour traces in shared
// memory).  The own traces are the ones the previous launch's phase D (or the
// trace kernel) stored: the same sum over the same line in the same order as
// own_trace of the stage input, so the same values.
template <class C, typename R, typename S, bool BC, int TE, int NT>
__device__ __forceinline__ void visc_ldg(const StageArgs &a, const S *Tw, const R *Ntr, const S *Nrm, const int *Nbr,
                                         R *Dc, int e0) {
  constexpr int NF = C::NF, NV = C::NV, DIM = C::DIM;
  for (int it = threadIdx.x; it < NF * TE; it += NT) {
    const int f = it / TE, e = it - f * TE;
    if (e0 + e >= a.nEle) continue;
    R own[NV], oth[NV], n[DIM];
#pragma unroll
    for (int v = 0; v < NV; v++) own[v] = (R)Tw[(v * NF + f) * TE + e];
#pragma unroll
    for (int d = 0; d < DIM; d++) n[d] = (R)Nrm[(d * NF + f) * TE + e];
    const int code = Nbr[f * TE + e];
    bool right = false;
    if (code >= 0) {
      right = code & 1;
#pragma unroll
      for (int v = 0; v < NV; v++) oth[v] = Ntr[(v * NF + f) * TE + e];
    } else {
      visc_ghost<C, R, BC>(a, code, own, n, oth);
    }
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

// Corrected physical gradient [DIM][NV] at solution point s of tile element e
// (gradient_phase, value for value): D U plus the correction by the common
// solution, then JGinv^T / detJ.
template <class C, typename R, typename S, int TE>
__device__ __forceinline__ void visc_point_gradient(const OpTab<R> &op, const R *Us, const R *Dc, const S *JG,
                                                    const S *Det, int s, int e, R *gout) {
  constexpr int NS = C::NS, NSP = C::NSP, NF = C::NF, NV = C::NV, DIM = C::DIM, N1 = C::N1;
  const int i = s % N1, j = (s / N1) % N1, k = s / (N1 * N1);
  const int ijk[3] = {i, j, k};
  int cf[2 * DIM], cs[2 * DIM], ca[2 * DIM];
  corr_fpts<C>(i, j, k, cf, cs, ca);
  R G[DIM][DIM];
#pragma unroll
  for (int d1 = 0; d1 < DIM; d1++)
#pragma unroll
    for (int d2 = 0; d2 < DIM; d2++) G[d1][d2] = (R)JG[((d1 * DIM + d2) * NS + s) * TE + e];
  const R invDet = (R)Det[s * TE + e];
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
      gout[d1 * NV + v] = invDet * t;
    }
  }
}

// ----------------------------------------------------------------------------
// Pass 1: projected viscous flux of every flux point of the tile.
// ----------------------------------------------------------------------------
template <class C, typename R, typename S, bool BC, int TE, int NT>
__global__ void __launch_bounds__(NT, (VGradT<C, R, S, TE, NT>::minb(BC)))
    fr_visc3_grad_tma_kernel(const StageArgs a, const __grid_constant__ ViscMaps m) {
  static_assert(C::DIM == 3 && sizeof(R) == sizeof(S), "3D, compute type = stored type");
  using T = VGradT<C, R, S, TE, NT>;
  constexpr int NS = C::NS, NSP = C::NSP, NF = C::NF, NV = C::NV, DIM = C::DIM;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char *const sb = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  R *Us = reinterpret_cast<R *>(sb + T::oUs);
  R *dU = reinterpret_cast<R *>(sb + T::odU);
  double *Stg = reinterpret_cast<double *>(sb + T::odU);
  R *Ntr = reinterpret_cast<R *>(sb + T::oNtr);
  R *Dc = reinterpret_cast<R *>(sb + T::oDc);
  S *JG = reinterpret_cast<S *>(sb + T::oJG);
  S *Det = reinterpret_cast<S *>(sb + T::oDet);
  S *Nrm = reinterpret_cast<S *>(sb + T::oNrm);
  int *Nbr = reinterpret_cast<int *>(sb + T::oNbr);
  S *Tw = reinterpret_cast<S *>(sb + T::oTw);
  uint64_t *bar = reinterpret_cast<uint64_t *>(sb + T::oBar);
  S *FvO = reinterpret_cast<S *>(Dc);   // output after the gradient has read Dc
  S *Fv2 = reinterpret_cast<S *>(Ntr);  // penalty projection after the LDG phase has read Ntr
  const OpTab<R> &op = stage_op<R>(a);
  const int tid = threadIdx.x, nTiles = (a.nEle + TE - 1) / TE;
  const bool inU = a.Uin_d != nullptr;
  bool ok = true;
  uint32_t par = 0;

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  // persistent: the block walks tiles blockIdx.x, + gridDim.x, ...; each
  // tile's inputs are prefetched into L2 one tile ahead
  for (int t = blockIdx.x, j = 0; t < nTiles; t += gridDim.x, j++) {
  const int e0 = t * TE;
  par = (uint32_t)(j & 1);
  if (tid == 0) {
    tma_wait_reads();  // the previous tile's stores have read shared memory
    const uint32_t bst = inU ? (uint32_t)(NV * NS * TE * 8) : (uint32_t)(NV * NSP * TE * sizeof(S));
    mbar_expect_tx(&bar[0], bst + (uint32_t)((nbr_by_tma<TE>() ? NF * TE * 4 : 0) +
                                             (DIM * NF * TE + NV * NF * TE) * sizeof(S)));
    if (inU) tma_load3d(Stg, &m.Uin, e0, 0, 0, &bar[0]);
    else tma_load4d(Us, &m.Uin, e0, 0, 0, 0, &bar[0]);
    if constexpr (nbr_by_tma<TE>()) tma_load2d(Nbr, &m.nbr, e0, 0, &bar[0]);
    tma_load3d(Nrm, &m.nrm, e0, 0, 0, &bar[0]);
    tma_load3d(Tw, &m.trIn, e0, 0, 0, &bar[0]);
    mbar_expect_tx(&bar[1], (uint32_t)((DIM * DIM * NS * TE + NS * TE) * sizeof(S)));
    tma_load3d(JG, &m.JG, e0, 0, 0, &bar[1]);
    tma_load2d(Det, &m.det, e0, 0, &bar[1]);
    const int tn = t + gridDim.x;
    if (tn < nTiles) {
      const int en = tn * TE;
      if (inU) tma_prefetch3d(&m.Uin, en, 0, 0);
      else tma_prefetch4d(&m.Uin, en, 0, 0, 0);
      if constexpr (nbr_by_tma<TE>()) tma_prefetch2d(&m.nbr, en, 0);
      tma_prefetch3d(&m.nrm, en, 0, 0);
      tma_prefetch3d(&m.trIn, en, 0, 0);
      tma_prefetch3d(&m.JG, en, 0, 0);
      tma_prefetch2d(&m.det, en, 0);
    }
  }
  if constexpr (!nbr_by_tma<TE>()) load_nbr_plain<C, TE, NT>(a, Nbr, e0);
  ok = mbar_wait(&bar[0], par);
  if (__syncthreads_or(!ok)) goto timeout;
  visc_gather<C, S, TE, NT>(a, a.trIn, Nbr, Ntr, e0);
  if (inU) visc_convert_input<C, R, TE, NT>(Stg, Us);
  cp_async_wait_all();
  __syncthreads();
  visc_ldg<C, R, S, BC, TE, NT>(a, Tw, Ntr, Nrm, Nbr, Dc, e0);
  ok = mbar_wait(&bar[1], par);
  if (__syncthreads_or(!ok)) goto timeout;
  // corrected gradient at the solution points (calcGradU_spts, correctGradU)
  for (int it = tid; it < NS * TE; it += NT) {
    const int s = it / TE, e = it - s * TE;
    if (e0 + e >= a.nEle) continue;
    R g[DIM * NV];
    visc_point_gradient<C, R, S, TE>(op, Us, Dc, JG, Det, s, e, g);
#pragma unroll
    for (int q = 0; q < DIM * NV; q++) dU[(q * NSP + sx<C>(s)) * TE + e] = g[q];
  }
  __syncthreads();
  // this side's viscous flux at every flux point, projected on the normal;
  // at a boundary face the whole viscous part of the boundary flux
  for (int it = tid; it < NF * TE; it += NT) {
    const int f = it / TE, e = it - f * TE;
    if (e0 + e >= a.nEle) continue;
    R u[NV], g[DIM * NV], n[DIM], Fv[DIM][NV];
#pragma unroll
    for (int v = 0; v < NV; v++) u[v] = (R)Tw[(v * NF + f) * TE + e];
    own_grad_trace<C, R, TE>(op, dU, f, e, g);
#pragma unroll
    for (int d = 0; d < DIM; d++) n[d] = (R)Nrm[(d * NF + f) * TE + e];
    visc_flux<C, R>(u, g, Fv, a.ph);
    const int code = Nbr[f * TE + e];
    if (code >= 0) {
#pragma unroll
      for (int v = 0; v < NV; v++) {
        R fn = 0;
#pragma unroll
        for (int d = 0; d < DIM; d++) fn += Fv[d][v] * n[d];
        FvO[(v * NF + f) * TE + e] = (S)fn;
        // the LDG penalty term of the reference reads FL[1] where FL[2] is
        // meant (src/face.cpp:245): the left side contributes n0 F0 + n1 F1 + n2 F1
        if (a.visc2) Fv2[(v * NF + f) * TE + e] = (S)(n[0] * Fv[0][v] + n[1] * Fv[1][v] + n[2] * Fv[1][v]);
      }
    } else if constexpr (NV == 1) {
      R bs = 0;  // centralFlux with a zero ghost gradient
#pragma unroll
      for (int d = 0; d < DIM; d++) bs += (R)0.5 * Fv[d][0] * n[d];
      FvO[f * TE + e] = (S)bs;
    } else if constexpr (BC) {
      R UR[NV], Fb[DIM][NV];
      visc_ghost<C, R, BC>(a, code, u, n, UR);
      if (-1 - code == BC_ADI_NOSLIP) {
        R gR[DIM * NV];
        adiabatic_gradient<DIM, R>(u, UR, g, gR, a.ph);
        visc_flux<C, R>(UR, gR, Fb, a.ph);
      } else {
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int v = 0; v < NV; v++) Fb[d][v] = Fv[d][v];
      }
#pragma unroll
      for (int v = 0; v < NV; v++) {
        R bn = 0;
#pragma unroll
        for (int d = 0; d < DIM; d++) bn += Fb[d][v] * n[d];
        FvO[(v * NF + f) * TE + e] = (S)bn;
      }
    }
  }
  fence_proxy_async();
  __syncthreads();
  if (tid == 0) {
    tma_store3d(&m.fvn, e0, 0, 0, FvO);
    if (a.visc2) tma_store3d(&m.fvn2, e0, 0, 0, Fv2);
    tma_commit();
  }
  }  // tiles
  if (tid == 0) tma_wait_reads();
  return;

timeout:
  if (tid == 0) {
    atomicOr(a.err, ERRF_TIMEOUT);
    for (int i = 0; i < 2; i++) mbar_wait(&bar[i], par);  // bounded: let copies in flight land
    tma_wait_reads();
  }
  cp_async_wait_all();
  __syncthreads();
}

// ----------------------------------------------------------------------------
// Pass 2: the RK stage.
// ----------------------------------------------------------------------------
template <class C, typename R, typename S, bool BC, int RS, int TE, int NT>
__global__ void __launch_bounds__(NT, (VStageT<C, R, S, TE, NT>::MINB))
    fr_visc3_stage_tma_kernel(const StageArgs a, const __grid_constant__ ViscMaps m) {
  static_assert(C::DIM == 3 && sizeof(R) == sizeof(S), "3D, compute type = stored type");
  using T = VStageT<C, R, S, TE, NT>;
  constexpr int NS = C::NS, NSP = C::NSP, NF = C::NF, NV = C::NV, DIM = C::DIM, N1 = C::N1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char *const sb = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  R *Us = reinterpret_cast<R *>(sb + T::oUs);
  R *Fs = reinterpret_cast<R *>(sb + T::oFs);
  R *Ntr = reinterpret_cast<R *>(sb + T::oNtr);
  R *Dc = reinterpret_cast<R *>(sb + T::oDc);
  S *JG = reinterpret_cast<S *>(sb + T::oJG);
  S *Det = reinterpret_cast<S *>(sb + T::oDet);
  S *Nrm = reinterpret_cast<S *>(sb + T::oNrm);
  S *DA = reinterpret_cast<S *>(sb + T::oDA);
  S *Fo = reinterpret_cast<S *>(sb + T::oFo);
  R *Fn = reinterpret_cast<R *>(sb + T::oFn);
  R *F2 = reinterpret_cast<R *>(sb + T::oF2);
  double *U0 = reinterpret_cast<double *>(sb + T::oU0);
  double *Acc = reinterpret_cast<double *>(sb + T::oAcc);
  S *Tw = reinterpret_cast<S *>(sb + T::oTw);
  int *const NbrE = reinterpret_cast<int *>(sb + T::oNbr), *const NbrO = reinterpret_cast<int *>(sb + T::oNbrB);
  uint64_t *bar = reinterpret_cast<uint64_t *>(sb + T::oBar);  // [3]: the next tile's codes
  R *Js = Dc;                             // jumps, after the gradient has read Dc
  S *Wst = reinterpret_cast<S *>(JG);     // new stage state, after the fluxes have read JG
  S *TrO = reinterpret_cast<S *>(Dc);     // new traces, after phase C has read the jumps
  const OpTab<R> &op = stage_op<R>(a);
  const int tid = threadIdx.x, flags = a.flags, nTiles = (a.nEle + TE - 1) / TE;
  const bool last = flags & SF_LAST, first = flags & SF_FIRST, jam = flags & SF_JAMESON;
  const TmaNeeds nd(a);
  const Phys &ph = a.ph;
  bool ok = true;
  uint32_t par = 0;
  int nbrLast = -1;  // thread 0: the tile during which the last next-tile codes load was issued

  if (tid == 0) {
    for (int i = 0; i < 4; i++) mbar_init(&bar[i], 1);
    fence_mbar_init();
  }
  __syncthreads();
  const double dtG = (a.dtLocal || a.grp) ? 0.0 : __ldg(a.dt);
  // persistent: the block walks tiles blockIdx.x, + gridDim.x, ...; each
  // tile's inputs are prefetched into L2 one tile ahead, and its neighbour
  // gathers are issued during the tile before (once that tile's phase B has
  // read its own), with the codes in two buffers by tile parity
  for (int t = blockIdx.x, j = 0; t < nTiles; t += gridDim.x, j++) {
  const int e0 = t * TE;
  int *const Nbr = (j & 1) ? NbrO : NbrE;  // this tile's codes
  par = (uint32_t)(j & 1);
  if (tid == 0) {
    tma_wait_reads();  // the previous tile's stores have read shared memory
    const uint32_t bst = nd.inU ? (uint32_t)(NV * NS * TE * 8) : (uint32_t)(NV * NSP * TE * sizeof(S));
    mbar_expect_tx(&bar[0], bst + (uint32_t)(nbr_by_tma<TE>() && j == 0 ? NF * TE * 4 : 0) +
                                (uint32_t)((DIM * NF * TE + DIM * DIM * NS * TE + NS * TE + NV * NF * TE) * sizeof(S)));
    if (nd.inU) tma_load3d(U0, &m.Uin, e0, 0, 0, &bar[0]);
    else tma_load4d(Us, &m.Uin, e0, 0, 0, 0, &bar[0]);
    if constexpr (nbr_by_tma<TE>()) {
      if (j == 0) tma_load2d(Nbr, &m.nbr, e0, 0, &bar[0]);
      // the next tile's codes, for its gathers issued after this tile's phase B
      const int tn = t + gridDim.x;
      if (tn < nTiles) {
        mbar_expect_tx(&bar[3], (uint32_t)(NF * TE * 4));
        tma_load2d((j & 1) ? NbrE : NbrO, &m.nbr, tn * TE, 0, &bar[3]);
        nbrLast = j;
      }
    }
    tma_load3d(Nrm, &m.nrm, e0, 0, 0, &bar[0]);
    tma_load3d(Tw, &m.trIn, e0, 0, 0, &bar[0]);
    tma_load3d(JG, &m.JG, e0, 0, 0, &bar[0]);
    tma_load2d(Det, &m.det, e0, 0, &bar[0]);
    mbar_expect_tx(&bar[1], (uint32_t)((NF * TE + NV * NF * TE) * sizeof(S)));
    tma_load2d(DA, &m.dA, e0, 0, &bar[1]);
    tma_load3d(Fo, &m.fvn, e0, 0, 0, &bar[1]);
    mbar_expect_tx(&bar[2], (uint32_t)((nd.needU0 ? NV * NS * TE * 8 : 0) + (nd.needAcc ? NV * NS * TE * 8 : 0)));
    if (nd.needU0) tma_load3d(U0, &m.U, e0, 0, 0, &bar[2]);
    if (nd.needAcc) tma_load3d(Acc, &m.Acc, e0, 0, 0, &bar[2]);
    const int tn = t + gridDim.x;
    if (tn < nTiles) {
      const int en = tn * TE;
      if (nd.inU) tma_prefetch3d(&m.Uin, en, 0, 0);
      else tma_prefetch4d(&m.Uin, en, 0, 0, 0);
      if constexpr (nbr_by_tma<TE>()) tma_prefetch2d(&m.nbr, en, 0);
      tma_prefetch3d(&m.nrm, en, 0, 0);
      tma_prefetch3d(&m.trIn, en, 0, 0);
      tma_prefetch3d(&m.JG, en, 0, 0);
      tma_prefetch2d(&m.det, en, 0);
      tma_prefetch2d(&m.dA, en, 0);
      tma_prefetch3d(&m.fvn, en, 0, 0);
      if (nd.needU0) tma_prefetch3d(&m.U, en, 0, 0);
      if (nd.needAcc) tma_prefetch3d(&m.Acc, en, 0, 0);
    }
  }
  if constexpr (!nbr_by_tma<TE>())
    if (j == 0) load_nbr_plain<C, TE, NT>(a, Nbr, e0);

  ok = mbar_wait(&bar[0], par);
  if (__syncthreads_or(!ok)) goto timeout;
  if (j == 0) {  // later tiles' gathers were issued during the tile before
    visc_gather<C, S, TE, NT>(a, a.trIn, Nbr, Ntr, e0);
    visc_gather<C, S, TE, NT>(a, a.fvnIn, Nbr, Fn, e0);
    if (a.visc2) visc_gather_left<C, S, TE, NT>(a, Nbr, F2, e0);
  }
  if (nd.inU) visc_convert_input<C, R, TE, NT>(U0, Us);
  cp_async_wait_all();
  __syncthreads();
  visc_ldg<C, R, S, BC, TE, NT>(a, Tw, Ntr, Nrm, Nbr, Dc, e0);
  __syncthreads();

  // ---- A: gradient, inviscid + viscous flux at the solution points,
  // transformed (calcInviscidFlux_spts + calcViscousFlux_spts)
  for (int it = tid; it < NS * TE; it += NT) {
    const int s = it / TE, e = it - s * TE;
    if (e0 + e >= a.nEle) continue;
    R g[DIM * NV], u[NV];
    visc_point_gradient<C, R, S, TE>(op, Us, Dc, JG, Det, s, e, g);
#pragma unroll
    for (int v = 0; v < NV; v++) u[v] = Us[(v * NSP + sx<C>(s)) * TE + e];
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
      for (int d2 = 0; d2 < DIM; d2++) G[d1][d2] = (R)JG[((d1 * DIM + d2) * NS + s) * TE + e];
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
  ok = mbar_wait(&bar[1], par);
  if (__syncthreads_or(!ok)) goto timeout;

  // ---- B: common inviscid + LDG viscous flux and the jumps
  for (int it = tid; it < NF * TE; it += NT) {
    const int f = it / TE, e = it - f * TE, eg = e0 + e;
    if (eg >= a.nEle) continue;
    int dir, side, s0, st;
    fpt_line<C>(f, dir, side, s0, st);
    R own[NV], dis[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) {
      R q = 0;
#pragma unroll
      for (int j = 0; j < N1; j++) q += op.lag[side][j] * Fs[((dir * NV + v) * NSP + sx<C>(s0 + j * st)) * TE + e];
      own[v] = (R)Tw[(v * NF + f) * TE + e];
      dis[v] = side ? q : -q;
    }
    R n[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) n[d] = (R)Nrm[(d * NF + f) * TE + e];
    const R dA = (R)DA[f * TE + e];
    const int code = Nbr[f * TE + e];
    R oth[NV];
    bool right = false;
    if (code >= 0) {
      right = code & 1;
#pragma unroll
      for (int v = 0; v < NV; v++) oth[v] = Ntr[(v * NF + f) * TE + e];
    } else {
      visc_ghost<C, R, BC>(a, code, own, n, oth);
    }
    const R *UL = right ? oth : own;
    const R *UR = right ? own : oth;
    R Fc[NV];
    const R ws = inviscid_common<C, R, BC, RS>(UL, UR, n, code, Fc, ph);
    if ((flags & SF_WAVESP) && !right && ws >= 0) a.waveSp[(size_t)f * a.nE + eg] = (double)ws;
    R nn = 0;
#pragma unroll
    for (int d = 0; d < DIM; d++) nn += n[d] * n[d];
    const R tau = (R)ph.tau;
    if (code >= 0) {
      const R pf = ldg_pen<DIM, R>(n, ph.penFact);
#pragma unroll
      for (int v = 0; v < NV; v++) {
        const R on = (R)Fo[(v * NF + f) * TE + e];
        const R xn = Fn[(v * NF + f) * TE + e];
        const R FLn = right ? xn : on, FRn = right ? on : xn;
        if constexpr (NV == 1) {
          Fc[v] += (R)0.5 * (FLn + FRn);  // centralFlux (src/flux.cpp:379-387)
        } else {
          // 3D: the left side's n0 F0 + n1 F1 + n2 F1 (src/face.cpp:245); it
          // only enters multiplied by the penalty factor, so without one any
          // finite value gives the same sum
          const R al = a.visc2 ? F2[(v * NF + f) * TE + e] : (right ? xn : on);
          const R jumpF = al - FRn;
          Fc[v] += (R)0.5 * (FLn + FRn) + pf * nn * jumpF + tau * nn * (UL[v] - UR[v]);
        }
      }
    } else {
      // boundary: the viscous part pass 1 formed from this side's gradient
      // trace (and the ghost gradient of an adiabatic wall)
      if constexpr (NV == 1) {
        Fc[0] += (R)Fo[f * TE + e];
      } else if constexpr (BC) {
#pragma unroll
        for (int v = 0; v < NV; v++) Fc[v] += (R)Fo[(v * NF + f) * TE + e] + tau * nn * (UL[v] - UR[v]);
      }
    }
#pragma unroll
    for (int v = 0; v < NV; v++) {
      const R fo = right ? -Fc[v] * dA : Fc[v] * dA;
      Js[(v * NF + f) * TE + e] = fo - dis[v];
    }
  }
  ok = mbar_wait(&bar[2], par);
  if (__syncthreads_or(!ok)) goto timeout;
  // phase B has read the neighbour buffers: the next tile's gathers land in
  // them while phases C and D run (each thread issues the items whose codes
  // it loaded itself when they come by plain loads; a failed wait skips
  // them and is caught at the next barrier)
  {
    const int tn = t + gridDim.x;
    if (tn < nTiles) {
      const int en = tn * TE;
      int *const Nn = (j & 1) ? NbrE : NbrO;
      bool okN = true;
      if constexpr (nbr_by_tma<TE>()) okN = mbar_wait(&bar[3], (uint32_t)(j & 1));
      else load_nbr_plain<C, TE, NT>(a, Nn, en);
      if (okN) {
        visc_gather<C, S, TE, NT>(a, a.trIn, Nn, Ntr, en);
        visc_gather<C, S, TE, NT>(a, a.fvnIn, Nn, Fn, en);
        if (a.visc2) visc_gather_left<C, S, TE, NT>(a, Nn, F2, en);
      }
      ok = okN;
    }
  }

  // ---- C: divergence + correction, the RK update (timeStepA/B) in FP64
  for (int it = tid; it < NS * TE; it += NT) {
    const int s = it / TE, e = it - s * TE, eg = e0 + e;
    if (eg >= a.nEle) continue;
    const int i = s % N1, j = (s / N1) % N1, k = s / (N1 * N1);
    const int ijk[3] = {i, j, k};
    int cf[2 * DIM], cs[2 * DIM], ca[2 * DIM];
    corr_fpts<C>(i, j, k, cf, cs, ca);
    const R idet = (R)Det[s * TE + e];  // 1 / detJ
    const double dtl = a.grp ? a.dt[a.grp[eg]] : a.dtLocal ? a.dt[eg] : dtG;
    const double kb = a.bCur * dtl, ka = a.aNext * dtl;
#pragma unroll
    for (int v = 0; v < NV; v++) {
      R acc = 0;
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        const int sd = d == 0 ? 1 : d == 1 ? N1 : N1 * N1;
        const int sbase = s - ijk[d] * sd;
#pragma unroll
        for (int q = 0; q < N1; q++)
          acc += op.dlag[ijk[d]][q] * Fs[((d * NV + v) * NSP + sx<C>(sbase + q * sd)) * TE + e];
      }
#pragma unroll
      for (int c = 0; c < 2 * DIM; c++) {
        const R gcf = cs[c] ? op.gR[ca[c]] : -op.gL[ca[c]];
        acc += gcf * Js[(v * NF + cf[c]) * TE + e];
      }
      const int o = (v * NS + s) * TE + e;
      if (flags & SF_DIVF) a.divF[((size_t)v * NS + s) * a.ldU + eg] = (double)acc;
      // divF / detJ in the arithmetic type, the stage coefficient x dt in FP64
      const double dj = (double)(acc * idet);
      double unew;
      if (jam) {
        unew = U0[o] - ka * dj;
        if (last) U0[o] = unew;
        else Wst[o] = (S)unew;
      } else {
        const double t = kb * dj;
        const double base = first ? U0[o] : Acc[o];
        if (last) {
          unew = base - t;
          U0[o] = unew;
        } else {
          Acc[o] = base - t;
          const double u0 = first ? base : U0[o];
          unew = u0 - ka * dj;
          Wst[o] = (S)unew;
        }
      }
      if (last && (v == 0 || v == NV - 1) && isnan(unew)) atomicOr(a.err, ERRF_NAN);
      Us[(v * NSP + sx<C>(s)) * TE + e] = (R)(last ? unew : (double)(S)unew);
    }
  }
  fence_proxy_async();
  if (__syncthreads_or(!ok)) goto timeout;
  if (tid == 0) {
    if (last) tma_store3d(&m.U, e0, 0, 0, U0);
    else {
      tma_store3d(&m.Wout, e0, 0, 0, Wst);
      if (!jam) tma_store3d(&m.Acc, e0, 0, 0, Acc);
    }
    tma_commit();
  }

  // ---- D: traces of the new state
  for (int it = tid; it < NF * TE; it += NT) {
    const int f = it / TE, e = it - f * TE;
    if (e0 + e >= a.nEle) continue;
    R t[NV];
    own_trace<C, R, TE>(op, Us, f, e, t);
#pragma unroll
    for (int v = 0; v < NV; v++) TrO[(v * NF + f) * TE + e] = (S)t[v];
  }
  fence_proxy_async();
  __syncthreads();
  if (tid == 0) {
    tma_store3d(&m.trOut, e0, 0, 0, TrO);
    tma_commit();
  }
  }  // tiles
  if ((flags & SF_TIME) && !a.grp && blockIdx.x == 0 && tid == 0) *a.time += dtG;
  if (tid == 0) tma_wait_reads();
  return;

timeout:
  if (tid == 0) {
    atomicOr(a.err, ERRF_TIMEOUT);
    for (int i = 0; i < 3; i++) mbar_wait(&bar[i], par);  // bounded: let copies in flight land
    if (nbrLast >= 0) mbar_wait(&bar[3], (uint32_t)(nbrLast & 1));
    tma_wait_reads();
  }
  cp_async_wait_all();
  __syncthreads();
}

}  // namespace frg
