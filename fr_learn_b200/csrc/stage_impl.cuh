// stage_impl.cuh -- launchers and the instantiation switch shared by the
// per-configuration translation units.  Include once per unit after defining
// FRG_UNIT_DIM (2 or 3), FRG_UNIT_R / FRG_UNIT_S (arithmetic / stored type)
// and FRG_UNIT_NAME (suffix of the exported functions).
#pragma once
#include "dispatch.h"
#include "kernels.cuh"
#include "kernels_tma.cuh"
#include "kernels_visc_tma.cuh"
#include "optab_upload.cuh"

namespace frg {
namespace {

template <class C, typename R, typename S, bool BC, int RS>
void launch_stage(const void *args, int nBlk, size_t smem, cudaStream_t st) {
  fr_stage_kernel<C, R, S, BC, RS><<<nBlk, C::NT, smem, st>>>(*static_cast<const StageArgs *>(args));
}
// A TMA stage kernel's launch; with SF_PDL it is a programmatic dependent of
// the previous kernel in the stream (its blocks may start while that kernel's
// last blocks run, see pdl_wait).
template <class K>
void launch_tma_stage(K kernel, const void *args, const void *maps, int nBlk, int nt, size_t smem, cudaStream_t st) {
  const StageArgs &a = *static_cast<const StageArgs *>(args);
  const TmaMaps &m = *static_cast<const TmaMaps *>(maps);
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(nBlk);
  cfg.blockDim = dim3(nt);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = (a.flags & SF_PDL) ? 1 : 0;
  cudaLaunchKernelEx(&cfg, kernel, a, m);
}
template <class C, typename R, typename S, bool BC, int RS, int TEV, int NTV>
void launch_stage_tma(const void *args, const void *maps, int nBlk, size_t smem, cudaStream_t st) {
  launch_tma_stage(fr_stage_tma_kernel<C, R, S, BC, RS, TEV, NTV>, args, maps, nBlk, NTV, smem, st);
}
template <class C, typename R, typename S, bool BC, int RS, int TEV, int NTV>
cudaError_t add_tma_variant(KernelSet &k) {
  using TT = TileT<C, R, S, TEV, NTV>;
  if (k.nTma >= KernelSet::kMaxTma) return cudaErrorInvalidValue;  // the variant table is full
  KernelSet::TmaVariant &v = k.tma[k.nTma++];
  v.launch = &launch_stage_tma<C, R, S, BC, RS, TEV, NTV>;
  v.TE = TT::TE;
  v.NT = NTV;
  v.smem = TT::SMEM;
  auto ft = fr_stage_tma_kernel<C, R, S, BC, RS, TEV, NTV>;
  cudaError_t e = cudaFuncSetAttribute(ft, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TT::SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ft, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  return e;
}
template <class C, typename R, typename S, bool BC, int RS, int TEV, int NTV, int NB>
void launch_stage_pipe(const void *args, const void *maps, int nBlk, size_t smem, cudaStream_t st) {
  launch_tma_stage(fr_stage_tma_pipe_kernel<C, R, S, BC, RS, TEV, NTV, NB>, args, maps, nBlk, NTV, smem, st);
}
template <class C, typename R, typename S, bool BC, int RS, int TEV, int NTV, int NB>
cudaError_t add_pipe_variant(KernelSet &k) {
  using TT = PipeT<C, R, S, TEV, NTV, NB>;
  if (k.nTma >= KernelSet::kMaxTma) return cudaErrorInvalidValue;  // the variant table is full
  KernelSet::TmaVariant &v = k.tma[k.nTma++];
  v.launch = &launch_stage_pipe<C, R, S, BC, RS, TEV, NTV, NB>;
  v.TE = TT::TE;
  v.NT = NTV;
  v.smem = TT::SMEM;
  v.persistent = 1;
  auto ft = fr_stage_tma_pipe_kernel<C, R, S, BC, RS, TEV, NTV, NB>;
  cudaError_t e = cudaFuncSetAttribute(ft, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TT::SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ft, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v.occ, ft, NTV, TT::SMEM);
  if (e == cudaSuccess && v.occ < 1) e = cudaErrorInvalidConfiguration;
  return e;
}
template <class C, typename R, typename S, bool BC, int RS, int TEV, int NTV>
void launch_stage_split(const void *args, const void *maps, int nBlk, size_t smem, cudaStream_t st) {
  launch_tma_stage(fr_stage_tma_split_kernel<C, R, S, BC, RS, TEV, NTV>, args, maps, nBlk, NTV, smem, st);
}
template <class C, typename R, typename S, bool BC, int RS, int TEV, int NTV>
cudaError_t add_split_variant(KernelSet &k) {
  using TT = SplitT<C, R, S, TEV, NTV>;
  if (k.nTma >= KernelSet::kMaxTma) return cudaErrorInvalidValue;  // the variant table is full
  KernelSet::TmaVariant &v = k.tma[k.nTma++];
  v.launch = &launch_stage_split<C, R, S, BC, RS, TEV, NTV>;
  v.TE = TT::TE;
  v.NT = NTV;
  v.smem = TT::SMEM;
  v.persistent = 1;
  auto ft = fr_stage_tma_split_kernel<C, R, S, BC, RS, TEV, NTV>;
  cudaError_t e = cudaFuncSetAttribute(ft, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TT::SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ft, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v.occ, ft, NTV, TT::SMEM);
  if (e == cudaSuccess && v.occ < 1) e = cudaErrorInvalidConfiguration;
  return e;
}
template <class C, typename R, typename S, bool BC, int RS>
void launch_stage_visc(const void *args, int nBlk, size_t smem, cudaStream_t st) {
  fr_stage_visc_kernel<C, R, S, BC, RS><<<nBlk, C::NT, smem, st>>>(*static_cast<const StageArgs *>(args));
}
template <class C, typename R, typename S, bool BC>
void launch_grad(const void *args, int nBlk, size_t smem, cudaStream_t st) {
  fr_visc_grad_kernel<C, R, S, BC><<<nBlk, C::NT, smem, st>>>(*static_cast<const StageArgs *>(args));
}
template <class C, typename R, typename S>
void launch_trace(const double *U, void *tr, int nE, int nEle, int ldU, int vcjh, cudaStream_t st) {
  long n = (long)C::NF * nE;
  fr_trace_kernel<C, R, S><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(U, static_cast<S *>(tr), nE, nEle, ldU,
                                                                         vcjh);
}
template <int DIM, int NV, typename S>
void launch_wavesp(const void *tr, const double *nrmOwn, double *ws, int NF, int nE, const Phys &ph, cudaStream_t st) {
  long n = (long)NF * nE;
  fr_wavesp_kernel<DIM, NV, S><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(static_cast<const S *>(tr), nrmOwn, ws,
                                                                             NF, nE, ph);
}

template <class C, typename R, typename S, bool BC, int RS>
bool make_set(KernelSet &k, std::string &err) {
  using T = Tile<C, R>;
  k.stage = &launch_stage<C, R, S, BC, RS>;
  k.trace = &launch_trace<C, R, S>;
  k.wavesp = &launch_wavesp<C::DIM, C::NV, S>;
  k.TE = T::TE;
  k.NT = C::NT;
  k.smem = T::SMEM;
  auto fn = fr_stage_kernel<C, R, S, BC, RS>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  if (e == cudaSuccess) {
    // load the trace kernel now (lazy module loading would otherwise load it
    // at its first launch, e.g. inside frg_calc_residual_noalloc)
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, fr_trace_kernel<C, R, S>);
  }
  if constexpr (C::DIM == 2) {
    // variant 0 is the default; the others are candidates for frg_autotune
    k.nTma = 0;
    if (e == cudaSuccess) e = add_tma_variant<C, R, S, BC, RS, 0, 128>(k);
    if (e == cudaSuccess) e = add_tma_variant<C, R, S, BC, RS, 0, 256>(k);
    if (e == cudaSuccess) e = add_tma_variant<C, R, S, BC, RS, -1, 128>(k);
    if (e == cudaSuccess) e = add_tma_variant<C, R, S, BC, RS, -1, 64>(k);
    if (e == cudaSuccess) e = add_tma_variant<C, R, S, BC, RS, -2, 64>(k);
    if (e == cudaSuccess) e = add_tma_variant<C, R, S, BC, RS, -2, 32>(k);
    // persistent, ring-buffered variants
    if (e == cudaSuccess) e = add_pipe_variant<C, R, S, BC, RS, 0, 160, 2>(k);
    if (e == cudaSuccess) e = add_pipe_variant<C, R, S, BC, RS, 0, 160, 3>(k);
    if (e == cudaSuccess) e = add_pipe_variant<C, R, S, BC, RS, 0, 256, 2>(k);
    if (e == cudaSuccess) e = add_pipe_variant<C, R, S, BC, RS, 0, 128, 2>(k);
    // persistent, FP64 buffers outside the ring (four blocks per SM)
    if (e == cudaSuccess) e = add_split_variant<C, R, S, BC, RS, 0, 160>(k);
    if (e == cudaSuccess) e = add_split_variant<C, R, S, BC, RS, 0, 128>(k);
  }
  if (e != cudaSuccess) { err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e); return false; }
  return true;
}

// 3D viscous TMA passes: tiles of 4 (FP32) or 2 (FP64) elements, the 16-byte
// minimum row of a TMA box; 128 threads for the gradient pass (three blocks
// per SM), 256 for the stage pass (two blocks per SM, by shared memory)
template <typename S>
constexpr int visc_tma_te() { return sizeof(S) == 4 ? 4 : 2; }
constexpr int kViscGradNT = 256, kViscStageNT = 256;
template <class C, typename R, typename S, bool BC>
void launch_visc3_grad(const void *args, const void *maps, int nBlk, size_t smem, cudaStream_t st) {
  fr_visc3_grad_tma_kernel<C, R, S, BC, visc_tma_te<S>(), kViscGradNT><<<nBlk, kViscGradNT, smem, st>>>(
      *static_cast<const StageArgs *>(args), *static_cast<const ViscMaps *>(maps));
}
template <class C, typename R, typename S, bool BC, int RS>
void launch_visc3_stage(const void *args, const void *maps, int nBlk, size_t smem, cudaStream_t st) {
  fr_visc3_stage_tma_kernel<C, R, S, BC, RS, visc_tma_te<S>(), kViscStageNT><<<nBlk, kViscStageNT, smem, st>>>(
      *static_cast<const StageArgs *>(args), *static_cast<const ViscMaps *>(maps));
}
template <class C0, typename R, typename S, bool BC, int RS>
cudaError_t add_visc3_tma(KernelSet &k) {
  using C = CfgV<C0>;  // the TMA tiles' point padding
  constexpr int TE = visc_tma_te<S>();
  using TG = VGradT<C, R, S, TE, kViscGradNT>;
  using TS = VStageT<C, R, S, TE, kViscStageNT>;
  if (TG::SMEM > 227 * 1024 || TS::SMEM > 227 * 1024) return cudaSuccess;  // not offered
  auto fg = fr_visc3_grad_tma_kernel<C, R, S, BC, TE, kViscGradNT>;
  auto fs = fr_visc3_stage_tma_kernel<C, R, S, BC, RS, TE, kViscStageNT>;
  cudaError_t e = cudaFuncSetAttribute(fg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TG::SMEM);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(fs, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TS::SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(fg, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(fs, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&k.vgradOcc, fg, kViscGradNT, TG::SMEM);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&k.vstageOcc, fs, kViscStageNT, TS::SMEM);
  if (e != cudaSuccess) return e;
  if (k.vgradOcc < 1 || k.vstageOcc < 1) return cudaErrorInvalidConfiguration;
  k.vgrad = &launch_visc3_grad<C, R, S, BC>;
  k.vstage = &launch_visc3_stage<C, R, S, BC, RS>;
  k.vTE = TE;
  k.vPadG = C::PADG;
  k.vgradSmem = TG::SMEM;
  k.vstageSmem = TS::SMEM;
  return cudaSuccess;
}

template <class C, typename R, typename S, bool BC, int RS>
bool make_set_visc(KernelSet &k, std::string &err) {
  using T = TileV<C, R>;
  k.stage = &launch_stage_visc<C, R, S, BC, RS>;
  k.grad = &launch_grad<C, R, S, BC>;
  k.trace = &launch_trace<C, R, S>;
  k.wavesp = &launch_wavesp<C::DIM, C::NV, S>;
  k.TE = T::TE;
  k.NT = C::NT;
  k.smem = T::SMEM;
  auto f1 = fr_stage_visc_kernel<C, R, S, BC, RS>;
  auto f2 = fr_visc_grad_kernel<C, R, S, BC>;
  cudaError_t e = cudaFuncSetAttribute(f1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(f2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(f1, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(f2, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  if (e == cudaSuccess) {
    cudaFuncAttributes fa;  // load the trace kernel now (see make_set)
    e = cudaFuncGetAttributes(&fa, fr_trace_kernel<C, R, S>);
  }
  if constexpr (C::DIM == 3)
    if (e == cudaSuccess) e = add_visc3_tma<C, R, S, BC, RS>(k);
  if (e != cudaSuccess) { err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e); return false; }
  return true;
}

template <class C, typename R, typename S, bool BC, int RS>
bool make_one(const KernelKey &key, KernelSet &k, std::string &err) {
  return key.viscous ? make_set_visc<C, R, S, BC, RS>(k, err) : make_set<C, R, S, BC, RS>(k, err);
}

template <int DIM, int P, int NV, typename R, typename S>
bool make_variant(const KernelKey &key, KernelSet &k, std::string &err) {
  using C = Cfg<DIM, P, NV>;
  if constexpr (NV == 1 || DIM == 3) {
    return key.bc ? make_one<C, R, S, true, 0>(key, k, err) : make_one<C, R, S, false, 0>(key, k, err);
  } else {
    if (key.riemann == 1)
      return key.bc ? make_one<C, R, S, true, 1>(key, k, err) : make_one<C, R, S, false, 1>(key, k, err);
    return key.bc ? make_one<C, R, S, true, 0>(key, k, err) : make_one<C, R, S, false, 0>(key, k, err);
  }
}

template <int DIM, int NV, typename R, typename S>
bool select_order(const KernelKey &key, KernelSet &k, std::string &err) {
  switch (key.P) {
    case 1: return make_variant<DIM, 1, NV, R, S>(key, k, err);
    case 2: return make_variant<DIM, 2, NV, R, S>(key, k, err);
    case 3: return make_variant<DIM, 3, NV, R, S>(key, k, err);
    case 4: return make_variant<DIM, 4, NV, R, S>(key, k, err);
    case 5:
      if constexpr (DIM == 2) return make_variant<DIM, 5, NV, R, S>(key, k, err);
      break;
  }
  err = "order not available for this dimension (2D: 1..5, 3D: 1..4)";
  return false;
}

}  // namespace
}  // namespace frg

#define FRG_CAT2(a, b) a##b
#define FRG_CAT(a, b) FRG_CAT2(a, b)

namespace frg {
bool FRG_CAT(select_, FRG_UNIT_NAME)(const KernelKey &key, KernelSet &k, std::string &err) {
  using R = FRG_UNIT_R;
  using S = FRG_UNIT_S;
  if (key.NV == 1) return select_order<FRG_UNIT_DIM, 1, R, S>(key, k, err);
  if (key.NV == FRG_UNIT_DIM + 2) return select_order<FRG_UNIT_DIM, FRG_UNIT_DIM + 2, R, S>(key, k, err);
  err = "unsupported field count";
  return false;
}
cudaError_t FRG_CAT(upload_tables_, FRG_UNIT_NAME)() { return upload_tables_impl(); }
}  // namespace frg
