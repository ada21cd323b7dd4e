// adjoint_impl.cuh -- launchers and the instantiation switch of the adjoint
// kernels; included once per dimension unit after defining FRG_ADJ_DIM.
#pragma once
#include <array>

#include "adjoint.cuh"
#include "adjoint_visc.cuh"
#include "dispatch.h"
#include "optab_upload.cuh"

namespace frg {
namespace {

constexpr int kAdjGrid = 148 * 8;  // grid-stride launches: 8 blocks per SM

template <class C>
void launch_adj_face(const AdjArgs &a, cudaStream_t st) {
  const long n = (long)C::NF * a.nE;
  const int nb = (int)std::min<long>((n + 255) / 256, kAdjGrid);
  fr_adj_face_kernel<C><<<nb, 256, 0, st>>>(a);
}
template <class C, bool BC, int RS>
void launch_adj_elem(const AdjArgs &a, cudaStream_t st) {
  using T = AdjTile<C>;
  const int nb = (a.nEle + T::TE - 1) / T::TE;
  fr_adj_elem_kernel<C, BC, RS><<<nb, T::NT, T::SMEM, st>>>(a);
}
template <class C>
void launch_entropy(const double *U, const double *detJ, const double *wvol, int nE, int L, const Phys &ph,
                    double *grad, double *part, cudaStream_t st) {
  fr_obj_entropy_kernel<C::DIM, C::NV><<<kAdjGrid, 256, 0, st>>>(U, detJ, wvol, C::NS, nE, L, ph, grad, part);
}
template <class C>
void launch_wallp(const double *U, const int *nbr, const double *dA, const double *wsurf, int vcjh, int nE, int L,
                  int bcWall, const Phys &ph, double *grad, double *part, cudaStream_t st) {
  fr_obj_wallp_kernel<C><<<(nE + 127) / 128, 128, 0, st>>>(U, nbr, dA, wsurf, vcjh, nE, L, bcWall, ph, grad, part);
}

// Viscous residuals: the forward gradient / projected-flux pass (the
// generic gradient kernel on the stage state), then the two adjoint passes.
template <class C, bool BC, int RS>
void launch_adjv_elem(const AdjArgs &a, cudaStream_t st) {
  using TV = TileV<C, double>;
  StageArgs f{};
  f.nE = a.nE;
  f.nEle = a.nEle;
  f.ldU = a.nE;
  f.Uin_d = a.Y;
  f.trIn = a.trY;
  f.nbr = a.nbr;
  f.nrm = a.nrm;
  f.dA = a.dA;
  f.JG = a.JG;
  f.detJ = a.detJ;
  f.err = a.err;
  f.vcjh = a.vcjh;
  f.flags = SF_RESIDUAL;
  f.fvnOut = a.v.fvn;
  f.fvn2Out = a.v.fvn2;
  f.visc2 = a.v.visc2;
  f.dUg = a.v.g;
  f.ph = a.ph;
  // this order's 1D operators for every VCJH scheme, built once
  static const std::array<Ops1D, 4> ops = [] {
    std::array<Ops1D, 4> t{};
    for (int sch = 0; sch < 4; sch++)
      if (!((sch == 3 && C::P < 2) || (sch == 2 && C::P == 0))) t[sch] = build_ops1d(C::P, sch);
    return t;
  }();
  set_stage_ops(f, ops[a.vcjh]);
  fr_visc_grad_kernel<C, double, double, BC><<<(a.nEle + TV::TE - 1) / TV::TE, C::NT, TV::SMEM, st>>>(f);
  using T = AdjViscTile<C>;
  fr_adjv_elem_kernel<C, BC, RS><<<(a.nEle + T::TE - 1) / T::TE, T::NT, T::SMEM, st>>>(a);
  fr_adjv_out_kernel<C, BC><<<(a.nEle + 3) / 4, 128, 0, st>>>(a);
}

template <class C, bool BC, int RS>
bool make_adjv(AdjSet &k, std::string &err) {
  using T = AdjViscTile<C>;
  using TV = TileV<C, double>;
  k.face = &launch_adj_face<C>;
  k.elem = &launch_adjv_elem<C, BC, RS>;
  k.TE = T::TE;
  k.elemLaunches = 3;
  if constexpr (C::NV > 1) {
    k.entropy = &launch_entropy<C>;
    k.wallp = &launch_wallp<C>;
    k.entropyBlocks = kAdjGrid;
  }
  cudaError_t e = cudaFuncSetAttribute(fr_adjv_elem_kernel<C, BC, RS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)T::SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(fr_visc_grad_kernel<C, double, double, BC>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TV::SMEM);
  if (e != cudaSuccess) { err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e); return false; }
  return true;
}

template <class C, bool BC, int RS>
bool make_adj(AdjSet &k, std::string &err) {
  using T = AdjTile<C>;
  k.face = &launch_adj_face<C>;
  k.elem = &launch_adj_elem<C, BC, RS>;
  k.TE = T::TE;
  if constexpr (C::NV > 1) {
    k.entropy = &launch_entropy<C>;
    k.wallp = &launch_wallp<C>;
    k.entropyBlocks = kAdjGrid;
  }
  cudaError_t e = cudaFuncSetAttribute(fr_adj_elem_kernel<C, BC, RS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)T::SMEM);
  if (e != cudaSuccess) { err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e); return false; }
  return true;
}

template <class C, bool BC, int RS>
bool make_adj(AdjSet &k, std::string &err, bool viscous) {
  if (viscous) return make_adjv<C, BC, RS>(k, err);
  return make_adj<C, BC, RS>(k, err);
}

template <int DIM, int P, int NV>
bool adj_variant(const KernelKey &key, AdjSet &k, std::string &err) {
  using C = Cfg<DIM, P, NV>;
  const bool v = key.viscous != 0;
  if constexpr (NV == 1 || DIM == 3) {
    return key.bc ? make_adj<C, true, 0>(k, err, v) : make_adj<C, false, 0>(k, err, v);
  } else {
    if (key.riemann == 1) return key.bc ? make_adj<C, true, 1>(k, err, v) : make_adj<C, false, 1>(k, err, v);
    return key.bc ? make_adj<C, true, 0>(k, err, v) : make_adj<C, false, 0>(k, err, v);
  }
}

template <int DIM, int NV>
bool adj_order(const KernelKey &key, AdjSet &k, std::string &err) {
  switch (key.P) {
    case 1: return adj_variant<DIM, 1, NV>(key, k, err);
    case 2: return adj_variant<DIM, 2, NV>(key, k, err);
    case 3: return adj_variant<DIM, 3, NV>(key, k, err);
    case 4: return adj_variant<DIM, 4, NV>(key, k, err);
    case 5:
      if constexpr (DIM == 2) return adj_variant<DIM, 5, NV>(key, k, err);
      break;
  }
  err = "adjoint: order not available for this dimension";
  return false;
}

}  // namespace

#define FRG_ADJ_CAT2(a, b) a##b
#define FRG_ADJ_CAT(a, b) FRG_ADJ_CAT2(a, b)

bool FRG_ADJ_CAT(select_adj_, FRG_ADJ_NAME)(const KernelKey &key, AdjSet &k, std::string &err) {
  if (key.precision != 0) { err = "adjoint: FP64 precision only"; return false; }
  if (key.NV == 1) return adj_order<FRG_ADJ_DIM, 1>(key, k, err);
  if (key.NV == FRG_ADJ_DIM + 2) return adj_order<FRG_ADJ_DIM, FRG_ADJ_DIM + 2>(key, k, err);
  err = "adjoint: unsupported field count";
  return false;
}
cudaError_t FRG_ADJ_CAT(upload_tables_adj_, FRG_ADJ_NAME)() { return upload_tables_impl(); }

}  // namespace frg
