// metrics.cu -- element metrics on the device from node coordinates: the
// reference's solver::calcTransforms (src/solver.cpp:1227-1356) and the
// solution-point positions of setPosSptsFpts (:904-951), as run again by
// solver::updateTransforms (:1358-1363) when the nodes of a mesh move.
//
// One thread per (point, element), element fastest.  Every sum and product is
// rounded on its own (__dadd_rn / __dmul_rn, no fused multiply-add) and in
// the host set-up's order, so the device metrics are bitwise the ones that
// csrc/setup.cpp computes for the same nodes; sqrt and the divisions are the
// correctly rounded IEEE operations on both sides.
#include <cuda_runtime.h>

#include <cstdint>

#include "dispatch.h"

namespace frg {
namespace {

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// J[a][k] = d x_k / d xi_a at one point from its rows of the derivative table
// (rows [a][pt][n], nPt points), element nodes X[n][k].
template <int D>
__device__ __forceinline__ void jacobian(const double *dsh, int nPt, int pt, int nN, const double *X, double J[3][3]) {
#pragma unroll
  for (int a = 0; a < D; a++) {
    const double *row = dsh + ((size_t)a * nPt + pt) * nN;
#pragma unroll
    for (int k = 0; k < D; k++) {
      double v = 0.0;
      for (int n = 0; n < nN; n++) v = add(v, mul(row[n], X[n * D + k]));
      J[a][k] = v;
    }
  }
}

// Adjugate (JGinv) and determinant in the host set-up's operation order.
template <int D>
__device__ __forceinline__ double adjugate(const double J[3][3], double G[3][3]) {
  if constexpr (D == 2) {
    G[0][0] = J[1][1]; G[0][1] = -J[1][0]; G[1][0] = -J[0][1]; G[1][1] = J[0][0];
    return sub(mul(J[0][0], J[1][1]), mul(J[0][1], J[1][0]));
  } else {
    const double xr = J[0][0], xs = J[1][0], xt = J[2][0], yr = J[0][1], ys = J[1][1], yt = J[2][1];
    const double zr = J[0][2], zs = J[1][2], zt = J[2][2];
    G[0][0] = sub(mul(ys, zt), mul(yt, zs)); G[0][1] = sub(mul(xt, zs), mul(xs, zt));
    G[0][2] = sub(mul(xs, yt), mul(xt, ys));
    G[1][0] = sub(mul(yt, zr), mul(yr, zt)); G[1][1] = sub(mul(xr, zt), mul(xt, zr));
    G[1][2] = sub(mul(xt, yr), mul(xr, yt));
    G[2][0] = sub(mul(yr, zs), mul(ys, zr)); G[2][1] = sub(mul(xs, zr), mul(xr, zs));
    G[2][2] = sub(mul(xr, ys), mul(xs, yr));
    return add(sub(mul(xr, sub(mul(ys, zt), mul(yt, zs))), mul(xs, sub(mul(yr, zt), mul(yt, zr)))),
               mul(xt, sub(mul(yr, zs), mul(ys, zr))));
  }
}

template <typename S>
__device__ __forceinline__ void put(void *p, size_t i, double v) {
  static_cast<S *>(p)[i] = (S)v;
}

// Check pass (out == nullptr): flags a negative Jacobian at any solution
// point and keeps the smallest such element.  Write pass: every metric.
template <int D, typename S>
__global__ void __launch_bounds__(256) fr_metrics_kernel(const double *__restrict__ xv, const double *__restrict__ tab,
                                                         const int *__restrict__ fdir, const int *__restrict__ fsgn,
                                                         int nN, int nS, int nF, int nE, int L, int check,
                                                         MetricOut out, unsigned *flag) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int nPt = check ? nS : nS + nF;
  if (idx >= (long)nPt * nE) return;
  const int pt = (int)(idx / nE), e = (int)(idx - (long)pt * nE);
  const double *X = xv + (size_t)e * nN * D;
  const double *shS = tab, *dS = tab + (size_t)nS * nN, *dF = dS + (size_t)D * nS * nN;
  double J[3][3], G[3][3];
  if (pt < nS) {
    const int s = pt;
    jacobian<D>(dS, nS, s, nN, X, J);
    const double det = adjugate<D>(J, G);
    if (check) {
      if (det < 0) {
        atomicOr(flag, 1u);
        atomicMin(flag + 1, (unsigned)e);
      }
      return;
    }
#pragma unroll
    for (int k = 0; k < D; k++) {
      double v = 0.0;
      for (int n = 0; n < nN; n++) v = add(v, mul(shS[(size_t)s * nN + n], X[n * D + k]));
      out.pos[((size_t)s * nE + e) * D + k] = v;
    }
    const size_t q = (size_t)s * L + e;
    out.detJd[q] = det;
    put<S>(out.detJs, q, det);
    put<S>(out.invDetS, q, __ddiv_rn(1.0, det));
#pragma unroll
    for (int a = 0; a < D; a++)
#pragma unroll
      for (int b = 0; b < D; b++) put<S>(out.JG, ((size_t)(a * D + b) * nS + s) * L + e, G[a][b]);
  } else {
    const int f = pt - nS;
    jacobian<D>(dF, nF, f, nN, X, J);
    adjugate<D>(J, G);
    const int dir = fdir[f];
    const double tn = (double)fsgn[f];
    double nv[3], mag = 0.0;
    // norm = JGinv^T tNorm, summed over every reference direction as the
    // host does (the other directions add exact zeros)
#pragma unroll
    for (int k = 0; k < D; k++) {
      nv[k] = 0.0;
#pragma unroll
      for (int a = 0; a < D; a++) nv[k] = add(nv[k], mul(G[a][k], a == dir ? tn : 0.0));
    }
#pragma unroll
    for (int k = 0; k < D; k++) mag = add(mag, mul(nv[k], nv[k]));
    mag = __dsqrt_rn(mag);
    if (fabs(mag) < 1e-10) {
      mag = 0.0;
#pragma unroll
      for (int k = 0; k < D; k++) nv[k] = 0.0;
    } else {
#pragma unroll
      for (int k = 0; k < D; k++) nv[k] = __ddiv_rn(nv[k], mag);
    }
    const size_t q = (size_t)f * L + e;
#pragma unroll
    for (int k = 0; k < D; k++) out.nrmOwn[(size_t)k * nF * L + q] = nv[k];
    out.dAd[q] = mag;
    put<S>(out.dAs, q, mag);
  }
}

// Second pass, one thread per (flux point, element): the normal the common
// flux uses (the face's left element's, intFace::setupRightState), and per
// element its volume sum(detJ * w) in solution-point order.
template <int D, typename S>
__global__ void __launch_bounds__(256) fr_metrics_face_kernel(const int *__restrict__ nbr, const double *__restrict__ wv,
                                                              int nS, int nF, int nE, int L, MetricOut out) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)nF * nE) return;
  const int f = (int)(idx / nE), e = (int)(idx - (long)f * nE);
  const size_t q = (size_t)f * L + e;
  const int c = nbr[q];
  const size_t src = (c >= 0 && (c & 1)) ? (size_t)(c >> 1) : q;
#pragma unroll
  for (int k = 0; k < D; k++) put<S>(out.nrmC, (size_t)k * nF * L + q, out.nrmOwn[(size_t)k * nF * L + src]);
  if (f == 0) {
    double v = 0.0;
    for (int s = 0; s < nS; s++) v = add(v, mul(out.detJd[(size_t)s * L + e], wv[s]));
    out.vol[e] = v;
  }
}

template <int D, typename S>
cudaError_t launch_all(const double *xv, const double *tab, const int *fdir, const int *fsgn, const double *wv,
                       const int *nbr, int nN, int nS, int nF, int nE, int L, int check, const MetricOut &out,
                       unsigned *flag, cudaStream_t st) {
  const long n = (long)(check ? nS : nS + nF) * nE;
  fr_metrics_kernel<D, S><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(xv, tab, fdir, fsgn, nN, nS, nF, nE, L, check,
                                                                        out, flag);
  if (check) return cudaGetLastError();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const long m = (long)nF * nE;
  fr_metrics_face_kernel<D, S><<<(unsigned)((m + 255) / 256), 256, 0, st>>>(nbr, wv, nS, nF, nE, L, out);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_metrics(int nDims, int storeBytes, const double *xv, const double *tab, const int *fdir,
                           const int *fsgn, const double *wv, const int *nbr, int nN, int nS, int nF, int nE, int L,
                           int check, const MetricOut &out, unsigned *flag, cudaStream_t st) {
  if (nDims == 2)
    return storeBytes == 8 ? launch_all<2, double>(xv, tab, fdir, fsgn, wv, nbr, nN, nS, nF, nE, L, check, out, flag, st)
                           : launch_all<2, float>(xv, tab, fdir, fsgn, wv, nbr, nN, nS, nF, nE, L, check, out, flag, st);
  return storeBytes == 8 ? launch_all<3, double>(xv, tab, fdir, fsgn, wv, nbr, nN, nS, nF, nE, L, check, out, flag, st)
                         : launch_all<3, float>(xv, tab, fdir, fsgn, wv, nbr, nN, nS, nF, nE, L, check, out, flag, st);
}

}  // namespace frg
