// integrals.cu -- the output integrals of the reference on the device:
//   solver::computeWallForce   (src/solver.cpp:1367-1378, src/boundFace.cpp:330-378)
//   solver::computeMassFlux    (src/solver.cpp:1380-1391, src/boundFace.cpp:380-418)
//   solver::integrateError     (src/solver.cpp:1507-1574) with calcError
//                              (src/funcs.cpp:1875-1979), testCase 1
// Each kernel writes one partial sum per block and output component; the
// host adds the partials in block order.  These run once per output step,
// not per RK stage.
#include <cuda_runtime.h>

#include "dispatch.h"
#include "physics.cuh"

namespace frg {
namespace {

// Flux point f's face line (the tensor-product geometry of kernels.cuh's
// fpt_line, for a run-time order): side of the face and first solution
// point / stride of the coordinate line through f.
__device__ void fpt_line_rt(int dim, int P, int f, int &side, int &s0, int &st) {
  const int N1 = P + 1;
  if (dim == 2) {
    const int face = f / N1, k = f - face * N1;
    switch (face) {
      case 0: side = 0; s0 = k; st = N1; break;
      case 1: side = 1; s0 = k * N1; st = 1; break;
      case 2: side = 1; s0 = P - k; st = N1; break;
      default: side = 0; s0 = (P - k) * N1; st = 1; break;
    }
  } else {
    const int P12 = N1 * N1, face = f / P12, k = f - face * P12, a = k % N1, b = k / N1;
    switch (face) {
      case 0: side = 0; s0 = a + N1 * b; st = P12; break;
      case 1: side = 1; s0 = (P - a) + N1 * b; st = P12; break;
      case 2: side = 0; s0 = N1 * a + P12 * b; st = 1; break;
      case 3: side = 1; s0 = N1 * (P - a) + P12 * b; st = 1; break;
      case 4: side = 0; s0 = (P - a) + P12 * b; st = N1; break;
      default: side = 1; s0 = a + P12 * b; st = N1; break;
    }
  }
}

// viscousStressTensor (src/flux.cpp:228-358)
template <int DIM>
__device__ void stress_tensor(const double *U, const double *g /*[DIM][NV]*/, double tau[3][3], const Phys &ph) {
  constexpr int NV = DIM + 2;
  auto G = [&](int a, int b) { return g[a * NV + b]; };
  const double rho = U[0], u = U[1] / rho, v = U[2] / rho;
  double e = U[DIM + 1] / rho - 0.5 * (u * u + v * v), w = 0.;
  if (DIM == 3) {
    w = U[3] / rho;
    e -= 0.5 * (w * w);
  }
  const double dRho_dx = G(0, 0), dRhoU_dx = G(0, 1), dRhoV_dx = G(0, 2);
  const double dRho_dy = G(1, 0), dRhoU_dy = G(1, 1), dRhoV_dy = G(1, 2);
  double dRho_dz = 0, dRhoU_dz = 0, dRhoW_dz = 0;
  if (DIM == 3) {
    dRho_dz = G(2, 0);
    dRhoU_dz = G(2, 1);
    dRhoW_dz = G(2, 3);
  }
  double mu = ph.mu;
  if (!ph.fixVis) {
    const double rt = (ph.gamma - 1.0) * e / ph.rt_inf;
    mu *= pow(rt, 1.5) * (1. + ph.c_sth) / (rt + ph.c_sth);
  }
  const double du_dx = (dRhoU_dx - dRho_dx * u) / rho, du_dy = (dRhoU_dy - dRho_dy * u) / rho;
  const double dv_dx = (dRhoV_dx - dRho_dx * v) / rho, dv_dy = (dRhoV_dy - dRho_dy * v) / rho;
  double du_dz = 0, dw_dz = 0;
  if (DIM == 3) {
    du_dz = (dRhoU_dz - dRho_dz * u) / rho;
    dw_dz = (dRhoW_dz - dRho_dz * w) / rho;
  }
  const double diag = (du_dx + dv_dy + dw_dz) / 3.0;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) tau[i][j] = 0;
  tau[0][0] = 2.0 * mu * (du_dx - diag);
  tau[1][1] = 2.0 * mu * (dv_dy - diag);
  tau[0][1] = tau[1][0] = mu * (du_dy + dv_dx);
  if (DIM == 3) {
    tau[0][2] = tau[2][0] = mu * (du_dz + dv_dx);
    tau[1][2] = tau[2][1] = mu * (du_dz + dv_dy);
    tau[2][2] = 2.0 * mu * (dw_dz - diag);
  }
}

// Block sum of NO values per thread into part[blockIdx.x * NO + j].
template <int NO>
__device__ void block_sum(double (&v)[NO], double *part) {
  __shared__ double sm[NO][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int j = 0; j < NO; j++) {
    double x = v[j];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sm[j][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x < NO) {
    double x = 0;
    for (int w = 0; w < nw; w++) x += sm[threadIdx.x][w];
    part[(size_t)blockIdx.x * NO + threadIdx.x] = x;
  }
}

template <typename S>
__device__ __forceinline__ double ld(const void *p, size_t i) {
  return (double)static_cast<const S *>(p)[i];
}

// One thread per (flux point, element): computeWallForce (kind 0, six sums)
// or computeMassFlux with errorNorm kind - 1 (nV sums) at boundary flux points.
template <int DIM, int NV, typename S>
__global__ void __launch_bounds__(256) fr_boundary_integral_kernel(const BndIntArgs a, double *part) {
  constexpr int NO = 6;
  double acc[NO] = {0, 0, 0, 0, 0, 0};
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int f = (int)(idx / a.L), e = (int)(idx - (long)f * a.L);
  const int code = (idx < (long)a.nF * a.L && e < a.nE) ? a.nbr[(size_t)f * a.L + e] : 0;
  const int bc = -1 - code;
  const bool wall = bc == BC_SLIP || bc == BC_ADI_NOSLIP || bc == BC_ISO_NOSLIP;
  const bool inout = bc == BC_CHAR || bc == BC_SUP_IN || bc == BC_SUP_OUT || bc == BC_SUB_IN || bc == BC_SUB_OUT;
  if (code < 0 && (a.kind == 0 ? wall : inout)) {
    const int N1 = a.P + 1, k = f % a.nFF;
    const double weight = DIM == 2 ? a.w1[k] : a.w1[k % N1] * a.w1[k / N1];
    double U[NV], n[DIM];
#pragma unroll
    for (int v = 0; v < NV; v++) U[v] = ld<S>(a.tr, ((size_t)v * a.nF + f) * a.L + e);
#pragma unroll
    for (int d = 0; d < DIM; d++) n[d] = a.nrm[((size_t)d * a.nF + f) * a.L + e];
    const double dA = a.dA[(size_t)f * a.L + e];
    double g[DIM * NV];
    if (a.viscous) {
      // the corrected gradient extrapolated to the flux point (extrapolateGradU)
      int side, s0, st;
      fpt_line_rt(DIM, a.P, f, side, s0, st);
#pragma unroll
      for (int q = 0; q < DIM * NV; q++) {
        double t = 0;
        for (int j = 0; j < N1; j++) t += a.lag[side][j] * ld<S>(a.dUg, ((size_t)q * a.nS + s0 + j * st) * a.L + e);
        g[q] = t;
      }
    }
    if (a.kind == 0) {
      if constexpr (NV > 1) {
        const double rho = U[0];
        double vMagSq = 0;
#pragma unroll
        for (int d = 0; d < DIM; d++) vMagSq += U[d + 1] * U[d + 1] / (rho * rho);
        const double p = (a.ph.gamma - 1) * (U[DIM + 1] - 0.5 * rho * vMagSq);
#pragma unroll
        for (int d = 0; d < DIM; d++) acc[d] = p * n[d] * dA * weight;
        if (a.viscous) {
          double tau[3][3];
          stress_tensor<DIM>(U, g, tau, a.ph);
#pragma unroll
          for (int d1 = 0; d1 < DIM; d1++)
#pragma unroll
            for (int d2 = 0; d2 < DIM; d2++) acc[3 + d1] -= tau[d1][d2] * n[d2] * dA * weight;
        }
      }
    } else {
      // the boundary face's common flux: Rusanov on the ghost state
      // (src/face.cpp:142-145), Lax-Friedrichs with a zero ghost state for
      // advection, plus the viscous part (src/face.cpp:177-287)
      double UR[NV], Fn[NV];
      if constexpr (NV == 1) {
        UR[0] = 0.0;
        lax_friedrichs<DIM, double>(U[0], UR[0], n, Fn, a.ph);
      } else {
        bc_ghost<DIM>(bc, U, n, UR, a.ph);  // in / out conditions: always known
        rusanov<DIM, NV, double, double>(U, UR, n, Fn, a.ph);
      }
      if (a.viscous) {
        double FL[DIM][NV];
        if constexpr (NV == 1) {
          viscous_flux_ad<DIM, double>(g, FL, a.ph);
          double t = 0;  // centralFlux with a zero ghost gradient
#pragma unroll
          for (int d = 0; d < DIM; d++) t += 0.5 * (FL[d][0] + 0.0) * n[d];
          Fn[0] += t;
        } else {
          viscous_flux<DIM, double>(U, g, FL, a.ph);
#pragma unroll
          for (int d = 0; d < DIM; d++)
#pragma unroll
            for (int v = 0; v < NV; v++) Fn[v] += (FL[d][v] + a.ph.tau * n[d] * (U[v] - UR[v])) * n[d];
        }
      }
      const int en = a.kind - 1;
#pragma unroll
      for (int v = 0; v < NV; v++)
        acc[v] = en == 0 ? Fn[v] * dA * weight
                         : en == 1 ? fabs(Fn[v]) * dA * weight * n[0] : (Fn[v] * dA) * (Fn[v] * dA) * weight * n[0];
    }
  }
  block_sum<NO>(acc, part);
}

// calcError (src/funcs.cpp:1875-1979), testCase 1, into err[NV].
template <int DIM, int NV>
__device__ void calc_error(const ErrIntArgs &a, const double *U, const double *x, double *err) {
  constexpr double PI = 3.141592653589793;
  const double xmin = a.box[0], xmax = a.box[1], ymin = a.box[2], ymax = a.box[3];
#pragma unroll
  for (int v = 0; v < NV; v++) err[v] = 0;
  if constexpr (NV > 1) {
    const double gamma = a.ph.gamma;
    if (a.icType == 0) {
      const double pfs = a.ph.pB, rhofsg = pow(a.ph.rhoB, gamma);
      const double rho = U[0], u = U[1] / rho, v = U[2] / rho, w = DIM == 2 ? 0 : U[3] / rho;
      const double p = (gamma - 1.) * (U[DIM + 1] - .5 * rho * (u * u + v * v + w * w));
      err[0] = p * rhofsg / (pow(rho, gamma) * pfs) - 1.;
    } else {
      const double eps = a.eps;
      double X = fmod((x[0] - a.time), (xmax - xmin)), Y = fmod((x[1] - a.time), (ymax - ymin));
      if (X > xmax) X -= (xmax - xmin);
      if (Y > ymax) Y -= (ymax - ymin);
      if (X < xmin) X += (xmax - xmin);
      if (Y < ymin) Y += (ymax - ymin);
      const double f = 1.0 - (X * X + Y * Y);
      const double rho =
          fmax(pow(1. - eps * eps * (gamma - 1.) / (8. * gamma * PI * PI) * exp(f), 1.0 / (gamma - 1.0)), 1e-10);
      const double vx = 1. - eps * Y / (2. * PI) * exp(f / 2.), vy = 1. + eps * X / (2. * PI) * exp(f / 2.);
      const double p = pow(rho, gamma);
      err[0] = rho;
      err[1] = rho * vx;
      err[2] = rho * vy;
      if (DIM == 3) err[3] = 0.;
      err[DIM + 1] = p / (gamma - 1) + (0.5 * rho * (vx * vx + vy * vy));
#pragma unroll
      for (int v = 0; v < NV; v++) err[v] = U[v] - err[v];
    }
  } else {
    double X = fabs(fmod((x[0] - a.time), (xmax - xmin))), Y = fabs(fmod((x[1] - a.time), (ymax - ymin)));
    if (X > (xmax - xmin) / 2) X -= (xmax - xmin);
    if (Y > (ymax - ymin) / 2) Y -= (ymax - ymin);
    double ex;
    if (a.icType == 0) ex = exp(-(X * X + Y * Y));
    else if (a.icType == 1) ex = 1 + sin(2. * PI * (x[0] + 5. - a.time) / 10.);
    else ex = cos(2 * PI * x[0] / 6.) * cos(2 * PI * x[1] / 6.) * cos(2 * PI * (DIM == 3 ? x[2] : 0.0) / 6.);
    err[0] = U[0] - ex;
  }
  if (a.errorNorm == 1)
#pragma unroll
    for (int v = 0; v < NV; v++) err[v] = fabs(err[v]);
  else if (a.errorNorm == 2)
#pragma unroll
    for (int v = 0; v < NV; v++) err[v] *= err[v];
}

// One thread per (quadrature point, element): the state and detJ
// interpolated to the point (interp null: the point is a solution point),
// its position from the element's nodes, the error times weight and detJ;
// errorNorm 0 also sums the state itself (2 NV outputs).
template <int DIM, int NV>
__global__ void __launch_bounds__(256) fr_error_integral_kernel(const ErrIntArgs a, double *part) {
  constexpr int NO = 2 * NV;
  double acc[NO];
#pragma unroll
  for (int j = 0; j < NO; j++) acc[j] = 0;
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int q = (int)(idx / a.nE), e = (int)(idx - (long)q * a.nE);
  if (idx < (long)a.nQ * a.nE) {
    double U[NV], det, x[3] = {0, 0, 0}, err[NV];
    if (a.interp) {
      det = 0;
#pragma unroll
      for (int v = 0; v < NV; v++) U[v] = 0;
      for (int s = 0; s < a.nS; s++) {
        const double c = a.interp[(size_t)q * a.nS + s];
#pragma unroll
        for (int v = 0; v < NV; v++) U[v] += c * a.U[((size_t)v * a.nS + s) * a.L + e];
        det += c * a.detJ[(size_t)s * a.L + e];
      }
    } else {
#pragma unroll
      for (int v = 0; v < NV; v++) U[v] = a.U[((size_t)v * a.nS + q) * a.L + e];
      det = a.detJ[(size_t)q * a.L + e];
    }
    for (int nn = 0; nn < a.nN; nn++) {
      const double sh = a.shape[(size_t)q * a.nN + nn];
#pragma unroll
      for (int d = 0; d < DIM; d++) x[d] += sh * a.xv[((size_t)e * a.nN + nn) * DIM + d];
    }
    calc_error<DIM, NV>(a, U, x, err);
    const double wd = a.wq[q] * det;
#pragma unroll
    for (int v = 0; v < NV; v++) {
      acc[v] = err[v] * wd;
      acc[NV + v] = U[v] * wd;
    }
  }
  block_sum<NO>(acc, part);
}

template <int DIM, int NV>
cudaError_t launch_bnd(const BndIntArgs &a, int sbytes, double *part, int nb, cudaStream_t st) {
  if (sbytes == 8) fr_boundary_integral_kernel<DIM, NV, double><<<nb, 256, 0, st>>>(a, part);
  else fr_boundary_integral_kernel<DIM, NV, float><<<nb, 256, 0, st>>>(a, part);
  return cudaGetLastError();
}

}  // namespace

int boundary_integral_blocks(int nF, int L) { return (int)(((long)nF * L + 255) / 256); }
int error_integral_blocks(int nQ, int nE) { return (int)(((long)nQ * nE + 255) / 256); }

cudaError_t launch_boundary_integral(const BndIntArgs &a, int storeBytes, double *part, cudaStream_t st) {
  const int nb = boundary_integral_blocks(a.nF, a.L);
  if (a.nDims == 2) return a.nV == 1 ? launch_bnd<2, 1>(a, storeBytes, part, nb, st)
                                     : launch_bnd<2, 4>(a, storeBytes, part, nb, st);
  return a.nV == 1 ? launch_bnd<3, 1>(a, storeBytes, part, nb, st) : launch_bnd<3, 5>(a, storeBytes, part, nb, st);
}

cudaError_t launch_error_integral(const ErrIntArgs &a, double *part, cudaStream_t st) {
  const int nb = error_integral_blocks(a.nQ, a.nE);
  if (a.nDims == 2) {
    if (a.nV == 1) fr_error_integral_kernel<2, 1><<<nb, 256, 0, st>>>(a, part);
    else fr_error_integral_kernel<2, 4><<<nb, 256, 0, st>>>(a, part);
  } else {
    if (a.nV == 1) fr_error_integral_kernel<3, 1><<<nb, 256, 0, st>>>(a, part);
    else fr_error_integral_kernel<3, 5><<<nb, 256, 0, st>>>(a, part);
  }
  return cudaGetLastError();
}

}  // namespace frg
