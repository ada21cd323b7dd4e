// dispatch.h -- host-side table of the kernels compiled for one configuration
// (dimension, order, fields, precision, boundary faces, Riemann solver).
// The instantiations live in four translation units (stage_{2d,3d}_{f64,f32}.cu)
// compiled in parallel; each also owns a copy of the 1D operator tables.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "physics.cuh"
#include "setup.h"

namespace frg {

struct KernelSet {
  void (*stage)(const void *args, int nBlk, size_t smem, cudaStream_t st) = nullptr;
  // viscous configurations: the gradient kernel launched before each stage
  void (*grad)(const void *args, int nBlk, size_t smem, cudaStream_t st) = nullptr;
  // traces of a double state: nE is the element stride of the trace array,
  // nEle the number of real elements, ldU the element stride of U
  void (*trace)(const double *U, void *tr, int nE, int nEle, int ldU, int vcjh, cudaStream_t st) = nullptr;
  void (*wavesp)(const void *tr, const double *nrmOwn, double *ws, int NF, int nE, const Phys &ph,
                 cudaStream_t st) = nullptr;
  // the fused-update stage kernel with TMA tile movement (2D inviscid), in
  // several tile shapes (elements x threads per block) for the autotuner;
  // `maps` points at a TmaMaps built for that variant's tile width
  struct TmaVariant {
    void (*launch)(const void *args, const void *maps, int nBlk, size_t smem, cudaStream_t st) = nullptr;
    int TE = 0, NT = 0;
    size_t smem = 0;
    // persistent variants: launched with (SMs x occ) blocks at most, each
    // walking tiles with a stride of the grid size
    int persistent = 0, occ = 0;
  };
  static constexpr int kMaxTma = 16;
  TmaVariant tma[kMaxTma];
  int nTma = 0;
  int TE = 0;       // elements per block
  int NT = 0;       // threads per block
  size_t smem = 0;  // dynamic shared memory per block
  // 3D viscous configurations: the fused update's two passes with TMA tile
  // movement (gradient / projected viscous flux, then the stage); `maps`
  // points at a ViscMaps built for tiles of vTE elements
  void (*vgrad)(const void *args, const void *maps, int nBlk, size_t smem, cudaStream_t st) = nullptr;
  void (*vstage)(const void *args, const void *maps, int nBlk, size_t smem, cudaStream_t st) = nullptr;
  int vTE = 0;
  int vPadG = 0;  // points per padding slot of their tiles' point layout
  // resident blocks per SM of the two passes (their grids are persistent:
  // at most SMs x this many blocks, each walking tiles)
  int vgradOcc = 0, vstageOcc = 0;
  size_t vgradSmem = 0, vstageSmem = 0;
};

struct KernelKey {
  int nDims, P, NV, precision, bc, riemann, viscous;
};

struct AdjArgs;
// The discrete-adjoint kernels of one configuration (FP64 only).
struct AdjSet {
  void (*face)(const AdjArgs &a, cudaStream_t st) = nullptr;
  void (*elem)(const AdjArgs &a, cudaStream_t st) = nullptr;
  // objectives: per-block partial sums into `part` (obj_blocks entries)
  void (*entropy)(const double *U, const double *detJ, const double *wvol, int nE, int L, const Phys &ph,
                  double *grad, double *part, cudaStream_t st) = nullptr;
  void (*wallp)(const double *U, const int *nbr, const double *dA, const double *wsurf, int vcjh, int nE, int L,
                int bcWall, const Phys &ph, double *grad, double *part, cudaStream_t st) = nullptr;
  int entropyBlocks = 0;  // partial sums written by `entropy` (grid size)
  int TE = 0;             // elements per block of `elem`
  int elemLaunches = 1;   // kernels `elem` launches (three for viscous residuals)
};
bool select_adj_2d(const KernelKey &key, AdjSet &k, std::string &err);
bool select_adj_3d(const KernelKey &key, AdjSet &k, std::string &err);
cudaError_t upload_tables_adj_2d();
cudaError_t upload_tables_adj_3d();

// Fills `k` for the key, or returns false with `err` set.
bool select_2d_f64(const KernelKey &key, KernelSet &k, std::string &err);
bool select_2d_f32(const KernelKey &key, KernelSet &k, std::string &err);
bool select_3d_f64(const KernelKey &key, KernelSet &k, std::string &err);
bool select_3d_f32(const KernelKey &key, KernelSet &k, std::string &err);

// Tensor-core operator GEMM (opgemm.cu): the operator image (hi/lo TF32
// halves as K-major core matrices), its shared-memory need, and the launch
// over a [field][K][ld] float array described by a 3D tensor map with a
// 128 x KP x 1 box.
void build_op_image(const double *op, int M, int K, int KP, int NP, std::vector<float> &img);
size_t op_gemm_smem(int KP, int NP);
cudaError_t launch_op_gemm(const CUtensorMap &mX, const float *Bimg, float *Y, int KP, int NP, int M, int ld,
                           int nEle, int nV, float beta, unsigned *err, cudaStream_t st);

// Element metrics on the device (metrics.cu), bitwise the host set-up's.
// Device arrays in the handle's layout, rows of L elements; `pos` in the
// reference layout [nS][nE][d].
struct MetricOut {
  double *pos, *detJd, *nrmOwn, *dAd, *vol;
  void *JG, *detJs, *invDetS, *nrmC, *dAs;  // stored type (storeBytes)
};
// check != 0: only tests the solution-point Jacobians, flag[0] |= 1 and
// flag[1] = min element when one is negative; else writes every metric.
// xv [nE][nN][d]; tab = shS, dS, dF of MetricTables back to back.
cudaError_t launch_metrics(int nDims, int storeBytes, const double *xv, const double *tab, const int *fdir,
                           const int *fsgn, const double *wv, const int *nbr, int nN, int nS, int nF, int nE, int L,
                           int check, const MetricOut &out, unsigned *flag, cudaStream_t st);

// Output integrals on the device (integrals.cu).  Boundary integrals of the
// current traces: kind 0 computeWallForce (6 sums: pressure, viscous), kind
// 1..3 computeMassFlux with errorNorm kind - 1 (nV sums); six partial sums per
// block (boundary_integral_blocks blocks).
struct BndIntArgs {
  int kind, nDims, nV, P, nF, nFF, nS, nE, L, viscous;
  const void *tr;     // traces [nV][nF][L], stored type
  const void *dUg;    // corrected gradient at the solution points [d][nV][nS][L] (viscous), stored type
  const int *nbr;     // [nF][L]
  const double *nrm;  // the element's own unit normal [d][nF][L]
  const double *dA;   // [nF][L]
  const double *w1;   // 1D Gauss weights [P+1] (device)
  double lag[2][6];   // 1D Lagrange basis at xi = -1 / +1
  Phys ph;
};
int boundary_integral_blocks(int nF, int L);
cudaError_t launch_boundary_integral(const BndIntArgs &a, int storeBytes, double *part, cudaStream_t st);
// integrateError: per (quadrature point, element), 2 nV partial sums per block
// (error_integral_blocks blocks): the error and the state, times weight and
// detJ.
struct ErrIntArgs {
  int nDims, nV, nS, nQ, nE, L, nN, icType, errorNorm;
  const double *U;       // [nV][nS][L]
  const double *detJ;    // [nS][L]
  const double *xv;      // [nE][nN][d] node coordinates
  const double *interp;  // [nQ][nS] solution points -> quadrature points, or null (nQ = nS)
  const double *shape;   // [nQ][nN] node shape functions at the quadrature points
  const double *wq;      // [nQ] quadrature weights
  double box[4];         // xmin, xmax, ymin, ymax of the analytic solution's period
  double time, eps;
  Phys ph;
};
int error_integral_blocks(int nQ, int nE);
cudaError_t launch_error_integral(const ErrIntArgs &a, double *part, cudaStream_t st);

// Uploads the 1D operator tables (all schemes, orders 0..5) into each unit.
cudaError_t upload_tables_2d_f64();
cudaError_t upload_tables_2d_f32();
cudaError_t upload_tables_3d_f64();
cudaError_t upload_tables_3d_f32();

}  // namespace frg
