// frgpu.cu -- the C ABI (include/frgpu.h): handle, device buffers, kernel
// dispatch over (dimension, order, fields, precision), the RK driver and its
// CUDA-graph replay.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <array>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/frgpu.h"
#include "dispatch.h"
#include "kernels.cuh"
#include "kernels_tma.cuh"
#include "kernels_visc_tma.cuh"
#include "adjoint.cuh"
#include "setup.h"

namespace frg {

// ----------------------------------------------------------------- kernels
// ele::calcDt (src/ele.cpp:1086-1105) per element, then the global minimum.
// A block covers 32 elements with 8 warps; warp w sums flux points w, w+8, ...
// of its lane's element (coalesced: a warp reads 32 consecutive elements of one
// flux point), the 8 partial sums are added in shared memory, then the minimum
// is taken with warp shuffles, per-block minima are stored and the last block
// to finish (threadfence + ticket counter) reduces them.  NaN wins the
// minimum so it is reported.
constexpr int kDtSlices = 8;
__global__ void __launch_bounds__(256) fr_dt_kernel(const double *__restrict__ waveSp, const double *__restrict__ dA,
                                                    const double *__restrict__ vol, const double *__restrict__ wsurf,
                                                    int NF, int NFF, int nE, int L, double cflFac, double *eleDt,
                                                    double *blockMin, unsigned *ticket, double *dtOut,
                                                    unsigned *err, const int *grp) {
  __shared__ double part[kDtSlices][32];
  __shared__ double wmin[32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, slice = threadIdx.x >> 5;
  const int e = blockIdx.x * 32 + lane;
  double sum = 0;
  if (e < nE)
    for (int f = slice; f < NF; f += kDtSlices) sum += waveSp[(size_t)f * L + e] * wsurf[f % NFF] * dA[(size_t)f * L + e];
  part[slice][lane] = sum;
  __syncthreads();
  if (slice == 0) {
    double my = INFINITY;
    if (e < nE) {
      double iw = 0;
      for (int k = 0; k < kDtSlices; k++) iw += part[k][lane];
      const double dte = cflFac * vol[e] / iw;  // (CFL * limit * 2) * vol / intWave
      eleDt[e] = dte;
      my = dte;
      if (grp) {  // ensemble mode: the minimum per group (dtOut preset to a huge value)
        if (!(dte > 1e-13)) atomicOr(err, ERRF_DT);
        if (dte > 0)  // a tiny dt is still used, as the reference does before its check
          atomicMin(reinterpret_cast<unsigned long long *>(dtOut + grp[e]),
                    (unsigned long long)__double_as_longlong(dte));
      }
    }
    if (grp) return;
    for (int o = 16; o > 0; o >>= 1) {
      const double t = __shfl_xor_sync(0xffffffffu, my, o);
      my = (isnan(t) || t < my) ? t : my;
    }
    if (lane == 0) {
      blockMin[blockIdx.x] = my;
      __threadfence();
      last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
  }
  __syncthreads();
  if (!last) return;
  double v = INFINITY;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
    const double t = ((volatile double *)blockMin)[b];
    v = (isnan(t) || t < v) ? t : v;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double t = __shfl_xor_sync(0xffffffffu, v, o);
    v = (isnan(t) || t < v) ? t : v;
  }
  if (lane == 0) wmin[slice] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = INFINITY;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) r = (isnan(wmin[w]) || wmin[w] < r) ? wmin[w] : r;
    *dtOut = r;
    if (isnan(r) || r < 1e-13) atomicOr(err, ERRF_DT);
    *ticket = 0;
  }
}

// Ensemble mode, once per step before the stages: each group's time advances
// by the dt its elements use this step, and the slot the last stage
// minimises the next dt into is reset.
__global__ void fr_group_step_kernel(const double *dtCur, double *dtNext, double *time, int nGrp) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nGrp) return;
  time[g] += dtCur[g];
  if (dtNext) dtNext[g] = __longlong_as_double(0x7f7f7f7f7f7f7f7fLL);
}

__global__ void fr_timestep_kernel(double *U, const double *U0, const double *divF, const double *detJ,
                                   const double *dt, int dtLocal, double coef, int modeB, int NS, int nE, int L,
                                   long total) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const long pe = i % ((long)NS * L);
  const int e = (int)(pe % L);
  if (e >= nE) return;
  const double dtl = dtLocal ? dt[e] : dt[0];
  if (modeB) U[i] -= coef * divF[i] / detJ[pe] * dtl;
  else U[i] = U0[i] - coef * divF[i] / detJ[pe] * dtl;
}

__global__ void fr_norm_kernel(const double *divF, const double *detJ, const double *wvol, int NV, int NS, int nE,
                               int L, int normType, double *partial, unsigned *ticket, double *out) {
  // one thread per element: its per-field norm (spt order as the reference),
  // then per-block totals over elements in index order
  extern __shared__ double sh[];  // [blockDim][NV]
  __shared__ bool last;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  for (int v = 0; v < NV; v++) {
    double r = 0;
    if (e < nE)
      for (int s = 0; s < NS; s++) {
        double dv = divF[((size_t)v * NS + s) * L + e], dj = detJ[(size_t)s * L + e];
        if (normType == 1) r += fabs(dv) * wvol[s];
        else if (normType == 2) r += dv * dv / dj * wvol[s];
        else r = fmax(fabs(dv) / dj, r);
      }
    sh[threadIdx.x * NV + v] = r;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int v = 0; v < NV; v++) {
      double t = 0;
      for (int i = 0; i < (int)blockDim.x; i++)
        t = normType == 3 ? fmax(t, sh[i * NV + v]) : t + sh[i * NV + v];
      partial[(size_t)blockIdx.x * NV + v] = t;
    }
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  for (int v = 0; v < NV; v++) {
    double t = 0;
    for (int b = 0; b < (int)gridDim.x; b++) {
      double x = ((volatile double *)partial)[(size_t)b * NV + v];
      t = normType == 3 ? fmax(t, x) : t + x;
    }
    out[v] = t;
  }
  *ticket = 0;
}

__global__ void fr_to_device_layout(const double *ref, double *dev, int NV, int NPT, int nE, int L) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;  // ref index
  const long total = (long)NV * NPT * nE;
  if (i >= total) return;
  const int v = (int)(i % NV);
  const long pe = i / NV;  // pt * nE + e
  const long pt = pe / nE, e = pe - pt * nE;
  dev[((long)v * NPT + pt) * L + e] = ref[i];
}
__global__ void fr_to_ref_layout(const double *dev, double *ref, int NV, int NPT, int nE, int L) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;  // ref index
  const long total = (long)NV * NPT * nE;
  if (i >= total) return;
  const int v = (int)(i % NV);
  const long pe = i / NV;
  const long pt = pe / nE, e = pe - pt * nE;
  ref[i] = dev[((long)v * NPT + pt) * L + e];
}
template <typename S>
__global__ void fr_cast_kernel(const double *in, S *out, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (S)in[i];
}

bool select_kernels(const KernelKey &key, KernelSet &k, std::string &err) {
  if (key.nDims == 2) return key.precision == FRG_FP64 ? select_2d_f64(key, k, err) : select_2d_f32(key, k, err);
  if (key.nDims == 3) return key.precision == FRG_FP64 ? select_3d_f64(key, k, err) : select_3d_f32(key, k, err);
  err = "unsupported dimension";
  return false;
}

}  // namespace frg

using namespace frg;

struct AdjState;  // discrete-adjoint buffers (end of this file)
void adj_free(frg_solver *s);
void adj_forget_graphs(frg_solver *s);

// -------------------------------------------------------------- the handle
struct frg_solver {
  frg_params p{};
  HostGeom g;
  Ops1D ops;
  KernelSet ks;
  int nV = 0, nS = 0, nF = 0, nE = 0, nBlk = 0, nRK = 0;
  int L = 0;  // element stride of device arrays: nE rounded up to a multiple of 32
  size_t sstore = 8;  // bytes of the stored type
  std::vector<double> RKa, RKb;
  cudaStream_t stream = nullptr, ownStream = nullptr;
  // device buffers
  double *U = nullptr, *U0 = nullptr, *Acc = nullptr, *divF[5] = {nullptr};
  void *W[2] = {nullptr, nullptr}, *tr[2] = {nullptr, nullptr};
  void *nrm = nullptr, *dAs = nullptr, *JG = nullptr, *detJs = nullptr;
  void *invDetS = nullptr;  // 1 / detJ in the stored type, for the TMA stage kernel
  void *fvn = nullptr, *fvn2 = nullptr;  // viscous: projected viscous flux per flux point
  void *dUg = nullptr;                   // viscous: corrected gradient at the solution points
  bool visc2 = false;                    // 3D with an LDG penalty: second projection needed
  double *detJd = nullptr, *nrmOwn = nullptr, *dAd = nullptr, *vol = nullptr, *wsurf = nullptr, *wvol = nullptr;
  int *nbr = nullptr;
  double *waveSp = nullptr, *eleDt = nullptr, *dtDev = nullptr, *timeDev = nullptr, *blockMin = nullptr;
  // ensemble mode (frg_set_groups): independent cases in one mesh, each
  // with its own dt (two slots of nGrp) and time
  int *grp = nullptr;
  int nGrp = 0;
  double *grpDt = nullptr, *grpTime = nullptr;
  int dtCur = 0;  // slot of dtDev[2] holding the current step's dt (two slots
                  // when the last stage computes the next step's dt)
  int dtLast = 0;  // slot of the dt the last step used or frg_calc_dt computed
  double *normPartial = nullptr, *normOut = nullptr, *scratchRef = nullptr;
  unsigned *err = nullptr, *ticket = nullptr;
  unsigned *hostFlag = nullptr;  // pinned host copy of the flag word (frg_update_host)
  int curTr = 0;
  bool trValid = false, divF0Valid = false, monitor = false;
  int iter = 0, initIter = 0;
  long long launches = 0;
  // captured steps, [dt mode][trace buffer][dt slot]: dt mode 0 = the previous
  // step's last stage already computed dt, 1 = dt kernel first, 2 = wave
  // speeds + dt first
  cudaGraphExec_t graph[3][2][2] = {};
  cudaGraph_t graphRaw[3][2][2] = {};  // the captured graphs (child nodes of an ensemble step)
  unsigned graphEpoch = 0;             // bumped whenever the captured graphs are dropped
  bool dtFresh = false;  // device dt was computed from the current wave speeds
  // tensor maps of the TMA stage kernel
  bool useTma = false;
  bool pdl = true;  // programmatic dependent launch between TMA stages (FRG_PDL=0: off)
  bool useGraph = true;  // steps replayed from captured graphs (FRG_GRAPH=0: launched directly)
  int nSM = 0;      // multiprocessors of the device (persistent grids)
  int tmaVar = 0;  // tile-shape variant of the TMA kernel (frg_autotune)
  int nBlkTma = 0;
  CUtensorMap mU, mAcc, mW[2], mTr[2], mJG, mDet, mNrm, mDA, mNbr;
  // tensor maps of the 3D viscous TMA passes (tiles of ks.vTE elements):
  // stage inputs W[i] in the padded point layout, and the rest
  bool useViscTma = false;
  struct {
    CUtensorMap Win[2], U, Acc, Wout[2], tr[2], JG, det, nrm, dA, nbr, fvn, fvn2;
  } vm;
  AdjState *adj = nullptr;
  // frg_apply_operator: operator images for the tensor-core GEMM, [which][dim]
  float *opImg[5][3] = {};
  // frg_update_geometry: node count, device copies of the nodes and of the
  // shape tables, the check flags and the solution-point positions
  int nNodes = 0;
  std::vector<double> xvHost;  // the current node coordinates (ParaView output)
  double *xvDev = nullptr, *geoTab = nullptr, *posDev = nullptr;
  int *geoInt = nullptr;
  unsigned *geoFlag = nullptr;
  bool waveStale = false;  // metrics changed: the next dt recomputes the wave speeds
  // frg_calc_residual_noalloc on a caller's stream: recorded on the handle's
  // stream so the caller's stream waits for pending uploads / geometry work
  cudaEvent_t noallocOrder = nullptr;
  // output integrals (frg_wall_force, frg_mass_flux, frg_integrate_error):
  // per-block partial sums, the 1D Gauss weights and the quadrature tables
  // of the last quadOrder used
  double *intPart = nullptr, *w1Dev = nullptr, *qShape = nullptr, *qInterp = nullptr, *qW = nullptr;
  size_t intPartCap = 0;
  int qOrder = -2;  // quadOrder of the cached tables (-1: the solution points)
};

namespace {
thread_local std::string g_err;

// getCFLLimit (src/global.cpp:45-66)
const double kCflLimit[6] = {1.393, 0.464, 0.235, 0.1453, 0.100, 0.0736};

frg_status fail(frg_status st, const char *fmt, ...);
}  // namespace
namespace frg {
// error reporting for the host-only units (restart.cpp)
frg_status set_error(frg_status st, const std::string &msg) { return fail(st, "%s", msg.c_str()); }
}  // namespace frg
namespace {
frg_status fail(frg_status st, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return st;
}
#define CK(x)                                                                                    \
  do {                                                                                           \
    cudaError_t e_ = (x);                                                                        \
    if (e_ != cudaSuccess) return fail(FRG_ERR_CUDA, "%s: %s (%s:%d)", #x, cudaGetErrorString(e_), \
                                       __FILE__, __LINE__);                                      \
  } while (0)

// Each kernel unit holds its own copy of the 1D operator tables.
bool g_tables[2][2] = {{false, false}, {false, false}};
frg_status upload_tables(int nDims, int prec) {
  bool &done = g_tables[nDims - 2][prec != FRG_FP64];
  if (done) return FRG_OK;
  cudaError_t e = nDims == 2 ? (prec == FRG_FP64 ? upload_tables_2d_f64() : upload_tables_2d_f32())
                             : (prec == FRG_FP64 ? upload_tables_3d_f64() : upload_tables_3d_f32());
  if (e != cudaSuccess) return fail(FRG_ERR_CUDA, "operator tables: %s", cudaGetErrorString(e));
  done = true;
  return FRG_OK;
}

Phys make_phys(const frg_params &p) {
  Phys ph{};
  ph.gamma = p.gamma;
  ph.adv[0] = p.advectVx; ph.adv[1] = p.advectVy; ph.adv[2] = p.advectVz;
  ph.lambda = p.lambda;
  ph.diffD = p.diffD;
  ph.rhoB = p.rhoBound; ph.vB[0] = p.uBound; ph.vB[1] = p.vBound; ph.vB[2] = p.wBound; ph.pB = p.pBound;
  ph.mu = p.mu_inf; ph.prandtl = p.prandtl; ph.c_sth = p.c_sth; ph.rt_inf = p.rt_inf;
  ph.penFact = p.penFact; ph.tau = p.tau;
  ph.TWall = p.TWall; ph.RGas = p.RGas; ph.vWall[0] = p.uWall; ph.vWall[1] = p.vWall; ph.vWall[2] = p.wWall;
  ph.fixVis = p.fixVis;
  ph.riemann = p.riemannType;
  return ph;
}

template <typename T>
frg_status dalloc(T **ptr, size_t count) {
  CK(cudaMalloc((void **)ptr, count * sizeof(T) + 16));
  CK(cudaMemset(*ptr, 0, count * sizeof(T) + 16));
  return FRG_OK;
}
frg_status dalloc_bytes(void **ptr, size_t bytes) {
  CK(cudaMalloc(ptr, bytes + 16));
  CK(cudaMemset(*ptr, 0, bytes + 16));
  return FRG_OK;
}
// copy a double host array to device in the stored precision
frg_status upload_store(frg_solver *s, void **dst, const std::vector<double> &src) {
  frg_status st = dalloc_bytes(dst, src.size() * s->sstore);
  if (st) return st;
  if (s->sstore == 8) {
    CK(cudaMemcpy(*dst, src.data(), src.size() * 8, cudaMemcpyHostToDevice));
  } else {
    std::vector<float> f(src.begin(), src.end());
    CK(cudaMemcpy(*dst, f.data(), f.size() * 4, cudaMemcpyHostToDevice));
  }
  return FRG_OK;
}
// Rows of nE values (element fastest) widened to the padded stride L.
std::vector<double> pad_rows(const std::vector<double> &src, int nE, int L, double fill) {
  const size_t rows = src.size() / nE;
  std::vector<double> out(rows * L, fill);
  for (size_t r = 0; r < rows; r++) std::memcpy(&out[r * L], &src[r * nE], nE * sizeof(double));
  return out;
}

frg_status upload_d(double **dst, const std::vector<double> &src) {
  frg_status st = dalloc(dst, src.size());
  if (st) return st;
  CK(cudaMemcpy(*dst, src.data(), src.size() * 8, cudaMemcpyHostToDevice));
  return FRG_OK;
}

frg_status post_launch(frg_solver *s) {
  s->launches++;
  CK(cudaGetLastError());
  return FRG_OK;
}

frg_status ensure_traces(frg_solver *s) {
  if (s->trValid) return FRG_OK;
  s->ks.trace(s->U, s->tr[s->curTr], s->L, s->nE, s->L, s->p.vcjhScheme, s->stream);
  frg_status st = post_launch(s);
  if (st) return st;
  s->trValid = true;
  return FRG_OK;
}

// dt slot `slot` (0/1): a scalar, or one value per group in ensemble mode
double *dt_slot(frg_solver *s, int slot) {
  return s->grp ? s->grpDt + (size_t)slot * s->nGrp : s->dtDev + slot;
}

StageArgs base_args(frg_solver *s) {
  StageArgs a{};
  a.nE = s->L;
  a.nEle = s->nE;
  a.ldU = s->L;
  a.nbr = s->nbr;
  a.nrm = s->nrm;
  a.dA = s->dAs;
  a.JG = s->JG;
  a.detJ = s->detJs;
  a.waveSp = s->waveSp;
  a.dt = s->p.dtType == 2 ? s->eleDt : dt_slot(s, s->dtCur);
  a.grp = s->grp;
  a.dtLocal = s->p.dtType == 2;
  a.time = s->timeDev;
  a.err = s->err;
  a.vcjh = s->p.vcjhScheme;
  a.ph = make_phys(s->p);
  a.fvnOut = s->fvn;
  a.fvnIn = s->fvn;
  a.fvn2Out = s->fvn2;
  a.fvn2In = s->fvn2;
  a.visc2 = s->visc2;
  a.vol = s->vol;
  a.dAd = s->dAd;
  a.wsurf = s->wsurf;
  a.blockMin = s->blockMin;
  a.dtNext = dt_slot(s, s->dtCur ^ 1);
  a.eleDt = s->eleDt;
  a.ticket = s->ticket;
  a.cflFac = s->p.CFL * kCflLimit[s->p.order] * 2;
  a.nff = s->g.nFF;
  set_stage_ops(a, s->ops);
  return a;
}

// cuTensorMapEncodeTiled, fetched from the driver through the runtime (no
// libcuda link dependency).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// 2D tensor map over rows x L elements (row stride L), box TE x rows.
frg_status make_map(CUtensorMap *m, void *base, CUtensorMapDataType dt, int esz, int rows, int L, int TE) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return fail(FRG_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  if (rows > 256 || ((size_t)TE * esz) % 16 || ((size_t)L * esz) % 16 || ((uintptr_t)base & 15))
    return fail(FRG_ERR_ARG, "tensor map shape not TMA-compatible");
  cuuint64_t dims[2] = {(cuuint64_t)L, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)L * esz};
  cuuint32_t box[2] = {(cuuint32_t)TE, (cuuint32_t)rows};
  cuuint32_t es[2] = {1, 1};
  CUresult r = enc(m, dt, 2, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(FRG_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return FRG_OK;
}

// Tensor map of `rank` dimensions: dims in elements (innermost first),
// strides in bytes of dimensions 1..rank-1, box extents.
frg_status make_map_nd(CUtensorMap *m, void *base, CUtensorMapDataType dt, int esz, int rank, const cuuint64_t *dims,
                       const cuuint64_t *strides, const cuuint32_t *box) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return fail(FRG_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  if (((size_t)box[0] * esz) % 16 || ((uintptr_t)base & 15)) return fail(FRG_ERR_ARG, "tensor map not TMA-compatible");
  for (int i = 0; i < rank; i++)
    if (box[i] < 1 || box[i] > 256) return fail(FRG_ERR_ARG, "tensor map box extent out of range");
  for (int i = 0; i < rank - 1; i++)
    if (strides[i] % 16) return fail(FRG_ERR_ARG, "tensor map stride not a multiple of 16 bytes");
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  CUresult r = enc(m, dt, (cuuint32_t)rank, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(FRG_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return FRG_OK;
}

// Maps of the 3D viscous TMA passes (kernels_visc_tma.cuh, ViscMaps).
frg_status setup_visc_tma(frg_solver *s) {
  const int TE = s->ks.vTE, d = s->p.nDims, n1 = s->p.order + 1, nS = s->nS, nF = s->nF, nV = s->nV;
  const cuuint64_t L = (cuuint64_t)s->L;
  const int es = (int)s->sstore;
  const CUtensorMapDataType ts = es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const cuuint32_t te = (cuuint32_t)TE;
  auto map3 = [&](CUtensorMap *m, void *base, CUtensorMapDataType dt, int esz, int rows, int planes) {
    const cuuint64_t dims[3] = {L, (cuuint64_t)rows, (cuuint64_t)planes};
    const cuuint64_t str[2] = {L * esz, L * esz * rows};
    const cuuint32_t box[3] = {te, (cuuint32_t)rows, (cuuint32_t)planes};
    return make_map_nd(m, base, dt, esz, 3, dims, str, box);
  };
  auto map2 = [&](CUtensorMap *m, void *base, CUtensorMapDataType dt, int esz, int rows) {
    const cuuint64_t dims[2] = {L, (cuuint64_t)rows};
    const cuuint64_t str[1] = {L * esz};
    const cuuint32_t box[2] = {te, (cuuint32_t)rows};
    return make_map_nd(m, base, dt, esz, 2, dims, str, box);
  };
  // stage input in the padded point layout: each group of pg points walked
  // with a box one point wider (the extra point is outside the tensor: zeros)
  const int pg = s->ks.vPadG;
  (void)n1;
  auto map_padded = [&](CUtensorMap *m, void *base) {
    const cuuint64_t dims[4] = {L, (cuuint64_t)pg, (cuuint64_t)(nS / pg), (cuuint64_t)nV};
    const cuuint64_t str[3] = {L * es, L * es * pg, L * es * nS};
    const cuuint32_t box[4] = {te, (cuuint32_t)(pg + 1), (cuuint32_t)(nS / pg), (cuuint32_t)nV};
    return make_map_nd(m, base, ts, es, 4, dims, str, box);
  };
  const CUtensorMapDataType f64 = CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  frg_status st;
  if ((st = map_padded(&s->vm.Win[0], s->W[0])) || (st = map_padded(&s->vm.Win[1], s->W[1])) ||
      (st = map3(&s->vm.U, s->U, f64, 8, nS, nV)) || (st = map3(&s->vm.Acc, s->Acc, f64, 8, nS, nV)) ||
      (st = map3(&s->vm.Wout[0], s->W[0], ts, es, nS, nV)) || (st = map3(&s->vm.Wout[1], s->W[1], ts, es, nS, nV)) ||
      (st = map3(&s->vm.tr[0], s->tr[0], ts, es, nF, nV)) || (st = map3(&s->vm.tr[1], s->tr[1], ts, es, nF, nV)) ||
      (st = map3(&s->vm.JG, s->JG, ts, es, nS, d * d)) || (st = map2(&s->vm.det, s->invDetS, ts, es, nS)) ||
      (st = map3(&s->vm.nrm, s->nrm, ts, es, nF, d)) || (st = map2(&s->vm.dA, s->dAs, ts, es, nF)) ||
      (st = map3(&s->vm.fvn, s->fvn, ts, es, nF, nV)) ||
      (st = map3(&s->vm.fvn2, s->visc2 ? s->fvn2 : s->fvn, ts, es, nF, nV)))
    return st;
  if (TE * 4 >= 16) {
    if ((st = map2(&s->vm.nbr, s->nbr, CU_TENSOR_MAP_DATA_TYPE_INT32, 4, nF))) return st;
  } else {
    s->vm.nbr = s->vm.det;  // codes read by plain loads; the map is not used
  }
  return FRG_OK;
}

frg_status setup_tma(frg_solver *s) {
  const int TE = s->ks.tma[s->tmaVar].TE, L = s->L, d = s->p.nDims;
  const CUtensorMapDataType ts = s->sstore == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const int es = (int)s->sstore, nvs = s->nV * s->nS, nvf = s->nV * s->nF;
  frg_status st;
  if ((st = make_map(&s->mU, s->U, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, nvs, L, TE)) ||
      (st = make_map(&s->mAcc, s->Acc, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, nvs, L, TE)) ||
      (st = make_map(&s->mW[0], s->W[0], ts, es, nvs, L, TE)) || (st = make_map(&s->mW[1], s->W[1], ts, es, nvs, L, TE)) ||
      (st = make_map(&s->mTr[0], s->tr[0], ts, es, nvf, L, TE)) ||
      (st = make_map(&s->mTr[1], s->tr[1], ts, es, nvf, L, TE)) ||
      (st = make_map(&s->mJG, s->JG, ts, es, d * d * s->nS, L, TE)) ||
      (st = make_map(&s->mDet, s->invDetS, ts, es, s->nS, L, TE)) ||
      (st = make_map(&s->mNrm, s->nrm, ts, es, d * s->nF, L, TE)) ||
      (st = make_map(&s->mDA, s->dAs, ts, es, s->nF, L, TE)) ||
      (st = make_map(&s->mNbr, s->nbr, CU_TENSOR_MAP_DATA_TYPE_INT32, 4, s->nF, L, TE)))
    return st;
  const KernelSet::TmaVariant &tv = s->ks.tma[s->tmaVar];
  if (tv.persistent) {
    int dev = 0, nSM = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nSM, cudaDevAttrMultiProcessorCount, dev));
    const int nTiles = (s->nE + TE - 1) / TE;
    s->nBlkTma = std::min(nTiles, nSM * tv.occ);
  } else {
    s->nBlkTma = L / TE;
  }
  return FRG_OK;
}

frg_status launch_stage_args(frg_solver *s, StageArgs &a) {
  if (s->ks.grad) {  // viscous: the gradient kernel first (same inputs)
    s->ks.grad(&a, s->nBlk, s->ks.smem, s->stream);
    frg_status st = post_launch(s);
    if (st) return st;
  }
  s->ks.stage(&a, s->nBlk, s->ks.smem, s->stream);
  return post_launch(s);
}


frg_status launch_dt(frg_solver *s) {
  int nb = (s->nE + 31) / 32;
  double fac = s->p.CFL * kCflLimit[s->p.order] * 2;
  if (s->grp) CK(cudaMemsetAsync(dt_slot(s, s->dtCur), 0x7F, (size_t)s->nGrp * 8, s->stream));
  fr_dt_kernel<<<nb, 256, 0, s->stream>>>(s->waveSp, s->dAd, s->vol, s->wsurf, s->nF, s->g.nFF, s->nE, s->L, fac,
                                           s->eleDt, s->blockMin, s->ticket, dt_slot(s, s->dtCur), s->err, s->grp);
  s->dtLast = s->dtCur;
  return post_launch(s);
}

frg_status launch_wavesp(frg_solver *s) {
  s->ks.wavesp(s->tr[s->curTr], s->nrmOwn, s->waveSp, s->nF, s->L, make_phys(s->p), s->stream);
  return post_launch(s);
}

void drop_graphs(frg_solver *s) {
  adj_forget_graphs(s);
  for (auto &r : s->graph)
    for (auto &q : r)
      for (auto &g : q)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  for (auto &r : s->graphRaw)
    for (auto &q : r)
      for (auto &g : q)
        if (g) { cudaGraphDestroy(g); g = nullptr; }
  s->graphEpoch++;
}

// The last stage of the TMA kernel computes the next step's global CFL dt.
bool fused_dt(const frg_solver *s) { return s->useTma && s->p.dtType == 1; }

frg_status launch_group_step(frg_solver *s) {
  fr_group_step_kernel<<<(s->nGrp + 127) / 128, 128, 0, s->stream>>>(
      dt_slot(s, s->dtCur), fused_dt(s) ? dt_slot(s, s->dtCur ^ 1) : nullptr, s->grpTime, s->nGrp);
  return post_launch(s);
}

// dt work at the start of the next fused step (see frg_solver::graph).
int dt_mode(const frg_solver *s) {
  if (s->p.dtType == 0) return 0;
  if (s->iter == s->initIter + 1 || s->waveStale) return 2;
  return (fused_dt(s) && s->dtFresh) ? 0 : 1;
}

// One fused step (the body of solver::update) on the stream.  With `ev`
// (2 + nRK events) an event is recorded before the dt kernels and after each
// launch, for frg_time_stages.  With the TMA kernel the last stage computes
// the next step's dt (calcDt reads the wave speeds the last stage leaves).
frg_status enqueue_step(frg_solver *s, int mode, cudaEvent_t *ev = nullptr) {
  frg_status st;
  if (ev) CK(cudaEventRecord(ev[0], s->stream));
  if (s->p.dtType != 0) {
    if (mode == 2 && (st = launch_wavesp(s))) return st;
    if (mode >= 1 && (st = launch_dt(s))) return st;
    // the slot the last stage will minimise into: reset by the first stage
    // (a memset only when one stage is also the last)
    if (fused_dt(s) && !s->grp && s->nRK == 1)
      CK(cudaMemsetAsync(s->dtDev + (s->dtCur ^ 1), 0x7F, sizeof(double), s->stream));
  }
  if (s->grp && (st = launch_group_step(s))) return st;
  if (ev) CK(cudaEventRecord(ev[1], s->stream));
  const int nRK = s->nRK;
  const bool jam = s->p.timeType == 5;
  double *const dtReset = (fused_dt(s) && !s->grp && nRK > 1) ? s->dtDev + (s->dtCur ^ 1) : nullptr;
  for (int k = 0; k < nRK; k++) {
    StageArgs a = base_args(s);
    const bool first = k == 0, last = k == nRK - 1;
    a.Uin_d = first ? s->U : nullptr;
    a.Uin_s = first ? nullptr : s->W[(k - 1) & 1];
    a.U0 = s->U;
    a.Acc = s->Acc;
    a.Uout = s->U;
    a.Wout = s->W[k & 1];
    a.trIn = s->tr[s->curTr];
    a.trOut = s->tr[s->curTr ^ 1];
    a.aNext = jam ? s->RKa[k + 1] : (last ? 0.0 : s->RKa[k + 1]);
    a.bCur = jam ? 0.0 : s->RKb[k];
    a.flags = (last ? SF_WAVESP | SF_LAST | SF_TIME : 0) | (first ? SF_FIRST : 0) | (jam ? SF_JAMESON : 0);
    a.dUg = s->dUg;
    if (first && s->monitor) {
      a.flags |= SF_DIVF;
      a.divF = s->divF[0];
    }
    if (last && fused_dt(s)) a.flags |= SF_DTNEXT;
    if (first) a.dtReset = dtReset;
    // stages after the first follow a stage kernel directly: programmatic
    // dependent launch (not when each launch is timed on its own)
    if (k > 0 && s->pdl && !ev) a.flags |= SF_PDL;
    if (s->useViscTma) {
      ViscMaps vm;
      vm.Uin = first ? s->vm.U : s->vm.Win[(k - 1) & 1];
      vm.U = s->vm.U;
      vm.Acc = s->vm.Acc;
      vm.Wout = s->vm.Wout[k & 1];
      vm.trOut = s->vm.tr[s->curTr ^ 1];
      vm.trIn = s->vm.tr[s->curTr];
      vm.JG = s->vm.JG;
      vm.det = s->vm.det;
      vm.nrm = s->vm.nrm;
      vm.dA = s->vm.dA;
      vm.nbr = s->vm.nbr;
      vm.fvn = s->vm.fvn;
      vm.fvn2 = s->vm.fvn2;
      const int nTiles = (s->nE + s->ks.vTE - 1) / s->ks.vTE;
      // the gradient pass one tile per block (measured faster than its
      // persistent form, which gains nothing from the L2 prefetch), the
      // stage pass persistent
      s->ks.vgrad(&a, &vm, nTiles, s->ks.vgradSmem, s->stream);
      if ((st = post_launch(s))) return st;
      s->ks.vstage(&a, &vm, std::min(nTiles, s->nSM * s->ks.vstageOcc), s->ks.vstageSmem, s->stream);
      st = post_launch(s);
    } else if (s->useTma) {
      TmaMaps mm;
      mm.U = s->mU;
      mm.Acc = s->mAcc;
      mm.Win = s->mW[k > 0 ? (k - 1) & 1 : 0];
      mm.Wout = s->mW[k & 1];
      mm.trOut = s->mTr[s->curTr ^ 1];
      mm.trIn = s->mTr[s->curTr];
      mm.JG = s->mJG;
      mm.det = s->mDet;
      mm.nrm = s->mNrm;
      mm.dA = s->mDA;
      mm.nbr = s->mNbr;
      const KernelSet::TmaVariant &tv = s->ks.tma[s->tmaVar];
      tv.launch(&a, &mm, s->nBlkTma, tv.smem, s->stream);
      st = post_launch(s);
    } else {
      st = launch_stage_args(s, a);
    }
    if (st) return st;
    if (ev) CK(cudaEventRecord(ev[2 + k], s->stream));
    s->curTr ^= 1;
  }
  return FRG_OK;
}

// The status of a flag word read back from the device (clears the device's).
frg_status flags_status(frg_solver *s, unsigned h) {
  if (h) {
    CK(cudaMemsetAsync(s->err, 0, sizeof(unsigned), s->stream));
    // writeResidual's order: the dt check first (src/output.cpp:823-824), then NaN
    if (h & ERRF_DT) return fail(FRG_ERR_DT, "Instability detected - dt approaching zero");
    if (h & ERRF_NAN) return fail(FRG_ERR_NAN, "NaN encountered in the solution");
    if (h & ERRF_BC) return fail(FRG_ERR_ARG, "Boundary condition not recognized");
    if (h & ERRF_ALIGN) return fail(FRG_ERR_CUDA, "operator GEMM: dynamic shared memory not 1024-byte aligned");
    if (h & ERRF_TIMEOUT) return fail(FRG_ERR_TIMEOUT, "a bounded device wait gave up");
  }
  return FRG_OK;
}

frg_status check_flags(frg_solver *s) {
  unsigned h = 0;
  CK(cudaMemcpyAsync(&h, s->err, sizeof h, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return flags_status(s, h);
}

frg_status unfused_update(frg_solver *s);

}  // namespace

// Device address of the allocation-free residual's scratch array on the
// current device (defined next to the array, below).
static frg_status noalloc_scratch_addr(void **out);

// ==================================================================== C ABI
extern "C" {

const char *frg_last_error(void) { return g_err.c_str(); }
const char *frg_version(void) { return "frgpu 0.1 sm_100a"; }

frg_status frg_create(const frg_params *params, const frg_mesh *mesh, frg_solver **out) {
  if (!params || !mesh || !out || !mesh->xv || !mesh->c2v) return fail(FRG_ERR_ARG, "null argument");
  *out = nullptr;
  const frg_params &p = *params;
  if (p.nDims != 2 && p.nDims != 3) return fail(FRG_ERR_ARG, "nDims must be 2 or 3");
  if (p.order < 1 || p.order > (p.nDims == 2 ? 5 : 4)) return fail(FRG_ERR_ARG, "order %d not supported", p.order);
  if (p.equation != 0 && p.equation != 1) return fail(FRG_ERR_ARG, "equation must be 0 or 1");
  if (p.equation == 1 && p.riemannType == 1 && p.nDims == 3)
    return fail(FRG_ERR_ARG, "Roe not implemented in 3D");
  if (p.vcjhScheme < 0 || p.vcjhScheme > 3 || (p.vcjhScheme == 3 && p.order < 2))
    return fail(FRG_ERR_ARG, "invalid VCJH scheme");
  if (p.precision != FRG_FP64 && p.precision != FRG_MIXED) return fail(FRG_ERR_ARG, "invalid precision");
  if (p.dtType < 0 || p.dtType > 2) return fail(FRG_ERR_ARG, "invalid dtType");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(FRG_ERR_CUDA, "no CUDA device");
  std::unique_ptr<frg_solver> s(new frg_solver());
  s->p = p;
  s->nV = p.equation == 0 ? 1 : p.nDims + 2;
  switch (p.timeType) {
    case 0: s->nRK = 1; s->RKa = {0}; s->RKb = {1}; break;
    case 2: s->nRK = 2; s->RKa = {0, 1.}; s->RKb = {1. / 2., 1. / 2.}; break;
    case 4: s->nRK = 4; s->RKa = {0., .5, .5, 1.}; s->RKb = {1. / 6., 1. / 3., 1. / 3., 1. / 6.}; break;
    case 5: s->nRK = 4; s->RKa = {0., 1. / 4., 1. / 3., 1. / 2., 1.0}; s->RKb = {0.}; break;
    default: return fail(FRG_ERR_ARG, "Time-Stepping type not supported.");
  }
  std::string err;
  frg_status st = build_geometry(p, *mesh, s->g, err);
  if (st) return fail(st, "%s", err.c_str());
  s->ops = build_ops1d(p.order, p.vcjhScheme);
  s->nNodes = mesh->nNodes;
  s->xvHost.assign(mesh->xv, mesh->xv + (size_t)mesh->nEles * mesh->nNodes * p.nDims);
  s->nS = s->g.nS; s->nF = s->g.nF; s->nE = s->g.nE;
  s->L = (s->nE + 31) & ~31;
  if ((st = upload_tables(p.nDims, p.precision))) return st;
  KernelKey key{p.nDims, p.order, s->nV, p.precision, s->g.nBndFaces > 0 ? 1 : 0, p.riemannType, p.viscous ? 1 : 0};
  if (!select_kernels(key, s->ks, err)) return fail(FRG_ERR_ARG, "%s", err.c_str());
  s->sstore = p.precision == FRG_FP64 ? 8 : 4;
  s->nBlk = (s->nE + s->ks.TE - 1) / s->ks.TE;
  CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  const size_t nSE = (size_t)s->nV * s->nS * s->L, nFE = (size_t)s->nV * s->nF * s->L;
  if ((st = dalloc(&s->U, nSE)) || (st = dalloc(&s->U0, nSE)) || (st = dalloc(&s->Acc, nSE))) return st;
  for (int i = 0; i < 2; i++) {
    if ((st = dalloc_bytes(&s->W[i], nSE * s->sstore))) return st;
    if ((st = dalloc_bytes(&s->tr[i], nFE * s->sstore))) return st;
  }
  if (p.viscous) {
    s->visc2 = p.nDims == 3 && p.penFact != 0.0;
    if ((st = dalloc_bytes(&s->fvn, nFE * s->sstore))) return st;
    if (s->visc2 && (st = dalloc_bytes(&s->fvn2, nFE * s->sstore))) return st;
    if ((st = dalloc_bytes(&s->dUg, (size_t)p.nDims * nSE * s->sstore))) return st;
  }
  const int nE = s->nE, L = s->L;
  if ((st = upload_store(s.get(), &s->nrm, pad_rows(s->g.nrmC, nE, L, 0.0))) ||
      (st = upload_store(s.get(), &s->dAs, pad_rows(s->g.dA, nE, L, 0.0))) ||
      (st = upload_store(s.get(), &s->JG, pad_rows(s->g.JG, nE, L, 0.0))) ||
      (st = upload_store(s.get(), &s->detJs, pad_rows(s->g.detJ, nE, L, 1.0))))
    return st;
  {
    std::vector<double> inv = pad_rows(s->g.detJ, nE, L, 1.0);
    for (double &x : inv) x = 1.0 / x;
    if ((st = upload_store(s.get(), &s->invDetS, inv))) return st;
  }
  if ((st = upload_d(&s->detJd, pad_rows(s->g.detJ, nE, L, 1.0))) ||
      (st = upload_d(&s->nrmOwn, pad_rows(s->g.nrmOwn, nE, L, 0.0))) ||
      (st = upload_d(&s->dAd, pad_rows(s->g.dA, nE, L, 0.0))) || (st = upload_d(&s->vol, pad_rows(s->g.vol, nE, L, 1.0))))
    return st;
  {
    std::vector<double> ws(s->g.nFF), wv(s->nS);
    const int n1 = p.order + 1;
    for (int k = 0; k < s->g.nFF; k++) ws[k] = p.nDims == 2 ? s->ops.w[k] : s->ops.w[k / n1] * s->ops.w[k % n1];
    for (int q = 0; q < s->nS; q++) {
      int i = q % n1, j = (q / n1) % n1, k = q / (n1 * n1);
      wv[q] = p.nDims == 2 ? s->ops.w[j] * s->ops.w[i] : s->ops.w[k] * s->ops.w[j] * s->ops.w[i];
    }
    if ((st = upload_d(&s->wsurf, ws)) || (st = upload_d(&s->wvol, wv))) return st;
  }
  {
    // neighbour codes with trace indices re-based on the padded stride
    std::vector<int> nb((size_t)s->nF * L, 0);
    for (int f = 0; f < s->nF; f++)
      for (int e = 0; e < nE; e++) {
        int c = s->g.nbr[(size_t)f * nE + e];
        if (c >= 0) {
          long t = c >> 1, fo = t / nE, eo = t - fo * nE, tp = fo * L + eo;
          if (tp >= (1L << 30)) return fail(FRG_ERR_ARG, "mesh too large for 30-bit trace index");
          c = (int)((tp << 1) | (c & 1));
        }
        nb[(size_t)f * L + e] = c;
      }
    CK(cudaMalloc(&s->nbr, nb.size() * sizeof(int)));
    CK(cudaMemcpy(s->nbr, nb.data(), nb.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  const int nbDt = (s->nE + 31) / 32;
  if ((st = dalloc(&s->waveSp, (size_t)s->nF * s->L)) || (st = dalloc(&s->eleDt, (size_t)s->L)) ||
      (st = dalloc(&s->dtDev, 2)) || (st = dalloc(&s->timeDev, 1)) || (st = dalloc(&s->blockMin, (size_t)s->L)) ||
      (st = dalloc(&s->normPartial, (size_t)nbDt * s->nV)) || (st = dalloc(&s->normOut, (size_t)s->nV)) ||
      (st = dalloc(&s->err, 1)) || (st = dalloc(&s->ticket, 1)))
    return st;
  CK(cudaMallocHost(&s->hostFlag, sizeof(unsigned)));
  if (p.dtType == 0) CK(cudaMemcpy(s->dtDev, &p.dt, sizeof(double), cudaMemcpyHostToDevice));
  if (s->ks.nTma > 0 && !s->ks.grad) {
    const char *env = getenv("FRG_KERNEL");
    s->useTma = !(env && std::strcmp(env, "generic") == 0);
    if (s->useTma && (st = setup_tma(s.get()))) return st;
    const char *pe = getenv("FRG_PDL");
    s->pdl = !(pe && std::strcmp(pe, "0") == 0);
  }
  {
    const char *ge = getenv("FRG_GRAPH");
    s->useGraph = !(ge && std::strcmp(ge, "0") == 0);
  }
  CK(cudaDeviceGetAttribute(&s->nSM, cudaDevAttrMultiProcessorCount, dev));
  if (s->ks.vgrad) {
    const char *env = getenv("FRG_KERNEL");
    s->useViscTma = !(env && std::strcmp(env, "generic") == 0);
    if (s->useViscTma && (st = setup_visc_tma(s.get()))) return st;
  }
  CK(cudaEventCreateWithFlags(&s->noallocOrder, cudaEventDisableTiming));
  {
    // the allocation-free residual's scratch address on this device, looked
    // up here so that the module holding it is resident before any
    // frg_calc_residual_noalloc call
    void *scratch = nullptr;
    if ((st = noalloc_scratch_addr(&scratch))) return st;
  }
  CK(cudaDeviceSynchronize());
  *out = s.release();
  return FRG_OK;
}

frg_status frg_inspect_geometry(const frg_params *params, const frg_mesh *mesh, int which, double *out,
                                long *count) {
  if (!params || !mesh || !count) return fail(FRG_ERR_ARG, "null argument");
  HostGeom g;
  std::string err;
  frg_status st = build_geometry(*params, *mesh, g, err);
  if (st) return fail(st, "%s", err.c_str());
  const int d = g.nDims, nS = g.nS, nF = g.nF, nE = g.nE;
  std::vector<double> r;
  switch (which) {
    case 0: r = g.pos_spts; break;
    case 1:
      r.resize(g.JG.size());
      for (int a = 0; a < d; a++)
        for (int b = 0; b < d; b++)
          for (int q = 0; q < nS; q++)
            for (int e = 0; e < nE; e++)
              r[(((size_t)a * nS + q) * nE + e) * d + b] = g.JG[(((size_t)a * d + b) * nS + q) * nE + e];
      break;
    case 2: r = g.detJ; break;
    case 3:
      r.resize(g.nrmOwn.size());
      for (int k = 0; k < d; k++)
        for (int f = 0; f < nF; f++)
          for (int e = 0; e < nE; e++) r[((size_t)f * nE + e) * d + k] = g.nrmOwn[((size_t)k * nF + f) * nE + e];
      break;
    case 4: r = g.dA; break;
    case 5: r.assign(g.faceTable.begin(), g.faceTable.end()); break;
    default: return fail(FRG_ERR_ARG, "unknown geometry item %d", which);
  }
  *count = (long)r.size();
  if (out) std::memcpy(out, r.data(), r.size() * sizeof(double));
  return FRG_OK;
}

frg_status frg_destroy(frg_solver *s) {
  if (!s) return FRG_OK;
  if (s->stream) cudaStreamSynchronize(s->stream);
  adj_free(s);
  drop_graphs(s);
  double *dp[] = {s->U, s->U0, s->Acc, s->divF[0], s->divF[1], s->divF[2], s->divF[3], s->divF[4], s->detJd,
                  s->nrmOwn, s->dAd, s->vol, s->wsurf, s->wvol, s->waveSp, s->eleDt, s->dtDev, s->timeDev,
                  s->blockMin, s->normPartial, s->normOut, s->scratchRef};
  for (double *q : dp) if (q) cudaFree(q);
  cudaFree(s->grpDt);
  cudaFree(s->grpTime);
  void *vp[] = {s->grp, s->W[0], s->W[1], s->tr[0], s->tr[1], s->nrm, s->dAs, s->JG, s->detJs, s->invDetS, s->nbr, s->err,
                s->ticket,
                s->fvn, s->fvn2, s->dUg};
  for (void *q : vp) if (q) cudaFree(q);
  for (auto &r : s->opImg)
    for (float *q : r) if (q) cudaFree(q);
  void *ip[] = {s->intPart, s->w1Dev, s->qShape, s->qInterp, s->qW};
  for (void *q : ip) if (q) cudaFree(q);
  void *gp[] = {s->xvDev, s->geoTab, s->posDev, s->geoInt, s->geoFlag};
  for (void *q : gp) if (q) cudaFree(q);
  if (s->noallocOrder) cudaEventDestroy(s->noallocOrder);
  if (s->hostFlag) cudaFreeHost(s->hostFlag);
  cudaStream_t own = s->ownStream ? s->ownStream : s->stream;  // a caller's stream is not ours to destroy
  if (own) cudaStreamDestroy(own);
  delete s;
  return FRG_OK;
}

frg_status frg_update_geometry(frg_solver *s, const double *xv) {
  if (!s || !xv) return fail(FRG_ERR_ARG, "null argument");
  const int d = s->p.nDims, nN = s->nNodes, nS = s->nS, nF = s->nF, nE = s->nE, L = s->L;
  const size_t nX = (size_t)nE * nN * d;
  if (!s->geoTab) {
    MetricTables t;
    std::string err;
    if (!metric_tables(d, s->p.order, s->p.vcjhScheme, nN, t, err)) return fail(FRG_ERR_ARG, "%s", err.c_str());
    std::vector<double> tab(t.shS);
    tab.insert(tab.end(), t.dS.begin(), t.dS.end());
    tab.insert(tab.end(), t.dF.begin(), t.dF.end());
    tab.insert(tab.end(), t.wv.begin(), t.wv.end());
    std::vector<int> fi(t.fdir);
    fi.insert(fi.end(), t.fsgn.begin(), t.fsgn.end());
    CK(cudaMalloc(&s->geoTab, tab.size() * 8));
    CK(cudaMemcpy(s->geoTab, tab.data(), tab.size() * 8, cudaMemcpyHostToDevice));
    CK(cudaMalloc(&s->geoInt, fi.size() * sizeof(int)));
    CK(cudaMemcpy(s->geoInt, fi.data(), fi.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&s->xvDev, nX * 8));
    CK(cudaMalloc(&s->posDev, (size_t)nS * nE * d * 8));
    CK(cudaMalloc(&s->geoFlag, 2 * sizeof(unsigned)));
  }
  const double *wv = s->geoTab + (size_t)nN * nS * (1 + d) + (size_t)nN * nF * d;
  const int *fdir = s->geoInt, *fsgn = s->geoInt + nF;
  CK(cudaMemcpyAsync(s->xvDev, xv, nX * 8, cudaMemcpyHostToDevice, s->stream));
  const unsigned init[2] = {0u, 0xffffffffu};
  CK(cudaMemcpyAsync(s->geoFlag, init, sizeof init, cudaMemcpyHostToDevice, s->stream));
  MetricOut out{s->posDev, s->detJd, s->nrmOwn, s->dAd, s->vol, s->JG, s->detJs, s->invDetS, s->nrm, s->dAs};
  // a negative Jacobian leaves the solver's metrics as they were
  CK(launch_metrics(d, (int)s->sstore, s->xvDev, s->geoTab, fdir, fsgn, wv, s->nbr, nN, nS, nF, nE, L, 1, out,
                    s->geoFlag, s->stream));
  unsigned flag[2];
  CK(cudaMemcpyAsync(flag, s->geoFlag, sizeof flag, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  s->launches += 1;
  if (flag[0]) return fail(FRG_ERR_NEG_JAC, "Negative Jacobian at solution points (element %u)", flag[1]);
  CK(launch_metrics(d, (int)s->sstore, s->xvDev, s->geoTab, fdir, fsgn, wv, s->nbr, nN, nS, nF, nE, L, 0, out,
                    s->geoFlag, s->stream));
  s->launches += 2;
  // the host copies that frg_download serves
  CK(cudaMemcpyAsync(s->g.pos_spts.data(), s->posDev, s->g.pos_spts.size() * 8, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaMemcpy2DAsync(s->g.detJ.data(), (size_t)nE * 8, s->detJd, (size_t)L * 8, (size_t)nE * 8, nS,
                       cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  std::memcpy(s->xvHost.data(), xv, nX * 8);
  s->waveStale = true;
  s->dtFresh = false;
  return FRG_OK;
}

frg_status frg_write_paraview(frg_solver *s, const char *dataFileName) {
  if (!s || !dataFileName) return fail(FRG_ERR_ARG, "null argument");
  if (s->grp) return fail(FRG_ERR_ARG, "ensemble mode: one time per case, write each case's solver");
  std::vector<double> U((size_t)s->nS * s->nE * s->nV);
  double t = 0.0;
  frg_status st;
  if ((st = frg_download(s, FRG_U_SPTS, 0, U.data())) || (st = frg_get_time(s, &t, nullptr, nullptr))) return st;
  const frg_mesh m{s->nE, s->nNodes, s->xvHost.data(), nullptr, nullptr};
  return frg_write_paraview_host(&s->p, &m, U.data(), t, s->iter, dataFileName);
}

frg_status frg_read_restart(frg_solver *s, const char *dataFileName, int restartIter) {
  if (!s || !dataFileName) return fail(FRG_ERR_ARG, "null argument");
  if (s->grp) return fail(FRG_ERR_ARG, "ensemble mode: restart each case's solver");
  std::vector<double> U((size_t)s->nS * s->nE * s->nV);
  double t = 0.0;
  frg_status st;
  if ((st = frg_read_restart_host(&s->p, s->nE, dataFileName, restartIter, U.data(), &t))) return st;
  if ((st = frg_upload(s, FRG_U_SPTS, U.data()))) return st;
  CK(cudaMemcpyAsync(s->timeDev, &t, 8, cudaMemcpyHostToDevice, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  // input::readInputFile: initIter = restartIter (src/input.cpp:417-421)
  return frg_set_iter(s, restartIter, restartIter);
}

frg_status frg_info(const frg_solver *s, int *nSpts, int *nFpts, int *nFields, int *nEles) {
  if (!s) return fail(FRG_ERR_ARG, "null handle");
  if (nSpts) *nSpts = s->nS;
  if (nFpts) *nFpts = s->nF;
  if (nFields) *nFields = s->nV;
  if (nEles) *nEles = s->nE;
  return FRG_OK;
}

frg_status frg_get_operator(const frg_solver *s, int which, int dim, double *out) {
  if (!s || !out || which < 0 || which > 4 || dim < 0 || dim >= s->p.nDims) return fail(FRG_ERR_ARG, "bad operator request");
  std::vector<double> m;
  dense_operator(s->p.nDims, s->ops, which, dim, m);
  std::memcpy(out, m.data(), m.size() * sizeof(double));
  return FRG_OK;
}

frg_status frg_set_operators(frg_solver *s, int order, const double *E, const double *D, const double *C,
                             const double *Efn) {
  if (!s || !E || !D || !C) return fail(FRG_ERR_ARG, "null argument");
  if (order != s->p.order) return fail(FRG_ERR_ARG, "operators of order %d for a solver of order %d", order, s->p.order);
  if (s->adj) return fail(FRG_ERR_ARG, "operators cannot change once the adjoint is set up");
  const int d = s->p.nDims, nS = s->nS, nF = s->nF;
  // the given matrices against one scheme's tensor-product operators
  auto matches = [&](const Ops1D &o) {
    std::vector<double> m;
    auto same = [&](const double *given, int which, int dim) {
      dense_operator(d, o, which, dim, m);
      double mx = 0, diff = 0;
      for (size_t i = 0; i < m.size(); i++) {
        mx = std::max(mx, std::fabs(m[i]));
        diff = std::max(diff, std::fabs(m[i] - given[i]));
      }
      return diff <= 1e-13 * std::max(mx, 1.0);
    };
    if (!same(E, 0, 0) || !same(C, 3, 0)) return false;
    for (int k = 0; k < d; k++) {
      if (!same(D + (size_t)k * nS * nS, 1, k)) return false;
      if (Efn && !same(Efn + (size_t)k * nF * nS, 2, k)) return false;
    }
    return true;
  };
  int scheme = -1;
  for (int v : {s->p.vcjhScheme, 0, 1, 2, 3}) {
    if (v == 3 && order < 2) continue;
    if (matches(build_ops1d(order, v))) {
      scheme = v;
      break;
    }
  }
  if (scheme < 0)
    return fail(FRG_ERR_ARG, "the matrices are not the FR operators of a VCJH scheme (DG, SD, HU, C+) at order %d "
                             "on the reference's Gauss points", order);
  if (scheme != s->p.vcjhScheme) {
    frg_status st;
    if ((st = frg_sync(s))) return st;
    s->p.vcjhScheme = scheme;
    s->ops = build_ops1d(order, scheme);
    drop_graphs(s);  // the captured stages carry the scheme
    for (auto &r : s->opImg)
      for (float *&q : r)
        if (q) { cudaFree(q); q = nullptr; }
  }
  return FRG_OK;
}

frg_status frg_apply_operator(frg_solver *s, int which, int dim, const float *X, float *Y, int ld, float beta) {
  if (!s || !X || !Y) return fail(FRG_ERR_ARG, "null argument");
  if (which < 0 || which > 4) return fail(FRG_ERR_ARG, "operator %d does not exist", which);
  const bool perDim = which == 1 || which == 2 || which == 4;
  if (dim < 0 || dim >= (perDim ? s->p.nDims : 1)) return fail(FRG_ERR_ARG, "bad operator dimension %d", dim);
  if (ld < s->nE || ld % 4 || ((uintptr_t)X & 15) || ((uintptr_t)Y & 15))
    return fail(FRG_ERR_ARG, "arrays must be 16-byte aligned with an element stride >= nEles and a multiple of 4");
  const int M = (which == 0 || which == 2) ? s->nF : s->nS;
  const int K = (which == 3 || which == 4) ? s->nF : s->nS;
  const int KP = (K + 7) & ~7, NP = (M + 15) & ~15;
  if (NP > 256 || KP > 256 || op_gemm_smem(KP, NP) > 227 * 1024)
    return fail(FRG_ERR_ARG, "operator %d x %d too large for the single-pass tensor-core kernel", M, K);
  float *&img = s->opImg[which][dim];
  if (!img) {
    std::vector<double> op;
    dense_operator(s->p.nDims, s->ops, which, dim, op);
    std::vector<float> h;
    build_op_image(op.data(), M, K, KP, NP, h);
    CK(cudaMalloc((void **)&img, h.size() * sizeof(float)));
    CK(cudaMemcpy(img, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  EncodeTiledFn enc = encode_fn();
  if (!enc) return fail(FRG_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  CUtensorMap mX;
  cuuint64_t dims[3] = {(cuuint64_t)ld, (cuuint64_t)K, (cuuint64_t)s->nV};
  cuuint64_t strides[2] = {(cuuint64_t)ld * 4, (cuuint64_t)ld * 4 * K};
  // boxes of 32 elements (128 bytes) x KP points, 32-byte chunks swizzled
  // within 128 bytes: the kernel's MN-major TF32 operand layout
  cuuint32_t box[3] = {32, (cuuint32_t)KP, 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = enc(&mX, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(X), dims, strides, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(FRG_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  CK(launch_op_gemm(mX, img, Y, KP, NP, M, ld, s->nE, s->nV, beta, s->err, s->stream));
  s->launches++;
  return FRG_OK;
}

static frg_status ref_scratch(frg_solver *s, size_t n) {
  if (!s->scratchRef) {
    size_t big = (size_t)s->nV * std::max(s->nS, s->nF) * s->nE;
    frg_status st = dalloc(&s->scratchRef, big);
    if (st) return st;
  }
  (void)n;
  return FRG_OK;
}

frg_status frg_upload(frg_solver *s, int array, const double *host) {
  if (!s || !host) return fail(FRG_ERR_ARG, "null argument");
  if (array != FRG_U_SPTS && array != FRG_U0) return fail(FRG_ERR_ARG, "array not uploadable");
  frg_status st = ref_scratch(s, 0);
  if (st) return st;
  const size_t n = (size_t)s->nV * s->nS * s->nE;
  CK(cudaMemcpyAsync(s->scratchRef, host, n * 8, cudaMemcpyHostToDevice, s->stream));
  fr_to_device_layout<<<(unsigned)((n + 255) / 256), 256, 0, s->stream>>>(s->scratchRef,
                                                                         array == FRG_U0 ? s->U0 : s->U, s->nV,
                                                                         s->nS, s->nE, s->L);
  if ((st = post_launch(s))) return st;
  if (array == FRG_U_SPTS) s->trValid = false;
  CK(cudaStreamSynchronize(s->stream));
  return FRG_OK;
}

frg_status frg_download(frg_solver *s, int array, int stage, double *host) {
  if (!s || !host) return fail(FRG_ERR_ARG, "null argument");
  frg_status st = ref_scratch(s, 0);
  if (st) return st;
  const double *src = nullptr;
  int npt = s->nS;
  switch (array) {
    case FRG_U_SPTS: src = s->U; break;
    case FRG_U0: src = s->U0; break;
    case FRG_DIVF:
      if (stage < 0 || stage >= s->nRK || !s->divF[stage]) return fail(FRG_ERR_ARG, "divF stage %d not computed", stage);
      src = s->divF[stage];
      break;
    case FRG_U_FPTS: {
      if ((st = ensure_traces(s))) return st;
      npt = s->nF;
      const size_t n = (size_t)s->nV * s->nF * s->L;
      if (s->sstore == 8) {
        src = (const double *)s->tr[s->curTr];
      } else {
        // widen float traces on the host
        std::vector<float> f(n);
        CK(cudaMemcpyAsync(f.data(), s->tr[s->curTr], n * 4, cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
        for (int v = 0; v < s->nV; v++)
          for (int q = 0; q < s->nF; q++)
            for (int e = 0; e < s->nE; e++)
              host[((size_t)q * s->nE + e) * s->nV + v] = f[((size_t)v * s->nF + q) * s->L + e];
        return FRG_OK;
      }
      break;
    }
    case FRG_POS_SPTS:
      std::memcpy(host, s->g.pos_spts.data(), s->g.pos_spts.size() * 8);
      return FRG_OK;
    case FRG_DETJAC:
      std::memcpy(host, s->g.detJ.data(), s->g.detJ.size() * 8);
      return FRG_OK;
    case FRG_WAVESP: {
      std::vector<double> w((size_t)s->nF * s->L);
      CK(cudaMemcpyAsync(w.data(), s->waveSp, w.size() * 8, cudaMemcpyDeviceToHost, s->stream));
      CK(cudaStreamSynchronize(s->stream));
      for (int f = 0; f < s->nF; f++)
        for (int e = 0; e < s->nE; e++) host[(size_t)e * s->nF + f] = w[(size_t)f * s->L + e];
      return FRG_OK;
    }
    case FRG_ELE_DT:
      CK(cudaMemcpyAsync(host, s->eleDt, (size_t)s->nE * 8, cudaMemcpyDeviceToHost, s->stream));
      CK(cudaStreamSynchronize(s->stream));
      return FRG_OK;
    default:
      return fail(FRG_ERR_ARG, "unknown array %d", array);
  }
  const size_t n = (size_t)s->nV * npt * s->nE;
  fr_to_ref_layout<<<(unsigned)((n + 255) / 256), 256, 0, s->stream>>>(src, s->scratchRef, s->nV, npt, s->nE, s->L);
  if ((st = post_launch(s))) return st;
  CK(cudaMemcpyAsync(host, s->scratchRef, n * 8, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return FRG_OK;
}

frg_status frg_set_initial_condition(frg_solver *s, int icType, double a0) {
  if (!s) return fail(FRG_ERR_ARG, "null handle");
  std::vector<double> U;
  std::string err;
  frg_status st = initial_condition(s->p, s->g, icType, a0, U, err);
  if (st) return fail(st, "%s", err.c_str());
  return frg_upload(s, FRG_U_SPTS, U.data());
}

}  // extern "C"

// ---- scratch of frg_calc_residual_noalloc
// The flux-point traces of the allocation-free residual live in this fixed
// array (16 MiB, 256-byte aligned), so that entry point calls no allocator.
// It is part of the library's device image: every GPU that loads the library
// holds it until the process exits.  Host code must not use the symbol as a
// pointer (it is a host-side stand-in); the device address is looked up once
// per device with cudaGetSymbolAddress and passed to the kernels.
constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];
namespace {
constexpr int kMaxDevices = 64;
void *g_noalloc_addr[kMaxDevices] = {nullptr};
std::mutex g_noalloc_mu;
}  // namespace

// Set-up once per device, with that device current: the array's device
// address by cudaGetSymbolAddress (the host-side symbol is not a device
// pointer).  frg_create calls this, so the lookup and the loading of this
// module happen there, not inside the allocation-free call.
static frg_status noalloc_scratch_addr(void **out) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(FRG_ERR_ARG, "device index %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(FRG_ERR_CUDA, "cudaGetSymbolAddress(noalloc scratch): %s", cudaGetErrorString(e));
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return FRG_OK;
}

extern "C" {

frg_status frg_calc_residual_noalloc(frg_solver *s, const double *U_dev, double *divF_dev, void *stream) {
  if (!s || !U_dev || !divF_dev) return fail(FRG_ERR_ARG, "null argument");
  // traces, and for viscous runs the projected viscous fluxes after them
  const size_t one = (size_t)s->nV * s->nF * s->L * s->sstore;
  const size_t oneAligned = (one + 255) & ~size_t(255);
  const size_t need = one + (s->ks.grad ? oneAligned * (s->visc2 ? 2 : 1) : 0);
  if (need > kNoAllocScratchBytes)
    return fail(FRG_ERR_ARG, "frg_calc_residual_noalloc: traces need %zu bytes, the scratch array holds %zu", need,
                kNoAllocScratchBytes);
  void *scratch = nullptr;
  frg_status sst = noalloc_scratch_addr(&scratch);  // looked up by frg_create on this device already
  if (sst) return sst;
  cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
  if (st != s->stream) {
    // after the work pending on the handle's stream (uploads, geometry
    // updates) that wrote the metrics this residual reads
    CK(cudaEventRecord(s->noallocOrder, s->stream));
    CK(cudaStreamWaitEvent(st, s->noallocOrder, 0));
  }
  // traces of the caller's state into the scratch array, then the residual
  s->ks.trace(U_dev, scratch, s->L, s->nE, s->nE, s->p.vcjhScheme, st);
  CK(cudaGetLastError());
  StageArgs a = base_args(s);
  a.ldU = s->nE;  // the caller's arrays are dense [nFields][nSpts][nEles]
  a.Uin_d = U_dev;
  a.trIn = scratch;
  a.divF = divF_dev;
  a.flags = SF_RESIDUAL;
  if (s->ks.grad) {
    unsigned char *base = static_cast<unsigned char *>(scratch);
    a.fvnOut = base + oneAligned;
    a.fvnIn = a.fvnOut;
    a.fvn2Out = s->visc2 ? base + 2 * oneAligned : nullptr;
    a.fvn2In = a.fvn2Out;
    s->ks.grad(&a, s->nBlk, s->ks.smem, st);
    CK(cudaGetLastError());
    s->launches += 1;
  }
  s->ks.stage(&a, s->nBlk, s->ks.smem, st);
  CK(cudaGetLastError());
  s->launches += 2;
  return FRG_OK;
}

frg_status frg_calc_residual(frg_solver *s, int step) {
  if (!s || step < 0 || step >= s->nRK) return fail(FRG_ERR_ARG, "bad step");
  frg_status st;
  if (!s->divF[step] && (st = dalloc(&s->divF[step], (size_t)s->nV * s->nS * s->L))) return st;
  // solver::extrapolateU always recomputes the traces of U_spts
  s->trValid = false;
  if ((st = ensure_traces(s))) return st;
  StageArgs a = base_args(s);
  a.Uin_d = s->U;
  a.trIn = s->tr[s->curTr];
  a.divF = s->divF[step];
  a.dUg = s->dUg;
  a.flags = SF_RESIDUAL | SF_WAVESP;
  s->dtFresh = false;  // the wave speeds changed
  if ((st = launch_stage_args(s, a))) return st;
  if (step == 0) s->divF0Valid = true;
  return FRG_OK;
}

frg_status frg_time_step_a(frg_solver *s, int step, double rkval) {
  if (!s || step < 0 || step >= s->nRK || !s->divF[step]) return fail(FRG_ERR_ARG, "bad step / residual missing");
  if (s->grp) return fail(FRG_ERR_ARG, "ensemble mode: advance with frg_update");
  const long n = (long)s->nV * s->nS * s->L;
  fr_timestep_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s->stream>>>(
      s->U, s->U0, s->divF[step], s->detJd, s->p.dtType == 2 ? s->eleDt : s->dtDev + s->dtCur, s->p.dtType == 2, rkval, 0,
      s->nS, s->nE, s->L, n);
  s->trValid = false;
  return post_launch(s);
}

frg_status frg_time_step_b(frg_solver *s, int step) {
  if (!s || step < 0 || step >= s->nRK || !s->divF[step]) return fail(FRG_ERR_ARG, "bad step / residual missing");
  if (s->grp) return fail(FRG_ERR_ARG, "ensemble mode: advance with frg_update");
  const long n = (long)s->nV * s->nS * s->L;
  fr_timestep_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s->stream>>>(
      s->U, s->U0, s->divF[step], s->detJd, s->p.dtType == 2 ? s->eleDt : s->dtDev + s->dtCur, s->p.dtType == 2,
      s->RKb[step], 1, s->nS, s->nE, s->L, n);
  s->trValid = false;
  return post_launch(s);
}

frg_status frg_copy_u_to_u0(frg_solver *s) {
  if (!s) return fail(FRG_ERR_ARG, "null handle");
  CK(cudaMemcpyAsync(s->U0, s->U, (size_t)s->nV * s->nS * s->L * 8, cudaMemcpyDeviceToDevice, s->stream));
  return FRG_OK;
}
frg_status frg_copy_u0_to_u(frg_solver *s) {
  if (!s) return fail(FRG_ERR_ARG, "null handle");
  CK(cudaMemcpyAsync(s->U, s->U0, (size_t)s->nV * s->nS * s->L * 8, cudaMemcpyDeviceToDevice, s->stream));
  s->trValid = false;
  return FRG_OK;
}

frg_status frg_calc_dt(frg_solver *s, double *dt_out) {
  if (!s) return fail(FRG_ERR_ARG, "null handle");
  if (s->grp) return fail(FRG_ERR_ARG, "ensemble mode: per-group dt via frg_update / frg_get_group_times");
  frg_status st;
  if (s->p.dtType != 0) {
    if (s->iter == s->initIter + 1 || s->waveStale) {
      // calcWaveSpFpts reads U_fpts as the last extrapolation left it
      if ((st = ensure_traces(s)) || (st = launch_wavesp(s))) return st;
      s->waveStale = false;
    }
    if ((st = launch_dt(s))) return st;
  }
  if ((st = check_flags(s))) return st;
  if (dt_out) {
    CK(cudaMemcpyAsync(dt_out, s->dtDev + s->dtCur, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
  }
  return FRG_OK;
}

// The captured graph of one fused step in the solver's current state
// (dt mode, trace buffer, dt slot), captured on first use.
static frg_status step_graph(frg_solver *s, int mode, cudaGraphExec_t *exec, cudaGraph_t *raw) {
  const int ct = s->curTr;
  cudaGraphExec_t &ge = s->graph[mode][ct][s->dtCur];
  cudaGraph_t &gr = s->graphRaw[mode][ct][s->dtCur];
  if (!ge) {
    const long long before = s->launches;
    CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    frg_status st = enqueue_step(s, mode);
    cudaError_t ce = cudaStreamEndCapture(s->stream, &gr);
    if (st) return st;
    if (ce != cudaSuccess) return fail(FRG_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
    CK(cudaGraphInstantiate(&ge, gr, 0));
    s->launches = before;
    s->curTr = ct;
  }
  if (exec) *exec = ge;
  if (raw) *raw = gr;
  return FRG_OK;
}

// Host bookkeeping after a captured step was launched.
static void step_done(frg_solver *s, int mode) {
  // count the kernels the graph holds
  s->launches += s->nRK * (s->ks.grad ? 2 : 1) + (s->p.dtType != 0 ? mode : 0) + (s->grp ? 1 : 0);
  s->curTr ^= (s->nRK & 1);
  s->dtFresh = fused_dt(s);
  s->dtLast = s->dtCur;
  s->dtCur ^= (int)s->dtFresh;
  if (mode == 2) s->waveStale = false;
}

}  // extern "C"
namespace {
// nsteps steps of the fused path enqueued on the handle's stream (captured
// steps replayed), without reading the flags back.
frg_status enqueue_updates(frg_solver *s, int nsteps) {
  frg_status st;
  // writeResidual's check (src/output.cpp:823-824); a CFL dt is checked on
  // the device where it is computed
  if (nsteps > 0 && s->p.dtType == 0 && !s->grp && !(s->p.dt >= 1e-13))
    return fail(FRG_ERR_DT, "Instability detected - dt approaching zero");
  if ((st = ensure_traces(s))) return st;
  for (int n = 0; n < nsteps; n++) {
    s->iter++;
    const int mode = dt_mode(s);
    if (s->useGraph) {
      cudaGraphExec_t ge;
      if ((st = step_graph(s, mode, &ge, nullptr))) return st;
      CK(cudaGraphLaunch(ge, s->stream));
    } else {
      // the same launches straight onto the stream (the bookkeeping below
      // counts and toggles as for a replayed graph)
      const long long before = s->launches;
      const int ct = s->curTr;
      if ((st = enqueue_step(s, mode))) return st;
      s->launches = before;
      s->curTr = ct;
    }
    step_done(s, mode);
  }
  if (nsteps > 0) s->divF0Valid = s->monitor;
  return FRG_OK;
}
}  // namespace
extern "C" {

frg_status frg_update(frg_solver *s, int nsteps) {
  if (!s || nsteps < 0) return fail(FRG_ERR_ARG, "bad arguments");
  frg_status st;
  if (s->p.timeType == 0 && s->p.dtType != 0) {
    if (s->grp) return fail(FRG_ERR_ARG, "ensemble mode: Forward Euler with CFL dt is not supported");
    // Forward Euler takes its CFL dt after the residual (src/solver.cpp:238-241):
    // the reference's unfused sequence
    for (int n = 0; n < nsteps; n++)
      if ((st = unfused_update(s))) return st;
    return check_flags(s);
  }
  if ((st = enqueue_updates(s, nsteps))) return st;
  return check_flags(s);
}

// Upload, steps, download and the flag word on the handle's stream with one
// synchronisation at the end (the host waits once per call, not after each
// part).  The state is written back even when a flag is raised: the
// reference's own solution array holds the failed step too when its check
// fires (src/output.cpp:823-841).
frg_status frg_update_host(frg_solver *s, double *U_host, int nsteps) {
  if (!s || !U_host || nsteps < 0) return fail(FRG_ERR_ARG, "bad arguments");
  frg_status st;
  if (s->p.timeType == 0 && s->p.dtType != 0) {  // the unfused sequence reads dt back per step
    if ((st = frg_upload(s, FRG_U_SPTS, U_host))) return st;
    if ((st = frg_update(s, nsteps))) return st;
    return frg_download(s, FRG_U_SPTS, 0, U_host);
  }
  if ((st = ref_scratch(s, 0))) return st;
  const size_t n = (size_t)s->nV * s->nS * s->nE;
  CK(cudaMemcpyAsync(s->scratchRef, U_host, n * 8, cudaMemcpyHostToDevice, s->stream));
  fr_to_device_layout<<<(unsigned)((n + 255) / 256), 256, 0, s->stream>>>(s->scratchRef, s->U, s->nV, s->nS, s->nE,
                                                                         s->L);
  if ((st = post_launch(s))) return st;
  s->trValid = false;
  if ((st = enqueue_updates(s, nsteps))) {
    cudaStreamSynchronize(s->stream);  // the upload still reads U_host
    return st;
  }
  fr_to_ref_layout<<<(unsigned)((n + 255) / 256), 256, 0, s->stream>>>(s->U, s->scratchRef, s->nV, s->nS, s->nE,
                                                                       s->L);
  if ((st = post_launch(s))) return st;
  CK(cudaMemcpyAsync(s->hostFlag, s->err, sizeof(unsigned), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaMemcpyAsync(U_host, s->scratchRef, n * 8, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return flags_status(s, *s->hostFlag);
}

frg_status frg_residual_norm(frg_solver *s, int normType, double *out) {
  if (!s || !out || normType < 1 || normType > 3) return fail(FRG_ERR_ARG, "bad arguments");
  if (!s->divF0Valid) return fail(FRG_ERR_ARG, "no stage-0 residual stored (call frg_calc_residual(0))");
  const int nb = (s->nE + 255) / 256;
  fr_norm_kernel<<<nb, 256, 256 * s->nV * sizeof(double), s->stream>>>(s->divF[0], s->detJd, s->wvol, s->nV, s->nS,
                                                                        s->nE, s->L, normType, s->normPartial, s->ticket,
                                                                        s->normOut);
  frg_status st = post_launch(s);
  if (st) return st;
  CK(cudaMemcpyAsync(out, s->normOut, (size_t)s->nV * 8, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return FRG_OK;
}

frg_status frg_set_monitor(frg_solver *s, int enable) {
  if (!s) return fail(FRG_ERR_ARG, "null handle");
  if ((enable != 0) == s->monitor) return FRG_OK;
  s->monitor = enable != 0;
  if (s->monitor && !s->divF[0]) {
    frg_status st = dalloc(&s->divF[0], (size_t)s->nV * s->nS * s->L);
    if (st) return st;
  }
  // the captured steps carry the old flags
  CK(cudaStreamSynchronize(s->stream));
  drop_graphs(s);
  return FRG_OK;
}

frg_status frg_get_time(const frg_solver *s, double *time, double *dt, int *iter) {
  if (!s) return fail(FRG_ERR_ARG, "null handle");
  // (ensemble mode: group 0's; all groups through frg_get_group_times)
  const double *tsrc = s->grp ? s->grpTime : s->timeDev;
  if (time) { CK(cudaMemcpyAsync(time, tsrc, 8, cudaMemcpyDeviceToHost, s->stream)); }
  if (dt) { CK(cudaMemcpyAsync(dt, dt_slot(const_cast<frg_solver *>(s), s->dtLast), 8, cudaMemcpyDeviceToHost, s->stream)); }
  CK(cudaStreamSynchronize(s->stream));
  if (iter) *iter = s->iter;
  return FRG_OK;
}

frg_status frg_set_iter(frg_solver *s, int iter, int initIter) {
  if (!s) return fail(FRG_ERR_ARG, "null handle");
  s->dtFresh = false;
  s->iter = iter;
  s->initIter = initIter;
  return FRG_OK;
}

frg_status frg_sync(frg_solver *s) {
  if (!s) return fail(FRG_ERR_ARG, "null handle");
  CK(cudaStreamSynchronize(s->stream));
  return check_flags(s);
}

frg_status frg_set_stream(frg_solver *s, void *stream) {
  if (!s) return fail(FRG_ERR_ARG, "null handle");
  CK(cudaStreamSynchronize(s->stream));
  if (!s->ownStream) s->ownStream = s->stream;
  s->stream = stream ? (cudaStream_t)stream : s->ownStream;
  return FRG_OK;
}

frg_status frg_tile_variant_count(const frg_solver *s, int *count) {
  if (!s || !count) return fail(FRG_ERR_ARG, "null argument");
  *count = s->useTma ? s->ks.nTma : 1;
  return FRG_OK;
}

frg_status frg_set_tile_variant(frg_solver *s, int variant) {
  if (!s) return fail(FRG_ERR_ARG, "null handle");
  if (!s->useTma) return variant == 0 ? FRG_OK : fail(FRG_ERR_ARG, "no TMA kernel in use");
  if (variant < 0 || variant >= s->ks.nTma) return fail(FRG_ERR_ARG, "tile variant out of range");
  CK(cudaStreamSynchronize(s->stream));
  drop_graphs(s);
  s->tmaVar = variant;
  return setup_tma(s);
}

frg_status frg_set_groups(frg_solver *s, const int *groupOfElement, int nGroups, const double *fixedDt) {
  if (!s || !groupOfElement || nGroups < 1) return fail(FRG_ERR_ARG, "bad arguments");
  if (s->p.dtType == 2) return fail(FRG_ERR_ARG, "ensemble mode: local dt (dtType 2) not supported");
  if (s->p.dtType == 0 && !fixedDt) return fail(FRG_ERR_ARG, "ensemble mode with dtType 0 needs one dt per group");
  std::vector<int> g((size_t)s->L, 0);
  for (int e = 0; e < s->nE; e++) {
    g[e] = groupOfElement[e];
    if (g[e] < 0 || g[e] >= nGroups) return fail(FRG_ERR_ARG, "element %d: group %d out of range", e, g[e]);
  }
  CK(cudaStreamSynchronize(s->stream));
  drop_graphs(s);
  cudaFree(s->grp);
  cudaFree(s->grpDt);
  cudaFree(s->grpTime);
  s->grp = nullptr;
  s->grpDt = s->grpTime = nullptr;
  frg_status st;
  if ((st = dalloc(&s->grp, g.size())) || (st = dalloc(&s->grpDt, 2 * (size_t)nGroups)) ||
      (st = dalloc(&s->grpTime, nGroups)))
    return st;
  CK(cudaMemcpy(s->grp, g.data(), g.size() * sizeof(int), cudaMemcpyHostToDevice));
  if (fixedDt) CK(cudaMemcpy(s->grpDt, fixedDt, (size_t)nGroups * 8, cudaMemcpyHostToDevice));
  s->nGrp = nGroups;
  s->dtCur = s->dtLast = 0;
  s->dtFresh = false;
  return FRG_OK;
}

frg_status frg_get_group_times(frg_solver *s, double *time, double *dt) {
  if (!s || !s->grp) return fail(FRG_ERR_ARG, "no groups set (frg_set_groups)");
  if (time) CK(cudaMemcpyAsync(time, s->grpTime, (size_t)s->nGrp * 8, cudaMemcpyDeviceToHost, s->stream));
  if (dt) CK(cudaMemcpyAsync(dt, dt_slot(s, s->dtLast), (size_t)s->nGrp * 8, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return FRG_OK;
}

frg_status frg_autotune(frg_solver *s, int nsteps, int *variant_out, double *ms_out) {
  if (!s || nsteps < 1) return fail(FRG_ERR_ARG, "bad arguments");
  const int nVar = s->useTma ? s->ks.nTma : 1;
  if (nVar > 1 && !(s->p.timeType == 0 && s->p.dtType != 0)) {
    // the trial steps advance the solution: keep everything they change
    const size_t nU = (size_t)s->nV * s->nS * s->L, nW = (size_t)s->nF * s->L, nD = (size_t)s->L;
    double *save = nullptr;
    const size_t nG = s->grp ? 3 * (size_t)s->nGrp : 0;
    frg_status st = dalloc(&save, 2 * nU + nW + nD + 3 + nG);
    if (st) return st;
    double *sU = save, *sD0 = save + nU, *sWs = save + 2 * nU, *sEd = sWs + nW, *sDt = sEd + nD, *sG = sDt + 3;
    const bool hadDiv = s->divF0Valid && s->divF[0];
    auto cp = [&](double *dst, const double *src, size_t n) {
      return cudaMemcpyAsync(dst, src, n * 8, cudaMemcpyDeviceToDevice, s->stream);
    };
    CK(cp(sU, s->U, nU));
    if (hadDiv) CK(cp(sD0, s->divF[0], nU));
    CK(cp(sWs, s->waveSp, nW));
    CK(cp(sEd, s->eleDt, nD));
    CK(cp(sDt, s->dtDev, 2));
    CK(cp(sDt + 2, s->timeDev, 1));
    if (nG) {
      CK(cp(sG, s->grpDt, 2 * (size_t)s->nGrp));
      CK(cp(sG + 2 * (size_t)s->nGrp, s->grpTime, s->nGrp));
    }
    const int iter = s->iter, dtCur = s->dtCur, dtLast = s->dtLast, curTr = s->curTr;
    const bool dtFresh = s->dtFresh, divValid = s->divF0Valid;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    // three interleaved rounds, the best of each candidate counts, so that a
    // clock ramp or a neighbour's burst does not decide
    static_assert(KernelSet::kMaxTma <= FRG_MAX_TILE_VARIANTS, "tile variants");
    double msv[KernelSet::kMaxTma];
    for (int v = 0; v < nVar; v++) msv[v] = 1e300;
    for (int round = 0; round < 3 && !st; round++)
      for (int v = 0; v < nVar && !st; v++) {
        CK(cudaStreamSynchronize(s->stream));
        drop_graphs(s);
        s->tmaVar = v;
        if ((st = setup_tma(s)) || (st = frg_update(s, 1))) break;
        CK(cudaEventRecord(e0, s->stream));
        if ((st = frg_update(s, nsteps))) break;
        CK(cudaEventRecord(e1, s->stream));
        CK(cudaEventSynchronize(e1));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        msv[v] = std::min(msv[v], (double)ms / nsteps);
      }
    int best = 0;
    for (int v = 0; v < nVar; v++) {
      if (ms_out) ms_out[v] = msv[v];
      if (msv[v] < msv[best]) best = v;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CK(cudaStreamSynchronize(s->stream));
    drop_graphs(s);
    s->tmaVar = best;
    frg_status st2 = setup_tma(s);
    CK(cp(s->U, sU, nU));
    if (hadDiv) CK(cp(s->divF[0], sD0, nU));
    CK(cp(s->waveSp, sWs, nW));
    CK(cp(s->eleDt, sEd, nD));
    CK(cp(s->dtDev, sDt, 2));
    CK(cp(s->timeDev, sDt + 2, 1));
    if (nG) {
      CK(cp(s->grpDt, sG, 2 * (size_t)s->nGrp));
      CK(cp(s->grpTime, sG + 2 * (size_t)s->nGrp, s->nGrp));
    }
    CK(cudaStreamSynchronize(s->stream));
    cudaFree(save);
    s->iter = iter;
    s->dtCur = dtCur;
    s->dtLast = dtLast;
    s->curTr = curTr;
    s->dtFresh = dtFresh;
    s->trValid = false;  // the trace buffers hold the trial steps' traces
    s->divF0Valid = divValid;
    if (st) return st;
    if (st2) return st2;
  } else if (ms_out) {
    ms_out[0] = 0;
  }
  if (variant_out) *variant_out = s->tmaVar;
  return FRG_OK;
}

frg_status frg_time_stages(frg_solver *s, int nsteps, void *flush, unsigned long long flushBytes, double *ms_out) {
  if (!s || !ms_out || nsteps < 1) return fail(FRG_ERR_ARG, "bad arguments");
  if (s->p.timeType == 0 && s->p.dtType != 0) return fail(FRG_ERR_ARG, "Forward Euler with CFL dt is not fused");
  frg_status st;
  if ((st = ensure_traces(s))) return st;
  const int nEv = 2 + s->nRK;
  std::vector<cudaEvent_t> ev(nEv);
  for (auto &e : ev) CK(cudaEventCreate(&e));
  std::vector<double> acc(1 + s->nRK, 0.0);
  for (int n = 0; n < nsteps && !st; n++) {
    if (flush) CK(cudaMemsetAsync(flush, n & 0xff, flushBytes, s->stream));
    s->iter++;
    const int mode = dt_mode(s);
    st = enqueue_step(s, mode, ev.data());
    if (mode == 2) s->waveStale = false;
    s->dtFresh = fused_dt(s);
    s->dtLast = s->dtCur;
    s->dtCur ^= (int)s->dtFresh;
    if (st) break;
    CK(cudaEventSynchronize(ev[nEv - 1]));
    for (int k = 0; k <= s->nRK; k++) {
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
      acc[k] += ms;
    }
  }
  for (auto &e : ev) cudaEventDestroy(e);
  if (st) return st;
  for (int k = 0; k <= s->nRK; k++) ms_out[k] = acc[k] / nsteps;
  return check_flags(s);
}

frg_status frg_launch_count(const frg_solver *s, long long *count) {
  if (!s || !count) return fail(FRG_ERR_ARG, "null argument");
  *count = s->launches;
  return FRG_OK;
}

}  // extern "C"

namespace {
// solver::update exactly as written (src/solver.cpp:212-250), on the device,
// one kernel per reference call.
frg_status unfused_update(frg_solver *s) {
  frg_status st;
  s->dtFresh = false;
  s->iter++;
  const int nRK = s->nRK;
  for (int step = 0; step < nRK - 1; step++) {
    if (step == 0 && s->p.dtType != 0 && (st = frg_calc_dt(s, nullptr))) return st;
    if (step == 0 && (st = frg_copy_u_to_u0(s))) return st;
    if ((st = frg_calc_residual(s, step)) || (st = frg_time_step_a(s, step, s->RKa[step + 1]))) return st;
  }
  if ((st = frg_calc_residual(s, nRK - 1))) return st;
  if (s->p.timeType < 5) {
    if (nRK > 1) { if ((st = frg_copy_u0_to_u(s))) return st; }
    else if (s->p.dtType != 0 && (st = frg_calc_dt(s, nullptr))) return st;
    for (int step = 0; step < nRK; step++)
      if ((st = frg_time_step_b(s, step))) return st;
  } else {
    if ((st = frg_time_step_a(s, nRK - 1, s->RKa[nRK]))) return st;
  }
  // time += dt
  double t = 0, dt = 0;
  CK(cudaMemcpyAsync(&t, s->timeDev, 8, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaMemcpyAsync(&dt, s->dtDev + s->dtCur, 8, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  t += dt;
  CK(cudaMemcpyAsync(s->timeDev, &t, 8, cudaMemcpyHostToDevice, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return FRG_OK;
}
}  // namespace

// ===================================================================== adjoint
// Discrete adjoint of frg_update (no counterpart in the reference): a forward
// run that keeps a checkpoint of U every k steps, then a reverse sweep that,
// per segment, recomputes the k steps from its checkpoint keeping every RK
// stage state, and reverses them stage by stage with the adjoint kernels.

struct AdjState {
  AdjSet ks;
  double *seed[2] = {nullptr, nullptr};  // stage seeds dJ/d(divF), ping-pong
  double *lam[2] = {nullptr, nullptr};   // adjoint of a step's final / initial state
  double *trY = nullptr, *fnbar = nullptr, *ybar = nullptr, *grad = nullptr, *part = nullptr;
  double *thetaBar = nullptr;
  double *thetaDir = nullptr;  // 5 doubles, device
  // viscous runs: forward gradient, projected fluxes and the pass buffers of
  // the viscous adjoint (AdjViscBufs)
  double *vg = nullptr, *vfvn = nullptr, *vfvn2 = nullptr, *vub = nullptr, *vufb = nullptr, *vdcb = nullptr;
  double *ckpt = nullptr;    // (nCkpt + 1) states: U at steps 0, k, 2k, ... and U_N last
  double *stages = nullptr;  // k * nRK stage states of one segment
  // checkpointed runs: a second set of stage slots, so that the reverse sweep
  // recomputes segment c-1 on the side stream while it reverses segment c
  double *stages2 = nullptr;
  cudaStream_t side = nullptr;
  cudaEvent_t evFork = nullptr, evJoin = nullptr;
  int ckptCap = 0, k = 0, nSteps = 0, stagesCap = 0;  // capacities in states / steps
  bool keepAll = false;  // the forward run kept every stage state
  // captured per-segment work of the reverse sweep, keyed by (kind, segment
  // length, buffer parities); valid while the buffers they name stay
  struct Captured {
    cudaGraphExec_t exec;
    int launches;
  };
  std::map<std::array<int, 4>, Captured> graphs;
  bool gradValid = false;
};

void adj_forget_graphs(frg_solver *s) {
  if (!s->adj) return;
  for (auto &g : s->adj->graphs) cudaGraphExecDestroy(g.second.exec);
  s->adj->graphs.clear();
}

void adj_free(frg_solver *s) {
  AdjState *a = s->adj;
  if (!a) return;
  for (auto &g : a->graphs) cudaGraphExecDestroy(g.second.exec);
  double *p[] = {a->seed[0], a->seed[1], a->lam[0], a->lam[1], a->trY, a->fnbar, a->ybar, a->grad, a->part,
                 a->thetaBar, a->thetaDir, a->ckpt, a->stages, a->stages2, a->vg, a->vfvn, a->vfvn2, a->vub,
                 a->vufb, a->vdcb};
  for (double *q : p) if (q) cudaFree(q);
  if (a->evFork) cudaEventDestroy(a->evFork);
  if (a->evJoin) cudaEventDestroy(a->evJoin);
  if (a->side) cudaStreamDestroy(a->side);
  delete a;
  s->adj = nullptr;
}

namespace {

// Seed of the last RK stage from the adjoint of a step's final state:
// gbar = -b_last * dt / detJ * lam.
__global__ void fr_adj_seed_kernel(const double *lam, const double *detJ, double *seed, double coef, int NV, int NS,
                                   int nE, int L, const int *grp, const double *dtGrp) {
  const long n = (long)NV * NS * L;
  for (long it = blockIdx.x * (long)blockDim.x + threadIdx.x; it < n; it += (long)gridDim.x * blockDim.x) {
    const int e = (int)(it % L), s = (int)((it / L) % NS);
    const double c = grp ? coef * dtGrp[grp[e]] : coef;
    seed[it] = e < nE ? c * lam[it] / detJ[(size_t)s * L + e] : 0.0;
  }
}

bool g_adj_tables[2] = {false, false};

frg_status adj_init(frg_solver *s) {
  if (s->adj) return FRG_OK;
  const frg_params &p = s->p;
  if (p.precision != FRG_FP64) return fail(FRG_ERR_ARG, "adjoint: FP64 precision only");
  if (!g_adj_tables[p.nDims - 2]) {
    cudaError_t e = p.nDims == 2 ? upload_tables_adj_2d() : upload_tables_adj_3d();
    if (e != cudaSuccess) return fail(FRG_ERR_CUDA, "adjoint tables: %s", cudaGetErrorString(e));
    g_adj_tables[p.nDims - 2] = true;
  }
  std::unique_ptr<AdjState> a(new AdjState);
  KernelKey key{p.nDims, p.order, s->nV, p.precision, s->g.nBndFaces > 0 ? 1 : 0, p.riemannType, p.viscous ? 1 : 0};
  std::string err;
  const bool ok = p.nDims == 2 ? select_adj_2d(key, a->ks, err) : select_adj_3d(key, a->ks, err);
  if (!ok) return fail(FRG_ERR_ARG, "%s", err.c_str());
  const size_t nSE = (size_t)s->nV * s->nS * s->L, nFE = (size_t)s->nV * s->nF * s->L;
  const size_t nPart = std::max(a->ks.entropyBlocks, (s->nE + 127) / 128);
  frg_status st;
  if ((st = dalloc(&a->seed[0], nSE)) || (st = dalloc(&a->seed[1], nSE)) || (st = dalloc(&a->lam[0], nSE)) ||
      (st = dalloc(&a->lam[1], nSE)) || (st = dalloc(&a->trY, nFE)) || (st = dalloc(&a->fnbar, nFE)) ||
      (st = dalloc(&a->ybar, nSE)) || (st = dalloc(&a->grad, nSE)) || (st = dalloc(&a->part, nPart)) ||
      (st = dalloc(&a->thetaBar, 1)) || (st = dalloc(&a->thetaDir, 5)) ||
      (p.viscous && ((st = dalloc(&a->vg, (size_t)p.nDims * nSE)) || (st = dalloc(&a->vfvn, nFE)) ||
                     (st = dalloc(&a->vfvn2, nFE)) || (st = dalloc(&a->vub, nSE)) || (st = dalloc(&a->vufb, nFE)) ||
                     (st = dalloc(&a->vdcb, nFE))))) {
    s->adj = a.release();
    return st;
  }
  AdjState *ap = a.get();
  s->adj = a.release();
  CK(cudaStreamCreateWithFlags(&ap->side, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&ap->evFork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&ap->evJoin, cudaEventDisableTiming));
  return FRG_OK;
}

AdjArgs adj_args(frg_solver *s, const double *Y, const double *gbar) {
  AdjArgs a{};
  a.nE = s->L;
  a.nEle = s->nE;
  a.Y = Y;
  a.gbar = gbar;
  a.trY = s->adj->trY;
  a.fnbar = s->adj->fnbar;
  a.nbr = s->nbr;
  a.nrm = static_cast<const double *>(s->nrm);
  a.dA = static_cast<const double *>(s->dAs);
  a.JG = static_cast<const double *>(s->JG);
  a.detJ = s->detJd;
  a.vcjh = s->p.vcjhScheme;
  a.err = s->err;
  a.thetaBar = s->adj->thetaBar;
  a.thetaDir = s->adj->thetaDir;
  a.grp = s->grp;
  a.dtGrp = s->grpDt;  // slot 0: the fixed per-group dt
  a.v = AdjViscBufs{s->adj->vg, s->adj->vfvn, s->adj->vfvn2, s->adj->vub, s->adj->vufb, s->adj->vdcb,
                    s->visc2 ? 1 : 0};
  a.ph = make_phys(s->p);
  return a;
}

frg_status adj_launch(frg_solver *s, const AdjArgs &a) {
  s->adj->ks.face(a, s->stream);
  frg_status st = post_launch(s);
  if (st) return st;
  s->adj->ks.elem(a, s->stream);
  s->launches += s->adj->ks.elemLaunches - 1;
  return post_launch(s);
}

void adj_drop_graphs(AdjState *a) {
  for (auto &g : a->graphs) cudaGraphExecDestroy(g.second.exec);
  a->graphs.clear();
}

// Runs `enqueue` through a CUDA graph captured on first use under `key`.
template <class F>
frg_status adj_replay(frg_solver *s, const std::array<int, 4> &key, F enqueue) {
  auto &gs = s->adj->graphs;
  auto it = gs.find(key);
  if (it == gs.end()) {
    const long long before = s->launches;
    cudaGraph_t gr;
    CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    frg_status st = enqueue();
    cudaError_t ce = cudaStreamEndCapture(s->stream, &gr);
    if (st) return st;
    if (ce != cudaSuccess) return fail(FRG_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
    cudaGraphExec_t ex;
    CK(cudaGraphInstantiate(&ex, gr, 0));
    CK(cudaGraphDestroy(gr));
    it = gs.emplace(key, AdjState::Captured{ex, (int)(s->launches - before)}).first;
    s->launches = before;
  }
  CK(cudaGraphLaunch(it->second.exec, s->stream));
  s->launches += it->second.launches;
  return FRG_OK;
}

// host [spt][ele][field] <-> device [field][spt][ele] state arrays
frg_status state_to_dev(frg_solver *s, const double *host, double *dev) {
  frg_status st = ref_scratch(s, 0);
  if (st) return st;
  const size_t n = (size_t)s->nV * s->nS * s->nE;
  CK(cudaMemcpyAsync(s->scratchRef, host, n * 8, cudaMemcpyHostToDevice, s->stream));
  fr_to_device_layout<<<(unsigned)((n + 255) / 256), 256, 0, s->stream>>>(s->scratchRef, dev, s->nV, s->nS, s->nE,
                                                                         s->L);
  return post_launch(s);
}
frg_status state_to_host(frg_solver *s, const double *dev, double *host) {
  frg_status st = ref_scratch(s, 0);
  if (st) return st;
  const size_t n = (size_t)s->nV * s->nS * s->nE;
  fr_to_ref_layout<<<(unsigned)((n + 255) / 256), 256, 0, s->stream>>>(dev, s->scratchRef, s->nV, s->nS, s->nE, s->L);
  if ((st = post_launch(s))) return st;
  CK(cudaMemcpyAsync(host, s->scratchRef, n * 8, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return FRG_OK;
}

// One RK step from U (on entry U_n, on exit U_{n+1}) keeping every stage
// state: Y[0] receives a copy of U_n and Y[k] (k = 1..nRK-1) the state stage
// k's residual is evaluated at.  Same kernels and arithmetic as frg_update:
// the TMA stage kernel where the update uses it (stage states through tensor
// maps made for the Y slots), else the generic one.  Traces of U must be
// current on entry (tr[curTr]) and are current on exit.
frg_status step_keep_stages(frg_solver *s, double *const *Y, bool advanceTime = false) {
  const size_t nSE = (size_t)s->nV * s->nS * s->L;
  CK(cudaMemcpyAsync(Y[0], s->U, nSE * 8, cudaMemcpyDeviceToDevice, s->stream));
  frg_status st;
  const int nRK = s->nRK;
  CUtensorMap mY[8];
  if (s->useTma)
    for (int k = 1; k < nRK; k++)
      if ((st = make_map(&mY[k], Y[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, s->nV * s->nS, s->L,
                         s->ks.tma[s->tmaVar].TE)))
        return st;
  for (int k = 0; k < nRK; k++) {
    StageArgs a = base_args(s);
    const bool first = k == 0, last = k == nRK - 1;
    a.trIn = s->tr[s->curTr];
    a.trOut = s->tr[s->curTr ^ 1];
    a.aNext = last ? 0.0 : s->RKa[k + 1];
    a.bCur = s->RKb[k];
    a.flags = (last ? SF_LAST : 0) | (first ? SF_FIRST : 0) | (last && advanceTime ? SF_TIME : 0);
    a.Acc = s->Acc;
    if (first && advanceTime && s->grp && (st = launch_group_step(s))) return st;
    if (s->useTma) {
      a.Uin_d = first ? s->U : nullptr;
      a.Uin_s = first ? nullptr : Y[k];
      TmaMaps mm;
      mm.U = s->mU;
      mm.Acc = s->mAcc;
      mm.Win = first ? s->mW[0] : mY[k];
      mm.Wout = last ? s->mW[0] : mY[k + 1];
      mm.trOut = s->mTr[s->curTr ^ 1];
      mm.trIn = s->mTr[s->curTr];
      mm.JG = s->mJG;
      mm.det = s->mDet;
      mm.nrm = s->mNrm;
      mm.dA = s->mDA;
      mm.nbr = s->mNbr;
      const KernelSet::TmaVariant &tv = s->ks.tma[s->tmaVar];
      tv.launch(&a, &mm, s->nBlkTma, tv.smem, s->stream);
      st = post_launch(s);
    } else {
      a.Uin_d = first ? Y[0] : nullptr;
      a.Uin_s = first ? nullptr : Y[k];
      a.U0 = Y[0];
      a.Uout = s->U;
      a.Wout = last ? nullptr : Y[k + 1];
      st = launch_stage_args(s, a);
    }
    if (st) return st;
    s->curTr ^= 1;
  }
  return FRG_OK;
}

frg_status adj_check_path(const frg_solver *s) {
  if (s->p.dtType != 0) return fail(FRG_ERR_ARG, "adjoint: fixed dt (dtType 0) required");
  if (s->p.timeType == 5) return fail(FRG_ERR_ARG, "adjoint: Jameson-form RK not supported");
  return FRG_OK;
}

}  // namespace

extern "C" {

}  // extern "C"

namespace {
// Partial-sum buffer of at least n doubles.
frg_status int_part(frg_solver *s, size_t n) {
  if (s->intPartCap >= n) return FRG_OK;
  if (s->intPart) CK(cudaFree(s->intPart));
  s->intPart = nullptr;
  CK(cudaMalloc(&s->intPart, n * 8));
  s->intPartCap = n;
  return FRG_OK;
}
// Sum of nOut components over nb blocks of partials, in block order.
frg_status sum_parts(frg_solver *s, int nb, int stride, int nOut, double *out) {
  std::vector<double> h((size_t)nb * stride);
  CK(cudaMemcpyAsync(h.data(), s->intPart, h.size() * 8, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  for (int j = 0; j < nOut; j++) {
    double t = 0;
    for (int b = 0; b < nb; b++) t += h[(size_t)b * stride + j];
    out[j] = t;
  }
  return FRG_OK;
}
// Traces of the current state and, for viscous runs, its corrected gradient
// at the solution points (what calcResidual(0) leaves in U_fpts / dU_spts).
frg_status boundary_inputs(frg_solver *s, BndIntArgs &b, int kind) {
  frg_status st;
  s->trValid = false;
  if ((st = ensure_traces(s))) return st;
  if (s->p.viscous) {
    StageArgs a = base_args(s);
    a.Uin_d = s->U;
    a.trIn = s->tr[s->curTr];
    a.dUg = s->dUg;
    a.flags = SF_RESIDUAL;
    s->ks.grad(&a, s->nBlk, s->ks.smem, s->stream);
    if ((st = post_launch(s))) return st;
  }
  if (!s->w1Dev) {
    CK(cudaMalloc(&s->w1Dev, 8 * (MAXP + 1)));
    CK(cudaMemcpy(s->w1Dev, s->ops.w, 8 * (MAXP + 1), cudaMemcpyHostToDevice));
  }
  b = BndIntArgs{};
  b.kind = kind;
  b.nDims = s->p.nDims;
  b.nV = s->nV;
  b.P = s->p.order;
  b.nF = s->nF;
  b.nFF = s->g.nFF;
  b.nS = s->nS;
  b.nE = s->nE;
  b.L = s->L;
  b.viscous = s->p.viscous;
  b.tr = s->tr[s->curTr];
  b.dUg = s->dUg;
  b.nbr = s->nbr;
  b.nrm = s->nrmOwn;
  b.dA = s->dAd;
  b.w1 = s->w1Dev;
  for (int side = 0; side < 2; side++)
    for (int j = 0; j <= MAXP; j++) b.lag[side][j] = s->ops.lag[side][j];
  b.ph = make_phys(s->p);
  return int_part(s, (size_t)boundary_integral_blocks(s->nF, s->L) * 6);
}
}  // namespace

extern "C" {

frg_status frg_wall_force(frg_solver *s, double *force) {
  if (!s || !force) return fail(FRG_ERR_ARG, "null argument");
  if (s->p.equation != 1) {
    for (int j = 0; j < 6; j++) force[j] = 0;
    return FRG_OK;
  }
  BndIntArgs b;
  frg_status st = boundary_inputs(s, b, 0);
  if (st) return st;
  CK(launch_boundary_integral(b, (int)s->sstore, s->intPart, s->stream));
  s->launches++;
  return sum_parts(s, boundary_integral_blocks(s->nF, s->L), 6, 6, force);
}

frg_status frg_mass_flux(frg_solver *s, int errorNorm, double *flux) {
  if (!s || !flux || errorNorm < 0 || errorNorm > 2) return fail(FRG_ERR_ARG, "bad arguments");
  BndIntArgs b;
  frg_status st = boundary_inputs(s, b, errorNorm + 1);
  if (st) return st;
  CK(launch_boundary_integral(b, (int)s->sstore, s->intPart, s->stream));
  s->launches++;
  return sum_parts(s, boundary_integral_blocks(s->nF, s->L), 6, s->nV, flux);
}

frg_status frg_integrate_error(frg_solver *s, int icType, double eps, int errorNorm, int quadOrder,
                               const double *box, double *err) {
  if (!s || !box || !err || errorNorm < 0 || errorNorm > 2) return fail(FRG_ERR_ARG, "bad arguments");
  const bool ns = s->p.equation == 1;
  if ((ns && icType != 0 && icType != 1) || (!ns && (icType < 0 || icType > 2)))
    return fail(FRG_ERR_ARG, "integrateError: icType %d has no analytic solution here", icType);
  const int d = s->p.nDims, nN = s->nNodes;
  // the node coordinates on the device (kept current by frg_update_geometry)
  if (!s->xvDev) {
    const size_t nX = (size_t)s->nE * nN * d;
    CK(cudaMalloc(&s->xvDev, nX * 8));
    CK(cudaMemcpy(s->xvDev, s->xvHost.data(), nX * 8, cudaMemcpyHostToDevice));
  }
  const int want = errorNorm == 0 ? -1 : quadOrder;
  int nQ = s->nS;
  if (s->qOrder != want) {
    std::vector<double> shp, itp, wq;
    std::string e;
    bool ok = want < 0 ? spt_shape_table(d, s->p.order, nN, shp, e)
                       : quad_tables(d, s->p.order, nN, quadOrder, shp, itp, wq, e);
    if (!ok) return fail(FRG_ERR_ARG, "%s", e.c_str());
    for (double **q : {&s->qShape, &s->qInterp, &s->qW})
      if (*q) { CK(cudaFree(*q)); *q = nullptr; }
    frg_status st;
    if ((st = upload_d(&s->qShape, shp))) return st;
    if (want >= 0 && ((st = upload_d(&s->qInterp, itp)) || (st = upload_d(&s->qW, wq)))) return st;
    s->qOrder = want;
  }
  if (want >= 0) nQ = d == 2 ? (quadOrder + 1) * (quadOrder + 1) : (quadOrder + 1) * (quadOrder + 1) * (quadOrder + 1);
  ErrIntArgs a{};
  a.nDims = d;
  a.nV = s->nV;
  a.nS = s->nS;
  a.nQ = nQ;
  a.nE = s->nE;
  a.L = s->L;
  a.nN = nN;
  a.icType = icType;
  a.errorNorm = errorNorm;
  a.U = s->U;
  a.detJ = s->detJd;
  a.xv = s->xvDev;
  a.interp = want >= 0 ? s->qInterp : nullptr;
  a.shape = s->qShape;
  a.wq = want >= 0 ? s->qW : s->wvol;
  for (int j = 0; j < 4; j++) a.box[j] = box[j];
  double t, dt;
  int it;
  frg_get_time(s, &t, &dt, &it);
  a.time = t;
  a.eps = eps;
  a.ph = make_phys(s->p);
  const int nb = error_integral_blocks(nQ, s->nE);
  frg_status st = int_part(s, (size_t)nb * 2 * s->nV);
  if (st) return st;
  CK(launch_error_integral(a, s->intPart, s->stream));
  s->launches++;
  std::vector<double> r(2 * s->nV);
  if ((st = sum_parts(s, nb, 2 * s->nV, 2 * s->nV, r.data()))) return st;
  for (int k = 0; k < s->nV; k++) {
    if (errorNorm == 0) err[k] = std::fabs(r[k] - r[s->nV + k]);
    else if (errorNorm == 2) err[k] = std::sqrt(std::fabs(r[k]));
    else err[k] = r[k];
  }
  return FRG_OK;
}

frg_status frg_objective(frg_solver *s, int kind, double *J, double *grad_host) {
  if (!s || !J) return fail(FRG_ERR_ARG, "null argument");
  frg_status st = adj_init(s);
  if (st) return st;
  AdjState *a = s->adj;
  const Phys ph = make_phys(s->p);
  int nPart = 0;
  if (kind == FRG_OBJ_ENTROPY) {
    if (!a->ks.entropy) return fail(FRG_ERR_ARG, "entropy objective needs the Euler equations");
    a->ks.entropy(s->U, s->detJd, s->wvol, s->nE, s->L, ph, a->grad, a->part, s->stream);
    nPart = a->ks.entropyBlocks;
  } else if (kind == FRG_OBJ_WALL_PRESSURE) {
    if (!a->ks.wallp) return fail(FRG_ERR_ARG, "wall-pressure objective needs the Euler equations");
    CK(cudaMemsetAsync(a->grad, 0, (size_t)s->nV * s->nS * s->L * 8, s->stream));
    a->ks.wallp(s->U, s->nbr, s->dAd, s->wsurf, s->p.vcjhScheme, s->nE, s->L, BC_SLIP, ph, a->grad, a->part,
                s->stream);
    nPart = (s->nE + 127) / 128;
  } else {
    return fail(FRG_ERR_ARG, "unknown objective %d", kind);
  }
  if ((st = post_launch(s))) return st;
  std::vector<double> part(nPart);
  CK(cudaMemcpyAsync(part.data(), a->part, nPart * 8, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  double t = 0;
  for (double x : part) t += x;
  *J = t;
  a->gradValid = true;
  if (grad_host) return state_to_host(s, a->grad, grad_host);
  return FRG_OK;
}

frg_status frg_residual_vjp(frg_solver *s, const double *gbar_host, const double *thetaDir, double *ubar_host,
                            double *thetaBar) {
  if (!s || !gbar_host || !ubar_host) return fail(FRG_ERR_ARG, "null argument");
  frg_status st = adj_init(s);
  if (st) return st;
  AdjState *ad = s->adj;
  if ((st = state_to_dev(s, gbar_host, ad->seed[0]))) return st;
  CK(cudaMemsetAsync(ad->thetaBar, 0, 8, s->stream));
  const double zero[5] = {0, 0, 0, 0, 0};
  CK(cudaMemcpy(ad->thetaDir, thetaDir ? thetaDir : zero, 5 * 8, cudaMemcpyHostToDevice));
  AdjArgs a = adj_args(s, s->U, ad->seed[0]);
  a.mode = ADJ_PLAIN;
  a.ybar = ad->ybar;
  if ((st = adj_launch(s, a))) return st;
  if (thetaBar) CK(cudaMemcpyAsync(thetaBar, ad->thetaBar, 8, cudaMemcpyDeviceToHost, s->stream));
  if ((st = state_to_host(s, ad->ybar, ubar_host))) return st;
  return check_flags(s);
}

frg_status frg_adjoint_forward(frg_solver *s, int nsteps, int checkpointEvery) {
  if (!s || nsteps < 1) return fail(FRG_ERR_ARG, "bad arguments");
  frg_status st;
  if ((st = adj_check_path(s)) || (st = adj_init(s))) return st;
  AdjState *a = s->adj;
  const size_t nSE = (size_t)s->nV * s->nS * s->L;
  if (checkpointEvery < 0) {
    // keep every stage state when they fit in half of the free memory (the
    // stage slots a previous run holds count as free)
    size_t freeB = 0, totalB = 0;
    CK(cudaMemGetInfo(&freeB, &totalB));
    const size_t held = (a->stages ? nSE * (size_t)a->stagesCap * s->nRK * 8 : 0) +
                        (a->stages2 ? nSE * (size_t)a->stagesCap * s->nRK * 8 : 0);
    const size_t need = nSE * (size_t)nsteps * s->nRK * 8;
    checkpointEvery = need <= (freeB + held) / 2 ? 0 : 25;
  }
  // checkpointEvery 0: keep every stage state of the run (no recomputation)
  const bool keepAll = checkpointEvery == 0;
  const int k = keepAll ? nsteps : std::min(checkpointEvery, nsteps);
  const int nCkpt = (nsteps + k - 1) / k;  // checkpoints at 0, k, ..., plus U_N
  CK(cudaStreamSynchronize(s->stream));
  adj_drop_graphs(a);  // they name the stage slots of the last run's layout
  if (a->ckpt && a->ckptCap < nCkpt + 1) { cudaFree(a->ckpt); a->ckpt = nullptr; }
  if (!a->ckpt) {
    if ((st = dalloc(&a->ckpt, nSE * (nCkpt + 1)))) return st;
    a->ckptCap = nCkpt + 1;
  }
  if (a->stages && a->stagesCap < k) {
    cudaFree(a->stages);
    cudaFree(a->stages2);
    a->stages = a->stages2 = nullptr;
  }
  if (!a->stages) {
    if ((st = dalloc(&a->stages, nSE * (size_t)k * s->nRK))) return st;
    a->stagesCap = k;
  }
  // the overlap's second slot set; without the memory the sweep runs serially
  if (!keepAll && nCkpt > 1 && !a->stages2 &&
      cudaMalloc(&a->stages2, nSE * (size_t)a->stagesCap * s->nRK * 8) != cudaSuccess) {
    cudaGetLastError();
    a->stages2 = nullptr;
  }
  a->k = k;
  a->nSteps = nsteps;
  a->keepAll = keepAll;
  if (keepAll) {
    CK(cudaMemcpyAsync(a->ckpt, s->U, nSE * 8, cudaMemcpyDeviceToDevice, s->stream));
    if ((st = ensure_traces(s))) return st;
    std::vector<double *> Y(s->nRK);
    for (int n = 0; n < nsteps; n++) {
      for (int q = 0; q < s->nRK; q++) Y[q] = a->stages + nSE * ((size_t)n * s->nRK + q);
      if ((st = step_keep_stages(s, Y.data(), true))) return st;
      s->iter++;
    }
    s->trValid = true;
    s->dtFresh = false;
  } else {
    for (int n = 0; n < nsteps; n += k) {
      CK(cudaMemcpyAsync(a->ckpt + nSE * (n / k), s->U, nSE * 8, cudaMemcpyDeviceToDevice, s->stream));
      if ((st = frg_update(s, std::min(k, nsteps - n)))) return st;
    }
  }
  CK(cudaMemcpyAsync(a->ckpt + nSE * nCkpt, s->U, nSE * 8, cudaMemcpyDeviceToDevice, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return check_flags(s);
}

frg_status frg_adjoint_mode(const frg_solver *s, int *checkpointEvery) {
  if (!s || !checkpointEvery) return fail(FRG_ERR_ARG, "null argument");
  if (!s->adj || s->adj->nSteps < 1) return fail(FRG_ERR_ARG, "adjoint: no recorded forward run (frg_adjoint_forward)");
  *checkpointEvery = s->adj->keepAll ? 0 : s->adj->k;
  return FRG_OK;
}

frg_status frg_adjoint_backward(frg_solver *s, const double *lamN_host, const double *thetaDir, double *lam0_host,
                                double *thetaBar) {
  if (!s) return fail(FRG_ERR_ARG, "null handle");
  AdjState *ad = s->adj;
  if (!ad || ad->nSteps < 1) return fail(FRG_ERR_ARG, "adjoint: no recorded forward run (frg_adjoint_forward)");
  frg_status st;
  const size_t nSE = (size_t)s->nV * s->nS * s->L;
  const int nRK = s->nRK, k = ad->k, N = ad->nSteps, nCkpt = (N + k - 1) / k;
  if (lamN_host) {
    if ((st = state_to_dev(s, lamN_host, ad->lam[0]))) return st;
  } else {
    if (!ad->gradValid) return fail(FRG_ERR_ARG, "adjoint: no seed and no objective gradient");
    CK(cudaMemcpyAsync(ad->lam[0], ad->grad, nSE * 8, cudaMemcpyDeviceToDevice, s->stream));
  }
  CK(cudaMemsetAsync(ad->thetaBar, 0, 8, s->stream));
  const double zero[5] = {0, 0, 0, 0, 0};
  CK(cudaMemcpy(ad->thetaDir, thetaDir ? thetaDir : zero, 5 * 8, cudaMemcpyHostToDevice));
  const double dt = s->p.dt;  // fixed dt (dtType 0)
  const int nb = (int)std::min<size_t>((nSE + 255) / 256, 148 * 8);
  // (ensemble mode: the per-group fixed dt multiplies per element)
  fr_adj_seed_kernel<<<nb, 256, 0, s->stream>>>(ad->lam[0], s->detJd, ad->seed[0],
                                                 -s->RKb[nRK - 1] * (s->grp ? 1.0 : dt), s->nV, s->nS, s->nE, s->L,
                                                 s->grp, s->grpDt);
  if ((st = post_launch(s))) return st;
  int cl = 0, cs = 0;  // current lam / seed buffers
  // Checkpointed runs recompute segment c-1 from its checkpoint on the side
  // stream while segment c is reversed on the solver's stream: the
  // recomputation writes U, the RK accumulator, the traces and the other set
  // of stage slots; the reversal reads only its own slots, the metrics and
  // the adjoint buffers.  The solver's stream waits for the side stream
  // before the next segment.  Without the second slot set: one after the other.
  const bool overlap = !ad->keepAll && ad->stages2 && nCkpt > 1;
  double *const bufs[2] = {ad->stages, overlap ? ad->stages2 : ad->stages};
  const cudaStream_t mainSt = s->stream;
  // recompute segment c into slot set b, keeping every stage state; one
  // captured graph per segment length, trace-buffer parity and slot set
  auto recompute = [&](int c, int b) -> frg_status {
    const int m = std::min(k, N - c * k);
    double *seg = bufs[b];
    CK(cudaMemcpyAsync(s->U, ad->ckpt + nSE * c, nSE * 8, cudaMemcpyDeviceToDevice, s->stream));
    s->trValid = false;
    frg_status e = ensure_traces(s);
    if (e) return e;
    const int tr0 = s->curTr;
    e = adj_replay(s, {2 * b, m, tr0, 0}, [&]() {
      std::vector<double *> Y(nRK);
      for (int j = 0; j < m; j++) {
        for (int q = 0; q < nRK; q++) Y[q] = seg + nSE * ((size_t)j * nRK + q);
        frg_status e2 = step_keep_stages(s, Y.data());
        if (e2) return e2;
      }
      return FRG_OK;
    });
    if (e) return e;
    s->curTr = tr0 ^ ((m * nRK) & 1);
    return FRG_OK;
  };
  if (!ad->keepAll && (st = recompute(nCkpt - 1, 0))) return st;
  int cur = 0;  // slot set holding the segment being reversed
  for (int c = nCkpt - 1; c >= 0; c--) {
    const int n0 = c * k, m = std::min(k, N - n0);
    double *seg = bufs[cur];
    const bool fork = overlap && c > 0;
    if (fork) {
      CK(cudaEventRecord(ad->evFork, mainSt));
      CK(cudaStreamWaitEvent(ad->side, ad->evFork, 0));
      s->stream = ad->side;
      st = recompute(c - 1, cur ^ 1);
      s->stream = mainSt;
      if (st) return st;
      CK(cudaEventRecord(ad->evJoin, ad->side));
    }
    // reverse the segment, stage by stage (captured when checkpointed: the
    // same slots serve every segment; a kept-all run is reversed once, launch
    // by launch)
    const int cl0 = cl, cs0 = cs;
    auto reverse = [&]() {
      int l = cl0, q2 = cs0;
      for (int j = m - 1; j >= 0; j--) {
        for (int q = nRK - 1; q >= 0; q--) {
          AdjArgs a = adj_args(s, seg + nSE * ((size_t)j * nRK + q), ad->seed[q2]);
          a.mode = ADJ_RK | (q == nRK - 1 ? ADJ_RK_FIRST : 0) | (q == 0 ? ADJ_RK_LAST : 0);
          a.lam = ad->lam[l];
          a.lamNew = ad->lam[l ^ 1];
          a.seedOut = ad->seed[q2 ^ 1];
          a.cLam = q == 0 ? s->RKb[nRK - 1] : s->RKb[q - 1];
          a.cY = q == 0 ? 0.0 : s->RKa[q];
          a.dt = dt;
          frg_status e = adj_launch(s, a);
          if (e) return e;
          q2 ^= 1;
        }
        l ^= 1;
      }
      return FRG_OK;
    };
    st = ad->keepAll ? reverse() : adj_replay(s, {1 + 2 * cur, m, cl0, cs0}, reverse);
    if (st) return st;
    cs = cs0 ^ ((m * nRK) & 1);
    cl = cl0 ^ (m & 1);
    if (fork) {
      CK(cudaStreamWaitEvent(mainSt, ad->evJoin, 0));
      cur ^= 1;
    } else if (!ad->keepAll && c > 0 && (st = recompute(c - 1, 0))) {
      return st;
    }
  }
  // the solution is the forward run's final state again
  CK(cudaMemcpyAsync(s->U, ad->ckpt + nSE * nCkpt, nSE * 8, cudaMemcpyDeviceToDevice, s->stream));
  s->trValid = false;
  if (thetaBar) CK(cudaMemcpyAsync(thetaBar, ad->thetaBar, 8, cudaMemcpyDeviceToHost, s->stream));
  if (lam0_host && (st = state_to_host(s, ad->lam[cl], lam0_host))) return st;
  CK(cudaStreamSynchronize(s->stream));
  return check_flags(s);
}

}  // extern "C"

// ==================================================================== ensemble
// Several handles (one per order of a batch of cases) advanced together: each
// step is ONE graph launch whose parallel branches are the handles' own
// captured steps (child graphs), so the orders' kernels share the GPU.

struct frg_ensemble {
  std::vector<frg_solver *> ss;
  cudaStream_t stream = nullptr, ownStream = nullptr;
  std::map<std::vector<int>, cudaGraphExec_t> graphs;  // per combination of the handles' step keys
  std::vector<unsigned> epochs;                        // the handles' graph epochs the graphs were built at
};

extern "C" {

frg_status frg_ensemble_create(frg_solver *const *solvers, int n, frg_ensemble **out) {
  if (!solvers || n < 1 || !out) return fail(FRG_ERR_ARG, "bad arguments");
  for (int i = 0; i < n; i++) {
    if (!solvers[i]) return fail(FRG_ERR_ARG, "null handle %d", i);
    if (solvers[i]->p.timeType == 0 && solvers[i]->p.dtType != 0)
      return fail(FRG_ERR_ARG, "handle %d: Forward Euler with CFL dt is not fused", i);
  }
  std::unique_ptr<frg_ensemble> e(new frg_ensemble);
  e->ss.assign(solvers, solvers + n);
  CK(cudaStreamCreateWithFlags(&e->ownStream, cudaStreamNonBlocking));
  e->stream = e->ownStream;
  *out = e.release();
  return FRG_OK;
}

frg_status frg_ensemble_set_stream(frg_ensemble *e, void *stream) {
  if (!e) return fail(FRG_ERR_ARG, "null ensemble");
  CK(cudaStreamSynchronize(e->stream));
  e->stream = stream ? (cudaStream_t)stream : e->ownStream;
  return FRG_OK;
}

frg_status frg_ensemble_update(frg_ensemble *e, int nsteps) {
  if (!e || nsteps < 0) return fail(FRG_ERR_ARG, "bad arguments");
  frg_status st;
  std::vector<unsigned> ep;
  for (frg_solver *s : e->ss) {
    if ((st = ensure_traces(s))) return st;
    CK(cudaStreamSynchronize(s->stream));
    ep.push_back(s->graphEpoch);
  }
  if (ep != e->epochs) {  // a handle re-captured its steps: rebuild
    for (auto &g : e->graphs) cudaGraphExecDestroy(g.second);
    e->graphs.clear();
    e->epochs = ep;
  }
  const size_t n = e->ss.size();
  std::vector<int> key(3 * n), mode(n);
  for (int step = 0; step < nsteps; step++) {
    for (size_t i = 0; i < n; i++) {
      frg_solver *s = e->ss[i];
      s->iter++;
      mode[i] = dt_mode(s);
      key[3 * i] = mode[i];
      key[3 * i + 1] = s->curTr;
      key[3 * i + 2] = s->dtCur;
    }
    auto it = e->graphs.find(key);
    if (it == e->graphs.end()) {
      cudaGraph_t g;
      CK(cudaGraphCreate(&g, 0));
      for (size_t i = 0; i < n; i++) {
        cudaGraph_t raw;
        if ((st = step_graph(e->ss[i], mode[i], nullptr, &raw))) return st;
        cudaGraphNode_t node;
        CK(cudaGraphAddChildGraphNode(&node, g, nullptr, 0, raw));
      }
      cudaGraphExec_t ex;
      CK(cudaGraphInstantiate(&ex, g, 0));
      CK(cudaGraphDestroy(g));
      it = e->graphs.emplace(key, ex).first;
    }
    CK(cudaGraphLaunch(it->second, e->stream));
    for (size_t i = 0; i < n; i++) step_done(e->ss[i], mode[i]);
  }
  CK(cudaStreamSynchronize(e->stream));
  for (frg_solver *s : e->ss) {
    if (nsteps > 0) s->divF0Valid = s->monitor;
    if ((st = check_flags(s))) return st;
  }
  return FRG_OK;
}

frg_status frg_ensemble_destroy(frg_ensemble *e) {
  if (!e) return FRG_OK;
  if (e->stream) cudaStreamSynchronize(e->stream);
  for (auto &g : e->graphs) cudaGraphExecDestroy(g.second);
  if (e->ownStream) cudaStreamDestroy(e->ownStream);
  delete e;
  return FRG_OK;
}

}  // extern "C"
