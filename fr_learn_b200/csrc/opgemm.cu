// opgemm.cu -- the FR operator matrices applied as batched dense GEMMs on the
// 5th-generation tensor cores (tcgen05), fed by TMA, in 3xTF32 split precision
// with FP32 accumulation in tensor memory.
//
// The reference applies every operator of its `oper` object as one row-major
// dgemm over all elements (oper::applySptsFpts, applyGradSpts,
// applyExtrapolateFn, applyCorrectDivF, applyCorrectGradU,
// src/operators.cpp:1191-1450): Y[M][nEles*nFields] = Op[M][K] X[K][...].
// Here the arrays are [field][point][element] with the element index fastest,
// so per field Y_v = Op X_v, computed transposed: for a tile of 128 elements,
//
//   D[e][m] = sum_k A[e][k] B[k][m],   A = X_v^T (M = elements),
//   B = Op^T (N = output points)
//
// A is read MN-major (elements contiguous) straight from the layout TMA lands
// the tile in: four boxes of 32 elements x KP points, each row of 128 bytes
// with its 32-byte chunks swizzled across 4-row groups -- the one MN-major
// layout the TF32 MMA accepts, SWIZZLE_128B_BASE32B (4-row x 128-byte atoms;
// 32-element groups LBO = KP * 128 bytes apart, 4-row groups 512 bytes apart),
// which TMA writes with CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B.  (The plain
// 128-byte swizzle, 16-byte chunks across 8 rows, is valid MN-major for
// 16-bit operands; for TF32 the MMA produced zeros from it.)  B (the operator, prepared on
// the host) is K-major without swizzle (8-row x 16-byte core matrices).  The
// accumulator's TMEM lane is the element and its column the output point:
// warp w reads lanes 32w..32w+31 and its 32 threads store 32 consecutive
// elements of each output point -- coalesced rows of Y.
//
// Split precision: x = hi + lo.  The tensor core reads a TF32 operand from
// an fp32 bit pattern with the low 13 mantissa bits dropped, so X's hi half
// is the landed tile itself (read as trunc(x)) and its lo half is the exact
// remainder x - trunc(x) (the same bits cleared by a mask, then a subtraction),
// formed by the block after the tile lands, elementwise at the same offsets
// of a second buffer: the swizzled positions need no reordering.  (Measured:
// were the low bits rounded instead, this split would be ~2^-11 off and the
// 1e-5 accuracy tests fail.)  Op's halves are prepared on the host: hi =
// tf32(op) to nearest, lo = tf32(op - hi).  D = A_hi B_hi + A_lo B_hi +
// A_hi B_lo; the dropped A_lo B_lo term and the truncation of the lo halves
// are ~2^-20 relative.
//
// Persistent blocks over (128-element tile, field) pairs, warp-specialised: a
// producer warp lands tiles (four [KP][32] boxes each, the operator image once
// as two bulk copies) in a ring of slots, four warps form the lo halves, one
// warp issues the MMAs into two TMEM accumulators in turn, eight warps drain
// them, all coupled by mbarriers, so a tile's load, split, MMAs and drain
// overlap the neighbouring tiles'.  Every wait is bounded; on expiry the block
// flags an error, lets its copies and MMAs land (bounded again), frees its
// TMEM and returns.  No multicast.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "dispatch.h"
#include "kernels_tma.cuh"

namespace frg {

// Shared-memory matrix descriptor (tcgen05 matrix descriptor): start,
// leading and stride byte offsets in 16-byte units (bits 0-13, 16-29,
// 32-45), version 1 in bits 46-47, base offset 0, layout type in bits 61-63
// (0: no swizzle, 1: 128-byte swizzle of 32-byte chunks).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo, uint32_t layout = 0) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | ((uint64_t)layout << 61);
}
constexpr uint32_t kLayoutSW128Base32 = 1;

// Instruction descriptor of kind::tf32: F32 accumulator (bits 4-5), TF32 A
// and B (bits 7-9, 10-12), A MN-major (bit 15), B K-major (bit 16 clear),
// N >> 3 in bits 17-22, M >> 4 in bits 24-28 with M = 128.
__host__ __device__ constexpr uint32_t idesc_tf32(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | (1u << 15) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
      "l"(ad), "l"(bd), "r"(idesc), "r"(accum)
      : "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_free(uint32_t tmem, int ncol) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncol) : "memory");
}

__device__ __forceinline__ void tma_load3d(void *dst, const CUtensorMap *m, int x, int y, int z, uint64_t *b) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(m), "r"(x), "r"(y), "r"(z), "r"(smem_u32(b))
      : "memory");
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *b) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(b))
               : "memory");
}

// Y_v = Op X_v (+ beta Y_v) over tiles of 128 elements of one field; tile t
// covers elements [128 (t % nT), +128) of field t / nT, nT = ceil(nEle/128).
// Persistent, one block per SM (block b takes tiles b, b + gridDim.x, ...),
// the work split by warps so that consecutive tiles overlap:
//   warp 8     producer: the operator image once, then each tile's four TMA
//              boxes into one of nA landing slots (a slot is reused once the
//              MMAs that read it have completed);
//   warps 4-7  split: the lo half of a landed tile into the lo buffer (once
//              the previous tile's MMAs have read that buffer);
//   warp 9     MMA: 3 x KP/8 tcgen05.mma of a split tile into one of two TMEM
//              accumulators (once the epilogue has drained it), then commits
//              to the accumulator's, the slot's and the lo buffer's mbarriers;
//   warps 0-3, 10-13  epilogue: drain an accumulator and store Y (warp w
//              reads TMEM lanes 32(w%4)..+31; warps 0-3 the first half of the
//              columns, warps 10-13 the second).
// While tile j is drained, tile j+1 is split and multiplied and the tiles up
// to j+nA land.  KP: K padded to a multiple of 8; NP: output points padded to
// a multiple of 16; M: real output points; ncol: TMEM columns per accumulator
// (a power of two >= NP; two accumulators).  Bimg: the operator image (see
// build_op_image).  mX: 3D map [field][K][ld] with box {32, KP, 1} and the
// 128-byte swizzle of 32-byte chunks.  Shared memory (1024-byte aligned): nA
// landing slots (each 4 x [KP][32], the A_hi operand as it lands), the A_lo
// buffer, the image (hi, then lo), then the mbarriers, the TMEM address and
// an abort word.  Every wait is bounded and warp-uniform: a wait that gives
// up sets the abort word, every role then leaves its loop, the producer lets
// its issued copies land and the MMA warp its issued MMAs complete (bounded
// again), the block flags ERRF_TIMEOUT and frees its TMEM.
constexpr int kOgThreads = 448;
constexpr int kOgMaxSlots = 4;
struct OgBars {
  uint64_t full[kOgMaxSlots], slotFree[kOgMaxSlots], img, splitDone, loFree, accFull[2], accEmpty[2];
  uint32_t tmem;
  int abort;
};
constexpr int kOgBarBytes = 256;
static_assert(sizeof(OgBars) <= kOgBarBytes, "barrier block");

__device__ __forceinline__ void mbar_arrive(uint64_t *b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
// Bounded, warp-uniform wait for an mbarrier phase (mask: the calling lanes):
// false when it gives up (then the abort word is set) or another role has
// aborted.
__device__ __forceinline__ bool og_wait(uint64_t *b, uint32_t par, volatile int *abortF, unsigned mask) {
  for (int i = 0; i < (1 << 22); i++) {
    const bool done = mbar_try_wait(b, par);
    if (__all_sync(mask, done)) return true;
    if ((i & 63) == 63 && __any_sync(mask, *abortF != 0)) return false;
  }
  *abortF = 1;
  return false;
}

__global__ void __launch_bounds__(kOgThreads, 1)
    fr_op_gemm_tc_kernel(const __grid_constant__ CUtensorMap mX, const float *__restrict__ Bimg, float *Y, int KP,
                         int NP, int M, int ncol, int nA, int ld, int nEle, int nV, float beta, unsigned *err) {
  // the swizzled tiles need 1024-byte alignment; the dynamic shared memory
  // starts there (checked: no slack is allocated)
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *const sb = smem_raw;
  if (smem_u32(smem_raw) & 1023u) {
    if (threadIdx.x == 0) atomicOr(err, ERRF_ALIGN);
    return;
  }
  const uint32_t aBytes = (uint32_t)KP * 512u;    // KP points x 128 elements x 4 bytes
  const uint32_t boxBytes = (uint32_t)KP * 128u;  // one [KP][32] box: the stride between 32-element groups
  const uint32_t bHalf = (uint32_t)KP * NP * 4u;
  unsigned char *const slots = sb;  // nA x aBytes
  float *const Alo = reinterpret_cast<float *>(sb + (size_t)nA * aBytes);
  unsigned char *const Bs = sb + (size_t)(nA + 1) * aBytes;  // hi, then lo
  OgBars *const sh = reinterpret_cast<OgBars *>(Bs + 2 * (size_t)bHalf);
  volatile int *const abortF = &sh->abort;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nT = (nEle + 127) / 128, nTiles = nT * nV;
  if ((int)blockIdx.x >= nTiles) return;

  if (tid == 0) {
    for (int s = 0; s < kOgMaxSlots; s++) {
      mbar_init(&sh->full[s], 1);
      mbar_init(&sh->slotFree[s], 1);
    }
    mbar_init(&sh->img, 1);
    mbar_init(&sh->splitDone, 128);
    mbar_init(&sh->loFree, 1);
    for (int a = 0; a < 2; a++) {
      mbar_init(&sh->accFull[a], 1);
      mbar_init(&sh->accEmpty[a], 256);
    }
    sh->abort = 0;
    fence_mbar_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sh->tmem)),
                 "r"(2 * ncol)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sh->tmem;

  if (warp == 8) {
    if (lane == 0) {
      // ---- producer
      int last[kOgMaxSlots];
      for (int s = 0; s < kOgMaxSlots; s++) last[s] = -1;
      mbar_expect_tx(&sh->img, 2u * bHalf);
      bulk_load(Bs, Bimg, bHalf, &sh->img);
      bulk_load(Bs + bHalf, reinterpret_cast<const unsigned char *>(Bimg) + bHalf, bHalf, &sh->img);
      for (int j = 0;; j++) {
        const int t = blockIdx.x + j * gridDim.x;
        if (t >= nTiles) break;
        const int s = j % nA;
        // the MMAs of the tile that used this slot before have read it
        if (j >= nA && !og_wait(&sh->slotFree[s], (uint32_t)(((j / nA) - 1) & 1), abortF, 1u)) break;
        mbar_expect_tx(&sh->full[s], aBytes);
        for (int q = 0; q < 4; q++)
          tma_load3d(slots + (size_t)s * aBytes + q * boxBytes, &mX, (t % nT) * 128 + 32 * q, 0, t / nT,
                     &sh->full[s]);
        last[s] = j;
      }
      // every issued copy lands before the block may exit (bounded)
      mbar_wait(&sh->img, 0);
      for (int s = 0; s < kOgMaxSlots; s++)
        if (last[s] >= 0) mbar_wait(&sh->full[s], (uint32_t)((last[s] / nA) & 1));
    }
    __syncwarp();
  } else if (warp == 9) {
    if (lane == 0) {
      // ---- MMA issuer
      const uint32_t idesc = idesc_tf32(NP);
      int lastJ = -1;
      if (og_wait(&sh->img, 0, abortF, 1u)) {
        for (int j = 0;; j++) {
          const int t = blockIdx.x + j * gridDim.x;
          if (t >= nTiles) break;
          const int s = j % nA, acc = j & 1;
          if (!og_wait(&sh->splitDone, (uint32_t)(j & 1), abortF, 1u)) break;
          // the epilogue has drained this accumulator's previous tile
          if (j >= 2 && !og_wait(&sh->accEmpty[acc], (uint32_t)(((j >> 1) - 1) & 1), abortF, 1u)) break;
          tc_fence_after();
          const uint32_t aHi = smem_u32(slots + (size_t)s * aBytes), aLo = smem_u32(Alo), bHi = smem_u32(Bs),
                         bLo = bHi + bHalf;
          const uint32_t d = tmem + (uint32_t)(acc * ncol);
          // A (MN-major, 32-byte-chunk swizzle): K step k is rows 8k..8k+7,
          // two 512-byte atoms of 4 rows, in every box; the boxes boxBytes
          // apart (leading offset), 4-row groups 512 bytes apart (stride
          // offset).  B (K-major, no swizzle): the two K halves 128 bytes
          // apart (leading offset), 8-row groups 256 bytes apart (stride
          // offset), NP/8 groups per K step
          for (int k = 0; k < KP / 8; k++) {
            const uint64_t ah = smem_desc(aHi + k * 1024, boxBytes, 512, kLayoutSW128Base32);
            const uint64_t al = smem_desc(aLo + k * 1024, boxBytes, 512, kLayoutSW128Base32);
            const uint64_t bh = smem_desc(bHi + k * NP * 32, 128, 256);
            const uint64_t bl = smem_desc(bLo + k * NP * 32, 128, 256);
            tc_mma(d, ah, bh, idesc, k > 0 ? 1u : 0u);
            tc_mma(d, al, bh, idesc, 1u);
            tc_mma(d, ah, bl, idesc, 1u);
          }
          // each commit arrives once these MMAs have completed
          tc_commit(&sh->accFull[acc]);
          tc_commit(&sh->slotFree[s]);
          tc_commit(&sh->loFree);
          lastJ = j;
        }
      }
      // every issued MMA completes before TMEM is freed (bounded)
      if (lastJ >= 0) mbar_wait(&sh->loFree, (uint32_t)(lastJ & 1));
    }
    __syncwarp();
  } else if (warp >= 4 && warp < 8) {
    // ---- split: lo halves, elementwise (the swizzle moves whole 32-byte
    // chunks, so lo keeps the landed positions); the landed tile is the hi
    // operand as it is
    for (int j = 0;; j++) {
      const int t = blockIdx.x + j * gridDim.x;
      if (t >= nTiles) break;
      const int s = j % nA;
      if (!og_wait(&sh->full[s], (uint32_t)((j / nA) & 1), abortF, 0xffffffffu)) break;
      // the previous tile's MMAs have read the lo buffer
      if (j >= 1 && !og_wait(&sh->loFree, (uint32_t)((j - 1) & 1), abortF, 0xffffffffu)) break;
      const uint4 *S4 = reinterpret_cast<const uint4 *>(slots + (size_t)s * aBytes);
      float4 *L4 = reinterpret_cast<float4 *>(Alo);
      for (int i = tid - 128; i < KP * 32; i += 128) {
        const uint4 x = S4[i];
        float4 l;
        l.x = __uint_as_float(x.x) - __uint_as_float(x.x & 0xFFFFE000u);
        l.y = __uint_as_float(x.y) - __uint_as_float(x.y & 0xFFFFE000u);
        l.z = __uint_as_float(x.z) - __uint_as_float(x.z & 0xFFFFE000u);
        l.w = __uint_as_float(x.w) - __uint_as_float(x.w & 0xFFFFE000u);
        L4[i] = l;
      }
      fence_proxy_async();  // the lo half is visible to the MMAs
      mbar_arrive(&sh->splitDone);
    }
  } else {
    // ---- epilogue: lane = element, columns = output points; two groups of
    // four warps, one per half of the columns
    const int quad = warp & 3, half = ((NP / 16 + 1) / 2) * 16;
    const int cb = warp < 4 ? 0 : half, ce = warp < 4 ? half : NP;
    for (int j = 0;; j++) {
      const int t = blockIdx.x + j * gridDim.x;
      if (t >= nTiles) break;
      const int acc = j & 1;
      if (!og_wait(&sh->accFull[acc], (uint32_t)((j >> 1) & 1), abortF, 0xffffffffu)) break;
      tc_fence_after();
      const int e = (t % nT) * 128 + 32 * quad + lane, v = t / nT;
      const uint32_t trow = tmem + (uint32_t)(acc * ncol) + ((uint32_t)(32 * quad) << 16);
      // up to 64 columns in flight per wait (four 16-column loads)
      for (int c1 = cb; c1 < ce; c1 += 64) {
        uint32_t r[64];
#pragma unroll
        for (int u = 0; u < 4; u++)
          if (c1 + 16 * u < ce)
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                "%13, %14, %15}, [%16];"
                : "=r"(r[16 * u + 0]), "=r"(r[16 * u + 1]), "=r"(r[16 * u + 2]), "=r"(r[16 * u + 3]),
                  "=r"(r[16 * u + 4]), "=r"(r[16 * u + 5]), "=r"(r[16 * u + 6]), "=r"(r[16 * u + 7]),
                  "=r"(r[16 * u + 8]), "=r"(r[16 * u + 9]), "=r"(r[16 * u + 10]), "=r"(r[16 * u + 11]),
                  "=r"(r[16 * u + 12]), "=r"(r[16 * u + 13]), "=r"(r[16 * u + 14]), "=r"(r[16 * u + 15])
                : "r"(trow + (uint32_t)(c1 + 16 * u)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (e < nEle) {
          float *y = Y + ((size_t)v * M + c1) * ld + e;
          const int nq = min(min(64, ce - c1), M - c1);
          if (beta == 0.f) {  // plain stores: no read of Y
#pragma unroll
            for (int q = 0; q < 64; q++)
              if (q < nq) __stcs(y + (size_t)q * ld, __uint_as_float(r[q]));
          } else {
#pragma unroll
            for (int q = 0; q < 64; q++)
              if (q < nq) y[(size_t)q * ld] = fmaf(beta, y[(size_t)q * ld], __uint_as_float(r[q]));
          }
        }
      }
      // the accumulator is free for the MMAs of tile j + 2
      tc_fence_before();
      mbar_arrive(&sh->accEmpty[acc]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (tid == 0 && *abortF) atomicOr(err, ERRF_TIMEOUT);
  if (warp == 0) {
    tc_fence_after();
    tmem_free(tmem, 2 * ncol);
  }
}

// ---------------------------------------------------------------- host side

static float tf32_round_host(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  if ((u & 0x7F800000u) != 0x7F800000u) u = (u + 0x1000u) & 0xFFFFE000u;  // nearest, ties away from zero
  else u &= 0xFFFFE000u;
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

// Operator image for B = Op^T (K-major): for K step s, 8-row group g of
// output points, K half h: an 8 x 4 core matrix, rows = output points
// 8g..8g+7, columns = inputs 8s+4h..+3; hi halves first, then lo halves.
void build_op_image(const double *op, int M, int K, int KP, int NP, std::vector<float> &img) {
  img.assign((size_t)2 * KP * NP, 0.f);
  const size_t half = (size_t)KP * NP;
  for (int s = 0; s < KP / 8; s++)
    for (int g = 0; g < NP / 8; g++)
      for (int h = 0; h < 2; h++)
        for (int r = 0; r < 8; r++)
          for (int c = 0; c < 4; c++) {
            const int n = 8 * g + r, k = 8 * s + 4 * h + c;
            const size_t o = (size_t)s * NP * 8 + (size_t)g * 64 + h * 32 + r * 4 + c;
            if (n >= M || k >= K) continue;
            const double x = op[(size_t)n * K + k];
            const float hi = tf32_round_host((float)x);
            const float lo = tf32_round_host((float)(x - (double)hi));
            img[o] = hi;
            img[half + o] = lo;
          }
}

// Landing slots for a KP x NP operator: as many as fit (at most kOgMaxSlots)
// beside the lo buffer and the image; 0 when fewer than two fit.
static int op_gemm_slots(int KP, int NP) {
  const size_t a = (size_t)KP * 512, fixed = a + (size_t)2 * KP * NP * 4 + kOgBarBytes;
  if (fixed + 2 * a > (size_t)227 * 1024) return 0;
  return (int)std::min<size_t>(kOgMaxSlots, ((size_t)227 * 1024 - fixed) / a);
}
size_t op_gemm_smem(int KP, int NP) {
  const int n = std::max(2, op_gemm_slots(KP, NP));
  return (size_t)(n + 1) * KP * 512 + (size_t)2 * KP * NP * 4 + kOgBarBytes;
}

cudaError_t launch_op_gemm(const CUtensorMap &mX, const float *Bimg, float *Y, int KP, int NP, int M, int ld,
                           int nEle, int nV, float beta, unsigned *err, cudaStream_t st) {
  int ncol = 32;
  while (ncol < NP) ncol <<= 1;
  const int nA = op_gemm_slots(KP, NP);
  if (nA < 2) return cudaErrorInvalidValue;
  size_t smem = op_gemm_smem(KP, NP);
  // keep (blocks per SM) x (TMEM columns of a block) within the SM's 512
  // columns, so a block never waits for another's allocation: with at most B
  // blocks allowed, each takes more than 1/(B+1) of the shared memory
  const size_t allowed = (size_t)(512 / (2 * ncol));
  const size_t minSmem = (size_t)(227 * 1024) / (allowed + 1) + 1;
  if (smem < minSmem) smem = minSmem;
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  // per device, once: the kernel's shared-memory limit and carveout, and the
  // SM count (host calls kept off the per-launch path)
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  static std::mutex mu;
  static std::map<int, int> smCount;
  int nSM = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = smCount.find(dev);
    if (it == smCount.end()) {
      e = cudaFuncSetAttribute(fr_op_gemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fr_op_gemm_tc_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
      if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nSM, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return e;
      smCount[dev] = nSM;
    } else {
      nSM = it->second;
    }
  }
  int occ = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fr_op_gemm_tc_kernel, kOgThreads, smem);
  if (e != cudaSuccess) return e;
  const int nTiles = (nEle + 127) / 128 * nV;
  const int grid = std::max(1, std::min(nTiles, nSM * std::max(occ, 1)));
  fr_op_gemm_tc_kernel<<<grid, kOgThreads, smem, st>>>(mX, Bimg, Y, KP, NP, M, ncol, nA, ld, nEle, nV, beta, err);
  return cudaGetLastError();
}

}  // namespace frg
