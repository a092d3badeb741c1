// FP64 chi0 contraction with TMA-staged operands (the plain-FP64 drop-in path).
//
//   eps(iw)[i][j] = delta_ij + sum_t M[t][i] D_w(t) M[t][j]      upper 64 x 128 tiles
//
// M is the transition-major packed tensor mp [nia_pad][npad] (auxiliary index
// contiguous).  Per k-tile of 16 transitions one thread issues TMA loads of
// 16 x 16 FP64 boxes with 128-byte swizzle (4 boxes for the 64 rows of the
// tile, 8 for its 128 columns) and of the 16 factors D_w(t) into a ring of four
// stages; four warps run the DMMA fragments (m8n8k4) from it, D_w applied to
// the A fragments as they are read (the element-wise scaling fused into the
// GEMM prologue).  Stages are recycled through mbarriers: lane 0 of warp 0
// refills the stage of k-tile kt - 2 with k-tile kt + 2 once every warp has
// released it, so the warps may drift by a k-tile instead of meeting at a
// block barrier every 16 transitions.  The fragment ownership, the MMA order
// over k and the epilogue are those of dgemm_mn_kernel<64, 128>, which stays
// the engine of the 128-row items.  All mbarrier waits are bounded.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "engine.cuh"
#include "tc_common.cuh"

namespace rigw {

namespace {

constexpr int kF64Stages = 4;
constexpr int kF64Lag = 2;                      // k-tiles between reading a stage and refilling it
constexpr int kF64Box = 16 * 16 * 8;            // 2 KB: 16 transitions x 16 auxiliary functions
constexpr int kF64OffB = 4 * kF64Box;           // 8 KB of A boxes, then 16 KB of B boxes
constexpr int kF64OffD = 12 * kF64Box;          // then the 16 factors D_w(t)
constexpr int kF64StageBytes = 25 * 1024;       // 24 KB + 128 B, rounded to 1 KB (swizzle atoms)
constexpr uint32_t kF64TxBytes = 12 * kF64Box + 16 * 8;
constexpr size_t kF64SmemBytes = size_t(kF64Stages) * kF64StageBytes + 1024 + 2 * kF64Stages * 8;
constexpr int kF64Threads = 128;

// 16-byte chunk c of row r of a 128-byte-swizzled box (row r = transition within the k-tile)
RIGW_DEVICE_INLINE uint32_t sw128(int r, int c) { return uint32_t(r * 128 + ((c ^ (r & 7)) << 4)); }

}  // namespace

__global__ void __launch_bounds__(kF64Threads, 2) syrk_f64_tma_kernel(const F64SyrkItem* __restrict__ items) {
  const F64SyrkItem it = items[blockIdx.x];
  const int jw = blockIdx.y;
  if (jw >= (it.nw > 0 ? it.nw : 1)) return;   // the whole CTA, before any barrier
  double* C = it.C + jw * it.sC;
  extern __shared__ uint8_t f64_smem_raw[];
  uint8_t* smem =
      reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(f64_smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kF64Stages * kF64StageBytes);
  uint64_t* empty = full + kF64Stages;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nk = it.ktiles;
  if (tid == 0) {
    for (int s = 0; s < kF64Stages; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], kF64Threads / 32);
    }
    tc::fence_mbar_init();
  }
  __syncthreads();

  int issued[kF64Stages] = {0, 0, 0, 0};   // used by thread 0 only
  auto issue = [&](int kt) {
    const int s = kt % kF64Stages;
    uint8_t* st = smem + s * kF64StageBytes;
    tc::mbar_arrive_expect_tx(&full[s], kF64TxBytes);
    const int k0 = kt * 16;
#pragma unroll
    for (int b = 0; b < 4; ++b) tc::tma_load_2d(st + b * kF64Box, it.tmap_m, &full[s], it.ti + 16 * b, k0);
#pragma unroll
    for (int b = 0; b < 8; ++b) tc::tma_load_2d(st + kF64OffB + b * kF64Box, it.tmap_m, &full[s], it.tj + 16 * b, k0);
    tc::tma_load_2d(st + kF64OffD, it.tmap_d, &full[s], k0, jw);
    ++issued[s];
  };
  if (tid == 0) {
    tc::tmap_acquire(it.tmap_m);
    tc::tmap_acquire(it.tmap_d);
    for (int kt = 0; kt < nk && kt < kF64Stages; ++kt) issue(kt);
  }

  const int q = lane >> 2;   // fragment row (A) / column (B) within the 8-wide tile
  const int r = lane & 3;    // fragment k index
  const int wn0 = warp * 32;
  const int nfrag = min(4, max(0, (it.n - wn0 + 7) >> 3));
  double acc[8][4][2];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  bool ok = true;
  for (int kt = 0; kt < nk; ++kt) {
    if (tid == 0 && kt >= kF64Lag) {
      const int kr = kt - kF64Lag, kn = kr + kF64Stages;
      if (kn < nk) {
        if (tc::mbar_wait(&empty[kr % kF64Stages], (kr / kF64Stages) & 1)) issue(kn);
        else ok = false;
      }
    }
    ok = __all_sync(0xffffffffu, ok);
    if (!ok) break;
    const int s = kt % kF64Stages;
    ok = __all_sync(0xffffffffu, tc::mbar_wait(&full[s], (kt / kF64Stages) & 1));
    if (!ok) break;
    const uint8_t* sa = smem + s * kF64StageBytes + (q >> 1) * kF64Box;          // A box of rows 8q .. 8q+7
    const uint8_t* sb = smem + s * kF64StageBytes + kF64OffB + (2 * warp) * kF64Box;
    const double* ks = reinterpret_cast<const double*>(smem + s * kF64StageBytes + kF64OffD);
#pragma unroll
    for (int k4 = 0; k4 < 4; ++k4) {
      const int kk = k4 * 4 + r;
      double a[8], b[4];
#pragma unroll
      for (int i2 = 0; i2 < 4; ++i2) {
        const double2 v = *reinterpret_cast<const double2*>(sa + sw128(kk, 4 * (q & 1) + i2));
        a[2 * i2] = v.x;
        a[2 * i2 + 1] = v.y;
      }
      const double sc = ks[kk];
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] *= sc;
#pragma unroll
      for (int j = 0; j < 4; ++j)
        b[j] = *reinterpret_cast<const double*>(sb + (j >> 1) * kF64Box + sw128(kk, (q >> 1) + 4 * (j & 1)) +
                                                (q & 1) * 8);
      if (nfrag == 4) {
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (j < nfrag)
#pragma unroll
            for (int i = 0; i < 8; ++i) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
      }
    }
    __syncwarp();
    if (lane == 0) tc::mbar_arrive(&empty[s]);
  }
  if (!ok && lane == 0) atomicOr(it.err, kErrTimeout);
  // no TMA write may land after the CTA exits: wait (bounded) for the last copy of every stage
  if (tid == 0)
    for (int s = 0; s < kF64Stages; ++s)
      if (issued[s] > 0 && !tc::mbar_wait(&full[s], (issued[s] - 1) & 1)) atomicOr(it.err, kErrTimeout);
  if (!ok) return;

  // Epilogue.  Lane (q, r) of warp w owns rows 8q + i (i < 8) and columns
  // 32 w + 8 j + 2 r + e (j < 4, e < 2); the identity on the diagonal.
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int row = 8 * q + i;
    if (row >= it.m) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int col = wn0 + 8 * j + 2 * r;
      if (col >= it.n) continue;
      double v0 = acc[i][j][0], v1 = acc[i][j][1];
      if (col - row == it.diag) v0 += 1.0;
      if (col + 1 - row == it.diag) v1 += 1.0;
      *reinterpret_cast<double2*>(C + size_t(row) * it.ldc + col) = make_double2(v0, v1);
    }
  }
}

// ---------------------------------------------------------------------------
// Host side
namespace {
PFN_cuTensorMapEncodeTiled_v12000 g_encode_f64 = nullptr;
}

Status make_f64_tmaps(void* host_maps, const double* mp, int npad, int nia_pad, const double* dscale, int nomega) {
  if (!g_encode_f64) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult qr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &qr) != cudaSuccess ||
        qr != cudaDriverEntryPointSuccess || !fn) {
      cudaGetLastError();
      return Status::fail(RIGW_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
    }
    g_encode_f64 = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  CUtensorMap* maps = reinterpret_cast<CUtensorMap*>(host_maps);
  {
    cuuint64_t dims[2] = {cuuint64_t(npad), cuuint64_t(nia_pad)};
    cuuint64_t strides[1] = {cuuint64_t(npad) * 8};
    cuuint32_t box[2] = {16, 16};
    cuuint32_t estr[2] = {1, 1};
    CUresult e = g_encode_f64(&maps[0], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(mp), dims, strides,
                              box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (e != CUDA_SUCCESS) return Status::fail(RIGW_ERR_CUDA, "cuTensorMapEncodeTiled (mp) failed (%d)", int(e));
  }
  {
    cuuint64_t dims[2] = {cuuint64_t(nia_pad), cuuint64_t(nomega)};
    cuuint64_t strides[1] = {cuuint64_t(nia_pad) * 8};
    cuuint32_t box[2] = {16, 1};
    cuuint32_t estr[2] = {1, 1};
    CUresult e = g_encode_f64(&maps[1], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(dscale), dims,
                              strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (e != CUDA_SUCCESS) return Status::fail(RIGW_ERR_CUDA, "cuTensorMapEncodeTiled (dscale) failed (%d)", int(e));
  }
  return Status::ok();
}

void launch_syrk_f64_tma(const F64SyrkItem* items, int n, int ny, cudaStream_t s) {
  if (n > 0 && ny > 0) syrk_f64_tma_kernel<<<dim3(n, ny), kF64Threads, kF64SmemBytes, s>>>(items);
}

cudaError_t prepare_syrk_f64_tma() {
  return cudaFuncSetAttribute(syrk_f64_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kF64SmemBytes));
}

}  // namespace rigw
