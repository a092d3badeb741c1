// Split-precision chi0 contraction on the 5th-generation tensor cores.
//
//   eps(iw) = 1 + S S^T,   S = M diag(sqrt(D_w)),   S = S_hi + S_lo  (bf16 hi/lo split)
//   S S^T  ~=  S_hi S_hi^T + S_hi S_lo^T + S_lo S_hi^T     (fp32 accumulation in TMEM)
//
// split_bf16x3_kernel: per 64x64 tile of the packed FP64 tensor, scales by
//   sqrt(D_w(t)) for every frequency and writes the hi/lo bf16 pair in the
//   K-major (transition-contiguous) layout the tensor cores read.
// syrk_bf16x3_kernel: one 128x128 upper tile of eps(iw) per CTA.  One thread
//   issues TMA loads (4 tiles of 128 rows x 64 bf16 per stage, 128-byte
//   swizzle) into a 3-stage ring, one thread issues tcgen05.mma (M=128, N=128,
//   K=16; 12 per stage) into two ping-pong TMEM accumulators, eight warps drain
//   them chunk by chunk into FP64, add the identity and store.  All mbarrier
//   waits are bounded.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include "engine.cuh"
#include "tc_common.cuh"

namespace rigw {

constexpr int kTcStages = 3;
constexpr int kTcTileBytes = 128 * 64 * 2;
constexpr int kTcStageBytes = 4 * kTcTileBytes;
constexpr size_t kTcSmemBytes = size_t(kTcStages) * kTcStageBytes + 1024 + 256;

// item: (prob, t0, p0, w0): split_t transitions from t0 x 64 rows from p0, the
// frequencies w0 .. w0+wgroup-1; 256 threads.
__global__ void __launch_bounds__(256) split_bf16x3_kernel(const ProbDev* __restrict__ probs,
                                                           const WorkItem* __restrict__ items) {
  const WorkItem wi = items[blockIdx.x];
  const ProbDev& p = probs[wi.prob];
  const int p0 = wi.b;
  constexpr int kWb = 16;            // frequencies per block of scale factors
  __shared__ double tile[64][65];   // [P][t]
  __shared__ double sc[kWb][64];    // sqrt(D_w(t0 + t)) for kWb frequencies
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  __nv_bfloat16* xs = reinterpret_cast<__nv_bfloat16*>(p.xs);
  const int w0 = wi.c, w1 = min(p.nomega, w0 + p.wgroup);   // this item's frequency group
  const int tend = min(p.nia_pad, wi.a + p.split_t);
  for (int t0 = wi.a; t0 < tend; t0 += 64) {               // 64-transition sub-tiles of the item
    __syncthreads();
    for (int idx = tid; idx < 64 * 64; idx += 256) {
      const int tt = idx >> 6, pp = idx & 63;
      tile[pp][tt] = p.mp[size_t(t0 + tt) * p.npad + p0 + pp];
    }
    // the scale factors of a block of frequencies, then its conversions without barriers
    for (int wb = w0; wb < w1; wb += kWb) {
      const int nwb = min(kWb, w1 - wb);
      __syncthreads();
      for (int idx = tid; idx < nwb * 64; idx += 256)
        sc[idx >> 6][idx & 63] = sqrt(p.dscale[size_t(wb + (idx >> 6)) * p.nia_pad + t0 + (idx & 63)]);
      __syncthreads();
      for (int w = wb; w < wb + nwb; ++w) {
        const int wl = w - w0;
        const double s0 = sc[w - wb][2 * lane], s1 = sc[w - wb][2 * lane + 1];
#pragma unroll
        for (int pr = 0; pr < 8; ++pr) {
          const int pp = warp * 8 + pr;
          const double v0 = tile[pp][2 * lane] * s0, v1 = tile[pp][2 * lane + 1] * s1;
          const __nv_bfloat16 h0 = __double2bfloat16(v0), h1 = __double2bfloat16(v1);
          const __nv_bfloat16 l0 = __double2bfloat16(v0 - double(__bfloat162float(h0)));
          const __nv_bfloat16 l1 = __double2bfloat16(v1 - double(__bfloat162float(h1)));
          const size_t hi_row = (size_t(2 * wl) * p.npad + p0 + pp) * p.kpad + t0;
          const size_t lo_row = (size_t(2 * wl + 1) * p.npad + p0 + pp) * p.kpad + t0;
          reinterpret_cast<__nv_bfloat162*>(xs + hi_row)[lane] = __halves2bfloat162(h0, h1);
          reinterpret_cast<__nv_bfloat162*>(xs + lo_row)[lane] = __halves2bfloat162(l0, l1);
        }
      }
    }
  }
}

// General operand split: 64 (rows) x 64 (K) tiles through shared memory, read
// along the source's contiguous index and written K-contiguous.
__global__ void __launch_bounds__(256) split_kmajor_kernel(const SplitOp op) {
  __shared__ double tile[64][65];   // [row][k]
  const int k0 = blockIdx.x * 64, r0 = blockIdx.y * 64, z = blockIdx.z;
  const double* src = op.src + size_t(z) * op.zs_src;
  __nv_bfloat16* dst = reinterpret_cast<__nv_bfloat16*>(op.dst) + size_t(z) * op.zs_dst;
  const bool rfast = op.rs == 1;
  for (int idx = threadIdx.x; idx < 64 * 64; idx += 256) {
    const int a = idx >> 6, b = idx & 63;
    const int rr = rfast ? b : a, kk = rfast ? a : b;
    const int r = r0 + rr, k = k0 + kk;
    tile[rr][kk] = (r < op.R && k < op.K) ? src[r * op.rs + k * op.ks] : 0.0;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < 64 * 64; idx += 256) {
    const int rr = idx >> 6, kk = idx & 63;
    const double v = tile[rr][kk];
    const __nv_bfloat16 h = __double2bfloat16(v);
    const __nv_bfloat16 l = __double2bfloat16(v - double(__bfloat162float(h)));
    const size_t o = size_t(r0 + rr) * op.Kpad + k0 + kk;
    dst[o] = h;
    dst[o + size_t(op.Rpad) * op.Kpad] = l;
  }
}

// K is consumed in chunks of kTcChunk k-tiles (512 transitions).  Each chunk
// accumulates in fp32 in one of two TMEM accumulators (128 columns each); eight
// epilogue warps drain a finished chunk into FP64 registers while the MMA warp
// fills the other accumulator.  The fp32 accumulation length is therefore
// bounded by the chunk, whatever the number of transitions.
constexpr int kTcChunk = 8;
constexpr int kTcThreads = 320;    // warp 0 TMA, warp 1 MMA, warps 2..9 epilogue

__global__ void __launch_bounds__(kTcThreads, 1) syrk_bf16x3_kernel(const TcItem* __restrict__ items) {
  TcItem it = items[blockIdx.x];
  const int jw = blockIdx.y;
  if (jw >= (it.nw > 0 ? it.nw : 1)) return;   // the whole CTA, before any barrier or TMEM use
  it.C += jw * it.sC;
  it.row_a += jw * it.srow;
  it.row_b += jw * it.srow;
  if (it.ea) {
    it.ea += jw * it.se;
    it.eb += jw * it.se;
  }
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kTcStages * kTcStageBytes);
  uint64_t* empty = full + kTcStages;
  uint64_t* accf = empty + kTcStages;     // [2] chunk accumulated
  uint64_t* acce = accf + 2;              // [2] chunk drained
  uint32_t* tslot = reinterpret_cast<uint32_t*>(acce + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  auto tile = [&](int s, int which) { return smem + s * kTcStageBytes + which * kTcTileBytes; };

  if (tid == 0) {
    for (int s = 0; s < kTcStages; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&accf[b], 1);
      tc::mbar_init(&acce[b], 8);
    }
    tc::fence_mbar_init();
  }
  if (warp == 0) tc::tmem_alloc(tslot, 256);
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tslot;
  const int nk = it.ktiles;
  const int nchunks = (nk + kTcChunk - 1) / kTcChunk;

  if (tid == 0) {
    // ---- TMA producer
    const void* tmb = it.tmap_b ? it.tmap_b : it.tmap;
    const int lob = it.tmap_b ? it.lo_off_b : it.lo_off;
    tc::tmap_acquire(it.tmap);
    if (it.tmap_b) tc::tmap_acquire(it.tmap_b);
    int issued[kTcStages] = {0, 0, 0};
    bool ok = true;
    for (int kt = 0; kt < nk && ok; ++kt) {
      const int s = kt % kTcStages;
      if (kt >= kTcStages && !tc::mbar_wait(&empty[s], ((kt / kTcStages) - 1) & 1)) {
        ok = false;
        break;
      }
      tc::mbar_arrive_expect_tx(&full[s], kTcStageBytes);
      const int k0 = kt * 64;
      tc::tma_load_2d(tile(s, 0), it.tmap, &full[s], k0, it.row_a);
      tc::tma_load_2d(tile(s, 1), it.tmap, &full[s], k0, it.row_a + it.lo_off);
      tc::tma_load_2d(tile(s, 2), tmb, &full[s], k0, it.row_b);
      tc::tma_load_2d(tile(s, 3), tmb, &full[s], k0, it.row_b + lob);
      ++issued[s];
    }
    if (!ok) atomicOr(it.err, kErrTimeout);
    for (int s = 0; s < kTcStages; ++s)
      if (issued[s] > 0 && !tc::mbar_wait(&full[s], (issued[s] - 1) & 1)) atomicOr(it.err, kErrTimeout);
  } else if (tid == 32) {
    // ---- MMA issuer
    constexpr uint32_t idesc = tc::idesc_bf16_f32(128, 128);
    bool ok = true;
    for (int kt = 0; kt < nk && ok; ++kt) {
      const int c = kt / kTcChunk, b = c & 1;
      const bool first = (kt % kTcChunk) == 0;
      if (first && c >= 2 && !tc::mbar_wait(&acce[b], ((c >> 1) - 1) & 1)) {
        ok = false;
        break;
      }
      const int s = kt % kTcStages;
      if (!tc::mbar_wait(&full[s], (kt / kTcStages) & 1)) {
        ok = false;
        break;
      }
      tc::tc_fence_after();
      const uint32_t d = tmem + uint32_t(b * 128);
      const uint64_t ah = tc::desc_kmajor_sw128(tile(s, 0)), al = tc::desc_kmajor_sw128(tile(s, 1));
      const uint64_t bh = tc::desc_kmajor_sw128(tile(s, 2)), bl = tc::desc_kmajor_sw128(tile(s, 3));
#pragma unroll
      for (int sub = 0; sub < 4; ++sub) {
        const uint64_t o = uint64_t(sub * 2);   // 16 bf16 = 32 bytes along K
        tc::mma_bf16(d, ah + o, bh + o, idesc, (first && sub == 0) ? 0u : 1u);
        tc::mma_bf16(d, ah + o, bl + o, idesc, 1u);
        tc::mma_bf16(d, al + o, bh + o, idesc, 1u);
      }
      tc::mma_commit(&empty[s]);
      if ((kt % kTcChunk) == kTcChunk - 1 || kt == nk - 1) tc::mma_commit(&accf[b]);
    }
    if (!ok) atomicOr(it.err, kErrTimeout);
  } else if (warp >= 2) {
    // ---- epilogue: drain each chunk into FP64 registers, then store the tile
    const int quad = warp & 3;                 // TMEM lanes 32*quad .. 32*quad+31 (rows)
    const int half = (warp - 2) >> 2;          // columns 64*half .. 64*half+63
    const int row = quad * 32 + lane;
    double acc[64];
#pragma unroll
    for (int j = 0; j < 64; ++j) acc[j] = 0.0;
    bool ok = true;
    for (int c = 0; c < nchunks; ++c) {
      const int b = c & 1;
      ok = __all_sync(0xffffffffu, tc::mbar_wait(&accf[b], (c >> 1) & 1));
      if (!ok) break;
      tc::tc_fence_after();
      const uint32_t base = tmem + uint32_t(b * 128 + half * 64) + (uint32_t(quad * 32) << 16);
      uint32_t r[32];
      tc::tmem_ld_32x32(base, r);
#pragma unroll
      for (int j = 0; j < 32; ++j) acc[j] += double(__uint_as_float(r[j]));
      tc::tmem_ld_32x32(base + 32, r);
#pragma unroll
      for (int j = 0; j < 32; ++j) acc[32 + j] += double(__uint_as_float(r[j]));
      tc::tc_fence_before();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&acce[b]);
    }
    if (ok && it.mrows == 0) {
      double* dst = it.C + size_t(row) * it.ldc + half * 64;
#pragma unroll
      for (int j = 0; j < 64; j += 2) {
        const int col = half * 64 + j;
        double v0 = acc[j], v1 = acc[j + 1];
        if (col - row == it.diag) v0 += 1.0;
        if (col + 1 - row == it.diag) v1 += 1.0;
        *reinterpret_cast<double2*>(dst + j) = make_double2(v0, v1);
      }
    } else if (ok) {
      // edge tile of a general product: rows < mrows, columns < ncols, no identity
      if (row < it.mrows) {
        double* dst = it.C + size_t(row) * it.ldc;
#pragma unroll
        for (int j = 0; j < 64; ++j)
          if (half * 64 + j < it.ncols) dst[half * 64 + j] = acc[j];
      }
    } else if (lane == 0) {
      atomicOr(it.err, kErrTimeout);
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 256);
}

// ---------------------------------------------------------------------------
// Host side
namespace {
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
}

bool bf16x3_available() {
  if (g_encode) return true;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !fn) {
    cudaGetLastError();
    return false;
  }
  g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  return true;
}

// Row-major [rows][kpad] tensor read in boxes of 128 rows x box_bytes (128: 128-byte
// swizzle; 64: 64-byte swizzle).
static Status make_kmajor_tmap(void* host_map, CUtensorMapDataType type, int esize, const void* base, int kpad,
                               long long rows, int box_bytes = 128) {
  if (!bf16x3_available()) return Status::fail(RIGW_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
  CUtensorMap* m = reinterpret_cast<CUtensorMap*>(host_map);
  cuuint64_t dims[2] = {cuuint64_t(kpad), cuuint64_t(rows)};
  cuuint64_t strides[1] = {cuuint64_t(kpad) * esize};
  cuuint32_t box[2] = {cuuint32_t(box_bytes / esize), 128};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = g_encode(m, type, 2, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        box_bytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return Status::fail(RIGW_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", int(r));
  return Status::ok();
}

Status make_split_tmap(void* host_map, const void* xs, int kpad, long long rows) {
  return make_kmajor_tmap(host_map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, xs, kpad, rows);
}

Status make_ozaki_tmap(void* host_map, const void* xq, int kpad, long long rows, int box_bytes) {
  return make_kmajor_tmap(host_map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, xq, kpad, rows, box_bytes);
}

void launch_split_bf16x3(const ProbDev* probs, const WorkItem* items, int n, cudaStream_t s) {
  if (n > 0) split_bf16x3_kernel<<<n, 256, 0, s>>>(probs, items);
}

void launch_split_kmajor(const SplitOp& op, cudaStream_t s) {
  if (op.Rpad > 0 && op.Kpad > 0 && op.nz > 0)
    split_kmajor_kernel<<<dim3(op.Kpad / 64, op.Rpad / 64, op.nz), 256, 0, s>>>(op);
}

void launch_syrk_bf16x3(const TcItem* items, int n, int ny, cudaStream_t s) {
  if (n > 0 && ny > 0) syrk_bf16x3_kernel<<<dim3(n, ny), kTcThreads, kTcSmemBytes, s>>>(items);
}

cudaError_t prepare_tc_kernels() {
  return cudaFuncSetAttribute(syrk_bf16x3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kTcSmemBytes));
}

}  // namespace rigw
