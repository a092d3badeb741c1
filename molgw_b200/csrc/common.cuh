// Shared device helpers of the RI-GW engine (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#ifndef RIGW_DEVICE_INLINE
#define RIGW_DEVICE_INLINE __device__ __forceinline__
#endif

namespace rigw {

constexpr double kPi = 3.14159265358979323;   // src/m_definitions.f90:50
constexpr int kPanel = 128;                    // Cholesky panel width (rows of one U block row)
constexpr int kMaxChains = 8;                  // frequency chains of the factorization stage (tuner's range)
constexpr int kAutoChains = 2;                 // chains without a tuning
constexpr int kChainPairs = 4;                 // (problem, frequency) pairs per chain at least
constexpr int kSplitGroup = 8;                 // frequencies sharing one bf16 hi/lo split buffer
constexpr size_t kSplitWholeBytes = size_t(1) << 30;   // below this, one buffer for all frequencies
constexpr size_t kSplitProblemBytes = size_t(4) << 30; // split buffer of one problem at most (>= one frequency)
constexpr size_t kSplitL2Bytes = size_t(48) << 20;     // split buffers that stay resident in the 126 MB L2
constexpr int kSplitT = 256;                   // transitions per item of the split / slice kernels

// Device-side error flags (bitmask written with atomicOr, read by the host after a stage).
enum DeviceError : int {
  kErrNone = 0,
  kErrNotSPD = 1,        // a pivot of eps(iw) was <= 0 (eps must be SPD with eigenvalues >= 1)
  kErrNonFinite = 2,     // NaN/Inf met in an output sentinel
  kErrPade = 4,          // zero denominator in the Thiele recursion
  kErrTimeout = 8,       // a bounded mbarrier wait gave up
};

RIGW_DEVICE_INLINE uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// 16-byte async copy global->shared; src_bytes==0 zero-fills the destination.
RIGW_DEVICE_INLINE void cp_async16(void* smem, const void* gmem, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(smem)), "l"(gmem),
               "r"(src_bytes));
}
RIGW_DEVICE_INLINE void cp_async8(void* smem, const void* gmem, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(smem)), "l"(gmem),
               "r"(src_bytes));
}
RIGW_DEVICE_INLINE void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
RIGW_DEVICE_INLINE void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// FP64 tensor-core MMA, D(8x8) += A(8x4, row) * B(4x8, col).
// Fragment ownership (lane l): a = A[l/4][l%4], b = B[l%4][l/4],
// c0,c1 = C[l/4][2*(l%4)+{0,1}].
RIGW_DEVICE_INLINE void dmma_8x8x4(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

RIGW_DEVICE_INLINE double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace rigw
