// Instantiations and launchers of the FP64 DMMA tile engine.
#include "kernels.cuh"

namespace rigw {

template <int BM, int BN>
static void launch_dgemm(const GemmItem* items, int n, int ny, cudaStream_t s) {
  if (n <= 0 || ny <= 0) return;
  using Cfg = DgemmCfg<BM, BN>;
  dgemm_mn_kernel<BM, BN><<<dim3(n, ny), Cfg::kThreads, Cfg::kSmemBytes, s>>>(items);
}

void launch_dgemm_128x128(const GemmItem* items, int n, int ny, cudaStream_t s) {
  launch_dgemm<128, 128>(items, n, ny, s);
}
void launch_dgemm_64x128(const GemmItem* items, int n, int ny, cudaStream_t s) {
  launch_dgemm<64, 128>(items, n, ny, s);
}

cudaError_t prepare_dgemm_kernels() {
  cudaError_t e = cudaFuncSetAttribute(dgemm_mn_kernel<128, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(DgemmCfg<128, 128>::kSmemBytes));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(dgemm_mn_kernel<64, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              int(DgemmCfg<64, 128>::kSmemBytes));
}

}  // namespace rigw
