// Kernel declarations of the RI-GW engine.
#pragma once
#include "common.cuh"
#include "dgemm_mn.cuh"
#include "problem.cuh"

namespace rigw {

// Generic work-list entry of the non-GEMM kernels: problem index + up to three
// kernel-specific integers.
struct WorkItem {
  int prob, a, b, c;
};

__global__ void pack_m_kernel(const ProbDev* probs, const WorkItem* items);
__global__ void init_rhs_kernel(const ProbDev* probs, const WorkItem* items);
__global__ void mnorm_kernel(const ProbDev* probs, const WorkItem* items);
__global__ void chol_diag_kernel(const ProbDev* probs, const WorkItem* items, int k);
__global__ void energy_kernel(const ProbDev* probs, const WorkItem* items);
__global__ void vchiv_kernel(const ProbDev* probs, const WorkItem* items);
__global__ void sigma_kernel(const ProbDev* probs, const WorkItem* items);
__global__ void pade_qp_kernel(const ProbDev* probs, const WorkItem* items);
__global__ void energy_sum_kernel(const ProbDev* probs, int nprob);

// AO -> MO transform helpers (kernels_aomo.cu).
struct AomoUnpackItem {
  const double* eri3;     // [naux][npair] pair-packed, diagonal x0.5
  const int* index_basis; // [npair][2] 1-based
  double* bfull;          // [nbf][nbf][naux_pad]
  int naux, naux_pad, npair, nbf, p0;
};
__global__ void aomo_unpack_kernel(const AomoUnpackItem* items);

// Host-side launchers of the DMMA tile engine (gemm_f64.cu).
void launch_dgemm_128x128(const GemmItem* items, int n, cudaStream_t s);
void launch_dgemm_64x128(const GemmItem* items, int n, cudaStream_t s);
cudaError_t prepare_dgemm_kernels();

}  // namespace rigw
