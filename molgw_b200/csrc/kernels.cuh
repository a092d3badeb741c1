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
constexpr int kDiagThreads = 256;  // threads of chol_diag_kernel
__global__ void chol_diag_kernel(const ProbDev* probs, const WorkItem* items, int k);
size_t chol_diag_smem_bytes();   // dynamic shared memory of chol_diag_kernel
__global__ void energy_kernel(const ProbDev* probs, const WorkItem* items);
__global__ void trace_kernel(const ProbDev* probs, const WorkItem* items);
__global__ void pad_eps_kernel(const ProbDev* probs, const WorkItem* items);
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

// Split-precision chi0 (syrk_bf16x3.cu): one 128x128 upper tile of eps(iw).
struct TcItem {
  const void* tmap;   // CUtensorMap of the problem's hi/lo tensor (rows: [wgroup][2][npad], cols: kpad)
  double* C;          // &eps[w][i0][j0]
  int* err;
  int row_a, row_b;   // tensor rows of the hi blocks of the A (i0) and B (j0) operands
  int lo_off;         // rows from a hi block to its lo block (npad)
  int ktiles;         // kpad / 64
  int ldc;            // npad
  int diag;           // i0 - j0: identity where (col - row) == diag
  // Ozaki INT8 (syrk_ozaki.cu): row_a/row_b address slice 1, lo_off is the row
  // distance between slices, ktiles = kpad / 128
  const int* ea;      // row exponents of the A rows (e_p, p = i0 ..)
  const int* eb;      // row exponents of the B rows (e_q, q = j0 ..)
  int slices;
  // The item covers nw frequencies (nw <= 0: one): CTA (item, j) (blockIdx.y = j < nw) uses
  // C + j*sC, tensor rows row_a/row_b + j*srow, exponents ea/eb + j*se.
  long long sC, se;
  int srow, nw;
  // General products: B from its own tensor map (nullptr: the A map) whose lo
  // rows (Ozaki: next slice) are lo_off_b below the hi rows (first slice); only
  // the first mrows x ncols of the tile are stored, without identity (0: all 128).
  const void* tmap_b;
  int lo_off_b, mrows, ncols;
};
void launch_split_bf16x3(const ProbDev* probs, const WorkItem* items, int n, cudaStream_t s);
// Split of a general FP64 operand into K-major bf16 hi/lo for the tensor-core
// kernel: element (r, k) of batch z is src[z*zs_src + r*rs + k*ks]; dst holds
// [2][Rpad][Kpad] per batch (hi rows, then lo rows), zero padded.
struct SplitOp {
  const double* src;
  long long rs, ks, zs_src;
  int R, K, Rpad, Kpad, nz;
  void* dst;
  long long zs_dst;   // elements between batches of dst
};
void launch_split_kmajor(const SplitOp& op, cudaStream_t s);
// Ozaki slicing of a general FP64 operand: element (r, k) of batch z is
// src[z*zs_src + r*rs + k*ks]; row r is scaled by 2^-e_r (e_r the exponent of
// max_k |x_rk|, to exps[z*Rpad + r]) and cut into `slices` int8 base-128 digits,
// stored K-contiguous as [nz][slices][Rpad][Kpad] (Kpad a multiple of 128, zero
// padded).  rmax is [nz][Rpad] scratch.
struct SliceOp {
  const double* src;
  long long rs, ks, zs_src;
  int R, K, Rpad, Kpad, nz, slices;
  void* dst;
  unsigned long long* rmax;
  int* exps;
};
void launch_slice_kmajor(const SliceOp& op, cudaStream_t s);
void launch_syrk_bf16x3(const TcItem* items, int n, int ny, cudaStream_t s);
void launch_ozaki_zero(const ProbDev* probs, const WorkItem* items, int n, cudaStream_t s);
void launch_ozaki_rowmax(const ProbDev* probs, const WorkItem* items, int n, cudaStream_t s);
void launch_ozaki_slice(const ProbDev* probs, const WorkItem* items, int n, cudaStream_t s);
void launch_syrk_ozaki(const TcItem* items, int n, int ny, cudaStream_t s);
// s <= 4: every slice pair of a k-tile from one stage (64-byte swizzled tensor map)
void launch_syrk_ozaki_fused(const TcItem* items, int n, int ny, cudaStream_t s);
constexpr int kOzaFusedMaxSlices = 4;
cudaError_t prepare_ozaki_kernels();
cudaError_t prepare_tc_kernels();

// FP64 chi0 with TMA-staged operands (syrk_f64_tma.cu): one 64 x 128 upper tile
// of eps(iw) = 1 + sum_t M[t][i] D_w(t) M[t][j] per CTA, frequency = blockIdx.y.
struct F64SyrkItem {
  const void* tmap_m;   // CUtensorMap of mp [nia_pad][npad] (16 x 16 boxes, 128-byte swizzle)
  const void* tmap_d;   // CUtensorMap of dscale [nomega][nia_pad] (16 x 1 boxes)
  double* C;            // &eps[0][ti][tj]
  int* err;
  int ti, tj;           // first auxiliary row (A) and column (B) of the tile
  int m, n;             // rows and columns stored (<= 64, <= 128, even)
  int ktiles;           // nia_pad / 16
  int ldc;              // npad
  int diag;             // ti - tj: identity where col - row == diag
  int nw;               // frequencies (grid y)
  long long sC;         // doubles between the eps blocks of two frequencies
};
void launch_syrk_f64_tma(const F64SyrkItem* items, int n, int ny, cudaStream_t s);
cudaError_t prepare_syrk_f64_tma();

// Host-side launchers of the DMMA tile engine (gemm_f64.cu).
// grid (n items) x (ny frequencies): CTAs with blockIdx.y >= item.nw return at once
void launch_dgemm_128x128(const GemmItem* items, int n, int ny, cudaStream_t s);
void launch_dgemm_64x128(const GemmItem* items, int n, int ny, cudaStream_t s);
cudaError_t prepare_dgemm_kernels();

}  // namespace rigw
