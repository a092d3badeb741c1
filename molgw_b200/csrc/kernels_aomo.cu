// AO -> MO transform of the RI 3-center integrals (src/m_eri_ao_mo.f90:416-582).
//
// The reference loops over the auxiliary index with a scalar pair loop
// (tmp1(:,k) += c_t(:,l) B ; tmp1(:,l) += c_t(:,k) B) followed by one small
// DGEMM per auxiliary function.  Here the pair-packed tensor of one chunk of
// auxiliary functions is unpacked once into the symmetric (nu, mu, P) block
// (diagonal pairs carry x0.5 in the packed form, src/m_eri_calculate.f90:1841,
// so the unpacked diagonal is twice the stored value), and both index
// transforms become two large DMMA products with P contiguous.
#include "kernels.cuh"

namespace rigw {

// item: tile of 32 pairs x 32 auxiliary functions; block (32, 8).
__global__ void __launch_bounds__(256) aomo_unpack_kernel(const AomoUnpackItem* __restrict__ items) {
  const AomoUnpackItem it = items[0];
  const int pair0 = blockIdx.x * 32;
  const int paux0 = blockIdx.y * 32;          // relative to the chunk start p0
  __shared__ double tile[32][33];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int pp = ty; pp < 32; pp += 8) {
    const int P = paux0 + pp;                  // chunk-relative
    const int pair = pair0 + tx;
    double v = 0.0;
    if (pair < it.npair && P < it.naux) v = it.eri3[size_t(it.p0 + P) * it.npair + pair];
    tile[pp][tx] = v;
  }
  __syncthreads();
  for (int q = ty; q < 32; q += 8) {
    const int pair = pair0 + q;
    const int P = paux0 + tx;
    if (pair >= it.npair || P >= it.naux) continue;
    const int mu = it.index_basis[2 * pair] - 1;
    const int nu = it.index_basis[2 * pair + 1] - 1;
    const double v = tile[tx][q];
    if (mu == nu) {
      it.bfull[(size_t(mu) * it.nbf + mu) * it.naux_pad + P] = 2.0 * v;
    } else {
      it.bfull[(size_t(mu) * it.nbf + nu) * it.naux_pad + P] = v;
      it.bfull[(size_t(nu) * it.nbf + mu) * it.naux_pad + P] = v;
    }
  }
}

}  // namespace rigw
