// Analytic continuation + QP equation on caller-provided device arrays, using a
// fixed device-resident scratch area instead of any device allocation.
//
// Who needs it: hosts that own the GPU memory themselves and may not call
// cudaMalloc - a Fortran code with its own device pool, an application with a
// caching allocator that forbids foreign allocations, or a serving loop whose
// memory is reserved up front.  cudaMalloc also synchronizes the device, which a
// latency-bound request loop cannot afford.
//
// The scratch lives in a file-scope __device__ array of kScratchBytes bytes.
// Every GPU that loads this library holds that array until the process exits.
// The host-side symbol is only a stand-in; its device address is obtained with
// cudaGetSymbolAddress, once per device, on the first call made on that device
// (with the device current).
// All calls share the array and it keeps the last call's contents: calls that
// overlap on the GPU (different streams, different host threads) race on it.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "engine.cuh"

namespace rigw {

namespace {

constexpr int kMaxSig = 64;          // Sigma states per call
constexpr int kMaxCalc = 128;        // evaluation points (nomega_sigma_calc)
constexpr int kMaxReal = 1025;       // real-grid points (2 * (nomega_sigma / 2) + 1)

struct ScratchLayout {
  ProbDev prob;
  WorkItem items[kMaxSig];
  int err;
  double qp[4 * kMaxSig];
  double zcalc[2 * kMaxCalc];
  double sigma_real[2 * kMaxSig * kMaxReal];
};
constexpr size_t kScratchBytes = (sizeof(ScratchLayout) + 255) / 256 * 256;   // ~1.06 MiB

__device__ __align__(256) unsigned char g_qp_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};

void set_msg(char* buf, size_t len, const char* msg) {
  if (buf && len) {
    std::strncpy(buf, msg, len - 1);
    buf[len - 1] = '\0';
  }
}

}  // namespace
}  // namespace rigw

extern "C" RIGW_API int rigw_qp_solve_noalloc(int device, int nsig, int nomega_sigma_calc, const double* omega_calc,
                                              const double* sigma_calc, const double* e_sig,
                                              const double* exchange_m_vxc, int technique, int nomega_sigma,
                                              double step_sigma, double step_sigma_calc, double eta, double efermi,
                                              double* energy_qp_g, double* energy_qp_z, double* zz, double* sigma,
                                              void* stream, char* errbuf, size_t errlen) {
  using namespace rigw;
  char msg[256];
  const int nreal = 2 * (nomega_sigma / 2) + 1;
  if (nsig < 1 || nsig > kMaxSig || nomega_sigma_calc < 1 || nomega_sigma_calc > kMaxCalc || nomega_sigma < 0 ||
      nreal > kMaxReal) {
    std::snprintf(msg, sizeof(msg),
                  "rigw_qp_solve_noalloc: sizes nsig=%d nomega_sigma_calc=%d nomega_sigma=%d exceed the fixed "
                  "scratch (nsig <= %d, nomega_sigma_calc <= %d, 2*(nomega_sigma/2)+1 <= %d)",
                  nsig, nomega_sigma_calc, nomega_sigma, kMaxSig, kMaxCalc, kMaxReal);
    set_msg(errbuf, errlen, msg);
    return RIGW_ERR_ARG;
  }
  if (technique != RIGW_PADE && technique != RIGW_HOMOLUMO) {
    set_msg(errbuf, errlen, "rigw_qp_solve_noalloc: unknown technique");
    return RIGW_ERR_ARG;
  }
  if (!sigma_calc || !e_sig || !energy_qp_g || (technique == RIGW_HOMOLUMO && !omega_calc) || device < 0 ||
      device >= kMaxDevices) {
    set_msg(errbuf, errlen, "rigw_qp_solve_noalloc: missing device array or bad device index");
    return RIGW_ERR_ARG;
  }
  int prev = -1;
  cudaGetDevice(&prev);
  auto fail = [&](cudaError_t e, const char* what) {
    std::snprintf(msg, sizeof(msg), "rigw_qp_solve_noalloc: %s: %s", what, cudaGetErrorString(e));
    set_msg(errbuf, errlen, msg);
    if (prev >= 0) cudaSetDevice(prev);
    return int(RIGW_ERR_CUDA);
  };
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(e, "cudaSetDevice");
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[device]) {
      void* ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, g_qp_scratch);
      if (e != cudaSuccess) return fail(e, "cudaGetSymbolAddress");
      g_scratch_ptr[device] = ptr;
    }
    base = static_cast<unsigned char*>(g_scratch_ptr[device]);
  }
  ScratchLayout* sd = reinterpret_cast<ScratchLayout*>(base);
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  ProbDev p;
  std::memset(&p, 0, sizeof(p));
  p.nsig = nsig;
  p.nc = nomega_sigma_calc;
  p.nsigma_half = nomega_sigma / 2;
  p.technique = technique;
  p.efermi = efermi;
  p.step_sigma = step_sigma;
  p.eta = eta;
  p.e_sig = e_sig;
  p.xc_sig = exchange_m_vxc;
  p.sigma_calc = const_cast<double*>(sigma_calc);
  p.sigma_real = sigma ? sigma : sd->sigma_real;
  p.qp = sd->qp;
  p.err = &sd->err;
  p.zcalc = omega_calc ? omega_calc : sd->zcalc;
  WorkItem items[kMaxSig];
  for (int k = 0; k < nsig; ++k) items[k] = {0, k, 0, 0};
  double z[2 * kMaxCalc];
  if (!omega_calc) {
    for (int k = 0; k < nomega_sigma_calc; ++k) {
      z[2 * k] = efermi;
      z[2 * k + 1] = step_sigma_calc * k;
    }
    if ((e = cudaMemcpyAsync(sd->zcalc, z, sizeof(double) * 2 * nomega_sigma_calc, cudaMemcpyHostToDevice, s)) !=
        cudaSuccess)
      return fail(e, "copy of the evaluation points");
  }
  if ((e = cudaMemcpyAsync(&sd->prob, &p, sizeof(p), cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return fail(e, "copy of the descriptor");
  if ((e = cudaMemcpyAsync(sd->items, items, sizeof(WorkItem) * nsig, cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return fail(e, "copy of the work list");
  if ((e = cudaMemsetAsync(&sd->err, 0, sizeof(int), s)) != cudaSuccess) return fail(e, "clear of the error flag");
  pade_qp_kernel<<<nsig, 256, 0, s>>>(&sd->prob, sd->items);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "pade_qp_kernel launch");
  const size_t w = sizeof(double), pitch = 4 * sizeof(double);
  if ((e = cudaMemcpy2DAsync(energy_qp_g, w, sd->qp + 0, pitch, w, nsig, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
    return fail(e, "copy of energy_qp_g");
  if (energy_qp_z &&
      (e = cudaMemcpy2DAsync(energy_qp_z, w, sd->qp + 1, pitch, w, nsig, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
    return fail(e, "copy of energy_qp_z");
  if (zz && (e = cudaMemcpy2DAsync(zz, w, sd->qp + 2, pitch, w, nsig, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
    return fail(e, "copy of zz");
  int err = 0;
  if ((e = cudaMemcpyAsync(&err, &sd->err, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return fail(e, "read of the error flag");
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return fail(e, "stream synchronize");
  if (prev >= 0) cudaSetDevice(prev);
  if (err) {
    std::snprintf(msg, sizeof(msg), "rigw_qp_solve_noalloc: non-finite QP energy or singular Pade recursion (%d)",
                  err);
    set_msg(errbuf, errlen, msg);
    return RIGW_ERR_NUMERIC;
  }
  set_msg(errbuf, errlen, "");
  return RIGW_OK;
}
