// Host-side engine: device memory accounting, batch plans (problem table +
// work lists + launch sequence), CUDA-graph replay.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/rigw.h"
#include <nvtx3/nvToolsExt.h>
#include "kernels.cuh"

namespace rigw {

// NVTX range named like the reference's stage timers (src/m_timing.f90:268-284);
// a no-op unless a profiler is attached.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};


struct Status {
  int code = RIGW_OK;
  std::string msg;
  static Status ok() { return {}; }
  static Status fail(int c, const char* fmt, ...) {
    Status s;
    s.code = c;
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    s.msg = buf;
    return s;
  }
  bool good() const { return code == RIGW_OK; }
};

#define RIGW_CUDA_TRY(expr)                                                                      \
  do {                                                                                           \
    cudaError_t e__ = (expr);                                                                    \
    if (e__ != cudaSuccess)                                                                      \
      return ::rigw::Status::fail(RIGW_ERR_CUDA, "%s failed: %s (%s:%d)", #expr,                 \
                                  cudaGetErrorString(e__), __FILE__, __LINE__);                  \
  } while (0)

#define RIGW_TRY(expr)             \
  do {                             \
    ::rigw::Status s__ = (expr);   \
    if (!s__.good()) return s__;   \
  } while (0)

class Context;

// Device allocation with named accounting against the context's HBM budget
// (the pattern of MOLGW's clean_allocate, src/m_memory.f90:16-92).
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  ~DeviceBuffer();
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  Status allocate(Context* ctx, size_t bytes, const char* name);
  void release();
  char* data() const { return ptr_; }
  size_t size() const { return bytes_; }

 private:
  Context* ctx_ = nullptr;
  char* ptr_ = nullptr;
  size_t bytes_ = 0;
};

inline bool is_ozaki(int precision) {
  return precision >= RIGW_OZAKI(RIGW_OZAKI_MIN_SLICES) && precision <= RIGW_OZAKI(RIGW_OZAKI_MAX_SLICES);
}
inline int ozaki_slices(int precision) { return is_ozaki(precision) ? precision - RIGW_OZAKI_INT8 : 0; }

// Shapes of one problem of a plan (derived from rigw_problem).
struct Shape {
  int naux, nocc, nvirt, nomega, nstate_p, nsig, nc, nsigma_half, technique, precision;
  int qp_only;
  int nocc2 = 0, nvirt2 = 0;   // second spin channel of the W window
  bool operator<(const Shape& o) const;
};

// Launch shapes of a plan that the autotuner chooses (rigw_autotune); zero
// fields mean the built-in rule.
struct Tuning {
  int chi0_rows = 64;     // FP64 chi0 items: rows per 128-column item (64 or 128)
  int update_rows = 64;   // trailing-update items: rows per 128-column item (64 or 128)
  int split_group = 0;    // split precision: frequencies per hi/lo buffer (0: automatic)
  int chains = 0;         // frequency chains of the factorization stage (0: automatic)
  int panel_group = 0;    // panels per trailing update (0: automatic, 16 for batches of >= 4 problems, else 2)
};
// Precision class of a batch (tunings are kept per mode and class):
// 0 FP64, 1 BF16x3, 2 Ozaki INT8, 3 mixed.
int precision_class(const std::vector<Shape>& shapes);
// Bytes of one frequency's split operands of a problem (0 for FP64).
size_t split_bytes_per_frequency(const Shape& sh);

enum PlanMode : int {
  kPlanFused = 0,      // chi0 -> eps -> factor -> [I | M_sigma] solve -> Sigma -> QP
  kPlanPolar = 1,      // chi0 -> eps -> factor -> I solve -> energies (factors stay resident)
  kPlanSigma = 2,      // M_sigma solve with resident factors -> Sigma
  kPlanQP = 3,         // continuation + QP from given sigma_calc
  kPlanPartial = 4,    // chi0 -> eps -> factor -> solves -> partial Sigma and energies (no QP):
                       // one frequency chunk of a problem, summed over chunks by the scheduler
};

struct PlanProblem {
  Shape sh;
  ProbDev dev;                 // device descriptor (input pointers patched per call)
  size_t off_in_m = 0, off_in_eocc = 0, off_in_evirt = 0, off_in_oocc = 0, off_in_ovirt = 0;
  size_t off_in_m2 = 0, off_in_eocc2 = 0, off_in_evirt2 = 0, off_in_oocc2 = 0, off_in_ovirt2 = 0;
  size_t off_in_omega = 0, off_in_weight = 0, off_in_msig = 0, off_in_ep = 0, off_in_esig = 0;
  size_t off_in_xc = 0, off_in_zcalc = 0, off_out = 0, off_sigma_in = 0;
};

// A batch plan: all device memory, the problem table, the work lists and the
// launch sequence of one group of problems.
class Plan {
 public:
  // tune: launch shapes (nullptr: the context's tuning for this mode and class)
  Status build(Context* ctx, PlanMode mode, const std::vector<Shape>& shapes,
               const std::vector<const ProbDev*>& factors, size_t* measure_only = nullptr,
               const Tuning* tune = nullptr);
  // Device bytes a plan of these shapes allocates (arena + work lists).
  static size_t measure(const std::vector<Shape>& shapes, PlanMode mode, const Tuning* tune = nullptr);
  const Tuning& tuning() const { return tune_; }
  // Copy inputs (host or device pointers) and run; results stay on the device.
  Status stage_inputs(const rigw_problem* probs, cudaStream_t s);
  Status stage_sigma_calc(int i, const double* sigma_calc_host, cudaStream_t s);
  Status launch(cudaStream_t s);
  Status fetch_results(const rigw_problem* probs, rigw_result* res, cudaStream_t s);
  Status check_errors(cudaStream_t s);
  float last_ms() const { return last_ms_; }
  std::vector<PlanProblem>& problems() { return probs_; }
  size_t bytes() const { return arena_.size(); }
  PlanMode mode() const { return mode_; }
  const std::vector<Shape>& shapes() const { return shapes_; }
  ~Plan();

  // launch statistics (kernels per launch sequence)
  int kernel_launches() const { return n_launches_; }

 private:
  void record(cudaStream_t s, int stage);
  Context* ctx_ = nullptr;
  PlanMode mode_ = kPlanFused;
  Tuning tune_;
  std::vector<Shape> shapes_;
  std::vector<PlanProblem> probs_;
  DeviceBuffer arena_;
  DeviceBuffer lists_;
  ProbDev* probs_dev_ = nullptr;
  int* err_dev_ = nullptr;
  // work lists (host copies + device offsets)
  std::vector<WorkItem> wl_pack_, wl_rhs_, wl_mnorm_, wl_energy_, wl_vchiv_, wl_sigma_, wl_pade_;
  std::vector<std::vector<WorkItem>> wl_diag_;
  std::vector<GemmItem> gl_syrk_;
  std::vector<F64SyrkItem> fl_syrk_;              // FP64 chi0, TMA-staged (64-row items)
  std::vector<std::vector<WorkItem>> wl_split_;   // per frequency group
  std::vector<std::vector<TcItem>> tl_syrk_;
  std::vector<WorkItem> wl_ozzero_, wl_rowmax_;    // Ozaki: row maxima over every frequency
  std::vector<std::vector<WorkItem>> wl_slice_;   // Ozaki: per frequency group
  std::vector<std::vector<TcItem>> tl_ozaki_, tl_ozaki4_;   // s >= 5 / s <= 4 (fused slice pairs)
  std::vector<std::vector<GemmItem>> gl_k2_, gl_k2n_, gl_k3_, gl_k3d_, gl_k3a_;
  std::vector<WorkItem> wl_trace_, wl_pad_;
  struct Launch {
    int kind;        // see Plan::record
    size_t off;      // byte offset of the list in lists_
    int count;
    int arg;
    int stream;      // 0: the plan's stream, 1: the lookahead stream
    int wait_ev;     // lookahead event to wait for before the launch (-1: none)
    int rec_ev;      // lookahead event to record after the launch (-1: none)
    int ny;          // grid y: frequencies covered by the items of the list
  };
  std::vector<cudaEvent_t> la_ev_;           // borrowed from the context
  std::vector<cudaStream_t> aux_streams_;   // streams 1.. of the launch sequence (0 is the plan's stream); borrowed
  int nchains_ = 1;
  int group_ = 2;          // panels per trailing update
  std::vector<Launch> seq_;
  cudaGraph_t stage_graph_[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaGraphExec_t stage_exec_[4] = {nullptr, nullptr, nullptr, nullptr};
  bool stage_empty_[4] = {false, false, false, false};
  cudaEvent_t stage_ev_[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  float last_ms_ = 0.0f;
  float stage_ms_[4] = {0, 0, 0, 0};
  bool replayed_ = false;
  int launches_ = 0;

 public:
  const float* stage_ms() const { return stage_ms_; }
  bool replayed() const { return replayed_; }

 private:
  int n_launches_ = 0;
  std::vector<ProbDev> host_table_;
};

class Context {
 public:
  int device = 0;
  cudaStream_t stream = nullptr;
  size_t budget = 0;
  size_t in_use = 0, peak = 0;
  std::string last_error;
  std::mutex mu;
  // plans by (mode, shapes); a repeated batch replays its CUDA graphs
  std::map<std::pair<int, std::vector<Shape>>, std::unique_ptr<Plan>> plan_cache;
  bool use_graphs = true;
  rigw_stats last_stats{};
  double host_build_ms = 0.0, host_capture_ms = 0.0;   // host time in plan builds / graph captures
  double host_alloc_ms = 0.0;                           // host time in device allocations
  // one spare device block: the arena of the last released plan, reused by the next
  static constexpr size_t kSpareMin = size_t(64) << 20;
  char* spare_ptr = nullptr;
  size_t spare_bytes = 0;
  void free_spare();
  // Streams and events shared by the plans of this context (a context runs one
  // plan at a time); created once: creating them per plan stalls behind the
  // work of other contexts.
  std::vector<cudaStream_t> aux_pool;
  std::vector<cudaEvent_t> order_pool;   // ordering events (no timing)
  cudaEvent_t stage_ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  Status borrow(int nstreams, int nevents, std::vector<cudaStream_t>* streams, std::vector<cudaEvent_t>* events);
  // Pinned host staging for the small inputs and outputs of one call: copies from
  // it are asynchronous (pageable sources make every copy wait for the stream).
  static constexpr size_t kHostStage = size_t(16) << 20;
  char* host_stage = nullptr;
  size_t host_stage_used = 0;
  char* stage_take(size_t bytes);   // nullptr when the area is full or unavailable
  void stage_reset() { host_stage_used = 0; }
  // Allocate a block of `bytes` now and keep it as the spare block, so that the
  // plans of this context take their arena from it instead of growing the pool.
  Status reserve(size_t bytes);
  cudaEvent_t sync_ev = nullptr;   // blocking-sync event: host waits sleep instead of spinning
  // Wait for the work queued on stream s (blocking wait on an event).
  Status sync(cudaStream_t s);
  // autotuned launch shapes by (mode, precision class)
  std::map<std::pair<int, int>, Tuning> tuned;
  Tuning tuning_for(int mode, const std::vector<Shape>& shapes) const {
    auto it = tuned.find({mode, precision_class(shapes)});
    return it == tuned.end() ? Tuning{} : it->second;
  }
  int priority = 0;   // CUDA stream priority of every stream of this context (lower = higher)
  // priority: 0 default; > 0 asks for the highest priority, < 0 for the lowest
  // blocking_waits: host waits sleep on an event (request-loop workers, many
  // threads) instead of spinning (one caller: lowest latency)
  Status init(int dev, size_t budget_bytes, int want_priority = 0, bool blocking_waits = false);
  ~Context();
};

struct Wpol {
  Context* ctx = nullptr;
  std::unique_ptr<Plan> plan;     // the kPlanPolar plan that owns eps/U, winv and U^-T
  Shape sh;
};

Status make_shape(const rigw_problem& p, Shape* sh);
size_t footprint(const Shape& sh, PlanMode mode);
void imag_grid(int n, double* omega, double* weight);
Status wpol_chi(Context& c, const Wpol& w, double* chi);
Status sox_selfenergy_imag(Context& c, const rigw_sox_problem& pr, double* sigma_sox);
Status sosex_selfenergy_imag(Context& c, const Wpol& w, const rigw_sosex_problem& pr, double* sigma);
Status g3w2_selfenergy_imag(Context& c, const Wpol& w, const rigw_g3w2_problem& pr, double* sigma);
Status gw_selfenergy_contour(Context& c, const rigw_contour_problem& pr, rigw_contour_result& res);
Status gw_density_matrix_imag(Context& c, const Wpol& w, const rigw_dm_problem& pr, double* p_matrix);
// RI integrals (ri_ints.cu): what = 2 (P|Q), 3 (mu nu|P) raw, 0 eri_3center with the metric.
Status ri_integrals(Context& c, const rigw_ri_problem& pr, int what, double* out, int* nkept);
// Eigenpairs of nw symmetric n x n matrices (n a multiple of 64, row-major, A[w] at A + w n^2):
// on return the diagonal of A[w] holds the eigenvalues and V[w][i][k] is component i of
// eigenvector k (eigh_jacobi.cu).  Adds its kernel launches to *launches.
Status eigh_jacobi_batched(Context& c, double* A, double* V, int n, int nw, cudaStream_t s, int* sweeps,
                           int* launches);
Status eri_3center_mo(Context& c, int nbf, int nstate, int npair, int naux, const int* index_basis,
                      const double* eri3, const double* c_matrix, int mstate_min, int mstate_max,
                      int nstate_min, int nstate_max, double* out, int precision, int flags = 0);
bool bf16x3_available();
Status validate_batch(int n, const rigw_problem* probs, std::vector<Shape>* shapes);
Status solve_batch(Context& c, int n, const rigw_problem* probs, rigw_result* res);
Status autotune(Context& c, int n, const rigw_problem* probs, rigw_tune_report* rep);
size_t available_bytes(Context& c);
Status make_split_tmap(void* host_map, const void* xs, int kpad, long long rows);
// The two tensor maps of the TMA-staged FP64 chi0 (256 bytes at host_maps):
// mp [nia_pad][npad] in 16 x 16 boxes with 128-byte swizzle, dscale [nomega][nia_pad] in 16 x 1 boxes.
Status make_f64_tmaps(void* host_maps, const double* mp, int npad, int nia_pad, const double* dscale, int nomega);
// box_bytes 128: 128-byte swizzle (syrk_ozaki_kernel); 64: 64-byte swizzle (syrk_ozaki_fused_kernel)
Status make_ozaki_tmap(void* host_map, const void* xq, int kpad, long long rows, int box_bytes = 128);

}  // namespace rigw
