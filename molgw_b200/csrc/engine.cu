// Host engine of the RI-GW library: plans, device memory, launch sequences.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <tuple>

#include "engine.cuh"

namespace rigw {

namespace {
constexpr size_t kAlign = 256;
inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }
inline int round_up(int v, int a) { return (v + a - 1) / a * a; }
}  // namespace

// ---------------------------------------------------------------------------
bool Shape::operator<(const Shape& o) const {
  return std::tie(naux, nocc, nvirt, nomega, nstate_p, nsig, nc, nsigma_half, technique, precision, qp_only, nocc2,
                  nvirt2) < std::tie(o.naux, o.nocc, o.nvirt, o.nomega, o.nstate_p, o.nsig, o.nc, o.nsigma_half,
                                     o.technique, o.precision, o.qp_only, o.nocc2, o.nvirt2);
}

Status make_shape(const rigw_problem& p, Shape* sh) {
  if (p.naux <= 0 || p.nocc < 0 || p.nvirt < 0 || p.nomega <= 0)
    return Status::fail(RIGW_ERR_ARG, "invalid W-window sizes naux=%d nocc=%d nvirt=%d nomega=%d", p.naux,
                        p.nocc, p.nvirt, p.nomega);
  if (p.nocc_2 < 0 || p.nvirt_2 < 0)
    return Status::fail(RIGW_ERR_ARG, "invalid second spin channel nocc_2=%d nvirt_2=%d", p.nocc_2, p.nvirt_2);
  if (p.nsig < 0 || p.nstate_p < 0)
    return Status::fail(RIGW_ERR_ARG, "invalid Sigma sizes nsig=%d nstate_p=%d", p.nsig, p.nstate_p);
  if (p.nomega_sigma_calc < 0 || p.nomega_sigma_calc > 128)
    return Status::fail(RIGW_ERR_ARG, "nomega_sigma_calc=%d outside [0,128]", p.nomega_sigma_calc);
  if (p.technique != RIGW_PADE && p.technique != RIGW_HOMOLUMO)
    return Status::fail(RIGW_ERR_ARG, "unknown technique %d", p.technique);
  if (p.precision != RIGW_FP64 && p.precision != RIGW_BF16X3 && !is_ozaki(p.precision))
    return Status::fail(RIGW_ERR_ARG, "unknown precision %d", p.precision);
  sh->naux = p.naux;
  sh->nocc = p.nocc;
  sh->nvirt = p.nvirt;
  sh->nocc2 = p.nocc_2;
  sh->nvirt2 = p.nvirt_2;
  sh->nomega = p.nomega;
  sh->nstate_p = p.nstate_p;
  sh->nsig = p.nsig;
  sh->nc = p.nomega_sigma_calc;
  sh->nsigma_half = p.nomega_sigma / 2;
  sh->technique = p.technique;
  sh->precision = p.precision;
  sh->qp_only = (p.flags & RIGW_PROBLEM_QP_ONLY) ? 1 : 0;
  return Status::ok();
}

// ---------------------------------------------------------------------------
DeviceBuffer::~DeviceBuffer() { release(); }

Status DeviceBuffer::allocate(Context* ctx, size_t bytes, const char* name) {
  release();
  if (bytes == 0) return Status::ok();
  ctx_ = ctx;
  // the context's spare block (the arena of a released plan) is reused as is
  if (ctx->spare_ptr && ctx->spare_bytes >= bytes) {
    ptr_ = ctx->spare_ptr;
    bytes_ = ctx->spare_bytes;
    ctx->spare_ptr = nullptr;
    ctx->spare_bytes = 0;
    return Status::ok();   // already counted in in_use
  }
  if (ctx->budget && ctx->in_use + bytes > ctx->budget) ctx->free_spare();
  if (ctx->budget && ctx->in_use + bytes > ctx->budget)
    return Status::fail(RIGW_ERR_NOMEM, "%s: %zu bytes exceed the HBM budget (%zu in use of %zu)", name, bytes,
                        ctx->in_use, ctx->budget);
  // Stream-ordered allocation from the device pool: memory released by a plan
  // stays mapped in the pool and is handed to the next plan without remapping.
  const auto t0 = std::chrono::steady_clock::now();
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&ptr_), bytes, ctx->stream);
  if (e != cudaSuccess && ctx->spare_ptr) {   // the spare block may be what is missing
    cudaGetLastError();
    ctx->free_spare();
    e = cudaMallocAsync(reinterpret_cast<void**>(&ptr_), bytes, ctx->stream);
  }
  if (e == cudaSuccess && !ctx->sync(ctx->stream).good()) e = cudaErrorUnknown;
  ctx->host_alloc_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (e != cudaSuccess) {
    ptr_ = nullptr;
    cudaGetLastError();
    return Status::fail(RIGW_ERR_NOMEM, "%s: cudaMallocAsync(%zu) failed: %s", name, bytes, cudaGetErrorString(e));
  }
  bytes_ = bytes;
  ctx->in_use += bytes;
  ctx->peak = std::max(ctx->peak, ctx->in_use);
  return Status::ok();
}

void DeviceBuffer::release() {
  if (ptr_) {
    ctx_->sync(ctx_->stream);
    if (bytes_ >= Context::kSpareMin && bytes_ > ctx_->spare_bytes) {
      // keep the larger block for the next plan of this context
      ctx_->free_spare();
      ctx_->spare_ptr = ptr_;
      ctx_->spare_bytes = bytes_;
    } else {
      cudaFreeAsync(ptr_, ctx_->stream);
      ctx_->in_use -= bytes_;
    }
  }
  ptr_ = nullptr;
  bytes_ = 0;
}

Status Context::reserve(size_t bytes) {
  free_spare();
  if (bytes < kSpareMin) return Status::ok();
  DeviceBuffer b;
  RIGW_TRY(b.allocate(this, bytes, "reserved arena"));
  b.release();   // a block of at least kSpareMin bytes becomes the spare block
  return Status::ok();
}

void Context::free_spare() {
  if (!spare_ptr) return;
  cudaFreeAsync(spare_ptr, stream);
  in_use -= spare_bytes;
  spare_ptr = nullptr;
  spare_bytes = 0;
}

// ---------------------------------------------------------------------------
Status Context::init(int dev, size_t budget_bytes, int want_priority, bool blocking_waits) {
  device = dev;
  budget = budget_bytes;
  RIGW_CUDA_TRY(cudaSetDevice(dev));
  int least = 0, greatest = 0;
  RIGW_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  priority = want_priority > 0 ? greatest : (want_priority < 0 ? least : 0);
  RIGW_CUDA_TRY(cudaStreamCreateWithPriority(&stream, cudaStreamNonBlocking, priority));
  if (blocking_waits)
    RIGW_CUDA_TRY(cudaEventCreateWithFlags(&sync_ev, cudaEventBlockingSync | cudaEventDisableTiming));
  for (auto& e : stage_ev) RIGW_CUDA_TRY(cudaEventCreate(&e));
  cudaMemPool_t pool;
  RIGW_CUDA_TRY(cudaDeviceGetDefaultMemPool(&pool, dev));
  uint64_t keep = ~uint64_t(0);
  RIGW_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  RIGW_CUDA_TRY(prepare_dgemm_kernels());
  RIGW_CUDA_TRY(prepare_syrk_f64_tma());
  RIGW_CUDA_TRY(prepare_tc_kernels());
  RIGW_CUDA_TRY(prepare_ozaki_kernels());
  RIGW_CUDA_TRY(cudaFuncSetAttribute(chol_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(chol_diag_smem_bytes())));
  return Status::ok();
}

Status Context::borrow(int nstreams, int nevents, std::vector<cudaStream_t>* streams,
                       std::vector<cudaEvent_t>* events) {
  while (int(aux_pool.size()) < nstreams) {
    cudaStream_t s = nullptr;
    RIGW_CUDA_TRY(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, priority));
    aux_pool.push_back(s);
  }
  while (int(order_pool.size()) < nevents) {
    cudaEvent_t e = nullptr;
    RIGW_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    order_pool.push_back(e);
  }
  streams->assign(aux_pool.begin(), aux_pool.begin() + nstreams);
  events->assign(order_pool.begin(), order_pool.begin() + nevents);
  return Status::ok();
}

char* Context::stage_take(size_t bytes) {
  if (!host_stage) {
    if (cudaHostAlloc(reinterpret_cast<void**>(&host_stage), kHostStage, cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();
      host_stage = nullptr;
      return nullptr;
    }
  }
  const size_t o = align_up(host_stage_used, kAlign);
  if (o + bytes > kHostStage) return nullptr;
  host_stage_used = o + bytes;
  return host_stage + o;
}

Status Context::sync(cudaStream_t s) {
  if (!sync_ev) {
    RIGW_CUDA_TRY(cudaStreamSynchronize(s));
    return Status::ok();
  }
  RIGW_CUDA_TRY(cudaEventRecord(sync_ev, s));
  RIGW_CUDA_TRY(cudaEventSynchronize(sync_ev));
  return Status::ok();
}

Context::~Context() {
  plan_cache.clear();
  free_spare();
  if (stream) {
    cudaStreamSynchronize(stream);
    cudaStreamDestroy(stream);
  }
  if (sync_ev) cudaEventDestroy(sync_ev);
  if (host_stage) cudaFreeHost(host_stage);
  for (auto& e : stage_ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : order_pool) cudaEventDestroy(e);
  for (auto& x : aux_pool) {
    cudaStreamSynchronize(x);
    cudaStreamDestroy(x);
  }
  // give the pool's unused memory back to the device (other contexts and
  // allocators of the process see it again)
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
  cudaGetLastError();
}

// ---------------------------------------------------------------------------
namespace {

struct Dims {
  int npad, npanel, nia, nia_pad, want_identity, moff, ncm, ldb, nreal;
};

Dims dims_of(const Shape& sh, PlanMode mode) {
  Dims d;
  d.npad = round_up(sh.naux, kPanel);
  d.npanel = d.npad / kPanel;
  d.nia = sh.nocc * sh.nvirt + sh.nocc2 * sh.nvirt2;
  // the int8 tensor-core K tile is 128 transitions (128 bytes), the bf16 one 64
  d.nia_pad = round_up(std::max(d.nia, 1), is_ozaki(sh.precision) ? 128 : 64);
  d.want_identity =
      (mode == kPlanPolar || ((mode == kPlanFused || mode == kPlanPartial) && !sh.qp_only)) ? 1 : 0;
  d.moff = d.want_identity ? d.npad : 0;
  d.ncm = (mode == kPlanFused || mode == kPlanSigma || mode == kPlanPartial) ? round_up(sh.nsig * sh.nstate_p, 8)
                                                                               : 0;
  d.ldb = d.moff + d.ncm;
  d.nreal = 2 * sh.nsigma_half + 1;
  return d;
}

}  // namespace

// Bytes of one frequency's split operands (bf16 hi/lo, or the Ozaki slices).
size_t split_bytes_per_frequency(const Shape& sh) {
  if (sh.precision == RIGW_FP64) return 0;
  const int npad = round_up(sh.naux, kPanel);
  const int nia = sh.nocc * sh.nvirt + sh.nocc2 * sh.nvirt2;
  const int nia_pad = round_up(std::max(nia, 1), is_ozaki(sh.precision) ? 128 : 64);
  return size_t(npad) * nia_pad * (is_ozaki(sh.precision) ? ozaki_slices(sh.precision) : 4);
}

namespace {

// Transitions per item of the split / slice / row-max kernels: wide items for
// large problems (fewer items to build), 64 otherwise (enough CTAs to fill the GPU).
int split_item_t(const Dims& d) { return (size_t(d.nia_pad / 64) * (d.npad / 64) >= 8192) ? kSplitT : 64; }

// Bump allocator over one arena; first pass measures, second pass assigns.
struct Layout {
  size_t cur = 0;
  size_t take(size_t bytes) {
    const size_t o = cur;
    cur = align_up(cur + std::max<size_t>(bytes, 1), kAlign);
    return o;
  }
};

}  // namespace

size_t footprint(const Shape& sh, PlanMode mode) { return Plan::measure({sh}, mode); }

Plan::~Plan() {
  for (int st = 0; st < 4; ++st) {
    if (stage_exec_[st]) cudaGraphExecDestroy(stage_exec_[st]);
    if (stage_graph_[st]) cudaGraphDestroy(stage_graph_[st]);
  }
}

size_t Plan::measure(const std::vector<Shape>& shapes, PlanMode mode, const Tuning* tune) {
  Plan p;
  size_t bytes = 0;
  Status s = p.build(nullptr, mode, shapes, {}, &bytes, tune);
  return s.good() ? bytes : size_t(-1);
}

int precision_class(const std::vector<Shape>& shapes) {
  int cls = -1;
  for (const Shape& sh : shapes) {
    const int c = sh.precision == RIGW_FP64 ? 0 : (sh.precision == RIGW_BF16X3 ? 1 : 2);
    cls = (cls < 0 || cls == c) ? c : 3;
  }
  return cls < 0 ? 0 : cls;
}

Status Plan::build(Context* ctx, PlanMode mode, const std::vector<Shape>& shapes,
                   const std::vector<const ProbDev*>& factors, size_t* measure_only, const Tuning* tune) {
  ctx_ = ctx;
  mode_ = mode;
  shapes_ = shapes;
  tune_ = tune ? *tune : (ctx ? ctx->tuning_for(mode, shapes) : Tuning{});
  if (tune_.chi0_rows != 128) tune_.chi0_rows = 64;
  if (tune_.update_rows != 128) tune_.update_rows = 64;
  const int np = int(shapes.size());
  probs_.assign(np, PlanProblem{});
  const bool factor = (mode == kPlanFused || mode == kPlanPolar || mode == kPlanPartial);
  const bool sigma = (mode == kPlanFused || mode == kPlanSigma || mode == kPlanPartial);
  const bool qp = (mode == kPlanFused || mode == kPlanQP);
  if (mode == kPlanSigma && int(factors.size()) != np && !measure_only)
    return Status::fail(RIGW_ERR_ARG, "sigma plan needs resident factors");
  const size_t D = sizeof(double);

  // Split precision: when the hi/lo buffers of every frequency of the batch are
  // small, one group holds all frequencies (one split and one tensor-core launch
  // with a full grid); otherwise groups of kSplitGroup frequencies share a buffer.
  size_t split_all = 0;
  for (const Shape& sh : shapes)
    if (factor && sh.precision != RIGW_FP64) {
      const Dims d = dims_of(sh, mode);
      split_all += size_t(sh.nomega) * d.npad * d.nia_pad * (is_ozaki(sh.precision) ? ozaki_slices(sh.precision) : 4);
    }
  const bool split_whole = split_all <= kSplitWholeBytes;
  auto split_group = [&](const Shape& sh) {
    if (tune_.split_group > 0) return std::max(1, std::min(sh.nomega, tune_.split_group));
    if (split_whole) return std::max(1, sh.nomega);
    // at most kSplitGroup frequencies, and at most kSplitProblemBytes per problem
    const Dims d = dims_of(sh, mode);
    const size_t per_w = size_t(d.npad) * d.nia_pad * (is_ozaki(sh.precision) ? ozaki_slices(sh.precision) : 4);
    const int cap = int(std::max<size_t>(1, kSplitProblemBytes / std::max<size_t>(per_w, 1)));
    return std::max(1, std::min({sh.nomega, kSplitGroup, cap}));
  };

  // ---- memory layout
  Layout L;
  struct Off {
    size_t mp, xs, tmap, rmax, xexp, tnorm, dscale, eps, winv, logdet, rhs, colsq, mnorm, vchiv, ew, tr, en, sc, sr, qp;
  };
  std::vector<Off> off(np);
  for (int i = 0; i < np; ++i) {
    const Shape& sh = shapes[i];
    const Dims d = dims_of(sh, mode);
    PlanProblem& pp = probs_[i];
    pp.sh = sh;
    if (factor) {
      pp.off_in_m = L.take(size_t(sh.nocc) * sh.nvirt * sh.naux * D);
      pp.off_in_eocc = L.take(size_t(sh.nocc) * D);
      pp.off_in_evirt = L.take(size_t(sh.nvirt) * D);
      pp.off_in_oocc = L.take(size_t(sh.nocc) * D);
      pp.off_in_ovirt = L.take(size_t(sh.nvirt) * D);
      const size_t nia2 = size_t(sh.nocc2) * sh.nvirt2;
      pp.off_in_m2 = L.take(nia2 * sh.naux * D);
      pp.off_in_eocc2 = L.take(size_t(sh.nocc2) * D);
      pp.off_in_evirt2 = L.take(size_t(sh.nvirt2) * D);
      pp.off_in_oocc2 = L.take(size_t(sh.nocc2) * D);
      pp.off_in_ovirt2 = L.take(size_t(sh.nvirt2) * D);
      pp.off_in_omega = L.take(size_t(sh.nomega) * D);
      pp.off_in_weight = L.take(size_t(sh.nomega) * D);
      off[i].mp = L.take(size_t(d.nia_pad) * d.npad * D);
      if (sh.precision == RIGW_FP64) {
        off[i].tmap = L.take(256);   // tensor maps of mp and dscale (TMA-staged FP64 chi0)
      } else if (sh.precision == RIGW_BF16X3) {
        off[i].xs = L.take(size_t(split_group(sh)) * 2 * d.npad * d.nia_pad * 2);
        off[i].tmap = L.take(128);
      } else if (is_ozaki(sh.precision)) {
        off[i].xs = L.take(size_t(split_group(sh)) * ozaki_slices(sh.precision) * d.npad * d.nia_pad);
        off[i].tmap = L.take(128);
        off[i].rmax = L.take(size_t(sh.nomega) * d.npad * sizeof(unsigned long long));
        off[i].xexp = L.take(size_t(sh.nomega) * d.npad * sizeof(int));
      }
      off[i].tnorm = L.take(size_t(d.nia_pad) * D);
      off[i].dscale = L.take(size_t(sh.nomega) * d.nia_pad * D);
      off[i].eps = L.take(size_t(sh.nomega) * d.npad * d.npad * D);
      off[i].winv = L.take(size_t(sh.nomega) * d.npanel * kPanel * kPanel * D);
      off[i].logdet = L.take(size_t(sh.nomega) * d.npanel * D);
      off[i].ew = L.take(size_t(sh.nomega) * 2 * D);
      off[i].tr = L.take(size_t(sh.nomega) * D);
      off[i].en = L.take(2 * D);
    }
    if (sigma) {
      pp.off_in_msig = L.take(size_t(sh.nsig) * sh.nstate_p * sh.naux * D);
      pp.off_in_ep = L.take(size_t(sh.nstate_p) * D);
      off[i].mnorm = L.take(size_t(d.ncm) * D);
      off[i].vchiv = L.take(size_t(sh.nomega) * d.ncm * D);
      if (mode == kPlanSigma) {
        pp.off_in_omega = L.take(size_t(sh.nomega) * D);
        pp.off_in_weight = L.take(size_t(sh.nomega) * D);
      }
    }
    if (d.ldb > 0) {
      off[i].rhs = L.take(size_t(sh.nomega) * d.npad * d.ldb * D);
      off[i].colsq = L.take(size_t(sh.nomega) * d.npanel * d.ldb * D);
    }
    if (sigma || qp) {
      pp.off_in_zcalc = L.take(size_t(2) * sh.nc * D);
      off[i].sc = L.take(size_t(2) * sh.nsig * sh.nc * D);
    }
    if (qp) {
      pp.off_in_esig = L.take(size_t(sh.nsig) * D);
      pp.off_in_xc = L.take(size_t(sh.nsig) * D);
      off[i].sr = L.take(size_t(2) * sh.nsig * d.nreal * D);
      off[i].qp = L.take(size_t(4) * sh.nsig * D);
    }
  }
  const size_t table_off = L.take(sizeof(ProbDev) * np);
  const size_t err_off = L.take(sizeof(int));
  if (measure_only) {
    // arena + a bound on the work lists (tiles of every stage, all frequencies)
    size_t lists = 0;
    for (const Shape& sh : shapes) {
      const Dims d = dims_of(sh, mode);
      const size_t t = size_t(d.npanel + 2) * (d.npanel + 2 + (d.ldb + 127) / 128) * 4;
      // GEMM items cover all frequencies of a chain; the WorkItem lists stay per frequency
      lists += size_t(kMaxChains + 1) * t * sizeof(GemmItem) +
               size_t(sh.nomega) * (d.npanel + 8) * sizeof(WorkItem) +
               size_t(d.nia_pad / 8 + d.npad * d.ldb / 1024 + 64) * 16;
      if (sh.precision != RIGW_FP64) {   // split items: (group, split_t transitions, 64 aux), + row maxima
        const int g = split_group(sh);
        lists += size_t((sh.nomega + g - 1) / g + 1) * (d.nia_pad / split_item_t(d) + 1) * (d.npad / 64) *
                     sizeof(WorkItem) +
                 size_t(sh.nomega) * d.npad / 4096 * sizeof(WorkItem) + 64;
      }
    }
    *measure_only = L.cur + lists + (size_t(1) << 20);
    return Status::ok();
  }
  RIGW_TRY(arena_.allocate(ctx, L.cur, "plan arena"));
  char* base = arena_.data();
  probs_dev_ = reinterpret_cast<ProbDev*>(base + table_off);
  err_dev_ = reinterpret_cast<int*>(base + err_off);
  auto dp = [&](size_t o) { return reinterpret_cast<double*>(base + o); };

  // ---- device descriptors
  for (int i = 0; i < np; ++i) {
    const Shape& sh = shapes[i];
    const Dims d = dims_of(sh, mode);
    ProbDev& p = probs_[i].dev;
    std::memset(&p, 0, sizeof(p));
    p.naux = sh.naux;
    p.npad = d.npad;
    p.nocc = sh.nocc;
    p.nvirt = sh.nvirt;
    p.nocc2 = sh.nocc2;
    p.nvirt2 = sh.nvirt2;
    p.nia1 = sh.nocc * sh.nvirt;
    p.nia = d.nia;
    p.nia_pad = d.nia_pad;
    p.nomega = sh.nomega;
    p.npanel = d.npanel;
    p.nsig = sh.nsig;
    p.nstate_p = sh.nstate_p;
    p.ncm = d.ncm;
    p.moff = d.moff;
    p.ldb = d.ldb;
    p.nc = sh.nc;
    p.nsigma_half = sh.nsigma_half;
    p.technique = sh.technique;
    p.want_identity = d.want_identity;
    if (factor) {
      p.mp = dp(off[i].mp);
      p.kpad = d.nia_pad;
      p.wgroup = split_group(sh);
      p.split_t = split_item_t(d);
      if (sh.precision == RIGW_BF16X3) {
        p.xs = base + off[i].xs;
        alignas(64) unsigned char map[128];
        RIGW_TRY(make_split_tmap(map, p.xs, d.nia_pad, (long long)p.wgroup * 2 * d.npad));
        RIGW_CUDA_TRY(cudaMemcpyAsync(base + off[i].tmap, map, sizeof(map), cudaMemcpyHostToDevice, ctx->stream));
      } else if (is_ozaki(sh.precision)) {
        p.slices = ozaki_slices(sh.precision);
        p.xs = base + off[i].xs;
        p.rmax = reinterpret_cast<unsigned long long*>(base + off[i].rmax);
        p.xexp = reinterpret_cast<int*>(base + off[i].xexp);
        alignas(64) unsigned char map[128];
        RIGW_TRY(make_ozaki_tmap(map, p.xs, d.nia_pad, (long long)p.wgroup * p.slices * d.npad,
                                 p.slices <= kOzaFusedMaxSlices ? 64 : 128));
        RIGW_CUDA_TRY(cudaMemcpyAsync(base + off[i].tmap, map, sizeof(map), cudaMemcpyHostToDevice, ctx->stream));
      }
      p.tnorm = dp(off[i].tnorm);
      p.dscale = dp(off[i].dscale);
      if (sh.precision == RIGW_FP64) {
        alignas(64) unsigned char maps[256];
        RIGW_TRY(make_f64_tmaps(maps, p.mp, d.npad, d.nia_pad, p.dscale, sh.nomega));
        RIGW_CUDA_TRY(cudaMemcpyAsync(base + off[i].tmap, maps, sizeof(maps), cudaMemcpyHostToDevice, ctx->stream));
      }
      p.eps = dp(off[i].eps);
      p.winv = dp(off[i].winv);
      p.logdet = dp(off[i].logdet);
      p.ew = dp(off[i].ew);
      p.treps = dp(off[i].tr);
      p.out_energies = dp(off[i].en);
    } else if (mode == kPlanSigma) {
      const ProbDev& f = *factors[i];
      p.eps = f.eps;
      p.winv = f.winv;
      p.npad = f.npad;
      p.npanel = f.npanel;
    }
    if (d.ldb > 0) {
      p.rhs = dp(off[i].rhs);
      p.colsq = dp(off[i].colsq);
    }
    if (sigma) {
      p.mnorm = dp(off[i].mnorm);
      p.vchiv = dp(off[i].vchiv);
    }
    if (sigma || qp) p.sigma_calc = dp(off[i].sc);
    if (qp) {
      p.sigma_real = dp(off[i].sr);
      p.qp = dp(off[i].qp);
    }
    p.err = err_dev_;
  }

  // ---- work lists
  const int BMN = 128;                  // column width of every DMMA item
  const int BMC = tune_.chi0_rows;      // row height of the FP64 chi0 items
  const int BM = tune_.update_rows;     // row height of the trailing-update items
  int max_panels = 0, npairs = 0;
  for (int i = 0; i < np; ++i) {
    max_panels = std::max(max_panels, probs_[i].dev.npanel);
    npairs += shapes[i].nomega;
  }
  // The factorization and solves of independent (problem, frequency) pairs run
  // as two chains on their own streams, each with its own one-panel lookahead,
  // so that one chain's launch tails and diagonal blocks overlap the other's GEMMs.
  // frequency chains: independent factorization sequences on their own streams,
  // at least kChainPairs (problem, frequency) pairs each
  nchains_ = tune_.chains > 0 ? std::max(1, std::min({tune_.chains, kMaxChains, npairs}))
                              : std::max(1, std::min(kAutoChains, npairs / kChainPairs));
  // panels per trailing update: longer updates pay off when many problems keep
  // the GPU busy; one or few problems keep pairs, whose factorization chain is shorter
  group_ = tune_.panel_group > 0 ? std::max(1, std::min(tune_.panel_group, 32)) : (np >= 4 ? 16 : 2);
  const int nlists = nchains_ * std::max(max_panels, 1);
  wl_diag_.assign(nlists, {});
  gl_k2_.assign(nlists, {});
  gl_k2n_.assign(nlists, {});
  gl_k3_.assign(nlists, {});
  gl_k3d_.assign(nlists, {});
  gl_k3a_.assign(nlists, {});
  int pair = 0;
  for (int i = 0; i < np; ++i) {
    const Shape& sh = shapes[i];
    const ProbDev& p = probs_[i].dev;
    const int npad = p.npad, ldb = p.ldb;
    if (factor) {
      for (int t0 = 0; t0 < p.nia_pad; t0 += 8) wl_pack_.push_back({i, t0, 0, 0});
      if (sh.precision == RIGW_BF16X3) {
        // frequencies in groups of p.wgroup sharing one hi/lo buffer: split(g), then chi0(g)
        for (int w0 = 0, g = 0; w0 < sh.nomega; w0 += p.wgroup, ++g) {
          if (int(wl_split_.size()) <= g) {
            wl_split_.resize(g + 1);
            tl_syrk_.resize(g + 1);
          }
          for (int t0 = 0; t0 < p.nia_pad; t0 += p.split_t)
            for (int p0 = 0; p0 < npad; p0 += 64) wl_split_[g].push_back({i, t0, p0, w0});
        }
        // one item per (group, tile) covering the group's frequencies
        for (int w0 = 0; w0 < sh.nomega; w0 += p.wgroup)
          for (int ti = 0; ti < npad; ti += BMN)
            for (int tj = ti; tj < npad; tj += BMN) {
              TcItem t{};
              t.tmap = base + off[i].tmap;
              t.C = p.eps + size_t(w0) * npad * npad + size_t(ti) * npad + tj;
              t.err = err_dev_;
              t.row_a = ti;
              t.row_b = tj;
              t.lo_off = npad;
              t.ktiles = p.kpad / 64;
              t.ldc = npad;
              t.diag = ti - tj;
              t.nw = std::min(p.wgroup, sh.nomega - w0);
              t.sC = (long long)npad * npad;
              t.srow = 2 * npad;
              tl_syrk_[w0 / p.wgroup].push_back(t);
            }
      }
      // FP64 chi0: upper 128-wide column strips in 64-row items (two CTAs per SM),
      // over the naux x naux block only; the identity pads are written afterwards
      if (is_ozaki(sh.precision)) {
        // row maxima of S over every frequency, then per frequency group: slices, chi0
        for (size_t e = 0; e < size_t(sh.nomega) * npad; e += 4096) wl_ozzero_.push_back({i, int(e), 0, 0});
        for (int t0 = 0; t0 < p.nia_pad; t0 += p.split_t)
          for (int p0 = 0; p0 < npad; p0 += 64) wl_rowmax_.push_back({i, t0, p0, 0});
        for (int w0 = 0, g = 0; w0 < sh.nomega; w0 += p.wgroup, ++g) {
          if (int(wl_slice_.size()) <= g) {
            wl_slice_.resize(g + 1);
            tl_ozaki_.resize(g + 1);
            tl_ozaki4_.resize(g + 1);
          }
          for (int t0 = 0; t0 < p.nia_pad; t0 += p.split_t)
            for (int p0 = 0; p0 < npad; p0 += 64) wl_slice_[g].push_back({i, t0, p0, w0});
        }
        for (int w0 = 0; w0 < sh.nomega; w0 += p.wgroup)
          for (int ti = 0; ti < npad; ti += BMN)
            for (int tj = ti; tj < npad; tj += BMN) {
              TcItem t{};
              t.tmap = base + off[i].tmap;
              t.C = p.eps + size_t(w0) * npad * npad + size_t(ti) * npad + tj;
              t.err = err_dev_;
              t.row_a = ti;
              t.row_b = tj;
              t.lo_off = npad;
              const bool fused = p.slices <= kOzaFusedMaxSlices;
              t.ktiles = p.kpad / (fused ? 64 : 128);
              t.ldc = npad;
              t.diag = ti - tj;
              t.ea = p.xexp + size_t(w0) * npad + ti;
              t.eb = p.xexp + size_t(w0) * npad + tj;
              t.slices = p.slices;
              t.nw = std::min(p.wgroup, sh.nomega - w0);
              t.sC = (long long)npad * npad;
              t.srow = p.slices * npad;
              t.se = npad;
              (fused ? tl_ozaki4_ : tl_ozaki_)[w0 / p.wgroup].push_back(t);
            }
      }
      if (sh.precision == RIGW_FP64) {
        // one item per tile covering every frequency (blockIdx.y); the tiles of a
        // row block start at its diagonal, so only the lower half of the
        // diagonal BMC x BMC block lies below it, and end at naux
        if (npad > sh.naux)
          for (int w = 0; w < sh.nomega; ++w) wl_pad_.push_back({i, w, 0, 0});
        // 64-row items: the TMA-staged kernel (its operands by TMA from the tensor
        // maps of mp and dscale); 128-row items (a tuner candidate): the cp.async engine
        if (BMC == 64)
          for (int ti = 0; ti < sh.naux; ti += BMC)
            for (int tj = ti; tj < sh.naux; tj += BMN) {
              F64SyrkItem f{};
              f.tmap_m = base + off[i].tmap;
              f.tmap_d = base + off[i].tmap + 128;
              f.C = p.eps + size_t(ti) * npad + tj;
              f.err = p.err;
              f.ti = ti;
              f.tj = tj;
              f.m = std::min(BMC, sh.naux - ti);
              f.n = std::min(BMN, sh.naux - tj);
              f.ktiles = p.nia_pad / 16;
              f.ldc = npad;
              f.diag = ti - tj;
              f.nw = sh.nomega;
              f.sC = (long long)npad * npad;
              fl_syrk_.push_back(f);
            }
        for (int ti = 0; BMC != 64 && ti < sh.naux; ti += BMC)
          for (int tj = ti; tj < sh.naux; tj += BMN) {
            GemmItem g{};
            g.A = p.mp + ti;
            g.B = p.mp + tj;
            g.lda = g.ldb = npad;
            g.C = p.eps + size_t(ti) * npad + tj;
            g.ldc = npad;
            g.kscale = p.dscale;
            g.m = std::min(BMC, sh.naux - ti);
            g.n = std::min(BMN, sh.naux - tj);
            g.k = p.nia_pad;
            g.flags = kAddIdentity;
            g.diag = ti - tj;
            g.alpha = 1.0;
            g.beta = 0.0;
            g.nw = sh.nomega;
            g.sC = (long long)npad * npad;
            g.sK = p.nia_pad;
            gl_syrk_.push_back(g);
          }
      }
      for (int w = 0; w < sh.nomega; ++w) wl_trace_.push_back({i, w, 0, 0});
    }
    if (ldb > 0) {
      for (int i0 = 0; i0 < npad; i0 += 32)
        for (int c0 = 0; c0 < ldb; c0 += 32) wl_rhs_.push_back({i, i0, c0, 0});
    }
    if (sigma)
      for (int c0 = 0; c0 < p.ncm; c0 += 8) wl_mnorm_.push_back({i, c0, 0, 0});
    for (int k = 0; k < p.npanel; ++k) {
      const int r0 = (k + 1) * kPanel;
      // frequency w belongs to chain (pair + w) % nchains; the items of one chain
      // cover its frequencies w0, w0 + nchains, ... (blockIdx.y)
      for (int ch = 0; ch < nchains_; ++ch) {
        const int w0 = ((ch - pair) % nchains_ + nchains_) % nchains_;
        if (w0 >= sh.nomega) continue;
        const int nw = (sh.nomega - w0 + nchains_ - 1) / nchains_;
        const long long step = nchains_;
        const int w = w0;
        double* E = p.eps + size_t(w) * npad * npad;
        double* R = p.rhs + size_t(w) * npad * ldb;
        const double* W = p.winv + (size_t(w) * p.npanel + k) * kPanel * kPanel;
        double* cs = p.colsq ? p.colsq + (size_t(w) * p.npanel + k) * ldb : nullptr;
        const long long sE = step * npad * npad, sR = step * npad * ldb;
        const long long sW = step * p.npanel * kPanel * kPanel, sQ = step * p.npanel * ldb;
        const int li = ch * max_panels + k;   // list of (chain, panel)
        if (factor)
          for (int wj = w0; wj < sh.nomega; wj += nchains_) wl_diag_[li].push_back({i, wj, 0, 0});
        auto k2 = [&](double* X, int ldx, int c0, int n, double* colsq) {
          GemmItem g{};
          g.A = W;
          g.lda = kPanel;
          g.B = X + size_t(k) * kPanel * ldx + c0;
          g.ldb = ldx;
          g.C = X + size_t(k) * kPanel * ldx + c0;
          g.ldc = ldx;
          g.colsq = colsq;
          g.m = kPanel;
          g.n = n;
          g.k = kPanel;
          g.alpha = 1.0;
          g.flags = kUpperA;   // W = U^-1 of the diagonal block is upper triangular
          g.nw = nw;
          g.sA = sW;
          g.sB = g.sC = (X == E) ? sE : sR;
          g.sQ = sQ;
          // the column block of the next panel goes first (the next diagonal block needs it)
          (X == E && c0 == r0 ? gl_k2n_[li] : gl_k2_[li]).push_back(g);
        };
        if (factor)
          for (int c0 = r0; c0 < npad; c0 += BMN) k2(E, npad, c0, std::min(BMN, npad - c0), nullptr);
        if (p.want_identity)
          for (int c0 = 0; c0 < r0; c0 += BMN) k2(R, ldb, c0, std::min(BMN, r0 - c0), cs + c0);
        for (int c0 = p.moff; c0 < ldb; c0 += BMN) k2(R, ldb, c0, std::min(BMN, ldb - c0), cs + c0);
        // Trailing update, panels in groups of G = group_: after panel k at position
        // j of its group (first panel kp = k - j) only the rows of panel k + 1 are
        // updated, with the U rows of panels kp .. k (K = (j+1) 128); after the last
        // panel of the group every row below it is updated once with the U rows of
        // the whole group, so each trailing tile is read and written once per group.
        // Items of the next diagonal block go to their own list (in both forms) so that
        // its factorization can start while the rest of the update runs (lookahead).
        const int jg = k % group_;
        const bool first_of_pair = jg != group_ - 1;           // not the group's last panel
        const int kp = k - jg;                                  // first panel of the U rows used
        const int kdim = (jg + 1) * kPanel;
        const int iend = first_of_pair ? std::min(npad, r0 + kPanel) : npad;
        auto k3 = [&](const double* Bsrc, int ldbs, double* Cdst, int ldc, int i0, int c0, int m, int n,
                      std::vector<GemmItem>& dst) {
          GemmItem g{};
          g.A = E + size_t(kp) * kPanel * npad + i0;
          g.lda = npad;
          g.B = Bsrc + size_t(kp) * kPanel * ldbs + c0;
          g.ldb = ldbs;
          g.C = Cdst + size_t(i0) * ldc + c0;
          g.Cin = g.C;
          g.ldc = ldc;
          g.m = m;
          g.n = n;
          g.k = kdim;
          g.alpha = -1.0;
          g.beta = 1.0;
          g.nw = nw;
          g.sA = sE;
          g.sB = (Bsrc == E) ? sE : sR;
          g.sC = (Cdst == E) ? sE : sR;
          dst.push_back(g);
        };
        std::vector<GemmItem>& rest = first_of_pair ? gl_k3a_[li] : gl_k3_[li];
        for (int i0 = r0; i0 < iend; i0 += BM) {
          const int m = std::min(BM, iend - i0);
          if (factor)
            for (int j0 = i0 / BMN * BMN; j0 < npad; j0 += BMN) {
              const bool next_diag = i0 < r0 + kPanel && j0 == r0;
              k3(E, npad, E, npad, i0, j0, m, std::min(BMN, npad - j0), next_diag ? gl_k3d_[li] : rest);
            }
          // I block: columns below r0 only (the U rows of panel kp have zeros beyond it there)
          if (p.want_identity)
            for (int c0 = 0; c0 < r0; c0 += BMN) k3(R, ldb, R, ldb, i0, c0, m, std::min(BMN, r0 - c0), rest);
          for (int c0 = p.moff; c0 < ldb; c0 += BMN) k3(R, ldb, R, ldb, i0, c0, m, std::min(BMN, ldb - c0), rest);
        }
      }
    }
    if (factor)
      for (int w = 0; w < sh.nomega; ++w) wl_energy_.push_back({i, w, 0, 0});
    if (sigma) {
      for (int w = 0; w < sh.nomega; ++w)
        for (int c0 = 0; c0 < p.ncm; c0 += 256) wl_vchiv_.push_back({i, w, c0, 0});
      for (int s = 0; s < sh.nsig; ++s)
        for (int kz = 0; kz < sh.nc; ++kz) wl_sigma_.push_back({i, s, kz, 0});
    }
    if (qp)
      for (int s = 0; s < sh.nsig; ++s) wl_pade_.push_back({i, s, 0, 0});
    pair += sh.nomega;
  }

  // chi0 items longest first: the block scheduler hands out CTAs in index order,
  // so a ragged batch ends on short tiles (results do not depend on the order)
  std::stable_sort(fl_syrk_.begin(), fl_syrk_.end(), [](const F64SyrkItem& a, const F64SyrkItem& b) {
    return double(a.ktiles) * a.m * a.n * std::max(a.nw, 1) > double(b.ktiles) * b.m * b.n * std::max(b.nw, 1);
  });
  std::stable_sort(gl_syrk_.begin(), gl_syrk_.end(), [](const GemmItem& a, const GemmItem& b) {
    return double(a.k) * a.m * a.n * std::max(a.nw, 1) > double(b.k) * b.m * b.n * std::max(b.nw, 1);
  });
  auto by_cost = [](const TcItem& a, const TcItem& b) {
    return double(a.ktiles) * std::max(a.nw, 1) > double(b.ktiles) * std::max(b.nw, 1);
  };
  for (auto& l : tl_syrk_) std::stable_sort(l.begin(), l.end(), by_cost);
  for (auto& l : tl_ozaki_) std::stable_sort(l.begin(), l.end(), by_cost);
  for (auto& l : tl_ozaki4_) std::stable_sort(l.begin(), l.end(), by_cost);

  // ---- upload the lists and the launch sequence
  size_t lbytes = 0;
  auto reserve = [&](size_t n) {
    const size_t o = lbytes;
    lbytes = align_up(lbytes + n, kAlign);
    return o;
  };
  struct Pending {
    int kind;
    const void* src;
    size_t bytes;
    int count;
    int arg;
    int stream, wait_ev, rec_ev;
    int ny;
  };
  std::vector<Pending> pend;
  auto add = [&](int kind, const void* src, size_t elem, size_t n, int arg, int stream = 0, int wait_ev = -1,
                 int rec_ev = -1) {
    if (n == 0) return false;
    // grid y of the item lists that cover several frequencies
    int ny = 1;
    if (kind == 1 || kind == 5 || kind == 6 || kind == 14)
      for (size_t j = 0; j < n; ++j) ny = std::max(ny, static_cast<const GemmItem*>(src)[j].nw);
    if (kind == 13 || kind == 20 || kind == 21)
      for (size_t j = 0; j < n; ++j) ny = std::max(ny, static_cast<const TcItem*>(src)[j].nw);
    if (kind == 22)
      for (size_t j = 0; j < n; ++j) ny = std::max(ny, static_cast<const F64SyrkItem*>(src)[j].nw);
    pend.push_back({kind, src, elem * n, int(n), arg, stream, wait_ev, rec_ev, ny});
    return true;
  };
  add(0, wl_pack_.data(), sizeof(WorkItem), wl_pack_.size(), 0);
  add(2, wl_rhs_.data(), sizeof(WorkItem), wl_rhs_.size(), 0);
  add(3, wl_mnorm_.data(), sizeof(WorkItem), wl_mnorm_.size(), 0);
  add(1, gl_syrk_.data(), sizeof(GemmItem), gl_syrk_.size(), 0);
  add(22, fl_syrk_.data(), sizeof(F64SyrkItem), fl_syrk_.size(), 0);
  for (size_t g = 0; g < wl_split_.size(); ++g) {
    add(12, wl_split_[g].data(), sizeof(WorkItem), wl_split_[g].size(), 0);
    add(13, tl_syrk_[g].data(), sizeof(TcItem), tl_syrk_[g].size(), 0);
  }
  add(17, wl_ozzero_.data(), sizeof(WorkItem), wl_ozzero_.size(), 0);
  add(18, wl_rowmax_.data(), sizeof(WorkItem), wl_rowmax_.size(), 0);
  for (size_t g = 0; g < wl_slice_.size(); ++g) {
    add(19, wl_slice_[g].data(), sizeof(WorkItem), wl_slice_[g].size(), 0);
    add(20, tl_ozaki_[g].data(), sizeof(TcItem), tl_ozaki_[g].size(), 0);
    add(21, tl_ozaki4_[g].data(), sizeof(TcItem), tl_ozaki4_[g].size(), 0);
  }
  add(16, wl_pad_.data(), sizeof(WorkItem), wl_pad_.size(), 0);
  add(15, wl_trace_.data(), sizeof(WorkItem), wl_trace_.size(), 0);
  // Panel loop of each chain with a one-panel lookahead.  After the diagonal block
  // of panel k: on the chain's main stream the panel solve of the next panel's
  // column block (K2n), then on the lookahead stream the update of the next
  // diagonal block (K3d) and its factorization, while the main stream solves the
  // rest of panel k (K2) and runs the rest of the trailing update (K3a / K3).  The
  // next panel's solve waits for both.  Streams: chain c uses 2c (main) and 2c+1
  // (lookahead); stream 0 is the plan's own stream.  Kind -1 launches nothing
  // (event marker).
  int nev = 0;
  const int fork_ev = nchains_ > 1 ? nev++ : -1;
  if (fork_ev >= 0) pend.push_back({-1, nullptr, 0, 0, 0, 0, -1, fork_ev, 1});
  std::vector<int> chain_end;
  for (int ch = 0; ch < nchains_; ++ch) {
    const int sm = 2 * ch, sl = 2 * ch + 1;
    int pending = ch > 0 ? fork_ev : -1;
    auto L = [&](int k) { return ch * max_panels + k; };
    for (int k = 0; k < max_panels; ++k) {
      if (k == 0 && add(4, wl_diag_[L(0)].data(), sizeof(WorkItem), wl_diag_[L(0)].size(), 0, sm, pending))
        pending = -1;
      const bool next = k + 1 < max_panels && !wl_diag_[L(k + 1)].empty();
      std::vector<GemmItem>& rest3 = k % group_ != group_ - 1 ? gl_k3a_[L(k)] : gl_k3_[L(k)];
      if (next && !gl_k2n_[L(k)].empty() && !gl_k3d_[L(k)].empty()) {
        const int ea = nev++, eb = nev++;
        add(5, gl_k2n_[L(k)].data(), sizeof(GemmItem), gl_k2n_[L(k)].size(), k, sm, pending, ea);
        pending = -1;
        add(14, gl_k3d_[L(k)].data(), sizeof(GemmItem), gl_k3d_[L(k)].size(), k, sl, ea);
        add(4, wl_diag_[L(k + 1)].data(), sizeof(WorkItem), wl_diag_[L(k + 1)].size(), k + 1, sl, -1, eb);
        add(5, gl_k2_[L(k)].data(), sizeof(GemmItem), gl_k2_[L(k)].size(), k, sm);
        add(6, rest3.data(), sizeof(GemmItem), rest3.size(), k, sm);
        pending = eb;
        continue;
      }
      // no next panel (or nothing to update ahead of it): everything on the main stream
      if (add(5, gl_k2n_[L(k)].data(), sizeof(GemmItem), gl_k2n_[L(k)].size(), k, sm, pending)) pending = -1;
      if (add(5, gl_k2_[L(k)].data(), sizeof(GemmItem), gl_k2_[L(k)].size(), k, sm, pending)) pending = -1;
      if (add(14, gl_k3d_[L(k)].data(), sizeof(GemmItem), gl_k3d_[L(k)].size(), k, sm, pending)) pending = -1;
      if (add(6, rest3.data(), sizeof(GemmItem), rest3.size(), k, sm, pending)) pending = -1;
      if (next && add(4, wl_diag_[L(k + 1)].data(), sizeof(WorkItem), wl_diag_[L(k + 1)].size(), k + 1, sm,
                      pending))
        pending = -1;
    }
    if (ch > 0) {
      const int ej = nev++;
      pend.push_back({-1, nullptr, 0, 0, 0, sm, pending, ej, 1});   // joins the lookahead, marks the chain's end
      chain_end.push_back(ej);
    } else if (pending >= 0) {
      pend.push_back({-1, nullptr, 0, 0, 0, 0, pending, -1, 1});
    }
  }
  for (int ej : chain_end) pend.push_back({-1, nullptr, 0, 0, 0, 0, ej, -1, 1});
  add(7, wl_energy_.data(), sizeof(WorkItem), wl_energy_.size(), 0);
  if (factor) pend.push_back({8, nullptr, 0, np, 0, 0, -1, -1, 1});
  add(9, wl_vchiv_.data(), sizeof(WorkItem), wl_vchiv_.size(), 0);
  add(10, wl_sigma_.data(), sizeof(WorkItem), wl_sigma_.size(), 0);
  add(11, wl_pade_.data(), sizeof(WorkItem), wl_pade_.size(), 0);
  std::vector<size_t> offs;
  for (auto& pd : pend) offs.push_back(pd.bytes ? reserve(pd.bytes) : 0);
  RIGW_TRY(lists_.allocate(ctx, std::max<size_t>(lbytes, kAlign), "plan work lists"));
  std::vector<char> host(lbytes);
  for (size_t j = 0; j < pend.size(); ++j) {
    if (pend[j].bytes) std::memcpy(host.data() + offs[j], pend[j].src, pend[j].bytes);
    seq_.push_back({pend[j].kind, offs[j], pend[j].count, pend[j].arg, pend[j].stream, pend[j].wait_ev,
                    pend[j].rec_ev, pend[j].ny});
  }
  RIGW_CUDA_TRY(cudaMemcpyAsync(lists_.data(), host.data(), lbytes, cudaMemcpyHostToDevice, ctx->stream));
  RIGW_TRY(ctx->sync(ctx->stream));   // the host staging vector goes out of scope
  RIGW_TRY(ctx->borrow(2 * nchains_ - 1, std::max(nev, 1), &aux_streams_, &la_ev_));
  for (int k = 0; k < 5; ++k) stage_ev_[k] = ctx->stage_ev[k];
  host_table_.resize(np);
  n_launches_ = int(seq_.size());
  return Status::ok();
}

// Stage of a launch kind: 0 input packing, 1 chi0, 2 eps factorization and
// solves, 3 energies / Sigma / QP.  Each stage is its own CUDA graph; CUDA
// events between the stage graphs time every replay stage by stage.
static int stage_of(int kind) {
  switch (kind) {
    case 0: case 2: case 3: return 0;
    case 1: case 12: case 13: case 15: case 16: case 17: case 18: case 19: case 20: case 21: case 22: return 1;
    case -1: case 4: case 5: case 6: case 14: return 2;
    default: return 3;
  }
}

void Plan::record(cudaStream_t s0, int stage) {
  char* lb = lists_.data();
  for (const Launch& L : seq_) {
    if (stage >= 0 && stage_of(L.kind) != stage) continue;
    cudaStream_t s = L.stream ? aux_streams_[L.stream - 1] : s0;
    if (L.wait_ev >= 0) cudaStreamWaitEvent(s, la_ev_[L.wait_ev], 0);
    if (L.kind < 0) {
      if (L.rec_ev >= 0) cudaEventRecord(la_ev_[L.rec_ev], s);
      continue;
    }
    const WorkItem* wl = reinterpret_cast<const WorkItem*>(lb + L.off);
    const GemmItem* gl = reinterpret_cast<const GemmItem*>(lb + L.off);
    switch (L.kind) {
      case 0: pack_m_kernel<<<L.count, 256, 0, s>>>(probs_dev_, wl); break;
      case 1:
        if (tune_.chi0_rows == 128) launch_dgemm_128x128(gl, L.count, L.ny, s);
        else launch_dgemm_64x128(gl, L.count, L.ny, s);
        break;
      case 6: case 14:
        if (tune_.update_rows == 128) launch_dgemm_128x128(gl, L.count, L.ny, s);
        else launch_dgemm_64x128(gl, L.count, L.ny, s);
        break;
      case 15: trace_kernel<<<L.count, 256, 0, s>>>(probs_dev_, wl); break;
      case 16: pad_eps_kernel<<<L.count, 256, 0, s>>>(probs_dev_, wl); break;
      case 12: launch_split_bf16x3(probs_dev_, wl, L.count, s); break;
      case 13: launch_syrk_bf16x3(reinterpret_cast<const TcItem*>(lb + L.off), L.count, L.ny, s); break;
      case 22: launch_syrk_f64_tma(reinterpret_cast<const F64SyrkItem*>(lb + L.off), L.count, L.ny, s); break;
      case 17: launch_ozaki_zero(probs_dev_, wl, L.count, s); break;
      case 18: launch_ozaki_rowmax(probs_dev_, wl, L.count, s); break;
      case 19: launch_ozaki_slice(probs_dev_, wl, L.count, s); break;
      case 20: launch_syrk_ozaki(reinterpret_cast<const TcItem*>(lb + L.off), L.count, L.ny, s); break;
      case 21: launch_syrk_ozaki_fused(reinterpret_cast<const TcItem*>(lb + L.off), L.count, L.ny, s); break;
      case 2: init_rhs_kernel<<<L.count, 256, 0, s>>>(probs_dev_, wl); break;
      case 3: mnorm_kernel<<<L.count, 256, 0, s>>>(probs_dev_, wl); break;
      case 4: chol_diag_kernel<<<L.count, kDiagThreads, chol_diag_smem_bytes(), s>>>(probs_dev_, wl, L.arg); break;
      case 5: launch_dgemm_128x128(gl, L.count, L.ny, s); break;
      case 7: energy_kernel<<<L.count, 256, 0, s>>>(probs_dev_, wl); break;
      case 8: energy_sum_kernel<<<(L.count + 127) / 128, 128, 0, s>>>(probs_dev_, L.count); break;
      case 9: vchiv_kernel<<<L.count, 256, 0, s>>>(probs_dev_, wl); break;
      case 10: sigma_kernel<<<L.count, 256, 0, s>>>(probs_dev_, wl); break;
      case 11: pade_qp_kernel<<<L.count, 256, 0, s>>>(probs_dev_, wl); break;
      default: break;
    }
    if (L.rec_ev >= 0) cudaEventRecord(la_ev_[L.rec_ev], s);
  }
}

// Gauss-Legendre imaginary grid (coeffs_gausslegint + the [0,1) -> [0,inf) map).
void imag_grid(int n, double* omega, double* weight) {
  const double pi = 3.14159265358979323;
  std::vector<double> x(n), w(n);
  const double tol = 1.0e-13, xl = 0.5, xmean = 0.5;
  for (int i = 1; i <= (n + 1) / 2; ++i) {
    double z = std::cos(pi * (i - 0.25) / (n + 0.5)), z1, pp, p1, p2, p3;
    do {
      p1 = 1.0;
      p2 = 0.0;
      for (int j = 1; j <= n; ++j) {
        p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = n * (p2 - z * p1) / (1.0 - z * z);
      z1 = z;
      z = z1 - p1 / pp;
    } while (std::fabs(z - z1) >= tol);
    x[i - 1] = xmean - xl * z;
    x[n - i] = xmean + xl * z;
    w[i - 1] = 2.0 * xl / ((1.0 - z * z) * pp * pp);
    w[n - i] = w[i - 1];
  }
  const double alpha = 1.0, beta = 2.0;
  for (int k = 0; k < n; ++k) {
    weight[k] = w[k] / (std::pow(2.0, alpha) - 1.0) * alpha * std::pow(1.0 - x[k], -alpha - 1.0) * beta;
    omega[k] = 1.0 / (std::pow(2.0, alpha) - 1.0) * (1.0 / std::pow(1.0 - x[k], alpha) - 1.0) * beta;
  }
}

Status Plan::stage_inputs(const rigw_problem* probs, cudaStream_t s) {
  char* base = arena_.data();
  auto dp = [&](size_t o) { return reinterpret_cast<double*>(base + o); };
  const bool factor = (mode_ == kPlanFused || mode_ == kPlanPolar || mode_ == kPlanPartial);
  const bool sigma = (mode_ == kPlanFused || mode_ == kPlanSigma || mode_ == kPlanPartial);
  const bool qp = (mode_ == kPlanFused || mode_ == kPlanQP);
  std::deque<std::vector<double>> keep;   // host sources of the copies below
  ctx_->stage_reset();
  // host -> device copy of `bytes`; small host sources go through the pinned staging area
  auto h2d = [&](void* dst, const void* src, size_t bytes) -> Status {
    cudaPointerAttributes a{};
    const bool dev_src = cudaPointerGetAttributes(&a, src) == cudaSuccess &&
                         (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged);
    cudaGetLastError();
    char* st = (!dev_src && bytes <= (size_t(1) << 20)) ? ctx_->stage_take(bytes) : nullptr;
    if (st) {
      std::memcpy(st, src, bytes);
      RIGW_CUDA_TRY(cudaMemcpyAsync(dst, st, bytes, cudaMemcpyHostToDevice, s));
    } else {
      RIGW_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, s));
    }
    return Status::ok();
  };
  for (size_t i = 0; i < probs_.size(); ++i) {
    const rigw_problem& q = probs[i];
    PlanProblem& pp = probs_[i];
    ProbDev& p = pp.dev;
    const Shape& sh = pp.sh;
    const bool on_dev = (q.flags & RIGW_PROBLEM_DEVICE_POINTERS) != 0;
    auto bind = [&](const double* user, size_t off, size_t n, const char* what, const double** slot) -> Status {
      if (n == 0) {
        *slot = dp(off);
        return Status::ok();
      }
      if (!user) return Status::fail(RIGW_ERR_ARG, "problem %zu: %s is NULL", i, what);
      if (on_dev) {
        *slot = user;
      } else {
        RIGW_TRY(h2d(dp(off), user, n * sizeof(double)));
        *slot = dp(off);
      }
      return Status::ok();
    };
    if (factor || sigma) {
      // frequency grid: caller's or Gauss-Legendre
      if (q.omega && q.weight) {
        // small arrays: always copied (host or device source), so that a frequency
        // chunk may pass host subsets of the grid beside device-resident tensors
        RIGW_TRY(h2d(dp(pp.off_in_omega), q.omega, sh.nomega * 8));
        RIGW_TRY(h2d(dp(pp.off_in_weight), q.weight, sh.nomega * 8));
        p.omega = dp(pp.off_in_omega);
        p.weight = dp(pp.off_in_weight);
      } else {
        keep.emplace_back(sh.nomega);
        std::vector<double>& om = keep.back();
        keep.emplace_back(sh.nomega);
        std::vector<double>& wt = keep.back();
        imag_grid(sh.nomega, om.data(), wt.data());
        RIGW_TRY(h2d(dp(pp.off_in_omega), om.data(), om.size() * 8));
        RIGW_TRY(h2d(dp(pp.off_in_weight), wt.data(), wt.size() * 8));
        p.omega = dp(pp.off_in_omega);
        p.weight = dp(pp.off_in_weight);
      }
    }
    if (factor) {
      const size_t nia = size_t(sh.nocc) * sh.nvirt;
      RIGW_TRY(bind(q.m_ia, pp.off_in_m, nia * sh.naux, "m_ia", &p.m_in));
      RIGW_TRY(bind(q.e_occ, pp.off_in_eocc, sh.nocc, "e_occ", &p.e_occ));
      RIGW_TRY(bind(q.e_virt, pp.off_in_evirt, sh.nvirt, "e_virt", &p.e_virt));
      RIGW_TRY(bind(q.occ_occ, pp.off_in_oocc, sh.nocc, "occ_occ", &p.occ_occ));
      RIGW_TRY(bind(q.occ_virt, pp.off_in_ovirt, sh.nvirt, "occ_virt", &p.occ_virt));
      const size_t nia2 = size_t(sh.nocc2) * sh.nvirt2;
      RIGW_TRY(bind(q.m_ia_2, pp.off_in_m2, nia2 * sh.naux, "m_ia_2", &p.m_in2));
      RIGW_TRY(bind(q.e_occ_2, pp.off_in_eocc2, sh.nocc2, "e_occ_2", &p.e_occ2));
      RIGW_TRY(bind(q.e_virt_2, pp.off_in_evirt2, sh.nvirt2, "e_virt_2", &p.e_virt2));
      RIGW_TRY(bind(q.occ_occ_2, pp.off_in_oocc2, sh.nocc2, "occ_occ_2", &p.occ_occ2));
      RIGW_TRY(bind(q.occ_virt_2, pp.off_in_ovirt2, sh.nvirt2, "occ_virt_2", &p.occ_virt2));
    }
    if (sigma) {
      RIGW_TRY(bind(q.m_pm, pp.off_in_msig, size_t(sh.nsig) * sh.nstate_p * sh.naux, "m_pm", &p.msig_in));
      RIGW_TRY(bind(q.e_p, pp.off_in_ep, sh.nstate_p, "e_p", &p.e_p));
    }
    if (sigma || qp) {
      if (q.omega_calc) {
        RIGW_TRY(bind(q.omega_calc, pp.off_in_zcalc, size_t(2) * sh.nc, "omega_calc", &p.zcalc));
      } else {
        if (sh.technique != RIGW_PADE)
          return Status::fail(RIGW_ERR_ARG, "problem %zu: homolumo technique needs omega_calc", i);
        keep.emplace_back(2 * sh.nc);
        std::vector<double>& z = keep.back();
        for (int k = 0; k < sh.nc; ++k) {
          z[2 * k] = q.efermi;
          z[2 * k + 1] = q.step_sigma_calc * k;
        }
        RIGW_TRY(h2d(dp(pp.off_in_zcalc), z.data(), z.size() * 8));
        p.zcalc = dp(pp.off_in_zcalc);
      }
    }
    if (qp) {
      RIGW_TRY(bind(q.e_sig, pp.off_in_esig, sh.nsig, "e_sig", &p.e_sig));
      if (q.exchange_m_vxc) {
        RIGW_TRY(bind(q.exchange_m_vxc, pp.off_in_xc, sh.nsig, "exchange_m_vxc", &p.xc_sig));
      } else {
        p.xc_sig = nullptr;
      }
      p.efermi = q.efermi;
      p.step_sigma = q.step_sigma;
      p.eta = q.eta;
    }
    host_table_[i] = p;
  }
  RIGW_TRY(h2d(probs_dev_, host_table_.data(), sizeof(ProbDev) * host_table_.size()));
  // copies from pageable host memory are staged before cudaMemcpyAsync returns:
  // the host vectors in `keep` may go out of scope without a wait
  return Status::ok();
}

Status Plan::stage_sigma_calc(int i, const double* sc, cudaStream_t s) {
  ProbDev& p = probs_[i].dev;
  RIGW_CUDA_TRY(cudaMemcpyAsync(p.sigma_calc, sc, sizeof(double) * 2 * p.nsig * p.nc, cudaMemcpyDefault, s));
  return Status::ok();
}

// NVTX labels of the four stages (the reference's timer names)
static const char* const kStageRange[4] = {"Response function chi on grid: packing",
                                           "Response function chi on grid: chi0",
                                           "Response function chi on grid: eps factorization and solves",
                                           "GW self-energy"};

Status Plan::launch(cudaStream_t s) {
  RIGW_CUDA_TRY(cudaMemsetAsync(err_dev_, 0, sizeof(int), s));
  // the first launch of a plan goes straight to the streams; a plan launched
  // again is captured into CUDA graphs once and replayed from then on
  if (ctx_->use_graphs && launches_++ > 0) {
    for (int st = 0; st < 4; ++st) {
      if (stage_exec_[st] || stage_empty_[st]) continue;
      bool any = false;
      for (const Launch& L : seq_) any |= stage_of(L.kind) == st;
      if (!any) {
        stage_empty_[st] = true;
        continue;
      }
      const auto t_cap = std::chrono::steady_clock::now();
      RIGW_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      record(s, st);
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamEndCapture(s, &g);
      if (e != cudaSuccess)
        return Status::fail(RIGW_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
      stage_graph_[st] = g;
      RIGW_CUDA_TRY(cudaGraphInstantiate(&stage_exec_[st], g, 0));
      ctx_->host_capture_ms +=
          std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_cap).count();
    }
    for (int st = 0; st < 4; ++st) {
      NvtxRange range(kStageRange[st]);
      RIGW_CUDA_TRY(cudaEventRecord(stage_ev_[st], s));
      if (stage_exec_[st]) RIGW_CUDA_TRY(cudaGraphLaunch(stage_exec_[st], s));
    }
    RIGW_CUDA_TRY(cudaEventRecord(stage_ev_[4], s));
    replayed_ = true;
  } else {
    replayed_ = false;
    for (int st = 0; st < 4; ++st) {
      NvtxRange range(kStageRange[st]);
      RIGW_CUDA_TRY(cudaEventRecord(stage_ev_[st], s));
      record(s, st);
      RIGW_CUDA_TRY(cudaGetLastError());
    }
    RIGW_CUDA_TRY(cudaEventRecord(stage_ev_[4], s));
  }
  return Status::ok();
}

Status Plan::check_errors(cudaStream_t s) {
  int err = 0;
  RIGW_CUDA_TRY(cudaMemcpyAsync(&err, err_dev_, sizeof(int), cudaMemcpyDeviceToHost, s));
  RIGW_TRY(ctx_->sync(s));
  RIGW_CUDA_TRY(cudaEventElapsedTime(&last_ms_, stage_ev_[0], stage_ev_[4]));
  for (int k = 0; k < 4; ++k) RIGW_CUDA_TRY(cudaEventElapsedTime(&stage_ms_[k], stage_ev_[k], stage_ev_[k + 1]));
  if (err & kErrNotSPD) return Status::fail(RIGW_ERR_NOT_SPD, "eps(iw) is not positive definite");
  if (err & kErrTimeout) return Status::fail(RIGW_ERR_TIMEOUT, "a bounded device wait expired");
  if (err & (kErrNonFinite | kErrPade))
    return Status::fail(RIGW_ERR_NUMERIC, "non-finite QP energy or singular Pade recursion (flags %d)", err);
  return Status::ok();
}

Status Plan::fetch_results(const rigw_problem* probs, rigw_result* res, cudaStream_t s) {
  // pass 1: every small output and input of the batch to pinned host memory, one wait
  const size_t np = probs_.size();
  ctx_->stage_reset();
  auto is_dev = [](const void* ptr) {
    cudaPointerAttributes a{};
    const bool d = cudaPointerGetAttributes(&a, ptr) == cudaSuccess &&
                   (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged);
    cudaGetLastError();
    return d;
  };
  struct Host {
    double* en = nullptr;      // [2]
    double* q = nullptr;       // [4 nsig]
    double* occ = nullptr;     // [nsig]
    double spin_fact = 2.0;    // occupation of a full state
    double* sc = nullptr;      // sigma_calc staged for a host destination
    double* sr = nullptr;      // sigma (real grid) staged for a host destination
  };
  std::vector<Host> h(np);
  std::vector<std::vector<double>> own;   // fallback when the staging area is full
  auto take = [&](size_t n) -> double* {
    char* st = ctx_->stage_take(n * sizeof(double));
    if (st) return reinterpret_cast<double*>(st);
    own.emplace_back(n);
    return own.back().data();
  };
  for (size_t i = 0; i < np; ++i) {
    const ProbDev& p = probs_[i].dev;
    rigw_result& r = res[i];
    const int nreal = 2 * p.nsigma_half + 1;
    const size_t nsc = size_t(2) * p.nsig * p.nc, nsr = size_t(2) * p.nsig * nreal;
    if (p.out_energies) {
      h[i].en = take(2);
      RIGW_CUDA_TRY(cudaMemcpyAsync(h[i].en, p.out_energies, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    if (r.sigma_calc && p.sigma_calc && mode_ != kPlanQP) {
      if (is_dev(r.sigma_calc)) {
        RIGW_CUDA_TRY(cudaMemcpyAsync(r.sigma_calc, p.sigma_calc, nsc * sizeof(double), cudaMemcpyDeviceToDevice, s));
      } else {
        h[i].sc = take(nsc);
        RIGW_CUDA_TRY(cudaMemcpyAsync(h[i].sc, p.sigma_calc, nsc * sizeof(double), cudaMemcpyDeviceToHost, s));
      }
    }
    if (r.sigma && p.sigma_real) {
      if (is_dev(r.sigma)) {
        RIGW_CUDA_TRY(cudaMemcpyAsync(r.sigma, p.sigma_real, nsr * sizeof(double), cudaMemcpyDeviceToDevice, s));
      } else {
        h[i].sr = take(nsr);
        RIGW_CUDA_TRY(cudaMemcpyAsync(h[i].sr, p.sigma_real, nsr * sizeof(double), cudaMemcpyDeviceToHost, s));
      }
    }
    if (p.qp) {
      h[i].q = take(4 * size_t(p.nsig));
      h[i].occ = take(p.nsig);
      std::fill(h[i].occ, h[i].occ + p.nsig, 0.0);
      h[i].spin_fact = ((probs[i].flags & RIGW_PROBLEM_SPIN_CHANNEL) || probs[i].nocc_2 > 0) ? 1.0 : 2.0;
      RIGW_CUDA_TRY(cudaMemcpyAsync(h[i].q, p.qp, 4 * p.nsig * sizeof(double), cudaMemcpyDeviceToHost, s));
      if (probs[i].occ_sig) {
        if (is_dev(probs[i].occ_sig))
          RIGW_CUDA_TRY(cudaMemcpyAsync(h[i].occ, probs[i].occ_sig, p.nsig * sizeof(double), cudaMemcpyDeviceToHost,
                                        s));
        else
          std::memcpy(h[i].occ, probs[i].occ_sig, p.nsig * sizeof(double));
      }
    }
  }
  RIGW_TRY(ctx_->sync(s));
  // pass 2: QP energies and output_homolumo on the host, copies to the caller's buffers
  std::deque<std::vector<double>> out_dev;   // host sources of copies to device destinations
  auto put = [&](double* dst, const double* src, size_t n) -> Status {
    if (is_dev(dst)) {
      out_dev.emplace_back(src, src + n);
      RIGW_CUDA_TRY(cudaMemcpyAsync(dst, out_dev.back().data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
    } else {
      std::memcpy(dst, src, n * sizeof(double));
    }
    return Status::ok();
  };
  for (size_t i = 0; i < np; ++i) {
    const ProbDev& p = probs_[i].dev;
    rigw_result& r = res[i];
    const int nreal = 2 * p.nsigma_half + 1;
    if (h[i].en) {
      r.erpa = h[i].en[0];
      r.egw = h[i].en[1];
    }
    if (h[i].sc) std::memcpy(r.sigma_calc, h[i].sc, size_t(2) * p.nsig * p.nc * sizeof(double));
    if (h[i].sr) std::memcpy(r.sigma, h[i].sr, size_t(2) * p.nsig * nreal * sizeof(double));
    if (h[i].q) {
      std::vector<double> g(p.nsig), z(p.nsig), zz(p.nsig);
      double eh = -HUGE_VAL, el = HUGE_VAL;
      for (int k = 0; k < p.nsig; ++k) {
        g[k] = h[i].q[4 * k];
        z[k] = h[i].q[4 * k + 1];
        zz[k] = h[i].q[4 * k + 2];
        // output_homolumo, src/m_hamiltonian_tools.f90:564-612 (spin_fact 2, or 1 per spin channel)
        if (h[i].occ[k] / h[i].spin_fact > 1.0e-5) eh = std::max(eh, g[k]);
        if (h[i].occ[k] / h[i].spin_fact < 1.0 - 1.0e-5) el = std::min(el, g[k]);
      }
      r.ehomo = eh;
      r.elumo = el;
      if (r.energy_qp_g) RIGW_TRY(put(r.energy_qp_g, g.data(), p.nsig));
      if (r.energy_qp_z) RIGW_TRY(put(r.energy_qp_z, z.data(), p.nsig));
      if (r.zz) RIGW_TRY(put(r.zz, zz.data(), p.nsig));
    }
    r.device_ms = last_ms_;
  }
  if (!out_dev.empty()) RIGW_TRY(ctx_->sync(s));   // the staged sources go out of scope
  return Status::ok();
}

}  // namespace rigw
