// extern "C" entry points of librigw (declared in include/rigw.h).
#include <algorithm>
#include <cstring>
#include <new>

#include "engine.cuh"

using rigw::Context;
using rigw::Plan;
using rigw::Shape;
using rigw::Status;

struct rigw_ctx {
  Context impl;
};
struct rigw_wpol {
  rigw::Wpol impl;
};

namespace {

int finish(rigw_ctx* ctx, const Status& s) {
  if (ctx) ctx->impl.last_error = s.good() ? std::string() : s.msg;
  return s.code;
}

Status run_batch(Context& c, rigw::PlanMode mode, int n, const rigw_problem* probs, rigw_result* res,
                 std::unique_ptr<Plan>* owned_plan, const std::vector<const rigw::ProbDev*>& factors,
                 const double* const* sigma_in) {
  std::vector<Shape> shapes(n);
  for (int i = 0; i < n; ++i) RIGW_TRY(rigw::make_shape(probs[i], &shapes[i]));
  if (mode != rigw::kPlanPolar)
    for (int i = 0; i < n; ++i)
      if (shapes[i].nc < 1 || shapes[i].nsig < 1 || shapes[i].nstate_p < 1)
        return Status::fail(RIGW_ERR_ARG, "problem %d: Sigma needs nomega_sigma_calc, nsig, nstate_p >= 1", i);
  for (int i = 0; i < n; ++i)
    if (probs[i].precision != RIGW_FP64 && !rigw::bf16x3_available())
      return Status::fail(RIGW_ERR_UNSUPPORTED, "precision %d not available", probs[i].precision);
  std::unique_ptr<Plan> fresh(new Plan());
  Status bs = fresh->build(&c, mode, shapes, factors);
  if (bs.code == RIGW_ERR_NOMEM && !c.plan_cache.empty()) {   // cached plans hold memory: drop them, retry once
    c.plan_cache.clear();
    fresh.reset(new Plan());
    bs = fresh->build(&c, mode, shapes, factors);
  }
  RIGW_TRY(bs);
  Plan* plan = fresh.get();
  RIGW_TRY(plan->stage_inputs(probs, c.stream));
  if (sigma_in)
    for (int i = 0; i < n; ++i) RIGW_TRY(plan->stage_sigma_calc(i, sigma_in[i], c.stream));
  RIGW_TRY(plan->launch(c.stream));
  Status err = plan->check_errors(c.stream);
  rigw_stats& st = c.last_stats;
  for (int k = 0; k < 4; ++k) st.stage_ms[k] = plan->stage_ms()[k];
  st.total_ms = plan->last_ms();
  st.kernel_launches = plan->kernel_launches();
  st.graph_replayed = plan->replayed() ? 1 : 0;
  st.device_bytes_in_use = c.in_use;
  st.device_bytes_peak = c.peak;
  st.chunks = n;
  st.waves = 1;
  RIGW_TRY(err);
  if (res) RIGW_TRY(plan->fetch_results(probs, res, c.stream));
  if (owned_plan) *owned_plan = std::move(fresh);
  return Status::ok();
}

}  // namespace

extern "C" {

int rigw_version(void) { return RIGW_VERSION; }

int rigw_last_stats(const rigw_ctx* ctx, rigw_stats* stats) {
  if (!ctx || !stats) return RIGW_ERR_ARG;
  *stats = ctx->impl.last_stats;
  return RIGW_OK;
}

int rigw_create(rigw_ctx** ctx, int device, size_t hbm_budget_bytes) {
  if (!ctx) return RIGW_ERR_ARG;
  *ctx = nullptr;
  rigw_ctx* c = new (std::nothrow) rigw_ctx();
  if (!c) return RIGW_ERR_NOMEM;
  Status s = c->impl.init(device, hbm_budget_bytes);
  if (!s.good()) {
    delete c;
    return s.code;
  }
  *ctx = c;
  return RIGW_OK;
}

int rigw_destroy(rigw_ctx* ctx) {
  if (!ctx) return RIGW_ERR_ARG;
  cudaSetDevice(ctx->impl.device);
  cudaStreamSynchronize(ctx->impl.stream);
  delete ctx;
  return RIGW_OK;
}

const char* rigw_last_error(const rigw_ctx* ctx) {
  if (!ctx) return "null context";
  return ctx->impl.last_error.c_str();
}

size_t rigw_footprint_bytes(int naux, int nocc, int nvirt, int nomega, int nstate_p, int nsig, int precision) {
  Shape sh{naux, nocc, nvirt, nomega, nstate_p, nsig, 0, 0, 0, precision, 0};
  return rigw::footprint(sh, rigw::kPlanFused);
}

int rigw_imag_grid(int nomega, double* omega, double* weight) {
  if (nomega <= 0 || !omega || !weight) return RIGW_ERR_ARG;
  rigw::imag_grid(nomega, omega, weight);
  return RIGW_OK;
}

int rigw_g0w0_batch(rigw_ctx* ctx, int nprob, const rigw_problem* probs, rigw_result* results) {
  if (!ctx) return RIGW_ERR_ARG;
  if (nprob <= 0 || !probs || !results) return finish(ctx, Status::fail(RIGW_ERR_ARG, "empty batch"));
  std::lock_guard<std::mutex> lock(ctx->impl.mu);
  cudaSetDevice(ctx->impl.device);
  return finish(ctx, rigw::solve_batch(ctx->impl, nprob, probs, results));
}

int rigw_autotune(rigw_ctx* ctx, int nprob, const rigw_problem* probs, rigw_tune_report* report) {
  if (!ctx) return RIGW_ERR_ARG;
  if (nprob <= 0 || !probs || !report) return finish(ctx, Status::fail(RIGW_ERR_ARG, "empty batch"));
  std::lock_guard<std::mutex> lock(ctx->impl.mu);
  cudaSetDevice(ctx->impl.device);
  return finish(ctx, rigw::autotune(ctx->impl, nprob, probs, report));
}

int rigw_g0w0(rigw_ctx* ctx, const rigw_problem* prob, rigw_result* result) {
  return rigw_g0w0_batch(ctx, 1, prob, result);
}

int rigw_polarizability_imag(rigw_ctx* ctx, const rigw_problem* prob, double* erpa, double* egw,
                             rigw_wpol** wpol) {
  if (!ctx) return RIGW_ERR_ARG;
  if (!prob || !wpol) return finish(ctx, Status::fail(RIGW_ERR_ARG, "null argument"));
  std::lock_guard<std::mutex> lock(ctx->impl.mu);
  cudaSetDevice(ctx->impl.device);
  *wpol = nullptr;
  rigw_wpol* w = new (std::nothrow) rigw_wpol();
  if (!w) return finish(ctx, Status::fail(RIGW_ERR_NOMEM, "host allocation"));
  rigw_result r{};
  Status s = run_batch(ctx->impl, rigw::kPlanPolar, 1, prob, &r, &w->impl.plan, {}, nullptr);
  if (!s.good()) {
    delete w;
    return finish(ctx, s);
  }
  w->impl.ctx = &ctx->impl;
  rigw::make_shape(*prob, &w->impl.sh);
  if (erpa) *erpa = r.erpa;
  if (egw) *egw = r.egw;
  *wpol = w;
  return finish(ctx, Status::ok());
}

int rigw_wpol_chi(rigw_ctx* ctx, const rigw_wpol* wpol, double* chi) {
  if (!ctx) return RIGW_ERR_ARG;
  if (!wpol || !chi) return finish(ctx, Status::fail(RIGW_ERR_ARG, "null argument"));
  std::lock_guard<std::mutex> lock(ctx->impl.mu);
  cudaSetDevice(ctx->impl.device);
  return finish(ctx, rigw::wpol_chi(ctx->impl, wpol->impl, chi));
}

int rigw_gw_selfenergy_imag(rigw_ctx* ctx, const rigw_wpol* wpol, const rigw_problem* prob, rigw_result* result) {
  if (!ctx) return RIGW_ERR_ARG;
  if (!wpol || !prob || !result) return finish(ctx, Status::fail(RIGW_ERR_ARG, "null argument"));
  if (prob->naux != wpol->impl.sh.naux || prob->nomega != wpol->impl.sh.nomega)
    return finish(ctx, Status::fail(RIGW_ERR_ARG, "problem does not match the resident polarizability"));
  std::lock_guard<std::mutex> lock(ctx->impl.mu);
  cudaSetDevice(ctx->impl.device);
  std::vector<const rigw::ProbDev*> f{&wpol->impl.plan->problems()[0].dev};
  std::unique_ptr<Plan> tmp;
  return finish(ctx, run_batch(ctx->impl, rigw::kPlanSigma, 1, prob, result, &tmp, f, nullptr));
}

int rigw_wpol_release(rigw_ctx* ctx, rigw_wpol* wpol) {
  if (!wpol) return RIGW_ERR_ARG;
  if (ctx) {
    std::lock_guard<std::mutex> lock(ctx->impl.mu);
    cudaSetDevice(ctx->impl.device);
    delete wpol;
    return RIGW_OK;
  }
  delete wpol;
  return RIGW_OK;
}

int rigw_qp_solve(rigw_ctx* ctx, const rigw_problem* prob, const double* sigma_calc, rigw_result* result) {
  if (!ctx) return RIGW_ERR_ARG;
  if (!prob || !sigma_calc || !result) return finish(ctx, Status::fail(RIGW_ERR_ARG, "null argument"));
  std::lock_guard<std::mutex> lock(ctx->impl.mu);
  cudaSetDevice(ctx->impl.device);
  std::unique_ptr<Plan> tmp;
  const double* sc[1] = {sigma_calc};
  return finish(ctx, run_batch(ctx->impl, rigw::kPlanQP, 1, prob, result, &tmp, {}, sc));
}

int rigw_sox_selfenergy_imag(rigw_ctx* ctx, const rigw_sox_problem* prob, double* sigma_sox) {
  if (!ctx) return RIGW_ERR_ARG;
  if (!prob || !sigma_sox) return finish(ctx, Status::fail(RIGW_ERR_ARG, "null argument"));
  std::lock_guard<std::mutex> lock(ctx->impl.mu);
  cudaSetDevice(ctx->impl.device);
  return finish(ctx, rigw::sox_selfenergy_imag(ctx->impl, *prob, sigma_sox));
}

int rigw_sosex_selfenergy_imag(rigw_ctx* ctx, const rigw_wpol* wpol, const rigw_sosex_problem* prob,
                               double* sigma_sosex) {
  if (!ctx) return RIGW_ERR_ARG;
  if (!wpol || !prob || !sigma_sosex) return finish(ctx, Status::fail(RIGW_ERR_ARG, "null argument"));
  std::lock_guard<std::mutex> lock(ctx->impl.mu);
  cudaSetDevice(ctx->impl.device);
  return finish(ctx, rigw::sosex_selfenergy_imag(ctx->impl, wpol->impl, *prob, sigma_sosex));
}

int rigw_g3w2_selfenergy_imag(rigw_ctx* ctx, const rigw_wpol* wpol, const rigw_g3w2_problem* prob,
                              double* sigma_g3w2) {
  if (!ctx) return RIGW_ERR_ARG;
  if (!wpol || !prob || !sigma_g3w2) return finish(ctx, Status::fail(RIGW_ERR_ARG, "null argument"));
  std::lock_guard<std::mutex> lock(ctx->impl.mu);
  cudaSetDevice(ctx->impl.device);
  return finish(ctx, rigw::g3w2_selfenergy_imag(ctx->impl, wpol->impl, *prob, sigma_g3w2));
}

int rigw_eri_2center(rigw_ctx* ctx, const rigw_ri_problem* prob, double* v2) {
  if (!ctx) return RIGW_ERR_ARG;
  if (!prob || !v2) return finish(ctx, Status::fail(RIGW_ERR_ARG, "null argument"));
  std::lock_guard<std::mutex> lock(ctx->impl.mu);
  cudaSetDevice(ctx->impl.device);
  return finish(ctx, rigw::ri_integrals(ctx->impl, *prob, 2, v2, nullptr));
}

int rigw_eri_3center_raw(rigw_ctx* ctx, const rigw_ri_problem* prob, double* eri3) {
  if (!ctx) return RIGW_ERR_ARG;
  if (!prob || !eri3) return finish(ctx, Status::fail(RIGW_ERR_ARG, "null argument"));
  std::lock_guard<std::mutex> lock(ctx->impl.mu);
  cudaSetDevice(ctx->impl.device);
  return finish(ctx, rigw::ri_integrals(ctx->impl, *prob, 3, eri3, nullptr));
}

int rigw_eri_3center(rigw_ctx* ctx, const rigw_ri_problem* prob, double* eri3, int* nauxil_kept) {
  if (!ctx) return RIGW_ERR_ARG;
  if (!prob || !eri3 || !nauxil_kept) return finish(ctx, Status::fail(RIGW_ERR_ARG, "null argument"));
  std::lock_guard<std::mutex> lock(ctx->impl.mu);
  cudaSetDevice(ctx->impl.device);
  return finish(ctx, rigw::ri_integrals(ctx->impl, *prob, 0, eri3, nauxil_kept));
}

int rigw_gw_density_matrix_imag(rigw_ctx* ctx, const rigw_wpol* wpol, const rigw_dm_problem* prob,
                                double* p_matrix) {
  if (!ctx) return RIGW_ERR_ARG;
  if (!wpol || !prob || !p_matrix) return finish(ctx, Status::fail(RIGW_ERR_ARG, "null argument"));
  std::lock_guard<std::mutex> lock(ctx->impl.mu);
  cudaSetDevice(ctx->impl.device);
  return finish(ctx, rigw::gw_density_matrix_imag(ctx->impl, wpol->impl, *prob, p_matrix));
}

int rigw_gw_selfenergy_contour(rigw_ctx* ctx, const rigw_contour_problem* prob, rigw_contour_result* result) {
  if (!ctx) return RIGW_ERR_ARG;
  if (!prob || !result) return finish(ctx, Status::fail(RIGW_ERR_ARG, "null argument"));
  std::lock_guard<std::mutex> lock(ctx->impl.mu);
  cudaSetDevice(ctx->impl.device);
  return finish(ctx, rigw::gw_selfenergy_contour(ctx->impl, *prob, *result));
}

int rigw_eri_3center_mo(rigw_ctx* ctx, int nbf, int nstate, int npair, int naux, const int* index_basis,
                        const double* eri3, const double* c_matrix, int mstate_min, int mstate_max,
                        int nstate_min, int nstate_max, double* out) {
  if (!ctx) return RIGW_ERR_ARG;
  std::lock_guard<std::mutex> lock(ctx->impl.mu);
  cudaSetDevice(ctx->impl.device);
  return finish(ctx, rigw::eri_3center_mo(ctx->impl, nbf, nstate, npair, naux, index_basis, eri3, c_matrix,
                                          mstate_min, mstate_max, nstate_min, nstate_max, out, RIGW_FP64));
}

int rigw_eri_3center_mo_precision(rigw_ctx* ctx, int nbf, int nstate, int npair, int naux, const int* index_basis,
                                  const double* eri3, const double* c_matrix, int mstate_min, int mstate_max,
                                  int nstate_min, int nstate_max, double* out, int precision) {
  if (!ctx) return RIGW_ERR_ARG;
  std::lock_guard<std::mutex> lock(ctx->impl.mu);
  cudaSetDevice(ctx->impl.device);
  return finish(ctx, rigw::eri_3center_mo(ctx->impl, nbf, nstate, npair, naux, index_basis, eri3, c_matrix,
                                          mstate_min, mstate_max, nstate_min, nstate_max, out, precision));
}

int rigw_eri_3center_mo_ex(rigw_ctx* ctx, int nbf, int nstate, int npair, int naux, const int* index_basis,
                           const double* eri3, const double* c_matrix, int mstate_min, int mstate_max,
                           int nstate_min, int nstate_max, double* out, int precision, int flags) {
  if (!ctx) return RIGW_ERR_ARG;
  std::lock_guard<std::mutex> lock(ctx->impl.mu);
  cudaSetDevice(ctx->impl.device);
  return finish(ctx, rigw::eri_3center_mo(ctx->impl, nbf, nstate, npair, naux, index_basis, eri3, c_matrix,
                                          mstate_min, mstate_max, nstate_min, nstate_max, out, precision, flags));
}

}  // extern "C"
