// Memory-bounded execution of a batch of G0W0 problems.
//
// A batch whose fused plan fits the device runs as one plan (four CUDA graphs).
// Otherwise every problem is split into frequency chunks that fit, the chunks of
// all problems are packed into waves under the memory budget, each wave runs as
// one partial plan (chi0, factorization, solves, partial Sigma_c and energies),
// the partial sums are accumulated in chunk order (deterministic), and one QP
// plan finishes all problems.  The frequency sum is the only coupling between
// chunks: Sigma_c(z) and both energies are sums over omega
// (src/m_gw_selfenergy_grid.f90:118-191, 290-321), which is also what makes the
// poorman frequency split of the reference (:626,658) exact.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <vector>

#include "engine.cuh"

namespace rigw {

size_t available_bytes(Context& c) {
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
    cudaGetLastError();
    free_b = 0;
  }
  // memory held by the stream-ordered pool but not in use is available as well
  cudaMemPool_t pool;
  uint64_t reserved = 0, used = 0;
  if (cudaDeviceGetDefaultMemPool(&pool, c.device) == cudaSuccess) {
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
  }
  cudaGetLastError();
  free_b += size_t(reserved > used ? reserved - used : 0);
  // the context's spare block is allocated but free for its next plan
  size_t avail = size_t(double(free_b) * 0.9) + c.spare_bytes;
  const size_t held = c.in_use - c.spare_bytes;
  if (c.budget) avail = std::min(avail, c.budget > held ? c.budget - held : 0);
  return avail;
}

namespace {

Status get_plan(Context& c, PlanMode mode, const std::vector<Shape>& shapes, Plan** out) {
  auto key = std::make_pair(int(mode), shapes);
  auto it = c.plan_cache.find(key);
  if (it != c.plan_cache.end()) {
    *out = it->second.get();
    return Status::ok();
  }
  if (c.plan_cache.size() >= 8) c.plan_cache.clear();
  const auto t0 = std::chrono::steady_clock::now();
  std::unique_ptr<Plan> p(new Plan());
  Status s = p->build(&c, mode, shapes, {});
  if (s.code == RIGW_ERR_NOMEM && !c.plan_cache.empty()) {   // cached plans hold memory: drop them, retry once
    c.plan_cache.clear();
    p.reset(new Plan());
    s = p->build(&c, mode, shapes, {});
  }
  RIGW_TRY(s);
  c.host_build_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  *out = p.get();
  c.plan_cache.emplace(key, std::move(p));
  return Status::ok();
}

void add_stats(Context& c, const Plan& p, bool first) {
  rigw_stats& st = c.last_stats;
  if (first) {
    std::memset(&st, 0, sizeof(st));
  }
  for (int k = 0; k < 4; ++k) st.stage_ms[k] += p.stage_ms()[k];
  st.total_ms += p.last_ms();
  st.kernel_launches += p.kernel_launches();
  st.graph_replayed = p.replayed() ? 1 : 0;
  st.device_bytes_in_use = c.in_use;
  st.device_bytes_peak = c.peak;
}

Status run_plan(Context& c, Plan* plan, const rigw_problem* probs, rigw_result* res,
                const std::vector<const double*>* sigma_in, bool first) {
  RIGW_TRY(plan->stage_inputs(probs, c.stream));
  if (sigma_in)
    for (size_t i = 0; i < sigma_in->size(); ++i) RIGW_TRY(plan->stage_sigma_calc(int(i), (*sigma_in)[i], c.stream));
  RIGW_TRY(plan->launch(c.stream));
  Status err = plan->check_errors(c.stream);
  add_stats(c, *plan, first);
  RIGW_TRY(err);
  return plan->fetch_results(probs, res, c.stream);
}

}  // namespace

Status validate_batch(int n, const rigw_problem* probs, std::vector<Shape>* shapes) {
  shapes->resize(n);
  for (int i = 0; i < n; ++i) {
    RIGW_TRY(make_shape(probs[i], &(*shapes)[i]));
    const Shape& s = (*shapes)[i];
    if (s.nc < 1 || s.nsig < 1 || s.nstate_p < 1)
      return Status::fail(RIGW_ERR_ARG, "problem %d: Sigma needs nomega_sigma_calc, nsig, nstate_p >= 1", i);
    if (probs[i].precision != RIGW_FP64 && !bf16x3_available())
      return Status::fail(RIGW_ERR_UNSUPPORTED, "precision %d not available", probs[i].precision);
  }
  return Status::ok();
}

Status solve_batch(Context& c, int n, const rigw_problem* probs, rigw_result* res) {
  std::vector<Shape> shapes;
  RIGW_TRY(validate_batch(n, probs, &shapes));
  // a batch of these shapes ran before: its plan (and graphs) are ready
  auto hit = c.plan_cache.find(std::make_pair(int(kPlanFused), shapes));
  if (hit != c.plan_cache.end()) {
    RIGW_TRY(run_plan(c, hit->second.get(), probs, res, nullptr, true));
    c.last_stats.chunks = n;
    c.last_stats.waves = 1;
    return Status::ok();
  }
  size_t avail = available_bytes(c);
  // plans cached for other shapes count as free memory for this decision
  size_t cached = 0;
  for (auto& kv : c.plan_cache) cached += kv.second->bytes();
  const size_t usable = avail + cached;

  // ---- fits: one fused plan
  const Tuning tune = c.tuning_for(kPlanFused, shapes);
  if (Plan::measure(shapes, kPlanFused, &tune) <= usable) {
    Plan* plan = nullptr;
    RIGW_TRY(get_plan(c, kPlanFused, shapes, &plan));
    RIGW_TRY(run_plan(c, plan, probs, res, nullptr, true));
    c.last_stats.chunks = n;
    c.last_stats.waves = 1;
    return Status::ok();
  }

  // ---- frequency chunks and waves
  c.plan_cache.clear();
  avail = available_bytes(c);
  struct Unit {
    int prob, w0, nw;
  };
  std::vector<Unit> units;
  std::vector<std::vector<double>> om(n), wt(n);
  for (int i = 0; i < n; ++i) {
    const Shape& sh = shapes[i];
    int wc = sh.nomega;
    for (; wc >= 1; --wc) {
      Shape s2 = sh;
      s2.nomega = wc;
      if (Plan::measure({s2}, kPlanPartial) <= avail) break;
    }
    if (wc < 1)
      return Status::fail(RIGW_ERR_NOMEM, "problem %d (naux=%d, nocc=%d, nvirt=%d) does not fit in %zu bytes even "
                          "one frequency at a time", i, sh.naux, sh.nocc, sh.nvirt, avail);
    om[i].resize(sh.nomega);
    wt[i].resize(sh.nomega);
    if (probs[i].omega && probs[i].weight) {
      RIGW_CUDA_TRY(cudaMemcpyAsync(om[i].data(), probs[i].omega, sh.nomega * 8, cudaMemcpyDefault, c.stream));
      RIGW_CUDA_TRY(cudaMemcpyAsync(wt[i].data(), probs[i].weight, sh.nomega * 8, cudaMemcpyDefault, c.stream));
      RIGW_TRY(c.sync(c.stream));
    } else {
      imag_grid(sh.nomega, om[i].data(), wt[i].data());
    }
    for (int w0 = 0; w0 < sh.nomega; w0 += wc) units.push_back({i, w0, std::min(wc, sh.nomega - w0)});
  }
  std::vector<std::vector<double>> acc_sig(n);
  std::vector<double> acc_en(2 * size_t(n), 0.0);
  for (int i = 0; i < n; ++i) acc_sig[i].assign(size_t(2) * shapes[i].nsig * shapes[i].nc, 0.0);

  bool first = true;
  int waves = 0;
  for (size_t u0 = 0; u0 < units.size();) {
    // greedy wave: units in order while the sum of their footprints fits
    size_t u1 = u0, used = 0;
    std::vector<Shape> wsh;
    while (u1 < units.size()) {
      Shape s2 = shapes[units[u1].prob];
      s2.nomega = units[u1].nw;
      const size_t b = Plan::measure({s2}, kPlanPartial);
      if (u1 > u0 && used + b > avail) break;
      used += b;
      wsh.push_back(s2);
      ++u1;
    }
    const int nu = int(u1 - u0);
    std::vector<rigw_problem> up(nu);
    std::vector<rigw_result> ur(nu);
    std::vector<std::vector<double>> usig(nu);
    for (int k = 0; k < nu; ++k) {
      const Unit& u = units[u0 + k];
      up[k] = probs[u.prob];
      up[k].nomega = u.nw;
      up[k].omega = om[u.prob].data() + u.w0;
      up[k].weight = wt[u.prob].data() + u.w0;
      usig[k].assign(size_t(2) * shapes[u.prob].nsig * shapes[u.prob].nc, 0.0);
      std::memset(&ur[k], 0, sizeof(rigw_result));
      ur[k].sigma_calc = usig[k].data();
    }
    Plan* plan = nullptr;
    RIGW_TRY(get_plan(c, kPlanPartial, wsh, &plan));
    RIGW_TRY(run_plan(c, plan, up.data(), ur.data(), nullptr, first));
    first = false;
    ++waves;
    for (int k = 0; k < nu; ++k) {
      const int i = units[u0 + k].prob;
      for (size_t q = 0; q < acc_sig[i].size(); ++q) acc_sig[i][q] += usig[k][q];
      acc_en[2 * i] += ur[k].erpa;
      acc_en[2 * i + 1] += ur[k].egw;
    }
    u0 = u1;
  }
  // ---- QP for every problem from the summed Sigma_c
  Plan* qplan = nullptr;
  RIGW_TRY(get_plan(c, kPlanQP, shapes, &qplan));
  std::vector<const double*> sin(n);
  for (int i = 0; i < n; ++i) sin[i] = acc_sig[i].data();
  RIGW_TRY(run_plan(c, qplan, probs, res, &sin, false));
  for (int i = 0; i < n; ++i) {
    res[i].erpa = acc_en[2 * i];
    res[i].egw = acc_en[2 * i + 1];
    if (res[i].sigma_calc)
      RIGW_CUDA_TRY(cudaMemcpyAsync(res[i].sigma_calc, acc_sig[i].data(), acc_sig[i].size() * 8, cudaMemcpyDefault,
                                    c.stream));
      RIGW_TRY(c.sync(c.stream));
    res[i].device_ms = c.last_stats.total_ms;
  }
  c.last_stats.chunks = int(units.size());
  c.last_stats.waves = waves;
  return Status::ok();
}

// ---------------------------------------------------------------------------
// Autotuner: times launch-shape candidates on the caller's batch (a plan that
// fits the device) and keeps the fastest per (fused mode, precision class) for
// every later plan of that class.  Coordinate descent: the chi0-stage shape
// (FP64 item height) by the chi0 stage time, then the
// factorization-stage shapes (trailing-update item height, chains) by the
// factorization stage time; every candidate is launched twice and timed on the
// second launch (CUDA events between the stage graphs).
Status autotune(Context& c, int n, const rigw_problem* probs, rigw_tune_report* rep) {
  std::vector<Shape> shapes;
  RIGW_TRY(validate_batch(n, probs, &shapes));
  std::memset(rep, 0, sizeof(*rep));
  c.plan_cache.clear();
  const size_t avail = available_bytes(c);
  const int cls = precision_class(shapes);
  bool any_fp64 = false;
  for (const Shape& sh : shapes) any_fp64 = any_fp64 || sh.precision == RIGW_FP64;
  Tuning best = c.tuning_for(kPlanFused, shapes);
  if (Plan::measure(shapes, kPlanFused, &best) > avail)
    return Status::fail(RIGW_ERR_NOMEM, "autotune: the batch does not fit the device in one plan");

  auto run = [&](const Tuning& t, float* stage) -> Status {
    if (Plan::measure(shapes, kPlanFused, &t) > avail) return Status::fail(RIGW_ERR_NOMEM, "candidate too large");
    Plan p;
    RIGW_TRY(p.build(&c, kPlanFused, shapes, {}, nullptr, &t));
    RIGW_TRY(p.stage_inputs(probs, c.stream));
    // the first launch runs directly, the later ones replay the captured graphs;
    // each stage keeps its fastest of three replays
    for (int k = 0; k < 4; ++k) stage[k] = 3.4e38f;
    for (int rep2 = 0; rep2 < 4; ++rep2) {
      RIGW_TRY(p.launch(c.stream));
      RIGW_TRY(p.check_errors(c.stream));
      if (rep2 > 0)
        for (int k = 0; k < 4; ++k) stage[k] = std::min(stage[k], float(p.stage_ms()[k]));
    }
    return Status::ok();
  };
  auto record = [&](const Tuning& t, const float* st) {
    if (rep->ncandidates >= RIGW_TUNE_MAX_CANDIDATES) return;
    const int k = rep->ncandidates++;
    rep->candidate[k][0] = t.chi0_rows;
    rep->candidate[k][1] = t.update_rows;
    rep->candidate[k][2] = t.split_group;
    rep->candidate[k][3] = t.chains;
    rep->candidate[k][4] = t.panel_group > 0 ? t.panel_group : (n >= 4 ? 16 : 2);
    rep->candidate_ms[k][0] = st[1];
    rep->candidate_ms[k][1] = st[2];
    rep->candidate_ms[k][2] = st[0] + st[1] + st[2] + st[3];
  };
  float bst[4];
  RIGW_TRY(run(best, bst));
  record(best, bst);
  rep->default_ms = bst[0] + bst[1] + bst[2] + bst[3];
  // try one field at a time; keep a candidate when its stage is faster
  auto try_field = [&](int Tuning::*field, std::initializer_list<int> values, int stage) -> Status {
    const int cur = best.*field;
    for (int v : values) {
      if (v == cur) continue;
      Tuning t = best;
      t.*field = v;
      float st[4];
      Status s = run(t, st);
      if (s.code == RIGW_ERR_NOMEM) continue;
      RIGW_TRY(s);
      record(t, st);
      if (st[stage] < bst[stage]) {
        best = t;
        std::memcpy(bst, st, sizeof(bst));
      }
    }
    return Status::ok();
  };
  if (any_fp64) RIGW_TRY(try_field(&Tuning::chi0_rows, {64, 128}, 1));
  // split precision: frequencies per hi/lo buffer, including a group whose
  // buffers stay resident in L2 between the split and the tensor-core launch
  bool any_split = false;
  size_t per_w = 0;
  for (const Shape& sh : shapes)
    if (sh.precision != RIGW_FP64) {
      any_split = true;
      per_w += split_bytes_per_frequency(sh);
    }
  if (any_split) {
    const int g_l2 = int(std::max<size_t>(1, kSplitL2Bytes / std::max<size_t>(per_w, 1)));
    RIGW_TRY(try_field(&Tuning::split_group, {g_l2, 8}, 1));
  }
  RIGW_TRY(try_field(&Tuning::update_rows, {64, 128}, 2));
  RIGW_TRY(try_field(&Tuning::chains, {1, 2, 4, 8}, 2));
  RIGW_TRY(try_field(&Tuning::panel_group, {2, 8, 16}, 2));
  c.tuned[{int(kPlanFused), cls}] = best;
  c.plan_cache.clear();
  rep->chi0_rows = best.chi0_rows;
  rep->update_rows = best.update_rows;
  rep->split_group = best.split_group;
  rep->chains = best.chains;
  rep->panel_group = best.panel_group > 0 ? best.panel_group : (n >= 4 ? 16 : 2);
  rep->precision_class = cls;
  rep->tuned_ms = bst[0] + bst[1] + bst[2] + bst[3];
  return Status::ok();
}

}  // namespace rigw
