// Stand-alone operations of the C ABI: explicit chi(iw) from resident factors
// and the AO -> MO transform.
#include <algorithm>
#include <cstring>

#include "engine.cuh"

namespace rigw {

namespace {
inline int round_up(int v, int a) { return (v + a - 1) / a * a; }

Status run_gemm_items(Context& c, const std::vector<GemmItem>& items, bool wide) {
  if (items.empty()) return Status::ok();
  DeviceBuffer buf;
  RIGW_TRY(buf.allocate(&c, items.size() * sizeof(GemmItem), "gemm items"));
  RIGW_CUDA_TRY(cudaMemcpyAsync(buf.data(), items.data(), items.size() * sizeof(GemmItem), cudaMemcpyHostToDevice,
                                c.stream));
  const GemmItem* d = reinterpret_cast<const GemmItem*>(buf.data());
  if (wide) launch_dgemm_128x128(d, int(items.size()), 1, c.stream);
  else launch_dgemm_64x128(d, int(items.size()), 1, c.stream);
  RIGW_CUDA_TRY(cudaGetLastError());
  RIGW_CUDA_TRY(cudaStreamSynchronize(c.stream));
  return Status::ok();
}
}  // namespace

// chi(iw) = eps^-1 - 1 = (U^-T)^T (U^-T) - 1, from the I-part of the resident solve.
Status wpol_chi(Context& c, const Wpol& w, double* chi) {
  Plan& plan = *w.plan;
  const ProbDev& p = plan.problems()[0].dev;
  const int npad = p.npad, naux = p.naux;
  DeviceBuffer out;
  RIGW_TRY(out.allocate(&c, size_t(npad) * npad * sizeof(double), "chi"));
  double* X = reinterpret_cast<double*>(out.data());
  for (int iw = 0; iw < p.nomega; ++iw) {
    const double* Y = p.rhs + size_t(iw) * npad * p.ldb;   // U^-T in columns [0, npad)
    std::vector<GemmItem> items;
    for (int i0 = 0; i0 < npad; i0 += 128)
      for (int j0 = 0; j0 < npad; j0 += 128) {
        GemmItem g{};
        g.A = Y + i0;
        g.lda = p.ldb;
        g.B = Y + j0;
        g.ldb = p.ldb;
        g.C = X + size_t(i0) * npad + j0;
        g.ldc = npad;
        g.m = std::min(128, npad - i0);
        g.n = std::min(128, npad - j0);
        g.k = npad;
        g.flags = kSubIdentity;
        g.diag = i0 - j0;
        g.alpha = 1.0;
        items.push_back(g);
      }
    RIGW_TRY(run_gemm_items(c, items, true));
    RIGW_CUDA_TRY(cudaMemcpy2D(chi + size_t(iw) * naux * naux, naux * sizeof(double), X, npad * sizeof(double),
                               naux * sizeof(double), naux, cudaMemcpyDeviceToHost));
  }
  return Status::ok();
}

// out[n][m][P] = sum_{mu,nu} C[m][mu] C[n][nu] B(mu nu, P)  (src/m_eri_ao_mo.f90:416-582).
namespace {
// One split operand of a tensor-core product: K-major bf16 hi/lo in `buf`, its
// tensor map (rows = nz * 2 * Rpad, columns = Kpad) at `map_dev`.
Status split_operand(Context& c, const SplitOp& shape, DeviceBuffer* buf, void* map_dev) {
  SplitOp op = shape;
  RIGW_TRY(buf->allocate(&c, size_t(op.nz) * 2 * op.Rpad * op.Kpad * 2, "split operand"));
  op.dst = buf->data();
  op.zs_dst = (long long)2 * op.Rpad * op.Kpad;
  launch_split_kmajor(op, c.stream);
  RIGW_CUDA_TRY(cudaGetLastError());
  alignas(64) unsigned char map[128];
  RIGW_TRY(make_split_tmap(map, op.dst, op.Kpad, (long long)op.nz * 2 * op.Rpad));
  RIGW_CUDA_TRY(cudaMemcpyAsync(map_dev, map, sizeof(map), cudaMemcpyHostToDevice, c.stream));
  return Status::ok();
}

// One Ozaki operand: `slices` int8 digit planes K-major in `buf`, row exponents
// in `exps` ([nz][Rpad]), its tensor map (rows = nz * slices * Rpad, columns =
// Kpad bytes) at `map_dev`.
Status slice_operand(Context& c, const SplitOp& shape, int slices, DeviceBuffer* buf, DeviceBuffer* exps,
                     void* map_dev) {
  SliceOp op{shape.src, shape.rs, shape.ks, shape.zs_src, shape.R, shape.K, shape.Rpad, shape.Kpad, shape.nz,
             slices, nullptr, nullptr, nullptr};
  const size_t rows = size_t(op.nz) * slices * op.Rpad;
  RIGW_TRY(buf->allocate(&c, rows * op.Kpad, "sliced operand"));
  RIGW_TRY(exps->allocate(&c, size_t(op.nz) * op.Rpad * (sizeof(int) + sizeof(unsigned long long)),
                          "row exponents"));
  op.dst = buf->data();
  op.rmax = reinterpret_cast<unsigned long long*>(exps->data());
  op.exps = reinterpret_cast<int*>(exps->data() + size_t(op.nz) * op.Rpad * sizeof(unsigned long long));
  launch_slice_kmajor(op, c.stream);
  RIGW_CUDA_TRY(cudaGetLastError());
  alignas(64) unsigned char map[128];
  RIGW_TRY(make_ozaki_tmap(map, op.dst, op.Kpad, (long long)rows));
  RIGW_CUDA_TRY(cudaMemcpyAsync(map_dev, map, sizeof(map), cudaMemcpyHostToDevice, c.stream));
  return Status::ok();
}
const int* exps_of(const DeviceBuffer& e, int nz, int Rpad) {
  return reinterpret_cast<const int*>(e.data() + size_t(nz) * Rpad * sizeof(unsigned long long));
}

Status run_tc_items(Context& c, const std::vector<TcItem>& items, bool ozaki = false) {
  if (items.empty()) return Status::ok();
  DeviceBuffer buf;
  RIGW_TRY(buf.allocate(&c, items.size() * sizeof(TcItem), "tensor-core items"));
  RIGW_CUDA_TRY(cudaMemcpyAsync(buf.data(), items.data(), items.size() * sizeof(TcItem), cudaMemcpyHostToDevice,
                                c.stream));
  if (ozaki)
    launch_syrk_ozaki(reinterpret_cast<const TcItem*>(buf.data()), int(items.size()), 1, c.stream);
  else
    launch_syrk_bf16x3(reinterpret_cast<const TcItem*>(buf.data()), int(items.size()), 1, c.stream);
  RIGW_CUDA_TRY(cudaGetLastError());
  return c.sync(c.stream);
}
}  // namespace

Status eri_3center_mo(Context& c, int nbf, int nstate, int npair, int naux, const int* index_basis,
                      const double* eri3, const double* c_matrix, int mstate_min, int mstate_max,
                      int nstate_min, int nstate_max, double* out, int precision, int flags) {
  if (nbf <= 0 || nstate <= 0 || npair <= 0 || naux <= 0 || !index_basis || !eri3 || !c_matrix || !out)
    return Status::fail(RIGW_ERR_ARG, "eri_3center_mo: invalid arguments");
  // RIGW_PROBLEM_DEVICE_POINTERS: the AO tensor is read and the MO tensor written
  // in device memory (index_basis and c_matrix, both small, stay host arrays)
  const bool on_dev = (flags & RIGW_PROBLEM_DEVICE_POINTERS) != 0;
  NvtxRange range("3-center AO to MO transform");
  if (precision != RIGW_FP64 && precision != RIGW_BF16X3 && !is_ozaki(precision))
    return Status::fail(RIGW_ERR_UNSUPPORTED, "eri_3center_mo: precision %d (FP64, BF16X3 or OZAKI(3..7))",
                        precision);
  const int ns = ozaki_slices(precision);
  const bool split = precision == RIGW_BF16X3 || ns > 0;
  if (split && !bf16x3_available()) return Status::fail(RIGW_ERR_UNSUPPORTED, "tensor maps unavailable");
  if (mstate_min < 1 || mstate_max > nstate || mstate_min > mstate_max || nstate_min < 1 ||
      nstate_max > nstate || nstate_min > nstate_max)
    return Status::fail(RIGW_ERR_ARG, "eri_3center_mo: state ranges outside [1, %d]", nstate);
  for (int q = 0; q < 2 * npair; ++q)
    if (index_basis[q] < 1 || index_basis[q] > nbf)
      return Status::fail(RIGW_ERR_ARG, "eri_3center_mo: index_basis entry %d out of [1, %d]", q, nbf);
  const int mc = mstate_max - mstate_min + 1, nc = nstate_max - nstate_min + 1;
  const int mcp = round_up(mc, 2), ncp = round_up(nc, 2);
  // C^T restricted to the two ranges: ctm[mu][m], ctn[nu][n] (m, n contiguous, even widths)
  std::vector<double> ctm(size_t(nbf) * mcp, 0.0), ctn(size_t(nbf) * ncp, 0.0);
  for (int mu = 0; mu < nbf; ++mu) {
    for (int m = 0; m < mc; ++m) ctm[size_t(mu) * mcp + m] = c_matrix[size_t(mstate_min - 1 + m) * nbf + mu];
    for (int n = 0; n < nc; ++n) ctn[size_t(mu) * ncp + n] = c_matrix[size_t(nstate_min - 1 + n) * nbf + mu];
  }
  // auxiliary chunk so that the unpacked (nu, mu, P) block stays below ~2 GB
  const size_t per_aux = size_t(nbf) * nbf * sizeof(double);
  int pc = int(std::max<size_t>(8, (size_t(2) << 30) / per_aux / 8 * 8));
  pc = std::min(pc, round_up(naux, 8));
  const int pcp = round_up(pc, 8);
  DeviceBuffer b_ctm, b_ctn, b_idx, b_eri, b_full, b_t, b_out, b_item;
  RIGW_TRY(b_ctm.allocate(&c, ctm.size() * 8, "aomo ctm"));
  RIGW_TRY(b_ctn.allocate(&c, ctn.size() * 8, "aomo ctn"));
  RIGW_TRY(b_idx.allocate(&c, size_t(2) * npair * sizeof(int), "aomo index"));
  if (!on_dev) RIGW_TRY(b_eri.allocate(&c, size_t(pc) * npair * 8, "aomo eri3 chunk"));
  RIGW_TRY(b_full.allocate(&c, size_t(nbf) * nbf * pcp * 8, "aomo unpacked"));
  RIGW_TRY(b_t.allocate(&c, size_t(ncp) * nbf * pcp * 8, "aomo half"));
  RIGW_TRY(b_out.allocate(&c, size_t(ncp) * mcp * pcp * 8, "aomo out chunk"));
  RIGW_TRY(b_item.allocate(&c, sizeof(AomoUnpackItem), "aomo item"));
  cudaStream_t s = c.stream;
  // stage times (CUDA events on the stream): AO tensor upload + unpack, the two
  // products with their operand splits, result download
  struct Events {
    cudaEvent_t e[6] = {};
    ~Events() {
      for (cudaEvent_t x : e)
        if (x) cudaEventDestroy(x);
    }
  } ev;
  for (cudaEvent_t& x : ev.e) RIGW_CUDA_TRY(cudaEventCreate(&x));
  double stage[3] = {0.0, 0.0, 0.0};
  int launches = 0;
  auto elapsed = [&](int a, int b) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev.e[a], ev.e[b]);
    return double(ms);
  };
  RIGW_CUDA_TRY(cudaEventRecord(ev.e[4], s));
  RIGW_CUDA_TRY(cudaMemcpyAsync(b_ctm.data(), ctm.data(), ctm.size() * 8, cudaMemcpyHostToDevice, s));
  RIGW_CUDA_TRY(cudaMemcpyAsync(b_ctn.data(), ctn.data(), ctn.size() * 8, cudaMemcpyHostToDevice, s));
  RIGW_CUDA_TRY(cudaMemcpyAsync(b_idx.data(), index_basis, size_t(2) * npair * sizeof(int), cudaMemcpyHostToDevice, s));
  double* dctm = reinterpret_cast<double*>(b_ctm.data());
  double* dctn = reinterpret_cast<double*>(b_ctn.data());
  double* dfull = reinterpret_cast<double*>(b_full.data());
  double* dt = reinterpret_cast<double*>(b_t.data());
  double* dout = reinterpret_cast<double*>(b_out.data());
  // split precision: C^T blocks split once; the unpacked tensor and the half
  // transform are split per auxiliary chunk (BF16x3 products, FP64 results)
  const int Kp = round_up(nbf, ns > 0 ? 128 : 64);   // 64 bf16 or 128 int8 per k-tile
  const int Rp1 = round_up(ncp, 128), Rp2 = round_up(mcp, 128), Rpw = round_up(nbf * pcp, 128);
  const int Rpp = round_up(pcp, 128);
  DeviceBuffer s_a1, s_a2, s_b1, s_b2, s_maps, s_err;
  DeviceBuffer e_a1, e_a2, e_b1, e_b2;   // Ozaki row exponents
  char* maps = nullptr;
  int* errp = nullptr;
  if (split) {
    RIGW_TRY(s_maps.allocate(&c, 4 * 128, "split tensor maps"));
    RIGW_TRY(s_err.allocate(&c, sizeof(int), "split error flag"));
    maps = s_maps.data();
    errp = reinterpret_cast<int*>(s_err.data());
    RIGW_CUDA_TRY(cudaMemsetAsync(errp, 0, sizeof(int), s));
    const SplitOp a1{dctn, 1, ncp, 0, ncp, nbf, Rp1, Kp, 1, nullptr, 0};
    const SplitOp a2{dctm, 1, mcp, 0, mcp, nbf, Rp2, Kp, 1, nullptr, 0};
    if (ns > 0) {
      RIGW_TRY(slice_operand(c, a1, ns, &s_a1, &e_a1, maps));
      RIGW_TRY(slice_operand(c, a2, ns, &s_a2, &e_a2, maps + 256));
    } else {
      RIGW_TRY(split_operand(c, a1, &s_a1, maps));
      RIGW_TRY(split_operand(c, a2, &s_a2, maps + 256));
    }
    launches += ns > 0 ? 4 : 2;
  }
  RIGW_CUDA_TRY(cudaEventRecord(ev.e[5], s));
  // rows between the first planes of two operand blocks (hi/lo, or the slices)
  const int planes = ns > 0 ? ns : 2;
  const int ktiles = ns > 0 ? Kp / 128 : Kp / 64;
  for (int p0 = 0; p0 < naux; p0 += pc) {
    const int cnt = std::min(pc, naux - p0);
    RIGW_CUDA_TRY(cudaEventRecord(ev.e[0], s));
    const double* chunk = eri3 + size_t(p0) * npair;
    if (!on_dev) {
      RIGW_CUDA_TRY(cudaMemcpyAsync(b_eri.data(), chunk, size_t(cnt) * npair * 8, cudaMemcpyHostToDevice, s));
      chunk = reinterpret_cast<const double*>(b_eri.data());
    }
    RIGW_CUDA_TRY(cudaMemsetAsync(dfull, 0, size_t(nbf) * nbf * pcp * 8, s));
    AomoUnpackItem it{chunk, reinterpret_cast<const int*>(b_idx.data()), dfull, cnt, pcp, npair, nbf, 0};
    RIGW_CUDA_TRY(cudaMemcpyAsync(b_item.data(), &it, sizeof(it), cudaMemcpyHostToDevice, s));
    dim3 grid((npair + 31) / 32, (cnt + 31) / 32);
    aomo_unpack_kernel<<<grid, 256, 0, s>>>(reinterpret_cast<const AomoUnpackItem*>(b_item.data()));
    RIGW_CUDA_TRY(cudaGetLastError());
    RIGW_CUDA_TRY(cudaEventRecord(ev.e[1], s));
    launches += 1 + (split ? (ns > 0 ? 6 : 4) : 2);
    const int wide = nbf * pcp;
    if (split) {
      // step 1: T[n][j] = sum_nu ctn^T[n][nu] B^T[j][nu],  j = (mu, P)
      const SplitOp b1{dfull, 1, wide, 0, wide, nbf, Rpw, Kp, 1, nullptr, 0};
      if (ns > 0)
        RIGW_TRY(slice_operand(c, b1, ns, &s_b1, &e_b1, maps + 128));
      else
        RIGW_TRY(split_operand(c, b1, &s_b1, maps + 128));
      std::vector<TcItem> t1;
      for (int i0 = 0; i0 < ncp; i0 += 128)
        for (int j0 = 0; j0 < wide; j0 += 128) {
          TcItem t{};
          t.tmap = maps;
          t.row_a = i0;
          t.lo_off = Rp1;
          t.tmap_b = maps + 128;
          t.row_b = j0;
          t.lo_off_b = Rpw;
          t.ktiles = ktiles;
          t.C = dt + size_t(i0) * wide + j0;
          t.ldc = wide;
          t.mrows = std::min(128, ncp - i0);
          t.ncols = std::min(128, wide - j0);
          t.err = errp;
          t.nw = 1;
          if (ns > 0) {
            t.slices = ns;
            t.ea = exps_of(e_a1, 1, Rp1) + i0;
            t.eb = exps_of(e_b1, 1, Rpw) + j0;
          }
          t1.push_back(t);
        }
      RIGW_TRY(run_tc_items(c, t1, ns > 0));
      // step 2: O[n][m][P] = sum_mu ctm^T[m][mu] T[n]^T[P][mu], every n in one launch
      const SplitOp b2{dt, 1, pcp, wide, pcp, nbf, Rpp, Kp, nc, nullptr, 0};
      if (ns > 0)
        RIGW_TRY(slice_operand(c, b2, ns, &s_b2, &e_b2, maps + 384));
      else
        RIGW_TRY(split_operand(c, b2, &s_b2, maps + 384));
      std::vector<TcItem> t2;
      for (int n = 0; n < nc; ++n)
        for (int i0 = 0; i0 < mcp; i0 += 128)
          for (int j0 = 0; j0 < pcp; j0 += 128) {
            TcItem t{};
            t.tmap = maps + 256;
            t.row_a = i0;
            t.lo_off = Rp2;
            t.tmap_b = maps + 384;
            t.row_b = n * planes * Rpp + j0;
            t.lo_off_b = Rpp;
            t.ktiles = ktiles;
            t.C = dout + (size_t(n) * mcp + i0) * pcp + j0;
            t.ldc = pcp;
            t.mrows = std::min(128, mcp - i0);
            t.ncols = std::min(128, pcp - j0);
            t.err = errp;
            t.nw = 1;
            if (ns > 0) {
              t.slices = ns;
              t.ea = exps_of(e_a2, 1, Rp2) + i0;
              t.eb = exps_of(e_b2, nc, Rpp) + size_t(n) * Rpp + j0;
            }
            t2.push_back(t);
          }
      RIGW_TRY(run_tc_items(c, t2, ns > 0));
      int herr = 0;
      RIGW_CUDA_TRY(cudaMemcpyAsync(&herr, errp, sizeof(int), cudaMemcpyDeviceToHost, s));
      RIGW_TRY(c.sync(s));
      if (herr) return Status::fail(RIGW_ERR_TIMEOUT, "eri_3center_mo: a bounded device wait expired");
    } else {
    // step 1: T[n][(mu,P)] = sum_nu ctn[nu][n] B[nu][(mu,P)]
    std::vector<GemmItem> g1;
    for (int i0 = 0; i0 < ncp; i0 += 128)
      for (int j0 = 0; j0 < wide; j0 += 128) {
        GemmItem g{};
        g.A = dctn + i0;
        g.lda = ncp;
        g.B = dfull + j0;
        g.ldb = wide;
        g.C = dt + size_t(i0) * wide + j0;
        g.ldc = wide;
        g.m = std::min(128, ncp - i0);
        g.n = std::min(128, wide - j0);
        g.k = nbf;
        g.alpha = 1.0;
        g1.push_back(g);
      }
    RIGW_TRY(run_gemm_items(c, g1, true));
    // step 2: O[n][m][P] = sum_mu ctm[mu][m] T[n][mu][P]
    std::vector<GemmItem> g2;
    for (int n = 0; n < nc; ++n)
      for (int i0 = 0; i0 < mcp; i0 += 128)
        for (int j0 = 0; j0 < pcp; j0 += 128) {
          GemmItem g{};
          g.A = dctm + i0;
          g.lda = mcp;
          g.B = dt + size_t(n) * wide + j0;
          g.ldb = pcp;
          g.C = dout + (size_t(n) * mcp + i0) * pcp + j0;
          g.ldc = pcp;
          g.m = std::min(128, mcp - i0);
          g.n = std::min(128, pcp - j0);
          g.k = nbf;
          g.alpha = 1.0;
          g2.push_back(g);
        }
    RIGW_TRY(run_gemm_items(c, g2, true));
    }
    // out[n][m][p0 : p0+cnt]
    RIGW_CUDA_TRY(cudaEventRecord(ev.e[2], s));
    for (int n = 0; n < nc; ++n)
      RIGW_CUDA_TRY(cudaMemcpy2DAsync(out + (size_t(n) * mc) * naux + p0, size_t(naux) * 8,
                                      dout + size_t(n) * mcp * pcp, size_t(pcp) * 8, size_t(cnt) * 8, mc,
                                      on_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
    RIGW_CUDA_TRY(cudaEventRecord(ev.e[3], s));
    RIGW_CUDA_TRY(cudaStreamSynchronize(s));
    stage[0] += elapsed(0, 1);
    stage[1] += elapsed(1, 2);
    stage[2] += elapsed(2, 3);
  }
  stage[1] += elapsed(4, 5);   // C uploads and the splits of the C operands
  rigw_stats st{};
  st.stage_ms[0] = stage[0];
  st.stage_ms[1] = stage[1];
  st.stage_ms[2] = stage[2];
  st.total_ms = elapsed(4, 3);
  st.kernel_launches = launches;
  st.chunks = (naux + pc - 1) / pc;
  st.waves = 1;
  c.last_stats = st;
  return Status::ok();
}

}  // namespace rigw
