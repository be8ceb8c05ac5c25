// lmb_batch_ops.cu -- batched multi-RHS / multi-lattice Wilson D^+D CG
// (lmb_cg_ddagd_batched): persistent work-list kernels, a CUDA graph per
// iteration and the (RHS block, tile) autotuner.
#include "lmb_batch.cuh"
#include "lmb_internal.cuh"

using namespace lmb;

namespace lmb {

// ---------------------------------------------------------------------------
// batched CG driver
// ---------------------------------------------------------------------------
struct BatchRun {
  std::vector<BatchGroup> groups;
  BatchGroup *d_groups = nullptr;
  int ntasks = 0;
  int nb = 1, nt = 128, family = 0;
  bool phase_t = false;  // every lattice's phases differ from 1 in t at most (PH_T stencils)
};

// resident blocks of a persistent launch of `kern` (SMs x blocks per SM), per
// device; a kernel with dynamic shared memory is first opted in to its size
// (static + dynamic above 48 KiB needs it)
template <class K>
int batch_resident(K kern, int nt, size_t smem) {
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, int> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair((const void *)kern, dev);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  if (smem > 0) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0, sms = 148;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, nt, smem) != cudaSuccess || per_sm < 1) per_sm = 1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cache[key] = per_sm * sms;
  return per_sm * sms;
}

template <int FAM, int NT, int NB, int PS>
int batch_stage_nt(lmb_ctx *ctx, const BatchRun &br, CGState *states, int stage, cudaStream_t st) {
  const int ng = (int)br.groups.size();
  int grid;
  if constexpr (FAM == 0) {
    grid = std::min(br.ntasks, batch_resident(batch_wilson_kernel<NT, NB, ROLE_K2, PS>, NT, 0));
    if (stage == 0) batch_wilson_kernel<NT, NB, ROLE_K1, PS><<<grid, NT, 0, st>>>(br.d_groups, ng, br.ntasks, states);
    if (stage == 1) batch_wilson_kernel<NT, NB, ROLE_K2, PS><<<grid, NT, 0, st>>>(br.d_groups, ng, br.ntasks, states);
  } else {
    constexpr size_t sm = batch_smem_bytes<NT>();
    const int g1 = batch_resident(batch_wilson_smem_kernel<NT, NB, ROLE_K1, PS>, NT, sm);
    grid = std::min(br.ntasks, batch_resident(batch_wilson_smem_kernel<NT, NB, ROLE_K2, PS>, NT, sm));
    if (stage == 0)
      batch_wilson_smem_kernel<NT, NB, ROLE_K1, PS><<<std::min(br.ntasks, g1), NT, sm, st>>>(br.d_groups, ng,
                                                                                            br.ntasks, states);
    if (stage == 1)
      batch_wilson_smem_kernel<NT, NB, ROLE_K2, PS><<<grid, NT, sm, st>>>(br.d_groups, ng, br.ntasks, states);
  }
  if (stage == 2) batch_p_update_kernel<NT, NB, PS><<<grid, NT, 0, st>>>(br.d_groups, ng, br.ntasks, states);
  if (stage == 3) batch_wilson64_kernel<NT, ROLE_D64, PS><<<grid, NT, 0, st>>>(br.d_groups, ng, br.ntasks, states);
  if (stage == 4) batch_wilson64_kernel<NT, ROLE_TRUE, PS><<<grid, NT, 0, st>>>(br.d_groups, ng, br.ntasks, states);
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}

// the x-adjacent pair family: K1, K2 and K3 (the FP64 passes run on the
// auxiliary register-family run)
template <int PHM>
int batch_pair_stage(lmb_ctx *ctx, const BatchRun &br, CGState *states, int stage, cudaStream_t st) {
  const int ng = (int)br.groups.size();
  const int grid = std::min(br.ntasks, batch_resident(batch_half_pair_kernel<ROLE_K2, PHM>, kDslashThreads, 0));
  if (stage == 0)
    batch_half_pair_kernel<ROLE_K1, PHM><<<grid, kDslashThreads, 0, st>>>(br.d_groups, ng, br.ntasks, states);
  else if (stage == 1)
    batch_half_pair_kernel<ROLE_K2, PHM><<<grid, kDslashThreads, 0, st>>>(br.d_groups, ng, br.ntasks, states);
  else if (stage == 2)
    batch_half_pair_p_kernel<<<grid, kDslashThreads, 0, st>>>(br.d_groups, ng, br.ntasks, states);
  else
    return fail(ctx, LMB_ERR_STATE, "the pair family runs its FP64 passes on the auxiliary run");
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}

// dispatch one stage (0 K1, 1 K2, 2 K3, 3 FP64 D, 4 FP64 true residual) for
// the run's family, tile NT and group size NB
template <int PS>
int batch_stage(lmb_ctx *ctx, const BatchRun &br, CGState *states, int stage, cudaStream_t st) {
  if constexpr (PS == PREC_HALF) {
    if (br.family == 2)
      return br.phase_t ? batch_pair_stage<PH_T>(ctx, br, states, stage, st)
                        : batch_pair_stage<PH_ANY>(ctx, br, states, stage, st);
  }
#define LMB_BATCH_CASE(FAM_, NT_, NB_) \
  if (br.family == FAM_ && br.nt == NT_ && br.nb == NB_) return batch_stage_nt<FAM_, NT_, NB_, PS>(ctx, br, states, stage, st);
  LMB_BATCH_CASE(0, 64, 1) LMB_BATCH_CASE(0, 64, 2) LMB_BATCH_CASE(0, 64, 4)
  LMB_BATCH_CASE(0, 128, 1) LMB_BATCH_CASE(0, 128, 2) LMB_BATCH_CASE(0, 128, 4)
  LMB_BATCH_CASE(0, 256, 1) LMB_BATCH_CASE(0, 256, 2) LMB_BATCH_CASE(0, 256, 4)
  LMB_BATCH_CASE(1, 64, 4) LMB_BATCH_CASE(1, 64, 8) LMB_BATCH_CASE(1, 64, 16)
  LMB_BATCH_CASE(1, 128, 4) LMB_BATCH_CASE(1, 128, 8) LMB_BATCH_CASE(1, 128, 16)
#undef LMB_BATCH_CASE
  return fail(ctx, LMB_ERR_UNSUPPORTED, "batched family %d, tile %d x rhs block %d not built", br.family, br.nt,
              br.nb);
}

template <int PS>
struct BatchMember {
  int lattice, rhs;
  Geom g;
  Padded pd;
  Field<PREC_DOUBLE, 12> b64, x64, r64, t64;
  Field<PS, 12> p, t, r;
  Field<PREC_SINGLE, 12> xl;
};

template <int PS>
int build_run(lmb_ctx *ctx, BatchRun &br, int family, int nb, int nt, const std::vector<BatchMember<PS>> &m,
              const std::vector<int> &member_lattice_start, const std::vector<int> &nrhs,
              const std::vector<lmb_batch_links *> &links, const std::vector<double> &kappa,
              const std::string &tag) {
  br.family = family;
  br.nb = nb;
  br.nt = nt;
  br.groups.clear();
  br.phase_t = true;
  int task = 0;
  size_t partial_words = 0;
  for (size_t l = 0; l < nrhs.size(); l++) {
    for (int r0 = 0; r0 < nrhs[l]; r0 += nb) {
      BatchGroup G{};
      const BatchMember<PS> &m0 = m[member_lattice_start[l] + r0];
      G.g = m0.g;
      G.U = links[l]->f12;
      G.Uh = links[l]->h12;
      G.U64 = links[l]->d12;
      G.nact = std::min(nb, nrhs[l] - r0);
      G.first_task = task;
      if (family == 2) {  // tasks (group of kPairTilesPerTask tiles of kDslashThreads pairs, member)
        const int64_t tiles = (G.g.V / 2 + kDslashThreads - 1) / kDslashThreads;
        G.ntasks = (int)((tiles + kPairTilesPerTask - 1) / kPairTilesPerTask) * G.nact;
      } else {
        G.ntasks = (int)((G.g.V + nt - 1) / nt);
      }
      if (phase_mode_of(G.g.phase_mask) != PH_T) br.phase_t = false;
      G.state0 = member_lattice_start[l] + r0;
      G.kappa = kappa[l];
      for (int r = 0; r < G.nact; r++) {
        const BatchMember<PS> &mm = m[G.state0 + r];
        G.p[r] = mm.p.data;
        G.t[r] = mm.t.data;
        G.r[r] = mm.r.data;
        G.pn[r] = mm.p.norm;
        G.tn[r] = mm.t.norm;
        G.rn[r] = mm.r.norm;
        G.xl[r] = mm.xl.data;
        G.b64[r] = mm.b64.data;
        G.x64[r] = mm.x64.data;
        G.r64[r] = mm.r64.data;
        G.t64[r] = mm.t64.data;
      }
      task += G.ntasks;
      partial_words += (size_t)G.ntasks * kMaxNB;  // the FP64 passes reduce kMaxNB slots
      br.groups.push_back(G);
    }
  }
  br.ntasks = task;
  double *partials = (double *)workspace(ctx, "batch_partials_" + tag, sizeof(double) * partial_words);
  unsigned *counters = (unsigned *)workspace(ctx, "batch_counters_" + tag, sizeof(unsigned) * br.groups.size());
  br.d_groups = (BatchGroup *)workspace(ctx, "batch_groups_" + tag, sizeof(BatchGroup) * br.groups.size());
  if (!partials || !counters || !br.d_groups) return fail(ctx, LMB_ERR_CUDA, "out of device memory (batch tables)");
  LMB_CUDA(ctx, cudaMemset(counters, 0, sizeof(unsigned) * br.groups.size()));
  size_t off = 0;
  for (size_t i = 0; i < br.groups.size(); i++) {
    br.groups[i].partials = partials + off;
    br.groups[i].counter = counters + i;
    off += (size_t)br.groups[i].ntasks * kMaxNB;
  }
  return LMB_OK;
}

int upload_groups(lmb_ctx *ctx, BatchRun &br, cudaStream_t st) {
  LMB_CUDA(ctx, cudaMemcpyAsync(br.d_groups, br.groups.data(), sizeof(BatchGroup) * br.groups.size(),
                                cudaMemcpyHostToDevice, st));
  return LMB_OK;
}

int batch_links_for(lmb_ctx *ctx, const lmb_batch_lattice &lat, const Geom &g, const Padded &pd,
                    lmb_batch_links **out, cudaStream_t st) {
  for (auto &bl : ctx->batch_links) {
    bool same = bl.V == g.V;
    for (int mu = 0; mu < 4 && same; mu++) same = bl.ptr[mu] == lat.U[mu] && bl.epoch[mu] == lat.epoch[mu];
    if (same) {
      *out = &bl;
      return LMB_OK;
    }
  }
  ctx->batch_links.emplace_back();
  lmb_batch_links &bl = ctx->batch_links.back();
  const int64_t V = g.V;
  double2 *d = (double2 *)workspace(ctx, "batch_pack", sizeof(double2) * 36 * V);
  if (!d) return fail(ctx, LMB_ERR_CUDA, "out of device memory (batched links)");
  pack_links_kernel<double2><<<grid_for(V, 256), 256, 0, st>>>(
      d, (const double2 *)lat.U[0], (const double2 *)lat.U[1], (const double2 *)lat.U[2],
      (const double2 *)lat.U[3], g, pd);
  LMB_CHECK_LAUNCH(ctx);
  unsigned *bits = (unsigned *)workspace(ctx, "su3dev", sizeof(unsigned));
  if (!bits) return fail(ctx, LMB_ERR_CUDA, "out of device memory (su3 check)");
  LMB_CUDA(ctx, cudaMemsetAsync(bits, 0, sizeof(unsigned), st));
  su3_deviation_kernel<<<1184, 256, 0, st>>>(d, V, bits);
  unsigned hb = 0;
  LMB_CUDA(ctx, cudaMemcpyAsync(&hb, bits, sizeof hb, cudaMemcpyDeviceToHost, st));
  LMB_CUDA(ctx, cudaStreamSynchronize(st));
  float dev;
  std::memcpy(&dev, &hb, sizeof dev);
  if (!(dev <= 1e-12f)) {
    ctx->batch_links.pop_back();
    return fail(ctx, LMB_ERR_UNSUPPORTED, "batched CG needs SU(3) links (deviation %.3g)", (double)dev);
  }
  LMB_CUDA(ctx, cudaMalloc(&bl.d12, sizeof(double2) * 24 * V));
  LMB_CUDA(ctx, cudaMalloc(&bl.f12, sizeof(float4) * 12 * V));
  LMB_CUDA(ctx, cudaMalloc(&bl.h12, sizeof(int4) * 6 * V));
  links_to_recon12_kernel<<<grid_for(V, 256), 256, 0, st>>>(bl.d12, bl.f12, bl.h12, d, V);
  LMB_CHECK_LAUNCH(ctx);
  for (int mu = 0; mu < 4; mu++) {
    bl.ptr[mu] = lat.U[mu];
    bl.epoch[mu] = lat.epoch[mu];
  }
  bl.V = V;
  *out = &bl;
  return LMB_OK;
}

template <int PS>
int cg_batched(lmb_ctx *ctx, const lmb_cg_params *prm, int nlat, const lmb_batch_lattice *lats,
               lmb_cg_result *res, lmb_batch_tuning *tuning, cudaStream_t st) {
  // geometry and links per lattice
  std::vector<Geom> geoms(nlat);
  std::vector<Padded> pads(nlat);
  std::vector<lmb_batch_links *> links(nlat);
  std::vector<int> nrhs(nlat), start(nlat);
  std::vector<double> kappa(nlat);
  std::string sig = std::string(PS == PREC_HALF ? "h;" : "s;") + std::to_string(ctx->batch_family) + ";";
  int total = 0;
  for (int l = 0; l < nlat; l++) {
    const lmb_batch_lattice &lat = lats[l];
    if (lat.nrhs <= 0 || !lat.x || !lat.b) return fail(ctx, LMB_ERR_ARG, "lattice %d has no right-hand sides", l);
    Geom g{};
    int64_t V = 1;
    int stride = 1;
    for (int mu = 0; mu < 4; mu++) {
      if (lat.L[mu] <= 0 || lat.nw < 0 || lat.nw > lat.L[mu]) return fail(ctx, LMB_ERR_ARG, "bad geometry of lattice %d", l);
      const double re = lat.phase_re[mu], im = lat.phase_im[mu], n = re * re + im * im;
      if (n == 0.0) return fail(ctx, LMB_ERR_ARG, "boundary phases must be nonzero because negative wraps use inv(phase)");
      g.L[mu] = lat.L[mu];
      g.stride[mu] = stride;
      stride *= lat.L[mu];
      V *= lat.L[mu];
      g.ph_fwd[mu][0] = re;
      g.ph_fwd[mu][1] = im;
      g.ph_bwd[mu][0] = re / n;
      g.ph_bwd[mu][1] = -im / n;
      if (!(re == 1.0 && im == 0.0)) g.phase_mask |= 1 << mu;
      pads[l].P[mu] = lat.L[mu] + 2 * lat.nw;
    }
    g.V = V;
    pads[l].nw = lat.nw;
    geoms[l] = g;
    for (int mu = 0; mu < 4; mu++)
      if (!lat.U[mu]) return fail(ctx, LMB_ERR_ARG, "gauge link U[%d] of lattice %d is null", mu + 1, l);
    int rc = batch_links_for(ctx, lat, g, pads[l], &links[l], st);
    if (rc) return rc;
    nrhs[l] = lat.nrhs;
    start[l] = total;
    total += lat.nrhs;
    kappa[l] = lat.kappa;
    char buf[96];
    snprintf(buf, sizeof buf, "%dx%dx%dx%d:%d;", lat.L[0], lat.L[1], lat.L[2], lat.L[3], lat.nrhs);
    sig += buf;
  }
  // fields of every member
  std::vector<BatchMember<PS>> m(total);
  for (int l = 0; l < nlat; l++)
    for (int r = 0; r < nrhs[l]; r++) {
      BatchMember<PS> &mm = m[start[l] + r];
      mm.lattice = l;
      mm.rhs = r;
      mm.g = geoms[l];
      mm.pd = pads[l];
      const std::string k = std::to_string(start[l] + r);
      // member fields sized by its own lattice (workspace grows on demand)
      const int64_t V = geoms[l].V;
      auto mk64 = [&](const std::string &n, Field<PREC_DOUBLE, 12> &f) {
        f.V = V;
        f.norm = nullptr;
        f.data = (double2 *)workspace(ctx, n, Field<PREC_DOUBLE, 12>::bytes(V));
        return f.data != nullptr;
      };
      const std::string ks = (PS == PREC_HALF ? "h" : "s") + k;
      if (!mk64("bt_b" + k, mm.b64) || !mk64("bt_x" + k, mm.x64) || !mk64("bt_r" + k, mm.r64) ||
          !mk64("bt_t" + k, mm.t64) || !make_field(ctx, "bt_p" + ks, mm.p, V) ||
          !make_field(ctx, "bt_tl" + ks, mm.t, V) || !make_field(ctx, "bt_rl" + ks, mm.r, V) ||
          !make_field(ctx, "bt_xl" + k, mm.xl, V))
        return fail(ctx, LMB_ERR_CUDA, "out of device memory (batched fields)");
    }
  CGState *states = (CGState *)workspace(ctx, "bt_states", sizeof(CGState) * total);
  if (!states) return fail(ctx, LMB_ERR_CUDA, "out of device memory (batched states)");
  std::vector<CGState> init(total);
  for (auto &s0 : init) {
    s0 = CGState{};
    s0.delta2 = prm->delta * prm->delta;
    s0.maxiter = prm->maxiter;
    s0.status = ST_RUNNING;
  }
  int rc;
  // ---- pack b and x of every member; p = b gives the tuning passes real data
  for (int i = 0; i < total; i++) {
    BatchMember<PS> &mm = m[i];
    const lmb_batch_lattice &lat = lats[mm.lattice];
    const unsigned grid = grid_for(mm.g.V, 256);
    pack_field_kernel<double2, PREC_DOUBLE, 12><<<grid, 256, 0, st>>>(mm.b64, (const double2 *)lat.b[mm.rhs], mm.g, mm.pd);
    pack_field_kernel<double2, PREC_DOUBLE, 12><<<grid, 256, 0, st>>>(mm.x64, (const double2 *)lat.x[mm.rhs], mm.g, mm.pd);
    convert_kernel<PS, PREC_DOUBLE, 12><<<grid_for(mm.g.V, kBlasThreads), kBlasThreads, 0, st>>>(mm.p, mm.b64,
                                                                                               mm.g.V);
    LMB_CHECK_LAUNCH(ctx);
  }
  // ---- autotune (RHS block, threads) on the stencil stages, once per shape set
  lmb_batch_tune tune;
  auto it = ctx->batch_tune.find(sig);
  if (it != ctx->batch_tune.end()) {
    tune = it->second;
  } else {
    double best = 1e30;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::vector<CGState> dummy(total);
    for (auto &d : dummy) {
      d = CGState{};
      d.status = ST_RUNNING;
      d.alpha = 0.0;
      d.rr = 1.0;
      d.maxrr = 1e300;
      d.delta2 = 0.0;
      d.maxiter = 1 << 30;
      d.tol2 = -1.0;
    }
    // (family, NB, NT): links in registers for NB <= 4, in shared memory
    // for NB 4..16
    // for NB 4..16; (2, 16, -): int16 x-adjacent pairs, every lattice's x
    // extent even
    bool even_x = true;
    for (int l = 0; l < nlat; l++) even_x = even_x && geoms[l].L[0] % 2 == 0;
    const int cand[16][3] = {{0, 1, 64},  {0, 1, 128}, {0, 1, 256}, {0, 2, 64},  {0, 2, 128},  {0, 2, 256},
                             {0, 4, 64},  {0, 4, 128}, {0, 4, 256}, {1, 4, 64},  {1, 4, 128},  {1, 8, 64},
                             {1, 8, 128}, {1, 16, 64}, {1, 16, 128}, {2, 16, 256}};
    for (const auto &cd : cand) {
      if (ctx->batch_family >= 0 && cd[0] != ctx->batch_family) continue;
      if (cd[0] == 2 && (PS != PREC_HALF || !even_x)) continue;
      BatchRun br;
      if ((rc = build_run<PS>(ctx, br, cd[0], cd[1], cd[2], m, start, nrhs, links, kappa, "tune"))) return rc;
      if ((rc = upload_groups(ctx, br, st))) return rc;
      LMB_CUDA(ctx, cudaMemcpyAsync(states, dummy.data(), sizeof(CGState) * total, cudaMemcpyHostToDevice, st));
      for (int w = 0; w < 2; w++) {
        if ((rc = batch_stage<PS>(ctx, br, states, 0, st))) return rc;
        if ((rc = batch_stage<PS>(ctx, br, states, 1, st))) return rc;
      }
      cudaEventRecord(e0, st);
      for (int w = 0; w < 3; w++) {
        if ((rc = batch_stage<PS>(ctx, br, states, 0, st))) return rc;
        if ((rc = batch_stage<PS>(ctx, br, states, 1, st))) return rc;
      }
      cudaEventRecord(e1, st);
      LMB_CUDA(ctx, cudaEventSynchronize(e1));
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best) {
        best = ms;
        tune.family = cd[0];
        tune.nb = cd[1];
        tune.nt = cd[2];
        tune.ms = ms / 3.0;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ctx->batch_tune[sig] = tune;
  }
  if (tune.nb == 0) return fail(ctx, LMB_ERR_UNSUPPORTED, "no batched kernel family fits these lattices");
  BatchRun br;
  if ((rc = build_run<PS>(ctx, br, tune.family, tune.nb, tune.nt, m, start, nrhs, links, kappa, "run"))) return rc;
  if ((rc = upload_groups(ctx, br, st))) return rc;
  // the FP64 passes (initial, reliable-update and final true residuals) run
  // on a register-family grouping of the same members, whatever the run's
  // family
  BatchRun aux;
  if ((rc = build_run<PS>(ctx, aux, 0, 4, 256, m, start, nrhs, links, kappa, "aux"))) return rc;
  if ((rc = upload_groups(ctx, aux, st))) return rc;
  LMB_CUDA(ctx, cudaMemcpyAsync(states, init.data(), sizeof(CGState) * total, cudaMemcpyHostToDevice, st));
  // ---- per-member setup: pack b and x, x_low = 0, |b|
  if (!ensure_partials(ctx, grid_for(1 << 24, kBlasThreads), 1))
    return fail(ctx, LMB_ERR_CUDA, "out of device memory (reduction partials)");
  for (int i = 0; i < total; i++) {
    BatchMember<PS> &mm = m[i];
    LMB_CUDA(ctx, cudaMemsetAsync(mm.xl.data, 0, Field<PREC_SINGLE, 12>::bytes(mm.g.V), st));
    norm_b_kernel<12><<<grid_for(mm.g.V, kBlasThreads), kBlasThreads, 0, st>>>(
        mm.b64, states + i, mm.g.V, prm->rtol, prm->atol, ctx->partials, ctx->counter);
    LMB_CHECK_LAUNCH(ctx);
  }
  // ---- r = b - D'D x for all members, p = r
  auto true_pass = [&](const std::vector<unsigned> &masks, int mode) -> int {
    for (size_t gi = 0; gi < aux.groups.size(); gi++) {
      aux.groups[gi].mask = masks[gi];
      aux.groups[gi].mode = mode;
    }
    int r2 = upload_groups(ctx, aux, st);
    if (r2) return r2;
    if ((r2 = batch_stage<PS>(ctx, aux, states, 3, st))) return r2;
    return batch_stage<PS>(ctx, aux, states, 4, st);
  };
  std::vector<unsigned> all_mask(aux.groups.size());
  for (size_t gi = 0; gi < aux.groups.size(); gi++) all_mask[gi] = (1u << aux.groups[gi].nact) - 1u;
  if ((rc = true_pass(all_mask, 0))) return rc;
  for (int i = 0; i < total; i++) {
    convert_kernel<PS, PS, 12><<<grid_for(m[i].g.V, kBlasThreads), kBlasThreads, 0, st>>>(m[i].p, m[i].r,
                                                                                         m[i].g.V);
  }
  LMB_CHECK_LAUNCH(ctx);
  std::vector<CGState> hs(total);
  auto read_all = [&]() -> int {
    LMB_CUDA(ctx, cudaMemcpyAsync(hs.data(), states, sizeof(CGState) * total, cudaMemcpyDeviceToHost, st));
    LMB_CUDA(ctx, cudaStreamSynchronize(st));
    return LMB_OK;
  };
  if ((rc = read_all())) return rc;
  bool fix = false;
  for (auto &x : hs) {
    if (!std::isfinite(x.bb)) { x.status = ST_BREAKDOWN; fix = true; }
    if (x.status == ST_RUNNING && prm->maxiter == 0) { x.status = ST_MAXITER; fix = true; }
  }
  if (fix) LMB_CUDA(ctx, cudaMemcpyAsync(states, hs.data(), sizeof(CGState) * total, cudaMemcpyHostToDevice, st));
  // ---- one iteration as a CUDA graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t cs;
  LMB_CUDA(ctx, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  LMB_CUDA(ctx, cudaStreamSynchronize(st));
  LMB_CUDA(ctx, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  int crc = batch_stage<PS>(ctx, br, states, 0, cs);
  if (!crc) crc = batch_stage<PS>(ctx, br, states, 1, cs);
  if (!crc) crc = batch_stage<PS>(ctx, br, states, 2, cs);
  cudaError_t ge = cudaStreamEndCapture(cs, &graph);
  if (crc || ge != cudaSuccess) {
    cudaStreamDestroy(cs);
    return crc ? crc : fail(ctx, LMB_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ge));
  }
  ge = cudaGraphInstantiate(&exec, graph, 0);
  if (ge != cudaSuccess) {
    cudaGraphDestroy(graph);
    cudaStreamDestroy(cs);
    return fail(ctx, LMB_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ge));
  }
  const int k = prm->check_interval > 0 ? prm->check_interval : 8;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double graph_ms = 0;
  long long graph_iters = 0;
  auto cleanup = [&]() {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    cudaStreamDestroy(cs);
  };
  auto any_running = [&]() {
    for (auto &x : hs)
      if (x.status == ST_RUNNING || x.status == ST_RELIABLE) return true;
    return false;
  };
  while (any_running()) {
    cudaEventRecord(e0, st);
    for (int i = 0; i < k; i++) {
      cudaError_t le = cudaGraphLaunch(exec, st);
      if (le != cudaSuccess) {
        cleanup();
        return fail(ctx, LMB_ERR_CUDA, "graph launch: %s", cudaGetErrorString(le));
      }
    }
    cudaEventRecord(e1, st);
    if ((rc = read_all())) { cleanup(); return rc; }
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    graph_ms += ms;
    graph_iters += k;
    // reliable updates for the paused members
    std::vector<unsigned> masks(aux.groups.size(), 0u);
    bool anyrel = false;
    for (size_t gi = 0; gi < aux.groups.size(); gi++)
      for (int r = 0; r < aux.groups[gi].nact; r++)
        if (hs[aux.groups[gi].state0 + r].status == ST_RELIABLE) {
          masks[gi] |= 1u << r;
          anyrel = true;
          BatchMember<PS> &mm = m[aux.groups[gi].state0 + r];
          fold_kernel<PREC_SINGLE, 12><<<grid_for(mm.g.V, kBlasThreads), kBlasThreads, 0, st>>>(mm.x64, mm.xl, mm.g.V);
        }
    if (anyrel) {
      if ((rc = true_pass(masks, 1))) { cleanup(); return rc; }
      for (size_t gi = 0; gi < aux.groups.size(); gi++)
        for (int r = 0; r < aux.groups[gi].nact; r++)
          if ((masks[gi] >> r) & 1) {
            BatchMember<PS> &mm = m[aux.groups[gi].state0 + r];
            cg_p_update_kernel<PS, 12><<<grid_for(mm.g.V, kBlasThreads), kBlasThreads, 0, st>>>(
                mm.p, mm.r, states + aux.groups[gi].state0 + r, mm.g.V);
          }
      LMB_CHECK_LAUNCH(ctx);
      if ((rc = read_all())) { cleanup(); return rc; }
    }
  }
  // ---- finish: fold, report true residuals, unpack
  for (int i = 0; i < total; i++)
    fold_kernel<PREC_SINGLE, 12><<<grid_for(m[i].g.V, kBlasThreads), kBlasThreads, 0, st>>>(m[i].x64, m[i].xl, m[i].g.V);
  std::vector<CGState> fin = hs;
  if ((rc = true_pass(all_mask, 2))) { cleanup(); return rc; }
  if ((rc = read_all())) { cleanup(); return rc; }
  for (int i = 0; i < total; i++) {
    const BatchMember<PS> &mm = m[i];
    const lmb_batch_lattice &lat = lats[mm.lattice];
    unpack_field_kernel<double2, PREC_DOUBLE, 12><<<grid_for(mm.g.V, 256), 256, 0, st>>>(
        (double2 *)lat.x[mm.rhs], mm.x64, mm.g, mm.pd);
  }
  LMB_CHECK_LAUNCH(ctx);
  LMB_CUDA(ctx, cudaStreamSynchronize(st));
  for (int i = 0; i < total; i++) {
    const CGState &f = fin[i];
    const double bn = std::sqrt(f.bb);
    const double rt = std::sqrt(hs[i].rr_true);
    const double rn = f.status == ST_BREAKDOWN ? NAN : (f.status == ST_CONVERGED ? std::sqrt(f.rr_true) : rt);
    lmb_cg_result &o = res[i];
    std::memset(&o, 0, sizeof o);
    o.converged = f.status == ST_CONVERGED;
    o.iterations = f.iter;
    o.residual_norm = rn;
    o.relative_residual = bn == 0.0 ? (rn == 0.0 ? 0.0 : INFINITY) : rn / bn;
    o.reason = f.status == ST_CONVERGED ? LMB_CG_CONVERGED
               : f.status == ST_MAXITER ? LMB_CG_MAXIMUM_ITERATIONS
               : f.status == ST_NONPOSITIVE ? LMB_CG_NONPOSITIVE_CURVATURE
                                             : LMB_CG_NUMERICAL_BREAKDOWN;
    o.reliable_updates = f.reliable_updates;
    o.true_residual_norm = rt;
    o.link_reals = 12;
  }
  if (tuning) {
    tuning->rhs_block = tune.nb;
    tuning->threads = tune.nt;
    tuning->ms_per_iteration = graph_iters ? graph_ms / graph_iters : 0.0;
    tuning->graph_iterations = (int)graph_iters;
    tuning->kernel_family = tune.family;
    tuning->ms_stencils = tune.ms;
  }
  cleanup();
  return LMB_OK;
}


}  // namespace lmb

extern "C" {

int lmb_cg_ddagd_batched(lmb_ctx *ctx, const lmb_cg_params *prm, int nlattices, const lmb_batch_lattice *lattices,
                         lmb_cg_result *results, lmb_batch_tuning *tuning, void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!prm || !lattices || !results || nlattices <= 0) return fail(ctx, LMB_ERR_ARG, "null or empty argument");
  if (prm->op != LMB_OP_WILSON) return fail(ctx, LMB_ERR_UNSUPPORTED, "batched CG is built for the Wilson operator");
  if (prm->precision != PREC_SINGLE && prm->precision != PREC_HALF)
    return fail(ctx, LMB_ERR_UNSUPPORTED,
                "batched CG runs FP32 arithmetic on FP32 or int16 fields (LMB_PREC_SINGLE / LMB_PREC_HALF)");
  if (!(prm->rtol >= 0) || !std::isfinite(prm->rtol)) return fail(ctx, LMB_ERR_ARG, "rtol must be nonnegative");
  if (!(prm->atol >= 0) || !std::isfinite(prm->atol)) return fail(ctx, LMB_ERR_ARG, "atol must be nonnegative");
  if (prm->maxiter < 0) return fail(ctx, LMB_ERR_ARG, "maxiter must be nonnegative");
  if (!(prm->delta > 0 && prm->delta < 1)) return fail(ctx, LMB_ERR_ARG, "reliable-update delta must lie in (0, 1)");
  if (prm->precision == PREC_HALF)
    return cg_batched<PREC_HALF>(ctx, prm, nlattices, lattices, results, tuning, as_stream(stream));
  return cg_batched<PREC_SINGLE>(ctx, prm, nlattices, lattices, results, tuning, as_stream(stream));
}


}  // extern "C"
