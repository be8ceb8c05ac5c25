// lmb_driver.cuh -- the operator-generic drivers: apply (pack, one stencil,
// unpack) and the D^+D CG with device-resident scalars and reliable updates.
// Each operator translation unit instantiates them for its policy
// (LMB_OP_INSTANCES), one precision per unit where that pays.
#pragma once
#include "lmb_internal.cuh"

namespace lmb {

// operator hooks with the 4D defaults: field volume, pack, unpack
template <class Op> int64_t op_volume(const lmb_ctx *ctx, const Op &) { return ctx->g.V; }
// reduction partials a CG stencil launch of the operator needs (one per block)
template <class Op> int64_t op_max_blocks(const lmb_ctx *ctx, const Op &op) {
  return grid_for(op_volume(ctx, op), kDslashThreads);
}
template <class Op, int PS, int NC>
int op_pack_in(lmb_ctx *ctx, const Op &, Field<PS, NC> &f, const void *src, cudaStream_t st) {
  return pack_in(ctx, f, src, st);
}
// operators on a block of a process grid: device slots for partial sums
// (nullptr: a whole lattice) and their sum over the ranks
template <class Op> double *op_local_sums(const lmb_ctx *, const Op &) { return nullptr; }
template <class Op> int op_allreduce_sums(lmb_ctx *, const Op &, cudaStream_t) { return LMB_OK; }
template <class Op, int PS, int NC>
int op_unpack_out(lmb_ctx *ctx, const Op &, void *dst, const Field<PS, NC> &f, cudaStream_t st) {
  return unpack_out(ctx, dst, f, st);
}

template <int PS, class Op>
int apply_generic(lmb_ctx *ctx, const Op &op, void *out, const void *in, int dagger, cudaStream_t st) {
  constexpr int NC = Op::NC;
  const int64_t V = op_volume(ctx, op);
  Field<PS, NC> fin, fout;
  if (!make_field(ctx, "apply_in", fin, V) || !make_field(ctx, "apply_out", fout, V))
    return fail(ctx, LMB_ERR_CUDA, "out of device memory (apply workspaces)");
  int rc = op_pack_in(ctx, op, fin, in, st);
  if (rc) return rc;
  EpiStore<PS, NC> epi{fout, nullptr};
  rc = dagger ? op.template launch<PS, 1>(ctx, fin, epi, st) : op.template launch<PS, 0>(ctx, fin, epi, st);
  if (rc) return rc;
  return op_unpack_out(ctx, op, out, fout, st);
}

// device time per application of the operator between two resident
// internal fields, input and output swapped after every application (the
// protocol of benchmark/HISQ_DIRAC_BENCHMARK_2026-08-17.md:10-31); two
// untimed applications first
template <int PS, class Op>
int time_generic(lmb_ctx *ctx, const Op &op, const void *in, int napply, int dagger, double *ms, cudaStream_t st) {
  constexpr int NC = Op::NC;
  const int64_t V = op_volume(ctx, op);
  Field<PS, NC> f[2];
  if (!make_field(ctx, "apply_in", f[0], V) || !make_field(ctx, "apply_out", f[1], V))
    return fail(ctx, LMB_ERR_CUDA, "out of device memory (apply workspaces)");
  int rc = op_pack_in(ctx, op, f[0], in, st);
  if (rc) return rc;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    return fail(ctx, LMB_ERR_CUDA, "event creation failed");
  }
  for (int i = 0; i < napply + 2 && rc == LMB_OK; i++) {
    if (i == 2) cudaEventRecord(e0, st);
    EpiStore<PS, NC> epi{f[(i + 1) & 1], nullptr};
    rc = dagger ? op.template launch<PS, 1>(ctx, f[i & 1], epi, st) : op.template launch<PS, 0>(ctx, f[i & 1], epi, st);
  }
  cudaEventRecord(e1, st);
  float t = 0.f;
  const cudaError_t e = cudaEventSynchronize(e1);
  if (e == cudaSuccess) cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  if (e != cudaSuccess) return fail(ctx, LMB_ERR_CUDA, "%s", cudaGetErrorString(e));
  *ms = napply > 0 ? (double)t / napply : 0.0;
  return LMB_OK;
}

template <class Op>
int time_dispatch(lmb_ctx *ctx, const Op &op, const void *in, int napply, int dagger, int prec, double *ms,
                  void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!in || !ms) return fail(ctx, LMB_ERR_ARG, "null argument");
  if (napply < 1) return fail(ctx, LMB_ERR_ARG, "napply must be positive");
  cudaStream_t st = as_stream(stream);
  int rc = op.prepare(ctx, prec, st);
  if (rc) return rc;
  switch (prec) {
    case PREC_DOUBLE: return time_generic<PREC_DOUBLE>(ctx, op, in, napply, dagger, ms, st);
    case PREC_SINGLE: return time_generic<PREC_SINGLE>(ctx, op, in, napply, dagger, ms, st);
    default: return time_generic<PREC_HALF>(ctx, op, in, napply, dagger, ms, st);
  }
}

template <class Op>
int apply_dispatch(lmb_ctx *ctx, const Op &op, void *out, const void *in, int dagger, int prec, void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!out || !in) return fail(ctx, LMB_ERR_ARG, "null field pointer");
  if (out == in) return fail(ctx, LMB_ERR_ARG, "mul! requires distinct result and input fields");
  cudaStream_t st = as_stream(stream);
  int rc = op.prepare(ctx, prec, st);
  if (rc) return rc;
  switch (prec) {
    case PREC_DOUBLE: return apply_generic<PREC_DOUBLE>(ctx, op, out, in, dagger, st);
    case PREC_SINGLE: return apply_generic<PREC_SINGLE>(ctx, op, out, in, dagger, st);
    default: return apply_generic<PREC_HALF>(ctx, op, out, in, dagger, st);
  }
}

// ---------------------------------------------------------------------------
// CG driver
// ---------------------------------------------------------------------------
struct EventPool {
  std::vector<cudaEvent_t> ev;
  void ensure(size_t n) {
    while (ev.size() < n) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      ev.push_back(e);
    }
  }
  ~EventPool() {
    for (auto e : ev) cudaEventDestroy(e);
  }
};

// K3: p = r + beta p; FP32 / int16 Wilson fields of an even volume use the
// two-site kernel (256-bit accesses)
template <int PS, int NC>
void launch_p_update(lmb_ctx *ctx, Field<PS, NC> &p, const Field<PS, NC> &r, int64_t V, cudaStream_t st) {
  if constexpr (PS != PREC_DOUBLE && NC == 12) {
    if (ctx->pair_sites && ctx->adj_sites && V % 2 == 0) {
      cg_p_update_adj_kernel<PS><<<grid_for(V / 2, kBlasThreads), kBlasThreads, 0, st>>>(p, r, ctx->st_dev, V);
      return;
    }
  }
  cg_p_update_kernel<PS, NC><<<grid_for(V, kBlasThreads), kBlasThreads, 0, st>>>(p, r, ctx->st_dev, V);
}

// PS: precision of the iterated fields (DOUBLE = plain FP64 CG), PX: of x_low
template <int PS, int PX, class Op>
int cg_run(lmb_ctx *ctx, const lmb_cg_params *prm, const Op &op, void *x_pad, const void *b_pad,
           lmb_cg_result *res, cudaStream_t st) {
  constexpr bool mixed = PS != PREC_DOUBLE;
  constexpr int NC = Op::NC;
  const int64_t V = op_volume(ctx, op);
  int rc;
  long long nl = 0;  // liblmb200 kernels launched by this solve
  Field<PREC_DOUBLE, NC> b64, x64, r64, t64;
  if (!make_field(ctx, "cg_b", b64, V) || !make_field(ctx, "cg_x", x64, V) || !make_field(ctx, "cg_r", r64, V) ||
      !make_field(ctx, "cg_t", t64, V))
    return fail(ctx, LMB_ERR_CUDA, "out of device memory (CG FP64 fields)");
  Field<PS, NC> p, rl, tl;
  Field<PX, NC> xl;
  if (!make_field(ctx, "cg_p", p, V)) return fail(ctx, LMB_ERR_CUDA, "out of device memory (CG p)");
  if constexpr (mixed) {
    if (!make_field(ctx, "cg_rl", rl, V) || !make_field(ctx, "cg_tl", tl, V) || !make_field(ctx, "cg_xl", xl, V))
      return fail(ctx, LMB_ERR_CUDA, "out of device memory (CG low-precision fields)");
  } else {
    rl = *(Field<PS, NC> *)&r64;
    tl = *(Field<PS, NC> *)&t64;
    xl = *(Field<PX, NC> *)&x64;
  }
  const unsigned dgrid = grid_for(V, kDslashThreads), bgrid = grid_for(V, kBlasThreads);
  const int64_t ogrid = op_max_blocks(ctx, op);
  int64_t pgrid = dgrid > bgrid ? dgrid : bgrid;
  if (ogrid > pgrid) pgrid = ogrid;
  if (!ensure_partials(ctx, pgrid, 2))
    return fail(ctx, LMB_ERR_CUDA, "out of device memory (reduction partials)");
  rc = op.prepare(ctx, PREC_DOUBLE, st);
  if (rc) return rc;
  // Links with a non-finite entry make D x non-finite for every x, so the
  // initial FP64 residual b - D'D x breaks the solve down at iteration 0 with
  // a NaN residual, as the reference's cg! does (cg.jl:93-104); the
  // low-precision copies are never built or used then.
  const bool finite_links = op.links_finite(ctx);
  if (mixed && finite_links) {
    rc = op.prepare(ctx, PS, st);
    if (rc) return rc;
  }

  // initial state
  CGState init{};
  init.delta2 = mixed ? prm->delta * prm->delta : 0.0;
  init.maxiter = prm->maxiter;
  init.status = ST_RUNNING;
  LMB_CUDA(ctx, cudaMemcpyAsync(ctx->st_dev, &init, sizeof init, cudaMemcpyHostToDevice, st));
  rc = op_pack_in(ctx, op, b64, b_pad, st);
  if (rc) return rc;
  rc = op_pack_in(ctx, op, x64, x_pad, st);
  if (rc) return rc;
  nl += 2;
  if constexpr (mixed) {
    LMB_CUDA(ctx, cudaMemsetAsync(xl.data, 0, Field<PX, NC>::bytes(V), st));
    if (xl.norm) LMB_CUDA(ctx, cudaMemsetAsync(xl.norm, 0, Field<PX, NC>::norm_bytes(V), st));
  }
  norm_bx_kernel<NC><<<bgrid, kBlasThreads, 0, st>>>(b64, x64, ctx->st_dev, V, prm->rtol, prm->atol,
                                                      ctx->partials, ctx->counter, op_local_sums(ctx, op));
  LMB_CHECK_LAUNCH(ctx);
  nl++;
  if (op_local_sums(ctx, op)) {  // a block of a process grid: sum |b|^2, |x0|^2 over the ranks
    rc = op_allreduce_sums(ctx, op, st);
    if (rc) return rc;
    set_norms_kernel<<<1, 32, 0, st>>>(ctx->st_dev, op_local_sums(ctx, op), prm->rtol, prm->atol);
    LMB_CHECK_LAUNCH(ctx);
  }
  rc = read_state(ctx, st);
  if (rc) return rc;
  // b - D'D 0 = b needs finite links (NaN * 0 is NaN); on a process grid the
  // shortcut's local |b|^2 would need a sum over the ranks, so it is skipped
  const bool zero_guess = ctx->st_host->xx == 0.0 && finite_links && !op_local_sums(ctx, op);
  // r = b - D'D x (FP64)
  auto true_residual = [&](int mode) -> int {
    EpiStore<PREC_DOUBLE, NC> e1{t64, nullptr};
    int r2 = op.template launch<PREC_DOUBLE, 0>(ctx, x64, e1, st);
    if (r2) return r2;
    nl += 2;
    EpiTrueResidual<PS, NC> e2{b64, r64, rl, mixed ? 1 : 0, mode, ctx->st_dev, ctx->partials, ctx->counter};
    return op.template launch<PREC_DOUBLE, 1>(ctx, t64, e2, st);
  };
  if (zero_guess) {
    // b - D'D 0 = b exactly: one pass instead of two FP64 stencils
    residual_of_zero_kernel<PS, NC><<<dgrid, kDslashThreads, 0, st>>>(b64, r64, rl, mixed ? 1 : 0, 0, ctx->st_dev,
                                                                      V, ctx->partials, ctx->counter);
    LMB_CHECK_LAUNCH(ctx);
    nl++;
  } else {
    rc = true_residual(0);
    if (rc) return rc;
  }
  convert_kernel<PS, PS, NC><<<bgrid, kBlasThreads, 0, st>>>(p, rl, V);
  LMB_CHECK_LAUNCH(ctx);
  nl++;
  rc = read_state(ctx, st);
  if (rc) return rc;
  CGState *hs = ctx->st_host;
  if (!std::isfinite(hs->bb)) hs->status = ST_BREAKDOWN;
  if (hs->status == ST_RUNNING && prm->maxiter == 0) hs->status = ST_MAXITER;
  if (mixed && !finite_links && hs->status == ST_RUNNING)  // finite in FP64, beyond FP32 range
    return fail(ctx, LMB_ERR_ARG, "gauge links lie beyond FP32 range: solve with FP64 fields");
  if (hs->status != ST_RUNNING)
    LMB_CUDA(ctx, cudaMemcpyAsync(ctx->st_dev, hs, sizeof(CGState), cudaMemcpyHostToDevice, st));

  const int k = prm->check_interval > 0 ? prm->check_interval : 8;
  EventPool pool;
  if (prm->profile) pool.ensure(4 * (size_t)k);
  double k1_ms = 0, k2_ms = 0;
  int k1_n = 0, k2_n = 0;

  EpiStoreNorm<PS, NC> epi1{tl, ctx->st_dev, ctx->partials, ctx->counter};
  EpiCGUpdate<PS, PX, NC> epi2{p, rl, xl, ctx->st_dev, ctx->partials, ctx->counter};
  while (hs->status == ST_RUNNING) {
    const int it0 = hs->iter;
    for (int i = 0; i < k; i++) {
      if (prm->profile) cudaEventRecord(pool.ev[4 * i], st);
      rc = op.template launch<PS, 0>(ctx, p, epi1, st);
      if (rc) return rc;
      nl++;
      if (prm->profile) cudaEventRecord(pool.ev[4 * i + 1], st);
      rc = op.template launch<PS, 1>(ctx, tl, epi2, st);
      if (rc) return rc;
      nl++;
      if (prm->profile) cudaEventRecord(pool.ev[4 * i + 2], st);
      launch_p_update<PS, NC>(ctx, p, rl, V, st);
      LMB_CHECK_LAUNCH(ctx);
      nl++;
      if (prm->profile) cudaEventRecord(pool.ev[4 * i + 3], st);
    }
    rc = read_state(ctx, st);
    if (rc) return rc;
    if (prm->profile) {
      const int real = hs->iter - it0 + (hs->status == ST_RELIABLE ? 1 : 0);
      for (int i = 0; i < real && i < k; i++) {
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, pool.ev[4 * i], pool.ev[4 * i + 1]);
        cudaEventElapsedTime(&b, pool.ev[4 * i + 1], pool.ev[4 * i + 2]);
        k1_ms += a;
        k2_ms += b;
        k1_n++;
        k2_n++;
      }
    }
    if (hs->status == ST_RELIABLE) {
      if constexpr (mixed) {
        fold_kernel<PX, NC><<<bgrid, kBlasThreads, 0, st>>>(x64, xl, V);
        LMB_CHECK_LAUNCH(ctx);
        nl++;
        // resume: the true-residual kernel runs regardless of the pause
        rc = true_residual(1);
        if (rc) return rc;
        launch_p_update<PS, NC>(ctx, p, rl, V, st);
        LMB_CHECK_LAUNCH(ctx);
        nl++;
        rc = read_state(ctx, st);
        if (rc) return rc;
      }
    }
  }
  if constexpr (mixed) {
    fold_kernel<PX, NC><<<bgrid, kBlasThreads, 0, st>>>(x64, xl, V);
    LMB_CHECK_LAUNCH(ctx);
    nl++;
  }
  const int status = hs->status;
  CGState final_state = *hs;
  // true residual for the report (does not change the outcome)
  if (!mixed || status != ST_CONVERGED) {
    rc = true_residual(2);
    if (rc) return rc;
    rc = read_state(ctx, st);
    if (rc) return rc;
  }
  const double rr_true = ctx->st_host->rr_true;
  rc = op_unpack_out(ctx, op, x_pad, x64, st);
  if (rc) return rc;
  nl++;
  LMB_CUDA(ctx, cudaStreamSynchronize(st));

  const double bn = std::sqrt(final_state.bb);
  double rn;
  if (status == ST_BREAKDOWN) rn = NAN;
  else rn = mixed ? std::sqrt(final_state.rr_true) : std::sqrt(final_state.rr);
  if (mixed && status != ST_CONVERGED && status != ST_BREAKDOWN) rn = std::sqrt(rr_true);
  res->converged = status == ST_CONVERGED;
  res->iterations = final_state.iter;
  res->residual_norm = rn;
  res->relative_residual = bn == 0.0 ? (rn == 0.0 ? 0.0 : INFINITY) : rn / bn;
  switch (status) {
    case ST_CONVERGED: res->reason = LMB_CG_CONVERGED; break;
    case ST_MAXITER: res->reason = LMB_CG_MAXIMUM_ITERATIONS; break;
    case ST_NONPOSITIVE: res->reason = LMB_CG_NONPOSITIVE_CURVATURE; break;
    default: res->reason = LMB_CG_NUMERICAL_BREAKDOWN; break;
  }
  res->reliable_updates = final_state.reliable_updates;
  res->true_residual_norm = std::sqrt(rr_true);
  res->dslash_ms = k1_ms;
  res->update_ms = k2_ms;
  res->dslash_launches = k1_n;
  res->update_launches = k2_n;
  res->kernel_launches = nl;
  res->link_reals = op.link_reals(ctx, PS);
  return LMB_OK;
}

template <class Op>
int cg_dispatch(lmb_ctx *ctx, const lmb_cg_params *prm, const Op &op, void *x, const void *b,
                lmb_cg_result *res, cudaStream_t st) {
  switch (prm->precision) {
    case PREC_DOUBLE: return cg_run<PREC_DOUBLE, PREC_DOUBLE>(ctx, prm, op, x, b, res, st);
    case PREC_SINGLE: return cg_run<PREC_SINGLE, PREC_SINGLE>(ctx, prm, op, x, b, res, st);
    case PREC_HALF: return cg_run<PREC_HALF, PREC_SINGLE>(ctx, prm, op, x, b, res, st);
    default: return fail(ctx, LMB_ERR_ARG, "unknown precision %d", prm->precision);
  }
}

// explicit instantiations of the drivers for one operator policy and one
// precision PS of the iterated fields (PX: precision of x_low); EXT = extern
// declares them, empty defines them
#define LMB_OP_INSTANCE(EXT, OP, PS, PX)                                                                  \
  EXT template int apply_generic<PS, OP>(lmb_ctx *, const OP &, void *, const void *, int, cudaStream_t); \
  EXT template int time_generic<PS, OP>(lmb_ctx *, const OP &, const void *, int, int, double *,         \
                                        cudaStream_t);                                                   \
  EXT template int cg_run<PS, PX, OP>(lmb_ctx *, const lmb_cg_params *, const OP &, void *, const void *, \
                                      lmb_cg_result *, cudaStream_t);
#define LMB_OP_INSTANCES(EXT, OP)                    \
  LMB_OP_INSTANCE(EXT, OP, PREC_DOUBLE, PREC_DOUBLE) \
  LMB_OP_INSTANCE(EXT, OP, PREC_SINGLE, PREC_SINGLE) \
  LMB_OP_INSTANCE(EXT, OP, PREC_HALF, PREC_SINGLE)

}  // namespace lmb
