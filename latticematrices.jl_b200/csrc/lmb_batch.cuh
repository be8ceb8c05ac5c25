// lmb_batch.cuh -- batched D'D CG: many right-hand sides of several lattices
// of different sizes in one launch per CG stage.
//
// Work list.  Right-hand sides of one lattice are grouped NB at a time; a
// task is (group, block of NT sites).  One persistent launch walks all tasks
// of all groups with a grid-stride loop, so small lattices (8^4 = 32 tasks)
// share the GPU with large ones.  A thread owns one site and applies each
// link it loads to the NB right-hand sides of its group: the links are read
// once per site per group instead of once per right-hand side.
//
// A second family (batch_wilson_smem_kernel) takes larger groups (NB up to
// 16): a block first copies the 8 links of each of its sites into shared
// memory, then runs the single-right-hand-side stencil once per member of the
// group reading the links from there, so a link is read from HBM once per
// group whatever NB is and the registers hold one right-hand side at a time.
// Both families store the iterated fields p, tmp, r in FP32 or in int16
// (PS); x_low stays FP32.  A third family (int16 only, even x extents) runs
// the single-lattice int16 stencil (two x-adjacent sites per thread,
// 256-bit loads, projection on the raw int16 words) on tasks (tile, member)
// with the member index fastest: the members of a group read the same
// links within a few microseconds, so the links come from HBM about once
// per tile and from L2 for the others.
//
// Every right-hand side runs its own CG (cg.jl:73-137) with device-resident
// scalars (CGState); a right-hand side that has finished or paused for a
// reliable update is skipped by all later kernels while the others go on.
// Reductions are per task (NB partial sums), and the last task of a group to
// finish reduces the group's partials and updates the NB states.
#pragma once
#include "lmb_solver.cuh"
#include "lmb_wilson.cuh"

namespace lmb {

constexpr int kMaxNB = 16;

struct BatchGroup {
  Geom g;
  const void *U;       // reconstruct-12 links: float4 (FP32 kernels) / double2 (FP64 kernels)
  const int4 *Uh;      // int16 reconstruct-12 links (x-adjacent pair family)
  const void *U64;     // FP64 reconstruct-12 links
  int nact;            // right-hand sides in the group (<= NB)
  int first_task;      // first task of the group in the work list
  int ntasks;          // tasks of the group (sites / NT rounded up)
  int state0;          // CGState index of the group's first right-hand side
  double kappa;
  // iterated fields in the storage of the run (float4 or int4 planes; the
  // int16 norms in pn / tn / rn), x_low FP32
  void *p[kMaxNB], *t[kMaxNB], *r[kMaxNB];
  float *pn[kMaxNB], *tn[kMaxNB], *rn[kMaxNB];
  float4 *xl[kMaxNB];
  double2 *b64[kMaxNB], *x64[kMaxNB], *r64[kMaxNB], *t64[kMaxNB];  // FP64 fields
  double *partials;    // ntasks * NB
  unsigned *counter;
  unsigned mask;       // FP64 passes: right-hand sides to process (bit per member)
  int mode;            // finalize_true mode of the FP64 true-residual pass
};

enum BatchRole { ROLE_K1 = 0, ROLE_K2 = 1, ROLE_D64 = 2, ROLE_TRUE = 3 };

// a member's field of storage PS
template <int PS> LMB_D Field<PS, 12> bfield(void *data, float *norm, int64_t V) {
  Field<PS, 12> f;
  f.data = (decltype(f.data))data;
  f.norm = norm;
  f.V = V;
  return f;
}

LMB_D int find_group(const BatchGroup *groups, int ngroups, int task) {
  int lo = 0, hi = ngroups - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (groups[mid].first_task <= task) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// stencil for NB right-hand sides sharing the link loads (FP32 arithmetic)
template <int DAG, int MU, int NB, int PS, class G>
LMB_D void hop_dir_multi(const Geom &g, int s, const int *c, const Field<PS, 12> *in, const bool *on,
                         const G &U, Cx<float> (*acc)[12]) {
  constexpr int FPM = DAG ? +1 : -1;
  constexpr int BPM = -FPM;
  Cx<float> p[12], h[6], uh[6], u[9];
  int wrap;
  const int sp = fwd_site(g, s, c, MU, 1, &wrap);
  U.load(MU, s, u);
#pragma unroll
  for (int r = 0; r < NB; r++) {
    if (!on[r]) continue;
    in[r].load(sp, p);
    project<FPM, MU>(p, h);
    if (wrap && ((g.phase_mask >> MU) & 1)) scale_phase(h, 6, g.ph_fwd[MU]);
    su3_mul_half(u, h, uh);
    reconstruct<FPM, MU>(acc[r], uh);
  }
  int wb;
  const int sm = bwd_site(g, s, c, MU, 1, &wb);
  U.load(MU, sm, u);
#pragma unroll
  for (int r = 0; r < NB; r++) {
    if (!on[r]) continue;
    in[r].load(sm, p);
    project<BPM, MU>(p, h);
    if (wb && ((g.phase_mask >> MU) & 1)) scale_phase(h, 6, g.ph_bwd[MU]);
    su3_adj_mul_half(u, h, uh);
    reconstruct<BPM, MU>(acc[r], uh);
  }
}

// K1 (tmp = D p, |tmp|^2) and K2 (D^+ tmp fused with the CG update), FP32
// arithmetic on fields stored as PS
template <int NT, int NB, int ROLE, int PS>
__global__ void __launch_bounds__(NT)
    batch_wilson_kernel(const BatchGroup *groups, int ngroups, int ntasks_total, CGState *states) {
  for (int task = blockIdx.x; task < ntasks_total; task += gridDim.x) {
    const int gi = find_group(groups, ngroups, task);
    const BatchGroup &G = groups[gi];
    bool on[NB];
    bool any = false;
#pragma unroll
    for (int r = 0; r < NB; r++) {
      on[r] = r < G.nact && ((volatile CGState *)states)[G.state0 + r].status == ST_RUNNING;
      any |= on[r];
    }
    if (!any) continue;  // uniform over the block
    const Geom &g = G.g;
    const int local = task - G.first_task;
    const int s = local * NT + threadIdx.x;
    const bool active = s < g.V;
    Field<PS, 12> in[NB];
#pragma unroll
    for (int r = 0; r < NB; r++)
      in[r] = ROLE == ROLE_K1 ? bfield<PS>(G.p[r], G.pn[r], g.V) : bfield<PS>(G.t[r], G.tn[r], g.V);
    double n2[NB], tot[NB];
#pragma unroll
    for (int r = 0; r < NB; r++) n2[r] = 0.0;
    if (active) {
      int c[4];
      site_coords(g, s, c);
      Cx<float> acc[NB][12];
#pragma unroll
      for (int r = 0; r < NB; r++)
#pragma unroll
        for (int k = 0; k < 12; k++) acc[r][k] = Cx<float>(0, 0);
      const Gauge12<PREC_SINGLE> U{(const float4 *)G.U, g.V, 1.f};
      constexpr int DAG = ROLE == ROLE_K2 ? 1 : 0;
      hop_dir_multi<DAG, 0, NB>(g, s, c, in, on, U, acc);
      hop_dir_multi<DAG, 1, NB>(g, s, c, in, on, U, acc);
      hop_dir_multi<DAG, 2, NB>(g, s, c, in, on, U, acc);
      hop_dir_multi<DAG, 3, NB>(g, s, c, in, on, U, acc);
      const float kappa = (float)G.kappa;
#pragma unroll
      for (int r = 0; r < NB; r++) {
        if (!on[r]) continue;
        Cx<float> psi[12], v[12];
        in[r].load(s, psi);
#pragma unroll
        for (int k = 0; k < 12; k++) v[k] = psi[k] - kappa * acc[r][k];
        if (ROLE == ROLE_K1) {
          Field<PS, 12> t = bfield<PS>(G.t[r], G.tn[r], g.V);
          t.store(s, v);
          n2[r] = sum_norm2(v, 12);
        } else {
          const float alpha = (float)states[G.state0 + r].alpha;
          Field<PS, 12> pf = bfield<PS>(G.p[r], G.pn[r], g.V), rf = bfield<PS>(G.r[r], G.rn[r], g.V);
          Field<PREC_SINGLE, 12> xf{G.xl[r], nullptr, g.V};
          Cx<float> pv[12], rv[12], xv[12];
          pf.load(s, pv);
          rf.load(s, rv);
          xf.load(s, xv);
#pragma unroll
          for (int k = 0; k < 12; k++) {
            rv[k] = rv[k] - alpha * v[k];
            xv[k] = xv[k] + alpha * pv[k];
          }
          rf.store(s, rv);
          xf.store(s, xv);
          n2[r] = sum_norm2(rv, 12);
        }
      }
    }
    if (grid_reduce_slots<NT, NB>(n2, G.partials, G.counter, tot, (unsigned)local, (unsigned)G.ntasks) &&
        threadIdx.x == 0) {
#pragma unroll
      for (int r = 0; r < NB; r++) {
        if (!on[r]) continue;
        if (ROLE == ROLE_K1) finalize_pAp(&states[G.state0 + r], tot[r]);
        else finalize_rr(&states[G.state0 + r], tot[r]);
      }
    }
    __syncthreads();  // the next task's status reads follow this task's finalize
  }
}

// FP64 passes for the members in G.mask: ROLE_D64 t64 = D x64;
// ROLE_TRUE r64 = b64 - D^+ t64, r (storage PS) = r64, |r64|^2 -> finalize_true.
// They run at the start, at reliable updates and at the end only, so one
// form serves every group size (kMaxNB reduction slots, members in a loop).
template <int NT, int ROLE, int PS>
__global__ void __launch_bounds__(NT)
    batch_wilson64_kernel(const BatchGroup *groups, int ngroups, int ntasks_total, CGState *states) {
  for (int task = blockIdx.x; task < ntasks_total; task += gridDim.x) {
    const int gi = find_group(groups, ngroups, task);
    const BatchGroup &G = groups[gi];
    if (!G.mask) continue;
    const Geom &g = G.g;
    const int local = task - G.first_task;
    const int s = local * NT + threadIdx.x;
    const bool active = s < g.V;
    double n2[kMaxNB], tot[kMaxNB];
    const Gauge12<PREC_DOUBLE> U{(const double2 *)G.U64, g.V, 1.f};
#pragma unroll 1
    for (int r = 0; r < kMaxNB; r++) {
      n2[r] = 0.0;
      if (!active || r >= G.nact || !((G.mask >> r) & 1)) continue;
      Cx<double> v[12];
      if (ROLE == ROLE_D64) {
        const Field<PREC_DOUBLE, 12> in{G.x64[r], nullptr, g.V};
        wilson_site<double, 0>(g, s, in, U, G.kappa, v);
        Field<PREC_DOUBLE, 12> t{G.t64[r], nullptr, g.V};
        t.store(s, v);
      } else {
        const Field<PREC_DOUBLE, 12> in{G.t64[r], nullptr, g.V};
        wilson_site<double, 1>(g, s, in, U, G.kappa, v);
        const Field<PREC_DOUBLE, 12> b{G.b64[r], nullptr, g.V};
        Field<PREC_DOUBLE, 12> rr{G.r64[r], nullptr, g.V};
        Field<PS, 12> rl = bfield<PS>(G.r[r], G.rn[r], g.V);
        Cx<double> bv[12];
        b.load(s, bv);
#pragma unroll
        for (int k = 0; k < 12; k++) v[k] = bv[k] - v[k];
        rr.store(s, v);
        rl.store(s, v);
        n2[r] = sum_norm2(v, 12);
      }
    }
    if (ROLE == ROLE_TRUE) {
      if (grid_reduce_slots<NT, kMaxNB>(n2, G.partials, G.counter, tot, (unsigned)local, (unsigned)G.ntasks) &&
          threadIdx.x == 0) {
#pragma unroll 1
        for (int r = 0; r < kMaxNB; r++)
          if (r < G.nact && ((G.mask >> r) & 1)) finalize_true(&states[G.state0 + r], tot[r], G.mode);
      }
      __syncthreads();
    }
  }
}

// K3 for all running members: p = r + beta p (FP32 arithmetic, storage PS)
template <int NT, int NB, int PS>
__global__ void __launch_bounds__(NT)
    batch_p_update_kernel(const BatchGroup *groups, int ngroups, int ntasks_total, const CGState *states) {
  for (int task = blockIdx.x; task < ntasks_total; task += gridDim.x) {
    const int gi = find_group(groups, ngroups, task);
    const BatchGroup &G = groups[gi];
    const int s = (task - G.first_task) * NT + threadIdx.x;
    if (s >= G.g.V) continue;
#pragma unroll
    for (int r = 0; r < NB; r++) {
      if (r >= G.nact) continue;
      const CGState &st = states[G.state0 + r];
      if (((volatile const CGState *)&st)->status != ST_RUNNING) continue;
      const float beta = (float)st.beta;
      Field<PS, 12> pf = bfield<PS>(G.p[r], G.pn[r], G.g.V), rf = bfield<PS>(G.r[r], G.rn[r], G.g.V);
      Cx<float> pv[12], rv[12];
      pf.load(s, pv);
      rf.load(s, rv);
#pragma unroll
      for (int k = 0; k < 12; k++) pv[k] = rv[k] + beta * pv[k];
      pf.store(s, pv);
    }
  }
}

// ---------------------------------------------------------------------------
// Shared-memory link family.  A block's NT threads own NT sites of one
// group; each copies the reconstruct-12 FP32 rows of its site's 8 links
// (U_mu(x), slot mu; U_mu(x - mu), slot 4 + mu; 3 float4 each) into shared
// memory once, then computes the stencil for the group's members one after
// another, reading the links from there.  Each thread reads only the slots it
// wrote, so no barrier separates the copy from the use.  Per member the norm
// is reduced over the warp at once (deterministic order) into red[r][warp].
// ---------------------------------------------------------------------------
template <int NT>
constexpr size_t batch_smem_bytes() {
  return sizeof(float4) * 24 * NT;
}

template <typename R>
LMB_D void smem_link(const float4 *sl, int slot, int NTv, int tid, Cx<R> *u) {
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const float4 t = sl[(slot * 3 + k) * NTv + tid];
    const int e0 = 2 * k, e1 = 2 * k + 1;
    u[(e0 / 3) + 3 * (e0 % 3)] = Cx<R>((R)t.x, (R)t.y);
    u[(e1 / 3) + 3 * (e1 % 3)] = Cx<R>((R)t.z, (R)t.w);
  }
  su3_third_row(u);
}

template <int NT, int NB, int ROLE, int PS>
__global__ void __launch_bounds__(NT)
    batch_wilson_smem_kernel(const BatchGroup *groups, int ngroups, int ntasks_total, CGState *states) {
  extern __shared__ float4 sl[];  // [24][NT]
  __shared__ double red[NB][NT / 32];
  constexpr int DAG = ROLE == ROLE_K2 ? 1 : 0;
  constexpr int FPM = DAG ? +1 : -1;
  constexpr int BPM = -FPM;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int task = blockIdx.x; task < ntasks_total; task += gridDim.x) {
    const int gi = find_group(groups, ngroups, task);
    const BatchGroup &G = groups[gi];
    unsigned onmask = 0;
    for (int r = 0; r < G.nact; r++)
      if (((volatile CGState *)states)[G.state0 + r].status == ST_RUNNING) onmask |= 1u << r;
    if (!onmask) continue;  // uniform over the block
    const Geom &g = G.g;
    const int local = task - G.first_task;
    const int s = local * NT + tid;
    const bool active = s < g.V;
    int c[4] = {0, 0, 0, 0}, nbf[4] = {0, 0, 0, 0}, nbb[4] = {0, 0, 0, 0};
    unsigned wf = 0, wb = 0;
    if (active) {
      site_coords(g, s, c);
      const float4 *U = (const float4 *)G.U;
#pragma unroll
      for (int mu = 0; mu < 4; mu++) {
        int w;
        nbf[mu] = fwd_site(g, s, c, mu, 1, &w);
        wf |= (unsigned)w << mu;
        nbb[mu] = bwd_site(g, s, c, mu, 1, &w);
        wb |= (unsigned)w << mu;
#pragma unroll
        for (int k = 0; k < 3; k++) {
          sl[(mu * 3 + k) * NT + tid] = __ldg(U + (mu * 3 + k) * g.V + s);
          sl[((4 + mu) * 3 + k) * NT + tid] = __ldg(U + (mu * 3 + k) * g.V + nbb[mu]);
        }
      }
    }
#pragma unroll 1
    for (int r = 0; r < NB; r++) {
      double n2 = 0.0;
      if (((onmask >> r) & 1u) && active) {
        const Field<PS, 12> in =
            ROLE == ROLE_K1 ? bfield<PS>(G.p[r], G.pn[r], g.V) : bfield<PS>(G.t[r], G.tn[r], g.V);
        Cx<float> acc[12];
#pragma unroll
        for (int k = 0; k < 12; k++) acc[k] = Cx<float>(0, 0);
#pragma unroll
        for (int mu = 0; mu < 4; mu++) {
          Cx<float> p[12], h[6], uh[6], u[9];
          in.load(nbf[mu], p);
          if (mu == 0) project<FPM, 0>(p, h);
          else if (mu == 1) project<FPM, 1>(p, h);
          else if (mu == 2) project<FPM, 2>(p, h);
          else project<FPM, 3>(p, h);
          if (((wf >> mu) & 1u) && ((g.phase_mask >> mu) & 1)) scale_phase(h, 6, g.ph_fwd[mu]);
          smem_link(sl, mu, NT, tid, u);
          su3_mul_half(u, h, uh);
          if (mu == 0) reconstruct<FPM, 0>(acc, uh);
          else if (mu == 1) reconstruct<FPM, 1>(acc, uh);
          else if (mu == 2) reconstruct<FPM, 2>(acc, uh);
          else reconstruct<FPM, 3>(acc, uh);
          in.load(nbb[mu], p);
          if (mu == 0) project<BPM, 0>(p, h);
          else if (mu == 1) project<BPM, 1>(p, h);
          else if (mu == 2) project<BPM, 2>(p, h);
          else project<BPM, 3>(p, h);
          if (((wb >> mu) & 1u) && ((g.phase_mask >> mu) & 1)) scale_phase(h, 6, g.ph_bwd[mu]);
          smem_link(sl, 4 + mu, NT, tid, u);
          su3_adj_mul_half(u, h, uh);
          if (mu == 0) reconstruct<BPM, 0>(acc, uh);
          else if (mu == 1) reconstruct<BPM, 1>(acc, uh);
          else if (mu == 2) reconstruct<BPM, 2>(acc, uh);
          else reconstruct<BPM, 3>(acc, uh);
        }
        const float kappa = (float)G.kappa;
        Cx<float> psi[12], v[12];
        in.load(s, psi);
#pragma unroll
        for (int k = 0; k < 12; k++) v[k] = psi[k] - kappa * acc[k];
        if (ROLE == ROLE_K1) {
          Field<PS, 12> t = bfield<PS>(G.t[r], G.tn[r], g.V);
          t.store(s, v);
          n2 = sum_norm2(v, 12);
        } else {
          const float alpha = (float)states[G.state0 + r].alpha;
          Field<PS, 12> pf = bfield<PS>(G.p[r], G.pn[r], g.V), rf = bfield<PS>(G.r[r], G.rn[r], g.V);
          Field<PREC_SINGLE, 12> xf{G.xl[r], nullptr, g.V};
          Cx<float> pv[12], rv[12], xv[12];
          pf.load(s, pv);
          rf.load(s, rv);
          xf.load(s, xv);
#pragma unroll
          for (int k = 0; k < 12; k++) {
            rv[k] = rv[k] - alpha * v[k];
            xv[k] = xv[k] + alpha * pv[k];
          }
          rf.store(s, rv);
          xf.store(s, xv);
          n2 = sum_norm2(rv, 12);
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) n2 += __shfl_xor_sync(0xffffffffu, n2, o);
      if (lane == 0) red[r][warp] = n2;
    }
    // the block's partials, then the group's last task reduces them in task
    // order and takes the scalar steps
    __shared__ bool last;
    __syncthreads();
    if (tid == 0) {
      double *part = G.partials + (size_t)NB * local;
#pragma unroll 1
      for (int r = 0; r < NB; r++) {
        double x = 0;
        for (int w = 0; w < NT / 32; w++) x += red[r][w];
        part[r] = x;
      }
      __threadfence();
      const unsigned ticket = atomicAdd(G.counter, 1u);
      last = ticket == (unsigned)G.ntasks - 1;
    }
    __syncthreads();
    if (last) {
      __threadfence();
#pragma unroll 1
      for (int r = 0; r < NB; r++) {
        double x = 0;
        for (int b = tid; b < G.ntasks; b += NT) x += ((volatile double *)G.partials)[(size_t)NB * b + r];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[r][warp] = x;
      }
      __syncthreads();
      if (tid == 0) {
#pragma unroll 1
        for (int r = 0; r < NB; r++) {
          if (!((onmask >> r) & 1u)) continue;
          double x = 0;
          for (int w = 0; w < NT / 32; w++) x += red[r][w];
          if (ROLE == ROLE_K1) finalize_pAp(&states[G.state0 + r], x);
          else finalize_rr(&states[G.state0 + r], x);
        }
        *G.counter = 0u;
      }
    }
    __syncthreads();  // the next task's status reads and shared-memory use follow this task's
  }
}

// ---------------------------------------------------------------------------
// x-adjacent pair family (int16 fields, FP32 arithmetic).  Task t of a group
// is (tile group = t / nact, member r = t % nact); a tile group is
// kPairTilesPerTask tiles of kDslashThreads pairs of x-adjacent sites, walked
// by one block with its norm carried in registers.  The stencil is the single-lattice one
// (half_adj_sites, Wilson without clover), the epilogue the CG one of
// EpiStoreNorm / EpiCGUpdate; each task leaves its block's sum in
// partials[t], and the group's last task sums every member's partials in
// tile order and takes the scalar steps.
// ---------------------------------------------------------------------------
constexpr int kPairTilesPerTask = 8;

LMB_D bool pair_task_done(const BatchGroup &G, int local, double n2, int ntiles, CGState *states, int role) {
  __shared__ double red[kDslashThreads / 32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) n2 += __shfl_xor_sync(0xffffffffu, n2, o);
  if (lane == 0) red[warp] = n2;
  __syncthreads();
  if (threadIdx.x == 0) {
    double x = 0;
    for (int w = 0; w < kDslashThreads / 32; w++) x += red[w];
    G.partials[local] = x;
    __threadfence();
    last = atomicAdd(G.counter, 1u) == (unsigned)G.ntasks - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
#pragma unroll 1
  for (int r = 0; r < G.nact; r++) {
    double x = 0;
    for (int b = threadIdx.x; b < ntiles; b += kDslashThreads)
      x += ((volatile double *)G.partials)[(size_t)b * G.nact + r];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    __syncthreads();
    if (lane == 0) red[warp] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
      double tot = 0;
      for (int w = 0; w < kDslashThreads / 32; w++) tot += red[w];
      CGState *st = &states[G.state0 + r];
      if (((volatile CGState *)st)->status == ST_RUNNING) {
        if (role == ROLE_K1) finalize_pAp(st, tot);
        else finalize_rr(st, tot);
      }
    }
  }
  if (threadIdx.x == 0) *G.counter = 0u;
  return true;
}

template <int ROLE, int PHM>
__global__ void __launch_bounds__(kDslashThreads, LMB_PAIR_MINB)
    batch_half_pair_kernel(const BatchGroup *groups, int ngroups, int ntasks_total, CGState *states) {
  constexpr int DAG = ROLE == ROLE_K2 ? 1 : 0;
  for (int task = blockIdx.x; task < ntasks_total; task += gridDim.x) {
    const int gi = find_group(groups, ngroups, task);
    const BatchGroup &G = groups[gi];
    const int local = task - G.first_task;
    const int tg = local / G.nact, r = local - tg * G.nact;
    const Geom &g = G.g;
    const int npairs = (int)(g.V >> 1), ntg = G.ntasks / G.nact;
    const bool running = ((volatile CGState *)states)[G.state0 + r].status == ST_RUNNING;  // uniform
    const Field<PREC_HALF, 12> in =
        ROLE == ROLE_K1 ? bfield<PREC_HALF>(G.p[r], G.pn[r], g.V) : bfield<PREC_HALF>(G.t[r], G.tn[r], g.V);
    const Gauge12<PREC_HALF> U{G.Uh, g.V, 1.f};
    const float kappa = (float)G.kappa;
    double n2 = 0.0;
#pragma unroll 1
    for (int tt = 0; tt < kPairTilesPerTask; tt++) {
      const int i = (tg * kPairTilesPerTask + tt) * kDslashThreads + threadIdx.x;
      const bool active = running && i < npairs;
      const int s0 = 2 * i;
      if (active) {
        Cx2 out[12];
        half_adj_sites<DAG, false, PHM>(g, s0, in, U, NoClover{g.V}, kappa, out);
        float2 q = f2(0.f);
        if (ROLE == ROLE_K1) {
          store_adj(bfield<PREC_HALF>(G.t[r], G.tn[r], g.V), s0, out);
#pragma unroll
          for (int k = 0; k < 12; k++) q = norm2_acc(out[k], q);
        } else {
          const float a = (float)states[G.state0 + r].alpha;
          const float2 pa = f2(a), na = f2(-a);
          const Field<PREC_HALF, 12> pf = bfield<PREC_HALF>(G.p[r], G.pn[r], g.V);
          const Field<PREC_HALF, 12> rf = bfield<PREC_HALF>(G.r[r], G.rn[r], g.V);
          const Field<PREC_SINGLE, 12> xf{G.xl[r], nullptr, g.V};
          Cx2 pv[12], rv[12], xv[12];
          load_adj_rw(pf, s0, pv);
          load_adj_rw(rf, s0, rv);
          load_adj_rw(xf, s0, xv);
#pragma unroll
          for (int k = 0; k < 12; k++) {
            rv[k] = Cx2(fma2(na, out[k].re, rv[k].re), fma2(na, out[k].im, rv[k].im));
            xv[k] = Cx2(fma2(pa, pv[k].re, xv[k].re), fma2(pa, pv[k].im, xv[k].im));
            q = norm2_acc(rv[k], q);
          }
          store_adj(rf, s0, rv);
          store_adj(xf, s0, xv);
        }
        n2 += (double)q.x + (double)q.y;
      }
    }
    pair_task_done(G, local, n2, ntg, states, ROLE);
    __syncthreads();  // the next task's status read follows this task's finalize
  }
}

// K3 of the pair family: p = r + beta p on the task's tile group (pairs, 256-bit)
__global__ void __launch_bounds__(kDslashThreads)
    batch_half_pair_p_kernel(const BatchGroup *groups, int ngroups, int ntasks_total, const CGState *states) {
  for (int task = blockIdx.x; task < ntasks_total; task += gridDim.x) {
    const int gi = find_group(groups, ngroups, task);
    const BatchGroup &G = groups[gi];
    const int local = task - G.first_task;
    const int tg = local / G.nact, r = local - tg * G.nact;
    const CGState &st = states[G.state0 + r];
    if (((volatile const CGState *)&st)->status != ST_RUNNING) continue;
    const float2 beta = f2((float)st.beta);
    const Field<PREC_HALF, 12> pf = bfield<PREC_HALF>(G.p[r], G.pn[r], G.g.V);
    const Field<PREC_HALF, 12> rf = bfield<PREC_HALF>(G.r[r], G.rn[r], G.g.V);
#pragma unroll 1
    for (int tt = 0; tt < kPairTilesPerTask; tt++) {
      const int i = (tg * kPairTilesPerTask + tt) * kDslashThreads + threadIdx.x;
      if (i >= (int)(G.g.V >> 1)) break;
      const int s0 = 2 * i;
      Cx2 pv[12], rv[12];
      load_adj_rw(pf, s0, pv);
      load_adj_rw(rf, s0, rv);
#pragma unroll
      for (int k = 0; k < 12; k++) pv[k] = Cx2(fma2(beta, pv[k].re, rv[k].re), fma2(beta, pv[k].im, rv[k].im));
      store_adj(pf, s0, pv);
    }
  }
}

}  // namespace lmb
