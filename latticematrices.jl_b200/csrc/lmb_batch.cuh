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
// Every right-hand side runs its own CG (cg.jl:73-137) with device-resident
// scalars (CGState); a right-hand side that has finished or paused for a
// reliable update is skipped by all later kernels while the others go on.
// Reductions are per task (NB partial sums), and the last task of a group to
// finish reduces the group's partials and updates the NB states.
#pragma once
#include "lmb_solver.cuh"

namespace lmb {

constexpr int kMaxNB = 4;

struct BatchGroup {
  Geom g;
  const void *U;       // reconstruct-12 links: float4 (FP32 kernels) / double2 (FP64 kernels)
  const void *U64;     // FP64 reconstruct-12 links
  int nact;            // right-hand sides in the group (<= NB)
  int first_task;      // first task of the group in the work list
  int ntasks;          // tasks of the group (sites / NT rounded up)
  int state0;          // CGState index of the group's first right-hand side
  double kappa;
  float4 *p[kMaxNB], *t[kMaxNB], *r[kMaxNB], *xl[kMaxNB];        // FP32 fields
  double2 *b64[kMaxNB], *x64[kMaxNB], *r64[kMaxNB], *t64[kMaxNB];  // FP64 fields
  double *partials;    // ntasks * NB
  unsigned *counter;
  unsigned mask;       // FP64 passes: right-hand sides to process (bit per member)
  int mode;            // finalize_true mode of the FP64 true-residual pass
};

enum BatchRole { ROLE_K1 = 0, ROLE_K2 = 1, ROLE_D64 = 2, ROLE_TRUE = 3 };

LMB_D int find_group(const BatchGroup *groups, int ngroups, int task) {
  int lo = 0, hi = ngroups - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (groups[mid].first_task <= task) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// FP32 stencil for NB right-hand sides sharing the link loads
template <int DAG, int MU, int NB, class G>
LMB_D void hop_dir_multi(const Geom &g, int s, const int *c, const Field<PREC_SINGLE, 12> *in, const bool *on,
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
template <int NT, int NB, int ROLE>
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
    Field<PREC_SINGLE, 12> in[NB];
#pragma unroll
    for (int r = 0; r < NB; r++) {
      in[r].data = ROLE == ROLE_K1 ? G.p[r] : G.t[r];
      in[r].norm = nullptr;
      in[r].V = g.V;
    }
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
          Field<PREC_SINGLE, 12> t{G.t[r], nullptr, g.V};
          t.store(s, v);
          n2[r] = sum_norm2(v, 12);
        } else {
          const float alpha = (float)states[G.state0 + r].alpha;
          Field<PREC_SINGLE, 12> pf{G.p[r], nullptr, g.V}, rf{G.r[r], nullptr, g.V}, xf{G.xl[r], nullptr, g.V};
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
// ROLE_TRUE r64 = b64 - D^+ t64, r (FP32) = r64, |r64|^2 -> finalize_true
template <int NT, int NB, int ROLE>
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
    double n2[NB], tot[NB];
    const Gauge12<PREC_DOUBLE> U{(const double2 *)G.U64, g.V, 1.f};
#pragma unroll
    for (int r = 0; r < NB; r++) {
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
        Field<PREC_SINGLE, 12> rl{G.r[r], nullptr, g.V};
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
      if (grid_reduce_slots<NT, NB>(n2, G.partials, G.counter, tot, (unsigned)local, (unsigned)G.ntasks) &&
          threadIdx.x == 0) {
#pragma unroll
        for (int r = 0; r < NB; r++)
          if (r < G.nact && ((G.mask >> r) & 1)) finalize_true(&states[G.state0 + r], tot[r], G.mode);
      }
      __syncthreads();
    }
  }
}

// K3 for all running members: p = r + beta p (FP32)
template <int NT, int NB>
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
      Field<PREC_SINGLE, 12> pf{G.p[r], nullptr, G.g.V}, rf{G.r[r], nullptr, G.g.V};
      Cx<float> pv[12], rv[12];
      pf.load(s, pv);
      rf.load(s, rv);
#pragma unroll
      for (int k = 0; k < 12; k++) pv[k] = rv[k] + beta * pv[k];
      pf.store(s, pv);
    }
  }
}

}  // namespace lmb
