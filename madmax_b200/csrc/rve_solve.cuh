// rve_solve.cuh -- the per-RVE solve shared by the batched kernel
// (rve_batch.cu) and the serving loop (serve.cu): FP64 element residual
// (micro/src/assembly.c:33-82), Jacobi-PCG corrections in precision T on
// the RVE's operator (assembled or stencil), FP64 update of u (micro/src/
// homogenize.c:184-215, with a relative stopping rule) and FP64 volume
// averages (micro/src/homogenize.c:344-368).
//
// One RVE is solved by a thread-block cluster of CL CTAs of NT threads
// (CL = 1: a single CTA, no cluster instructions).  Every loop is split over
// the cluster's CL*NT threads; partial sums are reduced in each CTA, then
// added across the cluster through distributed shared memory in rank order,
// so every CTA holds the same totals and computes the same CG scalars
// (deterministic, independent of scheduling).  Cluster barriers separate
// the phases in which a CTA reads rows another CTA wrote (the SpMM gathers,
// the residual gathers of u).  Vectors are component-major,
// v[(k*3 + d)*nn_pad + node], padding nodes zero; the stencil operator's
// input p is node-blocked (nbk_base).  The corrections are reliable updates
// of one CG recurrence: each refinement step replaces r by the true FP64
// residual and keeps the search direction.
#pragma once

#include <cooperative_groups.h>

#include "rve_device.cuh"

namespace sp {

namespace cg = cooperative_groups;

// A right-hand side whose norm is at most this fraction of the norm of its
// summed term magnitudes is cancellation round-off of an exactly zero one.
constexpr double SP_RHS_FLOOR = 1e-12;

// A correction that would take the residual to the final target ends at
// this fraction of it, so that the FP64 residual after the update meets the
// target with a margin.
constexpr double SP_FINAL_MARGIN = 0.5;

struct SolveArgs {
  int nrhs;
  double rtol, inner_rtol;
  int max_outer, max_inner;
  int warm;  // u's interior holds a start iterate other than 0
  double rtol_refine;  // target once a refinement step has run (<= rtol): a start
                       // iterate that already meets rtol is accepted as it is
  const double *rn0_given;  // warm start: the right-hand sides' norms [K] when the
                            // caller knows them (else one boundary-only residual)
  const double *kbd;  // FP64 stencil tables in shared memory (stencil_blocks<double>):
                      // the Dirichlet residual in stencil form; null: element form
  const double *eps;  // periodic conditions: [K][6] strains of the load cases (shared)
};

struct CgShared {
  double rn0[SP_MAX_RHS], rn[SP_MAX_RHS], rho[SP_MAX_RHS];
  double alpha[SP_MAX_RHS], beta[SP_MAX_RHS];
  double thr[SP_MAX_RHS];  // inner CG: r.r at which a load case's correction ends
  int act[SP_MAX_RHS];
  int keep[SP_MAX_RHS];    // load case k continues the last correction's direction
  int nact, done;
  unsigned amask;  // bit k: load case k still active in the inner CG
  // cluster reduction: [buffer][rank][value], written by every rank into
  // rank 0's copy
  double cpart[2][8][16];
  int phase;
};

// The right-hand side of the boundary values alone and its norms, once per
// RVE: kept out of line, so that its registers do not add to the CG loop's.
template <int K, typename T>
__device__ __noinline__ void rhs_stencil(int gt, int gnt, const MeshGeo &g,
                                         const uint8_t *__restrict__ etype, const double *kbd,
                                         const double *__restrict__ u, T *r, double *nrm2,
                                         double *scale2) {
  residual_stencil<K, T, true, true>(gt, gnt, g, etype, kbd, u, r, nrm2, scale2);
}

// Barrier over the threads that solve one RVE.
template <int CL>
__device__ inline void rve_sync() {
  if constexpr (CL == 1)
    __syncthreads();
  else
    cg::this_cluster().sync();
}

template <int CL>
__device__ inline int rve_rank() {
  if constexpr (CL == 1)
    return 0;
  else
    return (int)cg::this_cluster().block_rank();
}

// Sum NV per-thread partials over the CTA (and the cluster).  The totals
// end in red[32*NV + q] of every CTA, readable by warp 0; no trailing CTA
// barrier (the caller's warp-0 update follows, then a __syncthreads).
template <int NV, int CL>
__device__ inline void rve_reduce(const double *v, double *red, CgShared *sh) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; q++) {
    double w = v[q];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) w += __shfl_xor_sync(0xffffffffu, w, off);
    if (lane == 0) red[warp * NV + q] = w;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int q = 0; q < NV; q++) {
      double s = (lane < nw) ? red[lane * NV + q] : 0.0;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
      if (lane == 0) red[32 * NV + q] = s;
    }
    __syncwarp();
  }
  if constexpr (CL > 1) {
    cg::cluster_group cl = cg::this_cluster();
    const int ph = sh->phase;
    if (warp == 0 && lane < NV) {
      double *dst = cl.map_shared_rank(&sh->cpart[ph][cl.block_rank()][lane], 0);
      *dst = red[32 * NV + lane];
    }
    cl.sync();
    if (warp == 0 && lane < NV) {
      const double *src = cl.map_shared_rank(&sh->cpart[ph][0][0], 0);
      double s = 0.0;
      for (int r = 0; r < CL; r++) s += src[r * 16 + lane];
      red[32 * NV + lane] = s;
    }
    __syncwarp();
    if (threadIdx.x == 0) sh->phase = ph ^ 1;
  }
}

// The two operators the inner CG can apply: the node-sliced copy of the
// RVE's assembled ELL values, or the element-type stencil (no matrix in
// memory).  apply() computes q = A p and adds p.q per load case into dot.
template <typename T, int K>
struct EllOp {
  static constexpr bool kBlocked = false;  // p component-major
  const T *nsv;
  const int *nbr;
  __device__ void apply(int gt, int gnt, const MeshGeo &g, const T *p, T *q, double *dot,
                        unsigned, bool) const {
    spmm_ns<T, K, false>(gt, gnt, g, nsv, nbr, p, q, dot);
  }
};

// XO: the x-neighbour terms formed in the lane holding the values
// (spmm_stencil_xo), for up to 6 load cases in kernels with 128 registers a
// thread; its three accumulator sets spill heavily below that.
template <typename T, int K, bool PER = false, bool PT = false, bool XO = true>
struct StencilOp {
  static_assert(!PT || sizeof(T) == 4, "pattern tables serve the FP32 stencil");
  static constexpr bool kBlocked = true;  // p node-blocked (nbk_base)
  const T *kb;  // shared-memory blocks: stencil_blocks, or stencil_ptable when PT
  const uint8_t *etype;
  __device__ void apply(int gt, int gnt, const MeshGeo &g, const T *p, T *q, double *dot,
                        unsigned amask, bool rev) const {
    if constexpr (PT && !PER && K <= 6 && XO)
      spmm_stencil_xo<K>(gt, gnt, g, kb, etype, p, q, dot, amask, rev);
    else if constexpr (PT && !PER)
      spmm_stencil_xw<K>(gt, gnt, g, kb, etype, p, q, dot, amask, rev);
    else
      spmm_stencil<T, K, PER, PT>(gt, gnt, g, kb, etype, p, q, dot, amask, rev);
  }
};

// 16-byte vector of T
template <typename T>
struct V16 {
  static constexpr int E = 16 / sizeof(T);
  T v[E];
  __device__ static V16 load(const T *p) {
    V16 r;
    int4 w = *reinterpret_cast<const int4 *>(p);
    memcpy(r.v, &w, 16);
    return r;
  }
  __device__ void store(T *p) const {
    int4 w;
    memcpy(&w, v, 16);
    *reinterpret_cast<int4 *>(p) = w;
  }
};

// The two FP32 vector passes of a CG step, on 16-byte chunks in node order
// (chunk c at offset cm(c) + k*blk of load case k in the component-major
// vectors, pb(c) + k*pk in the operator's input p).  The vectors are
// distinct arrays (restrict-qualified), so the loads of every load case of a
// chunk may be issued before any of its stores.
//
// p = D^-1 r + beta p for the load cases in am; beta 0 starts afresh from
// D^-1 r without reading p (the work space may hold anything).
template <typename T, int K, typename W, typename CM, typename PB>
__device__ __forceinline__ void pass_dir(int gt, int gnt, int nch, bool rev, unsigned am,
                                         const T *be, size_t blk, size_t pk, CM cm, PB pb,
                                         const T *__restrict__ dinv, const T *__restrict__ r,
                                         T *__restrict__ p) {
  constexpr int E = W::E;
  for (int c0 = gt; c0 < nch; c0 += gnt) {
    const int c = rev ? nch - 1 - c0 : c0;
    const size_t oc = cm(c), op_ = pb(c);
    const W dv = W::load(dinv + oc);
#pragma unroll
    for (int k = 0; k < K; k++) {
      if (!((am >> k) & 1u)) continue;
      const size_t o = (size_t)k * blk + oc, opk = op_ + k * pk;
      const W rv = W::load(r + o);
      W pv;
      if (be[k] == T(0)) {
#pragma unroll
        for (int e = 0; e < E; e++) pv.v[e] = dv.v[e] * rv.v[e];
      } else {
        pv = W::load(p + opk);
#pragma unroll
        for (int e = 0; e < E; e++) pv.v[e] = dv.v[e] * rv.v[e] + be[k] * pv.v[e];
      }
      pv.store(p + opk);
    }
  }
}

// x += alpha p, r -= alpha q for the load cases in am; adds r.z and r.r
// (z = D^-1 r) per load case into m2[k] and m2[K + k].
template <typename T, int K, typename W, typename CM, typename PB>
__device__ __forceinline__ void pass_xr(int gt, int gnt, int nch, bool rev, unsigned am,
                                        const T *al, size_t blk, size_t pk, CM cm, PB pb,
                                        const T *__restrict__ dinv, T *__restrict__ x,
                                        const T *__restrict__ p, T *__restrict__ r,
                                        const T *__restrict__ q, double *m2) {
  constexpr int E = W::E;
  for (int c0 = gt; c0 < nch; c0 += gnt) {
    const int c = rev ? nch - 1 - c0 : c0;
    const size_t oc = cm(c), op_ = pb(c);
    const W dv = W::load(dinv + oc);
#pragma unroll
    for (int k = 0; k < K; k++) {
      if (!((am >> k) & 1u)) continue;
      const size_t o = (size_t)k * blk + oc;
      W xv = W::load(x + o), pv = W::load(p + op_ + k * pk), rv = W::load(r + o),
        qv = W::load(q + o);
#pragma unroll
      for (int e = 0; e < E; e++) {
        xv.v[e] += al[k] * pv.v[e];
        rv.v[e] -= al[k] * qv.v[e];
        m2[k] += (double)rv.v[e] * (double)(dv.v[e] * rv.v[e]);
        m2[K + k] += (double)rv.v[e] * (double)rv.v[e];
      }
      xv.store(x + o);
      rv.store(r + o);
    }
  }
}

// On entry u holds the start iterate with the boundary values of every load
// case (visible to the whole cluster).  On exit avg[q*12 + 0..5] =
// <strain>_q, avg[q*12 + 6..11] = <stress>_q (q < nrhs, shared memory of
// every CTA) and the return value describes the solve.  red: shared scratch
// of 33*16 doubles; sh: shared CG scalars.
// WIDE: the kernel has 128 registers a thread (at most 512 threads per SM),
// room for the per-node FP64 residual.
template <typename T, int K, int NT, int CL, typename Op, bool WIDE = false>
__device__ sp_solve_info solve_rve(const MeshGeo &g, const Op &op, const T *dinv,
                                   const uint8_t *etype, const double *sKe, const double *sD,
                                   const double *sBbar, double *u, T *r, T *x, T *p, T *q,
                                   const SolveArgs &P, double *red, CgShared *sh, double *avg) {
  using W = V16<T>;
  constexpr int E = W::E;
  const int t = threadIdx.x;
  const int lane = t & 31, warp = t >> 5;
  const int gt = rve_rank<CL>() * NT + t;  // index among the RVE's threads
  constexpr int GNT = CL * NT;
  const int blk = 3 * g.nn_pad;  // values per load case
  const int nch = blk / E;       // 16-byte chunks per load case
  if (t < SP_MAX_RHS) {
    sh->rn0[t] = 0.0;
    sh->act[t] = 0;
    sh->keep[t] = 0;
  }
  if (t == 0) sh->phase = 0;
  int outer = 0, inner = 0;
  rve_sync<CL>();
  if (P.warm && P.rn0_given) {
    if (t < K) sh->rn0[t] = (t < P.nrhs) ? P.rn0_given[t] : 0.0;
    __syncthreads();
    for (int k = 0; k < P.nrhs; k++) {
      if (sh->rn0[k] > 0.0) continue;
      for (int idx = gt; idx < blk; idx += GNT)
        if (idx % g.nn_pad < g.nn && !is_bnode(g, idx % g.nn_pad)) u[(size_t)k * blk + idx] = 0.0;
    }
    rve_sync<CL>();
  } else if (P.warm) {
    // The stopping rule is relative to the right-hand side, the residual of
    // the boundary values alone (not to the residual of the start iterate,
    // which a good warm start makes tiny).  A load case whose right-hand
    // side vanishes (is round-off of cancelling terms) has the solution 0
    // inside.
    double m0[2 * K];
#pragma unroll
    for (int k = 0; k < 2 * K; k++) m0[k] = 0.0;
    if (P.kbd)  // Dirichlet stencil tables: 27 instead of 64 neighbour reads per row
      rhs_stencil<K, T>(gt, GNT, g, etype, P.kbd, u, r, m0, m0 + K);
    else
      residual_soa<K, T, true, true>(gt, GNT, g, etype, sKe, u, r, m0, m0 + K);
    rve_reduce<2 * K, CL>(m0, red, sh);
    if (warp == 0 && lane < K) {
      const double rn = sqrt(red[64 * K + lane]), sc = sqrt(red[64 * K + K + lane]);
      sh->rn0[lane] = (rn <= SP_RHS_FLOOR * sc) ? 0.0 : rn;
    }
    __syncthreads();
    for (int k = 0; k < P.nrhs; k++) {
      if (sh->rn0[k] > 0.0) continue;
      for (int idx = gt; idx < blk; idx += GNT)
        if (idx % g.nn_pad < g.nn && !is_bnode(g, idx % g.nn_pad)) u[(size_t)k * blk + idx] = 0.0;
    }
    rve_sync<CL>();
  }
  // The vector passes walk 16-byte chunks in node order: chunk c covers E
  // nodes of stream segment sg = c / CPB (32 nodes of component d), whose
  // offset is cm(c) + k*blk for load case k in the component-major vectors
  // and pb(c) + k*32 in a node-blocked p (the stencil operator's input).
  constexpr int CPB = 32 / E;
  auto cm = [&](int c) -> size_t {
    const int sg = c / CPB, b = sg / 3, d = sg - 3 * b;
    return (size_t)d * g.nn_pad + b * 32 + (c - sg * CPB) * E;
  };
  auto pb = [&](int c) -> size_t {
    const int sg = c / CPB;
    return Op::kBlocked ? (size_t)sg * (32 * K) + (c - sg * CPB) * E : cm(c);
  };
  const size_t pk = Op::kBlocked ? 32 : blk;  // p offset between load cases
  // Consecutive passes over the vectors walk the nodes in opposite
  // directions, so each pass starts on the lines the previous one touched
  // last, which are still in L2.
  int npass = 0;
  // p = D^-1 r + beta p for the active load cases, chunk-major: the diagonal
  // is read once per chunk and the load cases' loads are independent
  auto pdir = [&](unsigned am) {
    T be[K];
#pragma unroll
    for (int k = 0; k < K; k++) be[k] = (T)sh->beta[k];
    const bool rev = (npass++ & 1) != 0;
    pass_dir<T, K, W>(gt, GNT, nch, rev, am, be, blk, pk, cm, pb, dinv, r, p);
  };
  for (;;) {
    // 3a. FP64 residual b = -K u -> r (type T) and its norms; on a cold
    // start the first one is the right-hand side, whose norm the later
    // ones are measured against (a right-hand side at the round-off level
    // of its own cancelling terms is zero: that load case is solved)
    {
      const bool first = outer == 0 && !P.warm;
      double m1[2 * K];
#pragma unroll
      for (int k = 0; k < 2 * K; k++) m1[k] = 0.0;
      if (g.periodic) {
        if (first)
          residual_per<K, T, true>(gt, GNT, g, etype, sKe, P.eps, u, r, m1, m1 + K);
        else
          residual_per<K, T>(gt, GNT, g, etype, sKe, P.eps, u, r, m1);
      } else if (P.kbd) {
        if (first)
          residual_stencil<K, T, true>(gt, GNT, g, etype, P.kbd, u, r, m1, m1 + K);
        else
          if constexpr (WIDE)
            residual_stencil_node<K, T>(gt, GNT, g, etype, P.kbd, u, r, m1);
          else
            residual_stencil<K, T>(gt, GNT, g, etype, P.kbd, u, r, m1);
      } else {
        if (first)
          residual_soa<K, T, false, true>(gt, GNT, g, etype, sKe, u, r, m1, m1 + K);
        else
          residual_soa<K, T>(gt, GNT, g, etype, sKe, u, r, m1);
      }
      if (first)
        rve_reduce<2 * K, CL>(m1, red, sh);
      else
        rve_reduce<K, CL>(m1, red, sh);
      const int tot = first ? 64 * K : 32 * K;  // where rve_reduce left the totals
      if (warp == 0) {
        bool notdone = false;
        if (lane < K) {
          double rn = sqrt(red[tot + lane]);
          if (first) sh->rn0[lane] = (rn <= SP_RHS_FLOOR * sqrt(red[tot + K + lane])) ? 0.0 : rn;
          sh->rn[lane] = rn;
          double rn0 = sh->rn0[lane];
          const double target = (outer == 0) ? P.rtol : P.rtol_refine;
          notdone = lane < P.nrhs && rn0 > 0.0 && rn > target * rn0;
          sh->act[lane] = notdone;
        }
        unsigned b = __ballot_sync(0xffffffffu, notdone);
        if (lane == 0) {
          sh->nact = __popc(b);
          sh->done = (b == 0) || outer >= P.max_outer;
        }
      }
      __syncthreads();
    }
    if (sh->done) break;
    // 3b. Jacobi-PCG on A x = r in precision T with x = 0.  The search
    // direction carries over from the previous correction (a reliable
    // update: r is replaced by the true residual, the Krylov recurrence goes
    // on), p = D^-1 r + beta p with beta = r.z / rho of the last step; the
    // first correction, or a load case that sat out the last one, starts
    // from p = D^-1 r.  A correction ends when r.r has fallen by inner_rtol^2
    // or below SP_FINAL_MARGIN of the final target.
    {
      double m2[2 * K];
#pragma unroll
      for (int k = 0; k < 2 * K; k++) m2[k] = 0.0;
      W zero;
#pragma unroll
      for (int e = 0; e < E; e++) zero.v[e] = T(0);
      for (int c = gt; c < nch; c += GNT) {
        const W dv = W::load(dinv + (size_t)c * E);
#pragma unroll
        for (int k = 0; k < K; k++) {
          const size_t o = (size_t)k * blk + (size_t)c * E;
          const W rv = W::load(r + o);
#pragma unroll
          for (int e = 0; e < E; e++) {
            m2[k] += (double)rv.v[e] * (double)(dv.v[e] * rv.v[e]);
            m2[K + k] += (double)rv.v[e] * (double)rv.v[e];
          }
          zero.store(x + o);
          zero.store(q + o);  // (entries an operator does not write stay 0)
        }
      }
      rve_reduce<2 * K, CL>(m2, red, sh);
      if (warp == 0) {
        bool a = false;
        if (lane < K) {
          const double rz = red[64 * K + lane], rr = red[64 * K + K + lane];
          a = sh->act[lane] && rr > 0.0;
          const double rho = sh->rho[lane];
          sh->beta[lane] = (a && sh->keep[lane] && rho != 0.0) ? rz / rho : 0.0;
          sh->rho[lane] = rz;
          const double fin = SP_FINAL_MARGIN * P.rtol_refine * sh->rn0[lane];
          sh->thr[lane] = fmax(P.inner_rtol * P.inner_rtol * rr, fin * fin);
          sh->act[lane] = a;
          sh->keep[lane] = a;
        }
        unsigned b = __ballot_sync(0xffffffffu, a);
        if (lane == 0) {
          sh->nact = __popc(b);
          sh->amask = b;
        }
      }
      __syncthreads();
      pdir(sh->amask);
      rve_sync<CL>();  // the SpMM gathers p rows of every CTA
    }
    int it = 0;
    while (sh->nact > 0 && it < P.max_inner) {
      // q = A p, alpha = rho / p.q
      {
        double m3[K];
#pragma unroll
        for (int k = 0; k < K; k++) m3[k] = 0.0;
        op.apply(gt, GNT, g, p, q, m3, sh->amask, (npass++ & 1) != 0);
        rve_reduce<K, CL>(m3, red, sh);
        if (warp == 0 && lane < K) {
          double pq = red[32 * K + lane];
          sh->alpha[lane] = (sh->act[lane] && pq != 0.0) ? sh->rho[lane] / pq : 0.0;
        }
        __syncthreads();
      }
      // x += alpha p, r -= alpha q; r.z, r.r
      {
        double m2[2 * K];
#pragma unroll
        for (int k = 0; k < 2 * K; k++) m2[k] = 0.0;
        // chunk-major: the diagonal is read once per chunk and the K load
        // cases' loads of one chunk are independent of each other
        T al[K];
#pragma unroll
        for (int k = 0; k < K; k++) al[k] = (T)sh->alpha[k];
        const unsigned am = sh->amask;  // converged load cases are left as they are
        const bool rev = (npass++ & 1) != 0;
        pass_xr<T, K, W>(gt, GNT, nch, rev, am, al, blk, pk, cm, pb, dinv, x, p, r, q, m2);
        rve_reduce<2 * K, CL>(m2, red, sh);
        if (warp == 0) {
          bool a = false;
          if (lane < K) {
            double rz = red[64 * K + lane], rr = red[64 * K + K + lane];
            a = sh->act[lane] && !(rr <= sh->thr[lane]);
            double rho = sh->rho[lane];
            sh->beta[lane] = (a && rho != 0.0) ? rz / rho : 0.0;
            if (a) sh->rho[lane] = rz;
            sh->act[lane] = a;
          }
          unsigned b = __ballot_sync(0xffffffffu, a);
          if (lane == 0) {
            sh->nact = __popc(b);
            sh->amask = b;
          }
        }
        __syncthreads();
      }
      it++;
      if (sh->nact == 0) break;
      // p = D^-1 r + beta p
      pdir(sh->amask);
      rve_sync<CL>();  // the next SpMM gathers p rows of every CTA
    }
    inner += it;
    // 3c. u += x in FP64
    for (int i = gt; i < K * blk; i += GNT) u[i] += (double)x[i];
    rve_sync<CL>();  // the residual gathers u rows of every CTA
    outer++;
  }

  // 4. averages per load case
  for (int qq = 0; qq < P.nrhs; qq++) {
    double acc[12];
#pragma unroll
    for (int v = 0; v < 12; v++) acc[v] = 0.0;
    if (g.periodic)
      average_per(gt, GNT, g, etype, sD, sBbar, P.eps + qq * 6, u, qq, acc);
    else
      average_soa(gt, GNT, g, etype, sD, sBbar, u, qq, acc);
    rve_reduce<12, CL>(acc, red, sh);
    if (t == 0)
      for (int v = 0; v < 12; v++) avg[qq * 12 + v] = red[32 * 12 + v] / g.vol;
    __syncthreads();
  }
  double worst = 0.0;
  for (int k = 0; k < P.nrhs; k++)
    if (sh->rn0[k] > 0.0) worst = fmax(worst, sh->rn[k] / sh->rn0[k]);
  rve_sync<CL>();
  sp_solve_info in;
  in.status = (worst <= P.rtol) ? SP_OK : SP_ERR_NOCONV;
  in.outer_its = outer;
  in.inner_its = inner;
  in.pad = 0;
  in.relres = worst;
  return in;
}

}  // namespace sp
