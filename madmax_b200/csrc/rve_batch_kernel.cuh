// rve_batch_kernel.cuh -- the batched persistent kernel (see rve_batch.cu),
// in a header so that its instantiations compile in parallel translation
// units (rve_batch_inst_*.cu).
#pragma once

#include "rve_solve.cuh"
#include "sp_cuda.h"

namespace sp {

// kernel operator variants: SP_OP_ELL, SP_OP_STENCIL, and the stencil under
// periodic boundary conditions
constexpr int SP_OP_STENCIL_PER = 2;

// whether a k_batch variant (FP32 or not, K load cases, kernel operator,
// 128 registers a thread) reads its stencil blocks from the pattern table,
// which it keeps in SP_PT_BYTES of dynamic shared memory; more than 6 load
// cases need the wide register budget
__host__ __device__ constexpr bool sp_batch_uses_ptable(bool fp32, int K, int op, bool wide = false) {
  return (op == SP_OP_STENCIL || op == SP_OP_STENCIL_PER) && fp32 && (K <= 6 || wide);
}

// Dynamic shared memory of a k_batch variant: the pattern table or nothing.
__host__ __device__ constexpr int sp_batch_dyn_smem(bool fp32, int K, int op, bool wide) {
  return sp_batch_uses_ptable(fp32, K, op, wide) ? SP_PT_BYTES : 0;
}

struct BatchPlan {
  MeshGeo geo; // node/element counts; h and vol per RVE
  const int *cols;
  const int *nbr;
  const uint8_t *slot;
  const int *color_elems;
  int color_off[9];
};

struct BatchRve {
  int plan, pad;
  double len[3];
  long long nsv_off, etype_off, dinv_off;
};

struct BatchParams {
  const BatchPlan *plans;
  const BatchRve *rves;
  const int *order;
  int nrve, nrhs;
  void *nsv;   // float or double pool: node-sliced ELL values per RVE
  void *dinv;  // float or double pool: component-major Jacobi diagonal per RVE
  const uint8_t *etype;
  const double *strains; // [nrve][nrhs][6]
  const double *mats;    // [nrve][4]
  double *out_stress;    // [nrve][nrhs][6]
  double *out_strain;
  sp_solve_info *out_info;
  double *ws_u;          // per CTA [K][3][max nn_pad] FP64
  void *ws_v;            // per CTA 4 x [K][3][max nn_pad] of T: r, x, p, q
  size_t ws_stride;      // K*3*max nn_pad
  size_t drm_stride;     // 3*max nn_pad
  void *ws_dinv;         // stencil operator: per CTA Jacobi diagonal [3][max nn_pad] of T
  int *counter;
  double rtol, inner_rtol;
  int max_outer, max_inner;
};

template <typename T, int K, int NT, int MINB, int CL, int OP>
__global__ void __launch_bounds__(NT, MINB) k_batch(BatchParams P) {
  constexpr bool PER = OP == SP_OP_STENCIL_PER;
  constexpr bool STENCIL = OP == SP_OP_STENCIL || PER;
  // FP32 stencil under Dirichlet conditions: pattern table in dynamic shared memory
  constexpr bool WIDE = NT * MINB <= 512;  // 128 registers a thread
  constexpr bool PT = sp_batch_uses_ptable(sizeof(T) == 4, K, OP, WIDE);
  __shared__ double sKe[2 * SP_KE];
  // FP64 stencil tables for the residual (an FP64 stencil batch has them in sKeT already)
  constexpr bool OWN_KBD = !PER && !(STENCIL && sizeof(T) == 8);
  __shared__ __align__(16) double sKBd[OWN_KBD ? SP_KB_SIZE : 2];
  // element blocks (stencil without the pattern table)
  __shared__ __align__(16) T sKeT[(STENCIL && !PT) ? SP_KB_SIZE : 4];
  extern __shared__ __align__(16) float s_ptab[];  // SP_PT_BYTES when PT
  __shared__ double sD[72], sBbar[144], sdsh[192];
  // block_sum<NV> needs 33*NV doubles; NV is at most max(2K, 12) <= 16
  __shared__ double red[33 * 16];
  __shared__ double savg[SP_MAX_RHS * 12];
  __shared__ CgShared sh;
  __shared__ double seps[SP_MAX_RHS * 6];
  __shared__ int s_job;
  const int t = threadIdx.x;
  const int rank = rve_rank<CL>();
  const int gt = rank * NT + t;
  constexpr int GNT = CL * NT;
  const int slot = blockIdx.x / CL;  // work space of this cluster
  if constexpr (PT) {
    // launched without the pattern table's shared memory: solve nothing,
    // mark every RVE this CTA would have taken as failed
    if (dynamic_smem_bytes() < (unsigned)SP_PT_BYTES) {
      if (t == 0 && rank == 0)
        for (int job = slot; job < P.nrve; job += gridDim.x / CL) {
          sp_solve_info bad = {};
          bad.status = SP_ERR_STATE;
          P.out_info[P.order[job]] = bad;
        }
      return;
    }
  }
  double *u = P.ws_u + (size_t)slot * P.ws_stride;
  T *ws = reinterpret_cast<T *>(P.ws_v) + (size_t)slot * 4 * P.ws_stride;
  T *r = ws, *x = ws + P.ws_stride, *p = ws + 2 * P.ws_stride, *q = ws + 3 * P.ws_stride;

  for (;;) {
    // rank 0 claims the next RVE and hands it to the cluster
    if (t == 0 && rank == 0) {
      int job = atomicAdd(P.counter, 1);
      if constexpr (CL == 1) {
        s_job = job;
      } else {
        cg::cluster_group cl = cg::this_cluster();
        for (int rr = 0; rr < CL; rr++) *cl.map_shared_rank(&s_job, rr) = job;
      }
    }
    rve_sync<CL>();
    int job = s_job;
    rve_sync<CL>();
    if (job >= P.nrve) break;
    const int rid = P.order[job];
    const BatchRve rv = P.rves[rid];
    const BatchPlan pl = P.plans[rv.plan];
    MeshGeo g = pl.geo;
    g.hx = rv.len[0] / g.nex;
    g.hy = rv.len[1] / g.ney;
    g.hz = rv.len[2] / g.nez;
    g.vol = rv.len[0] * rv.len[1] * rv.len[2];
    g.periodic = PER ? 1 : 0;
    const uint8_t *etype = P.etype + rv.etype_off;

    // 1. element operators (every CTA keeps its own copy)
    if (t < 2) iso_D(P.mats[rid * 4 + 2 * t], P.mats[rid * 4 + 2 * t + 1], sD + 36 * t);
    double h[3] = {g.hx, g.hy, g.hz};
    elem_ops_stage1(t, NT, h, sdsh);
    __syncthreads();
    elem_ops_stage2(t, NT, h, sdsh, sD, 2, sKe, sBbar);
    __syncthreads();
    if constexpr (OWN_KBD) stencil_blocks<double>(t, NT, sKe, sKBd);
    T *nsv = nullptr, *dinv;
    if constexpr (STENCIL) {
      // 2s. no assembly: the stencil block tables and the Jacobi diagonal
      dinv = reinterpret_cast<T *>(P.ws_dinv) + (size_t)slot * P.drm_stride;
      if constexpr (PT)
        stencil_ptable(t, NT, sKe, s_ptab);
      else
        stencil_blocks<T>(t, NT, sKe, sKeT);
      if constexpr (PER)
        stencil_dinv_per<T>(gt, GNT, g, etype, sKe, dinv);
      else
        stencil_dinv<T>(gt, GNT, g, etype, sKe, dinv);
    } else {
      nsv = reinterpret_cast<T *>(P.nsv) + rv.nsv_off;
      dinv = reinterpret_cast<T *>(P.dinv) + rv.dinv_off;
      // 2. assembly: every node-sliced block summed by its owner thread from
      //    the element matrices (FP64, one rounding), Dirichlet applied
      ns_from_elements<T>(gt, GNT, g, pl.cols, pl.nbr, etype, sKe, nsv, dinv);
    }
    if constexpr (PER) {
      // load cases: the fluctuation starts at 0; eps enters residual and averages
      for (int i = t; i < SP_MAX_RHS * 6; i += NT)
        seps[i] = (i < P.nrhs * 6) ? P.strains[(size_t)rid * P.nrhs * 6 + i] : 0.0;
      for (size_t i = gt; i < (size_t)K * 3 * g.nn_pad; i += GNT) u[i] = 0.0;
    } else {
      // load cases: u = eps . x at every node, the homogeneous affine field
      // (the start iterate; the boundary values stay)
      affine_soa<K>(gt, GNT, g, P.strains + (size_t)rid * P.nrhs * 6, P.nrhs, false, u, true);
    }
    rve_sync<CL>();

    SolveArgs sa;
    sa.nrhs = P.nrhs;
    sa.rtol = P.rtol;
    sa.rtol_refine = P.rtol;
    sa.rn0_given = nullptr;
    sa.kbd = PER ? nullptr : (OWN_KBD ? sKBd : reinterpret_cast<const double *>(sKeT));
    sa.inner_rtol = P.inner_rtol;
    sa.max_outer = P.max_outer;
    sa.max_inner = P.max_inner;
    // affine conditions start from the affine field, measured against the
    // right-hand side of the boundary values alone (one extra residual);
    // the periodic fluctuation starts at 0, which is the affine field too
    sa.warm = PER ? 0 : 1;
    sa.eps = seps;
    sp_solve_info in;
    if constexpr (STENCIL) {
      StencilOp<T, K, PER, PT, WIDE> op{PT ? reinterpret_cast<const T *>(s_ptab) : sKeT, etype};
      in = solve_rve<T, K, NT, CL, decltype(op), WIDE>(g, op, dinv, etype, sKe, sD, sBbar, u, r,
                                                       x, p, q, sa, red, &sh, savg);
    } else {
      EllOp<T, K> op{nsv, pl.nbr};
      in = solve_rve<T, K, NT, CL, decltype(op), WIDE>(g, op, dinv, etype, sKe, sD, sBbar, u, r,
                                                       x, p, q, sa, red, &sh, savg);
    }
    if (t == 0 && rank == 0) {
      for (int qq = 0; qq < P.nrhs; qq++) {
        size_t o = ((size_t)rid * P.nrhs + qq) * 6;
        for (int v = 0; v < 6; v++) {
          if (P.out_strain) P.out_strain[o + v] = savg[qq * 12 + v];
          P.out_stress[o + v] = savg[qq * 12 + 6 + v];
        }
      }
      P.out_info[rid] = in;
    }
    rve_sync<CL>();
  }
}

using BatchFn = void (*)(BatchParams);

// the instantiated shapes: (threads, min CTAs per SM, cluster, operator)
#define SP_BATCH_SHAPES(X, T, K) \
  X(T, K, 512, 1, 1, SP_OP_ELL) X(T, K, 512, 2, 1, SP_OP_ELL) X(T, K, 256, 2, 1, SP_OP_ELL) \
  X(T, K, 256, 4, 1, SP_OP_ELL) X(T, K, 512, 1, 2, SP_OP_ELL) X(T, K, 512, 2, 2, SP_OP_ELL) \
  X(T, K, 512, 1, 4, SP_OP_ELL) X(T, K, 512, 2, 4, SP_OP_ELL) X(T, K, 512, 1, 8, SP_OP_ELL) \
  X(T, K, 512, 2, 8, SP_OP_ELL) \
  X(T, K, 512, 1, 1, SP_OP_STENCIL) X(T, K, 512, 2, 1, SP_OP_STENCIL) \
  X(T, K, 256, 2, 1, SP_OP_STENCIL) X(T, K, 256, 4, 1, SP_OP_STENCIL) \
  X(T, K, 1024, 1, 1, SP_OP_STENCIL) X(T, K, 1024, 1, 2, SP_OP_STENCIL) \
  X(T, K, 1024, 1, 4, SP_OP_STENCIL) X(T, K, 1024, 1, 8, SP_OP_STENCIL) \
  X(T, K, 512, 1, 1, SP_OP_STENCIL_PER) X(T, K, 512, 2, 1, SP_OP_STENCIL_PER)
#define SP_BATCH_SHAPES_FP64(X, T, K) \
  X(T, K, 512, 1, 1, SP_OP_ELL) X(T, K, 512, 2, 1, SP_OP_ELL) \
  X(T, K, 512, 1, 1, SP_OP_STENCIL) X(T, K, 512, 2, 1, SP_OP_STENCIL) \
  X(T, K, 512, 1, 1, SP_OP_STENCIL_PER) X(T, K, 512, 2, 1, SP_OP_STENCIL_PER)

#define SP_BATCH_EXTERN(T, K, NT, MINB, CL, OP) \
  extern template __global__ void k_batch<T, K, NT, MINB, CL, OP>(BatchParams);
#define SP_BATCH_DEFINE(T, K, NT, MINB, CL, OP) \
  template __global__ void k_batch<T, K, NT, MINB, CL, OP>(BatchParams);

}  // namespace sp
