// rve_solve.cuh -- the per-RVE solve shared by the batched kernel
// (rve_batch.cu) and the serving loop (serve.cu), run by one CTA of NT
// threads: FP64 element residual (micro/src/assembly.c:33-82), Jacobi-PCG
// corrections in precision T on the RVE's node-sliced ELL values, FP64
// update of u (micro/src/homogenize.c:184-215, with a relative stopping
// rule) and FP64 volume averages (micro/src/homogenize.c:344-368).
//
// The CG scalars of the K load cases live in shared memory (CgShared) and
// are updated by warp 0 inside each reduction, so the threads carry no
// per-load-case state across the loop.  Vectors are component-major,
// v[(k*3 + d)*nn_pad + node], padding nodes zero.
#pragma once

#include "rve_device.cuh"

namespace sp {

struct SolveArgs {
  int nrhs;
  double rtol, inner_rtol;
  int max_outer, max_inner;
};

struct CgShared {
  double rn0[SP_MAX_RHS], rn[SP_MAX_RHS], rho[SP_MAX_RHS], rr0[SP_MAX_RHS];
  double alpha[SP_MAX_RHS], beta[SP_MAX_RHS];
  int act[SP_MAX_RHS];
  int nact, done;
};

// Block reduction of NV partial sums; the totals are left in
// red[32*NV .. 33*NV) for warp 0 (no trailing barrier: the caller's update
// runs in warp 0 and then synchronises).
template <int NV>
__device__ inline void block_reduce_w0(const double *v, double *red) {
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
}

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

// On entry u holds the start iterate with the boundary values of every load
// case.  On exit avg[q*12 + 0..5] = <strain>_q, avg[q*12 + 6..11] =
// <stress>_q (q < nrhs, shared memory) and the return value describes the
// solve.  red: shared scratch of 33*16 doubles; sh: shared CG scalars.
template <typename T, int K, int NT>
__device__ sp_solve_info solve_rve(const MeshGeo &g, const T *nsv, const int *nbr, const T *dinv,
                                   const uint8_t *etype, const double *sKe, const double *sD,
                                   const double *sBbar, double *u, T *r, T *x, T *p, T *q,
                                   const SolveArgs &P, double *red, CgShared *sh, double *avg) {
  using W = V16<T>;
  constexpr int E = W::E;
  const int t = threadIdx.x;
  const int lane = t & 31, warp = t >> 5;
  const int blk = 3 * g.nn_pad;  // values per load case
  const int nch = blk / E;       // 16-byte chunks per load case
  if (t < SP_MAX_RHS) {
    sh->rn0[t] = 0.0;
    sh->act[t] = 0;
  }
  int outer = 0, inner = 0;
  __syncthreads();
  for (;;) {
    // 3a. FP64 residual b = -K u -> r (type T) and its norms
    {
      double m1[K];
#pragma unroll
      for (int k = 0; k < K; k++) m1[k] = 0.0;
      residual_soa<K, T>(t, NT, g, etype, sKe, u, r, m1);
      block_reduce_w0<K>(m1, red);
      if (warp == 0) {
        bool notdone = false;
        if (lane < K) {
          double rn = sqrt(red[32 * K + lane]);
          if (outer == 0) sh->rn0[lane] = rn;
          sh->rn[lane] = rn;
          double rn0 = sh->rn0[lane];
          notdone = lane < P.nrhs && rn0 > 0.0 && rn > P.rtol * rn0;
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
    // 3b. Jacobi-PCG on A x = r in precision T: x = 0, p = z = D^-1 r
    {
      double m2[2 * K];
#pragma unroll
      for (int k = 0; k < 2 * K; k++) m2[k] = 0.0;
#pragma unroll
      for (int k = 0; k < K; k++) {
        for (int c = t; c < nch; c += NT) {
          size_t o = (size_t)k * blk + (size_t)c * E;
          W rv = W::load(r + o), dv = W::load(dinv + (size_t)c * E), zv, zero;
#pragma unroll
          for (int e = 0; e < E; e++) {
            zv.v[e] = dv.v[e] * rv.v[e];
            zero.v[e] = T(0);
            m2[k] += (double)rv.v[e] * (double)zv.v[e];
            m2[K + k] += (double)rv.v[e] * (double)rv.v[e];
          }
          zv.store(p + o);
          zero.store(x + o);
        }
      }
      block_reduce_w0<2 * K>(m2, red);
      if (warp == 0) {
        bool a = false;
        if (lane < K) {
          sh->rho[lane] = red[64 * K + lane];
          sh->rr0[lane] = red[64 * K + K + lane];
          a = sh->act[lane] && sh->rr0[lane] > 0.0;
          sh->act[lane] = a;
        }
        unsigned b = __ballot_sync(0xffffffffu, a);
        if (lane == 0) sh->nact = __popc(b);
      }
      __syncthreads();
    }
    const double tol2 = P.inner_rtol * P.inner_rtol;
    int it = 0;
    while (sh->nact > 0 && it < P.max_inner) {
      // q = A p, alpha = rho / p.q
      {
        double m3[K];
#pragma unroll
        for (int k = 0; k < K; k++) m3[k] = 0.0;
        spmm_ns<T, K, false>(t, NT, g, nsv, nbr, p, q, m3);
        block_reduce_w0<K>(m3, red);
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
#pragma unroll
        for (int k = 0; k < K; k++) {
          const T al = (T)sh->alpha[k];
          for (int c = t; c < nch; c += NT) {
            size_t o = (size_t)k * blk + (size_t)c * E;
            W xv = W::load(x + o), pv = W::load(p + o), rv = W::load(r + o), qv = W::load(q + o);
            W dv = W::load(dinv + (size_t)c * E);
#pragma unroll
            for (int e = 0; e < E; e++) {
              xv.v[e] += al * pv.v[e];
              rv.v[e] -= al * qv.v[e];
              m2[k] += (double)rv.v[e] * (double)(dv.v[e] * rv.v[e]);
              m2[K + k] += (double)rv.v[e] * (double)rv.v[e];
            }
            xv.store(x + o);
            rv.store(r + o);
          }
        }
        block_reduce_w0<2 * K>(m2, red);
        if (warp == 0) {
          bool a = false;
          if (lane < K) {
            double rz = red[64 * K + lane], rr = red[64 * K + K + lane];
            a = sh->act[lane] && !(rr <= tol2 * sh->rr0[lane]);
            double rho = sh->rho[lane];
            sh->beta[lane] = (a && rho != 0.0) ? rz / rho : 0.0;
            if (a) sh->rho[lane] = rz;
            sh->act[lane] = a;
          }
          unsigned b = __ballot_sync(0xffffffffu, a);
          if (lane == 0) sh->nact = __popc(b);
        }
        __syncthreads();
      }
      it++;
      if (sh->nact == 0) break;
      // p = D^-1 r + beta p
#pragma unroll
      for (int k = 0; k < K; k++) {
        const T be = (T)sh->beta[k];
        for (int c = t; c < nch; c += NT) {
          size_t o = (size_t)k * blk + (size_t)c * E;
          W rv = W::load(r + o), pv = W::load(p + o), dv = W::load(dinv + (size_t)c * E);
#pragma unroll
          for (int e = 0; e < E; e++) pv.v[e] = dv.v[e] * rv.v[e] + be * pv.v[e];
          pv.store(p + o);
        }
      }
      __syncthreads();
    }
    inner += it;
    // 3c. u += x in FP64
    for (int i = t; i < K * blk; i += NT) u[i] += (double)x[i];
    __syncthreads();
    outer++;
  }

  // 4. averages per load case
  for (int qq = 0; qq < P.nrhs; qq++) {
    double acc[12], tot[12];
#pragma unroll
    for (int v = 0; v < 12; v++) acc[v] = 0.0;
    average_soa(t, NT, g, etype, sD, sBbar, u, qq, acc);
    block_sum<12>(acc, red, tot);
    if (t == 0)
      for (int v = 0; v < 12; v++) avg[qq * 12 + v] = tot[v] / g.vol;
  }
  double worst = 0.0;
  for (int k = 0; k < P.nrhs; k++)
    if (sh->rn0[k] > 0.0) worst = fmax(worst, sh->rn[k] / sh->rn0[k]);
  __syncthreads();
  sp_solve_info in;
  in.status = (worst <= P.rtol) ? SP_OK : SP_ERR_NOCONV;
  in.outer_its = outer;
  in.inner_its = inner;
  in.pad = 0;
  in.relres = worst;
  return in;
}

}  // namespace sp
