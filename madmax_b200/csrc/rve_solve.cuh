// rve_solve.cuh -- the per-RVE solve shared by the batched kernel
// (rve_batch.cu) and the serving loop (serve.cu), run by one CTA of NT
// threads: FP64 element residual (micro/src/assembly.c:33-82), Jacobi-PCG
// corrections in precision T on the RVE's ELL values, FP64 update of u
// (micro/src/homogenize.c:184-215, with a relative stopping rule) and FP64
// volume averages (micro/src/homogenize.c:344-368).
#pragma once

#include "rve_device.cuh"

namespace sp {

struct SolveArgs {
  int nrhs;
  double rtol, inner_rtol;
  int max_outer, max_inner;
};

// On entry u holds the start iterate with the boundary values of every load
// case.  On exit avg[q*12 + 0..5] = <strain>_q, avg[q*12 + 6..11] =
// <stress>_q (q < nrhs, shared memory, valid in every thread) and the return
// value describes the solve.  red: shared scratch of 33*16 doubles.
template <typename T, int K, int L, int NT>
__device__ sp_solve_info solve_rve(const MeshGeo &g, const T *vals, const int *cols, const T *dinv,
                                   const uint8_t *etype, const double *sKe, const double *sD,
                                   const double *sBbar, double *u, T *r, T *x, T *p, T *q,
                                   const SolveArgs &P, double *red, double *avg) {
  const int t = threadIdx.x;
  const int n = g.ndof;
  double rn0[K], rn[K];
  int outer = 0, inner = 0;
  for (;;) {
    // 3a. FP64 residual b = -K u -> r (type T), norms
    double m1[K], nrm[K];
#pragma unroll
    for (int k = 0; k < K; k++) m1[k] = 0.0;
    residual_nodes<K, T>(t, NT, g, etype, sKe, u, r, m1);
    block_sum<K>(m1, red, nrm);
    bool done = true;
#pragma unroll
    for (int k = 0; k < K; k++) {
      rn[k] = sqrt(nrm[k]);
      if (outer == 0) rn0[k] = rn[k];
      if (k < P.nrhs && rn0[k] > 0.0 && rn[k] > P.rtol * rn0[k]) done = false;
    }
    if (done || outer >= P.max_outer) break;
    // 3b. Jacobi-PCG on A x = r in precision T
    double m2[2 * K], s2[2 * K];
#pragma unroll
    for (int k = 0; k < 2 * K; k++) m2[k] = 0.0;
    for (int i = t; i < n; i += NT) {
      T di = dinv[i];
#pragma unroll
      for (int k = 0; k < K; k++) {
        size_t ix = (size_t)i * K + k;
        T rv_ = r[ix];
        T z = di * rv_;
        x[ix] = T(0);
        p[ix] = z;
        m2[k] += (double)rv_ * (double)z;
        m2[K + k] += (double)rv_ * (double)rv_;
      }
    }
    block_sum<2 * K>(m2, red, s2);
    double rho[K], rr0[K];
    bool act[K];
    int nact = 0;
#pragma unroll
    for (int k = 0; k < K; k++) {
      rho[k] = s2[k];
      rr0[k] = s2[K + k];
      act[k] = (k < P.nrhs) && rr0[k] > 0.0 && rn0[k] > 0.0 && rn[k] > P.rtol * rn0[k];
      nact += act[k];
    }
    double tol2 = P.inner_rtol * P.inner_rtol;
    int it = 0;
    while (nact > 0 && it < P.max_inner) {
      double m3[K], pq[K];
#pragma unroll
      for (int k = 0; k < K; k++) m3[k] = 0.0;
      spmm<T, K, L, false>(t, NT, n, SP_WP, vals, cols, p, q, m3);
      block_sum<K>(m3, red, pq);
      T al[K];
#pragma unroll
      for (int k = 0; k < K; k++) al[k] = (act[k] && pq[k] != 0.0) ? (T)(rho[k] / pq[k]) : T(0);
#pragma unroll
      for (int k = 0; k < 2 * K; k++) m2[k] = 0.0;
      for (int i = t; i < n; i += NT) {
        T di = dinv[i];
#pragma unroll
        for (int k = 0; k < K; k++) {
          size_t ix = (size_t)i * K + k;
          x[ix] += al[k] * p[ix];
          T rv_ = r[ix] - al[k] * q[ix];
          r[ix] = rv_;
          m2[k] += (double)rv_ * (double)(di * rv_);
          m2[K + k] += (double)rv_ * (double)rv_;
        }
      }
      block_sum<2 * K>(m2, red, s2);
      T be[K];
      nact = 0;
#pragma unroll
      for (int k = 0; k < K; k++) {
        if (act[k] && s2[K + k] <= tol2 * rr0[k]) act[k] = false;
        be[k] = (act[k] && rho[k] != 0.0) ? (T)(s2[k] / rho[k]) : T(0);
        if (act[k]) rho[k] = s2[k];
        nact += act[k];
      }
      it++;
      if (nact == 0) break;
      for (int i = t; i < n; i += NT) {
        T di = dinv[i];
#pragma unroll
        for (int k = 0; k < K; k++) {
          size_t ix = (size_t)i * K + k;
          p[ix] = di * r[ix] + be[k] * p[ix];
        }
      }
      __syncthreads();
    }
    inner += it;
    // 3c. u += x in FP64
    for (size_t ix = t; ix < (size_t)n * K; ix += NT) u[ix] += (double)x[ix];
    __syncthreads();
    outer++;
  }

  // 4. averages per load case
  double worst = 0.0;
  for (int qq = 0; qq < P.nrhs; qq++) {
    double acc[12], tot[12];
#pragma unroll
    for (int v = 0; v < 12; v++) acc[v] = 0.0;
    average_elems<K>(t, NT, g, etype, sD, sBbar, u, qq, acc);
    block_sum<12>(acc, red, tot);
    if (t == 0)
      for (int v = 0; v < 12; v++) avg[qq * 12 + v] = tot[v] / g.vol;
  }
#pragma unroll
  for (int k = 0; k < K; k++)
    if (k < P.nrhs && rn0[k] > 0.0) worst = fmax(worst, rn[k] / rn0[k]);
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
