// pcg.cuh -- grid-wide Jacobi-preconditioned CG over an ELL matrix with K
// right-hand sides, as PETSc's KSPCG + PCJACOBI runs it (the reference's
// micro/src/homogenize.c:324-326 solve with -ksp_type cg -pc_type jacobi),
// convergence on the unpreconditioned residual: ||r_k|| <= rtol ||b_k||.
//
// One CG iteration is three kernels: q = A p (with p.q), the x/r update
// (with r.z and r.r) and the direction update.  Dot products are reduced
// deterministically: each block writes its partial sums, the last block to
// finish (atomic ticket, no waiting) adds them in a fixed order and updates
// the scalars.  The iteration loop runs on the device as a CUDA-graph
// conditional `while` node whose condition the update kernel clears when
// every right-hand side has converged or the iteration limit is reached.
#pragma once

#include <cooperative_groups.h>

#include <algorithm>

#include "sp_cuda.h"

namespace sp {

constexpr int PCG_THREADS = 256;

struct PcgState {
  double rho[SP_MAX_RHS], alpha[SP_MAX_RHS], beta[SP_MAX_RHS];
  double bb[SP_MAX_RHS], rr[SP_MAX_RHS];
  double rtol2;
  int active[SP_MAX_RHS];
  int its, max_its, nactive, pad;
};

// True in exactly one block: the last one to arrive.  The caller must reset
// *ticket to 0 from that block.
__device__ inline bool arrive_last(unsigned *ticket, bool *flag) {
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) *flag = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  return *flag;
}

// Block partial sums -> partial[blockIdx][NV]; the last block folds all
// partials in a fixed order and leaves the totals in tot[NV] (shared).
template <int NV>
__device__ inline bool grid_sum(const double *mine, double *partial, unsigned *ticket,
                                double *red, double *tot, bool *flag) {
  double b[NV];
  block_sum<NV>(mine, red, b);
  if (threadIdx.x == 0)
    #pragma unroll
    for (int q = 0; q < NV; q++) partial[blockIdx.x * NV + q] = b[q];
  if (!arrive_last(ticket, flag)) return false;
  double acc[NV];
  #pragma unroll
  for (int q = 0; q < NV; q++) acc[q] = 0.0;
  for (int blk = threadIdx.x; blk < (int)gridDim.x; blk += blockDim.x)
    #pragma unroll
    for (int q = 0; q < NV; q++) acc[q] += __ldcg(partial + blk * NV + q);
  block_sum<NV>(acc, red, tot);
  if (threadIdx.x == 0) *ticket = 0;
  return true;
}

// r = b - q (q = A x0) or r = b (x0 = 0), z = D^-1 r, p = z; totals rho, bb
template <typename T, int K>
__global__ void __launch_bounds__(PCG_THREADS)
    k_pcg_start(int n, const T *__restrict__ b, const T *__restrict__ q, const T *__restrict__ dinv,
                T *x, T *r, T *p, int x_zero, PcgState *st, double *partial, unsigned *ticket) {
  __shared__ double red[33 * 2 * K];
  __shared__ double tot[2 * K];
  __shared__ bool flag;
  double mine[2 * K];
  #pragma unroll
  for (int k = 0; k < 2 * K; k++) mine[k] = 0.0;
  int t = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
  for (int i = t; i < n; i += nt) {
    T di = dinv[i];
    #pragma unroll
    for (int k = 0; k < K; k++) {
      size_t x_ = (size_t)i * K + k;
      T bv = b[x_];
      T rv = x_zero ? bv : (T)(bv - q[x_]);
      if (x_zero) x[x_] = 0;
      r[x_] = rv;
      T z = di * rv;
      p[x_] = z;
      mine[k] += (double)rv * (double)z;
      mine[K + k] += (double)bv * (double)bv;
    }
  }
  if (grid_sum<2 * K>(mine, partial, ticket, red, tot, &flag) && threadIdx.x == 0) {
    int na = 0;
    #pragma unroll
    for (int k = 0; k < K; k++) {
      st->rho[k] = tot[k];
      st->bb[k] = tot[K + k];
      st->rr[k] = tot[k];
      // converged at start if b = 0 (also covers padding rhs)
      st->active[k] = (tot[K + k] > 0.0) && (k < st->nactive);
      st->alpha[k] = st->beta[k] = 0.0;
      na += st->active[k];
    }
    st->its = 0;
    st->nactive = na;
  }
}

// q = A p, alpha = rho / (p.q)
template <typename T, int K, int L>
__global__ void __launch_bounds__(PCG_THREADS)
    k_pcg_spmm(int n, int wp, const T *__restrict__ vals, const int *__restrict__ cols,
               const T *__restrict__ p, T *q, PcgState *st, double *partial, unsigned *ticket) {
  __shared__ double red[33 * K];
  __shared__ double tot[K];
  __shared__ bool flag;
  if (st->nactive == 0) return;
  double mine[K];
  #pragma unroll
  for (int k = 0; k < K; k++) mine[k] = 0.0;
  spmm<T, K, L>(blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, n, wp, vals, cols,
                p, q, mine);
  if (grid_sum<K>(mine, partial, ticket, red, tot, &flag) && threadIdx.x == 0)
    #pragma unroll
    for (int k = 0; k < K; k++)
      st->alpha[k] = (st->active[k] && tot[k] != 0.0) ? st->rho[k] / tot[k] : 0.0;
}

// x += alpha p, r -= alpha q, z = D^-1 r; rz, rr; convergence and beta
template <typename T, int K>
__global__ void __launch_bounds__(PCG_THREADS)
    k_pcg_update(int n, const T *__restrict__ p, const T *__restrict__ q,
                 const T *__restrict__ dinv, T *x, T *r, PcgState *st, double *partial,
                 unsigned *ticket, cudaGraphConditionalHandle h) {
  __shared__ double red[33 * 2 * K];
  __shared__ double tot[2 * K];
  __shared__ bool flag;
  if (st->nactive == 0) {
    if (blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h, 0);
    return;
  }
  T al[K];
  #pragma unroll
  for (int k = 0; k < K; k++) al[k] = (T)st->alpha[k];
  double mine[2 * K];
  #pragma unroll
  for (int k = 0; k < 2 * K; k++) mine[k] = 0.0;
  int t = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
  for (int i = t; i < n; i += nt) {
    T di = dinv[i];
    #pragma unroll
    for (int k = 0; k < K; k++) {
      size_t x_ = (size_t)i * K + k;
      x[x_] += al[k] * p[x_];
      T rv = r[x_] - al[k] * q[x_];
      r[x_] = rv;
      mine[k] += (double)rv * (double)(di * rv);
      mine[K + k] += (double)rv * (double)rv;
    }
  }
  if (grid_sum<2 * K>(mine, partial, ticket, red, tot, &flag) && threadIdx.x == 0) {
    int na = 0;
    #pragma unroll
    for (int k = 0; k < K; k++) {
      st->rr[k] = tot[K + k];
      if (st->active[k] && tot[K + k] <= st->rtol2 * st->bb[k]) st->active[k] = 0;
      st->beta[k] = (st->active[k] && st->rho[k] != 0.0) ? tot[k] / st->rho[k] : 0.0;
      if (st->active[k]) st->rho[k] = tot[k];
      na += st->active[k];
    }
    st->its++;
    if (st->its >= st->max_its) na = 0;
    st->nactive = na;
    if (na == 0) cudaGraphSetConditional(h, 0);
  }
}

// p = D^-1 r + beta p
template <typename T, int K>
__global__ void __launch_bounds__(PCG_THREADS)
    k_pcg_dir(int n, const T *__restrict__ r, const T *__restrict__ dinv, T *p,
              const PcgState *st) {
  if (st->nactive == 0) return;
  T be[K];
  #pragma unroll
  for (int k = 0; k < K; k++) be[k] = (T)st->beta[k];
  int t = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
  for (int i = t; i < n; i += nt) {
    T di = dinv[i];
    #pragma unroll
    for (int k = 0; k < K; k++) {
      size_t x_ = (size_t)i * K + k;
      p[x_] = di * r[x_] + be[k] * p[x_];
    }
  }
}

// y = A x without reductions (x0 residual, standalone SpMV)
template <typename T, int K, int L>
__global__ void __launch_bounds__(PCG_THREADS)
    k_spmm_plain(int n, int wp, const T *__restrict__ vals, const int *__restrict__ cols,
                 const T *__restrict__ x, T *y) {
  double dummy[K];
  #pragma unroll
  for (int k = 0; k < K; k++) dummy[k] = 0.0;
  spmm<T, K, L>(blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, n, wp, vals, cols,
                x, y, dummy);
}

// A captured Jacobi-PCG solve.  The prologue (optional q = A x0, then
// k_pcg_start) is launched directly; the iterations are one graph holding a
// single conditional `while` node over {spmm, update, dir}.  Built once per
// (matrix, buffers); every run solves A x = b for the current b (and x when
// x_zero == 0).  The caller writes st->nactive (= number of rhs),
// st->rtol2 and st->max_its before run().
template <typename T, int K, int L>
struct PcgGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int nblk = 0, n = 0, wp = 0, x_zero = 1;
  const T *vals = nullptr, *dinv = nullptr, *b = nullptr;
  const int *cols = nullptr;
  T *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr;
  PcgState *st = nullptr;
  double *partial = nullptr;
  unsigned *ticket = nullptr;

  int build(cudaStream_t s, int nblk_, int n_, int wp_, const T *vals_, const int *cols_,
            const T *dinv_, const T *b_, T *x_, T *r_, T *p_, T *q_, int x_zero_, PcgState *st_,
            double *partial_, unsigned *ticket_) {
    destroy();
    nblk = nblk_; n = n_; wp = wp_; vals = vals_; cols = cols_; dinv = dinv_; b = b_;
    x = x_; r = r_; p = p_; q = q_; x_zero = x_zero_; st = st_; partial = partial_;
    ticket = ticket_;
    SP_CUDA_TRY(cudaGraphCreate(&graph, 0));
    cudaGraphConditionalHandle h;
    SP_CUDA_TRY(cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wnode;
    SP_CUDA_TRY(cudaGraphAddNode(&wnode, graph, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    SP_CUDA_TRY(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0,
                                              cudaStreamCaptureModeThreadLocal));
    k_pcg_spmm<T, K, L><<<nblk, PCG_THREADS, 0, s>>>(n, wp, vals, cols, p, q, st, partial, ticket);
    k_pcg_update<T, K><<<nblk, PCG_THREADS, 0, s>>>(n, p, q, dinv, x, r, st, partial, ticket, h);
    k_pcg_dir<T, K><<<nblk, PCG_THREADS, 0, s>>>(n, r, dinv, p, st);
    cudaGraph_t cap;
    SP_CUDA_TRY(cudaStreamEndCapture(s, &cap));
    SP_CUDA_TRY(cudaGraphInstantiate(&exec, graph, 0));
    return SP_OK;
  }
  // Returns the number of kernels launched outside the loop (the loop
  // launches 3 per iteration; read st->its afterwards).
  int run(cudaStream_t s, int *fixed_launches) {
    int f = 1;
    if (!x_zero) {
      k_spmm_plain<T, K, L><<<nblk, PCG_THREADS, 0, s>>>(n, wp, vals, cols, x, q);
      f++;
    }
    k_pcg_start<T, K><<<nblk, PCG_THREADS, 0, s>>>(n, b, q, dinv, x, r, p, x_zero, st, partial,
                                                   ticket);
    SP_CUDA_TRY(cudaGetLastError());
    SP_CUDA_TRY(cudaGraphLaunch(exec, s));
    if (fixed_launches) *fixed_launches = f;
    return SP_OK;
  }
  void destroy() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
  ~PcgGraph() { destroy(); }
};

// The whole Jacobi-PCG (x0 = 0) in one cooperative launch, for matrices
// small enough that the three launches of an iteration cost more than their
// work.  Grid barriers separate the phases; a phase's per-block partial sums
// go to one of two partial arrays (two barriers lie between a block's read
// of an array and the next write to it), and every block folds the partials
// in the same order, so all blocks hold identical scalars without a
// broadcast and take the same exit: every right-hand side converged or
// st->max_its reached.  The vector reads of p are coherent: the kernel writes
// p itself.  Block 0 leaves the final state in st, as the graph solve does.
template <typename T, int K, int L>
__global__ void __launch_bounds__(PCG_THREADS)
    k_pcg_coop(int n, int wp, const T *__restrict__ vals, const int *__restrict__ cols,
               const T *__restrict__ dinv, const T *__restrict__ b, T *x, T *r, T *p, T *q,
               PcgState *st, double *part_a, double *part_b) {
  namespace cgr = cooperative_groups;
  cgr::grid_group grid = cgr::this_grid();
  __shared__ double red[33 * 2 * K];
  __shared__ double tot[2 * K];
  const int t = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
  const int nb = gridDim.x;
  // every block folds the partials of `part` (NV per block) in block order
  auto fold = [&](const double *part, int nv, double *out) {
    double acc[2 * K];
    #pragma unroll
    for (int v = 0; v < 2 * K; v++) acc[v] = 0.0;
    for (int blk = threadIdx.x; blk < nb; blk += blockDim.x)
      for (int v = 0; v < nv; v++) acc[v] += __ldcg(part + blk * nv + v);
    block_sum<2 * K>(acc, red, out);
  };
  auto publish = [&](const double *mine, double *part, int nv) {
    double bs[2 * K];
    block_sum<2 * K>(mine, red, bs);
    if (threadIdx.x == 0)
      for (int v = 0; v < nv; v++) part[blockIdx.x * nv + v] = bs[v];
  };
  const double rtol2 = st->rtol2;
  const int max_its = st->max_its, nrhs = st->nactive;
  // start: x = 0, r = b, p = z = D^-1 b; rho = r.z, bb = b.b
  double mine[2 * K];
  #pragma unroll
  for (int v = 0; v < 2 * K; v++) mine[v] = 0.0;
  for (int i = t; i < n; i += nt) {
    const T di = dinv[i];
    #pragma unroll
    for (int k = 0; k < K; k++) {
      const size_t o = (size_t)i * K + k;
      const T bv = b[o];
      x[o] = 0;
      r[o] = bv;
      const T z = di * bv;
      p[o] = z;
      mine[k] += (double)bv * (double)z;
      mine[K + k] += (double)bv * (double)bv;
    }
  }
  publish(mine, part_b, 2 * K);
  grid.sync();
  double rho[K], bb[K], rr[K], alpha[K], beta[K];
  int act[K];
  fold(part_b, 2 * K, tot);
  int na = 0;
  #pragma unroll
  for (int k = 0; k < K; k++) {
    rho[k] = tot[k];
    bb[k] = tot[K + k];
    rr[k] = bb[k];
    alpha[k] = beta[k] = 0.0;
    act[k] = bb[k] > 0.0 && k < nrhs;
    na += act[k];
  }
  int its = 0;
  while (na > 0 && its < max_its) {
    // q = A p, alpha = rho / p.q
    double pq[2 * K];
    #pragma unroll
    for (int v = 0; v < 2 * K; v++) pq[v] = 0.0;
    spmm<T, K, L, false>(t, nt, n, wp, vals, cols, p, q, pq);
    publish(pq, part_a, K);
    grid.sync();
    fold(part_a, K, tot);
    #pragma unroll
    for (int k = 0; k < K; k++) alpha[k] = (act[k] && tot[k] != 0.0) ? rho[k] / tot[k] : 0.0;
    // x += alpha p, r -= alpha q; r.z, r.r
    #pragma unroll
    for (int v = 0; v < 2 * K; v++) mine[v] = 0.0;
    for (int i = t; i < n; i += nt) {
      const T di = dinv[i];
      #pragma unroll
      for (int k = 0; k < K; k++) {
        const size_t o = (size_t)i * K + k;
        x[o] += (T)alpha[k] * p[o];
        const T rv = r[o] - (T)alpha[k] * q[o];
        r[o] = rv;
        mine[k] += (double)rv * (double)(di * rv);
        mine[K + k] += (double)rv * (double)rv;
      }
    }
    publish(mine, part_b, 2 * K);
    grid.sync();
    fold(part_b, 2 * K, tot);
    na = 0;
    #pragma unroll
    for (int k = 0; k < K; k++) {
      rr[k] = tot[K + k];
      if (act[k] && rr[k] <= rtol2 * bb[k]) act[k] = 0;
      beta[k] = (act[k] && rho[k] != 0.0) ? tot[k] / rho[k] : 0.0;
      if (act[k]) rho[k] = tot[k];
      na += act[k];
    }
    its++;
    if (na == 0 || its >= max_its) break;
    // p = D^-1 r + beta p
    for (int i = t; i < n; i += nt) {
      const T di = dinv[i];
      #pragma unroll
      for (int k = 0; k < K; k++) {
        const size_t o = (size_t)i * K + k;
        p[o] = di * r[o] + (T)beta[k] * p[o];
      }
    }
    grid.sync();
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    #pragma unroll
    for (int k = 0; k < K; k++) {
      st->rho[k] = rho[k];
      st->bb[k] = bb[k];
      st->rr[k] = rr[k];
      st->alpha[k] = alpha[k];
      st->beta[k] = beta[k];
      st->active[k] = act[k];
    }
    st->its = its;
    st->nactive = na;
  }
}

// A cooperative Jacobi-PCG solve of A x = b from x = 0 (k_pcg_coop): one
// launch per solve, as many blocks as can be resident at once (at most what
// the rows need).  The caller writes st->nactive (= number of rhs),
// st->rtol2 and st->max_its before run(); partial holds 2 x 2K doubles per
// block.
template <typename T, int K, int L>
struct PcgCoop {
  int nblk = 0, n = 0, wp = 0;
  const T *vals = nullptr, *dinv = nullptr, *b = nullptr;
  const int *cols = nullptr;
  T *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr;
  PcgState *st = nullptr;
  double *partial = nullptr;

  int build(const Device *d, int max_blk, int n_, int wp_, const T *vals_, const int *cols_,
            const T *dinv_, const T *b_, T *x_, T *r_, T *p_, T *q_, PcgState *st_,
            double *partial_) {
    n = n_; wp = wp_; vals = vals_; cols = cols_; dinv = dinv_; b = b_;
    x = x_; r = r_; p = p_; q = q_; st = st_; partial = partial_;
    int occ = 0;
    SP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_pcg_coop<T, K, L>,
                                                              PCG_THREADS, 0));
    if (occ < 1) return sp_set_error(SP_ERR_CUDA, "cooperative PCG: no block fits an SM");
    const long long need = ((long long)n * L + PCG_THREADS - 1) / PCG_THREADS;
    nblk = (int)std::min<long long>(std::min<long long>(need, (long long)d->nsm * occ), max_blk);
    if (nblk < 1) nblk = 1;
    return SP_OK;
  }
  int run(cudaStream_t s) {
    double *pa = partial, *pb = partial + (size_t)nblk * 2 * K;
    void *args[] = {(void *)&n, (void *)&wp, (void *)&vals, (void *)&cols, (void *)&dinv,
                    (void *)&b, (void *)&x, (void *)&r, (void *)&p, (void *)&q,
                    (void *)&st, (void *)&pa, (void *)&pb};
    SP_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)k_pcg_coop<T, K, L>, dim3(nblk),
                                            dim3(PCG_THREADS), args, 0, s));
    return SP_OK;
  }
};

}  // namespace sp
