// rve_plain.cu -- the plain GPU path: one RVE at a time, FP64 throughout,
// every step a grid-wide kernel.  This is the reference's micro solve
// (micro/src/homogenize.c:175-225, micro/src/assembly.c:33-137) moved to the
// GPU without batching or mixed precision: element operators, coloured
// scatter assembly into ELL, Dirichlet rows/columns, FP64 element residual,
// Jacobi-PCG (pcg.cuh) and FP64 volume averages.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "pcg.cuh"
#include "sp_cuda.h"

namespace sp {

constexpr int KMAX = SP_MAX_RHS;

// element operators for the two materials: one block
__global__ void k_rve_ops(MeshGeo g, const double *D, double *Ke, double *Bbar) {
  __shared__ double dsh[192];
  double h[3] = {g.hx, g.hy, g.hz};
  elem_ops_stage1(threadIdx.x, blockDim.x, h, dsh);
  __syncthreads();
  elem_ops_stage2(threadIdx.x, blockDim.x, h, dsh, D, 2, Ke, Bbar);
}

template <typename T>
__global__ void k_zero_vals(T *vals, int ndof) {
  ell_zero<T>(blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, vals, ndof);
}

template <typename T>
__global__ void k_scatter(MeshGeo g, const int *color_elems, int c0, int c1, const uint8_t *slot,
                          const uint8_t *etype, const double *Ke64, T *vals) {
  __shared__ T ke[2 * SP_KE];
  for (int x = threadIdx.x; x < 2 * SP_KE; x += blockDim.x) ke[x] = (T)Ke64[x];
  __syncthreads();
  scatter_colour<T>(blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, g, color_elems,
                    c0, c1, slot, etype, ke, vals);
}

template <typename T>
__global__ void k_bc(MeshGeo g, const int *cols, T *vals, T *dinv) {
  bc_and_dinv<T>(blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, g, cols, vals,
                 dinv);
}

template <int K>
__global__ void k_affine(MeshGeo g, const double *eps, int nrhs, double *u, bool inside) {
  affine_init<K>(blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, g, eps, nrhs, u,
                 inside);
}

// b = -K u (interior), 0 (boundary); norms[k] = ||b_k||^2
template <int K>
__global__ void __launch_bounds__(256)
    k_residual(MeshGeo g, const uint8_t *etype, const double *Ke64, const double *u, double *b,
               double *norms, double *partial, unsigned *ticket) {
  __shared__ double ke[2 * SP_KE];
  __shared__ double red[33 * K];
  __shared__ double tot[K];
  __shared__ bool flag;
  for (int x = threadIdx.x; x < 2 * SP_KE; x += blockDim.x) ke[x] = Ke64[x];
  __syncthreads();
  double mine[K];
  #pragma unroll
  for (int k = 0; k < K; k++) mine[k] = 0.0;
  residual_nodes<K, double>(blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, g,
                            etype, ke, u, b, mine);
  if (grid_sum<K>(mine, partial, ticket, red, tot, &flag) && threadIdx.x == 0)
    #pragma unroll
    for (int k = 0; k < K; k++) norms[k] = tot[k];
}

template <int K>
__global__ void k_add(int n, const double *x, double *u) {
  int t = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
  for (int i = t; i < n * K; i += nt) u[i] += x[i];
}

// averages of load case q: out[0..5] strain, out[6..11] stress
template <int K>
__global__ void __launch_bounds__(256)
    k_average(MeshGeo g, const uint8_t *etype, const double *D, const double *Bbar,
              const double *u, int q, double *out, double *partial, unsigned *ticket) {
  __shared__ double sD[72], sB[144];
  __shared__ double red[33 * 12];
  __shared__ double tot[12];
  __shared__ bool flag;
  for (int x = threadIdx.x; x < 72; x += blockDim.x) sD[x] = D[x];
  for (int x = threadIdx.x; x < 144; x += blockDim.x) sB[x] = Bbar[x];
  __syncthreads();
  double acc[12];
  #pragma unroll
  for (int v = 0; v < 12; v++) acc[v] = 0.0;
  average_elems<K>(blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, g, etype, sD,
                   sB, u, q, acc);
  if (grid_sum<12>(acc, partial, ticket, red, tot, &flag) && threadIdx.x == 0)
    #pragma unroll
    for (int v = 0; v < 12; v++) out[q * 12 + v] = tot[v] / g.vol;
}

// Per-element strain and stress of load case q (micro/src/homogenize.c:
// 370-395, get_elem_properties): the Gauss-weighted means over the element,
// Bbar u_e / vol_elm and D_t Bbar u_e / vol_elm; u is [ndof][K].
template <int K>
__global__ void k_elem_fields(MeshGeo g, const uint8_t *__restrict__ etype, const double *D,
                              const double *Bbar, const double *__restrict__ u, int q,
                              double *strain_e, double *stress_e) {
  const double vol_elm = g.hx * g.hy * g.hz;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.nelm; e += gridDim.x * blockDim.x) {
    int nod[8];
    elem_nodes(g, e, nod);
    double eps[6] = {0, 0, 0, 0, 0, 0};
    for (int a = 0; a < 8; a++)
      for (int d = 0; d < 3; d++) {
        double uv = u[(size_t)(nod[a] * 3 + d) * K + q];
        for (int v = 0; v < 6; v++) eps[v] = fma(Bbar[v * 24 + a * 3 + d], uv, eps[v]);
      }
    const double *C = D + etype[e] * 36;
    for (int v = 0; v < 6; v++) {
      double sv = 0.0;
      for (int w = 0; w < 6; w++) sv = fma(C[v * 6 + w], eps[w], sv);
      strain_e[(size_t)e * 6 + v] = eps[v] / vol_elm;
      stress_e[(size_t)e * 6 + v] = sv / vol_elm;
    }
  }
}

static int blocks_for(Device *d, long long items, int per_block) {
  long long b = (items + per_block - 1) / per_block;
  long long cap = (long long)d->nsm * 4;
  if (b < 1) b = 1;
  return (int)(b < cap ? b : cap);
}

}  // namespace sp

using namespace sp;

struct sp_rve_s {
  sp_rve_desc desc;
  DevPlan *plan = nullptr;
  MeshGeo g;
  int nfiber = 0, dev = -1, last_launches = 0;
  uint8_t *etype_h = nullptr;
  uint8_t *d_etype = nullptr;
  double *d_D = nullptr, *d_Ke = nullptr, *d_Bbar = nullptr;
  double *d_vals = nullptr, *d_dinv = nullptr;
  double *d_u = nullptr, *d_b = nullptr, *d_x = nullptr, *d_r = nullptr, *d_p = nullptr,
         *d_q = nullptr;
  double *d_eps = nullptr, *d_out = nullptr, *d_partial = nullptr;
  PcgState *d_st = nullptr;
  unsigned *d_ticket = nullptr;
  PcgGraph<double, 1, 32> *pcg1 = nullptr;
  PcgGraph<double, 6, 32> *pcg6 = nullptr;
  PcgGraph<double, 8, 32> *pcg8 = nullptr;
  size_t bytes = 0;
  int last_k = 0, last_nrhs = 0;  // padded and actual load cases of the last solve
};

static int rve_assemble(sp_rve *r, Device *d, cudaStream_t s) {
  MeshGeo &g = r->g;
  DevPlan *p = r->plan;
  k_rve_ops<<<1, SP_KE, 0, s>>>(g, r->d_D, r->d_Ke, r->d_Bbar);
  k_zero_vals<double><<<blocks_for(d, (long long)g.ndof * SP_WP / 2, 256), 256, 0, s>>>(r->d_vals,
                                                                                      g.ndof);
  for (int c = 0; c < 8; c++) {
    int c0 = p->color_off[c], c1 = p->color_off[c + 1];
    if (c1 == c0) continue;
    k_scatter<double><<<blocks_for(d, (long long)(c1 - c0) * SP_KE, 256), 256, 0, s>>>(
        g, p->color_elems, c0, c1, p->slot, r->d_etype, r->d_Ke, r->d_vals);
  }
  k_bc<double><<<blocks_for(d, g.ndof, 256), 256, 0, s>>>(g, p->cols, r->d_vals, r->d_dinv);
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

extern "C" int sp_rve_create(const sp_rve_desc *desc, sp_rve **out) {
  if (!desc || !out) return sp_set_error(SP_ERR_ARG, "sp_rve_create: null argument");
  for (int k = 0; k < 3; k++)
    if (desc->n[k] < 1 || desc->len[k] <= 0)
      return sp_set_error(SP_ERR_ARG, "sp_rve_create: bad mesh size or length");
  Device *d;
  SP_TRY(device(&d));
  sp_rve *r = new sp_rve_s();
  r->desc = *desc;
  r->dev = d->id;
  int rc = plan_acquire(desc->n, &r->plan);
  if (rc) {
    delete r;
    return rc;
  }
  r->g = make_geo(desc->n, desc->len);
  MeshGeo &g = r->g;
  r->etype_h = (uint8_t *)malloc(g.nelm);
  if (!r->etype_h) rc = sp_set_error(SP_ERR_NOMEM, "etype");
  if (!rc) rc = sp_classify_elements(desc, r->etype_h, &r->nfiber);
  size_t nv = (size_t)g.ndof * KMAX * sizeof(double);
  if (!rc) rc = dmalloc((void **)&r->d_etype, g.nelm, &r->bytes);
  if (!rc) rc = dmalloc((void **)&r->d_D, 72 * sizeof(double), &r->bytes);
  if (!rc) rc = dmalloc((void **)&r->d_Ke, 2 * SP_KE * sizeof(double), &r->bytes);
  if (!rc) rc = dmalloc((void **)&r->d_Bbar, 144 * sizeof(double), &r->bytes);
  if (!rc) rc = dmalloc((void **)&r->d_vals, (size_t)g.ndof * SP_WP * sizeof(double), &r->bytes);
  if (!rc) rc = dmalloc((void **)&r->d_dinv, (size_t)g.ndof * sizeof(double), &r->bytes);
  double **vecs[6] = {&r->d_u, &r->d_b, &r->d_x, &r->d_r, &r->d_p, &r->d_q};
  for (int v = 0; v < 6 && !rc; v++) rc = dmalloc((void **)vecs[v], nv, &r->bytes);
  if (!rc) rc = dmalloc((void **)&r->d_eps, KMAX * 6 * sizeof(double), &r->bytes);
  if (!rc) rc = dmalloc((void **)&r->d_out, KMAX * 16 * sizeof(double), &r->bytes);
  if (!rc) rc = dmalloc((void **)&r->d_partial, 4096 * 32 * sizeof(double), &r->bytes);
  if (!rc) rc = dmalloc((void **)&r->d_st, sizeof(PcgState), &r->bytes);
  if (!rc) rc = dmalloc((void **)&r->d_ticket, 64, &r->bytes);
  if (!rc) {
    double D[72];
    sp_iso_D(desc->E[0], desc->nu[0], D);
    sp_iso_D(desc->E[1], desc->nu[1], D + 36);
    cudaStream_t s = d->stream;
    if (cudaMemcpyAsync(r->d_etype, r->etype_h, g.nelm, cudaMemcpyHostToDevice, s) ||
        cudaMemcpyAsync(r->d_D, D, sizeof(D), cudaMemcpyHostToDevice, s) ||
        cudaMemsetAsync(r->d_ticket, 0, 64, s))
      rc = sp_set_error(SP_ERR_CUDA, "sp_rve_create: upload failed");
    if (!rc) rc = rve_assemble(r, d, s);
    if (!rc && cudaStreamSynchronize(s))
      rc = sp_set_error(SP_ERR_CUDA, "sp_rve_create: assembly failed: %s",
                        cudaGetErrorString(cudaGetLastError()));
  }
  if (rc) {
    sp_rve_destroy(r);
    return rc;
  }
  *out = r;
  return SP_OK;
}

extern "C" int sp_rve_destroy(sp_rve *r) {
  if (!r) return SP_OK;
  delete r->pcg1;
  delete r->pcg6;
  delete r->pcg8;
  void *bufs[] = {r->d_etype, r->d_D, r->d_Ke, r->d_Bbar, r->d_vals, r->d_dinv, r->d_u,
                  r->d_b, r->d_x, r->d_r, r->d_p, r->d_q, r->d_eps, r->d_out, r->d_partial,
                  r->d_st, r->d_ticket};
  for (void *b : bufs) cudaFree(b);
  plan_release(r->plan);
  free(r->etype_h);
  delete r;
  return SP_OK;
}

extern "C" int sp_rve_sizes(const sp_rve *r, int *ndof, int *nelm, int *nfiber) {
  if (!r) return sp_set_error(SP_ERR_ARG, "null rve");
  if (ndof) *ndof = r->g.ndof;
  if (nelm) *nelm = r->g.nelm;
  if (nfiber) *nfiber = r->nfiber;
  return SP_OK;
}

extern "C" int sp_rve_get_ell(sp_rve *r, int *cols, double *vals) {
  if (!r) return sp_set_error(SP_ERR_ARG, "null rve");
  Device *d;
  SP_TRY(device(&d));
  size_t n = (size_t)r->g.ndof * SP_WP;
  int *hc = (int *)malloc(n * sizeof(int));
  double *hv = (double *)malloc(n * sizeof(double));
  int rc = (!hc || !hv) ? sp_set_error(SP_ERR_NOMEM, "staging") : SP_OK;
  if (!rc && (cudaMemcpy(hc, r->plan->cols, n * sizeof(int), cudaMemcpyDeviceToHost) ||
              cudaMemcpy(hv, r->d_vals, n * sizeof(double), cudaMemcpyDeviceToHost)))
    rc = sp_set_error(SP_ERR_CUDA, "sp_rve_get_ell: copy failed");
  if (!rc)
    for (int row = 0; row < r->g.ndof; row++) {
      if (cols) memcpy(cols + (size_t)row * SP_ELL_WIDTH, hc + (size_t)row * SP_WP, 81 * sizeof(int));
      if (vals)
        memcpy(vals + (size_t)row * SP_ELL_WIDTH, hv + (size_t)row * SP_WP, 81 * sizeof(double));
    }
  free(hc);
  free(hv);
  return rc;
}

extern "C" int sp_rve_get_ke(sp_rve *r, double *ke_matrix, double *ke_fiber) {
  if (!r) return sp_set_error(SP_ERR_ARG, "null rve");
  Device *d;
  SP_TRY(device(&d));
  double h[2 * SP_KE];
  SP_CUDA_TRY(cudaMemcpy(h, r->d_Ke, sizeof(h), cudaMemcpyDeviceToHost));
  if (ke_matrix) memcpy(ke_matrix, h, SP_KE * sizeof(double));
  if (ke_fiber) memcpy(ke_fiber, h + SP_KE, SP_KE * sizeof(double));
  return SP_OK;
}

template <int K>
static int rve_solve_k(sp_rve *r, Device *d, PcgGraph<double, K, 32> *&pcg, int nrhs,
                       const double *strains, double rtol, double *strain_ave, double *stress_ave,
                       double *u_out, sp_solve_info *info) {
  cudaStream_t s = d->stream;
  MeshGeo &g = r->g;
  int nb_node = blocks_for(d, g.ndof / 3, 256);
  int nb_vec = blocks_for(d, (long long)g.ndof * K, 256);
  int nb_row = blocks_for(d, g.ndof, PCG_THREADS / 32);
  int launches = 0;
  if (!pcg) {
    pcg = new PcgGraph<double, K, 32>();
    SP_TRY(pcg->build(s, nb_row, g.ndof, SP_WP, r->d_vals, r->plan->cols, r->d_dinv, r->d_b,
                      r->d_x, r->d_r, r->d_p, r->d_q, 1, r->d_st, r->d_partial, r->d_ticket));
  }
  double eps[KMAX * 6] = {0};
  memcpy(eps, strains, (size_t)nrhs * 6 * sizeof(double));
  SP_CUDA_TRY(cudaMemcpyAsync(r->d_eps, eps, sizeof(eps), cudaMemcpyHostToDevice, s));
  k_affine<K><<<nb_vec, 256, 0, s>>>(g, r->d_eps, nrhs, r->d_u, false);
  launches++;
  double r0[KMAX] = {0}, rn[KMAX] = {0};
  int outer = 0, inner = 0, max_outer = 6;
  bool started = false;
  // Newton / refinement: b = -K u, solve A x = b, u += x  (micro/src/homogenize.c:184-215).
  // The first residual, of the boundary values alone, is the right-hand side
  // the stopping rule is relative to; the iteration then starts from the
  // homogeneous affine field eps . x inside (the exact solution for a
  // homogeneous RVE), which leaves the error near the material interfaces.
  for (;;) {
    double nrm[KMAX];
    k_residual<K><<<nb_node, 256, 0, s>>>(g, r->d_etype, r->d_Ke, r->d_u, r->d_b, r->d_out + 8 * 12,
                                         r->d_partial, r->d_ticket);
    launches++;
    SP_CUDA_TRY(cudaMemcpyAsync(nrm, r->d_out + 8 * 12, K * sizeof(double), cudaMemcpyDeviceToHost, s));
    SP_CUDA_TRY(cudaStreamSynchronize(s));
    if (!started) {
      for (int k = 0; k < nrhs; k++) r0[k] = sqrt(nrm[k]);
      k_affine<K><<<nb_vec, 256, 0, s>>>(g, r->d_eps, nrhs, r->d_u, true);
      launches++;
      started = true;
      continue;
    }
    bool done = true;
    for (int k = 0; k < nrhs; k++) {
      rn[k] = sqrt(nrm[k]);
      if (r0[k] > 0 && rn[k] > rtol * r0[k]) done = false;
    }
    if (done || outer >= max_outer) break;
    PcgState st0 = {};
    st0.nactive = nrhs;
    st0.rtol2 = (0.5 * rtol) * (0.5 * rtol);
    st0.max_its = 20000;
    SP_CUDA_TRY(cudaMemcpyAsync(r->d_st, &st0, sizeof(st0), cudaMemcpyHostToDevice, s));
    int fixed = 0;
    SP_TRY(pcg->run(s, &fixed));
    k_add<K><<<nb_vec, 256, 0, s>>>(g.ndof, r->d_x, r->d_u);
    PcgState st;
    SP_CUDA_TRY(cudaMemcpyAsync(&st, r->d_st, sizeof(st), cudaMemcpyDeviceToHost, s));
    SP_CUDA_TRY(cudaStreamSynchronize(s));
    launches += fixed + 3 * st.its + 1;
    inner += st.its;
    outer++;
  }
  for (int q = 0; q < nrhs; q++) {
    k_average<K><<<blocks_for(d, g.nelm, 256), 256, 0, s>>>(g, r->d_etype, r->d_D, r->d_Bbar,
                                                            r->d_u, q, r->d_out, r->d_partial,
                                                            r->d_ticket);
    launches++;
  }
  double out[KMAX * 12];
  SP_CUDA_TRY(cudaMemcpyAsync(out, r->d_out, sizeof(out), cudaMemcpyDeviceToHost, s));
  if (u_out) {
    // u is [ndof][K]; the caller wants [nrhs][ndof]
    double *h = (double *)malloc((size_t)g.ndof * K * sizeof(double));
    if (!h) return sp_set_error(SP_ERR_NOMEM, "u staging");
    cudaError_t e = cudaMemcpyAsync(h, r->d_u, (size_t)g.ndof * K * sizeof(double),
                                    cudaMemcpyDeviceToHost, s);
    if (!e) e = cudaStreamSynchronize(s);
    if (e) {
      free(h);
      return sp_set_error(SP_ERR_CUDA, "u download failed");
    }
    for (int k = 0; k < nrhs; k++)
      for (int i = 0; i < g.ndof; i++) u_out[(size_t)k * g.ndof + i] = h[(size_t)i * K + k];
    free(h);
  }
  SP_CUDA_TRY(cudaStreamSynchronize(s));
  double worst = 0.0;
  for (int k = 0; k < nrhs; k++) {
    if (strain_ave) memcpy(strain_ave + 6 * k, out + 12 * k, 6 * sizeof(double));
    if (stress_ave) memcpy(stress_ave + 6 * k, out + 12 * k + 6, 6 * sizeof(double));
    double rel = r0[k] > 0 ? rn[k] / r0[k] : 0.0;
    if (rel > worst) worst = rel;
  }
  r->last_launches = launches;
  r->last_k = K;
  r->last_nrhs = nrhs;
  int status = (worst <= rtol) ? SP_OK : SP_ERR_NOCONV;
  if (info) {
    info->status = status;
    info->outer_its = outer;
    info->inner_its = inner;
    info->pad = launches;
    info->relres = worst;
  }
  return status ? sp_set_error(status, "plain solve stopped at relres %.3e", worst) : SP_OK;
}

extern "C" int sp_rve_homogenize(sp_rve *r, int nrhs, const double *strains, double rtol,
                                 double *strain_ave, double *stress_ave, double *u_out,
                                 sp_solve_info *info) {
  if (!r || !strains || nrhs < 1 || nrhs > KMAX || !(rtol > 0))
    return sp_set_error(SP_ERR_ARG, "sp_rve_homogenize: bad argument");
  Device *d;
  SP_TRY(device(&d));
  if (nrhs == 1)
    return rve_solve_k<1>(r, d, r->pcg1, nrhs, strains, rtol, strain_ave, stress_ave, u_out, info);
  if (nrhs <= 6)
    return rve_solve_k<6>(r, d, r->pcg6, nrhs, strains, rtol, strain_ave, stress_ave, u_out, info);
  return rve_solve_k<8>(r, d, r->pcg8, nrhs, strains, rtol, strain_ave, stress_ave, u_out, info);
}

extern "C" int sp_rve_tangent(sp_rve *r, double rtol, double *C, sp_solve_info *info) {
  if (!r || !C) return sp_set_error(SP_ERR_ARG, "sp_rve_tangent: null argument");
  double eps[36] = {0}, st[36];
  for (int j = 0; j < 6; j++) eps[j * 6 + j] = 1.0;
  int rc = sp_rve_homogenize(r, 6, eps, rtol, nullptr, st, nullptr, info);
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) C[i * 6 + j] = st[j * 6 + i];
  return rc;
}

extern "C" int sp_rve_fields(sp_rve *r, int q, double *strain_e, double *stress_e, double *u,
                             double *residual) {
  if (!r) return sp_set_error(SP_ERR_ARG, "sp_rve_fields: null rve");
  if (r->last_nrhs < 1) return sp_set_error(SP_ERR_STATE, "sp_rve_fields: no solve yet");
  if (q < 0 || q >= r->last_nrhs)
    return sp_set_error(SP_ERR_RANGE, "sp_rve_fields: load case %d of %d", q, r->last_nrhs);
  Device *d;
  SP_TRY(device(&d));
  cudaStream_t s = d->stream;
  const MeshGeo &g = r->g;
  const size_t ne = (size_t)g.nelm * 6;
  double *dev = nullptr;
  SP_TRY(dmalloc((void **)&dev, 2 * ne * sizeof(double), nullptr));
  int nb = blocks_for(d, g.nelm, 256);
  switch (r->last_k) {
    case 1: k_elem_fields<1><<<nb, 256, 0, s>>>(g, r->d_etype, r->d_D, r->d_Bbar, r->d_u, q, dev, dev + ne); break;
    case 6: k_elem_fields<6><<<nb, 256, 0, s>>>(g, r->d_etype, r->d_D, r->d_Bbar, r->d_u, q, dev, dev + ne); break;
    default: k_elem_fields<8><<<nb, 256, 0, s>>>(g, r->d_etype, r->d_D, r->d_Bbar, r->d_u, q, dev, dev + ne); break;
  }
  cudaError_t e = cudaGetLastError();
  if (!e && strain_e) e = cudaMemcpyAsync(strain_e, dev, ne * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (!e && stress_e) e = cudaMemcpyAsync(stress_e, dev + ne, ne * sizeof(double), cudaMemcpyDeviceToHost, s);
  // u and the last residual are [ndof][K]: one strided column each
  if (!e && u)
    e = cudaMemcpy2DAsync(u, sizeof(double), r->d_u + q, r->last_k * sizeof(double), sizeof(double),
                          g.ndof, cudaMemcpyDeviceToHost, s);
  if (!e && residual)
    e = cudaMemcpy2DAsync(residual, sizeof(double), r->d_b + q, r->last_k * sizeof(double),
                          sizeof(double), g.ndof, cudaMemcpyDeviceToHost, s);
  if (!e) e = cudaStreamSynchronize(s);
  cudaFree(dev);
  if (e) return sp_set_error(SP_ERR_CUDA, "sp_rve_fields: %s", cudaGetErrorString(e));
  return SP_OK;
}

extern "C" int sp_rve_write_vtu(sp_rve *r, int q, const char *base) {
  if (!r || !base) return sp_set_error(SP_ERR_ARG, "sp_rve_write_vtu: null argument");
  const MeshGeo &g = r->g;
  std::vector<double> se((size_t)g.nelm * 6), st((size_t)g.nelm * 6), u(g.ndof), res(g.ndof);
  SP_TRY(sp_rve_fields(r, q, se.data(), st.data(), u.data(), res.data()));
  return sp_vtu_write(base, r->desc.n, r->desc.len, u.data(), res.data(), r->etype_h, se.data(),
                      st.data());
}
