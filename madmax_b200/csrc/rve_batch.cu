// rve_batch.cu -- batched, mixed-precision homogenization of many RVEs in
// one persistent launch.
//
// Each CTA takes the next RVE from a work counter (largest meshes first) and
// runs the whole micro solve of micro/src/homogenize.c:175-225 for all load
// cases of that RVE on its own:
//   1. element operators (D, Ke = sum B^T D B w, Bbar) in shared memory;
//   2. assembly: the RVE's ELL values by the 8-colour conflict-free scatter,
//      then Dirichlet rows/columns and the Jacobi diagonal;
//   3. refinement loop: FP64 residual b = -K u from the element operators
//      (the FP64 "true" residual), FP32 Jacobi-PCG on the ELL values for the
//      correction A x = b, u += x in FP64, until ||b_k|| <= rtol ||b_k,0||;
//   4. FP64 volume averages of strain and stress per load case.
// A CTA never waits on another CTA, so the kernel needs no grid barrier and
// no co-residency guarantee.  All reductions are CTA-local and deterministic:
// a RVE's result does not depend on which CTA solves it or on what else is
// in the batch.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>

#include "rve_solve.cuh"
#include "sp_cuda.h"

namespace sp {

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
  void *ws_rm;           // per CTA row-major assembly scratch [maxdof][84] of T
  void *ws_drm;          // per CTA row-major diagonal scratch [maxdof] of T
  size_t rm_stride;      // maxdof*84
  size_t drm_stride;     // maxdof rounded up to 4
  int *counter;
  double rtol, inner_rtol;
  int max_outer, max_inner;
};

template <typename T, int K, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_batch(BatchParams P) {
  __shared__ double sKe[2 * SP_KE];
  __shared__ T sKeT[2 * SP_KE];
  __shared__ double sD[72], sBbar[144], sdsh[192];
  // block_sum<NV> needs 33*NV doubles; NV is at most max(2K, 12) <= 16
  __shared__ double red[33 * 16];
  __shared__ double savg[SP_MAX_RHS * 12];
  __shared__ CgShared sh;
  __shared__ int s_job;
  const int t = threadIdx.x;
  double *u = P.ws_u + (size_t)blockIdx.x * P.ws_stride;
  T *ws = reinterpret_cast<T *>(P.ws_v) + (size_t)blockIdx.x * 4 * P.ws_stride;
  T *r = ws, *x = ws + P.ws_stride, *p = ws + 2 * P.ws_stride, *q = ws + 3 * P.ws_stride;
  T *vrm = reinterpret_cast<T *>(P.ws_rm) + (size_t)blockIdx.x * P.rm_stride;
  T *drm = reinterpret_cast<T *>(P.ws_drm) + (size_t)blockIdx.x * P.drm_stride;

  for (;;) {
    if (t == 0) s_job = atomicAdd(P.counter, 1);
    __syncthreads();
    int job = s_job;
    __syncthreads();
    if (job >= P.nrve) break;
    const int rid = P.order[job];
    const BatchRve rv = P.rves[rid];
    const BatchPlan pl = P.plans[rv.plan];
    MeshGeo g = pl.geo;
    g.hx = rv.len[0] / g.nex;
    g.hy = rv.len[1] / g.ney;
    g.hz = rv.len[2] / g.nez;
    g.vol = rv.len[0] * rv.len[1] * rv.len[2];
    T *nsv = reinterpret_cast<T *>(P.nsv) + rv.nsv_off;
    T *dinv = reinterpret_cast<T *>(P.dinv) + rv.dinv_off;
    const uint8_t *etype = P.etype + rv.etype_off;

    // 1. element operators
    if (t < 2) iso_D(P.mats[rid * 4 + 2 * t], P.mats[rid * 4 + 2 * t + 1], sD + 36 * t);
    double h[3] = {g.hx, g.hy, g.hz};
    elem_ops_stage1(t, NT, h, sdsh);
    __syncthreads();
    elem_ops_stage2(t, NT, h, sdsh, sD, 2, sKe, sBbar);
    __syncthreads();
    for (int i = t; i < 2 * SP_KE; i += NT) sKeT[i] = (T)sKe[i];
    // 2. assembly: coloured scatter into the row-major scratch, Dirichlet
    //    rows/columns, then the node-sliced copy the solve reads
    ell_zero<T>(t, NT, vrm, g.ndof);
    __syncthreads();
    for (int c = 0; c < 8; c++) {
      if (pl.color_off[c + 1] > pl.color_off[c])
        scatter_colour<T>(t, NT, g, pl.color_elems, pl.color_off[c], pl.color_off[c + 1], pl.slot,
                          etype, sKeT, vrm);
      __syncthreads();
    }
    bc_and_dinv<T>(t, NT, g, pl.cols, vrm, drm);
    __syncthreads();
    ns_from_rows<T>(t, NT, g, pl.cols, vrm, drm, nsv, dinv);
    // load cases: u = eps . x on the boundary, 0 inside
    affine_soa<K>(t, NT, g, P.strains + (size_t)rid * P.nrhs * 6, P.nrhs, false, u);
    __syncthreads();

    SolveArgs sa;
    sa.nrhs = P.nrhs;
    sa.rtol = P.rtol;
    sa.inner_rtol = P.inner_rtol;
    sa.max_outer = P.max_outer;
    sa.max_inner = P.max_inner;
    sp_solve_info in = solve_rve<T, K, NT>(g, nsv, pl.nbr, dinv, etype, sKe, sD, sBbar, u, r, x, p,
                                           q, sa, red, &sh, savg);
    if (t == 0) {
      for (int qq = 0; qq < P.nrhs; qq++) {
        size_t o = ((size_t)rid * P.nrhs + qq) * 6;
        for (int v = 0; v < 6; v++) {
          if (P.out_strain) P.out_strain[o + v] = savg[qq * 12 + v];
          P.out_stress[o + v] = savg[qq * 12 + 6 + v];
        }
      }
      P.out_info[rid] = in;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------- dispatch ---

using BatchFn = void (*)(BatchParams);

template <typename T, int K>
static BatchFn pick_shape(int threads, int ctas) {
  if (threads == 256) return ctas >= 4 ? k_batch<T, K, 256, 4> : k_batch<T, K, 256, 2>;
  return ctas >= 2 ? k_batch<T, K, 512, 2> : k_batch<T, K, 512, 1>;
}

static BatchFn pick(int prec, int K, int threads, int ctas) {
  if (prec == SP_PREC_FP64) {
    if (K == 1) return pick_shape<double, 1>(threads, ctas);
    if (K <= 6) return pick_shape<double, 6>(threads, ctas);
    return pick_shape<double, 8>(threads, ctas);
  }
  if (K == 1) return pick_shape<float, 1>(threads, ctas);
  if (K <= 6) return pick_shape<float, 6>(threads, ctas);
  return pick_shape<float, 8>(threads, ctas);
}

static int kpad(int nrhs) { return nrhs == 1 ? 1 : (nrhs <= 6 ? 6 : 8); }

}  // namespace sp

using namespace sp;

struct sp_batch_s {
  int nrve = 0, nrhs = 6, kp = 6, dev = -1, grid = 0, last_launches = 0;
  sp_batch_opts o;
  std::vector<DevPlan *> plans;
  std::vector<sp_rve_desc> descs;
  BatchParams P;
  BatchPlan *d_plans = nullptr;
  BatchRve *d_rves = nullptr;
  int *d_order = nullptr, *d_counter = nullptr;
  void *d_vals = nullptr, *d_dinv = nullptr;
  uint8_t *d_etype = nullptr;
  double *d_strains = nullptr, *d_mats = nullptr, *d_stress = nullptr, *d_strain = nullptr;
  sp_solve_info *d_info = nullptr;
  double *d_ws_u = nullptr;
  void *d_ws_v = nullptr, *d_ws_rm = nullptr, *d_ws_drm = nullptr;
  size_t bytes = 0;
};

extern "C" void sp_batch_opts_default(sp_batch_opts *o) {
  memset(o, 0, sizeof(*o));
  o->nrhs = 6;
  o->precision = SP_PREC_MIXED;
  o->rtol = 1e-8;
  o->inner_rtol = 1e-5;
  o->max_outer = 8;
  o->max_inner = 4000;
  o->threads = 512;
  o->lanes_per_row = 0;
  o->ctas_per_sm = 2;
}

extern "C" int sp_batch_destroy(sp_batch *b) {
  if (!b) return SP_OK;
  void *bufs[] = {b->d_plans, b->d_rves, b->d_order, b->d_counter, b->d_vals, b->d_dinv,
                  b->d_etype, b->d_strains, b->d_mats, b->d_stress, b->d_strain, b->d_info,
                  b->d_ws_u, b->d_ws_v, b->d_ws_rm, b->d_ws_drm};
  for (void *p : bufs) cudaFree(p);
  for (DevPlan *p : b->plans) plan_release(p);
  delete b;
  return SP_OK;
}

extern "C" int sp_batch_create(int nrve, const sp_rve_desc *descs, const sp_batch_opts *opts,
                               sp_batch **out) {
  if (nrve < 1 || !descs || !out) return sp_set_error(SP_ERR_ARG, "sp_batch_create: bad argument");
  sp_batch_opts o;
  if (opts)
    o = *opts;
  else
    sp_batch_opts_default(&o);
  if (o.nrhs < 1 || o.nrhs > SP_MAX_RHS)
    return sp_set_error(SP_ERR_ARG, "sp_batch_create: nrhs must be 1..%d", SP_MAX_RHS);
  if (o.precision != SP_PREC_MIXED && o.precision != SP_PREC_FP64)
    return sp_set_error(SP_ERR_ARG, "sp_batch_create: unknown precision");
  // CTA shape: 512 threads x 1 or 2 CTAs per SM, or 256 threads x 2 or 4
  if (o.threads == 0) o.threads = 512;
  if (o.threads != 256 && o.threads != 512)
    return sp_set_error(SP_ERR_ARG, "sp_batch_create: threads must be 256 or 512");
  if (o.ctas_per_sm == 0) o.ctas_per_sm = 2;
  if (o.threads == 512 && o.ctas_per_sm != 1 && o.ctas_per_sm != 2)
    return sp_set_error(SP_ERR_ARG, "sp_batch_create: 512-thread CTAs run 1 or 2 per SM");
  if (o.threads == 256 && o.ctas_per_sm != 2 && o.ctas_per_sm != 4)
    return sp_set_error(SP_ERR_ARG, "sp_batch_create: 256-thread CTAs run 2 or 4 per SM");
  o.lanes_per_row = 0;  // the node-sliced SpMM uses one lane per node (3 rows)
  if (o.max_outer < 1) o.max_outer = 8;
  if (o.max_inner < 1) o.max_inner = 4000;
  if (!(o.rtol > 0)) o.rtol = 1e-8;
  if (!(o.inner_rtol > 0)) o.inner_rtol = 1e-5;
  for (int i = 0; i < nrve; i++)
    for (int k = 0; k < 3; k++)
      if (descs[i].n[k] < 1 || descs[i].len[k] <= 0)
        return sp_set_error(SP_ERR_ARG, "sp_batch_create: RVE %d has a bad mesh", i);
  Device *d;
  SP_TRY(device(&d));
  sp_batch *b = new sp_batch_s();
  b->nrve = nrve;
  b->o = o;
  b->nrhs = o.nrhs;
  b->kp = kpad(o.nrhs);
  b->dev = d->id;
  b->descs.assign(descs, descs + nrve);
  const size_t tsz = (o.precision == SP_PREC_FP64) ? sizeof(double) : sizeof(float);
  int rc = SP_OK;
  // plans, one per distinct size
  std::map<std::vector<int>, int> plan_index;
  std::vector<BatchPlan> hplans;
  std::vector<BatchRve> hrves(nrve);
  long long voff = 0, eoff = 0, doff = 0;
  int maxdof = 0, maxnp = 0;
  for (int i = 0; i < nrve && !rc; i++) {
    std::vector<int> key(descs[i].n, descs[i].n + 3);
    auto it = plan_index.find(key);
    if (it == plan_index.end()) {
      DevPlan *p;
      rc = plan_acquire(descs[i].n, &p);
      if (rc) break;
      b->plans.push_back(p);
      BatchPlan bp;
      bp.geo = p->geo;
      bp.cols = p->cols;
      bp.nbr = p->nbr;
      bp.slot = p->slot;
      bp.color_elems = p->color_elems;
      for (int c = 0; c < 9; c++) bp.color_off[c] = p->color_off[c];
      it = plan_index.emplace(key, (int)hplans.size()).first;
      hplans.push_back(bp);
    }
    const MeshGeo &g = hplans[it->second].geo;
    BatchRve &r = hrves[i];
    r.plan = it->second;
    for (int k = 0; k < 3; k++) r.len[k] = descs[i].len[k];
    r.nsv_off = voff;
    r.etype_off = eoff;
    r.dinv_off = doff;
    voff += (long long)g.nn_pad * 243;
    eoff += (g.nelm + 15) / 16 * 16;
    doff += 3LL * g.nn_pad;
    maxdof = std::max(maxdof, g.ndof);
    maxnp = std::max(maxnp, g.nn_pad);
  }
  // host-side classification into one pinned staging buffer
  uint8_t *et = nullptr;
  if (!rc && cudaMallocHost((void **)&et, eoff ? eoff : 16))
    rc = sp_set_error(SP_ERR_NOMEM, "sp_batch_create: pinned staging");
  for (int i = 0; i < nrve && !rc; i++) rc = sp_classify_elements(&descs[i], et + hrves[i].etype_off, nullptr);
  // largest RVEs first (longest-processing-time order)
  std::vector<int> order(nrve);
  for (int i = 0; i < nrve; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
    return hplans[hrves[a].plan].geo.ndof > hplans[hrves[c].plan].geo.ndof;
  });
  int nrhs = o.nrhs, kp = b->kp;
  b->grid = d->nsm * o.ctas_per_sm;
  size_t stride = (size_t)kp * 3 * maxnp;
  size_t rm_stride = (size_t)maxdof * SP_WP, drm_stride = (size_t)(maxdof + 3) / 4 * 4;
  size_t *acct = &b->bytes;
  if (!rc) rc = dmalloc((void **)&b->d_plans, hplans.size() * sizeof(BatchPlan), acct);
  if (!rc) rc = dmalloc((void **)&b->d_rves, nrve * sizeof(BatchRve), acct);
  if (!rc) rc = dmalloc((void **)&b->d_order, nrve * sizeof(int), acct);
  if (!rc) rc = dmalloc((void **)&b->d_counter, 256, acct);
  if (!rc) rc = dmalloc(&b->d_vals, (size_t)voff * tsz, acct);
  if (!rc) rc = dmalloc(&b->d_dinv, (size_t)doff * tsz, acct);
  if (!rc) rc = dmalloc((void **)&b->d_etype, eoff, acct);
  if (!rc) rc = dmalloc((void **)&b->d_strains, (size_t)nrve * nrhs * 6 * sizeof(double), acct);
  if (!rc) rc = dmalloc((void **)&b->d_mats, (size_t)nrve * 4 * sizeof(double), acct);
  if (!rc) rc = dmalloc((void **)&b->d_stress, (size_t)nrve * nrhs * 6 * sizeof(double), acct);
  if (!rc) rc = dmalloc((void **)&b->d_strain, (size_t)nrve * nrhs * 6 * sizeof(double), acct);
  if (!rc) rc = dmalloc((void **)&b->d_info, (size_t)nrve * sizeof(sp_solve_info), acct);
  if (!rc) rc = dmalloc((void **)&b->d_ws_u, (size_t)b->grid * stride * sizeof(double), acct);
  if (!rc) rc = dmalloc(&b->d_ws_v, (size_t)b->grid * 4 * stride * tsz, acct);
  if (!rc) rc = dmalloc(&b->d_ws_rm, (size_t)b->grid * rm_stride * tsz, acct);
  if (!rc) rc = dmalloc(&b->d_ws_drm, (size_t)b->grid * drm_stride * tsz, acct);
  if (!rc) {
    // default inputs: unit strains e_0..e_{nrhs-1}, materials of the descriptors
    std::vector<double> eps((size_t)nrve * nrhs * 6, 0.0), mats((size_t)nrve * 4);
    for (int i = 0; i < nrve; i++) {
      for (int k = 0; k < nrhs; k++) eps[((size_t)i * nrhs + k) * 6 + (k % 6)] = 1.0;
      mats[i * 4 + 0] = descs[i].E[0];
      mats[i * 4 + 1] = descs[i].nu[0];
      mats[i * 4 + 2] = descs[i].E[1];
      mats[i * 4 + 3] = descs[i].nu[1];
    }
    if (cudaMemcpy(b->d_plans, hplans.data(), hplans.size() * sizeof(BatchPlan), cudaMemcpyHostToDevice) ||
        cudaMemcpy(b->d_rves, hrves.data(), nrve * sizeof(BatchRve), cudaMemcpyHostToDevice) ||
        cudaMemcpy(b->d_order, order.data(), nrve * sizeof(int), cudaMemcpyHostToDevice) ||
        cudaMemcpy(b->d_etype, et, eoff, cudaMemcpyHostToDevice) ||
        cudaMemcpy(b->d_strains, eps.data(), eps.size() * sizeof(double), cudaMemcpyHostToDevice) ||
        cudaMemcpy(b->d_mats, mats.data(), mats.size() * sizeof(double), cudaMemcpyHostToDevice) ||
        cudaMemset(b->d_info, 0, (size_t)nrve * sizeof(sp_solve_info)))
      rc = sp_set_error(SP_ERR_CUDA, "sp_batch_create: upload failed");
  }
  if (et) cudaFreeHost(et);
  if (rc) {
    sp_batch_destroy(b);
    return rc;
  }
  BatchParams &P = b->P;
  P.plans = b->d_plans;
  P.rves = b->d_rves;
  P.order = b->d_order;
  P.nrve = nrve;
  P.nrhs = nrhs;
  P.nsv = b->d_vals;
  P.dinv = b->d_dinv;
  P.etype = b->d_etype;
  P.strains = b->d_strains;
  P.mats = b->d_mats;
  P.out_stress = b->d_stress;
  P.out_strain = b->d_strain;
  P.out_info = b->d_info;
  P.ws_u = b->d_ws_u;
  P.ws_v = b->d_ws_v;
  P.ws_stride = stride;
  P.ws_rm = b->d_ws_rm;
  P.ws_drm = b->d_ws_drm;
  P.rm_stride = rm_stride;
  P.drm_stride = drm_stride;
  P.counter = b->d_counter;
  P.rtol = o.rtol;
  P.inner_rtol = o.inner_rtol;
  P.max_outer = o.max_outer;
  P.max_inner = o.max_inner;
  *out = b;
  return SP_OK;
}

extern "C" int sp_batch_device_bytes(const sp_batch *b, size_t *bytes) {
  if (!b || !bytes) return sp_set_error(SP_ERR_ARG, "null argument");
  size_t s = b->bytes;
  for (DevPlan *p : b->plans) s += p->bytes;
  *bytes = s;
  return SP_OK;
}

extern "C" int sp_batch_upload(sp_batch *b, const double *strains, const double *materials,
                               void *stream) {
  if (!b) return sp_set_error(SP_ERR_ARG, "null batch");
  Device *d;
  SP_TRY(device(&d));
  cudaStream_t s = pick_stream(stream, d);
  if (strains)
    SP_CUDA_TRY(cudaMemcpyAsync(b->d_strains, strains, (size_t)b->nrve * b->nrhs * 6 * sizeof(double),
                                cudaMemcpyHostToDevice, s));
  if (materials)
    SP_CUDA_TRY(cudaMemcpyAsync(b->d_mats, materials, (size_t)b->nrve * 4 * sizeof(double),
                                cudaMemcpyHostToDevice, s));
  return SP_OK;
}

extern "C" int sp_batch_launch(sp_batch *b, void *stream) {
  if (!b) return sp_set_error(SP_ERR_ARG, "null batch");
  Device *d;
  SP_TRY(device(&d));
  cudaStream_t s = pick_stream(stream, d);
  BatchFn fn = pick(b->o.precision, b->nrhs, b->o.threads, b->o.ctas_per_sm);
  SP_CUDA_TRY(cudaMemsetAsync(b->d_counter, 0, sizeof(int), s));
  fn<<<b->grid, b->o.threads, 0, s>>>(b->P);
  SP_CUDA_TRY(cudaGetLastError());
  b->last_launches = 1;
  return SP_OK;
}

extern "C" int sp_batch_download(sp_batch *b, double *stress, double *strain, sp_solve_info *info,
                                 void *stream) {
  if (!b) return sp_set_error(SP_ERR_ARG, "null batch");
  Device *d;
  SP_TRY(device(&d));
  cudaStream_t s = pick_stream(stream, d);
  size_t nb = (size_t)b->nrve * b->nrhs * 6 * sizeof(double);
  if (stress) SP_CUDA_TRY(cudaMemcpyAsync(stress, b->d_stress, nb, cudaMemcpyDeviceToHost, s));
  if (strain) SP_CUDA_TRY(cudaMemcpyAsync(strain, b->d_strain, nb, cudaMemcpyDeviceToHost, s));
  if (info)
    SP_CUDA_TRY(cudaMemcpyAsync(info, b->d_info, (size_t)b->nrve * sizeof(sp_solve_info),
                                cudaMemcpyDeviceToHost, s));
  return SP_OK;
}

extern "C" int sp_batch_homogenize(sp_batch *b, const double *strains, const double *materials,
                                   double *stress, double *strain, sp_solve_info *info,
                                   void *stream) {
  if (!b) return sp_set_error(SP_ERR_ARG, "null batch");
  Device *d;
  SP_TRY(device(&d));
  cudaStream_t s = pick_stream(stream, d);
  SP_TRY(sp_batch_upload(b, strains, materials, s));
  SP_TRY(sp_batch_launch(b, s));
  SP_TRY(sp_batch_download(b, stress, strain, info, s));
  SP_CUDA_TRY(cudaStreamSynchronize(s));
  if (info)
    for (int i = 0; i < b->nrve; i++)
      if (info[i].status) return sp_set_error(SP_ERR_NOCONV, "RVE %d did not converge (relres %.3e)", i, info[i].relres);
  return SP_OK;
}

extern "C" int sp_batch_last_launches(const sp_batch *b, int *launches) {
  if (!b || !launches) return sp_set_error(SP_ERR_ARG, "null argument");
  *launches = b->last_launches;
  return SP_OK;
}
