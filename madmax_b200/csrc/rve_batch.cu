// rve_batch.cu -- batched, mixed-precision homogenization of many RVEs in
// one persistent launch.
//
// Each CTA takes the next RVE from a work counter (largest meshes first) and
// runs the whole micro solve of micro/src/homogenize.c:175-225 for all load
// cases of that RVE on its own:
//   1. element operators (D, Ke = sum B^T D B w, Bbar) in shared memory;
//   2. the inner operator: by default (SP_OP_STENCIL) no matrix at all --
//      the element-type stencil reads the node's 27 neighbour blocks from a
//      table of the two materials' element blocks in shared memory, and only
//      the Jacobi diagonal is formed; with SP_OP_ELL the RVE's FP32 ELL
//      values are assembled by the 8-colour conflict-free scatter, with
//      Dirichlet rows/columns, into a node-sliced copy;
//   3. refinement loop: FP64 residual b = -K u from the FP64 element
//      operators (the "true" residual), FP32 Jacobi-PCG on the inner
//      operator for the correction A x = b (reliable updates: the search
//      direction carries over between corrections), u += x in FP64, until
//      ||b_k|| <= rtol ||b_k,0||;
//   4. FP64 volume averages of strain and stress per load case.
// A CTA never waits on another CTA, so the kernel needs no grid barrier and
// no co-residency guarantee.  All reductions are CTA-local and deterministic:
// a RVE's result does not depend on which CTA solves it or on what else is
// in the batch.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <array>
#include <map>
#include <mutex>
#include <vector>

#include "rve_batch_kernel.cuh"

namespace sp {

// ------------------------------------------------------------- dispatch ---

SP_BATCH_SHAPES(SP_BATCH_EXTERN, float, 1)
SP_BATCH_SHAPES(SP_BATCH_EXTERN, float, 6)
SP_BATCH_SHAPES(SP_BATCH_EXTERN, float, 8)
SP_BATCH_SHAPES_FP64(SP_BATCH_EXTERN, double, 1)
SP_BATCH_SHAPES_FP64(SP_BATCH_EXTERN, double, 6)
SP_BATCH_SHAPES_FP64(SP_BATCH_EXTERN, double, 8)

struct Shape {
  int threads, ctas, cluster, op;
};

constexpr int SP_TUNE_MAX = 8;
struct TuneRecord {
  int n = 0, best = 0, cached = 0;
  Shape shape[SP_TUNE_MAX];
  double rate[SP_TUNE_MAX];
};

template <typename T, int K>
static BatchFn pick_shape(const Shape &s) {
#define SP_BATCH_MATCH(T_, K_, NT, MINB, CL, OP) \
  if (s.threads == NT && s.ctas == MINB && s.cluster == CL && s.op == OP) \
    return k_batch<T_, K_, NT, MINB, CL, OP>;
  if constexpr (sizeof(T) == 4) {
    SP_BATCH_SHAPES(SP_BATCH_MATCH, T, K)
  } else {
    SP_BATCH_SHAPES_FP64(SP_BATCH_MATCH, T, K)
  }
#undef SP_BATCH_MATCH
  return nullptr;
}

static BatchFn pick(int prec, int K, const Shape &s) {
  if (prec == SP_PREC_FP64) {
    if (K == 1) return pick_shape<double, 1>(s);
    if (K <= 6) return pick_shape<double, 6>(s);
    return pick_shape<double, 8>(s);
  }
  if (K == 1) return pick_shape<float, 1>(s);
  if (K <= 6) return pick_shape<float, 6>(s);
  return pick_shape<float, 8>(s);
}

static int kpad(int nrhs) { return nrhs == 1 ? 1 : (nrhs <= 6 ? 6 : 8); }

// the kernel variant of an operator and boundary condition
static int kernel_op(const sp_batch_opts &o) {
  return (o.op == SP_OP_STENCIL && o.bc == SP_BC_PERIODIC) ? SP_OP_STENCIL_PER : o.op;
}

// A CTA shape's kernel, dynamic shared memory and persistent grid (as many
// clusters as can be resident at once); returns an error for a shape that is
// not instantiated or cannot be resident.
static int shape_setup(const sp_batch_opts &o, int kp, const Device *d, const Shape &sh,
                       BatchFn *fn_out, int *dyn_out, int *grid_out) {
  BatchFn fn = pick(o.precision, kp, sh);
  if (!fn)
    return sp_set_error(SP_ERR_ARG, "sp_batch_create: no kernel for %d threads x %d CTAs/SM, "
                        "cluster %d, %s operator in this precision", sh.threads, sh.ctas,
                        sh.cluster, o.op == SP_OP_ELL ? "assembled" : "stencil");
  int g = d->nsm * sh.ctas;
  const int dyn = sp_batch_dyn_smem(o.precision == SP_PREC_MIXED, kp, sh.op,
                                    sh.threads * sh.ctas <= 512);
  if (dyn && cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  dyn) != cudaSuccess) {
    cudaGetLastError();
    return sp_set_error(SP_ERR_CUDA, "sp_batch_create: %d bytes of dynamic shared memory refused",
                        dyn);
  }
  if (sh.cluster == 1) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void *)fn, sh.threads, dyn) !=
            cudaSuccess ||
        nb < 1) {
      cudaGetLastError();
      return sp_set_error(SP_ERR_CUDA, "sp_batch_create: %d-thread CTAs cannot be resident",
                          sh.threads);
    }
    g = d->nsm * std::min(sh.ctas, nb);
  } else {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(g);
    cfg.blockDim = dim3(sh.threads);
    cfg.dynamicSmemBytes = dyn;
    cudaLaunchAttribute at;
    at.id = cudaLaunchAttributeClusterDimension;
    at.val.clusterDim.x = sh.cluster;
    at.val.clusterDim.y = 1;
    at.val.clusterDim.z = 1;
    cfg.attrs = &at;
    cfg.numAttrs = 1;
    int ncl = 0;
    if (cudaOccupancyMaxActiveClusters(&ncl, (void *)fn, &cfg) != cudaSuccess || ncl < 1) {
      cudaGetLastError();
      return sp_set_error(SP_ERR_CUDA, "sp_batch_create: cluster of %d CTAs cannot be resident",
                          sh.cluster);
    }
    g = std::min(g, ncl * sh.cluster);
  }
  *fn_out = fn;
  *dyn_out = dyn;
  *grid_out = g;
  return SP_OK;
}

static int launch_shape(BatchFn fn, const Shape &sh, int grid, int dyn, cudaStream_t s,
                        const BatchParams &P) {
  if (sh.cluster == 1) {
    fn<<<grid, sh.threads, dyn, s>>>(P);
  } else {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(sh.threads);
    cfg.dynamicSmemBytes = dyn;
    cfg.stream = s;
    cudaLaunchAttribute at;
    at.id = cudaLaunchAttributeClusterDimension;
    at.val.clusterDim.x = sh.cluster;
    at.val.clusterDim.y = 1;
    at.val.clusterDim.z = 1;
    cfg.attrs = &at;
    cfg.numAttrs = 1;
    SP_CUDA_TRY(cudaLaunchKernelEx(&cfg, fn, P));
  }
  SP_CUDA_TRY(cudaGetLastError());
  return SP_OK;
}

// ------------------------------------------------------------ autotuner ---
//
// The instantiated one-CTA-per-RVE shapes of a kernel variant: threads per
// CTA x CTAs per SM, which fixes the registers a thread may use (65,536 /
// (threads x CTAs)): 128 at 512 x 1, 64 at 512 x 2 / 256 x 4 / 1024 x 1.
static std::vector<Shape> tune_candidates(const sp_batch_opts &o) {
  const int kop = kernel_op(o);
  if (kop == SP_OP_STENCIL_PER || o.precision == SP_PREC_FP64)
    return {{512, 1, 1, kop}, {512, 2, 1, kop}};
  if (kop == SP_OP_STENCIL)
    return {{512, 1, 1, kop}, {512, 2, 1, kop}, {256, 2, 1, kop}, {256, 4, 1, kop},
            {1024, 1, 1, kop}};
  return {{512, 1, 1, kop}, {512, 2, 1, kop}, {256, 2, 1, kop}, {256, 4, 1, kop}};
}

using TuneKey = std::array<int, 5>;  // device, kernel operator, precision, load cases, size class
static std::mutex g_tune_mu;
static std::map<TuneKey, TuneRecord> g_tune_cache;

// estimated cost of one RVE solve: dof x largest mesh edge (CG iterations
// grow with the edge)
static double rve_work(const MeshGeo &g) {
  return (double)g.ndof * std::max(g.nex, std::max(g.ney, g.nez));
}

}  // namespace sp

using namespace sp;

struct sp_batch_s {
  int nrve = 0, nrhs = 6, kp = 6, dev = -1, grid = 0, last_launches = 0;
  int dyn_smem = 0;  // dynamic shared memory of the kernel (pattern table)
  std::vector<long long> etype_off;  // per RVE: its materials in d_etype
  std::vector<int> nelm;
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
  void *d_ws_v = nullptr, *d_ws_dinv = nullptr;
  size_t bytes = 0;
  TuneRecord tune;  // the autotuner's trial (tune.n == 0: shape fixed by the caller)
  int tune_slots = 0;  // work spaces allocated while the autotuner runs
};

// Time every candidate shape on the same sample of the batch: 2 G RVEs, G
// the largest candidate grid, taken at even steps through the largest-first
// order (the batch's size mix, in its order), after an empty launch that
// loads the kernel.  The rate is the sample's estimated work over the
// launch time.  (A sample of 2 grids per candidate gives every candidate
// two waves, while the whole batch gives a small grid many more: the tail
// of the last wave then weighs on a large grid's trial less than on its
// real launches.)  The trial writes the outputs of the RVEs it solves; the
// batch's own launches overwrite them.
static int tune_trial(sp_batch *b, const std::vector<Shape> &cands, const std::vector<int> &order,
                      const std::vector<double> &work, const Device *d, TuneRecord *rec) {
  cudaStream_t s = d->stream;
  const int nrve = b->nrve;
  int *d_trial = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = SP_OK;
  if (cudaMalloc((void **)&d_trial, (size_t)nrve * sizeof(int)) != cudaSuccess ||
      cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    cudaGetLastError();
    rc = sp_set_error(SP_ERR_CUDA, "sp_batch_create: autotuner set-up failed");
  }
  rec->n = 0;
  double best = -1.0;
  // the common sample: 2 x the largest candidate grid (the work spaces hold
  // that many slots)
  const int T = std::min(nrve, 2 * b->tune_slots);
  std::vector<int> sample(T);
  double wsum = 0.0;
  for (int j = 0; j < T; j++) {
    sample[j] = order[(size_t)j * nrve / T];
    wsum += work[sample[j]];
  }
  if (!rc && cudaMemcpyAsync(d_trial, sample.data(), T * sizeof(int), cudaMemcpyHostToDevice, s))
    rc = sp_set_error(SP_ERR_CUDA, "sp_batch_create: autotuner upload failed");
  for (size_t c = 0; c < cands.size() && !rc && rec->n < SP_TUNE_MAX; c++) {
    BatchFn fn;
    int dyn, grid;
    if (shape_setup(b->o, b->kp, d, cands[c], &fn, &dyn, &grid) != SP_OK) continue;  // not resident
    if (grid / cands[c].cluster > b->tune_slots) continue;  // work spaces sized for fewer
    BatchParams P = b->P;
    P.order = d_trial;
    if (cudaMemsetAsync(b->d_counter, 0, sizeof(int), s)) {
      rc = sp_set_error(SP_ERR_CUDA, "sp_batch_create: autotuner upload failed");
      break;
    }
    P.nrve = 0;  // loads the kernel; every CTA finds no work
    rc = launch_shape(fn, cands[c], grid, dyn, s, P);
    if (rc) break;
    P.nrve = T;
    if (cudaMemsetAsync(b->d_counter, 0, sizeof(int), s) || cudaEventRecord(e0, s)) {
      rc = sp_set_error(SP_ERR_CUDA, "sp_batch_create: autotuner launch failed");
      break;
    }
    rc = launch_shape(fn, cands[c], grid, dyn, s, P);
    if (rc) break;
    float ms = 0.f;
    if (cudaEventRecord(e1, s) || cudaEventSynchronize(e1) || cudaEventElapsedTime(&ms, e0, e1)) {
      rc = sp_set_error(SP_ERR_CUDA, "sp_batch_create: autotuner timing failed");
      break;
    }
    const int k = rec->n++;
    rec->shape[k] = cands[c];
    rec->rate[k] = wsum / std::max(ms, 1e-3f);
    if (rec->rate[k] > best) {
      best = rec->rate[k];
      rec->best = k;
    }
  }
  if (!rc && rec->n == 0) rc = sp_set_error(SP_ERR_CUDA, "sp_batch_create: no CTA shape can run");
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(d_trial);
  return rc;
}


extern "C" void sp_batch_opts_default(sp_batch_opts *o) {
  memset(o, 0, sizeof(*o));
  o->nrhs = 6;
  o->precision = SP_PREC_MIXED;
  o->rtol = 1e-8;
  o->inner_rtol = 0.0;  // chosen by precision at create time
  o->max_outer = 8;
  o->max_inner = 4000;
  o->threads = 0;      // chosen per operator at create time
  o->lanes_per_row = 0;
  o->ctas_per_sm = 0;
  o->cluster = 1;
  o->op = SP_OP_STENCIL;
  o->bc = SP_BC_AFFINE;
}

extern "C" int sp_batch_destroy(sp_batch *b) {
  if (!b) return SP_OK;
  void *bufs[] = {b->d_plans, b->d_rves, b->d_order, b->d_counter, b->d_vals, b->d_dinv,
                  b->d_etype, b->d_strains, b->d_mats, b->d_stress, b->d_strain, b->d_info,
                  b->d_ws_u, b->d_ws_v, b->d_ws_dinv};
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
  // CTA shape: 512 threads x 1 or 2 CTAs per SM, 256 threads x 2 or 4, or
  // (stencil operator) 1024 threads x 1.  Unset: 512 x 1 for the stencil
  // (128 registers a thread: as fast as 1024 x 1 on affine n = 16-20 and
  // 20-26% faster on n = 8-12; 2.3x faster than 512 x 2 under periodic
  // conditions, whose 64-register build spills), 512 x 2 for the assembled
  // operator.
  if (o.tune != SP_TUNE_AUTO && o.tune != SP_TUNE_OFF)
    return sp_set_error(SP_ERR_ARG, "sp_batch_create: tune must be SP_TUNE_AUTO or SP_TUNE_OFF");
  // the autotuner picks the shape when the caller leaves it open
  const bool tune = o.threads == 0 && o.ctas_per_sm == 0 && o.cluster <= 1 && o.tune == SP_TUNE_AUTO;
  const bool one = o.op == SP_OP_STENCIL && o.cluster <= 1;
  if (o.threads == 0) o.threads = 512;
  if (o.ctas_per_sm == 0) o.ctas_per_sm = (o.threads == 1024 || (one && o.threads == 512)) ? 1 : 2;
  if (o.threads != 256 && o.threads != 512 && o.threads != 1024)
    return sp_set_error(SP_ERR_ARG, "sp_batch_create: threads must be 256, 512 or 1024");
  if (o.threads == 1024 && o.ctas_per_sm != 1)
    return sp_set_error(SP_ERR_ARG, "sp_batch_create: 1024-thread CTAs run 1 per SM");
  if (o.threads == 512 && o.ctas_per_sm != 1 && o.ctas_per_sm != 2)
    return sp_set_error(SP_ERR_ARG, "sp_batch_create: 512-thread CTAs run 1 or 2 per SM");
  if (o.threads == 256 && o.ctas_per_sm != 2 && o.ctas_per_sm != 4)
    return sp_set_error(SP_ERR_ARG, "sp_batch_create: 256-thread CTAs run 2 or 4 per SM");
  o.lanes_per_row = 0;  // the node-sliced SpMM uses one lane per node (3 rows)
  if (o.cluster == 0) o.cluster = 1;
  if (o.cluster != 1 && o.cluster != 2 && o.cluster != 4 && o.cluster != 8)
    return sp_set_error(SP_ERR_ARG, "sp_batch_create: cluster must be 1, 2, 4 or 8");
  if (o.op != SP_OP_ELL && o.op != SP_OP_STENCIL)
    return sp_set_error(SP_ERR_ARG, "sp_batch_create: unknown operator");
  if (o.bc != SP_BC_AFFINE && o.bc != SP_BC_PERIODIC)
    return sp_set_error(SP_ERR_ARG, "sp_batch_create: unknown boundary condition");
  if (o.bc == SP_BC_PERIODIC && o.op != SP_OP_STENCIL)
    return sp_set_error(SP_ERR_ARG, "sp_batch_create: periodic conditions need the stencil operator");
  if (o.bc == SP_BC_PERIODIC && (o.cluster != 1 || o.threads != 512))
    return sp_set_error(SP_ERR_ARG, "sp_batch_create: periodic conditions run 512-thread CTAs, no cluster");
  if (o.max_outer < 1) o.max_outer = 8;
  if (o.max_inner < 1) o.max_inner = 4000;
  if (!(o.rtol > 0)) o.rtol = 1e-8;
  // FP32 corrections of 3e-3 from the affine start, each replaced by the
  // FP64 residual, keep the rounding in the volume averages small; FP64
  // corrections, and periodic ones (whose element-form residual makes extra
  // refinement steps dear and which stay within 2e-9 of the oracle at 1e-4),
  // run longer
  if (!(o.inner_rtol > 0))
    o.inner_rtol = (o.precision == SP_PREC_FP64 || o.bc == SP_BC_PERIODIC) ? 1e-4 : 3e-3;
  for (int i = 0; i < nrve; i++)
    for (int k = 0; k < 3; k++) {
      if (descs[i].n[k] < 1 || descs[i].len[k] <= 0)
        return sp_set_error(SP_ERR_ARG, "sp_batch_create: RVE %d has a bad mesh", i);
      if (o.bc == SP_BC_PERIODIC && descs[i].n[k] < 2)
        return sp_set_error(SP_ERR_ARG, "sp_batch_create: periodic RVE %d needs 2 elements per axis", i);
    }
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
    eoff += (g.nelm + 15) / 16 * 16;
    if (o.op == SP_OP_ELL) {  // assembled values and diagonal kept per RVE
      voff += (long long)g.nn_pad * 243;
      doff += 3LL * g.nn_pad;
    }
    maxdof = std::max(maxdof, g.ndof);
    maxnp = std::max(maxnp, g.nn_pad);
    b->etype_off.push_back(r.etype_off);
    b->nelm.push_back(g.nelm);
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
  // persistent grid: as many clusters as can be resident at once.  Left to
  // the autotuner, the shape comes from the cache, or from a trial below
  // once the batch's data are on the device (its work spaces sized for the
  // largest candidate grid until then).
  std::vector<Shape> cands;
  std::vector<double> work(nrve);
  TuneKey tkey = {};
  bool trial = false;
  if (tune && !rc) {
    std::map<int, double> by_edge;
    for (int i = 0; i < nrve; i++) {
      const MeshGeo &g = hplans[hrves[i].plan].geo;
      work[i] = rve_work(g);
      by_edge[std::max(g.nex, std::max(g.ney, g.nez))] += work[i];
    }
    int dom = 0;
    double wmax = -1.0;
    for (auto &kv : by_edge)
      if (kv.second > wmax) {
        wmax = kv.second;
        dom = kv.first;
      }
    tkey = {d->id, kernel_op(o), o.precision, kp, dom};
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      auto it = g_tune_cache.find(tkey);
      if (it != g_tune_cache.end()) {
        b->tune = it->second;
        b->tune.cached = 1;
      }
    }
    if (b->tune.n) {
      const Shape &w = b->tune.shape[b->tune.best];
      o.threads = w.threads;
      o.ctas_per_sm = w.ctas;
    } else {
      trial = true;
      cands = tune_candidates(o);
      for (const Shape &c : cands) {
        BatchFn fn;
        int dyn, grid;
        if (shape_setup(o, kp, d, c, &fn, &dyn, &grid) == SP_OK)
          b->tune_slots = std::max(b->tune_slots, grid / c.cluster);
      }
      cudaGetLastError();
    }
    b->o = o;
  }
  if (!rc) {
    Shape sh{o.threads, o.ctas_per_sm, o.cluster, kernel_op(o)};
    BatchFn fn;
    rc = shape_setup(o, kp, d, sh, &fn, &b->dyn_smem, &b->grid);
  }
  size_t stride = (size_t)kp * 3 * maxnp;
  // (3*maxnp >= maxdof; a multiple of 96, so every slot starts 16-byte aligned)
  size_t drm_stride = (size_t)3 * maxnp;
  const bool ell = o.op == SP_OP_ELL;
  size_t *acct = &b->bytes;
  if (!rc) rc = dmalloc((void **)&b->d_plans, hplans.size() * sizeof(BatchPlan), acct);
  if (!rc) rc = dmalloc((void **)&b->d_rves, nrve * sizeof(BatchRve), acct);
  if (!rc) rc = dmalloc((void **)&b->d_order, nrve * sizeof(int), acct);
  if (!rc) rc = dmalloc((void **)&b->d_counter, 256, acct);
  if (!rc && ell) rc = dmalloc(&b->d_vals, (size_t)voff * tsz, acct);
  if (!rc && ell) rc = dmalloc(&b->d_dinv, (size_t)doff * tsz, acct);
  if (!rc) rc = dmalloc((void **)&b->d_etype, eoff, acct);
  if (!rc) rc = dmalloc((void **)&b->d_strains, (size_t)nrve * nrhs * 6 * sizeof(double), acct);
  if (!rc) rc = dmalloc((void **)&b->d_mats, (size_t)nrve * 4 * sizeof(double), acct);
  if (!rc) rc = dmalloc((void **)&b->d_stress, (size_t)nrve * nrhs * 6 * sizeof(double), acct);
  if (!rc) rc = dmalloc((void **)&b->d_strain, (size_t)nrve * nrhs * 6 * sizeof(double), acct);
  if (!rc) rc = dmalloc((void **)&b->d_info, (size_t)nrve * sizeof(sp_solve_info), acct);
  // one work space per cluster (for the largest candidate grid while tuning)
  const size_t slots = (size_t)std::max(b->grid / o.cluster, b->tune_slots);
  if (!rc) rc = dmalloc((void **)&b->d_ws_u, slots * stride * sizeof(double), acct);
  if (!rc) rc = dmalloc(&b->d_ws_v, slots * 4 * stride * tsz, acct);
  // stencil: one Jacobi diagonal [3][max nn_pad] per work space
  if (!rc && !ell) rc = dmalloc(&b->d_ws_dinv, slots * drm_stride * tsz, acct);
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
  P.drm_stride = drm_stride;
  P.ws_dinv = b->d_ws_dinv;
  P.counter = b->d_counter;
  P.rtol = o.rtol;
  P.inner_rtol = o.inner_rtol;
  P.max_outer = o.max_outer;
  P.max_inner = o.max_inner;
  if (trial) {
    rc = tune_trial(b, cands, order, work, d, &b->tune);
    if (!rc) {
      const Shape &w = b->tune.shape[b->tune.best];
      b->o.threads = w.threads;
      b->o.ctas_per_sm = w.ctas;
      BatchFn fn;
      rc = shape_setup(b->o, kp, d, w, &fn, &b->dyn_smem, &b->grid);
    }
    if (!rc) {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      g_tune_cache[tkey] = b->tune;
    }
    // keep only the work spaces the chosen grid uses
    const size_t keep = (size_t)(b->grid / b->o.cluster);
    if (!rc && keep < slots) {
      cudaFree(b->d_ws_u);
      cudaFree(b->d_ws_v);
      cudaFree(b->d_ws_dinv);
      b->d_ws_u = nullptr;
      b->d_ws_v = b->d_ws_dinv = nullptr;
      b->bytes -= slots * (stride * sizeof(double) + 4 * stride * tsz + (ell ? 0 : drm_stride * tsz));
      if (!rc) rc = dmalloc((void **)&b->d_ws_u, keep * stride * sizeof(double), acct);
      if (!rc) rc = dmalloc(&b->d_ws_v, keep * 4 * stride * tsz, acct);
      if (!rc && !ell) rc = dmalloc(&b->d_ws_dinv, keep * drm_stride * tsz, acct);
      P.ws_u = b->d_ws_u;
      P.ws_v = b->d_ws_v;
      P.ws_dinv = b->d_ws_dinv;
    }
    b->tune_slots = 0;
    if (rc) {
      sp_batch_destroy(b);
      return rc;
    }
  }
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

extern "C" int sp_batch_set_etype(sp_batch *b, int rve, const unsigned char *etype, void *stream) {
  if (!b || !etype) return sp_set_error(SP_ERR_ARG, "sp_batch_set_etype: null argument");
  if (rve < 0 || rve >= b->nrve)
    return sp_set_error(SP_ERR_ARG, "sp_batch_set_etype: RVE %d of %d", rve, b->nrve);
  for (int e = 0; e < b->nelm[rve]; e++)
    if (etype[e] > 1)
      return sp_set_error(SP_ERR_ARG, "sp_batch_set_etype: element %d has material %d (0 or 1)", e,
                          (int)etype[e]);
  Device *d;
  SP_TRY(device(&d));
  cudaStream_t s = pick_stream(stream, d);
  SP_CUDA_TRY(cudaMemcpyAsync(b->d_etype + b->etype_off[rve], etype, (size_t)b->nelm[rve],
                              cudaMemcpyHostToDevice, s));
  // ordered before the stream's next launch; a pinned source is read
  // asynchronously, so the caller keeps it until the stream reaches the copy
  return SP_OK;
}

extern "C" int sp_batch_launch(sp_batch *b, void *stream) {
  if (!b) return sp_set_error(SP_ERR_ARG, "null batch");
  Device *d;
  SP_TRY(device(&d));
  cudaStream_t s = pick_stream(stream, d);
  Shape sh{b->o.threads, b->o.ctas_per_sm, b->o.cluster, kernel_op(b->o)};
  BatchFn fn = pick(b->o.precision, b->nrhs, sh);
  SP_CUDA_TRY(cudaMemsetAsync(b->d_counter, 0, sizeof(int), s));
  SP_TRY(launch_shape(fn, sh, b->grid, b->dyn_smem, s, b->P));
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

extern "C" int sp_batch_tune_report(const sp_batch *b, int max, int *threads, int *ctas_per_sm,
                                    double *rate, int *ntried, int *chosen, int *from_cache) {
  if (!b) return sp_set_error(SP_ERR_ARG, "null batch");
  const TuneRecord &r = b->tune;
  for (int k = 0; k < r.n && k < max; k++) {
    if (threads) threads[k] = r.shape[k].threads;
    if (ctas_per_sm) ctas_per_sm[k] = r.shape[k].ctas;
    if (rate) rate[k] = r.rate[k];
  }
  if (ntried) *ntried = r.n;
  if (chosen) *chosen = r.best;
  if (from_cache) *from_cache = r.cached;
  return SP_OK;
}

extern "C" int sp_batch_last_launches(const sp_batch *b, int *launches) {
  if (!b || !launches) return sp_set_error(SP_ERR_ARG, "null argument");
  *launches = b->last_launches;
  return SP_OK;
}

extern "C" int sp_batch_shape(const sp_batch *b, int *threads, int *ctas_per_sm, int *grid) {
  if (!b) return sp_set_error(SP_ERR_ARG, "null batch");
  if (threads) *threads = b->o.threads;
  if (ctas_per_sm) *ctas_per_sm = b->o.ctas_per_sm;
  if (grid) *grid = b->grid;
  return SP_OK;
}
