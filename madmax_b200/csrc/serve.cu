// serve.cu -- device-resident request loop (continuous batching).
//
// Stands in for the micro process's request loop (micro/src/main.c:114-153)
// and its message_t exchange (inc/comm.h:18-27): a request carries a macro
// strain and a geometry id and returns the volume-averaged stress and the
// 6x6 tangent by the finite differences of micro/src/homogenize.c:59-94
// (delta 0.005), i.e. 7 load cases eps, eps + delta e_i solved together.
//
// Layout of the running loop (one persistent launch, relaunched by the host
// when it has gone idle):
//   - the host appends requests to a ring in mapped pinned memory and
//     publishes the count (`tail`);
//   - CTA 0 is a dispatcher: it polls the host count, copies new requests
//     into a device ring and publishes the device count;
//   - every other CTA is a worker slot: it claims the next published request
//     (atomic counter), solves it with the same per-RVE solve as the batched
//     kernel (rve_solve.cuh) -- on the element-type stencil (default) or on
//     the geometry's resident FP32 ELL matrix -- warm-started from that
//     geometry's previous solution, writes the result to mapped memory and
//     raises the request's done flag.  The warm start is a first-order
//     prediction from the previous request's 7 solutions (u(eps) and
//     u(eps + delta e_i) give the derivative of u in every strain direction),
//     or (SP_WARM_LAST) the previous request's solution of each load case
//     as it is.
// A request is picked up as soon as any slot is free, while other requests
// are still solving: their work overlaps on the device.  Every wait is
// bounded (idle_spin_limit polls); on expiry the CTA returns and the host
// relaunches the loop when new work arrives.
#include <time.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "rve_solve.cuh"
#include "sp_cuda.h"

namespace sp {

constexpr int SERVE_NT = 512;
constexpr int SERVE_K = 7;  // eps and eps + delta e_i, i = 0..5 (component-major vectors need no padding)
constexpr int SERVE_NRHS = 7;
constexpr double FD_DELTA = 0.005;  // micro/inc/micro.h:29

struct ServeGeom {
  MeshGeo g;
  const int *cols;
  const int *nbr;
  float *vals;  // node-sliced ELL values [nn_pad*243] (assembled operator only)
  float *dinv;  // component-major [3][nn_pad]
  const uint8_t *etype;
  double *Ke;   // [2][576]
  double *D;    // [72]
  double *Bbar; // [144]
  double *warm;     // [SERVE_K][3][nn_pad] solutions of the previous request
  double *warm_eps; // [SERVE_K][6] its load-case strains
  double *gram;     // [6][6] b_i . b_j of the unit-strain right-hand sides b_i = -K u_bc(e_i)
  const int *color_elems;
  const uint8_t *slot;
  int color_off[9];
  int has_warm;
};

struct ServeReq {
  int geom, pad;
  double strain[6];
};

struct ServeRes {
  double stress[6];
  double tangent[36];
  sp_solve_info info;
  volatile long long done; // ticket + 1 once the result is valid
};

struct ServeCtl { // mapped host memory
  volatile long long tail;
  volatile int stop;
  int pad;
};

struct ServeDev { // device memory
  unsigned long long claim;
  volatile long long dtail;
  volatile int dstop;
  volatile int dispatcher_gone;
  int err;
};

struct ServeParams {
  ServeGeom *geoms;
  int ngeom, cap;
  const ServeReq *hreq; // mapped ring
  ServeReq *dreq;       // device ring
  ServeRes *res;        // mapped ring
  const ServeCtl *ctl;
  ServeDev *dev;
  double *ws_u;
  float *ws_v;
  size_t stride;
  double rtol, inner_rtol, refine_rtol;
  int max_outer, max_inner, idle_limit;
  int warm_last;  // SP_WARM_LAST: start from the last solutions, no prediction
};

// Prepare every geometry once (a CTA takes geometries in turn): element
// operators kept in global memory and the Jacobi diagonal; for the assembled
// operator also the FP32 ELL values by the coloured scatter into the CTA's
// row-major scratch, Dirichlet rows/columns, then the node-sliced copy the
// solve reads.
template <int OP>
__global__ void __launch_bounds__(SERVE_NT) k_serve_assemble(ServeGeom *geoms, int ngeom,
                                                             const double *mats, float *scratch,
                                                             size_t rm_stride, size_t drm_stride) {
  __shared__ double sKe[2 * SP_KE], sD[72], sdsh[192], sB[144];
  __shared__ float sKe32[2 * SP_KE];
  const int t = threadIdx.x;
  float *vrm = scratch + (size_t)blockIdx.x * (rm_stride + drm_stride);
  float *drm = vrm + rm_stride;
  for (int gi = blockIdx.x; gi < ngeom; gi += gridDim.x) {
    ServeGeom &G = geoms[gi];
    MeshGeo g = G.g;
    if (t < 2) iso_D(mats[gi * 4 + 2 * t], mats[gi * 4 + 2 * t + 1], sD + 36 * t);
    double h[3] = {g.hx, g.hy, g.hz};
    elem_ops_stage1(t, SERVE_NT, h, sdsh);
    __syncthreads();
    elem_ops_stage2(t, SERVE_NT, h, sdsh, sD, 2, sKe, sB);
    __syncthreads();
    for (int i = t; i < 2 * SP_KE; i += SERVE_NT) {
      sKe32[i] = (float)sKe[i];
      G.Ke[i] = sKe[i];
    }
    for (int i = t; i < 72; i += SERVE_NT) G.D[i] = sD[i];
    for (int i = t; i < 144; i += SERVE_NT) G.Bbar[i] = sB[i];
    if constexpr (OP == SP_OP_STENCIL) {
      stencil_dinv<float>(t, SERVE_NT, g, G.etype, sKe, G.dinv);
      __syncthreads();
      continue;
    }
    ell_zero<float>(t, SERVE_NT, vrm, g.ndof);
    __syncthreads();
    for (int c = 0; c < 8; c++) {
      if (G.color_off[c + 1] > G.color_off[c])
        scatter_colour<float>(t, SERVE_NT, g, G.color_elems, G.color_off[c], G.color_off[c + 1],
                              G.slot, G.etype, sKe32, vrm);
      __syncthreads();
    }
    bc_and_dinv<float>(t, SERVE_NT, g, G.cols, vrm, drm);
    __syncthreads();
    ns_from_rows<float>(t, SERVE_NT, g, G.cols, vrm, drm, G.vals, G.dinv);
    __syncthreads();
  }
}

// Gram matrix of every geometry's unit-strain right-hand sides: the right-
// hand side of a strain eps is linear in it, b(eps) = sum_i eps_i b_i, so its
// norm is sqrt(eps^T G eps) without a residual pass.  scratch: per CTA two
// [6][3][max nn_pad] FP64 vectors.
__global__ void __launch_bounds__(SERVE_NT) k_serve_gram(ServeGeom *geoms, int ngeom,
                                                         double *scratch, size_t stride) {
  __shared__ double sKe[2 * SP_KE];
  __shared__ double seye[36];
  __shared__ double red[33 * 21];
  const int t = threadIdx.x;
  double *u = scratch + (size_t)blockIdx.x * 2 * stride, *b = u + stride;
  for (int i = t; i < 36; i += SERVE_NT) seye[i] = (i % 7 == 0) ? 1.0 : 0.0;
  for (int gi = blockIdx.x; gi < ngeom; gi += gridDim.x) {
    ServeGeom &G = geoms[gi];
    const MeshGeo g = G.g;
    for (int i = t; i < 2 * SP_KE; i += SERVE_NT) sKe[i] = G.Ke[i];
    __syncthreads();
    affine_soa<6>(t, SERVE_NT, g, seye, 6, false, u);
    __syncthreads();
    double nrm[6] = {0, 0, 0, 0, 0, 0};
    residual_soa<6, double>(t, SERVE_NT, g, G.etype, sKe, u, b, nrm);
    __syncthreads();
    const size_t blk = (size_t)3 * g.nn_pad;
    double acc[21];
#pragma unroll
    for (int q = 0; q < 21; q++) acc[q] = 0.0;
    for (size_t i = t; i < blk; i += SERVE_NT) {
      double v[6];
#pragma unroll
      for (int q = 0; q < 6; q++) v[q] = b[q * blk + i];
      int q = 0;
#pragma unroll
      for (int a = 0; a < 6; a++)
#pragma unroll
        for (int c = a; c < 6; c++) acc[q++] += v[a] * v[c];
    }
    double tot[21];
    block_sum<21>(acc, red, tot);
    if (t == 0) {
      int q = 0;
      for (int a = 0; a < 6; a++)
        for (int c = a; c < 6; c++, q++) G.gram[a * 6 + c] = G.gram[c * 6 + a] = tot[q];
    }
    __syncthreads();
  }
}

template <int OP, int MINB>
__global__ void __launch_bounds__(SERVE_NT, MINB) k_serve(ServeParams P) {
  constexpr bool STENCIL = OP == SP_OP_STENCIL;
  // one request slot per SM (128 registers a thread): the stencil reads its
  // blocks from the pattern table, in SP_PT_BYTES of dynamic shared memory
  constexpr bool PT = STENCIL && MINB == 1;
  __shared__ double sKe[2 * SP_KE], sD[72], sB[144];
  __shared__ __align__(16) float sKB[STENCIL && !PT ? SP_KB_SIZE : 4];
  extern __shared__ __align__(16) float s_ptab[];
  __shared__ __align__(16) double sKBd[SP_KB_SIZE];  // FP64 stencil tables (residual)
  __shared__ double red[33 * 16];
  __shared__ double savg[SP_MAX_RHS * 12];
  __shared__ double seps[SERVE_K * 6];
  __shared__ double spred[SERVE_K * 6];  // warm-start predictor coefficients
  __shared__ double srn0[SERVE_K];       // right-hand-side norms from the Gram matrix
  __shared__ CgShared sh;
  __shared__ long long s_job;
  __shared__ int s_geom;
  const int t = threadIdx.x;
  ServeDev *D = P.dev;

  if (blockIdx.x == 0) {
    // dispatcher: forward host requests into the device ring
    if (t >= 32) return;
    long long seen = D->dtail;
    int idle = 0;
    for (;;) {
      long long ht = 0;
      int hstop = 0;
      if (t == 0) {
        ht = P.ctl->tail;
        hstop = P.ctl->stop;
      }
      ht = __shfl_sync(0xffffffffu, ht, 0);
      hstop = __shfl_sync(0xffffffffu, hstop, 0);
      __threadfence_system();
      if (ht > seen) {
        for (long long i = seen + t; i < ht; i += 32) {
          const volatile ServeReq *src = P.hreq + (i % P.cap);
          ServeReq *dst = P.dreq + (i % P.cap);
          dst->geom = src->geom;
          for (int k = 0; k < 6; k++) dst->strain[k] = src->strain[k];
        }
        __threadfence();
        __syncwarp();
        if (t == 0) D->dtail = ht;
        seen = ht;
        idle = 0;
      } else if (hstop) {
        if (t == 0) D->dstop = 1;
        break;
      } else if (++idle > P.idle_limit) {
        break;
      }
      __nanosleep(1000);
    }
    if (t == 0) {
      __threadfence();
      D->dispatcher_gone = 1;
    }
    return;
  }

  // a slot launched without the pattern table's shared memory serves nothing
  // (the host's waits are bounded)
  if (PT && dynamic_smem_bytes() < (unsigned)SP_PT_BYTES) return;
  double *u = P.ws_u + (size_t)blockIdx.x * P.stride;
  float *ws = P.ws_v + (size_t)blockIdx.x * 4 * P.stride;
  float *r = ws, *x = ws + P.stride, *p = ws + 2 * P.stride, *q = ws + 3 * P.stride;
  for (;;) {
    // claim the next published request (bounded wait).  The dispatcher's
    // idle limit decides when the loop returns: a slot leaves when the
    // dispatcher has left or stop is set.  Its own bound, 8 times the
    // dispatcher's, is a safeguard only: slots that left one by one on their
    // own idle count would starve a loop whose dispatcher still runs.
    if (t == 0) {
      long long job = -1;
      long long idle = 0;
      for (;;) {
        unsigned long long h = *(volatile unsigned long long *)&D->claim;
        long long dt = D->dtail;
        if ((long long)h < dt) {
          if (atomicCAS(&D->claim, h, h + 1) == h) {
            job = (long long)h;
            break;
          }
          continue;
        }
        if (D->dstop || D->dispatcher_gone || ++idle > 8LL * P.idle_limit) break;
        __nanosleep(500);
      }
      __threadfence();
      s_job = job;
      if (job >= 0) {
        const ServeReq *rq = P.dreq + (job % P.cap);
        int gid = __ldcg(&rq->geom);
        s_geom = gid;
        for (int k = 0; k < SERVE_K * 6; k++) seps[k] = 0.0;
        for (int k = 0; k < 6; k++) {
          double e = __ldcg(&rq->strain[k]);
          for (int c = 0; c < SERVE_NRHS; c++) seps[c * 6 + k] = e;
        }
        for (int i = 0; i < 6; i++) seps[(i + 1) * 6 + i] = seps[(i + 1) * 6 + i] + FD_DELTA;
      }
    }
    __syncthreads();
    long long job = s_job;
    int gid = s_geom;
    if (job < 0) break;
    ServeRes *out = P.res + (job % P.cap);
    if (gid < 0 || gid >= P.ngeom) {
      if (t == 0) {
        out->info.status = SP_ERR_RANGE;
        out->info.outer_its = out->info.inner_its = 0;
        out->info.relres = 0.0;
        __threadfence_system();
        out->done = job + 1;
      }
      __syncthreads();
      continue;
    }
    ServeGeom &G = P.geoms[gid];
    const MeshGeo g = G.g;
    for (int i = t; i < 2 * SP_KE; i += SERVE_NT) sKe[i] = G.Ke[i];
    for (int i = t; i < 72; i += SERVE_NT) sD[i] = G.D[i];
    for (int i = t; i < 144; i += SERVE_NT) sB[i] = G.Bbar[i];
    // warm start from the geometry's previous request, whose solutions are
    // u(e0) and u(e0 + d e_i), i = 0..5: the first-order predictor
    //   u(e) ~ u(e0) + sum_i (e - e0)_i (u(e0 + d e_i) - u(e0)) / d
    // (exact for linear materials up to the previous solves' tolerance) for
    // every load case inside; eps . x on the boundary (below)
    const size_t nu = (size_t)SERVE_K * 3 * g.nn_pad;
    const bool warm = *(volatile int *)&G.has_warm;
    if (t < SERVE_K) {
      // ||b(eps_k)||^2 = eps_k^T G eps_k
      double s = 0.0;
      for (int a = 0; a < 6; a++)
        for (int c = 0; c < 6; c++) s += seps[t * 6 + a] * __ldg(G.gram + a * 6 + c) * seps[t * 6 + c];
      srn0[t] = sqrt(fmax(s, 0.0));
    }
    if (warm && P.warm_last) {
      // the last request's solution of each load case, shifted by the affine
      // field of the strain difference: u_last + (eps - eps_last) . x (the
      // boundary values become eps . x; exact for a homogeneous RVE, and
      // close when consecutive strains on a geometry are close)
      const size_t blk = (size_t)3 * g.nn_pad;
      for (size_t i = t; i < nu; i += SERVE_NT) {
        const int k = (int)(i / blk), rem = (int)(i % blk);
        const int d = rem / g.nn_pad, node = rem % g.nn_pad;
        double v = __ldcg(G.warm + i);
        if (node < g.nn) {
          const int ix = node % g.nx, iy = (node / g.nx) % g.ny, iz = node / (g.nx * g.ny);
          double de[6];
          for (int c = 0; c < 6; c++) de[c] = seps[k * 6 + c] - __ldcg(G.warm_eps + k * 6 + c);
          const double X = ix * g.hx, Y = iy * g.hy, Z = iz * g.hz;
          v += d == 0 ? de[0] * X + 0.5 * de[3] * Y + 0.5 * de[5] * Z
                      : (d == 1 ? 0.5 * de[3] * X + de[1] * Y + 0.5 * de[4] * Z
                                : 0.5 * de[5] * X + 0.5 * de[4] * Y + de[2] * Z);
        }
        u[i] = v;
      }
    } else if (warm) {
      if (t < SERVE_K * 6) {
        const int k = t / 6, j = t % 6;
        const double e0 = __ldcg(G.warm_eps + j);
        const double d = __ldcg(G.warm_eps + (j + 1) * 6 + j) - e0;
        spred[t] = (d != 0.0) ? (seps[k * 6 + j] - e0) / d : 0.0;
      }
      __syncthreads();
      const size_t blk = (size_t)3 * g.nn_pad;
      for (size_t i = t; i < blk; i += SERVE_NT) {
        const double w0 = __ldcg(G.warm + i);
        double dw[6];
#pragma unroll
        for (int j = 0; j < 6; j++) dw[j] = __ldcg(G.warm + (j + 1) * blk + i) - w0;
#pragma unroll
        for (int k = 0; k < SERVE_K; k++) {
          double v = w0;
#pragma unroll
          for (int j = 0; j < 6; j++) v = fma(spred[k * 6 + j], dw[j], v);
          u[k * blk + i] = v;
        }
      }
    }
    __syncthreads();
    if constexpr (PT)
      stencil_ptable(t, SERVE_NT, sKe, s_ptab);
    else if constexpr (STENCIL)
      stencil_blocks<float>(t, SERVE_NT, sKe, sKB);
    stencil_blocks<double>(t, SERVE_NT, sKe, sKBd);
    // a cold request (no earlier solution on this geometry) starts from the
    // homogeneous affine field inside; a warm one keeps its start inside
    affine_soa<SERVE_K>(t, SERVE_NT, g, seps, SERVE_NRHS, warm, u, !warm);
    __syncthreads();
    SolveArgs sa;
    sa.nrhs = SERVE_NRHS;
    sa.rtol = P.rtol;
    // a request whose prediction misses rtol is solved tighter, so that the
    // predictions from its solutions meet rtol without a solve (a start from
    // the last solutions is solved to rtol)
    sa.rtol_refine = P.warm_last ? P.rtol : P.refine_rtol;
    sa.inner_rtol = P.inner_rtol;
    sa.max_outer = P.max_outer;
    sa.max_inner = P.max_inner;
    sa.warm = 1;  // every start iterate is measured against the right-hand side's norm
    sa.rn0_given = srn0;
    sa.kbd = sKBd;
    sa.eps = nullptr;  // affine conditions: eps is carried by u's boundary values
    sp_solve_info in;
    if constexpr (STENCIL) {
      // one request slot per SM has 128 registers a thread: per-node FP64 residual
      StencilOp<float, SERVE_K, false, PT> op{PT ? s_ptab : sKB, G.etype};
      in = solve_rve<float, SERVE_K, SERVE_NT, 1, decltype(op), MINB == 1>(
          g, op, G.dinv, G.etype, sKe, sD, sB, u, r, x, p, q, sa, red, &sh, savg);
    } else {
      EllOp<float, SERVE_K> op{G.vals, G.nbr};
      in = solve_rve<float, SERVE_K, SERVE_NT, 1, decltype(op), MINB == 1>(
          g, op, G.dinv, G.etype, sKe, sD, sB, u, r, x, p, q, sa, red, &sh, savg);
    }
    // keep this request's solutions and strains as the geometry's next warm
    // start when it ran a refinement step (they then meet refine_rtol); a
    // request accepted on its prediction leaves the solved state in place,
    // so predictions do not drift from it
    const bool store = in.outer_its > 0 || !warm || P.warm_last;
    if (store) {
      for (size_t i = t; i < nu; i += SERVE_NT) __stcg(G.warm + i, u[i]);
      if (t < SERVE_K * 6) __stcg(G.warm_eps + t, seps[t]);
    }
    __threadfence();
    __syncthreads();
    if (t == 0) {
      if (store) G.has_warm = 1;
      for (int v = 0; v < 6; v++) out->stress[v] = savg[6 + v];
      // c_tangent[j*6 + i] = (stress(eps + d e_i)_j - stress(eps)_j) / (d e_i)
      // (micro/src/homogenize.c:79-80)
      for (int i = 0; i < 6; i++)
        for (int j = 0; j < 6; j++)
          out->tangent[j * 6 + i] =
              (savg[(i + 1) * 12 + 6 + j] - savg[6 + j]) / (seps[(i + 1) * 6 + i] - seps[i]);
      out->info = in;
      __threadfence_system();
      out->done = job + 1;
    }
    __syncthreads();
  }
}

static double now_s() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

// device bytes a resident geometry holds (the assembled operator adds its
// node-sliced FP32 values)
static size_t geom_bytes(const sp_rve_desc &d, int op) {
  size_t nn = (size_t)(d.n[0] + 1) * (d.n[1] + 1) * (d.n[2] + 1), np = (nn + 31) / 32 * 32;
  size_t nelm = (size_t)d.n[0] * d.n[1] * d.n[2];
  return (op == SP_OP_ELL ? np * 243 * 4 : 0) + 3 * np * 4 + nelm +
         (2 * SP_KE + 72 + 144) * 8 + (SERVE_K * (3 * np + 6) + 36) * 8 + 1024;
}

}  // namespace sp

using namespace sp;

struct sp_server_s {
  int ngeom = 0, dev = -1, grid = 0, cap = 0, running = 0;
  long long launches = 0;  // launches of the loop (the first, and every relaunch)
  double last_alive = 0.0;  // host time of the last liveness check of the loop
  sp_server_opts o;
  std::vector<DevPlan *> plans;
  std::vector<ServeGeom> hgeoms;
  ServeGeom *d_geoms = nullptr;
  std::vector<void *> dbufs;
  ServeReq *h_req = nullptr, *d_req_map = nullptr, *d_req = nullptr;
  ServeRes *h_res = nullptr, *d_res_map = nullptr;
  ServeCtl *h_ctl = nullptr, *d_ctl_map = nullptr;
  ServeDev *d_dev = nullptr;
  double *ws_u = nullptr;
  float *ws_v = nullptr;
  size_t stride = 0, bytes = 0;
  long long tail = 0, head_done = 0;
  cudaStream_t stream = nullptr;
  ServeParams P;
};

static int server_grid(sp_server *s, Device *d);

// the loop kernel for an operator and a CTAs-per-SM target
using ServeFn = void (*)(ServeParams);
static ServeFn serve_kernel(const sp_server_opts &o) {
  if (o.op == SP_OP_ELL) return o.ctas_per_sm == 1 ? k_serve<SP_OP_ELL, 1> : k_serve<SP_OP_ELL, 2>;
  return o.ctas_per_sm == 1 ? k_serve<SP_OP_STENCIL, 1> : k_serve<SP_OP_STENCIL, 2>;
}

// its dynamic shared memory: the pattern table of the one-slot stencil loop
static int serve_dyn_smem(const sp_server_opts &o) {
  return (o.op == SP_OP_STENCIL && o.ctas_per_sm == 1) ? SP_PT_BYTES : 0;
}

extern "C" void sp_server_opts_default(sp_server_opts *o) {
  memset(o, 0, sizeof(*o));
  o->hbm_budget = (size_t)150 * 1000 * 1000 * 1000;
  o->max_inflight = 0;
  o->queue_capacity = 65536;
  o->rtol = 1e-8;
  o->inner_rtol = 1e-4;
  o->idle_spin_limit = 2000000;
  o->op = SP_OP_STENCIL;
  o->ctas_per_sm = 0;
  o->refine_rtol = 0.0;
  o->warm_start = SP_WARM_PREDICT;
}

static int server_layout(int ngeom, const sp_rve_desc *descs, const sp_server_opts *o, int nsm,
                         int *slots, size_t *total, size_t *per_slot) {
  size_t resident = 0;
  std::map<std::vector<int>, int> seen;
  int maxnp = 0;
  for (int i = 0; i < ngeom; i++) {
    const sp_rve_desc &d = descs[i];
    for (int k = 0; k < 3; k++)
      if (d.n[k] < 1 || d.len[k] <= 0)
        return sp_set_error(SP_ERR_ARG, "geometry %d: bad mesh", i);
    resident += geom_bytes(d, o->op);
    std::vector<int> key(d.n, d.n + 3);
    if (!seen.count(key)) {
      seen[key] = 1;
      resident += plan_bytes(d.n);
    }
    maxnp = std::max(maxnp, ((d.n[0] + 1) * (d.n[1] + 1) * (d.n[2] + 1) + 31) / 32 * 32);
  }
  size_t slot = (size_t)SERVE_K * 3 * maxnp * (8 + 4 * 4);
  const int per_sm = o->ctas_per_sm ? o->ctas_per_sm : (o->op == SP_OP_STENCIL ? 1 : 2);
  int want = nsm * per_sm - 1;
  if (o->max_inflight > 0 && o->max_inflight < want) want = o->max_inflight;
  size_t budget = o->hbm_budget ? o->hbm_budget : (size_t)150e9;
  if (resident + slot > budget)
    return sp_set_error(SP_ERR_BUDGET, "geometries need %zu bytes, budget %zu", resident + slot,
                        budget);
  // HBM admission: as many concurrent request slots as the budget allows
  size_t fit = (budget - resident) / slot;
  if ((size_t)want > fit) want = (int)fit;
  *slots = want;
  *per_slot = slot;
  *total = resident + (size_t)(want + 1) * slot;
  return SP_OK;
}

extern "C" int sp_server_plan_bytes(int ngeom, const sp_rve_desc *descs, const sp_server_opts *opts,
                                    size_t *bytes) {
  if (ngeom < 1 || !descs || !bytes) return sp_set_error(SP_ERR_ARG, "bad argument");
  sp_server_opts o;
  if (opts) o = *opts; else sp_server_opts_default(&o);
  int slots;
  size_t per;
  return server_layout(ngeom, descs, &o, 148, &slots, bytes, &per);
}

extern "C" int sp_server_destroy(sp_server *s) {
  if (!s) return SP_OK;
  if (s->running) sp_server_stop(s);
  for (void *p : s->dbufs) cudaFree(p);
  cudaFree(s->d_geoms);
  cudaFree(s->d_req);
  cudaFree(s->d_dev);
  cudaFree(s->ws_u);
  cudaFree(s->ws_v);
  if (s->h_req) cudaFreeHost(s->h_req);
  if (s->h_res) cudaFreeHost(s->h_res);
  if (s->h_ctl) cudaFreeHost(s->h_ctl);
  if (s->stream) cudaStreamDestroy(s->stream);
  for (DevPlan *p : s->plans) plan_release(p);
  delete s;
  return SP_OK;
}

extern "C" int sp_server_create(int ngeom, const sp_rve_desc *descs, const sp_server_opts *opts,
                                sp_server **out) {
  if (ngeom < 1 || !descs || !out) return sp_set_error(SP_ERR_ARG, "sp_server_create: bad argument");
  sp_server_opts o;
  if (opts) o = *opts; else sp_server_opts_default(&o);
  if (o.queue_capacity <= 0) o.queue_capacity = 65536;
  if (!(o.rtol > 0)) o.rtol = 1e-8;
  if (!(o.inner_rtol > 0)) o.inner_rtol = 1e-4;
  if (!(o.refine_rtol > 0)) o.refine_rtol = 1e-2 * o.rtol;
  if (o.refine_rtol > o.rtol) o.refine_rtol = o.rtol;
  if (o.idle_spin_limit <= 0) o.idle_spin_limit = 2000000;
  if (o.op != SP_OP_ELL && o.op != SP_OP_STENCIL)
    return sp_set_error(SP_ERR_ARG, "sp_server_create: unknown operator");
  if (o.warm_start != SP_WARM_PREDICT && o.warm_start != SP_WARM_LAST)
    return sp_set_error(SP_ERR_ARG, "sp_server_create: unknown warm start");
  // the stencil solve of 7 load cases wants 128 registers (1 slot per SM)
  if (o.ctas_per_sm == 0) o.ctas_per_sm = (o.op == SP_OP_STENCIL) ? 1 : 2;
  if (o.ctas_per_sm != 1 && o.ctas_per_sm != 2)
    return sp_set_error(SP_ERR_ARG, "sp_server_create: ctas_per_sm must be 1 or 2");
  Device *d;
  SP_TRY(device(&d));
  int slots;
  size_t total, per_slot;
  SP_TRY(server_layout(ngeom, descs, &o, d->nsm, &slots, &total, &per_slot));
  if (slots < 1) return sp_set_error(SP_ERR_BUDGET, "budget leaves no request slot");
  sp_server *s = new sp_server_s();
  s->ngeom = ngeom;
  s->o = o;
  s->dev = d->id;
  s->cap = o.queue_capacity;
  s->grid = slots + 1; // + dispatcher
  int rc = server_grid(s, d);
  std::map<std::vector<int>, DevPlan *> pm;
  std::vector<double> mats((size_t)ngeom * 4);
  int maxdof = 0, maxnp = 0;
  s->hgeoms.resize(ngeom);
  for (int i = 0; i < ngeom && !rc; i++) {
    const sp_rve_desc &dd = descs[i];
    std::vector<int> key(dd.n, dd.n + 3);
    DevPlan *p;
    if (pm.count(key)) {
      p = pm[key];
    } else {
      rc = plan_acquire(dd.n, &p);
      if (rc) break;
      s->plans.push_back(p);
      pm[key] = p;
    }
    ServeGeom &G = s->hgeoms[i];
    memset(&G, 0, sizeof(G));
    G.g = make_geo(dd.n, dd.len);
    G.cols = p->cols;
    G.nbr = p->nbr;
    G.color_elems = p->color_elems;
    G.slot = p->slot;
    for (int c = 0; c < 9; c++) G.color_off[c] = p->color_off[c];
    maxdof = std::max(maxdof, G.g.ndof);
    maxnp = std::max(maxnp, G.g.nn_pad);
    size_t np = G.g.nn_pad, ne = G.g.nelm;
    void *b[7] = {};
    size_t sz[7] = {o.op == SP_OP_ELL ? np * 243 * 4 : 0, 3 * np * 4, ne + 16, 2 * SP_KE * 8,
                    72 * 8, 144 * 8, (SERVE_K * (3 * np + 6) + 36) * 8};
    for (int k = 0; k < 7 && !rc; k++) {
      if (!sz[k]) continue;
      rc = dmalloc(&b[k], sz[k], &s->bytes);
      if (!rc) s->dbufs.push_back(b[k]);
    }
    if (rc) break;
    G.vals = (float *)b[0];
    G.dinv = (float *)b[1];
    G.etype = (const uint8_t *)b[2];
    G.Ke = (double *)b[3];
    G.D = (double *)b[4];
    G.Bbar = (double *)b[5];
    G.warm = (double *)b[6];
    G.warm_eps = G.warm + (size_t)SERVE_K * 3 * np;
    G.gram = G.warm_eps + SERVE_K * 6;
    std::vector<uint8_t> et(ne);
    rc = sp_classify_elements(&dd, et.data(), nullptr);
    if (!rc && cudaMemcpy((void *)G.etype, et.data(), ne, cudaMemcpyHostToDevice))
      rc = sp_set_error(SP_ERR_CUDA, "etype upload");
    mats[i * 4 + 0] = dd.E[0];
    mats[i * 4 + 1] = dd.nu[0];
    mats[i * 4 + 2] = dd.E[1];
    mats[i * 4 + 3] = dd.nu[1];
  }
  s->stride = (size_t)SERVE_K * 3 * maxnp;
  double *d_mats = nullptr;
  float *d_scr = nullptr;
  size_t rm_stride = (size_t)maxdof * SP_WP, drm_stride = (size_t)(maxdof + 3) / 4 * 4;
  int nasm = std::min(ngeom, 2 * d->nsm);
  if (!rc) rc = dmalloc((void **)&s->d_geoms, ngeom * sizeof(ServeGeom), &s->bytes);
  if (!rc) rc = dmalloc((void **)&d_mats, mats.size() * sizeof(double), nullptr);
  if (!rc && o.op == SP_OP_ELL)
    rc = dmalloc((void **)&d_scr, (size_t)nasm * (rm_stride + drm_stride) * 4, nullptr);
  if (!rc) rc = dmalloc((void **)&s->d_req, (size_t)s->cap * sizeof(ServeReq), &s->bytes);
  if (!rc) rc = dmalloc((void **)&s->d_dev, sizeof(ServeDev), &s->bytes);
  if (!rc) rc = dmalloc((void **)&s->ws_u, (size_t)s->grid * s->stride * 8, &s->bytes);
  if (!rc) rc = dmalloc((void **)&s->ws_v, (size_t)s->grid * 4 * s->stride * 4, &s->bytes);
  if (!rc && (cudaHostAlloc((void **)&s->h_req, (size_t)s->cap * sizeof(ServeReq), cudaHostAllocMapped) ||
              cudaHostAlloc((void **)&s->h_res, (size_t)s->cap * sizeof(ServeRes), cudaHostAllocMapped) ||
              cudaHostAlloc((void **)&s->h_ctl, sizeof(ServeCtl), cudaHostAllocMapped)))
    rc = sp_set_error(SP_ERR_NOMEM, "mapped host ring allocation failed");
  if (!rc && (cudaHostGetDevicePointer((void **)&s->d_req_map, s->h_req, 0) ||
              cudaHostGetDevicePointer((void **)&s->d_res_map, s->h_res, 0) ||
              cudaHostGetDevicePointer((void **)&s->d_ctl_map, s->h_ctl, 0)))
    rc = sp_set_error(SP_ERR_CUDA, "mapped pointers unavailable");
  if (!rc && cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking))
    rc = sp_set_error(SP_ERR_CUDA, "stream");
  if (!rc) {
    memset(s->h_res, 0, (size_t)s->cap * sizeof(ServeRes));
    memset(s->h_ctl, 0, sizeof(ServeCtl));
    if (cudaMemcpy(s->d_geoms, s->hgeoms.data(), ngeom * sizeof(ServeGeom), cudaMemcpyHostToDevice) ||
        cudaMemcpy(d_mats, mats.data(), mats.size() * sizeof(double), cudaMemcpyHostToDevice) ||
        cudaMemset(s->d_dev, 0, sizeof(ServeDev)))
      rc = sp_set_error(SP_ERR_CUDA, "server upload");
  }
  if (!rc) {
    if (o.op == SP_OP_STENCIL)
      k_serve_assemble<SP_OP_STENCIL><<<nasm, SERVE_NT, 0, s->stream>>>(
          s->d_geoms, ngeom, d_mats, d_scr, rm_stride, drm_stride);
    else
      k_serve_assemble<SP_OP_ELL><<<nasm, SERVE_NT, 0, s->stream>>>(
          s->d_geoms, ngeom, d_mats, d_scr, rm_stride, drm_stride);
    if (cudaGetLastError() || cudaStreamSynchronize(s->stream))
      rc = sp_set_error(SP_ERR_CUDA, "geometry assembly failed");
  }
  if (!rc) {
    // Gram matrices of the unit-strain right-hand sides (temporary work space)
    const int ngram = std::min(ngeom, 64);
    const size_t gstride = (size_t)6 * 3 * maxnp;
    double *d_gs = nullptr;
    rc = dmalloc((void **)&d_gs, (size_t)ngram * 2 * gstride * sizeof(double), nullptr);
    if (!rc) {
      k_serve_gram<<<ngram, SERVE_NT, 0, s->stream>>>(s->d_geoms, ngeom, d_gs, gstride);
      if (cudaGetLastError() || cudaStreamSynchronize(s->stream))
        rc = sp_set_error(SP_ERR_CUDA, "geometry right-hand-side norms failed");
    }
    cudaFree(d_gs);
  }
  cudaFree(d_mats);
  cudaFree(d_scr);
  if (rc) {
    sp_server_destroy(s);
    return rc;
  }
  ServeParams &P = s->P;
  P.geoms = s->d_geoms;
  P.ngeom = ngeom;
  P.cap = s->cap;
  P.hreq = s->d_req_map;
  P.dreq = s->d_req;
  P.res = s->d_res_map;
  P.ctl = s->d_ctl_map;
  P.dev = s->d_dev;
  P.ws_u = s->ws_u;
  P.ws_v = s->ws_v;
  P.stride = s->stride;
  P.rtol = o.rtol;
  P.refine_rtol = o.refine_rtol;
  P.inner_rtol = o.inner_rtol;
  P.max_outer = 8;
  P.max_inner = 4000;
  P.idle_limit = o.idle_spin_limit;
  P.warm_last = o.warm_start == SP_WARM_LAST;
  *out = s;
  return SP_OK;
}

// Every CTA of the loop must be resident at once (workers wait for the
// dispatcher's counter): the grid never exceeds what the SMs hold.
static int server_grid(sp_server *s, Device *d) {
  int occ = 0;
  const int dyn = serve_dyn_smem(s->o);
  if (dyn)
    SP_CUDA_TRY(cudaFuncSetAttribute((const void *)serve_kernel(s->o),
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
  SP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, serve_kernel(s->o), SERVE_NT, dyn));
  if (occ < 1) return sp_set_error(SP_ERR_CUDA, "serving kernel does not fit an SM");
  int cap = d->nsm * occ;
  if (s->grid > cap) s->grid = cap;
  return SP_OK;
}

static int server_launch(sp_server *s) {
  // reset the liveness flags, keep the claim and device counters
  ServeDev z;
  SP_CUDA_TRY(cudaMemcpy(&z, s->d_dev, sizeof(z), cudaMemcpyDeviceToHost));
  z.dstop = 0;
  z.dispatcher_gone = 0;
  SP_CUDA_TRY(cudaMemcpyAsync(s->d_dev, &z, sizeof(z), cudaMemcpyHostToDevice, s->stream));
  SP_CUDA_TRY(cudaStreamSynchronize(s->stream));
  serve_kernel(s->o)<<<s->grid, SERVE_NT, serve_dyn_smem(s->o), s->stream>>>(s->P);
  SP_CUDA_TRY(cudaGetLastError());
  s->running = 1;
  s->launches++;
  return SP_OK;
}

// relaunch the loop if it went idle while requests are pending
// The loop's liveness check (a stream query, microseconds of driver time)
// runs at most every SP_KEEPALIVE_S: submit and poll call it once per
// request, thousands of times a millisecond under load.
constexpr double SP_KEEPALIVE_S = 50e-6;

static int server_keepalive(sp_server *s) {
  if (!s->running) return SP_OK;
  const double t = now_s();
  if (t - s->last_alive < SP_KEEPALIVE_S) return SP_OK;
  s->last_alive = t;
  cudaError_t q = cudaStreamQuery(s->stream);
  if (q == cudaErrorNotReady) return SP_OK;
  if (q != cudaSuccess) return sp_set_error(SP_ERR_CUDA, "serving loop failed: %s", cudaGetErrorString(q));
  if (s->h_ctl->stop) return SP_OK;
  ServeDev z;
  SP_CUDA_TRY(cudaMemcpy(&z, s->d_dev, sizeof(z), cudaMemcpyDeviceToHost));
  if ((long long)z.claim < s->tail) return server_launch(s);
  return SP_OK;
}

extern "C" int sp_server_start(sp_server *s) {
  if (!s) return sp_set_error(SP_ERR_ARG, "null server");
  if (s->running) return SP_OK;
  Device *d;
  SP_TRY(device(&d));
  s->h_ctl->stop = 0;
  return server_launch(s);
}

extern "C" int sp_server_submit(sp_server *s, int geometry, const double *strain, long long *ticket) {
  if (!s || !strain) return sp_set_error(SP_ERR_ARG, "null argument");
  if (geometry < 0 || geometry >= s->ngeom) return sp_set_error(SP_ERR_RANGE, "geometry %d", geometry);
  if (!s->running) return sp_set_error(SP_ERR_STATE, "server not started");
  if (s->tail - s->head_done >= s->cap) return sp_set_error(SP_ERR_BUDGET, "request ring full");
  long long i = s->tail;
  ServeReq &r = s->h_req[i % s->cap];
  r.geom = geometry;
  for (int k = 0; k < 6; k++) r.strain[k] = strain[k];
  s->h_res[i % s->cap].done = 0;
  std::atomic_thread_fence(std::memory_order_seq_cst);
  s->tail = i + 1;
  s->h_ctl->tail = i + 1;
  if (ticket) *ticket = i;
  return server_keepalive(s);
}

extern "C" int sp_server_poll(sp_server *s, long long ticket, double *stress, double *tangent,
                              sp_solve_info *info) {
  if (!s) return sp_set_error(SP_ERR_ARG, "null server");
  if (ticket < 0 || ticket >= s->tail || ticket < s->tail - s->cap)
    return sp_set_error(SP_ERR_RANGE, "ticket %lld not in the ring", ticket);
  ServeRes &r = s->h_res[ticket % s->cap];
  if (r.done != ticket + 1) {
    SP_TRY(server_keepalive(s));
    return SP_PENDING;
  }
  std::atomic_thread_fence(std::memory_order_acquire);
  if (stress) memcpy(stress, r.stress, sizeof(r.stress));
  if (tangent) memcpy(tangent, r.tangent, sizeof(r.tangent));
  if (info) *info = r.info;
  while (s->head_done < s->tail && s->h_res[s->head_done % s->cap].done == s->head_done + 1)
    s->head_done++;
  return SP_OK;
}

extern "C" int sp_server_status(const sp_server *s, int *loop_on_device, long long *launches,
                                long long *submitted) {
  if (!s) return sp_set_error(SP_ERR_ARG, "null server");
  if (loop_on_device) {
    cudaError_t q = cudaStreamQuery(s->stream);
    if (q != cudaSuccess && q != cudaErrorNotReady)
      return sp_set_error(SP_ERR_CUDA, "serving loop failed: %s", cudaGetErrorString(q));
    *loop_on_device = (q == cudaErrorNotReady);
  }
  if (launches) *launches = s->launches;
  if (submitted) *submitted = s->tail;
  return SP_OK;
}

extern "C" int sp_server_stop(sp_server *s) {
  if (!s) return sp_set_error(SP_ERR_ARG, "null server");
  if (!s->running) return SP_OK;
  s->h_ctl->stop = 1;
  std::atomic_thread_fence(std::memory_order_seq_cst);
  cudaError_t e = cudaStreamSynchronize(s->stream);
  s->running = 0;
  if (e) return sp_set_error(SP_ERR_CUDA, "serving loop: %s", cudaGetErrorString(e));
  // requests published after the loop saw stop: run them to completion
  ServeDev z;
  SP_CUDA_TRY(cudaMemcpy(&z, s->d_dev, sizeof(z), cudaMemcpyDeviceToHost));
  if ((long long)z.claim < s->tail) {
    s->h_ctl->stop = 0;
    SP_TRY(server_launch(s));
    s->h_ctl->stop = 1;
    std::atomic_thread_fence(std::memory_order_seq_cst);
    e = cudaStreamSynchronize(s->stream);
    s->running = 0;
    if (e) return sp_set_error(SP_ERR_CUDA, "serving loop: %s", cudaGetErrorString(e));
  }
  return SP_OK;
}

extern "C" int sp_server_replay(sp_server *s, int nreq, const int *geom, const double *strain,
                                const double *t_arrival, double *t_done, double *stress,
                                double *tangent, sp_solve_info *info, double timeout_s) {
  if (!s || nreq < 0 || !geom || !strain || !t_arrival || !t_done)
    return sp_set_error(SP_ERR_ARG, "sp_server_replay: bad argument");
  if (!s->running) SP_TRY(sp_server_start(s));
  long long base = s->tail;
  int next = 0, done = 0, scan = 0;
  std::vector<char> fin(nreq, 0);
  double t0 = now_s();
  while (done < nreq) {
    double now = now_s() - t0;
    if (now > timeout_s) return sp_set_error(SP_ERR_TIMEOUT, "replay timed out, %d of %d done", done, nreq);
    while (next < nreq && t_arrival[next] <= now && s->tail - s->head_done < s->cap) {
      long long tk;
      SP_TRY(sp_server_submit(s, geom[next], strain + 6 * (size_t)next, &tk));
      next++;
    }
    int polled = 0;
    for (int i = scan; i < next && polled < 4096; i++, polled++) {
      if (fin[i]) continue;
      int rc = sp_server_poll(s, base + i, stress ? stress + 6 * (size_t)i : nullptr,
                              tangent ? tangent + 36 * (size_t)i : nullptr, info ? info + i : nullptr);
      if (rc == SP_OK) {
        t_done[i] = now_s() - t0;
        fin[i] = 1;
        done++;
      } else if (rc != SP_PENDING) {
        return rc;
      }
    }
    while (scan < next && fin[scan]) scan++;
  }
  return SP_OK;
}
