// fe2.cu -- an FE2 step on one GPU: the macro Newton loop of macro/src/main.c:
// 202-256 on a structured 3D hex8 cantilever whose Gauss points take their
// stress and tangent from micro RVEs served by the serving loop (serve.cu).
//
// Per Newton iteration (all on the device except the micro requests of the
// per-Gauss-point mode):
//   1. Gauss-point strains eps = B u_e, components below strain_clip set to
//      zero (macro/src/assembly.c:305-322);
//   2. micro response: sigma = C eps with the RVE's FD tangent around zero
//      (linear micro materials: micro/src/init.c:54-59, micro/src/
//      homogenize.c:3-21), or one serving-loop request per Gauss point
//      (stress + FD tangent, micro/src/homogenize.c:59-94);
//   3. residual b = f_ext - sum_e sum_gp B^T sigma w, zero on clamped dofs
//      (macro/src/assembly.c:5-84; the reference's loading is Dirichlet
//      only, the traction here adds f_ext), gathered per dof so that no two
//      threads write one entry;
//   4. Jacobian K = sum_e sum_gp B^T C B w (macro/src/assembly.c:165-222)
//      into FP64 ELL by the 8-colour conflict-free scatter, clamped rows and
//      columns set to the identity (MatZeroRowsColumns, :208-214);
//   5. K dx = b by the FP64 Jacobi-PCG in one cooperative launch (pcg.cuh,
//      k_pcg_coop), u += dx.
// The iteration stops after newton_its, or when ||b|| <= newton_tol (the
// reference's check before assembling, macro/src/main.c:222-227).
#include <time.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pcg.cuh"
#include "rve_device.cuh"
#include "sp_cuda.h"

namespace sp {

constexpr int FE2_GP = 8;
constexpr int FE2_B = FE2_GP * 6 * SP_NC;  // B[gp][v][i]

// B matrices of the 8 Gauss points and the Gauss weight; every element of
// the structured box has the same shape, so one set serves all.
__global__ void k_fe2_ops(MeshGeo g, double *B, double *w) {
  __shared__ double dsh[192];
  const double h[3] = {g.hx, g.hy, g.hz};
  elem_ops_stage1(threadIdx.x, blockDim.x, h, dsh);
  __syncthreads();
  for (int x = threadIdx.x; x < FE2_B; x += blockDim.x) {
    int gp = x / (6 * SP_NC), v = (x / SP_NC) % 6, i = x % SP_NC;
    B[x] = bmat_entry(dsh, v, i, gp);
  }
  if (threadIdx.x == 0) *w = __ddiv_rn(dmul(dmul(h[0], h[1]), h[2]), 8.0);
}

// eps[e*8 + gp][v] = B_gp u_e, |eps_v| < clip -> 0 (macro/src/assembly.c:305-322)
__global__ void k_fe2_strain(MeshGeo g, const double *__restrict__ B, const double *__restrict__ u,
                             double clip, double *eps) {
  const int n = g.nelm * FE2_GP;
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n; x += gridDim.x * blockDim.x) {
    const int e = x / FE2_GP, gp = x % FE2_GP;
    int nod[8];
    elem_nodes(g, e, nod);
    double ue[SP_NC];
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
      for (int d = 0; d < 3; d++) ue[a * 3 + d] = u[(size_t)nod[a] * 3 + d];
    const double *Bg = B + gp * 6 * SP_NC;
    for (int v = 0; v < 6; v++) {
      double s = 0.0;
#pragma unroll
      for (int i = 0; i < SP_NC; i++) s = fma(Bg[v * SP_NC + i], ue[i], s);
      eps[(size_t)x * 6 + v] = (fabs(s) < clip) ? 0.0 : s;
    }
  }
}

// sigma = C eps with the RVE tangent of every Gauss point (linear micro)
__global__ void k_fe2_stress(int ngp, const double *__restrict__ eps, const int *__restrict__ gp_rve,
                             const double *__restrict__ clin, double *sig) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < ngp; x += gridDim.x * blockDim.x) {
    const double *C = clin + (size_t)gp_rve[x] * 36;
    for (int j = 0; j < 6; j++) {
      double s = 0.0;
      for (int i = 0; i < 6; i++) s = fma(C[j * 6 + i], eps[(size_t)x * 6 + i], s);
      sig[(size_t)x * 6 + j] = s;
    }
  }
}

__device__ inline bool fe2_clamped(const MeshGeo &g, int node) { return node % g.nx == 0; }

// b = f_ext - f_int on free dofs, 0 on clamped dofs; f_int gathered per dof
// over the (up to 8) elements of its node
__global__ void k_fe2_residual(MeshGeo g, const double *__restrict__ B, const double *w,
                               const double *__restrict__ sig, const double *__restrict__ fext,
                               double *b) {
  const double wv = *w;
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < g.ndof;
       row += gridDim.x * blockDim.x) {
    const int node = row / 3, d = row % 3;
    if (fe2_clamped(g, node)) {
      b[row] = 0.0;
      continue;
    }
    const int i = node % g.nx, j = (node / g.nx) % g.ny, k = node / (g.nx * g.ny);
    double f = 0.0;
    for (int c = 0; c < 8; c++) {
      const int ox = c & 1, oy = (c >> 1) & 1, oz = c >> 2;
      const int ex = i - 1 + ox, ey = j - 1 + oy, ez = k - 1 + oz;
      if (ex < 0 || ey < 0 || ez < 0 || ex >= g.nex || ey >= g.ney || ez >= g.nez) continue;
      const int e = ex + ey * g.nex + ez * g.nex * g.ney;
      const int col = hex8_local(1 - ox, 1 - oy, 1 - oz) * 3 + d;
      for (int gp = 0; gp < FE2_GP; gp++) {
        const double *s = sig + ((size_t)e * FE2_GP + gp) * 6;
        const double *Bg = B + gp * 6 * SP_NC;
#pragma unroll
        for (int v = 0; v < 6; v++) f = fma(Bg[v * SP_NC + col], s[v], f);
      }
    }
    b[row] = fext[row] - f * wv;
  }
}

// ||b||^2 in a fixed order (one block)
__global__ void k_fe2_norm2(int n, const double *__restrict__ b, double *out) {
  __shared__ double red[33];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s = fma(b[i], b[i], s);
  double t[1] = {s}, tot[1];
  block_sum<1>(t, red, tot);
  if (threadIdx.x == 0) *out = tot[0];
}

// One colour of the Jacobian scatter: Ke[i][j] = sum_gp sum_hk B[h][i] C[h][k]
// B[k][j] w for every element of the colour (elements of one colour share
// no node, so the writes of one launch are to distinct slots).
__global__ void k_fe2_assemble(MeshGeo g, const int *__restrict__ color_elems, int c0, int c1,
                               const uint8_t *__restrict__ slot, const double *__restrict__ B,
                               const double *w, const int *__restrict__ gp_rve,
                               const double *__restrict__ clin, const double *__restrict__ ctan,
                               double *vals) {
  const double wv = *w;
  const int nwork = (c1 - c0) * SP_KE;
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < nwork; x += gridDim.x * blockDim.x) {
    const int e = color_elems[c0 + x / SP_KE];
    const int ij = x % SP_KE, i = ij / SP_NC, j = ij % SP_NC;
    double s = 0.0;
    for (int gp = 0; gp < FE2_GP; gp++) {
      const double *C = ctan ? ctan + ((size_t)e * FE2_GP + gp) * 36
                             : clin + (size_t)gp_rve[(size_t)e * FE2_GP + gp] * 36;
      const double *Bg = B + gp * 6 * SP_NC;
      for (int h = 0; h < 6; h++) {
        const double bhi = Bg[h * SP_NC + i];
        if (bhi == 0.0) continue;
        double t = 0.0;
        for (int k = 0; k < 6; k++) t = fma(C[h * 6 + k], Bg[k * SP_NC + j], t);
        s = fma(bhi, t, s);
      }
    }
    int nod[8];
    elem_nodes(g, e, nod);
    const int row = nod[i / 3] * 3 + i % 3;
    vals[(size_t)row * SP_WP + slot[(size_t)e * SP_KE + ij]] += s * wv;
  }
}

// clamped rows and columns -> identity, Jacobi diagonal inverse
__global__ void k_fe2_bc(MeshGeo g, const int *__restrict__ cols, double *vals, double *dinv) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < g.ndof;
       row += gridDim.x * blockDim.x) {
    const bool brow = fe2_clamped(g, row / 3);
    const int *c = cols + (size_t)row * SP_WP;
    double *v = vals + (size_t)row * SP_WP;
    double diag = 0.0;
    for (int s = 0; s < SP_ELL_WIDTH; s++) {
      const int col = c[s];
      if (col < 0) break;
      if (brow)
        v[s] = (col == row) ? 1.0 : 0.0;
      else if (fe2_clamped(g, col / 3))
        v[s] = 0.0;
      if (col == row) diag = v[s];
    }
    dinv[row] = 1.0 / diag;
  }
}

__global__ void k_fe2_axpy(int n, const double *__restrict__ dx, double *u) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    u[i] += dx[i];
}

static double fe2_now() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

// splitmix64: the seeded Gauss-point -> RVE binding
static unsigned long long mix64(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

}  // namespace sp

using namespace sp;

struct sp_fe2_s {
  sp_fe2_desc d;
  MeshGeo g;
  DevPlan *plan = nullptr;
  sp_server *srv = nullptr;
  int ngp = 0, dev = -1;
  std::vector<int> gp_rve;
  std::vector<double> clin;  // [nrve][36]
  double *d_B = nullptr, *d_w = nullptr, *d_u = nullptr, *d_fext = nullptr, *d_b = nullptr;
  double *d_eps = nullptr, *d_sig = nullptr, *d_ctan = nullptr, *d_clin = nullptr;
  double *d_vals = nullptr, *d_dinv = nullptr, *d_vec = nullptr, *d_nrm = nullptr;
  int *d_gp_rve = nullptr;
  PcgState *d_st = nullptr;
  double *d_partial = nullptr;
  unsigned *d_ticket = nullptr;
  PcgCoop<double, 1, 8> *pcg = nullptr;
  int nblk = 0;
  cudaStream_t stream = nullptr;
};

extern "C" void sp_fe2_desc_default(sp_fe2_desc *d) {
  memset(d, 0, sizeof(*d));
  d->n[0] = 40;
  d->n[1] = 10;
  d->n[2] = 10;
  d->len[0] = 4.0;
  d->len[1] = 1.0;
  d->len[2] = 1.0;
  d->traction[2] = -1e6;
  d->newton_its = 5;
  d->newton_tol = 0.0;
  d->lin_rtol = 1e-10;
  d->strain_clip = 1e-6;
  d->micro = SP_FE2_LINEAR;
  d->seed = 2024;
}

extern "C" int sp_fe2_destroy(sp_fe2 *f) {
  if (!f) return SP_OK;
  delete f->pcg;
  void *bufs[] = {f->d_B, f->d_w, f->d_u, f->d_fext, f->d_b, f->d_eps, f->d_sig, f->d_ctan,
                  f->d_clin, f->d_vals, f->d_dinv, f->d_vec, f->d_nrm, f->d_gp_rve, f->d_st,
                  f->d_partial, f->d_ticket};
  for (void *p : bufs) cudaFree(p);
  if (f->srv) sp_server_destroy(f->srv);
  if (f->plan) plan_release(f->plan);
  if (f->stream) cudaStreamDestroy(f->stream);
  delete f;
  return SP_OK;
}

// micro tangents around zero strain, one serving-loop request per RVE
static int fe2_linear_tangents(sp_fe2 *f) {
  const int nr = f->d.nrve;
  std::vector<int> geom(nr);
  std::vector<double> strain((size_t)nr * 6, 0.0), t_arr(nr, 0.0), t_done(nr);
  std::vector<sp_solve_info> info(nr);
  for (int r = 0; r < nr; r++) geom[r] = r;
  f->clin.assign((size_t)nr * 36, 0.0);
  SP_TRY(sp_server_replay(f->srv, nr, geom.data(), strain.data(), t_arr.data(), t_done.data(),
                          nullptr, f->clin.data(), info.data(), 3600.0));
  // the loop's CTAs fill every SM while it waits for work: stop it so the
  // macro kernels run
  SP_TRY(sp_server_stop(f->srv));
  for (int r = 0; r < nr; r++)
    if (info[r].status) return sp_set_error(SP_ERR_NOCONV, "fe2: micro RVE %d did not converge", r);
  SP_CUDA_TRY(cudaMemcpy(f->d_clin, f->clin.data(), f->clin.size() * sizeof(double),
                         cudaMemcpyHostToDevice));
  return SP_OK;
}

extern "C" int sp_fe2_create(const sp_fe2_desc *desc, sp_fe2 **out) {
  if (!desc || !out) return sp_set_error(SP_ERR_ARG, "sp_fe2_create: null argument");
  const sp_fe2_desc &D = *desc;
  for (int k = 0; k < 3; k++)
    if (D.n[k] < 1 || !(D.len[k] > 0)) return sp_set_error(SP_ERR_ARG, "sp_fe2_create: bad macro mesh");
  if (D.nrve < 1 || !D.rves) return sp_set_error(SP_ERR_ARG, "sp_fe2_create: no micro RVEs");
  if (D.micro != SP_FE2_LINEAR && D.micro != SP_FE2_PER_GP)
    return sp_set_error(SP_ERR_ARG, "sp_fe2_create: unknown micro mode");
  if (D.newton_its < 1 || D.newton_its > SP_FE2_MAX_ITS)
    return sp_set_error(SP_ERR_ARG, "sp_fe2_create: newton_its must be 1..%d", SP_FE2_MAX_ITS);
  Device *dv;
  SP_TRY(device(&dv));
  sp_fe2 *f = new sp_fe2_s();
  f->d = D;
  f->d.rves = nullptr;  // not kept: the server holds the geometries
  f->d.gp_rve = nullptr;
  f->dev = dv->id;
  f->g = make_geo(D.n, D.len);
  f->ngp = f->g.nelm * FE2_GP;
  int rc = plan_acquire(D.n, &f->plan);
  f->gp_rve.resize(f->ngp);
  for (int i = 0; i < f->ngp && !rc; i++) {
    int r = D.gp_rve ? D.gp_rve[i] : (int)(mix64((unsigned long long)D.seed * 1000003ull + i) % D.nrve);
    if (r < 0 || r >= D.nrve) rc = sp_set_error(SP_ERR_RANGE, "sp_fe2_create: gp %d bound to RVE %d", i, r);
    f->gp_rve[i] = r;
  }
  const size_t nd = f->g.ndof, ng = f->ngp;
  if (!rc) rc = dmalloc((void **)&f->d_B, FE2_B * sizeof(double), nullptr);
  if (!rc) rc = dmalloc((void **)&f->d_w, sizeof(double), nullptr);
  if (!rc) rc = dmalloc((void **)&f->d_u, nd * sizeof(double), nullptr);
  if (!rc) rc = dmalloc((void **)&f->d_fext, nd * sizeof(double), nullptr);
  if (!rc) rc = dmalloc((void **)&f->d_b, nd * sizeof(double), nullptr);
  if (!rc) rc = dmalloc((void **)&f->d_eps, ng * 6 * sizeof(double), nullptr);
  if (!rc) rc = dmalloc((void **)&f->d_sig, ng * 6 * sizeof(double), nullptr);
  if (!rc && D.micro == SP_FE2_PER_GP) rc = dmalloc((void **)&f->d_ctan, ng * 36 * sizeof(double), nullptr);
  if (!rc) rc = dmalloc((void **)&f->d_clin, (size_t)D.nrve * 36 * sizeof(double), nullptr);
  if (!rc) rc = dmalloc((void **)&f->d_vals, nd * SP_WP * sizeof(double), nullptr);
  if (!rc) rc = dmalloc((void **)&f->d_dinv, nd * sizeof(double), nullptr);
  if (!rc) rc = dmalloc((void **)&f->d_vec, 4 * nd * sizeof(double), nullptr);
  if (!rc) rc = dmalloc((void **)&f->d_nrm, sizeof(double), nullptr);
  if (!rc) rc = dmalloc((void **)&f->d_gp_rve, ng * sizeof(int), nullptr);
  if (!rc) rc = dmalloc((void **)&f->d_st, sizeof(PcgState), nullptr);
  if (!rc) rc = dmalloc((void **)&f->d_partial, 4096 * 2 * sizeof(double), nullptr);
  if (!rc) rc = dmalloc((void **)&f->d_ticket, 64, nullptr);
  if (!rc && cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking))
    rc = sp_set_error(SP_ERR_CUDA, "sp_fe2_create: stream");
  if (!rc) {
    // consistent nodal forces of the uniform traction on the face x = len[0]
    std::vector<double> fext(nd, 0.0);
    const MeshGeo &g = f->g;
    for (int k = 0; k < g.nz; k++)
      for (int j = 0; j < g.ny; j++) {
        int cy = (j == 0 || j == g.ny - 1) ? 1 : 2, cz = (k == 0 || k == g.nz - 1) ? 1 : 2;
        double a = g.hy * g.hz * cy * cz / 4.0;
        int node = (g.nx - 1) + j * g.nx + k * g.nx * g.ny;
        for (int d = 0; d < 3; d++) fext[(size_t)node * 3 + d] = D.traction[d] * a;
      }
    if (cudaMemcpy(f->d_fext, fext.data(), nd * sizeof(double), cudaMemcpyHostToDevice) ||
        cudaMemcpy(f->d_gp_rve, f->gp_rve.data(), ng * sizeof(int), cudaMemcpyHostToDevice) ||
        cudaMemset(f->d_u, 0, nd * sizeof(double)) || cudaMemset(f->d_ticket, 0, 64))
      rc = sp_set_error(SP_ERR_CUDA, "sp_fe2_create: upload");
  }
  if (!rc) {
    k_fe2_ops<<<1, 256, 0, f->stream>>>(f->g, f->d_B, f->d_w);
    if (cudaGetLastError() || cudaStreamSynchronize(f->stream))
      rc = sp_set_error(SP_ERR_CUDA, "sp_fe2_create: element operators");
  }
  if (!rc) {
    sp_server_opts so;
    sp_server_opts_default(&so);
    rc = sp_server_create(D.nrve, D.rves, &so, &f->srv);
  }
  if (!rc && D.micro == SP_FE2_LINEAR) rc = fe2_linear_tangents(f);
  if (!rc) {
    // the macro system (14,883 dof for 40x10x10) is small: one cooperative
    // launch per solve instead of three launches per CG iteration
    f->pcg = new PcgCoop<double, 1, 8>();
    double *vr = f->d_vec, *vp = vr + nd, *vq = vp + nd, *vdx = vq + nd;
    Device *dv;
    rc = device(&dv);
    if (!rc)
      rc = f->pcg->build(dv, 2048, (int)nd, SP_WP, f->d_vals, f->plan->cols, f->d_dinv, f->d_b,
                         vdx, vr, vp, vq, f->d_st, f->d_partial);
    if (!rc) f->nblk = f->pcg->nblk;
  }
  if (rc) {
    sp_fe2_destroy(f);
    return rc;
  }
  *out = f;
  return SP_OK;
}

// micro stress + tangent for every Gauss point through the serving loop
static int fe2_per_gp(sp_fe2 *f, long long *requests) {
  const size_t ng = f->ngp;
  std::vector<double> eps(ng * 6), sig(ng * 6), ctan(ng * 36), t_arr(ng, 0.0), t_done(ng);
  std::vector<sp_solve_info> info(ng);
  SP_CUDA_TRY(cudaMemcpyAsync(eps.data(), f->d_eps, ng * 6 * sizeof(double), cudaMemcpyDeviceToHost,
                              f->stream));
  SP_CUDA_TRY(cudaStreamSynchronize(f->stream));
  SP_TRY(sp_server_replay(f->srv, (int)ng, f->gp_rve.data(), eps.data(), t_arr.data(),
                          t_done.data(), sig.data(), ctan.data(), info.data(), 3600.0));
  SP_TRY(sp_server_stop(f->srv));  // free the SMs for the macro kernels
  for (size_t i = 0; i < ng; i++)
    if (info[i].status) return sp_set_error(SP_ERR_NOCONV, "fe2: micro request %zu did not converge", i);
  *requests += (long long)ng;
  SP_CUDA_TRY(cudaMemcpyAsync(f->d_sig, sig.data(), ng * 6 * sizeof(double), cudaMemcpyHostToDevice,
                              f->stream));
  SP_CUDA_TRY(cudaMemcpyAsync(f->d_ctan, ctan.data(), ng * 36 * sizeof(double),
                              cudaMemcpyHostToDevice, f->stream));
  SP_CUDA_TRY(cudaStreamSynchronize(f->stream));
  return SP_OK;
}

extern "C" int sp_fe2_run(sp_fe2 *f, sp_fe2_info *info) {
  if (!f) return sp_set_error(SP_ERR_ARG, "sp_fe2_run: null handle");
  sp_fe2_info in;
  memset(&in, 0, sizeof(in));
  in.micro_requests = f->d.micro == SP_FE2_LINEAR ? f->d.nrve : 0;
  const MeshGeo &g = f->g;
  const size_t nd = g.ndof;
  cudaStream_t s = f->stream;
  const DevPlan *pl = f->plan;
  auto blocks = [](long long n) { return (int)std::min<long long>(4096, std::max<long long>(1, (n + 255) / 256)); };
  double *vdx = f->d_vec + 3 * nd;
  // phase timing: events around residual, assembly and solve of each iteration
  cudaEvent_t ev[4];
  for (auto &e : ev) SP_CUDA_TRY(cudaEventCreate(&e));
  struct EvGuard {
    cudaEvent_t *e;
    ~EvGuard() {
      for (int i = 0; i < 4; i++) cudaEventDestroy(e[i]);
    }
  } guard{ev};
  SP_CUDA_TRY(cudaMemsetAsync(f->d_u, 0, nd * sizeof(double), s));
  for (int it = 0; it < f->d.newton_its; it++) {
    double t0 = fe2_now();
    SP_CUDA_TRY(cudaEventRecord(ev[0], s));
    k_fe2_strain<<<blocks(f->ngp), 256, 0, s>>>(g, f->d_B, f->d_u, f->d.strain_clip, f->d_eps);
    SP_CUDA_TRY(cudaGetLastError());
    if (f->d.micro == SP_FE2_PER_GP) {
      double tm = fe2_now();
      SP_TRY(fe2_per_gp(f, &in.micro_requests));
      in.micro_s += fe2_now() - tm;
    } else {
      k_fe2_stress<<<blocks(f->ngp), 256, 0, s>>>(f->ngp, f->d_eps, f->d_gp_rve, f->d_clin, f->d_sig);
    }
    k_fe2_residual<<<blocks(nd), 256, 0, s>>>(g, f->d_B, f->d_w, f->d_sig, f->d_fext, f->d_b);
    k_fe2_norm2<<<1, 1024, 0, s>>>((int)nd, f->d_b, f->d_nrm);
    SP_CUDA_TRY(cudaGetLastError());
    SP_CUDA_TRY(cudaEventRecord(ev[1], s));
    double nrm2 = 0.0;
    SP_CUDA_TRY(cudaMemcpyAsync(&nrm2, f->d_nrm, sizeof(double), cudaMemcpyDeviceToHost, s));
    SP_CUDA_TRY(cudaStreamSynchronize(s));
    in.bnorm[it] = sqrt(nrm2);
    in.newton_its = it + 1;
    if (in.bnorm[it] <= f->d.newton_tol) {
      in.macro_s += fe2_now() - t0;
      break;
    }
    // Jacobian: zero, 8 colour scatters, clamped rows/columns
    SP_CUDA_TRY(cudaMemsetAsync(f->d_vals, 0, nd * SP_WP * sizeof(double), s));
    for (int c = 0; c < 8; c++) {
      int c0 = pl->color_off[c], c1 = pl->color_off[c + 1];
      if (c1 <= c0) continue;
      k_fe2_assemble<<<blocks((long long)(c1 - c0) * SP_KE), 256, 0, s>>>(
          g, pl->color_elems, c0, c1, pl->slot, f->d_B, f->d_w, f->d_gp_rve, f->d_clin,
          f->d.micro == SP_FE2_PER_GP ? f->d_ctan : nullptr, f->d_vals);
    }
    k_fe2_bc<<<blocks(nd), 256, 0, s>>>(g, pl->cols, f->d_vals, f->d_dinv);
    SP_CUDA_TRY(cudaGetLastError());
    SP_CUDA_TRY(cudaEventRecord(ev[2], s));
    // K dx = b
    PcgState st0 = {};
    st0.nactive = 1;
    st0.rtol2 = f->d.lin_rtol * f->d.lin_rtol;
    st0.max_its = 100000;
    SP_CUDA_TRY(cudaMemcpyAsync(f->d_st, &st0, sizeof(st0), cudaMemcpyHostToDevice, s));
    SP_TRY(f->pcg->run(s));
    k_fe2_axpy<<<blocks(nd), 256, 0, s>>>((int)nd, vdx, f->d_u);
    SP_CUDA_TRY(cudaGetLastError());
    SP_CUDA_TRY(cudaEventRecord(ev[3], s));
    PcgState st;
    SP_CUDA_TRY(cudaMemcpyAsync(&st, f->d_st, sizeof(st), cudaMemcpyDeviceToHost, s));
    SP_CUDA_TRY(cudaStreamSynchronize(s));
    float ms[3];
    for (int q = 0; q < 3; q++) SP_CUDA_TRY(cudaEventElapsedTime(&ms[q], ev[q], ev[q + 1]));
    in.residual_ms += ms[0];
    in.assemble_ms += ms[1];
    in.solve_ms += ms[2];
    in.pcg_its[it] = st.its;
    in.macro_s += fe2_now() - t0;
    if (st.active[0])
      return sp_set_error(SP_ERR_NOCONV, "fe2: macro PCG did not converge in %d its", st.its);
  }
  // mean displacement of the loaded face
  std::vector<double> u(nd);
  SP_CUDA_TRY(cudaMemcpy(u.data(), f->d_u, nd * sizeof(double), cudaMemcpyDeviceToHost));
  int cnt = 0;
  for (int k = 0; k < g.nz; k++)
    for (int j = 0; j < g.ny; j++, cnt++)
      for (int d = 0; d < 3; d++) in.tip[d] += u[((size_t)(g.nx - 1) + j * g.nx + k * g.nx * g.ny) * 3 + d];
  for (int d = 0; d < 3; d++) in.tip[d] /= cnt;
  if (info) *info = in;
  return SP_OK;
}

extern "C" int sp_fe2_displacement(const sp_fe2 *f, double *u) {
  if (!f || !u) return sp_set_error(SP_ERR_ARG, "sp_fe2_displacement: null argument");
  SP_CUDA_TRY(cudaMemcpy(u, f->d_u, (size_t)f->g.ndof * sizeof(double), cudaMemcpyDeviceToHost));
  return SP_OK;
}

extern "C" int sp_fe2_gp_rve(const sp_fe2 *f, int *gp_rve) {
  if (!f || !gp_rve) return sp_set_error(SP_ERR_ARG, "sp_fe2_gp_rve: null argument");
  memcpy(gp_rve, f->gp_rve.data(), f->gp_rve.size() * sizeof(int));
  return SP_OK;
}

extern "C" int sp_fe2_micro_tangents(const sp_fe2 *f, double *C) {
  if (!f || !C) return sp_set_error(SP_ERR_ARG, "sp_fe2_micro_tangents: null argument");
  if (f->clin.empty()) return sp_set_error(SP_ERR_STATE, "sp_fe2_micro_tangents: per-Gauss-point mode");
  memcpy(C, f->clin.data(), f->clin.size() * sizeof(double));
  return SP_OK;
}
