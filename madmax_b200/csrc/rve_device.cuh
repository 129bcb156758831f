// rve_device.cuh -- device building blocks of the micro-RVE hot path, shared
// by the plain one-RVE path (rve_plain.cu), the batched persistent kernel
// (rve_batch.cu) and the serving loop (serve.cu).
//
// Every routine is written for a cooperating group of `nt` threads with
// index `t` (a whole grid, or one CTA); the caller places the barriers.
//
// Layouts
//   ELL values/cols : [ndof][SP_WP] row-major, 84 slots (81 used), -1 cols
//                     and 0 values in unused slots.
//   vectors         : [ndof][K] (the K load cases of one dof adjacent).
//   Ke              : [type][24][24] row-major, i = 3*local_node + d.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "sp_internal.h"

namespace sp {

struct MeshGeo {
  int nx, ny, nz;    // nodes per axis
  int nex, ney, nez; // elements per axis
  int ndof, nelm;
  int nn, nn_pad;    // nodes, nodes rounded up to a multiple of 32
  double hx, hy, hz; // element edge lengths
  double vol;        // RVE volume
  int periodic;      // periodic boundary conditions (unknowns on the periodic grid)
  int pad;
};

__host__ __device__ inline bool is_bnode(const MeshGeo &g, int node) {
  int i = node % g.nx, j = (node / g.nx) % g.ny, k = node / (g.nx * g.ny);
  return i == 0 || j == 0 || k == 0 || i == g.nx - 1 || j == g.ny - 1 || k == g.nz - 1;
}

// hexa8 local node a -> corner offset (bit0 x, bit1 y, bit2 z), from the node
// order of src/fem.c:324-362 (0:---, 1:+--, 2:++-, 3:-+-, 4..7 same at z+)
__host__ __device__ inline int corner_x(int a) { return ((a & 3) == 1 || (a & 3) == 2) ? 1 : 0; }
__host__ __device__ inline int corner_y(int a) { return ((a & 3) >= 2) ? 1 : 0; }
__host__ __device__ inline int corner_z(int a) { return a >> 2; }

__device__ inline void elem_nodes(const MeshGeo &g, int e, int *nod) {
  int ex = e % g.nex, ey = (e / g.nex) % g.ney, ez = e / (g.nex * g.ney);
  int nxy = g.nx * g.ny;
  int n0 = ex + ey * g.nx + ez * nxy;
  nod[0] = n0;
  nod[1] = n0 + 1;
  nod[2] = n0 + g.nx + 1;
  nod[3] = n0 + g.nx;
#pragma unroll
  for (int a = 0; a < 4; a++) nod[4 + a] = nod[a] + nxy;
}

// exact (separately rounded) double arithmetic, matching the oracle's
// -ffp-contract=off build bit for bit
__device__ inline double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ inline double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ inline double dsub(double a, double b) { return __dsub_rn(a, b); }

// ------------------------------------------------------------- materials ---

// 3D isotropic D in Voigt (xx,yy,zz,xy,yz,xz) from E, nu, with the Lame
// constants of src/material.c:121-122
__device__ inline void iso_D(double E, double nu, double *D) {
  double lam = __ddiv_rn(dmul(E, nu), dmul(dadd(1.0, nu), dsub(1.0, dmul(2.0, nu))));
  double mu = __ddiv_rn(E, dmul(2.0, dadd(1.0, nu)));
  for (int i = 0; i < 36; i++) D[i] = 0.0;
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < 3; j++) D[i * 6 + j] = lam;
    D[i * 6 + i] = dadd(lam, dmul(2.0, mu));
    D[(3 + i) * 6 + (3 + i)] = mu;
  }
}

// ------------------------------------------------------ element operators ---

#define SP_GP 0.577350269189626

// dsh[a][d][gp] = dN_a/dxi_d(gp) * 2/h_d (src/fem.c:3-59 extended to 3D with
// the hexa8 tables of src/fem.c:309-405); 192 entries
__device__ inline double dsh_entry(int a, int d, int gp, const double h[3]) {
  int s[3] = {corner_x(a) ? 1 : -1, corner_y(a) ? 1 : -1, corner_z(a) ? 1 : -1};
  int q[3] = {corner_x(gp) ? 1 : -1, corner_y(gp) ? 1 : -1, corner_z(gp) ? 1 : -1};
  double f[3];
  for (int e = 0; e < 3; e++) {
    double x = q[e] * SP_GP;
    f[e] = (s[e] < 0) ? dsub(1.0, x) : dadd(1.0, x);
  }
  double v = s[d] * 1.0;
  for (int e = 0; e < 3; e++)
    if (e != d) v = dmul(v, f[e]);
  v = dmul(v, 0.125);
  return __ddiv_rn(dmul(v, 2.0), h[d]);
}

// B[v][i] at one Gauss point from dsh (micro/src/init.c:40-51 extended to 3D)
__device__ inline double bmat_entry(const double *dsh, int v, int i, int gp) {
  int a = i / 3, c = i % 3;
  const double *da = dsh + a * 24; // [d][gp]
  switch (v) {
    case 0: return c == 0 ? da[0 * 8 + gp] : 0.0;
    case 1: return c == 1 ? da[1 * 8 + gp] : 0.0;
    case 2: return c == 2 ? da[2 * 8 + gp] : 0.0;
    case 3: return c == 0 ? da[1 * 8 + gp] : (c == 1 ? da[0 * 8 + gp] : 0.0);
    case 4: return c == 1 ? da[2 * 8 + gp] : (c == 2 ? da[1 * 8 + gp] : 0.0);
    default: return c == 0 ? da[2 * 8 + gp] : (c == 2 ? da[0 * 8 + gp] : 0.0);
  }
}

// Group-cooperative set-up of the element operators for ntype materials:
//   dsh[192], Ke[t][576] = sum_gp B^T D_t B w (micro/src/assembly.c:97-108,
//   same summation order, terms with a zero factor skipped, which leaves the
//   sum unchanged), Bbar[6][24] = sum_gp w B(gp).
// Needs a barrier between the two calls.
__device__ inline void elem_ops_stage1(int t, int nt, const double h[3], double *dsh) {
  for (int x = t; x < 192; x += nt) {
    int a = x / 24, d = (x / 8) % 3, gp = x % 8;
    dsh[x] = dsh_entry(a, d, gp, h);
  }
}

__device__ inline void elem_ops_stage2(int t, int nt, const double h[3], const double *dsh,
                                       const double *D /*[ntype][36]*/, int ntype,
                                       double *Ke /*[ntype][576]*/, double *Bbar /*[144]*/) {
  double w = __ddiv_rn(dmul(dmul(h[0], h[1]), h[2]), 8.0);
  for (int x = t; x < ntype * SP_KE; x += nt) {
    int ty = x / SP_KE, ij = x % SP_KE, i = ij / SP_NC, j = ij % SP_NC;
    const double *C = D + ty * 36;
    double s = 0.0;
    for (int gp = 0; gp < 8; gp++) {
      for (int k = 0; k < 6; k++) {
        double bkj = bmat_entry(dsh, k, j, gp);
        if (bkj == 0.0) continue;
        for (int hh = 0; hh < 6; hh++) {
          double bhi = bmat_entry(dsh, hh, i, gp);
          double c = C[hh * 6 + k];
          if (bhi == 0.0 || c == 0.0) continue;
          s = dadd(s, dmul(dmul(dmul(bhi, c), bkj), w));
        }
      }
    }
    Ke[x] = s;
  }
  if (Bbar) {
    for (int x = t; x < 144; x += nt) {
      int v = x / 24, i = x % 24;
      double s = 0.0;
      for (int gp = 0; gp < 8; gp++) s = dadd(s, dmul(bmat_entry(dsh, v, i, gp), w));
      Bbar[x] = s;
    }
  }
}

// ------------------------------------------------------------- assembly ---

// Zero the values of an ELL matrix (ndof rows of SP_WP slots).
template <typename T>
__device__ inline void ell_zero(int t, int nt, T *vals, int ndof) {
  size_t n = (size_t)ndof * SP_WP;
  if (sizeof(T) == 4) {
    float4 *v4 = reinterpret_cast<float4 *>(vals);
    for (size_t x = t; x < n / 4; x += nt) v4[x] = make_float4(0.f, 0.f, 0.f, 0.f);
  } else {
    double2 *v2 = reinterpret_cast<double2 *>(vals);
    for (size_t x = t; x < n / 2; x += nt) v2[x] = make_double2(0.0, 0.0);
  }
}

// One colour of the conflict-free scatter: for every element e of the colour
// and every (i, j), vals[dof(e,i)][slot(e,i,j)] += Ke[type(e)][i][j].
// Elements of one colour (same parity of ex, ey, ez) share no node, so the
// work items of one colour write pairwise distinct slots; colours run in a
// fixed order, so the sums are deterministic.
template <typename T>
__device__ inline void scatter_colour(int t, int nt, const MeshGeo &g, const int *color_elems,
                                      int c0, int c1, const uint8_t *__restrict__ slot,
                                      const uint8_t *__restrict__ etype, const T *Ke /*[2][576]*/,
                                      T *vals) {
  int nwork = (c1 - c0) * SP_KE;
  for (int x = t; x < nwork; x += nt) {
    int e = color_elems[c0 + x / SP_KE];
    int ij = x % SP_KE;
    int i = ij / SP_NC;
    int nod[8];
    elem_nodes(g, e, nod);
    int row = nod[i / 3] * 3 + i % 3;
    int s = slot[(size_t)e * SP_KE + ij];
    vals[(size_t)row * SP_WP + s] += Ke[etype[e] * SP_KE + ij];
  }
}

// Dirichlet rows and columns of every boundary dof (micro/src/assembly.c:
// 112-135, the column cleared in every row) and the Jacobi diagonal inverse.
template <typename T>
__device__ inline void bc_and_dinv(int t, int nt, const MeshGeo &g, const int *__restrict__ cols,
                                   T *vals, T *dinv) {
  for (int row = t; row < g.ndof; row += nt) {
    bool brow = is_bnode(g, row / 3);
    const int *c = cols + (size_t)row * SP_WP;
    T *v = vals + (size_t)row * SP_WP;
    T diag = 0;
    for (int s = 0; s < SP_ELL_WIDTH; s++) {
      int col = c[s];
      if (col < 0) break;
      if (brow)
        v[s] = (col == row) ? T(1) : T(0);
      else if (is_bnode(g, col / 3))
        v[s] = T(0);
      if (col == row) diag = v[s];
    }
    dinv[row] = T(1) / diag;
  }
}

// ------------------------------------------------------------ load cases ---

// u = eps . x on boundary dofs (micro/src/homogenize.c:227-242, 335-342 in
// 3D), zero elsewhere -- or, with `inside`, eps . x at every node (the
// homogeneous affine start iterate); eps[k][6] Voigt with engineering shears.
template <int K>
__device__ inline void affine_init(int t, int nt, const MeshGeo &g, const double *eps, int nrhs,
                                   double *u, bool inside = false) {
  for (int x = t; x < g.ndof * K; x += nt) {
    int dof = x / K, k = x % K;
    int node = dof / 3, d = dof % 3;
    double val = 0.0;
    if (k < nrhs && (inside || is_bnode(g, node))) {
      int i = node % g.nx, j = (node / g.nx) % g.ny, kk = node / (g.nx * g.ny);
      double X = i * g.hx, Y = j * g.hy, Z = kk * g.hz;
      const double *e = eps + k * 6;
      if (d == 0)
        val = dadd(dadd(dmul(e[0], X), dmul(e[3] / 2, Y)), dmul(e[5] / 2, Z));
      else if (d == 1)
        val = dadd(dadd(dmul(e[3] / 2, X), dmul(e[1], Y)), dmul(e[4] / 2, Z));
      else
        val = dadd(dadd(dmul(e[5] / 2, X), dmul(e[4] / 2, Y)), dmul(e[2], Z));
    }
    u[x] = val;
  }
}

// Keep the interior of a warm start, overwrite the boundary with eps . x.
template <int K>
__device__ inline void affine_boundary(int t, int nt, const MeshGeo &g, const double *eps,
                                       int nrhs, double *u) {
  for (int x = t; x < g.ndof * K; x += nt) {
    int dof = x / K, k = x % K;
    int node = dof / 3, d = dof % 3;
    if (!is_bnode(g, node)) {
      if (k >= nrhs) u[x] = 0.0;
      continue;
    }
    double val = 0.0;
    if (k < nrhs) {
      int i = node % g.nx, j = (node / g.nx) % g.ny, kk = node / (g.nx * g.ny);
      double X = i * g.hx, Y = j * g.hy, Z = kk * g.hz;
      const double *e = eps + k * 6;
      if (d == 0)
        val = dadd(dadd(dmul(e[0], X), dmul(e[3] / 2, Y)), dmul(e[5] / 2, Z));
      else if (d == 1)
        val = dadd(dadd(dmul(e[3] / 2, X), dmul(e[1], Y)), dmul(e[4] / 2, Z));
      else
        val = dadd(dadd(dmul(e[5] / 2, X), dmul(e[4] / 2, Y)), dmul(e[2], Z));
    }
    u[x] = val;
  }
}

// ------------------------------------------------- FP64 element residual ---

// Newton right-hand side b = -K u on interior dofs, 0 on boundary dofs
// (micro/src/assembly.c:33-82 then negative_res, micro/src/homogenize.c:
// 289-303): one thread per dof row sums, over the (up to 8) elements of the
// row's node, Ke_t[row][:] u_e.  For linear elastic elements Ke_t u_e =
// sum_gp B^T sigma(B u_e) w exactly.  Writes b into rb (type R) and adds
// |b|^2 per load case into nrm2[K].
template <int K, typename R>
__device__ inline void residual_nodes(int t, int nt, const MeshGeo &g,
                                      const uint8_t *__restrict__ etype,
                                      const double *Ke /*[2][576], shared*/,
                                      const double *__restrict__ u, R *rb, double *nrm2) {
  for (int row = t; row < g.ndof; row += nt) {
    int node = row / 3, d = row % 3;
    int i = node % g.nx, j = (node / g.nx) % g.ny, k = node / (g.nx * g.ny);
    double acc[K];
#pragma unroll
    for (int q = 0; q < K; q++) acc[q] = 0.0;
    bool bnd = (i == 0 || j == 0 || k == 0 || i == g.nx - 1 || j == g.ny - 1 || k == g.nz - 1);
    if (!bnd) {
      // interior node: all 8 surrounding elements exist
#pragma unroll 1
      for (int c = 0; c < 8; c++) {
        int ox = (c & 1), oy = (c >> 1) & 1, oz = c >> 2;
        int ex = i - 1 + ox, ey = j - 1 + oy, ez = k - 1 + oz;
        int e = ex + ey * g.nex + ez * g.nex * g.ney;
        // local index of this node in element e: corner (1-ox, 1-oy, 1-oz)
        int cx = 1 - ox, cy = 1 - oy, cz = 1 - oz;
        int la = cz * 4 + ((cy == 0) ? (cx ? 1 : 0) : (cx ? 2 : 3));
        const double *ke = Ke + etype[e] * SP_KE + (la * 3 + d) * SP_NC;
        int n0 = ex + ey * g.nx + ez * g.nx * g.ny;
#pragma unroll 2
        for (int b = 0; b < 8; b++) {
          int nb = n0 + corner_x(b) + corner_y(b) * g.nx + corner_z(b) * g.nx * g.ny;
          const double *ub = u + (size_t)nb * 3 * K;
#pragma unroll
          for (int db = 0; db < 3; db++) {
            double kv = ke[b * 3 + db];
#pragma unroll
            for (int q = 0; q < K; q++) acc[q] = fma(kv, ub[db * K + q], acc[q]);
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < K; q++) {
      double b = -acc[q];
      rb[(size_t)row * K + q] = (R)b;
      nrm2[q] += b * b;
    }
  }
}

// --------------------------------------------------------------- SpMM ---

// Load the K values of one dof.  NC: the data is read-only for the whole
// kernel, so the non-coherent path may be used; otherwise (vectors the same
// kernel rewrites) plain loads keep CTA-level coherence after a barrier.
template <typename T, int K, bool NC>
__device__ inline void load_k(const T *p, T *o) {
  constexpr int B = (int)sizeof(T) * K;
  if constexpr (B % 16 == 0) {
    const int4 *q = reinterpret_cast<const int4 *>(p);
#pragma unroll
    for (int x = 0; x < B / 16; x++) {
      int4 w = NC ? __ldg(q + x) : q[x];
      memcpy(reinterpret_cast<char *>(o) + 16 * x, &w, 16);
    }
  } else if constexpr (B % 8 == 0) {
    const int2 *q = reinterpret_cast<const int2 *>(p);
#pragma unroll
    for (int x = 0; x < B / 8; x++) {
      int2 w = NC ? __ldg(q + x) : q[x];
      memcpy(reinterpret_cast<char *>(o) + 8 * x, &w, 8);
    }
  } else {
#pragma unroll
    for (int x = 0; x < K; x++) o[x] = NC ? __ldg(p + x) : p[x];
  }
}

// y = A x for K right-hand sides, L lanes per ELL row (L divides 32), 128-bit
// loads of values and column indices.  wp (row stride in slots) must be a
// multiple of 4 so that every row starts on a 16-byte boundary.  Also adds sum_row x.y per load case
// into dot[K] (lane 0 of each row group).  Every lane of a warp runs the same
// number of loop trips, so the shuffles always see the whole warp.  NC
// selects the non-coherent path for x (only when no thread of the kernel
// writes x).
template <typename T, int K, int L, bool NC = true>
__device__ inline void spmm(int t, int nt, int nrow, int wp, const T *__restrict__ vals,
                            const int *__restrict__ cols, const T *__restrict__ x, T *y,
                            double *dot) {
  constexpr int VEC = 16 / sizeof(T);    // values per 128-bit load
  const int NCH = wp / VEC;              // 21 (FP32) or 42 (FP64) chunks per 84-slot row
  constexpr int RPW = 32 / L;            // rows per warp per trip
  const int lane = t & 31;
  const int gl = lane % L;
  const int warp = t >> 5;
  const int nwarps = nt >> 5;
  for (int rb = warp * RPW; rb < nrow; rb += nwarps * RPW) {
    int row = rb + lane / L;
    bool valid = row < nrow;
    int rr = valid ? row : nrow - 1;
    float acc32[K];
    double acc64[K];
#pragma unroll
    for (int q = 0; q < K; q++) {
      acc32[q] = 0.f;
      acc64[q] = 0.0;
    }
    const T *vr = vals + (size_t)rr * wp;
    const int *cr = cols + (size_t)rr * wp;
    for (int ch = gl; ch < NCH; ch += L) {
      if constexpr (sizeof(T) == 4) {
        float4 v = __ldcs(reinterpret_cast<const float4 *>(vr) + ch);
        int4 c = __ldg(reinterpret_cast<const int4 *>(cr) + ch);
        float vv[4] = {v.x, v.y, v.z, v.w};
        int cc[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
        for (int s = 0; s < 4; s++) {
          int col = cc[s] < 0 ? 0 : cc[s];
          T xv[K];
          load_k<T, K, NC>(x + (size_t)col * K, xv);
#pragma unroll
          for (int q = 0; q < K; q++) acc32[q] = fmaf(vv[s], xv[q], acc32[q]);
        }
      } else {
        double2 v = __ldcs(reinterpret_cast<const double2 *>(vr) + ch);
        int2 c = __ldg(reinterpret_cast<const int2 *>(cr) + ch);
        double vv[2] = {v.x, v.y};
        int cc[2] = {c.x, c.y};
#pragma unroll
        for (int s = 0; s < 2; s++) {
          int col = cc[s] < 0 ? 0 : cc[s];
          T xv[K];
          load_k<T, K, NC>(x + (size_t)col * K, xv);
#pragma unroll
          for (int q = 0; q < K; q++) acc64[q] = fma(vv[s], (double)xv[q], acc64[q]);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < K; q++) {
      if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int off = L / 2; off > 0; off >>= 1)
          acc32[q] += __shfl_xor_sync(0xffffffffu, acc32[q], off);
      } else {
#pragma unroll
        for (int off = L / 2; off > 0; off >>= 1)
          acc64[q] += __shfl_xor_sync(0xffffffffu, acc64[q], off);
      }
    }
    if (valid && gl == 0) {
#pragma unroll
      for (int q = 0; q < K; q++) {
        T r = (sizeof(T) == 4) ? (T)acc32[q] : (T)acc64[q];
        y[(size_t)row * K + q] = r;
        dot[q] += (double)r * (double)x[(size_t)row * K + q];
      }
    }
  }
}

// y = A x on the 84-slot RVE layout with the row's value/column loads all
// issued before its gathers (the chunk count is a compile-time constant, so
// the loop unrolls and the loads overlap).  Same contract as spmm.
template <typename T, int K, int L, bool NC>
__device__ inline void spmm_rve(int t, int nt, int nrow, const T *__restrict__ vals,
                                const int *__restrict__ cols, const T *__restrict__ x, T *y,
                                double *dot) {
  constexpr int VEC = 16 / sizeof(T);
  constexpr int NCH = SP_WP / VEC;
  constexpr int NIT = (NCH + L - 1) / L;
  constexpr int RPW = 32 / L;
  using A = typename std::conditional<sizeof(T) == 4, float, double>::type;
  const int lane = t & 31;
  const int gl = lane % L;
  const int warp = t >> 5;
  const int nwarps = nt >> 5;
  for (int rb = warp * RPW; rb < nrow; rb += nwarps * RPW) {
    int row = rb + lane / L;
    bool valid = row < nrow;
    int rr = valid ? row : nrow - 1;
    const int4 *vr = reinterpret_cast<const int4 *>(vals + (size_t)rr * SP_WP);
    const int *cr = cols + (size_t)rr * SP_WP;
    int4 vv[NIT];
    int cc[NIT][VEC];
#pragma unroll
    for (int it = 0; it < NIT; it++) {
      int ch = gl + it * L;
      if (ch < NCH) {
        vv[it] = __ldcs(vr + ch);
        if constexpr (VEC == 4) {
          int4 c = __ldg(reinterpret_cast<const int4 *>(cr) + ch);
          cc[it][0] = c.x; cc[it][1] = c.y; cc[it][2] = c.z; cc[it][3] = c.w;
        } else {
          int2 c = __ldg(reinterpret_cast<const int2 *>(cr) + ch);
          cc[it][0] = c.x; cc[it][1] = c.y;
        }
      } else {
        vv[it] = make_int4(0, 0, 0, 0);
#pragma unroll
        for (int s = 0; s < VEC; s++) cc[it][s] = -1;
      }
    }
    A acc[K];
#pragma unroll
    for (int q = 0; q < K; q++) acc[q] = A(0);
#pragma unroll
    for (int it = 0; it < NIT; it++) {
      T v[VEC];
      memcpy(v, &vv[it], 16);
#pragma unroll
      for (int s = 0; s < VEC; s++) {
        int col = cc[it][s] < 0 ? 0 : cc[it][s];
        T xv[K];
        load_k<T, K, NC>(x + (size_t)col * K, xv);
#pragma unroll
        for (int q = 0; q < K; q++) acc[q] = fma((A)v[s], (A)xv[q], acc[q]);
      }
    }
#pragma unroll
    for (int q = 0; q < K; q++)
#pragma unroll
      for (int off = L / 2; off > 0; off >>= 1)
        acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], off);
    if (valid && gl == 0) {
      T o[K];
#pragma unroll
      for (int q = 0; q < K; q++) {
        o[q] = (T)acc[q];
        dot[q] += (double)o[q] * (double)x[(size_t)row * K + q];
      }
#pragma unroll
      for (int q = 0; q < K; q++) y[(size_t)row * K + q] = o[q];
    }
  }
}

// Row-chunked access to [rows][K] vectors with 16-byte loads: a super-chunk
// holds S = lcm(K, 16/sizeof(T)) values = RPC whole rows, so the load case of
// every element is a compile-time constant.  Vectors are padded to a
// multiple of 4 rows (zero-filled), which every RPC divides.
template <typename T, int K>
struct Chunks {
  static constexpr int E = 16 / sizeof(T);
  static constexpr int gcd(int a, int b) { return b ? gcd(b, a % b) : a; }
  static constexpr int S = K / gcd(K, E) * E;
  static constexpr int RPC = S / K;
  static constexpr int NV = S / E;
  __device__ static void load(const T *p, T *v) {
    const int4 *q = reinterpret_cast<const int4 *>(p);
#pragma unroll
    for (int i = 0; i < NV; i++) {
      int4 w = q[i];
      memcpy(reinterpret_cast<char *>(v) + 16 * i, &w, 16);
    }
  }
  __device__ static void store(T *p, const T *v) {
    int4 *q = reinterpret_cast<int4 *>(p);
#pragma unroll
    for (int i = 0; i < NV; i++) {
      int4 w;
      memcpy(&w, reinterpret_cast<const char *>(v) + 16 * i, 16);
      q[i] = w;
    }
  }
};

// ------------------------------------------------ node-sliced ELL path ---
//
// The batched and serving solves read each RVE's ELL matrix through a
// node-sliced copy of the same values: the 3x3 block (node a, group m) of
// rows 3a..3a+2, slots 3m..3m+2 is stored at
//   nsv[((s*27 + m)*9 + 3d + c)*32 + l],  a = 32 s + l,
// with the block's column node in nbr[(s*27 + m)*32 + l].  A warp owns a
// slice of 32 consecutive nodes, a lane one node (three rows).  Values,
// neighbour ids and the K-vectors of neighbours are then all read with
// whole-warp coalesced accesses (interior nodes of a slice share the group
// order, so their neighbours are consecutive too).  Vectors are
// component-major: v[(k*3 + d)*nn_pad + node].

// Row-major ELL (values after Dirichlet) -> node-sliced values and the
// component-major Jacobi diagonal.
template <typename T>
__device__ inline void ns_from_rows(int t, int nt, const MeshGeo &g, const int *__restrict__ cols,
                                    const T *vals_rm, const T *dinv_rm, T *nsv, T *dinv) {
  const size_t total = (size_t)(g.nn_pad / 32) * 27 * 9 * 32;
  for (size_t x = t; x < total; x += nt) {
    int l = (int)(x % 32);
    size_t q = x / 32;
    int i = (int)(q % 9);
    size_t sm = q / 9;
    int m = (int)(sm % 27), s = (int)(sm / 27);
    int a = s * 32 + l, d = i / 3, c = i % 3;
    T v = T(0);
    if (a < g.nn) {
      size_t o = (size_t)(3 * a + d) * SP_WP + 3 * m + c;
      if (cols[o] >= 0) v = vals_rm[o];
    }
    nsv[x] = v;
  }
  for (int x = t; x < 3 * g.nn_pad; x += nt) {
    int d = x / g.nn_pad, a = x % g.nn_pad;
    dinv[x] = (a < g.nn) ? dinv_rm[3 * a + d] : T(0);
  }
}

// y = A x (K right-hand sides) on the node-sliced layout; adds x.y per load
// case into dot[K].
template <typename T, int K, bool NC>
__device__ inline void spmm_ns(int t, int nt, const MeshGeo &g, const T *__restrict__ nsv,
                               const int *__restrict__ nbr, const T *__restrict__ x, T *y,
                               double *dot) {
  using A = typename std::conditional<sizeof(T) == 4, float, double>::type;
  const int lane = t & 31, warp = t >> 5, nwarps = nt >> 5;
  const int nslice = g.nn_pad / 32;
  const size_t blk = (size_t)3 * g.nn_pad;
  for (int s = warp; s < nslice; s += nwarps) {
    A acc[3][K];
#pragma unroll
    for (int d = 0; d < 3; d++)
#pragma unroll
      for (int k = 0; k < K; k++) acc[d][k] = A(0);
    const T *vs = nsv + (size_t)s * 27 * 9 * 32 + lane;
    const int *bs = nbr + (size_t)s * 27 * 32 + lane;
#pragma unroll 3
    for (int m = 0; m < 27; m++) {
      int b = __ldg(bs + m * 32);
      T v[9];
#pragma unroll
      for (int i = 0; i < 9; i++) v[i] = __ldcs(vs + (m * 9 + i) * 32);
#pragma unroll
      for (int k = 0; k < K; k++) {
        A xb[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const T *xp = x + k * blk + (size_t)c * g.nn_pad + b;
          xb[c] = NC ? (A)__ldg(xp) : (A)*xp;
        }
#pragma unroll
        for (int d = 0; d < 3; d++)
#pragma unroll
          for (int c = 0; c < 3; c++) acc[d][k] = fma((A)v[d * 3 + c], xb[c], acc[d][k]);
      }
    }
    const int a = s * 32 + lane;
#pragma unroll
    for (int k = 0; k < K; k++)
#pragma unroll
      for (int d = 0; d < 3; d++) {
        size_t o = k * blk + (size_t)d * g.nn_pad + a;
        T yv = (T)acc[d][k];
        dot[k] += (double)yv * (double)x[o];
        y[o] = yv;
      }
  }
}

// ------------------------------------------------ element-type stencil ---
//
// Every element of the structured RVE mesh has the same shape, so its
// assembled matrix is fixed by the element stiffnesses of the two materials
// and the material id of each element.  The stencil operator applies A x
// without reading an assembled matrix: for an interior node a and each of
// its 27 neighbours b it sums the 3x3 block
//   A_ab = sum over the elements e holding both a and b of Ke[type(e)][a_e][b_e]
// from shared-memory copies of the two Ke, then multiplies the block into the
// K right-hand sides.  Only interior nodes are computed.  Dirichlet rows are
// the identity and Dirichlet columns zero in the assembled matrix; the CG
// vectors are zero on boundary nodes, so a boundary row of A p is 0 and a
// boundary column contributes 0, which is what this operator gives when the
// caller keeps y zero on boundary nodes.

// hexa8 local node index of the element corner (cx, cy, cz) (node order of
// src/fem.c:324-362)
__host__ __device__ constexpr int hex8_local(int cx, int cy, int cz) {
  return cz * 4 + (cy == 0 ? (cx ? 1 : 0) : (cx ? 2 : 3));
}

// The node-sliced values of the assembled, Dirichlet-reduced matrix straight
// from the element matrices, without a row-major scratch or a scatter: the
// block (node a, group m) is owned by one thread, which sums, in FP64, the
// (a, b) blocks Ke[t][3la+d][3lb+c] of the elements holding a and its
// neighbour b = nbr(a, m), and rounds once to T.  Dirichlet rows are
// identity rows and Dirichlet columns zero, as bc_and_dinv leaves them;
// unused groups (cols < 0) are zero.  The same matrix as the coloured scatter
// followed by ns_from_rows, up to the rounding of the sums.  dinv: the
// component-major Jacobi diagonal (1 on Dirichlet rows, 0 on padding).
template <typename T>
__device__ inline void ns_from_elements(int t, int nt, const MeshGeo &g,
                                        const int *__restrict__ cols, const int *__restrict__ nbr,
                                        const uint8_t *__restrict__ etype,
                                        const double *Ke /*[2][576], shared*/, T *nsv, T *dinv) {
  const size_t total = (size_t)(g.nn_pad / 32) * 27 * 32;
  const int esy = g.nex, esz = g.nex * g.ney;
  for (size_t x = t; x < total; x += nt) {
    const int l = (int)(x % 32);
    const size_t sm = x / 32;
    const int m = (int)(sm % 27), s = (int)(sm / 27);
    const int a = s * 32 + l;
    double bv[9];
#pragma unroll
    for (int i = 0; i < 9; i++) bv[i] = 0.0;
    if (a < g.nn && cols[(size_t)(3 * a) * SP_WP + 3 * m] >= 0) {
      const int b = nbr[x];
      if (is_bnode(g, a)) {
        if (b == a) bv[0] = bv[4] = bv[8] = 1.0;
      } else if (!is_bnode(g, b)) {
        const int ia = a % g.nx, ja = (a / g.nx) % g.ny, ka = a / (g.nx * g.ny);
        const int dx = b % g.nx - ia, dy = (b / g.nx) % g.ny - ja, dz = b / (g.nx * g.ny) - ka;
        for (int c8 = 0; c8 < 8; c8++) {
          const int ox = c8 & 1, oy = (c8 >> 1) & 1, oz = c8 >> 2;
          const int bx = 1 - ox + dx, by = 1 - oy + dy, bz = 1 - oz + dz;
          if (bx < 0 || bx > 1 || by < 0 || by > 1 || bz < 0 || bz > 1) continue;
          const int e = (ia - 1 + ox) + (ja - 1 + oy) * esy + (ka - 1 + oz) * esz;
          const double *ke = Ke + (int)__ldg(etype + e) * SP_KE;
          const int la = hex8_local(1 - ox, 1 - oy, 1 - oz), lb = hex8_local(bx, by, bz);
#pragma unroll
          for (int d = 0; d < 3; d++)
#pragma unroll
            for (int c = 0; c < 3; c++) bv[3 * d + c] += ke[(3 * la + d) * SP_NC + 3 * lb + c];
        }
      }
    }
    T *dst = nsv + (size_t)(s * 27 + m) * 9 * 32 + l;
#pragma unroll
    for (int i = 0; i < 9; i++) dst[i * 32] = (T)bv[i];
  }
  for (int x = t; x < 3 * g.nn_pad; x += nt) {
    const int d = x / g.nn_pad, a = x % g.nn_pad;
    T v = T(0);
    if (a < g.nn) {
      if (is_bnode(g, a)) {
        v = T(1);
      } else {
        const int ia = a % g.nx, ja = (a / g.nx) % g.ny, ka = a / (g.nx * g.ny);
        double sdiag = 0.0;
        for (int c8 = 0; c8 < 8; c8++) {
          const int ox = c8 & 1, oy = (c8 >> 1) & 1, oz = c8 >> 2;
          const int e = (ia - 1 + ox) + (ja - 1 + oy) * esy + (ka - 1 + oz) * esz;
          const int la = hex8_local(1 - ox, 1 - oy, 1 - oz);
          sdiag += Ke[(int)__ldg(etype + e) * SP_KE + (3 * la + d) * SP_NC + 3 * la + d];
        }
        v = (T)(1.0 / sdiag);
      }
    }
    dinv[x] = v;
  }
}


constexpr int SP_KB_BLK = 12;                        // padded 3x3 block (16-byte rows for float)
// element blocks of one material, padded by 4 entries: the two materials'
// blocks then start in different shared-memory banks, so a warp whose lanes
// read the same block of both materials is served without bank conflicts
constexpr int SP_KB_TYPE = 64 * SP_KB_BLK + 4;
constexpr int SP_KA_OFF = 0;                         // KA[t][m]: 2 x 27 blocks
constexpr int SP_KE_OFF = 2 * 27 * SP_KB_BLK;        // KE[t][la][lb]: 2 x 64 blocks
constexpr int SP_KB_SIZE = SP_KE_OFF + 2 * SP_KB_TYPE;

// Shared tables of the stencil operator (T values, summed in FP64 and
// rounded once; block entry 3d + c, 3 zero pads):
//   KA[t][m]      the assembled block of neighbour m = (dx+1) + 3(dy+1) + 9(dz+1)
//                 of a node whose 8 elements are all of material t;
//   KE[t][la][lb] Ke[t][3la + d][3lb + c], the element blocks.
template <typename T>
__device__ inline void stencil_blocks(int t, int nt, const double *Ke /*[2][576]*/, T *KB) {
  for (int x = t; x < SP_KB_SIZE; x += nt) {
    double v = 0.0;
    // entry w of block b within the KA part or within one material's KE part
    const int r = x < SP_KE_OFF ? x : (x - SP_KE_OFF) % SP_KB_TYPE;
    const int w = r % SP_KB_BLK;
    if (w < 9 && r < 64 * SP_KB_BLK) {
      const int d = w / 3, cc = w % 3;
      if (x < SP_KE_OFF) {
        const int ty = x / (27 * SP_KB_BLK), m = (x / SP_KB_BLK) % 27;
        const int dx = m % 3 - 1, dy = (m / 3) % 3 - 1, dz = m / 9 - 1;
        for (int c = 0; c < 8; c++) {
          const int ox = c & 1, oy = (c >> 1) & 1, oz = c >> 2;
          const int bx = 1 - ox + dx, by = 1 - oy + dy, bz = 1 - oz + dz;
          if (bx < 0 || bx > 1 || by < 0 || by > 1 || bz < 0 || bz > 1) continue;
          const int la = hex8_local(1 - ox, 1 - oy, 1 - oz), lb = hex8_local(bx, by, bz);
          v += Ke[ty * SP_KE + (3 * la + d) * SP_NC + 3 * lb + cc];
        }
      } else {
        const int ty = (x - SP_KE_OFF) / SP_KB_TYPE, b = r / SP_KB_BLK;
        const int la = b / 8, lb = b % 8;
        v = Ke[ty * SP_KE + (3 * la + d) * SP_NC + 3 * lb + cc];
      }
    }
    KB[x] = (T)v;
  }
}

// Pattern tables of the FP32 stencil operator.  The block that couples a
// node with its neighbour m = (dx+1) + 3(dy+1) + 9(dz+1) is the sum of the
// element blocks of the sp_pt_n(m) elements the two nodes share (8 for the
// node itself, 4 across a face, 2 across an edge, 1 across a corner); with
// two materials it takes one of 2^sp_pt_n(m) values, one per material
// pattern of those elements.  The table holds every one of them, summed in
// FP64 and rounded once (416 blocks), so a node of any material mix reads
// its 27 blocks directly instead of summing up to 64 element blocks.
// Pattern bit i is the material of the i-th shared element in increasing
// corner order c = ox + 2oy + 4oz (the element at (i-1+ox, j-1+oy, k-1+oz)).
__host__ __device__ constexpr int sp_pt_n(int m) {
  return (m % 3 == 1 ? 2 : 1) * ((m / 3) % 3 == 1 ? 2 : 1) * (m / 9 == 1 ? 2 : 1);
}
__host__ __device__ constexpr int sp_pt_off(int m) {
  int o = 0;
  for (int i = 0; i < m; i++) o += 1 << sp_pt_n(i);
  return o;
}
constexpr int SP_PT_NREC = sp_pt_off(27);  // 416 blocks
// Layout: entries 0..7 of block b at [8b, 8b+8) (two 16-byte loads), entry 8
// at [8 * SP_PT_NREC + b]: 36 bytes read per block and 15 KB in all, no
// padding (records of 9 + 3 padding floats took 20 KB).
constexpr int SP_PT_BYTES = SP_PT_NREC * 9 * 4;
static_assert(SP_PT_NREC == 256 + 6 * 16 + 12 * 4 + 8 * 2, "pattern table size");

// The pattern-table block of a node with material mask `mask` (bit c: the
// element at corner c) for the neighbour at offset (dx, dy, dz).
__device__ __forceinline__ int sp_pt_index(unsigned mask, int dx, int dy, int dz) {
  unsigned q0 = 0, q1 = 0;
  int nb = 0;
#pragma unroll
  for (int c2 = 0; c2 < 4; c2++) {
    const int ox = c2 & 1, oy = c2 >> 1;
    if ((dx < 0 && ox) || (dx > 0 && !ox) || (dy < 0 && oy) || (dy > 0 && !oy)) continue;
    q0 |= ((mask >> c2) & 1u) << nb;
    q1 |= ((mask >> (c2 + 4)) & 1u) << nb;
    nb++;
  }
  const int m0 = (dx + 1) + 3 * (dy + 1);
  return dz < 0 ? sp_pt_off(m0) + (int)q0
                : (dz == 0 ? sp_pt_off(m0 + 9) + (int)(q0 | (q1 << nb)) : sp_pt_off(m0 + 18) + (int)q1);
}


// Bytes of dynamic shared memory the running kernel was launched with.  A
// kernel that keeps the pattern table there checks it first: a launch
// without it would read and write past the block's shared memory.
__device__ inline unsigned dynamic_smem_bytes() {
  unsigned v;
  asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(v));
  return v;
}

// Block `rec` of the pattern table into bv[9].
template <typename A>
__device__ __forceinline__ void pt_block(const float *PT, int rec, A *bv) {
  const float4 v0 = reinterpret_cast<const float4 *>(PT)[2 * rec];
  const float4 v1 = reinterpret_cast<const float4 *>(PT)[2 * rec + 1];
  bv[0] = (A)v0.x; bv[1] = (A)v0.y; bv[2] = (A)v0.z; bv[3] = (A)v0.w;
  bv[4] = (A)v1.x; bv[5] = (A)v1.y; bv[6] = (A)v1.z; bv[7] = (A)v1.w;
  bv[8] = (A)PT[8 * SP_PT_NREC + rec];
}

__device__ inline void stencil_ptable(int t, int nt, const double *Ke /*[2][576]*/, float *PT) {
  for (int x = t; x < SP_PT_NREC * 9; x += nt) {
    const int rec = x < 8 * SP_PT_NREC ? x / 8 : x - 8 * SP_PT_NREC;
    const int w = x < 8 * SP_PT_NREC ? x % 8 : 8;
    int m = 0;
    while (m < 26 && sp_pt_off(m + 1) <= rec) m++;
    const int p = rec - sp_pt_off(m);
    const int dx = m % 3 - 1, dy = (m / 3) % 3 - 1, dz = m / 9 - 1;
    const int d = w / 3, cc = w % 3;
    double v = 0.0;
    int i = 0;
    for (int c = 0; c < 8; c++) {
      const int ox = c & 1, oy = (c >> 1) & 1, oz = c >> 2;
      const int bx = 1 - ox + dx, by = 1 - oy + dy, bz = 1 - oz + dz;
      if (bx < 0 || bx > 1 || by < 0 || by > 1 || bz < 0 || bz > 1) continue;
      const int la = hex8_local(1 - ox, 1 - oy, 1 - oz), lb = hex8_local(bx, by, bz);
      v += Ke[((p >> i) & 1) * SP_KE + (3 * la + d) * SP_NC + 3 * lb + cc];
      i++;
    }
    PT[x] = (float)v;
  }
}

// Jacobi diagonal inverse of the stencil operator, component-major: for an
// interior node 1 / sum over its 8 elements of Ke[type][3la+d][3la+d]
// (summed in FP64, rounded once); 0 on boundary and padding nodes.
template <typename T>
__device__ inline void stencil_dinv(int t, int nt, const MeshGeo &g,
                                    const uint8_t *__restrict__ etype, const double *Ke, T *dinv) {
  for (int x = t; x < 3 * g.nn_pad; x += nt) {
    int d = x / g.nn_pad, node = x % g.nn_pad;
    T v = T(0);
    if (node < g.nn && !is_bnode(g, node)) {
      int i = node % g.nx, j = (node / g.nx) % g.ny, k = node / (g.nx * g.ny);
      double s = 0.0;
      for (int c = 0; c < 8; c++) {
        int ox = c & 1, oy = (c >> 1) & 1, oz = c >> 2;
        int e = (i - 1 + ox) + (j - 1 + oy) * g.nex + (k - 1 + oz) * g.nex * g.ney;
        int la = hex8_local(1 - ox, 1 - oy, 1 - oz);
        s += Ke[etype[e] * SP_KE + (3 * la + d) * SP_NC + 3 * la + d];
      }
      v = (T)(1.0 / s);
    }
    dinv[x] = v;
  }
}

// 3x3 block load from shared memory (16-byte loads) into bv.  A block read
// on its own goes through load_block, not add_block into zeros: 0 + w is not
// w for w = -0, so the compiler keeps those 9 additions (a sixth of the FP32
// pipe's work in the stencil SpMM).
template <typename T, typename A>
__device__ __forceinline__ void load_block(const T *src, A *bv) {
  constexpr int BW = SP_KB_BLK * (int)sizeof(T) / 16;
  T w[SP_KB_BLK];
#pragma unroll
  for (int q = 0; q < BW; q++) {
    int4 v = reinterpret_cast<const int4 *>(src)[q];
    memcpy(reinterpret_cast<char *>(w) + 16 * q, &v, 16);
  }
#pragma unroll
  for (int u = 0; u < 9; u++) bv[u] = (A)w[u];
}

// the same, accumulated into bv (sums of element blocks)
template <typename T, typename A>
__device__ inline void add_block(const T *src, A *bv) {
  constexpr int BW = SP_KB_BLK * (int)sizeof(T) / 16;
  T w[SP_KB_BLK];
#pragma unroll
  for (int q = 0; q < BW; q++) {
    int4 v = reinterpret_cast<const int4 *>(src)[q];
    memcpy(reinterpret_cast<char *>(w) + 16 * q, &v, 16);
  }
#pragma unroll
  for (int u = 0; u < 9; u++) bv[u] += (A)w[u];
}

// Node-blocked layout of the stencil SpMM's input vector: the 3K streams
// (component d, load case k) of 32 consecutive nodes lie next to each other,
//   v[((node / 32) * 3K + d*K + k) * 32 + node % 32],
// so the 3K values a lane gathers for one neighbour sit at compile-time
// offsets from one address (one address computation per neighbour instead
// of one per value).  A 16-byte chunk of 4 (FP32) or 2 (FP64) nodes of one
// stream is contiguous in both this and the component-major layout.
template <int K>
__device__ __forceinline__ size_t nbk_base(int node) {
  return (size_t)(node >> 5) * (96 * K) + (node & 31);
}

// Accumulators of the stencil SpMM: FP32 pairs of load cases updated with
// the packed FP32x2 FMA, or FP64 scalars.
template <typename T, int K>
struct StencilAcc;

template <int K>
struct StencilAcc<float, K> {
  static constexpr int KP = (K + 1) / 2;
  float2 v[3][KP];
  __device__ void zero() {
#pragma unroll
    for (int d = 0; d < 3; d++)
#pragma unroll
      for (int p = 0; p < KP; p++) v[d][p] = make_float2(0.f, 0.f);
  }
  // v[d][q] += bv(d, c) x(q, c), x(q, c) = xb[(c*K + q) * 32] (node-blocked),
  // for the pairs of load cases with an active case (bit q of amask;
  // warp-uniform)
  __device__ void fma_block(const float *bv, const float *xb, unsigned amask) {
#pragma unroll
    for (int p = 0; p < KP; p++) {
      if (!((amask >> (2 * p)) & 3u)) continue;
      float2 xv[3];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        xv[c].x = xb[(c * K + 2 * p) * 32];
        xv[c].y = (2 * p + 1 < K) ? xb[(c * K + 2 * p + 1) * 32] : 0.f;
      }
#pragma unroll
      for (int d = 0; d < 3; d++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const float b = bv[d * 3 + c];
          v[d][p] = __ffma2_rn(make_float2(b, b), xv[c], v[d][p]);
        }
    }
  }
  __device__ float get(int d, int q) const { return (q & 1) ? v[d][q >> 1].y : v[d][q >> 1].x; }
};

template <int K>
struct StencilAcc<double, K> {
  double v[3][K];
  __device__ void zero() {
#pragma unroll
    for (int d = 0; d < 3; d++)
#pragma unroll
      for (int q = 0; q < K; q++) v[d][q] = 0.0;
  }
  __device__ void fma_block(const double *bv, const double *xb, unsigned amask) {
#pragma unroll
    for (int q = 0; q < K; q++) {
      if (!((amask >> q) & 1u)) continue;
      double xv[3];
#pragma unroll
      for (int c = 0; c < 3; c++) xv[c] = xb[(c * K + q) * 32];
#pragma unroll
      for (int d = 0; d < 3; d++)
#pragma unroll
        for (int c = 0; c < 3; c++) v[d][q] = fma(bv[d * 3 + c], xv[c], v[d][q]);
    }
  }
  __device__ double get(int d, int q) const { return v[d][q]; }
};

// y = A x (K right-hand sides; x node-blocked (nbk_base), y component-major)
// with the stencil operator.
// Dirichlet (PER = false): interior nodes only; boundary and padding entries
// of y are not written.  Periodic (PER): every node of the periodic grid,
// neighbours and elements wrapped, y = 0 at the fixed node 0.  A warp takes
// 32 consecutive nodes (x fastest), a lane one node.  A warp whose nodes all
// lie inside one material reads that material's assembled blocks (one
// shared-memory broadcast per load); other warps sum each neighbour block
// from the element blocks of their own materials.  Adds x.y per load case
// into dot[K].  Load cases whose bit in amask is clear (converged; uniform
// across the block) are neither read nor written.  rev: the warps walk the
// node groups from the last to the first.  PT: KB is the FP32 pattern table
// (stencil_ptable) and every lane reads each of its 27 blocks from it by the
// material pattern of the (wrapped) elements it shares with the neighbour.
template <typename T, int K, bool PER = false, bool PT = false>
__device__ inline void spmm_stencil(int t, int nt, const MeshGeo &g, const T *KB,
                                    const uint8_t *__restrict__ etype, const T *x, T *y,
                                    double *dot, unsigned amask = ~0u, bool rev = false) {
  using A = typename std::conditional<sizeof(T) == 4, float, double>::type;
  const int lane = t & 31, warp = t >> 5, nwarps = nt >> 5;
  const int mx = PER ? g.nex : g.nx - 2, my = PER ? g.ney : g.ny - 2, mz = PER ? g.nez : g.nz - 2;
  const int ni = mx * my * mz;
  // node strides of the vectors and of the element grid
  const int sy = PER ? g.nex : g.nx, sz = PER ? g.nex * g.ney : g.nx * g.ny;
  const int esy = g.nex, esz = g.nex * g.ney;
  const size_t blk = (size_t)3 * g.nn_pad;
  const int ngr = (ni + 31) / 32;
  for (int gi = warp; gi < ngr; gi += nwarps) {
    const int s0 = (rev ? ngr - 1 - gi : gi) * 32;
    const int id = s0 + lane;
    const bool valid = id < ni;
    const int idc = valid ? id : ni - 1;
    const int ii = idc % mx, jj = (idc / mx) % my, kk = idc / (mx * my);
    const int i = PER ? ii : ii + 1, j = PER ? jj : jj + 1, k = PER ? kk : kk + 1;
    const int a = i + j * sy + k * sz;
    // periodic: offsets of the wrapped neighbours at -1 / +1 along each
    // axis (index 0 / 1) and of the wrapped elements below the node
    int xo[2], yo[2], zo[2], ex0 = i - 1, ey0 = j - 1, ez0 = k - 1;
    if constexpr (PER) {
      xo[0] = (i == 0) ? mx - 1 : -1;
      xo[1] = (i == mx - 1) ? 1 - mx : 1;
      yo[0] = ((j == 0) ? my - 1 : -1) * sy;
      yo[1] = ((j == my - 1) ? 1 - my : 1) * sy;
      zo[0] = ((k == 0) ? mz - 1 : -1) * sz;
      zo[1] = ((k == mz - 1) ? 1 - mz : 1) * sz;
      ex0 += (i == 0) ? g.nex : 0;
      ey0 += (j == 0) ? g.ney : 0;
      ez0 += (k == 0) ? g.nez : 0;
    }
    // neighbour (dx, dy, dz) of node a
    auto nbr_of = [&](int dx, int dy, int dz) {
      if constexpr (PER)
        return a + (dx ? xo[dx > 0] : 0) + (dy ? yo[dy > 0] : 0) + (dz ? zo[dz > 0] : 0);
      else
        return a + dx + dy * sy + dz * sz;
    };
    int tb[8];  // offset of the element's material blocks in KB
    unsigned mask = 0;
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int ox = c & 1, oy = (c >> 1) & 1, oz = c >> 2;
      const int e = (ox ? i : ex0) + (oy ? j : ey0) * esy + (oz ? k : ez0) * esz;
      const unsigned te = __ldg(etype + e);
      mask |= te << c;
      tb[c] = SP_KE_OFF + (int)te * SP_KB_TYPE;
    }
    StencilAcc<T, K> acc;
    acc.zero();
    const bool all0 = __all_sync(0xffffffffu, mask == 0u);
    const bool all1 = __all_sync(0xffffffffu, mask == 0xffu);
    if constexpr (PT) {
#pragma unroll 1
      for (int dz = -1; dz <= 1; dz++) {
#pragma unroll
        for (int mm = 0; mm < 9; mm++) {
          const int dx = mm % 3 - 1, dy = mm / 3 - 1;
          A bv[9];
          pt_block<A>(KB, sp_pt_index(mask, dx, dy, dz), bv);
          acc.fma_block(bv, x + nbk_base<K>(nbr_of(dx, dy, dz)), amask);
        }
      }
    } else if (all0 || all1) {
      // one material around every node of the warp: its assembled blocks
      const T *ka = KB + SP_KA_OFF + (all1 ? 27 * SP_KB_BLK : 0);
#pragma unroll 1
      for (int dz = -1; dz <= 1; dz++) {
#pragma unroll
        for (int mm = 0; mm < 9; mm++) {
          const int dx = mm % 3 - 1, dy = mm / 3 - 1;
          A bv[9];
          load_block<T, A>(ka + ((dz + 1) * 9 + mm) * SP_KB_BLK, bv);
          acc.fma_block(bv, x + nbk_base<K>(nbr_of(dx, dy, dz)), amask);
        }
      }
    } else {
      // neighbour planes dz = -1, 0, 1 in turn (a rolled loop bounds the
      // live registers); within a plane the 9 neighbours and their elements
      // unroll
#pragma unroll 1
      for (int dz = -1; dz <= 1; dz++) {
#pragma unroll
        for (int mm = 0; mm < 9; mm++) {
          const int dx = mm % 3 - 1, dy = mm / 3 - 1;
          A bv[9] = {};
#pragma unroll
          for (int c = 0; c < 8; c++) {
            const int ox = c & 1, oy = (c >> 1) & 1, oz = c >> 2;
            const int bx = 1 - ox + dx, by = 1 - oy + dy;
            if (bx < 0 || bx > 1 || by < 0 || by > 1) continue;  // resolved at compile time
            const int bz = 1 - oz + dz;                            // warp-uniform
            if (bz < 0 || bz > 1) continue;
            const int la = hex8_local(1 - ox, 1 - oy, 1 - oz);
            const int lb = hex8_local(bx, by, 0) + 4 * bz;
            add_block<T, A>(KB + tb[c] + (la * 8 + lb) * SP_KB_BLK, bv);
          }
          acc.fma_block(bv, x + nbk_base<K>(nbr_of(dx, dy, dz)), amask);
        }
      }
    }
    if (valid) {
#pragma unroll
      for (int q = 0; q < K; q++) {
        if (!((amask >> q) & 1u)) continue;
#pragma unroll
        for (int d = 0; d < 3; d++) {
          T yv = (PER && a == 0) ? T(0) : (T)acc.get(d, q);
          dot[q] += (double)yv * (double)x[nbk_base<K>(a) + (d * K + q) * 32];
          y[q * blk + (size_t)d * g.nn_pad + a] = yv;
        }
      }
    }
  }
}

// FP32 stencil SpMM under Dirichlet conditions with the x-neighbours taken
// from the warp.  A warp holds 32 consecutive interior nodes: lanes 1..30
// produce output, lanes 0 and 31 only supply values.  For each of the 9
// (dy, dz) neighbour rows a lane loads the 3K values of its own column
// (dx = 0, one gather); the dx = -1 / +1 values come from the adjacent
// lanes (shuffles), or are 0 where that neighbour is a boundary node (the
// CG vectors vanish on the Dirichlet boundary) -- exactly the case in which
// the adjacent lane holds a node of another row.  9 instead of 27 gathers
// per value; the materials and output are those of spmm_stencil.  KB is
// the pattern table (stencil_ptable): every lane reads its 27 blocks from
// it by the material pattern of the elements it shares with each neighbour.
// Used for K > 6 load cases, where the three accumulator sets of
// spmm_stencil_xo do not fit in the registers.
template <int K>
__device__ inline void spmm_stencil_xw(int t, int nt, const MeshGeo &g, const float *KB,
                                       const uint8_t *__restrict__ etype,
                                       const float *__restrict__ x, float *__restrict__ y,
                                       double *dot, unsigned amask, bool rev) {
  constexpr int KP = (K + 1) / 2;
  constexpr unsigned FULL = 0xffffffffu;
  const int lane = t & 31, warp = t >> 5, nwarps = nt >> 5;
  const int mx = g.nx - 2, my = g.ny - 2, mz = g.nz - 2;
  const int ni = mx * my * mz;
  const int sy = g.nx, sz = g.nx * g.ny;
  const int esy = g.nex, esz = g.nex * g.ney;
  const size_t blk = (size_t)3 * g.nn_pad;
  const int ngr = (ni + 29) / 30;
  for (int gi = warp; gi < ngr; gi += nwarps) {
    const int s0 = (rev ? ngr - 1 - gi : gi) * 30;
    const int id = s0 - 1 + lane;
    const bool out = lane >= 1 && lane <= 30 && id < ni;
    const int idc = min(max(id, 0), ni - 1);
    const int ii = idc % mx, jj = (idc / mx) % my, kk = idc / (mx * my);
    const int i = ii + 1, j = jj + 1, k = kk + 1;
    const int a = i + j * sy + k * sz;
    // the adjacent lanes hold the x-neighbours unless those are boundary nodes
    const bool lo = ii > 0, hi = ii < mx - 1;
    unsigned mask = 0;  // bit c: material of the element at corner c
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int ox = c & 1, oy = (c >> 1) & 1, oz = c >> 2;
      const int e = (i - 1 + ox) + (j - 1 + oy) * esy + (k - 1 + oz) * esz;
      mask |= (unsigned)__ldg(etype + e) << c;
    }
    float2 acc[3][KP];
#pragma unroll
    for (int d = 0; d < 3; d++)
#pragma unroll
      for (int p = 0; p < KP; p++) acc[d][p] = make_float2(0.f, 0.f);
    // the 9 (dy, dz) rows in turn, the next row's gathers issued before the
    // current row's products (two row buffers in registers)
    float2 xr[2][3][KP];
    auto gather = [&](int r, float2 (&xv)[3][KP]) {
      const int dy = r % 3 - 1, dz = r / 3 - 1;
      const float *xb = x + nbk_base<K>(a + dy * sy + dz * sz);
#pragma unroll
      for (int p = 0; p < KP; p++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
          xv[c][p] = make_float2(0.f, 0.f);
          if ((amask >> (2 * p)) & 3u) {
            xv[c][p].x = xb[(c * K + 2 * p) * 32];
            if (2 * p + 1 < K) xv[c][p].y = xb[(c * K + 2 * p + 1) * 32];
          }
        }
    };
    gather(0, xr[0]);
#pragma unroll
    for (int r = 0; r < 9; r++) {
      const int dy = r % 3 - 1, dz = r / 3 - 1;
      if (r + 1 < 9) gather(r + 1, xr[(r + 1) & 1]);
      const float2 (&xv)[3][KP] = xr[r & 1];
#pragma unroll
      for (int dx = -1; dx <= 1; dx++) {
        float bv[9];
        pt_block<float>(KB, sp_pt_index(mask, dx, dy, dz), bv);
#pragma unroll
        for (int p = 0; p < KP; p++) {
          if (!((amask >> (2 * p)) & 3u)) continue;
          float2 xs[3];
#pragma unroll
          for (int c = 0; c < 3; c++) {
            if (dx == 0) {
              xs[c] = xv[c][p];
            } else {
              float2 v;
              if (dx < 0) {
                v.x = __shfl_up_sync(FULL, xv[c][p].x, 1);
                v.y = __shfl_up_sync(FULL, xv[c][p].y, 1);
              } else {
                v.x = __shfl_down_sync(FULL, xv[c][p].x, 1);
                v.y = __shfl_down_sync(FULL, xv[c][p].y, 1);
              }
              xs[c] = (dx < 0 ? lo : hi) ? v : make_float2(0.f, 0.f);
            }
          }
#pragma unroll
          for (int d = 0; d < 3; d++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
              const float b = bv[d * 3 + c];
              acc[d][p] = __ffma2_rn(make_float2(b, b), xs[c], acc[d][p]);
            }
        }
      }
    }
    if (out) {
#pragma unroll
      for (int q = 0; q < K; q++) {
        if (!((amask >> q) & 1u)) continue;
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const float yv = (q & 1) ? acc[d][q >> 1].y : acc[d][q >> 1].x;
          dot[q] += (double)yv * (double)x[nbk_base<K>(a) + (d * K + q) * 32];
          y[q * blk + (size_t)d * g.nn_pad + a] = yv;
        }
      }
    }
  }
}

// FP32 stencil SpMM under Dirichlet conditions, the x-neighbour terms formed
// where the x values already are.  A warp holds 32 consecutive interior
// nodes: lanes 1..30 produce output, lanes 0 and 31 only contribute.  For
// each of the 9 (dy, dz) neighbour rows a lane gathers the 3K values of its
// own column (one gather per value instead of three) and multiplies them by
// three blocks: its own (dx = 0), the one its right neighbour b+1 would apply
// to them (b+1's dx = -1 block), and the one its left neighbour b-1 would
// apply (b-1's dx = +1 block).  Those two blocks depend on the materials of
// the elements the neighbour shares with the row, which are elements around
// this node too: b+1's ox = 0 elements are this node's ox = 1 elements, and
// b-1's ox = 1 elements its ox = 0 ones, so their pattern-table records are
// found from this lane's own mask.  The two partial sums cross lanes once per
// warp trip (36 shuffles instead of 324 for the inputs), and are added only
// where the neighbour is an interior node of the same row (the CG vectors
// vanish on the Dirichlet boundary).  Same blocks and products as
// spmm_stencil; the sums differ in order only.  The L1 data pipe, which
// serves the shuffles, the pattern-table loads and the gathers' L1 hits,
// bounds this operator; the shuffles were a third of its wavefronts, and
// the operator alone runs 22% faster in this form (n = 12..20).  The
// per-thread x.y partial sums stay in FP32 until the end of the call (fewer
// registers across the loop).  KB is the pattern table (stencil_ptable).
// The gathers stay under the active-pair condition: in this kernel that
// form compiles to the faster code (in a stand-alone harness it was the
// reverse), so changes here are judged by the batched kernel's time.
template <int K>
__device__ inline void spmm_stencil_xo(int t, int nt, const MeshGeo &g, const float *KB,
                                       const uint8_t *__restrict__ etype,
                                       const float *__restrict__ x, float *__restrict__ y,
                                       double *dot, unsigned amask, bool rev) {
  constexpr int KP = (K + 1) / 2;
  constexpr unsigned FULL = 0xffffffffu;
  const int lane = t & 31, warp = t >> 5, nwarps = nt >> 5;
  const int mx = g.nx - 2, my = g.ny - 2, mz = g.nz - 2;
  const int ni = mx * my * mz;
  const int sy = g.nx, sz = g.nx * g.ny;
  const int esy = g.nex, esz = g.nex * g.ney;
  const size_t blk = (size_t)3 * g.nn_pad;
  const int ngr = (ni + 29) / 30;
  // per-thread partial sums of x.y in FP32 (a few dozen terms), added to
  // the caller's FP64 sums once: six fewer registers across the loop
  float dotf[K];
#pragma unroll
  for (int q = 0; q < K; q++) dotf[q] = 0.f;
  for (int gi = warp; gi < ngr; gi += nwarps) {
    const int s0 = (rev ? ngr - 1 - gi : gi) * 30;
    const int id = s0 - 1 + lane;
    const bool out = lane >= 1 && lane <= 30 && id < ni;
    const int idc = min(max(id, 0), ni - 1);
    const int ii = idc % mx, jj = (idc / mx) % my, kk = idc / (mx * my);
    const int i = ii + 1, j = jj + 1, k = kk + 1;
    const int a = i + j * sy + k * sz;
    // the adjacent lanes hold the x-neighbours unless those are boundary nodes
    const bool lo = ii > 0, hi = ii < mx - 1;
    unsigned mask = 0;  // bit c: material of the element at corner c
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int ox = c & 1, oy = (c >> 1) & 1, oz = c >> 2;
      const int e = (i - 1 + ox) + (j - 1 + oy) * esy + (k - 1 + oz) * esz;
      mask |= (unsigned)__ldg(etype + e) << c;
    }
    // the masks b+1 and b-1 would use, as far as their dx = -1 / +1 blocks
    // read them (sp_pt_index reads only the ox = 0 / ox = 1 bits there)
    const unsigned mR = (mask >> 1) & 0x55u, mL = (mask << 1) & 0xAAu;
    float2 acc[3][3][KP];  // [own, for b+1, for b-1][d][load-case pair]
#pragma unroll
    for (int s = 0; s < 3; s++)
#pragma unroll
      for (int d = 0; d < 3; d++)
#pragma unroll
        for (int p = 0; p < KP; p++) acc[s][d][p] = make_float2(0.f, 0.f);
#pragma unroll
    for (int r = 0; r < 9; r++) {
      const int dy = r % 3 - 1, dz = r / 3 - 1;
      const float *xb = x + nbk_base<K>(a + dy * sy + dz * sz);
      float2 xv[3][KP];
#pragma unroll
      for (int p = 0; p < KP; p++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
          xv[c][p] = make_float2(0.f, 0.f);
          if ((amask >> (2 * p)) & 3u) {
            xv[c][p].x = xb[(c * K + 2 * p) * 32];
            if (2 * p + 1 < K) xv[c][p].y = xb[(c * K + 2 * p + 1) * 32];
          }
        }
#pragma unroll
      for (int s = 0; s < 3; s++) {
        const int rec = s == 0 ? sp_pt_index(mask, 0, dy, dz)
                               : (s == 1 ? sp_pt_index(mR, -1, dy, dz) : sp_pt_index(mL, 1, dy, dz));
        float bv[9];
        pt_block<float>(KB, rec, bv);
#pragma unroll
        for (int p = 0; p < KP; p++) {
          if (!((amask >> (2 * p)) & 3u)) continue;
#pragma unroll
          for (int d = 0; d < 3; d++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
              const float b = bv[d * 3 + c];
              acc[s][d][p] = __ffma2_rn(make_float2(b, b), xv[c][p], acc[s][d][p]);
            }
        }
      }
    }
#pragma unroll
    for (int p = 0; p < KP; p++) {
      if (!((amask >> (2 * p)) & 3u)) continue;
#pragma unroll
      for (int d = 0; d < 3; d++) {
        float2 v;
        v.x = __shfl_up_sync(FULL, acc[1][d][p].x, 1);
        v.y = __shfl_up_sync(FULL, acc[1][d][p].y, 1);
        if (lo) acc[0][d][p] = make_float2(acc[0][d][p].x + v.x, acc[0][d][p].y + v.y);
        v.x = __shfl_down_sync(FULL, acc[2][d][p].x, 1);
        v.y = __shfl_down_sync(FULL, acc[2][d][p].y, 1);
        if (hi) acc[0][d][p] = make_float2(acc[0][d][p].x + v.x, acc[0][d][p].y + v.y);
      }
    }
    if (out) {
#pragma unroll
      for (int q = 0; q < K; q++) {
        if (!((amask >> q) & 1u)) continue;
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const float yv = (q & 1) ? acc[0][d][q >> 1].y : acc[0][d][q >> 1].x;
          dotf[q] = fmaf(yv, x[nbk_base<K>(a) + (d * K + q) * 32], dotf[q]);
          y[q * blk + (size_t)d * g.nn_pad + a] = yv;
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < K; q++) dot[q] += (double)dotf[q];
}

// b = -K u on interior dofs in stencil form (Dirichlet conditions): one
// thread per interior dof row, the row of each of the node's 27 assembled
// 3x3 blocks (FP64, summed from the element blocks of its 8 elements,
// stencil_blocks<double>) times the neighbour's u, boundary neighbours
// included; 0 on boundary and padding dofs.  The same sums as residual_soa in
// another order, with 27 instead of 64 neighbour reads per row.  SCALE: adds
// the squared norm of the rows' sums of term magnitudes into scale2[K].
// BCONLY: u's interior values are read as 0, giving the right-hand side
// -K u_bc of the load cases whatever u holds inside.
template <int K, typename R, bool SCALE = false, bool BCONLY = false>
__device__ inline void residual_stencil(int t, int nt, const MeshGeo &g,
                                        const uint8_t *__restrict__ etype,
                                        const double *KBd /*stencil tables, shared*/,
                                        const double *__restrict__ u, R *rb, double *nrm2,
                                        double *scale2 = nullptr) {
  const size_t blk = (size_t)3 * g.nn_pad;
  for (int idx = t; idx < 3 * g.nn_pad; idx += nt) {
    const int node = idx % g.nn_pad;
    if (node >= g.nn || is_bnode(g, node))
#pragma unroll
      for (int q = 0; q < K; q++) rb[q * blk + idx] = (R)0;
  }
  const int mx = g.nx - 2, my = g.ny - 2, mz = g.nz - 2;
  const int ni = mx * my * mz;
  const int sy = g.nx, sz = g.nx * g.ny, esy = g.nex, esz = g.nex * g.ney;
  for (int r0 = t - (t & 31); r0 < 3 * ni; r0 += nt) {  // whole warps per trip
    const int rid = r0 + (t & 31);
    const bool valid = rid < 3 * ni;
    const int rc = valid ? rid : 3 * ni - 1;
    const int d = rc / ni, idc = rc - d * ni;
    const int i = 1 + idc % mx, j = 1 + (idc / mx) % my, k = 1 + idc / (mx * my);
    const int a = i + j * sy + k * sz;
    const int e0 = (i - 1) + (j - 1) * esy + (k - 1) * esz;
    int tb[8];
    unsigned mask = 0;
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const unsigned te = __ldg(etype + e0 + (c & 1) + ((c >> 1) & 1) * esy + (c >> 2) * esz);
      mask |= te << c;
      tb[c] = SP_KE_OFF + (int)te * SP_KB_TYPE;
    }
    const bool all0 = __all_sync(0xffffffffu, mask == 0u);
    const bool all1 = __all_sync(0xffffffffu, mask == 0xffu);
    double acc[K], mag[K];
#pragma unroll
    for (int q = 0; q < K; q++) acc[q] = mag[q] = 0.0;
#pragma unroll 1
    for (int dz = -1; dz <= 1; dz++) {
#pragma unroll
      for (int mm = 0; mm < 9; mm++) {
        const int dx = mm % 3 - 1, dy = mm / 3 - 1;
        double bv[3] = {0.0, 0.0, 0.0};
        if (all0 || all1) {
          const double *src = KBd + SP_KA_OFF + (all1 ? 27 * SP_KB_BLK : 0) +
                              ((dz + 1) * 9 + mm) * SP_KB_BLK + 3 * d;
#pragma unroll
          for (int c = 0; c < 3; c++) bv[c] = src[c];
        } else {
#pragma unroll
          for (int c8 = 0; c8 < 8; c8++) {
            const int ox = c8 & 1, oy = (c8 >> 1) & 1, oz = c8 >> 2;
            const int bx = 1 - ox + dx, by = 1 - oy + dy;
            if (bx < 0 || bx > 1 || by < 0 || by > 1) continue;
            const int bz = 1 - oz + dz;
            if (bz < 0 || bz > 1) continue;
            const int la = hex8_local(1 - ox, 1 - oy, 1 - oz);
            const int lb = hex8_local(bx, by, 0) + 4 * bz;
            const double *src = KBd + tb[c8] + (la * 8 + lb) * SP_KB_BLK + 3 * d;
#pragma unroll
            for (int c = 0; c < 3; c++) bv[c] += src[c];
          }
        }
        const int nb = a + dx + dy * sy + dz * sz;
        // (BCONLY) whether the neighbour is a boundary node
        const bool nbb = !BCONLY || i + dx == 0 || i + dx == g.nx - 1 || j + dy == 0 ||
                         j + dy == g.ny - 1 || k + dz == 0 || k + dz == g.nz - 1;
#pragma unroll
        for (int q = 0; q < K; q++)
#pragma unroll
          for (int c = 0; c < 3; c++) {
            const double uv = nbb ? u[q * blk + (size_t)c * g.nn_pad + nb] : 0.0;
            acc[q] = fma(bv[c], uv, acc[q]);
            if (SCALE) mag[q] += fabs(bv[c] * uv);
          }
      }
    }
    if (valid) {
#pragma unroll
      for (int q = 0; q < K; q++) {
        const double b = -acc[q];
        rb[q * blk + (size_t)d * g.nn_pad + a] = (R)b;
        nrm2[q] += b * b;
        if (SCALE) scale2[q] += mag[q] * mag[q];
      }
    }
  }
}

// residual_stencil with one thread per interior node instead of one per
// dof row: each u value is read once per node, not once per row (27 x 3K
// instead of 3 x 27 x 3K reads per node), for 2K x 3 FP64 accumulators a
// thread (kernels with 128 registers a thread).  Every row sum is formed in
// the same order as in residual_stencil, so the results are identical.
template <int K, typename R>
__device__ inline void residual_stencil_node(int t, int nt, const MeshGeo &g,
                                             const uint8_t *__restrict__ etype,
                                             const double *KBd /*stencil tables, shared*/,
                                             const double *__restrict__ u, R *rb, double *nrm2) {
  const size_t blk = (size_t)3 * g.nn_pad;
  for (int idx = t; idx < 3 * g.nn_pad; idx += nt) {
    const int node = idx % g.nn_pad;
    if (node >= g.nn || is_bnode(g, node))
#pragma unroll
      for (int q = 0; q < K; q++) rb[q * blk + idx] = (R)0;
  }
  const int mx = g.nx - 2, my = g.ny - 2, mz = g.nz - 2;
  const int ni = mx * my * mz;
  const int sy = g.nx, sz = g.nx * g.ny, esy = g.nex, esz = g.nex * g.ney;
  for (int n0 = t - (t & 31); n0 < ni; n0 += nt) {  // whole warps per trip
    const int nid = n0 + (t & 31);
    const bool valid = nid < ni;
    const int idc = valid ? nid : ni - 1;
    const int i = 1 + idc % mx, j = 1 + (idc / mx) % my, k = 1 + idc / (mx * my);
    const int a = i + j * sy + k * sz;
    const int e0 = (i - 1) + (j - 1) * esy + (k - 1) * esz;
    int tb[8];
    unsigned mask = 0;
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const unsigned te = __ldg(etype + e0 + (c & 1) + ((c >> 1) & 1) * esy + (c >> 2) * esz);
      mask |= te << c;
      tb[c] = SP_KE_OFF + (int)te * SP_KB_TYPE;
    }
    const bool all0 = __all_sync(0xffffffffu, mask == 0u);
    const bool all1 = __all_sync(0xffffffffu, mask == 0xffu);
    double acc[K][3];
#pragma unroll
    for (int q = 0; q < K; q++)
#pragma unroll
      for (int d = 0; d < 3; d++) acc[q][d] = 0.0;
#pragma unroll 1
    for (int dz = -1; dz <= 1; dz++) {
#pragma unroll
      for (int mm = 0; mm < 9; mm++) {
        const int dx = mm % 3 - 1, dy = mm / 3 - 1;
        double bv[9];
        if (all0 || all1) {
          const double *src = KBd + SP_KA_OFF + (all1 ? 27 * SP_KB_BLK : 0) +
                              ((dz + 1) * 9 + mm) * SP_KB_BLK;
#pragma unroll
          for (int w = 0; w < 9; w++) bv[w] = src[w];
        } else {
#pragma unroll
          for (int w = 0; w < 9; w++) bv[w] = 0.0;
#pragma unroll
          for (int c8 = 0; c8 < 8; c8++) {
            const int ox = c8 & 1, oy = (c8 >> 1) & 1, oz = c8 >> 2;
            const int bx = 1 - ox + dx, by = 1 - oy + dy;
            if (bx < 0 || bx > 1 || by < 0 || by > 1) continue;
            const int bz = 1 - oz + dz;
            if (bz < 0 || bz > 1) continue;
            const int la = hex8_local(1 - ox, 1 - oy, 1 - oz);
            const int lb = hex8_local(bx, by, 0) + 4 * bz;
            const double *src = KBd + tb[c8] + (la * 8 + lb) * SP_KB_BLK;
#pragma unroll
            for (int w = 0; w < 9; w++) bv[w] += src[w];
          }
        }
        const int nb = a + dx + dy * sy + dz * sz;
#pragma unroll
        for (int q = 0; q < K; q++)
#pragma unroll
          for (int c = 0; c < 3; c++) {
            const double uv = u[q * blk + (size_t)c * g.nn_pad + nb];
#pragma unroll
            for (int d = 0; d < 3; d++) acc[q][d] = fma(bv[d * 3 + c], uv, acc[q][d]);
          }
      }
    }
    if (valid) {
#pragma unroll
      for (int q = 0; q < K; q++)
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const double b = -acc[q][d];
          rb[q * blk + (size_t)d * g.nn_pad + a] = (R)b;
          nrm2[q] += b * b;
        }
    }
  }
}

// ------------------------------------------------------ periodic BCs ---
//
// Periodic boundary conditions by master-slave elimination: u = eps.x + w
// with the fluctuation w periodic, so the nodes at x = Lx (y = Ly, z = Lz)
// are the images of those at 0 and the unknowns live on the periodic grid of
// nex x ney x nez nodes, node i + nex (j + ney k).  All 8 corners are one
// periodic node, node 0, whose w is fixed to 0: the corners carry eps.x, as
// in the reference's 2D Lagrange-multiplier variant (micro/src/assembly.c:
// 175-220, corners prescribed and opposite faces tied by u+ - u- = eps.dl),
// and the rigid translations are removed.  The operator on w is P^T K P (the
// stencil with wrapped neighbours and elements), the right-hand side
// -P^T K (eps.x); u is never formed: residual and averages add eps.x per
// element from the element's own (unwrapped) node coordinates.

// component d of eps.x (engineering shears halved; micro/src/homogenize.c:
// 335-342 in 3D)
__device__ inline double affine_comp(const double *e, int d, double X, double Y, double Z) {
  if (d == 0) return dadd(dadd(dmul(e[0], X), dmul(e[3] / 2, Y)), dmul(e[5] / 2, Z));
  if (d == 1) return dadd(dadd(dmul(e[3] / 2, X), dmul(e[1], Y)), dmul(e[4] / 2, Z));
  return dadd(dadd(dmul(e[5] / 2, X), dmul(e[4] / 2, Y)), dmul(e[2], Z));
}

// b = -P^T K (eps.x + P w) on the free periodic dofs, 0 at node 0 and on
// padding; |b|^2 per load case into nrm2.  eps: [K][6] (shared).
template <int K, typename R, bool SCALE = false>
__device__ inline void residual_per(int t, int nt, const MeshGeo &g,
                                    const uint8_t *__restrict__ etype,
                                    const double *Ke /*[2][576], shared*/, const double *eps,
                                    const double *__restrict__ w, R *rb, double *nrm2,
                                    double *scale2 = nullptr) {
  const size_t blk = (size_t)3 * g.nn_pad;
  const int np = g.nelm;
  for (int idx = t; idx < 3 * g.nn_pad; idx += nt) {
    const int d = idx / g.nn_pad, node = idx % g.nn_pad;
    double acc[K], mag[K];
#pragma unroll
    for (int q = 0; q < K; q++) acc[q] = mag[q] = 0.0;
    if (node > 0 && node < np) {
      const int i = node % g.nex, j = (node / g.nex) % g.ney, k = node / (g.nex * g.ney);
#pragma unroll 1
      for (int c = 0; c < 8; c++) {
        const int ox = c & 1, oy = (c >> 1) & 1, oz = c >> 2;
        int ex = i - 1 + ox, ey = j - 1 + oy, ez = k - 1 + oz;
        ex += (ex < 0) ? g.nex : 0;
        ey += (ey < 0) ? g.ney : 0;
        ez += (ez < 0) ? g.nez : 0;
        const int e = ex + ey * g.nex + ez * g.nex * g.ney;
        const int la = hex8_local(1 - ox, 1 - oy, 1 - oz);
        const double *ke = Ke + etype[e] * SP_KE + (la * 3 + d) * SP_NC;
#pragma unroll 2
        for (int b = 0; b < 8; b++) {
          const int bx = ex + corner_x(b), by = ey + corner_y(b), bz = ez + corner_z(b);
          const int nb = (bx == g.nex ? 0 : bx) + g.nex * ((by == g.ney ? 0 : by) +
                                                           g.ney * (bz == g.nez ? 0 : bz));
          const double X = bx * g.hx, Y = by * g.hy, Z = bz * g.hz;
#pragma unroll
          for (int db = 0; db < 3; db++) {
            const double kv = ke[b * 3 + db];
#pragma unroll
            for (int q = 0; q < K; q++) {
              const double uv = affine_comp(eps + q * 6, db, X, Y, Z) +
                                w[q * blk + (size_t)db * g.nn_pad + nb];
              acc[q] = fma(kv, uv, acc[q]);
              if (SCALE) mag[q] += fabs(kv * uv);
            }
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < K; q++) {
      const double b = -acc[q];
      rb[q * blk + idx] = (R)b;
      nrm2[q] += b * b;
      if (SCALE) scale2[q] += mag[q] * mag[q];
    }
  }
}

// Jacobi diagonal inverse of the periodic stencil operator; 0 at node 0 and
// on padding.
template <typename T>
__device__ inline void stencil_dinv_per(int t, int nt, const MeshGeo &g,
                                        const uint8_t *__restrict__ etype, const double *Ke,
                                        T *dinv) {
  for (int x = t; x < 3 * g.nn_pad; x += nt) {
    const int d = x / g.nn_pad, node = x % g.nn_pad;
    T v = T(0);
    if (node > 0 && node < g.nelm) {
      const int i = node % g.nex, j = (node / g.nex) % g.ney, k = node / (g.nex * g.ney);
      double s = 0.0;
      for (int c = 0; c < 8; c++) {
        const int ox = c & 1, oy = (c >> 1) & 1, oz = c >> 2;
        int ex = i - 1 + ox, ey = j - 1 + oy, ez = k - 1 + oz;
        ex += (ex < 0) ? g.nex : 0;
        ey += (ey < 0) ? g.ney : 0;
        ez += (ez < 0) ? g.nez : 0;
        const int e = ex + ey * g.nex + ez * g.nex * g.ney;
        const int la = hex8_local(1 - ox, 1 - oy, 1 - oz);
        s += Ke[etype[e] * SP_KE + (3 * la + d) * SP_NC + 3 * la + d];
      }
      v = (T)(1.0 / s);
    }
    dinv[x] = v;
  }
}

// volume averages of load case q under periodic conditions: u_e = eps.x_e +
// w_e per element (see average_soa)
__device__ inline void average_per(int t, int nt, const MeshGeo &g,
                                   const uint8_t *__restrict__ etype, const double *D,
                                   const double *Bbar, const double *eps_q,
                                   const double *__restrict__ w, int q, double *acc) {
  const size_t blk = (size_t)3 * g.nn_pad;
  for (int e = t; e < g.nelm; e += nt) {
    const int ex = e % g.nex, ey = (e / g.nex) % g.ney, ez = e / (g.nex * g.ney);
    double eps[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll 1
    for (int a = 0; a < 8; a++) {
      const int bx = ex + corner_x(a), by = ey + corner_y(a), bz = ez + corner_z(a);
      const int nb = (bx == g.nex ? 0 : bx) + g.nex * ((by == g.ney ? 0 : by) +
                                                       g.ney * (bz == g.nez ? 0 : bz));
      const double X = bx * g.hx, Y = by * g.hy, Z = bz * g.hz;
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const double uv = affine_comp(eps_q, d, X, Y, Z) + w[q * blk + (size_t)d * g.nn_pad + nb];
#pragma unroll
        for (int v = 0; v < 6; v++) eps[v] = fma(Bbar[v * 24 + a * 3 + d], uv, eps[v]);
      }
    }
    const double *C = D + etype[e] * 36;
#pragma unroll
    for (int v = 0; v < 6; v++) {
      double s = 0.0;
#pragma unroll
      for (int x = 0; x < 6; x++) s = fma(C[v * 6 + x], eps[x], s);
      acc[v] += eps[v];
      acc[6 + v] += s;
    }
  }
}

// b = -K u on interior dofs, 0 on the boundary and on padding (component-
// major vectors; see residual_nodes for the arithmetic).  BCONLY: u's
// interior values are read as 0, giving the right-hand side -K u_bc of the
// load cases.  SCALE: also adds, per load case, the squared norm of the rows'
// sums of term magnitudes into scale2[K] (the size below which b is
// cancellation round-off).
template <int K, typename R, bool BCONLY = false, bool SCALE = false>
__device__ inline void residual_soa(int t, int nt, const MeshGeo &g,
                                    const uint8_t *__restrict__ etype,
                                    const double *Ke /*[2][576], shared*/,
                                    const double *__restrict__ u, R *rb, double *nrm2,
                                    double *scale2 = nullptr) {
  const size_t blk = (size_t)3 * g.nn_pad;
  for (int idx = t; idx < 3 * g.nn_pad; idx += nt) {
    int d = idx / g.nn_pad, node = idx % g.nn_pad;
    double acc[K], mag[K];
#pragma unroll
    for (int q = 0; q < K; q++) acc[q] = mag[q] = 0.0;
    if (node < g.nn) {
      int i = node % g.nx, j = (node / g.nx) % g.ny, k = node / (g.nx * g.ny);
      bool bnd = (i == 0 || j == 0 || k == 0 || i == g.nx - 1 || j == g.ny - 1 || k == g.nz - 1);
      if (!bnd) {
#pragma unroll 1
        for (int c = 0; c < 8; c++) {
          int ox = (c & 1), oy = (c >> 1) & 1, oz = c >> 2;
          int ex = i - 1 + ox, ey = j - 1 + oy, ez = k - 1 + oz;
          int e = ex + ey * g.nex + ez * g.nex * g.ney;
          int cx = 1 - ox, cy = 1 - oy, cz = 1 - oz;
          int la = cz * 4 + ((cy == 0) ? (cx ? 1 : 0) : (cx ? 2 : 3));
          const double *ke = Ke + etype[e] * SP_KE + (la * 3 + d) * SP_NC;
          int n0 = ex + ey * g.nx + ez * g.nx * g.ny;
#pragma unroll 2
          for (int b = 0; b < 8; b++) {
            int nb = n0 + corner_x(b) + corner_y(b) * g.nx + corner_z(b) * g.nx * g.ny;
            if (BCONLY && !is_bnode(g, nb)) continue;
#pragma unroll
            for (int db = 0; db < 3; db++) {
              double kv = ke[b * 3 + db];
#pragma unroll
              for (int q = 0; q < K; q++) {
                const double uv = u[q * blk + (size_t)db * g.nn_pad + nb];
                acc[q] = fma(kv, uv, acc[q]);
                if (SCALE) mag[q] += fabs(kv * uv);
              }
            }
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < K; q++) {
      double b = -acc[q];
      rb[q * blk + idx] = (R)b;
      nrm2[q] += b * b;
      if (SCALE) scale2[q] += mag[q] * mag[q];
    }
  }
}

// u = eps . x on boundary dofs; interior dofs are set to 0 (keep_inside =
// false) or kept (warm start), or (affine_inside) set to eps . x as well --
// the homogeneous affine field, the exact solution for a homogeneous RVE and
// a start iterate whose error in a composite lies near the material
// interfaces; load cases >= nrhs and padding are 0.
template <int K>
__device__ inline void affine_soa(int t, int nt, const MeshGeo &g, const double *eps, int nrhs,
                                  bool keep_inside, double *u, bool affine_inside = false) {
  const size_t blk = (size_t)3 * g.nn_pad;
  for (size_t x = t; x < K * blk; x += nt) {
    int k = (int)(x / blk);
    int rem = (int)(x % blk);
    int d = rem / g.nn_pad, node = rem % g.nn_pad;
    if (node >= g.nn || k >= nrhs) {
      u[x] = 0.0;
      continue;
    }
    if (!affine_inside && !is_bnode(g, node)) {
      if (!keep_inside) u[x] = 0.0;
      continue;
    }
    int i = node % g.nx, j = (node / g.nx) % g.ny, kk = node / (g.nx * g.ny);
    double X = i * g.hx, Y = j * g.hy, Z = kk * g.hz;
    const double *e = eps + k * 6;
    double val;
    if (d == 0)
      val = dadd(dadd(dmul(e[0], X), dmul(e[3] / 2, Y)), dmul(e[5] / 2, Z));
    else if (d == 1)
      val = dadd(dadd(dmul(e[3] / 2, X), dmul(e[1], Y)), dmul(e[4] / 2, Z));
    else
      val = dadd(dadd(dmul(e[5] / 2, X), dmul(e[4] / 2, Y)), dmul(e[2], Z));
    u[x] = val;
  }
}

// volume averages of load case q on component-major u (see average_elems)
__device__ inline void average_soa(int t, int nt, const MeshGeo &g,
                                   const uint8_t *__restrict__ etype, const double *D,
                                   const double *Bbar, const double *__restrict__ u, int q,
                                   double *acc) {
  const size_t blk = (size_t)3 * g.nn_pad;
  for (int e = t; e < g.nelm; e += nt) {
    int nod[8];
    elem_nodes(g, e, nod);
    double eps[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll 1
    for (int a = 0; a < 8; a++)
#pragma unroll
      for (int d = 0; d < 3; d++) {
        double uv = u[q * blk + (size_t)d * g.nn_pad + nod[a]];
#pragma unroll
        for (int v = 0; v < 6; v++) eps[v] = fma(Bbar[v * 24 + a * 3 + d], uv, eps[v]);
      }
    const double *C = D + etype[e] * 36;
#pragma unroll
    for (int v = 0; v < 6; v++) {
      double s = 0.0;
#pragma unroll
      for (int w = 0; w < 6; w++) s = fma(C[v * 6 + w], eps[w], s);
      acc[v] += eps[v];
      acc[6 + v] += s;
    }
  }
}

// --------------------------------------------------------- reductions ---

// Sum NV doubles over a CTA (deterministic order).  `red` is shared scratch
// of at least 32*NV doubles; the result is broadcast to all threads in out.
template <int NV>
__device__ inline void block_sum(const double *v, double *red, double *out) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double w[NV];
#pragma unroll
  for (int q = 0; q < NV; q++) {
    w[q] = v[q];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) w[q] += __shfl_xor_sync(0xffffffffu, w[q], off);
  }
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NV; q++) red[warp * NV + q] = w[q];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int q = 0; q < NV; q++) {
      double s = (lane < nw) ? red[lane * NV + q] : 0.0;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
      if (lane == 0) red[32 * NV + q] = s;
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NV; q++) out[q] = red[32 * NV + q];
  __syncthreads();
}

// ------------------------------------------------------------ averages ---

// Volume averages of strain and stress for load case q (micro/src/
// homogenize.c:344-368): per element sum_gp w B u_e = Bbar u_e, stress =
// D_t Bbar u_e.  Adds element sums into acc[12] (6 strain, 6 stress); the
// caller divides by the volume.
template <int K>
__device__ inline void average_elems(int t, int nt, const MeshGeo &g,
                                     const uint8_t *__restrict__ etype, const double *D /*[2][36]*/,
                                     const double *Bbar /*[144]*/, const double *__restrict__ u,
                                     int q, double *acc) {
  for (int e = t; e < g.nelm; e += nt) {
    int nod[8];
    elem_nodes(g, e, nod);
    double eps[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll 1
    for (int a = 0; a < 8; a++)
#pragma unroll
      for (int d = 0; d < 3; d++) {
        double uv = u[(size_t)(nod[a] * 3 + d) * K + q];
#pragma unroll
        for (int v = 0; v < 6; v++) eps[v] = fma(Bbar[v * 24 + a * 3 + d], uv, eps[v]);
      }
    const double *C = D + etype[e] * 36;
#pragma unroll
    for (int v = 0; v < 6; v++) {
      double s = 0.0;
#pragma unroll
      for (int w = 0; w < 6; w++) s = fma(C[v * 6 + w], eps[w], s);
      acc[v] += eps[v];
      acc[6 + v] += s;
    }
  }
}

}  // namespace sp
