/*
 * oracle.c -- CPU restatement of the sputnik micro-RVE homogenization path.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Plain C99, single-threaded, FP64,
 * written to follow the reference's arithmetic order where the reference has
 * code, and extended from 2D to 3D where it does not.  Every function names
 * the reference lines it restates.  Deviations from the reference, each
 * with its reason:
 *   D1 ell_set_zero_col returns at the first -1 slot of any row
 *      (src/ell.c:103-118): orc_ell_set_zero_col_ref keeps that behaviour,
 *      orc_ell_set_zero_col_full zeroes the column in every row (needed for a
 *      symmetric operator under CG).  Both give the same solution because
 *      the boundary entries of the Newton correction are zero.
 *   D2 get_elem_disp gathers x_ell[i] instead of x_ell[elem_index[i]]
 *      (micro/src/homogenize.c:409): fixed here.
 *   D3 fem_init_struct leaves the 3D Gauss points unset (src/fem.c:9-14):
 *      the hexa8 points of src/fem.c:324-362 are used.
 *   D5 x_ell/dx_ell start uninitialised (micro/src/alloc.c:51-53): zeroed.
 *   D6 ell_solve_jacobi's tolerance is absolute (inc/ell.h:13); the Newton
 *      loop here stops on a relative residual ||r(u)|| <= rtol*||r(u0)||.
 * 3D conventions the reference never wrote (pinned by this file only):
 *   node (i,j,k) -> i + j*nx + k*nx*ny; element (ex,ey,ez) likewise with
 *   nex,ney; hexa8 local node order of src/fem.c:324-362; Voigt order
 *   (xx, yy, zz, xy, yz, xz) with engineering shears; quadrature weight
 *   vol_elm/8; node coordinates i*hx (src/mesh.c:869-876).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define GP_COORD 0.577350269189626 /* literal used by src/fem.c:324-362 */

/* ---------------------------------------------------------------- mesh --- */

/* src/mesh.c:762-786 (sizes, h, volumes), extended with the z axis. */
int orc_mesh_init(orc_mesh *m, int dim, const int *n_nodes, const double *len) {
  if (!m || (dim != 2 && dim != 3)) return 1;
  memset(m, 0, sizeof(*m));
  m->dim = dim;
  m->lx = len[0];
  m->ly = len[1];
  m->lz = (dim == 3) ? len[2] : 1;
  m->nx = n_nodes[0];
  m->ny = n_nodes[1];
  m->nz = (dim == 3) ? n_nodes[2] : 1;
  if (m->nx < 2 || m->ny < 2 || (dim == 3 && m->nz < 2)) return 2;
  m->nn = m->nx * m->ny * m->nz;
  m->nex = m->nx - 1;
  m->ney = m->ny - 1;
  m->nez = (dim == 3) ? m->nz - 1 : 1;
  m->nelm = m->nex * m->ney * m->nez;
  m->hx = m->lx / m->nex;
  m->hy = m->ly / m->ney;
  m->hz = (dim == 2) ? 1 : (m->lz / m->nez);
  m->vol = m->lx * m->ly * m->lz;
  m->vol_elm = m->hx * m->hy * m->hz;
  m->npe = (dim == 2) ? 4 : 8;
  m->nvoi = (dim == 2) ? 3 : 6;
  m->ngp = (dim == 2) ? 4 : 8;
  m->ndof = m->nn * dim;
  return 0;
}

/* src/mesh.c:869-876 */
void orc_node_coord(const orc_mesh *m, int node, double *x) {
  int i = node % m->nx;
  int j = (node / m->nx) % m->ny;
  int k = node / (m->nx * m->ny);
  x[0] = i * m->hx;
  x[1] = j * m->hy;
  if (m->dim == 3) x[2] = k * m->hz;
}

/* src/mesh.c:878-888; 3D adds the top face in hexa8 order (src/fem.c:324-362) */
void orc_elem_nodes(const orc_mesh *m, int e, int *nods) {
  int ex = e % m->nex;
  int ey = (e / m->nex) % m->ney;
  int ez = e / (m->nex * m->ney);
  int nxy = m->nx * m->ny;
  int n0 = ex + ey * m->nx + ez * nxy;
  nods[0] = n0;
  nods[1] = n0 + 1;
  nods[2] = n0 + m->nx + 1;
  nods[3] = n0 + m->nx;
  if (m->dim == 3) {
    for (int a = 0; a < 4; a++) nods[4 + a] = nods[a] + nxy;
  }
}

/* src/mesh.c:890-902: idx[node*dim + d] = gnode*dim + d */
void orc_elem_dofs(const orc_mesh *m, int e, int *idx) {
  int nods[8];
  orc_elem_nodes(m, e, nods);
  for (int a = 0; a < m->npe; a++)
    for (int d = 0; d < m->dim; d++) idx[a * m->dim + d] = nods[a] * m->dim + d;
}

int orc_is_boundary_node(const orc_mesh *m, int node) {
  int i = node % m->nx;
  int j = (node / m->nx) % m->ny;
  int k = node / (m->nx * m->ny);
  if (i == 0 || i == m->nx - 1 || j == 0 || j == m->ny - 1) return 1;
  if (m->dim == 3 && (k == 0 || k == m->nz - 1)) return 1;
  return 0;
}

/* src/mesh.c:788-867 lists the 2D boundary; here every face node, ascending. */
int orc_boundary_nodes(const orc_mesh *m, int *nodes) {
  int c = 0;
  for (int n = 0; n < m->nn; n++)
    if (orc_is_boundary_node(m, n)) {
      if (nodes) nodes[c] = n;
      c++;
    }
  return c;
}

/* micro/src/homogenize.c:487-494, with the z axis added */
void orc_elem_centroid(const orc_mesh *m, int e, double *c) {
  c[0] = (e % m->nex + 0.5) * m->hx;
  c[1] = ((e / m->nex) % m->ney + 0.5) * m->hy;
  if (m->dim == 3) c[2] = (e / (m->nex * m->ney) + 0.5) * m->hz;
}

/* micro/src/micro_struct.c:98-129 (FIBER_CILIN) applied per element
 * (micro/src/micro_struct.c:176-185).  In 3D the fibers are z-aligned
 * cylinders: the test only reads the (x, y) centroid, as the reference's
 * d < 2 loop does. */
int orc_fiber_cilin_types(const orc_mesh *m, const double *size, int nx_fib, int ny_fib,
                          double radio, const double *desv, unsigned char *elem_type) {
  double lx = size[0], ly = size[1];
  double center[2] = {lx / 2, ly / 2};
  for (int e = 0; e < m->nelm; e++) {
    double cen[3];
    orc_elem_centroid(m, e, cen);
    int id = ORC_ID_MATRIX;
    for (int i = 0; i < nx_fib && id == ORC_ID_MATRIX; i++) {
      for (int j = 0; j < ny_fib; j++) {
        double dev[2];
        dev[0] = desv[0] - lx / 2 + (lx / nx_fib) / 2 + i * (lx / nx_fib);
        dev[1] = desv[1] - ly / 2 + (ly / ny_fib) / 2 + j * (ly / ny_fib);
        double l = 0.0;
        for (int d = 0; d < 2; d++) l = l + pow(cen[d] - (center[d] + dev[d]), 2);
        l = sqrt(l);
        if (l <= radio) {
          id = ORC_ID_FIBER;
          break;
        }
      }
    }
    elem_type[e] = (unsigned char)id;
  }
  return 0;
}

/* ----------------------------------------------------------------- fem --- */

/* src/fem.c:309-405: hexa8 Gauss points (weight 1), shapes and local
 * derivatives.  Layout: xp[gp][3], sh[node][gp], ds[node][dim][gp]. */
void orc_hexa8_tables(double *xp, double *sh, double *ds) {
  static const int sgn[8][3] = {{-1, -1, -1}, {+1, -1, -1}, {+1, +1, -1}, {-1, +1, -1},
                                {-1, -1, +1}, {+1, -1, +1}, {+1, +1, +1}, {-1, +1, +1}};
  for (int gp = 0; gp < 8; gp++)
    for (int d = 0; d < 3; d++) xp[gp * 3 + d] = sgn[gp][d] * GP_COORD;
  for (int gp = 0; gp < 8; gp++) {
    double x = xp[gp * 3 + 0], y = xp[gp * 3 + 1], z = xp[gp * 3 + 2];
    for (int a = 0; a < 8; a++) {
      /* (1 +/- xi) factors, written as in src/fem.c:366-404 */
      double fx = (sgn[a][0] < 0) ? (1.0 - x) : (1.0 + x);
      double fy = (sgn[a][1] < 0) ? (1.0 - y) : (1.0 + y);
      double fz = (sgn[a][2] < 0) ? (1.0 - z) : (1.0 + z);
      sh[a * 8 + gp] = fx * fy * fz * 0.125;
      ds[(a * 3 + 0) * 8 + gp] = sgn[a][0] * 1.0 * fy * fz * 0.125;
      ds[(a * 3 + 1) * 8 + gp] = sgn[a][1] * 1.0 * fx * fz * 0.125;
      ds[(a * 3 + 2) * 8 + gp] = sgn[a][2] * 1.0 * fx * fy * 0.125;
    }
  }
}

/* src/fem.c:3-59 (structured shortcut: dN/dx = dN/dxi * 2/h, w = vol/ngp),
 * 2D as written there, 3D from the hexa8 tables (deviation D3). */
void orc_struct_dsh(const orc_mesh *m, double *dsh, double *wp) {
  int dim = m->dim, ngp = m->ngp;
  if (dim == 2) {
    double xp[8] = {-GP_COORD, -GP_COORD, +GP_COORD, -GP_COORD,
                    +GP_COORD, +GP_COORD, -GP_COORD, +GP_COORD};
    double hx = m->hx, hy = m->hy;
    for (int gp = 0; gp < 4; gp++) {
#define DS2(a, d) dsh[((a) * 2 + (d)) * 4 + gp]
      DS2(0, 0) = -1 * (1 - xp[2 * gp + 1]) / 4 * 2 / hx;
      DS2(1, 0) = +1 * (1 - xp[2 * gp + 1]) / 4 * 2 / hx;
      DS2(2, 0) = +1 * (1 + xp[2 * gp + 1]) / 4 * 2 / hx;
      DS2(3, 0) = -1 * (1 + xp[2 * gp + 1]) / 4 * 2 / hx;
      DS2(0, 1) = -1 * (1 - xp[2 * gp + 0]) / 4 * 2 / hy;
      DS2(1, 1) = -1 * (1 + xp[2 * gp + 0]) / 4 * 2 / hy;
      DS2(2, 1) = +1 * (1 + xp[2 * gp + 0]) / 4 * 2 / hy;
      DS2(3, 1) = +1 * (1 - xp[2 * gp + 0]) / 4 * 2 / hy;
#undef DS2
    }
    double vol = hx * hy;
    for (int gp = 0; gp < ngp; gp++) wp[gp] = vol / ngp;
  } else {
    double xp[24], sh[64], ds[192];
    double h[3] = {m->hx, m->hy, m->hz};
    orc_hexa8_tables(xp, sh, ds);
    for (int a = 0; a < 8; a++)
      for (int d = 0; d < 3; d++)
        for (int gp = 0; gp < 8; gp++)
          dsh[(a * 3 + d) * 8 + gp] = ds[(a * 3 + d) * 8 + gp] * 2 / h[d];
    double vol = m->hx * m->hy * m->hz;
    for (int gp = 0; gp < ngp; gp++) wp[gp] = vol / ngp;
  }
}

/* micro/src/init.c:40-51 (2D), extended to 3D with Voigt (xx,yy,zz,xy,yz,xz).
 * Layout bmat[v][i][gp] with i = node*dim + d. */
void orc_bmat(const orc_mesh *m, const double *dsh, double *bmat) {
  int dim = m->dim, npe = m->npe, ngp = m->ngp, nvoi = m->nvoi, nc = npe * dim;
  memset(bmat, 0, sizeof(double) * nvoi * nc * ngp);
#define B(v, i, gp) bmat[((v) * nc + (i)) * ngp + (gp)]
#define D(a, d, gp) dsh[((a) * dim + (d)) * ngp + (gp)]
  for (int gp = 0; gp < ngp; gp++) {
    for (int a = 0; a < npe; a++) {
      if (dim == 2) {
        B(0, a * 2 + 0, gp) = D(a, 0, gp);
        B(1, a * 2 + 1, gp) = D(a, 1, gp);
        B(2, a * 2 + 0, gp) = D(a, 1, gp);
        B(2, a * 2 + 1, gp) = D(a, 0, gp);
      } else {
        B(0, a * 3 + 0, gp) = D(a, 0, gp);
        B(1, a * 3 + 1, gp) = D(a, 1, gp);
        B(2, a * 3 + 2, gp) = D(a, 2, gp);
        B(3, a * 3 + 0, gp) = D(a, 1, gp);
        B(3, a * 3 + 1, gp) = D(a, 0, gp);
        B(4, a * 3 + 1, gp) = D(a, 2, gp);
        B(4, a * 3 + 2, gp) = D(a, 1, gp);
        B(5, a * 3 + 0, gp) = D(a, 2, gp);
        B(5, a * 3 + 2, gp) = D(a, 0, gp);
      }
    }
  }
#undef B
#undef D
}

/* 2D: plane strain, src/material.c:36-59.  3D: isotropic from the Lame
 * constants of src/material.c:121-122. */
void orc_iso_D(int dim, double E, double nu, double *D) {
  if (dim == 2) {
    D[0] = 1.0 - nu; D[1] = nu;       D[2] = 0.0;
    D[3] = nu;       D[4] = 1.0 - nu; D[5] = 0.0;
    D[6] = 0.0;      D[7] = 0.0;      D[8] = (1 - 2 * nu) / 2;
    for (int i = 0; i < 9; i++) D[i] *= E / ((1 + nu) * (1 - 2 * nu));
  } else {
    double lam = (E * nu) / ((1 + nu) * (1 - 2 * nu));
    double mu = E / (2 * (1 + nu));
    for (int i = 0; i < 36; i++) D[i] = 0.0;
    for (int i = 0; i < 3; i++) {
      for (int j = 0; j < 3; j++) D[i * 6 + j] = lam;
      D[i * 6 + i] = lam + 2 * mu;
      D[(3 + i) * 6 + (3 + i)] = mu;
    }
  }
}

/* micro/src/assembly.c:97-108: Ke = sum_gp B^T C B w, same loop nest and
 * product order. */
void orc_elem_stiffness(const orc_mesh *m, const double *bmat, const double *wp, const double *C,
                        double *Ke) {
  int nc = m->npe * m->dim, nvoi = m->nvoi, ngp = m->ngp;
  for (int i = 0; i < nc * nc; i++) Ke[i] = 0.0;
#define B(v, i, gp) bmat[((v) * nc + (i)) * ngp + (gp)]
  for (int gp = 0; gp < ngp; gp++)
    for (int i = 0; i < nc; i++)
      for (int j = 0; j < nc; j++)
        for (int k = 0; k < nvoi; k++)
          for (int h = 0; h < nvoi; h++)
            Ke[i * nc + j] += B(h, i, gp) * C[h * nvoi + k] * B(k, j, gp) * wp[gp];
#undef B
}

/* ----------------------------------------------------------------- ELL --- */

/* src/ell.c:3-15 */
int orc_ell_init(orc_ell *a, int nrow, int ncol, int nnz) {
  if (!a) return 1;
  a->nrow = nrow;
  a->ncol = ncol;
  a->nnz = nnz;
  a->cols = (int *)malloc((size_t)nrow * nnz * sizeof(int));
  a->vals = (double *)malloc((size_t)nrow * nnz * sizeof(double));
  if (!a->cols || !a->vals) return 2;
  for (size_t i = 0; i < (size_t)nrow * nnz; i++) {
    a->cols[i] = -1;
    a->vals[i] = +0;
  }
  return 0;
}

void orc_ell_free(orc_ell *a) {
  free(a->cols);
  free(a->vals);
  a->cols = NULL;
  a->vals = NULL;
}

/* src/ell.c:46-73: first-touch insertion, accumulate on a repeated column */
int orc_ell_add_val(orc_ell *a, int row, int col, double val) {
  if (row >= a->nrow || col >= a->ncol) return 1;
  if (row < 0 || col < 0) return 2;
  int *c = a->cols + (size_t)row * a->nnz;
  double *v = a->vals + (size_t)row * a->nnz;
  for (int j = 0; j < a->nnz; j++) {
    if (c[j] == -1) {
      c[j] = col;
      v[j] = val;
      return 0;
    }
    if (c[j] == col) {
      v[j] += val;
      return 0;
    }
  }
  return 3;
}

/* src/ell.c:75-84 (note vals[i*nx + j]) */
int orc_ell_add_vals(orc_ell *a, const int *ix, int nx, const int *iy, int ny, const double *vals) {
  if (!a || !ix || !iy || !vals) return 1;
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++) orc_ell_add_val(a, ix[i], iy[j], vals[i * nx + j]);
  return 0;
}

/* src/ell.c:186-208 */
int orc_ell_get_val(const orc_ell *a, int row, int col, double *val) {
  if (row >= a->nrow || col >= a->ncol) return 1;
  if (row < 0 || col < 0) return 2;
  const int *c = a->cols + (size_t)row * a->nnz;
  for (int j = 0; j < a->nnz; j++) {
    if (c[j] == -1) {
      *val = 0.0;
      return 0;
    }
    if (c[j] == col) {
      *val = a->vals[(size_t)row * a->nnz + j];
      return 0;
    }
  }
  return 3;
}

/* src/ell.c:127-141: per row, slot order, stop at the first -1 */
int orc_ell_mvp(const orc_ell *a, const double *x, double *y) {
  if (!a || !x || !y) return 1;
  for (int i = 0; i < a->nrow; i++) {
    double s = 0;
    const int *c = a->cols + (size_t)i * a->nnz;
    const double *v = a->vals + (size_t)i * a->nnz;
    for (int j = 0; j < a->nnz; j++) {
      if (c[j] == -1) break;
      s += v[j] * x[c[j]];
    }
    y[i] = s;
  }
  return 0;
}

/* src/ell.c:86-101 */
int orc_ell_set_zero_row(orc_ell *a, int row, double diag) {
  int *c = a->cols + (size_t)row * a->nnz;
  double *v = a->vals + (size_t)row * a->nnz;
  for (int j = 0; j < a->nnz; j++) {
    if (c[j] == -1) return 0;
    v[j] = (c[j] == row) ? diag : 0.0;
  }
  return 0;
}

/* src/ell.c:103-118, including the early return at the first -1 of any row */
int orc_ell_set_zero_col_ref(orc_ell *a, int col, double diag) {
  for (int i = 0; i < a->nrow; i++) {
    int *c = a->cols + (size_t)i * a->nnz;
    double *v = a->vals + (size_t)i * a->nnz;
    for (int j = 0; j < a->nnz; j++) {
      if (c[j] == -1) return 0;
      if (c[j] == col) v[j] = (i == col) ? diag : 0.0;
    }
  }
  return 0;
}

/* deviation D1: the column is cleared in every row */
int orc_ell_set_zero_col_full(orc_ell *a, int col, double diag) {
  for (int i = 0; i < a->nrow; i++) {
    int *c = a->cols + (size_t)i * a->nnz;
    double *v = a->vals + (size_t)i * a->nnz;
    for (int j = 0; j < a->nnz; j++) {
      if (c[j] == -1) break;
      if (c[j] == col) v[j] = (i == col) ? diag : 0.0;
    }
  }
  return 0;
}

/* src/ell.c:120-124 */
int orc_ell_set_zero_mat(orc_ell *a) {
  for (int i = 0; i < a->nrow; i++) orc_ell_set_zero_row(a, i, 0.0);
  return 0;
}

/* ------------------------------------------------------------ assembly --- */

/* micro/src/assembly.c:84-137.  Every element of one material type has the
 * same Ke on a structured grid (same B, same C), so Ke_by_type[t] holds the
 * matrix the reference recomputes per element.  The BC loop clears every
 * boundary dof: rows always, columns with the reference's early-return
 * semantics (symmetric_bc = 0) or in every row (symmetric_bc = 1). */
int orc_assemble_jac(const orc_mesh *m, const unsigned char *etype, const double *Ke_by_type,
                     orc_ell *A, int symmetric_bc) {
  int nc = m->npe * m->dim;
  int idx[24];
  orc_ell_set_zero_mat(A);
  for (int e = 0; e < m->nelm; e++) {
    orc_elem_dofs(m, e, idx);
    orc_ell_add_vals(A, idx, nc, idx, nc, Ke_by_type + (size_t)etype[e] * nc * nc);
  }
  if (symmetric_bc) {
    /* zero rows first, then every column in one pass (same result as the
     * per-dof call sequence, which is order independent) */
    unsigned char *bmask = (unsigned char *)calloc(m->ndof, 1);
    for (int n = 0; n < m->nn; n++)
      if (orc_is_boundary_node(m, n))
        for (int d = 0; d < m->dim; d++) bmask[n * m->dim + d] = 1;
    for (int i = 0; i < A->nrow; i++) {
      int *c = A->cols + (size_t)i * A->nnz;
      double *v = A->vals + (size_t)i * A->nnz;
      for (int j = 0; j < A->nnz; j++) {
        if (c[j] == -1) break;
        if (bmask[i])
          v[j] = (c[j] == i) ? 1.0 : 0.0;
        else if (bmask[c[j]])
          v[j] = 0.0;
      }
    }
    free(bmask);
  } else {
    for (int n = 0; n < m->nn; n++) {
      if (!orc_is_boundary_node(m, n)) continue;
      for (int d = 0; d < m->dim; d++) {
        orc_ell_set_zero_row(A, n * m->dim + d, 1.0);
        orc_ell_set_zero_col_ref(A, n * m->dim + d, 1.0);
      }
    }
  }
  return 0;
}

/* micro/src/homogenize.c:416-428 (get_strain, with deviation D2) and
 * micro/src/material.c:20-28 (stress = C strain) */
static void strain_stress_gp(const orc_mesh *m, const double *bmat, const double *C,
                             const double *ue, int gp, double *strain, double *stress) {
  int nc = m->npe * m->dim, nvoi = m->nvoi, ngp = m->ngp;
  for (int v = 0; v < nvoi; v++) {
    strain[v] = 0.0;
    for (int i = 0; i < nc; i++) strain[v] += bmat[(v * nc + i) * ngp + gp] * ue[i];
  }
  for (int i = 0; i < nvoi; i++) {
    stress[i] = 0.0;
    for (int j = 0; j < nvoi; j++) stress[i] += C[i * nvoi + j] * strain[j];
  }
}

/* micro/src/assembly.c:33-82 */
int orc_assemble_res(const orc_mesh *m, const unsigned char *etype, const double *D_by_type,
                     const double *bmat, const double *wp, const double *u, double *res,
                     double *norm) {
  int nc = m->npe * m->dim, nvoi = m->nvoi, ngp = m->ngp;
  int idx[24];
  double ue[24], rese[24], strain[6], stress[6];
  for (int i = 0; i < m->ndof; i++) res[i] = 0.0;
  for (int e = 0; e < m->nelm; e++) {
    for (int i = 0; i < nc; i++) rese[i] = 0.0;
    orc_elem_dofs(m, e, idx);
    for (int i = 0; i < nc; i++) ue[i] = u[idx[i]];
    const double *C = D_by_type + (size_t)etype[e] * nvoi * nvoi;
    for (int gp = 0; gp < ngp; gp++) {
      strain_stress_gp(m, bmat, C, ue, gp, strain, stress);
      for (int i = 0; i < nc; i++)
        for (int j = 0; j < nvoi; j++)
          rese[i] += bmat[(j * nc + i) * ngp + gp] * stress[j] * wp[gp];
    }
    for (int i = 0; i < nc; i++) res[idx[i]] += rese[i];
  }
  for (int n = 0; n < m->nn; n++)
    if (orc_is_boundary_node(m, n))
      for (int d = 0; d < m->dim; d++) res[n * m->dim + d] = 0.0;
  double s = 0;
  for (int i = 0; i < m->ndof; i++) s += res[i] * res[i];
  *norm = sqrt(s);
  return 0;
}

/* micro/src/homogenize.c:227-242 (set_disp_0) and :335-342 (strain_x_coord),
 * 3D: u = eps . x with eps_xy = gamma_xy/2 etc. */
void orc_affine_bc(const orc_mesh *m, const double *strain, double *u) {
  for (int n = 0; n < m->nn; n++) {
    if (!orc_is_boundary_node(m, n)) continue;
    double x[3];
    orc_node_coord(m, n, x);
    if (m->dim == 2) {
      u[n * 2 + 0] = strain[0] * x[0] + strain[2] / 2 * x[1];
      u[n * 2 + 1] = strain[2] / 2 * x[0] + strain[1] * x[1];
    } else {
      u[n * 3 + 0] = strain[0] * x[0] + strain[3] / 2 * x[1] + strain[5] / 2 * x[2];
      u[n * 3 + 1] = strain[3] / 2 * x[0] + strain[1] * x[1] + strain[4] / 2 * x[2];
      u[n * 3 + 2] = strain[5] / 2 * x[0] + strain[4] / 2 * x[1] + strain[2] * x[2];
    }
  }
}

/* micro/src/homogenize.c:344-368 */
void orc_averages(const orc_mesh *m, const unsigned char *etype, const double *D_by_type,
                  const double *bmat, const double *wp, const double *u, double *strain_ave,
                  double *stress_ave) {
  int nc = m->npe * m->dim, nvoi = m->nvoi, ngp = m->ngp;
  int idx[24];
  double ue[24], strain[6], stress[6];
  for (int i = 0; i < nvoi; i++) strain_ave[i] = stress_ave[i] = 0.0;
  for (int e = 0; e < m->nelm; e++) {
    orc_elem_dofs(m, e, idx);
    for (int i = 0; i < nc; i++) ue[i] = u[idx[i]];
    const double *C = D_by_type + (size_t)etype[e] * nvoi * nvoi;
    for (int gp = 0; gp < ngp; gp++) {
      strain_stress_gp(m, bmat, C, ue, gp, strain, stress);
      for (int i = 0; i < nvoi; i++) {
        stress_ave[i] += stress[i] * wp[gp];
        strain_ave[i] += strain[i] * wp[gp];
      }
    }
  }
  for (int i = 0; i < nvoi; i++) {
    stress_ave[i] /= m->vol;
    strain_ave[i] /= m->vol;
  }
}

/* ------------------------------------------------------------- solvers --- */

/* src/ell.c:143-184, with max_its/min_err as arguments (inc/ell.h:12-13
 * gives 100000 and 1e-10) */
int orc_jacobi(const orc_ell *A, const double *b, double *x, int max_its, double min_err, int *its,
               double *err) {
  int n = A->nrow;
  double *r = (double *)malloc(n * sizeof(double));
  double *dinv = (double *)malloc(n * sizeof(double));
  for (int i = 0; i < n; i++) {
    orc_ell_get_val(A, i, i, &dinv[i]);
    dinv[i] = 1 / dinv[i];
  }
  int k = 0;
  double e = 0;
  while (k < max_its) {
    e = 0;
    orc_ell_mvp(A, x, r);
    for (int i = 0; i < n; i++) {
      r[i] -= b[i];
      e += r[i] * r[i];
    }
    e = sqrt(e);
    if (e < min_err) break;
    for (int i = 0; i < n; i++) x[i] -= dinv[i] * r[i];
    k++;
  }
  *its = k;
  *err = e;
  free(r);
  free(dinv);
  return 0;
}

static double dot(int n, const double *a, const double *b) {
  double s = 0;
  for (int i = 0; i < n; i++) s += a[i] * b[i];
  return s;
}

/* Jacobi-preconditioned CG as PETSc's KSPCG + PCJACOBI runs it
 * (micro/src/homogenize.c:324-326 with -ksp_type cg -pc_type jacobi), using
 * the unpreconditioned residual norm and convergence ||r|| <= rtol*||b||. */
int orc_pcg(const orc_ell *A, const double *b, double *x, double rtol, int max_its, int *its,
            double *relres) {
  int n = A->nrow;
  double *r = (double *)malloc(n * sizeof(double));
  double *z = (double *)malloc(n * sizeof(double));
  double *p = (double *)malloc(n * sizeof(double));
  double *q = (double *)malloc(n * sizeof(double));
  double *dinv = (double *)malloc(n * sizeof(double));
  for (int i = 0; i < n; i++) {
    double d;
    orc_ell_get_val(A, i, i, &d);
    dinv[i] = 1.0 / d;
  }
  double bnorm = sqrt(dot(n, b, b));
  orc_ell_mvp(A, x, q);
  for (int i = 0; i < n; i++) r[i] = b[i] - q[i];
  int k = 0;
  if (bnorm == 0.0) bnorm = 1.0;
  if (sqrt(dot(n, r, r)) > rtol * bnorm) {
    for (int i = 0; i < n; i++) p[i] = z[i] = dinv[i] * r[i];
    double rho = dot(n, r, z);
    while (k < max_its) {
      orc_ell_mvp(A, p, q);
      double alpha = rho / dot(n, p, q);
      for (int i = 0; i < n; i++) {
        x[i] += alpha * p[i];
        r[i] -= alpha * q[i];
      }
      k++;
      if (sqrt(dot(n, r, r)) <= rtol * bnorm) break;
      for (int i = 0; i < n; i++) z[i] = dinv[i] * r[i];
      double rho1 = dot(n, r, z);
      double beta = rho1 / rho;
      rho = rho1;
      for (int i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
    }
  }
  orc_ell_mvp(A, x, q);
  for (int i = 0; i < n; i++) r[i] = b[i] - q[i];
  *relres = sqrt(dot(n, r, r)) / bnorm;
  *its = k;
  free(r);
  free(z);
  free(p);
  free(q);
  free(dinv);
  return (k >= max_its) ? 4 : 0;
}

/* ------------------------------------------------------ homogenization --- */

typedef struct {
  double dsh[8 * 3 * 8], wp[8], bmat[6 * 24 * 8];
  double D[2 * 36], Ke[2 * 576];
} orc_ops;

static void build_ops(const orc_mesh *m, const orc_params *p, orc_ops *o) {
  int nvoi = m->nvoi, nc = m->npe * m->dim;
  orc_struct_dsh(m, o->dsh, o->wp);
  orc_bmat(m, o->dsh, o->bmat);
  for (int t = 0; t < 2; t++) {
    orc_iso_D(m->dim, p->E[t], p->nu[t], o->D + t * nvoi * nvoi);
    orc_elem_stiffness(m, o->bmat, o->wp, o->D + t * nvoi * nvoi, o->Ke + t * nc * nc);
  }
}

/* micro/src/homogenize.c:175-225 (homog_fe2) per load case: set_disp_0,
 * Newton with residual/jacobian/solve/add_x_dx, then get_averages.  The
 * Jacobian is assembled once (linear materials give the same matrix at
 * every Newton step). */
int orc_homogenize(const orc_mesh *m, const unsigned char *etype, const orc_params *p, int nrhs,
                   const double *strains, double *strain_ave, double *stress_ave, double *u_out,
                   double *stats) {
  orc_ops o;
  build_ops(m, p, &o);
  orc_ell A;
  int width = (m->dim == 2) ? 18 : 81; /* micro/src/alloc.c:6 */
  if (orc_ell_init(&A, m->ndof, m->ndof, width)) return 2;
  orc_assemble_jac(m, etype, o.Ke, &A, p->solver == 0);
  double *u = (double *)calloc(m->ndof, sizeof(double));
  double *res = (double *)malloc(m->ndof * sizeof(double));
  double *du = (double *)malloc(m->ndof * sizeof(double));
  int ierr = 0;
  for (int k = 0; k < nrhs; k++) {
    const double *eps = strains + k * m->nvoi;
    memset(u, 0, m->ndof * sizeof(double));
    orc_affine_bc(m, eps, u);
    double norm = 0, norm0 = -1;
    int nl = 0, lin_total = 0;
    while (nl < p->max_newton) {
      orc_assemble_res(m, etype, o.D, o.bmat, o.wp, u, res, &norm);
      if (norm0 < 0) norm0 = norm;
      if (norm <= p->rtol * norm0 || norm == 0.0) break;
      for (int i = 0; i < m->ndof; i++) {
        res[i] = -res[i];
        du[i] = 0.0;
      }
      int its = 0;
      double rr = 0;
      if (p->solver == 0)
        ierr |= orc_pcg(&A, res, du, p->lin_rtol, p->max_lin_its, &its, &rr);
      else
        orc_jacobi(&A, res, du, p->max_lin_its, p->lin_rtol * norm0, &its, &rr);
      lin_total += its;
      for (int i = 0; i < m->ndof; i++) u[i] += du[i];
      nl++;
    }
    orc_assemble_res(m, etype, o.D, o.bmat, o.wp, u, res, &norm);
    orc_averages(m, etype, o.D, o.bmat, o.wp, u, strain_ave + k * m->nvoi,
                 stress_ave + k * m->nvoi);
    if (u_out) memcpy(u_out + (size_t)k * m->ndof, u, m->ndof * sizeof(double));
    if (stats) {
      stats[k * 4 + 0] = nl;
      stats[k * 4 + 1] = lin_total;
      stats[k * 4 + 2] = (norm0 > 0) ? norm / norm0 : 0.0;
      stats[k * 4 + 3] = norm0;
    }
  }
  free(u);
  free(res);
  free(du);
  orc_ell_free(&A);
  return ierr;
}

int orc_unit_tangent(const orc_mesh *m, const unsigned char *etype, const orc_params *p,
                     double *C, double *stats) {
  int nvoi = m->nvoi;
  double strains[36] = {0}, sa[36], st[36];
  for (int j = 0; j < nvoi; j++) strains[j * nvoi + j] = 1.0;
  int ierr = orc_homogenize(m, etype, p, nvoi, strains, sa, st, NULL, stats);
  for (int i = 0; i < nvoi; i++)
    for (int j = 0; j < nvoi; j++) C[i * nvoi + j] = st[j * nvoi + i];
  return ierr;
}

/* micro/src/homogenize.c:59-94 */
int orc_fd_tangent(const orc_mesh *m, const unsigned char *etype, const orc_params *p,
                   const double *strain_mac, double *C, double *stress0) {
  int nvoi = m->nvoi;
  double strains[7 * 6] = {0}, sa[7 * 6], st[7 * 6];
  for (int k = 0; k <= nvoi; k++)
    for (int i = 0; i < nvoi; i++) strains[k * nvoi + i] = strain_mac[i];
  for (int i = 0; i < nvoi; i++) strains[(i + 1) * nvoi + i] += 0.005;
  int ierr = orc_homogenize(m, etype, p, nvoi + 1, strains, sa, st, NULL, NULL);
  for (int i = 0; i < nvoi; i++)
    for (int j = 0; j < nvoi; j++)
      C[j * nvoi + i] = (st[(i + 1) * nvoi + j] - st[j]) /
                        (strains[(i + 1) * nvoi + i] - strains[i]);
  if (stress0)
    for (int j = 0; j < nvoi; j++) stress0[j] = st[j];
  return ierr;
}
