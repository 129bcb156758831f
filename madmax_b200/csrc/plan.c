/*
 * plan.c -- host set-up of a structured 3D RVE mesh: the ELL column pattern
 * in the reference's insertion order, the element -> slot map used by the
 * GPU scatter, the 8-colour element partition and the element
 * classification.  All integer work, done once per distinct mesh size.
 */
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "sp_internal.h"

static __thread char g_err[512];

int sp_set_error(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

const char *sp_last_error(void) { return g_err; }

int sp_version(void) { return 100; }

/* weak: the reference's programs define their own (micro/src/main.c:16) */
#include "solvers.h"
__attribute__((weak)) solver_t solver;

/* Element dofs in hexa8 local order: idx[a*3 + d] = 3*node_a + d
 * (src/mesh.c:890-902 extended to 3D). */
static void elem_dofs(const sp_plan_host *p, int e, int *idx) {
  int ex = e % p->n[0], ey = (e / p->n[0]) % p->n[1], ez = e / (p->n[0] * p->n[1]);
  int nxy = p->nx * p->ny;
  int n0 = ex + ey * p->nx + ez * nxy;
  int nod[8] = {n0, n0 + 1, n0 + p->nx + 1, n0 + p->nx, 0, 0, 0, 0};
  for (int a = 0; a < 4; a++) nod[4 + a] = nod[a] + nxy;
  for (int a = 0; a < 8; a++)
    for (int d = 0; d < 3; d++) idx[a * 3 + d] = nod[a] * 3 + d;
}

/* Position of column node relative to row node as one of 27 codes. */
static int neighbour_code(const sp_plan_host *p, int row_node, int col_node) {
  int ri = row_node % p->nx, rj = (row_node / p->nx) % p->ny, rk = row_node / (p->nx * p->ny);
  int ci = col_node % p->nx, cj = (col_node / p->nx) % p->ny, ck = col_node / (p->nx * p->ny);
  return ((ck - rk + 1) * 3 + (cj - rj + 1)) * 3 + (ci - ri + 1);
}

/* Replays ell_add_vals over the element loop of micro/src/assembly.c:93-110:
 * each row receives a new column in the first free slot the first time an
 * element touches (row, col) (src/ell.c:46-73).  A 81-entry table per row,
 * keyed by (neighbour code, dof), replaces the reference's linear search;
 * the slots it hands out are the same. */
int sp_plan_build(const int *n, sp_plan_host *p) {
  memset(p, 0, sizeof(*p));
  p->nbr = NULL;
  if (n[0] < 1 || n[1] < 1 || n[2] < 1 || n[0] > 1024 || n[1] > 1024 || n[2] > 1024)
    return sp_set_error(SP_ERR_ARG, "mesh size %dx%dx%d out of range", n[0], n[1], n[2]);
  for (int d = 0; d < 3; d++) p->n[d] = n[d];
  p->nx = n[0] + 1;
  p->ny = n[1] + 1;
  p->nz = n[2] + 1;
  p->nn = p->nx * p->ny * p->nz;
  p->ndof = 3 * p->nn;
  p->nelm = n[0] * n[1] * n[2];
  if ((double)p->ndof * SP_WP > 2147483647.0)
    return sp_set_error(SP_ERR_ARG, "mesh too large for 32-bit ELL indices");
  p->cols = (int *)malloc((size_t)p->ndof * SP_WP * sizeof(int));
  p->slot = (uint8_t *)malloc((size_t)p->nelm * SP_KE);
  p->color_elems = (int *)malloc((size_t)p->nelm * sizeof(int));
  int8_t *tab = (int8_t *)malloc((size_t)p->ndof * 81);
  uint8_t *fill = (uint8_t *)calloc(p->ndof, 1);
  if (!p->cols || !p->slot || !p->color_elems || !tab || !fill) {
    free(tab);
    free(fill);
    sp_plan_free(p);
    return sp_set_error(SP_ERR_NOMEM, "plan allocation failed");
  }
  for (size_t i = 0; i < (size_t)p->ndof * SP_WP; i++) p->cols[i] = -1;
  memset(tab, -1, (size_t)p->ndof * 81);
  int idx[SP_NC];
  for (int e = 0; e < p->nelm; e++) {
    elem_dofs(p, e, idx);
    uint8_t *se = p->slot + (size_t)e * SP_KE;
    for (int i = 0; i < SP_NC; i++) {
      int row = idx[i];
      for (int j = 0; j < SP_NC; j++) {
        int col = idx[j];
        int key = neighbour_code(p, row / 3, col / 3) * 3 + col % 3;
        int8_t *t = tab + (size_t)row * 81 + key;
        if (*t < 0) {
          *t = (int8_t)fill[row]++;
          p->cols[(size_t)row * SP_WP + *t] = col;
        }
        se[i * SP_NC + j] = (uint8_t)*t;
      }
    }
  }
  free(tab);
  free(fill);
  /* colour = parity of (ex, ey, ez): elements of one colour share no node */
  int cnt[8] = {0};
  for (int e = 0; e < p->nelm; e++) {
    int ex = e % n[0], ey = (e / n[0]) % n[1], ez = e / (n[0] * n[1]);
    cnt[(ex & 1) | ((ey & 1) << 1) | ((ez & 1) << 2)]++;
  }
  p->color_off[0] = 0;
  for (int c = 0; c < 8; c++) p->color_off[c + 1] = p->color_off[c] + cnt[c];
  int pos[8];
  for (int c = 0; c < 8; c++) pos[c] = p->color_off[c];
  for (int e = 0; e < p->nelm; e++) {
    int ex = e % n[0], ey = (e / n[0]) % n[1], ez = e / (n[0] * n[1]);
    p->color_elems[pos[(ex & 1) | ((ey & 1) << 1) | ((ez & 1) << 2)]++] = e;
  }
  int inner = (p->nx - 2) * (p->ny - 2) * (p->nz - 2);
  p->boundary_nodes = p->nn - (inner > 0 ? inner : 0);
  /* Node-sliced view of the same ELL rows.  Slots come in node triples:
   * the first time an element touches (row, node b) it inserts b's three
   * dofs in a row (the j loop of ell_add_vals runs over local dofs), and the
   * three rows of one node receive the same columns in the same order.  So
   * slot 3m + c of row 3a + d holds column 3 b_m(a) + c, and the 3x3 block
   * (a, b_m) sits at slots 3m..3m+2 of rows 3a..3a+2.  nbr[s][m][l] = b_m of
   * node a = 32 s + l; unused groups and padding nodes point at a itself
   * (their values are zero). */
  p->nn_pad = (p->nn + 31) / 32 * 32;
  p->nslice = p->nn_pad / 32;
  p->nbr = (int *)malloc((size_t)p->nslice * 27 * 32 * sizeof(int));
  if (!p->nbr) {
    sp_plan_free(p);
    return sp_set_error(SP_ERR_NOMEM, "plan allocation failed");
  }
  for (int a = 0; a < p->nn_pad; a++) {
    int s = a / 32, l = a % 32;
    for (int m = 0; m < 27; m++) {
      int b = (a < p->nn) ? a : 0;
      if (a < p->nn) {
        int c0 = p->cols[(size_t)(3 * a) * SP_WP + 3 * m];
        if (c0 >= 0) {
          b = c0 / 3;
          /* the triple structure the slice layout relies on */
          for (int d = 0; d < 3; d++)
            for (int c = 0; c < 3; c++)
              if (p->cols[(size_t)(3 * a + d) * SP_WP + 3 * m + c] != 3 * b + c) {
                sp_plan_free(p);
                return sp_set_error(SP_ERR_ARG, "ELL rows are not in node triples");
              }
        }
      }
      p->nbr[((size_t)s * 27 + m) * 32 + l] = b;
    }
  }
  return SP_OK;
}

void sp_plan_free(sp_plan_host *p) {
  free(p->nbr);
  p->nbr = NULL;
  free(p->cols);
  free(p->slot);
  free(p->color_elems);
  p->cols = NULL;
  p->slot = NULL;
  p->color_elems = NULL;
}

int sp_ell_pattern(const int *n, int *cols) {
  if (!n || !cols) return sp_set_error(SP_ERR_ARG, "null argument");
  sp_plan_host p;
  int rc = sp_plan_build(n, &p);
  if (rc) return rc;
  for (int r = 0; r < p.ndof; r++)
    memcpy(cols + (size_t)r * SP_ELL_WIDTH, p.cols + (size_t)r * SP_WP,
           SP_ELL_WIDTH * sizeof(int));
  sp_plan_free(&p);
  return SP_OK;
}

/* micro/src/micro_struct.c:98-129 per element centroid
 * (micro/src/homogenize.c:487-494, z added).  z-aligned cylinders: only the
 * (x, y) centroid enters the test, with the reference's pow/sqrt and <=. */
int sp_classify_elements(const sp_rve_desc *d, uint8_t *etype, int *nfiber) {
  int nex = d->n[0], ney = d->n[1], nez = d->n[2];
  if (d->nx_fib < 1 || d->ny_fib < 1) return sp_set_error(SP_ERR_ARG, "fiber counts must be >= 1");
  double lx = d->len[0], ly = d->len[1];
  double hx = d->len[0] / nex, hy = d->len[1] / ney;
  double center[2] = {lx / 2, ly / 2};
  int nf = 0;
  /* the type of an element depends on (ex, ey) only: classify one z layer */
  for (int ey = 0; ey < ney; ey++) {
    for (int ex = 0; ex < nex; ex++) {
      double cen[2] = {(ex + 0.5) * hx, (ey + 0.5) * hy};
      int id = SP_ID_MATRIX;
      for (int i = 0; i < d->nx_fib && id == SP_ID_MATRIX; i++) {
        for (int j = 0; j < d->ny_fib; j++) {
          double dev[2];
          dev[0] = d->desv[0] - lx / 2 + (lx / d->nx_fib) / 2 + i * (lx / d->nx_fib);
          dev[1] = d->desv[1] - ly / 2 + (ly / d->ny_fib) / 2 + j * (ly / d->ny_fib);
          double l = 0.0;
          for (int k = 0; k < 2; k++) l = l + pow(cen[k] - (center[k] + dev[k]), 2);
          l = sqrt(l);
          if (l <= d->radius) {
            id = SP_ID_FIBER;
            break;
          }
        }
      }
      for (int ez = 0; ez < nez; ez++) etype[(size_t)ez * nex * ney + ey * nex + ex] = (uint8_t)id;
      if (id == SP_ID_FIBER) nf += nez;
    }
  }
  if (nfiber) *nfiber = nf;
  return SP_OK;
}

int sp_classify(const sp_rve_desc *d, unsigned char *etype) {
  if (!d || !etype) return sp_set_error(SP_ERR_ARG, "null argument");
  if (d->n[0] < 1 || d->n[1] < 1 || d->n[2] < 1) return sp_set_error(SP_ERR_ARG, "bad mesh size");
  return sp_classify_elements(d, etype, NULL);
}

/* isotropic elasticity from the Lame constants of src/material.c:121-122 */
void sp_iso_D(double E, double nu, double *D) {
  double lam = (E * nu) / ((1 + nu) * (1 - 2 * nu));
  double mu = E / (2 * (1 + nu));
  for (int i = 0; i < 36; i++) D[i] = 0.0;
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < 3; j++) D[i * 6 + j] = lam;
    D[i * 6 + i] = lam + 2 * mu;
    D[(3 + i) * 6 + (3 + i)] = mu;
  }
}
