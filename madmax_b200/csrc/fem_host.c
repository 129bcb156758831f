/*
 * fem_host.c -- the drop-in fem.h: element tables, structured-grid shape
 * derivatives and Jacobian helpers (src/fem.c).  Host code: these are
 * set-up tables, computed once.  The Gauss points and weights are the
 * reference's literal values (src/fem.c:104-362), and every table entry is
 * computed with the same operations in the same order, so the tables are
 * bit-identical to the reference's.  Layouts as in the reference:
 * xp[gp][dim], wp[gp], sh[node][gp], ds[node][dim][gp].
 */
#include <stdlib.h>

#include "fem.h"

double **xp_segm_2, *wp_segm_2, **sh_segm_2, ***ds_segm_2;
double **xp_tria_3, *wp_tria_3, **sh_tria_3, ***ds_tria_3;
double **xp_quad_4, *wp_quad_4, **sh_quad_4, ***ds_quad_4;
double **xp_tetra_4, *wp_tetra_4, **sh_tetra_4, ***ds_tetra_4;
double **xp_prism_6, *wp_prism_6, **sh_prism_6, ***ds_prism_6;
double **xp_hexa_8, *wp_hexa_8, **sh_hexa_8, ***ds_hexa_8;

#define G2 0.577350269189626 /* 1/sqrt(3) as written in src/fem.c */
#define T1 0.166666666666666
#define T2 0.666666666666666
#define TA 0.138196601125011
#define TB 0.585410196624968

/* allocate one element family: xp[ngp][dim], wp[ngp], sh[npe][ngp],
 * ds[npe][dim][ngp], zero-filled */
static int alloc_family(int npe, int dim, int ngp, double ***xp, double **wp, double ***sh,
                        double ****ds) {
  *xp = (double **)calloc(ngp, sizeof(double *));
  *wp = (double *)calloc(ngp, sizeof(double));
  *sh = (double **)calloc(npe, sizeof(double *));
  *ds = (double ***)calloc(npe, sizeof(double **));
  if (!*xp || !*wp || !*sh || !*ds) return 1;
  for (int g = 0; g < ngp; g++)
    if (!((*xp)[g] = (double *)calloc(dim, sizeof(double)))) return 1;
  for (int a = 0; a < npe; a++) {
    (*sh)[a] = (double *)calloc(ngp, sizeof(double));
    (*ds)[a] = (double **)calloc(dim, sizeof(double *));
    if (!(*sh)[a] || !(*ds)[a]) return 1;
    for (int d = 0; d < dim; d++)
      if (!((*ds)[a][d] = (double *)calloc(ngp, sizeof(double)))) return 1;
  }
  return 0;
}

/* tensor-product families (segm2, quad4, hexa8): node a sits at corner
 * sign s[a][d] = -1/+1; N_a = prod_d (1 + s x_d) * 2^-dim, and dN_a/dx_d is
 * the same product with factor d replaced by s[a][d] * 1.0 */
static void fill_tensor(int npe, int dim, int ngp, const int (*s)[3], double scale, double **xp,
                        double **sh, double ***ds) {
  for (int g = 0; g < ngp; g++) {
    for (int a = 0; a < npe; a++) {
      double f[3];
      for (int d = 0; d < dim; d++) f[d] = (s[a][d] < 0) ? (1.0 - xp[g][d]) : (1.0 + xp[g][d]);
      double n = f[0];
      for (int d = 1; d < dim; d++) n = n * f[d];
      sh[a][g] = n * scale;
      for (int d = 0; d < dim; d++) {
        double v = s[a][d] * 1.0;
        for (int e = 0; e < dim; e++)
          if (e != d) v = v * f[e];
        ds[a][d][g] = v * scale;
      }
    }
  }
}

static const int SGN1[2][3] = {{-1, 0, 0}, {+1, 0, 0}};
static const int SGN2[4][3] = {{-1, -1, 0}, {+1, -1, 0}, {+1, +1, 0}, {-1, +1, 0}};
static const int SGN3[8][3] = {{-1, -1, -1}, {+1, -1, -1}, {+1, +1, -1}, {-1, +1, -1},
                               {-1, -1, +1}, {+1, -1, +1}, {+1, +1, +1}, {-1, +1, +1}};

/* src/fem.c:61-408 */
int fem_init(void) {
  /* segm2: src/fem.c:63-87 */
  if (alloc_family(2, 1, 2, &xp_segm_2, &wp_segm_2, &sh_segm_2, &ds_segm_2)) return 1;
  for (int g = 0; g < 2; g++) {
    xp_segm_2[g][0] = (g == 0) ? -G2 : +G2;
    wp_segm_2[g] = +1.0;
    sh_segm_2[0][g] = +0.5 * (1.0 - xp_segm_2[g][0]);
    sh_segm_2[1][g] = +0.5 * (1.0 + xp_segm_2[g][0]);
    ds_segm_2[0][0][g] = -0.5;
    ds_segm_2[1][0][g] = +0.5;
  }

  /* tria3: src/fem.c:89-130 */
  if (alloc_family(3, 2, 3, &xp_tria_3, &wp_tria_3, &sh_tria_3, &ds_tria_3)) return 1;
  {
    static const double p[3][2] = {{T1, T1}, {T2, T1}, {T1, T2}};
    for (int g = 0; g < 3; g++) {
      xp_tria_3[g][0] = p[g][0];
      xp_tria_3[g][1] = p[g][1];
      wp_tria_3[g] = 1 / 6.0;
      sh_tria_3[0][g] = +1.0 - xp_tria_3[g][0] - xp_tria_3[g][1];
      sh_tria_3[1][g] = +xp_tria_3[g][0];
      sh_tria_3[2][g] = +xp_tria_3[g][1];
      ds_tria_3[0][0][g] = -1.0; ds_tria_3[0][1][g] = -1.0;
      ds_tria_3[1][0][g] = +1.0; ds_tria_3[1][1][g] = +0.0;
      ds_tria_3[2][0][g] = +0.0; ds_tria_3[2][1][g] = +1.0;
    }
  }

  /* quad4: src/fem.c:132-170 */
  if (alloc_family(4, 2, 4, &xp_quad_4, &wp_quad_4, &sh_quad_4, &ds_quad_4)) return 1;
  for (int g = 0; g < 4; g++) {
    xp_quad_4[g][0] = SGN2[g][0] * G2;
    xp_quad_4[g][1] = SGN2[g][1] * G2;
    wp_quad_4[g] = 1.0;
  }
  fill_tensor(4, 2, 4, SGN2, 0.25, xp_quad_4, sh_quad_4, ds_quad_4);

  /* tetra4: src/fem.c:173-229 */
  if (alloc_family(4, 3, 4, &xp_tetra_4, &wp_tetra_4, &sh_tetra_4, &ds_tetra_4)) return 1;
  for (int g = 0; g < 4; g++) {
    for (int d = 0; d < 3; d++) xp_tetra_4[g][d] = (g == d + 1) ? +TB : +TA;
    wp_tetra_4[g] = +0.041666666666666;
    sh_tetra_4[0][g] = 1.0 - xp_tetra_4[g][0] - xp_tetra_4[g][1] - xp_tetra_4[g][2];
    for (int a = 1; a < 4; a++) sh_tetra_4[a][g] = xp_tetra_4[g][a - 1];
    for (int d = 0; d < 3; d++) {
      ds_tetra_4[0][d][g] = -1.0;
      for (int a = 1; a < 4; a++) ds_tetra_4[a][d][g] = (a - 1 == d) ? +1.0 : +0.0;
    }
  }

  /* prism6: src/fem.c:232-307 (triangle x [-1,1], two Gauss levels) */
  if (alloc_family(6, 3, 6, &xp_prism_6, &wp_prism_6, &sh_prism_6, &ds_prism_6)) return 1;
  {
    static const double p[3][2] = {{T1, T1}, {T2, T1}, {T1, T2}};
    for (int g = 0; g < 6; g++) {
      xp_prism_6[g][0] = p[g % 3][0];
      xp_prism_6[g][1] = p[g % 3][1];
      xp_prism_6[g][2] = (g < 3) ? -G2 : +G2;
      wp_prism_6[g] = +0.166666666666666;
    }
    for (int g = 0; g < 6; g++) {
      double x = xp_prism_6[g][0], y = xp_prism_6[g][1], z = xp_prism_6[g][2];
      for (int top = 0; top < 2; top++) {
        double fz = top ? (1.0 + z) : (1.0 - z);
        double sz = top ? +1.0 : -1.0;
        int a0 = 3 * top;
        sh_prism_6[a0 + 0][g] = (1.0 - x - y) * fz * 0.5;
        ds_prism_6[a0 + 0][0][g] = -1.0 * fz * 0.5;
        ds_prism_6[a0 + 0][1][g] = -1.0 * fz * 0.5;
        ds_prism_6[a0 + 0][2][g] = sz * (1.0 - x - y) * 0.5;
        sh_prism_6[a0 + 1][g] = x * fz * 0.5;
        ds_prism_6[a0 + 1][0][g] = +1.0 * fz * 0.5;
        ds_prism_6[a0 + 1][1][g] = +0.0;
        ds_prism_6[a0 + 1][2][g] = sz * x * 0.5;
        sh_prism_6[a0 + 2][g] = y * fz * 0.5;
        ds_prism_6[a0 + 2][0][g] = +0.0;
        ds_prism_6[a0 + 2][1][g] = +1.0 * fz * 0.5;
        ds_prism_6[a0 + 2][2][g] = sz * y * 0.5;
      }
    }
  }

  /* hexa8: src/fem.c:309-405 */
  if (alloc_family(8, 3, 8, &xp_hexa_8, &wp_hexa_8, &sh_hexa_8, &ds_hexa_8)) return 1;
  for (int g = 0; g < 8; g++) {
    for (int d = 0; d < 3; d++) xp_hexa_8[g][d] = SGN3[g][d] * G2;
    wp_hexa_8[g] = +1.0;
  }
  fill_tensor(8, 3, 8, SGN3, 0.125, xp_hexa_8, sh_hexa_8, ds_hexa_8);
  (void)SGN1;
  return 0;
}

/* src/fem.c:3-59.  dsh[node][dim][gp] = dN/dxi * 2/h, wp[gp] = vol/ngp.
 * The 3D case, empty in the reference, uses the hexa8 Gauss points. */
int fem_init_struct(double ***sh, double ****dsh, double **wp, double *h, int dim) {
  if (dim != 2 && dim != 3) return 1;
  int npe = (dim == 2) ? 4 : 8, ngp = npe;
  double **xp, *w0, **s, ***ds;
  if (alloc_family(npe, dim, ngp, &xp, &w0, &s, &ds)) return 2;
  for (int g = 0; g < ngp; g++)
    for (int d = 0; d < dim; d++) xp[g][d] = ((dim == 2) ? SGN2[g][d] : SGN3[g][d]) * G2;
  if (dim == 2) {
    /* the reference's own 2D operation order: -1*(1-eta)/4*2/hx ... */
    for (int g = 0; g < 4; g++) {
      double x = xp[g][0], y = xp[g][1];
      s[0][g] = (1 - x) * (1 - y) / 4;
      s[1][g] = (1 + x) * (1 - y) / 4;
      s[2][g] = (1 + x) * (1 + y) / 4;
      s[3][g] = (1 - x) * (1 + y) / 4;
      ds[0][0][g] = -1 * (1 - y) / 4 * 2 / h[0];
      ds[1][0][g] = +1 * (1 - y) / 4 * 2 / h[0];
      ds[2][0][g] = +1 * (1 + y) / 4 * 2 / h[0];
      ds[3][0][g] = -1 * (1 + y) / 4 * 2 / h[0];
      ds[0][1][g] = -1 * (1 - x) / 4 * 2 / h[1];
      ds[1][1][g] = -1 * (1 + x) / 4 * 2 / h[1];
      ds[2][1][g] = +1 * (1 + x) / 4 * 2 / h[1];
      ds[3][1][g] = +1 * (1 - x) / 4 * 2 / h[1];
    }
  } else {
    fill_tensor(8, 3, 8, SGN3, 0.125, xp, s, ds);
    for (int a = 0; a < 8; a++)
      for (int d = 0; d < 3; d++)
        for (int g = 0; g < 8; g++) ds[a][d][g] = ds[a][d][g] * 2 / h[d];
  }
  double vol = h[0] * h[1] * ((dim == 3) ? h[2] : 1.0);
  for (int g = 0; g < ngp; g++) w0[g] = vol / ngp;
  for (int g = 0; g < ngp; g++) free(xp[g]);
  free(xp);
  *sh = s;
  *dsh = ds;
  *wp = w0;
  return 0;
}

/* src/fem.c:411-424: jac[i][j] = sum_n dsh[n][i][gp] coor[n*dim + j] */
int fem_calc_jac(int dim, int npe, int gp, double *coor, double ***dsh, double **jac) {
  if (jac == NULL || coor == NULL || dsh == NULL) return 1;
  for (int i = 0; i < dim; i++)
    for (int j = 0; j < dim; j++) {
      double s = 0.0;
      for (int n = 0; n < npe; n++) s += dsh[n][i][gp] * coor[n * dim + j];
      jac[i][j] = s;
    }
  return 0;
}

/* src/fem.c:426-457: cofactor inverse, det by first-row expansion */
int fem_invjac(int dim, double **jac, double **ijac, double *det) {
  if (jac == NULL || ijac == NULL) return 1;
  if (dim == 2) {
    double c00 = +jac[1][1], c01 = -jac[1][0];
    double c10 = -jac[0][1], c11 = +jac[0][0];
    *det = jac[0][0] * c00 + jac[0][1] * c01;
    ijac[0][0] = c00 / *det; ijac[0][1] = c10 / *det;
    ijac[1][0] = c01 / *det; ijac[1][1] = c11 / *det;
  } else if (dim == 3) {
    double c[3][3];
    c[0][0] = +jac[1][1] * jac[2][2] - jac[2][1] * jac[1][2];
    c[0][1] = -jac[1][0] * jac[2][2] + jac[2][0] * jac[1][2];
    c[0][2] = +jac[1][0] * jac[2][1] - jac[2][0] * jac[1][1];
    c[1][0] = -jac[0][1] * jac[2][2] + jac[2][1] * jac[0][2];
    c[1][1] = +jac[0][0] * jac[2][2] - jac[2][0] * jac[0][2];
    c[1][2] = -jac[0][0] * jac[2][1] + jac[2][0] * jac[0][1];
    c[2][0] = +jac[0][1] * jac[1][2] - jac[1][1] * jac[0][2];
    c[2][1] = -jac[0][0] * jac[1][2] + jac[1][0] * jac[0][2];
    c[2][2] = +jac[0][0] * jac[1][1] - jac[1][0] * jac[0][1];
    *det = jac[0][0] * c[0][0] + jac[0][1] * c[0][1] + jac[0][2] * c[0][2];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) ijac[i][j] = c[j][i] / *det;
  }
  return 0;
}

/* src/fem.c:459-471 */
int fem_trans_dsh(int dim, int nsh, int gp, double **ijac, double ***dsh_master, double ***dsh) {
  if (ijac == NULL || dsh_master == NULL || dsh == NULL) return 1;
  for (int a = 0; a < nsh; a++)
    for (int i = 0; i < dim; i++) {
      double s = 0.0;
      for (int j = 0; j < dim; j++) s += ijac[i][j] * dsh_master[a][j][gp];
      dsh[a][i][gp] = s;
    }
  return 0;
}

/* src/fem.c:473-620: table lookup by (npe, dim) */
static int family(int npe, int dim) {
  if (dim == 2 && npe == 3) return 1;
  if (dim == 2 && npe == 4) return 2;
  if (dim == 3 && npe == 4) return 3;
  if (dim == 3 && npe == 6) return 4;
  if (dim == 3 && npe == 8) return 5;
  return 0;
}

int fem_get_dsh_master(int npe, int dim, double ****dsh) {
  double ***t[6] = {NULL, ds_tria_3, ds_quad_4, ds_tetra_4, ds_prism_6, ds_hexa_8};
  int f = family(npe, dim);
  if (!f) return 1;
  *dsh = t[f];
  return 0;
}

int fem_get_sh(int npe, int dim, double ***sh) {
  double **t[6] = {NULL, sh_tria_3, sh_quad_4, sh_tetra_4, sh_prism_6, sh_hexa_8};
  int f = family(npe, dim);
  if (!f) return 1;
  *sh = t[f];
  return 0;
}

int fem_get_wp(int npe, int dim, double **wp) {
  double *t[6] = {NULL, wp_tria_3, wp_quad_4, wp_tetra_4, wp_prism_6, wp_hexa_8};
  int f = family(npe, dim);
  if (!f) return 1;
  *wp = t[f];
  return 0;
}
