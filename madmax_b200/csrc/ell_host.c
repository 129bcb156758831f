/*
 * ell_host.c -- the container half of the drop-in ell.h: the operations the
 * reference runs on the host (src/ell.c) keep their host semantics here, so
 * a caller that owns m->cols / m->vals sees the same memory contents, slot
 * order and return codes.  ell_mvp and ell_solve_jacobi (the compute half)
 * live in ell_gpu.cu.
 */
#include <stdio.h>
#include <stdlib.h>

#include "ell.h"
#include "sp_internal.h"

static int *row_cols(ell_matrix *m, int row) { return m->cols + (size_t)row * m->nnz; }
static double *row_vals(ell_matrix *m, int row) { return m->vals + (size_t)row * m->nnz; }

/* src/ell.c:3-15: caller owns the struct, the arrays are malloc'd here */
int ell_init(ell_matrix *m, int nrow, int ncol, int nnz) {
  if (m == NULL) return 1;
  m->nnz = nnz;
  m->nrow = nrow;
  m->ncol = ncol;
  size_t n = (size_t)nrow * (size_t)nnz;
  m->cols = (int *)malloc(n * sizeof(int));
  m->vals = (double *)malloc(n * sizeof(double));
  if (m->cols == NULL || m->vals == NULL) return 2;
  for (size_t i = 0; i < n; i++) {
    m->cols[i] = -1;
    m->vals[i] = 0.0;
  }
  return 0;
}

int ell_free(ell_matrix *m) {
  if (m == NULL) return 1;
  free(m->cols);
  free(m->vals);
  m->cols = NULL;
  m->vals = NULL;
  return 0;
}

/* Shared by set/add: index checks with the reference's messages and codes,
 * then a scan for `col` or the first empty slot.  Returns the slot, or a
 * negative error (-1 range, -2 negative, -3 full). */
static int find_slot(ell_matrix *m, int row, int col, const char *what) {
  if (row >= m->nrow || col >= m->ncol) {
    printf(RED "ell error: row %d or col %d greater than the dimension of the matrix\n" NRM, row,
           col);
    return -1;
  }
  if (row < 0 || col < 0) {
    printf(RED "ell error: negative values in row %d or col %d\n" NRM, row, col);
    return -2;
  }
  int *c = row_cols(m, row);
  for (int j = 0; j < m->nnz; j++)
    if (c[j] == -1 || c[j] == col) return j;
  printf(RED "ell error: not enought space to %s value in row %d and col %d\n" NRM, what, row, col);
  return -3;
}

/* src/ell.c:17-44 */
int ell_set_val(ell_matrix *m, int row, int col, double val) {
  int j = find_slot(m, row, col, "store");
  if (j < 0) return -j;
  row_cols(m, row)[j] = col;
  row_vals(m, row)[j] = val;
  return 0;
}

/* src/ell.c:46-73 */
int ell_add_val(ell_matrix *m, int row, int col, double val) {
  int j = find_slot(m, row, col, "add");
  if (j < 0) return -j;
  int *c = row_cols(m, row);
  double *v = row_vals(m, row);
  if (c[j] == -1) {
    c[j] = col;
    v[j] = val;
  } else {
    v[j] += val;
  }
  return 0;
}

/* src/ell.c:75-84 */
int ell_add_vals(ell_matrix *m, int *ix, int nx, int *iy, int ny, double *vals) {
  if (m == NULL || ix == NULL || iy == NULL || vals == NULL) return 1;
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++) ell_add_val(m, ix[i], iy[j], vals[i * nx + j]);
  return 0;
}

/* src/ell.c:86-101 */
int ell_set_zero_row(ell_matrix *m, int row, double diag_val) {
  if (m == NULL) return 1;
  int *c = row_cols(m, row);
  double *v = row_vals(m, row);
  for (int j = 0; j < m->nnz && c[j] != -1; j++) v[j] = (c[j] == row) ? diag_val : 0.0;
  return 0;
}

/* src/ell.c:103-118.  Kept as the reference behaves: the scan over rows
 * ends at the first empty slot met in any row. */
int ell_set_zero_col(ell_matrix *m, int col, double diag_val) {
  if (m == NULL) return 1;
  for (int i = 0; i < m->nrow; i++) {
    int *c = row_cols(m, i);
    double *v = row_vals(m, i);
    for (int j = 0; j < m->nnz; j++) {
      if (c[j] == -1) return 0;
      if (c[j] == col) v[j] = (i == col) ? diag_val : 0.0;
    }
  }
  return 0;
}

int ell_set_zero_col_full(ell_matrix *m, int col, double diag_val) {
  if (m == NULL) return 1;
  for (int i = 0; i < m->nrow; i++) {
    int *c = row_cols(m, i);
    double *v = row_vals(m, i);
    for (int j = 0; j < m->nnz && c[j] != -1; j++)
      if (c[j] == col) v[j] = (i == col) ? diag_val : 0.0;
  }
  return 0;
}

/* src/ell.c:120-124 */
int ell_set_zero_mat(ell_matrix *m) {
  if (m == NULL) return 1;
  for (int i = 0; i < m->nrow; i++) ell_set_zero_row(m, i, 0.0);
  return 0;
}

/* src/ell.c:186-208 */
int ell_get_val(ell_matrix *m, int row, int col, double *val) {
  if (row >= m->nrow || col >= m->ncol) {
    printf(RED "ell_get_val: row %d or col %d greater than the dimension of the matrix\n" NRM, row,
           col);
    return 1;
  }
  if (row < 0 || col < 0) {
    printf(RED "ell_get_val: negative values in row %d or col %d\n" NRM, row, col);
    return 2;
  }
  int *c = row_cols(m, row);
  for (int j = 0; j < m->nnz; j++) {
    if (c[j] == -1) {
      *val = 0.0;
      return 0;
    }
    if (c[j] == col) {
      *val = row_vals(m, row)[j];
      return 0;
    }
  }
  return 3;
}

/* src/ell.c:210-221 */
int ell_print_full(ell_matrix *m) {
  if (m == NULL) return 1;
  if (m->vals == NULL || m->cols == NULL) return 2;
  for (int i = 0; i < m->nrow; i++) {
    for (int j = 0; j < m->ncol; j++) {
      double v;
      int rc = ell_get_val(m, i, j, &v);
      printf("%lf%s", rc == 0 ? v : 0.0, (j == m->ncol - 1) ? "\n" : " ");
    }
  }
  return 0;
}
