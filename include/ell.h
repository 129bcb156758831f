/*
 * ell.h -- drop-in replacement for the reference's inc/ell.h (inc/ell.h:1-42).
 *
 * Same types, same function names and signatures, same return codes.  Link
 * the caller against libsputnik_b200.so instead of ell.o.  The container
 * calls (init / set / add / get / zero / print) run on the host exactly as
 * the reference defines them.  ell_mvp and ell_solve_jacobi run on the GPU
 * with the reference's arithmetic order and return a new code,
 * ELL_ERR_CUDA, when no CUDA device is usable: there is no CPU fallback.
 */
#ifndef ELL_H_
#define ELL_H_

#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#define NRM "\x1B[0m"
#define RED "\x1B[31m"
#define GRN "\x1B[32m"

/* default limits of ell_solve_jacobi (inc/ell.h:12-13) */
#define MAX_ITS 100000
#define MIN_ERR 1.0e-10

/* new return code (the reference uses 0..4) */
#define ELL_ERR_CUDA 5

#ifdef __cplusplus
extern "C" {
#endif

/* fixed-width row-major ELL: slot j of row i at [i*nnz + j]; cols == -1
 * marks an empty slot (inc/ell.h:15-21) */
typedef struct ell_matrix_ {
  int nrow;
  int ncol;
  int nnz;
  int *cols;
  double *vals;
} ell_matrix;

/* inc/ell.h:23-28 */
typedef struct ell_solver_ {
  int max_its;
  int its;
  double min_err;
  double err;
} ell_solver;

/* replaces src/ell.c:3-15 (ell_init) */
int ell_init(ell_matrix *m, int nrow, int ncol, int nnz);
/* replaces src/ell.c:17-44 */
int ell_set_val(ell_matrix *m, int row, int col, double val);
/* replaces src/ell.c:46-73 (first-touch insert, accumulate on repeat) */
int ell_add_val(ell_matrix *m, int row, int col, double val);
/* replaces src/ell.c:75-84 (vals indexed [i*nx + j]) */
int ell_add_vals(ell_matrix *m, int *ix, int nx, int *iy, int ny, double *vals);
/* replaces src/ell.c:127-141: y = m*x on the GPU, bit-identical to the
 * reference's per-row slot-order sum */
int ell_mvp(ell_matrix *m, double *x, double *y);
/* replaces src/ell.c:186-208 */
int ell_get_val(ell_matrix *m, int row, int col, double *val);
/* replaces src/ell.c:143-184: stationary Jacobi on the GPU, same iteration,
 * same absolute tolerance MIN_ERR and limit MAX_ITS; x is the initial guess
 * on entry */
int ell_solve_jacobi(ell_solver *solver, ell_matrix *m, double *b, double *x);
/* replaces src/ell.c:86-101 */
int ell_set_zero_row(ell_matrix *m, int row, double diag_val);
/* replaces src/ell.c:103-118, including its return at the first empty slot
 * of any row; ell_set_zero_col_full (sputnik_b200.h) clears every row */
int ell_set_zero_col(ell_matrix *m, int col, double diag_val);
/* replaces src/ell.c:120-124 */
int ell_set_zero_mat(ell_matrix *m);
/* replaces src/ell.c:210-221 */
int ell_print_full(ell_matrix *m);

#ifdef __cplusplus
}
#endif

#endif
