/*
 * fem.h -- drop-in replacement for the reference's inc/fem.h (inc/fem.h:1-50).
 *
 * Same functions and the same global table names.  The reference header
 * *defines* the table globals (inc/fem.h:19-47), which gcc >= 10 rejects at
 * link time without -fcommon; here they are declared extern and defined once
 * in libsputnik_b200.so.  fem_get_dsh is declared by the reference
 * (inc/fem.h:16) but never defined there, so it is not declared here either.
 * fem_init_struct also fills the 3D (hexa8) case, which the reference leaves
 * empty (src/fem.c:9-14).
 */
#ifndef FEM_H
#define FEM_H

#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#ifdef __cplusplus
extern "C" {
#endif

/* replaces src/fem.c:61-408: allocates and fills every element table */
int fem_init(void);
/* replaces src/fem.c:3-59: structured-grid shape functions, physical
 * derivatives dsh[node][dim][gp] = dN/dxi * 2/h and weights vol/ngp */
int fem_init_struct(double ***sh, double ****dsh, double **wp, double *h, int dim);
/* replaces src/fem.c:426-457 */
int fem_invjac(int dim, double **jac, double **ijac, double *det);
/* replaces src/fem.c:411-424 */
int fem_calc_jac(int dim, int npe, int gp, double *coor, double ***dsh, double **jac);
/* replaces src/fem.c:459-471 */
int fem_trans_dsh(int dim, int nsh, int gp, double **ijac, double ***dsh_master, double ***dsh);
/* replaces src/fem.c:474-520 */
int fem_get_dsh_master(int npe, int dim, double ****dsh);
/* replaces src/fem.c:523-569 */
int fem_get_sh(int npe, int dim, double ***sh);
/* replaces src/fem.c:572-620 */
int fem_get_wp(int npe, int dim, double **wp);

/* tables filled by fem_init: xp[gp][dim], wp[gp], sh[node][gp],
 * ds[node][dim][gp] (inc/fem.h:19-47) */
extern double **xp_segm_2;
extern double *wp_segm_2;
extern double **sh_segm_2;
extern double ***ds_segm_2;

extern double **xp_tria_3;
extern double *wp_tria_3;
extern double **sh_tria_3;
extern double ***ds_tria_3;

extern double **xp_quad_4;
extern double *wp_quad_4;
extern double **sh_quad_4;
extern double ***ds_quad_4;

extern double **xp_tetra_4;
extern double *wp_tetra_4;
extern double **sh_tetra_4;
extern double ***ds_tetra_4;

extern double **xp_prism_6;
extern double *wp_prism_6;
extern double **sh_prism_6;
extern double ***ds_prism_6;

extern double **xp_hexa_8;
extern double *wp_hexa_8;
extern double **sh_hexa_8;
extern double ***ds_hexa_8;

#ifdef __cplusplus
}
#endif

#endif
