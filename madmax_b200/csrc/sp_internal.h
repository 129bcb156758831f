/*
 * sp_internal.h -- declarations shared by the C and CUDA translation units
 * of libsputnik_b200.so.  Not installed; the public ABI is the headers in
 * include/.
 */
#ifndef SP_INTERNAL_H
#define SP_INTERNAL_H

#include <stddef.h>
#include <stdint.h>

#include "sputnik_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* device row width: 81 reference slots padded to 84 so that every row of
 * FP32 (336 B) and FP64 (672 B) values starts on a 16-byte boundary */
#define SP_WP 84
#define SP_NC 24   /* hexa8 element dofs */
#define SP_KE 576  /* SP_NC * SP_NC */

/* thread-local last error; returns code */
int sp_set_error(int code, const char *fmt, ...);

/* return a non-zero code from C host code */
#define SP_TRY_C(x)        \
  do {                     \
    int sp_rc_ = (x);      \
    if (sp_rc_) return sp_rc_; \
  } while (0)

/* Structured 3D mesh plan, shared by every RVE of the same mesh. */
typedef struct {
  int n[3];            /* elements per axis */
  int nx, ny, nz;      /* nodes per axis */
  int nn, ndof, nelm;
  int boundary_nodes;
  int color_off[9];    /* elements of colour c: color_elems[color_off[c] .. color_off[c+1]) */
  int nn_pad, nslice;  /* nodes rounded up to 32, slices of 32 nodes */
  int *cols;           /* host [ndof][SP_WP], first-touch order, -1 padded */
  int *nbr;            /* host [nslice][27][32]: neighbour node of group m (see plan.c) */
  uint8_t *slot;       /* host [nelm][576]: slot (within the row) of Ke entry (i, j) */
  int *color_elems;    /* host [nelm] */
} sp_plan_host;

int sp_plan_build(const int *n, sp_plan_host *p);
void sp_plan_free(sp_plan_host *p);

/* the classification arithmetic of micro/src/micro_struct.c:98-129 */
int sp_classify_elements(const sp_rve_desc *d, uint8_t *etype, int *nfiber);

/* isotropic elastic D (Voigt xx,yy,zz,xy,yz,xz) from E, nu */
void sp_iso_D(double E, double nu, double *D);

#ifdef __cplusplus
}
#endif

#endif
