/*
 * oracle.h -- CPU restatement of the sputnik micro-RVE homogenization path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference arm of bench.py may load this library, and only as
 * the checker or the timed CPU baseline.  The product library never links it.
 *
 * What it restates (reference paths are relative to the reference project):
 *   - structured mesh numbering ............ src/mesh.c:762-902 (2D) -> 3D
 *   - fiber_cilin element classification ... micro/src/micro_struct.c:98-129,
 *                                            micro/src/homogenize.c:487-494
 *   - hexa8 / quad4 tables ................. src/fem.c:3-59, 309-405
 *   - B matrix ............................. micro/src/init.c:40-51 (2D) -> 3D
 *   - isotropic elastic D .................. src/material.c:4-59, 121-122
 *   - ELL container + first-touch insert ... src/ell.c:3-221
 *   - Jacobian assembly + Dirichlet BC ..... micro/src/assembly.c:84-137
 *   - residual assembly .................... micro/src/assembly.c:33-82
 *   - affine boundary displacement ......... micro/src/homogenize.c:227-242, 335-342
 *   - Newton / solve / add_x_dx ............ micro/src/homogenize.c:175-225, 289-333
 *   - volume averages ...................... micro/src/homogenize.c:344-368
 *   - finite-difference tangent ............ micro/src/homogenize.c:59-94
 *   - Jacobi-preconditioned CG ............. PETSc KSPCG + PCJACOBI (third-party,
 *                                            not in the reference tree; restated
 *                                            from the published algorithm)
 *
 * Parity pins: the ELL container, insertion order, SpMV and stationary Jacobi
 * are checked bit-for-bit against the reference's own src/ell.c compiled from
 * its sources (oracle/_ref), and against unity/unity_ell.c's output.  The 2D
 * homogenized tensor is checked loosely against exs/README.md:154-157.  The
 * PETSc CG step has no reference code here: parity for it is unpinned and
 * rests on the direct residual check ||b - A x|| / ||b||.
 */
#ifndef SPUTNIK_ORACLE_H
#define SPUTNIK_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_ID_MATRIX 0
#define ORC_ID_FIBER 1

typedef struct {
  int dim;             /* 2 or 3 */
  int nx, ny, nz;      /* node counts per axis (nz = 1 in 2D) */
  int nex, ney, nez;   /* element counts per axis (nez = 1 in 2D) */
  int nelm, nn, npe;   /* elements, nodes, nodes per element */
  int nvoi, ngp, ndof; /* Voigt size, Gauss points, dofs = nn*dim */
  double lx, ly, lz, hx, hy, hz, vol, vol_elm;
} orc_mesh;

typedef struct {
  int nrow, ncol, nnz; /* nnz = fixed row width, as in the reference */
  int *cols;
  double *vals;
} orc_ell;

/* mesh */
int orc_mesh_init(orc_mesh *m, int dim, const int *n_nodes, const double *len);
void orc_node_coord(const orc_mesh *m, int node, double *x);
void orc_elem_nodes(const orc_mesh *m, int e, int *nods);
void orc_elem_dofs(const orc_mesh *m, int e, int *idx);
int orc_is_boundary_node(const orc_mesh *m, int node);
int orc_boundary_nodes(const orc_mesh *m, int *nodes); /* ascending; returns count */
void orc_elem_centroid(const orc_mesh *m, int e, double *c);

/* micro-structure: fiber_cilin (z-aligned cylinders in 3D) */
int orc_fiber_cilin_types(const orc_mesh *m, const double *size, int nx_fib, int ny_fib,
                          double radio, const double *desv, unsigned char *elem_type);

/* fem tables and operators */
void orc_hexa8_tables(double *xp /*[8][3]*/, double *sh /*[8][8]*/, double *ds /*[8][3][8]*/);
void orc_struct_dsh(const orc_mesh *m, double *dsh /*[npe][dim][ngp]*/, double *wp /*[ngp]*/);
void orc_bmat(const orc_mesh *m, const double *dsh, double *bmat /*[nvoi][npe*dim][ngp]*/);
void orc_iso_D(int dim, double E, double nu, double *D /*[nvoi*nvoi]*/);
void orc_elem_stiffness(const orc_mesh *m, const double *bmat, const double *wp, const double *D,
                        double *Ke /*[(npe*dim)^2]*/);

/* ELL container (restated semantics of src/ell.c) */
int orc_ell_init(orc_ell *a, int nrow, int ncol, int nnz);
void orc_ell_free(orc_ell *a);
int orc_ell_add_val(orc_ell *a, int row, int col, double val);
int orc_ell_add_vals(orc_ell *a, const int *ix, int nx, const int *iy, int ny, const double *vals);
int orc_ell_get_val(const orc_ell *a, int row, int col, double *val);
int orc_ell_mvp(const orc_ell *a, const double *x, double *y);
int orc_ell_set_zero_row(orc_ell *a, int row, double diag);
int orc_ell_set_zero_col_ref(orc_ell *a, int col, double diag);  /* reference semantics */
int orc_ell_set_zero_col_full(orc_ell *a, int col, double diag); /* every row */
int orc_ell_set_zero_mat(orc_ell *a);

/* assembly */
int orc_assemble_jac(const orc_mesh *m, const unsigned char *etype, const double *Ke_by_type,
                     orc_ell *A, int symmetric_bc);
int orc_assemble_res(const orc_mesh *m, const unsigned char *etype, const double *D_by_type,
                     const double *bmat, const double *wp, const double *u, double *res,
                     double *norm);
void orc_affine_bc(const orc_mesh *m, const double *strain, double *u);
void orc_averages(const orc_mesh *m, const unsigned char *etype, const double *D_by_type,
                  const double *bmat, const double *wp, const double *u, double *strain_ave,
                  double *stress_ave);

/* solvers */
int orc_jacobi(const orc_ell *A, const double *b, double *x, int max_its, double min_err, int *its,
               double *err);
int orc_pcg(const orc_ell *A, const double *b, double *x, double rtol, int max_its, int *its,
            double *relres);

/* homogenization driver: one RVE, nrhs macro strains (rows of strains[nrhs][nvoi]).
 * solver: 0 = Jacobi-PCG (1e-8 relative style), 1 = reference stationary Jacobi.
 * Outputs stress_ave/strain_ave [nrhs][nvoi]; u_out [nrhs][ndof] if non-null.
 * stats[0..3] per rhs: newton its, total linear its, final true relres, ||r0||. */
typedef struct {
  double E[2], nu[2]; /* [ORC_ID_MATRIX], [ORC_ID_FIBER] */
  double rtol;        /* relative tolerance on ||r(u)||/||r(u0)|| */
  double lin_rtol;    /* linear solver relative tolerance */
  int max_newton;
  int max_lin_its;
  int solver;
} orc_params;

int orc_homogenize(const orc_mesh *m, const unsigned char *etype, const orc_params *p, int nrhs,
                   const double *strains, double *strain_ave, double *stress_ave, double *u_out,
                   double *stats);
/* C[i][j] = <sigma_i>(e_j): 6 (or 3) unit-strain load cases */
int orc_unit_tangent(const orc_mesh *m, const unsigned char *etype, const orc_params *p,
                     double *C, double *stats);
/* finite-difference tangent around strain_mac, delta = 0.005 (micro/inc/micro.h:29) */
int orc_fd_tangent(const orc_mesh *m, const unsigned char *etype, const orc_params *p,
                   const double *strain_mac, double *C, double *stress0);

#ifdef __cplusplus
}
#endif
#endif
