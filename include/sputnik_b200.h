/*
 * sputnik_b200.h -- handle-based C ABI of libsputnik_b200.so, the B200
 * (sm_100a) implementation of the sputnik micro-RVE homogenization path.
 *
 * These entry points have no one-to-one counterpart in the reference: they
 * replace the micro program's homogenization driver (micro/src/homogenize.c,
 * micro/src/assembly.c, micro/src/init.c, micro/src/alloc.c) and its MPI
 * request loop (micro/src/main.c:114-153, inc/comm.h:18-27) with library
 * calls that keep matrices, solutions and work queues on the GPU.  Each
 * declaration names the reference code it stands in for.
 *
 * Conventions (as in the reference): every function returns int, 0 on
 * success, a small positive code on failure; the message of the last failure
 * on the calling thread is in sp_last_error().  No function aborts, traps or
 * falls back to the CPU: without a usable CUDA device the compute calls
 * return SP_ERR_CUDA.
 *
 * 3D conventions: node (i,j,k) -> i + j*nx + k*nx*ny, dof = 3*node + d;
 * hexa8 local node order of the reference's src/fem.c:324-362; Voigt order
 * (xx, yy, zz, xy, yz, xz) with engineering shear strains.
 */
#ifndef SPUTNIK_B200_H
#define SPUTNIK_B200_H

#include <stddef.h>

#include "ell.h"

#ifdef __cplusplus
extern "C" {
#endif

#define SP_OK 0
#define SP_ERR_ARG 1     /* bad argument or unsupported size */
#define SP_ERR_NOMEM 2   /* host or device allocation failed */
#define SP_ERR_RANGE 3   /* index outside the object */
#define SP_ERR_CUDA 5    /* no usable device or a CUDA call failed */
#define SP_ERR_NOCONV 6  /* a solve stopped at its iteration limit */
#define SP_ERR_BUDGET 7  /* request exceeds the HBM admission budget */
#define SP_ERR_TIMEOUT 8 /* a bounded device wait gave up */
#define SP_ERR_STATE 9   /* call not valid in the object's state */
#define SP_PENDING 10    /* sp_server_poll: result not ready yet */

#define SP_ID_MATRIX 0 /* micro/inc/micro_struct.h:13 */
#define SP_ID_FIBER 1  /* micro/inc/micro_struct.h:14 */

#define SP_MAX_RHS 8
#define SP_ELL_WIDTH 81 /* 3D ELL row width, micro/src/alloc.c:6 */

const char *sp_last_error(void);
int sp_version(void);
/* Select the CUDA device used by this thread's later calls (default 0). */
int sp_init(int device);
/* Number of usable CUDA devices (0 without a driver or GPU; never fails). */
int sp_device_count(void);

/* ------------------------------------------------------------- ELL extras */

/* src/ell.c:103-118 with the column cleared in every row (the reference
 * stops at the first empty slot of any row).  Host operation. */
int ell_set_zero_col_full(ell_matrix *m, int col, double diag_val);
/* Frees what ell_init allocated (the reference has no free). */
int ell_free(ell_matrix *m);

/* A copy of an ell_matrix resident on the GPU (rows padded to 84 slots). */
typedef struct sp_ell_dev_s sp_ell_dev;
int sp_ell_upload(const ell_matrix *m, sp_ell_dev **out);
int sp_ell_dev_free(sp_ell_dev *a);
/* y = A x with device pointers on `stream` (cudaStream_t, NULL = library
 * stream): one warp per row, 128-bit loads.  Result within rounding of the
 * reference's ell_mvp (src/ell.c:127-141). */
int sp_ell_dev_mvp(sp_ell_dev *a, const double *x_dev, double *y_dev, void *stream);
/* Same with host vectors (copies in and out). */
int sp_ell_dev_mvp_host(sp_ell_dev *a, const double *x, double *y);
/* Lanes per row of sp_ell_dev_mvp: 4, 8, 16 or 32 (0: the autotuner's
 * choice).  For 84-slot (RVE-shaped) rows, sp_ell_upload times every width
 * on the uploaded matrix and keeps the fastest (cached per device, row width
 * and row-count octave).  A tuning knob; the result does not depend on it
 * beyond rounding. */
int sp_ell_dev_set_lanes(sp_ell_dev *a, int lanes);
/* The lanes per row sp_ell_dev_mvp uses, the upload-time trial's time per
 * launch at 4, 8, 16 and 32 lanes (microseconds; trial_us may be NULL) and
 * whether the choice came from the autotuner's cache.  No counterpart in the
 * reference (its ell_mvp is a serial row loop, src/ell.c:127-141). */
int sp_ell_dev_lanes(const sp_ell_dev *a, int *lanes, float *trial_us, int *from_cache);
/* Rows, padded row width and stored (non-empty) slots of a device matrix. */
int sp_ell_dev_info(const sp_ell_dev *a, int *nrow, int *wp, long long *true_nnz);
/* Jacobi-preconditioned CG in FP64 on host vectors: the ELL path of the
 * reference's solve() (micro/src/homogenize.c:320-333) with PETSc's
 * KSPCG + PCJACOBI algorithm; stops at ||b - A x|| <= rtol ||b||.  x holds
 * the initial guess on entry. */
int sp_ell_dev_pcg(sp_ell_dev *a, const double *b, double *x, double rtol, int max_its,
                   int *its, double *relres);

/* Jacobi-preconditioned CG (the algorithm of sp_ell_dev_pcg) on an ELL
 * matrix the caller already holds in device memory, allocating nothing.
 * No counterpart in the reference: it is for callers that cannot allocate
 * device memory -- frameworks that own all device memory through their own
 * pool and forbid other allocations, and latency-bound loops that must stay
 * out of the CUDA allocator (whose calls synchronize the device).
 * cols_dev/vals_dev: [nrow][nnz] row-major, -1 marks an empty slot (the ell.h
 * layout); b_dev: right-hand side; x_dev: initial guess in, solution out; all
 * device pointers owned by the caller.  Stops at ||b - A x|| <= rtol ||b||.
 * Returns SP_ERR_RANGE for a column index outside [0, nrow) (the entry is
 * skipped, never read), SP_ERR_ARG for a row whose diagonal is zero or
 * absent, SP_ERR_NOCONV when the residual test fails (including a NaN
 * residual).  Work space is a fixed device array of the library (about
 * 8.4 MB per GPU, held until exit): nrow <= SP_NOALLOC_MAX_ROWS, else
 * SP_ERR_ARG.  The first call on a device looks up that array's address
 * (cudaGetSymbolAddress); make it before any stream capture.  Calls share
 * the array and each call resets what must start at zero; calls that
 * overlap on the GPU race, so serialize them.  stream NULL means the
 * per-thread default stream. */
#define SP_NOALLOC_MAX_ROWS 262144
int sp_ell_pcg_noalloc(int nrow, int nnz, const int *cols_dev, const double *vals_dev,
                       const double *b_dev, double *x_dev, double rtol, int max_its, int *its,
                       double *relres, void *stream);

/* --------------------------------------------------------------------- RVE */

/* One structured micro-RVE: mesh (src/mesh.c:762-867 extended to 3D),
 * fiber_cilin micro-structure (micro/src/micro_struct.c:3-37) and two linear
 * elastic materials (src/material.c:84-135). */
typedef struct {
  int n[3];       /* elements per axis (the reference's -struct_n minus 1) */
  double len[3];  /* RVE edge lengths (the micro_struct size) */
  int nx_fib, ny_fib;
  double radius;  /* fiber radius, element in fiber if centroid distance <= radius */
  double desv[2]; /* fiber offset from the centre */
  double E[2];    /* Young's modulus: [SP_ID_MATRIX], [SP_ID_FIBER] */
  double nu[2];   /* Poisson ratio:  [SP_ID_MATRIX], [SP_ID_FIBER] */
} sp_rve_desc;

typedef struct {
  int status;    /* 0 converged, SP_ERR_NOCONV otherwise */
  int outer_its; /* Newton / refinement steps (max over rhs) */
  int inner_its; /* CG iterations summed over steps (max over rhs) */
  int pad;
  double relres; /* final ||r(u)||/||r(u0)|| of the FP64 residual (max over rhs) */
} sp_solve_info;

/* Host-side element classification (micro/src/micro_struct.c:98-129 applied
 * as micro/src/micro_struct.c:176-185); fills etype[nelm]. */
int sp_classify(const sp_rve_desc *d, unsigned char *etype);
/* ELL pattern of an n[0] x n[1] x n[2] mesh in the reference's first-touch
 * insertion order (src/ell.c:46-73 driven by micro/src/assembly.c:93-110):
 * cols[ndof*81], -1 padded.  Host operation. */
int sp_ell_pattern(const int *n, int *cols);

typedef struct sp_rve_s sp_rve;
/* Builds the mesh plan, classifies elements, uploads and assembles the FP64
 * ELL Jacobian on the GPU (micro/src/assembly.c:84-137 with every boundary
 * row and column cleared). */
int sp_rve_create(const sp_rve_desc *d, sp_rve **out);
int sp_rve_destroy(sp_rve *r);
int sp_rve_sizes(const sp_rve *r, int *ndof, int *nelm, int *nfiber);
/* Downloads the assembled matrix in the reference layout (81 slots a row). */
int sp_rve_get_ell(sp_rve *r, int *cols, double *vals);
/* Per-material element stiffness (24x24, row-major) computed on the GPU. */
int sp_rve_get_ke(sp_rve *r, double *ke_matrix, double *ke_fiber);
/* Plain FP64 homogenization of nrhs macro strains (strains[nrhs][6]), one
 * RVE and one GPU kernel sequence at a time: micro/src/homogenize.c:175-225
 * (set_disp_0, Newton, Jacobi-PCG solve, add_x_dx) and :344-368 (averages).
 * Converged when ||r(u)|| <= rtol ||r(u0)||.  Outputs are host arrays
 * [nrhs][6]; u_out (optional) is [nrhs][ndof]. */
int sp_rve_homogenize(sp_rve *r, int nrhs, const double *strains, double rtol,
                      double *strain_ave, double *stress_ave, double *u_out, sp_solve_info *info);
/* 6x6 homogenized tangent C[i][j] = <sigma_i>(e_j) from six unit-strain load
 * cases solved together as one 6-rhs CG. */
int sp_rve_tangent(sp_rve *r, double rtol, double *C, sp_solve_info *info);
/* Fields of load case q of the last sp_rve_homogenize / sp_rve_tangent:
 * per-element strain and stress [nelm][6] (Gauss-weighted means over the
 * element, get_elem_properties of micro/src/homogenize.c:370-395), nodal
 * displacement and last residual [ndof].  Any output may be NULL. */
int sp_rve_fields(sp_rve *r, int q, double *strain_e, double *stress_e, double *u,
                  double *residual);
/* Writes base.pvtu and base_0.vtu (VTK XML, ascii) with the fields of load
 * case q: the arrays of the reference's micro_pvtu (micro/src/output.c:
 * 43-188). */
int sp_rve_write_vtu(sp_rve *r, int q, const char *base);
/* The VTK writer on host arrays of an n[0] x n[1] x n[2] hex8 box of edges
 * len[3]: u, res [3*nn] (NULL: zeros), etype [nelm], strain_e, stress_e
 * [nelm][6] (NULL: zeros). */
int sp_vtu_write(const char *base, const int *n, const double *len, const double *u,
                 const double *res, const unsigned char *etype, const double *strain_e,
                 const double *stress_e);

/* ------------------------------------------------------------------ batch */

#define SP_PREC_MIXED 0 /* FP32 ELL values + FP32 CG, FP64 residual refinement */
#define SP_PREC_FP64 1  /* FP64 values and CG */

#define SP_BC_AFFINE 0   /* u = eps.x on every boundary node (micro/src/homogenize.c:227-242) */
#define SP_BC_PERIODIC 1 /* u = eps.x + w, w periodic, corners at eps.x: the master-slave form
                            (BC_PER_MS, micro/inc/micro.h:26) of the reference's 2D periodic
                            conditions (micro/src/assembly.c:175-220, 272-354), in 3D */

#define SP_OP_ELL 0     /* inner CG on the RVE's assembled ELL values (coloured scatter) */
#define SP_OP_STENCIL 1 /* inner CG on the element-type stencil: A p from the two element
                           stiffnesses and the element materials, no matrix in memory */

typedef struct {
  int nrhs;          /* load cases per RVE, 1..8 (default 6) */
  int precision;     /* SP_PREC_MIXED (default) or SP_PREC_FP64 */
  double rtol;       /* FP64 residual target per rhs (default 1e-8) */
  double inner_rtol; /* CG residual reduction per refinement step (0: 3e-3 in mixed
                        precision under affine conditions -- short FP32 corrections,
                        each replaced by the FP64 residual, keep the rounding in the
                        volume averages small -- and 1e-4 in FP64 or under periodic
                        conditions) */
  int max_outer;     /* refinement steps (default 8) */
  int max_inner;     /* CG iterations per step (default 4000) */
  int threads;       /* threads per CTA: 256, 512, 1024 (0: chosen, see tune) */
  int lanes_per_row; /* unused by the batch: its operators give every lane one node */
  int ctas_per_sm;   /* resident CTAs per SM: 1 (1024 threads), 1 or 2 (512), 2 or 4 (256);
                        0: chosen, see tune */
  int cluster;       /* CTAs (thread-block cluster) solving one RVE: 1, 2, 4, 8 (assembled) */
  int op;            /* SP_OP_STENCIL (default) or SP_OP_ELL */
  int bc;            /* SP_BC_AFFINE (default) or SP_BC_PERIODIC (stencil only) */
  int tune;          /* with threads, ctas_per_sm 0 and cluster 1: SP_TUNE_AUTO (default)
                        times every instantiated CTA shape (threads x CTAs per SM, i.e.
                        registers per thread) on a sample of the batch at create time and
                        keeps the fastest, cached per device, kernel, precision, load cases
                        and dominant mesh size; SP_TUNE_OFF takes the fixed defaults (512 x 1
                        for the stencil, 512 x 2 for the assembled operator).  A tuned
                        batch's results do not depend on the launch, but the shape -- and so
                        the last bits of the sums -- may depend on the batch's composition;
                        fix threads and ctas_per_sm for bit-identical results across batches */
} sp_batch_opts;
#define SP_TUNE_AUTO 0
#define SP_TUNE_OFF 1

void sp_batch_opts_default(sp_batch_opts *o);

typedef struct sp_batch_s sp_batch;
/* nrve independent RVEs of any mix of sizes.  Classifies elements on the
 * host, builds one mesh plan per distinct size, allocates every RVE's ELL
 * values and the per-CTA work space on the GPU. */
int sp_batch_create(int nrve, const sp_rve_desc *descs, const sp_batch_opts *o, sp_batch **out);
int sp_batch_destroy(sp_batch *b);
/* Replaces the element materials of RVE `rve` (nelm bytes on the host, 0 =
 * matrix, 1 = fibre, elements x-fastest) for the following launches, in
 * place of its fibre-cylinder classification: any two-material voxel
 * micro-structure.  The copy runs on `stream` before its next launch; keep a
 * pinned `etype` unchanged until the stream has reached it.  No counterpart
 * in the reference, whose micro-structures are the fibre cylinders of
 * micro/src/micro_struct.c. */
int sp_batch_set_etype(sp_batch *b, int rve, const unsigned char *etype, void *stream);
/* Bytes of device memory held by the batch. */
int sp_batch_device_bytes(const sp_batch *b, size_t *bytes);
/* Queue the host->device copy of the step's inputs on `stream`:
 * strains[nrve][nrhs][6] (NULL: unit strains e_0..e_{nrhs-1}) and
 * materials[nrve][4] = (E_matrix, nu_matrix, E_fiber, nu_fiber) (NULL: from
 * the descriptors).  Host arrays should be pinned for asynchronous copies. */
int sp_batch_upload(sp_batch *b, const double *strains, const double *materials, void *stream);
/* One persistent launch: every RVE is assembled (coloured scatter into its
 * ELL), solved for all load cases to rtol and volume-averaged. */
int sp_batch_launch(sp_batch *b, void *stream);
/* Queue the device->host copy of the results: stress[nrve][nrhs][6],
 * strain[nrve][nrhs][6] (either may be NULL), info[nrve] (may be NULL). */
int sp_batch_download(sp_batch *b, double *stress, double *strain, sp_solve_info *info,
                      void *stream);
/* upload + launch + download + synchronize: the end-to-end call. */
int sp_batch_homogenize(sp_batch *b, const double *strains, const double *materials,
                        double *stress, double *strain, sp_solve_info *info, void *stream);
/* The CTA shape and persistent grid the batch launches with. */
int sp_batch_shape(const sp_batch *b, int *threads, int *ctas_per_sm, int *grid);
/* The autotuner's trial of this batch's shape: up to `max` candidates with
 * their threads, CTAs per SM and measured rate (estimated work units per ms:
 * sum over the trial's RVEs of dof x mesh edge), the index of the chosen one,
 * and whether the choice came from the process-wide cache (a batch of an
 * earlier create with the same key).  *ntried = 0 when the caller fixed the
 * shape.  No counterpart in the reference, which has no GPU kernels to tune;
 * it stands in for run-time solver choice (KSPSetFromOptions,
 * micro/src/alloc.c:42-43). */
int sp_batch_tune_report(const sp_batch *b, int max, int *threads, int *ctas_per_sm,
                         double *rate, int *ntried, int *chosen, int *from_cache);
/* Kernel launches made by the last sp_batch_launch (for accounting). */
int sp_batch_last_launches(const sp_batch *b, int *launches);

/* ---------------------------------------------------------------- serving */

/* A device-resident request loop standing in for the micro process's MPI
 * request loop (micro/src/main.c:114-153): requests carry a macro strain and
 * a geometry id and return the volume-averaged stress and the 6x6 tangent
 * (finite differences with delta 0.005, micro/src/homogenize.c:59-94), solved
 * as 7 load cases warm-started from that geometry's previous solution. */
typedef struct {
  size_t hbm_budget;    /* admission budget in bytes (0: 150 GB) */
  int max_inflight;     /* request slots solving at once (0: one per CTA) */
  int queue_capacity;   /* request ring size (0: 65536) */
  double rtol;          /* default 1e-8 */
  double inner_rtol;    /* CG residual reduction per refinement step (default 1e-4) */
  int idle_spin_limit;  /* empty polls of the dispatcher before the loop returns (0: default
                           2,000,000); the next submit relaunches it */
  int op;               /* SP_OP_STENCIL (default) or SP_OP_ELL */
  int ctas_per_sm;      /* request slots per SM: 1 or 2 (0: 1 for the stencil, 2 for ELL) */
  double refine_rtol;   /* a request whose warm-start prediction misses rtol is solved to
                           this tighter tolerance, so that predictions from its solutions
                           meet rtol without a solve (0: rtol / 100) */
  int warm_start;       /* SP_WARM_PREDICT (default): first-order prediction from the
                           geometry's last solved request; SP_WARM_LAST: each load case
                           starts from the geometry's last solution of that load case,
                           shifted by the affine field of the strain difference, and every
                           request is solved to rtol and kept as the next start */
} sp_server_opts;
#define SP_WARM_PREDICT 0
#define SP_WARM_LAST 1

void sp_server_opts_default(sp_server_opts *o);

typedef struct sp_server_s sp_server;
/* Makes every geometry resident (FP64 element operators, Jacobi diagonal,
 * warm-start store, and for SP_OP_ELL the assembled FP32 ELL values) while
 * the running total stays within the budget; returns SP_ERR_BUDGET,
 * creating nothing, if it does not. */
int sp_server_create(int ngeom, const sp_rve_desc *descs, const sp_server_opts *o,
                     sp_server **out);
int sp_server_destroy(sp_server *s);
/* Bytes the server would need for these geometries (no allocation). */
int sp_server_plan_bytes(int ngeom, const sp_rve_desc *descs, const sp_server_opts *o,
                         size_t *bytes);
/* Starts the device loop (a persistent kernel polling the request ring). */
int sp_server_start(sp_server *s);
/* Enqueue one request; returns its ticket (0, 1, 2, ...). */
int sp_server_submit(sp_server *s, int geometry, const double *strain, long long *ticket);
/* SP_OK and the results when the ticket is done, SP_PENDING otherwise.
 * stress[6], tangent[36] (row-major C[i][j] = d sigma_i / d eps_j). */
int sp_server_poll(sp_server *s, long long ticket, double *stress, double *tangent,
                   sp_solve_info *info);
/* Whether the loop is on the device now (it returns by itself after
 * idle_spin_limit empty polls and is relaunched by the next submit or poll
 * that finds work pending), how many times it has been launched, and how
 * many requests were submitted.  No counterpart in the reference, whose
 * request loop blocks in MPI_Recv (micro/src/main.c:114-120). */
int sp_server_status(const sp_server *s, int *loop_on_device, long long *launches,
                     long long *submitted);
/* Stops the device loop after the queued requests finish. */
int sp_server_stop(sp_server *s);
/* Open-loop load generator on the calling host thread: request i (geometry
 * geom[i], strain[i][6]) is submitted at t_arrival[i] seconds after the call
 * starts (non-decreasing); t_done[i] receives the time its result was seen,
 * so t_done[i] - t_arrival[i] is its latency including queueing.  Results
 * go to stress[nreq][6], tangent[nreq][36], info[nreq] (each may be NULL).
 * SP_ERR_TIMEOUT after timeout_s seconds. */
int sp_server_replay(sp_server *s, int nreq, const int *geom, const double *strain,
                     const double *t_arrival, double *t_done, double *stress, double *tangent,
                     sp_solve_info *info, double timeout_s);

/* --------------------------------------------------- macro-micro messages */

/* The reference's coupling message (message_t, inc/comm.h:18-27), field for
 * field: an MPI program's message_t buffer can be passed as an sp_message. */
#define SP_MAX_VOIGT 6
#define SP_ACTION_NULL 0               /* inc/comm.h:12-16 */
#define SP_ACTION_MICRO_CALC_STRESS 1
#define SP_ACTION_MICRO_CALC_C_TANGENT 2
#define SP_ACTION_MICRO_CALC_RHO 3
#define SP_ACTION_MICRO_END 4

typedef struct {
  int action;
  int num_voigt;
  double strain_mac[SP_MAX_VOIGT];
  double stress_ave[SP_MAX_VOIGT];
  double c_tangent_ave[SP_MAX_VOIGT * SP_MAX_VOIGT];
  double rho;
} sp_message;

#define SP_MICRO_LINEAR 0 /* like the reference for linear materials: one FD tangent
                             around zero, stress = C eps (micro/src/homogenize.c:3-21) */
#define SP_MICRO_SOLVE 1  /* every stress / tangent request solved at its strain */

/* One micro endpoint: answers messages for one geometry of a serving loop
 * (micro/src/main.c:114-153).  rho is what ACTION_MICRO_CALC_RHO returns
 * (the reference's constant is 1e7, micro/src/init.c:9). */
typedef struct sp_micro_s sp_micro;
int sp_micro_create(sp_server *srv, int geometry, int mode, double rho, sp_micro **out);
int sp_micro_destroy(sp_micro *m);
/* Fills the reply fields of msg for its action; SP_ERR_ARG for an unknown
 * action or num_voigt != 6. */
int sp_micro_handle(sp_micro *m, sp_message *msg);
/* The request loop over a caller's transport: receive, answer, send the
 * reply, until ACTION_MICRO_END (not answered).  The callbacks return 0 on
 * success. */
typedef int (*sp_message_recv)(sp_message *msg, void *ctx);
typedef int (*sp_message_send)(const sp_message *msg, void *ctx);
int sp_micro_serve(sp_micro *m, sp_message_recv recv, sp_message_send send, void *ctx,
                   long long *handled);
/* Serving-loop requests made so far. */
int sp_micro_requests(const sp_micro *m, long long *requests);

/* -------------------------------------------------------------------- FE2 */

/* An FE2 step on one GPU: the macro Newton loop of macro/src/main.c:202-256
 * (residual macro/src/assembly.c:5-84, Jacobian :165-222, clamped rows and
 * columns :208-214) on a structured hex8 cantilever of n[0] x n[1] x n[2]
 * elements, clamped at x = 0 and loaded by a uniform traction on x = len[0];
 * every macro Gauss point takes its stress and tangent from one of nrve
 * micro RVEs served by sp_server.  FP64 macro assembly and Jacobi-PCG. */
#define SP_FE2_LINEAR 0 /* linear micro materials: one FD tangent around zero strain
                           per RVE (micro/src/init.c:54-59), then sigma = C eps
                           (micro/src/homogenize.c:3-21) */
#define SP_FE2_PER_GP 1 /* one serving-loop request (stress + FD tangent) per Gauss
                           point per Newton iteration */
#define SP_FE2_MAX_ITS 16

typedef struct {
  int n[3];              /* macro elements per axis (default 40 x 10 x 10) */
  double len[3];         /* macro box edges (default 4 x 1 x 1) */
  double traction[3];    /* Pa on the face x = len[0] (default (0, 0, -1e6)) */
  int nrve;              /* micro RVEs */
  const sp_rve_desc *rves;
  const int *gp_rve;     /* [nelm*8] RVE of each Gauss point (element-major), NULL: seeded */
  int newton_its;        /* Newton iterations, 1..SP_FE2_MAX_ITS (default 5) */
  double newton_tol;     /* stop once ||b|| <= tol (default 0: all iterations) */
  double lin_rtol;       /* macro PCG relative tolerance (default 1e-10) */
  double strain_clip;    /* |eps_v| below this is set to 0 (reference: 1e-6,
                            macro/src/assembly.c:319) */
  int micro;             /* SP_FE2_LINEAR (default) or SP_FE2_PER_GP */
  int seed;              /* seed of the Gauss point -> RVE binding when gp_rve is NULL */
} sp_fe2_desc;

void sp_fe2_desc_default(sp_fe2_desc *d);

typedef struct {
  int newton_its;                 /* iterations run */
  int pcg_its[SP_FE2_MAX_ITS];    /* macro PCG iterations per Newton iteration */
  double bnorm[SP_FE2_MAX_ITS];   /* ||b|| at the start of each Newton iteration */
  double tip[3];                  /* mean displacement of the loaded face */
  long long micro_requests;       /* serving-loop requests made */
  double micro_s, macro_s;        /* wall time in micro requests / the macro loop */
  double residual_ms, assemble_ms, solve_ms; /* device time (CUDA events), summed over
                                                iterations: strains + stresses + residual,
                                                Jacobian assembly, PCG + update */
} sp_fe2_info;

typedef struct sp_fe2_s sp_fe2;
/* Builds the macro problem, starts a serving loop over the RVEs and, for
 * SP_FE2_LINEAR, obtains every RVE's tangent around zero strain. */
int sp_fe2_create(const sp_fe2_desc *d, sp_fe2 **out);
/* Runs the Newton loop from u = 0. */
int sp_fe2_run(sp_fe2 *f, sp_fe2_info *info);
/* Macro displacement, [3 * (n0+1) * (n1+1) * (n2+1)], node = i + nx (j + ny k). */
int sp_fe2_displacement(const sp_fe2 *f, double *u);
/* The Gauss point -> RVE binding, [nelm*8]. */
int sp_fe2_gp_rve(const sp_fe2 *f, int *gp_rve);
/* SP_FE2_LINEAR: the RVE tangents used, [nrve][36] row-major. */
int sp_fe2_micro_tangents(const sp_fe2 *f, double *C);
int sp_fe2_destroy(sp_fe2 *f);

#ifdef __cplusplus
}
#endif

#endif
