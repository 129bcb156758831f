/*
 * solvers.h -- drop-in replacement for the reference's inc/solvers.h
 * (inc/solvers.h:1-24).
 *
 * The solver selector stays as it is.  SOLVER_ELL_GPU is new: it names the
 * ELL Jacobi-PCG of libsputnik_b200.so.  The PETSc KSP printer
 * (inc/solvers.h:15-18) exists only when the caller builds with PETSc, and
 * the SLEPc include (inc/solvers.h:20-22) only when it builds with SLEPc, as
 * in the reference: the macro program is compiled with -DSLEPC and reaches
 * its EPS type through this header (macro/inc/macro.h:12).  This library
 * itself has no PETSc or SLEPc dependency.
 */
#ifndef SOLVERS_H
#define SOLVERS_H

#define SOLVER_NULL 0
#define SOLVER_PETSC 1
#define SOLVER_ELL_GPU 2

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int type;
} solver_t;

/* The reference's programs define this object (micro/src/main.c:16,
 * macro/src/main.c:15).  The library provides a weak definition so that a
 * caller without one still links; a caller's own definition takes
 * precedence. */
extern solver_t solver;

#ifdef __cplusplus
}
#endif

#ifdef PETSC
#include "petscksp.h"
int solvers_print_petsc_ksp_info(MPI_Comm COMM, KSP ksp);
#endif

#ifdef SLEPC
#include "slepceps.h"
#endif

#endif
