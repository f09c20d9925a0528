/*
 * FETI4I: C interface of the B200 Total-FETI dual solver.
 *
 * Drop-in replacement for ESPRESO's FETI4I library interface
 * (feeleewee/espreso include/feti4i.h).  Every declaration below keeps the
 * reference's name, argument order, types and meaning; the reference line it
 * replaces is given beside it.  The extensions are declared in
 * feti4i_ext.h.
 *
 * Differences in behaviour, all additive:
 *   - no MPI: one process, one GPU; FETI4IMPIInt stays a plain int and
 *     neighbours_size must be 0.  "mpi.h" is included as in the reference
 *     (include/feti4i.h:5); without a real MPI the single-process stand-in
 *     include/mpi.h serves it;
 *   - FETI4I_INT_WIDTH 64 (FETI4IInt = long, include/feti4i.h:25-30) is the
 *     ABI of libfeti4i_b200_i64.so; the default 32 that of libfeti4i_b200.so.
 *     Indices must still fit 32 bits (larger ones are rejected);
 *   - errors never terminate the process: a failing call records a message
 *     that FETI4IGetLastError() (feti4i_ext.h) returns;
 *   - FETI4IUpdateStiffnessMatrix/Rhs/Dirichlet, declared but not defined in
 *     the reference (include/feti4i.h:177-192), are implemented.
 */
#ifndef FETI4I_H_
#define FETI4I_H_

#include "mpi.h"

/* integer/real widths: include/feti4i.h:7-39 */
#ifndef FETI4I_INT_WIDTH
#define FETI4I_INT_WIDTH 32
#endif
#ifndef FETI4I_REAL_WIDTH
#define FETI4I_REAL_WIDTH 64
#endif

#if FETI4I_INT_WIDTH == 32
typedef int FETI4IInt;
#elif FETI4I_INT_WIDTH == 64
typedef long FETI4IInt;
#else
#error "Incorrect user-supplied value of FETI4I_INT_WIDTH"
#endif

typedef int FETI4IMPIInt;

#if FETI4I_REAL_WIDTH == 64
typedef double FETI4IReal;
#else
#error "Incorrect user-supplied value of FETI4I_REAL_WIDTH"
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* opaque handles: include/feti4i.h:49-52 */
typedef struct FETI4IStructMatrix *FETI4IMatrix;
typedef struct FETI4IStructInstance *FETI4IInstance;

/* include/feti4i.h:66 -- defaults: SUBDOMAINS 4, MAX_ITERATIONS 200, FETI_METHOD 0
 * (Total FETI), PRECONDITIONER 3 (Dirichlet), CGSOLVER 0 (PCG), N_MICS 2,
 * VERBOSE_LEVEL 1, MEASURE_LEVEL 0, PRINT_MATRICES 0, SC_SIZE 200 */
void FETI4ISetDefaultIntegerOptions(FETI4IInt *options);

/* include/feti4i.h:77 -- default PRECISION 1e-5 */
void FETI4ISetDefaultRealOptions(FETI4IReal *options);

/* include/feti4i.h:90 */
void FETI4ICreateStiffnessMatrix(FETI4IMatrix *matrix, FETI4IInt type, FETI4IInt indexBase);

/* include/feti4i.h:109 -- values row-major dofsSize x dofsSize; DOFs of an
 * element are ordered node by node (dofs[a*dpn + c] is component c of
 * nodes[a], dpn = dofsSize / nodesSize) */
void FETI4IAddElement(FETI4IMatrix matrix, FETI4IInt type, FETI4IInt nodesSize, FETI4IInt *nodes,
                      FETI4IInt dofsSize, FETI4IInt *dofs, FETI4IReal *values);

/* include/feti4i.h:142 */
void FETI4ICreateInstance(FETI4IInstance *instance, FETI4IMatrix matrix, FETI4IInt size, FETI4IReal *rhs,
                          FETI4IInt *l2g, FETI4IMPIInt neighbours_size, FETI4IMPIInt *neighbours,
                          FETI4IInt dirichlet_size, FETI4IInt *dirichlet_indices, FETI4IReal *dirichlet_values,
                          FETI4IInt *integer_options, FETI4IReal *real_options);

/* include/feti4i.h:166 */
void FETI4ISolve(FETI4IInstance instance, FETI4IInt solution_size, FETI4IReal *solution);

/* include/feti4i.h:177 */
void FETI4IUpdateStiffnessMatrix(FETI4IInstance instance, FETI4IMatrix stiffnessMatrix);
/* include/feti4i.h:182 */
void FETI4IUpdateRhs(FETI4IInstance instance, FETI4IInt size, FETI4IReal *values);
/* include/feti4i.h:188 */
void FETI4IUpdateDirichlet(FETI4IInstance instance, FETI4IInt size, FETI4IInt *indices, FETI4IReal *values);

/* include/feti4i.h:206 -- accepts a matrix or an instance handle */
void FETI4IDestroy(void *ptr);

#ifdef __cplusplus
}
#endif

/* include/feti4i.h:221-235 */
typedef enum {
    FETI4I_SUBDOMAINS,
    FETI4I_MAX_ITERATIONS,
    FETI4I_FETI_METHOD,
    FETI4I_PRECONDITIONER,
    FETI4I_CGSOLVER,
    FETI4I_N_MICS,
    FETI4I_VERBOSE_LEVEL,
    FETI4I_MEASURE_LEVEL,
    FETI4I_PRINT_MATRICES,
    FETI4I_SC_SIZE,
    FETI4I_INTEGER_OPTIONS_SIZE
} FETI4IIntegerOptions;

/* include/feti4i.h:244-248 */
typedef enum {
    FETI4I_PRECISION,
    FETI4I_REAL_OPTIONS_SIZE
} FETI4IRealOptions;

/* include/feti4i.h:255-259 */
typedef enum {
    FETI4I_REAL_SYMMETRIC_POSITIVE_DEFINITE,
    FETI4I_REAL_SYMMETRIC_INDEFINITE,
    FETI4I_REAL_UNSYMMETRIC
} FETI4IMatrixType;

/* include/feti4i.h:266-271 */
typedef enum {
    FETI4I_POINT,
    FETI4I_LINE,
    FETI4I_PLANE,
    FETI4I_VOLUME
} FETI4IElementType;

#endif /* FETI4I_H_ */
