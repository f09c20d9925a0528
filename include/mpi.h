/*
 * Minimal single-process MPI stand-in for callers built without MPI.
 *
 * ESPRESO's FETI4I header includes "mpi.h" (include/feti4i.h:5 of the reference), and callers such
 * as src/app/apitest.cpp call MPI_Init / MPI_Comm_rank / MPI_Finalize around the FETI4I calls.  The
 * B200 library runs one process on one GPU and needs no MPI, so this header lets such callers (and
 * the reference header itself) compile unchanged: one rank, rank 0, every call succeeds.
 *
 * A caller that links a real MPI includes that MPI's mpi.h before feti4i.h; this stand-in then
 * defines nothing (it checks MPI_VERSION, which every MPI implementation defines).
 */
#ifndef FETI4I_MPI_STANDIN_H_
#define FETI4I_MPI_STANDIN_H_

#ifndef MPI_VERSION
#define FETI4I_MPI_STANDIN 1

#include <stdlib.h>

typedef int MPI_Comm;
#define MPI_COMM_WORLD ((MPI_Comm)0)
#define MPI_COMM_SELF ((MPI_Comm)1)
#define MPI_SUCCESS 0

static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
static inline int MPI_Initialized(int *flag) { *flag = 1; return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm comm) { (void)comm; return MPI_SUCCESS; }
static inline int MPI_Abort(MPI_Comm comm, int code) { (void)comm; exit(code); return code; }

#endif /* MPI_VERSION */
#endif /* FETI4I_MPI_STANDIN_H_ */
