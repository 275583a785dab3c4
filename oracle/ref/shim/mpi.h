/* Test infrastructure only (oracle build). Project-written single-process stand-in
 * for the handful of MPI symbols the reference's logging macros touch
 * (include/Logger.h:170-186 call MPI_Comm_rank unconditionally when HAS_MPI is set,
 * include/ves3d_common.h:44-55). One rank, rank 0. */
#ifndef VES3D_ORACLE_MPI_SHIM_H
#define VES3D_ORACLE_MPI_SHIM_H

typedef int MPI_Comm;
#define MPI_COMM_WORLD 0
#define MPI_COMM_SELF 1

static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }

#endif
