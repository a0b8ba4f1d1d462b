/* Minimal MPI declarations so the reference's kernel files compile for the
 * per-kernel parity tests (test infrastructure; no MPI is ever called). */
#pragma once
typedef int MPI_Comm;
typedef int MPI_Datatype;
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_PROC_NULL (-1)
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Gather(const void *, int, MPI_Datatype, void *, int, MPI_Datatype, int, MPI_Comm) {
    return 0;
}
static inline double MPI_Wtime(void) { return 0.0; }
