/* Single-rank MPI shim -- test infrastructure only.
 * Lets the reference's own sources (which include <mpi.h>) build without an MPI
 * installation.  Every call behaves as a one-process job: rank 0 of 1, Cartesian
 * neighbours are MPI_PROC_NULL, reductions copy, point-to-point is never reached
 * at one rank (the reference returns early, mod_mpi.cu:107, mod_mpi_fault.cu:88). */
#ifndef DFD_REFSHIM_MPI_H
#define DFD_REFSHIM_MPI_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_PROC_NULL (-2)
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_INT 1
#define MPI_FLOAT 2
#define MPI_DOUBLE 3
#define MPI_MIN 1
#define MPI_MAX 2
#define MPI_SUM 3
int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm c, int *r);
int MPI_Comm_size(MPI_Comm c, int *s);
int MPI_Get_processor_name(char *name, int *len);
int MPI_Cart_create(MPI_Comm c, int nd, const int *dims, const int *periods, int reorder, MPI_Comm *out);
int MPI_Cart_coords(MPI_Comm c, int rank, int nd, int *coords);
int MPI_Cart_shift(MPI_Comm c, int dir, int disp, int *src, int *dst);
int MPI_Barrier(MPI_Comm c);
int MPI_Abort(MPI_Comm c, int code);
int MPI_Reduce(const void *in, void *out, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c);
int MPI_Sendrecv(const void *sb, int sn, MPI_Datatype st, int dst, int stag, void *rb, int rn, MPI_Datatype rt,
                 int src, int rtag, MPI_Comm c, MPI_Status *status);
#ifdef __cplusplus
}
#endif
#endif
