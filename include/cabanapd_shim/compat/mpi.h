/* Single-process stand-in for <mpi.h> so CabanaPD programs build unchanged
 * against the cabanapd_b200 front end (one GPU, one rank): add
 * -I include/cabanapd_shim/compat. Only the calls those programs make. */
#ifndef CABANAPD_SHIM_MPI_H
#define CABANAPD_SHIM_MPI_H

typedef int MPI_Comm;
#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0

static inline int MPI_Init(int* argc, char*** argv)
{
    (void)argc;
    (void)argv;
    return MPI_SUCCESS;
}
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm comm, int* rank)
{
    (void)comm;
    *rank = 0;
    return MPI_SUCCESS;
}
static inline int MPI_Comm_size(MPI_Comm comm, int* size)
{
    (void)comm;
    *size = 1;
    return MPI_SUCCESS;
}
static inline int MPI_Barrier(MPI_Comm comm)
{
    (void)comm;
    return MPI_SUCCESS;
}

#endif
