/*
 * Project-written single-process MPI stand-in (size 1) for compiling the
 * reference program PIC/3d_pic458_domain.c as the CPU oracle.
 * TEST INFRASTRUCTURE ONLY. Point-to-point calls can only address rank 0
 * (itself): a send is delivered into the oldest posted receive with the same
 * tag, as MPI would do for a self-message; collectives copy their input.
 */
#ifndef ORACLE_MPI_SHIM_H
#define ORACLE_MPI_SHIM_H

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_SUM 1
#define MPI_SUCCESS 0

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Irecv(void *buf, int count, MPI_Datatype type, int src, int tag, MPI_Comm comm,
              MPI_Request *req);
int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm);
int MPI_Wait(MPI_Request *req, MPI_Status *st);
int MPI_Allreduce(const void *in, void *out, int count, MPI_Datatype type, MPI_Op op,
                  MPI_Comm comm);
int MPI_Barrier(MPI_Comm comm);

/* Number of sends that found no posted receive (a self-exchange mismatch). */
int oracle_mpi_unmatched(void);

#endif
