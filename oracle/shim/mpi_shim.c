/* Implementation of the size-1 MPI stand-in declared in mpi.h (test infrastructure). */
#include <stdio.h>
#include <string.h>
#include "mpi.h"

#define ORACLE_MAX_POSTED 64

typedef struct { void *buf; long bytes; int tag; int live; } posted_recv;
static posted_recv g_posted[ORACLE_MAX_POSTED];
static int g_unmatched = 0;

static long type_size(MPI_Datatype t) { return t == MPI_DOUBLE ? 8 : 4; }

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return MPI_SUCCESS; }

int MPI_Irecv(void *buf, int count, MPI_Datatype type, int src, int tag, MPI_Comm comm,
              MPI_Request *req)
{
  (void)src; (void)comm;
  for (int i = 0; i < ORACLE_MAX_POSTED; ++i) {
    if (!g_posted[i].live) {
      g_posted[i].buf = buf;
      g_posted[i].bytes = (long)count * type_size(type);
      g_posted[i].tag = tag;
      g_posted[i].live = 1;
      *req = i;
      return MPI_SUCCESS;
    }
  }
  fprintf(stderr, "oracle mpi shim: too many posted receives\n");
  return 1;
}

int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm)
{
  (void)dest; (void)comm;
  const long bytes = (long)count * type_size(type);
  for (int i = 0; i < ORACLE_MAX_POSTED; ++i) {
    if (g_posted[i].live && g_posted[i].tag == tag) {
      const long n = bytes < g_posted[i].bytes ? bytes : g_posted[i].bytes;
      if (n > 0) memmove(g_posted[i].buf, buf, (size_t)n);
      g_posted[i].live = 0;
      return MPI_SUCCESS;
    }
  }
  g_unmatched++;
  return MPI_SUCCESS;
}

int MPI_Wait(MPI_Request *req, MPI_Status *st)
{
  (void)req;
  if (st) { st->MPI_SOURCE = 0; st->MPI_TAG = 0; st->MPI_ERROR = 0; }
  return MPI_SUCCESS;
}

int MPI_Allreduce(const void *in, void *out, int count, MPI_Datatype type, MPI_Op op,
                  MPI_Comm comm)
{
  (void)op; (void)comm;
  memmove(out, in, (size_t)((long)count * type_size(type)));
  return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm comm) { (void)comm; return MPI_SUCCESS; }
int oracle_mpi_unmatched(void) { return g_unmatched; }
