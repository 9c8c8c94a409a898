/* Implementation of the MPI stand-in declared in mpi.h (test infrastructure).
 *
 * Size 1 (no ORACLE_MPI_SIZE in the environment, or 1): point-to-point calls
 * address the process itself; a send is delivered into the oldest posted
 * receive with the same tag, as MPI does for a self-message.
 *
 * Size N > 1: ORACLE_MPI_RANK, ORACLE_MPI_SIZE and ORACLE_MPI_DIR name this
 * process's rank, the number of ranks and a directory for the rendezvous. On
 * the first call every rank listens on <dir>/r<rank>, connects to every lower
 * rank and accepts every higher one; a thread per peer drains that peer's
 * socket into a queue, so a send never blocks on the receiver. A receive
 * completes in MPI_Wait with the oldest queued message from its source and
 * tag (MPI's non-overtaking order). Collectives are sends to every rank;
 * MPI_Allreduce sums the contributions in rank order, so every rank gets the
 * same bits. A wait that sees nothing for ORACLE_MPI_TIMEOUT seconds (60)
 * exits the process with a message instead of hanging. */
#include <errno.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/socket.h>
#include <sys/un.h>
#include <time.h>
#include <unistd.h>
#include "mpi.h"

#define ORACLE_MAX_POSTED 256
#define ORACLE_MAX_RANKS 16
#define TAG_BARRIER (-1)
#define TAG_REDUCE (-2)

static long type_size(MPI_Datatype t) { return t == MPI_DOUBLE ? 8 : 4; }

/* ---------------------------------------------------------------- state */
typedef struct msg {
  struct msg *next;
  int tag;
  long bytes;
  unsigned char data[];
} msg;

typedef struct {
  msg *head, *tail;
} queue;

typedef struct { void *buf; long bytes; int src; int tag; int live; } posted_recv;

static int g_init = 0;
static int g_rank = 0, g_size = 1;
static int g_fd[ORACLE_MAX_RANKS];
static queue g_q[ORACLE_MAX_RANKS];
static pthread_mutex_t g_mu = PTHREAD_MUTEX_INITIALIZER;
static pthread_cond_t g_cv = PTHREAD_COND_INITIALIZER;
static posted_recv g_posted[ORACLE_MAX_POSTED];
static int g_unmatched = 0;
static int g_timeout = 60;

static void die(const char *what)
{
  fprintf(stderr, "oracle mpi shim (rank %d of %d): %s (%s)\n", g_rank, g_size, what, strerror(errno));
  exit(3);
}

static int write_all(int fd, const void *p, long n)
{
  const unsigned char *c = (const unsigned char *)p;
  while (n > 0) {
    const ssize_t w = write(fd, c, (size_t)n);
    if (w < 0) {
      if (errno == EINTR) continue;
      return -1;
    }
    c += w;
    n -= w;
  }
  return 0;
}

static int read_all(int fd, void *p, long n)
{
  unsigned char *c = (unsigned char *)p;
  while (n > 0) {
    const ssize_t r = read(fd, c, (size_t)n);
    if (r == 0) return -1;
    if (r < 0) {
      if (errno == EINTR) continue;
      return -1;
    }
    c += r;
    n -= r;
  }
  return 0;
}

static void enqueue(int src, int tag, const void *data, long bytes)
{
  msg *m = (msg *)malloc(sizeof(msg) + (size_t)(bytes > 0 ? bytes : 1));
  if (!m) die("out of memory");
  m->next = NULL;
  m->tag = tag;
  m->bytes = bytes;
  if (bytes > 0) memcpy(m->data, data, (size_t)bytes);
  pthread_mutex_lock(&g_mu);
  if (g_q[src].tail) g_q[src].tail->next = m;
  else g_q[src].head = m;
  g_q[src].tail = m;
  pthread_cond_broadcast(&g_cv);
  pthread_mutex_unlock(&g_mu);
}

/* Oldest message from src with tag, removed from the queue; waits for it. */
static msg *dequeue(int src, int tag)
{
  struct timespec until;
  clock_gettime(CLOCK_REALTIME, &until);
  until.tv_sec += g_timeout;
  pthread_mutex_lock(&g_mu);
  for (;;) {
    msg *prev = NULL;
    for (msg *m = g_q[src].head; m; prev = m, m = m->next) {
      if (m->tag != tag) continue;
      if (prev) prev->next = m->next;
      else g_q[src].head = m->next;
      if (g_q[src].tail == m) g_q[src].tail = prev;
      pthread_mutex_unlock(&g_mu);
      return m;
    }
    if (pthread_cond_timedwait(&g_cv, &g_mu, &until) == ETIMEDOUT) {
      pthread_mutex_unlock(&g_mu);
      fprintf(stderr, "oracle mpi shim (rank %d of %d): no message from rank %d with tag %d after %d s\n",
              g_rank, g_size, src, tag, g_timeout);
      exit(3);
    }
  }
}

static void *reader(void *arg)
{
  const int src = (int)(intptr_t)arg;
  for (;;) {
    int tag;
    long bytes;
    if (read_all(g_fd[src], &tag, sizeof(tag)) || read_all(g_fd[src], &bytes, sizeof(bytes))) return NULL;
    unsigned char *buf = (unsigned char *)malloc((size_t)(bytes > 0 ? bytes : 1));
    if (!buf) die("out of memory");
    if (bytes > 0 && read_all(g_fd[src], buf, bytes)) {
      free(buf);
      return NULL;
    }
    enqueue(src, tag, buf, bytes);
    free(buf);
  }
}

static void sock_path(struct sockaddr_un *a, const char *dir, int r)
{
  memset(a, 0, sizeof(*a));
  a->sun_family = AF_UNIX;
  snprintf(a->sun_path, sizeof(a->sun_path), "%s/r%d", dir, r);
}

static void init_once(void)
{
  if (g_init) return;
  g_init = 1;
  const char *s = getenv("ORACLE_MPI_SIZE");
  const char *r = getenv("ORACLE_MPI_RANK");
  const char *t = getenv("ORACLE_MPI_TIMEOUT");
  if (t) g_timeout = atoi(t);
  g_size = s ? atoi(s) : 1;
  g_rank = r ? atoi(r) : 0;
  if (g_size <= 1) {
    g_size = 1;
    g_rank = 0;
    return;
  }
  if (g_size > ORACLE_MAX_RANKS || g_rank < 0 || g_rank >= g_size) die("bad ORACLE_MPI_SIZE / ORACLE_MPI_RANK");
  const char *dir = getenv("ORACLE_MPI_DIR");
  if (!dir) die("ORACLE_MPI_DIR not set");
  const int ls = socket(AF_UNIX, SOCK_STREAM, 0);
  if (ls < 0) die("socket");
  struct sockaddr_un a;
  sock_path(&a, dir, g_rank);
  unlink(a.sun_path);
  if (bind(ls, (struct sockaddr *)&a, sizeof(a)) || listen(ls, ORACLE_MAX_RANKS)) die("bind/listen");
  for (int p = 0; p < g_rank; ++p) {  /* connect to every lower rank */
    const int fd = socket(AF_UNIX, SOCK_STREAM, 0);
    struct sockaddr_un b;
    sock_path(&b, dir, p);
    int ok = 0;
    for (int tries = 0; tries < 100 * g_timeout; ++tries) {
      if (connect(fd, (struct sockaddr *)&b, sizeof(b)) == 0) {
        ok = 1;
        break;
      }
      usleep(10000);
    }
    if (!ok) die("connect");
    if (write_all(fd, &g_rank, sizeof(g_rank))) die("hello");
    g_fd[p] = fd;
  }
  for (int n = g_rank + 1; n < g_size; ++n) {  /* accept every higher rank */
    const int fd = accept(ls, NULL, NULL);
    int who = -1;
    if (fd < 0 || read_all(fd, &who, sizeof(who)) || who <= g_rank || who >= g_size) die("accept");
    g_fd[who] = fd;
  }
  close(ls);
  for (int p = 0; p < g_size; ++p) {
    if (p == g_rank) continue;
    pthread_t th;
    if (pthread_create(&th, NULL, reader, (void *)(intptr_t)p)) die("pthread_create");
    pthread_detach(th);
  }
}

static void send_to(int dest, int tag, const void *buf, long bytes)
{
  if (dest == g_rank) {
    enqueue(dest, tag, buf, bytes);
    return;
  }
  if (write_all(g_fd[dest], &tag, sizeof(tag)) || write_all(g_fd[dest], &bytes, sizeof(bytes)) ||
      (bytes > 0 && write_all(g_fd[dest], buf, bytes)))
    die("send");
}

/* ------------------------------------------------------------------- API */
int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; init_once(); return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; init_once(); *r = g_rank; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; init_once(); *s = g_size; return MPI_SUCCESS; }

int MPI_Irecv(void *buf, int count, MPI_Datatype type, int src, int tag, MPI_Comm comm,
              MPI_Request *req)
{
  (void)comm;
  init_once();
  for (int i = 0; i < ORACLE_MAX_POSTED; ++i) {
    if (!g_posted[i].live) {
      g_posted[i].buf = buf;
      g_posted[i].bytes = (long)count * type_size(type);
      g_posted[i].src = g_size == 1 ? 0 : src;
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
  (void)comm;
  init_once();
  const long bytes = (long)count * type_size(type);
  if (g_size == 1) {
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
  if (dest < 0 || dest >= g_size) die("send to a rank outside the job");
  send_to(dest, tag, buf, bytes);
  return MPI_SUCCESS;
}

int MPI_Wait(MPI_Request *req, MPI_Status *st)
{
  if (st) { st->MPI_SOURCE = 0; st->MPI_TAG = 0; st->MPI_ERROR = 0; }
  if (g_size == 1) return MPI_SUCCESS;
  posted_recv *p = &g_posted[*req];
  if (!p->live) return MPI_SUCCESS;
  msg *m = dequeue(p->src, p->tag);
  const long n = m->bytes < p->bytes ? m->bytes : p->bytes;
  if (n > 0) memcpy(p->buf, m->data, (size_t)n);
  if (st) { st->MPI_SOURCE = p->src; st->MPI_TAG = p->tag; }
  free(m);
  p->live = 0;
  return MPI_SUCCESS;
}

int MPI_Allreduce(const void *in, void *out, int count, MPI_Datatype type, MPI_Op op,
                  MPI_Comm comm)
{
  (void)op; (void)comm;
  init_once();
  const long bytes = (long)count * type_size(type);
  if (g_size == 1) {
    memmove(out, in, (size_t)bytes);
    return MPI_SUCCESS;
  }
  for (int p = 0; p < g_size; ++p)
    if (p != g_rank) send_to(p, TAG_REDUCE, in, bytes);
  unsigned char *parts = (unsigned char *)malloc((size_t)(bytes * g_size + 1));
  if (!parts) die("out of memory");
  memcpy(parts + bytes * g_rank, in, (size_t)bytes);
  for (int p = 0; p < g_size; ++p) {
    if (p == g_rank) continue;
    msg *m = dequeue(p, TAG_REDUCE);
    memcpy(parts + bytes * p, m->data, (size_t)(m->bytes < bytes ? m->bytes : bytes));
    free(m);
  }
  for (int i = 0; i < count; ++i) {  /* rank order, the same on every rank */
    if (type == MPI_DOUBLE) {
      double s = 0.0;
      for (int p = 0; p < g_size; ++p) s += ((const double *)(parts + bytes * p))[i];
      ((double *)out)[i] = s;
    } else {
      int s = 0;
      for (int p = 0; p < g_size; ++p) s += ((const int *)(parts + bytes * p))[i];
      ((int *)out)[i] = s;
    }
  }
  free(parts);
  return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm comm)
{
  (void)comm;
  init_once();
  if (g_size == 1) return MPI_SUCCESS;
  for (int p = 0; p < g_size; ++p)
    if (p != g_rank) send_to(p, TAG_BARRIER, NULL, 0);
  for (int p = 0; p < g_size; ++p) {
    if (p == g_rank) continue;
    free(dequeue(p, TAG_BARRIER));
  }
  return MPI_SUCCESS;
}

int oracle_mpi_unmatched(void) { return g_unmatched; }
