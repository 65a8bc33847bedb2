/* mpi_stub.c -- point-to-point messages to self for the single-rank MPI
 * stand-in of oracle/mpi_stub/mpi.h (test infrastructure: linked only into
 * the oracle binary oracle/_ref/bam).  A send is buffered (copied) unless a
 * matching receive is already posted; a receive takes the oldest buffered
 * message of its tag or stays posted until a send arrives. */
#include <stdlib.h>
#include "mpi.h"

#define NREQ 65536
typedef struct msg { int tag; size_t bytes; void *data; struct msg *next; } msg;
typedef struct { int used, done, tag; void *buf; size_t cap, got; } req;

static msg *queue_head, *queue_tail;
static req reqs[NREQ];
static int nextreq = 1;

static int tag_match(int want, int have) { return want == MPI_ANY_TAG || want == have; }

static int new_req(void)
{
  for (int k = 0; k < NREQ; k++) {
    int i = (nextreq + k) % NREQ;
    if (i && !reqs[i].used) {
      nextreq = i + 1;
      reqs[i].used = 1;
      reqs[i].done = 0;
      return i;
    }
  }
  fprintf(stderr, "mpi stub: out of requests\n");
  exit(3);
}

static void deliver(const void *b, size_t bytes, int tag)
{
  /* oldest posted receive of this tag first */
  for (int i = 1; i < NREQ; i++)
    if (reqs[i].used && !reqs[i].done && reqs[i].buf && tag_match(reqs[i].tag, tag)) {
      if (bytes > reqs[i].cap) { fprintf(stderr, "mpi stub: message truncated\n"); exit(3); }
      memcpy(reqs[i].buf, b, bytes);
      reqs[i].got = bytes;
      reqs[i].done = 1;
      return;
    }
  msg *m = malloc(sizeof *m);
  m->tag = tag;
  m->bytes = bytes;
  m->data = malloc(bytes ? bytes : 1);
  memcpy(m->data, b, bytes);
  m->next = 0;
  if (queue_tail) queue_tail->next = m; else queue_head = m;
  queue_tail = m;
}

static msg *take(int tag, int remove)
{
  msg *p = 0, *m = queue_head;
  while (m && !tag_match(tag, m->tag)) { p = m; m = m->next; }
  if (m && remove) {
    if (p) p->next = m->next; else queue_head = m->next;
    if (queue_tail == m) queue_tail = p;
  }
  return m;
}

int MPI_Isend(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request *q)
{
  (void)d; (void)c;
  deliver(b, (size_t)n * t, tag);
  int i = new_req();
  reqs[i].done = 1;
  reqs[i].buf = 0;
  *q = i;
  return 0;
}

int MPI_Send(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c)
{
  (void)d; (void)c;
  deliver(b, (size_t)n * t, tag);
  return 0;
}

int MPI_Irecv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request *q)
{
  (void)s; (void)c;
  int i = new_req();
  reqs[i].tag = tag;
  reqs[i].buf = b;
  reqs[i].cap = (size_t)n * t;
  msg *m = take(tag, 1);
  if (m) {
    if (m->bytes > reqs[i].cap) { fprintf(stderr, "mpi stub: message truncated\n"); exit(3); }
    memcpy(b, m->data, m->bytes);
    reqs[i].got = m->bytes;
    reqs[i].done = 1;
    free(m->data);
    free(m);
  }
  *q = i;
  return 0;
}

int MPI_Recv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status *st)
{
  (void)s; (void)c;
  msg *m = take(tag, 1);
  if (!m) { fprintf(stderr, "mpi stub: receive without a message at one rank\n"); exit(3); }
  if (m->bytes > (size_t)n * t) { fprintf(stderr, "mpi stub: message truncated\n"); exit(3); }
  memcpy(b, m->data, m->bytes);
  if (st) { st->MPI_SOURCE = 0; st->MPI_TAG = m->tag; st->MPI_ERROR = 0; st->count = (int)m->bytes; }
  free(m->data);
  free(m);
  return 0;
}

int MPI_Waitall(int n, MPI_Request *q, MPI_Status *st)
{
  for (int k = 0; k < n; k++) {
    int i = q[k];
    if (i <= 0 || i >= NREQ || !reqs[i].used) continue;
    if (!reqs[i].done) { fprintf(stderr, "mpi stub: wait on a receive nobody sends at one rank\n"); exit(3); }
    if (st) { st[k].MPI_SOURCE = 0; st[k].MPI_TAG = reqs[i].tag; st[k].MPI_ERROR = 0; st[k].count = (int)reqs[i].got; }
    reqs[i].used = 0;
    q[k] = 0;
  }
  return 0;
}

int MPI_Probe(int s, int tag, MPI_Comm c, MPI_Status *st)
{
  (void)s; (void)c;
  msg *m = take(tag, 0);
  if (!m) { fprintf(stderr, "mpi stub: probe without a message at one rank\n"); exit(3); }
  if (st) { st->MPI_SOURCE = 0; st->MPI_TAG = m->tag; st->MPI_ERROR = 0; st->count = (int)m->bytes; }
  return 0;
}
