/* Single-rank MPI shim (test infrastructure; see mpi.h).
 *
 * With one rank a collective is a copy from the send to the receive buffer.
 * Point-to-point traffic can only address rank 0 itself: the reference
 * sends itself the stop flag (core/main.c:163-179) and the marker-loader
 * exchange (core/plasma_IO.c:196-220).  A send is matched against posted
 * receives with the same tag; if none is posted its bytes are copied into a
 * mailbox that a later receive drains.  A receive that can never be matched
 * aborts loudly instead of hanging.
 */
#include "mpi.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static size_t type_size (MPI_Datatype t) { return (size_t) (t % 100); }

typedef struct {
   int    used;
   int    done;
   int    is_recv;
   int    tag;
   void  *buf;
   size_t bytes;
} req_t;

typedef struct mail_s {
   int            tag;
   size_t         bytes;
   char          *data;
   struct mail_s *next;
} mail_t;

#define SHIM_MAX_REQ 65536
static req_t   reqs[SHIM_MAX_REQ];
static mail_t *mailbox = NULL;

static void shim_die (const char *what)
{
   fprintf (stderr, "mpi_shim: %s\n", what);
   abort ();
}

static MPI_Request new_req (int is_recv, int tag, void *buf, size_t bytes)
{
   for (long i = 1 ; i < SHIM_MAX_REQ ; ++i) {
      if (!reqs[i].used) {
         reqs[i] = (req_t) {1, 0, is_recv, tag, buf, bytes};
         return (MPI_Request) i;
      }
   }
   shim_die ("request table full");
   return MPI_REQUEST_NULL;
}

/* Delivers a message: to the oldest pending receive with the same tag, else
 * into the mailbox. */
static void deliver (const void *buf, size_t bytes, int tag)
{
   for (long i = 1 ; i < SHIM_MAX_REQ ; ++i) {
      req_t *r = reqs + i;
      if (r->used && r->is_recv && !r->done && (r->tag == tag || r->tag == MPI_ANY_TAG)) {
         if (bytes > r->bytes)
            shim_die ("message truncated");
         memcpy (r->buf, buf, bytes);
         r->bytes = bytes;
         r->done  = 1;
         return;
      }
   }
   mail_t *m = (mail_t *) malloc (sizeof (mail_t));
   m->data = (char *) malloc (bytes ? bytes : 1);
   memcpy (m->data, buf, bytes);
   m->tag = tag;
   m->bytes = bytes;
   m->next = NULL;
   mail_t **tail = &mailbox;
   while (*tail)
      tail = &(*tail)->next;
   *tail = m;
}

/* Takes a matching message from the mailbox; returns 1 on success. */
static int take_mail (void *buf, size_t cap, int tag, size_t *got)
{
   for (mail_t **p = &mailbox ; *p ; p = &(*p)->next) {
      mail_t *m = *p;
      if (m->tag == tag || tag == MPI_ANY_TAG) {
         if (m->bytes > cap)
            shim_die ("message truncated");
         memcpy (buf, m->data, m->bytes);
         *got = m->bytes;
         *p = m->next;
         free (m->data);
         free (m);
         return 1;
      }
   }
   return 0;
}

static void fill_status (MPI_Status *st, int tag, size_t bytes)
{
   if (st) {
      st->MPI_SOURCE = 0;
      st->MPI_TAG = tag;
      st->MPI_ERROR = MPI_SUCCESS;
      st->count_bytes = (int) bytes;
   }
}

int MPI_Init (int *argc, char ***argv) { (void) argc; (void) argv; return MPI_SUCCESS; }
int MPI_Finalize (void) { return MPI_SUCCESS; }
int MPI_Comm_size (MPI_Comm c, int *size) { (void) c; *size = 1; return MPI_SUCCESS; }
int MPI_Comm_rank (MPI_Comm c, int *rank) { (void) c; *rank = 0; return MPI_SUCCESS; }
int MPI_Barrier (MPI_Comm c) { (void) c; return MPI_SUCCESS; }
int MPI_Abort (MPI_Comm c, int code) { (void) c; exit (code); }

int MPI_Get_processor_name (char *name, int *len)
{
   strcpy (name, "localhost");
   *len = (int) strlen (name);
   return MPI_SUCCESS;
}

double MPI_Wtime (void)
{
   struct timespec ts;
   clock_gettime (CLOCK_MONOTONIC, &ts);
   return ts.tv_sec + 1e-9*ts.tv_nsec;
}

int MPI_Alloc_mem (long size, MPI_Info info, void *baseptr)
{
   (void) info;
   *(void **) baseptr = malloc ((size_t) (size > 0 ? size : 1));
   return *(void **) baseptr ? MPI_SUCCESS : 1;
}

int MPI_Free_mem (void *base) { free (base); return MPI_SUCCESS; }

int MPI_Bcast (void *b, int n, MPI_Datatype t, int root, MPI_Comm c)
{
   (void) b; (void) n; (void) t; (void) root; (void) c;
   return MPI_SUCCESS;
}

static void copy_in (const void *s, void *r, size_t bytes)
{
   if (s != MPI_IN_PLACE && s != r)
      memmove (r, s, bytes);
}

int MPI_Reduce (const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c)
{
   (void) op; (void) root; (void) c;
   copy_in (s, r, n*type_size (t));
   return MPI_SUCCESS;
}

int MPI_Allreduce (const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
   (void) op; (void) c;
   copy_in (s, r, n*type_size (t));
   return MPI_SUCCESS;
}

int MPI_Gather (const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, int root, MPI_Comm c)
{
   (void) rn; (void) rt; (void) root; (void) c;
   copy_in (s, r, sn*type_size (st));
   return MPI_SUCCESS;
}

int MPI_Alltoall (const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm c)
{
   (void) rn; (void) rt; (void) c;
   copy_in (s, r, sn*type_size (st));
   return MPI_SUCCESS;
}

int MPI_Isend (const void *buf, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *req)
{
   (void) c;
   if (dest != 0)
      shim_die ("send to a rank other than 0");
   deliver (buf, n*type_size (t), tag);
   MPI_Request h = new_req (0, tag, (void *) buf, n*type_size (t));
   reqs[h].done = 1;
   *req = h;
   return MPI_SUCCESS;
}

int MPI_Send (const void *buf, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c)
{
   (void) c;
   if (dest != 0)
      shim_die ("send to a rank other than 0");
   deliver (buf, n*type_size (t), tag);
   return MPI_SUCCESS;
}

int MPI_Irecv (void *buf, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *req)
{
   (void) c;
   if (src != 0 && src != MPI_ANY_SOURCE)
      shim_die ("receive from a rank other than 0");
   size_t got = 0;
   MPI_Request h = new_req (1, tag, buf, n*type_size (t));
   if (take_mail (buf, n*type_size (t), tag, &got)) {
      reqs[h].done = 1;
      reqs[h].bytes = got;
   }
   *req = h;
   return MPI_SUCCESS;
}

int MPI_Recv (void *buf, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Status *st)
{
   (void) c;
   if (src != 0 && src != MPI_ANY_SOURCE)
      shim_die ("receive from a rank other than 0");
   size_t got = 0;
   if (!take_mail (buf, n*type_size (t), tag, &got))
      shim_die ("blocking receive with no matching message (would deadlock)");
   fill_status (st, tag, got);
   return MPI_SUCCESS;
}

/* Completes request *r if done; returns 1 if it is done (or null). */
static int finish (MPI_Request *r, MPI_Status *st)
{
   if (*r == MPI_REQUEST_NULL) {
      fill_status (st, MPI_ANY_TAG, 0);
      return 1;
   }
   req_t *q = reqs + *r;
   if (!q->done)
      return 0;
   fill_status (st, q->tag, q->bytes);
   q->used = 0;
   *r = MPI_REQUEST_NULL;
   return 1;
}

int MPI_Test (MPI_Request *r, int *flag, MPI_Status *st)
{
   *flag = finish (r, st);
   return MPI_SUCCESS;
}

int MPI_Wait (MPI_Request *r, MPI_Status *st)
{
   if (!finish (r, st))
      shim_die ("wait on a receive nobody can satisfy (would deadlock)");
   return MPI_SUCCESS;
}

int MPI_Testany (int n, MPI_Request *rs, int *idx, int *flag, MPI_Status *st)
{
   int active = 0;
   for (int i = 0 ; i < n ; ++i) {
      if (rs[i] == MPI_REQUEST_NULL)
         continue;
      active = 1;
      if (finish (rs + i, st)) {
         *idx = i;
         *flag = 1;
         return MPI_SUCCESS;
      }
   }
   *idx = MPI_UNDEFINED;
   *flag = !active;
   return MPI_SUCCESS;
}

int MPI_Waitany (int n, MPI_Request *rs, int *idx, MPI_Status *st)
{
   int flag = 0;
   MPI_Testany (n, rs, idx, &flag, st);
   if (!flag)
      shim_die ("waitany on receives nobody can satisfy (would deadlock)");
   return MPI_SUCCESS;
}

int MPI_Waitall (int n, MPI_Request *rs, MPI_Status *sts)
{
   for (int i = 0 ; i < n ; ++i)
      if (!finish (rs + i, sts ? sts + i : NULL))
         shim_die ("waitall on a receive nobody can satisfy (would deadlock)");
   return MPI_SUCCESS;
}
