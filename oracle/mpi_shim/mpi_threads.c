/*
 * Multi-rank stand-in for <mpi.h> (same header, mpi.h), TEST
 * INFRASTRUCTURE: P ranks of one MPI_COMM_WORLD are P threads of one
 * process. It lets the reference's own C physics driver run its multi-rank
 * path -- the ghost exchange of physics_mpi_real_to_ghost
 * (src/physics/src/physics_mpi.c:47-122) every stage, the MIN of the CFL
 * step and the SUM of the residual norm every step -- as the CPU baseline,
 * on a host without an MPI library. Nothing in the product links it.
 *
 * Semantics kept from MPI for the calls the reference makes:
 *   - point to point: MPI_Isend copies the message into the receiver's
 *     mailbox for (source, destination), which is FIFO, so messages between
 *     two ranks are not overtaken (the reference posts one receive per
 *     peer and matches with MPI_ANY_TAG); MPI_Irecv registers the receive
 *     and MPI_Waitall completes this rank's registered receives;
 *   - collectives: every rank deposits its operand, a barrier, every rank
 *     reduces the operands in rank order (so all ranks get the same bits),
 *     a barrier; MPI_Reduce is MPI_Allreduce;
 *   - MPI_DOUBLE_INT pairs with MPI_MINLOC / MPI_MAXLOC (ties: lower index).
 * A receive that waits more than 120 s reports the deadlock and aborts the
 * process instead of hanging.
 */
#include "mpi.h"

#include <errno.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define MT_MAX_RANKS 256
#define MT_MAX_PENDING 1024
#define MT_SLOT_BYTES 64

typedef struct mt_msg {
    struct mt_msg *next;
    int count;
    double data[];
} mt_msg;

typedef struct {
    pthread_mutex_t mu;
    pthread_cond_t cv;
    mt_msg *head[MT_MAX_RANKS];  /* per source: FIFO */
    mt_msg *tail[MT_MAX_RANKS];
} mt_mailbox;

typedef struct {
    void *buf;
    int count;
    int source;
} mt_recv;

static int g_size = 1;
static int g_abort_code = 0;
static mt_mailbox *g_box = NULL;
static pthread_barrier_t g_bar;
static unsigned char g_slot[MT_MAX_RANKS][MT_SLOT_BYTES];
static __thread int t_rank = 0;
static __thread mt_recv t_pending[MT_MAX_PENDING];
static __thread int t_npending = 0;

typedef struct { double v; int i; } mt_double_int;

static size_t type_size(MPI_Datatype t)
{
    switch (t) {
    case MPI_INT:        return sizeof(int);
    case MPI_DOUBLE:     return sizeof(double);
    case MPI_DOUBLE_INT: return sizeof(mt_double_int);
    default:             return 0;
    }
}

/* Set-up of a world of `size` ranks (before the rank threads start). */
int oracle_mt_init(int size)
{
    if (size < 1 || size > MT_MAX_RANKS) return 1;
    g_size = size;
    g_abort_code = 0;
    g_box = (mt_mailbox *)calloc((size_t)size, sizeof(mt_mailbox));
    if (!g_box) return 1;
    for (int r = 0; r < size; r++) {
        pthread_mutex_init(&g_box[r].mu, NULL);
        pthread_cond_init(&g_box[r].cv, NULL);
    }
    return pthread_barrier_init(&g_bar, NULL, (unsigned)size) != 0;
}

void oracle_mt_finalize(void)
{
    if (!g_box) return;
    for (int r = 0; r < g_size; r++) {
        for (int s = 0; s < g_size; s++) {
            mt_msg *m = g_box[r].head[s];
            while (m) {
                mt_msg *n = m->next;
                free(m);
                m = n;
            }
        }
        pthread_mutex_destroy(&g_box[r].mu);
        pthread_cond_destroy(&g_box[r].cv);
    }
    free(g_box);
    g_box = NULL;
    pthread_barrier_destroy(&g_bar);
    g_size = 1;
}

/* The calling thread acts as rank r from now on. */
void oracle_mt_set_rank(int r)
{
    t_rank = r;
    t_npending = 0;
}

int oracle_mpi_take_abort_code(void)
{
    int c = g_abort_code;
    g_abort_code = 0;
    return c;
}

double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1.0e-9 * (double)ts.tv_nsec;
}

int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = t_rank; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = g_size; return MPI_SUCCESS; }

static void reduce_into(void *out, const void *in, int count, MPI_Datatype type, MPI_Op op)
{
    for (int k = 0; k < count; k++) {
        if (type == MPI_INT) {
            int a = ((int *)out)[k], b = ((const int *)in)[k];
            ((int *)out)[k] = op == MPI_SUM ? a + b : op == MPI_MIN ? (b < a ? b : a) : (b > a ? b : a);
        } else if (type == MPI_DOUBLE) {
            double a = ((double *)out)[k], b = ((const double *)in)[k];
            ((double *)out)[k] = op == MPI_SUM ? a + b : op == MPI_MIN ? (b < a ? b : a) : (b > a ? b : a);
        } else {
            mt_double_int *a = &((mt_double_int *)out)[k];
            const mt_double_int *b = &((const mt_double_int *)in)[k];
            int take = op == MPI_MINLOC ? (b->v < a->v || (b->v == a->v && b->i < a->i))
                                        : (b->v > a->v || (b->v == a->v && b->i < a->i));
            if (take) *a = *b;
        }
    }
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm)
{
    (void)comm;
    size_t bytes = (size_t)count * type_size(type);
    if (bytes > MT_SLOT_BYTES) {
        fprintf(stderr, "[mpi threads] collective of %zu bytes exceeds the stand-in's slot\n", bytes);
        abort();
    }
    memcpy(g_slot[t_rank], sendbuf, bytes);
    pthread_barrier_wait(&g_bar);
    unsigned char acc[MT_SLOT_BYTES];
    memcpy(acc, g_slot[0], bytes);
    for (int r = 1; r < g_size; r++) reduce_into(acc, g_slot[r], count, type, op);
    pthread_barrier_wait(&g_bar);
    memcpy(recvbuf, acc, bytes);
    return MPI_SUCCESS;
}

int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op, int root,
               MPI_Comm comm)
{
    (void)root;
    return MPI_Allreduce(sendbuf, recvbuf, count, type, op, comm);
}

int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm,
              MPI_Request *request)
{
    (void)tag; (void)comm;
    if (type != MPI_DOUBLE || dest < 0 || dest >= g_size) abort();
    mt_msg *m = (mt_msg *)malloc(sizeof(mt_msg) + sizeof(double) * (size_t)count);
    if (!m) abort();
    m->next = NULL;
    m->count = count;
    memcpy(m->data, buf, sizeof(double) * (size_t)count);
    mt_mailbox *b = &g_box[dest];
    pthread_mutex_lock(&b->mu);
    if (b->tail[t_rank]) b->tail[t_rank]->next = m;
    else b->head[t_rank] = m;
    b->tail[t_rank] = m;
    pthread_cond_broadcast(&b->cv);
    pthread_mutex_unlock(&b->mu);
    *request = -1;  /* complete: the message was copied */
    return MPI_SUCCESS;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request *request)
{
    (void)tag; (void)comm;
    if (type != MPI_DOUBLE || source < 0 || source >= g_size || t_npending >= MT_MAX_PENDING) abort();
    t_pending[t_npending].buf = buf;
    t_pending[t_npending].count = count;
    t_pending[t_npending].source = source;
    *request = t_npending++;
    return MPI_SUCCESS;
}

int MPI_Waitall(int count, MPI_Request *requests, MPI_Status *statuses)
{
    (void)count; (void)requests; (void)statuses;
    mt_mailbox *b = &g_box[t_rank];
    for (int k = 0; k < t_npending; k++) {
        mt_recv *rq = &t_pending[k];
        pthread_mutex_lock(&b->mu);
        while (!b->head[rq->source]) {
            struct timespec dl;
            clock_gettime(CLOCK_REALTIME, &dl);
            dl.tv_sec += 120;
            if (pthread_cond_timedwait(&b->cv, &b->mu, &dl) == ETIMEDOUT && !b->head[rq->source]) {
                fprintf(stderr, "[mpi threads] rank %d: no message from rank %d in 120 s\n", t_rank, rq->source);
                abort();
            }
        }
        mt_msg *m = b->head[rq->source];
        b->head[rq->source] = m->next;
        if (!m->next) b->tail[rq->source] = NULL;
        pthread_mutex_unlock(&b->mu);
        if (m->count != rq->count) {
            fprintf(stderr, "[mpi threads] rank %d: message of %d doubles from rank %d, receive of %d\n", t_rank,
                    m->count, rq->source, rq->count);
            abort();
        }
        memcpy(rq->buf, m->data, sizeof(double) * (size_t)m->count);
        free(m);
    }
    t_npending = 0;
    return MPI_SUCCESS;
}

int MPI_Abort(MPI_Comm comm, int errorcode)
{
    (void)comm;
    g_abort_code = errorcode;
    fprintf(stderr, "[mpi threads] MPI_Abort(%d) on rank %d\n", errorcode, t_rank);
    return MPI_SUCCESS;
}
