/*
 * Single-process MPI stand-in for the reference build (test infrastructure).
 * Collectives copy the caller's buffer; probes report no message; any
 * point-to-point transfer aborts, since one rank owns every column.
 */
#include "mpi.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static size_t type_size(MPI_Datatype t)
{
    switch (t) {
    case MPI_INT:
    case MPI_UNSIGNED:
        return 4;
    case MPI_DOUBLE:
    case MPI_LONG:
        return 8;
    case MPI_CHAR:
        return 1;
    default:
        if (t >= 1000)
            return (size_t)(t - 1000);
        fprintf(stderr, "mpi shim: unknown datatype %d\n", t);
        abort();
    }
}

static void no_p2p(const char* what)
{
    fprintf(stderr, "mpi shim: %s reached in a single-rank run\n", what);
    abort();
}

int MPI_Init(int* argc, char*** argv)
{
    (void)argc;
    (void)argv;
    return 0;
}
int MPI_Finalize(void) { return 0; }
int MPI_Comm_size(MPI_Comm comm, int* size)
{
    (void)comm;
    *size = 1;
    return 0;
}
int MPI_Comm_rank(MPI_Comm comm, int* rank)
{
    (void)comm;
    *rank = 0;
    return 0;
}
int MPI_Barrier(MPI_Comm comm)
{
    (void)comm;
    return 0;
}
double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int MPI_Allgather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                  int recvcount, MPI_Datatype recvtype, MPI_Comm comm)
{
    (void)recvcount;
    (void)recvtype;
    (void)comm;
    memmove(recvbuf, sendbuf, (size_t)sendcount * type_size(sendtype));
    return 0;
}
int MPI_Allgatherv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                   const int* recvcounts, const int* displs, MPI_Datatype recvtype,
                   MPI_Comm comm)
{
    (void)recvcounts;
    (void)comm;
    memmove((char*)recvbuf + (size_t)displs[0] * type_size(recvtype), sendbuf,
            (size_t)sendcount * type_size(sendtype));
    return 0;
}
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype datatype,
                  MPI_Op op, MPI_Comm comm)
{
    (void)op;
    (void)comm;
    memmove(recvbuf, sendbuf, (size_t)count * type_size(datatype));
    return 0;
}
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype datatype, MPI_Op op,
               int root, MPI_Comm comm)
{
    (void)op;
    (void)root;
    (void)comm;
    memmove(recvbuf, sendbuf, (size_t)count * type_size(datatype));
    return 0;
}
int MPI_Scan(const void* sendbuf, void* recvbuf, int count, MPI_Datatype datatype, MPI_Op op,
             MPI_Comm comm)
{
    (void)op;
    (void)comm;
    memmove(recvbuf, sendbuf, (size_t)count * type_size(datatype));
    return 0;
}
int MPI_Gather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
               int recvcount, MPI_Datatype recvtype, int root, MPI_Comm comm)
{
    (void)recvcount;
    (void)recvtype;
    (void)root;
    (void)comm;
    memmove(recvbuf, sendbuf, (size_t)sendcount * type_size(sendtype));
    return 0;
}
int MPI_Bcast(void* buffer, int count, MPI_Datatype datatype, int root, MPI_Comm comm)
{
    (void)buffer;
    (void)count;
    (void)datatype;
    (void)root;
    (void)comm;
    return 0;
}

int MPI_Send(const void* buf, int count, MPI_Datatype datatype, int dest, int tag,
             MPI_Comm comm)
{
    (void)buf, (void)count, (void)datatype, (void)dest, (void)tag, (void)comm;
    no_p2p("MPI_Send");
    return 1;
}
int MPI_Isend(const void* buf, int count, MPI_Datatype datatype, int dest, int tag,
              MPI_Comm comm, MPI_Request* request)
{
    (void)buf, (void)count, (void)datatype, (void)dest, (void)tag, (void)comm, (void)request;
    no_p2p("MPI_Isend");
    return 1;
}
int MPI_Recv(void* buf, int count, MPI_Datatype datatype, int source, int tag, MPI_Comm comm,
             MPI_Status* status)
{
    (void)buf, (void)count, (void)datatype, (void)source, (void)tag, (void)comm, (void)status;
    no_p2p("MPI_Recv");
    return 1;
}
int MPI_Irecv(void* buf, int count, MPI_Datatype datatype, int source, int tag,
              MPI_Comm comm, MPI_Request* request)
{
    (void)buf, (void)count, (void)datatype, (void)source, (void)tag, (void)comm, (void)request;
    no_p2p("MPI_Irecv");
    return 1;
}
int MPI_Test(MPI_Request* request, int* flag, MPI_Status* status)
{
    (void)request;
    (void)status;
    *flag = 1;
    return 0;
}
int MPI_Testall(int count, MPI_Request* requests, int* flag, MPI_Status* statuses)
{
    (void)count;
    (void)requests;
    (void)statuses;
    *flag = 1;
    return 0;
}
int MPI_Wait(MPI_Request* request, MPI_Status* status)
{
    (void)request;
    (void)status;
    return 0;
}
int MPI_Iprobe(int source, int tag, MPI_Comm comm, int* flag, MPI_Status* status)
{
    (void)source;
    (void)tag;
    (void)comm;
    (void)status;
    *flag = 0;
    return 0;
}
int MPI_Type_contiguous(int count, MPI_Datatype oldtype, MPI_Datatype* newtype)
{
    *newtype = (MPI_Datatype)(1000 + (size_t)count * type_size(oldtype));
    return 0;
}
int MPI_Type_commit(MPI_Datatype* datatype)
{
    (void)datatype;
    return 0;
}
