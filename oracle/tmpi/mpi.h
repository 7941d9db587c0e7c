/*
 * mpi.h -- a thread-rank stand-in for the MPI subset the reference's CPU
 * driver calls, so that its own code (RIKEN-RCCS/hpl-ai main.cpp and the
 * headers it includes) runs as one process on one host with no MPI
 * installed.
 *
 * TEST INFRASTRUCTURE ONLY: used by oracle/build_ref.sh to build the
 * reference under oracle/_ref for the oracle's pins and the CPU baseline.
 * The product (libhplai.so, driver.out) neither includes nor links it.
 *
 * Each rank is a std::thread of one process (tmpi.cpp starts TMPI_NP of
 * them, default 4, each running the reference's main).  Semantics:
 *   - point to point: sends are eager (the data is copied at the call);
 *     receives match on (communicator, source, tag) in posting order, as MPI
 *     orders messages between one pair of ranks;
 *   - collectives (Ibcast, Allreduce, Barrier, Comm_split) are matched by a
 *     per-communicator sequence number; the root of an Ibcast deposits a copy
 *     and never blocks, other ranks complete at Wait/Test; Allreduce reduces
 *     the contributions in rank order;
 *   - MPI_PROC_NULL peers complete at once.
 * Only the calls and constants the reference uses are provided.
 */
#ifndef TMPI_MPI_H
#define TMPI_MPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct tmpi_request *MPI_Request;
typedef struct {
	int MPI_SOURCE;
	int MPI_TAG;
	int MPI_ERROR;
} MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_SUCCESS 0
#define MPI_PROC_NULL (-2)
#define MPI_REQUEST_NULL ((MPI_Request)0)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)
#define MPI_MAX_PROCESSOR_NAME 256

enum { MPI_THREAD_SINGLE = 0, MPI_THREAD_FUNNELED = 1, MPI_THREAD_SERIALIZED = 2, MPI_THREAD_MULTIPLE = 3 };
enum {
	MPI_BYTE = 1,
	MPI_CHAR,
	MPI_SHORT,
	MPI_INT,
	MPI_UNSIGNED,
	MPI_FLOAT,
	MPI_DOUBLE,
	MPI_INT64_T,
	MPI_UINT64_T,
	MPI_LONG_LONG
};
enum { MPI_SUM = 1, MPI_MAX, MPI_MIN };

int MPI_Init(int *argc, char ***argv);
int MPI_Init_thread(int *argc, char ***argv, int required, int *provided);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
double MPI_Wtime(void);
int MPI_Get_processor_name(char *name, int *len);

int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm);
int MPI_Comm_free(MPI_Comm *comm);

int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Status *status);
int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag, void *recvbuf,
	int recvcount, MPI_Datatype recvtype, int source, int recvtag, MPI_Comm comm, MPI_Status *status);
int MPI_Wait(MPI_Request *req, MPI_Status *status);
int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *statuses);
int MPI_Test(MPI_Request *req, int *flag, MPI_Status *status);
int MPI_Testall(int count, MPI_Request *reqs, int *flag, MPI_Status *statuses);

int MPI_Ibcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm, MPI_Request *req);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Barrier(MPI_Comm comm);

#ifdef __cplusplus
}
#endif

#endif
