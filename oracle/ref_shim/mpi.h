/* Stand-in for <mpi.h> used to compile the reference's own sources here.
 *
 * TEST INFRASTRUCTURE ONLY (oracle/_ref): the container has no MPI, and the
 * reference's step loop only needs the handful of calls below.  Semantics:
 *
 *   * One process is one rank.  By default the world has one rank (rank 0 of
 *     1), which is what a single-rank `mpirun -np 1 show` run does: every
 *     Send/Recv in the reference is guarded by rank tests that never fire, and
 *     Allreduce/Reduce/Bcast copy the local buffer.
 *   * FELIS_REF_NRANKS / FELIS_REF_RANK (environment) let one process play rank
 *     r of n for timing only: boundary() then gives it the reference's slice
 *     block (boundary.cpp:33-46) and loadBeam its randskip, but no message
 *     crosses processes: MPI_Send drops its data and MPI_Recv fills zeros, and
 *     the reductions stay local.  The arithmetic per rank is the reference's;
 *     results of such a run are not used for parity.
 *   * MPI_Abort and MPI_Finalize-then-exit paths end the process with the
 *     given code (the driver runs as a child process).
 *
 * The calls the reference makes on its loop and setup path (file:line):
 *   MPI_Comm_rank/size  everywhere; MPI_Barrier fieldShareZ.cpp:67,77,
 *   wakeField.cpp:47,128,157; MPI_Send/Recv fieldShareZ.cpp:60-75,
 *   updateTotalEnergy.cpp:60-67, loadBeam.cpp:257-265; MPI_Allreduce
 *   twiss.cpp:62-64; MPI_Reduce wakeField.cpp:194; MPI_Bcast wakeField.cpp:199;
 *   MPI_Abort particlePush.cpp:67,237,423,512, solveField.cpp:230,444;
 *   MPI_Finalize parameterSetting.cpp:277.
 */
#ifndef FELIS_REF_SHIM_MPI_H
#define FELIS_REF_SHIM_MPI_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef struct {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
} MPI_Status;

#define MPI_COMM_WORLD ((MPI_Comm)1)
#define MPI_INFO_NULL ((MPI_Info)0)
#define MPI_SUCCESS 0

/* datatype codes carry their size in bytes */
#define MPI_CHAR ((MPI_Datatype)0x101)
#define MPI_INT ((MPI_Datatype)0x204)
#define MPI_UNSIGNED ((MPI_Datatype)0x304)
#define MPI_FLOAT ((MPI_Datatype)0x404)
#define MPI_LONG ((MPI_Datatype)0x508)
#define MPI_UNSIGNED_LONG ((MPI_Datatype)0x608)
#define MPI_LONG_LONG ((MPI_Datatype)0x708)
#define MPI_DOUBLE ((MPI_Datatype)0x808)

#define MPI_SUM ((MPI_Op)1)
#define MPI_MAX ((MPI_Op)2)
#define MPI_MIN ((MPI_Op)3)

int MPI_Init(int* argc, char*** argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Barrier(MPI_Comm comm);
int MPI_Send(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Status* status);
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm);
int MPI_Bcast(void* buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Abort(MPI_Comm comm, int code);

#ifdef __cplusplus
}
#endif

#endif
