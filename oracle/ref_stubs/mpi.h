/* Declarations only, so that the reference's src/interp3.cpp compiles without
 * an MPI installation (test infrastructure: oracle/build_ref.py).  The
 * single-process shim (oracle/ref_shim.cpp) defines the functions; none of
 * them is reached by the interpolation kernels it calls. */
#pragma once
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef struct { int s; } MPI_Status;
#define MPI_REQUEST_NULL 0
#define MPI_DOUBLE 1
#define MPI_FLOAT 2
#define MPI_INT 3
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_COMM_WORLD 0
int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*);
int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*);
int MPI_Wait(MPI_Request*, MPI_Status*);
int MPI_Type_vector(int, int, int, MPI_Datatype, MPI_Datatype*);
int MPI_Type_commit(MPI_Datatype*);
int MPI_Type_free(MPI_Datatype*);
int MPI_Comm_size(MPI_Comm, int*);
int MPI_Comm_rank(MPI_Comm, int*);
int MPI_Alltoall(const void*, int, MPI_Datatype, void*, int, MPI_Datatype, MPI_Comm);
