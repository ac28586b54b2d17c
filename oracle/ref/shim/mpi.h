/* Single-process MPI for building HemePure as a CPU oracle (test infrastructure only).
 *
 * Only the subset of MPI-3 the reference's sources name is declared.  Every
 * communicator has exactly one rank; collectives copy the send buffer into the
 * receive buffer through the datatype's type map; point-to-point messages are
 * messages to self, matched in order by (communicator, tag), which is what the
 * Windkessel iolets rely on even on one rank (lb/iolets/BoundaryComms.cc:48-80).
 * MPI-IO maps onto POSIX file descriptors.  Handles are small integers, as in
 * MPICH's ABI.
 */
#ifndef HB_REF_SHIM_MPI_H
#define HB_REF_SHIM_MPI_H

#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
#include "std_headers.h"
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Group;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_Request;
typedef int MPI_Errhandler;
typedef int MPI_Win;
typedef int MPI_File;
typedef intptr_t MPI_Aint;
typedef long long MPI_Offset;

typedef struct MPI_Status {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
  long long count_bytes;
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_ERR_TRUNCATE 14
#define MPI_ERR_FILE 27
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_MAX_ERROR_STRING 256
#define MPI_UNDEFINED (-32766)
#define MPI_ANY_SOURCE (-2)
#define MPI_ANY_TAG (-1)
#define MPI_PROC_NULL (-1)

#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_GROUP_NULL 0
#define MPI_GROUP_EMPTY 1
#define MPI_INFO_NULL 0
#define MPI_REQUEST_NULL 0
#define MPI_WIN_NULL 0
#define MPI_FILE_NULL 0
#define MPI_ERRORS_RETURN 1
#define MPI_ERRORS_ARE_FATAL 2

#define MPI_IDENT 0
#define MPI_CONGRUENT 1
#define MPI_SIMILAR 2
#define MPI_UNEQUAL 3

#define MPI_COMM_TYPE_SHARED 1

/* Predefined datatypes: the handle is an index into the shim's type table. */
#define MPI_DATATYPE_NULL 0
#define MPI_CHAR 1
#define MPI_SIGNED_CHAR 2
#define MPI_UNSIGNED_CHAR 3
#define MPI_SHORT 4
#define MPI_UNSIGNED_SHORT 5
#define MPI_INT 6
#define MPI_UNSIGNED 7
#define MPI_LONG 8
#define MPI_UNSIGNED_LONG 9
#define MPI_LONG_LONG 10
#define MPI_UNSIGNED_LONG_LONG 11
#define MPI_FLOAT 12
#define MPI_DOUBLE 13
#define MPI_LONG_DOUBLE 14
#define MPI_WCHAR 15
#define MPI_BYTE 16
#define MPI_LONG_LONG_INT MPI_LONG_LONG
#define MPI_INT64_T MPI_LONG_LONG
#define MPI_UINT64_T MPI_UNSIGNED_LONG_LONG

#define MPI_OP_NULL 0
#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_SUM 3
#define MPI_PROD 4

#define MPI_MODE_RDONLY 2
#define MPI_MODE_RDWR 8
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1
#define MPI_MODE_EXCL 64
#define MPI_MODE_APPEND 128
#define MPI_SEEK_SET 600
#define MPI_SEEK_CUR 602
#define MPI_SEEK_END 604

#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_BOTTOM ((void*)0)
#define MPI_IN_PLACE ((void*)-1)

int MPI_Init(int* argc, char*** argv);
int MPI_Initialized(int* flag);
int MPI_Finalize(void);
int MPI_Finalized(int* flag);
int MPI_Abort(MPI_Comm comm, int code);
double MPI_Wtime(void);
int MPI_Get_processor_name(char* name, int* len);
int MPI_Error_string(int code, char* str, int* len);
int MPI_Comm_set_errhandler(MPI_Comm comm, MPI_Errhandler h);

int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* out);
int MPI_Comm_free(MPI_Comm* comm);
int MPI_Comm_compare(MPI_Comm a, MPI_Comm b, int* result);
int MPI_Comm_group(MPI_Comm comm, MPI_Group* grp);
int MPI_Comm_create(MPI_Comm comm, MPI_Group grp, MPI_Comm* out);
int MPI_Comm_create_group(MPI_Comm comm, MPI_Group grp, int tag, MPI_Comm* out);
int MPI_Comm_split_type(MPI_Comm comm, int type, int key, MPI_Info info, MPI_Comm* out);
int MPI_Graph_create(MPI_Comm comm, int nnodes, const int index[], const int edges[], int reorder,
                     MPI_Comm* out);
int MPI_Graph_neighbors_count(MPI_Comm comm, int rank, int* n);
int MPI_Graph_neighbors(MPI_Comm comm, int rank, int maxn, int neighbours[]);

int MPI_Group_rank(MPI_Group grp, int* rank);
int MPI_Group_size(MPI_Group grp, int* size);
int MPI_Group_incl(MPI_Group grp, int n, const int ranks[], MPI_Group* out);
int MPI_Group_excl(MPI_Group grp, int n, const int ranks[], MPI_Group* out);
int MPI_Group_free(MPI_Group* grp);

int MPI_Get_address(const void* location, MPI_Aint* address);
int MPI_Type_create_struct(int count, const int blocklengths[], const MPI_Aint displacements[],
                           const MPI_Datatype types[], MPI_Datatype* out);
int MPI_Type_create_resized(MPI_Datatype type, MPI_Aint lb, MPI_Aint extent, MPI_Datatype* out);
int MPI_Type_commit(MPI_Datatype* type);
int MPI_Type_free(MPI_Datatype* type);
int MPI_Type_size(MPI_Datatype type, int* size);
int MPI_Type_get_extent(MPI_Datatype type, MPI_Aint* lb, MPI_Aint* extent);

int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void* buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op, int root,
               MPI_Comm comm);
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op,
                  MPI_Comm comm);
int MPI_Gather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int recvcount,
               MPI_Datatype recvtype, int root, MPI_Comm comm);
int MPI_Gatherv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                const int recvcounts[], const int displs[], MPI_Datatype recvtype, int root,
                MPI_Comm comm);
int MPI_Allgather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                  int recvcount, MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Scatter(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                int recvcount, MPI_Datatype recvtype, int root, MPI_Comm comm);
int MPI_Alltoall(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                 int recvcount, MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Neighbor_allgather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                           int recvcount, MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Neighbor_allgatherv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                            const int recvcounts[], const int displs[], MPI_Datatype recvtype,
                            MPI_Comm comm);

int MPI_Send(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm);
int MPI_Ssend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm,
             MPI_Status* status);
int MPI_Isend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm,
              MPI_Request* req);
int MPI_Irecv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm,
              MPI_Request* req);
int MPI_Wait(MPI_Request* req, MPI_Status* status);
int MPI_Waitall(int count, MPI_Request reqs[], MPI_Status statuses[]);
int MPI_Test(MPI_Request* req, int* flag, MPI_Status* status);
int MPI_Testall(int count, MPI_Request reqs[], int* flag, MPI_Status statuses[]);

int MPI_Info_create(MPI_Info* info);
int MPI_Info_set(MPI_Info info, const char* key, const char* value);
int MPI_Info_free(MPI_Info* info);

int MPI_File_open(MPI_Comm comm, const char* filename, int amode, MPI_Info info, MPI_File* fh);
int MPI_File_close(MPI_File* fh);
int MPI_File_get_size(MPI_File fh, MPI_Offset* size);
int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype, MPI_Datatype filetype,
                      const char* datarep, MPI_Info info);
int MPI_File_read(MPI_File fh, void* buf, int count, MPI_Datatype type, MPI_Status* status);
int MPI_File_read_at(MPI_File fh, MPI_Offset offset, void* buf, int count, MPI_Datatype type,
                     MPI_Status* status);
int MPI_File_write(MPI_File fh, const void* buf, int count, MPI_Datatype type, MPI_Status* status);
int MPI_File_write_at(MPI_File fh, MPI_Offset offset, const void* buf, int count, MPI_Datatype type,
                      MPI_Status* status);
int MPI_File_write_ordered(MPI_File fh, const void* buf, int count, MPI_Datatype type,
                           MPI_Status* status);
int MPI_File_seek_shared(MPI_File fh, MPI_Offset offset, int whence);
int MPI_File_get_position_shared(MPI_File fh, MPI_Offset* offset);

int MPI_Win_allocate_shared(MPI_Aint size, int disp_unit, MPI_Info info, MPI_Comm comm, void* baseptr,
                            MPI_Win* win);
int MPI_Win_shared_query(MPI_Win win, int rank, MPI_Aint* size, int* disp_unit, void* baseptr);
int MPI_Win_fence(int assert_, MPI_Win win);
int MPI_Win_free(MPI_Win* win);

int MPI_Get_count(const MPI_Status* status, MPI_Datatype type, int* count);

#ifdef __cplusplus
}
#endif

#endif
