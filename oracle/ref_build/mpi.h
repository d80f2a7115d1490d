// Single-rank MPI subset for compiling the reference's solver sources
// (src/*.cpp) without an MPI library: the declarations those sources use,
// with the semantics of a communicator of size 1 (oracle/ref_build/
// mpi_shim.cpp).  Collectives copy the send buffer to the receive buffer;
// point-to-point and persistent requests, which a one-rank all-to-all
// solve never posts, abort with a message.  Test infrastructure of the
// oracle only.
#pragma once
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Group;
typedef int MPI_Info;
typedef int MPI_Request;
typedef long MPI_Aint;
typedef long long MPI_Offset;
typedef struct {
    int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;
typedef struct mpi_shim_file* MPI_File;

#define MPI_SUCCESS 0
#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_GROUP_NULL 0
#define MPI_INFO_NULL 0
#define MPI_REQUEST_NULL 0
#define MPI_UNDEFINED (-32766)
#define MPI_IDENT 0
#define MPI_CONGRUENT 1
#define MPI_SIMILAR 2
#define MPI_UNEQUAL 3
#define MPI_CART 1
#define MPI_GRAPH 2
#define MPI_DIST_GRAPH 3
#define MPI_COMM_TYPE_SHARED 1
#define MPI_MAX_OBJECT_NAME 128
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_UNWEIGHTED ((int*)1)
#define MPI_WEIGHTS_EMPTY ((int*)2)
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1
#define MPI_MODE_EXCL 64
#define MPI_SEEK_SET 600
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1

// predefined datatypes (handle = index into the size table of mpi_shim.cpp)
#define MPI_CHAR 1
#define MPI_INT 2
#define MPI_LONG 3
#define MPI_UNSIGNED_LONG 4
#define MPI_DOUBLE 5
#define MPI_LONG_INT 6
#define MPI_CXX_BOOL 7
#define MPI_BYTE 8

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_MAXLOC 4
#define MPI_MINLOC 5
#define MPI_LAND 6
#define MPI_LOR 7

int MPI_Init(int* argc, char*** argv);
int MPI_Init_thread(int* argc, char*** argv, int required, int* provided);
int MPI_Initialized(int* flag);
int MPI_Finalize(void);
double MPI_Wtime(void);

int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* newcomm);
int MPI_Comm_free(MPI_Comm* comm);
int MPI_Comm_compare(MPI_Comm a, MPI_Comm b, int* result);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm* newcomm);
int MPI_Comm_split_type(MPI_Comm comm, int type, int key, MPI_Info info, MPI_Comm* newcomm);
int MPI_Comm_create(MPI_Comm comm, MPI_Group group, MPI_Comm* newcomm);
int MPI_Comm_group(MPI_Comm comm, MPI_Group* group);
int MPI_Comm_set_name(MPI_Comm comm, const char* name);
int MPI_Comm_get_name(MPI_Comm comm, char* name, int* len);
int MPI_Comm_set_info(MPI_Comm comm, MPI_Info info);
int MPI_Topo_test(MPI_Comm comm, int* status);
int MPI_Cart_create(MPI_Comm comm, int ndims, const int* dims, const int* periods, int reorder, MPI_Comm* newcomm);
int MPI_Cart_sub(MPI_Comm comm, const int* remain, MPI_Comm* newcomm);
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int* coords);
int MPI_Cart_rank(MPI_Comm comm, const int* coords, int* rank);
int MPI_Dist_graph_create(MPI_Comm comm, int n, const int* sources, const int* degrees, const int* destinations,
                          const int* weights, MPI_Info info, int reorder, MPI_Comm* newcomm);
int MPI_Dist_graph_create_adjacent(MPI_Comm comm, int indegree, const int* sources, const int* sourceweights, int outdegree,
                                   const int* destinations, const int* destweights, MPI_Info info, int reorder,
                                   MPI_Comm* newcomm);
int MPI_Dist_graph_neighbors_count(MPI_Comm comm, int* indegree, int* outdegree, int* weighted);
int MPI_Dist_graph_neighbors(MPI_Comm comm, int maxindegree, int* sources, int* sourceweights, int maxoutdegree,
                             int* destinations, int* destweights);

int MPI_Group_incl(MPI_Group group, int n, const int* ranks, MPI_Group* newgroup);
int MPI_Group_free(MPI_Group* group);
int MPI_Group_translate_ranks(MPI_Group a, int n, const int* ranks_a, MPI_Group b, int* ranks_b);

int MPI_Info_create(MPI_Info* info);
int MPI_Info_set(MPI_Info info, const char* key, const char* value);
int MPI_Info_free(MPI_Info* info);

int MPI_Type_vector(int count, int blocklength, int stride, MPI_Datatype old, MPI_Datatype* newtype);
int MPI_Type_create_hvector(int count, int blocklength, MPI_Aint stride, MPI_Datatype old, MPI_Datatype* newtype);
int MPI_Type_dup(MPI_Datatype old, MPI_Datatype* newtype);
int MPI_Type_commit(MPI_Datatype* type);
int MPI_Type_free(MPI_Datatype* type);

int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void* buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Reduce(const void* send, void* recv, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm);
int MPI_Allreduce(const void* send, void* recv, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Scan(const void* send, void* recv, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Gather(const void* send, int scount, MPI_Datatype stype, void* recv, int rcount, MPI_Datatype rtype, int root,
               MPI_Comm comm);
int MPI_Gatherv(const void* send, int scount, MPI_Datatype stype, void* recv, const int* rcounts, const int* displs,
                MPI_Datatype rtype, int root, MPI_Comm comm);
int MPI_Allgather(const void* send, int scount, MPI_Datatype stype, void* recv, int rcount, MPI_Datatype rtype,
                  MPI_Comm comm);
int MPI_Alltoall(const void* send, int scount, MPI_Datatype stype, void* recv, int rcount, MPI_Datatype rtype,
                 MPI_Comm comm);
int MPI_Alltoallv(const void* send, const int* scounts, const int* sdispls, MPI_Datatype stype, void* recv,
                  const int* rcounts, const int* rdispls, MPI_Datatype rtype, MPI_Comm comm);
int MPI_Ialltoallv(const void* send, const int* scounts, const int* sdispls, MPI_Datatype stype, void* recv,
                   const int* rcounts, const int* rdispls, MPI_Datatype rtype, MPI_Comm comm, MPI_Request* req);

int MPI_Isend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Irecv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Send_init(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Recv_init(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Start(MPI_Request* req);
int MPI_Startall(int n, MPI_Request* reqs);
int MPI_Wait(MPI_Request* req, MPI_Status* status);
int MPI_Waitall(int n, MPI_Request* reqs, MPI_Status* statuses);
int MPI_Waitany(int n, MPI_Request* reqs, int* index, MPI_Status* status);
int MPI_Testsome(int n, MPI_Request* reqs, int* outcount, int* indices, MPI_Status* statuses);
int MPI_Request_free(MPI_Request* req);

int MPI_File_open(MPI_Comm comm, const char* filename, int amode, MPI_Info info, MPI_File* fh);
int MPI_File_seek(MPI_File fh, MPI_Offset offset, int whence);
int MPI_File_write_at(MPI_File fh, MPI_Offset offset, const void* buf, int count, MPI_Datatype type, MPI_Status* status);
int MPI_File_close(MPI_File* fh);

#ifdef __cplusplus
}
#endif
