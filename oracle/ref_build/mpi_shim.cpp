// One-rank semantics behind oracle/ref_build/mpi.h: every communicator has
// size 1 and rank 0, a collective copies the send buffer to the receive
// buffer (predefined datatypes only), a request completes when it is
// posted.  Derived datatypes exist as handles so that the reference can
// build and free them; moving data with one, and point-to-point or
// persistent requests, abort: the reference's all-to-all solve on one rank
// does neither.  Test infrastructure of the oracle only.
#include "mpi.h"

#include <string.h>
#include <sys/time.h>

#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>

namespace {

std::mutex g_mu;
int g_next_comm = 2;
int g_next_type = 100;
std::map<int, std::string> g_names;
std::map<int, int> g_topo;  // communicator -> MPI_CART / MPI_DIST_GRAPH

size_t type_size(MPI_Datatype t) {
    switch (t) {
        case MPI_CHAR: return 1;
        case MPI_INT: return sizeof(int);
        case MPI_LONG: return sizeof(long);
        case MPI_UNSIGNED_LONG: return sizeof(unsigned long);
        case MPI_DOUBLE: return sizeof(double);
        case MPI_LONG_INT: {
            struct li {
                long v;
                int i;
            };
            return sizeof(li);
        }
        case MPI_CXX_BOOL: return sizeof(bool);
        case MPI_BYTE: return 1;
    }
    std::fprintf(stderr, "mpi shim: data moved with derived datatype %d (not provided on one rank)\n", t);
    std::abort();
}

[[noreturn]] void unsupported(const char* what) {
    std::fprintf(stderr, "mpi shim: %s is not provided by the one-rank stand-in\n", what);
    std::abort();
}

int new_comm(int topo) {
    std::lock_guard<std::mutex> lk(g_mu);
    const int c = g_next_comm++;
    if (topo) g_topo[c] = topo;
    return c;
}

void copy(const void* send, void* recv, size_t bytes) {
    if (send != recv && bytes) memmove(recv, send, bytes);
}

}  // namespace

extern "C" {

int MPI_Init(int*, char***) { return MPI_SUCCESS; }
int MPI_Init_thread(int*, char***, int required, int* provided) {
    if (provided) *provided = required;
    return MPI_SUCCESS;
}
int MPI_Initialized(int* flag) {
    *flag = 1;
    return MPI_SUCCESS;
}
int MPI_Finalize(void) { return MPI_SUCCESS; }
double MPI_Wtime(void) {
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    return (double)tv.tv_sec + 1e-6 * (double)tv.tv_usec;
}

int MPI_Comm_size(MPI_Comm, int* size) {
    *size = 1;
    return MPI_SUCCESS;
}
int MPI_Comm_rank(MPI_Comm, int* rank) {
    *rank = 0;
    return MPI_SUCCESS;
}
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* newcomm) {
    int topo = 0;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_topo.find(comm);
        if (it != g_topo.end()) topo = it->second;
    }
    *newcomm = new_comm(topo);
    return MPI_SUCCESS;
}
int MPI_Comm_free(MPI_Comm* comm) {
    *comm = MPI_COMM_NULL;
    return MPI_SUCCESS;
}
int MPI_Comm_compare(MPI_Comm a, MPI_Comm b, int* result) {
    *result = (a == b) ? MPI_IDENT : MPI_CONGRUENT;
    return MPI_SUCCESS;
}
int MPI_Comm_split(MPI_Comm, int color, int, MPI_Comm* newcomm) {
    *newcomm = (color == MPI_UNDEFINED) ? MPI_COMM_NULL : new_comm(0);
    return MPI_SUCCESS;
}
int MPI_Comm_split_type(MPI_Comm, int type, int, MPI_Info, MPI_Comm* newcomm) {
    *newcomm = (type == MPI_UNDEFINED) ? MPI_COMM_NULL : new_comm(0);
    return MPI_SUCCESS;
}
int MPI_Comm_create(MPI_Comm, MPI_Group group, MPI_Comm* newcomm) {
    *newcomm = (group == MPI_GROUP_NULL) ? MPI_COMM_NULL : new_comm(0);
    return MPI_SUCCESS;
}
int MPI_Comm_group(MPI_Comm, MPI_Group* group) {
    *group = 1;
    return MPI_SUCCESS;
}
int MPI_Comm_set_name(MPI_Comm comm, const char* name) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_names[comm] = name;
    return MPI_SUCCESS;
}
int MPI_Comm_get_name(MPI_Comm comm, char* name, int* len) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_names.find(comm);
    std::string s = (it != g_names.end()) ? it->second : (comm == MPI_COMM_WORLD ? "MPI_COMM_WORLD" : "");
    if (s.size() >= MPI_MAX_OBJECT_NAME) s.resize(MPI_MAX_OBJECT_NAME - 1);
    memcpy(name, s.c_str(), s.size() + 1);
    *len = (int)s.size();
    return MPI_SUCCESS;
}
int MPI_Comm_set_info(MPI_Comm, MPI_Info) { return MPI_SUCCESS; }
int MPI_Topo_test(MPI_Comm comm, int* status) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_topo.find(comm);
    *status = (it != g_topo.end()) ? it->second : MPI_UNDEFINED;
    return MPI_SUCCESS;
}
int MPI_Cart_create(MPI_Comm, int ndims, const int* dims, const int*, int, MPI_Comm* newcomm) {
    int n = 1;
    for (int i = 0; i < ndims; ++i) n *= dims[i];
    if (n != 1) unsupported("a Cartesian grid of more than one rank");
    *newcomm = new_comm(MPI_CART);
    return MPI_SUCCESS;
}
int MPI_Cart_sub(MPI_Comm, const int*, MPI_Comm* newcomm) {
    *newcomm = new_comm(MPI_CART);
    return MPI_SUCCESS;
}
int MPI_Cart_coords(MPI_Comm, int, int maxdims, int* coords) {
    for (int i = 0; i < maxdims; ++i) coords[i] = 0;
    return MPI_SUCCESS;
}
int MPI_Cart_rank(MPI_Comm, const int*, int* rank) {
    *rank = 0;
    return MPI_SUCCESS;
}
int MPI_Dist_graph_create(MPI_Comm, int, const int*, const int*, const int*, const int*, MPI_Info, int, MPI_Comm* newcomm) {
    *newcomm = new_comm(MPI_DIST_GRAPH);
    return MPI_SUCCESS;
}
int MPI_Dist_graph_create_adjacent(MPI_Comm, int, const int*, const int*, int, const int*, const int*, MPI_Info, int,
                                   MPI_Comm* newcomm) {
    *newcomm = new_comm(MPI_DIST_GRAPH);
    return MPI_SUCCESS;
}
int MPI_Dist_graph_neighbors_count(MPI_Comm, int* indegree, int* outdegree, int* weighted) {
    *indegree = 0;
    *outdegree = 0;
    *weighted = 0;
    return MPI_SUCCESS;
}
int MPI_Dist_graph_neighbors(MPI_Comm, int, int*, int*, int, int*, int*) { return MPI_SUCCESS; }

int MPI_Group_incl(MPI_Group, int n, const int*, MPI_Group* newgroup) {
    *newgroup = (n > 0) ? 1 : MPI_GROUP_NULL;
    return MPI_SUCCESS;
}
int MPI_Group_free(MPI_Group* group) {
    *group = MPI_GROUP_NULL;
    return MPI_SUCCESS;
}
int MPI_Group_translate_ranks(MPI_Group, int n, const int* ranks_a, MPI_Group, int* ranks_b) {
    for (int i = 0; i < n; ++i) ranks_b[i] = (ranks_a[i] == 0) ? 0 : MPI_UNDEFINED;
    return MPI_SUCCESS;
}

int MPI_Info_create(MPI_Info* info) {
    *info = 1;
    return MPI_SUCCESS;
}
int MPI_Info_set(MPI_Info, const char*, const char*) { return MPI_SUCCESS; }
int MPI_Info_free(MPI_Info* info) {
    *info = MPI_INFO_NULL;
    return MPI_SUCCESS;
}

static int new_type(MPI_Datatype* t) {
    std::lock_guard<std::mutex> lk(g_mu);
    *t = g_next_type++;
    return MPI_SUCCESS;
}
int MPI_Type_vector(int, int, int, MPI_Datatype, MPI_Datatype* newtype) { return new_type(newtype); }
int MPI_Type_create_hvector(int, int, MPI_Aint, MPI_Datatype, MPI_Datatype* newtype) { return new_type(newtype); }
int MPI_Type_dup(MPI_Datatype, MPI_Datatype* newtype) { return new_type(newtype); }
int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
int MPI_Type_free(MPI_Datatype* type) {
    *type = 0;
    return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
int MPI_Reduce(const void* send, void* recv, int count, MPI_Datatype type, MPI_Op, int, MPI_Comm) {
    copy(send, recv, (size_t)count * type_size(type));
    return MPI_SUCCESS;
}
int MPI_Allreduce(const void* send, void* recv, int count, MPI_Datatype type, MPI_Op, MPI_Comm) {
    copy(send, recv, (size_t)count * type_size(type));
    return MPI_SUCCESS;
}
int MPI_Scan(const void* send, void* recv, int count, MPI_Datatype type, MPI_Op, MPI_Comm) {
    copy(send, recv, (size_t)count * type_size(type));
    return MPI_SUCCESS;
}
int MPI_Gather(const void* send, int scount, MPI_Datatype stype, void* recv, int, MPI_Datatype, int, MPI_Comm) {
    copy(send, recv, (size_t)scount * type_size(stype));
    return MPI_SUCCESS;
}
int MPI_Gatherv(const void* send, int scount, MPI_Datatype stype, void* recv, const int*, const int* displs,
                MPI_Datatype rtype, int, MPI_Comm) {
    copy(send, (char*)recv + (size_t)displs[0] * type_size(rtype), (size_t)scount * type_size(stype));
    return MPI_SUCCESS;
}
int MPI_Allgather(const void* send, int scount, MPI_Datatype stype, void* recv, int, MPI_Datatype, MPI_Comm) {
    copy(send, recv, (size_t)scount * type_size(stype));
    return MPI_SUCCESS;
}
int MPI_Alltoall(const void* send, int scount, MPI_Datatype stype, void* recv, int, MPI_Datatype, MPI_Comm) {
    copy(send, recv, (size_t)scount * type_size(stype));
    return MPI_SUCCESS;
}
int MPI_Alltoallv(const void* send, const int* scounts, const int* sdispls, MPI_Datatype stype, void* recv, const int*,
                  const int* rdispls, MPI_Datatype rtype, MPI_Comm) {
    copy((const char*)send + (size_t)sdispls[0] * type_size(stype), (char*)recv + (size_t)rdispls[0] * type_size(rtype),
         (size_t)scounts[0] * type_size(stype));
    return MPI_SUCCESS;
}
int MPI_Ialltoallv(const void* send, const int* scounts, const int* sdispls, MPI_Datatype stype, void* recv,
                   const int* rcounts, const int* rdispls, MPI_Datatype rtype, MPI_Comm comm, MPI_Request* req) {
    *req = MPI_REQUEST_NULL;
    return MPI_Alltoallv(send, scounts, sdispls, stype, recv, rcounts, rdispls, rtype, comm);
}

int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { unsupported("MPI_Isend"); }
int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { unsupported("MPI_Irecv"); }
int MPI_Send_init(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { unsupported("MPI_Send_init"); }
int MPI_Recv_init(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { unsupported("MPI_Recv_init"); }
int MPI_Start(MPI_Request*) { unsupported("MPI_Start"); }
int MPI_Startall(int n, MPI_Request*) {
    if (n > 0) unsupported("MPI_Startall");
    return MPI_SUCCESS;
}
int MPI_Wait(MPI_Request* req, MPI_Status*) {
    *req = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}
int MPI_Waitall(int n, MPI_Request* reqs, MPI_Status*) {
    for (int i = 0; i < n; ++i) reqs[i] = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}
int MPI_Waitany(int, MPI_Request*, int* index, MPI_Status*) {
    *index = MPI_UNDEFINED;
    return MPI_SUCCESS;
}
int MPI_Testsome(int, MPI_Request*, int* outcount, int*, MPI_Status*) {
    *outcount = MPI_UNDEFINED;
    return MPI_SUCCESS;
}
int MPI_Request_free(MPI_Request* req) {
    *req = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}

}  // extern "C"

struct mpi_shim_file {
    FILE* f;
};

extern "C" {

int MPI_File_open(MPI_Comm, const char* filename, int amode, MPI_Info, MPI_File* fh) {
    if ((amode & MPI_MODE_EXCL) && (amode & MPI_MODE_CREATE)) {
        if (FILE* e = std::fopen(filename, "rb")) {
            std::fclose(e);
            return 1;
        }
    }
    FILE* f = std::fopen(filename, "wb");
    if (!f) return 1;
    *fh = new mpi_shim_file{f};
    return MPI_SUCCESS;
}
int MPI_File_seek(MPI_File fh, MPI_Offset offset, int) { return std::fseek(fh->f, (long)offset, SEEK_SET) == 0 ? 0 : 1; }
int MPI_File_write_at(MPI_File fh, MPI_Offset offset, const void* buf, int count, MPI_Datatype type, MPI_Status*) {
    std::fseek(fh->f, (long)offset, SEEK_SET);
    std::fwrite(buf, type_size(type), (size_t)count, fh->f);
    return MPI_SUCCESS;
}
int MPI_File_close(MPI_File* fh) {
    std::fclose((*fh)->f);
    delete *fh;
    *fh = nullptr;
    return MPI_SUCCESS;
}

}  // extern "C"
