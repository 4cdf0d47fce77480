/*
 * Single-process stand-in for <mpi.h>, used ONLY to build the reference
 * Shadowfax flux-pass sources into the CPU oracle harness (test
 * infrastructure, never part of the product library).
 *
 * Semantics: one rank (rank 0 of size 1).  Collectives copy the send buffer
 * into the receive buffer; pack/unpack are plain memcpy with the datatype's
 * byte size.  Point-to-point calls are never reached by the reference code at
 * size 1 (every halo routine returns early when MPIGlobal::size < 2), so they
 * abort loudly if they are.
 */
#ifndef SFX_SHIM_MPI_H
#define SFX_SHIM_MPI_H

#include <cstdio>
#include <cstdlib>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Errhandler;

struct MPI_Status {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
    int count_bytes;
};

#define MPI_SUCCESS 0
#define MPI_ERR_COMM 5
#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_REQUEST_NULL 0
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_ERRORS_RETURN 1
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)

/* datatypes: the value is the element size in bytes times 16 plus a tag so
 * that types of equal size stay distinct */
#define MPI_CHAR (1 * 16 + 0)
#define MPI_PACKED (1 * 16 + 1)
#define MPI_INT (4 * 16 + 0)
#define MPI_UNSIGNED (4 * 16 + 1)
#define MPI_LONG (8 * 16 + 0)
#define MPI_UNSIGNED_LONG (8 * 16 + 1)
#define MPI_DOUBLE (8 * 16 + 2)

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

static inline int sfx_shim_typesize(MPI_Datatype t) {
    return t / 16;
}

static inline void sfx_shim_unreachable(const char* what) {
    std::fprintf(stderr, "single-rank MPI shim: %s is not available\n", what);
    std::abort();
}

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Finalize() { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int* rank) {
    *rank = 0;
    return MPI_SUCCESS;
}
static inline int MPI_Comm_size(MPI_Comm, int* size) {
    *size = 1;
    return MPI_SUCCESS;
}
static inline int MPI_Abort(MPI_Comm, int code) {
    std::exit(code ? code : 1);
    return MPI_SUCCESS;
}
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) {
    return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t,
                                MPI_Op, MPI_Comm) {
    if(s != r) std::memmove(r, s, (size_t)n * sfx_shim_typesize(t));
    return MPI_SUCCESS;
}
static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t,
                             MPI_Op, int, MPI_Comm) {
    if(s != r) std::memmove(r, s, (size_t)n * sfx_shim_typesize(t));
    return MPI_SUCCESS;
}
static inline int MPI_Scan(const void* s, void* r, int n, MPI_Datatype t,
                           MPI_Op, MPI_Comm) {
    if(s != r) std::memmove(r, s, (size_t)n * sfx_shim_typesize(t));
    return MPI_SUCCESS;
}
static inline int MPI_Exscan(const void*, void*, int, MPI_Datatype, MPI_Op,
                             MPI_Comm) {
    return MPI_SUCCESS;
}
static inline int MPI_Allgather(const void* s, int n, MPI_Datatype t, void* r,
                                int, MPI_Datatype, MPI_Comm) {
    if(s != r) std::memmove(r, s, (size_t)n * sfx_shim_typesize(t));
    return MPI_SUCCESS;
}
static inline int MPI_Gather(const void* s, int n, MPI_Datatype t, void* r,
                             int, MPI_Datatype, int, MPI_Comm) {
    if(s != r) std::memmove(r, s, (size_t)n * sfx_shim_typesize(t));
    return MPI_SUCCESS;
}
static inline int MPI_Pack(const void* in, int n, MPI_Datatype t, void* out,
                           int, int* pos, MPI_Comm) {
    size_t b = (size_t)n * sfx_shim_typesize(t);
    std::memcpy((char*)out + *pos, in, b);
    *pos += (int)b;
    return MPI_SUCCESS;
}
static inline int MPI_Unpack(const void* in, int, int* pos, void* out, int n,
                             MPI_Datatype t, MPI_Comm) {
    size_t b = (size_t)n * sfx_shim_typesize(t);
    std::memcpy(out, (const char*)in + *pos, b);
    *pos += (int)b;
    return MPI_SUCCESS;
}
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm,
                            MPI_Request*) {
    sfx_shim_unreachable("MPI_Isend");
    return MPI_SUCCESS;
}
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm,
                            MPI_Request*) {
    sfx_shim_unreachable("MPI_Irecv");
    return MPI_SUCCESS;
}
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm,
                           MPI_Status*) {
    sfx_shim_unreachable("MPI_Recv");
    return MPI_SUCCESS;
}
static inline int MPI_Probe(int, int, MPI_Comm, MPI_Status*) {
    sfx_shim_unreachable("MPI_Probe");
    return MPI_SUCCESS;
}
static inline int MPI_Iprobe(int, int, MPI_Comm, int* flag, MPI_Status*) {
    *flag = 0;
    return MPI_SUCCESS;
}
static inline int MPI_Get_count(const MPI_Status* st, MPI_Datatype t,
                                int* n) {
    *n = st ? st->count_bytes / sfx_shim_typesize(t) : 0;
    return MPI_SUCCESS;
}
static inline int MPI_Test(MPI_Request*, int* flag, MPI_Status*) {
    *flag = 1;
    return MPI_SUCCESS;
}
static inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) {
    return MPI_SUCCESS;
}
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm* out) {
    *out = c;
    return MPI_SUCCESS;
}
static inline int MPI_Comm_free(MPI_Comm* c) {
    *c = MPI_COMM_NULL;
    return MPI_SUCCESS;
}
static inline int MPI_Comm_split(MPI_Comm c, int, int, MPI_Comm* out) {
    *out = c;
    return MPI_SUCCESS;
}
static inline int MPI_Comm_set_errhandler(MPI_Comm, MPI_Errhandler) {
    return MPI_SUCCESS;
}
static inline int MPI_Get_processor_name(char* name, int* len) {
    std::strcpy(name, "localhost");
    *len = 9;
    return MPI_SUCCESS;
}

#endif
