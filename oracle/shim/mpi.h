/*
 * Single-rank MPI stand-in used ONLY to compile the reference's sources for the oracle
 * (test infrastructure, never part of the product).
 *
 * With one rank every collective is a local copy (Allreduce/Allgather(v)/Alltoall(v)/Bcast)
 * or a no-op (Barrier).  Datatypes are integer handles whose value encodes their size;
 * a derived struct type records its extent.  Only the calls the reference makes are
 * provided (inventory: src/phase1/{init,seed,partition,phase1}.cpp, src/phase2/phase2.cpp,
 * src/utils.cpp, src/main.cpp).
 */
#ifndef ORACLE_SHIM_MPI_H
#define ORACLE_SHIM_MPI_H

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef long MPI_Aint;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_INFO_NULL 0
#define MPI_COMM_TYPE_SHARED 1
#define MPI_SUCCESS 0
#define MPI_IN_PLACE ((void *)1)

/* builtin datatypes: handle = size in bytes (+ a tag in the high bits to keep them distinct) */
#define MPI_BYTE          ((MPI_Datatype)(0x100 | 1))
#define MPI_CHAR          ((MPI_Datatype)(0x200 | 1))
#define MPI_INT           ((MPI_Datatype)(0x300 | 4))
#define MPI_UNSIGNED      ((MPI_Datatype)(0x400 | 4))
#define MPI_DOUBLE        ((MPI_Datatype)(0x500 | 8))
#define MPI_LONG          ((MPI_Datatype)(0x600 | 8))
#define MPI_UNSIGNED_LONG ((MPI_Datatype)(0x700 | 8))
#define MPI_UINT64_T      ((MPI_Datatype)(0x800 | 8))
#define MPI_INT64_T       ((MPI_Datatype)(0x900 | 8))

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_BOR 4

namespace oracle_mpi {
/* derived types live in a small table; their handles start at 0x10000 */
struct DerivedTable {
    long extent[64];
    int n;
};
inline DerivedTable &derived() {
    static DerivedTable t = {{0}, 0};
    return t;
}
inline size_t type_size(MPI_Datatype t) {
    if (t >= 0x10000) return (size_t)derived().extent[t - 0x10000];
    return (size_t)(t & 0xff);
}
}  // namespace oracle_mpi

static inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Initialized(int *flag) { *flag = 1; return MPI_SUCCESS; }
static inline int MPI_Finalized(int *flag) { *flag = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_split_type(MPI_Comm, int, int, MPI_Info, MPI_Comm *out) {
    *out = MPI_COMM_WORLD;
    return MPI_SUCCESS;
}
static inline int MPI_Comm_free(MPI_Comm *c) { *c = MPI_COMM_NULL; return MPI_SUCCESS; }
static inline int MPI_Abort(MPI_Comm, int code) {
    fflush(stdout);
    fprintf(stderr, "[oracle-mpi] MPI_Abort(%d)\n", code);
    exit(code == 0 ? 1 : code);
}
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }

static inline void oracle_mpi_copy(const void *src, void *dst, int count, MPI_Datatype t) {
    if (src == MPI_IN_PLACE || src == dst || count <= 0) return;
    memmove(dst, src, (size_t)count * oracle_mpi::type_size(t));
}

static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
    oracle_mpi_copy(s, r, n, t);
    return MPI_SUCCESS;
}
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Allgather(const void *s, int sc, MPI_Datatype st, void *r, int, MPI_Datatype, MPI_Comm) {
    oracle_mpi_copy(s, r, sc, st);
    return MPI_SUCCESS;
}
static inline int MPI_Allgatherv(const void *s, int sc, MPI_Datatype st, void *r, const int *, const int *displs,
                                 MPI_Datatype rt, MPI_Comm) {
    oracle_mpi_copy(s, (char *)r + (size_t)displs[0] * oracle_mpi::type_size(rt), sc, st);
    return MPI_SUCCESS;
}
static inline int MPI_Iallgatherv(const void *s, int sc, MPI_Datatype st, void *r, const int *rc, const int *displs,
                                  MPI_Datatype rt, MPI_Comm c, MPI_Request *req) {
    *req = 0;
    return MPI_Allgatherv(s, sc, st, r, rc, displs, rt, c);
}
static inline int MPI_Wait(MPI_Request *, MPI_Status *) { return MPI_SUCCESS; }
static inline int MPI_Alltoall(const void *s, int sc, MPI_Datatype st, void *r, int, MPI_Datatype, MPI_Comm) {
    oracle_mpi_copy(s, r, sc, st);
    return MPI_SUCCESS;
}
static inline int MPI_Alltoallv(const void *s, const int *sc, const int *sd, MPI_Datatype st, void *r, const int *,
                                const int *rd, MPI_Datatype rt, MPI_Comm) {
    oracle_mpi_copy((const char *)s + (size_t)sd[0] * oracle_mpi::type_size(st),
                    (char *)r + (size_t)rd[0] * oracle_mpi::type_size(rt), sc[0], st);
    return MPI_SUCCESS;
}
static inline int MPI_Get_address(const void *p, MPI_Aint *a) { *a = (MPI_Aint)p; return MPI_SUCCESS; }
static inline int MPI_Type_create_struct(int n, const int *bl, const MPI_Aint *disp, const MPI_Datatype *types,
                                         MPI_Datatype *out) {
    long ext = 0;
    for (int i = 0; i < n; ++i) {
        long end = (long)disp[i] + (long)bl[i] * (long)oracle_mpi::type_size(types[i]);
        if (end > ext) ext = end;
    }
    oracle_mpi::DerivedTable &t = oracle_mpi::derived();
    int slot = t.n < 64 ? t.n++ : 63;
    t.extent[slot] = ext;
    *out = 0x10000 + slot;
    return MPI_SUCCESS;
}
static inline int MPI_Type_commit(MPI_Datatype *) { return MPI_SUCCESS; }
static inline int MPI_Type_free(MPI_Datatype *t) { *t = 0; return MPI_SUCCESS; }
static inline int MPI_Get_processor_name(char *name, int *len) {
    strcpy(name, "localhost");
    *len = 9;
    return MPI_SUCCESS;
}

#endif
