/* Single-rank MPI stand-in for the CPU checker build of the reference (test infrastructure only).
 *
 * The container has no MPI. On one rank every MPI call the reference's Stokes path makes is either a
 * no-op or a copy: reductions and gathers copy the send buffer into the receive buffer (MPI_IN_PLACE
 * leaves it), point-to-point calls never fire because same-rank interface pairs are direct copies
 * (communication_plan.hpp), and size/rank are 1/0. Datatypes encode their element size. MPI-IO maps onto stdio
 * (one process writes the whole file). */
#ifndef TN_REF_MPI_STUB_H
#define TN_REF_MPI_STUB_H

#include <stddef.h>
#include <string.h>

#ifdef __cplusplus
extern "C++" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Group;
typedef int MPI_Info;
typedef int MPI_Errhandler;
typedef long long MPI_Offset;
typedef long long MPI_Aint;
typedef int MPI_File;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_MAX_ERROR_STRING 256
#define MPI_UNDEFINED (-32766)
#define MPI_PROC_NULL (-2)
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)

#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_COMM_NULL 0
#define MPI_GROUP_NULL 0
#define MPI_INFO_NULL 0
#define MPI_REQUEST_NULL 0
#define MPI_ERRORS_RETURN 1
#define MPI_ERRORS_ARE_FATAL 0
#define MPI_STATUS_IGNORE ((MPI_Status*) 0)
#define MPI_STATUSES_IGNORE ((MPI_Status*) 0)
#define MPI_IN_PLACE ((void*) 1)
#define MPI_BOTTOM ((void*) 0)

#define MPI_MODE_RDONLY 2
#define MPI_MODE_RDWR 8
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1

/* datatype handle = element size in bytes (distinct types of equal size need not be told apart) */
#define MPI_DATATYPE_NULL 0
#define MPI_CHAR ((MPI_Datatype) sizeof(char))
#define MPI_SIGNED_CHAR ((MPI_Datatype) sizeof(signed char))
#define MPI_UNSIGNED_CHAR ((MPI_Datatype) sizeof(unsigned char))
#define MPI_BYTE ((MPI_Datatype) 1)
#define MPI_SHORT ((MPI_Datatype) sizeof(short))
#define MPI_UNSIGNED_SHORT ((MPI_Datatype) sizeof(unsigned short))
#define MPI_INT ((MPI_Datatype) sizeof(int))
#define MPI_UNSIGNED ((MPI_Datatype) sizeof(unsigned))
#define MPI_LONG ((MPI_Datatype) sizeof(long))
#define MPI_UNSIGNED_LONG ((MPI_Datatype) sizeof(unsigned long))
#define MPI_LONG_LONG ((MPI_Datatype) sizeof(long long))
#define MPI_LONG_LONG_INT MPI_LONG_LONG
#define MPI_UNSIGNED_LONG_LONG ((MPI_Datatype) sizeof(unsigned long long))
#define MPI_FLOAT ((MPI_Datatype) sizeof(float))
#define MPI_DOUBLE ((MPI_Datatype) sizeof(double))
#define MPI_LONG_DOUBLE ((MPI_Datatype) sizeof(long double))
#define MPI_CXX_BOOL ((MPI_Datatype) sizeof(bool))
#define MPI_C_BOOL ((MPI_Datatype) sizeof(bool))

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_PROD 4
#define MPI_LAND 5
#define MPI_LOR 6

static inline int tn_mpi_copy_(const void* s, void* r, int n, MPI_Datatype t)
{
    if (s != MPI_IN_PLACE && s != r && n > 0) memcpy(r, s, (size_t) n * (size_t) t);
    return MPI_SUCCESS;
}

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Finalize() { return MPI_SUCCESS; }
static inline int MPI_Initialized(int* f) { *f = 1; return MPI_SUCCESS; }
static inline int MPI_Finalized(int* f) { *f = 0; return MPI_SUCCESS; }
static inline int MPI_Abort(MPI_Comm, int) { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_set_errhandler(MPI_Comm, MPI_Errhandler) { return MPI_SUCCESS; }
static inline int MPI_Comm_split(MPI_Comm c, int color, int, MPI_Comm* n)
{
    *n = (color == MPI_UNDEFINED) ? MPI_COMM_NULL : c;
    return MPI_SUCCESS;
}
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm* n) { *n = c; return MPI_SUCCESS; }
static inline int MPI_Comm_free(MPI_Comm* c) { *c = MPI_COMM_NULL; return MPI_SUCCESS; }
static inline int MPI_Comm_group(MPI_Comm, MPI_Group* g) { *g = 1; return MPI_SUCCESS; }
static inline int MPI_Group_free(MPI_Group* g) { *g = MPI_GROUP_NULL; return MPI_SUCCESS; }
static inline int MPI_Group_size(MPI_Group, int* s) { *s = 1; return MPI_SUCCESS; }
static inline int MPI_Group_translate_ranks(MPI_Group, int n, const int* r1, MPI_Group, int* r2)
{
    for (int i = 0; i < n; ++i) r2[i] = r1[i];
    return MPI_SUCCESS;
}
static inline int MPI_Error_string(int, char* s, int* len)
{
    const char* m = "single-rank MPI stand-in";
    strcpy(s, m);
    *len = (int) strlen(m);
    return MPI_SUCCESS;
}
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm)
{
    return tn_mpi_copy_(s, r, n, t);
}
static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm)
{
    return tn_mpi_copy_(s, r, n, t);
}
static inline int MPI_Scan(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm)
{
    return tn_mpi_copy_(s, r, n, t);
}
static inline int MPI_Exscan(const void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Allgather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, MPI_Comm)
{
    return tn_mpi_copy_(s, r, n, t);
}
static inline int MPI_Gather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, int, MPI_Comm)
{
    return tn_mpi_copy_(s, r, n, t);
}
static inline int MPI_Allgatherv(const void* s, int n, MPI_Datatype t, void* r, const int*, const int* displs,
                                 MPI_Datatype rt, MPI_Comm)
{
    return tn_mpi_copy_(s, (char*) r + (size_t) displs[0] * (size_t) rt, n, t);
}
static inline int MPI_Alltoallv(const void* s, const int* sc, const int* sd, MPI_Datatype st, void* r, const int*,
                                const int* rd, MPI_Datatype rt, MPI_Comm)
{
    if (sc[0] > 0) memcpy((char*) r + (size_t) rd[0] * (size_t) rt, (const char*) s + (size_t) sd[0] * (size_t) st,
                          (size_t) sc[0] * (size_t) st);
    return MPI_SUCCESS;
}
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* q)
{
    *q = MPI_REQUEST_NULL;
    return MPI_ERR_OTHER; /* never reached on one rank */
}
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* q)
{
    *q = MPI_REQUEST_NULL;
    return MPI_ERR_OTHER;
}
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return MPI_SUCCESS; }
static inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return MPI_SUCCESS; }
static inline int MPI_Waitany(int, MPI_Request*, int* idx, MPI_Status*)
{
    *idx = MPI_UNDEFINED;
    return MPI_SUCCESS;
}
static inline int MPI_Type_create_hindexed(int, const int*, const MPI_Aint*, MPI_Datatype, MPI_Datatype* n)
{
    *n = MPI_DATATYPE_NULL;
    return MPI_ERR_OTHER;
}
static inline int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
static inline int MPI_Type_free(MPI_Datatype*) { return MPI_SUCCESS; }
static inline double MPI_Wtime() { return 0.0; }

/* MPI-IO on one rank: a small table of stdio handles (the reference's XDMF writer and checkpoint reader) */
#include <stdio.h>
struct tn_mpi_files_ {
    FILE* f[64];
};
static inline tn_mpi_files_& tn_mpi_files() { static tn_mpi_files_ t = {}; return t; }
static inline int MPI_File_open(MPI_Comm, const char* path, int amode, MPI_Info, MPI_File* fh)
{
    FILE* f = 0;
    if (amode & MPI_MODE_RDONLY) f = fopen(path, "rb");
    else {
        f = fopen(path, "r+b");
        if (!f && (amode & MPI_MODE_CREATE)) f = fopen(path, "w+b");
    }
    if (!f) return MPI_ERR_OTHER;
    for (int i = 1; i < 64; ++i)
        if (!tn_mpi_files().f[i]) { tn_mpi_files().f[i] = f; *fh = i; return MPI_SUCCESS; }
    fclose(f);
    return MPI_ERR_OTHER;
}
static inline int MPI_File_close(MPI_File* fh)
{
    if (*fh > 0 && *fh < 64 && tn_mpi_files().f[*fh]) { fclose(tn_mpi_files().f[*fh]); tn_mpi_files().f[*fh] = 0; }
    *fh = 0;
    return MPI_SUCCESS;
}
static inline int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype, MPI_Datatype, const char*, MPI_Info)
{
    return fseek(tn_mpi_files().f[fh], (long) disp, SEEK_SET) == 0 ? MPI_SUCCESS : MPI_ERR_OTHER;
}
static inline int MPI_File_write_all(MPI_File fh, const void* buf, int count, MPI_Datatype t, MPI_Status*)
{
    size_t n = (size_t) count * (size_t) t;
    return fwrite(buf, 1, n, tn_mpi_files().f[fh]) == n ? MPI_SUCCESS : MPI_ERR_OTHER;
}
static inline int MPI_File_read_all(MPI_File fh, void* buf, int count, MPI_Datatype t, MPI_Status*)
{
    size_t n = (size_t) count * (size_t) t;
    return fread(buf, 1, n, tn_mpi_files().f[fh]) == n ? MPI_SUCCESS : MPI_ERR_OTHER;
}
static inline int MPI_File_get_size(MPI_File fh, MPI_Offset* size)
{
    FILE* f = tn_mpi_files().f[fh];
    long  p = ftell(f);
    fseek(f, 0, SEEK_END);
    *size = ftell(f);
    fseek(f, p, SEEK_SET);
    return MPI_SUCCESS;
}

#ifdef __cplusplus
}
#endif

#endif
