/*
 * Single-rank MPI stand-in used ONLY to compile the reference's host C files
 * (src/awp/mesh.c, src/awp/cerjan.c, src/awp/grid.c, and the point-set set-up
 * files listed in oracle/Makefile) into the CPU checker
 * library oracle/_ref/libawpref_host.so.  It is test infrastructure: the
 * product never includes it.
 *
 * It also lets the link-symbol test compile pmcl3d.c and the rest of the
 * reference's lpmcl3d host files (tests/test_dropin_link.py) to list the
 * launchers they call; calls it does not declare stay undefined there.
 *
 * Semantics are those of MPI with a world of exactly one rank:
 *   - rank 0, size 1;
 *   - Bcast is a no-op, Allreduce copies send -> recv;
 *   - the MPI-IO subarray read path is never reached at PX=PY=1 (mesh.c:145
 *     takes the plain fopen/fread branch), so the File_* calls report failure.
 */
#ifndef AWP_ORACLE_MPI_STUB_H
#define AWP_ORACLE_MPI_STUB_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype; /* value = element size in bytes */
typedef int MPI_Op;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef long long MPI_Aint;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
typedef int MPI_Request;
typedef int MPI_File;

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_COMM_WORLD 0
#define MPI_FLOAT ((MPI_Datatype)sizeof(float))
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))
#define MPI_INT ((MPI_Datatype)sizeof(int))
#define MPI_OFFSET ((MPI_Datatype)sizeof(long long))
#define MPI_BYTE ((MPI_Datatype)1)
#define MPI_CHAR ((MPI_Datatype)1)
#define MPI_UINT32_T ((MPI_Datatype)4)
#define MPI_UINT64_T ((MPI_Datatype)8)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#ifndef MPI_AINT
#define MPI_AINT ((MPI_Datatype)sizeof(long long))
#endif
#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_SUM 3
#define MPI_ORDER_C 0
#define MPI_MODE_RDONLY 2
#define MPI_MODE_CREATE 1
#define MPI_MODE_WRONLY 4
#define MPI_INFO_NULL 0
#define MPI_UNDEFINED (-32766)
#define MPI_MAX_ERROR_STRING 256

static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return 0; }
static inline int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c) {
  (void)b; (void)n; (void)t; (void)root; (void)c; return 0;
}
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t,
                                MPI_Op op, MPI_Comm c) {
  (void)op; (void)c;
  if (s != r) memcpy(r, s, (size_t)n * (size_t)t);
  return 0;
}
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
static inline int MPI_Abort(MPI_Comm c, int e) { (void)c; fprintf(stderr, "MPI_Abort(%d)\n", e); exit(e); }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Error_string(int e, char *s, int *len) {
  *len = snprintf(s, 64, "mpi stub error %d", e); return 0;
}
static inline int MPI_Type_create_subarray(int nd, const int *a, const int *b, const int *c,
                                           int o, MPI_Datatype t, MPI_Datatype *nt) {
  (void)nd; (void)a; (void)b; (void)c; (void)o; *nt = t; return MPI_ERR_OTHER;
}
static inline int MPI_Type_commit(MPI_Datatype *t) { (void)t; return MPI_ERR_OTHER; }
static inline int MPI_File_open(MPI_Comm c, const char *f, int m, MPI_Info i, MPI_File *fh) {
  (void)c; (void)f; (void)m; (void)i; *fh = 0; return MPI_ERR_OTHER;
}
static inline int MPI_File_set_view(MPI_File fh, MPI_Offset d, MPI_Datatype e, MPI_Datatype f,
                                    const char *r, MPI_Info i) {
  (void)fh; (void)d; (void)e; (void)f; (void)r; (void)i; return MPI_ERR_OTHER;
}
static inline int MPI_File_read_all(MPI_File fh, void *b, int n, MPI_Datatype t, MPI_Status *s) {
  (void)fh; (void)b; (void)n; (void)t; (void)s; return MPI_ERR_OTHER;
}
static inline int MPI_File_close(MPI_File *fh) { (void)fh; return MPI_ERR_OTHER; }

#endif
