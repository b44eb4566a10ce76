/* Single-rank MPI stand-in used only to compile the reference's CPU solver
 * sources as the parity oracle (test infrastructure, never shipped).
 * Every collective is the identity on one rank; point-to-point calls are
 * no-ops (a one-zone, one-rank run never issues them); MPI-IO is unsupported. */
#ifndef PHX_ORACLE_MPI_SHIM_H
#define PHX_ORACLE_MPI_SHIM_H
#include <string.h>
#include <stdlib.h>
#include <stdio.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef int MPI_File;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; int count; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_REQUEST_NULL 0
#define MPI_INFO_NULL 0
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1

/* datatype handles encode their byte size */
#define MPI_CHAR 1
#define MPI_BYTE 1
#define MPI_INT 4
#define MPI_INTEGER 4
#define MPI_FLOAT 0x104
#define MPI_DOUBLE 8
#define MPI_DOUBLE_PRECISION 8
#define MPI_LONG_LONG 0x108
#define MPI_DOUBLE_INT 12
#define MPI_2INT 0x208

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_MAXLOC 4
#define MPI_MINLOC 5
#define MPI_BCAST 6

static inline int phx_mpi_size(MPI_Datatype t) { return t & 0xff; }
static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Initialized(int *f) { *f = 1; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Abort(MPI_Comm, int code) { fprintf(stderr, "MPI_Abort(%d)\n", code); exit(code ? code : 1); }
static inline int MPI_Comm_size(MPI_Comm, int *n) { *n = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm *o) { *o = c; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Get_processor_name(char *n, int *len) { strcpy(n, "oracle"); *len = 6; return 0; }
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm)
{ if (s != r && r) memmove(r, s, (size_t)n * phx_mpi_size(t)); return 0; }
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm)
{ if (s != r && r) memmove(r, s, (size_t)n * phx_mpi_size(t)); return 0; }
static inline int MPI_Scan(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm)
{ if (s != r && r) memmove(r, s, (size_t)n * phx_mpi_size(t)); return 0; }
static inline int MPI_Allgather(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, MPI_Comm)
{ if (s != r && r) memmove(r, s, (size_t)n * phx_mpi_size(t)); return 0; }
static inline int MPI_Gather(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, int, MPI_Comm)
{ if (s != r && r) memmove(r, s, (size_t)n * phx_mpi_size(t)); return 0; }
static inline int MPI_Gatherv(const void *s, int n, MPI_Datatype t, void *r, const int *, const int *d, MPI_Datatype, int, MPI_Comm)
{ if (r) memmove((char *)r + (size_t)(d ? d[0] : 0) * phx_mpi_size(t), s, (size_t)n * phx_mpi_size(t)); return 0; }
static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return 0; }
static inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *q) { *q = 0; return 0; }
static inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *q) { *q = 0; return 0; }
static inline int MPI_Wait(MPI_Request *, MPI_Status *) { return 0; }
static inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return 0; }
static inline int MPI_Get_count(const MPI_Status *, MPI_Datatype, int *c) { *c = 0; return 0; }
static inline int MPI_File_open(MPI_Comm, const char *, int, MPI_Info, MPI_File *) { return 1; }
static inline int MPI_File_close(MPI_File *) { return 0; }
static inline int MPI_File_write_at(MPI_File, MPI_Offset, const void *, int, MPI_Datatype, MPI_Status *) { return 1; }
static inline int MPI_File_write_at_all(MPI_File, MPI_Offset, const void *, int, MPI_Datatype, MPI_Status *) { return 1; }
static inline int MPI_File_get_position(MPI_File, MPI_Offset *o) { *o = 0; return 0; }
#endif
