/*
 * Serial single-rank MPI stand-in used ONLY to compile the reference VBCSR
 * headers into the CPU oracle (oracle/_ref).  Test infrastructure, never part
 * of the shipped library.
 *
 * Written from the MPI-3 standard's C bindings.  MPI_Initialized reports 0, so
 * every reference DistGraph takes its serial branch (rank 0, size 1) and the
 * collectives below only ever see a one-rank communicator: each one copies its
 * send buffer to its receive buffer (or does nothing for MPI_IN_PLACE).
 */
#ifndef VBCSR_ORACLE_MPI_STUB_H
#define VBCSR_ORACLE_MPI_STUB_H

#include <stddef.h>
#include <string.h>
#include <stdlib.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_INFO_NULL 0
#define MPI_REQUEST_NULL 0
#define MPI_COMM_TYPE_SHARED 1
#define MPI_IDENT 0
#define MPI_CONGRUENT 1
#define MPI_SIMILAR 2
#define MPI_UNEQUAL 3
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)1)
#define MPI_UNDEFINED (-32766)

/* Datatype handles encode their byte size in the low byte. */
#define MPI_BYTE ((MPI_Datatype)0x0101)
#define MPI_CHAR ((MPI_Datatype)0x0201)
#define MPI_INT ((MPI_Datatype)0x0304)
#define MPI_UNSIGNED ((MPI_Datatype)0x0404)
#define MPI_FLOAT ((MPI_Datatype)0x0504)
#define MPI_LONG ((MPI_Datatype)0x0608)
#define MPI_LONG_LONG ((MPI_Datatype)0x0708)
#define MPI_LONG_LONG_INT MPI_LONG_LONG
#define MPI_UNSIGNED_LONG ((MPI_Datatype)0x0808)
#define MPI_UNSIGNED_LONG_LONG ((MPI_Datatype)0x0908)
#define MPI_INT64_T ((MPI_Datatype)0x0a08)
#define MPI_UINT64_T ((MPI_Datatype)0x0b08)
#define MPI_DOUBLE ((MPI_Datatype)0x0c08)
#define MPI_C_DOUBLE_COMPLEX ((MPI_Datatype)0x0d10)
#define MPI_CXX_DOUBLE_COMPLEX ((MPI_Datatype)0x0e10)
#define MPI_C_FLOAT_COMPLEX ((MPI_Datatype)0x0f08)
#define MPI_CXX_FLOAT_COMPLEX ((MPI_Datatype)0x1008)
#define MPI_2INT ((MPI_Datatype)0x1108)
#define MPI_DOUBLE_INT ((MPI_Datatype)0x1210)

#define MPI_SUM ((MPI_Op)1)
#define MPI_MAX ((MPI_Op)2)
#define MPI_MIN ((MPI_Op)3)
#define MPI_PROD ((MPI_Op)4)
#define MPI_LOR ((MPI_Op)5)
#define MPI_LAND ((MPI_Op)6)
#define MPI_BOR ((MPI_Op)7)
#define MPI_MAXLOC ((MPI_Op)8)
#define MPI_MINLOC ((MPI_Op)9)

static inline size_t vbcsr_stub_type_size(MPI_Datatype t) { return (size_t)(t & 0xff); }

static inline void vbcsr_stub_copy(const void* s, void* r, size_t n) {
  if (s != MPI_IN_PLACE && s != NULL && r != NULL && s != r && n) memmove(r, s, n);
}

static inline int MPI_Init(int* a, char*** b) { (void)a; (void)b; return 0; }
static inline int MPI_Init_thread(int* a, char*** b, int req, int* prov) {
  (void)a; (void)b; if (prov) *prov = req; return 0;
}
static inline int MPI_Initialized(int* flag) { *flag = 0; return 0; }
static inline int MPI_Finalized(int* flag) { *flag = 0; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Abort(MPI_Comm c, int code) { (void)c; exit(code); return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int* r) { (void)c; *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int* s) { (void)c; *s = 1; return 0; }
static inline int MPI_Comm_compare(MPI_Comm a, MPI_Comm b, int* res) {
  *res = (a == b) ? MPI_IDENT : MPI_CONGRUENT; return 0;
}
static inline int MPI_Comm_free(MPI_Comm* c) { *c = MPI_COMM_NULL; return 0; }
static inline int MPI_Comm_split_type(MPI_Comm c, int t, int k, MPI_Info i, MPI_Comm* out) {
  (void)t; (void)k; (void)i; *out = c; return 0;
}
static inline MPI_Comm MPI_Comm_f2c(int f) { return (MPI_Comm)f; }
static inline int MPI_Comm_c2f(MPI_Comm c) { return (int)c; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
static inline double MPI_Wtime(void) {
  struct timespec ts; clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
static inline int MPI_Type_size(MPI_Datatype t, int* s) { *s = (int)vbcsr_stub_type_size(t); return 0; }

static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op o, MPI_Comm c) {
  (void)o; (void)c; vbcsr_stub_copy(s, r, (size_t)n * vbcsr_stub_type_size(t)); return 0;
}
static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op o, int root, MPI_Comm c) {
  (void)o; (void)root; (void)c; vbcsr_stub_copy(s, r, (size_t)n * vbcsr_stub_type_size(t)); return 0;
}
static inline int MPI_Exscan(const void* s, void* r, int n, MPI_Datatype t, MPI_Op o, MPI_Comm c) {
  /* rank 0's receive buffer is undefined by the standard; leave it. */
  (void)s; (void)r; (void)n; (void)t; (void)o; (void)c; return 0;
}
static inline int MPI_Bcast(void* b, int n, MPI_Datatype t, int root, MPI_Comm c) {
  (void)b; (void)n; (void)t; (void)root; (void)c; return 0;
}
static inline int MPI_Allgather(const void* s, int sn, MPI_Datatype st, void* r, int rn, MPI_Datatype rt, MPI_Comm c) {
  (void)rn; (void)rt; (void)c; vbcsr_stub_copy(s, r, (size_t)sn * vbcsr_stub_type_size(st)); return 0;
}
static inline int MPI_Allgatherv(const void* s, int sn, MPI_Datatype st, void* r, const int* rc, const int* rd, MPI_Datatype rt, MPI_Comm c) {
  (void)rc; (void)c;
  vbcsr_stub_copy(s, (char*)r + (size_t)rd[0] * vbcsr_stub_type_size(rt), (size_t)sn * vbcsr_stub_type_size(st));
  return 0;
}
static inline int MPI_Gather(const void* s, int sn, MPI_Datatype st, void* r, int rn, MPI_Datatype rt, int root, MPI_Comm c) {
  (void)rn; (void)rt; (void)root; (void)c; vbcsr_stub_copy(s, r, (size_t)sn * vbcsr_stub_type_size(st)); return 0;
}
static inline int MPI_Gatherv(const void* s, int sn, MPI_Datatype st, void* r, const int* rc, const int* rd, MPI_Datatype rt, int root, MPI_Comm c) {
  (void)rc; (void)root; (void)c;
  if (r) vbcsr_stub_copy(s, (char*)r + (size_t)rd[0] * vbcsr_stub_type_size(rt), (size_t)sn * vbcsr_stub_type_size(st));
  return 0;
}
static inline int MPI_Scatterv(const void* s, const int* sc, const int* sd, MPI_Datatype st, void* r, int rn, MPI_Datatype rt, int root, MPI_Comm c) {
  (void)sc; (void)root; (void)c;
  if (s && r != MPI_IN_PLACE)
    vbcsr_stub_copy((const char*)s + (size_t)sd[0] * vbcsr_stub_type_size(st), r, (size_t)rn * vbcsr_stub_type_size(rt));
  return 0;
}
static inline int MPI_Alltoall(const void* s, int sn, MPI_Datatype st, void* r, int rn, MPI_Datatype rt, MPI_Comm c) {
  (void)rn; (void)rt; (void)c; vbcsr_stub_copy(s, r, (size_t)sn * vbcsr_stub_type_size(st)); return 0;
}
static inline int MPI_Alltoallv(const void* s, const int* sc, const int* sd, MPI_Datatype st, void* r, const int* rc, const int* rd, MPI_Datatype rt, MPI_Comm c) {
  (void)rc; (void)c;
  vbcsr_stub_copy((const char*)s + (size_t)sd[0] * vbcsr_stub_type_size(st),
                  (char*)r + (size_t)rd[0] * vbcsr_stub_type_size(rt),
                  (size_t)sc[0] * vbcsr_stub_type_size(st));
  return 0;
}
static inline int MPI_Isend(const void* b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request* q) {
  (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; *q = MPI_REQUEST_NULL; return 0;
}
static inline int MPI_Irecv(void* b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request* q) {
  (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; *q = MPI_REQUEST_NULL; return 0;
}
static inline int MPI_Send(const void* b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c) {
  (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; return 0;
}
static inline int MPI_Recv(void* b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status* st) {
  (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; (void)st; return 0;
}
static inline int MPI_Wait(MPI_Request* q, MPI_Status* s) { (void)s; *q = MPI_REQUEST_NULL; return 0; }
static inline int MPI_Waitall(int n, MPI_Request* q, MPI_Status* s) {
  (void)s; for (int i = 0; i < n; ++i) q[i] = MPI_REQUEST_NULL; return 0;
}
static inline int MPI_Waitany(int n, MPI_Request* q, int* idx, MPI_Status* s) {
  (void)q; (void)s; *idx = (n > 0) ? 0 : MPI_UNDEFINED; if (n > 0) q[0] = MPI_REQUEST_NULL; return 0;
}

#endif
