/*
 * Single-rank MPI stand-in used ONLY to compile the reference HPCrack sources
 * into the test oracle (oracle/_ref).  It is test infrastructure: nothing in
 * the product library includes it.
 *
 * Semantics (one rank, Cartesian topology 1x1x1):
 *   - every rank query answers 0, every size query answers 1;
 *   - MPI_Cart_coords gives coordinates (0,0,0); neighbours of a 1x1x1
 *     topology are MPI_PROC_NULL, so the halo exchange in
 *     include/mpi_communications.h:39-60 (SendRecv) becomes a no-op, exactly
 *     as MPI defines send/recv to MPI_PROC_NULL;
 *   - MPI_Reduce / MPI_Bcast / MPI_Gather on one rank copy the send buffer
 *     (pcg_utilities.cpp:29-31, phase_field_max_search.cpp:31-32,
 *     strain_history.cpp:128-129, vtk_output.cpp:351-356);
 *   - derived datatypes are opaque integers with no effect.
 */
#ifndef HPC_ORACLE_MPI_STUB_H
#define HPC_ORACLE_MPI_STUB_H

#include <string.h>
#include <time.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_PROC_NULL (-2)
#define MPI_SUCCESS 0
#define MPI_THREAD_FUNNELED 1

#define MPI_DOUBLE 8
#define MPI_INT 4
#define MPI_SHORT 2
#define MPI_FLOAT 5

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

static inline size_t hpc_mpi_type_size_(MPI_Datatype t) {
  switch (t) {
    case MPI_DOUBLE: return 8;
    case MPI_INT: return 4;
    case MPI_FLOAT: return 4;
    case MPI_SHORT: return 2;
    default: return 0;
  }
}

static inline int MPI_Init_thread(int* argc, char*** argv, int req, int* prov) {
  (void)argc; (void)argv; *prov = req; return MPI_SUCCESS;
}
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm c, int* n) { (void)c; *n = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm c, int* r) { (void)c; *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_free(MPI_Comm* c) { (void)c; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return MPI_SUCCESS; }

static inline int MPI_Cart_create(MPI_Comm old, int nd, const int* dims, const int* periods,
                                  int reorder, MPI_Comm* out) {
  (void)old; (void)nd; (void)dims; (void)periods; (void)reorder; *out = 1; return MPI_SUCCESS;
}
static inline int MPI_Cart_coords(MPI_Comm c, int rank, int nd, int* coords) {
  (void)c; (void)rank; for (int i = 0; i < nd; ++i) coords[i] = 0; return MPI_SUCCESS;
}
static inline int MPI_Cart_rank(MPI_Comm c, const int* coords, int* rank) {
  (void)c; (void)coords; *rank = 0; return MPI_SUCCESS;
}
static inline int MPI_Cart_sub(MPI_Comm c, const int* remain, MPI_Comm* out) {
  (void)c; (void)remain; *out = 2; return MPI_SUCCESS;
}

static inline int MPI_Type_contiguous(int n, MPI_Datatype o, MPI_Datatype* t) {
  (void)n; (void)o; *t = 100; return MPI_SUCCESS;
}
static inline int MPI_Type_vector(int c, int b, int s, MPI_Datatype o, MPI_Datatype* t) {
  (void)c; (void)b; (void)s; (void)o; *t = 101; return MPI_SUCCESS;
}
static inline int MPI_Type_indexed(int c, const int* b, const int* d, MPI_Datatype o,
                                   MPI_Datatype* t) {
  (void)c; (void)b; (void)d; (void)o; *t = 102; return MPI_SUCCESS;
}
static inline int MPI_Type_commit(MPI_Datatype* t) { (void)t; return MPI_SUCCESS; }
static inline int MPI_Type_free(MPI_Datatype* t) { (void)t; return MPI_SUCCESS; }

/* Point-to-point: the only peers a 1x1x1 topology has are MPI_PROC_NULL. */
static inline int MPI_Ssend(const void* b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c) {
  (void)b; (void)n; (void)t; (void)dest; (void)tag; (void)c; return MPI_SUCCESS;
}
static inline int MPI_Recv(void* b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c,
                           MPI_Status* s) {
  (void)b; (void)n; (void)t; (void)src; (void)tag; (void)c;
  if (s) { s->MPI_SOURCE = src; s->MPI_TAG = tag; s->MPI_ERROR = 0; }
  return MPI_SUCCESS;
}

static inline int MPI_Reduce(const void* sb, void* rb, int n, MPI_Datatype t, MPI_Op op, int root,
                             MPI_Comm c) {
  (void)op; (void)root; (void)c;
  if (sb != rb) memcpy(rb, sb, (size_t)n * hpc_mpi_type_size_(t));
  return MPI_SUCCESS;
}
static inline int MPI_Bcast(void* b, int n, MPI_Datatype t, int root, MPI_Comm c) {
  (void)b; (void)n; (void)t; (void)root; (void)c; return MPI_SUCCESS;
}
static inline int MPI_Gather(const void* sb, int sn, MPI_Datatype st, void* rb, int rn,
                             MPI_Datatype rt, int root, MPI_Comm c) {
  (void)rn; (void)rt; (void)root; (void)c;
  memcpy(rb, sb, (size_t)sn * hpc_mpi_type_size_(st));
  return MPI_SUCCESS;
}
static inline double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

#ifdef __cplusplus
}
#endif

#endif
