/*
 * Single-rank MPI stand-in used only to compile the reference TORCH sources
 * (src/MPI/MPI_Wrapper.cpp) into the CPU oracle binary.  Test infrastructure:
 * this file is never linked into the product library.
 *
 * Semantics: one process, rank 0 of 1.  Point-to-point calls are never
 * reached with nproc == 1 (the reference only sends across partitions);
 * they abort loudly if they ever are.  Reductions copy input to output,
 * which is the exact single-rank result of MPI_Allreduce.
 */
#ifndef ORACLE_MPI_STUB_H
#define ORACLE_MPI_STUB_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_File;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_MAX_PROCESSOR_NAME 64
#define MPI_INT 1
#define MPI_INTEGER 1
#define MPI_FLOAT 2
#define MPI_DOUBLE 3
#define MPI_CHAR 4
#define MPI_MIN 10
#define MPI_MAX 11
#define MPI_SUM 12
#define MPI_INFO_NULL 0
#define MPI_MODE_CREATE 1
#define MPI_MODE_WRONLY 2
#define MPI_STATUS_IGNORE ((MPI_Status*)0)

static inline size_t oracle_mpi_type_size(MPI_Datatype t) {
	switch (t) {
	case MPI_INT: return sizeof(int);
	case MPI_FLOAT: return sizeof(float);
	case MPI_DOUBLE: return sizeof(double);
	default: return 1;
	}
}

static inline void oracle_mpi_unreachable(const char* what) {
	fprintf(stderr, "single-rank MPI stub: %s reached with one rank\n", what);
	abort();
}

static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Get_processor_name(char* name, int* len) {
	strcpy(name, "oracle");
	*len = 6;
	return 0;
}
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) {
	oracle_mpi_unreachable("MPI_Send");
	return 1;
}
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) {
	oracle_mpi_unreachable("MPI_Recv");
	return 1;
}
static inline int MPI_Allreduce(const void* in, void* out, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
	memmove(out, in, (size_t)n * oracle_mpi_type_size(t));
	return 0;
}
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Abort(MPI_Comm, int code) { exit(code ? code : 1); return 0; }
static inline int MPI_File_open(MPI_Comm, const char*, int, MPI_Info, MPI_File*) {
	oracle_mpi_unreachable("MPI_File_open");
	return 1;
}
static inline int MPI_File_set_view(MPI_File, long, MPI_Datatype, MPI_Datatype, const char*, MPI_Info) { return 0; }
static inline int MPI_File_write(MPI_File, const void*, int, MPI_Datatype, MPI_Status*) { return 0; }
static inline int MPI_File_close(MPI_File*) { return 0; }

#endif
