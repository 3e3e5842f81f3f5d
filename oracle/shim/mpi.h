/* Test-only stand-in for <mpi.h> used to compile the reference TiltRec CPU
 * sources (TiltRec-mpi / TiltRecZ-mpi) without an MPI installation.
 *
 * Oracle infrastructure: only the test suite and the CPU-baseline leg of the
 * benchmark load what is built from this header.
 *
 * Semantics: a single rank (rank 0 of 1).  Collectives are identities
 * (MPI_Allreduce with MPI_IN_PLACE leaves the buffer as is, which is exactly
 * what a 1-rank sum does), MPI-IO maps onto POSIX file descriptors.
 * A datatype is represented by its size in bytes.
 */
#ifndef ORACLE_SHIM_MPI_H
#define ORACLE_SHIM_MPI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_File;
typedef long long MPI_Offset;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_MAX_ERROR_STRING 256
#define MPI_COMM_WORLD 0
#define MPI_INFO_NULL 0
#define MPI_FILE_NULL (-1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)

#define MPI_CHAR 1
#define MPI_UNSIGNED_CHAR 1
#define MPI_BYTE 1
#define MPI_SHORT 2
#define MPI_INT 4
#define MPI_FLOAT 4
#define MPI_DOUBLE 8

#define MPI_SUM 0

#define MPI_MODE_RDONLY 2
#define MPI_MODE_RDWR 8
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1

#define MPI_SEEK_SET 600
#define MPI_SEEK_CUR 602
#define MPI_SEEK_END 604

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Get_processor_name(char *name, int *resultlen);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count,
                  MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag,
             MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype type, int source, int tag,
             MPI_Comm comm, MPI_Status *status);
int MPI_Error_string(int errorcode, char *string, int *resultlen);

int MPI_File_open(MPI_Comm comm, const char *filename, int amode,
                  MPI_Info info, MPI_File *fh);
int MPI_File_close(MPI_File *fh);
int MPI_File_seek(MPI_File fh, MPI_Offset offset, int whence);
int MPI_File_read(MPI_File fh, void *buf, int count, MPI_Datatype type,
                  MPI_Status *status);
int MPI_File_write(MPI_File fh, const void *buf, int count, MPI_Datatype type,
                   MPI_Status *status);
int MPI_File_set_size(MPI_File fh, MPI_Offset size);

#ifdef __cplusplus
}
#endif

#endif
