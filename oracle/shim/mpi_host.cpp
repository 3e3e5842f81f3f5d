// Single-rank host implementation of the MPI subset declared in shim/mpi.h.
// Oracle infrastructure for compiling the reference CPU sources; MPI-IO calls
// become POSIX pread/pwrite on a per-handle file position.
#include "mpi.h"

#include <errno.h>
#include <fcntl.h>
#include <stdio.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

#include <mutex>
#include <unordered_map>

namespace {
std::mutex g_mu;
std::unordered_map<int, long long> g_pos;  // file descriptor -> current offset

long long &pos_of(int fd) {
  std::lock_guard<std::mutex> lk(g_mu);
  return g_pos[fd];
}
}  // namespace

extern "C" {

int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm, int *rank) {
  *rank = 0;
  return MPI_SUCCESS;
}
int MPI_Comm_size(MPI_Comm, int *size) {
  *size = 1;
  return MPI_SUCCESS;
}
int MPI_Get_processor_name(char *name, int *len) {
  snprintf(name, MPI_MAX_PROCESSOR_NAME, "localhost");
  *len = (int)strlen(name);
  return MPI_SUCCESS;
}
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count,
                  MPI_Datatype type, MPI_Op, MPI_Comm) {
  // One rank: the sum over ranks is the rank's own buffer.
  if (sendbuf != MPI_IN_PLACE && sendbuf != recvbuf)
    memcpy(recvbuf, sendbuf, (size_t)count * (size_t)type);
  return MPI_SUCCESS;
}
int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) {
  return MPI_ERR_OTHER;  // no peer exists in a one-rank world
}
int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) {
  return MPI_ERR_OTHER;
}
int MPI_Error_string(int code, char *s, int *len) {
  snprintf(s, MPI_MAX_ERROR_STRING, "mpi shim error %d", code);
  *len = (int)strlen(s);
  return MPI_SUCCESS;
}

int MPI_File_open(MPI_Comm, const char *filename, int amode, MPI_Info,
                  MPI_File *fh) {
  int flags = 0;
  if (amode & MPI_MODE_RDWR)
    flags = O_RDWR;
  else if (amode & MPI_MODE_WRONLY)
    flags = O_WRONLY;
  else
    flags = O_RDONLY;
  if (amode & MPI_MODE_CREATE) flags |= O_CREAT;
  int fd = open(filename, flags, 0644);
  if (fd < 0) {
    *fh = MPI_FILE_NULL;
    return MPI_ERR_OTHER;
  }
  pos_of(fd) = 0;
  *fh = fd;
  return MPI_SUCCESS;
}
int MPI_File_close(MPI_File *fh) {
  if (*fh >= 0) {
    {
      std::lock_guard<std::mutex> lk(g_mu);
      g_pos.erase(*fh);
    }
    close(*fh);
  }
  *fh = MPI_FILE_NULL;
  return MPI_SUCCESS;
}
int MPI_File_seek(MPI_File fh, MPI_Offset offset, int whence) {
  if (fh < 0) return MPI_ERR_OTHER;
  long long &p = pos_of(fh);
  if (whence == MPI_SEEK_SET)
    p = offset;
  else if (whence == MPI_SEEK_CUR)
    p += offset;
  else {
    struct stat st;
    fstat(fh, &st);
    p = (long long)st.st_size + offset;
  }
  return MPI_SUCCESS;
}
int MPI_File_read(MPI_File fh, void *buf, int count, MPI_Datatype type,
                  MPI_Status *) {
  if (fh < 0) return MPI_ERR_OTHER;
  long long &p = pos_of(fh);
  size_t want = (size_t)count * (size_t)type;
  size_t got = 0;
  while (got < want) {
    ssize_t r = pread(fh, (char *)buf + got, want - got, p + (long long)got);
    if (r <= 0) break;
    got += (size_t)r;
  }
  p += (long long)got;
  return got == want ? MPI_SUCCESS : MPI_ERR_OTHER;
}
int MPI_File_write(MPI_File fh, const void *buf, int count, MPI_Datatype type,
                   MPI_Status *) {
  if (fh < 0) return MPI_ERR_OTHER;
  long long &p = pos_of(fh);
  size_t want = (size_t)count * (size_t)type;
  size_t put = 0;
  while (put < want) {
    ssize_t r =
        pwrite(fh, (const char *)buf + put, want - put, p + (long long)put);
    if (r <= 0) break;
    put += (size_t)r;
  }
  p += (long long)put;
  return put == want ? MPI_SUCCESS : MPI_ERR_OTHER;
}
int MPI_File_set_size(MPI_File fh, MPI_Offset size) {
  if (fh < 0) return MPI_ERR_OTHER;
  return ftruncate(fh, (off_t)size) == 0 ? MPI_SUCCESS : MPI_ERR_OTHER;
}

}  // extern "C"
