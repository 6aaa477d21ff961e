/*
 * Single-process stand-in for the subset of MPI that the hydro2d / hydro3d host
 * programs call (hydro2d/main.cxx, hydro3d/main.cxx). It lets those programs be
 * compiled unchanged on a machine without an MPI installation, with exactly one
 * rank. Every collective degenerates to a copy of the send buffer, because with one
 * rank the reduction of one contribution is that contribution.
 *
 * Call sites covered (hydro2d/main.cxx): MPI_Init/Comm_rank/Comm_size :439-441,
 * MPI_Abort :447, MPI_Barrier :223,396,420,681,683,804,817, MPI_Allreduce
 * :263,586,660,781, MPI_Reduce :778, MPI_Exscan :209, MPI_File_* :215-234,
 * MPI_Isend/Irecv/Waitall :402-418 (two-rank path; never reached with one rank),
 * MPI_Finalize :590,902. hydro3d/main.cxx uses the same set.
 *
 * Faithful detail: the byte count copied by a collective is count x size of the
 * MPI datatype passed, not of the C object, so a double reduced as MPI_FLOAT keeps
 * only 4 bytes, as a real MPI library would transfer.
 */
#ifndef HYDRO_COMPAT_MPI_H
#define HYDRO_COMPAT_MPI_H

#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/types.h>
#include <unistd.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_Request;
typedef long long MPI_Offset;
typedef struct { int fd; } *MPI_File;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 0
#define MPI_COMM_SELF 1
#define MPI_INFO_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

/* datatype handles encode their byte size */
#define MPI_CHAR 1
#define MPI_INT 4
#define MPI_FLOAT 0x104
#define MPI_DOUBLE 8
#define MPI_OFFSET 0x108

#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3

#define MPI_MODE_CREATE 1
#define MPI_MODE_WRONLY 2

static inline size_t hydro_mpi_type_size(MPI_Datatype t) { return (size_t)(t & 0xff); }

static inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return MPI_SUCCESS; }
static inline int MPI_Abort(MPI_Comm, int code) { exit(code); }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }

static inline int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype t, MPI_Op, MPI_Comm)
{
    if (send != recv) memcpy(recv, send, (size_t)count * hydro_mpi_type_size(t));
    return MPI_SUCCESS;
}

static inline int MPI_Reduce(const void *send, void *recv, int count, MPI_Datatype t, MPI_Op, int, MPI_Comm)
{
    if (send != recv) memcpy(recv, send, (size_t)count * hydro_mpi_type_size(t));
    return MPI_SUCCESS;
}

/* rank 0's receive buffer is undefined after an exclusive scan; leave it untouched */
static inline int MPI_Exscan(const void *, void *, int, MPI_Datatype, MPI_Op, MPI_Comm) { return MPI_SUCCESS; }

/* point-to-point calls exist only on the two-rank path; with one rank they are unreachable */
static inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *r)
{
    fprintf(stderr, "single-rank MPI stand-in: MPI_Isend is not available\n");
    *r = 0;
    return 1;
}
static inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *r)
{
    fprintf(stderr, "single-rank MPI stand-in: MPI_Irecv is not available\n");
    *r = 0;
    return 1;
}
static inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return MPI_SUCCESS; }

static inline int MPI_File_open(MPI_Comm, const char *name, int mode, MPI_Info, MPI_File *fh)
{
    int flags = 0;
    if (mode & MPI_MODE_CREATE) flags |= O_CREAT;
    flags |= (mode & MPI_MODE_WRONLY) ? O_WRONLY : O_RDWR;
    int fd = open(name, flags, 0644);
    if (fd < 0) { *fh = 0; return 1; }
    *fh = (MPI_File)malloc(sizeof(**fh));
    (*fh)->fd = fd;
    return MPI_SUCCESS;
}
static inline int MPI_File_set_size(MPI_File fh, MPI_Offset size)
{
    if (!fh) return 1;
    return ftruncate(fh->fd, (off_t)size) == 0 ? MPI_SUCCESS : 1;
}
static inline int MPI_File_write_at(MPI_File fh, MPI_Offset off, const void *buf, int count, MPI_Datatype t,
                                    MPI_Status *)
{
    if (!fh) return 1;
    size_t left = (size_t)count * hydro_mpi_type_size(t);
    const char *p = (const char *)buf;
    off_t pos = (off_t)off;
    while (left > 0) {
        ssize_t w = pwrite(fh->fd, p, left, pos);
        if (w <= 0) return 1;
        left -= (size_t)w; p += w; pos += w;
    }
    return MPI_SUCCESS;
}
static inline int MPI_File_close(MPI_File *fh)
{
    if (!fh || !*fh) return 1;
    close((*fh)->fd);
    free(*fh);
    *fh = 0;
    return MPI_SUCCESS;
}

#endif /* HYDRO_COMPAT_MPI_H */
