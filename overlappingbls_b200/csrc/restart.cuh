// restart.cuh -- restart files of the reference (012_io.f90:496-589 checkpoint_final,
// 102_01_ic.f90:682-737 read_flow_field, 202_parallel.f90:1084-1250 write/read_file_mpi_3d).
//
// A field in the file is the global FP64 array (nxt, nyt, nzt-1) in Fortran order: the
// interior levels 1..nz-1 of every z-rank, rank r's block at z offset r*(nz-1) (the MPI
// subarray start (0, 0, (nz-1)*coordz) with npy = 1), at byte offset disp0.  On the GPU a
// field is (ldx, nyt, 0:nz) in the storage type.
//
// Transfer: the levels go through the file in chunks of whole planes.  Each chunk is
// packed on the GPU (pads dropped, widened to FP64) into one of two device chunks, copied
// into one of two pinned host chunks and written with pwrite while the GPU packs and
// copies the next one; reading runs the same pipeline backwards (pread, copy, unpack).
#pragma once
#include <cuda_runtime.h>

#include <string>

namespace obl {

struct IoStage {
    double *dev[2] = {nullptr, nullptr};
    double *host[2] = {nullptr, nullptr};   // pinned
    cudaEvent_t ev[2] = {nullptr, nullptr};
    size_t cap = 0;                          // doubles per chunk
};

// chunks of up to `doubles` doubles (at least one plane); returns an OBL_* status
int io_stage_reserve(IoStage &s, size_t doubles, std::string &err);
void io_stage_free(IoStage &s);

// Levels 1..nz-1, x < nxt of the device field var (zeros when var is null) written as
// FP64 at byte offset off of the open file fd.
template <typename T>
int io_write_field(IoStage &s, cudaStream_t st, int fd, long long off, const T *var, int nxt, int ldx, int nyt,
                   int nz, std::string &err);
// Levels 1..nz-1, x < nxt of the device field var read from byte offset off of fd (the
// pads and levels 0, nz are left as they are).
template <typename T>
int io_read_field(IoStage &s, cudaStream_t st, int fd, long long off, T *var, int nxt, int ldx, int nyt, int nz,
                  std::string &err);

} // namespace obl
