// restart.cu -- the restart-file transfer pipeline (see restart.cuh).
#include "restart.cuh"

#include <cerrno>
#include <cstring>
#include <unistd.h>

#include "obl.h"

namespace obl {

// dst (nxt, nyt, nl) FP64 <- levels z0 .. z0+nl-1 of var (ldx, nyt, .)
template <typename T>
__global__ void k_pack_f64(double *dst, const T *var, int nxt, int ldx, int nyt, int z0, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / nxt;
        const int x = (int)(i - r * nxt), y = (int)(r % nyt), l = (int)(r / nyt);
        dst[i] = (double)var[((long long)(z0 + l) * nyt + y) * ldx + x];
    }
}

template <typename T>
__global__ void k_unpack_f64(T *var, const double *src, int nxt, int ldx, int nyt, int z0, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / nxt;
        const int x = (int)(i - r * nxt), y = (int)(r % nyt), l = (int)(r / nyt);
        var[((long long)(z0 + l) * nyt + y) * ldx + x] = (T)src[i];
    }
}

static unsigned grid_for(long long n)
{
    const long long want = (n + 255) / 256;
    return (unsigned)(want < 148 * 16 ? want : 148 * 16);
}

static int io_err(std::string &err, const std::string &what)
{
    err = what + ": " + std::strerror(errno);
    return OBL_ERR_IO;
}

static int cu_err(std::string &err, cudaError_t e, const char *what)
{
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return OBL_ERR_CUDA;
}

static int write_all(int fd, const void *p, size_t n, long long off, std::string &err)
{
    const char *c = (const char *)p;
    while (n) {
        const ssize_t w = pwrite(fd, c, n, (off_t)off);
        if (w < 0) {
            if (errno == EINTR) continue;
            return io_err(err, "pwrite");
        }
        c += w;
        n -= (size_t)w;
        off += w;
    }
    return OBL_OK;
}

static int read_all(int fd, void *p, size_t n, long long off, std::string &err)
{
    char *c = (char *)p;
    while (n) {
        const ssize_t r = pread(fd, c, n, (off_t)off);
        if (r < 0) {
            if (errno == EINTR) continue;
            return io_err(err, "pread");
        }
        if (r == 0) {
            err = "restart file too short: " + std::to_string(n) + " bytes missing at offset " + std::to_string(off);
            return OBL_ERR_IO;
        }
        c += r;
        n -= (size_t)r;
        off += r;
    }
    return OBL_OK;
}

int io_stage_reserve(IoStage &s, size_t doubles, std::string &err)
{
    if (s.cap >= doubles) return OBL_OK;
    io_stage_free(s);
    for (int k = 0; k < 2; ++k) {
        if (cudaMalloc(&s.dev[k], doubles * sizeof(double)) != cudaSuccess ||
            cudaHostAlloc(&s.host[k], doubles * sizeof(double), cudaHostAllocDefault) != cudaSuccess ||
            cudaEventCreateWithFlags(&s.ev[k], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            io_stage_free(s);
            err = "restart staging: allocation of 2 x " + std::to_string(doubles * sizeof(double)) + " bytes failed";
            return OBL_ERR_NOMEM;
        }
    }
    s.cap = doubles;
    return OBL_OK;
}

void io_stage_free(IoStage &s)
{
    for (int k = 0; k < 2; ++k) {
        if (s.dev[k]) cudaFree(s.dev[k]);
        if (s.host[k]) cudaFreeHost(s.host[k]);
        if (s.ev[k]) cudaEventDestroy(s.ev[k]);
        s.dev[k] = nullptr;
        s.host[k] = nullptr;
        s.ev[k] = nullptr;
    }
    s.cap = 0;
}

template <typename T>
int io_write_field(IoStage &s, cudaStream_t st, int fd, long long off, const T *var, int nxt, int ldx, int nyt,
                   int nz, std::string &err)
{
    const long long plane = (long long)nxt * nyt;
    const int L = nz - 1, per = (int)(s.cap / plane);
    if (per < 1) {
        err = "restart staging smaller than one plane";
        return OBL_ERR_ARG;
    }
    const int nch = (L + per - 1) / per;
    cudaError_t e;
    int rc;
    // chunk c: levels 1 + c*per .. ; packed on the GPU, copied to host[c%2]; the file
    // write of chunk c-1 overlaps the GPU work of chunk c
    for (int c = 0; c <= nch; ++c) {
        if (c < nch) {
            const int z0 = 1 + c * per, nl = (L - c * per) < per ? (L - c * per) : per;
            const long long n = plane * nl;
            double *d = s.dev[c & 1], *h = s.host[c & 1];
            if (var) {
                k_pack_f64<T><<<grid_for(n), 256, 0, st>>>(d, var, nxt, ldx, nyt, z0, n);
                if ((e = cudaGetLastError()) != cudaSuccess) return cu_err(err, e, "restart pack");
                if ((e = cudaMemcpyAsync(h, d, n * sizeof(double), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
                    return cu_err(err, e, "restart copy");
            } else if ((e = cudaMemsetAsync(d, 0, n * sizeof(double), st)) != cudaSuccess ||
                       (e = cudaMemcpyAsync(h, d, n * sizeof(double), cudaMemcpyDeviceToHost, st)) != cudaSuccess) {
                return cu_err(err, e, "restart zeros");
            }
            if ((e = cudaEventRecord(s.ev[c & 1], st)) != cudaSuccess) return cu_err(err, e, "restart event");
        }
        if (c > 0) {
            const int p = c - 1;
            const int nl = (L - p * per) < per ? (L - p * per) : per;
            if ((e = cudaEventSynchronize(s.ev[p & 1])) != cudaSuccess) return cu_err(err, e, "restart copy");
            if ((rc = write_all(fd, s.host[p & 1], (size_t)(plane * nl) * sizeof(double),
                                off + (long long)p * per * plane * (long long)sizeof(double), err))) {
                cudaStreamSynchronize(st);   // nothing may still copy into the pinned chunks
                return rc;
            }
        }
    }
    return OBL_OK;
}

template <typename T>
int io_read_field(IoStage &s, cudaStream_t st, int fd, long long off, T *var, int nxt, int ldx, int nyt, int nz,
                  std::string &err)
{
    const long long plane = (long long)nxt * nyt;
    const int L = nz - 1, per = (int)(s.cap / plane);
    if (per < 1) {
        err = "restart staging smaller than one plane";
        return OBL_ERR_ARG;
    }
    const int nch = (L + per - 1) / per;
    auto levels = [&](int c) { return (L - c * per) < per ? (L - c * per) : per; };
    cudaError_t e;
    int rc;
    if ((rc = read_all(fd, s.host[0], (size_t)(plane * levels(0)) * sizeof(double), off, err))) return rc;
    // chunk c: copied up from host[c%2] and unpacked; the file read of chunk c+1 into the
    // other host chunk overlaps it (that chunk's previous copy, c-1, is waited for first)
    for (int c = 0; c < nch; ++c) {
        const long long n = plane * levels(c);
        double *d = s.dev[c & 1], *h = s.host[c & 1];
        if ((e = cudaMemcpyAsync(d, h, n * sizeof(double), cudaMemcpyHostToDevice, st)) != cudaSuccess)
            return cu_err(err, e, "restart copy");
        if ((e = cudaEventRecord(s.ev[c & 1], st)) != cudaSuccess) return cu_err(err, e, "restart event");
        k_unpack_f64<T><<<grid_for(n), 256, 0, st>>>(var, d, nxt, ldx, nyt, 1 + c * per, n);
        if ((e = cudaGetLastError()) != cudaSuccess) return cu_err(err, e, "restart unpack");
        if (c + 1 < nch) {
            const int q = c + 1;
            if (q >= 2 && (e = cudaEventSynchronize(s.ev[q & 1])) != cudaSuccess) return cu_err(err, e, "restart copy");
            if ((rc = read_all(fd, s.host[q & 1], (size_t)(plane * levels(q)) * sizeof(double),
                               off + (long long)q * per * plane * (long long)sizeof(double), err))) {
                cudaStreamSynchronize(st);   // nothing may still copy out of the pinned chunks
                return rc;
            }
        }
    }
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cu_err(err, e, "restart unpack");
    return OBL_OK;
}

template int io_write_field<float>(IoStage &, cudaStream_t, int, long long, const float *, int, int, int, int,
                                   std::string &);
template int io_write_field<double>(IoStage &, cudaStream_t, int, long long, const double *, int, int, int, int,
                                    std::string &);
template int io_read_field<float>(IoStage &, cudaStream_t, int, long long, float *, int, int, int, int, std::string &);
template int io_read_field<double>(IoStage &, cudaStream_t, int, long long, double *, int, int, int, int,
                                   std::string &);

} // namespace obl
