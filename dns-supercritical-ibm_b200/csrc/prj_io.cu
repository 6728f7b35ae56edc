// prj_io.cu -- the reference's field files (src/mod_io.f90:7-149), host and device.
//
// A file is stream-unformatted: three 4-byte integers nx, nz, ny, then the
// nx*nz*ny interior values as float64, x fastest, then z, then y (the order of
// cfd_write_arr's loops, :113-121), in the machine's byte order.  The device
// forms move the field in chunks of y-planes through two pinned host buffers,
// so the file transfer of one chunk overlaps the host<->device copy of the
// other.  Reads check the header against the expected grid, as cfd_read_arr
// does (:24-33), and report a mismatch as an error instead of stopping.
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/projection.h"
#include "prj_internal.h"

namespace {

int io_fail(int code, const char* fmt, const char* a = "", long b = 0, long c = 0, long d = 0) {
    char buf[512];
    std::snprintf(buf, sizeof(buf), fmt, a, b, c, d);
    return prj::record_error(code, buf);
}

struct File {
    FILE* f = nullptr;
    ~File() {
        if (f) std::fclose(f);
    }
};

bool dims_ok(int nx, int nz, int ny) { return nx >= 1 && nz >= 1 && ny >= 1; }

// element offset of interior point (0, 0, k) and the row pitch of the array form
size_t plane_offset(int nx, int nz, int k, int halo) {
    if (!halo) return (size_t)k * nz * nx;
    return 1 + (size_t)(nx + 2) * (1 + (size_t)(nz + 2) * (size_t)(k + 1));
}
size_t row_pitch(int nx, int halo) { return (size_t)(halo ? nx + 2 : nx); }

int open_read(File& fh, const char* path, int nx, int nz, int ny) {
    fh.f = std::fopen(path, "rb");
    if (!fh.f) return io_fail(PRJ_ERR_ARG, "cannot open %s for reading", path);
    int hdr[3];
    if (std::fread(hdr, sizeof(int), 3, fh.f) != 3) return io_fail(PRJ_ERR_ARG, "%s: short header", path);
    if (hdr[0] != nx || hdr[1] != nz || hdr[2] != ny)
        return io_fail(PRJ_ERR_ARG, "%s: grid mismatch, file has %ld x %ld x %ld", path, hdr[0], hdr[1], hdr[2]);
    return PRJ_OK;
}

int open_write(File& fh, const char* path, int nx, int nz, int ny) {
    fh.f = std::fopen(path, "wb");
    if (!fh.f) return io_fail(PRJ_ERR_ARG, "cannot open %s for writing", path);
    const int hdr[3] = {nx, nz, ny};
    if (std::fwrite(hdr, sizeof(int), 3, fh.f) != 3) return io_fail(PRJ_ERR_ARG, "%s: write failed", path);
    return PRJ_OK;
}

// pinned double buffer, chunk = whole y-planes of about 64 MB
struct Staging {
    double* buf[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
    cudaStream_t st = nullptr;
    int planes = 1;
    ~Staging() {
        if (st) cudaStreamSynchronize(st);
        for (int i = 0; i < 2; i++) {
            if (buf[i]) cudaFreeHost(buf[i]);
            if (done[i]) cudaEventDestroy(done[i]);
        }
        if (st) cudaStreamDestroy(st);
    }
    int init(int nx, int nz, int ny) {
        const size_t plane = (size_t)nx * nz * sizeof(double);
        planes = (int)std::max<size_t>(1, std::min<size_t>((size_t)ny, ((size_t)64 << 20) / plane));
        for (int i = 0; i < 2; i++) {
            if (cudaMallocHost((void**)&buf[i], plane * planes) != cudaSuccess ||
                cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming) != cudaSuccess)
                return io_fail(PRJ_ERR_OOM, "pinned staging%s of %ld bytes failed", "", (long)(plane * planes));
        }
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
            return io_fail(PRJ_ERR_CUDA, "stream creation failed");
        return PRJ_OK;
    }
};

// makes `device` current (and restores the caller's device on exit), then waits
// for the device's pending work, so the array is neither being written nor read
struct OnDevice {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit OnDevice(int device) {
        cudaGetDevice(&prev);
        err = cudaSetDevice(device);
        if (err == cudaSuccess) err = cudaDeviceSynchronize();
    }
    ~OnDevice() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// copy planes [k0, k0 + n) between a contiguous host chunk and the device array
cudaError_t copy_planes(double* d, int nx, int nz, int k0, int n, int halo, double* h, bool to_device, cudaStream_t st) {
    const size_t w = (size_t)nx * sizeof(double);
    for (int k = 0; k < n; k++) {
        double* dp = d + plane_offset(nx, nz, k0 + k, halo);
        double* hp = h + (size_t)k * nz * nx;
        const size_t dpitch = row_pitch(nx, halo) * sizeof(double);
        const cudaError_t e = to_device ? cudaMemcpy2DAsync(dp, dpitch, hp, w, w, nz, cudaMemcpyHostToDevice, st)
                                        : cudaMemcpy2DAsync(hp, w, dp, dpitch, w, nz, cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace

extern "C" {

int prj_field_read_header(const char* path, int* nx, int* nz, int* ny) {
    if (!path || !nx || !nz || !ny) return io_fail(PRJ_ERR_ARG, "NULL argument%s");
    File fh;
    fh.f = std::fopen(path, "rb");
    if (!fh.f) return io_fail(PRJ_ERR_ARG, "cannot open %s for reading", path);
    int hdr[3];
    if (std::fread(hdr, sizeof(int), 3, fh.f) != 3) return io_fail(PRJ_ERR_ARG, "%s: short header", path);
    *nx = hdr[0];
    *nz = hdr[1];
    *ny = hdr[2];
    return PRJ_OK;
}

int prj_field_write(const char* path, int nx, int nz, int ny, const double* h_src, int halo) {
    if (!path || !h_src || !dims_ok(nx, nz, ny)) return io_fail(PRJ_ERR_ARG, "bad path, array or grid%s");
    File fh;
    int rc = open_write(fh, path, nx, nz, ny);
    if (rc) return rc;
    for (int k = 0; k < ny; k++)
        for (int j = 0; j < nz; j++) {
            const double* row = h_src + plane_offset(nx, nz, k, halo) + (size_t)j * row_pitch(nx, halo);
            if (std::fwrite(row, sizeof(double), (size_t)nx, fh.f) != (size_t)nx)
                return io_fail(PRJ_ERR_ARG, "%s: write failed", path);
        }
    if (std::fclose(fh.f) != 0) {
        fh.f = nullptr;
        return io_fail(PRJ_ERR_ARG, "%s: close failed", path);
    }
    fh.f = nullptr;
    return PRJ_OK;
}

int prj_field_read(const char* path, int nx, int nz, int ny, double* h_dst, int halo) {
    if (!path || !h_dst || !dims_ok(nx, nz, ny)) return io_fail(PRJ_ERR_ARG, "bad path, array or grid%s");
    File fh;
    int rc = open_read(fh, path, nx, nz, ny);
    if (rc) return rc;
    for (int k = 0; k < ny; k++)
        for (int j = 0; j < nz; j++) {
            double* row = h_dst + plane_offset(nx, nz, k, halo) + (size_t)j * row_pitch(nx, halo);
            if (std::fread(row, sizeof(double), (size_t)nx, fh.f) != (size_t)nx)
                return io_fail(PRJ_ERR_ARG, "%s: file shorter than its grid", path);
        }
    return PRJ_OK;
}

int prj_field_read_device(const char* path, int nx, int nz, int ny, double* d_dst, int halo, int device) {
    if (!path || !d_dst || !dims_ok(nx, nz, ny)) return io_fail(PRJ_ERR_ARG, "bad path, array or grid%s");
    OnDevice od(device);
    if (od.err != cudaSuccess) return io_fail(PRJ_ERR_CUDA, "device %s unavailable", cudaGetErrorString(od.err));
    File fh;
    int rc = open_read(fh, path, nx, nz, ny);
    if (rc) return rc;
    Staging s;
    if ((rc = s.init(nx, nz, ny))) return rc;
    const size_t plane = (size_t)nx * nz;
    int c = 0;
    for (int k0 = 0; k0 < ny; k0 += s.planes, c ^= 1) {
        const int n = std::min(s.planes, ny - k0);
        // the copy that last used this buffer must be done before the file overwrites it
        if (cudaEventSynchronize(s.done[c]) != cudaSuccess) return io_fail(PRJ_ERR_CUDA, "staging wait failed%s");
        if (std::fread(s.buf[c], sizeof(double), plane * n, fh.f) != plane * n)
            return io_fail(PRJ_ERR_ARG, "%s: file shorter than its grid", path);
        if (copy_planes(d_dst, nx, nz, k0, n, halo, s.buf[c], true, s.st) != cudaSuccess ||
            cudaEventRecord(s.done[c], s.st) != cudaSuccess)
            return io_fail(PRJ_ERR_CUDA, "host to device copy failed%s");
    }
    if (cudaStreamSynchronize(s.st) != cudaSuccess) return io_fail(PRJ_ERR_CUDA, "copy failed%s");
    return PRJ_OK;
}

int prj_field_write_device(const char* path, int nx, int nz, int ny, const double* d_src, int halo, int device) {
    if (!path || !d_src || !dims_ok(nx, nz, ny)) return io_fail(PRJ_ERR_ARG, "bad path, array or grid%s");
    OnDevice od(device);
    if (od.err != cudaSuccess) return io_fail(PRJ_ERR_CUDA, "device %s unavailable", cudaGetErrorString(od.err));
    File fh;
    int rc = open_write(fh, path, nx, nz, ny);
    if (rc) return rc;
    Staging s;
    if ((rc = s.init(nx, nz, ny))) return rc;
    const size_t plane = (size_t)nx * nz;
    const int nch = (ny + s.planes - 1) / s.planes;
    auto issue = [&](int ch) {
        const int k0 = ch * s.planes, n = std::min(s.planes, ny - k0);
        if (copy_planes(const_cast<double*>(d_src), nx, nz, k0, n, halo, s.buf[ch & 1], false, s.st) != cudaSuccess ||
            cudaEventRecord(s.done[ch & 1], s.st) != cudaSuccess)
            return false;
        return true;
    };
    if (!issue(0)) return io_fail(PRJ_ERR_CUDA, "device to host copy failed%s");
    for (int ch = 0; ch < nch; ch++) {
        // chunk ch + 1 streams in while chunk ch goes to the file
        if (ch + 1 < nch && !issue(ch + 1)) return io_fail(PRJ_ERR_CUDA, "device to host copy failed%s");
        if (cudaEventSynchronize(s.done[ch & 1]) != cudaSuccess) return io_fail(PRJ_ERR_CUDA, "staging wait failed%s");
        const int n = std::min(s.planes, ny - ch * s.planes);
        if (std::fwrite(s.buf[ch & 1], sizeof(double), plane * n, fh.f) != plane * n)
            return io_fail(PRJ_ERR_ARG, "%s: write failed", path);
        // chunk ch + 2 reuses this buffer: issued only after the write above
    }
    if (std::fclose(fh.f) != 0) {
        fh.f = nullptr;
        return io_fail(PRJ_ERR_ARG, "%s: close failed", path);
    }
    fh.f = nullptr;
    return PRJ_OK;
}

}  // extern "C"
