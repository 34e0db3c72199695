// ARTS data files, the solver states the reference reads and writes (core/data.f90:217-284
// data_read, :379-457 data_write_full3D; written by the init_flow tools through
// library/fileio_c.c, tools/init_flow/param.f90:113-148). Layout, native byte order:
//   int32 nx, ny, nz, nvars | float64 dt, time | nvars names of 8 blank-padded characters |
//   nvars fields of nx*ny*nz float64, each in Fortran order (i fastest)
// so variable v starts at byte 32 + 8*nvars + 8*nx*ny*nz*v (data.f90:270-271).
//
// The reader takes a sub-block (a rank's interior, data.f90:197-200) of the named variables
// straight into a species-major destination -- the layout of every batch entry point of this
// library -- on the host or on the device. Device transfers go through two pinned staging
// buffers: while one is copied to the device on the handle's stream, the file is read into the
// other.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "tiger_chem.h"
#include "tng_runtime.h"

using namespace tng;

namespace {

constexpr int kNameLen = 8;  // str_short (library/string.f90:3)
constexpr size_t kStage = size_t(16) << 20;  // bytes per pinned staging buffer

struct File {
  int fd = -1;
  ~File() {
    if (fd >= 0) close(fd);
  }
};

bool read_all(int fd, void* buf, size_t n, off_t off) {
  char* p = (char*)buf;
  while (n > 0) {
    const ssize_t r = pread(fd, p, n, off);
    if (r <= 0) return false;
    p += r, n -= (size_t)r, off += r;
  }
  return true;
}

bool write_all(int fd, const void* buf, size_t n, off_t off) {
  const char* p = (const char*)buf;
  while (n > 0) {
    const ssize_t r = pwrite(fd, p, n, off);
    if (r <= 0) return false;
    p += r, n -= (size_t)r, off += r;
  }
  return true;
}

std::string trimmed(const char* s, int n) {
  int e = n;
  while (e > 0 && (s[e - 1] == ' ' || s[e - 1] == '\0')) --e;
  return std::string(s, (size_t)e);
}

struct Header {
  int dims[4];
  double dt, time;
  std::vector<std::string> names;
  off_t data0;
};

int read_header(int fd, const char* who, const char* path, Header* h) {
  struct stat st;
  if (fstat(fd, &st) != 0) return set_error(TNG_ERR_ARG, "%s: cannot stat %s", who, path);
  unsigned char hd[32];
  if (!read_all(fd, hd, 32, 0)) return set_error(TNG_ERR_ARG, "%s: %s is shorter than a data-file header", who, path);
  std::memcpy(h->dims, hd, 16);
  std::memcpy(&h->dt, hd + 16, 8);
  std::memcpy(&h->time, hd + 24, 8);
  if (h->dims[0] <= 0 || h->dims[1] <= 0 || h->dims[2] <= 0 || h->dims[3] < 0 || h->dims[3] > 100000)
    return set_error(TNG_ERR_ARG, "%s: %s has an invalid header (%d x %d x %d, %d variables)", who, path, h->dims[0],
                     h->dims[1], h->dims[2], h->dims[3]);
  const int nv = h->dims[3];
  std::vector<char> nm((size_t)nv * kNameLen);
  if (nv && !read_all(fd, nm.data(), nm.size(), 32)) return set_error(TNG_ERR_ARG, "%s: %s: truncated names", who, path);
  h->names.clear();
  for (int v = 0; v < nv; ++v) h->names.push_back(trimmed(nm.data() + (size_t)v * kNameLen, kNameLen));
  h->data0 = 32 + (off_t)nv * kNameLen;
  const long long ncell = (long long)h->dims[0] * h->dims[1] * h->dims[2];
  if ((long long)st.st_size < (long long)h->data0 + 8LL * ncell * nv)
    return set_error(TNG_ERR_ARG, "%s: %s is shorter than its header announces", who, path);
  return TNG_OK;
}

// Pinned double-buffered staging between the file and device memory.
struct Stage {
  void* buf[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  bool used[2] = {false, false};
  int cur = 0;
  ~Stage() {
    for (int i = 0; i < 2; ++i) {
      if (ev[i]) cudaEventSynchronize(ev[i]), cudaEventDestroy(ev[i]);
      if (buf[i]) cudaFreeHost(buf[i]);
    }
  }
  cudaError_t init() {
    for (int i = 0; i < 2; ++i) {
      cudaError_t e = cudaHostAlloc(&buf[i], kStage, cudaHostAllocDefault);
      if (e != cudaSuccess) return e;
      if ((e = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming)) != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  // the next free buffer (waits for the copy that last used it)
  char* next() {
    cur ^= 1;
    if (used[cur]) cudaEventSynchronize(ev[cur]);
    return (char*)buf[cur];
  }
  void issued(cudaStream_t st) {
    cudaEventRecord(ev[cur], st);
    used[cur] = true;
  }
};

}  // namespace

extern "C" int tng_data_info(const char* path, int* dims, double* dt, double* time, char* names, int names_len) {
  if (!path || !dims) return set_error(TNG_ERR_ARG, "tng_data_info: null argument");
  File f;
  if ((f.fd = open(path, O_RDONLY)) < 0) return set_error(TNG_ERR_ARG, "tng_data_info: cannot open %s", path);
  Header h;
  int rc = read_header(f.fd, "tng_data_info", path, &h);
  if (rc) return rc;
  std::memcpy(dims, h.dims, sizeof(h.dims));
  if (dt) *dt = h.dt;
  if (time) *time = h.time;
  if (names) {
    const int need = h.dims[3] * kNameLen;
    if (names_len < need) return set_error(TNG_ERR_ARG, "tng_data_info: names buffer needs %d bytes", need);
    for (int v = 0; v < h.dims[3]; ++v) {
      char* d = names + (size_t)v * kNameLen;
      std::memset(d, ' ', kNameLen);
      std::memcpy(d, h.names[v].data(), h.names[v].size());
    }
  }
  return TNG_OK;
}

extern "C" int tng_data_read(tng_chem* hc, const char* path, const char* const* vars, int nvar, const int* start,
                             const int* count, double* out, int64_t ld, int flags) {
  if (!path || (!vars && nvar > 0) || nvar < 0 || (!out && nvar > 0))
    return set_error(TNG_ERR_ARG, "tng_data_read: null argument");
  if (flags != TNG_HOST_PTRS && flags != TNG_DEVICE_PTRS) return set_error(TNG_ERR_ARG, "tng_data_read: bad flags");
  if (flags == TNG_DEVICE_PTRS && !hc) return set_error(TNG_ERR_ARG, "tng_data_read: device output needs a handle");
  File f;
  if ((f.fd = open(path, O_RDONLY)) < 0) return set_error(TNG_ERR_ARG, "tng_data_read: cannot open %s", path);
  Header h;
  int rc = read_header(f.fd, "tng_data_read", path, &h);
  if (rc) return rc;
  const int nx = h.dims[0], ny = h.dims[1], nz = h.dims[2];
  int s[3] = {0, 0, 0}, c[3] = {nx, ny, nz};
  if (start) std::copy(start, start + 3, s);
  if (count) std::copy(count, count + 3, c);
  for (int d = 0; d < 3; ++d)
    if (s[d] < 0 || c[d] <= 0 || s[d] + c[d] > h.dims[d])
      return set_error(TNG_ERR_ARG, "tng_data_read: block outside the %d x %d x %d grid", nx, ny, nz);
  const long long ncell = (long long)c[0] * c[1] * c[2];
  if (ld < ncell) return set_error(TNG_ERR_ARG, "tng_data_read: ld < cells of the block");
  std::vector<int> idx(nvar);
  for (int v = 0; v < nvar; ++v) {
    if (!vars[v]) return set_error(TNG_ERR_ARG, "tng_data_read: null variable name");
    const std::string want = trimmed(vars[v], (int)strnlen(vars[v], 64));
    auto it = std::find(h.names.begin(), h.names.end(), want);
    if (it == h.names.end()) return set_error(TNG_ERR_ARG, "tng_data_read: %s has no variable '%s'", path, want.c_str());
    idx[v] = (int)(it - h.names.begin());
  }
  const long long plane = (long long)nx * ny, field = plane * nz;
  const bool whole_lines = (c[0] == nx);
  const bool whole_planes = whole_lines && (c[1] == ny);
  // file offset (bytes) of (i, j, k) of variable v
  auto off = [&](int v, long long i, long long j, long long k) {
    return h.data0 + 8 * ((off_t)idx[v] * field + i + (off_t)nx * j + (off_t)plane * k);
  };
  if (flags == TNG_HOST_PTRS) {
    for (int v = 0; v < nvar; ++v) {
      double* dst = out + (size_t)v * ld;
      if (whole_planes) {
        if (!read_all(f.fd, dst, 8 * (size_t)ncell, off(v, 0, 0, s[2]))) goto io_error;
        continue;
      }
      for (long long k = 0; k < c[2]; ++k)
        for (long long j = 0; j < c[1]; ++j)
          if (!read_all(f.fd, dst + c[0] * (j + (long long)c[1] * k), 8 * (size_t)c[0], off(v, s[0], s[1] + j, s[2] + k)))
            goto io_error;
    }
    return TNG_OK;
  }
  {
    DeviceGuard g(hc->cfg.device);
    Stage stg;
    cudaError_t e = stg.init();
    if (e != cudaSuccess) return cuda_error(e, "tng_data_read: staging");
    const size_t cap = kStage / 8;
    for (int v = 0; v < nvar; ++v) {
      double* dst = out + (size_t)v * ld;
      // walk the block in file order, filling a staging buffer with consecutive destination cells
      long long done = 0;
      while (done < ncell) {
        double* buf = (double*)stg.next();
        const long long take = std::min<long long>((long long)cap, ncell - done);
        long long got = 0;
        while (got < take) {
          const long long cell = done + got;
          const long long i = cell % c[0], jk = cell / c[0];
          const long long j = jk % c[1], k = jk / c[1];
          // the run of consecutive cells contiguous in the file from here
          const long long run = whole_planes ? take - got
                                : whole_lines ? std::min(take - got, (long long)c[0] * c[1] - (c[0] * j + i))
                                              : std::min(take - got, (long long)c[0] - i);
          if (!read_all(f.fd, buf + got, 8 * (size_t)run, off(v, s[0] + i, s[1] + j, s[2] + k))) goto io_error;
          got += run;
        }
        e = cudaMemcpyAsync(dst + done, buf, 8 * (size_t)take, cudaMemcpyHostToDevice, hc->stream);
        if (e != cudaSuccess) return cuda_error(e, "tng_data_read");
        stg.issued(hc->stream);
        done += take;
      }
    }
    if ((e = cudaStreamSynchronize(hc->stream)) != cudaSuccess) return cuda_error(e, "tng_data_read");
    return TNG_OK;
  }
io_error:
  return set_error(TNG_ERR_ARG, "tng_data_read: read error in %s", path);
}

extern "C" int tng_data_write(tng_chem* hc, const char* path, const int* dims, const char* const* vars, int nvar,
                              double dt, double time, const double* fields, int64_t ld, int flags) {
  if (!path || !dims || nvar < 0 || (nvar > 0 && (!vars || !fields)))
    return set_error(TNG_ERR_ARG, "tng_data_write: null argument");
  if (flags != TNG_HOST_PTRS && flags != TNG_DEVICE_PTRS) return set_error(TNG_ERR_ARG, "tng_data_write: bad flags");
  if (flags == TNG_DEVICE_PTRS && !hc) return set_error(TNG_ERR_ARG, "tng_data_write: device input needs a handle");
  if (dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0) return set_error(TNG_ERR_ARG, "tng_data_write: bad grid size");
  const long long ncell = (long long)dims[0] * dims[1] * dims[2];
  if (ld < ncell) return set_error(TNG_ERR_ARG, "tng_data_write: ld < cells of the grid");
  std::vector<char> head(32 + (size_t)nvar * kNameLen, ' ');
  const int d4[4] = {dims[0], dims[1], dims[2], nvar};
  std::memcpy(head.data(), d4, 16);
  std::memcpy(head.data() + 16, &dt, 8);
  std::memcpy(head.data() + 24, &time, 8);
  for (int v = 0; v < nvar; ++v) {
    if (!vars[v]) return set_error(TNG_ERR_ARG, "tng_data_write: null variable name");
    const size_t n = strnlen(vars[v], 64);
    if (n > (size_t)kNameLen) return set_error(TNG_ERR_ARG, "tng_data_write: name '%s' longer than 8", vars[v]);
    std::memcpy(head.data() + 32 + (size_t)v * kNameLen, vars[v], n);
  }
  File f;
  if ((f.fd = open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644)) < 0)
    return set_error(TNG_ERR_ARG, "tng_data_write: cannot create %s", path);
  if (!write_all(f.fd, head.data(), head.size(), 0)) return set_error(TNG_ERR_ARG, "tng_data_write: write error");
  const off_t data0 = (off_t)head.size();
  if (flags == TNG_HOST_PTRS) {
    for (int v = 0; v < nvar; ++v)
      if (!write_all(f.fd, fields + (size_t)v * ld, 8 * (size_t)ncell, data0 + 8 * (off_t)ncell * v))
        return set_error(TNG_ERR_ARG, "tng_data_write: write error");
    return TNG_OK;
  }
  DeviceGuard g(hc->cfg.device);
  Stage stg;
  cudaError_t e = stg.init();
  if (e != cudaSuccess) return cuda_error(e, "tng_data_write: staging");
  const long long cap = (long long)(kStage / 8);
  // copy chunk n+1 to the host while chunk n is written to the file
  struct Pending {
    char* buf;
    long long n;
    off_t at;
  };
  std::vector<Pending> pend;
  for (int v = 0; v < nvar; ++v)
    for (long long done = 0; done < ncell; done += cap) {
      const long long take = std::min(cap, ncell - done);
      char* buf = stg.next();
      // the buffer's previous chunk (if any) was already written below before being reused
      e = cudaMemcpyAsync(buf, fields + (size_t)v * ld + done, 8 * (size_t)take, cudaMemcpyDeviceToHost, hc->stream);
      if (e != cudaSuccess) return cuda_error(e, "tng_data_write");
      stg.issued(hc->stream);
      pend.push_back({buf, take, data0 + 8 * ((off_t)ncell * v + done)});
      if (pend.size() == 2) {  // write the older chunk (its copy is done once its event is)
        cudaEventSynchronize(stg.ev[stg.cur ^ 1]);
        if (!write_all(f.fd, pend[0].buf, 8 * (size_t)pend[0].n, pend[0].at))
          return set_error(TNG_ERR_ARG, "tng_data_write: write error");
        pend.erase(pend.begin());
      }
    }
  if ((e = cudaStreamSynchronize(hc->stream)) != cudaSuccess) return cuda_error(e, "tng_data_write");
  for (const Pending& p : pend)
    if (!write_all(f.fd, p.buf, 8 * (size_t)p.n, p.at)) return set_error(TNG_ERR_ARG, "tng_data_write: write error");
  return TNG_OK;
}
