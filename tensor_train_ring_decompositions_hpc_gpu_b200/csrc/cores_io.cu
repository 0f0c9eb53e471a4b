// Core files: header + column-major FP32 cores (format in include/ttrsvd.h).
#include <stdio.h>
#include <string.h>

#include <vector>

#include "kernels.cuh"

namespace {

constexpr char kMagic[8] = {'T', 'T', 'R', 'C', 'O', 'R', 'E', '1'};

struct Header {
  int kind = 0, d = 0, dtype = 0;
  long long n[TT_MAX_ORDER] = {0};
  long long r[TT_MAX_ORDER + 1] = {0};
};

struct File {
  FILE* f = nullptr;
  explicit File(const char* path, const char* mode) : f(fopen(path, mode)) {}
  ~File() {
    if (f) fclose(f);
  }
};

int io_error(const char* what, const char* path) {
  ttr::set_error(TT_ERR_IO, "%s: %s", what, path ? path : "(null)");
  return TT_ERR_IO;
}

int read_header(FILE* f, const char* path, Header& h) {
  char magic[8];
  int words[4];
  if (fread(magic, 1, 8, f) != 8 || memcmp(magic, kMagic, 8) != 0) return io_error("not a core file", path);
  if (fread(words, sizeof(int), 4, f) != 4) return io_error("truncated header", path);
  h.kind = words[0];
  h.d = words[1];
  h.dtype = words[2];
  if ((h.kind != 0 && h.kind != 1) || h.d < 2 || h.d > TT_MAX_ORDER || h.dtype != 0)
    return io_error("unsupported header (kind, order or dtype)", path);
  if (fread(h.n, sizeof(long long), h.d, f) != (size_t)h.d ||
      fread(h.r, sizeof(long long), h.d + 1, f) != (size_t)h.d + 1)
    return io_error("truncated header", path);
  for (int k = 0; k < h.d; ++k)
    if (h.n[k] < 1 || h.n[k] > (1LL << 31)) return io_error("bad mode size", path);
  for (int k = 0; k <= h.d; ++k)
    if (h.r[k] < 1 || h.r[k] > (1LL << 31)) return io_error("bad rank", path);
  return TT_OK;
}

}  // namespace

extern "C" int tt_cores_save(const char* path, int d, const int* n, const int* r, int ring,
                             const float* const* cores, int device) {
  if (!path || !n || !r || !cores) {
    ttr::set_error(TT_ERR_ARG, "null argument");
    return TT_ERR_ARG;
  }
  if (d < 2 || d > TT_MAX_ORDER) {
    ttr::set_error(TT_ERR_SHAPE, "order %d", d);
    return TT_ERR_SHAPE;
  }
  for (int k = 0; k < d; ++k)
    if (!cores[k] || n[k] < 1 || r[k] < 1 || r[k + 1] < 1) {
      ttr::set_error(TT_ERR_ARG, "core %d: null pointer or non-positive size", k);
      return TT_ERR_ARG;
    }
  File fo(path, "wb");
  if (!fo.f) return io_error("cannot open for writing", path);
  const int words[4] = {ring ? 1 : 0, d, 0, 0};
  long long nn[TT_MAX_ORDER], rr[TT_MAX_ORDER + 1];
  for (int k = 0; k < d; ++k) nn[k] = n[k];
  for (int k = 0; k <= d; ++k) rr[k] = r[k];
  if (fwrite(kMagic, 1, 8, fo.f) != 8 || fwrite(words, sizeof(int), 4, fo.f) != 4 ||
      fwrite(nn, sizeof(long long), d, fo.f) != (size_t)d ||
      fwrite(rr, sizeof(long long), d + 1, fo.f) != (size_t)d + 1)
    return io_error("write failed", path);
  std::vector<float> stage;
  for (int k = 0; k < d; ++k) {
    const size_t cnt = (size_t)r[k] * n[k] * r[k + 1];
    const float* src = cores[k];
    if (device) {
      stage.resize(cnt);
      TT_CUDA(cudaMemcpy(stage.data(), cores[k], cnt * sizeof(float), cudaMemcpyDeviceToHost));
      src = stage.data();
    }
    if (fwrite(src, sizeof(float), cnt, fo.f) != cnt) return io_error("write failed", path);
  }
  if (fflush(fo.f) != 0) return io_error("write failed", path);
  return TT_OK;
}

extern "C" int tt_cores_header(const char* path, int* d, int* n, int* r, int* ring) {
  if (!path || !d || !n || !r || !ring) {
    ttr::set_error(TT_ERR_ARG, "null argument");
    return TT_ERR_ARG;
  }
  File fi(path, "rb");
  if (!fi.f) return io_error("cannot open", path);
  Header h;
  TT_TRY(read_header(fi.f, path, h));
  *d = h.d;
  *ring = h.kind;
  for (int k = 0; k < h.d; ++k) n[k] = (int)h.n[k];
  for (int k = 0; k <= h.d; ++k) r[k] = (int)h.r[k];
  return TT_OK;
}

extern "C" int tt_cores_load(const char* path, float* const* cores, int device) {
  if (!path || !cores) {
    ttr::set_error(TT_ERR_ARG, "null argument");
    return TT_ERR_ARG;
  }
  File fi(path, "rb");
  if (!fi.f) return io_error("cannot open", path);
  Header h;
  TT_TRY(read_header(fi.f, path, h));
  std::vector<float> stage;
  for (int k = 0; k < h.d; ++k) {
    if (!cores[k]) {
      ttr::set_error(TT_ERR_ARG, "null core pointer %d", k);
      return TT_ERR_ARG;
    }
    const size_t cnt = (size_t)(h.r[k] * h.n[k] * h.r[k + 1]);
    float* dst = cores[k];
    if (device) {
      stage.resize(cnt);
      dst = stage.data();
    }
    if (fread(dst, sizeof(float), cnt, fi.f) != cnt) return io_error("truncated core data", path);
    if (device) TT_CUDA(cudaMemcpy(cores[k], stage.data(), cnt * sizeof(float), cudaMemcpyHostToDevice));
  }
  return TT_OK;
}
