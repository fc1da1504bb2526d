// api_gio.cu -- GIO POSIX state files (io/gio.ipp) read and written
// straight from and into device memory.
//
// One file holds one field of one rank: a header followed by the field's
// Ftype values in the E-vector order of the device array.  The header is,
// field by field (io/gio.ipp:459-503 writes it, 587-620 reads it back,
// 676-690 gives its size):
//   int32  ivers                 format version
//   int32  dim
//   uint64 nelems
//   int32  porder[numr * dim]    numr = 1 if ivers == 0, else nelems
//   int32  gtype                 GElemType: 0 regular, 1 deformed, 2 embedded
//   uint64 cycle
//   Ftype  time
//   int32  multivar
//   uint64 elemids[nelems]       GKEY element keys
// Ftype is the state's float type (double, or float for a single-precision
// build); the file does not record it.  The data that follow are
// nelems * prod_d (porder[0][d] + 1) values for ivers 0, else
// sum_e prod_d (porder[e][d] + 1) (io/gio.ipp:416-429).
//
// The field streams through two pinned staging buffers: while one chunk is
// copied between HBM and host memory on the context's stream, the other is
// written to (or read from) the file, so that disk and PCIe/C2C traffic
// overlap and no host copy of the whole field is ever held.
#include <cstdio>
#include <cstring>
#include <vector>

#include "gf_common.cuh"

namespace {

constexpr size_t kChunk = size_t(32) << 20;  // bytes per staging buffer

size_t header_bytes(int ivers, int dim, uint64_t nelems, int fbytes) {
  const uint64_t numr = ivers == 0 ? 1 : nelems;
  return 32 + 4 * numr * (uint64_t)dim + (uint64_t)fbytes + 8 * nelems;
}

// values per field from the expansion orders (io/gio.ipp:416-429)
bool count_data(int ivers, int dim, uint64_t nelems, const int *porder, uint64_t *nd) {
  uint64_t total = 0;
  const uint64_t numr = ivers == 0 ? 1 : nelems;
  for (uint64_t r = 0; r < numr; r++) {
    uint64_t nt = 1;
    for (int d = 0; d < dim; d++) {
      if (porder[r * dim + d] < 0) return false;
      nt *= (uint64_t)porder[r * dim + d] + 1;
    }
    total += nt;
  }
  *nd = ivers == 0 ? total * nelems : total;
  return true;
}

template <typename V>
void put(std::vector<unsigned char> &b, V v) {
  const size_t o = b.size();
  b.resize(o + sizeof(V));
  memcpy(b.data() + o, &v, sizeof(V));
}

struct File {
  FILE *fp = nullptr;
  ~File() {
    if (fp) fclose(fp);
  }
};

// Two pinned staging buffers and one event each, released on scope exit.
struct Staging {
  void *buf[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  cudaError_t init(size_t bytes) {
    for (int i = 0; i < 2; i++) {
      cudaError_t e = cudaHostAlloc(&buf[i], bytes, cudaHostAllocDefault);
      if (e != cudaSuccess) return e;
      e = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  ~Staging() {
    for (int i = 0; i < 2; i++) {
      if (ev[i]) cudaEventSynchronize(ev[i]), cudaEventDestroy(ev[i]);
      if (buf[i]) cudaFreeHost(buf[i]);
    }
  }
};

int fbytes_of(int dtype) { return dtype == GF_F64 ? 8 : dtype == GF_F32 ? 4 : 0; }

int check_header(gf_context *ctx, const gf_gio_header *h, const int *porder, uint64_t *nd) {
  GF_REQUIRE(ctx, h->dim >= 1 && h->dim <= 3, "GIO dim %d out of range", h->dim);
  GF_REQUIRE(ctx, h->nelems > 0, "GIO header with no elements");
  GF_REQUIRE(ctx, h->gtype >= 0 && h->gtype <= 2, "GIO gtype %d is not a GElemType", h->gtype);
  GF_REQUIRE(ctx, porder != nullptr, "porder missing");
  GF_REQUIRE(ctx, count_data(h->ivers, h->dim, h->nelems, porder, nd), "negative expansion order");
  return GF_OK;
}

// The header as bytes (io/gio.ipp:459-503 field order).
std::vector<unsigned char> header_image(const gf_gio_header *h, const int *porder,
                                        const uint64_t *elemids, int fb) {
  std::vector<unsigned char> hb;
  const uint64_t numr = h->ivers == 0 ? 1 : h->nelems;
  hb.reserve(header_bytes(h->ivers, h->dim, h->nelems, fb));
  put<int32_t>(hb, h->ivers);
  put<int32_t>(hb, h->dim);
  put<uint64_t>(hb, h->nelems);
  for (uint64_t i = 0; i < numr * (uint64_t)h->dim; i++) put<int32_t>(hb, porder[i]);
  put<int32_t>(hb, h->gtype);
  put<uint64_t>(hb, h->cycle);
  if (fb == 8) put<double>(hb, h->time);
  else put<float>(hb, (float)h->time);
  put<int32_t>(hb, h->multivar);
  for (uint64_t e = 0; e < h->nelems; e++) put<uint64_t>(hb, elemids ? elemids[e] : 0);
  return hb;
}

}  // namespace

extern "C" int64_t gf_gio_header_bytes(int ivers, int dim, uint64_t nelems, int dtype) {
  const int fb = fbytes_of(dtype);
  if (!fb || dim < 1 || dim > 3) return GF_ERR_ARG;
  return (int64_t)header_bytes(ivers, dim, nelems, fb);
}

extern "C" int gf_gio_write_header(gf_ctx_t ctx, const char *path, const gf_gio_header *h,
                                   const int *porder, const uint64_t *elemids, int dtype) {
  GF_REQUIRE(ctx, path && h, "bad arguments");
  const int fb = fbytes_of(dtype);
  GF_REQUIRE(ctx, fb, "unknown dtype %d", dtype);
  uint64_t nd = 0;
  int rc = check_header(ctx, h, porder, &nd);
  if (rc) return rc;
  const std::vector<unsigned char> hb = header_image(h, porder, elemids, fb);
  File f;
  f.fp = fopen(path, "wb");
  if (!f.fp) return gf_fail(ctx, GF_ERR_IO, "cannot open %s for writing", path);
  if (fwrite(hb.data(), 1, hb.size(), f.fp) != hb.size())
    return gf_fail(ctx, GF_ERR_IO, "short header write to %s", path);
  const int e = fclose(f.fp);
  f.fp = nullptr;
  return e == 0 ? GF_OK : gf_fail(ctx, GF_ERR_IO, "closing %s failed", path);
}

extern "C" int gf_gio_write_data(gf_ctx_t ctx, const char *path, int dtype, const void *u,
                                 uint64_t n, uint64_t offset) {
  if (!ctx) return GF_ERR_ARG;
  GF_REQUIRE(ctx, path && (u || n == 0), "bad arguments");
  const int fb = fbytes_of(dtype);
  GF_REQUIRE(ctx, fb, "unknown dtype %d", dtype);
  GF_CUDA(ctx, cudaSetDevice(ctx->device));
  File f;
  f.fp = fopen(path, "r+b");
  if (!f.fp || fseek(f.fp, (long)offset, SEEK_SET) != 0)
    return gf_fail(ctx, GF_ERR_IO, "cannot open %s at byte %llu for writing", path,
                   (unsigned long long)offset);
  const size_t total = (size_t)n * fb;
  if (total) {
    const size_t chunk = total < kChunk ? total : kChunk;
    Staging s;
    GF_CUDA(ctx, s.init(chunk));
    const unsigned char *src = (const unsigned char *)u;
    const size_t nchunks = (total + chunk - 1) / chunk;
    auto issue = [&](size_t k) -> cudaError_t {
      const size_t off = k * chunk, len = total - off < chunk ? total - off : chunk;
      cudaError_t e = cudaMemcpyAsync(s.buf[k & 1], src + off, len, cudaMemcpyDeviceToHost,
                                      ctx->stream);
      return e == cudaSuccess ? cudaEventRecord(s.ev[k & 1], ctx->stream) : e;
    };
    GF_CUDA(ctx, issue(0));
    for (size_t k = 0; k < nchunks; k++) {
      GF_CUDA(ctx, cudaEventSynchronize(s.ev[k & 1]));
      if (k + 1 < nchunks) GF_CUDA(ctx, issue(k + 1));
      const size_t off = k * chunk, len = total - off < chunk ? total - off : chunk;
      if (fwrite(s.buf[k & 1], 1, len, f.fp) != len)
        return gf_fail(ctx, GF_ERR_IO, "short data write to %s", path);
    }
  }
  const int e = fclose(f.fp);
  f.fp = nullptr;
  return e == 0 ? GF_OK : gf_fail(ctx, GF_ERR_IO, "closing %s failed", path);
}

extern "C" int gf_gio_write(gf_ctx_t ctx, const char *path, const gf_gio_header *h,
                            const int *porder, const uint64_t *elemids, int dtype, const void *u,
                            uint64_t n) {
  if (!ctx) return GF_ERR_ARG;
  GF_REQUIRE(ctx, path && h && (u || n == 0), "bad arguments");
  const int fb = fbytes_of(dtype);
  GF_REQUIRE(ctx, fb, "unknown dtype %d", dtype);
  uint64_t nd = 0;
  int rc = check_header(ctx, h, porder, &nd);
  if (rc) return rc;
  GF_REQUIRE(ctx, nd == n, "field has %llu values, the header's orders give %llu",
             (unsigned long long)n, (unsigned long long)nd);
  rc = gf_gio_write_header(ctx, path, h, porder, elemids, dtype);
  if (rc) return rc;
  return gf_gio_write_data(ctx, path, dtype, u, n, header_bytes(h->ivers, h->dim, h->nelems, fb));
}

extern "C" int gf_gio_read_header(gf_ctx_t ctx, const char *path, int dtype, gf_gio_header *h,
                                  int *porder, int64_t porder_cap, uint64_t *elemids,
                                  int64_t elemids_cap) {
  // ctx may be NULL here: the header is host data, errors then go to stderr
  GF_REQUIRE(ctx, path && h, "bad arguments");
  File f;
  f.fp = fopen(path, "rb");
  if (!f.fp) return gf_fail(ctx, GF_ERR_IO, "cannot open %s", path);
  if (fseek(f.fp, 0, SEEK_END) != 0) return gf_fail(ctx, GF_ERR_IO, "cannot seek %s", path);
  const long fsize = ftell(f.fp);
  rewind(f.fp);
  int32_t ivers = 0, dim = 0;
  uint64_t nelems = 0;
  if (fread(&ivers, 4, 1, f.fp) != 1 || fread(&dim, 4, 1, f.fp) != 1 ||
      fread(&nelems, 8, 1, f.fp) != 1)
    return gf_fail(ctx, GF_ERR_IO, "%s: truncated GIO header", path);
  if (dim < 1 || dim > 3 || nelems == 0 || nelems > (uint64_t)fsize)
    return gf_fail(ctx, GF_ERR_IO, "%s: not a GIO file (dim %d, nelems %llu)", path, dim,
                   (unsigned long long)nelems);
  const uint64_t numr = ivers == 0 ? 1 : nelems;
  std::vector<int32_t> po(numr * dim);
  if (fread(po.data(), 4, po.size(), f.fp) != po.size())
    return gf_fail(ctx, GF_ERR_IO, "%s: truncated GIO header", path);
  uint64_t nd = 0;
  if (!count_data(ivers, dim, nelems, po.data(), &nd))
    return gf_fail(ctx, GF_ERR_IO, "%s: negative expansion order", path);
  // The file does not record Ftype.  With it the file holds the header and
  // k >= 1 fields of nd values (k > 1: a multivar collective file); a wrong
  // Ftype breaks that unless nd == 1.  dtype -1 takes the size that fits.
  auto fits = [&](int cand) {
    const uint64_t hb = header_bytes(ivers, dim, nelems, cand), fld = nd * (uint64_t)cand;
    return (uint64_t)fsize >= hb + fld && ((uint64_t)fsize - hb) % fld == 0;
  };
  int fb = fbytes_of(dtype);
  if (dtype == -1) {
    for (int cand : {8, 4})
      if (!fb && fits(cand)) fb = cand;
  }
  if (!fb)
    return gf_fail(ctx, dtype == -1 ? GF_ERR_IO : GF_ERR_ARG,
                   "%s: cannot determine the float size (dtype %d, %ld bytes)", path, dtype, fsize);
  if (!fits(fb))
    return gf_fail(ctx, GF_ERR_IO, "%s: %ld bytes do not hold a header and whole fields of %d-byte values",
                   path, fsize, fb);
  int32_t gtype = 0, imulti = 0;
  uint64_t cycle = 0;
  double time = 0.0;
  float time32 = 0.0f;
  bool ok = fread(&gtype, 4, 1, f.fp) == 1 && fread(&cycle, 8, 1, f.fp) == 1;
  ok = ok && (fb == 8 ? fread(&time, 8, 1, f.fp) == 1 : fread(&time32, 4, 1, f.fp) == 1);
  ok = ok && fread(&imulti, 4, 1, f.fp) == 1;
  if (!ok) return gf_fail(ctx, GF_ERR_IO, "%s: truncated GIO header", path);
  if (fb == 4) time = time32;
  if (elemids) {
    GF_REQUIRE(ctx, elemids_cap >= (int64_t)nelems, "elemids needs %llu entries",
               (unsigned long long)nelems);
    if (fread(elemids, 8, nelems, f.fp) != nelems)
      return gf_fail(ctx, GF_ERR_IO, "%s: truncated element keys", path);
  }
  if (porder) {
    GF_REQUIRE(ctx, porder_cap >= (int64_t)po.size(), "porder needs %llu entries",
               (unsigned long long)po.size());
    memcpy(porder, po.data(), po.size() * 4);
  }
  h->ivers = ivers;
  h->dim = dim;
  h->nelems = nelems;
  h->gtype = gtype;
  h->cycle = cycle;
  h->time = time;
  h->multivar = imulti;
  h->float_bytes = fb;
  h->header_bytes = header_bytes(ivers, dim, nelems, fb);
  h->ndata = nd;
  h->porder_rows = (int64_t)numr;
  return GF_OK;
}

extern "C" int gf_gio_read_data(gf_ctx_t ctx, const char *path, int dtype, void *u, uint64_t n,
                                uint64_t offset) {
  if (!ctx) return GF_ERR_ARG;
  GF_REQUIRE(ctx, path && (u || n == 0), "bad arguments");
  const int fb = fbytes_of(dtype);
  GF_REQUIRE(ctx, fb, "unknown dtype %d", dtype);
  GF_CUDA(ctx, cudaSetDevice(ctx->device));
  File f;
  f.fp = fopen(path, "rb");
  if (!f.fp || fseek(f.fp, (long)offset, SEEK_SET) != 0)
    return gf_fail(ctx, GF_ERR_IO, "cannot open %s at byte %llu", path,
                   (unsigned long long)offset);
  const size_t total = (size_t)n * fb;
  if (total) {
    const size_t chunk = total < kChunk ? total : kChunk;
    Staging s;
    GF_CUDA(ctx, s.init(chunk));
    unsigned char *dst = (unsigned char *)u;
    const size_t nchunks = (total + chunk - 1) / chunk;
    for (size_t k = 0; k < nchunks; k++) {
      const size_t off = k * chunk, len = total - off < chunk ? total - off : chunk;
      // the copy issued from this buffer two chunks ago must be done
      if (k >= 2) GF_CUDA(ctx, cudaEventSynchronize(s.ev[k & 1]));
      if (fread(s.buf[k & 1], 1, len, f.fp) != len) {
        cudaStreamSynchronize(ctx->stream);
        return gf_fail(ctx, GF_ERR_IO, "%s: truncated field data", path);
      }
      GF_CUDA(ctx, cudaMemcpyAsync(dst + off, s.buf[k & 1], len, cudaMemcpyHostToDevice,
                                   ctx->stream));
      GF_CUDA(ctx, cudaEventRecord(s.ev[k & 1], ctx->stream));
    }
    GF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return GF_OK;
}

extern "C" int gf_gio_read(gf_ctx_t ctx, const char *path, int dtype, void *u, uint64_t n,
                           gf_gio_header *hout) {
  if (!ctx) return GF_ERR_ARG;
  GF_REQUIRE(ctx, path && (u || n == 0), "bad arguments");
  gf_gio_header h;
  int rc = gf_gio_read_header(ctx, path, dtype, &h, nullptr, 0, nullptr, 0);
  if (rc) return rc;
  GF_REQUIRE(ctx, h.ndata == n, "%s holds %llu values, the field has %llu", path,
             (unsigned long long)h.ndata, (unsigned long long)n);
  rc = gf_gio_read_data(ctx, path, dtype, u, n, h.header_bytes);
  if (rc) return rc;
  if (hout) *hout = h;
  return GF_OK;
}
