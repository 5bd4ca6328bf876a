// ANA ".f0" files: the on-disk format of SNAPI's observed Stokes cubes, model cubes and results.
//
// Host code (no kernels).  Follows the reference's reader and writer:
//   header check and decoding    cmlib/ana_read.cc:17-58 (ck_synch_hd), 74-111 (ana_fzread)
//   uncompressed element data    cmlib/ana_read.cc:151-177
//   writer                       cmlib/ana_write.cc:129-175 (ana_fzwrite)
//   streaming writer             cmlib/ana_write.cc:177-239 (ana_file / ana_file::append)
//
// File layout (little endian, as every ana_fzwrite writes it): nhb header blocks of 512 bytes,
// then the elements with dim[0] varying fastest.  Block 0: int32 synch pattern 0x5555aaaa at 0;
// bytes subf (4; bit 0 compressed, >= 128 big-endian data), source (5), nhb (6), datyp (7),
// ndim (8), file_class (9); int32 cbytes at 10 (the data size in bytes, low 32 bits); int32
// dim[16] at 192; text[256] at 256.  Blocks 1.. carry only more text at 256.
//
// Deviations from the reference, all where it has no defined behaviour: element counts are 64-bit
// (the reference multiplies in int), a truncated file is an error (the reference's read loop never
// ends), ndim outside 1..16 and type codes outside 0..5 are errors (it indexes past its tables),
// a zero nhb counts as one block, and an empty header text writes one block (the reference writes
// none).  Compressed files (anacrunch, integer types only) are refused: every cube on the
// inversion path is float32 or float64, which the reference never compresses.
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <atomic>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include "../../include/snapi_cuda.h"
#include "snapi_f0_internal.h"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

const int kTypeSize[6] = {1, 2, 4, 4, 8, 8};  // ANA_VAR_SZ (cmlib/ana_io.h:11)

uint32_t rd32(const uint8_t *p) { return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24; }
void wr32(uint8_t *p, uint32_t v) {
  p[0] = (uint8_t)v; p[1] = (uint8_t)(v >> 8); p[2] = (uint8_t)(v >> 16); p[3] = (uint8_t)(v >> 24);
}

bool read_full(int fd, void *buf, size_t n, off_t off) {
  uint8_t *b = (uint8_t *)buf;
  while (n) {
    ssize_t r = pread(fd, b, n, off);
    if (r < 0 && errno == EINTR) continue;
    if (r <= 0) return false;
    b += r; n -= (size_t)r; off += r;
  }
  return true;
}

bool write_full(int fd, const void *buf, size_t n, off_t off) {
  const uint8_t *b = (const uint8_t *)buf;
  while (n) {
    ssize_t r = pwrite(fd, b, n, off);
    if (r < 0 && errno == EINTR) continue;
    if (r <= 0) return false;
    b += r; n -= (size_t)r; off += r;
  }
  return true;
}

void bswap_elems(uint8_t *p, int64_t n, int esz) {
  if (esz == 1) return;
  for (int64_t i = 0; i < n; ++i, p += esz)
    for (int a = 0, b = esz - 1; a < b; ++a, --b) { uint8_t t = p[a]; p[a] = p[b]; p[b] = t; }
}

template <typename T>
void convert_from(const uint8_t *src, int type, int64_t n, T *dst) {
  switch (type) {
    case SNAPI_F0_INT8:    for (int64_t i = 0; i < n; ++i) dst[i] = (T)((const int8_t *)src)[i]; break;
    case SNAPI_F0_INT16:   for (int64_t i = 0; i < n; ++i) { int16_t v; memcpy(&v, src + 2 * i, 2); dst[i] = (T)v; } break;
    case SNAPI_F0_INT32:   for (int64_t i = 0; i < n; ++i) { int32_t v; memcpy(&v, src + 4 * i, 4); dst[i] = (T)v; } break;
    case SNAPI_F0_FLOAT32: for (int64_t i = 0; i < n; ++i) { float v; memcpy(&v, src + 4 * i, 4); dst[i] = (T)v; } break;
    case SNAPI_F0_FLOAT64: for (int64_t i = 0; i < n; ++i) { double v; memcpy(&v, src + 8 * i, 8); dst[i] = (T)v; } break;
    case SNAPI_F0_INT64:   for (int64_t i = 0; i < n; ++i) { int64_t v; memcpy(&v, src + 8 * i, 8); dst[i] = (T)v; } break;
  }
}

// The header blocks ana_fzwrite writes (cmlib/ana_write.cc:129-175).
std::vector<uint8_t> make_header(int type, int ndim, const long long *dim, const char *header, uint64_t nbytes) {
  int nhead = 1;
  if (header) {
    size_t len = strlen(header);
    nhead = (int)((len + 254) / 255);
    if (nhead > 15) nhead = 15;
    if (nhead < 1) nhead = 1;
  }
  std::vector<uint8_t> h((size_t)nhead * 512, 0);
  wr32(h.data(), 0x5555aaaau);
  h[4] = 0;                 // subf: uncompressed, little endian
  h[5] = 0;                 // source
  h[6] = (uint8_t)nhead;
  h[7] = (uint8_t)type;
  h[8] = (uint8_t)ndim;
  wr32(h.data() + 10, (uint32_t)nbytes);
  for (int d = 0; d < ndim; ++d) wr32(h.data() + 192 + 4 * d, (uint32_t)(int32_t)dim[d]);
  if (header) {
    const char *p = header;
    for (int i = 0; i < nhead; ++i) {
      size_t len = strlen(p);
      if (len > 255) len = 255;
      memcpy(h.data() + (size_t)i * 512 + 256, p, len);
      p += len;
    }
  }
  return h;
}

int check_dims(int type, int ndim, const long long *dim, int64_t *nelem) {
  if (type < 0 || type > 5) return fail(SNAPI_EINVAL, "f0: type code outside 0..5");
  if (ndim < 1 || ndim > SNAPI_F0_MAX_DIM || !dim) return fail(SNAPI_EINVAL, "f0: ndim outside 1..16");
  int64_t n = 1;
  for (int d = 0; d < ndim; ++d) {
    if (dim[d] < 0 || dim[d] > 0x7fffffffLL) return fail(SNAPI_EINVAL, "f0: dimension outside 0..2^31-1");
    n *= dim[d];
    if (n > (int64_t(1) << 50)) return fail(SNAPI_EINVAL, "f0: too many elements");
  }
  *nelem = n;
  return SNAPI_OK;
}

}  // namespace

namespace snapi_f0 {

int parse(int fd, snapi_f0_info *info) {
  memset(info, 0, sizeof(*info));
  uint8_t b0[512];
  if (!read_full(fd, b0, 512, 0)) return fail(SNAPI_EINVAL, "f0: file shorter than one header block");
  uint32_t synch = rd32(b0);
  // ck_synch_hd: the pattern as the machine reads it; a reversed one flips the data byte order
  const bool syncpat = synch == 0x5555aaaau, revsyncpat = synch == 0xaaaa5555u;
  if (!syncpat && !revsyncpat) return fail(SNAPI_EINVAL, "f0: file does not have the F0 synch pattern");
  info->reversed_synch = revsyncpat ? 1 : 0;
  int nhb = b0[6];
  if (nhb > 15) return fail(SNAPI_EINVAL, "f0: more than 15 header blocks");
  if (nhb < 1) nhb = 1;
  info->nhb = nhb;
  info->type = b0[7];
  info->ndim = b0[8];
  if (info->type > 5) return fail(SNAPI_EINVAL, "f0: unknown data type code");
  if (info->ndim < 1 || info->ndim > SNAPI_F0_MAX_DIM) return fail(SNAPI_EINVAL, "f0: ndim outside 1..16");
  const int subf = b0[4];
  int swap = subf >= 128 ? 1 : 0;              // big-endian data
  if (info->reversed_synch) swap = !swap;       // "file contains strange data" (ana_read.cc:106)
  info->swap = swap;
  info->compressed = subf & 1;
  std::vector<uint8_t> rest((size_t)(nhb - 1) * 512);
  if (nhb > 1 && !read_full(fd, rest.data(), rest.size(), 512))
    return fail(SNAPI_EINVAL, "f0: file shorter than its header blocks");
  std::string text;
  for (int i = 0; i < nhb; ++i) {
    const uint8_t *t = (i == 0 ? b0 : rest.data() + (size_t)(i - 1) * 512) + 256;
    size_t len = strnlen((const char *)t, 256);
    text.append((const char *)t, len);
  }
  if (text.size() >= sizeof(info->header)) text.resize(sizeof(info->header) - 1);
  memcpy(info->header, text.data(), text.size());
  info->header[text.size()] = 0;
  int64_t n = 1;
  for (int d = 0; d < info->ndim; ++d) {
    info->dim[d] = (int32_t)rd32(b0 + 192 + 4 * d);
    if (info->dim[d] < 0) return fail(SNAPI_EINVAL, "f0: negative dimension");
    n *= info->dim[d];
    if (n > (int64_t(1) << 50)) return fail(SNAPI_EINVAL, "f0: too many elements");
  }
  info->nelem = n;
  info->data_offset = (long long)nhb * 512;
  return SNAPI_OK;
}

int type_size(int type) { return (type >= 0 && type <= 5) ? kTypeSize[type] : 0; }

// Elements [first, first + count) of an open, uncompressed file into out (converted to out_type:
// the file's own type, FLOAT32 or FLOAT64), native byte order.  scratch is reused between calls.
int read_range(int fd, const snapi_f0_info &info, long long first, long long count, void *out, int out_type,
               std::vector<uint8_t> &scratch) {
  if (info.compressed) return fail(SNAPI_EINVAL, "f0: compressed (anacrunch) files are not read by this library");
  if (first < 0 || count < 0 || first + count > info.nelem) return fail(SNAPI_EINVAL, "f0: element range outside the file");
  if (out_type != info.type && out_type != SNAPI_F0_FLOAT32 && out_type != SNAPI_F0_FLOAT64)
    return fail(SNAPI_EINVAL, "f0: out_type must be the file's type, FLOAT32 or FLOAT64");
  if (!count) return SNAPI_OK;
  const int esz = kTypeSize[info.type];
  const size_t nb = (size_t)count * esz;
  const off_t off = (off_t)info.data_offset + (off_t)first * esz;
  uint8_t *dst = out_type == info.type ? (uint8_t *)out : nullptr;
  if (!dst) {
    if (scratch.size() < nb) scratch.resize(nb);
    dst = scratch.data();
  }
  if (!read_full(fd, dst, nb, off)) return fail(SNAPI_EINVAL, "f0: unexpected end of file");
  if (info.swap) bswap_elems(dst, count, esz);
  if (out_type == info.type) return SNAPI_OK;
  if (out_type == SNAPI_F0_FLOAT32) convert_from(dst, info.type, count, (float *)out);
  else convert_from(dst, info.type, count, (double *)out);
  return SNAPI_OK;
}

void set_error(const std::string &msg) { g_err = msg; }

}  // namespace snapi_f0

struct snapi_f0_file {
  int fd = -1;
  int64_t nelem = 0;
  int esz = 0;
  int64_t data_offset = 0;
  std::atomic<int64_t> written{0};
  bool io_error = false;
};

extern "C" {

const char *snapi_f0_error(void) { return g_err.c_str(); }

int snapi_f0_stat(const char *path, snapi_f0_info *info) {
  if (!path || !info) return fail(SNAPI_EINVAL, "f0: null argument");
  int fd = open(path, O_RDONLY);
  if (fd < 0) return fail(SNAPI_EINVAL, std::string("f0: cannot open ") + path);
  int st = snapi_f0::parse(fd, info);
  close(fd);
  return st;
}

int snapi_f0_read(const char *path, long long first, long long count, void *out, int out_type) {
  if (!path || (!out && count > 0)) return fail(SNAPI_EINVAL, "f0: null argument");
  int fd = open(path, O_RDONLY);
  if (fd < 0) return fail(SNAPI_EINVAL, std::string("f0: cannot open ") + path);
  snapi_f0_info info;
  int st = snapi_f0::parse(fd, &info);
  std::vector<uint8_t> scratch;
  if (!st) st = snapi_f0::read_range(fd, info, first, count, out, out_type, scratch);
  close(fd);
  return st;
}

snapi_f0_file *snapi_f0_create(const char *path, int type, int ndim, const long long *dim, const char *header,
                               int *status) {
  int64_t n = 0;
  int st = path ? check_dims(type, ndim, dim, &n) : fail(SNAPI_EINVAL, "f0: null path");
  if (st) { if (status) *status = st; return nullptr; }
  int fd = open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
  if (fd < 0) {
    st = fail(SNAPI_EINVAL, std::string("f0: cannot create ") + path);
    if (status) *status = st;
    return nullptr;
  }
  const uint64_t nbytes = (uint64_t)n * kTypeSize[type];
  std::vector<uint8_t> h = make_header(type, ndim, dim, header, nbytes);
  if (!write_full(fd, h.data(), h.size(), 0)) {
    close(fd);
    st = fail(SNAPI_EINVAL, std::string("f0: write failed on ") + path);
    if (status) *status = st;
    return nullptr;
  }
  snapi_f0_file *f = new snapi_f0_file;
  f->fd = fd;
  f->nelem = n;
  f->esz = kTypeSize[type];
  f->data_offset = (int64_t)h.size();
  if (status) *status = SNAPI_OK;
  return f;
}

int snapi_f0_write_at(snapi_f0_file *f, long long first, long long count, const void *data) {
  if (!f || (!data && count > 0)) return fail(SNAPI_EINVAL, "f0: null argument");
  if (first < 0 || count < 0 || first + count > f->nelem) return fail(SNAPI_EINVAL, "f0: element range outside the file");
  if (!count) return SNAPI_OK;
  if (!write_full(f->fd, data, (size_t)count * f->esz, (off_t)(f->data_offset + first * f->esz))) {
    f->io_error = true;
    return fail(SNAPI_EINVAL, "f0: write failed");
  }
  f->written += count;
  return SNAPI_OK;
}

int snapi_f0_close(snapi_f0_file *f) {
  if (!f) return fail(SNAPI_EINVAL, "f0: null file");
  int st = SNAPI_OK;
  if (f->io_error) st = fail(SNAPI_EINVAL, "f0: a write failed");
  else if (f->written.load() != f->nelem)  // ana_file::~ana_file (ana_write.cc:220-224)
    st = fail(SNAPI_EINVAL, "f0: closed with " + std::to_string(f->written.load()) + " of " +
                                std::to_string(f->nelem) + " elements written");
  if (close(f->fd) != 0 && !st) st = fail(SNAPI_EINVAL, "f0: close failed");
  delete f;
  return st;
}

int snapi_f0_write(const char *path, const void *data, int type, int ndim, const long long *dim, const char *header) {
  int st = SNAPI_OK;
  snapi_f0_file *f = snapi_f0_create(path, type, ndim, dim, header, &st);
  if (!f) return st;
  st = snapi_f0_write_at(f, 0, f->nelem, data);
  int st2 = snapi_f0_close(f);
  return st ? st : st2;
}

}  // extern "C"
