// `.bin` raster reader/writer (format described in binfile.hpp).
#include "binfile.hpp"
#include "types.hpp"

#include <cerrno>
#include <cstring>
#include <fcntl.h>
#include <unistd.h>

namespace mapb {

namespace {

struct Fd {
  int fd = -1;
  ~Fd() { if (fd >= 0) ::close(fd); }
};

void pread_all(int fd, void *dst, size_t len, size_t off, const std::string &path) {
  size_t done = 0;
  while (done < len) {
    ssize_t r = ::pread(fd, (char *)dst + done, len - done, (off_t)(off + done));
    if (r < 0) throw MapError("read of '" + path + "' failed: " + std::strerror(errno));
    if (r == 0) throw MapError("file '" + path + "' is shorter than its header says");
    done += (size_t)r;
  }
}

void pwrite_all(int fd, const void *src, size_t len, size_t off, const std::string &path) {
  size_t done = 0;
  while (done < len) {
    ssize_t r = ::pwrite(fd, (const char *)src + done, len - done, (off_t)(off + done));
    if (r < 0) throw MapError("write of '" + path + "' failed: " + std::strerror(errno));
    done += (size_t)r;
  }
}

}  // namespace

BinHeader bin_read_header(const std::string &path) {
  Fd f;
  f.fd = ::open(path.c_str(), O_RDONLY);
  if (f.fd < 0) throw MapError("cannot open '" + path + "' for reading: " + std::strerror(errno));
  int32_t w[8] = {0};
  pread_all(f.fd, w, 2 * sizeof(int32_t), 0, path);
  BinHeader h;
  h.dtype = w[0];
  h.numdim = w[1];
  if (h.dtype <= NONE_DATATYPE || h.dtype >= N_DATATYPE) throw MapError("'" + path + "': invalid data type in header");
  if (h.numdim != D2) throw MapError("'" + path + "': only 2-D rasters are supported");
  pread_all(f.fd, w + 2, 5 * sizeof(int32_t), 2 * sizeof(int32_t), path);
  h.ds0 = w[2];
  h.ds1 = w[3];
  h.memorder = w[4];
  h.bs0 = w[5];
  h.bs1 = w[6];
  if (h.ds0 <= 0 || h.ds1 <= 0) throw MapError("'" + path + "': invalid data size in header");
  if (h.memorder != ROW && h.memorder != ROW + BLK) throw MapError("'" + path + "': unsupported memory order");
  if (h.memorder == ROW + BLK && (h.bs0 <= 0 || h.bs1 <= 0)) throw MapError("'" + path + "': invalid block size");
  if (h.memorder == ROW && (h.bs0 <= 0 || h.bs1 <= 0)) { h.bs0 = h.ds0; h.bs1 = h.ds1; }
  return h;
}

void bin_read_dense(const std::string &path, const BinHeader &h, void *dst) {
  Fd f;
  f.fd = ::open(path.c_str(), O_RDONLY);
  if (f.fd < 0) throw MapError("cannot open '" + path + "' for reading: " + std::strerror(errno));
  const size_t es = dt_size(h.dtype);
  char *out = (char *)dst;
  if (h.memorder == ROW) {
    pread_all(f.fd, out, (size_t)h.ds0 * h.ds1 * es, BIN_PAGE, path);
    return;
  }
  const int nb0 = (h.ds0 + h.bs0 - 1) / h.bs0, nb1 = (h.ds1 + h.bs1 - 1) / h.bs1;
  const size_t block_bytes = (size_t)h.bs0 * h.bs1 * es;
  std::vector<char> blk(block_bytes);
  for (int b1 = 0; b1 < nb1; b1++) {
    for (int b0 = 0; b0 < nb0; b0++) {
      size_t off = BIN_PAGE + ((size_t)b1 * nb0 + b0) * block_bytes;
      pread_all(f.fd, blk.data(), block_bytes, off, path);
      const int w = std::min(h.bs0, h.ds0 - b0 * h.bs0), hh = std::min(h.bs1, h.ds1 - b1 * h.bs1);
      for (int y = 0; y < hh; y++)
        std::memcpy(out + (((size_t)b1 * h.bs1 + y) * h.ds0 + (size_t)b0 * h.bs0) * es, blk.data() + (size_t)y * h.bs0 * es,
                    (size_t)w * es);
    }
  }
}

void bin_write_dense(const std::string &path, const BinHeader &h, const void *src) {
  Fd f;
  f.fd = ::open(path.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
  if (f.fd < 0) throw MapError("cannot open '" + path + "' for writing: " + std::strerror(errno));
  std::vector<char> page(BIN_PAGE, 0);
  int32_t w[7] = {h.dtype, h.numdim, h.ds0, h.ds1, h.memorder, h.bs0, h.bs1};
  std::memcpy(page.data(), w, sizeof(w));
  pwrite_all(f.fd, page.data(), BIN_PAGE, 0, path);
  const size_t es = dt_size(h.dtype);
  const char *in = (const char *)src;
  if (h.memorder == ROW) {
    pwrite_all(f.fd, in, (size_t)h.ds0 * h.ds1 * es, BIN_PAGE, path);
    return;
  }
  const int nb0 = (h.ds0 + h.bs0 - 1) / h.bs0, nb1 = (h.ds1 + h.bs1 - 1) / h.bs1;
  const size_t block_bytes = (size_t)h.bs0 * h.bs1 * es;
  std::vector<char> blk(block_bytes);
  for (int b1 = 0; b1 < nb1; b1++) {
    for (int b0 = 0; b0 < nb0; b0++) {
      std::memset(blk.data(), 0, block_bytes);
      const int bw = std::min(h.bs0, h.ds0 - b0 * h.bs0), bh = std::min(h.bs1, h.ds1 - b1 * h.bs1);
      for (int y = 0; y < bh; y++)
        std::memcpy(blk.data() + (size_t)y * h.bs0 * es, in + (((size_t)b1 * h.bs1 + y) * h.ds0 + (size_t)b0 * h.bs0) * es,
                    (size_t)bw * es);
      pwrite_all(f.fd, blk.data(), block_bytes, BIN_PAGE + ((size_t)b1 * nb0 + b0) * block_bytes, path);
    }
  }
}

}  // namespace mapb
