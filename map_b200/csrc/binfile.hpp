// The reference's `.bin` raster file format (file/binary.cpp:221-404):
// a 4096-byte header page holding, as native int32 values,
//   data_type, num_dim, data_size[num], mem_order, block_size[num]
// followed by the cells. For mem_order ROW+BLK the cells are stored block by
// block (blocks in row-major block order, file/binary.cpp:344-385), each block a
// full block_size[0] x block_size[1] row-major array, edge blocks padded.
// For mem_order ROW the cells are one dense row-major array.
#pragma once

#include <string>
#include <vector>

namespace mapb {

struct BinHeader {
  int dtype = 0;
  int numdim = 0;
  int ds0 = 0, ds1 = 0;
  int memorder = 0;
  int bs0 = 0, bs1 = 0;
};

constexpr size_t BIN_PAGE = 4096;

BinHeader bin_read_header(const std::string &path);
// Reads the whole raster into a dense row-major buffer (ds0 x ds1 cells).
void bin_read_dense(const std::string &path, const BinHeader &h, void *dst);
// Writes a dense row-major buffer as a `.bin` file with the given layout.
void bin_write_dense(const std::string &path, const BinHeader &h, const void *src);

}  // namespace mapb
