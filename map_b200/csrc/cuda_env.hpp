// Thin CUDA layer replacing the reference's OpenCL wrapper (cle/OclEnv.hpp:50-453):
// device selection, NVRTC compilation of generated kernels for sm_100a with an
// in-memory and on-disk cubin cache, module loading and kernel launch through
// driver entry points obtained from the runtime (no link-time libcuda
// dependency, so the library also loads on machines without a GPU driver).
#pragma once

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

struct CUfunc_st;
struct CUmod_st;
struct CUstream_st;

namespace mapb {

struct CompiledModule {
  CUmod_st *module = nullptr;
  std::vector<unsigned char> cubin;
};

struct KernelHandle {
  CUfunc_st *fn = nullptr;
  size_t max_dyn_smem = 0;
};

class CudaEnv {
 public:
  static CudaEnv &get();

  // Compiles `source` (which includes "map_common.cuh") for sm_100a; returns the cubin.
  // Works without a GPU. Results are cached in memory and on disk.
  const std::vector<unsigned char> &compile(const std::string &source);
  std::string compile_log() const { return last_log_; }

  // Device side (require a GPU)
  void ensure_device();
  bool device_ready() const { return device_ready_; }
  KernelHandle kernel(const std::string &source, const std::string &name, size_t dyn_smem);
  void launch(const KernelHandle &k, int grid, int block, size_t smem, CUstream_st *stream, void *args, size_t args_size);
  void launch_cluster(const KernelHandle &k, int grid, int block, int cluster, size_t smem, CUstream_st *stream, void *args);
  // a grid of gx x gy CTAs (the Local / Focal kernels: the region's tiles)
  void launch_2d(const KernelHandle &k, int gx, int gy, int block, size_t smem, CUstream_st *stream, void *args);
  // programmatic dependent launch of gx x gy CTAs (the kernel waits with griddepcontrol.wait)
  void launch_pdl(const KernelHandle &k, int gx, int gy, int block, size_t smem, CUstream_st *stream, void *args);
  int occupancy(const KernelHandle &k, int block, size_t smem);   // resident CTAs per SM
  // Writes `value` (elem_size bytes: 1, 2 or 4) into every element of a width x
  // height 2-D array; false (nothing done) for other element sizes.
  bool fill_2d(void *dst, size_t pitch, const void *value, int elem_size, size_t width, size_t height,
               CUstream_st *stream);
  void encode_tma_2d(void *desc128, int dtype, const void *base, uint64_t width, uint64_t height, uint64_t pitch_bytes,
                     uint32_t box_w, uint32_t box_h);
  CUstream_st *stream() const { return stream_; }
  int sm_count() const { return sm_count_; }
  int device() const { return device_; }
  std::string device_name() const { return device_name_; }
  uint32_t *err_word() const { return err_word_; }
  int launches() const { return launches_; }
  void count_launch() { launches_++; }
  void set_device(int d);

  static std::string cache_dir();

 private:
  CudaEnv() = default;
  std::string last_log_;
  bool device_ready_ = false;
  int device_ = 0;
  int sm_count_ = 0;
  std::string device_name_;
  CUstream_st *stream_ = nullptr;
  uint32_t *err_word_ = nullptr;
  std::atomic<int> launches_{0};
};

// CUDA runtime error check helper
void cuda_check(int err, const char *what);

}  // namespace mapb
