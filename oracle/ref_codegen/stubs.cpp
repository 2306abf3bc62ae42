// No-op implementations of the OpenCL and libtiff entry points declared by the
// stand-in headers in stub/ -- TEST INFRASTRUCTURE ONLY.
//
// They let the reference's runtime (its DAG, simplifier, fusion compiler and
// OpenCL kernel generators, compiled from the reference's own sources) run on
// a machine without an OpenCL platform: one fake GPU device is reported, every
// object handle is a distinct dummy, builds and launches succeed without doing
// anything, and device reads leave host memory untouched. The reference prints
// each kernel it generates (runtime/skeleton/*Skeleton.cpp versionCode), which
// is what oracle/ref_codegen/dump_kernels.py collects; the computed rasters are
// meaningless and never used.
#include "CL/cl.h"
#include "tiffio.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

namespace {
std::mutex mtx;
uintptr_t next_handle = 0x1000;
template <class T> T handle() {
  std::lock_guard<std::mutex> lk(mtx);
  next_handle += 0x10;
  return reinterpret_cast<T>(next_handle);
}
void put_str(void *dst, size_t size, const char *s, size_t *ret) {
  const size_t n = std::strlen(s) + 1;
  if (dst && size) {
    std::memset(dst, 0, size);
    std::memcpy(dst, s, n < size ? n : size - 1);
  }
  if (ret) *ret = n;
}
template <class T> void put_val(void *dst, size_t size, T v, size_t *ret) {
  if (dst && size) {
    std::memset(dst, 0, size);
    std::memcpy(dst, &v, sizeof(T) < size ? sizeof(T) : size);
  }
  if (ret) *ret = sizeof(T);
}
}  // namespace

extern "C" {

cl_int clGetPlatformIDs(cl_uint n, cl_platform_id *ids, cl_uint *num) {
  if (ids && n) ids[0] = reinterpret_cast<cl_platform_id>(0x100);
  if (num) *num = 1;
  return CL_SUCCESS;
}
cl_int clGetPlatformInfo(cl_platform_id, cl_platform_info, size_t size, void *v, size_t *ret) {
  put_str(v, size, "stub OpenCL platform", ret);
  return CL_SUCCESS;
}
cl_int clGetDeviceIDs(cl_platform_id, cl_device_type, cl_uint n, cl_device_id *ids, cl_uint *num) {
  if (ids && n) ids[0] = reinterpret_cast<cl_device_id>(0x200);
  if (num) *num = 1;
  return CL_SUCCESS;
}
cl_int clGetDeviceInfo(cl_device_id, cl_device_info p, size_t size, void *v, size_t *ret) {
  if (p == CL_DEVICE_TYPE) put_val<cl_device_type>(v, size, CL_DEVICE_TYPE_GPU, ret);
  else if (p == CL_DEVICE_NAME || p == CL_DEVICE_VENDOR || p == CL_DEVICE_VERSION || p == CL_DEVICE_PROFILE)
    put_str(v, size, "stub", ret);
  else if (p == CL_DEVICE_EXTENSIONS) put_str(v, size, "cl_khr_fp64 cl_khr_int64_base_atomics", ret);
  else if (p == CL_DEVICE_GLOBAL_MEM_SIZE) put_val<cl_ulong>(v, size, (cl_ulong)16 << 30, ret);
  else if (p == CL_DEVICE_MAX_MEM_ALLOC_SIZE) put_val<cl_ulong>(v, size, (cl_ulong)4 << 30, ret);
  else if (p == CL_DEVICE_LOCAL_MEM_SIZE) put_val<cl_ulong>(v, size, (cl_ulong)48 << 10, ret);
  else if (p == CL_DEVICE_MAX_COMPUTE_UNITS) put_val<cl_uint>(v, size, 16, ret);
  else if (p == CL_DEVICE_MAX_WORK_GROUP_SIZE) put_val<size_t>(v, size, 1024, ret);
  else if (p == CL_DEVICE_AVAILABLE || p == CL_DEVICE_COMPILER_AVAILABLE) put_val<cl_bool>(v, size, CL_TRUE, ret);
  else put_val<cl_ulong>(v, size, 0, ret);
  return CL_SUCCESS;
}
cl_int clCreateSubDevices(cl_device_id, const cl_device_partition_property *, cl_uint n, cl_device_id *ids, cl_uint *num) {
  if (ids && n) ids[0] = handle<cl_device_id>();
  if (num) *num = 1;
  return CL_SUCCESS;
}
cl_context clCreateContext(const cl_context_properties *, cl_uint, const cl_device_id *,
                           void (*)(const char *, const void *, size_t, void *), void *, cl_int *err) {
  if (err) *err = CL_SUCCESS;
  return handle<cl_context>();
}
cl_int clReleaseContext(cl_context) { return CL_SUCCESS; }
cl_command_queue clCreateCommandQueue(cl_context, cl_device_id, cl_command_queue_properties, cl_int *err) {
  if (err) *err = CL_SUCCESS;
  return handle<cl_command_queue>();
}
cl_int clReleaseCommandQueue(cl_command_queue) { return CL_SUCCESS; }
cl_mem clCreateBuffer(cl_context, cl_mem_flags, size_t, void *, cl_int *err) {
  if (err) *err = CL_SUCCESS;
  return handle<cl_mem>();
}
cl_mem clCreateSubBuffer(cl_mem, cl_mem_flags, cl_buffer_create_type, const void *, cl_int *err) {
  if (err) *err = CL_SUCCESS;
  return handle<cl_mem>();
}
cl_int clReleaseMemObject(cl_mem) { return CL_SUCCESS; }
cl_program clCreateProgramWithSource(cl_context, cl_uint, const char **, const size_t *, cl_int *err) {
  if (err) *err = CL_SUCCESS;
  return handle<cl_program>();
}
cl_int clBuildProgram(cl_program, cl_uint, const cl_device_id *, const char *, void (*)(cl_program, void *), void *) {
  return CL_SUCCESS;
}
cl_int clGetProgramBuildInfo(cl_program, cl_device_id, cl_program_build_info, size_t size, void *v, size_t *ret) {
  put_str(v, size, "", ret);
  return CL_SUCCESS;
}
cl_int clReleaseProgram(cl_program) { return CL_SUCCESS; }
// With MAP_STUB_LOG_ARGS set, kernel creation and by-value kernel arguments are
// logged to stderr ("KERNEL <handle> <name>", "ARG <handle> <index> <hex bytes>"),
// which shows the scalar values the reference passes to its kernels.
static bool log_args() {
  static const bool on = std::getenv("MAP_STUB_LOG_ARGS") != nullptr;
  return on;
}
cl_kernel clCreateKernel(cl_program, const char *name, cl_int *err) {
  if (err) *err = CL_SUCCESS;
  cl_kernel k = handle<cl_kernel>();
  if (log_args()) {
    std::lock_guard<std::mutex> lk(mtx);
    std::fprintf(stderr, "KERNEL %p %s\n", (void *)k, name);
  }
  return k;
}
cl_int clReleaseKernel(cl_kernel) { return CL_SUCCESS; }
cl_int clSetKernelArg(cl_kernel k, cl_uint idx, size_t size, const void *v) {
  if (log_args() && v && size <= 8) {
    std::lock_guard<std::mutex> lk(mtx);
    std::fprintf(stderr, "ARG %p %u ", (void *)k, idx);
    for (size_t i = 0; i < size; i++) std::fprintf(stderr, "%02x", ((const unsigned char *)v)[i]);
    std::fprintf(stderr, "\n");
  }
  return CL_SUCCESS;
}
cl_int clEnqueueNDRangeKernel(cl_command_queue, cl_kernel, cl_uint, const size_t *, const size_t *, const size_t *, cl_uint,
                              const cl_event *, cl_event *) {
  return CL_SUCCESS;
}
cl_int clEnqueueReadBuffer(cl_command_queue, cl_mem, cl_bool, size_t, size_t, void *, cl_uint, const cl_event *, cl_event *) {
  return CL_SUCCESS;
}
cl_int clEnqueueWriteBuffer(cl_command_queue, cl_mem, cl_bool, size_t, size_t, const void *, cl_uint, const cl_event *,
                            cl_event *) {
  return CL_SUCCESS;
}
cl_int clEnqueueCopyBuffer(cl_command_queue, cl_mem, cl_mem, size_t, size_t, size_t, cl_uint, const cl_event *, cl_event *) {
  return CL_SUCCESS;
}
cl_int clEnqueueFillBuffer(cl_command_queue, cl_mem, const void *, size_t, size_t, size_t, cl_uint, const cl_event *,
                           cl_event *) {
  return CL_SUCCESS;
}
void *clEnqueueMapBuffer(cl_command_queue, cl_mem, cl_bool, cl_map_flags, size_t, size_t size, cl_uint, const cl_event *,
                         cl_event *, cl_int *err) {
  if (err) *err = CL_SUCCESS;
  return std::calloc(size ? size : 1, 1);   // host staging the reference reads and writes; kept until exit
}
cl_int clEnqueueUnmapMemObject(cl_command_queue, cl_mem, void *, cl_uint, const cl_event *, cl_event *) { return CL_SUCCESS; }
cl_event clCreateUserEvent(cl_context, cl_int *err) {
  if (err) *err = CL_SUCCESS;
  return handle<cl_event>();
}
cl_int clReleaseEvent(cl_event) { return CL_SUCCESS; }
cl_int clFinish(cl_command_queue) { return CL_SUCCESS; }

// ---- libtiff: every file open fails (the kernel dump reads and writes .bin files only)
TIFF *TIFFOpen(const char *, const char *) { return nullptr; }
void TIFFClose(TIFF *) {}
int TIFFGetField(TIFF *, uint32_t, ...) { return 0; }
int TIFFSetField(TIFF *, uint32_t, ...) { return 0; }
int TIFFMergeFieldInfo(TIFF *, const TIFFFieldInfo *, uint32_t) { return 0; }
TIFFExtendProc TIFFSetTagExtender(TIFFExtendProc p) { return p; }
tsize_t TIFFReadTile(TIFF *, void *, uint32_t, uint32_t, uint32_t, uint16_t) { return -1; }
tsize_t TIFFWriteTile(TIFF *, void *, uint32_t, uint32_t, uint32_t, uint16_t) { return -1; }

}  // extern "C"
