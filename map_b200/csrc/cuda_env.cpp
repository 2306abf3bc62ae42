// CUDA device layer: NVRTC compilation with a cubin cache, module loading and
// launches through driver entry points (see cuda_env.hpp).
#include "cuda_env.hpp"
#include "types.hpp"

#include <cuda.h>
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvrtc.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <unordered_map>

namespace mapb {

namespace {

#include "skeleton_embed.inc"   // kSkeletonHeaders[] = {name, source}

typedef CUresult (*PFN_ModuleLoadData)(CUmodule *, const void *);
typedef CUresult (*PFN_ModuleGetFunction)(CUfunction *, CUmodule, const char *);
typedef CUresult (*PFN_LaunchKernel)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, CUstream,
                                     void **, void **);
typedef CUresult (*PFN_FuncSetAttribute)(CUfunction, CUfunction_attribute, int);
typedef CUresult (*PFN_LaunchKernelEx)(const CUlaunchConfig *, CUfunction, void **, void **);
typedef CUresult (*PFN_TensorMapEncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                             const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                             CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
typedef CUresult (*PFN_GetErrorString)(CUresult, const char **);
typedef CUresult (*PFN_Occupancy)(int *, CUfunction, int, size_t);
typedef CUresult (*PFN_MemsetD2D8)(CUdeviceptr, size_t, unsigned char, size_t, size_t, CUstream);
typedef CUresult (*PFN_MemsetD2D16)(CUdeviceptr, size_t, unsigned short, size_t, size_t, CUstream);
typedef CUresult (*PFN_MemsetD2D32)(CUdeviceptr, size_t, unsigned int, size_t, size_t, CUstream);

struct Driver {
  PFN_ModuleLoadData moduleLoadData = nullptr;
  PFN_ModuleGetFunction moduleGetFunction = nullptr;
  PFN_LaunchKernel launchKernel = nullptr;
  PFN_LaunchKernelEx launchKernelEx = nullptr;
  PFN_FuncSetAttribute funcSetAttribute = nullptr;
  PFN_TensorMapEncodeTiled tensorMapEncodeTiled = nullptr;
  PFN_GetErrorString getErrorString = nullptr;
  PFN_Occupancy occupancy = nullptr;
  PFN_MemsetD2D8 memsetD2D8 = nullptr;
  PFN_MemsetD2D16 memsetD2D16 = nullptr;
  PFN_MemsetD2D32 memsetD2D32 = nullptr;
};

Driver g_drv;
std::mutex g_mtx;
std::map<std::string, std::vector<unsigned char>> g_cubins;   // key: source hash
std::map<std::string, CUmodule> g_modules;                   // key: source hash
std::map<std::string, KernelHandle> g_kernels;               // key: source hash + name
// Launch-path lookup by kernel name (names carry a hash of their group's
// source) and source length, so a launch does not hash the source again.
struct FastEntry { size_t source_size; KernelHandle h; };
std::unordered_map<std::string, FastEntry> g_fast;

std::string hash_hex(const std::string &s) {
  uint64_t h = 1469598103934665603ull;
  for (unsigned char c : s) { h ^= c; h *= 1099511628211ull; }
  char b[17];
  std::snprintf(b, sizeof b, "%016llx", (unsigned long long)h);
  return b;
}

const char *kNvrtcOpts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "--fmad=false", "-lineinfo", "-DMAPB_NVRTC=1"};

// compile options, NVRTC version and skeleton header hashes (fixed for the process)
const std::string &options_key() {
  static const std::string key = [] {
    std::string k;
    for (const char *o : kNvrtcOpts) k += std::string(o) + " ";
    int maj = 0, min = 0;
    nvrtcVersion(&maj, &min);
    k += std::to_string(maj) + "." + std::to_string(min);
    for (auto &h : kSkeletonHeaders) k += hash_hex(h.source);
    return k;
  }();
  return key;
}

void drv_check(CUresult r, const char *what) {
  if (r == CUDA_SUCCESS) return;
  const char *s = "unknown";
  if (g_drv.getErrorString) g_drv.getErrorString(r, &s);
  throw MapError(std::string(what) + " failed: " + s + " (" + std::to_string((int)r) + ")");
}

template <class F> void load_entry(F &fp, const char *name) {
  void *p = nullptr;
  cudaDriverEntryPointQueryResult q;
  cudaError_t e = cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q);
  if (e != cudaSuccess || p == nullptr || q != cudaDriverEntryPointSuccess)
    throw MapError(std::string("driver entry point ") + name + " unavailable");
  fp = reinterpret_cast<F>(p);
}

}  // namespace

void cuda_check(int err, const char *what) {
  if (err != cudaSuccess)
    throw MapError(std::string(what) + " failed: " + cudaGetErrorString((cudaError_t)err));
}

CudaEnv &CudaEnv::get() {
  static CudaEnv env;
  return env;
}

std::string CudaEnv::cache_dir() {
  if (const char *e = std::getenv("MAP_B200_KCACHE")) return e;
  Dl_info info;
  if (dladdr((void *)&CudaEnv::get, &info) && info.dli_fname) {
    std::string p = info.dli_fname;
    size_t s = p.rfind('/');
    if (s != std::string::npos) return p.substr(0, s) + "/_kcache";
  }
  return "/tmp/map_b200_kcache";
}

const std::vector<unsigned char> &CudaEnv::compile(const std::string &source) {
  const std::string key = hash_hex(source + "\n//" + options_key());
  {
    std::lock_guard<std::mutex> lk(g_mtx);
    auto it = g_cubins.find(key);
    if (it != g_cubins.end()) return it->second;
  }
  // disk cache
  const std::string dir = cache_dir();
  const std::string file = dir + "/" + key + ".cubin";
  {
    std::ifstream f(file, std::ios::binary);
    if (f) {
      std::vector<unsigned char> buf((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
      if (!buf.empty()) {
        std::lock_guard<std::mutex> lk(g_mtx);
        return g_cubins[key] = std::move(buf);
      }
    }
  }
  // NVRTC runs outside the lock so that several groups compile in parallel
  nvrtcProgram prog;
  std::vector<const char *> hsrc, hname;
  for (auto &h : kSkeletonHeaders) {
    hsrc.push_back(h.source);
    hname.push_back(h.name);
  }
  nvrtcResult r = nvrtcCreateProgram(&prog, source.c_str(), "map_kernel.cu", (int)hsrc.size(), hsrc.data(), hname.data());
  if (r != NVRTC_SUCCESS) throw MapError(std::string("nvrtcCreateProgram: ") + nvrtcGetErrorString(r));
  r = nvrtcCompileProgram(prog, (int)(sizeof(kNvrtcOpts) / sizeof(kNvrtcOpts[0])), kNvrtcOpts);
  size_t logn = 0;
  nvrtcGetProgramLogSize(prog, &logn);
  std::string log(logn, '\0');
  if (logn) nvrtcGetProgramLog(prog, &log[0]);
  if (r != NVRTC_SUCCESS) {
    nvrtcDestroyProgram(&prog);
    throw MapError("kernel compilation failed: " + log + "\n--- source ---\n" + source);
  }
  size_t n = 0;
  nvrtcGetCUBINSize(prog, &n);
  std::vector<unsigned char> cubin(n);
  nvrtcGetCUBIN(prog, (char *)cubin.data());
  nvrtcDestroyProgram(&prog);
  // best-effort disk cache write (atomic rename)
  ::mkdir(dir.c_str(), 0755);
  const std::string tmp = file + ".tmp" + std::to_string(::getpid()) + "_" + std::to_string((uintptr_t)&cubin);
  {
    std::ofstream f(tmp, std::ios::binary);
    if (f) f.write((const char *)cubin.data(), (std::streamsize)cubin.size());
  }
  if (std::rename(tmp.c_str(), file.c_str()) != 0) std::remove(tmp.c_str());
  std::lock_guard<std::mutex> lk(g_mtx);
  last_log_ = log;
  return g_cubins[key] = std::move(cubin);
}

void CudaEnv::set_device(int d) {
  if (device_ready_ && d != device_) throw MapError("the device cannot change after it has been set up");
  device_ = d;
}

void CudaEnv::ensure_device() {
  if (device_ready_) return;
  std::lock_guard<std::mutex> lk(g_mtx);
  if (device_ready_) return;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    throw MapError(std::string("no CUDA device available: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "0 devices"));
  if (device_ >= n) throw MapError("device index out of range");
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  cuda_check(cudaFree(0), "context creation");
  cudaDeviceProp prop;
  cuda_check(cudaGetDeviceProperties(&prop, device_), "cudaGetDeviceProperties");
  if (prop.major != 10 || prop.minor != 0)
    throw MapError(std::string("this build targets sm_100a (B200); found ") + prop.name + " sm_" +
                   std::to_string(prop.major) + std::to_string(prop.minor));
  sm_count_ = prop.multiProcessorCount;
  device_name_ = prop.name;
  load_entry(g_drv.moduleLoadData, "cuModuleLoadData");
  load_entry(g_drv.moduleGetFunction, "cuModuleGetFunction");
  load_entry(g_drv.launchKernel, "cuLaunchKernel");
  load_entry(g_drv.launchKernelEx, "cuLaunchKernelEx");
  load_entry(g_drv.funcSetAttribute, "cuFuncSetAttribute");
  load_entry(g_drv.tensorMapEncodeTiled, "cuTensorMapEncodeTiled");
  load_entry(g_drv.getErrorString, "cuGetErrorString");
  load_entry(g_drv.occupancy, "cuOccupancyMaxActiveBlocksPerMultiprocessor");
  load_entry(g_drv.memsetD2D8, "cuMemsetD2D8Async");
  load_entry(g_drv.memsetD2D16, "cuMemsetD2D16Async");
  load_entry(g_drv.memsetD2D32, "cuMemsetD2D32Async");
  cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  cuda_check(cudaMalloc(&err_word_, sizeof(uint32_t)), "cudaMalloc(error word)");
  cuda_check(cudaMemset(err_word_, 0, sizeof(uint32_t)), "cudaMemset");
  device_ready_ = true;
}

KernelHandle CudaEnv::kernel(const std::string &source, const std::string &name, size_t dyn_smem) {
  ensure_device();
  {
    std::lock_guard<std::mutex> lk(g_mtx);
    auto f = g_fast.find(name);
    if (f != g_fast.end() && f->second.source_size == source.size() && f->second.h.max_dyn_smem >= dyn_smem)
      return f->second.h;
  }
  const auto &cubin = compile(source);
  std::lock_guard<std::mutex> lk(g_mtx);
  const std::string key = hash_hex(source) + "/" + name;
  auto it = g_kernels.find(key);
  if (it != g_kernels.end() && it->second.max_dyn_smem >= dyn_smem) {
    g_fast[name] = FastEntry{source.size(), it->second};
    return it->second;
  }
  const std::string mkey = hash_hex(source);
  CUmodule mod;
  auto mit = g_modules.find(mkey);
  if (mit == g_modules.end()) {
    drv_check(g_drv.moduleLoadData(&mod, cubin.data()), "cuModuleLoadData");
    g_modules[mkey] = mod;
  } else {
    mod = mit->second;
  }
  KernelHandle h;
  CUfunction fn;
  drv_check(g_drv.moduleGetFunction(&fn, mod, name.c_str()), ("cuModuleGetFunction(" + name + ")").c_str());
  h.fn = reinterpret_cast<CUfunc_st *>(fn);
  if (dyn_smem > 48 * 1024)
    drv_check(g_drv.funcSetAttribute(fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)dyn_smem),
              "cuFuncSetAttribute");
  h.max_dyn_smem = dyn_smem;
  g_kernels[key] = h;
  g_fast[name] = FastEntry{source.size(), h};
  return h;
}

void CudaEnv::launch(const KernelHandle &k, int grid, int block, size_t smem, CUstream_st *stream, void *args, size_t) {
  if (grid <= 0) return;
  void *params[] = {args};
  drv_check(g_drv.launchKernel(reinterpret_cast<CUfunction>(k.fn), (unsigned)grid, 1, 1, (unsigned)block, 1, 1, (unsigned)smem,
                               reinterpret_cast<CUstream>(stream), params, nullptr),
            "cuLaunchKernel");
  launches_++;
}

// A launch that may begin while the previous kernel of the stream is still
// running (programmatic dependent launch): its CTAs become resident as the
// previous grid's CTAs exit and run their prologue; the kernel must execute
// griddepcontrol.wait (map_common.cuh griddep_wait) before it touches global
// memory, which waits for the previous grid to complete and its writes to be
// visible. Used for the generated Local / Focal kernels, which all do.
void CudaEnv::launch_2d(const KernelHandle &k, int gx, int gy, int block, size_t smem, CUstream_st *stream, void *args) {
  if (gx <= 0 || gy <= 0) return;
  void *params[] = {args};
  drv_check(g_drv.launchKernel(reinterpret_cast<CUfunction>(k.fn), (unsigned)gx, (unsigned)gy, 1, (unsigned)block, 1, 1,
                               (unsigned)smem, reinterpret_cast<CUstream>(stream), params, nullptr),
            "cuLaunchKernel");
  launches_++;
}

void CudaEnv::launch_pdl(const KernelHandle &k, int grid, int gy, int block, size_t smem, CUstream_st *stream, void *args) {
  if (grid <= 0 || gy <= 0) return;
  void *params[] = {args};
  CUlaunchAttribute attr;
  attr.id = CU_LAUNCH_ATTRIBUTE_PROGRAMMATIC_STREAM_SERIALIZATION;
  attr.value.programmaticStreamSerializationAllowed = 1;
  CUlaunchConfig cfg = {};
  cfg.gridDimX = (unsigned)grid;
  cfg.gridDimY = (unsigned)gy;
  cfg.gridDimZ = 1;
  cfg.blockDimX = (unsigned)block;
  cfg.blockDimY = 1;
  cfg.blockDimZ = 1;
  cfg.sharedMemBytes = (unsigned)smem;
  cfg.hStream = reinterpret_cast<CUstream>(stream);
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  drv_check(g_drv.launchKernelEx(&cfg, reinterpret_cast<CUfunction>(k.fn), params, nullptr), "cuLaunchKernelEx");
  launches_++;
}

// A launch whose CTAs form 1-D thread-block clusters of `cluster` CTAs (grid a
// multiple of it): the CTAs of a cluster run at once on one GPC and share
// their shared memory.
void CudaEnv::launch_cluster(const KernelHandle &k, int grid, int block, int cluster, size_t smem, CUstream_st *stream,
                             void *args) {
  if (grid <= 0) return;
  if (cluster <= 0 || grid % cluster != 0) throw MapError("cluster launch: grid is not a multiple of the cluster size");
  void *params[] = {args};
  CUlaunchAttribute attr;
  attr.id = CU_LAUNCH_ATTRIBUTE_CLUSTER_DIMENSION;
  attr.value.clusterDim.x = (unsigned)cluster;
  attr.value.clusterDim.y = 1;
  attr.value.clusterDim.z = 1;
  CUlaunchConfig cfg = {};
  cfg.gridDimX = (unsigned)grid;
  cfg.gridDimY = 1;
  cfg.gridDimZ = 1;
  cfg.blockDimX = (unsigned)block;
  cfg.blockDimY = 1;
  cfg.blockDimZ = 1;
  cfg.sharedMemBytes = (unsigned)smem;
  cfg.hStream = reinterpret_cast<CUstream>(stream);
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  drv_check(g_drv.launchKernelEx(&cfg, reinterpret_cast<CUfunction>(k.fn), params, nullptr), "cuLaunchKernelEx");
  launches_++;
}

int CudaEnv::occupancy(const KernelHandle &k, int block, size_t smem) {
  int n = 0;
  drv_check(g_drv.occupancy(&n, reinterpret_cast<CUfunction>(k.fn), block, smem), "cuOccupancyMaxActiveBlocksPerMultiprocessor");
  return n;
}

void CudaEnv::encode_tma_2d(void *desc128, int dtype, const void *base, uint64_t width, uint64_t height, uint64_t pitch_bytes,
                            uint32_t box_w, uint32_t box_h) {
  ensure_device();
  CUtensorMapDataType t;
  switch (dtype) {
    case U8: case S8: case B8: t = CU_TENSOR_MAP_DATA_TYPE_UINT8; break;
    case U16: case S16: t = CU_TENSOR_MAP_DATA_TYPE_UINT16; break;
    case U32: t = CU_TENSOR_MAP_DATA_TYPE_UINT32; break;
    case S32: t = CU_TENSOR_MAP_DATA_TYPE_INT32; break;
    case F32: t = CU_TENSOR_MAP_DATA_TYPE_FLOAT32; break;
    case U64: t = CU_TENSOR_MAP_DATA_TYPE_UINT64; break;
    case S64: t = CU_TENSOR_MAP_DATA_TYPE_INT64; break;
    case F64: t = CU_TENSOR_MAP_DATA_TYPE_FLOAT64; break;
    default: throw MapError("TMA: unsupported data type");
  }
  if (((uintptr_t)base & 15) != 0) throw MapError("TMA: base address not 16-byte aligned");
  if ((pitch_bytes & 15) != 0) throw MapError("TMA: pitch not a multiple of 16 bytes");
  if ((box_w * dt_size(dtype)) % 16 != 0) throw MapError("TMA: box row not a multiple of 16 bytes");
  cuuint64_t dims[2] = {width, height};
  cuuint64_t strides[1] = {pitch_bytes};
  cuuint32_t box[2] = {box_w, box_h};
  cuuint32_t estr[2] = {1, 1};
  drv_check(g_drv.tensorMapEncodeTiled(reinterpret_cast<CUtensorMap *>(desc128), t, 2, const_cast<void *>(base), dims, strides,
                                       box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                       CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE),
            "cuTensorMapEncodeTiled");
}

bool CudaEnv::fill_2d(void *dst, size_t pitch, const void *value, int elem_size, size_t width, size_t height,
                      CUstream_st *stream) {
  if (width == 0 || height == 0) return true;
  const CUdeviceptr d = (CUdeviceptr)(uintptr_t)dst;
  if (elem_size == 1) {
    unsigned char v;
    std::memcpy(&v, value, 1);
    drv_check(g_drv.memsetD2D8(d, pitch, v, width, height, (CUstream)stream), "cuMemsetD2D8Async");
  } else if (elem_size == 2) {
    unsigned short v;
    std::memcpy(&v, value, 2);
    drv_check(g_drv.memsetD2D16(d, pitch, v, width, height, (CUstream)stream), "cuMemsetD2D16Async");
  } else if (elem_size == 4) {
    unsigned int v;
    std::memcpy(&v, value, 4);
    drv_check(g_drv.memsetD2D32(d, pitch, v, width, height, (CUstream)stream), "cuMemsetD2D32Async");
  } else {
    return false;
  }
  return true;
}

}  // namespace mapb
