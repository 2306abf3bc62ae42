// Build-time self-check: instantiates the skeleton building blocks under nvcc
// for sm_100a (the same headers NVRTC compiles generated kernels against).
#include "common.cuh"

struct __align__(64) CheckArgs {
  TmaDesc tm[1];
  RasterArg in[1];
  RasterArg out[1];
  Geom g;
  u32 *err;
};

extern "C" __global__ void __launch_bounds__(256) selfcheck_focal(const __grid_constant__ CheckArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  const Tile t = tile_of<64, 32>(a.g, blockIdx.x);
  u64 *bar = (u64 *)(smem + 72 * 34 * 4);
  if (tile_interior<64, 32>(a.g, t, 1, 1)) {
    if (threadIdx.x == 0) { mbar_init(bar, 1); fence_mbar_init(); }
    __syncthreads();
    if (threadIdx.x == 0) {
      mbar_arrive_expect_tx(bar, 72 * 34 * 4);
      tma_load_2d(smem, &a.tm[0], bar, t.x0 - 4, t.y0 - 1);
    }
    if (!mbar_wait_bounded(bar, 0, 1u << 14)) { skel_fail(a.err, ERR_TMA_TIMEOUT); return; }
    const SmemTap<float, 72, 4, 1> f{(const float *)smem};
    const int x = t.x0 + threadIdx.x % 64, y = t.y0 + threadIdx.x / 64;
    str<float>(a.out[0], x, y, f.tap(x, y, threadIdx.x % 64, threadIdx.x / 64, -1, 1));
  } else {
    const GatherTap<float> f{a.in[0], &a.g};
    const int x = t.x0 + threadIdx.x % 64, y = t.y0 + threadIdx.x / 64;
    if (x < t.xe && y < t.ye) str<float>(a.out[0], x, y, f.tap(x, y, 0, 0, -1, 1));
  }
}

extern "C" __global__ void __launch_bounds__(256) selfcheck_reduce(const float *in, double *out, u8 *o8, int n) {
  __shared__ Scalar8 scratch[8];
  float acc = 0.f;
  double m = -1.0 / 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    acc = RedOp<1, float>::f(acc, in[i]);
    m = RedOp<6, double>::f(m, (double)in[i]);
  }
  float r = block_reduce<1, float>(acc, scratch);
  double r2 = block_reduce<6, double>(m, scratch);
  u32 c0 = (u32)n, c1 = 0u;
  philox2x32_10(c0, c1, 7u);
  if (threadIdx.x == 0) { out[0] = r; out[1] = r2; o8[0] = (u8)c0; }
}
