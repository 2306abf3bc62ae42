// Device building blocks of the Radiating (radial scan) and Spreading (flow
// accumulation) skeletons.
#pragma once
#include "map_common.cuh"

// Octants of a radial scan: primary unit (p0,p1) and secondary unit (q0,q1).
// A cell at (d0, d1) from the start, 0 <= d1 <= d0, lies at start + d0*p + d1*q
// (the reference's eight RadialCase pairs, runtime/Direction.hpp:71-164).
__device__ __forceinline__ void octant_units(int o, int &p0, int &p1, int &q0, int &q1) {
  const int P[8][4] = {{0, -1, 1, 0}, {1, 0, 0, -1}, {1, 0, 0, 1}, {0, 1, 1, 0},
                       {0, 1, -1, 0}, {-1, 0, 0, 1}, {-1, 0, 0, -1}, {0, -1, -1, 0}};
  p0 = P[o][0]; p1 = P[o][1]; q0 = P[o][2]; q1 = P[o][3];
}

// Linear interpolation of the two previous cells along the ray
// (runtime/skeleton/util.cpp:564): a at (d0-1, d1), b at (d0-1, d1-1).
template <class T> __device__ __forceinline__ T radial_lit(T a, T b, int d0, int d1) {
  if (d1 == 0) return a;
  if (d0 == d1) return b;
  T w = (T)d1 / (T)d0 * ((T)d0 - (T)1.0f) - ((T)d1 - (T)1.0f);
  return a * w + b * ((T)1.0f - w);
}

// D8 code -> direction index (E, SE, S, SW, W, NW, N, NE), -1 when the code is
// not a single direction.
__device__ __forceinline__ int d8_index(u8 c) {
  if (c == 0 || (c & (c - 1)) != 0) return -1;
  return __ffs((int)c) - 1;
}
__device__ __forceinline__ int d8_dx(int d) { const int t[8] = {1, 1, 0, -1, -1, -1, 0, 1}; return t[d]; }
__device__ __forceinline__ int d8_dy(int d) { const int t[8] = {0, 1, 1, 1, 0, -1, -1, -1}; return t[d]; }

// Downstream cell of (x, y) along its D8 code, or -1.
__device__ __forceinline__ s64 d8_down(const RasterArg &dir, int W, int H, int x, int y) {
  int d = d8_index(ldr<u8>(dir, x, y));
  if (d < 0) return -1;
  int nx = x + d8_dx(d), ny = y + d8_dy(d);
  if (nx < 0 || ny < 0 || nx >= W || ny >= H) return -1;
  return (s64)ny * W + nx;
}

template <class T> __device__ __forceinline__ T ld_coherent(const RasterArg &r, int x, int y) {
  return __ldcg(row_ptr<T>(r, y) + x);
}
template <class T> __device__ __forceinline__ T *cell_ptr(const RasterArg &r, int x, int y) {
  return (T *)(r.p + (u64)(s64)y * (u64)r.pitch) + x;
}
// Decrements *p with acquire-release ordering at device scope (the caller's earlier
// writes are visible to whoever sees the result, and later reads see theirs);
// returns the previous value.
__device__ __forceinline__ s32 atomic_dec_acq_rel(s32 *p) {
  s32 old;
  asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], -1;" : "=r"(old) : "l"(p) : "memory");
  return old;
}
__device__ __forceinline__ void atomic_add_any(s32 *p, s32 v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add_any(u32 *p, u32 v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add_any(float *p, float v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add_any(double *p, double v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add_any(s64 *p, s64 v) { atomicAdd((unsigned long long *)p, (unsigned long long)v); }
__device__ __forceinline__ void atomic_add_any(u64 *p, u64 v) { atomicAdd((unsigned long long *)p, (unsigned long long)v); }
