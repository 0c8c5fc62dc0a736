// Common device-side definitions for the TorChannel B200 step kernels.
//
// Internal HBM layout (x fastest, DOFs only):
//   u, v  : [nz][ny][nx]     plane k <-> reference cell k+1, row j <-> j+1,
//                            column i <-> i+1 (reference arrays carry ghosts)
//   w     : [nz+1][ny][nx]   plane f <-> reference face f; planes 0 and nz are
//                            the walls and always hold 0
//   p     : [nz][ny][nx]
// x/y ghosts do not exist in memory: the reference's periodic ghost copies
// (solver.py:45-75) are index wraps here.  z ghosts of u/v (solver.py:50-67)
// are formed on the fly: below the bottom wall -q[0], above the top wall
// -q[nz-1] (no-slip) or +q[nz-1] (free-slip).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tc {

// ---- bounds-checked builds -----------------------------------------------
// Built with -DTC_BOUNDS_CHECK, every access of the step kernels written as
// TC_IN(i, n, w) ? access : fallback first checks that the w elements from
// index i lie inside the n elements of their buffer; an access out of range
// is skipped (loads give 0) and sets tc_bounds_word, with the code
// file id * 100000 + source line of the first such access in tc_bounds_where
// (tc_bounds_error() reads and clears both).  Without the flag TC_IN is
// `true` and the accesses compile as written.  File ids: TC_FILE_ID of each
// source (1 tc_step.cuh, 2 tc_rhs_tma.cuh, 3 tc_poisson.cuh).
#ifdef TC_BOUNDS_CHECK
__device__ unsigned int tc_bounds_word;
__device__ int tc_bounds_where;
__device__ __noinline__ bool tc_bounds_fail(int where) {
  if (atomicOr(&tc_bounds_word, 1u) == 0u) atomicExch(&tc_bounds_where, where);
  return false;
}
#define TC_IN(i, n, w) \
  (((size_t)(i) + (size_t)(w) <= (size_t)(n)) || ::tc::tc_bounds_fail(TC_FILE_ID * 100000 + __LINE__))
#else
#define TC_IN(i, n, w) true
#endif

template <class T> struct cpx { T x, y; };

template <class T> __device__ __forceinline__ cpx<T> cmake(T a, T b) { cpx<T> r; r.x = a; r.y = b; return r; }
template <class T> __device__ __forceinline__ cpx<T> cadd(cpx<T> a, cpx<T> b) { return cmake<T>(a.x + b.x, a.y + b.y); }
template <class T> __device__ __forceinline__ cpx<T> csub(cpx<T> a, cpx<T> b) { return cmake<T>(a.x - b.x, a.y - b.y); }
template <class T> __device__ __forceinline__ cpx<T> cmul(cpx<T> a, cpx<T> b) {
  return cmake<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <class T> __device__ __forceinline__ cpx<T> cconj(cpx<T> a) { return cmake<T>(a.x, -a.y); }
template <class T> __device__ __forceinline__ cpx<T> cscale(cpx<T> a, T s) { return cmake<T>(a.x * s, a.y * s); }

// Grid description passed by value to every kernel.  Reciprocal tables are
// stored both in FP64 and in the storage type T (for FP32 stencils).
template <class T> struct Grid {
  int nx, ny, nz;
  T idx, idy;            // 1/dx, 1/dy
  T nu_idx2, nu_idy2;    // nu/dx^2, nu/dy^2
  T nu;
  const T* idzf;         // 1/dz_f[k], k < nz
  const T* idzc;         // 1/dz_c[k], k <= nz
  int top_neumann;       // 1: free-slip top wall
  int rhs_fused;         // 1: explicit RHS with the reference CUDA-path edge planes
  // Base profile of u (mixed precision): u is stored as u - U0[k] so that the
  // FP32 values stay small; nullptr in the FP64 form.
  const T* ubase_t;      // U0[k] in the storage type
  const double* ubase_d; // U0[k] in FP64
};

__host__ __device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

__host__ __device__ __forceinline__ size_t pidx(int k, int j, int i, int ny, int nx) {
  return ((size_t)k * ny + j) * nx + i;
}

template <class T> __device__ __forceinline__ T ldg(const T* p) { return __ldg(p); }

// Block-wide FP64 sum; every thread gets the result.  blockDim.x*y*z <= 1024.
__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  int nt = blockDim.x * blockDim.y * blockDim.z;
  int w = t >> 5, l = t & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  int nw = (nt + 31) >> 5;
  if (t < 32) {
    r = (t < nw) ? sh[t] : 0.0;
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    if (t == 0) sh[0] = r;
  }
  __syncthreads();
  r = sh[0];
  __syncthreads();
  return r;
}

__device__ __forceinline__ double block_max(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  int nt = blockDim.x * blockDim.y * blockDim.z;
  int w = t >> 5, l = t & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  int nw = (nt + 31) >> 5;
  if (t < 32) {
    r = (t < nw) ? sh[t] : 0.0;
    for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, o));
    if (t == 0) sh[0] = r;
  }
  __syncthreads();
  r = sh[0];
  __syncthreads();
  return r;
}

// Device error word bits (read by the host at sync points only).
enum : int {
  TCE_NONFINITE = 1,
  TCE_BOUNDS = 2,
  TCE_TIMEOUT = 4,  // a bounded wait for a bulk copy ran out
};

}  // namespace tc
