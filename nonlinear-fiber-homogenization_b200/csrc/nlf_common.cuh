// Shared definitions for the nlfiber-b200 CUDA library (sm_100a).
//
// Device layout of every nodal field: vec-major SoA, [vec][component][x][y][z] with z fastest, where
// vec = cell * m + load case. N = nx * ny * nz voxels = nodes = elements (periodic grid). The element
// e = (i, j, k) owns the nodes e + (ax, ay, az), a = ax + 2 ay + 4 az (nlfiber/linear.py:22,80-92).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#define NLF_OK 0
#define NLF_NOT_CONVERGED 1
#define NLF_BREAKDOWN 2
#define NLF_EBADARG (-1)
#define NLF_ECUDA (-2)
#define NLF_ETIMEOUT (-3)

namespace nlf {

void set_error(const char* fmt, ...);

// Raises the dynamic shared memory limit of a kernel to at least `bytes` and never lowers it: handles of
// different grid sizes may launch the same kernel from several host threads at once, and a lowered limit would
// fail another thread's launch. Thread-safe.
cudaError_t raise_dyn_smem(const void* func, int bytes);
template <typename F>
cudaError_t raise_dyn_smem(F* func, int bytes) {
  return raise_dyn_smem(reinterpret_cast<const void*>(func), bytes);
}

#define NLF_CUDA_TRY(expr)                                                                     \
  do {                                                                                         \
    cudaError_t _e = (expr);                                                                   \
    if (_e != cudaSuccess) {                                                                   \
      ::nlf::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #expr, cudaGetErrorString(_e));    \
      return NLF_ECUDA;                                                                        \
    }                                                                                          \
  } while (0)

#define NLF_CHECK_LAUNCH() NLF_CUDA_TRY(cudaGetLastError())

#define NLF_TRY(expr)        \
  do {                       \
    int _s = (expr);         \
    if (_s < 0) return _s;   \
  } while (0)

template <typename T>
struct cplx {
  T x, y;
};

template <typename T>
__device__ __forceinline__ cplx<T> cmul(cplx<T> a, cplx<T> b) {
  return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename T>
__device__ __forceinline__ cplx<T> cadd(cplx<T> a, cplx<T> b) { return {a.x + b.x, a.y + b.y}; }
template <typename T>
__device__ __forceinline__ cplx<T> csub(cplx<T> a, cplx<T> b) { return {a.x - b.x, a.y - b.y}; }
template <typename T>
__device__ __forceinline__ cplx<T> cconj(cplx<T> a) { return {a.x, -a.y}; }

__host__ __device__ __forceinline__ int wrap(int i, int n) {
  i %= n;
  return i < 0 ? i + n : i;
}

__host__ __device__ __forceinline__ bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

__host__ __device__ __forceinline__ int ilog2(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return l;
}

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n >> 1); }

// x / d with a shift when d is a power of two (the usual grid sides)
__device__ __forceinline__ int fdiv(int x, int d) { return is_pow2(d) ? (x >> (31 - __clz(d))) : x / d; }

// Block-wide sum of K doubles; result valid in thread 0. `sh` needs 32*K doubles.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double x = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    v[k] = x;
  }
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) sh[wid * K + k] = v[k];
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double x = lane < nw ? sh[lane * K + k] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      v[k] = x;
    }
  }
  __syncthreads();
}

}  // namespace nlf
