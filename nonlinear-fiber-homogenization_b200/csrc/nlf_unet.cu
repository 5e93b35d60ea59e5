// Warm-start U-Net: maps a density cell to the 6 unit-strain correctors (18 channels, u / n0), whose prediction
// is the initial guess u0 of the corrector solve (nlfiber/linear.py:209-212, `solve(s, Es, u0)`, and
// `C_full(rho, u0)` :231-236; the reference always starts from u0 = 0). Architecture, loss and parameter layout
// are those of the NumPy oracle oracle/unet_ref.py.
//
// Layout: activations channels-last BF16 [nb][n0][n1][n2][C]; gradients FP32. Every 3x3x3 (and the final 1x1)
// convolution, forward and backward-data, is an implicit GEMM on the tcgen05 tensor cores: M = 128 voxels per
// CTA, N = output channels, K = (tap, input channel), BF16 operands gathered (periodic wrap) into shared memory
// by cp.async, FP32 accumulators in TMEM, one thread issuing the MMAs and committing them to an mbarrier per
// pipeline stage. The weight gradient is the same machinery with M = (tap, input channel), N = output channel
// and K = voxels, reading both operands in their channels-last (MN-major) layout directly.
#include <cuda_bf16.h>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include "nlf_internal.h"
#include "nlf_prof.cuh"
#include "nlf_tc.cuh"

namespace nlf {
namespace unet {

using bf16 = __nv_bfloat16;

constexpr int kStages = 4;
constexpr uint32_t kStageA = 128 * 128;  // 128 rows x 64 K elements of BF16
constexpr int kOut = 18;                 // 6 cases x 3 components

__device__ __forceinline__ int wrapi(int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); }

// voxel index of (i, j, k) + sign * off(t), off(t) = (t / 9 - 1, t / 3 % 3 - 1, t % 3 - 1), periodic
__device__ __forceinline__ long nbr(int i, int j, int k, int t, int sign, int n0, int n1, int n2) {
  const int di = sign * (t / 9 - 1), dj = sign * ((t / 3) % 3 - 1), dk = sign * (t % 3 - 1);
  return ((long)wrapi(i + di, n0) * n1 + wrapi(j + dj, n1)) * n2 + wrapi(k + dk, n2);
}

// ---- the tcgen05 main loop -------------------------------------------------------------------------------------
// nsteps stages of K = 64 (4 MMAs of K = 16) into the TMEM accumulator; ld(stage_smem_addr, step) issues the
// cp.async copies of one step. A 4-deep ring: the copies of step k + 3 are issued after the MMAs of step k, once
// the MMAs of step k - 1 (the previous user of that slot) have completed. The u-th completion of a slot's
// mbarrier has parity u & 1, and no slot is committed again before every thread has seen its previous
// completion. Returns false, uniformly over the CTA, when an mbarrier wait timed out (*err raised).
template <int NPAD, class Loader>
__device__ bool mainloop(const Loader& ld, int nsteps, uint32_t su, uint64_t* mbar, uint32_t tmem, uint32_t idesc,
                         int* err) {
  constexpr uint32_t SB = kStageA + NPAD * 128;
  int bad = 0;  // this thread's wait timed out; the CTA leaves together through __syncthreads_or
  for (int s = 0; s < kStages - 1; ++s) {
    if (s < nsteps) ld(su + s * SB, s);
    tc::cp_commit();
  }
  for (int kb = 0; kb < nsteps; ++kb) {
    const int st = kb % kStages;
    tc::cp_wait<kStages - 2>();
    tc::fence_proxy_async();
    if (__syncthreads_or(bad)) return false;
    if (threadIdx.x == 0) {
      tc::fence_after();
      const uint32_t a0 = su + st * SB, b0 = a0 + kStageA;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)
        tc::mma_bf16(tmem, tc::sdesc(a0 + kk * 256), tc::sdesc(b0 + kk * 256), idesc, (kb | kk) != 0);
      tc::commit(tc::smem_u32(&mbar[st]));
    }
    const int nx = kb + kStages - 1;
    if (nx < nsteps) {
      if (kb >= 1 && !tc::mbar_wait(tc::smem_u32(&mbar[(kb - 1) % kStages]), ((kb - 1) / kStages) & 1, err))
        bad = 1;
      if (!bad) ld(su + (nx % kStages) * SB, nx);
    }
    tc::cp_commit();
  }
  const int last = nsteps - 1;
  if (!bad && !tc::mbar_wait(tc::smem_u32(&mbar[last % kStages]), (last / kStages) & 1, err)) bad = 1;
  tc::cp_wait<0>();
  return !__syncthreads_or(bad);
}

template <int NPAD>
constexpr uint32_t tmem_cols() {
  return NPAD <= 32 ? 32u : (NPAD <= 64 ? 64u : 128u);
}

// CTA prologue / epilogue shared by the kernels: TMEM allocation by warp 0, mbarrier init by thread 0.
template <int NPAD>
__device__ __forceinline__ uint32_t tc_setup(uint32_t* s_tmem, uint64_t* mbar) {
  if ((threadIdx.x >> 5) == 0) {
    tc::tmem_alloc(tc::smem_u32(s_tmem), tmem_cols<NPAD>());
    tc::tmem_relinquish();
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) tc::mbar_init(tc::smem_u32(&mbar[s]), 1);
    tc::mbar_fence_init();
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  return *s_tmem;
}
template <int NPAD>
__device__ __forceinline__ void tc_teardown(uint32_t tmem) {
  tc::fence_before();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) tc::tmem_dealloc(tmem, tmem_cols<NPAD>());
}

__device__ __forceinline__ uint32_t aligned_smem(uint8_t* raw) {
  const uint32_t a = tc::smem_u32(raw);
  return (a + 1023u) & ~1023u;
}

// ---- convolution (forward and backward-data), K-major operands ---------------------------------------------------
struct ConvArgs {
  const bf16* x;      // [nb * nvox][cin]
  const bf16* w;      // [ntaps][NPAD][cin]: rows = output channels (zero beyond cout)
  const float* bias;  // [cout] or null
  void* y;            // [nb * nvox][ystride], BF16 or FP32
  int nb, n0, n1, n2, cin, cout, ystride, ntaps, sign, relu, out_f32;
  int* err;
};

template <int NPAD>
struct ConvLoad {
  const bf16* x;
  const bf16* w;
  int cin, ck, kt, ntaps, sign, n0, n1, n2;
  long bofs;
  int i, j, k;
  bool valid;
  __device__ void operator()(uint32_t su, int step) const {
    const int tid = threadIdx.x;
    const uint32_t arow = su + (tid >> 3) * tc::kSBO + (tid & 7) * 16;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int col = step * 8 + c;
      const bf16* src = x;
      uint32_t nbytes = 0;
      if (valid && col < kt) {
        const int tap = col / ck, ch = col - tap * ck;
        src = x + (bofs + nbr(i, j, k, ntaps == 27 ? tap : 13, sign, n0, n1, n2)) * cin + ch * 8;
        nbytes = 16;
      }
      tc::cp16(arow + c * 128, src, nbytes);
    }
    for (int q = tid; q < NPAD * 8; q += 128) {
      const int n = q % NPAD, c = q / NPAD;
      const int col = step * 8 + c;
      const bf16* src = w;
      uint32_t nbytes = 0;
      if (col < kt) {
        const int tap = col / ck, ch = col - tap * ck;
        src = w + ((long)tap * NPAD + n) * cin + ch * 8;
        nbytes = 16;
      }
      tc::cp16(su + kStageA + (n >> 3) * tc::kSBO + c * 128 + (n & 7) * 16, src, nbytes);
    }
  }
};

template <int NPAD>
__global__ void __launch_bounds__(128) k_conv_tc(ConvArgs a) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ uint64_t mbar[kStages];
  __shared__ uint32_t s_tmem;
  const uint32_t su = aligned_smem(smem_raw);
  const uint32_t tmem = tc_setup<NPAD>(&s_tmem, mbar);
  const int tid = threadIdx.x, warp = tid >> 5;
  const long nvox = (long)a.n0 * a.n1 * a.n2, total = (long)a.nb * nvox;
  const long v = (long)blockIdx.x * 128 + tid;
  ConvLoad<NPAD> ld;
  ld.x = a.x;
  ld.w = a.w;
  ld.cin = a.cin;
  ld.ck = a.cin / 8;
  ld.kt = a.ntaps * ld.ck;
  ld.ntaps = a.ntaps;
  ld.sign = a.sign;
  ld.n0 = a.n0;
  ld.n1 = a.n1;
  ld.n2 = a.n2;
  ld.valid = v < total;
  {
    const long b = ld.valid ? v / nvox : 0, l = ld.valid ? v - b * nvox : 0;
    ld.bofs = b * nvox;
    ld.i = (int)(l / ((long)a.n1 * a.n2));
    ld.j = (int)((l / a.n2) % a.n1);
    ld.k = (int)(l % a.n2);
  }
  const int nsteps = (ld.kt + 7) / 8;
  if (mainloop<NPAD>(ld, nsteps, su, mbar, tmem, tc::idesc_bf16(NPAD, 0, 0), a.err)) {
    tc::fence_after();
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
    for (int c0 = 0; c0 < NPAD; c0 += 16) {
      uint32_t r[16];
      tc::ld16(trow + c0, r);
      tc::wait_ld();
      if (v < total) {
        float f[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const int co = c0 + q;
          f[q] = __uint_as_float(r[q]) + ((a.bias && co < a.cout) ? a.bias[co] : 0.f);
          if (a.relu) f[q] = fmaxf(f[q], 0.f);
        }
        if (a.out_f32) {
          float* yp = static_cast<float*>(a.y) + v * a.ystride + c0;
          if (c0 + 16 <= a.cout && (a.ystride & 3) == 0) {
#pragma unroll
            for (int q = 0; q < 16; q += 4) *reinterpret_cast<float4*>(yp + q) = make_float4(f[q], f[q + 1], f[q + 2], f[q + 3]);
          } else {
            for (int q = 0; q < 16 && c0 + q < a.cout; ++q) yp[q] = f[q];
          }
        } else {
          bf16* yp = static_cast<bf16*>(a.y) + v * a.ystride + c0;
          if (c0 + 16 <= a.cout && (a.ystride & 7) == 0) {
            uint4 pk[2];
            __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(pk);
#pragma unroll
            for (int q = 0; q < 8; ++q) h[q] = __floats2bfloat162_rn(f[2 * q], f[2 * q + 1]);
            reinterpret_cast<uint4*>(yp)[0] = pk[0];
            reinterpret_cast<uint4*>(yp)[1] = pk[1];
          } else {
            for (int q = 0; q < 16 && c0 + q < a.cout; ++q) yp[q] = __float2bfloat16_rn(f[q]);
          }
        }
      }
    }
  }
  tc_teardown<NPAD>(tmem);
}

// ---- weight gradient, MN-major operands --------------------------------------------------------------------------
// part[chunk][q][co] = sum over the chunk's voxels v of x[v + off(tap)][ci] g[v][co], q = tap * cin + ci.
struct DwArgs {
  const bf16* x;  // [nb * nvox][cin] (the layer's input)
  const bf16* g;  // [nb * nvox][NPAD] (the gradient at the layer's output, masked, zero beyond cout)
  float* part;    // [nchunk][rows_pad][NPAD]
  int nb, n0, n1, n2, cin, ntaps, rows, rows_pad;
  long vpc;  // voxels per chunk, a multiple of 64
  int* err;
};

template <int NPAD>
struct DwLoad {
  const bf16* x;
  const bf16* g;
  int cin, rows, ntaps, n0, n1, n2, mt;
  long nvox, vbeg, vend;
  __device__ void operator()(uint32_t su, int step) const {
    const int tid = threadIdx.x, kv = tid & 63;
    const long v = vbeg + (long)step * 64 + kv;
    const bool vv = v < vend;
    long b = 0, l = 0;
    if (vv) {
      b = v / nvox;
      l = v - b * nvox;
    }
    const int i = (int)(l / ((long)n1 * n2)), j = (int)((l / n2) % n1), k = (int)(l % n2);
    const uint32_t koff = (kv >> 3) * 128 + (kv & 7) * 16;
#pragma unroll
    for (int it = 0; it < 8; ++it) {
      const int mg = (tid >> 6) + 2 * it;
      const int q0 = mt * 128 + mg * 8;
      const bf16* src = x;
      uint32_t nbytes = 0;
      if (vv && q0 < rows) {
        const int tap = q0 / cin, ci0 = q0 - tap * cin;
        src = x + (b * nvox + nbr(i, j, k, ntaps == 27 ? tap : 13, 1, n0, n1, n2)) * cin + ci0;
        nbytes = 16;
      }
      tc::cp16(su + mg * tc::kSBO + koff, src, nbytes);
    }
#pragma unroll
    for (int it = 0; it < NPAD / 16; ++it) {
      const int ng = (tid >> 6) + 2 * it;
      tc::cp16(su + kStageA + ng * tc::kSBO + koff, vv ? g + v * NPAD + ng * 8 : g, vv ? 16u : 0u);
    }
  }
};

template <int NPAD>
__global__ void __launch_bounds__(128) k_dw_tc(DwArgs a) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ uint64_t mbar[kStages];
  __shared__ uint32_t s_tmem;
  const uint32_t su = aligned_smem(smem_raw);
  const uint32_t tmem = tc_setup<NPAD>(&s_tmem, mbar);
  const int tid = threadIdx.x, warp = tid >> 5;
  const long nvox = (long)a.n0 * a.n1 * a.n2, total = (long)a.nb * nvox;
  DwLoad<NPAD> ld;
  ld.x = a.x;
  ld.g = a.g;
  ld.cin = a.cin;
  ld.rows = a.rows;
  ld.ntaps = a.ntaps;
  ld.n0 = a.n0;
  ld.n1 = a.n1;
  ld.n2 = a.n2;
  ld.mt = blockIdx.x;
  ld.nvox = nvox;
  ld.vbeg = (long)blockIdx.y * a.vpc;
  ld.vend = ld.vbeg + a.vpc < total ? ld.vbeg + a.vpc : total;
  const int nsteps = (int)((ld.vend - ld.vbeg + 63) / 64);
  if (mainloop<NPAD>(ld, nsteps, su, mbar, tmem, tc::idesc_bf16(NPAD, 1, 1), a.err)) {
    tc::fence_after();
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    float* out = a.part + ((long)blockIdx.y * a.rows_pad + (long)blockIdx.x * 128 + tid) * NPAD;
#pragma unroll 1
    for (int c0 = 0; c0 < NPAD; c0 += 16) {
      uint32_t r[16];
      tc::ld16(trow + c0, r);
      tc::wait_ld();
#pragma unroll
      for (int q = 0; q < 16; q += 4)
        *reinterpret_cast<float4*>(out + c0 + q) = make_float4(__uint_as_float(r[q]), __uint_as_float(r[q + 1]),
                                                               __uint_as_float(r[q + 2]), __uint_as_float(r[q + 3]));
    }
  }
  tc_teardown<NPAD>(tmem);
}

// dW[t][co][ci] (ci < cin_true, co < cout) = sum over chunks of part[chunk][t * cin + ci][co], in chunk order
__global__ void k_dw_reduce(const float* __restrict__ part, int nchunk, int rows_pad, int npad, int ntaps, int cin,
                            int cin_true, int cout, float* __restrict__ dW) {
  const long n = (long)ntaps * cout * cin_true;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
    const int ci = (int)(idx % cin_true), co = (int)((idx / cin_true) % cout), t = (int)(idx / ((long)cin_true * cout));
    const long q = (long)t * cin + ci;
    float s = 0.f;
    for (int c = 0; c < nchunk; ++c) s += part[((long)c * rows_pad + q) * npad + co];
    dW[idx] = s;
  }
}

// per-channel sums of g [V][C] (bias gradient): block partials then a fixed-order final sum
__global__ void k_colsum_part(const bf16* __restrict__ g, long V, int C, float* __restrict__ part) {
  __shared__ float red[256];
  const int lanes = blockDim.x / C, c = threadIdx.x % C, lane = threadIdx.x / C;
  float s = 0.f;
  if (lane < lanes)
    for (long v = (long)blockIdx.x * lanes + lane; v < V; v += (long)gridDim.x * lanes)
      s += __bfloat162float(g[v * C + c]);
  red[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x < C) {
    float t = 0.f;
    for (int l = 0; l < lanes; ++l) t += red[l * C + threadIdx.x];
    part[(long)blockIdx.x * C + threadIdx.x] = t;
  }
}
__global__ void k_colsum_fin(const float* __restrict__ part, int nblk, int C, int cout, float* __restrict__ db) {
  const int c = threadIdx.x;
  if (c >= cout) return;
  float s = 0.f;
  for (int b = 0; b < nblk; ++b) s += part[(long)b * C + c];
  db[c] = s;
}

// ---- elementwise -------------------------------------------------------------------------------------------------
// x0[v] = (rho[v], 0, ..., 0): the 1-channel input padded to 8 channels
__global__ void k_input(const float* __restrict__ rho, long V, bf16* __restrict__ x0) {
  for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < V; v += (long)gridDim.x * blockDim.x) {
    uint4 pk = make_uint4(0, 0, 0, 0);
    reinterpret_cast<bf16*>(&pk)[0] = __float2bfloat16_rn(rho[v]);
    reinterpret_cast<uint4*>(x0)[v] = pk;
  }
}

// coarse (c0, c1, c2) -> fine voxel index of child (a, b, c)
__device__ __forceinline__ long child(long cv, int a, int n0c, int n1c, int n2c) {
  const long bb = cv / ((long)n0c * n1c * n2c), l = cv - bb * n0c * n1c * n2c;
  const int i = (int)(l / ((long)n1c * n2c)), j = (int)((l / n2c) % n1c), k = (int)(l % n2c);
  const int n1 = 2 * n1c, n2 = 2 * n2c;
  return bb * 8L * n0c * n1c * n2c + ((long)(2 * i + (a & 1)) * n1 + 2 * j + ((a >> 1) & 1)) * n2 + 2 * k + (a >> 2);
}
__device__ __forceinline__ long parent(long fv, int n0, int n1, int n2) {
  const long bb = fv / ((long)n0 * n1 * n2), l = fv - bb * n0 * n1 * n2;
  const int i = (int)(l / ((long)n1 * n2)), j = (int)((l / n2) % n1), k = (int)(l % n2);
  return bb * ((long)n0 * n1 * n2 / 8) + ((long)(i >> 1) * (n1 >> 1) + (j >> 1)) * (n2 >> 1) + (k >> 1);
}

// out[coarse][c] = mean of the 8 children (n*c = coarse grid)
__global__ void k_pool(const bf16* __restrict__ in, long Vc, int C, int n0c, int n1c, int n2c, bf16* __restrict__ out) {
  const long n = Vc * C;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
    const long cv = idx / C;
    const int c = (int)(idx - cv * C);
    float s = 0.f;
#pragma unroll
    for (int a = 0; a < 8; ++a) s += __bfloat162float(in[child(cv, a, n0c, n1c, n2c) * C + c]);
    out[idx] = __float2bfloat16_rn(0.125f * s);
  }
}

// c[v] = (a[parent(v)] (Ca channels), s[v] (Cb channels)) on the fine grid n*
__global__ void k_up_concat(const bf16* __restrict__ a, int Ca, const bf16* __restrict__ s, int Cb, long V, int n0,
                            int n1, int n2, bf16* __restrict__ c) {
  const int C = Ca + Cb;
  const long n = V * C;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
    const long v = idx / C;
    const int ch = (int)(idx - v * C);
    c[idx] = ch < Ca ? a[parent(v, n0, n1, n2) * Ca + ch] : s[v * Cb + ch - Ca];
  }
}

// da[coarse][c] = sum over the 8 children of dc[child][c] (first Ca channels of a row of Cc)
__global__ void k_up_bwd(const float* __restrict__ dc, int Cc, int Ca, long Vc, int n0c, int n1c, int n2c,
                         float* __restrict__ da) {
  const long n = Vc * Ca;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
    const long cv = idx / Ca;
    const int c = (int)(idx - cv * Ca);
    float s = 0.f;
#pragma unroll
    for (int a = 0; a < 8; ++a) s += dc[child(cv, a, n0c, n1c, n2c) * Cc + c];
    da[idx] = s;
  }
}

// G[v][c] = bf16((a[v][c] > 0) * (d[v * ds + doff + c] + p[parent(v)][c] / 8)), p optional (average-pool gradient)
__global__ void k_mask(const bf16* __restrict__ a, const float* __restrict__ d, int ds, int doff,
                       const float* __restrict__ p, long V, int C, int n0, int n1, int n2, bf16* __restrict__ G) {
  const long n = V * C;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
    const long v = idx / C;
    const int c = (int)(idx - v * C);
    float g = d[v * ds + doff + c];
    if (p) g += 0.125f * p[parent(v, n0, n1, n2) * C + c];
    G[idx] = __float2bfloat16_rn(__bfloat162float(a[idx]) > 0.f ? g : 0.f);
  }
}

// loss partials sum_v w (y - t)^2 and G = 2 w (y - t) / 18 (channels 18..cg-1 zero)
__global__ void k_loss(const float* __restrict__ y, const float* __restrict__ t, const float* __restrict__ w, long V,
                       int cg, bf16* __restrict__ G, double* __restrict__ part) {
  __shared__ double red[32];
  double acc = 0.0;
  for (long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < V; v += (long)gridDim.x * blockDim.x) {
    const float wv = w[v];
    for (int c = 0; c < cg; ++c) {
      float gv = 0.f;
      if (c < kOut) {
        const float d = y[v * kOut + c] - t[v * kOut + c];
        acc += (double)wv * d * d;
        gv = 2.f * wv * d / kOut;
      }
      G[v * cg + c] = __float2bfloat16_rn(gv);
    }
  }
  double s[1] = {acc};
  block_sum<1>(s, red);
  if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}

// Adam (Kingma & Ba 2015) with bias corrections c1 = 1 / (1 - b1^t), c2 = 1 / (1 - b2^t)
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       long n, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  }
}

// BF16 copies of one layer's FP32 weights W [t][cout][cin]: wf [t][nf][cinp] (forward, rows = co) and
// wb [t][nb][nf] (backward-data, rows = ci), zero-padded
__global__ void k_pack(const float* __restrict__ W, int ntaps, int cout, int cin, int nf, int cinp, int nbk,
                       bf16* __restrict__ wf, bf16* __restrict__ wb) {
  const long nF = (long)ntaps * nf * cinp, nB = wb ? (long)ntaps * nbk * nf : 0;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < nF + nB; idx += (long)gridDim.x * blockDim.x) {
    if (idx < nF) {
      const int ci = (int)(idx % cinp), co = (int)((idx / cinp) % nf), t = (int)(idx / ((long)cinp * nf));
      wf[idx] = __float2bfloat16_rn(co < cout && ci < cin ? W[((long)t * cout + co) * cin + ci] : 0.f);
    } else {
      const long j = idx - nF;
      const int co = (int)(j % nf), ci = (int)((j / nf) % nbk), t = (int)(j / ((long)nf * nbk));
      wb[j] = __float2bfloat16_rn(co < cout && ci < cin ? W[((long)t * cout + co) * cin + ci] : 0.f);
    }
  }
}

// ---- host --------------------------------------------------------------------------------------------------------
struct Layer {
  int cin, cout, ntaps, relu;
  int cinp;  // stored input channels (multiple of 8)
  int nf;    // forward MMA N = output channels padded to 16 (= channels of this layer's G)
  int nbk;   // backward-data MMA N = input channels padded to 16
  long woff, boff;
  bf16* wf = nullptr;
  bf16* wb = nullptr;
};

inline int up16(int c) { return (c + 15) / 16 * 16; }
inline unsigned grid_for(long n, int nt = 256) { return (unsigned)std::min<long>((n + nt - 1) / nt, 148L * 16); }

template <int NPAD>
int conv_npad(const ConvArgs& a, cudaStream_t st) {
  const long total = (long)a.nb * a.n0 * a.n1 * a.n2;
  const size_t smem = 1024 + kStages * (kStageA + NPAD * 128);
  NLF_CUDA_TRY(raise_dyn_smem(k_conv_tc<NPAD>, (int)smem));
  k_conv_tc<NPAD><<<(unsigned)((total + 127) / 128), 128, smem, st>>>(a);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}
template <int NPAD>
int dw_npad(const DwArgs& a, int mtiles, int nchunk, cudaStream_t st) {
  const size_t smem = 1024 + kStages * (kStageA + NPAD * 128);
  NLF_CUDA_TRY(raise_dyn_smem(k_dw_tc<NPAD>, (int)smem));
  k_dw_tc<NPAD><<<dim3(mtiles, nchunk), 128, smem, st>>>(a);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}

int launch_conv(int npad, const ConvArgs& a, cudaStream_t st) {
  ProfScope ps_(PK_UNET_CONV, st);
  switch (npad) {
    case 16: return conv_npad<16>(a, st);
    case 32: return conv_npad<32>(a, st);
    case 48: return conv_npad<48>(a, st);
    case 64: return conv_npad<64>(a, st);
    case 80: return conv_npad<80>(a, st);
    case 96: return conv_npad<96>(a, st);
    case 112: return conv_npad<112>(a, st);
    case 128: return conv_npad<128>(a, st);
  }
  set_error("unet: unsupported channel padding %d", npad);
  return NLF_EBADARG;
}
int launch_dw(int npad, const DwArgs& a, int mtiles, int nchunk, cudaStream_t st) {
  ProfScope ps_(PK_UNET_WGRAD, st);
  switch (npad) {
    case 16: return dw_npad<16>(a, mtiles, nchunk, st);
    case 32: return dw_npad<32>(a, mtiles, nchunk, st);
    case 48: return dw_npad<48>(a, mtiles, nchunk, st);
    case 64: return dw_npad<64>(a, mtiles, nchunk, st);
    case 80: return dw_npad<80>(a, mtiles, nchunk, st);
    case 96: return dw_npad<96>(a, mtiles, nchunk, st);
    case 112: return dw_npad<112>(a, mtiles, nchunk, st);
    case 128: return dw_npad<128>(a, mtiles, nchunk, st);
  }
  set_error("unet: unsupported channel padding %d", npad);
  return NLF_EBADARG;
}

struct Arena {
  char* base;
  size_t off = 0;
  explicit Arena(void* b) : base((char*)b) {}
  template <typename T>
  T* take(size_t count) {
    off = (off + 255) & ~(size_t)255;
    T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off += count * sizeof(T);
    return p;
  }
};

// activations and gradients of one (nb, n0, n1, n2) batch
struct Acts {
  bf16 *x0, *a[10], *p1, *p2, *c1, *c2;
  float* y;
  bf16* G[11];
  float *dA10, *dA9, *dC2, *dA8, *dA7, *dC1, *dA6, *dA5, *dP2, *dA3, *dP1, *dA1;
  float *part, *cpart;
  double* lpart;
};

}  // namespace unet
}  // namespace nlf

using namespace nlf;
using namespace nlf::unet;

struct nlf_unet {
  int w[3];
  long nparam = 0;
  Layer L[11];
  float *params = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
  bf16* wbuf = nullptr;
  int step = 0;
  bool packed = false;
  DevBuf ws;
  int* err = nullptr;
  size_t part_cap = 0;
};

namespace {

constexpr int kLossBlocks = 256;
constexpr int kColBlocks = 64;

bool dev_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// splitmix64 + Box-Muller: seeded standard normals for the He initialisation
struct Rng {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
  double normal() {
    const double u1 = uniform(), u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

// the carve of Acts for a batch; returns the bytes needed (base == nullptr: measure only)
size_t carve(nlf_unet* u, void* base, int nb, int n0, int n1, int n2, Acts& A) {
  Arena R(base);
  const long V0 = (long)nb * n0 * n1 * n2, V1 = V0 / 8, V2 = V0 / 64;
  const int w0 = u->w[0], w1 = u->w[1], w2 = u->w[2];
  A.x0 = R.take<bf16>(V0 * 8);
  const long lv[10] = {V0, V0, V1, V1, V2, V2, V1, V1, V0, V0};
  for (int k = 0; k < 10; ++k) A.a[k] = R.take<bf16>(lv[k] * u->L[k].cout);
  A.p1 = R.take<bf16>(V1 * w0);
  A.p2 = R.take<bf16>(V2 * w1);
  A.c1 = R.take<bf16>(V1 * (w2 + w1));
  A.c2 = R.take<bf16>(V0 * (w1 + w0));
  A.y = R.take<float>(V0 * kOut);
  const long gv[11] = {V0, V0, V1, V1, V2, V2, V1, V1, V0, V0, V0};
  for (int k = 0; k < 11; ++k) A.G[k] = R.take<bf16>(gv[k] * u->L[k].nf);
  A.dA10 = R.take<float>(V0 * w0);
  A.dA9 = R.take<float>(V0 * w0);
  A.dC2 = R.take<float>(V0 * (w1 + w0));
  A.dA8 = R.take<float>(V1 * w1);
  A.dA7 = R.take<float>(V1 * w1);
  A.dC1 = R.take<float>(V1 * (w2 + w1));
  A.dA6 = R.take<float>(V2 * w2);
  A.dA5 = R.take<float>(V2 * w2);
  A.dP2 = R.take<float>(V2 * w1);
  A.dA3 = R.take<float>(V1 * w1);
  A.dP1 = R.take<float>(V1 * w0);
  A.dA1 = R.take<float>(V0 * w0);
  A.part = R.take<float>(u->part_cap);
  A.cpart = R.take<float>((size_t)kColBlocks * 128);
  A.lpart = R.take<double>(kLossBlocks);
  return R.off;
}

// weight-gradient partial layout of one layer: m-tiles x chunks
void dw_plan(const Layer& l, long total, int& mtiles, int& nchunk, long& vpc) {
  const int rows = l.ntaps * l.cinp;
  mtiles = (rows + 127) / 128;
  long want = std::max<long>(1, 600 / mtiles);
  want = std::min<long>(want, (total + 63) / 64);
  vpc = ((total + want - 1) / want + 63) / 64 * 64;
  nchunk = (int)((total + vpc - 1) / vpc);
}

int check_shape(nlf_unet* u, int nb, int n0, int n1, int n2) {
  if (!u || nb < 1 || n0 < 4 || n1 < 4 || n2 < 4 || n0 % 4 || n1 % 4 || n2 % 4) {
    set_error("unet: the grid must be at least 4 and divisible by 4 along every axis (got %d x %d x %d, batch %d)",
              n0, n1, n2, nb);
    return NLF_EBADARG;
  }
  return NLF_OK;
}

int prepare(nlf_unet* u, int nb, int n0, int n1, int n2, Acts& A, cudaStream_t st) {
  const long V0 = (long)nb * n0 * n1 * n2;
  const int level[11] = {0, 0, 1, 1, 2, 2, 1, 1, 0, 0, 0};
  size_t cap = 0;
  for (int k = 0; k < 11; ++k) {
    int mt, nc;
    long vpc;
    dw_plan(u->L[k], V0 >> (3 * level[k]), mt, nc, vpc);
    cap = std::max(cap, (size_t)nc * mt * 128 * u->L[k].nf);
  }
  u->part_cap = cap;
  const size_t need = carve(u, nullptr, nb, n0, n1, n2, A);
  NLF_TRY(u->ws.reserve(need));
  carve(u, u->ws.ptr, nb, n0, n1, n2, A);
  if (!u->packed) {
    for (Layer& l : u->L) {
      const long n = (long)l.ntaps * l.nf * l.cinp + (long)l.ntaps * l.nbk * l.nf;
      k_pack<<<grid_for(n), 256, 0, st>>>(u->params + l.woff, l.ntaps, l.cout, l.cin, l.nf, l.cinp, l.nbk, l.wf,
                                          l.wb);
      NLF_CHECK_LAUNCH();
    }
    u->packed = true;
  }
  NLF_CUDA_TRY(cudaMemsetAsync(u->err, 0, sizeof(int), st));
  return NLF_OK;
}

ConvArgs conv_args(nlf_unet* u, const Layer& l, const bf16* x, void* y, int nb, int n0, int n1, int n2, bool fwd) {
  ConvArgs a;
  a.x = x;
  a.y = y;
  a.nb = nb;
  a.n0 = n0;
  a.n1 = n1;
  a.n2 = n2;
  a.ntaps = l.ntaps;
  a.err = u->err;
  if (fwd) {
    a.w = l.wf;
    a.bias = u->params + l.boff;
    a.cin = l.cinp;
    a.cout = l.cout;
    a.ystride = l.ntaps == 1 ? kOut : l.cout;
    a.sign = 1;
    a.relu = l.relu;
    a.out_f32 = l.relu ? 0 : 1;
  } else {
    a.w = l.wb;
    a.bias = nullptr;
    a.cin = l.nf;
    a.cout = l.cin;
    a.ystride = l.cin;
    a.sign = -1;
    a.relu = 0;
    a.out_f32 = 1;
  }
  return a;
}

int forward(nlf_unet* u, const Acts& A, const float* rho, int nb, int n0, int n1, int n2, cudaStream_t st) {
  const long V0 = (long)nb * n0 * n1 * n2, V1 = V0 / 8, V2 = V0 / 64;
  const int w0 = u->w[0], w1 = u->w[1], w2 = u->w[2];
  const int m0 = n0 / 2, m1 = n1 / 2, m2 = n2 / 2;
  {
    ProfScope ps_(PK_UNET_MISC, st);
    k_input<<<grid_for(V0), 256, 0, st>>>(rho, V0, A.x0);
    NLF_CHECK_LAUNCH();
  }
  auto conv = [&](int k, const bf16* x, void* y, int a0, int a1, int a2) {
    return launch_conv(u->L[k].nf, conv_args(u, u->L[k], x, y, nb, a0, a1, a2, true), st);
  };
  NLF_TRY(conv(0, A.x0, A.a[0], n0, n1, n2));
  NLF_TRY(conv(1, A.a[0], A.a[1], n0, n1, n2));
  {
    ProfScope ps_(PK_UNET_MISC, st);
    k_pool<<<grid_for(V1 * w0), 256, 0, st>>>(A.a[1], V1, w0, m0, m1, m2, A.p1);
    NLF_CHECK_LAUNCH();
  }
  NLF_TRY(conv(2, A.p1, A.a[2], m0, m1, m2));
  NLF_TRY(conv(3, A.a[2], A.a[3], m0, m1, m2));
  {
    ProfScope ps_(PK_UNET_MISC, st);
    k_pool<<<grid_for(V2 * w1), 256, 0, st>>>(A.a[3], V2, w1, m0 / 2, m1 / 2, m2 / 2, A.p2);
    NLF_CHECK_LAUNCH();
  }
  NLF_TRY(conv(4, A.p2, A.a[4], m0 / 2, m1 / 2, m2 / 2));
  NLF_TRY(conv(5, A.a[4], A.a[5], m0 / 2, m1 / 2, m2 / 2));
  {
    ProfScope ps_(PK_UNET_MISC, st);
    k_up_concat<<<grid_for(V1 * (w2 + w1)), 256, 0, st>>>(A.a[5], w2, A.a[3], w1, V1, m0, m1, m2, A.c1);
    NLF_CHECK_LAUNCH();
  }
  NLF_TRY(conv(6, A.c1, A.a[6], m0, m1, m2));
  NLF_TRY(conv(7, A.a[6], A.a[7], m0, m1, m2));
  {
    ProfScope ps_(PK_UNET_MISC, st);
    k_up_concat<<<grid_for(V0 * (w1 + w0)), 256, 0, st>>>(A.a[7], w1, A.a[1], w0, V0, n0, n1, n2, A.c2);
    NLF_CHECK_LAUNCH();
  }
  NLF_TRY(conv(8, A.c2, A.a[8], n0, n1, n2));
  NLF_TRY(conv(9, A.a[8], A.a[9], n0, n1, n2));
  NLF_TRY(conv(10, A.a[9], A.y, n0, n1, n2));
  return NLF_OK;
}

// dW, db of layer k from its input x (level grid a*) and its G
int wgrad(nlf_unet* u, const Acts& A, int k, const bf16* x, int nb, int a0, int a1, int a2, cudaStream_t st) {
  const Layer& l = u->L[k];
  const long total = (long)nb * a0 * a1 * a2;
  int mt, nc;
  long vpc;
  dw_plan(l, total, mt, nc, vpc);
  DwArgs d;
  d.x = x;
  d.g = A.G[k];
  d.part = A.part;
  d.nb = nb;
  d.n0 = a0;
  d.n1 = a1;
  d.n2 = a2;
  d.cin = l.cinp;
  d.ntaps = l.ntaps;
  d.rows = l.ntaps * l.cinp;
  d.rows_pad = mt * 128;
  d.vpc = vpc;
  d.err = u->err;
  NLF_TRY(launch_dw(l.nf, d, mt, nc, st));
  ProfScope ps_(PK_UNET_MISC, st);
  const long nw = (long)l.ntaps * l.cout * l.cin;
  k_dw_reduce<<<grid_for(nw), 256, 0, st>>>(A.part, nc, mt * 128, l.nf, l.ntaps, l.cinp, l.cin, l.cout,
                                            u->grad + l.woff);
  NLF_CHECK_LAUNCH();
  k_colsum_part<<<kColBlocks, 256, 0, st>>>(A.G[k], total, l.nf, A.cpart);
  NLF_CHECK_LAUNCH();
  k_colsum_fin<<<1, 128, 0, st>>>(A.cpart, kColBlocks, l.nf, l.cout, u->grad + l.boff);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}

int bwd_data(nlf_unet* u, int k, const bf16* G, float* dx, int nb, int a0, int a1, int a2, cudaStream_t st) {
  return launch_conv(u->L[k].nbk, conv_args(u, u->L[k], G, dx, nb, a0, a1, a2, false), st);
}

int mask(const bf16* a, const float* d, int ds, int doff, const float* p, long V, int C, int a0, int a1, int a2,
         bf16* G, cudaStream_t st) {
  ProfScope ps_(PK_UNET_MISC, st);
  k_mask<<<grid_for(V * C), 256, 0, st>>>(a, d, ds, doff, p, V, C, a0, a1, a2, G);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}

int backward(nlf_unet* u, const Acts& A, int nb, int n0, int n1, int n2, cudaStream_t st) {
  const long V0 = (long)nb * n0 * n1 * n2, V1 = V0 / 8, V2 = V0 / 64;
  const int w0 = u->w[0], w1 = u->w[1], w2 = u->w[2];
  const int m0 = n0 / 2, m1 = n1 / 2, m2 = n2 / 2, q0 = m0 / 2, q1 = m1 / 2, q2 = m2 / 2;
  // G[10] (the loss gradient) is in place
  NLF_TRY(wgrad(u, A, 10, A.a[9], nb, n0, n1, n2, st));
  NLF_TRY(bwd_data(u, 10, A.G[10], A.dA10, nb, n0, n1, n2, st));
  NLF_TRY(mask(A.a[9], A.dA10, w0, 0, nullptr, V0, w0, n0, n1, n2, A.G[9], st));
  NLF_TRY(wgrad(u, A, 9, A.a[8], nb, n0, n1, n2, st));
  NLF_TRY(bwd_data(u, 9, A.G[9], A.dA9, nb, n0, n1, n2, st));
  NLF_TRY(mask(A.a[8], A.dA9, w0, 0, nullptr, V0, w0, n0, n1, n2, A.G[8], st));
  NLF_TRY(wgrad(u, A, 8, A.c2, nb, n0, n1, n2, st));
  NLF_TRY(bwd_data(u, 8, A.G[8], A.dC2, nb, n0, n1, n2, st));
  {
    ProfScope ps_(PK_UNET_MISC, st);
    k_up_bwd<<<grid_for(V1 * w1), 256, 0, st>>>(A.dC2, w1 + w0, w1, V1, m0, m1, m2, A.dA8);
    NLF_CHECK_LAUNCH();
  }
  NLF_TRY(mask(A.a[7], A.dA8, w1, 0, nullptr, V1, w1, m0, m1, m2, A.G[7], st));
  NLF_TRY(wgrad(u, A, 7, A.a[6], nb, m0, m1, m2, st));
  NLF_TRY(bwd_data(u, 7, A.G[7], A.dA7, nb, m0, m1, m2, st));
  NLF_TRY(mask(A.a[6], A.dA7, w1, 0, nullptr, V1, w1, m0, m1, m2, A.G[6], st));
  NLF_TRY(wgrad(u, A, 6, A.c1, nb, m0, m1, m2, st));
  NLF_TRY(bwd_data(u, 6, A.G[6], A.dC1, nb, m0, m1, m2, st));
  {
    ProfScope ps_(PK_UNET_MISC, st);
    k_up_bwd<<<grid_for(V2 * w2), 256, 0, st>>>(A.dC1, w2 + w1, w2, V2, q0, q1, q2, A.dA6);
    NLF_CHECK_LAUNCH();
  }
  NLF_TRY(mask(A.a[5], A.dA6, w2, 0, nullptr, V2, w2, q0, q1, q2, A.G[5], st));
  NLF_TRY(wgrad(u, A, 5, A.a[4], nb, q0, q1, q2, st));
  NLF_TRY(bwd_data(u, 5, A.G[5], A.dA5, nb, q0, q1, q2, st));
  NLF_TRY(mask(A.a[4], A.dA5, w2, 0, nullptr, V2, w2, q0, q1, q2, A.G[4], st));
  NLF_TRY(wgrad(u, A, 4, A.p2, nb, q0, q1, q2, st));
  NLF_TRY(bwd_data(u, 4, A.G[4], A.dP2, nb, q0, q1, q2, st));
  NLF_TRY(mask(A.a[3], A.dC1, w2 + w1, w2, A.dP2, V1, w1, m0, m1, m2, A.G[3], st));
  NLF_TRY(wgrad(u, A, 3, A.a[2], nb, m0, m1, m2, st));
  NLF_TRY(bwd_data(u, 3, A.G[3], A.dA3, nb, m0, m1, m2, st));
  NLF_TRY(mask(A.a[2], A.dA3, w1, 0, nullptr, V1, w1, m0, m1, m2, A.G[2], st));
  NLF_TRY(wgrad(u, A, 2, A.p1, nb, m0, m1, m2, st));
  NLF_TRY(bwd_data(u, 2, A.G[2], A.dP1, nb, m0, m1, m2, st));
  NLF_TRY(mask(A.a[1], A.dC2, w1 + w0, w1, A.dP1, V0, w0, n0, n1, n2, A.G[1], st));
  NLF_TRY(wgrad(u, A, 1, A.a[0], nb, n0, n1, n2, st));
  NLF_TRY(bwd_data(u, 1, A.G[1], A.dA1, nb, n0, n1, n2, st));
  NLF_TRY(mask(A.a[0], A.dA1, w0, 0, nullptr, V0, w0, n0, n1, n2, A.G[0], st));
  NLF_TRY(wgrad(u, A, 0, A.x0, nb, n0, n1, n2, st));
  return NLF_OK;
}

int finish(nlf_unet* u, cudaStream_t st) {
  int e = 0;
  NLF_CUDA_TRY(cudaMemcpyAsync(&e, u->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  if (e) {
    set_error("unet: a tensor-core pipeline wait timed out");
    return NLF_ETIMEOUT;
  }
  return NLF_OK;
}

}  // namespace

extern "C" {

NLF_API int nlf_unet_create(nlf_unet** out, int w0, int w1, int w2, unsigned long long seed) {
  if (!out || w0 < 16 || w1 < 16 || w2 < 16 || w0 % 16 || w1 % 16 || w2 % 16 || w2 + w1 > 128 || w1 + w0 > 128) {
    set_error("nlf_unet_create: widths must be multiples of 16 with w2 + w1 <= 128 and w1 + w0 <= 128");
    return NLF_EBADARG;
  }
  *out = nullptr;
  nlf_unet* u = new nlf_unet();
  u->w[0] = w0;
  u->w[1] = w1;
  u->w[2] = w2;
  const int spec[11][4] = {{1, w0, 27, 1},  {w0, w0, 27, 1},      {w0, w1, 27, 1}, {w1, w1, 27, 1},
                           {w1, w2, 27, 1}, {w2, w2, 27, 1},      {w2 + w1, w1, 27, 1}, {w1, w1, 27, 1},
                           {w1 + w0, w0, 27, 1}, {w0, w0, 27, 1}, {w0, kOut, 1, 0}};
  long off = 0, wsz = 0;
  for (int k = 0; k < 11; ++k) {
    Layer& l = u->L[k];
    l.cin = spec[k][0];
    l.cout = spec[k][1];
    l.ntaps = spec[k][2];
    l.relu = spec[k][3];
    l.cinp = (l.cin + 7) / 8 * 8;
    l.nf = up16(l.cout);
    l.nbk = up16(l.cin);
    l.woff = off;
    off += (long)l.ntaps * l.cout * l.cin;
    l.boff = off;
    off += l.cout;
    wsz += (long)l.ntaps * l.nf * l.cinp + (k ? (long)l.ntaps * l.nbk * l.nf : 0) + 128;
  }
  u->nparam = off;
  std::vector<float> h(off, 0.f);
  Rng rng{seed};
  for (const Layer& l : u->L) {
    const double std = l.relu ? std::sqrt(2.0 / (l.cin * l.ntaps)) : 1e-2 / std::sqrt((double)l.cin * l.ntaps);
    for (long i = 0; i < (long)l.ntaps * l.cout * l.cin; ++i) h[l.woff + i] = (float)(rng.normal() * std);
  }
  cudaError_t e = cudaMalloc(&u->params, 4 * off * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&u->wbuf, wsz * sizeof(bf16));
  if (e == cudaSuccess) e = cudaMalloc(&u->err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpy(u->params, h.data(), off * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(u->params + off, 0, 3 * off * sizeof(float));
  if (e != cudaSuccess) {
    set_error("nlf_unet_create: %s", cudaGetErrorString(e));
    nlf_unet_destroy(u);
    return NLF_ECUDA;
  }
  u->grad = u->params + off;
  u->m = u->params + 2 * off;
  u->v = u->params + 3 * off;
  bf16* p = u->wbuf;
  for (int k = 0; k < 11; ++k) {
    Layer& l = u->L[k];
    l.wf = p;
    p += ((long)l.ntaps * l.nf * l.cinp + 63) / 64 * 64;
    if (k) {
      l.wb = p;
      p += ((long)l.ntaps * l.nbk * l.nf + 63) / 64 * 64;
    }
  }
  *out = u;
  return NLF_OK;
}

NLF_API int nlf_unet_destroy(nlf_unet* u) {
  if (!u) return NLF_OK;
  cudaFree(u->params);
  cudaFree(u->wbuf);
  cudaFree(u->err);
  u->ws.release();
  delete u;
  return NLF_OK;
}

NLF_API long long nlf_unet_param_count(const nlf_unet* u) { return u ? u->nparam : 0; }

NLF_API int nlf_unet_get_params(nlf_unet* u, float* out, void* stream) {
  if (!u || !out) {
    set_error("nlf_unet_get_params: bad arguments");
    return NLF_EBADARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  NLF_CUDA_TRY(cudaMemcpyAsync(out, u->params, u->nparam * sizeof(float),
                               dev_ptr(out) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  return NLF_OK;
}

NLF_API int nlf_unet_set_params(nlf_unet* u, const float* in, void* stream) {
  if (!u || !in) {
    set_error("nlf_unet_set_params: bad arguments");
    return NLF_EBADARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  NLF_CUDA_TRY(cudaMemcpyAsync(u->params, in, u->nparam * sizeof(float),
                               dev_ptr(in) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  NLF_CUDA_TRY(cudaMemsetAsync(u->m, 0, 2 * u->nparam * sizeof(float), st));
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  u->step = 0;
  u->packed = false;
  return NLF_OK;
}

NLF_API int nlf_unet_forward(nlf_unet* u, int nb, int nx, int ny, int nz, const float* rho, float* y, void* stream) {
  NLF_TRY(check_shape(u, nb, nx, ny, nz));
  if (!dev_ptr(rho) || !dev_ptr(y)) {
    set_error("nlf_unet_forward: rho and y must be device pointers");
    return NLF_EBADARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  Acts A;
  NLF_TRY(prepare(u, nb, nx, ny, nz, A, st));
  NLF_TRY(forward(u, A, rho, nb, nx, ny, nz, st));
  NLF_CUDA_TRY(cudaMemcpyAsync(y, A.y, (size_t)nb * nx * ny * nz * kOut * sizeof(float), cudaMemcpyDeviceToDevice,
                               st));
  return finish(u, st);
}

NLF_API int nlf_unet_backward(nlf_unet* u, int nb, int nx, int ny, int nz, const float* rho, const float* target,
                              const float* weight, double* loss, float* grad, void* stream) {
  NLF_TRY(check_shape(u, nb, nx, ny, nz));
  if (!dev_ptr(rho) || !dev_ptr(target) || !dev_ptr(weight)) {
    set_error("nlf_unet_backward: rho, target and weight must be device pointers");
    return NLF_EBADARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  Acts A;
  NLF_TRY(prepare(u, nb, nx, ny, nz, A, st));
  NLF_TRY(forward(u, A, rho, nb, nx, ny, nz, st));
  const long V0 = (long)nb * nx * ny * nz;
  {
    ProfScope ps_(PK_UNET_MISC, st);
    k_loss<<<kLossBlocks, 256, 0, st>>>(A.y, target, weight, V0, u->L[10].nf, A.G[10], A.lpart);
    NLF_CHECK_LAUNCH();
  }
  NLF_TRY(backward(u, A, nb, nx, ny, nz, st));
  std::vector<double> lp(kLossBlocks);
  NLF_CUDA_TRY(cudaMemcpyAsync(lp.data(), A.lpart, kLossBlocks * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (grad)
    NLF_CUDA_TRY(cudaMemcpyAsync(grad, u->grad, u->nparam * sizeof(float),
                                 dev_ptr(grad) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
  NLF_TRY(finish(u, st));
  if (loss) {
    double s = 0.0;
    for (double v : lp) s += v;
    *loss = s / kOut;
  }
  return NLF_OK;
}

NLF_API int nlf_unet_adam_step(nlf_unet* u, double lr, double beta1, double beta2, double eps, void* stream) {
  if (!u || !(lr >= 0) || !(beta1 >= 0 && beta1 < 1) || !(beta2 >= 0 && beta2 < 1) || !(eps > 0)) {
    set_error("nlf_unet_adam_step: bad arguments");
    return NLF_EBADARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  u->step += 1;
  const float c1 = (float)(1.0 / (1.0 - std::pow(beta1, u->step))), c2 = (float)(1.0 / (1.0 - std::pow(beta2, u->step)));
  {
    ProfScope ps_(PK_UNET_MISC, st);
    k_adam<<<grid_for(u->nparam), 256, 0, st>>>(u->params, u->grad, u->m, u->v, u->nparam, (float)lr, (float)beta1,
                                                 (float)beta2, (float)eps, c1, c2);
    NLF_CHECK_LAUNCH();
  }
  u->packed = false;
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  return NLF_OK;
}

}  // extern "C"
