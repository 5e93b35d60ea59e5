// FFT preconditioner of the periodic corrector solve: z = irfftn(Kinv(k) rfftn(r)) (nlfiber/linear.py:154-170),
// optionally with node scaling w = S^-0.47 on both sides (z = w .* irfftn(Kinv rfftn(w .* r))).
//
// Three passes over a half spectrum stored [vec][comp][ky][x][kz], kz in [0, nz/2]:
//   A  one CTA per (vec, comp, x-plane): real plane -> 2D transform along z (real, packed as a half-length
//      complex FFT) and y, in shared memory; writes (ky, x, kz) rows.
//   B  one CTA per (vec, ky, kz-chunk): the three components' x-lines -> forward FFT along x, 3x3 Kinv
//      multiply per wavenumber, inverse FFT along x, in shared memory.
//   C  one CTA per (vec, comp, x-plane): inverse y then inverse real z, scale by 1/N (and w), write the real
//      field and the reduction partials the PCG needs (sum z, (r, z), sum r, (r, r)).
// Power-of-two lines use an iterative radix-2 FFT; other lengths (small test grids) a direct DFT.
// Kinv is the reference's symbol: the FFT of the unit-stiffness impulse response, which is the real symmetric
// sum over the 27 stencil blocks W_d cos(k.d); K(0) = I; Kinv = inv(K + 1e-12 |tr K| I); Kinv(0) = 0.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <type_traits>
#include "nlf_internal.h"
#include "nlf_prof.cuh"

namespace nlf {

// r-point DFT (r in {2, 4, 8}) of a[0..r) in registers; INV selects e^{+2 pi i jk/r}.
template <typename T, bool INV>
__device__ __forceinline__ void dft4(cplx<T>& a0, cplx<T>& a1, cplx<T>& a2, cplx<T>& a3) {
  const cplx<T> s0 = cadd(a0, a2), d0 = csub(a0, a2), s1 = cadd(a1, a3), d1 = csub(a1, a3);
  // forward: X1 = d0 - i d1, X3 = d0 + i d1; inverse swaps them
  const cplx<T> id1{-d1.y, d1.x};
  a0 = cadd(s0, s1);
  a2 = csub(s0, s1);
  a1 = INV ? cadd(d0, id1) : csub(d0, id1);
  a3 = INV ? csub(d0, id1) : cadd(d0, id1);
}

template <typename T, bool INV>
__device__ __forceinline__ void dft_small(cplx<T> (&a)[8], int r) {
  if (r == 2) {
    const cplx<T> t = csub(a[0], a[1]);
    a[0] = cadd(a[0], a[1]);
    a[1] = t;
  } else if (r == 4) {
    dft4<T, INV>(a[0], a[1], a[2], a[3]);
  } else {
    // split into even / odd 4-point DFTs, then X_k = E_k + W^k O_k, X_{k+4} = E_k - W^k O_k
    cplx<T> e0 = a[0], e1 = a[2], e2 = a[4], e3 = a[6], o0 = a[1], o1 = a[3], o2 = a[5], o3 = a[7];
    dft4<T, INV>(e0, e1, e2, e3);
    dft4<T, INV>(o0, o1, o2, o3);
    const T c = T(0.70710678118654752440084436210485);
    // W^1 o1, W^2 o2, W^3 o3 with W = e^{-+2 pi i / 8}
    cplx<T> w1, w2, w3;
    if (!INV) {
      w1 = {c * (o1.x + o1.y), c * (o1.y - o1.x)};
      w2 = {o2.y, -o2.x};
      w3 = {c * (o3.y - o3.x), -c * (o3.x + o3.y)};
    } else {
      w1 = {c * (o1.x - o1.y), c * (o1.x + o1.y)};
      w2 = {-o2.y, o2.x};
      w3 = {-c * (o3.x + o3.y), c * (o3.x - o3.y)};
    }
    a[0] = cadd(e0, o0);
    a[4] = csub(e0, o0);
    a[1] = cadd(e1, w1);
    a[5] = csub(e1, w1);
    a[2] = cadd(e2, w2);
    a[6] = csub(e2, w2);
    a[3] = cadd(e3, w3);
    a[7] = csub(e3, w3);
  }
}

// One Stockham autosort stage of radix r over `nlines` lines (src -> dst, same layout). Ns is the product of the
// radices of the previous stages. Butterfly j reads x[j + t n/r], twiddles by e^{-+2 pi i t k/(Ns r)} with
// k = j mod Ns, and writes the r outputs to (j / Ns) Ns r + k + t Ns.
template <typename T, bool INV>
__device__ void stockham_stage(const cplx<T>* src, cplx<T>* dst, int n, int r, int Ns, int nlines, int inner_n,
                               int outer_stride, int inner_stride, int es, const cplx<T>* __restrict__ tw) {
  const int nr = n / r, tstride = n / (Ns * r), total = nlines * nr;
  const int lgNs = ilog2(Ns);
  for (int wi = threadIdx.x; wi < total; wi += blockDim.x) {
    int l, j;
    if (es == 1) {
      l = fdiv(wi, nr);
      j = wi - l * nr;
    } else {  // strided lines: neighbouring threads take neighbouring lines (contiguous in memory)
      j = fdiv(wi, nlines);
      l = wi - j * nlines;
    }
    const int lo = fdiv(l, inner_n);
    const int b = lo * outer_stride + (l - lo * inner_n) * inner_stride;
    const int k = j & (Ns - 1);
    cplx<T> a[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      if (t < r) {
        a[t] = src[b + (j + t * nr) * es];
        if (t > 0 && k > 0) {
          cplx<T> w = tw[t * k * tstride];
          if (INV) w.y = -w.y;
          a[t] = cmul(a[t], w);
        }
      }
    }
    dft_small<T, INV>(a, r);
    const int base = ((j >> lgNs) * r << lgNs) + k;
#pragma unroll
    for (int t = 0; t < 8; ++t)
      if (t < r) dst[b + (base + t * Ns) * es] = a[t];
  }
}

// Power-of-two transform by Stockham stages of radix 8/4/2 (an even number of stages when n >= 4, so the result
// ends in `buf`), ping-ponging with `scratch` (same size and layout as buf). Ends with __syncthreads().
template <typename T>
__device__ void lines_fft_stockham(cplx<T>* buf, int n, int nlines, int inner_n, int outer_stride,
                                   int inner_stride, int es, const cplx<T>* __restrict__ tw, bool inv,
                                   cplx<T>* scratch) {
  const int e = ilog2(n);
  int S = (e + 2) / 3;
  if ((S & 1) && e >= 2) ++S;
  cplx<T>* src = buf;
  cplx<T>* dst = scratch;
  int Ns = 1;
  for (int st = 0; st < S; ++st) {
    const int ex = e / S + (st < e % S ? 1 : 0);
    const int r = 1 << ex;
    if (inv)
      stockham_stage<T, true>(src, dst, n, r, Ns, nlines, inner_n, outer_stride, inner_stride, es, tw);
    else
      stockham_stage<T, false>(src, dst, n, r, Ns, nlines, inner_n, outer_stride, inner_stride, es, tw);
    __syncthreads();
    cplx<T>* t = src;
    src = dst;
    dst = t;
    Ns *= r;
  }
  if (src != buf) {  // odd stage count (n == 2): copy back
    for (int idx = threadIdx.x; idx < nlines * n; idx += blockDim.x) {
      const int l = idx / n, j = idx - l * n;
      const int b = (l / inner_n) * outer_stride + (l % inner_n) * inner_stride;
      buf[b + j * es] = src[b + j * es];
    }
    __syncthreads();
  }
}

// Transform `nlines` lines of length n in shared memory. Line l starts at
// (l / inner_n) * outer_stride + (l % inner_n) * inner_stride, elements are `es` apart. tw[k] = e^{-2 pi i k/n}.
// `scratch` (nlines * n entries) is used by non-power-of-two lengths only. Ends with __syncthreads().
template <typename T>
__device__ void lines_fft(cplx<T>* buf, int n, int nlines, int inner_n, int outer_stride, int inner_stride,
                          int es, const cplx<T>* __restrict__ tw, bool inv, cplx<T>* scratch, bool pingpong) {
  const int tid = threadIdx.x, nt = blockDim.x;
  if (n == 1) return;
  if (is_pow2(n) && pingpong) {
    lines_fft_stockham(buf, n, nlines, inner_n, outer_stride, inner_stride, es, tw, inv, scratch);
    return;
  }
  if (is_pow2(n)) {
    const int lg = ilog2(n);
    for (int idx = tid; idx < nlines * n; idx += nt) {
      const int l = idx >> lg, j = idx & (n - 1);
      const int r = (int)(__brev((unsigned)j) >> (32 - lg));
      if (j < r) {
        const int b = (l / inner_n) * outer_stride + (l % inner_n) * inner_stride;
        const cplx<T> t = buf[b + j * es];
        buf[b + j * es] = buf[b + r * es];
        buf[b + r * es] = t;
      }
    }
    __syncthreads();
    const int nh = n >> 1;
    for (int half = 1, lh = 0; half < n; half <<= 1, ++lh) {
      const int tstep = n / (2 * half);
      for (int idx = tid; idx < nlines * nh; idx += nt) {
        const int l = idx / nh, t = idx - l * nh;
        const int pos = t & (half - 1), grp = t >> lh;
        const int i0 = grp * 2 * half + pos, i1 = i0 + half;
        const int b = (l / inner_n) * outer_stride + (l % inner_n) * inner_stride;
        cplx<T> w = tw[pos * tstep];
        if (inv) w.y = -w.y;
        const cplx<T> a = buf[b + i0 * es];
        const cplx<T> c = cmul(buf[b + i1 * es], w);
        buf[b + i0 * es] = cadd(a, c);
        buf[b + i1 * es] = csub(a, c);
      }
      __syncthreads();
    }
  } else {
    for (int idx = tid; idx < nlines * n; idx += nt) {
      const int l = idx / n, j = idx - l * n;
      const int b = (l / inner_n) * outer_stride + (l % inner_n) * inner_stride;
      scratch[idx] = buf[b + j * es];
    }
    __syncthreads();
    for (int idx = tid; idx < nlines * n; idx += nt) {
      const int l = idx / n, k = idx - l * n;
      const int b = (l / inner_n) * outer_stride + (l % inner_n) * inner_stride;
      cplx<T> acc{T(0), T(0)};
      int e = 0;
      for (int j = 0; j < n; ++j) {
        cplx<T> w = tw[e];
        if (inv) w.y = -w.y;
        acc = cadd(acc, cmul(scratch[l * n + j], w));
        e += k;
        if (e >= n) e -= n;
      }
      buf[b + k * es] = acc;
    }
    __syncthreads();
  }
}

// Packed real FFT post-processing along rows of length n (even), M = n/2: Z (first M entries of each row,
// the FFT of x[2j] + i x[2j+1]) -> X_k, k = 0..M (row entries 0..M). wn[k] = e^{-2 pi i k / n}.
template <typename T>
__device__ void real_post(cplx<T>* buf, int rows, int rs, int n, const cplx<T>* __restrict__ wn) {
  const int M = n >> 1, H = M / 2 + 1;
  for (int idx = threadIdx.x; idx < rows * H; idx += blockDim.x) {
    const int row = idx / H, k = idx - row * H;
    cplx<T>* z = buf + row * rs;
    if (k == 0) {
      const cplx<T> z0 = z[0];
      z[0] = {z0.x + z0.y, T(0)};
      z[M] = {z0.x - z0.y, T(0)};
    } else if (2 * k == M) {
      z[k] = cconj(z[k]);
    } else {
      const cplx<T> a = z[k], b = z[M - k];
      // E_k = (a + conj b)/2, O_k = -i (a - conj b)/2
      const cplx<T> Ek{(a.x + b.x) * T(0.5), (a.y - b.y) * T(0.5)};
      const cplx<T> Ok{(a.y + b.y) * T(0.5), -(a.x - b.x) * T(0.5)};
      const cplx<T> Em{(b.x + a.x) * T(0.5), (b.y - a.y) * T(0.5)};
      const cplx<T> Om{(b.y + a.y) * T(0.5), -(b.x - a.x) * T(0.5)};
      z[k] = cadd(Ek, cmul(wn[k], Ok));
      z[M - k] = cadd(Em, cmul(wn[M - k], Om));
    }
  }
  __syncthreads();
}

// Inverse of real_post: X_k (k = 0..M) -> Z_k = E_k + i O_k (k < M), E_k = (X_k + conj X_{M-k})/2,
// O_k = (X_k - conj X_{M-k}) conj(wn[k]) / 2.
template <typename T>
__device__ void real_pre(cplx<T>* buf, int rows, int rs, int n, const cplx<T>* __restrict__ wn) {
  const int M = n >> 1, H = M / 2 + 1;
  for (int idx = threadIdx.x; idx < rows * H; idx += blockDim.x) {
    const int row = idx / H, k = idx - row * H;
    cplx<T>* z = buf + row * rs;
    if (k == 0) {
      // X_0 and X_M of a real signal are real; their imaginary parts are rounding and are dropped (as irfft does)
      const T a = z[0].x, b = z[M].x;
      z[0] = {(a + b) * T(0.5), (a - b) * T(0.5)};
    } else if (2 * k == M) {
      z[k] = cconj(z[k]);
    } else {
      const cplx<T> a = z[k], b = z[M - k];
      const cplx<T> Ek{(a.x + b.x) * T(0.5), (a.y - b.y) * T(0.5)};
      const cplx<T> Dk{(a.x - b.x) * T(0.5), (a.y + b.y) * T(0.5)};
      const cplx<T> Ok = cmul(Dk, cconj(wn[k]));
      const cplx<T> Em{(b.x + a.x) * T(0.5), (b.y - a.y) * T(0.5)};
      const cplx<T> Dm{(b.x - a.x) * T(0.5), (b.y + a.y) * T(0.5)};
      const cplx<T> Om = cmul(Dm, cconj(wn[M - k]));
      z[k] = {Ek.x - Ok.y, Ek.y + Ok.x};
      z[M - k] = {Em.x - Om.y, Em.y + Om.x};
    }
  }
  __syncthreads();
}

template <typename T>
struct Vec2;
template <>
struct Vec2<float> {
  using type = float2;
};
template <>
struct Vec2<double> {
  using type = double2;
};

struct FftDims {
  int n0, n1, n2, n2h, rs;  // rs: shared row stride of a (y, z) plane
  bool pp;                  // power-of-two lines ping-pong with an equal-size scratch (Stockham)
  long N, NS;
  int off0, off1, off2, off2h;
};

// Optional fusions of the PCG iteration into the passes (all pointers may be null):
//   A: r <- r - alpha (Ap - mean Ap) before the transform (written back), partials (sum r, sum r^2) per plane
//   B: Parseval partial of (w r, K0^-1 w r) = (r, z) per CTA (the half spectrum weighted 1 or 2 per kz)
//   C: partial sum z per plane (mean removal), without reading r
//   C (register-resident FP64 passes, x and p set): x <- x + alpha p, p <- z + beta p in place of writing z, for
//      the cells that ran this iteration (status bit 1), alpha and beta from vs
struct PcgFuse {
  const void* Ap;         // A: Ap of this iteration (T, same layout as r)
  const VecState* vs;     // A: alpha and mean Ap per vector; C with x/p: alpha and beta
  double* partA;          // [vec][comp][x-plane][2]
  double* partB;          // [vec][ky][chunk]
  double* partC;          // [vec][comp][x-plane]
  double* x;              // C: PCG iterate and search direction ([vec][comp][N]), FP64
  double* p;
};

// global loads issued together before their first use: enough bytes in flight per thread for HBM latency while
// keeping the plane kernels at 3 CTAs of 256 threads per SM (at most 85 registers)
template <typename T>
constexpr int batch() {
  return sizeof(T) == 8 ? 4 : 8;
}

// ---- pass A --------------------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256, 3) k_fft_a(T* __restrict__ r, const T* __restrict__ w, cplx<T>* __restrict__ spec, FftDims d, int m,
                        const cplx<T>* __restrict__ tw, const CellState* __restrict__ cs,
                        unsigned long long* __restrict__ units, int ukind, PcgFuse fu) {
  extern __shared__ unsigned char smem_raw[];
  cplx<T>* buf = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* scratch = buf + d.n1 * d.rs;
  __shared__ double red[32 * 2];
  const int x = blockIdx.x, c = blockIdx.y, vec = blockIdx.z;
  if (cs && !cs[vec / m].active) return;
  prof_count(units, ukind);
  T* rp = r + ((long)vec * 3 + c) * d.N + (long)x * d.n1 * d.n2;
  const T* wp = w ? w + (long)(vec / m) * d.N + (long)x * d.n1 * d.n2 : nullptr;
  const T* ap = fu.Ap ? static_cast<const T*>(fu.Ap) + ((long)vec * 3 + c) * d.N + (long)x * d.n1 * d.n2 : nullptr;
  T al = T(0), mu = T(0);
  if (ap) {
    al = (T)fu.vs[vec].alpha;
    mu = (T)fu.vs[vec].mean[c];
  }
  double acc[2] = {0.0, 0.0};
  constexpr int kBatch = batch<T>();
  const bool packed = (d.n2 % 2) == 0;
  if (packed) {
    const int M = d.n2 / 2, total = d.n1 * M;
    using V2 = typename Vec2<T>::type;
    V2* rp2 = reinterpret_cast<V2*>(rp);  // pair j of row y is element y M + j (N and n2 even)
    const V2* wp2 = reinterpret_cast<const V2*>(wp);
    const V2* ap2 = reinterpret_cast<const V2*>(ap);
    for (int base = threadIdx.x; base < total; base += kBatch * blockDim.x) {
      V2 rv[kBatch], av[kBatch], wv[kBatch];
#pragma unroll
      for (int u = 0; u < kBatch; ++u) {
        const int idx = base + u * blockDim.x;
        if (idx < total) {
          rv[u] = rp2[idx];
          if (ap) av[u] = ap2[idx];
          if (wp) wv[u] = wp2[idx];
        }
      }
#pragma unroll
      for (int u = 0; u < kBatch; ++u) {
        const int idx = base + u * blockDim.x;
        if (idx < total) {
          V2 v = rv[u];
          if (ap) {
            v.x -= al * (av[u].x - mu);
            v.y -= al * (av[u].y - mu);
            rp2[idx] = v;
          }
          acc[0] += (double)v.x + (double)v.y;
          acc[1] += (double)v.x * (double)v.x + (double)v.y * (double)v.y;
          if (wp) {
            v.x *= wv[u].x;
            v.y *= wv[u].y;
          }
          const int y = fdiv(idx, M), j = idx - y * M;
          buf[y * d.rs + j] = {v.x, v.y};
        }
      }
    }
    __syncthreads();
    lines_fft(buf, M, d.n1, d.n1, 0, d.rs, 1, tw + d.off2h, false, scratch, d.pp);
    real_post(buf, d.n1, d.rs, d.n2, tw + d.off2);
  } else {
    for (int idx = threadIdx.x; idx < d.n1 * d.n2; idx += blockDim.x) {
      const int y = idx / d.n2, z = idx - y * d.n2;
      T v = rp[idx];
      if (ap) {
        v -= al * (ap[idx] - mu);
        rp[idx] = v;
      }
      acc[0] += (double)v;
      acc[1] += (double)v * (double)v;
      if (wp) v *= wp[idx];
      buf[y * d.rs + z] = {v, T(0)};
    }
    __syncthreads();
    lines_fft(buf, d.n2, d.n1, d.n1, 0, d.rs, 1, tw + d.off2, false, scratch, d.pp);
  }
  // y transform on the n2h columns
  lines_fft(buf, d.n1, d.n2h, d.n2h, 0, 1, d.rs, tw + d.off1, false, scratch, d.pp);
  cplx<T>* sp = spec + ((long)vec * 3 + c) * d.NS;
#pragma unroll 4
  for (int idx = threadIdx.x; idx < d.n1 * d.n2h; idx += blockDim.x) {
    const int ky = idx / d.n2h, kz = idx - ky * d.n2h;
    sp[((long)ky * d.n0 + x) * d.n2h + kz] = buf[ky * d.rs + kz];
  }
  if (fu.partA) {
    block_sum<2>(acc, red);
    if (threadIdx.x == 0) {
      double* o = fu.partA + (((long)vec * 3 + c) * d.n0 + x) * 2;
      o[0] = acc[0];
      o[1] = acc[1];
    }
  }
}

// ---- pass B --------------------------------------------------------------------------------------------------
template <typename T>
__global__ void k_fft_b(cplx<T>* __restrict__ spec, const T* __restrict__ kinv, FftDims d, int kc, int m,
                        const cplx<T>* __restrict__ tw, const CellState* __restrict__ cs,
                        unsigned long long* __restrict__ units, int ukind, PcgFuse fu) {
  extern __shared__ unsigned char smem_raw[];
  cplx<T>* buf = reinterpret_cast<cplx<T>*>(smem_raw);  // [3][n0][kc]
  cplx<T>* scratch = buf + 3 * d.n0 * kc;
  __shared__ double red[32];
  const int ky = blockIdx.x, kz0 = blockIdx.y * kc, vec = blockIdx.z;
  if (cs && !cs[vec / m].active) return;
  prof_count(units, ukind);
  const int nkz = min(kc, d.n2h - kz0);
  const int total = 3 * d.n0 * kc;
  constexpr int kBatch = batch<T>();
  for (int base = threadIdx.x; base < total; base += kBatch * blockDim.x) {
    cplx<T> v[kBatch];
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const int idx = base + u * blockDim.x;
      v[u] = {T(0), T(0)};
      if (idx < total) {
        const int c = idx / (d.n0 * kc), rem = idx - c * d.n0 * kc;
        const int xx = rem / kc, kz = rem - xx * kc;
        if (kz < nkz) v[u] = spec[((long)vec * 3 + c) * d.NS + ((long)ky * d.n0 + xx) * d.n2h + kz0 + kz];
      }
    }
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const int idx = base + u * blockDim.x;
      if (idx < total) buf[idx] = v[u];
    }
  }
  __syncthreads();
  lines_fft(buf, d.n0, 3 * kc, kc, d.n0 * kc, 1, kc, tw + d.off0, false, scratch, d.pp);
  double dot[1] = {0.0};
  const bool even = (d.n2 % 2) == 0;
#pragma unroll 2
  for (int idx = threadIdx.x; idx < d.n0 * kc; idx += blockDim.x) {
    const int kx = idx / kc, kz = idx - kx * kc;
    if (kz < nkz) {
      const T* K = kinv + (((long)kx * d.n1 + ky) * d.n2h + kz0 + kz) * 6;
      const T kxx = K[0], kyy = K[1], kzz = K[2], kyz = K[3], kxz = K[4], kxy = K[5];
      const cplx<T> a = buf[idx], b = buf[d.n0 * kc + idx], c = buf[2 * d.n0 * kc + idx];
      const cplx<T> ua{kxx * a.x + kxy * b.x + kxz * c.x, kxx * a.y + kxy * b.y + kxz * c.y};
      const cplx<T> ub{kxy * a.x + kyy * b.x + kyz * c.x, kxy * a.y + kyy * b.y + kyz * c.y};
      const cplx<T> uc{kxz * a.x + kyz * b.x + kzz * c.x, kxz * a.y + kyz * b.y + kzz * c.y};
      if (fu.partB) {
        // Parseval on the half spectrum: kz = 0 (and nz/2 for even nz) once, the others twice
        const int kzg = kz0 + kz;
        const double wt = (kzg == 0 || (even && 2 * kzg == d.n2)) ? 1.0 : 2.0;
        dot[0] += wt * ((double)a.x * ua.x + (double)a.y * ua.y + (double)b.x * ub.x + (double)b.y * ub.y +
                        (double)c.x * uc.x + (double)c.y * uc.y);
      }
      buf[idx] = ua;
      buf[d.n0 * kc + idx] = ub;
      buf[2 * d.n0 * kc + idx] = uc;
    }
  }
  __syncthreads();
  lines_fft(buf, d.n0, 3 * kc, kc, d.n0 * kc, 1, kc, tw + d.off0, true, scratch, d.pp);
#pragma unroll 4
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int c = idx / (d.n0 * kc), rem = idx - c * d.n0 * kc;
    const int xx = rem / kc, kz = rem - xx * kc;
    if (kz < nkz) spec[((long)vec * 3 + c) * d.NS + ((long)ky * d.n0 + xx) * d.n2h + kz0 + kz] = buf[idx];
  }
  if (fu.partB) {
    block_sum<1>(dot, red);
    if (threadIdx.x == 0) fu.partB[((long)vec * d.n1 + ky) * gridDim.y + blockIdx.y] = dot[0];
  }
}

// ---- pass C --------------------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256, 3) k_fft_c(const cplx<T>* __restrict__ spec, const T* __restrict__ w, const T* __restrict__ r,
                        T* __restrict__ z, FftDims d, int m, const cplx<T>* __restrict__ tw,
                        const CellState* __restrict__ cs, double* __restrict__ partial,
                        unsigned long long* __restrict__ units, int ukind, PcgFuse fu) {
  extern __shared__ unsigned char smem_raw[];
  cplx<T>* buf = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* scratch = buf + d.n1 * d.rs;
  __shared__ double red[32 * 4];
  const int x = blockIdx.x, c = blockIdx.y, vec = blockIdx.z;
  if (cs && !cs[vec / m].active) return;
  prof_count(units, ukind);
  const cplx<T>* sp = spec + ((long)vec * 3 + c) * d.NS;
  constexpr int kBatch = batch<T>();
  {
    const int total = d.n1 * d.n2h;
    for (int base = threadIdx.x; base < total; base += kBatch * blockDim.x) {
      cplx<T> v[kBatch];
#pragma unroll
      for (int u = 0; u < kBatch; ++u) {
        const int idx = base + u * blockDim.x;
        if (idx < total) {
          const int ky = idx / d.n2h, kz = idx - ky * d.n2h;
          v[u] = sp[((long)ky * d.n0 + x) * d.n2h + kz];
        }
      }
#pragma unroll
      for (int u = 0; u < kBatch; ++u) {
        const int idx = base + u * blockDim.x;
        if (idx < total) {
          const int ky = idx / d.n2h, kz = idx - ky * d.n2h;
          buf[ky * d.rs + kz] = v[u];
        }
      }
    }
  }
  __syncthreads();
  lines_fft(buf, d.n1, d.n2h, d.n2h, 0, 1, d.rs, tw + d.off1, true, scratch, d.pp);
  const bool packed = (d.n2 % 2) == 0;
  if (packed) {
    real_pre(buf, d.n1, d.rs, d.n2, tw + d.off2);
    lines_fft(buf, d.n2 / 2, d.n1, d.n1, 0, d.rs, 1, tw + d.off2h, true, scratch, d.pp);
  } else {
    // rebuild the full row from Hermitian symmetry, then a length-n2 inverse DFT
    for (int idx = threadIdx.x; idx < d.n1 * d.n2; idx += blockDim.x) {
      const int y = idx / d.n2, k = idx - y * d.n2;
      if (k >= d.n2h) buf[y * d.rs + k] = cconj(buf[y * d.rs + (d.n2 - k)]);
    }
    __syncthreads();
    lines_fft(buf, d.n2, d.n1, d.n1, 0, d.rs, 1, tw + d.off2, true, scratch, d.pp);
  }
  // the packed z transform has length n2/2, so its unnormalised inverse carries n0 n1 n2/2
  const T norm = T((packed ? 2.0 : 1.0) / (double)d.N);
  const long pbase = ((long)vec * 3 + c) * d.N + (long)x * d.n1 * d.n2;
  const T* wp = w ? w + (long)(vec / m) * d.N + (long)x * d.n1 * d.n2 : nullptr;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  if (packed) {  // one complex entry = the pair (2j, 2j+1) of a row: vector loads and stores of two reals
    using V2 = typename Vec2<T>::type;
    const int M = d.n2 / 2, total = d.n1 * M;
    const V2* wp2 = reinterpret_cast<const V2*>(wp);
    const V2* rp2 = reinterpret_cast<const V2*>(r + pbase);
    V2* zp2 = reinterpret_cast<V2*>(z + pbase);
    for (int base = threadIdx.x; base < total; base += kBatch * blockDim.x) {
      V2 wv[kBatch], rv[kBatch];
#pragma unroll
      for (int u = 0; u < kBatch; ++u) {
        const int idx = base + u * blockDim.x;
        if (idx < total) {
          if (wp) wv[u] = wp2[idx];
          if (partial) rv[u] = rp2[idx];
        }
      }
#pragma unroll
      for (int u = 0; u < kBatch; ++u) {
        const int idx = base + u * blockDim.x;
        if (idx < total) {
          const int y = fdiv(idx, M), j = idx - y * M;
          const cplx<T> q = buf[y * d.rs + j];
          V2 v{q.x * norm, q.y * norm};
          if (wp) {
            v.x *= wv[u].x;
            v.y *= wv[u].y;
          }
          zp2[idx] = v;
          acc[0] += (double)v.x + (double)v.y;
          if (partial) {
            acc[1] += (double)rv[u].x * (double)v.x + (double)rv[u].y * (double)v.y;
            acc[2] += (double)rv[u].x + (double)rv[u].y;
            acc[3] += (double)rv[u].x * (double)rv[u].x + (double)rv[u].y * (double)rv[u].y;
          }
        }
      }
    }
  } else {
    for (int idx = threadIdx.x; idx < d.n1 * d.n2; idx += blockDim.x) {
      const int y = idx / d.n2, zz = idx - y * d.n2;
      T v = buf[y * d.rs + zz].x * norm;
      if (wp) v *= wp[idx];
      z[pbase + idx] = v;
      acc[0] += (double)v;
      if (partial) {
        const double rv = (double)r[pbase + idx];
        acc[1] += rv * (double)v;
        acc[2] += rv;
        acc[3] += rv * rv;
      }
    }
  }
  if (partial || fu.partC) {
    block_sum<4>(acc, red);
    if (threadIdx.x == 0) {
      if (partial) {
        double* o = partial + (((long)vec * 3 + c) * d.n0 + x) * 4;
        o[0] = acc[0];
        o[1] = acc[1];
        o[2] = acc[2];
        o[3] = acc[3];
      }
      if (fu.partC) fu.partC[((long)vec * 3 + c) * d.n0 + x] = acc[0];
    }
  }
}

// ---- register-resident passes for cubic grids of 32 or 64 (FP64) ---------------------------------------------
// A line of n = R L points (R = 4 or 8) lives in a group of L lanes with R registers each. Natural distribution:
// lane l holds x[l + L r] in register r. Transposed distribution: lane l holds X[k1 + R brev(l)] in register k1 (brev over
// log2 L bits). fft_nat_in maps natural -> transposed (register DFT, twiddle, cross-lane decimation in frequency
// by warp shuffles); fft_tr_in maps transposed -> natural (cross-lane decimation in time, twiddle, register
// DFT). Both compute the plain DFT (INV: conjugate twiddles, no scaling); tw[k] = e^{-2 pi i k / n}.
__device__ __forceinline__ cplx<double> shfl_xor_c(cplx<double> v, int m) {
  return {__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m)};
}
__device__ __forceinline__ cplx<double> shfl_c(cplx<double> v, int src) {
  return {__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src)};
}
template <bool INV>
__device__ __forceinline__ cplx<double> twid(const cplx<double>* __restrict__ tw, int e) {
  const cplx<double> w = tw[e];
  return INV ? cplx<double>{w.x, -w.y} : w;
}
template <int L>
__device__ __forceinline__ int brevL(int l) {
  return L == 1 ? 0 : (int)(__brev((unsigned)l) >> (32 - ilog2c(L)));
}

template <int R, bool INV>
__device__ __forceinline__ void dft_reg(cplx<double> (&a)[R]) {
  if constexpr (R == 8) {
    dft_small<double, INV>(a, 8);
  } else {
    static_assert(R == 4, "register DFT of 4 or 8 points");
    dft4<double, INV>(a[0], a[1], a[2], a[3]);
  }
}

// The twiddles one lane needs for lines of n = R L points, read once from the table: W_n^{l k1} (k1 < R) and the
// cross-lane stage factors W_{2s}^{l mod s} (stage s = 2^j in slot j).
template <int L, int R>
struct LaneTw {
  static constexpr int NS = ilog2c(L) > 0 ? ilog2c(L) : 1;
  cplx<double> r[R];
  cplx<double> st[NS];
  __device__ __forceinline__ void load(const cplx<double>* __restrict__ tw, int l) {
    constexpr int n = R * L;
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) r[k1] = (l && k1) ? tw[l * k1] : cplx<double>{1.0, 0.0};
#pragma unroll
    for (int j = 0; j < NS; ++j) {
      const int s = 1 << j;
      st[j] = (L > 1) ? tw[(l & (s - 1)) * (n / (2 * s))] : cplx<double>{1.0, 0.0};
    }
  }
  __device__ __forceinline__ cplx<double> rr(int k1) const { return r[k1]; }
  __device__ __forceinline__ cplx<double> ss(int j) const { return st[j]; }
};
// The same twiddles read on use from a lane-major shared-memory table (fewer registers, more CTAs per SM): row
// k1 - 1 (k1 = 1..R-1) holds W_n^{l k1} and row R - 1 + j the stage-j factor, for lanes l = 0..L-1 side by side.
// The L lanes of a line read L consecutive entries of one row (no bank conflicts, no index arithmetic beyond the
// lane's base). Entries equal those LaneTw reads from the table, (1, 0) for l = 0.
template <int L, int R>
struct LaneTab {
  static constexpr int NS = ilog2c(L) > 0 ? ilog2c(L) : 1;
  static constexpr int ROWS = (R - 1) + NS;
  static constexpr int SIZE = ROWS * L;
};
// Fills a lane-major table from a twiddle table of n = R L entries (tw[k] = e^{-2 pi i k / n}); no barrier.
template <int L, int R>
__device__ __forceinline__ void stage_lane_tab(cplx<double>* __restrict__ dst, const cplx<double>* __restrict__ tw) {
  constexpr int n = R * L;
  for (int i = threadIdx.x; i < LaneTab<L, R>::SIZE; i += blockDim.x) {
    const int row = i / L, l = i - row * L;
    int k;
    if (row < R - 1) {
      k = l * (row + 1);
    } else {
      const int s = 1 << (row - (R - 1));
      k = (l & (s - 1)) * (n / (2 * s));
    }
    dst[i] = (L > 1 && k) ? tw[k] : cplx<double>{1.0, 0.0};
  }
}
template <int L, int R>
struct LaneTwS {
  const cplx<double>* b;  // the lane's column of a LaneTab<L, R> table in shared memory
  __device__ __forceinline__ void load(const cplx<double>* tab, int lane) { b = tab + lane; }
  __device__ __forceinline__ cplx<double> rr(int k1) const { return k1 ? b[(k1 - 1) * L] : cplx<double>{1.0, 0.0}; }
  __device__ __forceinline__ cplx<double> ss(int j) const {
    return (L > 1) ? b[(R - 1 + j) * L] : cplx<double>{1.0, 0.0};
  }
};
template <int L, int R, bool SMT>
using TwT = typename std::conditional<SMT, LaneTwS<L, R>, LaneTw<L, R>>::type;

// Shared-memory twiddles of the shared-twiddle variants of passes A and C: lane-major tables of the y lines (N / 8
// lanes of 8) and of the z lines (N / 16 lanes of 8), and the post-processing table (N entries) stored permuted
// within aligned runs of 8 (entry k at swz_tw(k)): the 4 lanes of a row read entries k1 + 8 k2, which then fall in
// different bank groups. stage_tw ends with a barrier.
__device__ __forceinline__ int swz_tw(int k) { return (k & ~7) | ((k ^ (k >> 3)) & 7); }
template <int N>
struct SmTw {
  cplx<double> y[LaneTab<N / 8, 8>::SIZE], z[LaneTab<N / 16, 8>::SIZE], n2[N];
};
template <int N>
__device__ __forceinline__ void stage_tw(SmTw<N>& st, const cplx<double>* __restrict__ tw_y,
                                         const cplx<double>* __restrict__ tw_z, const cplx<double>* __restrict__ tw_n2) {
  stage_lane_tab<N / 8, 8>(st.y, tw_y);
  stage_lane_tab<N / 16, 8>(st.z, tw_z);
  for (int i = threadIdx.x; i < N; i += blockDim.x) st.n2[swz_tw(i)] = tw_n2[i];
  __syncthreads();
}

// 16-byte asynchronous global -> shared copy (cp.async, L2 only)
__device__ __forceinline__ void cp16_async(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

template <bool INV>
__device__ __forceinline__ cplx<double> cj(cplx<double> w) {
  return INV ? cplx<double>{w.x, -w.y} : w;
}

// The cross-lane butterflies run the same arithmetic on both lanes of a pair, with no per-element selects: a lane
// of the upper half (up) takes the sign -1 and its stage twiddle w, a lane of the lower half +1 and w = 1 (a
// product by (1, 0) is exact). The results equal those of the two-sided form
//   natural in:    lower a + pv, upper (pv - a) w
//   transposed in: lower a + w pv, upper pv - w a
// (the pair's lanes share w, so in the transposed form the upper lane forms w a and hands it to the lower one).
// NL lines at once (the same lanes and twiddles, e.g. the three components of a column): each stage's sign,
// twiddle and lane twiddle are formed once, and the lines' butterflies interleave (NL independent chains).
template <int L, int R, bool INV, class TW, int NL>
__device__ __forceinline__ void fft_nat_in_n(cplx<double> (&a)[NL][R], int l, const TW& T) {
#pragma unroll
  for (int n = 0; n < NL; ++n) dft_reg<R, INV>(a[n]);
  if (L == 1) return;
#pragma unroll
  for (int k1 = 1; k1 < R; ++k1) {
    const cplx<double> t = cj<INV>(T.rr(k1));
#pragma unroll
    for (int n = 0; n < NL; ++n) a[n][k1] = cmul(a[n][k1], t);
  }
#pragma unroll
  for (int j = ilog2c(L) - 1; j >= 0; --j) {
    const int s = 1 << j;
    const bool up = (l & s) != 0;
    const cplx<double> w = cj<INV>(T.ss(j));
    const cplx<double> wl = up ? w : cplx<double>{1.0, 0.0};
    const double sg = up ? -1.0 : 1.0;
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1)
#pragma unroll
      for (int n = 0; n < NL; ++n) {
        const cplx<double> pv = shfl_xor_c(a[n][k1], s);
        const cplx<double> d{fma(sg, a[n][k1].x, pv.x), fma(sg, a[n][k1].y, pv.y)};  // a + pv, or pv - a
        a[n][k1] = cmul(d, wl);
      }
  }
}
template <int L, int R, bool INV, class TW, int NL>
__device__ __forceinline__ void fft_tr_in_n(cplx<double> (&a)[NL][R], int l, const TW& T) {
  if (L > 1) {
#pragma unroll
    for (int j = 0; j < ilog2c(L); ++j) {
      const int s = 1 << j;
      const bool up = (l & s) != 0;
      const cplx<double> w = cj<INV>(T.ss(j));
      const cplx<double> wl = up ? w : cplx<double>{1.0, 0.0};
      const double sg = up ? -1.0 : 1.0;
#pragma unroll
      for (int k1 = 0; k1 < R; ++k1)
#pragma unroll
        for (int n = 0; n < NL; ++n) {
          const cplx<double> c = cmul(wl, a[n][k1]);  // the upper element times w, or the lower one as it is
          const cplx<double> pv = shfl_xor_c(c, s);
          a[n][k1] = {fma(sg, c.x, pv.x), fma(sg, c.y, pv.y)};  // a + w pv, or pv - w a
        }
    }
#pragma unroll
    for (int k1 = 1; k1 < R; ++k1) {
      const cplx<double> t = cj<INV>(T.rr(k1));
#pragma unroll
      for (int n = 0; n < NL; ++n) a[n][k1] = cmul(a[n][k1], t);
    }
  }
#pragma unroll
  for (int n = 0; n < NL; ++n) dft_reg<R, INV>(a[n]);
}
template <int L, int R, bool INV, class TW>
__device__ __forceinline__ void fft_nat_in(cplx<double> (&a)[R], int l, const TW& T) {
  fft_nat_in_n<L, R, INV, TW, 1>(reinterpret_cast<cplx<double>(&)[1][R]>(a), l, T);
}
template <int L, int R, bool INV, class TW>
__device__ __forceinline__ void fft_tr_in(cplx<double> (&a)[R], int l, const TW& T) {
  fft_tr_in_n<L, R, INV, TW, 1>(reinterpret_cast<cplx<double>(&)[1][R]>(a), l, T);
}

// shared plane index of bin kz in a row: within each run of 8 bins the low 3 bits are xor-ed with the run index
// (the row-wise writes of pass A and the reads of pass C touch 8 bins that are 8 apart)
template <int M>
__device__ __forceinline__ int swz(int kz) {
  return kz < M ? ((kz & ~7) | ((kz ^ (kz >> 3)) & 7)) : kz;
}

template <int N>
struct Fast {
  static constexpr int M = N / 2, H = M + 1;
  static constexpr int Lz = M / 8, Ly = N / 8;
  static constexpr int P = 256 / (N * Lz);  // x-planes per CTA of passes A and C
  // pass B: lines of N = 4 Lb points in Lb lanes; a CTA takes KY ky rows, or half the kz range of one row (N = 64)
  static constexpr int Lb = N / 4;
  static constexpr int KY = (N == 64) ? 1 : 2;
  static constexpr int KZC = (N == 64) ? 2 : 1;            // kz chunks per ky row (one CTA each)
  static constexpr int KZN = (H + KZC - 1) / KZC;          // kz per chunk
  static constexpr int NTB = ((KY * KZN * Lb) + 31) / 32 * 32;
  // row stride (16-byte entries) of pass B's staged slabs: KZN is odd, so the 8 x rows a quarter-warp reads or
  // writes at one kz land in 8 different bank groups
  static constexpr int KPB = KZN;
  // plane buffer of passes A and C: [P][N rows][HS] (16-byte entries), bin kz of row y at slot(y, kz): the rows
  // are padded (N = 64: 40 entries, N = 32: 24) and the bins permuted within each aligned run of 8 by the row and
  // the run index, so that a quarter-warp's 16-byte accesses hit 8 different bank groups in every access pattern
  // of the passes. N = 64: 8 rows of one column (y = l + 8 q, and y = k1 + 8 brev(l) when the y transform writes
  // back), and 4 bins k1 + 8 k2 (or their mirrors M - k) of 2 adjacent rows. N = 32: 4 rows of 2 adjacent columns
  // (y = l + 4 q, and k1 + 8 brev(l)), and 2 bins k1 + 8 k2 of 4 adjacent rows. The row term of the N = 32 map
  // was found by an exhaustive search over maps of this form.
  static constexpr int HS = (N == 64) ? 40 : (N == 32) ? 24 : H;
  // row stride, in double pairs, of the real-row views of the same buffer (staged variants, one plane per CTA)
  static constexpr int PS = (N == 64) ? N / 2 + 4 : N / 2;
  static constexpr size_t smem_plane() { return (size_t)P * N * HS * sizeof(cplx<double>); }
  __device__ static __forceinline__ int slot(int y, int kz) {
    if constexpr (N == 64) {
      const int h = ((((y & 1) << 2) | ((y & 7) >> 1)) ^ (y >> 3)) & 7;
      return (kz & ~7) | ((kz ^ (kz >> 3) ^ h) & 7);
    } else if constexpr (N == 32) {
      const int h = (2 * (y & 7) + 2 * (y >> 3)) & 7;
      return (kz & ~7) | ((kz ^ (kz >> 3) ^ h) & 7);
    } else {
      return swz<M>(kz);
    }
  }
};
static_assert(Fast<64>::PS * 64 <= Fast<64>::P * 64 * Fast<64>::HS, "real-row view fits the plane buffer");

// deterministic block sum of K values: warp shuffles, per-warp slots, thread 0 adds the warps in order
template <int K>
__device__ __forceinline__ void block_sum_ordered(double (&v)[K], double* red /* [32][K] */) {
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  const int wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) red[wid * K + k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int w = 1; w < nw; ++w)
#pragma unroll
      for (int k = 0; k < K; ++k) v[k] += red[w * K + k];
}

// Pass A: (fused) r update and sums; w r; packed real z FFT + real post-processing per row; y FFT per column.
// SMT: twiddles from a shared-memory copy of the tables, 3 CTAs per SM instead of 2. STG (with SMT, one plane
// per CTA): the r update, the sums and the node scaling run over the plane in whole 512-byte rows (coalesced)
// and reach the FFT's layout through the plane buffer.
template <int N, bool SMT, bool STG = false>
__global__ void __launch_bounds__(256, SMT ? 3 : 2)
    k_fa_fast(double* __restrict__ r, const double* __restrict__ w, cplx<double>* __restrict__ spec, int m,
              const cplx<double>* __restrict__ tw_y, const cplx<double>* __restrict__ tw_z,
              const cplx<double>* __restrict__ tw_n2, const CellState* __restrict__ cs,
              unsigned long long* __restrict__ units, int ukind, PcgFuse fu) {
  using F = Fast<N>;
  constexpr int M = F::M, H = F::H, Lz = F::Lz, Ly = F::Ly, P = F::P;
  constexpr long NN = (long)N * N * N;
  // SOUT (shared twiddles, one plane per CTA): the y transforms write back into the plane buffer, and the plane's
  // spectrum goes out in whole rows afterwards (instead of 64-byte pieces of 8 rows per warp store)
  constexpr bool SOUT = SMT && P == 1;
  extern __shared__ unsigned char smem_raw[];
  cplx<double>* sm = reinterpret_cast<cplx<double>*>(smem_raw);  // [P][N rows][HS]
  __shared__ double red[32 * 2 * P];
  const int c = blockIdx.y, vec = blockIdx.z;
  if (!vec_live(cs, vec, m)) return;
  prof_count(units, ukind);
  __shared__ SmTw<N> stw;
  if constexpr (SMT) {
    stage_tw<N>(stw, tw_y, tw_z, tw_n2);
    tw_y = stw.y;
    tw_z = stw.z;
    tw_n2 = stw.n2;
  }
  const int t = threadIdx.x;
  const int p = t / (N * Lz), rem = t - p * (N * Lz), y = rem / Lz, l = rem - y * Lz;
  const int x = blockIdx.x * P + p;
  const long roff = ((long)vec * 3 + c) * NN + ((long)x * N + y) * N;  // start of the row (x, y, :)
  const double2* rp2 = reinterpret_cast<const double2*>(r + roff);
  const double2* ap2 = fu.Ap ? reinterpret_cast<const double2*>(static_cast<const double*>(fu.Ap) + roff) : nullptr;
  const double2* wp2 = w ? reinterpret_cast<const double2*>(w + (long)(vec / m) * NN + ((long)x * N + y) * N) : nullptr;
  cplx<double> a[8];
  double sr = 0.0, srr = 0.0;
  if constexpr (STG && P == 1) {
    // the plane in whole 512-byte rows: each warp takes one row of r, Ap and w per step (coalesced) for the r
    // update, the sums and the scaling; w r goes through the plane buffer to the FFT's layout
    double2* vs2 = reinterpret_cast<double2*>(sm);  // [N rows][PS] (N / 2 pairs used)
    const long poff = ((long)vec * 3 + c) * NN + (long)x * N * N;
    double2* rq = reinterpret_cast<double2*>(r + poff);
    const double2* aq = fu.Ap ? reinterpret_cast<const double2*>(static_cast<const double*>(fu.Ap) + poff) : nullptr;
    const double2* wq = w ? reinterpret_cast<const double2*>(w + (long)(vec / m) * NN + (long)x * N * N) : nullptr;
    const double al = aq ? fu.vs[vec].alpha : 0.0, mu = aq ? fu.vs[vec].mean[c] : 0.0;
    constexpr int PAIRS = N * N / 2;
#pragma unroll 4
    for (int j = t; j < PAIRS; j += 256) {
      double2 v = rq[j];
      if (aq) {
        const double2 u = aq[j];
        v.x -= al * (u.x - mu);
        v.y -= al * (u.y - mu);
        rq[j] = v;
      }
      sr += v.x + v.y;
      srr += v.x * v.x + v.y * v.y;
      if (wq) {
        const double2 ww = wq[j];
        v.x *= ww.x;
        v.y *= ww.y;
      }
      vs2[(j / (N / 2)) * F::PS + (j % (N / 2))] = v;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const double2 v = vs2[y * F::PS + l + Lz * q];
      a[q] = {v.x, v.y};
    }
    __syncthreads();  // the plane buffer takes the rows' spectra next
  } else {
    double2 v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = rp2[l + Lz * q];
    if (ap2) {
      const double al = fu.vs[vec].alpha, mu = fu.vs[vec].mean[c];
      double2 u[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) u[q] = ap2[l + Lz * q];
      double2* rw2 = reinterpret_cast<double2*>(r + roff);
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        v[q].x -= al * (u[q].x - mu);
        v[q].y -= al * (u[q].y - mu);
        rw2[l + Lz * q] = v[q];
      }
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      sr += v[q].x + v[q].y;
      srr += v[q].x * v[q].x + v[q].y * v[q].y;
    }
    if (wp2) {
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const double2 ww = wp2[l + Lz * q];
        v[q].x *= ww.x;
        v[q].y *= ww.y;
      }
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) a[q] = {v[q].x, v[q].y};
  }
  // packed z FFT: a[k1] = Z[k1 + 8 brev(l)]
  {
    TwT<Lz, 8, SMT> T;
    T.load(tw_z, l);
    fft_nat_in<Lz, 8, false>(a, l, T);
  }
  const int k2 = brevL<Lz>(l);
  cplx<double>* row = sm + ((long)p * N + y) * F::HS;
  {
    // k1 = 0 partner: bin M - 8 k2 = 8 ((Lz - k2) mod Lz)
    const int lane0 = (t & 31) - l;
    const cplx<double> b0 = shfl_c(a[0], lane0 + brevL<Lz>((Lz - k2) & (Lz - 1)));
    cplx<double> bz[8];
    bz[0] = b0;
#pragma unroll
    for (int k1 = 1; k1 < 8; ++k1) bz[k1] = shfl_xor_c(a[8 - k1], Lz - 1);
#pragma unroll
    for (int k1 = 0; k1 < 8; ++k1) {
      const int k = k1 + 8 * k2;
      cplx<double> R;
      if (k == 0) {
        R = {a[0].x + a[0].y, 0.0};
        row[F::slot(y, M)] = {a[0].x - a[0].y, 0.0};
      } else {
        const cplx<double> A = a[k1], B = bz[k1];  // X_k, X_{M-k}
        const cplx<double> E{(A.x + B.x) * 0.5, (A.y - B.y) * 0.5};
        const cplx<double> O{(A.y + B.y) * 0.5, -(A.x - B.x) * 0.5};
        R = cadd(E, cmul(tw_n2[SMT ? swz_tw(k) : k], O));
      }
      row[F::slot(y, k)] = R;
    }
  }
  if (fu.partA) {
    double v2[2] = {sr, srr};
    // per-plane sums: the threads of a plane are contiguous and a multiple of 32
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v2[k] += __shfl_down_sync(0xffffffffu, v2[k], o);
    if ((t & 31) == 0) {
      red[(t >> 5) * 2] = v2[0];
      red[(t >> 5) * 2 + 1] = v2[1];
    }
  }
  __syncthreads();
  if (fu.partA && t < P) {
    constexpr int WPP = N * Lz / 32;  // warps per plane
    double s0 = 0.0, s1 = 0.0;
    for (int q = 0; q < WPP; ++q) {
      s0 += red[(t * WPP + q) * 2];
      s1 += red[(t * WPP + q) * 2 + 1];
    }
    double* o = fu.partA + (((long)vec * 3 + c) * N + blockIdx.x * P + t) * 2;
    o[0] = s0;
    o[1] = s1;
  }
  // y FFT per (plane, kz) column: groups of Ly lanes
  constexpr int G = 256 / Ly, TASKS = P * H, IT = (TASKS + G - 1) / G;
  const int g = t / Ly, ly = t - g * Ly;
  cplx<double>* sp = spec + ((long)vec * 3 + c) * ((long)N * N * H);
  TwT<Ly, 8, SMT> Ty;
  Ty.load(tw_y, ly);
#pragma unroll 1
  for (int it = 0; it < IT; ++it) {
    const int task = g + it * G;
    const bool ok = task < TASKS;
    if (!__any_sync(0xffffffffu, ok)) break;  // whole warp past the last column
    const int pp = ok ? task / H : 0, kz = ok ? task - pp * H : 0;
    cplx<double> b[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) b[q] = sm[((long)pp * N + ly + Ly * q) * F::HS + F::slot(ly + Ly * q, kz)];
    fft_nat_in<Ly, 8, false>(b, ly, Ty);
    if (ok) {
      const int xx = blockIdx.x * P + pp, kb = 8 * brevL<Ly>(ly);
      if constexpr (SOUT) {
        // back into the column's slots (every lane of the group has read the column: the shuffles order it)
#pragma unroll
        for (int k1 = 0; k1 < 8; ++k1) sm[((long)pp * N + k1 + kb) * F::HS + F::slot(k1 + kb, kz)] = b[k1];
      } else {
#pragma unroll
        for (int k1 = 0; k1 < 8; ++k1) sp[((long)(k1 + kb) * N + xx) * H + kz] = b[k1];
      }
    }
  }
  if constexpr (SOUT) {
    // the plane's spectrum rows [ky][x][0, H) out in whole rows, walked in slot order (the pad slots skipped)
    __syncthreads();
    for (int i = t; i < N * F::HS; i += 256) {
      const int ky = i / F::HS, sl = i - ky * F::HS;
      const int kz = F::slot(ky, sl);  // slot() permutes each aligned run of 8 as an involution
      if (kz < H && F::slot(ky, kz) == sl) sp[((long)ky * N + blockIdx.x) * H + kz] = sm[(long)ky * F::HS + sl];
    }
  }
}

// The inverse preconditioner symbol at one wavenumber in closed form (the same values as the Kinv table, to
// rounding). For the Q1 element with exact (2x2x2 Gauss) integration the unit-stiffness symbol factorises into the
// 1D symbols of the linear hat, m = (2 + cos t) / 3 (mass), s = 2 - 2 cos t (stiffness) and g = sin t (gradient):
// S_aa = s_a m_b m_c, S_ab = g_a g_b m_c, K = lam S + mu (tr S I + S); then (K + 1e-12 |tr K| I)^-1, and 0 at k = 0
// (nlfiber/linear.py:154-165). The y and z factors are per thread; (mx, sx, gx) per x frequency.
struct SymYZ {
  double my, sy, gy, mz, sz, gz;
};
__device__ __forceinline__ SymYZ sym_yz(cplx<double> ty, cplx<double> tz) {
  const double cy = ty.x, cz = tz.x;
  return {(2.0 + cy) * (1.0 / 3.0), 2.0 - 2.0 * cy, -ty.y, (2.0 + cz) * (1.0 / 3.0), 2.0 - 2.0 * cz, -tz.y};
}
__device__ __forceinline__ void kinv_closed(const SymYZ& q, double cx, double gx, double lam, double mu,
                                            double (&out)[6]) {
  const double mx = (2.0 + cx) * (1.0 / 3.0), sx = 2.0 - 2.0 * cx;
  const double Sxx = sx * q.my * q.mz, Syy = mx * q.sy * q.mz, Szz = mx * q.my * q.sz;
  const double Syz = mx * q.gy * q.gz, Sxz = gx * q.gz * q.my, Sxy = gx * q.gy * q.mz;
  const double lm = lam + mu, tr = Sxx + Syy + Szz;
  double a = lm * Sxx + mu * tr, b = lm * Syy + mu * tr, c = lm * Szz + mu * tr;
  const double d = lm * Syz, e = lm * Sxz, f = lm * Sxy;
  const double reg = 1e-12 * fabs(a + b + c);
  a += reg;
  b += reg;
  c += reg;
  // inverse of [[a f e] [f b d] [e d c]]
  const double cxx = b * c - d * d, cxy = d * e - c * f, cxz = d * f - b * e;
  const double cyy = a * c - e * e, cyz = e * f - a * d, czz = a * b - f * f;
  const double id = 1.0 / (a * cxx + f * cxy + e * cxz);
  out[0] = cxx * id;
  out[1] = cyy * id;
  out[2] = czz * id;
  out[3] = cyz * id;
  out[4] = cxz * id;
  out[5] = cxy * id;
}

__device__ __forceinline__ int tw_slot(int i) { return i ^ ((i >> 3) & 7); }

// Pass B: x FFT of the three components of each (ky, kz) column, 3x3 Kinv, Parseval (r, z) partial, inverse.
// CLOSED: the Kinv entries are computed in closed form from the twiddles and the medium's (lam, mu) instead of
// read from the table; the x twiddles are then read from a shared-memory copy of the table, which keeps the CTA
// (9 warps) at 96 registers, the most for 2 CTAs per SM (an SMSP takes 5 of the 18 warps). The x transforms read
// their twiddles from a lane-major copy (LaneTab); the symbol's entries kx = k1 + 4 brev(l), ky and kz come from a
// copy of the table that holds entry i at tw_slot(i) = i ^ ((i >> 3) & 7), so that the 8 lanes of a quarter-warp
// read their kx entries from 8 different bank groups (8 wavefronts each in table order).
// STG (cubes of 64, with CLOSED): the CTA's three [x][kz-chunk] slabs are copied whole into shared memory by
// cp.async (272-byte row pieces instead of 16-byte pieces over 16 x rows per warp), transformed from there, and
// written back the same way; rows of KZN (odd) entries spread the column accesses over all bank groups.
template <int N, bool CLOSED, bool STG = false>
__global__ void __launch_bounds__(Fast<N>::NTB, 2)
    k_fb_fast(cplx<double>* __restrict__ spec, const double* __restrict__ kinv, int m,
              const cplx<double>* __restrict__ tw_x, const CellState* __restrict__ cs,
              unsigned long long* __restrict__ units, int ukind, PcgFuse fu, double lam, double mu) {
  using F = Fast<N>;
  constexpr int M = F::M, H = F::H, L = F::Lb, KY = F::KY, KZC = F::KZC, KZN = F::KZN, KP = F::KPB;
  static_assert(!STG || KY == 1, "staged pass B takes one ky row per CTA");
  __shared__ double red[32];
  __shared__ cplx<double> twsh[N];
  __shared__ cplx<double> twl[CLOSED ? LaneTab<L, 4>::SIZE : 1];
  extern __shared__ __align__(16) unsigned char fb_raw[];
  cplx<double>* sb = reinterpret_cast<cplx<double>*>(fb_raw);  // STG: [3][N][KP]
  const int vec = blockIdx.z;
  if (!vec_live(cs, vec, m)) return;
  prof_count(units, ukind);
  if constexpr (CLOSED) {
    for (int i = threadIdx.x; i < N; i += blockDim.x) twsh[tw_slot(i)] = tw_x[i];
    stage_lane_tab<L, 4>(twl, tw_x);
    __syncthreads();
    tw_x = twsh;
  }
  const int t = threadIdx.x, task = t / L, l = t - task * L;
  const int kyl = task / KZN, kzl = task - kyl * KZN;
  const int kz = blockIdx.y * KZN + kzl;
  const bool ok = kyl < KY && kz < H;
  const int ky = blockIdx.x * KY + (ok ? kyl : 0);
  const long NS = (long)N * N * H;
  const int kz0 = blockIdx.y * KZN, nkz = min(KZN, H - kz0);
  if constexpr (STG) {
    for (int i = t; i < 3 * N * KZN; i += blockDim.x) {
      const int c = i / (N * KZN), rr = i - c * (N * KZN), x = rr / KZN, kk = rr - x * KZN;
      if (kk < nkz)
        cp16_async(sb + (c * N + x) * KP + kk, spec + ((long)vec * 3 + c) * NS + ((long)blockIdx.x * N + x) * H + kz0 + kk);
    }
    cp_async_commit();
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
  }
  cplx<double> a[3][4];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if constexpr (STG)
        a[c][q] = ok ? sb[(c * N + l + L * q) * KP + kzl] : cplx<double>{0.0, 0.0};
      else
        a[c][q] = ok ? spec[((long)vec * 3 + c) * NS + ((long)ky * N + l + L * q) * H + kz] : cplx<double>{0.0, 0.0};
    }
  typename std::conditional<CLOSED, LaneTwS<L, 4>, LaneTw<L, 4>>::type T;
  T.load(CLOSED ? twl : tw_x, l);
  fft_nat_in_n<L, 4, false>(a, l, T);
  double dot[1] = {0.0};
  const double wt = (kz == 0 || kz == M) ? 1.0 : 2.0;
  const int kb = 4 * brevL<L>(l);
  SymYZ q{};
  if constexpr (CLOSED) q = sym_yz(tw_x[tw_slot(ky)], tw_x[tw_slot(ok ? kz : 0)]);
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    double Kv[6];
    if constexpr (CLOSED) {
      const int kx = k1 + kb;
      if (kx == 0 && ky == 0 && kz == 0) {
#pragma unroll
        for (int i = 0; i < 6; ++i) Kv[i] = 0.0;
      } else {
        const cplx<double> tx = tw_x[tw_slot(kx)];
        kinv_closed(q, tx.x, -tx.y, lam, mu, Kv);
      }
    } else {
      const double* K = kinv + (((long)(k1 + kb) * N + ky) * H + (ok ? kz : 0)) * 6;
#pragma unroll
      for (int i = 0; i < 6; ++i) Kv[i] = K[i];
    }
    const double kxx = Kv[0], kyy = Kv[1], kzz = Kv[2], kyz = Kv[3], kxz = Kv[4], kxy = Kv[5];
    const cplx<double> A = a[0][k1], B = a[1][k1], C = a[2][k1];
    const cplx<double> ua{kxx * A.x + kxy * B.x + kxz * C.x, kxx * A.y + kxy * B.y + kxz * C.y};
    const cplx<double> ub{kxy * A.x + kyy * B.x + kyz * C.x, kxy * A.y + kyy * B.y + kyz * C.y};
    const cplx<double> uc{kxz * A.x + kyz * B.x + kzz * C.x, kxz * A.y + kyz * B.y + kzz * C.y};
    dot[0] += wt * (A.x * ua.x + A.y * ua.y + B.x * ub.x + B.y * ub.y + C.x * uc.x + C.y * uc.y);
    a[0][k1] = ua;
    a[1][k1] = ub;
    a[2][k1] = uc;
  }
  fft_tr_in_n<L, 4, true>(a, l, T);
  if (ok)
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if constexpr (STG)
          sb[(c * N + l + L * q) * KP + kzl] = a[c][q];
        else
          spec[((long)vec * 3 + c) * NS + ((long)ky * N + l + L * q) * H + kz] = a[c][q];
      }
  if constexpr (STG) {
    __syncthreads();
    for (int i = t; i < 3 * N * KZN; i += blockDim.x) {
      const int c = i / (N * KZN), rr = i - c * (N * KZN), x = rr / KZN, kk = rr - x * KZN;
      if (kk < nkz) spec[((long)vec * 3 + c) * NS + ((long)blockIdx.x * N + x) * H + kz0 + kk] = sb[(c * N + x) * KP + kk];
    }
  }
  if (fu.partB) {
    if (!ok) dot[0] = 0.0;
    block_sum_ordered<1>(dot, red);
    // layout [vec][ky][KZC]: the CTA's sum in its first slot, zeros in the slots of its other ky rows
    if (t < KY) fu.partB[((long)vec * N + blockIdx.x * KY + t) * KZC + blockIdx.y] = (t == 0) ? dot[0] : 0.0;
  }
}

// Epilogue of the fused pass C for one thread's 8 double pairs of a z row (pair i = l + Lz q, q < 8):
// z = norm a w (w = 1 unscaled), x += alpha p, p = z + beta p. Two halves of 4 pairs keep the loads of w, p and
// x in flight together without holding all 24 pairs.
template <int Lz>
__device__ __forceinline__ void px_row(const cplx<double> (&a)[8], double norm, const double2* __restrict__ wp2,
                                       double2* __restrict__ xp2, double2* __restrict__ pp2, int l, double al,
                                       double be) {
#pragma unroll
  for (int hf = 0; hf < 2; ++hf) {
    double2 ww[4], po[4], xo[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = l + Lz * (4 * hf + q);
      ww[q] = wp2 ? wp2[i] : make_double2(1.0, 1.0);
      po[q] = pp2[i];
      xo[q] = xp2[i];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = l + Lz * (4 * hf + q);
      const cplx<double> v = a[4 * hf + q];
      xp2[i] = make_double2(xo[q].x + al * po[q].x, xo[q].y + al * po[q].y);
      pp2[i] = make_double2((v.x * norm) * ww[q].x + be * po[q].x, (v.y * norm) * ww[q].y + be * po[q].y);
    }
  }
}

// Pass C: inverse y FFT per column; real pre-processing + inverse packed z FFT per row; scale, w; sums (or the
// fused x/p update, fu.p set).
// SMT: twiddles from a shared-memory copy of the tables, 3 CTAs per SM instead of 2. STG (with SMT): the plane's
// spectrum rows are first copied whole into the plane buffer by cp.async (coalesced 16-byte pieces), and the y
// transforms run in place there; at N = 64 it runs 4 CTAs per SM (64 registers, a few spilled: measured 7.2 -> 6.5
// us per vector in the fused iteration, where pass A at 4 CTAs per SM loses).
template <int N, bool SMT, bool STG = false>
__global__ void __launch_bounds__(256, SMT ? ((STG && N == 64) ? 4 : 3) : 2)
    k_fc_fast(const cplx<double>* __restrict__ spec, const double* __restrict__ w, const double* __restrict__ r,
              double* __restrict__ z, int m, const cplx<double>* __restrict__ tw_y,
              const cplx<double>* __restrict__ tw_z, const cplx<double>* __restrict__ tw_n2,
              const CellState* __restrict__ cs, double* __restrict__ partial, unsigned long long* __restrict__ units,
              int ukind, PcgFuse fu) {
  using F = Fast<N>;
  constexpr int M = F::M, H = F::H, Lz = F::Lz, Ly = F::Ly, P = F::P;
  constexpr long NN = (long)N * N * N;
  extern __shared__ unsigned char smem_raw[];
  cplx<double>* sm = reinterpret_cast<cplx<double>*>(smem_raw);
  __shared__ double red[32 * 4];
  const int c = blockIdx.y, vec = blockIdx.z;
  if (!(fu.p ? vec_ran(cs, vec, m) : vec_live(cs, vec, m))) return;
  prof_count(units, ukind);
  __shared__ SmTw<N> stw;
  if constexpr (SMT) {
    stage_tw<N>(stw, tw_y, tw_z, tw_n2);
    tw_y = stw.y;
    tw_z = stw.z;
    tw_n2 = stw.n2;
  }
  const int t = threadIdx.x;
  const cplx<double>* sp = spec + ((long)vec * 3 + c) * ((long)N * N * H);
  if constexpr (STG) {
    // walked in slot order (8 consecutive threads fill one aligned run of 8 slots: no bank conflicts); the pad
    // slots of a row are skipped
    constexpr int HS = F::HS;
    for (int i = t; i < P * N * HS; i += 256) {
      const int pp = i / (N * HS), rr = i - pp * (N * HS), ky = rr / HS, sl = rr - ky * HS;
      const int kz = F::slot(ky, sl);  // slot() permutes each aligned run of 8 as an involution
      if (kz < H && F::slot(ky, kz) == sl)
        cp16_async(sm + ((long)pp * N + ky) * HS + sl, sp + ((long)ky * N + blockIdx.x * P + pp) * H + kz);
    }
    cp_async_commit();
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
  }
  {
    constexpr int G = 256 / Ly, TASKS = P * H, IT = (TASKS + G - 1) / G;
    const int g = t / Ly, ly = t - g * Ly;
    TwT<Ly, 8, SMT> Ty;
    Ty.load(tw_y, ly);
#pragma unroll 1
    for (int it = 0; it < IT; ++it) {
      const int task = g + it * G;
      const bool ok = task < TASKS;
      if (!__any_sync(0xffffffffu, ok)) break;  // whole warp past the last column
      const int pp = ok ? task / H : 0, kz = ok ? task - pp * H : 0;
      const int xx = blockIdx.x * P + pp;
      cplx<double> b[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        if constexpr (STG)
          b[q] = sm[((long)pp * N + ly + Ly * q) * F::HS + F::slot(ly + Ly * q, kz)];
        else
          b[q] = ok ? sp[((long)(ly + Ly * q) * N + xx) * H + kz] : cplx<double>{0.0, 0.0};
      }
      fft_nat_in<Ly, 8, true>(b, ly, Ty);
      if (ok) {
        const int yb = 8 * brevL<Ly>(ly);
#pragma unroll
        for (int k1 = 0; k1 < 8; ++k1) sm[((long)pp * N + k1 + yb) * F::HS + F::slot(k1 + yb, kz)] = b[k1];
      }
    }
  }
  __syncthreads();
  const int p = t / (N * Lz), rem = t - p * (N * Lz), y = rem / Lz, l = rem - y * Lz;
  const int x = blockIdx.x * P + p;
  const cplx<double>* row = sm + ((long)p * N + y) * F::HS;
  cplx<double> a[8];
  const int k2 = brevL<Lz>(l);
#pragma unroll
  for (int k1 = 0; k1 < 8; ++k1) {
    const int k = k1 + 8 * k2;
    if (k == 0) {
      // X_0 and X_M of a real signal are real: their imaginary parts are rounding and are dropped
      const double A = row[F::slot(y, 0)].x, B = row[F::slot(y, M)].x;
      a[k1] = {(A + B) * 0.5, (A - B) * 0.5};
    } else {
      const cplx<double> A = row[F::slot(y, k)], B = row[F::slot(y, M - k)];
      const cplx<double> E{(A.x + B.x) * 0.5, (A.y - B.y) * 0.5};
      const cplx<double> D{(A.x - B.x) * 0.5, (A.y + B.y) * 0.5};
      const cplx<double> O = cmul(D, cconj(tw_n2[SMT ? swz_tw(k) : k]));
      a[k1] = {E.x - O.y, E.y + O.x};
    }
  }
  {
    TwT<Lz, 8, SMT> T;
    T.load(tw_z, l);
    fft_tr_in<Lz, 8, true>(a, l, T);
  }
  // the packed z transform has length N/2, so its unnormalised inverse carries N^3 / 2
  constexpr double norm = 2.0 / (double)NN;
  const long roff = ((long)vec * 3 + c) * NN + ((long)x * N + y) * N;
  const double2* wp2 = w ? reinterpret_cast<const double2*>(w + (long)(vec / m) * NN + ((long)x * N + y) * N) : nullptr;
  if constexpr (STG) {
    if (fu.p && P == 1) {
      // the x/p update in whole 512-byte rows: z goes through the plane buffer (after every row's reads of it)
      // and each warp then updates one row of x and p per step (coalesced), w, x and p read the same way
      double2* zs = reinterpret_cast<double2*>(sm);  // [N rows][PS] (N / 2 pairs used)
      __syncthreads();
#pragma unroll
      for (int q = 0; q < 8; ++q) zs[y * F::PS + l + Lz * q] = make_double2(a[q].x * norm, a[q].y * norm);
      __syncthreads();
      const long poff = ((long)vec * 3 + c) * NN + (long)x * N * N;
      const double2* wq2 = w ? reinterpret_cast<const double2*>(w + (long)(vec / m) * NN + (long)x * N * N) : nullptr;
      double2* xq2 = reinterpret_cast<double2*>(fu.x + poff);
      double2* pq2 = reinterpret_cast<double2*>(fu.p + poff);
      const double al = fu.vs[vec].alpha, be = fu.vs[vec].beta;
      constexpr int PAIRS = N * N / 2;
#pragma unroll 4
      for (int j = t; j < PAIRS; j += 256) {
        const double2 ww = wq2 ? wq2[j] : make_double2(1.0, 1.0), po = pq2[j], xo = xq2[j],
                      zz = zs[(j / (N / 2)) * F::PS + (j % (N / 2))];
        xq2[j] = make_double2(xo.x + al * po.x, xo.y + al * po.y);
        pq2[j] = make_double2(zz.x * ww.x + be * po.x, zz.y * ww.y + be * po.y);
      }
      return;
    }
  }
  if (fu.p) {  // partial and partC are null here, so no thread reaches the barrier below
    px_row<Lz>(a, norm, wp2, reinterpret_cast<double2*>(fu.x + roff), reinterpret_cast<double2*>(fu.p + roff), l,
               fu.vs[vec].alpha, fu.vs[vec].beta);
    return;
  }
  double2* zp2 = reinterpret_cast<double2*>(z + roff);
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  double2 ww[8];
  if (wp2)
#pragma unroll
    for (int q = 0; q < 8; ++q) ww[q] = wp2[l + Lz * q];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    double2 v{a[q].x * norm, a[q].y * norm};
    if (wp2) {
      v.x *= ww[q].x;
      v.y *= ww[q].y;
    }
    zp2[l + Lz * q] = v;
    acc[0] += v.x + v.y;
    if (partial) {
      const double2 rv = reinterpret_cast<const double2*>(r + roff)[l + Lz * q];
      acc[1] += rv.x * v.x + rv.y * v.y;
      acc[2] += rv.x + rv.y;
      acc[3] += rv.x * rv.x + rv.y * rv.y;
    }
  }
  if (partial || fu.partC) {
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_down_sync(0xffffffffu, acc[k], o);
    if ((t & 31) == 0)
#pragma unroll
      for (int k = 0; k < 4; ++k) red[(t >> 5) * 4 + k] = acc[k];
    __syncthreads();
    if (t < P) {
      constexpr int WPP = N * Lz / 32;
      double s[4] = {0.0, 0.0, 0.0, 0.0};
      for (int q = 0; q < WPP; ++q)
#pragma unroll
        for (int k = 0; k < 4; ++k) s[k] += red[(t * WPP + q) * 4 + k];
      const long pl = ((long)vec * 3 + c) * N + blockIdx.x * P + t;
      if (partial)
#pragma unroll
        for (int k = 0; k < 4; ++k) partial[pl * 4 + k] = s[k];
      if (fu.partC) fu.partC[pl] = s[0];
    }
  }
}


// Pass C, persistent and pipelined (cubes of 64): each CTA walks the planes (vec, comp, x) blockIdx.x,
// blockIdx.x + gridDim.x, ... of active cells; while it transforms one plane, the spectrum rows of its next
// plane stream into the other of two shared staging buffers by cp.async. Same arithmetic as k_fc_fast.
template <int N>
__global__ void __launch_bounds__(256, 2)
    k_fc_pipe(const cplx<double>* __restrict__ spec, const double* __restrict__ w, const double* __restrict__ r,
              double* __restrict__ z, int m, int nvec, const cplx<double>* __restrict__ tw_y,
              const cplx<double>* __restrict__ tw_z, const cplx<double>* __restrict__ tw_n2,
              const CellState* __restrict__ cs, double* __restrict__ partial, unsigned long long* __restrict__ units,
              int ukind, PcgFuse fu) {
  using F = Fast<N>;
  constexpr int M = F::M, H = F::H, Lz = F::Lz, Ly = F::Ly;
  static_assert(F::P == 1, "one plane per step");
  constexpr long NN = (long)N * N * N;
  extern __shared__ unsigned char smem_raw[];
  cplx<double>* stage = reinterpret_cast<cplx<double>*>(smem_raw);  // [2][N ky][H kz]
  cplx<double>* T = stage + 2 * N * H;                               // [N y][H kz] (swizzled kz)
  __shared__ double red[8 * 4];
  const int t = threadIdx.x;
  const long nplanes = (long)nvec * 3 * N;
  auto active = [&](long j) {
    if (!cs) return true;
    const int vec = (int)(j / (3 * N));
    return fu.p ? vec_ran(cs, vec, m) : vec_live(cs, vec, m);
  };
  auto next_active = [&](long j) {
    while (j < nplanes && !active(j)) j += gridDim.x;
    return j;
  };
  auto issue = [&](long j, int b) {
    const int vec = (int)(j / (3 * N)), c = (int)((j / N) % 3), x = (int)(j % N);
    const cplx<double>* sp = spec + ((long)vec * 3 + c) * ((long)N * N * H) + (long)x * H;
    cplx<double>* dst = stage + b * N * H;
    for (int i = t; i < N * H; i += 256) {
      const int ky = i / H, kz = i - ky * H;
      cp16_async(dst + i, sp + (long)ky * N * H + kz);
    }
  };
  long j = next_active(blockIdx.x);
  if (j < nplanes) issue(j, 0);
  cp_async_commit();
  for (int it = 0; j < nplanes; ++it) {
    const long jn = next_active(j + gridDim.x);
    if (jn < nplanes) issue(jn, (it + 1) & 1);
    cp_async_commit();
    cp_async_wait1();
    __syncthreads();  // plane j staged
    const int vec = (int)(j / (3 * N)), c = (int)((j / N) % 3), x = (int)(j % N);
    if (units && c == 0 && x == 0 && t == 0) atomicAdd(units + ukind, 1ull);
    const cplx<double>* S = stage + (it & 1) * N * H;
    {
      constexpr int G = 256 / Ly, IT = (H + G - 1) / G;
      const int g = t / Ly, ly = t - g * Ly;
      LaneTw<Ly, 8> Ty;
      Ty.load(tw_y, ly);
#pragma unroll 1
      for (int q2 = 0; q2 < IT; ++q2) {
        const int kz = g + q2 * G;
        const bool ok = kz < H;
        if (!__any_sync(0xffffffffu, ok)) break;
        cplx<double> b[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) b[q] = ok ? S[(ly + Ly * q) * H + kz] : cplx<double>{0.0, 0.0};
        fft_nat_in<Ly, 8, true>(b, ly, Ty);
        if (ok) {
          const int yb = 8 * brevL<Ly>(ly);
#pragma unroll
          for (int k1 = 0; k1 < 8; ++k1) T[(k1 + yb) * H + swz<M>(kz)] = b[k1];
        }
      }
    }
    __syncthreads();  // T complete; S free
    const int y = t / Lz, l = t - y * Lz;
    const cplx<double>* row = T + y * H;
    cplx<double> a[8];
    const int k2 = brevL<Lz>(l);
#pragma unroll
    for (int k1 = 0; k1 < 8; ++k1) {
      const int k = k1 + 8 * k2;
      if (k == 0) {
        const double A = row[swz<M>(0)].x, B = row[swz<M>(M)].x;
        a[k1] = {(A + B) * 0.5, (A - B) * 0.5};
      } else {
        const cplx<double> A = row[swz<M>(k)], B = row[swz<M>(M - k)];
        const cplx<double> E{(A.x + B.x) * 0.5, (A.y - B.y) * 0.5};
        const cplx<double> D{(A.x - B.x) * 0.5, (A.y + B.y) * 0.5};
        const cplx<double> O = cmul(D, cconj(tw_n2[k]));
        a[k1] = {E.x - O.y, E.y + O.x};
      }
    }
    {
      LaneTw<Lz, 8> Tz;
      Tz.load(tw_z, l);
      fft_tr_in<Lz, 8, true>(a, l, Tz);
    }
    constexpr double norm = 2.0 / (double)NN;
    const long roff = ((long)vec * 3 + c) * NN + ((long)x * N + y) * N;
    const double2* wp2 = w ? reinterpret_cast<const double2*>(w + (long)(vec / m) * NN + ((long)x * N + y) * N) : nullptr;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (fu.p) {
      px_row<Lz>(a, norm, wp2, reinterpret_cast<double2*>(fu.x + roff), reinterpret_cast<double2*>(fu.p + roff), l,
                 fu.vs[vec].alpha, fu.vs[vec].beta);
    } else {
      double2* zp2 = reinterpret_cast<double2*>(z + roff);
      double2 ww[8];
      if (wp2)
#pragma unroll
        for (int q = 0; q < 8; ++q) ww[q] = wp2[l + Lz * q];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        double2 v{a[q].x * norm, a[q].y * norm};
        if (wp2) {
          v.x *= ww[q].x;
          v.y *= ww[q].y;
        }
        zp2[l + Lz * q] = v;
        acc[0] += v.x + v.y;
        if (partial) {
          const double2 rv = reinterpret_cast<const double2*>(r + roff)[l + Lz * q];
          acc[1] += rv.x * v.x + rv.y * v.y;
          acc[2] += rv.x + rv.y;
          acc[3] += rv.x * rv.x + rv.y * rv.y;
        }
      }
    }
    if (partial || fu.partC) {
#pragma unroll
      for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_down_sync(0xffffffffu, acc[k], o);
      if ((t & 31) == 0)
#pragma unroll
        for (int k = 0; k < 4; ++k) red[(t >> 5) * 4 + k] = acc[k];
    }
    __syncthreads();  // T reads done (next plane rewrites it); warp sums in red
    if ((partial || fu.partC) && t == 0) {
      double s4[4] = {0.0, 0.0, 0.0, 0.0};
      for (int q = 0; q < 8; ++q)
#pragma unroll
        for (int k = 0; k < 4; ++k) s4[k] += red[q * 4 + k];
      const long pl = ((long)vec * 3 + c) * N + x;
      if (partial)
#pragma unroll
        for (int k = 0; k < 4; ++k) partial[pl * 4 + k] = s4[k];
      if (fu.partC) fu.partC[pl] = s4[0];
    }
    j = jn;
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// Pass B with staged slabs (cubes of 64 only; other grids have no such variant)
template <int N>
static int launch_fb_staged(dim3 grid, cplx<double>* spec, const double* kinv, int m, const cplx<double>* twx,
                            const CellState* cs, unsigned long long* units, const PcgFuse& fu, double lam0,
                            double mu0, cudaStream_t st) {
  if constexpr (N == 64) {
    constexpr size_t sbb = (size_t)3 * N * Fast<N>::KPB * sizeof(cplx<double>);
    NLF_CUDA_TRY(raise_dyn_smem(k_fb_fast<N, true, true>, (int)sbb));
    k_fb_fast<N, true, true><<<grid, Fast<N>::NTB, sbb, st>>>(spec, kinv, m, twx, cs, units, PK_FFTB64, fu, lam0, mu0);
    NLF_CHECK_LAUNCH();
    return NLF_OK;
  } else {
    set_error("pass B: no staged variant for n = %d", N);
    return NLF_EBADARG;
  }
}

// stages: bit 0 pass A, bit 1 pass B, bit 2 pass C
template <int N>
static int launch_fast(const LinearHandle& h, int nvec, int m, double* r, double* z, cplx<double>* spec,
                       const double* w, const CellState* cs, double* partial, const PcgFuse& fu, int* nchunk,
                       int stages, cudaStream_t st) {
  using F = Fast<N>;
  const cplx<double>* tw = h.t64.tw;
  const size_t plane = F::smem_plane();
  const bool smt = h.fft_smt != 0;
  NLF_CUDA_TRY(raise_dyn_smem(k_fa_fast<N, false>, (int)plane));
  NLF_CUDA_TRY(raise_dyn_smem(k_fc_fast<N, false>, (int)plane));
  NLF_CUDA_TRY(raise_dyn_smem(k_fa_fast<N, true>, (int)plane));
  NLF_CUDA_TRY(raise_dyn_smem(k_fc_fast<N, true>, (int)plane));
  NLF_CUDA_TRY(raise_dyn_smem(k_fa_fast<N, true, true>, (int)plane));
  NLF_CUDA_TRY(raise_dyn_smem(k_fc_fast<N, true, true>, (int)plane));
  if (nchunk) *nchunk = F::KZC;
  unsigned long long* units = prof_units();
  const cplx<double>* twx = tw + h.tw.off0;
  const cplx<double>* twy = tw + h.tw.off1;
  const cplx<double>* twn2 = tw + h.tw.off2;
  const cplx<double>* twz = tw + h.tw.off2h;
  if (stages & 1) {
    ProfScope ps(PK_FFTA64, st);
    const dim3 grid(N / F::P, 3, nvec);
    if (h.fft_smt == 3)
      k_fa_fast<N, true, true><<<grid, 256, plane, st>>>(r, w, spec, m, twy, twz, twn2, cs, units, PK_FFTA64, fu);
    else if (smt)
      k_fa_fast<N, true><<<grid, 256, plane, st>>>(r, w, spec, m, twy, twz, twn2, cs, units, PK_FFTA64, fu);
    else
      k_fa_fast<N, false><<<grid, 256, plane, st>>>(r, w, spec, m, twy, twz, twn2, cs, units, PK_FFTA64, fu);
    NLF_CHECK_LAUNCH();
  }
  if (stages & 2) {
    ProfScope ps(PK_FFTB64, st);
    // the scaled preconditioner (w given) inverts its own reference medium
    const double* kinv = w ? h.t64s.kinv : h.t64.kinv;
    // the medium of the inverse: the scaled preconditioner's reference medium, else the material
    const double nu0 = w ? h.scaled_ref_nu : h.nu;
    const double lam0 = h.E * nu0 / ((1.0 + nu0) * (1.0 - 2.0 * nu0)), mu0 = h.E / (2.0 * (1.0 + nu0));
    const dim3 grid(N / F::KY, F::KZC, nvec);
    if (N == 64 && h.pcb_closed == 2) {
      NLF_TRY(launch_fb_staged<N>(grid, spec, kinv, m, twx, cs, units, fu, lam0, mu0, st));
    } else if (h.pcb_closed) {
      k_fb_fast<N, true><<<grid, F::NTB, 0, st>>>(spec, kinv, m, twx, cs, units, PK_FFTB64, fu, lam0, mu0);
    } else {
      k_fb_fast<N, false><<<grid, F::NTB, 0, st>>>(spec, kinv, m, twx, cs, units, PK_FFTB64, fu, lam0, mu0);
    }
    NLF_CHECK_LAUNCH();
  }
  if (stages & 4) {
    ProfScope ps(PK_FFTC64, st);
    if (h.fft_smt >= 2) {
      k_fc_fast<N, true, true><<<dim3(N / F::P, 3, nvec), 256, plane, st>>>(spec, w, r, z, m, twy, twz, twn2, cs,
                                                                           partial, units, PK_FFTC64, fu);
    } else if (smt) {
      k_fc_fast<N, true><<<dim3(N / F::P, 3, nvec), 256, plane, st>>>(spec, w, r, z, m, twy, twz, twn2, cs, partial,
                                                                     units, PK_FFTC64, fu);
    } else if constexpr (N == 64) {
      const size_t pipe = (size_t)3 * N * F::H * sizeof(cplx<double>);  // two staging planes and the transpose
      NLF_CUDA_TRY(raise_dyn_smem(k_fc_pipe<N>, (int)pipe));
      const long planes = (long)nvec * 3 * N;
      const int grid = (int)std::min<long>(planes, 2L * h.nsm);
      k_fc_pipe<N><<<grid, 256, pipe, st>>>(spec, w, r, z, m, nvec, twy, twz, twn2, cs, partial, units, PK_FFTC64, fu);
    } else {
      k_fc_fast<N, false><<<dim3(N / F::P, 3, nvec), 256, plane, st>>>(spec, w, r, z, m, twy, twz, twn2, cs,
                                                                      partial, units, PK_FFTC64, fu);
    }
    NLF_CHECK_LAUNCH();
  }
  return NLF_OK;
}

// the register-resident passes apply to FP64 cubes of 32 or 64 (NLF_FFT_GENERIC=1 forces the generic passes)
static int fast_n(const LinearHandle& h) {
  static const bool generic = [] {
    const char* e = std::getenv("NLF_FFT_GENERIC");
    return e && e[0] == '1';
  }();
  const Geom& g = h.g;
  if (generic || g.n0 != g.n1 || g.n1 != g.n2) return 0;
  return (g.n0 == 32 || g.n0 == 64) ? g.n0 : 0;
}

static FftDims fft_dims(const LinearHandle& h) {
  FftDims d;
  d.n0 = h.g.n0;
  d.n1 = h.g.n1;
  d.n2 = h.g.n2;
  d.n2h = h.g.n2h;
  d.rs = (d.n2 % 2 == 0) ? d.n2h : d.n2;
  d.N = h.g.N;
  d.NS = h.g.NS;
  d.off0 = h.tw.off0;
  d.off1 = h.tw.off1;
  d.off2 = h.tw.off2;
  d.off2h = h.tw.off2h;
  return d;
}

static bool any_non_pow2(const FftDims& d) {
  return !is_pow2(d.n0) || !is_pow2(d.n1) || (d.n2 % 2 == 0 ? !is_pow2(d.n2 / 2) : d.n2 > 1);
}

// kz chunk of pass B: the largest balanced chunk whose buffers (x2 with a ping-pong scratch) stay under `target`
template <typename T>
static int pick_kc(const FftDims& d, size_t target, int mult) {
  int chunks = 1;
  auto need = [&](int k) { return (size_t)3 * d.n0 * k * sizeof(cplx<T>) * mult; };
  while (chunks < d.n2h && need((d.n2h + chunks - 1) / chunks) > target) ++chunks;
  return (d.n2h + chunks - 1) / chunks;
}

template <typename T>
static cplx<T>* twiddles(const LinearHandle& h);
template <>
cplx<double>* twiddles<double>(const LinearHandle& h) { return h.t64.tw; }
template <>
cplx<float>* twiddles<float>(const LinearHandle& h) { return h.t32.tw; }
// Kinv of the material (the reference's preconditioner) or of the scaled preconditioner's reference medium
template <typename T>
static const T* kinv_table(const LinearHandle& h, bool scaled);
template <>
const double* kinv_table<double>(const LinearHandle& h, bool scaled) { return scaled ? h.t64s.kinv : h.t64.kinv; }
template <>
const float* kinv_table<float>(const LinearHandle& h, bool scaled) { return scaled ? h.t32s.kinv : h.t32.kinv; }

template <typename T>
static int precond_impl(const LinearHandle& h, int nvec, int m, T* r, T* z, cplx<T>* spec, const T* w,
                        const CellState* cs, double* partial, const PcgFuse& fu, int* nchunk, cudaStream_t st) {
  if constexpr (sizeof(T) == 8) {
    const int nf = fast_n(h);
    if (nf == 64) return launch_fast<64>(h, nvec, m, r, z, spec, w, cs, partial, fu, nchunk, 7, st);
    if (nf == 32) return launch_fast<32>(h, nvec, m, r, z, spec, w, cs, partial, fu, nchunk, 7, st);
  }
  FftDims d = fft_dims(h);
  const bool np2 = any_non_pow2(d);
  const int cap = (h.smem_optin > 0 ? h.smem_optin : 48 * 1024) - 2048;  // room for static shared memory
  const size_t plane1 = (size_t)d.n1 * d.rs * sizeof(cplx<T>);
  // Stockham ping-pong needs a scratch plane; non-power-of-two lines need it for the DFT anyway
  d.pp = 2 * plane1 <= (size_t)cap;
  const size_t plane = plane1 * ((d.pp || np2) ? 2 : 1);
  if (plane > (size_t)cap) {
    set_error("precond: a (%d x %d) plane needs %zu B of shared memory (> %d)", d.n1, d.n2, plane, cap);
    return NLF_EBADARG;
  }
  const int mult = (d.pp || np2) ? 2 : 1;
  const int kc = pick_kc<T>(d, std::min<size_t>(64 * 1024, (size_t)cap), mult);
  const size_t smemb = (size_t)3 * d.n0 * kc * sizeof(cplx<T>) * mult;
  if (nchunk) *nchunk = (d.n2h + kc - 1) / kc;
  const cplx<T>* tw = twiddles<T>(h);
  NLF_CUDA_TRY(raise_dyn_smem(k_fft_a<T>, (int)plane));
  NLF_CUDA_TRY(raise_dyn_smem(k_fft_c<T>, (int)plane));
  NLF_CUDA_TRY(raise_dyn_smem(k_fft_b<T>, (int)smemb));
  const int nt = 256;
  const bool f32 = sizeof(T) == 4;
  unsigned long long* units = prof_units();
  {
    const int kind = f32 ? PK_FFTA32 : PK_FFTA64;
    ProfScope ps(kind, st);
    k_fft_a<T><<<dim3(d.n0, 3, nvec), nt, plane, st>>>(r, w, spec, d, m, tw, cs, units, kind, fu);
    NLF_CHECK_LAUNCH();
  }
  {
    const int kind = f32 ? PK_FFTB32 : PK_FFTB64;
    ProfScope ps(kind, st);
    k_fft_b<T><<<dim3(d.n1, (d.n2h + kc - 1) / kc, nvec), nt, smemb, st>>>(spec, kinv_table<T>(h, w != nullptr), d, kc, m, tw,
                                                                          cs, units, kind, fu);
    NLF_CHECK_LAUNCH();
  }
  {
    const int kind = f32 ? PK_FFTC32 : PK_FFTC64;
    ProfScope ps(kind, st);
    k_fft_c<T><<<dim3(d.n0, 3, nvec), nt, plane, st>>>(spec, w, r, z, d, m, tw, cs, partial, units, kind, fu);
    NLF_CHECK_LAUNCH();
  }
  return NLF_OK;
}

template <typename T>
int launch_precond(const LinearHandle& h, int nvec, int m, const T* r, T* z, cplx<T>* spec, const T* w,
                   const CellState* cs, double* partial, cudaStream_t st) {
  PcgFuse fu{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  return precond_impl<T>(h, nvec, m, const_cast<T*>(r), z, spec, w, cs, partial, fu, nullptr, st);
}

template <typename T>
int launch_precond_pcg(const LinearHandle& h, int nvec, int m, T* r, const T* Ap, const VecState* vs, T* z,
                       cplx<T>* spec, const T* w, const CellState* cs, double* partA, double* partB, double* partC,
                       int* nchunk, cudaStream_t st) {
  PcgFuse fu{Ap, vs, partA, partB, partC, nullptr, nullptr};
  return precond_impl<T>(h, nvec, m, r, z, spec, w, cs, nullptr, fu, nchunk, st);
}

bool precond_fuses_px(const LinearHandle& h) { return fast_n(h) != 0; }

static int launch_fast_stages(const LinearHandle& h, int nvec, int m, double* r, cplx<double>* spec, const double* w,
                              const CellState* cs, const PcgFuse& fu, int* nchunk, int stages, cudaStream_t st) {
  const int nf = fast_n(h);
  if (nf == 64) return launch_fast<64>(h, nvec, m, r, nullptr, spec, w, cs, nullptr, fu, nchunk, stages, st);
  if (nf == 32) return launch_fast<32>(h, nvec, m, r, nullptr, spec, w, cs, nullptr, fu, nchunk, stages, st);
  set_error("fused pass C: no register-resident passes for a %d x %d x %d grid", h.g.n0, h.g.n1, h.g.n2);
  return NLF_EBADARG;
}

int launch_precond_pcg_ab(const LinearHandle& h, int nvec, int m, double* r, const double* Ap, const VecState* vs,
                          cplx<double>* spec, const double* w, const CellState* cs, double* partA, double* partB,
                          int* nchunk, cudaStream_t st) {
  PcgFuse fu{Ap, vs, partA, partB, nullptr, nullptr, nullptr};
  return launch_fast_stages(h, nvec, m, r, spec, w, cs, fu, nchunk, 3, st);
}

int launch_precond_pcg_cpx(const LinearHandle& h, int nvec, int m, cplx<double>* spec, const double* w,
                           const VecState* vs, const CellState* cs, double* x, double* p, cudaStream_t st) {
  PcgFuse fu{nullptr, vs, nullptr, nullptr, nullptr, x, p};
  return launch_fast_stages(h, nvec, m, nullptr, spec, w, cs, fu, nullptr, 4, st);
}

template int launch_precond_pcg<float>(const LinearHandle&, int, int, float*, const float*, const VecState*, float*,
                                       cplx<float>*, const float*, const CellState*, double*, double*, double*, int*,
                                       cudaStream_t);
template int launch_precond_pcg<double>(const LinearHandle&, int, int, double*, const double*, const VecState*,
                                        double*, cplx<double>*, const double*, const CellState*, double*, double*,
                                        double*, int*, cudaStream_t);

template int launch_precond<float>(const LinearHandle&, int, int, const float*, float*, cplx<float>*,
                                   const float*, const CellState*, double*, cudaStream_t);
template int launch_precond<double>(const LinearHandle&, int, int, const double*, double*, cplx<double>*,
                                    const double*, const CellState*, double*, cudaStream_t);

// ---- tables ----------------------------------------------------------------------------------------------------
__global__ void k_kinv(const double* __restrict__ W27, int n0, int n1, int n2, int n2h, double* __restrict__ k64,
                       float* __restrict__ k32) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long NS = (long)n0 * n1 * n2h;
  if (idx >= NS) return;
  const int kz = (int)(idx % n2h), ky = (int)((idx / n2h) % n1), kx = (int)(idx / ((long)n2h * n1));
  double K[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) K[q] = 0.0;
  for (int dx = -1; dx <= 1; ++dx)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dz = -1; dz <= 1; ++dz) {
        // cos(2 pi (kx dx / n0 + ky dy / n1 + kz dz / n2)), with the phase reduced to [0, 1) turns
        double ph = (double)((kx * dx) % n0 + n0) / n0 + (double)((ky * dy) % n1 + n1) / n1 +
                    (double)((kz * dz) % n2 + n2) / n2;
        ph -= floor(ph);
        const double cs = cospi(2.0 * ph);
        const double* Wd = W27 + ((dx + 1) * 9 + (dy + 1) * 3 + (dz + 1)) * 9;
#pragma unroll
        for (int q = 0; q < 9; ++q) K[q] += Wd[q] * cs;
      }
  double out[6];
  if (idx == 0) {
    for (int q = 0; q < 6; ++q) out[q] = 0.0;
  } else {
    // symmetric part (the antisymmetric part cancels analytically) + regularisation
    const double a = K[0], b = 0.5 * (K[1] + K[3]), c = 0.5 * (K[2] + K[6]);
    const double d = K[4], e = 0.5 * (K[5] + K[7]), f = K[8];
    const double reg = 1e-12 * fabs(a + d + f);
    const double A = a + reg, D = d + reg, F = f + reg;
    // inverse of [[A b c] [b D e] [c e F]]
    const double c00 = D * F - e * e, c01 = c * e - b * F, c02 = b * e - c * D;
    const double c11 = A * F - c * c, c12 = b * c - A * e, c22 = A * D - b * b;
    const double det = A * c00 + b * c01 + c * c02;
    const double id = 1.0 / det;
    out[0] = c00 * id;  // xx
    out[1] = c11 * id;  // yy
    out[2] = c22 * id;  // zz
    out[3] = c12 * id;  // yz
    out[4] = c02 * id;  // xz
    out[5] = c01 * id;  // xy
  }
  for (int q = 0; q < 6; ++q) {
    k64[idx * 6 + q] = out[q];
    k32[idx * 6 + q] = (float)out[q];
  }
}

// Kinv (FP64 and FP32) of the unit-stiffness operator with stencil W, into k64 and k32 (NS x 6 each)
int kinv_tables(const LinearHandle& h, const double (&W)[27][9], double* k64, float* k32) {
  const Geom& g = h.g;
  double* dW = nullptr;
  NLF_CUDA_TRY(cudaMalloc(&dW, sizeof(W)));
  cudaError_t e = cudaMemcpy(dW, W, sizeof(W), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_kinv<<<(unsigned)((g.NS + 255) / 256), 256>>>(dW, g.n0, g.n1, g.n2, g.n2h, k64, k32);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  cudaFree(dW);
  if (e != cudaSuccess) {
    set_error("kinv table: %s", cudaGetErrorString(e));
    return NLF_ECUDA;
  }
  return NLF_OK;
}

int build_tables(LinearHandle& h) {
  const Geom& g = h.g;
  // twiddles: lengths n0, n1, n2, n2/2 (full circles, e^{-2 pi i k / L}, k < L)
  std::vector<double> twr, twi;
  auto add = [&](int L) {
    const int off = (int)twr.size();
    for (int k = 0; k < L; ++k) {
      const double a = -2.0 * 3.14159265358979323846 * (double)k / (double)L;
      twr.push_back(std::cos(a));
      twi.push_back(std::sin(a));
    }
    return off;
  };
  h.tw.off0 = add(g.n0);
  h.tw.off1 = add(g.n1);
  h.tw.off2 = add(g.n2);
  h.tw.off2h = add(g.n2 % 2 == 0 ? g.n2 / 2 : 1);
  h.tw.total = (int)twr.size();
  std::vector<cplx<double>> t64(twr.size());
  std::vector<cplx<float>> t32(twr.size());
  for (size_t i = 0; i < twr.size(); ++i) {
    t64[i] = {twr[i], twi[i]};
    t32[i] = {(float)twr[i], (float)twi[i]};
  }
  NLF_CUDA_TRY(cudaMalloc(&h.t64.tw, t64.size() * sizeof(cplx<double>)));
  NLF_CUDA_TRY(cudaMalloc(&h.t32.tw, t32.size() * sizeof(cplx<float>)));
  NLF_CUDA_TRY(cudaMemcpy(h.t64.tw, t64.data(), t64.size() * sizeof(cplx<double>), cudaMemcpyHostToDevice));
  NLF_CUDA_TRY(cudaMemcpy(h.t32.tw, t32.data(), t32.size() * sizeof(cplx<float>), cudaMemcpyHostToDevice));
  NLF_CUDA_TRY(cudaMalloc(&h.t64.kinv, g.NS * 6 * sizeof(double)));
  NLF_CUDA_TRY(cudaMalloc(&h.t32.kinv, g.NS * 6 * sizeof(float)));
  NLF_CUDA_TRY(cudaMalloc(&h.t64s.kinv, g.NS * 6 * sizeof(double)));
  NLF_CUDA_TRY(cudaMalloc(&h.t32s.kinv, g.NS * 6 * sizeof(float)));
  NLF_TRY(kinv_tables(h, h.W27, h.t64.kinv, h.t32.kinv));
  return kinv_tables(h, h.W27s, h.t64s.kinv, h.t32s.kinv);
}

}  // namespace nlf
