// Binary cells on the GPU: the binarization of a smoothed density field with floating solid removed
// (nlfiber/density.py:96-149 DensityMap.binary, upsample_periodic, _dilate_periodic) and the periodic
// connected components it relies on (nlfiber/topology.py:8-63 periodic_label, spanning, remove_floating).
//
//   upsample   periodic multilinear resampling of the cell-centred field to side m (axis by axis, numpy's
//              arithmetic: (1 - w) a + w b without contraction), then exact_symmetrize: fold the 2^d mirror
//              images (0.5 (a + b) axis by axis), sum the d! axis permutations in itertools order, / d!, one
//              value per symmetry orbit copied to the whole cell of side 2 (m / 2)
//   threshold  b = u > quantile(u, 1 - v) (numpy's "linear" quantile: two order statistics by radix select on
//              the device, the interpolation on the host)
//   label      periodic connected components (26 / 8 neighbours, or 6 / 4 faces) by lock-free union-find:
//              every label points to a smaller voxel index (L[x] <= x), a union links the larger root to the
//              smaller with atomicMin and, when another thread got there first, carries on with the root it
//              found, so every loop ends (each failed link lowers the larger of the two roots)
//   spanning   a component is kept if it touches every slice along every axis: a bitmap of slices per
//              component and axis, filled with warp-aggregated atomicOr
//   grow       the kept solid loses volume; it grows back through the void voxels touching it (the periodic
//              3^d dilation minus the solid), highest u first: the k-th largest u on the front by radix select
//
// Voxel i of a cell of side n is (x, y, z) in C order (z fastest; squares (x, y)). Labels are int32, so a cell
// holds fewer than 2^31 voxels.
#include <algorithm>
#include <cmath>
#include <climits>
#include <cstring>

#include "nlf_common.cuh"
#include "nlf_internal.h"
#include "../../include/nlf.h"

namespace nlf {
namespace {

constexpr int kTpThreads = 256;
constexpr int kScanThreads = 1024;

bool tp_on_dev(const void* p) {
  if (!p) return false;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

size_t tp_al(size_t b) { return (b + 255) & ~(size_t)255; }

// order-preserving map of doubles to unsigned keys (ascending keys = ascending values; no NaNs here)
__device__ __forceinline__ unsigned long long okey(double x) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double from_okey(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)b);
}

struct Cell {
  int d, n;
  long N;
};

__device__ __forceinline__ void coords(const Cell& c, long i, int* x) {
  if (c.d == 3) {
    x[2] = (int)(i % c.n);
    x[1] = (int)((i / c.n) % c.n);
    x[0] = (int)(i / ((long)c.n * c.n));
  } else {
    x[1] = (int)(i % c.n);
    x[0] = (int)(i / c.n);
    x[2] = 0;
  }
}
__device__ __forceinline__ long vox(const Cell& c, int x0, int x1, int x2) {
  return c.d == 3 ? ((long)x0 * c.n + x1) * c.n + x2 : (long)x0 * c.n + x1;
}
__device__ __forceinline__ int wrapn(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// CTA-wide count of a predicate added to *cnt (every thread of the CTA must call it)
__device__ __forceinline__ void cta_count(bool f, unsigned long long* cnt) {
  const int c = __syncthreads_count(f);
  if (threadIdx.x == 0 && c) atomicAdd(cnt, (unsigned long long)c);
}

// ---- threshold, front, grow, keep -------------------------------------------------------------------------
__global__ void k_tp_threshold(long N, const double* __restrict__ u, double thr, uint8_t* __restrict__ b,
                               unsigned long long* cnt) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  bool f = false;
  if (i < N) {
    f = u[i] > thr;
    b[i] = f;
  }
  cta_count(f, cnt);
}

// front = (3^d dilation of b) and not b (nlfiber/density.py:125-130 _dilate_periodic, then & ~b)
__global__ void k_tp_front(Cell c, const uint8_t* __restrict__ b, uint8_t* __restrict__ front,
                           unsigned long long* cnt) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  bool f = false;
  if (i < c.N && !b[i]) {
    int x[3];
    coords(c, i, x);
    const int r2 = c.d == 3 ? 1 : 0;
    for (int a = -1; a <= 1 && !f; ++a)
      for (int e = -1; e <= 1 && !f; ++e)
        for (int g = -r2; g <= r2 && !f; ++g)
          f = b[vox(c, wrapn(x[0] + a, c.n), wrapn(x[1] + e, c.n), c.d == 3 ? wrapn(x[2] + g, c.n) : 0)] != 0;
  }
  if (i < c.N) front[i] = f;
  cta_count(f, cnt);
}

// b |= front & (u >= t); counts the solid voxels after the growth
__global__ void k_tp_grow(long N, const double* __restrict__ u, const uint8_t* __restrict__ front, double t,
                          uint8_t* __restrict__ b, unsigned long long* cnt) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  bool f = false;
  if (i < N) {
    f = b[i] != 0;
    if (!f && front[i] && u[i] >= t) {
      f = true;
      b[i] = 1;
    }
  }
  cta_count(f, cnt);
}

// ---- union-find labelling -----------------------------------------------------------------------------------
__global__ void k_tp_label_init(long N, const uint8_t* __restrict__ b, int* __restrict__ L) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < N) L[i] = b[i] ? (int)i : -1;
}

// root of a: labels only ever decrease and L[x] <= x, so the walk ends; reads bypass L1 (other SMs link roots)
__device__ __forceinline__ int tp_find(const int* L, int a) {
  int p = __ldcg(L + a);
  while (p != a) {
    a = p;
    p = __ldcg(L + a);
  }
  return a;
}

// joins the sets of a and b: link the larger root to the smaller one; when the larger root was linked elsewhere
// meanwhile (atomicMin returns old < it), carry on uniting with that label, which keeps the overwritten link's
// connection. Each failed round lowers max(a, b) strictly, so the loop ends.
__device__ __forceinline__ void tp_unite(int* L, int a, int b) {
  while (true) {
    a = tp_find(L, a);
    b = tp_find(L, b);
    if (a == b) return;
    if (a > b) {
      const int t = a;
      a = b;
      b = t;
    }
    const int old = atomicMin(L + b, a);
    if (old == b) return;
    b = old;
  }
}

// one thread per solid voxel, unions with its solid neighbours at the forward half of the neighbourhood
// (offsets whose first nonzero component is positive; periodic), faces only when `faces`
__global__ void k_tp_label_merge(Cell c, int faces, const uint8_t* __restrict__ b, int* L) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= c.N || !b[i]) return;
  int x[3];
  coords(c, i, x);
  const int r2 = c.d == 3 ? 1 : 0;
  for (int a = 0; a <= 1; ++a)
    for (int e = -1; e <= 1; ++e)
      for (int g = -r2; g <= r2; ++g) {
        if (a == 0 && (e < 0 || (e == 0 && g <= 0))) continue;  // forward half only
        if (faces && (a != 0) + (e != 0) + (g != 0) != 1) continue;
        const long j = vox(c, wrapn(x[0] + a, c.n), wrapn(x[1] + e, c.n), c.d == 3 ? wrapn(x[2] + g, c.n) : 0);
        if (j != i && b[j]) tp_unite(L, (int)i, (int)j);
      }
}

__global__ void k_tp_label_flatten(long N, int* L) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < N && L[i] >= 0) L[i] = tp_find(L, (int)i);
}

// component numbering in the order of the roots (each component's smallest voxel index): roots per CTA, an
// exclusive scan of those counts, then each root's rank
__global__ void k_tp_root_count(long N, const int* __restrict__ L, int* __restrict__ bc) {
  const long i = blockIdx.x * (long)kScanThreads + threadIdx.x;
  const int c = __syncthreads_count(i < N && L[i] == (int)i);
  if (threadIdx.x == 0) bc[blockIdx.x] = c;
}

__global__ void k_tp_scan(int nb, int* bc, int* total) {
  __shared__ int ws[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int base = 0; base < nb; base += kScanThreads) {
    const int i = base + threadIdx.x;
    const int v = i < nb ? bc[i] : 0;
    int s = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += t;
    }
    if (lane == 31) ws[w] = s;
    __syncthreads();
    if (w == 0) {
      int q = ws[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, q, o);
        if (lane >= o) q += t;
      }
      ws[lane] = q;
    }
    __syncthreads();
    const int incl = s + (w > 0 ? ws[w - 1] : 0) + carry;
    if (i < nb) bc[i] = incl - v;
    __syncthreads();
    if (threadIdx.x == kScanThreads - 1) carry = incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void k_tp_root_assign(long N, const int* __restrict__ L, const int* __restrict__ boff,
                                 int* __restrict__ rid) {
  __shared__ int wc[32];
  const long i = blockIdx.x * (long)kScanThreads + threadIdx.x;
  const bool f = i < N && L[i] == (int)i;
  const unsigned m = __ballot_sync(0xffffffffu, f);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) wc[w] = __popc(m);
  __syncthreads();
  int off = boff[blockIdx.x];
  for (int q = 0; q < w; ++q) off += wc[q];
  if (f) rid[i] = off + __popc(m & ((1u << lane) - 1));
}

// labels 1..ncomp (0 for void)
__global__ void k_tp_labels_out(long N, const int* __restrict__ L, const int* __restrict__ rid,
                                int* __restrict__ lab) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < N) lab[i] = L[i] >= 0 ? rid[L[i]] + 1 : 0;
}

// slices touched per component and axis: bit (x_a mod 32) of word x_a / 32 of row (id, a); lanes that hit the
// same word OR their bits first (all 32 lanes of a warp run this: the grid covers whole warps)
__global__ void k_tp_touch(Cell c, const int* __restrict__ L, const int* __restrict__ rid, int W,
                           unsigned* __restrict__ touch) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const bool have = i < c.N && L[i] >= 0;
  int x[3] = {0, 0, 0};
  int id = 0;
  if (have) {
    coords(c, i, x);
    id = rid[L[i]];
  }
  const int lane = threadIdx.x & 31;
  for (int a = 0; a < c.d; ++a) {
    const long long key = have ? ((long long)id * c.d + a) * W + (x[a] >> 5) : -1ll;
    const unsigned bit = have ? 1u << (x[a] & 31) : 0u;
    const unsigned grp = __match_any_sync(0xffffffffu, key);
    const unsigned v = __reduce_or_sync(grp, bit);
    if (have && lane == __ffs(grp) - 1) atomicOr(touch + key, v);
  }
}

__global__ void k_tp_span(int ncomp, int d, int n, int W, const unsigned* __restrict__ touch,
                          uint8_t* __restrict__ span, int* nspan) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= ncomp) return;
  bool ok = true;
  for (int a = 0; a < d && ok; ++a)
    for (int w = 0; w < W && ok; ++w) {
      const int bits = (w == W - 1) ? n - 32 * w : 32;
      const unsigned want = bits >= 32 ? 0xffffffffu : ((1u << bits) - 1u);
      ok = touch[((long)id * d + a) * W + w] == want;
    }
  span[id] = ok;
  if (ok) atomicAdd(nspan, 1);
}

__global__ void k_tp_keep(long N, const int* __restrict__ L, const int* __restrict__ rid,
                          const uint8_t* __restrict__ span, uint8_t* __restrict__ b, unsigned long long* cnt) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  bool f = false;
  if (i < N && L[i] >= 0) {
    f = span[rid[L[i]]] != 0;
    b[i] = f;
  }
  cta_count(f, cnt);
}

// ---- order statistics: radix select over 8-bit digits of the ordered keys ---------------------------------------
struct SelState {
  unsigned long long prefix;  // digits chosen so far
  long long rank;             // rank still to skip among the keys that match the prefix
  double value;               // the selected value after the last digit
  int err;                    // 1: rank beyond the count
  int pad_;
};

__global__ void k_tp_sel_hist(long N, const double* __restrict__ u, const uint8_t* __restrict__ mask,
                              const SelState* __restrict__ st, int shift, unsigned* __restrict__ hist) {
  __shared__ unsigned sh[256];
  for (int t = threadIdx.x; t < 256; t += blockDim.x) sh[t] = 0;
  __syncthreads();
  const unsigned long long hm = shift >= 56 ? 0ull : (~0ull << (shift + 8));
  const unsigned long long want = st->prefix & hm;
  const long stride = (long)gridDim.x * blockDim.x;
  for (long base = (long)blockIdx.x * blockDim.x; base < N; base += stride) {  // uniform per warp
    const long i = base + threadIdx.x;
    int bin = 256;
    if (i < N && (!mask || mask[i])) {
      const unsigned long long k = okey(u[i]);
      if ((k & hm) == want) bin = (int)((k >> shift) & 255ull);
    }
    const unsigned grp = __match_any_sync(0xffffffffu, bin);
    if (bin < 256 && (threadIdx.x & 31) == __ffs(grp) - 1) atomicAdd(sh + bin, (unsigned)__popc(grp));
  }
  __syncthreads();
  for (int t = threadIdx.x; t < 256; t += blockDim.x)
    if (sh[t]) atomicAdd(hist + t, sh[t]);
}

// picks the digit whose bin holds the remaining rank, clears the histogram for the next digit
__global__ void k_tp_sel_pick(SelState* st, unsigned* hist, int shift) {
  if (threadIdx.x == 0) {
    long long r = st->rank;
    int bin = -1;
    for (int q = 0; q < 256; ++q) {
      const long long c = hist[q];
      if (r < c) {
        bin = q;
        break;
      }
      r -= c;
    }
    if (bin < 0) {
      st->err = 1;
    } else {
      st->prefix |= (unsigned long long)bin << shift;
      st->rank = r;
      if (shift == 0) st->value = from_okey(st->prefix);
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < 256; t += blockDim.x) hist[t] = 0;
}

// ---- upsampling and exact symmetrization ------------------------------------------------------------------------
// nlfiber/density.py:133-149: the source position of output index X of side m, as numpy computes it:
// x = (X + 0.5) * n / m - 0.5, i0 = floor(x), w = x - i0; taps i0 mod n and (i0 + 1) mod n
struct Tap {
  int i0, i1;
  double w, w1;  // w and 1 - w
};
__device__ __forceinline__ Tap up_tap(int X, int n, int m) {
  const double x = __dsub_rn(__ddiv_rn(__dmul_rn(__dadd_rn((double)X, 0.5), (double)n), (double)m), 0.5);
  const double f = floor(x);
  Tap t;
  const int i0 = (int)f;
  t.w = __dsub_rn(x, f);
  t.w1 = __dsub_rn(1.0, t.w);
  t.i0 = ((i0 % n) + n) % n;
  t.i1 = (((i0 + 1) % n) + n) % n;
  return t;
}
// (1 - w) a + w b with numpy's rounding (two products, one sum; no fused multiply-add)
__device__ __forceinline__ double up_lerp(const Tap& t, double a, double b) {
  return __dadd_rn(__dmul_rn(t.w1, a), __dmul_rn(t.w, b));
}

// value of the upsampled field at output index (X0, X1, X2) of side m: lerps along axis 0, then 1, then 2
__device__ double up_at3(const double* __restrict__ u, int n, int m, int X0, int X1, int X2) {
  const Tap a = up_tap(X0, n, m), b = up_tap(X1, n, m), c = up_tap(X2, n, m);
  auto U = [&](int i, int j, int k) { return __ldg(u + ((long)i * n + j) * n + k); };
  auto s0 = [&](int j, int k) { return up_lerp(a, U(a.i0, j, k), U(a.i1, j, k)); };
  auto s1 = [&](int k) { return up_lerp(b, s0(b.i0, k), s0(b.i1, k)); };
  return up_lerp(c, s1(c.i0), s1(c.i1));
}
__device__ double up_at2(const double* __restrict__ u, int n, int m, int X0, int X1) {
  const Tap a = up_tap(X0, n, m), b = up_tap(X1, n, m);
  auto U = [&](int i, int j) { return __ldg(u + (long)i * n + j); };
  auto s0 = [&](int j) { return up_lerp(a, U(a.i0, j), U(a.i1, j)); };
  return up_lerp(b, s0(b.i0), s0(b.i1));
}

// one thread per point of the octant (h = m / 2 per axis) whose indices are sorted: the exact_symmetrize value of
// its orbit (fold over the 2^d mirror images of the side-2h cell axis by axis, then the d! permutations added in
// itertools order and divided by d!; nlfiber/symmetry.py:44-65)
__global__ void k_tp_up_orbit(int d, int n, int m, const double* __restrict__ u, double* __restrict__ oct) {
  const int h = m / 2, s = 2 * h;
  const long NO = d == 3 ? (long)h * h * h : (long)h * h;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= NO) return;
  if (d == 3) {
    const int c = (int)(t % h), b = (int)((t / h) % h), a = (int)(t / ((long)h * h));
    if (!(a <= b && b <= c)) return;
    auto f0 = [&](int i, int j, int k) {
      return __dmul_rn(0.5, __dadd_rn(up_at3(u, n, m, i, j, k), up_at3(u, n, m, s - 1 - i, j, k)));
    };
    auto f1 = [&](int i, int j, int k) { return __dmul_rn(0.5, __dadd_rn(f0(i, j, k), f0(i, s - 1 - j, k))); };
    auto F = [&](int i, int j, int k) { return __dmul_rn(0.5, __dadd_rn(f1(i, j, k), f1(i, j, s - 1 - k))); };
    double v = F(a, b, c);
    v = __dadd_rn(v, F(a, c, b));
    v = __dadd_rn(v, F(b, a, c));
    v = __dadd_rn(v, F(c, a, b));
    v = __dadd_rn(v, F(b, c, a));
    v = __dadd_rn(v, F(c, b, a));
    oct[t] = __ddiv_rn(v, 6.0);
  } else {
    const int b = (int)(t % h), a = (int)(t / h);
    if (a > b) return;
    auto f0 = [&](int i, int j) {
      return __dmul_rn(0.5, __dadd_rn(up_at2(u, n, m, i, j), up_at2(u, n, m, s - 1 - i, j)));
    };
    auto F = [&](int i, int j) { return __dmul_rn(0.5, __dadd_rn(f0(i, j), f0(i, s - 1 - j))); };
    oct[t] = __ddiv_rn(__dadd_rn(F(a, b), F(b, a)), 2.0);
  }
}

// the full cell of side 2h: each voxel takes its orbit's value (mirror into the octant, sort the indices)
__global__ void k_tp_up_scatter(int d, int h, const double* __restrict__ oct, double* __restrict__ out) {
  const int s = 2 * h;
  const long N = d == 3 ? (long)s * s * s : (long)s * s;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= N) return;
  int x[3] = {0, 0, 0};
  if (d == 3) {
    x[2] = (int)(t % s);
    x[1] = (int)((t / s) % s);
    x[0] = (int)(t / ((long)s * s));
  } else {
    x[1] = (int)(t % s);
    x[0] = (int)(t / s);
  }
  for (int a = 0; a < d; ++a) x[a] = x[a] < h ? x[a] : s - 1 - x[a];
  if (d == 3) {
    int p = x[0], q = x[1], r = x[2], w;
    if (p > q) { w = p; p = q; q = w; }
    if (q > r) { w = q; q = r; r = w; }
    if (p > q) { w = p; p = q; q = w; }
    out[t] = oct[((long)p * h + q) * h + r];
  } else {
    const int p = min(x[0], x[1]), q = max(x[0], x[1]);
    out[t] = oct[(long)p * h + q];
  }
}

inline unsigned nblk(long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// numpy's "linear" quantile (Hyndman-Fan method 7) of n sorted values, as numpy 2 evaluates it: virtual index
// (n - 1) q, previous = floor, next = previous + 1 (both the last value when the index reaches n - 1, both the
// first when it is negative), gamma = index - previous, then a + (b - a) gamma, or b - (b - a)(1 - gamma) when
// gamma >= 0.5. `value(k)` gives the k-th smallest.
template <typename F>
static int quantile_linear(long long n, double q, F value, double* out) {
  const double vi = (double)(n - 1) * q;
  long long prev, next;
  if (vi >= (double)(n - 1)) {
    prev = next = n - 1;
  } else if (vi < 0.0) {
    prev = next = 0;
  } else {
    prev = (long long)std::floor(vi);
    next = prev + 1;
  }
  const double pidx = vi >= (double)(n - 1) ? -1.0 : (vi < 0.0 ? 0.0 : (double)prev);
  const double g = vi - pidx;
  double a, b;
  NLF_TRY(value(prev, &a));
  if (next == prev) {
    b = a;
  } else {
    NLF_TRY(value(next, &b));
  }
  // each product rounded on its own (volatile keeps a host compiler from fusing it into the sum)
  const double diff = b - a;
  volatile double p = diff * g;
  double r = a + p;
  if (g >= 0.5) {
    volatile double p1 = diff * (1.0 - g);
    r = b - p1;
  }
  *out = r;
  return NLF_OK;
}

}  // namespace nlf

using namespace nlf;

struct nlf_topo {
  int d = 3, n = 0;
  long N = 0;
  int nb = 0;                  // CTAs of kScanThreads voxels (root numbering)
  int* L = nullptr;            // [N] union-find labels (-1 void)
  int* rid = nullptr;          // [N] component number of each root
  int* bc = nullptr;           // [nb + 1] roots per CTA, then their exclusive scan; [nb] the total
  uint8_t* front = nullptr;    // [N]
  uint8_t* bst = nullptr;      // [N] staging of a host b
  double* ust = nullptr;       // [N] staging of a host u
  unsigned* hist = nullptr;    // [256]
  SelState* sel = nullptr;
  unsigned long long* cnt = nullptr;  // [4] device counters
  int* nspan = nullptr;
  DevBuf touch;                // [ncomp][d][W] slice bitmaps
  DevBuf span;                 // [ncomp]
  DevBuf lab;                  // int32 staging of host labels
  void* pin = nullptr;         // pinned host scalars
};

namespace {

struct Pinned {
  unsigned long long cnt[4];
  SelState sel;
  int total;
  int nspan;
};

int tp_sync_read(nlf_topo* T, cudaStream_t st) {
  Pinned* P = (Pinned*)T->pin;
  NLF_CUDA_TRY(cudaMemcpyAsync(P->cnt, T->cnt, sizeof(P->cnt), cudaMemcpyDeviceToHost, st));
  NLF_CUDA_TRY(cudaMemcpyAsync(&P->sel, T->sel, sizeof(SelState), cudaMemcpyDeviceToHost, st));
  NLF_CUDA_TRY(cudaMemcpyAsync(&P->total, T->bc + T->nb, sizeof(int), cudaMemcpyDeviceToHost, st));
  NLF_CUDA_TRY(cudaMemcpyAsync(&P->nspan, T->nspan, sizeof(int), cudaMemcpyDeviceToHost, st));
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  return NLF_OK;
}

Cell tp_cell(const nlf_topo* T) { return Cell{T->d, T->n, T->N}; }

// union-find labels of b (L), component numbers of the roots (rid) and their count (synchronizes)
int tp_label(nlf_topo* T, const uint8_t* b, int faces, int* ncomp, cudaStream_t st) {
  const Cell c = tp_cell(T);
  const unsigned g = nblk(T->N, kTpThreads);
  k_tp_label_init<<<g, kTpThreads, 0, st>>>(T->N, b, T->L);
  k_tp_label_merge<<<g, kTpThreads, 0, st>>>(c, faces, b, T->L);
  k_tp_label_flatten<<<g, kTpThreads, 0, st>>>(T->N, T->L);
  k_tp_root_count<<<T->nb, kScanThreads, 0, st>>>(T->N, T->L, T->bc);
  k_tp_scan<<<1, kScanThreads, 0, st>>>(T->nb, T->bc, T->bc + T->nb);
  k_tp_root_assign<<<T->nb, kScanThreads, 0, st>>>(T->N, T->L, T->bc, T->rid);
  NLF_CHECK_LAUNCH();
  NLF_TRY(tp_sync_read(T, st));
  *ncomp = ((Pinned*)T->pin)->total;
  return NLF_OK;
}

// nlfiber/topology.py:57-63 on b in place: keep the spanning components; returns the kept solid count
int tp_remove_floating(nlf_topo* T, uint8_t* b, int* ncomp_out, int* nspan_out, long long* nsolid,
                       cudaStream_t st) {
  int ncomp = 0;
  NLF_TRY(tp_label(T, b, 0, &ncomp, st));
  const int W = (T->n + 31) / 32;
  const size_t tb = (size_t)(ncomp > 0 ? ncomp : 1) * T->d * W * sizeof(unsigned);
  NLF_TRY(T->touch.reserve(tb));
  NLF_TRY(T->span.reserve((size_t)(ncomp > 0 ? ncomp : 1)));
  NLF_CUDA_TRY(cudaMemsetAsync(T->touch.ptr, 0, tb, st));
  NLF_CUDA_TRY(cudaMemsetAsync(T->nspan, 0, sizeof(int), st));
  NLF_CUDA_TRY(cudaMemsetAsync(T->cnt, 0, 4 * sizeof(unsigned long long), st));
  const Cell c = tp_cell(T);
  const unsigned g = nblk(T->N, kTpThreads);
  if (ncomp > 0) {
    k_tp_touch<<<g, kTpThreads, 0, st>>>(c, T->L, T->rid, W, (unsigned*)T->touch.ptr);
    k_tp_span<<<nblk(ncomp, kTpThreads), kTpThreads, 0, st>>>(ncomp, T->d, T->n, W, (const unsigned*)T->touch.ptr,
                                                              (uint8_t*)T->span.ptr, T->nspan);
    k_tp_keep<<<g, kTpThreads, 0, st>>>(T->N, T->L, T->rid, (const uint8_t*)T->span.ptr, b, T->cnt);
    NLF_CHECK_LAUNCH();
  }
  NLF_TRY(tp_sync_read(T, st));
  const Pinned* P = (const Pinned*)T->pin;
  if (ncomp_out) *ncomp_out = ncomp;
  if (nspan_out) *nspan_out = ncomp > 0 ? P->nspan : 0;
  *nsolid = ncomp > 0 ? (long long)P->cnt[0] : 0;
  return NLF_OK;
}

// the rank-th smallest (0-based) of u over the voxels where mask is set (all when mask is NULL); synchronizes
int tp_select(nlf_topo* T, const double* u, const uint8_t* mask, long long rank, double* value, cudaStream_t st) {
  SelState s0{};
  s0.rank = rank;
  NLF_CUDA_TRY(cudaMemcpyAsync(T->sel, &s0, sizeof(SelState), cudaMemcpyHostToDevice, st));
  NLF_CUDA_TRY(cudaMemsetAsync(T->hist, 0, 256 * sizeof(unsigned), st));
  const unsigned g = (unsigned)std::min<long>(nblk(T->N, kTpThreads), 148L * 8);
  for (int shift = 56; shift >= 0; shift -= 8) {
    k_tp_sel_hist<<<g, kTpThreads, 0, st>>>(T->N, u, mask, T->sel, shift, T->hist);
    k_tp_sel_pick<<<1, 256, 0, st>>>(T->sel, T->hist, shift);
  }
  NLF_CHECK_LAUNCH();
  NLF_TRY(tp_sync_read(T, st));
  const Pinned* P = (const Pinned*)T->pin;
  if (P->sel.err) {
    set_error("nlf_topo_select: rank %lld beyond the selected voxels", rank);
    return NLF_EBADARG;
  }
  *value = P->sel.value;
  return NLF_OK;
}

int tp_count_reset(nlf_topo* T, cudaStream_t st) {
  NLF_CUDA_TRY(cudaMemsetAsync(T->cnt, 0, 4 * sizeof(unsigned long long), st));
  return NLF_OK;
}

}  // namespace

NLF_API int nlf_topo_create(nlf_topo** out, int d, int n) {
  if (!out || (d != 2 && d != 3) || n < 1 || (d == 3 ? (long)n * n * n : (long)n * n) > (1L << 30)) {
    set_error("nlf_topo_create: bad arguments (d 2 or 3, n >= 1, at most 2^30 voxels)");
    return NLF_EBADARG;
  }
  *out = nullptr;
  nlf_topo* T = new nlf_topo();
  T->d = d;
  T->n = n;
  T->N = d == 3 ? (long)n * n * n : (long)n * n;
  T->nb = (int)nblk(T->N, kScanThreads);
  const size_t N = (size_t)T->N;
  const size_t o_L = 0, o_rid = tp_al(o_L + N * 4), o_bc = tp_al(o_rid + N * 4),
               o_front = tp_al(o_bc + (size_t)(T->nb + 1) * 4), o_bst = tp_al(o_front + N),
               o_ust = tp_al(o_bst + N), o_hist = tp_al(o_ust + N * 8), o_sel = tp_al(o_hist + 256 * 4),
               o_cnt = tp_al(o_sel + sizeof(SelState)), o_ns = tp_al(o_cnt + 4 * 8), total = tp_al(o_ns + 4);
  char* base = nullptr;
  if (cudaMalloc(&base, total) != cudaSuccess || cudaMallocHost(&T->pin, sizeof(Pinned)) != cudaSuccess) {
    cudaGetLastError();
    if (base) cudaFree(base);
    delete T;
    set_error("nlf_topo_create: out of memory (%zu bytes)", total);
    return NLF_ECUDA;
  }
  T->L = (int*)(base + o_L);
  T->rid = (int*)(base + o_rid);
  T->bc = (int*)(base + o_bc);
  T->front = (uint8_t*)(base + o_front);
  T->bst = (uint8_t*)(base + o_bst);
  T->ust = (double*)(base + o_ust);
  T->hist = (unsigned*)(base + o_hist);
  T->sel = (SelState*)(base + o_sel);
  T->cnt = (unsigned long long*)(base + o_cnt);
  T->nspan = (int*)(base + o_ns);
  *out = T;
  return NLF_OK;
}

NLF_API int nlf_topo_destroy(nlf_topo* T) {
  if (!T) return NLF_OK;
  cudaFree(T->L);
  if (T->pin) cudaFreeHost(T->pin);
  T->touch.release();
  T->span.release();
  T->lab.release();
  delete T;
  return NLF_OK;
}

NLF_API int nlf_topo_label(nlf_topo* T, const uint8_t* b, int faces, int32_t* labels, int* ncomp, void* stream) {
  if (!T || !b || !labels || !ncomp) {
    set_error("nlf_topo_label: bad arguments");
    return NLF_EBADARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const uint8_t* bd = b;
  if (!tp_on_dev(b)) {
    NLF_CUDA_TRY(cudaMemcpyAsync(T->bst, b, (size_t)T->N, cudaMemcpyHostToDevice, st));
    bd = T->bst;
  }
  NLF_TRY(tp_label(T, bd, faces ? 1 : 0, ncomp, st));
  const bool dl = tp_on_dev(labels);
  int* ld = labels;
  if (!dl) {
    NLF_TRY(T->lab.reserve((size_t)T->N * 4));
    ld = (int*)T->lab.ptr;
  }
  k_tp_labels_out<<<nblk(T->N, kTpThreads), kTpThreads, 0, st>>>(T->N, T->L, T->rid, ld);
  NLF_CHECK_LAUNCH();
  if (!dl) NLF_CUDA_TRY(cudaMemcpyAsync(labels, ld, (size_t)T->N * 4, cudaMemcpyDeviceToHost, st));
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  return NLF_OK;
}

NLF_API int nlf_topo_remove_floating(nlf_topo* T, uint8_t* b, int* ncomp, int* nspan, long long* nsolid,
                                     void* stream) {
  if (!T || !b) {
    set_error("nlf_topo_remove_floating: bad arguments");
    return NLF_EBADARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const bool db = tp_on_dev(b);
  uint8_t* bd = db ? b : T->bst;
  if (!db) NLF_CUDA_TRY(cudaMemcpyAsync(bd, b, (size_t)T->N, cudaMemcpyHostToDevice, st));
  long long ns = 0;
  NLF_TRY(tp_remove_floating(T, bd, ncomp, nspan, &ns, st));
  if (nsolid) *nsolid = ns;
  if (!db) {
    NLF_CUDA_TRY(cudaMemcpyAsync(b, bd, (size_t)T->N, cudaMemcpyDeviceToHost, st));
    NLF_CUDA_TRY(cudaStreamSynchronize(st));
  }
  return NLF_OK;
}

NLF_API int nlf_topo_select(nlf_topo* T, const double* u, const uint8_t* mask, long long rank, double* value,
                            void* stream) {
  if (!T || !u || !value || rank < 0 || rank >= T->N) {
    set_error("nlf_topo_select: bad arguments (0 <= rank < voxels)");
    return NLF_EBADARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const double* ud = u;
  if (!tp_on_dev(u)) {
    NLF_CUDA_TRY(cudaMemcpyAsync(T->ust, u, (size_t)T->N * 8, cudaMemcpyHostToDevice, st));
    ud = T->ust;
  }
  const uint8_t* md = mask;
  if (mask && !tp_on_dev(mask)) {
    NLF_CUDA_TRY(cudaMemcpyAsync(T->front, mask, (size_t)T->N, cudaMemcpyHostToDevice, st));
    md = T->front;
  }
  return tp_select(T, ud, md, rank, value, st);
}

NLF_API int nlf_quantile_linear(long long n, double q, const double* sorted, double* out) {
  if (n < 1 || !sorted || !out || !std::isfinite(q)) {
    set_error("nlf_quantile_linear: bad arguments");
    return NLF_EBADARG;
  }
  return quantile_linear(n, q, [&](long long k, double* v) { *v = sorted[k]; return NLF_OK; }, out);
}

NLF_API int nlf_topo_binary(nlf_topo* T, const double* u, double v, int remove_floating, uint8_t* b, int* iters,
                            void* stream) {
  if (!T || !u || !b || !std::isfinite(v)) {
    set_error("nlf_topo_binary: bad arguments");
    return NLF_EBADARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const double* ud = u;
  if (!tp_on_dev(u)) {
    NLF_CUDA_TRY(cudaMemcpyAsync(T->ust, u, (size_t)T->N * 8, cudaMemcpyHostToDevice, st));
    ud = T->ust;
  }
  const bool db = tp_on_dev(b);
  uint8_t* bd = db ? b : T->bst;
  const long long N = T->N;
  const unsigned g = nblk(N, kTpThreads);
  // nlfiber/density.py:105: b = u > quantile(u, 1 - v)
  double thr = 0.0;
  NLF_TRY(quantile_linear(N, 1.0 - v, [&](long long k, double* x) { return tp_select(T, ud, nullptr, k, x, st); },
                          &thr));
  NLF_TRY(tp_count_reset(T, st));
  k_tp_threshold<<<g, kTpThreads, 0, st>>>(N, ud, thr, bd, T->cnt);
  NLF_CHECK_LAUNCH();
  int it = 0;
  if (remove_floating) {
    // nlfiber/density.py:106-121: remove the floating pieces, then grow the kept solid back to v through the
    // void voxels touching it, the k highest u of that front at a time
    long long ns = 0;
    for (; it < 500; ++it) {
      NLF_TRY(tp_remove_floating(T, bd, nullptr, nullptr, &ns, st));
      const double missing = v - (double)ns / (double)N;
      if (missing * (double)N < 1.0 || ns == 0) break;
      NLF_TRY(tp_count_reset(T, st));
      k_tp_front<<<g, kTpThreads, 0, st>>>(tp_cell(T), bd, T->front, T->cnt);
      NLF_CHECK_LAUNCH();
      NLF_TRY(tp_sync_read(T, st));
      const long long nf = (long long)((const Pinned*)T->pin)->cnt[0];
      if (nf == 0) break;
      long long k = (long long)std::nearbyint(missing * (double)N);
      k = std::min(std::max(k, 1LL), nf);
      double t = 0.0;
      NLF_TRY(tp_select(T, ud, T->front, nf - k, &t, st));
      NLF_TRY(tp_count_reset(T, st));
      k_tp_grow<<<g, kTpThreads, 0, st>>>(N, ud, T->front, t, bd, T->cnt);
      NLF_CHECK_LAUNCH();
    }
    NLF_TRY(tp_remove_floating(T, bd, nullptr, nullptr, &ns, st));
  }
  if (iters) *iters = it;
  if (!db) NLF_CUDA_TRY(cudaMemcpyAsync(b, bd, (size_t)N, cudaMemcpyDeviceToHost, st));
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  return NLF_OK;
}

NLF_API int nlf_upsample_sym(int d, int n, int m, const double* u, double* out, void* stream) {
  if ((d != 2 && d != 3) || n < 1 || m < 2 || !u || !out ||
      (d == 3 ? (long)m * m * m : (long)m * m) > (1L << 30)) {
    set_error("nlf_upsample_sym: bad arguments (d 2 or 3, n >= 1, m >= 2, at most 2^30 voxels)");
    return NLF_EBADARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int h = m / 2, s = 2 * h;
  const long NI = d == 3 ? (long)n * n * n : (long)n * n, NO = d == 3 ? (long)h * h * h : (long)h * h,
             NS = d == 3 ? (long)s * s * s : (long)s * s;
  const bool du = tp_on_dev(u), dout = tp_on_dev(out);
  const size_t o_u = 0, o_oct = tp_al(du ? 0 : (size_t)NI * 8), o_out = tp_al(o_oct + (size_t)NO * 8),
               total = tp_al(o_out + (dout ? 0 : (size_t)NS * 8));
  char* base = nullptr;
  NLF_CUDA_TRY(cudaMallocAsync((void**)&base, total, st));
  const double* ud = du ? u : (const double*)(base + o_u);
  double* outd = dout ? out : (double*)(base + o_out);
  int rc = NLF_OK;
  if (!du && cudaMemcpyAsync(base + o_u, u, (size_t)NI * 8, cudaMemcpyHostToDevice, st) != cudaSuccess) rc = NLF_ECUDA;
  if (rc == NLF_OK) {
    k_tp_up_orbit<<<nblk(NO, kTpThreads), kTpThreads, 0, st>>>(d, n, m, ud, (double*)(base + o_oct));
    k_tp_up_scatter<<<nblk(NS, kTpThreads), kTpThreads, 0, st>>>(d, h, (const double*)(base + o_oct), outd);
    if (cudaGetLastError() != cudaSuccess) rc = NLF_ECUDA;
  }
  if (rc == NLF_OK && !dout &&
      cudaMemcpyAsync(out, outd, (size_t)NS * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    rc = NLF_ECUDA;
  cudaFreeAsync(base, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) rc = NLF_ECUDA;
  if (rc != NLF_OK) set_error("nlf_upsample_sym: CUDA error %s", cudaGetErrorString(cudaGetLastError()));
  return rc;
}
