// Density map on the GPU: pre-density phi (octant) -> physical density rho (full periodic cell) with an exact
// volume fraction (nlfiber/density.py:23-91 DensityMap.smooth / rho, threshold, solve_eta; nlfiber/symmetry.py
// sym_perm, mirror, fold, exact_symmetrize). Cubes (d = 3), batched over cells, as below; squares (d = 2) take the
// same steps with kernels of their own (k2_*: quadrant, 2 permutations, 4 mirror images, orbits of sorted pairs):
//
//   phis = sym_perm(phi)                 octant (n_o)^3: mean of the 6 axis permutations, numpy's order
//   u    = k * mirror(phis)              periodic cone filter of radius r on the full cell (n = 2 n_o)^3, as a
//                                        direct sum over the nonzero taps of the grid kernel (the reference
//                                        multiplies rfftn's; the two agree to rounding)
//   us   = u / (std(u) + 1e-12)
//   o    = sym_perm(fold(us)) at one octant point per symmetry orbit (sorted index triples a <= b <= c), which
//          exact_symmetrize copies to every voxel of the orbit
//   eta  : mean over the cell of sigmoid(beta (o - eta)) = v, by 200 bisection halvings from
//          [min o - 40 / beta, max o + 40 / beta] and 3 Newton steps (nlfiber/density.py:43-63)
//   rho  = sigmoid(beta (o - eta)), once per orbit, copied to the full cell
//
// The full cell is 8 mirrored copies of the octant and the octant holds each orbit value `mult` times (1, 3 or
// 6), so every mean over the cell is sum_orbits mult f(o) / n_o^3: the bisection runs over the orbits only
// (5,984 at n_o = 32 instead of 262,144 voxels), one 2-CTA cluster per cell with fixed-order reductions.
#include <cmath>
#include <cstdlib>
#include <vector>

#include <cooperative_groups.h>

#include "nlf_common.cuh"
#include "nlf_internal.h"
#include "nlf_prof.cuh"
#include "../../include/nlf.h"

namespace nlf {

namespace cg = cooperative_groups;

constexpr int kEtaThreads = 1024;
constexpr int kEtaCta = 2;  // CTAs (one cluster) per cell in the volume bisection

struct DensityHandle {
  int d = 3;  // 3: cubes, octant (n_o)^3; 2: squares, quadrant (n_o)^2 (tables and kernels of their own)
  int n_o = 0, n = 0, R = 0, ntap = 0, halo = 0;
  double r = 0.0;
  int* tap_off = nullptr;     // [ntap][3] kernel offsets g (-n / 2 < g <= n / 2) with k(g) > 0
  double* tap_w = nullptr;    // [ntap] k(g), normalised to sum 1
  int* orbit_of = nullptr;    // [n_o^3] orbit of each octant point (its sorted index triple)
  int* orbit_abc = nullptr;   // [R][3] the sorted triple a <= b <= c of each orbit, lexicographic order
  double* orbit_mult = nullptr;  // [R] number of octant points in the orbit
  DevBuf ws;   // forward intermediates
  DevBuf wsb;  // vector-Jacobian product
};

// Forward intermediates of one density_run, kept in the handle's workspace
struct DensWs {
  double *F = nullptr, *u = nullptr, *psum = nullptr, *pvar = nullptr, *orb = nullptr, *ro = nullptr,
         *eta = nullptr;
  int nsum = 0, nvar = 0;
};

namespace {

__device__ __forceinline__ double sigmoid(double t) { return 1.0 / (1.0 + exp(-t)); }

// phis = sym_perm(phi) per octant point: numpy sums transpose(x, p) over itertools.permutations((0, 1, 2)) in
// order, starting from 0, then divides by 6
__global__ void k_dens_symphi(int n_o, const double* __restrict__ phi, double* __restrict__ phis) {
  const long NO = (long)n_o * n_o * n_o;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= NO) return;
  const int cell = blockIdx.y;
  const int c = (int)(t % n_o), b = (int)((t / n_o) % n_o), a = (int)(t / ((long)n_o * n_o));
  const double* x = phi + (long)cell * NO;
  auto at = [&](int i, int j, int k) { return x[((long)i * n_o + j) * n_o + k]; };
  double s = at(a, b, c);
  s = s + at(a, c, b);
  s = s + at(b, a, c);
  s = s + at(c, a, b);
  s = s + at(b, c, a);
  s = s + at(c, b, a);
  phis[(long)cell * NO + t] = s / 6.0;
}

__device__ __forceinline__ int fold_idx(int i, int n_o) { return i < n_o ? i : 2 * n_o - 1 - i; }

// y - d wrapped into [0, n) for |d| < n, then folded onto the octant (mirror: index i >= n_o is n - 1 - i)
__device__ __forceinline__ int wrap_fold(int y, int d, int n, int n_o) {
  int i = y - d;
  i = i < 0 ? i + n : (i >= n ? i - n : i);
  return i < n_o ? i : n - 1 - i;
}

// u(y) = sum_g k(g) f(y - g) with f = mirror(phis) (the circular convolution that irfftn(rfftn(f) rfftn(k))
// evaluates); taps (signed offsets, |g| < n per axis) staged in shared memory
__global__ void k_dens_filter(int n_o, int ntap, const int* __restrict__ tap_off, const double* __restrict__ tap_w,
                              const double* __restrict__ phis, double* __restrict__ u, double* __restrict__ psum) {
  __shared__ double red[32];
  extern __shared__ unsigned char smem_raw[];
  double* sw = reinterpret_cast<double*>(smem_raw);
  int* so = reinterpret_cast<int*>(sw + ntap);
  for (int i = threadIdx.x; i < ntap; i += blockDim.x) {
    sw[i] = tap_w[i];
    so[3 * i] = tap_off[3 * i];
    so[3 * i + 1] = tap_off[3 * i + 1];
    so[3 * i + 2] = tap_off[3 * i + 2];
  }
  __syncthreads();
  const int n = 2 * n_o;
  const long N = (long)n * n * n, NO = (long)n_o * n_o * n_o;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const int cell = blockIdx.y;
  double acc = 0.0;
  if (t < N) {
    const int k = (int)(t % n), j = (int)((t / n) % n), i = (int)(t / ((long)n * n));
    const double* f = phis + (long)cell * NO;
    for (int q = 0; q < ntap; ++q) {
      const int ii = wrap_fold(i, so[3 * q], n, n_o), jj = wrap_fold(j, so[3 * q + 1], n, n_o),
                kk = wrap_fold(k, so[3 * q + 2], n, n_o);
      acc += sw[q] * f[(ii * n_o + jj) * n_o + kk];
    }
    u[(long)cell * N + t] = acc;
  }
  double a[1] = {acc};
  block_sum<1>(a, red);
  if (threadIdx.x == 0) psum[(long)cell * gridDim.x + blockIdx.x] = a[0];
}

// The same filter on a tile of kTX x kTY z-lines per CTA: the tile's region of mirror(phis) with a halo of H
// (the largest tap offset per axis) is staged in shared memory once, then every voxel sums its taps from there
// in the same order as k_dens_filter (same bits).
constexpr int kTX = 2, kTY = 8;

__host__ __device__ __forceinline__ size_t tile_smem(int n, int H, int ntap) {
  return (size_t)ntap * (sizeof(double) + sizeof(int)) +
         (size_t)(kTX + 2 * H) * (kTY + 2 * H) * (n + 2 * H) * sizeof(double);
}

__global__ void k_dens_filter_tile(int n_o, int H, int ntap, const int* __restrict__ tap_off,
                                   const double* __restrict__ tap_w, const double* __restrict__ phis,
                                   double* __restrict__ u, double* __restrict__ psum) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ double red[32];
  const int n = 2 * n_o;
  const int SX = kTX + 2 * H, SY = kTY + 2 * H, SZ = n + 2 * H;
  double* S = reinterpret_cast<double*>(smem_raw);
  double* sw = S + (size_t)SX * SY * SZ;
  int* soff = reinterpret_cast<int*>(sw + ntap);  // tap offset in the staged array: value at y - g
  for (int i = threadIdx.x; i < ntap; i += blockDim.x) {
    sw[i] = tap_w[i];
    soff[i] = -((tap_off[3 * i] * SY + tap_off[3 * i + 1]) * SZ + tap_off[3 * i + 2]);
  }
  const int cell = blockIdx.y;
  const int tiles_y = (n + kTY - 1) / kTY;
  const int x0 = (blockIdx.x / tiles_y) * kTX, y0 = (blockIdx.x % tiles_y) * kTY;
  const long NO = (long)n_o * n_o * n_o, N = (long)n * n * n;
  const double* f = phis + (long)cell * NO;
  // one warp per staged z-row; a tile may overhang the cell (n not a multiple of the tile) by more than one
  // period in x and y (full wraps there), z spans [-H, n + H) with H <= n / 2 (one conditional wrap)
  const int lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  for (int row = threadIdx.x >> 5; row < SX * SY; row += nwarp) {
    const int sx = row / SY, sy = row - sx * SY;
    const int X = fold_idx(wrap(x0 + sx - H, n), n_o), Y = fold_idx(wrap(y0 + sy - H, n), n_o);
    const double* fr = f + (X * n_o + Y) * n_o;
    for (int sz = lane; sz < SZ; sz += 32) S[row * SZ + sz] = fr[wrap_fold(sz, H, n, n_o)];
  }
  __syncthreads();
  // each thread sums kVox voxels at once, taps outermost (each voxel still adds its taps in order)
  constexpr int kVox = 4;
  double tot = 0.0;
  const int total = kTX * kTY * n;
  for (int q0 = 0; q0 < total; q0 += kVox * blockDim.x) {
    int base[kVox];
    long dst[kVox];
    double acc[kVox];
#pragma unroll
    for (int v = 0; v < kVox; ++v) {
      const int q = q0 + threadIdx.x + v * blockDim.x;
      const int qn = fdiv(q, n), z = q - qn * n, y = qn % kTY, x = qn / kTY;
      const bool ok = q < total && x0 + x < n && y0 + y < n;
      base[v] = ok ? ((x + H) * SY + (y + H)) * SZ + (z + H) : (H * SY + H) * SZ + H;  // else a safe interior point
      dst[v] = ok ? (long)cell * N + ((long)(x0 + x) * n + (y0 + y)) * n + z : -1;
      acc[v] = 0.0;
    }
    for (int t = 0; t < ntap; ++t) {
      const double w = sw[t];
      const int o = soff[t];
#pragma unroll
      for (int v = 0; v < kVox; ++v) acc[v] += w * S[base[v] + o];
    }
#pragma unroll
    for (int v = 0; v < kVox; ++v)
      if (dst[v] >= 0) {
        u[dst[v]] = acc[v];
        tot += acc[v];
      }
  }
  double a[1] = {tot};
  block_sum<1>(a, red);
  if (threadIdx.x == 0) psum[(long)cell * gridDim.x + blockIdx.x] = a[0];
}

// sum of the nb partials of one cell in a fixed order (lane-strided, then a shuffle tree), by warp 0; every CTA
// that calls it gets the same bits. Result in thread 0.
__device__ __forceinline__ double warp0_sum(const double* __restrict__ part, int nb) {
  double s = 0.0;
  if (threadIdx.x < 32) {
    for (int b = threadIdx.x; b < nb; b += 32) s += part[b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  }
  return s;
}

// pvar[cell][blk] = partial sum of (u - mean u)^2 over the CTA's share of the cell (the second pass of std)
__global__ void k_dens_var(long N, int nsum, const double* __restrict__ u, const double* __restrict__ psum,
                           double* __restrict__ pvar) {
  __shared__ double red[32];
  __shared__ double s_mean;
  const int cell = blockIdx.y;
  const double tot = warp0_sum(psum + (long)cell * nsum, nsum);
  if (threadIdx.x == 0) s_mean = tot / (double)N;
  __syncthreads();
  const double mu = s_mean;
  const double* x = u + (long)cell * N;
  double a[1] = {0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const double d = x[i] - mu;
    a[0] += d * d;
  }
  block_sum<1>(a, red);
  if (threadIdx.x == 0) pvar[(long)cell * gridDim.x + blockIdx.x] = a[0];
}

// F[i][j][k] = fold(u / den) on the octant: mirror images averaged axis by axis (x, then y, then z: 0.5 (a + b)
// each), den = std(u) + 1e-12 from the k_dens_var partials (each CTA sums them in the same order)
__global__ void k_dens_fold(int n_o, const double* __restrict__ u, int nvar, const double* __restrict__ pvar,
                            double* __restrict__ F) {
  __shared__ double s_den;
  const int cell = blockIdx.y, n = 2 * n_o;
  const long N = (long)n * n * n, NO = (long)n_o * n_o * n_o;
  const double tot = warp0_sum(pvar + (long)cell * nvar, nvar);
  if (threadIdx.x == 0) s_den = sqrt(tot / (double)N) + 1e-12;
  __syncthreads();
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= NO) return;
  const int k = (int)(t % n_o), j = (int)((t / n_o) % n_o), i = (int)(t / ((long)n_o * n_o));
  const double* x = u + (long)cell * N;
  const double dd = s_den;
  auto us = [&](int ii, int jj, int kk) { return x[((long)ii * n + jj) * n + kk] / dd; };
  auto f0 = [&](int ii, int jj, int kk) { return 0.5 * (us(ii, jj, kk) + us(n - 1 - ii, jj, kk)); };
  auto f1 = [&](int ii, int jj, int kk) { return 0.5 * (f0(ii, jj, kk) + f0(ii, n - 1 - jj, kk)); };
  F[(long)cell * NO + t] = 0.5 * (f1(i, j, k) + f1(i, j, n - 1 - k));
}

// o[orbit] = sym_perm(F) at the orbit's sorted triple (the sum of the 6 permutations in numpy's order, / 6)
__global__ void k_dens_orbits(int n_o, int R, const int* __restrict__ orbit_abc, const double* __restrict__ F,
                              double* __restrict__ o) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  const int cell = blockIdx.y;
  const double* x = F + (long)cell * n_o * n_o * n_o;
  auto f2 = [&](int i, int j, int k) { return x[((long)i * n_o + j) * n_o + k]; };
  const int a = orbit_abc[3 * r], b = orbit_abc[3 * r + 1], c = orbit_abc[3 * r + 2];
  double s = f2(a, b, c);
  s = s + f2(a, c, b);
  s = s + f2(b, a, c);
  s = s + f2(c, a, b);
  s = s + f2(b, c, a);
  s = s + f2(c, b, a);
  o[(long)cell * R + r] = s / 6.0;
}

__device__ __forceinline__ double cta_minmax(double v, double* red, bool mx) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    const double w = __shfl_down_sync(0xffffffffu, v, s);
    v = mx ? fmax(v, w) : fmin(v, w);
  }
  if (lane == 0) red[wid] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = red[0];
    for (int q = 1; q < nw; ++q) m = mx ? fmax(m, red[q]) : fmin(m, red[q]);
    red[32] = m;
  }
  __syncthreads();
  const double m = red[32];
  __syncthreads();
  return m;
}

// Sum over the CTA of v in a fixed order; the result is valid in thread 0 only
__device__ __forceinline__ double cta_sum0(double v, double* red) {
  double a[1] = {v};
  block_sum<1>(a, red);
  return a[0];
}

// sum_{r = r0, r0 + rs, ... < R} mult[r] sigmoid(beta (x[r] - c)), added in that order; four terms at a time are
// evaluated independently so their latencies overlap
__device__ __forceinline__ double orbit_vol(const double* __restrict__ x, const double* __restrict__ mult, int r0,
                                            int rs, int R, double beta, double c) {
  double acc = 0.0;
  for (int r = r0; r < R; r += 4 * rs) {
    double t[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int q = r + k * rs;
      t[k] = q < R ? mult[q] * sigmoid(beta * (x[q] - c)) : 0.0;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (r + k * rs < R) acc += t[k];
  }
  return acc;
}

// Cluster-wide total of a per-CTA value (valid in thread 0 of the CTA): each CTA publishes it in slot `buf`
// of its own shared memory, one cluster barrier, then every thread adds all CTAs' slots in rank order, so every
// thread of the cluster holds the same bits. Slots alternate so that one barrier per combine suffices (a CTA
// rewrites a slot only after the next barrier, which its peers pass after reading it).
__device__ __forceinline__ double cluster_total(cg::cluster_group& cl, double v, double* slots, int& buf, int op) {
  if (threadIdx.x == 0) slots[buf] = v;
  cl.sync();
  double t = *cl.map_shared_rank(slots + buf, 0);
  for (int q = 1; q < kEtaCta; ++q) {
    const double w = *cl.map_shared_rank(slots + buf, q);
    t = op == 0 ? t + w : (op == 1 ? fmin(t, w) : fmax(t, w));
  }
  buf ^= 1;
  return t;
}

// eta[cell] with mean(sigmoid(beta (o - eta))) = v[cell] (nlfiber/density.py:43-63), then rho of every orbit,
// ro = sigmoid(beta (o - eta)). A cluster of kEtaCta CTAs per cell: CTA q takes the orbits q B + t + k kEtaCta B
// (B threads) and the per-step sums are combined across the cluster, so every CTA takes the same decisions.
__global__ void __cluster_dims__(kEtaCta, 1, 1) __launch_bounds__(kEtaThreads)
    k_dens_eta(double NO, int R, const double* __restrict__ o, const double* __restrict__ mult,
               const double* __restrict__ vol, double beta, double* __restrict__ eta_out, double* __restrict__ ro) {
  __shared__ double red[33];
  __shared__ double slots[2];
  cg::cluster_group cl = cg::this_cluster();
  const int cell = blockIdx.x / kEtaCta, rank = (int)cl.block_rank();
  const int r0 = rank * blockDim.x + threadIdx.x, rs = kEtaCta * blockDim.x;
  const double* x = o + (long)cell * R;
  const double v = vol[cell];  // NO: points of the octant (quadrant), each orbit holding mult of them
  int buf = 0;
  double mn = INFINITY, mxv = -INFINITY;
  for (int r = r0; r < R; r += rs) {
    mn = fmin(mn, x[r]);
    mxv = fmax(mxv, x[r]);
  }
  double lo = cluster_total(cl, cta_minmax(mn, red, false), slots, buf, 1) - 40.0 / beta;
  double hi = cluster_total(cl, cta_minmax(mxv, red, true), slots, buf, 2) + 40.0 / beta;
  // 200 halvings as in the reference; once a step leaves (lo, hi) unchanged (they are adjacent doubles or
  // equal, so mid is one of them), every later step computes the same mid and decision, so the loop stops there
  // with the bracket the 200 steps would end with
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (lo + hi);
    const double acc = orbit_vol(x, mult, r0, rs, R, beta, mid);
    const bool big = cluster_total(cl, cta_sum0(acc, red), slots, buf, 0) / NO > v;  // volume too large: raise eta
    const double lo1 = big ? mid : lo, hi1 = big ? hi : mid;
    if (lo1 == lo && hi1 == hi) break;
    lo = lo1;
    hi = hi1;
  }
  double eta = 0.5 * (lo + hi);
  for (int it = 0; it < 3; ++it) {
    double s1 = 0.0, s2 = 0.0;
    for (int r = r0; r < R; r += rs) {
      const double s = sigmoid(beta * (x[r] - eta));
      s1 += mult[r] * s;
      s2 += mult[r] * (beta * s * (1.0 - s));
    }
    const double ms = cluster_total(cl, cta_sum0(s1, red), slots, buf, 0) / NO;
    const double dv = -(cluster_total(cl, cta_sum0(s2, red), slots, buf, 0) / NO);
    eta = eta - (ms - v) / (dv == 0.0 ? -1.0 : dv);
  }
  if (rank == 0 && threadIdx.x == 0) eta_out[cell] = eta;
  for (int r = r0; r < R; r += rs) ro[(long)cell * R + r] = sigmoid(beta * (x[r] - eta));
  cl.sync();  // no CTA leaves while a peer may still read its slots
}

// rho and the smoothed field o on the full cell: copies of the orbit values
__global__ void k_dens_rho(int n_o, int R, const int* __restrict__ orbit_of, const double* __restrict__ o,
                           const double* __restrict__ ro, double* __restrict__ rho, double* __restrict__ u_out) {
  const int n = 2 * n_o;
  const long N = (long)n * n * n;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= N) return;
  const int cell = blockIdx.y;
  const int k = (int)(t % n), j = (int)((t / n) % n), i = (int)(t / ((long)n * n));
  const int q = orbit_of[((long)fold_idx(i, n_o) * n_o + fold_idx(j, n_o)) * n_o + fold_idx(k, n_o)];
  if (rho) rho[(long)cell * N + t] = ro[(long)cell * R + q];
  if (u_out) u_out[(long)cell * N + t] = o[(long)cell * R + q];
}

// ---- vector-Jacobian product of the map (the cotangent of phi for a cotangent of rho) -------------------------
// Transposes, in reverse order of the forward map: threshold with the implicit d eta (d eta / du_j =
// d_j / sum d, d = s (1 - s)); exact_symmetrize^T = the mean over each symmetry orbit of the full cell; the
// unit-std scaling (d std / du_j = (u_j - mean u) / (N std)); the cone filter (its own transpose, k(g) = k(-g));
// mirror^T (the octant sum of the 8 mirror images); sym_perm^T = sym_perm.

// go[p] = sum of g over the 8 mirror images of octant point p, axis by axis (x, then y, then z)
__global__ void k_dv_mirror_t(int n_o, const double* __restrict__ g, double* __restrict__ go) {
  const int n = 2 * n_o;
  const long NO = (long)n_o * n_o * n_o, N = (long)n * n * n;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= NO) return;
  const int vec = blockIdx.y;
  const int c = (int)(t % n_o), b = (int)((t / n_o) % n_o), a = (int)(t / ((long)n_o * n_o));
  const double* x = g + (long)vec * N;
  auto x1 = [&](int j, int k) { return x[((long)a * n + j) * n + k] + x[((long)(n - 1 - a) * n + j) * n + k]; };
  const int b1 = n - 1 - b, c1 = n - 1 - c;
  go[(long)vec * NO + t] = (x1(b, c) + x1(b1, c)) + (x1(b, c1) + x1(b1, c1));
}

// Per orbit r of vector vec (cell vec / nrow): W_r = beta d_r gs_r, gs_r the sum of go over the orbit's distinct
// permutations (the orbit's sum of the rho cotangent), d_r = s_r (1 - s_r); then the orbit mean of the threshold's
// transpose, ubs_r = W_r / (8 mult_r) - d_r (sum_r W_r) / (8 sum_r mult_r d_r). One CTA per vector.
__global__ void __launch_bounds__(1024) k_dv_orbits(int n_o, int R, int nrow, const int* __restrict__ orbit_abc,
                                                    const double* __restrict__ mult, const double* __restrict__ ro,
                                                    const double* __restrict__ go, double beta,
                                                    double* __restrict__ ubs) {
  __shared__ double red[32 * 2];  // block_sum<2> scratch
  __shared__ double s_w, s_d;
  const int vec = blockIdx.x, cell = vec / nrow;
  const long NO = (long)n_o * n_o * n_o;
  const double* G = go + (long)vec * NO;
  const double* sr = ro + (long)cell * R;
  double* out = ubs + (long)vec * R;
  auto at = [&](int i, int j, int k) { return G[((long)i * n_o + j) * n_o + k]; };
  double acc[2] = {0.0, 0.0};
  for (int r = threadIdx.x; r < R; r += blockDim.x) {
    const int a = orbit_abc[3 * r], b = orbit_abc[3 * r + 1], c = orbit_abc[3 * r + 2];
    double gs = at(a, b, c);
    if (a == b && b == c) {
    } else if (a == b) {
      gs = gs + at(a, c, a);
      gs = gs + at(c, a, a);
    } else if (b == c) {
      gs = gs + at(b, a, b);
      gs = gs + at(b, b, a);
    } else {
      gs = gs + at(a, c, b);
      gs = gs + at(b, a, c);
      gs = gs + at(b, c, a);
      gs = gs + at(c, a, b);
      gs = gs + at(c, b, a);
    }
    const double d = sr[r] * (1.0 - sr[r]);
    const double W = beta * d * gs;
    out[r] = W;
    acc[0] += W;
    acc[1] += mult[r] * d;
  }
  block_sum<2>(acc, red);
  if (threadIdx.x == 0) {
    s_w = acc[0];
    s_d = 8.0 * acc[1];
  }
  __syncthreads();
  const double k = s_w / s_d;
  for (int r = threadIdx.x; r < R; r += blockDim.x) {
    const double d = sr[r] * (1.0 - sr[r]);
    out[r] = out[r] / (8.0 * mult[r]) - d * k;
  }
}

// pdot[vec][blk] = partial sum over the cell of ubs[orbit(x)] u(x)
__global__ void k_dv_dot(int n_o, int R, int nrow, const int* __restrict__ orbit_of, const double* __restrict__ ubs,
                         const double* __restrict__ u, double* __restrict__ pdot) {
  __shared__ double red[32];
  const int n = 2 * n_o, vec = blockIdx.y, cell = vec / nrow;
  const long N = (long)n * n * n;
  const double* uc = u + (long)cell * N;
  const double* ub = ubs + (long)vec * R;
  double a[1] = {0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const int k = (int)(i % n), j = (int)((i / n) % n), x = (int)(i / ((long)n * n));
    a[0] += ub[orbit_of[((long)fold_idx(x, n_o) * n_o + fold_idx(j, n_o)) * n_o + fold_idx(k, n_o)]] * uc[i];
  }
  block_sum<1>(a, red);
  if (threadIdx.x == 0) pdot[(long)vec * gridDim.x + blockIdx.x] = a[0];
}

// uf[vec] = the cone filter of ubar(x) = ubs[orbit(x)] / D - cc (u(x) - mean) / (N sd), the transpose of the
// unit-std scaling applied to the orbit-mean cotangent (D = sd + 1e-12, cc = sum ubs u / D^2; mean and sd from
// the forward's partials). Tiled as k_dens_filter_tile, the staged values computed from that expression.
__global__ void k_dv_filter_tile(int n_o, int H, int ntap, int nrow, int R, const int* __restrict__ tap_off,
                                 const double* __restrict__ tap_w, const int* __restrict__ orbit_of,
                                 const double* __restrict__ ubs, const double* __restrict__ u, int nsum,
                                 const double* __restrict__ psum, int nvar, const double* __restrict__ pvar,
                                 int ndot, const double* __restrict__ pdot, double* __restrict__ uf) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ double sc[4];
  const int n = 2 * n_o;
  const int SX = kTX + 2 * H, SY = kTY + 2 * H, SZ = n + 2 * H;
  double* S = reinterpret_cast<double*>(smem_raw);
  double* sw = S + (size_t)SX * SY * SZ;
  int* soff = reinterpret_cast<int*>(sw + ntap);
  for (int i = threadIdx.x; i < ntap; i += blockDim.x) {
    sw[i] = tap_w[i];
    soff[i] = -((tap_off[3 * i] * SY + tap_off[3 * i + 1]) * SZ + tap_off[3 * i + 2]);
  }
  const int vec = blockIdx.y, cell = vec / nrow;
  const long N = (long)n * n * n;
  {
    const double t0 = warp0_sum(psum + (long)cell * nsum, nsum);
    const double t1 = warp0_sum(pvar + (long)cell * nvar, nvar);
    const double t2 = warp0_sum(pdot + (long)vec * ndot, ndot);
    if (threadIdx.x == 0) {
      const double sd = sqrt(t1 / (double)N), D = sd + 1e-12;
      sc[0] = t0 / (double)N;       // mean u
      sc[1] = D;
      sc[2] = t2 / (D * D);         // cc
      sc[3] = (double)N * sd;
    }
  }
  __syncthreads();
  const double mean = sc[0], D = sc[1], cc = sc[2], Nsd = sc[3];
  const int tiles_y = (n + kTY - 1) / kTY;
  const int x0 = (blockIdx.x / tiles_y) * kTX, y0 = (blockIdx.x % tiles_y) * kTY;
  const double* uc = u + (long)cell * N;
  const double* ub = ubs + (long)vec * R;
  const int lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  for (int row = threadIdx.x >> 5; row < SX * SY; row += nwarp) {
    const int sx = row / SY, sy = row - sx * SY;
    const int X = wrap(x0 + sx - H, n), Y = wrap(y0 + sy - H, n);
    const int* orow = orbit_of + ((long)fold_idx(X, n_o) * n_o + fold_idx(Y, n_o)) * n_o;
    const double* urow = uc + ((long)X * n + Y) * n;
    for (int sz = lane; sz < SZ; sz += 32) {
      int Z = sz - H;
      Z = Z < 0 ? Z + n : (Z >= n ? Z - n : Z);
      S[row * SZ + sz] = ub[orow[fold_idx(Z, n_o)]] / D - cc * (urow[Z] - mean) / Nsd;
    }
  }
  __syncthreads();
  constexpr int kVox = 4;
  const int total = kTX * kTY * n;
  for (int q0 = 0; q0 < total; q0 += kVox * blockDim.x) {
    int base[kVox];
    long dst[kVox];
    double acc[kVox];
#pragma unroll
    for (int v = 0; v < kVox; ++v) {
      const int q = q0 + threadIdx.x + v * blockDim.x;
      const int qn = fdiv(q, n), z = q - qn * n, y = qn % kTY, x = qn / kTY;
      const bool ok = q < total && x0 + x < n && y0 + y < n;
      base[v] = ok ? ((x + H) * SY + (y + H)) * SZ + (z + H) : (H * SY + H) * SZ + H;
      dst[v] = ok ? (long)vec * N + ((long)(x0 + x) * n + (y0 + y)) * n + z : -1;
      acc[v] = 0.0;
    }
    for (int t = 0; t < ntap; ++t) {
      const double w = sw[t];
      const int o = soff[t];
#pragma unroll
      for (int v = 0; v < kVox; ++v) acc[v] += w * S[base[v] + o];
    }
#pragma unroll
    for (int v = 0; v < kVox; ++v)
      if (dst[v] >= 0) uf[dst[v]] = acc[v];
  }
}

// ---- square cells (d = 2): quadrant (n_o)^2 -> full cell (2 n_o)^2, the same steps with 2 permutations, 4 mirror
// images and orbits of sorted pairs a <= b (multiplicity 1 or 2); one thread per point, as small as these cells are

// phis = sym_perm(phi): numpy adds transpose(x, (0, 1)) then transpose(x, (1, 0)), then divides by 2
__global__ void k2_symphi(int n_o, const double* __restrict__ phi, double* __restrict__ phis) {
  const long NO = (long)n_o * n_o;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= NO) return;
  const int cell = blockIdx.y, b = (int)(t % n_o), a = (int)(t / n_o);
  const double* x = phi + (long)cell * NO;
  phis[(long)cell * NO + t] = (x[(long)a * n_o + b] + x[(long)b * n_o + a]) / 2.0;
}

// u(y) = sum_g k(g) f(y - g), f = mirror(phis); psum[cell][blk] = the CTA's partial sum of u
__global__ void k2_filter(int n_o, int ntap, const int* __restrict__ tap_off, const double* __restrict__ tap_w,
                          const double* __restrict__ phis, double* __restrict__ u, double* __restrict__ psum) {
  __shared__ double red[32];
  const int n = 2 * n_o;
  const long N = (long)n * n, NO = (long)n_o * n_o;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const int cell = blockIdx.y;
  double acc = 0.0;
  if (t < N) {
    const int j = (int)(t % n), i = (int)(t / n);
    const double* f = phis + (long)cell * NO;
    for (int q = 0; q < ntap; ++q) {
      const int ii = wrap_fold(i, tap_off[3 * q], n, n_o), jj = wrap_fold(j, tap_off[3 * q + 1], n, n_o);
      acc += tap_w[q] * f[(long)ii * n_o + jj];
    }
    u[(long)cell * N + t] = acc;
  }
  double a[1] = {acc};
  block_sum<1>(a, red);
  if (threadIdx.x == 0) psum[(long)cell * gridDim.x + blockIdx.x] = a[0];
}

// F = fold(u / den) on the quadrant (x, then y: 0.5 (a + b) each), den = std(u) + 1e-12 from the k_dens_var partials
__global__ void k2_fold(int n_o, const double* __restrict__ u, int nvar, const double* __restrict__ pvar,
                        double* __restrict__ F) {
  __shared__ double s_den;
  const int cell = blockIdx.y, n = 2 * n_o;
  const long N = (long)n * n, NO = (long)n_o * n_o;
  const double tot = warp0_sum(pvar + (long)cell * nvar, nvar);
  if (threadIdx.x == 0) s_den = sqrt(tot / (double)N) + 1e-12;
  __syncthreads();
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= NO) return;
  const int j = (int)(t % n_o), i = (int)(t / n_o);
  const double* x = u + (long)cell * N;
  const double dd = s_den;
  auto us = [&](int ii, int jj) { return x[(long)ii * n + jj] / dd; };
  auto f0 = [&](int ii, int jj) { return 0.5 * (us(ii, jj) + us(n - 1 - ii, jj)); };
  F[(long)cell * NO + t] = 0.5 * (f0(i, j) + f0(i, n - 1 - j));
}

// o[orbit] = sym_perm(F) at the orbit's sorted pair
__global__ void k2_orbits(int n_o, int R, const int* __restrict__ orbit_abc, const double* __restrict__ F,
                          double* __restrict__ o) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  const int cell = blockIdx.y;
  const double* x = F + (long)cell * n_o * n_o;
  const int a = orbit_abc[3 * r], b = orbit_abc[3 * r + 1];
  o[(long)cell * R + r] = (x[(long)a * n_o + b] + x[(long)b * n_o + a]) / 2.0;
}

// rho and the smoothed field on the full cell: copies of the orbit values
__global__ void k2_rho(int n_o, int R, const int* __restrict__ orbit_of, const double* __restrict__ o,
                       const double* __restrict__ ro, double* __restrict__ rho, double* __restrict__ u_out) {
  const int n = 2 * n_o;
  const long N = (long)n * n;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= N) return;
  const int cell = blockIdx.y, j = (int)(t % n), i = (int)(t / n);
  const int q = orbit_of[(long)fold_idx(i, n_o) * n_o + fold_idx(j, n_o)];
  if (rho) rho[(long)cell * N + t] = ro[(long)cell * R + q];
  if (u_out) u_out[(long)cell * N + t] = o[(long)cell * R + q];
}

// go[p] = sum of g over the 4 mirror images of quadrant point p (x, then y)
__global__ void k2_mirror_t(int n_o, const double* __restrict__ g, double* __restrict__ go) {
  const int n = 2 * n_o;
  const long NO = (long)n_o * n_o, N = (long)n * n;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= NO) return;
  const int vec = blockIdx.y, b = (int)(t % n_o), a = (int)(t / n_o);
  const double* x = g + (long)vec * N;
  auto x1 = [&](int j) { return x[(long)a * n + j] + x[(long)(n - 1 - a) * n + j]; };
  go[(long)vec * NO + t] = x1(b) + x1(n - 1 - b);
}

// Per orbit r: W_r = beta d_r gs_r (gs_r the orbit's sum of go, d_r = s_r (1 - s_r)), then the orbit mean of the
// threshold's transpose, ubs_r = W_r / (4 mult_r) - d_r (sum W) / (4 sum mult d). One CTA per vector.
__global__ void __launch_bounds__(1024) k2_dv_orbits(int n_o, int R, int nrow, const int* __restrict__ orbit_abc,
                                                     const double* __restrict__ mult, const double* __restrict__ ro,
                                                     const double* __restrict__ go, double beta,
                                                     double* __restrict__ ubs) {
  __shared__ double red[32 * 2];
  __shared__ double s_w, s_d;
  const int vec = blockIdx.x, cell = vec / nrow;
  const double* G = go + (long)vec * n_o * n_o;
  const double* sr = ro + (long)cell * R;
  double* out = ubs + (long)vec * R;
  double acc[2] = {0.0, 0.0};
  for (int r = threadIdx.x; r < R; r += blockDim.x) {
    const int a = orbit_abc[3 * r], b = orbit_abc[3 * r + 1];
    double gs = G[(long)a * n_o + b];
    if (a != b) gs = gs + G[(long)b * n_o + a];
    const double d = sr[r] * (1.0 - sr[r]);
    const double W = beta * d * gs;
    out[r] = W;
    acc[0] += W;
    acc[1] += mult[r] * d;
  }
  block_sum<2>(acc, red);
  if (threadIdx.x == 0) {
    s_w = acc[0];
    s_d = 4.0 * acc[1];
  }
  __syncthreads();
  const double k = s_w / s_d;
  for (int r = threadIdx.x; r < R; r += blockDim.x) {
    const double d = sr[r] * (1.0 - sr[r]);
    out[r] = out[r] / (4.0 * mult[r]) - d * k;
  }
}

// pdot[vec][blk] = partial sum over the cell of ubs[orbit(x)] u(x)
__global__ void k2_dv_dot(int n_o, int R, int nrow, const int* __restrict__ orbit_of, const double* __restrict__ ubs,
                          const double* __restrict__ u, double* __restrict__ pdot) {
  __shared__ double red[32];
  const int n = 2 * n_o, vec = blockIdx.y, cell = vec / nrow;
  const long N = (long)n * n;
  const double* uc = u + (long)cell * N;
  const double* ub = ubs + (long)vec * R;
  double a[1] = {0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const int j = (int)(i % n), x = (int)(i / n);
    a[0] += ub[orbit_of[(long)fold_idx(x, n_o) * n_o + fold_idx(j, n_o)]] * uc[i];
  }
  block_sum<1>(a, red);
  if (threadIdx.x == 0) pdot[(long)vec * gridDim.x + blockIdx.x] = a[0];
}

// uf[vec] = the cone filter of ubar(x) = ubs[orbit(x)] / D - cc (u(x) - mean) / (N sd) (the transpose of the
// unit-std scaling applied to the orbit-mean cotangent; D = sd + 1e-12, cc = sum ubs u / D^2)
__global__ void k2_dv_filter(int n_o, int ntap, int nrow, int R, const int* __restrict__ tap_off,
                             const double* __restrict__ tap_w, const int* __restrict__ orbit_of,
                             const double* __restrict__ ubs, const double* __restrict__ u, int nsum,
                             const double* __restrict__ psum, int nvar, const double* __restrict__ pvar, int ndot,
                             const double* __restrict__ pdot, double* __restrict__ uf) {
  __shared__ double sc[4];
  const int n = 2 * n_o, vec = blockIdx.y, cell = vec / nrow;
  const long N = (long)n * n;
  {
    const double t0 = warp0_sum(psum + (long)cell * nsum, nsum);
    const double t1 = warp0_sum(pvar + (long)cell * nvar, nvar);
    const double t2 = warp0_sum(pdot + (long)vec * ndot, ndot);
    if (threadIdx.x == 0) {
      const double sd = sqrt(t1 / (double)N), D = sd + 1e-12;
      sc[0] = t0 / (double)N;
      sc[1] = D;
      sc[2] = t2 / (D * D);
      sc[3] = (double)N * sd;
    }
  }
  __syncthreads();
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= N) return;
  const double mean = sc[0], D = sc[1], cc = sc[2], Nsd = sc[3];
  const double* uc = u + (long)cell * N;
  const double* ub = ubs + (long)vec * R;
  const int j = (int)(t % n), i = (int)(t / n);
  double acc = 0.0;
  for (int q = 0; q < ntap; ++q) {
    int ii = i - tap_off[3 * q], jj = j - tap_off[3 * q + 1];
    ii = ii < 0 ? ii + n : (ii >= n ? ii - n : ii);
    jj = jj < 0 ? jj + n : (jj >= n ? jj - n : jj);
    const double ubar = ub[orbit_of[(long)fold_idx(ii, n_o) * n_o + fold_idx(jj, n_o)]] / D -
                        cc * (uc[(long)ii * n + jj] - mean) / Nsd;
    acc += tap_w[q] * ubar;
  }
  uf[(long)vec * N + t] = acc;
}

bool dens_on_dev(const void* p) {
  if (!p) return false;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

// Host tables of one octant side and filter radius (nlfiber/density.py:23-31 hat_kernel_fft before its rfftn;
// nlfiber/symmetry.py:74-96 free_index / representative_index)
static int density_tables(DensityHandle& h) {
  const int n = h.n, n_o = h.n_o;
  // the cone kernel on the periodic grid: k(g) = max(0, r - |min-image g|), normalised (a delta if all zero)
  std::vector<int> off;  // [ntap][3]; the third offset is 0 on squares
  std::vector<double> w;
  double sum = 0.0;
  const int nz = h.d == 3 ? n : 1;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
      for (int k = 0; k < nz; ++k) {
        const double gi = std::min(i, n - i), gj = std::min(j, n - j), gk = std::min(k, n - k);
        const double val = std::max(0.0, h.r - std::sqrt(gi * gi + gj * gj + gk * gk));
        if (val > 0.0) {
          off.insert(off.end(), {i <= n / 2 ? i : i - n, j <= n / 2 ? j : j - n, k <= n / 2 ? k : k - n});
          w.push_back(val);
          sum += val;
        }
      }
  if (w.empty()) {
    off = {0, 0, 0};
    w = {1.0};
    sum = 1.0;
  }
  if (w.size() > 8192) {
    set_error("nlf_density_create: filter radius %g gives %zu taps (at most 8192)", h.r, w.size());
    return NLF_EBADARG;
  }
  for (double& x : w) x /= sum;
  h.ntap = (int)w.size();
  h.halo = 0;
  for (int x : off) h.halo = std::max(h.halo, std::abs(x));
  // orbits: sorted triples (pairs on squares) in lexicographic order, their multiplicity, and the orbit of every
  // octant (quadrant) point
  std::vector<int> abc, of(h.d == 3 ? (size_t)n_o * n_o * n_o : (size_t)n_o * n_o, -1);
  std::vector<double> mult;
  if (h.d == 2) {
    for (int a = 0; a < n_o; ++a)
      for (int b = a; b < n_o; ++b) {
        const int id = (int)mult.size();
        abc.insert(abc.end(), {a, b, 0});
        mult.push_back(a == b ? 1.0 : 2.0);
        of[(size_t)a * n_o + b] = id;
        of[(size_t)b * n_o + a] = id;
      }
  } else {
    for (int a = 0; a < n_o; ++a)
      for (int b = a; b < n_o; ++b)
        for (int c = b; c < n_o; ++c) {
          const int id = (int)mult.size();
          abc.insert(abc.end(), {a, b, c});
          mult.push_back((a == b && b == c) ? 1.0 : (a == b || b == c) ? 3.0 : 6.0);
          const int p[6][3] = {{a, b, c}, {a, c, b}, {b, a, c}, {b, c, a}, {c, a, b}, {c, b, a}};
          for (auto& q : p) of[((size_t)q[0] * n_o + q[1]) * n_o + q[2]] = id;
        }
  }
  h.R = (int)mult.size();
  NLF_CUDA_TRY(cudaMalloc(&h.tap_off, off.size() * sizeof(int)));
  NLF_CUDA_TRY(cudaMalloc(&h.tap_w, w.size() * sizeof(double)));
  NLF_CUDA_TRY(cudaMalloc(&h.orbit_of, of.size() * sizeof(int)));
  NLF_CUDA_TRY(cudaMalloc(&h.orbit_abc, abc.size() * sizeof(int)));
  NLF_CUDA_TRY(cudaMalloc(&h.orbit_mult, mult.size() * sizeof(double)));
  NLF_CUDA_TRY(cudaMemcpy(h.tap_off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice));
  NLF_CUDA_TRY(cudaMemcpy(h.tap_w, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice));
  NLF_CUDA_TRY(cudaMemcpy(h.orbit_of, of.data(), of.size() * sizeof(int), cudaMemcpyHostToDevice));
  NLF_CUDA_TRY(cudaMemcpy(h.orbit_abc, abc.data(), abc.size() * sizeof(int), cudaMemcpyHostToDevice));
  NLF_CUDA_TRY(cudaMemcpy(h.orbit_mult, mult.data(), mult.size() * sizeof(double), cudaMemcpyHostToDevice));
  return NLF_OK;
}

static void density_free(DensityHandle& h) {
  cudaFree(h.tap_off);
  cudaFree(h.tap_w);
  cudaFree(h.orbit_of);
  cudaFree(h.orbit_abc);
  cudaFree(h.orbit_mult);
  h.ws.release();
  h.wsb.release();
}

// the whole map for ncell cells on device arrays; rho, u_out, eta_out may each be null
static int density_run(DensityHandle& h, int ncell, const double* phi, const double* vol, double beta, double* rho,
                       double* u_out, double* eta_out, cudaStream_t st, DensWs* keep = nullptr) {
  const int n_o = h.n_o, n = h.n;
  const bool sq = h.d == 2;
  const long NO = sq ? (long)n_o * n_o : (long)n_o * n_o * n_o, N = sq ? (long)n * n : (long)n * n * n;
  // the tiled filter when its staged region fits in shared memory (cone radii up to ~6 at 64^3), else the gather
  // (NLF_DENSITY_GATHER=1 forces the gather)
  const size_t tsm = tile_smem(n, h.halo, h.ntap);
  static const bool force_gather = [] {
    const char* e = std::getenv("NLF_DENSITY_GATHER");
    return e && e[0] == '1';
  }();
  const bool tiled = !sq && tsm <= 200 * 1024 && !force_gather;
  const int ntile = ((n + kTX - 1) / kTX) * ((n + kTY - 1) / kTY);
  const int nsum = tiled ? ntile : (int)((N + 255) / 256), nvar = (int)std::min<long>(128, (N + 2047) / 2048);
  const size_t o_phis = 0, o_u = al256(o_phis + (size_t)ncell * NO * 8),
               o_sum = al256(o_u + (size_t)ncell * N * 8), o_var = al256(o_sum + (size_t)ncell * nsum * 8),
               o_orb = al256(o_var + (size_t)ncell * nvar * 8), o_ro = al256(o_orb + (size_t)ncell * h.R * 8),
               o_eta = al256(o_ro + (size_t)ncell * h.R * 8), total = al256(o_eta + (size_t)ncell * 8);
  NLF_TRY(h.ws.reserve(total));
  char* b = (char*)h.ws.ptr;
  double* phis = reinterpret_cast<double*>(b + o_phis);
  double* u = reinterpret_cast<double*>(b + o_u);
  double* psum = reinterpret_cast<double*>(b + o_sum);
  double* pvar = reinterpret_cast<double*>(b + o_var);
  double* orb = reinterpret_cast<double*>(b + o_orb);
  double* ro = reinterpret_cast<double*>(b + o_ro);
  double* eta = eta_out ? eta_out : reinterpret_cast<double*>(b + o_eta);
  if (keep) {
    keep->F = phis;
    keep->u = u;
    keep->psum = psum;
    keep->pvar = pvar;
    keep->orb = orb;
    keep->ro = ro;
    keep->eta = eta;
    keep->nsum = nsum;
    keep->nvar = nvar;
  }
  if (sq) {
    {
      ProfScope ps(PK_DENS_FILTER, st);
      k2_symphi<<<dim3((unsigned)((NO + 255) / 256), ncell), 256, 0, st>>>(n_o, phi, phis);
      NLF_CHECK_LAUNCH();
      k2_filter<<<dim3((unsigned)nsum, ncell), 256, 0, st>>>(n_o, h.ntap, h.tap_off, h.tap_w, phis, u, psum);
      NLF_CHECK_LAUNCH();
    }
    {
      ProfScope ps(PK_DENS_VAR, st);
      k_dens_var<<<dim3((unsigned)nvar, ncell), 256, 0, st>>>(N, nsum, u, psum, pvar);
      NLF_CHECK_LAUNCH();
    }
    {
      ProfScope ps(PK_DENS_FOLD, st);
      k2_fold<<<dim3((unsigned)((NO + 255) / 256), ncell), 256, 0, st>>>(n_o, u, nvar, pvar, phis);
      NLF_CHECK_LAUNCH();
      k2_orbits<<<dim3((unsigned)((h.R + 255) / 256), ncell), 256, 0, st>>>(n_o, h.R, h.orbit_abc, phis, orb);
      NLF_CHECK_LAUNCH();
    }
    {
      ProfScope ps(PK_DENS_ETA, st);
      k_dens_eta<<<ncell * kEtaCta, kEtaThreads, 0, st>>>((double)NO, h.R, orb, h.orbit_mult, vol, beta, eta, ro);
      NLF_CHECK_LAUNCH();
    }
    {
      ProfScope ps(PK_DENS_RHO, st);
      k2_rho<<<dim3((unsigned)((N + 255) / 256), ncell), 256, 0, st>>>(n_o, h.R, h.orbit_of, orb, ro, rho, u_out);
      NLF_CHECK_LAUNCH();
    }
    return NLF_OK;
  }
  {
    ProfScope ps(PK_DENS_FILTER, st);
    k_dens_symphi<<<dim3((unsigned)((NO + 255) / 256), ncell), 256, 0, st>>>(n_o, phi, phis);
    NLF_CHECK_LAUNCH();
    if (tiled) {
      if (tsm > 48 * 1024) NLF_CUDA_TRY(raise_dyn_smem(k_dens_filter_tile, (int)tsm));
      k_dens_filter_tile<<<dim3((unsigned)ntile, ncell), 256, tsm, st>>>(n_o, h.halo, h.ntap, h.tap_off, h.tap_w,
                                                                         phis, u, psum);
    } else {
      const size_t tap_smem = (size_t)h.ntap * (sizeof(double) + 3 * sizeof(int));
      if (tap_smem > 48 * 1024) NLF_CUDA_TRY(raise_dyn_smem(k_dens_filter, (int)tap_smem));
      k_dens_filter<<<dim3((unsigned)nsum, ncell), 256, tap_smem, st>>>(n_o, h.ntap, h.tap_off, h.tap_w, phis, u,
                                                                         psum);
    }
    NLF_CHECK_LAUNCH();
  }
  {
    ProfScope ps(PK_DENS_VAR, st);
    k_dens_var<<<dim3((unsigned)nvar, ncell), 256, 0, st>>>(N, nsum, u, psum, pvar);
    NLF_CHECK_LAUNCH();
  }
  {
    ProfScope ps(PK_DENS_FOLD, st);
    k_dens_fold<<<dim3((unsigned)((NO + 255) / 256), ncell), 256, 0, st>>>(n_o, u, nvar, pvar, phis);
    NLF_CHECK_LAUNCH();
    k_dens_orbits<<<dim3((unsigned)((h.R + 255) / 256), ncell), 256, 0, st>>>(n_o, h.R, h.orbit_abc, phis, orb);
    NLF_CHECK_LAUNCH();
  }
  {
    ProfScope ps(PK_DENS_ETA, st);
    k_dens_eta<<<ncell * kEtaCta, kEtaThreads, 0, st>>>((double)NO, h.R, orb, h.orbit_mult, vol, beta, eta, ro);
    NLF_CHECK_LAUNCH();
  }
  {
    ProfScope ps(PK_DENS_RHO, st);
    k_dens_rho<<<dim3((unsigned)((N + 255) / 256), ncell), 256, 0, st>>>(n_o, h.R, h.orbit_of, orb, ro, rho,
                                                                          u_out);
    NLF_CHECK_LAUNCH();
  }
  return NLF_OK;
}

// phi_bar (ncell, nrow, n_o^3) = the cotangents of phi for the rho cotangents gbar (ncell, nrow, n^3): the
// forward map again (its intermediates stay in the handle's workspace), then the transposes
static int density_vjp_run(DensityHandle& h, int ncell, int nrow, const double* phi, const double* vol, double beta,
                           const double* gbar, double* phibar, cudaStream_t st) {
  const int n_o = h.n_o, n = h.n, nvec = ncell * nrow;
  const bool sq = h.d == 2;
  const long NO = sq ? (long)n_o * n_o : (long)n_o * n_o * n_o, N = sq ? (long)n * n : (long)n * n * n;
  const size_t tsm = sq ? 0 : tile_smem(n, h.halo, h.ntap);
  if (tsm > 200 * 1024) {
    set_error("nlf_density_vjp: the filter radius %g needs %zu B of shared memory per tile (at most 200 KiB)", h.r,
              tsm);
    return NLF_EBADARG;
  }
  DensWs f;
  NLF_TRY(density_run(h, ncell, phi, vol, beta, nullptr, nullptr, nullptr, st, &f));
  const int ndot = (int)std::min<long>(128, (N + 2047) / 2048);
  const int ntile = ((n + kTX - 1) / kTX) * ((n + kTY - 1) / kTY);
  const size_t o_go = 0, o_ubs = al256(o_go + (size_t)nvec * NO * 8), o_dot = al256(o_ubs + (size_t)nvec * h.R * 8),
               o_uf = al256(o_dot + (size_t)nvec * ndot * 8), o_mt = al256(o_uf + (size_t)nvec * N * 8),
               total = al256(o_mt + (size_t)nvec * NO * 8);
  NLF_TRY(h.wsb.reserve(total));
  char* b = (char*)h.wsb.ptr;
  double* go = reinterpret_cast<double*>(b + o_go);
  double* ubs = reinterpret_cast<double*>(b + o_ubs);
  double* pdot = reinterpret_cast<double*>(b + o_dot);
  double* uf = reinterpret_cast<double*>(b + o_uf);
  double* mt = reinterpret_cast<double*>(b + o_mt);
  ProfScope ps(PK_DENS_VJP, st);
  const dim3 goct((unsigned)((NO + 255) / 256), nvec);
  if (sq) {
    k2_mirror_t<<<goct, 256, 0, st>>>(n_o, gbar, go);
    NLF_CHECK_LAUNCH();
    k2_dv_orbits<<<nvec, 1024, 0, st>>>(n_o, h.R, nrow, h.orbit_abc, h.orbit_mult, f.ro, go, beta, ubs);
    NLF_CHECK_LAUNCH();
    k2_dv_dot<<<dim3((unsigned)ndot, nvec), 256, 0, st>>>(n_o, h.R, nrow, h.orbit_of, ubs, f.u, pdot);
    NLF_CHECK_LAUNCH();
    k2_dv_filter<<<dim3((unsigned)((N + 255) / 256), nvec), 256, 0, st>>>(n_o, h.ntap, nrow, h.R, h.tap_off, h.tap_w,
                                                                           h.orbit_of, ubs, f.u, f.nsum, f.psum,
                                                                           f.nvar, f.pvar, ndot, pdot, uf);
    NLF_CHECK_LAUNCH();
    k2_mirror_t<<<goct, 256, 0, st>>>(n_o, uf, mt);
    NLF_CHECK_LAUNCH();
    k2_symphi<<<goct, 256, 0, st>>>(n_o, mt, phibar);
    NLF_CHECK_LAUNCH();
    return NLF_OK;
  }
  k_dv_mirror_t<<<goct, 256, 0, st>>>(n_o, gbar, go);
  NLF_CHECK_LAUNCH();
  k_dv_orbits<<<nvec, 1024, 0, st>>>(n_o, h.R, nrow, h.orbit_abc, h.orbit_mult, f.ro, go, beta, ubs);
  NLF_CHECK_LAUNCH();
  k_dv_dot<<<dim3((unsigned)ndot, nvec), 256, 0, st>>>(n_o, h.R, nrow, h.orbit_of, ubs, f.u, pdot);
  NLF_CHECK_LAUNCH();
  if (tsm > 48 * 1024) NLF_CUDA_TRY(raise_dyn_smem(k_dv_filter_tile, (int)tsm));
  k_dv_filter_tile<<<dim3((unsigned)ntile, nvec), 256, tsm, st>>>(n_o, h.halo, h.ntap, nrow, h.R, h.tap_off, h.tap_w,
                                                                  h.orbit_of, ubs, f.u, f.nsum, f.psum, f.nvar,
                                                                  f.pvar, ndot, pdot, uf);
  NLF_CHECK_LAUNCH();
  k_dv_mirror_t<<<goct, 256, 0, st>>>(n_o, uf, mt);
  NLF_CHECK_LAUNCH();
  k_dens_symphi<<<goct, 256, 0, st>>>(n_o, mt, phibar);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}

}  // namespace nlf

using namespace nlf;

struct nlf_density {
  DensityHandle h;
  DevBuf io;
};

extern "C" {

NLF_API int nlf_density_create(nlf_density** out, int n_o, double r) { return nlf_density_create_d(out, n_o, 3, r); }

NLF_API int nlf_density_create_d(nlf_density** out, int n_o, int d, double r) {
  if (!out || (d != 2 && d != 3) || n_o < 1 || n_o > (d == 3 ? 512 : 4096) || !(r >= 0.0) || !std::isfinite(r)) {
    set_error("nlf_density_create: bad arguments (d 2 or 3, n_o in [1, 512] for cubes or [1, 4096] for squares, "
              "r >= 0 finite)");
    return NLF_EBADARG;
  }
  *out = nullptr;
  nlf_density* H = new nlf_density();
  H->h.d = d;
  H->h.n_o = n_o;
  H->h.n = 2 * n_o;
  H->h.r = r;
  const int rc = density_tables(H->h);
  if (rc != NLF_OK) {
    density_free(H->h);
    delete H;
    return rc;
  }
  *out = H;
  return NLF_OK;
}

NLF_API int nlf_density_destroy(nlf_density* H) {
  if (!H) return NLF_OK;
  density_free(H->h);
  H->io.release();
  delete H;
  return NLF_OK;
}

NLF_API int nlf_density_orbits(const nlf_density* H) { return H ? H->h.R : -1; }

NLF_API int nlf_density_rho(nlf_density* H, int ncell, const double* phi, const double* v, double beta,
                            double* rho, double* u, double* eta, void* stream) {
  if (!H || ncell < 1 || !phi || !v || !(beta > 0.0) || !std::isfinite(beta) || (!rho && !u && !eta)) {
    set_error("nlf_density_rho: bad arguments (ncell >= 1, phi, v, beta > 0 and at least one output)");
    return NLF_EBADARG;
  }
  DensityHandle& h = H->h;
  cudaStream_t st = (cudaStream_t)stream;
  const long NO = h.d == 2 ? (long)h.n_o * h.n_o : (long)h.n_o * h.n_o * h.n_o,
             N = h.d == 2 ? (long)h.n * h.n : (long)h.n * h.n * h.n;
  const bool dphi = dens_on_dev(phi), dv = dens_on_dev(v), drho = !rho || dens_on_dev(rho),
             du = !u || dens_on_dev(u), deta = !eta || dens_on_dev(eta);
  const size_t o_phi = 0, o_v = al256(o_phi + (dphi ? 0 : (size_t)ncell * NO * 8)),
               o_rho = al256(o_v + (dv ? 0 : (size_t)ncell * 8)),
               o_u = al256(o_rho + (drho ? 0 : (size_t)ncell * N * 8)),
               o_eta = al256(o_u + (du ? 0 : (size_t)ncell * N * 8)), total = al256(o_eta + (size_t)ncell * 8);
  NLF_TRY(H->io.reserve(total));
  char* b = (char*)H->io.ptr;
  const double* phid = phi;
  const double* vd = v;
  if (!dphi) {
    NLF_CUDA_TRY(cudaMemcpyAsync(b + o_phi, phi, (size_t)ncell * NO * 8, cudaMemcpyHostToDevice, st));
    phid = reinterpret_cast<const double*>(b + o_phi);
  }
  if (!dv) {
    NLF_CUDA_TRY(cudaMemcpyAsync(b + o_v, v, (size_t)ncell * 8, cudaMemcpyHostToDevice, st));
    vd = reinterpret_cast<const double*>(b + o_v);
  }
  double* rhod = drho ? rho : reinterpret_cast<double*>(b + o_rho);
  double* ud = du ? u : reinterpret_cast<double*>(b + o_u);
  double* etad = deta ? eta : reinterpret_cast<double*>(b + o_eta);
  if (!etad) etad = reinterpret_cast<double*>(b + o_eta);
  NLF_TRY(density_run(h, ncell, phid, vd, beta, rhod, ud, etad, st));
  if (rho && !drho) NLF_CUDA_TRY(cudaMemcpyAsync(rho, rhod, (size_t)ncell * N * 8, cudaMemcpyDeviceToHost, st));
  if (u && !du) NLF_CUDA_TRY(cudaMemcpyAsync(u, ud, (size_t)ncell * N * 8, cudaMemcpyDeviceToHost, st));
  if (eta && !deta) NLF_CUDA_TRY(cudaMemcpyAsync(eta, etad, (size_t)ncell * 8, cudaMemcpyDeviceToHost, st));
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  return NLF_OK;
}

NLF_API int nlf_density_vjp(nlf_density* H, int ncell, int nrow, const double* phi, const double* v, double beta,
                            const double* rho_bar, double* phi_bar, void* stream) {
  if (!H || ncell < 1 || nrow < 1 || !phi || !v || !rho_bar || !phi_bar || !(beta > 0.0) || !std::isfinite(beta)) {
    set_error("nlf_density_vjp: bad arguments (ncell, nrow >= 1, phi, v, rho_bar, phi_bar, beta > 0)");
    return NLF_EBADARG;
  }
  DensityHandle& h = H->h;
  cudaStream_t st = (cudaStream_t)stream;
  const long NO = h.d == 2 ? (long)h.n_o * h.n_o : (long)h.n_o * h.n_o * h.n_o,
             N = h.d == 2 ? (long)h.n * h.n : (long)h.n * h.n * h.n;
  const size_t nvec = (size_t)ncell * nrow;
  const bool dphi = dens_on_dev(phi), dv = dens_on_dev(v), dg = dens_on_dev(rho_bar), dout = dens_on_dev(phi_bar);
  const size_t o_phi = 0, o_v = al256(o_phi + (dphi ? 0 : (size_t)ncell * NO * 8)),
               o_g = al256(o_v + (dv ? 0 : (size_t)ncell * 8)), o_out = al256(o_g + (dg ? 0 : nvec * N * 8)),
               total = al256(o_out + (dout ? 0 : nvec * NO * 8));
  NLF_TRY(H->io.reserve(total));
  char* b = (char*)H->io.ptr;
  const double* phid = phi;
  const double* vd = v;
  const double* gd = rho_bar;
  if (!dphi) {
    NLF_CUDA_TRY(cudaMemcpyAsync(b + o_phi, phi, (size_t)ncell * NO * 8, cudaMemcpyHostToDevice, st));
    phid = reinterpret_cast<const double*>(b + o_phi);
  }
  if (!dv) {
    NLF_CUDA_TRY(cudaMemcpyAsync(b + o_v, v, (size_t)ncell * 8, cudaMemcpyHostToDevice, st));
    vd = reinterpret_cast<const double*>(b + o_v);
  }
  if (!dg) {
    NLF_CUDA_TRY(cudaMemcpyAsync(b + o_g, rho_bar, nvec * N * 8, cudaMemcpyHostToDevice, st));
    gd = reinterpret_cast<const double*>(b + o_g);
  }
  double* outd = dout ? phi_bar : reinterpret_cast<double*>(b + o_out);
  NLF_TRY(density_vjp_run(h, ncell, nrow, phid, vd, beta, gd, outd, st));
  if (!dout) NLF_CUDA_TRY(cudaMemcpyAsync(phi_bar, outd, nvec * NO * 8, cudaMemcpyDeviceToHost, st));
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  return NLF_OK;
}

}  // extern "C"
