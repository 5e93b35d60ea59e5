// Matrix-free periodic Q1 stiffness operator, load vector and C / dC assembly.
//
// apply  y = K(s) x = scatter(s_e Ke gather(x))            nlfiber/linear.py:80-92,143-144
// load   f_I = scatter(s_e (E_I G))                          nlfiber/linear.py:146-149
// C      C_IJ = mean_e s_e b_e(E_I + u_I, E_J + u_J)          nlfiber/linear.py:220-229
// dC/drho (correctors held fixed)                            nlfiber/linear.py:10-12,137-141,259-264
//
// The apply kernel marches a CTA along x (the slowest axis) over a TY x TZ tile of the (y, z) plane. Each
// thread owns one element of the (TY+1) x (TZ+1) element layer that touches the tile (one element row and
// column of halo). Per layer it reads its 8 corner nodes from the two shared node planes of the layer, computes
// the 24 element forces with the mode form of Ke, adds the
// forces on the finished plane to the top-corner forces carried from the previous layer, and publishes them
// to shared memory; each output node then sums its 4 in-plane element contributions. Node planes are
// prefetched three layers ahead into a three-slot ring, so one barrier per layer suffices. Every output node is
// written once, with a fixed summation order (deterministic), and the whole 27-point stencil stays on chip.
#include <climits>

#include "nlf_internal.h"
#include "nlf_prof.cuh"

namespace nlf {

// Asynchronous global -> shared copy of one element (4 or 8 bytes, through L1), and a wait for this thread's
// copies in flight.
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* dst, const T* src) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte elements");
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src),
               "n"((int)sizeof(T))
               : "memory");
}
__device__ __forceinline__ void cp_async_commit_all() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_none() { asm volatile("cp.async.wait_all;" ::: "memory"); }

template <typename T, int TY, int TZ, int MINB>
__global__ void __launch_bounds__(((TY + 1) * (TZ + 1) + 31) / 32 * 32, MINB)
k_apply(const T* __restrict__ s, const T* __restrict__ x, T* __restrict__ y, int n0, int n1, int n2, int m,
        int lx, const CellState* __restrict__ cs, ModeC<T> kc, double* __restrict__ partial,
        unsigned long long* __restrict__ units, int ukind) {
  constexpr int HY = TY + 2, HZ = TZ + 2, EY = TY + 1, EZ = TZ + 1;
  constexpr int NE = EY * EZ;
  constexpr int NT = (NE + 31) / 32 * 32;
  constexpr int NP = HY * HZ;
  constexpr int PF = (3 * NP + NT - 1) / NT;  // plane values each thread prefetches per layer
  constexpr int PFF = (3 * NP) / NT;          // ... of which the first PFF exist for every thread
  // One barrier per layer. Dynamic shared memory (apply_smem<T, TY, TZ>() bytes): a ring of three node planes
  // [3][3 comps][NP] and element forces [2][4 corners][3 comps][NE] (alternating buffers). Plane k + 3 is copied
  // into the slot of plane k by cp.async after the barrier of layer k (the last layer that reads plane k); each
  // thread waits for its copies before the barrier of layer k + 1, which publishes the plane before layer k + 2
  // reads it. An element's stiffness scale is read by its own thread only and stays in a register. The slots are
  // tracked as offsets that rotate every layer (no index arithmetic mod 3), and every offset into a vector is
  // 32-bit (the host bounds 3 N below 2^31).
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* const pl = reinterpret_cast<T*>(smem_raw);
  T* const g = pl + 9 * NP;
  __shared__ int gys[HY], gzs[HZ];
  __shared__ double red[32 * 4];

  const int vec = blockIdx.z, cell = vec / m;
  if (!vec_live(cs, vec, m)) return;
  prof_count(units, ukind);
  const int P = n1 * n2, N = n0 * P;
  const int ntz = (n2 + TZ - 1) / TZ;
  const int z0 = (blockIdx.x % ntz) * TZ, y0 = (blockIdx.x / ntz) * TY;
  const int xb = blockIdx.y * lx, xe = min(xb + lx, n0);
  const T* __restrict__ xv = x + (long)vec * 3 * N;
  T* __restrict__ yv = y + (long)vec * 3 * N;
  const T* __restrict__ sv = s + (long)cell * N;
  const int tid = threadIdx.x;

  for (int i = tid; i < HY; i += NT) gys[i] = wrap(y0 - 1 + i, n1);
  for (int i = tid; i < HZ; i += NT) gzs[i] = wrap(z0 - 1 + i, n2);
  __syncthreads();

  // per-thread offsets (within a node plane of the vector) of the plane values this thread loads
  int poff[PF];
#pragma unroll
  for (int i = 0; i < PF; ++i) {
    const int idx = tid + i * NT;
    poff[i] = -1;
    if (idx < 3 * NP) {
      const int c = idx / NP, r = idx - c * NP;
      const int hy = r / HZ, hz = r - hy * HZ;
      poff[i] = c * N + gys[hy] * n2 + gzs[hz];
    }
  }
  // thread -> element: the EY x TZ elements right of the halo column run along rows of TZ threads, so that a
  // half-warp's 8-byte accesses (node corners, forces, scales) fall on 16 consecutive words of one row (no bank
  // conflicts when TZ is a multiple of 16); the EY halo-column elements follow. e = ey EZ + ez indexes the
  // element's force and scale slots.
  const bool ev = tid < NE;
  const int ey = tid < EY * TZ ? tid / TZ : tid - EY * TZ;
  const int ez = tid < EY * TZ ? 1 + (tid - (tid / TZ) * TZ) : 0;
  const int e = ey * EZ + ez;
  const int soff = ev ? gys[ey] * n2 + gzs[ez] : 0;
  int cidx[4];  // in-plane corner q = ay + 2 az of this element, in node-plane coordinates
#pragma unroll
  for (int q = 0; q < 4; ++q) cidx[q] = (ey + (q & 1)) * HZ + ez + (q >> 1);
  const int ty = tid / TZ, tz = tid - (tid / TZ) * TZ;
  const bool outp = tid < TY * TZ;
  const bool ownv = outp && y0 + ty < n1 && z0 + tz < n2;  // this thread writes output node (y0 + ty, z0 + tz)
  const int own = (ty + 1) * HZ + tz + 1;                   // the output node in node-plane coordinates
  const int inpl = (y0 + ty) * n2 + z0 + tz;               // ... and within a plane of the vector
  const int e00 = (ty + 1) * EZ + (tz + 1);  // node (ty+1, tz+1) is corner q = ay + 2az of element (ty+1-ay, tz+1-az)

  // prologue: node planes xb - 1, xb, xb + 1 into ring slots 0, 1, 2 and the element scales of layer xb - 1
#pragma unroll
  for (int i = 0; i < PF; ++i)
    if (i < PFF || poff[i] >= 0) {
      const int idx = tid + i * NT;
#pragma unroll
      for (int j = 0; j < 3; ++j) pl[j * 3 * NP + idx] = __ldg(xv + (wrap(xb - 1 + j, n0) * P + poff[i]));
    }
  T s_cur = ev ? __ldg(sv + (wrap(xb - 1, n0) * P + soff)) : T(0);  // scale of this element in layer k
  __syncthreads();

  T ft[3][4];  // top-corner forces carried to the next layer
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int q = 0; q < 4; ++q) ft[c][q] = T(0);
  double acc[4] = {0.0, 0.0, 0.0, 0.0};

  int r0 = 0, r1 = 3 * NP, r2 = 6 * NP;  // ring slots of planes k, k + 1, k + 2
  int gc = 0;                            // this layer's force buffer (the other: 12 NE - gc)
  int pofs = wrap(xb + 2, n0) * P;       // plane k + 3 within the vector
  int sofs = wrap(xb, n0) * P + soff;    // this element's scale in layer k + 1
  int kofs = (xb - 1) * P;               // plane k
#pragma unroll 2
  for (int k = xb - 1; k < xe; ++k) {
    const bool pnext = k + 3 <= xe, snext = k + 1 < xe;
    const T s_nxt = (snext && ev) ? __ldg(sv + sofs) : T(0);  // the element's scale in layer k + 1
    const T* lo = pl + r0;
    const T* hi = pl + r1;
    T* gk = g + gc;
    T xo[3] = {T(0), T(0), T(0)};
    if (ev) {
      // (carrying the lower corners in registers instead of re-reading them measured slower: register pressure)
      T v[3][8], f[3][8];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          v[c][2 * q] = lo[c * NP + cidx[q]];
          v[c][2 * q + 1] = hi[c * NP + cidx[q]];
        }
      const ModeC<T> ks = scale_modec(kc, s_cur);
      element_force(v, ks, f);
      if (k >= xb) {
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int q = 0; q < 4; ++q) gk[(q * 3 + c) * NE + e] = ft[c][q] + f[c][2 * q];
      }
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int q = 0; q < 4; ++q) ft[c][q] = f[c][2 * q + 1];
    }
    if (partial && ownv && k >= xb) {
#pragma unroll
      for (int c = 0; c < 3; ++c) xo[c] = lo[c * NP + own];
    }
    cp_async_wait_none();  // this thread's copies of plane k + 2 (issued in layer k - 1)
    __syncthreads();       // gk complete; every read of plane k is done; plane k + 2 visible
    if (k >= xb && ownv) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const T* gc0 = gk + c * NE;
        const T o = (gc0[e00] + gc0[3 * NE + e00 - EZ]) + (gc0[6 * NE + e00 - 1] + gc0[9 * NE + e00 - EZ - 1]);
        yv[c * N + kofs + inpl] = o;
        if (partial) {
          acc[c] += (double)o;
          acc[3] += (double)xo[c] * (double)o;
        }
      }
    }
    if (pnext) {
#pragma unroll
      for (int i = 0; i < PF; ++i)
        if (i < PFF || poff[i] >= 0)
          cp_async_elem(pl + (r0 + tid + i * NT), xv + (pofs + poff[i]));  // plane k + 3 replaces plane k
      cp_async_commit_all();
    }
    const int rt = r0;
    r0 = r1;
    r1 = r2;
    r2 = rt;
    gc = 12 * NE - gc;
    s_cur = s_nxt;
    pofs += P;
    if (pofs == N) pofs = 0;
    sofs += P;
    if (sofs >= N) sofs -= N;
    kofs += P;
  }
  if (partial) {
    block_sum<4>(acc, red);
    if (tid == 0) {
      const long blk = blockIdx.x + (long)gridDim.x * blockIdx.y;
      const long nblk = (long)gridDim.x * gridDim.y;
      double* o = partial + ((long)vec * nblk + blk) * 4;
      o[0] = acc[0];
      o[1] = acc[1];
      o[2] = acc[2];
      o[3] = acc[3];
    }
  }
}

// Shared-memory bytes of a k_apply tile.
template <typename T, int TY, int TZ>
constexpr size_t apply_smem() {
  constexpr int NP = (TY + 2) * (TZ + 2), NE = (TY + 1) * (TZ + 1);
  return sizeof(T) * (9 * NP + 24 * NE);
}

template <typename T, int TY, int TZ, int MINB>
static int launch_apply_tile(const LinearHandle& h, const T* s, int m, int nvec, const T* x, T* y,
                             const CellState* cs, double* partial, int* nblk_out, cudaStream_t st) {
  constexpr int NT = ((TY + 1) * (TZ + 1) + 31) / 32 * 32;
  constexpr size_t smem = apply_smem<T, TY, TZ>();
  const Geom& g = h.g;
  const int tiles = ((g.n2 + TZ - 1) / TZ) * ((g.n1 + TY - 1) / TY);
  // marches of 16 planes (one halo plane per 16 re-read). The split depends on the grid and the handle's tile
  // alone, so that the partial sums of a vector, and with them every PCG scalar, are the same whatever else is in
  // the batch.
  const int lx = g.n0 >= 32 ? 16 : g.n0;
  const int chunks = (g.n0 + lx - 1) / lx;
  if (3 * g.N > (long)INT_MAX) {
    set_error("apply: 3 n0 n1 n2 = %ld exceeds the 32-bit offsets of the kernel", 3 * g.N);
    return NLF_EBADARG;
  }
  if (tiles * chunks > kApplyMaxBlocks) {
    set_error("apply: %d blocks per vector exceed the partial-sum buffer (%d)", tiles * chunks, kApplyMaxBlocks);
    return NLF_EBADARG;
  }
  if (nblk_out) *nblk_out = tiles * chunks;
  dim3 grid(tiles, chunks, nvec);
  const int kind = sizeof(T) == 4 ? PK_APPLY32 : PK_APPLY64;
  NLF_CUDA_TRY(raise_dyn_smem(k_apply<T, TY, TZ, MINB>, (int)smem));
  ProfScope ps(kind, st);
  k_apply<T, TY, TZ, MINB><<<grid, NT, smem, st>>>(s, x, y, g.n0, g.n1, g.n2, m, lx, cs, make_modec<T>(h.lam, h.mu),
                                                    partial, prof_units(), kind);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}

// The tile variants of the apply (output tile TY x TZ of the (y, z) plane, minimum resident CTAs per SM, which
// caps the registers): variant 0 is the default; the autotuner (nlf_linear_autotune) may pick another per handle.
#define NLF_APPLY_VARIANTS_F64(X) X(0, 8, 16, 3) X(1, 4, 16, 5) X(2, 8, 8, 5) X(3, 16, 8, 3) X(4, 4, 32, 2) \
  X(5, 8, 16, 4) X(6, 2, 32, 4) X(7, 8, 32, 1)
#define NLF_APPLY_VARIANTS_F32(X) X(0, 8, 32, 2) X(1, 8, 16, 3) X(2, 4, 32, 4) X(3, 16, 32, 1) X(4, 16, 16, 2)

int apply_variants(bool fp64) {
#define NLF_COUNT(i, ty, tz, mb) +1
  return fp64 ? (0 NLF_APPLY_VARIANTS_F64(NLF_COUNT)) : (0 NLF_APPLY_VARIANTS_F32(NLF_COUNT));
#undef NLF_COUNT
}

void apply_variant_tile(bool fp64, int v, int* ty, int* tz, int* minb) {
#define NLF_TILE(i, a, b, c) \
  if (v == i) {             \
    *ty = a;                \
    *tz = b;                \
    *minb = c;              \
  }
  *ty = *tz = *minb = 0;
  if (fp64) {
    NLF_APPLY_VARIANTS_F64(NLF_TILE)
  } else {
    NLF_APPLY_VARIANTS_F32(NLF_TILE)
  }
#undef NLF_TILE
}

template <typename T>
int launch_apply(const LinearHandle& h, const T* s, int m, int nvec, const T* x, T* y, const CellState* cs,
                 double* partial, int* nblk_out, cudaStream_t st) {
  const int v = h.apply_variant[sizeof(T) == 8 ? 1 : 0];
#define NLF_CASE(i, ty, tz, mb) \
  case i:                       \
    return launch_apply_tile<T, ty, tz, mb>(h, s, m, nvec, x, y, cs, partial, nblk_out, st);
  if constexpr (sizeof(T) == 8) {
    switch (v) { NLF_APPLY_VARIANTS_F64(NLF_CASE) default: break; }
  } else {
    switch (v) { NLF_APPLY_VARIANTS_F32(NLF_CASE) default: break; }
  }
#undef NLF_CASE
  set_error("apply: no tile variant %d", v);
  return NLF_EBADARG;
}

template int launch_apply<float>(const LinearHandle&, const float*, int, int, const float*, float*,
                                 const CellState*, double*, int*, cudaStream_t);
template int launch_apply<double>(const LinearHandle&, const double*, int, int, const double*, double*,
                                  const CellState*, double*, int*, cudaStream_t);

// ---- load: f[cell][I][c][n] = sign * sum_a s(n - off_a) fe[I][3a + c] -----------------------------------
__global__ void k_load(const double* __restrict__ s, const double* __restrict__ fe, int m, int n0, int n1,
                       int n2, double* __restrict__ f, double sign) {
  const long N = (long)n0 * n1 * n2;
  const long n = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const int cell = blockIdx.y;
  if (n >= N) return;
  const int k = (int)(n % n2), j = (int)((n / n2) % n1), i = (int)(n / ((long)n1 * n2));
  const double* sv = s + (long)cell * N;
  double se[8];
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int ii = wrap(i - (a & 1), n0), jj = wrap(j - ((a >> 1) & 1), n1), kk = wrap(k - (a >> 2), n2);
    se[a] = sv[((long)ii * n1 + jj) * n2 + kk];
  }
  for (int I = 0; I < m; ++I) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double acc = 0.0;
#pragma unroll
      for (int a = 0; a < 8; ++a) acc += se[a] * fe[I * 24 + 3 * a + c];
      f[(((long)cell * m + I) * 3 + c) * N + n] = sign * acc;
    }
  }
}

int launch_load(const LinearHandle& h, const double* s, const double* fe, int m, int ncell, double* f,
                double sign, cudaStream_t st) {
  const long N = h.g.N;
  dim3 grid((unsigned)((N + 255) / 256), ncell);
  ProfScope ps(PK_LOAD, st);
  k_load<<<grid, 256, 0, st>>>(s, fe, m, h.g.n0, h.g.n1, h.g.n2, f, sign);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}

// ---- C and dC/drho ----------------------------------------------------------------------------------------
// b_IJ(e) = E_I D E_J + E_I . D eps_J + E_J . D eps_I + u_I^T Ke u_J, with eps the element-mean strain of the
// corrector (G u = D mean(B) u, nlfiber/linear.py:112) and u^T Ke u in mode form (c'_I . M c'_J).
constexpr int kMaxM = 6;
constexpr int kMaxPairs = kMaxM * (kMaxM + 1) / 2;

__device__ __forceinline__ void gather_modes(const double* __restrict__ u, long N, const long (&nid)[8],
                                             double (&c)[3][8]) {
#pragma unroll
  for (int cc = 0; cc < 3; ++cc) {
#pragma unroll
    for (int a = 0; a < 8; ++a) c[cc][a] = u[cc * N + nid[a]];
    butterfly8(c[cc]);
  }
}

__device__ __forceinline__ void mean_stress(const double (&c)[3][8], double lam, double mu, double (&sig)[6]) {
  // Voigt strain (engineering shear) of the constant-strain mode: H[c][d] = c'[c][1<<d] / 4
  const double e0 = 0.25 * c[0][1], e1 = 0.25 * c[1][2], e2 = 0.25 * c[2][4];
  const double g12 = 0.25 * (c[1][4] + c[2][2]), g02 = 0.25 * (c[0][4] + c[2][1]),
               g01 = 0.25 * (c[0][2] + c[1][1]);
  const double tr = lam * (e0 + e1 + e2);
  sig[0] = tr + 2.0 * mu * e0;
  sig[1] = tr + 2.0 * mu * e1;
  sig[2] = tr + 2.0 * mu * e2;
  sig[3] = mu * g12;
  sig[4] = mu * g02;
  sig[5] = mu * g01;
}

__global__ void __launch_bounds__(128) k_bilinear(const double* __restrict__ s, const double* __restrict__ Es,
                                                  const double* __restrict__ EDE, int m, int n0, int n1,
                                                  int n2, double lam, double mu, const double* __restrict__ u,
                                                  double* __restrict__ Cpart, const double* __restrict__ rho,
                                                  double emin, double pexp, double* __restrict__ dC) {
  __shared__ double red[32 * kMaxPairs];
  const long N = (long)n0 * n1 * n2;
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const int cell = blockIdx.y;
  const bool valid = e < N;
  double acc[kMaxPairs];
#pragma unroll
  for (int q = 0; q < kMaxPairs; ++q) acc[q] = 0.0;
  if (valid) {
    const int k = (int)(e % n2), j = (int)((e / n2) % n1), i = (int)(e / ((long)n1 * n2));
    long nid[8];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const int ii = wrap(i + (a & 1), n0), jj = wrap(j + ((a >> 1) & 1), n1), kk = wrap(k + (a >> 2), n2);
      nid[a] = ((long)ii * n1 + jj) * n2 + kk;
    }
    const double se = s[(long)cell * N + e];
    double ds = 0.0;
    if (dC) {
      const double r = rho[(long)cell * N + e];
      const double rc = r > 1.0 ? 1.0 : (r < 0.0 ? 0.0 : r);
      ds = (r > 1.0 || r < 0.0) ? 0.0 : (1.0 - emin) * pexp * pow(rc, pexp - 1.0);
      ds /= (double)N;
    }
    const ModeC<double> unit = make_modec<double>(lam, mu);
    const double* ub = u + (long)cell * m * 3 * N;
    int q = 0;
    for (int I = 0; I < m; ++I) {
      double cI[3][8], fI[3][8], sI[6];
      gather_modes(ub + (long)I * 3 * N, N, nid, cI);
      mode_force(cI, unit, fI);
      mean_stress(cI, lam, mu, sI);
      for (int J = I; J < m; ++J, ++q) {
        double cJ[3][8], sJ[6];
        if (J == I) {
#pragma unroll
          for (int cc = 0; cc < 3; ++cc)
#pragma unroll
            for (int a = 0; a < 8; ++a) cJ[cc][a] = cI[cc][a];
#pragma unroll
          for (int v = 0; v < 6; ++v) sJ[v] = sI[v];
        } else {
          gather_modes(ub + (long)J * 3 * N, N, nid, cJ);
          mean_stress(cJ, lam, mu, sJ);
        }
        double b = EDE[I * m + J];
#pragma unroll
        for (int v = 0; v < 6; ++v) b += Es[I * 6 + v] * sJ[v] + Es[J * 6 + v] * sI[v];
#pragma unroll
        for (int cc = 0; cc < 3; ++cc)
#pragma unroll
          for (int a = 1; a < 8; ++a) b += cJ[cc][a] * fI[cc][a];
        // accumulate into the pair slot (unrolled index keeps acc in registers)
#pragma unroll
        for (int t = 0; t < kMaxPairs; ++t)
          if (t == q) acc[t] += se * b;
        if (dC) {
          double* o = dC + ((long)cell * m * m) * N;
          o[((long)I * m + J) * N + e] = ds * b;
          o[((long)J * m + I) * N + e] = ds * b;
        }
      }
    }
  }
  block_sum<kMaxPairs>(acc, red);
  if (threadIdx.x == 0) {
    double* o = Cpart + ((long)cell * gridDim.x + blockIdx.x) * kMaxPairs;
#pragma unroll
    for (int t = 0; t < kMaxPairs; ++t) o[t] = acc[t];
  }
}

__global__ void k_reduce_C(const double* __restrict__ Cpart, int nblk, int m, double invN,
                           double* __restrict__ C) {
  const int cell = blockIdx.x;
  const int npair = m * (m + 1) / 2;
  for (int t = threadIdx.x; t < npair; t += blockDim.x) {
    double a = 0.0;
    for (int b = 0; b < nblk; ++b) a += Cpart[((long)cell * nblk + b) * kMaxPairs + t];
    // pair t -> (I, J), I <= J, in the order of k_bilinear
    int I = 0, rem = t;
    while (rem >= m - I) {
      rem -= m - I;
      ++I;
    }
    const int J = I + rem;
    C[((long)cell * m + I) * m + J] = a * invN;
    C[((long)cell * m + J) * m + I] = a * invN;
  }
}

// sbar_e = sum_I lam_I,e . (Ke u_I,e + G^T E_I) = sum_I (c'_lam,I . M c'_u,I + E_I . D eps(lam_I)): the VJP in s
// of <lam, residual(s, Es, u)>, the backward of the reference's corrector custom VJP (nlfiber/linear.py:124-131).
// With rho, the same times ds/drho (rhobar). u, lam: SoA [cell][I][comp][N]; one thread per element.
__global__ void __launch_bounds__(128) k_adjoint_sbar(const double* __restrict__ Es, int m, int n0, int n1, int n2,
                                                      double lam, double mu, const double* __restrict__ u,
                                                      const double* __restrict__ lamv, const double* __restrict__ rho,
                                                      double emin, double pexp, double* __restrict__ out) {
  const long N = (long)n0 * n1 * n2;
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const int cell = blockIdx.y;
  if (e >= N) return;
  const int k = (int)(e % n2), j = (int)((e / n2) % n1), i = (int)(e / ((long)n1 * n2));
  long nid[8];
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int ii = wrap(i + (a & 1), n0), jj = wrap(j + ((a >> 1) & 1), n1), kk = wrap(k + (a >> 2), n2);
    nid[a] = ((long)ii * n1 + jj) * n2 + kk;
  }
  const ModeC<double> unit = make_modec<double>(lam, mu);
  double acc = 0.0;
  for (int I = 0; I < m; ++I) {
    const long off = ((long)cell * m + I) * 3 * N;
    double cu[3][8], fu[3][8], cl[3][8], sl[6];
    gather_modes(u + off, N, nid, cu);
    mode_force(cu, unit, fu);
    gather_modes(lamv + off, N, nid, cl);
    mean_stress(cl, lam, mu, sl);
    double b = 0.0;
#pragma unroll
    for (int v = 0; v < 6; ++v) b += Es[I * 6 + v] * sl[v];
#pragma unroll
    for (int cc = 0; cc < 3; ++cc)
#pragma unroll
      for (int a = 1; a < 8; ++a) b += cl[cc][a] * fu[cc][a];
    acc += b;
  }
  if (rho) {
    const double r = rho[(long)cell * N + e];
    const double rc = r > 1.0 ? 1.0 : (r < 0.0 ? 0.0 : r);
    acc *= (r > 1.0 || r < 0.0) ? 0.0 : (1.0 - emin) * pexp * pow(rc, pexp - 1.0);
  }
  out[(long)cell * N + e] = acc;
}

int launch_adjoint_sbar(const LinearHandle& h, const double* Es, int m, int ncell, const double* u,
                        const double* lamv, const double* rho, double* out, cudaStream_t st) {
  const long N = h.g.N;
  ProfScope ps(PK_BILINEAR, st);
  k_adjoint_sbar<<<dim3((unsigned)((N + 127) / 128), ncell), 128, 0, st>>>(Es, m, h.g.n0, h.g.n1, h.g.n2, h.lam,
                                                                           h.mu, u, lamv, rho, h.emin, h.p, out);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}

int launch_bilinear(const LinearHandle& h, const double* s, const double* EsEDE, int m, int ncell,
                    const double* u, double* Cpart, int* nblk, const double* rho, double* dC, cudaStream_t st) {
  if (m > kMaxM) {
    set_error("bilinear: at most %d load cases per cell (got %d)", kMaxM, m);
    return NLF_EBADARG;
  }
  const long N = h.g.N;
  const int nb = (int)((N + 127) / 128);
  *nblk = nb;
  dim3 grid(nb, ncell);
  ProfScope ps(PK_BILINEAR, st);
  k_bilinear<<<grid, 128, 0, st>>>(s, EsEDE, EsEDE + m * 6, m, h.g.n0, h.g.n1, h.g.n2, h.lam, h.mu, u, Cpart,
                                   rho, h.emin, h.p, dC);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}

int launch_reduce_C(const LinearHandle& h, const double* Cpart, int nblk, int m, int ncell, double* C,
                    cudaStream_t st) {
  ProfScope ps(PK_OTHER, st);
  k_reduce_C<<<ncell, 32, 0, st>>>(Cpart, nblk, m, 1.0 / (double)h.g.N, C);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}

}  // namespace nlf
