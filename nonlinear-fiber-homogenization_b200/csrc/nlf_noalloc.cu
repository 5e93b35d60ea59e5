// C_IJ assembly that allocates nothing: nlf_bilinear_noalloc.
//
// Who needs it: code that may not call cudaMalloc while it runs, e.g. a handler invoked by a framework that
// owns all device memory through its own pool (an XLA / JAX custom call, a caching allocator that must see
// every byte), code running inside another library's callback, or a service that has pre-reserved its memory
// and must not fail on allocation mid-request. Such callers already hold device arrays for the inputs and
// the output; what the regular path (nlf_bilinear) adds on top is staging buffers and a scratch array of
// per-block partial sums, both from the handle's cudaMalloc'ed workspace. This variant keeps the partial sums
// in a fixed file-scope device array instead and reads the correctors in the caller's (reference) layout, so
// it needs neither a handle nor any allocation.
//
// Limits: at most kNaCells cells and kNaCases load cases per call. Every call uses the same array: two calls
// whose kernels overlap on the GPU (different streams, or different host threads) race on it and give wrong
// results; serialise them. Each call writes every partial it later reads, so nothing needs clearing between
// calls, and the array keeps the last call's partials.
//
// Set-up: the first call on a device (with that device current) looks up the array's device address with
// cudaGetSymbolAddress and remembers it per device. Make that first call before any stream capture. The
// remembered address belongs to the device's current context: after cudaDeviceReset on that device it is stale,
// so a process that resets a device must not call this entry point on it again.
#include <atomic>
#include <cstring>
#include "nlf_internal.h"

namespace nlf {
namespace {

constexpr int kNaCells = 64;   // cells per call
constexpr int kNaCases = 6;    // load cases per cell
constexpr int kNaPairs = kNaCases * (kNaCases + 1) / 2;
constexpr int kNaBlocks = 64;  // CTAs per cell (grid-stride over the cell's elements)
constexpr int kNaThreads = 128;
constexpr int kNaMaxDevices = 64;

// 64 cells x 64 CTAs x 21 pairs x 8 B = 672 KiB, held by every GPU that loads the library until exit.
static __device__ __align__(256) double g_na_scratch[kNaCells * kNaBlocks * kNaPairs];

// per device ordinal: the scratch array's device address (every writer stores the same value)
std::atomic<double*> g_na_addr[kNaMaxDevices] = {};

struct NaArgs {
  double Es[kNaCases * 6];
  double EDE[kNaCases * kNaCases];
  double lam, mu;
  int m, n0, n1, n2;
};

__device__ __forceinline__ void na_modes(const double* __restrict__ u, const long (&nid)[8], double (&c)[3][8]) {
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const double* p = u + nid[a] * 3;
    c[0][a] = p[0];
    c[1][a] = p[1];
    c[2][a] = p[2];
  }
  butterfly8(c[0]);
  butterfly8(c[1]);
  butterfly8(c[2]);
}

// D times the Voigt strain of the constant-strain mode (H[c][d] = c'[c][1<<d] / 4, engineering shear)
__device__ __forceinline__ void na_stress(const double (&c)[3][8], double lam, double mu, double (&sig)[6]) {
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

// One CTA-row of partials per (cell, block): pair sums of s_e b_IJ(e) over the block's elements.
__global__ void __launch_bounds__(kNaThreads) k_na_partials(NaArgs a, const double* __restrict__ s,
                                                             const double* __restrict__ u,
                                                             double* __restrict__ scratch) {
  __shared__ double red[32 * kNaPairs];
  const long N = (long)a.n0 * a.n1 * a.n2;
  const int cell = blockIdx.y;
  const ModeC<double> unit = make_modec<double>(a.lam, a.mu);
  double acc[kNaPairs];
#pragma unroll
  for (int q = 0; q < kNaPairs; ++q) acc[q] = 0.0;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < N; e += (long)gridDim.x * blockDim.x) {
    const int k = (int)(e % a.n2), j = (int)((e / a.n2) % a.n1), i = (int)(e / ((long)a.n1 * a.n2));
    long nid[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int ii = wrap(i + (q & 1), a.n0), jj = wrap(j + ((q >> 1) & 1), a.n1), kk = wrap(k + (q >> 2), a.n2);
      nid[q] = ((long)ii * a.n1 + jj) * a.n2 + kk;
    }
    const double se = s[(long)cell * N + e];
    const double* ub = u + (long)cell * a.m * N * 3;
    int q = 0;
    for (int I = 0; I < a.m; ++I) {
      double cI[3][8], fI[3][8], sI[6];
      na_modes(ub + (long)I * N * 3, nid, cI);
      mode_force(cI, unit, fI);
      na_stress(cI, a.lam, a.mu, sI);
      for (int J = I; J < a.m; ++J, ++q) {
        double cJ[3][8], sJ[6];
        na_modes(ub + (long)J * N * 3, nid, cJ);
        na_stress(cJ, a.lam, a.mu, sJ);
        double b = a.EDE[I * a.m + J];
#pragma unroll
        for (int v = 0; v < 6; ++v) b += a.Es[I * 6 + v] * sJ[v] + a.Es[J * 6 + v] * sI[v];
#pragma unroll
        for (int cc = 0; cc < 3; ++cc)
#pragma unroll
          for (int p = 1; p < 8; ++p) b += cJ[cc][p] * fI[cc][p];
#pragma unroll
        for (int t = 0; t < kNaPairs; ++t)
          if (t == q) acc[t] += se * b;
      }
    }
  }
  block_sum<kNaPairs>(acc, red);
  if (threadIdx.x == 0) {
    double* o = scratch + ((long)cell * gridDim.x + blockIdx.x) * kNaPairs;
#pragma unroll
    for (int t = 0; t < kNaPairs; ++t) o[t] = acc[t];  // written in full, so no clearing is needed
  }
}

__global__ void k_na_reduce(const double* __restrict__ scratch, int nblk, int m, double invN,
                            double* __restrict__ C) {
  const int cell = blockIdx.x;
  const int npair = m * (m + 1) / 2;
  for (int t = threadIdx.x; t < npair; t += blockDim.x) {
    double sum = 0.0;
    for (int b = 0; b < nblk; ++b) sum += scratch[((long)cell * nblk + b) * kNaPairs + t];
    int I = 0, rem = t;
    while (rem >= m - I) {
      rem -= m - I;
      ++I;
    }
    const int J = I + rem;
    C[((long)cell * m + I) * m + J] = sum * invN;
    C[((long)cell * m + J) * m + I] = sum * invN;
  }
}

// Device (or managed) memory at all, whichever device it belongs to.
bool on_device(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

// Device memory of device `dev`: a pointer into another GPU's memory would make the kernels read and write
// that GPU over the interconnect (or fault without peer access). Managed memory is reachable from every device.
bool on_device_of(const void* p, int dev) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeManaged || (at.type == cudaMemoryTypeDevice && at.device == dev);
}

}  // namespace
}  // namespace nlf

using namespace nlf;

extern "C" NLF_API int nlf_bilinear_noalloc(int nx, int ny, int nz, double E, double nu, int ncell,
                                            const double* s, const double* Es, int m, const double* u,
                                            double* C, void* stream) {
  if (nx < 1 || ny < 1 || nz < 1 || !(E > 0) || !(nu > -1.0) || !(nu < 0.5) || !s || !Es || !u || !C) {
    set_error("nlf_bilinear_noalloc: bad arguments");
    return NLF_EBADARG;
  }
  if (ncell < 1 || ncell > kNaCells || m < 1 || m > kNaCases) {
    set_error("nlf_bilinear_noalloc: at most %d cells and %d load cases per call (got %d cells, %d cases); "
              "split the batch or use nlf_bilinear", kNaCells, kNaCases, ncell, m);
    return NLF_EBADARG;
  }
  if (on_device(Es)) {
    set_error("nlf_bilinear_noalloc: Es is read on the host and must be a host array (m, 6)");
    return NLF_EBADARG;
  }
  int dev = 0;
  NLF_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNaMaxDevices) {
    set_error("nlf_bilinear_noalloc: device ordinal %d out of range", dev);
    return NLF_EBADARG;
  }
  if (!on_device_of(s, dev) || !on_device_of(u, dev) || !on_device_of(C, dev)) {
    set_error("nlf_bilinear_noalloc: s, u and C must be device pointers of the current device %d "
              "(it copies nothing; use nlf_bilinear for host arrays)", dev);
    return NLF_EBADARG;
  }
  double* scratch = g_na_addr[dev].load(std::memory_order_acquire);
  if (!scratch) {  // first call on this device: look up the scratch array's device address
    void* p = nullptr;
    NLF_CUDA_TRY(cudaGetSymbolAddress(&p, g_na_scratch));
    scratch = static_cast<double*>(p);
    g_na_addr[dev].store(scratch, std::memory_order_release);
  }
  NaArgs a;
  std::memset(&a, 0, sizeof(a));
  const double lam = E * nu / ((1 + nu) * (1 - 2 * nu)), mu = E / (2 * (1 + nu));
  a.lam = lam;
  a.mu = mu;
  a.m = m;
  a.n0 = nx;
  a.n1 = ny;
  a.n2 = nz;
  double D[6][6] = {};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) D[i][j] = lam;
  for (int i = 0; i < 3; ++i) D[i][i] = lam + 2 * mu;
  for (int i = 3; i < 6; ++i) D[i][i] = mu;
  for (int i = 0; i < m * 6; ++i) a.Es[i] = Es[i];
  for (int I = 0; I < m; ++I)
    for (int J = 0; J < m; ++J) {
      double v = 0.0;
      for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) v += Es[I * 6 + i] * D[i][j] * Es[J * 6 + j];
      a.EDE[I * m + J] = v;
    }
  cudaStream_t st = (cudaStream_t)stream;
  const long N = (long)nx * ny * nz;
  k_na_partials<<<dim3(kNaBlocks, ncell), kNaThreads, 0, st>>>(a, s, u, scratch);
  NLF_CHECK_LAUNCH();
  k_na_reduce<<<ncell, 32, 0, st>>>(scratch, kNaBlocks, m, 1.0 / (double)N, C);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}
