// Handle, batched PCG drivers and the C ABI of the small-strain homogenization path (nlfiber/linear.py).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <array>
#include <map>
#include <mutex>
#include <unordered_map>
#include <vector>
#include "nlf_vec.cuh"
#include "nlf_prof.cuh"

namespace nlf {

// ---- errors ----------------------------------------------------------------------------------------------------
static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

cudaError_t raise_dyn_smem(const void* func, int bytes) {
  static std::mutex mu;
  static std::unordered_map<const void*, int> cur;
  std::lock_guard<std::mutex> lock(mu);
  int& c = cur[func];
  if (bytes <= c) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) c = bytes;
  return e;
}

int DevBuf::reserve(size_t n) {
  if (n <= bytes) return NLF_OK;
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
  const size_t want = n + n / 8;  // grow with slack
  cudaError_t e = cudaMalloc(&ptr, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    ptr = nullptr;
    set_error("workspace: cudaMalloc(%zu B) failed: %s", want, cudaGetErrorString(e));
    return NLF_ECUDA;
  }
  bytes = want;
  return NLF_OK;
}

void DevBuf::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
}

// Bump allocator over a workspace; a first pass with base == nullptr measures the size.
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

static bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// ---- host element matrices (nlfiber/linear.py:21-77,108-112) ----------------------------------------------------
static void element_matrices(LinearHandle& h) {
  const double g1[2] = {0.5 - 1.0 / (2.0 * std::sqrt(3.0)), 0.5 + 1.0 / (2.0 * std::sqrt(3.0))};
  double gp[8][3], dN[8][8][3];
  for (int g = 0; g < 8; ++g) {
    gp[g][0] = g1[g & 1];
    gp[g][1] = g1[(g >> 1) & 1];
    gp[g][2] = g1[(g >> 2) & 1];
  }
  for (int g = 0; g < 8; ++g)
    for (int a = 0; a < 8; ++a) {
      const int i = a & 1, j = (a >> 1) & 1, k = (a >> 2) & 1;
      const double x = gp[g][0], y = gp[g][1], z = gp[g][2];
      const double fx = i ? x : 1 - x, fy = j ? y : 1 - y, fz = k ? z : 1 - z;
      const double sx = i ? 1 : -1, sy = j ? 1 : -1, sz = k ? 1 : -1;
      dN[g][a][0] = sx * fy * fz;
      dN[g][a][1] = fx * sy * fz;
      dN[g][a][2] = fx * fy * sz;
    }
  double D[6][6] = {};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) D[i][j] = h.lam;
  for (int i = 0; i < 3; ++i) D[i][i] = h.lam + 2 * h.mu;
  for (int i = 3; i < 6; ++i) D[i][i] = h.mu;
  std::memcpy(h.Dm, D, sizeof(D));
  std::memset(h.Ke, 0, sizeof(h.Ke));
  std::memset(h.Gm, 0, sizeof(h.Gm));
  for (int g = 0; g < 8; ++g) {
    double B[6][24] = {};
    for (int a = 0; a < 8; ++a) {
      const double dx = dN[g][a][0], dy = dN[g][a][1], dz = dN[g][a][2];
      const int c = 3 * a;
      B[0][c] = dx;
      B[1][c + 1] = dy;
      B[2][c + 2] = dz;
      B[3][c + 1] = dz;
      B[3][c + 2] = dy;
      B[4][c + 0] = dz;
      B[4][c + 2] = dx;
      B[5][c + 0] = dy;
      B[5][c + 1] = dx;
    }
    double DB[6][24] = {};
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 24; ++j)
        for (int k = 0; k < 6; ++k) DB[i][j] += D[i][k] * B[k][j];
    for (int i = 0; i < 24; ++i)
      for (int j = 0; j < 24; ++j)
        for (int k = 0; k < 6; ++k) h.Ke[i][j] += B[k][i] * DB[k][j] / 8.0;
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 24; ++j) h.Gm[i][j] += DB[i][j] / 8.0;
  }
  // 27-point stencil blocks of the unit-stiffness operator: W_d = sum_{a,b: off_a - off_b = d} Ke_ab
  auto stencil = [](const double (&K)[24][24], double (&W27)[27][9]) {
    std::memset(W27, 0, sizeof(W27));
    for (int a = 0; a < 8; ++a)
      for (int b = 0; b < 8; ++b) {
        const int dx = (a & 1) - (b & 1), dy = ((a >> 1) & 1) - ((b >> 1) & 1), dz = (a >> 2) - (b >> 2);
        double* W = W27[(dx + 1) * 9 + (dy + 1) * 3 + (dz + 1)];
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) W[r * 3 + c] += K[3 * a + r][3 * b + c];
      }
  };
  stencil(h.Ke, h.W27);
  // the scaled preconditioner's reference medium: the same element with Poisson ratio h.scaled_ref_nu
  {
    const double nu0 = h.scaled_ref_nu, lam0 = h.E * nu0 / ((1.0 + nu0) * (1.0 - 2.0 * nu0)),
                 mu0 = h.E / (2.0 * (1.0 + nu0));
    double D0[6][6] = {}, K0[24][24] = {};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) D0[i][j] = lam0;
    for (int i = 0; i < 3; ++i) D0[i][i] = lam0 + 2 * mu0;
    for (int i = 3; i < 6; ++i) D0[i][i] = mu0;
    for (int g = 0; g < 8; ++g) {
      double B[6][24] = {};
      for (int a = 0; a < 8; ++a) {
        const double dx = dN[g][a][0], dy = dN[g][a][1], dz = dN[g][a][2];
        const int c = 3 * a;
        B[0][c] = dx;
        B[1][c + 1] = dy;
        B[2][c + 2] = dz;
        B[3][c + 1] = dz;
        B[3][c + 2] = dy;
        B[4][c + 0] = dz;
        B[4][c + 2] = dx;
        B[5][c + 0] = dy;
        B[5][c + 1] = dx;
      }
      for (int i = 0; i < 24; ++i)
        for (int j = 0; j < 24; ++j)
          for (int k = 0; k < 6; ++k)
            for (int l = 0; l < 6; ++l) K0[i][j] += B[k][i] * D0[k][l] * B[l][j] / 8.0;
    }
    stencil(K0, h.W27s);
  }
}

int rebuild_scaled_kinv(LinearHandle& h, double nu) {
  if (!(nu > -1.0) || !(nu < 0.5)) {
    set_error("scaled preconditioner: reference Poisson ratio %g outside (-1, 0.5)", nu);
    return NLF_EBADARG;
  }
  h.scaled_ref_nu = nu;
  element_matrices(h);
  return kinv_tables(h, h.W27s, h.t64s.kinv, h.t32s.kinv);
}

// ---- PCG ---------------------------------------------------------------------------------------------------------
struct PcgCtl {
  double tol;
  int maxit;
  int check_every;
  int scale_x0;
  double energy_tol;  // > 0: energy stopping rule (needs ede)
  Ede ede;
  int per_case = 0;   // > 0: per-case stopping with this probation (fused FP64 iterations only)
};

template <typename T>
struct PcgSet {
  int ncell = 0, m = 0, nvec = 0;
  T *x = nullptr, *r = nullptr, *p = nullptr, *Ap = nullptr, *z = nullptr;
  cplx<T>* spec = nullptr;
  const T* s = nullptr;
  const T* w = nullptr;
  VecState* vs = nullptr;
  CellState* cs = nullptr;
  double *part_ap = nullptr, *part_pc = nullptr, *part_st = nullptr, *part_b = nullptr;
  double* ring = nullptr;  // [nvec][kEnergyWindow]
  int* d_count = nullptr;
};

struct Pinned {
  int* count = nullptr;
  Pinned() { cudaMallocHost(&count, sizeof(int)); }
  ~Pinned() {
    if (count) cudaFreeHost(count);
  }
};

template <typename T>
static void carve_pcg(Arena& A, const LinearHandle& h, PcgSet<T>& P, int ncell, int m) {
  P.ncell = ncell;
  P.m = m;
  P.nvec = ncell * m;
  const size_t V = (size_t)P.nvec * 3 * h.g.N;
  P.x = A.take<T>(V);
  P.r = A.take<T>(V);
  P.p = A.take<T>(V);
  P.Ap = A.take<T>(V);
  P.z = A.take<T>(V);
  P.spec = A.take<cplx<T>>((size_t)P.nvec * 3 * h.g.NS);
  P.vs = A.take<VecState>(P.nvec);
  P.cs = A.take<CellState>(ncell);
  // apply partials: tiles * x-chunks <= kApplyMaxBlocks blocks per vec
  P.part_ap = A.take<double>((size_t)P.nvec * kApplyMaxBlocks * 4);
  P.part_pc = A.take<double>((size_t)P.nvec * 3 * h.g.n0 * 4);
  P.part_b = A.take<double>((size_t)P.nvec * h.g.n1 * h.g.n2h);  // pass-B chunks <= n2h per ky
  P.part_st = A.take<double>((size_t)P.nvec * 3 * kStatsBlocks * 2);
  P.ring = A.take<double>((size_t)P.nvec * kEnergyWindow);
  P.d_count = A.take<int>(4);
}

template <typename T>
static int pcg_iteration(const LinearHandle& h, PcgSet<T>& P, const PcgCtl& ctl, cudaStream_t st) {
  const long N = h.g.N;
  int nblk = 0;
  NLF_TRY(launch_mark(P.cs, P.ncell, st));
  NLF_TRY(launch_apply<T>(h, P.s, P.m, P.nvec, P.p, P.Ap, P.cs, P.part_ap, &nblk, st));
  NLF_TRY(launch_fin_apply(P.nvec, P.m, P.part_ap, nblk, N, P.vs, P.cs, 0, st));
  double* partA = P.part_pc;
  int nchunk = 0;
  if constexpr (sizeof(T) == 8) {
    if (precond_fuses_px(h)) {
      // r update, (r, r) and (r, z) ride on passes A and B; the control sets beta; pass C updates x and p
      NLF_TRY(launch_precond_pcg_ab(h, P.nvec, P.m, P.r, P.Ap, P.vs, P.spec, P.w, P.cs, partA, P.part_b, &nchunk, st));
      NLF_TRY(launch_fin_pc_fused(P.ncell, P.m, h.g.n0, h.g.n1, N, partA, P.part_b, nullptr, nchunk, P.vs, P.cs,
                                  ctl.tol, ctl.maxit, P.ring, ctl.energy_tol, ctl.per_case, st));
      return launch_precond_pcg_cpx(h, P.nvec, P.m, P.spec, P.w, P.vs, P.cs, P.x, P.p, st);
    }
  }
  // r update, (r, r), (r, z) and the sums ride on the FFT passes; x += alpha p rides on the p update
  double* partC = P.part_pc + (size_t)P.nvec * 3 * h.g.n0 * 2;
  NLF_TRY(launch_precond_pcg<T>(h, P.nvec, P.m, P.r, P.Ap, P.vs, P.z, P.spec, P.w, P.cs, partA, P.part_b, partC,
                                &nchunk, st));
  NLF_TRY(launch_fin_pc_fused(P.ncell, P.m, h.g.n0, h.g.n1, N, partA, P.part_b, partC, nchunk, P.vs, P.cs, ctl.tol,
                              ctl.maxit, P.ring, ctl.energy_tol, 0, st));
  NLF_TRY(launch_px<T>(N, P.nvec, P.m, P.x, P.p, P.z, P.vs, P.cs, st));
  return NLF_OK;
}

static int count_active(const CellState* cs, int ncell, int* d_count, int* h_count, cudaStream_t st) {
  NLF_TRY(launch_count_active(cs, ncell, d_count, st));
  NLF_CUDA_TRY(cudaMemcpyAsync(h_count, d_count, sizeof(int), cudaMemcpyDeviceToHost, st));
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  return *h_count;
}

// The first cell..cell+count-1 of a PCG set as a set of its own (same partial-sum buffers).
template <typename T>
static PcgSet<T> pcg_view(const PcgSet<T>& P, const LinearHandle& h, int cell, int count) {
  PcgSet<T> v = P;
  const size_t V = (size_t)P.m * 3 * h.g.N * cell;
  v.ncell = count;
  v.nvec = count * P.m;
  v.x += V;
  v.r += V;
  v.p += V;
  v.Ap += V;
  v.z += V;
  v.spec += (size_t)P.m * 3 * h.g.NS * cell;
  if (v.s) v.s += (size_t)h.g.N * cell;
  if (v.w) v.w += (size_t)h.g.N * cell;
  v.vs += (size_t)P.m * cell;
  v.cs += cell;
  if (v.ring) v.ring += (size_t)P.m * kEnergyWindow * cell;
  return v;
}

// Start of the lock-step PCG (nlfiber/linear.py:173-183): x0 = proj(x) or 0, r = b - proj(A x0), z = M r,
// p = proj(z), the first (r, z) and the per-cell active flags. b: [nvec][3][N] in Tb, already mean-free.
template <typename T, typename Tb>
static int pcg_init(const LinearHandle& h, PcgSet<T>& P, const Tb* b, bool x_given, const PcgCtl& ctl,
                    const int* mask, cudaStream_t st) {
  const long N = h.g.N;
  NLF_TRY(launch_cs_init(P.cs, P.ncell, mask, st));
  NLF_TRY(launch_stats<Tb>(h, P.nvec, P.m, b, P.cs, P.part_st, P.vs, 1, st));
  if (x_given) {
    NLF_TRY(launch_stats<T>(h, P.nvec, P.m, P.x, P.cs, P.part_st, P.vs, 0, st));
    NLF_TRY(launch_sub_mean<T>(h, P.nvec, P.m, P.x, P.vs, P.cs, st));
  } else {
    NLF_CUDA_TRY(cudaMemsetAsync(P.x, 0, (size_t)P.nvec * 3 * N * sizeof(T), st));
  }
  int nblk = 0;
  NLF_TRY(launch_apply<T>(h, P.s, P.m, P.nvec, P.x, P.Ap, P.cs, P.part_ap, &nblk, st));
  NLF_TRY(launch_fin_apply(P.nvec, P.m, P.part_ap, nblk, N, P.vs, P.cs, 1, st));
  if (x_given && ctl.scale_x0) NLF_TRY((launch_x0_scale<Tb, T>(h, P.nvec, P.m, b, P.x, P.Ap, P.cs, P.part_st, P.vs, st)));
  if (ctl.energy_tol > 0.0)
    NLF_TRY((launch_energy_init<Tb, T>(h, P.ncell, P.m, P.s, ctl.ede, b, P.x, P.Ap, x_given, P.cs, P.part_st, P.vs,
                                       st)));
  NLF_TRY((launch_r_init<Tb, T>(N, P.nvec, P.m, P.r, b, P.Ap, P.vs, P.cs, st)));
  NLF_TRY(launch_precond<T>(h, P.nvec, P.m, P.r, P.z, P.spec, P.w, P.cs, P.part_pc, st));
  NLF_TRY(launch_fin_pc(P.ncell, P.m, h.g.n0, N, P.part_pc, P.vs, P.cs, ctl.tol, ctl.maxit, 1, st));
  NLF_TRY(launch_p<T>(N, P.nvec, P.m, P.p, P.z, P.vs, P.cs, 1, st));
  return NLF_OK;
}

// `k` PCG iterations, either launched one by one on `st` or, with graphs, captured once into `exec` on the
// handle's own stream and replayed there, ordered after and before the work on `st` by events. The set's
// pointers must stay the same while `exec` lives.
struct IterGraph {
  cudaGraphExec_t exec = nullptr;
  int k = 0;
  ~IterGraph() {
    if (exec) cudaGraphExecDestroy(exec);
  }
};

static int graph_stream(LinearHandle& h) {
  if (h.gst) return NLF_OK;
  NLF_CUDA_TRY(cudaStreamCreateWithFlags(&h.gst, cudaStreamNonBlocking));
  NLF_CUDA_TRY(cudaEventCreateWithFlags(&h.gev[0], cudaEventDisableTiming));
  NLF_CUDA_TRY(cudaEventCreateWithFlags(&h.gev[1], cudaEventDisableTiming));
  return NLF_OK;
}

template <typename T>
static int run_iterations(LinearHandle& h, PcgSet<T>& P, const PcgCtl& ctl, int k, bool graphs, IterGraph& G,
                          cudaStream_t st) {
  if (!graphs || prof_on()) {
    for (int i = 0; i < k; ++i) NLF_TRY(pcg_iteration<T>(h, P, ctl, st));
    return NLF_OK;
  }
  NLF_TRY(graph_stream(h));
  if (!G.exec || G.k != k) {
    if (G.exec) {
      cudaGraphExecDestroy(G.exec);
      G.exec = nullptr;
    }
    cudaGraph_t graph = nullptr;
    NLF_CUDA_TRY(cudaStreamBeginCapture(h.gst, cudaStreamCaptureModeThreadLocal));
    int rc = NLF_OK;
    for (int i = 0; i < k && rc == NLF_OK; ++i) rc = pcg_iteration<T>(h, P, ctl, h.gst);
    const cudaError_t e = cudaStreamEndCapture(h.gst, &graph);
    if (rc != NLF_OK || e != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      if (rc != NLF_OK) return rc;
      NLF_CUDA_TRY(e);
    }
    const cudaError_t ei = cudaGraphInstantiate(&G.exec, graph, 0);
    cudaGraphDestroy(graph);
    NLF_CUDA_TRY(ei);
    G.k = k;
  }
  NLF_CUDA_TRY(cudaEventRecord(h.gev[0], st));
  NLF_CUDA_TRY(cudaStreamWaitEvent(h.gst, h.gev[0], 0));
  NLF_CUDA_TRY(cudaGraphLaunch(G.exec, h.gst));
  NLF_CUDA_TRY(cudaEventRecord(h.gev[1], h.gst));
  NLF_CUDA_TRY(cudaStreamWaitEvent(st, h.gev[1], 0));
  return NLF_OK;
}

// x <- proj(x) for the vectors of a set whose iterations ran the fused pass C (which leaves z unprojected)
template <typename T>
static int project_x(const LinearHandle& h, PcgSet<T>& P, cudaStream_t st) {
  if constexpr (sizeof(T) == 8) {
    if (precond_fuses_px(h)) {
      NLF_TRY(launch_stats<T>(h, P.nvec, P.m, P.x, nullptr, P.part_st, P.vs, 0, st));
      NLF_TRY(launch_sub_mean<T>(h, P.nvec, P.m, P.x, P.vs, nullptr, st));
    }
  }
  return NLF_OK;
}

// Lock-step PCG for K x = b on the mean-free subspace (nlfiber/linear.py:173-203), batched over cells.
// b: [nvec][3][N] in Tb, already mean-free. x: initial guess if x_given (projected here), else zero.
// mask: device per-cell flags of the cells to solve (nullptr: all).
template <typename T, typename Tb>
static int pcg(LinearHandle& h, PcgSet<T>& P, const Tb* b, bool x_given, const PcgCtl& ctl, const int* mask,
               int* h_count, bool graphs, cudaStream_t st) {
  NLF_TRY((pcg_init<T, Tb>(h, P, b, x_given, ctl, mask, st)));
  int act = count_active(P.cs, P.ncell, P.d_count, h_count, st);
  if (act < 0) return act;
  int done = 0;
  const int every = ctl.check_every > 0 ? ctl.check_every : 1;
  IterGraph G;
  while (act > 0 && done < ctl.maxit) {
    NLF_TRY(run_iterations<T>(h, P, ctl, every, graphs, G, st));
    done += every;
    act = count_active(P.cs, P.ncell, P.d_count, h_count, st);
    if (act < 0) return act;
  }
  return project_x<T>(h, P, st);
}

static bool poison_workspace() {
  static const bool on = [] {
    const char* e = std::getenv("NLF_POISON_WORKSPACE");
    return e && e[0] == '1';
  }();
  return on;
}

// ---- a whole solve on staged device inputs ---------------------------------------------------------------------
struct SolveIn {
  int ncell, m;
  const double* s64;  // [ncell][N]
  const double* b64;  // [ncell][m][3][N], mean-free (nullptr: build from fe = Es G)
  const double* fe;   // device (m, 24) when b64 == nullptr
  const double* x0;   // AoS (ncell, m, N, 3) device FP64 or nullptr
  bool has_ede;       // E_I D E_I known (a solve from strains, m <= 6): the energy stopping rule is available
  Ede ede;
};

static nlf_solve_opts resolve_opts(const LinearHandle& h, const nlf_solve_opts* o) {
  nlf_solve_opts r;
  nlf_default_opts(&r);
  if (o) r = *o;
  if (r.tol < 0) r.tol = h.tol;
  if (r.maxit < 0) r.maxit = h.maxit;
  if (r.check_every < 1) r.check_every = 1;
  if (r.inner_maxit < 1) r.inner_maxit = 1;
  if (r.max_sweeps < 1) r.max_sweeps = 1;
  if (r.slots < 0) r.slots = 0;
  return r;
}

// Status of one finished cell from its cases' VecState: breakdown if a residual is not finite, not converged
// if a case still has ||r|| > tol ||b|| (it ran out of iterations), else ok.
static int cell_status(const VecState* v, int m, double tol) {
  int st = NLF_OK;
  for (int I = 0; I < m; ++I) {
    if (!std::isfinite(v[I].rr)) return NLF_BREAKDOWN;
    if (std::sqrt(v[I].rr) > tol * v[I].bn) st = NLF_NOT_CONVERGED;
  }
  return st;
}
static int worse(int a, int b) { return (a == NLF_BREAKDOWN || b == NLF_BREAKDOWN) ? NLF_BREAKDOWN : std::max(a, b); }

struct PinnedBuf {
  void* p = nullptr;
  explicit PinnedBuf(size_t n) {
    if (cudaMallocHost(&p, n) != cudaSuccess) p = nullptr;
  }
  ~PinnedBuf() {
    if (p) cudaFreeHost(p);
  }
};

// FP64 PCG of ncell cells through `o.slots` slots: each slot runs the lock-step PCG of one cell at a time
// (the same iteration as the all-cells batch, so each cell's result is the same), and at every poll the cells
// that stopped are copied out and their slots restarted on the next queued cells.
static int solve_slots(LinearHandle& h, const SolveIn& in, const nlf_solve_opts& o, double* xout, int* iters_h,
                       cudaStream_t st) {
  const int ncell = in.ncell, m = in.m, S = o.slots;
  const long N = h.g.N;
  const size_t Vc = (size_t)m * 3 * N;  // the vectors of one cell
  const bool scaled = o.precond == NLF_PC_FFT_SCALED;
  PcgSet<double> P;
  double *s_sl = nullptr, *w_sl = nullptr, *b_sl = nullptr;
  for (int pass = 0; pass < 2; ++pass) {
    Arena A(pass ? h.ws.ptr : nullptr);
    s_sl = A.take<double>((size_t)S * N);
    w_sl = scaled ? A.take<double>((size_t)S * N) : nullptr;
    b_sl = A.take<double>((size_t)S * Vc);
    carve_pcg<double>(A, h, P, S, m);
    if (pass == 0) {
      NLF_TRY(h.ws.reserve(A.off));
    } else if (poison_workspace()) {
      NLF_CUDA_TRY(cudaMemsetAsync(h.ws.ptr, 0xFF, A.off, st));
    }
  }
  P.s = s_sl;
  P.w = w_sl;
  // Host snapshots of the slots' state, kLook chunks ahead: the host reads the snapshot taken after chunk j while
  // chunks up to j + kLook are already queued, so the GPU does not wait for a busy host between chunks. A slot
  // refilled while reading snapshot j still shows its previous cell in the snapshots up to j + kLook (copied
  // before the refill was queued), so it is read again from snapshot j + kLook + 1 on. A stopped cell's slot
  // therefore idles for kLook extra chunks, which costs no GPU time: the kernels skip inactive cells.
  constexpr int kLook = 3, kRing = kLook + 1;
  const size_t snap = S * sizeof(CellState) + (size_t)S * m * sizeof(VecState);
  PinnedBuf pin(kRing * snap);
  if (!pin.p) {
    set_error("cudaMallocHost failed");
    return NLF_ECUDA;
  }
  CellState* csb[kRing];
  VecState* vsb[kRing];
  for (int k = 0; k < kRing; ++k) {
    csb[k] = reinterpret_cast<CellState*>(static_cast<char*>(pin.p) + k * snap);
    vsb[k] = reinterpret_cast<VecState*>(csb[k] + S);
  }
  struct Events {
    cudaEvent_t e[kRing] = {};
    ~Events() {
      for (cudaEvent_t x : e)
        if (x) cudaEventDestroy(x);
    }
  } ev;
  for (int k = 0; k < kRing; ++k) NLF_CUDA_TRY(cudaEventCreateWithFlags(&ev.e[k], cudaEventDisableTiming));
  NLF_CUDA_TRY(cudaMemsetAsync(P.cs, 0, S * sizeof(CellState), st));  // every slot empty and inactive
  const PcgCtl ctl{o.tol, o.maxit, o.check_every, o.scale_x0, in.has_ede ? o.energy_tol : 0.0, in.ede,
                   precond_fuses_px(h) ? o.per_case : 0};
  std::vector<int> slot_cell(S, -1);
  std::vector<long> valid_from(S, 0);  // first snapshot index that shows the slot's current cell
  int next = 0;
  auto start = [&](int sl) -> int {
    const int c = next++;
    slot_cell[sl] = c;
    double* ss = s_sl + (size_t)sl * N;
    double* bs = b_sl + (size_t)sl * Vc;
    PcgSet<double> v = pcg_view(P, h, sl, 1);
    NLF_CUDA_TRY(cudaMemcpyAsync(ss, in.s64 + (size_t)c * N, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (scaled) NLF_TRY(launch_node_scaling(h, 1, ss, nullptr, w_sl + (size_t)sl * N, nullptr, st));
    // b = -proj(load) (nlfiber/linear.py:176,206)
    if (in.b64) {
      NLF_CUDA_TRY(cudaMemcpyAsync(bs, in.b64 + (size_t)c * Vc, Vc * sizeof(double), cudaMemcpyDeviceToDevice, st));
    } else {
      NLF_TRY(launch_load(h, ss, in.fe, m, 1, bs, -1.0, st));
    }
    NLF_TRY(launch_cs_init(v.cs, 1, nullptr, st));
    NLF_TRY(launch_stats<double>(h, m, m, bs, v.cs, P.part_st, v.vs, 0, st));
    NLF_TRY(launch_sub_mean<double>(h, m, m, bs, v.vs, v.cs, st));
    const bool xg = in.x0 != nullptr;
    if (xg) NLF_TRY((launch_aos_to_soa<double, double>(N, m, in.x0 + (size_t)c * Vc, v.x, 1.0, st)));
    return pcg_init<double, double>(h, v, bs, xg, ctl, nullptr, st);
  };
  auto take_snapshot = [&](long k) -> int {
    const int b = (int)(k % kRing);
    NLF_CUDA_TRY(cudaMemcpyAsync(csb[b], P.cs, S * sizeof(CellState), cudaMemcpyDeviceToHost, st));
    NLF_CUDA_TRY(cudaMemcpyAsync(vsb[b], P.vs, (size_t)S * m * sizeof(VecState), cudaMemcpyDeviceToHost, st));
    NLF_CUDA_TRY(cudaEventRecord(ev.e[b], st));
    return NLF_OK;
  };
  for (int sl = 0; sl < S && next < ncell; ++sl) NLF_TRY(start(sl));
  const int every = ctl.check_every > 0 ? ctl.check_every : 1;
  IterGraph G;
  int status = NLF_OK;
  NLF_TRY(take_snapshot(0));  // the state after the starts (cells may stop before their first iteration)
  for (long k = 1; k < kLook; ++k) {
    NLF_TRY(run_iterations<double>(h, P, ctl, every, o.use_graphs != 0, G, st));
    NLF_TRY(take_snapshot(k));
  }
  for (long j = 0;; ++j) {
    NLF_TRY(run_iterations<double>(h, P, ctl, every, o.use_graphs != 0, G, st));
    NLF_TRY(take_snapshot(j + kLook));
    NLF_CUDA_TRY(cudaEventSynchronize(ev.e[j % kRing]));
    const CellState* cs_h = csb[j % kRing];
    const VecState* vs_h = vsb[j % kRing];
    int nact = 0;
    for (int sl = 0; sl < S; ++sl) {
      const int c = slot_cell[sl];
      if (c < 0) continue;
      if (valid_from[sl] > j || cs_h[sl].active) {
        ++nact;
        continue;
      }
      iters_h[c] = cs_h[sl].it;
      status = worse(status, cell_status(vs_h + (size_t)sl * m, m, o.tol));
      PcgSet<double> v = pcg_view(P, h, sl, 1);
      NLF_TRY(project_x<double>(h, v, st));
      NLF_CUDA_TRY(cudaMemcpyAsync(xout + (size_t)c * Vc, P.x + (size_t)sl * Vc, Vc * sizeof(double),
                                   cudaMemcpyDeviceToDevice, st));
      slot_cell[sl] = -1;
      if (next < ncell) {
        NLF_TRY(start(sl));
        valid_from[sl] = j + kLook + 1;
        ++nact;
      }
    }
    if (nact == 0) {
      NLF_CUDA_TRY(cudaEventSynchronize(ev.e[(j + kLook) % kRing]));  // the last snapshot's copy
      break;
    }
  }
  return status;
}

// Runs the solve; writes the FP64 corrector (SoA) to `xout` ([ncell][m][3][N]) and iterations to iters_h.
static int solve_core(LinearHandle& h, const SolveIn& in, const nlf_solve_opts& o, double* xout, int* iters_h,
                      cudaStream_t st) {
  const int ncell = in.ncell, m = in.m, nvec = ncell * m;
  const long N = h.g.N;
  const size_t V = (size_t)nvec * 3 * N;
  const bool mixed = o.precision == NLF_PREC_MIXED;
  const bool scaled = o.precond == NLF_PC_FFT_SCALED;
  // slot refill holds only `slots` cells of PCG state: dispatch before sizing the all-cells workspace
  if (!mixed && o.slots > 0 && o.slots < ncell) return solve_slots(h, in, o, xout, iters_h, st);
  Pinned pin;
  if (!pin.count) {
    set_error("cudaMallocHost failed");
    return NLF_ECUDA;
  }
  std::vector<int> it_total(ncell, 0);
  std::vector<CellState> csh(ncell);
  for (int pass = 0; pass < 2; ++pass) {
    Arena A(pass ? h.ws.ptr : nullptr);
    double* b64 = A.take<double>(V);
    double* w64 = scaled && !mixed ? A.take<double>((size_t)ncell * N) : nullptr;
    float* s32 = mixed ? A.take<float>((size_t)ncell * N) : nullptr;
    float* w32 = mixed && scaled ? A.take<float>((size_t)ncell * N) : nullptr;
    PcgSet<double> P64;
    PcgSet<float> P32;
    double* ax64 = nullptr;
    VecState* vs_o = nullptr;
    CellState* cs_o = nullptr;
    double* part_ap = nullptr;
    double* part_st = nullptr;
    int* mask = nullptr;
    if (!mixed) {
      carve_pcg<double>(A, h, P64, ncell, m);
    } else {
      carve_pcg<float>(A, h, P32, ncell, m);
      ax64 = A.take<double>(V);
      vs_o = A.take<VecState>(nvec);
      cs_o = A.take<CellState>(ncell);
      part_ap = A.take<double>((size_t)nvec * kApplyMaxBlocks * 4);
      part_st = A.take<double>((size_t)nvec * 3 * kStatsBlocks * 2);
      mask = A.take<int>(ncell);
    }
    if (pass == 0) {
      NLF_TRY(h.ws.reserve(A.off));
      continue;
    }
    // NLF_POISON_WORKSPACE=1 fills the workspace with NaN first, so that any read of a value the solve has
    // not written shows up in its result (a debugging aid used by the tests).
    if (poison_workspace()) NLF_CUDA_TRY(cudaMemsetAsync(h.ws.ptr, 0xFF, A.off, st));
    // right-hand side b = -proj(load) (nlfiber/linear.py:176,206)
    if (in.b64) {
      NLF_CUDA_TRY(cudaMemcpyAsync(b64, in.b64, V * sizeof(double), cudaMemcpyDeviceToDevice, st));
    } else {
      NLF_TRY(launch_load(h, in.s64, in.fe, m, ncell, b64, -1.0, st));
    }
    {
      // project b (all cells active for this)
      CellState* cs = mixed ? cs_o : P64.cs;
      VecState* vs = mixed ? vs_o : P64.vs;
      double* ps = mixed ? part_st : P64.part_st;
      NLF_TRY(launch_cs_init(cs, ncell, nullptr, st));
      NLF_TRY(launch_stats<double>(h, nvec, m, b64, cs, ps, vs, 0, st));
      NLF_TRY(launch_sub_mean<double>(h, nvec, m, b64, vs, cs, st));
    }
    if (!mixed) {
      P64.s = in.s64;
      P64.w = w64;
      if (scaled) NLF_TRY(launch_node_scaling(h, ncell, in.s64, nullptr, w64, nullptr, st));
      const bool xg = in.x0 != nullptr;
      if (xg) NLF_TRY((launch_aos_to_soa<double, double>(N, nvec, in.x0, P64.x, 1.0, st)));
      PcgCtl ctl{o.tol, o.maxit, o.check_every, o.scale_x0, in.has_ede ? o.energy_tol : 0.0, in.ede,
                 precond_fuses_px(h) ? o.per_case : 0};
      NLF_TRY((pcg<double, double>(h, P64, b64, xg, ctl, nullptr, pin.count, o.use_graphs != 0, st)));
      NLF_CUDA_TRY(cudaMemcpyAsync(xout, P64.x, V * sizeof(double), cudaMemcpyDeviceToDevice, st));
      NLF_CUDA_TRY(cudaMemcpyAsync(csh.data(), P64.cs, ncell * sizeof(CellState), cudaMemcpyDeviceToHost, st));
      NLF_CUDA_TRY(cudaStreamSynchronize(st));
      std::vector<VecState> vsh(nvec);
      NLF_CUDA_TRY(cudaMemcpy(vsh.data(), P64.vs, nvec * sizeof(VecState), cudaMemcpyDeviceToHost));
      int status = NLF_OK;
      for (int c = 0; c < ncell; ++c) {
        iters_h[c] = csh[c].it;
        status = worse(status, cell_status(&vsh[(size_t)c * m], m, o.tol));
      }
      return status;
    }
    // ---- mixed precision: FP32 PCG inside FP64 iterative refinement ----
    NLF_TRY(launch_node_scaling(h, ncell, in.s64, s32, nullptr, w32, st));
    P32.s = s32;
    P32.w = w32;
    double* x64 = xout;
    NLF_TRY(launch_stats<double>(h, nvec, m, b64, cs_o, part_st, vs_o, 1, st));  // bn
    if (in.x0) {
      NLF_TRY((launch_aos_to_soa<double, double>(N, nvec, in.x0, x64, 1.0, st)));
      NLF_TRY(launch_stats<double>(h, nvec, m, x64, cs_o, part_st, vs_o, 0, st));
      NLF_TRY(launch_sub_mean<double>(h, nvec, m, x64, vs_o, cs_o, st));
    } else {
      NLF_CUDA_TRY(cudaMemsetAsync(x64, 0, V * sizeof(double), st));
    }
    std::vector<VecState> vsh(nvec);
    std::vector<int> conv(ncell, 0), maskh(ncell, 0);
    int status = NLF_OK;
    for (int sweep = 0;; ++sweep) {
      // r64 = b - proj(K x) in FP64 (the refinement residual)
      NLF_TRY(launch_cs_init(cs_o, ncell, nullptr, st));
      int nblk = 0;
      NLF_TRY(launch_apply<double>(h, in.s64, m, nvec, x64, ax64, cs_o, part_ap, &nblk, st));
      NLF_TRY(launch_fin_apply(nvec, m, part_ap, nblk, N, vs_o, cs_o, 1, st));
      NLF_TRY((launch_r_init<double, double>(N, nvec, m, ax64, b64, ax64, vs_o, cs_o, st)));
      NLF_TRY(launch_stats<double>(h, nvec, m, ax64, cs_o, part_st, vs_o, 2, st));
      NLF_CUDA_TRY(cudaMemcpyAsync(vsh.data(), vs_o, nvec * sizeof(VecState), cudaMemcpyDeviceToHost, st));
      NLF_CUDA_TRY(cudaStreamSynchronize(st));
      int nact = 0;
      for (int c = 0; c < ncell; ++c) {
        bool ok = true;
        for (int I = 0; I < m; ++I) {
          const VecState& v = vsh[c * m + I];
          if (!std::isfinite(v.rr)) status = NLF_BREAKDOWN;
          if (std::sqrt(v.rr) > o.tol * v.bn) ok = false;
        }
        conv[c] = ok;
        maskh[c] = !ok && it_total[c] < o.maxit && sweep < o.max_sweeps;
        nact += maskh[c];
      }
      if (nact == 0 || status == NLF_BREAKDOWN) break;
      NLF_CUDA_TRY(cudaMemcpyAsync(mask, maskh.data(), ncell * sizeof(int), cudaMemcpyHostToDevice, st));
      NLF_TRY(launch_cs_init(cs_o, ncell, mask, st));
      NLF_TRY(launch_r_to32(N, nvec, m, ax64, P32.z, vs_o, cs_o, st));  // P32.z holds the FP32 rhs for init
      // the FP32 inner solve reads its rhs from a buffer it does not overwrite: use Ap's slot via a copy
      float* rhs32 = reinterpret_cast<float*>(ax64);  // ax64 is free until the next sweep
      NLF_CUDA_TRY(cudaMemcpyAsync(rhs32, P32.z, V * sizeof(float), cudaMemcpyDeviceToDevice, st));
      int cap = o.inner_maxit;
      for (int c = 0; c < ncell; ++c)
        if (maskh[c]) cap = std::min(cap, std::max(1, o.maxit - it_total[c]));
      PcgCtl ctl{o.inner_tol, cap, o.check_every, 0, 0.0, Ede{}};
      NLF_TRY((pcg<float, float>(h, P32, rhs32, false, ctl, mask, pin.count, o.use_graphs != 0, st)));
      NLF_TRY(launch_x_update(N, nvec, m, x64, P32.x, vs_o, cs_o, st));
      NLF_CUDA_TRY(cudaMemcpyAsync(csh.data(), P32.cs, ncell * sizeof(CellState), cudaMemcpyDeviceToHost, st));
      NLF_CUDA_TRY(cudaStreamSynchronize(st));
      for (int c = 0; c < ncell; ++c)
        if (maskh[c]) it_total[c] += csh[c].it;
    }
    for (int c = 0; c < ncell; ++c) {
      iters_h[c] = it_total[c];
      if (!conv[c] && status == NLF_OK) status = NLF_NOT_CONVERGED;
    }
    return status;
  }
  return NLF_OK;
}

}  // namespace nlf

using namespace nlf;

struct nlf_linear {
  LinearHandle h;
};

namespace nlf {
LinearHandle& linear_handle(nlf_linear* h) { return h->h; }
}  // namespace nlf

// ---- staging helpers --------------------------------------------------------------------------------------------
namespace {

// Device view of an input array: the pointer itself when it is device memory, else a copy in `buf`.
struct InView {
  const double* d = nullptr;
};

int stage_in(const double* src, size_t count, DevBuf& buf, size_t buf_off, InView& v, cudaStream_t st) {
  if (!src) {
    v.d = nullptr;
    return NLF_OK;
  }
  if (is_device_ptr(src)) {
    v.d = src;
    return NLF_OK;
  }
  double* dst = reinterpret_cast<double*>((char*)buf.ptr + buf_off);
  NLF_CUDA_TRY(cudaMemcpyAsync(dst, src, count * sizeof(double), cudaMemcpyHostToDevice, st));
  v.d = dst;
  return NLF_OK;
}

int copy_out(double* dst, const double* dsrc, size_t count, cudaStream_t st) {
  NLF_CUDA_TRY(cudaMemcpyAsync(dst, dsrc, count * sizeof(double), is_device_ptr(dst) ? cudaMemcpyDeviceToDevice
                                                                                      : cudaMemcpyDeviceToHost,
                               st));
  return NLF_OK;
}

size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

bool bad_handle(nlf_linear* h) {
  if (!h) {
    set_error("null handle");
    return true;
  }
  return false;
}

void es_to_fe(const LinearHandle& h, const double* Es, int m, std::vector<double>& fe) {
  fe.assign((size_t)m * 24, 0.0);
  for (int I = 0; I < m; ++I)
    for (int j = 0; j < 24; ++j) {
      double a = 0.0;
      for (int i = 0; i < 6; ++i) a += Es[I * 6 + i] * h.Gm[i][j];
      fe[(size_t)I * 24 + j] = a;
    }
}

int host_copy_small(const double* src, size_t count, std::vector<double>& out) {
  out.resize(count);
  if (is_device_ptr(src)) {
    NLF_CUDA_TRY(cudaMemcpy(out.data(), src, count * sizeof(double), cudaMemcpyDeviceToHost));
  } else {
    std::memcpy(out.data(), src, count * sizeof(double));
  }
  return NLF_OK;
}

}  // namespace

extern "C" {

NLF_API const char* nlf_last_error(void) { return g_err; }
NLF_API const char* nlf_version(void) { return "nlfiber-b200 0.1 (sm_100a)"; }

NLF_API void nlf_default_opts(nlf_solve_opts* o) {
  if (!o) return;
  o->precision = NLF_PREC_FP64;
  o->precond = NLF_PC_FFT;
  o->tol = -1.0;
  o->maxit = -1;
  o->inner_tol = 1e-3;
  o->inner_maxit = 200;
  o->max_sweeps = 20;
  o->check_every = 8;
  o->use_graphs = 0;
  o->per_case = 0;
  o->slots = 0;
  o->scale_x0 = 0;
  o->energy_tol = 0.0;
}

NLF_API int nlf_linear_create(nlf_linear** out, int nx, int ny, int nz, double E, double nu, double emin, double p,
                              double tol, int maxit) {
  if (!out || nx < 1 || ny < 1 || nz < 1 || nx > 1024 || ny > 1024 || nz > 1024 || !(E > 0) || !(nu > -1.0) ||
      !(nu < 0.5) || maxit < 0) {
    set_error("nlf_linear_create: bad arguments (shape %d x %d x %d, E %g, nu %g, maxit %d)", nx, ny, nz, E, nu,
              maxit);
    return NLF_EBADARG;
  }
  *out = nullptr;
  nlf_linear* H = new nlf_linear();
  LinearHandle& h = H->h;
  h.g.n0 = nx;
  h.g.n1 = ny;
  h.g.n2 = nz;
  h.g.n2h = nz / 2 + 1;
  h.g.N = (long)nx * ny * nz;
  h.g.NS = (long)nx * ny * h.g.n2h;
  h.E = E;
  h.nu = nu;
  h.emin = emin;
  h.p = p;
  h.tol = tol;
  h.maxit = maxit;
  h.lam = E * nu / ((1 + nu) * (1 - 2 * nu));
  h.mu = E / (2 * (1 + nu));
  element_matrices(h);
  cudaError_t e = cudaGetDevice(&h.dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h.nsm, cudaDevAttrMultiProcessorCount, h.dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h.dev);
  if (e != cudaSuccess) {
    set_error("nlf_linear_create: %s", cudaGetErrorString(e));
    delete H;
    return NLF_ECUDA;
  }
  int st = build_tables(h);
  if (st != NLF_OK) {
    nlf_linear_destroy(H);
    return st;
  }
  *out = H;
  return NLF_OK;
}

NLF_API int nlf_linear_destroy(nlf_linear* H) {
  if (!H) return NLF_OK;
  LinearHandle& h = H->h;
  if (h.gst) cudaStreamDestroy(h.gst);
  for (cudaEvent_t e : h.gev)
    if (e) cudaEventDestroy(e);
  cudaFree(h.t64.kinv);
  cudaFree(h.t32.kinv);
  cudaFree(h.t64s.kinv);
  cudaFree(h.t32s.kinv);
  cudaFree(h.t64.tw);
  cudaFree(h.t32.tw);
  h.ws.release();
  h.io.release();
  h.io2.release();
  h.part.release();
  delete H;
  return NLF_OK;
}

NLF_API int nlf_stiffness_scale(nlf_linear* H, int ncell, const double* rho, double* s, void* stream) {
  if (bad_handle(H) || ncell < 0 || !rho || !s) {
    set_error("nlf_stiffness_scale: bad arguments");
    return NLF_EBADARG;
  }
  LinearHandle& h = H->h;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t cnt = (size_t)ncell * h.g.N;
  NLF_TRY(h.io.reserve(al(cnt * 8) * 2));
  InView r;
  NLF_TRY(stage_in(rho, cnt, h.io, 0, r, st));
  double* sd = is_device_ptr(s) ? s : reinterpret_cast<double*>((char*)h.io.ptr + al(cnt * 8));
  NLF_TRY(launch_stiffness_scale(h, (long)cnt, r.d, sd, st));
  if (sd != s) NLF_TRY(copy_out(s, sd, cnt, st));
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  return NLF_OK;
}

NLF_API int nlf_apply_K_ex(nlf_linear* H, const double* s, int nvec, const double* u, double* y, int precision,
                           void* stream) {
  if (bad_handle(H) || nvec < 1 || !s || !u || !y ||
      (precision != NLF_PREC_FP64 && precision != NLF_PREC_MIXED)) {
    set_error("nlf_apply_K: bad arguments");
    return NLF_EBADARG;
  }
  LinearHandle& h = H->h;
  cudaStream_t st = (cudaStream_t)stream;
  const long N = h.g.N;
  const size_t V = (size_t)nvec * 3 * N;
  NLF_TRY(h.io.reserve(2 * al(N * 8) + 3 * al(V * 8)));
  char* b = (char*)h.io.ptr;
  InView sv, uv;
  NLF_TRY(stage_in(s, N, h.io, 0, sv, st));
  NLF_TRY(stage_in(u, V, h.io, al(N * 8), uv, st));
  double* xs = reinterpret_cast<double*>(b + al(N * 8) + al(V * 8));
  double* ys = reinterpret_cast<double*>(b + al(N * 8) + 2 * al(V * 8));
  double* yd = is_device_ptr(y) ? y : xs;
  if (precision == NLF_PREC_FP64) {
    NLF_TRY((launch_aos_to_soa<double, double>(N, nvec, uv.d, xs, 1.0, st)));
    NLF_TRY(launch_apply<double>(h, sv.d, nvec, nvec, xs, ys, nullptr, nullptr, nullptr, st));
    NLF_TRY((launch_soa_to_aos<double, double>(N, nvec, ys, yd, st)));
  } else {
    float* x32 = reinterpret_cast<float*>(xs);
    float* y32 = reinterpret_cast<float*>(ys);
    float* s32 = reinterpret_cast<float*>(b + al(N * 8) + 3 * al(V * 8));
    NLF_TRY(launch_node_scaling(h, 1, sv.d, s32, nullptr, nullptr, st));
    NLF_TRY((launch_aos_to_soa<double, float>(N, nvec, uv.d, x32, 1.0, st)));
    NLF_TRY(launch_apply<float>(h, s32, nvec, nvec, x32, y32, nullptr, nullptr, nullptr, st));
    NLF_TRY((launch_soa_to_aos<float, double>(N, nvec, y32, yd, st)));
  }
  if (yd != y) NLF_TRY(copy_out(y, yd, V, st));
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  return NLF_OK;
}

// ---- autotuner of the apply tile -----------------------------------------------------------------------------
namespace {
// deterministic pseudo-random fill: a[i] = lo + (hi - lo) * u_i, u_i in [0, 1) from a hash of (seed, i)
__global__ void k_tune_fill(double* __restrict__ a, long n, unsigned seed, double lo, double hi, int logscale) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    unsigned long long z = (unsigned long long)i * 0x9E3779B97F4A7C15ull + seed;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);
    a[i] = logscale ? exp(log(lo) + (log(hi) - log(lo)) * u) : lo + (hi - lo) * u;
  }
}
__global__ void k_tune_f32(const double* __restrict__ a, float* __restrict__ b, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) b[i] = (float)a[i];
}
std::mutex g_tune_mu;
std::map<std::array<int, 4>, int> g_tune_cache;  // (n0, n1, n2, fp64) -> variant
}  // namespace

NLF_API int nlf_apply_variants(int precision) {
  return apply_variants(precision == NLF_PREC_FP64);
}

NLF_API int nlf_linear_set_apply_variant(nlf_linear* H, int precision, int variant) {
  if (bad_handle(H) || (precision != NLF_PREC_FP64 && precision != NLF_PREC_MIXED) || variant < 0 ||
      variant >= apply_variants(precision == NLF_PREC_FP64)) {
    set_error("nlf_linear_set_apply_variant: bad arguments");
    return NLF_EBADARG;
  }
  H->h.apply_variant[precision == NLF_PREC_FP64 ? 1 : 0] = variant;
  return NLF_OK;
}

NLF_API int nlf_linear_get_apply_variant(nlf_linear* H, int precision, int* variant, int* ty, int* tz, int* minb) {
  if (bad_handle(H) || (precision != NLF_PREC_FP64 && precision != NLF_PREC_MIXED) || !variant) {
    set_error("nlf_linear_get_apply_variant: bad arguments");
    return NLF_EBADARG;
  }
  const bool f64 = precision == NLF_PREC_FP64;
  *variant = H->h.apply_variant[f64 ? 1 : 0];
  int a, b, c;
  apply_variant_tile(f64, *variant, &a, &b, &c);
  if (ty) *ty = a;
  if (tz) *tz = b;
  if (minb) *minb = c;
  return NLF_OK;
}

NLF_API int nlf_linear_set_kinv_mode(nlf_linear* H, int mode) {
  if (bad_handle(H) || mode < 0 || mode > 2 || (mode == 2 && H->h.g.n0 != 64)) {
    set_error("nlf_linear_set_kinv_mode: bad arguments");
    return NLF_EBADARG;
  }
  H->h.pcb_closed = mode;
  return NLF_OK;
}

NLF_API int nlf_linear_get_kinv_mode(nlf_linear* H) { return bad_handle(H) ? NLF_EBADARG : H->h.pcb_closed; }

NLF_API int nlf_linear_set_fft_twiddles(nlf_linear* H, int shared) {
  if (bad_handle(H) || shared < 0 || shared > 3) {
    set_error("nlf_linear_set_fft_twiddles: bad arguments");
    return NLF_EBADARG;
  }
  H->h.fft_smt = shared;
  return NLF_OK;
}

NLF_API int nlf_linear_get_fft_twiddles(nlf_linear* H) { return bad_handle(H) ? NLF_EBADARG : H->h.fft_smt; }

NLF_API int nlf_linear_autotune(nlf_linear* H, int precision, int nvec, int reps, int force, double* ms_out,
                                void* stream) {
  if (bad_handle(H) || (precision != NLF_PREC_FP64 && precision != NLF_PREC_MIXED) || nvec < 1 || reps < 1) {
    set_error("nlf_linear_autotune: bad arguments");
    return NLF_EBADARG;
  }
  LinearHandle& h = H->h;
  const bool f64 = precision == NLF_PREC_FP64;
  const int nv = apply_variants(f64);
  const std::array<int, 4> key{h.g.n0, h.g.n1, h.g.n2, f64 ? 1 : 0};
  if (!force && !ms_out) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      h.apply_variant[f64 ? 1 : 0] = it->second % 1000;
      if (f64) {
        h.pcb_closed = (it->second / 1000) % 4;
        h.fft_smt = (it->second / 1000) / 4;
      }
      return NLF_OK;
    }
  }
  cudaStream_t st = (cudaStream_t)stream;
  const long N = h.g.N;
  const size_t V = (size_t)nvec * 3 * N;
  const size_t w = f64 ? 8 : 4;
  // s, x, y and the partials in the staging buffer (FP64 s and x are filled, then converted for FP32)
  NLF_TRY(h.io.reserve(al(N * 8) + 2 * al(V * 8) + al((size_t)nvec * kApplyMaxBlocks * 4 * 8)));
  char* b = (char*)h.io.ptr;
  double* s64 = reinterpret_cast<double*>(b);
  double* x64 = reinterpret_cast<double*>(b + al(N * 8));
  double* y64 = reinterpret_cast<double*>(b + al(N * 8) + al(V * 8));
  double* part = reinterpret_cast<double*>(b + al(N * 8) + 2 * al(V * 8));
  k_tune_fill<<<256, 256, 0, st>>>(s64, N, 1u, h.emin > 0 ? h.emin : 1e-9, 1.0, 1);
  k_tune_fill<<<1024, 256, 0, st>>>(x64, (long)V, 2u, -1.0, 1.0, 0);
  NLF_CHECK_LAUNCH();
  void* sv = s64;
  void* xv = x64;
  void* yv = y64;
  if (!f64) {  // FP32 copies in the upper halves of the FP64 buffers
    float* s32 = reinterpret_cast<float*>(y64);
    float* x32 = reinterpret_cast<float*>(x64) + V;
    k_tune_f32<<<256, 256, 0, st>>>(s64, s32, N);
    k_tune_f32<<<1024, 256, 0, st>>>(x64, x32, (long)V);
    NLF_CHECK_LAUNCH();
    sv = s32;
    xv = x32;
    yv = reinterpret_cast<float*>(y64) + N;
  }
  (void)w;
  cudaEvent_t e0, e1;
  NLF_CUDA_TRY(cudaEventCreate(&e0));
  NLF_CUDA_TRY(cudaEventCreate(&e1));
  const int keep = h.apply_variant[f64 ? 1 : 0];
  int best = keep, rc = NLF_OK;
  float best_ms = 0.0f;
  for (int v = 0; v < nv && rc == NLF_OK; ++v) {
    h.apply_variant[f64 ? 1 : 0] = v;
    auto run = [&]() {
      return f64 ? launch_apply<double>(h, (const double*)sv, 6, nvec, (const double*)xv, (double*)yv, nullptr,
                                        part, nullptr, st)
                 : launch_apply<float>(h, (const float*)sv, 6, nvec, (const float*)xv, (float*)yv, nullptr, part,
                                       nullptr, st);
    };
    rc = run();  // warm-up
    if (rc != NLF_OK) break;
    cudaEventRecord(e0, st);
    for (int r = 0; r < reps && rc == NLF_OK; ++r) rc = run();
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      rc = NLF_ECUDA;
      set_error("nlf_linear_autotune: %s", cudaGetErrorString(cudaGetLastError()));
      break;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= (float)reps;
    if (ms_out) ms_out[v] = ms;
    if (v == 0 || ms < best_ms) {
      best_ms = ms;
      best = v;
    }
  }
  h.apply_variant[f64 ? 1 : 0] = rc == NLF_OK ? best : keep;
  // FP64 cubes with the register-resident FFT passes: pass B with the Kinv table or in closed form, timed on the
  // scaled preconditioner of the same vectors (node scaling from s)
  int pcb = 0;
  if (rc == NLF_OK && f64 && precond_fuses_px(h)) {
    DevBuf& tb = h.io2;
    rc = tb.reserve(al(N * 8) + al((size_t)nvec * 3 * h.g.NS * 16));
    double* w64 = rc == NLF_OK ? static_cast<double*>(tb.ptr) : nullptr;
    cplx<double>* spec = rc == NLF_OK ? reinterpret_cast<cplx<double>*>(static_cast<char*>(tb.ptr) + al(N * 8))
                                      : nullptr;
    if (rc == NLF_OK) rc = launch_node_scaling(h, 1, s64, nullptr, w64, nullptr, st);
    float best_pc = 0.0f;
    const int nk = h.g.n0 == 64 ? 3 : 2;  // Kinv modes: table, closed form, closed form with staged slabs (64^3)
    for (int v = 0; v < 4 * nk && rc == NLF_OK; ++v) {  // v = Kinv mode + nk x twiddle / staging mode (0 .. 3)
      h.pcb_closed = v % nk;
      h.fft_smt = v / nk;
      rc = launch_precond<double>(h, nvec, 6, x64, y64, spec, w64, nullptr, part, st);
      if (rc != NLF_OK) break;
      cudaEventRecord(e0, st);
      for (int r = 0; r < reps && rc == NLF_OK; ++r) rc = launch_precond<double>(h, nvec, 6, x64, y64, spec, w64,
                                                                              nullptr, part, st);
      cudaEventRecord(e1, st);
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        rc = NLF_ECUDA;
        set_error("nlf_linear_autotune: %s", cudaGetErrorString(cudaGetLastError()));
        break;
      }
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      ms /= (float)reps;
      if (ms_out) ms_out[nv + v] = ms;
      if (v == 0 || ms < best_pc) {
        best_pc = ms;
        pcb = v;
      }
    }
    h.pcb_closed = rc == NLF_OK ? pcb % nk : 0;
    h.fft_smt = rc == NLF_OK ? pcb / nk : 0;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != NLF_OK) return rc;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache[key] = best + 1000 * (h.pcb_closed + 4 * h.fft_smt);
  return NLF_OK;
}

NLF_API int nlf_apply_K(nlf_linear* H, const double* s, int nvec, const double* u, double* y, void* stream) {
  return nlf_apply_K_ex(H, s, nvec, u, y, NLF_PREC_FP64, stream);
}

NLF_API int nlf_load(nlf_linear* H, const double* s, const double* Es, int m, double* f, void* stream) {
  if (bad_handle(H) || m < 1 || !s || !Es || !f) {
    set_error("nlf_load: bad arguments");
    return NLF_EBADARG;
  }
  LinearHandle& h = H->h;
  cudaStream_t st = (cudaStream_t)stream;
  const long N = h.g.N;
  const size_t V = (size_t)m * 3 * N;
  std::vector<double> Esh, fe;
  NLF_TRY(host_copy_small(Es, (size_t)m * 6, Esh));
  es_to_fe(h, Esh.data(), m, fe);
  NLF_TRY(h.io.reserve(al(N * 8) + al(fe.size() * 8) + 2 * al(V * 8)));
  char* b = (char*)h.io.ptr;
  InView sv;
  NLF_TRY(stage_in(s, N, h.io, 0, sv, st));
  double* fed = reinterpret_cast<double*>(b + al(N * 8));
  NLF_CUDA_TRY(cudaMemcpyAsync(fed, fe.data(), fe.size() * 8, cudaMemcpyHostToDevice, st));
  double* fs = reinterpret_cast<double*>(b + al(N * 8) + al(fe.size() * 8));
  double* fa = reinterpret_cast<double*>(b + al(N * 8) + al(fe.size() * 8) + al(V * 8));
  NLF_TRY(launch_load(h, sv.d, fed, m, 1, fs, 1.0, st));
  double* fd = is_device_ptr(f) ? f : fa;
  NLF_TRY((launch_soa_to_aos<double, double>(N, m, fs, fd, st)));
  if (fd != f) NLF_TRY(copy_out(f, fd, V, st));
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  return NLF_OK;
}

NLF_API int nlf_precond_ex(nlf_linear* H, int nvec, const double* r, double* z, int precision, int precond,
                           const double* s, void* stream) {
  if (bad_handle(H) || nvec < 1 || !r || !z || (precision != NLF_PREC_FP64 && precision != NLF_PREC_MIXED) ||
      (precond != NLF_PC_FFT && precond != NLF_PC_FFT_SCALED) || (precond == NLF_PC_FFT_SCALED && !s)) {
    set_error("nlf_precond: bad arguments");
    return NLF_EBADARG;
  }
  LinearHandle& h = H->h;
  cudaStream_t st = (cudaStream_t)stream;
  const long N = h.g.N;
  const size_t V = (size_t)nvec * 3 * N;
  const size_t S = (size_t)nvec * 3 * h.g.NS * 2;
  NLF_TRY(h.io.reserve(3 * al(V * 8) + al(S * 8) + 3 * al(N * 8)));
  char* b = (char*)h.io.ptr;
  InView rv, sv;
  NLF_TRY(stage_in(r, V, h.io, 0, rv, st));
  const size_t o_s = 3 * al(V * 8) + al(S * 8);
  NLF_TRY(stage_in(s, N, h.io, o_s, sv, st));
  void* wbuf = b + o_s + al(N * 8);
  const bool scaled = precond == NLF_PC_FFT_SCALED;
  double* rs = reinterpret_cast<double*>(b + al(V * 8));
  double* zs = reinterpret_cast<double*>(b + 2 * al(V * 8));
  double* zd = is_device_ptr(z) ? z : rs;
  if (precision == NLF_PREC_FP64) {
    double* w = scaled ? reinterpret_cast<double*>(wbuf) : nullptr;
    if (scaled) NLF_TRY(launch_node_scaling(h, 1, sv.d, nullptr, w, nullptr, st));
    cplx<double>* spec = reinterpret_cast<cplx<double>*>(b + 3 * al(V * 8));
    NLF_TRY((launch_aos_to_soa<double, double>(N, nvec, rv.d, rs, 1.0, st)));
    NLF_TRY(launch_precond<double>(h, nvec, nvec, rs, zs, spec, w, nullptr, nullptr, st));  // one cell
    NLF_TRY((launch_soa_to_aos<double, double>(N, nvec, zs, zd, st)));
  } else {
    float* w = scaled ? reinterpret_cast<float*>(wbuf) : nullptr;
    if (scaled) NLF_TRY(launch_node_scaling(h, 1, sv.d, nullptr, nullptr, w, st));
    cplx<float>* spec = reinterpret_cast<cplx<float>*>(b + 3 * al(V * 8));
    float* r32 = reinterpret_cast<float*>(rs);
    float* z32 = reinterpret_cast<float*>(zs);
    NLF_TRY((launch_aos_to_soa<double, float>(N, nvec, rv.d, r32, 1.0, st)));
    NLF_TRY(launch_precond<float>(h, nvec, nvec, r32, z32, spec, w, nullptr, nullptr, st));  // one cell
    NLF_TRY((launch_soa_to_aos<float, double>(N, nvec, z32, zd, st)));
  }
  if (zd != z) NLF_TRY(copy_out(z, zd, V, st));
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  return NLF_OK;
}

NLF_API int nlf_precond(nlf_linear* H, int nvec, const double* r, double* z, void* stream) {
  return nlf_precond_ex(H, nvec, r, z, NLF_PREC_FP64, NLF_PC_FFT, nullptr, stream);
}

static int solve_entry(nlf_linear* H, int ncell, const double* s, const double* Es, const double* bsrc, int m,
                       const double* u0, double* u, int* iters, const nlf_solve_opts* opts, void* stream) {
  LinearHandle& h = H->h;
  cudaStream_t st = (cudaStream_t)stream;
  const long N = h.g.N;
  const int nvec = ncell * m;
  const size_t V = (size_t)nvec * 3 * N;
  const nlf_solve_opts o = resolve_opts(h, opts);
  std::vector<double> fe;
  if (Es) {
    std::vector<double> Esh;
    NLF_TRY(host_copy_small(Es, (size_t)m * 6, Esh));
    es_to_fe(h, Esh.data(), m, fe);
  }
  // io: s | fe | b (SoA) | u0 (AoS) | x (SoA) | u (AoS)
  const size_t o_s = 0, o_fe = al((size_t)ncell * N * 8), o_b = o_fe + al(m * 24 * 8 + 8);
  const size_t o_u0 = o_b + (bsrc ? al(V * 8) : 0);
  const size_t o_x = o_u0 + (u0 && !is_device_ptr(u0) ? al(V * 8) : 0);
  const size_t o_u = o_x + al(V * 8);
  NLF_TRY(h.io.reserve(o_u + al(V * 8)));
  char* b = (char*)h.io.ptr;
  InView sv, u0v;
  NLF_TRY(stage_in(s, (size_t)ncell * N, h.io, o_s, sv, st));
  double* fed = reinterpret_cast<double*>(b + o_fe);
  if (Es) NLF_CUDA_TRY(cudaMemcpyAsync(fed, fe.data(), fe.size() * 8, cudaMemcpyHostToDevice, st));
  double* bsoa = nullptr;
  if (bsrc) {
    InView bv;
    NLF_TRY(stage_in(bsrc, V, h.io, o_x, bv, st));  // staging through the x slot, converted below
    bsoa = reinterpret_cast<double*>(b + o_b);
    NLF_TRY((launch_aos_to_soa<double, double>(N, nvec, bv.d, bsoa, 1.0, st)));
  }
  NLF_TRY(stage_in(u0, V, h.io, o_u0, u0v, st));
  double* xs = reinterpret_cast<double*>(b + o_x);
  SolveIn in{ncell, m, sv.d, bsoa, fed, u0v.d, false, Ede{}};
  if (Es && m <= 6) {
    std::vector<double> Esh;
    NLF_TRY(host_copy_small(Es, (size_t)m * 6, Esh));
    in.has_ede = true;
    for (int I = 0; I < m; ++I) {
      double a = 0.0;
      for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) a += Esh[I * 6 + i] * h.Dm[i][j] * Esh[I * 6 + j];
      in.ede.v[I] = a;
    }
  }
  std::vector<int> it(ncell, 0);
  int status = solve_core(h, in, o, xs, it.data(), st);
  if (status < 0) return status;
  double* ud = is_device_ptr(u) ? u : reinterpret_cast<double*>(b + o_u);
  NLF_TRY((launch_soa_to_aos<double, double>(N, nvec, xs, ud, st)));
  if (ud != u) NLF_TRY(copy_out(u, ud, V, st));
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  if (iters) {
    if (is_device_ptr(iters)) {
      NLF_CUDA_TRY(cudaMemcpy(iters, it.data(), ncell * sizeof(int), cudaMemcpyHostToDevice));
    } else {
      std::memcpy(iters, it.data(), ncell * sizeof(int));
    }
  }
  return status;
}

NLF_API int nlf_linear_solve(nlf_linear* H, int ncell, const double* s, const double* Es, int m, const double* u0,
                             double* u, int* iters, const nlf_solve_opts* opts, void* stream) {
  if (bad_handle(H) || ncell < 1 || m < 1 || !s || !Es || !u) {
    set_error("nlf_linear_solve: bad arguments");
    return NLF_EBADARG;
  }
  return solve_entry(H, ncell, s, Es, nullptr, m, u0, u, iters, opts, stream);
}

NLF_API int nlf_linear_solve_rhs(nlf_linear* H, int ncell, const double* s, int m, const double* b, double* u,
                                 int* iters, const nlf_solve_opts* opts, void* stream) {
  if (bad_handle(H) || ncell < 1 || m < 1 || !s || !b || !u) {
    set_error("nlf_linear_solve_rhs: bad arguments");
    return NLF_EBADARG;
  }
  return solve_entry(H, ncell, s, nullptr, b, m, nullptr, u, iters, opts, stream);
}

static int bilinear_entry(nlf_linear* H, int ncell, const double* s, const double* rho, const double* Es, int m,
                          const double* u, double* C, double* dC, void* stream) {
  LinearHandle& h = H->h;
  cudaStream_t st = (cudaStream_t)stream;
  const long N = h.g.N;
  const int nvec = ncell * m;
  const size_t V = (size_t)nvec * 3 * N;
  std::vector<double> Esh;
  NLF_TRY(host_copy_small(Es, (size_t)m * 6, Esh));
  std::vector<double> EsEDE((size_t)m * 6 + (size_t)m * m);
  for (int i = 0; i < m * 6; ++i) EsEDE[i] = Esh[i];
  for (int I = 0; I < m; ++I)
    for (int J = 0; J < m; ++J) {
      double a = 0.0;
      for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) a += Esh[I * 6 + i] * h.Dm[i][j] * Esh[J * 6 + j];
      EsEDE[(size_t)m * 6 + I * m + J] = a;
    }
  const int nb = (int)((N + 127) / 128);
  const size_t o_s = 0, o_r = al((size_t)ncell * N * 8), o_u = o_r + al((size_t)ncell * N * 8);
  const size_t o_us = o_u + al(V * 8), o_e = o_us + al(V * 8), o_cp = o_e + al(EsEDE.size() * 8);
  const size_t o_c = o_cp + al((size_t)ncell * nb * 21 * 8);
  const size_t o_dc = o_c + al((size_t)ncell * m * m * 8);
  const size_t dcount = dC ? (size_t)ncell * m * m * N : 0;
  NLF_TRY(h.io.reserve(o_dc + al(dcount * 8) + 256));
  char* b = (char*)h.io.ptr;
  InView sv, rv, uv;
  double* sd = nullptr;
  if (rho) {
    NLF_TRY(stage_in(rho, (size_t)ncell * N, h.io, o_r, rv, st));
    sd = reinterpret_cast<double*>(b + o_s);
    NLF_TRY(launch_stiffness_scale(h, (long)ncell * N, rv.d, sd, st));
  } else {
    NLF_TRY(stage_in(s, (size_t)ncell * N, h.io, o_s, sv, st));
    sd = const_cast<double*>(sv.d);
  }
  NLF_TRY(stage_in(u, V, h.io, o_u, uv, st));
  double* us = reinterpret_cast<double*>(b + o_us);
  NLF_TRY((launch_aos_to_soa<double, double>(N, nvec, uv.d, us, 1.0, st)));
  double* ed = reinterpret_cast<double*>(b + o_e);
  NLF_CUDA_TRY(cudaMemcpyAsync(ed, EsEDE.data(), EsEDE.size() * 8, cudaMemcpyHostToDevice, st));
  double* cp = reinterpret_cast<double*>(b + o_cp);
  double* cd = reinterpret_cast<double*>(b + o_c);
  double* dcd = dC ? (is_device_ptr(dC) ? dC : reinterpret_cast<double*>(b + o_dc)) : nullptr;
  int nblk = 0;
  NLF_TRY(launch_bilinear(h, sd, ed, m, ncell, us, cp, &nblk, rho ? rv.d : nullptr, dcd, st));
  NLF_TRY(launch_reduce_C(h, cp, nblk, m, ncell, cd, st));
  if (C) NLF_TRY(copy_out(C, cd, (size_t)ncell * m * m, st));
  if (dC && dcd != dC) NLF_TRY(copy_out(dC, dcd, dcount, st));
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  return NLF_OK;
}

NLF_API int nlf_bilinear(nlf_linear* H, int ncell, const double* s, const double* Es, int m, const double* u,
                         double* C, void* stream) {
  if (bad_handle(H) || ncell < 1 || m < 1 || m > 6 || !s || !Es || !u || !C) {
    set_error("nlf_bilinear: bad arguments (1 <= m <= 6)");
    return NLF_EBADARG;
  }
  return bilinear_entry(H, ncell, s, nullptr, Es, m, u, C, nullptr, stream);
}

NLF_API int nlf_dC_drho(nlf_linear* H, int ncell, const double* rho, const double* Es, int m, const double* u,
                        double* dC, void* stream) {
  if (bad_handle(H) || ncell < 1 || m < 1 || m > 6 || !rho || !Es || !u || !dC) {
    set_error("nlf_dC_drho: bad arguments (1 <= m <= 6)");
    return NLF_EBADARG;
  }
  return bilinear_entry(H, ncell, nullptr, rho, Es, m, u, nullptr, dC, stream);
}

NLF_API int nlf_correctors_vjp(nlf_linear* H, int ncell, const double* s, const double* rho, const double* Es, int m,
                               const double* u, const double* ubar, double* sbar, double* lam, int* iters,
                               const nlf_solve_opts* opts, void* stream) {
  if (bad_handle(H) || ncell < 1 || m < 1 || m > 6 || (!s && !rho) || !Es || !u || !ubar || !sbar) {
    set_error("nlf_correctors_vjp: bad arguments (s or rho, Es, u, ubar, sbar; 1 <= m <= 6)");
    return NLF_EBADARG;
  }
  LinearHandle& h = H->h;
  cudaStream_t st = (cudaStream_t)stream;
  const long N = h.g.N;
  const int nvec = ncell * m;
  const size_t V = (size_t)nvec * 3 * N;
  // io2 (the solve stages through io): s | rho | ubar -> b = -ubar (AoS) | lam (AoS) | u, lam (SoA) | Es | out
  const size_t o_s = 0, o_r = al((size_t)ncell * N * 8), o_b = o_r + al((size_t)ncell * N * 8),
               o_l = o_b + al(V * 8), o_us = o_l + al(V * 8), o_ls = o_us + al(V * 8), o_e = o_ls + al(V * 8),
               o_o = o_e + al((size_t)m * 6 * 8), total = o_o + al((size_t)ncell * N * 8);
  NLF_TRY(h.io2.reserve(total));
  char* b = (char*)h.io2.ptr;
  InView rv;
  double* sd = reinterpret_cast<double*>(b + o_s);
  if (rho) {
    NLF_TRY(stage_in(rho, (size_t)ncell * N, h.io2, o_r, rv, st));
    NLF_TRY(launch_stiffness_scale(h, (long)ncell * N, rv.d, sd, st));
  } else if (is_device_ptr(s)) {
    NLF_CUDA_TRY(cudaMemcpyAsync(sd, s, (size_t)ncell * N * 8, cudaMemcpyDeviceToDevice, st));
  } else {
    NLF_CUDA_TRY(cudaMemcpyAsync(sd, s, (size_t)ncell * N * 8, cudaMemcpyHostToDevice, st));
  }
  // b = -ubar (the solve projects it: K lam = -proj(ubar), nlfiber/linear.py:127)
  double* bd = reinterpret_cast<double*>(b + o_b);
  NLF_CUDA_TRY(cudaMemcpyAsync(bd, ubar, V * 8, is_device_ptr(ubar) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                               st));
  NLF_TRY((launch_aos_to_soa<double, double>(N, nvec, bd, reinterpret_cast<double*>(b + o_us), -1.0, st)));
  NLF_TRY((launch_soa_to_aos<double, double>(N, nvec, reinterpret_cast<double*>(b + o_us), bd, st)));
  double* ld = reinterpret_cast<double*>(b + o_l);
  int status = solve_entry(H, ncell, sd, nullptr, bd, m, nullptr, ld, iters, opts, stream);
  if (status < 0) return status;
  // u and lam to SoA, then sbar (or rhobar)
  InView uv;
  double* us = reinterpret_cast<double*>(b + o_us);
  double* ls = reinterpret_cast<double*>(b + o_ls);
  if (is_device_ptr(u)) {
    NLF_TRY((launch_aos_to_soa<double, double>(N, nvec, u, us, 1.0, st)));
  } else {
    NLF_CUDA_TRY(cudaMemcpyAsync(ls, u, V * 8, cudaMemcpyHostToDevice, st));  // staged through the lam slot
    NLF_TRY((launch_aos_to_soa<double, double>(N, nvec, ls, us, 1.0, st)));
  }
  NLF_TRY((launch_aos_to_soa<double, double>(N, nvec, ld, ls, 1.0, st)));
  std::vector<double> Esh;
  NLF_TRY(host_copy_small(Es, (size_t)m * 6, Esh));
  double* ed = reinterpret_cast<double*>(b + o_e);
  NLF_CUDA_TRY(cudaMemcpyAsync(ed, Esh.data(), Esh.size() * 8, cudaMemcpyHostToDevice, st));
  double* od = is_device_ptr(sbar) ? sbar : reinterpret_cast<double*>(b + o_o);
  NLF_TRY(launch_adjoint_sbar(h, ed, m, ncell, us, ls, rho ? rv.d : nullptr, od, st));
  if (od != sbar) NLF_TRY(copy_out(sbar, od, (size_t)ncell * N, st));
  if (lam) NLF_TRY(copy_out(lam, ld, V, st));
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  return status;
}

NLF_API int nlf_C_full(nlf_linear* H, int ncell, const double* rho, const double* u0, double* C, double* u,
                       double* dC, int* iters, const nlf_solve_opts* opts, void* stream) {
  if (bad_handle(H) || ncell < 1 || !rho || !C) {
    set_error("nlf_C_full: bad arguments");
    return NLF_EBADARG;
  }
  LinearHandle& h = H->h;
  cudaStream_t st = (cudaStream_t)stream;
  const long N = h.g.N;
  const int m = 6;
  const size_t V = (size_t)ncell * m * 3 * N;
  // separate staging (io2) so that the solve's own io staging does not clobber rho / s / u
  NLF_TRY(h.io2.reserve(2 * al((size_t)ncell * N * 8) + al(V * 8)));
  char* b = (char*)h.io2.ptr;
  InView rv;
  NLF_TRY(stage_in(rho, (size_t)ncell * N, h.io2, 0, rv, st));
  double* sd = reinterpret_cast<double*>(b + al((size_t)ncell * N * 8));
  NLF_TRY(launch_stiffness_scale(h, (long)ncell * N, rv.d, sd, st));
  double* ud = (u && is_device_ptr(u)) ? u : reinterpret_cast<double*>(b + 2 * al((size_t)ncell * N * 8));
  double eye[36] = {};
  for (int i = 0; i < 6; ++i) eye[i * 6 + i] = 1.0;
  int status = nlf_linear_solve(H, ncell, sd, eye, m, u0, ud, iters, opts, stream);
  if (status < 0) return status;
  int s2 = bilinear_entry(H, ncell, sd, dC ? rv.d : nullptr, eye, m, ud, C, dC, stream);
  if (s2 < 0) return s2;
  if (u && ud != u) {
    NLF_TRY(copy_out(u, ud, V, st));
    NLF_CUDA_TRY(cudaStreamSynchronize(st));
  }
  return status;
}

NLF_API int nlf_precond_symbol(nlf_linear* H, double* kinv6) {
  if (bad_handle(H) || !kinv6) {
    set_error("nlf_precond_symbol: bad arguments");
    return NLF_EBADARG;
  }
  LinearHandle& h = H->h;
  NLF_CUDA_TRY(cudaMemcpy(kinv6, h.t64.kinv, h.g.NS * 6 * sizeof(double),
                          is_device_ptr(kinv6) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost));
  return NLF_OK;
}

}  // extern "C"
