// Elementwise and reduction kernels of the batched lock-step PCG (nlfiber/linear.py:173-203).
//
// Every vector is [vec][comp][N]; vec = cell * m + case. Reductions write per-CTA FP64 partials that a
// finalize kernel sums in a fixed order (deterministic). A cell whose CellState.active is 0 is skipped by
// every kernel, which reproduces the reference's lock-step `while_loop` per cell inside a batch of cells.
#include "nlf_vec.cuh"
#include "nlf_prof.cuh"

namespace nlf {

// ---- layout conversion -------------------------------------------------------------------------------------
template <typename Tin, typename Tout>
__global__ void k_aos_to_soa(long N, const Tin* __restrict__ in, Tout* __restrict__ out, double scale) {
  const long n = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long vec = blockIdx.y;
  if (n >= N) return;
  const Tin* p = in + (vec * N + n) * 3;
#pragma unroll
  for (int c = 0; c < 3; ++c) out[(vec * 3 + c) * N + n] = (Tout)((double)p[c] * scale);
}

template <typename Tin, typename Tout>
__global__ void k_soa_to_aos(long N, const Tin* __restrict__ in, Tout* __restrict__ out) {
  const long n = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long vec = blockIdx.y;
  if (n >= N) return;
  Tout* p = out + (vec * N + n) * 3;
#pragma unroll
  for (int c = 0; c < 3; ++c) p[c] = (Tout)in[(vec * 3 + c) * N + n];
}

template <typename Tin, typename Tout>
int launch_aos_to_soa(long N, int nvec, const Tin* in, Tout* out, double scale, cudaStream_t st) {
  if (nvec == 0) return NLF_OK;
  ProfScope ps_(PK_OTHER, st);
  k_aos_to_soa<Tin, Tout><<<dim3((unsigned)((N + 255) / 256), nvec), 256, 0, st>>>(N, in, out, scale);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}
template <typename Tin, typename Tout>
int launch_soa_to_aos(long N, int nvec, const Tin* in, Tout* out, cudaStream_t st) {
  if (nvec == 0) return NLF_OK;
  ProfScope ps_(PK_OTHER, st);
  k_soa_to_aos<Tin, Tout><<<dim3((unsigned)((N + 255) / 256), nvec), 256, 0, st>>>(N, in, out);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}
template int launch_aos_to_soa<double, double>(long, int, const double*, double*, double, cudaStream_t);
template int launch_aos_to_soa<double, float>(long, int, const double*, float*, double, cudaStream_t);
template int launch_soa_to_aos<double, double>(long, int, const double*, double*, cudaStream_t);
template int launch_soa_to_aos<float, double>(long, int, const float*, double*, cudaStream_t);

// ---- stiffness scale, node scaling of the scaled preconditioner -----------------------------------------------
__device__ __forceinline__ double clip01(double r) { return r > 1.0 ? 1.0 : (r < 0.0 ? 0.0 : r); }

__global__ void k_stiffness_scale(long count, const double* __restrict__ rho, double* __restrict__ s, double emin,
                                  double p) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < count) s[i] = emin + (1.0 - emin) * pow(clip01(rho[i]), p);
}

int launch_stiffness_scale(const LinearHandle& h, long count, const double* rho, double* s, cudaStream_t st) {
  if (count == 0) return NLF_OK;
  ProfScope ps_(PK_OTHER, st);
  k_stiffness_scale<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(count, rho, s, h.emin, h.p);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}

// s32 = (float) s; w = (root mean square of s over the 8 elements around each node)^-kNodeScaleExp
__global__ void k_node_scaling(int n0, int n1, int n2, const double* __restrict__ s, float* __restrict__ s32,
                               double* __restrict__ w64, float* __restrict__ w32) {
  const long N = (long)n0 * n1 * n2;
  const long n = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const int cell = blockIdx.y;
  if (n >= N) return;
  const double* sv = s + (long)cell * N;
  if (s32) s32[(long)cell * N + n] = (float)sv[n];
  if (w64 || w32) {
    const int k = (int)(n % n2), j = (int)((n / n2) % n1), i = (int)(n / ((long)n1 * n2));
    // w = S^-0.47, S = root mean square of the 8 element scales around the node. Of the power means tried on
    // 64^3 cells of the benchmark generator, p = 2 needed the fewest PCG iterations (17 % fewer than the
    // arithmetic mean, 6 % fewer than the maximum; geometric and harmonic means fail at 1e-9 contrast). The
    // exponent is sharp around its optimum: 0.47 needs 13-15 % fewer iterations than 0.5 on the benchmark cells
    // and on held-out seeds alike; 0.40 needs 38 % more than 0.47, 0.55 2.4 times as many.
    double acc = 0.0;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const int ii = wrap(i - (a & 1), n0), jj = wrap(j - ((a >> 1) & 1), n1), kk = wrap(k - (a >> 2), n2);
      const double v = sv[((long)ii * n1 + jj) * n2 + kk];
      acc += v * v;
    }
    const double w = pow(acc * 0.125, -0.5 * kNodeScaleExp);
    if (w64) w64[(long)cell * N + n] = w;
    if (w32) w32[(long)cell * N + n] = (float)w;
  }
}

int launch_node_scaling(const LinearHandle& h, int ncell, const double* s, float* s32, double* w64, float* w32,
                        cudaStream_t st) {
  if (ncell == 0) return NLF_OK;
  ProfScope ps_(PK_OTHER, st);
  k_node_scaling<<<dim3((unsigned)((h.g.N + 255) / 256), ncell), 256, 0, st>>>(h.g.n0, h.g.n1, h.g.n2, s, s32,
                                                                               w64, w32);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}

// ---- statistics: per (vec, comp) sum and sum of squares ------------------------------------------------------
template <typename T>
__global__ void k_stats(long N, const T* __restrict__ x, const CellState* __restrict__ cs, int m,
                        double* __restrict__ partial) {
  __shared__ double red[32 * 2];
  const int c = blockIdx.y, vec = blockIdx.z;
  if (cs && !cs[vec / m].active) return;
  const T* p = x + ((long)vec * 3 + c) * N;
  double acc[2] = {0.0, 0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const double v = (double)p[i];
    acc[0] += v;
    acc[1] += v * v;
  }
  block_sum<2>(acc, red);
  if (threadIdx.x == 0) {
    double* o = partial + (((long)vec * 3 + c) * gridDim.x + blockIdx.x) * 2;
    o[0] = acc[0];
    o[1] = acc[1];
  }
}

// what: 0 -> mean[c] = sum_c / N; 1 -> bn = sqrt(sum of squares) + 1e-300; 2 -> rr = sum of squares
__global__ void k_fin_stats(const double* __restrict__ partial, int nb, long N, int nvec, VecState* __restrict__ vs,
                            const CellState* __restrict__ cs, int m, int what) {
  const int vec = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (vec >= nvec) return;
  if (cs && !cs[vec / m].active) return;
  double s[3] = {0, 0, 0}, q = 0.0;
  for (int c = 0; c < 3; ++c) {
    for (int b = lane; b < nb; b += 32) {
      const double* o = partial + (((long)vec * 3 + c) * nb + b) * 2;
      s[c] += o[0];
      q += o[1];
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s[0] += __shfl_down_sync(0xffffffffu, s[0], o);
    s[1] += __shfl_down_sync(0xffffffffu, s[1], o);
    s[2] += __shfl_down_sync(0xffffffffu, s[2], o);
    q += __shfl_down_sync(0xffffffffu, q, o);
  }
  if (lane == 0) {
    if (what == 0) {
      vs[vec].mean[0] = s[0] / (double)N;
      vs[vec].mean[1] = s[1] / (double)N;
      vs[vec].mean[2] = s[2] / (double)N;
    } else if (what == 1) {
      vs[vec].bn = sqrt(q) + 1e-300;
    } else {
      vs[vec].rr = q;
    }
  }
}

template <typename T>
int launch_stats(const LinearHandle& h, int nvec, int m, const T* x, const CellState* cs, double* partial,
                 VecState* vs, int what, cudaStream_t st) {
  if (nvec == 0) return NLF_OK;
  const int nb = kStatsBlocks;
  ProfScope ps_(PK_STATS, st);
  k_stats<T><<<dim3(nb, 3, nvec), 256, 0, st>>>(h.g.N, x, cs, m, partial);
  NLF_CHECK_LAUNCH();
  ProfScope ps2_(PK_FIN, st);
  k_fin_stats<<<(nvec + 7) / 8, 256, 0, st>>>(partial, nb, h.g.N, nvec, vs, cs, m, what);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}
template int launch_stats<float>(const LinearHandle&, int, int, const float*, const CellState*, double*, VecState*,
                                 int, cudaStream_t);
template int launch_stats<double>(const LinearHandle&, int, int, const double*, const CellState*, double*,
                                  VecState*, int, cudaStream_t);

// x[c] -= mean[c]
template <typename T>
__global__ void k_sub_mean(long N, T* __restrict__ x, const VecState* __restrict__ vs,
                           const CellState* __restrict__ cs, int m) {
  const int vec = blockIdx.z, c = blockIdx.y;
  if (cs && !cs[vec / m].active) return;
  const T mu = (T)vs[vec].mean[c];
  T* p = x + ((long)vec * 3 + c) * N;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) p[i] -= mu;
}

template <typename T>
int launch_sub_mean(const LinearHandle& h, int nvec, int m, T* x, const VecState* vs, const CellState* cs,
                    cudaStream_t st) {
  if (nvec == 0) return NLF_OK;
  const int nb = (int)std::min<long>((h.g.N + 255) / 256, 256);
  ProfScope ps_(PK_OTHER, st);
  k_sub_mean<T><<<dim3(nb, 3, nvec), 256, 0, st>>>(h.g.N, x, vs, cs, m);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}
template int launch_sub_mean<float>(const LinearHandle&, int, int, float*, const VecState*, const CellState*,
                                    cudaStream_t);
template int launch_sub_mean<double>(const LinearHandle&, int, int, double*, const VecState*, const CellState*,
                                     cudaStream_t);

// ---- PCG steps ---------------------------------------------------------------------------------------------
// After the apply: mean[c] of Ap, pAp = (p, Ap - mean) and alpha = rz / pAp (pAp == 0 -> 1).
// init = 1: only the means (r = b - proj(A x) at the start).
__global__ void k_fin_apply(const double* __restrict__ partial, int nblk, long N, int nvec, VecState* __restrict__ vs,
                            const CellState* __restrict__ cs, int m, int init) {
  const int vec = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (vec >= nvec) return;
  if (!vec_live(cs, vec, m)) return;
  double a[4] = {0, 0, 0, 0};
  for (int b = lane; b < nblk; b += 32) {
    const double* o = partial + ((long)vec * nblk + b) * 4;
    a[0] += o[0];
    a[1] += o[1];
    a[2] += o[2];
    a[3] += o[3];
  }
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a[k] += __shfl_down_sync(0xffffffffu, a[k], o);
  if (lane == 0) {
    VecState& v = vs[vec];
    v.mean[0] = a[0] / (double)N;
    v.mean[1] = a[1] / (double)N;
    v.mean[2] = a[2] / (double)N;
    if (!init) {
      const double pAp = a[3];  // (p, Ap - mean Ap) = (p, Ap) since p is mean-free
      v.alpha = v.rz / (pAp == 0.0 ? 1.0 : pAp);
    }
  }
}


// r = b - (Ax - mean)
template <typename Tb, typename T>
__global__ void k_r_init(long N, T* __restrict__ r, const Tb* __restrict__ b, const T* __restrict__ Ax,
                         const VecState* __restrict__ vs, const CellState* __restrict__ cs, int m) {
  const int vec = blockIdx.z, c = blockIdx.y;
  if (cs && !cs[vec / m].active) return;
  const double mu = vs[vec].mean[c];
  const long off = ((long)vec * 3 + c) * N;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
    r[off + i] = (T)((double)b[off + i] - ((double)Ax[off + i] - mu));
}

// After the preconditioner: mean[c] of z, rz1 = (r, z - mean z), rr = (r, r); per-cell lock-step control.
// One block per cell, one warp per case. init = 1: rz = rz1, it stays 0. Otherwise beta = rz1 / rz, it += 1.
// active = it < maxit && any case with sqrt(rr) > tol * bn (nlfiber/linear.py:185-188).
__global__ void k_fin_pc(const double* __restrict__ partial, int n0, long N, VecState* __restrict__ vs,
                         CellState* __restrict__ cs, int m, double tol, int maxit, int init) {
  __shared__ int go;
  const int cell = blockIdx.x;
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (!cs[cell].active) return;
  if (threadIdx.x == 0) go = 0;
  __syncthreads();
  if (wid < m) {
    const int vec = cell * m + wid;
    double a[3][4];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int k = 0; k < 4; ++k) a[c][k] = 0.0;
    for (int c = 0; c < 3; ++c)
      for (int x = lane; x < n0; x += 32) {
        const double* o = partial + (((long)vec * 3 + c) * n0 + x) * 4;
#pragma unroll
        for (int k = 0; k < 4; ++k) a[c][k] += o[k];
      }
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a[c][k] += __shfl_down_sync(0xffffffffu, a[c][k], o);
    if (lane == 0) {
      VecState& v = vs[vec];
      double rz1 = 0.0, rr = 0.0;
      for (int c = 0; c < 3; ++c) {
        const double mz = a[c][0] / (double)N;
        v.mean[c] = mz;
        rz1 += a[c][1] - mz * a[c][2];
        rr += a[c][3];
      }
      if (!init) v.beta = rz1 / (v.rz == 0.0 ? 1.0 : v.rz);
      if (init) v.streak = 0;
      v.rz = rz1;
      v.rr = rr;
      if (sqrt(rr) > tol * v.bn) atomicOr(&go, 1);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    CellState& s = cs[cell];
    if (!init) s.it += 1;
    s.active = (s.it < maxit) && go;
  }
}

// p = (z - mean z) + beta p   (init: p = z - mean z). Runs for cells active at the start of the iteration,
// which is signalled by `was` (the pre-iteration flag kept in CellState.status bit 1).
template <typename T>
__global__ void k_p(long N, T* __restrict__ p, const T* __restrict__ z, const VecState* __restrict__ vs,
                    const CellState* __restrict__ cs, int m, int init) {
  const int vec = blockIdx.z, c = blockIdx.y;
  if (cs && !(cs[vec / m].status & 2)) return;
  const T be = (T)vs[vec].beta, mu = (T)vs[vec].mean[c];
  const long off = ((long)vec * 3 + c) * N;
  if (init) {  // p is not read: it holds stale workspace contents
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
      p[off + i] = z[off + i] - mu;
  } else {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
      p[off + i] = (z[off + i] - mu) + be * p[off + i];
  }
}

// Fused form of k_fin_pc for an iteration whose preconditioner passes also updated r:
//   partA [vec][3][n0][2]: sum r, (r, r) of the updated residual (FFT pass A)
//   partB [vec][n1][nchunk]: Parseval partials of (r, z) on the half spectrum, unnormalised (pass B)
//   partC [vec][3][n0]: sum z (pass C), or null when pass C runs after this kernel (fused x/p update, z not
//   projected)
// rz1 = (r, z - mean z) = (r, z) - sum_c mean z_c sum r_c (partC null: rz1 = (r, z)); the control is that of
// k_fin_pc.
__global__ void k_fin_pc_fused(const double* __restrict__ partA, const double* __restrict__ partB,
                               const double* __restrict__ partC, int nchunk, int n0, int n1, long N,
                               VecState* __restrict__ vs, CellState* __restrict__ cs, int m, double tol, int maxit,
                               double* __restrict__ ring, double etol, int probation) {
  __shared__ double s_nc[8], s_w[8];
  __shared__ int s_res[8];
  const int cell = blockIdx.x;
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (!cs[cell].active) return;
  const int itk = cs[cell].it;  // index of the iteration that just ran
  const int stopped = cs[cell].stopped;
  if (wid < m) {
    const int vec = cell * m + wid;
    if ((stopped >> wid) & 1) {
      // a case that stopped on its own keeps its state; it counts as holding both rules, and its error-energy
      // base N C_II enters the cell's scale as before
      if (lane == 0) {
        s_res[wid] = 1;
        s_w[wid] = 0.0;
        s_nc[wid] = vs[vec].ebase - vs[vec].esum;
      }
    } else {
      double sr[3] = {0, 0, 0}, sz[3] = {0, 0, 0}, rr = 0.0, dot = 0.0;
      for (int c = 0; c < 3; ++c)
        for (int x = lane; x < n0; x += 32) {
          const long i = ((long)vec * 3 + c) * n0 + x;
          sr[c] += partA[2 * i];
          rr += partA[2 * i + 1];
          if (partC) sz[c] += partC[i];
        }
      for (int i = lane; i < n1 * nchunk; i += 32) dot += partB[(long)vec * n1 * nchunk + i];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          sr[c] += __shfl_down_sync(0xffffffffu, sr[c], o);
          sz[c] += __shfl_down_sync(0xffffffffu, sz[c], o);
        }
        rr += __shfl_down_sync(0xffffffffu, rr, o);
        dot += __shfl_down_sync(0xffffffffu, dot, o);
      }
      if (etol > 0.0) {
        // energy rule: the error energy ||x* - x_k||_K^2 = sum_{j >= k} alpha_j (r_j, z_j) (Hestenes-Stiefel),
        // estimated by the last kEnergyWindow terms; N C_II(x_k) = ebase - esum
        const double term = vs[vec].alpha * vs[vec].rz;
        double* rg = ring + (long)vec * kEnergyWindow;
        const int nw = min(itk + 1, kEnergyWindow), slot = itk % kEnergyWindow;
        double w = (lane < nw && lane != slot) ? rg[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
        if (lane == 0) {
          rg[slot] = term;
          VecState& v = vs[vec];
          v.esum += term;
          s_w[wid] = w + term;
          s_nc[wid] = v.ebase - v.esum;
        }
      }
      if (lane == 0) {
        VecState& v = vs[vec];
        double rz1 = dot / (double)N;
        if (partC)
          for (int c = 0; c < 3; ++c) {
            const double mz = sz[c] / (double)N;
            v.mean[c] = mz;
            rz1 -= mz * sr[c];
          }
        v.beta = rz1 / (v.rz == 0.0 ? 1.0 : v.rz);
        v.rz = rz1;
        v.rr = rr;
        s_res[wid] = sqrt(rr) <= tol * v.bn;
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // the energy rule of case I: its window sum at most etol times the cell's largest N C_JJ (after a full window)
    bool eok[8];
    double cmax = 0.0;
    for (int I = 0; I < m; ++I) cmax = fmax(cmax, s_nc[I]);
    for (int I = 0; I < m; ++I)
      eok[I] = etol <= 0.0 || (itk + 1 >= kEnergyWindow && cmax > 0.0 && s_w[I] <= etol * cmax);
    bool go = false, eall = true;
    for (int I = 0; I < m; ++I) {
      go = go || !s_res[I];
      eall = eall && eok[I];
    }
    CellState& s = cs[cell];
    int stop = stopped;
    if (probation > 0)
      for (int I = 0; I < m; ++I) {
        if ((stopped >> I) & 1) continue;
        VecState& v = vs[cell * m + I];
        v.streak = (s_res[I] && eok[I]) ? v.streak + 1 : 0;
        if (v.streak >= probation) stop |= 1 << I;
      }
    s.stopped = stop;
    s.it += 1;
    // lock-step: the cell stops when every case meets the residual rule and (with the energy guard) the energy
    // rule in the same iteration; with per-case stopping also when every case has stopped on its own
    s.active = (s.it < maxit) && (go || (etol > 0.0 && !eall)) && stop != (1 << m) - 1;
  }
}

// ebase[vec] = ede[I] * sum(s of the cell), esum = 0; one block per cell
template <typename T>
__global__ void k_energy_base(const T* __restrict__ s, long N, int m, Ede ede, VecState* __restrict__ vs,
                              const CellState* __restrict__ cs) {
  __shared__ double red[32];
  const int cell = blockIdx.x;
  if (cs && !cs[cell].active) return;
  double acc[1] = {0.0};
  for (long i = threadIdx.x; i < N; i += blockDim.x) acc[0] += (double)s[(long)cell * N + i];
  block_sum<1>(acc, red);
  if (threadIdx.x == 0)
    for (int I = 0; I < m; ++I) {
      vs[cell * m + I].ebase = ede.v[I] * acc[0];
      vs[cell * m + I].esum = 0.0;
    }
}

// ebase += x0.K x0 - 2 (b, x0) from the k_x0_dots partials
__global__ void k_energy_x0(const double* __restrict__ partial, int nb, int nvec, VecState* __restrict__ vs,
                            const CellState* __restrict__ cs, int m) {
  const int vec = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (vec >= nvec) return;
  if (cs && !cs[vec / m].active) return;
  double bx = 0.0, xax = 0.0;
  for (int k = lane; k < 3 * nb; k += 32) {
    bx += partial[((long)vec * 3 * nb + k) * 2];
    xax += partial[((long)vec * 3 * nb + k) * 2 + 1];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    bx += __shfl_down_sync(0xffffffffu, bx, o);
    xax += __shfl_down_sync(0xffffffffu, xax, o);
  }
  if (lane == 0) vs[vec].ebase += xax - 2.0 * bx;
}

// x += alpha p; p = (z - mean z) + beta p, for the cells that ran this iteration (status bit 1)
template <typename T>
__global__ void k_px(long N, T* __restrict__ x, T* __restrict__ p, const T* __restrict__ z,
                     const VecState* __restrict__ vs, const CellState* __restrict__ cs, int m) {
  const int vec = blockIdx.z, c = blockIdx.y;
  if (cs && !(cs[vec / m].status & 2)) return;
  const T al = (T)vs[vec].alpha, be = (T)vs[vec].beta, mu = (T)vs[vec].mean[c];
  const long off = ((long)vec * 3 + c) * N;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const T po = p[off + i];
    x[off + i] += al * po;
    p[off + i] = (z[off + i] - mu) + be * po;
  }
}

// ---- energy-optimal scaling of an initial guess ------------------------------------------------------------
// partial[vec][c][blk] = ((b, x), (x, Ax - mean Ax)) over the block's share of component c
template <typename Tb, typename T>
__global__ void k_x0_dots(long N, const Tb* __restrict__ b, const T* __restrict__ x, const T* __restrict__ Ax,
                          const VecState* __restrict__ vs, const CellState* __restrict__ cs, int m,
                          double* __restrict__ partial) {
  __shared__ double red[32 * 2];
  const int c = blockIdx.y, vec = blockIdx.z;
  if (cs && !cs[vec / m].active) return;
  const long off = ((long)vec * 3 + c) * N;
  const double mu = vs[vec].mean[c];
  double acc[2] = {0.0, 0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const double xv = (double)x[off + i];
    acc[0] += (double)b[off + i] * xv;
    acc[1] += xv * ((double)Ax[off + i] - mu);
  }
  block_sum<2>(acc, red);
  if (threadIdx.x == 0) {
    double* o = partial + (((long)vec * 3 + c) * gridDim.x + blockIdx.x) * 2;
    o[0] = acc[0];
    o[1] = acc[1];
  }
}

__global__ void k_x0_fin(const double* __restrict__ partial, int nb, int nvec, VecState* __restrict__ vs,
                         const CellState* __restrict__ cs, int m) {
  const int vec = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (vec >= nvec) return;
  if (cs && !cs[vec / m].active) return;
  double bx = 0.0, xax = 0.0;
  for (int k = lane; k < 3 * nb; k += 32) {
    bx += partial[((long)vec * 3 * nb + k) * 2];
    xax += partial[((long)vec * 3 * nb + k) * 2 + 1];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    bx += __shfl_down_sync(0xffffffffu, bx, o);
    xax += __shfl_down_sync(0xffffffffu, xax, o);
  }
  if (lane == 0) {
    const double beta = (xax > 0.0 && isfinite(bx / xax)) ? bx / xax : 0.0;
    VecState& v = vs[vec];
    v.x0scale = beta;
    v.mean[0] *= beta;
    v.mean[1] *= beta;
    v.mean[2] *= beta;
  }
}

template <typename T>
__global__ void k_x0_apply(long N, T* __restrict__ x, T* __restrict__ Ax, const VecState* __restrict__ vs,
                           const CellState* __restrict__ cs, int m) {
  const int vec = blockIdx.z, c = blockIdx.y;
  if (cs && !cs[vec / m].active) return;
  const T be = (T)vs[vec].x0scale;
  const long off = ((long)vec * 3 + c) * N;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    x[off + i] *= be;
    Ax[off + i] *= be;
  }
}

// status bit 1 <- active (marks the cells that run the current iteration, for k_p after k_fin_pc)
__global__ void k_mark(CellState* cs, int ncell) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < ncell) {
    const int live = cs[c].active ? (2 | (((~cs[c].stopped) & 0x3F) << 4)) : 0;
    cs[c].status = (cs[c].status & ~(2 | (0x3F << 4))) | live;
  }
}

__global__ void k_cs_init(CellState* cs, int ncell, const int* __restrict__ mask) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < ncell) {
    cs[c].it = 0;
    cs[c].active = mask ? mask[c] : 1;
    cs[c].status = cs[c].active ? (2 | (0x3F << 4)) : 0;
    cs[c].stopped = 0;
  }
}

__global__ void k_count_active(const CellState* __restrict__ cs, int ncell, int* __restrict__ out) {
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  int local = 0;
  for (int c = threadIdx.x; c < ncell; c += blockDim.x) local += cs[c].active ? 1 : 0;
  atomicAdd(&cnt, local);
  __syncthreads();
  if (threadIdx.x == 0) *out = cnt;
}

// ---- mixed precision refinement -----------------------------------------------------------------------------
// scale = sqrt(rr) (1 if 0); r32 = r64 / scale
__global__ void k_r_to32(long N, const double* __restrict__ r64, float* __restrict__ r32, VecState* __restrict__ vs,
                         const CellState* __restrict__ cs, int m) {
  const int vec = blockIdx.z, c = blockIdx.y;
  if (cs && !cs[vec / m].active) return;
  const double rr = vs[vec].rr;
  const double sc = rr > 0.0 ? sqrt(rr) : 1.0;
  if (blockIdx.x == 0 && threadIdx.x == 0 && c == 0) vs[vec].scale = sc;
  const double inv = 1.0 / sc;
  const long off = ((long)vec * 3 + c) * N;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
    r32[off + i] = (float)(r64[off + i] * inv);
}

// x64 += scale * x32
__global__ void k_x_update(long N, double* __restrict__ x64, const float* __restrict__ x32,
                           const VecState* __restrict__ vs, const CellState* __restrict__ cs, int m) {
  const int vec = blockIdx.z, c = blockIdx.y;
  if (cs && !cs[vec / m].active) return;
  const double sc = vs[vec].scale;
  const long off = ((long)vec * 3 + c) * N;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
    x64[off + i] += sc * (double)x32[off + i];
}

// ---- launch helpers ----------------------------------------------------------------------------------------
static inline dim3 vec_grid(long N, int nvec) {
  return dim3((unsigned)std::min<long>((N + 255) / 256, 512), 3, nvec);
}

int launch_fin_apply(int nvec, int m, const double* partial, int nblk, long N, VecState* vs, const CellState* cs,
                     int init, cudaStream_t st) {
  ProfScope ps_(PK_FIN, st);
  k_fin_apply<<<(nvec + 7) / 8, 256, 0, st>>>(partial, nblk, N, nvec, vs, cs, m, init);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}
template <typename Tb, typename T>
int launch_r_init(long N, int nvec, int m, T* r, const Tb* b, const T* Ax, const VecState* vs, const CellState* cs,
                  cudaStream_t st) {
  ProfScope ps_(PK_OTHER, st);
  k_r_init<Tb, T><<<vec_grid(N, nvec), 256, 0, st>>>(N, r, b, Ax, vs, cs, m);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}
int launch_fin_pc(int ncell, int m, int n0, long N, const double* partial, VecState* vs, CellState* cs, double tol,
                  int maxit, int init, cudaStream_t st) {
  ProfScope ps_(PK_FIN, st);
  k_fin_pc<<<ncell, 32 * m, 0, st>>>(partial, n0, N, vs, cs, m, tol, maxit, init);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}
template <typename T>
int launch_p(long N, int nvec, int m, T* p, const T* z, const VecState* vs, const CellState* cs, int init,
             cudaStream_t st) {
  ProfScope ps_(PK_P, st);
  k_p<T><<<vec_grid(N, nvec), 256, 0, st>>>(N, p, z, vs, cs, m, init);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}
int launch_fin_pc_fused(int ncell, int m, int n0, int n1, long N, const double* partA, const double* partB,
                        const double* partC, int nchunk, VecState* vs, CellState* cs, double tol, int maxit,
                        double* ring, double etol, int probation, cudaStream_t st) {
  ProfScope ps_(PK_FIN, st);
  k_fin_pc_fused<<<ncell, 32 * m, 0, st>>>(partA, partB, partC, nchunk, n0, n1, N, vs, cs, m, tol, maxit, ring,
                                           etol, probation);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}
template <typename T>
int launch_px(long N, int nvec, int m, T* x, T* p, const T* z, const VecState* vs, const CellState* cs,
              cudaStream_t st) {
  ProfScope ps_(PK_P, st);
  k_px<T><<<vec_grid(N, nvec), 256, 0, st>>>(N, x, p, z, vs, cs, m);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}
template int launch_px<float>(long, int, int, float*, float*, const float*, const VecState*, const CellState*,
                              cudaStream_t);
template int launch_px<double>(long, int, int, double*, double*, const double*, const VecState*, const CellState*,
                               cudaStream_t);
template <typename Tb, typename T>
int launch_x0_scale(const LinearHandle& h, int nvec, int m, const Tb* b, T* x, T* Ax, const CellState* cs,
                    double* partial, VecState* vs, cudaStream_t st) {
  const long N = h.g.N;
  ProfScope ps_(PK_OTHER, st);
  k_x0_dots<Tb, T><<<dim3(kStatsBlocks, 3, nvec), 256, 0, st>>>(N, b, x, Ax, vs, cs, m, partial);
  NLF_CHECK_LAUNCH();
  k_x0_fin<<<(nvec + 7) / 8, 256, 0, st>>>(partial, kStatsBlocks, nvec, vs, cs, m);
  NLF_CHECK_LAUNCH();
  k_x0_apply<T><<<vec_grid(N, nvec), 256, 0, st>>>(N, x, Ax, vs, cs, m);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}
template int launch_x0_scale<double, double>(const LinearHandle&, int, int, const double*, double*, double*,
                                             const CellState*, double*, VecState*, cudaStream_t);
template int launch_x0_scale<float, float>(const LinearHandle&, int, int, const float*, float*, float*,
                                           const CellState*, double*, VecState*, cudaStream_t);
template <typename Tb, typename T>
int launch_energy_init(const LinearHandle& h, int ncell, int m, const T* s, const Ede& ede, const Tb* b, const T* x,
                       const T* Ax, bool x_given, const CellState* cs, double* partial, VecState* vs,
                       cudaStream_t st) {
  const long N = h.g.N;
  const int nvec = ncell * m;
  ProfScope ps_(PK_OTHER, st);
  k_energy_base<T><<<ncell, 512, 0, st>>>(s, N, m, ede, vs, cs);
  NLF_CHECK_LAUNCH();
  if (x_given) {
    k_x0_dots<Tb, T><<<dim3(kStatsBlocks, 3, nvec), 256, 0, st>>>(N, b, x, Ax, vs, cs, m, partial);
    NLF_CHECK_LAUNCH();
    k_energy_x0<<<(nvec + 7) / 8, 256, 0, st>>>(partial, kStatsBlocks, nvec, vs, cs, m);
    NLF_CHECK_LAUNCH();
  }
  return NLF_OK;
}
template int launch_energy_init<double, double>(const LinearHandle&, int, int, const double*, const Ede&,
                                                const double*, const double*, const double*, bool, const CellState*,
                                                double*, VecState*, cudaStream_t);
template int launch_energy_init<float, float>(const LinearHandle&, int, int, const float*, const Ede&, const float*,
                                              const float*, const float*, bool, const CellState*, double*, VecState*,
                                              cudaStream_t);
int launch_mark(CellState* cs, int ncell, cudaStream_t st) {
  ProfScope ps_(PK_OTHER, st);
  k_mark<<<(ncell + 127) / 128, 128, 0, st>>>(cs, ncell);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}
int launch_cs_init(CellState* cs, int ncell, const int* mask, cudaStream_t st) {
  ProfScope ps_(PK_OTHER, st);
  k_cs_init<<<(ncell + 127) / 128, 128, 0, st>>>(cs, ncell, mask);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}
int launch_count_active(const CellState* cs, int ncell, int* out, cudaStream_t st) {
  ProfScope ps_(PK_OTHER, st);
  k_count_active<<<1, 256, 0, st>>>(cs, ncell, out);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}
int launch_r_to32(long N, int nvec, int m, const double* r64, float* r32, VecState* vs, const CellState* cs,
                  cudaStream_t st) {
  ProfScope ps_(PK_OTHER, st);
  k_r_to32<<<vec_grid(N, nvec), 256, 0, st>>>(N, r64, r32, vs, cs, m);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}
int launch_x_update(long N, int nvec, int m, double* x64, const float* x32, const VecState* vs, const CellState* cs,
                    cudaStream_t st) {
  ProfScope ps_(PK_OTHER, st);
  k_x_update<<<vec_grid(N, nvec), 256, 0, st>>>(N, x64, x32, vs, cs, m);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}

template int launch_r_init<double, double>(long, int, int, double*, const double*, const double*, const VecState*,
                                           const CellState*, cudaStream_t);
template int launch_r_init<float, float>(long, int, int, float*, const float*, const float*, const VecState*,
                                         const CellState*, cudaStream_t);
template int launch_p<float>(long, int, int, float*, const float*, const VecState*, const CellState*, int,
                             cudaStream_t);
template int launch_p<double>(long, int, int, double*, const double*, const VecState*, const CellState*, int,
                              cudaStream_t);

}  // namespace nlf
