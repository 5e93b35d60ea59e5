// Internal declarations of the nlfiber-b200 library: the linear handle, its workspace and the launchers.
#pragma once
#include <vector>
#include "nlf_common.cuh"
#include "nlf_element.cuh"
#include "../../include/nlf.h"

namespace nlf {

// Grid geometry of one handle. N = n0 * n1 * n2; the half spectrum has n2h = n2 / 2 + 1 z-frequencies.
struct Geom {
  int n0, n1, n2;  // x (slowest), y, z (fastest)
  int n2h;         // n2 / 2 + 1
  long N;          // voxels
  long NS;         // half-spectrum entries per component: n0 * n1 * n2h
};

// FP64 scalars of one PCG vector (one cell and load case).
struct VecState {
  double bn;       // ||b|| + 1e-300
  double rz;       // (r, z)
  double alpha, beta;
  double rr;       // (r, r)
  double scale;    // refinement scale of the right-hand side (mixed precision)
  double mean[3];  // per-component mean for the next projection
  double x0scale;  // energy-optimal multiple of the initial guess (scale_x0)
  double ebase;    // N C_II at the start: (E D E) sum(s) + x0.K x0 - 2 (b, x0)   (energy stopping rule)
  double esum;     // sum over the iterations so far of alpha_j (r_j, z_j)
  int streak;      // per-case stopping: consecutive iterations in which this case met both stopping rules
  int pad_;
};

// energy stopping rule: E_I D E_I of the cases (m <= 6) and the window of alpha (r, z) terms it sums
struct Ede {
  double v[6];
};
constexpr int kEnergyWindow = 32;

// apply partial sums: at most this many blocks (tiles x x-chunks) per vector
constexpr int kApplyMaxBlocks = 4096;

// exponent of the node scaling of the scaled preconditioner, w = S^-kNodeScaleExp
constexpr double kNodeScaleExp = 0.47;

// Poisson ratio of the reference medium whose FFT inverse the scaled preconditioner wraps (its Young's modulus
// does not matter: PCG is invariant to scaling the preconditioner). The unscaled preconditioner keeps the
// material's own (E, nu), as the reference does.
constexpr double kScaledRefNu = 0.0;

// Per-cell PCG control. `active` follows the reference's lock-step cond (nlfiber/linear.py:185-188). With
// per-case stopping, `stopped` has bit I set once load case I stopped on its own; `status` bit 1 says the cell
// runs the current iteration, bit 4 + I that case I does (both set by the mark at the start of the iteration).
struct CellState {
  int it;
  int active;
  int status;
  int stopped;
};

// vector vec = cell m + case takes part in the current iteration (its cell is active, the case has not stopped)
__host__ __device__ inline bool vec_live(const CellState* cs, int vec, int m) {
  if (!cs) return true;
  const CellState& c = cs[vec / m];
  return c.active && !((c.stopped >> (vec % m)) & 1);
}
// vector vec ran the current iteration (marked live at its start)
__host__ __device__ inline bool vec_ran(const CellState* cs, int vec, int m) {
  return !cs || ((cs[vec / m].status >> (4 + vec % m)) & 1);
}

// Grow-only device buffer.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  int reserve(size_t n);
  void release();
};

template <typename T>
struct Tables {
  T* kinv = nullptr;     // (n0, n1, n2h, 6)
  cplx<T>* tw = nullptr;  // twiddles, see tw_off
};

struct Twiddle {
  int off0, off1, off2, off2h;  // offsets of the length-n0, n1, n2, n2/2 tables (each of its length)
  int total;
};

struct LinearHandle {
  Geom g;
  double E, nu, emin, p, tol, lam, mu;
  int maxit;
  double Ke[24][24];
  double Gm[6][24];
  double Dm[6][6];
  double W27[27][9];  // unit-stiffness stencil blocks W_d, d = (dx+1)*9 + (dy+1)*3 + (dz+1)
  double W27s[27][9];  // the same for the scaled preconditioner's reference medium (Poisson ratio scaled_ref_nu)
  double scaled_ref_nu = kScaledRefNu;
  Twiddle tw;
  Tables<double> t64;
  Tables<float> t32;
  Tables<double> t64s;  // Kinv of the scaled preconditioner's reference medium (twiddles shared with t64)
  Tables<float> t32s;
  DevBuf ws;          // solver workspace
  DevBuf io;          // staging for host <-> device copies
  DevBuf io2;
  DevBuf part;        // reduction partials
  DevBuf kinv_rgb;    // spare
  int dev = 0;
  int nsm = 148;
  int smem_optin = 0;
  // CUDA graph replay of PCG iterations: captured and launched on a handle-owned stream ordered after the
  // caller's stream by events (capture is not possible on the legacy default stream)
  cudaStream_t gst = nullptr;
  cudaEvent_t gev[2] = {nullptr, nullptr};
  // apply tile variant per precision ([0] FP32, [1] FP64); 0 = default, set by nlf_linear_autotune
  int apply_variant[2] = {0, 0};
  // FP64 cube pass B: 1 = Kinv entries in closed form (no table reads), 0 = from the table
  int pcb_closed = 0;
  // FP64 cube passes A and C: 0 = twiddles in registers (2 CTAs per SM), 1 = from shared memory (3 per SM),
  // 2 = as 1 with pass C's spectrum rows staged through shared memory and its x/p update in whole rows
  // (coalesced), 3 = as 2 with pass A's row inputs coalesced too
  int fft_smt = 0;
};

// ---- launchers (all asynchronous on `st`) ----
// element operator
template <typename T>
int launch_apply(const LinearHandle& h, const T* s, int m, int nvec, const T* x, T* y,
                 const CellState* cs, double* partial, int* nblk_out, cudaStream_t st);
// tile variants of the apply: how many there are, and the tile (TY, TZ, minimum CTAs per SM) of variant v
int apply_variants(bool fp64);
void apply_variant_tile(bool fp64, int v, int* ty, int* tz, int* minb);
int launch_load(const LinearHandle& h, const double* s, const double* fe /*(m,24) on device*/, int m,
                int ncell, double* f, double sign, cudaStream_t st);
int launch_bilinear(const LinearHandle& h, const double* s, const double* Es /*device (m,6)*/, int m,
                    int ncell, const double* u, double* Cpart, int* nblk, const double* rho, double* dC,
                    cudaStream_t st);
// sbar_e = sum_I lam_I,e . (Ke u_I,e + G^T E_I) (times ds/drho when rho is given); Es device (m, 6); u, lam SoA
int launch_adjoint_sbar(const LinearHandle& h, const double* Es, int m, int ncell, const double* u,
                        const double* lamv, const double* rho, double* out, cudaStream_t st);
int launch_reduce_C(const LinearHandle& h, const double* Cpart, int nblk, int m, int ncell, double* C,
                    cudaStream_t st);

// FFT preconditioner: z = w .* irfftn(Kinv rfftn(w .* r)) (w == nullptr: unscaled)
template <typename T>
int launch_precond(const LinearHandle& h, int nvec, int m, const T* r, T* z, cplx<T>* spec, const T* w,
                   const CellState* cs, double* partial /*[nvec][3][n0][4]: sum z, (r,z), sum r, (r,r)*/,
                   cudaStream_t st);
// The same transform inside a PCG iteration, fused with the neighbouring vector work: pass A first updates
// r <- r - alpha (Ap - mean Ap) in place and writes partA [nvec][3][n0][2] (sum r, (r, r)); pass B writes the
// Parseval partials of (r, z) to partB [nvec][n1][nchunk]; pass C writes sum z to partC [nvec][3][n0].
template <typename T>
int launch_precond_pcg(const LinearHandle& h, int nvec, int m, T* r, const T* Ap, const VecState* vs, T* z,
                       cplx<T>* spec, const T* w, const CellState* cs, double* partA, double* partB, double* partC,
                       int* nchunk, cudaStream_t st);
// FP64 grids with register-resident passes (cubes of 32 and 64) split the fused iteration around the control:
// passes A and B as in launch_precond_pcg; then, once beta is known, pass C transforms back and, instead of
// writing z, updates x <- x + alpha p and p <- z + beta p for the cells that ran this iteration. z is not
// projected, so p and x pick up per-component constants; K annihilates constants, so alpha, beta and r are
// those of the projected iteration, and the caller projects x when the solve ends.
bool precond_fuses_px(const LinearHandle& h);
int launch_precond_pcg_ab(const LinearHandle& h, int nvec, int m, double* r, const double* Ap, const VecState* vs,
                          cplx<double>* spec, const double* w, const CellState* cs, double* partA, double* partB,
                          int* nchunk, cudaStream_t st);
int launch_precond_pcg_cpx(const LinearHandle& h, int nvec, int m, cplx<double>* spec, const double* w,
                           const VecState* vs, const CellState* cs, double* x, double* p, cudaStream_t st);
int build_tables(LinearHandle& h);
int kinv_tables(const LinearHandle& h, const double (&W)[27][9], double* k64, float* k32);
// Rebuild the scaled preconditioner's Kinv tables for a reference medium of Poisson ratio nu (the handle's
// element, unit stiffness). The finite-strain solver uses the material's own nu there.
int rebuild_scaled_kinv(LinearHandle& h, double nu);

// stiffness scale only (s = emin + (1 - emin) clip01(rho)^p)
int launch_stiffness_scale(const LinearHandle& h, long count, const double* rho, double* s, cudaStream_t st);

template <typename Tin, typename Tout>
int launch_aos_to_soa(long N, int nvec, const Tin* in, Tout* out, double scale, cudaStream_t st);
template <typename Tin, typename Tout>
int launch_soa_to_aos(long N, int nvec, const Tin* in, Tout* out, cudaStream_t st);

}  // namespace nlf
