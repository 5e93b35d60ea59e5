// Finite-strain periodic homogenization (nlfiber/mech.py): energy, residual, mean stress, matrix-free tangent
// matvec and the preconditioned CG of the Newton step, on the GPU in FP64.
//
// The reference gets the residual by autodiff of the energy and stores the Gauss-point tangent, 648 doubles per
// element (mech.py:154-169,227-238). Here the first Piola stress P = d psi_eff / dF and the tangent action
// dP = d2 psi_eff / dF dF : dF are closed forms evaluated at each of the 8 Gauss points from the state, so a
// tangent matvec reads the state and the direction and nothing else:
//   psi_eff(F) = psi(F_g) - psi_lin(F_g) + psi_lin(F),   F_g = I + gamma (F - I)       (mech.py:134-139)
//   P_eff      = gamma (P(F_g) - sig_lin(F_g)) + sig_lin(F)
//   dP_eff     = gamma^2 (dP(F_g; dF) - dsig_lin(dF)) + dsig_lin(dF)
//   neo-Hookean: P = mu (F - F^-T) + lam lnJ F^-T,
//                dP = mu dF + (mu - lam lnJ) F^-T dF^T F^-T + lam (F^-T : dF) F^-T.
// Element forces go to a [24][N] buffer; a gather kernel sums the 8 contributions of each node in a fixed order.
// Inside the Newton step's CG the state is fixed, so the CG computes the state-dependent part of dP once per solve
// (k_mech_tan_cache: F_g^-T and mu - lam ln det F_g at every Gauss point, 80 doubles per element) and its matvec
// (k_mech_hvp_tc) reads that instead of recomputing F, the inverse and the log; it also takes the direction's
// gradients and forces in the element's mode form, and sums dP only at the free macro entries.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>
#include "nlf_element.cuh"
#include "nlf_vec.cuh"
#include "nlf_prof.cuh"

namespace nlf {

__constant__ double cDN[8][8][3];  // shape-function gradients [gauss][node][dim] (nlfiber/linear.py:33-41)

struct MechDev {
  int n0, n1, n2;
  long N;
  double lam, mu, wq;
  int material;  // 0 linear, 1 neo-Hookean
  int use_gamma;
  const double* s;
  const double* gamma;
};

// ---- material laws ---------------------------------------------------------------------------------------------
__device__ __forceinline__ double det3(const double (&F)[9]) {
  return F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) +
         F[2] * (F[3] * F[7] - F[4] * F[6]);
}

// G = F^-T = cof(F) / det F
__device__ __forceinline__ void inv_t3(const double (&F)[9], double J, double (&G)[9]) {
  const double iJ = 1.0 / J;
  G[0] = (F[4] * F[8] - F[5] * F[7]) * iJ;
  G[1] = -(F[3] * F[8] - F[5] * F[6]) * iJ;
  G[2] = (F[3] * F[7] - F[4] * F[6]) * iJ;
  G[3] = -(F[1] * F[8] - F[2] * F[7]) * iJ;
  G[4] = (F[0] * F[8] - F[2] * F[6]) * iJ;
  G[5] = -(F[0] * F[7] - F[1] * F[6]) * iJ;
  G[6] = (F[1] * F[5] - F[2] * F[4]) * iJ;
  G[7] = -(F[0] * F[5] - F[2] * F[3]) * iJ;
  G[8] = (F[0] * F[4] - F[1] * F[3]) * iJ;
}

__device__ __forceinline__ double psi_lin(const double (&F)[9], double lam, double mu) {
  const double e0 = F[0] - 1.0, e1 = F[4] - 1.0, e2 = F[8] - 1.0;
  const double e01 = 0.5 * (F[1] + F[3]), e02 = 0.5 * (F[2] + F[6]), e12 = 0.5 * (F[5] + F[7]);
  const double tr = e0 + e1 + e2;
  return 0.5 * lam * tr * tr + mu * (e0 * e0 + e1 * e1 + e2 * e2 + 2.0 * (e01 * e01 + e02 * e02 + e12 * e12));
}

// P += c * sig_lin(F) (sym gradient of F - I)
__device__ __forceinline__ void add_sig_lin(const double (&F)[9], double lam, double mu, double c, double (&P)[9]) {
  const double tr = lam * (F[0] + F[4] + F[8] - 3.0);
  P[0] += c * (tr + 2.0 * mu * (F[0] - 1.0));
  P[4] += c * (tr + 2.0 * mu * (F[4] - 1.0));
  P[8] += c * (tr + 2.0 * mu * (F[8] - 1.0));
  const double s01 = mu * (F[1] + F[3]), s02 = mu * (F[2] + F[6]), s12 = mu * (F[5] + F[7]);
  P[1] += c * s01;
  P[3] += c * s01;
  P[2] += c * s02;
  P[6] += c * s02;
  P[5] += c * s12;
  P[7] += c * s12;
}

// dP += c * dsig_lin(dF)
__device__ __forceinline__ void add_dsig_lin(const double (&d)[9], double lam, double mu, double c, double (&P)[9]) {
  const double tr = lam * (d[0] + d[4] + d[8]);
  P[0] += c * (tr + 2.0 * mu * d[0]);
  P[4] += c * (tr + 2.0 * mu * d[4]);
  P[8] += c * (tr + 2.0 * mu * d[8]);
  const double s01 = mu * (d[1] + d[3]), s02 = mu * (d[2] + d[6]), s12 = mu * (d[5] + d[7]);
  P[1] += c * s01;
  P[3] += c * s01;
  P[2] += c * s02;
  P[6] += c * s02;
  P[5] += c * s12;
  P[7] += c * s12;
}

__device__ __forceinline__ double psi_nh(const double (&F)[9], double lam, double mu) {
  const double J = det3(F);
  double I1 = 0.0;
#pragma unroll
  for (int q = 0; q < 9; ++q) I1 += F[q] * F[q];
  const double lnJ = log(J);  // NaN for J <= 0, as the reference's jnp.log
  return 0.5 * mu * (I1 - 3.0) - mu * lnJ + 0.5 * lam * lnJ * lnJ;
}

__device__ __forceinline__ void add_P_nh(const double (&F)[9], double lam, double mu, double c, double (&P)[9]) {
  const double J = det3(F);
  double G[9];
  inv_t3(F, J, G);
  const double lnJ = log(J);
#pragma unroll
  for (int q = 0; q < 9; ++q) P[q] += c * (mu * (F[q] - G[q]) + lam * lnJ * G[q]);
}

// dP += c (mu dF + cm G dF^T G + lam (G : dF) G) with G = F^-T and cm = mu - lam lnJ given (the tangent cache of
// the CG holds them per Gauss point; add_dP_nh computes them from F)
__device__ __forceinline__ void add_dP_nh_g(const double (&G)[9], double cm, const double (&d)[9], double lam,
                                            double mu, double c, double (&P)[9]) {
  double GdF = 0.0;
#pragma unroll
  for (int q = 0; q < 9; ++q) GdF += G[q] * d[q];
  // T = G dF^T G: T_ij = sum_kl G_ik dF_lk G_lj
  double M[9];  // M = G dF^T: M_il = sum_k G_ik dF_lk
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int l = 0; l < 3; ++l) M[i * 3 + l] = G[i * 3] * d[l * 3] + G[i * 3 + 1] * d[l * 3 + 1] + G[i * 3 + 2] * d[l * 3 + 2];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const double T = M[i * 3] * G[j] + M[i * 3 + 1] * G[3 + j] + M[i * 3 + 2] * G[6 + j];
      P[i * 3 + j] += c * (mu * d[i * 3 + j] + cm * T + lam * GdF * G[i * 3 + j]);
    }
}

// G = F^-T and cm = mu - lam ln det F
__device__ __forceinline__ void nh_point(const double (&F)[9], double lam, double mu, double (&G)[9], double& cm) {
  const double J = det3(F);
  inv_t3(F, J, G);
  cm = mu - lam * log(J);
}

__device__ __forceinline__ void add_dP_nh(const double (&F)[9], const double (&d)[9], double lam, double mu,
                                          double c, double (&P)[9]) {
  double G[9], cm;
  nh_point(F, lam, mu, G, cm);
  add_dP_nh_g(G, cm, d, lam, mu, c, P);
}

// psi_eff, P_eff, dP_eff (mech.py:134-139) at one Gauss point, scaled by c = wq s
__device__ __forceinline__ double psi_eff(const MechDev& a, const double (&F)[9], double gam) {
  if (a.material == 0) return psi_lin(F, a.lam, a.mu);
  if (!a.use_gamma) return psi_nh(F, a.lam, a.mu);
  double Fg[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) Fg[q] = (q % 4 == 0 ? 1.0 : 0.0) + gam * (F[q] - (q % 4 == 0 ? 1.0 : 0.0));
  return psi_nh(Fg, a.lam, a.mu) - psi_lin(Fg, a.lam, a.mu) + psi_lin(F, a.lam, a.mu);
}

__device__ __forceinline__ void add_P_eff(const MechDev& a, const double (&F)[9], double gam, double c,
                                          double (&P)[9]) {
  if (a.material == 0) {
    add_sig_lin(F, a.lam, a.mu, c, P);
    return;
  }
  if (!a.use_gamma) {
    add_P_nh(F, a.lam, a.mu, c, P);
    return;
  }
  double Fg[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) Fg[q] = (q % 4 == 0 ? 1.0 : 0.0) + gam * (F[q] - (q % 4 == 0 ? 1.0 : 0.0));
  add_P_nh(Fg, a.lam, a.mu, c * gam, P);
  add_sig_lin(Fg, a.lam, a.mu, -c * gam, P);
  add_sig_lin(F, a.lam, a.mu, c, P);
}

__device__ __forceinline__ void add_dP_eff(const MechDev& a, const double (&F)[9], const double (&d)[9], double gam,
                                           double c, double (&P)[9]) {
  if (a.material == 0) {
    add_dsig_lin(d, a.lam, a.mu, c, P);
    return;
  }
  if (!a.use_gamma) {
    add_dP_nh(F, d, a.lam, a.mu, c, P);
    return;
  }
  double Fg[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) Fg[q] = (q % 4 == 0 ? 1.0 : 0.0) + gam * (F[q] - (q % 4 == 0 ? 1.0 : 0.0));
  add_dP_nh(Fg, d, a.lam, a.mu, c * gam * gam, P);
  add_dsig_lin(d, a.lam, a.mu, c * (1.0 - gam * gam), P);
}

// the neo-Hookean point quantities of the tangent at F: G = F_g^-T and cm = mu - lam ln det F_g of the WLS
// argument F_g = I + gamma (F - I) (F itself without WLS)
__device__ __forceinline__ void tan_point(const MechDev& a, const double (&F)[9], double gam, double (&G)[9],
                                          double& cm) {
  if (!a.use_gamma) {
    nh_point(F, a.lam, a.mu, G, cm);
    return;
  }
  double Fg[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) Fg[q] = (q % 4 == 0 ? 1.0 : 0.0) + gam * (F[q] - (q % 4 == 0 ? 1.0 : 0.0));
  nh_point(Fg, a.lam, a.mu, G, cm);
}

// add_dP_eff of the neo-Hookean material from the cached point quantities (G, cm)
__device__ __forceinline__ void add_dP_eff_g(const MechDev& a, const double (&G)[9], double cm, const double (&d)[9],
                                             double gam, double c, double (&P)[9]) {
  if (!a.use_gamma) {
    add_dP_nh_g(G, cm, d, a.lam, a.mu, c, P);
    return;
  }
  add_dP_nh_g(G, cm, d, a.lam, a.mu, c * gam * gam, P);
  add_dsig_lin(d, a.lam, a.mu, c * (1.0 - gam * gam), P);
}

// ---- element kernel ------------------------------------------------------------------------------------------
// MODE 0: energy, element forces of P, sum of P (10 partials); 1: element forces of dP, sum of dP (9);
// 2: energy only (1). Vectors are SoA [3][N]; fe is [24][N] (dof 3a + c of the element's node a).
constexpr int kMechThreads = 128;
constexpr int kTanCache = 10;  // cached doubles per Gauss point: G = F_g^-T (9), cm

template <int MODE>
__global__ void __launch_bounds__(kMechThreads) k_mech_elem(MechDev a, const double* __restrict__ w,
                                                            const double* __restrict__ Fbar,
                                                            const double* __restrict__ v,
                                                            const double* __restrict__ dFm,
                                                            double* __restrict__ fe, double* __restrict__ partial) {
  constexpr bool TAN = MODE == 1;
  constexpr int NP = MODE == 0 ? 10 : (TAN ? 9 : 1);
  __shared__ double red[32 * NP];
  double acc[NP];
#pragma unroll
  for (int q = 0; q < NP; ++q) acc[q] = 0.0;
  double Fb[9], dM[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    Fb[q] = Fbar[q];
    dM[q] = TAN ? dFm[q] : 0.0;
  }
  const long N = a.N;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < N; e += (long)gridDim.x * blockDim.x) {
    const int k = (int)(e % a.n2), j = (int)((e / a.n2) % a.n1), i = (int)(e / ((long)a.n1 * a.n2));
    // the element's 8 nodes e + (ax, ay, az): periodic neighbours by a compare, not a modulo
    const long ip = (i + 1 == a.n0 ? 0 : i + 1), jp = (j + 1 == a.n1 ? 0 : j + 1), kp = (k + 1 == a.n2 ? 0 : k + 1);
    long nid[8];
#pragma unroll
    for (int q = 0; q < 8; ++q)
      nid[q] = (((q & 1) ? ip : i) * a.n1 + (((q >> 1) & 1) ? jp : j)) * a.n2 + ((q >> 2) ? kp : k);
    double wn[3][8];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int q = 0; q < 8; ++q) wn[c][q] = w[c * N + nid[q]];
    double vn[3][8];
    if (TAN) {
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int q = 0; q < 8; ++q) vn[c][q] = v[c * N + nid[q]];
    }
    const double cs = a.wq * a.s[e];
    const double gam = a.use_gamma ? a.gamma[e] : 1.0;
    double fa[3][8];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int q = 0; q < 8; ++q) fa[c][q] = 0.0;
#pragma unroll 1
    for (int g = 0; g < 8; ++g) {
      double F[9];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          double h = 0.0;
#pragma unroll
          for (int q = 0; q < 8; ++q) h += wn[c][q] * cDN[g][q][d];
          F[c * 3 + d] = Fb[c * 3 + d] + h;
        }
      double P[9];
#pragma unroll
      for (int q = 0; q < 9; ++q) P[q] = 0.0;
      if (MODE == 0 || MODE == 2) acc[0] += cs * psi_eff(a, F, gam);
      if (MODE == 0) add_P_eff(a, F, gam, cs, P);
      if (TAN) {
        double dF[9];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            double h = 0.0;
#pragma unroll
            for (int q = 0; q < 8; ++q) h += vn[c][q] * cDN[g][q][d];
            dF[c * 3 + d] = dM[c * 3 + d] + h;
          }
        add_dP_eff(a, F, dF, gam, cs, P);
      }
      if (MODE != 2) {
#pragma unroll
        for (int q = 0; q < 9; ++q) acc[(MODE == 0 ? 1 : 0) + q] += P[q];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int q = 0; q < 8; ++q)
            fa[c][q] += P[c * 3] * cDN[g][q][0] + P[c * 3 + 1] * cDN[g][q][1] + P[c * 3 + 2] * cDN[g][q][2];
      }
    }
    if (MODE != 2) {
#pragma unroll
      for (int q = 0; q < 8; ++q)
#pragma unroll
        for (int c = 0; c < 3; ++c) fe[(long)(3 * q + c) * N + e] = fa[c][q];
    }
  }
  block_sum<NP>(acc, red);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NP; ++q) partial[(long)blockIdx.x * NP + q] = acc[q];
  }
}

// Tangent cache of a CG solve at the state (w, Fbar) of the neo-Hookean material: G = F_g^-T and
// cm = mu - lam ln det F_g at each Gauss point of each element, tc[(g kTanCache + q) N + e], computed once instead
// of in every matvec (F, F_g, det, the inverse and the log are fixed while the CG runs).
__global__ void __launch_bounds__(kMechThreads) k_mech_tan_cache(MechDev a, const double* __restrict__ w,
                                                                 const double* __restrict__ Fbar,
                                                                 double* __restrict__ tc) {
  double Fb[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) Fb[q] = Fbar[q];
  const long N = a.N;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < N; e += (long)gridDim.x * blockDim.x) {
    const int k = (int)(e % a.n2), j = (int)((e / a.n2) % a.n1), i = (int)(e / ((long)a.n1 * a.n2));
    const long ip = (i + 1 == a.n0 ? 0 : i + 1), jp = (j + 1 == a.n1 ? 0 : j + 1), kp = (k + 1 == a.n2 ? 0 : k + 1);
    double wn[3][8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const long nid = (((q & 1) ? ip : i) * a.n1 + (((q >> 1) & 1) ? jp : j)) * a.n2 + ((q >> 2) ? kp : k);
#pragma unroll
      for (int c = 0; c < 3; ++c) wn[c][q] = w[c * N + nid];
    }
    const double gam = a.use_gamma ? a.gamma[e] : 1.0;
#pragma unroll 1
    for (int g = 0; g < 8; ++g) {
      double F[9];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          double h = 0.0;
#pragma unroll
          for (int q = 0; q < 8; ++q) h += wn[c][q] * cDN[g][q][d];
          F[c * 3 + d] = Fb[c * 3 + d] + h;
        }
      double G[9], cm;
      tan_point(a, F, gam, G, cm);
      double* t = tc + (long)g * kTanCache * N + e;
#pragma unroll
      for (int q = 0; q < 9; ++q) t[q * N] = G[q];
      t[9 * N] = cm;
    }
  }
}

// out[c][n] = sum_a fe[3a + c][n - off_a]
__global__ void k_mech_gather(long N, int n0, int n1, int n2, const double* __restrict__ fe, double* __restrict__ out) {
  const long n = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (n >= N) return;
  const int k = (int)(n % n2), j = (int)((n / n2) % n1), i = (int)(n / ((long)n1 * n2));
  const long im = (i == 0 ? n0 - 1 : i - 1), jm = (j == 0 ? n1 - 1 : j - 1), km = (k == 0 ? n2 - 1 : k - 1);
  double o[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const long e = (((q & 1) ? im : i) * n1 + (((q >> 1) & 1) ? jm : j)) * n2 + ((q >> 2) ? km : k);
#pragma unroll
    for (int c = 0; c < 3; ++c) o[c] += fe[(long)(3 * q + c) * N + e];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) out[c * N + n] = o[c];
}

// sum of nb partial rows of width NP into out[NP]
// (one block of kSumThreads: thread t adds rows t, t + kSumThreads, ... of every column, then the block adds the
// threads' sums in a fixed order, so the result does not depend on timing; a single thread per column would walk
// the nb rows as one chain of dependent loads)
constexpr int kSumThreads = 256;

template <int NP>
__global__ void __launch_bounds__(kSumThreads) k_mech_sum(const double* __restrict__ partial, int nb,
                                                          double* __restrict__ out) {
  __shared__ double red[32 * NP];
  double a[NP];
#pragma unroll
  for (int q = 0; q < NP; ++q) a[q] = 0.0;
  for (int b = threadIdx.x; b < nb; b += kSumThreads)
#pragma unroll
    for (int q = 0; q < NP; ++q) a[q] += partial[(long)b * NP + q];
  block_sum<NP>(a, red);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < NP; ++q) out[q] = a[q];
}

__global__ void k_mech_scale(int n0, int n1, int n2, const double* __restrict__ rho, double emin, double p,
                             double wb, double r0, double* __restrict__ s, double* __restrict__ gamma,
                             double* __restrict__ logs) {
  const long N = (long)n0 * n1 * n2;
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= N) return;
  const double r = rho[e];
  const double rc = r > 1.0 ? 1.0 : (r < 0.0 ? 0.0 : r);
  const double v = pow(rc, p);
  s[e] = emin + (1.0 - emin) * v;  // mech.py:105-106
  logs[e] = log(s[e]);
  if (wb > 0.0)  // mech.py:108-113
    gamma[e] = (tanh(wb * r0) + tanh(wb * (v - r0))) / (tanh(wb * r0) + tanh(wb * (1.0 - r0)));
}

// displacement gradient at the Gauss points: H[g][n][c][d] = sum_a w_c(e + off_a) DN[g][a][d]
__global__ void k_mech_gradw(long N, int n0, int n1, int n2, const double* __restrict__ w, double* __restrict__ H) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= N) return;
  const int k = (int)(e % n2), j = (int)((e / n2) % n1), i = (int)(e / ((long)n1 * n2));
  double wn[3][8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const long nd = ((long)wrap(i + (q & 1), n0) * n1 + wrap(j + ((q >> 1) & 1), n1)) * n2 + wrap(k + (q >> 2), n2);
#pragma unroll
    for (int c = 0; c < 3; ++c) wn[c][q] = w[c * N + nd];
  }
  for (int g = 0; g < 8; ++g)
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        double h = 0.0;
#pragma unroll
        for (int q = 0; q < 8; ++q) h += wn[c][q] * cDN[g][q][d];
        H[(((long)g * N + e) * 3 + c) * 3 + d] = h;
      }
}

// ---- third-order elastic constants (mech.py:458-493) ------------------------------------------------------------
// f(s) = wq sum_{g,e} s_e psi_eff(I + sum_I s_I H_I), H_I = voigt(I) + grad chi_I. At s = 0 (F = I) the
// derivatives have closed forms: f''_IJ = wq sum s (lam trH_I trH_J + mu (H_I : H_J + tr H_I H_J)) for either
// material (the WLS factor gamma cancels: psi_NH''(I) = psi_lin''), and for the neo-Hookean material
// f'''_IJK = wq sum s gamma^3 [-mu tr((H_I H_J + H_J H_I) H_K) - lam (trH_I tr H_J H_K + trH_J tr H_K H_I +
// trH_K tr H_I H_J)] (psi_NH'''(I); the quadratic parts drop out). Outputs per CTA: the 21 distinct f''_IJ
// (I <= J) then the 56 distinct f'''_IJK (I <= J <= K), without wq; accumulators in shared memory, one column
// per thread, reduced in a fixed order.
constexpr int kToecOut = 77, kToecThreads = 256, kToecWarps = kToecThreads / 32;

__host__ __device__ __forceinline__ double voigt_entry(int I, int c, int d) {
  // the symmetric tensor of Voigt unit strain I (engineering shear: off-diagonals 1/2), Voigt xx yy zz yz xz xy
  const int a = I < 3 ? I : (I == 3 ? 1 : 0), b = I < 3 ? I : (I == 5 ? 1 : 2);
  if (I < 3) return (c == a && d == a) ? 1.0 : 0.0;
  return ((c == a && d == b) || (c == b && d == a)) ? 0.5 : 0.0;
}

// output q -> (I, J) for q < 21 (I <= J), (I, J, K) for q >= 21 (I <= J <= K), lexicographic
__constant__ signed char cToecIdx[kToecOut][3];

// One warp per element: lanes 0..17 form grad chi_I (row c of I = lane / 3, c = lane % 3) at the 8 Gauss points
// into the warp's shared H[g][I][3][3] (plus voigt(I)); then lane l accumulates outputs l, l + 32, l + 64 over
// the 8 Gauss points in registers. At the end the CTA's partial sums are reduced in a fixed order.
__global__ void __launch_bounds__(kToecThreads) k_mech_toec(MechDev d, const double* __restrict__ chi,
                                                            double* __restrict__ part) {
  __shared__ double Hs[kToecWarps][8][6][9];
  __shared__ double red[kToecWarps][kToecOut];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long N = d.N;
  const bool nh = d.material == 1;
  double acc[3] = {0.0, 0.0, 0.0};
  int oi[3][3];
  int nout = 0;
  for (int r = 0; r < 3; ++r) {
    const int q = lane + 32 * r;
    if (q < kToecOut) {
      oi[r][0] = cToecIdx[q][0];
      oi[r][1] = cToecIdx[q][1];
      oi[r][2] = cToecIdx[q][2];
      nout = r + 1;
    }
  }
  double (*H)[6][9] = Hs[wid];
  for (long e = (long)blockIdx.x * kToecWarps + wid; e < N; e += (long)gridDim.x * kToecWarps) {
    const int k = (int)(e % d.n2), j = (int)((e / d.n2) % d.n1), i = (int)(e / ((long)d.n1 * d.n2));
    if (lane < 18) {
      const int I = lane / 3, c = lane - 3 * (lane / 3);
      double nv[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const long nd = ((long)wrap(i + (q & 1), d.n0) * d.n1 + wrap(j + ((q >> 1) & 1), d.n1)) * d.n2 +
                        wrap(k + (q >> 2), d.n2);
        nv[q] = chi[((long)I * 3 + c) * N + nd];
      }
#pragma unroll
      for (int g = 0; g < 8; ++g)
#pragma unroll
        for (int dd = 0; dd < 3; ++dd) {
          double h = 0.0;
#pragma unroll
          for (int q = 0; q < 8; ++q) h += nv[q] * cDN[g][q][dd];
          H[g][I][c * 3 + dd] = h + voigt_entry(I, c, dd);
        }
    }
    __syncwarp();
    const double se = d.s[e];
    const double ga = d.use_gamma ? d.gamma[e] : 1.0;
    const double w3 = nh ? se * ga * ga * ga : 0.0;
    for (int r = 0; r < nout; ++r) {
      const int I = oi[r][0], J = oi[r][1], K = oi[r][2];
      const int q = lane + 32 * r;
      double sum = 0.0;
      for (int g = 0; g < 8; ++g) {
        const double* A = H[g][I];
        const double* B = H[g][J];
        const double trA = A[0] + A[4] + A[8], trB = B[0] + B[4] + B[8];
        if (q < 21) {
          double dd = 0.0, qq = 0.0;
#pragma unroll
          for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b2 = 0; b2 < 3; ++b2) {
              dd += A[a * 3 + b2] * B[a * 3 + b2];
              qq += A[a * 3 + b2] * B[b2 * 3 + a];
            }
          sum += se * (d.lam * trA * trB + d.mu * (dd + qq));
        } else if (nh) {
          const double* Cc = H[g][K];
          const double trC = Cc[0] + Cc[4] + Cc[8];
          double t1 = 0.0, qAB = 0.0, qBC = 0.0, qCA = 0.0;
#pragma unroll
          for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              double pac = 0.0;  // (AB + BA)[a][c]
#pragma unroll
              for (int b2 = 0; b2 < 3; ++b2) pac += A[a * 3 + b2] * B[b2 * 3 + c] + B[a * 3 + b2] * A[b2 * 3 + c];
              t1 += pac * Cc[c * 3 + a];
              qAB += A[a * 3 + c] * B[c * 3 + a];
              qBC += B[a * 3 + c] * Cc[c * 3 + a];
              qCA += Cc[a * 3 + c] * A[c * 3 + a];
            }
          sum += w3 * (-d.mu * t1 - d.lam * (trA * qBC + trB * qCA + trC * qAB));
        }
      }
      acc[r] += sum;
    }
    __syncwarp();  // H is rewritten for the next element
  }
  for (int r = 0; r < nout; ++r) red[wid][lane + 32 * r] = acc[r];
  __syncthreads();
  for (int q = threadIdx.x; q < kToecOut; q += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < kToecWarps; ++w) s += red[w][q];
    part[(long)blockIdx.x * kToecOut + q] = s;
  }
}

__global__ void k_mech_toec_reduce(const double* __restrict__ part, int nblk, double wq, double* __restrict__ out) {
  const int q = threadIdx.x;
  if (q >= kToecOut) return;
  double s = 0.0;
  for (int b = 0; b < nblk; ++b) s += part[(long)b * kToecOut + q];
  out[q] = wq * s;
}

// ---- CG (mech.py:264-290) on z = (w [3][N], macro tail [k]) ------------------------------------------------------
struct MechCG {
  double bn, rz, pap, alpha, beta, rr, scale;  // scale = N / sws of the w preconditioner
  double mAp[3], mz[3];
  double dmac[9];
  double tol;
  int k, it, maxit, done, conv, neg, ran;
};

constexpr int kCgBlocks = 256;

// partials over the vector: [sum a_w (3), sum a.b (w part)]
__global__ void k_cg_dot(long N, const double* __restrict__ a, const double* __restrict__ b,
                         const MechCG* __restrict__ st, double* __restrict__ partial) {
  __shared__ double red[32 * 4];
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  if (!st->done) {
#pragma unroll
    for (int c = 0; c < 3; ++c)
      for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
        const double x = a[c * N + i];
        acc[c] += x;
        acc[3] += x * b[c * N + i];
      }
  }
  block_sum<4>(acc, red);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < 4; ++q) partial[blockIdx.x * 4 + q] = acc[q];
}

// after Ap = H p: mean of Ap's w part, pAp (tail included, p is mean-free), alpha and the negative-curvature flag
__global__ void k_cg_fin_pap(long N, const double* __restrict__ partial, int nb, const double* __restrict__ p,
                             const double* __restrict__ Ap, MechCG* st) {
  if (st->done) return;
  // one warp: lane-strided partial sums, then a shuffle reduction (fixed order)
  double s[4] = {0, 0, 0, 0};
  for (int b = threadIdx.x; b < nb; b += 32)
    for (int q = 0; q < 4; ++q) s[q] += partial[b * 4 + q];
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s[q] += __shfl_down_sync(0xffffffffu, s[q], o);
  if (threadIdx.x != 0) return;
  double pap = s[3];
  for (int t = 0; t < st->k; ++t) pap += p[3 * N + t] * Ap[3 * N + t];
  for (int c = 0; c < 3; ++c) st->mAp[c] = s[c] / (double)N;
  st->pap = pap;
  st->neg = pap <= 0.0;
  st->alpha = st->neg ? 0.0 : st->rz / pap;
  st->ran = 1;
}

// x1 = x + a p, r1 = r - a (Ap - mean): on negative curvature x = z0 at it == 0 else x unchanged
__global__ void k_cg_xr(long N, double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                        const double* __restrict__ Ap, const double* __restrict__ z0, const MechCG* __restrict__ st) {
  if (st->done) return;
  const double a = st->alpha;
  const bool neg = st->neg, first = st->it == 0;
  const int k = st->k;
  const long i0 = blockIdx.x * (long)blockDim.x + threadIdx.x, step = (long)gridDim.x * blockDim.x;
#pragma unroll
  for (int c = 0; c <= 3; ++c) {  // c = 3: the macro tail (k entries)
    const long off = c * N, len = c < 3 ? N : k;
    const double mu = c < 3 ? st->mAp[c] : 0.0;
    for (long i = i0; i < len; i += step) {
      r[off + i] -= a * (Ap[off + i] - mu);
      if (neg) {
        if (first) x[off + i] = z0[off + i];
      } else {
        x[off + i] += a * p[off + i];
      }
    }
  }
}

// after the preconditioner (w part unscaled in zf): mean of z, rz1, rr, convergence, beta, counters
__global__ void k_cg_fin_pc(long N, int n0, const double* __restrict__ partial, const double* __restrict__ r,
                            MechCG* st, int init) {
  if (st->done) return;
  // one warp: lane-strided partial sums over the x-planes, then a shuffle reduction (fixed order)
  double a[3][4];
  for (int c = 0; c < 3; ++c)
    for (int q = 0; q < 4; ++q) {
      double v = 0.0;
      for (int x = threadIdx.x; x < n0; x += 32) v += partial[((long)c * n0 + x) * 4 + q];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      a[c][q] = v;
    }
  if (threadIdx.x != 0) return;
  double rz1 = 0.0, rr = 0.0;
  for (int c = 0; c < 3; ++c) {
    st->mz[c] = a[c][0] / (double)N;
    rz1 += st->scale * (a[c][1] - st->mz[c] * a[c][2]);
    rr += a[c][3];
  }
  for (int t = 0; t < st->k; ++t) {
    const double rt = r[3 * N + t];
    rz1 += rt * rt / st->dmac[t];
    rr += rt * rt;
  }
  st->rr = rr;
  if (init) {
    st->bn = sqrt(rr) + 1e-300;
    st->rz = rz1;
    return;
  }
  const bool conv1 = sqrt(rr) <= st->tol * st->bn;
  st->beta = rz1 / (st->rz == 0.0 ? 1.0 : st->rz);
  st->rz = rz1;
  st->it += 1;
  st->conv = conv1 && !st->neg;
  st->done = st->neg || conv1 || st->it >= st->maxit;
}

// p1 = scale (zf - mean) + beta p (w part), r_t / dmac_t + beta p_t (tail); init: p = z0 = M b (also kept in z0)
__global__ void k_cg_p(long N, double* __restrict__ p, const double* __restrict__ zf, const double* __restrict__ r,
                       double* __restrict__ z0, const MechCG* __restrict__ st, int init) {
  if (!init && !st->ran) return;
  const double be = init ? 0.0 : st->beta, sc = st->scale;
  const int k = st->k;
  const long i0 = blockIdx.x * (long)blockDim.x + threadIdx.x, step = (long)gridDim.x * blockDim.x;
#pragma unroll
  for (int c = 0; c <= 3; ++c) {  // c = 3: the macro tail (k entries)
    const long off = c * N, len = c < 3 ? N : k;
    const double mu = c < 3 ? st->mz[c] : 0.0;
    for (long i = i0; i < len; i += step) {
      const double z = c < 3 ? sc * (zf[off + i] - mu) : r[off + i] / st->dmac[i];
      if (init) {
        p[off + i] = z;
        z0[off + i] = z;
      } else {
        p[off + i] = z + be * p[off + i];
      }
    }
  }
}

__global__ void k_cg_clear_ran(MechCG* st) { st->ran = 0; }

// free macro index pairs (a, b) of the mixed control, packed as 3 a + b
struct FreeIdx {
  int k;
  int ab[9];
};

// Tangent matvec of the CG from the tangent cache (k_mech_tan_cache, neo-Hookean material): the element forces of
// dP for the direction (v, dFm) and the sums of dP at the first KF free macro entries fi.ab (partial rows of 9, the
// other entries 0; k_cg_aptail reads the free ones). Only the free macro entries are summed: the CG's tail needs no
// others.
//
// The direction's gradient and the element forces are taken in the mode form of the trilinear element (as in the
// linear operator, nlf_element.cuh): the butterfly c = H v of the 8 nodal values gives u = sum_p c_p 2^-z(p)
// prod_{d in p} X_d on X in [-1/2, 1/2]^3 (z(p) the zero bits of p), so at a Gauss point X = (sx, sy, sz) h,
// h = 1 / (2 sqrt 3):
//   du/dx = k1 + sy k3 + sz k5 + sy sz k7,  du/dy = k2 + sx k3 + sz k6 + sx sz k7,  du/dz = k4 + sx k5 + sy k6 + sx sy k7
// with k1,2,4 = c / 4, k3,5,6 = c h / 2, k7 = c h^2. The macro direction is the linear field dFm X, whose modes are
// k1,2,4 += dFm[.][x, y, z]. The forces are the transpose: signed sums of P over the Gauss points per mode, scaled
// the same way, then the transposed butterfly f = H^T m.
// asynchronous copy of one double global -> shared (through L1), and the waits for this thread's copy groups
__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit_group() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;" ::"n"(PENDING) : "memory");
}

template <int KF>
__global__ void __launch_bounds__(kMechThreads, 3) k_mech_hvp_tc(MechDev a, const double* __restrict__ v,
                                                                 const double* __restrict__ dFm, FreeIdx fi,
                                                                 double* __restrict__ fe,
                                                                 double* __restrict__ partial,
                                                                 const double* __restrict__ tc) {
  constexpr int NA = KF > 0 ? KF : 1;
  constexpr double h = 0.28867513459481288225;  // 1 / (2 sqrt 3)
  __shared__ double red[32 * NA];
  // the cache entries of the next Gauss point are copied into this thread's own slots while the current one is
  // computed (each thread reads only what it copied, so its own wait suffices: no barrier)
  __shared__ double stage[2][kTanCache][kMechThreads];
  const int tid = threadIdx.x;
  double acc[NA];
#pragma unroll
  for (int j = 0; j < NA; ++j) acc[j] = 0.0;
  const long N = a.N;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < N; e += (long)gridDim.x * blockDim.x) {
    const int k = (int)(e % a.n2), j = (int)((e / a.n2) % a.n1), i = (int)(e / ((long)a.n1 * a.n2));
    const long ip = (i + 1 == a.n0 ? 0 : i + 1), jp = (j + 1 == a.n1 ? 0 : j + 1), kp = (k + 1 == a.n2 ? 0 : k + 1);
    double km[3][8];  // scaled modes k1..k7 of each component (km[c][0] unused)
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const long nid = (((q & 1) ? ip : i) * a.n1 + (((q >> 1) & 1) ? jp : j)) * a.n2 + ((q >> 2) ? kp : k);
#pragma unroll
      for (int c = 0; c < 3; ++c) km[c][q] = v[c * N + nid];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      butterfly8(km[c]);
      km[c][1] = 0.25 * km[c][1] + dFm[c * 3];
      km[c][2] = 0.25 * km[c][2] + dFm[c * 3 + 1];
      km[c][4] = 0.25 * km[c][4] + dFm[c * 3 + 2];
      km[c][3] *= 0.5 * h;
      km[c][5] *= 0.5 * h;
      km[c][6] *= 0.5 * h;
      km[c][7] *= h * h;
    }
    {
      const double* t0 = tc + e;
#pragma unroll
      for (int q = 0; q < kTanCache; ++q) cp_async8(&stage[0][q][tid], t0 + (long)q * N);
      cp_async_commit_group();
    }
    const double cs = a.wq * a.s[e];
    const double gam = a.use_gamma ? a.gamma[e] : 1.0;
    double nm[3][8];  // signed sums of P per mode (nm[c][0] unused)
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int q = 0; q < 8; ++q) nm[c][q] = 0.0;
#pragma unroll 1
    for (int g = 0; g < 8; ++g) {
      const double sx = (g & 1) ? 1.0 : -1.0, sy = ((g >> 1) & 1) ? 1.0 : -1.0, sz = (g >> 2) ? 1.0 : -1.0;
      const double syz = sy * sz, sxz = sx * sz, sxy = sx * sy;
      double dF[9];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        dF[c * 3] = km[c][1] + sy * km[c][3] + sz * km[c][5] + syz * km[c][7];
        dF[c * 3 + 1] = km[c][2] + sx * km[c][3] + sz * km[c][6] + sxz * km[c][7];
        dF[c * 3 + 2] = km[c][4] + sx * km[c][5] + sy * km[c][6] + sxy * km[c][7];
      }
      if (g + 1 < 8) {
        const double* tn = tc + (long)(g + 1) * kTanCache * N + e;
#pragma unroll
        for (int q = 0; q < kTanCache; ++q) cp_async8(&stage[(g + 1) & 1][q][tid], tn + (long)q * N);
        cp_async_commit_group();
        cp_async_wait_group<1>();  // this Gauss point's copies are done, the next one's may still be in flight
      } else {
        cp_async_wait_group<0>();
      }
      double G[9];
#pragma unroll
      for (int q = 0; q < 9; ++q) G[q] = stage[g & 1][q][tid];
      const double cmg = stage[g & 1][9][tid];
      double P[9];
#pragma unroll
      for (int q = 0; q < 9; ++q) P[q] = 0.0;
      add_dP_eff_g(a, G, cmg, dF, gam, cs, P);
#pragma unroll
      for (int jf = 0; jf < KF; ++jf) {
        double pj = 0.0;
#pragma unroll
        for (int q = 0; q < 9; ++q) pj = (q == fi.ab[jf]) ? P[q] : pj;
        acc[jf] += pj;
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double px = P[c * 3], py = P[c * 3 + 1], pz = P[c * 3 + 2];
        nm[c][1] += px;
        nm[c][2] += py;
        nm[c][4] += pz;
        nm[c][3] += sy * px + sx * py;
        nm[c][5] += sz * px + sx * pz;
        nm[c][6] += sz * py + sy * pz;
        nm[c][7] += syz * px + sxz * py + sxy * pz;
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      nm[c][0] = 0.0;
      nm[c][1] *= 0.25;
      nm[c][2] *= 0.25;
      nm[c][4] *= 0.25;
      nm[c][3] *= 0.5 * h;
      nm[c][5] *= 0.5 * h;
      nm[c][6] *= 0.5 * h;
      nm[c][7] *= h * h;
      butterfly8_t(nm[c]);
    }
#pragma unroll
    for (int q = 0; q < 8; ++q)
#pragma unroll
      for (int c = 0; c < 3; ++c) fe[(long)(3 * q + c) * N + e] = nm[c][q];
  }
  if constexpr (KF > 0) {
    block_sum<NA>(acc, red);
    if (threadIdx.x == 0) {
      double row[9];
#pragma unroll
      for (int q = 0; q < 9; ++q) row[q] = 0.0;
#pragma unroll
      for (int jf = 0; jf < KF; ++jf)
#pragma unroll
        for (int q = 0; q < 9; ++q)
          if (q == fi.ab[jf]) row[q] = acc[jf];
#pragma unroll
      for (int q = 0; q < 9; ++q) partial[(long)blockIdx.x * 9 + q] = row[q];
    }
  }
}

// dFm (9, row-major) = sum_j p_tail[j] e_(a_j b_j): the macro part of the CG direction enters the element pass
__global__ void k_cg_dfm(const double* __restrict__ ptail, FreeIdx f, double* __restrict__ dfm) {
  const int q = threadIdx.x;
  if (q < 9) {
    double v = 0.0;
    for (int j = 0; j < f.k; ++j)
      if (f.ab[j] == q) v = ptail[j];
    dfm[q] = v;
  }
}

// Ap_tail[j] = the P-bar sensitivity sum9 at the free entry j
__global__ void k_cg_aptail(const double* __restrict__ sum9, FreeIdx f, double* __restrict__ aptail) {
  const int j = threadIdx.x;
  if (j < f.k) aptail[j] = sum9[f.ab[j]];
}

// b = proj(b): subtract the mean of the w part (in place) using k_cg_dot partials of (b, b)
__global__ void k_cg_mean_sub(long N, double* __restrict__ b, const double* __restrict__ partial, int nb) {
  __shared__ double m[3];
  if (threadIdx.x < 3) {
    double a = 0.0;
    for (int q = 0; q < nb; ++q) a += partial[q * 4 + threadIdx.x];
    m[threadIdx.x] = a / (double)N;
  }
  __syncthreads();
  for (int c = 0; c < 3; ++c)
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
      b[c * N + i] -= m[c];
}

}  // namespace nlf

using namespace nlf;

struct nlf_mech {
  nlf_linear* lin = nullptr;  // FFT tables and geometry of the preconditioner
  MechDev d{};
  double wls_b = 0.0, wls_r0 = 0.0, emin = 0.0, p = 3.0, sws = 1.0;
  bool rho_set = false;
  DevBuf state;  // s, gamma, logs
  DevBuf ws;     // vectors and partials
  DevBuf io;     // staging
  // CG iterations replayed from a CUDA graph on a handle-owned stream, ordered after and before the caller's
  // stream by events (capture is not possible on the legacy default stream)
  cudaStream_t gst = nullptr;
  cudaEvent_t gev[2] = {nullptr, nullptr};
  int pc_mode = NLF_PC_FFT;  // NLF_PC_FFT: the reference's N K0^-1 / sws; NLF_PC_FFT_SCALED: N w K0^-1 w
  double* wnode = nullptr;   // w = (root mean square of s over the 8 elements around a node)^-0.47, in `state`
};

namespace {

size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

bool on_dev(const void* p) {
  if (!p) return false;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

// device copy of a (count) float64 input: the pointer itself or a staged copy at io + off
int stage(const double* src, size_t count, DevBuf& io, size_t off, const double** out, cudaStream_t st) {
  if (!src) {
    *out = nullptr;
    return NLF_OK;
  }
  if (on_dev(src)) {
    *out = src;
    return NLF_OK;
  }
  double* dst = reinterpret_cast<double*>((char*)io.ptr + off);
  NLF_CUDA_TRY(cudaMemcpyAsync(dst, src, count * sizeof(double), cudaMemcpyHostToDevice, st));
  *out = dst;
  return NLF_OK;
}

int copy_back(double* dst, const double* src, size_t count, cudaStream_t st) {
  NLF_CUDA_TRY(cudaMemcpyAsync(dst, src, count * sizeof(double),
                               on_dev(dst) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
  return NLF_OK;
}

LinearHandle& lin_of(nlf_mech* H);

}  // namespace

// access to the linear handle's internals (defined in nlf_linear.cu)
namespace nlf {
LinearHandle& linear_handle(nlf_linear* h);
}

namespace {
LinearHandle& lin_of(nlf_mech* H) { return nlf::linear_handle(H->lin); }

// one element pass of MODE over the SoA state w (device) with macro Fbar (device 9), direction v, dFm
template <int MODE>
int mech_pass(nlf_mech* H, const double* w, const double* Fb, const double* v, const double* dFm, double* fe,
              double* partial, int* nb, cudaStream_t st) {
  const long N = H->d.N;
  const int blocks = (int)std::min<long>((N + kMechThreads - 1) / kMechThreads, 4L * 148 * 4);
  *nb = blocks;
  ProfScope ps(PK_MECH_ELEM, st);
  k_mech_elem<MODE><<<blocks, kMechThreads, 0, st>>>(H->d, w, Fb, v, dFm, fe, partial);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}

// the tangent cache of a CG solve at (w, Fbar) (neo-Hookean material only)
int tan_cache(nlf_mech* H, const double* w, const double* Fb, double* tc, cudaStream_t st) {
  const long N = H->d.N;
  const int blocks = (int)std::min<long>((N + kMechThreads - 1) / kMechThreads, 4L * 148 * 4);
  ProfScope ps(PK_MECH_TANC, st);
  k_mech_tan_cache<<<blocks, kMechThreads, 0, st>>>(H->d, w, Fb, tc);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}

// the CG's tangent matvec from the cache; the free macro entries' sums of dP go to partial rows of 9
int hvp_cached(nlf_mech* H, const double* v, const double* dFm, const FreeIdx& fi, double* fe, double* partial,
               int* nb, const double* tc, cudaStream_t st) {
  const long N = H->d.N;
  const int blocks = (int)std::min<long>((N + kMechThreads - 1) / kMechThreads, 4L * 148 * 4);
  *nb = blocks;
  ProfScope ps(PK_MECH_ELEM, st);
  if (fi.k == 0)
    k_mech_hvp_tc<0><<<blocks, kMechThreads, 0, st>>>(H->d, v, dFm, fi, fe, partial, tc);
  else if (fi.k <= 2)
    k_mech_hvp_tc<2><<<blocks, kMechThreads, 0, st>>>(H->d, v, dFm, fi, fe, partial, tc);
  else
    k_mech_hvp_tc<9><<<blocks, kMechThreads, 0, st>>>(H->d, v, dFm, fi, fe, partial, tc);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}

int gather(nlf_mech* H, const double* fe, double* out, cudaStream_t st) {
  const long N = H->d.N;
  ProfScope ps(PK_MECH_GATHER, st);
  k_mech_gather<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(N, H->d.n0, H->d.n1, H->d.n2, fe, out);
  NLF_CHECK_LAUNCH();
  return NLF_OK;
}

bool bad(nlf_mech* H) {
  if (!H || !H->rho_set) {
    set_error("mech handle is null or has no density (call nlf_mech_set_rho)");
    return true;
  }
  return false;
}

}  // namespace

extern "C" {

NLF_API int nlf_mech_create(nlf_mech** out, int nx, int ny, int nz, double E, double nu, int material,
                            double wls_b, double wls_r0, double emin, double p) {
  if (!out || (material != 0 && material != 1)) {
    set_error("nlf_mech_create: bad arguments (material 0 = linear, 1 = neo-Hookean)");
    return NLF_EBADARG;
  }
  *out = nullptr;
  nlf_mech* H = new nlf_mech();
  int stc = nlf_linear_create(&H->lin, nx, ny, nz, E, nu, emin, p, 1e-9, 1);
  if (stc != NLF_OK) {
    delete H;
    return stc;
  }
  // the node-scaled CG preconditioner of the finite-strain tangent inverts the material's own medium: the
  // Poisson-ratio-0 medium of the linear solve needs more CG iterations here (502 against 343 per load step on
  // the 64^3 compression bench)
  stc = rebuild_scaled_kinv(lin_of(H), nu);
  if (stc != NLF_OK) {
    nlf_linear_destroy(H->lin);
    delete H;
    return stc;
  }
  const LinearHandle& L = lin_of(H);
  H->d.n0 = nx;
  H->d.n1 = ny;
  H->d.n2 = nz;
  H->d.N = L.g.N;
  H->d.lam = L.lam;
  H->d.mu = L.mu;
  H->d.wq = 1.0 / (8.0 * (double)L.g.N);
  H->d.material = material;
  H->d.use_gamma = (material == 1 && wls_b > 0.0) ? 1 : 0;
  H->wls_b = wls_b;
  H->wls_r0 = wls_r0;
  H->emin = emin;
  H->p = p;
  // shape-function gradients at the Gauss points (nlfiber/linear.py:22-41)
  double dN[8][8][3];
  const double g1[2] = {0.5 - 1.0 / (2.0 * std::sqrt(3.0)), 0.5 + 1.0 / (2.0 * std::sqrt(3.0))};
  for (int g = 0; g < 8; ++g)
    for (int a = 0; a < 8; ++a) {
      const double x = g1[g & 1], y = g1[(g >> 1) & 1], z = g1[(g >> 2) & 1];
      const int i = a & 1, j = (a >> 1) & 1, k = (a >> 2) & 1;
      const double fx = i ? x : 1 - x, fy = j ? y : 1 - y, fz = k ? z : 1 - z;
      const double sx = i ? 1 : -1, sy = j ? 1 : -1, sz = k ? 1 : -1;
      dN[g][a][0] = sx * fy * fz;
      dN[g][a][1] = fx * sy * fz;
      dN[g][a][2] = fx * fy * sz;
    }
  cudaError_t e = cudaMemcpyToSymbol(cDN, dN, sizeof(dN));
  if (e != cudaSuccess) {
    set_error("nlf_mech_create: %s", cudaGetErrorString(e));
    nlf_linear_destroy(H->lin);
    delete H;
    return NLF_ECUDA;
  }
  *out = H;
  return NLF_OK;
}

NLF_API int nlf_mech_destroy(nlf_mech* H) {
  if (!H) return NLF_OK;
  if (H->gst) cudaStreamDestroy(H->gst);
  for (cudaEvent_t e : H->gev)
    if (e) cudaEventDestroy(e);
  H->state.release();
  H->ws.release();
  H->io.release();
  nlf_linear_destroy(H->lin);
  delete H;
  return NLF_OK;
}

NLF_API int nlf_mech_set_rho(nlf_mech* H, const double* rho, double* s_out, double* gamma_out, double* sws_out,
                             void* stream) {
  if (!H || !rho) {
    set_error("nlf_mech_set_rho: bad arguments");
    return NLF_EBADARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const long N = H->d.N;
  NLF_TRY(H->state.reserve(4 * al(N * 8)));
  NLF_TRY(H->io.reserve(al(N * 8)));
  const double* rd = nullptr;
  NLF_TRY(stage(rho, N, H->io, 0, &rd, st));
  double* s = reinterpret_cast<double*>(H->state.ptr);
  double* gam = reinterpret_cast<double*>((char*)H->state.ptr + al(N * 8));
  double* logs = reinterpret_cast<double*>((char*)H->state.ptr + 2 * al(N * 8));
  k_mech_scale<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(H->d.n0, H->d.n1, H->d.n2, rd, H->emin, H->p, H->wls_b,
                                                            H->wls_r0, s, gam, logs);
  NLF_CHECK_LAUNCH();
  H->d.s = s;
  H->d.gamma = gam;
  H->wnode = reinterpret_cast<double*>((char*)H->state.ptr + 3 * al(N * 8));
  NLF_TRY(launch_node_scaling(lin_of(H), 1, s, nullptr, H->wnode, nullptr, st));
  // sws = exp(mean log s) (mech.py:292-294), FP64 on the host from the device values
  std::vector<double> lg(N);
  NLF_CUDA_TRY(cudaMemcpyAsync(lg.data(), logs, N * 8, cudaMemcpyDeviceToHost, st));
  if (s_out) NLF_TRY(copy_back(s_out, s, N, st));
  if (gamma_out && H->wls_b > 0.0) NLF_TRY(copy_back(gamma_out, gam, N, st));
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  double a = 0.0;
  for (long i = 0; i < N; ++i) a += lg[i];
  H->sws = std::exp(a / (double)N);
  if (sws_out) *sws_out = H->sws;
  // the handle's work buffers at the largest size any of its calls takes (energy, hvp, grad_w, toec, and the CG
  // with the 9 macro unknowns at most), so that no later call allocates or frees device memory: a free while
  // another host thread captures a CUDA graph would invalidate that capture
  {
    const size_t V = al(3 * N * 8), part = al(4096 * 10 * 8);
    const size_t Lz = al((3 * N + 9) * 8);
    const size_t eh = 4 * V + al(24 * N * 8) + 256 + part + 256;  // energy and hvp
    const size_t gw = V + al(72 * N * 8);                         // grad_w
    const int nblk = (int)std::min<long>(4 * 148, (N + kToecWarps - 1) / kToecWarps);
    const size_t te = al(18 * N * 8) + al((size_t)nblk * kToecOut * 8) + al(kToecOut * 8);
    const size_t cgw = V + 5 * Lz + V + al(24 * N * 8) + al(3 * lin_of(H).g.NS * 16) + part +
                       al(3 * (size_t)H->d.n0 * 4 * 8) + al(256) + al(sizeof(MechCG)) +
                       (H->d.material == 1 ? al((size_t)8 * kTanCache * N * 8) : 0);
    NLF_TRY(H->ws.reserve(std::max(std::max(eh, gw), std::max(te, cgw))));
    NLF_TRY(H->io.reserve(std::max(al(18 * N * 8), 2 * Lz)));
  }
  H->rho_set = true;
  return NLF_OK;
}

// energy W; residual gw = dW/dw (nx, ny, nz, 3) and mean stress P = dW/dFbar (3, 3) when not NULL
NLF_API int nlf_mech_energy(nlf_mech* H, const double* w, const double* Fbar, double* W, double* gw, double* P,
                            void* stream) {
  if (bad(H) || !w || !Fbar || !W) {
    if (H && H->rho_set) set_error("nlf_mech_energy: bad arguments");
    return NLF_EBADARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const long N = H->d.N;
  const size_t o_w = 0, o_ws = al(3 * N * 8), o_fe = o_ws + al(3 * N * 8), o_g = o_fe + al(24 * N * 8);
  const size_t o_gs = o_g + al(3 * N * 8), o_fb = o_gs + al(3 * N * 8), o_p = o_fb + 256, o_sum = o_p + al(4096 * 10 * 8);
  NLF_TRY(H->ws.reserve(o_sum + 256));
  char* b = (char*)H->ws.ptr;
  NLF_TRY(H->io.reserve(al(3 * N * 8)));
  const double* wd = nullptr;
  NLF_TRY(stage(w, 3 * N, H->io, 0, &wd, st));
  double* ws = reinterpret_cast<double*>(b + o_ws);
  NLF_TRY((launch_aos_to_soa<double, double>(N, 1, wd, ws, 1.0, st)));
  double* fbd = reinterpret_cast<double*>(b + o_fb);
  NLF_CUDA_TRY(cudaMemcpyAsync(fbd, Fbar, 9 * 8, on_dev(Fbar) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  double* part = reinterpret_cast<double*>(b + o_p);
  double* sum = reinterpret_cast<double*>(b + o_sum);
  double* fe = reinterpret_cast<double*>(b + o_fe);
  int nb = 0;
  const bool want_g = gw || P;
  if (want_g) {
    NLF_TRY(mech_pass<0>(H, ws, fbd, nullptr, nullptr, fe, part, &nb, st));
    k_mech_sum<10><<<1, kSumThreads, 0, st>>>(part, nb, sum);
  } else {
    NLF_TRY(mech_pass<2>(H, ws, fbd, nullptr, nullptr, nullptr, part, &nb, st));
    k_mech_sum<1><<<1, kSumThreads, 0, st>>>(part, nb, sum);
  }
  NLF_CHECK_LAUNCH();
  double h[10];
  NLF_CUDA_TRY(cudaMemcpyAsync(h, sum, (want_g ? 10 : 1) * 8, cudaMemcpyDeviceToHost, st));
  if (gw) {
    double* gs = reinterpret_cast<double*>(b + o_gs);
    NLF_TRY(gather(H, fe, gs, st));
    double* gd = on_dev(gw) ? gw : reinterpret_cast<double*>(b + o_g);
    NLF_TRY((launch_soa_to_aos<double, double>(N, 1, gs, gd, st)));
    if (gd != gw) NLF_TRY(copy_back(gw, gd, 3 * N, st));
  }
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  *W = h[0];
  if (P) std::memcpy(P, h + 1, 9 * 8);
  return NLF_OK;
}

// tangent at (w, Fbar) applied to (v, dFm): hv (nx, ny, nz, 3) and hP (3, 3) = d(mean stress)
NLF_API int nlf_mech_hvp(nlf_mech* H, const double* w, const double* Fbar, const double* v, const double* dFm,
                         double* hv, double* hP, void* stream) {
  if (bad(H) || !w || !Fbar || !v || !dFm || !hv) {
    if (H && H->rho_set) set_error("nlf_mech_hvp: bad arguments");
    return NLF_EBADARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const long N = H->d.N;
  const size_t V = al(3 * N * 8);
  const size_t o_ws = 0, o_vs = V, o_fe = 2 * V, o_o = o_fe + al(24 * N * 8), o_os = o_o + V, o_fb = o_os + V;
  const size_t o_p = o_fb + 256, o_sum = o_p + al(4096 * 10 * 8);
  NLF_TRY(H->ws.reserve(o_sum + 256));
  NLF_TRY(H->io.reserve(2 * V));
  char* b = (char*)H->ws.ptr;
  const double *wd = nullptr, *vd = nullptr;
  NLF_TRY(stage(w, 3 * N, H->io, 0, &wd, st));
  NLF_TRY(stage(v, 3 * N, H->io, V, &vd, st));
  double* ws = reinterpret_cast<double*>(b + o_ws);
  double* vs = reinterpret_cast<double*>(b + o_vs);
  NLF_TRY((launch_aos_to_soa<double, double>(N, 1, wd, ws, 1.0, st)));
  NLF_TRY((launch_aos_to_soa<double, double>(N, 1, vd, vs, 1.0, st)));
  double* fbd = reinterpret_cast<double*>(b + o_fb);
  NLF_CUDA_TRY(cudaMemcpyAsync(fbd, Fbar, 72, on_dev(Fbar) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  NLF_CUDA_TRY(cudaMemcpyAsync(fbd + 9, dFm, 72, on_dev(dFm) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  double* fe = reinterpret_cast<double*>(b + o_fe);
  double* part = reinterpret_cast<double*>(b + o_p);
  double* sum = reinterpret_cast<double*>(b + o_sum);
  int nb = 0;
  NLF_TRY(mech_pass<1>(H, ws, fbd, vs, fbd + 9, fe, part, &nb, st));
  k_mech_sum<9><<<1, kSumThreads, 0, st>>>(part, nb, sum);
  NLF_CHECK_LAUNCH();
  double* os = reinterpret_cast<double*>(b + o_os);
  NLF_TRY(gather(H, fe, os, st));
  double* od = on_dev(hv) ? hv : reinterpret_cast<double*>(b + o_o);
  NLF_TRY((launch_soa_to_aos<double, double>(N, 1, os, od, st)));
  if (od != hv) NLF_TRY(copy_back(hv, od, 3 * N, st));
  double h[9];
  NLF_CUDA_TRY(cudaMemcpyAsync(h, sum, 72, cudaMemcpyDeviceToHost, st));
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  if (hP) std::memcpy(hP, h, 72);
  return NLF_OK;
}

// mech.py:187-189 precond_w: N x the linear FFT preconditioner (the mech operator carries wq = 1 / (8N))
NLF_API int nlf_mech_precond_w(nlf_mech* H, const double* r, double* z, void* stream) {
  if (!H || !r || !z) {
    set_error("nlf_mech_precond_w: bad arguments");
    return NLF_EBADARG;
  }
  const LinearHandle& L = lin_of(H);
  if (H->pc_mode == NLF_PC_FFT_SCALED) {
    if (!H->rho_set) {
      set_error("nlf_mech_precond_w: the scaled preconditioner needs nlf_mech_set_rho first");
      return NLF_EBADARG;
    }
    NLF_TRY(nlf_precond_ex(H->lin, 1, r, z, NLF_PREC_FP64, NLF_PC_FFT_SCALED, H->d.s, stream));
  } else {
    NLF_TRY(nlf_precond(H->lin, 1, r, z, stream));
  }
  // scale in place (z is host or device)
  const long n = 3 * L.g.N;
  if (on_dev(z)) {
    std::vector<double> t(n);
    NLF_CUDA_TRY(cudaMemcpy(t.data(), z, n * 8, cudaMemcpyDeviceToHost));
    for (long i = 0; i < n; ++i) t[i] *= (double)L.g.N;
    NLF_CUDA_TRY(cudaMemcpy(z, t.data(), n * 8, cudaMemcpyHostToDevice));
  } else {
    for (long i = 0; i < n; ++i) z[i] *= (double)L.g.N;
  }
  return NLF_OK;
}

NLF_API int nlf_mech_set_precond(nlf_mech* H, int precond) {
  if (!H || (precond != NLF_PC_FFT && precond != NLF_PC_FFT_SCALED)) {
    set_error("nlf_mech_set_precond: bad arguments");
    return NLF_EBADARG;
  }
  H->pc_mode = precond;
  return NLF_OK;
}

// displacement gradient at the Gauss points (mech.py:127-129): H (8, nx, ny, nz, 3, 3)
NLF_API int nlf_mech_grad_w(nlf_mech* H, const double* w, double* Hout, void* stream) {
  if (!H || !w || !Hout) {
    set_error("nlf_mech_grad_w: bad arguments");
    return NLF_EBADARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const long N = H->d.N;
  const size_t V = al(3 * N * 8);
  NLF_TRY(H->ws.reserve(V + al(72 * N * 8)));
  NLF_TRY(H->io.reserve(V));
  const double* wd = nullptr;
  NLF_TRY(stage(w, 3 * N, H->io, 0, &wd, st));
  double* ws = reinterpret_cast<double*>(H->ws.ptr);
  NLF_TRY((launch_aos_to_soa<double, double>(N, 1, wd, ws, 1.0, st)));
  double* hd = on_dev(Hout) ? Hout : reinterpret_cast<double*>((char*)H->ws.ptr + V);
  k_mech_gradw<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(N, H->d.n0, H->d.n1, H->d.n2, ws, hd);
  NLF_CHECK_LAUNCH();
  if (hd != Hout) NLF_TRY(copy_back(Hout, hd, 72 * N, st));
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  return NLF_OK;
}

NLF_API int nlf_mech_toec(nlf_mech* H, const double* chi, double* C, double* T, void* stream) {
  if (bad(H) || !chi || !C || !T) {
    if (H && H->rho_set) set_error("nlf_mech_toec: bad arguments");
    return NLF_EBADARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const long N = H->d.N;
  const int nblk = (int)std::min<long>(4 * 148, (N + kToecWarps - 1) / kToecWarps);
  const size_t o_soa = 0, o_part = al(18 * N * 8), o_out = o_part + al((size_t)nblk * kToecOut * 8);
  NLF_TRY(H->ws.reserve(o_out + al(kToecOut * 8)));
  NLF_TRY(H->io.reserve(al(18 * N * 8)));
  const double* cd = nullptr;
  NLF_TRY(stage(chi, 18 * N, H->io, 0, &cd, st));
  char* b = (char*)H->ws.ptr;
  double* soa = reinterpret_cast<double*>(b + o_soa);
  double* part = reinterpret_cast<double*>(b + o_part);
  double* out = reinterpret_cast<double*>(b + o_out);
  NLF_TRY((launch_aos_to_soa<double, double>(N, 6, cd, soa, 1.0, st)));
  static bool idx_ready[64] = {};  // the output -> index table, uploaded once per device
  static std::mutex idx_mu;
  int dev = 0;
  NLF_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_error("nlf_mech_toec: device index %d out of range", dev);
    return NLF_EBADARG;
  }
  {
    std::lock_guard<std::mutex> lock(idx_mu);
    if (!idx_ready[dev]) {
      signed char idx[kToecOut][3];
      int q = 0;
      for (int I = 0; I < 6; ++I)
        for (int J = I; J < 6; ++J, ++q) {
          idx[q][0] = (signed char)I;
          idx[q][1] = (signed char)J;
          idx[q][2] = 0;
        }
      for (int I = 0; I < 6; ++I)
        for (int J = I; J < 6; ++J)
          for (int K = J; K < 6; ++K, ++q) {
            idx[q][0] = (signed char)I;
            idx[q][1] = (signed char)J;
            idx[q][2] = (signed char)K;
          }
      NLF_CUDA_TRY(cudaMemcpyToSymbol(cToecIdx, idx, sizeof(idx)));
      idx_ready[dev] = true;
    }
  }
  {
    ProfScope ps(PK_MECH_ELEM, st);
    k_mech_toec<<<nblk, kToecThreads, 0, st>>>(H->d, soa, part);
    NLF_CHECK_LAUNCH();
    k_mech_toec_reduce<<<1, 128, 0, st>>>(part, nblk, H->d.wq, out);
    NLF_CHECK_LAUNCH();
  }
  double o[kToecOut];
  NLF_CUDA_TRY(cudaMemcpyAsync(o, out, sizeof(o), cudaMemcpyDeviceToHost, st));
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  // C, f''' as full symmetric arrays, then T = f''' - 3 Sym_IJK C(e_I, voigt(e_J e_K)) (mech.py:482-492)
  double Cm[6][6], T3[6][6][6];
  int q = 0;
  for (int I = 0; I < 6; ++I)
    for (int J = I; J < 6; ++J, ++q) Cm[I][J] = Cm[J][I] = o[q];
  for (int I = 0; I < 6; ++I)
    for (int J = I; J < 6; ++J)
      for (int K = J; K < 6; ++K, ++q) {
        const int p[6][3] = {{I, J, K}, {I, K, J}, {J, I, K}, {J, K, I}, {K, I, J}, {K, J, I}};
        for (auto& x : p) T3[x[0]][x[1]][x[2]] = o[q];
      }
  // X[:, J, K] = Voigt vector of the symmetric part of voigt(J) voigt(K)
  auto vt = [](int I, double (&M)[3][3]) {
    for (auto& r : M)
      for (double& x : r) x = 0.0;
    const int a = I < 3 ? I : (I == 3 ? 1 : 0), bb = I < 3 ? I : (I == 5 ? 1 : 2);
    if (I < 3) {
      M[a][a] = 1.0;
    } else {
      M[a][bb] = M[bb][a] = 0.5;
    }
  };
  double X[6][6][6];
  for (int J = 0; J < 6; ++J)
    for (int K = 0; K < 6; ++K) {
      double A[3][3], Bm[3][3], P[3][3];
      vt(J, A);
      vt(K, Bm);
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
          P[r][c] = 0.0;
          for (int m = 0; m < 3; ++m) P[r][c] += A[r][m] * Bm[m][c];
        }
      double S[3][3];
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) S[r][c] = 0.5 * (P[r][c] + P[c][r]);
      const double v[6] = {S[0][0], S[1][1], S[2][2], 2 * S[1][2], 2 * S[0][2], 2 * S[0][1]};
      for (int i = 0; i < 6; ++i) X[i][J][K] = v[i];
    }
  double CX[6][6][6];
  for (int i = 0; i < 6; ++i)
    for (int J = 0; J < 6; ++J)
      for (int K = 0; K < 6; ++K) {
        double a = 0.0;
        for (int m = 0; m < 6; ++m) a += Cm[i][m] * X[m][J][K];
        CX[i][J][K] = a;
      }
  double Ch[36], Th[216];
  for (int I = 0; I < 6; ++I)
    for (int J = 0; J < 6; ++J) {
      Ch[I * 6 + J] = Cm[I][J];
      for (int K = 0; K < 6; ++K) {
        const double sym = (CX[I][J][K] + CX[I][K][J] + CX[J][I][K] + CX[J][K][I] + CX[K][I][J] + CX[K][J][I]) / 6.0;
        Th[(I * 6 + J) * 6 + K] = T3[I][J][K] - 3.0 * sym;
      }
    }
  if (on_dev(C)) {
    NLF_CUDA_TRY(cudaMemcpy(C, Ch, sizeof(Ch), cudaMemcpyHostToDevice));
  } else {
    std::memcpy(C, Ch, sizeof(Ch));
  }
  if (on_dev(T)) {
    NLF_CUDA_TRY(cudaMemcpy(T, Th, sizeof(Th), cudaMemcpyHostToDevice));
  } else {
    std::memcpy(T, Th, sizeof(Th));
  }
  return NLF_OK;
}

// mech.py:264-290 _cg_impl at the linearization point (w, Fbar): solve H x = b for z-vectors
// (w (nx, ny, nz, 3) flattened, then the k macro unknowns Fbar[free[2j], free[2j+1]]).
// dmac: (k,) macro preconditioner diagonal; sws: stiffness scale of the w preconditioner.
// Outputs x (3N + k), *it, *conv, *neg (negative curvature met).
// graph captures of nlf_mech_cg (and the destruction of their executables) one at a time in the process
static std::mutex g_capture_mu;

NLF_API int nlf_mech_cg(nlf_mech* H, const double* w, const double* Fbar, int k, const int* free_idx,
                        const double* b, const double* dmac, double sws, double tol, int maxit, double* x, int* it,
                        int* conv, int* neg, int check_every, void* stream) {
  if (bad(H) || !w || !Fbar || !b || !x || k < 0 || k > 9 || (k > 0 && (!free_idx || !dmac)) || maxit < 0) {
    if (H && H->rho_set) set_error("nlf_mech_cg: bad arguments");
    return NLF_EBADARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  LinearHandle& L = lin_of(H);
  const long N = H->d.N;
  const long Lz = 3 * N + k;
  // workspace: w, b->r, x, p, Ap, zf, z0, fe, spec, partials, state
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += al(bytes);
    return o;
  };
  const size_t o_w = take(3 * N * 8), o_r = take(Lz * 8), o_x = take(Lz * 8), o_p = take(Lz * 8),
               o_ap = take(Lz * 8), o_zf = take(3 * N * 8), o_z0 = take(Lz * 8), o_fe = take(24 * N * 8),
               o_sp = take(3 * L.g.NS * 16), o_pa = take(4096 * 10 * 8), o_pc = take(3 * L.g.n0 * 4 * 8),
               o_fb = take(256), o_st = take(sizeof(MechCG));
  const bool cached = H->d.material == 1;
  const size_t o_tc = cached ? take((size_t)8 * kTanCache * N * 8) : 0;
  NLF_TRY(H->ws.reserve(off));
  NLF_TRY(H->io.reserve(2 * al(Lz * 8)));
  char* B = (char*)H->ws.ptr;
  double* ws = reinterpret_cast<double*>(B + o_w);
  double* r = reinterpret_cast<double*>(B + o_r);
  double* xs = reinterpret_cast<double*>(B + o_x);
  double* p = reinterpret_cast<double*>(B + o_p);
  double* Ap = reinterpret_cast<double*>(B + o_ap);
  double* zf = reinterpret_cast<double*>(B + o_zf);
  double* z0 = reinterpret_cast<double*>(B + o_z0);
  double* fe = reinterpret_cast<double*>(B + o_fe);
  cplx<double>* spec = reinterpret_cast<cplx<double>*>(B + o_sp);
  double* part = reinterpret_cast<double*>(B + o_pa);
  double* ppc = reinterpret_cast<double*>(B + o_pc);
  double* fbd = reinterpret_cast<double*>(B + o_fb);
  MechCG* stt = reinterpret_cast<MechCG*>(B + o_st);
  double* tc = cached ? reinterpret_cast<double*>(B + o_tc) : nullptr;
  // inputs: w -> SoA; b -> r (SoA w part + tail)
  const double *wd = nullptr, *bd = nullptr;
  NLF_TRY(stage(w, 3 * N, H->io, 0, &wd, st));
  NLF_TRY(stage(b, Lz, H->io, al(Lz * 8), &bd, st));
  NLF_TRY((launch_aos_to_soa<double, double>(N, 1, wd, ws, 1.0, st)));
  NLF_TRY((launch_aos_to_soa<double, double>(N, 1, bd, r, 1.0, st)));
  if (k) NLF_CUDA_TRY(cudaMemcpyAsync(r + 3 * N, bd + 3 * N, k * 8, cudaMemcpyDeviceToDevice, st));
  NLF_CUDA_TRY(cudaMemcpyAsync(fbd, Fbar, 72, on_dev(Fbar) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  if (cached) NLF_TRY(tan_cache(H, ws, fbd, tc, st));
  MechCG hs;
  std::memset(&hs, 0, sizeof(hs));
  hs.k = k;
  hs.maxit = maxit;
  hs.tol = tol;
  const bool scaled = H->pc_mode == NLF_PC_FFT_SCALED;
  const double* wpc = scaled ? H->wnode : nullptr;
  hs.scale = scaled ? (double)N : (double)N / sws;
  for (int j = 0; j < k; ++j) hs.dmac[j] = dmac[j];
  hs.done = maxit == 0 ? 1 : 0;
  NLF_CUDA_TRY(cudaMemcpyAsync(stt, &hs, sizeof(hs), cudaMemcpyHostToDevice, st));
  NLF_CUDA_TRY(cudaMemsetAsync(xs, 0, Lz * 8, st));
  const int vb = kCgBlocks, vt = 256;
  // b = proj(b) (mech.py:267)
  k_cg_dot<<<vb, vt, 0, st>>>(N, r, r, stt, part);
  k_cg_mean_sub<<<vb, vt, 0, st>>>(N, r, part, vb);
  NLF_CHECK_LAUNCH();
  // z0 = M b, p = z0, rz = (b, z0), bn = ||b||
  NLF_TRY(launch_precond<double>(L, 1, 1, r, zf, spec, wpc, nullptr, ppc, st));
  k_cg_fin_pc<<<1, 32, 0, st>>>(N, L.g.n0, ppc, r, stt, 1);
  k_cg_p<<<vb, vt, 0, st>>>(N, p, zf, r, z0, stt, 1);
  NLF_CHECK_LAUNCH();
  // the macro unknowns enter the element pass as dFm = sum_j p_tail[j] E_sel_j; built on the device
  FreeIdx fi{};
  fi.k = k;
  for (int j = 0; j < k; ++j) fi.ab[j] = 3 * free_idx[2 * j] + free_idx[2 * j + 1];
  const int every = check_every > 0 ? check_every : 8;
  int nb = 0;
  auto chunk = [&](cudaStream_t s) -> int {
    for (int q = 0; q < every; ++q) {
      k_cg_clear_ran<<<1, 1, 0, s>>>(stt);
      // Ap = H p; the macro part of p enters as dFm (fbd[9..17])
      k_cg_dfm<<<1, 32, 0, s>>>(p + 3 * N, fi, fbd + 9);
      if (cached)
        NLF_TRY(hvp_cached(H, p, fbd + 9, fi, fe, part, &nb, tc, s));
      else
        NLF_TRY(mech_pass<1>(H, ws, fbd, p, fbd + 9, fe, part, &nb, s));
      double* sum9 = part + 4096 * 9;
      k_mech_sum<9><<<1, kSumThreads, 0, s>>>(part, nb, sum9);
      NLF_TRY(gather(H, fe, Ap, s));
      if (k) k_cg_aptail<<<1, 32, 0, s>>>(sum9, fi, Ap + 3 * N);
      // proj(Ap) and pAp
      {
        ProfScope ps(PK_OTHER, s);
        k_cg_dot<<<vb, vt, 0, s>>>(N, Ap, p, stt, part + 4096 * 10 - 4 * vb);
        k_cg_fin_pap<<<1, 32, 0, s>>>(N, part + 4096 * 10 - 4 * vb, vb, p, Ap, stt);
        k_cg_xr<<<vb, vt, 0, s>>>(N, xs, r, p, Ap, z0, stt);
      }
      NLF_CHECK_LAUNCH();
      NLF_TRY(launch_precond<double>(L, 1, 1, r, zf, spec, wpc, nullptr, ppc, s));
      {
        ProfScope ps(PK_OTHER, s);
        k_cg_fin_pc<<<1, 32, 0, s>>>(N, L.g.n0, ppc, r, stt, 0);
        k_cg_p<<<vb, vt, 0, s>>>(N, p, zf, r, z0, stt, 0);
      }
      NLF_CHECK_LAUNCH();
    }
    return NLF_OK;
  };
  // graph replay of the chunk unless the profiler (per-launch events) is on
  cudaGraphExec_t gexec = nullptr;
  if (!prof_on()) {
    if (!H->gst) {
      NLF_CUDA_TRY(cudaStreamCreateWithFlags(&H->gst, cudaStreamNonBlocking));
      NLF_CUDA_TRY(cudaEventCreateWithFlags(&H->gev[0], cudaEventDisableTiming));
      NLF_CUDA_TRY(cudaEventCreateWithFlags(&H->gev[1], cudaEventDisableTiming));
    }
    cudaGraph_t graph = nullptr;
    // one capture at a time in the process, and no graph destroyed meanwhile: solves of different cells may run
    // from several host threads
    std::lock_guard<std::mutex> capture_lock(g_capture_mu);
    NLF_CUDA_TRY(cudaStreamBeginCapture(H->gst, cudaStreamCaptureModeThreadLocal));
    const int rc = chunk(H->gst);
    const cudaError_t e = cudaStreamEndCapture(H->gst, &graph);
    if (rc != NLF_OK || e != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      if (rc != NLF_OK) return rc;
      NLF_CUDA_TRY(e);
    }
    const cudaError_t ei = cudaGraphInstantiate(&gexec, graph, 0);
    cudaGraphDestroy(graph);
    NLF_CUDA_TRY(ei);
  }
  struct ExecGuard {
    cudaGraphExec_t g;
    ~ExecGuard() {
      if (g) {
        std::lock_guard<std::mutex> lock(g_capture_mu);
        cudaGraphExecDestroy(g);
      }
    }
  } guard{gexec};
  int host_done = hs.done, iters = 0;
  while (!host_done) {
    if (gexec) {
      NLF_CUDA_TRY(cudaEventRecord(H->gev[0], st));
      NLF_CUDA_TRY(cudaStreamWaitEvent(H->gst, H->gev[0], 0));
      NLF_CUDA_TRY(cudaGraphLaunch(gexec, H->gst));
      NLF_CUDA_TRY(cudaEventRecord(H->gev[1], H->gst));
      NLF_CUDA_TRY(cudaStreamWaitEvent(st, H->gev[1], 0));
    } else {
      NLF_TRY(chunk(st));
    }
    iters += every;
    NLF_CUDA_TRY(cudaMemcpyAsync(&hs, stt, sizeof(hs), cudaMemcpyDeviceToHost, st));
    NLF_CUDA_TRY(cudaStreamSynchronize(st));
    host_done = hs.done || iters >= maxit + every;
  }
  // x (SoA + tail) -> caller layout
  double* xo = on_dev(x) ? x : reinterpret_cast<double*>((char*)H->io.ptr);
  NLF_TRY((launch_soa_to_aos<double, double>(N, 1, xs, xo, st)));
  if (k) NLF_CUDA_TRY(cudaMemcpyAsync(xo + 3 * N, xs + 3 * N, k * 8, cudaMemcpyDeviceToDevice, st));
  if (xo != x) NLF_TRY(copy_back(x, xo, Lz, st));
  NLF_CUDA_TRY(cudaStreamSynchronize(st));
  if (it) *it = hs.it;
  if (conv) *conv = hs.conv;
  if (neg) *neg = hs.done && !hs.conv && hs.neg;
  return NLF_OK;
}

}  // extern "C"
