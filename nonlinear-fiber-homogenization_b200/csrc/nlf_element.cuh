// Trilinear hexahedron (Q1, unit cube, isotropic material) element operator in mode form.
//
// The reference forms the element stiffness Ke = sum_g B_g^T D B_g / 8 with 2x2x2 Gauss points and applies it
// as a dense 24x24 matvec (nlfiber/linear.py:57-71,108-112,143-144). Because 2x2x2 Gauss integrates the Q1
// energy of a unit cube exactly, Ke equals the exact element stiffness, which is block-diagonal in the
// Hadamard ("mode") basis of the trilinear field: u = sum_p c_p xi^px eta^py zeta^pz on [-1/2, 1/2]^3 with
// the Legendre-orthogonal weights 1, 1/12, 1/144. Ke u_e is therefore
//   c  = H u        (sum/difference butterfly along x, y, z; 23 adds per component)
//   f  = M(s) c     (constant-strain mode, three shear-bending modes coupled pairwise, the twist mode)
//   Ke u = H^T f    (transposed butterfly)
// which is ~200 flops instead of 1152, with the same value to rounding. Node order a = ax + 2ay + 4az
// (x is the slowest array axis, z the fastest), mode index p = px + 2py + 4pz.
#pragma once
#include "nlf_common.cuh"

namespace nlf {

// Material constants of the mode operator for unit stiffness scale, already divided by the butterfly
// normalisation (c' = 2^{#zeros(p)} c): l1 = lam/16, m1 = mu/16, l2 = lam/48, m2 = mu/48,
// k7 = (lam + 4 mu)/144.
template <typename T>
struct ModeC {
  T l1, m1, l2, m2, k7;
};

template <typename T>
__host__ __device__ inline ModeC<T> make_modec(double lam, double mu) {
  ModeC<T> c;
  c.l1 = (T)(lam / 16.0);
  c.m1 = (T)(mu / 16.0);
  c.l2 = (T)(lam / 48.0);
  c.m2 = (T)(mu / 48.0);
  c.k7 = (T)((lam + 4.0 * mu) / 144.0);
  return c;
}

// In-place forward butterfly of 8 corner values -> 8 mode coefficients (unnormalised sums/differences).
template <typename T>
__device__ __forceinline__ void butterfly8(T (&v)[8]) {
#pragma unroll
  for (int a = 0; a < 8; a += 2) {  // x pairs (a, a+1)
    T s = v[a] + v[a + 1], d = v[a + 1] - v[a];
    v[a] = s;
    v[a + 1] = d;
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {  // y pairs (a, a+2)
    int a = (q & 1) + ((q >> 1) << 2);
    T s = v[a] + v[a + 2], d = v[a + 2] - v[a];
    v[a] = s;
    v[a + 2] = d;
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {  // z pairs (a, a+4)
    T s = v[a] + v[a + 4], d = v[a + 4] - v[a];
    v[a] = s;
    v[a + 4] = d;
  }
}

// Transposed butterfly: mode forces -> 8 nodal forces. (s, d) -> (s - d, s + d) per level.
template <typename T>
__device__ __forceinline__ void butterfly8_t(T (&v)[8]) {
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    T s = v[a], d = v[a + 4];
    v[a] = s - d;
    v[a + 4] = s + d;
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    int a = (q & 1) + ((q >> 1) << 2);
    T s = v[a], d = v[a + 2];
    v[a] = s - d;
    v[a + 2] = s + d;
  }
#pragma unroll
  for (int a = 0; a < 8; a += 2) {
    T s = v[a], d = v[a + 1];
    v[a] = s - d;
    v[a + 1] = s + d;
  }
}

// Mode-space force f = M c for mode coefficients c[comp][p] (p = 1..7 used; c[*][0] ignored).
// The result f[comp][p] has f[*][0] = 0. Constants `k` already include the element stiffness scale.
template <typename T>
__device__ __forceinline__ void mode_force(const T (&c)[3][8], const ModeC<T>& k, T (&f)[3][8]) {
  // constant-strain mode: H[comp][d] = c[comp][1 << d]
  {
    const T h00 = c[0][1], h01 = c[0][2], h02 = c[0][4];
    const T h10 = c[1][1], h11 = c[1][2], h12 = c[1][4];
    const T h20 = c[2][1], h21 = c[2][2], h22 = c[2][4];
    const T ltr = k.l1 * (h00 + h11 + h22);
    const T m2 = k.m1 + k.m1;
    const T s01 = k.m1 * (h01 + h10), s02 = k.m1 * (h02 + h20), s12 = k.m1 * (h12 + h21);
    f[0][1] = ltr + m2 * h00;
    f[1][2] = ltr + m2 * h11;
    f[2][4] = ltr + m2 * h22;
    f[1][1] = s01;  // sigma[1][x]
    f[0][2] = s01;  // sigma[0][y]
    f[2][1] = s02;  // sigma[2][x]
    f[0][4] = s02;  // sigma[0][z]
    f[2][2] = s12;  // sigma[2][y]
    f[1][4] = s12;  // sigma[1][z]
  }
  // shear-bending modes: a = c[.][3] (x,y), b = c[.][5] (x,z), g = c[.][6] (y,z)
  {
    const T a0 = c[0][3], a1 = c[1][3], a2 = c[2][3];
    const T b0 = c[0][5], b1 = c[1][5], b2 = c[2][5];
    const T g0 = c[0][6], g1 = c[1][6], g2 = c[2][6];
    const T l = k.l2, m = k.m2, m2 = k.m2 + k.m2;
    const T trx = l * (a1 + b2);  // mode xi:   H[.][y] = a, H[.][z] = b
    const T tre = l * (a0 + g2);  // mode eta:  H[.][x] = a, H[.][z] = g
    const T trz = l * (b0 + g1);  // mode zeta: H[.][x] = b, H[.][y] = g
    const T ba = m * (b1 + a2), ag = m * (a2 + g0), bg = m * (b1 + g0);
    // f3 = sigma_xi[.][y] + sigma_eta[.][x]
    f[0][3] = m * a0 + (tre + m2 * a0);
    f[1][3] = (trx + m2 * a1) + m * a1;
    f[2][3] = ba + ag;
    // f5 = sigma_xi[.][z] + sigma_zeta[.][x]
    f[0][5] = m * b0 + (trz + m2 * b0);
    f[1][5] = ba + bg;
    f[2][5] = (trx + m2 * b2) + m * b2;
    // f6 = sigma_eta[.][z] + sigma_zeta[.][y]
    f[0][6] = ag + bg;
    f[1][6] = m * g1 + (trz + m2 * g1);
    f[2][6] = (tre + m2 * g2) + m * g2;
  }
  f[0][7] = k.k7 * c[0][7];
  f[1][7] = k.k7 * c[1][7];
  f[2][7] = k.k7 * c[2][7];
  f[0][0] = T(0);
  f[1][0] = T(0);
  f[2][0] = T(0);
}

template <typename T>
__device__ __forceinline__ ModeC<T> scale_modec(const ModeC<T>& k, T s) {
  return ModeC<T>{k.l1 * s, k.m1 * s, k.l2 * s, k.m2 * s, k.k7 * s};
}

// Element force: v[comp][a] (nodal values, overwritten) -> f[comp][a] = s Ke u_e.
template <typename T>
__device__ __forceinline__ void element_force(T (&v)[3][8], const ModeC<T>& ks, T (&f)[3][8]) {
  butterfly8(v[0]);
  butterfly8(v[1]);
  butterfly8(v[2]);
  mode_force(v, ks, f);
  butterfly8_t(f[0]);
  butterfly8_t(f[1]);
  butterfly8_t(f[2]);
}

}  // namespace nlf
