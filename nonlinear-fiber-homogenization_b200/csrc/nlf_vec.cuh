// Launchers of the PCG vector and reduction kernels (nlf_vec.cu).
#pragma once
#include <algorithm>
#include "nlf_internal.h"

namespace nlf {

constexpr int kStatsBlocks = 64;

int launch_node_scaling(const LinearHandle& h, int ncell, const double* s, float* s32, double* w64, float* w32,
                        cudaStream_t st);
template <typename T>
int launch_stats(const LinearHandle& h, int nvec, int m, const T* x, const CellState* cs, double* partial,
                 VecState* vs, int what, cudaStream_t st);
template <typename T>
int launch_sub_mean(const LinearHandle& h, int nvec, int m, T* x, const VecState* vs, const CellState* cs,
                    cudaStream_t st);
int launch_fin_apply(int nvec, int m, const double* partial, int nblk, long N, VecState* vs, const CellState* cs,
                     int init, cudaStream_t st);
template <typename Tb, typename T>
int launch_r_init(long N, int nvec, int m, T* r, const Tb* b, const T* Ax, const VecState* vs, const CellState* cs,
                  cudaStream_t st);
int launch_fin_pc(int ncell, int m, int n0, long N, const double* partial, VecState* vs, CellState* cs, double tol,
                  int maxit, int init, cudaStream_t st);
template <typename T>
int launch_p(long N, int nvec, int m, T* p, const T* z, const VecState* vs, const CellState* cs, int init,
             cudaStream_t st);
// fused iteration: (r, z), sums and the lock-step control from the FFT passes' partials; x and p updates together.
// probation > 0 (per-case stopping): a load case stops on its own once both stopping rules have held for that many
// consecutive iterations (CellState::stopped); the cell stops when all its cases have, or by the lock-step rule.
int launch_fin_pc_fused(int ncell, int m, int n0, int n1, long N, const double* partA, const double* partB,
                        const double* partC, int nchunk, VecState* vs, CellState* cs, double tol, int maxit,
                        double* ring, double etol, int probation, cudaStream_t st);
// energy stopping rule, at the start of a solve: ebase = ede[I] sum(s of the cell) (+ x0.K x0 - 2 (b, x0) when
// x_given; Ax holds K x0 and its means), esum = 0
template <typename Tb, typename T>
int launch_energy_init(const LinearHandle& h, int ncell, int m, const T* s, const Ede& ede, const Tb* b, const T* x,
                       const T* Ax, bool x_given, const CellState* cs, double* partial, VecState* vs,
                       cudaStream_t st);
template <typename T>
int launch_px(long N, int nvec, int m, T* x, T* p, const T* z, const VecState* vs, const CellState* cs,
              cudaStream_t st);
// x <- beta x, Ax <- beta Ax (and its means) with beta = (b, x) / (x, Ax - mean Ax) per vector (0 if not positive)
template <typename Tb, typename T>
int launch_x0_scale(const LinearHandle& h, int nvec, int m, const Tb* b, T* x, T* Ax, const CellState* cs,
                    double* partial, VecState* vs, cudaStream_t st);
int launch_mark(CellState* cs, int ncell, cudaStream_t st);
int launch_cs_init(CellState* cs, int ncell, const int* mask, cudaStream_t st);
int launch_count_active(const CellState* cs, int ncell, int* out, cudaStream_t st);
int launch_r_to32(long N, int nvec, int m, const double* r64, float* r32, VecState* vs, const CellState* cs,
                  cudaStream_t st);
int launch_x_update(long N, int nvec, int m, double* x64, const float* x32, const VecState* vs, const CellState* cs,
                    cudaStream_t st);

}  // namespace nlf
