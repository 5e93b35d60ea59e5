/* nlfiber-b200: C ABI of the B200 (sm_100a) voxel homogenization hot path.
 *
 * One shared library, libnlf.so, replaces the hot path of the reference package nlfiber
 * (redcican/nonlinear-fiber-homogenization): the small-strain corrector solve of nlfiber/linear.py and the
 * matrix-free neo-Hookean residual / tangent matvec inside nlfiber/mech.py's Newton-CG.
 *
 * Conventions shared by every entry point
 *  - Plain pointers and sizes only. Any array argument may be a HOST pointer (the library copies it in or
 *    out on `stream`, synchronously for outputs) or a DEVICE pointer of the current device (used in place);
 *    the kind is detected per pointer.
 *  - Arrays use the reference layouts, C order, float64: a density or stiffness-scale field is (nx, ny, nz);
 *    a corrector / nodal field is (m, nx, ny, nz, 3) per cell; batched calls prepend the cell axis.
 *    2D (plane strain) cells are nz = 1 (nlfiber/linear.py:100-106).
 *  - `stream` is a cudaStream_t (NULL = legacy default stream).
 *  - Return codes: 0 ok; 1 not converged (outputs and iteration counts are still written; the reference
 *    returns silently with it == maxit, nlfiber/linear.py:188,217); 2 breakdown (non-finite values);
 *    -1 bad argument; -2 CUDA error; -3 device wait timed out. The message of the last error of the
 *    calling thread is returned by nlf_last_error(). Nothing aborts the process.
 */
#ifndef NLF_H_
#define NLF_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NLF_API __attribute__((visibility("default")))

typedef struct nlf_linear nlf_linear;
typedef struct nlf_mech nlf_mech;

/* Solver precision. */
#define NLF_PREC_FP64 0  /* the reference algorithm in FP64: the drop-in and the plain GPU baseline */
#define NLF_PREC_MIXED 1 /* FP32 operator + PCG inside FP64 iterative refinement; FP64 dots */

/* Preconditioner. */
#define NLF_PC_FFT 0        /* the reference's unit-stiffness FFT inverse (nlfiber/linear.py:154-170) */
#define NLF_PC_FFT_SCALED 1 /* S^-a K0^-1 S^-a, a = 0.47, with S the root mean square of the stiffness scales
                               of the 8 elements around each node and K0 the unit operator of a reference
                               medium with Poisson ratio 0 (same converged solution, far fewer iterations at
                               high contrast) */

typedef struct nlf_solve_opts {
  int precision;     /* NLF_PREC_* */
  int precond;       /* NLF_PC_* */
  double tol;        /* stop when every case of a cell has ||r|| <= tol ||b|| (< 0: use the handle's tol) */
  int maxit;         /* total PCG iterations per cell (< 0: use the handle's maxit) */
  double inner_tol;  /* NLF_PREC_MIXED: relative residual reduction of one FP32 inner solve */
  int inner_maxit;   /* NLF_PREC_MIXED: iteration cap of one FP32 inner solve */
  int max_sweeps;    /* NLF_PREC_MIXED: cap on FP64 refinement sweeps */
  int check_every;   /* host convergence poll period in iterations (>= 1) */
  int use_graphs;    /* capture check_every PCG iterations in a CUDA graph once per solve and replay it
                        (ignored while nlf_profile is on) */
  int slots;         /* NLF_PREC_FP64: cells solved at once (0 or >= ncell: all cells in lock-step). With
                        0 < slots < ncell a converged cell hands its slot to the next queued cell at the next
                        poll, so the batch stays full until the queue runs dry. Same per-cell result. */
  int scale_x0;      /* with an initial guess u0: start from beta u0 instead, beta (per case) minimising the
                        energy 1/2 x.Kx - b.x over the multiples of u0 (so never further from the solution in the
                        energy norm than u0 = 0). 0: the reference's start x0 = proj(u0). */
  double energy_tol; /* > 0 (solves from strains Es, FP64): energy guard. A cell stops only when, besides the
                        residual rule, the last 32 terms alpha_j (r_j, z_j) of its PCG sum to at most
                        energy_tol * N * max_J C_JJ for every case I. That sum estimates ||u_I - u*_I||_K^2 =
                        N (C_II(u) - C_II*) (Hestenes-Stiefel), which bounds every |C_IJ(u) - C*_IJ|; C_JJ comes
                        from the same recurrences. It keeps cells whose residual is small but whose C is not
                        (near-mechanisms of the solid) running; it never stops a cell earlier. 0: residual rule only. */
  int per_case;      /* > 0 (FP64 cubes of 32 or 64): per-case stopping. A load case stops on its own once the
                        residual rule (and the energy guard, if on) has held for this many consecutive iterations;
                        its corrector is then frozen while the cell's other cases go on, and the cell stops when all
                        its cases have (or by the lock-step rule). The probation guards against cases whose
                        residual dips below tol before a slow mode of the cell surfaces. 0: lock-step per cell, the
                        reference's rule (nlfiber/linear.py:185-188). */
} nlf_solve_opts;

NLF_API const char* nlf_last_error(void);
NLF_API const char* nlf_version(void);
NLF_API void nlf_default_opts(nlf_solve_opts* opts);

/* ---- small-strain homogenization (nlfiber/linear.py) --------------------------------------------------- */

/* nlfiber/linear.py:102-113 LinearHomogenization.__init__(shape, E, nu, emin, p, dtype, tol, maxit):
 * element matrices, preconditioner symbol and workspaces for one grid shape. */
NLF_API int nlf_linear_create(nlf_linear** h, int nx, int ny, int nz, double E, double nu, double emin,
                              double p, double tol, int maxit);
NLF_API int nlf_linear_destroy(nlf_linear* h);

/* nlfiber/linear.py:137-141 stiffness_scale: s = emin + (1 - emin) clip01(rho)^p for ncell cells. */
NLF_API int nlf_stiffness_scale(nlf_linear* h, int ncell, const double* rho, double* s, void* stream);

/* nlfiber/linear.py:143-144 apply_K: y = K(s) u for `nvec` nodal fields sharing one s (FP64). */
NLF_API int nlf_apply_K(nlf_linear* h, const double* s, int nvec, const double* u, double* y, void* stream);

/* apply_K in a chosen arithmetic: precision NLF_PREC_FP64 (as nlf_apply_K) or NLF_PREC_MIXED (the FP32
 * operator of the mixed-precision solver; inputs and outputs stay float64 arrays). */
NLF_API int nlf_apply_K_ex(nlf_linear* h, const double* s, int nvec, const double* u, double* y, int precision,
                           void* stream);

/* nlfiber/linear.py:146-149 load: f_I = a(E_I, .) for Es (m, 6); f is (m, nx, ny, nz, 3). */
NLF_API int nlf_load(nlf_linear* h, const double* s, const double* Es, int m, double* f, void* stream);

/* nlfiber/linear.py:167-170 precond: z = irfftn(Kinv rfftn(r)) for `nvec` fields (FP64). */
NLF_API int nlf_precond(nlf_linear* h, int nvec, const double* r, double* z, void* stream);

/* precond in a chosen arithmetic and preconditioner: precond NLF_PC_FFT (s ignored, may be NULL) or
 * NLF_PC_FFT_SCALED (s: the cell's stiffness scale (nx, ny, nz); z = w irfftn(Kinv0 rfftn(w r)) with
 * w = (root mean square of s over the 8 elements around each node)^-0.47 and Kinv0 the symbol inverse of the
 * same element with Poisson ratio 0). */
NLF_API int nlf_precond_ex(nlf_linear* h, int nvec, const double* r, double* z, int precision, int precond,
                           const double* s, void* stream);

/* nlfiber/linear.py:205-217 solve(s, Es, u0) -> (u, it) for ncell cells of this shape, m cases each.
 * s: (ncell, nx, ny, nz); Es: (m, 6); u0: (ncell, m, nx, ny, nz, 3) or NULL (zeros); u: same shape, out;
 * iters: (ncell,) out. opts NULL = FP64 reference algorithm with the handle's tol and maxit. */
NLF_API int nlf_linear_solve(nlf_linear* h, int ncell, const double* s, const double* Es, int m,
                             const double* u0, double* u, int* iters, const nlf_solve_opts* opts,
                             void* stream);

/* nlfiber/linear.py:208-210 _solve_rhs(s, b): PCG from zero for right-hand sides b (ncell, m, ..., 3). */
NLF_API int nlf_linear_solve_rhs(nlf_linear* h, int ncell, const double* s, int m, const double* b,
                                 double* u, int* iters, const nlf_solve_opts* opts, void* stream);

/* nlfiber/linear.py:220-229 bilinear(s, Es, u) -> C (ncell, m, m). */
NLF_API int nlf_bilinear(nlf_linear* h, int ncell, const double* s, const double* Es, int m,
                         const double* u, double* C, void* stream);

/* dC_IJ/drho_e with the correctors held fixed: the value of the reference's VJP of bilinear through
 * stiffness_scale (nlfiber/linear.py:10-12,137-141,220-229,259-264). rho: (ncell, nx, ny, nz);
 * dC: (ncell, m, m, nx, ny, nz). */
NLF_API int nlf_dC_drho(nlf_linear* h, int ncell, const double* rho, const double* Es, int m,
                        const double* u, double* dC, void* stream);

/* C_IJ assembly that allocates nothing (no counterpart in the reference). For callers that may not call
 * cudaMalloc while they run (a handler inside a framework that owns all device memory, code inside another
 * library's callback, a service with pre-reserved memory) and already hold device arrays: s (ncell, nx, ny, nz),
 * u (ncell, m, nx, ny, nz, 3) and C (ncell, m, m) must be device pointers of the current device; Es (m, 6) is a
 * host array. Same values as nlf_bilinear. No handle: the grid shape and material are arguments. At most 64
 * cells and 6 load cases per call (-1 with a message beyond). The partial sums live in a fixed 672 KiB device
 * array held by every GPU that loads the library; calls that overlap on the GPU race on it, so serialise them.
 * The first call on a device looks up that array's address; make it before any stream capture. That address
 * belongs to the device's context: after cudaDeviceReset of a device, do not call this entry point on it again.
 * Pointers into another GPU's memory are rejected (-1). Asynchronous on `stream`: C is ready when the stream
 * reaches it. */
NLF_API int nlf_bilinear_noalloc(int nx, int ny, int nz, double E, double nu, int ncell, const double* s,
                                 const double* Es, int m, const double* u, double* C, void* stream);

/* nlfiber/linear.py:118-134 the backward of `correctors`' custom VJP: for the cotangent ubar (ncell, m, nx, ny, nz,
 * 3) of the correctors u of (s, Es), lam solves K(s) lam = -proj(ubar) (PCG from zero with `opts`, as _solve_rhs)
 * and sbar_e = sum_I lam_I,e . (Ke u_I,e + G^T E_I), the VJP of residual(s, Es, u) in s. Give s (ncell, nx, ny,
 * nz), or rho instead of s: then s = stiffness_scale(rho) and sbar is the cotangent of rho (times ds/drho,
 * nlfiber/linear.py:137-141). Es (m, 6), m <= 6; lam (the shape of u) and iters (ncell) may be NULL. Returns the
 * solve's status. */
NLF_API int nlf_correctors_vjp(nlf_linear* h, int ncell, const double* s, const double* rho, const double* Es, int m,
                               const double* u, const double* ubar, double* sbar, double* lam, int* iters,
                               const nlf_solve_opts* opts, void* stream);

/* nlfiber/linear.py:231-236 C_full(rho, u0) for a batch: rho -> s -> 6 unit strains -> PCG -> C.
 * u0, u, dC may be NULL (cold start / corrector not returned / no sensitivities).
 * C: (ncell, 6, 6); u: (ncell, 6, nx, ny, nz, 3); dC: (ncell, 6, 6, nx, ny, nz); iters: (ncell,). */
NLF_API int nlf_C_full(nlf_linear* h, int ncell, const double* rho, const double* u0, double* C,
                       double* u, double* dC, int* iters, const nlf_solve_opts* opts, void* stream);

/* Kinv of the reference's preconditioner (nlfiber/linear.py:154-165), real symmetric 3x3 per wavenumber:
 * out (nx, ny, nz/2+1, 6) in the order xx yy zz yz xz xy. */
NLF_API int nlf_precond_symbol(nlf_linear* h, double* kinv6);

/* ---- tile autotuner (no counterpart in the reference, whose operator is a dense einsum that XLA compiles) ------
 * The stiffness apply has several tile variants (TY x TZ output tile of the (y, z) plane, minimum resident CTAs
 * per SM); variant 0 is the default. nlf_linear_autotune times every variant of one precision on `nvec`
 * synthetic vectors of the handle's grid (`reps` launches each, CUDA events on `stream`) and keeps the fastest
 * for this handle. Its choice is cached per (grid, precision) for the process, so later handles of the same grid
 * take it without timing unless `force` is set or `ms_out` (one time per variant, milliseconds per launch) is
 * given. On FP64 cubes of 32 or 64 it also times the preconditioner with its Kinv entries read from the table
 * (mode 0), computed in closed form (mode 1), or that with pass B's slabs staged through shared memory (mode 2,
 * 64^3 only; nlf_linear_set_kinv_mode), and passes A and C with their
 * twiddles in registers (0), read from a shared-memory copy of the tables at 3 CTAs per SM (1), that with pass
 * C's spectrum rows and x/p update moved in whole rows through shared memory (2; pass C at 4 CTAs per SM at
 * 64^3), or with pass A's row inputs
 * coalesced the same way too (3;
 * nlf_linear_set_fft_twiddles): ms_out[nvariants + kinv mode + nk twiddle mode], nk = 3 Kinv modes at 64^3
 * and 2 at 32^3, so at most twelve entries. Results of
 * different variants agree to rounding (the apply's partial sums follow the tile), and one handle's results do not
 * depend on the batch. Synchronizes the stream. */
NLF_API int nlf_apply_variants(int precision);
NLF_API int nlf_linear_set_kinv_mode(nlf_linear* h, int mode);
NLF_API int nlf_linear_get_kinv_mode(nlf_linear* h);
NLF_API int nlf_linear_set_fft_twiddles(nlf_linear* h, int shared);
NLF_API int nlf_linear_get_fft_twiddles(nlf_linear* h);
NLF_API int nlf_linear_set_apply_variant(nlf_linear* h, int precision, int variant);
NLF_API int nlf_linear_get_apply_variant(nlf_linear* h, int precision, int* variant, int* ty, int* tz, int* minb);
NLF_API int nlf_linear_autotune(nlf_linear* h, int precision, int nvec, int reps, int force, double* ms_out,
                                void* stream);

/* ---- finite-strain homogenization (nlfiber/mech.py) ------------------------------------------------------- */

/* nlfiber/mech.py:91-103 Cell(rho, E, nu, material, wls, emin, p) without the density: material 0 = linear,
 * 1 = neo-Hookean; wls_b <= 0 means no void interpolation (wls=None). */
NLF_API int nlf_mech_create(nlf_mech** h, int nx, int ny, int nz, double E, double nu, int material, double wls_b,
                            double wls_r0, double emin, double p);
NLF_API int nlf_mech_destroy(nlf_mech* h);
/* mech.py:101-113,292-294: s = emin + (1 - emin) clip01(rho)^p and the WLS gamma on the device; optional copies of
 * s, gamma (nx, ny, nz) and the preconditioner scale sws = exp(mean log s). */
NLF_API int nlf_mech_set_rho(nlf_mech* h, const double* rho, double* s, double* gamma, double* sws, void* stream);
/* mech.py:141-152,166-169,191-192 energy / jax.grad: W = wq sum_g sum_e s psi_eff(Fbar + H_g); gw = dW/dw
 * (nx, ny, nz, 3) and P = dW/dFbar (3, 3, the mean stress) when not NULL. */
NLF_API int nlf_mech_energy(nlf_mech* h, const double* w, const double* Fbar, double* W, double* gw, double* P,
                            void* stream);
/* mech.py:154-164,227-238 tangent_g + hvp_A, matrix-free: the second derivative of W at (w, Fbar) applied to the
 * direction (v (nx, ny, nz, 3), dFbar (3, 3)) -> (hv (nx, ny, nz, 3), hP (3, 3)). */
NLF_API int nlf_mech_hvp(nlf_mech* h, const double* w, const double* Fbar, const double* v, const double* dFbar,
                         double* hv, double* hP, void* stream);
/* mech.py:172-189 precond_w: inverse of the homogeneous unit-stiffness operator (N x the linear symbol). */
NLF_API int nlf_mech_precond_w(nlf_mech* h, const double* r, double* z, void* stream);
/* Preconditioner of nlf_mech_cg and nlf_mech_precond_w: NLF_PC_FFT (default) is the reference's
 * N K0^-1 / sws (mech.py:264-294); NLF_PC_FFT_SCALED is N w K0'^-1 w with w the node stiffness scaling and K0'
 * the Poisson-ratio-0 reference medium of nlf_precond_ex (sws then unused). Same Newton-CG solution to the same tolerances; far fewer CG iterations
 * at high contrast. No counterpart in the reference. */
NLF_API int nlf_mech_set_precond(nlf_mech* h, int precond);
/* mech.py:127-129 grad_w: displacement gradient at the Gauss points, H (8, nx, ny, nz, 3, 3). */
NLF_API int nlf_mech_grad_w(nlf_mech* h, const double* w, double* H, void* stream);
/* mech.py:264-290 _cg_impl at the linearization point (w, Fbar) with k free macro components
 * free_idx = (a0, b0, a1, b1, ...): PCG for H x = b on z-vectors (3N + k: w then the macro unknowns), with the
 * reference's guards (negative curvature exit, x = M b if it happens at the first iteration). */
NLF_API int nlf_mech_cg(nlf_mech* h, const double* w, const double* Fbar, int k, const int* free_idx, const double* b,
                        const double* dmac, double sws, double tol, int maxit, double* x, int* it, int* conv, int* neg,
                        int check_every, void* stream);

/* nlfiber/mech.py:458-493 toec(cell, chi): C (6, 6) and the Lagrangian-strain third-order elastic constants
 * T (6, 6, 6) of the cell (its s and gamma from nlf_mech_set_rho, its material) from the linear correctors chi
 * (6, nx, ny, nz, 3) of the 6 unit Voigt strains (same stiffness scale, E and nu): C = f''(0),
 * T = f'''(0) - 3 Sym C(e_I, voigt(e_J e_K)) with f(s) = wq sum_{g,e} s_e psi_eff(I + sum_I s_I H_I),
 * H_I = voigt(I) + grad chi_I. The reference differentiates f by autodiff; here f'' and f''' at F = I are
 * closed forms (the neo-Hookean energy's; zero third derivative for the linear material). C, T host or device. */
NLF_API int nlf_mech_toec(nlf_mech* cell, const double* chi, double* C, double* T, void* stream);

/* ---- learned warm start ----------------------------------------------------------------------------------
 * A 3-level U-Net (widths w0, w1, w2; periodic 3x3x3 convolutions, ReLU, 2x average pooling, nearest
 * upsampling with skip concatenation, a final 1x1 convolution to 18 channels) maps a density cell to the 6
 * unit-strain correctors as u / nx (channels-last, case-major: channel 3 I + c). Its prediction is the u0 of
 * nlf_C_full / nlf_linear_solve. No counterpart in the reference, whose solve always starts from u0 = 0
 * (nlfiber/linear.py:209-212, the u0 argument of solve and C_full :231-236). The convolutions run as BF16
 * implicit GEMMs on the tensor cores with FP32 accumulation; parameters, gradients and Adam moments are FP32.
 * Flat parameter layout: per layer W (ntaps, cout, cin) then b (cout), layers in network order. */
typedef struct nlf_unet nlf_unet;

/* widths multiples of 16 with w1 + w0 <= 128 and w2 + w1 <= 128; He-normal weights from `seed`. */
NLF_API int nlf_unet_create(nlf_unet** out, int w0, int w1, int w2, unsigned long long seed);
NLF_API int nlf_unet_destroy(nlf_unet* net);
NLF_API long long nlf_unet_param_count(const nlf_unet* net);
/* FP32 parameters to / from a host or device buffer of nlf_unet_param_count floats; set_params also resets the
 * Adam state. */
NLF_API int nlf_unet_get_params(nlf_unet* net, float* out, void* stream);
NLF_API int nlf_unet_set_params(nlf_unet* net, const float* in, void* stream);
/* y (nb, nx, ny, nz, 18) = net(rho (nb, nx, ny, nz)); device FP32 buffers; nx, ny, nz divisible by 4. */
NLF_API int nlf_unet_forward(nlf_unet* net, int nb, int nx, int ny, int nz, const float* rho, float* y,
                             void* stream);
/* loss = sum_v weight[v] sum_c (y - target)^2 / 18 and its gradient w.r.t. the parameters (kept for
 * nlf_unet_adam_step; also copied to `grad` when not NULL, host or device). rho, target, weight: device FP32. */
NLF_API int nlf_unet_backward(nlf_unet* net, int nb, int nx, int ny, int nz, const float* rho, const float* target,
                              const float* weight, double* loss, float* grad, void* stream);
/* One Adam step (Kingma & Ba 2015, bias-corrected) with the gradient of the last nlf_unet_backward. */
NLF_API int nlf_unet_adam_step(nlf_unet* net, double lr, double beta1, double beta2, double eps, void* stream);

/* ---- density map (nlfiber/density.py, nlfiber/symmetry.py) ------------------------------------------------
 * The input side of the solve: a pre-density phi on the symmetric octant (n_o)^3 becomes the physical density
 * rho of the full periodic cell (2 n_o)^3 with mean(rho) = v exactly; on squares (d = 2) the quadrant (n_o)^2
 * becomes the cell (2 n_o)^2. Below, read (n_o, n_o, n_o) and (n, n, n) as (n_o, n_o) and (n, n) for squares. */
typedef struct nlf_density nlf_density;

/* nlfiber/density.py:75-82 DensityMap.__init__(n_o, d, r, v) without v: the periodic cone filter of radius r
 * voxels (density.py:23-31; at most 8192 nonzero taps) and the symmetry orbits of the octant (quadrant)
 * (symmetry.py:74-96). nlf_density_create is nlf_density_create_d with d = 3. */
NLF_API int nlf_density_create(nlf_density** out, int n_o, double r);
NLF_API int nlf_density_create_d(nlf_density** out, int n_o, int d, double r);
NLF_API int nlf_density_destroy(nlf_density* dm);
/* Number of symmetry orbits of the octant (sorted index triples; pairs on squares; symmetry.py:20-22 n_free);
 * -1 for NULL. */
NLF_API int nlf_density_orbits(const nlf_density* dm);
/* nlfiber/density.py:84-94 DensityMap.smooth and rho (threshold / solve_eta, density.py:43-72) for ncell cells:
 * phi (ncell, n_o, n_o, n_o) octant pre-densities (symmetrized here, as sym_perm does in smooth); v (ncell,) the
 * volume fraction of each cell; beta > 0 the sharpness. Outputs, each NULL when not wanted (at least one):
 * rho (ncell, n, n, n); u (ncell, n, n, n) the smoothed, exactly symmetric field of DensityMap.smooth;
 * eta (ncell,) the threshold with mean(sigmoid(beta (u - eta))) = v. The filter is applied as a direct periodic
 * sum over its taps (the reference multiplies FFTs: equal to rounding). */
NLF_API int nlf_density_rho(nlf_density* dm, int ncell, const double* phi, const double* v, double beta,
                            double* rho, double* u, double* eta, void* stream);

/* Vector-Jacobian product of nlf_density_rho (what JAX's reverse mode gives for DensityMap.rho,
 * nlfiber/density.py:66-94, with the implicit d eta of `threshold`): for nrow cotangents rho_bar (ncell, nrow,
 * n, n, n) of rho, phi_bar (ncell, nrow, n_o, n_o, n_o) = (d rho / d phi)^T rho_bar. Recomputes the forward map.
 * nlfiber/fiber.py:34-39 (Fiber.value_and_jac) pulls the 3 rows of dc/drho back through this map. */
NLF_API int nlf_density_vjp(nlf_density* dm, int ncell, int nrow, const double* phi, const double* v, double beta,
                            const double* rho_bar, double* phi_bar, void* stream);

/* ---- binary cells (nlfiber/density.py:96-149, nlfiber/topology.py:8-63) ------------------------------------
 * The binary check of a design: the smoothed field thresholded at its volume fraction, floating solid removed
 * and the volume grown back. A topology handle serves one cell side n (n^3 voxels, n^2 on squares, at most
 * 2^30); b is a byte per voxel (0 void, 1 solid; NumPy bool), C order. Host or device pointers. A handle is not
 * shared between host threads. */
typedef struct nlf_topo nlf_topo;

NLF_API int nlf_topo_create(nlf_topo** out, int d, int n);
NLF_API int nlf_topo_destroy(nlf_topo* t);
/* nlfiber/topology.py:8-43 periodic_label: connected components of the periodic cell, 26 neighbours (8 on
 * squares) or, with faces = 1, the 6 faces (4 edges; the void's dual connectivity, topology.py:90). labels[i]
 * is 1..ncomp, numbered in the order of each component's first voxel (the reference numbers them in its own
 * scan order: the same components), 0 for void. */
NLF_API int nlf_topo_label(nlf_topo* t, const uint8_t* b, int faces, int32_t* labels, int* ncomp, void* stream);
/* nlfiber/topology.py:46-63 remove_floating, in place: keeps the components (26 / 8 neighbours) that touch
 * every slice along every axis. Optional outputs: components, spanning components, solid voxels kept. */
NLF_API int nlf_topo_remove_floating(nlf_topo* t, uint8_t* b, int* ncomp, int* nspan, long long* nsolid,
                                     void* stream);
/* The rank-th smallest (0-based) of u over the voxels where mask != 0 (all voxels when mask is NULL). */
NLF_API int nlf_topo_select(nlf_topo* t, const double* u, const uint8_t* mask, long long rank, double* value,
                            void* stream);
/* nlfiber/density.py:96-122 DensityMap.binary after the smoothing: u (the smoothed, exactly symmetric field of
 * nlf_density_rho, upsampled by nlf_upsample_sym when up > 1) -> b = u > quantile(u, 1 - v); with
 * remove_floating, floating pieces are removed and the solid grown back towards v through the void voxels that
 * touch it, highest u first (at most 500 rounds, the number run in *iters), then removed once more. */
NLF_API int nlf_topo_binary(nlf_topo* t, const double* u, double v, int remove_floating, uint8_t* b, int* iters,
                            void* stream);
/* nlfiber/density.py:133-149 upsample_periodic of a cell-centred field of side n to side m, then
 * nlfiber/symmetry.py:60-65 exact_symmetrize: out has side 2 (m / 2). Bitwise numpy's arithmetic. */
NLF_API int nlf_upsample_sym(int d, int n, int m, const double* u, double* out, void* stream);
/* numpy's default ("linear") quantile q of n sorted host values, with numpy's rounding: the interpolation
 * nlf_topo_binary applies to its two order statistics. Host only. */
NLF_API int nlf_quantile_linear(long long n, double q, const double* sorted, double* out);

/* ---- kernel profiler ------------------------------------------------------------------------------------- */

/* Turns the kernel-level profiler on (1) or off (0) and resets it. When on, every kernel launch of the library
 * is bracketed by CUDA events on its stream and the units of work that actually ran (vectors of active cells)
 * are counted on the device. Process-wide and not thread-safe; off by default. No counterpart in the
 * reference (which has no tracing, nlfiber/qoi.py:81,106 only records wall-clock seconds). */
NLF_API int nlf_profile(int on);
/* Per kernel class k < n (n >= the number of classes): total event-timed milliseconds, launches and units.
 * Synchronizes the device. Returns the number of classes. */
NLF_API int nlf_profile_report(double* total_ms, long long* launches, unsigned long long* units, int n);
/* Name of kernel class k ("apply_f32", "fft_a_f32", ...); "" when out of range. */
NLF_API const char* nlf_profile_name(int kind);

#ifdef __cplusplus
}
#endif
#endif /* NLF_H_ */
