// XLA FFI custom-call target of the corrector solve, for callers inside jax.jit / jax.vjp (nlfiber/fiber.py:27-39
// calls LinearHomogenization.invariants there; the solve sits under stop_gradient, nlfiber/linear.py:259-264).
//
// Built only where jaxlib's FFI headers exist (the Makefile's `jax` target asks jax.ffi.include_dir()); it links
// libnlf.so and calls its C ABI with XLA's device buffers, which the ABI uses in place. Registered from Python by
// nlfiber_b200.jax_ffi as "nlf_linear_solve" on the CUDA platform.
//
//   operands : s (ncell, nx, ny, nz) f64, Es (m, 6) f64, u0 (ncell, m, nx, ny, nz, 3) f64
//   results  : u (ncell, m, nx, ny, nz, 3) f64, iterations (ncell,) s32
//   attributes: E, nu, emin, p, tol (f64), maxit, precond (0 the reference's FFT inverse, 1 node-scaled), slots
//   (i64)
//
// Es is read on the host by the ABI's load assembly, so it must be a host-visible copy: the handler copies the
// (m, 6) block to the host on the call's stream first. Handles (element matrices, Kinv tables, workspace) are
// cached per (shape, material) for the process; a solve synchronizes the stream (the library polls convergence).
#include <cuda_runtime.h>

#include <array>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "nlf.h"
#include "xla/ffi/api/ffi.h"

namespace ffi = xla::ffi;

namespace {

using Key = std::tuple<int, int, int, double, double, double, double>;
std::mutex g_mu;
std::map<Key, nlf_linear*> g_handles;

nlf_linear* handle_for(int nx, int ny, int nz, double E, double nu, double emin, double p, std::string* err) {
  std::lock_guard<std::mutex> lk(g_mu);
  const Key k{nx, ny, nz, E, nu, emin, p};
  auto it = g_handles.find(k);
  if (it != g_handles.end()) return it->second;
  nlf_linear* h = nullptr;
  if (nlf_linear_create(&h, nx, ny, nz, E, nu, emin, p, 1e-9, 4000) != 0) {
    *err = nlf_last_error();
    return nullptr;
  }
  g_handles[k] = h;
  return h;
}

ffi::Error LinearSolve(cudaStream_t stream, ffi::Buffer<ffi::F64> s, ffi::Buffer<ffi::F64> Es,
                       ffi::Buffer<ffi::F64> u0, ffi::ResultBuffer<ffi::F64> u, ffi::ResultBuffer<ffi::S32> iters,
                       double E, double nu, double emin, double p, double tol, int64_t maxit, int64_t precond,
                       int64_t slots) {
  const auto sd = s.dimensions();
  const auto ed = Es.dimensions();
  if (sd.size() != 4 || ed.size() != 2 || ed[1] != 6)
    return ffi::Error::InvalidArgument("nlf_linear_solve: s must be (ncell, nx, ny, nz) and Es (m, 6)");
  const int ncell = static_cast<int>(sd[0]), nx = static_cast<int>(sd[1]), ny = static_cast<int>(sd[2]),
            nz = static_cast<int>(sd[3]), m = static_cast<int>(ed[0]);
  std::string err;
  nlf_linear* h = handle_for(nx, ny, nz, E, nu, emin, p, &err);
  if (!h) return ffi::Error::Internal("nlf_linear_create: " + err);
  std::vector<double> es(static_cast<size_t>(m) * 6);
  if (cudaMemcpyAsync(es.data(), Es.typed_data(), es.size() * sizeof(double), cudaMemcpyDeviceToHost, stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return ffi::Error::Internal("nlf_linear_solve: copy of Es failed");
  nlf_solve_opts o;
  nlf_default_opts(&o);
  o.tol = tol;
  o.maxit = static_cast<int>(maxit);
  o.precond = static_cast<int>(precond);
  o.slots = static_cast<int>(slots);
  o.use_graphs = 1;
  o.check_every = 16;
  const int st = nlf_linear_solve(h, ncell, s.typed_data(), es.data(), m, u0.typed_data(), u->typed_data(),
                                  iters->typed_data(), &o, stream);
  if (st < 0) return ffi::Error::Internal(std::string("nlf_linear_solve: ") + nlf_last_error());
  return ffi::Error::Success();  // not converged (1) is the reference's silent it == maxit
}

}  // namespace

XLA_FFI_DEFINE_HANDLER_SYMBOL(NlfLinearSolve, LinearSolve,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()  // s
                                  .Arg<ffi::Buffer<ffi::F64>>()  // Es
                                  .Arg<ffi::Buffer<ffi::F64>>()  // u0
                                  .Ret<ffi::Buffer<ffi::F64>>()  // u
                                  .Ret<ffi::Buffer<ffi::S32>>()  // iterations
                                  .Attr<double>("E")
                                  .Attr<double>("nu")
                                  .Attr<double>("emin")
                                  .Attr<double>("p")
                                  .Attr<double>("tol")
                                  .Attr<int64_t>("maxit")
                                  .Attr<int64_t>("precond")
                                  .Attr<int64_t>("slots"));
