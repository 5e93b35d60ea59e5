// Kernel-level profiler (see nlf_prof.cuh) and its C ABI.
#include <vector>
#include "nlf_internal.h"
#include "nlf_prof.cuh"

namespace nlf {

namespace {
struct Rec {
  int kind;
  cudaEvent_t a, b;
};
bool g_on = false;
std::vector<Rec> g_recs;
std::vector<cudaEvent_t> g_pool;
unsigned long long* g_units = nullptr;

cudaEvent_t take_event() {
  if (!g_pool.empty()) {
    cudaEvent_t e = g_pool.back();
    g_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

void recycle() {
  for (auto& r : g_recs) {
    g_pool.push_back(r.a);
    g_pool.push_back(r.b);
  }
  g_recs.clear();
}

const char* kNames[PK_COUNT] = {"apply_f32", "apply_f64", "fft_a_f32", "fft_b_f32", "fft_c_f32",
                                "fft_a_f64", "fft_b_f64", "fft_c_f64", "p_update",
                                "stats",     "finalize",  "bilinear",  "load",      "other",
                                "unet_conv", "unet_wgrad", "unet_misc", "mech_elem", "mech_gather",
                                "dens_filter", "dens_var", "dens_fold", "dens_eta", "dens_rho", "dens_vjp",
                                "mech_tan_cache"};
}  // namespace

bool prof_on() { return g_on; }

int prof_begin(int kind, cudaStream_t st) {
  if (!g_on) return -1;
  Rec r{kind, take_event(), take_event()};
  cudaEventRecord(r.a, st);
  g_recs.push_back(r);
  return (int)g_recs.size() - 1;
}

void prof_end(int slot, cudaStream_t st) {
  if (slot < 0 || slot >= (int)g_recs.size()) return;
  cudaEventRecord(g_recs[slot].b, st);
}

unsigned long long* prof_units() { return g_on ? g_units : nullptr; }

}  // namespace nlf

using namespace nlf;

extern "C" {

NLF_API int nlf_profile(int on) {
  recycle();
  if (!g_units) NLF_CUDA_TRY(cudaMalloc(&g_units, PK_COUNT * sizeof(unsigned long long)));
  NLF_CUDA_TRY(cudaMemset(g_units, 0, PK_COUNT * sizeof(unsigned long long)));
  g_on = on != 0;
  return NLF_OK;
}

NLF_API int nlf_profile_report(double* total_ms, long long* launches, unsigned long long* units, int n) {
  if (n < PK_COUNT || !total_ms || !launches || !units) {
    set_error("nlf_profile_report: need arrays of at least %d entries", (int)PK_COUNT);
    return NLF_EBADARG;
  }
  NLF_CUDA_TRY(cudaDeviceSynchronize());
  for (int k = 0; k < PK_COUNT; ++k) {
    total_ms[k] = 0.0;
    launches[k] = 0;
    units[k] = 0;
  }
  for (auto& r : g_recs) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
      total_ms[r.kind] += ms;
      launches[r.kind] += 1;
    } else {
      cudaGetLastError();
    }
  }
  if (g_units) NLF_CUDA_TRY(cudaMemcpy(units, g_units, PK_COUNT * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  return PK_COUNT;
}

NLF_API const char* nlf_profile_name(int kind) { return (kind >= 0 && kind < PK_COUNT) ? kNames[kind] : ""; }

}  // extern "C"
