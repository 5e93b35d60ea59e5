// Kernel-level profiler of libnlf.so: CUDA events around each launch of a named kernel class, plus a device
// counter of the (vector x kernel) units that actually ran (CTAs of converged cells exit early, so the
// launched grid over-counts). Off by default; nlf_profile(1) turns it on and resets it. Not thread-safe.
#pragma once
#include <cuda_runtime.h>

namespace nlf {

enum ProfKind {
  PK_APPLY32 = 0, PK_APPLY64, PK_FFTA32, PK_FFTB32, PK_FFTC32, PK_FFTA64, PK_FFTB64, PK_FFTC64,
  PK_P, PK_STATS, PK_FIN, PK_BILINEAR, PK_LOAD, PK_OTHER, PK_UNET_CONV, PK_UNET_WGRAD,
  PK_UNET_MISC, PK_MECH_ELEM, PK_MECH_GATHER, PK_DENS_FILTER, PK_DENS_VAR, PK_DENS_FOLD, PK_DENS_ETA, PK_DENS_RHO, PK_DENS_VJP, PK_MECH_TANC, PK_COUNT
};

bool prof_on();
int prof_begin(int kind, cudaStream_t st);  // returns a slot, or -1 when off
void prof_end(int slot, cudaStream_t st);
unsigned long long* prof_units();          // device counters [PK_COUNT], nullptr when off

// Counts one unit for `kind` from the first CTA of a vector (blockIdx.x == blockIdx.y == 0).
__device__ __forceinline__ void prof_count(unsigned long long* units, int kind) {
  if (units && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) atomicAdd(units + kind, 1ull);
}

struct ProfScope {
  int slot;
  cudaStream_t st;
  ProfScope(int kind, cudaStream_t s) : slot(prof_begin(kind, s)), st(s) {}
  ~ProfScope() { prof_end(slot, st); }
};

}  // namespace nlf
