// Launch bracketing for the opt-in profiler (cjx_profile.cu).
#pragma once
#include <cuda_runtime.h>

namespace cjx {
void prof_begin(cudaStream_t s);
void prof_end(const char* name, cudaStream_t s);
bool prof_active();  // profiling enabled on the calling thread
}  // namespace cjx
