// Opt-in per-kernel timing: while enabled on the calling thread, every kernel
// launch the library makes is bracketed by a pair of CUDA events on its
// stream.  cjx_profile_read() waits for the events and returns, per kernel
// name, the number of launches and their summed device time.
#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "cjx_common.cuh"
#include "cjx_profile.cuh"

namespace cjx {

struct ProfRecord {
  const char* name;
  cudaEvent_t start, stop;
};

struct ProfState {
  bool on = false;
  std::vector<ProfRecord> records;
  std::vector<cudaEvent_t> pool;
  cudaEvent_t pending_start = nullptr;
};

static thread_local ProfState g_prof;

static cudaEvent_t take_event() {
  if (!g_prof.pool.empty()) {
    cudaEvent_t e = g_prof.pool.back();
    g_prof.pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

void prof_begin(cudaStream_t s) {
  if (!g_prof.on) return;
  g_prof.pending_start = take_event();
  cudaEventRecord(g_prof.pending_start, s);
}

void prof_end(const char* name, cudaStream_t s) {
  if (!g_prof.on || !g_prof.pending_start) return;
  cudaEvent_t stop = take_event();
  cudaEventRecord(stop, s);
  g_prof.records.push_back({name, g_prof.pending_start, stop});
  g_prof.pending_start = nullptr;
}

bool prof_active() { return g_prof.on; }

}  // namespace cjx

using namespace cjx;

extern "C" {

int cjx_profile_enable(int on) {
  g_prof.on = on != 0;
  return CJX_OK;
}

int cjx_profile_read(char* names, int64_t* counts, double* total_ms, int max_kernels, int* n_kernels) {
  if (!names || !counts || !total_ms || !n_kernels || max_kernels < 1)
    return fail(CJX_ERR_INVALID_ARGUMENT, "cjx_profile_read: null output or max_kernels < 1");
  std::vector<std::string> keys;
  std::vector<int64_t> cnt;
  std::vector<double> ms;
  int rc = CJX_OK;
  for (auto& r : g_prof.records) {
    float t = 0.f;
    cudaError_t e = cudaEventSynchronize(r.stop);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, r.start, r.stop);
    if (e != cudaSuccess && rc == CJX_OK) rc = check_cuda(e, "cjx_profile_read");
    size_t k = 0;
    while (k < keys.size() && keys[k] != r.name) ++k;
    if (k == keys.size()) {
      keys.emplace_back(r.name);
      cnt.push_back(0);
      ms.push_back(0.0);
    }
    cnt[k] += 1;
    ms[k] += t;
    g_prof.pool.push_back(r.start);
    g_prof.pool.push_back(r.stop);
  }
  g_prof.records.clear();
  const int n = (int)std::min<size_t>(keys.size(), (size_t)max_kernels);
  for (int i = 0; i < n; ++i) {
    std::memset(names + 32 * i, 0, 32);
    std::strncpy(names + 32 * i, keys[i].c_str(), 31);
    counts[i] = cnt[i];
    total_ms[i] = ms[i];
  }
  *n_kernels = n;
  return rc;
}

}  // extern "C"
