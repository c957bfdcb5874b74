// Launch accounting and per-kernel CUDA-event timing of the library's own kernels, plus an
// FP64 throughput probe used as the roofline denominator of the FP64 transform kernels.
//
// Timing is off by default.  When enabled, the launch sites of the timed kernel classes record
// an event pair on the stream they launch on; sle_prof_collect() waits for the recorded events
// and accumulates their durations, so the numbers are the kernels' own device time measured in
// the run that uses them.
#include "sle_internal.cuh"

#include <atomic>
#include <cstdlib>
#include <cstring>

#include <mutex>
#include <vector>

namespace sle {

namespace {
struct Pending {
  int cls;
  double units;
  cudaEvent_t a, b;
};
struct Profiler {
  std::mutex mu;
  bool enabled = false;
  std::vector<cudaEvent_t> free_events;
  std::vector<Pending> pending;
  double ms[PROF_NCLS] = {};
  double units[PROF_NCLS] = {};
  long long count[PROF_NCLS] = {};
};
Profiler g_prof;
unsigned long long g_launches = 0;

cudaEvent_t take_event() {
  if (!g_prof.free_events.empty()) {
    cudaEvent_t e = g_prof.free_events.back();
    g_prof.free_events.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}
}  // namespace

bool prof_enabled() { return g_prof.enabled; }

// programmatic launch mode: -1 until first read (then from SLEVOLVE_B200_NO_PDL), 0 or 1
static std::atomic<int> g_pdl{-1};

bool pdl_enabled() {
  int v = g_pdl.load(std::memory_order_relaxed);
  if (v < 0) {
    const char* e = std::getenv("SLEVOLVE_B200_NO_PDL");
    int unset = -1;
    g_pdl.compare_exchange_strong(unset, (e && e[0] != '\0' && std::strcmp(e, "0") != 0) ? 0 : 1);
    v = g_pdl.load();
  }
  return v != 0;
}

void note_launch(int n) {
  __atomic_fetch_add(&g_launches, (unsigned long long)(long long)n, __ATOMIC_RELAXED);
}

ProfToken prof_begin(int cls, double units, cudaStream_t st) {
  ProfToken t{cls, units, nullptr};
  if (!g_prof.enabled) return t;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return t;
  std::lock_guard<std::mutex> lk(g_prof.mu);
  t.a = take_event();
  cudaEventRecord(reinterpret_cast<cudaEvent_t>(t.a), st);
  return t;
}

void prof_end(const ProfToken& t, cudaStream_t st) {
  if (!t.a) return;
  std::lock_guard<std::mutex> lk(g_prof.mu);
  cudaEvent_t b = take_event();
  cudaEventRecord(b, st);
  g_prof.pending.push_back(Pending{t.cls, t.units, reinterpret_cast<cudaEvent_t>(t.a), b});
}

// FP64 FMA throughput probe: 8 independent FMA chains per thread.
__global__ void k_fp64_probe(int iters, double seed, double* out) {
  double a[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) a[q] = seed + 1e-3 * (threadIdx.x + q);
  const double b = 0.999999, c = 1e-9;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int q = 0; q < 8; ++q) a[q] = fma(a[q], b, c);
  }
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < 8; ++q) s += a[q];
  if (s == 12345.678) out[0] = s;  // keeps the chains alive; never true for these inputs
}

}  // namespace sle

using namespace sle;

extern "C" int sle_set_programmatic_launch(int on, int* previous) {
  const int prev = pdl_enabled() ? 1 : 0;
  g_pdl.store(on ? 1 : 0);
  if (previous) *previous = prev;
  return SLE_OK;
}

extern "C" int sle_prof_enable(int on) {
  std::lock_guard<std::mutex> lk(g_prof.mu);
  g_prof.enabled = on != 0;
  return SLE_OK;
}

extern "C" int sle_prof_collect(void) {
  std::lock_guard<std::mutex> lk(g_prof.mu);
  for (const Pending& p : g_prof.pending) {
    cudaError_t e = cudaEventSynchronize(p.b);
    if (e != cudaSuccess) {
      set_error("sle_prof_collect: %s", cudaGetErrorString(e));
      return SLE_ERR_CUDA;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, p.a, p.b);
    g_prof.ms[p.cls] += ms;
    g_prof.units[p.cls] += p.units;
    g_prof.count[p.cls] += 1;
    g_prof.free_events.push_back(p.a);
    g_prof.free_events.push_back(p.b);
  }
  g_prof.pending.clear();
  return SLE_OK;
}

extern "C" int sle_prof_reset(void) {
  std::lock_guard<std::mutex> lk(g_prof.mu);
  for (int c = 0; c < PROF_NCLS; ++c) {
    g_prof.ms[c] = 0.0;
    g_prof.units[c] = 0.0;
    g_prof.count[c] = 0;
  }
  __atomic_store_n(&g_launches, 0ull, __ATOMIC_RELAXED);
  return SLE_OK;
}

extern "C" int sle_prof_read(int cls, double* ms, long long* count, double* units) {
  if (cls < 0 || cls >= PROF_NCLS) {
    set_error("sle_prof_read: class %d out of range", cls);
    return SLE_ERR_BAD_ARG;
  }
  std::lock_guard<std::mutex> lk(g_prof.mu);
  if (ms) *ms = g_prof.ms[cls];
  if (count) *count = g_prof.count[cls];
  if (units) *units = g_prof.units[cls];
  return SLE_OK;
}

extern "C" long long sle_launch_count(void) {
  return (long long)__atomic_load_n(&g_launches, __ATOMIC_RELAXED);
}

extern "C" int sle_probe_fp64_tflops(double* tflops) {
  if (!tflops) {
    set_error("sle_probe_fp64_tflops: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  int dev = 0, nsm = 0;
  SLE_CUDA(cudaGetDevice(&dev));
  SLE_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  double* out = nullptr;
  SLE_CUDA(cudaMalloc(&out, sizeof(double)));
  const int blocks = nsm * 8, threads = 256, iters = 4096;
  cudaEvent_t a, b;
  SLE_CUDA(cudaEventCreate(&a));
  SLE_CUDA(cudaEventCreate(&b));
  k_fp64_probe<<<blocks, threads>>>(iters, 1.0, out);  // warm-up
  SLE_CUDA(cudaEventRecord(a));
  for (int r = 0; r < 5; ++r) k_fp64_probe<<<blocks, threads>>>(iters, 1.0 + r, out);
  SLE_CUDA(cudaEventRecord(b));
  SLE_CUDA(cudaEventSynchronize(b));
  float ms = 0.0f;
  SLE_CUDA(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  const double flops = 5.0 * blocks * threads * (double)iters * 8.0 * 2.0;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return SLE_OK;
}
