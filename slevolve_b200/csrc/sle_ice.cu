// Ice history of the outer driver on the device.  The reference's driver builds a custom ice
// history from its cached ice files (run_outer.py:156-174, option --ice-seq): an entry "i" is
// file i, an entry "i:j:w" the blend (1 - w) I_i + w I_j, formed there with NumPy elementwise
// arithmetic on the host.  Here the blend is formed on the device from snapshots already there,
// with the same operations and roundings (1 - w once, two products, one sum; no fused
// multiply-add), so the grid is bit-for-bit the reference's.
#include "sle_internal.cuh"

#include <algorithm>

namespace sle {
namespace {

__global__ void __launch_bounds__(256) k_ice_blend(double* __restrict__ out, const double* __restrict__ a,
                                                   const double* __restrict__ b, double w, long long n) {
  const double wa = __dsub_rn(1.0, w);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = __dadd_rn(__dmul_rn(wa, __ldg(a + i)), __dmul_rn(w, __ldg(b + i)));
}

// Water-volume residual of the segmented initial-topography guess (init_topo_segmented.py:84-90)
// for T0 = (Tp + c) + S: per cell g0 = grounded(I0, T0), C0 = (T0 < 0) and not g0, then the
// area-weighted sums of max(-T0, 0) C0 and of dI = I0 g0 - Ip gp, each cell's terms formed with
// the reference's operations.  Block b sums cells b, b + G, ... in a fixed tree; the last block to
// finish adds the G partial sums in block order (deterministic).
constexpr int TOPO_BLOCKS = 296;
constexpr int TOPO_THREADS = 256;

__device__ __forceinline__ bool grounded_cell(double I, double T, double rhoi, double rhow) {
  return (I > 0.0) && ((T > 0.0) || (__dmul_rn(rhoi, I) > __dmul_rn(rhow, fabs(T))));
}

__global__ void __launch_bounds__(TOPO_THREADS) k_topo_residual(const double* __restrict__ tp,
                                                                const double* __restrict__ s, double c,
                                                                const double* __restrict__ i0,
                                                                const double* __restrict__ ip,
                                                                const unsigned char* __restrict__ gp,
                                                                const double* __restrict__ wrow, int nlon,
                                                                long long n, double rhoi, double rhow,
                                                                double* partial, unsigned int* counter,
                                                                double* out) {
  double v = 0.0, d = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double T0 = __dadd_rn(__dadd_rn(tp[i], c), s[i]);
    const double I0 = i0[i], area = wrow[i / nlon];
    const bool g0 = grounded_cell(I0, T0, rhoi, rhow);
    const double C0 = (T0 < 0.0 && !g0) ? 1.0 : 0.0;
    const double vol = __dmul_rn(__dmul_rn(fmax(-T0, 0.0), C0), area);
    const double dI = __dsub_rn(__dmul_rn(I0, g0 ? 1.0 : 0.0), __dmul_rn(ip[i], gp[i] ? 1.0 : 0.0));
    v = __dadd_rn(v, vol);
    d = __dadd_rn(d, __dmul_rn(dI, area));
  }
  __shared__ double sv[TOPO_THREADS], sd[TOPO_THREADS];
  sv[threadIdx.x] = v;
  sd[threadIdx.x] = d;
  __syncthreads();
  for (int o = TOPO_THREADS / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sv[threadIdx.x] = __dadd_rn(sv[threadIdx.x], sv[threadIdx.x + o]);
      sd[threadIdx.x] = __dadd_rn(sd[threadIdx.x], sd[threadIdx.x + o]);
    }
    __syncthreads();
  }
  __shared__ bool last;
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = sv[0];
    partial[2 * blockIdx.x + 1] = sd[0];
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    const volatile double* vp = partial;
    double a = 0.0, b = 0.0;
    for (unsigned int k = 0; k < gridDim.x; ++k) {
      a = __dadd_rn(a, vp[2 * k]);
      b = __dadd_rn(b, vp[2 * k + 1]);
    }
    out[0] = a;
    out[1] = b;
    *counter = 0u;   // ready for the next launch (stream order)
  }
}

}  // namespace
}  // namespace sle

using namespace sle;

extern "C" int sle_ice_blend(double* out, const double* a, const double* b, double w, long long n, void* stream) {
  if (n < 0 || (n > 0 && (!out || !a || !b))) {
    set_error("sle_ice_blend: NULL buffer or negative length");
    return SLE_ERR_BAD_ARG;
  }
  if (n == 0) return SLE_OK;
  int dev = 0, nsm = 0;
  SLE_CUDA(cudaGetDevice(&dev));
  SLE_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const long long want = (n + 255) / 256;
  const unsigned grid = (unsigned)std::max(1LL, std::min<long long>(want, 8LL * std::max(nsm, 1)));
  note_launch();
  k_ice_blend<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(out, a, b, w, n);
  SLE_CUDA(cudaGetLastError());
  return SLE_OK;
}

extern "C" int sle_topo_residual(const double* tp, const double* s, double c, const double* i0, const double* ip,
                                 const unsigned char* gp, const double* wrow, int nlat, int nlon, double rhoi,
                                 double rhow, void* scratch, double* out2, void* stream) {
  if (nlat <= 0 || nlon <= 0 || !tp || !s || !i0 || !ip || !gp || !wrow || !scratch || !out2) {
    set_error("sle_topo_residual: NULL buffer or empty grid");
    return SLE_ERR_BAD_ARG;
  }
  const long long n = (long long)nlat * nlon;
  double* part = static_cast<double*>(scratch);
  unsigned int* counter = reinterpret_cast<unsigned int*>(part + 2 * TOPO_BLOCKS + 2);
  double* dout = part + 2 * TOPO_BLOCKS;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  note_launch();
  k_topo_residual<<<TOPO_BLOCKS, TOPO_THREADS, 0, st>>>(tp, s, c, i0, ip, gp, wrow, nlon, n, rhoi, rhow, part,
                                                         counter, dout);
  SLE_CUDA(cudaGetLastError());
  SLE_CUDA(cudaMemcpyAsync(out2, dout, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  SLE_CUDA(cudaStreamSynchronize(st));
  return SLE_OK;
}

extern "C" long long sle_topo_scratch_bytes(void) {
  return (long long)((2 * TOPO_BLOCKS + 2) * sizeof(double) + 16);
}
