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
