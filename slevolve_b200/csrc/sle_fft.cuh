// Complex helpers and the shared-memory Stockham FFT used by the transform kernels, for
// double2 (FP64 transforms) and float2 (mixed-precision transforms).
#pragma once
#include <cuda_runtime.h>

namespace sle {

template <typename V> struct ScalarOf;
template <> struct ScalarOf<double2> { using type = double; };
template <> struct ScalarOf<float2> { using type = float; };

__device__ __forceinline__ double2 mkc(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ float2 mkc(float a, float b) { return make_float2(a, b); }

template <typename V>
__device__ __forceinline__ V cadd(V a, V b) { return mkc(a.x + b.x, a.y + b.y); }
template <typename V>
__device__ __forceinline__ V csub(V a, V b) { return mkc(a.x - b.x, a.y - b.y); }
template <typename V>
__device__ __forceinline__ V cmul(V a, V b) {
  return mkc(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename V, typename S>
__device__ __forceinline__ V cscale(V a, S s) { return mkc(a.x * s, a.y * s); }

// a * (-i), or a * (+i) when inv
template <typename V>
__device__ __forceinline__ V mul_mi(V a, bool inv) {
  return inv ? mkc(-a.y, a.x) : mkc(a.y, -a.x);
}

// Stockham FFT of length N = nlon/2 on complex rows in shared memory: radix-8 passes while at
// least 8 points remain per sub-transform, then one radix-4 or radix-2 pass.  A pass of radix R
// with current sub-transform size Ns maps in[j + r q] (q = N/R, k = j mod Ns) through the
// twiddles exp(-+2 pi i r k/(Ns R)) and an R-point DFT in registers to
// out[(j - k) R + k + r Ns].  tw[t] = exp(-2 pi i t / (2 N)) for t < N; larger t use
// tw[t - N] = -exp(...).
template <typename V>
__device__ __forceinline__ void dft8(V (&v)[8], bool inv) {
  using S = typename ScalarOf<V>::type;
  const S h = (S)0.70710678118654752440;  // cos(pi/4)
  V a0 = cadd(v[0], v[4]), a4 = csub(v[0], v[4]);
  V a1 = cadd(v[1], v[5]), a5 = csub(v[1], v[5]);
  V a2 = cadd(v[2], v[6]), a6 = csub(v[2], v[6]);
  V a3 = cadd(v[3], v[7]), a7 = csub(v[3], v[7]);
  // a5 *= W, a6 *= W^2, a7 *= W^3 with W = exp(-+2 pi i / 8)
  const S s = inv ? h : -h;
  a5 = mkc(h * a5.x - s * a5.y, h * a5.y + s * a5.x);
  a6 = mul_mi(a6, inv);
  a7 = mkc(-h * a7.x - s * a7.y, -h * a7.y + s * a7.x);
  V b0 = cadd(a0, a2), b2 = csub(a0, a2), b1 = cadd(a1, a3), b3 = mul_mi(csub(a1, a3), inv);
  V b4 = cadd(a4, a6), b6 = csub(a4, a6), b5 = cadd(a5, a7), b7 = mul_mi(csub(a5, a7), inv);
  v[0] = cadd(b0, b1);
  v[1] = cadd(b4, b5);
  v[2] = cadd(b2, b3);
  v[3] = cadd(b6, b7);
  v[4] = csub(b0, b1);
  v[5] = csub(b4, b5);
  v[6] = csub(b2, b3);
  v[7] = csub(b6, b7);
}

// One Stockham pass of radix R on two rows of N points (compile-time sizes: all index
// arithmetic folds to shifts and masks).  Sub-transform size before the pass: NS.
template <int N, int R, int NS, bool INV, typename V>
__device__ __forceinline__ void fft_pass_c(const V* __restrict__ in, V* __restrict__ out,
                                           const V* __restrict__ tw) {
  constexpr int Q = N / R;
  constexpr int TSTEP = 2 * N / (NS * R);
  for (int idx = threadIdx.x; idx < 2 * Q; idx += blockDim.x) {
    const int r = idx / Q, j = idx % Q;
    const int k = j % NS;
    const V* src = in + r * N;
    V v[R];
#pragma unroll
    for (int u = 0; u < R; ++u) v[u] = src[j + u * Q];
    if (NS > 1) {
#pragma unroll
      for (int u = 1; u < R; ++u) {
        const int t = u * k * TSTEP;
        V w = (t < N) ? tw[t] : mkc(-tw[t - N].x, -tw[t - N].y);
        if (INV) w.y = -w.y;
        v[u] = cmul(v[u], w);
      }
    }
    if (R == 8) {
      dft8(reinterpret_cast<V(&)[8]>(v), INV);
    } else if (R == 4) {
      const V a0 = cadd(v[0], v[2]), a2 = csub(v[0], v[2]);
      const V a1 = cadd(v[1], v[3]), a3 = mul_mi(csub(v[1], v[3]), INV);
      v[0] = cadd(a0, a1);
      v[1] = cadd(a2, a3);
      v[2] = csub(a0, a1);
      v[3] = csub(a2, a3);
    } else {
      const V a0 = cadd(v[0], v[1]), a1 = csub(v[0], v[1]);
      v[0] = a0;
      v[1] = a1;
    }
    V* dst = out + r * N + (j - k) * R + k;
#pragma unroll
    for (int u = 0; u < R; ++u) dst[u * NS] = v[u];
  }
}

// Radix-8 passes while at least 8 points remain per sub-transform, then one radix-4 or 2 pass.
template <int N, int NS, bool INV, typename V>
__device__ __forceinline__ V* stockham_c(V* A, V* B, const V* tw) {
  if constexpr (NS >= N) {
    return A;
  } else {
    constexpr int REM = N / NS;
    constexpr int R = (REM >= 8) ? 8 : REM;
    fft_pass_c<N, R, NS, INV, V>(A, B, tw);
    __syncthreads();
    return stockham_c<N, NS * R, INV, V>(B, A, tw);
  }
}

// launch over the supported sizes N = 4 .. 2048 (nlon = 8 .. 4096)
#define SLE_FFT_SWITCH(N2, CALL) \
  switch (N2) {                  \
    case 4: CALL(4); break;      \
    case 8: CALL(8); break;      \
    case 16: CALL(16); break;    \
    case 32: CALL(32); break;    \
    case 64: CALL(64); break;    \
    case 128: CALL(128); break;  \
    case 256: CALL(256); break;  \
    case 512: CALL(512); break;  \
    case 1024: CALL(1024); break; \
    default: CALL(2048); break;  \
  }

inline int fft_threads(int n2) { return n2 / 4 > 32 ? n2 / 4 : 32; }

}  // namespace sle
