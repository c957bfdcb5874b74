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

// Stockham FFT of length N = nlon/2 on the two complex rows (north, south) of a block, in place
// in shared memory: radix-8 passes while at least 8 points remain per sub-transform, then one
// radix-4 or radix-2 pass.  A pass of radix R with current sub-transform size Ns maps
// in[j + r q] (q = N/R, k = j mod Ns) through the twiddles exp(-+2 pi i r k/(Ns R)) and an
// R-point DFT in registers to out[(j - k) R + k + r Ns].  Every thread reads its inputs into
// registers before the block synchronises and overwrites the row, so one buffer of 2N points
// suffices.  The twiddles come from the table laid out below (global memory, read through the
// read-only cache).  The first pass may read from any source (global rows, a fused
// pre-processing step) and the last may write to any sink.
template <bool INV, typename V>
__device__ __forceinline__ void dft8(V (&v)[8]) {
  using S = typename ScalarOf<V>::type;
  const S h = (S)0.70710678118654752440;  // cos(pi/4)
  V a0 = cadd(v[0], v[4]), a4 = csub(v[0], v[4]);
  V a1 = cadd(v[1], v[5]), a5 = csub(v[1], v[5]);
  V a2 = cadd(v[2], v[6]), a6 = csub(v[2], v[6]);
  V a3 = cadd(v[3], v[7]), a7 = csub(v[3], v[7]);
  // a5 *= W, a6 *= W^2, a7 *= W^3 with W = exp(-+2 pi i / 8)
  const S s = INV ? h : -h;
  a5 = mkc(h * a5.x - s * a5.y, h * a5.y + s * a5.x);
  a6 = mul_mi(a6, INV);
  a7 = mkc(-h * a7.x - s * a7.y, -h * a7.y + s * a7.x);
  V b0 = cadd(a0, a2), b2 = csub(a0, a2), b1 = cadd(a1, a3), b3 = mul_mi(csub(a1, a3), INV);
  V b4 = cadd(a4, a6), b6 = csub(a4, a6), b5 = cadd(a5, a7), b7 = mul_mi(csub(a5, a7), INV);
  v[0] = cadd(b0, b1);
  v[1] = cadd(b4, b5);
  v[2] = cadd(b2, b3);
  v[3] = cadd(b6, b7);
  v[4] = csub(b0, b1);
  v[5] = csub(b4, b5);
  v[6] = csub(b2, b3);
  v[7] = csub(b6, b7);
}

template <int R, bool INV, typename V>
__device__ __forceinline__ void dft_r(V (&v)[R]) {
  if constexpr (R == 8) {
    dft8<INV>(v);
  } else if constexpr (R == 4) {
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
}

// Twiddle table of an N-point transform (nlon = 2N real points).  Entries t < N hold
// exp(-2 pi i t / (2N)).  After them, for each pass of sub-transform size NS > 1 (NS = 8, 64, ...:
// every pass before the last has radix 8) and radix R, the factors the pass multiplies by,
// W(u k 2N / (NS R)) for u = 1 .. R-1 and k < NS, at index N + NS - 8 + (u - 1) NS + k, with
// W(t) = tw[t] for t < N and -tw[t - N] above: the threads of a warp (consecutive k) read
// consecutive entries.  tw_table_len(N) entries in all.
__host__ __device__ constexpr int tw_pass_index(int n, int ns, int u, int k) { return n + ns - 8 + (u - 1) * ns + k; }
__host__ __device__ constexpr int tw_table_len(int n) { return n >= 8 ? 2 * n - 8 : n; }

// Row-FFT blocks transform NR rows of N points (NR = 2: the north and south rows of one
// latitude pair; NR = 4: two pairs); one radix-8 butterfly per thread and pass.
__host__ __device__ constexpr int fft_nt(int nr, int n2) { return nr * n2 / 8 > 32 ? nr * n2 / 8 : 32; }
inline int fft_threads(int nr, int n2) { return fft_nt(nr, n2); }

// Shared-memory row layouts, chosen so that the accesses of the passes are free of bank conflicts
// (a warp's 16-byte accesses are served eight threads at a time, 8-byte ones sixteen at a time):
// the stride-8 writes of the first pass, the stride-8 groups of the NS = 8 pass, the unit-stride
// accesses of the others, and same-index accesses to different rows in the fold's epilogue.
// 16-byte entries (8 per 128-byte bank row): one padding entry every 8, row r starts r entries
// further on.  8-byte entries (16 per bank row): row r at r (N + 2), and within a row index i is
// stored at i XOR s(i), s(i) = bits 4, 5, 6 of i in bits 0, 1, 2 and bit 6 again in bit 3, a
// permutation within each aligned group of 16 (the identity below 16).
__host__ __device__ constexpr int fpad(int p) { return p + (p >> 3); }
inline size_t fft_smem_bytes(int nr, int n2, size_t entry) { return (size_t)(fpad(nr * n2) + 4 * nr + 1) * entry; }

// Sources and sinks of a pass: (row r, index i) -> value.
template <int N, typename V>
struct SmemRows {
  V* a;
  __device__ __forceinline__ static int slot(int r, int i) {
    if constexpr (sizeof(V) == 16) {
      return fpad(r * N + i) + r;
    } else {
      return r * (N + 2) + (i ^ (((i >> 4) & 7) | ((i >> 3) & 8)));
    }
  }
  __device__ __forceinline__ V operator()(int r, int i) const { return a[slot(r, i)]; }
  __device__ __forceinline__ void put(int r, int i, V v) const { a[slot(r, i)] = v; }
};
// Grid rows of latitude pairs j0, j0 + 1, ...: row r = north (r even) or south (r odd) row of
// pair r / 2.  `rowlen` points per row.
template <typename V>
struct GlobalPairRows {
  const V* g;
  int j0, nlat, rowlen;
  __device__ __forceinline__ V operator()(int r, int i) const {
    const int j = j0 + (r >> 1);
    const int row = (r & 1) ? nlat - 1 - j : j;
    return __ldg(g + (size_t)row * rowlen + i);
  }
};

// Rows of an analysis source (FieldSpec kinds: grid, mask, ice on a mask, T0 (C* - C*0),
// dsl C*) for latitude pairs j0, j0 + 1, ...; two cells per complex point.
template <int KIND>
struct TypedPairRows {
  const double* g;
  const unsigned char* m0;
  const unsigned char* m1;
  int j0, nlat, nlon;
  __device__ __forceinline__ double2 operator()(int r, int i) const {
    const int j = j0 + (r >> 1);
    const int row = (r & 1) ? nlat - 1 - j : j;
    return src_pair<KIND>(g, m0, m1, (size_t)row * nlon + 2 * i);
  }
};

// Output rows of an inverse transform (north row, south row of latitude pair j), with the
// optional epilogue out2 = grid * mul2 on the same rows (null: none).
struct GridRowsOut {
  double2* rn;
  double2* rs;
  double2* on;
  double2* os;
  const double2* mn;
  const double2* ms;
  __device__ __forceinline__ void put(int r, int i, double2 v) const {
    (r ? rs : rn)[i] = v;
    if (on) {
      const double2 w = __ldg((r ? ms : mn) + i);
      (r ? os : on)[i] = make_double2(v.x * w.x, v.y * w.y);
    }
  }
};

// One pass of radix R over NR rows, sub-transform size NS before the pass.  ALIAS: the source
// is the destination buffer (synchronise between the reads and the writes).
template <int NR, int N, int R, int NS, bool INV, bool ALIAS, typename V, typename Src, typename Dst>
__device__ __forceinline__ void fft_pass(const Src& src, const Dst& dst, const V* __restrict__ tw) {
  constexpr int NT = fft_nt(NR, N);
  constexpr int Q = N / R;
  constexpr int IT = (NR * Q + NT - 1) / NT;
  static_assert(NS == 1 || NS >= 8, "every pass before the last has radix 8");
  V v[IT][R];
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int idx = threadIdx.x + it * NT;
    if ((NR * Q) % NT == 0 || idx < NR * Q) {
      const int r = idx / Q, j = idx % Q;
      const int k = j % NS;
      V w[R];
      if (NS > 1) {
        const V* tp = tw + tw_pass_index(N, NS, 1, k);
#pragma unroll
        for (int u = 1; u < R; ++u) {
          w[u] = __ldg(tp + (u - 1) * NS);
          if (INV) w[u].y = -w[u].y;
        }
      }
#pragma unroll
      for (int u = 0; u < R; ++u) v[it][u] = src(r, j + u * Q);
      if (NS > 1) {
#pragma unroll
        for (int u = 1; u < R; ++u) v[it][u] = cmul(v[it][u], w[u]);
      }
    }
  }
  if (ALIAS) __syncthreads();
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int idx = threadIdx.x + it * NT;
    if ((NR * Q) % NT == 0 || idx < NR * Q) {
      const int r = idx / Q, j = idx % Q;
      const int k = j % NS;
      dft_r<R, INV>(v[it]);
      const int base = (j - k) * R + k;
#pragma unroll
      for (int u = 0; u < R; ++u) dst.put(r, base + u * NS, v[it][u]);
    }
  }
  __syncthreads();
}

template <int N, int NS>
struct FftRadix {
  static constexpr int R = (N / NS >= 8) ? 8 : N / NS;
};

// Passes NS .. N of the transform held in A (shared memory), the last one into `sink`.
template <int NR, int N, int NS, bool INV, typename V, typename Sink>
__device__ __forceinline__ void fft_rest(V* A, const V* tw, const Sink& sink) {
  if constexpr (NS < N) {
    constexpr int R = FftRadix<N, NS>::R;
    if constexpr (NS * R >= N) {
      fft_pass<NR, N, R, NS, INV, false>(SmemRows<N, V>{A}, sink, tw);
    } else {
      fft_pass<NR, N, R, NS, INV, true>(SmemRows<N, V>{A}, SmemRows<N, V>{A}, tw);
      fft_rest<NR, N, NS * R, INV>(A, tw, sink);
    }
  }
}

// Whole transform of NR rows: first pass from `src` into A, the rest in place, the last pass
// into `sink` (SmemRows{A} to keep the result in A).  N >= 2.
template <int NR, int N, bool INV, typename V, typename Src, typename Sink>
__device__ __forceinline__ void fft_rows(const Src& src, V* A, const V* tw, const Sink& sink) {
  constexpr int R = FftRadix<N, 1>::R;
  if constexpr (R >= N) {
    fft_pass<NR, N, R, 1, INV, false>(src, sink, tw);
  } else {
    fft_pass<NR, N, R, 1, INV, false>(src, SmemRows<N, V>{A}, tw);
    fft_rest<NR, N, R, INV>(A, tw, sink);
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


}  // namespace sle
