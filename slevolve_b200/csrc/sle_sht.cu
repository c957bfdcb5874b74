// Gauss-Legendre spherical-harmonic transform for sm_100a, FP64.
//
// Same transform as the reference (SLEvolve python/slevolve/sht.py:148-343, Fortran spharmt):
//   analysis   U[l,m] = (sum_j P~_lm(mu_j) (S or D by the parity of l-m)_m(j)) / 1.41421356,
//              S/D = (F_north(m) w_j +/- F_south(m) w_j) / nlon, F = rFFT of the grid rows;
//   synthesis  G_north/south(m, j) = 1.41421356 * sum_l U[l,m] P~_lm(mu_j) over even +/- odd l-m,
//              grid rows = unnormalised inverse real FFT of G (Im of m = 0 ignored).
//
// Design (B200):
//   * One kernel per latitude pair does the row FFTs (radix-2 Stockham in shared memory on
//     nlon/2-point complex sequences, real/complex split) and the north/south fold.
//   * The Legendre functions are regenerated on the fly in FP64 with a two-term recurrence
//     Q_l = mu Q_{l-1} + be_l Q_{l-2} (P~_l = cf_l Q_l) that restarts every SEG degrees from
//     seeds computed once per plan with the reference's own normalised recursion
//     (sht.py:105-144).  Segments are the work units: analysis = one warp per (m, segment),
//     latitudes spread over the lanes (8 per lane at nlat = 512), the latitude sum done by a
//     transposing warp reduction over 8 degrees at a time; synthesis = one block per pair of
//     orders (m, L-m) with one warp per 32-latitude group, coefficients staged in shared memory.
//   * (segment, latitude-group) blocks whose |P~| never exceeds 1e-35 (near the poles at high
//     m) are skipped.
#include "sle_internal.cuh"
#include "sle_fft.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>
#include <vector>

namespace sle {

static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}

// --------------------------------------------------------------------------- helpers
// (complex helpers and the Stockham FFT: sle_fft.cuh)

// Sum a per-lane vector v[0..V) over the 32 lanes of a warp.  After the call lane `l` holds
// in v[0] the warp total of value index (l >> (5 - log2 V)).  log2(V) exchange stages each
// halve the live values (send the half the partner keeps), then plain butterflies.
template <int V>
__device__ __forceinline__ void warp_transpose_reduce(double (&v)[V], int lane) {
  static_assert(V >= 1 && V <= 32 && (V & (V - 1)) == 0, "V must be a power of two <= 32");
#pragma unroll
  for (int C = V, o = 16; C > 1; C >>= 1, o >>= 1) {
    const bool up = (lane & o) != 0;
#pragma unroll
    for (int c = 0; c < C / 2; ++c) {
      const double send = up ? v[c] : v[c + C / 2];
      const double keep = up ? v[c + C / 2] : v[c];
      v[c] = keep + __shfl_xor_sync(0xffffffffu, send, o);
    }
  }
  constexpr int LOGV = (V >= 32) ? 5 : (V >= 16) ? 4 : (V >= 8) ? 3 : (V >= 4) ? 2 : (V >= 2) ? 1 : 0;
#pragma unroll
  for (int o = 16 >> LOGV; o > 0; o >>= 1) v[0] += __shfl_xor_sync(0xffffffffu, v[0], o);
}

// ------------------------------------------------------------------- plan set-up kernels
// Gauss-Legendre nodes and weights: the Newton iteration of the reference gaulw
// (sht.py:65-101), per node, in the same operation order (no contraction into FMA).
__global__ void k_gauss_nodes(int n, double tol, double* mu, double* w, int* fail) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double pi = 3.141592653589793;  // 4*atan(1) in binary64
  double z = cos(__ddiv_rn(__dmul_rn(pi, __dsub_rn((double)(i + 1), 0.25)), __dadd_rn((double)n, 0.5)));
  double zfin = 0.0, ppfin = 1.0;
  bool done = false;
  for (int sweep = 0; sweep < 10 && !done; ++sweep) {
    double p1 = 1.0, p2 = 0.0;
    for (int k = 1; k <= n; ++k) {
      const double p3 = p2;
      p2 = p1;
      const double a = __dmul_rn(__dmul_rn(__dsub_rn(2.0 * k, 1.0), z), p2);
      const double b = __dmul_rn(__dsub_rn((double)k, 1.0), p3);
      p1 = __ddiv_rn(__dsub_rn(a, b), (double)k);
    }
    const double pp = __ddiv_rn(__dmul_rn((double)n, __dsub_rn(__dmul_rn(z, p1), p2)),
                                __dsub_rn(__dmul_rn(z, z), 1.0));
    const double z1 = z;
    z = __dsub_rn(z1, __ddiv_rn(p1, pp));
    if (fabs(__dsub_rn(z, z1)) < tol) {
      zfin = z;
      ppfin = pp;
      done = true;
    }
  }
  if (!done) atomicExch(fail, 1);
  mu[i] = zfin;
  w[i] = __ddiv_rn(2.0, __dmul_rn(__dmul_rn(__dsub_rn(1.0, __dmul_rn(zfin, zfin)), ppfin), ppfin));
}

// Seeds of every (segment, latitude) and the per-(segment, group) maximum of |P~|.  P~ follows
// the reference LEGEND recursion (sht.py:105-144) operation by operation.  A segment starting at
// degree l0 > m stores (Q_{l0-2}, Q_{l0-1}) in its own scale (P~_l = cf_l Q_l with cf_l0 = 1,
// so Q_{l0-1} = P~_{l0-1} / eps_l0 and Q_{l0-2} = P~_{l0-2} / (eps_l0 eps_{l0-1})); the first
// segment (l0 = m) stores (P~_mm, 0) and uses be_m = 1.  Every degree of every segment then
// follows the same update Q_l = mu Q_{l-1} + be_l Q_{l-2}.
__global__ void k_legendre_tables(sle::ShtDev P, double2* seeds, double* segmax) {
  const int m = blockIdx.x, g = blockIdx.y, lane = threadIdx.x;
  const int j = g * 32 + lane;
  const bool ok = j < P.nh;
  const double x = ok ? P.mu[j] : 0.0;
  const double sinsq = __dsub_rn(1.0, __dmul_rn(x, x));
  double A = 1.0, B = 0.0, prod = 1.0;
  for (int i = 1; i <= m; ++i) {
    A = __dadd_rn(A, 2.0);
    B = __dadd_rn(B, 2.0);
    prod = __ddiv_rn(__dmul_rn(__dmul_rn(prod, sinsq), A), B);
  }
  const int L = P.lmax;
  const double pmm = __dsqrt_rn(__dmul_rn(0.5, prod));
  const double pm1 = __dmul_rn(__dmul_rn(__dsqrt_rn((double)(2 * m + 3)), x), pmm);
  const int np1 = m + 1;
  const double eps_m1 = __dsqrt_rn(__ddiv_rn((double)(np1 * np1 - m * m), (double)(4 * np1 * np1 - 1)));
  double t = __dsub_rn(__dmul_rn(x, pm1), __dmul_rn(eps_m1, pmm));  // x P_{n-1} - eps_{n-1} P_{n-2}
  double prev1 = 0.0, prev2 = 0.0, eps_prev = 0.0;
  double smax = 0.0;
  int seg = P.segoff[m];
  for (int l = m; l <= L; ++l) {
    double pl, eps_l;
    if (l == m) {
      pl = pmm;
      eps_l = 0.0;
    } else if (l == m + 1) {
      pl = pm1;
      eps_l = eps_m1;
    } else {
      eps_l = __dsqrt_rn(__ddiv_rn((double)(l * l - m * m), (double)(4 * l * l - 1)));
      pl = __ddiv_rn(t, eps_l);
      t = __dsub_rn(__dmul_rn(x, pl), __dmul_rn(eps_l, prev1));
    }
    const int r = (l - m) % SEG;
    if (r == 0 && ok) {
      double2 sd;
      if (l == m) {
        sd = make_double2(pmm, 0.0);
      } else {
        sd = make_double2(__ddiv_rn(prev2, __dmul_rn(eps_l, eps_prev)), __ddiv_rn(prev1, eps_l));
      }
      seeds[(size_t)seg * P.nh + j] = sd;
    }
    smax = fmax(smax, ok ? fabs(pl) : 0.0);
    if (r == SEG - 1 || l == L) {
      double v = smax;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
      if (lane == 0) segmax[(size_t)seg * P.ngrp + g] = v;
      smax = 0.0;
      ++seg;
    }
    prev2 = prev1;
    prev1 = pl;
    eps_prev = eps_l;
  }
}

// Recurrence coefficients in segment scale: cf (P~ = cf Q) and be_l = -eps_{l-1}^2 (be_m = 1).
__global__ void k_legendre_coef(sle::ShtDev P, double* be, double* cf) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= P.nseg) return;
  const int m = P.seg_m[s], l0 = P.seg_l0[s];
  const int l1 = min(l0 + SEG, P.lmax + 1);
  const long long base = P.moff[m] + (l0 - m);
  double c = 1.0;
  cf[base] = 1.0;
  if (l0 == m) {
    be[base] = 1.0;  // Q_m = be_m * P~_mm with the first segment's seeds (P~_mm, 0)
  } else {
    const int k = l0 - 1;
    be[base] = -__ddiv_rn((double)(k * k - m * m), (double)(4 * k * k - 1));
  }
  for (int l = l0 + 1; l < l1; ++l) {
    const double eps = __dsqrt_rn(__ddiv_rn((double)(l * l - m * m), (double)(4 * l * l - 1)));
    c = __ddiv_rn(c, eps);
    cf[base + (l - l0)] = c;
    const int k = l - 1;
    be[base + (l - l0)] = -__ddiv_rn((double)(k * k - m * m), (double)(4 * k * k - 1));
  }
}

__global__ void k_istart(sle::ShtDev P, const double* segmax, unsigned char* istart) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= P.nseg) return;
  int g = 0;
  while (g < P.ngrp && segmax[(size_t)s * P.ngrp + g] < SIG_THRESHOLD) ++g;
  istart[s] = (unsigned char)g;
}

__global__ void k_lidx(sle::ShtDev P, int* lidx) {
  const int m = blockIdx.x;
  const long long base = P.moff[m];
  for (int l = m + threadIdx.x; l <= P.lmax; l += blockDim.x) lidx[base + (l - m)] = l;
}

struct GridPtrs {
  const double* p[MAXF];
  int kind[MAXF];                  // analysis source (SrcKind)
  const unsigned char* m0[MAXF];
  const unsigned char* m1[MAXF];
};
struct OutGridPtrs {
  double* p[MAXF];
  double* out2[MAXF];        // optional epilogue out2 = grid * mul2
  const double* mul2[MAXF];
};
struct SpecPtrs {
  double2* p[MAXF];
};
struct CSpecPtrs {
  const double2* p[MAXF];
};

// Row rFFT of the north row j and south row nlat-1-j of field blockIdx.y, then the fold
// S = F_N w_j/nlon + F_S w_j/nlon, D = F_N w_j/nlon - F_S w_j/nlon for m <= lmax
// (sht.py:277-287).  X layout [f][0=S,1=D][m][j].  N = nlon/2 complex points per row.
// The row FFTs of one latitude pair for a source kind known at compile time.
template <int N>
struct FoldRows64 {
  const double* g;
  const unsigned char* m0;
  const unsigned char* m1;
  int j, nlat;
  const double2* tw;
  double2* A;
  template <int K>
  __device__ __forceinline__ void operator()() const {
    fft_rows<2, N, false>(TypedPairRows<K>{g, m0, m1, j, nlat, 2 * N}, A, tw, SmemRows<N, double2>{A});
  }
};

template <int N>
__global__ void __launch_bounds__(fft_nt(2, N)) k_fft_fold(sle::ShtDev P, GridPtrs g) {
  extern __shared__ double2 sm[];
  double2* A = sm;
  const int j = blockIdx.x, f = blockIdx.y;
  if (field_gated_off(P, f)) return;
  with_src_kind(g.kind[f], FoldRows64<N>{g.p[f], g.m0[f], g.m1[f], j, P.nlat, P.tw, A});
  const SmemRows<N, double2> Z{A};
  const double wn = P.wn[j], ws = P.ws[j];
  double2* XS = P.X + ((size_t)(f * 2 + 0) * P.nm) * P.nh;
  double2* XD = P.X + ((size_t)(f * 2 + 1) * P.nm) * P.nh;
  for (int m = threadIdx.x; m < P.nm; m += blockDim.x) {
    double2 xr[2];
    const double2 twm = (m > 0 && m < N) ? __ldg(P.tw + m) : make_double2(1.0, 0.0);
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const double2 z0 = Z(r, 0);
      if (m == 0) {
        xr[r] = make_double2(z0.x + z0.y, 0.0);
      } else if (m == N) {
        xr[r] = make_double2(z0.x - z0.y, 0.0);
      } else {
        const double2 zm = Z(r, m);
        const double2 zn = Z(r, N - m);
        const double2 zc = make_double2(zn.x, -zn.y);
        const double2 e = cscale(cadd(zm, zc), 0.5);
        const double2 dz = csub(zm, zc);
        const double2 o = make_double2(0.5 * dz.y, -0.5 * dz.x);  // (zm - zc) / (2i)
        xr[r] = cadd(e, cmul(twm, o));
      }
    }
    const double2 a = cscale(xr[0], wn);
    const double2 b = cscale(xr[1], ws);
    XS[(size_t)m * P.nh + j] = cadd(a, b);
    XD[(size_t)m * P.nh + j] = csub(a, b);
  }
}

// Inverse: north spectrum E + O, south E - O (m <= lmax, 0 above), unnormalised inverse
// real FFT of both rows (sht.py:330-339 with the nlon scaling folded out); field blockIdx.y.
// The half-length complex packing is formed while the first FFT pass reads its inputs; the last
// pass writes the output rows (and the optional epilogue out2 = grid * mul2).
template <int N>
struct UnfoldSrc64 {
  const double2* E;   // [m][j] planes of the field, at latitude j
  const double2* O;
  const double2* tw;
  int nm, nh;
  __device__ __forceinline__ double2 g(int r, int m) const {
    if (m >= nm) return make_double2(0.0, 0.0);
    const double2 e = E[(size_t)m * nh], o = O[(size_t)m * nh];
    return r ? csub(e, o) : cadd(e, o);
  }
  __device__ __forceinline__ double2 operator()(int r, int m) const {
    double2 x, y;
    if (m == 0) {
      x = make_double2(g(r, 0).x, 0.0);
      y = make_double2(g(r, N).x, 0.0);
    } else {
      x = g(r, m);
      const double2 c = g(r, N - m);
      y = make_double2(c.x, -c.y);
    }
    const double2 e = cadd(x, y);
    const double2 t = __ldg(tw + m);
    const double2 wc = make_double2(t.x, -t.y);  // exp(+2 pi i m / nlon)
    const double2 o = cmul(csub(x, y), wc);
    return make_double2(e.x - o.y, e.y + o.x);  // e + i o
  }
};

template <int N>
__global__ void __launch_bounds__(fft_nt(2, N)) k_ifft_unfold(sle::ShtDev P, OutGridPtrs g) {
  extern __shared__ double2 sm[];
  double2* A = sm;
  const int j = blockIdx.x, f = blockIdx.y;
  if (field_gated_off(P, f)) return;
  const int js = P.nlat - 1 - j;
  const double2* E = P.EO + ((size_t)(f * 2 + 0) * P.nm) * P.nh + j;
  const double2* O = P.EO + ((size_t)(f * 2 + 1) * P.nm) * P.nh + j;
  const size_t ro = (size_t)j * (2 * N), rso = (size_t)js * (2 * N);
  double* out2 = g.out2[f];
  const double* mul2 = g.mul2[f];
  GridRowsOut sink{reinterpret_cast<double2*>(g.p[f] + ro), reinterpret_cast<double2*>(g.p[f] + rso),
                     out2 ? reinterpret_cast<double2*>(out2 + ro) : nullptr,
                     out2 ? reinterpret_cast<double2*>(out2 + rso) : nullptr,
                     out2 ? reinterpret_cast<const double2*>(mul2 + ro) : nullptr,
                     out2 ? reinterpret_cast<const double2*>(mul2 + rso) : nullptr};
  fft_rows<2, N, true>(UnfoldSrc64<N>{E, O, P.tw, P.nm, P.nh}, A, P.tw, sink);
}



// ------------------------------------------------------------------ Legendre analysis
constexpr int ANA_TL = 4;      // degrees per warp reduction
constexpr int ANA_NAMAX = 8;   // latitude groups per lane in one pass
constexpr int ANA_WARPS = 4;   // warps (independent segments) per block

// One batch of TL consecutive degrees: advance the recurrence of the NA latitudes of this lane,
// form the per-lane products with the folded input of the degree's parity, and reduce over
// the warp.  Degree t of the batch has parity t (segments start at even l - m).
template <int NA>
__device__ __forceinline__ void ana_batch(const double* __restrict__ sbe, const double (&mu)[NA],
                                          double (&qa)[NA], double (&qb)[NA], const double2 (&xs)[NA],
                                          const double2 (&xd)[NA], double (&v)[2 * ANA_TL], int lane) {
  // the latitude sum of each degree uses up to four independent partial sums (short chains)
  constexpr int NP = (NA >= 4) ? 4 : NA;
#pragma unroll
  for (int t = 0; t < ANA_TL; ++t) {
    double re[NP], im[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p) re[p] = im[p] = 0.0;
    const double b = sbe[t];
#pragma unroll
    for (int i = 0; i < NA; ++i) {
      const double q = fma(mu[i], qb[i], b * qa[i]);
      qa[i] = qb[i];
      qb[i] = q;
      const double2 x = (t & 1) ? xd[i] : xs[i];
      re[i % NP] = fma(q, x.x, re[i % NP]);
      im[i % NP] = fma(q, x.y, im[i % NP]);
    }
    double sr = re[0], si = im[0];
    if (NP == 4) {
      sr = (re[0] + re[1]) + (re[2] + re[3]);
      si = (im[0] + im[1]) + (im[2] + im[3]);
    } else if (NP == 2) {
      sr = re[0] + re[1];
      si = im[0] + im[1];
    }
    v[2 * t] = sr;
    v[2 * t + 1] = si;
  }
  warp_transpose_reduce<2 * ANA_TL>(v, lane);
}

// Degrees l0 .. l0+len-1 of segment s over the latitude groups g0 .. g0+NA-1 (groups at or
// beyond ngrp hold no latitudes).  The staged recurrence coefficients are zero-padded to a
// whole number of batches; the extra degrees are computed and discarded.
template <int NA>
__device__ __forceinline__ void ana_segment(const sle::ShtDev& P, int s, int g0, const double2* __restrict__ Xf,
                                            double2* __restrict__ Uf, int lane, bool accumulate,
                                            double* __restrict__ sbe, double* __restrict__ scf) {
  constexpr int SHIFT = (ANA_TL == 8) ? 1 : (ANA_TL == 4) ? 2 : 3;  // 5 - log2(2 ANA_TL)
  const int m = P.seg_m[s], l0 = P.seg_l0[s];
  const int len = min(SEG, P.lmax + 1 - l0);
  const int nh = P.nh;
  const long long base = P.moff[m] + (l0 - m);
  for (int t = lane; t < SEG; t += 32) {
    sbe[t] = (t < len) ? P.be[base + t] : 0.0;
    scf[t] = (t < len) ? P.cf[base + t] : 0.0;
  }
  const double2* XS = Xf + (size_t)m * nh;
  const double2* XD = Xf + (size_t)(P.nm + m) * nh;
  double mu[NA], qa[NA], qb[NA];
  double2 xs[NA], xd[NA];
#pragma unroll
  for (int i = 0; i < NA; ++i) {
    const int j = (g0 + i) * 32 + lane;
    const bool ok = j < nh;
    mu[i] = ok ? P.mu[j] : 0.0;
    const double2 sd = ok ? P.seeds[(size_t)s * nh + j] : make_double2(0.0, 0.0);
    qa[i] = sd.x;
    qb[i] = sd.y;
    xs[i] = ok ? XS[j] : make_double2(0.0, 0.0);
    xd[i] = ok ? XD[j] : make_double2(0.0, 0.0);
  }
  __syncwarp();
  const int idx = lane >> SHIFT;
  const int tw_ = idx >> 1, c = idx & 1;
  const bool writer = (lane & ((1 << SHIFT) - 1)) == 0;
  for (int off = 0; off < len; off += ANA_TL) {
    double v[2 * ANA_TL];
    ana_batch<NA>(sbe + off, mu, qa, qb, xs, xd, v, lane);
    if (writer && off + tw_ < len) {
      const double val = __ddiv_rn(v[0] * scf[off + tw_], SQRT2_LEGACY);
      double* dst = reinterpret_cast<double*>(Uf + base + off + tw_) + c;
      *dst = accumulate ? (*dst + val) : val;
    }
  }
  __syncwarp();
}

__device__ void ana_zero_segment(const sle::ShtDev& P, int s, double2* Uf, int lane) {
  const int m = P.seg_m[s], l0 = P.seg_l0[s];
  const int l1 = min(l0 + SEG, P.lmax + 1);
  const long long base = P.moff[m] + (l0 - m);
  for (int l = l0 + lane; l < l1; l += 32) Uf[base + (l - l0)] = make_double2(0.0, 0.0);
}

__global__ void __launch_bounds__(32 * ANA_WARPS, 3) k_leg_ana(sle::ShtDev P, SpecPtrs out) {
  __shared__ double scoef[ANA_WARPS][2][SEG];
  const int wib = threadIdx.x >> 5;
  const int warp = blockIdx.x * ANA_WARPS + wib;
  const int lane = threadIdx.x & 31;
  if (warp >= P.nseg) return;
  const int f = blockIdx.y;
  if (field_gated_off(P, f)) return;
  const double2* Xf = P.X + (size_t)f * 2 * P.nm * P.nh;
  double2* Uf = out.p[f];
  const int s = P.ana_order[warp];
  int gfirst = P.istart[s];
  if (gfirst >= P.ngrp) {
    ana_zero_segment(P, s, Uf, lane);
    return;
  }
  double* sbe = scoef[wib][0];
  double* scf = scoef[wib][1];
  // latitude groups gfirst .. ngrp-1 in passes of up to ANA_NAMAX groups; a pass of na groups
  // runs the smallest instance NA >= na.  The first pass starts NA - na groups closer to the
  // pole when that stays inside the grid (those groups hold negligible but valid values and no
  // other pass covers them); later passes start where the previous one ended and mask groups
  // beyond the grid.
  bool acc = false;
  int g = gfirst;
  while (g < P.ngrp) {
    const int na = min(P.ngrp - g, ANA_NAMAX);
    const int NA = (na > 4) ? 8 : (na > 2) ? 4 : na;
    const int g0 = acc ? g : max(0, min(g, P.ngrp - NA));
    switch (NA) {
      case 1: ana_segment<1>(P, s, g0, Xf, Uf, lane, acc, sbe, scf); break;
      case 2: ana_segment<2>(P, s, g0, Xf, Uf, lane, acc, sbe, scf); break;
      case 4: ana_segment<4>(P, s, g0, Xf, Uf, lane, acc, sbe, scf); break;
      default: ana_segment<8>(P, s, g0, Xf, Uf, lane, acc, sbe, scf); break;
    }
    acc = true;
    g = g0 + NA;
  }
}

// ----------------------------------------------------------------- Legendre synthesis
// Block per pair of orders (p, lmax-p); warp per 64 latitudes (two per lane); E (even l-m) and
// O (odd l-m) sums of cf_l * 1.41421356 * U_l * Q_l over the segments where the warp's outer
// latitude group is significant.
__global__ void __launch_bounds__(512, 1) k_leg_syn(sle::ShtDev P, CSpecPtrs in) {
  extern __shared__ double smd[];
  const int f = blockIdx.y;
  if (field_gated_off(P, f)) return;
  const int p = blockIdx.x;
  const int L = P.lmax;
  double2* Uc = reinterpret_cast<double2*>(smd);          // [nm]
  double* bes = smd + 2 * P.nm;                            // [nm]
  const double2* U = in.p[f];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j0 = w * 64 + lane, j1 = j0 + 32;
  const bool ok0 = j0 < P.nh, ok1 = j1 < P.nh;
  const double x0 = ok0 ? P.mu[j0] : 0.0, x1 = ok1 ? P.mu[j1] : 0.0;
  const int gouter = min(2 * w + 1, P.ngrp - 1);
  double2* Ef = P.EO + ((size_t)(f * 2 + 0) * P.nm) * P.nh;
  double2* Of = P.EO + ((size_t)(f * 2 + 1) * P.nm) * P.nh;
  for (int pass = 0; pass < 2; ++pass) {
    const int m = (pass == 0) ? p : L - p;
    if (pass == 1 && m == p) break;
    const long long base = P.moff[m];
    const int nl = L - m + 1;
    __syncthreads();
    for (int t = threadIdx.x; t < nl; t += blockDim.x) {
      const double c = P.cf[base + t] * SQRT2_LEGACY;
      const double2 u = U[base + t];
      Uc[t] = make_double2(u.x * c, u.y * c);
      bes[t] = P.be[base + t];
    }
    __syncthreads();
    double2 E0 = make_double2(0.0, 0.0), O0 = E0, E1 = E0, O1 = E0;
    for (int s = P.segoff[m]; s < P.segoff[m + 1]; ++s) {
      if (gouter < (int)P.istart[s]) continue;
      const int l0 = P.seg_l0[s];
      const int l1 = min(l0 + SEG, L + 1);
      const double2 s0 = ok0 ? P.seeds[(size_t)s * P.nh + j0] : make_double2(0.0, 0.0);
      const double2 s1 = ok1 ? P.seeds[(size_t)s * P.nh + j1] : make_double2(0.0, 0.0);
      double qa0 = s0.x, qb0 = s0.y, qa1 = s1.x, qb1 = s1.y;
      int r = l0 - m;
      const int rend = l1 - m;
      for (; r + 2 <= rend; r += 2) {
        double2 u = Uc[r];
        double b = bes[r];
        double q0 = fma(x0, qb0, b * qa0), q1 = fma(x1, qb1, b * qa1);
        qa0 = qb0; qb0 = q0; qa1 = qb1; qb1 = q1;
        E0.x = fma(u.x, q0, E0.x); E0.y = fma(u.y, q0, E0.y);
        E1.x = fma(u.x, q1, E1.x); E1.y = fma(u.y, q1, E1.y);
        u = Uc[r + 1];
        b = bes[r + 1];
        q0 = fma(x0, qb0, b * qa0);
        q1 = fma(x1, qb1, b * qa1);
        qa0 = qb0; qb0 = q0; qa1 = qb1; qb1 = q1;
        O0.x = fma(u.x, q0, O0.x); O0.y = fma(u.y, q0, O0.y);
        O1.x = fma(u.x, q1, O1.x); O1.y = fma(u.y, q1, O1.y);
      }
      if (r < rend) {  // odd-length tail: one more even degree
        const double2 u = Uc[r];
        const double b = bes[r];
        const double q0 = fma(x0, qb0, b * qa0), q1 = fma(x1, qb1, b * qa1);
        E0.x = fma(u.x, q0, E0.x); E0.y = fma(u.y, q0, E0.y);
        E1.x = fma(u.x, q1, E1.x); E1.y = fma(u.y, q1, E1.y);
      }
    }
    if (ok0) {
      Ef[(size_t)m * P.nh + j0] = E0;
      Of[(size_t)m * P.nh + j0] = O0;
    }
    if (ok1) {
      Ef[(size_t)m * P.nh + j1] = E1;
      Of[(size_t)m * P.nh + j1] = O1;
    }
  }
}

// ---------------------------------------------------------------- dense <-> packed
__global__ void k_pack(sle::ShtDev P, const double2* dense, double2* packed) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)P.nm * P.nm;
  if (i >= n) return;
  const int l = (int)(i / P.nm), m = (int)(i - (long long)l * P.nm);
  if (m <= l) packed[P.moff[m] + (l - m)] = dense[i];
}

__global__ void k_unpack(sle::ShtDev P, const double2* packed, double2* dense) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)P.nm * P.nm;
  if (i >= n) return;
  const int l = (int)(i / P.nm), m = (int)(i - (long long)l * P.nm);
  dense[i] = (m <= l) ? packed[P.moff[m] + (l - m)] : make_double2(0.0, 0.0);
}

// ------------------------------------------------------------------------ launchers
static size_t fft_smem(const ShtDev& d) { return fft_smem_bytes(2, d.n2, sizeof(double2)); }
static int syn_threads(const ShtDev& d) { return 32 * ((d.ngrp + 1) / 2); }
static size_t syn_smem(const ShtDev& d) { return (size_t)3 * d.nm * sizeof(double); }

// One FP64 launch group (1..MAXF fields).
static int fp64_analysis(sle_sht* plan, const FieldSpec* fs, int nf, cudaStream_t st, int prof_cls) {
  ShtDev d = plan->d;
  GridPtrs g{};
  SpecPtrs o{};
  for (int f = 0; f < nf; ++f) {
    g.p[f] = fs[f].grid;
    g.kind[f] = fs[f].kind;
    g.m0[f] = fs[f].m0;
    g.m1[f] = fs[f].m1;
    o.p[f] = fs[f].spec;
    d.gset[f] = fs[f].skip_set;
    d.gclr[f] = fs[f].skip_clear;
  }
  ProfToken t0 = prof_begin(PROF_FFT, nf, st);
#define SLE_LAUNCH_FOLD(NN) k_fft_fold<NN><<<dim3(d.nh, nf), fft_threads(2, NN), fft_smem(d), st>>>(d, g)
  SLE_FFT_SWITCH(d.n2, SLE_LAUNCH_FOLD)
#undef SLE_LAUNCH_FOLD
  prof_end(t0, st);
  const int warps_per_block = ANA_WARPS;
  dim3 grid((d.nseg + warps_per_block - 1) / warps_per_block, nf);
  ProfToken t1 = prof_begin(prof_cls, nf, st);
  k_leg_ana<<<grid, 32 * warps_per_block, 0, st>>>(d, o);
  prof_end(t1, st);
  note_launch(2);
  SLE_CUDA(cudaGetLastError());
  return SLE_OK;
}

static int fp64_synthesis(sle_sht* plan, const FieldSpec* fs, int nf, cudaStream_t st) {
  ShtDev d = plan->d;
  CSpecPtrs c{};
  OutGridPtrs g{};
  for (int f = 0; f < nf; ++f) {
    c.p[f] = fs[f].spec;
    g.p[f] = fs[f].grid;
    g.out2[f] = fs[f].epi_out;
    g.mul2[f] = fs[f].epi_mul;
    d.gset[f] = fs[f].skip_set;
    d.gclr[f] = fs[f].skip_clear;
  }
  const int npairs = (d.nm + 1) / 2;
  ProfToken t0 = prof_begin(PROF_LEG_SYN, nf, st);
  k_leg_syn<<<dim3(npairs, nf), syn_threads(d), syn_smem(d), st>>>(d, c);
  prof_end(t0, st);
  ProfToken t1 = prof_begin(PROF_IFFT, nf, st);
#define SLE_LAUNCH_IFFT(NN) k_ifft_unfold<NN><<<dim3(d.nh, nf), fft_threads(2, NN), fft_smem(d), st>>>(d, g)
  SLE_FFT_SWITCH(d.n2, SLE_LAUNCH_IFFT)
#undef SLE_LAUNCH_IFFT
  prof_end(t1, st);
  note_launch(2);
  SLE_CUDA(cudaGetLastError());
  return SLE_OK;
}

static MxFieldArgs mx_args(const FieldSpec* fs, int nf) {
  MxFieldArgs a{};
  a.nf = nf;
  for (int f = 0; f < nf; ++f) {
    a.grid[f] = fs[f].grid;
    a.spec[f] = fs[f].spec;
    a.skip_set[f] = fs[f].skip_set;
    a.skip_clear[f] = fs[f].skip_clear;
    a.epi_out[f] = fs[f].epi_out;
    a.epi_mul[f] = fs[f].epi_mul;
    a.kind[f] = fs[f].kind;
    a.m0[f] = fs[f].m0;
    a.m1[f] = fs[f].m1;
  }
  return a;
}

int sht_analysis_list(sle_sht* plan, const FieldSpec* f, int n, cudaStream_t st, int prof_cls) {
  if (n < 1) return SLE_OK;
  const bool mx = plan->precision == SLE_PREC_MIXED;
  const int group = mx ? plan->tune_fpl : MAXF;
  // equal groups (the tensor-core kernels' cost depends on the launch, not on its width)
  const int ngroups = (n + group - 1) / group;
  for (int g = 0; g < ngroups; ++g) {
    const int lo = (int)((long long)n * g / ngroups), hi = (int)((long long)n * (g + 1) / ngroups);
    if (mx) {
      SLE_TRY(sht_mx_analysis(plan, mx_args(f + lo, hi - lo), plan->mx_status, st, prof_cls));
    } else {
      SLE_TRY(fp64_analysis(plan, f + lo, hi - lo, st, prof_cls));
    }
  }
  return SLE_OK;
}

int sht_synthesis_list(sle_sht* plan, const FieldSpec* f, int n, cudaStream_t st, bool b_ready) {
  if (n < 1) return SLE_OK;
  const bool mx = plan->precision == SLE_PREC_MIXED;
  const int group = mx ? plan->tune_fpl : MAXF;
  const int ngroups = (n + group - 1) / group;
  for (int g = 0; g < ngroups; ++g) {
    const int lo = (int)((long long)n * g / ngroups), hi = (int)((long long)n * (g + 1) / ngroups);
    if (mx) {
      SLE_TRY(sht_mx_synthesis(plan, mx_args(f + lo, hi - lo), plan->mx_status, st, b_ready && ngroups == 1));
    } else {
      SLE_TRY(fp64_synthesis(plan, f + lo, hi - lo, st));
    }
  }
  return SLE_OK;
}

int sht_pack(sle_sht* plan, const double2* dense, double2* packed, cudaStream_t st) {
  const long long n = (long long)plan->d.nm * plan->d.nm;
  k_pack<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(plan->d, dense, packed);
  note_launch();
  SLE_CUDA(cudaGetLastError());
  return SLE_OK;
}

int sht_unpack(sle_sht* plan, const double2* packed, double2* dense, cudaStream_t st) {
  const long long n = (long long)plan->d.nm * plan->d.nm;
  k_unpack<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(plan->d, packed, dense);
  note_launch();
  SLE_CUDA(cudaGetLastError());
  return SLE_OK;
}

// ---------------------------------------------------------------------- plan create
template <typename T>
static int dalloc(T** p, size_t n) {
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T) + 16);
  if (e != cudaSuccess) {
    set_error("cudaMalloc(%zu bytes) failed: %s", n * sizeof(T), cudaGetErrorString(e));
    *p = nullptr;
    return SLE_ERR_OOM;
  }
  return SLE_OK;
}

static void plan_free(sle_sht* p) {
  if (!p) return;
  void* ptrs[] = {p->mu, p->w, p->wn, p->ws, p->be, p->cf, p->moff, p->lidx, p->segoff,
                  p->seg_m, p->seg_l0, p->ana_order, p->seeds, p->tw, p->X, p->EO, p->istart,
                  p->packbuf, p->mx_xf, p->mx_twf, p->mx_gns, p->mx_bsyn, p->mx_s0, p->mx_abort,
                  p->mx_ana_units, p->mx_syn_units, p->mx_syn_seg, p->mx_tab_ana, p->mx_tab_syn,
                  p->mx_ana_cta, p->mx_syn_cta, p->mx_bpos};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  delete p;
}

static int plan_build(sle_sht* p, int nlat, int nlon, int lmax) {
  ShtDev& d = p->d;
  d.nlat = nlat;
  d.nlon = nlon;
  d.lmax = lmax;
  d.nh = nlat / 2;
  d.nm = lmax + 1;
  d.n2 = nlon / 2;
  d.log2n2 = 0;
  while ((1 << d.log2n2) < d.n2) ++d.log2n2;
  d.ngrp = (d.nh + 31) / 32;
  d.ncoef = (long long)d.nm * (d.nm + 1) / 2;
  // host tables: packed offsets, segments
  std::vector<long long> moff(d.nm + 1);
  std::vector<int> segoff(d.nm + 1), seg_m, seg_l0;
  for (int m = 0; m <= d.nm; ++m) moff[m] = (long long)m * (lmax + 1) - (long long)m * (m - 1) / 2;
  for (int m = 0; m < d.nm; ++m) {
    segoff[m] = (int)seg_m.size();
    for (int l0 = m; l0 <= lmax; l0 += SEG) {
      seg_m.push_back(m);
      seg_l0.push_back(l0);
    }
  }
  segoff[d.nm] = (int)seg_m.size();
  d.nseg = (int)seg_m.size();

  SLE_TRY(dalloc(&p->mu, nlat));
  SLE_TRY(dalloc(&p->w, nlat));
  SLE_TRY(dalloc(&p->wn, d.nh));
  SLE_TRY(dalloc(&p->ws, d.nh));
  SLE_TRY(dalloc(&p->moff, d.nm + 1));
  SLE_TRY(dalloc(&p->lidx, d.ncoef));
  SLE_TRY(dalloc(&p->segoff, d.nm + 1));
  SLE_TRY(dalloc(&p->seg_m, d.nseg));
  SLE_TRY(dalloc(&p->seg_l0, d.nseg));
  SLE_TRY(dalloc(&p->ana_order, d.nseg));
  SLE_TRY(dalloc(&p->seeds, (size_t)d.nseg * d.nh));
  SLE_TRY(dalloc(&p->be, d.ncoef));
  SLE_TRY(dalloc(&p->cf, d.ncoef));
  SLE_TRY(dalloc(&p->istart, d.nseg));
  SLE_TRY(dalloc(&p->tw, tw_table_len(d.n2)));
  SLE_TRY(dalloc(&p->X, (size_t)MAXF * 2 * d.nm * d.nh));
  SLE_TRY(dalloc(&p->EO, (size_t)MAXF * 2 * d.nm * d.nh));
  SLE_TRY(dalloc(&p->packbuf, (size_t)MAXF * d.ncoef));
  double* segmax = nullptr;
  int* fail = nullptr;
  SLE_TRY(dalloc(&segmax, (size_t)d.nseg * d.ngrp));
  SLE_TRY(dalloc(&fail, 1));
  SLE_CUDA(cudaMemset(fail, 0, sizeof(int)));
  SLE_CUDA(cudaMemcpy(p->moff, moff.data(), moff.size() * sizeof(long long), cudaMemcpyHostToDevice));
  SLE_CUDA(cudaMemcpy(p->segoff, segoff.data(), segoff.size() * sizeof(int), cudaMemcpyHostToDevice));
  SLE_CUDA(cudaMemcpy(p->seg_m, seg_m.data(), seg_m.size() * sizeof(int), cudaMemcpyHostToDevice));
  SLE_CUDA(cudaMemcpy(p->seg_l0, seg_l0.data(), seg_l0.size() * sizeof(int), cudaMemcpyHostToDevice));
  // twiddles exp(-2 pi i t / nlon), from long-double sin/cos rounded once, then the same values
  // in the order each FFT pass reads them (layout in sle_fft.cuh)
  std::vector<double2> tw(tw_table_len(d.n2));
  for (int t = 0; t < d.n2; ++t) {
    const long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)t / (long double)nlon;
    tw[t] = make_double2((double)cosl(a), (double)sinl(a));
  }
  for (int ns = 1, n = d.n2; ns < n;) {
    const int r = n / ns >= 8 ? 8 : n / ns;
    if (ns > 1) {
      for (int u = 1; u < r; ++u) {
        for (int k = 0; k < ns; ++k) {
          const int t = u * k * (2 * n / (ns * r));
          const int at = tw_pass_index(n, ns, u, k);
          if (at >= (int)tw.size() || t >= 2 * n) {
            set_error("twiddle table: index %d of %zu out of range", at, tw.size());
            cudaFree(segmax);
            cudaFree(fail);
            return SLE_ERR_STATE;
          }
          tw[at] = t < n ? tw[t] : make_double2(-tw[t - n].x, -tw[t - n].y);
        }
      }
    }
    ns *= r;
  }
  SLE_CUDA(cudaMemcpy(p->tw, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice));

  d.mu = p->mu;
  d.w = p->w;
  d.wn = p->wn;
  d.ws = p->ws;
  d.moff = p->moff;
  d.lidx = p->lidx;
  d.segoff = p->segoff;
  d.seg_m = p->seg_m;
  d.seg_l0 = p->seg_l0;
  d.seeds = p->seeds;
  d.be = p->be;
  d.cf = p->cf;
  d.istart = p->istart;
  d.ana_order = p->ana_order;
  d.tw = p->tw;
  d.X = p->X;
  d.EO = p->EO;

  const double tol = std::pow(0.1, 15);  // 0.1**15 as in the reference
  k_gauss_nodes<<<(nlat + 127) / 128, 128>>>(nlat, tol, p->mu, p->w, fail);
  SLE_CUDA(cudaGetLastError());
  // folded weights w/nlon (north rows 0..nh-1, south rows nlat-1 .. nh)
  std::vector<double> mu(nlat), w(nlat), wn(d.nh), ws(d.nh);
  SLE_CUDA(cudaMemcpy(mu.data(), p->mu, nlat * sizeof(double), cudaMemcpyDeviceToHost));
  SLE_CUDA(cudaMemcpy(w.data(), p->w, nlat * sizeof(double), cudaMemcpyDeviceToHost));
  int hfail = 0;
  SLE_CUDA(cudaMemcpy(&hfail, fail, sizeof(int), cudaMemcpyDeviceToHost));
  if (hfail) {
    set_error("gauss nodes: Newton iteration did not converge");
    cudaFree(segmax);
    cudaFree(fail);
    return SLE_ERR_BAD_SHAPE;
  }
  for (int j = 0; j < d.nh; ++j) {
    wn[j] = w[j] / (double)nlon;
    ws[j] = w[nlat - 1 - j] / (double)nlon;
  }
  SLE_CUDA(cudaMemcpy(p->wn, wn.data(), d.nh * sizeof(double), cudaMemcpyHostToDevice));
  SLE_CUDA(cudaMemcpy(p->ws, ws.data(), d.nh * sizeof(double), cudaMemcpyHostToDevice));

  k_lidx<<<d.nm, 128>>>(d, p->lidx);
  k_legendre_tables<<<dim3(d.nm, d.ngrp), 32>>>(d, p->seeds, segmax);
  k_legendre_coef<<<(d.nseg + 127) / 128, 128>>>(d, p->be, p->cf);
  k_istart<<<(d.nseg + 127) / 128, 128>>>(d, segmax, p->istart);
  SLE_CUDA(cudaGetLastError());
  std::vector<unsigned char> ist(d.nseg);
  SLE_CUDA(cudaMemcpy(ist.data(), p->istart, d.nseg, cudaMemcpyDeviceToHost));
  cudaFree(segmax);
  cudaFree(fail);
  // analysis order: most work first (segment length x active latitude groups)
  std::vector<int> order(d.nseg);
  std::iota(order.begin(), order.end(), 0);
  std::vector<long long> work(d.nseg);
  long long done = 0, total = 0;
  for (int s = 0; s < d.nseg; ++s) {
    const int len = std::min(SEG, lmax + 1 - seg_l0[s]);
    work[s] = (long long)len * (d.ngrp - ist[s]);
    done += work[s];
    total += (long long)len * d.ngrp;
  }
  p->work_frac = total ? (double)done / (double)total : 1.0;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work[a] > work[b]; });
  SLE_CUDA(cudaMemcpy(p->ana_order, order.data(), d.nseg * sizeof(int), cudaMemcpyHostToDevice));

#define SLE_ATTR_FFT(NN)                                                                              \
  do {                                                                                                \
    SLE_CUDA(cudaFuncSetAttribute(k_fft_fold<NN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fft_smem(d)));    \
    SLE_CUDA(cudaFuncSetAttribute(k_ifft_unfold<NN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fft_smem(d))); \
    SLE_CUDA(cudaFuncSetAttribute(k_fft_fold<NN>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));               \
    SLE_CUDA(cudaFuncSetAttribute(k_ifft_unfold<NN>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));            \
  } while (0)
  SLE_FFT_SWITCH(d.n2, SLE_ATTR_FFT)
#undef SLE_ATTR_FFT
  SLE_CUDA(cudaFuncSetAttribute(k_leg_syn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)syn_smem(d)));
  SLE_CUDA(cudaDeviceSynchronize());
  return SLE_OK;
}

// ------------------------------------------------------------ allocation-free analysis
// Scratch of sle_sht_analysis_noalloc: the folded row FFT (S and D) of one field for grids of
// up to 512 latitudes and lmax up to 511, 2 x 512 x 256 complex128 = 4 MiB.  It is part of the
// module image, so every GPU that loads this library holds it until the process exits.
constexpr int NOALLOC_MAX_NM = 512;
constexpr int NOALLOC_MAX_NH = 256;
static __device__ __align__(256) double2 g_noalloc_fold[2 * NOALLOC_MAX_NM * NOALLOC_MAX_NH];

}  // namespace sle

// ============================================================================ C ABI
using namespace sle;

namespace {
// Device address of g_noalloc_fold per device, looked up once per device (the host-side name of
// a __device__ array is not a device address and must never be passed to a kernel).
std::mutex g_noalloc_mu;
constexpr int NOALLOC_MAX_DEVICES = 128;
double2* g_noalloc_addr[NOALLOC_MAX_DEVICES] = {};
}  // namespace

extern "C" int sle_abi_version(void) { return SLE_ABI_VERSION; }
extern "C" const char* sle_last_error(void) { return g_err; }

extern "C" int sle_sht_create(int nlat, int nlon, int lmax, sle_sht** out) {
  if (!out) {
    set_error("sle_sht_create: out is NULL");
    return SLE_ERR_BAD_ARG;
  }
  *out = nullptr;
  if (nlat < 2 || nlat % 2 != 0) {
    set_error("nlat must be even");
    return SLE_ERR_BAD_SHAPE;
  }
  if (lmax < 0 || lmax > nlon / 2) {
    set_error("lmax must be <= nlon/2");
    return SLE_ERR_BAD_SHAPE;
  }
  if (nlon < 8 || (nlon & (nlon - 1)) != 0) {
    set_error("nlon must be a power of two >= 8 (got %d)", nlon);
    return SLE_ERR_BAD_SHAPE;
  }
  if (nlat > 2048 || nlon > 4096) {
    set_error("grid %d x %d exceeds the supported maximum 2048 x 4096", nlat, nlon);
    return SLE_ERR_BAD_SHAPE;
  }
  sle_sht* p = new sle_sht();
  std::memset(p, 0, sizeof(sle_sht));
  // launch shape of the mixed-precision transforms (sle_sht_set_tuning changes it)
  p->tune_fpl = MX_MAXF;
  p->tune_stages = 4;
  p->tune_fold_rows = 8;
  int rc = plan_build(p, nlat, nlon, lmax);
  if (rc != SLE_OK) {
    plan_free(p);
    return rc;
  }
  *out = p;
  return SLE_OK;
}

extern "C" int sle_sht_destroy(sle_sht* plan) {
  plan_free(plan);
  return SLE_OK;
}

extern "C" int sle_sht_info(const sle_sht* plan, int* nlat, int* nlon, int* lmax, long long* ncoef) {
  if (!plan) {
    set_error("sle_sht_info: NULL plan");
    return SLE_ERR_BAD_ARG;
  }
  if (nlat) *nlat = plan->d.nlat;
  if (nlon) *nlon = plan->d.nlon;
  if (lmax) *lmax = plan->d.lmax;
  if (ncoef) *ncoef = plan->d.ncoef;
  return SLE_OK;
}

extern "C" int sle_sht_work_fraction(const sle_sht* plan, double* frac) {
  if (!plan || !frac) {
    set_error("sle_sht_work_fraction: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  *frac = plan->work_frac;
  return SLE_OK;
}

extern "C" int sle_sht_gauss(const sle_sht* plan, double* mu_host, double* w_host) {
  if (!plan) {
    set_error("sle_sht_gauss: NULL plan");
    return SLE_ERR_BAD_ARG;
  }
  if (mu_host) SLE_CUDA(cudaMemcpy(mu_host, plan->mu, plan->d.nlat * sizeof(double), cudaMemcpyDeviceToHost));
  if (w_host) SLE_CUDA(cudaMemcpy(w_host, plan->w, plan->d.nlat * sizeof(double), cudaMemcpyDeviceToHost));
  return SLE_OK;
}

static bool aligned16(const void* p) { return p && (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// A mixed-precision kernel that timed out leaves the plan's abort flag raised: report it (the
// check synchronises only on plans that use the tensor-core path).
static int check_abort(sle_sht* plan) {
  if (plan->precision != SLE_PREC_MIXED) return SLE_OK;
  int flag = 0;
  SLE_TRY(sht_mx_abort_flag(plan, &flag));
  if (flag) {
    set_error("a tensor-core transform kernel timed out waiting on its pipeline");
    return SLE_ERR_TIMEOUT;
  }
  return SLE_OK;
}

extern "C" int sle_sht_analysis(sle_sht* plan, int nfields, const double* const* grids_dev,
                                void* const* coeffs_dev, int layout, void* stream) {
  if (!plan || !grids_dev || !coeffs_dev) {
    set_error("sle_sht_analysis: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  const int maxf = (layout == SLE_LAYOUT_PACKED) ? MAX_CALL_FIELDS : MAXF;
  if (nfields < 1 || nfields > maxf) {
    set_error("sle_sht_analysis: nfields must be 1..%d for this layout", maxf);
    return SLE_ERR_BAD_ARG;
  }
  for (int f = 0; f < nfields; ++f)
    if (!aligned16(grids_dev[f]) || !aligned16(coeffs_dev[f])) {
      set_error("sle_sht_analysis: device buffers must be non-NULL and 16-byte aligned");
      return SLE_ERR_BAD_ARG;
    }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  std::vector<double2*> outp(nfields);
  for (int f = 0; f < nfields; ++f)
    outp[f] = (layout == SLE_LAYOUT_PACKED) ? reinterpret_cast<double2*>(coeffs_dev[f])
                                            : plan->packbuf + (size_t)f * plan->d.ncoef;
  std::vector<FieldSpec> fs(nfields, FieldSpec{});
  for (int f = 0; f < nfields; ++f) {
    fs[f].grid = const_cast<double*>(grids_dev[f]);
    fs[f].spec = outp[f];
  }
  SLE_TRY(sht_analysis_list(plan, fs.data(), nfields, st));
  SLE_TRY(check_abort(plan));
  if (layout != SLE_LAYOUT_PACKED)
    for (int f = 0; f < nfields; ++f)
      SLE_TRY(sht_unpack(plan, outp[f], reinterpret_cast<double2*>(coeffs_dev[f]), st));
  return SLE_OK;
}

extern "C" int sle_sht_synthesis(sle_sht* plan, int nfields, const void* const* coeffs_dev, int layout,
                                 double* const* grids_dev, void* stream) {
  if (!plan || !grids_dev || !coeffs_dev) {
    set_error("sle_sht_synthesis: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  const int maxf = (layout == SLE_LAYOUT_PACKED) ? MAX_CALL_FIELDS : MAXF;
  if (nfields < 1 || nfields > maxf) {
    set_error("sle_sht_synthesis: nfields must be 1..%d for this layout", maxf);
    return SLE_ERR_BAD_ARG;
  }
  for (int f = 0; f < nfields; ++f)
    if (!aligned16(grids_dev[f]) || !aligned16(coeffs_dev[f])) {
      set_error("sle_sht_synthesis: device buffers must be non-NULL and 16-byte aligned");
      return SLE_ERR_BAD_ARG;
    }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  std::vector<const double2*> inp(nfields);
  for (int f = 0; f < nfields; ++f) {
    if (layout == SLE_LAYOUT_PACKED) {
      inp[f] = reinterpret_cast<const double2*>(coeffs_dev[f]);
    } else {
      double2* pb = plan->packbuf + (size_t)f * plan->d.ncoef;
      SLE_TRY(sht_pack(plan, reinterpret_cast<const double2*>(coeffs_dev[f]), pb, st));
      inp[f] = pb;
    }
  }
  std::vector<FieldSpec> fs(nfields, FieldSpec{});
  for (int f = 0; f < nfields; ++f) {
    fs[f].grid = grids_dev[f];
    fs[f].spec = const_cast<double2*>(inp[f]);
  }
  SLE_TRY(sht_synthesis_list(plan, fs.data(), nfields, st));
  return check_abort(plan);
}

extern "C" int sle_sht_set_precision(sle_sht* plan, int precision) {
  if (!plan) {
    set_error("sle_sht_set_precision: NULL plan");
    return SLE_ERR_BAD_ARG;
  }
  if (precision != SLE_PREC_FP64 && precision != SLE_PREC_MIXED) {
    set_error("sle_sht_set_precision: unknown precision %d", precision);
    return SLE_ERR_BAD_ARG;
  }
  if (precision == SLE_PREC_MIXED) SLE_TRY(sht_mx_prepare(plan));
  plan->precision = precision;
  return SLE_OK;
}

extern "C" int sle_sht_set_tuning(sle_sht* plan, const sle_mx_tuning* t) {
  if (!plan || !t) {
    set_error("sle_sht_set_tuning: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  if (t->fields_per_launch < 1 || t->fields_per_launch > MX_MAXF || (t->stages != 2 && t->stages != 4) ||
      (t->fold_rows != 4 && t->fold_rows != 8)) {
    set_error("sle_sht_set_tuning: fields_per_launch 1..%d, stages 2 or 4, fold_rows 4 or 8 (got %d, %d, %d)",
              MX_MAXF, t->fields_per_launch, t->stages, t->fold_rows);
    return SLE_ERR_BAD_ARG;
  }
  plan->tune_fpl = t->fields_per_launch;
  plan->tune_stages = t->stages;
  plan->tune_fold_rows = t->fold_rows;
  return SLE_OK;
}

extern "C" int sle_sht_get_tuning(const sle_sht* plan, sle_mx_tuning* t) {
  if (!plan || !t) {
    set_error("sle_sht_get_tuning: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  t->fields_per_launch = plan->tune_fpl;
  t->stages = plan->tune_stages;
  t->fold_rows = plan->tune_fold_rows;
  return SLE_OK;
}

extern "C" int sle_sht_pack(sle_sht* plan, const void* dense_dev, void* packed_dev, void* stream) {
  if (!plan || !dense_dev || !packed_dev) {
    set_error("sle_sht_pack: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  return sht_pack(plan, reinterpret_cast<const double2*>(dense_dev), reinterpret_cast<double2*>(packed_dev),
                  reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int sle_sht_unpack(sle_sht* plan, const void* packed_dev, void* dense_dev, void* stream) {
  if (!plan || !dense_dev || !packed_dev) {
    set_error("sle_sht_unpack: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  return sht_unpack(plan, reinterpret_cast<const double2*>(packed_dev), reinterpret_cast<double2*>(dense_dev),
                    reinterpret_cast<cudaStream_t>(stream));
}

// One analysis (one field, packed output) whose scratch is the fixed array g_noalloc_fold instead
// of memory from cudaMalloc.  The call launches the same two kernels as sle_sht_analysis; the
// first call on a device looks up the array's device address (cudaGetSymbolAddress) with that
// device current.  No element of the scratch needs clearing: every element the second kernel
// reads is written earlier in the same call by the first.  The FP64 kernels run whatever the
// plan's precision setting is.
extern "C" int sle_sht_analysis_noalloc(sle_sht* plan, const double* grid_dev, void* coeffs_packed_dev,
                                        void* stream) {
  if (!plan) {
    set_error("sle_sht_analysis_noalloc: NULL plan");
    return SLE_ERR_BAD_ARG;
  }
  if (!aligned16(grid_dev) || !aligned16(coeffs_packed_dev)) {
    set_error("sle_sht_analysis_noalloc: device buffers must be non-NULL and 16-byte aligned");
    return SLE_ERR_BAD_ARG;
  }
  if (plan->d.nm > NOALLOC_MAX_NM || plan->d.nh > NOALLOC_MAX_NH) {
    set_error("sle_sht_analysis_noalloc: grid %d x %d with lmax %d exceeds the fixed scratch "
              "(at most 512 latitudes and lmax 511); use sle_sht_analysis",
              plan->d.nlat, plan->d.nlon, plan->d.lmax);
    return SLE_ERR_BAD_SHAPE;
  }
  int dev = -1;
  SLE_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
    set_error("sle_sht_analysis_noalloc: device ordinal %d out of range", dev);
    return SLE_ERR_BAD_ARG;
  }
  double2* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
      void* p = nullptr;
      SLE_CUDA(cudaGetSymbolAddress(&p, g_noalloc_fold));
      g_noalloc_addr[dev] = reinterpret_cast<double2*>(p);
    }
    scratch = g_noalloc_addr[dev];
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  ShtDev d = plan->d;
  d.X = scratch;
  GridPtrs g{};
  g.p[0] = grid_dev;
  SpecPtrs o{};
  o.p[0] = reinterpret_cast<double2*>(coeffs_packed_dev);
#define SLE_LAUNCH_FOLD1(NN) k_fft_fold<NN><<<dim3(d.nh, 1), fft_threads(2, NN), fft_smem(d), st>>>(d, g)
  SLE_FFT_SWITCH(d.n2, SLE_LAUNCH_FOLD1)
#undef SLE_LAUNCH_FOLD1
  k_leg_ana<<<dim3((d.nseg + ANA_WARPS - 1) / ANA_WARPS, 1), 32 * ANA_WARPS, 0, st>>>(d, o);
  SLE_CUDA(cudaGetLastError());
  note_launch(2);
  return SLE_OK;
}
