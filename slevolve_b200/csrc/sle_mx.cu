// Mixed-precision Gauss-Legendre transforms for sm_100a: split-TF32 ("3xTF32") Legendre
// contractions on the 5th-generation tensor cores (tcgen05.mma, accumulators in TMEM), FP64
// everywhere else the precision of the step depends on.
//
// Same transform as the FP64 path and the reference (SLEvolve python/slevolve/sht.py:274-343):
//   analysis   U[l,m] = sum_j P~_lm(mu_j) X_m^{par(l-m)}(j) / 1.41421356
//   synthesis  G_m^{N,S}(j) = sum_l 1.41421356 U[l,m] P~_lm(mu_j) over even +- odd l-m.
// Per order m both are real GEMMs over the complex fields of a launch (2 columns per field):
//   analysis   D[l][n] = sum_j  P[l][j]  B[n][j],   B = folded FFT (S for even, D for odd l-m)
//   synthesis  D[j][n] = sum_l  P[l][j]  B[n][l],   B = coefficients of one parity
// with each operand split into TF32 hi + lo and D += Ahi Bhi + Ahi Blo + Alo Bhi in FP32.
//
// Row FFTs, folds and the degree-0 coefficient are FP64; the fold output is rounded to FP32
// before the split and the synthesis accumulators are read back as FP32.
// What stays FP64: the Legendre recurrence (regenerated on the fly in every CTA from the FP64
// seeds of the plan, Q_l = mu Q_{l-1} + be_l Q_{l-2}, P~ = cf Q, then split), the Gauss nodes and
// weights, and the degree-0 coefficient: analysis computes U_00 from FP64 row sums of the input
// grid; synthesis leaves l = 0 out of the tensor-core sum and adds its uniform contribution to
// the output grid in FP64.
//
// Kernel structure (one CTA per work unit, 11 warps):
//   warps 0-7   produce the A operand (Legendre values) of K-chunk stages 0 and 1 (4 warps each),
//               warps 0-3 then read the accumulators out of TMEM (epilogue)
//   warp 8      allocates TMEM and issues the MMAs from one thread
//   warps 9-10  stage and split the B operand of stages 0 and 1
// Stages hand over through mbarriers; tcgen05.commit releases a stage when its MMAs are done.
// Every wait is bounded: on timeout the CTA raises the plan's abort flag (and the caller's status
// word), stops waiting and releases its TMEM.
#include "sle_internal.cuh"
#include "sle_fft.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace sle {
namespace {

constexpr int KC = 32;                        // K elements per chunk: one 128-byte row of TF32
constexpr int TILE_A = 128 * 128;             // 128 rows x 128 bytes
constexpr int TILE_B = MX_NMAX * 128;         // MX_NMAX rows x 128 bytes
constexpr int STAGE_BYTES = 4 * TILE_A + 4 * TILE_B;
constexpr int NSTAGE = 2;
constexpr int MISC_BYTES = 8192 + 1024;       // coefficients + barriers + bookkeeping
constexpr int MX_SMEM = 1024 + NSTAGE * STAGE_BYTES + MISC_BYTES;
constexpr int MX_THREADS = 11 * 32;
constexpr int ANA_SPAN = 256;                 // degrees per analysis unit (128 per parity)
constexpr long long WAIT_LIMIT = 1ll << 31;   // clock cycles (~1 s) before a wait gives up

static_assert(MX_SMEM <= 232448, "mixed transform shared memory exceeds the sm_100a limit");

// ------------------------------------------------------------------ PTX wrappers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t a) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(a) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t a, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(a), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void tc_alloc(uint32_t holder, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(holder), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tc_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tc_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}
// D[tmem] (+)= A[smem desc] * B[smem desc]; M = 128, N from the instruction descriptor, K = 8.
__device__ __forceinline__ void tc_mma_tf32(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}
// 32 lanes x 16 consecutive 32-bit columns from TMEM (lane = thread of the warp)
__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor of a K-major tile in the 128-byte swizzle layout: rows of
// 128 bytes (32 TF32), 8-row groups 1024 bytes apart, tile base 1024-byte aligned.  The K
// sub-block kk (8 TF32 = 32 bytes) of one MMA starts 32*kk bytes into the row.
__device__ __forceinline__ uint64_t sdesc_sw128(uint32_t saddr) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor: D F32, A and B TF32, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Byte offset of element (row, k) (4-byte elements, k < 32) in a 128-byte-swizzled K-major tile.
__device__ __forceinline__ uint32_t sw128(int row, int k) {
  return (uint32_t)(row * 128 + ((((k >> 2) ^ (row & 7)) << 4) | ((k & 3) << 2)));
}
// Byte offset of the 16-byte chunk c of row `row`.
__device__ __forceinline__ uint32_t sw128_chunk(int row, int c) {
  return (uint32_t)(row * 128 + ((c ^ (row & 7)) << 4));
}

__device__ __forceinline__ void sts32(uint32_t a, uint32_t v) {
  asm volatile("st.shared.b32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}
__device__ __forceinline__ void sts128(uint32_t a, uint32_t x, uint32_t y, uint32_t z, uint32_t w) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(a), "r"(x), "r"(y), "r"(z), "r"(w) : "memory");
}

// ------------------------------------------------------------- precision splits
// TF32 bit pattern of a double whose mantissa below its top 10 bits is zero, given its high
// word; magnitudes below FP32's normal range (2^-126) become zero.
__device__ __forceinline__ uint32_t tf32_from_dhi(uint32_t a) {
  const uint32_t e = (a >> 20) & 0x7FFu;
  const uint32_t f = (a & 0x80000000u) | ((e - 896u) << 23) | ((a & 0x000FFC00u) << 3);
  return (e < 897u) ? 0u : f;
}

// p = hi + lo with hi the nearest TF32 (ties away from zero, decided on the high word) and lo
// the nearest TF32 of the exact remainder: |p - hi - lo| <= 2^-22 |p| for |p| >= 2^-100.
__device__ __forceinline__ void split_f64(double p, uint32_t& hi, uint32_t& lo) {
  const uint32_t a = ((uint32_t)__double2hiint(p) + 0x200u) & 0xFFFFFC00u;
  const double r = p - __hiloint2double((int)a, 0);
  const uint32_t b = ((uint32_t)__double2hiint(r) + 0x200u) & 0xFFFFFC00u;
  hi = tf32_from_dhi(a);
  lo = tf32_from_dhi(b);
}

__device__ __forceinline__ void split_f32(float x, uint32_t& hi, uint32_t& lo) {
  hi = (__float_as_uint(x) + 0x1000u) & 0xFFFFE000u;
  const float r = x - __uint_as_float(hi);
  lo = (__float_as_uint(r) + 0x1000u) & 0xFFFFE000u;
}

// ------------------------------------------------------------------ bounded waits
struct Abort {
  int* flag;     // plan-wide abort word
  int* status;   // caller's status word (may be null)
};

__device__ __forceinline__ void raise_abort(const Abort& ab) {
  atomicExch(ab.flag, 1);
  if (ab.status) atomicExch(ab.status, SLE_ERR_TIMEOUT);
}

// Wait for the completion of the phase of parity `parity`; false (abort raised) after the time
// limit or as soon as another CTA raised the abort flag.
__device__ __noinline__ bool mbar_wait(uint32_t a, uint32_t parity, const Abort& ab) {
  const long long t0 = clock64();
  int spins = 0;
  while (!mbar_try_wait(a, parity)) {
    if ((++spins & 255) == 0) {
      if (*reinterpret_cast<volatile int*>(ab.flag) != 0) return false;
      if (clock64() - t0 > WAIT_LIMIT) {
        raise_abort(ab);
        return false;
      }
    }
  }
  return true;
}

__device__ __forceinline__ bool field_off(const MxFieldArgs& a, int f) {
  if (a.skip_set[f] && *a.skip_set[f] != 0) return true;
  if (a.skip_clear[f] && *a.skip_clear[f] == 0) return true;
  return false;
}

// Shared-memory layout common to both contraction kernels.
struct Smem {
  uint8_t* base;        // generic pointer, 1024-aligned
  uint32_t sbase;       // shared-window address of base
  __device__ uint32_t a_tile(int stage, int par, int lo) const {
    return sbase + stage * STAGE_BYTES + (par * 2 + lo) * TILE_A;
  }
  __device__ uint32_t b_tile(int stage, int par, int lo) const {
    return sbase + stage * STAGE_BYTES + 4 * TILE_A + (par * 2 + lo) * TILE_B;
  }
  __device__ uint8_t* misc() const { return base + NSTAGE * STAGE_BYTES; }
};

__device__ __forceinline__ Smem smem_layout(uint8_t* raw) {
  const uint32_t s = smem_u32(raw);
  const uint32_t al = (s + 1023u) & ~1023u;
  return Smem{raw + (al - s), al};
}

// misc region: [0, 8192) coefficients (double2), then barriers and bookkeeping
struct Misc {
  double2* coef;
  uint64_t* bar;        // full[2], empty[2], accum, drain
  uint32_t* tmem_holder;
  int* active;          // [MX_MAXF]
  int* chunks;          // [64]
  int* nch;
  int* any;
};
__device__ __forceinline__ Misc misc_layout(const Smem& S) {
  uint8_t* p = S.misc();
  Misc m;
  m.coef = reinterpret_cast<double2*>(p);
  m.bar = reinterpret_cast<uint64_t*>(p + 8192);
  m.tmem_holder = reinterpret_cast<uint32_t*>(p + 8192 + 64);
  m.active = reinterpret_cast<int*>(p + 8192 + 128);
  m.chunks = reinterpret_cast<int*>(p + 8192 + 128 + 4 * MX_MAXF);
  m.nch = reinterpret_cast<int*>(p + 8192 + 128 + 4 * MX_MAXF + 4 * 64);
  m.any = m.nch + 1;
  return m;
}


// TMEM use (512 columns): [0, 2N) correction accumulator (Ahi*Blo + Alo*Bhi of every chunk),
// then nbuf main accumulators of 2N columns (Ahi*Bhi), chunk i into buffer i % nbuf; each
// accumulator holds [even parity N columns][odd parity N columns].  The tensor core's FP32
// accumulation truncates, so its error grows with the number of MMAs summed into one
// accumulator: the main products (the large ones) are spread over fresh buffers and the
// buffers are added in FP64 by the epilogue.
constexpr uint32_t TMEM_COLS = 512;
__device__ __forceinline__ int main_buffers(int nch, int ncols) {
  return max(1, min(nch, ((int)TMEM_COLS - 2 * ncols) / (2 * ncols)));
}

// MMA issue loop shared by both kernels: chunk i uses stage i & 1.
__device__ void mma_loop(const Smem& S, const Misc& M, uint32_t tmem, int nch, int ncols, const Abort& ab) {
  const uint32_t idesc = idesc_tf32(128, ncols);
  const uint32_t full0 = smem_u32(&M.bar[0]), empty0 = smem_u32(&M.bar[2]), accum = smem_u32(&M.bar[4]);
  const int nbuf = main_buffers(nch, ncols);
  for (int i = 0; i < nch; ++i) {
    const int st = i & 1;
    if (!mbar_wait(full0 + 8 * st, (uint32_t)((i >> 1) & 1), ab)) {
      // aborted: let the MMAs already issued finish (bounded) before TMEM is released
      if (i > 0) {
        const uint32_t drain = smem_u32(&M.bar[5]);
        tc_commit(drain);
        const long long t0 = clock64();
        while (!mbar_try_wait(drain, 0u) && clock64() - t0 < WAIT_LIMIT) {
        }
      }
      return;
    }
    tc_fence_after();
    const uint32_t dmain = tmem + (uint32_t)(2 * ncols * (1 + i % nbuf));
    const bool fresh = i < nbuf;
#pragma unroll
    for (int kk = 0; kk < KC / 8; ++kk) {
#pragma unroll
      for (int par = 0; par < 2; ++par) {
        const uint64_t ah = sdesc_sw128(S.a_tile(st, par, 0) + 32 * kk);
        const uint64_t al = sdesc_sw128(S.a_tile(st, par, 1) + 32 * kk);
        const uint64_t bh = sdesc_sw128(S.b_tile(st, par, 0) + 32 * kk);
        const uint64_t bl = sdesc_sw128(S.b_tile(st, par, 1) + 32 * kk);
        const uint32_t off = (uint32_t)(par * ncols);
        tc_mma_tf32(dmain + off, ah, bh, idesc, (fresh && kk == 0) ? 0u : 1u);
        tc_mma_tf32(tmem + off, ah, bl, idesc, (i == 0 && kk == 0) ? 0u : 1u);
        tc_mma_tf32(tmem + off, al, bh, idesc, 1u);
      }
    }
    tc_commit(empty0 + 8 * st);
  }
  if (nch > 0) tc_commit(accum);
}

// Accumulator columns [16 cb, 16 cb + 16) of both parities for this thread's TMEM lane, summed
// over the correction and main buffers in FP64 (in that order).
__device__ __forceinline__ void acc_read(uint32_t lanebase, int nch, int ncols, int cb, double (&ev)[16],
                                         double (&od)[16]) {
  uint32_t re[16], ro[16];
  tc_ld16(lanebase + (uint32_t)(16 * cb), re);
  tc_ld16(lanebase + (uint32_t)(ncols + 16 * cb), ro);
  tc_wait_ld();
#pragma unroll
  for (int u = 0; u < 16; ++u) {
    ev[u] = (double)__uint_as_float(re[u]);
    od[u] = (double)__uint_as_float(ro[u]);
  }
  const int nb = min(nch, main_buffers(nch, ncols));
  for (int b = 0; b < nb; ++b) {
    const uint32_t base = lanebase + (uint32_t)(2 * ncols * (1 + b));
    tc_ld16(base + (uint32_t)(16 * cb), re);
    tc_ld16(base + (uint32_t)(ncols + 16 * cb), ro);
    tc_wait_ld();
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      ev[u] += (double)__uint_as_float(re[u]);
      od[u] += (double)__uint_as_float(ro[u]);
    }
  }
}

// Common prologue: barriers, gates, TMEM.  Returns the TMEM base (all threads).
__device__ uint32_t prologue(const Misc& M, const MxFieldArgs& a, uint32_t tcols) {
  const int warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    mbar_init(smem_u32(&M.bar[0]), 5);   // full: 4 producer warps + 1 loader warp
    mbar_init(smem_u32(&M.bar[1]), 5);
    mbar_init(smem_u32(&M.bar[2]), 1);   // empty: one tcgen05.commit
    mbar_init(smem_u32(&M.bar[3]), 1);
    mbar_init(smem_u32(&M.bar[4]), 1);   // accumulators complete
    mbar_init(smem_u32(&M.bar[5]), 1);   // drain after an abort
    fence_mbar_init();
  }
  if (threadIdx.x < MX_MAXF) M.active[threadIdx.x] = (threadIdx.x < a.nf) && !field_off(a, threadIdx.x);
  if (warp == 8) {
    tc_alloc(smem_u32(M.tmem_holder), tcols);
    tc_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x == 0) {
    int any = 0;
    for (int f = 0; f < a.nf; ++f) any |= M.active[f];
    *M.any = any;
  }
  const uint32_t t = *M.tmem_holder;
  __syncthreads();
  return t;
}

__device__ void epilogue_release(uint32_t tmem, uint32_t tcols) {
  tc_fence_before();
  __syncthreads();
  if ((threadIdx.x >> 5) == 8) {
    tc_fence_after();
    tc_dealloc(tmem, tcols);
  }
}

// ==================================================================== analysis
// Unit (m, s): degrees lbase = m + 256 s .. lbase + 255 (clipped at lmax), rows r of the even /
// odd tile are degrees lbase + 2r / lbase + 2r + 1.  K = latitudes in chunks of 32 starting at
// the first chunk any of the unit's four segments needs.
__global__ void __launch_bounds__(MX_THREADS, 1) k_ana_tc(ShtDev P, MxFieldArgs a, int* status) {
  extern __shared__ uint8_t smraw[];
  const Smem S = smem_layout(smraw);
  const Misc M = misc_layout(S);
  const Abort ab{P.mx_abort, status};
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int2 unit = P.mx_ana_units[blockIdx.x];
  const int m = unit.x, s = unit.y, L = P.lmax;
  const int lbase = m + ANA_SPAN * s;
  const int nd = min(ANA_SPAN, L + 1 - lbase);
  const int nsegu = (nd + SEG - 1) / SEG;
  const int seg0 = P.segoff[m] + (ANA_SPAN / SEG) * s;
  int kstart = P.ngrp;
  for (int q = 0; q < nsegu; ++q) kstart = min(kstart, (int)P.istart[seg0 + q]);
  const int nch = P.ngrp - kstart;
  const int ncols = a.ncols;
  const uint32_t tcols = TMEM_COLS;
  const long long cbase = P.moff[m] + (lbase - m);
  for (int t = threadIdx.x; t < nd; t += blockDim.x) M.coef[t] = make_double2(P.be[cbase + t], P.cf[cbase + t]);
  const uint32_t tmem = prologue(M, a, tcols);
  if (*M.any && *reinterpret_cast<volatile int*>(P.mx_abort) == 0) {
    const uint32_t empty0 = smem_u32(&M.bar[2]), full0 = smem_u32(&M.bar[0]);
    if (warp < 8) {
      // ---- producers: segment q of the unit, stage g
      const int g = warp >> 2, q = warp & 3;
      const bool valid = q < nsegu;
      const int seg = seg0 + q;
      const int ist = valid ? (int)P.istart[seg] : P.ngrp;
      const int len = valid ? min(SEG, nd - SEG * q) : 0;
      int round = 0;
      for (int i = g; i < nch; i += 2, ++round) {
        const int c = kstart + i;
        if (!mbar_wait(empty0 + 8 * g, (uint32_t)((round & 1) ^ 1), ab)) break;
        if (valid) {
          const uint32_t aeh = S.a_tile(g, 0, 0), ael = S.a_tile(g, 0, 1);
          const uint32_t aoh = S.a_tile(g, 1, 0), aol = S.a_tile(g, 1, 1);
          if (c < ist) {
            // negligible block: zero rows 32q .. 32q+31 of all four tiles
            for (int e = lane; e < 32 * 8; e += 32) {
              const int row = SEG / 2 * q + (e >> 3), ch = e & 7;
              const uint32_t o = sw128_chunk(row, ch);
              sts128(aeh + o, 0, 0, 0, 0);
              sts128(ael + o, 0, 0, 0, 0);
              sts128(aoh + o, 0, 0, 0, 0);
              sts128(aol + o, 0, 0, 0, 0);
            }
          } else {
            const int j = KC * c + lane;
            const double mu = P.mu[j];
            const double2 sd = P.seeds[(size_t)seg * P.nh + j];
            double qa = sd.x, qb = sd.y;
            const double2* cf = M.coef + SEG * q;
            for (int t = 0; t < len; t += 2) {
              const int row = SEG / 2 * q + (t >> 1);
              const uint32_t o = sw128(row, lane);
              double2 bc = cf[t];
              double qn = fma(mu, qb, bc.x * qa);
              qa = qb;
              qb = qn;
              uint32_t h, l;
              split_f64(bc.y * qn, h, l);
              sts32(aeh + o, h);
              sts32(ael + o, l);
              if (t + 1 < len) {
                bc = cf[t + 1];
                qn = fma(mu, qb, bc.x * qa);
                qa = qb;
                qb = qn;
                split_f64(bc.y * qn, h, l);
                sts32(aoh + o, h);
                sts32(aol + o, l);
              }
            }
          }
        }
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) mbar_arrive(full0 + 8 * g);
      }
    } else if (warp == 8) {
      if (lane == 0) mma_loop(S, M, tmem, nch, ncols, ab);
      __syncwarp();
    } else {
      // ---- B loader: folded FFT chunk (S rows, D rows) split into TF32 hi / lo
      const int lw = warp - 9;
      const int nrow = 2 * a.nf;
      int round = 0;
      for (int i = lw; i < nch; i += 2, ++round) {
        const int c = kstart + i;
        if (!mbar_wait(empty0 + 8 * lw, (uint32_t)((round & 1) ^ 1), ab)) break;
#pragma unroll
        for (int par = 0; par < 2; ++par) {
          const float* src = P.mx_xf + (((size_t)m * 2 + par) * P.ngrp + c) * (size_t)(MX_NMAX * KC);
          const uint32_t bh = S.b_tile(lw, par, 0), bl = S.b_tile(lw, par, 1);
          for (int n = 0; n < nrow; n += 4) {
            float v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) v[u] = (n + u < nrow) ? __ldg(src + (n + u) * KC + lane) : 0.0f;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              if (n + u < nrow) {
                uint32_t h, l;
                split_f32(v[u], h, l);
                const uint32_t o = sw128(n + u, lane);
                sts32(bh + o, h);
                sts32(bl + o, l);
              }
            }
          }
        }
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) mbar_arrive(full0 + 8 * lw);
      }
    }
    // ---- epilogue: warps 0-3 own TMEM lanes 0-127 = rows of both parity tiles
    if (warp < 4) {
      const int r = 32 * warp + lane;
      const int le = lbase + 2 * r;
      bool ok = true;
      if (nch > 0) {
        ok = mbar_wait(smem_u32(&M.bar[4]), 0u, ab);
        tc_fence_after();
      }
      ok = __all_sync(0xffffffffu, ok);
      if (ok) {
        const double inv = 1.0 / SQRT2_LEGACY;
        const uint32_t lanebase = tmem + ((uint32_t)(32 * warp) << 16);
        for (int cb = 0; cb < (2 * a.nf + 15) / 16; ++cb) {
          double ve[16], vo[16];
          if (nch > 0) {
            acc_read(lanebase, nch, ncols, cb, ve, vo);
          } else {
#pragma unroll
            for (int u = 0; u < 16; ++u) ve[u] = vo[u] = 0.0;
          }
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int f = 8 * cb + u;
            if (f < a.nf && M.active[f] && le <= L) {
              double2* dst = a.spec[f] + P.moff[m] + (le - m);
              const double2 ev = make_double2(ve[2 * u] * inv, ve[2 * u + 1] * inv);
              if (le + 1 <= L) {
                dst[0] = ev;
                dst[1] = make_double2(vo[2 * u] * inv, vo[2 * u + 1] * inv);
              } else {
                dst[0] = ev;
              }
            }
          }
        }
        // degree 0 in FP64 from the row sums of the fold: U_00 = sqrt(0.5) sum_j S_0(j) / 1.41421356
        __syncwarp();
        if (m == 0 && s == 0 && warp == 0 && lane < a.nf && M.active[lane]) {
          const double* s0 = P.mx_s0 + (size_t)lane * P.nh;
          double acc = 0.0;
          for (int j = 0; j < P.nh; ++j) acc += s0[j];
          a.spec[lane][0] = make_double2(__dmul_rn(__dsqrt_rn(0.5), acc) / SQRT2_LEGACY, 0.0);
        }
      }
    }
  }
  epilogue_release(tmem, tcols);
}

// =================================================================== synthesis
// Unit (m, t): latitudes 128 t .. 128 t + 127 (rows; clipped at nh), K = degrees of m in
// segments of 64 (32 even + 32 odd), skipping segments negligible on the whole tile.
__global__ void __launch_bounds__(MX_THREADS, 1) k_syn_tc(ShtDev P, MxFieldArgs a, int* status) {
  extern __shared__ uint8_t smraw[];
  const Smem S = smem_layout(smraw);
  const Misc M = misc_layout(S);
  const Abort ab{P.mx_abort, status};
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int2 unit = P.mx_syn_units[blockIdx.x];
  const int m = unit.x, t = unit.y, L = P.lmax;
  const int ncols = a.ncols;
  const uint32_t tcols = TMEM_COLS;
  const int nl = L - m + 1;
  const long long cbase = P.moff[m];
  for (int u = threadIdx.x; u < nl; u += blockDim.x) M.coef[u] = make_double2(P.be[cbase + u], P.cf[cbase + u]);
  if (threadIdx.x == 0) {
    const int glast = min(P.ngrp, 4 * t + 4) - 1;
    int n = 0;
    for (int q = 0; q < P.segoff[m + 1] - P.segoff[m]; ++q)
      if ((int)P.istart[P.segoff[m] + q] <= glast) M.chunks[n++] = q;
    *M.nch = n;
  }
  const uint32_t tmem = prologue(M, a, tcols);
  const int nch = *M.nch;
  if (*M.any && *reinterpret_cast<volatile int*>(P.mx_abort) == 0) {
    const uint32_t empty0 = smem_u32(&M.bar[2]), full0 = smem_u32(&M.bar[0]);
    if (warp < 8) {
      // ---- producers: rows 32 wq .. 32 wq + 31 of the tile, stage g
      const int g = warp >> 2, wq = warp & 3;
      const int row = 32 * wq + lane;
      const int j = 128 * t + row;
      const int grp = j >> 5;
      const bool okrow = j < P.nh;
      const double mu = okrow ? P.mu[j] : 0.0;
      int round = 0;
      for (int i = g; i < nch; i += 2, ++round) {
        if (!mbar_wait(empty0 + 8 * g, (uint32_t)((round & 1) ^ 1), ab)) break;
        const int q = M.chunks[i];
        const int seg = P.segoff[m] + q;
        const int l0 = m + SEG * q;
        const int len = min(SEG, L + 1 - l0);
        const uint32_t aeh = S.a_tile(g, 0, 0), ael = S.a_tile(g, 0, 1);
        const uint32_t aoh = S.a_tile(g, 1, 0), aol = S.a_tile(g, 1, 1);
        if (okrow) {
          if (grp < (int)P.istart[seg]) {
#pragma unroll
            for (int ch = 0; ch < 8; ++ch) {
              const uint32_t o = sw128_chunk(row, ch);
              sts128(aeh + o, 0, 0, 0, 0);
              sts128(ael + o, 0, 0, 0, 0);
              sts128(aoh + o, 0, 0, 0, 0);
              sts128(aol + o, 0, 0, 0, 0);
            }
          } else {
            const double2 sd = P.seeds[(size_t)seg * P.nh + j];
            double qa = sd.x, qb = sd.y;
            const double2* cf = M.coef + SEG * q;
            for (int ch = 0; ch < 8; ++ch) {
              uint32_t eh[4], el[4], oh[4], ol[4];
#pragma unroll
              for (int v = 0; v < 4; ++v) {
                const int te = 8 * ch + 2 * v;
                eh[v] = el[v] = oh[v] = ol[v] = 0u;
                if (te < len) {
                  const double2 bc = cf[te];
                  const double qn = fma(mu, qb, bc.x * qa);
                  qa = qb;
                  qb = qn;
                  split_f64(bc.y * qn, eh[v], el[v]);
                }
                if (te + 1 < len) {
                  const double2 bc = cf[te + 1];
                  const double qn = fma(mu, qb, bc.x * qa);
                  qa = qb;
                  qb = qn;
                  split_f64(bc.y * qn, oh[v], ol[v]);
                }
              }
              const uint32_t o = sw128_chunk(row, ch);
              sts128(aeh + o, eh[0], eh[1], eh[2], eh[3]);
              sts128(ael + o, el[0], el[1], el[2], el[3]);
              sts128(aoh + o, oh[0], oh[1], oh[2], oh[3]);
              sts128(aol + o, ol[0], ol[1], ol[2], ol[3]);
            }
          }
        }
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) mbar_arrive(full0 + 8 * g);
      }
    } else if (warp == 8) {
      if (lane == 0) mma_loop(S, M, tmem, nch, ncols, ab);
      __syncwarp();
    } else {
      // ---- B loader: 1.41421356 U[l, m] of the segment, rows 2f (Re) and 2f+1 (Im), K = the
      // degree's index in its parity; l = 0 is left out (added in FP64 by the inverse FFT)
      const int lw = warp - 9;
      int round = 0;
      for (int i = lw; i < nch; i += 2, ++round) {
        if (!mbar_wait(empty0 + 8 * lw, (uint32_t)((round & 1) ^ 1), ab)) break;
        const int q = M.chunks[i];
        const int l0 = m + SEG * q;
        const int len = min(SEG, L + 1 - l0);
        for (int f = 0; f < a.nf; ++f) {
          const double2* U = a.spec[f] + cbase + (l0 - m);
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int tt = lane + 32 * h;
            double2 u = make_double2(0.0, 0.0);
            if (tt < len && !(m == 0 && l0 + tt == 0) && M.active[f]) u = U[tt];
            const int par = tt & 1, k = tt >> 1;
            uint32_t rh, rl, ih, il;
            split_f64(u.x * SQRT2_LEGACY, rh, rl);
            split_f64(u.y * SQRT2_LEGACY, ih, il);
            const uint32_t bh = S.b_tile(lw, par, 0), bl = S.b_tile(lw, par, 1);
            sts32(bh + sw128(2 * f, k), rh);
            sts32(bl + sw128(2 * f, k), rl);
            sts32(bh + sw128(2 * f + 1, k), ih);
            sts32(bl + sw128(2 * f + 1, k), il);
          }
        }
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) mbar_arrive(full0 + 8 * lw);
      }
    }
    // ---- epilogue: north = E + O, south = E - O for the tile's latitudes
    if (warp < 4) {
      const int r = 32 * warp + lane;
      const int j = 128 * t + r;
      bool ok = true;
      if (nch > 0) {
        ok = mbar_wait(smem_u32(&M.bar[4]), 0u, ab);
        tc_fence_after();
      }
      ok = __all_sync(0xffffffffu, ok);
      if (ok) {
        const uint32_t lanebase = tmem + ((uint32_t)(32 * warp) << 16);
        for (int cb = 0; cb < (2 * a.nf + 15) / 16; ++cb) {
          double ve[16], vo[16];
          if (nch > 0) {
            acc_read(lanebase, nch, ncols, cb, ve, vo);
          } else {
#pragma unroll
            for (int u = 0; u < 16; ++u) ve[u] = vo[u] = 0.0;
          }
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int f = 8 * cb + u;
            if (f < a.nf && M.active[f] && j < P.nh) {
              float2* gn = P.mx_gns + ((size_t)(2 * f) * P.nm + m) * P.nh;
              float2* gs = P.mx_gns + ((size_t)(2 * f + 1) * P.nm + m) * P.nh;
              gn[j] = make_float2((float)(ve[2 * u] + vo[2 * u]), (float)(ve[2 * u + 1] + vo[2 * u + 1]));
              gs[j] = make_float2((float)(ve[2 * u] - vo[2 * u]), (float)(ve[2 * u + 1] - vo[2 * u + 1]));
            }
          }
        }
      }
    }
  }
  epilogue_release(tmem, tcols);
}

// ============================================================== row FFT kernels
// Row rFFT (FP64) of the north row j and south row nlat-1-j of field blockIdx.y, fold with the
// weights (FP64), output rounded to FP32 in the analysis B layout X[m][par][chunk][row][k]
// (row 2f = Re, 2f+1 = Im, chunk = j / 32, k = j % 32).  The m = 0 fold (row sums) is also kept
// in FP64 in s0[f][j] for the FP64 degree-0 coefficient.
template <int N>
__global__ void __launch_bounds__((N / 4 > 32) ? N / 4 : 32) k_fold_mx(ShtDev P, MxFieldArgs a) {
  extern __shared__ double2 smd2[];
  double2* tw = smd2;
  double2* A = smd2 + N;
  double2* B = A + 2 * N;
  const int j = blockIdx.x, f = blockIdx.y;
  if (field_off(a, f)) return;
  const int js = P.nlat - 1 - j;
  const double2* rn = reinterpret_cast<const double2*>(a.grid[f] + (size_t)j * (2 * N));
  const double2* rs = reinterpret_cast<const double2*>(a.grid[f] + (size_t)js * (2 * N));
  for (int t = threadIdx.x; t < N; t += blockDim.x) {
    tw[t] = P.tw[t];
    A[t] = rn[t];
    A[N + t] = rs[t];
  }
  __syncthreads();
  const double2* Z = stockham_c<N, 1, false>(A, B, tw);
  const double wn = P.wn[j], ws = P.ws[j];
  const int c = j >> 5, k = j & 31;
  for (int m = threadIdx.x; m < P.nm; m += blockDim.x) {
    double2 xr[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const double2* z = Z + r * N;
      if (m == 0) {
        xr[r] = make_double2(z[0].x + z[0].y, 0.0);
      } else if (m == N) {
        xr[r] = make_double2(z[0].x - z[0].y, 0.0);
      } else {
        const double2 zm = z[m];
        const double2 zc = make_double2(z[N - m].x, -z[N - m].y);
        const double2 e = cscale(cadd(zm, zc), 0.5);
        const double2 dz = csub(zm, zc);
        const double2 o = make_double2(0.5 * dz.y, -0.5 * dz.x);  // (zm - zc) / (2i)
        xr[r] = cadd(e, cmul(tw[m], o));
      }
    }
    const double2 an = cscale(xr[0], wn), bs = cscale(xr[1], ws);
    if (m == 0) P.mx_s0[(size_t)f * P.nh + j] = an.x + bs.x;
    float* xs = P.mx_xf + ((((size_t)m * 2 + 0) * P.ngrp + c) * MX_NMAX + 2 * f) * KC + k;
    float* xd = P.mx_xf + ((((size_t)m * 2 + 1) * P.ngrp + c) * MX_NMAX + 2 * f) * KC + k;
    xs[0] = (float)(an.x + bs.x);
    xs[KC] = (float)(an.y + bs.y);
    xd[0] = (float)(an.x - bs.x);
    xd[KC] = (float)(an.y - bs.y);
  }
}

// Inverse: north and south Legendre sums of field blockIdx.y (FP32 accumulators, m <= lmax, 0
// above), unnormalised inverse real FFT in FP64, plus the FP64 degree-0 term
// 1.41421356 sqrt(0.5) Re U_00 in every cell; optional epilogue out2 = grid * mul2.
template <int N>
__global__ void __launch_bounds__((N / 4 > 32) ? N / 4 : 32) k_unfold_mx(ShtDev P, MxFieldArgs a) {
  extern __shared__ double2 smd2[];
  __shared__ double2 nyq[2];
  double2* tw = smd2;
  double2* A = smd2 + N;
  double2* B = A + 2 * N;
  const int j = blockIdx.x, f = blockIdx.y;
  if (field_off(a, f)) return;
  const int js = P.nlat - 1 - j;
  const float2* GN = P.mx_gns + (size_t)(2 * f) * P.nm * P.nh;
  const float2* GS = P.mx_gns + (size_t)(2 * f + 1) * P.nm * P.nh;
  const double c00 = __dmul_rn(__dmul_rn(SQRT2_LEGACY, a.spec[f][0].x), __dsqrt_rn(0.5));
  for (int t = threadIdx.x; t < N; t += blockDim.x) tw[t] = P.tw[t];
  for (int m = threadIdx.x; m <= N; m += blockDim.x) {
    double2 gn = make_double2(0.0, 0.0), gs = gn;
    if (m < P.nm) {
      const float2 vn = GN[(size_t)m * P.nh + j], vs = GS[(size_t)m * P.nh + j];
      gn = make_double2(vn.x, vn.y);
      gs = make_double2(vs.x, vs.y);
    }
    if (m == 0) {
      gn.x += c00;
      gs.x += c00;
    }
    if (m < N) {
      B[m] = gn;
      B[N + m] = gs;
    } else {
      nyq[0] = gn;
      nyq[1] = gs;
    }
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < 2 * N; idx += blockDim.x) {
    const int r = idx / N;
    const int m = idx % N;
    double2 x, y;
    if (m == 0) {
      x = make_double2(B[r * N].x, 0.0);
      y = make_double2(nyq[r].x, 0.0);
    } else {
      x = B[r * N + m];
      const double2 c = B[r * N + N - m];
      y = make_double2(c.x, -c.y);
    }
    const double2 e = cadd(x, y);
    const double2 wc = make_double2(tw[m].x, -tw[m].y);  // exp(+2 pi i m / nlon)
    const double2 o = cmul(csub(x, y), wc);
    A[r * N + m] = make_double2(e.x - o.y, e.y + o.x);  // e + i o
  }
  __syncthreads();
  const double2* Z = stockham_c<N, 1, true>(A, B, tw);
  double2* rn = reinterpret_cast<double2*>(a.grid[f] + (size_t)j * (2 * N));
  double2* rs = reinterpret_cast<double2*>(a.grid[f] + (size_t)js * (2 * N));
  double* out2 = a.epi_out[f];
  const double* mul2 = a.epi_mul[f];
  for (int t = threadIdx.x; t < N; t += blockDim.x) {
    const double2 vn = Z[t], vs = Z[N + t];
    rn[t] = vn;
    rs[t] = vs;
    if (out2) {
      const double2 mn = reinterpret_cast<const double2*>(mul2 + (size_t)j * (2 * N))[t];
      const double2 ms = reinterpret_cast<const double2*>(mul2 + (size_t)js * (2 * N))[t];
      reinterpret_cast<double2*>(out2 + (size_t)j * (2 * N))[t] = make_double2(vn.x * mn.x, vn.y * mn.y);
      reinterpret_cast<double2*>(out2 + (size_t)js * (2 * N))[t] = make_double2(vs.x * ms.x, vs.y * ms.y);
    }
  }
}

size_t mx_fft_smem(const ShtDev& d) { return (size_t)5 * d.n2 * sizeof(double2); }

template <typename T>
int mx_alloc(T** p, size_t n) {
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T) + 16);
  if (e != cudaSuccess) {
    set_error("cudaMalloc(%zu bytes) for the mixed-precision transform failed: %s", n * sizeof(T),
              cudaGetErrorString(e));
    *p = nullptr;
    return SLE_ERR_OOM;
  }
  return SLE_OK;
}

}  // namespace

// ------------------------------------------------------------------ host side
int sht_mx_prepare(sle_sht* p) {
  if (p->mx_ready) return SLE_OK;
  ShtDev& d = p->d;
  if (d.nh % KC != 0) {
    set_error("mixed precision needs nlat to be a multiple of 64 (got %d)", d.nlat);
    return SLE_ERR_BAD_SHAPE;
  }
  if (d.nm > 512) {
    set_error("mixed precision supports lmax <= 511 (got %d)", d.lmax);
    return SLE_ERR_BAD_SHAPE;
  }
  const size_t nxf = (size_t)d.nm * 2 * d.ngrp * MX_NMAX * KC;
  SLE_TRY(mx_alloc(&p->mx_xf, nxf));
  SLE_TRY(mx_alloc(&p->mx_gns, (size_t)2 * MX_MAXF * d.nm * d.nh));
  SLE_TRY(mx_alloc(&p->mx_s0, (size_t)MX_MAXF * d.nh));
  SLE_TRY(mx_alloc(&p->mx_abort, 1));
  SLE_CUDA(cudaMemset(p->mx_xf, 0, nxf * sizeof(float)));
  SLE_CUDA(cudaMemset(p->mx_gns, 0, (size_t)2 * MX_MAXF * d.nm * d.nh * sizeof(float2)));
  SLE_CUDA(cudaMemset(p->mx_abort, 0, sizeof(int)));
  // work units, most work first (generation work ~ degrees x significant latitude groups)
  std::vector<unsigned char> ist(d.nseg);
  std::vector<int> segoff(d.nm + 1);
  SLE_CUDA(cudaMemcpy(ist.data(), p->istart, d.nseg, cudaMemcpyDeviceToHost));
  SLE_CUDA(cudaMemcpy(segoff.data(), p->segoff, (d.nm + 1) * sizeof(int), cudaMemcpyDeviceToHost));
  const int L = d.lmax;
  std::vector<std::pair<long long, int2>> au, su;
  for (int m = 0; m <= L; ++m) {
    const int nl = L - m + 1;
    for (int s = 0; s * ANA_SPAN < nl; ++s) {
      long long w = 1;
      const int nd = std::min(ANA_SPAN, nl - ANA_SPAN * s);
      for (int q = 0; q * SEG < nd; ++q) {
        const int seg = segoff[m] + (ANA_SPAN / SEG) * s + q;
        w += (long long)std::min(SEG, nd - SEG * q) * (d.ngrp - ist[seg]);
      }
      au.push_back({w, make_int2(m, s)});
    }
    const int ntile = (d.nh + 127) / 128;
    for (int t = 0; t < ntile; ++t) {
      long long w = 1;
      for (int seg = segoff[m]; seg < segoff[m + 1]; ++seg) {
        const int l0 = m + SEG * (seg - segoff[m]);
        const int g0 = 4 * t, g1 = std::min(d.ngrp, 4 * t + 4);
        const int sig = std::max(0, g1 - std::max(g0, (int)ist[seg]));
        w += (long long)std::min(SEG, L + 1 - l0) * sig;
      }
      su.push_back({w, make_int2(m, t)});
    }
  }
  auto by_work = [](const std::pair<long long, int2>& x, const std::pair<long long, int2>& y) {
    return x.first > y.first;
  };
  std::stable_sort(au.begin(), au.end(), by_work);
  std::stable_sort(su.begin(), su.end(), by_work);
  std::vector<int2> av, sv;
  for (auto& e : au) av.push_back(e.second);
  for (auto& e : su) sv.push_back(e.second);
  SLE_TRY(mx_alloc(&p->mx_ana_units, av.size()));
  SLE_TRY(mx_alloc(&p->mx_syn_units, sv.size()));
  SLE_CUDA(cudaMemcpy(p->mx_ana_units, av.data(), av.size() * sizeof(int2), cudaMemcpyHostToDevice));
  SLE_CUDA(cudaMemcpy(p->mx_syn_units, sv.data(), sv.size() * sizeof(int2), cudaMemcpyHostToDevice));
  p->n_ana_units = (int)av.size();
  p->n_syn_units = (int)sv.size();
  d.mx_xf = p->mx_xf;
  d.mx_gns = p->mx_gns;
  d.mx_s0 = p->mx_s0;
  d.mx_abort = p->mx_abort;
  d.mx_ana_units = p->mx_ana_units;
  d.mx_syn_units = p->mx_syn_units;
  SLE_CUDA(cudaFuncSetAttribute(k_ana_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, MX_SMEM));
  SLE_CUDA(cudaFuncSetAttribute(k_syn_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, MX_SMEM));
#define SLE_ATTR_MX(NN)                                                                                        \
  do {                                                                                                         \
    SLE_CUDA(cudaFuncSetAttribute(k_fold_mx<NN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mx_fft_smem(d))); \
    SLE_CUDA(cudaFuncSetAttribute(k_unfold_mx<NN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mx_fft_smem(d))); \
  } while (0)
  SLE_FFT_SWITCH(d.n2, SLE_ATTR_MX)
#undef SLE_ATTR_MX
  p->mx_ready = 1;
  return SLE_OK;
}

static int mx_check_args(const MxFieldArgs& a, const char* what) {
  if (a.nf < 1 || a.nf > MX_MAXF) {
    set_error("%s: 1..%d fields per mixed-precision launch (got %d)", what, MX_MAXF, a.nf);
    return SLE_ERR_BAD_ARG;
  }
  if (a.ncols < 2 * a.nf || a.ncols % 16 != 0 || a.ncols > MX_NMAX) {
    set_error("%s: bad column count %d for %d fields", what, a.ncols, a.nf);
    return SLE_ERR_BAD_ARG;
  }
  return SLE_OK;
}

int mx_cols(int nf) { return std::max(16, (2 * nf + 15) / 16 * 16); }

int sht_mx_analysis(sle_sht* p, const MxFieldArgs& a0, int* status, cudaStream_t st) {
  SLE_TRY(sht_mx_prepare(p));
  MxFieldArgs a = a0;
  if (a.ncols == 0) a.ncols = mx_cols(a.nf);
  SLE_TRY(mx_check_args(a, "mixed analysis"));
  const ShtDev& d = p->d;
  ProfToken t0 = prof_begin(PROF_FFT, a.nf, st);
#define SLE_LAUNCH_MXF(NN) k_fold_mx<NN><<<dim3(d.nh, a.nf), fft_threads(NN), mx_fft_smem(d), st>>>(d, a)
  SLE_FFT_SWITCH(d.n2, SLE_LAUNCH_MXF)
#undef SLE_LAUNCH_MXF
  prof_end(t0, st);
  ProfToken t1 = prof_begin(PROF_LEG_ANA, a.nf, st);
  k_ana_tc<<<p->n_ana_units, MX_THREADS, MX_SMEM, st>>>(d, a, status);
  prof_end(t1, st);
  note_launch(2);
  SLE_CUDA(cudaGetLastError());
  return SLE_OK;
}

int sht_mx_synthesis(sle_sht* p, const MxFieldArgs& a0, int* status, cudaStream_t st) {
  SLE_TRY(sht_mx_prepare(p));
  MxFieldArgs a = a0;
  if (a.ncols == 0) a.ncols = mx_cols(a.nf);
  SLE_TRY(mx_check_args(a, "mixed synthesis"));
  const ShtDev& d = p->d;
  ProfToken t0 = prof_begin(PROF_LEG_SYN, a.nf, st);
  k_syn_tc<<<p->n_syn_units, MX_THREADS, MX_SMEM, st>>>(d, a, status);
  prof_end(t0, st);
  ProfToken t1 = prof_begin(PROF_IFFT, a.nf, st);
#define SLE_LAUNCH_MXU(NN) k_unfold_mx<NN><<<dim3(d.nh, a.nf), fft_threads(NN), mx_fft_smem(d), st>>>(d, a)
  SLE_FFT_SWITCH(d.n2, SLE_LAUNCH_MXU)
#undef SLE_LAUNCH_MXU
  prof_end(t1, st);
  note_launch(2);
  SLE_CUDA(cudaGetLastError());
  return SLE_OK;
}

int sht_mx_abort_flag(sle_sht* p, int* flag) {
  *flag = 0;
  if (!p->mx_ready) return SLE_OK;
  SLE_CUDA(cudaMemcpy(flag, p->mx_abort, sizeof(int), cudaMemcpyDeviceToHost));
  return SLE_OK;
}

}  // namespace sle
