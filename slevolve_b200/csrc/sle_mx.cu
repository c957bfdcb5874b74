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
// with each FP32 operand split as x = hi + lo, hi = x read as TF32 by the MMA (its 13 low
// mantissa bits ignored) and lo = TF32(x - hi), and D += Ahi Bhi + Ahi Blo + Alo Bhi in FP32.
//
// Precision: the Legendre values come from the FP64 recurrence of the plan
// (Q_l = mu Q_{l-1} + be_l Q_{l-2}, P~ = cf Q), rounded once to FP32 when the plan is prepared
// and stored in the tensor cores' shared-memory tile order; the kernel splits them, and the B
// operands, into TF32 hi + lo in shared memory.  The row FFTs of this form run in FP32; the
// degree-0 terms are FP64: analysis computes U_00 from FP64 row sums of the input grid,
// synthesis leaves l = 0 out of the tensor-core sum and adds its uniform contribution to the
// output grid in FP64.  The tensor core's FP32 accumulation truncates on every MMA, which for
// a sum whose terms share a sign loses about one unit in the last place per MMA: a unit's chunks
// go to two accumulator pairs in turn (chunk k to pair k mod 2, so no accumulator takes more than
// 16 of the 32 MMAs of a full unit), each pair a main accumulator for the large products
// (Ahi Bhi) beside a correction accumulator for the small ones; the epilogue adds the four in
// FP64.
// Every launch computes all MX_NMAX columns with the same accumulation structure, so a field's
// result does not depend on the other fields of its launch or on the launch shape.
//
// Kernel structure (persistent: one CTA per SM over the work units, 18 warps, 2 or 4 stages of
// one half each (a launch-shape choice), a half being one parity of one 32-wide K chunk):
//   warp 13     loader: per half, one bulk copy of the FP32 A tile (16 KB) and the B data
//               (analysis: one 4-D TMA tensor load of the folded FFT; synthesis: one bulk copy)
//               into stage q % stages
//   warps 4-11  splitters, group g takes the halves q = g mod 2: the TF32 lo tiles of A and B
//               (the FP32 tiles serve as hi; the analysis B box is first moved to the hi tile)
//   warp 12     allocates TMEM and issues the MMAs from one thread: a unit's halves of parity 0
//               (all its chunks), then those of parity 1, each parity into its own TMEM half
//   warps 0-3   epilogue, two groups (warp w reads TMEM lanes 32 (w mod 4) ..): analysis,
//   14-17       warps 0-3 parity 0 and warps 14-17 parity 1; synthesis, warps 0-3 fields 0-15 and
//               warps 14-17 fields 16-31 of both parities.  A parity's TMEM half goes to the next
//               unit's MMAs of that parity once read (the other parity's MMAs run meanwhile); the
//               accumulators are added up in FP64 and the results written
// Stages hand over through mbarriers; tcgen05.commit releases a stage when its MMAs are done.
// Every wait is bounded: on timeout the CTA raises the plan's abort flag (and the caller's status
// word), stops waiting, lets issued MMAs and copies land and releases its TMEM.  No load uses
// cluster multicast; every copy reads this GPU's own memory.
#include "sle_internal.cuh"
#include "sle_fft.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <vector>

namespace sle {
namespace {

constexpr int KC = 32;                        // K elements per chunk: one 128-byte row of TF32
constexpr int TILE_F = 128 * KC;              // words of one A tile (128 rows x 32)
constexpr int TILE_A = TILE_F * 4;            // 16 KB
constexpr int SLOT_WORDS = 2 * TILE_F;        // Legendre table slot: FP32 A tiles of both parities
constexpr int TILE_B = MX_NMAX * 128;         // MX_NMAX rows x 128 bytes = 8 KB
constexpr int STAGE_BYTES = 2 * TILE_A + 2 * TILE_B;   // one parity of a chunk: A hi / lo, B hi / lo
constexpr int NSTAGE_MAX = 4;                 // pipeline stages: 2 or 4 (a launch-time choice)
constexpr int MISC_BYTES = 1024;              // barriers + bookkeeping
constexpr int EVEN_BYTES = 128 * MX_NMAX * 4;   // synthesis: the even-degree sums of a unit (FP32, 128 rows)
constexpr int mx_smem(int nst, bool syn = false) { return 1024 + nst * STAGE_BYTES + MISC_BYTES + (syn ? EVEN_BYTES : 0); }
constexpr int W_SPL = 4;                      // warps 4..11: splitters (two groups of four)
constexpr int W_MMA = 12;                     // TMEM owner, MMA issue
constexpr int W_LOAD = 13;                    // bulk / TMA loads
constexpr int W_EPI1 = 14;                    // warps 14..17: epilogue of parity 1 (warps 0..3: parity 0)
constexpr int TC_THREADS = 18 * 32;
constexpr int ANA_SPAN = 256;                 // degrees per analysis unit (128 per parity)
constexpr long long WAIT_LIMIT = 1ll << 31;   // clock cycles (~1 s) before a wait gives up
constexpr uint32_t TMEM_COLS = 512;
constexpr uint32_t PAR_COLS = 256;            // TMEM columns per parity: NPAIR [main | correction] pairs
constexpr int NPAIR = 2;                      // accumulator pairs (chunk k into pair k mod NPAIR)
constexpr int BBLOCK = MX_NMAX * KC;          // floats of one synthesis B block
constexpr int MAX_CTA_UNITS = 16;            // work units per CTA staged in shared memory
// fixed cost of a work unit (its epilogue), in half-chunk times, from per-CTA timings at L = 511
// with 32 fields: analysis ~1180 cycles per half + ~5800 per unit, synthesis ~570 per half +
// ~13800 per unit (measured before its epilogue wrote one 16-byte store per sum pair; its CTAs
// stay within 3 % of each other)
constexpr double ANA_UNIT_COST = 5.0;
constexpr double SYN_UNIT_COST = 24.0;
constexpr int NCOLS = MX_NMAX;                // accumulator columns of every launch (2 per field slot)
static_assert(512 + 16 * MAX_CTA_UNITS <= MISC_BYTES, "misc shared memory too small");

static_assert(NSTAGE_MAX % 2 == 0, "a stage must always hold halves of one parity");
static_assert(mx_smem(NSTAGE_MAX, true) <= 232448, "mixed transform shared memory exceeds the sm_100a limit");
static_assert(TILE_B == MX_NMAX * 128, "full-width MMAs read B hi and B lo as one tile of 2 MX_NMAX rows");
static_assert(2 * NPAIR * 2 * MX_NMAX <= (int)TMEM_COLS && NPAIR * 2 * MX_NMAX == (int)PAR_COLS,
              "accumulators exceed TMEM");

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

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t a, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
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

// Bulk copy global -> this CTA's shared memory (no multicast), completion counted on `mbar`.
// Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}

// 4-D TMA tensor load (tile mode, no multicast) of the tensor map's box at (x, y, z, w).
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, int x, int y, int z, int w,
                                            uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(mbar)
      : "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void named_bar(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// AND of `v` over the `n` threads that reach named barrier `id` (all of them must).
__device__ __forceinline__ bool bar_and(int id, int n, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\tbar.red.and.pred p, %2, %3, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(id), "r"(n)
      : "memory");
  return r != 0;
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

// Offset (in 4-byte elements) of (row, k), k < 32, in a 128-byte-swizzled K-major tile.
__host__ __device__ __forceinline__ int sw_off(int row, int k) {
  return row * KC + ((((k >> 2) ^ (row & 7)) << 2) | (k & 3));
}

// ------------------------------------------------------------- precision splits
// The lo part for a hi part that is x itself read as TF32: a kind::tf32 MMA ignores the 13 low
// mantissa bits of an FP32 operand, so x serves as hi = trunc(x) unchanged and only
// lo = TF32(x - trunc(x)) is written (|x - trunc(x) - lo| <= 2^-21 |x|).
__device__ __forceinline__ uint32_t lo_of_trunc(float x) {
  const float r = x - __uint_as_float(__float_as_uint(x) & 0xFFFFE000u);
  return (__float_as_uint(r) + 0x1000u) & 0xFFFFE000u;
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

__device__ __forceinline__ bool mbar_test_wait(uint32_t a, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(a), "r"(parity)
      : "memory");
  return ok != 0;
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

// The same for the single-thread roles (loader, MMA issuer): an inline test first, then a spin
// on the non-suspending test_wait, so the thread resumes as soon as the phase completes.
__device__ __noinline__ bool mbar_spin_slow(uint32_t a, uint32_t parity, const Abort& ab) {
  const long long t0 = clock64();
  int spins = 0;
  while (!mbar_test_wait(a, parity)) {
    if ((++spins & 1023) == 0) {
      if (*reinterpret_cast<volatile int*>(ab.flag) != 0) return false;
      if (clock64() - t0 > WAIT_LIMIT) {
        raise_abort(ab);
        return false;
      }
    }
  }
  return true;
}
__device__ __forceinline__ bool mbar_spin(uint32_t a, uint32_t parity, const Abort& ab) {
  return mbar_test_wait(a, parity) || mbar_spin_slow(a, parity, ab);
}

__device__ __forceinline__ bool field_off(const MxFieldArgs& a, int f) {
  if (a.skip_set[f] && *a.skip_set[f] != 0) return true;
  if (a.skip_clear[f] && *a.skip_clear[f] == 0) return true;
  return false;
}

// Shared memory of a stage (one parity of one chunk): A tiles [hi][lo] (the parity's FP32
// Legendre tile lands in hi and is split in place), then B tiles [hi][lo] (the raw B data lands
// in lo).
struct Smem {
  uint8_t* base;        // generic pointer, 1024-aligned
  uint32_t sbase;       // shared-window address of base
  int nst;              // stages of this launch
  __device__ uint32_t a_tile(int stage, int lo) const { return sbase + stage * STAGE_BYTES + lo * TILE_A; }
  __device__ uint8_t* a_ptr(int stage, int lo) const { return base + stage * STAGE_BYTES + lo * TILE_A; }
  __device__ uint32_t b_tile(int stage, int lo) const {
    return sbase + stage * STAGE_BYTES + 2 * TILE_A + lo * TILE_B;
  }
  __device__ uint8_t* b_ptr(int stage, int lo) const { return base + stage * STAGE_BYTES + 2 * TILE_A + lo * TILE_B; }
  __device__ uint8_t* misc() const { return base + nst * STAGE_BYTES; }
  __device__ float* even() const { return reinterpret_cast<float*>(base + nst * STAGE_BYTES + MISC_BYTES); }
};

__device__ __forceinline__ Smem smem_layout(uint8_t* raw, int nst) {
  const uint32_t s = smem_u32(raw);
  const uint32_t al = (s + 1023u) & ~1023u;
  return Smem{raw + (al - s), al, nst};
}

// Barriers: full[nst] (splitters -> MMA), empty[nst] (MMA commit -> loader), raw[nst] (copies
// landed -> splitters), accum[2] (a unit's MMAs of one parity done -> epilogue), tfree[2]
// (epilogue done reading that parity's accumulators -> MMA), drain (MMAs issued before an
// abort); each stage group has room for the largest stage count.
enum { BAR_FULL = 0, BAR_EMPTY = NSTAGE_MAX, BAR_RAW = 2 * NSTAGE_MAX, BAR_ACCUM = 3 * NSTAGE_MAX,
       BAR_TFREE = 3 * NSTAGE_MAX + 2, BAR_DRAIN = 3 * NSTAGE_MAX + 4, NBAR = 3 * NSTAGE_MAX + 5 };
static_assert(NBAR * 8 <= 192, "barrier area too small");
struct Misc {
  uint64_t* bar;
  uint32_t* tmem_holder;
  int* active;          // [MX_MAXF]
  int* any;
  int4* units;          // [MAX_CTA_UNITS]: this CTA's work units, staged by the prologue
  __device__ uint32_t b(int i) const { return smem_u32(bar + i); }
};
__device__ __forceinline__ Misc misc_layout(const Smem& S) {
  uint8_t* p = S.misc();
  Misc m;
  m.bar = reinterpret_cast<uint64_t*>(p);                      // 17 barriers
  m.tmem_holder = reinterpret_cast<uint32_t*>(p + 192);
  m.active = reinterpret_cast<int*>(p + 256);
  m.any = reinterpret_cast<int*>(p + 256 + 4 * MX_MAXF);
  m.units = reinterpret_cast<int4*>(p + 512);
  return m;
}

// TMEM use (512 columns): per parity p, at 256 p, NPAIR accumulator pairs of 2N columns (N =
// MX_NMAX): pair b holds the main accumulator (Ahi*Bhi of the chunks k = b mod NPAIR) and right
// after it the correction accumulator (Ahi*Blo + Alo*Bhi of the same chunks), so that Ahi*Bhi and
// Ahi*Blo are one MMA of 2N columns over the adjacent B hi and B lo tiles.  Every launch computes
// all N columns (2 per field slot; slots beyond the launch's fields are not read), so that a
// field's accumulation does not depend on how many fields share its launch.  A unit runs its
// parity-0 halves first, then its parity-1 halves: while the epilogue drains one parity's half of
// TMEM, the MMAs of the other parity run.

// MMAs of one parity `par` of chunk k of a unit (stage st): four K steps of 8, each one
// M128 x N128 MMA (Ahi [Bhi | Blo] into [main | correction]) and one M128 x N64 (Alo Bhi into the
// correction).  The K sub-block kk starts 32 kk bytes into the tile rows: +2 kk in the
// descriptor's start-address field.
__device__ __forceinline__ void mma_half(const Smem& S, uint32_t tmem, int st, int par, int k) {
  const uint64_t ah = sdesc_sw128(S.a_tile(st, 0)), al = sdesc_sw128(S.a_tile(st, 1));
  const uint64_t bh = sdesc_sw128(S.b_tile(st, 0));
  const uint32_t idesc = idesc_tf32(128, NCOLS), idesc2 = idesc_tf32(128, 2 * NCOLS);
  // B hi rows [0, N) and B lo rows [0, N) are 2N consecutive rows (TILE_B = N rows)
  const uint32_t dm = tmem + PAR_COLS * (uint32_t)par + (uint32_t)(2 * NCOLS * (k % NPAIR));
  const uint32_t dc = dm + (uint32_t)NCOLS;
  const bool fresh = k < NPAIR;
#pragma unroll
  for (int kk = 0; kk < KC / 8; ++kk) {
    const uint64_t d = (uint64_t)(2 * kk);
    tc_mma_tf32(dm, ah + d, bh + d, idesc2, (fresh && kk == 0) ? 0u : 1u);   // [main | corr]
    tc_mma_tf32(dc, al + d, bh + d, idesc, 1u);
  }
}

// Accumulator columns [16 cb, 16 cb + 16) of one parity (TMEM address `base` of this thread's
// lane and that parity), summed in FP64 over the pairs in use (min(nch, NPAIR)): the corrections
// first, then the main accumulators.  All loads of a block are issued before one wait.
__device__ __forceinline__ void acc_read(uint32_t base, int nch, int cb, double (&v)[16]) {
  uint32_t c0[16], c1[16], m0[16], m1[16];
  const uint32_t off = (uint32_t)(16 * cb);
  tc_ld16(base + (uint32_t)NCOLS + off, c0);
  tc_ld16(base + off, m0);
  if (nch > 1) {
    tc_ld16(base + (uint32_t)(3 * NCOLS) + off, c1);
    tc_ld16(base + (uint32_t)(2 * NCOLS) + off, m1);
  }
  tc_wait_ld();
  if (nch > 1) {
#pragma unroll
    for (int u = 0; u < 16; ++u)
      v[u] = (((double)__uint_as_float(c0[u]) + (double)__uint_as_float(c1[u])) + (double)__uint_as_float(m0[u])) +
             (double)__uint_as_float(m1[u]);
  } else {
#pragma unroll
    for (int u = 0; u < 16; ++u) v[u] = (double)__uint_as_float(c0[u]) + (double)__uint_as_float(m0[u]);
  }
}

// Common prologue: barriers, gates, TMEM.  Returns the TMEM base (all threads).
__device__ uint32_t prologue(const Smem& S, const Misc& M, const MxFieldArgs& a, const int4* units, int2 rg,
                             int tfree_warps) {
  const int warp = threadIdx.x >> 5;
  if (threadIdx.x < MAX_CTA_UNITS && (int)threadIdx.x < rg.y) M.units[threadIdx.x] = units[rg.x + threadIdx.x];
  if (threadIdx.x == 0) {
    for (int i = 0; i < S.nst; ++i) {
      mbar_init(M.b(BAR_FULL + i), 4);    // the 4 splitter warps of the stage
      mbar_init(M.b(BAR_EMPTY + i), 1);   // one tcgen05.commit
      mbar_init(M.b(BAR_RAW + i), 1);     // loader's expect_tx
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(M.b(BAR_ACCUM + i), 1);   // one tcgen05.commit (or arrive for an empty unit)
      mbar_init(M.b(BAR_TFREE + i), tfree_warps);   // the epilogue warps that read the parity
    }
    mbar_init(M.b(BAR_DRAIN), 1);
    fence_mbar_init();
  }
  if (threadIdx.x < MX_MAXF) M.active[threadIdx.x] = (threadIdx.x < a.nf) && !field_off(a, threadIdx.x);
  if (warp == W_MMA) {
    tc_alloc(smem_u32(M.tmem_holder), TMEM_COLS);
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

__device__ void epilogue_release(uint32_t tmem) {
  tc_fence_before();
  __syncthreads();
  if ((threadIdx.x >> 5) == W_MMA) {
    tc_fence_after();
    tc_dealloc(tmem, TMEM_COLS);
  }
}

// Wait for a phase with only the time limit (not the abort flag): used to let copies already
// in flight land before the CTA exits.
__device__ __noinline__ void mbar_wait_drain(uint32_t a, uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_try_wait(a, parity)) {
    if (clock64() - t0 > WAIT_LIMIT) return;
  }
}

// ===================================================== Legendre tables (once per plan)
// The A operand of every chunk is precomputed from the FP64 recurrence, rounded to FP32 and
// stored in the tile order of the shared-memory stage: slot = [par0][par1], each 128 rows x 32
// (2 TILE_F words); the transform kernel splits it into TF32 hi / lo.  Entries below the
// significance threshold of their (segment, latitude group) and rows or columns outside the
// unit stay zero (the table is zeroed first).

// Analysis unit (m, span s): rows r of parity p = degree lbase + 2r + p, K = latitudes
// 32c .. 32c + 31 for the chunks c = kstart .. ngrp - 1.  Warp (segment q, chunk parity g).
__global__ void __launch_bounds__(256) k_tab_ana(ShtDev P, uint32_t* tab) {
  const int4 unit = P.mx_ana_units[blockIdx.x];
  const int m = unit.x, s = unit.y, kstart = unit.z;
  const long long off = unit.w;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = warp & 3, g = warp >> 2;
  const int L = P.lmax;
  const int lbase = m + ANA_SPAN * s;
  const int nd = min(ANA_SPAN, L + 1 - lbase);
  if (SEG * q >= nd) return;
  const int seg = P.segoff[m] + (ANA_SPAN / SEG) * s + q;
  const int len = min(SEG, nd - SEG * q);
  const long long cbase = P.moff[m] + (lbase - m) + SEG * q;
  for (int c = kstart + g; c < P.ngrp; c += 2) {
    if (c < (int)P.istart[seg]) continue;
    uint32_t* slot = tab + (off + (c - kstart)) * SLOT_WORDS;
    const int j = KC * c + lane;
    const double mu = P.mu[j];
    const double2 sd = P.seeds[(size_t)seg * P.nh + j];
    double qa = sd.x, qb = sd.y;
    for (int t = 0; t < len; ++t) {
      const double qn = fma(mu, qb, P.be[cbase + t] * qa);
      qa = qb;
      qb = qn;
      const int o = sw_off(SEG / 2 * q + (t >> 1), lane);
      slot[(t & 1) * TILE_F + o] = __float_as_uint(__double2float_rn(P.cf[cbase + t] * qn));
    }
  }
}

// Synthesis unit (m, latitude tile t): rows = latitudes 128 t + row, chunk i = segment
// seg_list[off + i] of m (K = the degree's index in its parity).  Thread per latitude row.
__global__ void __launch_bounds__(128) k_tab_syn(ShtDev P, uint32_t* tab) {
  const int4 unit = P.mx_syn_units[blockIdx.x];
  const int m = unit.x, t = unit.y, nch = unit.z;
  const long long off = unit.w;
  const int row = threadIdx.x;
  const int j = 128 * t + row;
  if (j >= P.nh) return;
  const int grp = j >> 5;
  const double mu = P.mu[j];
  for (int i = 0; i < nch; ++i) {
    const int seg = P.mx_syn_seg[off + i];
    if (grp < (int)P.istart[seg]) continue;
    const int l0 = P.seg_l0[seg];
    const int len = min(SEG, P.lmax + 1 - l0);
    const long long cbase = P.moff[m] + (l0 - m);
    uint32_t* slot = tab + (off + i) * SLOT_WORDS;
    const double2 sd = P.seeds[(size_t)seg * P.nh + j];
    double qa = sd.x, qb = sd.y;
    for (int tt = 0; tt < len; ++tt) {
      const double qn = fma(mu, qb, P.be[cbase + tt] * qa);
      qa = qb;
      qb = qn;
      const int o = sw_off(row, tt >> 1);
      slot[(tt & 1) * TILE_F + o] = __float_as_uint(__double2float_rn(P.cf[cbase + tt] * qn));
    }
  }
}

// ============================================================ Legendre contraction
// A split: the FP32 Legendre values landed in the hi tile of the stage and serve as hi as they
// are (the MMA reads them as TF32, trunc(x)); the lo tile gets TF32(x - trunc(x)).  Elementwise,
// so the tile order does not matter.
__device__ __forceinline__ void split_a(const Smem& S, int st, int tid) {
  constexpr int NV = TILE_F / 4 / 128;   // 16-byte vectors per thread
  const uint4* hp = reinterpret_cast<const uint4*>(S.a_ptr(st, 0));
  uint4* lp = reinterpret_cast<uint4*>(S.a_ptr(st, 1));
  uint4 v[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) v[q] = hp[tid + 128 * q];
#pragma unroll
  for (int q = 0; q < NV; ++q)
    lp[tid + 128 * q] = make_uint4(lo_of_trunc(__uint_as_float(v[q].x)), lo_of_trunc(__uint_as_float(v[q].y)),
                                   lo_of_trunc(__uint_as_float(v[q].z)), lo_of_trunc(__uint_as_float(v[q].w)));
}

// Analysis B data of one parity: the TMA box of the folded FFT is [field][32 latitudes][re, im]
// (8 bytes per entry) in the stage's B lo tile; the 4 splitter warps read it, synchronise, and
// write rows 2f (re) / 2f+1 (im) of the B hi tile (the FP32 values, read as TF32 by the MMA)
// and of the B lo tile (TF32 of x - trunc(x)).
__device__ __forceinline__ void split_b_ana(const Smem& S, int st, int nf, int tid, int bar_id) {
  const float2* box = reinterpret_cast<const float2*>(S.b_ptr(st, 1));
  float2 v[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int e = tid + 128 * u;
    v[u] = ((e >> 5) < nf) ? box[e] : make_float2(0.f, 0.f);
  }
  named_bar(bar_id, 128);
  uint32_t* hp = reinterpret_cast<uint32_t*>(S.b_ptr(st, 0));
  uint32_t* lp = reinterpret_cast<uint32_t*>(S.b_ptr(st, 1));
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int e = tid + 128 * u;
    const int f = e >> 5, k = e & 31;
    if (f >= nf) continue;
    const int o0 = sw_off(2 * f, k), o1 = sw_off(2 * f + 1, k);
    hp[o0] = __float_as_uint(v[u].x);
    lp[o0] = lo_of_trunc(v[u].x);
    hp[o1] = __float_as_uint(v[u].y);
    lp[o1] = lo_of_trunc(v[u].y);
  }
}

// Synthesis B data of one parity: the raw block lands in the hi tile, already in the tile order,
// and serves as hi as it is; the lo tile gets TF32(x - trunc(x)).
__device__ __forceinline__ void split_b_syn(const Smem& S, int st, int nrow, int tid) {
  const uint32_t* hp = reinterpret_cast<const uint32_t*>(S.b_ptr(st, 0));
  uint32_t* lp = reinterpret_cast<uint32_t*>(S.b_ptr(st, 1));
  for (int e = tid; e < nrow * KC; e += 128) lp[e] = lo_of_trunc(__uint_as_float(hp[e]));
}

// Work unit u (the CTA's i-th): (m, span | latitude tile, chunk count, first table slot).
template <bool SYN>
__device__ __forceinline__ void unit_info(const ShtDev& P, const Misc& M, int u, int i, int4& unit, int& nch) {
  unit = (i < MAX_CTA_UNITS) ? M.units[i] : (SYN ? P.mx_syn_units[u] : P.mx_ana_units[u]);
  nch = SYN ? unit.z : P.ngrp - unit.z;
}

// Persistent CTAs (one per SM), each over its own run of work units (P.mx_*_cta).  Analysis
// units: rows of D = degrees, columns = (Re, Im) of the fields; synthesis: rows = latitudes.
// The CTA's work is a sequence of halves q (per unit: parity 0 of its chunks 0 .. nch - 1, then
// parity 1 of the same chunks): warp 13 streams each half's Legendre tile and B data into stage
// q % NST; splitter group g = (warp - 4) / 4 splits the halves q = g mod 2 (the stages of that
// parity); warp 12 issues the MMAs of a unit's parity p once the epilogue has read parity p of
// the unit before out of TMEM; warps 0-3 and 14-17 drain the unit (analysis: one parity per
// group; synthesis: one half of the fields per group, both parities).
template <bool SYN, int NST>
__global__ void __launch_bounds__(TC_THREADS, 1)
    k_leg_tc(ShtDev P, MxFieldArgs a, int* status, const __grid_constant__ CUtensorMap tmx, int zbox) {
  static_assert(NST % 2 == 0 && NST <= NSTAGE_MAX, "stage count");
  extern __shared__ uint8_t smraw[];
  pdl_trigger();   // one CTA per SM, all resident: the next kernel may queue behind them
  const Smem S = smem_layout(smraw, NST);
  const Misc M = misc_layout(S);
  const Abort ab{P.mx_abort, status};
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int L = P.lmax;
  const uint32_t* tab = SYN ? P.mx_tab_syn : P.mx_tab_ana;
  // this CTA's work units: rg.y units from rg.x on (the plan balances the CTAs' totals)
  const int2 rg = (SYN ? P.mx_syn_cta : P.mx_ana_cta)[blockIdx.x];
  const uint32_t tmem = prologue(S, M, a, SYN ? P.mx_syn_units : P.mx_ana_units, rg, SYN ? 8 : 4);
  if (*M.any && *reinterpret_cast<volatile int*>(P.mx_abort) == 0) {
    const int nrow = 2 * a.nf;
    if (warp == W_LOAD) {
      // ---- loader: half q of the CTA's sequence into stage q % NST
      if (lane == 0) {
        const uint32_t bbytes = SYN ? (uint32_t)nrow * 128u : (uint32_t)zbox * 32u * 8u;
        int q = 0, i = 0;
        bool ok = true;
        for (int u = rg.x; i < rg.y && ok; ++u, ++i) {
          int4 unit;
          int nch;
          unit_info<SYN>(P, M, u, i, unit, nch);
          for (int h = 0; h < 2 * nch; ++h, ++q) {
            const int par = h >= nch ? 1 : 0, k = h - par * nch, st = q % NST;
            if (!mbar_spin(M.b(BAR_EMPTY + st), (uint32_t)(((q / NST) & 1) ^ 1), ab)) {
              ok = false;
              break;
            }
            const uint32_t raw = M.b(BAR_RAW + st);
            mbar_arrive_expect_tx(raw, (uint32_t)TILE_A + bbytes);
            bulk_g2s(S.a_tile(st, 0), tab + ((long long)unit.w + k) * SLOT_WORDS + par * TILE_F, (uint32_t)TILE_A,
                     raw);
            if (SYN) {
              const int seg = P.mx_syn_seg[unit.w + k];
              bulk_g2s(S.b_tile(st, 0), P.mx_bsyn + ((size_t)seg * 2 + par) * BBLOCK, (uint32_t)nrow * 128u, raw);
            } else {
              tma_load_4d(S.b_tile(st, 1), &tmx, 2 * KC * (unit.z + k), par, unit.x, 0, raw);
            }
          }
        }
        // copies in flight land before the CTA exits: the last phase issued on each stage
        for (int st = 0; st < NST; ++st) {
          const int n_st = (q + NST - 1 - st) / NST;   // loads issued on stage st
          if (n_st > 0) mbar_wait_drain(M.b(BAR_RAW + st), (uint32_t)((n_st - 1) & 1));
        }
      }
      __syncwarp();
    } else if (warp == W_MMA) {
      if (lane == 0) {
        int q = 0, i = 0;
        bool ok = true, issued = false;
        for (int u = rg.x; i < rg.y && ok; ++u, ++i) {
          int4 unit;
          int nch;
          unit_info<SYN>(P, M, u, i, unit, nch);
          for (int par = 0; par < 2 && ok; ++par) {
            if (!mbar_spin(M.b(BAR_TFREE + par), (uint32_t)((i & 1) ^ 1), ab)) {
              ok = false;
              break;
            }
            tc_fence_after();
            for (int k = 0; k < nch; ++k, ++q) {
              const int st = q % NST;
              if (!mbar_spin(M.b(BAR_FULL + st), (uint32_t)((q / NST) & 1), ab)) {
                ok = false;
                break;
              }
              tc_fence_after();
              mma_half(S, tmem, st, par, k);
              issued = true;
              tc_commit(M.b(BAR_EMPTY + st));
            }
            if (!ok) break;
            if (nch > 0) tc_commit(M.b(BAR_ACCUM + par));
            else mbar_arrive(M.b(BAR_ACCUM + par));
          }
        }
        if (!ok && issued) {
          // aborted: let the MMAs already issued finish (bounded) before TMEM is released
          tc_commit(M.b(BAR_DRAIN));
          mbar_wait_drain(M.b(BAR_DRAIN), 0u);
        }
      }
      __syncwarp();
    } else if (warp >= W_SPL && warp < W_MMA) {
      // ---- splitters: group g takes the halves q = g mod 2 (the stages of that parity)
      const int g = (warp - W_SPL) >> 2, tid = threadIdx.x - 32 * W_SPL - 128 * g;
      int q = 0, i = 0;
      bool ok = true;
      for (int u = rg.x; i < rg.y && ok; ++u, ++i) {
        int4 unit;
        int nch;
        unit_info<SYN>(P, M, u, i, unit, nch);
        for (int h = 0; h < 2 * nch; ++h, ++q) {
          if ((q & 1) != g) continue;
          const int st = q % NST;
          // every wait is bounded, so all four warps of the group reach the vote; they go on
          // (and meet at the named barrier of the B split) only together
          const bool w = mbar_wait(M.b(BAR_RAW + st), (uint32_t)((q / NST) & 1), ab);
          if (!bar_and(1 + g, 128, w)) {
            ok = false;
            break;
          }
          split_a(S, st, tid);
          if (SYN) split_b_syn(S, st, nrow, tid);
          else split_b_ana(S, st, a.nf, tid, 1 + g);
          fence_proxy_async();
          __syncwarp();
          if (lane == 0) mbar_arrive(M.b(BAR_FULL + st));
        }
      }
    } else if (SYN) {
      // ---- synthesis epilogue: warps 0-3 take the fields 0-15, warps 14-17 the fields 16-31
      // (column blocks 2h, 2h + 1 for group h), of both parities; warp w owns TMEM lanes
      // 32 (w mod 4) .. 32 (w mod 4) + 31.  The even-degree sums wait in shared memory (FP32, each
      // thread its own row: [column][row]) until the odd-degree ones are read, so that each
      // (field, latitude, order) gets one 16-byte store.
      const int h = warp >= W_EPI1 ? 1 : 0;
      const int r = 32 * (warp & 3) + lane;
      int i = 0;
      for (int u = rg.x; i < rg.y; ++u, ++i) {
        int4 unit;
        int nch;
        unit_info<SYN>(P, M, u, i, unit, nch);
        const int m = unit.x;
        const int j = 128 * unit.y + r;                 // latitude of row r
        const uint32_t rowbase = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
        const int ncb = (2 * a.nf + 15) / 16;
        const int cb0 = 2 * h, cb1 = min(ncb, 2 * h + 2);
        float4* gq = reinterpret_cast<float4*>(P.mx_gns) + (size_t)j * P.nm + m;
        const size_t gfield = (size_t)P.nh * P.nm;
        float* ev = S.even() + r;
        bool okp = true;
        for (int par = 0; par < 2; ++par) {
          const bool w = mbar_wait(M.b(BAR_ACCUM + par), (uint32_t)(i & 1), ab);
          if (!__all_sync(0xffffffffu, w)) {
            okp = false;
            break;
          }
          tc_fence_after();
#pragma unroll 1
          for (int cb = cb0; cb < cb1; ++cb) {
            double v[16];
            if (nch > 0) {
              acc_read(rowbase + PAR_COLS * (uint32_t)par, nch, cb, v);
            } else {
#pragma unroll
              for (int q = 0; q < 16; ++q) v[q] = 0.0;
            }
            if (par == 0) {
#pragma unroll
              for (int q = 0; q < 16; ++q) ev[(16 * cb + q) * 128] = (float)v[q];
            } else if (j < P.nh) {
#pragma unroll
              for (int q = 0; q < 8; ++q) {
                const int f = 8 * cb + q;
                if (f >= a.nf || !M.active[f]) continue;
                // the even- and odd-degree sums E, O of latitude j (the unfold forms E +- O)
                gq[f * gfield] = make_float4(ev[(16 * cb + 2 * q) * 128], ev[(16 * cb + 2 * q + 1) * 128], (float)v[2 * q],
                                             (float)v[2 * q + 1]);
              }
            }
          }
          // this group's columns of the parity are in registers: its TMEM half goes to the next
          // unit once both groups have read it
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(M.b(BAR_TFREE + par));
        }
        if (!okp) break;
      }
    } else {
      // ---- analysis epilogue: warps 0-3 (parity 0) and 14-17 (parity 1); warp w owns TMEM lanes
      // 32 (w mod 4) .. 32 (w mod 4) + 31
      const int par = warp >= W_EPI1 ? 1 : 0;
      const int r = 32 * (warp & 3) + lane;
      const double inv = 1.0 / SQRT2_LEGACY;
      int i = 0;
      for (int u = rg.x; i < rg.y; ++u, ++i) {
        int4 unit;
        int nch;
        unit_info<SYN>(P, M, u, i, unit, nch);
        const int m = unit.x;
        const uint32_t lanebase = tmem + PAR_COLS * (uint32_t)par + ((uint32_t)(32 * (warp & 3)) << 16);
        const int le = m + ANA_SPAN * unit.y + 2 * r;   // even degree of row r
        const int ncb = (2 * a.nf + 15) / 16;
        // this thread's output element: coefficient (le + par, m) of every field (when le + par <= L)
        const long long abase = (long long)P.moff[m] + (le - m);
        const bool w = mbar_wait(M.b(BAR_ACCUM + par), (uint32_t)(i & 1), ab);
        if (!__all_sync(0xffffffffu, w)) break;
        tc_fence_after();
        const bool live = le + par <= L;
        for (int cb = 0; cb < ncb; ++cb) {
          double v[16];
          if (nch > 0) {
            acc_read(lanebase, nch, cb, v);
          } else {
#pragma unroll
            for (int q = 0; q < 16; ++q) v[q] = 0.0;
          }
          if (cb == ncb - 1) {
            // this parity's accumulators are in registers: its TMEM half goes to the next unit
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(M.b(BAR_TFREE + par));
          }
          if (!live) continue;
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const int f = 8 * cb + q;
            if (f >= a.nf || !M.active[f]) continue;
            a.spec[f][abase + par] = make_double2(v[2 * q] * inv, v[2 * q + 1] * inv);
          }
        }
        if (par == 0 && m == 0 && unit.y == 0) {
          // degree 0 in FP64 from the row sums of the fold: U_00 = sqrt(0.5) sum_j S_0(j) / 1.41421356;
          // warp w sums the fields w, w + 4, ... (lane-strided partial sums, then a fixed
          // butterfly: the same order in every launch)
          __syncwarp();
          for (int f = warp; f < a.nf; f += 4) {
            if (!M.active[f]) continue;
            const double* s0 = P.mx_s0 + (size_t)f * P.nh;
            double acc = 0.0;
            for (int jj = lane; jj < P.nh; jj += 32) acc += s0[jj];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) a.spec[f][0] = make_double2(__dmul_rn(__dsqrt_rn(0.5), acc) / SQRT2_LEGACY, 0.0);
          }
        }
      }
    }
  }
  epilogue_release(tmem);
}

// ============================================================== row FFT kernels
// Row rFFT in FP32 of the north and south rows of the NR / 2 latitudes j0 = (NR / 2) blockIdx.x
// .. of field blockIdx.y (NR = 4 or 8 rows per block, a launch-shape choice) and the fold with
// the weights, output FP32: X[f][m][0][j] = S, X[f][m][1][j] = D (complex, 8 bytes per entry),
// latitude fastest (four latitudes fill one 32-byte sector of each plane), the layout whose 32-latitude rows of one parity the analysis
// kernel's TMA box reads.  The m = 0
// fold (the weighted row sums) is formed in FP64 from the FP64 grid values, in s0[f][j], for the
// FP64 degree-0 coefficient.
template <int K>
struct FoldSrcMx {
  TypedPairRows<K> src;
  double* acc;          // this thread's FP64 sum of the values it reads (one row per thread)
  __device__ __forceinline__ float2 operator()(int r, int i) const {
    const double2 v = src(r, i);
    *acc = (*acc + v.x) + v.y;
    return make_float2((float)v.x, (float)v.y);
  }
};

// The FP32 row FFTs of NR / 2 latitude pairs for a source kind known at compile time.
template <int N, int NR>
struct FoldRowsMx {
  const double* g;
  const unsigned char* m0;
  const unsigned char* m1;
  int j0, nlat;
  const float2* tw;
  float2* A;
  double* acc;
  template <int K>
  __device__ __forceinline__ void operator()() const {
    fft_rows<NR, N, false>(FoldSrcMx<K>{TypedPairRows<K>{g, m0, m1, j0, nlat, 2 * N}, acc}, A, tw,
                                SmemRows<N, float2>{A});
  }
};

template <int N, int NR>
__global__ void __launch_bounds__(fft_nt(NR, N), fft_nt(NR, N) <= 512 ? 3 : 1) k_fold_mx(ShtDev P, MxFieldArgs a) {
  extern __shared__ float2 smf2[];
  float2* A = smf2;
  constexpr int NLAT = NR / 2;               // latitudes of the block
  const int j0 = NLAT * blockIdx.x, f = blockIdx.y;
  pdl_wait();
  pdl_trigger();
  if (field_off(a, f)) return;
  constexpr int NT = fft_nt(NR, N);
  constexpr int Q = N / FftRadix<N, 1>::R;   // first-pass items per row: one per thread
  double acc = 0.0;
  with_src_kind(a.kind[f], FoldRowsMx<N, NR>{a.grid[f], a.m0[f], a.m1[f], j0, P.nlat, P.twf, A, &acc});
  // FP64 row sums: the Q threads r Q .. r Q + Q - 1 hold the partial sums of row r (Q a power
  // of two): a butterfly within aligned groups of min(Q, 32) lanes, then the warps of a row in
  // order
  __shared__ double rowtot[NR];
  {
    const int t = threadIdx.x;
    double v = (t < NR * Q) ? acc : 0.0;
    constexpr int W = Q < 32 ? Q : 32;
#pragma unroll
    for (int o = W / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if constexpr (Q <= 32) {
      if (t < NR * Q && t % Q == 0) rowtot[t / Q] = v;
    } else {
      __shared__ double wsum[NT / 32];
      if ((t & 31) == 0) wsum[t >> 5] = v;
      __syncthreads();
      if (t < NR) {
        double sum = 0.0;
        for (int w = t * (Q / 32); w < (t + 1) * (Q / 32); ++w) sum += wsum[w];
        rowtot[t] = sum;
      }
    }
    __syncthreads();
  }
  const SmemRows<N, float2> Z{A};
  float2* X = reinterpret_cast<float2*>(P.mx_xf) + (size_t)f * P.nm * P.nh * 2;
  for (int e = threadIdx.x; e < NLAT * P.nm; e += NT) {
    // consecutive threads: the latitudes of one order (one 32-byte sector of each X plane)
    const int m = e / NLAT, q = e % NLAT, j = j0 + q;
    float2 xr[2];
    const float2 twm = (m > 0 && m < N) ? __ldg(P.twf + m) : make_float2(1.f, 0.f);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int r = 2 * q + h;
      const float2 z0 = Z(r, 0);
      if (m == 0) {
        xr[h] = make_float2(z0.x + z0.y, 0.f);
      } else if (m == N) {
        xr[h] = make_float2(z0.x - z0.y, 0.f);
      } else {
        const float2 zm = Z(r, m);
        const float2 zn = Z(r, N - m);
        const float2 zc = make_float2(zn.x, -zn.y);
        const float2 ev = cscale(cadd(zm, zc), 0.5f);
        const float2 dz = csub(zm, zc);
        const float2 o = make_float2(0.5f * dz.y, -0.5f * dz.x);  // (zm - zc) / (2i)
        xr[h] = cadd(ev, cmul(twm, o));
      }
    }
    const double wn = P.wn[j], ws = P.ws[j];
    const float2 an = cscale(xr[0], (float)wn), bs = cscale(xr[1], (float)ws);
    if (m == 0) {
      // S_0(j) in FP64: the weighted sums of the north and south rows of latitude j
      P.mx_s0[(size_t)f * P.nh + j] = wn * rowtot[2 * q] + ws * rowtot[2 * q + 1];
    }
    X[((size_t)m * 2 + 0) * P.nh + j] = make_float2(an.x + bs.x, an.y + bs.y);   // S (even l - m)
    X[((size_t)m * 2 + 1) * P.nh + j] = make_float2(an.x - bs.x, an.y - bs.y);   // D (odd l - m)
  }
}

// Inverse: even- and odd-degree Legendre sums E, O of field blockIdx.y (FP32, m <= lmax, 0
// above; one 16-byte entry per order, north = E + O and south = E - O formed in FP32 as they are
// read), unnormalised inverse real FFT in FP32; the output rows get the FP64
// degree-0 term 1.41421356 sqrt(0.5) Re U_00 added in FP64; optional epilogue out2 = grid * mul2.
// The half-length complex packing of the real inverse transform is formed while the first FFT
// pass reads its inputs; the last pass writes the output rows.
template <int N>
struct UnfoldSrcMx {
  const float4* G;   // [m] of this latitude pair
  const float2* tw;
  int nm;
  __device__ __forceinline__ float2 g(int r, int m) const {
    if (m >= nm) return make_float2(0.f, 0.f);
    const float4 v = __ldg(G + m);   // (E, O): north = E + O, south = E - O
    return r ? make_float2(v.x - v.z, v.y - v.w) : make_float2(v.x + v.z, v.y + v.w);
  }
  __device__ __forceinline__ float2 operator()(int r, int m) const {
    float2 x, y;
    if (m == 0) {
      x = make_float2(g(r, 0).x, 0.f);
      y = make_float2(g(r, N).x, 0.f);
    } else {
      x = g(r, m);
      const float2 c = g(r, N - m);
      y = make_float2(c.x, -c.y);
    }
    const float2 e = cadd(x, y);
    const float2 t = __ldg(tw + m);
    const float2 wc = make_float2(t.x, -t.y);  // exp(+2 pi i m / nlon)
    const float2 o = cmul(csub(x, y), wc);
    return make_float2(e.x - o.y, e.y + o.x);  // e + i o
  }
};

// FP32 values of the inverse FFT -> FP64 grid rows plus the degree-0 term.
struct GridRowsOutMx {
  GridRowsOut out;
  double c00;
  __device__ __forceinline__ void put(int r, int i, float2 v) const {
    out.put(r, i, make_double2((double)v.x + c00, (double)v.y + c00));
  }
};

// `ahead`: the blocks resident on the device at once; the sums of the block that many places
// further on (and the multiplier rows of its epilogue) are prefetched into L2.
template <int N>
__global__ void __launch_bounds__(fft_nt(2, N)) k_unfold_mx(ShtDev P, MxFieldArgs a, int ahead) {
  extern __shared__ float2 smf2[];
  float2* A = smf2;
  const int j = blockIdx.x, f = blockIdx.y;
  pdl_wait();
  pdl_trigger();
  int bx, by;
  if (threadIdx.x < 3 && block_ahead(ahead, bx, by) && !field_off(a, by)) {
    if (threadIdx.x == 0) {
      prefetch_l2(reinterpret_cast<const float4*>(P.mx_gns) + ((size_t)by * P.nh + bx) * P.nm,
                  (uint32_t)(P.nm * sizeof(float4)));
    } else if (a.epi_out[by]) {
      const int row = (threadIdx.x == 1) ? bx : P.nlat - 1 - bx;
      prefetch_l2(a.epi_mul[by] + (size_t)row * (2 * N), (uint32_t)(2 * N * sizeof(double)));
    }
  }
  if (field_off(a, f)) return;
  const int js = P.nlat - 1 - j;
  const float4* G = reinterpret_cast<const float4*>(P.mx_gns) + ((size_t)f * P.nh + j) * P.nm;
  const double c00 = __dmul_rn(__dmul_rn(SQRT2_LEGACY, a.spec[f][0].x), __dsqrt_rn(0.5));
  const size_t ro = (size_t)j * (2 * N), rso = (size_t)js * (2 * N);
  double* out2 = a.epi_out[f];
  const double* mul2 = a.epi_mul[f];
  const GridRowsOut rows{reinterpret_cast<double2*>(a.grid[f] + ro), reinterpret_cast<double2*>(a.grid[f] + rso),
                         out2 ? reinterpret_cast<double2*>(out2 + ro) : nullptr,
                         out2 ? reinterpret_cast<double2*>(out2 + rso) : nullptr,
                         out2 ? reinterpret_cast<const double2*>(mul2 + ro) : nullptr,
                         out2 ? reinterpret_cast<const double2*>(mul2 + rso) : nullptr};
  fft_rows<2, N, true>(UnfoldSrcMx<N>{G, P.twf, P.nm}, A, P.twf, GridRowsOutMx{rows, c00});
}

// Synthesis B operand: per segment s (order m, degrees l0..l0+63) and parity, rows 2f / 2f+1 =
// Re / Im of 1.41421356 U_f[l, m] rounded to FP32, k = the degree's index in its parity, in the
// tile order (MX_NMAX x 32 per block).  l = 0 is left out (the inverse FFT adds it in FP64);
// degrees beyond lmax are zero.  Block (segment, group of 4 fields), 64 threads per field.
__global__ void __launch_bounds__(256) k_bsyn_mx(ShtDev P, MxFieldArgs a) {
  const int s = blockIdx.x;
  const int f = 4 * blockIdx.y + (threadIdx.x >> 6);
  const int t = threadIdx.x & 63;
  if (f >= a.nf || field_off(a, f)) return;
  const int m = P.seg_m[s], l0 = P.seg_l0[s];
  const int len = min(SEG, P.lmax + 1 - l0);
  double2 u = make_double2(0.0, 0.0);
  if (t < len && !(m == 0 && l0 + t == 0)) u = a.spec[f][P.moff[m] + (l0 - m) + t];
  float* blk = P.mx_bsyn + ((size_t)s * 2 + (t & 1)) * BBLOCK;
  const int k = t >> 1;
  blk[sw_off(2 * f, k)] = (float)(u.x * SQRT2_LEGACY);
  blk[sw_off(2 * f + 1, k)] = (float)(u.y * SQRT2_LEGACY);
}

size_t mx_fold_smem(const ShtDev& d, int nr) { return fft_smem_bytes(nr, d.n2, sizeof(float2)); }
size_t mx_unfold_smem(const ShtDev& d) { return fft_smem_bytes(2, d.n2, sizeof(float2)); }

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

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link-time libcuda).
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

constexpr int ZBOX[3] = {8, 16, 32};

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
  const size_t nx4 = (size_t)MX_MAXF * d.nh * d.nm;   // 16-byte entries of X and of the sums
  SLE_TRY(mx_alloc(&p->mx_xf, 4 * nx4));
  SLE_TRY(mx_alloc(&p->mx_gns, 2 * nx4));
  SLE_TRY(mx_alloc(&p->mx_bsyn, (size_t)d.nseg * 2 * BBLOCK));
  SLE_TRY(mx_alloc(&p->mx_s0, (size_t)MX_MAXF * d.nh));
  SLE_TRY(mx_alloc(&p->mx_abort, 1));
  SLE_CUDA(cudaMemset(p->mx_xf, 0, 4 * nx4 * sizeof(float)));
  SLE_CUDA(cudaMemset(p->mx_gns, 0, 2 * nx4 * sizeof(float2)));
  SLE_CUDA(cudaMemset(p->mx_bsyn, 0, (size_t)d.nseg * 2 * BBLOCK * sizeof(float)));
  SLE_CUDA(cudaMemset(p->mx_abort, 0, sizeof(int)));
  {
    // FP32 twiddle table (same layout), rounded from the plan's FP64 one
    const int ntw = tw_table_len(d.n2);
    std::vector<double2> tw64(ntw);
    std::vector<float2> tw32(ntw);
    SLE_CUDA(cudaMemcpy(tw64.data(), p->tw, ntw * sizeof(double2), cudaMemcpyDeviceToHost));
    for (int t = 0; t < ntw; ++t) tw32[t] = make_float2((float)tw64[t].x, (float)tw64[t].y);
    SLE_TRY(mx_alloc(&p->mx_twf, (size_t)ntw));
    SLE_CUDA(cudaMemcpy(p->mx_twf, tw32.data(), ntw * sizeof(float2), cudaMemcpyHostToDevice));
  }
  // work units; each unit's chunks are contiguous slots of its Legendre table
  std::vector<unsigned char> ist(d.nseg);
  std::vector<int> segoff(d.nm + 1);
  SLE_CUDA(cudaMemcpy(ist.data(), p->istart, d.nseg, cudaMemcpyDeviceToHost));
  SLE_CUDA(cudaMemcpy(segoff.data(), p->segoff, (d.nm + 1) * sizeof(int), cudaMemcpyDeviceToHost));
  const int L = d.lmax;
  // a unit's estimated cost in half-chunk times: its halves plus a fixed per-unit cost (pipeline
  // turn-around and epilogue)
  struct AU { double w; int m, s, kstart; };
  struct SU { double w; int m, t; std::vector<int> segs; };
  std::vector<AU> au;
  std::vector<SU> su;
  for (int m = 0; m <= L; ++m) {
    const int nl = L - m + 1;
    for (int s = 0; s * ANA_SPAN < nl; ++s) {
      const int nd = std::min(ANA_SPAN, nl - ANA_SPAN * s);
      int kstart = d.ngrp;
      for (int q = 0; q * SEG < nd; ++q) kstart = std::min(kstart, (int)ist[segoff[m] + (ANA_SPAN / SEG) * s + q]);
      au.push_back({2.0 * (d.ngrp - kstart) + ANA_UNIT_COST, m, s, kstart});
    }
    const int ntile = (d.nh + 127) / 128;
    for (int t = 0; t < ntile; ++t) {
      SU u{0, m, t, {}};
      const int glast = std::min(d.ngrp, 4 * t + 4) - 1;
      for (int seg = segoff[m]; seg < segoff[m + 1]; ++seg)
        if ((int)ist[seg] <= glast) u.segs.push_back(seg);
      u.w = 2.0 * u.segs.size() + SYN_UNIT_COST;
      su.push_back(u);
    }
  }
  std::stable_sort(au.begin(), au.end(), [](const AU& x, const AU& y) { return x.w > y.w; });
  std::stable_sort(su.begin(), su.end(), [](const SU& x, const SU& y) { return x.w > y.w; });
  {
    int dev = 0, nsm = 0;
    SLE_CUDA(cudaGetDevice(&dev));
    SLE_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    p->n_sm = std::max(1, nsm);
  }
  // CTA b of a launch of G = min(n, SMs) CTAs takes a run of consecutive units: longest first,
  // each unit goes to the CTA with the least estimated work so far (ties: the lowest index);
  // within a CTA the units keep that order
  auto balance = [&](auto& v, std::vector<int2>& cta) {
    const int n = (int)v.size(), G = std::max(1, std::min(n, p->n_sm));
    std::vector<double> load(G, 0.0);
    std::vector<std::vector<int>> of(G);
    for (int i = 0; i < n; ++i) {
      int b = 0;
      for (int c = 1; c < G; ++c)
        if (load[c] < load[b]) b = c;
      load[b] += v[i].w;
      of[b].push_back(i);
    }
    auto out = v;
    cta.assign(G, make_int2(0, 0));
    int pos = 0;
    for (int b = 0; b < G; ++b) {
      cta[b] = make_int2(pos, (int)of[b].size());
      for (int i : of[b]) out[pos++] = v[i];
    }
    v.swap(out);
  };
  std::vector<int2> acta, scta;
  balance(au, acta);
  balance(su, scta);
  std::vector<int4> av, sv;
  std::vector<int> segs;
  long long na = 0, ns = 0;
  for (const AU& u : au) {
    av.push_back(make_int4(u.m, u.s, u.kstart, (int)na));
    na += d.ngrp - u.kstart;
  }
  for (const SU& u : su) {
    sv.push_back(make_int4(u.m, u.t, (int)u.segs.size(), (int)ns));
    for (int sg : u.segs) segs.push_back(sg);
    ns += (long long)u.segs.size();
  }
  {
    // synthesis B position of every packed coefficient (mx_bsyn_put): segment seg of order m
    // holds degrees l0 = m + 64 q .. l0 + 63; degree l sits at t = l - l0 in the block of parity
    // t & 1, K index t / 2
    std::vector<int> bpos((size_t)d.ncoef);
    for (int m = 0; m <= L; ++m) {
      const long long mo = (long long)m * (L + 1) - (long long)m * (m - 1) / 2;
      for (int l = m; l <= L; ++l) {
        const int seg = segoff[m] + (l - m) / SEG, t = (l - m) % SEG;
        bpos[(size_t)(mo + l - m)] = ((seg * 2 + (t & 1)) * BBLOCK) * 32 + (t >> 1);
      }
    }
    SLE_TRY(mx_alloc(&p->mx_bpos, bpos.size()));
    SLE_CUDA(cudaMemcpy(p->mx_bpos, bpos.data(), bpos.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  SLE_TRY(mx_alloc(&p->mx_ana_units, av.size()));
  SLE_TRY(mx_alloc(&p->mx_syn_units, sv.size()));
  SLE_TRY(mx_alloc(&p->mx_ana_cta, acta.size()));
  SLE_TRY(mx_alloc(&p->mx_syn_cta, scta.size()));
  SLE_CUDA(cudaMemcpy(p->mx_ana_cta, acta.data(), acta.size() * sizeof(int2), cudaMemcpyHostToDevice));
  SLE_CUDA(cudaMemcpy(p->mx_syn_cta, scta.data(), scta.size() * sizeof(int2), cudaMemcpyHostToDevice));
  p->n_ana_cta = (int)acta.size();
  p->n_syn_cta = (int)scta.size();
  SLE_TRY(mx_alloc(&p->mx_syn_seg, segs.size() + 1));
  SLE_CUDA(cudaMemcpy(p->mx_ana_units, av.data(), av.size() * sizeof(int4), cudaMemcpyHostToDevice));
  SLE_CUDA(cudaMemcpy(p->mx_syn_units, sv.data(), sv.size() * sizeof(int4), cudaMemcpyHostToDevice));
  if (!segs.empty())
    SLE_CUDA(cudaMemcpy(p->mx_syn_seg, segs.data(), segs.size() * sizeof(int), cudaMemcpyHostToDevice));
  p->n_ana_units = (int)av.size();
  p->n_syn_units = (int)sv.size();
  // Legendre tables: FP64 recurrence rounded to FP32 (the kernel splits them), zero where negligible
  const size_t tab_a = (size_t)na * SLOT_WORDS, tab_s = (size_t)ns * SLOT_WORDS;
  SLE_TRY(mx_alloc(&p->mx_tab_ana, tab_a + 1));
  SLE_TRY(mx_alloc(&p->mx_tab_syn, tab_s + 1));
  SLE_CUDA(cudaMemset(p->mx_tab_ana, 0, tab_a * sizeof(uint32_t)));
  SLE_CUDA(cudaMemset(p->mx_tab_syn, 0, tab_s * sizeof(uint32_t)));
  p->mx_table_bytes = (double)(tab_a + tab_s) * sizeof(uint32_t);
  d.twf = p->mx_twf;
  d.mx_xf = p->mx_xf;
  d.mx_gns = p->mx_gns;
  d.mx_bsyn = p->mx_bsyn;
  d.mx_s0 = p->mx_s0;
  d.mx_abort = p->mx_abort;
  d.mx_ana_units = p->mx_ana_units;
  d.mx_syn_units = p->mx_syn_units;
  d.mx_ana_cta = p->mx_ana_cta;
  d.mx_syn_cta = p->mx_syn_cta;
  d.mx_syn_seg = p->mx_syn_seg;
  d.mx_tab_ana = p->mx_tab_ana;
  d.mx_tab_syn = p->mx_tab_syn;
  k_tab_ana<<<p->n_ana_units, 256>>>(d, p->mx_tab_ana);
  k_tab_syn<<<p->n_syn_units, 128>>>(d, p->mx_tab_syn);
  SLE_CUDA(cudaGetLastError());
  SLE_CUDA(cudaDeviceSynchronize());
  // TMA maps of X[f][m][par][j][2]: dims (2 nh floats, 2 parities, nm orders, MX_MAXF fields),
  // boxes (2 x 32 latitudes, 1, 1, 8 | 16 | 32 fields)
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled is not available from the driver");
    return SLE_ERR_CUDA;
  }
  for (int zi = 0; zi < 3; ++zi) {
    const cuuint64_t dims[4] = {(cuuint64_t)2 * d.nh, 2, (cuuint64_t)d.nm, (cuuint64_t)MX_MAXF};
    const cuuint64_t strides[3] = {(cuuint64_t)8 * d.nh, (cuuint64_t)16 * d.nh, (cuuint64_t)16 * d.nh * d.nm};
    const cuuint32_t box[4] = {2 * KC, 1, 1, (cuuint32_t)ZBOX[zi]};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = enc(reinterpret_cast<CUtensorMap*>(p->mx_tmap[zi]), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                           p->mx_xf, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
      set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
      return SLE_ERR_CUDA;
    }
  }
  SLE_CUDA(cudaFuncSetAttribute(k_leg_tc<false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx_smem(2)));
  SLE_CUDA(cudaFuncSetAttribute(k_leg_tc<true, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx_smem(2, true)));
  SLE_CUDA(cudaFuncSetAttribute(k_leg_tc<false, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx_smem(4)));
  SLE_CUDA(cudaFuncSetAttribute(k_leg_tc<true, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx_smem(4, true)));
#define SLE_ATTR_MX(NN)                                                                                        \
  do {                                                                                                         \
    SLE_CUDA(cudaFuncSetAttribute(k_fold_mx<NN, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mx_fold_smem(d, 4)));    \
    SLE_CUDA(cudaFuncSetAttribute(k_fold_mx<NN, 4>, cudaFuncAttributePreferredSharedMemoryCarveout, 100)); \
    SLE_CUDA(cudaFuncSetAttribute(k_fold_mx<NN, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mx_fold_smem(d, 8)));    \
    SLE_CUDA(cudaFuncSetAttribute(k_fold_mx<NN, 8>, cudaFuncAttributePreferredSharedMemoryCarveout, 100)); \
    SLE_CUDA(cudaFuncSetAttribute(k_unfold_mx<NN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mx_unfold_smem(d)));      \
    SLE_CUDA(cudaFuncSetAttribute(k_unfold_mx<NN>, cudaFuncAttributePreferredSharedMemoryCarveout, 100)); \
    SLE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p->unfold_ahead, k_unfold_mx<NN>,                    \
                                                           fft_threads(2, NN), mx_unfold_smem(d)));              \
  } while (0)
  SLE_FFT_SWITCH(d.n2, SLE_ATTR_MX)
#undef SLE_ATTR_MX
  p->unfold_ahead *= p->n_sm;
  p->mx_ready = 1;
  return SLE_OK;
}

static int mx_check_args(const MxFieldArgs& a, const char* what) {
  if (a.nf < 1 || a.nf > MX_MAXF) {
    set_error("%s: 1..%d fields per mixed-precision launch (got %d)", what, MX_MAXF, a.nf);
    return SLE_ERR_BAD_ARG;
  }
  return SLE_OK;
}

int sht_mx_analysis(sle_sht* p, const MxFieldArgs& a, int* status, cudaStream_t st, int prof_cls) {
  SLE_TRY(sht_mx_prepare(p));
  SLE_TRY(mx_check_args(a, "mixed analysis"));
  const ShtDev& d = p->d;
  ProfToken t0 = prof_begin(PROF_FFT, a.nf, st);
#define SLE_LAUNCH_MXF4(NN) \
  SLE_CUDA(launch_pdl(k_fold_mx<NN, 4>, dim3(d.nh / 2, a.nf), dim3(fft_threads(4, NN)), mx_fold_smem(d, 4), st, d, a))
#define SLE_LAUNCH_MXF8(NN) \
  SLE_CUDA(launch_pdl(k_fold_mx<NN, 8>, dim3(d.nh / 4, a.nf), dim3(fft_threads(8, NN)), mx_fold_smem(d, 8), st, d, a))
  if (p->tune_fold_rows == 4) {
    SLE_FFT_SWITCH(d.n2, SLE_LAUNCH_MXF4)
  } else {
    SLE_FFT_SWITCH(d.n2, SLE_LAUNCH_MXF8)
  }
#undef SLE_LAUNCH_MXF4
#undef SLE_LAUNCH_MXF8
  prof_end(t0, st);
  const int zi = (a.nf <= ZBOX[0]) ? 0 : (a.nf <= ZBOX[1]) ? 1 : 2;
  const CUtensorMap* map = reinterpret_cast<const CUtensorMap*>(p->mx_tmap[zi]);
  ProfToken t1 = prof_begin(prof_cls, a.nf, st);
  if (p->tune_stages == 2)
    k_leg_tc<false, 2><<<p->n_ana_cta, TC_THREADS, mx_smem(2), st>>>(d, a, status, *map, ZBOX[zi]);
  else
    k_leg_tc<false, 4><<<p->n_ana_cta, TC_THREADS, mx_smem(4), st>>>(d, a, status, *map, ZBOX[zi]);
  prof_end(t1, st);
  note_launch(2);
  SLE_CUDA(cudaGetLastError());
  return SLE_OK;
}

int sht_mx_synthesis(sle_sht* p, const MxFieldArgs& a, int* status, cudaStream_t st, bool b_ready) {
  SLE_TRY(sht_mx_prepare(p));
  SLE_TRY(mx_check_args(a, "mixed synthesis"));
  const ShtDev& d = p->d;
  const CUtensorMap* map = reinterpret_cast<const CUtensorMap*>(p->mx_tmap[0]);
  ProfToken t0 = prof_begin(PROF_LEG_SYN, a.nf, st);
  if (!b_ready) k_bsyn_mx<<<dim3(d.nseg, (a.nf + 3) / 4), 256, 0, st>>>(d, a);
  if (p->tune_stages == 2)
    k_leg_tc<true, 2><<<p->n_syn_cta, TC_THREADS, mx_smem(2, true), st>>>(d, a, status, *map, 0);
  else
    k_leg_tc<true, 4><<<p->n_syn_cta, TC_THREADS, mx_smem(4, true), st>>>(d, a, status, *map, 0);
  prof_end(t0, st);
  ProfToken t1 = prof_begin(PROF_IFFT, a.nf, st);
#define SLE_LAUNCH_MXU(NN) \
  SLE_CUDA(launch_pdl(k_unfold_mx<NN>, dim3(d.nh, a.nf), dim3(fft_threads(2, NN)), mx_unfold_smem(d), st, d, a, p->unfold_ahead))
  SLE_FFT_SWITCH(d.n2, SLE_LAUNCH_MXU)
#undef SLE_LAUNCH_MXU
  prof_end(t1, st);
  note_launch(3);
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
