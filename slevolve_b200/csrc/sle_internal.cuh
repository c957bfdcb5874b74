// Internal definitions shared by the transform and solver translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>

#include "../../include/slevolve_b200.h"

namespace sle {

void set_error(const char* fmt, ...);

#define SLE_CUDA(call)                                                                    \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) {                                                              \
      sle::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,   \
                     __LINE__);                                                           \
      return SLE_ERR_CUDA;                                                                \
    }                                                                                     \
  } while (0)

#define SLE_TRY(expr)          \
  do {                         \
    int rc_ = (expr);          \
    if (rc_ != SLE_OK) return rc_; \
  } while (0)

// Degrees per Legendre segment: the recurrence restarts from stored seeds at every
// segment start, which bounds the growth of the segment scale factor to ~2^SEG and
// gives the kernels independent work units.
constexpr int SEG = 64;
// |P~_lm(mu_j)| below this in a whole (segment, 32-latitude group) is treated as zero.
// Contributions skipped are < nh * 1e-35 * max|field| (~1e-29 m for Earth-sized fields).
constexpr double SIG_THRESHOLD = 1.0e-35;
// The legacy literal of spat2spec / spec2spat (SLEvolve sht.py:60-61), not sqrt(2).
constexpr double SQRT2_LEGACY = 1.41421356;
constexpr int MAXF = 4;   // fields per batched transform launch (FP64 path); per call with the dense layout
constexpr int MAX_CALL_FIELDS = 256;   // fields per transform call with the packed layout
constexpr int MX_MAXF = 32;          // fields per mixed-precision transform launch
constexpr int MX_NMAX = 2 * MX_MAXF; // B-operand rows (Re, Im per field)

// Synthesis B operand entry of one packed coefficient for field slot f of a mixed-precision
// launch: 1.41421356 U rounded to FP32 in rows 2f (Re) and 2f + 1 (Im) of its (segment, parity)
// block, at K index k, in the tensor cores' 128-byte-swizzled tile order of 32 entries per row.
// bpos = (block's first entry) * 32 + k, from the plan's mx_bpos table.
__device__ __forceinline__ void mx_bsyn_put(float* bsyn, int bpos, int f, double2 u) {
  float* blk = bsyn + (bpos >> 5);
  const int k = bpos & 31, r0 = 2 * f, r1 = 2 * f + 1;
  blk[r0 * 32 + ((((k >> 2) ^ (r0 & 7)) << 2) | (k & 3))] = (float)(u.x * SQRT2_LEGACY);
  blk[r1 * 32 + ((((k >> 2) ^ (r1 & 7)) << 2) | (k & 3))] = (float)(u.y * SQRT2_LEGACY);
}

// Prefetch of `bytes` of global memory into L2 (a hint; nothing waits for it).  The bulk prefetch
// wants a 16-byte aligned start and a multiple of 16 bytes; anything else is left out.
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
  if (((reinterpret_cast<uintptr_t>(p) | bytes) & 15u) != 0 || bytes == 0) return;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// The block `ahead` places on from this one in launch order (x fastest), whose inputs this one
// prefetches into L2: false past the grid's end.
__device__ __forceinline__ bool block_ahead(int ahead, int& bx, int& by) {
  const long long lin = (long long)blockIdx.y * gridDim.x + blockIdx.x + ahead;
  if (ahead <= 0 || lin >= (long long)gridDim.x * gridDim.y) return false;
  by = (int)(lin / gridDim.x);
  bx = (int)(lin - (long long)by * gridDim.x);
  return true;
}

// Programmatic dependent launch.  A kernel launched by launch_pdl may be scheduled while the
// kernel before it in the stream is finishing; it calls pdl_wait() before its first access to
// global memory, which returns once that kernel has completed and its writes are visible (at once
// for a plain launch).  Every kernel launched this way waits unconditionally, so the ordering
// stays transitive along the stream.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// Lets the next kernel of the stream, if launched by launch_pdl, be scheduled once every block of
// this one has passed here (its blocks then wait in pdl_wait for this kernel to complete).
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Programmatic launches are on unless SLEVOLVE_B200_NO_PDL is set (to a non-empty value other
// than "0") when the library first launches one, or sle_set_programmatic_launch turned them off.
bool pdl_enabled();

template <typename... P, typename... A>
inline cudaError_t launch_pdl(void (*k)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A&&... args) {
  cudaLaunchConfig_t c = {};
  c.gridDim = grid;
  c.blockDim = block;
  c.dynamicSmemBytes = smem;
  c.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  c.attrs = at;
  c.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&c, k, static_cast<A&&>(args)...);
}


// Device view of a transform plan, passed to kernels by value.
struct ShtDev {
  int nlat, nlon, lmax, nh, nm, n2, log2n2, ngrp, nseg;
  long long ncoef;
  const double* mu;           // [nlat] Gauss nodes, north -> south
  const double* w;            // [nlat] Gauss weights
  const double* wn;           // [nh] w / nlon, northern rows
  const double* ws;           // [nh] w / nlon, southern rows (row nlat-1-j)
  const long long* moff;      // [nm+1] packed offset of order m
  const int* lidx;            // [ncoef] degree of each packed index
  const int* segoff;          // [nm+1] first segment of order m
  const int* seg_m;           // [nseg] order of segment
  const int* seg_l0;          // [nseg] first degree of segment
  const double2* seeds;       // [nseg][nh] (Q_l0, Q_l0+1) in segment scale
  const double* be;           // [ncoef] Q_l = mu Q_{l-1} + be_l Q_{l-2}
  const double* cf;           // [ncoef] P~_l = cf_l Q_l (segment scale)
  const unsigned char* istart;// [nseg] first significant latitude group of the segment
  const int* ana_order;       // [nseg] segment processing order for the analysis (long first)
  const double2* tw;          // [n2] exp(-2 pi i t / nlon)
  double2* X;                 // [MAXF][2][nm][nh] folded rFFT (S then D) of analysed grids
  double2* EO;                // [MAXF][2][nm][nh] even/odd Legendre sums of synthesised fields
  // Per-field gates of a launch (device flags read at kernel entry): field f is skipped (its
  // outputs left as they are) when gset[f] && *gset[f] != 0, or gclr[f] && *gclr[f] == 0.
  const int* gset[MAXF];
  const int* gclr[MAXF];
  // mixed-precision transforms (set once the plan prepared them)
  const float2* twf;          // [n2] FP32 twiddles of the mixed-precision row FFTs
  float* mx_xf;               // [MX_MAXF][nm][2][nh][2] folded FP32 rFFT: S, D (complex) per order
  float2* mx_gns;             // [MX_MAXF][nh][nm][2] even / odd-degree Legendre sums (synthesis)
  float* mx_bsyn;             // [nseg][2][MX_NMAX][32] synthesis B operand (FP32, tile order)
  double* mx_s0;              // [MX_MAXF][nh] FP64 fold of the row sums (degree 0)
  int* mx_abort;              // raised by a tensor-core kernel whose wait timed out
  const int4* mx_ana_units;   // (m, span, first chunk, table slot) analysis units, in runs per CTA
  const int4* mx_syn_units;   // (m, latitude tile, chunks, table slot) synthesis units
  const int2* mx_ana_cta;     // (first unit, units) of each CTA of an analysis launch
  const int2* mx_syn_cta;     // the same for a synthesis launch
  const int* mx_syn_seg;      // segment of each synthesis table slot
  const uint32_t* mx_tab_ana; // Legendre tables: [slot][par][128][32] FP32, 128-byte-swizzled tile order
  const uint32_t* mx_tab_syn;
};

__device__ __forceinline__ bool field_gated_off(const ShtDev& P, int f) {
  if (P.gset[f] && *P.gset[f] != 0) return true;
  if (P.gclr[f] && *P.gclr[f] == 0) return true;
  return false;
}

// What an analysis reads for a field (cell c): SRC_GRID grid[c]; SRC_MASK the 0/1 byte m0[c];
// SRC_ICE m0[c] ? grid[c] : grid[c] * 0 (ice on its grounded mask); SRC_TO
// grid[c] * (m0[c] - m1[c]) (T0 (C* - C*0)); SRC_PROD grid[c] * m0[c] (dsl C*).  The products are
// the ones the step would otherwise write out as FP64 grids, in the same arithmetic.
enum SrcKind { SRC_GRID = 0, SRC_MASK = 1, SRC_ICE = 2, SRC_TO = 3, SRC_PROD = 4 };

// One field of a transform call: input and output, optional gates (see ShtDev::gset/gclr), the
// analysis source kind and, for synthesis, the optional epilogue epi_out = grid * epi_mul.
struct FieldSpec {
  double* grid;
  double2* spec;
  const int* skip_set;
  const int* skip_clear;
  double* epi_out;
  const double* epi_mul;
  int kind;
  const unsigned char* m0;
  const unsigned char* m1;
};

// Two neighbouring cells c, c + 1 (c even) of an analysis source of kind KIND.
template <int KIND>
__device__ __forceinline__ double2 src_pair(const double* g, const unsigned char* m0, const unsigned char* m1,
                                            size_t c) {
  if constexpr (KIND == SRC_GRID) {
    return __ldg(reinterpret_cast<const double2*>(g + c));
  } else if constexpr (KIND == SRC_MASK) {
    const uchar2 a = *reinterpret_cast<const uchar2*>(m0 + c);
    return make_double2(a.x ? 1.0 : 0.0, a.y ? 1.0 : 0.0);
  } else {
    const uchar2 a = *reinterpret_cast<const uchar2*>(m0 + c);
    const double2 v = __ldg(reinterpret_cast<const double2*>(g + c));
    if constexpr (KIND == SRC_ICE) {
      return make_double2(a.x ? v.x : __dmul_rn(v.x, 0.0), a.y ? v.y : __dmul_rn(v.y, 0.0));
    } else if constexpr (KIND == SRC_TO) {
      const uchar2 z = *reinterpret_cast<const uchar2*>(m1 + c);
      return make_double2(__dmul_rn(v.x, __dsub_rn(a.x ? 1.0 : 0.0, z.x ? 1.0 : 0.0)),
                          __dmul_rn(v.y, __dsub_rn(a.y ? 1.0 : 0.0, z.y ? 1.0 : 0.0)));
    } else {
      return make_double2(__dmul_rn(v.x, a.x ? 1.0 : 0.0), __dmul_rn(v.y, a.y ? 1.0 : 0.0));
    }
  }
}

// Calls body.template operator()<KIND>() for the run-time source kind (one branch per block, so
// each kind's loads stay straight-line code).
template <typename Body>
__device__ __forceinline__ void with_src_kind(int kind, const Body& body) {
  switch (kind) {
    case SRC_MASK: body.template operator()<SRC_MASK>(); break;
    case SRC_ICE: body.template operator()<SRC_ICE>(); break;
    case SRC_TO: body.template operator()<SRC_TO>(); break;
    case SRC_PROD: body.template operator()<SRC_PROD>(); break;
    default: body.template operator()<SRC_GRID>(); break;
  }
}

// Fields of one mixed-precision transform launch.  Field f is skipped (its outputs left as
// they are) when *skip_set[f] != 0 or *skip_clear[f] == 0 (null pointers never skip).
// Synthesis epilogue: epi_out[f] = grid[f] * epi_mul[f] when epi_out[f] is set.
struct MxFieldArgs {
  int nf;
  double* grid[MX_MAXF];           // analysis input / synthesis output
  double2* spec[MX_MAXF];          // analysis output / synthesis input (packed)
  const int* skip_set[MX_MAXF];
  const int* skip_clear[MX_MAXF];
  double* epi_out[MX_MAXF];
  const double* epi_mul[MX_MAXF];
  int kind[MX_MAXF];               // analysis source (SrcKind)
  const unsigned char* m0[MX_MAXF];
  const unsigned char* m1[MX_MAXF];
};

}  // namespace sle

struct sle_sht {
  sle::ShtDev d;
  // owned allocations
  double *mu, *w, *wn, *ws, *be, *cf;
  long long* moff;
  int *lidx, *segoff, *seg_m, *seg_l0, *ana_order;
  double2 *seeds, *tw, *X, *EO;
  unsigned char* istart;
  double2* packbuf;           // [MAXF][ncoef] packed staging for dense-layout calls
  double* skipped_frac;       // host value: fraction of (l, m, j) work skipped
  double work_frac;
  int precision;              // SLE_PREC_FP64 or SLE_PREC_MIXED
  int* mx_status;             // device status word raised on a tensor-core timeout (may be null)
  // mixed-precision transform buffers (allocated on first use)
  int mx_ready;
  float* mx_xf;
  float2* mx_twf;
  float2* mx_gns;
  float* mx_bsyn;
  int* mx_bpos;                  // [ncoef] synthesis B position of each packed coefficient (mx_bsyn_put)
  double* mx_s0;
  int* mx_abort;
  int4 *mx_ana_units, *mx_syn_units;
  int2 *mx_ana_cta, *mx_syn_cta;
  int* mx_syn_seg;
  uint32_t *mx_tab_ana, *mx_tab_syn;
  alignas(64) unsigned char mx_tmap[3][128];   // TMA maps of mx_xf (boxes of 8, 16, 32 fields)
  double mx_table_bytes;
  int n_ana_units, n_syn_units;
  int n_ana_cta, n_syn_cta;       // CTAs of an analysis / synthesis launch
  int n_sm;                      // SMs of the device (persistent transform grid)
  // blocks of the unfold resident on the device at once (occupancy x SMs): each block prefetches
  // into L2 the input of the block that many places further on in launch order
  int unfold_ahead;
  // launch shape of the mixed-precision transforms (sle_sht_set_tuning): fields per tensor-core
  // launch, pipeline stages of the tensor-core kernel, rows per row-FFT block of the fold
  int tune_fpl, tune_stages, tune_fold_rows;
};

namespace sle {
// Launch accounting / per-kernel event timing (sle_prof.cu).
// PROF_ANA_STEP: the Legendre analysis of the inner iteration's rO (every stepping field active).
// Classes 6-10: the inner loop's elementwise passes (units = slots not yet converged).
enum ProfClass { PROF_FFT = 0, PROF_LEG_ANA = 1, PROF_LEG_SYN = 2, PROF_IFFT = 3, PROF_ADVANCE = 4,
                 PROF_ANA_STEP = 5, PROF_B18 = 6, PROF_UPDATE = 7, PROF_REFRESH1 = 8, PROF_REFRESH2 = 9,
                 PROF_DICE = 10, PROF_NCLS = 11 };
struct ProfToken {
  int cls;
  double units;
  void* a;
};
void note_launch(int n = 1);
bool prof_enabled();
ProfToken prof_begin(int cls, double units, cudaStream_t st);
void prof_end(const ProfToken& t, cudaStream_t st);

// Transforms of a list of fields (packed spectra), launched in groups of MAXF (FP64) or
// MX_MAXF (mixed) fields with the precision of the plan (sle_sht.cu).
int sht_analysis_list(sle_sht* plan, const FieldSpec* f, int n, cudaStream_t st, int prof_cls = PROF_LEG_ANA);
// b_ready (mixed precision, n <= the plan's fields per launch): field f's B operand was written by
// mx_bsyn_put with slot f, so the launch skips forming it
int sht_synthesis_list(sle_sht* plan, const FieldSpec* f, int n, cudaStream_t st, bool b_ready = false);
int sht_pack(sle_sht* plan, const double2* dense, double2* packed, cudaStream_t st);
// Mixed-precision transforms (sle_mx.cu).  `status` (device int, may be null) receives
// SLE_ERR_TIMEOUT if a tensor-core kernel gave up waiting.
int sht_mx_prepare(sle_sht* plan);
int sht_mx_analysis(sle_sht* plan, const MxFieldArgs& a, int* status, cudaStream_t st,
                    int prof_cls = PROF_LEG_ANA);
// b_ready: the synthesis B operand of the launch's fields is already in place (mx_bsyn_put)
int sht_mx_synthesis(sle_sht* plan, const MxFieldArgs& a, int* status, cudaStream_t st, bool b_ready = false);
int sht_mx_abort_flag(sle_sht* plan, int* flag);
int sht_unpack(sle_sht* plan, const double2* packed, double2* dense, cudaStream_t st);
}  // namespace sle
