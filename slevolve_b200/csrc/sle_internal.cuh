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
constexpr int MAXF = 4;   // fields per batched transform call

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
  // Optional per-field gates of an analysis launch (device flags read at kernel entry): field f
  // is skipped when bit f of gate_conv_mask is set and *gate_conv != 0, or when bit f of
  // gate_chg_mask is set and *gate_chg == 0.
  const int* gate_conv;
  const int* gate_chg;
  unsigned gate_conv_mask, gate_chg_mask;
};

__device__ __forceinline__ bool field_gated_off(const ShtDev& P, int f) {
  if (((P.gate_conv_mask >> f) & 1u) && *P.gate_conv != 0) return true;
  if (((P.gate_chg_mask >> f) & 1u) && *P.gate_chg == 0) return true;
  return false;
}

struct AnaGate {
  const int* conv;
  const int* chg;
  unsigned conv_mask, chg_mask;
};

// Epilogue of the inverse-FFT kernel: out2 = g * mul2 (e.g. rO = dsl * C*).
struct SynEpilogue {
  double* out2;
  const double* mul2;
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
};

namespace sle {
// Launch accounting / per-kernel event timing (sle_prof.cu).
enum ProfClass { PROF_FFT = 0, PROF_LEG_ANA = 1, PROF_LEG_SYN = 2, PROF_IFFT = 3, PROF_ADVANCE = 4,
                 PROF_NCLS = 5 };
struct ProfToken {
  int cls;
  double units;
  void* a;
};
void note_launch(int n = 1);
bool prof_enabled();
ProfToken prof_begin(int cls, double units, cudaStream_t st);
void prof_end(const ProfToken& t, cudaStream_t st);

// Launch helpers implemented in sle_sht.cu, used by the solver.
int sht_analysis_packed(sle_sht* plan, int nf, const double* const* grids, double2* const* out,
                        cudaStream_t st, const AnaGate* gate = nullptr);
int sht_synthesis_packed(sle_sht* plan, int nf, const double2* const* coeffs, double* const* grids,
                         const SynEpilogue* epi, cudaStream_t st);
int sht_pack(sle_sht* plan, const double2* dense, double2* packed, cudaStream_t st);
int sht_unpack(sle_sht* plan, const double2* packed, double2* dense, cudaStream_t st);
}  // namespace sle
