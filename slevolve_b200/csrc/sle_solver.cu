// The SLEvolve time step on the device (SLEvolve python/slevolve/solver.py:521-1144) for a batch
// of independent solves ("slots") on one grid size, FP64 or mixed-precision transforms.
//
// Every slot has its own Earth model, step length, topography, ice history, modal state and
// convergence; the kernels cover all slots of the batch in one launch (blockIdx.y = slot), so a
// step of B solves costs the launches of one.  All state lives in HBM for the life of the
// handle, laid out buffer-major: grid buffer g of slot b at grid + (g * nslot + b) * ng, spectra
// in the packed order-major triangle (complex128) likewise, the modal state R[slot][k][packed].
// Elementwise kernels reproduce the reference's NumPy statement order with explicitly rounded
// operations (no FMA contraction); reductions are deterministic (fixed partition, last-block
// finalisation in index order), so a slot's results do not depend on the other slots.
//
// The inner fixed-point loop is a CUDA graph with a device-evaluated WHILE condition: it runs
// while any stepping slot is unconverged; a slot that converged is marked done at the end of
// that iteration and every kernel of later iterations skips it.
//
// The single-solve C API (sle_solver_*) is a batch of one slot.
#include "sle_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <utility>
#include <vector>

namespace sle {

constexpr double EPS0 = 2.220446049250313e-16;   // numpy finfo(float64).eps (solver.py:33)
constexpr double PI_LEGACY = 3.1415926535898;    // truncated literal (solver.py:31)
constexpr int GR_MAXACC = 3;                      // solver.py:38
constexpr int MAX_INNER = 9999;                   // solver.py:1049

// Constants of the rotation block (solver.py:910-975), computed on the host with the
// reference's expressions, one record per slot (they depend on the slot's Earth model).
struct RotConst {
  double c_il22, c_il02, c_il12;   // -8 PI a^4/(3 sqrt5), -8 PI a^4/sqrt30, 8 PI a^4/sqrt30
  double alpha;                    // 1 / (1 - kTE2/kf)
  double inv_CmA, inv_kf, inv_C;   // 1/(C-A), 1/kf, 1.0/C
  double kf;                       // the ramp's implicit m divides by kf itself
  double onepk;                    // 1 + kE2
  double r2w2_3, r2w2_6s5, r2w2_s30, r2w2_s120;
  double ekhTE, hTE2, gacc;
  double rhoi, rhow;
};

// Per-slot step record, mirrored to pinned host memory.
struct Scal {
  double conserv, sa, so, xi;
  double K00;
  int numiter, converged, status, gr_nacc, gr_changed, gr_reguess, gr_ice_an, done;
  unsigned int nd;
  int cs_changed;        // C* (hence tO) changed in this iteration's refresh
  double diag[5];        // slc_ocn00, c00, slc_b00, cst00 (real parts), ice00
  // rotation
  double il[9], mm[3], lam[18];
  double oldil[9], oldm[3], dlam_prev2[6];
  double sum_il[9], sum_m[3], sum_tsl[6], sum_trr[6];
  double dsl_rot[6], rr_rot[6];
  double dil[9], dm[3], dlam_cur2[6];
  double p_il[9], p_m[3], p_lambda[6];
};

// Per-slot parameters of one step, uploaded before the step's kernels.
struct SlotStep {
  int active;   // the slot steps in this call
  int first;    // its first step (old-ice analysis on T0, solver.py:868-873)
  int mode;     // first guess: 0 eustatic, 1 extrap uniform, 2 extrap variable
  int hsel;     // which extrap history buffer holds the most recent load increment
  double c1, c2;
  // cross-pass warm start (solver_opt.py:400-403, 514-528, 932-947): this step's entry of the
  // slot's reuse store, read before the step (null = no entry yet) and written at its end
  const double2* warm_ds;          // converged load increment of this step, previous pass
  const unsigned char* warm_mask;  // converged ocean function of this step, previous pass
  double2* rec_ds;                 // where this pass's converged increment goes
  unsigned char* rec_mask;         // where this pass's converged ocean function goes
  int rates;                       // read the analytic rate spectra before the commit
  double rate_h;                   // the step's length (years)
  int horiz;                       // read the horizontal-displacement potential before the commit
  // second-order load placement (ramp, solver.py:348-368): the slot's table for this step length,
  // [omphi (K nl), ttl c_sl (nl), ttl c_rr (nl)], and the degree-2 weights c_il, c_m, c_tsl, c_trr
  int ramp;
  const double* ramp_tab;
  double c_il, c_m, c_tsl, c_trr;
};

enum GridId {
  G_TINIT, G_TOPO_PREV, G_DSL, G_DELTASL, G_TOPO, G_RR, G_ICE, G_ICE_PREV, G_TMP, G_TMP3, G_TMP4, NGRID
};
// 0/1 grids as bytes: ocean function (step 0 and current), beta = grounded-ice complement
// (step 0 and current), C* (step 0 and current), the grounded ("keep") mask of the current I*
// (I* = keep ? ice : ice * 0) and the candidate keep mask of a grounded re-guess.  The FP64
// fields derived from them (C*, I*, tO = T0 (C* - C*0), rO = dsl C*) are formed by the transforms
// as they read them (SrcKind) instead of being written out.
enum MaskId { M_CXY0, M_BETA0, M_CSTAR0, M_CXY, M_GR, M_BETA, M_CSTAR, M_GRNEW, NMASK };
enum SpecId {
  S_P_LOAD, S_P_ICE, S_P_OCEAN, S_PREV_ICE, S_VISC, S_RAD, S_ICELM, S_OLDICE, S_DICE, S_DI, S_CSTARLM,
  S_TOLM, S_ROLM, S_LOAD, S_DSCUR, S_SL, S_SLTOT, S_RRLM, S_HA, S_HB, S_SP0, S_SP1, S_SP2, S_SP3, NSPEC
};

struct Dev {
  int nlat, nlon, nl, nslot, K;
  long long ng, ncoef;
  const int* lidx;
  double* grid;                 // [NGRID][nslot][ng]
  unsigned char* mask;          // [NMASK][nslot][ng]
  double2* spec;                // [NSPEC][nslot][ncoef]
  double2* R;                   // [nslot][K][ncoef]
  const int* nmod;              // [nslot][nl]
  const double *s_kl, *decay, *omd, *a_sl, *a_rr;   // [nslot][K][nl]
  const double *ttl, *ttlekhl, *ttlhe;             // [nslot][nl]
  const double *a_il, *a_m, *a_tsl, *a_trr;        // [nslot][K]
  const RotConst* rc;           // [nslot]
  double *r_il, *r_m, *r_lam;   // [nslot][K][9 | 3 | 6]
  Scal* sc;                     // [nslot]
  const SlotStep* ss;           // [nslot]
  double* partials;             // [nslot][npart]
  long long npart, part_grid;
  unsigned int* counter;        // [nslot][4]
  double* rows;                 // [nslot][4][nlat]
  const double* w;              // Gauss weights
  double rhoi, rhow, epsilon1;
  int checkmarine, tpw, calcRG, opt_dsl;
  // blocks resident at once of the modal advance and of the load update (each block prefetches
  // into L2 the inputs of the block that many places on)
  int adv_ahead, upd_ahead;
  long long i20, i21, i22;      // packed indices of (l=2, m=0..2)
  int slot0;                    // slot of blockIdx.y == 0
  __host__ __device__ double* g(int id, int b) const { return grid + ((size_t)id * nslot + b) * ng; }
  __host__ __device__ unsigned char* m(int id, int b) const { return mask + ((size_t)id * nslot + b) * ng; }
  __host__ __device__ double2* sp(int id, int b) const { return spec + ((size_t)id * nslot + b) * ncoef; }
  __host__ __device__ size_t kl(int b) const { return (size_t)b * K * nl; }
};

// ------------------------------------------------------------------ reduction helpers
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block sum (fixed order).  Every thread of the block must call it.
__device__ double block_sum(double v, double* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double t = 0.0;
  if (w == 0) {
    t = (lane < nw) ? sh[lane] : 0.0;
    t = warp_sum(t);
  }
  return t;  // valid in warp 0
}

// After each block of the slot stored its partial, the last block to arrive sums the partials in
// index order and returns true (in all its threads) with *total set; others return false.  Only
// thread 0's writes (the partial) are fenced before the block's ticket: a thread whose other
// global writes the last block reads must __threadfence() them itself before calling.
__device__ bool last_block_total(double part, double* partials, unsigned int* counter, double* total,
                                 double* sh) {
  __shared__ bool is_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = part;
    __threadfence();
    const unsigned int t = atomicAdd(counter, 1u);
    is_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
  double v = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) v += ((volatile double*)partials)[i];
  v = block_sum(v, sh);
  if (threadIdx.x == 0) {
    *total = v;
    *counter = 0u;
  }
  __syncthreads();
  return true;
}

// true in all threads of the slot's last block to finish (after every block passed this point)
// The last block of the slot to arrive returns true (fencing as last_block_total).
__device__ bool last_block(unsigned int* counter) {
  __shared__ bool is_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int t = atomicAdd(counter, 1u);
    is_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
  if (threadIdx.x == 0) *counter = 0u;
  return true;
}

__device__ __forceinline__ double cabs_(double2 z) { return hypot(z.x, z.y); }

// numpy complex division a / b (Smith's method with a reciprocal scale, loops.c.src)
__device__ __forceinline__ double2 np_cdiv(double2 a, double2 b) {
  if (fabs(b.x) >= fabs(b.y)) {
    const double rat = __ddiv_rn(b.y, b.x);
    const double scl = __ddiv_rn(1.0, __dadd_rn(b.x, __dmul_rn(b.y, rat)));
    return make_double2(__dmul_rn(__dadd_rn(a.x, __dmul_rn(a.y, rat)), scl),
                        __dmul_rn(__dsub_rn(a.y, __dmul_rn(a.x, rat)), scl));
  }
  const double rat = __ddiv_rn(b.x, b.y);
  const double scl = __ddiv_rn(1.0, __dadd_rn(b.y, __dmul_rn(b.x, rat)));
  return make_double2(__dmul_rn(__dadd_rn(__dmul_rn(a.x, rat), a.y), scl),
                      __dmul_rn(__dsub_rn(__dmul_rn(a.y, rat), a.x), scl));
}

__device__ __forceinline__ double2 np_cmul(double2 a, double2 b) {
  return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                      __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}

__device__ __forceinline__ double2 ld2(const double* p, long long i) {
  return reinterpret_cast<const double2*>(p)[i];
}
__device__ __forceinline__ void st2(double* p, long long i, double a, double b) {
  reinterpret_cast<double2*>(p)[i] = make_double2(a, b);
}
// mask cells 2i, 2i + 1
__device__ __forceinline__ uchar2 ldm2(const unsigned char* p, long long i) {
  return reinterpret_cast<const uchar2*>(p)[i];
}
__device__ __forceinline__ void stm2(unsigned char* p, long long i, bool a, bool b) {
  reinterpret_cast<uchar2*>(p)[i] = make_uchar2(a ? 1 : 0, b ? 1 : 0);
}

// grounded ice on topography `topo` (flotation test, solver.py:655-659)
__device__ __forceinline__ bool icestar_keep(double ice, double topo, double rhow, double rhoi) {
  return (topo > 0.0) || (ice > __ddiv_rn(__dmul_rn(fabs(topo), rhow), rhoi));
}
__device__ __forceinline__ double icestar_on(double ice, double topo, double rhow, double rhoi) {
  return icestar_keep(ice, topo, rhow, rhoi) ? ice : __dmul_rn(ice, 0.0);
}

// ------------------------------------------------------------------------- kernels
// Grid kernels process two neighbouring cells per thread (16-byte loads; nlon is even),
// spectral kernels one coefficient per thread; blockIdx.y selects the slot.  Every kernel of a
// step returns at once for a slot marked done (not stepping, or converged earlier).

#define SLOT_OR_RETURN()                        \
  const int b = D.slot0 + (int)blockIdx.y;      \
  Scal* sc = D.sc + b;                          \
  if (sc->done) return;

__global__ void k_set_decay(Dev D, int b, double dt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= D.K * D.nl) return;
  const int k = i / D.nl, l = i - k * D.nl;
  const size_t o = D.kl(b);
  double d = 0.0;
  if (l >= 1 && k < D.nmod[(size_t)b * D.nl + l]) d = exp(__ddiv_rn(__dmul_rn(-D.s_kl[o + i], dt), 1000.0));
  const_cast<double*>(D.decay)[o + i] = d;
  const_cast<double*>(D.omd)[o + i] = __dsub_rn(1.0, d);
}

// Step prologue of every slot: stepping slots get their per-step counters reset; the others are
// marked done (and converged) so that every kernel of the step skips them.
__global__ void k_step_begin(Dev D) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= D.nslot) return;
  Scal* sc = D.sc + b;
  if (D.ss[b].active) {
    sc->numiter = 0;
    sc->converged = 0;
    sc->status = 0;
    sc->gr_nacc = 0;
    sc->gr_changed = 0;
    sc->gr_reguess = 0;
    sc->gr_ice_an = 0;
    sc->done = 0;
  } else {
    sc->done = 1;
    sc->converged = 1;
  }
}

// Degree-2 rotational states and their sums (solver.py:409-421): one thread per component
// (9 il, 3 m, 6 lambda re/im), modes summed in ascending order; then the snapshot of the
// committed rotational loads (oldil, oldm, dlambda_prev2; solver.py:837-839).
__device__ void rot_advance_block(const Dev& D, int b, Scal* sc) {
  __shared__ double sd[64], sa[4][64], sp[18];
  const int q = threadIdx.x;
  const int nmod2 = (D.nl > 2) ? D.nmod[(size_t)b * D.nl + 2] : 0;
  const int n2 = (D.nl > 2) ? min(nmod2, 64) : 0;
  const size_t o = D.kl(b);
  const double* al = D.a_il + (size_t)b * D.K;
  const double* am = D.a_m + (size_t)b * D.K;
  const double* at = D.a_tsl + (size_t)b * D.K;
  const double* ar = D.a_trr + (size_t)b * D.K;
  for (int k = q; k < n2; k += blockDim.x) {
    sd[k] = D.decay[o + (size_t)k * D.nl + 2];
    sa[0][k] = al[k];
    sa[1][k] = am[k];
    sa[2][k] = at[k];
    sa[3][k] = ar[k];
  }
  if (q < 9) sp[q] = sc->p_il[q];
  else if (q < 12) sp[q] = sc->p_m[q - 9];
  else if (q < 18) sp[q] = sc->p_lambda[q - 12];
  __syncthreads();
  double* r_il = D.r_il + (size_t)b * D.K * 9;
  double* r_m = D.r_m + (size_t)b * D.K * 3;
  double* r_lam = D.r_lam + (size_t)b * D.K * 6;
  if (q < 18) {
    double* r = (q < 9) ? r_il + q : (q < 12) ? r_m + (q - 9) : r_lam + (q - 12);
    const int stride = (q < 9) ? 9 : (q < 12) ? 3 : 6;
    const double p = sp[q];
    double acc = 0.0, acc2 = 0.0;
    for (int k = 0; k < n2; ++k) {
      const double d = sd[k];
      const double om = __dsub_rn(1.0, d);
      const double x = __dadd_rn(__dmul_rn(d, r[k * stride]), __dmul_rn(om, p));
      r[k * stride] = x;
      if (q < 9) {
        acc = __dadd_rn(acc, __dmul_rn(sa[0][k], x));
      } else if (q < 12) {
        acc = __dadd_rn(acc, __dmul_rn(sa[1][k], x));
      } else {
        acc = __dadd_rn(acc, __dmul_rn(sa[2][k], x));
        acc2 = __dadd_rn(acc2, __dmul_rn(sa[3][k], x));
      }
    }
    if (q < 9) sc->sum_il[q] = acc;
    else if (q < 12) sc->sum_m[q - 9] = acc;
    else {
      sc->sum_tsl[q - 12] = acc;
      sc->sum_trr[q - 12] = acc2;
    }
  }
  if (q == 0) {
    for (int i = 0; i < 9; ++i) sc->oldil[i] = sp[i];
    for (int i = 0; i < 3; ++i) sc->oldm[i] = sp[9 + i];
    for (int i = 0; i < 6; ++i) sc->dlam_prev2[i] = sp[12 + i];
    for (int i = 0; i < 6; ++i) sc->dsl_rot[i] = sc->rr_rot[i] = sc->dlam_cur2[i] = 0.0;
    for (int i = 0; i < 9; ++i) sc->dil[i] = 0.0;
    for (int i = 0; i < 3; ++i) sc->dm[i] = 0.0;
  }
}

// R_k <- d R_k + (1-d) P ; visc = sum_k a_sl R_k ; rad = sum_k a_rr R_k   (solver.py:386-407)
// The first block of each slot advances the degree-2 rotational state instead.  Each block first
// prefetches into L2 the state rows and the load of the block one resident wave further on in
// launch order, so that the DRAM keeps reading while the blocks before it compute and store.
__global__ void __launch_bounds__(256) k_advance(Dev D) {
  int bx, by;
  if (threadIdx.x <= D.K && block_ahead(D.adv_ahead, bx, by) && bx > 0 && !D.sc[D.slot0 + by].done) {
    const int b2 = D.slot0 + by;
    const long long i0 = (long long)(bx - 1) * blockDim.x;
    const uint32_t bytes = (uint32_t)min((long long)blockDim.x, D.ncoef - i0) * (uint32_t)sizeof(double2);
    prefetch_l2((int)threadIdx.x < D.K ? D.R + ((size_t)b2 * D.K + threadIdx.x) * D.ncoef + i0
                                       : D.sp(S_P_LOAD, b2) + i0,
                bytes);
  }
  SLOT_OR_RETURN();
  if (blockIdx.x == 0) {   // scheduled first: its serial work overlaps the grid
    rot_advance_block(D, b, sc);
    return;
  }
  const long long i = (long long)(blockIdx.x - 1) * blockDim.x + threadIdx.x;
  if (i >= D.ncoef) return;
  double2* R = D.R + (size_t)b * D.K * D.ncoef;
  const int l = D.lidx[i];
  const double2 p = D.sp(S_P_LOAD, b)[i];
  const size_t o = D.kl(b);
  double2 v = make_double2(0.0, 0.0), r = v;
  const int nk = D.nmod[(size_t)b * D.nl + l];
  // modes in groups of 8: the group's state loads before its stores; the coefficient tables are
  // read-only (__ldg), so their loads are free to move
  constexpr int U = 8;
  for (int k0 = 0; k0 < nk; k0 += U) {
    double2 x[U];
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (k0 + u < nk) x[u] = R[(size_t)(k0 + u) * D.ncoef + i];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = k0 + u;
      if (k < nk) {
        const size_t kl = o + (size_t)k * D.nl + l;
        const double d = __ldg(D.decay + kl), om = __ldg(D.omd + kl), as = __ldg(D.a_sl + kl),
                     ar = __ldg(D.a_rr + kl);
        double2 y;
        y.x = __dadd_rn(__dmul_rn(x[u].x, d), __dmul_rn(p.x, om));
        y.y = __dadd_rn(__dmul_rn(x[u].y, d), __dmul_rn(p.y, om));
        R[(size_t)k * D.ncoef + i] = y;
        v.x = __dadd_rn(v.x, __dmul_rn(y.x, as));
        v.y = __dadd_rn(v.y, __dmul_rn(y.y, as));
        r.x = __dadd_rn(r.x, __dmul_rn(y.x, ar));
        r.y = __dadd_rn(r.y, __dmul_rn(y.y, ar));
      }
    }
  }
  D.sp(S_VISC, b)[i] = v;
  D.sp(S_RAD, b)[i] = r;
}

// Step prologue on the grid (solver.py:853-887): I* on the previous topography (its keep mask),
// beta, C* = C beta (tO = T0 (C* - C*0) is formed by its analysis); at the slot's first step also
// I* of the previous ice on T0.
__global__ void k_ice_grid(Dev D) {
  SLOT_OR_RETURN();
  const long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (2 * h >= D.ng) return;
  const double2 v = ld2(D.g(G_ICE, b), h), tp = ld2(D.g(G_TOPO_PREV, b), h);
  uchar2 cx = ldm2(D.m(M_CXY, b), h);
  const unsigned char* wm = D.ss[b].warm_mask;
  if (wm) {  // warm start: the converged ocean function of this step in the previous pass
    cx = make_uchar2(wm[2 * h] ? 1 : 0, wm[2 * h + 1] ? 1 : 0);
    stm2(D.m(M_CXY, b), h, cx.x, cx.y);
  }
  if (!isfinite(v.x) || !isfinite(v.y)) sc->status = SLE_ERR_NONFINITE;
  bool keep[2], bt[2];
  const double vv[2] = {v.x, v.y}, tt[2] = {tp.x, tp.y};
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    keep[u] = !D.checkmarine || icestar_keep(vv[u], tt[u], D.rhow, D.rhoi);
    const double is = keep[u] ? vv[u] : __dmul_rn(vv[u], 0.0);
    bt[u] = is < EPS0;
  }
  stm2(D.m(M_GR, b), h, keep[0], keep[1]);
  stm2(D.m(M_BETA, b), h, bt[0], bt[1]);
  stm2(D.m(M_CSTAR, b), h, cx.x && bt[0], cx.y && bt[1]);
  if (D.ss[b].first) {
    const double2 vp = ld2(D.g(G_ICE_PREV, b), h), ti = ld2(D.g(G_TINIT, b), h);
    const double o0 = D.checkmarine ? icestar_on(vp.x, ti.x, D.rhow, D.rhoi) : vp.x;
    const double o1 = D.checkmarine ? icestar_on(vp.y, ti.y, D.rhow, D.rhoi) : vp.y;
    st2(D.g(G_TMP, b), h, o0, o1);
  }
}

// The rotation block (solver.py:910-975) for the coming inner iteration, one thread; writes
// il, m, Lambda, their increments and the degree-2 rotational sea-level / radial terms.  Runs
// in the one-block control kernels (k_rotation, k_loop_cond), one thread per slot.
__device__ void rotation_block(const Dev& D, int b, Scal* sc) {
  const RotConst& C = D.rc[b];
  const double2* dScur = D.sp(S_DSCUR, b);
  const double2* dI = D.sp(S_DI, b);
  // every input first: the record's fields are global memory and the stores below could alias
  // them as far as the compiler knows (each load of this serial code is a round trip)
  const double2 s20 = __ldcg(dScur + D.i20), s21 = __ldcg(dScur + D.i21);
  const double2 i20 = __ldcg(dI + D.i20), i21 = __ldcg(dI + D.i21);
  double sum_il[9], sum_m[3], sum_tsl[6], sum_trr[6], dprev[6], oldil[9], oldm[3];
  for (int q = 0; q < 9; ++q) {
    sum_il[q] = sc->sum_il[q];
    oldil[q] = sc->oldil[q];
  }
  for (int q = 0; q < 3; ++q) {
    sum_m[q] = sc->sum_m[q];
    oldm[q] = sc->oldm[q];
  }
  for (int q = 0; q < 6; ++q) {
    sum_tsl[q] = sc->sum_tsl[q];
    sum_trr[q] = sc->sum_trr[q];
    dprev[q] = sc->dlam_prev2[q];
  }
  const double z20r = __dadd_rn(__dmul_rn(C.rhow, s20.x), __dmul_rn(C.rhoi, i20.x));
  const double z21r = __dadd_rn(__dmul_rn(C.rhow, s21.x), __dmul_rn(C.rhoi, i21.x));
  const double z21i = __dadd_rn(__dmul_rn(C.rhow, s21.y), __dmul_rn(C.rhoi, i21.y));
  // only il[0:3, 2] and lam[0,0], lam[2, 0:3] are ever non-zero (solver.py:916-919, 950-956)
  double il[9];
  for (int q = 0; q < 9; ++q) il[q] = 0.0;
  il[8] = __dmul_rn(C.c_il22, z20r);
  il[2] = __dmul_rn(C.c_il02, z21r);
  il[5] = __dmul_rn(C.c_il12, z21i);
  double mm[3];
  const SlotStep& ss = D.ss[b];
  if (ss.ramp) {
    // the current increments carry 1 - phi of their viscous response, implicit in m
    // (solver.py:922-935): sil = sum_il + c_il dil, m_i = alpha (...) / (1 - alpha c_m / kf)
    double sil[9];
    for (int q = 0; q < 9; ++q) sil[q] = __dadd_rn(sum_il[q], __dmul_rn(ss.c_il, __dsub_rn(il[q], oldil[q])));
    const double den = __dsub_rn(1.0, __ddiv_rn(__dmul_rn(C.alpha, ss.c_m), C.kf));
    for (int i = 0; i < 2; ++i) {
      const double a = __dadd_rn(__dmul_rn(C.onepk, il[i * 3 + 2]), sil[i * 3 + 2]);
      const double sm = __dsub_rn(sum_m[i], __dmul_rn(ss.c_m, oldm[i]));
      mm[i] = __ddiv_rn(__dmul_rn(C.alpha, __dadd_rn(__dmul_rn(C.inv_CmA, a), __dmul_rn(C.inv_kf, sm))), den);
    }
    mm[2] = __dmul_rn(-C.inv_C, __dadd_rn(__dmul_rn(C.onepk, il[8]), sil[8]));
  } else {
    for (int i = 0; i < 2; ++i) {
      const double a = __dadd_rn(__dmul_rn(C.onepk, il[i * 3 + 2]), sum_il[i * 3 + 2]);
      mm[i] = __dmul_rn(C.alpha, __dadd_rn(__dmul_rn(C.inv_CmA, a), __dmul_rn(C.inv_kf, sum_m[i])));
    }
    mm[2] = __dmul_rn(-C.inv_C, __dadd_rn(__dmul_rn(C.onepk, il[8]), sum_il[8]));
  }
  const double m1 = mm[0], m2 = mm[1], m3 = mm[2];
  const double m1s = __dmul_rn(m1, m1), m2s = __dmul_rn(m2, m2), m3s = __dmul_rn(m3, m3);
  double lam[18];
  for (int q = 0; q < 18; ++q) lam[q] = 0.0;
  lam[0] = __dmul_rn(C.r2w2_3, __dadd_rn(__dadd_rn(__dadd_rn(m1s, m2s), m3s), __dmul_rn(2.0, m3)));
  lam[12] = __dmul_rn(C.r2w2_6s5, __dsub_rn(__dsub_rn(__dadd_rn(m1s, m2s), __dmul_rn(2.0, m3s)), __dmul_rn(4.0, m3)));
  const double op = __dadd_rn(1.0, m3);
  lam[14] = __dmul_rn(-C.r2w2_s30, __dmul_rn(m1, op));
  lam[15] = __dmul_rn(-C.r2w2_s30, __dmul_rn(-m2, op));
  lam[16] = __dmul_rn(C.r2w2_s120, __dsub_rn(m2s, m1s));
  lam[17] = __dmul_rn(C.r2w2_s120, __dmul_rn(__dmul_rn(2.0, m1), m2));
  double dsl_rot[6], rr_rot[6], dcur[6];
  for (int q = 0; q < 3; ++q) {
    const double dr = __dsub_rn(lam[12 + 2 * q], dprev[2 * q]);
    const double di = __dsub_rn(lam[13 + 2 * q], dprev[2 * q + 1]);
    const double tr = __dadd_rn(dprev[2 * q], dr);
    const double ti = __dadd_rn(dprev[2 * q + 1], di);
    double tsr = sum_tsl[2 * q], tsi = sum_tsl[2 * q + 1], trr = sum_trr[2 * q], tri = sum_trr[2 * q + 1];
    if (ss.ramp) {   // solver.py:964-966
      tsr = __dadd_rn(tsr, __dmul_rn(ss.c_tsl, dr));
      tsi = __dadd_rn(tsi, __dmul_rn(ss.c_tsl, di));
      trr = __dadd_rn(trr, __dmul_rn(ss.c_trr, dr));
      tri = __dadd_rn(tri, __dmul_rn(ss.c_trr, di));
    }
    dsl_rot[2 * q] = __ddiv_rn(__dadd_rn(__dmul_rn(C.ekhTE, tr), tsr), C.gacc);
    dsl_rot[2 * q + 1] = __ddiv_rn(__dadd_rn(__dmul_rn(C.ekhTE, ti), tsi), C.gacc);
    rr_rot[2 * q] = __ddiv_rn(__dadd_rn(__dmul_rn(C.hTE2, tr), trr), C.gacc);
    rr_rot[2 * q + 1] = __ddiv_rn(__dadd_rn(__dmul_rn(C.hTE2, ti), tri), C.gacc);
    dcur[2 * q] = dr;
    dcur[2 * q + 1] = di;
  }
  for (int q = 0; q < 6; ++q) {
    sc->dsl_rot[q] = dsl_rot[q];
    sc->rr_rot[q] = rr_rot[q];
    sc->dlam_cur2[q] = dcur[q];
  }
  for (int q = 0; q < 9; ++q) {
    sc->il[q] = il[q];
    sc->dil[q] = __dsub_rn(il[q], oldil[q]);
  }
  for (int q = 0; q < 3; ++q) {
    sc->mm[q] = mm[q];
    sc->dm[q] = __dsub_rn(mm[q], oldm[q]);
  }
  for (int q = 0; q < 18; ++q) sc->lam[q] = lam[q];
}

// dice = I*_lm - old ; dI = p_ice + dice ; first guess of the load increment ; dS_cur ;
// so = sum|load_inc|  (solver.py:868-905; extrap solver_opt.py:504-513).  old = the analysed
// previous ice at the slot's first step, else the committed I*_lm of the last step (copied into
// oldice here).  The last block evaluates the rotation block for the first inner iteration.
__global__ void k_pre_spec(Dev D) {
  SLOT_OR_RETURN();
  __shared__ double sh[32];
  const SlotStep ss = D.ss[b];
  const double2* icelm = D.sp(S_ICELM, b);
  double2* oldice = D.sp(S_OLDICE, b);
  const double2* osrc = ss.first ? oldice : D.sp(S_PREV_ICE, b);
  const double2* h1 = D.sp(ss.hsel ? S_HB : S_HA, b);
  const double2* h2 = D.sp(ss.hsel ? S_HA : S_HB, b);
  const double2* cstarlm = D.sp(S_CSTARLM, b);
  double acc = 0.0;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < D.ncoef) {
    const double2 o0 = osrc[0];
    const double2 dice00 = make_double2(__dsub_rn(icelm[0].x, o0.x), __dsub_rn(icelm[0].y, o0.y));
    const double fr = -D.rhoi / D.rhow;
    const double2 s00 = make_double2(__dmul_rn(fr, dice00.x), __dmul_rn(fr, dice00.y));
    const double2 a = icelm[i], o = osrc[i];
    if (!ss.first) oldice[i] = o;
    const double2 d = make_double2(__dsub_rn(a.x, o.x), __dsub_rn(a.y, o.y));
    D.sp(S_DICE, b)[i] = d;
    const double2 pi = D.sp(S_P_ICE, b)[i];
    D.sp(S_DI, b)[i] = make_double2(__dadd_rn(pi.x, d.x), __dadd_rn(pi.y, d.y));
    double2 g;
    if (ss.warm_ds) {
      g = ss.warm_ds[i];   // warm start replaces the eustatic / extrapolated guess
    } else if (ss.mode == 0) {
      g = np_cmul(np_cdiv(cstarlm[i], cstarlm[0]), s00);
    } else if (ss.mode == 1) {
      const double2 u = h1[i], v = h2[i];
      g = make_double2(__dsub_rn(__dmul_rn(u.x, 2.0), v.x), __dsub_rn(__dmul_rn(u.y, 2.0), v.y));
    } else {
      const double2 u = h1[i], v = h2[i];
      g = make_double2(__dsub_rn(__dmul_rn(u.x, ss.c1), __dmul_rn(ss.c2, v.x)),
                       __dsub_rn(__dmul_rn(u.y, ss.c1), __dmul_rn(ss.c2, v.y)));
    }
    D.sp(S_LOAD, b)[i] = g;
    if (ss.mode == 0 && !ss.warm_ds) {
      D.sp(S_DSCUR, b)[i] = make_double2(0.0, 0.0);
    } else {
      const double2 p = D.sp(S_P_OCEAN, b)[i];
      D.sp(S_DSCUR, b)[i] = make_double2(__dadd_rn(p.x, g.x), __dadd_rn(p.y, g.y));
    }
    acc = cabs_(g);
  }
  const double part = block_sum(acc, sh);
  double tot;
  if (last_block_total(part, D.partials + (size_t)b * D.npart, D.counter + 4 * b, &tot, sh)) {
    if (threadIdx.x == 0) sc->so = tot;
  }
}

// Eq. B18 (solver.py:977-991) plus the degree-2 rotational term of the current iteration.  With
// bsyn (mixed precision, the iteration's synthesis one launch), the result goes straight into
// that launch's B operand as field b instead of the FP64 spectrum, of which only (0, 0) is kept
// (the degree-0 term the unfold adds in FP64).
__global__ void k_b18(Dev D, float* bsyn, const int* bpos) {
  SLOT_OR_RETURN();
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= D.ncoef) return;
  if (i == 0) {
    sc->gr_changed = 0;  // the previous iteration's mask changes are consumed
    sc->cs_changed = 0;
  }
  const int l = D.lidx[i];
  const double2 a = D.sp(S_DI, b)[i], bb = D.sp(S_P_OCEAN, b)[i], c = D.sp(S_LOAD, b)[i];
  const double2 v = D.sp(S_VISC, b)[i];
  const double te = D.ttlekhl[(size_t)b * D.nl + l], t = D.ttl[(size_t)b * D.nl + l];
  double re = __dadd_rn(__dadd_rn(__dmul_rn(a.x, D.rhoi), __dmul_rn(bb.x, D.rhow)), __dmul_rn(c.x, D.rhow));
  double im = __dadd_rn(__dadd_rn(__dmul_rn(a.y, D.rhoi), __dmul_rn(bb.y, D.rhow)), __dmul_rn(c.y, D.rhow));
  re = __dadd_rn(__dmul_rn(re, te), __dmul_rn(v.x, t));
  im = __dadd_rn(__dmul_rn(im, te), __dmul_rn(v.y, t));
  const SlotStep& ss = D.ss[b];
  if (ss.ramp) {   // same-step viscous weight of the current increment (solver.py:988-989)
    const double tc = ss.ramp_tab[(size_t)D.K * D.nl + l];
    const double2 d = D.sp(S_DICE, b)[i];
    re = __dadd_rn(re, __dmul_rn(tc, __dadd_rn(__dmul_rn(D.rhoi, d.x), __dmul_rn(D.rhow, c.x))));
    im = __dadd_rn(im, __dmul_rn(tc, __dadd_rn(__dmul_rn(D.rhoi, d.y), __dmul_rn(D.rhow, c.y))));
  }
  if (D.tpw) {
    const int q = (i == D.i20) ? 0 : (i == D.i21) ? 1 : (i == D.i22) ? 2 : -1;
    if (q >= 0) {
      re = __dadd_rn(re, sc->dsl_rot[2 * q]);
      im = __dadd_rn(im, sc->dsl_rot[2 * q + 1]);
    }
  }
  if (bsyn) {
    mx_bsyn_put(bsyn, __ldg(bpos + i), b, i == 0 ? make_double2(0.0, 0.0) : make_double2(re, im));
    if (i == 0) D.sp(S_SL, b)[0] = make_double2(re, im);
  } else {
    D.sp(S_SL, b)[i] = make_double2(re, im);
  }
}

// conserv, the load update and xi (solver.py:1002-1030):
//   new = ((-dSprev + rO) + C*_lm conserv) - tO ;  dS_cur = dSprev + new ;  sa = sum|new|
// The slot's last block decides its convergence.  Each block first prefetches into L2 the four
// input spectra of the block one resident wave further on in launch order.
__global__ void k_update(Dev D) {
  pdl_wait();
  pdl_trigger();
  {
    int bx, by;
    if (threadIdx.x < 4 && block_ahead(D.upd_ahead, bx, by) && !D.sc[D.slot0 + by].done) {
      const int b2 = D.slot0 + by;
      const long long i0 = (long long)bx * blockDim.x;
      const int id = threadIdx.x == 0 ? S_P_OCEAN : threadIdx.x == 1 ? S_ROLM : threadIdx.x == 2 ? S_CSTARLM : S_TOLM;
      prefetch_l2(D.sp(id, b2) + i0,
                  (uint32_t)min((long long)blockDim.x, D.ncoef - i0) * (uint32_t)sizeof(double2));
    }
  }
  SLOT_OR_RETURN();
  __shared__ double sh[32];
  const double2* dSprev = D.sp(S_P_OCEAN, b);
  const double2* rOlm = D.sp(S_ROLM, b);
  const double2* cstarlm = D.sp(S_CSTARLM, b);
  const double2* tOlm = D.sp(S_TOLM, b);
  const double2* dI = D.sp(S_DI, b);
  // conserv = ((1 / C*_00) * (-(rhoi/rhow) dI_00 - rO_00 + tO_00)).real
  const double2 c00 = cstarlm[0];
  const double2 rinv = np_cdiv(make_double2(1.0, 0.0), c00);
  const double fr = __dmul_rn(-1.0, __ddiv_rn(D.rhoi, D.rhow));
  const double2 d00 = dI[0], r00 = rOlm[0], t00 = tOlm[0];
  const double2 x = make_double2(__dadd_rn(__dsub_rn(__dmul_rn(fr, d00.x), r00.x), t00.x),
                                 __dadd_rn(__dsub_rn(__dmul_rn(fr, d00.y), r00.y), t00.y));
  const double conserv = __dsub_rn(__dmul_rn(rinv.x, x.x), __dmul_rn(rinv.y, x.y));
  double acc = 0.0;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < D.ncoef) {
    const double2 p = dSprev[i], r = rOlm[i], c = cstarlm[i], t = tOlm[i];
    double nr = __dadd_rn(-p.x, r.x), ni = __dadd_rn(-p.y, r.y);
    nr = __dadd_rn(nr, __dmul_rn(c.x, conserv));
    ni = __dadd_rn(ni, __dmul_rn(c.y, conserv));
    nr = __dsub_rn(nr, t.x);
    ni = __dsub_rn(ni, t.y);
    D.sp(S_LOAD, b)[i] = make_double2(nr, ni);
    // dS_cur = dS_prev + new: the rotation block of the next iteration reads its degree-2 entries;
    // the commit forms the whole of it from the converged increment (the same sum)
    if (i == D.i20 || i == D.i21) D.sp(S_DSCUR, b)[i] = make_double2(__dadd_rn(p.x, nr), __dadd_rn(p.y, ni));
    acc = hypot(nr, ni);
  }
  const double part = block_sum(acc, sh);
  double sa;
  if (last_block_total(part, D.partials + (size_t)b * D.npart, D.counter + 4 * b, &sa, sh)) {
    if (threadIdx.x == 0) {
      const double so = sc->so;
      double xi;
      if (fabs(sa - so) < EPS0 && fabs(so) < EPS0) xi = 0.0;
      else if (fabs(so) < EPS0) xi = fabs((sa - so) / (EPS0 * 10.0));
      else xi = fabs((sa - so) / so);
      sc->conserv = conserv;
      sc->sa = sa;
      sc->xi = xi;
      sc->so = sa;
      sc->numiter += 1;
      if (sc->status != 0 || !(xi == xi) || !isfinite(sa)) {
        if (sc->status == 0) sc->status = SLE_ERR_NONFINITE;
        sc->converged = 1;
      } else if (xi <= D.epsilon1) {
        sc->converged = 1;
      } else if (sc->numiter >= MAX_INNER) {
        sc->status = SLE_ERR_NONCONVERGED;
        sc->converged = 1;
      }
    }
  }
}

// sl_tot = sl_inc with conserv added to (0,0) (plain path, solver.py:1017-1021)
__global__ void k_sltot(Dev D) {
  SLOT_OR_RETURN();
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= D.ncoef) return;
  double2 v = D.sp(S_SL, b)[i];
  if (i == 0) v.x = __dadd_rn(v.x, sc->conserv);
  D.sp(S_SLTOT, b)[i] = v;
}

// deltasl (dsl identity) and, when not converged, the ocean function of the refreshed
// topography and the grounded-ice test on it (solver.py:1032-1037, 661-684).
__global__ void k_refresh1(Dev D) {
  pdl_wait();
  pdl_trigger();
  SLOT_OR_RETURN();
  __shared__ double sh[32];
  const bool conv = sc->converged != 0;
  const bool test = !conv && D.checkmarine && sc->gr_nacc < GR_MAXACC;
  const double cadd = D.opt_dsl ? __dmul_rn(sc->conserv, sc->K00) : 0.0;
  double cnt = 0.0;
  const long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (2 * h < D.ng) {
    // every input first (the stores below could alias them as far as the compiler knows)
    double* deltasl = D.g(G_DELTASL, b);
    const double2 a = ld2(D.opt_dsl ? D.g(G_DSL, b) : deltasl, h);
    double2 ti = make_double2(0.0, 0.0), ic = ti;
    uchar2 be = make_uchar2(0, 0);
    if (!conv) ti = ld2(D.g(G_TINIT, b), h);
    if (test) {
      ic = ld2(D.g(G_ICE, b), h);
      be = ldm2(D.m(M_BETA, b), h);
    }
    double ds[2] = {a.x, a.y};
    if (D.opt_dsl) {
      ds[0] = __dadd_rn(a.x, cadd);
      ds[1] = __dadd_rn(a.y, cadd);
      // only the converged iteration's deltasl is an output; the others only feed the masks below
      if (conv) st2(deltasl, h, ds[0], ds[1]);
    }
    if (!conv) {
      const double t0 = __dsub_rn(ti.x, ds[0]), t1 = __dsub_rn(ti.y, ds[1]);
      stm2(D.m(M_CXY, b), h, t0 < 0.0, t1 < 0.0);
      if (test) {
        const bool k0 = icestar_keep(ic.x, t0, D.rhow, D.rhoi), k1 = icestar_keep(ic.y, t1, D.rhow, D.rhoi);
        const double g0 = k0 ? ic.x : __dmul_rn(ic.x, 0.0), g1 = k1 ? ic.y : __dmul_rn(ic.y, 0.0);
        stm2(D.m(M_GRNEW, b), h, k0, k1);
        if ((g0 < EPS0) != (be.x != 0)) cnt += 1.0;
        if ((g1 < EPS0) != (be.y != 0)) cnt += 1.0;
      }
    }
  }
  if (!test) return;
  const double part = block_sum(cnt, sh);
  double tot;
  if (last_block_total(part, D.partials + (size_t)b * D.npart + D.part_grid, D.counter + 4 * b + 1, &tot, sh)) {
    if (threadIdx.x == 0) {
      sc->gr_reguess += 1;
      sc->nd = (unsigned int)tot;
      if (tot > 0.0) {
        sc->gr_changed = 1;
        sc->gr_nacc += 1;
        sc->gr_ice_an += 1;
      } else {
        sc->gr_changed = 0;
      }
    }
  }
}

// C* on the refreshed ocean function; accepted grounded-ice mask (solver.py:664-684).  tO =
// T0 (C* - C*0) is formed by its analysis.
__global__ void k_refresh2(Dev D) {
  pdl_wait();
  pdl_trigger();
  SLOT_OR_RETURN();
  const long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (2 * h >= D.ng || sc->converged) return;
  const bool changed = sc->gr_changed != 0;
  // every input first (the stores below could alias them as far as the compiler knows)
  const uchar2 cx = ldm2(D.m(M_CXY, b), h), prev = ldm2(D.m(M_CSTAR, b), h);
  uchar2 k = make_uchar2(0, 0), bt = make_uchar2(0, 0);
  double2 ic = make_double2(0.0, 0.0);
  if (changed) {
    k = ldm2(D.m(M_GRNEW, b), h);
    ic = ld2(D.g(G_ICE, b), h);
  } else {
    bt = ldm2(D.m(M_BETA, b), h);
  }
  if (changed) {
    const double g0 = k.x ? ic.x : __dmul_rn(ic.x, 0.0), g1 = k.y ? ic.y : __dmul_rn(ic.y, 0.0);
    reinterpret_cast<uchar2*>(D.m(M_GR, b))[h] = k;
    bt = make_uchar2(g0 < EPS0, g1 < EPS0);
    reinterpret_cast<uchar2*>(D.m(M_BETA, b))[h] = bt;
  }
  const uchar2 c = make_uchar2(cx.x && bt.x, cx.y && bt.y);
  // C* and tO only change where a cell of C* flips; without a flip their re-analyses are
  // skipped (the inputs, hence the spectra, are bit-identical to the last ones)
  if (prev.x != c.x || prev.y != c.y) {
    sc->cs_changed = 1;
    reinterpret_cast<uchar2*>(D.m(M_CSTAR, b))[h] = c;
  }
}

// The same pass over eight cells per thread (8-byte mask loads and stores, four double2 ice
// loads), for grids whose cell count is a multiple of 8; per cell the arithmetic of k_refresh2.
__device__ __forceinline__ unsigned char byte_of(uint2 v, int i) {
  return (unsigned char)(((i < 4 ? v.x : v.y) >> (8 * (i & 3))) & 0xffu);
}
__global__ void k_refresh2_x8(Dev D) {
  pdl_wait();
  pdl_trigger();
  SLOT_OR_RETURN();
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (8 * q >= D.ng || sc->converged) return;
  const bool changed = sc->gr_changed != 0;
  const uint2 cx = reinterpret_cast<const uint2*>(D.m(M_CXY, b))[q];
  const uint2 prev = reinterpret_cast<const uint2*>(D.m(M_CSTAR, b))[q];
  uint2 k = make_uint2(0u, 0u), bt = make_uint2(0u, 0u);
  double2 ic[4];
  if (changed) {
    k = reinterpret_cast<const uint2*>(D.m(M_GRNEW, b))[q];
#pragma unroll
    for (int u = 0; u < 4; ++u) ic[u] = ld2(D.g(G_ICE, b), 4 * q + u);
  } else {
    bt = reinterpret_cast<const uint2*>(D.m(M_BETA, b))[q];
  }
  if (changed) {
    unsigned int lo = 0u, hi = 0u;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const double v = (i & 1) ? ic[i >> 1].y : ic[i >> 1].x;
      const double gi = byte_of(k, i) ? v : __dmul_rn(v, 0.0);
      const unsigned int bit = (gi < EPS0) ? 1u : 0u;
      if (i < 4) lo |= bit << (8 * i);
      else hi |= bit << (8 * (i - 4));
    }
    bt = make_uint2(lo, hi);
    reinterpret_cast<uint2*>(D.m(M_GR, b))[q] = k;
    reinterpret_cast<uint2*>(D.m(M_BETA, b))[q] = bt;
  }
  unsigned int clo = 0u, chi = 0u;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const unsigned int ci = (byte_of(cx, i) && byte_of(bt, i)) ? 1u : 0u;
    if (i < 4) clo |= ci << (8 * i);
    else chi |= ci << (8 * (i - 4));
  }
  if (clo != prev.x || chi != prev.y) {
    sc->cs_changed = 1;
    reinterpret_cast<uint2*>(D.m(M_CSTAR, b))[q] = make_uint2(clo, chi);
  }
}

// dice, dI after a grounded-mask change.  Such a change is rare after the first iterations, so
// each slot gets a fixed row of blocks that stride over its coefficients: a slot whose mask did
// not change costs DICE_BLOCKS early exits instead of one per 256 coefficients.
constexpr int DICE_BLOCKS = 64;
__global__ void __launch_bounds__(256) k_dice(Dev D) {
  pdl_wait();
  SLOT_OR_RETURN();
  if (sc->converged || !sc->gr_changed) return;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < D.ncoef; i += stride) {
    const double2 a = D.sp(S_ICELM, b)[i], o = D.sp(S_OLDICE, b)[i], p = D.sp(S_P_ICE, b)[i];
    const double2 d = make_double2(__dsub_rn(a.x, o.x), __dsub_rn(a.y, o.y));
    D.sp(S_DICE, b)[i] = d;
    D.sp(S_DI, b)[i] = make_double2(__dadd_rn(p.x, d.x), __dadd_rn(p.y, d.y));
  }
}

// End of an inner iteration: slots that converged (or failed) are done from the next iteration
// on; the loop goes on while any slot is not, and each such slot (one thread per slot) evaluates
// the rotation block of its next iteration.  A raised tensor-core timeout ends every slot.
// The rotation block of the first inner iteration of every stepping slot (one thread per slot),
// after the step prologue has formed dS_cur and dI.
__global__ void k_rotation(Dev D) {
  for (int b = threadIdx.x; b < D.nslot; b += blockDim.x) {
    Scal* sc = D.sc + b;
    if (!sc->done && D.tpw) rotation_block(D, b, sc);
  }
}

__global__ void k_loop_cond(Dev D, const int* bstatus, cudaGraphConditionalHandle loop) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  const int bs = *bstatus;
  for (int b = threadIdx.x; b < D.nslot; b += blockDim.x) {
    Scal* sc = D.sc + b;
    if (sc->done) continue;
    if (bs != 0) {
      if (sc->status == 0) sc->status = bs;
      sc->converged = 1;
    }
    if (sc->converged) {
      sc->done = 1;
    } else {
      atomicOr(&any, 1);
      // the rotation block of the coming iteration (solver.py:910-975) from this iteration's
      // dS_cur and the current dI (after a grounded re-guess, the re-analysed one)
      if (D.tpw) rotation_block(D, b, sc);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0 && loop) cudaGraphSetConditional(loop, any ? 1u : 0u);
}

// After the loop: re-open the slots that step in this call for the post-loop kernels.
__global__ void k_reopen(Dev D) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= D.nslot) return;
  if (D.ss[b].active) D.sc[b].done = 0;
}

// Radial displacement spectrum (solver.py:1054-1069)
__global__ void k_rr(Dev D) {
  SLOT_OR_RETURN();
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= D.ncoef || sc->status) return;
  const int l = D.lidx[i];
  const double2 a = D.sp(S_DI, b)[i], bb = D.sp(S_P_OCEAN, b)[i], c = D.sp(S_LOAD, b)[i];
  const double2 v = D.sp(S_RAD, b)[i];
  const double th = D.ttlhe[(size_t)b * D.nl + l], t = D.ttl[(size_t)b * D.nl + l];
  double re = __dadd_rn(__dadd_rn(__dmul_rn(a.x, D.rhoi), __dmul_rn(bb.x, D.rhow)), __dmul_rn(c.x, D.rhow));
  double im = __dadd_rn(__dadd_rn(__dmul_rn(a.y, D.rhoi), __dmul_rn(bb.y, D.rhow)), __dmul_rn(c.y, D.rhow));
  re = __dadd_rn(__dmul_rn(re, th), __dmul_rn(v.x, t));
  im = __dadd_rn(__dmul_rn(im, th), __dmul_rn(v.y, t));
  const SlotStep& ss = D.ss[b];
  if (ss.ramp) {   // solver.py:1065-1067
    const double tc = ss.ramp_tab[(size_t)(D.K + 1) * D.nl + l];
    const double2 d = D.sp(S_DICE, b)[i];
    re = __dadd_rn(re, __dmul_rn(tc, __dadd_rn(__dmul_rn(D.rhoi, d.x), __dmul_rn(D.rhow, c.x))));
    im = __dadd_rn(im, __dmul_rn(tc, __dadd_rn(__dmul_rn(D.rhoi, d.y), __dmul_rn(D.rhow, c.y))));
  }
  if (D.tpw) {
    const int q = (i == D.i20) ? 0 : (i == D.i21) ? 1 : (i == D.i22) ? 2 : -1;
    if (q >= 0) {
      re = __dadd_rn(re, sc->rr_rot[2 * q]);
      im = __dadd_rn(im, sc->rr_rot[2 * q + 1]);
    }
  }
  D.sp(S_RRLM, b)[i] = make_double2(re, im);
}

// commit (solver.py:1080-1096): cur = rhoi dice + rhow load (l = 0 zeroed); p_load += cur;
// p_ice = dI ; p_ocean = dS_cur ; prev_ice = I*_lm ; extrap history (the older buffer) = load;
// thread 0 also commits the rotational increments and records I*_00.
// Analytic rate spectra (per year) at the end of the step, read before the commit
// (solver.py:464-474, 766-785): with cur = the step's load increment (formed as k_commit forms
// it), P = the load committed before the step and q = sum_k w_k R_k over the degree's modes,
//   rs = (ws P - q) + wsphi cur,  dsl = (ttlekhl cur) / h + ttl rs   (sea level, w = w_sl)
//   rr likewise with w_rr,        drr = (ttlhe cur) / h + ttl rr     (radial)
// and zero at degree 0; each operation rounded as NumPy rounds it.  The degree-2 rotational rates
// are added on the host.
__global__ void k_rate_spec(Dev D, double2* rspec, const double* rtab, double* rrec, double* rrot) {
  SLOT_OR_RETURN();
  const SlotStep& ss = D.ss[b];
  if (!ss.rates || sc->status) return;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= D.ncoef) return;
  double2* dsl = rspec + ((size_t)b * 2 + 0) * D.ncoef;
  double2* drr = rspec + ((size_t)b * 2 + 1) * D.ncoef;
  if (i == 0) {
    const double2 d0 = D.sp(S_DICE, b)[0];
    rrec[2 * b] = d0.x;
    rrec[2 * b + 1] = d0.y;
    // the degree-2 modal states as the commit finds them (with ramp placement it changes them)
    const int K = D.K;
    double* o = rrot + (size_t)b * 18 * K;
    for (int q = 0; q < 9 * K; ++q) o[q] = D.r_il[(size_t)b * K * 9 + q];
    for (int q = 0; q < 3 * K; ++q) o[9 * K + q] = D.r_m[(size_t)b * K * 3 + q];
    for (int q = 0; q < 6 * K; ++q) o[12 * K + q] = D.r_lam[(size_t)b * K * 6 + q];
  }
  const int l = D.lidx[i];
  if (l == 0) {
    dsl[i] = make_double2(0.0, 0.0);
    drr[i] = make_double2(0.0, 0.0);
    return;
  }
  const int nl = D.nl, K = D.K;
  const double2 ld = D.sp(S_LOAD, b)[i], d = D.sp(S_DICE, b)[i];
  const double2 cur = make_double2(__dadd_rn(__dmul_rn(d.x, D.rhoi), __dmul_rn(ld.x, D.rhow)),
                                   __dadd_rn(__dmul_rn(d.y, D.rhoi), __dmul_rn(ld.y, D.rhow)));
  const double2 P = D.sp(S_P_LOAD, b)[i];
  const double* t = rtab + (size_t)b * (2 * K + 4) * nl;
  const double *w_sl = t, *w_rr = t + (size_t)K * nl, *ws_sl = t + (size_t)2 * K * nl, *ws_rr = ws_sl + nl,
               *wp_sl = ws_rr + nl, *wp_rr = wp_sl + nl;
  double2 qs = make_double2(0.0, 0.0), qr = qs;
  const double2* R = D.R + (size_t)b * K * D.ncoef;
  const int nk = D.nmod[(size_t)b * nl + l];
  for (int k = 0; k < nk; ++k) {
    const double2 r = R[(size_t)k * D.ncoef + i];
    const double a = w_sl[(size_t)k * nl + l], c = w_rr[(size_t)k * nl + l];
    qs = make_double2(__dadd_rn(qs.x, __dmul_rn(a, r.x)), __dadd_rn(qs.y, __dmul_rn(a, r.y)));
    qr = make_double2(__dadd_rn(qr.x, __dmul_rn(c, r.x)), __dadd_rn(qr.y, __dmul_rn(c, r.y)));
  }
  const double h = ss.rate_h;
  const size_t tl = (size_t)b * nl + l;
  const double ttl = D.ttl[tl], tek = D.ttlekhl[tl], the = D.ttlhe[tl];
  double2 rs, rr;
  rs.x = __dadd_rn(__dsub_rn(__dmul_rn(ws_sl[l], P.x), qs.x), __dmul_rn(wp_sl[l], cur.x));
  rs.y = __dadd_rn(__dsub_rn(__dmul_rn(ws_sl[l], P.y), qs.y), __dmul_rn(wp_sl[l], cur.y));
  rr.x = __dadd_rn(__dsub_rn(__dmul_rn(ws_rr[l], P.x), qr.x), __dmul_rn(wp_rr[l], cur.x));
  rr.y = __dadd_rn(__dsub_rn(__dmul_rn(ws_rr[l], P.y), qr.y), __dmul_rn(wp_rr[l], cur.y));
  dsl[i] = make_double2(__dadd_rn(__ddiv_rn(__dmul_rn(tek, cur.x), h), __dmul_rn(ttl, rs.x)),
                        __dadd_rn(__ddiv_rn(__dmul_rn(tek, cur.y), h), __dmul_rn(ttl, rs.y)));
  drr[i] = make_double2(__dadd_rn(__ddiv_rn(__dmul_rn(the, cur.x), h), __dmul_rn(ttl, rr.x)),
                        __dadd_rn(__ddiv_rn(__dmul_rn(the, cur.y), h), __dmul_rn(ttl, rr.y)));
}

// Horizontal-displacement potential (solver.py:687-720, horizontal read-out), read before the
// commit: with A = (rhoi dI* + rhow dS_prev) + rhow load (the load of the radial term, formed as
// k_rr forms it) and visc_h = sum_k a_hl R_k over the degree's modes,
//   Psi = (ttl l^E) A + ttl visc_h,  zero at degree 0;
// the degree-2 rotational term is added on the host.
__global__ void k_horiz_spec(Dev D, double2* hspec, const double* htab) {
  SLOT_OR_RETURN();
  if (!D.ss[b].horiz || sc->status) return;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= D.ncoef) return;
  double2* out = hspec + (size_t)b * D.ncoef;
  const int l = D.lidx[i];
  if (l == 0) {
    out[i] = make_double2(0.0, 0.0);
    return;
  }
  const int nl = D.nl, K = D.K;
  const double* a_hl = htab + (size_t)b * (K + 1) * nl;
  const double ttlle = a_hl[(size_t)K * nl + l];
  const double2 a = D.sp(S_DI, b)[i], bb = D.sp(S_P_OCEAN, b)[i], c = D.sp(S_LOAD, b)[i];
  const double re = __dadd_rn(__dadd_rn(__dmul_rn(a.x, D.rhoi), __dmul_rn(bb.x, D.rhow)), __dmul_rn(c.x, D.rhow));
  const double im = __dadd_rn(__dadd_rn(__dmul_rn(a.y, D.rhoi), __dmul_rn(bb.y, D.rhow)), __dmul_rn(c.y, D.rhow));
  double2 v = make_double2(0.0, 0.0);
  const double2* R = D.R + (size_t)b * K * D.ncoef;
  const int nk = D.nmod[(size_t)b * nl + l];
  for (int k = 0; k < nk; ++k) {
    const double2 r = R[(size_t)k * D.ncoef + i];
    const double w = a_hl[(size_t)k * nl + l];
    v = make_double2(__dadd_rn(v.x, __dmul_rn(w, r.x)), __dadd_rn(v.y, __dmul_rn(w, r.y)));
  }
  const double t = D.ttl[(size_t)b * nl + l];
  out[i] = make_double2(__dadd_rn(__dmul_rn(ttlle, re), __dmul_rn(t, v.x)),
                        __dadd_rn(__dmul_rn(ttlle, im), __dmul_rn(t, v.y)));
}

__global__ void k_commit(Dev D, int extrap) {
  SLOT_OR_RETURN();
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= D.ncoef || sc->status) return;
  if (i == 0) {
    if (D.tpw) {
      for (int q = 0; q < 9; ++q) sc->p_il[q] = __dadd_rn(sc->p_il[q], sc->dil[q]);
      for (int q = 0; q < 3; ++q) sc->p_m[q] = __dadd_rn(sc->p_m[q], sc->dm[q]);
      for (int q = 0; q < 6; ++q) sc->p_lambda[q] = __dadd_rn(sc->p_lambda[q], sc->dlam_cur2[q]);
    }
    sc->diag[4] = D.sp(S_ICELM, b)[0].x;
  }
  const int l = D.lidx[i];
  double2 cur = make_double2(0.0, 0.0);
  const double2 ld = D.sp(S_LOAD, b)[i];
  if (l != 0) {
    const double2 d = D.sp(S_DICE, b)[i];
    cur = make_double2(__dadd_rn(__dmul_rn(d.x, D.rhoi), __dmul_rn(ld.x, D.rhow)),
                       __dadd_rn(__dmul_rn(d.y, D.rhoi), __dmul_rn(ld.y, D.rhow)));
  }
  const SlotStep& ss = D.ss[b];
  if (ss.ramp) {
    // second-order placement: the step's increment already carries 1 - phi_k of its response in
    // every mode (solver.py:450-452, 486-499); at degree 2 the rotational states likewise
    const double* omphi = ss.ramp_tab;
    double2* R = D.R + (size_t)b * D.K * D.ncoef;
    const int nk = D.nmod[(size_t)b * D.nl + l];
    for (int k = 0; k < nk; ++k) {
      const double w = omphi[(size_t)k * D.nl + l];
      const double2 r = R[(size_t)k * D.ncoef + i];
      R[(size_t)k * D.ncoef + i] = make_double2(__dadd_rn(r.x, __dmul_rn(w, cur.x)), __dadd_rn(r.y, __dmul_rn(w, cur.y)));
    }
    if (i == 0 && D.tpw && D.nl > 2) {
      const int n2 = D.nmod[(size_t)b * D.nl + 2];
      double* r_il = D.r_il + (size_t)b * D.K * 9;
      double* r_m = D.r_m + (size_t)b * D.K * 3;
      double* r_lam = D.r_lam + (size_t)b * D.K * 6;
      for (int k = 0; k < n2; ++k) {
        const double c = omphi[(size_t)k * D.nl + 2];
        for (int q = 0; q < 9; ++q) r_il[k * 9 + q] = __dadd_rn(r_il[k * 9 + q], __dmul_rn(c, sc->dil[q]));
        for (int q = 0; q < 3; ++q) r_m[k * 3 + q] = __dadd_rn(r_m[k * 3 + q], __dmul_rn(c, sc->dm[q]));
        for (int q = 0; q < 6; ++q) r_lam[k * 6 + q] = __dadd_rn(r_lam[k * 6 + q], __dmul_rn(c, sc->dlam_cur2[q]));
      }
    }
  }
  double2* p_load = D.sp(S_P_LOAD, b);
  const double2 p = p_load[i];
  p_load[i] = make_double2(__dadd_rn(p.x, cur.x), __dadd_rn(p.y, cur.y));
  D.sp(S_P_ICE, b)[i] = D.sp(S_DI, b)[i];
  {
    // dS_cur of the converged iteration: dS_prev + its load increment, as the update forms it
    const double2 po = D.sp(S_P_OCEAN, b)[i];
    D.sp(S_P_OCEAN, b)[i] = make_double2(__dadd_rn(po.x, ld.x), __dadd_rn(po.y, ld.y));
  }
  D.sp(S_PREV_ICE, b)[i] = D.sp(S_ICELM, b)[i];
  if (extrap) D.sp(D.ss[b].hsel ? S_HA : S_HB, b)[i] = ld;
  if (D.ss[b].rec_ds) D.ss[b].rec_ds[i] = ld;
}

// Post-step topography / ocean function (solver.py:1099-1101) and, for the diag option, the
// row sums of the four degree-0 diagnostics (solver_opt.py:893-916): block per row; the slot's
// last block forms U00 = sum_j P~_00 w_j rowsum_j / (nlon 1.41421356), P~_00 = sqrt(0.5).
// Without diag the three diagnostic grids are written for full analyses instead.
__global__ void k_post_grid(Dev D, int diag) {
  SLOT_OR_RETURN();
  __shared__ double sh[32];
  const int j = blockIdx.x;
  if (sc->status) return;
  double a = 0.0, bs = 0.0, c = 0.0, d = 0.0;
  const long long row = (long long)j * (D.nlon / 2);
  const double *deltasl = D.g(G_DELTASL, b), *tinit = D.g(G_TINIT, b);
  const unsigned char* beta = D.m(M_BETA, b);
  double *topo = D.g(G_TOPO, b), *topo_prev = D.g(G_TOPO_PREV, b);
  unsigned char* cxy = D.m(M_CXY, b);
  double *slc = D.g(G_TMP, b), *slcb = D.g(G_TMP3, b), *cstar = D.g(G_TMP4, b);
  unsigned char* rec_mask = D.ss[b].rec_mask;
  for (int t = threadIdx.x; t < D.nlon / 2; t += blockDim.x) {
    const long long h = row + t;
    const double2 ds = ld2(deltasl, h), ti = ld2(tinit, h);
    const uchar2 bb = ldm2(beta, h);
    const double dsv[2] = {ds.x, ds.y}, tiv[2] = {ti.x, ti.y}, bv[2] = {bb.x ? 1.0 : 0.0, bb.y ? 1.0 : 0.0};
    double tp[2], o[2], s1[2], s2[2], cs[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      tp[u] = __dsub_rn(tiv[u], dsv[u]);
      o[u] = (tp[u] < 0.0) ? 1.0 : 0.0;
      s1[u] = __dmul_rn(dsv[u], o[u]);
      s2[u] = __dmul_rn(s1[u], bv[u]);
      cs[u] = __dmul_rn(o[u], bv[u]);
      a += s1[u];
      bs += o[u];
      c += s2[u];
      d += cs[u];
    }
    st2(topo, h, tp[0], tp[1]);
    st2(topo_prev, h, tp[0], tp[1]);
    stm2(cxy, h, o[0] != 0.0, o[1] != 0.0);
    if (rec_mask) {
      rec_mask[2 * h] = o[0] != 0.0;
      rec_mask[2 * h + 1] = o[1] != 0.0;
    }
    if (!diag) {
      st2(slc, h, s1[0], s1[1]);
      st2(slcb, h, s2[0], s2[1]);
      st2(cstar, h, cs[0], cs[1]);
    }
  }
  if (!diag) return;
  double* rows = D.rows + (size_t)b * 4 * D.nlat;
  a = block_sum(a, sh);
  bs = block_sum(bs, sh);
  c = block_sum(c, sh);
  d = block_sum(d, sh);
  if (threadIdx.x == 0) {
    rows[j] = a;
    rows[D.nlat + j] = bs;
    rows[2 * D.nlat + j] = c;
    rows[3 * D.nlat + j] = d;
  }
  if (!last_block(D.counter + 4 * b + 3)) return;
  for (int q = 0; q < 4; ++q) {
    double acc = 0.0;
    for (int jj = threadIdx.x; jj < D.nlat; jj += blockDim.x) acc += D.w[jj] * ((volatile double*)rows)[q * D.nlat + jj];
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) sc->diag[q] = sqrt(0.5) * acc / (double)D.nlon / SQRT2_LEGACY;
    __syncthreads();
  }
}

// Without the diag option: the (0,0) coefficients of the four diagnostic analyses
__global__ void k_diag00(Dev D) {
  const int b = D.slot0 + (int)blockIdx.x;
  Scal* sc = D.sc + b;
  if (sc->done || sc->status || threadIdx.x != 0) return;
  sc->diag[0] = D.sp(S_SP0, b)[0].x;
  sc->diag[1] = D.sp(S_SP1, b)[0].x;
  sc->diag[2] = D.sp(S_SP2, b)[0].x;
  sc->diag[3] = D.sp(S_SP3, b)[0].x;
}

__global__ void k_grid_add(long long n, const double* a, const double* c, double* out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = __dadd_rn(a[i], c[i]);
}

__global__ void k_init_grid(Dev D, int b) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= D.ng) return;
  const double t = D.g(G_TINIT, b)[i];
  const bool c = t < 0.0;
  D.m(M_CXY0, b)[i] = c;
  D.m(M_CXY, b)[i] = c;
  D.g(G_TOPO_PREV, b)[i] = t;
  const double v = D.g(G_ICE_PREV, b)[i];
  const bool keep = !D.checkmarine || icestar_keep(v, t, D.rhow, D.rhoi);
  const double gg = keep ? v : __dmul_rn(v, 0.0);
  D.m(M_GR, b)[i] = keep;
  const bool bt = gg < EPS0;
  D.m(M_BETA0, b)[i] = bt;
  D.m(M_CSTAR0, b)[i] = c && bt;
}

// FP64 grid of a mask (0/1) or of I* = keep ? ice : ice * 0, for the getters.
__global__ void k_mask_grid(long long n, const unsigned char* m, const double* ice, double* out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = ice ? (m[i] ? ice[i] : __dmul_rn(ice[i], 0.0)) : (m[i] ? 1.0 : 0.0);
}

__global__ void k_finite(long long n, const double* a, unsigned int* bad) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && !isfinite(a[i])) atomicOr(bad, 1u);
}

// Slot record after loading: not stepping, K00 of the grid.
__global__ void k_slot_reset(Dev D, int b, double K00) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  Scal* sc = D.sc + b;
  memset(sc, 0, sizeof(Scal));
  sc->K00 = K00;
  sc->converged = 1;
  sc->done = 1;
}

}  // namespace sle

// ============================================================================ handle
using namespace sle;

namespace {

struct SlotHost {
  int loaded, inited;
  // reuse store (device): [capacity][ncoef] increments and [capacity][ng] masks; the first
  // `valid` steps hold entries of an earlier pass
  double2* rs_ds;
  unsigned char* rs_mask;
  int rs_cap, rs_valid;
  int iter, nhist, hsel;
  double dt, dt_cur, dt_hist[2];
  double ocean_area0, oceanBeta_area0, ice_volume0;
  sle_step_info last;
};

}  // namespace

struct sle_batch {
  sle_config cfg;
  int nslot, K;
  sle_sht* plan;
  cudaStream_t st;
  Dev D;
  // device allocations
  double* grid;
  unsigned char* mask;
  double2 *spec, *R;
  int* nmod;
  double *s_kl, *decay, *omd, *a_sl, *a_rr, *ttl, *ttlekhl, *ttlhe, *a_il, *a_m, *a_tsl, *a_trr;
  RotConst* rc;
  double *r_il, *r_m, *r_lam;
  Scal* sc;
  SlotStep* ss;
  double* partials;
  unsigned int* counter;
  double* rows;
  unsigned int* badflag;
  int* bstatus;            // batch-wide status raised by a tensor-core timeout
  // analytic rates read-out (opt-in per slot): rate spectra [nslot][2][ncoef] (sea level, radial),
  // weight tables [nslot][2 K nl + 4 nl] (w_sl, w_rr, ws_sl, ws_rr, wsphi_sl, wsphi_rr) and a
  // record [nslot][2] (dI*_00 of the step)
  double2* rate_spec;
  double* rate_tab;
  double* rate_rec;
  double* rate_rot;   // [nslot][18 K]: the degree-2 modal states before the commit
  std::vector<char> rates_on;
  // horizontal read-out (opt-in per slot): potential spectra [nslot][ncoef], weights
  // [nslot][K nl + nl] (a_hl = l_k / s_k, then ttl l^E)
  double2* horiz_spec;
  double* horiz_tab;
  std::vector<char> horiz_on;
  // ramp placement (opt-in per slot): tables [nslot][(K + 2) nl] and the degree-2 weights
  double* ramp_tab;
  std::vector<char> ramp_on;
  std::vector<double> ramp_c;   // [nslot][4]
  // pinned mirrors
  Scal* hsc;
  SlotStep* hss;
  std::vector<SlotHost> slot;
  double K00;
  // inner loop as a CUDA graph with a device-evaluated WHILE condition
  cudaGraph_t loop_graph;
  cudaGraphExec_t loop_exec;
  int use_graph;
  // a step enqueued by batch_step_begin and not yet finished by batch_step_end
  bool pending = false;
  bool pending_graph = false;
  std::vector<int> pending_act;
  long long body_launches;   // kernels in one iteration of the graph body
  int iter_active = 0;       // host-driven loop: stepping slots not yet converged (timing units)
  // static field lists of the loop body
  std::vector<FieldSpec> f_syn_sl, f_ana_ro, f_syn_sltot, f_ana_refresh, f_ana_regr;
};

struct sle_solver {
  sle_batch* b;
};

namespace {

template <typename T>
int dalloc(T** p, size_t n) {
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), (n ? n : 1) * sizeof(T));
  if (e != cudaSuccess) {
    set_error("cudaMalloc(%zu bytes) failed: %s", n * sizeof(T), cudaGetErrorString(e));
    *p = nullptr;
    return SLE_ERR_OOM;
  }
  return SLE_OK;
}

inline unsigned nb(long long n, int bs = 256) { return (unsigned)((n + bs - 1) / bs); }

void batch_free(sle_batch* s) {
  if (!s) return;
  void* ptrs[] = {s->grid, s->mask, s->spec, s->R, s->nmod, s->s_kl, s->decay, s->omd, s->a_sl, s->a_rr, s->ttl,
                  s->ttlekhl, s->ttlhe, s->a_il, s->a_m, s->a_tsl, s->a_trr, s->rc, s->r_il, s->r_m,
                  s->r_lam, s->sc, s->ss, s->partials, s->counter, s->rows, s->badflag, s->bstatus,
                  s->rate_spec, s->rate_tab, s->rate_rec, s->rate_rot, s->horiz_spec, s->horiz_tab, s->ramp_tab};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  if (s->hsc) cudaFreeHost(s->hsc);
  if (s->hss) cudaFreeHost(s->hss);
  if (s->loop_exec) cudaGraphExecDestroy(s->loop_exec);
  if (s->loop_graph) cudaGraphDestroy(s->loop_graph);
  if (s->st) cudaStreamDestroy(s->st);
  if (s->plan) sle_sht_destroy(s->plan);
  delete s;
}

int upload(void* dst, const void* src, size_t bytes, int on_device, cudaStream_t st) {
  SLE_CUDA(cudaMemcpyAsync(dst, src, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  return SLE_OK;
}

int sync_scal(sle_batch* s) {
  SLE_CUDA(cudaMemcpyAsync(s->hsc, s->sc, sizeof(Scal) * s->nslot, cudaMemcpyDeviceToHost, s->st));
  SLE_CUDA(cudaStreamSynchronize(s->st));
  return SLE_OK;
}

int check_finite(sle_batch* s, const double* dev, long long n, const char* what) {
  SLE_CUDA(cudaMemsetAsync(s->badflag, 0, sizeof(unsigned int), s->st));
  note_launch();
  k_finite<<<nb(n), 256, 0, s->st>>>(n, dev, s->badflag);
  unsigned int bad = 0;
  SLE_CUDA(cudaMemcpyAsync(&bad, s->badflag, sizeof(unsigned int), cudaMemcpyDeviceToHost, s->st));
  SLE_CUDA(cudaStreamSynchronize(s->st));
  if (bad) {
    set_error("%s contains NaN or Inf", what);
    return SLE_ERR_NONFINITE;
  }
  return SLE_OK;
}

int set_dt(sle_batch* s, int b, double dt) {
  SlotHost& h = s->slot[b];
  if (dt == h.dt_cur) return SLE_OK;
  note_launch();
  k_set_decay<<<nb((long long)s->K * s->D.nl), 256, 0, s->st>>>(s->D, b, dt);
  SLE_CUDA(cudaGetLastError());
  h.dt_cur = dt;
  return SLE_OK;
}

FieldSpec fspec(double* grid, double2* spec, const int* skip_set = nullptr, const int* skip_clear = nullptr,
                double* epi_out = nullptr, const double* epi_mul = nullptr) {
  return FieldSpec{grid, spec, skip_set, skip_clear, epi_out, epi_mul, SRC_GRID, nullptr, nullptr};
}
// analysis inputs formed from masks (SrcKind): a 0/1 mask, ice on its keep mask, T0 (C* - C*0),
// a grid times a mask
FieldSpec fmask(const unsigned char* m, double2* spec, const int* skip_set = nullptr,
                const int* skip_clear = nullptr) {
  return FieldSpec{nullptr, spec, skip_set, skip_clear, nullptr, nullptr, SRC_MASK, m, nullptr};
}
FieldSpec fice(double* ice, const unsigned char* keep, double2* spec, const int* skip_set = nullptr,
               const int* skip_clear = nullptr) {
  return FieldSpec{ice, spec, skip_set, skip_clear, nullptr, nullptr, SRC_ICE, keep, nullptr};
}
FieldSpec fto(double* tinit, const unsigned char* cstar, const unsigned char* cstar0, double2* spec,
              const int* skip_set = nullptr, const int* skip_clear = nullptr) {
  return FieldSpec{tinit, spec, skip_set, skip_clear, nullptr, nullptr, SRC_TO, cstar, cstar0};
}
FieldSpec fprod(double* grid, const unsigned char* m, double2* spec, const int* skip_set = nullptr,
                const int* skip_clear = nullptr) {
  return FieldSpec{grid, spec, skip_set, skip_clear, nullptr, nullptr, SRC_PROD, m, nullptr};
}

double fourpiR2(const sle_batch* s, double x) {
  // x * 4 * PI * radius**2 with the reference's left-to-right association
  return ((x * 4.0) * PI_LEGACY) * std::pow(s->cfg.radius, 2);
}

// One inner iteration (solver.py:909-1045) for every slot as a fixed kernel sequence: every
// decision is read on the device, so the same sequence serves the host-driven loop and the
// graph body.
int enqueue_iteration(sle_batch* s, cudaGraphConditionalHandle loop) {
  const Dev& D = s->D;
  cudaStream_t st = s->st;
  const long long nc = D.ncoef, ng = D.ng;
  const unsigned B = (unsigned)s->nslot;
  const double act = (double)s->iter_active;   // per-class timing units: slots still iterating
  note_launch();
  ProfToken t = prof_begin(PROF_B18, act, st);
  // mixed precision with the dsl identity (the spectrum has no other reader) and the synthesis
  // one launch (field b = slot b): B18 writes the synthesis B operand itself
  const int nsyn = (int)s->f_syn_sl.size();
  const bool fuse = s->cfg.precision == SLE_PREC_MIXED && s->cfg.opt_dsl && s->plan->mx_ready &&
                    nsyn <= std::min(MX_MAXF, s->plan->tune_fpl);
  k_b18<<<dim3(nb(nc), B), 256, 0, st>>>(D, fuse ? s->plan->mx_bsyn : nullptr, fuse ? s->plan->mx_bpos : nullptr);
  prof_end(t, st);
  SLE_TRY(sht_synthesis_list(s->plan, s->f_syn_sl.data(), nsyn, st, fuse));
  SLE_TRY(sht_analysis_list(s->plan, s->f_ana_ro.data(), (int)s->f_ana_ro.size(), st, PROF_ANA_STEP));
  note_launch();
  t = prof_begin(PROF_UPDATE, act, st);
  SLE_CUDA(launch_pdl(k_update, dim3(nb(nc), B), dim3(256), 0, st, D));
  prof_end(t, st);
  if (!s->cfg.opt_dsl) {
    note_launch();
    k_sltot<<<dim3(nb(nc), B), 256, 0, st>>>(D);
    SLE_TRY(sht_synthesis_list(s->plan, s->f_syn_sltot.data(), (int)s->f_syn_sltot.size(), st));
  }
  note_launch(2);
  t = prof_begin(PROF_REFRESH1, act, st);
  SLE_CUDA(launch_pdl(k_refresh1, dim3(nb(ng / 2), B), dim3(256), 0, st, D));
  prof_end(t, st);
  t = prof_begin(PROF_REFRESH2, act, st);
  if (ng % 8 == 0) SLE_CUDA(launch_pdl(k_refresh2_x8, dim3(nb(ng / 8), B), dim3(256), 0, st, D));
  else SLE_CUDA(launch_pdl(k_refresh2, dim3(nb(ng / 2), B), dim3(256), 0, st, D));
  prof_end(t, st);
  // C* and tO (when a cell of C* flipped), I* (when the grounded mask changed) for the next
  // iteration; skipped for slots that converged
  SLE_TRY(sht_analysis_list(s->plan, s->f_ana_refresh.data(), (int)s->f_ana_refresh.size(), st));
  SLE_TRY(sht_analysis_list(s->plan, s->f_ana_regr.data(), (int)s->f_ana_regr.size(), st));
  note_launch(2);
  t = prof_begin(PROF_DICE, act, st);
  SLE_CUDA(launch_pdl(k_dice, dim3(std::min(nb(nc), (unsigned)DICE_BLOCKS), B), dim3(256), 0, st, D));
  prof_end(t, st);
  k_loop_cond<<<1, 128, 0, st>>>(D, s->bstatus, loop);
  SLE_CUDA(cudaGetLastError());
  return SLE_OK;
}

int build_loop_graph(sle_batch* s) {
  cudaGraph_t g = nullptr;
  SLE_CUDA(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle h;
  cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 1u, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    set_error("cudaGraphConditionalHandleCreate: %s", cudaGetErrorString(e));
    return SLE_ERR_CUDA;
  }
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  e = cudaGraphAddNode(&node, g, nullptr, 0, &np);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    set_error("cudaGraphAddNode(conditional): %s", cudaGetErrorString(e));
    return SLE_ERR_CUDA;
  }
  cudaGraph_t body = np.conditional.phGraph_out[0];
  e = cudaStreamBeginCaptureToGraph(s->st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    set_error("cudaStreamBeginCaptureToGraph: %s", cudaGetErrorString(e));
    return SLE_ERR_CUDA;
  }
  const long long before = sle_launch_count();
  const int rc = enqueue_iteration(s, h);
  s->body_launches = sle_launch_count() - before;
  note_launch(-(int)s->body_launches);  // counted per executed iteration at the end of each step
  cudaGraph_t captured = nullptr;
  e = cudaStreamEndCapture(s->st, &captured);
  if (rc != SLE_OK || e != cudaSuccess) {
    cudaGraphDestroy(g);
    if (rc != SLE_OK) return rc;
    set_error("cudaStreamEndCapture: %s", cudaGetErrorString(e));
    return SLE_ERR_CUDA;
  }
  cudaGraphExec_t ex = nullptr;
  e = cudaGraphInstantiate(&ex, g, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    set_error("cudaGraphInstantiate: %s", cudaGetErrorString(e));
    return SLE_ERR_CUDA;
  }
  s->loop_graph = g;
  s->loop_exec = ex;
  return SLE_OK;
}

int check_slot(const sle_batch* s, int slot, const char* what) {
  if (s->pending) {
    set_error("%s: a step is in flight (end it with sle_batch_step_end first)", what);
    return SLE_ERR_STATE;
  }
  if (slot < 0 || slot >= s->nslot) {
    set_error("%s: slot %d outside 0..%d", what, slot, s->nslot - 1);
    return SLE_ERR_BAD_ARG;
  }
  return SLE_OK;
}

// Earth model of one slot: arrays, per-slot rotation constants, decay for dt.
int set_earth(sle_batch* s, int b, const sle_earth* earth, double dt) {
  const int nl = s->D.nl, K = s->K;
  if (!earth) {
    set_error("sle_batch_load: NULL earth");
    return SLE_ERR_BAD_ARG;
  }
  if (earth->nmodes < 0 || earth->nmodes > K) {
    set_error("sle_batch_load: %d modes, the batch holds at most %d", earth->nmodes, K);
    return SLE_ERR_BAD_ARG;
  }
  const int Ke = earth->nmodes;
  std::vector<int> nm(earth->nmod, earth->nmod + nl);
  for (int l = 0; l < nl; ++l) {
    if (nm[l] < 0 || nm[l] > Ke) {
      set_error("sle_batch_load: nmod[%d]=%d outside 0..%d", l, nm[l], Ke);
      return SLE_ERR_BAD_ARG;
    }
  }
  if (nl > 2 && nm[2] > 64) {
    set_error("sle_batch_load: %d relaxation modes at degree 2 (at most 64 supported)", nm[2]);
    return SLE_ERR_UNSUPPORTED;
  }
  // [K][nl] arrays padded from the slot's Ke modes to the batch's K
  std::vector<double> sk((size_t)K * nl, 0.0), asl((size_t)K * nl, 0.0), arr((size_t)K * nl, 0.0);
  std::copy(earth->s, earth->s + (size_t)Ke * nl, sk.begin());
  std::copy(earth->a_sl, earth->a_sl + (size_t)Ke * nl, asl.begin());
  std::copy(earth->a_rr, earth->a_rr + (size_t)Ke * nl, arr.begin());
  std::vector<double> ail(K, 0.0), am(K, 0.0), atsl(K, 0.0), atrr(K, 0.0);
  if (Ke > 0) {
    std::copy(earth->a_il, earth->a_il + Ke, ail.begin());
    std::copy(earth->a_m, earth->a_m + Ke, am.begin());
    std::copy(earth->a_tsl, earth->a_tsl + Ke, atsl.begin());
    std::copy(earth->a_trr, earth->a_trr + Ke, atrr.begin());
  }
  const size_t o = s->D.kl(b);
  cudaStream_t st = s->st;
  SLE_CUDA(cudaMemcpyAsync(s->s_kl + o, sk.data(), sizeof(double) * K * nl, cudaMemcpyHostToDevice, st));
  SLE_CUDA(cudaMemcpyAsync(s->a_sl + o, asl.data(), sizeof(double) * K * nl, cudaMemcpyHostToDevice, st));
  SLE_CUDA(cudaMemcpyAsync(s->a_rr + o, arr.data(), sizeof(double) * K * nl, cudaMemcpyHostToDevice, st));
  SLE_CUDA(cudaMemcpyAsync(s->ttl + (size_t)b * nl, earth->ttl, sizeof(double) * nl, cudaMemcpyHostToDevice, st));
  SLE_CUDA(cudaMemcpyAsync(s->ttlekhl + (size_t)b * nl, earth->ttlekhl, sizeof(double) * nl, cudaMemcpyHostToDevice, st));
  SLE_CUDA(cudaMemcpyAsync(s->ttlhe + (size_t)b * nl, earth->ttlhe, sizeof(double) * nl, cudaMemcpyHostToDevice, st));
  SLE_CUDA(cudaMemcpyAsync(s->a_il + (size_t)b * K, ail.data(), sizeof(double) * K, cudaMemcpyHostToDevice, st));
  SLE_CUDA(cudaMemcpyAsync(s->a_m + (size_t)b * K, am.data(), sizeof(double) * K, cudaMemcpyHostToDevice, st));
  SLE_CUDA(cudaMemcpyAsync(s->a_tsl + (size_t)b * K, atsl.data(), sizeof(double) * K, cudaMemcpyHostToDevice, st));
  SLE_CUDA(cudaMemcpyAsync(s->a_trr + (size_t)b * K, atrr.data(), sizeof(double) * K, cudaMemcpyHostToDevice, st));
  SLE_CUDA(cudaMemcpyAsync(s->nmod + (size_t)b * nl, nm.data(), sizeof(int) * nl, cudaMemcpyHostToDevice, st));
  // rotation constants (solver.py:910-975), same expressions as the reference
  const sle_config* cfg = &s->cfg;
  RotConst C;
  const double a4 = std::pow(cfg->radius, 4);
  C.c_il22 = (-8 * PI_LEGACY * a4) / (3 * std::sqrt(5.0));
  C.c_il02 = (-8 * PI_LEGACY * a4) / std::sqrt(30.0);
  C.c_il12 = (8 * PI_LEGACY * a4) / std::sqrt(30.0);
  C.alpha = 1 / (1 - earth->kTE2 / cfg->kf);
  C.inv_CmA = 1 / (cfg->moiC - cfg->moiA);
  C.inv_kf = 1 / cfg->kf;
  C.kf = cfg->kf;
  C.inv_C = 1.0 / cfg->moiC;
  C.onepk = 1 + earth->kE2;
  const double r2w2 = std::pow(cfg->radius, 2) * std::pow(cfg->omega, 2);
  C.r2w2_3 = r2w2 / 3.0;
  C.r2w2_6s5 = r2w2 / (6.0 * std::sqrt(5.0));
  C.r2w2_s30 = r2w2 / std::sqrt(30.0);
  C.r2w2_s120 = r2w2 / std::sqrt(5.0 * 24.0);
  C.ekhTE = 1 + earth->kTE2 - earth->hTE2;
  C.hTE2 = earth->hTE2;
  C.gacc = cfg->gacc;
  C.rhoi = cfg->rhoi;
  C.rhow = cfg->rhow;
  SLE_CUDA(cudaMemcpyAsync(s->rc + b, &C, sizeof(RotConst), cudaMemcpyHostToDevice, st));
  SlotHost& h = s->slot[b];
  h.dt = dt;
  h.dt_cur = -1.0;
  SLE_TRY(set_dt(s, b, dt));
  SLE_CUDA(cudaStreamSynchronize(st));
  h.loaded = 1;
  h.inited = 0;
  return SLE_OK;
}

// Step 0 of one slot (solver.py:550-581): masks, areas and volume; zero modal and history state.
int init_slot(sle_batch* s, int b, const double* topo0, const double* ice0, int on_device, double* ocean_area0,
              double* oceanBeta_area0, double* ice_volume0) {
  const Dev& D = s->D;
  const size_t gb = sizeof(double) * D.ng;
  cudaStream_t st = s->st;
  SlotHost& h = s->slot[b];
  if (!h.loaded) {
    set_error("slot %d has no Earth model", b);
    return SLE_ERR_STATE;
  }
  SLE_TRY(upload(D.g(G_TINIT, b), topo0, gb, on_device, st));
  SLE_TRY(upload(D.g(G_ICE_PREV, b), ice0, gb, on_device, st));
  SLE_TRY(check_finite(s, D.g(G_TINIT, b), D.ng, "topography"));
  SLE_TRY(check_finite(s, D.g(G_ICE_PREV, b), D.ng, "initial ice"));
  note_launch();
  k_init_grid<<<nb(D.ng), 256, 0, st>>>(D, b);
  SLE_CUDA(cudaGetLastError());
  // step-0 areas and volume from full analyses (solver.py:571-581)
  const FieldSpec f3[3] = {fmask(D.m(M_CXY0, b), D.sp(S_SP0, b)), fmask(D.m(M_CSTAR0, b), D.sp(S_SP1, b)),
                           fice(D.g(G_ICE_PREV, b), D.m(M_GR, b), D.sp(S_SP2, b))};
  SLE_TRY(sht_analysis_list(s->plan, f3, 3, st));
  double2 v[3];
  SLE_CUDA(cudaMemcpyAsync(&v[0], D.sp(S_SP0, b), sizeof(double2), cudaMemcpyDeviceToHost, st));
  SLE_CUDA(cudaMemcpyAsync(&v[1], D.sp(S_SP1, b), sizeof(double2), cudaMemcpyDeviceToHost, st));
  SLE_CUDA(cudaMemcpyAsync(&v[2], D.sp(S_SP2, b), sizeof(double2), cudaMemcpyDeviceToHost, st));
  // modal, rotational and history state start at zero
  const long long nc = D.ncoef;
  SLE_CUDA(cudaMemsetAsync(D.R + (size_t)b * s->K * nc, 0, sizeof(double2) * s->K * nc, st));
  const int zero_specs[] = {S_P_LOAD, S_P_ICE, S_P_OCEAN, S_PREV_ICE, S_HA, S_HB};
  for (int z : zero_specs) SLE_CUDA(cudaMemsetAsync(D.sp(z, b), 0, sizeof(double2) * nc, st));
  const size_t K = s->K ? s->K : 1;
  SLE_CUDA(cudaMemsetAsync(s->r_il + (size_t)b * s->K * 9, 0, sizeof(double) * 9 * K, st));
  SLE_CUDA(cudaMemsetAsync(s->r_m + (size_t)b * s->K * 3, 0, sizeof(double) * 3 * K, st));
  SLE_CUDA(cudaMemsetAsync(s->r_lam + (size_t)b * s->K * 6, 0, sizeof(double) * 6 * K, st));
  note_launch();
  k_slot_reset<<<1, 32, 0, st>>>(D, b, s->K00);
  SLE_CUDA(cudaGetLastError());
  SLE_CUDA(cudaStreamSynchronize(st));
  h.ocean_area0 = fourpiR2(s, v[0].x);
  h.oceanBeta_area0 = fourpiR2(s, v[1].x);
  h.ice_volume0 = fourpiR2(s, v[2].x);
  if (ocean_area0) *ocean_area0 = h.ocean_area0;
  if (oceanBeta_area0) *oceanBeta_area0 = h.oceanBeta_area0;
  if (ice_volume0) *ice_volume0 = h.ice_volume0;
  h.iter = 0;
  h.nhist = 0;
  h.hsel = 0;
  h.dt_hist[0] = h.dt_hist[1] = h.dt;
  h.inited = 1;
  std::memset(&h.last, 0, sizeof(h.last));
  return SLE_OK;
}

int batch_create(const sle_config* cfg, int nslot, int kmax, sle_batch** out) {
  if (!cfg || !out) {
    set_error("sle_batch_create: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  *out = nullptr;
  if (nslot < 1 || nslot > 4096) {
    set_error("sle_batch_create: nslots must be 1..4096 (got %d)", nslot);
    return SLE_ERR_BAD_ARG;
  }
  if (kmax < 0 || kmax > 4096) {
    set_error("sle_batch_create: max_modes out of range");
    return SLE_ERR_BAD_ARG;
  }
  if (cfg->precision != SLE_PREC_FP64 && cfg->precision != SLE_PREC_MIXED) {
    set_error("sle_batch_create: unknown precision %d", cfg->precision);
    return SLE_ERR_BAD_ARG;
  }
  sle_batch* s = new sle_batch();
  s->cfg = *cfg;
  s->nslot = nslot;
  s->K = kmax;
  int rc = sle_sht_create(cfg->nlat, cfg->nlon, cfg->lmax, &s->plan);
  if (rc != SLE_OK) {
    delete s;
    return rc;
  }
#define TRY(x)                \
  do {                        \
    rc = (x);                 \
    if (rc != SLE_OK) {       \
      batch_free(s);          \
      return rc;              \
    }                         \
  } while (0)
#define TRYC(x)                                                                       \
  do {                                                                                \
    cudaError_t e_ = (x);                                                             \
    if (e_ != cudaSuccess) {                                                          \
      set_error("%s failed: %s", #x, cudaGetErrorString(e_));                          \
      batch_free(s);                                                                  \
      return SLE_ERR_CUDA;                                                            \
    }                                                                                 \
  } while (0)
  TRYC(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
  const int nl = cfg->lmax + 1;
  const long long ng = (long long)cfg->nlat * cfg->nlon;
  const long long nc = s->plan->d.ncoef;
  const int K = kmax;
  const size_t B = (size_t)nslot;
  TRY(dalloc(&s->grid, (size_t)NGRID * B * ng));
  TRY(dalloc(&s->mask, (size_t)NMASK * B * ng));
  TRY(dalloc(&s->spec, (size_t)NSPEC * B * nc));
  TRY(dalloc(&s->R, B * K * nc + 1));
  TRY(dalloc(&s->nmod, B * nl));
  double** kl_arrays[] = {&s->s_kl, &s->decay, &s->omd, &s->a_sl, &s->a_rr};
  for (double** p : kl_arrays) TRY(dalloc(p, B * K * nl + 1));
  double** l_arrays[] = {&s->ttl, &s->ttlekhl, &s->ttlhe};
  for (double** p : l_arrays) TRY(dalloc(p, B * nl));
  double** k_arrays[] = {&s->a_il, &s->a_m, &s->a_tsl, &s->a_trr};
  for (double** p : k_arrays) TRY(dalloc(p, B * K + 1));
  TRY(dalloc(&s->rc, B));
  TRY(dalloc(&s->r_il, B * K * 9 + 1));
  TRY(dalloc(&s->r_m, B * K * 3 + 1));
  TRY(dalloc(&s->r_lam, B * K * 6 + 1));
  TRY(dalloc(&s->sc, B));
  TRY(dalloc(&s->ss, B));
  const long long part_grid = (long long)nb(nc) + 32;
  const long long npart = part_grid + nb(ng / 2) + 64;
  TRY(dalloc(&s->partials, B * npart));
  TRY(dalloc(&s->counter, B * 4));
  TRY(dalloc(&s->rows, B * 4 * cfg->nlat));
  TRY(dalloc(&s->badflag, 1));
  TRY(dalloc(&s->bstatus, 1));
  TRYC(cudaMallocHost(reinterpret_cast<void**>(&s->hsc), sizeof(Scal) * B));
  TRYC(cudaMallocHost(reinterpret_cast<void**>(&s->hss), sizeof(SlotStep) * B));
  TRYC(cudaMemset(s->counter, 0, sizeof(unsigned int) * 4 * B));
  TRYC(cudaMemset(s->bstatus, 0, sizeof(int)));
  TRYC(cudaMemset(s->sc, 0, sizeof(Scal) * B));
  TRYC(cudaMemset(s->ss, 0, sizeof(SlotStep) * B));
  TRYC(cudaMemset(s->nmod, 0, sizeof(int) * B * nl));
  s->slot.assign(B, SlotHost{});
  if (cfg->precision == SLE_PREC_MIXED) {
    TRY(sle_sht_set_precision(s->plan, SLE_PREC_MIXED));
    s->plan->mx_status = s->bstatus;   // a tensor-core timeout ends the step with SLE_ERR_TIMEOUT
  }
  // device view
  Dev& D = s->D;
  D.nlat = cfg->nlat;
  D.nlon = cfg->nlon;
  D.nl = nl;
  D.nslot = nslot;
  D.K = K;
  D.ng = ng;
  D.ncoef = nc;
  D.lidx = s->plan->d.lidx;
  D.grid = s->grid;
  D.mask = s->mask;
  D.spec = s->spec;
  D.R = s->R;
  {
    int dev = 0, nsm = 0, per_sm = 0;
    TRYC(cudaGetDevice(&dev));
    TRYC(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    TRYC(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_advance, 256, 0));
    D.adv_ahead = per_sm * nsm;
    TRYC(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_update, 256, 0));
    D.upd_ahead = per_sm * nsm;
  }
  D.nmod = s->nmod;
  D.s_kl = s->s_kl;
  D.decay = s->decay;
  D.omd = s->omd;
  D.a_sl = s->a_sl;
  D.a_rr = s->a_rr;
  D.ttl = s->ttl;
  D.ttlekhl = s->ttlekhl;
  D.ttlhe = s->ttlhe;
  D.a_il = s->a_il;
  D.a_m = s->a_m;
  D.a_tsl = s->a_tsl;
  D.a_trr = s->a_trr;
  D.rc = s->rc;
  D.r_il = s->r_il;
  D.r_m = s->r_m;
  D.r_lam = s->r_lam;
  D.sc = s->sc;
  D.ss = s->ss;
  D.partials = s->partials;
  D.npart = npart;
  D.part_grid = part_grid;
  D.counter = s->counter;
  D.rows = s->rows;
  D.w = s->plan->d.w;
  D.rhoi = cfg->rhoi;
  D.rhow = cfg->rhow;
  D.epsilon1 = cfg->epsilon1;
  D.checkmarine = cfg->checkmarine;
  D.tpw = cfg->tpw && nl > 2;
  D.calcRG = cfg->calcRG;
  D.opt_dsl = cfg->opt_dsl;
  D.slot0 = 0;
  const int L = cfg->lmax;
  D.i20 = 2;
  D.i21 = (long long)(L + 1) + 1;
  D.i22 = (long long)2 * (L + 1) - 1 + 0;
  // static field lists of the loop body: every slot, gated by its flags
  for (int b = 0; b < nslot; ++b) {
    Scal* sb = s->sc + b;
    s->f_syn_sl.push_back(fspec(D.g(G_DSL, b), D.sp(S_SL, b), &sb->done));
    s->f_ana_ro.push_back(fprod(D.g(G_DSL, b), D.m(M_CSTAR, b), D.sp(S_ROLM, b), &sb->done));
    s->f_syn_sltot.push_back(fspec(D.g(G_DELTASL, b), D.sp(S_SLTOT, b), &sb->done));
  }
  // Mixed precision: two lists by gate, C* and tO (open when a cell of C* flipped) and I* (open on
  // a grounded-mask change, rare after the first iterations), so that the I* tensor-core launches
  // end at once instead of running for C* / tO fields mixed in with them.  FP64 (four fields per
  // launch, gates checked per block): one list.
  const bool split_gates = cfg->precision == SLE_PREC_MIXED;
  for (int b = 0; b < nslot; ++b) {
    Scal* sb = s->sc + b;
    (split_gates ? s->f_ana_regr : s->f_ana_refresh)
        .push_back(fice(D.g(G_ICE, b), D.m(M_GR, b), D.sp(S_ICELM, b), &sb->converged, &sb->gr_changed));
    s->f_ana_refresh.push_back(fmask(D.m(M_CSTAR, b), D.sp(S_CSTARLM, b), &sb->converged, &sb->cs_changed));
    s->f_ana_refresh.push_back(fto(D.g(G_TINIT, b), D.m(M_CSTAR, b), D.m(M_CSTAR0, b), D.sp(S_TOLM, b),
                                   &sb->converged, &sb->cs_changed));
  }
  // SLEVOLVE_B200_HOST_LOOP=1 drives the inner loop from the host (same kernels; used to profile
  // the loop body, whose kernels profilers do not report inside conditional graph nodes)
  {
    const char* e = std::getenv("SLEVOLVE_B200_HOST_LOOP");
    s->use_graph = !(e && e[0] == '1');
  }
  // K00 = synth(e00)[0,0] (solver_opt.py:320-325): the same for every slot of the grid
  s->K00 = 0.0;
  if (cfg->opt_dsl) {
    double2* e00 = D.sp(S_SP3, 0);
    double* g0 = D.g(G_TMP, 0);
    TRYC(cudaMemset(e00, 0, sizeof(double2) * nc));
    const double2 one = make_double2(1.0, 0.0);
    TRYC(cudaMemcpy(e00, &one, sizeof(double2), cudaMemcpyHostToDevice));
    const FieldSpec f1 = fspec(g0, e00);
    TRY(sht_synthesis_list(s->plan, &f1, 1, s->st));
    TRYC(cudaStreamSynchronize(s->st));
    TRYC(cudaMemcpy(&s->K00, g0, sizeof(double), cudaMemcpyDeviceToHost));
  }
  TRYC(cudaStreamSynchronize(s->st));
  *out = s;
  return SLE_OK;
#undef TRY
#undef TRYC
}

// One time step of the slots with ice[b] != NULL.
// Enqueue one step of the slots with ice[b] != NULL on the batch's stream; batch_step_end waits
// for it and reads the slots' records.
int batch_step_begin(sle_batch* s, const double* const* ice, int on_device, const double* dt_years) {
  if (s->pending) {
    set_error("sle_batch_step_begin: the previous step was not ended");
    return SLE_ERR_STATE;
  }
  const Dev& D = s->D;
  cudaStream_t st = s->st;
  const long long nc = D.ncoef, ng = D.ng;
  const int B = s->nslot;
  std::vector<int> act;
  for (int b = 0; b < B; ++b) {
    if (!ice[b]) continue;
    if (!s->slot[b].inited) {
      set_error("sle_batch_step: slot %d is not initialised", b);
      return SLE_ERR_STATE;
    }
    act.push_back(b);
  }
  s->pending_act = act;
  s->pending_graph = false;
  s->pending = true;
  if (act.empty()) return SLE_OK;
  // per-slot step parameters
  for (int b = 0; b < B; ++b) s->hss[b] = SlotStep{0, 0, 0, 0, 0.0, 0.0, nullptr, nullptr, nullptr, nullptr};
  for (int b : act) {
    SlotHost& h = s->slot[b];
    double dt = h.dt;
    if (dt_years && dt_years[b] > 0.0) {
      dt = dt_years[b];
      h.dt = dt;
    }
    SLE_TRY(set_dt(s, b, dt));
    h.iter += 1;
    SlotStep& p = s->hss[b];
    p.active = 1;
    p.first = h.iter == 1;
    p.hsel = h.hsel;
    p.rates = (b < (int)s->rates_on.size() && s->rates_on[b]) ? 1 : 0;
    p.rate_h = dt;
    p.horiz = (b < (int)s->horiz_on.size() && s->horiz_on[b]) ? 1 : 0;
    p.ramp = (b < (int)s->ramp_on.size() && s->ramp_on[b]) ? 1 : 0;
    if (p.ramp) {
      p.ramp_tab = s->ramp_tab + (size_t)b * (s->K + 2) * s->D.nl;
      p.c_il = s->ramp_c[4 * b];
      p.c_m = s->ramp_c[4 * b + 1];
      p.c_tsl = s->ramp_c[4 * b + 2];
      p.c_trr = s->ramp_c[4 * b + 3];
    }
    if (s->cfg.inner_extrap && h.nhist >= 2) {
      const double dt0 = dt, dt1 = h.dt_hist[0], dt2 = h.dt_hist[1];
      if (dt0 == dt1 && dt1 == dt2) {
        p.mode = 1;
      } else {
        p.mode = 2;
        const double w = (dt0 + dt1) / (dt1 + dt2);
        p.c1 = dt0 / dt1 * (1.0 + w);
        p.c2 = dt0 / dt2 * w;
      }
    }
    if (h.rs_ds && h.iter <= h.rs_cap) {
      const size_t e = (size_t)(h.iter - 1);
      p.rec_ds = h.rs_ds + e * nc;
      p.rec_mask = h.rs_mask + e * ng;
      if (h.iter <= h.rs_valid) {
        p.warm_ds = p.rec_ds;
        p.warm_mask = p.rec_mask;
      }
    }
    SLE_TRY(upload(D.g(G_ICE, b), ice[b], sizeof(double) * ng, on_device, st));
  }
  SLE_CUDA(cudaMemcpyAsync(s->ss, s->hss, sizeof(SlotStep) * B, cudaMemcpyHostToDevice, st));
  SLE_CUDA(cudaMemsetAsync(s->bstatus, 0, sizeof(int), st));
  const unsigned UB = (unsigned)B;
  note_launch(3);
  k_step_begin<<<nb(B, 128), 128, 0, st>>>(D);
  // ---- modal advance (solver.py:835)
  ProfToken tadv = prof_begin(PROF_ADVANCE, (double)act.size(), st);
  k_advance<<<dim3(nb(nc) + 1, UB), 256, 0, st>>>(D);
  prof_end(tadv, st);
  // ---- ice and ocean grids, their analyses (the stepping slots only)
  k_ice_grid<<<dim3(nb(ng / 2), UB), 256, 0, st>>>(D);
  SLE_CUDA(cudaGetLastError());
  {
    std::vector<FieldSpec> f;
    for (int b : act) {
      f.push_back(fice(D.g(G_ICE, b), D.m(M_GR, b), D.sp(S_ICELM, b)));
      f.push_back(fmask(D.m(M_CSTAR, b), D.sp(S_CSTARLM, b)));
      f.push_back(fto(D.g(G_TINIT, b), D.m(M_CSTAR, b), D.m(M_CSTAR0, b), D.sp(S_TOLM, b)));
      if (s->hss[b].first) f.push_back(fspec(D.g(G_TMP, b), D.sp(S_OLDICE, b)));
    }
    SLE_TRY(sht_analysis_list(s->plan, f.data(), (int)f.size(), st));
  }
  // ---- first guess
  note_launch(2);
  k_pre_spec<<<dim3(nb(nc), UB), 256, 0, st>>>(D);
  k_rotation<<<1, 128, 0, st>>>(D);
  SLE_CUDA(cudaGetLastError());

  // ---- inner fixed-point loop (solver.py:907-1051): a CUDA graph whose WHILE condition is set
  // at the end of each iteration (any slot unconverged); with per-kernel profiling on, the same
  // sequence is driven from the host.
  const bool graph_step = s->use_graph && !prof_enabled();
  s->pending_graph = graph_step;
  if (graph_step) {
    if (!s->loop_exec) SLE_TRY(build_loop_graph(s));
    SLE_CUDA(cudaGraphLaunch(s->loop_exec, st));
  } else {
    s->iter_active = (int)act.size();
    for (int host_iter = 0;; ++host_iter) {
      if (host_iter > MAX_INNER + 2) {  // the device flags must have stopped the loop by now
        set_error("inner loop control lost (device iteration counter did not advance)");
        return SLE_ERR_STATE;
      }
      SLE_TRY(enqueue_iteration(s, 0));
      SLE_TRY(sync_scal(s));
      int left = 0;
      for (int b : act) left += !s->hsc[b].done;
      s->iter_active = left;
      if (!left) break;
    }
  }
  note_launch();
  k_reopen<<<nb(B, 128), 128, 0, st>>>(D);

  // ---- radial displacement (solver.py:1054-1072)
  if (s->cfg.calcRG) {
    note_launch();
    k_rr<<<dim3(nb(nc), UB), 256, 0, st>>>(D);
    std::vector<FieldSpec> f;
    for (int b : act) f.push_back(fspec(D.g(G_RR, b), D.sp(S_RRLM, b), &s->sc[b].status));
    SLE_TRY(sht_synthesis_list(s->plan, f.data(), (int)f.size(), st));
  }
  // ---- analytic rates of the slots that asked for them, read before the commit
  {
    bool any_rates = false;
    for (int b : act) any_rates |= s->hss[b].rates != 0;
    if (any_rates) {
      note_launch();
      k_rate_spec<<<dim3(nb(nc), UB), 256, 0, st>>>(D, s->rate_spec, s->rate_tab, s->rate_rec, s->rate_rot);
    }
    bool any_horiz = false;
    for (int b : act) any_horiz |= s->hss[b].horiz != 0;
    if (any_horiz) {
      note_launch();
      k_horiz_spec<<<dim3(nb(nc), UB), 256, 0, st>>>(D, s->horiz_spec, s->horiz_tab);
    }
  }
  // ---- commit (solver.py:1080-1096); extrap history (solver_opt.py:817-822)
  note_launch();
  k_commit<<<dim3(nb(nc), UB), 256, 0, st>>>(D, s->cfg.inner_extrap);
  // ---- topography / ocean function and the degree-0 diagnostics
  note_launch();
  k_post_grid<<<dim3(D.nlat, UB), 256, 0, st>>>(D, s->cfg.opt_diag);
  if (!s->cfg.opt_diag) {
    std::vector<FieldSpec> f;
    for (int b : act) {
      const int* gs = &s->sc[b].status;
      f.push_back(fspec(D.g(G_TMP, b), D.sp(S_SP0, b), gs));
      f.push_back(fmask(D.m(M_CXY, b), D.sp(S_SP1, b), gs));
      f.push_back(fspec(D.g(G_TMP3, b), D.sp(S_SP2, b), gs));
      f.push_back(fspec(D.g(G_TMP4, b), D.sp(S_SP3, b), gs));
    }
    SLE_TRY(sht_analysis_list(s->plan, f.data(), (int)f.size(), st));
    note_launch();
    k_diag00<<<UB, 32, 0, st>>>(D);
  }
  SLE_CUDA(cudaGetLastError());
  return SLE_OK;
}

int batch_step_end(sle_batch* s, sle_step_info* info) {
  if (!s->pending) {
    set_error("sle_batch_step_end: no step was begun");
    return SLE_ERR_STATE;
  }
  s->pending = false;
  const std::vector<int> act = s->pending_act;
  const bool graph_step = s->pending_graph;
  if (act.empty()) return SLE_OK;
  SLE_TRY(sync_scal(s));
  int first_bad = SLE_OK;
  int maxiter = 0;
  for (int b : act) maxiter = std::max(maxiter, s->hsc[b].numiter);
  if (graph_step) note_launch((int)(maxiter * s->body_launches));
  for (int b : act) {
    SlotHost& h = s->slot[b];
    const Scal& f = s->hsc[b];
    sle_step_info& o = h.last;
    std::memset(&o, 0, sizeof(o));
    o.iter = h.iter;
    o.numiter = f.numiter;
    o.status = f.status;
    o.xi = f.xi;
    o.gr_reguess = f.gr_reguess;
    o.gr_ice_analyses = f.gr_ice_an;
    if (f.status != SLE_OK) {
      if (first_bad == SLE_OK) {
        first_bad = f.status;
        if (f.status == SLE_ERR_NONCONVERGED)
          set_error("inner loop failed to converge, xi=%.17g", f.xi);
        else if (f.status == SLE_ERR_TIMEOUT)
          set_error("a tensor-core transform kernel timed out waiting on its pipeline");
        else
          set_error("non-finite value in the inner loop (xi=%g)", f.xi);
      }
      if (info) info[b] = o;
      continue;
    }
    if (s->cfg.inner_extrap) {
      h.hsel ^= 1;
      h.dt_hist[1] = h.dt_hist[0];
      h.dt_hist[0] = h.dt;
      h.nhist = std::min(2, h.nhist + 1);
    }
    const double slc_ocn00 = f.diag[0], c00 = f.diag[1], slc_b00 = f.diag[2], cst00 = f.diag[3];
    if (s->cfg.opt_diag) {
      // float arithmetic of solver_opt.py:909-914
      const double a4 = 4 * PI_LEGACY * std::pow(s->cfg.radius, 2);
      o.ocean_area = c00 * a4;
      o.oceanBeta_area = cst00 * a4;
      o.gmslc_ocn = slc_ocn00 / c00;
      o.gmslc_ocnBeta = slc_b00 / cst00;
    } else {
      // complex [0,0] ratios of solver.py:1105-1113 (imaginary parts are exactly zero)
      o.ocean_area = fourpiR2(s, c00);
      o.oceanBeta_area = fourpiR2(s, cst00);
      o.gmslc_ocn = slc_ocn00 * (1.0 / c00);
      o.gmslc_ocnBeta = slc_b00 * (1.0 / cst00);
    }
    o.ice_volume = fourpiR2(s, f.diag[4]);
    std::memcpy(o.il, f.il, sizeof(o.il));
    std::memcpy(o.mm, f.mm, sizeof(o.mm));
    std::memcpy(o.lam, f.lam, sizeof(o.lam));
    if (info) info[b] = o;
  }
  return first_bad;
}

int batch_step(sle_batch* s, const double* const* ice, int on_device, const double* dt_years,
               sle_step_info* info) {
  const int rc = batch_step_begin(s, ice, on_device, dt_years);
  if (rc != SLE_OK) {
    if (s->pending) {   // a launch failed part-way: wait for what was enqueued before reporting
      s->pending = false;
      cudaStreamSynchronize(s->st);
    }
    return rc;
  }
  return batch_step_end(s, info);
}

int batch_get(sle_batch* s, int b, int field, void* dst, int dst_on_device) {
  const Dev& D = s->D;
  const size_t gb = sizeof(double) * D.ng;
  const cudaMemcpyKind kind = dst_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  const double* src = nullptr;
  switch (field) {
    case SLE_F_TGRID: src = D.g(G_TOPO, b); break;
    case SLE_F_OCEAN:
    case SLE_F_BETA:
    case SLE_F_ICESTAR:
    case SLE_F_OCEAN0:
    case SLE_F_BETA0: {
      const int mid = field == SLE_F_OCEAN ? M_CXY : field == SLE_F_BETA ? M_BETA : field == SLE_F_ICESTAR ? M_GR
                      : field == SLE_F_OCEAN0 ? M_CXY0 : M_BETA0;
      double* out = dst_on_device ? static_cast<double*>(dst) : D.g(G_TMP4, b);
      note_launch();
      k_mask_grid<<<nb(D.ng), 256, 0, s->st>>>(D.ng, D.m(mid, b), field == SLE_F_ICESTAR ? D.g(G_ICE, b) : nullptr,
                                              out);
      SLE_CUDA(cudaGetLastError());
      if (dst_on_device) {
        SLE_CUDA(cudaStreamSynchronize(s->st));
        return SLE_OK;
      }
      src = out;
      break;
    }
    case SLE_F_R: src = D.g(G_RR, b); break;
    case SLE_F_DELTASL: src = D.g(G_DELTASL, b); break;
    case SLE_F_G:
      note_launch();
      k_grid_add<<<nb(D.ng), 256, 0, s->st>>>(D.ng, D.g(G_DELTASL, b), D.g(G_RR, b), D.g(G_TMP, b));
      SLE_CUDA(cudaGetLastError());
      src = D.g(G_TMP, b);
      break;
    case SLE_F_DS_CONVERGED:
    case SLE_F_LOAD_INC: {
      const double2* p = (field == SLE_F_DS_CONVERGED) ? D.sp(S_P_OCEAN, b) : D.sp(S_LOAD, b);
      double2* dense = s->plan->packbuf;  // staging (nm*nm <= 4*ncoef)
      SLE_TRY(sht_unpack(s->plan, p, dense, s->st));
      const size_t bytes = sizeof(double2) * (size_t)D.nl * D.nl;
      SLE_CUDA(cudaMemcpyAsync(dst, dense, bytes, kind, s->st));
      SLE_CUDA(cudaStreamSynchronize(s->st));
      return SLE_OK;
    }
    default:
      set_error("sle_solver_get: unknown field %d", field);
      return SLE_ERR_BAD_ARG;
  }
  SLE_CUDA(cudaMemcpyAsync(dst, src, gb, kind, s->st));
  SLE_CUDA(cudaStreamSynchronize(s->st));
  return SLE_OK;
}

}  // namespace

// ------------------------------------------------------------------ batch C ABI
extern "C" int sle_batch_create(const sle_config* cfg, int nslots, int max_modes, sle_batch** out) {
  return batch_create(cfg, nslots, max_modes, out);
}

extern "C" int sle_batch_destroy(sle_batch* b) {
  if (b) cudaStreamSynchronize(b->st);
  batch_free(b);
  return SLE_OK;
}

extern "C" int sle_batch_load(sle_batch* b, int slot, const sle_earth* earth, double dt_years, const double* topo0,
                              const double* ice0, int on_device, double* ocean_area0, double* oceanBeta_area0,
                              double* ice_volume0) {
  if (!b || !topo0 || !ice0) {
    set_error("sle_batch_load: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  SLE_TRY(check_slot(b, slot, "sle_batch_load"));
  if (!(dt_years > 0.0)) {
    set_error("sle_batch_load: dt_years must be > 0");
    return SLE_ERR_BAD_ARG;
  }
  SLE_TRY(set_earth(b, slot, earth, dt_years));
  return init_slot(b, slot, topo0, ice0, on_device, ocean_area0, oceanBeta_area0, ice_volume0);
}

extern "C" int sle_batch_release(sle_batch* b, int slot) {
  if (!b) {
    set_error("sle_batch_release: NULL batch");
    return SLE_ERR_BAD_ARG;
  }
  SLE_TRY(check_slot(b, slot, "sle_batch_release"));
  b->slot[slot].loaded = 0;
  b->slot[slot].inited = 0;
  b->slot[slot].rs_ds = nullptr;
  b->slot[slot].rs_mask = nullptr;
  b->slot[slot].rs_cap = b->slot[slot].rs_valid = 0;
  return SLE_OK;
}

// ----------------------------------------------------------------- snapshots
// One slot's whole state as a host byte image: a header (configuration it belongs to, the host
// bookkeeping of the slot), then every per-slot device buffer in a fixed order.  The device
// sections hold more than the state a step carries forward (all grids, masks and spectra of the
// slot, not only the modal state, load history, topography and masks of the last step), so a
// restored slot continues bit for bit as the original would have.  The reference checkpoints the
// same state (fortran/src/modal_state_mod.f90:445-477: shapes, decay, loads and modal states) in
// a stream file of its own format; this image is not that format.
namespace {

constexpr uint32_t SNAP_MAGIC = 0x534C4553u;   // "SLES"
constexpr uint32_t SNAP_VERSION = 1;

struct SnapHeader {
  uint32_t magic, version;
  int32_t nlat, nlon, lmax, K, precision, flags;
  long long nbytes;
  // host bookkeeping of the slot (SlotHost without the caller-owned reuse store)
  int32_t iter, nhist, hsel, pad;
  double dt, dt_cur, dt_hist[2];
  double ocean_area0, oceanBeta_area0, ice_volume0;
  sle_step_info last;
};

int snap_flags(const sle_config& c) {
  return (c.tpw ? 1 : 0) | (c.checkmarine ? 2 : 0) | (c.calcRG ? 4 : 0) | (c.opt_dsl ? 8 : 0) |
         (c.opt_diag ? 16 : 0) | (c.inner_extrap ? 32 : 0);
}

// The device sections of slot b: (device address, bytes), in image order.
std::vector<std::pair<void*, size_t>> snap_sections(sle_batch* s, int b) {
  const Dev& D = s->D;
  const size_t ng = (size_t)D.ng, nc = (size_t)D.ncoef, nl = (size_t)D.nl, K = (size_t)s->K;
  std::vector<std::pair<void*, size_t>> v;
  for (int g = 0; g < NGRID; ++g) v.push_back({D.g(g, b), sizeof(double) * ng});
  for (int m = 0; m < NMASK; ++m) v.push_back({D.m(m, b), ng});
  for (int q = 0; q < NSPEC; ++q) v.push_back({D.sp(q, b), sizeof(double2) * nc});
  if (K) v.push_back({D.R + (size_t)b * K * nc, sizeof(double2) * K * nc});
  v.push_back({s->nmod + (size_t)b * nl, sizeof(int) * nl});
  double* kl[] = {s->s_kl, s->decay, s->omd, s->a_sl, s->a_rr};
  if (K)
    for (double* p : kl) v.push_back({p + (size_t)b * K * nl, sizeof(double) * K * nl});
  double* l1[] = {s->ttl, s->ttlekhl, s->ttlhe};
  for (double* p : l1) v.push_back({p + (size_t)b * nl, sizeof(double) * nl});
  if (K) {
    double* k1[] = {s->a_il, s->a_m, s->a_tsl, s->a_trr};
    for (double* p : k1) v.push_back({p + (size_t)b * K, sizeof(double) * K});
    v.push_back({s->r_il + (size_t)b * K * 9, sizeof(double) * K * 9});
    v.push_back({s->r_m + (size_t)b * K * 3, sizeof(double) * K * 3});
    v.push_back({s->r_lam + (size_t)b * K * 6, sizeof(double) * K * 6});
  }
  v.push_back({s->rc + b, sizeof(RotConst)});
  v.push_back({s->sc + b, sizeof(Scal)});
  return v;
}

long long snap_bytes(sle_batch* s) {
  long long n = (long long)sizeof(SnapHeader);
  for (const auto& sec : snap_sections(s, 0)) n += (long long)sec.second;
  return n;
}

int batch_snapshot(sle_batch* s, int b, void* dst, long long nbytes) {
  SLE_TRY(check_slot(s, b, "sle_batch_snapshot"));
  const SlotHost& h = s->slot[b];
  if (!h.inited) {
    set_error("sle_batch_snapshot: slot %d holds no solve", b);
    return SLE_ERR_STATE;
  }
  const long long need = snap_bytes(s);
  if (!dst || nbytes < need) {
    set_error("sle_batch_snapshot: the image needs %lld bytes (got %lld)", need, nbytes);
    return SLE_ERR_BAD_ARG;
  }
  SnapHeader hd;
  std::memset(&hd, 0, sizeof(hd));
  hd.magic = SNAP_MAGIC;
  hd.version = SNAP_VERSION;
  hd.nlat = s->cfg.nlat;
  hd.nlon = s->cfg.nlon;
  hd.lmax = s->cfg.lmax;
  hd.K = s->K;
  hd.precision = s->cfg.precision;
  hd.flags = snap_flags(s->cfg);
  hd.nbytes = need;
  hd.iter = h.iter;
  hd.nhist = h.nhist;
  hd.hsel = h.hsel;
  hd.dt = h.dt;
  hd.dt_cur = h.dt_cur;
  hd.dt_hist[0] = h.dt_hist[0];
  hd.dt_hist[1] = h.dt_hist[1];
  hd.ocean_area0 = h.ocean_area0;
  hd.oceanBeta_area0 = h.oceanBeta_area0;
  hd.ice_volume0 = h.ice_volume0;
  hd.last = h.last;
  unsigned char* out = static_cast<unsigned char*>(dst);
  std::memcpy(out, &hd, sizeof(hd));
  size_t off = sizeof(hd);
  for (const auto& sec : snap_sections(s, b)) {
    SLE_CUDA(cudaMemcpyAsync(out + off, sec.first, sec.second, cudaMemcpyDeviceToHost, s->st));
    off += sec.second;
  }
  SLE_CUDA(cudaStreamSynchronize(s->st));
  return SLE_OK;
}

int batch_restore(sle_batch* s, int b, const void* src, long long nbytes) {
  SLE_TRY(check_slot(s, b, "sle_batch_restore"));
  const long long need = snap_bytes(s);
  if (!src || nbytes < (long long)sizeof(SnapHeader)) {
    set_error("sle_batch_restore: no snapshot image given");
    return SLE_ERR_BAD_ARG;
  }
  SnapHeader hd;
  std::memcpy(&hd, src, sizeof(hd));
  if (hd.magic != SNAP_MAGIC || hd.version != SNAP_VERSION) {
    set_error("sle_batch_restore: not a snapshot image of this library (magic %08x, version %u)", hd.magic,
              hd.version);
    return SLE_ERR_BAD_ARG;
  }
  if (hd.nlat != s->cfg.nlat || hd.nlon != s->cfg.nlon || hd.lmax != s->cfg.lmax || hd.K != s->K ||
      hd.precision != s->cfg.precision || hd.flags != snap_flags(s->cfg)) {
    set_error("sle_batch_restore: the image belongs to a %d x %d, lmax %d, %d-mode solve of precision %d and "
              "options %d; this batch is %d x %d, lmax %d, %d modes, precision %d, options %d",
              hd.nlat, hd.nlon, hd.lmax, hd.K, hd.precision, hd.flags, s->cfg.nlat, s->cfg.nlon, s->cfg.lmax,
              s->K, s->cfg.precision, snap_flags(s->cfg));
    return SLE_ERR_BAD_SHAPE;
  }
  if (hd.nbytes != need || nbytes < need) {
    set_error("sle_batch_restore: image of %lld bytes, this batch's images have %lld", nbytes, need);
    return SLE_ERR_BAD_ARG;
  }
  const unsigned char* in = static_cast<const unsigned char*>(src);
  size_t off = sizeof(hd);
  for (const auto& sec : snap_sections(s, b)) {
    SLE_CUDA(cudaMemcpyAsync(sec.first, in + off, sec.second, cudaMemcpyHostToDevice, s->st));
    off += sec.second;
  }
  SLE_CUDA(cudaStreamSynchronize(s->st));
  SlotHost& h = s->slot[b];
  h = SlotHost{};
  h.loaded = 1;
  h.inited = 1;
  h.iter = hd.iter;
  h.nhist = hd.nhist;
  h.hsel = hd.hsel;
  h.dt = hd.dt;
  h.dt_cur = hd.dt_cur;
  h.dt_hist[0] = hd.dt_hist[0];
  h.dt_hist[1] = hd.dt_hist[1];
  h.ocean_area0 = hd.ocean_area0;
  h.oceanBeta_area0 = hd.oceanBeta_area0;
  h.ice_volume0 = hd.ice_volume0;
  h.last = hd.last;
  return SLE_OK;
}

}  // namespace

extern "C" int sle_batch_snapshot_bytes(const sle_batch* b, long long* nbytes) {
  if (!b || !nbytes) {
    set_error("sle_batch_snapshot_bytes: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  *nbytes = snap_bytes(const_cast<sle_batch*>(b));
  return SLE_OK;
}

extern "C" int sle_batch_snapshot(sle_batch* b, int slot, void* dst, long long nbytes) {
  if (!b) {
    set_error("sle_batch_snapshot: NULL batch");
    return SLE_ERR_BAD_ARG;
  }
  return batch_snapshot(b, slot, dst, nbytes);
}

extern "C" int sle_batch_restore(sle_batch* b, int slot, const void* src, long long nbytes) {
  if (!b) {
    set_error("sle_batch_restore: NULL batch");
    return SLE_ERR_BAD_ARG;
  }
  return batch_restore(b, slot, src, nbytes);
}

extern "C" int sle_batch_set_tuning(sle_batch* b, const sle_mx_tuning* t) {
  if (!b) {
    set_error("sle_batch_set_tuning: NULL batch");
    return SLE_ERR_BAD_ARG;
  }
  if (b->pending) {
    set_error("sle_batch_set_tuning: a step is in flight");
    return SLE_ERR_STATE;
  }
  SLE_TRY(sle_sht_set_tuning(b->plan, t));
  // the captured inner-loop graph holds the old launch shape: capture it again at the next step
  if (b->loop_exec) cudaGraphExecDestroy(b->loop_exec);
  if (b->loop_graph) cudaGraphDestroy(b->loop_graph);
  b->loop_exec = nullptr;
  b->loop_graph = nullptr;
  return SLE_OK;
}

extern "C" int sle_batch_set_reuse(sle_batch* b, int slot, void* ds_store, void* mask_store, int capacity,
                                   int valid) {
  if (!b) {
    set_error("sle_batch_set_reuse: NULL batch");
    return SLE_ERR_BAD_ARG;
  }
  SLE_TRY(check_slot(b, slot, "sle_batch_set_reuse"));
  if (ds_store && (!mask_store || capacity < 1 || valid < 0 || valid > capacity)) {
    set_error("sle_batch_set_reuse: need both stores, capacity >= 1 and 0 <= valid <= capacity");
    return SLE_ERR_BAD_ARG;
  }
  if (ds_store && (reinterpret_cast<uintptr_t>(ds_store) & 15)) {
    set_error("sle_batch_set_reuse: the increment store must be 16-byte aligned");
    return SLE_ERR_BAD_ARG;
  }
  SlotHost& h = b->slot[slot];
  h.rs_ds = reinterpret_cast<double2*>(ds_store);
  h.rs_mask = reinterpret_cast<unsigned char*>(mask_store);
  h.rs_cap = ds_store ? capacity : 0;
  h.rs_valid = ds_store ? valid : 0;
  return SLE_OK;
}

extern "C" int sle_batch_step(sle_batch* b, const double* const* ice, int on_device, const double* dt_years,
                              sle_step_info* info) {
  if (!b || !ice) {
    set_error("sle_batch_step: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  return batch_step(b, ice, on_device, dt_years, info);
}

extern "C" int sle_batch_step_begin(sle_batch* b, const double* const* ice, int on_device,
                                    const double* dt_years) {
  if (!b || !ice) {
    set_error("sle_batch_step_begin: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  const int rc = batch_step_begin(b, ice, on_device, dt_years);
  if (rc != SLE_OK && b->pending) {
    b->pending = false;
    cudaStreamSynchronize(b->st);
  }
  return rc;
}

extern "C" int sle_batch_step_end(sle_batch* b, sle_step_info* info) {
  if (!b) {
    set_error("sle_batch_step_end: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  return batch_step_end(b, info);
}

extern "C" int sle_batch_get(sle_batch* b, int slot, int field, void* dst, int dst_on_device) {
  if (!b || !dst) {
    set_error("sle_batch_get: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  SLE_TRY(check_slot(b, slot, "sle_batch_get"));
  return batch_get(b, slot, field, dst, dst_on_device);
}

extern "C" int sle_batch_stream(sle_batch* b, void** stream) {
  if (!b || !stream) {
    set_error("sle_batch_stream: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  *stream = reinterpret_cast<void*>(b->st);
  return SLE_OK;
}

extern "C" int sle_batch_info(const sle_batch* b, int* nslots, int* max_modes, long long* device_bytes) {
  if (!b) {
    set_error("sle_batch_info: NULL batch");
    return SLE_ERR_BAD_ARG;
  }
  if (nslots) *nslots = b->nslot;
  if (max_modes) *max_modes = b->K;
  if (device_bytes) {
    const long long B = b->nslot, ng = b->D.ng, nc = b->D.ncoef, K = b->K, nl = b->D.nl;
    *device_bytes = B * (NGRID * ng * 8 + NMASK * ng + NSPEC * nc * 16 + K * nc * 16 + 5 * K * nl * 8 + 3 * nl * 8 +
                         (long long)sizeof(Scal) + b->D.npart * 8 + 4LL * b->cfg.nlat * 8);
  }
  return SLE_OK;
}

// ----------------------------------------------------- single-solve C ABI (one slot)
extern "C" int sle_solver_create(const sle_config* cfg, const sle_earth* earth, sle_solver** out) {
  if (!cfg || !earth || !out) {
    set_error("sle_solver_create: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  *out = nullptr;
  if (earth->nmodes < 0 || earth->nmodes > 4096) {
    set_error("sle_solver_create: nmodes out of range");
    return SLE_ERR_BAD_ARG;
  }
  sle_batch* b = nullptr;
  SLE_TRY(batch_create(cfg, 1, earth->nmodes, &b));
  const int rc = set_earth(b, 0, earth, cfg->dt_years);
  if (rc != SLE_OK) {
    batch_free(b);
    return rc;
  }
  sle_solver* s = new sle_solver();
  s->b = b;
  *out = s;
  return SLE_OK;
}

extern "C" int sle_solver_destroy(sle_solver* s) {
  if (!s) return SLE_OK;
  sle_batch_destroy(s->b);
  delete s;
  return SLE_OK;
}

extern "C" int sle_solver_stream(sle_solver* s, void** stream) {
  if (!s || !stream) {
    set_error("sle_solver_stream: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  *stream = reinterpret_cast<void*>(s->b->st);
  return SLE_OK;
}

extern "C" int sle_solver_init(sle_solver* s, const double* topo0, const double* ice0, int on_device,
                               double* ocean_area0, double* oceanBeta_area0, double* ice_volume0) {
  if (!s || !topo0 || !ice0) {
    set_error("sle_solver_init: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  return init_slot(s->b, 0, topo0, ice0, on_device, ocean_area0, oceanBeta_area0, ice_volume0);
}

extern "C" int sle_solver_step(sle_solver* s, const double* ice, int on_device, double dt_years,
                               sle_step_info* info) {
  if (!s || !ice) {
    set_error("sle_solver_step: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  if (!s->b->slot[0].inited) {
    set_error("sle_solver_step: call sle_solver_init first");
    return SLE_ERR_STATE;
  }
  const double* ices[1] = {ice};
  const double dts[1] = {dt_years};
  sle_step_info o;
  const int rc = batch_step(s->b, ices, on_device, dts, &o);
  if (info) *info = o;
  return rc;
}

extern "C" int sle_solver_snapshot_bytes(const sle_solver* s, long long* nbytes) {
  if (!s) {
    set_error("sle_solver_snapshot_bytes: NULL solver");
    return SLE_ERR_BAD_ARG;
  }
  return sle_batch_snapshot_bytes(s->b, nbytes);
}

extern "C" int sle_solver_snapshot(sle_solver* s, void* dst, long long nbytes) {
  if (!s) {
    set_error("sle_solver_snapshot: NULL solver");
    return SLE_ERR_BAD_ARG;
  }
  return batch_snapshot(s->b, 0, dst, nbytes);
}

extern "C" int sle_solver_restore(sle_solver* s, const void* src, long long nbytes) {
  if (!s) {
    set_error("sle_solver_restore: NULL solver");
    return SLE_ERR_BAD_ARG;
  }
  return batch_restore(s->b, 0, src, nbytes);
}

extern "C" int sle_solver_set_reuse(sle_solver* s, void* ds_store, void* mask_store, int capacity, int valid) {
  if (!s) {
    set_error("sle_solver_set_reuse: NULL solver");
    return SLE_ERR_BAD_ARG;
  }
  return sle_batch_set_reuse(s->b, 0, ds_store, mask_store, capacity, valid);
}

extern "C" int sle_solver_set_rate_tables(sle_solver* s, const double* tab) {
  if (!s) {
    set_error("sle_solver_set_rate_tables: NULL solver");
    return SLE_ERR_BAD_ARG;
  }
  sle_batch* b = s->b;
  b->rates_on.resize(b->nslot, 0);
  if (!tab) {
    b->rates_on[0] = 0;
    return SLE_OK;
  }
  const size_t nl = (size_t)b->D.nl, per = (size_t)(2 * b->K + 4) * nl;
  if (!b->rate_spec) {
    SLE_TRY(dalloc(&b->rate_spec, (size_t)b->nslot * 2 * b->D.ncoef));
    SLE_TRY(dalloc(&b->rate_tab, (size_t)b->nslot * per));
    SLE_TRY(dalloc(&b->rate_rec, (size_t)b->nslot * 2));
    SLE_TRY(dalloc(&b->rate_rot, (size_t)b->nslot * 18 * b->K));
  }
  SLE_CUDA(cudaMemcpyAsync(b->rate_tab, tab, per * sizeof(double), cudaMemcpyHostToDevice, b->st));
  SLE_CUDA(cudaStreamSynchronize(b->st));
  b->rates_on[0] = 1;
  return SLE_OK;
}

extern "C" int sle_solver_get_rates(sle_solver* s, void* dsl, void* drr, double* rec, double* rot) {
  if (!s || !dsl || !drr || !rec || !rot) {
    set_error("sle_solver_get_rates: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  sle_batch* b = s->b;
  if (b->rates_on.empty() || !b->rates_on[0] || !b->rate_spec) {
    set_error("sle_solver_get_rates: no rate tables set (sle_solver_set_rate_tables before the step)");
    return SLE_ERR_STATE;
  }
  const Dev& D = b->D;
  const size_t dense = sizeof(double2) * (size_t)D.nl * D.nl;
  double2* stage = b->plan->packbuf;  // staging (nm*nm <= 4*ncoef)
  for (int q = 0; q < 2; ++q) {
    SLE_TRY(sht_unpack(b->plan, b->rate_spec + (size_t)q * D.ncoef, stage, b->st));
    SLE_CUDA(cudaMemcpyAsync(q ? drr : dsl, stage, dense, cudaMemcpyDeviceToHost, b->st));
    SLE_CUDA(cudaStreamSynchronize(b->st));
  }
  double dice[2];
  SLE_CUDA(cudaMemcpy(dice, b->rate_rec, sizeof(dice), cudaMemcpyDeviceToHost));
  const Scal& f = b->hsc[0];
  rec[0] = dice[0];
  rec[1] = dice[1];
  for (int q = 0; q < 9; ++q) rec[2 + q] = f.oldil[q];
  for (int q = 0; q < 3; ++q) rec[11 + q] = f.oldm[q];
  for (int q = 0; q < 6; ++q) rec[14 + q] = f.dlam_prev2[q];
  SLE_CUDA(cudaMemcpy(rot, b->rate_rot, sizeof(double) * 18 * b->K, cudaMemcpyDeviceToHost));
  return SLE_OK;
}

extern "C" int sle_solver_set_ramp(sle_solver* s, const double* tab) {
  if (!s) {
    set_error("sle_solver_set_ramp: NULL solver");
    return SLE_ERR_BAD_ARG;
  }
  sle_batch* b = s->b;
  b->ramp_on.resize(b->nslot, 0);
  b->ramp_c.resize((size_t)4 * b->nslot, 0.0);
  if (!tab) {
    b->ramp_on[0] = 0;
    return SLE_OK;
  }
  const size_t per = (size_t)(b->K + 2) * b->D.nl;
  if (!b->ramp_tab) SLE_TRY(dalloc(&b->ramp_tab, (size_t)b->nslot * per));
  SLE_CUDA(cudaMemcpyAsync(b->ramp_tab, tab, per * sizeof(double), cudaMemcpyHostToDevice, b->st));
  SLE_CUDA(cudaStreamSynchronize(b->st));
  for (int q = 0; q < 4; ++q) b->ramp_c[q] = tab[per + q];
  b->ramp_on[0] = 1;
  return SLE_OK;
}

extern "C" int sle_solver_set_horizontal(sle_solver* s, const double* tab) {
  if (!s) {
    set_error("sle_solver_set_horizontal: NULL solver");
    return SLE_ERR_BAD_ARG;
  }
  sle_batch* b = s->b;
  b->horiz_on.resize(b->nslot, 0);
  if (!tab) {
    b->horiz_on[0] = 0;
    return SLE_OK;
  }
  const size_t per = (size_t)(b->K + 1) * b->D.nl;
  if (!b->horiz_spec) {
    SLE_TRY(dalloc(&b->horiz_spec, (size_t)b->nslot * b->D.ncoef));
    SLE_TRY(dalloc(&b->horiz_tab, (size_t)b->nslot * per));
  }
  SLE_CUDA(cudaMemcpyAsync(b->horiz_tab, tab, per * sizeof(double), cudaMemcpyHostToDevice, b->st));
  SLE_CUDA(cudaStreamSynchronize(b->st));
  b->horiz_on[0] = 1;
  return SLE_OK;
}

extern "C" int sle_solver_get_horizontal(sle_solver* s, void* psi, double* r_lam, double* lam12) {
  if (!s || !psi || !r_lam || !lam12) {
    set_error("sle_solver_get_horizontal: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  sle_batch* b = s->b;
  if (b->horiz_on.empty() || !b->horiz_on[0] || !b->horiz_spec) {
    set_error("sle_solver_get_horizontal: the read-out is off (sle_solver_set_horizontal before the step)");
    return SLE_ERR_STATE;
  }
  const Dev& D = b->D;
  double2* stage = b->plan->packbuf;  // staging (nm*nm <= 4*ncoef)
  SLE_TRY(sht_unpack(b->plan, b->horiz_spec, stage, b->st));
  SLE_CUDA(cudaMemcpyAsync(psi, stage, sizeof(double2) * (size_t)D.nl * D.nl, cudaMemcpyDeviceToHost, b->st));
  SLE_CUDA(cudaStreamSynchronize(b->st));
  SLE_CUDA(cudaMemcpy(r_lam, b->r_lam, sizeof(double) * 6 * b->K, cudaMemcpyDeviceToHost));
  const Scal& f = b->hsc[0];
  for (int q = 0; q < 6; ++q) {
    lam12[q] = f.dlam_prev2[q];
    lam12[6 + q] = f.dlam_cur2[q];
  }
  return SLE_OK;
}

extern "C" int sle_solver_get(sle_solver* s, int field, void* dst, int dst_on_device) {
  if (!s || !dst) {
    set_error("sle_solver_get: NULL argument");
    return SLE_ERR_BAD_ARG;
  }
  return batch_get(s->b, 0, field, dst, dst_on_device);
}
