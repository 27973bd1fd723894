// akmc_kernels.cu -- sm_100a kernels of the vacancy-hop path.
//
// One sector round of the synchronous sublattice (src/algorithms/sl/sublattice.inl:64-177)
// runs as three launches:
//   k_bucket   one thread per vacancy: find its domain block, keep it if it lies in
//              the block's active sector, append it to the block's list;
//   k_hop      one CTA per active block: stage the sector plus a 2-cell halo (occupancy
//              bytes and the int32 density cache) into shared memory and run the hop
//              loop there.  Evaluator warp w evaluates jump directions w, w + kEvalWarps,
//              ... of a vacancy (its 32 lanes split the 76 sites of a jump); the control
//              warp forms the ordered total, selects, performs the hop and keeps the
//              vacancy list and the clock; each hop writes its two occupancy bytes and 78
//              densities through to global memory;
//   k_finalize one thread per block: clock of blocks without vacancies, next round.
// Concurrently active sectors are at least 4 cells apart, so the staged regions of
// different blocks never overlap and no atomics are needed on the lattice.
#include <cuda_runtime.h>

#include <cfloat>
#include <algorithm>
#include <cstdint>

#include "akmc_device.h"

namespace akmc {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kStageRows = 4;  // rows of the staged region each warp has in flight
// Blocks a k_flow thread may visit per sweep, until it takes one.  Measured on the 256^3 lattice
// and the 512 batched boxes: 2 and 3 cost 1.7% and 4.5% on the 256^3 lattice and gain nothing
// on the batched boxes.
#ifndef AKMC_SWEEP_VISITS
#define AKMC_SWEEP_VISITS 1
#endif
constexpr int kSweepVisits = AKMC_SWEEP_VISITS;
// Nanoseconds a k_flow CTA sleeps after a sweep that moved no block on (0: none).
#ifndef AKMC_SWEEP_SLEEP_NS
#define AKMC_SWEEP_SLEEP_NS 256
#endif
enum : int { kPairBond = 0, kEam64 = 1, kEam32 = 2 };  // energy kinds, one kernel instance each
// CTA shape: W warps evaluate the 8 jump directions (warp w takes jumps w, w + W, ...), one
// more warp controls the hop loop.  The hop kernels are built for W = 8 (one jump per warp) and
// W = 4 (two jumps per warp, two CTAs per SM); a context picks one (akmc_context_config).
template <int W>
struct Shape {
  static_assert(8 % W == 0, "whole jump directions per warp");
  static constexpr int kEvalWarps = W;
  static constexpr int kJumpsPerWarp = 8 / W;
  static constexpr int kThreads = 32 * (W + 1);
  static constexpr int kCtl = 32 * W;  // control thread: first lane of the control warp
  // CTAs per SM the register budget is cut for: two 5-warp CTAs fit (10 warps, at most 3 per SM
  // partition), two 9-warp ones would cut a thread to 96 registers.
  static constexpr int kCtasPerSm = W <= 4 ? 2 : 1;
};
constexpr int kMaxThreads = Shape<8>::kThreads;
// The shape's constants under their short names inside a kernel or device function of shape W.
#define AKMC_SHAPE(W)                                         \
  constexpr int kEvalWarps = Shape<W>::kEvalWarps;            \
  constexpr int kJumpsPerWarp = Shape<W>::kJumpsPerWarp;      \
  constexpr int kThreads = Shape<W>::kThreads;                \
  constexpr int kCtl = Shape<W>::kCtl;                        \
  (void)kEvalWarps;                                           \
  (void)kJumpsPerWarp;                                        \
  (void)kThreads;                                             \
  (void)kCtl

__device__ __forceinline__ int wrap1(int v, int m) { return v < 0 ? v + m : (v >= m ? v - m : v); }

// Reference rank split: block k of n cells over p blocks starts at k (n/p) + min(k, n%p).
__device__ __forceinline__ int block_of(int c, int n, int p) {
  const int q = n / p, r = n % p;
  const int big = r * (q + 1);
  return c < big ? c / (q + 1) : r + (c - big) / q;
}

struct Region {
  int slo[3], w[3];
  int ox, oy, oz;  // origin in sites (x doubled); may be negative (periodic wrap)
  int LX, LY, LZ, n;  // row pitch in sites and rows of the shared layout, its sites
  int LXt, xo, nt;    // region row width, its first site within the pitch, sites staged
  int ey, ez;         // rows of the region in y and z (LY, LZ: the pitch, the job's box with tma)
  int tma;            // staged by one tensor copy per array
  int hx;             // cells before the sector in x within the pitch (the 2-cell halo, plus xo / 2)
  int bulk;           // rows staged by bulk copies: bo occupancy bytes and br densities each
  int bo, br;
};

// The staged region of a block's sector: the sector and a 2-cell halo.  Rows are staged
// whole by the bulk-copy unit when the job allows it (J.bulk: rows of a multiple of 16 sites,
// 16-byte aligned arrays, shared memory sized for the wider rows): each row's span is rounded
// out to 16-site boundaries from its unwrapped origin R.ox (which may lie before the row or run
// past its end: the sector never wraps, its halo may), so every copy starts on a 16-byte
// boundary.  A span that crosses the row's end (or starts before it) is copied as two pieces,
// each inside the row; the span must not be longer than the row.
__device__ __forceinline__ void make_region(const BlockDev& B, const JobDev& J, int sec, Region& R) {
  for (int d = 0; d < 3; ++d) {
    const int half = (B.c1[d] - B.c0[d]) / 2;
    if ((sec >> d) & 1) {
      R.slo[d] = B.c0[d] + half;
      R.w[d] = B.c1[d] - B.c0[d] - half;
    } else {
      R.slo[d] = B.c0[d];
      R.w[d] = half;
    }
  }
  R.ox = 2 * (R.slo[0] - 2);
  R.oy = R.slo[1] - 2;
  R.oz = R.slo[2] - 2;
  R.LX = 2 * (R.w[0] + 4);
  R.LY = R.w[1] + 4;
  R.LZ = R.w[2] + 4;
  R.LXt = R.LX;
  R.xo = 0;
  R.bulk = 0;
  R.bo = R.br = 0;
  if (J.bulk) {
    const int x0 = R.ox & ~15;  // rounds down, negative origins included
    const int xo = R.ox - x0;
    const int bo = (xo + R.LXt + 15) & ~15;
    // the span [x0, x0 + bo) lies inside the row and its halo (always, for blocks of >= 8 cells:
    // x0 >= -16 and x0 + bo <= sx + 19)
    if (x0 >= -kHaloL && x0 + bo <= J.sx + kHaloR) {
      R.xo = xo;
      R.ox = x0;
      R.LX = (R.LXt + 14 + 15) & ~15;  // one pitch for every alignment: tables stay valid
      R.bo = bo;
      R.br = (xo + R.LXt + 3) & ~3;
      R.bulk = 1;
    }
  }
  R.ey = R.LY;
  R.ez = R.LZ;
  R.tma = 0;
  if (R.bulk && J.tma) {
    // every region of the job takes the box as its pitch (the shell tables stay valid across
    // them); one that does not wrap in y or z is one box of the lattice
    R.LX = J.tbox[0];
    R.LY = J.tbox[1];
    R.LZ = J.tbox[2];
    R.tma = R.oy >= 0 && R.oy + R.ey <= J.sy && R.oz >= 0 && R.oz + R.ez <= J.sz;
  }
  R.hx = R.slo[0] - R.ox / 2;
  R.n = R.LX * R.LY * R.LZ;
  R.nt = R.tma ? R.n : R.LXt * R.ey * R.ez;
}

// Shared-memory working set of one CTA (followed by the staged region).
struct Smem {
  double b1[25], b2[25];
  union {                       // phi_XY(shell s) - phi_XY(shell t), index (X*4+Y)*64 + s*8 + t,
    double dphi64[4 * 4 * 64];  // in the precision of the kernel's kind
    float dphi32[4 * 4 * 64];
  };
  int32_t dfq[4 * 64];          // f_X(shell s) - f_X(shell t) in Q.24, index X*64 + s*8 + t
  int32_t fq1[4];               // f_X at the first shell
  int32_t d1[2][8];             // 1nn local offsets by x parity
  int32_t w1[2][8];             // 1nn packed (dx, dy, dz)
  int32_t d2[6];
  int32_t jl[2][8][kJumpN];     // int16 local offset | (s*8+t) << 16
  int32_t rl[2][8][kRefreshN];  // packed (dx, dy, dz) | (s*8+t) << 24
  int32_t vidx[kMaxV];          // vacancy table index of record k
  // Vacancy records in two sets: a hop selected from set c writes set c ^ 1 (see run_block).
  int32_t vloc[2][kMaxV], vlid[2][kMaxV];               // local site, global site id
  int16_t vcx[2][kMaxV], vcy[2][kMaxV], vcz[2][kMaxV];  // local coordinates (x in doubled sites)
  int32_t vgx[2][kMaxV], vgy[2][kMaxV], vgz[2][kMaxV];  // global coordinates
  uint8_t vact[2][kMaxV];       // vacancy still inside the active sector
  // the same record packed for the selection, which every warp reads: (local site, local x, y,
  // z) and (global x, y, z, site id), two 16-byte loads instead of seven
  alignas(16) int4 vpk[2][kMaxV][2];
  int32_t ord[2][kMaxV];        // the active vacancies in z-y-x order (ascending site id)
  int32_t nord[2];
  uint8_t vX[2][kMaxV][8];      // code of jump b's target atom (0: the target is a vacancy)
  alignas(16) double rates[2][kMaxV][8];
  // F-table window, two planes: FP64 (c0, c1) x kFWin then (c2, c3) x kFWin;
  // FP32 (hi, lo, c1, c2) x kFWin then c3 x kFWin
  alignas(16) unsigned char fwin[kFWin * 32];
  alignas(8) uint64_t mbar;                    // completion barrier of the window's bulk copy
  uint64_t mbar_st;                            // completion barrier of the region's bulk copies
  uint32_t mbar_phase, mbst_phase;
  int32_t win_pot;                             // potential (and precision) the window holds
  int32_t tab_key[2];                          // potential, kind and region strides the tables hold
  // hop-loop control, written by the control thread, in slots of the iteration parity
  double ctl_u[2];         // the selection's uniform, drawn ahead
  int32_t ctl_stop[2];     // the sector's window is reached (or the hop cap): no more selections
  uint64_t xsn[2][4];      // selection stream after the uniform drawn ahead
  int32_t ctl_ok;          // the region's copies arrived
  int32_t fin;             // record set that holds the block's vacancies after run_block
  uint64_t xs[4], xt[4];  // the block's selection / residence-time streams while it runs
  // asynchronous schedule (k_flow)
  int8_t flow_lag[8][27];
  int32_t flow_cand[kMaxThreads];
  int32_t flow_ncand, flow_stop, flow_progress, flow_more;
  int32_t fv[kFlowSlots], fslot[kFlowSlots], fnv;  // the sector's vacancies and their slots
  int32_t fsite[kFlowSlots];                        // their sites
  int64_t flow_cr[kMaxThreads], flow_ct[kMaxThreads];  // round and target of each round handed over
  unsigned long long flow_cvv[kMaxThreads];             // its block's vacancy-slot valid bits
  int64_t cur_r, cur_t;   // the block's round and target for its next chained round
  int32_t bc0[3], bc1[3];  // the running block's area and its job's block count, kept for the
  int32_t bnb;             // post-round updates (a reload after the round's stores is an L2 trip)
  int64_t hops_out;       // the block's hop count after run_block
  // run_block's control thread: hops at the start, hops, n_act sum and evaluations of the
  // block-round, the sector's clock and its threshold
  int64_t c_hop0, c_nh, c_nact, c_evals;
  double c_time, c_thr;
  double c_nu, c_kT;  // the job's attempt frequency and kT (the rates' constants)
  double c_rkT;       // RN(1 / kT): the rates' exponent arguments without a division
  double pre_evo;         // the active sector's clock, read while the region's copies fly
  // device counters summed per CTA and added once when the kernel ends (per-round atomics on
  // the same addresses from every CTA queue up); hops of the current job likewise
  unsigned long long acc[6];  // counters 0 (hops), 1, 3, 4, 5, 6
  int32_t acc_job;
  unsigned long long acc_job_hops;
};

// --- bulk copy global -> shared with an mbarrier (cp.async.bulk, TMA unit) -----------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Arms the barrier for `bytes` of bulk copies (then issued with bulk_copy).
__device__ __forceinline__ void bulk_expect(uint64_t* bar, uint32_t bytes) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Global -> shared bulk copy; addresses 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// Waits for the barrier phase with an iteration limit; false when the limit is reached.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase) {
  for (int it = 0; it < (1 << 22); ++it) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// F-table access: cells inside the shared-memory window, the rest from global memory.
struct FTab {
  const unsigned char* win;
  int kw0;
  const Potential* pot;      // the full tables (far cells), read on the rare path only
  unsigned int* status;
#ifdef AKMC_PHASE_PROFILE
  unsigned long long* prof;  // sub-phase cycles of the evaluation
#endif
};

// Job constants of the running block, held in registers (the job record sits in global
// memory, where every store of the hop loop would otherwise force a reload).
struct JobC {
  uint8_t* occ;
  int32_t* rho;
  int sx, sy, sz, px;
};

#if defined(AKMC_PHASE_PROFILE) && !defined(AKMC_FLOW_PROFILE) && !defined(AKMC_HOP_PROFILE)
#define EVAL_T(i)                                                                       \
  do {                                                                                  \
    if (threadIdx.x == 0) {                                                             \
      const long long t_ = clock64();                                                   \
      atomicAdd(FT.prof + (i), static_cast<unsigned long long>(t_ - tev));              \
      tev = t_;                                                                         \
    }                                                                                   \
  } while (0)
#else
#define EVAL_T(i) \
  do {            \
  } while (0)
#endif

__device__ __forceinline__ int local_delta(int32_t w, const Region& R) {
  return unpack_dx(w) + R.LX * (unpack_dy(w) + R.LY * unpack_dz(w));
}

// Region layout after Smem: int32 densities, then occupancy bytes (16-byte aligned).
__device__ __forceinline__ uint8_t* occ_of(int32_t* rho_s, int nreg) {
  return reinterpret_cast<uint8_t*>(rho_s) + ((static_cast<size_t>(nreg) * 4 + 127) & ~static_cast<size_t>(127));
}

template <int W>
__device__ void load_tables(Smem& sm, const Potential& P, const Geometry& G, const Region& R, int kind) {
  AKMC_SHAPE(W);
  const bool eam = kind != kPairBond;
  const int tid = threadIdx.x;
  if (tid < 25) {
    sm.b1[tid] = P.b1[tid / 5][tid % 5];
    sm.b2[tid] = P.b2[tid / 5][tid % 5];
  }
  if (tid < 16) {
    const int32_t w = G.nn1[tid >> 3][tid & 7];
    sm.d1[tid >> 3][tid & 7] = local_delta(w, R);
    sm.w1[tid >> 3][tid & 7] = w;
  }
  if (tid < 6) sm.d2[tid] = local_delta(G.nn2[tid], R);
  if (eam) {
    if (tid < 4) sm.fq1[tid] = P.fq[tid][1];
    for (int i = tid; i < 4 * 4 * 64; i += kThreads) {
      const int xy = i >> 6, hs = (i >> 3) & 7, ht = i & 7;
      const double* ph = &P.phi64[0][0][0] + xy * 8;
      const float* pf = &P.phi32[0][0][0] + xy * 8;
      if (kind == kEam64) sm.dphi64[i] = ph[hs] - ph[ht];
      else sm.dphi32[i] = pf[hs] - pf[ht];
      if (i < 4 * 64) sm.dfq[i] = P.fq[i >> 6][hs] - P.fq[i >> 6][ht];
    }
    for (int i = tid; i < 2 * 8 * kJumpN; i += kThreads) {
      const int32_t w = __ldg(&G.jump[0][0][0] + i);
      (&sm.jl[0][0][0])[i] = (local_delta(w, R) & 0xffff) | ((unpack_sh_s(w) * 8 + unpack_sh_t(w)) << 16);
    }
    for (int i = tid; i < 2 * 8 * kRefreshN; i += kThreads) {
      const int32_t w = __ldg(&G.refresh[0][0][0] + i);
      (&sm.rl[0][0][0])[i] = (w & 0xffffff) | ((unpack_sh_s(w) * 8 + unpack_sh_t(w)) << 24);
    }
  }
}

__device__ __forceinline__ int sdelta(int32_t e) { return static_cast<int16_t>(e & 0xffff); }
__device__ __forceinline__ int jshells(int32_t e) { return (e >> 16) & 63; }
__device__ __forceinline__ int rshells(int32_t e) { return (e >> 24) & 63; }

// Cells outside the shared-memory window (rare): global memory, range-checked.
__device__ __noinline__ double F64_far(const double2* g64lo, const double2* g64hi, unsigned int* status, int32_t r,
                                       double p) {
  const int k = r >> kRhoCellShift;
  int kc = k;
  if (r < 0 || k > kTabN - 2) {
    atomicOr(status, kErrRhoRange);
    kc = r < 0 ? 0 : kTabN - 2;
  }
  const double2 lo = __ldg(g64lo + kc), hi = __ldg(g64hi + kc);
  return cubic_d(lo.x, lo.y, hi.x, hi.y, p);
}

__device__ __forceinline__ double F64(const FTab& T, int32_t r) {
  const int k = r >> kRhoCellShift;
  // p = (r mod 2^17) * 2^-17, built in the exponent field: 1 + m 2^-17 minus 1 (both exact)
  const double p = __hiloint2double(0x3FF00000 | ((r & kRhoFracMask) << 3), 0) - 1.0;
  const unsigned kk = static_cast<unsigned>(k - T.kw0);
  if (kk < static_cast<unsigned>(kFWin)) {
    const double2 lo = reinterpret_cast<const double2*>(T.win)[kk];
    const double2 hi = reinterpret_cast<const double2*>(T.win)[kFWin + kk];
    return cubic_d(lo.x, lo.y, hi.x, hi.y, p);
  }
  return F64_far(T.pot->F64lo, T.pot->F64hi, T.status, r, p);
}

// A cell known to lie inside the shared-memory window.
__device__ __forceinline__ double F64win(const FTab& T, int32_t r) {
  const int kk = (r >> kRhoCellShift) - T.kw0;
  const double p = __hiloint2double(0x3FF00000 | ((r & kRhoFracMask) << 3), 0) - 1.0;
  const double2 lo = reinterpret_cast<const double2*>(T.win)[kk];
  const double2 hi = reinterpret_cast<const double2*>(T.win)[kFWin + kk];
  return cubic_d(lo.x, lo.y, hi.x, hi.y, p);
}
__device__ __forceinline__ FCell32 cell32win(const FTab& T, int32_t r) {
  const int kk = (r >> kRhoCellShift) - T.kw0;
  const float4 a = reinterpret_cast<const float4*>(T.win)[kk];
  FCell32 c;
  c.hi = a.x; c.lo = a.y; c.c1 = a.z; c.c2 = a.w;
  c.c3 = reinterpret_cast<const float*>(T.win + kFWin * 16)[kk];
  c.pad0 = c.pad1 = c.pad2 = 0.f;
  return c;
}

__device__ __forceinline__ FCell32 cell32(const FTab& T, int32_t r) {
  const int k = r >> kRhoCellShift;
  const unsigned kk = static_cast<unsigned>(k - T.kw0);
  float4 a;
  float c3;
  if (kk < static_cast<unsigned>(kFWin)) {
    a = reinterpret_cast<const float4*>(T.win)[kk];
    c3 = reinterpret_cast<const float*>(T.win + kFWin * 16)[kk];
  } else {
    int kc = k;
    if (r < 0 || k > kTabN - 2) {
      atomicOr(T.status, kErrRhoRange);
      kc = r < 0 ? 0 : kTabN - 2;
    }
    a = __ldg(T.pot->F32a + kc);
    c3 = __ldg(T.pot->F32b + kc);
  }
  FCell32 c;
  c.hi = a.x; c.lo = a.y; c.c1 = a.z; c.c2 = a.w; c.c3 = c3;
  c.pad0 = c.pad1 = c.pad2 = 0.f;
  return c;
}

// Rates of vacancy k of record set `set`, all 8 jumps, CTA-collective (no barrier inside; the
// caller synchronises before the rates are read).  Warp b evaluates jump b.
//  pair-bond: lanes 0..3 run the four bond counts of VacRatesSolver::deltaE
//             (vacancy_rates_solver.cpp:45-116), each summed in the reference order;
//  EAM:       lane q sums sites i = q, q+32, q+64 of the jump's list; the 32 partials
//             merge by a xor butterfly (16, 8, 4, 2, 1), then the moving atom's own
//             embedding change is added.
// l is the vacancy's local site (its record's vloc), d1b[p] jump b's 1nn offset for x parity p.
template <int KIND>
__device__ void eval_vacancy(Smem& sm, int set, const uint8_t* occ_s, const int32_t* rho_s, int k, int l, int b,
                             const int32_t (&d1b)[2], const FTab& FT, const JobC& jc, const int32_t (&jr)[2][3],
                             double* de_out) {
  const int lane = threadIdx.x & 31;
  const int q = lane;
  const int p = l & 1;
  const int tl = l + (p ? d1b[1] : d1b[0]);
  const uint8_t Xc = occ_s[tl];
  const bool avail = is_atom(Xc);
  double dE = 0.0;
#ifdef AKMC_PHASE_PROFILE
  long long tev = clock64();
#endif
  if (KIND == kPairBond) {
    double energy = 0.0;
    if (avail && q < 4) {
      const bool at_t = (q & 1) != 0;
      const int center = at_t ? tl : l;
      const int pc = at_t ? (p ^ 1) : p;
      const uint8_t src = (q == 0 || q == 3) ? static_cast<uint8_t>(kV) : Xc;
      const int ovr = q == 2 ? tl : (q == 3 ? l : -1);
      const uint8_t ovr_code = q == 2 ? static_cast<uint8_t>(kV) : Xc;
      const int si = bond_index(src);
      for (int b2 = 0; b2 < 8; ++b2) {
        const int nb = center + sm.d1[pc][b2];
        const uint8_t o = nb == ovr ? ovr_code : occ_s[nb];
        energy += sm.b1[bond_index(o) * 5 + si];
      }
#pragma unroll
      for (int b2 = 0; b2 < 6; ++b2) {
        if (!((0x2F >> b2) & 1)) continue;  // PeriodLatticeList::get2nnStatus
        const int nb = center + sm.d2[b2];
        const uint8_t o = nb == ovr ? ovr_code : occ_s[nb];
        energy += sm.b2[bond_index(o) * 5 + si];
      }
    }
    const double pair = energy + __shfl_down_sync(kFull, energy, 1);  // q0: e_before, q2: e_after
    const double after = __shfl_down_sync(kFull, pair, 2);
    dE = after - pair;
  } else if (KIND == kEam64) {
    double acc = 0.0, EX = 0.0;
    const int X = atom_index(Xc);  // read only when avail
    if (avail) {
      // gather: this lane's sites (q, q+32, q+64 of the jump's list; lanes 12..31 have two),
      // their occupancy, densities and shell codes, and the moving atom's own two densities
      uint8_t o[3];
      int32_t r0[3], r1[3];
      int h[3];
      bool in[3];
#pragma unroll
      for (int u = 0; u < 3; ++u) {
        in[u] = q + 32 * u < kJumpN;
        const int32_t e = p ? jr[1][u] : jr[0][u];  // 0 outside the list: the vacancy's own site
        const int j = l + sdelta(e);
        h[u] = jshells(e);
        o[u] = occ_s[j];
        r0[u] = rho_s[j];
        r1[u] = r0[u] + sm.dfq[X * 64 + h[u]];
      }
      const int32_t rx1 = rho_s[l] - sm.fq1[X], rx0 = rho_s[tl];
      // every cell inside the shared-memory window (nearly always): one straight run of loads
      // and polynomials; otherwise the general path, which reads far cells from global memory
      bool win = static_cast<unsigned>((rx1 >> kRhoCellShift) - FT.kw0) < static_cast<unsigned>(kFWin) &&
                 static_cast<unsigned>((rx0 >> kRhoCellShift) - FT.kw0) < static_cast<unsigned>(kFWin);
#pragma unroll
      for (int u = 0; u < 3; ++u)
        win = win && (!in[u] || (static_cast<unsigned>((r0[u] >> kRhoCellShift) - FT.kw0) < static_cast<unsigned>(kFWin) &&
                                 static_cast<unsigned>((r1[u] >> kRhoCellShift) - FT.kw0) < static_cast<unsigned>(kFWin)));
      double t[3];
      if (win) {
        EX = F64win(FT, rx1) - F64win(FT, rx0);
#pragma unroll
        for (int u = 0; u < 3; ++u) t[u] = in[u] ? F64win(FT, r1[u]) - F64win(FT, r0[u]) : 0.0;
      } else {
        EX = F64(FT, rx1) - F64(FT, rx0);
#pragma unroll
        for (int u = 0; u < 3; ++u) t[u] = in[u] ? F64(FT, r1[u]) - F64(FT, r0[u]) : 0.0;
      }
      // site term (F(r+d) - F(r)) + (phi_s - phi_t), summed in list order
#pragma unroll
      for (int u = 0; u < 3; ++u)
        if (in[u] && o[u] != kV) acc += t[u] + sm.dphi64[(X * 4 + atom_index(o[u])) * 64 + h[u]];
    }
#pragma unroll
    EVAL_T(0);
    for (int m = 16; m >= 1; m >>= 1) acc = acc + __shfl_xor_sync(kFull, acc, m);
    EVAL_T(1);
    if (avail && q == 0) dE = EX + acc;
    EVAL_T(2);
  } else {
    Comp32 acc;
    acc.s = 0.f;
    acc.c = 0.f;
    const int X = atom_index(Xc);  // read only when avail
    if (avail) {
      uint8_t o[3];
      int32_t r0[3], r1[3];
      int h[3];
      bool in[3];
#pragma unroll
      for (int u = 0; u < 3; ++u) {
        in[u] = q + 32 * u < kJumpN;
        const int32_t e = p ? jr[1][u] : jr[0][u];
        const int j = l + sdelta(e);
        h[u] = jshells(e);
        o[u] = occ_s[j];
        r0[u] = rho_s[j];
        r1[u] = r0[u] + sm.dfq[X * 64 + h[u]];
      }
      bool win = true;
#pragma unroll
      for (int u = 0; u < 3; ++u)
        win = win && (!in[u] || (static_cast<unsigned>((r0[u] >> kRhoCellShift) - FT.kw0) < static_cast<unsigned>(kFWin) &&
                                 static_cast<unsigned>((r1[u] >> kRhoCellShift) - FT.kw0) < static_cast<unsigned>(kFWin)));
      float t[3];
      if (win) {
#pragma unroll
        for (int u = 0; u < 3; ++u) t[u] = in[u] ? dF32(cell32win(FT, r1[u]), cell32win(FT, r0[u]), r1[u], r0[u]) : 0.f;
      } else {
#pragma unroll
        for (int u = 0; u < 3; ++u) t[u] = in[u] ? dF32(cell32(FT, r1[u]), cell32(FT, r0[u]), r1[u], r0[u]) : 0.f;
      }
#pragma unroll
      for (int u = 0; u < 3; ++u)
        if (in[u] && o[u] != kV) kahan_add(acc, t[u] + sm.dphi32[(X * 4 + atom_index(o[u])) * 64 + h[u]]);
    }
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) {
      Comp32 o;
      o.s = __shfl_xor_sync(kFull, acc.s, m);
      o.c = __shfl_xor_sync(kFull, acc.c, m);
      acc = comp_merge(acc, o);
    }
    if (avail && q == 0) {
      const int32_t r1 = rho_s[l] - sm.fq1[X];
      const int32_t r0 = rho_s[tl];
      const float EX = dF32(cell32(FT, r1), cell32(FT, r0), r1, r0);
      const float dEf = EX + (acc.s - acc.c);
      dE = static_cast<double>(dEf);
    }
  }
  if (q == 0) {
    sm.rates[set][k][b] = avail ? arrhenius_rk(sm.c_nu, sm.c_kT, sm.c_rkT, Xc, dE) : 0.0;
    sm.vX[set][k][b] = avail ? Xc : 0;
    if (de_out) de_out[k * 8 + b] = avail ? dE : 0.0;  // akmc_calculate only
  }
  if (KIND == kEam64) EVAL_T(3);
}

// Bulk staging of a region (R.bulk): the bulk-copy unit moves whole rows, R.bo occupancy bytes
// and R.br densities from the row's 16-site boundary R.ox (unwrapped; the row's halo holds the
// sites past either end), into shared rows of pitch R.LX; thread t0 + k nt issues row
// t0 + k nt, one copy per array.  The barrier is armed for the bytes of every row (stage_bytes).
__device__ __forceinline__ void stage_rows(const Region& R, const uint8_t* occ, const int32_t* rho, int px, int sy, int sz,
                                           bool eam, uint8_t* occ_s, int32_t* rho_s, uint64_t* bar, int t0, int nt) {
  asm volatile("fence.proxy.async;" ::: "memory");  // generic accesses before, copies after
  const int nrows = R.ey * R.ez;
  for (int row = t0; row < nrows; row += nt) {
    const int ly = row % R.ey, lz = row / R.ey;
    const int gy = wrap1(R.oy + ly, sy), gz = wrap1(R.oz + lz, sz);
    const int64_t first = static_cast<int64_t>(px) * (gy + static_cast<int64_t>(sy) * gz) + kHaloL + R.ox;
    const int l = R.LX * (ly + R.LY * lz);  // the shared row (pitch LX, LY)
    bulk_copy(occ_s + l, occ + first, static_cast<uint32_t>(R.bo), bar);
    if (eam) bulk_copy(rho_s + l, rho + first, static_cast<uint32_t>(4 * R.br), bar);
  }
}
// Bytes the bulk staging of region R moves (the barrier's transaction count).
__device__ __forceinline__ uint32_t stage_bytes(const Region& R, bool eam) {
  if (R.tma) return static_cast<uint32_t>(R.n) * (eam ? 5u : 1u);
  return static_cast<uint32_t>(R.ey * R.ez) * static_cast<uint32_t>(R.bo + (eam ? 4 * R.br : 0));
}
// Tensor staging of a region (R.tma): one 3D tile copy per array of the job's box from entry
// (kHaloL + R.ox, R.oy, R.oz) of the lattice (x a multiple of 16 entries: 16-byte aligned in both
// arrays), into shared memory laid out with the box as pitch.  Parts of the box past the region
// are staged too and never read; parts past the array are filled with zeros.  One thread issues
// both copies.
__device__ __forceinline__ void stage_tensor(const Region& R, const void* tmaps, int job, bool eam, uint8_t* occ_s,
                                             int32_t* rho_s, uint64_t* bar) {
  asm volatile("fence.proxy.async;" ::: "memory");  // generic accesses before, copies after
  const unsigned char* m = static_cast<const unsigned char*>(tmaps) + static_cast<size_t>(job) * 256;
  const int x = kHaloL + R.ox, y = R.oy, z = R.oz;
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          smem_u32(occ_s)),
      "l"(m), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
  if (eam)
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            smem_u32(rho_s)),
        "l"(m + 128), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// Phase profile (builds with -DAKMC_PHASE_PROFILE): thread 0 accumulates the cycles
// between consecutive CTA barriers into counters[8 + phase].
#ifdef AKMC_PHASE_PROFILE
#define AKMC_PHASE(i)                                                                           \
  do {                                                                                          \
    if (threadIdx.x == 0) {                                                                     \
      const long long t_ = clock64();                                                           \
      atomicAdd(a.counters + 8 + (i), static_cast<unsigned long long>(t_ - tph));               \
      tph = t_;                                                                                 \
    }                                                                                           \
  } while (0)
#else
#define AKMC_PHASE(i) \
  do {              \
  } while (0)
#endif
// Staging sub-phases (builds with -DAKMC_FLOW_PROFILE): counters 16..19.
#ifdef AKMC_FLOW_PROFILE
#define AKMC_STAGE_T(k)                                                                         \
  do {                                                                                          \
    if (threadIdx.x == 0) {                                                                     \
      const long long t_ = clock64();                                                           \
      atomicAdd(a.counters + 16 + (k), static_cast<unsigned long long>(t_ - tsub));             \
      tsub = t_;                                                                                \
    }                                                                                           \
  } while (0)
#else
#define AKMC_STAGE_T(k) \
  do {                \
  } while (0)
#endif

// Hop-loop sub-phases (builds with -DAKMC_PHASE_PROFILE -DAKMC_HOP_PROFILE=1): thread 0 (an
// evaluator) adds its cycles per stage into counters 16..19, the control thread into 20..22,
// and counts the iterations in 23.  With -DAKMC_HOP_PROFILE=2 thread 0's four counters split
// the perform stage instead (HOP_P).
#if defined(AKMC_PHASE_PROFILE) && defined(AKMC_HOP_PROFILE)
#define HOP_T(k)                                                                                           \
  do {                                                                                                     \
    if (threadIdx.x == 0 || threadIdx.x == kCtl) {                                                         \
      const long long t_ = clock64();                                                                      \
      atomicAdd(a.counters + (threadIdx.x == 0 ? 16 : 20) + (k), static_cast<unsigned long long>(t_ - thp)); \
      thp = t_;                                                                                            \
    }                                                                                                      \
  } while (0)
#else
#define HOP_T(k) \
  do {           \
  } while (0)
#endif
#if defined(AKMC_PHASE_PROFILE) && defined(AKMC_HOP_PROFILE) && AKMC_HOP_PROFILE == 2
#define HOP_P(k)                                                                       \
  do {                                                                                 \
    if (threadIdx.x == 0) {                                                            \
      const long long t_ = clock64();                                                  \
      atomicAdd(a.counters + 16 + (k), static_cast<unsigned long long>(t_ - thp));     \
      thp = t_;                                                                        \
    }                                                                                  \
  } while (0)
#undef HOP_T
#define HOP_T(k)                                                                       \
  do {                                                                                 \
    if (threadIdx.x == 0) thp = clock64();                                             \
  } while (0)
#else
#define HOP_P(k) \
  do {           \
  } while (0)
#endif

// The hop loop of one block's active sector (or one per-hop API step), CTA-collective.
// round_now is the block's round (its completed rounds), read by the caller.
// The evaluator warps evaluate rates (warp w: jumps w, w + kEvalWarps, ...) and refresh
// densities; the control warp keeps the ordered vacancy list, selects, performs the occupancy
// swap and runs the clock.
// vlist holds the ids of the cnt_in vacancies inside the sector (any order).  Returns
// false, uniformly, when the sector's clock is already past its window: nothing ran and
// the vacancy arrays of sm were not filled.
template <int KIND, int W>
__device__ bool run_block(const RoundArgs& a, int gb, Smem& sm, uint8_t* occ_s, int32_t* rho_s,
                          const int32_t* vlist, int cnt_in, int64_t round_now, bool flowpre = false) {
  AKMC_SHAPE(W);
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const bool evaluator = warp < kEvalWarps;
#ifdef AKMC_PHASE_PROFILE
  long long tph = clock64();
#endif
#ifdef AKMC_FLOW_PROFILE
  long long tsub = clock64();
#endif
  BlockDev& B = a.blocks[gb];
  const JobDev& J = a.jobs[B.job];
  const Potential& P = a.pots[J.pot];
  const bool eam = KIND != kPairBond;
  // the block record, the lattice and the vacancy table are read at L2 (__ldcg): under the
  // asynchronous schedule another SM may have written them since this SM last looked
  const int sec = a.mode == kModeRound ? sector_of_round(round_now) : a.api_sector;
  // flowpre (k_flow): the caller issued a bulk region's copies on mbar_st already, and left the
  // sector's clock (sm.pre_evo), the streams (sm.xs, sm.xt) and the vacancies' sites (sm.fsite)
  // in shared memory, read while the copies were in flight
  double thr = 0.0;
  if (a.mode == kModeRound) {
    const int64_t step = round_now >> 3;
    thr = static_cast<double>(step + 1) * J.window - (flowpre ? sm.pre_evo : __ldcg(&B.evo[sec]));
    if (!(0.0 < thr)) {  // sector_time stays 0 (sublattice.inl:82)
      if (flowpre && tid == kCtl) {  // copies already issued complete first: the buffer is reused next
        Region R0;
        make_region(B, J, sec, R0);
        if (R0.bulk) {
          if (mbar_wait(&sm.mbar_st, sm.mbst_phase)) sm.mbst_phase ^= 1u;
          else atomicOr(a.status, kErrTimeout);
        }
      }
      return false;
    }
  }
  JobC jc;
  jc.occ = J.occ;
  jc.rho = J.rho;
  jc.sx = J.sx;
  jc.sy = J.sy;
  jc.sz = J.sz;
  jc.px = J.px;

  Region R;
  make_region(B, J, sec, R);
  if (tid == 0) {  // before the barrier below; the evaluations read them
    sm.c_nu = J.nu;
    sm.c_kT = J.kT;
    sm.c_rkT = 1.0 / J.kT;
  }
  // F-table window: one bulk copy issued by the control thread, overlapped with the staging
  const int win_key = J.pot * 2 + (KIND == kEam32 ? 1 : 0);
  const bool need_win = eam && sm.win_pot != win_key;
  // the shell tables and neighbour lists depend on the potential, the kind and the region's
  // row strides only: kept from the CTA's previous block when those match
  const int tab0 = J.pot * 4 + KIND, tab1 = R.LX | (R.LY << 16);
  const bool need_tab = sm.tab_key[0] != tab0 || sm.tab_key[1] != tab1;
  const int nrows = R.LY * R.LZ;
  if (R.bulk && !flowpre && tid == kCtl)  // armed before any copy is issued (after the barrier below)
    bulk_expect(&sm.mbar_st, stage_bytes(R, eam));
  __syncthreads();  // every thread has read win_pot and tab_key; the previous item's readers are done
  AKMC_STAGE_T(0);
  if (need_win && tid == kCtl) {
    if (KIND == kEam32) {
      bulk_expect(&sm.mbar, kFWin * 20u);
      bulk_copy(sm.fwin, P.F32a + P.fwin0, kFWin * 16u, &sm.mbar);
      bulk_copy(sm.fwin + kFWin * 16, P.F32b + P.fwin0, kFWin * 4u, &sm.mbar);
    } else {
      bulk_expect(&sm.mbar, kFWin * 32u);
      bulk_copy(sm.fwin, P.F64lo + P.fwin0, kFWin * 16u, &sm.mbar);
      bulk_copy(sm.fwin + kFWin * 16, P.F64hi + P.fwin0, kFWin * 16u, &sm.mbar);
    }
  }
  if (need_tab) {
    load_tables<W>(sm, P, *a.geo, R, KIND);
    if (tid == 0) {
      sm.tab_key[0] = tab0;
      sm.tab_key[1] = tab1;
    }
  }
  FTab FT;
  FT.win = sm.fwin;
  FT.kw0 = P.fwin0;
  FT.pot = &P;
  FT.status = a.status;
#ifdef AKMC_PHASE_PROFILE
  FT.prof = a.counters + 16;
#endif
  AKMC_STAGE_T(1);

  // stage the region: warp w takes rows w, w+9, ...; kStageRows rows of loads are issued
  // before any shared-memory store so they are all in flight (rows hold <= 64 sites)
  if (!R.bulk) {
    // row positions of the region's x span (the halo holds the sites past either end)
    const int gx0 = kHaloL + R.ox + lane, gx1 = gx0 + 32;
    const bool has0 = lane < R.LX, has1 = lane + 32 < R.LX;
    constexpr int kW = kThreads / 32;
    for (int row0 = warp; row0 < nrows; row0 += kStageRows * kW) {
      uint8_t ov[kStageRows][2];
      int32_t rv[kStageRows][2];
#pragma unroll
      for (int k = 0; k < kStageRows; ++k) {
        const int row = row0 + kW * k;
        if (row < nrows) {
          const int ly = row % R.LY, lz = row / R.LY;
          const int gy = wrap1(R.oy + ly, jc.sy), gz = wrap1(R.oz + lz, jc.sz);
          const int64_t base = static_cast<int64_t>(jc.px) * (gy + static_cast<int64_t>(jc.sy) * gz);
          if (has0) {
            ov[k][0] = __ldcg(jc.occ + base + gx0);
            if (eam) rv[k][0] = __ldcg(jc.rho + base + gx0);
          }
          if (has1) {
            ov[k][1] = __ldcg(jc.occ + base + gx1);
            if (eam) rv[k][1] = __ldcg(jc.rho + base + gx1);
          }
        }
      }
#pragma unroll
      for (int k = 0; k < kStageRows; ++k) {
        const int row = row0 + kW * k;
        if (row < nrows) {
          const int l = lane + R.LX * row;
          if (has0) {
            occ_s[l] = ov[k][0];
            if (eam) rho_s[l] = rv[k][0];
          }
          if (has1) {
            occ_s[l + 32] = ov[k][1];
            if (eam) rho_s[l + 32] = rv[k][1];
          }
        }
      }
    }
  } else if (!flowpre) {
    if (R.tma) {
      if (tid == kCtl) stage_tensor(R, a.tmaps, B.job, eam, occ_s, rho_s, &sm.mbar_st);
    } else {
      stage_rows(R, jc.occ, jc.rho, jc.px, jc.sy, jc.sz, eam, occ_s, rho_s, &sm.mbar_st, tid, kThreads);
    }
  }
  AKMC_STAGE_T(2);
  const int cnt = cnt_in;
  if (tid < cnt) {
    const int v = vlist[tid];
    const int s = flowpre ? sm.fsite[tid] : __ldcg(&a.vac_site[v]);
    const int X = s % jc.sx;
    const int t = s / jc.sx;
    const int y = t % jc.sy;
    const int z = t / jc.sy;
    const int lx = X - R.ox, ly = y - R.oy, lz = z - R.oz;
    sm.vidx[tid] = v;
    sm.vloc[0][tid] = lx + R.LX * (ly + R.LY * lz);
    sm.vlid[0][tid] = s;
    sm.vcx[0][tid] = static_cast<int16_t>(lx);
    sm.vcy[0][tid] = static_cast<int16_t>(ly);
    sm.vcz[0][tid] = static_cast<int16_t>(lz);
    sm.vgx[0][tid] = X;
    sm.vgy[0][tid] = y;
    sm.vgz[0][tid] = z;
    sm.vact[0][tid] = 1;
    sm.vpk[0][tid][0] = make_int4(lx + R.LX * (ly + R.LY * lz), lx, ly, lz);
    sm.vpk[0][tid][1] = make_int4(X, y, z, s);
  }
  __syncthreads();
  AKMC_STAGE_T(3);
  AKMC_PHASE(0);
  if (tid == kCtl) {
    // z-y-x scan order of ABVIModel::calcRates = ascending site id inside a sector
    for (int i = 0; i < cnt; ++i) {
      int j = i;
      while (j > 0 && sm.vlid[0][sm.ord[0][j - 1]] > sm.vlid[0][i]) {
        sm.ord[0][j] = sm.ord[0][j - 1];
        --j;
      }
      sm.ord[0][j] = i;
    }
    sm.nord[0] = cnt;
    uint64_t x[4];
    for (int i = 0; i < 4; ++i) {
      if (flowpre) {
        x[i] = sm.xs[i];
      } else {
        x[i] = __ldcg(&B.xs[i]);
        sm.xs[i] = x[i];
        sm.xt[i] = __ldcg(&B.xt[i]);
      }
    }
    // the first selection's uniform, drawn ahead; the stream moves on only if a selection uses it
    sm.ctl_u[0] = a.mode == kModeRound ? uniform_co(x) : 0.0;
    for (int i = 0; i < 4; ++i) sm.xsn[0][i] = x[i];
    sm.ctl_stop[0] = 0;
    sm.ctl_ok = 1;
    sm.fin = 0;
    if (need_win) {
      if (mbar_wait(&sm.mbar, sm.mbar_phase)) {
        sm.mbar_phase ^= 1u;
        sm.win_pot = win_key;
      } else {
        atomicOr(a.status, kErrTimeout);
        mbar_wait(&sm.mbar, sm.mbar_phase);  // bounded second wait for the copy in flight
        sm.win_pot = -1;
        sm.ctl_ok = 0;
      }
    }
    if (R.bulk) {  // the region's rows
      if (mbar_wait(&sm.mbar_st, sm.mbst_phase)) {
        sm.mbst_phase ^= 1u;
      } else {
        atomicOr(a.status, kErrTimeout);
        if (mbar_wait(&sm.mbar_st, sm.mbst_phase)) sm.mbst_phase ^= 1u;  // bounded second wait
        sm.ctl_ok = 0;
      }
    }
  }
  __syncthreads();
  AKMC_PHASE(1);
  if (!sm.ctl_ok) return true;
  // this lane's entries of its warp's jump lists, both x parities
  int32_t jr[kJumpsPerWarp][2][3];
#pragma unroll
  for (int jj = 0; jj < kJumpsPerWarp; ++jj)
#pragma unroll
    for (int u = 0; u < 3; ++u) {
      const int i = lane + 32 * u;
      const bool in = eam && evaluator && i < kJumpN;
      const int b = warp + kEvalWarps * jj;
      jr[jj][0][u] = in ? sm.jl[0][b][i] : 0;
      jr[jj][1][u] = in ? sm.jl[1][b][i] : 0;
    }
  // and its jumps' 1nn offsets, both x parities
  int32_t d1r[kJumpsPerWarp][2];
#pragma unroll
  for (int jj = 0; jj < kJumpsPerWarp; ++jj) {
    const int b = evaluator ? warp + kEvalWarps * jj : 0;
    d1r[jj][0] = sm.d1[0][b];
    d1r[jj][1] = sm.d1[1][b];
  }
  double* const de_out = a.mode == kModeCalc ? a.api_de : nullptr;
  const int D = eam ? 4 : 3;  // a hop changes the rates of vacancies within D cells of its origin

  // first evaluation: every vacancy of the sector, into record set 0
  if (evaluator) {
    for (int k = 0; k < cnt; ++k) {
      const int l = sm.vloc[0][k];
#pragma unroll
      for (int jj = 0; jj < kJumpsPerWarp; ++jj)
        eval_vacancy<KIND>(sm, 0, occ_s, rho_s, k, l, warp + kEvalWarps * jj, d1r[jj], FT, jc, jr[jj], de_out);
    }
  }
  __syncthreads();
  AKMC_PHASE(2);

  // Hop loop, one CTA barrier per hop.  The vacancy records, the ordered list, the rates and the
  // jump targets come in two sets: a hop selected from set c writes set n = c ^ 1, which the next
  // hop reads, so no write of a hop meets a read of the same hop.  Every warp selects for itself
  // (the ordered sum and the scan are deterministic: every warp finds the same hop), then:
  //  - the evaluator warps perform it (occupancy swap, the 78 density deltas, set n), meet at a
  //    named barrier, and evaluate the vacancies the hop made dirty into set n;
  //  - the control warp runs the hop's clock, writes its event, decides whether the sector's
  //    window is reached and draws the next selection's uniform, into the control slots of the
  //    next iteration (indexed by iteration parity).
  // A selection that finds no jump (u * total reached no running sum) advances the clock only and
  // keeps set c.
  // the control thread's running values live in shared memory (sm.c_*): held in registers they
  // would be live in every thread across the loop
  if (tid == kCtl) {
    sm.c_hop0 = __ldcg(&B.hops);
    sm.c_nh = 0;
    sm.c_nact = 0;
    sm.c_evals = cnt;
    sm.c_time = 0.0;
    sm.c_thr = thr;
  }
  int c = 0;   // record set of the current selection
  int it = 0;  // iteration parity: control slots
  // vacancy k of record set `set` lies within D cells of the cell (qx, qy, qz) and in the sector
  auto dirty = [&](int set, int k, int qx, int qy, int qz) -> bool {
    return sm.vact[set][k] && abs((sm.vcx[set][k] >> 1) - qx) <= D && abs(sm.vcy[set][k] - qy) <= D &&
           abs(sm.vcz[set][k] - qz) <= D;
  };
#if defined(AKMC_PHASE_PROFILE) && defined(AKMC_HOP_PROFILE)
  long long thp = clock64();
#endif
  while (true) {
    // the active count and the first active vacancy, read with the loop's stop word
    const int nord = sm.nord[c];
    const int k0 = sm.ord[c][0];
    if (sm.ctl_stop[it]) break;
    const int n = c ^ 1;
    // With one active vacancy (nearly every sector at these dilutions) that vacancy is the one
    // that hops: its record is read while lane 0 selects (k0 is any value when nord != 1).
    const int kq = nord == 1 ? k0 : 0;
    const int4 pa = sm.vpk[c][kq][0], pb = sm.vpk[c][kq][1];
    int s = pa.x;
    int vx2 = pa.y, qy = pa.z, qz = pa.w;
    int sX = pb.x, sY = pb.y, sZ = pb.z;
    // [1] selection: lane 0 of every warp forms the ordered total (ABVIModel::calcRates,
    // kmc.cpp:68-115), then finds the first of the same running sums above u * total
    // (ABVIModel::select, kmc.cpp:242-309).  Jumps onto a vacancy hold 0.0, which leaves a
    // positive sum unchanged.  With one active vacancy the running sums of the total's pass stay
    // in registers (its 8 rates read in four 16-byte loads) and are compared afterwards,
    // independently of one another, instead of being formed a second time.
    int isel = -1, stop = 0;
    double total = 0.0, u = 0.0;
    if (lane == 0) {
      double pv[8];
      if (nord == 1) {
        const double2* r2 = reinterpret_cast<const double2*>(sm.rates[c][kq]);
        const double2 a0 = r2[0], a1 = r2[1], a2 = r2[2], a3 = r2[3];
        pv[0] = total + a0.x;
        pv[1] = pv[0] + a0.y;
        pv[2] = pv[1] + a1.x;
        pv[3] = pv[2] + a1.y;
        pv[4] = pv[3] + a2.x;
        pv[5] = pv[4] + a2.y;
        pv[6] = pv[5] + a3.x;
        pv[7] = pv[6] + a3.y;
        total = pv[7];
      } else {
        for (int i = 0; i < nord; ++i) {
          const double* r = sm.rates[c][sm.ord[c][i]];
#pragma unroll
          for (int bb = 0; bb < 8; ++bb) total += r[bb];
        }
      }
      if (a.mode == kModeCalc) {
        stop = 1;
      } else if (total == 0.0 || fabs(total) < DBL_EPSILON) {  // sublattice.inl:108-112
        stop = 2;
      } else {
        u = a.mode == kModeSelectPerform ? a.api_u : sm.ctl_u[it];
        const double expected = u * total;  // ModelAdapter::selectAndPerform
        if (nord == 1) {
#pragma unroll
          for (int q = 7; q >= 0; --q)
            if (pv[q] > expected) isel = q;
        } else {
          double acc = 0.0;
          for (int i = 0; i < nord && isel < 0; ++i) {
            const double* r = sm.rates[c][sm.ord[c][i]];
            for (int bb = 0; bb < 8; ++bb) {
              acc += r[bb];
              if (acc > expected) {
                isel = i * 8 + bb;
                break;
              }
            }
          }
        }
      }
    }
    isel = __shfl_sync(kFull, isel, 0);
    stop = __shfl_sync(kFull, stop, 0);
    HOP_T(0);
    if (stop) {
      if (tid == kCtl) {
        if (stop == 1) {  // akmc_calculate: the sector's vacancies with their jump rates
          *a.api_total = total;
          for (int i = 0; i < cnt; ++i) {
            a.api_sites[i] = sm.vact[c][i] ? sm.vlid[c][i] : -1;
            for (int bb = 0; bb < 8; ++bb) a.api_rates[i * 8 + bb] = sm.rates[c][i][bb];
          }
          *a.api_count = cnt;
        } else {
          if (a.mode == kModeSelectPerform) {
            a.api_event->from_site = -1;
            a.api_event->total = total;
          }
          sm.c_time = sm.c_thr;
        }
      }
      break;
    }
    // the selected jump: vacancy ksel of set c, direction bsel, atom X
    const bool hop = isel >= 0;
    const int bsel = hop ? (isel & 7) : 0;
    int ksel = kq;
    if (nord != 1) {  // several active vacancies: the selected one's record
      ksel = hop ? sm.ord[c][isel >> 3] : 0;
      const int4 qa = sm.vpk[c][ksel][0], qb = sm.vpk[c][ksel][1];
      s = qa.x;
      vx2 = qa.y;
      qy = qa.z;
      qz = qa.w;
      sX = qb.x;
      sY = qb.y;
      sZ = qb.z;
    }
    const int p = s & 1;
    const int X = hop ? sm.vX[c][ksel][bsel] : 0;
    const int32_t wg = sm.w1[p][bsel];
    const int snew = s + sm.d1[p][bsel];  // the vacancy's local site after the hop
    const int qx = vx2 >> 1;
    const int nlx = vx2 + unpack_dx(wg), nly = qy + unpack_dy(wg), nlz = qz + unpack_dz(wg);
    const bool nact = (nlx >> 1) >= R.hx && (nlx >> 1) < R.hx + R.w[0] && nly >= 2 && nly < 2 + R.w[1] &&
                      nlz >= 2 && nlz < 2 + R.w[2];
    const int ngx = wrap1(sX + unpack_dx(wg), jc.sx), ngy = wrap1(sY + unpack_dy(wg), jc.sy),
              ngz = wrap1(sZ + unpack_dz(wg), jc.sz);
    const int32_t to_g = ngx + jc.sx * (ngy + jc.sy * ngz);
    HOP_P(0);
    if (evaluator) {
      if (hop) {
        // [2] perform (ABVIModel::perform, kmc.cpp:358-396) on the staged region, written
        // through, and set n: items 0..77 the density deltas, 78 the occupancy swap, 79 the
        // ordered list, then one record and 8 rates per vacancy.  With 8 evaluator warps no warp
        // holds two kinds of item (a warp runs its kinds one after another): warps 0-2 the
        // deltas, warp 3 the swap, warp 4 the list, warps 5-7 the records and rates.
        const int nitems = kRefreshN + 2 + 9 * cnt;
        int i0 = tid, lim = nitems, step = kCtl;
        if (kEvalWarps == 8) {
          static_assert(kRefreshN <= 96, "three warps of density deltas");
          if (tid < 96) {
            lim = kRefreshN;
          } else if (tid == 96 || tid == 128) {
            i0 = tid == 96 ? kRefreshN : kRefreshN + 1;
            lim = i0 + 1;
          } else if (tid >= 160) {
            i0 = kRefreshN + 2 + (tid - 160);
            step = 96;
          } else {
            lim = 0;
          }
        }
        for (int i = i0; i < lim; i += step) {
          if (i < kRefreshN) {
            if (eam) {
              const int32_t e = sm.rl[p][bsel][i];
              const int j = s + local_delta(e, R);
              const int32_t v = rho_s[j] + sm.dfq[atom_index(static_cast<uint8_t>(X)) * 64 + rshells(e)];
              rho_s[j] = v;
              const int gx = wrap1(sX + unpack_dx(e), jc.sx), gy = wrap1(sY + unpack_dy(e), jc.sy),
                        gz = wrap1(sZ + unpack_dz(e), jc.sz);
              lattice_put(jc.rho + static_cast<int64_t>(jc.px) * (gy + static_cast<int64_t>(jc.sy) * gz), jc.sx, gx, v);
            }
          } else if (i == kRefreshN) {
            occ_s[snew] = kV;
            occ_s[s] = static_cast<uint8_t>(X);
            lattice_put(jc.occ + static_cast<int64_t>(jc.px) * (ngy + static_cast<int64_t>(jc.sy) * ngz), jc.sx, ngx,
                        static_cast<uint8_t>(kV));
            lattice_put(jc.occ + static_cast<int64_t>(jc.px) * (sY + static_cast<int64_t>(jc.sy) * sZ), jc.sx, sX,
                        static_cast<uint8_t>(X));
          } else if (i == kRefreshN + 1) {
            // the hopped vacancy leaves its place in the ordered list and re-enters at its new
            // site id if it is still inside the sector
            const int pos = isel >> 3;
            int m = 0;
            for (int q = 0; q < nord; ++q)
              if (q != pos) sm.ord[n][m++] = sm.ord[c][q];
            if (nact) {
              int j = m;
              while (j > 0 && sm.vlid[c][sm.ord[n][j - 1]] > to_g) {
                sm.ord[n][j] = sm.ord[n][j - 1];
                --j;
              }
              sm.ord[n][j] = ksel;
              ++m;
            }
            sm.nord[n] = m;
          } else if (i < kRefreshN + 2 + cnt) {
            const int k = i - kRefreshN - 2;
            if (k == ksel) {
              sm.vloc[n][k] = snew;
              sm.vlid[n][k] = to_g;
              sm.vcx[n][k] = static_cast<int16_t>(nlx);
              sm.vcy[n][k] = static_cast<int16_t>(nly);
              sm.vcz[n][k] = static_cast<int16_t>(nlz);
              sm.vgx[n][k] = ngx;
              sm.vgy[n][k] = ngy;
              sm.vgz[n][k] = ngz;
              sm.vact[n][k] = nact ? 1 : 0;
              sm.vpk[n][k][0] = make_int4(snew, nlx, nly, nlz);
              sm.vpk[n][k][1] = make_int4(ngx, ngy, ngz, to_g);
            } else {
              sm.vloc[n][k] = sm.vloc[c][k];
              sm.vlid[n][k] = sm.vlid[c][k];
              sm.vcx[n][k] = sm.vcx[c][k];
              sm.vcy[n][k] = sm.vcy[c][k];
              sm.vcz[n][k] = sm.vcz[c][k];
              sm.vgx[n][k] = sm.vgx[c][k];
              sm.vgy[n][k] = sm.vgy[c][k];
              sm.vgz[n][k] = sm.vgz[c][k];
              sm.vact[n][k] = sm.vact[c][k];
              sm.vpk[n][k][0] = sm.vpk[c][k][0];
              sm.vpk[n][k][1] = sm.vpk[c][k][1];
            }
          } else {
            // rates of vacancy q / 8, jump q % 8 carried over; the dirty ones are overwritten below
            const int q = i - kRefreshN - 2 - cnt;
            (&sm.rates[n][0][0])[q] = (&sm.rates[c][0][0])[q];
            (&sm.vX[n][0][0])[q] = (&sm.vX[c][0][0])[q];
          }
        }
        HOP_P(1);
        asm volatile("bar.sync 1, %0;" ::"n"(kCtl) : "memory");  // the evaluator warps only
        HOP_P(2);
        HOP_T(1);
        // [3] + [4] the vacancies within D cells of the hop's origin, evaluated into set n
        // (the hopped vacancy alone: dirty while it stays inside the sector, at its new site)
        for (int base = 0; base < cnt; base += 32) {
          const int k = base + lane;
          unsigned m = cnt == 1 ? (nact ? 1u : 0u) : __ballot_sync(kFull, k < cnt && dirty(n, k, qx, qy, qz));
          while (m) {
            const int kk = base + __ffs(m) - 1;
            m &= m - 1;
            const int l = cnt == 1 ? snew : sm.vloc[n][kk];
#pragma unroll
            for (int jj = 0; jj < kJumpsPerWarp; ++jj)
              eval_vacancy<KIND>(sm, n, occ_s, rho_s, kk, l, warp + kEvalWarps * jj, d1r[jj], FT, jc, jr[jj], nullptr);
          }
        }
        HOP_T(2);
      }
    } else {  // control warp: the hop's clock and event, the next iteration's decision and uniform
      int nd = 0;
      if (hop && cnt == 1) {
        nd = nact ? 1 : 0;
      } else if (hop) {
        // the dirty count, from set c with the hopped vacancy at its new cell
        for (int base = 0; base < cnt; base += 32) {
          const int k = base + lane;
          const bool d = k < cnt && (k == ksel ? nact : dirty(c, k, qx, qy, qz));
          nd += __popc(__ballot_sync(kFull, d));
        }
      }
      if (lane == 0) {
        const int nx = it ^ 1;
        int nstop = 0;
        if (a.mode == kModeSelectPerform) {  // the per-hop entry point stops after one selection
          akmc_event* e = a.api_event;
          e->round = 0;
          e->hop = sm.c_hop0;
          e->from_site = hop ? sm.vlid[c][ksel] : -1;
          e->to_site = hop ? to_g : -1;
          e->block = B.local_id;
          e->species = X;
          e->u = u;
          e->total = total;
          e->dt = 0.0;
          e->n_act = nord;
          e->n_dirty = nd;
          e->job = B.job;
          e->reserved = 0;
          if (hop) {
            sm.c_nh = 1;
            sm.c_evals += nd;
            sm.c_nact += nord;
          }
          nstop = 1;
        } else {
          // the selection used the uniform drawn ahead: the stream moves on
          for (int i = 0; i < 4; ++i) sm.xs[i] = sm.xsn[it][i];
          const double u2 = uniform_oc(sm.xt);  // sublattice.inl:118-120
          const double dt = -port_log(u2) / total;
          sm.c_time += dt;
          if (hop) {
            sm.c_nh += 1;
            sm.c_evals += nd;
            sm.c_nact += nord;
            if (a.log_cap > 0) {
              const unsigned long long slot = atomicAdd(a.log_count, 1ull);
              if (slot < static_cast<unsigned long long>(a.log_cap)) {
                akmc_event* e = a.log + slot;
                e->round = round_now;
                e->hop = sm.c_hop0 + sm.c_nh - 1;
                e->from_site = sm.vlid[c][ksel];
                e->to_site = to_g;
                e->block = B.local_id;
                e->species = X;
                e->u = u;
                e->total = total;
                e->dt = dt;
                e->n_act = nord;
                e->n_dirty = nd;
                e->job = B.job;
                e->reserved = 0;
              } else {
                atomicOr(a.status, kErrLogOverflow);
              }
            }
          }
          if (!(sm.c_time < sm.c_thr)) nstop = 1;
          if (sm.c_nh >= a.hop_cap) {
            atomicOr(a.status, kErrHopCap);
            nstop = 1;
          }
          if (!nstop) {  // the next selection's uniform, committed only if a selection uses it
            uint64_t x[4] = {sm.xs[0], sm.xs[1], sm.xs[2], sm.xs[3]};
            sm.ctl_u[nx] = uniform_co(x);
            for (int i = 0; i < 4; ++i) sm.xsn[nx][i] = x[i];
          }
        }
        sm.ctl_stop[nx] = nstop;
      }
      HOP_T(1);
    }
    __syncthreads();  // set n (or c), the clock's decision and the next uniform visible
    HOP_T(threadIdx.x == 0 ? 3 : 2);
    HOP_P(3);
#if defined(AKMC_PHASE_PROFILE) && defined(AKMC_HOP_PROFILE)
    if (tid == 0) atomicAdd(a.counters + 23, 1ull);
#endif
    AKMC_PHASE(5);
    if (hop) c = n;
    it ^= 1;
  }
  __syncthreads();
  AKMC_PHASE(6);
  if (tid == 0) sm.fin = c;  // every thread holds the same c
  if (a.mode == kModeCalc) return true;
  if (tid == kCtl) {
    const int64_t nh = sm.c_nh;
    if (a.mode == kModeRound) {
      // (k_flow read the clock while the region's copies flew: no second round trip)
      B.evo[sec] = (flowpre ? sm.pre_evo : __ldcg(&B.evo[sec])) + sm.c_time;
      for (int i = 0; i < 4; ++i) {
        B.xs[i] = sm.xs[i];
        B.xt[i] = sm.xt[i];
      }
    }
    B.hops = sm.c_hop0 + nh;
    sm.hops_out = sm.c_hop0 + nh;
    if (sm.acc_job != B.job) {
      if (sm.acc_job >= 0 && sm.acc_job_hops)
        atomicAdd(reinterpret_cast<unsigned long long*>(&a.jobs[sm.acc_job].hops), sm.acc_job_hops);
      sm.acc_job = B.job;
      sm.acc_job_hops = 0;
    }
    sm.acc_job_hops += static_cast<unsigned long long>(nh);
    sm.acc[0] += static_cast<unsigned long long>(nh);
    sm.acc[1] += static_cast<unsigned long long>(sm.c_evals);
    sm.acc[2] += 1ull;
    sm.acc[3] += static_cast<unsigned long long>(sm.c_nact);
    sm.acc[4] += static_cast<unsigned long long>(R.nt);
    sm.acc[5] += static_cast<unsigned long long>(nh * (eam ? 2 + kRefreshN : 2));
  }
  // the lattice was written through at every hop; only the vacancy positions remain
  if (tid < cnt) a.vac_site[sm.vidx[tid]] = sm.vlid[c][tid];
  return true;
}

// The region's arrays after Smem, each starting on a 128-byte boundary of the shared window
// (tensor copies want it; hop_smem_bytes leaves room for the padding).
__device__ __forceinline__ void carve(uint8_t* smem, int nreg, Smem*& sm, uint8_t*& occ_s, int32_t*& rho_s) {
  sm = reinterpret_cast<Smem*>(smem);
  uint8_t* p = smem + sizeof(Smem);
  p += (128u - (smem_u32(p) & 127u)) & 127u;
  rho_s = reinterpret_cast<int32_t*>(p);
  occ_s = occ_of(rho_s, nreg);
}

__device__ void dispatch_block(const RoundArgs& a, int gb, uint8_t* smem) {
  const BlockDev& B = a.blocks[gb];
  const JobDev& J = a.jobs[B.job];
  const int sec = a.mode == kModeRound ? sector_of_round(B.round) : a.api_sector;
  Region R;
  make_region(B, J, sec, R);
  Smem* sm;
  uint8_t* occ_s;
  int32_t* rho_s;
  carve(smem, R.n, sm, occ_s, rho_s);
  const int32_t* vl = a.blk_list + static_cast<int64_t>(gb) * kMaxV;
  const int cnt = min(B.cnt, kMaxV);
  if (J.model == AKMC_MODEL_PAIRBOND) run_block<kPairBond, 8>(a, gb, *sm, occ_s, rho_s, vl, cnt, B.round);
  else if (J.precision == AKMC_FP32C) run_block<kEam32, 8>(a, gb, *sm, occ_s, rho_s, vl, cnt, B.round);
  else run_block<kEam64, 8>(a, gb, *sm, occ_s, rho_s, vl, cnt, B.round);
}

__global__ void k_bucket(RoundArgs a) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= a.nvac) return;
  const int j = a.vac_job[v];
  if (j < 0) return;  // a free entry of the vacancy table (a context with room for admitted jobs)
  const JobDev& J = a.jobs[j];
  if (J.done) return;
  if (a.mode != kModeRound && j != a.api_job) return;
  const int sec = a.mode == kModeRound ? sector_of_round(J.round) : a.api_sector;
  const int s = a.vac_site[v];
  const int X = s % J.sx;
  const int t = s / J.sx;
  const int c[3] = {X >> 1, t % J.sy, t / J.sy};
  int k[3];
  for (int d = 0; d < 3; ++d) k[d] = block_of(c[d], J.n[d], J.nb[d]);
  const int gb = J.block0 + k[0] + J.nb[0] * (k[1] + J.nb[1] * k[2]);
  BlockDev& B = a.blocks[gb];
  for (int d = 0; d < 3; ++d) {
    const int half = (B.c1[d] - B.c0[d]) / 2;
    const int hi = (c[d] - B.c0[d]) >= half ? 1 : 0;
    if (hi != ((sec >> d) & 1)) return;
  }
  const int slot = atomicAdd(&B.cnt, 1);
  if (slot >= kMaxV) {
    atomicOr(a.status, kErrVacOverflow);
    return;
  }
  a.blk_list[static_cast<int64_t>(gb) * kMaxV + slot] = v;
  if (slot == 0) {
    const int q = atomicAdd(a.n_active, 1);
    a.active[q] = gb;
  }
}

__device__ void init_cta_smem(uint8_t* smem) {
  Smem* sm = reinterpret_cast<Smem*>(smem);
  if (threadIdx.x == 0) {
    sm->win_pot = -1;
    sm->tab_key[0] = sm->tab_key[1] = -1;
    sm->mbar_phase = 0;
    sm->mbst_phase = 0;
    mbar_init(&sm->mbar);
    mbar_init(&sm->mbar_st);
    for (int i = 0; i < 6; ++i) sm->acc[i] = 0;
    sm->acc_job = -1;
    sm->acc_job_hops = 0;
  }
  __syncthreads();
}

// Adds the CTA's counters (summed by the control thread) to the device counters; CTA-wide.
template <int W>
__device__ void cta_flush(const RoundArgs& a, uint8_t* smem) {
  AKMC_SHAPE(W);
  Smem* sm = reinterpret_cast<Smem*>(smem);
  __syncthreads();
  if (threadIdx.x == kCtl) {
    const int idx[6] = {0, 1, 3, 4, 5, 6};
    for (int i = 0; i < 6; ++i)
      if (sm->acc[i]) atomicAdd(a.counters + idx[i], sm->acc[i]);
    if (sm->acc_job >= 0 && sm->acc_job_hops)
      atomicAdd(reinterpret_cast<unsigned long long*>(&a.jobs[sm->acc_job].hops), sm->acc_job_hops);
  }
}

__device__ __forceinline__ int job_kind(const JobDev& J) {
  return J.model == AKMC_MODEL_PAIRBOND ? kPairBond : (J.precision == AKMC_FP32C ? kEam32 : kEam64);
}

// One kernel per energy kind, so each holds only its own hop loop (instruction-cache
// footprint); items of other kinds are left to their kernel.
template <int KIND, int W>
__global__ void __launch_bounds__(Shape<W>::kThreads, Shape<W>::kCtasPerSm) k_hop(RoundArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int na = *a.n_active;
  if (static_cast<int>(blockIdx.x) >= na) return;
  init_cta_smem(smem);
  for (int item = blockIdx.x; item < na; item += gridDim.x) {
    const int gb = a.active[item];
    const BlockDev& B = a.blocks[gb];
    if (job_kind(a.jobs[B.job]) != KIND) continue;
    Region R;
    make_region(B, a.jobs[B.job], sector_of_round(B.round), R);
    Smem* sm;
    uint8_t* occ_s;
    int32_t* rho_s;
    carve(smem, R.n, sm, occ_s, rho_s);
    run_block<KIND, W>(a, gb, *sm, occ_s, rho_s, a.blk_list + static_cast<int64_t>(gb) * kMaxV, min(B.cnt, kMaxV),
                       B.round);
  }
  cta_flush<W>(a, smem);
}

// ---------------------------------------------------------------------------
// Asynchronous round schedule.  A block's round r may run once, for every neighbour
// offset d in {-1,0,1}^3, the neighbour block has completed its latest earlier round
// whose staged region (sector plus a 2-cell halo) meets region r (flow_lag); rounds of
// different blocks then run in any order and the result equals the round-by-round
// schedule (sublattice.inl:61-179): a round reads and writes only its region, every
// write that a region can see comes from an earlier round that it waits for, and rounds
// that run at the same time have disjoint regions.  Each block keeps the ids of the
// vacancies in its area in kFlowSlots slots; a hop that carries a vacancy into a
// neighbour's area moves the id there.
//
// k_flow is persistent.  Each sweep a thread takes one block: while the block's next
// round is ready and its sector holds no vacancy, the thread runs that round alone (the
// clock jumps to the window, sublattice.inl:108-112); a ready round with vacancies is
// handed to the CTA, which runs the hop loop for it.  A block is held with a lease while
// anything works on it, and nothing waits while holding a lease.  The lease and the block's
// completed rounds share one 64-bit word (fstate = rounds << 1 | leased): one compare-and-swap
// reads the round and takes the lease, and one store after a fence publishes the rounds run
// and frees the lease together.  B.round is refreshed from the word when the launch ends.
// A single-block job's rounds depend on nothing else, so the CTA that ran one runs the next
// straight away when it holds no other round of the sweep (its hop budget is checked here, at
// each time-step boundary).

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Release/acquire fence at GPU scope (lighter than the sequentially consistent __threadfence).
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
#ifdef AKMC_PUBLISH_FENCE
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
#endif
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ unsigned int ld_relaxed_u32(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

// Rounds back to the latest earlier round of the neighbour at offset (dx, dy, dz) whose
// region meets this round's (phase = round mod 8), 0 if none ever does.  Per dimension a
// +1 neighbour's regions meet ours only between our high half and its low half (block
// edges >= 8 cells, halos of 2), a -1 neighbour's only between our low half and its high.
__device__ int flow_lag(int phase, int dx, int dy, int dz) {
  const int now = sector_of_round(phase);
  const int d[3] = {dx, dy, dz};
  for (int k = 1; k <= 8; ++k) {
    const int then = sector_of_round(phase + 8 - k);
    bool meet = true;
    for (int a = 0; a < 3; ++a) {
      const int hn = (now >> a) & 1, ht = (then >> a) & 1;
      if (d[a] == 1) meet = meet && hn == 1 && ht == 0;
      if (d[a] == -1) meet = meet && hn == 0 && ht == 1;
    }
    if (meet) return k;
  }
  return 0;
}

__device__ __forceinline__ int wrapb(int v, int m) { return v < 0 ? v + m : (v >= m ? v - m : v); }

// Global index of the neighbour of block local_id at offset o (o = (dz+1)*9 + (dy+1)*3 + dx+1).
__device__ __forceinline__ int flow_neighbour(const JobDev& J, int local_id, int o) {
  const int bx = local_id % J.nb[0], by = (local_id / J.nb[0]) % J.nb[1], bz = local_id / (J.nb[0] * J.nb[1]);
  return J.block0 + wrapb(bx + o % 3 - 1, J.nb[0]) +
         J.nb[0] * (wrapb(by + (o / 3) % 3 - 1, J.nb[1]) + J.nb[1] * wrapb(bz + o / 9 - 1, J.nb[2]));
}

// Whether round r of the block may run.  The neighbours' round counters are read with
// relaxed loads, all in flight at once, and a fence follows a positive answer (the acquire
// pattern): the writes of the rounds waited for become visible to this thread.
// A multi-block job with a hop budget ends at the end of the first time step at which the hops
// of all its blocks reach the budget, so its round b at a time-step boundary (b = 8, 16, ...)
// runs only once every block of the job has reached b; the blocks' hops at b (hops_at, written
// when each reached b) then decide.  Blocks of the job are thus never a whole time step apart,
// and the two hops_at slots never hold a boundary someone still reads.  Returns 0 while a block
// is behind, 1 to run round b, 2 when the job ends at b.
__device__ int budget_gate(const RoundArgs& a, const JobDev& J, int64_t b) {
  if (J.hop_budget <= 0 || J.nblocks == 1 || b == 0 || (b & 7)) return 1;
  bool all = true;
  for (int k = 0; k < J.nblocks; ++k)
    all &= static_cast<int64_t>(ld_relaxed_u64(&a.fstate[J.block0 + k]) >> 1) >= b;
  if (!all) return 0;
  fence_acq_rel();  // the hops_at written before those rounds were published
  const int slot = static_cast<int>((b >> 3) & 1);
  int64_t sum = 0;
  for (int k = 0; k < J.nblocks; ++k) sum += __ldcg(&a.blocks[J.block0 + k].hops_at[slot]);
  return sum >= J.hop_budget ? 2 : 1;
}

// Flags word of a block's row of RoundArgs::nbr: the energy kind (kNbrFree for a free block
// slot) and whether the job's hop budget gates its rounds at time-step boundaries (budget_gate).
constexpr int kNbrFree = 3, kNbrKindMask = 3, kNbrGate = 4;

// The neighbours' completed rounds relative to round r0 (P[o] = rounds - r0, clamped to
// +-2^30; the block itself never holds it back: 2^30), read with relaxed loads, all in flight at
// once, from the block's row of the neighbour table.  The caller fences after the loads (an
// acquire) before it reads what those rounds wrote.  (Relative int32 counts keep the snapshot in
// 27 registers.)
constexpr int32_t kAhead = 1 << 30;
// The block's row of the neighbour table: 27 neighbours and the flags word (y[27]).
__device__ __forceinline__ void flow_row(const RoundArgs& a, int gb, int (&y)[28]) {
  const int4* row = reinterpret_cast<const int4*>(a.nbr + static_cast<int64_t>(gb) * kNbrStride);
#pragma unroll
  for (int q = 0; q < 7; ++q) {
    const int4 v = __ldcg(row + q);
    y[4 * q] = v.x;
    y[4 * q + 1] = v.y;
    y[4 * q + 2] = v.z;
    y[4 * q + 3] = v.w;
  }
}
__device__ __forceinline__ void flow_snapshot(const RoundArgs& a, int gb, const int (&y)[28], int64_t r0,
                                              int32_t (&P)[27]) {
  // only the word's low 32 bits are read (27 registers in flight, not 54): neighbours of one job
  // are within a few rounds of each other, so the difference taken modulo 2^31 is exact
  const uint32_t base = static_cast<uint32_t>(r0) & 0x7fffffffu;
#pragma unroll
  for (int o = 0; o < 27; ++o) {
    if (y[o] == gb) {
      P[o] = kAhead;
    } else {
      const uint32_t lo = ld_relaxed_u32(reinterpret_cast<const unsigned int*>(&a.fstate[y[o]]));
      P[o] = static_cast<int32_t>(((lo >> 1) - base) << 1) >> 1;  // sign from bit 30
    }
  }
}

// Whether a snapshot relative to r0 lets round r0 + d run (the neighbours' rounds it waits for
// are complete).
__device__ __forceinline__ bool flow_ready(const int32_t (&P)[27], int64_t r0, int d, const int8_t (*lag)[27]) {
  const int ph = static_cast<int>((r0 + d) & 7);
  bool ok = true;
#pragma unroll
  for (int o = 0; o < 27; ++o) {
    const int k = lag[ph][o];
    if (k && P[o] < d - k + 1) ok = false;
  }
  return ok;
}

__device__ __forceinline__ bool site_in_sector(const BlockDev& B, const JobDev& J, int sec, int32_t s) {
  const int X = s % J.sx;
  const int t = s / J.sx;
  const int c[3] = {X >> 1, t % J.sy, t / J.sy};
  for (int d = 0; d < 3; ++d) {
    const int half = (B.c1[d] - B.c0[d]) / 2;
    const int lo = (sec >> d) & 1 ? B.c0[d] + half : B.c0[d];
    const int hi = (sec >> d) & 1 ? B.c1[d] : B.c0[d] + half;
    if (c[d] < lo || c[d] >= hi) return false;
  }
  return true;
}

// Block whose area holds site s (the reference's rank split, as k_bucket) and the sector of that
// block the site lies in.
__device__ __noinline__ int owner_sector(const JobDev& J, int32_t s, int* sec) {
  const int X = s % J.sx;
  const int t = s / J.sx;
  const int c[3] = {X >> 1, t % J.sy, t / J.sy};
  int k[3];
  int q = 0;
  for (int d = 0; d < 3; ++d) {
    k[d] = block_of(c[d], J.n[d], J.nb[d]);
    const int lo = k[d] * (J.n[d] / J.nb[d]) + min(k[d], J.n[d] % J.nb[d]);  // the rank split
    const int hi = (k[d] + 1) * (J.n[d] / J.nb[d]) + min(k[d] + 1, J.n[d] % J.nb[d]);
    if (c[d] - lo >= (hi - lo) / 2) q |= 1 << d;
  }
  *sec = q;
  return J.block0 + k[0] + J.nb[0] * (k[1] + J.nb[1] * k[2]);
}

// Puts vacancy v into block o's slots: claim a free slot, write the id, then mark it valid.
__device__ void flow_give(const RoundArgs& a, int o, int v, int32_t site, int osec) {
  for (int tries = 0; tries < 4 * kFlowSlots; ++tries) {
    const unsigned long long m = *reinterpret_cast<volatile unsigned long long*>(&a.vclaim[o]);
    if (m == ~0ull) break;
    const int slot = __ffsll(static_cast<long long>(~m)) - 1;
    const unsigned long long bit = 1ull << slot;
    if (atomicOr(&a.vclaim[o], bit) & bit) continue;  // taken meanwhile
    a.vslot[static_cast<int64_t>(o) * kFlowSlots + slot] = v;
    a.vsite[static_cast<int64_t>(o) * kFlowSlots + slot] = site;
    fence_acq_rel();
    atomicOr(&a.vvalid[o], bit);
    atomicOr(&a.vsec[o], 1u << osec);
    return;
  }
  atomicOr(a.status, kErrVacOverflow);
}

// Publishes the block's completed rounds (rn) and keeps (keep = 1) or frees the lease, with
// one release store.  Release is cumulative: writes of other threads of the CTA that a barrier
// ordered before this call are released too.  (-DAKMC_PUBLISH_FENCE: a fence and a relaxed
// store instead, the form measured before.)  `reached`: this lease holder moved the
// block onto its target (each block is counted once).
__device__ __forceinline__ void flow_publish(const RoundArgs& a, int gb, int64_t rn, int keep, bool reached,
                                             int kind) {
#ifdef AKMC_PUBLISH_FENCE
  fence_acq_rel();
  st_relaxed_u64(&a.fstate[gb], (static_cast<unsigned long long>(rn) << 1) | static_cast<unsigned long long>(keep));
#else
  st_release_u64(&a.fstate[gb], (static_cast<unsigned long long>(rn) << 1) | static_cast<unsigned long long>(keep));
#endif
  if (reached) atomicAdd(&a.flow_done[kind], 1);
}

// Lease held, one thread, the block at round r0: runs the block's ready rounds whose sectors
// hold no vacancy (the clock jumps to the window, sublattice.inl:108-112), up to 64 in one
// batch, and leaves the block's round in *rn (the caller publishes it).  A round is ready when
// the snapshot of the neighbours' round counters (the sweep's, Pin, or one read here with all
// loads in flight together) already covers it, and the vacancy slots read after the snapshot
// hold every vacancy those rounds can see (a round that could bring one into such a sector
// overlaps it, so it is in the snapshot).  Returns true when it stops at a ready round with vacancies, false when the next
// round is not ready or the target is reached.  *reached: this call moved the block onto its
// target (by running rounds, or by a budget moving the target down to r0); false for a block
// that was at its target already (a stale sweep read).
__device__ bool flow_advance(const RoundArgs& a, BlockDev& B, const JobDev& J, int gb, const int8_t (*lag)[27],
                             int64_t r0, const int32_t (*Pin)[27], int64_t* rn, bool* reached, int64_t* tgt,
                             unsigned long long* vv = nullptr) {
  *rn = r0;
  *reached = false;
  // one round of loads, all in flight together: the target, the job's constants, the block's
  // hops and clocks and its vacancy slots (the lease is held: nothing else writes them but gives)
  const int64_t t_old = __ldcg(&B.target);
  const int64_t hops = __ldcg(&B.hops);  // empty rounds add none
  const int nbl = J.nblocks;
  const int64_t budget = J.hop_budget;
  const double window = J.window;
  double evo[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) evo[k] = __ldcg(&B.evo[k]);
  // sectors holding a vacancy (the slots' sector mask)
  unsigned occ_sec = __ldcg(&a.vsec[gb]);
  // and, for the round this call may hand over, the valid bits of the block's vacancy slots, read
  // last and with acquire: the slots' ids and sites (written before a give sets its bit) are read
  // after it, by the CTA's threads past a barrier.  Every vacancy that can lie in the round's
  // sector came with a round this lease's snapshot covers; only the lease holder clears bits.
  if (vv) *vv = ld_acquire_u64(&a.vvalid[gb]);
  *tgt = t_old;
  if (r0 >= t_old) return false;
  // a single-block job with a hop budget ends at the end of the first time step at which its
  // hops reached the budget: once they have, its target moves down to the next boundary at or
  // after r0 (never below r0)
  int64_t target = t_old;
  if (nbl == 1 && budget > 0 && hops >= budget) {
    const int64_t b = (r0 + 7) & ~static_cast<int64_t>(7);
    if (b < target) {
      target = b;
      B.target = b;
      B.budget_end = 1;
    }
  }
  *tgt = target;
  if (r0 >= target) {
    *reached = true;
    return false;
  }
  // the sweep's snapshot, taken before the lease and fenced after it (rounds only grow, so an
  // earlier snapshot is a safe one), or a fresh one
  int32_t P[27];
  if (Pin) {
#pragma unroll
    for (int o = 0; o < 27; ++o) P[o] = (*Pin)[o];
  } else if (J.nblocks == 1) {  // every neighbour is the block itself: nothing to wait for
#pragma unroll
    for (int o = 0; o < 27; ++o) P[o] = kAhead;
  } else {
    int y[28];
    flow_row(a, gb, y);
    flow_snapshot(a, gb, y, r0, P);
    fence_acq_rel();
    occ_sec = __ldcg(&a.vsec[gb]);  // with the vacancies those rounds gave the block
  }
  const int64_t last = min(target, r0 + 64);
  int64_t r = r0;
  bool stop_full = false;
  while (r < last) {
    if (!flow_ready(P, r0, static_cast<int>(r - r0), lag)) break;
    const int g = budget_gate(a, J, r);
    if (g == 0) break;
    if (g == 2) {  // the job ends at this boundary: the block's target moves down to it
      B.target = r;
      B.budget_end = 1;
      target = r;
      *tgt = r;
      break;
    }
    const int sec = sector_of_round(r);
    if ((occ_sec >> sec) & 1u) {
      stop_full = true;
      break;
    }
    double e = evo[0];
#pragma unroll
    for (int k = 1; k < 8; ++k) e = k == sec ? evo[k] : e;
    const double thr = static_cast<double>((r >> 3) + 1) * window - e;
    double sector_time = 0.0;
    if (sector_time < thr) sector_time = thr;
    const double ne = e + sector_time;
#pragma unroll
    for (int k = 0; k < 8; ++k) evo[k] = k == sec ? ne : evo[k];
    ++r;
    if ((r & 7) == 0) B.hops_at[(r >> 3) & 1] = hops;
  }
  if (r > r0) {
#pragma unroll
    for (int k = 0; k < 8; ++k) B.evo[k] = evo[k];
  }
  *rn = r;
  *reached = r == target;  // the lease holder alone moves the target
  *tgt = target;
  return stop_full;
}

// Rounds with vacancies a CTA takes per sweep: a.flow_take (0: every ready round its threads
// found).  Measured on the 256^3 lattice and the 512 batched boxes: taking every ready round
// found, one round per block at a time, beats taking one per sweep (others left to idle CTAs)
// and beats chaining up to 8 rounds of one block of a multi-block job.  Single-block jobs chain:
// their next round waits for nothing.
template <int KIND, int W>
__global__ void __launch_bounds__(Shape<W>::kThreads, Shape<W>::kCtasPerSm) k_flow(RoundArgs a) {
  AKMC_SHAPE(W);
  const int kFlowTake = a.flow_take > 0 && a.flow_take < kThreads ? a.flow_take : kThreads;
  extern __shared__ __align__(16) uint8_t smem[];
  Smem* sm0 = reinterpret_cast<Smem*>(smem);
  const int tid = threadIdx.x;
  init_cta_smem(smem);
  for (int i = tid; i < 8 * 27; i += kThreads) {
    const int o = i % 27;
    sm0->flow_lag[i / 27][o] = static_cast<int8_t>(flow_lag(i / 27, o % 3 - 1, (o / 3) % 3 - 1, o / 9 - 1));
  }
  const int nb = a.nblocks;
  int cursor = static_cast<int>((static_cast<int64_t>(blockIdx.x) * nb) / gridDim.x);
  const uint64_t t_begin = globaltimer_ns();  // a time-boxed launch takes no new round after its budget
  if (tid == 0) sm0->flow_stop = 0;
#ifdef AKMC_PHASE_PROFILE
  long long t_sweep = 0, t_hop = 0, n_sweep = 0, n_full = 0, t0 = 0;
#endif
  for (int64_t sweep = 0;; ++sweep) {
#ifdef AKMC_PHASE_PROFILE
    if (tid == 0) t0 = clock64();
#endif
    if (tid == 0) {
      sm0->flow_ncand = 0;
      sm0->flow_progress = 0;
    }
    __syncthreads();
    if (sm0->flow_stop) break;  // decided during the previous sweep
    // thread 0 reads the launch's progress and status while the sweep's visits are in flight,
    // and decides after its own visit whether the CTA stops after this sweep's rounds
    int need = 0, done = 0;
    unsigned st = 0;
    if (tid == 0) {
      need = *reinterpret_cast<volatile int*>(&a.flow_need[KIND]);
      done = *reinterpret_cast<volatile int*>(&a.flow_done[KIND]);
      st = *reinterpret_cast<volatile unsigned*>(a.status);
    }

    // sweep: thread tid looks after blocks (cursor + tid + k kThreads) mod nb, k < kSweepVisits,
    // until it takes one: a visit that finds nothing to do ends after one or two round trips,
    // while the sweep lasts as long as its slowest visit (one that takes a block)
#pragma unroll 1
    for (int vis = 0; vis < kSweepVisits; ++vis) {
      const int off = tid + vis * kThreads;
      if (off >= nb) break;
      int gb = cursor + off;
      if (gb >= nb) gb -= nb;
      BlockDev& B = a.blocks[gb];
      // one round of loads decides whether to look closer: the block's word, target, job, and its
      // row of the neighbour table with the flags (energy kind, free slot)
      int y[28];
      flow_row(a, gb, y);
      const unsigned long long w = ld_relaxed_u64(&a.fstate[gb]);
      const int64_t t0 = __ldcg(&B.target);
      const int bj = __ldcg(&B.job);
      const int64_t r = static_cast<int64_t>(w >> 1);
      int32_t P[27];
      bool ok = (y[27] & kNbrKindMask) == KIND && !(w & 1ull) && r < t0;
      if (ok) {  // a second: the neighbours' rounds
        flow_snapshot(a, gb, y, r, P);
        ok = flow_ready(P, r, 0, sm0->flow_lag);
      }
      // a multi-block job with a hop budget: its round at a time-step boundary waits for the job's
      // other blocks (a job that ends there is taken, to mark it)
      if (ok && (y[27] & kNbrGate) && budget_gate(a, a.jobs[bj], r) == 0) ok = false;
      // the lease, then one fence: the snapshot's and the word's reads become acquires
      if (ok && atomicCAS(&a.fstate[gb], w, w | 1ull) == w) {
        fence_acq_rel();
        const JobDev& J = a.jobs[bj];
        int64_t rn = r, tgt = 0;
        int keep = 0;
        bool reached = false;
        unsigned long long vv = 0;
        if (flow_advance(a, B, J, gb, sm0->flow_lag, r, &P, &rn, &reached, &tgt, &vv)) {
          const int i = atomicAdd(&sm0->flow_ncand, 1);
          if (i < kFlowTake) {
            sm0->flow_cand[i] = gb;
            sm0->flow_cvv[i] = vv;
            sm0->flow_cr[i] = rn;
            sm0->flow_ct[i] = tgt;
            keep = 1;
          }
        }
        if (rn > r) sm0->flow_progress = 1;
        flow_publish(a, gb, rn, keep, reached, KIND);
        break;
      }
    }
    if (tid == 0) {
      int stop = done >= need || (st & (kErrVacOverflow | kErrRhoRange | kErrHopCap | kErrTimeout)) != 0;
      if (a.time_budget_ns > 0 && globaltimer_ns() - t_begin >= static_cast<uint64_t>(a.time_budget_ns)) stop = 1;
      if (!stop && sweep + 1 >= a.flow_sweep_limit) {  // watchdog; the default 2^24 no launch of <= 1024 rounds needs
        atomicOr(a.status, kErrTimeout);
        stop = 1;
      }
      sm0->flow_stop = stop;
    }
    __syncthreads();
#ifdef AKMC_PHASE_PROFILE
    if (tid == 0) {
      const long long t1 = clock64();
      t_sweep += t1 - t0;
      t0 = t1;
      ++n_sweep;
    }
#endif

    // the hop loop for each round handed over; a single-block job's next rounds follow while
    // the launch's target allows (empty ones in between run on thread 0)
    const int ncand = min(sm0->flow_ncand, kFlowTake);
    for (int c = 0; c < ncand; ++c) {
      const int gb = sm0->flow_cand[c];
      // the round and target the sweep left (a chained round: the previous link's)
      int64_t r = sm0->flow_cr[c], target = sm0->flow_ct[c];
      for (int link = 0;; ++link) {
#ifdef AKMC_PHASE_PROFILE
        long long tw = clock64();
#endif
        BlockDev& B = a.blocks[gb];
        const JobDev& J = a.jobs[B.job];
        // the thread that found this round ready read the neighbours' round counters and then
        // fenced (an acquire), and a CTA barrier followed: every thread's reads come after the
        // rounds it waits for (shared data is read at L2)
        const int sec = sector_of_round(r);
        Region R;
        make_region(B, J, sec, R);
        Smem* sm;
        uint8_t* occ_s;
        int32_t* rho_s;
        carve(smem, R.n, sm, occ_s, rho_s);
        if (tid == 0) {
          sm->fnv = 0;
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            sm->bc0[d] = B.c0[d];
            sm->bc1[d] = B.c1[d];
          }
          sm->bnb = J.nblocks;
        }
        if (R.bulk && tid == kCtl) bulk_expect(&sm->mbar_st, stage_bytes(R, KIND != kPairBond));
        __syncthreads();  // the previous round's readers are done; the copies' barrier is armed
        // the region's bulk copies first: the slots, clocks and streams are read while they fly
        if (R.tma) {
          if (tid == kCtl) stage_tensor(R, a.tmaps, B.job, KIND != kPairBond, occ_s, rho_s, &sm->mbar_st);
        } else if (R.bulk) {
          stage_rows(R, J.occ, J.rho, J.px, J.sy, J.sz, KIND != kPairBond, occ_s, rho_s, &sm->mbar_st, tid, kThreads);
        }
        if (tid < kFlowSlots) {
          // the sweep read the valid bits when it handed the round over; a chained round reads them
          const unsigned long long m = link == 0 ? sm0->flow_cvv[c] : ld_acquire_u64(&a.vvalid[gb]);
          if ((m >> tid) & 1ull) {
            const int v = __ldcg(&a.vslot[static_cast<int64_t>(gb) * kFlowSlots + tid]);
            const int32_t st = __ldcg(&a.vsite[static_cast<int64_t>(gb) * kFlowSlots + tid]);
            if (site_in_sector(B, J, sec, st)) {
              const int i = atomicAdd(&sm->fnv, 1);
              sm->fv[i] = v;
              sm->fsite[i] = st;
              sm->fslot[i] = tid;
            }
          }
        } else if (tid < kFlowSlots + 10) {
          // the block's hops, the sector's clock and the two streams, one value per thread, while
          // the control thread issues the copies
          const int q = tid - kFlowSlots;
          if (q == 0) sm->hops_out = __ldcg(&B.hops);  // run_block replaces it if the round runs
          else if (q == 1) sm->pre_evo = __ldcg(&B.evo[sec]);
          else if (q < 6) sm->xs[q - 2] = __ldcg(&B.xs[q - 2]);
          else sm->xt[q - 6] = __ldcg(&B.xt[q - 6]);
        }
        __syncthreads();
        const int cnt = sm->fnv;
#ifdef AKMC_PHASE_PROFILE
        if (tid == 0) {
          atomicAdd(a.counters + 12, static_cast<unsigned long long>(clock64() - tw));  // [4] before the hop loop
          tw = clock64();
        }
#endif
        const bool ran = run_block<KIND, W>(a, gb, *sm, occ_s, rho_s, sm->fv, cnt, r, true);
#ifdef AKMC_PHASE_PROFILE
        if (tid == 0) tw = clock64();
#endif
        // the sector's vacancies move: its bit of the block's sector mask goes, and comes back
        // below for each one still in the block (with the bit of the sector it is in now)
        if (ran && tid == 0) atomicAnd(&a.vsec[gb], ~(1u << sector_of_round(r)));
        __syncthreads();
        // vacancies carried into a neighbour's area change owner (only if the round ran:
        // otherwise nothing moved and the vacancy arrays of sm hold another round's data)
        if (ran && tid < cnt) {
          // a vacancy still inside the block's area keeps its owner and slot (its site updated);
          // only one that left it needs the owner lookup
          const int f = sm->fin;
          const int cx = sm->vgx[f][tid] >> 1, cy = sm->vgy[f][tid], cz = sm->vgz[f][tid];
          const int* c0 = sm->bc0;
          const int* c1 = sm->bc1;
          const bool inside = cx >= c0[0] && cx < c1[0] && cy >= c0[1] && cy < c1[1] && cz >= c0[2] && cz < c1[2];
          const int32_t site = sm->vlid[f][tid];
          int osec = 0, o = gb;
          if (inside)
            osec = (cx - c0[0] >= (c1[0] - c0[0]) / 2 ? 1 : 0) | (cy - c0[1] >= (c1[1] - c0[1]) / 2 ? 2 : 0) |
                   (cz - c0[2] >= (c1[2] - c0[2]) / 2 ? 4 : 0);
          else
            o = owner_sector(J, site, &osec);
          if (o == gb) {
            a.vsite[static_cast<int64_t>(gb) * kFlowSlots + sm->fslot[tid]] = site;
            atomicOr(&a.vsec[gb], 1u << osec);
          } else {
            flow_give(a, o, sm->vidx[tid], site, osec);
            const unsigned long long bit = 1ull << sm->fslot[tid];
            atomicAnd(&a.vvalid[gb], ~bit);
            fence_acq_rel();
            atomicAnd(&a.vclaim[gb], ~bit);
          }
        }
        __syncthreads();
        if (tid == 0) {
#ifdef AKMC_FLOW_PROFILE
          const long long q0 = clock64();
#endif
          // round r ran (it was below the target when handed over); the target is the lease
          // holder's to move, and it is this CTA
          int64_t rn = r + 1, tgt = target;
          if ((rn & 7) == 0) B.hops_at[(rn >> 3) & 1] = sm->hops_out;
          bool more = false, reached = rn >= target;
          const bool in_time =
              a.time_budget_ns <= 0 || globaltimer_ns() - t_begin < static_cast<uint64_t>(a.time_budget_ns);
          if (!reached && sm->bnb == 1 && c + 1 == ncand && in_time) {
            // a single-block job: its next rounds wait for nothing, so keep the lease and run on
            // -- when no other round this CTA took in the sweep is waiting for it
            more = flow_advance(a, B, J, gb, sm0->flow_lag, r + 1, nullptr, &rn, &reached, &tgt);
          }
#ifdef AKMC_FLOW_PROFILE
          const long long q1 = clock64();
#endif
          sm->flow_progress = 1;
          sm->flow_more = more;
          sm->cur_r = rn;
          sm->cur_t = tgt;
          flow_publish(a, gb, rn, more ? 1 : 0, reached, KIND);
#ifdef AKMC_FLOW_PROFILE
          atomicAdd(a.counters + 20, static_cast<unsigned long long>(q1 - q0));
          atomicAdd(a.counters + 21, static_cast<unsigned long long>(clock64() - q1));
          atomicAdd(a.counters + 23, static_cast<unsigned long long>(q0 - tw));
#endif
        }
        __syncthreads();
#ifdef AKMC_PHASE_PROFILE
        if (tid == 0) {
          ++n_full;
          atomicAdd(a.counters + 15, static_cast<unsigned long long>(clock64() - tw));  // [7] after the hop loop
        }
#endif
        if (!sm0->flow_more) break;
        r = sm0->cur_r;
        target = sm0->cur_t;
      }
    }
#ifdef AKMC_PHASE_PROFILE
    if (tid == 0) t_hop += clock64() - t0;
#endif
    if (AKMC_SWEEP_SLEEP_NS > 0 && !sm0->flow_progress) __nanosleep(AKMC_SWEEP_SLEEP_NS);
    cursor += kSweepVisits * kThreads;
    if (cursor >= nb) cursor %= nb;
  }
  cta_flush<W>(a, smem);
#if defined(AKMC_PHASE_PROFILE) && !defined(AKMC_FLOW_PROFILE) && !defined(AKMC_HOP_PROFILE)
  if (tid == 0) {  // scheduler profile: [12] sweep cycles, [13] hop-loop cycles, [14] sweeps, [15] full rounds
    atomicAdd(a.counters + 20, static_cast<unsigned long long>(t_sweep));
    atomicAdd(a.counters + 21, static_cast<unsigned long long>(t_hop));
    atomicAdd(a.counters + 22, static_cast<unsigned long long>(n_sweep));
    atomicAdd(a.counters + 23, static_cast<unsigned long long>(n_full));
  }
#endif
}

// Per block: target round of this launch, lease and slots cleared; counts the blocks with
// rounds to run per energy kind.
__global__ void k_flow_prep(RoundArgs a) {
  const int gb = blockIdx.x * blockDim.x + threadIdx.x;
  if (gb >= a.nblocks) return;
  BlockDev& B = a.blocks[gb];
  B.cnt = 0;
  a.vclaim[gb] = 0;
  a.vvalid[gb] = 0;
  a.vcount[gb] = 0;
  a.vsec[gb] = 0;
  int32_t* row = a.nbr + static_cast<int64_t>(gb) * kNbrStride;
  if (B.job < 0) {  // a free block slot: nothing to run
    B.target = B.round;
    a.fstate[gb] = static_cast<unsigned long long>(B.round) << 1;
    for (int o = 0; o < 27; ++o) row[o] = gb;
    row[27] = kNbrFree;
    return;
  }
  const JobDev& J = a.jobs[B.job];
  for (int o = 0; o < 27; ++o) row[o] = flow_neighbour(J, B.local_id, o);
  row[27] = job_kind(J) | (J.hop_budget > 0 && J.nblocks > 1 ? kNbrGate : 0);
  // up to flow_rounds of the block's remaining rounds (hop budgets are checked by the kernel,
  // at time-step boundaries); a block sitting at a boundary records its hops there
  int64_t L = B.remaining < a.flow_rounds ? B.remaining : a.flow_rounds;
  if ((B.round & 7) == 0) B.hops_at[(B.round >> 3) & 1] = B.hops;
  int64_t t = B.done ? B.round : B.round + L;
  B.budget_end = 0;  // a budget that ends the job moves this target down again inside the launch
  if (J.max_rounds > 0 && t > J.max_rounds) t = J.max_rounds > B.round ? J.max_rounds : B.round;
  B.remaining -= t - B.round;
  B.target = t;
  a.fstate[gb] = static_cast<unsigned long long>(B.round) << 1;
  if (t > B.round) atomicAdd(&a.flow_need[job_kind(J)], 1);
}

// Per vacancy: into the slots of the block whose area holds it.
__global__ void k_flow_slots(RoundArgs a) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= a.nvac || a.vac_job[v] < 0) return;
  const JobDev& J = a.jobs[a.vac_job[v]];
  int osec = 0;
  const int o = owner_sector(J, a.vac_site[v], &osec);
  const int slot = atomicAdd(&a.vcount[o], 1);
  if (slot >= kFlowSlots) {
    atomicOr(a.status, kErrVacOverflow);
    return;
  }
  a.vslot[static_cast<int64_t>(o) * kFlowSlots + slot] = v;
  a.vsite[static_cast<int64_t>(o) * kFlowSlots + slot] = a.vac_site[v];
  atomicOr(&a.vclaim[o], 1ull << slot);
  atomicOr(&a.vvalid[o], 1ull << slot);
  atomicOr(&a.vsec[o], 1u << osec);
}

// After the flow kernels: job round and done flags as k_finalize leaves them.
__global__ void k_flow_finalize(RoundArgs a) {
  const int gb = blockIdx.x * blockDim.x + threadIdx.x;
  if (gb == 0 && a.time_budget_ns <= 0) atomicAdd(a.counters + 2, static_cast<unsigned long long>(a.flow_rounds));
  if (gb >= a.nblocks) return;
  BlockDev& B = a.blocks[gb];
  B.cnt = 0;
  B.round = static_cast<int64_t>(a.fstate[gb] >> 1);
  if (B.job < 0) return;
  // rounds of the call a time-boxed launch left to run go back to the block's remaining ones
  if (B.target > B.round) B.remaining += B.target - B.round;
  JobDev& J = a.jobs[B.job];
  // a hop budget ended the job inside the launch (the block reached the boundary its budget set);
  // or, when every block ran to the call's target (no time box), the job's hops (J.hops, added
  // when k_flow ended) reach the budget on a time-step boundary, as the round-by-round finalize
  // decides
  const int done = B.done || (J.max_rounds > 0 && B.round >= J.max_rounds) || (B.budget_end && B.round >= B.target) ||
                   (a.time_budget_ns <= 0 && J.hop_budget > 0 && (B.round & 7) == 0 && J.hops >= J.hop_budget);
  B.done = done;
  if (B.local_id == 0) {
    J.round = B.round;
    J.done = done;
  }
}

__global__ void k_finalize(RoundArgs a) {
  const int gb = blockIdx.x * blockDim.x + threadIdx.x;
  if (gb == 0) {
    *a.n_active = 0;
    atomicAdd(a.counters + 2, 1ull);
  }
  if (gb >= a.nblocks) return;
  BlockDev& B = a.blocks[gb];
  const int had = B.cnt;
  B.cnt = 0;
  if (B.job < 0) return;  // a free block slot
  JobDev& J = a.jobs[B.job];
  // J.done is only written here, by the job's block 0, so other blocks read their own flag
  if (B.done) return;
  if (had == 0) {  // no vacancy in the sector: total = 0, sector_time = threshold (sublattice.inl:108-112)
    const int sec = sector_of_round(B.round);
    const int64_t step = B.round >> 3;
    const double thr = static_cast<double>(step + 1) * J.window - B.evo[sec];
    double sector_time = 0.0;
    if (sector_time < thr) sector_time = thr;
    B.evo[sec] += sector_time;
  }
  B.round += 1;
  // a hop budget is checked at time-step boundaries (every 8 rounds)
  const int done = (J.hop_budget > 0 && (B.round & 7) == 0 && J.hops >= J.hop_budget) ||
                   (J.max_rounds > 0 && B.round >= J.max_rounds);
  B.done = done;
  if (B.local_id == 0) {
    J.round = B.round;
    J.done = done;
  }
}

__global__ void __launch_bounds__(Shape<8>::kThreads, 1) k_api_block(RoundArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  const JobDev& J = a.jobs[a.api_job];
  if (*a.n_active == 0) {  // no vacancy in the sector
    if (threadIdx.x == 0) {
      if (a.mode == kModeCalc) {
        *a.api_total = 0.0;
        *a.api_count = 0;
      } else {
        a.api_event->from_site = -1;
        a.api_event->total = 0.0;
      }
    }
    return;
  }
  init_cta_smem(smem);
  dispatch_block(a, J.block0, smem);
  cta_flush<8>(a, smem);
}
__global__ void k_api_reset(RoundArgs a) {
  const JobDev& J = a.jobs[a.api_job];
  a.blocks[J.block0].cnt = 0;
  *a.n_active = 0;
}

// Density cache of a whole lattice: rho_i = sum over the 58 neighbours j within the cutoff of
// f_{X_j}(shell) in Q.24.  A CTA takes tiles of 32 x 8 x 4 sites (x doubled), stages each with
// its halo (4 sites in x, 2 in y and z, periodic) and the f table by occupancy code in shared
// memory, and sums from there.  The 58 neighbours of the 5 BCC shells are a fixed geometric
// set, enumerated at compile time: every term is one byte read of the tile and one read of the
// f table at immediate offsets.  The sums are exact integers, so the term order does not matter.
constexpr int kRhoTX = 32, kRhoTY = 8, kRhoTZ = 4, kRhoHX = 4, kRhoHY = 2, kRhoHZ = 2;
constexpr int kRhoLX = kRhoTX + 2 * kRhoHX, kRhoLY = kRhoTY + 2 * kRhoHY, kRhoLZ = kRhoTZ + 2 * kRhoHZ;

struct RhoNb {
  int off, sh;  // tile offset, shell code 1..5
};
// Squared distance of sites (X0, 0, 0) and (X0 + dX, dy, dz) in (a/2)^2 units: corner sites
// (X even) sit at (X, 2y, 2z), centre sites at (X, 2y + 1, 2z + 1).
__host__ __device__ constexpr int rho_d2(int p0, int dX, int dy, int dz) {
  const int p1 = (p0 + dX) & 1;
  const int hy = 2 * dy + p1 - p0, hz = 2 * dz + p1 - p0;
  return dX * dX + hy * hy + hz * hz;
}
__host__ __device__ constexpr int rho_shell(int d2) {
  return d2 == 3 ? 1 : d2 == 4 ? 2 : d2 == 8 ? 3 : d2 == 11 ? 4 : d2 == 12 ? 5 : 0;
}
// k-th neighbour (k < 58) of a site of x parity p within the 5 shells.
__host__ __device__ constexpr RhoNb rho_nbr(int p, int k) {
  int n = 0;
  for (int dz = -2; dz <= 2; ++dz)
    for (int dy = -2; dy <= 2; ++dy)
      for (int dX = -4; dX <= 4; ++dX) {
        const int sh = (dX || dy || dz) ? rho_shell(rho_d2(p, dX, dy, dz)) : 0;
        if (!sh) continue;
        if (n == k) return RhoNb{dX + kRhoLX * (dy + kRhoLY * dz), sh};
        ++n;
      }
  return RhoNb{0, 0};
}
__host__ __device__ constexpr int rho_count(int p) {
  int n = 0;
  for (int dz = -2; dz <= 2; ++dz)
    for (int dy = -2; dy <= 2; ++dy)
      for (int dX = -4; dX <= 4; ++dX) n += (dX || dy || dz) && rho_shell(rho_d2(p, dX, dy, dz)) ? 1 : 0;
  return n;
}
static_assert(rho_count(0) == kShellNb && rho_count(1) == kShellNb, "58 neighbours in the 5 BCC shells");

template <int P, int K>
__device__ __forceinline__ int32_t rho_terms(const uint8_t* t, const int32_t* fqc) {
  if constexpr (K == kShellNb) {
    return 0;
  } else {
    constexpr RhoNb e = rho_nbr(P, K);
    return fqc[t[e.off] * 8 + e.sh] + rho_terms<P, K + 1>(t, fqc);
  }
}

// f in Q.24 by occupancy code and shell into shared memory; V and other codes 0.
__device__ void rho_table(int32_t* fqc, const Potential* pot) {
  for (int i = threadIdx.x; i < 16 * 8; i += blockDim.x) {
    const int code = i >> 3;
    const bool atom = code == 1 || code == 2 || code == 4 || code == 8;
    fqc[i] = atom ? pot->fq[species_index(static_cast<uint8_t>(code))][i & 7] : 0;
  }
}

// One tile of the density build (tix-th tile of the lattice); CTA-collective, 256 threads.
__device__ void rho_tile(const uint8_t* occ, int32_t* rho, int32_t sx, int32_t sy, int32_t sz, int32_t px, int64_t tix,
                         uint8_t* tile, const int32_t* fqc) {
  const int tid = threadIdx.x;
  const int nx = (sx + kRhoTX - 1) / kRhoTX, ny = (sy + kRhoTY - 1) / kRhoTY;
  const int x0 = static_cast<int>(tix % nx) * kRhoTX;
  const int y0 = static_cast<int>((tix / nx) % ny) * kRhoTY;
  const int z0 = static_cast<int>(tix / (static_cast<int64_t>(nx) * ny)) * kRhoTZ;
  __syncthreads();  // table written; the previous tile's readers are done
  for (int i = tid; i < kRhoLX * kRhoLY * kRhoLZ; i += blockDim.x) {
    const int lx = i % kRhoLX, t = i / kRhoLX, ly = t % kRhoLY, lz = t / kRhoLY;
    // periodic wrap without division: coordinates start at most one halo below 0 and end
    // below 3 box lengths (sx >= 16 sites, sy, sz >= 8 cells)
    int gx = x0 - kRhoHX + lx, gy = y0 - kRhoHY + ly, gz = z0 - kRhoHZ + lz;
    gx += gx < 0 ? sx : 0;
    gy += gy < 0 ? sy : 0;
    gz += gz < 0 ? sz : 0;
#pragma unroll
    for (int w = 0; w < 2; ++w) {
      gx -= gx >= sx ? sx : 0;
      gy -= gy >= sy ? sy : 0;
      gz -= gz >= sz ? sz : 0;
    }
    tile[i] = __ldg(occ + kHaloL + gx + static_cast<int64_t>(px) * (gy + static_cast<int64_t>(sy) * gz));
  }
  __syncthreads();
  // each warp takes sites of one x parity (both parities' sums are unrolled code): warp w
  // covers rows 2 (w / 2) and 2 (w / 2) + 1, the 16 sites of parity w % 2 of each
  for (int k = tid; k < kRhoTX * kRhoTY * kRhoTZ; k += blockDim.x) {
    const int w = k >> 5, ln = k & 31;
    const int p = w & 1, row = ((w >> 1) << 1) + (ln >> 4);
    const int lx = 2 * (ln & 15) + p, ly = row % kRhoTY, lz = row / kRhoTY;
    const int gx = x0 + lx, gy = y0 + ly, gz = z0 + lz;
    if (gx >= sx || gy >= sy || gz >= sz) continue;
    const uint8_t* t = tile + (lx + kRhoHX) + kRhoLX * ((ly + kRhoHY) + kRhoLY * (lz + kRhoHZ));
    const int32_t acc = p ? rho_terms<1, 0>(t, fqc) : rho_terms<0, 0>(t, fqc);
    lattice_put(rho + static_cast<int64_t>(px) * (gy + static_cast<int64_t>(sy) * gz), sx, gx, acc);
  }
}

__host__ __device__ __forceinline__ int64_t rho_tiles(int32_t sx, int32_t sy, int32_t sz) {
  return static_cast<int64_t>((sx + kRhoTX - 1) / kRhoTX) * ((sy + kRhoTY - 1) / kRhoTY) *
         ((sz + kRhoTZ - 1) / kRhoTZ);
}

__global__ void __launch_bounds__(256) k_init_rho(const uint8_t* occ, int32_t* rho, int32_t sx, int32_t sy,
                                                  int32_t sz, int32_t px, const Potential* pot) {
  __shared__ uint8_t tile[kRhoLX * kRhoLY * kRhoLZ];
  __shared__ int32_t fqc[16 * 8];
  rho_table(fqc, pot);
  const int64_t ntiles = rho_tiles(sx, sy, sz);
  for (int64_t tix = blockIdx.x; tix < ntiles; tix += gridDim.x) rho_tile(occ, rho, sx, sy, sz, px, tix, tile, fqc);
}

// The density build of every EAM job of a context in one launch: global tile t belongs to the
// job k with tile0[k] <= t < tile0[k + 1] (jobs[k] its index).
__global__ void __launch_bounds__(256) k_init_rho_jobs(RoundArgs a, const int64_t* tile0, const int32_t* jobs,
                                                       int32_t njobs) {
  __shared__ uint8_t tile[kRhoLX * kRhoLY * kRhoLZ];
  __shared__ int32_t fqc[16 * 8];
  int pot = -1;
  for (int64_t t = blockIdx.x; t < tile0[njobs]; t += gridDim.x) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {  // last k with tile0[k] <= t
      const int mid = (lo + hi + 1) >> 1;
      if (tile0[mid] <= t) lo = mid;
      else hi = mid - 1;
    }
    const JobDev& J = a.jobs[jobs[lo]];
    if (J.pot != pot) {  // uniform over the CTA
      __syncthreads();
      rho_table(fqc, a.pots + J.pot);
      pot = J.pot;
    }
    rho_tile(J.occ, J.rho, J.sx, J.sy, J.sz, J.px, t - tile0[lo], tile, fqc);
  }
}

// Whole-context lattice load: chunk c copies its sites from the staging buffer into its job's
// occupancy and appends the vacancies to the job's slice of the vacancy table.
__global__ void k_scatter_collect(RoundArgs a, const uint8_t* stage, const SiteChunk* chunks, int32_t* counts) {
  const SiteChunk c = chunks[blockIdx.x];
  const JobDev& J = a.jobs[c.job];
  for (int64_t i = threadIdx.x; i < c.n; i += blockDim.x) {
    const uint8_t o = stage[c.stage0 + i];
    const int32_t s = static_cast<int32_t>(c.site0 + i);
    lattice_put(J.occ + static_cast<int64_t>(J.px) * (s / J.sx), J.sx, s % J.sx, o);
    if (o == kV) {
      const int k = atomicAdd(counts + c.job, 1);
      if (k < c.nvac) {
        a.vac_site[c.vac0 + k] = static_cast<int32_t>(c.site0 + i);
        a.vac_job[c.vac0 + k] = c.job;
      }
    }
  }
}

__global__ void k_check_counts(const int32_t* counts, const int32_t* want, int32_t njobs, unsigned int* status) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < njobs && counts[j] != want[j]) atomicOr(status, kErrVacCount);
}

// Whole-context lattice read-back: the reverse copy into the staging buffer.
__global__ void k_gather(RoundArgs a, uint8_t* stage, const SiteChunk* chunks) {
  const SiteChunk c = chunks[blockIdx.x];
  const JobDev& J = a.jobs[c.job];
  for (int64_t i = threadIdx.x; i < c.n; i += blockDim.x)
    stage[c.stage0 + i] = J.occ[lattice_index(static_cast<int32_t>(c.site0 + i), J.sx, J.px)];
}

__global__ void k_collect_vacancies(const uint8_t* occ, int64_t n, int32_t sx, int32_t px, int32_t* vac_site,
                                    int32_t* vac_job, int32_t job, int32_t cap, int32_t* count) {
  for (int64_t s = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; s < n;
       s += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (occ[lattice_index(static_cast<int32_t>(s), sx, px)] != kV) continue;
    const int k = atomicAdd(count, 1);
    if (k < cap) {
      vac_site[k] = static_cast<int32_t>(s);
      vac_job[k] = job;
    }
  }
}

// The halo entries of every row of a lattice whose main entries were written by a plain copy:
// row r, entry p outside [kHaloL, kHaloL + sx) takes site (p - kHaloL) mod sx of the row.
template <typename T>
__global__ void k_fill_halo(T* lat, int32_t sx, int32_t px, int64_t nrows) {
  const int nh = kHaloL + kHaloR;
  const int64_t n = nrows * nh;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t row = i / nh;
    const int k = static_cast<int>(i - row * nh);
    const int p = k < kHaloL ? k : sx + k;  // [0, kHaloL) then [kHaloL + sx, kHaloL + sx + kHaloR)
    int x = (p - kHaloL) % sx;
    if (x < 0) x += sx;
    T* r = lat + row * px;
    r[p] = r[kHaloL + x];
  }
}

__global__ void k_device_math(const double* x, int64_t n, double* e, double* l) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  e[i] = port_exp(x[i]);
  l[i] = port_log(x[i]);
}

}  // namespace

size_t hop_smem_bytes(int max_region_sites) {
  return sizeof(Smem) + 128 + ((static_cast<size_t>(max_region_sites) * 4 + 127) & ~static_cast<size_t>(127)) +
         static_cast<size_t>(max_region_sites) + 16;
}

template <int W>
void launch_hops(const RoundArgs& a, int hop_grid, size_t smem, cudaStream_t st) {
  constexpr int T = Shape<W>::kThreads;
  if (a.kind_mask & (1 << kEam64)) k_hop<kEam64, W><<<hop_grid, T, smem, st>>>(a);
  if (a.kind_mask & (1 << kEam32)) k_hop<kEam32, W><<<hop_grid, T, smem, st>>>(a);
  if (a.kind_mask & (1 << kPairBond)) k_hop<kPairBond, W><<<hop_grid, T, smem, st>>>(a);
}
template <int W>
void launch_flows(const RoundArgs& a, int grid, size_t smem, cudaStream_t st) {
  constexpr int T = Shape<W>::kThreads;
  if (a.kind_mask & (1 << kEam64)) k_flow<kEam64, W><<<grid, T, smem, st>>>(a);
  if (a.kind_mask & (1 << kEam32)) k_flow<kEam32, W><<<grid, T, smem, st>>>(a);
  if (a.kind_mask & (1 << kPairBond)) k_flow<kPairBond, W><<<grid, T, smem, st>>>(a);
}

int launch_round(const RoundArgs& a, int hop_grid, size_t smem, void* stream, void* ev0, void* ev1) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (a.nvac > 0) k_bucket<<<(a.nvac + 127) / 128, 128, 0, st>>>(a);
  if (ev0) cudaEventRecord(static_cast<cudaEvent_t>(ev0), st);
  if (a.eval_warps == 4) launch_hops<4>(a, hop_grid, smem, st);
  else launch_hops<8>(a, hop_grid, smem, st);
  if (ev1) cudaEventRecord(static_cast<cudaEvent_t>(ev1), st);
  k_finalize<<<(a.nblocks + 127) / 128, 128, 0, st>>>(a);
  return static_cast<int>(cudaGetLastError());
}

int launch_api(const RoundArgs& a, size_t smem, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (a.nvac > 0) k_bucket<<<(a.nvac + 127) / 128, 128, 0, st>>>(a);
  k_api_block<<<1, Shape<8>::kThreads, smem, st>>>(a);
  k_api_reset<<<1, 1, 0, st>>>(a);
  return static_cast<int>(cudaGetLastError());
}

__global__ void k_flow_begin(RoundArgs a, int64_t n) {
  const int gb = blockIdx.x * blockDim.x + threadIdx.x;
  if (gb < a.nblocks) a.blocks[gb].remaining = n;
}

int launch_flow_begin(const RoundArgs& a, int64_t n, void* stream) {
  k_flow_begin<<<(a.nblocks + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(a, n);
  return static_cast<int>(cudaGetLastError());
}

int launch_flow(const RoundArgs& a, int grid, size_t smem, void* stream, void* ev0, void* ev1) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaMemsetAsync(a.flow_need, 0, 3 * sizeof(int32_t), st);
  cudaMemsetAsync(a.flow_done, 0, 3 * sizeof(int32_t), st);
  k_flow_prep<<<(a.nblocks + 127) / 128, 128, 0, st>>>(a);
  if (a.nvac > 0) k_flow_slots<<<(a.nvac + 127) / 128, 128, 0, st>>>(a);
  if (ev0) cudaEventRecord(static_cast<cudaEvent_t>(ev0), st);
  if (a.eval_warps == 4) launch_flows<4>(a, grid, smem, st);
  else launch_flows<8>(a, grid, smem, st);
  if (ev1) cudaEventRecord(static_cast<cudaEvent_t>(ev1), st);
  k_flow_finalize<<<(a.nblocks + 127) / 128, 128, 0, st>>>(a);
  return static_cast<int>(cudaGetLastError());
}

int hop_ctas_per_sm(int eval_warps) { return eval_warps == 4 ? Shape<4>::kCtasPerSm : Shape<8>::kCtasPerSm; }

int configure_hop_smem(size_t smem) {
  const void* kernels[] = {
      reinterpret_cast<const void*>(k_hop<kEam64, 8>),     reinterpret_cast<const void*>(k_hop<kEam32, 8>),
      reinterpret_cast<const void*>(k_hop<kPairBond, 8>),  reinterpret_cast<const void*>(k_hop<kEam64, 4>),
      reinterpret_cast<const void*>(k_hop<kEam32, 4>),     reinterpret_cast<const void*>(k_hop<kPairBond, 4>),
      reinterpret_cast<const void*>(k_flow<kEam64, 8>),    reinterpret_cast<const void*>(k_flow<kEam32, 8>),
      reinterpret_cast<const void*>(k_flow<kPairBond, 8>), reinterpret_cast<const void*>(k_flow<kEam64, 4>),
      reinterpret_cast<const void*>(k_flow<kEam32, 4>),    reinterpret_cast<const void*>(k_flow<kPairBond, 4>),
      reinterpret_cast<const void*>(k_api_block)};
  cudaError_t e = cudaSuccess;
  for (const void* f : kernels)
    if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  return static_cast<int>(e);
}

int launch_init_rho(uint8_t* occ, int32_t* rho, int32_t sx, int32_t sy, int32_t sz, const Potential* pot,
                    const Geometry* geo, unsigned int* status, void* stream) {
  (void)status;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t blocks = std::min<int64_t>(rho_tiles(sx, sy, sz), 148 * 16);
  (void)geo;
  k_init_rho<<<static_cast<int>(blocks), 256, 0, st>>>(occ, rho, sx, sy, sz, lattice_pitch(sx), pot);
  return static_cast<int>(cudaGetLastError());
}

__global__ void k_check_vacancy_count(const int32_t* count, int32_t want, unsigned int* status) {
  if (*count != want) atomicOr(status, kErrVacCount);
}

int launch_init_rho_jobs(const RoundArgs& a, const JobsLoad& L, void* stream) {
  if (L.neam > 0)
    k_init_rho_jobs<<<static_cast<int>(std::min<int64_t>(L.eam_tiles, 148 * 16)), 256, 0,
                      static_cast<cudaStream_t>(stream)>>>(a, L.tile0, L.eam_jobs, L.neam);
  return static_cast<int>(cudaGetLastError());
}

int launch_load_jobs(const RoundArgs& a, const JobsLoad& L, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(L.counts, 0, sizeof(int32_t) * L.njobs, st);
  if (e != cudaSuccess) return static_cast<int>(e);
  k_scatter_collect<<<L.nchunks, 256, 0, st>>>(a, L.stage, L.chunks, L.counts);
  k_check_counts<<<(L.njobs + 127) / 128, 128, 0, st>>>(L.counts, L.want, L.njobs, a.status);
  return launch_init_rho_jobs(a, L, stream);
}


int launch_gather_jobs(const RoundArgs& a, const JobsLoad& L, void* stream) {
  k_gather<<<L.nchunks, 256, 0, static_cast<cudaStream_t>(stream)>>>(a, L.stage, L.chunks);
  return static_cast<int>(cudaGetLastError());
}

int launch_collect_vacancies(const uint8_t* occ, int64_t n, int32_t sx, int32_t* vac_site, int32_t* vac_job,
                             int32_t job, int32_t cap, int32_t* count, unsigned int* status, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int64_t blocks = (n + 255) / 256;
  if (blocks > 148 * 64) blocks = 148 * 64;
  cudaMemsetAsync(count, 0, sizeof(int32_t), st);
  k_collect_vacancies<<<static_cast<int>(blocks), 256, 0, st>>>(occ, n, sx, lattice_pitch(sx), vac_site, vac_job, job,
                                                                cap, count);
  k_check_vacancy_count<<<1, 1, 0, st>>>(count, cap, status);
  return static_cast<int>(cudaGetLastError());
}

template <typename T>
int fill_halo(T* lat, int32_t sx, int64_t nrows, void* stream) {
  const int64_t n = nrows * (kHaloL + kHaloR);
  const int blocks = static_cast<int>(std::min<int64_t>((n + 255) / 256, 148 * 64));
  if (n > 0) k_fill_halo<T><<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(lat, sx, lattice_pitch(sx), nrows);
  return static_cast<int>(cudaGetLastError());
}
int launch_fill_halo(uint8_t* lat, int32_t sx, int64_t nrows, void* stream) { return fill_halo(lat, sx, nrows, stream); }
int launch_fill_halo(int32_t* lat, int32_t sx, int64_t nrows, void* stream) { return fill_halo(lat, sx, nrows, stream); }

int launch_device_math(const double* x, int64_t n, double* e, double* l, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_device_math<<<static_cast<int>((n + 255) / 256), 256, 0, st>>>(x, n, e, l);
  return static_cast<int>(cudaGetLastError());
}

// Round scratch of akmc_run_rounds_noalloc (2.1 MB): block vacancy lists, active-block
// list and active count for kNoAllocMaxBlocks blocks, with the count 256-byte aligned.
constexpr size_t kNoAllocWords = static_cast<size_t>(kNoAllocMaxBlocks) * (kMaxV + 1) + 64;
static __device__ __align__(256) int32_t g_noalloc_scratch[kNoAllocWords];

int noalloc_scratch(int32_t** base) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  *base = e == cudaSuccess ? static_cast<int32_t*>(p) : nullptr;
  return static_cast<int>(e);
}

}  // namespace akmc
