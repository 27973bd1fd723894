// akmc_kernels.cu -- sm_100a kernels of the vacancy-hop path.
//
// One sector round of the synchronous sublattice (src/algorithms/sl/sublattice.inl:64-177)
// runs as three launches:
//   k_bucket   one thread per vacancy: find its domain block, keep it if it lies in
//              the block's active sector, append it to the block's list;
//   k_hop      one warp per active block: stage the sector plus a 2-cell halo
//              (occupancy bytes and the int32 density cache) into shared memory,
//              run the hop loop there (rates, ordered total, selection, perform with
//              density refresh, recompute of the vacancies the hop touched, clock),
//              write the region back;
//   k_finalize one thread per block: clock of blocks without vacancies, next round.
// Concurrently active sectors are at least 4 cells apart, so the staged regions of
// different blocks never overlap and no atomics are needed on the lattice.
#include <cuda_runtime.h>

#include <cfloat>

#include "akmc_device.h"

namespace akmc {
namespace {

constexpr unsigned kFull = 0xffffffffu;

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
  int LX, LY, LZ, n;
};

__device__ __forceinline__ void make_region(const BlockDev& B, int sec, Region& R) {
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
  R.n = R.LX * R.LY * R.LZ;
}

// Shared-memory working set of one warp (followed by the staged region).
struct Smem {
  double b1[25], b2[25];
  double phi64[4 * 4 * 8];
  float phi32[4 * 4 * 8];
  int32_t fq[4 * 8];
  int32_t d1[2][8];
  int32_t d2[6];
  int32_t jl[2][8][kJumpN];     // int16 delta | sh_s << 16 | sh_t << 20
  int32_t rl[2][8][kRefreshN];
  int32_t vidx[kMaxV], vloc[kMaxV], vlid[kMaxV], ord[kMaxV];
  uint8_t vact[kMaxV], vavail[kMaxV], vdirty[kMaxV], vpad[kMaxV];
  double rates[kMaxV][8];
  alignas(16) unsigned char fwin[kFWin * 32];  // F-table window: double c0..c3 or FCell32 per cell
  alignas(8) uint64_t mbar;                    // completion barrier of the window's bulk copy
  uint32_t mbar_phase;
  int32_t win_pot;                             // potential (and precision) the window holds
};

// --- bulk copy global -> shared with an mbarrier (cp.async.bulk, TMA unit) -----------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
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
  const double* g64;
  const FCell32* g32;
  unsigned int* status;
};

__device__ __forceinline__ int local_delta(int32_t w, const Region& R) {
  return unpack_dx(w) + R.LX * (unpack_dy(w) + R.LY * unpack_dz(w));
}

__device__ void load_tables(Smem& sm, const Potential& P, const Geometry& G, const Region& R, bool eam) {
  const int lane = threadIdx.x;
  for (int i = lane; i < 25; i += 32) {
    sm.b1[i] = P.b1[i / 5][i % 5];
    sm.b2[i] = P.b2[i / 5][i % 5];
  }
  for (int i = lane; i < 128; i += 32) {
    sm.phi64[i] = (&P.phi64[0][0][0])[i];
    sm.phi32[i] = (&P.phi32[0][0][0])[i];
  }
  if (lane < 32) sm.fq[lane] = (&P.fq[0][0])[lane];
  if (lane < 16) sm.d1[lane >> 3][lane & 7] = local_delta(G.nn1[lane >> 3][lane & 7], R);
  if (lane < 6) sm.d2[lane] = local_delta(G.nn2[lane], R);
  if (eam) {
    for (int i = lane; i < 2 * 8 * kJumpN; i += 32) {
      const int32_t w = (&G.jump[0][0][0])[i];
      (&sm.jl[0][0][0])[i] = (local_delta(w, R) & 0xffff) | (unpack_sh_s(w) << 16) | (unpack_sh_t(w) << 20);
    }
    for (int i = lane; i < 2 * 8 * kRefreshN; i += 32) {
      const int32_t w = (&G.refresh[0][0][0])[i];
      (&sm.rl[0][0][0])[i] = (local_delta(w, R) & 0xffff) | (unpack_sh_s(w) << 16) | (unpack_sh_t(w) << 20);
    }
  }
}

__device__ __forceinline__ int sdelta(int32_t e) { return static_cast<int16_t>(e & 0xffff); }
__device__ __forceinline__ int sshs(int32_t e) { return (e >> 16) & 0xf; }
__device__ __forceinline__ int ssht(int32_t e) { return (e >> 20) & 0xf; }

__device__ __forceinline__ double F64(const FTab& T, int32_t r) {
  const int k = r >> kRhoCellShift;
  const double p = static_cast<double>(r & kRhoFracMask) * 0x1p-17;
  const unsigned kk = static_cast<unsigned>(k - T.kw0);
  double2 lo, hi;
  if (kk < static_cast<unsigned>(kFWin)) {
    const double2* c = reinterpret_cast<const double2*>(T.win) + 2 * kk;
    lo = c[0];
    hi = c[1];
  } else {
    int kc = k;
    if (r < 0 || k > kTabN - 2) {
      atomicOr(T.status, kErrRhoRange);
      kc = r < 0 ? 0 : kTabN - 2;
    }
    const double2* c = reinterpret_cast<const double2*>(T.g64) + 2 * kc;
    lo = __ldg(c);
    hi = __ldg(c + 1);
  }
  return cubic_d(lo.x, lo.y, hi.x, hi.y, p);
}

__device__ __forceinline__ FCell32 cell32(const FTab& T, int32_t r) {
  const int k = r >> kRhoCellShift;
  const unsigned kk = static_cast<unsigned>(k - T.kw0);
  float4 a, b;
  if (kk < static_cast<unsigned>(kFWin)) {
    const float4* q = reinterpret_cast<const float4*>(T.win) + 2 * kk;
    a = q[0];
    b = q[1];
  } else {
    int kc = k;
    if (r < 0 || k > kTabN - 2) {
      atomicOr(T.status, kErrRhoRange);
      kc = r < 0 ? 0 : kTabN - 2;
    }
    const float4* q = reinterpret_cast<const float4*>(T.g32 + kc);
    a = __ldg(q);
    b = __ldg(q + 1);
  }
  FCell32 c;
  c.hi = a.x; c.lo = a.y; c.c1 = a.z; c.c2 = a.w; c.c3 = b.x;
  c.pad0 = c.pad1 = c.pad2 = 0.f;
  return c;
}

enum : int { kPairBond = 0, kEam64 = 1, kEam32 = 2 };

// Rates of vacancy k of the list, all 8 jumps, warp-collective.
// Lane = 4 b + q: jump b, quarter q.
//  pair-bond: q selects one of the four bond counts of VacRatesSolver::deltaE
//             (vacancy_rates_solver.cpp:45-116), each summed in the reference order;
//  EAM:       q sums sites i = q, q+4, ... of the jump's site list, merged
//             (p0 + p2) + (p1 + p3), then the moving atom's own embedding change.
template <int KIND>
__device__ void eval_vacancy(Smem& sm, const uint8_t* occ_s, const int32_t* rho_s, int k, const FTab& FT,
                             const JobDev& J) {
  const int lane = threadIdx.x & 31;
  const int b = lane >> 2, q = lane & 3;
  const int l = sm.vloc[k];
  const int p = l & 1;
  const int tl = l + sm.d1[p][b];
  const uint8_t Xc = occ_s[tl];
  const bool avail = is_atom(Xc);
  double dE = 0.0;
  if (KIND == kPairBond) {
    double energy = 0.0;
    if (avail) {
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
    double acc = 0.0;
    const int X = species_index(Xc);
    if (avail) {
      const int32_t* L = sm.jl[p][b];
      // site term (F(r + d) - F(r)) + (phi_s - phi_t); a vacancy contributes nothing
      auto term = [&](int32_t e, bool& atom) {
        const int j = l + sdelta(e);
        const uint8_t o = occ_s[j];
        atom = o != kV;
        const int Y = atom ? species_index(o) : 0;
        const int ss = sshs(e), st = ssht(e);
        const int32_t r = rho_s[j];
        const int32_t d = sm.fq[X * 8 + ss] - sm.fq[X * 8 + st];
        const double Fa = F64(FT, r + d);
        const double Fb = F64(FT, r);
        return (Fa - Fb) + (sm.phi64[(X * 4 + Y) * 8 + ss] - sm.phi64[(X * 4 + Y) * 8 + st]);
      };
      int i = q;
      for (; i + 4 < kJumpN; i += 8) {  // two sites per iteration, accumulated in list order
        bool a0, a1;
        const double T0 = term(L[i], a0);
        const double T1 = term(L[i + 4], a1);
        if (a0) acc += T0;
        if (a1) acc += T1;
      }
      for (; i < kJumpN; i += 4) {
        bool a0;
        const double T0 = term(L[i], a0);
        if (a0) acc += T0;
      }
    }
    const double s2 = acc + __shfl_xor_sync(kFull, acc, 2);
    const double tsum = s2 + __shfl_xor_sync(kFull, s2, 1);
    if (avail && q == 0) {
      const double EX = F64(FT, rho_s[l] - sm.fq[X * 8 + 1]) - F64(FT, rho_s[tl]);
      dE = EX + tsum;
    }
  } else {
    Comp32 acc;
    acc.s = 0.f;
    acc.c = 0.f;
    const int X = species_index(Xc);
    if (avail) {
      const int32_t* L = sm.jl[p][b];
      auto term = [&](int32_t e, bool& atom) {
        const int j = l + sdelta(e);
        const uint8_t o = occ_s[j];
        atom = o != kV;
        const int Y = atom ? species_index(o) : 0;
        const int ss = sshs(e), st = ssht(e);
        const int32_t r = rho_s[j];
        const int32_t r1 = r + (sm.fq[X * 8 + ss] - sm.fq[X * 8 + st]);
        return dF32(cell32(FT, r1), cell32(FT, r), r1, r) +
               (sm.phi32[(X * 4 + Y) * 8 + ss] - sm.phi32[(X * 4 + Y) * 8 + st]);
      };
      int i = q;
      for (; i + 4 < kJumpN; i += 8) {
        bool a0, a1;
        const float T0 = term(L[i], a0);
        const float T1 = term(L[i + 4], a1);
        if (a0) kahan_add(acc, T0);
        if (a1) kahan_add(acc, T1);
      }
      for (; i < kJumpN; i += 4) {
        bool a0;
        const float T0 = term(L[i], a0);
        if (a0) kahan_add(acc, T0);
      }
    }
    Comp32 o2;
    o2.s = __shfl_xor_sync(kFull, acc.s, 2);
    o2.c = __shfl_xor_sync(kFull, acc.c, 2);
    Comp32 m = comp_merge(acc, o2);
    Comp32 o1;
    o1.s = __shfl_xor_sync(kFull, m.s, 1);
    o1.c = __shfl_xor_sync(kFull, m.c, 1);
    m = comp_merge(m, o1);
    if (avail && q == 0) {
      const int32_t r1 = rho_s[l] - sm.fq[X * 8 + 1];
      const int32_t r0 = rho_s[tl];
      const float EX = dF32(cell32(FT, r1), cell32(FT, r0), r1, r0);
      const float dEf = EX + (m.s - m.c);
      dE = static_cast<double>(dEf);
    }
  }
  if (q == 0) sm.rates[k][b] = avail ? arrhenius(J.nu, J.kT, Xc, dE) : 0.0;
  const unsigned bal = __ballot_sync(kFull, avail && q == 0);
  if (lane == 0) {
    uint8_t m = 0;
    for (int bb = 0; bb < 8; ++bb)
      if ((bal >> (4 * bb)) & 1u) m |= static_cast<uint8_t>(1u << bb);
    sm.vavail[k] = m;
  }
  __syncwarp();
}

__device__ __forceinline__ void local_cell(const Region& R, int l, int& cx, int& cy, int& cz) {
  const int lx = l % R.LX;
  const int t = l / R.LX;
  cx = lx >> 1;
  cy = t % R.LY;
  cz = t / R.LY;
}

// The hop loop of one block's active sector (or one per-hop API step).
template <int KIND>
__device__ void run_block(const RoundArgs& a, int gb, Smem& sm, uint8_t* occ_s, int32_t* rho_s) {
  const int lane = threadIdx.x & 31;
  BlockDev& B = a.blocks[gb];
  JobDev& J = a.jobs[B.job];
  const Potential& P = a.pots[J.pot];
  const bool eam = KIND != kPairBond;
  const int sec = a.mode == kModeRound ? sector_of_round(B.round) : a.api_sector;
  double thr = 0.0;
  if (a.mode == kModeRound) {
    const int64_t step = B.round >> 3;
    thr = static_cast<double>(step + 1) * J.window - B.evo[sec];
    if (!(0.0 < thr)) return;  // sector_time stays 0 (sublattice.inl:82)
  }
  Region R;
  make_region(B, sec, R);
  // F-table window: one bulk copy issued by lane 0, overlapped with the staging below
  const int win_key = J.pot * 2 + (KIND == kEam32 ? 1 : 0);
  const bool need_win = eam && sm.win_pot != win_key;
  __syncwarp();
  if (need_win && lane == 0) {
    const void* src = KIND == kEam32 ? static_cast<const void*>(P.F32 + P.fwin0)
                                     : static_cast<const void*>(P.Fcoef + 4 * static_cast<int64_t>(P.fwin0));
    bulk_load(sm.fwin, src, kFWin * 32u, &sm.mbar);
  }
  load_tables(sm, P, *a.geo, R, eam);
  FTab FT;
  FT.win = sm.fwin;
  FT.kw0 = P.fwin0;
  FT.g64 = P.Fcoef;
  FT.g32 = P.F32;
  FT.status = a.status;

  // stage the region: rows (fixed y, z) of LX <= 64 sites, lanes along x; eight rows
  // of loads are issued before any shared-memory store so they are all in flight
  {
    const int nrows = R.LY * R.LZ;
    const int gx0 = wrap1(R.ox + lane, J.sx), gx1 = wrap1(R.ox + lane + 32, J.sx);
    const bool has0 = lane < R.LX, has1 = lane + 32 < R.LX;
    for (int row0 = 0; row0 < nrows; row0 += 8) {
      uint8_t ov[8][2];
      int32_t rv[8][2];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int row = row0 + k;
        if (row < nrows) {
          const int ly = row % R.LY, lz = row / R.LY;
          const int gy = wrap1(R.oy + ly, J.sy), gz = wrap1(R.oz + lz, J.sz);
          const int64_t base = static_cast<int64_t>(J.sx) * (gy + static_cast<int64_t>(J.sy) * gz);
          if (has0) {
            ov[k][0] = J.occ[base + gx0];
            if (eam) rv[k][0] = J.rho[base + gx0];
          }
          if (has1) {
            ov[k][1] = J.occ[base + gx1];
            if (eam) rv[k][1] = J.rho[base + gx1];
          }
        }
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int row = row0 + k;
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
  }
  const int cnt = min(B.cnt, kMaxV);
  for (int i = lane; i < cnt; i += 32) {
    const int v = a.blk_list[static_cast<int64_t>(gb) * kMaxV + i];
    const int s = a.vac_site[v];
    const int X = s % J.sx;
    const int t = s / J.sx;
    const int y = t % J.sy;
    const int z = t / J.sy;
    sm.vidx[i] = v;
    sm.vloc[i] = (X - R.ox) + R.LX * ((y - R.oy) + R.LY * (z - R.oz));
    sm.vlid[i] = s;
    sm.vact[i] = 1;
    sm.vdirty[i] = 0;
  }
  __syncwarp();
  int nord = cnt;
  if (lane == 0) {  // z-y-x scan order of ABVIModel::calcRates = ascending site id inside a sector
    for (int i = 0; i < cnt; ++i) {
      int j = i;
      while (j > 0 && sm.vlid[sm.ord[j - 1]] > sm.vlid[i]) {
        sm.ord[j] = sm.ord[j - 1];
        --j;
      }
      sm.ord[j] = i;
    }
  }
  if (need_win) {
    bool ok = true;
    if (lane == 0) {
      ok = mbar_wait(&sm.mbar, sm.mbar_phase);
      if (ok) {
        sm.mbar_phase ^= 1u;
        sm.win_pot = win_key;
      } else {
        atomicOr(a.status, kErrTimeout);
        mbar_wait(&sm.mbar, sm.mbar_phase);  // bounded second wait for the copy in flight
        sm.win_pot = -1;
      }
    }
    ok = __shfl_sync(kFull, ok ? 1 : 0, 0) != 0;
    if (!ok) return;
  }
  __syncwarp();
  for (int k = 0; k < cnt; ++k) eval_vacancy<KIND>(sm, occ_s, rho_s, k, FT, J);
  int64_t evals = cnt;

  uint64_t xs[4], xt[4];
  for (int i = 0; i < 4; ++i) {
    xs[i] = B.xs[i];
    xt[i] = B.xt[i];
  }
  const int64_t hop0 = B.hops;
  int64_t nh = 0;
  int64_t nact_sum = 0;
  double sector_time = 0.0;
  const int D = eam ? 4 : 3;
  while (true) {
    double total = 0.0;
    if (lane == 0) {
      for (int i = 0; i < nord; ++i) {
        const int k = sm.ord[i];
        const uint8_t m = sm.vavail[k];
        for (int bb = 0; bb < 8; ++bb)
          if ((m >> bb) & 1) total += sm.rates[k][bb];
      }
    }
    total = __shfl_sync(kFull, total, 0);
    if (a.mode == kModeCalc) {
      if (lane == 0) *a.api_total = total;
      break;
    }
    if (total == 0.0 || fabs(total) < DBL_EPSILON) {  // sublattice.inl:108-112
      if (a.mode == kModeSelectPerform && lane == 0) {
        a.api_event->from_site = -1;
        a.api_event->total = total;
      }
      sector_time = thr;
      break;
    }
    double u = 0.0;
    int ksel = -1, bsel = -1;
    if (lane == 0) {
      u = a.mode == kModeSelectPerform ? a.api_u : uniform_co(xs);
      const double expected = u * total;  // ModelAdapter::selectAndPerform
      double acc = 0.0;
      for (int i = 0; i < nord && ksel < 0; ++i) {  // ABVIModel::select (kmc.cpp:242-309)
        const int k = sm.ord[i];
        const uint8_t m = sm.vavail[k];
        for (int bb = 0; bb < 8; ++bb) {
          if (!((m >> bb) & 1)) continue;
          acc += sm.rates[k][bb];
          if (acc > expected) {
            ksel = k;
            bsel = bb;
            break;
          }
        }
      }
    }
    ksel = __shfl_sync(kFull, ksel, 0);
    bsel = __shfl_sync(kFull, bsel, 0);
    const int nact_before = nord;
    int nd = 0;
    int64_t from_g = -1, to_g = -1;
    uint8_t Xc = 0;
    if (ksel >= 0) {
      // ABVIModel::perform (kmc.cpp:358-396) on the staged region
      const int s = sm.vloc[ksel];
      const int p = s & 1;
      const int tl = s + sm.d1[p][bsel];
      Xc = occ_s[tl];
      // global coordinates of s; the hop writes through to global memory (the staged
      // regions of concurrent blocks are disjoint, so global stays the shared truth)
      from_g = sm.vlid[ksel];
      const int sX = static_cast<int>(from_g % J.sx);
      const int sT = static_cast<int>(from_g / J.sx);
      const int sY = sT % J.sy, sZ = sT / J.sy;
      auto gsite = [&](int32_t w) {
        const int gx = wrap1(sX + unpack_dx(w), J.sx), gy = wrap1(sY + unpack_dy(w), J.sy),
                  gz = wrap1(sZ + unpack_dz(w), J.sz);
        return static_cast<int64_t>(gx) + static_cast<int64_t>(J.sx) * (gy + static_cast<int64_t>(J.sy) * gz);
      };
      to_g = gsite(a.geo->nn1[p][bsel]);
      __syncwarp();
      if (lane == 0) {
        occ_s[tl] = kV;
        occ_s[s] = Xc;
        J.occ[to_g] = kV;
        J.occ[from_g] = Xc;
      }
      if (eam) {
        const int X = species_index(Xc);
        for (int i = lane; i < kRefreshN; i += 32) {
          const int32_t e = sm.rl[p][bsel][i];
          const int j = s + sdelta(e);
          const int32_t v = rho_s[j] + (sm.fq[X * 8 + sshs(e)] - sm.fq[X * 8 + ssht(e)]);
          rho_s[j] = v;
          J.rho[gsite(a.geo->refresh[p][bsel][i])] = v;
        }
      }
      __syncwarp();
      if (lane == 0) {
        sm.vloc[ksel] = tl;
        sm.vlid[ksel] = static_cast<int32_t>(to_g);
        int cx, cy, cz;
        local_cell(R, tl, cx, cy, cz);
        const bool in = cx >= 2 && cx < 2 + R.w[0] && cy >= 2 && cy < 2 + R.w[1] && cz >= 2 && cz < 2 + R.w[2];
        int pos = 0;
        while (sm.ord[pos] != ksel) ++pos;
        for (int i = pos; i + 1 < nord; ++i) sm.ord[i] = sm.ord[i + 1];
        --nord;
        if (in) {
          int j = nord;
          while (j > 0 && sm.vlid[sm.ord[j - 1]] > sm.vlid[ksel]) {
            sm.ord[j] = sm.ord[j - 1];
            --j;
          }
          sm.ord[j] = ksel;
          ++nord;
        } else {
          sm.vact[ksel] = 0;
        }
        int sx, sy, sz;
        local_cell(R, s, sx, sy, sz);
        for (int i = 0; i < nord; ++i) {
          const int k = sm.ord[i];
          int vx, vy, vz;
          local_cell(R, sm.vloc[k], vx, vy, vz);
          if (abs(vx - sx) <= D && abs(vy - sy) <= D && abs(vz - sz) <= D) {
            sm.vdirty[k] = 1;
            ++nd;
          }
        }
      }
      nord = __shfl_sync(kFull, nord, 0);
      nd = __shfl_sync(kFull, nd, 0);
      __syncwarp();
      for (int k = 0; k < cnt; ++k) {
        if (!sm.vdirty[k]) continue;
        eval_vacancy<KIND>(sm, occ_s, rho_s, k, FT, J);
        if (lane == 0) sm.vdirty[k] = 0;
        __syncwarp();
      }
      evals += nd;
      nact_sum += nact_before;
      ++nh;
    }
    if (a.mode == kModeSelectPerform) {
      if (lane == 0) {
        akmc_event* e = a.api_event;
        e->round = 0;
        e->hop = hop0;
        e->from_site = from_g;
        e->to_site = to_g;
        e->block = B.local_id;
        e->species = Xc;
        e->u = u;
        e->total = total;
        e->dt = 0.0;
        e->n_act = nact_before;
        e->n_dirty = nd;
        e->job = B.job;
        e->reserved = 0;
      }
      break;
    }
    if (lane == 0) {
      const double u2 = uniform_oc(xt);  // sublattice.inl:118-120
      const double dt = -port_log(u2) / total;
      sector_time += dt;
      if (ksel >= 0 && a.log_cap > 0) {
        const unsigned long long slot = atomicAdd(a.log_count, 1ull);
        if (slot < static_cast<unsigned long long>(a.log_cap)) {
          akmc_event* e = a.log + slot;
          e->round = B.round;
          e->hop = hop0 + nh - 1;
          e->from_site = from_g;
          e->to_site = to_g;
          e->block = B.local_id;
          e->species = Xc;
          e->u = u;
          e->total = total;
          e->dt = dt;
          e->n_act = nact_before;
          e->n_dirty = nd;
          e->job = B.job;
          e->reserved = 0;
        } else {
          atomicOr(a.status, kErrLogOverflow);
        }
      }
    }
    sector_time = __shfl_sync(kFull, sector_time, 0);
    if (!(sector_time < thr)) break;
    if (nh >= a.hop_cap) {
      if (lane == 0) atomicOr(a.status, kErrHopCap);
      break;
    }
  }
  __syncwarp();
  if (a.mode == kModeCalc) return;
  if (lane == 0) {
    if (a.mode == kModeRound) {
      B.evo[sec] += sector_time;
      for (int i = 0; i < 4; ++i) {
        B.xs[i] = xs[i];
        B.xt[i] = xt[i];
      }
    }
    B.hops += nh;
    if (nh) atomicAdd(reinterpret_cast<unsigned long long*>(&J.hops), static_cast<unsigned long long>(nh));
    atomicAdd(a.counters + 0, static_cast<unsigned long long>(nh));
    atomicAdd(a.counters + 1, static_cast<unsigned long long>(evals));
    atomicAdd(a.counters + 3, 1ull);
    atomicAdd(a.counters + 4, static_cast<unsigned long long>(nact_sum));
    atomicAdd(a.counters + 5, static_cast<unsigned long long>(R.n));
    if (nh) atomicAdd(a.counters + 6, static_cast<unsigned long long>(nh * (eam ? 2 + kRefreshN : 2)));
  }
  if (nh == 0) return;
  // the lattice was written through at every hop; only the vacancy positions remain
  for (int i = lane; i < cnt; i += 32) a.vac_site[sm.vidx[i]] = sm.vlid[i];
}

__device__ __forceinline__ void carve(uint8_t* smem, int nreg, Smem*& sm, uint8_t*& occ_s, int32_t*& rho_s) {
  sm = reinterpret_cast<Smem*>(smem);
  uint8_t* p = smem + ((sizeof(Smem) + 15) & ~static_cast<size_t>(15));
  rho_s = reinterpret_cast<int32_t*>(p);
  occ_s = p + static_cast<size_t>(nreg) * 4;
}

__device__ void dispatch_block(const RoundArgs& a, int gb, uint8_t* smem) {
  const BlockDev& B = a.blocks[gb];
  const JobDev& J = a.jobs[B.job];
  const int sec = a.mode == kModeRound ? sector_of_round(B.round) : a.api_sector;
  Region R;
  make_region(B, sec, R);
  Smem* sm;
  uint8_t* occ_s;
  int32_t* rho_s;
  carve(smem, R.n, sm, occ_s, rho_s);
  if (J.model == AKMC_MODEL_PAIRBOND) run_block<kPairBond>(a, gb, *sm, occ_s, rho_s);
  else if (J.precision == AKMC_FP32C) run_block<kEam32>(a, gb, *sm, occ_s, rho_s);
  else run_block<kEam64>(a, gb, *sm, occ_s, rho_s);
}

__global__ void k_bucket(RoundArgs a) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= a.nvac) return;
  const int j = a.vac_job[v];
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
    sm->mbar_phase = 0;
    mbar_init(&sm->mbar);
  }
  __syncwarp();
}

__global__ void __launch_bounds__(32) k_hop(RoundArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int na = *a.n_active;
  if (static_cast<int>(blockIdx.x) >= na) return;
  init_cta_smem(smem);
  for (int item = blockIdx.x; item < na; item += gridDim.x) {
    dispatch_block(a, a.active[item], smem);
    __syncwarp();
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
  JobDev& J = a.jobs[B.job];
  const int had = B.cnt;
  B.cnt = 0;
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
  const int done = (J.hop_budget > 0 && J.hops >= J.hop_budget) || (J.max_rounds > 0 && B.round >= J.max_rounds);
  B.done = done;
  if (B.local_id == 0) {
    J.round = B.round;
    J.done = done;
  }
}

__global__ void k_api_block(RoundArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  const JobDev& J = a.jobs[a.api_job];
  if (*a.n_active == 0) {  // no vacancy in the sector
    if (threadIdx.x == 0) {
      if (a.mode == kModeCalc) *a.api_total = 0.0;
      else {
        a.api_event->from_site = -1;
        a.api_event->total = 0.0;
      }
    }
    return;
  }
  init_cta_smem(smem);
  dispatch_block(a, J.block0, smem);
}

__global__ void k_api_reset(RoundArgs a) {
  const JobDev& J = a.jobs[a.api_job];
  a.blocks[J.block0].cnt = 0;
  *a.n_active = 0;
}

__global__ void k_init_rho(const uint8_t* occ, int32_t* rho, int32_t sx, int32_t sy, int32_t sz,
                           const Potential* pot, const Geometry* geo) {
  const int64_t n = static_cast<int64_t>(sx) * sy * sz;
  for (int64_t s = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; s < n;
       s += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int X = static_cast<int>(s % sx);
    const int64_t t = s / sx;
    const int y = static_cast<int>(t % sy);
    const int z = static_cast<int>(t / sy);
    const int p = X & 1;
    int32_t acc = 0;
    for (int i = 0; i < kShellNb; ++i) {
      const int32_t w = geo->nbr[p][i];
      int gx = X + unpack_dx(w), gy = y + unpack_dy(w), gz = z + unpack_dz(w);
      gx = gx < 0 ? gx + sx : (gx >= sx ? gx - sx : gx);
      gy = gy < 0 ? gy + sy : (gy >= sy ? gy - sy : gy);
      gz = gz < 0 ? gz + sz : (gz >= sz ? gz - sz : gz);
      const uint8_t o = occ[gx + static_cast<int64_t>(sx) * (gy + static_cast<int64_t>(sy) * gz)];
      if (o != kV) acc += pot->fq[species_index(o)][unpack_sh_s(w)];
    }
    rho[s] = acc;
  }
}

__global__ void k_collect_vacancies(const uint8_t* occ, int64_t n, int32_t* vac_site, int32_t* vac_job, int32_t job,
                                    int32_t cap, int32_t* count) {
  for (int64_t s = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; s < n;
       s += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (occ[s] != kV) continue;
    const int k = atomicAdd(count, 1);
    if (k < cap) {
      vac_site[k] = static_cast<int32_t>(s);
      vac_job[k] = job;
    }
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
  return ((sizeof(Smem) + 15) & ~static_cast<size_t>(15)) + static_cast<size_t>(max_region_sites) * 5 + 16;
}

int launch_round(const RoundArgs& a, int hop_grid, size_t smem, void* stream, void* ev0, void* ev1) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (a.nvac > 0) k_bucket<<<(a.nvac + 127) / 128, 128, 0, st>>>(a);
  if (ev0) cudaEventRecord(static_cast<cudaEvent_t>(ev0), st);
  k_hop<<<hop_grid, 32, smem, st>>>(a);
  if (ev1) cudaEventRecord(static_cast<cudaEvent_t>(ev1), st);
  k_finalize<<<(a.nblocks + 127) / 128, 128, 0, st>>>(a);
  return static_cast<int>(cudaGetLastError());
}

int launch_api(const RoundArgs& a, size_t smem, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (a.nvac > 0) k_bucket<<<(a.nvac + 127) / 128, 128, 0, st>>>(a);
  k_api_block<<<1, 32, smem, st>>>(a);
  k_api_reset<<<1, 1, 0, st>>>(a);
  return static_cast<int>(cudaGetLastError());
}

int configure_hop_smem(size_t smem) {
  cudaError_t e = cudaFuncSetAttribute(k_hop, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return static_cast<int>(e);
  e = cudaFuncSetAttribute(k_api_block, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  return static_cast<int>(e);
}

int launch_init_rho(uint8_t* occ, int32_t* rho, int32_t sx, int32_t sy, int32_t sz, const Potential* pot,
                    const Geometry* geo, unsigned int* status, void* stream) {
  (void)status;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t n = static_cast<int64_t>(sx) * sy * sz;
  int64_t blocks = (n + 255) / 256;
  if (blocks > 148 * 64) blocks = 148 * 64;
  k_init_rho<<<static_cast<int>(blocks), 256, 0, st>>>(occ, rho, sx, sy, sz, pot, geo);
  return static_cast<int>(cudaGetLastError());
}

int launch_collect_vacancies(const uint8_t* occ, int64_t n, int32_t* vac_site, int32_t* vac_job, int32_t job,
                             int32_t cap, int32_t* count, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int64_t blocks = (n + 255) / 256;
  if (blocks > 148 * 64) blocks = 148 * 64;
  k_collect_vacancies<<<static_cast<int>(blocks), 256, 0, st>>>(occ, n, vac_site, vac_job, job, cap, count);
  return static_cast<int>(cudaGetLastError());
}

int launch_device_math(const double* x, int64_t n, double* e, double* l, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_device_math<<<static_cast<int>((n + 255) / 256), 256, 0, st>>>(x, n, e, l);
  return static_cast<int>(cudaGetLastError());
}

}  // namespace akmc
