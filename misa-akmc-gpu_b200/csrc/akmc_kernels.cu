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

__device__ __forceinline__ double F64(const Potential& P, int32_t r, unsigned int* status) {
  int k = r >> kRhoCellShift;
  if (r < 0 || k > kTabN - 2) {
    atomicOr(status, kErrRhoRange);
    k = r < 0 ? 0 : kTabN - 2;
  }
  const double p = static_cast<double>(r & kRhoFracMask) * 0x1p-17;
  const double2* c = reinterpret_cast<const double2*>(P.Fcoef) + 2 * k;
  const double2 lo = __ldg(c), hi = __ldg(c + 1);
  return cubic_d(lo.x, lo.y, hi.x, hi.y, p);
}

__device__ __forceinline__ FCell32 cell32(const Potential& P, int32_t r, unsigned int* status) {
  int k = r >> kRhoCellShift;
  if (r < 0 || k > kTabN - 2) {
    atomicOr(status, kErrRhoRange);
    k = r < 0 ? 0 : kTabN - 2;
  }
  const float4* q = reinterpret_cast<const float4*>(P.F32 + k);
  const float4 a = __ldg(q), b = __ldg(q + 1);
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
__device__ void eval_vacancy(Smem& sm, const uint8_t* occ_s, const int32_t* rho_s, int k, const Potential& P,
                             const JobDev& J, unsigned int* status) {
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
      for (int i = q; i < kJumpN; i += 4) {
        const int32_t e = L[i];
        const int j = l + sdelta(e);
        const uint8_t o = occ_s[j];
        if (o == kV) continue;
        const int Y = species_index(o);
        const int ss = sshs(e), st = ssht(e);
        const int32_t r = rho_s[j];
        const int32_t d = sm.fq[X * 8 + ss] - sm.fq[X * 8 + st];
        const double Fa = F64(P, r + d, status);
        const double Fb = F64(P, r, status);
        const double T = (Fa - Fb) + (sm.phi64[(X * 4 + Y) * 8 + ss] - sm.phi64[(X * 4 + Y) * 8 + st]);
        acc += T;
      }
    }
    const double s2 = acc + __shfl_xor_sync(kFull, acc, 2);
    const double tsum = s2 + __shfl_xor_sync(kFull, s2, 1);
    if (avail && q == 0) {
      const double EX = F64(P, rho_s[l] - sm.fq[X * 8 + 1], status) - F64(P, rho_s[tl], status);
      dE = EX + tsum;
    }
  } else {
    Comp32 acc;
    acc.s = 0.f;
    acc.c = 0.f;
    const int X = species_index(Xc);
    if (avail) {
      const int32_t* L = sm.jl[p][b];
      for (int i = q; i < kJumpN; i += 4) {
        const int32_t e = L[i];
        const int j = l + sdelta(e);
        const uint8_t o = occ_s[j];
        if (o == kV) continue;
        const int Y = species_index(o);
        const int ss = sshs(e), st = ssht(e);
        const int32_t r = rho_s[j];
        const int32_t r1 = r + (sm.fq[X * 8 + ss] - sm.fq[X * 8 + st]);
        const float T = dF32(cell32(P, r1, status), cell32(P, r, status), r1, r) +
                        (sm.phi32[(X * 4 + Y) * 8 + ss] - sm.phi32[(X * 4 + Y) * 8 + st]);
        kahan_add(acc, T);
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
      const float EX = dF32(cell32(P, r1, status), cell32(P, r0, status), r1, r0);
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

__device__ __forceinline__ int64_t global_site(const JobDev& J, const Region& R, int l) {
  const int lx = l % R.LX;
  const int t = l / R.LX;
  const int ly = t % R.LY;
  const int lz = t / R.LY;
  const int X = wrap1(R.ox + lx, J.sx);
  const int y = wrap1(R.oy + ly, J.sy);
  const int z = wrap1(R.oz + lz, J.sz);
  return static_cast<int64_t>(X) + static_cast<int64_t>(J.sx) * (y + static_cast<int64_t>(J.sy) * z);
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
  load_tables(sm, P, *a.geo, R, eam);

  // stage the region: one row (fixed y, z) at a time, lanes along x
  for (int row = 0; row < R.LY * R.LZ; ++row) {
    const int ly = row % R.LY, lz = row / R.LY;
    const int gy = wrap1(R.oy + ly, J.sy), gz = wrap1(R.oz + lz, J.sz);
    const int64_t base = static_cast<int64_t>(J.sx) * (gy + static_cast<int64_t>(J.sy) * gz);
    for (int lx = lane; lx < R.LX; lx += 32) {
      const int gx = wrap1(R.ox + lx, J.sx);
      const int l = lx + R.LX * row;
      occ_s[l] = J.occ[base + gx];
      if (eam) rho_s[l] = J.rho[base + gx];
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
  __syncwarp();
  for (int k = 0; k < cnt; ++k) eval_vacancy<KIND>(sm, occ_s, rho_s, k, P, J, a.status);
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
      __syncwarp();
      if (lane == 0) {
        occ_s[tl] = kV;
        occ_s[s] = Xc;
      }
      if (eam) {
        const int X = species_index(Xc);
        for (int i = lane; i < kRefreshN; i += 32) {
          const int32_t e = sm.rl[p][bsel][i];
          rho_s[s + sdelta(e)] += sm.fq[X * 8 + sshs(e)] - sm.fq[X * 8 + ssht(e)];
        }
      }
      __syncwarp();
      if (lane == 0) {
        from_g = sm.vlid[ksel];
        to_g = global_site(J, R, tl);
        sm.vloc[ksel] = tl;
        int cx, cy, cz;
        local_cell(R, tl, cx, cy, cz);
        const bool in = cx >= 2 && cx < 2 + R.w[0] && cy >= 2 && cy < 2 + R.w[1] && cz >= 2 && cz < 2 + R.w[2];
        int pos = 0;
        while (sm.ord[pos] != ksel) ++pos;
        for (int i = pos; i + 1 < nord; ++i) sm.ord[i] = sm.ord[i + 1];
        --nord;
        if (in) {
          sm.vlid[ksel] = static_cast<int32_t>(to_g);
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
        eval_vacancy<KIND>(sm, occ_s, rho_s, k, P, J, a.status);
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
    if (nh) atomicAdd(a.counters + 6, static_cast<unsigned long long>(R.n));
  }
  if (nh == 0) return;
  for (int i = lane; i < cnt; i += 32) a.vac_site[sm.vidx[i]] = static_cast<int32_t>(global_site(J, R, sm.vloc[i]));
  for (int row = 0; row < R.LY * R.LZ; ++row) {
    const int ly = row % R.LY, lz = row / R.LY;
    const int gy = wrap1(R.oy + ly, J.sy), gz = wrap1(R.oz + lz, J.sz);
    const int64_t base = static_cast<int64_t>(J.sx) * (gy + static_cast<int64_t>(J.sy) * gz);
    for (int lx = lane; lx < R.LX; lx += 32) {
      const int gx = wrap1(R.ox + lx, J.sx);
      const int l = lx + R.LX * row;
      J.occ[base + gx] = occ_s[l];
      if (eam) J.rho[base + gx] = rho_s[l];
    }
  }
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

__global__ void __launch_bounds__(32) k_hop(RoundArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int na = *a.n_active;
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
