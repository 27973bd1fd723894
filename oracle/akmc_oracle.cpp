// akmc_oracle.cpp -- CPU restatement of the MISA-AKMC vacancy-hop path.
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, never the product.
// Compiled with -ffp-contract=off so every multiply and add rounds on its own;
// where a fused multiply-add is part of the defined arithmetic it is written as
// std::fma / std::fmaf.
//
// Reference files restated (paths inside panzhija/MISA-AKMC-GPU) are cited at
// each function.  Deviations from the reference, all deliberate:
//  * periodicity by direct modular wrap instead of self-halo exchange
//    (equivalent for a single rank: the ghost images of the active sector lie in
//    inactive sectors, src/algorithms/sl/sublattice.inl:348-631);
//  * several "ranks" of one box are domain blocks of one shared array; the
//    sector regions of concurrently active blocks (+2-cell halo) are disjoint;
//  * vacancy placement clears every solute on the chosen site (the reference
//    clears only Cu, src/creation.cpp:149-157, leaving stale Ni/Mn entries);
//  * the EAM energy model exists only here (reference: vacancy_rates_solver.cpp:42-43).
#include "akmc_oracle.h"

#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// models/abvi/rate/rates_types.h:16
constexpr double kBoltzmann = 8.617330350E-5;
// src/algorithms/sl/sublattice.h:21-30 (X_HIGH = bit 0, Y_HIGH = bit 1, Z_HIGH = bit 2)
constexpr int kSectorOrder[8] = {0, 7, 2, 5, 3, 4, 1, 6};

// src/lattice/lattice_types.h:20-36
enum : uint8_t { kV = 0, kFe = 1, kCu = 2, kNi = 4, kMn = 8 };

inline int species_index(uint8_t code) {  // Fe, Cu, Ni, Mn -> 0..3
  switch (code) {
    case kFe: return 0;
    case kCu: return 1;
    case kNi: return 2;
    case kMn: return 3;
    default: return -1;
  }
}
inline int bond_index(uint8_t code) {  // V, Fe, Cu, Ni, Mn -> 0..4
  switch (code) {
    case kV: return 0;
    case kFe: return 1;
    case kCu: return 2;
    case kNi: return 3;
    case kMn: return 4;
    default: return -1;
  }
}
inline bool is_atom(uint8_t code) { return code == kFe || code == kCu || code == kNi || code == kMn; }

// ---------------------------------------------------------------------------
// Portable exp / log: the same IEEE operation sequence runs on the host and on
// the GPU, so rates and clocks agree bit for bit.
// exp: Cody & Waite argument reduction x = k ln2 + r (ln2 split in a 32-bit
//      head and a tail), Taylor polynomial of degree 13 for e^r on |r| <= ln2/2
//      as 1 + (r + r^2 T(r)) with the tail T in Estrin's scheme, scaling by 2^k
//      through the exponent field.
// log: x = m 2^e with m in [sqrt(1/2), sqrt(2)); log m = 2 atanh(s),
//      s = (m-1)/(m+1), atanh series to s^25.
// ---------------------------------------------------------------------------
constexpr double kLn2Hi = 0x1.62e42fee00000p-1;
constexpr double kLn2Lo = 0x1.a39ef35793c76p-33;
constexpr double kInvLn2 = 0x1.71547652b82fep+0;
constexpr double kSqrt2 = 0x1.6a09e667f3bcdp+0;

inline double from_bits(uint64_t b) { double d; std::memcpy(&d, &b, 8); return d; }
inline uint64_t to_bits(double d) { uint64_t b; std::memcpy(&b, &d, 8); return b; }

inline double scale_pow2(double p, int k) {
  // p in [0.7, 1.5); result p * 2^k, exact when the result is normal.
  if (k > 1023) return p * from_bits(uint64_t(2046) << 52) * from_bits(uint64_t(k - 1023 + 1023) << 52);
  if (k < -1022) {
    return p * from_bits(uint64_t(1) << 52) * from_bits(uint64_t(k + 1022 + 1023) << 52);
  }
  return p * from_bits(uint64_t(k + 1023) << 52);
}

double port_exp(double x) {
  if (x != x) return x;
  if (x > 709.782712893384) return HUGE_VAL;
  if (x < -745.1332191019412) return 0.0;
  const double kd = std::rint(x * kInvLn2);
  const int k = static_cast<int>(kd);
  double r = std::fma(-kd, kLn2Hi, x);
  r = std::fma(-kd, kLn2Lo, r);
  // e^r = 1 + (r + r^2 T(r)), T(r) = sum of r^(i-2) / i! for i = 2..13 in Estrin's scheme:
  // pairs (1/i! + r/(i+1)!), then powers r^2, r^4, r^8 (the device runs the same operations)
  const double r2 = r * r, r4 = r2 * r2, r8 = r4 * r4;
  const double p23 = std::fma(0x1.5555555555555p-3, r, 0.5);                     // 1/2! + r/3!
  const double p45 = std::fma(0x1.1111111111111p-7, r, 0x1.5555555555555p-5);    // 1/4!, 1/5!
  const double p67 = std::fma(0x1.a01a01a01a01ap-13, r, 0x1.6c16c16c16c17p-10);  // 1/6!, 1/7!
  const double p89 = std::fma(0x1.71de3a556c734p-19, r, 0x1.a01a01a01a01ap-16);  // 1/8!, 1/9!
  const double p1011 = std::fma(0x1.ae64567f544e4p-26, r, 0x1.27e4fb7789f5cp-22);  // 1/10!, 1/11!
  const double p1213 = std::fma(0x1.6124613a86d09p-33, r, 0x1.1eed8eff8d898p-29);  // 1/12!, 1/13!
  const double t0 = std::fma(p45, r2, p23), t1 = std::fma(p89, r2, p67), t2 = std::fma(p1213, r2, p1011);
  const double T = std::fma(t2, r8, std::fma(t1, r4, t0));
  const double p = 1.0 + std::fma(r2, T, r);
  return scale_pow2(p, k);
}

double port_log(double x) {
  if (x != x || x < 0.0) return std::numeric_limits<double>::quiet_NaN();
  if (x == 0.0) return -HUGE_VAL;
  if (x == HUGE_VAL) return x;
  uint64_t b = to_bits(x);
  int e = static_cast<int>((b >> 52) & 0x7ff);
  if (e == 0) {  // subnormal: scale into the normal range
    x = x * 0x1p54;
    b = to_bits(x);
    e = static_cast<int>((b >> 52) & 0x7ff) - 54;
  }
  e -= 1023;
  double m = from_bits((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);  // [1, 2)
  if (m > kSqrt2) {
    m = m * 0.5;
    e += 1;
  }
  const double s = (m - 1.0) / (m + 1.0);
  const double z = s * s;
  double p = 0x1.47ae147ae147bp-5;  // 1/25
  p = std::fma(p, z, 0x1.642c8590b2164p-5);  // 1/23
  p = std::fma(p, z, 0x1.8618618618618p-5);  // 1/21
  p = std::fma(p, z, 0x1.af286bca1af28p-5);  // 1/19
  p = std::fma(p, z, 0x1.e1e1e1e1e1e1ep-5);  // 1/17
  p = std::fma(p, z, 0x1.1111111111111p-4);  // 1/15
  p = std::fma(p, z, 0x1.3b13b13b13b14p-4);  // 1/13
  p = std::fma(p, z, 0x1.745d1745d1746p-4);  // 1/11
  p = std::fma(p, z, 0x1.c71c71c71c71cp-4);  // 1/9
  p = std::fma(p, z, 0x1.2492492492492p-3);  // 1/7
  p = std::fma(p, z, 0x1.999999999999ap-3);  // 1/5
  p = std::fma(p, z, 0x1.5555555555555p-2);  // 1/3
  const double t = s + s;
  const double logm = std::fma(t * z, p, t);
  const double ed = static_cast<double>(e);
  return std::fma(ed, kLn2Hi, std::fma(ed, kLn2Lo, logm));
}

// ---------------------------------------------------------------------------
// RNG.  xoshiro256** (Blackman & Vigna 2018) seeded through splitmix64.
// A stream is named by (seed, tag, index): tag 1 = alloy types, 2 = vacancies,
// 3 = event selection, 4 = residence time, 5 = EAM parameters; index = block.
// ---------------------------------------------------------------------------
inline uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
inline uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
struct Xoshiro {
  uint64_t s[4];
  uint64_t next() {
    const uint64_t r = rotl64(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl64(s[3], 45);
    return r;
  }
  double uniform() { return static_cast<double>(next() >> 11) * 0x1p-53; }              // [0, 1)
  double uniform_open0() { return static_cast<double>((next() >> 11) + 1) * 0x1p-53; }  // (0, 1]
  uint64_t below(uint64_t n) { return static_cast<uint64_t>((static_cast<unsigned __int128>(next()) * n) >> 64); }
};
enum : uint64_t { kTagTypes = 1, kTagVacancy = 2, kTagSelect = 3, kTagTime = 4, kTagPotential = 5 };
Xoshiro make_stream(uint64_t seed, uint64_t tag, uint64_t index) {
  uint64_t h = mix64(seed ^ (tag * 0xD1B54A32D192ED03ULL));
  h = mix64(h ^ (index * 0x9E3779B97F4A7C15ULL + 0x632BE59BD9B4E019ULL));
  Xoshiro x;
  for (int i = 0; i < 4; ++i) {
    h += 0x9E3779B97F4A7C15ULL;
    x.s[i] = mix64(h);
  }
  if ((x.s[0] | x.s[1] | x.s[2] | x.s[3]) == 0) x.s[0] = 1;
  return x;
}

// ---------------------------------------------------------------------------
// Pair-bond tables: table 7 of Vincent, Becquart & Domain, J. Nucl. Mater. 351
// (2006) 88-99, as tabulated in models/abvi/rate/bonds/bonds_counter.cpp:13-33.
// Index order V, Fe, Cu, Ni, Mn.
// ---------------------------------------------------------------------------
struct BondTables {
  double b1[5][5], b2[5][5];
  BondTables() {
    auto set = [](double t[5][5], int i, int j, double v) { t[i][j] = v; t[j][i] = v; };
    set(b1, 1, 1, -0.778); set(b1, 0, 0, 0.315); set(b1, 2, 2, -0.581); set(b1, 3, 3, -0.793); set(b1, 4, 4, -0.438);
    set(b1, 0, 1, -0.161); set(b1, 1, 2, -0.609); set(b1, 1, 3, -0.821); set(b1, 1, 4, -0.648);
    set(b1, 0, 2, -0.103); set(b1, 0, 3, -0.234); set(b1, 0, 4, -0.151);
    set(b1, 2, 3, -0.692); set(b1, 2, 4, -0.519); set(b1, 3, 4, -0.831);
    set(b2, 1, 1, -0.389); set(b2, 0, 0, -0.214); set(b2, 2, 2, -0.389); set(b2, 3, 3, -0.389); set(b2, 4, 4, -0.389);
    set(b2, 0, 1, -0.161); set(b2, 1, 2, -0.344); set(b2, 1, 3, -0.399); set(b2, 1, 4, -0.364);
    set(b2, 0, 2, -0.206); set(b2, 0, 3, -0.351); set(b2, 0, 4, -0.206);
    set(b2, 2, 3, -0.344); set(b2, 2, 4, -0.249); set(b2, 3, 4, -0.464);
  }
};
const BondTables kBonds;

// models/abvi/rate/vacancy_rates_solver.cpp:14-27
inline double e0_of(uint8_t code) {
  switch (code) {
    case kFe: return 0.62;
    case kCu: return 0.54;
    case kNi: return 0.68;
    case kMn: return 1.03;
    default: return 0;
  }
}

// ---------------------------------------------------------------------------
// Neighbour offsets in doubled-x coordinates (dX, dy, dz).
// 1nn order: LatListMeta::getIdBy1nnOffset (src/lattice/lattice_list_meta.cpp:22-70).
// 2nn order: PeriodLatticeList::get2nn2 (src/lattice/period_lattice_list.cpp:234-256),
// status mask 0x2F (period_lattice_list.cpp:15-18): entry 4 = (x, y+1, z) never counted.
// ---------------------------------------------------------------------------
struct Off { int dx, dy, dz; };
constexpr Off kNN1[2][8] = {
    {{-1, -1, -1}, {-1, -1, 0}, {-1, 0, -1}, {-1, 0, 0}, {1, -1, -1}, {1, -1, 0}, {1, 0, -1}, {1, 0, 0}},
    {{-1, 0, 0}, {-1, 0, 1}, {-1, 1, 0}, {-1, 1, 1}, {1, 0, 0}, {1, 0, 1}, {1, 1, 0}, {1, 1, 1}}};
constexpr Off kNN2[6] = {{-2, 0, 0}, {0, -1, 0}, {0, 0, -1}, {0, 0, 1}, {0, 1, 0}, {2, 0, 0}};
constexpr unsigned kNN2Status = 0x2F;

// EAM shells: squared distance in (a/2)^2 units.
constexpr int kShellD2[5] = {3, 4, 8, 11, 12};
constexpr int kShellSelf = 6;  // shell code of the site itself (no density from itself)

inline int half_coord_d2(int X0, int dX, int dy, int dz) {
  // half-lattice coordinates: corner (X even) -> (X, 2y, 2z); centre -> (X, 2y+1, 2z+1)
  const int p0 = X0 & 1;
  const int p1 = (X0 + dX) & 1;
  const int hx = dX;
  const int hy = 2 * dy + p1 - p0;
  const int hz = 2 * dz + p1 - p0;
  return hx * hx + hy * hy + hz * hz;
}
inline int shell_of_d2(int d2, int nsh) {
  for (int i = 0; i < nsh; ++i)
    if (kShellD2[i] == d2) return i + 1;
  return 0;
}

struct ShellNb { int dx, dy, dz, sh; };
struct JumpEntry { int dx, dy, dz, sh_s, sh_t; };

struct EamGeometry {
  int nsh = 0;
  std::vector<ShellNb> nb[2];           // neighbours within rc, order (sh, dz, dy, dX)
  std::vector<JumpEntry> dE[2][8];      // (N(s) u N(t)) \ {s,t} with sh_s != sh_t, order (dz, dy, dX)
  std::vector<JumpEntry> refresh[2][8]; // dE list plus s and t
  void build(int nshells) {
    nsh = nshells;
    for (int p = 0; p < 2; ++p) {
      nb[p].clear();
      for (int dz = -3; dz <= 3; ++dz)
        for (int dy = -3; dy <= 3; ++dy)
          for (int dx = -5; dx <= 5; ++dx) {
            if (!dx && !dy && !dz) continue;
            const int sh = shell_of_d2(half_coord_d2(p, dx, dy, dz), nsh);
            if (sh) nb[p].push_back({dx, dy, dz, sh});
          }
      std::stable_sort(nb[p].begin(), nb[p].end(), [](const ShellNb& a, const ShellNb& b) {
        if (a.sh != b.sh) return a.sh < b.sh;
        if (a.dz != b.dz) return a.dz < b.dz;
        if (a.dy != b.dy) return a.dy < b.dy;
        return a.dx < b.dx;
      });
      for (int b = 0; b < 8; ++b) {
        const Off t = kNN1[p][b];
        auto& L = dE[p][b];
        auto& R = refresh[p][b];
        L.clear();
        R.clear();
        for (int dz = -4; dz <= 4; ++dz)
          for (int dy = -4; dy <= 4; ++dy)
            for (int dx = -6; dx <= 6; ++dx) {
              const bool is_s = !dx && !dy && !dz;
              const bool is_t = dx == t.dx && dy == t.dy && dz == t.dz;
              const int sh_s = is_s ? kShellSelf : shell_of_d2(half_coord_d2(p, dx, dy, dz), nsh);
              const int sh_t = is_t ? kShellSelf
                                    : shell_of_d2(half_coord_d2(p + t.dx, dx - t.dx, dy - t.dy, dz - t.dz), nsh);
              if (sh_s == 0 && sh_t == 0) continue;
              if (sh_s == sh_t) continue;
              R.push_back({dx, dy, dz, sh_s, sh_t});
              if (!is_s && !is_t) L.push_back({dx, dy, dz, sh_s, sh_t});
            }
      }
    }
  }
};

// ---------------------------------------------------------------------------
// Synthetic Johnson-form EAM (the model the configs name; not in the reference).
//   phi_XX(r) = A exp(-alpha (r/re - 1)) - B exp(-beta (r/re - 1))
//   f_X(r)    = fe exp(-beta (r/re - 1)),  fe = 1
//   F(rho)    = -sqrt(rho)
//   phi_XY    = 1/2 [ f_Y/f_X phi_XX + f_X/f_Y phi_YY ]   (Johnson 1989 alloy rule)
// A, B, alpha, beta, re per species: Fe-like base x (1 + 0.1 (2u - 1)).
// phi, f tabulated on 5000 points of [0, rc]; F on 5000 points of rho step 2^-7.
// Cubic (Catmull-Rom) interpolation per cell.  f at the shells is quantised to
// 2^-24 so the density cache is an exact int32 sum.
// ---------------------------------------------------------------------------
constexpr int kTabN = 5000;
constexpr double kRhoStep = 0x1p-7;
constexpr int kRhoCellShift = 17;  // rho (Q.24) >> 17 = cell index for step 2^-7
constexpr double kRhoScale = 0x1p24;
const double kBase[5] = {0.80, 0.45, 8.0, 4.5, 2.4725};  // A, B, alpha, beta, re (Fe-like base)

void catmull_coefs(const std::vector<double>& F, int k, double c[4]) {
  const int n = static_cast<int>(F.size());
  auto m = [&](int i) {
    if (i <= 0) return F[1] - F[0];
    if (i >= n - 1) return F[n - 1] - F[n - 2];
    return 0.5 * (F[i + 1] - F[i - 1]);
  };
  const double mk = m(k), mk1 = m(k + 1);
  c[0] = F[k];
  c[1] = mk;
  c[2] = ((3.0 * (F[k + 1] - F[k])) - (2.0 * mk)) - mk1;
  c[3] = ((2.0 * (F[k] - F[k + 1])) + mk) + mk1;
}
inline double cubic_eval(const double c[4], double p) {
  return std::fma(std::fma(std::fma(c[3], p, c[2]), p, c[1]), p, c[0]);
}
double interp_table(const std::vector<double>& T, double step, double x) {
  const double q = x / step;
  int k = static_cast<int>(std::floor(q));
  if (k > static_cast<int>(T.size()) - 2) k = static_cast<int>(T.size()) - 2;
  const double p = q - static_cast<double>(k);
  double c[4];
  catmull_coefs(T, k, c);
  return cubic_eval(c, p);
}

struct Eam {
  int nsh = 0;
  double par[4][5];          // A, B, alpha, beta, re
  double rsh[5];
  double f_sh[4][5];
  double phi_sh[4][4][5];
  int32_t fq[4][7];          // [0] none, [1..5] shells, [6] self
  double phi64[4][4][7];     // pair table with zeros at none/self
  float phi32[4][4][7];
  std::vector<double> coef;  // kTabN x 4 (double)
  std::vector<float> hi, lo, c1f, c2f, c3f;

  void build(uint64_t pot_seed, double a, double rc, int nshells) {
    nsh = nshells;
    Xoshiro x = make_stream(pot_seed, kTagPotential, 0);
    for (int s = 0; s < 4; ++s)
      for (int p = 0; p < 5; ++p) {
        const double u = x.uniform();
        par[s][p] = kBase[p] * (1.0 + 0.1 * (2.0 * u - 1.0));
      }
    for (int i = 0; i < 5; ++i) rsh[i] = a * std::sqrt(static_cast<double>(kShellD2[i])) / 2.0;
    const double dr = rc / static_cast<double>(kTabN - 1);
    double phi_pure[4][5];
    for (int s = 0; s < 4; ++s) {
      std::vector<double> ft(kTabN), pt(kTabN);
      const double A = par[s][0], B = par[s][1], al = par[s][2], be = par[s][3], re = par[s][4];
      for (int k = 0; k < kTabN; ++k) {
        const double r = static_cast<double>(k) * dr;
        ft[k] = 1.0 * std::exp(-be * (r / re - 1.0));
        pt[k] = A * std::exp(-al * (r / re - 1.0)) - B * std::exp(-be * (r / re - 1.0));
      }
      for (int i = 0; i < 5; ++i) {
        f_sh[s][i] = interp_table(ft, dr, rsh[i]);
        phi_pure[s][i] = interp_table(pt, dr, rsh[i]);
      }
    }
    for (int X = 0; X < 4; ++X)
      for (int Y = 0; Y < 4; ++Y)
        for (int i = 0; i < 5; ++i) {
          if (X == Y) {
            phi_sh[X][Y][i] = phi_pure[X][i];
          } else {
            const double fx = f_sh[X][i], fy = f_sh[Y][i];
            phi_sh[X][Y][i] = 0.5 * ((fy / fx) * phi_pure[X][i] + (fx / fy) * phi_pure[Y][i]);
          }
        }
    for (int X = 0; X < 4; ++X) {
      fq[X][0] = 0;
      fq[X][6] = 0;
      for (int i = 0; i < 5; ++i) fq[X][i + 1] = (i < nsh) ? static_cast<int32_t>(std::llround(f_sh[X][i] * kRhoScale)) : 0;
      for (int Y = 0; Y < 4; ++Y) {
        for (int j = 0; j < 7; ++j) {
          const double v = (j >= 1 && j <= 5 && j - 1 < nsh) ? phi_sh[X][Y][j - 1] : 0.0;
          phi64[X][Y][j] = v;
          phi32[X][Y][j] = static_cast<float>(v);
        }
      }
    }
    std::vector<double> Ft(kTabN);
    for (int k = 0; k < kTabN; ++k) Ft[k] = -std::sqrt(static_cast<double>(k) * kRhoStep);
    coef.assign(static_cast<size_t>(kTabN) * 4, 0.0);
    hi.assign(kTabN, 0.f); lo.assign(kTabN, 0.f); c1f.assign(kTabN, 0.f); c2f.assign(kTabN, 0.f); c3f.assign(kTabN, 0.f);
    for (int k = 0; k + 1 < kTabN; ++k) {
      double c[4];
      catmull_coefs(Ft, k, c);
      for (int j = 0; j < 4; ++j) coef[static_cast<size_t>(k) * 4 + j] = c[j];
      hi[k] = static_cast<float>(c[0]);
      lo[k] = static_cast<float>(c[0] - static_cast<double>(hi[k]));
      c1f[k] = static_cast<float>(c[1]);
      c2f[k] = static_cast<float>(c[2]);
      c3f[k] = static_cast<float>(c[3]);
    }
  }

  // F(rho) in FP64 from the fixed-point density; cell = r >> 17.
  double F64(int32_t r) const {
    const int k = r >> kRhoCellShift;
    const double p = static_cast<double>(r & ((1 << kRhoCellShift) - 1)) * 0x1p-17;
    return cubic_eval(&coef[static_cast<size_t>(k) * 4], p);
  }
  // F(r1) - F(r0) in FP32: node difference from the hi/lo split plus polynomial difference.
  float dF32(int32_t r1, int32_t r0) const {
    const int k1 = r1 >> kRhoCellShift, k0 = r0 >> kRhoCellShift;
    const float p1 = static_cast<float>(r1 & ((1 << kRhoCellShift) - 1)) * 0x1p-17f;
    const float p0 = static_cast<float>(r0 & ((1 << kRhoCellShift) - 1)) * 0x1p-17f;
    const float q1 = std::fmaf(std::fmaf(c3f[k1], p1, c2f[k1]), p1, c1f[k1]) * p1;
    const float q0 = std::fmaf(std::fmaf(c3f[k0], p0, c2f[k0]), p0, c1f[k0]) * p0;
    const float node = (hi[k1] - hi[k0]) + (lo[k1] - lo[k0]);
    return node + (q1 - q0);
  }
};

// Kahan state and its commutative merge (two-sum of the heads, corrections added).
struct Comp { float s = 0.f, c = 0.f; };
inline void kahan_add(Comp& a, float v) {
  const float y = v - a.c;
  const float t = a.s + y;
  a.c = (t - a.s) - y;
  a.s = t;
}
inline Comp comp_merge(const Comp& a, const Comp& b) {
  const float s = a.s + b.s;
  const float bb = s - a.s;
  const float e = (a.s - (s - bb)) + (b.s - bb);
  Comp r;
  r.s = s;
  r.c = (a.c + b.c) - e;
  return r;
}

// ---------------------------------------------------------------------------
struct Block {
  double evo[8];
  Xoshiro xs, xt;
  std::mt19937 ms, mt;
  int64_t hops = 0;
};

struct VacRec {
  int64_t site;
  uint8_t avail;
  double rates[8];
};

struct Job {
  ao_config c{};
  int64_t n[3]{};
  int64_t sx = 0, sy = 0, sz = 0, ns = 0;
  int nb[3]{};
  std::vector<int64_t> bstart[3];
  int nblocks = 0;
  std::vector<uint8_t> occ;
  std::vector<int32_t> rho;
  bool eam_on = false;
  Eam eam;
  EamGeometry geo;
  std::vector<Block> blk;
  int64_t round = 0, hops = 0;
  std::vector<ao_event> events;
  int64_t st_nact = 0, st_dirty = 0, st_start = 0;
  bool small_blocks = false;  // a block edge < 8 cells: sector halos would overlap

  inline int64_t wrap(int64_t v, int64_t m) const {
    v %= m;
    return v < 0 ? v + m : v;
  }
  inline int64_t site(int64_t X, int64_t y, int64_t z) const {
    return wrap(X, sx) + sx * (wrap(y, sy) + sy * wrap(z, sz));
  }
  inline void coords(int64_t s, int64_t& X, int64_t& y, int64_t& z) const {
    X = s % sx;
    y = (s / sx) % sy;
    z = s / (sx * sy);
  }
  inline int64_t nbr(int64_t s, int dx, int dy, int dz) const {
    int64_t X, y, z;
    coords(s, X, y, z);
    return site(X + dx, y + dy, z + dz);
  }
  inline double EXP(double x) const { return c.math_mode == AO_MATH_LIBM ? std::exp(x) : port_exp(x); }
  inline double LOG(double x) const { return c.math_mode == AO_MATH_LIBM ? std::log(x) : port_log(x); }

  void compute_rho() {
    if (!eam_on) return;
    rho.assign(static_cast<size_t>(ns), 0);
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < ns; ++s) {
      int64_t X, y, z;
      coords(s, X, y, z);
      const auto& L = geo.nb[X & 1];
      int32_t acc = 0;
      for (const auto& e : L) {
        const uint8_t o = occ[static_cast<size_t>(site(X + e.dx, y + e.dy, z + e.dz))];
        if (o != kV) acc += eam.fq[species_index(o)][e.sh];
      }
      rho[static_cast<size_t>(s)] = acc;
    }
  }

  // BondsCounter::count / count_exchange (bonds_counter.cpp:35-129): 1nn then masked 2nn,
  // summed in order; `ovr` is the site whose type is replaced by `ovr_code`.
  double bond_count(int64_t s, uint8_t src, int64_t ovr, uint8_t ovr_code) const {
    int64_t X, y, z;
    coords(s, X, y, z);
    const int p = static_cast<int>(X & 1);
    const int si = bond_index(src);
    double energy = 0.0;
    for (int b = 0; b < 8; ++b) {
      const int64_t q = site(X + kNN1[p][b].dx, y + kNN1[p][b].dy, z + kNN1[p][b].dz);
      const uint8_t o = (q == ovr) ? ovr_code : occ[static_cast<size_t>(q)];
      energy += kBonds.b1[bond_index(o)][si];
    }
    for (int b = 0; b < 6; ++b) {
      if (!((kNN2Status >> b) & 1)) continue;
      const int64_t q = site(X + kNN2[b].dx, y + kNN2[b].dy, z + kNN2[b].dz);
      const uint8_t o = (q == ovr) ? ovr_code : occ[static_cast<size_t>(q)];
      energy += kBonds.b2[bond_index(o)][si];
    }
    return energy;
  }

  // VacRatesSolver::deltaE (vacancy_rates_solver.cpp:29-172), pair-bond branch.
  double dE_pairbond(int64_t s, int64_t t, uint8_t X) const {
    const double e_src_before = bond_count(s, kV, -1, 0);
    const double e_des_before = bond_count(t, X, -1, 0);
    const double e_before = e_src_before + e_des_before;
    const double e_src_after = bond_count(s, X, t, kV);
    const double e_des_after = bond_count(t, kV, s, X);
    const double e_after = e_src_after + e_des_after;
    return e_after - e_before;
  }

  // EAM dE in the defined order: 32 interleaved partial sums over the jump's site
  // list (entry i -> partial i mod 32), merged by a xor butterfly (partner distance
  // 16, 8, 4, 2, 1; p[i] <- p[i] + p[i ^ m]), plus the moving atom's own embedding
  // change.
  static double butterfly32(double* p) {
    for (int m = 16; m >= 1; m >>= 1) {
      double t[32];
      for (int i = 0; i < 32; ++i) t[i] = p[i] + p[i ^ m];
      for (int i = 0; i < 32; ++i) p[i] = t[i];
    }
    return p[0];
  }
  static Comp butterfly32(Comp* p) {
    for (int m = 16; m >= 1; m >>= 1) {
      Comp t[32];
      for (int i = 0; i < 32; ++i) t[i] = comp_merge(p[i], p[i ^ m]);
      for (int i = 0; i < 32; ++i) p[i] = t[i];
    }
    return p[0];
  }
  double dE_eam64(int64_t s, int b, uint8_t Xc) const {
    int64_t X0, y0, z0;
    coords(s, X0, y0, z0);
    const int p = static_cast<int>(X0 & 1);
    const int X = species_index(Xc);
    const auto& L = geo.dE[p][b];
    double acc[32];
    for (double& v : acc) v = 0.0;
    for (size_t i = 0; i < L.size(); ++i) {
      const auto& e = L[i];
      const int64_t j = site(X0 + e.dx, y0 + e.dy, z0 + e.dz);
      const uint8_t o = occ[static_cast<size_t>(j)];
      if (o == kV) continue;
      const int Y = species_index(o);
      const int32_t r = rho[static_cast<size_t>(j)];
      const int32_t d = eam.fq[X][e.sh_s] - eam.fq[X][e.sh_t];
      const double Fa = eam.F64(r + d);
      const double Fb = eam.F64(r);
      const double T = (Fa - Fb) + (eam.phi64[X][Y][e.sh_s] - eam.phi64[X][Y][e.sh_t]);
      acc[i & 31] += T;
    }
    const double tsum = butterfly32(acc);
    const int64_t t = site(X0 + kNN1[p][b].dx, y0 + kNN1[p][b].dy, z0 + kNN1[p][b].dz);
    const double EX = eam.F64(rho[static_cast<size_t>(s)] - eam.fq[X][1]) - eam.F64(rho[static_cast<size_t>(t)]);
    return EX + tsum;
  }

  double dE_eam32(int64_t s, int b, uint8_t Xc) const {
    int64_t X0, y0, z0;
    coords(s, X0, y0, z0);
    const int p = static_cast<int>(X0 & 1);
    const int X = species_index(Xc);
    const auto& L = geo.dE[p][b];
    Comp acc[32];
    for (size_t i = 0; i < L.size(); ++i) {
      const auto& e = L[i];
      const int64_t j = site(X0 + e.dx, y0 + e.dy, z0 + e.dz);
      const uint8_t o = occ[static_cast<size_t>(j)];
      if (o == kV) continue;
      const int Y = species_index(o);
      const int32_t r = rho[static_cast<size_t>(j)];
      const int32_t d = eam.fq[X][e.sh_s] - eam.fq[X][e.sh_t];
      const float T = eam.dF32(r + d, r) + (eam.phi32[X][Y][e.sh_s] - eam.phi32[X][Y][e.sh_t]);
      kahan_add(acc[i & 31], T);
    }
    const Comp m = butterfly32(acc);
    const int64_t t = site(X0 + kNN1[p][b].dx, y0 + kNN1[p][b].dy, z0 + kNN1[p][b].dz);
    const float EX = eam.dF32(rho[static_cast<size_t>(s)] - eam.fq[X][1], rho[static_cast<size_t>(t)]);
    const float dE = EX + (m.s - m.c);
    return static_cast<double>(dE);
  }

  // RatesSolver::rate / arrhenius (rates_solver.cpp:12-26).
  double rate_of(uint8_t X, double dE) const {
    const double Ea = e0_of(X) + dE / 2;
    return c.attempt_freq * EXP(-Ea / (kBoltzmann * c.temperature));
  }

  // VacancyHash::beforeRatesUpdate2 / updateRates2 (vac_hash.cpp:7-37): available
  // directions are atom neighbours; rates of the others stay 0.
  void vacancy_rates(int64_t s, VacRec& v, double* de8 = nullptr) const {
    int64_t X0, y0, z0;
    coords(s, X0, y0, z0);
    const int p = static_cast<int>(X0 & 1);
    v.site = s;
    v.avail = 0;
    for (int b = 0; b < 8; ++b) {
      v.rates[b] = 0.0;
      if (de8) de8[b] = 0.0;
      const int64_t t = site(X0 + kNN1[p][b].dx, y0 + kNN1[p][b].dy, z0 + kNN1[p][b].dz);
      const uint8_t o = occ[static_cast<size_t>(t)];
      if (!is_atom(o)) continue;
      v.avail |= static_cast<uint8_t>(1u << b);
      double dE;
      if (!eam_on) dE = dE_pairbond(s, t, o);
      else if (c.precision == AO_FP32C) dE = dE_eam32(s, b, o);
      else dE = dE_eam64(s, b, o);
      if (de8) de8[b] = dE;
      v.rates[b] = rate_of(o, dE);
    }
  }

  void block_cells(int b, int sec, int64_t lo[3], int64_t hi[3]) const {
    const int bi[3] = {b % nb[0], (b / nb[0]) % nb[1], b / (nb[0] * nb[1])};
    for (int d = 0; d < 3; ++d) {
      const int64_t s0 = bstart[d][static_cast<size_t>(bi[d])], s1 = bstart[d][static_cast<size_t>(bi[d]) + 1];
      const int64_t half = (s1 - s0) / 2;
      if ((sec >> d) & 1) {
        lo[d] = s0 + half;
        hi[d] = s1;
      } else {
        lo[d] = s0;
        hi[d] = s0 + half;
      }
    }
  }

  double draw_select(Block& B) const {
    if (c.rng_mode == AO_RNG_MT19937_REF) return static_cast<double>(B.ms()) * (1.0 / 4294967295.0);
    return B.xs.uniform();
  }
  double draw_time(Block& B) const {
    if (c.rng_mode == AO_RNG_MT19937_REF) {
      std::uniform_real_distribution<double> dis(0, 1);
      return dis(B.mt);
    }
    return B.xt.uniform_open0();
  }

  inline int64_t min_image(int64_t d, int64_t m) const {
    d = d < 0 ? -d : d;
    d %= m;
    return std::min(d, m - d);
  }
  bool near_cells(int64_t a, int64_t b, int64_t D) const {
    int64_t Xa, ya, za, Xb, yb, zb;
    coords(a, Xa, ya, za);
    coords(b, Xb, yb, zb);
    return min_image((Xa >> 1) - (Xb >> 1), n[0]) <= D && min_image(ya - yb, n[1]) <= D && min_image(za - zb, n[2]) <= D;
  }

  // One block's sector in one round: SubLattice::startTimeLoop body
  // (src/algorithms/sl/sublattice.inl:64-140), CPU wrappers (:192-211).
  int run_block(int b, int64_t rnd, std::vector<ao_event>& ev, int64_t st[4]) {
    const int sec = kSectorOrder[rnd % 8];
    const int64_t step = rnd / 8;
    int64_t lo[3], hi[3];
    block_cells(b, sec, lo, hi);
    Block& B = blk[static_cast<size_t>(b)];
    const double thr = static_cast<double>(step + 1) * c.window - B.evo[sec];
    double sector_time = 0.0;
    std::vector<VacRec> vr;
    bool first = true;
    const int64_t D = eam_on ? 4 : 3;
    int64_t guard = 0;
    while (sector_time < thr) {
      // ABVIModel::calcRates (models/abvi/kmc.cpp:68-115): z-y-x scan of the sector.
      vr.clear();
      double total = 0.0;
      for (int64_t z = lo[2]; z < hi[2]; ++z)
        for (int64_t y = lo[1]; y < hi[1]; ++y)
          for (int64_t X = 2 * lo[0]; X < 2 * hi[0]; ++X) {
            const int64_t s = X + sx * (y + sy * z);
            if (occ[static_cast<size_t>(s)] != kV) continue;
            VacRec v;
            vacancy_rates(s, v);
            for (int k = 0; k < 8; ++k)
              if ((v.avail >> k) & 1) total += v.rates[k];
            vr.push_back(v);
          }
      if (first) {
        st[3] += static_cast<int64_t>(vr.size());
        first = false;
      }
      if (total == 0.0 || std::fabs(total) < DBL_EPSILON) {
        sector_time = thr;
      } else {
        // ModelAdapter::selectAndPerform (src/models/model_adapter.h:95-101)
        const double u = draw_select(B);
        const double expected = u * total;
        // ABVIModel::select (kmc.cpp:242-309)
        double acc = 0.0;
        int64_t from = -1;
        int dir = -1;
        for (const auto& v : vr) {
          for (int k = 0; k < 8; ++k) {
            acc += v.rates[k];
            if (acc > expected) {
              from = v.site;
              dir = k;
              break;
            }
          }
          if (from >= 0) break;
        }
        int64_t to = -1;
        int64_t nd = 0;
        uint8_t X = 0;
        if (from >= 0) {
          // ABVIModel::perform (kmc.cpp:358-396)
          int64_t X0, y0, z0;
          coords(from, X0, y0, z0);
          const int p = static_cast<int>(X0 & 1);
          to = site(X0 + kNN1[p][dir].dx, y0 + kNN1[p][dir].dy, z0 + kNN1[p][dir].dz);
          X = occ[static_cast<size_t>(to)];
          occ[static_cast<size_t>(to)] = kV;
          occ[static_cast<size_t>(from)] = X;
          if (eam_on) {
            const int xs = species_index(X);
            for (const auto& e : geo.refresh[p][dir]) {
              const int64_t j = site(X0 + e.dx, y0 + e.dy, z0 + e.dz);
              rho[static_cast<size_t>(j)] += eam.fq[xs][e.sh_s] - eam.fq[xs][e.sh_t];
            }
          }
          // device work model: vacancies of the sector within D cells of the hop
          nd = 0;
          for (const auto& v : vr) {
            const int64_t vs = (v.site == from) ? to : v.site;
            int64_t vX, vy, vz;
            coords(vs, vX, vy, vz);
            const int64_t cx = vX >> 1;
            const bool in = cx >= lo[0] && cx < hi[0] && vy >= lo[1] && vy < hi[1] && vz >= lo[2] && vz < hi[2];
            if (in && near_cells(vs, from, D)) ++nd;
          }
          st[0] += 1;
          st[1] += static_cast<int64_t>(vr.size());
          st[2] += nd;
          B.hops += 1;
        }
        // sublattice.inl:118-120
        const double u2 = draw_time(B);
        const double dt = -LOG(u2) / total;
        sector_time += dt;
        if (from >= 0 && c.log_events) {
          ao_event e{};
          e.round = rnd;
          e.hop = B.hops - 1;
          e.from_site = from;
          e.to_site = to;
          e.block = b;
          e.species = X;
          e.u = u;
          e.total = total;
          e.dt = dt;
          e.n_act = static_cast<int32_t>(vr.size());
          e.n_dirty = static_cast<int32_t>(nd);
          ev.push_back(e);
        }
      }
      if (++guard > 100000000) return -10;
    }
    B.evo[sec] += sector_time;
    return 0;
  }

  int run_round() {
    if (small_blocks) return -3;
    const int64_t rnd = round;
    std::vector<std::vector<ao_event>> ev(static_cast<size_t>(nblocks));
    std::vector<std::array<int64_t, 4>> st(static_cast<size_t>(nblocks), {0, 0, 0, 0});
    int rc = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(min : rc)
    for (int b = 0; b < nblocks; ++b) {
      const int r = run_block(b, rnd, ev[static_cast<size_t>(b)], st[static_cast<size_t>(b)].data());
      if (r < rc) rc = r;
    }
    if (rc) return rc;
    for (int b = 0; b < nblocks; ++b) {
      hops += st[static_cast<size_t>(b)][0];
      st_nact += st[static_cast<size_t>(b)][1];
      st_dirty += st[static_cast<size_t>(b)][2];
      st_start += st[static_cast<size_t>(b)][3];
      if (c.log_events) events.insert(events.end(), ev[static_cast<size_t>(b)].begin(), ev[static_cast<size_t>(b)].end());
    }
    ++round;
    return 0;
  }

  // Asynchronous order: each (block, round) runs as soon as, for every neighbour offset
  // d in {-1,0,1}^3, the neighbour has completed its latest earlier round whose staged
  // region (sector plus a 2-cell halo) overlaps this round's region.  Items are taken in
  // a random order among the ready ones; the result must equal run_round's.
  static int flow_lag(int phase, const int d[3]) {
    const int now = kSectorOrder[phase];
    for (int k = 1; k <= 8; ++k) {
      const int then = kSectorOrder[(phase - k + 8) % 8];
      bool ov = true;
      for (int a = 0; a < 3 && ov; ++a) {
        const int hn = (now >> a) & 1, ht = (then >> a) & 1;
        if (d[a] == 1) ov = hn == 1 && ht == 0;    // the +1 neighbour's low half meets our high half
        if (d[a] == -1) ov = hn == 0 && ht == 1;   // the -1 neighbour's high half meets our low half
      }
      if (ov) return k;
    }
    return 0;  // no region of that neighbour ever meets this one
  }
  int run_rounds_flow(int64_t n_rounds, uint64_t order_seed) {
    if (small_blocks) return -3;
    const int64_t r0 = round;
    std::vector<int64_t> done(static_cast<size_t>(nblocks), r0);  // rounds completed
    Xoshiro pick = make_stream(order_seed, 99, 0);
    std::vector<int> ready;
    for (;;) {
      ready.clear();
      bool all = true;
      for (int b = 0; b < nblocks; ++b) {
        const int64_t r = done[static_cast<size_t>(b)];
        if (r >= r0 + n_rounds) continue;
        all = false;
        const int bi[3] = {b % nb[0], (b / nb[0]) % nb[1], b / (nb[0] * nb[1])};
        bool ok = true;
        for (int dz = -1; dz <= 1 && ok; ++dz)
          for (int dy = -1; dy <= 1 && ok; ++dy)
            for (int dx = -1; dx <= 1 && ok; ++dx) {
              const int d[3] = {dx, dy, dz};
              const int k = flow_lag(static_cast<int>(r % 8), d);
              if (!k) continue;
              int yi[3];
              for (int a = 0; a < 3; ++a) yi[a] = (bi[a] + d[a] + nb[a]) % nb[a];
              const int y = yi[0] + nb[0] * (yi[1] + nb[1] * yi[2]);
              if (done[static_cast<size_t>(y)] < r - k + 1) ok = false;
            }
        if (ok) ready.push_back(b);
      }
      if (all) break;
      if (ready.empty()) return -11;  // no item ready: the rule would deadlock
      int b = ready[0];
      if (order_seed) {
        b = ready[static_cast<size_t>(pick.below(ready.size()))];
      } else {  // seed 0: the ready block furthest ahead, to stretch the skew between blocks
        for (int c2 : ready)
          if (done[static_cast<size_t>(c2)] > done[static_cast<size_t>(b)]) b = c2;
      }
      std::vector<ao_event> ev;
      int64_t st[4] = {0, 0, 0, 0};
      const int rc = run_block(b, done[static_cast<size_t>(b)], ev, st);
      if (rc) return rc;
      hops += st[0];
      st_nact += st[1];
      st_dirty += st[2];
      st_start += st[3];
      if (c.log_events) events.insert(events.end(), ev.begin(), ev.end());
      ++done[static_cast<size_t>(b)];
    }
    round = r0 + n_rounds;
    return 0;
  }
};

int64_t ratio_total(const ao_config& c) {
  int64_t t = 0;
  for (int i = 0; i < 4; ++i) t += c.ratio[i];
  return t;
}
// LatticeTypes::randomAtomsType (src/lattice/lattice_types.cpp:9-19)
uint8_t pick_type(const ao_config& c, int64_t hit) {
  int64_t acc = 0;
  for (int i = 0; i < 4; ++i) {
    acc += c.ratio[i];
    if (acc >= hit) return static_cast<uint8_t>(c.type_codes[i]);
  }
  return kFe;
}

void create_xoshiro(Job& J) {
  const int64_t R = ratio_total(J.c);
  Xoshiro xt = make_stream(J.c.seed, kTagTypes, 0);
  for (int64_t s = 0; s < J.ns; ++s) {
    const int64_t hit = 1 + static_cast<int64_t>(xt.below(static_cast<uint64_t>(R)));
    J.occ[static_cast<size_t>(s)] = pick_type(J.c, hit);
  }
  Xoshiro xv = make_stream(J.c.seed, kTagVacancy, 0);
  int64_t placed = 0;
  while (placed < J.c.n_vacancies) {
    const int64_t s = static_cast<int64_t>(xv.below(static_cast<uint64_t>(J.ns)));
    if (J.occ[static_cast<size_t>(s)] != kV) {
      J.occ[static_cast<size_t>(s)] = kV;
      ++placed;
    }
  }
}

// creation::createAtomsRandom / createRandom (src/creation.cpp:18-164) for one rank:
// one draw per site of the ghost-padded array in z-y-x order, ghost = ceil(rc/a).
// creation::createAtomsRandom (src/creation.cpp:18-94) for one rank holding the whole box: one
// uniform_int_distribution<>(1, sum ratio) draw per site of the ghost-padded array (ghost =
// ceil(cutoff / lattice_const) cells) in z-y-x order with mt19937(create_types).
void create_atoms_mt(Job& J) {
  const int64_t R = ratio_total(J.c);
  const int64_t g = static_cast<int64_t>(std::ceil(J.c.cutoff / J.c.lattice_const));
  const int64_t px = 2 * (J.n[0] + 2 * g), py = J.n[1] + 2 * g, pz = J.n[2] + 2 * g;
  std::uniform_int_distribution<> types_dis(1, static_cast<int>(R));
  std::mt19937 types_rng(static_cast<std::mt19937::result_type>(J.c.seed));
  for (int64_t z = 0; z < pz; ++z)
    for (int64_t y = 0; y < py; ++y)
      for (int64_t x = 0; x < px; ++x) {
        const int64_t hit = types_dis(types_rng);
        const uint8_t t = pick_type(J.c, hit);
        const int64_t ix = x - 2 * g, iy = y - g, iz = z - g;
        if (ix >= 0 && ix < J.sx && iy >= 0 && iy < J.sy && iz >= 0 && iz < J.sz)
          J.occ[static_cast<size_t>(ix + J.sx * (iy + J.sy * iz))] = t;
      }
}

// creation::createRandom's vacancies (src/creation.cpp:126-160): uniform_int_distribution<long
// long>(0, sites - 1) with mt19937(create_vacancy) until n_vacancies distinct sites hold one.
void create_mt(Job& J) {
  create_atoms_mt(J);
  std::uniform_int_distribution<long long> va_dis(0, J.ns - 1);
  std::mt19937 va_rng(static_cast<std::mt19937::result_type>(J.c.seed_vacancy));
  int64_t placed = 0;
  while (placed < J.c.n_vacancies) {
    int64_t id = va_dis(va_rng);
    const int64_t x = id % J.sx;
    id /= J.sx;
    const int64_t y = id % J.sy;
    const int64_t z = id / J.sy;
    const size_t s = static_cast<size_t>(x + J.sx * (y + J.sy * z));
    if (J.occ[s] != kV) {
      J.occ[s] = kV;
      ++placed;
    }
  }
}

// creation::createFromPile (src/creation.cpp:184-230): the alloy of createAtomsRandom, then a
// vacancy at every position of the pile file (x doubled, y, z) that lies inside the box; positions
// outside it are skipped and repeated ones change nothing.  The reference marks the vacancy in
// LatticesList::_lattices only, which its hash-set occupancy store never reads; here the site
// becomes a vacancy of the occupancy, whatever atom it held (as createRandom's placement).
void create_pile(Job& J) {
  create_atoms_mt(J);
  for (int64_t i = 0; i < J.c.pile_n; ++i) {
    const int64_t x = J.c.pile_xyz[3 * i], y = J.c.pile_xyz[3 * i + 1], z = J.c.pile_xyz[3 * i + 2];
    if (x < 0 || x >= J.sx || y < 0 || y >= J.sy || z < 0 || z >= J.sz) continue;  // isIn(x / 2, y, z)
    J.occ[static_cast<size_t>(x + J.sx * (y + J.sy * z))] = kV;
  }
}

void set_err(char* err, int errlen, const char* msg) {
  if (err && errlen > 0) std::snprintf(err, static_cast<size_t>(errlen), "%s", msg);
}

}  // namespace

extern "C" {

void* ao_create(const ao_config* cfg, char* err, int errlen) {
  auto J = std::make_unique<Job>();
  J->c = *cfg;
  for (int d = 0; d < 3; ++d) {
    J->n[d] = cfg->box[d];
    J->nb[d] = cfg->blocks[d] > 0 ? cfg->blocks[d] : 1;
    // static evaluation needs distinct neighbour sites (EAM reaches +-2 cells);
    // running the sector schedule additionally needs block edges >= 8 (ao_run*)
    if (J->n[d] < (cfg->energy_model == AO_MODEL_EAM ? 6 : 4)) { set_err(err, errlen, "box edge too small"); return nullptr; }
    if (J->nb[d] > J->n[d]) { set_err(err, errlen, "more blocks than cells"); return nullptr; }
    // reference rank split: low = coord*(n/p) + min(coord, n%p)  (simulation.cpp:116 comments)
    J->bstart[d].resize(static_cast<size_t>(J->nb[d]) + 1);
    for (int k = 0; k <= J->nb[d]; ++k)
      J->bstart[d][static_cast<size_t>(k)] = k * (J->n[d] / J->nb[d]) + std::min<int64_t>(k, J->n[d] % J->nb[d]);
    for (int k = 0; k < J->nb[d]; ++k)
      if (J->bstart[d][static_cast<size_t>(k) + 1] - J->bstart[d][static_cast<size_t>(k)] < 8) J->small_blocks = true;
  }
  J->sx = 2 * J->n[0];
  J->sy = J->n[1];
  J->sz = J->n[2];
  J->ns = J->sx * J->sy * J->sz;
  J->nblocks = J->nb[0] * J->nb[1] * J->nb[2];
  J->eam_on = cfg->energy_model == AO_MODEL_EAM;
  int nsh = 0;
  for (int i = 0; i < 5; ++i)
    if (cfg->lattice_const * std::sqrt(static_cast<double>(kShellD2[i])) / 2.0 < cfg->cutoff) nsh = i + 1;
  if (2.0 * cfg->lattice_const < cfg->cutoff) { set_err(err, errlen, "cutoff reaches the 6th shell"); return nullptr; }
  if (J->eam_on) {
    J->geo.build(nsh);
    J->eam.build(cfg->pot_seed, cfg->lattice_const, cfg->cutoff, nsh);
    // every density the path can reach must stay inside the F table
    int64_t rmax = 0;
    const int counts[5] = {8, 6, 12, 24, 8};
    for (int i = 0; i < nsh; ++i) {
      int32_t m = 0;
      for (int X = 0; X < 4; ++X) m = std::max(m, J->eam.fq[X][i + 1]);
      rmax += static_cast<int64_t>(counts[i]) * m;
    }
    if ((rmax >> kRhoCellShift) > kTabN - 3) { set_err(err, errlen, "density range exceeds the F table"); return nullptr; }
  }
  J->occ.assign(static_cast<size_t>(J->ns), kFe);
  if (cfg->creation_mode == AO_CREATE_XOSHIRO) create_xoshiro(*J);
  else if (cfg->creation_mode == AO_CREATE_MT19937_REF) create_mt(*J);
  else if (cfg->creation_mode == AO_CREATE_MT19937_PILE) create_pile(*J);
  J->compute_rho();
  J->blk.resize(static_cast<size_t>(J->nblocks));
  for (int b = 0; b < J->nblocks; ++b) {
    Block& B = J->blk[static_cast<size_t>(b)];
    for (double& e : B.evo) e = 0.0;
    B.xs = make_stream(cfg->seed, kTagSelect, static_cast<uint64_t>(b));
    B.xt = make_stream(cfg->seed, kTagTime, static_cast<uint64_t>(b));
    B.ms = std::mt19937();
    B.mt = std::mt19937(static_cast<std::mt19937::result_type>(cfg->seed_time_inc));
  }
  return J.release();
}

void ao_destroy(void* h) { delete static_cast<Job*>(h); }
int64_t ao_nsites(void* h) { return static_cast<Job*>(h)->ns; }
int32_t ao_nblocks(void* h) { return static_cast<Job*>(h)->nblocks; }

int ao_set_occupancy(void* h, const uint8_t* occ, int64_t n) {
  Job* J = static_cast<Job*>(h);
  if (n != J->ns) return -1;
  for (int64_t i = 0; i < n; ++i)
    if (occ[i] != kV && !is_atom(occ[i])) return -2;
  std::memcpy(J->occ.data(), occ, static_cast<size_t>(n));
  J->compute_rho();
  return 0;
}
int ao_get_occupancy(void* h, uint8_t* out) {
  Job* J = static_cast<Job*>(h);
  std::memcpy(out, J->occ.data(), static_cast<size_t>(J->ns));
  return 0;
}
int ao_get_rho(void* h, int32_t* out) {
  Job* J = static_cast<Job*>(h);
  if (!J->eam_on) return -1;
  std::memcpy(out, J->rho.data(), static_cast<size_t>(J->ns) * 4);
  return 0;
}
int ao_run_rounds_flow(void* h, int64_t n_rounds, uint64_t order_seed) {
  return static_cast<Job*>(h)->run_rounds_flow(n_rounds, order_seed);
}

int ao_run_rounds(void* h, int64_t n_rounds) {
  Job* J = static_cast<Job*>(h);
  for (int64_t i = 0; i < n_rounds; ++i) {
    const int r = J->run_round();
    if (r) return r;
  }
  return 0;
}
// A hop budget is checked at sublattice time-step boundaries (every 8 sector rounds): the job
// ends at the end of the first time step at which its hop count has reached the budget.
int ao_run(void* h, int64_t hop_budget, int64_t max_rounds) {
  Job* J = static_cast<Job*>(h);
  for (int64_t i = 0; i < max_rounds; ++i) {
    if (hop_budget > 0 && J->round % 8 == 0 && J->hops >= hop_budget) break;
    const int r = J->run_round();
    if (r) return r;
  }
  return 0;
}
int64_t ao_round(void* h) { return static_cast<Job*>(h)->round; }
int64_t ao_total_hops(void* h) { return static_cast<Job*>(h)->hops; }
int64_t ao_num_events(void* h) { return static_cast<int64_t>(static_cast<Job*>(h)->events.size()); }
int ao_get_events(void* h, ao_event* out, int64_t start, int64_t n) {
  Job* J = static_cast<Job*>(h);
  if (start < 0 || start + n > static_cast<int64_t>(J->events.size())) return -1;
  std::memcpy(out, J->events.data() + start, static_cast<size_t>(n) * sizeof(ao_event));
  return 0;
}
int ao_get_block_state(void* h, double* evo, int64_t* hops) {
  Job* J = static_cast<Job*>(h);
  for (int b = 0; b < J->nblocks; ++b) {
    for (int k = 0; k < 8; ++k) evo[b * 8 + k] = J->blk[static_cast<size_t>(b)].evo[k];
    hops[b] = J->blk[static_cast<size_t>(b)].hops;
  }
  return 0;
}
int ao_stats(void* h, int64_t* out4) {
  Job* J = static_cast<Job*>(h);
  out4[0] = J->hops;
  out4[1] = J->st_nact;
  out4[2] = J->st_dirty;
  out4[3] = J->st_start;
  return 0;
}
int ao_vacancy_rates(void* h, int64_t site, double* rates8, double* de8) {
  Job* J = static_cast<Job*>(h);
  if (site < 0 || site >= J->ns || J->occ[static_cast<size_t>(site)] != kV) return -1;
  VacRec v;
  J->vacancy_rates(site, v, de8);
  for (int k = 0; k < 8; ++k) rates8[k] = v.rates[k];
  return v.avail;
}
double ao_bond_count(void* h, int64_t site, int32_t src_code) {
  Job* J = static_cast<Job*>(h);
  return J->bond_count(site, static_cast<uint8_t>(src_code), -1, 0);
}
int ao_eam_export(void* h, double* params, double* f_sh, double* phi_sh, int32_t* fq, double* coef) {
  Job* J = static_cast<Job*>(h);
  if (!J->eam_on) return -1;
  const Eam& E = J->eam;
  for (int s = 0; s < 4; ++s) {
    for (int p = 0; p < 5; ++p) params[s * 5 + p] = E.par[s][p];
    for (int i = 0; i < 5; ++i) f_sh[s * 5 + i] = E.f_sh[s][i];
    for (int t = 0; t < 4; ++t)
      for (int i = 0; i < 5; ++i) phi_sh[(s * 4 + t) * 5 + i] = E.phi_sh[s][t][i];
    for (int j = 0; j < 7; ++j) fq[s * 7 + j] = E.fq[s][j];
  }
  std::memcpy(coef, E.coef.data(), E.coef.size() * sizeof(double));
  return 0;
}
// MEventHook::onStepFinished isolated-Cu count (profiles/m_event_hook.cpp:17-55) and
// the Cu cluster-size histogram by 1nn connectivity.
int ao_cluster_stats(void* h, int64_t* isolated_cu, int64_t* hist, int64_t hist_len) {
  Job* J = static_cast<Job*>(h);
  std::vector<int64_t> label(static_cast<size_t>(J->ns), -1);
  int64_t iso = 0;
  for (int64_t i = 0; i < hist_len; ++i) hist[i] = 0;
  std::vector<int64_t> stack;
  for (int64_t s = 0; s < J->ns; ++s) {
    if (J->occ[static_cast<size_t>(s)] != kCu) continue;
    int64_t X, y, z;
    J->coords(s, X, y, z);
    const int p = static_cast<int>(X & 1);
    bool has = false;
    for (int b = 0; b < 8 && !has; ++b)
      has = J->occ[static_cast<size_t>(J->site(X + kNN1[p][b].dx, y + kNN1[p][b].dy, z + kNN1[p][b].dz))] == kCu;
    if (!has) ++iso;
    if (label[static_cast<size_t>(s)] >= 0) continue;
    int64_t size = 0;
    stack.push_back(s);
    label[static_cast<size_t>(s)] = s;
    while (!stack.empty()) {
      const int64_t q = stack.back();
      stack.pop_back();
      ++size;
      int64_t qX, qy, qz;
      J->coords(q, qX, qy, qz);
      const int qp = static_cast<int>(qX & 1);
      for (int b = 0; b < 8; ++b) {
        const int64_t r = J->site(qX + kNN1[qp][b].dx, qy + kNN1[qp][b].dy, qz + kNN1[qp][b].dz);
        if (J->occ[static_cast<size_t>(r)] == kCu && label[static_cast<size_t>(r)] < 0) {
          label[static_cast<size_t>(r)] = s;
          stack.push_back(r);
        }
      }
    }
    const int64_t bin = size < hist_len ? size : hist_len - 1;
    hist[bin] += 1;
  }
  *isolated_cu = iso;
  return 0;
}

int ao_neighbours(void* h, int64_t site, int64_t* nn1, int64_t* nn2) {
  Job* J = static_cast<Job*>(h);
  if (site < 0 || site >= J->ns) return -1;
  int64_t X, y, z;
  J->coords(site, X, y, z);
  const int p = static_cast<int>(X & 1);
  for (int b = 0; b < 8; ++b) nn1[b] = J->site(X + kNN1[p][b].dx, y + kNN1[p][b].dy, z + kNN1[p][b].dz);
  for (int b = 0; b < 6; ++b) nn2[b] = J->site(X + kNN2[b].dx, y + kNN2[b].dy, z + kNN2[b].dz);
  return 0;
}

double ao_exp(double x) { return port_exp(x); }
double ao_log(double x) { return port_log(x); }
int ao_xoshiro_stream(uint64_t seed, uint64_t tag, uint64_t index, uint64_t* out, int64_t n) {
  Xoshiro x = make_stream(seed, tag, index);
  for (int64_t i = 0; i < n; ++i) out[i] = x.next();
  return 0;
}
int ao_mt19937_draws(uint64_t seed, int use_default_seed, int canonical, double* out, int64_t n) {
  std::mt19937 m = use_default_seed ? std::mt19937() : std::mt19937(static_cast<std::mt19937::result_type>(seed));
  std::uniform_real_distribution<double> dis(0, 1);
  for (int64_t i = 0; i < n; ++i) out[i] = canonical ? dis(m) : static_cast<double>(m()) * (1.0 / 4294967295.0);
  return 0;
}

}  // extern "C"
