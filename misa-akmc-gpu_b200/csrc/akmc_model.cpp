// akmc_model.cpp -- host-side model construction: neighbour geometry, the
// synthetic Johnson EAM, pair-bond tables, lattice creation, cluster statistics.
#include "akmc_model.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace akmc {

namespace {

// 1nn offsets (dX, dy, dz) by x parity in LatListMeta::getIdBy1nnOffset order
// (src/lattice/lattice_list_meta.cpp:22-70).
const int kNN1[2][8][3] = {
    {{-1, -1, -1}, {-1, -1, 0}, {-1, 0, -1}, {-1, 0, 0}, {1, -1, -1}, {1, -1, 0}, {1, 0, -1}, {1, 0, 0}},
    {{-1, 0, 0}, {-1, 0, 1}, {-1, 1, 0}, {-1, 1, 1}, {1, 0, 0}, {1, 0, 1}, {1, 1, 0}, {1, 1, 1}}};
// 2nn offsets in PeriodLatticeList::get2nn2 order (src/lattice/period_lattice_list.cpp:234-256).
const int kNN2[6][3] = {{-2, 0, 0}, {0, -1, 0}, {0, 0, -1}, {0, 0, 1}, {0, 1, 0}, {2, 0, 0}};
// BCC shells within 2a: squared distance in (a/2)^2 units.
const int kShellD2[5] = {3, 4, 8, 11, 12};
constexpr int kSelf = 6;

// squared distance between site (X0, 0, 0) and (X0 + dX, dy, dz) in (a/2)^2 units;
// corner sites (X even) sit at (X, 2y, 2z), centre sites at (X, 2y + 1, 2z + 1).
int dist2(int X0, int dX, int dy, int dz) {
  const int p0 = X0 & 1, p1 = (X0 + dX) & 1;
  const int hy = 2 * dy + p1 - p0, hz = 2 * dz + p1 - p0;
  return dX * dX + hy * hy + hz * hz;
}
int shell_code(int d2, int nsh) {
  for (int i = 0; i < nsh; ++i)
    if (kShellD2[i] == d2) return i + 1;
  return 0;
}

}  // namespace

int shells_within(double lattice_const, double cutoff) {
  int n = 0;
  for (int i = 0; i < 5; ++i)
    if (lattice_const * std::sqrt(static_cast<double>(kShellD2[i])) / 2.0 < cutoff) n = i + 1;
  return n;
}

void build_geometry(Geometry& g, int nsh) {
  std::memset(&g, 0, sizeof(g));
  for (int p = 0; p < 2; ++p)
    for (int b = 0; b < 8; ++b) g.nn1[p][b] = pack_entry(kNN1[p][b][0], kNN1[p][b][1], kNN1[p][b][2], 0, 0);
  for (int b = 0; b < 6; ++b) g.nn2[b] = pack_entry(kNN2[b][0], kNN2[b][1], kNN2[b][2], 0, 0);
  for (int p = 0; p < 2; ++p) {
    int n = 0;
    for (int dz = -3; dz <= 3; ++dz)
      for (int dy = -3; dy <= 3; ++dy)
        for (int dx = -5; dx <= 5; ++dx) {
          if (!dx && !dy && !dz) continue;
          const int sh = shell_code(dist2(p, dx, dy, dz), nsh);
          if (sh && n < kShellNb) g.nbr[p][n++] = pack_entry(dx, dy, dz, sh, 0);
        }
    for (int b = 0; b < 8; ++b) {
      const int tx = kNN1[p][b][0], ty = kNN1[p][b][1], tz = kNN1[p][b][2];
      int nl = 0, nr = 0;
      // dE site list: (N(s) u N(t)) minus s and t, ordered by (dz, dy, dX) relative to s;
      // every site of the union lies in different shells of s and t.
      for (int dz = -4; dz <= 4; ++dz)
        for (int dy = -4; dy <= 4; ++dy)
          for (int dx = -6; dx <= 6; ++dx) {
            const bool is_s = !dx && !dy && !dz;
            const bool is_t = dx == tx && dy == ty && dz == tz;
            const int ss = is_s ? kSelf : shell_code(dist2(p, dx, dy, dz), nsh);
            const int st = is_t ? kSelf : shell_code(dist2(p + tx, dx - tx, dy - ty, dz - tz), nsh);
            if ((ss == 0 && st == 0) || ss == st) continue;
            if (nr < kRefreshN) g.refresh[p][b][nr++] = pack_entry(dx, dy, dz, ss, st);
            if (!is_s && !is_t && nl < kJumpN) g.jump[p][b][nl++] = pack_entry(dx, dy, dz, ss, st);
          }
    }
  }
}

void pairbond_tables(double b1[5][5], double b2[5][5]) {
  // Vincent, Becquart & Domain, J. Nucl. Mater. 351 (2006) 88, table 7, as used by
  // models/abvi/rate/bonds/bonds_counter.cpp:13-33.  Index order V, Fe, Cu, Ni, Mn.
  struct E { int i, j; double v1, v2; };
  const E t[] = {{1, 1, -0.778, -0.389}, {0, 0, 0.315, -0.214}, {2, 2, -0.581, -0.389}, {3, 3, -0.793, -0.389},
                 {4, 4, -0.438, -0.389}, {0, 1, -0.161, -0.161}, {1, 2, -0.609, -0.344}, {1, 3, -0.821, -0.399},
                 {1, 4, -0.648, -0.364}, {0, 2, -0.103, -0.206}, {0, 3, -0.234, -0.351}, {0, 4, -0.151, -0.206},
                 {2, 3, -0.692, -0.344}, {2, 4, -0.519, -0.249}, {3, 4, -0.831, -0.464}};
  for (const E& e : t) {
    b1[e.i][e.j] = b1[e.j][e.i] = e.v1;
    b2[e.i][e.j] = b2[e.j][e.i] = e.v2;
  }
}

// Cubic (Catmull-Rom) coefficients of cell k of a uniformly tabulated function.
void cell_coefs(const double* F, int n, int k, double c[4]) {
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

static double table_value(const std::vector<double>& T, double step, double x) {
  const int n = static_cast<int>(T.size());
  int k = static_cast<int>(std::floor(x / step));
  if (k > n - 2) k = n - 2;
  const double p = x / step - static_cast<double>(k);
  double c[4];
  cell_coefs(T.data(), n, k, c);
  return std::fma(std::fma(std::fma(c[3], p, c[2]), p, c[1]), p, c[0]);
}

int eam_johnson(uint64_t seed, double a, double rc, akmc_eam_tables* out, double params[4][5]) {
  const int nsh = shells_within(a, rc);
  if (nsh < 1 || 2.0 * a < rc) return -1;
  std::memset(out, 0, sizeof(*out));
  out->n_shells = nsh;
  // Fe-like base values of A (eV), B (eV), alpha, beta, re (Angstrom); each species
  // draws base * (1 + 0.1 (2u - 1)) from the xoshiro stream (seed, tag 5).
  const double base[5] = {0.80, 0.45, 8.0, 4.5, 2.4725};
  uint64_t st[4];
  xoshiro_seed(st, seed, kTagPotential, 0);
  double par[4][5];
  for (int s = 0; s < 4; ++s)
    for (int p = 0; p < 5; ++p) par[s][p] = base[p] * (1.0 + 0.1 * (2.0 * uniform_co(st) - 1.0));
  if (params) std::memcpy(params, par, sizeof(par));
  const double dr = rc / static_cast<double>(kTabN - 1);
  double rsh[5];
  for (int i = 0; i < 5; ++i) rsh[i] = a * std::sqrt(static_cast<double>(kShellD2[i])) / 2.0;
  double phi_pure[4][5];
  for (int s = 0; s < 4; ++s) {
    std::vector<double> f(kTabN), phi(kTabN);
    const double A = par[s][0], B = par[s][1], al = par[s][2], be = par[s][3], re = par[s][4];
    for (int k = 0; k < kTabN; ++k) {
      const double r = static_cast<double>(k) * dr;
      f[k] = 1.0 * std::exp(-be * (r / re - 1.0));
      phi[k] = A * std::exp(-al * (r / re - 1.0)) - B * std::exp(-be * (r / re - 1.0));
    }
    for (int i = 0; i < 5; ++i) {
      out->f_shell[s][i] = table_value(f, dr, rsh[i]);
      phi_pure[s][i] = table_value(phi, dr, rsh[i]);
    }
  }
  for (int X = 0; X < 4; ++X)
    for (int Y = 0; Y < 4; ++Y)
      for (int i = 0; i < 5; ++i) {
        if (X == Y) {
          out->phi_shell[X][Y][i] = phi_pure[X][i];
        } else {  // Johnson (1989) alloy rule
          const double fx = out->f_shell[X][i], fy = out->f_shell[Y][i];
          out->phi_shell[X][Y][i] = 0.5 * ((fy / fx) * phi_pure[X][i] + (fx / fy) * phi_pure[Y][i]);
        }
      }
  for (int k = 0; k < kTabN; ++k) out->F[k] = -std::sqrt(static_cast<double>(k) * 0x1p-7);
  return 0;
}

int build_potential(const akmc_eam_tables* t, Potential& P, std::vector<double>& coef, std::vector<FCell32>& f32) {
  std::memset(&P, 0, sizeof(P));
  pairbond_tables(P.b1, P.b2);
  coef.assign(static_cast<size_t>(kTabN) * 4, 0.0);
  f32.assign(kTabN, FCell32{});
  if (!t) return 0;
  const int nsh = t->n_shells;
  if (nsh < 1 || nsh > 5) return -1;
  for (int X = 0; X < 4; ++X) {
    for (int i = 0; i < 5; ++i) {
      const double f = i < nsh ? t->f_shell[X][i] : 0.0;
      if (!(f >= 0.0) || f > 64.0) return -1;
      P.fq[X][i + 1] = static_cast<int32_t>(std::llround(f * 0x1p24));
    }
    for (int Y = 0; Y < 4; ++Y)
      for (int i = 0; i < 5; ++i) {
        const double v = i < nsh ? t->phi_shell[X][Y][i] : 0.0;
        P.phi64[X][Y][i + 1] = v;
        P.phi32[X][Y][i + 1] = static_cast<float>(v);
      }
  }
  // every reachable density must stay inside the F table: at most all 58 neighbours
  // of the densest species
  const int counts[5] = {8, 6, 12, 24, 8};
  int64_t rmax = 0;
  for (int i = 0; i < nsh; ++i) {
    int32_t m = 0;
    for (int X = 0; X < 4; ++X) m = std::max(m, P.fq[X][i + 1]);
    rmax += static_cast<int64_t>(counts[i]) * m;
  }
  if ((rmax >> kRhoCellShift) > kTabN - 3) return -2;
  // shared-memory window of the F table around the density of bulk Fe
  int64_t rbulk = 0;
  for (int i = 0; i < nsh; ++i) rbulk += static_cast<int64_t>(counts[i]) * P.fq[0][i + 1];
  const int kb = static_cast<int>(rbulk >> kRhoCellShift);
  // window start a multiple of 4 cells: the bulk copies of its planes start 16-byte aligned
  P.fwin0 = std::max(0, std::min(kb - (3 * kFWin) / 4, kTabN - 2 - kFWin)) & ~3;
  for (int k = 0; k + 1 < kTabN; ++k) {
    double c[4];
    cell_coefs(t->F, kTabN, k, c);
    for (int j = 0; j < 4; ++j) coef[static_cast<size_t>(k) * 4 + j] = c[j];
    FCell32& e = f32[k];
    e.hi = static_cast<float>(c[0]);
    e.lo = static_cast<float>(c[0] - static_cast<double>(e.hi));
    e.c1 = static_cast<float>(c[1]);
    e.c2 = static_cast<float>(c[2]);
    e.c3 = static_cast<float>(c[3]);
  }
  return 0;
}

void block_split(int64_t n, int p, std::vector<int32_t>& start) {
  start.resize(static_cast<size_t>(p) + 1);
  for (int k = 0; k <= p; ++k)
    start[static_cast<size_t>(k)] = static_cast<int32_t>(k * (n / p) + std::min<int64_t>(k, n % p));
}

int create_lattice(const int64_t box[3], const int32_t codes[4], const int64_t ratio[4], int64_t nvac,
                   uint64_t seed, uint8_t* occ, int64_t n) {
  const int64_t ns = 2 * box[0] * box[1] * box[2];
  if (n != ns || nvac < 0 || nvac > ns) return -1;
  int64_t total = 0;
  for (int i = 0; i < 4; ++i) {
    if (ratio[i] < 0) return -1;
    if (ratio[i] > 0 && !is_atom(static_cast<uint8_t>(codes[i]))) return -1;
    total += ratio[i];
  }
  if (total <= 0) return -1;
  uint64_t st[4];
  xoshiro_seed(st, seed, kTagTypes, 0);
  for (int64_t s = 0; s < ns; ++s) {
    // hit in [1, total]; LatticeTypes::randomAtomsType (src/lattice/lattice_types.cpp:9-19)
    const int64_t hit =
        1 + static_cast<int64_t>((static_cast<unsigned __int128>(xoshiro_next(st)) * static_cast<uint64_t>(total)) >> 64);
    int64_t acc = 0;
    uint8_t t = kFe;
    for (int i = 0; i < 4; ++i) {
      acc += ratio[i];
      if (acc >= hit) {
        t = static_cast<uint8_t>(codes[i]);
        break;
      }
    }
    occ[s] = t;
  }
  xoshiro_seed(st, seed, kTagVacancy, 0);
  int64_t placed = 0;
  while (placed < nvac) {
    const int64_t s =
        static_cast<int64_t>((static_cast<unsigned __int128>(xoshiro_next(st)) * static_cast<uint64_t>(ns)) >> 64);
    if (occ[s] != kV) {
      occ[s] = kV;
      ++placed;
    }
  }
  return 0;
}

int cluster_stats(const uint8_t* occ, const int64_t box[3], int64_t* isolated, int64_t* hist, int64_t hist_len) {
  const int64_t sx = 2 * box[0], sy = box[1], sz = box[2], ns = sx * sy * sz;
  auto nb = [&](int64_t s, int b) {
    const int64_t X = s % sx, t = s / sx, y = t % sy, z = t / sy;
    const int p = static_cast<int>(X & 1);
    const int64_t gx = (X + kNN1[p][b][0] + sx) % sx, gy = (y + kNN1[p][b][1] + sy) % sy,
                  gz = (z + kNN1[p][b][2] + sz) % sz;
    return gx + sx * (gy + sy * gz);
  };
  for (int64_t i = 0; i < hist_len; ++i) hist[i] = 0;
  std::vector<uint8_t> seen(static_cast<size_t>(ns), 0);
  std::vector<int64_t> stack;
  int64_t iso = 0;
  for (int64_t s = 0; s < ns; ++s) {
    if (occ[s] != kCu) continue;
    bool has = false;
    for (int b = 0; b < 8 && !has; ++b) has = occ[nb(s, b)] == kCu;
    if (!has) ++iso;
    if (seen[static_cast<size_t>(s)]) continue;
    int64_t size = 0;
    stack.push_back(s);
    seen[static_cast<size_t>(s)] = 1;
    while (!stack.empty()) {
      const int64_t q = stack.back();
      stack.pop_back();
      ++size;
      for (int b = 0; b < 8; ++b) {
        const int64_t r = nb(q, b);
        if (occ[r] == kCu && !seen[static_cast<size_t>(r)]) {
          seen[static_cast<size_t>(r)] = 1;
          stack.push_back(r);
        }
      }
    }
    if (hist_len > 0) hist[size < hist_len ? size : hist_len - 1] += 1;
  }
  *isolated = iso;
  return 0;
}

}  // namespace akmc
