// shim_driver.cpp -- test harness around misa-akmc-gpu_b200/integration/gpu_simulate_b200.cpp.
//
// It stands where the reference's ABVIModel and SubLattice stand: it owns a PeriodLatticeList
// (the reference's own class, src/lattice/period_lattice_list.h), fills its occupancy hash sets
// (src/lattice/lattices_list.h:329-333) from a lattice in the engine's site layout, and calls the
// free functions of gpu/gpu_simulate.h as ABVIModel::calcRatesGPU and selectAndPerformOnGPU do
// (models/abvi/kmc.cpp:118-211).  The lattice is read back through the hash sets only.
#include <cstdint>
#include <cstdlib>

#include "gpu_simulate.h"
#include "lattice/period_lattice_list.h"

namespace {
PeriodLatticeList* g_lat = nullptr;
int64_t g_n[3] = {0, 0, 0};
std::array<std::vector<ChangeLattice>, 7> g_ghost;
std::array<std::unordered_set<_type_lattice_id>, 8> g_sx, g_sy, g_sz;

_type_lattice_id lid_of(int64_t s) {
  const int64_t X = s % (2 * g_n[0]), t = s / (2 * g_n[0]);
  return g_lat->meta.getLId(X + g_lat->meta.ghost_x, t % g_n[1] + g_lat->meta.ghost_y, t / g_n[1] + g_lat->meta.ghost_z);
}
}  // namespace

extern "C" {

// A periodic box of nx*ny*nz cells with `ghost` ghost cells per side, its hash sets filled from
// occ (engine codes V 0, Fe 1, Cu 2, Ni 4, Mn 8), then initialize_gpu and gpu_prepare.
int shim_prepare(const uint8_t* occ, int64_t nx, int64_t ny, int64_t nz, int64_t ghost, double nu, double T) {
  delete g_lat;
  g_lat = new PeriodLatticeList(LatListMeta(nx, ny, nz, ghost, ghost, ghost));
  g_n[0] = nx;
  g_n[1] = ny;
  g_n[2] = nz;
  for (int64_t s = 0; s < 2 * nx * ny * nz; ++s) {
    const _type_lattice_id id = lid_of(s);
    switch (occ[s]) {
      case 0: g_lat->vac_hash.emplace(id, VacancyHash{}); break;
      case 2: g_lat->cu_hash.insert(id); break;
      case 4: g_lat->ni_hash.insert(id); break;
      case 8: g_lat->mn_hash.insert(id); break;
      case 1: break;
      default: return -1;
    }
  }
  initialize_gpu(0);
  gpu_prepare(nu, T, g_lat, nullptr);
  return 0;
}

// The first calculation of a sector goes through first_calculate_GPU with malloc'd id arrays
// (freed by the callee, as in the reference), later ones through calculate_GPU.
double shim_calculate(int sect, int first) {
  if (first) {
    auto* a = static_cast<_type_lattice_id*>(std::malloc(sizeof(_type_lattice_id)));
    auto* b = static_cast<_type_lattice_id*>(std::malloc(sizeof(_type_lattice_id)));
    return first_calculate_GPU(a, 0, b, 0, sect);
  }
  return calculate_GPU(comm::Region<comm::_type_lattice_size>{}, sect);
}

void shim_select(double u, int sect, unsigned int sector_id) {
  selectAndPerformEventGPU(u, 0, 0, sect, g_ghost, sector_id, g_sx, g_sy, g_sz);
}

void shim_sector_final(int sect) { sector_final(sect); }

// The lattice as the hash sets hold it; returns the number of sites found in more than one set.
int64_t shim_occupancy(uint8_t* out) {
  int64_t multi = 0;
  for (int64_t s = 0; s < 2 * g_n[0] * g_n[1] * g_n[2]; ++s) {
    const _type_lattice_id id = lid_of(s);
    const int in = static_cast<int>(g_lat->vac_hash.count(id) + g_lat->cu_hash.count(id) + g_lat->ni_hash.count(id) +
                                    g_lat->mn_hash.count(id));
    multi += in > 1;
    out[s] = static_cast<uint8_t>(getType(id));
  }
  return multi;
}

void shim_final() {
  gpu_final();
  delete g_lat;
  g_lat = nullptr;
}

}  // extern "C"
