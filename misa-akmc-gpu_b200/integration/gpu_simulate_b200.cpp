// gpu_simulate_b200.cpp -- the reference's GPU backend interface (gpu/gpu_simulate.h:31-66)
// implemented on the B200 engine's C ABI (include/akmc.h).
//
// A maintainer of MISA-AKMC links this file and libakmc_b200.so in place of gpu/gpu_simulate.hip.
// ABVIModel (models/abvi/kmc.cpp:118-211) and SubLattice::startTimeLoop
// (src/algorithms/sl/sublattice.inl:61-179) stay as they are and keep calling the free functions
// below.  The shim serves one rank that holds the whole periodic box, so the MPI ghost and
// surface bookkeeping of the HIP backend (add_ghost, add_surface) has nothing to record.
//
// Occupancy lives in the LatticesList hash sets (vac_hash, cu_hash, ni_hash, mn_hash;
// src/lattice/lattices_list.h:329-333), Fe being "in none": creation::createAtomsRandom never
// fills LatticesList::_lattices (src/creation.cpp:36).  So gpu_prepare reads every site's type
// through the hash sets, as getType does in the HIP backend (gpu/gpu_simulate.hip:2042-2060), and
// every hop the device performs is applied back to the hash sets, as exchange_lattices does
// (gpu/gpu_simulate.hip:2062-2091).  Event hooks and the lattice dump then read the live lattice.
//
// Errors: the reference exits on any device error (gpu/gpuError.hip:5-37); the shim keeps that
// policy at this boundary and prints the engine's message first.
#include "gpu_simulate.h"

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "akmc.h"

namespace {

akmc_ctx* g_ctx = nullptr;     // one context per process, like the HIP backend's globals
int32_t g_job = -1;
int32_t g_device = 0;
LatticesList* g_list = nullptr;  // the caller's lattice: the source of truth on the host
int64_t g_nx = 0, g_ny = 0, g_nz = 0;  // box cells
int64_t g_gx = 0, g_gy = 0, g_gz = 0;  // ghost offsets of the local coordinates (x doubled)
constexpr int kRing[8] = {0, 7, 2, 5, 3, 4, 1, 6};  // sector order (src/algorithms/sl/sublattice.h:21-30)

void check(akmc_status s, const char* where) {
  if (s == AKMC_OK) return;
  char msg[256] = {0};
  if (g_ctx) akmc_last_error(g_ctx, msg, sizeof msg);
  std::fprintf(stderr, "%s: %s (%s)\n", where, akmc_status_string(s), msg);
  std::exit(EXIT_FAILURE);
}

// Engine site id (x doubled, no ghost layers) <-> the reference's local lattice id.
_type_lattice_id ref_id(int64_t site) {
  const int64_t X = site % (2 * g_nx), t = site / (2 * g_nx);
  return g_list->meta.getLId(X + g_gx, t % g_ny + g_gy, t / g_ny + g_gz);
}

LatticeTypes::lat_type type_of_code(int32_t code) {
  switch (code) {
    case AKMC_V: return LatticeTypes::V;
    case AKMC_CU: return LatticeTypes::Cu;
    case AKMC_NI: return LatticeTypes::Ni;
    case AKMC_MN: return LatticeTypes::Mn;
    default: return LatticeTypes::Fe;
  }
}

}  // namespace

// initialize_gpu (gpu/gpu_simulate.h:47): device process_rank % device count.
void initialize_gpu(int process_rank) { check(akmc_initialize_gpu(process_rank, &g_device), "initialize_gpu"); }

// gpu_prepare (gpu/gpu_simulate.h:51): the box's occupancy, read through the hash sets, becomes
// one single-domain pair-bond job of the engine (the reference's energy model, FP64).
void gpu_prepare(const double v, const double T, LatticesList* p_list, comm::ColoredDomain* /*p_domain*/) {
  g_list = p_list;
  const LatListMeta& m = p_list->meta;  // box_x and ghost_x are doubled
  g_nx = m.box_x / 2;
  g_ny = m.box_y;
  g_nz = m.box_z;
  g_gx = m.ghost_x;
  g_gy = m.ghost_y;
  g_gz = m.ghost_z;
  std::vector<uint8_t> occ(static_cast<size_t>(2 * g_nx * g_ny * g_nz));
  for (size_t s = 0; s < occ.size(); ++s) occ[s] = static_cast<uint8_t>(getType(ref_id(static_cast<int64_t>(s))));
  if (g_ctx) check(akmc_destroy(g_ctx), "akmc_destroy");
  g_ctx = nullptr;
  akmc_context_config cc = {};
  cc.device = g_device;
  check(akmc_create(&cc, &g_ctx), "akmc_create");
  akmc_job_config jc = {};
  jc.box[0] = g_nx;
  jc.box[1] = g_ny;
  jc.box[2] = g_nz;
  jc.blocks[0] = jc.blocks[1] = jc.blocks[2] = 1;  // one domain: the host drives every hop
  jc.energy_model = AKMC_MODEL_PAIRBOND;           // models/abvi/rate/bonds/pair_bond.hpp
  jc.precision = AKMC_FP64;
  jc.rng = AKMC_RNG_XOSHIRO;                       // unused by the per-hop calls: u comes from the caller
  jc.lattice_const = 2.855;                        // the pair-bond model reads no distances
  jc.cutoff_radius = 5.6;
  jc.attempt_freq = v;
  jc.temperature = T;
  jc.sector_window = 3.0e-7;                       // src/simulation.h:73-74
  check(akmc_add_job(g_ctx, &jc, occ.data(), static_cast<int64_t>(occ.size()), &g_job), "akmc_add_job");
  check(akmc_prepare(g_ctx), "akmc_prepare");
}

// firstSectLocalToGpu (gpu/gpu_simulate.h:31): the device bins the sector's vacancies itself.
// The reference's callee frees its caller's array (gpu/gpu_simulate.hip:1207); so does this one.
void firstSectLocalToGpu(_type_lattice_id* vac_ids, _type_lattice_count /*n*/) { std::free(vac_ids); }

// calculate_GPU (gpu/gpu_simulate.h:35): the ordered total rate of sector loop index `sect`.
double calculate_GPU(const comm::Region<comm::_type_lattice_size> /*region*/, int sect) {
  double total = 0.0;
  check(akmc_calculate(g_ctx, g_job, kRing[sect & 7], &total), "calculate_GPU");
  return total;
}

// first_calculate_GPU (gpu/gpu_simulate.h:33): the first calculation of a sector.  The id arrays
// (vacancies left in the sector, and the next sector's early part) are freed, as the reference's
// callee frees them (gpu/gpu_simulate.hip:1379-1380).
double first_calculate_GPU(_type_lattice_id* aft, _type_lattice_count /*n_aft*/, _type_lattice_id* adv,
                           _type_lattice_count /*n_adv*/, int sect) {
  std::free(aft);
  std::free(adv);
  return calculate_GPU(comm::Region<comm::_type_lattice_size>{}, sect);
}

// selectAndPerformEventGPU (gpu/gpu_simulate.h:37-41): selects the first jump whose running
// total exceeds u * total in z-y-x vacancy order, performs it on the device lattice and applies
// it to the host hash sets.
void selectAndPerformEventGPU(double u, int /*rank*/, _type_lattice_count /*step*/, int /*sect*/,
                              std::array<std::vector<ChangeLattice>, 7>& /*exchange_ghost*/,
                              const unsigned int sector_id,
                              std::array<std::unordered_set<_type_lattice_id>, 8>& /*surface_x*/,
                              std::array<std::unordered_set<_type_lattice_id>, 8>& /*surface_y*/,
                              std::array<std::unordered_set<_type_lattice_id>, 8>& /*surface_z*/) {
  akmc_event ev;
  check(akmc_select_and_perform(g_ctx, g_job, static_cast<int32_t>(sector_id), u, &ev), "selectAndPerformEventGPU");
  if (ev.from_site < 0) return;  // u * total reached no jump
  dev_event h;
  h.from_id = ref_id(ev.from_site);
  h.to_id = ref_id(ev.to_site);
  h.to_type = LatticeTypes(type_of_code(ev.species));
  exchange_lattices(h);
}

// calculateNextAdvRegion / sector_final (gpu/gpu_simulate.h:43-45): the HIP backend rotates its
// per-vacancy caches here; the engine keeps no host or device caches between calls.
void calculateNextAdvRegion(int /*sect*/) {}
void sector_final(int /*sect*/) {}

// gpu_final (gpu/gpu_simulate.h:49): reports any deferred device error and frees the context.
// The host hash sets already hold every hop.
void gpu_final() {
  if (!g_ctx) return;
  check(akmc_gpu_final(g_ctx), "gpu_final");
  check(akmc_destroy(g_ctx), "akmc_destroy");
  g_ctx = nullptr;
  g_job = -1;
}

// getType (gpu/gpu_simulate.h:53): a site's type from the hash sets; Fe is in none of them.
LatticeTypes::lat_type getType(_type_lattice_id id) {
  if (g_list->vac_hash.count(id)) return LatticeTypes::V;
  if (g_list->cu_hash.count(id)) return LatticeTypes::Cu;
  if (g_list->mn_hash.count(id)) return LatticeTypes::Mn;
  if (g_list->ni_hash.count(id)) return LatticeTypes::Ni;
  return LatticeTypes::Fe;
}

// exchange_lattices (gpu/gpu_simulate.h:55): a performed hop on the hash sets.  The vacancy moves
// from from_id to to_id; the atom of type to_type moves the other way (Fe is in no set).
void exchange_lattices(dev_event e) {
  auto it = g_list->vac_hash.find(e.from_id);
  if (it == g_list->vac_hash.end()) {
    std::fprintf(stderr, "exchange_lattices: no vacancy at site %lld\n", static_cast<long long>(e.from_id));
    std::exit(EXIT_FAILURE);
  }
  g_list->vac_hash.erase(it);
  g_list->vac_hash.emplace(e.to_id, VacancyHash{});
  std::unordered_set<_type_lattice_id>* set = nullptr;
  switch (e.to_type._type) {
    case LatticeTypes::Cu: set = &g_list->cu_hash; break;
    case LatticeTypes::Ni: set = &g_list->ni_hash; break;
    case LatticeTypes::Mn: set = &g_list->mn_hash; break;
    default: break;
  }
  if (set) {
    set->erase(e.to_id);
    set->insert(e.from_id);
  }
}

// add_ghost / add_surface / initInfo (gpu/gpu_simulate.h:57-66): helpers of the HIP backend for
// the MPI ghost exchange and its per-vacancy neighbour caches.  One rank holding the whole
// periodic box exchanges nothing, and the engine builds no host caches.
void add_ghost(std::array<std::vector<ChangeLattice>, 7>& /*exchange_ghost*/, _type_lattice_id /*x*/,
               _type_lattice_id /*y*/, _type_lattice_id /*z*/, Lattice /*lat_to*/, const unsigned int /*sector_id*/) {}
void initInfo(_type_lattice_count /*vac_total*/, _type_lattice_id* /*vac_ids*/, dev_Vacancy* /*h_vacancy*/,
              dev_nnLattice* /*h_nn*/) {}
void add_surface(_type_lattice_id /*surface_id*/, std::array<std::unordered_set<_type_lattice_id>, 8>& /*x*/,
                 std::array<std::unordered_set<_type_lattice_id>, 8>& /*y*/,
                 std::array<std::unordered_set<_type_lattice_id>, 8>& /*z*/) {}
