// akmc_device.h -- device-side state of the vacancy-hop engine (internal).
#pragma once

#include <stdint.h>
#include <vector_types.h>

#include "../../include/akmc.h"
#include "akmc_common.cuh"

namespace akmc {

constexpr int kMaxV = AKMC_MAX_SECTOR_VACANCIES;  // vacancies per block and sector
constexpr int kNoAllocMaxBlocks = AKMC_NOALLOC_MAX_BLOCKS;
constexpr int kJumpN = 76;                        // |N(s) u N(t)| - 2 sites per jump
constexpr int kRefreshN = 78;                     // density refresh sites per jump
constexpr int kShellNb = 58;                      // neighbours within the 5-shell cutoff
constexpr int kNbrStride = 32;  // words per block of RoundArgs::nbr (one 128-byte line)
constexpr int kFlowSlots = 64;                    // vacancies held in one domain block's area

// Packed neighbour entry: int8 dX | int8 dy << 8 | int8 dz << 16 | (sh_s | sh_t << 4) << 24,
// dX in doubled-x site units; shell codes 0 = outside the cutoff, 1..5 shells, 6 = the site itself.
AK_HD int unpack_dx(int32_t w) { return static_cast<int8_t>(w & 0xff); }
AK_HD int unpack_dy(int32_t w) { return static_cast<int8_t>((w >> 8) & 0xff); }
AK_HD int unpack_dz(int32_t w) { return static_cast<int8_t>((w >> 16) & 0xff); }
AK_HD int unpack_sh_s(int32_t w) { return (w >> 24) & 0xf; }
AK_HD int unpack_sh_t(int32_t w) { return (w >> 28) & 0xf; }
AK_HD int32_t pack_entry(int dx, int dy, int dz, int sh_s, int sh_t) {
  return static_cast<int32_t>((static_cast<uint32_t>(dx) & 0xffu) | ((static_cast<uint32_t>(dy) & 0xffu) << 8) |
                              ((static_cast<uint32_t>(dz) & 0xffu) << 16) |
                              ((static_cast<uint32_t>(sh_s) | (static_cast<uint32_t>(sh_t) << 4)) << 24));
}

// Geometry tables (built on the host, one copy in global memory).
struct Geometry {
  int32_t nn1[2][8];                 // 1nn, LatListMeta::getIdBy1nnOffset order by x parity
  int32_t nn2[6];                    // 2nn, PeriodLatticeList::get2nn2 order (mask 0x2F)
  int32_t nbr[2][kShellNb];          // EAM shell neighbours (sh in sh_s)
  int32_t jump[2][8][kJumpN];        // EAM dE site list of jump b, order (dz, dy, dX)
  int32_t refresh[2][8][kRefreshN];  // density refresh list of jump b (incl. s and t)
};

// Per-potential tables.
struct Potential {
  int32_t fq[4][8];         // density contribution (Q.24) by species and shell code
  double phi64[4][4][8];    // pair energy by (moving species, neighbour species, shell code)
  float phi32[4][4][8];
  double b1[5][5], b2[5][5];  // pair-bond 1nn / 2nn tables (V, Fe, Cu, Ni, Mn)
  // F(rho) cells in two planes, so that a cell's two 16-byte halves fall into
  // different shared-memory bank groups for random cells
  const double2* F64lo;     // (c0, c1) per cell
  const double2* F64hi;     // (c2, c3) per cell
  const float4* F32a;       // (hi, lo, c1, c2) per cell
  const float* F32b;        // c3 per cell
  int32_t fwin0;            // first F-table cell of the shared-memory window
  int32_t pad;
};

// F-table cells kept in shared memory: rho in [bulk Fe - 6, bulk Fe + 2]; cells
// outside the window are read from global memory (same values, slower).
constexpr int kFWin = 1024;

// Device lattice layout.  Each x row of a job (sx sites) is stored with a periodic halo:
// kHaloL sites on its left hold copies of the row's last sites, kHaloR on its right copies of its
// first ones, in a row of lattice_pitch(sx) entries (a multiple of 16).  Site (x, y, z) sits at
// kHaloL + x + pitch (y + sy z), and every write of a site writes its halo copies too
// (lattice_put), so a span of a row from x = -kHaloL to x = sx + kHaloR is contiguous: a sector
// region's row, rounded out to 16-site boundaries, is one aligned bulk copy whatever the box.
// Position p of a row (0 <= p < kHaloL + sx + kHaloR) holds site (p - kHaloL) mod sx; the rest
// of the pitch is padding.
constexpr int kHaloL = 16, kHaloR = 32;
AK_HD int32_t lattice_pitch(int32_t sx) { return (kHaloL + sx + kHaloR + 15) & ~15; }
AK_HD int64_t lattice_entries(int32_t sx, int32_t sy, int32_t sz) {
  return static_cast<int64_t>(lattice_pitch(sx)) * sy * sz;
}
// Entry of site id s = x + sx (y + sy z).
AK_HD int64_t lattice_index(int32_t s, int32_t sx, int32_t px) {
  return kHaloL + s % sx + static_cast<int64_t>(px) * (s / sx);
}
// Writes site x of a row (row = the row's first entry) and its halo copies: only sites within
// kHaloR of the row's start or kHaloL of its end have one (rows shorter than the halo, several).
template <typename T>
AK_HD void lattice_put(T* row, int32_t sx, int32_t x, T v) {
  row[kHaloL + x] = v;
  if (x < kHaloR || x >= sx - kHaloL) {
    for (int p = kHaloL + x - sx; p >= 0; p -= sx) row[p] = v;
    for (int p = kHaloL + x + sx; p < kHaloL + sx + kHaloR; p += sx) row[p] = v;
  }
}

struct JobDev {
  uint8_t* occ;       // lattice_entries(sx, sy, sz) occupancy codes, halo layout
  int32_t* rho;       // the same layout, densities
  int32_t n[3];       // cells
  int32_t sx, sy, sz; // sites per dimension (sx = 2 n[0])
  int32_t px;         // row pitch of the device lattice (lattice_pitch(sx))
  int32_t tma;        // 1: every region has the box tbox as its shared-memory pitch, and a region
                      // that does not wrap in y or z is staged by one tensor copy per array through
                      // the job's tensor maps (RoundArgs::tmaps)
  int32_t tbox[3];    // the box: the job's widest region, x rounded out as the bulk form rounds it
  int32_t pad_tbox;
  int32_t nb[3];      // domain blocks per dimension
  int32_t block0;     // first global block
  int32_t nblocks;
  int32_t model, precision, pot;
  int32_t done;
  int32_t bulk;       // 1: regions that do not wrap in x are staged by bulk copies of whole rows
  int64_t round;
  int64_t hops;
  int64_t hop_budget, max_rounds;
  double nu, kT, window;
};

struct BlockDev {
  int32_t job, local_id;
  int32_t c0[3], c1[3];  // block cells [c0, c1)
  int64_t round;
  int64_t hops;
  double evo[8];         // per-sector evolution time
  uint64_t xs[4], xt[4]; // selection / residence-time streams
  int32_t cnt;           // vacancies bucketed into the active sector this round
  int32_t done;          // the job finished at or before this block's last round
  int64_t target;        // asynchronous schedule: round this launch runs the block up to
  int64_t remaining;     // asynchronous schedule: rounds of the akmc_run_rounds call still to run
  int64_t hops_at[2];    // asynchronous schedule: hops when the block reached time-step boundary b,
                         // in slot (b / 8) & 1 (a multi-block job's hop budget is checked there)
  int32_t budget_end;    // asynchronous schedule: the hop budget set the block's target (the job
                         // ends when the block reaches it)
  int32_t pad2;
};

enum : uint32_t {
  kErrVacOverflow = 1u,
  kErrRhoRange = 2u,
  kErrHopCap = 4u,
  kErrLogOverflow = 8u,
  kErrApiState = 16u,
  kErrTimeout = 32u,
  kErrVacCount = 64u,  // a loaded lattice does not hold its job's vacancy count
};

enum : int32_t { kModeRound = 0, kModeCalc = 1, kModeSelectPerform = 2 };

struct RoundArgs {
  JobDev* jobs;
  int32_t njobs;
  int32_t nblocks;
  BlockDev* blocks;
  int32_t* vac_site;
  int32_t* vac_job;
  int32_t nvac;
  int32_t mode;
  int32_t kind_mask;  // energy kinds present: bit 0 pair-bond, 1 EAM FP64, 2 EAM FP32-comp
  int32_t* blk_list;  // nblocks * kMaxV
  int32_t* active;    // nblocks
  int32_t* n_active;
  const Potential* pots;
  const Geometry* geo;
  akmc_event* log;
  unsigned long long* log_count;
  int64_t log_cap;
  unsigned int* status;
  unsigned long long* counters;  // hops, evaluations, rounds, blocks, n_act sum, staged sites, written sites, -
  int64_t hop_cap;
  // asynchronous round schedule (k_flow)
  unsigned long long* fstate;   // per block: rounds completed << 1, | 1 while a thread or CTA holds it
  unsigned long long* vclaim;   // per block: slots of vslot taken
  unsigned long long* vvalid;   // per block: slots of vslot holding a vacancy id
  int32_t* vslot;               // per block: kFlowSlots ids of the vacancies in its area
  int32_t* vsite;               // per block: their sites (kept with the ids by whoever moves them)
  int32_t* vcount;              // per block: fill counter while the slots are rebuilt
  unsigned int* vsec;           // per block: bit s set while a vacancy of its area lies in sector s
  const void* tmaps;            // per job slot: two 128-byte tensor maps (occupancy, densities)
  int32_t* nbr;                 // per block, kNbrStride words: the 27 neighbour blocks (offset
                                // o = (dz+1)*9 + (dy+1)*3 + dx+1) and a flags word (k_flow_prep)
  int32_t* flow_need;           // per energy kind: blocks with rounds to run in this launch
  int32_t* flow_done;           // per energy kind: blocks that reached their target
  int64_t flow_rounds;          // rounds this launch adds to every unfinished block
  int64_t flow_sweep_limit;     // sweeps per CTA before the launch gives up (kErrTimeout)
  int64_t time_budget_ns;       // > 0: the launch takes no new round after this long (akmc_run_for)
  int32_t flow_take;            // rounds with vacancies a CTA takes per sweep (0: all it found)
  int32_t eval_warps;           // CTA shape of the hop kernels: 8 or 4 evaluator warps
  // per-hop entry points
  int32_t api_job, api_sector;
  double api_u;
  double* api_total;
  akmc_event* api_event;
  double* api_de;         // kMaxV * 8: ΔE of each jump of the last akmc_calculate
  double* api_rates;      // kMaxV * 8: its rates
  int32_t* api_sites;     // kMaxV: vacancy sites (-1: left the sector)
  int32_t* api_count;
};

// Kernel launchers (akmc_kernels.cu).
size_t hop_smem_bytes(int max_region_sites);
int configure_hop_smem(size_t smem);
int hop_ctas_per_sm(int eval_warps);  // CTAs of the hop kernels the register budget allows per SM
// ev0/ev1 (cudaEvent_t or null) are recorded around the hop kernel.
int launch_round(const RoundArgs& a, int hop_grid, size_t smem, void* stream, void* ev0, void* ev1);
// Collects the vacancies of one job's lattice into its slice of the vacancy table and sets
// kErrVacCount in *status unless exactly cap were found.
int launch_collect_vacancies(const uint8_t* occ, int64_t n, int32_t sx, int32_t* vac_site, int32_t* vac_job,
                             int32_t job, int32_t cap, int32_t* count, unsigned int* status, void* stream);
// Refreshes the halo entries of every row of a lattice (halo layout, rows of sx sites).
int launch_fill_halo(uint8_t* lat, int32_t sx, int64_t nrows, void* stream);
int launch_fill_halo(int32_t* lat, int32_t sx, int64_t nrows, void* stream);
int launch_api(const RoundArgs& a, size_t smem, void* stream);
int launch_init_rho(uint8_t* occ, int32_t* rho, int32_t sx, int32_t sy, int32_t sz, const Potential* pot,
                    const Geometry* geo, unsigned int* status, void* stream);
int launch_device_math(const double* x, int64_t n, double* e, double* l, void* stream);
// n rounds of every unfinished block under the asynchronous schedule (no job may have a
// hop budget); grid = persistent CTAs of the flow kernels.
int launch_flow(const RoundArgs& a, int grid, size_t smem, void* stream, void* ev0, void* ev1);
// Sets every block's remaining rounds to n before the launches of one akmc_run_rounds call.
int launch_flow_begin(const RoundArgs& a, int64_t n, void* stream);

// Whole-context lattice transfers (akmc_load_occupancies / akmc_get_occupancies): the lattices
// of all jobs back to back in a staging buffer, cut into chunks of one job each.
struct SiteChunk {
  int32_t job, vac0, nvac, pad;
  int64_t site0, n, stage0;  // first site in the job, sites, offset in the staging buffer
};
struct JobsLoad {
  const uint8_t* stage_in;  // unused by the kernels (host side)
  uint8_t* stage;
  const SiteChunk* chunks;
  int32_t nchunks, njobs;
  int32_t* counts;          // vacancies found per job
  const int32_t* want;      // vacancies each job holds
  const int64_t* tile0;     // density tiles of the EAM jobs, prefix (neam + 1)
  const int32_t* eam_jobs;  // job index of each EAM job
  int32_t neam;
  int64_t eam_tiles;
};
int launch_load_jobs(const RoundArgs& a, const JobsLoad& L, void* stream);
int launch_init_rho_jobs(const RoundArgs& a, const JobsLoad& L, void* stream);  // uses a.jobs, a.pots
int launch_gather_jobs(const RoundArgs& a, const JobsLoad& L, void* stream);

// Cu cluster statistics of one job's occupancy (akmc_cluster.cu).  list, parent and size hold
// one int32 per site; iso and hist are cleared by the launch.
struct ClusterArgs {
  const uint8_t* occ;  // halo layout
  int64_t ns;
  int32_t sx, sy, sz, bins;
  int32_t px, pad;
  int32_t* list;
  unsigned int* n_list;
  int32_t* parent;
  int32_t* size;
  unsigned long long* iso;
  unsigned long long* hist;
  unsigned int* status;
};
int launch_cluster_stats(const ClusterArgs& c, void* stream);
// Device address of the fixed round scratch (current device): kNoAllocMaxBlocks * kMaxV
// block-list slots, then kNoAllocMaxBlocks active-list slots, then the active count.
int noalloc_scratch(int32_t** base);

}  // namespace akmc
