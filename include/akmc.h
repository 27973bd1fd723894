/*
 * akmc.h -- C ABI of libakmc_b200.so, the B200 (sm_100a) vacancy-hop engine.
 *
 * Drop-in boundary for the GPU backend of MISA-AKMC (panzhija/MISA-AKMC-GPU).
 * The reference's ABVIModel (models/abvi/kmc.cpp) drives its backend through
 * the free functions of gpu/gpu_simulate.h:31-66 on the types of
 * gpu/DeviceVacRatesSolver.h:7-25.  Each of those entry points has a
 * counterpart below (cited at the declaration); the fused entry points
 * (akmc_run_rounds, akmc_run) run the whole sector schedule of
 * src/algorithms/sl/sublattice.inl:24-190 on the device.
 *
 * Plain C types only.  Every call returns an akmc_status and never exits the
 * process (the reference exits on any HIP error, gpu/gpuError.hip:5-37).
 * A context is used by one host thread at a time.
 */
#ifndef AKMC_H
#define AKMC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define AKMC_API __attribute__((visibility("default")))
#else
#define AKMC_API
#endif

typedef enum akmc_status {
  AKMC_OK = 0,
  AKMC_EINVAL = -1,     /* bad argument or configuration */
  AKMC_ENOMEM = -2,     /* device or host allocation failed, or over the memory budget */
  AKMC_ECUDA = -3,      /* CUDA runtime error (message in akmc_last_error) */
  AKMC_ETIMEOUT = -4,   /* a bounded device wait gave up */
  AKMC_EBUSY = -5,      /* resource in use (server full, call in flight) */
  AKMC_ESTATE = -6,     /* call out of order (e.g. run before prepare) */
  AKMC_EOVERFLOW = -7,  /* a per-sector vacancy list or the event log overflowed */
  AKMC_ERANGE = -8,     /* a density left the F table or a round exceeded its hop cap */
  AKMC_ENOTFOUND = -9   /* unknown job id */
} akmc_status;

enum { AKMC_MODEL_PAIRBOND = 0, AKMC_MODEL_EAM = 1 };
enum { AKMC_FP64 = 0, AKMC_FP32C = 1 };
enum { AKMC_RNG_XOSHIRO = 0 };

/* Occupancy codes (src/lattice/lattice_types.h:20-36). */
enum { AKMC_V = 0, AKMC_FE = 1, AKMC_CU = 2, AKMC_NI = 4, AKMC_MN = 8 };

/* Maximum vacancies in the active sector of one domain block. */
#define AKMC_MAX_SECTOR_VACANCIES 64

/* Most domain blocks (summed over the jobs of a context) that akmc_run_rounds_noalloc serves. */
#define AKMC_NOALLOC_MAX_BLOCKS 8192

/*
 * EAM model on the rigid BCC lattice: pair and density functions at the five
 * shells within the cutoff (species order Fe, Cu, Ni, Mn) and the embedding
 * function F(rho) at rho = k * 2^-7, k = 0..4999.  The density f is used in
 * 2^-24 fixed point, so the per-site density cache is an exact int32 sum.
 */
typedef struct akmc_eam_tables {
  int32_t n_shells;
  int32_t reserved;
  double f_shell[4][5];
  double phi_shell[4][4][5];
  double F[5000];
} akmc_eam_tables;

/* One AKMC job: a periodic box decomposed into domain blocks, each block with
 * the 8 sectors of the synchronous sublattice. */
typedef struct akmc_job_config {
  int64_t box[3];           /* cells per dimension (config.yaml box.size) */
  int32_t blocks[3];        /* domain blocks per dimension; 1,1,1 = single domain */
  int32_t energy_model;     /* AKMC_MODEL_* */
  int32_t precision;        /* AKMC_FP64 / AKMC_FP32C (EAM only) */
  int32_t rng;              /* AKMC_RNG_XOSHIRO */
  double lattice_const;     /* Angstrom (box.lattice_const) */
  double cutoff_radius;     /* Angstrom (box.cutoff_radius) */
  double attempt_freq;      /* 1/s (simulation.attempt_freq) */
  double temperature;       /* K (simulation.temperature) */
  double sector_window;     /* s; the reference hard-codes 3e-7 (src/simulation.h:73-74) */
  uint64_t seed;            /* xoshiro256** streams of event selection and time, per block */
  int64_t hop_budget;       /* job ends at the end of the first time step (8 sector rounds) at
                               which its hop count has reached it; <= 0: none */
  int64_t max_rounds;       /* job ends after this many sector rounds; <= 0: none */
  const akmc_eam_tables* eam; /* EAM model (copied at akmc_add_job); NULL for pair-bond */
} akmc_job_config;

/* One performed hop; the layout of dev_event (gpu/DeviceVacRatesSolver.h:20-25)
 * extended with the selection draw, the total rate and the residence time. */
typedef struct akmc_event {
  int64_t round;
  int64_t hop;        /* hop index within its block */
  int64_t from_site;  /* vacancy site before the hop (dev_event.from_id) */
  int64_t to_site;    /* vacancy site after the hop (dev_event.to_id) */
  int32_t block;      /* domain block within the job */
  int32_t species;    /* code of the atom that moved (dev_event.to_type) */
  double u;
  double total;
  double dt;
  int32_t n_act;      /* vacancies in the sector when the hop was selected */
  int32_t n_dirty;    /* vacancies whose rates the hop invalidated */
  int32_t job;
  int32_t reserved;
} akmc_event;

typedef struct akmc_job_state {
  int64_t round;
  int64_t hops;
  int32_t done;
  int32_t n_blocks;
  int64_t n_sites;
  int64_t n_vacancies;
} akmc_job_state;

typedef struct akmc_context_config {
  int32_t device;              /* CUDA device ordinal */
  int32_t graph_rounds;        /* sector rounds per captured CUDA graph (0: 32) */
  void* stream;                /* cudaStream_t to run on; NULL: the context creates one */
  int64_t event_log_capacity;  /* 0: no event log */
  int64_t hop_cap_per_round;   /* per block and round; 0: 1e7 */
  int64_t flow_sweep_limit;    /* AKMC_SCHEDULE_FLOW watchdog: sweeps per CTA and launch before
                                  the launch gives up with AKMC_ETIMEOUT; 0: 2^24.  Rounds
                                  already published stay complete; recover from a snapshot. */
  /* Room for jobs admitted after akmc_prepare (akmc_admit_job); max_jobs = 0: none.  The device
   * tables are sized at akmc_prepare for this many jobs, domain blocks and vacancies held at
   * once (the jobs added before akmc_prepare included), and shared memory for domain blocks of
   * up to max_block_edge cells (0: 24). */
  int32_t max_jobs;
  int32_t max_block_edge;
  int64_t max_blocks;
  int64_t max_vacancies;
  /* Launch shape of the hop kernels (autotuned by akmc_b200.autotune): eval_warps = warps that
   * evaluate a vacancy's 8 jumps, 8 (one jump each, one CTA per SM; 0 = 8) or 4 (two jumps each,
   * two CTAs per SM); flow_take = rounds with vacancies a CTA of the dependency-driven schedule
   * takes per sweep (0: all it finds).  Results do not depend on either. */
  int32_t eval_warps;
  int32_t flow_take;
} akmc_context_config;

typedef struct akmc_ctx akmc_ctx;

AKMC_API const char* akmc_status_string(akmc_status s);
AKMC_API akmc_status akmc_last_error(akmc_ctx* ctx, char* buf, int32_t len);

/* initialize_gpu (gpu/gpu_simulate.h:47, gpu_simulate.hip:1764-1769): selects
 * device process_rank % device_count.  Unlike the reference it does not reset
 * the device. */
AKMC_API akmc_status akmc_initialize_gpu(int32_t process_rank, int32_t* device);

AKMC_API akmc_status akmc_create(const akmc_context_config* cfg, akmc_ctx** out);
AKMC_API akmc_status akmc_destroy(akmc_ctx* ctx);

/* Registers a job.  occ holds the occupancy codes of the 2*nx*ny*nz sites,
 * site id = x + 2nx (y + ny z) with x doubled (LatListMeta::getLId,
 * src/lattice/lattice_list_meta.h:103-106); every AKMC_V site is a vacancy.
 * The library copies the array; the caller keeps ownership (the reference's
 * firstSectLocalToGpu frees its caller's array, gpu_simulate.hip:1207). */
AKMC_API akmc_status akmc_add_job(akmc_ctx* ctx, const akmc_job_config* cfg, const uint8_t* occ, int64_t n_sites,
                                  int32_t* job_id);

/* gpu_prepare (gpu/gpu_simulate.h:51, gpu_simulate.hip:1771-1831): allocates the
 * device state of every registered job, uploads the lattices and builds the
 * density caches. */
AKMC_API akmc_status akmc_prepare(akmc_ctx* ctx);

/* No reference counterpart (the reference runs one box per process).  Continuous batching:
 * adds a job to a prepared context created with room for it (akmc_context_config.max_jobs),
 * between calls that run rounds, without touching the jobs already running.  Its lattice,
 * density cache, vacancies and random streams go into free slots of the device tables; it
 * starts at round 0 and advances with every later akmc_run_rounds, its trajectory the same as
 * alone.  A retired job's slot id may be given out again.  EBUSY when the context has no room
 * left (jobs, blocks, vacancies or potentials), EINVAL for blocks larger than max_block_edge. */
AKMC_API akmc_status akmc_admit_job(akmc_ctx* ctx, const akmc_job_config* cfg, const uint8_t* occ, int64_t n_sites,
                                    int32_t* job_id);
/* Frees an admitted or added job's slots and device memory (read its results first); the other
 * jobs run on untouched.  Later calls that name the job return ENOTFOUND. */
AKMC_API akmc_status akmc_retire_job(akmc_ctx* ctx, int32_t job);

/* Runs n sector rounds of every unfinished job on the device (the loop body of
 * SubLattice::startTimeLoop, sublattice.inl:64-177, for all domain blocks at
 * once).  Asynchronous on the context stream; errors surface at akmc_sync. */
AKMC_API akmc_status akmc_run_rounds(akmc_ctx* ctx, int64_t n_rounds);
/* No reference counterpart.  akmc_run_rounds without any allocation: the same
 * three launches per round, one by one (no CUDA graph is instantiated), with the
 * per-round scratch (block vacancy lists, active-block list, active count) in a
 * fixed device array of the library instead of context memory.  It serves up to
 * AKMC_NOALLOC_MAX_BLOCKS domain blocks and returns AKMC_EINVAL beyond that.
 * The first call on a device looks up the scratch address with that device
 * current; make it before any stream capture.  The scratch is shared by all
 * contexts of a device: calls whose rounds overlap on the device race.  Kernel
 * timing mode is not applied. */
AKMC_API akmc_status akmc_run_rounds_noalloc(akmc_ctx* ctx, int64_t n_rounds);
/* No reference counterpart.  Up to n_rounds more rounds of every unfinished job, in one launch of
 * the dependency-driven schedule that takes no new round after max_us microseconds: each job
 * advances as far as its own rounds allow in that time, so small jobs are not held to the pace
 * of large ones (the server's chunks).  Jobs end at different rounds; a later call continues
 * each where it stopped, and the trajectories are the same as with akmc_run_rounds.  Contexts on
 * the round-by-round schedule run min(n_rounds, graph_rounds) rounds instead.  Asynchronous, as
 * akmc_run_rounds; akmc_get_job_states tells where each job is. */
AKMC_API akmc_status akmc_run_for(akmc_ctx* ctx, int64_t n_rounds, int64_t max_us);
/* Order in which akmc_run_rounds runs the rounds of different domain blocks.
 * ROUNDS: every block finishes round r before any starts r+1 (SubLattice::startTimeLoop,
 * sublattice.inl:61-179, with the blocks as MPI ranks).  FLOW: a block's round waits only
 * for the neighbour rounds whose staged regions (sector plus a 2-cell halo) overlap it, so
 * blocks with few hops run ahead; results are identical to ROUNDS.  Under FLOW a job's hop
 * budget is checked inside the launch: the blocks of a multi-block budget job wait for one
 * another at each time-step boundary.  AUTO (default): FLOW when the context holds
 * more than one domain block and every block area starts with at most 32 vacancies, else
 * ROUNDS.  akmc_run_rounds_noalloc always runs ROUNDS. */
enum { AKMC_SCHEDULE_AUTO = 0, AKMC_SCHEDULE_ROUNDS = 1, AKMC_SCHEDULE_FLOW = 2 };
AKMC_API akmc_status akmc_set_round_schedule(akmc_ctx* ctx, int32_t schedule);
/* The schedule akmc_run_rounds uses (ROUNDS or FLOW), AUTO resolved; after akmc_prepare. */
AKMC_API akmc_status akmc_get_round_schedule(akmc_ctx* ctx, int32_t* effective);
/* Runs until every job is done (hop budget or max_rounds) or max_rounds pass. */
AKMC_API akmc_status akmc_run(akmc_ctx* ctx, int64_t max_rounds);
AKMC_API akmc_status akmc_sync(akmc_ctx* ctx);
AKMC_API void* akmc_stream(akmc_ctx* ctx);

/* gpu_final (gpu/gpu_simulate.h:49, gpu_simulate.hip:1833-1872): waits for the
 * device and reports any deferred error. */
AKMC_API akmc_status akmc_gpu_final(akmc_ctx* ctx);

AKMC_API akmc_status akmc_get_job_state(akmc_ctx* ctx, int32_t job, akmc_job_state* st);
/* Every job's state with one device read; n_jobs must be the context's job count. */
AKMC_API akmc_status akmc_get_job_states(akmc_ctx* ctx, akmc_job_state* out, int32_t n_jobs);
AKMC_API akmc_status akmc_get_occupancy(akmc_ctx* ctx, int32_t job, uint8_t* out, int64_t n_sites);
AKMC_API akmc_status akmc_get_rho(akmc_ctx* ctx, int32_t job, int32_t* out, int64_t n_sites);
/* evo[nblocks][8]: per-sector evolution time (SectorMeta, sublattice.h:17-33); hops[nblocks]. */
AKMC_API akmc_status akmc_get_block_clocks(akmc_ctx* ctx, int32_t job, double* evo, int64_t* hops, int32_t n_blocks);
/* Copies the event log (all jobs, device order) and empties it. */
AKMC_API akmc_status akmc_get_events(akmc_ctx* ctx, akmc_event* out, int64_t capacity, int64_t* n_out);
/* Device-side counters: [0] hops, [1] vacancy rate evaluations, [2] rounds run,
 * [3] active blocks processed, [4] sum over hops of the sector's vacancy count,
 * [5] region sites staged into shared memory, [6] region sites written back, [7] reserved. */
AKMC_API akmc_status akmc_get_counters(akmc_ctx* ctx, int64_t* out8);

/* Cycle profile of the hop kernel's phases (thread 0, summed over blocks): [0] staging,
 * [1] list sort and table window, [2] first evaluations, [3] selection, [4] perform,
 * [5] re-evaluation and clock, [6] tail; EAM FP64 evaluation sub-phases: [8] site loop,
 * [9] butterfly, [10] own-embedding term, [11] rate.  All zero unless the library was
 * built with -DAKMC_PHASE_PROFILE. */
AKMC_API akmc_status akmc_get_phase_cycles(akmc_ctx* ctx, int64_t* out16);

/* Replaces the lattice of a prepared job (same box and vacancy count) and
 * restarts it: density cache rebuilt on the device, clocks, rounds and RNG
 * streams reset as after akmc_prepare.  gpu_prepare's lattice upload
 * (gpu_simulate.hip:1771-1831) for a new box.  Asynchronous on the context's
 * stream: from pinned memory, occ must stay unchanged until the stream is
 * synchronised, and a lattice with another vacancy count is reported
 * (AKMC_EINVAL) by the next synchronising call. */
AKMC_API akmc_status akmc_load_occupancy(akmc_ctx* ctx, int32_t job, const uint8_t* occ, int64_t n_sites);

/* All jobs at once: the lattices of every job of the context back to back in job order
 * (total_sites = the sum of their sites).  akmc_load_occupancies is akmc_load_occupancy for
 * every job, with one host copy and one launch of each kernel for the whole context
 * (asynchronous; errors as there).  akmc_get_occupancies reads them all back the same way. */
AKMC_API akmc_status akmc_load_occupancies(akmc_ctx* ctx, const uint8_t* occ, int64_t total_sites);
AKMC_API akmc_status akmc_get_occupancies(akmc_ctx* ctx, uint8_t* out, int64_t total_sites);

/* Restart snapshots.  The reference's restart is a stub (pkmc.cpp:183-184); this one holds
 * a job's lattice, its rounds, hop counts, sector clocks and random streams per block, in a
 * versioned byte buffer with a checksum.  Restored into a job added with the same
 * configuration and potential (checked) and prepared, the run continues exactly as the
 * uninterrupted one: same events, clocks and lattice.  Save between runs; it synchronises. */
AKMC_API akmc_status akmc_snapshot_size(akmc_ctx* ctx, int32_t job, int64_t* bytes);
AKMC_API akmc_status akmc_save_snapshot(akmc_ctx* ctx, int32_t job, uint8_t* buf, int64_t capacity, int64_t* written);
AKMC_API akmc_status akmc_restore_snapshot(akmc_ctx* ctx, int32_t job, const uint8_t* buf, int64_t n);

/* Kernel timing mode: while enabled, akmc_run_rounds launches each round on its
 * own (no CUDA graph) with CUDA events around the hop kernel on the context
 * stream; akmc_get_kernel_timing returns their summed time and the launch count. */
AKMC_API akmc_status akmc_set_kernel_timing(akmc_ctx* ctx, int32_t enable);
AKMC_API akmc_status akmc_get_kernel_timing(akmc_ctx* ctx, double* hop_kernel_ms, int64_t* hop_launches);

/*
 * Per-hop entry points for a single-domain job, with the host driving the
 * sector loop, the RNG and the clock exactly as ABVIModel + SubLattice do.
 */
/* calculate_GPU / first_calculate_GPU (gpu_simulate.h:33-35, gpu_simulate.hip:1211-1716):
 * rates of every vacancy in sector sector_id; returns their ordered sum. */
AKMC_API akmc_status akmc_calculate(akmc_ctx* ctx, int32_t job, int32_t sector_id, double* total);
/* The jumps behind the last akmc_calculate, as the device vacancy records hold
 * them (d_vacancy_adv[].rates, gpu_simulate.hip:476-480): for each of the n_out
 * vacancies of the sector, in list order, its site (-1 if it has left the
 * sector), the 8 jumps' ΔE in eV (0 for a jump onto a vacancy) and rates in Hz
 * (0 likewise).  delta_e and rates hold 8 * capacity values.  AKMC_EINVAL with
 * n_out set when capacity is too small; n_out = 0 before any akmc_calculate. */
AKMC_API akmc_status akmc_get_calculated_rates(akmc_ctx* ctx, int32_t* sites, double* delta_e, double* rates,
                                               int64_t capacity, int64_t* n_out);
/* selectAndPerformEventGPU (gpu_simulate.h:37-41, gpu_simulate.hip:1388-1449):
 * selects the first event whose cumulative rate exceeds u * total in z-y-x
 * order and performs it.  ev->from_site < 0 when no event is selected. */
AKMC_API akmc_status akmc_select_and_perform(akmc_ctx* ctx, int32_t job, int32_t sector_id, double u,
                                             akmc_event* ev);

/* Helpers. */
/* Synthetic Johnson-form EAM for Fe, Cu, Ni, Mn from a seed (xoshiro stream tag 5). */
AKMC_API akmc_status akmc_eam_johnson(uint64_t seed, double lattice_const, double cutoff_radius,
                                      akmc_eam_tables* out);
/* Random alloy and vacancies (creation::createRandom, src/creation.cpp:96-164) with
 * xoshiro256** streams: one draw per site in site-id order, then vacancies. */
AKMC_API akmc_status akmc_create_lattice(const int64_t box[3], const int32_t type_codes[4], const int64_t ratio[4],
                                         int64_t n_vacancies, uint64_t seed, uint8_t* occ, int64_t n_sites);
/* Isolated-Cu count (profiles/m_event_hook.cpp:17-55) and Cu cluster-size histogram (1nn):
 * hist[k] = clusters of k atoms, the last bin holding all larger ones.  Host code. */
AKMC_API akmc_status akmc_cluster_stats(const uint8_t* occ, const int64_t box[3], int64_t* isolated_cu, int64_t* hist,
                                        int64_t hist_len);
/* The same statistics of a job's resident lattice, computed on the device (the reference
 * computes them on the host from its hash sets, m_event_hook.cpp:17-55).  hist_len <=
 * AKMC_CLUSTER_MAX_BINS.  The first call for a job size allocates 12 bytes per site. */
#define AKMC_CLUSTER_MAX_BINS 4096
AKMC_API akmc_status akmc_job_cluster_stats(akmc_ctx* ctx, int32_t job, int64_t* isolated_cu, int64_t* hist,
                                            int64_t hist_len);

/*
 * config.yaml of the reference (profiles/config/config_parsing.cpp:54-230, keys of
 * examples/config.yaml) plus an optional `kmc:` block read only by this library:
 * energy_model (pairbond|eam), precision (fp64|fp32c), blocks [bx,by,bz],
 * creation (reference|xoshiro), sector_window, hop_budget, seed, pot_seed.
 */
typedef struct akmc_run_config {
  int64_t box[3];
  double lattice_const;
  double cutoff_radius;
  int32_t create_random;
  int32_t n_types;            /* single-atom alloy entries, YAML order */
  int32_t type_codes[4];
  int64_t ratio[4];
  int64_t va_count;
  int64_t seed_create_types, seed_create_vacancy, seed_event_selection, seed_time_inc;
  double temperature, physics_time, attempt_freq, dpasm1;
  int64_t steps_limit;
  int32_t isgenr;
  int32_t energy_model, precision, creation;
  int32_t blocks[3];
  int32_t reserved;
  double sector_window;
  int64_t hop_budget;
  uint64_t seed, pot_seed;
  int64_t dump_interval, logs_interval;
  char dump_file_path[256];
  char logs_file[256];
  int32_t create_pipe;        /* create.pipe.enable (ConfigParsing::parseCreate, config_parsing.cpp:171-189) */
  int32_t reserved2;
  char pipe_input_box[256];   /* create.pipe.input_box: vacancy positions "x y z" (x doubled), whitespace
                                 separated, read by akmc_config_lattice relative to the working directory */
} akmc_run_config;

AKMC_API akmc_status akmc_config_parse(const char* yaml_text, akmc_run_config* out, char* err, int32_t errlen);
/* The lattice of a config: creation = reference reproduces creation::createRandom's
 * mt19937 draw order (ghost sites included, src/creation.cpp:18-164).  With create.pipe the
 * alloy is drawn the same way and the vacancies are the in-box positions of the pile file
 * (creation::createFromPile, src/creation.cpp:184-230); EINVAL if the file cannot be read. */
AKMC_API akmc_status akmc_config_lattice(const akmc_run_config* cfg, uint8_t* occ, int64_t n_sites);
AKMC_API akmc_status akmc_config_job(const akmc_run_config* cfg, const akmc_eam_tables* eam, akmc_job_config* out);
/* SubLattice::startTimeLoop (sublattice.inl:24-190) for a single-domain job,
 * driven from the host over akmc_calculate / akmc_select_and_perform with the
 * job's xoshiro selection and time streams; events and the 8 sector clocks out. */
AKMC_API akmc_status akmc_host_time_loop(akmc_ctx* ctx, int32_t job, int64_t n_rounds, uint64_t seed, double window,
                                         akmc_event* events, int64_t capacity, int64_t* n_events, double* evo8);
/* LatticeDump::dump format (profiles/io/lattice_dump.cpp:14-62). */
AKMC_API akmc_status akmc_dump_lattice(const uint8_t* occ, const int64_t box[3], int32_t ghost, const char* path);

/* Device checks of the shared arithmetic: port_exp/port_log of x[i] on the GPU. */
AKMC_API akmc_status akmc_device_math(akmc_ctx* ctx, const double* x, int64_t n, double* exp_out, double* log_out);

/*
 * Job server: many independent jobs (parameter sweeps, ensembles, requests) on one GPU, with
 * continuous batching.  Submitted jobs queue; worker lanes (one host thread, one CUDA stream and
 * one context each) admit queued jobs in arrival order into their running context as the
 * device-memory budget and the context's room allow (akmc_admit_job), advance all of their live
 * jobs together in chunks of rounds, and publish each job's result, and free its memory, as soon
 * as that job is done (akmc_retire_job).  A job's state stays in device memory from admission to
 * its end, and its result is the one it has alone.  The server is internally synchronised: any
 * host thread may submit and poll.  This replaces running one MPI job per box.
 */
typedef struct akmc_server akmc_server;
typedef struct akmc_server_config {
  int32_t device;           /* CUDA device ordinal */
  int32_t lanes;            /* lanes, each with its own context and stream (0: 2) */
  int64_t budget_bytes;     /* device memory the running jobs of all lanes may hold (0: 8 GiB) */
  int32_t max_batch_jobs;   /* jobs one lane runs at once (0: 512) */
  int32_t chunk_rounds;     /* rounds per chunk of a lane whose context runs round by round (0: 16) */
  int32_t order;            /* admission order of queued jobs: AKMC_SERVE_FIFO (arrival) or
                               AKMC_SERVE_SMALLEST_BUDGET (smallest hop budget first; jobs
                               without a budget last; ties in arrival order) */
  int32_t chunk_us;         /* wall time of a chunk (akmc_run_for) between admissions and checks
                               for finished jobs, in microseconds (0: 2000) */
} akmc_server_config;
enum { AKMC_SERVE_FIFO = 0, AKMC_SERVE_SMALLEST_BUDGET = 1 };
typedef struct akmc_job_result {
  int64_t hops;
  int64_t rounds;
  double submit_s;          /* server clock (seconds since akmc_server_create) */
  double start_s;           /* a lane took it */
  double finish_s;          /* the result was published */
  int32_t status;           /* akmc_status of the job */
  int32_t n_blocks;
  char error[128];          /* akmc_last_error of its lane's context when status != AKMC_OK */
  uint64_t clocks_fnv;      /* FNV-1a 64 of the bytes of every domain block's 8 sector clocks (FP64)
                               and hop count (int64), block after block, as akmc_get_block_clocks
                               gives them: the end state of the job's clocks in one word */
} akmc_job_result;
AKMC_API akmc_status akmc_server_create(const akmc_server_config* cfg, akmc_server** out);
/* Queues a job (cfg, its EAM tables and occ are copied).  The job must end by itself: a hop
 * budget or max_rounds.  EINVAL for a job no lane could run (bad config, domain blocks larger
 * than 24 cells, or more device memory than the whole budget). */
AKMC_API akmc_status akmc_server_submit(akmc_server* s, const akmc_job_config* cfg, const uint8_t* occ,
                                        int64_t n_sites, int64_t* ticket);
/* ready = 1 once the job is done: res is filled and, when occ_out is not NULL, the final
 * lattice copied (n_sites bytes); the job's record is then released.  ready = 0 while it
 * queues or runs.  ENOTFOUND for an unknown or already collected ticket. */
AKMC_API akmc_status akmc_server_poll(akmc_server* s, int64_t ticket, akmc_job_result* res, uint8_t* occ_out,
                                      int64_t n_sites, int32_t* ready);
/* akmc_server_poll that blocks up to timeout_s seconds (ETIMEOUT if the job is not done). */
AKMC_API akmc_status akmc_server_wait(akmc_server* s, int64_t ticket, double timeout_s, akmc_job_result* res,
                                      uint8_t* occ_out, int64_t n_sites);
/* Jobs queued or running, and jobs done but not collected. */
AKMC_API akmc_status akmc_server_stats(akmc_server* s, int64_t* queued, int64_t* running, int64_t* done);
/* Finishes the running batches, fails the queued jobs (status AKMC_ESTATE) and frees the
 * server. */
/* Where the lanes' time went, summed over lanes: seconds8 = [0] changing the job sets (creating
 * the lanes' contexts, admitting and retiring jobs), [1] running chunks (rounds and the job-state
 * read), [2] reading results, [3] waiting for work; parts of [0]: [4] admitting, [5] creating the
 * contexts, [6] retiring, [7] 0; counts3 = chunks run, live jobs summed over chunks (their ratio
 * is the mean number of jobs a chunk advanced), contexts created. */
AKMC_API akmc_status akmc_server_profile(akmc_server* s, double* seconds8, int64_t* counts3);
AKMC_API akmc_status akmc_server_shutdown(akmc_server* s);

#ifdef __cplusplus
}
#endif

#endif /* AKMC_H */
