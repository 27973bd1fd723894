/*
 * akmc_oracle.h -- C API of the CPU oracle for the AKMC vacancy-hop path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: the parity tests,
 * the smoke check and the cpu_baseline leg of the benchmark call it.  Nothing in
 * the product (libakmc_b200.so, the host layer, the kernels) includes or links it.
 *
 * The oracle restates the CPU path of MISA-AKMC (panzhija/MISA-AKMC-GPU):
 *   - lattice ids / neighbours   src/lattice/lattice_list_meta.{h,cpp}, src/lattice/period_lattice_list.cpp
 *   - pair-bond dE               models/abvi/rate/vacancy_rates_solver.cpp:29-172,
 *                                models/abvi/rate/bonds/bonds_counter.cpp:13-129
 *   - rate                       models/abvi/rate/rates_solver.cpp:12-26, rates_types.h:16
 *   - scan / select / perform    models/abvi/kmc.cpp:68-115, 242-309, 358-396
 *   - sector schedule and clock  src/algorithms/sl/sublattice.inl:24-190, sublattice.h:17-33
 *   - RNG use                    src/models/model_adapter.h:88-105, src/utils/random/random.cpp:35-41
 *   - creation                   src/creation.cpp:18-164
 *   - isolated-Cu statistic      profiles/m_event_hook.cpp:17-55
 * and adds the synthetic Johnson-form EAM model and the xoshiro256** streams,
 * which the reference does not have (its EAM branch returns 0,
 * vacancy_rates_solver.cpp:42-43).
 */
#ifndef AKMC_ORACLE_H
#define AKMC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { AO_MODEL_PAIRBOND = 0, AO_MODEL_EAM = 1 };
enum { AO_FP64 = 0, AO_FP32C = 1 };
enum { AO_RNG_XOSHIRO = 0, AO_RNG_MT19937_REF = 1 };
enum { AO_MATH_PORTABLE = 0, AO_MATH_LIBM = 1 };
enum { AO_CREATE_XOSHIRO = 0, AO_CREATE_MT19937_REF = 1, AO_CREATE_EXTERNAL = 2, AO_CREATE_MT19937_PILE = 3 };

typedef struct ao_config {
  int64_t box[3];         /* cells per dimension (config.yaml box.size) */
  int32_t blocks[3];      /* domain blocks per dimension (1,1,1 = single domain) */
  int32_t energy_model;   /* AO_MODEL_* */
  int32_t precision;      /* AO_FP64 / AO_FP32C (EAM only) */
  int32_t rng_mode;       /* AO_RNG_* */
  int32_t math_mode;      /* AO_MATH_PORTABLE: own exp/log; AO_MATH_LIBM: libm exp/log */
  int32_t creation_mode;  /* AO_CREATE_* */
  int32_t log_events;     /* 1: record every hop */
  double lattice_const;   /* Angstrom */
  double cutoff;          /* Angstrom */
  double attempt_freq;    /* 1/s */
  double temperature;     /* K */
  double window;          /* sector time window T, s (reference: 3e-7) */
  uint64_t seed;          /* xoshiro job seed; mt mode: seeds.create_types */
  uint64_t seed_vacancy;  /* mt mode: seeds.create_vacancy */
  uint64_t seed_time_inc; /* mt mode: seeds.time_inc */
  uint64_t pot_seed;      /* seed of the synthetic EAM parameter draw */
  int32_t type_codes[4];  /* alloy species codes in config order (reference: YAML map order) */
  int64_t ratio[4];       /* alloy ratio of type_codes[i] */
  int64_t n_vacancies;
  /* AO_CREATE_MT19937_PILE: vacancy positions (x doubled, y, z) of the pile file, pile_n triples */
  const int64_t* pile_xyz;
  int64_t pile_n;
} ao_config;

typedef struct ao_event {
  int64_t round;
  int64_t hop;        /* hop index within its block */
  int64_t from_site;  /* vacancy site before the hop */
  int64_t to_site;    /* vacancy site after the hop */
  int32_t block;
  int32_t species;    /* code of the atom that moved (Fe=1, Cu=2, Ni=4, Mn=8) */
  double u;           /* selection uniform */
  double total;       /* total rate of the sector */
  double dt;          /* residence time */
  int32_t n_act;      /* vacancies in the sector when the hop was selected */
  int32_t n_dirty;    /* vacancies whose rates the hop invalidates (device rule) */
} ao_event;

void* ao_create(const ao_config* cfg, char* err, int errlen);
void ao_destroy(void* h);

int64_t ao_nsites(void* h);
int32_t ao_nblocks(void* h);
int ao_set_occupancy(void* h, const uint8_t* occ, int64_t n);
int ao_get_occupancy(void* h, uint8_t* out);
int ao_get_rho(void* h, int32_t* out);

/* Runs whole sector rounds.  ao_run stops at the end of the first round in
 * which the job's hop count reaches hop_budget (<=0: no budget), or after
 * max_rounds rounds. Returns 0 on success, negative on error. */
int ao_run_rounds(void* h, int64_t n_rounds);
int ao_run(void* h, int64_t hop_budget, int64_t max_rounds);
/* n_rounds rounds of every block in a random dependency-respecting order instead of
 * round by round (a block's round waits only for the neighbour rounds whose staged
 * regions overlap it).  order_seed 0 always runs the ready block furthest ahead.
 * Must leave the same state and events as ao_run_rounds. */
int ao_run_rounds_flow(void* h, int64_t n_rounds, uint64_t order_seed);

int64_t ao_round(void* h);
int64_t ao_total_hops(void* h);
int64_t ao_num_events(void* h);
int ao_get_events(void* h, ao_event* out, int64_t start, int64_t n);
int ao_get_block_state(void* h, double* evo /* nblocks*8 */, int64_t* hops /* nblocks */);
/* stats: [0]=hops [1]=sum of n_act over hops [2]=sum of n_dirty [3]=rate evaluations at round starts */
int ao_stats(void* h, int64_t* out4);

/* Rate evaluation of one vacancy with the current lattice. */
int ao_vacancy_rates(void* h, int64_t site, double* rates8, double* de8);
double ao_bond_count(void* h, int64_t site, int32_t src_code);

/* The EAM tables the oracle built, for comparison with the product's tables. */
int ao_eam_export(void* h, double* params /*4x5*/, double* f_sh /*4x5*/, double* phi_sh /*4x4x5*/,
                  int32_t* fq /*4x7*/, double* coef /*5000x4*/);

/* 1nn ids in LatListMeta::getIdBy1nnOffset order and 2nn ids in get2nn2 order. */
int ao_neighbours(void* h, int64_t site, int64_t* nn1 /*8*/, int64_t* nn2 /*6*/);

int ao_cluster_stats(void* h, int64_t* isolated_cu, int64_t* hist, int64_t hist_len);

/* The oracle's portable exp/log and its xoshiro256** streams (known-answer tests). */
double ao_exp(double x);
double ao_log(double x);
int ao_xoshiro_stream(uint64_t seed, uint64_t tag, uint64_t index, uint64_t* out, int64_t n);
int ao_mt19937_draws(uint64_t seed, int use_default_seed, int canonical, double* out, int64_t n);

#ifdef __cplusplus
}
#endif

#endif
