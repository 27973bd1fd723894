// akmc_api.cu -- the C ABI of include/akmc.h over the kernels of akmc_kernels.cu.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "akmc_device.h"
#include "akmc_model.h"

using namespace akmc;

namespace {

struct HostJob {
  akmc_job_config cfg{};
  bool has_eam = false;
  akmc_eam_tables eam{};
  std::vector<uint8_t> occ;
  int64_t nsites = 0;
  int64_t nvac = 0;
  int32_t block0 = 0, nblocks = 0;
  int32_t vac0 = 0;
  int32_t pot = 0;
  int32_t area_max = 0;   // most vacancies in one of its block areas at the start
  bool live = true;       // false: a retired slot (akmc_retire_job)
  std::vector<int32_t> split[3];
  uint8_t* d_occ = nullptr;
  int32_t* d_rho = nullptr;
  CUtensorMap tmap[2];    // occupancy and density maps of the device lattice (JobDev::tma)
};

struct DevPot {
  Potential P;
  double* d_coef = nullptr;  // planes (c0, c1) then (c2, c3), kTabN cells each
  float* d_f32 = nullptr;    // planes (hi, lo, c1, c2) then c3
  std::vector<double> coef;
  std::vector<FCell32> f32;
  bool has_eam = false;
  akmc_eam_tables src{};
};

const char* cuda_name(int e) { return cudaGetErrorString(static_cast<cudaError_t>(e)); }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against the driver
// library); null when the driver does not offer it.
PFN_cuTensorMapEncodeTiled_v12000 tensor_encode() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return static_cast<PFN_cuTensorMapEncodeTiled_v12000>(nullptr);
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// The tensor map of a job's device lattice array (halo layout, element size es): 3D tensor of
// (pitch, sy, sz) entries, box = the job's widest staged region.  False if it cannot be encoded
// (the job then stages by row copies).
bool encode_lattice_map(CUtensorMap* m, void* base, int es, int32_t sx, int32_t sy, int32_t sz, const int32_t box[3]) {
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_encode();
  if (!enc || !base) return false;
  for (int d = 0; d < 3; ++d)
    if (box[d] < 1 || box[d] > 256) return false;
  if ((box[0] * es) % 16) return false;
  const cuuint64_t px = static_cast<cuuint64_t>(lattice_pitch(sx));
  const cuuint64_t dim[3] = {px, static_cast<cuuint64_t>(sy), static_cast<cuuint64_t>(sz)};
  const cuuint64_t stride[2] = {px * es, px * es * dim[1]};
  const cuuint32_t bdim[3] = {static_cast<cuuint32_t>(box[0]), static_cast<cuuint32_t>(box[1]), static_cast<cuuint32_t>(box[2])};
  const cuuint32_t estride[3] = {1, 1, 1};
  return enc(m, es == 1 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_INT32, 3, base, dim, stride, bdim,
             estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

struct akmc_ctx {
  akmc_context_config cfg{};
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;
  std::vector<HostJob> jobs;
  std::vector<DevPot> pots;
  // x and y extents of every job's tensor box: the widest of the context's jobs (and of the
  // blocks an admitted job may have), so that every region shares one row and plane pitch and
  // the shell tables built for it hold from one job to the next
  int32_t ubox[2] = {0, 0};
  bool prepared = false;
  int32_t nblocks = 0, nvac = 0;
  // device state
  JobDev* d_jobs = nullptr;
  BlockDev* d_blocks = nullptr;
  int32_t* d_vac_site = nullptr;
  int32_t* d_vac_job = nullptr;
  int32_t* d_blk_list = nullptr;
  int32_t* d_active = nullptr;
  int32_t* d_n_active = nullptr;
  Potential* d_pots = nullptr;
  Geometry* d_geo = nullptr;
  akmc_event* d_log = nullptr;
  unsigned long long* d_log_count = nullptr;
  unsigned int* d_status = nullptr;
  unsigned long long* d_counters = nullptr;
  double* d_api_total = nullptr;
  akmc_event* d_api_event = nullptr;
  double* d_api_de = nullptr;
  double* d_api_rates = nullptr;
  int32_t* d_api_sites = nullptr;
  int32_t* d_api_count = nullptr;
  size_t smem = 0;
  int hop_grid = 0;
  int grid_sms = 0, grid_fit = 1, grid_resident = 1;  // SMs, CTAs per SM by shared memory / by registers
  RoundArgs args{};
  cudaGraphExec_t graph = nullptr;
  cudaGraph_t graph_def = nullptr;
  int graph_rounds = 0;
  int32_t* d_vac_count = nullptr;
  // asynchronous round schedule
  int32_t schedule = AKMC_SCHEDULE_AUTO;
  bool flow_ok = false;  // more than one block, and every block area starts with few enough vacancies
  int flow_grid = 0;
  unsigned long long* d_fstate = nullptr;
  unsigned long long* d_vclaim = nullptr;
  unsigned long long* d_vvalid = nullptr;
  int32_t* d_vslot = nullptr;
  int32_t* d_vsite = nullptr;
  int32_t* d_vcount = nullptr;
  int32_t* d_nbr = nullptr;
  unsigned char* d_tmaps = nullptr;  // per job slot: two 128-byte tensor maps
  unsigned int* d_vsec = nullptr;
  int32_t* d_flow = nullptr;  // flow_need[3], flow_done[3]
  // cluster statistics scratch: list, parent, size (one int32 per site of the largest job
  // measured so far), then n_list, the isolated count and the histogram
  int32_t* d_cl = nullptr;
  int64_t cl_sites = 0;
  unsigned long long* d_cl_misc = nullptr;
  // whole-context lattice transfers: staging buffer, chunk table, per-job vacancy counts,
  // density tiles of the EAM jobs (built at the first transfer)
  uint8_t* d_stage = nullptr;
  SiteChunk* d_chunks = nullptr;
  int32_t* d_job_counts = nullptr;
  int32_t* d_job_want = nullptr;
  int64_t* d_tile0 = nullptr;
  int32_t* d_eam_jobs = nullptr;
  JobsLoad jl{};
  int64_t total_sites = 0;
  // kernel timing mode: rounds launched one by one with events around the hop kernel
  bool timing = false;
  std::vector<cudaEvent_t> ev;
  double hop_ms = 0.0;
  int64_t hop_launches = 0;
  // host images of the initial device records (akmc_load_occupancy resets from them)
  std::vector<JobDev> h_jobs;
  std::vector<BlockDev> h_blocks;
  // room for jobs admitted after akmc_prepare: capacities of the device tables, the largest
  // block edge an admitted job may have, and the table ranges not in use ([start, end))
  int32_t cap_jobs = 0, cap_blocks = 0, cap_vac = 0, cap_pots = 0;
  int32_t max_edge = 0;
  bool bulk_ok = false;  // shared memory sized for bulk staging
  std::vector<std::pair<int32_t, int32_t>> free_blocks, free_vac;
};

namespace {

akmc_status fail(akmc_ctx* c, akmc_status s, const std::string& msg) {
  if (c) c->err = msg;
  return s;
}
#define CK(call)                                                                                       \
  do {                                                                                                 \
    cudaError_t e_ = (call);                                                                           \
    if (e_ != cudaSuccess) return fail(ctx, AKMC_ECUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
  } while (0)

// Device memory is stream-ordered (cudaMallocAsync / cudaFreeAsync on the context's stream):
// unlike cudaMalloc and cudaFree, neither waits for other contexts' work on the device, so
// contexts that build and tear down while others run (the server's lanes) do not stall.
template <class T>
cudaError_t dalloc(cudaStream_t s, T** p, size_t n) {
  return cudaMallocAsync(reinterpret_cast<void**>(p), std::max<size_t>(n, 1) * sizeof(T), s);
}
void dfree(cudaStream_t s, void* p) {
  if (p) cudaFreeAsync(p, s);
}

akmc_status check_status(akmc_ctx* ctx) {
  unsigned int st = 0;
  CK(cudaMemcpyAsync(&st, ctx->d_status, sizeof(st), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (!st) return AKMC_OK;
  CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(unsigned int), ctx->stream));
  if (st & kErrVacOverflow)
    return fail(ctx, AKMC_EOVERFLOW, "more than 64 vacancies in one sector (or, under AKMC_SCHEDULE_FLOW, one block area)");
  if (st & kErrRhoRange) return fail(ctx, AKMC_ERANGE, "a density left the F table");
  if (st & kErrHopCap) return fail(ctx, AKMC_ERANGE, "a block exceeded the hop cap of one round");
  if (st & kErrLogOverflow) return fail(ctx, AKMC_EOVERFLOW, "event log full");
  if (st & kErrTimeout) return fail(ctx, AKMC_ETIMEOUT, "a bounded device wait or loop gave up");
  if (st & kErrVacCount)
    return fail(ctx, AKMC_EINVAL, "a lattice given to akmc_load_occupancy does not hold its job's vacancy count");
  return fail(ctx, AKMC_ESTATE, "device reported status " + std::to_string(st));
}

void free_device(akmc_ctx* ctx) {
  for (cudaEvent_t e : ctx->ev) cudaEventDestroy(e);
  ctx->ev.clear();
  dfree(ctx->stream, ctx->d_vac_count);
  ctx->d_vac_count = nullptr;
  void* flow_ptrs[] = {ctx->d_fstate, ctx->d_vclaim, ctx->d_vvalid, ctx->d_vslot, ctx->d_vsite,
                       ctx->d_vcount, ctx->d_nbr,    ctx->d_vsec,   ctx->d_flow};
  for (void* p : flow_ptrs) dfree(ctx->stream, p);
  ctx->d_fstate = nullptr;
  ctx->d_vclaim = ctx->d_vvalid = nullptr;
  ctx->d_vslot = ctx->d_vcount = ctx->d_nbr = ctx->d_flow = nullptr;
  ctx->d_vsec = nullptr;
  ctx->d_vsite = nullptr;
  dfree(ctx->stream, ctx->d_tmaps);
  ctx->d_tmaps = nullptr;
  dfree(ctx->stream, ctx->d_cl);
  dfree(ctx->stream, ctx->d_cl_misc);
  ctx->d_cl = nullptr;
  ctx->d_cl_misc = nullptr;
  ctx->cl_sites = 0;
  void* jl_ptrs[] = {ctx->d_stage, ctx->d_chunks, ctx->d_job_counts, ctx->d_job_want, ctx->d_tile0, ctx->d_eam_jobs};
  for (void* p : jl_ptrs) dfree(ctx->stream, p);
  ctx->d_stage = nullptr;
  ctx->d_chunks = nullptr;
  ctx->d_job_counts = ctx->d_job_want = ctx->d_eam_jobs = nullptr;
  ctx->d_tile0 = nullptr;
  ctx->jl = JobsLoad{};
  ctx->total_sites = 0;
  if (ctx->graph) cudaGraphExecDestroy(ctx->graph);
  if (ctx->graph_def) cudaGraphDestroy(ctx->graph_def);
  ctx->graph = nullptr;
  ctx->graph_def = nullptr;
  for (auto& j : ctx->jobs) {
    dfree(ctx->stream, j.d_occ);
    dfree(ctx->stream, j.d_rho);
    j.d_occ = nullptr;
    j.d_rho = nullptr;
  }
  for (auto& p : ctx->pots) {
    dfree(ctx->stream, p.d_coef);
    dfree(ctx->stream, p.d_f32);
    p.d_coef = nullptr;
    p.d_f32 = nullptr;
  }
  void* ptrs[] = {ctx->d_jobs, ctx->d_blocks, ctx->d_vac_site, ctx->d_vac_job, ctx->d_blk_list, ctx->d_active,
                  ctx->d_n_active, ctx->d_pots, ctx->d_geo, ctx->d_log, ctx->d_log_count, ctx->d_status,
                  ctx->d_counters, ctx->d_api_total, ctx->d_api_event, ctx->d_api_de, ctx->d_api_rates,
                  ctx->d_api_sites, ctx->d_api_count};
  for (void* p : ptrs) dfree(ctx->stream, p);
  ctx->d_jobs = nullptr;
  ctx->d_blocks = nullptr;
  ctx->d_vac_site = ctx->d_vac_job = ctx->d_blk_list = ctx->d_active = ctx->d_n_active = nullptr;
  ctx->d_pots = nullptr;
  ctx->d_geo = nullptr;
  ctx->d_log = nullptr;
  ctx->d_log_count = nullptr;
  ctx->d_status = nullptr;
  ctx->d_counters = nullptr;
  ctx->d_api_total = nullptr;
  ctx->d_api_event = nullptr;
  ctx->d_api_de = ctx->d_api_rates = nullptr;
  ctx->d_api_sites = ctx->d_api_count = nullptr;
  ctx->prepared = false;
}

// Sites of the largest staged region of a job.  With bulk staging a region's rows are
// rounded out to 16-site boundaries, which start up to 14 sites before the region, so the
// rows are laid out with a pitch of the region's width plus 14, rounded up to 16.
int region_sites(const HostJob& j, bool bulk) {
  int64_t mx = 1;
  for (int d = 0; d < 3; ++d) {
    int wmax = 0;
    for (size_t k = 0; k + 1 < j.split[d].size(); ++k) {
      const int w = j.split[d][k + 1] - j.split[d][k];
      wmax = std::max(wmax, w - w / 2);
    }
    int ext = (wmax + 4) * (d == 0 ? 2 : 1);
    if (bulk && d == 0) ext = (ext + 14 + 15) & ~15;
    mx *= ext;
  }
  return static_cast<int>(mx);
}

// The job's own tensor box: its widest region, x rounded out as the bulk form rounds it (the
// sizes region_sites multiplies).
void job_box(const HostJob& j, int32_t box[3]) {
  for (int d = 0; d < 3; ++d) {
    int wmax = 0;
    for (size_t k = 0; k + 1 < j.split[d].size(); ++k) {
      const int w = j.split[d][k + 1] - j.split[d][k];
      wmax = std::max(wmax, w - w / 2);
    }
    box[d] = d == 0 ? (2 * (wmax + 4) + 14 + 15) & ~15 : wmax + 4;
  }
}

// Bulk staging works for every job: the device lattice's rows carry a periodic halo and a pitch
// of a multiple of 16 sites (lattice_pitch), so a region's rows start on 16-byte boundaries.
bool bulk_rows(const HostJob&) { return true; }

// Plain copies between a job's host lattice (rows of sx entries) and the main part of its device
// rows (pitch px, after the kHaloL halo entries); a host-to-device copy refreshes the halos.
template <typename T>
cudaError_t lattice_upload(T* dev, const T* host, int64_t sx, int64_t nrows, cudaStream_t st) {
  const int64_t px = lattice_pitch(static_cast<int32_t>(sx));
  cudaError_t e = cudaMemcpy2DAsync(dev + kHaloL, static_cast<size_t>(px) * sizeof(T), host, static_cast<size_t>(sx) * sizeof(T),
                                    static_cast<size_t>(sx) * sizeof(T), static_cast<size_t>(nrows), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  return static_cast<cudaError_t>(launch_fill_halo(dev, static_cast<int32_t>(sx), nrows, st));
}
template <typename T>
cudaError_t lattice_download(T* host, const T* dev, int64_t sx, int64_t nrows, cudaStream_t st) {
  const int64_t px = lattice_pitch(static_cast<int32_t>(sx));
  return cudaMemcpy2DAsync(host, static_cast<size_t>(sx) * sizeof(T), dev + kHaloL, static_cast<size_t>(px) * sizeof(T),
                           static_cast<size_t>(sx) * sizeof(T), static_cast<size_t>(nrows), cudaMemcpyDeviceToHost, st);
}

// Restart snapshot layout: SnapHeader, then one SnapBlock per domain block, then the
// occupancy bytes.  All fields little-endian, as the host writes them.
struct SnapHeader {
  char magic[8];  // "AKMCSNAP"
  uint32_t version, header_bytes;
  int64_t box[3];
  int32_t blocks[3];
  int32_t model, precision, rng;
  double lattice_const, cutoff, attempt_freq, temperature, window;
  uint64_t seed, eam_hash;
  int64_t round, hops;
  int32_t done, nblocks;
  int64_t nsites, nvac;
  uint64_t checksum;  // FNV-1a 64 of every byte after the header
};
struct SnapBlock {
  int64_t round, hops;
  double evo[8];
  uint64_t xs[4], xt[4];
  int32_t done, pad;
};
constexpr uint32_t kSnapVersion = 2;

// Checksum of the snapshot payload: an FNV-1a step per 64-bit little-endian word (the tail
// zero-padded and tagged with its length), with an xor-shift after each multiply so that
// high bits mix down.  It detects damaged or truncated buffers; it is not cryptographic.
uint64_t fnv1a(const uint8_t* p, size_t n, uint64_t h = 1469598103934665603ull) {
  size_t i = 0;
  for (; i + 8 <= n; i += 8) {
    uint64_t w;
    std::memcpy(&w, p + i, 8);
    h = (h ^ w) * 1099511628211ull;
    h ^= h >> 29;
  }
  uint64_t w = 0;
  std::memcpy(&w, p + i, n - i);
  h = (h ^ w ^ (static_cast<uint64_t>(n - i) << 56)) * 1099511628211ull;
  return h ^ (h >> 29);
}

uint64_t eam_hash(const HostJob& j) {
  return j.has_eam ? fnv1a(reinterpret_cast<const uint8_t*>(&j.eam), sizeof(j.eam)) : 0;
}

bool live_job(const akmc_ctx* ctx, int32_t job) {
  return job >= 0 && job < static_cast<int32_t>(ctx->jobs.size()) && ctx->jobs[static_cast<size_t>(job)].live;
}

int64_t snapshot_bytes(const HostJob& j) {
  return static_cast<int64_t>(sizeof(SnapHeader)) + j.nblocks * static_cast<int64_t>(sizeof(SnapBlock)) + j.nsites;
}

}  // namespace

extern "C" {

AKMC_API const char* akmc_status_string(akmc_status s) {
  switch (s) {
    case AKMC_OK: return "ok";
    case AKMC_EINVAL: return "invalid argument";
    case AKMC_ENOMEM: return "out of memory";
    case AKMC_ECUDA: return "CUDA error";
    case AKMC_ETIMEOUT: return "timed out";
    case AKMC_EBUSY: return "busy";
    case AKMC_ESTATE: return "invalid state";
    case AKMC_EOVERFLOW: return "overflow";
    case AKMC_ERANGE: return "out of range";
    case AKMC_ENOTFOUND: return "not found";
  }
  return "unknown";
}

AKMC_API akmc_status akmc_last_error(akmc_ctx* ctx, char* buf, int32_t len) {
  if (!ctx || !buf || len <= 0) return AKMC_EINVAL;
  std::snprintf(buf, static_cast<size_t>(len), "%s", ctx->err.c_str());
  return AKMC_OK;
}

AKMC_API akmc_status akmc_initialize_gpu(int32_t process_rank, int32_t* device) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return AKMC_ECUDA;
  const int d = (process_rank < 0 ? 0 : process_rank) % n;
  if (cudaSetDevice(d) != cudaSuccess) return AKMC_ECUDA;
  if (device) *device = d;
  return AKMC_OK;
}

AKMC_API akmc_status akmc_create(const akmc_context_config* cfg, akmc_ctx** out) {
  if (!out) return AKMC_EINVAL;
  *out = nullptr;
  akmc_ctx* ctx = new (std::nothrow) akmc_ctx();
  if (!ctx) return AKMC_ENOMEM;
  if (cfg) ctx->cfg = *cfg;
  if (ctx->cfg.graph_rounds <= 0) ctx->cfg.graph_rounds = 32;
  if (ctx->cfg.hop_cap_per_round <= 0) ctx->cfg.hop_cap_per_round = 10000000;
  if (ctx->cfg.flow_sweep_limit <= 0) ctx->cfg.flow_sweep_limit = int64_t(1) << 24;
  if (ctx->cfg.eval_warps == 0) ctx->cfg.eval_warps = 8;
  if ((ctx->cfg.eval_warps != 8 && ctx->cfg.eval_warps != 4) || ctx->cfg.flow_take < 0) {
    delete ctx;
    return AKMC_EINVAL;
  }
  if (cudaSetDevice(ctx->cfg.device) != cudaSuccess) {
    delete ctx;
    return AKMC_ECUDA;
  }
  if (ctx->cfg.stream) {
    ctx->stream = static_cast<cudaStream_t>(ctx->cfg.stream);
  } else {
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete ctx;
      return AKMC_ECUDA;
    }
    ctx->own_stream = true;
  }
  // freed device memory stays in the device's default pool (this process only), so the next
  // context reuses it without a round trip through the driver
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, ctx->cfg.device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  *out = ctx;
  return AKMC_OK;
}

AKMC_API akmc_status akmc_destroy(akmc_ctx* ctx) {
  if (!ctx) return AKMC_EINVAL;
  cudaSetDevice(ctx->cfg.device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  free_device(ctx);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);  // the stream-ordered frees
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return AKMC_OK;
}

AKMC_API void* akmc_stream(akmc_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

}  // extern "C"

namespace {

// A job's configuration and lattice checked and copied into j (akmc_add_job, akmc_admit_job).
akmc_status check_job(akmc_ctx* ctx, const akmc_job_config* cfg, const uint8_t* occ, int64_t n_sites, HostJob& j) {
  j.cfg = *cfg;
  j.cfg.eam = nullptr;
  for (int d = 0; d < 3; ++d) {
    if (cfg->box[d] < 8 || cfg->box[d] > (1 << 20)) return fail(ctx, AKMC_EINVAL, "box edge must be in [8, 2^20] cells");
    const int p = cfg->blocks[d] > 0 ? cfg->blocks[d] : 1;
    block_split(cfg->box[d], p, j.split[d]);
    for (int k = 0; k < p; ++k)
      if (j.split[d][k + 1] - j.split[d][k] < 8)
        return fail(ctx, AKMC_EINVAL, "domain block edges must be >= 8 cells (sector halos may not overlap)");
  }
  j.nsites = 2 * cfg->box[0] * cfg->box[1] * cfg->box[2];
  if (j.nsites != n_sites) return fail(ctx, AKMC_EINVAL, "n_sites != 2*nx*ny*nz");
  if (j.nsites >= (int64_t(1) << 31)) return fail(ctx, AKMC_EINVAL, "more than 2^31 sites in one job");
  if (cfg->energy_model != AKMC_MODEL_PAIRBOND && cfg->energy_model != AKMC_MODEL_EAM)
    return fail(ctx, AKMC_EINVAL, "unknown energy model");
  if (cfg->precision != AKMC_FP64 && cfg->precision != AKMC_FP32C) return fail(ctx, AKMC_EINVAL, "unknown precision");
  if (cfg->rng != AKMC_RNG_XOSHIRO) return fail(ctx, AKMC_EINVAL, "unsupported rng");
  if (!(cfg->temperature > 0) || !(cfg->attempt_freq > 0) || !(cfg->sector_window > 0))
    return fail(ctx, AKMC_EINVAL, "temperature, attempt_freq and sector_window must be > 0");
  if (cfg->energy_model == AKMC_MODEL_EAM) {
    if (!cfg->eam) return fail(ctx, AKMC_EINVAL, "EAM job without tables");
    j.has_eam = true;
    j.eam = *cfg->eam;
    if (j.eam.n_shells != 5 || shells_within(cfg->lattice_const, cfg->cutoff_radius) != 5 ||
        2.0 * cfg->lattice_const < cfg->cutoff_radius)
      return fail(ctx, AKMC_EINVAL, "the EAM path needs exactly the 5 BCC shells inside the cutoff");
  }
  j.occ.assign(occ, occ + n_sites);
  for (int64_t s = 0; s < n_sites; ++s) {
    if (occ[s] == kV) ++j.nvac;
    else if (!is_atom(occ[s])) return fail(ctx, AKMC_EINVAL, "invalid occupancy code at site " + std::to_string(s));
  }
  j.nblocks = (cfg->blocks[0] > 0 ? cfg->blocks[0] : 1) * (cfg->blocks[1] > 0 ? cfg->blocks[1] : 1) *
              (cfg->blocks[2] > 0 ? cfg->blocks[2] : 1);
  for (size_t k = 0; k + 1 < j.split[0].size(); ++k) {
    const int w = j.split[0][k + 1] - j.split[0][k];
    if (2 * (w - w / 2 + 4) > 64)  // staged rows hold at most 64 sites (two per lane)
      return fail(ctx, AKMC_EINVAL, "sector wider than 28 cells in x; use more domain blocks");
  }
  // vacancies per block area (the dependency-driven schedule keeps each area's in 64 slots)
  std::vector<int32_t> per(static_cast<size_t>(j.nblocks), 0);
  const int nbx = static_cast<int>(j.split[0].size()) - 1, nby = static_cast<int>(j.split[1].size()) - 1;
  for (int64_t s = 0; s < n_sites; ++s) {
    if (occ[s] != kV) continue;
    const int64_t X = s % (2 * cfg->box[0]), t = s / (2 * cfg->box[0]);
    const int64_t c[3] = {X >> 1, t % cfg->box[1], t / cfg->box[1]};
    int bi[3];
    for (int d = 0; d < 3; ++d) {
      const auto& sp = j.split[d];
      bi[d] = static_cast<int>(std::upper_bound(sp.begin(), sp.end(), static_cast<int32_t>(c[d])) - sp.begin()) - 1;
    }
    j.area_max = std::max(j.area_max, ++per[static_cast<size_t>(bi[0] + nbx * (bi[1] + nby * bi[2]))]);
  }
  return AKMC_OK;
}

// Largest block edge of a job, over the three dimensions.
int max_block_edge(const HostJob& j) {
  int e = 0;
  for (int d = 0; d < 3; ++d)
    for (size_t k = 0; k + 1 < j.split[d].size(); ++k) e = std::max(e, j.split[d][k + 1] - j.split[d][k]);
  return e;
}

// Sites of the staged region of a block of edge e in every dimension (the largest a job with
// blocks of at most e cells stages), rows padded as region_sites pads them.
int region_sites_edge(int e, bool bulk) {
  const int h = e - e / 2 + 4;
  int ext = 2 * h;
  if (bulk) ext = (ext + 14 + 15) & ~15;
  return ext * h * h;
}

// The potential table entry of job j: an equal one already held, else a new entry (built on the
// host; uploaded by upload_pot).  -1 when the context has no room for another potential.
int find_or_add_pot(akmc_ctx* ctx, HostJob& j, int* rc) {
  *rc = 0;
  if (!j.has_eam) return 0;
  for (size_t i = 1; i < ctx->pots.size(); ++i)
    if (ctx->pots[i].has_eam && std::memcmp(&ctx->pots[i].src, &j.eam, sizeof(j.eam)) == 0) return static_cast<int>(i);
  if (ctx->cap_pots > 0 && static_cast<int32_t>(ctx->pots.size()) >= ctx->cap_pots) return -1;
  DevPot p;
  p.has_eam = true;
  p.src = j.eam;
  *rc = build_potential(&j.eam, p.P, p.coef, p.f32);
  if (*rc) return -1;
  ctx->pots.push_back(std::move(p));
  return static_cast<int>(ctx->pots.size() - 1);
}

// Device tables of potential i: F coefficients in two FP64 planes and the FP32 cells, and the
// Potential record pointing at them (written to hp).
akmc_status upload_pot(akmc_ctx* ctx, size_t i, Potential& hp) {
  DevPot& p = ctx->pots[i];
  std::vector<double> c64(static_cast<size_t>(kTabN) * 4);
  std::vector<float> c32(static_cast<size_t>(kTabN) * 5);
  for (size_t k = 0; k < static_cast<size_t>(kTabN); ++k) {
    for (int jj = 0; jj < 2; ++jj) {
      c64[2 * k + jj] = p.coef[4 * k + jj];
      c64[2 * kTabN + 2 * k + jj] = p.coef[4 * k + 2 + jj];
    }
    const FCell32& f = p.f32[k];
    c32[4 * k + 0] = f.hi;
    c32[4 * k + 1] = f.lo;
    c32[4 * k + 2] = f.c1;
    c32[4 * k + 3] = f.c2;
    c32[4 * static_cast<size_t>(kTabN) + k] = f.c3;
  }
  CK(dalloc(ctx->stream, &p.d_coef, c64.size()));
  CK(dalloc(ctx->stream, &p.d_f32, c32.size()));
  CK(cudaMemcpyAsync(p.d_coef, c64.data(), c64.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(p.d_f32, c32.data(), c32.size() * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));  // the staging vectors go out of scope
  hp = p.P;
  hp.F64lo = reinterpret_cast<const double2*>(p.d_coef);
  hp.F64hi = reinterpret_cast<const double2*>(p.d_coef) + kTabN;
  hp.F32a = reinterpret_cast<const float4*>(p.d_f32);
  hp.F32b = p.d_f32 + 4 * static_cast<size_t>(kTabN);
  return AKMC_OK;
}

// Device memory of job j (occupancy uploaded; density cache allocated) and its records: the
// JobDev, its blocks and its slice of the vacancy table (sites in id order), for slot ji.
akmc_status setup_job(akmc_ctx* ctx, int32_t ji, JobDev& J, BlockDev* hb, int32_t* vsite, int32_t* vjob) {
  HostJob& j = ctx->jobs[static_cast<size_t>(ji)];
  const int32_t sx = 2 * static_cast<int32_t>(j.cfg.box[0]);
  const int64_t nrows = j.cfg.box[1] * j.cfg.box[2];
  const size_t entries = static_cast<size_t>(lattice_entries(sx, static_cast<int32_t>(j.cfg.box[1]),
                                                             static_cast<int32_t>(j.cfg.box[2])));
  CK(dalloc(ctx->stream, &j.d_occ, entries));
  CK(lattice_upload(j.d_occ, j.occ.data(), sx, nrows, ctx->stream));
  if (j.has_eam) CK(dalloc(ctx->stream, &j.d_rho, entries));
  std::memset(&J, 0, sizeof(J));
  J.occ = j.d_occ;
  J.rho = j.d_rho;
  J.px = lattice_pitch(sx);
  J.bulk = ctx->bulk_ok && (reinterpret_cast<uintptr_t>(j.d_occ) & 15) == 0 &&
           (reinterpret_cast<uintptr_t>(j.d_rho) & 15) == 0;
  // the tensor copies' box: the job's widest region in z, the context's widest in x and y (the
  // pitch every region of the context shares)
  job_box(j, J.tbox);
  J.tbox[0] = std::max(J.tbox[0], ctx->ubox[0]);
  J.tbox[1] = std::max(J.tbox[1], ctx->ubox[1]);
  std::memset(j.tmap, 0, sizeof(j.tmap));
  const int32_t sy = static_cast<int32_t>(j.cfg.box[1]), sz = static_cast<int32_t>(j.cfg.box[2]);
  J.tma = J.bulk && encode_lattice_map(&j.tmap[0], j.d_occ, 1, sx, sy, sz, J.tbox) &&
          (!j.has_eam || encode_lattice_map(&j.tmap[1], j.d_rho, 4, sx, sy, sz, J.tbox));
  for (int d = 0; d < 3; ++d) {
    J.n[d] = static_cast<int32_t>(j.cfg.box[d]);
    J.nb[d] = static_cast<int32_t>(j.split[d].size() - 1);
  }
  J.sx = 2 * J.n[0];
  J.sy = J.n[1];
  J.sz = J.n[2];
  J.block0 = j.block0;
  J.nblocks = j.nblocks;
  J.model = j.cfg.energy_model;
  J.precision = j.cfg.precision;
  J.pot = j.pot;
  J.hop_budget = j.cfg.hop_budget;
  J.max_rounds = j.cfg.max_rounds;
  J.nu = j.cfg.attempt_freq;
  J.kT = kBoltzmann * j.cfg.temperature;
  J.window = j.cfg.sector_window;
  for (int b = 0; b < j.nblocks; ++b) {
    BlockDev& B = hb[b];
    std::memset(&B, 0, sizeof(B));
    B.job = ji;
    B.local_id = b;
    const int bi[3] = {b % J.nb[0], (b / J.nb[0]) % J.nb[1], b / (J.nb[0] * J.nb[1])};
    for (int d = 0; d < 3; ++d) {
      B.c0[d] = j.split[d][static_cast<size_t>(bi[d])];
      B.c1[d] = j.split[d][static_cast<size_t>(bi[d]) + 1];
    }
    xoshiro_seed(B.xs, j.cfg.seed, kTagSelect, static_cast<uint64_t>(b));
    xoshiro_seed(B.xt, j.cfg.seed, kTagTime, static_cast<uint64_t>(b));
  }
  int32_t k = 0;
  for (int64_t s = 0; s < j.nsites; ++s)
    if (j.occ[static_cast<size_t>(s)] == kV) {
      vsite[k] = static_cast<int32_t>(s);
      vjob[k] = ji;
      ++k;
    }
  return AKMC_OK;
}

// A free block slot and a free job slot as the kernels see them.
BlockDev free_block_record() {
  BlockDev B;
  std::memset(&B, 0, sizeof(B));
  B.job = -1;
  B.done = 1;
  return B;
}
JobDev free_job_record() {
  JobDev J;
  std::memset(&J, 0, sizeof(J));
  J.done = 1;
  return J;
}

// First-fit allocation of n consecutive entries from a list of free [start, end) ranges.
int32_t take_range(std::vector<std::pair<int32_t, int32_t>>& fr, int32_t n) {
  if (n == 0) return 0;
  for (size_t i = 0; i < fr.size(); ++i)
    if (fr[i].second - fr[i].first >= n) {
      const int32_t at = fr[i].first;
      fr[i].first += n;
      if (fr[i].first == fr[i].second) fr.erase(fr.begin() + static_cast<std::ptrdiff_t>(i));
      return at;
    }
  return -1;
}
void give_range(std::vector<std::pair<int32_t, int32_t>>& fr, int32_t at, int32_t n) {
  if (n == 0) return;
  fr.emplace_back(at, at + n);
  std::sort(fr.begin(), fr.end());
  std::vector<std::pair<int32_t, int32_t>> m;
  for (const auto& r : fr) {
    if (!m.empty() && m.back().second >= r.first) m.back().second = std::max(m.back().second, r.second);
    else m.push_back(r);
  }
  fr.swap(m);
}

// Energy kinds present; whether AUTO may pick the dependency-driven schedule (more than one
// block in use, and every live job's block areas start with at most 32 vacancies); and the
// extent of the tables the kernels walk: every slot below the highest one in use (free slots
// below it are skipped by the kernels), so a context with room for many jobs pays only for the
// ones it holds; the launch grids follow.
void refresh_job_set(akmc_ctx* ctx) {
  int mask = 0, area = 0;
  int32_t hb = 0, hv = 0, hj = 0, live_blocks = 0;
  for (size_t k = 0; k < ctx->jobs.size(); ++k) {
    const auto& j = ctx->jobs[k];
    if (!j.live) continue;
    mask |= 1 << (j.cfg.energy_model == AKMC_MODEL_PAIRBOND ? 0 : (j.cfg.precision == AKMC_FP32C ? 2 : 1));
    area = std::max(area, j.area_max);
    hb = std::max(hb, j.block0 + j.nblocks);
    hv = std::max(hv, j.vac0 + static_cast<int32_t>(j.nvac));
    hj = static_cast<int32_t>(k) + 1;
    live_blocks += j.nblocks;
  }
  RoundArgs& a = ctx->args;
  a.kind_mask = mask;
  a.nblocks = std::max(hb, 1);  // block slot 0 is free when nothing is held: every kernel skips it
  a.nvac = hv;
  a.njobs = std::max(hj, 1);
  ctx->nblocks = a.nblocks;
  ctx->nvac = a.nvac;
  ctx->hop_grid = std::max(1, std::min(a.nblocks, ctx->grid_sms * ctx->grid_fit));
  ctx->flow_grid = std::max(1, std::min(a.nblocks, ctx->grid_sms * ctx->grid_resident));
  ctx->flow_ok = area <= kFlowSlots / 2 && live_blocks > 1;
}

// After the job set changed: the captured round graph and the whole-context transfer tables
// describe the old set; they are rebuilt when next needed.
void drop_job_set_caches(akmc_ctx* ctx) {
  if (ctx->graph) cudaGraphExecDestroy(ctx->graph);
  if (ctx->graph_def) cudaGraphDestroy(ctx->graph_def);
  ctx->graph = nullptr;
  ctx->graph_def = nullptr;
  void* jl_ptrs[] = {ctx->d_stage, ctx->d_chunks, ctx->d_job_counts, ctx->d_job_want, ctx->d_tile0, ctx->d_eam_jobs};
  for (void* p : jl_ptrs) dfree(ctx->stream, p);
  ctx->d_stage = nullptr;
  ctx->d_chunks = nullptr;
  ctx->d_job_counts = ctx->d_job_want = ctx->d_eam_jobs = nullptr;
  ctx->d_tile0 = nullptr;
  ctx->jl = JobsLoad{};
  ctx->total_sites = 0;
}

}  // namespace

extern "C" {

AKMC_API akmc_status akmc_add_job(akmc_ctx* ctx, const akmc_job_config* cfg, const uint8_t* occ, int64_t n_sites,
                                  int32_t* job_id) {
  if (!ctx || !cfg || !occ) return AKMC_EINVAL;
  if (ctx->prepared) return fail(ctx, AKMC_ESTATE, "jobs must be added before akmc_prepare (akmc_admit_job after it)");
  HostJob j;
  const akmc_status st = check_job(ctx, cfg, occ, n_sites, j);
  if (st != AKMC_OK) return st;
  ctx->jobs.push_back(std::move(j));
  if (job_id) *job_id = static_cast<int32_t>(ctx->jobs.size() - 1);
  return AKMC_OK;
}

static akmc_status build_rho_tables(akmc_ctx* ctx);

AKMC_API akmc_status akmc_prepare(akmc_ctx* ctx) {
  if (!ctx) return AKMC_EINVAL;
  if (ctx->prepared) return AKMC_OK;
  const bool room = ctx->cfg.max_jobs > 0;
  if (ctx->jobs.empty() && !room) return fail(ctx, AKMC_ESTATE, "no jobs");
  CK(cudaSetDevice(ctx->cfg.device));
  // potentials: pair-bond tables in every entry; EAM tables deduplicated by content
  ctx->pots.clear();
  {
    DevPot pb;
    if (build_potential(nullptr, pb.P, pb.coef, pb.f32)) return fail(ctx, AKMC_EINVAL, "potential");
    ctx->pots.push_back(std::move(pb));
  }
  ctx->cap_pots = 0;  // no limit while the initial jobs are added
  int max_region = 0, max_region_bulk = 0;
  int32_t nb = 0, nv = 0;
  for (auto& j : ctx->jobs) {
    int rc = 0;
    j.pot = find_or_add_pot(ctx, j, &rc);
    if (rc == -2) return fail(ctx, AKMC_ERANGE, "EAM densities can exceed the F table");
    if (rc || j.pot < 0) return fail(ctx, AKMC_EINVAL, "invalid EAM tables");
    j.block0 = nb;
    j.vac0 = nv;
    nb += j.nblocks;
    nv += static_cast<int32_t>(j.nvac);
    max_region = std::max(max_region, region_sites(j, false));
    max_region_bulk = std::max(max_region_bulk, region_sites(j, bulk_rows(j)));
  }
  // room for jobs admitted later: tables sized to the configured capacities, shared memory to
  // the largest block edge an admitted job may have
  ctx->max_edge = room ? (ctx->cfg.max_block_edge > 0 ? ctx->cfg.max_block_edge : 24) : 0;
  if (room) {
    if (ctx->max_edge < 8 || 2 * (ctx->max_edge - ctx->max_edge / 2 + 4) > 64)
      return fail(ctx, AKMC_EINVAL, "max_block_edge must be in [8, 56] cells");
    max_region = std::max(max_region, region_sites_edge(ctx->max_edge, false));
    max_region_bulk = std::max(max_region_bulk, region_sites_edge(ctx->max_edge, true));
  }
  // the shared x and y pitch of the tensor boxes, and the largest box with it
  ctx->ubox[0] = ctx->ubox[1] = 0;
  for (auto& j : ctx->jobs) {
    int32_t b[3];
    job_box(j, b);
    ctx->ubox[0] = std::max(ctx->ubox[0], b[0]);
    ctx->ubox[1] = std::max(ctx->ubox[1], b[1]);
  }
  const int he = room ? ctx->max_edge - ctx->max_edge / 2 + 4 : 0;
  if (room) {
    ctx->ubox[0] = std::max(ctx->ubox[0], (2 * he + 14 + 15) & ~15);
    ctx->ubox[1] = std::max(ctx->ubox[1], he);
  }
  for (auto& j : ctx->jobs) {
    int32_t b[3];
    job_box(j, b);
    max_region_bulk = std::max(max_region_bulk, ctx->ubox[0] * ctx->ubox[1] * b[2]);
  }
  if (room) max_region_bulk = std::max(max_region_bulk, ctx->ubox[0] * ctx->ubox[1] * he);
  ctx->cap_jobs = std::max<int32_t>(static_cast<int32_t>(ctx->jobs.size()), room ? ctx->cfg.max_jobs : 0);
  ctx->cap_blocks = std::max<int32_t>(nb, room ? static_cast<int32_t>(std::min<int64_t>(ctx->cfg.max_blocks, INT32_MAX)) : 0);
  ctx->cap_vac = std::max<int32_t>(nv, room ? static_cast<int32_t>(std::min<int64_t>(ctx->cfg.max_vacancies, INT32_MAX)) : 0);
  if (room && (ctx->cap_blocks < 1 || ctx->cap_vac < 1)) return fail(ctx, AKMC_EINVAL, "max_blocks and max_vacancies must be > 0");
  ctx->cap_pots = static_cast<int32_t>(ctx->pots.size()) + (room ? 16 : 0);
  int dev_smem = 0;
  CK(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->cfg.device));
  // bulk staging where its wider rows fit, else row loads everywhere
  ctx->bulk_ok = hop_smem_bytes(max_region_bulk) <= static_cast<size_t>(dev_smem);
  ctx->smem = hop_smem_bytes(ctx->bulk_ok ? max_region_bulk : max_region);
  if (ctx->smem > static_cast<size_t>(dev_smem))
    return fail(ctx, AKMC_EINVAL, "sector region does not fit in shared memory; use more domain blocks");
  {
    // The attribute belongs to the kernel, not to this context: set it to the device's
    // limit, so that another context with smaller regions cannot lower it under this one.
    const int e = configure_hop_smem(static_cast<size_t>(dev_smem));
    if (e) return fail(ctx, AKMC_ECUDA, std::string("cudaFuncSetAttribute: ") + cuda_name(e));
  }
  int sms = 148;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->cfg.device));
  int smem_sm = 0;
  CK(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, ctx->cfg.device));
  // CTAs resident per SM: as many as the registers allow (hop_ctas_per_sm) and two staged
  // regions (plus the 1 KB the SM reserves per CTA) fit; k_flow is persistent, one CTA per
  // slot.  k_hop also gets a second wave where two regions fit.
  const int fit = std::max(1, std::min(2, static_cast<int>(smem_sm / (ctx->smem + 1024))));
  const int resident = std::min(fit, hop_ctas_per_sm(ctx->cfg.eval_warps));
  const int32_t cb = ctx->cap_blocks;
  ctx->grid_sms = sms;
  ctx->grid_fit = fit;
  ctx->grid_resident = resident;

  // geometry and potentials
  Geometry geo;
  build_geometry(geo, 5);
  CK(dalloc(ctx->stream, &ctx->d_geo, 1));
  CK(cudaMemcpyAsync(ctx->d_geo, &geo, sizeof(geo), cudaMemcpyHostToDevice, ctx->stream));
  std::vector<Potential> hp(ctx->pots.size());
  for (size_t i = 0; i < ctx->pots.size(); ++i) {
    const akmc_status st = upload_pot(ctx, i, hp[i]);
    if (st != AKMC_OK) return st;
  }
  CK(dalloc(ctx->stream, &ctx->d_pots, static_cast<size_t>(ctx->cap_pots)));
  CK(cudaMemcpyAsync(ctx->d_pots, hp.data(), hp.size() * sizeof(Potential), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));  // hp leaves scope

  // jobs, blocks, vacancies; free slots as the kernels skip them
  std::vector<JobDev> hj(static_cast<size_t>(ctx->cap_jobs), free_job_record());
  std::vector<BlockDev> hb(static_cast<size_t>(cb), free_block_record());
  std::vector<int32_t> vsite(static_cast<size_t>(ctx->cap_vac), 0), vjob(static_cast<size_t>(ctx->cap_vac), -1);
  for (size_t ji = 0; ji < ctx->jobs.size(); ++ji) {
    HostJob& j = ctx->jobs[ji];
    const akmc_status st = setup_job(ctx, static_cast<int32_t>(ji), hj[ji], hb.data() + j.block0, vsite.data() + j.vac0,
                                     vjob.data() + j.vac0);
    if (st != AKMC_OK) return st;
  }
  ctx->free_blocks.clear();
  ctx->free_vac.clear();
  if (cb > nb) ctx->free_blocks.emplace_back(nb, cb);
  if (ctx->cap_vac > nv) ctx->free_vac.emplace_back(nv, ctx->cap_vac);
  const size_t ncap = static_cast<size_t>(cb);
  CK(dalloc(ctx->stream, &ctx->d_jobs, hj.size()));
  CK(dalloc(ctx->stream, &ctx->d_blocks, hb.size()));
  CK(dalloc(ctx->stream, &ctx->d_vac_site, vsite.size()));
  CK(dalloc(ctx->stream, &ctx->d_vac_job, vjob.size()));
  CK(dalloc(ctx->stream, &ctx->d_blk_list, ncap * kMaxV));
  CK(dalloc(ctx->stream, &ctx->d_active, ncap));
  CK(dalloc(ctx->stream, &ctx->d_n_active, 1));
  CK(dalloc(ctx->stream, &ctx->d_status, 1));
  CK(dalloc(ctx->stream, &ctx->d_counters, 24));
  CK(dalloc(ctx->stream, &ctx->d_vac_count, 1));
  CK(dalloc(ctx->stream, &ctx->d_fstate, ncap));
  CK(dalloc(ctx->stream, &ctx->d_vclaim, ncap));
  CK(dalloc(ctx->stream, &ctx->d_vvalid, ncap));
  CK(dalloc(ctx->stream, &ctx->d_vslot, ncap * kFlowSlots));
  CK(dalloc(ctx->stream, &ctx->d_vsite, ncap * kFlowSlots));
  CK(dalloc(ctx->stream, &ctx->d_vcount, ncap));
  CK(dalloc(ctx->stream, &ctx->d_nbr, ncap * kNbrStride));
  CK(dalloc(ctx->stream, &ctx->d_vsec, ncap));
  {
    // every job slot's two tensor maps (filled for the jobs added so far; admitted jobs later)
    std::vector<unsigned char> tm(static_cast<size_t>(ctx->cap_jobs) * 256, 0);
    for (size_t ji = 0; ji < ctx->jobs.size(); ++ji) std::memcpy(tm.data() + ji * 256, ctx->jobs[ji].tmap, 256);
    CK(dalloc(ctx->stream, &ctx->d_tmaps, tm.size()));
    CK(cudaMemcpyAsync(ctx->d_tmaps, tm.data(), tm.size(), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));  // tm leaves scope
  }
  CK(dalloc(ctx->stream, &ctx->d_flow, 6));
  CK(dalloc(ctx->stream, &ctx->d_log_count, 1));
  CK(dalloc(ctx->stream, &ctx->d_api_total, 1));
  CK(dalloc(ctx->stream, &ctx->d_api_event, 1));
  CK(dalloc(ctx->stream, &ctx->d_api_de, static_cast<size_t>(kMaxV) * 8));
  CK(dalloc(ctx->stream, &ctx->d_api_rates, static_cast<size_t>(kMaxV) * 8));
  CK(dalloc(ctx->stream, &ctx->d_api_sites, static_cast<size_t>(kMaxV)));
  CK(dalloc(ctx->stream, &ctx->d_api_count, 1));
  CK(cudaMemsetAsync(ctx->d_api_count, 0, sizeof(int32_t), ctx->stream));
  if (ctx->cfg.event_log_capacity > 0) CK(dalloc(ctx->stream, &ctx->d_log, static_cast<size_t>(ctx->cfg.event_log_capacity)));
  CK(cudaMemcpyAsync(ctx->d_jobs, hj.data(), hj.size() * sizeof(JobDev), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_blocks, hb.data(), hb.size() * sizeof(BlockDev), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_vac_site, vsite.data(), vsite.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_vac_job, vjob.data(), vjob.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(ctx->d_n_active, 0, 4, ctx->stream));
  CK(cudaMemsetAsync(ctx->d_status, 0, 4, ctx->stream));
  CK(cudaMemsetAsync(ctx->d_counters, 0, 192, ctx->stream));
  CK(cudaMemsetAsync(ctx->d_log_count, 0, 8, ctx->stream));
  CK(cudaMemsetAsync(ctx->d_fstate, 0, ncap * 8, ctx->stream));
  {  // density caches of every EAM job, one launch
    const akmc_status rt = build_rho_tables(ctx);
    if (rt != AKMC_OK) return rt;
    if (ctx->jl.neam > 0) {
      RoundArgs ra{};
      ra.jobs = ctx->d_jobs;
      ra.pots = ctx->d_pots;
      const int e = launch_init_rho_jobs(ra, ctx->jl, ctx->stream);
      if (e) return fail(ctx, AKMC_ECUDA, std::string("init rho: ") + cuda_name(e));
    }
  }
  RoundArgs& a = ctx->args;
  std::memset(&a, 0, sizeof(a));
  a.jobs = ctx->d_jobs;
  a.njobs = ctx->cap_jobs;
  a.nblocks = cb;
  a.blocks = ctx->d_blocks;
  a.vac_site = ctx->d_vac_site;
  a.vac_job = ctx->d_vac_job;
  a.nvac = ctx->cap_vac;
  a.mode = kModeRound;
  a.blk_list = ctx->d_blk_list;
  a.active = ctx->d_active;
  a.n_active = ctx->d_n_active;
  a.pots = ctx->d_pots;
  a.geo = ctx->d_geo;
  a.log = ctx->d_log;
  a.log_count = ctx->d_log_count;
  a.log_cap = ctx->cfg.event_log_capacity;
  a.status = ctx->d_status;
  a.counters = ctx->d_counters;
  a.hop_cap = ctx->cfg.hop_cap_per_round;
  a.flow_sweep_limit = ctx->cfg.flow_sweep_limit;
  a.api_job = -1;
  a.api_sector = -1;
  a.api_total = ctx->d_api_total;
  a.api_event = ctx->d_api_event;
  a.api_de = ctx->d_api_de;
  a.api_rates = ctx->d_api_rates;
  a.api_sites = ctx->d_api_sites;
  a.api_count = ctx->d_api_count;
  a.fstate = ctx->d_fstate;
  a.vclaim = ctx->d_vclaim;
  a.vvalid = ctx->d_vvalid;
  a.vslot = ctx->d_vslot;
  a.vsite = ctx->d_vsite;
  a.vcount = ctx->d_vcount;
  a.nbr = ctx->d_nbr;
  a.vsec = ctx->d_vsec;
  a.tmaps = ctx->d_tmaps;
  a.flow_need = ctx->d_flow;
  a.flow_done = ctx->d_flow + 3;
  a.flow_take = ctx->cfg.flow_take;
  a.eval_warps = ctx->cfg.eval_warps;
  refresh_job_set(ctx);
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->h_jobs = hj;
  ctx->h_blocks = hb;
  ctx->prepared = true;
  return AKMC_OK;
}

AKMC_API akmc_status akmc_admit_job(akmc_ctx* ctx, const akmc_job_config* cfg, const uint8_t* occ, int64_t n_sites,
                                    int32_t* job_id) {
  if (!ctx || !cfg || !occ) return AKMC_EINVAL;
  if (!ctx->prepared) return fail(ctx, AKMC_ESTATE, "akmc_admit_job needs a prepared context (akmc_add_job before it)");
  if (ctx->max_edge <= 0) return fail(ctx, AKMC_ESTATE, "the context was created without room for admitted jobs (max_jobs)");
  CK(cudaSetDevice(ctx->cfg.device));
  HostJob j;
  akmc_status st = check_job(ctx, cfg, occ, n_sites, j);
  if (st != AKMC_OK) return st;
  if (max_block_edge(j) > ctx->max_edge)
    return fail(ctx, AKMC_EINVAL, "domain blocks larger than the context's max_block_edge (" +
                                      std::to_string(ctx->max_edge) + " cells); use more blocks");
  int32_t slot = -1;
  for (size_t k = 0; k < ctx->jobs.size() && slot < 0; ++k)
    if (!ctx->jobs[k].live) slot = static_cast<int32_t>(k);
  if (slot < 0 && static_cast<int32_t>(ctx->jobs.size()) >= ctx->cap_jobs)
    return fail(ctx, AKMC_EBUSY, "no free job slot (max_jobs " + std::to_string(ctx->cap_jobs) + ")");
  j.block0 = take_range(ctx->free_blocks, j.nblocks);
  if (j.block0 < 0) return fail(ctx, AKMC_EBUSY, "no room for the job's domain blocks (max_blocks)");
  j.vac0 = take_range(ctx->free_vac, static_cast<int32_t>(j.nvac));
  if (j.vac0 < 0) {
    give_range(ctx->free_blocks, j.block0, j.nblocks);
    return fail(ctx, AKMC_EBUSY, "no room for the job's vacancies (max_vacancies)");
  }
  const size_t npots = ctx->pots.size();
  int rc = 0;
  j.pot = find_or_add_pot(ctx, j, &rc);
  if (j.pot < 0 || rc) {
    give_range(ctx->free_blocks, j.block0, j.nblocks);
    give_range(ctx->free_vac, j.vac0, static_cast<int32_t>(j.nvac));
    if (rc == -2) return fail(ctx, AKMC_ERANGE, "EAM densities can exceed the F table");
    return fail(ctx, rc ? AKMC_EINVAL : AKMC_EBUSY, rc ? "invalid EAM tables" : "no room for another potential");
  }
  if (ctx->pots.size() > npots) {
    Potential hp;
    st = upload_pot(ctx, npots, hp);
    if (st != AKMC_OK) return st;
    CK(cudaMemcpyAsync(ctx->d_pots + npots, &hp, sizeof(hp), cudaMemcpyHostToDevice, ctx->stream));
  }
  if (slot < 0) {
    slot = static_cast<int32_t>(ctx->jobs.size());
    ctx->jobs.emplace_back();
  }
  ctx->jobs[static_cast<size_t>(slot)] = std::move(j);
  HostJob& h = ctx->jobs[static_cast<size_t>(slot)];
  JobDev J;
  std::vector<BlockDev> hb(static_cast<size_t>(h.nblocks));
  std::vector<int32_t> vsite(static_cast<size_t>(h.nvac)), vjob(static_cast<size_t>(h.nvac));
  st = setup_job(ctx, slot, J, hb.data(), vsite.data(), vjob.data());
  if (st != AKMC_OK) return st;
  CK(cudaMemcpyAsync(ctx->d_tmaps + static_cast<size_t>(slot) * 256, h.tmap, 256, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_jobs + slot, &J, sizeof(J), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_blocks + h.block0, hb.data(), hb.size() * sizeof(BlockDev), cudaMemcpyHostToDevice,
                     ctx->stream));
  if (h.nvac) {
    CK(cudaMemcpyAsync(ctx->d_vac_site + h.vac0, vsite.data(), vsite.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->d_vac_job + h.vac0, vjob.data(), vjob.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
  }
  if (h.has_eam) {
    const int e = launch_init_rho(h.d_occ, h.d_rho, 2 * static_cast<int32_t>(h.cfg.box[0]),
                                  static_cast<int32_t>(h.cfg.box[1]), static_cast<int32_t>(h.cfg.box[2]),
                                  ctx->d_pots + h.pot, ctx->d_geo, ctx->d_status, ctx->stream);
    if (e) return fail(ctx, AKMC_ECUDA, std::string("init rho: ") + cuda_name(e));
  }
  ctx->h_jobs[static_cast<size_t>(slot)] = J;
  std::copy(hb.begin(), hb.end(), ctx->h_blocks.begin() + h.block0);
  refresh_job_set(ctx);
  drop_job_set_caches(ctx);
  CK(cudaStreamSynchronize(ctx->stream));  // the host records leave scope
  if (job_id) *job_id = slot;
  return AKMC_OK;
}

AKMC_API akmc_status akmc_retire_job(akmc_ctx* ctx, int32_t job) {
  if (!ctx) return AKMC_EINVAL;
  if (!ctx->prepared) return fail(ctx, AKMC_ESTATE, "akmc_prepare first");
  if (job < 0 || job >= static_cast<int32_t>(ctx->jobs.size()) || !ctx->jobs[static_cast<size_t>(job)].live)
    return AKMC_ENOTFOUND;
  CK(cudaSetDevice(ctx->cfg.device));
  HostJob& h = ctx->jobs[static_cast<size_t>(job)];
  const JobDev J = free_job_record();
  const std::vector<BlockDev> hb(static_cast<size_t>(h.nblocks), free_block_record());
  CK(cudaMemcpyAsync(ctx->d_jobs + job, &J, sizeof(J), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_blocks + h.block0, hb.data(), hb.size() * sizeof(BlockDev), cudaMemcpyHostToDevice,
                     ctx->stream));
  if (h.nvac) CK(cudaMemsetAsync(ctx->d_vac_job + h.vac0, 0xff, static_cast<size_t>(h.nvac) * 4, ctx->stream));
  dfree(ctx->stream, h.d_occ);
  dfree(ctx->stream, h.d_rho);
  h.d_occ = nullptr;
  h.d_rho = nullptr;
  ctx->h_jobs[static_cast<size_t>(job)] = J;
  std::copy(hb.begin(), hb.end(), ctx->h_blocks.begin() + h.block0);
  give_range(ctx->free_blocks, h.block0, h.nblocks);
  give_range(ctx->free_vac, h.vac0, static_cast<int32_t>(h.nvac));
  h.live = false;
  h.occ.clear();
  h.occ.shrink_to_fit();
  refresh_job_set(ctx);
  drop_job_set_caches(ctx);
  CK(cudaStreamSynchronize(ctx->stream));  // the host records leave scope
  return AKMC_OK;
}

AKMC_API akmc_status akmc_load_occupancy(akmc_ctx* ctx, int32_t job, const uint8_t* occ, int64_t n_sites) {
  if (!ctx || !occ) return AKMC_EINVAL;
  if (!ctx->prepared) return fail(ctx, AKMC_ESTATE, "akmc_prepare first");
  if (!live_job(ctx, job)) return AKMC_ENOTFOUND;
  HostJob& j = ctx->jobs[static_cast<size_t>(job)];
  if (n_sites != j.nsites) return fail(ctx, AKMC_EINVAL, "n_sites does not match the job");
  CK(cudaSetDevice(ctx->cfg.device));
  const int32_t sx = 2 * static_cast<int32_t>(j.cfg.box[0]);
  CK(lattice_upload(j.d_occ, occ, sx, j.cfg.box[1] * j.cfg.box[2], ctx->stream));
  int e = launch_collect_vacancies(j.d_occ, n_sites, sx, ctx->d_vac_site + j.vac0, ctx->d_vac_job + j.vac0, job,
                                   static_cast<int32_t>(j.nvac), ctx->d_vac_count, ctx->d_status, ctx->stream);
  if (e) return fail(ctx, AKMC_ECUDA, std::string("collect vacancies: ") + cuda_name(e));
  if (j.has_eam) {
    e = launch_init_rho(j.d_occ, j.d_rho, 2 * static_cast<int32_t>(j.cfg.box[0]), static_cast<int32_t>(j.cfg.box[1]),
                        static_cast<int32_t>(j.cfg.box[2]), ctx->d_pots + j.pot, ctx->d_geo, ctx->d_status,
                        ctx->stream);
    if (e) return fail(ctx, AKMC_ECUDA, std::string("init rho: ") + cuda_name(e));
  }
  CK(cudaMemcpyAsync(ctx->d_jobs + job, &ctx->h_jobs[static_cast<size_t>(job)], sizeof(JobDev), cudaMemcpyHostToDevice,
                     ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_blocks + j.block0, &ctx->h_blocks[static_cast<size_t>(j.block0)],
                     static_cast<size_t>(j.nblocks) * sizeof(BlockDev), cudaMemcpyHostToDevice, ctx->stream));
  return AKMC_OK;  // a wrong vacancy count is reported by the next synchronising call
}

AKMC_API akmc_status akmc_snapshot_size(akmc_ctx* ctx, int32_t job, int64_t* bytes) {
  if (!ctx || !bytes) return AKMC_EINVAL;
  if (!live_job(ctx, job)) return AKMC_ENOTFOUND;
  *bytes = snapshot_bytes(ctx->jobs[static_cast<size_t>(job)]);
  return AKMC_OK;
}

AKMC_API akmc_status akmc_save_snapshot(akmc_ctx* ctx, int32_t job, uint8_t* buf, int64_t capacity, int64_t* written) {
  if (!ctx || !buf || !written) return AKMC_EINVAL;
  *written = 0;
  if (!ctx->prepared) return fail(ctx, AKMC_ESTATE, "akmc_prepare first");
  if (!live_job(ctx, job)) return AKMC_ENOTFOUND;
  const HostJob& j = ctx->jobs[static_cast<size_t>(job)];
  const int64_t need = snapshot_bytes(j);
  if (capacity < need) return fail(ctx, AKMC_EINVAL, "snapshot needs " + std::to_string(need) + " bytes");
  CK(cudaSetDevice(ctx->cfg.device));
  JobDev J;
  std::vector<BlockDev> B(static_cast<size_t>(j.nblocks));
  uint8_t* occ = buf + sizeof(SnapHeader) + j.nblocks * sizeof(SnapBlock);
  CK(cudaMemcpyAsync(&J, ctx->d_jobs + job, sizeof(J), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(B.data(), ctx->d_blocks + j.block0, B.size() * sizeof(BlockDev), cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(lattice_download(occ, j.d_occ, 2 * j.cfg.box[0], j.cfg.box[1] * j.cfg.box[2], ctx->stream));
  const akmc_status st = akmc_sync(ctx);  // also the last run's errors
  if (st != AKMC_OK) return st;
  for (int32_t b = 0; b < j.nblocks; ++b) {
    SnapBlock r{};
    r.round = B[static_cast<size_t>(b)].round;
    r.hops = B[static_cast<size_t>(b)].hops;
    for (int k = 0; k < 8; ++k) r.evo[k] = B[static_cast<size_t>(b)].evo[k];
    for (int k = 0; k < 4; ++k) {
      r.xs[k] = B[static_cast<size_t>(b)].xs[k];
      r.xt[k] = B[static_cast<size_t>(b)].xt[k];
    }
    r.done = B[static_cast<size_t>(b)].done;
    std::memcpy(buf + sizeof(SnapHeader) + b * sizeof(SnapBlock), &r, sizeof(r));
  }
  SnapHeader h{};
  std::memcpy(h.magic, "AKMCSNAP", 8);
  h.version = kSnapVersion;
  h.header_bytes = sizeof(SnapHeader);
  for (int d = 0; d < 3; ++d) {
    h.box[d] = j.cfg.box[d];
    h.blocks[d] = j.cfg.blocks[d] > 0 ? j.cfg.blocks[d] : 1;
  }
  h.model = j.cfg.energy_model;
  h.precision = j.cfg.precision;
  h.rng = j.cfg.rng;
  h.lattice_const = j.cfg.lattice_const;
  h.cutoff = j.cfg.cutoff_radius;
  h.attempt_freq = j.cfg.attempt_freq;
  h.temperature = j.cfg.temperature;
  h.window = j.cfg.sector_window;
  h.seed = j.cfg.seed;
  h.eam_hash = eam_hash(j);
  h.round = J.round;
  h.hops = J.hops;
  h.done = J.done;
  h.nblocks = j.nblocks;
  h.nsites = j.nsites;
  h.nvac = j.nvac;
  h.checksum = fnv1a(buf + sizeof(SnapHeader), static_cast<size_t>(need) - sizeof(SnapHeader));
  std::memcpy(buf, &h, sizeof(h));
  *written = need;
  return AKMC_OK;
}

AKMC_API akmc_status akmc_restore_snapshot(akmc_ctx* ctx, int32_t job, const uint8_t* buf, int64_t n) {
  if (!ctx || !buf) return AKMC_EINVAL;
  if (!ctx->prepared) return fail(ctx, AKMC_ESTATE, "akmc_prepare first");
  if (!live_job(ctx, job)) return AKMC_ENOTFOUND;
  const HostJob& j = ctx->jobs[static_cast<size_t>(job)];
  SnapHeader h{};
  if (n < static_cast<int64_t>(sizeof(h))) return fail(ctx, AKMC_EINVAL, "not a snapshot: too short");
  std::memcpy(&h, buf, sizeof(h));
  if (std::memcmp(h.magic, "AKMCSNAP", 8) != 0 || h.header_bytes != sizeof(SnapHeader))
    return fail(ctx, AKMC_EINVAL, "not a snapshot");
  if (h.version != kSnapVersion) return fail(ctx, AKMC_EINVAL, "snapshot version " + std::to_string(h.version));
  if (n != snapshot_bytes(j) || h.nsites != j.nsites || h.nblocks != j.nblocks || h.nvac != j.nvac)
    return fail(ctx, AKMC_EINVAL, "snapshot of a job of another size");
  bool same = h.model == j.cfg.energy_model && h.precision == j.cfg.precision && h.rng == j.cfg.rng &&
              h.lattice_const == j.cfg.lattice_const && h.cutoff == j.cfg.cutoff_radius &&
              h.attempt_freq == j.cfg.attempt_freq && h.temperature == j.cfg.temperature &&
              h.window == j.cfg.sector_window && h.eam_hash == eam_hash(j);
  for (int d = 0; d < 3; ++d)
    same = same && h.box[d] == j.cfg.box[d] && h.blocks[d] == (j.cfg.blocks[d] > 0 ? j.cfg.blocks[d] : 1);
  if (!same) return fail(ctx, AKMC_EINVAL, "snapshot of another job configuration or potential");
  if (fnv1a(buf + sizeof(h), static_cast<size_t>(n) - sizeof(h)) != h.checksum)
    return fail(ctx, AKMC_EINVAL, "snapshot checksum mismatch");
  const uint8_t* occ = buf + sizeof(h) + j.nblocks * sizeof(SnapBlock);
  // the lattice, its vacancy table and density cache, and the initial records ...
  akmc_status st = akmc_load_occupancy(ctx, job, occ, j.nsites);
  if (st != AKMC_OK) return st;
  // ... then the saved counters, clocks and random streams over them
  JobDev J = ctx->h_jobs[static_cast<size_t>(job)];
  J.round = h.round;
  J.hops = h.hops;
  J.done = h.done;
  std::vector<BlockDev> B(ctx->h_blocks.begin() + j.block0, ctx->h_blocks.begin() + j.block0 + j.nblocks);
  for (int32_t b = 0; b < j.nblocks; ++b) {
    SnapBlock r;
    std::memcpy(&r, buf + sizeof(h) + b * sizeof(SnapBlock), sizeof(r));
    BlockDev& d = B[static_cast<size_t>(b)];
    d.round = r.round;
    d.hops = r.hops;
    for (int k = 0; k < 8; ++k) d.evo[k] = r.evo[k];
    for (int k = 0; k < 4; ++k) {
      d.xs[k] = r.xs[k];
      d.xt[k] = r.xt[k];
    }
    d.done = r.done;
    d.cnt = 0;
  }
  CK(cudaMemcpyAsync(ctx->d_jobs + job, &J, sizeof(J), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_blocks + j.block0, B.data(), B.size() * sizeof(BlockDev), cudaMemcpyHostToDevice,
                     ctx->stream));
  return akmc_sync(ctx);  // B and J leave scope; also reports a lattice with a wrong vacancy count
}

// Density tiles of the EAM jobs (prefix over jobs) for the one-launch density build.
static akmc_status build_rho_tables(akmc_ctx* ctx) {
  if (ctx->d_tile0) return AKMC_OK;
  std::vector<int32_t> eam_jobs;
  std::vector<int64_t> tile0{0};
  for (size_t k = 0; k < ctx->jobs.size(); ++k) {
    const HostJob& j = ctx->jobs[k];
    if (!j.has_eam || !j.live) continue;
    const int64_t sx = 2 * j.cfg.box[0], sy = j.cfg.box[1], sz = j.cfg.box[2];
    eam_jobs.push_back(static_cast<int32_t>(k));
    tile0.push_back(tile0.back() + ((sx + 31) / 32) * ((sy + 7) / 8) * ((sz + 3) / 4));
  }
  CK(dalloc(ctx->stream, &ctx->d_tile0, tile0.size()));
  CK(dalloc(ctx->stream, &ctx->d_eam_jobs, std::max<size_t>(1, eam_jobs.size())));
  CK(cudaMemcpy(ctx->d_tile0, tile0.data(), tile0.size() * sizeof(int64_t), cudaMemcpyHostToDevice));
  if (!eam_jobs.empty())
    CK(cudaMemcpy(ctx->d_eam_jobs, eam_jobs.data(), eam_jobs.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  ctx->jl.tile0 = ctx->d_tile0;
  ctx->jl.eam_jobs = ctx->d_eam_jobs;
  ctx->jl.neam = static_cast<int32_t>(eam_jobs.size());
  ctx->jl.eam_tiles = tile0.back();
  return AKMC_OK;
}

// Tables of the whole-context transfers, built once after akmc_prepare.
static akmc_status setup_jobs_load(akmc_ctx* ctx) {
  if (ctx->d_stage) return AKMC_OK;
  const akmc_status rt = build_rho_tables(ctx);
  if (rt != AKMC_OK) return rt;
  constexpr int64_t kChunk = 1 << 16;
  std::vector<SiteChunk> ch;
  std::vector<int32_t> want;
  int64_t off = 0;
  for (size_t k = 0; k < ctx->jobs.size(); ++k) {
    const HostJob& j = ctx->jobs[k];
    if (!j.live) {  // a retired slot: no sites, and no vacancies expected
      want.push_back(0);
      continue;
    }
    for (int64_t s0 = 0; s0 < j.nsites; s0 += kChunk) {
      SiteChunk c{};
      c.job = static_cast<int32_t>(k);
      c.vac0 = j.vac0;
      c.nvac = static_cast<int32_t>(j.nvac);
      c.site0 = s0;
      c.n = std::min(kChunk, j.nsites - s0);
      c.stage0 = off + s0;
      ch.push_back(c);
    }
    off += j.nsites;
    want.push_back(static_cast<int32_t>(j.nvac));
  }
  if (ch.size() > static_cast<size_t>(INT32_MAX)) return fail(ctx, AKMC_EINVAL, "too many sites");
  CK(dalloc(ctx->stream, &ctx->d_stage, static_cast<size_t>(off)));
  CK(dalloc(ctx->stream, &ctx->d_chunks, ch.size()));
  CK(dalloc(ctx->stream, &ctx->d_job_counts, want.size()));
  CK(dalloc(ctx->stream, &ctx->d_job_want, want.size()));
  CK(cudaMemcpy(ctx->d_chunks, ch.data(), ch.size() * sizeof(SiteChunk), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->d_job_want, want.data(), want.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  JobsLoad& L = ctx->jl;
  L.stage = ctx->d_stage;
  L.chunks = ctx->d_chunks;
  L.nchunks = static_cast<int32_t>(ch.size());
  L.njobs = static_cast<int32_t>(want.size());
  L.counts = ctx->d_job_counts;
  L.want = ctx->d_job_want;
  ctx->total_sites = off;
  return AKMC_OK;
}

AKMC_API akmc_status akmc_load_occupancies(akmc_ctx* ctx, const uint8_t* occ, int64_t total_sites) {
  if (!ctx || !occ) return AKMC_EINVAL;
  if (!ctx->prepared) return fail(ctx, AKMC_ESTATE, "akmc_prepare first");
  CK(cudaSetDevice(ctx->cfg.device));
  const akmc_status st = setup_jobs_load(ctx);
  if (st != AKMC_OK) return st;
  if (total_sites != ctx->total_sites) return fail(ctx, AKMC_EINVAL, "total_sites must be the sum of the jobs' sites");
  CK(cudaMemcpyAsync(ctx->d_stage, occ, static_cast<size_t>(total_sites), cudaMemcpyHostToDevice, ctx->stream));
  const int e = launch_load_jobs(ctx->args, ctx->jl, ctx->stream);
  if (e) return fail(ctx, AKMC_ECUDA, std::string("load: ") + cuda_name(e));
  CK(cudaMemcpyAsync(ctx->d_jobs, ctx->h_jobs.data(), ctx->h_jobs.size() * sizeof(JobDev), cudaMemcpyHostToDevice,
                     ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_blocks, ctx->h_blocks.data(), ctx->h_blocks.size() * sizeof(BlockDev),
                     cudaMemcpyHostToDevice, ctx->stream));
  return AKMC_OK;  // a wrong vacancy count is reported by the next synchronising call
}

AKMC_API akmc_status akmc_get_occupancies(akmc_ctx* ctx, uint8_t* out, int64_t total_sites) {
  if (!ctx || !out) return AKMC_EINVAL;
  if (!ctx->prepared) return fail(ctx, AKMC_ESTATE, "akmc_prepare first");
  CK(cudaSetDevice(ctx->cfg.device));
  const akmc_status st = setup_jobs_load(ctx);
  if (st != AKMC_OK) return st;
  if (total_sites != ctx->total_sites) return fail(ctx, AKMC_EINVAL, "total_sites must be the sum of the jobs' sites");
  const int e = launch_gather_jobs(ctx->args, ctx->jl, ctx->stream);
  if (e) return fail(ctx, AKMC_ECUDA, std::string("gather: ") + cuda_name(e));
  CK(cudaMemcpyAsync(out, ctx->d_stage, static_cast<size_t>(total_sites), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return AKMC_OK;
}

AKMC_API akmc_status akmc_set_kernel_timing(akmc_ctx* ctx, int32_t enable) {
  if (!ctx) return AKMC_EINVAL;
  ctx->timing = enable != 0;
  ctx->hop_ms = 0.0;
  ctx->hop_launches = 0;
  return AKMC_OK;
}

AKMC_API akmc_status akmc_get_kernel_timing(akmc_ctx* ctx, double* hop_kernel_ms, int64_t* hop_launches) {
  if (!ctx || !hop_kernel_ms || !hop_launches) return AKMC_EINVAL;
  *hop_kernel_ms = ctx->hop_ms;
  *hop_launches = ctx->hop_launches;
  return AKMC_OK;
}

AKMC_API akmc_status akmc_run_rounds(akmc_ctx* ctx, int64_t n_rounds) {
  if (!ctx) return AKMC_EINVAL;
  if (!ctx->prepared) return fail(ctx, AKMC_ESTATE, "akmc_prepare first");
  if (n_rounds <= 0) return AKMC_OK;
  CK(cudaSetDevice(ctx->cfg.device));
  RoundArgs a = ctx->args;
  a.mode = kModeRound;
  const bool flow = ctx->schedule == AKMC_SCHEDULE_FLOW || (ctx->schedule == AKMC_SCHEDULE_AUTO && ctx->flow_ok);
  if (flow) {
    // up to 1024 rounds per launch of the persistent flow kernels
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ctx->timing) {
      while (ctx->ev.size() < 2) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        ctx->ev.push_back(e);
      }
      e0 = ctx->ev[0];
      e1 = ctx->ev[1];
    }
    // each block runs n_rounds (fewer if its job ends: hop budgets are checked by the kernel at
    // time-step boundaries), up to 1024 per launch
    {
      const int e = launch_flow_begin(a, n_rounds, ctx->stream);
      if (e) return fail(ctx, AKMC_ECUDA, std::string("launch: ") + cuda_name(e));
    }
    const int64_t per = 1024;
    const int64_t launches = (n_rounds + per - 1) / per;
    for (int64_t k = 0; k < launches; ++k) {
      a.flow_rounds = per;
      const int e = launch_flow(a, ctx->flow_grid, ctx->smem, ctx->stream, e0, e1);
      if (e) return fail(ctx, AKMC_ECUDA, std::string("launch: ") + cuda_name(e));
      if (ctx->timing) {
        CK(cudaStreamSynchronize(ctx->stream));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        ctx->hop_ms += ms;
        ctx->hop_launches += 1;
      }
    }
    return AKMC_OK;
  }
  if (ctx->timing) {
    // one launch sequence per round, events around every hop kernel
    const size_t pool = 512;
    while (ctx->ev.size() < 2 * pool) {
      cudaEvent_t e;
      CK(cudaEventCreate(&e));
      ctx->ev.push_back(e);
    }
    int64_t left = n_rounds;
    while (left > 0) {
      const int64_t n = std::min<int64_t>(left, static_cast<int64_t>(pool));
      for (int64_t r = 0; r < n; ++r) {
        const int e = launch_round(a, ctx->hop_grid, ctx->smem, ctx->stream, ctx->ev[2 * r], ctx->ev[2 * r + 1]);
        if (e) return fail(ctx, AKMC_ECUDA, std::string("launch: ") + cuda_name(e));
      }
      CK(cudaStreamSynchronize(ctx->stream));
      for (int64_t r = 0; r < n; ++r) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ctx->ev[2 * r], ctx->ev[2 * r + 1]));
        ctx->hop_ms += ms;
        ctx->hop_launches += 1;
      }
      left -= n;
    }
    return AKMC_OK;
  }
  const int chunk = ctx->cfg.graph_rounds;
  if (n_rounds >= chunk && !ctx->graph) {
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    int e = 0;
    for (int r = 0; r < chunk && !e; ++r) e = launch_round(a, ctx->hop_grid, ctx->smem, ctx->stream, nullptr, nullptr);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &g);
    if (e || ce != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return fail(ctx, AKMC_ECUDA, std::string("graph capture: ") + cuda_name(e ? e : ce));
    }
    const cudaError_t ie = cudaGraphInstantiate(&ctx->graph, g, 0);
    if (ie != cudaSuccess) {
      cudaGraphDestroy(g);
      return fail(ctx, AKMC_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
    }
    ctx->graph_def = g;
    ctx->graph_rounds = chunk;
  }
  int64_t left = n_rounds;
  while (ctx->graph && left >= ctx->graph_rounds) {
    CK(cudaGraphLaunch(ctx->graph, ctx->stream));
    left -= ctx->graph_rounds;
  }
  for (; left > 0; --left) {
    const int e = launch_round(a, ctx->hop_grid, ctx->smem, ctx->stream, nullptr, nullptr);
    if (e) return fail(ctx, AKMC_ECUDA, std::string("launch: ") + cuda_name(e));
  }
  return AKMC_OK;
}

AKMC_API akmc_status akmc_run_for(akmc_ctx* ctx, int64_t n_rounds, int64_t max_us) {
  if (!ctx) return AKMC_EINVAL;
  if (!ctx->prepared) return fail(ctx, AKMC_ESTATE, "akmc_prepare first");
  if (n_rounds <= 0) return AKMC_OK;
  if (max_us <= 0) return fail(ctx, AKMC_EINVAL, "max_us must be > 0");
  const bool flow = ctx->schedule == AKMC_SCHEDULE_FLOW || (ctx->schedule == AKMC_SCHEDULE_AUTO && ctx->flow_ok);
  if (!flow) return akmc_run_rounds(ctx, std::min<int64_t>(n_rounds, ctx->cfg.graph_rounds));
  CK(cudaSetDevice(ctx->cfg.device));
  RoundArgs a = ctx->args;
  a.mode = kModeRound;
  a.flow_rounds = n_rounds;
  a.time_budget_ns = max_us * 1000;
  int e = launch_flow_begin(a, n_rounds, ctx->stream);
  if (!e) e = launch_flow(a, ctx->flow_grid, ctx->smem, ctx->stream, nullptr, nullptr);
  if (e) return fail(ctx, AKMC_ECUDA, std::string("launch: ") + cuda_name(e));
  return AKMC_OK;
}

namespace {
// Per-device address of the fixed round scratch, looked up on the first call with the device current.
constexpr int kNoAllocDevices = 64;
std::mutex g_noalloc_mu;
int32_t* g_noalloc_base[kNoAllocDevices] = {};
}  // namespace

AKMC_API akmc_status akmc_run_rounds_noalloc(akmc_ctx* ctx, int64_t n_rounds) {
  if (!ctx) return AKMC_EINVAL;
  if (!ctx->prepared) return fail(ctx, AKMC_ESTATE, "akmc_prepare first");
  if (ctx->nblocks > kNoAllocMaxBlocks)
    return fail(ctx, AKMC_EINVAL, "akmc_run_rounds_noalloc: " + std::to_string(ctx->nblocks) +
                                      " domain blocks exceed AKMC_NOALLOC_MAX_BLOCKS (" +
                                      std::to_string(kNoAllocMaxBlocks) + ")");
  const int dev = ctx->cfg.device;
  if (dev < 0 || dev >= kNoAllocDevices)
    return fail(ctx, AKMC_EINVAL, "akmc_run_rounds_noalloc: device index beyond " + std::to_string(kNoAllocDevices));
  if (n_rounds <= 0) return AKMC_OK;
  CK(cudaSetDevice(dev));
  int32_t* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_base[dev]) {
      const int e = noalloc_scratch(&g_noalloc_base[dev]);
      if (e) return fail(ctx, AKMC_ECUDA, std::string("cudaGetSymbolAddress(round scratch): ") + cuda_name(e));
    }
    base = g_noalloc_base[dev];
  }
  RoundArgs a = ctx->args;
  a.mode = kModeRound;
  a.blk_list = base;
  a.active = base + static_cast<size_t>(kNoAllocMaxBlocks) * kMaxV;
  a.n_active = a.active + kNoAllocMaxBlocks;
  // k_bucket appends to the active list from a zero count (k_finalize re-zeroes it each
  // round); the block lists and the active list are written before they are read.
  CK(cudaMemsetAsync(a.n_active, 0, sizeof(int32_t), ctx->stream));
  for (int64_t r = 0; r < n_rounds; ++r) {
    const int e = launch_round(a, ctx->hop_grid, ctx->smem, ctx->stream, nullptr, nullptr);
    if (e) return fail(ctx, AKMC_ECUDA, std::string("launch: ") + cuda_name(e));
  }
  return AKMC_OK;
}

AKMC_API akmc_status akmc_set_round_schedule(akmc_ctx* ctx, int32_t schedule) {
  if (!ctx) return AKMC_EINVAL;
  if (schedule < AKMC_SCHEDULE_AUTO || schedule > AKMC_SCHEDULE_FLOW)
    return fail(ctx, AKMC_EINVAL, "schedule: AKMC_SCHEDULE_AUTO, _ROUNDS or _FLOW");
  ctx->schedule = schedule;
  return AKMC_OK;
}

AKMC_API akmc_status akmc_get_round_schedule(akmc_ctx* ctx, int32_t* effective) {
  if (!ctx || !effective) return AKMC_EINVAL;
  if (!ctx->prepared) return fail(ctx, AKMC_ESTATE, "akmc_prepare first");
  const bool flow = ctx->schedule == AKMC_SCHEDULE_FLOW || (ctx->schedule == AKMC_SCHEDULE_AUTO && ctx->flow_ok);
  *effective = flow ? AKMC_SCHEDULE_FLOW : AKMC_SCHEDULE_ROUNDS;
  return AKMC_OK;
}

AKMC_API akmc_status akmc_sync(akmc_ctx* ctx) {
  if (!ctx) return AKMC_EINVAL;
  if (!ctx->prepared) return AKMC_OK;
  CK(cudaStreamSynchronize(ctx->stream));
  return check_status(ctx);
}

AKMC_API akmc_status akmc_gpu_final(akmc_ctx* ctx) { return akmc_sync(ctx); }

AKMC_API akmc_status akmc_run(akmc_ctx* ctx, int64_t max_rounds) {
  if (!ctx) return AKMC_EINVAL;
  if (!ctx->prepared) return fail(ctx, AKMC_ESTATE, "akmc_prepare first");
  std::vector<JobDev> hj(ctx->jobs.size());
  int64_t done_rounds = 0;
  const int64_t step = std::max<int64_t>(ctx->cfg.graph_rounds, 1);
  while (max_rounds <= 0 || done_rounds < max_rounds) {
    const int64_t n = max_rounds > 0 ? std::min(step, max_rounds - done_rounds) : step;
    akmc_status s = akmc_run_rounds(ctx, n);
    if (s) return s;
    done_rounds += n;
    CK(cudaMemcpyAsync(hj.data(), ctx->d_jobs, hj.size() * sizeof(JobDev), cudaMemcpyDeviceToHost, ctx->stream));
    s = akmc_sync(ctx);
    if (s) return s;
    bool all = true;
    for (auto& J : hj) all = all && J.done;
    if (all) break;
  }
  return AKMC_OK;
}

AKMC_API akmc_status akmc_get_job_state(akmc_ctx* ctx, int32_t job, akmc_job_state* st) {
  if (!ctx || !st) return AKMC_EINVAL;
  if (!live_job(ctx, job)) return AKMC_ENOTFOUND;
  const HostJob& j = ctx->jobs[static_cast<size_t>(job)];
  std::memset(st, 0, sizeof(*st));
  st->n_blocks = j.nblocks;
  st->n_sites = j.nsites;
  st->n_vacancies = j.nvac;
  if (!ctx->prepared) return AKMC_OK;
  JobDev J;
  CK(cudaMemcpyAsync(&J, ctx->d_jobs + job, sizeof(J), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  st->round = J.round;
  st->hops = J.hops;
  st->done = J.done;
  return AKMC_OK;
}

AKMC_API akmc_status akmc_get_job_states(akmc_ctx* ctx, akmc_job_state* out, int32_t n_jobs) {
  if (!ctx || (!out && n_jobs > 0)) return AKMC_EINVAL;
  if (n_jobs != static_cast<int32_t>(ctx->jobs.size()))
    return fail(ctx, AKMC_EINVAL, "n_jobs must equal the context's job count");
  if (n_jobs == 0) return AKMC_OK;
  std::vector<JobDev> J(static_cast<size_t>(n_jobs));
  if (ctx->prepared) {
    CK(cudaSetDevice(ctx->cfg.device));
    CK(cudaMemcpyAsync(J.data(), ctx->d_jobs, J.size() * sizeof(JobDev), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  for (int32_t k = 0; k < n_jobs; ++k) {
    const HostJob& j = ctx->jobs[static_cast<size_t>(k)];
    akmc_job_state& st = out[k];
    std::memset(&st, 0, sizeof(st));
    st.n_blocks = j.nblocks;
    st.n_sites = j.nsites;
    st.n_vacancies = j.nvac;
    if (ctx->prepared) {
      st.round = J[static_cast<size_t>(k)].round;
      st.hops = J[static_cast<size_t>(k)].hops;
      st.done = J[static_cast<size_t>(k)].done;
    }
  }
  return AKMC_OK;
}

AKMC_API akmc_status akmc_get_occupancy(akmc_ctx* ctx, int32_t job, uint8_t* out, int64_t n_sites) {
  if (!ctx || !out) return AKMC_EINVAL;
  if (!live_job(ctx, job)) return AKMC_ENOTFOUND;
  const HostJob& j = ctx->jobs[static_cast<size_t>(job)];
  if (n_sites != j.nsites) return AKMC_EINVAL;
  if (!ctx->prepared) {
    std::memcpy(out, j.occ.data(), static_cast<size_t>(n_sites));
    return AKMC_OK;
  }
  CK(lattice_download(out, j.d_occ, 2 * j.cfg.box[0], j.cfg.box[1] * j.cfg.box[2], ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return AKMC_OK;
}

AKMC_API akmc_status akmc_get_rho(akmc_ctx* ctx, int32_t job, int32_t* out, int64_t n_sites) {
  if (!ctx || !out) return AKMC_EINVAL;
  if (!live_job(ctx, job)) return AKMC_ENOTFOUND;
  const HostJob& j = ctx->jobs[static_cast<size_t>(job)];
  if (n_sites != j.nsites || !j.has_eam) return AKMC_EINVAL;
  if (!ctx->prepared) return fail(ctx, AKMC_ESTATE, "akmc_prepare first");
  CK(lattice_download(out, j.d_rho, 2 * j.cfg.box[0], j.cfg.box[1] * j.cfg.box[2], ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return AKMC_OK;
}

AKMC_API akmc_status akmc_get_block_clocks(akmc_ctx* ctx, int32_t job, double* evo, int64_t* hops, int32_t n_blocks) {
  if (!ctx || !evo || !hops) return AKMC_EINVAL;
  if (!live_job(ctx, job)) return AKMC_ENOTFOUND;
  const HostJob& j = ctx->jobs[static_cast<size_t>(job)];
  if (n_blocks != j.nblocks) return AKMC_EINVAL;
  if (!ctx->prepared) return fail(ctx, AKMC_ESTATE, "akmc_prepare first");
  std::vector<BlockDev> hb(static_cast<size_t>(j.nblocks));
  CK(cudaMemcpyAsync(hb.data(), ctx->d_blocks + j.block0, hb.size() * sizeof(BlockDev), cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  for (int b = 0; b < j.nblocks; ++b) {
    for (int k = 0; k < 8; ++k) evo[b * 8 + k] = hb[static_cast<size_t>(b)].evo[k];
    hops[b] = hb[static_cast<size_t>(b)].hops;
  }
  return AKMC_OK;
}

AKMC_API akmc_status akmc_get_events(akmc_ctx* ctx, akmc_event* out, int64_t capacity, int64_t* n_out) {
  if (!ctx || !n_out) return AKMC_EINVAL;
  *n_out = 0;
  if (!ctx->prepared || !ctx->d_log) return AKMC_OK;
  unsigned long long n = 0;
  CK(cudaMemcpyAsync(&n, ctx->d_log_count, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  const int64_t avail = std::min<int64_t>(static_cast<int64_t>(n), ctx->cfg.event_log_capacity);
  const int64_t m = std::min<int64_t>(avail, capacity);
  if (m > 0 && out)
    CK(cudaMemcpyAsync(out, ctx->d_log, static_cast<size_t>(m) * sizeof(akmc_event), cudaMemcpyDeviceToHost,
                       ctx->stream));
  CK(cudaMemsetAsync(ctx->d_log_count, 0, 8, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  *n_out = m;
  if (static_cast<int64_t>(n) > ctx->cfg.event_log_capacity) return fail(ctx, AKMC_EOVERFLOW, "event log overflowed");
  return AKMC_OK;
}

AKMC_API akmc_status akmc_get_phase_cycles(akmc_ctx* ctx, int64_t* out16) {
  if (!ctx || !out16) return AKMC_EINVAL;
  for (int i = 0; i < 16; ++i) out16[i] = 0;
  if (!ctx->prepared) return AKMC_OK;
  unsigned long long c[16];
  CK(cudaMemcpyAsync(c, ctx->d_counters + 8, sizeof(c), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < 16; ++i) out16[i] = static_cast<int64_t>(c[i]);
  return AKMC_OK;
}

AKMC_API akmc_status akmc_get_counters(akmc_ctx* ctx, int64_t* out8) {
  if (!ctx || !out8) return AKMC_EINVAL;
  if (!ctx->prepared) {
    for (int i = 0; i < 8; ++i) out8[i] = 0;
    return AKMC_OK;
  }
  unsigned long long c[8];
  CK(cudaMemcpyAsync(c, ctx->d_counters, sizeof(c), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < 8; ++i) out8[i] = static_cast<int64_t>(c[i]);
  return AKMC_OK;
}

static akmc_status api_step(akmc_ctx* ctx, int32_t job, int32_t sector_id, int32_t mode, double u) {
  if (!ctx->prepared) return fail(ctx, AKMC_ESTATE, "akmc_prepare first");
  if (!live_job(ctx, job)) return AKMC_ENOTFOUND;
  if (ctx->jobs[static_cast<size_t>(job)].nblocks != 1)
    return fail(ctx, AKMC_EINVAL, "the per-hop entry points drive single-domain jobs");
  if (sector_id < 0 || sector_id > 7) return fail(ctx, AKMC_EINVAL, "sector id in [0, 7]");
  CK(cudaSetDevice(ctx->cfg.device));
  RoundArgs a = ctx->args;
  a.mode = mode;
  a.api_job = job;
  a.api_sector = sector_id;
  a.api_u = u;
  a.log_cap = 0;
  const int e = launch_api(a, ctx->smem, ctx->stream);
  if (e) return fail(ctx, AKMC_ECUDA, std::string("launch: ") + cuda_name(e));
  return AKMC_OK;
}

AKMC_API akmc_status akmc_calculate(akmc_ctx* ctx, int32_t job, int32_t sector_id, double* total) {
  if (!ctx || !total) return AKMC_EINVAL;
  akmc_status s = api_step(ctx, job, sector_id, kModeCalc, 0.0);
  if (s) return s;
  CK(cudaMemcpyAsync(total, ctx->d_api_total, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  return akmc_sync(ctx);
}

AKMC_API akmc_status akmc_get_calculated_rates(akmc_ctx* ctx, int32_t* sites, double* delta_e, double* rates,
                                               int64_t capacity, int64_t* n_out) {
  if (!ctx || !n_out || capacity < 0 || (capacity > 0 && (!sites || !delta_e || !rates))) return AKMC_EINVAL;
  *n_out = 0;
  if (!ctx->prepared) return fail(ctx, AKMC_ESTATE, "akmc_prepare first");
  CK(cudaSetDevice(ctx->cfg.device));
  int32_t n = 0;
  CK(cudaMemcpyAsync(&n, ctx->d_api_count, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  *n_out = n;
  if (n > capacity) return fail(ctx, AKMC_EINVAL, "capacity below the sector's vacancy count");
  if (n == 0) return AKMC_OK;
  CK(cudaMemcpyAsync(sites, ctx->d_api_sites, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(delta_e, ctx->d_api_de, sizeof(double) * 8 * n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(rates, ctx->d_api_rates, sizeof(double) * 8 * n, cudaMemcpyDeviceToHost, ctx->stream));
  return akmc_sync(ctx);
}

AKMC_API akmc_status akmc_select_and_perform(akmc_ctx* ctx, int32_t job, int32_t sector_id, double u,
                                             akmc_event* ev) {
  if (!ctx || !ev) return AKMC_EINVAL;
  akmc_status s = api_step(ctx, job, sector_id, kModeSelectPerform, u);
  if (s) return s;
  CK(cudaMemcpyAsync(ev, ctx->d_api_event, sizeof(akmc_event), cudaMemcpyDeviceToHost, ctx->stream));
  return akmc_sync(ctx);
}

AKMC_API akmc_status akmc_eam_johnson(uint64_t seed, double lattice_const, double cutoff_radius,
                                      akmc_eam_tables* out) {
  if (!out) return AKMC_EINVAL;
  return eam_johnson(seed, lattice_const, cutoff_radius, out, nullptr) ? AKMC_EINVAL : AKMC_OK;
}

AKMC_API akmc_status akmc_create_lattice(const int64_t box[3], const int32_t type_codes[4], const int64_t ratio[4],
                                         int64_t n_vacancies, uint64_t seed, uint8_t* occ, int64_t n_sites) {
  if (!box || !type_codes || !ratio || !occ) return AKMC_EINVAL;
  return create_lattice(box, type_codes, ratio, n_vacancies, seed, occ, n_sites) ? AKMC_EINVAL : AKMC_OK;
}

AKMC_API akmc_status akmc_cluster_stats(const uint8_t* occ, const int64_t box[3], int64_t* isolated_cu, int64_t* hist,
                                        int64_t hist_len) {
  if (!occ || !box || !isolated_cu || (!hist && hist_len > 0)) return AKMC_EINVAL;
  return cluster_stats(occ, box, isolated_cu, hist, hist_len) ? AKMC_EINVAL : AKMC_OK;
}

AKMC_API akmc_status akmc_job_cluster_stats(akmc_ctx* ctx, int32_t job, int64_t* isolated_cu, int64_t* hist,
                                            int64_t hist_len) {
  if (!ctx || !isolated_cu || hist_len < 0 || hist_len > AKMC_CLUSTER_MAX_BINS || (hist_len > 0 && !hist))
    return AKMC_EINVAL;
  if (!ctx->prepared) return fail(ctx, AKMC_ESTATE, "akmc_prepare first");
  if (!live_job(ctx, job)) return AKMC_ENOTFOUND;
  const HostJob& j = ctx->jobs[static_cast<size_t>(job)];
  CK(cudaSetDevice(ctx->cfg.device));
  if (ctx->cl_sites < j.nsites) {
    CK(cudaStreamSynchronize(ctx->stream));
    dfree(ctx->stream, ctx->d_cl);
    ctx->d_cl = nullptr;
    ctx->cl_sites = 0;
    CK(dalloc(ctx->stream, &ctx->d_cl, static_cast<size_t>(3 * j.nsites)));
    ctx->cl_sites = j.nsites;
  }
  if (!ctx->d_cl_misc) CK(dalloc(ctx->stream, &ctx->d_cl_misc, 2 + AKMC_CLUSTER_MAX_BINS));
  ClusterArgs c{};
  c.occ = j.d_occ;
  c.ns = j.nsites;
  c.sx = 2 * static_cast<int32_t>(j.cfg.box[0]);
  c.px = lattice_pitch(c.sx);
  c.sy = static_cast<int32_t>(j.cfg.box[1]);
  c.sz = static_cast<int32_t>(j.cfg.box[2]);
  c.bins = hist_len > 0 ? static_cast<int32_t>(hist_len) : 1;
  c.list = ctx->d_cl;
  c.parent = ctx->d_cl + j.nsites;
  c.size = ctx->d_cl + 2 * j.nsites;
  c.n_list = reinterpret_cast<unsigned int*>(ctx->d_cl_misc);
  c.iso = ctx->d_cl_misc + 1;
  c.hist = ctx->d_cl_misc + 2;
  c.status = ctx->d_status;
  const int e = launch_cluster_stats(c, ctx->stream);
  if (e) return fail(ctx, AKMC_ECUDA, std::string("launch: ") + cuda_name(e));
  std::vector<unsigned long long> h(static_cast<size_t>(1 + c.bins));
  CK(cudaMemcpyAsync(h.data(), c.iso, sizeof(unsigned long long) * h.size(), cudaMemcpyDeviceToHost, ctx->stream));
  const akmc_status st = akmc_sync(ctx);
  if (st != AKMC_OK) return st;
  *isolated_cu = static_cast<int64_t>(h[0]);
  for (int64_t k = 0; k < hist_len; ++k) hist[k] = static_cast<int64_t>(h[static_cast<size_t>(1 + k)]);
  return AKMC_OK;
}

AKMC_API akmc_status akmc_device_math(akmc_ctx* ctx, const double* x, int64_t n, double* exp_out, double* log_out) {
  if (!ctx || !x || !exp_out || !log_out || n <= 0) return AKMC_EINVAL;
  CK(cudaSetDevice(ctx->cfg.device));
  double *dx = nullptr, *de = nullptr, *dl = nullptr;
  CK(dalloc(ctx->stream, &dx, static_cast<size_t>(n)));
  CK(dalloc(ctx->stream, &de, static_cast<size_t>(n)));
  CK(dalloc(ctx->stream, &dl, static_cast<size_t>(n)));
  cudaMemcpyAsync(dx, x, static_cast<size_t>(n) * 8, cudaMemcpyHostToDevice, ctx->stream);
  const int e = launch_device_math(dx, n, de, dl, ctx->stream);
  cudaMemcpyAsync(exp_out, de, static_cast<size_t>(n) * 8, cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(log_out, dl, static_cast<size_t>(n) * 8, cudaMemcpyDeviceToHost, ctx->stream);
  const cudaError_t se = cudaStreamSynchronize(ctx->stream);
  dfree(ctx->stream, dx);
  dfree(ctx->stream, de);
  dfree(ctx->stream, dl);
  if (e) return fail(ctx, AKMC_ECUDA, cuda_name(e));
  if (se != cudaSuccess) return fail(ctx, AKMC_ECUDA, cudaGetErrorString(se));
  return AKMC_OK;
}

}  // extern "C"
