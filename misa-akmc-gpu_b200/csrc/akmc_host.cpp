// akmc_host.cpp -- host-side mirror of the reference's driver around the GPU path:
//   * config.yaml reader for the schema of profiles/config/config_parsing.cpp:54-230
//     (a small YAML-subset parser: block maps, flow sequences, scalars, comments);
//   * lattice creation in the reference's draw order (src/creation.cpp:18-164);
//   * SubLattice::startTimeLoop (src/algorithms/sl/sublattice.inl:24-190) driven over
//     the per-hop entry points, as ABVIModel drives gpu/gpu_simulate.h;
//   * the lattice dump of profiles/io/lattice_dump.cpp:14-62.
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <random>
#include <string>
#include <vector>

#include "akmc_device.h"
#include "akmc_model.h"

namespace {

// ---------------------------------------------------------------------------
// YAML subset: indentation-structured block maps, "key: value", flow sequences
// "[a, b, c]", quoted or plain scalars, '#' comments.  Enough for config.yaml.
struct Node {
  std::string scalar;
  std::vector<std::string> seq;
  std::vector<std::pair<std::string, Node>> map;  // document order (the alloy order matters)
  bool is_map = false, is_seq = false;
  const Node* get(const std::string& k) const {
    for (const auto& kv : map)
      if (kv.first == k) return &kv.second;
    return nullptr;
  }
};

std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t\r");
  if (a == std::string::npos) return "";
  size_t b = s.find_last_not_of(" \t\r");
  return s.substr(a, b - a + 1);
}
std::string strip_comment(const std::string& s) {
  bool q1 = false, q2 = false;
  for (size_t i = 0; i < s.size(); ++i) {
    const char c = s[i];
    if (c == '\'' && !q2) q1 = !q1;
    else if (c == '"' && !q1) q2 = !q2;
    else if (c == '#' && !q1 && !q2 && (i == 0 || s[i - 1] == ' ' || s[i - 1] == '\t')) return s.substr(0, i);
  }
  return s;
}
std::string unquote(const std::string& s) {
  if (s.size() >= 2 && ((s.front() == '"' && s.back() == '"') || (s.front() == '\'' && s.back() == '\'')))
    return s.substr(1, s.size() - 2);
  return s;
}

struct Line {
  int indent;
  std::string key, value;
};

bool parse_yaml(const std::string& text, Node& root, std::string& err) {
  std::vector<Line> lines;
  size_t pos = 0;
  int lineno = 0;
  while (pos <= text.size()) {
    size_t e = text.find('\n', pos);
    if (e == std::string::npos) e = text.size();
    std::string raw = strip_comment(text.substr(pos, e - pos));
    pos = e + 1;
    ++lineno;
    if (trim(raw).empty()) continue;
    int ind = 0;
    while (ind < static_cast<int>(raw.size()) && raw[static_cast<size_t>(ind)] == ' ') ++ind;
    const std::string body = trim(raw);
    if (body == "---") continue;
    const size_t colon = body.find(':');
    if (colon == std::string::npos) {
      err = "line " + std::to_string(lineno) + ": expected 'key: value'";
      return false;
    }
    lines.push_back({ind, unquote(trim(body.substr(0, colon))), trim(body.substr(colon + 1))});
  }
  // recursive descent over indentation levels
  std::vector<std::pair<int, Node*>> stack{{-1, &root}};
  root.is_map = true;
  for (size_t i = 0; i < lines.size(); ++i) {
    const Line& L = lines[i];
    while (stack.size() > 1 && L.indent <= stack.back().first) stack.pop_back();
    Node* parent = stack.back().second;
    parent->is_map = true;
    parent->map.push_back({L.key, Node()});
    Node& n = parent->map.back().second;
    if (L.value.empty()) {
      stack.push_back({L.indent, &n});
    } else if (L.value.front() == '[') {
      if (L.value.back() != ']') {
        err = "unterminated sequence for key " + L.key;
        return false;
      }
      n.is_seq = true;
      std::string inner = L.value.substr(1, L.value.size() - 2);
      size_t p = 0;
      while (p <= inner.size()) {
        size_t c = inner.find(',', p);
        if (c == std::string::npos) c = inner.size();
        const std::string item = trim(inner.substr(p, c - p));
        if (!item.empty()) n.seq.push_back(unquote(item));
        p = c + 1;
      }
    } else {
      n.scalar = unquote(L.value);
    }
  }
  return true;
}

bool to_i64(const Node* n, int64_t& v) {
  if (!n || n->is_map || n->is_seq) return false;
  char* end = nullptr;
  const double d = std::strtod(n->scalar.c_str(), &end);
  if (end == n->scalar.c_str()) return false;
  v = static_cast<int64_t>(d);
  return true;
}
bool to_f64(const Node* n, double& v) {
  if (!n || n->is_map || n->is_seq) return false;
  char* end = nullptr;
  v = std::strtod(n->scalar.c_str(), &end);
  return end != n->scalar.c_str();
}
bool to_bool(const Node* n, bool dflt) {
  if (!n) return dflt;
  const std::string s = n->scalar;
  if (s == "true" || s == "True" || s == "yes" || s == "on" || s == "1") return true;
  if (s == "false" || s == "False" || s == "no" || s == "off" || s == "0") return false;
  return dflt;
}

int type_code(const std::string& s) {  // lat::LatTypes (profiles/config/lattice_types_string.cpp:43-80)
  if (s == "V") return akmc::kV;
  if (s == "Fe") return akmc::kFe;
  if (s == "Cu") return akmc::kCu;
  if (s == "Ni") return akmc::kNi;
  if (s == "Mn") return akmc::kMn;
  static const char* dumbbells[] = {"FeFe", "FeCu", "FeNi", "FeMn", "CuCu", "CuNi", "CuMn", "NiNi", "NiMn", "MnMn"};
  for (const char* d : dumbbells)
    if (s == d) return 0x100;
  return -1;
}

void set_err(char* err, int32_t len, const std::string& m) {
  if (err && len > 0) std::snprintf(err, static_cast<size_t>(len), "%s", m.c_str());
}

}  // namespace

extern "C" {

AKMC_API akmc_status akmc_config_parse(const char* text, akmc_run_config* out, char* err, int32_t errlen) {
  if (!text || !out) return AKMC_EINVAL;
  std::memset(out, 0, sizeof(*out));
  out->sector_window = 3.0e-7;
  out->blocks[0] = out->blocks[1] = out->blocks[2] = 1;
  out->energy_model = AKMC_MODEL_PAIRBOND;
  out->seed = 42;
  out->pot_seed = 42;
  Node root;
  std::string e;
  if (!parse_yaml(text, root, e)) {
    set_err(err, errlen, e);
    return AKMC_EINVAL;
  }
  // box (ConfigParsing::parseBox, config_parsing.cpp:106-130)
  const Node* box = root.get("box");
  if (!box) return set_err(err, errlen, "box in config is not specified."), AKMC_EINVAL;
  const Node* size = box->get("size");
  if (!size || !size->is_seq || size->seq.size() != 3) return set_err(err, errlen, "box size must be 3."), AKMC_EINVAL;
  for (int d = 0; d < 3; ++d) out->box[d] = std::atoll(size->seq[static_cast<size_t>(d)].c_str());
  if (!to_f64(box->get("lattice_const"), out->lattice_const))
    return set_err(err, errlen, "lattice const must be set in config."), AKMC_EINVAL;
  if (!to_f64(box->get("cutoff_radius"), out->cutoff_radius))
    return set_err(err, errlen, "cutoff radius must be set in config."), AKMC_EINVAL;
  // simulation (parseSim)
  const Node* sim = root.get("simulation");
  if (!sim) return set_err(err, errlen, "simulation in config is not specified."), AKMC_EINVAL;
  to_f64(sim->get("temperature"), out->temperature);
  to_f64(sim->get("physics_time"), out->physics_time);
  to_i64(sim->get("steps_limit"), out->steps_limit);
  to_f64(sim->get("attempt_freq"), out->attempt_freq);
  to_f64(sim->get("dpasm1"), out->dpasm1);
  out->isgenr = to_bool(sim->get("isgenr"), false) ? 1 : 0;
  // create (parseCreate, config_parsing.cpp:150-205): random first, else pipe; restart is
  // reported as unsupported (this library restarts from its own snapshots)
  const Node* create = root.get("create");
  if (!create) return set_err(err, errlen, "create in config is not specified."), AKMC_EINVAL;
  const Node* random = create->get("random");
  const Node* pipe = create->get("pipe");
  const bool random_on = random && to_bool(random->get("enable"), false);
  const bool pipe_on = !random_on && pipe && to_bool(pipe->get("enable"), false);
  if (random_on || pipe_on) {
    if (random_on) {
      out->create_random = 1;
      to_i64(random->get("va_count"), out->va_count);
    } else {
      // the pipe option takes its alloy from create.random.alloy, as the reference does
      // (config_parsing.cpp:177); the vacancy count is that of the pile file
      out->create_pipe = 1;
      out->va_count = -1;
      if (const Node* ib = pipe->get("input_box"))
        std::snprintf(out->pipe_input_box, sizeof(out->pipe_input_box), "%s", ib->scalar.c_str());
      if (!out->pipe_input_box[0]) return set_err(err, errlen, "create.pipe.input_box is empty."), AKMC_EINVAL;
    }
    const Node* alloy = random ? random->get("alloy") : nullptr;
    if (!alloy || !alloy->is_map) return set_err(err, errlen, "alloy must be a map in config."), AKMC_EINVAL;
    for (const auto& kv : alloy->map) {
      const int c = type_code(kv.first);
      int64_t r = 0;
      to_i64(&kv.second, r);
      if (c < 0) return set_err(err, errlen, "unknown alloy type " + kv.first), AKMC_EINVAL;
      if (c == 0x100) {
        if (r != 0) return set_err(err, errlen, "dumbbell alloy entries are outside the vacancy path"), AKMC_EINVAL;
        continue;
      }
      if (c == akmc::kV || out->n_types >= 4) return set_err(err, errlen, "alloy: at most Fe, Cu, Ni, Mn"), AKMC_EINVAL;
      out->type_codes[out->n_types] = c;
      out->ratio[out->n_types] = r;
      ++out->n_types;
    }
  } else {
    const Node* restart = create->get("restart");
    if (restart && to_bool(restart->get("enable"), false))
      return set_err(err, errlen,
                     "create.restart is not supported; restart from a snapshot (akmc_restore_snapshot)"),
             AKMC_EINVAL;
    return set_err(err, errlen, "no create option in config."), AKMC_EINVAL;
  }
  // seeds (parseSeeds)
  const Node* seeds = root.get("seeds");
  if (!seeds) return set_err(err, errlen, "seeds in config is not specified."), AKMC_EINVAL;
  to_i64(seeds->get("create_types"), out->seed_create_types);
  to_i64(seeds->get("create_vacancy"), out->seed_create_vacancy);
  to_i64(seeds->get("event_selection"), out->seed_event_selection);
  to_i64(seeds->get("time_inc"), out->seed_time_inc);
  // output (parseOutput)
  if (const Node* output = root.get("output")) {
    if (const Node* dump = output->get("dump")) {
      to_i64(dump->get("interval"), out->dump_interval);
      if (const Node* fp = dump->get("file_path")) std::snprintf(out->dump_file_path, sizeof(out->dump_file_path), "%s", fp->scalar.c_str());
    }
    if (const Node* logs = output->get("logs")) {
      to_i64(logs->get("interval"), out->logs_interval);
      if (const Node* lf = logs->get("logs_file")) std::snprintf(out->logs_file, sizeof(out->logs_file), "%s", lf->scalar.c_str());
    }
  }
  // optional kmc: block of this implementation (ignored by the reference)
  if (const Node* k = root.get("kmc")) {
    if (const Node* m = k->get("energy_model")) out->energy_model = m->scalar == "eam" ? AKMC_MODEL_EAM : AKMC_MODEL_PAIRBOND;
    if (const Node* p = k->get("precision")) out->precision = p->scalar == "fp32c" ? AKMC_FP32C : AKMC_FP64;
    if (const Node* b = k->get("blocks")) {
      if (!b->is_seq || b->seq.size() != 3) return set_err(err, errlen, "kmc.blocks must be 3"), AKMC_EINVAL;
      for (int d = 0; d < 3; ++d) out->blocks[d] = std::atoi(b->seq[static_cast<size_t>(d)].c_str());
    }
    if (const Node* c = k->get("creation")) out->creation = c->scalar == "xoshiro" ? 1 : 0;
    to_f64(k->get("sector_window"), out->sector_window);
    to_i64(k->get("hop_budget"), out->hop_budget);
    int64_t s = 0;
    if (to_i64(k->get("seed"), s)) out->seed = static_cast<uint64_t>(s);
    if (to_i64(k->get("pot_seed"), s)) out->pot_seed = static_cast<uint64_t>(s);
  }
  if (out->n_types == 0) return set_err(err, errlen, "alloy has no atoms"), AKMC_EINVAL;
  return AKMC_OK;
}

// creation::createAtomsRandom / createRandom for one rank (src/creation.cpp:18-164):
// one uniform_int_distribution<>(1, sum ratio) draw per site of the ghost-padded
// array (ghost = ceil(cutoff / lattice_const)) in z-y-x order with mt19937(create_types),
// then vacancies from uniform_int_distribution<long long>(0, sites - 1) with
// mt19937(create_vacancy).  creation = 1 uses the xoshiro streams instead.
//
// create.pipe (creation::createFromPile, src/creation.cpp:184-230): the same alloy draws, then a
// vacancy at every position "x y z" (x doubled) of the pile file that lies inside the box, read
// as the reference reads it (`while (file >> x >> y >> z)`); positions outside the box are
// skipped.  The reference marks these vacancies in LatticesList::_lattices only, which its
// hash-set occupancy store never reads; here the site becomes a vacancy, whatever atom it held.
AKMC_API akmc_status akmc_config_lattice(const akmc_run_config* cfg, uint8_t* occ, int64_t n_sites) {
  if (!cfg || !occ) return AKMC_EINVAL;
  const int64_t sx = 2 * cfg->box[0], sy = cfg->box[1], sz = cfg->box[2];
  if (n_sites != sx * sy * sz) return AKMC_EINVAL;
  if (!cfg->create_pipe && (cfg->va_count < 0 || cfg->va_count > n_sites)) return AKMC_EINVAL;
  std::vector<int64_t> pile;
  if (cfg->create_pipe) {
    if (cfg->creation == 1) return AKMC_EINVAL;  // the pile file is a reference-order creation
    std::ifstream f(cfg->pipe_input_box);
    if (!f) return AKMC_EINVAL;
    int64_t x, y, z;
    while (f >> x >> y >> z) {
      pile.push_back(x);
      pile.push_back(y);
      pile.push_back(z);
    }
  }
  int64_t codes64[4] = {0, 0, 0, 0};
  int32_t codes[4] = {akmc::kFe, akmc::kFe, akmc::kFe, akmc::kFe};
  int64_t total = 0;
  for (int i = 0; i < cfg->n_types; ++i) {
    codes[i] = cfg->type_codes[i];
    codes64[i] = cfg->ratio[i];
    total += cfg->ratio[i];
  }
  if (total <= 0 || total > 0x7fffffff) return AKMC_EINVAL;
  if (cfg->creation == 1)
    return akmc::create_lattice(cfg->box, codes, codes64, cfg->va_count, cfg->seed, occ, n_sites) ? AKMC_EINVAL
                                                                                                  : AKMC_OK;
  const int64_t g = static_cast<int64_t>(std::ceil(cfg->cutoff_radius / cfg->lattice_const));
  const int64_t px = 2 * (cfg->box[0] + 2 * g), py = sy + 2 * g, pz = sz + 2 * g;
  std::uniform_int_distribution<> types_dis(1, static_cast<int>(total));
  std::mt19937 types_rng(static_cast<std::mt19937::result_type>(cfg->seed_create_types));
  for (int64_t z = 0; z < pz; ++z)
    for (int64_t y = 0; y < py; ++y)
      for (int64_t x = 0; x < px; ++x) {
        const int64_t hit = types_dis(types_rng);
        int64_t acc = 0;
        uint8_t t = akmc::kFe;
        for (int i = 0; i < cfg->n_types; ++i) {
          acc += cfg->ratio[i];
          if (acc >= hit) {
            t = static_cast<uint8_t>(codes[i]);
            break;
          }
        }
        const int64_t ix = x - 2 * g, iy = y - g, iz = z - g;
        if (ix >= 0 && ix < sx && iy >= 0 && iy < sy && iz >= 0 && iz < sz) occ[ix + sx * (iy + sy * iz)] = t;
      }
  if (cfg->create_pipe) {
    for (size_t i = 0; i + 2 < pile.size(); i += 3) {
      const int64_t x = pile[i], y = pile[i + 1], z = pile[i + 2];
      if (x < 0 || x >= sx || y < 0 || y >= sy || z < 0 || z >= sz) continue;  // isIn(x / 2, y, z)
      occ[x + sx * (y + sy * z)] = akmc::kV;
    }
    return AKMC_OK;
  }
  std::uniform_int_distribution<long long> va_dis(0, n_sites - 1);
  std::mt19937 va_rng(static_cast<std::mt19937::result_type>(cfg->seed_create_vacancy));
  int64_t placed = 0;
  while (placed < cfg->va_count) {
    int64_t id = va_dis(va_rng);
    const int64_t x = id % sx;
    id /= sx;
    const int64_t y = id % sy, z = id / sy;
    uint8_t& o = occ[x + sx * (y + sy * z)];
    if (o != akmc::kV) {  // the reference clears only Cu here (creation.cpp:149-157); every solute is cleared
      o = akmc::kV;
      ++placed;
    }
  }
  return AKMC_OK;
}

AKMC_API akmc_status akmc_config_job(const akmc_run_config* cfg, const akmc_eam_tables* eam, akmc_job_config* out) {
  if (!cfg || !out) return AKMC_EINVAL;
  std::memset(out, 0, sizeof(*out));
  for (int d = 0; d < 3; ++d) {
    out->box[d] = cfg->box[d];
    out->blocks[d] = cfg->blocks[d] > 0 ? cfg->blocks[d] : 1;
  }
  out->energy_model = cfg->energy_model;
  out->precision = cfg->precision;
  out->rng = AKMC_RNG_XOSHIRO;
  out->lattice_const = cfg->lattice_const;
  out->cutoff_radius = cfg->cutoff_radius;
  out->attempt_freq = cfg->attempt_freq;
  out->temperature = cfg->temperature;
  out->sector_window = cfg->sector_window > 0 ? cfg->sector_window : 3.0e-7;
  out->seed = cfg->seed;
  out->hop_budget = cfg->hop_budget;
  // SubLattice::startTimeLoop: time_steps = ceil(physics_time / T), 8 sector rounds each
  out->max_rounds = cfg->physics_time > 0 ? 8 * static_cast<int64_t>(std::ceil(cfg->physics_time / out->sector_window)) : 0;
  out->eam = cfg->energy_model == AKMC_MODEL_EAM ? eam : nullptr;
  if (cfg->energy_model == AKMC_MODEL_EAM && !eam) return AKMC_EINVAL;
  return AKMC_OK;
}

// SubLattice::startTimeLoop (sublattice.inl:61-140) for one domain, host-driven:
// per hop akmc_calculate (calcRatesWrapper) then, when the total is non-zero,
// akmc_select_and_perform (selectPerformWrapper) and the residence-time clock.
AKMC_API akmc_status akmc_host_time_loop(akmc_ctx* ctx, int32_t job, int64_t n_rounds, uint64_t seed, double window,
                                         akmc_event* events, int64_t capacity, int64_t* n_events, double* evo8) {
  if (!ctx || n_rounds < 0 || !(window > 0)) return AKMC_EINVAL;
  uint64_t xs[4], xt[4];
  akmc::xoshiro_seed(xs, seed, akmc::kTagSelect, 0);
  akmc::xoshiro_seed(xt, seed, akmc::kTagTime, 0);
  double evo[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int64_t nev = 0, hops = 0;
  for (int64_t rnd = 0; rnd < n_rounds; ++rnd) {
    const int sector = akmc::sector_of_round(rnd);
    const int64_t step = rnd >> 3;
    const double thr = static_cast<double>(step + 1) * window - evo[sector];
    double sector_time = 0.0;
    while (sector_time < thr) {
      double total = 0.0;
      akmc_status s = akmc_calculate(ctx, job, sector, &total);
      if (s) return s;
      if (total == 0.0 || std::fabs(total) < DBL_EPSILON) {
        sector_time = thr;
        continue;
      }
      const double u = akmc::uniform_co(xs);
      akmc_event ev;
      s = akmc_select_and_perform(ctx, job, sector, u, &ev);
      if (s) return s;
      const double u2 = akmc::uniform_oc(xt);
      const double dt = -akmc::port_log(u2) / total;
      sector_time += dt;
      if (ev.from_site >= 0) {
        if (events && nev < capacity) {
          ev.round = rnd;
          ev.hop = hops;
          ev.dt = dt;
          events[nev] = ev;
        }
        ++nev;
        ++hops;
      }
    }
    evo[sector] += sector_time;
  }
  if (n_events) *n_events = nev;
  if (evo8) std::memcpy(evo8, evo, sizeof(evo));
  return (events && nev > capacity) ? AKMC_EOVERFLOW : AKMC_OK;
}

// LatticeDump::dump (profiles/io/lattice_dump.cpp:14-62): site count, blank line,
// then "type x y z" in z-y-x order with the local (ghost-offset) coordinates of a
// single rank; centre sites at half-integer coordinates.
AKMC_API akmc_status akmc_dump_lattice(const uint8_t* occ, const int64_t box[3], int32_t ghost, const char* path) {
  if (!occ || !box || !path || ghost < 0) return AKMC_EINVAL;
  FILE* f = std::fopen(path, "w");
  if (!f) return AKMC_EINVAL;
  const int64_t sx = 2 * box[0], sy = box[1], sz = box[2];
  std::fprintf(f, "%lld\n\n", static_cast<long long>(sx * sy * sz));
  auto name = [](uint8_t c) {
    switch (c) {
      case akmc::kV: return "V";
      case akmc::kFe: return "Fe";
      case akmc::kCu: return "Cu";
      case akmc::kNi: return "Ni";
      case akmc::kMn: return "Mn";
      default: return "?";
    }
  };
  for (int64_t z = 0; z < sz; ++z)
    for (int64_t y = 0; y < sy; ++y)
      for (int64_t X = 0; X < sx; ++X) {
        const int64_t lx = X + 2 * ghost, ly = y + ghost, lz = z + ghost;
        const char* t = name(occ[X + sx * (y + sy * z)]);
        if (lx % 2 == 0)
          std::fprintf(f, "%s\t%lld\t%lld\t%lld\n", t, static_cast<long long>(lx / 2), static_cast<long long>(ly),
                       static_cast<long long>(lz));
        else
          std::fprintf(f, "%s\t%g\t%g\t%g\n", t, static_cast<double>(lx / 2) + 0.5, static_cast<double>(ly) + 0.5,
                       static_cast<double>(lz) + 0.5);
      }
  std::fclose(f);
  return AKMC_OK;
}

}  // extern "C"
