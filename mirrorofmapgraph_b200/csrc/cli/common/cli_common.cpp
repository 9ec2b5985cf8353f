// cli_common.cpp -- see cli_common.h.
#include "cli_common.h"

#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <random>
#include <sstream>

namespace mgcli {

void Config::registerInt(const std::string &name, int64_t def, const std::string &desc) {
  params_[name] = Param{true, (double)def, desc};
}

void Config::registerDouble(const std::string &name, double def, const std::string &desc) {
  params_[name] = Param{false, def, desc};
}

bool Config::parseParameterString(const std::string &s) {
  std::string tok;
  std::stringstream ss(s);
  bool ok = true;
  while (ss >> tok) {
    // a token may itself hold comma-separated assignments
    size_t start = 0;
    while (start <= tok.size()) {
      const size_t comma = tok.find(',', start);
      const std::string a = tok.substr(start, comma == std::string::npos ? std::string::npos : comma - start);
      start = comma == std::string::npos ? tok.size() + 1 : comma + 1;
      if (a.empty()) continue;
      const size_t eq = a.find('=');
      const std::string name = a.substr(0, eq);
      auto it = params_.find(name);
      if (it == params_.end() || eq == std::string::npos) {
        std::fprintf(stderr, "Variable '%s' not registered\n", name.c_str());
        ok = false;
        continue;
      }
      it->second.value = std::strtod(a.c_str() + eq + 1, nullptr);
    }
  }
  return ok;
}

bool Config::parseFile(const std::string &path) {
  std::ifstream fin(path);
  if (!fin) {
    std::fprintf(stderr, "Error opening file '%s'\n", path.c_str());
    return false;
  }
  std::string line;
  bool ok = true;
  while (std::getline(fin, line)) ok = parseParameterString(line) && ok;
  return ok;
}

int64_t Config::getInt(const std::string &name) const {
  auto it = params_.find(name);
  if (it == params_.end()) {
    std::fprintf(stderr, "parameter '%s' not registered\n", name.c_str());
    std::exit(1);
  }
  return (int64_t)it->second.value;
}

double Config::getDouble(const std::string &name) const {
  auto it = params_.find(name);
  if (it == params_.end()) {
    std::fprintf(stderr, "parameter '%s' not registered\n", name.c_str());
    std::exit(1);
  }
  return it->second.value;
}

void Config::printOptions() const {
  for (const auto &kv : params_) std::printf("           %s: %s\n", kv.first.c_str(), kv.second.desc.c_str());
}

void register_common(Config &cfg, bool sources) {
  cfg.registerInt("verbose", 0, "Print out frontier size in each iteration (default 0)");
  cfg.registerInt("device", 0, "The device to use (default 0)");
  cfg.registerInt("iter_num", INT_MAX, "The number of iterations to perform (default INT_MAX)");
  cfg.registerInt("run_CPU", 0, "Run CPU implementation for testing (default 0)");
  cfg.registerDouble("max_queue_sizing", 1.5,
                     "The frontier queue size is this value times the number of vertices in the graph (default 1.5)");
  cfg.registerInt("threshold", 10000,
                  "When frontier size is larger than threshold, two-phase strategy is used otherwise dynamic "
                  "scheduling it used (default 10000)");
  cfg.registerInt("stats", 0, "Print out degree histogram (default 0)");
  cfg.registerInt("directed", 1, "The graph is directed (default 1)");
  if (sources) {
    cfg.registerInt("src", 1, "Starting vertex (default 1)");
    cfg.registerInt("origin", 1, "The origin (0 or 1) for the starting vertices (default 1)");
    cfg.registerInt("num_src", 1, "The number of starting vertices when random sources is specified (default 1)");
  }
}

static void usage(const char *prog, const Config &cfg, const char *extra) {
  std::printf("Usage: %s -g <graph.mtx> [-s <sources file | RANDOM>] [-o <output file>]\n"
              "          [-p \"name=value ...\"] [-c <parameter file>] [-help]\n%s\nParameters:\n",
              prog, extra);
  cfg.printOptions();
}

bool parse_args(int argc, char **argv, Config &cfg, Args &args, const char *usage_extra) {
  for (int i = 1; i < argc; i++) {
    const char *a = argv[i];
    const bool has_next = i + 1 < argc;
    if (!std::strcmp(a, "-help")) {
      usage(argv[0], cfg, usage_extra);
      return false;
    } else if ((!std::strcmp(a, "-graph") || !std::strcmp(a, "-g")) && has_next) {
      args.graph = argv[++i];
    } else if ((!std::strcmp(a, "-output") || !std::strcmp(a, "-o")) && has_next) {
      args.output = argv[++i];
    } else if ((!std::strcmp(a, "-sources") || !std::strcmp(a, "-s")) && has_next) {
      args.sources = argv[++i];
    } else if ((!std::strcmp(a, "-parameters") || !std::strcmp(a, "-p")) && has_next) {
      cfg.parseParameterString(argv[++i]);
    } else if (!std::strcmp(a, "-c") && has_next) {
      cfg.parseFile(argv[++i]);
    }
  }
  if (args.graph.empty()) {
    usage(argv[0], cfg, usage_extra);
    return false;
  }
  return true;
}

std::vector<int32_t> select_sources(const Config &cfg, const Args &args, const mg_host_csr &g) {
  std::vector<int32_t> srcs;
  const int64_t origin = cfg.getInt("origin");
  if (args.sources.empty()) {
    int64_t s = cfg.getInt("src");
    if (origin == 1) s--;
    srcs.push_back((int32_t)s);
    std::printf("Single source vertex: %d\n", srcs[0]);
  } else if (args.sources == "RANDOM") {
    const int64_t k = cfg.getInt("num_src");
    std::printf("Using %lld random starting vertices!\n", (long long)k);
    std::mt19937_64 rng(std::random_device{}());
    int64_t with_edges = 0;
    for (int64_t v = 0; v < g.n; v++) with_edges += g.row_offsets[v + 1] > g.row_offsets[v];
    while ((int64_t)srcs.size() < k && with_edges > 0) {
      const int32_t v = (int32_t)(rng() % (uint64_t)g.n);
      if (g.row_offsets[v + 1] > g.row_offsets[v]) srcs.push_back(v);
    }
  } else {
    std::printf("Using source file: %s!\n", args.sources.c_str());
    FILE *f = std::fopen(args.sources.c_str(), "r");
    if (!f) {
      std::printf("Source file open error!\n");
      std::exit(0);
    }
    int v;
    while ((int)srcs.size() < 1000 && std::fscanf(f, "%d", &v) == 1) srcs.push_back(origin == 1 ? v - 1 : v);
    std::fclose(f);
    std::printf("number of srcs used: %d\n", (int)srcs.size());
  }
  return srcs;
}

void print_trace(const Config &cfg, mg_graph *g) {
  if (cfg.getInt("verbose") == 0) return;
  std::vector<mg_level_record> rec(MG_TRACE_LEVELS);
  int32_t cnt = 0;
  check(mg_graph_trace(g, rec.data(), MG_TRACE_LEVELS, &cnt), "mg_graph_trace");
  for (int32_t i = 0; i < cnt; i++)
    std::printf("iteration %d: frontier %lld, frontier edges %lld, %s%s%.3g\n", rec[i].level,
                (long long)rec[i].frontier, (long long)rec[i].frontier_edges,
                rec[i].direction == MG_DIR_PULL ? "pull" : "push", rec[i].value != 0.0 ? ", residual " : "",
                rec[i].value != 0.0 ? rec[i].value : 0.0);
}

void check(mg_status st, const char *where) {
  if (st != MG_OK) {
    std::fprintf(stderr, "%s: %s: %s\n", where, mg_status_string(st), mg_last_error());
    std::exit(1);
  }
}

mg_host_csr load_market(const std::string &path) {
  mg_host_csr g;
  std::memset(&g, 0, sizeof(g));
  check(mg_read_market(path.c_str(), 0, &g), "mg_read_market");
  std::printf("Loaded %s: %lld vertices, %lld edges\n", path.c_str(), (long long)g.n, (long long)g.m);
  return g;
}

mg_graph *upload(const mg_host_csr &g, bool with_values, mg_dtype vt) {
  mg_graph *dg = nullptr;
  const void *vals = nullptr;
  if (with_values) vals = vt == MG_DTYPE_F32 ? (const void *)g.weights_f32 : (const void *)g.weights_i32;
  check(mg_graph_create(g.row_offsets, g.col_idx, vals, vals ? vt : MG_DTYPE_NONE, g.n, g.m, 0, &dg),
        "mg_graph_create");
  return dg;
}

}  // namespace mgcli
