// cli_common.h -- shared pieces of the BFS / SSSP / CC / PageRank command-line
// drivers: the reference's Config parameter registry (Algorithms/BFS/config.h,
// config.cpp:30-113, per-program defaults in Algorithms/*/register.h), its
// argument surface (-g/-graph, -o/-output, -s/-sources, -p/-parameters, -c,
// -help; Algorithms/BFS/bfs.cu:241-300) and its source selection (single src,
// a file of sources, or RANDOM; bfs.cu:338-400). The drivers run on the engine's
// C ABI (mapgraph_b200.h) only.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "mapgraph_b200.h"
#include "mapgraph_b200_io.h"

namespace mgcli {

// A typed parameter: int or double, with its description.
struct Param {
  bool is_int = true;
  double value = 0;
  std::string desc;
};

class Config {
 public:
  void registerInt(const std::string &name, int64_t def, const std::string &desc);
  void registerDouble(const std::string &name, double def, const std::string &desc);
  // "name=value name2=value2" (separators: space or comma).
  bool parseParameterString(const std::string &s);
  // One parameter string per line.
  bool parseFile(const std::string &path);
  int64_t getInt(const std::string &name) const;
  double getDouble(const std::string &name) const;
  void printOptions() const;

 private:
  std::map<std::string, Param> params_;
};

// Registers the parameters every driver shares (Algorithms/BFS/register.h).
void register_common(Config &cfg, bool sources);

struct Args {
  std::string graph, output, sources;
};

// Parses argv; returns false (after printing usage) when -help is given or no
// graph file is named.
bool parse_args(int argc, char **argv, Config &cfg, Args &args, const char *usage_extra);

// Source vertices: the "src" parameter (origin-adjusted), every line of a file
// (origin-adjusted, at most 1000), or num_src random vertices with out-edges.
std::vector<int32_t> select_sources(const Config &cfg, const Args &args, const mg_host_csr &g);

// Loads a Matrix Market file; exits with a message on failure.
mg_host_csr load_market(const std::string &path);

// Creates the device graph; exits with the engine's error detail on failure.
mg_graph *upload(const mg_host_csr &g, bool with_values, mg_dtype vt);

// Exits with the engine's message when st != MG_OK.
void check(mg_status st, const char *where);

// verbose=1: the last run's per-level records (the reference prints the frontier
// size of every iteration, GASengine/enactor_vertex_centric.cuh:2528-2546).
void print_trace(const Config &cfg, mg_graph *g);

}  // namespace mgcli
