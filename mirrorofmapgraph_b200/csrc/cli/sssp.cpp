// sssp -- single-source shortest paths driver (the reference's
// Algorithms/SSSP/sssp.cu command line): int32 edge values from the market file
// (with_value=1, unit weights otherwise); the output file holds the last source's
// distances, one per line (2147483647 unreached).
#include <cstdio>
#include <vector>

#include "cli_common.h"

int main(int argc, char **argv) {
  mgcli::Config cfg;
  mgcli::register_common(cfg, true);
  cfg.registerInt("with_value", 1, "Whether to load edge values from market file (default 1)");
  mgcli::Args args;
  if (!mgcli::parse_args(argc, argv, cfg, args, "Single-source shortest paths from each source.")) return 1;
  mg_host_csr h = mgcli::load_market(args.graph);
  const std::vector<int32_t> srcs = mgcli::select_sources(cfg, args, h);
  mg_graph *g = mgcli::upload(h, cfg.getInt("with_value") != 0, MG_DTYPE_I32);
  mg_opts o{};
  o.directed = (int32_t)cfg.getInt("directed");
  o.iter_num = (int32_t)std::min<int64_t>(cfg.getInt("iter_num"), INT32_MAX);
  std::vector<int32_t> dist(h.n);
  for (int32_t s : srcs) {
    if (s < 0 || s >= h.n) {
      std::fprintf(stderr, "source %d out of range\n", s);
      return 1;
    }
    mg_stats st;
    mgcli::check(mg_sssp(g, &s, 1, dist.data(), &o, &st), "mg_sssp");
    mgcli::print_trace(cfg, g);
    std::printf("Kernel time took: %.4f ms\n", st.kernel_ms);
    std::printf("Total iteration: %lld\n", (long long)st.iterations);
    std::printf("Traversed edge: %lld\n", (long long)st.edges_traversed);
  }
  if (!args.output.empty()) {
    FILE *f = std::fopen(args.output.c_str(), "w");
    for (int64_t i = 0; i < h.n; i++) std::fprintf(f, "%lld\n", (long long)dist[i]);
    std::fclose(f);
  }
  mg_graph_destroy(g);
  mg_host_csr_free(&h);
  return 0;
}
