// bfs -- breadth-first search driver (the reference's Algorithms/BFS/bfs.cu:241-518
// command line): depth of every vertex from each source in turn; the output file
// holds the last source's depths, one per line (-1 unreached).
#include <chrono>
#include <cstdio>
#include <vector>

#include "cli_common.h"

int main(int argc, char **argv) {
  mgcli::Config cfg;
  mgcli::register_common(cfg, true);
  cfg.registerInt("with_value", 0, "Whether to load edge values from market file (default 0)");
  mgcli::Args args;
  if (!mgcli::parse_args(argc, argv, cfg, args, "Breadth-first search from each source.")) return 1;
  mg_host_csr h = mgcli::load_market(args.graph);
  const std::vector<int32_t> srcs = mgcli::select_sources(cfg, args, h);
  mg_graph *g = mgcli::upload(h, false, MG_DTYPE_NONE);
  mg_opts o{};
  o.directed = (int32_t)cfg.getInt("directed");
  o.iter_num = (int32_t)std::min<int64_t>(cfg.getInt("iter_num"), INT32_MAX);
  o.threshold = (int32_t)cfg.getInt("threshold");
  std::vector<int32_t> depth(h.n);
  for (int32_t s : srcs) {
    if (s < 0 || s >= h.n) {
      std::fprintf(stderr, "source %d out of range\n", s);
      return 1;
    }
    std::printf("num_srcs=%d, src=%d, iter_num=%d\n", (int)srcs.size(), s, o.iter_num);
    mg_stats st;
    mgcli::check(mg_bfs(g, &s, 1, depth.data(), &o, &st), "mg_bfs");
    mgcli::print_trace(cfg, g);
    std::printf("Kernel time took: %.4f ms\n", st.kernel_ms);
    std::printf("Total iteration: %lld\n", (long long)st.iterations);
    std::printf("Traversed edge: %lld\n", (long long)st.edges_traversed);
    std::printf("GTEPS: %.3f\n", st.kernel_ms > 0 ? st.edges_traversed / (st.kernel_ms * 1e6) : 0.0);
  }
  if (!args.output.empty()) {
    FILE *f = std::fopen(args.output.c_str(), "w");
    for (int64_t i = 0; i < h.n; i++) std::fprintf(f, "%d\n", depth[i]);
    std::fclose(f);
  }
  mg_graph_destroy(g);
  mg_host_csr_free(&h);
  return 0;
}
