// pagerank -- PageRank driver (the reference's Algorithms/PageRank/PageRank.cu
// command line): the reference's formula x = 0.15 + 0.85 * sum x_u / deg_u with
// its 0.01 delta frontier (mode=0, default), or the normalised power iteration
// (mode=1, alpha, tol); the output file holds one rank per line.
#include <cstdio>
#include <vector>

#include "cli_common.h"

int main(int argc, char **argv) {
  mgcli::Config cfg;
  mgcli::register_common(cfg, false);
  cfg.registerDouble("tol", 0.1, "The tolerance for correctness check (default 0.1)");
  cfg.registerInt("mode", 0, "0: the reference's delta-frontier PageRank; 1: normalised power iteration (default 0)");
  cfg.registerDouble("alpha", 0.85, "Damping factor of the normalised mode (default 0.85)");
  cfg.registerDouble("pr_tol", 1e-6, "L1 residual stop of the normalised mode (default 1e-6)");
  mgcli::Args args;
  if (!mgcli::parse_args(argc, argv, cfg, args, "PageRank over the in-edges.")) return 1;
  mg_host_csr h = mgcli::load_market(args.graph);
  mg_graph *g = mgcli::upload(h, false, MG_DTYPE_NONE);
  mg_pr_opts o{};
  o.mode = cfg.getInt("mode") == 1 ? MG_PR_NORMALIZED : MG_PR_REFCOMPAT;
  o.directed = (int32_t)cfg.getInt("directed");
  const int64_t it = cfg.getInt("iter_num");
  o.max_iter = it >= INT32_MAX ? 0 : (int32_t)it;
  if (o.mode == MG_PR_NORMALIZED) {  // REFCOMPAT keeps the reference's 0.01 delta frontier
    o.alpha = cfg.getDouble("alpha");
    o.tol = cfg.getDouble("pr_tol");
  }
  std::vector<float> rank(h.n);
  mg_stats st;
  mgcli::check(mg_pagerank(g, nullptr, 1, rank.data(), &o, &st), "mg_pagerank");
  mgcli::print_trace(cfg, g);
  std::printf("Kernel time took: %.4f ms\n", st.kernel_ms);
  std::printf("Total iteration: %lld\n", (long long)st.iterations);
  if (!args.output.empty()) {
    FILE *f = std::fopen(args.output.c_str(), "w");
    for (int64_t i = 0; i < h.n; i++) std::fprintf(f, "%f\n", rank[i]);
    std::fclose(f);
  }
  mg_graph_destroy(g);
  mg_host_csr_free(&h);
  return 0;
}
