// cc -- connected components driver (the reference's Algorithms/CC/cc.cu
// command line): weakly connected components; the output file holds each vertex's
// label (the smallest vertex id of its component), one per line.
#include <cstdio>
#include <vector>

#include "cli_common.h"

int main(int argc, char **argv) {
  mgcli::Config cfg;
  mgcli::register_common(cfg, false);
  mgcli::Args args;
  if (!mgcli::parse_args(argc, argv, cfg, args, "Connected components (weak).")) return 1;
  mg_host_csr h = mgcli::load_market(args.graph);
  mg_graph *g = mgcli::upload(h, false, MG_DTYPE_NONE);
  std::vector<int32_t> label(h.n);
  mg_opts o{};
  mg_stats st;
  mgcli::check(mg_cc(g, label.data(), &o, &st), "mg_cc");
  int64_t ncomp = 0;
  for (int64_t i = 0; i < h.n; i++) ncomp += label[i] == i;
  std::printf("Kernel time took: %.4f ms\n", st.kernel_ms);
  std::printf("Components: %lld\n", (long long)ncomp);
  if (!args.output.empty()) {
    FILE *f = std::fopen(args.output.c_str(), "w");
    for (int64_t i = 0; i < h.n; i++) std::fprintf(f, "%d\n", label[i]);
    std::fclose(f);
  }
  mg_graph_destroy(g);
  mg_host_csr_free(&h);
  return 0;
}
