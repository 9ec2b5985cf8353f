// pending.cu -- entry points not implemented yet; they report MG_ERR_UNSUPPORTED.
#include "mg_internal.h"

extern "C" {
mg_status mg_bfs_batch(mg_graph *, const int32_t *, int32_t, int32_t *, const mg_opts *, mg_stats *) { mg_set_error("not implemented"); return MG_ERR_UNSUPPORTED; }
mg_status mg_sssp_batch(mg_graph *, const int32_t *, int32_t, int32_t *, const mg_opts *, mg_stats *) { mg_set_error("not implemented"); return MG_ERR_UNSUPPORTED; }
mg_status mg_bfs_ragged(mg_graph *, const int32_t *, int32_t *, const mg_opts *, mg_stats *) { mg_set_error("not implemented"); return MG_ERR_UNSUPPORTED; }
}
