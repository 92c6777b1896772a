// Learned preconditioner: message-passing network over the particle neighbor graph.
// (Placeholder until the network kernels land: reports "not ready".)
#include "ops.cuh"

namespace lsmps_gpu {

bool mpnn_ready(lsmps_ctx* ctx) { return ctx->have_mpnn; }

void mpnn_warm_start(lsmps_ctx*, const float*, float*) {
    throw Error{LSMPS_ERR_STATE, "message-passing network not available"};
}

void mpnn_init(lsmps_ctx*, uint32_t) { throw Error{LSMPS_ERR_STATE, "message-passing network not available"}; }
void mpnn_add_sample(lsmps_ctx*) { throw Error{LSMPS_ERR_STATE, "message-passing network not available"}; }
void mpnn_train(lsmps_ctx*, const lsmps_mpnn_train_opts*, float*) {
    throw Error{LSMPS_ERR_STATE, "message-passing network not available"};
}
void mpnn_save(lsmps_ctx*, const char*) { throw Error{LSMPS_ERR_STATE, "message-passing network not available"}; }
void mpnn_load(lsmps_ctx*, const char*) { throw Error{LSMPS_ERR_STATE, "message-passing network not available"}; }

}  // namespace lsmps_gpu
