// Learned preconditioner: per-node / per-edge scalings of the chain blocks.
#include "ctx.cuh"

namespace cicy {

void learned_scalings(Ctx& c, const cicy_params& p, const SolverSystem& ss, int n_chains, int r_flag, const float** node_scale,
                      const float** edge_scale) {
    (void)c; (void)p; (void)ss; (void)n_chains; (void)r_flag;
    *node_scale = nullptr;
    *edge_scale = nullptr;
}

}  // namespace cicy
