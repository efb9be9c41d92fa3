// The context behind the opaque radm2_ctx handle (shared by radm2_capi.cu and radm2_mlp.cu).
#pragma once

#include <string>
#include <vector>

#include "../../include/radm2.h"
#include "radm2_internal.h"

struct radm2_ctx {
    radm2_opts o{};
    int nsm = 0;
    cudaStream_t own = nullptr;
    cudaStream_t st = nullptr;
    cudaStream_t st_up = nullptr, st_down = nullptr;  // copy streams of the pipelined host path
    std::vector<cudaEvent_t> pipe_ev;                 // per chunk: inputs up, chunk integrated
    int ncell = 0, ld = 0;
    double *var = nullptr, *fix = nullptr, *temp = nullptr, *rcn = nullptr, *jv = nullptr, *rconst = nullptr;
    bool have_rcn = false;
    bool rconst_valid = false;
    double *h0 = nullptr;
    int *order = nullptr;
    int *status = nullptr, *nacc = nullptr, *nrej = nullptr;
    double *hfirst = nullptr, *hexit = nullptr, *texit = nullptr;
    int *queue = nullptr;  // one counter per split
    int queue_cap = 0;
    double *scratch = nullptr;
    size_t scratch_bytes = 0;
    double *stage = nullptr;
    size_t stage_bytes = 0;
    void *partials = nullptr;
    radm2::RunResult *d_res = nullptr, *h_res = nullptr;
    int res_cap = 0;
    size_t bytes = 0;
    std::string err;
    radm2_stats stats{};
    // cached split graph
    cudaGraphExec_t gexec = nullptr;
    std::vector<unsigned char> gkey;
    int graph_kernels = 0;  // kernel nodes of the cached split graph
    // solver-kernel timing
    bool timing = false;
    std::vector<cudaEvent_t> ev;  // start/stop pairs, one per result slot
    int ev_used = 0;
    double kernel_ms = 0.0;
    int kernel_launches = 0;
    // learned seeding work arrays (radm2_seed_cells)
    unsigned int *seed_keys = nullptr;
    int *seed_idx = nullptr;
    void *seed_tmp = nullptr;
    size_t seed_tmp_bytes = 0;
    int seed_cap = 0;
    float *seed_x = nullptr, *seed_y = nullptr;  // [seed_cap][84] features, [seed_cap][2] predictions
    bool use_h0 = true, use_order = true;  // whether the solver reads h0 / order when set
    radm2_mlp *mlp = nullptr;               // attached network: seeds every integration
    int mlp_order = 0;  // 0 none, 1 cells by predicted cost, 2 chunks of 32 cells by cost
    int coop_selftest = 0;  // next integrations: the cooperative kernel's wait-limit self-test
};

namespace radm2 {
// Drop a cached split graph (its baked-in arguments changed).
void ctx_drop_graph(radm2_ctx *c);
// Learned seeding (radm2_mlp.cu): buffers, then the stream-ordered kernels.
int mlp_prepare_seed(radm2_ctx *c, radm2_mlp *m, int order);
cudaError_t mlp_enqueue_seed(radm2_ctx *c, radm2_mlp *m, double dt, int order, int lo = 0, int count = -1);
unsigned int mlp_generation(const radm2_mlp *m);
void mlp_detach(radm2_mlp *m);
}  // namespace radm2
