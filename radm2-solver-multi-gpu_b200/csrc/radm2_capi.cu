// C ABI of the B200 RADM2 solver (include/radm2.h): context, device buffers,
// IPAR/RPAR parsing with the reference's checks, kernel launches and the
// CUDA-graph operator-split loop.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/radm2.h"
#include "radm2_internal.h"
#include "gen/radm2_wrf.h"

using namespace radm2;

#include "radm2_ctx.h"

namespace {

int fail_cuda(radm2_ctx *c, cudaError_t e, const char *what)
{
    c->err = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return RADM2_E_NOMEM;
    return RADM2_E_CUDA;
}

#define CK(call)                                          \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return fail_cuda(c, e_, #call); \
    } while (0)

template <typename T>
int dalloc(radm2_ctx *c, T **p, size_t count)
{
    if (*p) {
        cudaFree(*p);
        *p = nullptr;
    }
    if (count == 0) return RADM2_OK;
    cudaError_t e = cudaMalloc((void **)p, count * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail_cuda(c, e, "cudaMalloc");
    }
    c->bytes += count * sizeof(T);
    return RADM2_OK;
}

void free_cells(radm2_ctx *c)
{
    void *ptrs[] = {c->var, c->fix, c->temp, c->rcn, c->jv, c->rconst, c->h0, c->order, c->status,
                    c->nacc, c->nrej, c->hfirst, c->hexit, c->texit};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    c->var = c->fix = c->temp = c->rcn = c->jv = c->rconst = nullptr;
    c->h0 = nullptr;
    c->order = nullptr;
    c->status = c->nacc = c->nrej = nullptr;
    c->hfirst = c->hexit = c->texit = nullptr;
    c->ncell = c->ld = 0;
    c->rconst_valid = false;
}

void drop_graph(radm2_ctx *c)
{
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    c->gexec = nullptr;
    c->gkey.clear();
    c->graph_kernels = 0;
}

// Kernel nodes of a captured graph (memset, copy and event nodes are not counted).
int count_kernel_nodes(cudaGraph_t g)
{
    size_t n = 0;
    if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess) return -1;
    std::vector<cudaGraphNode_t> nodes(n);
    if (n && cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return -1;
    int k = 0;
    for (size_t i = 0; i < n; i++) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) k++;
    }
    return k;
}

int ensure_cells(radm2_ctx *c, int ncell)
{
    if (ncell == c->ncell && c->var) return RADM2_OK;
    drop_graph(c);
    free_cells(c);
    const int ld = (ncell + 31) / 32 * 32;
    int rc;
    if ((rc = dalloc(c, &c->var, (size_t)NVAR * ld))) return rc;
    if ((rc = dalloc(c, &c->fix, (size_t)NFIX * ld))) return rc;
    if ((rc = dalloc(c, &c->temp, (size_t)ld))) return rc;
    if ((rc = dalloc(c, &c->rcn, (size_t)ld))) return rc;
    if ((rc = dalloc(c, &c->jv, (size_t)NPH * ld))) return rc;
    if ((rc = dalloc(c, &c->rconst, (size_t)NREACT * ld))) return rc;
    if ((rc = dalloc(c, &c->status, (size_t)ld))) return rc;
    if ((rc = dalloc(c, &c->nacc, (size_t)ld))) return rc;
    if ((rc = dalloc(c, &c->nrej, (size_t)ld))) return rc;
    if ((rc = dalloc(c, &c->hfirst, (size_t)ld))) return rc;
    if ((rc = dalloc(c, &c->hexit, (size_t)ld))) return rc;
    if ((rc = dalloc(c, &c->texit, (size_t)ld))) return rc;
    c->ncell = ncell;
    c->ld = ld;
    return RADM2_OK;
}

int ensure_stage(radm2_ctx *c, size_t bytes)
{
    if (bytes <= c->stage_bytes) return RADM2_OK;
    if (c->stage) cudaFree(c->stage);
    c->stage = nullptr;
    c->stage_bytes = 0;
    CK(cudaMalloc((void **)&c->stage, bytes));
    c->stage_bytes = bytes;
    return RADM2_OK;
}

int ensure_results(radm2_ctx *c, int n)
{
    if (n <= c->res_cap) return RADM2_OK;
    drop_graph(c);
    if (c->d_res) cudaFree(c->d_res);
    if (c->h_res) cudaFreeHost(c->h_res);
    if (c->queue) cudaFree(c->queue);
    c->d_res = nullptr;
    c->h_res = nullptr;
    c->queue = nullptr;
    c->res_cap = 0;
    CK(cudaMalloc((void **)&c->d_res, sizeof(RunResult) * n));
    CK(cudaMallocHost((void **)&c->h_res, sizeof(RunResult) * n));
    CK(cudaMalloc((void **)&c->queue, sizeof(int) * n));
    c->res_cap = n;
    return RADM2_OK;
}

// Upload host AoS [n][m] into device SoA [m][ld] through the staging buffer.
int upload_aos(radm2_ctx *c, const double *host, int m, double *dst)
{
    const size_t bytes = (size_t)c->ncell * m * sizeof(double);
    int rc = ensure_stage(c, bytes);
    if (rc) return rc;
    CK(cudaMemcpyAsync(c->stage, host, bytes, cudaMemcpyHostToDevice, c->st));
    CK(launch_aos_to_soa(c->ncell, m, c->ld, c->stage, dst, c->st));
    return RADM2_OK;
}

int download_aos(radm2_ctx *c, const double *src, int m, double *host)
{
    const size_t bytes = (size_t)c->ncell * m * sizeof(double);
    int rc = ensure_stage(c, bytes);
    if (rc) return rc;
    CK(launch_soa_to_aos(c->ncell, m, c->ld, src, c->stage, c->st));
    CK(cudaMemcpyAsync(host, c->stage, bytes, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return RADM2_OK;
}

// Unit roundoff computed as mgpu.cu:949-973 does (halving until 1 + eps == 1).
double wlamch()
{
    double eps = std::pow(0.5, 16);
    int i;
    for (i = 17; i <= 80; i++) {
        eps = eps * 0.5;
        volatile double suma = 1.0 + eps;
        if (suma <= 1.0) break;
    }
    if (i == 80) return 2.2e-16;
    return eps * 2.0;
}

inline double maxh(double a, double b) { return (a >= b) ? a : b; }
inline double minh(double b, double c) { return (b < c) ? b : c; }
inline double absh(double x) { return (x >= 0) ? x : -x; }

}  // namespace

// IPAR[10..16] (Nfun, Njac, Nstp, Nacc, Nrej, Ndec, Nsol; mgpu.cu:3835-3845) from the 64-bit
// totals of one integration.  Each slot saturates at INT_MAX instead of wrapping: the int
// counters of the reference's interface overflow on large batches (3 solves per attempt over
// 4M cells x 24 splits is ~2.4e9 solves).  radm2_stats keeps the exact 64-bit totals.
void radm2::add_step_counters(int *IPAR, long long nacc, long long nrej, long long nfail, int autonomous)
{
    const long long natt = nacc + nrej, nouter = nacc + nfail;
    const long long add[7] = {nouter * (autonomous ? 1 : 2) + natt, nouter, natt, nacc, nrej, natt, 3 * natt};
    for (int k = 0; k < 7; k++) {
        const long long v = (long long)IPAR[10 + k] + add[k];
        IPAR[10 + k] = v > INT_MAX ? INT_MAX : (v < INT_MIN ? INT_MIN : (int)v);
    }
}

// IPAR/RPAR parsing and validation, mgpu.cu:3684-3811 (same checks, same order, same codes).
int radm2::parse_params(double Tstart, double Tend, const double *AbsTol, const double *RelTol, const double *RPAR,
                 const int *IPAR, int float_coeffs, SolveParams *p, int *autonomous)
{
    static const double ros_M[3] = {RADM2_ROS_M0, RADM2_ROS_M1, RADM2_ROS_M2};
    static const double ros_E[3] = {RADM2_ROS_E0, RADM2_ROS_E1, RADM2_ROS_E2};
    std::memset(p, 0, sizeof *p);
    p->Tstart = Tstart;
    p->Tend = Tend;
    *autonomous = !(IPAR[0] == 0);
    const bool vector_tol = (IPAR[1] == 0);
    const int uplim = vector_tol ? NVAR : 1;
    int max_steps = (IPAR[2] == 0) ? 100000 : IPAR[2];
    if (max_steps < 0) return -1;
    if ((IPAR[3] < 1) || (IPAR[3] > 5)) return -2;
    p->Roundoff = wlamch();
    p->Hmin = RPAR[0];
    if (RPAR[0] < 0.0) return -3;
    p->Hmax = (RPAR[1] == 0.0) ? absh(Tend - Tstart) : minh(absh(RPAR[1]), absh(Tend - Tstart));
    if (RPAR[1] < 0.0) return -3;
    p->Hstart = (RPAR[2] == 0.0) ? maxh(p->Hmin, DELTA_MIN) : minh(absh(RPAR[2]), absh(Tend - Tstart));
    if (RPAR[2] < 0.0) return -3;
    p->FacMin = (RPAR[3] == 0.0) ? 0.2 : RPAR[3];
    if (RPAR[3] < 0.0) return -4;
    p->FacMax = (RPAR[4] == 0.0) ? 6.0 : RPAR[4];
    if (RPAR[4] < 0.0) return -4;
    p->FacRej = (RPAR[5] == 0.0) ? 0.1 : RPAR[5];
    if (RPAR[5] < 0.0) return -4;
    p->FacSafe = (RPAR[6] == 0.0) ? 0.9 : RPAR[6];
    if (RPAR[6] < 0.0) return -4;
    for (int i = 0; i < uplim; i++)
        if ((AbsTol[i] <= 0.0) || (RelTol[i] <= 10.0 * p->Roundoff) || (RelTol[i] >= 1.0)) return -5;
    if (IPAR[3] != 2) return -2;  // only ROS-3 is wired (mgpu.cu:3803-3811)
    for (int i = 0; i < NVAR; i++) {
        p->AbsTol[i] = vector_tol ? AbsTol[i] : AbsTol[0];
        p->RelTol[i] = vector_tol ? RelTol[i] : RelTol[0];
    }
    for (int i = 0; i < 3; i++) {
        p->M[i] = float_coeffs ? (double)(float)ros_M[i] : ros_M[i];
        p->E[i] = float_coeffs ? (double)(float)ros_E[i] : ros_E[i];
    }
    p->max_steps = max_steps;
    p->direction = (Tend >= Tstart) ? +1 : -1;
    return 1;
}

namespace {

int key_of(const radm2_ctx *c, int bs)
{
    return variant_key(bs, c->o.placement, c->o.min_blocks > 1 ? c->o.min_blocks : 1);
}

cudaError_t variant_info(radm2_ctx *c, int bs, SolverInfo *info)
{
    if (c->o.cells_per_thread == 2) return solver_info_cpt2(bs, c->o.schedule, info);
    if (c->o.schedule == RADM2_SCHED_COOP) {
        if (c->o.parity) return bs == 256 ? solver_info_coopx_g8(info) : cudaErrorInvalidValue;
        return bs == 128 ? solver_info_coop_g4(info) : bs == 256 ? solver_info_coop_g8(info) : cudaErrorInvalidValue;
    }
    const bool fp32 = c->o.precision == RADM2_PREC_FP32LU;
    const bool pers = c->o.schedule == RADM2_SCHED_PERSISTENT;
    const int k = key_of(c, bs);
    if (c->o.parity) return pers ? solver_info_fp64x_persistent(k, info) : solver_info_fp64x_static(k, info);
    if (fp32 && c->o.refine_sweeps == 0)
        return pers ? solver_info_fp32d_persistent(k, info) : solver_info_fp32d_static(k, info);
    if (fp32) return pers ? solver_info_fp32_persistent(k, info) : solver_info_fp32_static(k, info);
    return pers ? solver_info_fp64_persistent(k, info) : solver_info_fp64_static(k, info);
}

int default_block_threads(const radm2_opts &o)
{
    if (o.schedule == RADM2_SCHED_COOP) return 256;
    if (o.placement == RADM2_PLACE_GLOBAL || o.placement == RADM2_PLACE_LU_TMEM ||
        o.placement == RADM2_PLACE_LU_TMEM_WIDE)
        return 128;
    if (o.placement == RADM2_PLACE_LU_SMEM && o.precision == RADM2_PREC_FP32LU) return 64;
    return 32;
}

int launch_geometry(radm2_ctx *c, int *bs_out, int *grid_out, size_t *scratch_out)
{
    const int bs = c->o.block_threads ? c->o.block_threads : default_block_threads(c->o);
    SolverInfo info;
    cudaError_t e = variant_info(c, bs, &info);
    if (e != cudaSuccess || info.blocks_per_sm < 1) {
        c->err = "solver variant not built for this precision/placement/block size";
        (void)cudaGetLastError();
        return RADM2_E_ARG;
    }
    const int cpb = bs * (c->o.cells_per_thread == 2 ? 2 : 1);  // cells per block
    int grid;
    if (c->o.schedule == RADM2_SCHED_COOP) {  // 32 cells per block, one block per SM
        grid = c->nsm * info.blocks_per_sm;
        const int need = (c->ncell + 31) / 32;
        if (grid > need) grid = need;
    } else if (c->o.schedule == RADM2_SCHED_PERSISTENT) {
        int bpsm = c->o.blocks_per_sm > 0 ? c->o.blocks_per_sm : info.blocks_per_sm;
        if (bpsm > info.blocks_per_sm) bpsm = info.blocks_per_sm;
        grid = c->nsm * bpsm;
        const int need = (c->ncell + cpb - 1) / cpb;
        if (grid > need) grid = need;
    } else {
        grid = (c->ncell + cpb - 1) / cpb;
    }
    if (grid < 1) grid = 1;
    *bs_out = bs;
    *grid_out = grid;
    *scratch_out = (size_t)grid * bs * info.global_words * sizeof(double);
    if (c->o.schedule == RADM2_SCHED_COOP)  // per block: the rate constants of its 32 cells
        *scratch_out = (size_t)grid * NREACT * 32 * sizeof(double);
    return RADM2_OK;
}

int ensure_scratch(radm2_ctx *c, size_t bytes)
{
    if (bytes <= c->scratch_bytes) return RADM2_OK;
    drop_graph(c);
    if (c->scratch) cudaFree(c->scratch);
    c->scratch = nullptr;
    c->scratch_bytes = 0;
    CK(cudaMalloc((void **)&c->scratch, bytes));
    c->scratch_bytes = bytes;
    return RADM2_OK;
}

SolveArgs make_args(radm2_ctx *c, const SolveParams &p, int *queue)
{
    SolveArgs a;
    std::memset(&a, 0, sizeof a);
    a.p = p;
    a.ncell = c->ncell;
    a.ld = c->ld;
    a.var = c->var;
    a.fix = c->fix;
    a.rconst = c->rconst;
    a.h0 = c->use_h0 ? c->h0 : nullptr;
    a.order = c->use_order ? c->order : nullptr;
    a.queue = queue;
    a.scratch = c->scratch;
    a.status = c->status;
    a.nacc = c->nacc;
    a.nrej = c->nrej;
    a.hfirst = c->hfirst;
    a.hexit = c->hexit;
    a.texit = c->texit;
    a.refine = c->o.refine_sweeps;
    a.coop_selftest = c->coop_selftest;
    return a;
}

cudaError_t launch_solver(radm2_ctx *c, const SolveArgs &a, int bs, int grid)
{
    const bool fp32 = c->o.precision == RADM2_PREC_FP32LU;
    const bool pers = c->o.schedule == RADM2_SCHED_PERSISTENT;
    const int k = key_of(c, bs);
    if (c->o.cells_per_thread == 2) return launch_solver_cpt2(a, bs, c->o.schedule, grid, c->st);
    if (c->o.schedule == RADM2_SCHED_COOP) {
        if (c->o.parity) return launch_solver_coopx_g8(a, grid, c->st);
        return bs == 128 ? launch_solver_coop_g4(a, grid, c->st) : launch_solver_coop_g8(a, grid, c->st);
    }
    if (c->o.parity)  // reference arithmetic: divisions kept, no multiply-add contraction
        return pers ? launch_solver_fp64x_persistent(a, k, grid, c->st) : launch_solver_fp64x_static(a, k, grid, c->st);
    if (fp32 && c->o.refine_sweeps == 0)  // the variants without the refinement code
        return pers ? launch_solver_fp32d_persistent(a, k, grid, c->st) : launch_solver_fp32d_static(a, k, grid, c->st);
    if (fp32)
        return pers ? launch_solver_fp32_persistent(a, k, grid, c->st) : launch_solver_fp32_static(a, k, grid, c->st);
    return pers ? launch_solver_fp64_persistent(a, k, grid, c->st) : launch_solver_fp64_static(a, k, grid, c->st);
}

// Record a kernel-timing event.  Under stream capture the External flag makes the record
// a graph node (re-recorded on every replay); outside capture it is a plain record (the
// flag is only valid while capturing).
cudaError_t record_timing_event(radm2_ctx *c, cudaEvent_t ev)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(c->st, &cs);
    if (e != cudaSuccess) return e;
    return cs == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(ev, c->st, cudaEventRecordExternal)
                                               : cudaEventRecord(ev, c->st);
}

// Enqueue one integration of every cell: queue reset, solver, outcome reduction into d_res[slot].
int enqueue_integration(radm2_ctx *c, const SolveParams &p, int slot, int bs, int grid)
{
    if (c->mlp) CK(mlp_enqueue_seed(c, c->mlp, std::fabs(p.Tend - p.Tstart), c->mlp_order));
    CK(cudaMemsetAsync(c->queue + slot, 0, sizeof(int), c->st));
    SolveArgs a = make_args(c, p, c->queue + slot);
    if (c->timing) {
        while ((int)c->ev.size() < 2 * (slot + 1)) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            c->ev.push_back(e);
        }
        CK(record_timing_event(c, c->ev[2 * slot]));
    }
    CK(launch_solver(c, a, bs, grid));
    if (c->timing) {
        CK(record_timing_event(c, c->ev[2 * slot + 1]));
        if (slot + 1 > c->ev_used) c->ev_used = slot + 1;
    }
    CK(launch_reduce(c->ncell, c->status, c->nacc, c->nrej, c->texit, c->hexit, c->partials, c->d_res + slot, c->st));
    return RADM2_OK;
}

int ensure_rconst(radm2_ctx *c)
{
    if (c->rconst_valid) return RADM2_OK;
    CK(launch_rconst(c->ncell, c->ld, c->jv, c->temp, c->fix, c->have_rcn ? c->rcn : nullptr, c->rconst, c->st));
    c->rconst_valid = true;
    return RADM2_OK;
}

// Fold results of nres integrations into IPAR/RPAR/stats; returns IERR.
int finish(radm2_ctx *c, int nres, int autonomous, double *RPAR, int *IPAR, int direction)
{
    if (c->timing) {
        for (int i = 0; i < c->ev_used && i < nres; i++) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, c->ev[2 * i], c->ev[2 * i + 1]) == cudaSuccess) {
                c->kernel_ms += ms;
                c->kernel_launches++;
            } else {
                (void)cudaGetLastError();
            }
        }
        c->ev_used = 0;
    }
    long long nacc = 0, nrej = 0, nfail = 0;
    int worst = 1, max_att = 0;
    double tmin = 0, tmax = 0, hmin = 0;
    for (int i = 0; i < nres; i++) {
        const RunResult &r = c->h_res[i];
        nacc += r.nacc;
        nrej += r.nrej;
        nfail += r.nfail;
        if (r.worst < worst) worst = r.worst;
        if (r.max_att > max_att) max_att = r.max_att;
        if (i == nres - 1) {
            tmin = r.tmin;
            tmax = r.tmax;
            hmin = r.hmin;
        }
    }
    add_step_counters(IPAR, nacc, nrej, nfail, autonomous);
    RPAR[10] = direction > 0 ? tmin : tmax;
    RPAR[11] = hmin;
    c->stats.n_accepted = nacc;
    c->stats.n_rejected = nrej;
    c->stats.n_failed = nfail;
    c->stats.worst_status = worst;
    if (worst == RADM2_E_CUDA) c->err = "solver: a bounded wait between cooperating warps ran out";
    c->stats.max_steps_cell = max_att;
    c->stats.texit_min = RPAR[10];
    c->stats.hexit_min = hmin;
    return worst;
}

bool valid_ctx(const radm2_ctx *c) { return c != nullptr; }

}  // namespace

void radm2::ctx_drop_graph(radm2_ctx *c) { drop_graph(c); }

extern "C" {

int radm2_opts_default(radm2_opts *o)
{
    if (!o) return RADM2_E_ARG;
    std::memset(o, 0, sizeof *o);
    o->device = 0;
    o->precision = RADM2_PREC_FP64;
    o->refine_sweeps = 1;
    o->schedule = RADM2_SCHED_STATIC;
    o->block_threads = 0;
    o->blocks_per_sm = 0;
    o->float_coeffs = 1;
    o->placement = RADM2_PLACE_GLOBAL;
    o->min_blocks = 0;
    o->parity = 0;
    o->cells_per_thread = 1;
    return RADM2_OK;
}

int radm2_create(radm2_ctx **out, const radm2_opts *opts)
{
    if (!out) return RADM2_E_ARG;
    *out = nullptr;
    radm2_opts o;
    if (opts)
        o = *opts;
    else
        radm2_opts_default(&o);
    if (o.precision != RADM2_PREC_FP64 && o.precision != RADM2_PREC_FP32LU) return RADM2_E_ARG;
    if (o.schedule != RADM2_SCHED_STATIC && o.schedule != RADM2_SCHED_PERSISTENT && o.schedule != RADM2_SCHED_COOP)
        return RADM2_E_ARG;
    if (o.schedule == RADM2_SCHED_COOP &&
        (o.precision != RADM2_PREC_FP64 || o.placement != RADM2_PLACE_GLOBAL || o.min_blocks > 1))
        return RADM2_E_ARG;
    if (o.refine_sweeps < 0 || o.refine_sweeps > 2) return RADM2_E_ARG;
    if (o.placement != RADM2_PLACE_GLOBAL && o.placement != RADM2_PLACE_LU_SMEM && o.placement != RADM2_PLACE_ALL_SMEM &&
        o.placement != RADM2_PLACE_LU_TMEM && o.placement != RADM2_PLACE_LU_TMEM_WIDE)
        return RADM2_E_ARG;
    if (o.placement == RADM2_PLACE_LU_TMEM && o.precision != RADM2_PREC_FP64) return RADM2_E_ARG;
    if (o.placement == RADM2_PLACE_LU_TMEM_WIDE && (o.precision != RADM2_PREC_FP64 || o.schedule != RADM2_SCHED_PERSISTENT))
        return RADM2_E_ARG;
    if (o.parity != 0 && o.parity != 1) return RADM2_E_ARG;
    if (o.cells_per_thread == 0) o.cells_per_thread = 1;
    if (o.cells_per_thread != 1 && o.cells_per_thread != 2) return RADM2_E_ARG;
    if (o.cells_per_thread == 2 && (o.precision != RADM2_PREC_FP64 || o.placement != RADM2_PLACE_GLOBAL ||
                                    o.min_blocks > 1 || o.parity || o.schedule == RADM2_SCHED_COOP))
        return RADM2_E_ARG;
    if (o.parity && (o.precision != RADM2_PREC_FP64 || (o.placement != RADM2_PLACE_GLOBAL &&
                                                         o.placement != RADM2_PLACE_LU_TMEM &&
                                                         o.placement != RADM2_PLACE_LU_TMEM_WIDE)))
        return RADM2_E_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= o.device || o.device < 0) return RADM2_E_NODEV;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, o.device) != cudaSuccess) return RADM2_E_NODEV;
    if (prop.major != 10) return RADM2_E_NODEV;  // built for sm_100a only
    radm2_ctx *c = new radm2_ctx();
    c->o = o;
    c->nsm = prop.multiProcessorCount;
    if (cudaSetDevice(o.device) != cudaSuccess || cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return RADM2_E_CUDA;
    }
    c->st = c->own;
    if (cudaMalloc(&c->partials, reduce_partials_bytes()) != cudaSuccess || ensure_results(c, 8) != RADM2_OK) {
        radm2_destroy(c);
        return RADM2_E_NOMEM;
    }
    *out = c;
    return RADM2_OK;
}

int radm2_destroy(radm2_ctx *c)
{
    if (!c) return RADM2_E_ARG;
    cudaSetDevice(c->o.device);
    if (c->st) cudaStreamSynchronize(c->st);
    drop_graph(c);
    free_cells(c);
    for (cudaEvent_t e : c->ev) cudaEventDestroy(e);
    cudaFree(c->seed_keys);
    cudaFree(c->seed_idx);
    cudaFree(c->seed_tmp);
    cudaFree(c->seed_x);
    cudaFree(c->seed_y);
    if (c->mlp) radm2::mlp_detach(c->mlp);
    if (c->scratch) cudaFree(c->scratch);
    if (c->stage) cudaFree(c->stage);
    if (c->partials) cudaFree(c->partials);
    if (c->d_res) cudaFree(c->d_res);
    if (c->h_res) cudaFreeHost(c->h_res);
    if (c->queue) cudaFree(c->queue);
    for (cudaEvent_t e : c->pipe_ev) cudaEventDestroy(e);
    if (c->st_up) cudaStreamDestroy(c->st_up);
    if (c->st_down) cudaStreamDestroy(c->st_down);
    if (c->own) cudaStreamDestroy(c->own);
    delete c;
    return RADM2_OK;
}

const char *radm2_error_string(int code)
{
    switch (code) {
        case 1: return "success";
        case 0: return "ok";
        case -1: return "Improper value for maximal no of steps";
        case -2: return "Selected Rosenbrock method not implemented";
        case -3: return "Hmin/Hmax/Hstart must be positive";
        case -4: return "FacMin/FacMax/FacRej must be positive";
        case -5: return "Improper tolerance values";
        case -6: return "No of steps exceeds maximum bound";
        case -7: return "Step size too small (T + H/10 = T) or H < Roundoff";
        case -8: return "Matrix is repeatedly singular";
        case RADM2_E_ARG: return "invalid argument";
        case RADM2_E_CUDA: return "CUDA runtime error";
        case RADM2_E_NOMEM: return "device allocation failed";
        case RADM2_E_STATE: return "call out of order";
        case RADM2_E_NODEV: return "no usable sm_100 device";
        case RADM2_E_TOOBIG: return "size exceeds the documented maximum";
        default: return "unknown error code";
    }
}

const char *radm2_last_error(const radm2_ctx *c) { return c ? c->err.c_str() : "null context"; }

int radm2_set_stream(radm2_ctx *c, void *stream)
{
    if (!valid_ctx(c)) return RADM2_E_ARG;
    drop_graph(c);
    c->st = stream ? (cudaStream_t)stream : c->own;
    return RADM2_OK;
}

int radm2_synchronize(radm2_ctx *c)
{
    if (!valid_ctx(c)) return RADM2_E_ARG;
    CK(cudaStreamSynchronize(c->st));
    return RADM2_OK;
}

int radm2_set_inputs(radm2_ctx *c, int ncell, const double *VAR, const double *FIX, const double *TEMP,
                     const double *RC_N2O5, const double *JV)
{
    if (!valid_ctx(c) || ncell <= 0 || !VAR || !FIX || !TEMP || !JV) return RADM2_E_ARG;
    CK(cudaSetDevice(c->o.device));
    int rc = ensure_cells(c, ncell);
    if (rc) return rc;
    if ((rc = upload_aos(c, VAR, NVAR, c->var))) return rc;
    if ((rc = upload_aos(c, FIX, NFIX, c->fix))) return rc;
    if ((rc = upload_aos(c, JV, NPH, c->jv))) return rc;
    CK(cudaMemcpyAsync(c->temp, TEMP, sizeof(double) * ncell, cudaMemcpyHostToDevice, c->st));
    c->have_rcn = RC_N2O5 != nullptr;
    if (RC_N2O5) CK(cudaMemcpyAsync(c->rcn, RC_N2O5, sizeof(double) * ncell, cudaMemcpyHostToDevice, c->st));
    c->rconst_valid = false;
    return RADM2_OK;
}

int radm2_set_state(radm2_ctx *c, const double *VAR)
{
    if (!valid_ctx(c) || !VAR) return RADM2_E_ARG;
    if (!c->var) return RADM2_E_STATE;
    return upload_aos(c, VAR, NVAR, c->var);
}

int radm2_get_state(radm2_ctx *c, double *VAR)
{
    if (!valid_ctx(c) || !VAR) return RADM2_E_ARG;
    if (!c->var) return RADM2_E_STATE;
    return download_aos(c, c->var, NVAR, VAR);
}

int radm2_get_inputs(radm2_ctx *c, double *VAR, double *FIX, double *TEMP, double *RC_N2O5, double *JV)
{
    if (!valid_ctx(c)) return RADM2_E_ARG;
    if (!c->var) return RADM2_E_STATE;
    int rc = RADM2_OK;
    if (VAR && (rc = download_aos(c, c->var, NVAR, VAR))) return rc;
    if (FIX && (rc = download_aos(c, c->fix, NFIX, FIX))) return rc;
    if (TEMP && (rc = download_aos(c, c->temp, 1, TEMP))) return rc;
    if (RC_N2O5) {
        if (!c->have_rcn) return RADM2_E_STATE;  // inputs came without rc_n2o5 (formula used)
        if ((rc = download_aos(c, c->rcn, 1, RC_N2O5))) return rc;
    }
    if (JV && (rc = download_aos(c, c->jv, NPH, JV))) return rc;
    return RADM2_OK;
}

int radm2_set_inputs_device(radm2_ctx *c, int ncell, int ld, const double *var, const double *fix,
                            const double *temp, const double *rc_n2o5, const double *jv)
{
    if (!valid_ctx(c) || ncell <= 0 || ld < ncell || !var || !fix || !temp || !jv) return RADM2_E_ARG;
    CK(cudaSetDevice(c->o.device));
    int rc = ensure_cells(c, ncell);
    if (rc) return rc;
    const size_t w = sizeof(double) * ncell, sp = sizeof(double) * ld, dp = sizeof(double) * c->ld;
    CK(cudaMemcpy2DAsync(c->var, dp, var, sp, w, NVAR, cudaMemcpyDeviceToDevice, c->st));
    CK(cudaMemcpy2DAsync(c->fix, dp, fix, sp, w, NFIX, cudaMemcpyDeviceToDevice, c->st));
    CK(cudaMemcpy2DAsync(c->jv, dp, jv, sp, w, NPH, cudaMemcpyDeviceToDevice, c->st));
    CK(cudaMemcpyAsync(c->temp, temp, w, cudaMemcpyDeviceToDevice, c->st));
    c->have_rcn = rc_n2o5 != nullptr;
    if (rc_n2o5) CK(cudaMemcpyAsync(c->rcn, rc_n2o5, w, cudaMemcpyDeviceToDevice, c->st));
    c->rconst_valid = false;
    return RADM2_OK;
}

int radm2_get_state_device(radm2_ctx *c, double *var, int ld)
{
    if (!valid_ctx(c) || !var || ld < c->ncell) return RADM2_E_ARG;
    if (!c->var) return RADM2_E_STATE;
    CK(cudaMemcpy2DAsync(var, sizeof(double) * ld, c->var, sizeof(double) * c->ld, sizeof(double) * c->ncell, NVAR,
                         cudaMemcpyDeviceToDevice, c->st));
    return RADM2_OK;
}

int radm2_set_state_device(radm2_ctx *c, const double *var, int ld)
{
    if (!valid_ctx(c) || !var || ld < c->ncell) return RADM2_E_ARG;
    if (!c->var) return RADM2_E_STATE;
    CK(cudaMemcpy2DAsync(c->var, sizeof(double) * c->ld, var, sizeof(double) * ld, sizeof(double) * c->ncell, NVAR,
                         cudaMemcpyDeviceToDevice, c->st));
    return RADM2_OK;
}

int radm2_update_rconst(radm2_ctx *c)
{
    if (!valid_ctx(c)) return RADM2_E_ARG;
    if (!c->var) return RADM2_E_STATE;
    c->rconst_valid = false;
    return ensure_rconst(c);
}

int radm2_get_rconst(radm2_ctx *c, double *RCONST)
{
    if (!valid_ctx(c) || !RCONST) return RADM2_E_ARG;
    if (!c->var) return RADM2_E_STATE;
    int rc = ensure_rconst(c);
    if (rc) return rc;
    return download_aos(c, c->rconst, NREACT, RCONST);
}

int radm2_set_rconst(radm2_ctx *c, const double *RCONST)
{
    if (!valid_ctx(c) || !RCONST) return RADM2_E_ARG;
    if (!c->var) return RADM2_E_STATE;
    int rc = upload_aos(c, RCONST, NREACT, c->rconst);
    if (rc) return rc;
    c->rconst_valid = true;
    return RADM2_OK;
}

int radm2_rosenbrock(radm2_ctx *c, double Tstart, double Tend, const double *AbsTol, const double *RelTol,
                     double *RPAR, int *IPAR)
{
    if (!valid_ctx(c) || !AbsTol || !RelTol || !RPAR || !IPAR) return RADM2_E_ARG;
    if (!c->var) return RADM2_E_STATE;
    CK(cudaSetDevice(c->o.device));
    SolveParams p;
    int autonomous = 1;
    int ierr = parse_params(Tstart, Tend, AbsTol, RelTol, RPAR, IPAR, c->o.float_coeffs, &p, &autonomous);
    if (ierr != 1) return ierr;
    int rc = ensure_rconst(c);
    if (rc) return rc;
    int bs, grid;
    size_t sbytes;
    if ((rc = launch_geometry(c, &bs, &grid, &sbytes))) return rc;
    if ((rc = ensure_scratch(c, sbytes))) return rc;
    if (c->mlp && (rc = mlp_prepare_seed(c, c->mlp, c->mlp_order))) return rc;
    if ((rc = enqueue_integration(c, p, 0, bs, grid))) return rc;
    CK(cudaMemcpyAsync(c->h_res, c->d_res, sizeof(RunResult), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return finish(c, 1, autonomous, RPAR, IPAR, p.direction);
}

// Host-buffer integration with the transfers hidden behind the solve: the batch is cut into
// nchunk consecutive chunks.  Chunk k's inputs go up (copy stream, then a transpose to the
// struct-of-arrays arrays) while chunk k-1 integrates (rate constants, optional seeding,
// solver, statistics on the context's stream) and chunk k-2's states come back (transpose
// and copy on a second copy stream).  Events order each chunk's three steps.
int radm2_rosenbrock_host(radm2_ctx *c, int ncell, double *VAR, const double *FIX, const double *TEMP,
                          const double *RC_N2O5, const double *JV, double Tstart, double Tend, const double *AbsTol,
                          const double *RelTol, double *RPAR, int *IPAR, int nchunk)
{
    if (!valid_ctx(c) || ncell <= 0 || !VAR || !FIX || !TEMP || !JV || !AbsTol || !RelTol || !RPAR || !IPAR)
        return RADM2_E_ARG;
    CK(cudaSetDevice(c->o.device));
    SolveParams p;
    int autonomous = 1;
    int ierr = parse_params(Tstart, Tend, AbsTol, RelTol, RPAR, IPAR, c->o.float_coeffs, &p, &autonomous);
    if (ierr != 1) return ierr;
    int rc = ensure_cells(c, ncell);
    if (rc) return rc;
    c->have_rcn = RC_N2O5 != nullptr;
    c->rconst_valid = false;  // recomputed per chunk below
    nchunk = std::max(1, std::min(nchunk, (ncell + 1023) / 1024));
    int bs, grid;
    size_t sbytes;
    if ((rc = launch_geometry(c, &bs, &grid, &sbytes))) return rc;
    if ((rc = ensure_scratch(c, sbytes))) return rc;
    if ((rc = ensure_results(c, nchunk))) return rc;
    if (c->mlp && (rc = mlp_prepare_seed(c, c->mlp, 0))) return rc;
    // staging: inputs in the reference layout (VAR, FIX, TEMP, RC_N2O5, JV), then the states
    const int win = NVAR + NFIX + 2 + NPH;
    const size_t n = (size_t)ncell;
    if ((rc = ensure_stage(c, sizeof(double) * n * (win + NVAR)))) return rc;
    double *sv = c->stage, *sf = sv + n * NVAR, *st_ = sf + n * NFIX, *sr = st_ + n, *sj = sr + n, *so = sj + n * NPH;
    if (!c->st_up) CK(cudaStreamCreateWithFlags(&c->st_up, cudaStreamNonBlocking));
    if (!c->st_down) CK(cudaStreamCreateWithFlags(&c->st_down, cudaStreamNonBlocking));
    while ((int)c->pipe_ev.size() < 2 * nchunk) {
        cudaEvent_t e;
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        c->pipe_ev.push_back(e);
    }
    const bool order_was = c->use_order;
    c->use_order = false;  // a chunk's cells are integrated in index order
    const double dt = std::fabs(p.Tend - p.Tstart);
    // Chunk sizes: with three or more chunks the first and the last are a fifth of a middle
    // one.  Only the first chunk's upload and the last chunk's download are not hidden
    // behind an integration, and a cell's copies take a fraction of its integration time,
    // so small edge chunks still cover the middle chunks' copies.
    std::vector<size_t> bound(nchunk + 1, 0);
    {
        const double edge = nchunk >= 3 ? 0.2 : 1.0, total = 2.0 * edge + (nchunk - 2 > 0 ? nchunk - 2 : 0);
        double acc = 0.0;
        for (int k = 0; k < nchunk; k++) {
            acc += (k == 0 || k == nchunk - 1) ? edge : 1.0;
            bound[k + 1] = (k == nchunk - 1) ? n : (size_t)((double)n * (acc / total));
        }
        bool ok = true;
        for (int k = 0; k < nchunk; k++) ok = ok && bound[k + 1] > bound[k];
        if (!ok)  // (not reached: a chunk holds at least 1024 cells) equal chunks
            for (int k = 0; k <= nchunk; k++) bound[k] = n * (size_t)k / (size_t)nchunk;
    }
    for (int k = 0; k < nchunk; k++) {
        const int lo = (int)bound[k], hi = (int)bound[k + 1], m = hi - lo;
        const size_t l = (size_t)lo;
        // up: copies of this chunk's rows, then the transposes into the cell arrays
        CK(cudaMemcpyAsync(sv + l * NVAR, VAR + l * NVAR, sizeof(double) * m * NVAR, cudaMemcpyHostToDevice, c->st_up));
        CK(cudaMemcpyAsync(sf + l * NFIX, FIX + l * NFIX, sizeof(double) * m * NFIX, cudaMemcpyHostToDevice, c->st_up));
        CK(cudaMemcpyAsync(st_ + l, TEMP + l, sizeof(double) * m, cudaMemcpyHostToDevice, c->st_up));
        if (RC_N2O5) CK(cudaMemcpyAsync(sr + l, RC_N2O5 + l, sizeof(double) * m, cudaMemcpyHostToDevice, c->st_up));
        CK(cudaMemcpyAsync(sj + l * NPH, JV + l * NPH, sizeof(double) * m * NPH, cudaMemcpyHostToDevice, c->st_up));
        CK(launch_aos_to_soa(m, NVAR, c->ld, sv + l * NVAR, c->var + lo, c->st_up));
        CK(launch_aos_to_soa(m, NFIX, c->ld, sf + l * NFIX, c->fix + lo, c->st_up));
        CK(cudaMemcpyAsync(c->temp + lo, st_ + l, sizeof(double) * m, cudaMemcpyDeviceToDevice, c->st_up));
        if (RC_N2O5) CK(cudaMemcpyAsync(c->rcn + lo, sr + l, sizeof(double) * m, cudaMemcpyDeviceToDevice, c->st_up));
        CK(launch_aos_to_soa(m, NPH, c->ld, sj + l * NPH, c->jv + lo, c->st_up));
        CK(cudaEventRecord(c->pipe_ev[2 * k], c->st_up));
        // integrate the chunk
        CK(cudaStreamWaitEvent(c->st, c->pipe_ev[2 * k], 0));
        CK(launch_rconst(m, c->ld, c->jv + lo, c->temp + lo, c->fix + lo, RC_N2O5 ? c->rcn + lo : nullptr,
                         c->rconst + lo, c->st));
        if (c->mlp) CK(mlp_enqueue_seed(c, c->mlp, dt, 0, lo, m));
        CK(cudaMemsetAsync(c->queue + k, 0, sizeof(int), c->st));
        SolveArgs a = make_args(c, p, c->queue + k);
        a.ncell = m;
        a.var += lo;
        a.fix += lo;
        a.rconst += lo;
        if (a.h0) a.h0 += lo;
        a.status += lo;
        a.nacc += lo;
        a.nrej += lo;
        a.hfirst += lo;
        a.hexit += lo;
        a.texit += lo;
        int kg = grid;
        const int cpb = bs * (c->o.cells_per_thread == 2 ? 2 : 1);
        if (c->o.schedule == RADM2_SCHED_COOP) kg = std::min(grid, (m + 31) / 32);
        else if (c->o.schedule == RADM2_SCHED_PERSISTENT) kg = std::min(grid, (m + cpb - 1) / cpb);
        else kg = (m + cpb - 1) / cpb;
        CK(launch_solver(c, a, bs, std::max(kg, 1)));
        CK(launch_reduce(m, c->status + lo, c->nacc + lo, c->nrej + lo, c->texit + lo, c->hexit + lo, c->partials,
                         c->d_res + k, c->st));
        CK(cudaEventRecord(c->pipe_ev[2 * k + 1], c->st));
        // down: this chunk's states
        CK(cudaStreamWaitEvent(c->st_down, c->pipe_ev[2 * k + 1], 0));
        CK(launch_soa_to_aos(m, NVAR, c->ld, c->var + lo, so + l * NVAR, c->st_down));
        CK(cudaMemcpyAsync(VAR + l * NVAR, so + l * NVAR, sizeof(double) * m * NVAR, cudaMemcpyDeviceToHost,
                           c->st_down));
    }
    c->use_order = order_was;
    CK(cudaMemcpyAsync(c->h_res, c->d_res, sizeof(RunResult) * nchunk, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    CK(cudaStreamSynchronize(c->st_down));
    CK(cudaStreamSynchronize(c->st_up));
    // one result over all chunks: counters summed, exit times and steps at their extremes
    RunResult tot = c->h_res[0];
    for (int k = 1; k < nchunk; k++) {
        const RunResult &r = c->h_res[k];
        tot.nacc += r.nacc;
        tot.nrej += r.nrej;
        tot.nfail += r.nfail;
        tot.worst = std::min(tot.worst, r.worst);
        tot.max_att = std::max(tot.max_att, r.max_att);
        tot.tmin = std::min(tot.tmin, r.tmin);
        tot.tmax = std::max(tot.tmax, r.tmax);
        tot.hmin = std::min(tot.hmin, r.hmin);
    }
    c->h_res[0] = tot;
    c->rconst_valid = true;
    return finish(c, 1, autonomous, RPAR, IPAR, p.direction);
}

int radm2_run_split(radm2_ctx *c, int nsplit, double dt, const double *AbsTol, const double *RelTol, double *RPAR,
                    int *IPAR, int use_graph)
{
    if (!valid_ctx(c) || nsplit <= 0 || !(dt > 0.0) || !AbsTol || !RelTol || !RPAR || !IPAR) return RADM2_E_ARG;
    if (!c->var) return RADM2_E_STATE;
    CK(cudaSetDevice(c->o.device));
    double rpar[20];
    std::memcpy(rpar, RPAR, sizeof rpar);
    if (rpar[2] == 0.0) rpar[2] = 0.01 * dt;  // the reference driver's Hstart ratio (mgpu.cu:3873)
    SolveParams p;
    int autonomous = 1;
    int ierr = parse_params(0.0, dt, AbsTol, RelTol, rpar, IPAR, c->o.float_coeffs, &p, &autonomous);
    if (ierr != 1) return ierr;
    int rc = ensure_rconst(c);
    if (rc) return rc;
    int bs, grid;
    size_t sbytes;
    if ((rc = launch_geometry(c, &bs, &grid, &sbytes))) return rc;
    if ((rc = ensure_scratch(c, sbytes))) return rc;
    if ((rc = ensure_results(c, nsplit))) return rc;
    if (c->mlp && (rc = mlp_prepare_seed(c, c->mlp, c->mlp_order))) return rc;
    if (!use_graph) {
        for (int s = 0; s < nsplit; s++)
            if ((rc = enqueue_integration(c, p, s, bs, grid))) return rc;
        CK(cudaMemcpyAsync(c->h_res, c->d_res, sizeof(RunResult) * nsplit, cudaMemcpyDeviceToHost, c->st));
    } else {
        // The graph bakes in the launch arguments; rebuild it when any of them change.
        SolveArgs a0 = make_args(c, p, c->queue);
        const uintptr_t extra[9] = {(uintptr_t)nsplit,
                                    (uintptr_t)bs,
                                    (uintptr_t)grid,
                                    (uintptr_t)((c->o.cells_per_thread * 64 + c->o.parity * 16 + c->o.precision * 4 +
                                                 c->o.schedule) * (1ull << 32) +
                                                (unsigned)key_of(c, bs)),
                                    reinterpret_cast<uintptr_t>(c->mlp),
                                    (uintptr_t)mlp_generation(c->mlp),
                                    (uintptr_t)c->mlp_order,
                                    reinterpret_cast<uintptr_t>(c->seed_x),
                                    reinterpret_cast<uintptr_t>(c->seed_keys)};
        std::vector<unsigned char> key(sizeof a0 + sizeof extra);
        std::memcpy(key.data(), &a0, sizeof a0);
        std::memcpy(key.data() + sizeof a0, extra, sizeof extra);
        if (!c->gexec || key != c->gkey) {
            drop_graph(c);
            cudaGraph_t g;
            CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
            for (int s = 0; s < nsplit && rc == RADM2_OK; s++) rc = enqueue_integration(c, p, s, bs, grid);
            if (rc == RADM2_OK) {
                cudaError_t e = cudaMemcpyAsync(c->h_res, c->d_res, sizeof(RunResult) * nsplit,
                                                cudaMemcpyDeviceToHost, c->st);
                if (e != cudaSuccess) rc = fail_cuda(c, e, "capture memcpy");
            }
            cudaError_t e = cudaStreamEndCapture(c->st, &g);
            if (rc) return rc;
            if (e != cudaSuccess) return fail_cuda(c, e, "cudaStreamEndCapture");
            c->graph_kernels = count_kernel_nodes(g);
            e = cudaGraphInstantiate(&c->gexec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                c->gexec = nullptr;
                return fail_cuda(c, e, "cudaGraphInstantiate");
            }
            c->gkey = key;
        }
        if (c->timing) c->ev_used = nsplit;  // the graph's event nodes re-record every replay
        CK(cudaGraphLaunch(c->gexec, c->st));
    }
    CK(cudaStreamSynchronize(c->st));
    return finish(c, nsplit, autonomous, RPAR, IPAR, p.direction);
}

int radm2_get_cell_stats(radm2_ctx *c, int *status, int *nacc, int *nrej, double *hfirst, double *hexit)
{
    if (!valid_ctx(c)) return RADM2_E_ARG;
    if (!c->var) return RADM2_E_STATE;
    const int n = c->ncell;
    if (status) CK(cudaMemcpyAsync(status, c->status, sizeof(int) * n, cudaMemcpyDeviceToHost, c->st));
    if (nacc) CK(cudaMemcpyAsync(nacc, c->nacc, sizeof(int) * n, cudaMemcpyDeviceToHost, c->st));
    if (nrej) CK(cudaMemcpyAsync(nrej, c->nrej, sizeof(int) * n, cudaMemcpyDeviceToHost, c->st));
    if (hfirst) CK(cudaMemcpyAsync(hfirst, c->hfirst, sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
    if (hexit) CK(cudaMemcpyAsync(hexit, c->hexit, sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return RADM2_OK;
}

int radm2_add_step_counters(int *IPAR, long long n_accepted, long long n_rejected, long long n_failed, int autonomous)
{
    if (!IPAR || n_accepted < 0 || n_rejected < 0 || n_failed < 0) return RADM2_E_ARG;
    add_step_counters(IPAR, n_accepted, n_rejected, n_failed, autonomous);
    return RADM2_OK;
}

int radm2_get_stats(radm2_ctx *c, radm2_stats *out)
{
    if (!valid_ctx(c) || !out) return RADM2_E_ARG;
    *out = c->stats;
    return RADM2_OK;
}

int radm2_set_cell_hstart(radm2_ctx *c, const double *h0)
{
    if (!valid_ctx(c)) return RADM2_E_ARG;
    if (!c->var) return RADM2_E_STATE;
    drop_graph(c);
    if (!h0) {
        if (c->h0) cudaFree(c->h0);
        c->h0 = nullptr;
        return RADM2_OK;
    }
    if (!c->h0) CK(cudaMalloc((void **)&c->h0, sizeof(double) * c->ld));
    CK(cudaMemcpyAsync(c->h0, h0, sizeof(double) * c->ncell, cudaMemcpyHostToDevice, c->st));
    c->use_h0 = true;
    return RADM2_OK;
}

int radm2_set_cell_order(radm2_ctx *c, const int *order)
{
    if (!valid_ctx(c)) return RADM2_E_ARG;
    if (!c->var) return RADM2_E_STATE;
    drop_graph(c);
    if (!order) {
        if (c->order) cudaFree(c->order);
        c->order = nullptr;
        return RADM2_OK;
    }
    std::vector<char> seen(c->ncell, 0);
    for (int i = 0; i < c->ncell; i++) {
        if (order[i] < 0 || order[i] >= c->ncell || seen[order[i]]) {
            c->err = "cell order is not a permutation";
            return RADM2_E_ARG;
        }
        seen[order[i]] = 1;
    }
    if (!c->order) CK(cudaMalloc((void **)&c->order, sizeof(int) * c->ld));
    CK(cudaMemcpyAsync(c->order, order, sizeof(int) * c->ncell, cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    c->use_order = true;
    return RADM2_OK;
}

int radm2_set_kernel_timing(radm2_ctx *c, int enable)
{
    if (!valid_ctx(c)) return RADM2_E_ARG;
    drop_graph(c);  // captured graphs must be rebuilt with (or without) the event nodes
    c->timing = enable != 0;
    c->kernel_ms = 0.0;
    c->kernel_launches = 0;
    c->ev_used = 0;
    return RADM2_OK;
}

int radm2_get_graph_kernels(const radm2_ctx *c, int *kernels)
{
    if (!valid_ctx(c) || !kernels) return RADM2_E_ARG;
    *kernels = c->gexec ? c->graph_kernels : 0;
    return RADM2_OK;
}

int radm2_get_kernel_time(radm2_ctx *c, double *ms, int *launches)
{
    if (!valid_ctx(c) || !ms || !launches) return RADM2_E_ARG;
    *ms = c->kernel_ms;
    *launches = c->kernel_launches;
    c->kernel_ms = 0.0;
    c->kernel_launches = 0;
    return RADM2_OK;
}

// ---------------------------------------------------------------- WRF -> KPP conversion

int radm2_wrf_grid_default(radm2_wrf_grid *g)
{
    if (!g) return RADM2_E_ARG;
    const int init[9] = RADM2_WRF_REF_GRID_INIT;
    std::memcpy(g, init, sizeof init);
    return RADM2_OK;
}

static bool wrf_grid_ok(const radm2_wrf_grid *g)
{
    return g && g->ni > 0 && g->nk > 0 && g->nj > 0 && g->wi > 0 && g->wk > 0 && g->wj > 0 && g->i0 >= 0 &&
           g->k0 >= 0 && g->j0 >= 0 && g->i0 + g->wi <= g->ni && g->k0 + g->wk <= g->nk && g->j0 + g->wj <= g->nj &&
           (long long)g->wi * g->wk * g->wj <= (1LL << 30) && (long long)g->ni * g->nk * g->nj <= (1LL << 31);
}

int radm2_convert_wrf_device(radm2_ctx *c, const radm2_wrf_grid *g, const double *ph, const double *chem,
                             const double *rad, const double *phy, const double *moist)
{
    if (!valid_ctx(c) || !wrf_grid_ok(g) || !ph || !chem || !rad || !phy || !moist) return RADM2_E_ARG;
    CK(cudaSetDevice(c->o.device));
    int rc = ensure_cells(c, g->wi * g->wk * g->wj);
    if (rc) return rc;
    WrfGrid wg;
    std::memcpy(&wg, g, sizeof wg);
    CK(launch_convert_wrf(wg, ph, chem, rad, phy, moist, c->ld, c->var, c->fix, c->temp, c->rcn, c->jv, c->st));
    c->have_rcn = true;
    c->rconst_valid = false;
    return RADM2_OK;
}

int radm2_convert_wrf(radm2_ctx *c, const radm2_wrf_grid *g, const double *ph, const double *chem, const double *rad,
                      const double *phy, const double *moist)
{
    if (!valid_ctx(c) || !wrf_grid_ok(g) || !ph || !chem || !rad || !phy || !moist) return RADM2_E_ARG;
    CK(cudaSetDevice(c->o.device));
    // only the fields the conversion reads travel: ph 0..27, chem / rad up to the last
    // mapped field, phy 0..2, moist 0..1
    const size_t fs = (size_t)g->ni * g->nk * g->nj;
    const int counts[5] = {RADM2_WRF_NPH_USED, RADM2_WRF_NCHEM_USED, RADM2_WRF_NRAD_USED, 3, 2};
    const double *src[5] = {ph, chem, rad, phy, moist};
    size_t total = 0;
    for (int f = 0; f < 5; f++) total += counts[f] * fs;
    int rc = ensure_stage(c, total * sizeof(double));
    if (rc) return rc;
    const double *dev[5];
    size_t off = 0;
    for (int f = 0; f < 5; f++) {
        CK(cudaMemcpyAsync(c->stage + off, src[f], counts[f] * fs * sizeof(double), cudaMemcpyHostToDevice, c->st));
        dev[f] = c->stage + off;
        off += counts[f] * fs;
    }
    rc = radm2_convert_wrf_device(c, g, dev[0], dev[1], dev[2], dev[3], dev[4]);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->st));  // the staging buffer is reused by the next upload
    return RADM2_OK;
}

int radm2_get_ncell(const radm2_ctx *c) { return c ? c->ncell : RADM2_E_ARG; }

int radm2_get_opts(const radm2_ctx *c, radm2_opts *out)
{
    if (!c || !out) return RADM2_E_ARG;
    *out = c->o;
    return RADM2_OK;
}

// ---------------------------------------------------------------- autotuner
//
// Times every built solver variant of the context's precision -- both schedules, every
// (block size, placement, register cap) -- on a strided sample of the context's own cells
// for one split, in a scratch context on the same device, and writes the fastest into the
// context's options.  Every candidate integrates the same sample from the same state and
// must take the same steps; the solver-kernel time (CUDA events) decides.
int radm2_autotune(radm2_ctx *c, double dt, const double *AbsTol, const double *RelTol, const double *RPAR,
                   const int *IPAR, int sample_cells, radm2_tune_entry *table, int table_len, int *n_entries)
{
    if (!valid_ctx(c) || !(dt > 0.0) || !AbsTol || !RelTol || !RPAR || !IPAR || sample_cells < 0 || table_len < 0 ||
        (table_len > 0 && !table))
        return RADM2_E_ARG;
    if (!c->var) return RADM2_E_STATE;
    CK(cudaSetDevice(c->o.device));
    const int n = std::min(c->ncell, sample_cells > 0 ? sample_cells : 262144);
    const int stride = c->ncell / n;

    struct Cand {
        int sched, bs, place, minb, cpt;
    };
    std::vector<Cand> cands;
    if (c->o.precision == RADM2_PREC_FP64) {  // cooperative blocks: 4 or 8 warps per 32 cells
        if (!c->o.parity) cands.push_back({RADM2_SCHED_COOP, 128, RADM2_PLACE_GLOBAL, 1, 1});
        cands.push_back({RADM2_SCHED_COOP, 256, RADM2_PLACE_GLOBAL, 1, 1});
        if (!c->o.parity)  // two cells per thread
            for (int sched = RADM2_SCHED_STATIC; sched <= RADM2_SCHED_PERSISTENT; sched++)
                for (int bs : {64, 128}) cands.push_back({sched, bs, RADM2_PLACE_GLOBAL, 1, 2});
    }
    for (int sched = RADM2_SCHED_STATIC; sched <= RADM2_SCHED_PERSISTENT; sched++) {
#define RADM2_TUNE_CAND(BS_, PL_, MB_) cands.push_back({sched, BS_, PL_, MB_, 1});
        if (c->o.parity && sched == RADM2_SCHED_PERSISTENT) {
            RADM2_VARIANTS_FP64X_PERS(RADM2_TUNE_CAND)
        } else if (c->o.parity) {
            RADM2_VARIANTS_FP64X(RADM2_TUNE_CAND)
        } else if (c->o.precision == RADM2_PREC_FP32LU) {
            RADM2_VARIANTS_FP32(RADM2_TUNE_CAND)
        } else if (sched == RADM2_SCHED_PERSISTENT) {
            RADM2_VARIANTS_FP64_PERS(RADM2_TUNE_CAND)
        } else {
            RADM2_VARIANTS_FP64(RADM2_TUNE_CAND)
        }
#undef RADM2_TUNE_CAND
    }

    // scratch context holding the strided sample (its own stream; the caller's stream is
    // drained first so the sample sees the current state)
    CK(cudaStreamSynchronize(c->st));
    radm2_ctx *t = nullptr;
    int rc = radm2_create(&t, &c->o);
    if (rc) return rc;
    double *y0 = nullptr;
    auto fail = [&](int code) {
        if (y0) cudaFree(y0);
        radm2_destroy(t);
        return code;
    };
    if ((rc = ensure_cells(t, n))) {
        c->err = t->err;
        return fail(rc);
    }
    cudaError_t e = launch_gather_rows(n, NVAR, c->ld, stride, c->var, t->ld, t->var, t->st);
    if (e == cudaSuccess) e = launch_gather_rows(n, NFIX, c->ld, stride, c->fix, t->ld, t->fix, t->st);
    if (e == cudaSuccess) e = launch_gather_rows(n, 1, c->ld, stride, c->temp, t->ld, t->temp, t->st);
    if (e == cudaSuccess) e = launch_gather_rows(n, NPH, c->ld, stride, c->jv, t->ld, t->jv, t->st);
    if (e == cudaSuccess && c->have_rcn) e = launch_gather_rows(n, 1, c->ld, stride, c->rcn, t->ld, t->rcn, t->st);
    t->have_rcn = c->have_rcn;
    t->rconst_valid = false;
    if (e == cudaSuccess) e = cudaMalloc((void **)&y0, sizeof(double) * NVAR * t->ld);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(y0, t->var, sizeof(double) * NVAR * t->ld, cudaMemcpyDeviceToDevice, t->st);
    if (e != cudaSuccess) {
        fail_cuda(c, e, "autotune sample");
        return fail(RADM2_E_CUDA);
    }
    t->timing = true;

    // One split of the sample with candidate k: solver-kernel ms (-1 if it did not run) and
    // the step attempts it took.
    auto time_cand = [&](const Cand &k, long long *att) {
        t->o.schedule = k.sched;
        t->o.block_threads = k.bs;
        t->o.placement = k.place;
        t->o.min_blocks = k.minb;
        t->o.cells_per_thread = k.cpt;
        t->o.blocks_per_sm = 0;
        drop_graph(t);
        double ms = -1.0;
        *att = -1;
        if (cudaMemcpyAsync(t->var, y0, sizeof(double) * NVAR * t->ld, cudaMemcpyDeviceToDevice, t->st) ==
            cudaSuccess) {
            double rpar[20];
            int ipar[20];
            std::memcpy(rpar, RPAR, sizeof rpar);
            std::memcpy(ipar, IPAR, sizeof ipar);
            if (rpar[2] == 0.0) rpar[2] = 0.01 * dt;
            double kms0 = 0.0;
            int kl0 = 0;
            radm2_get_kernel_time(t, &kms0, &kl0);  // reset the accumulators
            const int ierr = radm2_rosenbrock(t, 0.0, dt, AbsTol, RelTol, rpar, ipar);
            double kms = 0.0;
            int kl = 0;
            if (ierr == 1 && radm2_get_kernel_time(t, &kms, &kl) == RADM2_OK && kl == 1) {
                ms = kms;
                *att = (long long)ipar[13] + ipar[14];
            }
        }
        (void)cudaGetLastError();  // a variant that cannot run here is skipped, not fatal
        return ms;
    };

    // First pass over every candidate.  A candidate counts only if it takes the same step
    // attempts as the first one that ran (every variant integrates the same cells).
    const size_t nc = cands.size();
    std::vector<double> ms(nc, -1.0);
    std::vector<long long> att(nc, -1);
    long long attempts0 = -1;
    {  // untimed warm-up split: the first launch on a fresh context runs slow
        long long a = -1;
        (void)time_cand(cands[0], &a);
    }
    for (size_t i = 0; i < nc; i++) {
        ms[i] = time_cand(cands[i], &att[i]);
        if (ms[i] >= 0.0 && attempts0 < 0) attempts0 = att[i];
        if (ms[i] >= 0.0 && att[i] != attempts0) ms[i] = -1.0;
    }
    auto pick = [&]() {
        int b = -1;
        for (size_t i = 0; i < nc; i++)
            if (ms[i] >= 0.0 && (b < 0 || ms[i] < ms[b])) b = (int)i;
        return b;
    };
    // Second pass: a single timing can come out slow (a one-off stall), so every candidate
    // within 2x of the best is timed again and keeps its faster time.
    int best = pick();
    if (best >= 0) {
        const double lim = 2.0 * ms[best];
        for (size_t i = 0; i < nc; i++) {
            if (ms[i] < 0.0 || ms[i] > lim) continue;
            long long a2 = -1;
            const double m2 = time_cand(cands[i], &a2);
            if (m2 >= 0.0 && a2 == attempts0) ms[i] = std::min(ms[i], m2);
        }
        best = pick();
    }
    int count = 0;
    for (size_t i = 0; i < nc; i++) {
        const Cand &k = cands[i];
        if (count < table_len) {
            radm2_tune_entry &te = table[count];
            te.schedule = k.sched;
            te.block_threads = k.bs;
            te.placement = k.place;
            te.min_blocks = k.minb;
            te.cells_per_thread = k.cpt;
            te.ms = ms[i];
            te.attempts = att[i];
        }
        count++;
    }
    if (n_entries) *n_entries = count;
    cudaFree(y0);
    y0 = nullptr;
    radm2_destroy(t);
    if (best < 0) {
        c->err = "autotune: no solver variant ran on this device";
        return RADM2_E_CUDA;
    }
    drop_graph(c);
    c->o.schedule = cands[best].sched;
    c->o.block_threads = cands[best].bs;
    c->o.placement = cands[best].place;
    c->o.min_blocks = cands[best].minb;
    c->o.cells_per_thread = cands[best].cpt;
    c->o.blocks_per_sm = 0;
    return RADM2_OK;
}

size_t radm2_device_bytes(const radm2_ctx *c)
{
    if (!c) return 0;
    return c->bytes + c->scratch_bytes + c->stage_bytes;
}

int radm2_coop_selftest_wait_limit(radm2_ctx *c)
{
    if (!valid_ctx(c)) return RADM2_E_ARG;
    if (!c->var) return RADM2_E_STATE;
    if (c->o.schedule != RADM2_SCHED_COOP) return RADM2_E_ARG;
    double atol[NVAR], rtol[NVAR], rpar[20] = {0};
    int ipar[20] = {0};
    for (int i = 0; i < NVAR; i++) {
        atol[i] = 1.0;
        rtol[i] = 1e-3;
    }
    ipar[0] = 1;
    ipar[3] = 2;
    drop_graph(c);
    // cells the aborted blocks never take keep their status: start from a neutral 0
    CK(cudaMemsetAsync(c->status, 0, sizeof(int) * c->ld, c->st));
    c->coop_selftest = 1;
    const int ierr = radm2_rosenbrock(c, 0.0, 600.0, atol, rtol, rpar, ipar);
    c->coop_selftest = 0;
    drop_graph(c);
    if (ierr != RADM2_E_CUDA) return RADM2_E_STATE;
    c->err.clear();
    return RADM2_OK;
}

int radm2_selfcheck(void)
{
    // Layout bounds of every solver variant (host arithmetic only, no device needed).
    const int bad = solver_layout_check_fp64_static() | solver_layout_check_fp64_persistent() |
                    solver_layout_check_fp32_static() | solver_layout_check_fp32_persistent() |
                    solver_layout_check_fp32d_static() | solver_layout_check_fp32d_persistent() |
                    solver_layout_check_fp64x_static() | solver_layout_check_fp64x_persistent() |
                    solver_layout_check_cpt2();
    return bad ? RADM2_E_STATE : RADM2_OK;
}

const char *radm2_version(void)
{
    return "radm2-b200 1.1 sm_100a (fp64 | fp64 reference arithmetic | fp32-LU+IR) x (static | persistent)";
}

// ---------------------------------------------------------------- mechanism kernels on host arrays

static int mech_call(radm2_ctx *c, int n, int kind, int fp32, const double *V, const double *FIX, const double *RCT,
                     double *out, double *G, double *X, int *sing)
{
    if (!valid_ctx(c) || n <= 0) return RADM2_E_ARG;
    CK(cudaSetDevice(c->o.device));
    const int ld = (n + 31) / 32 * 32;
    double *dv = nullptr, *df = nullptr, *dr = nullptr, *dout = nullptr, *stage = nullptr;
    int *ds = nullptr;
    const size_t cap = (size_t)ld * NJVS;
    cudaError_t e = cudaSuccess;
    auto up = [&](const double *h, int m, double *d) {
        if (e != cudaSuccess) return;
        e = cudaMemcpyAsync(stage, h, sizeof(double) * n * m, cudaMemcpyHostToDevice, c->st);
        if (e == cudaSuccess) e = launch_aos_to_soa(n, m, ld, stage, d, c->st);
    };
    auto down = [&](const double *d, int m, double *h) {
        if (e != cudaSuccess) return;
        e = launch_soa_to_aos(n, m, ld, d, stage, c->st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(h, stage, sizeof(double) * n * m, cudaMemcpyDeviceToHost, c->st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    };
    e = cudaMalloc((void **)&stage, sizeof(double) * cap);
    if (e == cudaSuccess) e = cudaMalloc((void **)&dout, sizeof(double) * cap);
    if (kind < 2) {
        if (e == cudaSuccess) e = cudaMalloc((void **)&dv, sizeof(double) * ld * NVAR);
        if (e == cudaSuccess) e = cudaMalloc((void **)&df, sizeof(double) * ld * NFIX);
        if (e == cudaSuccess) e = cudaMalloc((void **)&dr, sizeof(double) * ld * NREACT);
        up(V, NVAR, dv);
        up(FIX, NFIX, df);
        up(RCT, NREACT, dr);
        if (e == cudaSuccess) e = kind == 0 ? launch_fun(n, ld, dv, df, dr, dout, c->st) : launch_jac(n, ld, dv, df, dr, dout, c->st);
        down(dout, kind == 0 ? NVAR : NJVS, out);
    } else {
        if (e == cudaSuccess) e = cudaMalloc((void **)&dv, sizeof(double) * ld * NVAR);
        if (e == cudaSuccess) e = cudaMalloc((void **)&ds, sizeof(int) * ld);
        up(G, NJVS, dout);
        up(X, NVAR, dv);
        if (e == cudaSuccess) e = launch_decomp_solve(n, ld, fp32, dout, dv, ds, c->st);
        down(dout, NJVS, G);
        down(dv, NVAR, X);
        if (e == cudaSuccess) e = cudaMemcpy(sing, ds, sizeof(int) * n, cudaMemcpyDeviceToHost);
    }
    cudaFree(stage);
    cudaFree(dout);
    cudaFree(dv);
    cudaFree(df);
    cudaFree(dr);
    cudaFree(ds);
    if (e != cudaSuccess) return fail_cuda(c, e, "mechanism kernel");
    return RADM2_OK;
}

int radm2_fun(radm2_ctx *c, int n, const double *V, const double *FIX, const double *RCT, double *VDOT)
{
    if (!V || !FIX || !RCT || !VDOT) return RADM2_E_ARG;
    return mech_call(c, n, 0, 0, V, FIX, RCT, VDOT, nullptr, nullptr, nullptr);
}

int radm2_jac(radm2_ctx *c, int n, const double *V, const double *FIX, const double *RCT, double *JVS)
{
    if (!V || !FIX || !RCT || !JVS) return RADM2_E_ARG;
    return mech_call(c, n, 1, 0, V, FIX, RCT, JVS, nullptr, nullptr, nullptr);
}

int radm2_decomp_solve(radm2_ctx *c, int n, int precision, double *G, double *X, int *sing)
{
    if (!G || !X || !sing || (precision != RADM2_PREC_FP64 && precision != RADM2_PREC_FP32LU)) return RADM2_E_ARG;
    return mech_call(c, n, 2, precision == RADM2_PREC_FP32LU, nullptr, nullptr, nullptr, nullptr, G, X, sing);
}

}  // extern "C"
