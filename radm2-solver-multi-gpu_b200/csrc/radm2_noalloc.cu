// radm2_rosenbrock_noalloc: the integration for callers that cannot allocate device
// memory.
//
// Some callers may not call cudaMalloc while they run: a host framework that reserved all
// of the GPU's memory for its own pool at start-up (a later cudaMalloc fails or steals from
// that pool), and real-time or certified couplings whose device memory budget is fixed at
// initialisation and may not grow once the model is running.  This entry point takes device
// pointers for the inputs and outputs and keeps everything else it needs -- the solver
// kernel's per-thread scratch slots, the rate-constant table and the per-cell bookkeeping --
// in one statically sized array in this file.  It runs the same rate-constant, solver and
// reduction kernels as radm2_rosenbrock (the solver with the working set of each cell in
// shared memory, so its global scratch is small).
//
// The array is a __device__ object: every GPU that loads the library holds its
// RADM2_NOALLOC_BYTES until the process exits.  Host code cannot use the array's name as
// a device address (in host code it names a host-side stand-in), so the address is
// fetched with cudaGetSymbolAddress on the first call made with a given device and CUDA
// context current, and passed to the kernels.
#include <cstring>
#include <mutex>

#include "../../include/radm2.h"
#include "radm2_internal.h"
#include "radm2_solver.cuh"  // working-set layout constants (no kernel is instantiated here)

using namespace radm2;

namespace {

constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// Offsets of the carved regions (bytes).
constexpr int kBlockThreads = 32;       // solver variant: 32 threads, RC/state/LU in shared memory
constexpr int kMaxBlocks = 256;         // persistent grid: one block per SM, up to 256 SMs
constexpr size_t kCells = RADM2_NOALLOC_MAX_CELLS;
constexpr size_t kOffRconst = 0;
constexpr size_t kOffNacc = kOffRconst + align256(sizeof(double) * NREACT * kCells);
constexpr size_t kOffNrej = kOffNacc + align256(sizeof(int) * kCells);
constexpr size_t kOffStatus = kOffNrej + align256(sizeof(int) * kCells);
constexpr size_t kOffHfirst = kOffStatus + align256(sizeof(int) * kCells);
constexpr size_t kOffHexit = kOffHfirst + align256(sizeof(double) * kCells);
constexpr size_t kOffTexit = kOffHexit + align256(sizeof(double) * kCells);
constexpr size_t kOffQueue = kOffTexit + align256(sizeof(double) * kCells);
constexpr size_t kOffPartials = kOffQueue + 256;
constexpr size_t kPartialsCap = 64 * 1024;
constexpr size_t kOffResult = kOffPartials + kPartialsCap;
constexpr size_t kOffScratch = kOffResult + align256(sizeof(RunResult));
constexpr size_t kScratchBytes =
    sizeof(double) * (size_t)Layout<double, PLACE_LU_SMEM | PLACE_RCY_SMEM>::global_words * kBlockThreads * kMaxBlocks;
constexpr size_t kTotal = kOffScratch + align256(kScratchBytes);
static_assert(kTotal <= (size_t)RADM2_NOALLOC_BYTES, "no-alloc area larger than documented");

// The statically sized device area (one per GPU that loads this library).
__device__ __align__(256) unsigned char g_noalloc_area[RADM2_NOALLOC_BYTES];

std::mutex g_setup_mutex;
// Per device: the CUDA context the address was looked up in, and the address.  A device
// reset (cudaDeviceReset) or a new primary context reloads the module at a new address, so
// the cached address is only reused while the same context is current.
struct AreaSlot {
    void *ctx;
    void *addr;
};
AreaSlot g_area[256];

using CtxGetCurrentFn = int (*)(void **);
CtxGetCurrentFn ctx_get_current()
{
    static CtxGetCurrentFn fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<CtxGetCurrentFn>(f);
    }();
    return fn;
}

// Device address of the area on the current device and context (set-up on the first call
// with that pair current; without the context query, looked up on every call).
cudaError_t area_address(int device, unsigned char **out)
{
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    void *ctx = nullptr;
    CtxGetCurrentFn get = ctx_get_current();
    const bool known_ctx = get && get(&ctx) == 0 && ctx;
    if (!known_ctx || !g_area[device].addr || g_area[device].ctx != ctx) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_area);
        if (e != cudaSuccess) return e;
        g_area[device].ctx = known_ctx ? ctx : nullptr;
        g_area[device].addr = known_ctx ? p : nullptr;
        *out = static_cast<unsigned char *>(p);
        return cudaSuccess;
    }
    *out = static_cast<unsigned char *>(g_area[device].addr);
    return cudaSuccess;
}

}  // namespace

extern "C" int radm2_rosenbrock_noalloc(int ncell, int ld, double *var, const double *fix, const double *temp,
                                        const double *rc_n2o5, const double *jv, double Tstart, double Tend,
                                        const double *AbsTol, const double *RelTol, double *RPAR, int *IPAR,
                                        int *status, void *stream)
{
    if (ncell <= 0 || ld < ncell || !var || !fix || !temp || !jv || !AbsTol || !RelTol || !RPAR || !IPAR)
        return RADM2_E_ARG;
    if ((size_t)ld > kCells) return RADM2_E_TOOBIG;  // ncell <= ld <= RADM2_NOALLOC_MAX_CELLS
    if (reduce_partials_bytes() > kPartialsCap) return RADM2_E_STATE;
    int device = 0, major = 0, nsm = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 256 ||
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device) != cudaSuccess || major != 10 ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return RADM2_E_NODEV;
    SolveParams p;
    int autonomous = 1;
    const int ierr0 = parse_params(Tstart, Tend, AbsTol, RelTol, RPAR, IPAR, 1, &p, &autonomous);
    if (ierr0 != 1) return ierr0;
    const int key = variant_key(kBlockThreads, PLACE_LU_SMEM | PLACE_RCY_SMEM, 1);
    SolverInfo info;
    if (solver_info_fp64_persistent(key, &info) != cudaSuccess || info.blocks_per_sm < 1) return RADM2_E_CUDA;
    int grid = nsm * info.blocks_per_sm;
    if (grid > kMaxBlocks) grid = kMaxBlocks;
    const int need = (ncell + kBlockThreads - 1) / kBlockThreads;
    if (grid > need) grid = need;

    unsigned char *area = nullptr;
    if (area_address(device, &area) != cudaSuccess) return RADM2_E_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    double *rconst = reinterpret_cast<double *>(area + kOffRconst);
    int *queue = reinterpret_cast<int *>(area + kOffQueue);
    RunResult *d_res = reinterpret_cast<RunResult *>(area + kOffResult);
    SolveArgs a;
    std::memset(&a, 0, sizeof a);
    a.p = p;
    a.ncell = ncell;
    a.ld = ld;
    a.var = var;
    a.fix = fix;
    a.rconst = rconst;
    a.queue = queue;
    a.scratch = reinterpret_cast<double *>(area + kOffScratch);
    a.status = status ? status : reinterpret_cast<int *>(area + kOffStatus);
    a.nacc = reinterpret_cast<int *>(area + kOffNacc);
    a.nrej = reinterpret_cast<int *>(area + kOffNrej);
    a.hfirst = reinterpret_cast<double *>(area + kOffHfirst);
    a.hexit = reinterpret_cast<double *>(area + kOffHexit);
    a.texit = reinterpret_cast<double *>(area + kOffTexit);
    a.refine = 0;

    // The area keeps the previous call's contents: the work-queue counter must start at 0;
    // every other region is fully rewritten before it is read.
    if (cudaMemsetAsync(queue, 0, sizeof(int), st) != cudaSuccess) return RADM2_E_CUDA;
    if (launch_rconst(ncell, ld, jv, temp, fix, rc_n2o5, rconst, st) != cudaSuccess) return RADM2_E_CUDA;
    if (launch_solver_fp64_persistent(a, key, grid, st) != cudaSuccess) return RADM2_E_CUDA;
    if (launch_reduce(ncell, a.status, a.nacc, a.nrej, a.texit, a.hexit, area + kOffPartials, d_res, st) !=
        cudaSuccess)
        return RADM2_E_CUDA;
    RunResult r;
    if (cudaMemcpyAsync(&r, d_res, sizeof r, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return RADM2_E_CUDA;

    add_step_counters(IPAR, r.nacc, r.nrej, r.nfail, autonomous);
    RPAR[10] = p.direction > 0 ? r.tmin : r.tmax;
    RPAR[11] = r.hmin;
    return r.worst;
}
