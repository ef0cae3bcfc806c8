// mfree_ctx.h -- the context behind the opaque mfree_ctx handle, shared by
// the single-scene ABI (mfree_host.cu) and the batch/serving ABI
// (mfree_batch.cu).  Host code only.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "mfree.h"
#include "mfree_kernels.cuh"
#include "mfree_tool.h"

namespace mfree {
namespace host {

int fail(int code, const std::string &msg);

}  // namespace host
}  // namespace mfree

#define CUDA_TRY(x)                                                                        \
    do {                                                                                   \
        cudaError_t e_ = (x);                                                              \
        if (e_ != cudaSuccess)                                                             \
            return mfree::host::fail(e_ == cudaErrorMemoryAllocation ? MFREE_ERR_OOM : MFREE_ERR_CUDA,  \
                        std::string(#x) + ": " + cudaGetErrorString(e_));                 \
    } while (0)

namespace mfree {
namespace host {

// NVTX range around a host-side call or kernel launch, for timeline tools
// (Nsight Systems); with no tool attached a push/pop costs a few nanoseconds
struct TraceRange {
    explicit TraceRange(const char *name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange &) = delete;
    TraceRange &operator=(const TraceRange &) = delete;
};
// the step's kernels in launch order (the ids of mfree_get_kernel_times)
constexpr const char *KERNEL_TRACE_NAMES[MFREE_NUM_KERNELS] = {
    "kb_clock", "kb_hash", "kb_scan_reduce", "kb_scan_top", "kb_scan_down", "kb_scatter",
    "kb_cell_fixup", "kb_gather_predict", "kb_interact", "kb_finalize", "kb_force_final"};

struct DevTool {
    HostTool host;
    std::vector<float> verts;  // input vertices (x, y, z), for output
    int algorithm = MFREE_CONTACT_HASHED;
    float vel[3] = {0, 0, 0};
    float alpha = 0.1f, mu = 0.f;
    float birth = -3.402823466e+38f, death = 3.402823466e+38f;
    float4 *d_tri = nullptr;  // 10 arrays of float4, back to back
    int *d_cells = nullptr;
    int ntri_dev = 0;
};

}  // namespace host
}  // namespace mfree

struct mfree_ctx {
    int n_init = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int device = 0, num_sms = 148;
    // host-side configuration
    mfree_phys phys{};
    mfree_corr corr{};
    mfree_joco joco{};
    mfree_trml twp{}, ttool{};
    mfree_options opt{};
    bool plastic = false;
    bool grid_set = false;
    float g_bbmin[3], g_bbmax[3], g_dx = 0.f, g_vel[3] = {0, 0, 0};
    long nx = 0, ny = 0, nz = 0, num_cell = 0;
    bool grid_adaptive = false;  // unlocked grid: box and cell edge from the particles every step
    long max_cell = 0;           // its cell limit (the scratch is sized for it)
    int *d_bbox = nullptr, *h_bbox = nullptr;  // its bounding-box reduction (device, page-locked host)
    double *d_energy = nullptr;  // mfree_get_energies: results, then per-block partials
    bool blank_set = false;
    float b_min[3], b_max[3], b_vel[3] = {0, 0, 0}, b_vmax = 0.f;
    float dt = 0.f, t = 0.f;
    bool time_set = false;
    std::vector<std::unique_ptr<mfree::host::DevTool>> tools;
    // device memory
    mfree::State st[2]{};
    int cur = 0;
    mfree::Records rec{};
    mfree::Scratch scr{};
    mfree::DevClock *d_clk = nullptr;
    float *d_forces = nullptr;
    size_t scratch_cells = 0;  // num_cell the scratch was sized for
    std::vector<void *> allocs, scratch_allocs;
    size_t bytes = 0, scratch_bytes = 0;  // device memory held (state, scratch; tools in bytes)
    bool clock_dirty = true;  // host-side scalars changed: rewrite the device clock
    bool pending = false;     // a step has run since the clock was written
    long long steps = 0;
    // per-kernel timing (eager steps)
    bool timing = false;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> tev;
    std::vector<cudaEvent_t> event_pool;
    double kernel_ms[MFREE_NUM_KERNELS] = {0};
    int kernel_n[MFREE_NUM_KERNELS] = {0};
    cudaEvent_t timer[2] = {nullptr, nullptr};
    // active count of the last step, copied back asynchronously: a step that
    // left no particle makes the next call return MFREE_ERR_EMPTY (the
    // reference exits there, grid_gpu_base.cu:159-163)
    int *h_nact = nullptr;
    cudaEvent_t nact_ev = nullptr;
    bool nact_pending = false;
    // the captured step (one graph serves both state parities)
    cudaGraphExec_t graph = nullptr;
    int graph_record_every = -1;
    // one-scene table of the batched kernels (ensure_table)
    unsigned char *d_table = nullptr;
    int2 *d_tiles = nullptr;  // the pair kernel's list of non-empty tiles (grid-sized scratch)
    int ntiles = 0;           // tiles of the grid at the table's depth
    mfree::BatchTable T{};
    unsigned long long table_version = ~0ull;
    int table_record_every = -1;
    // batches: the owning batch (NULL: none), the stream to return to on
    // retirement, and a counter bumped whenever the step arguments may change
    mfree_batch *owner = nullptr;
    cudaStream_t home_stream = nullptr;
    unsigned long long version = 0;
    bool inject_staging = false;  // mfree_inject_fault: staging waits run out (tests)
    // asynchronous particle output (mfree_output.cu), created on first use
    struct OutputJob *output = nullptr;
};


namespace mfree {
namespace host {

int default_lpp();
int default_tile_depth();
int hash_blocks(const mfree_ctx *c);
int scan_tiles(const mfree_ctx *c);
StepArgs make_args(mfree_ctx *c);
int ready(mfree_ctx *c);
int check_empty(mfree_ctx *c, bool wait);
int note_active_count(mfree_ctx *c);
void invalidate_graphs(mfree_ctx *c);
// allocates the grid-sized scratch (cell counters, cell table, scan sums)
int ensure_scratch(mfree_ctx *c);
// allocates a context's device memory and stream (no state upload)
int alloc_ctx(int n, cudaStream_t stream, std::unique_ptr<mfree_ctx> &out);
// a copy of c (configuration, tools, current state and clock) on stream s
int clone_ctx(const mfree_ctx *c, cudaStream_t s, std::unique_ptr<mfree_ctx> &out);
// waits for and frees the context's output job (mfree_output.cu)
int finish_output(mfree_ctx *c, bool release);
size_t scene_bytes(int n, long long num_cell);
inline size_t single_table_bytes() { return 2 * sizeof(mfree::StepArgs) + 10 * sizeof(int); }
// device memory the context holds, in bytes
size_t device_bytes(const mfree_ctx *c);

}  // namespace host
}  // namespace mfree
