// mfree_host.cu -- the C ABI (include/mfree.h): context, device memory, step
// orchestration and state import/export.
//
// Reference host path replaced: particle_gpu construction (particle_gpu.cu:20-117),
// the constant uploads (actions_gpu.cu:659-710, interactions_gpu.cu:552-608,
// tool_3d_gpu.cu:683-812), the grid and blanking objects (grid_gpu_base.cu:237-273,
// blanking.cpp), leap_frog::step (leap_frog.cu:121-195) and the process globals
// of mfree_gpu_3d.cpp:41-48.
//
// A step is 11 kernels on one stream with no host synchronisation (N lives on
// the device), so it can also be captured once into a CUDA graph and replayed.
#include <climits>
#include <cstdint>
#include <cstddef>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "mfree_ctx.h"

using namespace mfree;
using namespace mfree::host;

namespace {
thread_local std::string g_err;
}  // namespace

int mfree::host::fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

void mfree::set_last_error(const std::string &msg) { g_err = msg; }

namespace mfree {
namespace host {

// Context memory comes from one stream-ordered memory pool per device that
// keeps what is freed (unlimited release threshold): contexts created and
// destroyed one after another -- served requests, the autotuner's copies, a
// caller's repeated jobs -- reuse it without a new cudaMalloc, and freeing
// needs no device-wide synchronisation.  The pool is created on first use on
// each device.
cudaMemPool_t context_pool(int dev) {
    static std::mutex m;
    static std::vector<cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lock(m);
    if (int(pools.size()) <= dev) pools.resize(size_t(dev) + 1, nullptr);
    if (!pools[dev]) {
        cudaMemPoolProps pr{};
        pr.allocType = cudaMemAllocationTypePinned;
        pr.location.type = cudaMemLocationTypeDevice;
        pr.location.id = dev;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &pr) != cudaSuccess) return nullptr;
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        pools[dev] = pool;
    }
    return pools[dev];
}

template <class T> int dalloc(mfree_ctx *c, T **p, size_t n, std::vector<void *> &list) {
    void *q = nullptr;
    cudaMemPool_t pool = context_pool(c->device);
    if (!pool) return fail(MFREE_ERR_CUDA, "cudaMemPoolCreate failed");
    cudaError_t e = cudaMallocFromPoolAsync(&q, std::max<size_t>(n, 1) * sizeof(T), pool, c->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(MFREE_ERR_OOM, std::string("cudaMallocFromPoolAsync: ") + cudaGetErrorString(e));
    }
    list.push_back(q);
    *p = (T *)q;
    (&list == &c->scratch_allocs ? c->scratch_bytes : c->bytes) += std::max<size_t>(n, 1) * sizeof(T);
    return MFREE_OK;
}

size_t device_bytes(const mfree_ctx *c) { return c->bytes + c->scratch_bytes; }

// stream-ordered: the memory returns to the pool once the stream's earlier work is done
void free_list(std::vector<void *> &l, cudaStream_t s) {
    for (void *p : l) cudaFreeAsync(p, s);
    l.clear();
}

void invalidate_graphs(mfree_ctx *c) {
    c->version++;
    if (c->graph) cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
    c->graph_record_every = -1;
}

int default_lpp() { return 8; }
int default_tile_depth() { return 6; }

Params make_params(const mfree_ctx *c) {
    Params P{};
    P.mass = c->phys.mass;
    P.K = c->phys.K;
    P.G = c->phys.G;
    P.rho0 = c->phys.rho0;
    {
        float c0 = std::sqrt(c->phys.rho0 != 0.f ? c->phys.K / c->phys.rho0 : 0.f);
        P.c0sq = c0 * c0;
    }
    P.wdeltap = c->corr.wdeltap;
    P.inv_wdeltap = c->corr.wdeltap > 0.f ? 1.0f / c->corr.wdeltap : 0.f;
    P.stresseps = c->corr.stresseps;
    P.xspheps = c->corr.xspheps;
    P.av_alpha = c->corr.alpha;
    P.av_beta = c->corr.beta;
    P.av_eta = c->corr.eta;
    P.wp_alpha = c->twp.alpha;
    P.wp_cp = c->twp.cp;
    P.wp_tq = c->twp.tq;
    P.wp_Tinit = c->twp.T_init;
    P.wp_eta = c->twp.eta;
    P.tool_alpha = c->ttool.alpha;
    P.thermal = (c->twp.alpha != 0.f || c->ttool.alpha != 0.f) ? 1 : 0;
    P.fric_heat = c->twp.eta != 0.f ? 1 : 0;
    P.jc_A = c->joco.A;
    P.jc_B = c->joco.B;
    P.jc_C = c->joco.C;
    P.jc_n = c->joco.n;
    P.jc_m = c->joco.m;
    P.jc_Tmelt = c->joco.Tmelt;
    P.jc_Tref = c->joco.Tref;
    P.jc_epsdot_ref = c->joco.eps_dot_ref;
    P.jc_clamp = c->joco.clamp_temp;
    P.plastic = c->plastic ? 1 : 0;
    P.max_secant_iter = c->opt.max_secant_iter > 0 ? c->opt.max_secant_iter : 100;
    P.cspm = c->opt.cspm;
    P.conduction = c->opt.conduction;
    P.precision = c->opt.precision;
    P.diagnostics = c->opt.diagnostics;
    P.friction_tool_vel = c->opt.friction_tool_vel;
    P.full_stencil = c->opt.full_stencil ? 1 : 0;
    P.gnx = int(c->nx);
    P.gny = int(c->ny);
    P.gnz = int(c->nz);
    P.num_cell = int(c->num_cell);
    P.gdx = c->g_dx;
    P.grid_moving = !c->grid_adaptive && (c->g_vel[0] != 0.f || c->g_vel[1] != 0.f || c->g_vel[2] != 0.f) ? 1 : 0;
    for (int d = 0; d < 3; d++) {
        P.grid_vel[d] = c->g_vel[d];
        P.grid_min0[d] = c->g_bbmin[d];
        P.blank_min0[d] = c->b_min[d];
        P.blank_max0[d] = c->b_max[d];
        P.blank_vel[d] = c->b_vel[d];
    }
    P.blank_on = c->blank_set ? 1 : 0;
    P.vmax2 = c->b_vmax * c->b_vmax;
    P.dt = c->dt;
    P.n_init = c->n_init;
    P.num_tools = int(c->tools.size());
    for (int d = 0; d < 3; d++) P.tool0_vel[d] = c->tools.empty() ? 0.f : c->tools[0]->vel[d];
    P.record_every = 0;
    P.tile_z = c->opt.tile_depth > 0 ? c->opt.tile_depth : default_tile_depth();
    P.stage_extra = c->inject_staging ? 16 : 0;
    return P;
}

int hash_blocks(const mfree_ctx *c) { return (c->n_init + HASH_BLOCK - 1) / HASH_BLOCK; }
int scan_tiles(const mfree_ctx *c) { return int((c->num_cell + 1 + SCAN_TILE - 1) / SCAN_TILE); }

StepArgs make_args(mfree_ctx *c) {
    StepArgs a{};
    a.p = make_params(c);
    a.a = c->st[c->cur];
    a.b = c->st[c->cur ^ 1];
    a.r = c->rec;
    a.s = c->scr;
    a.clk = c->d_clk;
    for (size_t k = 0; k < c->tools.size() && k < size_t(MAX_TOOLS); k++) {
        const DevTool &t = *c->tools[k];
        ToolDev &d = a.tools[k];
        const int n = t.ntri_dev;
        d.p1 = t.d_tri;
        d.p2 = t.d_tri + n;
        d.p3 = t.d_tri + 2 * n;
        d.n = t.d_tri + 3 * n;
        d.np1 = t.d_tri + 4 * n;
        d.np2 = t.d_tri + 5 * n;
        d.np3 = t.d_tri + 6 * n;
        d.ne1 = t.d_tri + 7 * n;
        d.ne2 = t.d_tri + 8 * n;
        d.ne3 = t.d_tri + 9 * n;
        d.cells = t.d_cells;
        d.num_tris = t.host.boxed.empty() ? 0 : n;
        d.nx = t.host.nx;
        d.ny = t.host.ny;
        d.nz = t.host.nz;
        d.dx = t.host.dx;
        for (int q = 0; q < 3; q++) d.vel[q] = t.vel[q];
        d.alpha = t.alpha;
        d.mu = t.mu;
        d.hashed = t.algorithm == MFREE_CONTACT_HASHED ? 1 : 0;
        d.birth = t.birth;
        d.death = t.death;
    }
    return a;
}

// scratch that depends on the grid size
int ensure_scratch(mfree_ctx *c) {
    // an unlocked grid changes its cell count every step: its scratch holds max_cell cells
    const long cells = c->grid_adaptive ? c->max_cell : c->num_cell;
    if (c->scratch_cells == size_t(cells) && !c->scratch_allocs.empty()) return MFREE_OK;
    free_list(c->scratch_allocs, c->stream);
    c->scratch_bytes = 0;
    auto &L = c->scratch_allocs;
    int st;
    if ((st = dalloc(c, &c->scr.count, cells + 1, L))) return st;
    if ((st = dalloc(c, &c->scr.first, cells + 2 + SCAN_TILE, L))) return st;
    if ((st = dalloc(c, &c->scr.tile_sum, (cells + 1 + SCAN_TILE - 1) / SCAN_TILE + 1, L))) return st;
    // the pair kernel's tile list: a tile of any depth holds a cell at least
    if ((st = dalloc(c, &c->d_tiles, cells + 1, L))) return st;
    CUDA_TRY(cudaMemsetAsync(c->scr.count, 0, sizeof(int) * (cells + 1), c->stream));
    c->scratch_cells = size_t(cells);
    invalidate_graphs(c);
    return MFREE_OK;
}

int write_clock(mfree_ctx *c) {
    DevClock h{};
    h.t = c->t;
    h.pending = 0;
    h.n_active = c->n_init;
    h.record = 0;
    h.step_index = c->steps;
    h.parity = c->cur;
    for (int d = 0; d < 3; d++) {
        h.blank_min[d] = c->b_min[d];
        h.blank_max[d] = c->b_max[d];
        h.grid_min[d] = c->g_bbmin[d];
    }
    for (size_t k = 0; k < c->tools.size(); k++)
        for (int d = 0; d < 3; d++) {
            h.tool[k].bbmin[d] = c->tools[k]->host.bbmin[d];
            h.tool[k].bbmax[d] = c->tools[k]->host.bbmax[d];
        }
    // keep the device counters
    DevClock old{};
    CUDA_TRY(cudaMemcpyAsync(&old, c->d_clk, sizeof(DevClock), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    h.secant_failures = old.secant_failures;
    h.out_of_grid = old.out_of_grid;
    h.contact_cap = old.contact_cap;
    h.nan_blanked = old.nan_blanked;
    h.staging_timeouts = old.staging_timeouts;
    h.n_active = old.n_active ? old.n_active : c->n_init;
    CUDA_TRY(cudaMemcpyAsync(c->d_clk, &h, sizeof(DevClock), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->clock_dirty = false;
    c->pending = false;
    return MFREE_OK;
}

int ready(mfree_ctx *c) {
    if (!c->grid_set) return fail(MFREE_ERR_ARG, "mfree_set_grid must be called before stepping");
    if (!c->time_set || !(c->dt > 0.f)) return fail(MFREE_ERR_ARG, "mfree_set_time must set dt > 0 before stepping");
    if (c->phys.mass <= 0.f || c->phys.rho0 <= 0.f) return fail(MFREE_ERR_ARG, "mfree_set_physics: mass and rho0 must be > 0");
    if (c->tools.size() > size_t(MAX_TOOLS)) return fail(MFREE_ERR_ARG, "too many tools");
    int lpp = c->opt.lanes_per_particle;
    if (lpp != 0 && lpp != 8 && lpp != 16 && lpp != 32)
        return fail(MFREE_ERR_ARG, "lanes_per_particle must be 0, 8, 16 or 32");
    if (c->opt.conduction < 0 || c->opt.conduction > 2) return fail(MFREE_ERR_ARG, "bad conduction mode");
    if (c->opt.tile_depth < 0 || c->opt.tile_depth > TILE_Z_MAX) return fail(MFREE_ERR_ARG, "tile_depth must be 0..8");
    int st = ensure_scratch(c);
    if (st) return st;
    {
        const StepArgs a = make_args(c);
        cudaError_t e = launch_interact_batch(BatchTable{}, lpp ? lpp : default_lpp(), a.p.cspm != 0, a.p.conduction,
                                              a.p.precision != 0, 0, c->stream);
        if (e != cudaSuccess) return fail(MFREE_ERR_CUDA, std::string("pair kernel setup: ") + cudaGetErrorString(e));
    }
    if (c->clock_dirty) return write_clock(c);
    return MFREE_OK;
}

cudaEvent_t pooled_event(mfree_ctx *c) {
    if (!c->event_pool.empty()) {
        cudaEvent_t e = c->event_pool.back();
        c->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// The context's one-scene table: its step arguments for both state parities
// (the clock kernel flips the parity on the device) and the block counts of
// each kernel family.  A single scene runs the batched kernels over this
// table, so its arithmetic is the same compiled code alone and in a batch.
// Uploaded again only when the arguments may have changed (setters bump the
// context's version); never inside a stream capture.
int ensure_table(mfree_ctx *c, int record_every) {
    if (c->d_table && c->table_version == c->version && c->table_record_every == record_every) return MFREE_OK;
    if (!c->d_table) {
        int st = dalloc(c, &c->d_table, single_table_bytes(), c->allocs);
        if (st) return st;
    }
    StepArgs args[2];
    const int keep = c->cur;
    for (int p = 0; p < 2; p++) {
        c->cur = p;
        args[p] = make_args(c);
        args[p].p.record_every = record_every;
    }
    c->cur = keep;
    const Params &P = args[0].p;
    const int ntiles = num_tiles(P);
    const int pre[10] = {0, hash_blocks(c), 0, scan_tiles(c), 0, int((c->num_cell + 255) / 256), 0, ntiles, 0, 0};
    StepArgs *da = (StepArgs *)c->d_table;
    int *di = (int *)(da + 2);
    // pageable sources: the call returns once the bytes are staged
    CUDA_TRY(cudaMemcpyAsync(da, args, sizeof(args), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(di, pre, sizeof(pre), cudaMemcpyHostToDevice, c->stream));
    c->T.args = da;
    c->T.pblk = di;
    c->T.stile = di + 2;
    c->T.cblk = di + 4;
    c->T.itile = di + 6;
    c->T.tile_next = di + 8;
    c->T.tile_count = di + 9;
    c->T.tile_list = c->d_tiles;
    c->T.nscenes = 1;
    c->ntiles = ntiles;
    c->table_version = c->version;
    c->table_record_every = record_every;
    return MFREE_OK;
}

// the kernels of one step; record_mode as kb_clock (2: every record_every
// steps of the scene's step index)
int enqueue_step(mfree_ctx *c, int record_mode, int record_every, bool timed = false) {
    int st = ensure_table(c, record_every);
    if (st) return st;
    const BatchTable &T = c->T;
    const Params &P = make_args(c).p;
    cudaStream_t s = c->stream;
    const int hb = hash_blocks(c), tiles = scan_tiles(c);
    const int nb = (c->n_init + 255) / 256;
    const int lpp = c->opt.lanes_per_particle ? c->opt.lanes_per_particle : default_lpp();
    cudaError_t le = cudaSuccess;
    auto run = [&](int id, auto &&launch) {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (timed) {
            e0 = pooled_event(c);
            e1 = pooled_event(c);
            cudaEventRecord(e0, s);
        }
        const TraceRange range(KERNEL_TRACE_NAMES[id]);
        launch();
        if (timed) {
            cudaEventRecord(e1, s);
            c->tev.push_back({id, {e0, e1}});
        }
    };
    run(0, [&] { kb_clock<<<1, 32, 0, s>>>(T, record_mode); });
    run(1, [&] { kb_hash<<<hb, HASH_BLOCK, 0, s>>>(T); });
    run(2, [&] { kb_scan_reduce<<<tiles, SCAN_THREADS, 0, s>>>(T); });
    run(3, [&] { kb_scan_top<<<1, 1024, 0, s>>>(T); });
    run(4, [&] { kb_scan_down<<<tiles, SCAN_THREADS, 0, s>>>(T); });
    run(5, [&] { kb_scatter<<<hb, HASH_BLOCK, 0, s>>>(T); });
    run(6, [&] { kb_cell_fixup<<<int((c->num_cell + 255) / 256) + (c->ntiles + 255) / 256, 256, 0, s>>>(T); });
    run(7, [&] { le = launch_gather_predict_batch(T, P.precision != 0, nb, s); });
    if (le == cudaSuccess)
        run(8, [&] { le = launch_interact_batch(T, lpp, P.cspm != 0, P.conduction, P.precision != 0, c->num_sms, s); });
    if (le != cudaSuccess) return fail(MFREE_ERR_CUDA, std::string("step launch: ") + cudaGetErrorString(le));
    run(9, [&] { kb_finalize<<<nb, 256, 0, s>>>(T); });
    if (!c->tools.empty()) run(10, [&] { kb_force_final<<<1, 256, 0, s>>>(T); });
    CUDA_TRY(cudaGetLastError());
    return MFREE_OK;
}

int copy_records(mfree_ctx *c, std::vector<Rec> &dst) {
    const int n = c->n_init;
    std::vector<float4> raw(size_t(REC_N) * n);
    CUDA_TRY(cudaMemcpyAsync(raw.data(), c->rec.f[0], sizeof(float4) * raw.size(), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    dst.resize(n);
    for (int i = 0; i < n; i++) {
        const float4 *x = raw.data() + size_t(n) + size_t(i) * REC_X;  // V, A, B, R, C of particle i
        dst[i] = Rec{raw[i], x[REC_V - 1], x[REC_A - 1], x[REC_B - 1], x[REC_R - 1], x[REC_C - 1]};
    }
    return MFREE_OK;
}

int copy_field_raw(mfree_ctx *c, const float4 *src, std::vector<float4> &dst) {
    dst.resize(c->n_init);
    CUDA_TRY(cudaMemcpyAsync(dst.data(), src, sizeof(float4) * c->n_init, cudaMemcpyDeviceToHost, c->stream));
    return MFREE_OK;
}

int check_empty(mfree_ctx *c, bool wait) {
    if (!c->nact_pending) return MFREE_OK;
    if (!wait && cudaEventQuery(c->nact_ev) != cudaSuccess) return MFREE_OK;
    CUDA_TRY(cudaEventSynchronize(c->nact_ev));
    c->nact_pending = false;
    if (c->h_nact[2] > 0)
        return fail(MFREE_ERR_TIMEOUT, "a staging wait of the pair kernel ran out: the step is incomplete (" +
                                           std::to_string(c->h_nact[2]) + " waits)");
    if (c->h_nact[0] == 0) return fail(MFREE_ERR_EMPTY, "all particles are blanked (outside the blanking box)");
    return MFREE_OK;
}

int note_active_count(mfree_ctx *c) {
    if (!c->h_nact) {
        CUDA_TRY(cudaMallocHost(&c->h_nact, 3 * sizeof(int)));
        CUDA_TRY(cudaEventCreateWithFlags(&c->nact_ev, cudaEventDisableTiming));
    }
    // n_active, record, staging_timeouts: adjacent in the device clock
    static_assert(offsetof(DevClock, staging_timeouts) == offsetof(DevClock, n_active) + 2 * sizeof(int), "clock layout");
    CUDA_TRY(cudaMemcpyAsync(c->h_nact, &c->d_clk->n_active, 3 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaEventRecord(c->nact_ev, c->stream));
    c->nact_pending = true;
    return MFREE_OK;
}

// device memory of a context: both state copies, the neighbour records, the
// per-particle scratch, the clock and the force outputs (the grid-sized
// scratch follows in ensure_scratch)
int alloc_ctx(int n, cudaStream_t stream, std::unique_ptr<mfree_ctx> &out) {
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    auto c = std::make_unique<mfree_ctx>();
    c->n_init = n;
    c->stream = stream;
    if (!c->stream) {  // own stream: graph capture is not allowed on the legacy default stream
        CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->own_stream = true;
    }
    c->device = dev;
    CUDA_TRY(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, dev));
    c->opt.max_secant_iter = 100;
    auto &L = c->allocs;
    auto bail = [&](int st) {
        free_list(c->allocs, c->stream);
        if (c->own_stream) cudaStreamDestroy(c->stream);
        return st;
    };
    int st;
    for (int b = 0; b < 2; b++) {
        State &S = c->st[b];
        float4 **f[] = {&S.pos4, &S.vel4, &S.sa4, &S.sb4, &S.da4, &S.dv4, &S.dsa4, &S.dsb4,
                        &S.fc4, &S.ft4, &S.bc4, &S.lo4, &S.lo4b};
        for (auto p : f)
            if ((st = dalloc(c.get(), p, n, L))) return bail(st);
    }
    {
        float4 *base = nullptr;
        if ((st = dalloc(c.get(), &base, size_t(REC_N) * n, L))) return bail(st);
        c->rec.f[REC_P] = base;
        for (int k = REC_V; k < REC_N; k++) c->rec.f[k] = base + size_t(n) + (k - REC_V);
    }
    if ((st = dalloc(c.get(), &c->scr.key, n, L))) return bail(st);
    if ((st = dalloc(c.get(), &c->scr.key_sorted, n, L))) return bail(st);
    if ((st = dalloc(c.get(), &c->scr.perm, n, L))) return bail(st);
    if ((st = dalloc(c.get(), &c->scr.blank_block, (n + HASH_BLOCK - 1) / HASH_BLOCK + 1, L))) return bail(st);
    if ((st = dalloc(c.get(), &c->scr.nnb, n, L))) return bail(st);
    if ((st = dalloc(c.get(), &c->scr.pos_half, n, L))) return bail(st);
    if ((st = dalloc(c.get(), &c->scr.nrm, n, L))) return bail(st);
    if ((st = dalloc(c.get(), &c->scr.force_part, size_t((n + 255) / 256) * 3 * MAX_TOOLS, L))) return bail(st);
    if ((st = dalloc(c.get(), &c->d_clk, 1, L))) return bail(st);
    if ((st = dalloc(c.get(), &c->d_forces, 3 * MAX_TOOLS, L))) return bail(st);
    c->scr.forces = c->d_forces;
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMemsetAsync(c->d_clk, 0, sizeof(DevClock), c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->d_forces, 0, sizeof(float) * 3 * MAX_TOOLS, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->scr.nnb, 0, sizeof(int) * n, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->scr.pos_half, 0, sizeof(float4) * n, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->scr.nrm, 0, sizeof(float4) * n, c->stream);
    if (e != cudaSuccess) return bail(fail(MFREE_ERR_CUDA, std::string("alloc_ctx: ") + cudaGetErrorString(e)));
    out = std::move(c);
    return MFREE_OK;
}

// the bytes alloc_ctx + ensure_scratch take (dalloc's max(n, 1) rule included)
size_t scene_bytes(int n, long long num_cell) {
    auto b = [](long long k, size_t sz) { return size_t(std::max<long long>(k, 1)) * sz; };
    const long long hb = (n + HASH_BLOCK - 1) / HASH_BLOCK, fb = (n + 255) / 256;
    const long long tiles = (num_cell + 1 + SCAN_TILE - 1) / SCAN_TILE;
    size_t t = 26 * b(n, sizeof(float4)) + b(REC_N * (long long)n, sizeof(float4));
    t += 3 * b(n, sizeof(int)) + b(hb + 1, sizeof(int)) + b(n, sizeof(int)) + 2 * b(n, sizeof(float4));
    t += b(fb * 3 * MAX_TOOLS, sizeof(float)) + b(1, sizeof(DevClock)) + b(3 * MAX_TOOLS, sizeof(float));
    t += b(num_cell + 1, sizeof(int)) + b(num_cell + 2 + SCAN_TILE, sizeof(int)) + b(tiles + 1, sizeof(int));
    t += b(num_cell + 1, sizeof(int2));
    t += single_table_bytes();
    return t;
}

int clone_ctx(const mfree_ctx *src, cudaStream_t s, std::unique_ptr<mfree_ctx> &out) {
    std::unique_ptr<mfree_ctx> c;
    int st = alloc_ctx(src->n_init, s, c);
    if (st) return st;
    c->phys = src->phys;
    c->corr = src->corr;
    c->joco = src->joco;
    c->twp = src->twp;
    c->ttool = src->ttool;
    c->opt = src->opt;
    c->plastic = src->plastic;
    c->grid_set = src->grid_set;
    for (int d = 0; d < 3; d++) {
        c->g_bbmin[d] = src->g_bbmin[d];
        c->g_bbmax[d] = src->g_bbmax[d];
        c->g_vel[d] = src->g_vel[d];
        c->b_min[d] = src->b_min[d];
        c->b_max[d] = src->b_max[d];
        c->b_vel[d] = src->b_vel[d];
    }
    c->g_dx = src->g_dx;
    c->nx = src->nx;
    c->ny = src->ny;
    c->nz = src->nz;
    c->num_cell = src->num_cell;
    c->grid_adaptive = src->grid_adaptive;
    c->max_cell = src->max_cell;
    c->blank_set = src->blank_set;
    c->b_vmax = src->b_vmax;
    c->dt = src->dt;
    c->t = src->t;
    c->time_set = src->time_set;
    c->steps = src->steps;
    c->cur = src->cur;
    c->pending = src->pending;
    for (const auto &t : src->tools) {
        auto d = std::make_unique<DevTool>(*t);
        d->d_tri = nullptr;
        d->d_cells = nullptr;
        const size_t ntri = size_t(10) * std::max(t->ntri_dev, 1), ncell = t->host.cells.size();
        CUDA_TRY(cudaMalloc(&d->d_tri, sizeof(float4) * ntri));
        CUDA_TRY(cudaMalloc(&d->d_cells, sizeof(int) * ncell));
        CUDA_TRY(cudaMemcpyAsync(d->d_tri, t->d_tri, sizeof(float4) * ntri, cudaMemcpyDeviceToDevice, s));
        CUDA_TRY(cudaMemcpyAsync(d->d_cells, t->d_cells, sizeof(int) * ncell, cudaMemcpyDeviceToDevice, s));
        c->bytes += sizeof(float4) * ntri + sizeof(int) * ncell;
        c->tools.push_back(std::move(d));
    }
    if ((st = ensure_scratch(c.get()))) return st;
    const State &A = src->st[src->cur], &B = c->st[src->cur];
    const float4 *from[] = {A.pos4, A.vel4, A.sa4, A.sb4, A.da4, A.dv4, A.dsa4, A.dsb4, A.fc4, A.ft4, A.bc4, A.lo4, A.lo4b};
    float4 *to[] = {B.pos4, B.vel4, B.sa4, B.sb4, B.da4, B.dv4, B.dsa4, B.dsb4, B.fc4, B.ft4, B.bc4, B.lo4, B.lo4b};
    for (int k = 0; k < 13; k++)
        CUDA_TRY(cudaMemcpyAsync(to[k], from[k], sizeof(float4) * src->n_init, cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(c->d_clk, src->d_clk, sizeof(DevClock), cudaMemcpyDeviceToDevice, s));
    c->clock_dirty = false;
    out = std::move(c);
    return MFREE_OK;
}

}  // namespace host
}  // namespace mfree

// ======================================================================= ABI
extern "C" {

const char *mfree_last_error(void) { return g_err.c_str(); }

int mfree_create(int n, const float *pos4, const float *vel4, const float *rho, const float *T, const float *h,
                 const float *fixed, const float *tool_p, void *stream, mfree_ctx **out) {
    if (!out || n <= 0 || !pos4 || !vel4 || !rho || !h) return fail(MFREE_ERR_ARG, "mfree_create: bad arguments");
    *out = nullptr;
    std::unique_ptr<mfree_ctx> c;
    int st = alloc_ctx(n, (cudaStream_t)stream, c);
    if (st) return st;
    // the caller's arrays go to the device as they are (staged in the record
    // buffer, which the first step overwrites) and a kernel builds the state:
    // the reference constructor's semantics, zeros except the given fields
    {
        float *stage = reinterpret_cast<float *>(c->rec.f[0]);  // REC_N * 4 floats per particle >= 8 + 5 here
        const size_t nn = size_t(n);
        float *d_pos = stage, *d_vel = stage + 4 * nn, *d_rho = stage + 8 * nn, *d_h = stage + 9 * nn;
        float *d_T = T ? stage + 10 * nn : nullptr, *d_fix = fixed ? stage + 11 * nn : nullptr,
              *d_tool = tool_p ? stage + 12 * nn : nullptr;
        auto up = [&](float *d, const float *hsrc, size_t count) {
            return cudaMemcpyAsync(d, hsrc, sizeof(float) * count, cudaMemcpyHostToDevice, c->stream);
        };
        CUDA_TRY(up(d_pos, pos4, 4 * nn));
        CUDA_TRY(up(d_vel, vel4, 4 * nn));
        CUDA_TRY(up(d_rho, rho, nn));
        CUDA_TRY(up(d_h, h, nn));
        if (T) CUDA_TRY(up(d_T, T, nn));
        if (fixed) CUDA_TRY(up(d_fix, fixed, nn));
        if (tool_p) CUDA_TRY(up(d_tool, tool_p, nn));
        CUDA_TRY(launch_init_state(n, reinterpret_cast<const float4 *>(d_pos), reinterpret_cast<const float4 *>(d_vel),
                                   d_rho, d_T, d_h, d_fix, d_tool, c->st[0], c->scr.perm, c->stream));
    }
    CUDA_TRY(cudaMemsetAsync(c->rec.f[0], 0, sizeof(float4) * REC_N * n, c->stream));
    CUDA_TRY(cudaMemsetAsync(c->scr.key_sorted, 0, sizeof(int) * n, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    *out = c.release();
    return MFREE_OK;
}

int mfree_destroy(mfree_ctx *c) {
    if (!c) return MFREE_OK;
    if (c->owner) return fail(MFREE_ERR_ARG, "mfree_destroy: the context belongs to a batch (retire it first)");
    finish_output(c, true);
    cudaStreamSynchronize(c->stream);
    invalidate_graphs(c);
    for (auto &t : c->tools) {
        if (t->d_tri) cudaFree(t->d_tri);
        if (t->d_cells) cudaFree(t->d_cells);
    }
    free_list(c->scratch_allocs, c->stream);
    free_list(c->allocs, c->stream);
    for (auto &t : c->tev) {
        cudaEventDestroy(t.second.first);
        cudaEventDestroy(t.second.second);
    }
    for (auto e : c->event_pool) cudaEventDestroy(e);
    for (auto e : c->timer)
        if (e) cudaEventDestroy(e);
    if (c->h_nact) cudaFreeHost(c->h_nact);
    if (c->h_bbox) cudaFreeHost(c->h_bbox);
    if (c->nact_ev) cudaEventDestroy(c->nact_ev);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
    return MFREE_OK;
}

int mfree_set_physics(mfree_ctx *c, const mfree_phys *p) {
    if (!c || !p) return fail(MFREE_ERR_ARG, "null argument");
    if (p->mass == 0.f || std::isnan(p->mass)) return fail(MFREE_ERR_ARG, "invalid particle mass");
    c->phys = *p;
    invalidate_graphs(c);
    return MFREE_OK;
}
int mfree_set_correctors(mfree_ctx *c, const mfree_corr *p) {
    if (!c || !p) return fail(MFREE_ERR_ARG, "null argument");
    c->corr = *p;
    invalidate_graphs(c);
    return MFREE_OK;
}
int mfree_set_johnson_cook(mfree_ctx *c, const mfree_joco *p) {
    if (!c || !p) return fail(MFREE_ERR_ARG, "null argument");
    c->joco = *p;
    c->plastic = true;
    invalidate_graphs(c);
    return MFREE_OK;
}
int mfree_set_thermal_workpiece(mfree_ctx *c, const mfree_trml *p) {
    if (!c || !p) return fail(MFREE_ERR_ARG, "null argument");
    c->twp = *p;
    invalidate_graphs(c);
    return MFREE_OK;
}
int mfree_set_thermal_tool(mfree_ctx *c, const mfree_trml *p) {
    if (!c || !p) return fail(MFREE_ERR_ARG, "null argument");
    c->ttool = *p;
    invalidate_graphs(c);
    return MFREE_OK;
}
int mfree_set_options(mfree_ctx *c, const mfree_options *o) {
    if (!c || !o) return fail(MFREE_ERR_ARG, "null argument");
    c->opt = *o;
    if (c->opt.max_secant_iter <= 0) c->opt.max_secant_iter = 100;
    invalidate_graphs(c);
    return MFREE_OK;
}
int mfree_get_options(const mfree_ctx *c, mfree_options *o) {
    if (!c || !o) return fail(MFREE_ERR_ARG, "null argument");
    *o = c->opt;
    return MFREE_OK;
}

int mfree_set_grid(mfree_ctx *c, const float bbmin[3], const float bbmax[3], float h) {
    if (!c || !bbmin || !bbmax || !(h > 0.f)) return fail(MFREE_ERR_ARG, "mfree_set_grid: bad arguments");
    // set_geometry (grid_gpu_base.cu:237-273) in float, as the reference
    for (int d = 0; d < 3; d++) {
        c->g_bbmin[d] = float(double(bbmin[d]) - 1e-6);
        c->g_bbmax[d] = float(double(bbmax[d]) + 1e-6);
    }
    float kernel_width = 2.f;
    c->g_dx = float(double(h * kernel_width) / 2.);
    float lx = c->g_bbmax[0] - c->g_bbmin[0], ly = c->g_bbmax[1] - c->g_bbmin[1], lz = c->g_bbmax[2] - c->g_bbmin[2];
    c->nx = long(std::ceil(lx / c->g_dx));
    c->ny = long(std::ceil(ly / c->g_dx));
    c->nz = long(std::ceil(lz / c->g_dx));
    if (c->nx <= 0 || c->ny <= 0 || c->nz <= 0) return fail(MFREE_ERR_ARG, "empty grid");
    long nc = c->nx * c->ny * c->nz;
    if (nc >= long(INT_MAX) / 2) return fail(MFREE_ERR_ARG, "grid has too many cells");
    c->num_cell = nc;
    c->grid_set = true;
    c->grid_adaptive = false;
    c->clock_dirty = true;
    invalidate_graphs(c);
    return MFREE_OK;
}
int mfree_set_grid_adaptive(mfree_ctx *c, long max_cell) {
    if (!c || max_cell < 2 || max_cell >= long(INT_MAX) / 2) return fail(MFREE_ERR_ARG, "mfree_set_grid_adaptive: bad arguments");
    if (c->owner) return fail(MFREE_ERR_ARG, "mfree_set_grid_adaptive: the context belongs to a batch");
    c->grid_adaptive = true;
    c->max_cell = max_cell;
    // a placeholder grid until the first step bounds the particles
    c->nx = c->ny = c->nz = 1;
    c->num_cell = 1;
    c->g_dx = 0.f;
    for (int d = 0; d < 3; d++) c->g_bbmin[d] = c->g_bbmax[d] = 0.f;
    c->grid_set = true;
    c->clock_dirty = true;
    invalidate_graphs(c);
    return MFREE_OK;
}
int mfree_set_grid_velocity(mfree_ctx *c, const float vel[3]) {
    if (!c || !vel) return fail(MFREE_ERR_ARG, "null argument");
    for (int d = 0; d < 3; d++) c->g_vel[d] = vel[d];
    invalidate_graphs(c);
    return MFREE_OK;
}
int mfree_set_blanking(mfree_ctx *c, const float bbmin[3], const float bbmax[3], const float *bbvel3, float max_vel) {
    if (!c || !bbmin || !bbmax) return fail(MFREE_ERR_ARG, "null argument");
    for (int d = 0; d < 3; d++) {
        c->b_min[d] = bbmin[d];
        c->b_max[d] = bbmax[d];
        c->b_vel[d] = bbvel3 ? bbvel3[d] : 0.f;
    }
    c->b_vmax = max_vel;
    c->blank_set = true;
    c->clock_dirty = true;
    invalidate_graphs(c);
    return MFREE_OK;
}
int mfree_set_time(mfree_ctx *c, float dt, float t) {
    if (!c || !(dt > 0.f)) return fail(MFREE_ERR_ARG, "mfree_set_time: dt must be > 0");
    if (c->pending) {  // bring the host clock in line with the device before overwriting
        mfree_sync(c);
    }
    c->dt = dt;
    c->t = t;
    c->time_set = true;
    c->clock_dirty = true;
    invalidate_graphs(c);
    return MFREE_OK;
}
int mfree_get_time(const mfree_ctx *c, float *dt, float *t) {
    if (!c) return fail(MFREE_ERR_ARG, "null argument");
    if (dt) *dt = c->dt;
    if (t) *t = c->pending ? c->t + c->dt : c->t;  // main() adds dt after each step
    return MFREE_OK;
}

int mfree_add_tool(mfree_ctx *c, const float *verts, int nv, const int *tris, int nt, const float vel[3],
                   float contact_alpha, float mu, int algorithm, int *tool_index) {
    if (!c || !verts || !tris || !vel) return fail(MFREE_ERR_ARG, "mfree_add_tool: null argument");
    if (c->tools.size() >= size_t(MAX_TOOLS)) return fail(MFREE_ERR_ARG, "mfree_add_tool: at most 8 tools");
    if (algorithm != MFREE_CONTACT_HASHED && algorithm != MFREE_CONTACT_EXHAUSTIVE)
        return fail(MFREE_ERR_ARG, "mfree_add_tool: unknown contact algorithm");
    auto t = std::make_unique<DevTool>();
    std::string err;
    if (!build_host_tool(t->host, verts, nv, tris, nt, err)) return fail(MFREE_ERR_ARG, "mfree_add_tool: " + err);
    t->algorithm = algorithm;
    t->verts.assign(verts, verts + 3 * size_t(nv));
    for (int d = 0; d < 3; d++) t->vel[d] = vel[d];
    t->alpha = contact_alpha;
    t->mu = mu;
    const std::vector<HostTri> &src = algorithm == MFREE_CONTACT_HASHED ? t->host.boxed : t->host.tris;
    const int n = int(src.size());
    t->ntri_dev = n;
    std::vector<float4> h(size_t(10) * std::max(n, 1));
    auto f4 = [](Vec3f v) { return make_float4(v.x, v.y, v.z, 0.f); };
    for (int k = 0; k < n; k++) {
        const HostTri &q = src[k];
        h[k] = f4(q.p1);
        h[n + k] = f4(q.p2);
        h[2 * n + k] = f4(q.p3);
        h[3 * n + k] = f4(q.n);
        h[4 * n + k] = f4(q.np1);
        h[5 * n + k] = f4(q.np2);
        h[6 * n + k] = f4(q.np3);
        h[7 * n + k] = f4(q.ne1);
        h[8 * n + k] = f4(q.ne2);
        h[9 * n + k] = f4(q.ne3);
    }
    CUDA_TRY(cudaMalloc(&t->d_tri, sizeof(float4) * h.size()));
    CUDA_TRY(cudaMemcpy(t->d_tri, h.data(), sizeof(float4) * h.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMalloc(&t->d_cells, sizeof(int) * t->host.cells.size()));
    c->bytes += sizeof(float4) * h.size() + sizeof(int) * t->host.cells.size();
    CUDA_TRY(cudaMemcpy(t->d_cells, t->host.cells.data(), sizeof(int) * t->host.cells.size(), cudaMemcpyHostToDevice));
    c->tools.push_back(std::move(t));
    if (tool_index) *tool_index = int(c->tools.size()) - 1;
    c->clock_dirty = true;
    invalidate_graphs(c);
    return MFREE_OK;
}
int mfree_tool_set_birth_death(mfree_ctx *c, int k, float birth, float death) {
    if (!c || k < 0 || k >= int(c->tools.size())) return fail(MFREE_ERR_ARG, "bad tool index");
    c->tools[k]->birth = birth;
    c->tools[k]->death = death;
    invalidate_graphs(c);
    return MFREE_OK;
}
int mfree_get_tool_forces(mfree_ctx *c, float *out3) {
    if (!c || !out3) return fail(MFREE_ERR_ARG, "null argument");
    if (c->tools.empty()) return MFREE_OK;
    CUDA_TRY(cudaMemcpyAsync(out3, c->d_forces, sizeof(float) * 3 * c->tools.size(), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return MFREE_OK;
}
int mfree_get_tool_info(mfree_ctx *c, int k, int *num_tris, int *num_boxed, int *grid_n3, float *bbmin3,
                        float *bbmax3, float *cell_dx) {
    if (!c || k < 0 || k >= int(c->tools.size())) return fail(MFREE_ERR_ARG, "bad tool index");
    const HostTool &t = c->tools[k]->host;
    if (num_tris) *num_tris = int(t.tris.size());
    if (num_boxed) *num_boxed = int(t.boxed.size());
    if (grid_n3) { grid_n3[0] = t.nx; grid_n3[1] = t.ny; grid_n3[2] = t.nz; }
    for (int d = 0; d < 3; d++) {
        if (bbmin3) bbmin3[d] = t.bbmin[d];
        if (bbmax3) bbmax3[d] = t.bbmax[d];
    }
    if (cell_dx) *cell_dx = t.dx;
    return MFREE_OK;
}
int mfree_get_tool_normals(mfree_ctx *c, int k, float *out) {
    if (!c || !out || k < 0 || k >= int(c->tools.size())) return fail(MFREE_ERR_ARG, "bad tool index");
    const HostTool &t = c->tools[k]->host;
    for (size_t i = 0; i < t.tris.size(); i++) {
        const HostTri &q = t.tris[i];
        const Vec3f v[7] = {q.n, q.np1, q.np2, q.np3, q.ne1, q.ne2, q.ne3};
        for (int a = 0; a < 7; a++) {
            out[i * 21 + a * 3] = v[a].x;
            out[i * 21 + a * 3 + 1] = v[a].y;
            out[i * 21 + a * 3 + 2] = v[a].z;
        }
    }
    return MFREE_OK;
}
int mfree_get_tool_cells(mfree_ctx *c, int k, int *cells, int *boxed_src) {
    if (!c || k < 0 || k >= int(c->tools.size())) return fail(MFREE_ERR_ARG, "bad tool index");
    const HostTool &t = c->tools[k]->host;
    if (cells) std::memcpy(cells, t.cells.data(), sizeof(int) * t.cells.size());
    if (boxed_src) std::memcpy(boxed_src, t.boxed_src.data(), sizeof(int) * t.boxed_src.size());
    return MFREE_OK;
}

// Bounding box of the first n particles of the current order and their
// largest h (update_geometry's unlocked branch, grid_gpu_base.cu:185-204; n =
// the active count when blanking is on, as particles->N, else n_init).
// Floats are reduced as order-preserving int keys, so atomicMin/atomicMax give
// the exact extremes; NaN coordinates are left out.
__device__ __forceinline__ int float_key(float f) {
    const int b = __float_as_int(f);
    return b >= 0 ? b : b ^ 0x7fffffff;
}
float key_float(int k) {
    const int b = k >= 0 ? k : k ^ 0x7fffffff;
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}
__global__ void k_bbox_init(int *out) {
    if (threadIdx.x < 7) out[threadIdx.x] = threadIdx.x < 3 ? INT_MAX : INT_MIN;  // min xyz, max xyz, max h
}
__global__ void __launch_bounds__(256) k_bbox(const float4 *pos, int n_init, const DevClock *clk, int use_active,
                                              int *out) {
    const int n = use_active ? min(clk->n_active, n_init) : n_init;
    int k[7] = {INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN, INT_MIN};
    for (int i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) {
        const float4 p = pos[i];
        const float v[4] = {p.x, p.y, p.z, p.w};
#pragma unroll
        for (int d = 0; d < 3; d++)
            if (!isnan(v[d])) {
                k[d] = min(k[d], float_key(v[d]));
                k[3 + d] = max(k[3 + d], float_key(v[d]));
            }
        if (!isnan(p.w)) k[6] = max(k[6], float_key(p.w));
    }
#pragma unroll
    for (int d = 0; d < 7; d++) k[d] = d < 3 ? __reduce_min_sync(0xffffffffu, k[d]) : __reduce_max_sync(0xffffffffu, k[d]);
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int d = 0; d < 7; d++) {
            if (d < 3) atomicMin(out + d, k[d]);
            else atomicMax(out + d, k[d]);
        }
    }
}

// the unlocked grid of this step from the particles (grid_gpu_base.cu:185-233),
// in the reference's float arithmetic
int adapt_grid(mfree_ctx *c) {
    if (!c->d_bbox) {
        int st = dalloc(c, &c->d_bbox, 8, c->allocs);
        if (st) return st;
        CUDA_TRY(cudaMallocHost(&c->h_bbox, 8 * sizeof(int)));
    }
    const int blocks = std::max(1, std::min((c->n_init + 255) / 256, 4 * c->num_sms));
    k_bbox_init<<<1, 32, 0, c->stream>>>(c->d_bbox);
    k_bbox<<<blocks, 256, 0, c->stream>>>(c->st[c->cur].pos4, c->n_init, c->d_clk, c->blank_set ? 1 : 0, c->d_bbox);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(c->h_bbox, c->d_bbox, 7 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (c->h_bbox[0] == INT_MAX || c->h_bbox[6] == INT_MIN)
        return fail(MFREE_ERR_EMPTY, "the unlocked grid has no particle to bound");
    float bbmin[3], bbmax[3];
    for (int d = 0; d < 3; d++) {
        bbmin[d] = float(double(key_float(c->h_bbox[d])) - 1e-6);
        bbmax[d] = float(double(key_float(c->h_bbox[3 + d])) + 1e-6);
    }
    const float kernel_width = 2.f;
    const float dx = key_float(c->h_bbox[6]) * kernel_width / 2;
    long n3[3];
    for (int d = 0; d < 3; d++) {
        const float l = bbmax[d] - bbmin[d];
        const float q = std::ceil(l / dx);
        if (!(q >= 1.f && q < 1e9f)) return fail(MFREE_ERR_ARG, "the unlocked grid has an unusable size");
        n3[d] = long(q);
    }
    const long nc = n3[0] * n3[1] * n3[2];
    if (nc >= c->max_cell)
        return fail(MFREE_ERR_ARG, "the unlocked grid needs " + std::to_string(nc) + " cells, max_cell is " +
                                       std::to_string(c->max_cell) + " (grid_gpu_base.cu:227-232 asserts)");
    bool same = dx == c->g_dx && n3[0] == c->nx && n3[1] == c->ny && n3[2] == c->nz;
    for (int d = 0; d < 3; d++) same = same && bbmin[d] == c->g_bbmin[d] && bbmax[d] == c->g_bbmax[d];
    if (same) return MFREE_OK;
    for (int d = 0; d < 3; d++) {
        c->g_bbmin[d] = bbmin[d];
        c->g_bbmax[d] = bbmax[d];
    }
    c->g_dx = dx;
    c->nx = n3[0];
    c->ny = n3[1];
    c->nz = n3[2];
    c->num_cell = nc;
    invalidate_graphs(c);  // the step arguments hold the grid: the table is written again
    return MFREE_OK;
}

int mfree_step(mfree_ctx *c, int record_forces) {
    if (!c) return fail(MFREE_ERR_ARG, "null context");
    const TraceRange range("mfree_step");
    if (c->owner) return fail(MFREE_ERR_ARG, "mfree_step: the context belongs to a batch (mfree_batch_step steps it)");
    int st = ready(c);
    if (st) return st;
    if ((st = check_empty(c, false))) return st;
    if (c->grid_adaptive && (st = adapt_grid(c))) return st;
    if ((st = enqueue_step(c, record_forces ? 1 : 0, 0, c->timing))) return st;
    if ((st = note_active_count(c))) return st;
    c->cur ^= 1;
    if (c->pending) c->t = c->t + c->dt;
    c->pending = true;
    c->steps++;
    return MFREE_OK;
}

int mfree_advance(mfree_ctx *c, int nsteps, int record_every, int use_graph) {
    if (!c || nsteps < 0) return fail(MFREE_ERR_ARG, "bad arguments");
    const TraceRange range("mfree_advance");
    if (c->owner) return fail(MFREE_ERR_ARG, "mfree_advance: the context belongs to a batch (mfree_batch_step steps it)");
    int st = ready(c);
    if (st) return st;
    if ((st = check_empty(c, false))) return st;
    if (!use_graph || c->grid_adaptive) {  // an unlocked grid is read back before every step: no graph
        for (int k = 0; k < nsteps; k++) {
            const bool rec = record_every > 0 && (c->steps % record_every) == 0;
            if (c->grid_adaptive && (st = adapt_grid(c))) return st;
            if ((st = enqueue_step(c, rec ? 1 : 0, 0))) return st;
            c->cur ^= 1;
            if (c->pending) c->t = c->t + c->dt;
            c->pending = true;
            c->steps++;
        }
        return MFREE_OK;
    }
    if (!c->graph || c->graph_record_every != record_every) {
        invalidate_graphs(c);
        // one graph serves both state parities (the parity flips on the device)
        if ((st = ensure_table(c, record_every))) return st;
        cudaGraph_t g = nullptr;
        CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        int e = enqueue_step(c, 2, record_every);
        cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
        if (e) {
            if (g) cudaGraphDestroy(g);
            return e;
        }
        if (ce != cudaSuccess) return fail(MFREE_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
        cudaError_t ie = cudaGraphInstantiate(&c->graph, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) return fail(MFREE_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
        c->graph_record_every = record_every;
    }
    for (int k = 0; k < nsteps; k++) {
        CUDA_TRY(cudaGraphLaunch(c->graph, c->stream));
        c->cur ^= 1;
        if (c->pending) c->t = c->t + c->dt;
        c->pending = true;
        c->steps++;
    }
    return note_active_count(c);
}

int mfree_set_kernel_timing(mfree_ctx *c, int on) {
    if (!c) return fail(MFREE_ERR_ARG, "null context");
    c->timing = on != 0;
    return MFREE_OK;
}

int mfree_get_kernel_times(mfree_ctx *c, double *ms, int *launches) {
    if (!c) return fail(MFREE_ERR_ARG, "null context");
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    for (auto &t : c->tev) {
        float x = 0.f;
        CUDA_TRY(cudaEventElapsedTime(&x, t.second.first, t.second.second));
        c->kernel_ms[t.first] += x;
        c->kernel_n[t.first] += 1;
        c->event_pool.push_back(t.second.first);
        c->event_pool.push_back(t.second.second);
    }
    c->tev.clear();
    for (int k = 0; k < MFREE_NUM_KERNELS; k++) {
        if (ms) ms[k] = c->kernel_ms[k];
        if (launches) launches[k] = c->kernel_n[k];
        c->kernel_ms[k] = 0.0;
        c->kernel_n[k] = 0;
    }
    return MFREE_OK;
}

int mfree_timer_start(mfree_ctx *c) {
    if (!c) return fail(MFREE_ERR_ARG, "null context");
    for (auto &e : c->timer)
        if (!e) CUDA_TRY(cudaEventCreate(&e));
    CUDA_TRY(cudaEventRecord(c->timer[0], c->stream));
    return MFREE_OK;
}

int mfree_timer_stop(mfree_ctx *c, double *ms) {
    if (!c || !ms || !c->timer[0]) return fail(MFREE_ERR_ARG, "timer not started");
    CUDA_TRY(cudaEventRecord(c->timer[1], c->stream));
    CUDA_TRY(cudaEventSynchronize(c->timer[1]));
    float x = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&x, c->timer[0], c->timer[1]));
    *ms = x;
    return MFREE_OK;
}

int mfree_set_device(int device) {
    CUDA_TRY(cudaSetDevice(device));
    return MFREE_OK;
}

int mfree_probe_fp32_peak(double *tflops) {
    if (!tflops) return fail(MFREE_ERR_ARG, "null argument");
    int dev = 0, sms = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    *tflops = fp32_peak_probe(sms);
    if (!(*tflops > 0.0)) return fail(MFREE_ERR_CUDA, "FP32 probe failed");
    return MFREE_OK;
}

int mfree_sync(mfree_ctx *c) {
    if (!c) return fail(MFREE_ERR_ARG, "null context");
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return check_empty(c, true);
}

int mfree_get_counts(const mfree_ctx *c, int *n_active, int *n_init) {
    if (!c) return fail(MFREE_ERR_ARG, "null context");
    if (n_init) *n_init = c->n_init;
    if (n_active) {
        DevClock h{};
        CUDA_TRY(cudaMemcpyAsync(&h, c->d_clk, sizeof(DevClock), cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(cudaStreamSynchronize(c->stream));
        *n_active = c->steps ? h.n_active : c->n_init;
    }
    return MFREE_OK;
}

int mfree_inject_fault(mfree_ctx *c, int kind) {
    if (!c) return fail(MFREE_ERR_ARG, "null context");
    if (kind != MFREE_FAULT_NONE && kind != MFREE_FAULT_STAGING_WAIT) return fail(MFREE_ERR_ARG, "unknown fault kind");
    c->inject_staging = kind == MFREE_FAULT_STAGING_WAIT;
    invalidate_graphs(c);  // the step arguments change
    return MFREE_OK;
}

int mfree_get_counters(mfree_ctx *c, mfree_counters *o) {
    if (!c || !o) return fail(MFREE_ERR_ARG, "null argument");
    DevClock h{};
    CUDA_TRY(cudaMemcpyAsync(&h, c->d_clk, sizeof(DevClock), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    o->steps = c->steps;
    o->secant_failures = int64_t(h.secant_failures);
    o->out_of_grid = int64_t(h.out_of_grid);
    o->contact_search_cap = int64_t(h.contact_cap);
    o->nan_blanked = int64_t(h.nan_blanked);
    o->staging_timeouts = int64_t(h.staging_timeouts);
    o->full_stencil_steps = int64_t(h.full_stencil_steps);
    o->bounds_errors = int64_t(h.bounds_errors);
    o->pse_zero_targets = int64_t(h.pse_zero_targets);
    return MFREE_OK;
}

// FP64 energy and CFL reductions: per-block partials in double, then one
// block sums them in a fixed order (deterministic)
constexpr int ENERGY_BLOCK = 256, ENERGY_VALUES = 5;
__global__ void __launch_bounds__(ENERGY_BLOCK) k_energy_partial(State S, const DevClock *clk, int n_init, int stepped,
                                                                 int prec, float mass,
                                                                 float K, float G, float rho0, float c0sq, float cp,
                                                                 float T0, double *part) {
    __shared__ double red[ENERGY_VALUES][ENERGY_BLOCK / 32];
    const int n = stepped ? min(clk->n_active, n_init) : n_init;  // active particles lead the sorted order
    const int i = blockIdx.x * ENERGY_BLOCK + threadIdx.x;
    double v[ENERGY_VALUES] = {0.0, 0.0, 0.0, 0.0, 1e300};
    if (i < n) {
        const float4 vel = S.vel4[i], sa = S.sa4[i], sb = S.sb4[i], pos = S.pos4[i];
        if (S.fc4[i].w != 1.f && S.ft4[i].w != 1.f) {  // workpiece, not blanked
            double vx = vel.x, vy = vel.y, vz = vel.z;
            const double rho = vel.w;
            if (prec) {  // the precision form: velocity = hi + lo of the compensated accumulation
                const float4 lo = S.lo4[i], lob = S.lo4b[i];
                vx += double(lo.w);
                vy += double(lob.x);
                vz += double(lob.y);
            }
            const double v2 = vx * vx + vy * vy + vz * vz;
            const double ss = double(sa.x) * sa.x + double(sa.y) * sa.y + double(sa.z) * sa.z +
                              2.0 * (double(sa.w) * sa.w + double(sb.x) * sb.x + double(sb.y) * sb.y);
            const double p = double(c0sq) * (rho - double(rho0));
            const double vol = double(mass) / rho;
            v[0] = 0.5 * double(mass) * v2;
            v[1] = vol * ss / (4.0 * double(G));
            v[2] = vol * p * p / (2.0 * double(K));
            v[3] = double(mass) * double(cp) * (double(sb.z) - double(T0));
            v[4] = double(pos.w) / (sqrt(double(K) / rho) + sqrt(v2));
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < ENERGY_VALUES; k++) {
        double x = v[k];
        for (int o = 16; o >= 1; o >>= 1) {
            const double y = __shfl_xor_sync(0xffffffffu, x, o);
            x = k < 4 ? x + y : fmin(x, y);
        }
        if (lane == 0) red[k][warp] = x;
    }
    __syncthreads();
    if (threadIdx.x < ENERGY_VALUES) {
        const int k = threadIdx.x;
        double x = red[k][0];
        for (int w = 1; w < ENERGY_BLOCK / 32; w++) x = k < 4 ? x + red[k][w] : fmin(x, red[k][w]);
        part[size_t(blockIdx.x) * ENERGY_VALUES + k] = x;
    }
}
__global__ void __launch_bounds__(ENERGY_VALUES * 32) k_energy_final(const double *part, int nb, double *out) {
    const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double x = k < 4 ? 0.0 : 1e300;
    for (int b = lane; b < nb; b += 32) {
        const double y = part[size_t(b) * ENERGY_VALUES + k];
        x = k < 4 ? x + y : fmin(x, y);
    }
    for (int o = 16; o >= 1; o >>= 1) {
        const double y = __shfl_xor_sync(0xffffffffu, x, o);
        x = k < 4 ? x + y : fmin(x, y);
    }
    if (lane == 0) out[k] = x;
}

int mfree_get_energies(mfree_ctx *c, double out[5]) {
    if (!c || !out) return fail(MFREE_ERR_ARG, "null argument");
    if (!(c->phys.G > 0.f) || !(c->phys.K > 0.f) || !(c->phys.rho0 > 0.f))
        return fail(MFREE_ERR_ARG, "mfree_get_energies: physics constants not set");
    const int nb = std::max(1, (c->n_init + ENERGY_BLOCK - 1) / ENERGY_BLOCK);
    if (!c->d_energy) {
        int st = dalloc(c, &c->d_energy, size_t(nb) * ENERGY_VALUES + ENERGY_VALUES, c->allocs);
        if (st) return st;
    }
    const float c0 = std::sqrt(c->phys.K / c->phys.rho0);
    k_energy_partial<<<nb, ENERGY_BLOCK, 0, c->stream>>>(c->st[c->cur], c->d_clk, c->n_init, c->steps > 0 ? 1 : 0,
                                                          c->opt.precision ? 1 : 0, c->phys.mass,
                                                          c->phys.K, c->phys.G, c->phys.rho0, c0 * c0, c->twp.cp,
                                                          c->twp.T_init, c->d_energy + ENERGY_VALUES);
    k_energy_final<<<1, ENERGY_VALUES * 32, 0, c->stream>>>(c->d_energy + ENERGY_VALUES, nb, c->d_energy);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(out, c->d_energy, sizeof(double) * ENERGY_VALUES, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return MFREE_OK;
}

int mfree_bounds_checked(void) {
#ifdef MFREE_BOUNDS_CHECK
    return 1;
#else
    return 0;
#endif
}

int mfree_field_width(int f) {
    switch (f) {
        case MFREE_POS: case MFREE_VEL: case MFREE_VEL_BC: case MFREE_POS_HALF: return 4;
        case MFREE_S: case MFREE_R: case MFREE_S_T: return 9;
        case MFREE_FC: case MFREE_FT: case MFREE_NRM: case MFREE_POS_T: case MFREE_VEL_T: return 3;
        default: return (f >= 0 && f < MFREE_NUM_FIELDS) ? 1 : -1;
    }
}

namespace {

// symmetric 6 (xx yy zz xy xz yz) -> GLM column-major 9
inline void sym_to_9(const float s[6], float *o) {
    o[0] = s[0]; o[1] = s[3]; o[2] = s[4];
    o[3] = s[3]; o[4] = s[1]; o[5] = s[5];
    o[6] = s[4]; o[7] = s[5]; o[8] = s[2];
}

// One field of the state in the reference layout, written by the device
// straight into page-locked host memory (dst is its device alias).  A block's
// 256 entries are assembled in shared memory and stored as one contiguous run,
// so the writes that cross the host link are whole lines.  Fields the kernel
// does not know (returns false) go through the host path below.
__host__ __device__ constexpr bool field_on_device(int f) {
    return f == MFREE_POS || f == MFREE_VEL || f == MFREE_VEL_BC || f == MFREE_H || f == MFREE_RHO || f == MFREE_S ||
           f == MFREE_S_T || f == MFREE_FC || f == MFREE_FT || f == MFREE_POS_T || f == MFREE_VEL_T ||
           f == MFREE_FIXED || f == MFREE_EPS_PL_DOT || f == MFREE_BLANKED || f == MFREE_TOOL_PARTICLE ||
           f == MFREE_EPS_PL || f == MFREE_T || f == MFREE_RHO_T || f == MFREE_T_T || f == MFREE_ID;
}

__global__ void __launch_bounds__(256) k_get_field(int f, int w, State S, int n, float *dst) {
    __shared__ float buf[256 * 9];
    const int i0 = blockIdx.x * 256, i = i0 + threadIdx.x;
    if (i < n) {
        float *o = buf + threadIdx.x * w;
        auto xyz = [&](float4 v) { o[0] = v.x; o[1] = v.y; o[2] = v.z; if (w == 4) o[3] = 0.f; };
        auto sym9 = [&](float4 a, float4 b) {  // (xx yy zz xy) (xz yz): GLM column-major 3x3
            o[0] = a.x; o[1] = a.w; o[2] = b.x;
            o[3] = a.w; o[4] = a.y; o[5] = b.y;
            o[6] = b.x; o[7] = b.y; o[8] = a.z;
        };
        switch (f) {
            case MFREE_POS: xyz(S.pos4[i]); break;
            case MFREE_VEL: xyz(S.vel4[i]); break;
            case MFREE_VEL_BC: xyz(S.bc4[i]); break;
            case MFREE_H: o[0] = S.pos4[i].w; break;
            case MFREE_RHO: o[0] = S.vel4[i].w; break;
            case MFREE_S: sym9(S.sa4[i], S.sb4[i]); break;
            case MFREE_S_T: sym9(S.dsa4[i], S.dsb4[i]); break;
            case MFREE_FC: xyz(S.fc4[i]); break;
            case MFREE_FT: xyz(S.ft4[i]); break;
            case MFREE_POS_T: xyz(S.da4[i]); break;
            case MFREE_VEL_T: xyz(S.dv4[i]); break;
            case MFREE_FIXED: o[0] = S.dsb4[i].w; break;
            case MFREE_EPS_PL_DOT: o[0] = S.dsb4[i].z; break;
            case MFREE_BLANKED: o[0] = S.ft4[i].w; break;
            case MFREE_TOOL_PARTICLE: o[0] = S.fc4[i].w; break;
            case MFREE_EPS_PL: o[0] = S.sb4[i].w; break;
            case MFREE_T: o[0] = S.sb4[i].z; break;
            case MFREE_RHO_T: o[0] = S.da4[i].w; break;
            case MFREE_T_T: o[0] = S.dv4[i].w; break;
            case MFREE_ID: o[0] = S.bc4[i].w; break;  // the id's int bits
            default: break;
        }
    }
    __syncthreads();
    const int cnt = min(256, n - i0) * w;
    float *d = dst + size_t(i0) * w;
    for (int k = threadIdx.x; k < cnt; k += 256) d[k] = buf[k];
}

// the device path of mfree_get_field: 1 when done, 0 when out is not
// page-locked memory the device can write (the host path then runs)
int get_field_pinned(mfree_ctx *c, int f, float *out, int *st) {
    *st = MFREE_OK;
    if (!field_on_device(f)) return 0;
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, out) != cudaSuccess) {
        cudaGetLastError();  // not a pointer CUDA knows: clear the error
        return 0;
    }
    if (at.type != cudaMemoryTypeHost || !at.devicePointer) return 0;
    const int n = c->n_init, w = mfree_field_width(f);
    if (n > 0) {
        k_get_field<<<(n + 255) / 256, 256, 0, c->stream>>>(f, w, c->st[c->cur], n, (float *)at.devicePointer);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) *st = fail(MFREE_ERR_CUDA, std::string("mfree_get_field: ") + cudaGetErrorString(e));
    }
    return 1;
}

int get_field_impl(mfree_ctx *c, int f, float *fo, double *dout) {
    const int n = c->n_init;
    const State &S = c->st[c->cur];
    if (fo && !dout) {
        int st = MFREE_OK;
        if (get_field_pinned(c, f, fo, &st)) return st;
    }
    std::vector<float4> A, B, C;
    int st = 0;
    const int w = mfree_field_width(f);
    if (w < 0) return fail(MFREE_ERR_ARG, "unknown field");
    std::vector<float> tmp(size_t(n) * w);
    auto put = [&](int i, int k, float v) { tmp[size_t(i) * w + k] = v; };
    auto ints = [&](const int *dsrc, bool map_hash) -> int {
        std::vector<int> v(n);
        CUDA_TRY(cudaMemcpyAsync(v.data(), dsrc, sizeof(int) * n, cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(cudaStreamSynchronize(c->stream));
        for (int i = 0; i < n; i++) {
            int x = v[i];
            if (map_hash && x >= int(c->num_cell)) x = INT_MAX;
            if (fo) std::memcpy(&fo[i], &x, 4);
            if (dout) dout[i] = double(x);
        }
        return MFREE_OK;
    };
    switch (f) {
        case MFREE_POS:
        case MFREE_VEL: {
            if ((st = copy_field_raw(c, f == MFREE_POS ? S.pos4 : S.vel4, A))) return st;
            if (c->opt.precision && dout) {
                if ((st = copy_field_raw(c, S.lo4, B))) return st;
                if ((st = copy_field_raw(c, S.lo4b, C))) return st;
            }
            CUDA_TRY(cudaStreamSynchronize(c->stream));
            for (int i = 0; i < n; i++) {
                put(i, 0, A[i].x); put(i, 1, A[i].y); put(i, 2, A[i].z); put(i, 3, 0.f);
            }
            if (c->opt.precision && dout) {
                for (int i = 0; i < n; i++) {
                    double lo[3] = {f == MFREE_POS ? B[i].x : B[i].w, f == MFREE_POS ? B[i].y : C[i].x,
                                    f == MFREE_POS ? B[i].z : C[i].y};
                    dout[4 * i] = double(A[i].x) + lo[0];
                    dout[4 * i + 1] = double(A[i].y) + lo[1];
                    dout[4 * i + 2] = double(A[i].z) + lo[2];
                    dout[4 * i + 3] = 0.0;
                }
                return MFREE_OK;
            }
            break;
        }
        case MFREE_VEL_BC:
            if ((st = copy_field_raw(c, S.bc4, A))) return st;
            CUDA_TRY(cudaStreamSynchronize(c->stream));
            for (int i = 0; i < n; i++) { put(i, 0, A[i].x); put(i, 1, A[i].y); put(i, 2, A[i].z); put(i, 3, 0.f); }
            break;
        case MFREE_H:
            if ((st = copy_field_raw(c, S.pos4, A))) return st;
            CUDA_TRY(cudaStreamSynchronize(c->stream));
            for (int i = 0; i < n; i++) put(i, 0, A[i].w);
            break;
        case MFREE_RHO:
            if ((st = copy_field_raw(c, S.vel4, A))) return st;
            CUDA_TRY(cudaStreamSynchronize(c->stream));
            for (int i = 0; i < n; i++) put(i, 0, A[i].w);
            break;
        case MFREE_P: {
            std::vector<Rec> R;
            if ((st = copy_records(c, R))) return st;
            float c0 = std::sqrt(c->phys.rho0 != 0.f ? c->phys.K / c->phys.rho0 : 0.f);
            for (int i = 0; i < n; i++) put(i, 0, R[i].P.w == 1.f ? 0.f : c0 * c0 * (R[i].V.w - c->phys.rho0));
            break;
        }
        case MFREE_S:
        case MFREE_S_T: {
            if ((st = copy_field_raw(c, f == MFREE_S ? S.sa4 : S.dsa4, A))) return st;
            if ((st = copy_field_raw(c, f == MFREE_S ? S.sb4 : S.dsb4, B))) return st;
            CUDA_TRY(cudaStreamSynchronize(c->stream));
            for (int i = 0; i < n; i++) {
                float s6[6] = {A[i].x, A[i].y, A[i].z, A[i].w, B[i].x, B[i].y};
                sym_to_9(s6, &tmp[size_t(i) * 9]);
            }
            break;
        }
        case MFREE_R: {
            std::vector<Rec> R;
            if ((st = copy_records(c, R))) return st;
            for (int i = 0; i < n; i++) {
                float s6[6] = {R[i].R.x, R[i].R.y, R[i].R.z, R[i].R.w, R[i].C.x, R[i].C.y};
                sym_to_9(s6, &tmp[size_t(i) * 9]);
            }
            break;
        }
        case MFREE_FC:
        case MFREE_FT:
        case MFREE_POS_T:
        case MFREE_VEL_T: {
            const float4 *src = f == MFREE_FC ? S.fc4 : f == MFREE_FT ? S.ft4 : f == MFREE_POS_T ? S.da4 : S.dv4;
            if ((st = copy_field_raw(c, src, A))) return st;
            CUDA_TRY(cudaStreamSynchronize(c->stream));
            for (int i = 0; i < n; i++) { put(i, 0, A[i].x); put(i, 1, A[i].y); put(i, 2, A[i].z); }
            break;
        }
        case MFREE_NRM:
        case MFREE_POS_HALF: {
            if (!c->opt.diagnostics) return fail(MFREE_ERR_ARG, "field kept only with options.diagnostics = 1");
            if ((st = copy_field_raw(c, f == MFREE_NRM ? c->scr.nrm : c->scr.pos_half, A))) return st;
            CUDA_TRY(cudaStreamSynchronize(c->stream));
            for (int i = 0; i < n; i++) {
                put(i, 0, A[i].x); put(i, 1, A[i].y); put(i, 2, A[i].z);
                if (w == 4) put(i, 3, 0.f);
            }
            break;
        }
        case MFREE_FIXED:
        case MFREE_EPS_PL_DOT:
            if ((st = copy_field_raw(c, S.dsb4, A))) return st;
            CUDA_TRY(cudaStreamSynchronize(c->stream));
            for (int i = 0; i < n; i++) put(i, 0, f == MFREE_FIXED ? A[i].w : A[i].z);
            break;
        case MFREE_BLANKED:
            if ((st = copy_field_raw(c, S.ft4, A))) return st;
            CUDA_TRY(cudaStreamSynchronize(c->stream));
            for (int i = 0; i < n; i++) put(i, 0, A[i].w);
            break;
        case MFREE_TOOL_PARTICLE:
            if ((st = copy_field_raw(c, S.fc4, A))) return st;
            CUDA_TRY(cudaStreamSynchronize(c->stream));
            for (int i = 0; i < n; i++) put(i, 0, A[i].w);
            break;
        case MFREE_EPS_PL:
        case MFREE_T:
            if ((st = copy_field_raw(c, S.sb4, A))) return st;
            CUDA_TRY(cudaStreamSynchronize(c->stream));
            for (int i = 0; i < n; i++) put(i, 0, f == MFREE_T ? A[i].z : A[i].w);
            break;
        case MFREE_RHO_T:
        case MFREE_T_T:
            if ((st = copy_field_raw(c, f == MFREE_RHO_T ? S.da4 : S.dv4, A))) return st;
            CUDA_TRY(cudaStreamSynchronize(c->stream));
            for (int i = 0; i < n; i++) put(i, 0, A[i].w);
            break;
        case MFREE_NUM_NBH:
            if (!c->opt.diagnostics) return fail(MFREE_ERR_ARG, "field kept only with options.diagnostics = 1");
            return ints(c->scr.nnb, false);
        case MFREE_IDX:
            return ints(c->scr.perm, false);
        case MFREE_HASH:
            return ints((const int *)c->scr.key_sorted, true);
        case MFREE_ID: {
            if ((st = copy_field_raw(c, S.bc4, A))) return st;
            CUDA_TRY(cudaStreamSynchronize(c->stream));
            for (int i = 0; i < n; i++) {
                int id;
                std::memcpy(&id, &A[i].w, 4);
                if (fo) std::memcpy(&fo[i], &id, 4);
                if (dout) dout[i] = double(id);
            }
            return MFREE_OK;
        }
        default:
            return fail(MFREE_ERR_ARG, "unknown field");
    }
    if (fo) std::memcpy(fo, tmp.data(), sizeof(float) * tmp.size());
    if (dout)
        for (size_t k = 0; k < tmp.size(); k++) dout[k] = double(tmp[k]);
    return MFREE_OK;
}

}  // namespace

int mfree_get_field(mfree_ctx *c, int f, void *out) {
    if (!c || !out) return fail(MFREE_ERR_ARG, "null argument");
    return get_field_impl(c, f, (float *)out, nullptr);
}
int mfree_get_field_f64(mfree_ctx *c, int f, double *out) {
    if (!c || !out) return fail(MFREE_ERR_ARG, "null argument");
    return get_field_impl(c, f, nullptr, out);
}

int mfree_set_field(mfree_ctx *c, int f, const void *in) {
    if (!c || !in) return fail(MFREE_ERR_ARG, "null argument");
    const int n = c->n_init;
    const State &S = c->st[c->cur];
    const float *v = (const float *)in;
    std::vector<float4> A, B;
    int st;
    auto rw = [&](float4 *dst, std::vector<float4> &buf, auto fn) -> int {
        if ((st = copy_field_raw(c, dst, buf))) return st;
        CUDA_TRY(cudaStreamSynchronize(c->stream));
        for (int i = 0; i < n; i++) fn(i, buf[i]);
        CUDA_TRY(cudaMemcpyAsync(dst, buf.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, c->stream));
        CUDA_TRY(cudaStreamSynchronize(c->stream));
        return MFREE_OK;
    };
    invalidate_graphs(c);
    switch (f) {
        case MFREE_POS: return rw(S.pos4, A, [&](int i, float4 &x) { x.x = v[4*i]; x.y = v[4*i+1]; x.z = v[4*i+2]; });
        case MFREE_VEL: return rw(S.vel4, A, [&](int i, float4 &x) { x.x = v[4*i]; x.y = v[4*i+1]; x.z = v[4*i+2]; });
        case MFREE_VEL_BC: return rw(S.bc4, A, [&](int i, float4 &x) { x.x = v[4*i]; x.y = v[4*i+1]; x.z = v[4*i+2]; });
        case MFREE_H: return rw(S.pos4, A, [&](int i, float4 &x) { x.w = v[i]; });
        case MFREE_RHO: return rw(S.vel4, A, [&](int i, float4 &x) { x.w = v[i]; });
        case MFREE_S:
            if ((st = rw(S.sa4, A, [&](int i, float4 &x) { x.x = v[9*i]; x.y = v[9*i+4]; x.z = v[9*i+8]; x.w = v[9*i+1]; }))) return st;
            return rw(S.sb4, B, [&](int i, float4 &x) { x.x = v[9*i+2]; x.y = v[9*i+5]; });
        case MFREE_S_T:
            if ((st = rw(S.dsa4, A, [&](int i, float4 &x) { x.x = v[9*i]; x.y = v[9*i+4]; x.z = v[9*i+8]; x.w = v[9*i+1]; }))) return st;
            return rw(S.dsb4, B, [&](int i, float4 &x) { x.x = v[9*i+2]; x.y = v[9*i+5]; });
        case MFREE_FC: return rw(S.fc4, A, [&](int i, float4 &x) { x.x = v[3*i]; x.y = v[3*i+1]; x.z = v[3*i+2]; });
        case MFREE_FT: return rw(S.ft4, A, [&](int i, float4 &x) { x.x = v[3*i]; x.y = v[3*i+1]; x.z = v[3*i+2]; });
        case MFREE_POS_T: return rw(S.da4, A, [&](int i, float4 &x) { x.x = v[3*i]; x.y = v[3*i+1]; x.z = v[3*i+2]; });
        case MFREE_VEL_T: return rw(S.dv4, A, [&](int i, float4 &x) { x.x = v[3*i]; x.y = v[3*i+1]; x.z = v[3*i+2]; });
        case MFREE_RHO_T: return rw(S.da4, A, [&](int i, float4 &x) { x.w = v[i]; });
        case MFREE_T_T: return rw(S.dv4, A, [&](int i, float4 &x) { x.w = v[i]; });
        case MFREE_FIXED: return rw(S.dsb4, A, [&](int i, float4 &x) { x.w = v[i]; });
        case MFREE_EPS_PL_DOT: return rw(S.dsb4, A, [&](int i, float4 &x) { x.z = v[i]; });
        case MFREE_BLANKED: return rw(S.ft4, A, [&](int i, float4 &x) { x.w = v[i]; });
        case MFREE_TOOL_PARTICLE: return rw(S.fc4, A, [&](int i, float4 &x) { x.w = v[i]; });
        case MFREE_EPS_PL: return rw(S.sb4, A, [&](int i, float4 &x) { x.w = v[i]; });
        case MFREE_T: return rw(S.sb4, A, [&](int i, float4 &x) { x.z = v[i]; });
        default: return fail(MFREE_ERR_ARG, "field cannot be set");
    }
}

namespace {
float4 *state_array(mfree_ctx *c, int a) {
    const State &S = c->st[c->cur];
    float4 *const arr[MFREE_NUM_ARRAYS] = {S.pos4, S.vel4, S.sa4, S.sb4, S.da4,  S.dv4,  S.dsa4,
                                           S.dsb4, S.fc4,  S.ft4, S.bc4, S.lo4, S.lo4b};
    return a >= 0 && a < MFREE_NUM_ARRAYS ? arr[a] : nullptr;
}
}  // namespace

int mfree_get_array(mfree_ctx *c, int a, float *out4) {
    if (!c || !out4) return fail(MFREE_ERR_ARG, "null argument");
    float4 *src = state_array(c, a);
    if (!src) return fail(MFREE_ERR_ARG, "mfree_get_array: unknown array");
    CUDA_TRY(cudaMemcpyAsync(out4, src, sizeof(float4) * size_t(c->n_init), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return MFREE_OK;
}
int mfree_set_array(mfree_ctx *c, int a, const float *in4) {
    if (!c || !in4) return fail(MFREE_ERR_ARG, "null argument");
    float4 *dst = state_array(c, a);
    if (!dst) return fail(MFREE_ERR_ARG, "mfree_set_array: unknown array");
    invalidate_graphs(c);
    CUDA_TRY(cudaMemcpyAsync(dst, in4, sizeof(float4) * size_t(c->n_init), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return MFREE_OK;
}
int mfree_array_device_ptr(mfree_ctx *c, int a, void **dptr) {
    if (!c || !dptr) return fail(MFREE_ERR_ARG, "null argument");
    float4 *p = state_array(c, a);
    if (!p) return fail(MFREE_ERR_ARG, "mfree_array_device_ptr: unknown array");
    *dptr = p;
    return MFREE_OK;
}

int mfree_get_cells(mfree_ctx *c, int *cs, int *ce) {
    if (!c || !cs || !ce) return fail(MFREE_ERR_ARG, "null argument");
    if (!c->grid_set || c->scratch_allocs.empty()) return fail(MFREE_ERR_ARG, "no step has run");
    std::vector<int> first(c->num_cell + 1);
    CUDA_TRY(cudaMemcpyAsync(first.data(), c->scr.first, sizeof(int) * (c->num_cell + 1), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    for (long k = 0; k < c->num_cell; k++) {
        if (first[k + 1] > first[k]) {
            cs[k] = first[k];
            ce[k] = first[k + 1];
        } else {
            cs[k] = -1;
            ce[k] = -1;
        }
    }
    return MFREE_OK;
}

int mfree_get_grid(const mfree_ctx *c, long *nx, long *ny, long *nz, float *bbmin3, float *dx) {
    if (!c || !c->grid_set) return fail(MFREE_ERR_ARG, "grid not set");
    if (nx) *nx = c->nx;
    if (ny) *ny = c->ny;
    if (nz) *nz = c->nz;
    if (bbmin3)
        for (int d = 0; d < 3; d++) bbmin3[d] = c->g_bbmin[d];
    if (dx) *dx = c->g_dx;
    return MFREE_OK;
}

void mfree_free(void *p) { free(p); }

}  // extern "C"
