// mfree_batch.cu -- batches of independent cutting scenes stepped together,
// the runtime under the serving loop (include/mfree.h, "batches").
//
// The reference steps one scene per process (main(), mfree_gpu_3d.cpp:75-218):
// this file has no counterpart there.  A batch owns contexts (mfree_ctx) of
// any sizes and steps all of them with one launch per kernel of the step:
//   * each scene keeps its own state, cell grid and cell list (a segment of
//     its own), clock and tools; nothing is shared between scenes;
//   * a device table lists every scene's step arguments, once per state
//     parity (the clock kernel flips a scene's parity on the device, so one
//     captured graph serves scenes admitted at different steps), and per
//     kernel family the first block of every scene;
//   * the pair kernel is persistent over the tiles of all scenes (one queue);
//   * a step of the whole batch can be captured once into a CUDA graph and
//     replayed; the graph is captured again when scenes join or leave.
// Scenes join (admit) and leave (retire, or stop at their step count) between
// steps, bounded by a device-memory budget: continuous batching.  Because
// every scene's arithmetic is the single-scene step's own code on its own
// data, a scene's results are the same alone and in a batch for the same
// pair-loop tiling.
#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "mfree_ctx.h"

using namespace mfree;
using namespace mfree::host;

namespace {

struct Slot {
    mfree_ctx *c = nullptr;
    long long done = 0, target = 0;
    int status = 2;               // 0 running, 1 done, 2 free, < 0 error status
    size_t bytes = 0;             // device memory charged to the budget
    unsigned long long built = 0; // context version the table was built from
};

}  // namespace

struct mfree_batch {
    size_t budget = 0, used = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int device = 0, num_sms = 148;
    int lpp = 8, tile_z = 6;
    bool variant_set = false, cspm = false, prec = false;
    int cond = 0;
    std::vector<Slot> slots;
    // device table: StepArgs[2 cap] | 4 prefixes of cap + 1 ints | queue counter
    void *d_table = nullptr;
    int cap = 0;
    int2 *d_tiles = nullptr;  // the pair kernel's tile list over every scene
    int tiles_cap = 0;
    BatchTable T{};
    std::vector<int> run;  // slots in the table, in table order
    int tot_pblk = 0, tot_stile = 0, tot_cblk = 0, tot_itile = 0;
    bool dirty = true;
    int table_record_every = -1;
    cudaGraphExec_t graph = nullptr;
    cudaEvent_t timer[2] = {nullptr, nullptr};
};

namespace {

size_t table_bytes(int cap) {
    return sizeof(StepArgs) * 2 * size_t(cap) + sizeof(int) * (4 * size_t(cap + 1) + 2);
}

void drop_graph(mfree_batch *b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
}

bool live(const Slot &s) { return s.c != nullptr && s.status == 0; }

// rebuild the device table for the running slots (stream-ordered upload;
// the graph is dropped, it holds the old grid sizes)
int build_table(mfree_batch *b, int record_every) {
    drop_graph(b);
    b->run.clear();
    for (int k = 0; k < int(b->slots.size()); k++)
        if (live(b->slots[k])) b->run.push_back(k);
    const int n = int(b->run.size());
    b->T.nscenes = n;
    b->table_record_every = record_every;
    b->dirty = false;
    if (n == 0) return MFREE_OK;
    if (n > b->cap) {
        CUDA_TRY(cudaStreamSynchronize(b->stream));  // the old table may still be read
        if (b->d_table) cudaFree(b->d_table);
        b->d_table = nullptr;
        const int cap = std::max(n, 2 * b->cap);
        CUDA_TRY(cudaMalloc(&b->d_table, table_bytes(cap)));
        b->cap = cap;
    }
    StepArgs *dargs = (StepArgs *)b->d_table;
    int *dint = (int *)(dargs + 2 * size_t(b->cap));
    b->T.args = dargs;
    b->T.pblk = dint;
    b->T.stile = dint + (b->cap + 1);
    b->T.cblk = dint + 2 * (b->cap + 1);
    b->T.itile = dint + 3 * (b->cap + 1);
    b->T.tile_next = dint + 4 * (b->cap + 1);
    b->T.tile_count = dint + 4 * (b->cap + 1) + 1;
    std::vector<StepArgs> args(2 * size_t(n));
    std::vector<int> pre(4 * size_t(b->cap + 1), 0);
    int *pb = pre.data(), *ps = pb + (b->cap + 1), *pc = ps + (b->cap + 1), *pt = pc + (b->cap + 1);
    for (int s = 0; s < n; s++) {
        Slot &sl = b->slots[b->run[s]];
        mfree_ctx *c = sl.c;
        int st = ready(c);
        if (st) {
            sl.status = st;
            b->dirty = true;  // build again without it on the next call
            return st;
        }
        sl.built = c->version;
        const int keep = c->cur;
        for (int p = 0; p < 2; p++) {
            c->cur = p;
            StepArgs a = make_args(c);
            a.p.record_every = record_every;
            a.p.tile_z = b->tile_z;
            args[2 * s + p] = a;
        }
        c->cur = keep;
        const Params &P = args[2 * s].p;
        pb[s + 1] = pb[s] + hash_blocks(c);
        ps[s + 1] = ps[s] + scan_tiles(c);
        pc[s + 1] = pc[s] + int((c->num_cell + 255) / 256);
        pt[s + 1] = pt[s] + num_tiles(P);
    }
    b->tot_pblk = pb[n];
    b->tot_stile = ps[n];
    b->tot_cblk = pc[n];
    b->tot_itile = pt[n];
    if (b->tot_itile > b->tiles_cap) {  // the tile list of all scenes
        CUDA_TRY(cudaStreamSynchronize(b->stream));  // the old list may still be read
        const int cap = std::max(b->tot_itile, 2 * b->tiles_cap);
        if (b->d_tiles) cudaFree(b->d_tiles);
        b->d_tiles = nullptr;
        b->tiles_cap = 0;
        CUDA_TRY(cudaMalloc(&b->d_tiles, sizeof(int2) * size_t(cap)));
        b->tiles_cap = cap;
    }
    b->T.tile_list = b->d_tiles;
    // pageable sources: the call returns once the bytes are staged, so the
    // vectors may go; the device copy stays ordered on the stream
    CUDA_TRY(cudaMemcpyAsync(dargs, args.data(), sizeof(StepArgs) * args.size(), cudaMemcpyHostToDevice, b->stream));
    CUDA_TRY(cudaMemcpyAsync(dint, pre.data(), sizeof(int) * pre.size(), cudaMemcpyHostToDevice, b->stream));
    cudaError_t e = launch_interact_batch(b->T, b->lpp, b->cspm, b->cond, b->prec, 0, b->stream);
    if (e != cudaSuccess) return fail(MFREE_ERR_CUDA, std::string("batched pair kernel setup: ") + cudaGetErrorString(e));
    return MFREE_OK;
}

// the kernels of one batch step (record_mode as kb_clock; 2 = every
// Params::record_every steps of each scene's own step index)
int enqueue_batch_step(mfree_batch *b, int record_mode) {
    const TraceRange range("mfree_batch_step");
    const BatchTable &T = b->T;
    cudaStream_t s = b->stream;
    const int n = T.nscenes;
    kb_clock<<<(n + 127) / 128, 128, 0, s>>>(T, record_mode);
    kb_hash<<<b->tot_pblk, HASH_BLOCK, 0, s>>>(T);
    kb_scan_reduce<<<b->tot_stile, SCAN_THREADS, 0, s>>>(T);
    kb_scan_top<<<n, 1024, 0, s>>>(T);
    kb_scan_down<<<b->tot_stile, SCAN_THREADS, 0, s>>>(T);
    kb_scatter<<<b->tot_pblk, HASH_BLOCK, 0, s>>>(T);
    kb_cell_fixup<<<b->tot_cblk + (b->tot_itile + 255) / 256, 256, 0, s>>>(T);
    cudaError_t e = launch_gather_predict_batch(T, b->prec, b->tot_pblk, s);
    if (e == cudaSuccess) e = launch_interact_batch(T, b->lpp, b->cspm, b->cond, b->prec, b->num_sms, s);
    if (e != cudaSuccess) return fail(MFREE_ERR_CUDA, std::string("batched step launch: ") + cudaGetErrorString(e));
    kb_finalize<<<b->tot_pblk, 256, 0, s>>>(T);
    kb_force_final<<<n, 256, 0, s>>>(T);
    CUDA_TRY(cudaGetLastError());
    return MFREE_OK;
}

int capture(mfree_batch *b) {
    cudaGraph_t g = nullptr;
    CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int e = enqueue_batch_step(b, 2);
    cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
    if (e) {
        if (g) cudaGraphDestroy(g);
        return e;
    }
    if (ce != cudaSuccess) return fail(MFREE_ERR_CUDA, std::string("batch graph capture: ") + cudaGetErrorString(ce));
    cudaError_t ie = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) return fail(MFREE_ERR_CUDA, std::string("batch graph instantiate: ") + cudaGetErrorString(ie));
    return MFREE_OK;
}

// host mirror of one step of a context (as mfree_advance keeps it)
void advance_host(mfree_ctx *c) {
    c->cur ^= 1;
    if (c->pending) c->t = c->t + c->dt;
    c->pending = true;
    c->steps++;
}

// lagged all-blanked check of every running scene: a scene whose last step
// left no particle stops with MFREE_ERR_EMPTY
void poll_empty(mfree_batch *b, bool wait) {
    for (auto &sl : b->slots) {
        if (!live(sl)) continue;
        int st = check_empty(sl.c, wait);
        if (st) {
            sl.status = st;
            b->dirty = true;
        }
    }
}

int bad_slot(mfree_batch *b, int slot) {
    return !b || slot < 0 || slot >= int(b->slots.size()) || b->slots[slot].c == nullptr;
}

}  // namespace

extern "C" {

int mfree_batch_create(size_t hbm_budget, void *stream, mfree_batch **out) {
    if (!out) return fail(MFREE_ERR_ARG, "mfree_batch_create: null output");
    *out = nullptr;
    auto b = std::make_unique<mfree_batch>();
    b->budget = hbm_budget;
    CUDA_TRY(cudaGetDevice(&b->device));
    CUDA_TRY(cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, b->device));
    b->stream = (cudaStream_t)stream;
    if (!b->stream) {
        CUDA_TRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        b->own_stream = true;
    }
    b->lpp = default_lpp();
    b->tile_z = default_tile_depth();
    *out = b.release();
    return MFREE_OK;
}

int mfree_batch_destroy(mfree_batch *b) {
    if (!b) return MFREE_OK;
    cudaStreamSynchronize(b->stream);
    drop_graph(b);
    for (auto &sl : b->slots)
        if (sl.c) {
            sl.c->owner = nullptr;
            sl.c->stream = sl.c->home_stream;
            mfree_destroy(sl.c);
        }
    if (b->d_table) cudaFree(b->d_table);
    if (b->d_tiles) cudaFree(b->d_tiles);
    for (auto e : b->timer)
        if (e) cudaEventDestroy(e);
    if (b->own_stream) cudaStreamDestroy(b->stream);
    delete b;
    return MFREE_OK;
}

int mfree_batch_admit(mfree_batch *b, mfree_ctx *c, long long steps, int *slot) {
    if (!b || !c) return fail(MFREE_ERR_ARG, "mfree_batch_admit: null argument");
    if (c->owner) return fail(MFREE_ERR_ARG, "mfree_batch_admit: the context already belongs to a batch");
    if (c->grid_adaptive) return fail(MFREE_ERR_ARG, "mfree_batch_admit: a context with an unlocked grid steps alone");
    if (c->device != b->device) return fail(MFREE_ERR_ARG, "mfree_batch_admit: the context is on another device");
    int st = ready(c);
    if (st) return st;
    const bool cspm = c->opt.cspm != 0, prec = c->opt.precision != 0;
    const int cond = c->opt.conduction;
    bool held = false;
    for (auto &sl : b->slots) held |= sl.c != nullptr;
    if (held && b->variant_set && (cspm != b->cspm || prec != b->prec || cond != b->cond))
        return fail(MFREE_ERR_ARG, "mfree_batch_admit: the scene's cspm/conduction/precision options differ from the batch's");
    const size_t bytes = device_bytes(c);
    if (b->budget && b->used + bytes > b->budget)
        return fail(MFREE_ERR_BUDGET, "mfree_batch_admit: " + std::to_string(bytes) + " bytes do not fit the budget (" +
                                          std::to_string(b->budget - b->used) + " left)");
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    b->variant_set = true;
    b->cspm = cspm;
    b->prec = prec;
    b->cond = cond;
    c->home_stream = c->stream;
    c->stream = b->stream;
    c->owner = b;
    invalidate_graphs(c);  // its own graphs ran on its own stream
    int k = 0;
    while (k < int(b->slots.size()) && b->slots[k].c) k++;
    if (k == int(b->slots.size())) b->slots.emplace_back();
    Slot &sl = b->slots[k];
    sl = Slot{};
    sl.c = c;
    sl.target = steps;
    sl.status = 0;
    sl.bytes = bytes;
    b->used += bytes;
    b->dirty = true;
    if (slot) *slot = k;
    return MFREE_OK;
}

int mfree_batch_step(mfree_batch *b, int nsteps, int record_every, int use_graph) {
    if (!b || nsteps < 0) return fail(MFREE_ERR_ARG, "mfree_batch_step: bad arguments");
    int left = nsteps;
    while (left > 0) {
        poll_empty(b, false);
        for (auto &sl : b->slots)
            if (live(sl) && sl.c->version != sl.built) b->dirty = true;  // a setter changed the scene
        if (b->dirty || b->table_record_every != record_every) {
            int st = build_table(b, record_every);
            if (st) return st;
        }
        if (b->T.nscenes == 0) break;
        int chunk = left;
        for (int k : b->run) {
            const Slot &sl = b->slots[k];
            if (sl.target > 0) chunk = int(std::min<long long>(chunk, sl.target - sl.done));
        }
        if (use_graph) {
            if (!b->graph) {
                int st = capture(b);
                if (st) return st;
            }
            for (int i = 0; i < chunk; i++) CUDA_TRY(cudaGraphLaunch(b->graph, b->stream));
        } else {
            for (int i = 0; i < chunk; i++) {
                int st = enqueue_batch_step(b, 2);
                if (st) return st;
            }
        }
        for (int k : b->run) {
            Slot &sl = b->slots[k];
            for (int i = 0; i < chunk; i++) advance_host(sl.c);
            sl.done += chunk;
            int st = note_active_count(sl.c);
            if (st) return st;
            if (sl.target > 0 && sl.done >= sl.target) {
                sl.status = 1;
                b->dirty = true;
            }
        }
        left -= chunk;
    }
    return MFREE_OK;
}

int mfree_batch_query(mfree_batch *b, int slot, long long *done, long long *target, int *status) {
    if (!b || slot < 0 || slot >= int(b->slots.size())) return fail(MFREE_ERR_ARG, "mfree_batch_query: bad slot");
    const Slot &sl = b->slots[slot];
    if (sl.c && sl.status == 0) poll_empty(b, false);
    if (done) *done = sl.done;
    if (target) *target = sl.target;
    if (status) *status = sl.c ? sl.status : 2;
    return MFREE_OK;
}

int mfree_batch_context(mfree_batch *b, int slot, mfree_ctx **ctx) {
    if (bad_slot(b, slot) || !ctx) return fail(MFREE_ERR_ARG, "mfree_batch_context: bad slot");
    *ctx = b->slots[slot].c;
    return MFREE_OK;
}

int mfree_batch_retire(mfree_batch *b, int slot, mfree_ctx **ctx) {
    if (bad_slot(b, slot)) return fail(MFREE_ERR_ARG, "mfree_batch_retire: bad slot");
    Slot &sl = b->slots[slot];
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    mfree_ctx *c = sl.c;
    c->owner = nullptr;
    c->stream = c->home_stream;
    invalidate_graphs(c);
    b->used -= sl.bytes;
    if (sl.status == 0) b->dirty = true;
    sl = Slot{};
    if (ctx) {
        *ctx = c;
        return MFREE_OK;
    }
    return mfree_destroy(c);
}

int mfree_batch_info(mfree_batch *b, int *scenes, int *running, size_t *bytes, size_t *budget) {
    if (!b) return fail(MFREE_ERR_ARG, "mfree_batch_info: null batch");
    int n = 0, r = 0;
    for (auto &sl : b->slots) {
        n += sl.c != nullptr;
        r += live(sl);
    }
    if (scenes) *scenes = n;
    if (running) *running = r;
    if (bytes) *bytes = b->used;
    if (budget) *budget = b->budget;
    return MFREE_OK;
}

int mfree_batch_set_tiling(mfree_batch *b, int lpp, int tile_depth) {
    if (!b) return fail(MFREE_ERR_ARG, "mfree_batch_set_tiling: null batch");
    if (lpp != 0 && lpp != 8 && lpp != 16 && lpp != 32)
        return fail(MFREE_ERR_ARG, "lanes_per_particle must be 0, 8, 16 or 32");
    if (tile_depth < 0 || tile_depth > TILE_Z_MAX) return fail(MFREE_ERR_ARG, "tile_depth must be 0..8");
    if (lpp) b->lpp = lpp;
    if (tile_depth) b->tile_z = tile_depth;
    b->dirty = true;
    return MFREE_OK;
}

int mfree_batch_get_tiling(mfree_batch *b, int *lpp, int *tile_depth) {
    if (!b) return fail(MFREE_ERR_ARG, "mfree_batch_get_tiling: null batch");
    if (lpp) *lpp = b->lpp;
    if (tile_depth) *tile_depth = b->tile_z;
    return MFREE_OK;
}

int mfree_batch_autotune(mfree_batch *b, int trial_steps, int *lpp_out, int *tz_out, double *ms_best) {
    if (!b || trial_steps <= 0) return fail(MFREE_ERR_ARG, "mfree_batch_autotune: bad arguments");
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    // copies of the running scenes in a batch of their own, on this stream
    mfree_batch *tb = nullptr;
    int st = mfree_batch_create(0, b->stream, &tb);
    if (st) return st;
    std::unique_ptr<mfree_batch, int (*)(mfree_batch *)> hold(tb, mfree_batch_destroy);
    for (auto &sl : b->slots) {
        if (!live(sl)) continue;
        std::unique_ptr<mfree_ctx> cl;
        if ((st = clone_ctx(sl.c, b->stream, cl))) return st;
        cl->home_stream = b->stream;
        mfree_ctx *raw = cl.release();
        raw->stream = b->stream;
        if ((st = mfree_batch_admit(tb, raw, 0, nullptr))) {
            mfree_destroy(raw);
            return st;
        }
    }
    int nrun = 0;
    mfree_batch_info(tb, nullptr, &nrun, nullptr, nullptr);
    if (nrun == 0) return fail(MFREE_ERR_ARG, "mfree_batch_autotune: no running scene to time");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    double best = 1e300;
    int blpp = b->lpp, btz = b->tile_z;
    const int lpps[] = {8, 16, 32};
    for (int lpp : lpps)
        for (int tz = 4; tz <= TILE_Z_MAX && !st; tz++) {
            if ((st = mfree_batch_set_tiling(tb, lpp, tz))) break;
            if ((st = mfree_batch_step(tb, 1, 0, 1))) break;  // capture + warm-up
            cudaEventRecord(e0, b->stream);
            if ((st = mfree_batch_step(tb, trial_steps, 0, 1))) break;
            cudaEventRecord(e1, b->stream);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) {
                best = ms;
                blpp = lpp;
                btz = tz;
            }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    b->lpp = blpp;
    b->tile_z = btz;
    b->dirty = true;
    if (lpp_out) *lpp_out = blpp;
    if (tz_out) *tz_out = btz;
    if (ms_best) *ms_best = best / trial_steps;
    return MFREE_OK;
}

int mfree_batch_sync(mfree_batch *b) {
    if (!b) return fail(MFREE_ERR_ARG, "mfree_batch_sync: null batch");
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    return MFREE_OK;
}

int mfree_batch_timer_start(mfree_batch *b) {
    if (!b) return fail(MFREE_ERR_ARG, "mfree_batch_timer_start: null batch");
    for (auto &e : b->timer)
        if (!e) CUDA_TRY(cudaEventCreate(&e));
    CUDA_TRY(cudaEventRecord(b->timer[0], b->stream));
    return MFREE_OK;
}

int mfree_batch_timer_stop(mfree_batch *b, double *ms) {
    if (!b || !ms || !b->timer[0]) return fail(MFREE_ERR_ARG, "mfree_batch_timer_stop: no timer started");
    CUDA_TRY(cudaEventRecord(b->timer[1], b->stream));
    CUDA_TRY(cudaEventSynchronize(b->timer[1]));
    float f = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&f, b->timer[0], b->timer[1]));
    *ms = f;
    return MFREE_OK;
}

int mfree_device_bytes(const mfree_ctx *c, size_t *bytes) {
    if (!c || !bytes) return fail(MFREE_ERR_ARG, "mfree_device_bytes: null argument");
    *bytes = device_bytes(c);
    return MFREE_OK;
}

size_t mfree_scene_bytes(int n, long long num_cell) { return scene_bytes(n, num_cell); }

}  // extern "C"
