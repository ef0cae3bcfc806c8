// mfree_state.cu -- checkpoint and resume of a context.
//
// The reference has no checkpoint (its nearest relatives seed positions from a
// VTK frame, vtk_reader.cpp:29-69, and temperatures from a text file,
// interp_utils.cpp:65-99).  mfree_export_state writes everything a step reads
// into one binary record: the configuration (the constant blocks, grid,
// blanking, options, time), the tools as their input meshes, the device clock
// (time, state parity, tool boxes, counters), the last recorded tool forces
// and the 13 particle-state arrays in the current sorted order.
// mfree_import_state rebuilds a context from it; the tools' triangle grids are
// rebuilt from the meshes by the same code, so stepping the imported context
// gives bitwise the results the exported one gives.
#include <climits>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "mfree_ctx.h"

using namespace mfree;
using namespace mfree::host;

namespace {

constexpr char MAGIC[8] = {'M', 'F', 'R', 'E', 'E', 'S', 'T', '1'};
constexpr uint32_t VERSION = 2;
constexpr int NSTATE = 13;

struct Header {
    char magic[8];
    uint32_t version;
    uint32_t n_init;
    uint32_t num_tools;
    uint32_t device_clock_bytes;
    uint64_t total_bytes;
};

struct Config {
    mfree_phys phys;
    mfree_corr corr;
    mfree_joco joco;
    mfree_trml twp, ttool;
    mfree_options opt;
    int32_t plastic, grid_set, blank_set, time_set, pending, cur;
    float g_bbmin[3], g_bbmax[3], g_dx, g_vel[3];
    int64_t nx, ny, nz, num_cell;
    int64_t grid_adaptive, max_cell;
    float b_min[3], b_max[3], b_vel[3], b_vmax;
    float dt, t;
    int64_t steps;
};

struct ToolRec {
    int32_t nv, nt, algorithm, pad;
    float vel[3], alpha, mu, birth, death;
};

struct Writer {
    unsigned char *p;  // NULL: only count
    size_t n = 0;
    void put(const void *src, size_t b) {
        if (p) std::memcpy(p + n, src, b);
        n += b;
    }
};

struct Reader {
    const unsigned char *p;
    size_t size, n = 0;
    bool get(void *dst, size_t b) {
        if (n + b > size) return false;
        std::memcpy(dst, p + n, b);
        n += b;
        return true;
    }
};

float4 **state_arrays(State &S, float4 **out) {
    float4 *f[NSTATE] = {S.pos4, S.vel4, S.sa4, S.sb4, S.da4, S.dv4, S.dsa4, S.dsb4, S.fc4, S.ft4, S.bc4, S.lo4, S.lo4b};
    for (int k = 0; k < NSTATE; k++) out[k] = f[k];
    return out;
}

}  // namespace

extern "C" {

int mfree_export_state(mfree_ctx *c, void *buf, size_t *size) {
    if (!c || !size) return fail(MFREE_ERR_ARG, "mfree_export_state: null argument");
    const size_t n = size_t(c->n_init);
    size_t need = sizeof(Header) + sizeof(Config) + sizeof(DevClock) + sizeof(float) * 3 * MAX_TOOLS +
                  sizeof(float4) * NSTATE * n;
    for (auto &t : c->tools) need += sizeof(ToolRec) + sizeof(float) * t->verts.size() + sizeof(int) * 3 * t->host.tris.size();
    if (!buf) {
        *size = need;
        return MFREE_OK;
    }
    if (*size < need) return fail(MFREE_ERR_ARG, "mfree_export_state: buffer too small (" + std::to_string(need) + " bytes needed)");
    Header h{};
    std::memcpy(h.magic, MAGIC, 8);
    h.version = VERSION;
    h.n_init = uint32_t(n);
    h.num_tools = uint32_t(c->tools.size());
    h.device_clock_bytes = uint32_t(sizeof(DevClock));
    h.total_bytes = need;
    Config g{};
    g.phys = c->phys;
    g.corr = c->corr;
    g.joco = c->joco;
    g.twp = c->twp;
    g.ttool = c->ttool;
    g.opt = c->opt;
    g.plastic = c->plastic;
    g.grid_set = c->grid_set;
    g.blank_set = c->blank_set;
    g.time_set = c->time_set;
    g.pending = c->pending;
    g.cur = c->cur;
    for (int d = 0; d < 3; d++) {
        g.g_bbmin[d] = c->g_bbmin[d];
        g.g_bbmax[d] = c->g_bbmax[d];
        g.g_vel[d] = c->g_vel[d];
        g.b_min[d] = c->b_min[d];
        g.b_max[d] = c->b_max[d];
        g.b_vel[d] = c->b_vel[d];
    }
    g.g_dx = c->g_dx;
    g.nx = c->nx;
    g.ny = c->ny;
    g.nz = c->nz;
    g.num_cell = c->num_cell;
    g.grid_adaptive = c->grid_adaptive ? 1 : 0;
    g.max_cell = c->max_cell;
    g.b_vmax = c->b_vmax;
    g.dt = c->dt;
    g.t = c->t;
    g.steps = c->steps;
    // the device part: clock (unless a write of the host values is pending), forces, state
    DevClock clk{};
    std::vector<float> forces(3 * MAX_TOOLS);
    std::vector<float4> st(NSTATE * n);
    float4 *arr[NSTATE];
    state_arrays(c->st[c->cur], arr);
    CUDA_TRY(cudaMemcpyAsync(&clk, c->d_clk, sizeof(DevClock), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaMemcpyAsync(forces.data(), c->d_forces, sizeof(float) * forces.size(), cudaMemcpyDeviceToHost, c->stream));
    for (int k = 0; k < NSTATE; k++)
        CUDA_TRY(cudaMemcpyAsync(st.data() + size_t(k) * n, arr[k], sizeof(float4) * n, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    const int32_t clock_dirty = c->clock_dirty;  // the host values are newer than the device clock
    Writer w{(unsigned char *)buf};
    w.put(&h, sizeof(h));
    w.put(&g, sizeof(g));
    for (auto &t : c->tools) {
        ToolRec r{};
        r.nv = int32_t(t->verts.size() / 3);
        r.nt = int32_t(t->host.tris.size());
        r.algorithm = t->algorithm;
        r.pad = 0;
        for (int d = 0; d < 3; d++) r.vel[d] = t->vel[d];
        r.alpha = t->alpha;
        r.mu = t->mu;
        r.birth = t->birth;
        r.death = t->death;
        w.put(&r, sizeof(r));
        w.put(t->verts.data(), sizeof(float) * t->verts.size());
        for (auto &tr : t->host.tris) {
            const int32_t ix[3] = {tr.i1, tr.i2, tr.i3};
            w.put(ix, sizeof(ix));
        }
    }
    clk.pending = clock_dirty ? -1 : clk.pending;  // -1: rewrite the clock from the host values on import
    w.put(&clk, sizeof(clk));
    w.put(forces.data(), sizeof(float) * forces.size());
    w.put(st.data(), sizeof(float4) * st.size());
    *size = w.n;
    return MFREE_OK;
}

int mfree_import_state(const void *buf, size_t size, void *stream, mfree_ctx **out) {
    if (!buf || !out) return fail(MFREE_ERR_ARG, "mfree_import_state: null argument");
    *out = nullptr;
    Reader r{(const unsigned char *)buf, size};
    Header h{};
    Config g{};
    if (!r.get(&h, sizeof(h)) || std::memcmp(h.magic, MAGIC, 8) != 0)
        return fail(MFREE_ERR_ARG, "mfree_import_state: not an exported state");
    if (h.version != VERSION || h.device_clock_bytes != sizeof(DevClock))
        return fail(MFREE_ERR_ARG, "mfree_import_state: exported by an incompatible version");
    if (h.total_bytes != size || h.n_init == 0) return fail(MFREE_ERR_ARG, "mfree_import_state: truncated or bad record");
    if (!r.get(&g, sizeof(g))) return fail(MFREE_ERR_ARG, "mfree_import_state: truncated record");
    if (h.n_init >= uint64_t(INT_MAX)) return fail(MFREE_ERR_ARG, "mfree_import_state: bad particle count");
    // the grid sizes the cell scratch and indexes the hash and the scans: a
    // record whose sizes disagree would make the device read and write out of
    // bounds, so it is refused
    if (g.grid_set || g.grid_adaptive) {
        // num_cell == nx * ny * nz, tested by division so that no product overflows
        const bool dims_ok = g.nx > 0 && g.ny > 0 && g.nz > 0 && g.num_cell > 0 &&
                             g.num_cell < int64_t(INT_MAX) / 2 && g.num_cell % g.nx == 0 &&
                             (g.num_cell / g.nx) % g.ny == 0 && g.num_cell / g.nx / g.ny == g.nz;
        const bool adaptive_ok = !g.grid_adaptive || (g.max_cell >= 2 && g.max_cell < int64_t(INT_MAX) / 2 &&
                                                      g.num_cell < g.max_cell);
        // an unlocked grid that has not stepped yet holds a placeholder cell edge of 0
        const bool dx_ok = std::isfinite(g.g_dx) && (g.grid_adaptive ? g.g_dx >= 0.f : g.g_dx > 0.f);
        if (!dims_ok || !adaptive_ok || !dx_ok)
            return fail(MFREE_ERR_ARG, "mfree_import_state: inconsistent grid sizes in the record");
    }
    std::unique_ptr<mfree_ctx> c;
    int st = alloc_ctx(int(h.n_init), (cudaStream_t)stream, c);
    if (st) return st;
    auto bail = [&](int code) {
        mfree_destroy(c.release());
        return code;
    };
    c->phys = g.phys;
    c->corr = g.corr;
    c->joco = g.joco;
    c->twp = g.twp;
    c->ttool = g.ttool;
    c->opt = g.opt;
    c->plastic = g.plastic != 0;
    c->grid_set = g.grid_set != 0;
    c->blank_set = g.blank_set != 0;
    for (int d = 0; d < 3; d++) {
        c->g_bbmin[d] = g.g_bbmin[d];
        c->g_bbmax[d] = g.g_bbmax[d];
        c->g_vel[d] = g.g_vel[d];
        c->b_min[d] = g.b_min[d];
        c->b_max[d] = g.b_max[d];
        c->b_vel[d] = g.b_vel[d];
    }
    c->g_dx = g.g_dx;
    c->nx = long(g.nx);
    c->ny = long(g.ny);
    c->nz = long(g.nz);
    c->num_cell = long(g.num_cell);
    c->grid_adaptive = g.grid_adaptive != 0;
    c->max_cell = long(g.max_cell);
    c->b_vmax = g.b_vmax;
    for (uint32_t k = 0; k < h.num_tools; k++) {
        ToolRec tr{};
        if (!r.get(&tr, sizeof(tr)) || tr.nv <= 0 || tr.nt <= 0) return bail(fail(MFREE_ERR_ARG, "mfree_import_state: bad tool"));
        std::vector<float> v(3 * size_t(tr.nv));
        std::vector<int> t(3 * size_t(tr.nt));
        if (!r.get(v.data(), sizeof(float) * v.size()) || !r.get(t.data(), sizeof(int) * t.size()))
            return bail(fail(MFREE_ERR_ARG, "mfree_import_state: truncated tool"));
        int idx = 0;
        if ((st = mfree_add_tool(c.get(), v.data(), tr.nv, t.data(), tr.nt, tr.vel, tr.alpha, tr.mu, tr.algorithm, &idx)))
            return bail(st);
        c->tools[idx]->birth = tr.birth;
        c->tools[idx]->death = tr.death;
    }
    // time and counters after the tools (adding a tool marks the clock for a rewrite)
    c->dt = g.dt;
    c->t = g.t;
    c->time_set = g.time_set != 0;
    c->steps = g.steps;
    c->cur = g.cur & 1;
    c->pending = g.pending != 0;
    DevClock clk{};
    std::vector<float> forces(3 * MAX_TOOLS);
    const size_t n = h.n_init;
    std::vector<float4> stv(NSTATE * n);
    if (!r.get(&clk, sizeof(clk)) || !r.get(forces.data(), sizeof(float) * forces.size()) ||
        !r.get(stv.data(), sizeof(float4) * stv.size()))
        return bail(fail(MFREE_ERR_ARG, "mfree_import_state: truncated state"));
    if (c->grid_set && (st = ensure_scratch(c.get()))) return bail(st);
    float4 *arr[NSTATE];
    state_arrays(c->st[c->cur], arr);
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < NSTATE && e == cudaSuccess; k++)
        e = cudaMemcpyAsync(arr[k], stv.data() + size_t(k) * n, sizeof(float4) * n, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(c->d_forces, forces.data(), sizeof(float) * forces.size(), cudaMemcpyHostToDevice, c->stream);
    const bool rewrite = clk.pending < 0;
    if (!rewrite && e == cudaSuccess) e = cudaMemcpyAsync(c->d_clk, &clk, sizeof(DevClock), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return bail(fail(MFREE_ERR_CUDA, std::string("mfree_import_state: ") + cudaGetErrorString(e)));
    c->clock_dirty = rewrite;
    invalidate_graphs(c.get());
    *out = c.release();
    return MFREE_OK;
}

}  // extern "C"
