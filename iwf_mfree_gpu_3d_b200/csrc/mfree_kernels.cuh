// mfree_kernels.cuh -- kernel declarations and helpers shared by the step's
// translation units.
#pragma once

#include <string>

#include "mfree_device.cuh"

namespace mfree {

constexpr int HASH_BLOCK = 256;
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;
constexpr int NRES = 20;           // reduced accumulators per particle

// half-step state x + dt/2 * xdot of the predictor (leap_frog.cu:42-70); the
// pair kernel's epilogue recomputes it with the same expressions
struct HalfStep {
    float x, y, z, vx, vy, vz, rho, T;
    float S[6];  // xx yy zz xy xz yz
};

template <bool PREC>
__device__ __forceinline__ HalfStep half_step(float h2, float4 pos, float4 vel, float4 sa, float4 sb, float4 da,
                                              float4 dv, float4 dsa, float4 dsb, float4 lo, float4 lob) {
    HalfStep o;
    if (PREC) {
        o.x = pos.x + fmaf(h2, da.x, lo.x);
        o.y = pos.y + fmaf(h2, da.y, lo.y);
        o.z = pos.z + fmaf(h2, da.z, lo.z);
        o.vx = vel.x + fmaf(h2, dv.x, lo.w);
        o.vy = vel.y + fmaf(h2, dv.y, lob.x);
        o.vz = vel.z + fmaf(h2, dv.z, lob.y);
    } else {
        o.x = fmaf(h2, da.x, pos.x);
        o.y = fmaf(h2, da.y, pos.y);
        o.z = fmaf(h2, da.z, pos.z);
        o.vx = fmaf(h2, dv.x, vel.x);
        o.vy = fmaf(h2, dv.y, vel.y);
        o.vz = fmaf(h2, dv.z, vel.z);
    }
    o.rho = fmaf(h2, da.w, vel.w);
    o.T = fmaf(h2, dv.w, sb.z);
    o.S[0] = fmaf(h2, dsa.x, sa.x);
    o.S[1] = fmaf(h2, dsa.y, sa.y);
    o.S[2] = fmaf(h2, dsa.z, sa.z);
    o.S[3] = fmaf(h2, dsa.w, sa.w);
    o.S[4] = fmaf(h2, dsb.x, sb.x);
    o.S[5] = fmaf(h2, dsb.y, sb.y);
    return o;
}

// particle inside the box of tool k at this step (the contact kernels' early
// reject, tool_3d_gpu.cu:607-614), for a tool that is set up and alive
__device__ __forceinline__ bool in_tool_box(const StepArgs &a, int k, float x, float y, float z) {
    const ToolDev &T = a.tools[k];
    if (T.num_tris == 0) return false;
    const DevClock *c = a.clk;
    if (c->t < T.birth || c->t > T.death) return false;
    const ToolClock &b = c->tool[k];
    return x > b.bbmin[0] && x < b.bbmax[0] && y > b.bbmin[1] && y < b.bbmax[1] && z > b.bbmin[2] && z < b.bbmax[2];
}
__device__ __forceinline__ bool contact_candidate(const StepArgs &a, float x, float y, float z) {
    bool in = false;
    for (int k = 0; k < a.p.num_tools; k++) in |= in_tool_box(a, k, x, y, z);
    return in;
}

// ------------------------------------------------------ batched launches --
// The step's kernels run over a table of scenes: one scene (a context's own
// one-entry table) or many independent scenes of a batch, one launch per
// kernel either way, so a scene's arithmetic is the same compiled code alone
// and in a batch.  Every scene keeps
// its own state, cell list (a segment of its own) and clock; the table lists
// each scene's arguments once per state parity and, per kernel family, the
// first block (or tile) of every scene: block b of a launch belongs to the
// scene s with prefix[s] <= b < prefix[s + 1].
struct BatchTable {
    const StepArgs *args;  // [2 s + parity]
    const int *pblk;       // particle blocks of 256 threads (hash, scatter, gather, finalize)
    const int *stile;      // scan tiles of SCAN_TILE cells
    const int *cblk;       // cell blocks of 256 threads (cell fix-up)
    const int *itile;      // pair-kernel tiles
    int nscenes;
    int *tile_next;        // work queue of the pair kernel: next entry of tile_list (reset by kb_clock)
    int *tile_count;       // entries of tile_list (reset by kb_clock)
    int2 *tile_list;       // non-empty pair-kernel tiles of every scene: (tile of the scene, scene)
};

// Pair-kernel tile = TX x TY x tile_z cells of a scene's cell grid, numbered
// z fastest, then y, then x
constexpr int TX = 4, TY = 4;
struct TileGeo {
    int X0, Y0, Z0, zl, nzr;
};
__host__ __device__ __forceinline__ TileGeo tile_geo(const Params &P, int t) {
    const int TZ = P.tile_z;
    const int nty = (P.gny + TY - 1) / TY, ntz = (P.gnz + TZ - 1) / TZ;
    const int tz = t % ntz, txy = t / ntz, ty = txy % nty, tx = txy / nty;
    TileGeo g;
    g.X0 = tx * TX;
    g.Y0 = ty * TY;
    g.Z0 = tz * TZ;
    g.zl = g.Z0 - 2 > 0 ? g.Z0 - 2 : 0;
    const int zh = g.Z0 + TZ + 1 < P.gnz - 1 ? g.Z0 + TZ + 1 : P.gnz - 1;
    g.nzr = zh - g.zl + 2;  // cell starts per halo column of the tile (inclusive end)
    return g;
}
__host__ __device__ __forceinline__ int num_tiles(const Params &P) {
    return ((P.gnx + TX - 1) / TX) * ((P.gny + TY - 1) / TY) * ((P.gnz + P.tile_z - 1) / P.tile_z);
}

// scene of block x: the last s with prefix[s] <= x (prefix has nscenes + 1 entries)
__device__ __forceinline__ int find_scene(const int *__restrict__ prefix, int nscenes, int x) {
    int lo = 0, hi = nscenes - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= x) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// scene s's arguments for the parity of its current step, read in place
// (read-only through the kernel, so the loads stay in L1 after the first warp)
__device__ __forceinline__ const StepArgs &scene_args(const BatchTable &T, int s) {
    const StepArgs *a0 = T.args + 2 * s;
    return a0[a0->clk->parity & 1];
}

// copies scene s's arguments for the parity of its current step into shared
// memory; every thread of the block calls it, a barrier must follow
__device__ __forceinline__ void load_scene_args(StepArgs &dst, const BatchTable &T, int s) {
    const StepArgs *a0 = T.args + 2 * s;
    const int4 *src = reinterpret_cast<const int4 *>(a0 + (a0->clk->parity & 1));
    int4 *d = reinterpret_cast<int4 *>(&dst);
    for (int k = threadIdx.x; k < int(sizeof(StepArgs) / 16); k += blockDim.x) d[k] = src[k];
}

__global__ void kb_clock(BatchTable T, int record_mode);
__global__ void kb_hash(BatchTable T);
__global__ void kb_scan_reduce(BatchTable T);
__global__ void kb_scan_top(BatchTable T);
__global__ void kb_scan_down(BatchTable T);
__global__ void kb_scatter(BatchTable T);
__global__ void kb_cell_fixup(BatchTable T);
cudaError_t launch_gather_predict_batch(const BatchTable &T, bool precision, int blocks, cudaStream_t s);
__global__ void kb_finalize(BatchTable T);
__global__ void kb_force_final(BatchTable T);
// one pair-kernel launch over the tiles of every scene (all scenes share the
// variant); grid <= 0 only prepares the variant
cudaError_t launch_interact_batch(const BatchTable &T, int lanes_per_particle, bool cspm, int conduction,
                                  bool precision, int grid, cudaStream_t s);

// the sort kernels on arguments passed by value, for the allocation-free
// cell-list build (mfree_static.cu)
__global__ void k_scan_reduce(StepArgs a);
__global__ void k_scan_top(StepArgs a, int num_tiles, int num_hash_blocks);
__global__ void k_scan_down(StepArgs a);
__global__ void k_scatter(StepArgs a);
__global__ void k_cell_fixup(StepArgs a);

// initial particle state from the constructor's device arrays (mfree_create)
cudaError_t launch_init_state(int n, const float4 *pos, const float4 *vel, const float *rho, const float *T,
                              const float *h, const float *fixed, const float *tool_p, const State &S, int *perm,
                              cudaStream_t s);

// message returned by mfree_last_error() (mfree_host.cu)
void set_last_error(const std::string &msg);

// sustained FP32 FMA throughput of the current device in TFLOP/s (mfree_probe.cu)
double fp32_peak_probe(int num_sms);

}  // namespace mfree
