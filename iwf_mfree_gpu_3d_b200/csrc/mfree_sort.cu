// mfree_sort.cu -- start of the step: clock, blanking + cell hash, stable
// counting sort by cell, and the gather that fuses the reorder with the
// predictor, the equation of state and the artificial stress.
//
// Reference path replaced (src/leap_frog.cu:133-151):
//   blanking::update + do_blanking          actions_gpu.cu:489-531, blanking.cpp:43-51
//   grid_base::update_geometry (locked)     grid_gpu_base.cu:166-183
//   compute_hashes                          grid_gpu_base.cu:41-63
//   adapt_particle_number (thrust::count)   grid_gpu_base.cu:141-164
//   do_sort: sequence + stable sort_by_key, cell range build, reorder_data
//                                           grid_gpu_green.cu:24-125,265-297
//   init, predict                           leap_frog.cu:30-70
//   do_material_eos, do_corrector_artificial_stress  actions_gpu.cu:40-132
//
// The sort is a stable counting sort: an atomic histogram of cell ids, an
// exclusive scan (which is also the cell-range table the pair loop reads),
// an atomic scatter and a per-cell fix-up that orders each cell's entries by
// their previous index.  The result equals thrust's stable sort_by_key of
// (cell id, 0..n-1): cells ascending, previous order inside a cell, blanked
// particles (cell id INT_MAX in the reference) last in previous order.
// N stays on the device: no host round trip per step.
#include "mfree_kernels.cuh"

namespace mfree {

// ----------------------------------------------------------------- clock --
// batched kernels: block b of the launch is block b - prefix[s] of scene s,
// whose arguments the block reads in place (a copy into shared memory, one
// barrier per block, cost these short blocks more than it saved)
template <class F> __device__ __forceinline__ void run_batched(const BatchTable &T, const int *prefix, F &&body) {
    const int s = find_scene(prefix, T.nscenes, blockIdx.x);
    body(scene_args(T, s), int(blockIdx.x) - prefix[s]);
}

// record_mode: 0 no, 1 yes, 2 every Params::record_every steps
__device__ __forceinline__ void clock_body(const StepArgs &a, int record_mode) {
    DevClock *c = a.clk;
    const Params &P = a.p;
    if (c->pending) {
        c->t = c->t + P.dt;  // main(): global_time_current += dt after each iteration
        c->parity ^= 1;      // the last step's output is this step's input
    }
    c->pending = 1;
    c->max_disp = 0u;
    const float t = c->t;
    c->record = record_mode == 1 ? 1
                : record_mode == 2 ? (P.record_every > 0 && (c->step_index % P.record_every) == 0)
                                   : 0;
    c->step_index++;
    if (P.blank_on)
        for (int d = 0; d < 3; d++) {
            c->blank_min[d] = P.blank_min0[d] + t * P.blank_vel[d];
            c->blank_max[d] = P.blank_max0[d] + t * P.blank_vel[d];
        }
    if (P.grid_moving)
        for (int d = 0; d < 3; d++) c->grid_min[d] = P.grid_min0[d] + t * P.grid_vel[d];
    for (int k = 0; k < P.num_tools; k++) {
        if (a.tools[k].num_tris == 0) continue;  // update_tool returns early without boxed triangles
        for (int d = 0; d < 3; d++) {
            c->tool[k].bbmin[d] += P.dt * a.tools[k].vel[d];
            c->tool[k].bbmax[d] += P.dt * a.tools[k].vel[d];
        }
    }
}

// one thread per scene; thread 0 also resets the batch's pair-kernel queue
__global__ void kb_clock(BatchTable T, int record_mode) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s == 0) {
        *T.tile_next = 0;
        *T.tile_count = 0;
    }
    if (s < T.nscenes) clock_body(T.args[2 * s], record_mode);
}

// ------------------------------------------------- blanking + cell hash --
__device__ __forceinline__ void hash_body(const StepArgs &a, int bid) {
    const Params &P = a.p;
    const int i = bid * HASH_BLOCK + threadIdx.x;
    int blank = 0;
    unsigned counted = 0xffffffffu;  // the cell this particle is counted in (none: all ones)
    if (i < P.n_init) {
        float4 p = a.a.pos4[i];
        float4 ft = a.a.ft4[i];
        float blanked = ft.w;
        if (P.blank_on) {
            float4 v = a.a.vel4[i];
            const DevClock *c = a.clk;
            bool fast = __fadd_rn(__fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y)), __fmul_rn(v.z, v.z)) >= P.vmax2;
            bool in = p.x >= c->blank_min[0] && p.x <= c->blank_max[0] && p.y >= c->blank_min[1] &&
                      p.y <= c->blank_max[1] && p.z >= c->blank_min[2] && p.z <= c->blank_max[2];
            if (fast || !in) {
                blanked = 1.f;
            } else if (blanked != 0.f) {
                // inside and slow: the reference unblanks unless a rate is NaN/Inf
                // (actions_gpu.cu:504-529), and a particle that is not blanked
                // stays so either way -- the rates are read only to unblank
                float4 da = a.a.da4[i], dv = a.a.dv4[i], dsa = a.a.dsa4[i], dsb = a.a.dsb4[i];
                bool bad = nan_or_inf(da.x) || nan_or_inf(da.y) || nan_or_inf(da.z) || nan_or_inf(dv.x) ||
                           nan_or_inf(dv.y) || nan_or_inf(dv.z) || nan_or_inf(dsa.x) || nan_or_inf(dsa.y) ||
                           nan_or_inf(dsa.z) || nan_or_inf(dsa.w) || nan_or_inf(dsb.y) || nan_or_inf(dsb.x) ||
                           nan_or_inf(da.w) || nan_or_inf(dv.w);
                if (!bad) blanked = 0.f;
            }
            if (blanked == 1.f) {  // count blanked particles carrying a NaN/Inf position or rate
                float4 da = a.a.da4[i], dv = a.a.dv4[i], dsa = a.a.dsa4[i], dsb = a.a.dsb4[i];
                bool bad = nan_or_inf(p.x) || nan_or_inf(p.y) || nan_or_inf(p.z) || nan_or_inf(da.x) ||
                           nan_or_inf(da.y) || nan_or_inf(da.z) || nan_or_inf(dv.x) || nan_or_inf(dv.y) ||
                           nan_or_inf(dv.z) || nan_or_inf(dsa.x) || nan_or_inf(dsa.y) || nan_or_inf(dsa.z) ||
                           nan_or_inf(dsa.w) || nan_or_inf(dsb.x) || nan_or_inf(dsb.y) || nan_or_inf(da.w) ||
                           nan_or_inf(dv.w);
                if (bad) atomicAdd(&a.clk->nan_blanked, 1ull);
            }
        }
        unsigned key = unsigned(P.num_cell);
        if (blanked != 1.f) {
            const float *gmin = P.grid_moving ? a.clk->grid_min : P.grid_min0;
            int ix = int(__fdiv_rn(__fsub_rn(p.x, gmin[0]), P.gdx));
            int iy = int(__fdiv_rn(__fsub_rn(p.y, gmin[1]), P.gdx));
            int iz = int(__fdiv_rn(__fsub_rn(p.z, gmin[2]), P.gdx));
            if (ix >= 0 && ix < P.gnx && iy >= 0 && iy < P.gny && iz >= 0 && iz < P.gnz) {
                key = unsigned((ix * P.gny + iy) * P.gnz + iz);
            } else {
                blanked = 1.f;  // outside the cell grid but not blanked: taken out (counted)
                atomicAdd(&a.clk->out_of_grid, 1ull);
            }
        }
        if (blanked != ft.w) {
            ft.w = blanked;
            a.a.ft4[i] = ft;
        }
        a.s.key[i] = key;
        if (key < unsigned(P.num_cell)) counted = key;
        else blank = 1;
    }
    // the cell counts: particles come in last step's sorted order, so a
    // warp's keys run in stretches of one cell; the first lane of each
    // stretch adds its length (about 14 atomics a warp instead of 32)
    {
        const int lane = threadIdx.x & 31;
        const unsigned prev = __shfl_up_sync(0xffffffffu, counted, 1);
        const bool start = lane == 0 || prev != counted;
        const unsigned starts = __ballot_sync(0xffffffffu, start);
        if (start && counted != 0xffffffffu) {
            const unsigned after = starts & ~((2u << lane) - 1u);
            const int end = after ? __ffs(after) - 1 : 32;
            atomicAdd(&a.s.count[counted], end - lane);
        }
    }
    int nb = __syncthreads_count(blank);
    if (threadIdx.x == 0) a.s.blank_block[bid] = nb;
}
__global__ void __launch_bounds__(HASH_BLOCK) kb_hash(BatchTable T) {
    run_batched(T, T.pblk, [](const StepArgs &a, int b) { hash_body(a, b); });
}

// ------------------------------------------------------------- the scan --
// exclusive scan of count[0..num_cell) into first[0..num_cell]; first[num_cell] = N
__device__ __forceinline__ int block_exclusive_scan(int v, int *warp_sums, int &total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < (blockDim.x >> 5) ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        warp_sums[lane] = w;  // inclusive
    }
    __syncthreads();
    int pre = warp > 0 ? warp_sums[warp - 1] : 0;
    total = warp_sums[(blockDim.x >> 5) - 1];
    __syncthreads();
    return pre + x - v;
}

__device__ __forceinline__ void scan_reduce_body(const StepArgs &a, int bid) {
    __shared__ int ws[32];
    const int nc = a.p.num_cell;
    const int base = bid * SCAN_TILE;
    int s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        int c = base + threadIdx.x + k * SCAN_THREADS;
        if (c < nc) s += a.s.count[c];
    }
    int total;
    block_exclusive_scan(s, ws, total);
    if (threadIdx.x == 0) a.s.tile_sum[bid] = total;
}
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_reduce(StepArgs a) { scan_reduce_body(a, blockIdx.x); }
__global__ void __launch_bounds__(SCAN_THREADS) kb_scan_reduce(BatchTable T) {
    run_batched(T, T.stile, [](const StepArgs &a, int b) { scan_reduce_body(a, b); });
}

// one block: exclusive scans of the tile sums and of the blanked-per-block counts
__device__ __forceinline__ void scan_top_body(const StepArgs &a, int num_tiles, int num_hash_blocks) {
    __shared__ int ws[32];
    __shared__ int carry;
    for (int pass = 0; pass < 2; pass++) {
        int *arr = pass == 0 ? a.s.tile_sum : a.s.blank_block;
        const int n = pass == 0 ? num_tiles : num_hash_blocks;
        if (threadIdx.x == 0) carry = 0;
        __syncthreads();
        for (int b0 = 0; b0 < n; b0 += 1024) {
            int idx = b0 + threadIdx.x;
            int v = idx < n ? arr[idx] : 0;
            int total;
            int ex = block_exclusive_scan(v, ws, total);
            int c0 = carry;
            if (idx < n) arr[idx] = c0 + ex;
            __syncthreads();
            if (threadIdx.x == 0) carry = c0 + total;
            __syncthreads();
        }
        if (pass == 0 && threadIdx.x == 0) a.clk->n_active = carry;
        __syncthreads();
    }
}
__global__ void __launch_bounds__(1024) k_scan_top(StepArgs a, int num_tiles, int num_hash_blocks) {
    scan_top_body(a, num_tiles, num_hash_blocks);
}
// one block per scene
__global__ void __launch_bounds__(1024) kb_scan_top(BatchTable T) {
    __shared__ StepArgs sa;
    load_scene_args(sa, T, blockIdx.x);
    __syncthreads();
    const int tiles = (sa.p.num_cell + 1 + SCAN_TILE - 1) / SCAN_TILE;
    const int hb = (sa.p.n_init + HASH_BLOCK - 1) / HASH_BLOCK;
    scan_top_body(sa, tiles, hb);
}

__device__ __forceinline__ void scan_down_body(const StepArgs &a, int bid) {
    __shared__ int ws[32];
    const int nc = a.p.num_cell;
    const int base = bid * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    int s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        int c = base + k;
        v[k] = c < nc ? a.s.count[c] : 0;
        s += v[k];
    }
    int total;
    int ex = block_exclusive_scan(s, ws, total) + a.s.tile_sum[bid];
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        int c = base + k;
        if (c <= nc) a.s.first[c] = ex;  // first[nc] = N
        ex += v[k];
    }
}
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_down(StepArgs a) { scan_down_body(a, blockIdx.x); }
__global__ void __launch_bounds__(SCAN_THREADS) kb_scan_down(BatchTable T) {
    run_batched(T, T.stile, [](const StepArgs &a, int b) { scan_down_body(a, b); });
}

// ---------------------------------------------------------- the scatter --
__device__ __forceinline__ void scatter_body(const StepArgs &a, int bid) {
    __shared__ int ws[32];
    const Params &P = a.p;
    const int i = bid * HASH_BLOCK + threadIdx.x;
    const int N = a.clk->n_active;
    unsigned key = i < P.n_init ? a.s.key[i] : 0u;
    int blank = (i < P.n_init && key >= unsigned(P.num_cell)) ? 1 : 0;
    int total;
    int rank = block_exclusive_scan(blank, ws, total);
    // one atomic per stretch of equal keys in the warp (the hash kernel's
    // stretches): its first lane takes the stretch's length off the cell's
    // count (which leaves count[] zero for the next step) and the stretch
    // fills its slots in lane order, so it arrives in increasing index order
    // and the per-cell fix-up below has little to move
    const int lane = threadIdx.x & 31;
    const unsigned counted = (i < P.n_init && !blank) ? key : 0xffffffffu;
    const unsigned prev = __shfl_up_sync(0xffffffffu, counted, 1);
    const bool start = lane == 0 || prev != counted;
    const unsigned starts = __ballot_sync(0xffffffffu, start);
    const unsigned upto = starts & ((2u << lane) - 1u);  // starts at or below this lane
    const int head = 31 - __clz(upto);
    const unsigned after = starts & ~((2u << lane) - 1u);
    const int end = after ? __ffs(after) - 1 : 32;
    int old = 0;
    if (start && counted != 0xffffffffu) old = atomicSub(&a.s.count[counted], end - lane);
    old = __shfl_sync(0xffffffffu, old, head);
    if (i >= P.n_init) return;
    if (!blank) {
        const int d = a.s.first[key] + old - (end - head) + (lane - head);
        if (bounds_ok(a.clk, d, P.n_init)) a.s.perm[d] = i;
    } else {
        const int d = N + a.s.blank_block[bid] + rank;
        if (bounds_ok(a.clk, d, P.n_init)) a.s.perm[d] = i;
    }
}
__global__ void __launch_bounds__(HASH_BLOCK) k_scatter(StepArgs a) { scatter_body(a, blockIdx.x); }
__global__ void __launch_bounds__(HASH_BLOCK) kb_scatter(BatchTable T) {
    run_batched(T, T.pblk, [](const StepArgs &a, int b) { scatter_body(a, b); });
}

// order each cell's entries by previous index (stable within the cell)
__device__ __forceinline__ void cell_fixup_body(const StepArgs &a, int bid) {
    const int c = bid * 256 + threadIdx.x;
    if (c >= a.p.num_cell) return;
    const int s = a.s.first[c], e = a.s.first[c + 1];
    if (e - s < 2) return;
    if (!bounds_ok(a.clk, s, a.p.n_init) || !bounds_ok(a.clk, e - 1, a.p.n_init)) return;
    int *p = a.s.perm;
    for (int k = s + 1; k < e; k++) {
        int v = p[k];
        int m = k - 1;
        while (m >= s && p[m] > v) {
            p[m + 1] = p[m];
            m--;
        }
        p[m + 1] = v;
    }
}
__global__ void __launch_bounds__(256) k_cell_fixup(StepArgs a) { cell_fixup_body(a, blockIdx.x); }

// The pair kernel's list of non-empty tiles: one thread per tile of every
// scene; a tile with a particle in one of its target cells is appended as
// (tile of its scene, scene), one atomic per warp.  The order of the list
// changes which block runs a tile, never a result.
__device__ __forceinline__ void tile_list_body(const BatchTable &T, int g) {
    const int total = T.itile[T.nscenes];
    bool ne = false;
    int s = 0, t = 0;
    if (g < total) {
        s = find_scene(T.itile, T.nscenes, g);
        t = g - T.itile[s];
        const StepArgs *a0 = T.args + 2 * s;
        const StepArgs &a = a0[a0->clk->parity & 1];
        const Params &P = a.p;
        const int nx = P.gnx, ny = P.gny, nz = P.gnz;
        const TileGeo G = tile_geo(P, t);
        const int zend = min(G.Z0 + P.tile_z - 1, nz - 1) + 1;
        const int *__restrict__ first = a.s.first;
        for (int c = 0; c < TX * TY; c++) {
            const int cx = G.X0 + c / TY, cy = G.Y0 + c % TY;
            if (cx < nx && cy < ny && G.Z0 < nz) {
                const int cb = (cx * ny + cy) * nz;
                ne |= first[cb + zend] > first[cb + G.Z0];
            }
        }
    }
    const unsigned m = __ballot_sync(0xffffffffu, ne);
    if (m == 0) return;
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(T.tile_count, __popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (ne) T.tile_list[base + __popc(m & ((1u << lane) - 1u))] = make_int2(t, s);
}

// blocks past the cell blocks of every scene build the tile list (the cell
// starts are final once the scatter has run)
__global__ void __launch_bounds__(256) kb_cell_fixup(BatchTable T) {
    const int nb = T.cblk[T.nscenes];
    if (int(blockIdx.x) >= nb) {
        tile_list_body(T, (int(blockIdx.x) - nb) * 256 + int(threadIdx.x));
        return;
    }
    run_batched(T, T.cblk, [](const StepArgs &a, int b) { cell_fixup_body(a, b); });
}

// --------------------------------------------- gather + predictor + EOS --
template <bool PREC> __device__ __forceinline__ void gather_predict_body(const StepArgs &a, int bid) {
    const Params &P = a.p;
    const int i = bid * 256 + threadIdx.x;
    if (i >= P.n_init) return;
    const int N = a.clk->n_active;
    int src = a.s.perm[i];
    if (src < 0 || src >= P.n_init) {  // cannot happen for a consistent sort; never read out of bounds
        atomicAdd(&a.clk->out_of_grid, 1ull << 32);
        src = i;
    }
    const State &A = a.a, &B = a.b;
    float4 pos = A.pos4[src], vel = A.vel4[src], sa = A.sa4[src], sb = A.sb4[src];
    float4 da = A.da4[src], dv = A.dv4[src], dsa = A.dsa4[src], dsb = A.dsb4[src];
    float4 fc = A.fc4[src], ft = A.ft4[src], bc = A.bc4[src];
    B.pos4[i] = pos; B.vel4[i] = vel; B.sa4[i] = sa; B.sb4[i] = sb;
    B.da4[i] = da; B.dv4[i] = dv; B.dsa4[i] = dsa; B.dsb4[i] = dsb;
    B.fc4[i] = fc; B.ft4[i] = ft; B.bc4[i] = bc;
    float4 lo = make_float4(0.f, 0.f, 0.f, 0.f), lob = lo;
    if (PREC) {
        lo = A.lo4[src];
        lob = A.lo4b[src];
        B.lo4[i] = lo;
        B.lo4b[i] = lob;
    }
    a.s.key_sorted[i] = a.s.key[src];
    if (i >= N) return;  // blanked: frozen
    const float h2 = 0.5f * P.dt;
    HalfStep hs = half_step<PREC>(h2, pos, vel, sa, sb, da, dv, dsa, dsb, lo, lob);
    {   // the step's largest predictor move in cells (the pair kernel's pruning margin): a
        // warp maximum, raised in the clock only when it is larger than the value there
        float d = fmaxf(fabsf(hs.x - pos.x), fmaxf(fabsf(hs.y - pos.y), fabsf(hs.z - pos.z))) / P.gdx;
        if (!(d <= PRUNE_DISP_MAX)) d = 2.0f * PRUNE_DISP_MAX;  // NaN, Inf or beyond the cap
        const unsigned act = __activemask();
        const unsigned m = __reduce_max_sync(act, __float_as_uint(d));  // d >= 0: bits order as values
        if ((threadIdx.x & 31) == __ffs(act) - 1 && m > *(volatile unsigned *)&a.clk->max_disp) {
            const unsigned cap = __float_as_uint(PRUNE_DISP_MAX);
            const unsigned old = atomicMax(&a.clk->max_disp, m);
            if (m > cap && old <= cap) atomicAdd(&a.clk->full_stencil_steps, 1ull);  // once per step
        }
    }
    const bool tool = fc.w == 1.f;
    float prs = 0.f;
    float Rr[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (!tool) {
        prs = P.c0sq * (hs.rho - P.rho0);
        if (P.stresseps != 0.f)
            artificial_stress(hs.S[0], hs.S[1], hs.S[2], hs.S[3], hs.S[4], hs.S[5], prs, hs.rho, P.stresseps, Rr);
    }
    const float ir2 = 1.0f / (hs.rho * hs.rho);
    const Records &r = a.r;
    r.f[REC_P][i] = make_float4(hs.x, hs.y, hs.z, fc.w);  // raw tool_particle value
    float4 *x = r.f[REC_V] + size_t(i) * REC_X;  // V, A, B, R, C interleaved
    x[REC_V - 1] = make_float4(hs.vx, hs.vy, hs.vz, hs.rho);
    x[REC_A - 1] = make_float4((hs.S[0] - prs) * ir2, (hs.S[1] - prs) * ir2, (hs.S[2] - prs) * ir2, hs.S[3] * ir2);
    x[REC_B - 1] = make_float4(hs.S[4] * ir2, hs.S[5] * ir2, sqrtf(P.K / hs.rho), pos.w);
    x[REC_R - 1] = make_float4(Rr[0], Rr[1], Rr[2], Rr[3]);
    x[REC_C - 1] = make_float4(Rr[4], Rr[5], hs.T, P.mass / hs.rho);
    if (P.diagnostics) a.s.pos_half[i] = make_float4(hs.x, hs.y, hs.z, 0.f);
}
template <bool PREC> __global__ void __launch_bounds__(256) kb_gather_predict(BatchTable T) {
    run_batched(T, T.pblk, [](const StepArgs &a, int b) { gather_predict_body<PREC>(a, b); });
}

// the initial state of a context from the constructor's arrays (particle_gpu,
// particle_gpu.cu:20-117: zeros except the given fields); the optional arrays
// may be NULL
__global__ void __launch_bounds__(256) k_init_state(int n, const float4 *pos, const float4 *vel, const float *rho,
                                                    const float *T, const float *h, const float *fixed,
                                                    const float *tool_p, State S, int *perm) {
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= n) return;
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 p = pos[i], v = vel[i];
    S.pos4[i] = make_float4(p.x, p.y, p.z, h[i]);
    S.vel4[i] = make_float4(v.x, v.y, v.z, rho[i]);
    S.sa4[i] = z;
    S.sb4[i] = make_float4(0.f, 0.f, T ? T[i] : 0.f, 0.f);
    S.da4[i] = z;
    S.dv4[i] = z;
    S.dsa4[i] = z;
    S.dsb4[i] = make_float4(0.f, 0.f, 0.f, fixed ? fixed[i] : 0.f);
    S.fc4[i] = make_float4(0.f, 0.f, 0.f, tool_p ? tool_p[i] : 0.f);
    S.ft4[i] = z;
    S.bc4[i] = make_float4(0.f, 0.f, 0.f, __int_as_float(i));  // creation index
    S.lo4[i] = z;
    S.lo4b[i] = z;
    perm[i] = i;
}

cudaError_t launch_init_state(int n, const float4 *pos, const float4 *vel, const float *rho, const float *T,
                              const float *h, const float *fixed, const float *tool_p, const State &S, int *perm,
                              cudaStream_t s) {
    k_init_state<<<(n + 255) / 256, 256, 0, s>>>(n, pos, vel, rho, T, h, fixed, tool_p, S, perm);
    return cudaGetLastError();
}

cudaError_t launch_gather_predict_batch(const BatchTable &T, bool precision, int blocks, cudaStream_t s) {
    if (precision) kb_gather_predict<true><<<blocks, 256, 0, s>>>(T);
    else kb_gather_predict<false><<<blocks, 256, 0, s>>>(T);
    return cudaGetLastError();
}

}  // namespace mfree
