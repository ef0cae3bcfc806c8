// mfree_static.cu -- the cell-list build of the step (cell hash, stable
// counting sort, cell ranges) for callers that cannot allocate device memory.
//
// mfree_step keeps its sort scratch (cell ids, per-cell counters, scan sums)
// in buffers the context allocates with cudaMalloc.  Some callers may not do
// that while they run: hosts whose device memory is reserved up front by their
// own allocator, and code that cannot afford the implicit device
// synchronisation a cudaMalloc may cause.  mfree_cell_list_static runs the
// same kernels with the scratch in a file-scope __device__ array of fixed size
// instead, and allocates nothing.
//
// Limits and sharing: at most MFREE_STATIC_MAX_PARTICLES particles and
// MFREE_STATIC_MAX_CELLS grid cells (about 3 MiB of device memory, held on
// every GPU that loads the library until the process exits).  All calls share
// the one array and it keeps the last call's contents: the per-cell counters
// are cleared at the start of each call, and calls that overlap on the GPU
// (different streams, or different host threads on one device) race on it.
#include <atomic>
#include <cstring>
#include <string>

#include "mfree.h"
#include "mfree_kernels.cuh"

namespace mfree {

namespace {

constexpr int MAX_N = MFREE_STATIC_MAX_PARTICLES;
constexpr int MAX_CELLS = MFREE_STATIC_MAX_CELLS;
constexpr int MAX_TILES = (MAX_CELLS + 1 + SCAN_TILE - 1) / SCAN_TILE + 1;
constexpr int MAX_HASH_BLOCKS = (MAX_N + HASH_BLOCK - 1) / HASH_BLOCK + 1;

struct StaticScratch {
    unsigned key[MAX_N];
    int count[MAX_CELLS + 1];
    int tile_sum[MAX_TILES];
    int blank_block[MAX_HASH_BLOCKS];
    DevClock clk;
};

// the scratch itself; host code must not pass its name to a kernel (on the
// host it is only a stand-in), it passes the device address found below
static __device__ __align__(256) StaticScratch g_static_scratch;

// device address of the array, looked up once per device by the first call
// on it (several host threads may make that first call at once: each finds
// the same address, and the atomic makes the store and the later loads
// well-defined).  After cudaDeviceReset the array lives at a new address the
// cache does not know: a process that resets a device must not call this
// entry point on that device again.
constexpr int MAX_DEVICES = 64;
std::atomic<StaticScratch *> g_scratch_addr[MAX_DEVICES];

// cell hash of plain positions: the step's kb_hash without blanking.  A
// position outside the grid, or with a NaN or infinite coordinate, goes to the
// tail like a blanked particle.  As in the step (and the reference's
// truncating (int) cast), a coordinate less than one cell below the grid's
// lower corner still falls in cell 0 of that axis.
__global__ void __launch_bounds__(HASH_BLOCK) k_hash_positions(StepArgs a, const float4 *pos, float bx, float by,
                                                               float bz) {
    const Params &P = a.p;
    const int i = blockIdx.x * HASH_BLOCK + threadIdx.x;
    int blank = 0;
    if (i < P.n_init) {
        const float4 p = pos[i];
        unsigned key = unsigned(P.num_cell);
        const bool finite = isfinite(p.x) && isfinite(p.y) && isfinite(p.z);
        const int ix = int(__fdiv_rn(__fsub_rn(p.x, bx), P.gdx));
        const int iy = int(__fdiv_rn(__fsub_rn(p.y, by), P.gdx));
        const int iz = int(__fdiv_rn(__fsub_rn(p.z, bz), P.gdx));
        if (finite && ix >= 0 && ix < P.gnx && iy >= 0 && iy < P.gny && iz >= 0 && iz < P.gnz)
            key = unsigned((ix * P.gny + iy) * P.gnz + iz);
        a.s.key[i] = key;
        if (key < unsigned(P.num_cell)) atomicAdd(&a.s.count[key], 1);
        else blank = 1;
    }
    const int nb = __syncthreads_count(blank);
    if (threadIdx.x == 0) a.s.blank_block[blockIdx.x] = nb;
}

int sfail(int code, const std::string &m) {
    set_last_error(m);
    return code;
}

}  // namespace

}  // namespace mfree

using namespace mfree;

extern "C" int mfree_cell_list_static(const float *pos4, int n, const float bbmin[3], float dx, int nx, int ny, int nz,
                                      int *perm, int *cell_first, void *stream) {
    if (!pos4 || !perm || !cell_first || !bbmin || n <= 0 || nx <= 0 || ny <= 0 || nz <= 0 || !(dx > 0.f))
        return sfail(MFREE_ERR_ARG, "mfree_cell_list_static: bad arguments");
    const long long ncell = (long long)nx * ny * nz;
    if (n > MAX_N)
        return sfail(MFREE_ERR_ARG, "mfree_cell_list_static: " + std::to_string(n) + " particles exceed the static limit of " +
                                        std::to_string(MAX_N));
    if (ncell > MAX_CELLS)
        return sfail(MFREE_ERR_ARG, "mfree_cell_list_static: " + std::to_string(ncell) +
                                        " grid cells exceed the static limit of " + std::to_string(MAX_CELLS));
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return sfail(MFREE_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= MAX_DEVICES) return sfail(MFREE_ERR_ARG, "mfree_cell_list_static: device index too large");
    StaticScratch *S = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (!S) {  // set-up, once per device, with that device current
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_static_scratch);
        if (e != cudaSuccess || !ptr)
            return sfail(MFREE_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        S = (StaticScratch *)ptr;
        g_scratch_addr[dev].store(S, std::memory_order_release);
    }
    cudaStream_t s = (cudaStream_t)stream;
    StepArgs a{};
    a.p.n_init = n;
    a.p.num_cell = int(ncell);
    a.p.gnx = nx;
    a.p.gny = ny;
    a.p.gnz = nz;
    a.p.gdx = dx;
    a.s.key = S->key;
    a.s.count = S->count;
    a.s.first = cell_first;
    a.s.tile_sum = S->tile_sum;
    a.s.blank_block = S->blank_block;
    a.s.perm = perm;
    a.clk = &S->clk;
    const int hb = (n + HASH_BLOCK - 1) / HASH_BLOCK;
    const int tiles = int((ncell + 1 + SCAN_TILE - 1) / SCAN_TILE);
    e = cudaMemsetAsync(S->count, 0, sizeof(int) * size_t(ncell + 1), s);  // the last call may have left counts
    if (e != cudaSuccess) return sfail(MFREE_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    k_hash_positions<<<hb, HASH_BLOCK, 0, s>>>(a, (const float4 *)pos4, bbmin[0], bbmin[1], bbmin[2]);
    k_scan_reduce<<<tiles, SCAN_THREADS, 0, s>>>(a);
    k_scan_top<<<1, 1024, 0, s>>>(a, tiles, hb);
    k_scan_down<<<tiles, SCAN_THREADS, 0, s>>>(a);
    k_scatter<<<hb, HASH_BLOCK, 0, s>>>(a);
    k_cell_fixup<<<int((ncell + 255) / 256), 256, 0, s>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return sfail(MFREE_ERR_CUDA, std::string("cell list kernels: ") + cudaGetErrorString(e));
    return MFREE_OK;
}
