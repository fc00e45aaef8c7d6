// noalloc.cu -- particle binning by cell that never allocates device memory.
//
// Some callers cannot call cudaMalloc once they are running: real-time simulation loops that
// must not stall on an allocation after start-up, and host applications or plugin frameworks
// whose own allocator owns all device memory and only ever hands out buffers it manages.  For
// them this file offers the sort-by-cell (the same binning as the SORT stage) with every
// temporary it needs kept in one fixed-size array compiled into the library.  The caller
// still provides the input positions and the output arrays.
//
// Limits: at most kNaMaxParticles particles and a grid of at most kNaMaxCells cells per call.
// The array is device memory that every GPU which loads this library holds until the process
// exits (about 5.2 MB).  All calls share it and it keeps the previous call's contents, so the
// per-cell counters are cleared at the start of every call, and calls that may run at the
// same time on the GPU (different streams, threads, or overlapping work) race on it.
#include <mutex>

#include "state.cuh"

namespace {

constexpr long long kNaMaxParticles = 1ll << 20;  // 1,048,576 particles
constexpr long long kNaMaxCells = 1ll << 18;      // 262,144 cells (a 64^3 grid)
constexpr long long kNaTileSums = kNaMaxCells / 4096 + 2;
constexpr long long kNaWords = kNaMaxCells + kNaMaxParticles + kNaTileSums;

// Scratch layout (uint32 words): per-cell counts | per-particle arrival offsets | scan tiles.
static __device__ __align__(256) uint32_t g_na_scratch[kNaWords];

// Device addresses of g_na_scratch, looked up once per device with that device current.
std::mutex g_na_mutex;
uint32_t* g_na_addr[64] = {nullptr};

__global__ void k_na_key(const float* __restrict__ pos, long long n, int dim, uint32_t* __restrict__ cell,
                         uint32_t* __restrict__ counts, uint32_t* __restrict__ offsets) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float maxd = (float)dim;
    int ci = ariel::cell_coord(maxd, pos[3 * i]);
    int cj = ariel::cell_coord(maxd, pos[3 * i + 1]);
    int ck = ariel::cell_coord(maxd, pos[3 * i + 2]);
    uint32_t c = (uint32_t)(((long long)ci * dim + cj) * dim + ck);
    cell[i] = c;
    offsets[i] = atomicAdd(&counts[c], 1u);
}

__global__ void k_na_scatter(long long n, const uint32_t* __restrict__ cell, const uint32_t* __restrict__ offsets,
                             const uint32_t* __restrict__ start, uint32_t* __restrict__ order) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t c = cell[i];
    order[start[c] + offsets[i]] = (uint32_t)i;
}

// Ascending particle id inside each cell, the order ParticleGrid::Sort appends them.
__global__ void k_na_cells(long long ncells, const uint32_t* __restrict__ start, uint32_t* __restrict__ order) {
    long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    uint32_t a = start[c], b = start[c + 1];
    for (uint32_t i = a + 1; i < b; ++i) {
        uint32_t v = order[i];
        uint32_t j = i;
        while (j > a && order[j - 1] > v) {
            order[j] = order[j - 1];
            --j;
        }
        order[j] = v;
    }
}

// Finds this device's copy of the scratch array.  Host code only knows the array's host-side
// stand-in symbol, which must never be handed to a kernel; the device address comes from
// cudaGetSymbolAddress with the device current.
ariel_status na_scratch(uint32_t** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return ARIEL_ERR_NO_DEVICE;
    }
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_na_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? ARIEL_ERR_NO_DEVICE : ARIEL_ERR_CUDA;
        }
        g_na_addr[dev] = (uint32_t*)p;
    }
    *out = g_na_addr[dev];
    return ARIEL_OK;
}

}  // namespace

extern "C" ariel_status ariel_sort_by_cell_noalloc(const float* pos, int64_t n, int32_t dim, uint32_t* particle_cell,
                                                   uint32_t* cell_start, uint32_t* order, void* stream) {
    if (n < 0 || dim < 1 || (n > 0 && (!pos || !particle_cell || !order)) || !cell_start)
        return ARIEL_ERR_INVALID_ARG;
    const long long ncells = (long long)dim * dim * dim;
    if (n > kNaMaxParticles || ncells > kNaMaxCells) return ARIEL_ERR_INVALID_ARG;
    uint32_t* scratch = nullptr;
    ariel_status st = na_scratch(&scratch);
    if (st != ARIEL_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    uint32_t* counts = scratch;
    uint32_t* offsets = scratch + kNaMaxCells;
    uint32_t* tiles = scratch + kNaMaxCells + kNaMaxParticles;
    // the counters hold the previous call's values
    if (cudaMemsetAsync(counts, 0, sizeof(uint32_t) * (size_t)ncells, s) != cudaSuccess) {
        cudaGetLastError();
        return ARIEL_ERR_CUDA;
    }
    if (n > 0) {
        k_na_key<<<ariel::grid_for(n), ariel::kBlock, 0, s>>>(pos, n, dim, particle_cell, counts, offsets);
        ariel::count_launch();
    }
    if (ariel::launch_scan_u32(counts, cell_start, ncells, tiles, s) != cudaSuccess) return ARIEL_ERR_CUDA;
    if (n > 0) {
        k_na_scatter<<<ariel::grid_for(n), ariel::kBlock, 0, s>>>(n, particle_cell, offsets, cell_start, order);
        k_na_cells<<<ariel::grid_for(ncells), ariel::kBlock, 0, s>>>(ncells, cell_start, order);
        ariel::count_launch(2);
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ARIEL_OK : ARIEL_ERR_CUDA;
}
