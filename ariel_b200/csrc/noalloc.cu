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
//
// Order inside a cell: particles arrive in a cell in atomic order, and each cell's ids are then
// put in ascending order -- by one thread for cells of at most 32 particles, by a block in
// shared memory (bitonic network) up to 4096, and above that by a block that ranks every id
// against the whole cell (work quadratic in that cell's size; positions outside the unit cube
// are clamped into the edge cells, which is how such cells arise).
#include "state.cuh"

namespace {

constexpr long long kNaMaxParticles = 1ll << 20;  // 1,048,576 particles
constexpr long long kNaMaxCells = 1ll << 18;      // 262,144 cells (a 64^3 grid)
constexpr long long kNaTileSums = kNaMaxCells / 4096 + 2;
constexpr long long kNaWords = kNaMaxCells + kNaMaxParticles + kNaTileSums;
constexpr int kNaSmallCell = 32;    // cells up to this size: one thread, insertion sort
constexpr int kNaSharedCell = 4096; // cells up to this size: one block, bitonic sort in shared memory
constexpr int kNaBigBlock = 256;

// Scratch layout (uint32 words): per-cell counts | per-particle arrival offsets | scan tiles.
// After the scan and the scatter the first two regions are free again: the counts region then
// lists the cells too large for one thread, the offsets region is the large-cell sort's
// buffer, and the first scan word counts the listed cells.
static __device__ __align__(256) uint32_t g_na_scratch[kNaWords];

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

// Ascending particle id inside each cell, the order ParticleGrid::Sort appends them.  Cells of
// more than kNaSmallCell particles are listed for k_na_cells_big.
__global__ void k_na_cells_small(long long ncells, const uint32_t* __restrict__ start, uint32_t* __restrict__ order,
                                 uint32_t* __restrict__ big_list, uint32_t* __restrict__ big_count) {
    long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    uint32_t a = start[c], b = start[c + 1];
    if (b - a > (uint32_t)kNaSmallCell) {
        big_list[atomicAdd(big_count, 1u)] = (uint32_t)c;
        return;
    }
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

// One block per listed cell (grid-stride over the list).  Up to kNaSharedCell ids: bitonic sort
// of the cell padded to a power of two in shared memory.  Beyond: every id's rank is the number
// of smaller ids in the cell (ids are distinct), written to `tmp` at that rank, then copied back.
__global__ void __launch_bounds__(kNaBigBlock) k_na_cells_big(const uint32_t* __restrict__ start,
                                                              uint32_t* __restrict__ order,
                                                              const uint32_t* __restrict__ big_list,
                                                              const uint32_t* __restrict__ big_count,
                                                              uint32_t* __restrict__ tmp) {
    __shared__ uint32_t sh[kNaSharedCell];
    const uint32_t nbig = *big_count;
    for (uint32_t bi = blockIdx.x; bi < nbig; bi += gridDim.x) {
        const uint32_t c = big_list[bi];
        const uint32_t a = start[c], m = start[c + 1] - a;
        if (m <= (uint32_t)kNaSharedCell) {
            uint32_t p2 = 1;
            while (p2 < m) p2 <<= 1;
            for (uint32_t i = threadIdx.x; i < p2; i += blockDim.x) sh[i] = i < m ? order[a + i] : 0xFFFFFFFFu;
            __syncthreads();
            for (uint32_t k = 2; k <= p2; k <<= 1) {
                for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                    for (uint32_t i = threadIdx.x; i < p2; i += blockDim.x) {
                        uint32_t l = i ^ j;
                        if (l > i) {
                            uint32_t x = sh[i], y = sh[l];
                            bool up = (i & k) == 0;
                            if ((x > y) == up) {
                                sh[i] = y;
                                sh[l] = x;
                            }
                        }
                    }
                    __syncthreads();
                }
            }
            for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) order[a + i] = sh[i];
            __syncthreads();
        } else {
            for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
                const uint32_t v = order[a + i];
                uint32_t rank = 0;
                for (uint32_t q = 0; q < m; ++q) rank += order[a + q] < v ? 1u : 0u;
                tmp[a + rank] = v;
            }
            __syncthreads();
            for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) order[a + i] = tmp[a + i];
            __syncthreads();
        }
    }
}

// This device's copy of the scratch array.  Host code only knows the array's host-side
// stand-in symbol, which must never be handed to a kernel; the device address comes from
// cudaGetSymbolAddress with the device current.  It is looked up on every call (a host-side
// lookup once the module is loaded, no allocation), so it stays right if the caller resets the
// device and the module is loaded again at another address.
ariel_status na_scratch(uint32_t** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_na_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? ARIEL_ERR_NO_DEVICE : ARIEL_ERR_CUDA;
    }
    *out = (uint32_t*)p;
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
        // the scan is done with its tiles: its first word counts the cells too large for one thread
        uint32_t* big_count = tiles;
        if (cudaMemsetAsync(big_count, 0, sizeof(uint32_t), s) != cudaSuccess) {
            cudaGetLastError();
            return ARIEL_ERR_CUDA;
        }
        k_na_cells_small<<<ariel::grid_for(ncells), ariel::kBlock, 0, s>>>(ncells, cell_start, order, counts,
                                                                          big_count);
        int sms = 148;
        int dev = 0;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        k_na_cells_big<<<(unsigned)(2 * sms), kNaBigBlock, 0, s>>>(cell_start, order, counts, big_count, offsets);
        ariel::count_launch(3);
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ARIEL_OK : ARIEL_ERR_CUDA;
}
