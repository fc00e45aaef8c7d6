// scan.cu -- exclusive prefix sum of uint32 counts (cell histograms, FLUID-cell compaction).
//
// Three passes over tiles of 4096 values: per-tile sums, one block scanning the tile sums,
// per-tile scan plus offset.  Integer arithmetic, so the result does not depend on the order
// in which blocks run.
#include <atomic>

#include "state.cuh"

namespace ariel {

namespace {
constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
    const unsigned lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= (unsigned)o) v += t;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread; returns the exclusive prefix and the
// block total through *total.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warp_sums[kScanThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t inc = warp_incl_scan(v);
    if (lane == 31) warp_sums[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        constexpr int kWarps = kScanThreads / 32;
        uint32_t w = lane < kWarps ? warp_sums[lane] : 0;
        __syncwarp();
        uint32_t wi = warp_incl_scan(w);
        if (lane < kWarps) warp_sums[lane] = wi - w;
        if (lane == kWarps - 1) *total = wi;
    }
    __syncthreads();
    uint32_t r = warp_sums[wid] + inc - v;
    __syncthreads();
    return r;
}

__global__ void k_tile_sums(const uint32_t* __restrict__ in, long long n, uint32_t* __restrict__ sums) {
    long long base = (long long)blockIdx.x * kTile;
    uint32_t acc = 0;
#pragma unroll
    for (int it = 0; it < kScanItems; ++it) {
        long long i = base + (long long)it * kScanThreads + threadIdx.x;
        if (i < n) acc += in[i];
    }
    __shared__ uint32_t tot;
    block_excl_scan(acc, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void k_scan_sums(uint32_t* sums, long long nt) {
    __shared__ uint32_t carry_s;
    if (threadIdx.x == 0) carry_s = 0;
    __syncthreads();
    for (long long b = 0; b < nt; b += kScanThreads) {
        long long i = b + threadIdx.x;
        uint32_t v = i < nt ? sums[i] : 0;
        __shared__ uint32_t tot;
        uint32_t ex = block_excl_scan(v, &tot);
        uint32_t carry = carry_s;
        if (i < nt) sums[i] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry_s = carry + tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[nt] = carry_s;
}

__global__ void k_tile_scan(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, long long n,
                            const uint32_t* __restrict__ sums, long long nt) {
    long long base = (long long)blockIdx.x * kTile + (long long)threadIdx.x * kScanItems;
    uint32_t vals[kScanItems];
    uint32_t acc = 0;
#pragma unroll
    for (int it = 0; it < kScanItems; ++it) {
        long long i = base + it;
        vals[it] = i < n ? in[i] : 0;
        acc += vals[it];
    }
    __shared__ uint32_t tot;
    uint32_t ex = block_excl_scan(acc, &tot) + sums[blockIdx.x];
#pragma unroll
    for (int it = 0; it < kScanItems; ++it) {
        long long i = base + it;
        if (i < n) out[i] = ex;
        ex += vals[it];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = sums[nt];
}

std::atomic<long long> g_launches{0};
}  // namespace

void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

size_t scan_tmp_bytes(long long n) { return sizeof(uint32_t) * (size_t)((n + kTile - 1) / kTile + 2); }

cudaError_t launch_scan_u32(const uint32_t* in, uint32_t* out, long long n, void* tmp, cudaStream_t st) {
    long long nt = (n + kTile - 1) / kTile;
    uint32_t* sums = (uint32_t*)tmp;
    if (nt == 0) {
        cudaMemsetAsync(out, 0, sizeof(uint32_t), st);
        return cudaGetLastError();
    }
    k_tile_sums<<<(unsigned)nt, kScanThreads, 0, st>>>(in, n, sums);
    k_scan_sums<<<1, kScanThreads, 0, st>>>(sums, nt);
    k_tile_scan<<<(unsigned)nt, kScanThreads, 0, st>>>(in, out, n, sums, nt);
    count_launch(3);
    return cudaGetLastError();
}

}  // namespace ariel
