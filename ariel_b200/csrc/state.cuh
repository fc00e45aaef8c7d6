// state.cuh -- the device-pointer bundle every kernel receives by value, and the launcher API
// between the host orchestration (host.cu) and the kernel files.
#pragma once

#include "common.cuh"

namespace ariel {

struct DevState {
    int k;  // scenes
    int any_solid;
    const SceneDev* scenes;
    const long long* p_pref;  // k+1: packed particle begins
    const long long* c_pref;  // k+1: packed cell begins
    const long long* f_pref;  // k+1: packed face begins
    long long np, nc, nf;

    // particle state, id order
    float4* pos4;  // x y z mass
    float4* vel4;  // u v w type-bits
    float4* pt4;   // StoreTemp position (solid scenes only)
    float4* ut4;   // StoreTemp velocity (solid scenes only)
    // sort products
    uint32_t* key;    // particle -> packed cell
    uint32_t* off;    // particle -> arrival offset inside its cell
    uint32_t* count;  // cell -> particles
    uint32_t* start;  // cell -> first slot (nc+1)
    uint32_t* sid;    // slot -> packed particle id (ascending inside a cell)
    float4* spos4;    // slot copies
    float4* svel4;
    float4* gpos4;    // slot -> P2G record: clamped grid position and mass (FLUID), far away
                      // for other particles so that they fall outside every face's radius
    float* dens;      // slot -> density
    // static solid particles binned by cell (positions never change)
    uint32_t* solid_start;  // nc+1
    float4* solid_pos;      // unit coordinates, id order inside a cell
    // grids
    uint8_t* flags;
    float* L;
    float* D;
    float* P;
    double* P64;
    float* u;   // m_mgrid faces
    float* pu;  // m_mgrid_previous faces
    // error word for bounded device waits
    int* dev_error;
    // reseeding pass (allocated when it is enabled): per cell the particles to give and to
    // receive, and their exclusive scans (nc + 1 entries)
    int any_reseed;
    uint32_t* rs_excess;
    uint32_t* rs_escan;
    uint32_t* rs_deficit;
    uint32_t* rs_dscan;
};

// Launchers (each returns cudaGetLastError()).
cudaError_t launch_begin(const DevState& S, cudaStream_t st);
cudaError_t launch_sort(const DevState& S, void* scan_tmp, cudaStream_t st);
cudaError_t launch_density(const DevState& S, cudaStream_t st);
cudaError_t launch_forces(const DevState& S, cudaStream_t st);
// faces: faces per thread (1, 2, 4), or 0 to choose by the number of faces
cudaError_t launch_p2g(const DevState& S, int faces, cudaStream_t st);
cudaError_t launch_classify(const DevState& S, int init_density, cudaStream_t st);
cudaError_t launch_boundary_div(const DevState& S, cudaStream_t st);
cudaError_t launch_gradient(const DevState& S, cudaStream_t st);
cudaError_t launch_extrapolate(const DevState& S, cudaStream_t st);
cudaError_t launch_g2p_advect(const DevState& S, cudaStream_t st);
cudaError_t launch_resample(const DevState& S, void* scan_tmp, cudaStream_t st);
cudaError_t launch_scatter_density(const DevState& S, float* out, cudaStream_t st);
cudaError_t launch_fill_dens(const DevState& S, float value, cudaStream_t st);
// xyz-interleaved host layout <-> float4 state (w components kept); unpack flags non-finite
// input in *err (bit 1).
cudaError_t launch_unpack_state(float4* pos4, float4* vel4, const float* pos, const float* vel, long long n,
                                int* err, cudaStream_t st);
cudaError_t launch_pack_state(const float4* pos4, const float4* vel4, float* pos, float* vel, long long n,
                              cudaStream_t st);

// Exclusive scan of n uint32 values into out[0..n] (out[n] = total).  tmp must hold
// scan_tmp_bytes(n) bytes.
size_t scan_tmp_bytes(long long n);
cudaError_t launch_scan_u32(const uint32_t* in, uint32_t* out, long long n, void* tmp, cudaStream_t st);

// Kernel-launch accounting (one increment per launched kernel).
void count_launch(int n = 1);
long long launch_count();

inline unsigned grid_for(long long n, int block = kBlock) { return (unsigned)((n + block - 1) / block); }

}  // namespace ariel
