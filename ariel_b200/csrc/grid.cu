// grid.cu -- fused cell/face stencils of FlipSim::Step on sm_100a.
//
//   k_classify      MarkCellTypes + CellSDF/BuildSDF      (particlegrid.cpp:75-138)
//   k_boundary_div  StorePreviousGrid + EnforceBoundaryVelocity + divergence + FlipGrid
//                   (flip.cpp:324-363, particlegridoperations.inl:45-104, flip.cpp:420-437,
//                    solver.inl:42-56)
//   k_gradient      SubtractPressureGradient + EnforceBoundaryVelocity (flip.cpp:568-680)
//   k_extrapolate   ExtrapolateVelocity + SubtractPreviousGrid (flip.cpp:452-566, 365-410)
//
// Each output face has exactly one writing thread, so no stage needs atomics and every result
// is the reference's expression evaluated in its order.
#include "state.cuh"

namespace ariel {

namespace {

#define SCENE_PREFIX(pref_src)                   \
    __shared__ long long pref_s[kMaxScenes + 1]; \
    load_prefix<kMaxScenes>(pref_s, (pref_src), S.k)

struct FaceIdx {
    long long base;  // packed face begin of the scene
    long long per;   // faces per axis: n*n*(n+1)
    int n;
    __device__ __forceinline__ long long x(int i, int j, int k) const { return base + ((long long)i * n + j) * n + k; }
    __device__ __forceinline__ long long y(int i, int j, int k) const {
        return base + per + ((long long)i * (n + 1) + j) * n + k;
    }
    __device__ __forceinline__ long long z(int i, int j, int k) const {
        return base + 2 * per + ((long long)i * n + j) * (n + 1) + k;
    }
};


// ------------------------------------------------------------------------------------------
__global__ void k_classify(DevState S) {
    SCENE_PREFIX(S.c_pref);
    long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= S.nc) return;
    const SceneDev& D = S.scenes[find_scene(pref_s, S.k, c)];
    uint32_t a = S.start[c], b = S.start[c + 1];
    bool solid = false, nonfluid = false;
    float accm = 0.0f;
    for (uint32_t t = a; t < b; ++t) {
        int ty = type_of(S.svel4[t]);
        if (ty == ARIEL_SOLID) solid = true;
        if (!nonfluid) {
            if (ty == ARIEL_FLUID)
                accm += S.dens[t];
            else
                nonfluid = true;
        }
    }
    float sdf = nonfluid ? 1.0f : D.sdf0 - accm;
    S.L[c] = sdf;
    uint8_t flag = ARIEL_AIR;
    if (solid)
        flag = ARIEL_SOLID;
    else if (sdf < 0.0f)
        flag = ARIEL_FLUID;
    S.flags[c] = flag;
}

// ------------------------------------------------------------------------------------------
__device__ __forceinline__ float check_wall(const uint8_t* __restrict__ A, long long c) {
    return A[c] == ARIEL_SOLID ? 1.0f : -1.0f;
}

// Each thread of the cell stencils takes kCellsPerThread consecutive cells; as with faces, only
// the first cell and the first cell of a new row need the scene lookup and the index decoding.
constexpr int kCellsPerThread = 4;
template <class F>
__device__ __forceinline__ void for_cells(const DevState& S, const long long* pref_s, F&& body) {
    const long long c0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * kCellsPerThread;
    const SceneDev* D = nullptr;
    int i = 0, j = 0, k = 0;
#pragma unroll 1
    for (int q = 0; q < kCellsPerThread; ++q) {
        const long long c = c0 + q;
        if (c >= S.nc) return;
        if (D == nullptr || k + 1 >= D->n) {
            D = &S.scenes[find_scene(pref_s, S.k, c)];
            cell_ijk(*D, c - D->c_begin, i, j, k);
        } else {
            ++k;
        }
        body(c, *D, i, j, k);
    }
}

__global__ void k_boundary_div(DevState S) {
    SCENE_PREFIX(S.c_pref);
    for_cells(S, pref_s, [&](long long c, const SceneDev& D, int i, int j, int k) {
        const int n = D.n;
        FaceIdx F{D.f_begin, (long long)n * n * (n + 1), n};
        const uint8_t* A = S.flags;
        const long long cb = D.c_begin;
        auto cell = [&](int a, int b, int cc) { return cb + ((long long)a * n + b) * n + cc; };
        // enforced value of an x/y/z face from its raw value
        auto enf_x = [&](int fi, int fj, int fk, float raw) {
            if (fi == 0 || fi == n) return 0.0f;
            if (check_wall(A, cell(fi, fj, fk)) * check_wall(A, cell(fi - 1, fj, fk)) < 0) return 0.0f;
            return raw;
        };
        auto enf_y = [&](int fi, int fj, int fk, float raw) {
            if (fj == 0 || fj == n) return 0.0f;
            if (check_wall(A, cell(fi, fj, fk)) * check_wall(A, cell(fi, fj - 1, fk)) < 0) return 0.0f;
            return raw;
        };
        auto enf_z = [&](int fi, int fj, int fk, float raw) {
            if (fk == 0 || fk == n) return 0.0f;
            if (check_wall(A, cell(fi, fj, fk)) * check_wall(A, cell(fi, fj, fk - 1)) < 0) return 0.0f;
            return raw;
        };
        float* U = S.u;
        float* PU = S.pu;
        // owned faces: the low face of each axis, plus the domain-closing high face
        long long fx0 = F.x(i, j, k), fy0 = F.y(i, j, k), fz0 = F.z(i, j, k);
        float rx0 = U[fx0], ry0 = U[fy0], rz0 = U[fz0];
        float ex0 = enf_x(i, j, k, rx0), ey0 = enf_y(i, j, k, ry0), ez0 = enf_z(i, j, k, rz0);
        long long fx1 = F.x(i + 1, j, k), fy1 = F.y(i, j + 1, k), fz1 = F.z(i, j, k + 1);
        // a neighbour may already have replaced its raw value by the enforced one; enforcement is
        // idempotent, so either reading gives the same enforced value
        float rx1 = U[fx1], ry1 = U[fy1], rz1 = U[fz1];
        float ex1 = enf_x(i + 1, j, k, rx1), ey1 = enf_y(i, j + 1, k, ry1), ez1 = enf_z(i, j, k + 1, rz1);
        PU[fx0] = rx0;
        PU[fy0] = ry0;
        PU[fz0] = rz0;
        U[fx0] = ex0;
        U[fy0] = ey0;
        U[fz0] = ez0;
        if (i == n - 1) {
            PU[fx1] = rx1;
            U[fx1] = ex1;
        }
        if (j == n - 1) {
            PU[fy1] = ry1;
            U[fy1] = ey1;
        }
        if (k == n - 1) {
            PU[fz1] = rz1;
            U[fz1] = ez1;
        }
        float divergence = (ex1 - ex0 + ey1 - ey0 + ez1 - ez0) / D.h;
        S.D[c] = -divergence;
    });
}

// ------------------------------------------------------------------------------------------
// Each thread of the face kernels takes kFacesPerThread consecutive faces of the packed face
// space.  Faces along k are consecutive within a row, so only the first face and the first face
// after a row's end (a new row, axis block or scene) need the scene lookup and the index
// decoding; the others are the previous face with k + 1.  The per-face work stays what it was.
constexpr int kFacesPerThread = 4;
template <class F>
__device__ __forceinline__ void for_faces(const DevState& S, const long long* pref_s, F&& body) {
    const long long g0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * kFacesPerThread;
    const SceneDev* D = nullptr;
    int axis = 0, i = 0, j = 0, k = 0, ek = 0;
#pragma unroll 1
    for (int q = 0; q < kFacesPerThread; ++q) {
        const long long g = g0 + q;
        if (g >= S.nf) return;
        if (D == nullptr || k + 1 >= ek) {
            D = &S.scenes[find_scene(pref_s, S.k, g)];
            face_ijk(*D, g - D->f_begin, axis, i, j, k);
            ek = D->n + (axis == 2 ? 1 : 0);
        } else {
            ++k;
        }
        body(g, *D, axis, i, j, k);
    }
}

__global__ void k_gradient(DevState S) {
    SCENE_PREFIX(S.f_pref);
    for_faces(S, pref_s, [&](long long g, const SceneDev& D, int axis, int i, int j, int k) {
        const int n = D.n;
        const long long cb = D.c_begin;
        const int di = axis == 0, dj = axis == 1, dk = axis == 2;
        const int m = axis == 0 ? i : (axis == 1 ? j : k);
        float v = S.u[g];
        if (m > 0 && m < n) {
            long long cf = cb + ((long long)i * n + j) * n + k;
            long long cbk = cb + ((long long)(i - di) * n + (j - dj)) * n + (k - dk);
            const float* P = S.P;
            const float* L = S.L;
            float pf = P[cf], pb = P[cbk];
            if (D.subcell && L[cf] * L[cbk] < 0.0f) {
                pf = L[cf] < 0.0f ? P[cf] : L[cf] / gmin(1.0e-3f, L[cbk]) * P[cbk];
                pb = L[cbk] < 0.0f ? P[cbk] : L[cbk] / gmin(1.0e-6f, L[cf]) * P[cf];
            }
            v -= (pf - pb) / D.h;
            // EnforceBoundaryVelocity: faces between a SOLID and a non-SOLID cell
            if (check_wall(S.flags, cf) * check_wall(S.flags, cbk) < 0) v = 0.0f;
        } else {
            v = 0.0f;  // domain boundary face
        }
        S.u[g] = v;
    });
}

// ------------------------------------------------------------------------------------------
__global__ void k_extrapolate(DevState S) {
    SCENE_PREFIX(S.f_pref);
    for_faces(S, pref_s, [&](long long g, const SceneDev& D, int axis, int i, int j, int k) {
        const int n = D.n;
        const long long cb = D.c_begin;
        const uint8_t* A = S.flags;
        const int di = axis == 0, dj = axis == 1, dk = axis == 2;
        const int ex = n + di, ey = n + dj, ez = n + dk;  // face-grid extents of this axis
        // mark: face touches a FLUID cell; wallmark: both sides SOLID or outside (flip.cpp:460-510)
        auto marks = [&](int a, int b, int c, bool& mark, bool& wall) {
            int m = axis == 0 ? a : (axis == 1 ? b : c);
            bool has_lo = m > 0, has_hi = m < n;
            uint8_t lo = has_lo ? A[cb + ((long long)(a - di) * n + (b - dj)) * n + (c - dk)] : 0;
            uint8_t hi = has_hi ? A[cb + ((long long)a * n + b) * n + c] : 0;
            mark = (has_lo && lo == ARIEL_FLUID) || (has_hi && hi == ARIEL_FLUID);
            wall = (!has_lo || lo == ARIEL_SOLID) && (!has_hi || hi == ARIEL_SOLID);
        };
        auto fidx = [&](int a, int b, int c) {
            return D.f_begin + (long long)axis * n * n * (n + 1) + ((long long)a * ey + b) * ez + c;
        };
        float v = S.u[g];
        bool mark, wall;
        marks(i, j, k, mark, wall);
        if (!mark && wall) {
            unsigned wsum = 0;
            float sum = 0.0f;
            const int q[6][3] = {{i - 1, j, k}, {i + 1, j, k}, {i, j - 1, k}, {i, j + 1, k}, {i, j, k - 1}, {i, j, k + 1}};
            for (int qk = 0; qk < 6; ++qk) {
                int a = q[qk][0], b = q[qk][1], c = q[qk][2];
                if (a >= 0 && a < ex && b >= 0 && b < ey && c >= 0 && c < ez) {
                    bool qm, qw;
                    marks(a, b, c, qm, qw);
                    if (qm) {
                        wsum++;
                        sum += S.u[fidx(a, b, c)];
                    }
                }
            }
            if (wsum) {
                v = sum / wsum;
                S.u[g] = v;
            }
        }
        S.pu[g] = v - S.pu[g];
    });
}

}  // namespace

cudaError_t launch_classify(const DevState& S, int init_density, cudaStream_t st) {
    (void)init_density;
    if (S.nc == 0) return cudaSuccess;
    k_classify<<<grid_for(S.nc), kBlock, 0, st>>>(S);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_boundary_div(const DevState& S, cudaStream_t st) {
    if (S.nc == 0) return cudaSuccess;
    k_boundary_div<<<grid_for((S.nc + kCellsPerThread - 1) / kCellsPerThread), kBlock, 0, st>>>(S);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_gradient(const DevState& S, cudaStream_t st) {
    if (S.nf == 0) return cudaSuccess;
    k_gradient<<<grid_for((S.nf + kFacesPerThread - 1) / kFacesPerThread), kBlock, 0, st>>>(S);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_extrapolate(const DevState& S, cudaStream_t st) {
    if (S.nf == 0) return cudaSuccess;
    k_extrapolate<<<grid_for((S.nf + kFacesPerThread - 1) / kFacesPerThread), kBlock, 0, st>>>(S);
    count_launch();
    return cudaGetLastError();
}

}  // namespace ariel
