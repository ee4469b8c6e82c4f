// MHD pieces of the device path: face-to-cell B averaging
// (CT::computeBodyField, MHD/B_fields.cpp:70-89) used by initialize_B_fields,
// and the launcher of the 2D constrained-transport step.
#pragma once

#include "grid.cuh"

namespace dgpu {

// Grid2D/3D::initialize_B_fields after the boundary fill (B_fields.cpp:117-149):
// every cell, ghosts included, takes the average of its two face values per
// component (2D keeps the cell's z face value), pressure untouched.
__global__ void k_init_body_fields(Geo G, Geo FG, double* __restrict__ w, const double* __restrict__ B) {
    const int ng = G.g;
    const long long ex = G.ext[0], ey = G.ext[1], ez = G.ext[2];
    const long long total = ex * ey * ez;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % ez) - (G.dim == 3 ? ng : 0);
        const int j = (int)((t / ez) % ey) - ng;
        const int i = (int)(t / (ey * ez)) - ng;
        const long long FP = FG.plane;
        double bx, by, bz;
        long long m;
        if (G.dim == 2) {
            m = gidx2(G, i, j);
            const long long f = gidx2(FG, i, j);
            bx = (B[f] + B[gidx2(FG, i + 1, j)]) * 0.5;
            by = (B[FP + f] + B[FP + gidx2(FG, i, j + 1)]) * 0.5;
            bz = B[2 * FP + f];
        } else {
            m = gidx3(G, i, j, k);
            const long long f = gidx3(FG, i, j, k);
            bx = (B[f] + B[gidx3(FG, i + 1, j, k)]) * 0.5;
            by = (B[FP + f] + B[FP + gidx3(FG, i, j + 1, k)]) * 0.5;
            bz = (B[2 * FP + f] + B[2 * FP + gidx3(FG, i, j, k + 1)]) * 0.5;
        }
        w[5 * G.plane + m] = bx;
        w[6 * G.plane + m] = by;
        w[7 * G.plane + m] = bz;
    }
}

inline int launch_init_body_fields(const Geo& G, const Geo& FG, double* w, const double* B, cudaStream_t s) {
    const long long total = (long long)G.ext[0] * G.ext[1] * G.ext[2];
    int blocks = (int)((total + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_init_body_fields<<<blocks, 256, 0, s>>>(G, FG, w, B);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// 2D MHD CTU + CT step launcher; returns -1 while the kernel is not built.
template <int SOLVER>
inline int launch_step2d_mhd(const Geo&, const Geo&, const double*, double*, const double*, double*, StepCtl*,
                             const StepArgs&, cudaStream_t) {
    return -1;
}

}  // namespace dgpu
