// Device-side grid description, step control block and shared helpers.
//
// Storage is structure-of-arrays: one FP64 plane per primitive field (rho, p,
// vx, vy, vz[, Bx, By, Bz]) over the ghost-padded grid, plus (MHD) three planes
// of face-centred B over the (n+1)-per-dimension padded face grid. Index order
// follows the reference (ExtendedArray.hpp:75,125): the last index is the
// contiguous one, so warps map onto j (2D) or k (3D) and loads coalesce.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fluid.cuh"
#include "riemann.cuh"

namespace dgpu {

struct MlpNet;

// Geometry of one padded array (cells or faces).
struct Geo {
    int dim;            // 1, 2 or 3
    int n[3];           // interior extents (1 for unused axes)
    int g;              // ghost width, all axes
    int ext[3];         // padded extents n + 2g (1 for unused axes)
    long long pitch;    // elements between consecutive values of the second-to-last index
    long long pitch2;   // elements between consecutive values of the first index (3D)
    long long plane;    // elements per field plane
};

// Cell index (i,j,k) in interior coordinates (ghosts negative / >= n).
__device__ __forceinline__ long long gidx1(const Geo& G, int i) { return (long long)(i + G.g); }
__device__ __forceinline__ long long gidx2(const Geo& G, int i, int j) {
    return (long long)(i + G.g) * G.pitch + (j + G.g);
}
__device__ __forceinline__ long long gidx3(const Geo& G, int i, int j, int k) {
    return (long long)(i + G.g) * G.pitch2 + (long long)(j + G.g) * G.pitch + (k + G.g);
}

// Mutable per-grid state the kernels of one advance share. Lives in device
// memory; the host reads it back after a batch of steps.
struct StepCtl {
    double remaining;              // interval left in the current advance (CFL.cpp:188-213)
    double t1;                     // dt of the current step
    double max_speed;              // max CFL signal speed seen by the last prologue
    double elapsed;                // sum of the committed steps' dt in this advance
    unsigned long long err_key;    // min over failures of (stage << 56 | linear cell index); ~0 = none
    int err;                       // non-zero once any failure was seen this batch
    int done;                      // advance finished (interval consumed or step budget reached)
    int have_prev;                 // a step was taken earlier in this advance
    int steps_done;                // successful steps in this advance
    int max_steps;                 // step budget (<= 0: unlimited)
    int check_cfl;                 // advance(dt, check_cfl)
    int cur;                       // batched step: buffer holding the current state
    int pad0;
    // statistics (summed over all face solves of committed and failed steps)
    unsigned long long pivots_exact, hlld_to_hlle, newton_iters, exact_calls, trrs, muscl_first_order;
    unsigned long long cap_hits, guess_rejects, judge_reruns;
    // grid barrier of the cooperative prologue (arrivals, generation) and its
    // ghost-ring max CFL speed (bits of a non-negative double)
    unsigned bar_arrive, bar_gen;
    unsigned long long ring_bits;
    // interior max CFL speed (bits of a non-negative double): slots 0/1 ping-pong
    // with the state buffers, slot 2 is scratch for cfl_time. Kept last: the
    // host rewrites everything before it when a new advance starts.
    unsigned long long vmax[3];
};

enum ErrStage : int {
    ST_NONE = 0,
    ST_PRELIM_FLUX = 1,   // Riemann pivot failed on a predictor / transverse flux
    ST_FINAL_FLUX = 2,    // Riemann pivot failed on a final flux
    ST_NAN = 3,           // non-finite conservative state in applyFluxes (Unsplit.cpp:267,284)
    ST_UNPHYSICAL = 4,    // unphysical committed state (Unsplit.cpp:97,192; Splitting.cpp:109)
    ST_CFL_ZERO = 5,      // max signal speed zero (CFL.cpp:102,117,134)
    ST_BARRIER = 6,       // a grid barrier of the cooperative prologue gave up waiting
    ST_TILE_LOAD = 7,     // a tile load into shared memory did not complete within its wait limit
};

__device__ __forceinline__ void record_error(StepCtl* ctl, int stage, long long cell) {
    unsigned long long key = ((unsigned long long)stage << 56) | ((unsigned long long)cell & 0x00FFFFFFFFFFFFFFull);
    atomicMin(&ctl->err_key, key);
    atomicExch(&ctl->err, 1);
}

// Non-negative doubles order like their bit patterns, so the CFL max reduces
// with an integer atomicMax. NaN speeds are skipped like std::max skips them
// when the running maximum is the first argument (CFL.cpp:100,114,130).
__device__ __forceinline__ double speed_max(double a, double b) { return smax(a, b); }
__device__ __forceinline__ void atomic_max_speed(unsigned long long* slot, double v) {
    if (v > 0.0) atomicMax(slot, (unsigned long long)__double_as_longlong(v));
}

// Block-wide max of a per-thread value (NaN-skipping). Returns the result in
// every thread. scratch needs 32 doubles.
__device__ __forceinline__ double block_max(double v, double* scratch) {
    for (int o = 16; o > 0; o >>= 1) v = speed_max(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? scratch[threadIdx.x] : 0.0;
    if (warp == 0)
        for (int o = 16; o > 0; o >>= 1) v = speed_max(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0) scratch[0] = v;
    __syncthreads();
    v = scratch[0];
    __syncthreads();
    return v;
}

// CFL signal speed of one cell (CFL.cpp:28-84). cfl: 0 MAX, 1 ADD, p>1 p-norm.
template <bool MHD>
__device__ __forceinline__ double cfl_speed(const Prim<double>& W, int cfl, double dx, double dy, double dz) {
    double a;
    if constexpr (MHD) a = fast_speed_max(W);
    else a = sound_speed(W);
    double speed = 0;
    if (cfl == 0) {
        if (dx > 1e-14) speed = (fabs(W.vx) + a) / dx;
        if (dy > 1e-14) speed = smax(speed, (fabs(W.vy) + a) / dy);
        if (dz > 1e-14) speed = smax(speed, (fabs(W.vz) + a) / dz);
    } else if (cfl == 1) {
        if (dx > 1e-14) speed = (fabs(W.vx) + a) / dx;
        if (dy > 1e-14) speed += (fabs(W.vy) + a) / dy;
        if (dz > 1e-14) speed += (fabs(W.vz) + a) / dz;
    } else {
        double p = (double)cfl;
        if (dx > 1e-14) speed = pow((fabs(W.vx) + a) / dx, p);
        if (dy > 1e-14) speed += pow((fabs(W.vy) + a) / dy, p);
        if (dz > 1e-14) speed += pow((fabs(W.vz) + a) / dz, p);
        speed = pow(speed, 1.0 / p);
    }
    return speed;
}
// 1D grids use |v.x| + a without dividing by dx (CFL.cpp:88-105).
template <bool MHD>
__device__ __forceinline__ double cfl_speed_1d(const Prim<double>& W) {
    double a;
    if constexpr (MHD) a = fast_speed_max(W);
    else a = sound_speed(W);
    return fabs(W.vx) + a;
}

template <bool MHD>
__device__ __forceinline__ double grid_cfl_speed(const Prim<double>& W, int dim, int cfl, double dx, double dy,
                                                 double dz) {
    if (dim == 1) return cfl_speed_1d<MHD>(W);
    return cfl_speed<MHD>(W, cfl, dx, dy, dz);
}

// Field-plane accessors.
template <bool MHD>
__device__ __forceinline__ Prim<double> load_prim(const double* __restrict__ w, long long plane, long long m) {
    Prim<double> r;
    r.rho = w[m];
    r.p = w[plane + m];
    r.vx = w[2 * plane + m];
    r.vy = w[3 * plane + m];
    r.vz = w[4 * plane + m];
    if constexpr (MHD) {
        r.Bx = w[5 * plane + m];
        r.By = w[6 * plane + m];
        r.Bz = w[7 * plane + m];
    } else {
        r.Bx = r.By = r.Bz = 0;
    }
    return r;
}
template <bool MHD>
__device__ __forceinline__ void store_prim(double* __restrict__ w, long long plane, long long m, const Prim<double>& r) {
    w[m] = r.rho;
    w[plane + m] = r.p;
    w[2 * plane + m] = r.vx;
    w[3 * plane + m] = r.vy;
    w[4 * plane + m] = r.vz;
    if constexpr (MHD) {
        w[5 * plane + m] = r.Bx;
        w[6 * plane + m] = r.By;
        w[7 * plane + m] = r.Bz;
    }
}

// Warp-aggregated statistics: one atomic per warp and counter instead of one
// per thread (threads that left early are simply not in the mask).
__device__ __forceinline__ void warp_add_stat(unsigned long long* dst, unsigned v) {
    const unsigned mask = __activemask();
    const unsigned sum = __reduce_add_sync(mask, v);
    if ((threadIdx.x & 31) == (unsigned)(__ffs(mask) - 1) && sum) atomicAdd(dst, (unsigned long long)sum);
}

// Parameters every step kernel receives by value.
struct StepArgs {
    double dx, dy, dz;
    int limiter;
    int cfl;
    int exact_max_iters;
    double exact_tol;
    int ct_energy;
    int slot_out;        // vmax slot the epilogue accumulates into
    int forced;          // retry: use ctl->t1 even if err was set earlier in this batch
    int exact_guess;     // GuessMode of the exact solver
    double guess_err;    // GUESS_PERFECT's relative error of the start
    NewtonLog nlog;      // converged-solve sample log (rows null: off)
    const MlpNet* mlp;   // learned guess network (GUESS_LEARNED)
};

__host__ __device__ __forceinline__ ExactOpts exact_opts(const StepArgs& sa) {
    return ExactOpts{sa.exact_max_iters, sa.exact_tol, sa.exact_guess, sa.nlog, sa.guess_err};
}

}  // namespace dgpu
