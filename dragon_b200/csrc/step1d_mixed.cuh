// Mixed FP32/FP64 1D hydro sweep (Godunov::sweep + Grid1D::unsplit_step,
// Splitting.cpp:67-115): the FP64 tile of step_hydro.cuh (step1d_tile) with
// the MUSCL-Hancock half states, the limiters and the Riemann fluxes in FP32,
// and FP64 where stability needs it (mixed.cuh): the predictor's energy and
// every pressure recovery, and the conservative update of the FP64 state by
// the FP32 flux differences. With HLLC the tile carries its pressures as FP32
// offsets from the smallest FP64 pressure it loads (the normal-momentum flux
// rho u^2 + p then loses no mantissa to a large p; the offset cancels in each
// cell's flux difference).
//
// One tile of TS cells per call: the single-grid sweep (step1d_mixed.cu) runs
// one tile per CTA, the batched step (batch_mixed.cu) runs tiles as work
// items; both translation units are compiled with FMA contraction and fast
// single-precision division / square root, and both run the same arithmetic
// (batch.cu includes this header for the FP64 batch, which never runs it).
#pragma once

#include "mixed.cuh"
#include "step_hydro.cuh"

namespace dgpu {

// Cells per mixed 1D tile, in the single-grid sweep and in a batch alike: the
// pressure reference is a per-tile quantity, so the tiling is part of the
// arithmetic. 254 cells: the half states (256 cells) and faces (255) of a
// tile fit one round of a 256-thread CTA (the single-grid launch's threads,
// kMx1dThreads, and the batched step's).
constexpr int kMx1dTile = 254, kMx1dThreads = 256;

// Block-wide minimum of a per-thread value (a 1D block); every thread gets it.
__device__ __forceinline__ double tile_min_1d(double v, double* scratch) {
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? scratch[threadIdx.x] : INFINITY;
    if (warp == 0)
        for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0) scratch[0] = v;
    __syncthreads();
    v = scratch[0];
    __syncthreads();
    return v;
}

template <int SOLVER, int TS>
__device__ __forceinline__ void step1d_tile_mx(const Geo& G, const double* __restrict__ win, double* __restrict__ wout,
                                               StepCtl* ctl, const StepArgs& sa, int tile) {
    __shared__ float sw[5][TS + 4];
    __shared__ float sL[5][TS + 2], sR[5][TS + 2];
    __shared__ float sF[5][TS + 1];
    __shared__ double red[32];
    __shared__ int s_skip;
    if (cta_should_skip(ctl, &s_skip)) return;
    const int np = G.n[0] + 2 * G.g;  // padded cells
    const int p0 = tile * TS;
    const long long PL = G.plane;
    const double dt = *(volatile double*)&ctl->t1;
    const double dt_dx = dt / sa.dx;
    const float fdx = (float)dt_dx;
    const ExactOpts eo = exact_opts(sa);
    FaceStats st{0, 0, 0, 0, 0};
    int first_order = 0;

    // pressure reference: the smallest pressure the tile loads (HLLC), else 0
    double pref = 0.0;
    if constexpr (SOLVER == RS_HLLC) {
        double pmin = INFINITY;
        for (int q = threadIdx.x; q < TS + 4; q += blockDim.x) {
            const int p = p0 - 2 + q;
            if (p >= 0 && p < np) pmin = fmin(pmin, win[PL + p]);
        }
        pref = tile_min_1d(pmin, red);
        if (!(pref > 0.0 && pref < INFINITY)) pref = 0.0;
    }
    const float pref_f = (float)pref;

    for (int q = threadIdx.x; q < TS + 4; q += blockDim.x) {  // cell p = p0 - 2 + q
        const int p = p0 - 2 + q;
        if (p >= 0 && p < np) {
#pragma unroll
            for (int f = 0; f < 5; f++) sw[f][q] = (float)win[f * PL + p];
            sw[1][q] = (float)(win[PL + p] - pref);
        }
    }
    __syncthreads();
    auto getw = [&](int q) { return Prim<float>{sw[0][q], sw[1][q], sw[2][q], sw[3][q], sw[4][q], 0.f, 0.f, 0.f}; };
    auto put = [&](float (*arr)[TS + 2], int q, const Prim<float>& r) {
        arr[0][q] = r.rho; arr[1][q] = r.p; arr[2][q] = r.vx; arr[3][q] = r.vy; arr[4][q] = r.vz;
    };
    auto get = [&](float (*arr)[TS + 2], int q) {
        return Prim<float>{arr[0][q], arr[1][q], arr[2][q], arr[3][q], arr[4][q], 0.f, 0.f, 0.f};
    };

    // half states for cells p in [p0-1, p0+TS]; local index q = p - p0 + 1
    for (int q = threadIdx.x; q < TS + 2; q += blockDim.x) {
        const int p = p0 - 1 + q;
        if (p >= 1 && p <= np - 2) {
            Prim<float> oL, oR;
            first_order += !muscl_off(sa.limiter, getw(q), oL, getw(q + 1), oR, getw(q + 2), fdx, pref, pref_f);
            put(sL, q, oL);
            put(sR, q, oR);
        }
    }
    __syncthreads();
    // faces p in [p0-1, p0+TS-1] between cells p and p+1; the outermost faces
    // see the unreconstructed edge cells, as the FP64 sweep does
    for (int q = threadIdx.x; q < TS + 1; q += blockDim.x) {
        const int p = p0 - 1 + q;
        if (p < 0 || p > np - 2) continue;
        const Prim<float> L = (p == 0) ? getw(q + 1) : get(sR, q);
        const Prim<float> R = (p + 1 == np - 1) ? getw(q + 2) : get(sL, q + 1);
        Cons<float> F;
        if (!face_flux_off<SOLVER, 0>(L, R, fdx, eo, F, &st, pref, pref_f)) record_error(ctl, ST_FINAL_FLUX, p);
        sF[0][q] = F.rho; sF[1][q] = F.E; sF[2][q] = F.mx; sF[3][q] = F.my; sF[4][q] = F.mz;
    }
    __syncthreads();
    // FP64 update of the FP64 state by the FP32 flux differences
    double vmax = 0.0;
    for (int q = threadIdx.x; q < TS; q += blockDim.x) {  // cell p = p0 + q
        const int p = p0 + q;
        if (p >= np) continue;
        const Prim<double> w0 = load_prim<false>(win, PL, p);
        Prim<double> nw = w0;
        if (p >= 1 && p <= np - 2) {
            Cons<double> U = to_cons64<false>(w0);
            double* u5[5] = {&U.rho, &U.E, &U.mx, &U.my, &U.mz};
#pragma unroll
            for (int f = 0; f < 5; f++) *u5[f] += ((double)sF[f][q] - (double)sF[f][q + 1]) * dt_dx;
            nw = to_prim64<false>(U);
            // the FP64 sweep applies the last interior face's flux difference
            // to this cell a second time with both sides that face (a zero
            // difference): a conservative round trip
            if (p == np - 2) nw = to_prim64<false>(to_cons64<false>(nw));
        }
        const int c = p - G.g;
        if (c >= 0 && c < G.n[0]) {
            if (!is_physical<false>(nw)) record_error(ctl, ST_UNPHYSICAL, p);
            vmax = speed_max(vmax, cfl_speed_1d_mx<false>(nw));
        }
        store_prim<false>(wout, PL, p, nw);
    }
    vmax = block_max(vmax, red);
    if (threadIdx.x == 0) atomic_max_speed(&ctl->vmax[sa.slot_out], vmax);
    if (st.pivot_exact) atomicAdd(&ctl->pivots_exact, (unsigned long long)st.pivot_exact);
    if (st.newton_iters) atomicAdd(&ctl->newton_iters, (unsigned long long)st.newton_iters);
    if (st.exact_calls) atomicAdd(&ctl->exact_calls, (unsigned long long)st.exact_calls);
    if (st.trrs) atomicAdd(&ctl->trrs, (unsigned long long)st.trrs);
    if (st.cap_hits) atomicAdd(&ctl->cap_hits, (unsigned long long)st.cap_hits);
    if (first_order) atomicAdd(&ctl->muscl_first_order, (unsigned long long)first_order);
}

// The 1D MHD sweep (cell-centred B; the HLLD / HLL / HLLE fluxes) in mixed
// precision: FP32 MUSCL (no face-B source terms in 1D, as the FP64 sweep) and
// fluxes on absolute pressures, FP64 energies in every FP32 reconstruction,
// FP64 update of the FP64 state, the FP64 sweep's index ranges and end faces.
template <int SOLVER, int TS>
__device__ __forceinline__ void step1d_tile_mx_mhd(const Geo& G, const double* __restrict__ win,
                                                   double* __restrict__ wout, StepCtl* ctl, const StepArgs& sa,
                                                   int tile) {
    constexpr int NF = 8;
    __shared__ float sw[NF][TS + 4];
    __shared__ float sL[NF][TS + 2], sR[NF][TS + 2];
    __shared__ float sF[NF][TS + 1];
    __shared__ double red[32];
    __shared__ int s_skip;
    if (cta_should_skip(ctl, &s_skip)) return;
    const int np = G.n[0] + 2 * G.g;
    const int p0 = tile * TS;
    const long long PL = G.plane;
    const double dt = *(volatile double*)&ctl->t1;
    const double dt_dx = dt / sa.dx;
    const float fdx = (float)dt_dx;
    const ExactOpts eo = exact_opts(sa);
    FaceStats st{0, 0, 0, 0, 0};
    int first_order = 0;
    for (int q = threadIdx.x; q < TS + 4; q += blockDim.x) {  // cell p = p0 - 2 + q
        const int p = p0 - 2 + q;
        if (p >= 0 && p < np)
#pragma unroll
            for (int f = 0; f < NF; f++) sw[f][q] = (float)win[f * PL + p];
    }
    __syncthreads();
    auto getw = [&](int q) {
        return Prim<float>{sw[0][q], sw[1][q], sw[2][q], sw[3][q], sw[4][q], sw[5][q], sw[6][q], sw[7][q]};
    };
    auto put = [&](float (*arr)[TS + 2], int q, const Prim<float>& r) {
        arr[0][q] = r.rho; arr[1][q] = r.p; arr[2][q] = r.vx; arr[3][q] = r.vy; arr[4][q] = r.vz;
        arr[5][q] = r.Bx; arr[6][q] = r.By; arr[7][q] = r.Bz;
    };
    auto get = [&](float (*arr)[TS + 2], int q) {
        return Prim<float>{arr[0][q], arr[1][q], arr[2][q], arr[3][q], arr[4][q], arr[5][q], arr[6][q], arr[7][q]};
    };
    for (int q = threadIdx.x; q < TS + 2; q += blockDim.x) {  // cells p in [p0-1, p0+TS]
        const int p = p0 - 1 + q;
        if (p >= 1 && p <= np - 2) {
            Prim<float> oL, oR;
            first_order += !muscl_mixed<true>(sa.limiter, getw(q), oL, getw(q + 1), oR, getw(q + 2), fdx, 0.f, 0.f, 0.f);
            put(sL, q, oL);
            put(sR, q, oR);
        }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < TS + 1; q += blockDim.x) {  // faces p in [p0-1, p0+TS-1]
        const int p = p0 - 1 + q;
        if (p < 0 || p > np - 2) continue;
        const Prim<float> L = (p == 0) ? getw(q + 1) : get(sR, q);
        const Prim<float> R = (p + 1 == np - 1) ? getw(q + 2) : get(sL, q + 1);
        Cons<float> F;
        if (!face_flux_mixed<true, SOLVER, 0>(L, R, fdx, eo, F, &st)) record_error(ctl, ST_FINAL_FLUX, p);
        sF[0][q] = F.rho; sF[1][q] = F.E; sF[2][q] = F.mx; sF[3][q] = F.my; sF[4][q] = F.mz;
        sF[5][q] = F.Bx; sF[6][q] = F.By; sF[7][q] = F.Bz;
    }
    __syncthreads();
    double vmax = 0.0;
    for (int q = threadIdx.x; q < TS; q += blockDim.x) {  // cell p = p0 + q
        const int p = p0 + q;
        if (p >= np) continue;
        const Prim<double> w0 = load_prim<true>(win, PL, p);
        Prim<double> nw = w0;
        if (p >= 1 && p <= np - 2) {
            Cons<double> U = to_cons64<true>(w0);
            double* u8[NF] = {&U.rho, &U.E, &U.mx, &U.my, &U.mz, &U.Bx, &U.By, &U.Bz};
#pragma unroll
            for (int f = 0; f < NF; f++) *u8[f] += ((double)sF[f][q] - (double)sF[f][q + 1]) * dt_dx;
            nw = to_prim64<true>(U);
            // the FP64 sweep's second, zero-difference round trip on cell np-2
            if (p == np - 2) nw = to_prim64<true>(to_cons64<true>(nw));
        }
        const int c = p - G.g;
        if (c >= 0 && c < G.n[0]) {
            if (!is_physical<true>(nw)) record_error(ctl, ST_UNPHYSICAL, p);
            vmax = speed_max(vmax, cfl_speed_1d_mx<true>(nw));
        }
        store_prim<true>(wout, PL, p, nw);
    }
    vmax = block_max(vmax, red);
    if (threadIdx.x == 0) atomic_max_speed(&ctl->vmax[sa.slot_out], vmax);
    if (st.hlld_to_hlle) atomicAdd(&ctl->hlld_to_hlle, (unsigned long long)st.hlld_to_hlle);
    if (first_order) atomicAdd(&ctl->muscl_first_order, (unsigned long long)first_order);
}

}  // namespace dgpu
