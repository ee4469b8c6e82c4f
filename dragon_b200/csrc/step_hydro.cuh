// Fused unsplit step kernels for hydro grids (1D sweep, 2D CTU).
//
// 2D: one CTA owns a TI x TJ tile of output cells and recomputes a two-cell
// halo, so reconstruction, the predictor (CTU) fluxes, the transverse
// corrections, the final fluxes and the conservative update run in one pass
// over HBM (Grid2D::unsplit_step, Unsplit.cpp:28-111, with ctu_sweep_hydro and
// correctState, CTU.cpp:206-278). Every intermediate lives in shared memory.
// The tile covers exactly the faces and cells the reference computes, so the
// set of Riemann pivots that can fail is the same.
#pragma once

#include "grid.cuh"
#include "recon.cuh"
#include "riemann.cuh"
#include "tma.cuh"

namespace dgpu {

template <int TI, int TJ>
struct Smem2DH {
    static constexpr int HI = TI + 2, HJ = TJ + 2;
    static constexpr int WC = TJ + 6;  // tile columns as loaded: the halo, plus one for an odd first column
    double hs[4][5][HI][HJ];  // xL, xR, yL, yR half states (primitive)
    union U {
        double w[5][TI + 4][WC];  // w[f][a][b + off]: tile row a, column b, off the load's column offset
        struct F {
            double fx[5][TI + 1][TJ + 2];
            double fy[5][TI + 2][TJ + 1];
        } f;
    } u;
    double red[32];
    unsigned long long stat[7];
    uint64_t bar;
};

// First padded column of a tile's TMA box (even, so the box starts 16-byte
// aligned) and the offset of the tile's own first column inside the box.
__device__ __forceinline__ int tile_col0(int j0, int g) { return (j0 - 2 + g) & ~1; }
__device__ __forceinline__ int tile_off(int j0, int g) { return (j0 - 2 + g) & 1; }

enum { HS_XL = 0, HS_XR = 1, HS_YL = 2, HS_YR = 3 };

template <int TI, int TJ>
__device__ __forceinline__ Prim<double> hs_get(const Smem2DH<TI, TJ>& S, int k, int a, int b) {
    Prim<double> r;
    r.rho = S.hs[k][0][a][b];
    r.p = S.hs[k][1][a][b];
    r.vx = S.hs[k][2][a][b];
    r.vy = S.hs[k][3][a][b];
    r.vz = S.hs[k][4][a][b];
    r.Bx = r.By = r.Bz = 0;
    return r;
}
template <int TI, int TJ>
__device__ __forceinline__ void hs_put(Smem2DH<TI, TJ>& S, int k, int a, int b, const Prim<double>& r) {
    S.hs[k][0][a][b] = r.rho;
    S.hs[k][1][a][b] = r.p;
    S.hs[k][2][a][b] = r.vx;
    S.hs[k][3][a][b] = r.vy;
    S.hs[k][4][a][b] = r.vz;
}

__device__ __forceinline__ int ld_flag(const int* p) { return *(const volatile int*)p; }

// CTA-uniform early exit: thread 0 reads the error / done words once and the
// whole block follows its decision, so no thread skips a barrier the others
// reach.
__device__ __forceinline__ bool cta_should_skip(const StepCtl* ctl, int* s_flag) {
    if (threadIdx.x == 0) *s_flag = ld_flag(&ctl->err) | ld_flag(&ctl->done);
    __syncthreads();
    return *s_flag != 0;
}

// Copies the ghost cells a boundary tile owns from the input to the output
// buffer, so the committed array keeps the ghosts the prologue filled
// (Unsplit.cpp:106 commits the interior only).
template <int NF>
__device__ __forceinline__ void copy_ghosts_2d(const Geo& G, const double* __restrict__ win, double* __restrict__ wout,
                                               int i0, int j0, int TI, int TJ) {
    const int nx = G.n[0], ny = G.n[1], g = G.g;
    const bool first_i = i0 == 0, last_i = i0 + TI >= nx, first_j = j0 == 0, last_j = j0 + TJ >= ny;
    if (!(first_i || last_i || first_j || last_j)) return;
    const int lo_i = first_i ? -g : i0, hi_i = last_i ? nx + g : i0 + TI;
    const int lo_j = first_j ? -g : j0, hi_j = last_j ? ny + g : j0 + TJ;
    const int wj = hi_j - lo_j;
    const int total = (hi_i - lo_i) * wj;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        const int i = lo_i + t / wj, j = lo_j + t % wj;
        if (i >= 0 && i < nx && j >= 0 && j < ny) continue;
        const long long m = gidx2(G, i, j);
#pragma unroll
        for (int f = 0; f < NF; f++) wout[f * G.plane + m] = win[f * G.plane + m];
    }
}

template <int SOLVER, int TI, int TJ, int NT>
__global__ void __launch_bounds__(NT, NT >= 512 ? 1 : 2)
k_step2d_hydro(Geo G, const double* __restrict__ win, double* __restrict__ wout, StepCtl* ctl, StepArgs sa,
               const __grid_constant__ CUtensorMap tile_map) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    Smem2DH<TI, TJ>& S = *reinterpret_cast<Smem2DH<TI, TJ>*>(smem_raw);
    __shared__ int s_skip;
    if (cta_should_skip(ctl, &s_skip)) return;

    const int nx = G.n[0], ny = G.n[1], g = G.g;
    const long long PL = G.plane;
    const int i0 = blockIdx.y * TI, j0 = blockIdx.x * TJ;
    const double dt = *(volatile double*)&ctl->t1;
    const double dt_dx = dt / sa.dx, dt_dy = dt / sa.dy;
    const double hdx = 0.5 * dt_dx, hdy = 0.5 * dt_dy;
    const ExactOpts eo = exact_opts(sa);
    FaceStats st{0, 0, 0, 0, 0};
    int first_order = 0;
    if (threadIdx.x < 7) S.stat[threadIdx.x] = 0;

    // P0: tile + two-cell halo of the primitive state, one TMA copy of the five
    // planes (padded rows i0-2+g .., columns from the even column at or
    // before j0-2+g); cells past the padded array read zeros and are not used
    static_assert(sizeof(double) * 4 * 5 * (TI + 2) * (TJ + 2) % 128 == 0, "the tile must start 128-byte aligned");
    const int off = tile_off(j0, g);
    if (!load_state_tile(&S.u.w[0][0][0], &tile_map, tile_col0(j0, g), i0 - 2 + g,
                         (unsigned)sizeof(S.u.w), &S.bar, ctl))
        return;

    // P1: MUSCL-Hancock half states in x and y for cells [-1, TI] x [-1, TJ]
    // (computeHalfStates_X/Y, Unsplit.cpp:292-342)
    constexpr int HI = TI + 2, HJ = TJ + 2;
    for (int t = threadIdx.x; t < HI * HJ; t += NT) {
        const int a = t / HJ, b = t % HJ;
        const int i = i0 - 1 + a, j = j0 - 1 + b;
        if (!(i >= -1 && i <= nx && j >= -1 && j <= ny)) continue;
        auto W = [&](int aa, int bb) {
            Prim<double> r;
            bb += off;
            r.rho = S.u.w[0][aa][bb]; r.p = S.u.w[1][aa][bb];
            r.vx = S.u.w[2][aa][bb]; r.vy = S.u.w[3][aa][bb]; r.vz = S.u.w[4][aa][bb];
            r.Bx = r.By = r.Bz = 0;
            return r;
        };
        const Prim<double> wc = W(a + 1, b + 1);
        Prim<double> oL, oR;
        first_order += !muscl<false>(sa.limiter, W(a, b + 1), oL, wc, oR, W(a + 2, b + 1), dt_dx, 0.0, 0.0, 0.0);
        hs_put(S, HS_XL, a, b, oL);
        hs_put(S, HS_XR, a, b, oR);
        Prim<double> yl = W(a + 1, b), yc = wc, yr = W(a + 1, b + 2);
        swap_xy(yl); swap_xy(yc); swap_xy(yr);
        first_order += !muscl<false>(sa.limiter, yl, oL, yc, oR, yr, dt_dy, 0.0, 0.0, 0.0);
        swap_xy(oL); swap_xy(oR);
        hs_put(S, HS_YL, a, b, oL);
        hs_put(S, HS_YR, a, b, oR);
    }
    __syncthreads();

    // P2: predictor fluxes (ctu_sweep_hydro, CTU.cpp:206-218):
    // F_X on faces [0, TI] x rows [-1, TJ], F_Y on rows [-1, TI] x faces [0, TJ]
    constexpr int NFX = (TI + 1) * (TJ + 2), NFY = (TI + 2) * (TJ + 1);
    for (int t = threadIdx.x; t < NFX + NFY; t += NT) {
        Cons<double> F;
        if (t < NFX) {
            const int a = t / (TJ + 2), b = t % (TJ + 2);
            const int i = i0 + a, j = j0 - 1 + b;
            if (!(i <= nx && j >= -1 && j <= ny)) continue;
            bool ok = face_flux<false, SOLVER, 0>(hs_get(S, HS_XR, a, b), hs_get(S, HS_XL, a + 1, b), dt_dx, eo, F, &st);
            if (!ok) record_error(ctl, ST_PRELIM_FLUX, (long long)(i + g) * (ny + 2 * g) + (j + g));
            S.u.f.fx[0][a][b] = F.rho; S.u.f.fx[1][a][b] = F.E; S.u.f.fx[2][a][b] = F.mx;
            S.u.f.fx[3][a][b] = F.my; S.u.f.fx[4][a][b] = F.mz;
        } else {
            const int q = t - NFX;
            const int a = q / (TJ + 1), b = q % (TJ + 1);
            const int i = i0 - 1 + a, j = j0 + b;
            if (!(i >= -1 && i <= nx && j <= ny)) continue;
            bool ok = face_flux<false, SOLVER, 1>(hs_get(S, HS_YR, a, b), hs_get(S, HS_YL, a, b + 1), dt_dy, eo, F, &st);
            if (!ok) record_error(ctl, ST_PRELIM_FLUX, (long long)(i + g) * (ny + 2 * g) + (j + g));
            S.u.f.fy[0][a][b] = F.rho; S.u.f.fy[1][a][b] = F.E; S.u.f.fy[2][a][b] = F.mx;
            S.u.f.fy[3][a][b] = F.my; S.u.f.fy[4][a][b] = F.mz;
        }
    }
    __syncthreads();

    // P3: transverse corrections in conservative variables (correctState, CTU.cpp:264-278)
    constexpr int NCX = HI * TJ, NCY = TI * HJ;
    for (int t = threadIdx.x; t < NCX + NCY; t += NT) {
        if (t < NCX) {
            const int a = t / TJ, b = t % TJ + 1;
            const int i = i0 - 1 + a, j = j0 - 1 + b;
            if (!(i >= -1 && i <= nx && j < ny)) continue;
            Cons<double> tr;
            tr.rho = (S.u.f.fy[0][a][b] - S.u.f.fy[0][a][b - 1]) * hdy;
            tr.E = (S.u.f.fy[1][a][b] - S.u.f.fy[1][a][b - 1]) * hdy;
            tr.mx = (S.u.f.fy[2][a][b] - S.u.f.fy[2][a][b - 1]) * hdy;
            tr.my = (S.u.f.fy[3][a][b] - S.u.f.fy[3][a][b - 1]) * hdy;
            tr.mz = (S.u.f.fy[4][a][b] - S.u.f.fy[4][a][b - 1]) * hdy;
            hs_put(S, HS_XL, a, b, to_prim<false>(c_sub<false>(to_cons<false>(hs_get(S, HS_XL, a, b)), tr)));
            hs_put(S, HS_XR, a, b, to_prim<false>(c_sub<false>(to_cons<false>(hs_get(S, HS_XR, a, b)), tr)));
        } else {
            const int q = t - NCX;
            const int a = q / HJ + 1, b = q % HJ;
            const int i = i0 - 1 + a, j = j0 - 1 + b;
            if (!(i < nx && j >= -1 && j <= ny)) continue;
            Cons<double> tr;
            tr.rho = (S.u.f.fx[0][a][b] - S.u.f.fx[0][a - 1][b]) * hdx;
            tr.E = (S.u.f.fx[1][a][b] - S.u.f.fx[1][a - 1][b]) * hdx;
            tr.mx = (S.u.f.fx[2][a][b] - S.u.f.fx[2][a - 1][b]) * hdx;
            tr.my = (S.u.f.fx[3][a][b] - S.u.f.fx[3][a - 1][b]) * hdx;
            tr.mz = (S.u.f.fx[4][a][b] - S.u.f.fx[4][a - 1][b]) * hdx;
            hs_put(S, HS_YL, a, b, to_prim<false>(c_sub<false>(to_cons<false>(hs_get(S, HS_YL, a, b)), tr)));
            hs_put(S, HS_YR, a, b, to_prim<false>(c_sub<false>(to_cons<false>(hs_get(S, HS_YR, a, b)), tr)));
        }
    }
    __syncthreads();

    // P4: final fluxes (computeFlux_X/Y, Unsplit.cpp:64-65,210-225)
    constexpr int NGX = (TI + 1) * TJ, NGY = TI * (TJ + 1);
    for (int t = threadIdx.x; t < NGX + NGY; t += NT) {
        Cons<double> F;
        if (t < NGX) {
            const int a = t / TJ, b = t % TJ;
            const int i = i0 + a, j = j0 + b;
            if (!(i <= nx && j < ny)) continue;
            bool ok = face_flux<false, SOLVER, 0>(hs_get(S, HS_XR, a, b + 1), hs_get(S, HS_XL, a + 1, b + 1), dt_dx, eo, F, &st);
            if (!ok) record_error(ctl, ST_FINAL_FLUX, (long long)(i + g) * (ny + 2 * g) + (j + g));
            S.u.f.fx[0][a][b + 1] = F.rho; S.u.f.fx[1][a][b + 1] = F.E; S.u.f.fx[2][a][b + 1] = F.mx;
            S.u.f.fx[3][a][b + 1] = F.my; S.u.f.fx[4][a][b + 1] = F.mz;
        } else {
            const int q = t - NGX;
            const int a = q / (TJ + 1), b = q % (TJ + 1);
            const int i = i0 + a, j = j0 + b;
            if (!(i < nx && j <= ny)) continue;
            bool ok = face_flux<false, SOLVER, 1>(hs_get(S, HS_YR, a + 1, b), hs_get(S, HS_YL, a + 1, b + 1), dt_dy, eo, F, &st);
            if (!ok) record_error(ctl, ST_FINAL_FLUX, (long long)(i + g) * (ny + 2 * g) + (j + g));
            S.u.f.fy[0][a + 1][b] = F.rho; S.u.f.fy[1][a + 1][b] = F.E; S.u.f.fy[2][a + 1][b] = F.mx;
            S.u.f.fy[3][a + 1][b] = F.my; S.u.f.fy[4][a + 1][b] = F.mz;
        }
    }
    __syncthreads();

    // P5: conservative update, finiteness / physicality, CFL speed of the new state
    // (applyFluxes, Unsplit.cpp:256-270, and the check at Unsplit.cpp:95-99)
    double vmax = 0.0;
    for (int t = threadIdx.x; t < TI * TJ; t += NT) {
        const int a = t / TJ, b = t % TJ;
        const int i = i0 + a, j = j0 + b;
        if (!(i < nx && j < ny)) continue;
        const long long m = gidx2(G, i, j);
        Prim<double> w0 = load_prim<false>(win, PL, m);
        Cons<double> U = to_cons<false>(w0);
        Cons<double> d;
        d.rho = (S.u.f.fx[0][a][b + 1] - S.u.f.fx[0][a + 1][b + 1]) * dt_dx;
        d.E = (S.u.f.fx[1][a][b + 1] - S.u.f.fx[1][a + 1][b + 1]) * dt_dx;
        d.mx = (S.u.f.fx[2][a][b + 1] - S.u.f.fx[2][a + 1][b + 1]) * dt_dx;
        d.my = (S.u.f.fx[3][a][b + 1] - S.u.f.fx[3][a + 1][b + 1]) * dt_dx;
        d.mz = (S.u.f.fx[4][a][b + 1] - S.u.f.fx[4][a + 1][b + 1]) * dt_dx;
        U = c_add<false>(U, d);
        d.rho = (S.u.f.fy[0][a + 1][b] - S.u.f.fy[0][a + 1][b + 1]) * dt_dy;
        d.E = (S.u.f.fy[1][a + 1][b] - S.u.f.fy[1][a + 1][b + 1]) * dt_dy;
        d.mx = (S.u.f.fy[2][a + 1][b] - S.u.f.fy[2][a + 1][b + 1]) * dt_dy;
        d.my = (S.u.f.fy[3][a + 1][b] - S.u.f.fy[3][a + 1][b + 1]) * dt_dy;
        d.mz = (S.u.f.fy[4][a + 1][b] - S.u.f.fy[4][a + 1][b + 1]) * dt_dy;
        U = c_add<false>(U, d);
        Prim<double> nw = to_prim<false>(U);
        if (!is_finite<false>(U)) record_error(ctl, ST_NAN, (long long)(i + g) * (ny + 2 * g) + (j + g));
        else if (!is_physical<false>(nw)) record_error(ctl, ST_UNPHYSICAL, (long long)(i + g) * (ny + 2 * g) + (j + g));
        store_prim<false>(wout, PL, m, nw);
        vmax = speed_max(vmax, cfl_speed<false>(nw, sa.cfl, sa.dx, sa.dy, 0.0));
    }
    copy_ghosts_2d<5>(G, win, wout, i0, j0, TI, TJ);

    vmax = block_max(vmax, S.red);
    if (threadIdx.x == 0) atomic_max_speed(&ctl->vmax[sa.slot_out], vmax);
    // statistics
    if (st.pivot_exact) atomicAdd(&S.stat[0], (unsigned long long)st.pivot_exact);
    if (st.newton_iters) atomicAdd(&S.stat[2], (unsigned long long)st.newton_iters);
    if (st.exact_calls) atomicAdd(&S.stat[3], (unsigned long long)st.exact_calls);
    if (st.trrs) atomicAdd(&S.stat[4], (unsigned long long)st.trrs);
    if (first_order) atomicAdd(&S.stat[5], (unsigned long long)first_order);
    if (st.cap_hits) atomicAdd(&S.stat[6], (unsigned long long)st.cap_hits);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (S.stat[0]) atomicAdd(&ctl->pivots_exact, S.stat[0]);
        if (S.stat[2]) atomicAdd(&ctl->newton_iters, S.stat[2]);
        if (S.stat[3]) atomicAdd(&ctl->exact_calls, S.stat[3]);
        if (S.stat[4]) atomicAdd(&ctl->trrs, S.stat[4]);
        if (S.stat[5]) atomicAdd(&ctl->muscl_first_order, S.stat[5]);
        if (S.stat[6]) atomicAdd(&ctl->cap_hits, S.stat[6]);
    }
}

// ---------------------------------------------------------------------------
// 1D sweep (Godunov::sweep and Grid1D::unsplit_step, Splitting.cpp:67-115).
// Cells are addressed by padded index p in [0, n+2g). Faces p sit between
// cells p and p+1. The first face takes the raw leftmost ghost as its left
// state and the last face the raw rightmost ghost as its right state; every
// cell but the two outermost is updated, and cell n+2g-2 gets the reference's
// second zero-flux round trip (Splitting.cpp:93-94). All cells are committed.
// One tile of TS cells (cells tile*TS ...), any number of threads (the
// phases stride by blockDim.x). k_step1d runs one tile per CTA, the batched
// step runs tiles as work items.
template <bool MHD, int SOLVER, int TS>
__device__ __forceinline__ void step1d_tile(const Geo& G, const double* __restrict__ win, double* __restrict__ wout,
                                            StepCtl* ctl, const StepArgs& sa, int tile) {
    constexpr int NF = MHD ? 8 : 5;
    __shared__ double sw[NF][TS + 4];
    __shared__ double sL[NF][TS + 2], sR[NF][TS + 2];
    __shared__ double sF[NF][TS + 1];
    __shared__ double red[32];
    __shared__ int s_skip;
    if (cta_should_skip(ctl, &s_skip)) return;
    const int np = G.n[0] + 2 * G.g;   // padded cells
    const int p0 = tile * TS;
    const long long PL = G.plane;
    const double dt = *(volatile double*)&ctl->t1;
    const double dt_dx = dt / sa.dx;
    const ExactOpts eo = exact_opts(sa);
    FaceStats st{0, 0, 0, 0, 0};
    int first_order = 0;

    auto getw = [&](int q) {  // q in local w coordinates (p = p0 - 2 + q)
        Prim<double> r;
        r.rho = sw[0][q]; r.p = sw[1][q]; r.vx = sw[2][q]; r.vy = sw[3][q]; r.vz = sw[4][q];
        if constexpr (MHD) { r.Bx = sw[5][q]; r.By = sw[6][q]; r.Bz = sw[7][q]; }
        else r.Bx = r.By = r.Bz = 0;
        return r;
    };
    auto put = [&](double (*arr)[TS + 2], int q, const Prim<double>& r) {
        arr[0][q] = r.rho; arr[1][q] = r.p; arr[2][q] = r.vx; arr[3][q] = r.vy; arr[4][q] = r.vz;
        if constexpr (MHD) { arr[5][q] = r.Bx; arr[6][q] = r.By; arr[7][q] = r.Bz; }
    };
    auto get = [&](double (*arr)[TS + 2], int q) {
        Prim<double> r;
        r.rho = arr[0][q]; r.p = arr[1][q]; r.vx = arr[2][q]; r.vy = arr[3][q]; r.vz = arr[4][q];
        if constexpr (MHD) { r.Bx = arr[5][q]; r.By = arr[6][q]; r.Bz = arr[7][q]; }
        else r.Bx = r.By = r.Bz = 0;
        return r;
    };

    for (int q = threadIdx.x; q < TS + 4; q += blockDim.x) {
        const int p = p0 - 2 + q;
        if (p >= 0 && p < np)
            for (int f = 0; f < NF; f++) sw[f][q] = win[f * PL + p];
    }
    __syncthreads();
    // half states for cells p in [p0-1, p0+TS]; local index q = p - p0 + 1
    for (int q = threadIdx.x; q < TS + 2; q += blockDim.x) {
        const int p = p0 - 1 + q;
        if (p >= 1 && p <= np - 2) {
            Prim<double> oL, oR;
            first_order += !muscl<MHD>(sa.limiter, getw(q), oL, getw(q + 1), oR, getw(q + 2), dt_dx, 0.0, 0.0, 0.0);
            put(sL, q, oL);
            put(sR, q, oR);
        }
    }
    __syncthreads();
    // faces p in [p0-1, p0+TS-1]; local index q = p - p0 + 1
    for (int q = threadIdx.x; q < TS + 1; q += blockDim.x) {
        const int p = p0 - 1 + q;
        if (p < 0 || p > np - 2) continue;
        Prim<double> L = (p == 0) ? getw(q + 1) : get(sR, q);
        Prim<double> Rt = (p + 1 == np - 1) ? getw(q + 2) : get(sL, q + 1);
        Cons<double> F;
        bool ok = face_flux<MHD, SOLVER, 0>(L, Rt, dt_dx, eo, F, &st);
        if (!ok) record_error(ctl, ST_FINAL_FLUX, p);
        sF[0][q] = F.rho; sF[1][q] = F.E; sF[2][q] = F.mx; sF[3][q] = F.my; sF[4][q] = F.mz;
        if constexpr (MHD) { sF[5][q] = F.Bx; sF[6][q] = F.By; sF[7][q] = F.Bz; }
    }
    __syncthreads();
    double vmax = 0.0;
    for (int q = threadIdx.x; q < TS; q += blockDim.x) {   // cell p = p0 + q
        const int p = p0 + q;
        if (p < np) {
            Prim<double> w0 = getw(q + 2);
            Prim<double> nw = w0;
            auto fget = [&](int qq) {
                Cons<double> c;
                c.rho = sF[0][qq]; c.E = sF[1][qq]; c.mx = sF[2][qq]; c.my = sF[3][qq]; c.mz = sF[4][qq];
                if constexpr (MHD) { c.Bx = sF[5][qq]; c.By = sF[6][qq]; c.Bz = sF[7][qq]; }
                else c.Bx = c.By = c.Bz = 0;
                return c;
            };
            if (p >= 1 && p <= np - 2) {
                Cons<double> fl = fget(q), fr = fget(q + 1);
                nw = to_prim<MHD>(c_add<MHD>(to_cons<MHD>(w0), c_mul<MHD>(c_sub<MHD>(fl, fr), dt_dx)));
                if (p == np - 2)
                    nw = to_prim<MHD>(c_add<MHD>(to_cons<MHD>(nw), c_mul<MHD>(c_sub<MHD>(fr, fr), dt_dx)));
            }
            const int c = p - G.g;
            if (c >= 0 && c < G.n[0]) {
                if (!is_physical<MHD>(nw)) record_error(ctl, ST_UNPHYSICAL, p);
                vmax = speed_max(vmax, cfl_speed_1d<MHD>(nw));
            }
            store_prim<MHD>(wout, PL, p, nw);
        }
    }
    vmax = block_max(vmax, red);
    if (threadIdx.x == 0) atomic_max_speed(&ctl->vmax[sa.slot_out], vmax);
    if (st.pivot_exact) atomicAdd(&ctl->pivots_exact, (unsigned long long)st.pivot_exact);
    if (st.hlld_to_hlle) atomicAdd(&ctl->hlld_to_hlle, (unsigned long long)st.hlld_to_hlle);
    if (st.newton_iters) atomicAdd(&ctl->newton_iters, (unsigned long long)st.newton_iters);
    if (st.exact_calls) atomicAdd(&ctl->exact_calls, (unsigned long long)st.exact_calls);
    if (st.trrs) atomicAdd(&ctl->trrs, (unsigned long long)st.trrs);
    if (st.cap_hits) atomicAdd(&ctl->cap_hits, (unsigned long long)st.cap_hits);
    if (first_order) atomicAdd(&ctl->muscl_first_order, (unsigned long long)first_order);
}

template <bool MHD, int SOLVER, int TS, int NT>
__global__ void __launch_bounds__(NT)
k_step1d(Geo G, const double* __restrict__ win, double* __restrict__ wout, StepCtl* ctl, StepArgs sa) {
    step1d_tile<MHD, SOLVER, TS>(G, win, wout, ctl, sa, blockIdx.x);
}

}  // namespace dgpu
