// Mixed-precision fused 2D CTU hydro step.
//
// Same tile schedule as the FP64 kernel (load, MUSCL x/y, predictor fluxes,
// transverse corrections, final fluxes, update, all in shared memory), with
// the tile data and the Riemann/MUSCL arithmetic in FP32 and, per the mixed
// design, FP64 kept for: the state in HBM, every pressure recovery from a
// conservative state (mixed.cuh), and the conservative flux-difference
// accumulation into U. With HLLC the tile holds its pressures as offsets from
// the smallest FP64 pressure it loads (mixed.cuh, pressure offset), so the
// normal-momentum fluxes do not round the absolute pressure.
// This translation unit is compiled with FMA contraction
// and fast single-precision division / square root (--fmad=true
// -prec-div=false -prec-sqrt=false -ftz=true); none of these flags changes
// double-precision arithmetic.
#include <cuda_runtime.h>

#include "launchers.h"
#include "mixed.cuh"
#include "step_hydro.cuh"

namespace dgpu {

template <int TI, int TJ>
struct SmemMixed {
    static constexpr int HI = TI + 2, HJ = TJ + 2;
    float hs[4][5][HI][HJ];
    union U {
        float w[5][TI + 4][TJ + 4];
        struct F {
            float fx[5][TI + 1][TJ + 2];
            float fy[5][TI + 2][TJ + 1];
        } f;
    } u;
    double red[32];
    unsigned long long stat[6];
    uint64_t bar;
};

template <int TI, int TJ>
__device__ __forceinline__ Prim<float> hsm_get(const SmemMixed<TI, TJ>& S, int k, int a, int b) {
    return Prim<float>{S.hs[k][0][a][b], S.hs[k][1][a][b], S.hs[k][2][a][b], S.hs[k][3][a][b], S.hs[k][4][a][b], 0.f,
                       0.f, 0.f};
}
template <int TI, int TJ>
__device__ __forceinline__ void hsm_put(SmemMixed<TI, TJ>& S, int k, int a, int b, const Prim<float>& r) {
    S.hs[k][0][a][b] = r.rho;
    S.hs[k][1][a][b] = r.p;
    S.hs[k][2][a][b] = r.vx;
    S.hs[k][3][a][b] = r.vy;
    S.hs[k][4][a][b] = r.vz;
}

// Block-wide minimum of a per-thread value; every thread gets it. scratch: 32 doubles.
__device__ __forceinline__ double block_min(double v, double* scratch) {
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

// Three CTAs per SM (80 registers, 72.7 KB shared memory each): measured 14 %
// faster than two CTAs at 110 registers on a 2048^2 shear layer, same results.
template <int SOLVER, int TI, int TJ, int NT>
__global__ void __launch_bounds__(NT, NT >= 384 ? 2 : 3)
k_step2d_hydro_mixed(Geo G, const double* __restrict__ win, double* __restrict__ wout, StepCtl* ctl, StepArgs sa,
                     const __grid_constant__ CUtensorMap tile_map) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    SmemMixed<TI, TJ>& S = *reinterpret_cast<SmemMixed<TI, TJ>*>(smem_raw);
    __shared__ int s_skip;
    if (cta_should_skip(ctl, &s_skip)) return;

    const int nx = G.n[0], ny = G.n[1], g = G.g;
    const long long PL = G.plane;
    const int i0 = blockIdx.y * TI, j0 = blockIdx.x * TJ;
    const double dt = *(volatile double*)&ctl->t1;
    const double dt_dx = dt / sa.dx, dt_dy = dt / sa.dy;
    const float fdx = (float)dt_dx, fdy = (float)dt_dy, hdx = (float)(0.5 * dt_dx), hdy = (float)(0.5 * dt_dy);
    const ExactOpts eo = exact_opts(sa);
    FaceStats st{0, 0, 0, 0, 0};
    int first_order = 0;
    if (threadIdx.x < 6) S.stat[threadIdx.x] = 0;

    constexpr int WI = TI + 4, WJ = TJ + 4, WC = TJ + 6;
    // the FP64 tile (five planes, padded rows i0-2+g .., columns from the even
    // column at or before j0-2+g) arrives by one TMA copy into a staging area
    // that the half states overwrite later
    static_assert(sizeof(double) * 5 * WI * WC <= sizeof(S.hs), "the FP64 tile must fit in the half-state area");
    double* stg = reinterpret_cast<double*>(&S.hs[0][0][0][0]);
    const int off = (j0 - 2 + g) & 1;
    if (!load_state_tile(stg, &tile_map, (j0 - 2 + g) & ~1, i0 - 2 + g, (unsigned)(sizeof(double) * 5 * WI * WC),
                         &S.bar, ctl))
        return;
    auto T = [&](int f, int a, int b) { return stg[(f * WI + a) * WC + b + off]; };
    // pressure reference of the tile (mixed.cuh, pressure offset): the smallest
    // pressure it loads, with HLLC; zero (absolute pressures) otherwise
    double pref = 0.0;
    if constexpr (SOLVER == RS_HLLC) {
        double pmin = INFINITY;
        for (int t = threadIdx.x; t < WI * WJ; t += NT) {
            const int a = t / WJ, b = t % WJ;
            const int i = i0 - 2 + a, j = j0 - 2 + b;
            if (i >= -g && i < nx + g && j >= -g && j < ny + g) pmin = fmin(pmin, T(1, a, b));
        }
        pref = block_min(pmin, S.red);
        if (!(pref > 0.0 && pref < INFINITY)) pref = 0.0;
    }
    const float pref_f = (float)pref;
    for (int t = threadIdx.x; t < WI * WJ; t += NT) {
        const int a = t / WJ, b = t % WJ;
        const int i = i0 - 2 + a, j = j0 - 2 + b;
        if (i >= -g && i < nx + g && j >= -g && j < ny + g) {
#pragma unroll
            for (int f = 0; f < 5; f++) S.u.w[f][a][b] = (float)T(f, a, b);
            S.u.w[1][a][b] = (float)(T(1, a, b) - pref);
        }
    }
    __syncthreads();

    constexpr int HI = TI + 2, HJ = TJ + 2;
    for (int t = threadIdx.x; t < HI * HJ; t += NT) {
        const int a = t / HJ, b = t % HJ;
        const int i = i0 - 1 + a, j = j0 - 1 + b;
        if (!(i >= -1 && i <= nx && j >= -1 && j <= ny)) continue;
        auto W = [&](int aa, int bb) {
            return Prim<float>{S.u.w[0][aa][bb], S.u.w[1][aa][bb], S.u.w[2][aa][bb], S.u.w[3][aa][bb],
                               S.u.w[4][aa][bb], 0.f, 0.f, 0.f};
        };
        const Prim<float> wc = W(a + 1, b + 1);
        Prim<float> oL, oR;
        first_order += !muscl_off(sa.limiter, W(a, b + 1), oL, wc, oR, W(a + 2, b + 1), fdx, pref, pref_f);
        hsm_put(S, HS_XL, a, b, oL);
        hsm_put(S, HS_XR, a, b, oR);
        Prim<float> yl = W(a + 1, b), yc = wc, yr = W(a + 1, b + 2);
        swap_xy(yl); swap_xy(yc); swap_xy(yr);
        first_order += !muscl_off(sa.limiter, yl, oL, yc, oR, yr, fdy, pref, pref_f);
        swap_xy(oL); swap_xy(oR);
        hsm_put(S, HS_YL, a, b, oL);
        hsm_put(S, HS_YR, a, b, oR);
    }
    __syncthreads();

    constexpr int NFX = (TI + 1) * (TJ + 2), NFY = (TI + 2) * (TJ + 1);
    for (int t = threadIdx.x; t < NFX + NFY; t += NT) {
        Cons<float> F;
        if (t < NFX) {
            const int a = t / (TJ + 2), b = t % (TJ + 2);
            const int i = i0 + a, j = j0 - 1 + b;
            if (!(i <= nx && j >= -1 && j <= ny)) continue;
            if (!face_flux_off<SOLVER, 0>(hsm_get(S, HS_XR, a, b), hsm_get(S, HS_XL, a + 1, b), fdx, eo, F, &st, pref,
                                          pref_f))
                record_error(ctl, ST_PRELIM_FLUX, (long long)(i + g) * (ny + 2 * g) + (j + g));
            S.u.f.fx[0][a][b] = F.rho; S.u.f.fx[1][a][b] = F.E; S.u.f.fx[2][a][b] = F.mx;
            S.u.f.fx[3][a][b] = F.my; S.u.f.fx[4][a][b] = F.mz;
        } else {
            const int q = t - NFX;
            const int a = q / (TJ + 1), b = q % (TJ + 1);
            const int i = i0 - 1 + a, j = j0 + b;
            if (!(i >= -1 && i <= nx && j <= ny)) continue;
            if (!face_flux_off<SOLVER, 1>(hsm_get(S, HS_YR, a, b), hsm_get(S, HS_YL, a, b + 1), fdy, eo, F, &st, pref,
                                          pref_f))
                record_error(ctl, ST_PRELIM_FLUX, (long long)(i + g) * (ny + 2 * g) + (j + g));
            S.u.f.fy[0][a][b] = F.rho; S.u.f.fy[1][a][b] = F.E; S.u.f.fy[2][a][b] = F.mx;
            S.u.f.fy[3][a][b] = F.my; S.u.f.fy[4][a][b] = F.mz;
        }
    }
    __syncthreads();

    constexpr int NCX = HI * TJ, NCY = TI * HJ;
    for (int t = threadIdx.x; t < NCX + NCY; t += NT) {
        if (t < NCX) {
            const int a = t / TJ, b = t % TJ + 1;
            const int i = i0 - 1 + a, j = j0 - 1 + b;
            if (!(i >= -1 && i <= nx && j < ny)) continue;
            Cons<float> tr;
            tr.rho = (S.u.f.fy[0][a][b] - S.u.f.fy[0][a][b - 1]) * hdy;
            tr.E = (S.u.f.fy[1][a][b] - S.u.f.fy[1][a][b - 1]) * hdy;
            tr.mx = (S.u.f.fy[2][a][b] - S.u.f.fy[2][a][b - 1]) * hdy;
            tr.my = (S.u.f.fy[3][a][b] - S.u.f.fy[3][a][b - 1]) * hdy;
            tr.mz = (S.u.f.fy[4][a][b] - S.u.f.fy[4][a][b - 1]) * hdy;
            tr.Bx = tr.By = tr.Bz = 0.f;
            hsm_put(S, HS_XL, a, b, correct_off(hsm_get(S, HS_XL, a, b), tr, pref, pref_f));
            hsm_put(S, HS_XR, a, b, correct_off(hsm_get(S, HS_XR, a, b), tr, pref, pref_f));
        } else {
            const int q = t - NCX;
            const int a = q / HJ + 1, b = q % HJ;
            const int i = i0 - 1 + a, j = j0 - 1 + b;
            if (!(i < nx && j >= -1 && j <= ny)) continue;
            Cons<float> tr;
            tr.rho = (S.u.f.fx[0][a][b] - S.u.f.fx[0][a - 1][b]) * hdx;
            tr.E = (S.u.f.fx[1][a][b] - S.u.f.fx[1][a - 1][b]) * hdx;
            tr.mx = (S.u.f.fx[2][a][b] - S.u.f.fx[2][a - 1][b]) * hdx;
            tr.my = (S.u.f.fx[3][a][b] - S.u.f.fx[3][a - 1][b]) * hdx;
            tr.mz = (S.u.f.fx[4][a][b] - S.u.f.fx[4][a - 1][b]) * hdx;
            tr.Bx = tr.By = tr.Bz = 0.f;
            hsm_put(S, HS_YL, a, b, correct_off(hsm_get(S, HS_YL, a, b), tr, pref, pref_f));
            hsm_put(S, HS_YR, a, b, correct_off(hsm_get(S, HS_YR, a, b), tr, pref, pref_f));
        }
    }
    __syncthreads();

    constexpr int NGX = (TI + 1) * TJ, NGY = TI * (TJ + 1);
    for (int t = threadIdx.x; t < NGX + NGY; t += NT) {
        Cons<float> F;
        if (t < NGX) {
            const int a = t / TJ, b = t % TJ;
            const int i = i0 + a, j = j0 + b;
            if (!(i <= nx && j < ny)) continue;
            if (!face_flux_off<SOLVER, 0>(hsm_get(S, HS_XR, a, b + 1), hsm_get(S, HS_XL, a + 1, b + 1), fdx, eo, F, &st,
                                          pref, pref_f))
                record_error(ctl, ST_FINAL_FLUX, (long long)(i + g) * (ny + 2 * g) + (j + g));
            S.u.f.fx[0][a][b + 1] = F.rho; S.u.f.fx[1][a][b + 1] = F.E; S.u.f.fx[2][a][b + 1] = F.mx;
            S.u.f.fx[3][a][b + 1] = F.my; S.u.f.fx[4][a][b + 1] = F.mz;
        } else {
            const int q = t - NGX;
            const int a = q / (TJ + 1), b = q % (TJ + 1);
            const int i = i0 + a, j = j0 + b;
            if (!(i < nx && j <= ny)) continue;
            if (!face_flux_off<SOLVER, 1>(hsm_get(S, HS_YR, a + 1, b), hsm_get(S, HS_YL, a + 1, b + 1), fdy, eo, F, &st,
                                          pref, pref_f))
                record_error(ctl, ST_FINAL_FLUX, (long long)(i + g) * (ny + 2 * g) + (j + g));
            S.u.f.fy[0][a + 1][b] = F.rho; S.u.f.fy[1][a + 1][b] = F.E; S.u.f.fy[2][a + 1][b] = F.mx;
            S.u.f.fy[3][a + 1][b] = F.my; S.u.f.fy[4][a + 1][b] = F.mz;
        }
    }
    __syncthreads();

    // FP64 conservative accumulation of the FP32 flux differences, FP64 pressure recovery
    double vmax = 0.0;
    for (int t = threadIdx.x; t < TI * TJ; t += NT) {
        const int a = t / TJ, b = t % TJ;
        const int i = i0 + a, j = j0 + b;
        if (!(i < nx && j < ny)) continue;
        const long long m = gidx2(G, i, j);
        Cons<double> U = to_cons64<false>(load_prim<false>(win, PL, m));
        double* u5[5] = {&U.rho, &U.E, &U.mx, &U.my, &U.mz};
#pragma unroll
        for (int f = 0; f < 5; f++) {
            *u5[f] += ((double)S.u.f.fx[f][a][b + 1] - (double)S.u.f.fx[f][a + 1][b + 1]) * dt_dx;
            *u5[f] += ((double)S.u.f.fy[f][a + 1][b] - (double)S.u.f.fy[f][a + 1][b + 1]) * dt_dy;
        }
        const Prim<double> nw = to_prim64<false>(U);
        if (!is_finite<false>(U)) record_error(ctl, ST_NAN, (long long)(i + g) * (ny + 2 * g) + (j + g));
        else if (!is_physical<false>(nw)) record_error(ctl, ST_UNPHYSICAL, (long long)(i + g) * (ny + 2 * g) + (j + g));
        store_prim<false>(wout, PL, m, nw);
        vmax = speed_max(vmax, cfl_speed_mx<false>(nw, sa.cfl, sa.dx, sa.dy, 0.0));
    }
    copy_ghosts_2d<5>(G, win, wout, i0, j0, TI, TJ);

    vmax = block_max(vmax, S.red);
    if (threadIdx.x == 0) atomic_max_speed(&ctl->vmax[sa.slot_out], vmax);
    if (st.pivot_exact) atomicAdd(&S.stat[0], (unsigned long long)st.pivot_exact);
    if (first_order) atomicAdd(&S.stat[5], (unsigned long long)first_order);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (S.stat[0]) atomicAdd(&ctl->pivots_exact, S.stat[0]);
        if (S.stat[5]) atomicAdd(&ctl->muscl_first_order, S.stat[5]);
    }
}

constexpr int kMxTI = kMx2dTI, kMxTJ = kMx2dTJ, kMxNT = 256;

template <int SOLVER>
static int launch_mixed_t(const Geo& G, const double* win, double* wout, StepCtl* ctl, const StepArgs& sa,
                          const CUtensorMap* map, cudaStream_t st) {
    auto kern = k_step2d_hydro_mixed<SOLVER, kMxTI, kMxTJ, kMxNT>;
    const size_t smem = sizeof(SmemMixed<kMxTI, kMxTJ>);
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 1;
        attr = true;
    }
    dim3 grid((G.n[1] + kMxTJ - 1) / kMxTJ, (G.n[0] + kMxTI - 1) / kMxTI);
    kern<<<grid, kMxNT, smem, st>>>(G, win, wout, ctl, sa, *map);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int launch_step2d_hydro_mixed(int solver, const Geo& G, const double* win, double* wout, StepCtl* ctl,
                              const StepArgs& sa, const CUtensorMap* map, cudaStream_t st) {
    switch (solver) {
        case RS_HLLC: return launch_mixed_t<RS_HLLC>(G, win, wout, ctl, sa, map, st);
        case RS_HLL: return launch_mixed_t<RS_HLL>(G, win, wout, ctl, sa, map, st);
        case RS_HLLE: return launch_mixed_t<RS_HLLE>(G, win, wout, ctl, sa, map, st);
        case RS_ROE: return launch_mixed_t<RS_ROE>(G, win, wout, ctl, sa, map, st);
        default: return launch_mixed_t<RS_EXACT>(G, win, wout, ctl, sa, map, st);
    }
}

}  // namespace dgpu
