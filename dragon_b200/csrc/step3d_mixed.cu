// Mixed FP32/FP64 3D CTU hydro step: the five kernels of step3d.cuh
// (Grid3D::unsplit_step hydro branch, Unsplit.cpp:115-206; the 12-solve
// ctu_sweep_hydro, CTU.cpp:222-370) with FP32 reconstruction, limiters,
// transverse corrections and Riemann fluxes, FP32 intermediates (half the
// scratch traffic of the FP64 step), and FP64 where the 2D mixed path keeps
// it: the energy and pressure recovery of every primitive state an FP32
// correction produces (mixed.cuh, prim_from) and the conservative
// accumulation of the flux differences into the FP64 state. Pressures are
// absolute (no per-tile offset: these are flat kernels). Index ranges, the
// order of the corrections and the retry-relevant failure points are those of
// the FP64 step. Compiled with FMA contraction and fast single-precision
// division / square root, like the other mixed translation units.
#include "launchers.h"
#include "mixed.cuh"
#include "step3d.cuh"

namespace dgpu {

namespace {

// The FP64 step's scratch planes read as FP32 planes of the same length.
struct Mx3 {
    float* hs;   // 6 x 5 planes: xL, xR, yL, yR, zL, zR
    float* pf;   // 3 x 5 planes: predictor fluxes, then final fluxes
    float* cf;   // 6 x 5 planes: the six corner-corrected fluxes
    long long plane;
};

__device__ __forceinline__ Prim<float> ldf5(const float* a, long long P, long long m) {
    return Prim<float>{__ldg(a + m), __ldg(a + P + m), __ldg(a + 2 * P + m), __ldg(a + 3 * P + m),
                       __ldg(a + 4 * P + m), 0.f, 0.f, 0.f};
}
__device__ __forceinline__ void stf5(float* a, long long P, long long m, const Prim<float>& w) {
    a[m] = w.rho; a[P + m] = w.p; a[2 * P + m] = w.vx; a[3 * P + m] = w.vy; a[4 * P + m] = w.vz;
}
__device__ __forceinline__ Cons<float> ldcf5(const float* a, long long P, long long m) {
    return Cons<float>{__ldg(a + m), __ldg(a + P + m), __ldg(a + 2 * P + m), __ldg(a + 3 * P + m),
                       __ldg(a + 4 * P + m), 0.f, 0.f, 0.f};
}
__device__ __forceinline__ void stcf5(float* a, long long P, long long m, const Cons<float>& u) {
    a[m] = u.rho; a[P + m] = u.E; a[2 * P + m] = u.mx; a[3 * P + m] = u.my; a[4 * P + m] = u.mz;
}
__device__ __forceinline__ Prim<float> f32_prim(const Prim<double>& w) {
    return Prim<float>{(float)w.rho, (float)w.p, (float)w.vx, (float)w.vy, (float)w.vz, 0.f, 0.f, 0.f};
}

// K1: MUSCL half states along x, y, z for cells [-1, n]^3.
__global__ void __launch_bounds__(256, 3) k_h3m_halfstates(Step3DArgs A, Mx3 X) {
    __shared__ int s;
    if (h3_skip(A.ctl, &s)) return;
    const Geo& G = A.G;
    const int lo[3] = {-1, -1, -1}, ext[3] = {G.n[0] + 2, G.n[1] + 2, G.n[2] + 2};
    int i, j, k;
    if (!box_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, lo, ext, i, j, k)) return;
    const double dt = *(const volatile double*)&A.ctl->t1;
    const float dts[3] = {(float)(dt / A.sa.dx), (float)(dt / A.sa.dy), (float)(dt / A.sa.dz)};
    const long long P = G.plane, SP = X.plane, m = gidx3(G, i, j, k);
    const Prim<float> wc = f32_prim(ld5(A.w, P, m));
    int fo = 0;
#pragma unroll
    for (int ax = 0; ax < 3; ax++) {
        const int di = ax == 0, dj = ax == 1, dk = ax == 2;
        Prim<float> wl = f32_prim(ld5(A.w, P, gidx3(G, i - di, j - dj, k - dk)));
        Prim<float> wr = f32_prim(ld5(A.w, P, gidx3(G, i + di, j + dj, k + dk)));
        Prim<float> c = wc, L, R;
        if (ax == 1) { swap_xy(wl); swap_xy(c); swap_xy(wr); }
        if (ax == 2) { swap_xz(wl); swap_xz(c); swap_xz(wr); }
        fo += !muscl_mixed<false>(A.sa.limiter, wl, L, c, R, wr, dts[ax], 0.f, 0.f, 0.f);
        if (ax == 1) { swap_xy(L); swap_xy(R); }
        if (ax == 2) { swap_xz(L); swap_xz(R); }
        stf5(X.hs + (10 * ax) * SP, SP, m, L);
        stf5(X.hs + (10 * ax + 5) * SP, SP, m, R);
    }
    warp_add_stat(&A.ctl->muscl_first_order, fo);
}

template <int SOLVER, int AX>
__device__ __forceinline__ void h3m_solve(const Step3DArgs& A, const Mx3& X, float* out, long long m,
                                          const Prim<float>& L, const Prim<float>& R, float dtn, int stage,
                                          FaceStats* st) {
    Cons<float> F;
    if (!face_flux_mixed<false, SOLVER, AX>(L, R, dtn, exact_opts(A.sa), F, st)) record_error(A.ctl, stage, m);
    stcf5(out, X.plane, m, F);
}

template <int SOLVER, int AX>
__device__ __forceinline__ void h3m_flux(const Step3DArgs& A, const Mx3& X, float* out, int i, int j, int k, float dtn,
                                         int stage, FaceStats* st) {
    const Geo& G = A.G;
    const long long SP = X.plane;
    const int di = AX == 0, dj = AX == 1, dk = AX == 2;
    const long long m = gidx3(G, i, j, k);
    h3m_solve<SOLVER, AX>(A, X, out, m, ldf5(X.hs + (10 * AX + 5) * SP, SP, gidx3(G, i - di, j - dj, k - dk)),
                          ldf5(X.hs + (10 * AX) * SP, SP, m), dtn, stage, st);
}

// K2: predictor fluxes (CTU.cpp:230-232).
template <int SOLVER>
__global__ void __launch_bounds__(256, 3) k_h3m_prelim(Step3DArgs A, Mx3 X) {
    __shared__ int s;
    if (h3_skip(A.ctl, &s)) return;
    const Geo& G = A.G;
    const int lo[3] = {-1, -1, -1}, ext[3] = {G.n[0] + 2, G.n[1] + 2, G.n[2] + 2};
    int i, j, k;
    if (!box_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, lo, ext, i, j, k)) return;
    const double dt = *(const volatile double*)&A.ctl->t1;
    FaceStats st{0, 0, 0, 0, 0};
    const long long SP = X.plane;
    if (i >= 0) h3m_flux<SOLVER, 0>(A, X, X.pf, i, j, k, (float)(dt / A.sa.dx), ST_PRELIM_FLUX, &st);
    if (j >= 0) h3m_flux<SOLVER, 1>(A, X, X.pf + 5 * SP, i, j, k, (float)(dt / A.sa.dy), ST_PRELIM_FLUX, &st);
    if (k >= 0) h3m_flux<SOLVER, 2>(A, X, X.pf + 10 * SP, i, j, k, (float)(dt / A.sa.dz), ST_PRELIM_FLUX, &st);
    h3_stats(A.ctl, st);
}

// One corner-corrected flux (computeCTUFlux_*, CTU.cpp:306-370).
template <int SOLVER, int AX, int TD>
__device__ __forceinline__ void h3m_ctu_flux(const Step3DArgs& A, const Mx3& X, const float* T, float* out, int i,
                                             int j, int k, float dtn, float dtT, FaceStats* st) {
    const Geo& G = A.G;
    const long long SP = X.plane;
    const int di = AX == 0, dj = AX == 1, dk = AX == 2;
    const int ti = TD == 0, tj = TD == 1, tk = TD == 2;
    auto trans = [&](int a, int b, int c) {
        return c_mul<false>(c_sub<false>(ldcf5(T, SP, gidx3(G, a + ti, b + tj, c + tk)), ldcf5(T, SP, gidx3(G, a, b, c))),
                            dtT);
    };
    const long long m = gidx3(G, i, j, k);
    const Prim<float> L = correct_mixed<false>(ldf5(X.hs + (10 * AX + 5) * SP, SP, gidx3(G, i - di, j - dj, k - dk)),
                                               trans(i - di, j - dj, k - dk));
    const Prim<float> R = correct_mixed<false>(ldf5(X.hs + (10 * AX) * SP, SP, m), trans(i, j, k));
    h3m_solve<SOLVER, AX>(A, X, out, m, L, R, dtn, ST_PRELIM_FLUX, st);
}

// K3: the six corner-corrected fluxes over the reference's ranges.
template <int SOLVER>
__global__ void __launch_bounds__(256, 3) k_h3m_ctu(Step3DArgs A, Mx3 X) {
    __shared__ int s;
    if (h3_skip(A.ctl, &s)) return;
    const Geo& G = A.G;
    const int lo[3] = {-1, -1, -1}, ext[3] = {G.n[0] + 2, G.n[1] + 2, G.n[2] + 2};
    int i, j, k;
    if (!box_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, lo, ext, i, j, k)) return;
    const int nx = G.n[0], ny = G.n[1], nz = G.n[2];
    const double dt = *(const volatile double*)&A.ctl->t1;
    const double dt_dx = dt / A.sa.dx, dt_dy = dt / A.sa.dy, dt_dz = dt / A.sa.dz;
    const float fx = (float)dt_dx, fy = (float)dt_dy, fz = (float)dt_dz;
    const float tx = (float)(dt_dx / 3.0), ty = (float)(dt_dy / 3.0), tz = (float)(dt_dz / 3.0);
    const long long SP = X.plane;
    const float* FX = X.pf;
    const float* FY = X.pf + 5 * SP;
    const float* FZ = X.pf + 10 * SP;
    FaceStats st{0, 0, 0, 0, 0};
    if (i >= 0 && k >= 0 && k < nz) h3m_ctu_flux<SOLVER, 0, 2>(A, X, FZ, X.cf, i, j, k, fx, tz, &st);
    if (j >= 0 && k >= 0 && k < nz) h3m_ctu_flux<SOLVER, 1, 2>(A, X, FZ, X.cf + 5 * SP, i, j, k, fy, tz, &st);
    if (i >= 0 && j >= 0 && j < ny) h3m_ctu_flux<SOLVER, 0, 1>(A, X, FY, X.cf + 10 * SP, i, j, k, fx, ty, &st);
    if (j >= 0 && j < ny && k >= 0) h3m_ctu_flux<SOLVER, 2, 1>(A, X, FY, X.cf + 15 * SP, i, j, k, fz, ty, &st);
    if (i >= 0 && i < nx && j >= 0) h3m_ctu_flux<SOLVER, 1, 0>(A, X, FX, X.cf + 20 * SP, i, j, k, fy, tx, &st);
    if (i >= 0 && i < nx && k >= 0) h3m_ctu_flux<SOLVER, 2, 0>(A, X, FX, X.cf + 25 * SP, i, j, k, fz, tx, &st);
    h3_stats(A.ctl, st);
}

// One transverse correction U - (F(m + e_D) - F(m)) * w with the energy in FP64.
template <int D>
__device__ __forceinline__ Prim<float> h3m_corrected_once(const Step3DArgs& A, const Mx3& X, const Prim<float>& s,
                                                          const float* F, float w, int i, int j, int k) {
    const Geo& G = A.G;
    const long long SP = X.plane;
    const Cons<float> tr = c_mul<false>(
        c_sub<false>(ldcf5(F, SP, gidx3(G, i + (D == 0), j + (D == 1), k + (D == 2))), ldcf5(F, SP, gidx3(G, i, j, k))),
        w);
    return correct_mixed<false>(s, tr);
}

// The corrected half state of a cell along AX (SIDE 0: low face, 1: high),
// the two sequential corrections of correctState (CTU.cpp:246-260).
template <int AX, int SIDE>
__device__ __forceinline__ Prim<float> h3m_corrected(const Step3DArgs& A, const Mx3& X, const float h[3], int i, int j,
                                                     int k) {
    const long long SP = X.plane;
    const float* cf = X.cf;
    Prim<float> s = ldf5(X.hs + (10 * AX + 5 * SIDE) * SP, SP, gidx3(A.G, i, j, k));
    if constexpr (AX == 0) {
        s = h3m_corrected_once<1>(A, X, s, cf + 5 * SP, h[1], i, j, k);    // F_Yz
        s = h3m_corrected_once<2>(A, X, s, cf + 15 * SP, h[2], i, j, k);   // F_Zy
    } else if constexpr (AX == 1) {
        s = h3m_corrected_once<0>(A, X, s, cf, h[0], i, j, k);             // F_Xz
        s = h3m_corrected_once<2>(A, X, s, cf + 25 * SP, h[2], i, j, k);   // F_Zx
    } else {
        s = h3m_corrected_once<0>(A, X, s, cf + 10 * SP, h[0], i, j, k);   // F_Xy
        s = h3m_corrected_once<1>(A, X, s, cf + 20 * SP, h[1], i, j, k);   // F_Yx
    }
    return s;
}

template <int SOLVER, int AX>
__device__ __forceinline__ void h3m_final_flux(const Step3DArgs& A, const Mx3& X, const float h[3], int i, int j,
                                               int k, float dtn, FaceStats* st) {
    const int di = AX == 0, dj = AX == 1, dk = AX == 2;
    const long long m = gidx3(A.G, i, j, k);
    h3m_solve<SOLVER, AX>(A, X, X.pf + 5 * AX * X.plane, m, h3m_corrected<AX, 1>(A, X, h, i - di, j - dj, k - dk),
                          h3m_corrected<AX, 0>(A, X, h, i, j, k), dtn, ST_FINAL_FLUX, st);
}

// K4: final fluxes from the corrected half states.
template <int SOLVER>
__global__ void __launch_bounds__(256, 3) k_h3m_final(Step3DArgs A, Mx3 X) {
    __shared__ int s;
    if (h3_skip(A.ctl, &s)) return;
    const Geo& G = A.G;
    const int lo[3] = {0, 0, 0}, ext[3] = {G.n[0] + 1, G.n[1] + 1, G.n[2] + 1};
    int i, j, k;
    if (!box_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, lo, ext, i, j, k)) return;
    const int nx = G.n[0], ny = G.n[1], nz = G.n[2];
    const double dt = *(const volatile double*)&A.ctl->t1;
    const float h[3] = {(float)(0.5 * (dt / A.sa.dx)), (float)(0.5 * (dt / A.sa.dy)), (float)(0.5 * (dt / A.sa.dz))};
    FaceStats st{0, 0, 0, 0, 0};
    if (j < ny && k < nz) h3m_final_flux<SOLVER, 0>(A, X, h, i, j, k, (float)(dt / A.sa.dx), &st);
    if (i < nx && k < nz) h3m_final_flux<SOLVER, 1>(A, X, h, i, j, k, (float)(dt / A.sa.dy), &st);
    if (i < nx && j < ny) h3m_final_flux<SOLVER, 2>(A, X, h, i, j, k, (float)(dt / A.sa.dz), &st);
    h3_stats(A.ctl, st);
}

// K5: FP64 accumulation of the FP32 flux differences into the FP64 state,
// FP64 pressure recovery, physicality, CFL speed of the committed state.
__global__ void __launch_bounds__(256) k_h3m_update(Step3DArgs A, Mx3 X) {
    __shared__ int s;
    __shared__ double red[32];
    if (h3_skip(A.ctl, &s)) return;
    const Geo& G = A.G;
    const int lo[3] = {0, 0, 0}, ext[3] = {G.n[0], G.n[1], G.n[2]};
    int i, j, k;
    double vmax = 0.0;
    if (box_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, lo, ext, i, j, k)) {
        const double dt = *(const volatile double*)&A.ctl->t1;
        const double d[3] = {dt / A.sa.dx, dt / A.sa.dy, dt / A.sa.dz};
        const long long P = G.plane, SP = X.plane, m = gidx3(G, i, j, k);
        Cons<double> U = to_cons64<false>(ld5(A.w, P, m));
        const long long up[3] = {gidx3(G, i + 1, j, k), gidx3(G, i, j + 1, k), gidx3(G, i, j, k + 1)};
        double* u5[5] = {&U.rho, &U.E, &U.mx, &U.my, &U.mz};
#pragma unroll
        for (int ax = 0; ax < 3; ax++) {
            const float* F = X.pf + 5 * ax * SP;
#pragma unroll
            for (int f = 0; f < 5; f++)
                *u5[f] += ((double)__ldg(F + f * SP + m) - (double)__ldg(F + f * SP + up[ax])) * d[ax];
        }
        const Prim<double> nw = to_prim64<false>(U);
        if (!is_finite<false>(U)) record_error(A.ctl, ST_NAN, m);
        else if (!is_physical<false>(nw)) record_error(A.ctl, ST_UNPHYSICAL, m);
        st5(A.wout, P, m, nw);
        vmax = cfl_speed_mx<false>(nw, A.sa.cfl, A.sa.dx, A.sa.dy, A.sa.dz);
    }
    vmax = block_max(vmax, red);
    if (threadIdx.x == 0) atomic_max_speed(&A.ctl->vmax[A.sa.slot_out], vmax);
}

template <int SOLVER>
int go(const Geo& G, const double* w, double* wout, const Hydro3DScratch& S, StepCtl* ctl, const StepArgs& sa,
       cudaStream_t st) {
    Step3DArgs A{G, w, wout, S, ctl, sa};
    const Mx3 X{reinterpret_cast<float*>(S.hs), reinterpret_cast<float*>(S.pf), reinterpret_cast<float*>(S.cf),
                S.plane};
    auto blocks = [](long long n) { return (int)((n + 255) / 256); };
    const long long box = (long long)(G.n[0] + 2) * (G.n[1] + 2) * (G.n[2] + 2);
    const long long fbox = (long long)(G.n[0] + 1) * (G.n[1] + 1) * (G.n[2] + 1);
    const long long cells = (long long)G.n[0] * G.n[1] * G.n[2];
    if (cudaMemcpyAsync(wout, w, sizeof(double) * 5 * G.plane, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return 1;
    k_h3m_halfstates<<<blocks(box), 256, 0, st>>>(A, X);
    k_h3m_prelim<SOLVER><<<blocks(box), 256, 0, st>>>(A, X);
    k_h3m_ctu<SOLVER><<<blocks(box), 256, 0, st>>>(A, X);
    k_h3m_final<SOLVER><<<blocks(fbox), 256, 0, st>>>(A, X);
    k_h3m_update<<<blocks(cells), 256, 0, st>>>(A, X);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace

int launch_step3d_hydro_mixed(int solver, const Geo& G, const double* w, double* wout, const Hydro3DScratch& S,
                              StepCtl* ctl, const StepArgs& sa, cudaStream_t st) {
    switch (solver) {
        case RS_HLL: return go<RS_HLL>(G, w, wout, S, ctl, sa, st);
        case RS_HLLE: return go<RS_HLLE>(G, w, wout, S, ctl, sa, st);
        case RS_ROE: return go<RS_ROE>(G, w, wout, S, ctl, sa, st);
        case RS_EXACT: return go<RS_EXACT>(G, w, wout, S, ctl, sa, st);
        default: return go<RS_HLLC>(G, w, wout, S, ctl, sa, st);
    }
}

}  // namespace dgpu
