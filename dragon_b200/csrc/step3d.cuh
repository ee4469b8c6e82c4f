// 3D unsplit CTU hydro step (Grid3D::unsplit_step hydro branch,
// Unsplit.cpp:115-206; the 12-solve ctu_sweep_hydro, CTU.cpp:222-370) as
// five kernels over global intermediates:
//   K1 half states along x, y, z for cells [-1, n]^3
//   K2 predictor fluxes (CTU.cpp:229-232)
//   K3 the six corner-corrected fluxes F_Xz, F_Yz, F_Xy, F_Zy, F_Yx, F_Zx
//      (computeCTUFlux_X/Y/Z, CTU.cpp:306-370; dt/3 transverse weights)
//   K4 final fluxes (Unsplit.cpp:102-105) from the half states with their two
//      sequential transverse corrections (correctState, CTU.cpp:246-260,
//      280-301) applied where the face reads them, not written back
//   K5 conservative update, physicality, CFL speed
// Index ranges are the reference's, so every Riemann pivot that can fail does.
#pragma once

#include "grid.cuh"
#include "mlp.cuh"
#include "recon.cuh"
#include "riemann.cuh"
#include "scratch.h"

namespace dgpu {

struct Step3DArgs {
    Geo G;
    const double* w;
    double* wout;
    Hydro3DScratch S;
    StepCtl* ctl;
    StepArgs sa;
};

__device__ __forceinline__ bool h3_skip(const StepCtl* ctl, int* s) {
    if (threadIdx.x == 0) *s = (*(const volatile int*)&ctl->err) | (*(const volatile int*)&ctl->done);
    __syncthreads();
    return *s != 0;
}

// cell of a flat launch over the box [lo, lo + ext) per axis, last index fastest
__device__ __forceinline__ bool box_cell(long long t, const int* lo, const int* ext, int& i, int& j, int& k) {
    const long long ek = ext[2], ej = ext[1];
    if (t >= (long long)ext[0] * ej * ek) return false;
    k = lo[2] + (int)(t % ek);
    j = lo[1] + (int)((t / ek) % ej);
    i = lo[0] + (int)(t / (ek * ej));
    return true;
}

// Every array a kernel of this step reads is one it does not write (state ->
// half states -> predictor fluxes -> corner fluxes -> final fluxes -> new
// state), so the loads go through the read-only path: the compiler may then
// issue a later face's loads before an earlier face's stores.
__device__ __forceinline__ Prim<double> ld5(const double* a, long long P, long long m) {
    Prim<double> r;
    r.rho = __ldg(a + m);
    r.p = __ldg(a + P + m);
    r.vx = __ldg(a + 2 * P + m);
    r.vy = __ldg(a + 3 * P + m);
    r.vz = __ldg(a + 4 * P + m);
    r.Bx = r.By = r.Bz = 0;
    return r;
}
__device__ __forceinline__ void st5(double* a, long long P, long long m, const Prim<double>& w) { store_prim<false>(a, P, m, w); }
__device__ __forceinline__ Cons<double> ldc5(const double* a, long long P, long long m) {
    return Cons<double>{__ldg(a + m), __ldg(a + P + m), __ldg(a + 2 * P + m), __ldg(a + 3 * P + m), __ldg(a + 4 * P + m),
                        0, 0, 0};
}
__device__ __forceinline__ void stc5(double* a, long long P, long long m, const Cons<double>& u) {
    a[m] = u.rho; a[P + m] = u.E; a[2 * P + m] = u.mx; a[3 * P + m] = u.my; a[4 * P + m] = u.mz;
}

// K1: MUSCL half states along all three axes (computeHalfStates_X/Y/Z, Unsplit.cpp:344-436).
static __global__ void k_h3_halfstates(Step3DArgs A) {
    __shared__ int s;
    if (h3_skip(A.ctl, &s)) return;
    const Geo& G = A.G;
    const int lo[3] = {-1, -1, -1}, ext[3] = {G.n[0] + 2, G.n[1] + 2, G.n[2] + 2};
    int i, j, k;
    if (!box_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, lo, ext, i, j, k)) return;
    const double dt = *(const volatile double*)&A.ctl->t1;
    const double dts[3] = {dt / A.sa.dx, dt / A.sa.dy, dt / A.sa.dz};
    const long long P = G.plane, m = gidx3(G, i, j, k);
    const Prim<double> wc = ld5(A.w, P, m);
    int fo = 0;
#pragma unroll
    for (int ax = 0; ax < 3; ax++) {
        const int di = ax == 0, dj = ax == 1, dk = ax == 2;
        Prim<double> wl = ld5(A.w, P, gidx3(G, i - di, j - dj, k - dk));
        Prim<double> wr = ld5(A.w, P, gidx3(G, i + di, j + dj, k + dk));
        Prim<double> c = wc, L, R;
        if (ax == 1) { swap_xy(wl); swap_xy(c); swap_xy(wr); }
        if (ax == 2) { swap_xz(wl); swap_xz(c); swap_xz(wr); }
        fo += !muscl<false>(A.sa.limiter, wl, L, c, R, wr, dts[ax], 0.0, 0.0, 0.0);
        if (ax == 1) { swap_xy(L); swap_xy(R); }
        if (ax == 2) { swap_xz(L); swap_xz(R); }
        st5(A.S.hs + (10 * ax) * A.S.plane, A.S.plane, m, L);
        st5(A.S.hs + (10 * ax + 5) * A.S.plane, A.S.plane, m, R);
    }
    warp_add_stat(&A.ctl->muscl_first_order, fo);
}

template <int SOLVER, int AX>
__device__ __forceinline__ void h3_flux(const Step3DArgs& A, double* out, int i, int j, int k, double dtn,
                                        int stage, FaceStats* st) {
    const Geo& G = A.G;
    const long long SP = A.S.plane;
    const int di = AX == 0, dj = AX == 1, dk = AX == 2;
    const long long m = gidx3(G, i, j, k);
    Prim<double> L = ld5(A.S.hs + (10 * AX + 5) * SP, SP, gidx3(G, i - di, j - dj, k - dk));
    Prim<double> R = ld5(A.S.hs + (10 * AX) * SP, SP, m);
    Cons<double> F;
    const ExactOpts eo = exact_opts(A.sa);
    if (!face_flux<false, SOLVER, AX>(L, R, dtn, eo, F, st)) record_error(A.ctl, stage, m);
    stc5(out, SP, m, F);
}

// Weights of the two transverse corrections of the half states along AX, in
// the reference's order (CTU.cpp:246-260): x states by F_Yz (dt/2dy) then
// F_Zy (dt/2dz); y states by F_Xz then F_Zx; z states by F_Xy then F_Yx.
struct H3Half {
    double hx, hy, hz;
};

// One transverse correction of a half state at cell m: U - (F(m + e_D) - F(m)) * w.
template <int D>
__device__ __forceinline__ Prim<double> h3_corrected_once(const Step3DArgs& A, const Prim<double>& s, const double* F,
                                                          double w, int i, int j, int k) {
    const Geo& G = A.G;
    const long long SP = A.S.plane;
    const Cons<double> tr = c_mul<false>(
        c_sub<false>(ldc5(F, SP, gidx3(G, i + (D == 0), j + (D == 1), k + (D == 2))), ldc5(F, SP, gidx3(G, i, j, k))), w);
    return to_prim<false>(c_sub<false>(to_cons<false>(s), tr));
}

// The corrected half state of cell (i,j,k) along AX (SIDE 0: the state at the
// cell's low face, 1: at its high face), computed where the final flux needs
// it instead of written back by a separate pass: the same two sequential
// corrections with the same operands, so the value is bit-identical.
template <int AX, int SIDE>
__device__ __forceinline__ Prim<double> h3_corrected(const Step3DArgs& A, const H3Half& h, int i, int j, int k) {
    const long long SP = A.S.plane;
    const double* cf = A.S.cf;
    Prim<double> s = ld5(A.S.hs + (10 * AX + 5 * SIDE) * SP, SP, gidx3(A.G, i, j, k));
    if constexpr (AX == 0) {
        s = h3_corrected_once<1>(A, s, cf + 5 * SP, h.hy, i, j, k);    // F_Yz
        s = h3_corrected_once<2>(A, s, cf + 15 * SP, h.hz, i, j, k);   // F_Zy
    } else if constexpr (AX == 1) {
        s = h3_corrected_once<0>(A, s, cf, h.hx, i, j, k);             // F_Xz
        s = h3_corrected_once<2>(A, s, cf + 25 * SP, h.hz, i, j, k);   // F_Zx
    } else {
        s = h3_corrected_once<0>(A, s, cf + 10 * SP, h.hx, i, j, k);   // F_Xy
        s = h3_corrected_once<1>(A, s, cf + 20 * SP, h.hy, i, j, k);   // F_Yx
    }
    return s;
}

// Final flux through the AX face of cell (i,j,k) from the corrected states of
// the cells on either side.
template <int SOLVER, int AX>
__device__ __forceinline__ void h3_final_flux(const Step3DArgs& A, const H3Half& h, int i, int j, int k, double dtn,
                                              FaceStats* st) {
    const long long SP = A.S.plane;
    const int di = AX == 0, dj = AX == 1, dk = AX == 2;
    const long long m = gidx3(A.G, i, j, k);
    const Prim<double> L = h3_corrected<AX, 1>(A, h, i - di, j - dj, k - dk);
    const Prim<double> R = h3_corrected<AX, 0>(A, h, i, j, k);
    Cons<double> F;
    if (!face_flux<false, SOLVER, AX>(L, R, dtn, exact_opts(A.sa), F, st)) record_error(A.ctl, ST_FINAL_FLUX, m);
    stc5(A.S.pf + 5 * AX * SP, SP, m, F);
}

__device__ __forceinline__ H3Half h3_half(const Step3DArgs& A, double dt) {
    return H3Half{0.5 * (dt / A.sa.dx), 0.5 * (dt / A.sa.dy), 0.5 * (dt / A.sa.dz)};
}

__device__ __forceinline__ void h3_stats(StepCtl* ctl, const FaceStats& st) {
    warp_add_stat(&ctl->pivots_exact, st.pivot_exact);
    warp_add_stat(&ctl->newton_iters, st.newton_iters);
    warp_add_stat(&ctl->exact_calls, st.exact_calls);
    warp_add_stat(&ctl->trrs, st.trrs);
    warp_add_stat(&ctl->cap_hits, st.cap_hits);
    warp_add_stat(&ctl->guess_rejects, st.guess_rejects);
    warp_add_stat(&ctl->judge_reruns, st.judge_reruns);
}

// ---------------------------------------------------------------------------
// Learned-guess variants of the three flux kernels (exact solver only). The
// network runs as a warp collective on the tensor cores, so these kernels
// keep every lane of a warp converged up to the inference: lanes without a
// face carry a neutral state instead of returning early, and the solve that
// follows is predicated on the face being real.

__device__ __forceinline__ Prim<double> neutral_state() {
    Prim<double> w = zero_prim<double>();
    w.rho = 1.0;
    w.p = 1.0;
    return w;
}

template <int AX>
__device__ __forceinline__ LearnedGuess<double> learned_guess_face(const Step3DArgs& A, const Prim<double>& L,
                                                                   const Prim<double>& R, bool valid) {
    Prim<double> Ln = L, Rn = R;
    swap_axis<AX>(Ln);
    swap_axis<AX>(Rn);
    return mlp_guess_warp(A.sa.mlp, Ln, Rn, valid);
}

template <int AX>
__device__ __forceinline__ void h3_flux_learned(const Step3DArgs& A, double* out, bool valid, int i, int j, int k,
                                                double dtn, int stage, FaceStats* st) {
    const Geo& G = A.G;
    const long long SP = A.S.plane;
    const int di = AX == 0, dj = AX == 1, dk = AX == 2;
    Prim<double> L = neutral_state(), R = neutral_state();
    long long m = 0;
    if (valid) {
        m = gidx3(G, i, j, k);
        L = ld5(A.S.hs + (10 * AX + 5) * SP, SP, gidx3(G, i - di, j - dj, k - dk));
        R = ld5(A.S.hs + (10 * AX) * SP, SP, m);
    }
    const LearnedGuess<double> g = learned_guess_face<AX>(A, L, R, valid);
    if (!valid) return;
    Cons<double> F;
    if (!face_flux<false, RS_EXACT, AX>(L, R, dtn, exact_opts(A.sa), F, st, &g)) record_error(A.ctl, stage, m);
    stc5(out, SP, m, F);
}

template <int AX, int TD>
__device__ __forceinline__ void h3_ctu_flux_learned(const Step3DArgs& A, const double* T, double* out, bool valid,
                                                    int i, int j, int k, double dtn, double dtT, FaceStats* st) {
    const Geo& G = A.G;
    const long long SP = A.S.plane;
    const int di = AX == 0, dj = AX == 1, dk = AX == 2;
    const int ti = TD == 0, tj = TD == 1, tk = TD == 2;
    Prim<double> L = neutral_state(), R = neutral_state();
    long long m = 0;
    if (valid) {
        auto trans = [&](int a, int b, int c) {
            const Cons<double> t1 = ldc5(T, SP, gidx3(G, a + ti, b + tj, c + tk)), t0 = ldc5(T, SP, gidx3(G, a, b, c));
            return c_mul<false>(c_sub<false>(t1, t0), dtT);
        };
        m = gidx3(G, i, j, k);
        L = to_prim<false>(c_sub<false>(to_cons<false>(ld5(A.S.hs + (10 * AX + 5) * SP, SP, gidx3(G, i - di, j - dj, k - dk))),
                                        trans(i - di, j - dj, k - dk)));
        R = to_prim<false>(c_sub<false>(to_cons<false>(ld5(A.S.hs + (10 * AX) * SP, SP, m)), trans(i, j, k)));
    }
    const LearnedGuess<double> g = learned_guess_face<AX>(A, L, R, valid);
    if (!valid) return;
    Cons<double> F;
    if (!face_flux<false, RS_EXACT, AX>(L, R, dtn, exact_opts(A.sa), F, st, &g))
        record_error(A.ctl, ST_PRELIM_FLUX, m);
    stc5(out, SP, m, F);
}

static __global__ void k_h3_prelim_learned(Step3DArgs A) {
    __shared__ int s;
    if (h3_skip(A.ctl, &s)) return;
    const Geo& G = A.G;
    const int lo[3] = {-1, -1, -1}, ext[3] = {G.n[0] + 2, G.n[1] + 2, G.n[2] + 2};
    int i = 0, j = 0, k = 0;
    const bool in = box_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, lo, ext, i, j, k);
    const double dt = *(const volatile double*)&A.ctl->t1;
    FaceStats st{};
    const long long SP = A.S.plane;
    h3_flux_learned<0>(A, A.S.pf, in && i >= 0, i, j, k, dt / A.sa.dx, ST_PRELIM_FLUX, &st);
    h3_flux_learned<1>(A, A.S.pf + 5 * SP, in && j >= 0, i, j, k, dt / A.sa.dy, ST_PRELIM_FLUX, &st);
    h3_flux_learned<2>(A, A.S.pf + 10 * SP, in && k >= 0, i, j, k, dt / A.sa.dz, ST_PRELIM_FLUX, &st);
    h3_stats(A.ctl, st);
}

static __global__ void k_h3_ctu_learned(Step3DArgs A) {
    __shared__ int s;
    if (h3_skip(A.ctl, &s)) return;
    const Geo& G = A.G;
    const int lo[3] = {-1, -1, -1}, ext[3] = {G.n[0] + 2, G.n[1] + 2, G.n[2] + 2};
    int i = 0, j = 0, k = 0;
    const bool in = box_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, lo, ext, i, j, k);
    const int nx = G.n[0], ny = G.n[1], nz = G.n[2];
    const double dt = *(const volatile double*)&A.ctl->t1;
    const double dt_dx = dt / A.sa.dx, dt_dy = dt / A.sa.dy, dt_dz = dt / A.sa.dz;
    const long long SP = A.S.plane;
    const double* FX = A.S.pf;
    const double* FY = A.S.pf + 5 * SP;
    const double* FZ = A.S.pf + 10 * SP;
    FaceStats st{};
    h3_ctu_flux_learned<0, 2>(A, FZ, A.S.cf, in && i >= 0 && k >= 0 && k < nz, i, j, k, dt_dx, dt_dz / 3.0, &st);
    h3_ctu_flux_learned<1, 2>(A, FZ, A.S.cf + 5 * SP, in && j >= 0 && k >= 0 && k < nz, i, j, k, dt_dy, dt_dz / 3.0, &st);
    h3_ctu_flux_learned<0, 1>(A, FY, A.S.cf + 10 * SP, in && i >= 0 && j >= 0 && j < ny, i, j, k, dt_dx, dt_dy / 3.0, &st);
    h3_ctu_flux_learned<2, 1>(A, FY, A.S.cf + 15 * SP, in && j >= 0 && j < ny && k >= 0, i, j, k, dt_dz, dt_dy / 3.0, &st);
    h3_ctu_flux_learned<1, 0>(A, FX, A.S.cf + 20 * SP, in && i >= 0 && i < nx && j >= 0, i, j, k, dt_dy, dt_dx / 3.0, &st);
    h3_ctu_flux_learned<2, 0>(A, FX, A.S.cf + 25 * SP, in && i >= 0 && i < nx && k >= 0, i, j, k, dt_dz, dt_dx / 3.0, &st);
    h3_stats(A.ctl, st);
}

template <int AX>
__device__ __forceinline__ void h3_final_flux_learned(const Step3DArgs& A, const H3Half& h, bool valid, int i, int j,
                                                      int k, double dtn, FaceStats* st) {
    const int di = AX == 0, dj = AX == 1, dk = AX == 2;
    Prim<double> L = neutral_state(), R = neutral_state();
    long long m = 0;
    if (valid) {
        m = gidx3(A.G, i, j, k);
        L = h3_corrected<AX, 1>(A, h, i - di, j - dj, k - dk);
        R = h3_corrected<AX, 0>(A, h, i, j, k);
    }
    const LearnedGuess<double> g = learned_guess_face<AX>(A, L, R, valid);
    if (!valid) return;
    Cons<double> F;
    if (!face_flux<false, RS_EXACT, AX>(L, R, dtn, exact_opts(A.sa), F, st, &g)) record_error(A.ctl, ST_FINAL_FLUX, m);
    stc5(A.S.pf + 5 * AX * A.S.plane, A.S.plane, m, F);
}

static __global__ void k_h3_final_learned(Step3DArgs A) {
    __shared__ int s;
    if (h3_skip(A.ctl, &s)) return;
    const Geo& G = A.G;
    const int lo[3] = {0, 0, 0}, ext[3] = {G.n[0] + 1, G.n[1] + 1, G.n[2] + 1};
    int i = 0, j = 0, k = 0;
    const bool in = box_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, lo, ext, i, j, k);
    const int nx = G.n[0], ny = G.n[1], nz = G.n[2];
    const double dt = *(const volatile double*)&A.ctl->t1;
    const H3Half h = h3_half(A, dt);
    FaceStats st{};
    h3_final_flux_learned<0>(A, h, in && j < ny && k < nz, i, j, k, dt / A.sa.dx, &st);
    h3_final_flux_learned<1>(A, h, in && i < nx && k < nz, i, j, k, dt / A.sa.dy, &st);
    h3_final_flux_learned<2>(A, h, in && i < nx && j < ny, i, j, k, dt / A.sa.dz, &st);
    h3_stats(A.ctl, st);
}

// K2: predictor fluxes F_X on [0,nx]x[-1,ny]x[-1,nz], F_Y on [-1,nx]x[0,ny]x[-1,nz],
// F_Z on [-1,nx]x[-1,ny]x[0,nz] (CTU.cpp:230-232).
// Two CTAs per SM for every solver: the Roe instantiations use 136-148
// registers unbounded (one CTA per SM) and ran 33 % faster capped at 128.
template <int SOLVER>
__global__ void __launch_bounds__(256, 2) k_h3_prelim(Step3DArgs A) {
    __shared__ int s;
    if (h3_skip(A.ctl, &s)) return;
    const Geo& G = A.G;
    const int lo[3] = {-1, -1, -1}, ext[3] = {G.n[0] + 2, G.n[1] + 2, G.n[2] + 2};
    int i, j, k;
    if (!box_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, lo, ext, i, j, k)) return;
    const double dt = *(const volatile double*)&A.ctl->t1;
    FaceStats st{0, 0, 0, 0, 0};
    const long long SP = A.S.plane;
    if (i >= 0) h3_flux<SOLVER, 0>(A, A.S.pf, i, j, k, dt / A.sa.dx, ST_PRELIM_FLUX, &st);
    if (j >= 0) h3_flux<SOLVER, 1>(A, A.S.pf + 5 * SP, i, j, k, dt / A.sa.dy, ST_PRELIM_FLUX, &st);
    if (k >= 0) h3_flux<SOLVER, 2>(A, A.S.pf + 10 * SP, i, j, k, dt / A.sa.dz, ST_PRELIM_FLUX, &st);
    h3_stats(A.ctl, st);
}

// One corner-corrected flux (computeCTUFlux_*, CTU.cpp:306-370): the half
// states on both sides of face q along AX are corrected by the transverse
// predictor flux T along TD with weight dtT, then solved along AX.
template <int SOLVER, int AX, int TD>
__device__ __forceinline__ void h3_ctu_flux(const Step3DArgs& A, const double* T, double* out, int i, int j, int k,
                                            double dtn, double dtT, FaceStats* st) {
    const Geo& G = A.G;
    const long long SP = A.S.plane;
    const int di = AX == 0, dj = AX == 1, dk = AX == 2;
    const int ti = TD == 0, tj = TD == 1, tk = TD == 2;
    auto trans = [&](int a, int b, int c) {
        const Cons<double> t1 = ldc5(T, SP, gidx3(G, a + ti, b + tj, c + tk)), t0 = ldc5(T, SP, gidx3(G, a, b, c));
        return c_mul<false>(c_sub<false>(t1, t0), dtT);
    };
    const Prim<double> L = to_prim<false>(c_sub<false>(
        to_cons<false>(ld5(A.S.hs + (10 * AX + 5) * SP, SP, gidx3(G, i - di, j - dj, k - dk))), trans(i - di, j - dj, k - dk)));
    const long long m = gidx3(G, i, j, k);
    const Prim<double> R = to_prim<false>(c_sub<false>(to_cons<false>(ld5(A.S.hs + (10 * AX) * SP, SP, m)), trans(i, j, k)));
    Cons<double> F;
    const ExactOpts eo = exact_opts(A.sa);
    if (!face_flux<false, SOLVER, AX>(L, R, dtn, eo, F, st)) record_error(A.ctl, ST_PRELIM_FLUX, m);
    stc5(out, SP, m, F);
}

// K3: the six corner-corrected fluxes over the reference's ranges: on the
// normal axis faces [0, n]; on the transverse-flux axis cells [0, n); on the
// third axis cells [-1, n].
template <int SOLVER>
__global__ void __launch_bounds__(256, 2) k_h3_ctu(Step3DArgs A) {
    __shared__ int s;
    if (h3_skip(A.ctl, &s)) return;
    const Geo& G = A.G;
    const int lo[3] = {-1, -1, -1}, ext[3] = {G.n[0] + 2, G.n[1] + 2, G.n[2] + 2};
    int i, j, k;
    if (!box_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, lo, ext, i, j, k)) return;
    const int nx = G.n[0], ny = G.n[1], nz = G.n[2];
    const double dt = *(const volatile double*)&A.ctl->t1;
    const double dt_dx = dt / A.sa.dx, dt_dy = dt / A.sa.dy, dt_dz = dt / A.sa.dz;
    const long long SP = A.S.plane;
    const double* FX = A.S.pf;
    const double* FY = A.S.pf + 5 * SP;
    const double* FZ = A.S.pf + 10 * SP;
    FaceStats st{0, 0, 0, 0, 0};
    // F_Xz: i in [0,nx], j in [-1,ny], k in [0,nz)
    if (i >= 0 && k >= 0 && k < nz) h3_ctu_flux<SOLVER, 0, 2>(A, FZ, A.S.cf, i, j, k, dt_dx, dt_dz / 3.0, &st);
    // F_Yz: i in [-1,nx], j in [0,ny], k in [0,nz)
    if (j >= 0 && k >= 0 && k < nz) h3_ctu_flux<SOLVER, 1, 2>(A, FZ, A.S.cf + 5 * SP, i, j, k, dt_dy, dt_dz / 3.0, &st);
    // F_Xy: i in [0,nx], j in [0,ny), k in [-1,nz]
    if (i >= 0 && j >= 0 && j < ny) h3_ctu_flux<SOLVER, 0, 1>(A, FY, A.S.cf + 10 * SP, i, j, k, dt_dx, dt_dy / 3.0, &st);
    // F_Zy: i in [-1,nx], j in [0,ny), k in [0,nz]
    if (j >= 0 && j < ny && k >= 0) h3_ctu_flux<SOLVER, 2, 1>(A, FY, A.S.cf + 15 * SP, i, j, k, dt_dz, dt_dy / 3.0, &st);
    // F_Yx: i in [0,nx), j in [0,ny], k in [-1,nz]
    if (i >= 0 && i < nx && j >= 0) h3_ctu_flux<SOLVER, 1, 0>(A, FX, A.S.cf + 20 * SP, i, j, k, dt_dy, dt_dx / 3.0, &st);
    // F_Zx: i in [0,nx), j in [-1,ny], k in [0,nz]
    if (i >= 0 && i < nx && k >= 0) h3_ctu_flux<SOLVER, 2, 0>(A, FX, A.S.cf + 25 * SP, i, j, k, dt_dz, dt_dx / 3.0, &st);
    h3_stats(A.ctl, st);
}

// K4: final fluxes on [0,n] along the normal axis, [0,n) on the others, from
// the half states corrected on the fly (correctState, CTU.cpp:246-260,280-301:
// x states by F_Yz then F_Zy, y states by F_Xz then F_Zx, z states by F_Xy then
// F_Yx). Every state a final face reads lies in the reference's corrected
// range (x states: cells [-1,nx] x [0,ny) x [0,nz), and likewise).
template <int SOLVER>
__global__ void __launch_bounds__(256, 2) k_h3_final(Step3DArgs A) {
    __shared__ int s;
    if (h3_skip(A.ctl, &s)) return;
    const Geo& G = A.G;
    const int lo[3] = {0, 0, 0}, ext[3] = {G.n[0] + 1, G.n[1] + 1, G.n[2] + 1};
    int i, j, k;
    if (!box_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, lo, ext, i, j, k)) return;
    const int nx = G.n[0], ny = G.n[1], nz = G.n[2];
    const double dt = *(const volatile double*)&A.ctl->t1;
    const H3Half h = h3_half(A, dt);
    FaceStats st{0, 0, 0, 0, 0};
    if (j < ny && k < nz) h3_final_flux<SOLVER, 0>(A, h, i, j, k, dt / A.sa.dx, &st);
    if (i < nx && k < nz) h3_final_flux<SOLVER, 1>(A, h, i, j, k, dt / A.sa.dy, &st);
    if (i < nx && j < ny) h3_final_flux<SOLVER, 2>(A, h, i, j, k, dt / A.sa.dz, &st);
    h3_stats(A.ctl, st);
}

// K5: conservative update of the interior (applyFluxes 3D, Unsplit.cpp:272-288),
// physicality, CFL speed of the committed state.
static __global__ void k_h3_update(Step3DArgs A) {
    __shared__ int s;
    __shared__ double red[32];
    if (h3_skip(A.ctl, &s)) return;
    const Geo& G = A.G;
    const int lo[3] = {0, 0, 0}, ext[3] = {G.n[0], G.n[1], G.n[2]};
    int i, j, k;
    double vmax = 0.0;
    if (box_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, lo, ext, i, j, k)) {
        const double dt = *(const volatile double*)&A.ctl->t1;
        const double dt_dx = dt / A.sa.dx, dt_dy = dt / A.sa.dy, dt_dz = dt / A.sa.dz;
        const long long P = G.plane, SP = A.S.plane, m = gidx3(G, i, j, k);
        const double* FX = A.S.pf;
        const double* FY = A.S.pf + 5 * SP;
        const double* FZ = A.S.pf + 10 * SP;
        Cons<double> U = to_cons<false>(ld5(A.w, P, m));
        U = c_add<false>(U, c_mul<false>(c_sub<false>(ldc5(FX, SP, m), ldc5(FX, SP, gidx3(G, i + 1, j, k))), dt_dx));
        U = c_add<false>(U, c_mul<false>(c_sub<false>(ldc5(FY, SP, m), ldc5(FY, SP, gidx3(G, i, j + 1, k))), dt_dy));
        U = c_add<false>(U, c_mul<false>(c_sub<false>(ldc5(FZ, SP, m), ldc5(FZ, SP, gidx3(G, i, j, k + 1))), dt_dz));
        const Prim<double> nw = to_prim<false>(U);
        if (!is_finite<false>(U)) record_error(A.ctl, ST_NAN, m);
        else if (!is_physical<false>(nw)) record_error(A.ctl, ST_UNPHYSICAL, m);
        st5(A.wout, P, m, nw);
        vmax = cfl_speed<false>(nw, A.sa.cfl, A.sa.dx, A.sa.dy, A.sa.dz);
    }
    vmax = block_max(vmax, red);
    if (threadIdx.x == 0) atomic_max_speed(&A.ctl->vmax[A.sa.slot_out], vmax);
}

// learned: the exact solver takes its Newton start from the network (sa.mlp).
template <int SOLVER>
inline int launch_step3d_hydro_t(const Geo& G, const double* w, double* wout, const Hydro3DScratch& S, StepCtl* ctl,
                               const StepArgs& sa, cudaStream_t st, bool learned = false) {
    Step3DArgs A{G, w, wout, S, ctl, sa};
    auto blocks = [](long long n) { return (int)((n + 255) / 256); };
    const long long box = (long long)(G.n[0] + 2) * (G.n[1] + 2) * (G.n[2] + 2);
    const long long fbox = (long long)(G.n[0] + 1) * (G.n[1] + 1) * (G.n[2] + 1);
    const long long cells = (long long)G.n[0] * G.n[1] * G.n[2];
    if (cudaMemcpyAsync(wout, w, sizeof(double) * 5 * G.plane, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return 1;
    k_h3_halfstates<<<blocks(box), 256, 0, st>>>(A);
    if constexpr (SOLVER == RS_EXACT) {
        if (learned) {
            k_h3_prelim_learned<<<blocks(box), 256, 0, st>>>(A);
            k_h3_ctu_learned<<<blocks(box), 256, 0, st>>>(A);
            k_h3_final_learned<<<blocks(fbox), 256, 0, st>>>(A);
            k_h3_update<<<blocks(cells), 256, 0, st>>>(A);
            return cudaGetLastError() == cudaSuccess ? 0 : 1;
        }
    }
    k_h3_prelim<SOLVER><<<blocks(box), 256, 0, st>>>(A);
    k_h3_ctu<SOLVER><<<blocks(box), 256, 0, st>>>(A);
    k_h3_final<SOLVER><<<blocks(fbox), 256, 0, st>>>(A);
    k_h3_update<<<blocks(cells), 256, 0, st>>>(A);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace dgpu
