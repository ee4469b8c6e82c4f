// MHD constrained-transport pieces of the device path.
//
// The 2D CTU + CT step (Grid2D::unsplit_step MHD branch, Unsplit.cpp:28-111;
// ctu_sweep_MHD 2D, CTU.cpp:133-203; CT::*, Electric.cpp and B_fields.cpp)
// runs as seven kernels over global intermediates, one per data dependency of
// the reference:
//   K1 half states (MUSCL with the face-B source terms) + body E of w
//   K2 predictor fluxes
//   K3 corner E0 (arithmetic average + upwinding against the body E)
//   K4 half-step face B, half-step cells, their body E, CTU corrections
//   K5 final fluxes
//   K6 final corner E (upwinded against the half-step body E)
//   K7 conservative update, Faraday, face->cell B with the energy gate,
//      physicality and the next step's CFL speed
// Each kernel covers exactly the index ranges the reference loops over, so the
// arithmetic (and every failure) is the reference's.
#pragma once

#include <algorithm>

#include "frame.cuh"
#include "grid.cuh"
#include "recon.cuh"
#include "riemann.cuh"
#include "scratch.h"

namespace dgpu {

// Grid2D/3D::initialize_B_fields after the boundary fill (B_fields.cpp:117-149):
// every cell, ghosts included, takes the average of its two face values per
// component (2D keeps the cell's z face value), pressure untouched.
static __global__ void k_init_body_fields(Geo G, Geo FG, double* __restrict__ w, const double* __restrict__ B) {
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

inline int launch_init_body_fields_t(const Geo& G, const Geo& FG, double* w, const double* B, cudaStream_t s) {
    const long long total = (long long)G.ext[0] * G.ext[1] * G.ext[2];
    int blocks = (int)((total + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_init_body_fields<<<blocks, 256, 0, s>>>(G, FG, w, B);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

__device__ __forceinline__ void store_cons8(double* __restrict__ a, long long P, long long m, const Cons<double>& u) {
    a[m] = u.rho; a[P + m] = u.E; a[2 * P + m] = u.mx; a[3 * P + m] = u.my; a[4 * P + m] = u.mz;
    a[5 * P + m] = u.Bx; a[6 * P + m] = u.By; a[7 * P + m] = u.Bz;
}
__device__ __forceinline__ Cons<double> load_cons8(const double* __restrict__ a, long long P, long long m) {
    Cons<double> u;
    u.rho = a[m]; u.E = a[P + m]; u.mx = a[2 * P + m]; u.my = a[3 * P + m]; u.mz = a[4 * P + m];
    u.Bx = a[5 * P + m]; u.By = a[6 * P + m]; u.Bz = a[7 * P + m];
    return u;
}
struct V3 { double x, y, z; };
__device__ __forceinline__ V3 load_v3(const double* __restrict__ a, long long P, long long m) {
    return V3{a[m], a[P + m], a[2 * P + m]};
}
__device__ __forceinline__ void store_v3(double* __restrict__ a, long long P, long long m, V3 v) {
    a[m] = v.x; a[P + m] = v.y; a[2 * P + m] = v.z;
}
// cross(w.B, w.v) (Arithmetic.cpp:95-101)
__device__ __forceinline__ V3 body_e(const Prim<double>& w) {
    return V3{w.By * w.vz - w.Bz * w.vy, w.Bz * w.vx - w.Bx * w.vz, w.Bx * w.vy - w.By * w.vx};
}
// upwindCorr (Electric.cpp:52-57)
__device__ __forceinline__ double upcorr(double m, double em, double ep, double rm, double rp) {
    if (m > 1e-18) return 0.25 * (em - rm);
    if (m < -1e-18) return 0.25 * (ep - rp);
    return 0.125 * (em + ep - rm - rp);
}
// shouldProtectThermal, compile-time forms of B_fields.cpp:91-114 (BETA_GATED: 8 pi p / B^2 <= 0.1)
__device__ __forceinline__ bool protect_thermal(const Prim<double>& w, int mode) {
    if (mode == 0) return false;
    if (mode == 1) return true;
    double B2 = dot3(w.Bx, w.By, w.Bz, w.Bx, w.By, w.Bz);
    if (B2 == 0) return false;
    double beta = k8pi * w.p / dot3(w.Bx, w.By, w.Bz, w.Bx, w.By, w.Bz);
    return beta <= 0.1;
}
// computeBodyField (B_fields.cpp:70-79)
__device__ __forceinline__ Prim<double> body_field(Prim<double> w, double bx, double by, double bz, int mode) {
    if (!protect_thermal(w, mode)) {
        Cons<double> U = to_cons<true>(w);
        U.Bx = bx; U.By = by; U.Bz = bz;
        return to_prim<true>(U);
    }
    w.Bx = bx; w.By = by; w.Bz = bz;
    return w;
}

struct Mhd2DArgs {
    Geo G, FG;
    const double* w;     // cell state in
    double* wout;
    const double* B;     // face B in
    double* Bout;
    MhdScratch S;
    StepCtl* ctl;
    StepArgs sa;
};

__device__ __forceinline__ bool mhd_skip(const StepCtl* ctl, int* s) {
    if (threadIdx.x == 0 && threadIdx.y == 0) *s = (*(const volatile int*)&ctl->err) | (*(const volatile int*)&ctl->done);
    __syncthreads();
    return *s != 0;
}
__device__ __forceinline__ double mhd_dt(const StepCtl* ctl) { return *(const volatile double*)&ctl->t1; }

// A 32 x 8 tile of cells: block coordinates (bx along j, by along i) and the
// thread's place in it. The phase kernels take it from their 2D launch; the
// batched step takes it from a work item.
struct Tile2 {
    int bx, by, tx, ty;
};
constexpr int kTileJ = 32, kTileI = 8;
__device__ __forceinline__ Tile2 launch_tile() {
    return Tile2{(int)blockIdx.x, (int)blockIdx.y, (int)threadIdx.x, (int)threadIdx.y};
}

// Cell (i, j) of tile T in a sweep covering [i0, i0 + ni) x [j0, j0 + nj).
__device__ __forceinline__ bool cell_of(const Tile2& T, int i0, int ni, int j0, int nj, int& i, int& j) {
    j = j0 + T.bx * kTileJ + T.tx;
    i = i0 + T.by * kTileI + T.ty;
    return i < i0 + ni && j < j0 + nj;
}

// K1: half states for cells [-2, nx+1]^2 (computeHalfStates_X/Y, Unsplit.cpp:292-342,
// copyFaceFields_X/Y, B_fields.cpp:166-183) and the body E of w (bodyElectric g=1).
__device__ __forceinline__ void mhd2d_halfstates(const Mhd2DArgs& A, const Tile2& T) {
    __shared__ int s;
    if (mhd_skip(A.ctl, &s)) return;
    int i, j;
    if (!cell_of(T, -2, A.G.n[0] + 4, -2, A.G.n[1] + 4, i, j)) return;
    const double dt = mhd_dt(A.ctl), dt_dx = dt / A.sa.dx, dt_dy = dt / A.sa.dy;
    const Geo& G = A.G;
    const Geo& F = A.FG;
    const long long P = G.plane, FP = F.plane, SP = A.S.plane;
    auto W = [&](int a, int b) { return load_prim<true>(A.w, P, gidx2(G, a, b)); };
    const double bx0 = A.B[gidx2(F, i, j)], bx1 = A.B[gidx2(F, i + 1, j)];
    const double by0 = A.B[FP + gidx2(F, i, j)], by1 = A.B[FP + gidx2(F, i, j + 1)];
    const double dBx = (bx1 - bx0) * dt_dx, dBy = (by1 - by0) * dt_dy;
    const Prim<double> wc = W(i, j);
    const long long m = gidx2(F, i, j);
    int fo = 0;
    Prim<double> L, R;
    fo += !muscl<true>(A.sa.limiter, W(i - 1, j), L, wc, R, W(i + 1, j), dt_dx, dBx, dBy, 0.0);
    L.Bx = bx0;
    R.Bx = bx1;
    store_prim<true>(A.S.hs, SP, m, L);
    store_prim<true>(A.S.hs + 8 * SP, SP, m, R);
    Prim<double> yl = W(i, j - 1), yc = wc, yr = W(i, j + 1);
    swap_xy(yl); swap_xy(yc); swap_xy(yr);
    // swapped source terms: dB.y from the x faces, dB.x from the y faces
    fo += !muscl<true>(A.sa.limiter, yl, L, yc, R, yr, dt_dy, dBy, dBx, 0.0);
    swap_xy(L); swap_xy(R);
    L.By = by0;
    R.By = by1;
    store_prim<true>(A.S.hs + 16 * SP, SP, m, L);
    store_prim<true>(A.S.hs + 24 * SP, SP, m, R);
    store_v3(A.S.er, SP, m, body_e(wc));
    warp_add_stat(&A.ctl->muscl_first_order, fo);
}

// K2: predictor fluxes: x faces [-1, nx+1] x rows [-2, ny+1], y faces cols
// [-2, nx+1] x [-1, ny+1] (ctu_sweep_MHD, CTU.cpp:140-141).
template <int SOLVER>
__device__ __forceinline__ void mhd2d_prelim(const Mhd2DArgs& A, const Tile2& T) {
    __shared__ int s;
    if (mhd_skip(A.ctl, &s)) return;
    int i, j;
    if (!cell_of(T, -2, A.G.n[0] + 4, -2, A.G.n[1] + 4, i, j)) return;
    const double dt = mhd_dt(A.ctl), dt_dx = dt / A.sa.dx, dt_dy = dt / A.sa.dy;
    const Geo& F = A.FG;
    const long long SP = A.S.plane;
    const ExactOpts eo = exact_opts(A.sa);
    FaceStats st{0, 0, 0, 0, 0};
    const int nx = A.G.n[0], ny = A.G.n[1];
    Cons<double> Fl;
    if (i >= -1 && i <= nx + 1 && j <= ny + 1) {
        Prim<double> L = load_prim<true>(A.S.hs + 8 * SP, SP, gidx2(F, i - 1, j));
        Prim<double> R = load_prim<true>(A.S.hs, SP, gidx2(F, i, j));
        face_flux<true, SOLVER, 0>(L, R, dt_dx, eo, Fl, &st);
        store_cons8(A.S.fx, SP, gidx2(F, i, j), Fl);
    }
    if (i <= nx + 1 && j >= -1 && j <= ny + 1) {
        Prim<double> L = load_prim<true>(A.S.hs + 24 * SP, SP, gidx2(F, i, j - 1));
        Prim<double> R = load_prim<true>(A.S.hs + 16 * SP, SP, gidx2(F, i, j));
        face_flux<true, SOLVER, 1>(L, R, dt_dy, eo, Fl, &st);
        store_cons8(A.S.fy, SP, gidx2(F, i, j), Fl);
    }
    warp_add_stat(&A.ctl->hlld_to_hlle, st.hlld_to_hlle);
}

// Corner E from face fluxes plus Gardiner-Stone upwinding against a body E
// (CT::computeElectric + CT::upwindElectric, Electric.cpp:24-33,59-74).
__device__ __forceinline__ V3 corner_e(const Mhd2DArgs& A, const double* __restrict__ eref, int i, int j) {
    const Geo& F = A.FG;
    const long long SP = A.S.plane;
    const double* fx = A.S.fx;
    const double* fy = A.S.fy;
    auto FXv = [&](int a, int b, int c) { return fx[c * SP + gidx2(F, a, b)]; };
    auto FYv = [&](int a, int b, int c) { return fy[c * SP + gidx2(F, a, b)]; };
    auto ER = [&](int a, int b) { return load_v3(eref, SP, gidx2(F, a, b)); };
    // field slots in a flux plane set: 0 rho, 1 E, 2-4 momentum, 5 Bx, 6 By, 7 Bz
    V3 e;
    e.x = -FYv(i, j, 7);
    e.y = FXv(i, j, 7);
    e.z = (FYv(i - 1, j, 5) - FXv(i, j - 1, 6) + FYv(i, j, 5) - FXv(i, j, 6)) * 0.25;
    const V3 r00 = ER(i, j), r10 = ER(i - 1, j), r01 = ER(i, j - 1), r11 = ER(i - 1, j - 1);
    e.z += upcorr(FXv(i, j, 0), FYv(i - 1, j, 5), FYv(i, j, 5), r10.z, r00.z);
    e.z += upcorr(FXv(i, j - 1, 0), FYv(i - 1, j, 5), FYv(i, j, 5), r11.z, r01.z);
    e.z += upcorr(FYv(i, j, 0), -FXv(i, j - 1, 6), -FXv(i, j, 6), r01.z, r00.z);
    e.z += upcorr(FYv(i - 1, j, 0), -FXv(i, j - 1, 6), -FXv(i, j, 6), r11.z, r10.z);
    e.x += 0.25 * (-2 * FYv(i, j, 7) - r00.x - r01.x);
    e.y += 0.25 * (2 * FXv(i, j, 7) - r00.y - r10.y);
    return e;
}

// K3: predictor corner E on edges [-1, nx+1]^2 against the body E of w.
__device__ __forceinline__ void mhd2d_e0(const Mhd2DArgs& A, const Tile2& T) {
    __shared__ int s;
    if (mhd_skip(A.ctl, &s)) return;
    int i, j;
    if (!cell_of(T, -1, A.G.n[0] + 3, -1, A.G.n[1] + 3, i, j)) return;
    store_v3(A.S.e0, A.S.plane, gidx2(A.FG, i, j), corner_e(A, A.S.er, i, j));
}

// K4: for cells [-1, nx]^2: half-step face B (Faraday with E0 and dt/2,
// B_fields.cpp:21-40), the half-step cell (applyFluxes g=1 with the predictor
// fluxes) with face->cell B, its body E, and the CTU corrections of the four
// half states with the MHD source terms (CTU.cpp:143-202).
__device__ __forceinline__ void mhd2d_half(const Mhd2DArgs& A, const Tile2& T) {
    __shared__ int s;
    if (mhd_skip(A.ctl, &s)) return;
    int i, j;
    if (!cell_of(T, -1, A.G.n[0] + 2, -1, A.G.n[1] + 2, i, j)) return;
    const double dt = mhd_dt(A.ctl), dt_dx = dt / A.sa.dx, dt_dy = dt / A.sa.dy;
    const double hdx = 0.5 * dt_dx, hdy = 0.5 * dt_dy;
    const Geo& G = A.G;
    const Geo& F = A.FG;
    const long long P = G.plane, FP = F.plane, SP = A.S.plane;
    auto E0 = [&](int a, int b) { return load_v3(A.S.e0, SP, gidx2(F, a, b)); };
    const V3 e00 = E0(i, j), e10 = E0(i + 1, j), e01 = E0(i, j + 1), e11 = E0(i + 1, j + 1);
    // half-step faces around the cell
    const double bxh0 = A.B[gidx2(F, i, j)] - (e01.z - e00.z) * hdy;
    const double bxh1 = A.B[gidx2(F, i + 1, j)] - (e11.z - e10.z) * hdy;
    const double byh0 = A.B[FP + gidx2(F, i, j)] - -(e10.z - e00.z) * hdx;
    const double byh1 = A.B[FP + gidx2(F, i, j + 1)] - -(e11.z - e01.z) * hdx;
    const double bzh = A.B[2 * FP + gidx2(F, i, j)] - ((e10.y - e00.y) * hdx - (e01.x - e00.x) * hdy);
    // half-step cell and its body E
    const Prim<double> W = load_prim<true>(A.w, P, gidx2(G, i, j));
    const long long m = gidx2(F, i, j);
    const Cons<double> px0 = load_cons8(A.S.fx, SP, m), px1 = load_cons8(A.S.fx, SP, gidx2(F, i + 1, j));
    const Cons<double> py0 = load_cons8(A.S.fy, SP, m), py1 = load_cons8(A.S.fy, SP, gidx2(F, i, j + 1));
    {
        Cons<double> U = to_cons<true>(W);
        U = c_add<true>(U, c_mul<true>(c_sub<true>(px0, px1), hdx));
        U = c_add<true>(U, c_mul<true>(c_sub<true>(py0, py1), hdy));
        if (!is_finite<true>(U)) record_error(A.ctl, ST_NAN, m);
        Prim<double> wh = to_prim<true>(U);
        wh = body_field(wh, (bxh0 + bxh1) * 0.5, (byh0 + byh1) * 0.5, bzh, A.sa.ct_energy);
        store_v3(A.S.eh, SP, m, body_e(wh));
    }
    // CTU corrections (CTU.cpp:163-201)
    const double dBx = (A.B[gidx2(F, i + 1, j)] - A.B[gidx2(F, i, j)]) * dt_dx;
    const double dBy = (A.B[FP + gidx2(F, i, j + 1)] - A.B[FP + gidx2(F, i, j)]) * dt_dy;
    {
        Cons<double> corr = c_mul<true>(c_mul<true>(c_sub<true>(py0, py1), 0.5), dt_dy);
        corr.Bx = corr.By = corr.Bz = 0;
        const double lim_z = lim_minmod(-dBy, dBx);
        corr.E += k1_8pi * (W.Bz * W.vz * lim_z);
        corr.Bz = 0.5 * dt_dy * (e01.x - e00.x) + 0.5 * W.vz * lim_z;
        Cons<double> uL = c_add<true>(to_cons<true>(load_prim<true>(A.S.hs, SP, m)), corr);
        Cons<double> uR = c_add<true>(to_cons<true>(load_prim<true>(A.S.hs + 8 * SP, SP, m)), corr);
        uL.Bx = bxh0;
        uR.Bx = bxh1;
        store_prim<true>(A.S.hs, SP, m, to_prim<true>(uL));
        store_prim<true>(A.S.hs + 8 * SP, SP, m, to_prim<true>(uR));
    }
    {
        Cons<double> corr = c_mul<true>(c_mul<true>(c_sub<true>(px0, px1), 0.5), dt_dx);
        corr.Bx = corr.By = corr.Bz = 0;
        const double lim_z = lim_minmod(-dBx, dBy);
        corr.E += k1_8pi * (W.Bz * W.vz * lim_z);
        corr.Bz = -0.5 * dt_dx * (e10.y - e00.y) + 0.5 * W.vz * lim_z;
        Cons<double> uL = c_add<true>(to_cons<true>(load_prim<true>(A.S.hs + 16 * SP, SP, m)), corr);
        Cons<double> uR = c_add<true>(to_cons<true>(load_prim<true>(A.S.hs + 24 * SP, SP, m)), corr);
        uL.By = byh0;
        uR.By = byh1;
        store_prim<true>(A.S.hs + 16 * SP, SP, m, to_prim<true>(uL));
        store_prim<true>(A.S.hs + 24 * SP, SP, m, to_prim<true>(uR));
    }
}

// K5: final fluxes, x faces [0, nx] x rows [-1, ny], y faces cols [-1, nx] x
// [0, ny] (Unsplit.cpp:58-60).
template <int SOLVER>
__device__ __forceinline__ void mhd2d_final_flux(const Mhd2DArgs& A, const Tile2& T) {
    __shared__ int s;
    if (mhd_skip(A.ctl, &s)) return;
    int i, j;
    if (!cell_of(T, -1, A.G.n[0] + 2, -1, A.G.n[1] + 2, i, j)) return;
    const double dt = mhd_dt(A.ctl), dt_dx = dt / A.sa.dx, dt_dy = dt / A.sa.dy;
    const Geo& F = A.FG;
    const long long SP = A.S.plane;
    const ExactOpts eo = exact_opts(A.sa);
    FaceStats st{0, 0, 0, 0, 0};
    Cons<double> Fl;
    if (i >= 0) {
        Prim<double> L = load_prim<true>(A.S.hs + 8 * SP, SP, gidx2(F, i - 1, j));
        Prim<double> R = load_prim<true>(A.S.hs, SP, gidx2(F, i, j));
        face_flux<true, SOLVER, 0>(L, R, dt_dx, eo, Fl, &st);
        store_cons8(A.S.fx, SP, gidx2(F, i, j), Fl);
    }
    if (j >= 0) {
        Prim<double> L = load_prim<true>(A.S.hs + 24 * SP, SP, gidx2(F, i, j - 1));
        Prim<double> R = load_prim<true>(A.S.hs + 16 * SP, SP, gidx2(F, i, j));
        face_flux<true, SOLVER, 1>(L, R, dt_dy, eo, Fl, &st);
        store_cons8(A.S.fy, SP, gidx2(F, i, j), Fl);
    }
    warp_add_stat(&A.ctl->hlld_to_hlle, st.hlld_to_hlle);
}

// K6: final corner E on edges [0, nx]^2 against the half-step body E.
__device__ __forceinline__ void mhd2d_efinal(const Mhd2DArgs& A, const Tile2& T) {
    __shared__ int s;
    if (mhd_skip(A.ctl, &s)) return;
    int i, j;
    if (!cell_of(T, 0, A.G.n[0] + 1, 0, A.G.n[1] + 1, i, j)) return;
    store_v3(A.S.e0, A.S.plane, gidx2(A.FG, i, j), corner_e(A, A.S.eh, i, j));
}

// K7: interior cells: conservative update (applyFluxes), Faraday on the faces
// the cell owns (B_fields.cpp:21-40), face->cell B with the energy gate,
// physicality and the CFL speed of the committed state.
__device__ __forceinline__ void mhd2d_update(const Mhd2DArgs& A, const Tile2& T) {
    __shared__ int s;
    __shared__ double red[32];
    if (mhd_skip(A.ctl, &s)) return;
    int i, j;
    const bool in = cell_of(T, 0, A.G.n[0], 0, A.G.n[1], i, j);
    const double dt = mhd_dt(A.ctl), dt_dx = dt / A.sa.dx, dt_dy = dt / A.sa.dy;
    const Geo& G = A.G;
    const Geo& F = A.FG;
    const long long P = G.plane, FP = F.plane, SP = A.S.plane;
    double vmax = 0.0;
    if (in) {
        const int nx = G.n[0], ny = G.n[1];
        auto E = [&](int a, int b) { return load_v3(A.S.e0, SP, gidx2(F, a, b)); };
        const V3 e00 = E(i, j), e10 = E(i + 1, j), e01 = E(i, j + 1), e11 = E(i + 1, j + 1);
        const double bx0 = A.B[gidx2(F, i, j)] - (e01.z - e00.z) * dt_dy;
        const double bx1 = A.B[gidx2(F, i + 1, j)] - (e11.z - e10.z) * dt_dy;
        const double by0 = A.B[FP + gidx2(F, i, j)] - -(e10.z - e00.z) * dt_dx;
        const double by1 = A.B[FP + gidx2(F, i, j + 1)] - -(e11.z - e01.z) * dt_dx;
        const double bz = A.B[2 * FP + gidx2(F, i, j)] - ((e10.y - e00.y) * dt_dx - (e01.x - e00.x) * dt_dy);
        const long long mc = gidx2(G, i, j), mf = gidx2(F, i, j);
        Cons<double> U = to_cons<true>(load_prim<true>(A.w, P, mc));
        U = c_add<true>(U, c_mul<true>(c_sub<true>(load_cons8(A.S.fx, SP, mf),
                                                   load_cons8(A.S.fx, SP, gidx2(F, i + 1, j))), dt_dx));
        U = c_add<true>(U, c_mul<true>(c_sub<true>(load_cons8(A.S.fy, SP, mf),
                                                   load_cons8(A.S.fy, SP, gidx2(F, i, j + 1))), dt_dy));
        if (!is_finite<true>(U)) record_error(A.ctl, ST_NAN, mc);
        Prim<double> nw = body_field(to_prim<true>(U), (bx0 + bx1) * 0.5, (by0 + by1) * 0.5, bz, A.sa.ct_energy);
        if (!is_physical<true>(nw)) record_error(A.ctl, ST_UNPHYSICAL, mc);
        store_prim<true>(A.wout, P, mc, nw);
        A.Bout[mf] = bx0;
        A.Bout[FP + mf] = by0;
        A.Bout[2 * FP + mf] = bz;
        if (i == nx - 1) A.Bout[gidx2(F, nx, j)] = bx1;
        if (j == ny - 1) A.Bout[FP + gidx2(F, i, ny)] = by1;
        vmax = cfl_speed<true>(nw, A.sa.cfl, A.sa.dx, A.sa.dy, 0.0);
    }
    // block-wide max over a 2D block
    for (int o = 16; o > 0; o >>= 1) vmax = speed_max(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nthr = blockDim.x * blockDim.y;
    if ((tid & 31) == 0) red[tid >> 5] = vmax;
    __syncthreads();
    if (tid == 0) {
        double m = 0.0;
        for (int w = 0; w < (nthr + 31) / 32; w++) m = speed_max(m, red[w]);
        atomic_max_speed(&A.ctl->vmax[A.sa.slot_out], m);
    }
}

// The ghost frame of the 2D MHD step's output buffers: every cell and face the
// update phase does not write, copied from the inputs so the committed arrays
// keep the ghosts the prologue filled (the reference commits the interior
// only, Unsplit.cpp:104-107). The update writes cells [0, nx) x [0, ny),
// x faces [0, nx] x [0, ny), y faces [0, nx) x [0, ny] and the cell-centred
// Bz [0, nx) x [0, ny); the frame is the rest of each padded array, about
// 4 g (n + g) points per array instead of the whole array.

// Copies frame points [k0, k1) (of mhd2d_frame_points) with the calling
// threads: thread tid of nthr.
__device__ __forceinline__ void mhd2d_copy_frame(const Geo& G, const Geo& FG, const double* __restrict__ w,
                                                 double* __restrict__ wout, const double* __restrict__ B,
                                                 double* __restrict__ Bout, long long k0, long long k1, long long tid,
                                                 long long nthr) {
    const int nx = G.n[0], ny = G.n[1], g = G.g;
    const long long nc = frame_count(-g, nx + g, -g, ny + g, 0, nx, 0, ny);
    const long long nf0 = frame_count(-g, nx + 1 + g, -g, ny + 1 + g, 0, nx + 1, 0, ny);
    const long long nf1 = frame_count(-g, nx + 1 + g, -g, ny + 1 + g, 0, nx, 0, ny + 1);
    for (long long k = k0 + tid; k < k1; k += nthr) {
        int i, j;
        if (k < nc) {
            if (!frame_point(k, -g, nx + g, -g, ny + g, 0, nx, 0, ny, i, j)) continue;
            const long long m = gidx2(G, i, j);
#pragma unroll
            for (int f = 0; f < 8; f++) wout[f * G.plane + m] = w[f * G.plane + m];
            continue;
        }
        long long q = k - nc;
        int comp;
        bool ok;
        if (q < nf0) {
            comp = 0;
            ok = frame_point(q, -g, nx + 1 + g, -g, ny + 1 + g, 0, nx + 1, 0, ny, i, j);
        } else if ((q -= nf0) < nf1) {
            comp = 1;
            ok = frame_point(q, -g, nx + 1 + g, -g, ny + 1 + g, 0, nx, 0, ny + 1, i, j);
        } else {
            q -= nf1;
            comp = 2;
            ok = frame_point(q, -g, nx + 1 + g, -g, ny + 1 + g, 0, nx, 0, ny, i, j);
        }
        if (!ok) continue;
        const long long m = comp * FG.plane + gidx2(FG, i, j);
        Bout[m] = B[m];
    }
}

// Kernels of the single-grid step: one 32 x 8 tile per CTA.
// The first kernel also copies the ghost frame of the output buffers from
// the inputs (grid-stride over the frame points; the step writes the rest).
static __global__ void k_mhd2d_halfstates(Mhd2DArgs A) {
    const long long nthr = (long long)gridDim.x * gridDim.y * blockDim.x * blockDim.y;
    const long long tid = ((long long)blockIdx.y * gridDim.x + blockIdx.x) * (blockDim.x * blockDim.y) +
                          threadIdx.y * blockDim.x + threadIdx.x;
    mhd2d_copy_frame(A.G, A.FG, A.w, A.wout, A.B, A.Bout, 0, mhd2d_frame_points(A.G.n[0], A.G.n[1], A.G.g), tid, nthr);
    mhd2d_halfstates(A, launch_tile());
}
// The flux kernels carry two CTAs per SM (<= 128 registers): at their natural
// ~166 registers one 256-thread CTA fits, and the HLLD chains stall on latency.
template <int SOLVER>
__global__ void __launch_bounds__(256, 2) k_mhd2d_prelim(Mhd2DArgs A) { mhd2d_prelim<SOLVER>(A, launch_tile()); }
static __global__ void k_mhd2d_e0(Mhd2DArgs A) { mhd2d_e0(A, launch_tile()); }
static __global__ void __launch_bounds__(256, 2) k_mhd2d_half(Mhd2DArgs A) { mhd2d_half(A, launch_tile()); }
template <int SOLVER>
__global__ void __launch_bounds__(256, 2) k_mhd2d_final_flux(Mhd2DArgs A) { mhd2d_final_flux<SOLVER>(A, launch_tile()); }
static __global__ void k_mhd2d_efinal(Mhd2DArgs A) { mhd2d_efinal(A, launch_tile()); }
static __global__ void k_mhd2d_update(Mhd2DArgs A) { mhd2d_update(A, launch_tile()); }

// 2D MHD CTU + CT step: the seven kernels in order; the first also copies
// the ghost frame of the output buffers from the inputs (mhd2d_copy_frame).
template <int SOLVER>
inline int launch_step2d_mhd_t(const Geo& G, const Geo& FG, const double* w, double* wout, const double* B, double* Bout,
                             const MhdScratch& S, StepCtl* ctl, const StepArgs& sa, cudaStream_t st) {
    Mhd2DArgs A{G, FG, w, wout, B, Bout, S, ctl, sa};
    const dim3 blk(kTileJ, kTileI);
    auto grid_for = [&](int ni, int nj) { return dim3((nj + kTileJ - 1) / kTileJ, (ni + kTileI - 1) / kTileI); };
    const int nx = G.n[0], ny = G.n[1];
    k_mhd2d_halfstates<<<grid_for(nx + 4, ny + 4), blk, 0, st>>>(A);
    k_mhd2d_prelim<SOLVER><<<grid_for(nx + 4, ny + 4), blk, 0, st>>>(A);
    k_mhd2d_e0<<<grid_for(nx + 3, ny + 3), blk, 0, st>>>(A);
    k_mhd2d_half<<<grid_for(nx + 2, ny + 2), blk, 0, st>>>(A);
    k_mhd2d_final_flux<SOLVER><<<grid_for(nx + 2, ny + 2), blk, 0, st>>>(A);
    k_mhd2d_efinal<<<grid_for(nx + 1, ny + 1), blk, 0, st>>>(A);
    k_mhd2d_update<<<grid_for(nx, ny), blk, 0, st>>>(A);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace dgpu
