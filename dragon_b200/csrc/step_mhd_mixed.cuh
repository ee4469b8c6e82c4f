// Mixed FP32/FP64 2D MHD CTU + CT step: the seven phases of step_mhd.cuh
// with FP32 reconstruction, limiters, HLLD / HLL / HLLE fluxes, CTU
// corrections and FP32 intermediates in HBM (half the scratch traffic), and
// FP64 where stability or the invariants need it:
//   * every pressure recovery from a conservative state (total energy carried
//     in FP64 from the FP64 energy of the state it started from);
//   * the half-step and final conservative updates (applyFluxes) accumulated
//     in FP64 from the FP64 state;
//   * Faraday's law on the faces (B_fields.cpp:21-40) in FP64, so the face
//     update keeps div B at FP64 roundoff for any edge E;
//   * the edge E averaging and upwinding (Electric.cpp) in FP64 from the FP32
//     fluxes.
// Each phase is a device body over one 32 x 8 tile (Tile2): the single-grid
// step (step_mhd_mixed.cu) runs one tile per CTA, the batched step
// (batch_mixed.cu) runs tiles as work items; both translation units are
// compiled with FMA contraction and fast single-precision division / square
// root (batch.cu includes this header for the FP64 batch, which never runs
// these bodies). Where the compiler fuses a multiply into an add
// depends on the code a body is inlined into, so the two kernels can round an
// FP32 value differently (kept inline: out of line, the single-grid step ran
// 21 % slower).
#pragma once

#include "mixed.cuh"
#include "step_mhd.cuh"

namespace dgpu {

struct Mhd2DMixedArgs {
    Geo G, FG;
    const double* w;
    double* wout;
    const double* B;
    double* Bout;
    MhdScratchF S;
    StepCtl* ctl;
    StepArgs sa;
};

// shouldProtectThermal (B_fields.cpp:91-114) without the division: for
// B^2 > 0, 8 pi p / B^2 <= 0.1 is 8 pi p <= 0.1 B^2 (rounding differs only at
// the threshold, which the mixed path is not held to).
__device__ __forceinline__ bool protect_thermal_mx(const Prim<double>& w, int mode) {
    if (mode == 0) return false;
    if (mode == 1) return true;
    const double B2 = dot3(w.Bx, w.By, w.Bz, w.Bx, w.By, w.Bz);
    if (B2 == 0) return false;
    return k8pi * w.p <= 0.1 * B2;
}

// computeBodyField (B_fields.cpp:70-79) with the mixed path's FP64 conversions.
__device__ __forceinline__ Prim<double> body_field64(Prim<double> w, double bx, double by, double bz, int mode) {
    if (!protect_thermal_mx(w, mode)) {
        Cons<double> U = to_cons64<true>(w);
        U.Bx = bx; U.By = by; U.Bz = bz;
        return to_prim64<true>(U);
    }
    w.Bx = bx; w.By = by; w.Bz = bz;
    return w;
}

__device__ __forceinline__ void st_prim8f(float* a, long long P, long long m, const Prim<float>& w) {
    a[m] = w.rho; a[P + m] = w.p; a[2 * P + m] = w.vx; a[3 * P + m] = w.vy; a[4 * P + m] = w.vz;
    a[5 * P + m] = w.Bx; a[6 * P + m] = w.By; a[7 * P + m] = w.Bz;
}
__device__ __forceinline__ Prim<float> ld_prim8f(const float* a, long long P, long long m) {
    return Prim<float>{a[m], a[P + m], a[2 * P + m], a[3 * P + m], a[4 * P + m], a[5 * P + m], a[6 * P + m], a[7 * P + m]};
}
__device__ __forceinline__ void st_cons8f(float* a, long long P, long long m, const Cons<float>& u) {
    a[m] = u.rho; a[P + m] = u.E; a[2 * P + m] = u.mx; a[3 * P + m] = u.my; a[4 * P + m] = u.mz;
    a[5 * P + m] = u.Bx; a[6 * P + m] = u.By; a[7 * P + m] = u.Bz;
}
__device__ __forceinline__ Cons<double> ld_cons8d(const float* a, long long P, long long m) {
    Cons<double> u;
    u.rho = a[m]; u.E = a[P + m]; u.mx = a[2 * P + m]; u.my = a[3 * P + m]; u.mz = a[4 * P + m];
    u.Bx = a[5 * P + m]; u.By = a[6 * P + m]; u.Bz = a[7 * P + m];
    return u;
}
__device__ __forceinline__ V3 ld_v3d(const float* a, long long P, long long m) { return V3{a[m], a[P + m], a[2 * P + m]}; }
__device__ __forceinline__ void st_v3f(float* a, long long P, long long m, V3 v) {
    a[m] = (float)v.x; a[P + m] = (float)v.y; a[2 * P + m] = (float)v.z;
}

// K1: FP32 half states (MUSCL-Hancock with FP64 predictor energy) and the
// body E of w.
__device__ __forceinline__ void mx_halfstates(const Mhd2DMixedArgs& A, const Tile2& T) {
    __shared__ int s;
    if (mhd_skip(A.ctl, &s)) return;
    int i, j;
    if (!cell_of(T, -2, A.G.n[0] + 4, -2, A.G.n[1] + 4, i, j)) return;
    const double dt = mhd_dt(A.ctl), dt_dx = dt / A.sa.dx, dt_dy = dt / A.sa.dy;
    const Geo& G = A.G;
    const Geo& F = A.FG;
    const long long P = G.plane, FP = F.plane, SP = A.S.plane;
    auto W = [&](int a, int b) { return cvt<float>(load_prim<true>(A.w, P, gidx2(G, a, b))); };
    const double bx0 = A.B[gidx2(F, i, j)], bx1 = A.B[gidx2(F, i + 1, j)];
    const double by0 = A.B[FP + gidx2(F, i, j)], by1 = A.B[FP + gidx2(F, i, j + 1)];
    const float dBx = (float)((bx1 - bx0) * dt_dx), dBy = (float)((by1 - by0) * dt_dy);
    const Prim<double> wc64 = load_prim<true>(A.w, P, gidx2(G, i, j));
    const Prim<float> wc = cvt<float>(wc64);
    const long long m = gidx2(F, i, j);
    int fo = 0;
    Prim<float> L, R;
    fo += !muscl_mixed<true>(A.sa.limiter, W(i - 1, j), L, wc, R, W(i + 1, j), (float)dt_dx, dBx, dBy, 0.f);
    L.Bx = (float)bx0;
    R.Bx = (float)bx1;
    st_prim8f(A.S.hs, SP, m, L);
    st_prim8f(A.S.hs + 8 * SP, SP, m, R);
    Prim<float> yl = W(i, j - 1), yc = wc, yr = W(i, j + 1);
    swap_xy(yl); swap_xy(yc); swap_xy(yr);
    fo += !muscl_mixed<true>(A.sa.limiter, yl, L, yc, R, yr, (float)dt_dy, dBy, dBx, 0.f);
    swap_xy(L); swap_xy(R);
    L.By = (float)by0;
    R.By = (float)by1;
    st_prim8f(A.S.hs + 16 * SP, SP, m, L);
    st_prim8f(A.S.hs + 24 * SP, SP, m, R);
    st_v3f(A.S.er, SP, m, body_e(wc64));
    warp_add_stat(&A.ctl->muscl_first_order, fo);
}

// K2 / K5: FP32 Riemann fluxes over the given ranges (predictor: the x faces
// [-1, nx+1] x rows [-2, ny+1] and the y faces; final: [0, nx] x [-1, ny]).
template <int SOLVER, bool FINAL>
__device__ __forceinline__ void mx_fluxes(const Mhd2DMixedArgs& A, const Tile2& T) {
    __shared__ int s;
    if (mhd_skip(A.ctl, &s)) return;
    int i, j;
    const int e = FINAL ? 1 : 2;
    if (!cell_of(T, -e, A.G.n[0] + 2 * e, -e, A.G.n[1] + 2 * e, i, j)) return;
    const double dt = mhd_dt(A.ctl);
    const float dt_dx = (float)(dt / A.sa.dx), dt_dy = (float)(dt / A.sa.dy);
    const Geo& F = A.FG;
    const long long SP = A.S.plane;
    const ExactOpts eo = exact_opts(A.sa);
    FaceStats st{};
    const int nx = A.G.n[0], ny = A.G.n[1];
    Cons<float> Fl;
    const bool xf = FINAL ? (i >= 0) : (i >= -1 && i <= nx + 1 && j <= ny + 1);
    const bool yf = FINAL ? (j >= 0) : (i <= nx + 1 && j >= -1 && j <= ny + 1);
    if (xf) {
        face_flux_mixed<true, SOLVER, 0>(ld_prim8f(A.S.hs + 8 * SP, SP, gidx2(F, i - 1, j)),
                                         ld_prim8f(A.S.hs, SP, gidx2(F, i, j)), dt_dx, eo, Fl, &st);
        st_cons8f(A.S.fx, SP, gidx2(F, i, j), Fl);
    }
    if (yf) {
        face_flux_mixed<true, SOLVER, 1>(ld_prim8f(A.S.hs + 24 * SP, SP, gidx2(F, i, j - 1)),
                                         ld_prim8f(A.S.hs + 16 * SP, SP, gidx2(F, i, j)), dt_dy, eo, Fl, &st);
        st_cons8f(A.S.fy, SP, gidx2(F, i, j), Fl);
    }
    warp_add_stat(&A.ctl->hlld_to_hlle, st.hlld_to_hlle);
}

// Corner E in FP64 from the FP32 fluxes and reference body E (corner_e of
// step_mhd.cuh on FP32 intermediates).
__device__ __forceinline__ V3 corner_e_mx(const Mhd2DMixedArgs& A, const float* __restrict__ eref, int i, int j) {
    const Geo& F = A.FG;
    const long long SP = A.S.plane;
    auto FXv = [&](int a, int b, int c) { return (double)A.S.fx[c * SP + gidx2(F, a, b)]; };
    auto FYv = [&](int a, int b, int c) { return (double)A.S.fy[c * SP + gidx2(F, a, b)]; };
    auto ER = [&](int a, int b) { return ld_v3d(eref, SP, gidx2(F, a, b)); };
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

// K3 / K6: corner E on edges [-1, nx+1]^2 (predictor, against the body E of
// w) or [0, nx]^2 (final, against the half-step body E).
template <bool FINAL>
__device__ __forceinline__ void mx_edges(const Mhd2DMixedArgs& A, const Tile2& T) {
    __shared__ int s;
    if (mhd_skip(A.ctl, &s)) return;
    int i, j;
    const int lo = FINAL ? 0 : -1, ext = FINAL ? 1 : 3;
    if (!cell_of(T, lo, A.G.n[0] + ext, lo, A.G.n[1] + ext, i, j)) return;
    st_v3f(A.S.e0, A.S.plane, gidx2(A.FG, i, j), corner_e_mx(A, FINAL ? A.S.eh : A.S.er, i, j));
}

// K4: half-step face B (FP64 Faraday, dt/2), half-step cells (FP64 update)
// with their body E, and the FP32 CTU corrections of the half states with the
// FP64 energy carried through.
__device__ __forceinline__ void mx_half(const Mhd2DMixedArgs& A, const Tile2& T) {
    __shared__ int s;
    if (mhd_skip(A.ctl, &s)) return;
    int i, j;
    if (!cell_of(T, -1, A.G.n[0] + 2, -1, A.G.n[1] + 2, i, j)) return;
    const double dt = mhd_dt(A.ctl), dt_dx = dt / A.sa.dx, dt_dy = dt / A.sa.dy;
    const double hdx = 0.5 * dt_dx, hdy = 0.5 * dt_dy;
    const Geo& G = A.G;
    const Geo& F = A.FG;
    const long long P = G.plane, FP = F.plane, SP = A.S.plane;
    auto E0 = [&](int a, int b) { return ld_v3d(A.S.e0, SP, gidx2(F, a, b)); };
    const V3 e00 = E0(i, j), e10 = E0(i + 1, j), e01 = E0(i, j + 1), e11 = E0(i + 1, j + 1);
    const double bxh0 = A.B[gidx2(F, i, j)] - (e01.z - e00.z) * hdy;
    const double bxh1 = A.B[gidx2(F, i + 1, j)] - (e11.z - e10.z) * hdy;
    const double byh0 = A.B[FP + gidx2(F, i, j)] - -(e10.z - e00.z) * hdx;
    const double byh1 = A.B[FP + gidx2(F, i, j + 1)] - -(e11.z - e01.z) * hdx;
    const double bzh = A.B[2 * FP + gidx2(F, i, j)] - ((e10.y - e00.y) * hdx - (e01.x - e00.x) * hdy);
    const Prim<double> W = load_prim<true>(A.w, P, gidx2(G, i, j));
    const long long m = gidx2(F, i, j);
    const Cons<double> px0 = ld_cons8d(A.S.fx, SP, m), px1 = ld_cons8d(A.S.fx, SP, gidx2(F, i + 1, j));
    const Cons<double> py0 = ld_cons8d(A.S.fy, SP, m), py1 = ld_cons8d(A.S.fy, SP, gidx2(F, i, j + 1));
    {
        Cons<double> U = to_cons64<true>(W);
        U = c_add<true>(U, c_mul<true>(c_sub<true>(px0, px1), hdx));
        U = c_add<true>(U, c_mul<true>(c_sub<true>(py0, py1), hdy));
        if (!is_finite<true>(U)) record_error(A.ctl, ST_NAN, m);
        Prim<double> wh = to_prim64<true>(U);
        wh = body_field64(wh, (bxh0 + bxh1) * 0.5, (byh0 + byh1) * 0.5, bzh, A.sa.ct_energy);
        st_v3f(A.S.eh, SP, m, body_e(wh));
    }
    const double dBx = (A.B[gidx2(F, i + 1, j)] - A.B[gidx2(F, i, j)]) * dt_dx;
    const double dBy = (A.B[FP + gidx2(F, i, j + 1)] - A.B[FP + gidx2(F, i, j)]) * dt_dy;
    // one corrected pair: u = cons(h) + corr with the face B substituted, FP64 energy
    auto correct = [&](float* pl, float* pr, const Cons<double>& corr, int comp, double bl, double br) {
        const Prim<float> hl = ld_prim8f(pl, SP, m), hr = ld_prim8f(pr, SP, m);
        const Cons<float> cf = cvt<float>(corr);
        Cons<float> ul = c_add<true>(to_cons<true>(hl), cf), ur = c_add<true>(to_cons<true>(hr), cf);
        if (comp == 0) { ul.Bx = (float)bl; ur.Bx = (float)br; }
        else { ul.By = (float)bl; ur.By = (float)br; }
        st_prim8f(pl, SP, m, prim_from<true>(ul, energy64<true>(hl) + corr.E));
        st_prim8f(pr, SP, m, prim_from<true>(ur, energy64<true>(hr) + corr.E));
    };
    {
        Cons<double> corr = c_mul<true>(c_mul<true>(c_sub<true>(py0, py1), 0.5), dt_dy);
        corr.Bx = corr.By = corr.Bz = 0;
        const double lim_z = lim_minmod(-dBy, dBx);
        corr.E += k1_8pi * (W.Bz * W.vz * lim_z);
        corr.Bz = 0.5 * dt_dy * (e01.x - e00.x) + 0.5 * W.vz * lim_z;
        correct(A.S.hs, A.S.hs + 8 * SP, corr, 0, bxh0, bxh1);
    }
    {
        Cons<double> corr = c_mul<true>(c_mul<true>(c_sub<true>(px0, px1), 0.5), dt_dx);
        corr.Bx = corr.By = corr.Bz = 0;
        const double lim_z = lim_minmod(-dBx, dBy);
        corr.E += k1_8pi * (W.Bz * W.vz * lim_z);
        corr.Bz = -0.5 * dt_dx * (e10.y - e00.y) + 0.5 * W.vz * lim_z;
        correct(A.S.hs + 16 * SP, A.S.hs + 24 * SP, corr, 1, byh0, byh1);
    }
}

// K7: FP64 conservative update from the FP32 fluxes, FP64 Faraday, face->cell
// B with the energy gate, physicality and the next CFL speed.
__device__ __forceinline__ void mx_update(const Mhd2DMixedArgs& A, const Tile2& T) {
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
        auto E = [&](int a, int b) { return ld_v3d(A.S.e0, SP, gidx2(F, a, b)); };
        const V3 e00 = E(i, j), e10 = E(i + 1, j), e01 = E(i, j + 1), e11 = E(i + 1, j + 1);
        const double bx0 = A.B[gidx2(F, i, j)] - (e01.z - e00.z) * dt_dy;
        const double bx1 = A.B[gidx2(F, i + 1, j)] - (e11.z - e10.z) * dt_dy;
        const double by0 = A.B[FP + gidx2(F, i, j)] - -(e10.z - e00.z) * dt_dx;
        const double by1 = A.B[FP + gidx2(F, i, j + 1)] - -(e11.z - e01.z) * dt_dx;
        const double bz = A.B[2 * FP + gidx2(F, i, j)] - ((e10.y - e00.y) * dt_dx - (e01.x - e00.x) * dt_dy);
        const long long mc = gidx2(G, i, j), mf = gidx2(F, i, j);
        Cons<double> U = to_cons64<true>(load_prim<true>(A.w, P, mc));
        U = c_add<true>(U, c_mul<true>(c_sub<true>(ld_cons8d(A.S.fx, SP, mf), ld_cons8d(A.S.fx, SP, gidx2(F, i + 1, j))), dt_dx));
        U = c_add<true>(U, c_mul<true>(c_sub<true>(ld_cons8d(A.S.fy, SP, mf), ld_cons8d(A.S.fy, SP, gidx2(F, i, j + 1))), dt_dy));
        if (!is_finite<true>(U)) record_error(A.ctl, ST_NAN, mc);
        Prim<double> nw = body_field64(to_prim64<true>(U), (bx0 + bx1) * 0.5, (by0 + by1) * 0.5, bz, A.sa.ct_energy);
        if (!is_physical<true>(nw)) record_error(A.ctl, ST_UNPHYSICAL, mc);
        store_prim<true>(A.wout, P, mc, nw);
        A.Bout[mf] = bx0;
        A.Bout[FP + mf] = by0;
        A.Bout[2 * FP + mf] = bz;
        if (i == nx - 1) A.Bout[gidx2(F, nx, j)] = bx1;
        if (j == ny - 1) A.Bout[FP + gidx2(F, i, ny)] = by1;
        vmax = cfl_speed_mx<true>(nw, A.sa.cfl, A.sa.dx, A.sa.dy, 0.0);
    }
    for (int o = 16; o > 0; o >>= 1) vmax = speed_max(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nthr = blockDim.x * blockDim.y;
    if ((tid & 31) == 0) red[tid >> 5] = vmax;
    __syncthreads();
    if (tid == 0) {
        double mm = 0.0;
        for (int w = 0; w < (nthr + 31) / 32; w++) mm = speed_max(mm, red[w]);
        atomic_max_speed(&A.ctl->vmax[A.sa.slot_out], mm);
    }
}

}  // namespace dgpu
