// 3D MHD CTU + CT step (Grid3D::unsplit_step MHD branch, Unsplit.cpp:115-206;
// the 6-solve ctu_sweep_MHD, CTU.cpp:34-131; CT::computeElectric /
// upwindElectric / bodyElectric 3D, Electric.cpp:37-126; Faraday and body
// fields 3D, B_fields.cpp:41-63,79-88,144-162) as seven kernels over global
// intermediates on the face grid:
//   K1 half states along x, y, z (MUSCL with the face-B source terms, face B
//      copied into the normal component) and the body E of w, cells [-2, n+1]
//   K2 predictor fluxes F_X [-1, nx+1] x [-2, ny+1] x [-2, nz+1] (and
//      cyclic), CTU.cpp:42-44
//   K3 predictor edge E0 on [-1, n+1]^3, upwinded against the body E of w
//   K4 cells [-1, n]^3: half-step faces (Faraday, dt/2), the half-step cell
//      (applyFluxes g=1) with face->cell B and its body E, and the CTU
//      corrections of the six half states with the MHD source terms
//   K5 final fluxes (F_X on [0, nx] x [-1, ny] x [-1, nz], cyclic)
//   K6 final edge E on [0, n]^3, upwinded against the half-step body E
//   K7 interior cells: conservative update, Faraday on the faces the cell
//      owns, face->cell B with the energy gate, physicality, CFL speed
// Every sweep covers the reference's index range, in its operand order.
#pragma once

#include "step3d.cuh"
#include "step_mhd.cuh"

namespace dgpu {

struct Mhd3DArgs {
    Geo G, FG;
    const double* w;
    double* wout;
    const double* B;
    double* Bout;
    Mhd3DScratch S;
    StepCtl* ctl;
    StepArgs sa;
};

// half-state planes: hs + 8 * (2 * axis + side), side 0 = L, 1 = R
__device__ __forceinline__ double* m3_hs(const Mhd3DArgs& A, int axis, int side) {
    return A.S.hs + (long long)8 * (2 * axis + side) * A.S.plane;
}
__device__ __forceinline__ const double* m3_flux(const Mhd3DArgs& A, int axis) {
    return axis == 0 ? A.S.fx : axis == 1 ? A.S.fy : A.S.fz;
}
__device__ __forceinline__ double* m3_flux_w(const Mhd3DArgs& A, int axis) {
    return axis == 0 ? A.S.fx : axis == 1 ? A.S.fy : A.S.fz;
}

// Read-only loads (ld.global.nc). Every array these are used on is one the
// calling kernel does not write; the half states that k_m3_half corrects in
// place keep plain loads there.
__device__ __forceinline__ double m3_ld(const double* a, long long m) { return __ldg(a + m); }
__device__ __forceinline__ Prim<double> m3_ld_prim(const double* a, long long P, long long m) {
    return Prim<double>{__ldg(a + m),         __ldg(a + P + m),     __ldg(a + 2 * P + m), __ldg(a + 3 * P + m),
                        __ldg(a + 4 * P + m), __ldg(a + 5 * P + m), __ldg(a + 6 * P + m), __ldg(a + 7 * P + m)};
}
__device__ __forceinline__ Cons<double> m3_ld_cons(const double* a, long long P, long long m) {
    return Cons<double>{__ldg(a + m),         __ldg(a + P + m),     __ldg(a + 2 * P + m), __ldg(a + 3 * P + m),
                        __ldg(a + 4 * P + m), __ldg(a + 5 * P + m), __ldg(a + 6 * P + m), __ldg(a + 7 * P + m)};
}
__device__ __forceinline__ V3 m3_ld_v3(const double* a, long long P, long long m) {
    return V3{__ldg(a + m), __ldg(a + P + m), __ldg(a + 2 * P + m)};
}

__device__ __forceinline__ bool m3_cell(long long t, int lo, int hi_incl, const Geo& G, int& i, int& j, int& k) {
    const int lo3[3] = {lo, lo, lo};
    const int ext[3] = {G.n[0] + hi_incl - lo + 1, G.n[1] + hi_incl - lo + 1, G.n[2] + hi_incl - lo + 1};
    return box_cell(t, lo3, ext, i, j, k);
}

// K1
// Two CTAs per SM: natural register use (132; 196 for k_m3_half) leaves one,
// and the capped builds measured 5 % faster on the 3D MHD step.
static __global__ void __launch_bounds__(256, 2) k_m3_halfstates(Mhd3DArgs A) {
    __shared__ int s;
    if (h3_skip(A.ctl, &s)) return;
    int i, j, k;
    if (!m3_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, -2, 1, A.G, i, j, k)) return;
    const double dt = *(const volatile double*)&A.ctl->t1;
    const double dt_dx = dt / A.sa.dx, dt_dy = dt / A.sa.dy, dt_dz = dt / A.sa.dz;
    const Geo& G = A.G;
    const Geo& F = A.FG;
    const long long P = G.plane, FP = F.plane, SP = A.S.plane;
    auto W = [&](int a, int b, int c) { return m3_ld_prim(A.w, P, gidx3(G, a, b, c)); };
    const long long f = gidx3(F, i, j, k);
    const double bx0 = m3_ld(A.B, f), bx1 = m3_ld(A.B, gidx3(F, i + 1, j, k));
    const double by0 = m3_ld(A.B, FP + f), by1 = m3_ld(A.B, FP + gidx3(F, i, j + 1, k));
    const double bz0 = m3_ld(A.B, 2 * FP + f), bz1 = m3_ld(A.B, 2 * FP + gidx3(F, i, j, k + 1));
    const double dBx = (bx1 - bx0) * dt_dx, dBy = (by1 - by0) * dt_dy, dBz = (bz1 - bz0) * dt_dz;
    const Prim<double> wc = W(i, j, k);
    int fo = 0;
    Prim<double> L, R;
    // x (computeHalfStates_X 3D, Unsplit.cpp:351-378)
    fo += !muscl<true>(A.sa.limiter, W(i - 1, j, k), L, wc, R, W(i + 1, j, k), dt_dx, dBx, dBy, dBz);
    L.Bx = bx0;
    R.Bx = bx1;
    store_prim<true>(m3_hs(A, 0, 0), SP, f, L);
    store_prim<true>(m3_hs(A, 0, 1), SP, f, R);
    // y, swapped XY (Unsplit.cpp:379-407)
    {
        Prim<double> a = W(i, j - 1, k), c = wc, b = W(i, j + 1, k);
        swap_xy(a); swap_xy(c); swap_xy(b);
        fo += !muscl<true>(A.sa.limiter, a, L, c, R, b, dt_dy, dBy, dBx, dBz);
        swap_xy(L); swap_xy(R);
        L.By = by0;
        R.By = by1;
        store_prim<true>(m3_hs(A, 1, 0), SP, f, L);
        store_prim<true>(m3_hs(A, 1, 1), SP, f, R);
    }
    // z, swapped XZ (Unsplit.cpp:408-436)
    {
        Prim<double> a = W(i, j, k - 1), c = wc, b = W(i, j, k + 1);
        swap_xz(a); swap_xz(c); swap_xz(b);
        fo += !muscl<true>(A.sa.limiter, a, L, c, R, b, dt_dz, dBz, dBy, dBx);
        swap_xz(L); swap_xz(R);
        L.Bz = bz0;
        R.Bz = bz1;
        store_prim<true>(m3_hs(A, 2, 0), SP, f, L);
        store_prim<true>(m3_hs(A, 2, 1), SP, f, R);
    }
    store_v3(A.S.er, SP, f, body_e(wc));
    warp_add_stat(&A.ctl->muscl_first_order, fo);
}

template <int SOLVER, int AX>
__device__ __forceinline__ void m3_face_flux(const Mhd3DArgs& A, int i, int j, int k, double dtn, FaceStats* st) {
    const Geo& F = A.FG;
    const long long SP = A.S.plane;
    const int di = AX == 0, dj = AX == 1, dk = AX == 2;
    const Prim<double> L = m3_ld_prim(m3_hs(A, AX, 1), SP, gidx3(F, i - di, j - dj, k - dk));
    const Prim<double> R = m3_ld_prim(m3_hs(A, AX, 0), SP, gidx3(F, i, j, k));
    Cons<double> Fl;
    face_flux<true, SOLVER, AX>(L, R, dtn, exact_opts(A.sa), Fl, st);
    store_cons8(m3_flux_w(A, AX), SP, gidx3(F, i, j, k), Fl);
}

// K2 (box [-2, n+1]^3) and K5 (box [-1, n]^3): faces along an axis from its
// lower bound (-1 predictor, 0 final) up to the box's top.
template <int SOLVER, bool FINAL>
__global__ void __launch_bounds__(256, 2) k_m3_fluxes(Mhd3DArgs A) {
    __shared__ int s;
    if (h3_skip(A.ctl, &s)) return;
    int i, j, k;
    const int lo = FINAL ? -1 : -2, hi = FINAL ? 0 : 1;
    if (!m3_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, lo, hi, A.G, i, j, k)) return;
    const double dt = *(const volatile double*)&A.ctl->t1;
    const int f0 = FINAL ? 0 : -1;
    FaceStats st{};
    if (i >= f0) m3_face_flux<SOLVER, 0>(A, i, j, k, dt / A.sa.dx, &st);
    if (j >= f0) m3_face_flux<SOLVER, 1>(A, i, j, k, dt / A.sa.dy, &st);
    if (k >= f0) m3_face_flux<SOLVER, 2>(A, i, j, k, dt / A.sa.dz, &st);
    warp_add_stat(&A.ctl->hlld_to_hlle, st.hlld_to_hlle);
}

// Edge E (CT::computeElectric 3D + CT::upwindElectric 3D) against eref.
__device__ __forceinline__ V3 m3_edge_e(const Mhd3DArgs& A, const double* __restrict__ eref, int i, int j, int k) {
    const Geo& F = A.FG;
    const long long SP = A.S.plane;
    auto X = [&](int a, int b, int c, int q) { return m3_ld(A.S.fx, q * SP + gidx3(F, a, b, c)); };
    auto Y = [&](int a, int b, int c, int q) { return m3_ld(A.S.fy, q * SP + gidx3(F, a, b, c)); };
    auto Z = [&](int a, int b, int c, int q) { return m3_ld(A.S.fz, q * SP + gidx3(F, a, b, c)); };
    auto ER = [&](int a, int b, int c) { return m3_ld_v3(eref, SP, gidx3(F, a, b, c)); };
    // flux planes: 0 rho, 1 E, 2-4 momentum, 5 Bx, 6 By, 7 Bz
    V3 e;
    e.x = (Z(i, j - 1, k, 6) - Y(i, j, k - 1, 7) + Z(i, j, k, 6) - Y(i, j, k, 7)) * 0.25;
    e.y = (X(i, j, k - 1, 7) - Z(i - 1, j, k, 5) + X(i, j, k, 7) - Z(i, j, k, 5)) * 0.25;
    e.z = (Y(i - 1, j, k, 5) - X(i, j - 1, k, 6) + Y(i, j, k, 5) - X(i, j, k, 6)) * 0.25;
    const V3 r000 = ER(i, j, k), r100 = ER(i - 1, j, k), r010 = ER(i, j - 1, k), r001 = ER(i, j, k - 1);
    const V3 r101 = ER(i - 1, j, k - 1), r110 = ER(i - 1, j - 1, k), r011 = ER(i, j - 1, k - 1);
    // X upwinds
    e.y += upcorr(X(i, j, k, 0), -Z(i - 1, j, k, 5), -Z(i, j, k, 5), r100.y, r000.y);
    e.y += upcorr(X(i, j, k - 1, 0), -Z(i - 1, j, k, 5), -Z(i, j, k, 5), r101.y, r001.y);
    e.z += upcorr(X(i, j, k, 0), Y(i - 1, j, k, 5), Y(i, j, k, 5), r100.z, r000.z);
    e.z += upcorr(X(i, j - 1, k, 0), Y(i - 1, j, k, 5), Y(i, j, k, 5), r110.z, r010.z);
    // Y upwinds
    e.x += upcorr(Y(i, j, k, 0), Z(i, j - 1, k, 6), Z(i, j, k, 6), r010.x, r000.x);
    e.x += upcorr(Y(i, j, k - 1, 0), Z(i, j - 1, k, 6), Z(i, j, k, 6), r011.x, r001.x);
    e.z += upcorr(Y(i, j, k, 0), -X(i, j - 1, k, 6), -X(i, j, k, 6), r010.z, r000.z);
    e.z += upcorr(Y(i - 1, j, k, 0), -X(i, j - 1, k, 6), -X(i, j, k, 6), r110.z, r100.z);
    // Z upwinds
    e.x += upcorr(Z(i, j, k, 0), -Y(i, j, k - 1, 7), -Y(i, j, k, 7), r001.x, r000.x);
    e.x += upcorr(Z(i, j - 1, k, 0), -Y(i, j, k - 1, 7), -Y(i, j, k, 7), r011.x, r010.x);
    e.y += upcorr(Z(i, j, k, 0), X(i, j, k - 1, 7), X(i, j, k, 7), r001.y, r000.y);
    e.y += upcorr(Z(i - 1, j, k, 0), X(i, j, k - 1, 7), X(i, j, k, 7), r101.y, r100.y);
    return e;
}

// K3 (edges [-1, n+1]^3, against the body E of w) and K6 (edges [0, n]^3,
// against the half-step body E).
template <bool FINAL>
__global__ void k_m3_edges(Mhd3DArgs A) {
    __shared__ int s;
    if (h3_skip(A.ctl, &s)) return;
    int i, j, k;
    if (!m3_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, FINAL ? 0 : -1, FINAL ? 0 : 1, A.G, i, j, k)) return;
    store_v3(A.S.e0, A.S.plane, gidx3(A.FG, i, j, k), m3_edge_e(A, FINAL ? A.S.eh : A.S.er, i, j, k));
}

// Faraday on one face with edge E e and weights (CT::Faraday 3D, B_fields.cpp:41-63).
struct M3Faces {
    double bx0, bx1, by0, by1, bz0, bz1;
};
__device__ __forceinline__ M3Faces m3_faraday(const Mhd3DArgs& A, int i, int j, int k, double hx, double hy, double hz) {
    const Geo& F = A.FG;
    const long long FP = F.plane, SP = A.S.plane;
    auto E = [&](int a, int b, int c) { return m3_ld_v3(A.S.e0, SP, gidx3(F, a, b, c)); };
    auto bx = [&](int a) {
        return m3_ld(A.B, gidx3(F, a, j, k)) - ((E(a, j + 1, k).z - E(a, j, k).z) * hy - (E(a, j, k + 1).y - E(a, j, k).y) * hz);
    };
    auto by = [&](int b) {
        return m3_ld(A.B, FP + gidx3(F, i, b, k)) - ((E(i, b, k + 1).x - E(i, b, k).x) * hz - (E(i + 1, b, k).z - E(i, b, k).z) * hx);
    };
    auto bz = [&](int c) {
        return m3_ld(A.B, 2 * FP + gidx3(F, i, j, c)) - ((E(i + 1, j, c).y - E(i, j, c).y) * hx - (E(i, j + 1, c).x - E(i, j, c).x) * hy);
    };
    return M3Faces{bx(i), bx(i + 1), by(j), by(j + 1), bz(k), bz(k + 1)};
}

// K4
static __global__ void __launch_bounds__(256, 2) k_m3_half(Mhd3DArgs A) {
    __shared__ int s;
    if (h3_skip(A.ctl, &s)) return;
    int i, j, k;
    if (!m3_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, -1, 0, A.G, i, j, k)) return;
    const double dt = *(const volatile double*)&A.ctl->t1;
    const double dt_dx = dt / A.sa.dx, dt_dy = dt / A.sa.dy, dt_dz = dt / A.sa.dz;
    const double hdx = 0.5 * dt_dx, hdy = 0.5 * dt_dy, hdz = 0.5 * dt_dz;
    const Geo& G = A.G;
    const Geo& F = A.FG;
    const long long P = G.plane, FP = F.plane, SP = A.S.plane;
    const long long m = gidx3(F, i, j, k);
    const M3Faces h = m3_faraday(A, i, j, k, hdx, hdy, hdz);
    const Prim<double> W = m3_ld_prim(A.w, P, gidx3(G, i, j, k));
    const Cons<double> px0 = m3_ld_cons(A.S.fx, SP, m), px1 = m3_ld_cons(A.S.fx, SP, gidx3(F, i + 1, j, k));
    const Cons<double> py0 = m3_ld_cons(A.S.fy, SP, m), py1 = m3_ld_cons(A.S.fy, SP, gidx3(F, i, j + 1, k));
    const Cons<double> pz0 = m3_ld_cons(A.S.fz, SP, m), pz1 = m3_ld_cons(A.S.fz, SP, gidx3(F, i, j, k + 1));
    {
        // applyFluxes g=1 at dt/2 (Unsplit.cpp:272-288), computeBodyFields, bodyElectric
        Cons<double> U = to_cons<true>(W);
        U = c_add<true>(U, c_mul<true>(c_sub<true>(px0, px1), hdx));
        U = c_add<true>(U, c_mul<true>(c_sub<true>(py0, py1), hdy));
        U = c_add<true>(U, c_mul<true>(c_sub<true>(pz0, pz1), hdz));
        if (!is_finite<true>(U)) record_error(A.ctl, ST_NAN, m);
        Prim<double> wh = to_prim<true>(U);
        wh = body_field(wh, (h.bx0 + h.bx1) * 0.5, (h.by0 + h.by1) * 0.5, (h.bz0 + h.bz1) * 0.5, A.sa.ct_energy);
        store_v3(A.S.eh, SP, m, body_e(wh));
    }
    // CTU corrections (CTU.cpp:66-129)
    const double dBx = (m3_ld(A.B, gidx3(F, i + 1, j, k)) - m3_ld(A.B, m)) * dt_dx;
    const double dBy = (m3_ld(A.B, FP + gidx3(F, i, j + 1, k)) - m3_ld(A.B, FP + m)) * dt_dy;
    const double dBz = (m3_ld(A.B, 2 * FP + gidx3(F, i, j, k + 1)) - m3_ld(A.B, 2 * FP + m)) * dt_dz;
    auto E0 = [&](int a, int b, int c) { return m3_ld_v3(A.S.e0, SP, gidx3(F, a, b, c)); };
    auto apply = [&](int axis, Cons<double> corr, double bl, double br) {
        double* pl = m3_hs(A, axis, 0);
        double* pr = m3_hs(A, axis, 1);
        Cons<double> uL = c_add<true>(to_cons<true>(load_prim<true>(pl, SP, m)), corr);
        Cons<double> uR = c_add<true>(to_cons<true>(load_prim<true>(pr, SP, m)), corr);
        if (axis == 0) { uL.Bx = bl; uR.Bx = br; }
        else if (axis == 1) { uL.By = bl; uR.By = br; }
        else { uL.Bz = bl; uR.Bz = br; }
        store_prim<true>(pl, SP, m, to_prim<true>(uL));
        store_prim<true>(pr, SP, m, to_prim<true>(uR));
    };
    {   // x states
        Cons<double> corr = c_mul<true>(c_add<true>(c_mul<true>(c_sub<true>(py0, py1), dt_dy),
                                                     c_mul<true>(c_sub<true>(pz0, pz1), dt_dz)), 0.5);
        corr.Bx = corr.By = corr.Bz = 0;
        const double lim_y = lim_minmod(-dBz, dBx), lim_z = lim_minmod(-dBy, dBx);
        corr.E += k1_8pi * (W.By * W.vy * lim_y + W.Bz * W.vz * lim_z);
        corr.By = -0.25 * dt_dz * (E0(i, j, k + 1).x - E0(i, j, k).x + E0(i, j + 1, k + 1).x - E0(i, j + 1, k).x) +
                  0.5 * W.vy * lim_y;
        corr.Bz = 0.25 * dt_dy * (E0(i, j + 1, k).x - E0(i, j, k).x + E0(i, j + 1, k + 1).x - E0(i, j, k + 1).x) +
                  0.5 * W.vz * lim_z;
        apply(0, corr, h.bx0, h.bx1);
    }
    {   // y states
        Cons<double> corr = c_mul<true>(c_add<true>(c_mul<true>(c_sub<true>(px0, px1), dt_dx),
                                                     c_mul<true>(c_sub<true>(pz0, pz1), dt_dz)), 0.5);
        corr.Bx = corr.By = corr.Bz = 0;
        const double lim_x = lim_minmod(-dBz, dBy), lim_z = lim_minmod(-dBx, dBy);
        corr.E += k1_8pi * (W.Bx * W.vx * lim_x + W.Bz * W.vz * lim_z);
        corr.Bx = 0.25 * dt_dz * (E0(i, j, k + 1).y - E0(i, j, k).y + E0(i + 1, j, k + 1).y - E0(i + 1, j, k).y) +
                  0.5 * W.vx * lim_x;
        corr.Bz = -0.25 * dt_dx * (E0(i + 1, j, k).y - E0(i, j, k).y + E0(i + 1, j, k + 1).y - E0(i, j, k + 1).y) +
                  0.5 * W.vz * lim_z;
        apply(1, corr, h.by0, h.by1);
    }
    {   // z states
        Cons<double> corr = c_mul<true>(c_add<true>(c_mul<true>(c_sub<true>(px0, px1), dt_dx),
                                                     c_mul<true>(c_sub<true>(py0, py1), dt_dy)), 0.5);
        corr.Bx = corr.By = corr.Bz = 0;
        const double lim_x = lim_minmod(-dBy, dBz), lim_y = lim_minmod(-dBx, dBz);
        corr.E += k1_8pi * (W.Bx * W.vx * lim_x + W.By * W.vy * lim_y);
        corr.Bx = -0.25 * dt_dy * (E0(i, j + 1, k).z - E0(i, j, k).z + E0(i + 1, j + 1, k).z - E0(i + 1, j, k).z) +
                  0.5 * W.vx * lim_x;
        corr.By = 0.25 * dt_dx * (E0(i + 1, j, k).z - E0(i, j, k).z + E0(i + 1, j + 1, k).z - E0(i, j + 1, k).z) +
                  0.5 * W.vy * lim_y;
        apply(2, corr, h.bz0, h.bz1);
    }
}

// K7
static __global__ void k_m3_update(Mhd3DArgs A) {
    __shared__ int s;
    __shared__ double red[32];
    if (h3_skip(A.ctl, &s)) return;
    int i = 0, j = 0, k = 0;
    const bool in = m3_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, 0, -1, A.G, i, j, k);
    double vmax = 0.0;
    if (in) {
        const double dt = *(const volatile double*)&A.ctl->t1;
        const double dt_dx = dt / A.sa.dx, dt_dy = dt / A.sa.dy, dt_dz = dt / A.sa.dz;
        const Geo& G = A.G;
        const Geo& F = A.FG;
        const long long P = G.plane, FP = F.plane, SP = A.S.plane;
        const int nx = G.n[0], ny = G.n[1], nz = G.n[2];
        const long long mc = gidx3(G, i, j, k), mf = gidx3(F, i, j, k);
        const M3Faces b = m3_faraday(A, i, j, k, dt_dx, dt_dy, dt_dz);
        Cons<double> U = to_cons<true>(m3_ld_prim(A.w, P, mc));
        U = c_add<true>(U, c_mul<true>(c_sub<true>(m3_ld_cons(A.S.fx, SP, mf), m3_ld_cons(A.S.fx, SP, gidx3(F, i + 1, j, k))), dt_dx));
        U = c_add<true>(U, c_mul<true>(c_sub<true>(m3_ld_cons(A.S.fy, SP, mf), m3_ld_cons(A.S.fy, SP, gidx3(F, i, j + 1, k))), dt_dy));
        U = c_add<true>(U, c_mul<true>(c_sub<true>(m3_ld_cons(A.S.fz, SP, mf), m3_ld_cons(A.S.fz, SP, gidx3(F, i, j, k + 1))), dt_dz));
        if (!is_finite<true>(U)) record_error(A.ctl, ST_NAN, mc);
        Prim<double> nw = body_field(to_prim<true>(U), (b.bx0 + b.bx1) * 0.5, (b.by0 + b.by1) * 0.5, (b.bz0 + b.bz1) * 0.5,
                                     A.sa.ct_energy);
        if (!is_physical<true>(nw)) record_error(A.ctl, ST_UNPHYSICAL, mc);
        store_prim<true>(A.wout, P, mc, nw);
        A.Bout[mf] = b.bx0;
        A.Bout[FP + mf] = b.by0;
        A.Bout[2 * FP + mf] = b.bz0;
        if (i == nx - 1) A.Bout[gidx3(F, nx, j, k)] = b.bx1;
        if (j == ny - 1) A.Bout[FP + gidx3(F, i, ny, k)] = b.by1;
        if (k == nz - 1) A.Bout[2 * FP + gidx3(F, i, j, nz)] = b.bz1;
        vmax = cfl_speed<true>(nw, A.sa.cfl, A.sa.dx, A.sa.dy, A.sa.dz);
    }
    vmax = block_max(vmax, red);
    if (threadIdx.x == 0) atomic_max_speed(&A.ctl->vmax[A.sa.slot_out], vmax);
}

template <int SOLVER>
inline int launch_step3d_mhd_t(const Geo& G, const Geo& FG, const double* w, double* wout, const double* B, double* Bout,
                               const Mhd3DScratch& S, StepCtl* ctl, const StepArgs& sa, cudaStream_t st) {
    Mhd3DArgs A{G, FG, w, wout, B, Bout, S, ctl, sa};
    auto blocks = [&](int lo, int hi) {
        const long long n = (long long)(G.n[0] + hi - lo + 1) * (G.n[1] + hi - lo + 1) * (G.n[2] + hi - lo + 1);
        return (int)((n + 255) / 256);
    };
    if (cudaMemcpyAsync(wout, w, sizeof(double) * 8 * G.plane, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return 1;
    if (cudaMemcpyAsync(Bout, B, sizeof(double) * 3 * FG.plane, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return 1;
    k_m3_halfstates<<<blocks(-2, 1), 256, 0, st>>>(A);
    k_m3_fluxes<SOLVER, false><<<blocks(-2, 1), 256, 0, st>>>(A);
    k_m3_edges<false><<<blocks(-1, 1), 256, 0, st>>>(A);
    k_m3_half<<<blocks(-1, 0), 256, 0, st>>>(A);
    k_m3_fluxes<SOLVER, true><<<blocks(-1, 0), 256, 0, st>>>(A);
    k_m3_edges<true><<<blocks(0, 0), 256, 0, st>>>(A);
    k_m3_update<<<blocks(0, -1), 256, 0, st>>>(A);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace dgpu
