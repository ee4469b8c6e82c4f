// Mixed FP32/FP64 3D MHD CTU + CT step: the seven kernels of step_mhd3d.cuh
// (Grid3D::unsplit_step MHD branch, Unsplit.cpp:115-206; the 6-solve
// ctu_sweep_MHD, CTU.cpp:34-131; CT 3D, Electric.cpp:37-126; Faraday and
// body fields 3D, B_fields.cpp:41-63,79-88,144-162) with FP32 reconstruction,
// limiters, transverse corrections and Riemann solves, and FP32 half states
// and fluxes (the 72 largest scratch planes: half the traffic of the FP64
// step's intermediates). FP64 stays where the 2D mixed MHD step keeps it:
// every energy and pressure recovery (mixed.cuh, prim_from), the edge
// electric fields (summed in FP64 from the FP32 fluxes), Faraday's law on
// the faces, the half-step cell and the conservative update of the FP64
// state, so the face update keeps div B at FP64 roundoff. Index ranges,
// operand roles and failure points are those of the FP64 step. Compiled with
// FMA contraction and fast single-precision division / square root, like the
// other mixed translation units.
#include "launchers.h"
#include "mixed.cuh"
#include "step_mhd3d.cuh"

namespace dgpu {

namespace {

// FP32 views of the FP64 step's half-state and flux planes (same plane length).
struct Mx3M {
    float* hs;  // 6 x 8 planes: xL, xR, yL, yR, zL, zR
    float* fx;  // 8 planes each: predictor, then final fluxes
    float* fy;
    float* fz;
    long long plane;
};

__device__ __forceinline__ float* m3m_hs(const Mx3M& X, int axis, int side) {
    return X.hs + (long long)8 * (2 * axis + side) * X.plane;
}
__device__ __forceinline__ float* m3m_flux(const Mx3M& X, int axis) { return axis == 0 ? X.fx : axis == 1 ? X.fy : X.fz; }

__device__ __forceinline__ Prim<float> ldf8(const float* a, long long P, long long m) {
    return Prim<float>{__ldg(a + m),         __ldg(a + P + m),     __ldg(a + 2 * P + m), __ldg(a + 3 * P + m),
                       __ldg(a + 4 * P + m), __ldg(a + 5 * P + m), __ldg(a + 6 * P + m), __ldg(a + 7 * P + m)};
}
// plain loads: the half states k_m3m_half corrects in place
__device__ __forceinline__ Prim<float> ldf8_rw(const float* a, long long P, long long m) {
    return Prim<float>{a[m], a[P + m], a[2 * P + m], a[3 * P + m], a[4 * P + m], a[5 * P + m], a[6 * P + m], a[7 * P + m]};
}
__device__ __forceinline__ void stf8(float* a, long long P, long long m, const Prim<float>& w) {
    a[m] = w.rho; a[P + m] = w.p; a[2 * P + m] = w.vx; a[3 * P + m] = w.vy;
    a[4 * P + m] = w.vz; a[5 * P + m] = w.Bx; a[6 * P + m] = w.By; a[7 * P + m] = w.Bz;
}
__device__ __forceinline__ Cons<float> ldcf8(const float* a, long long P, long long m) {
    return Cons<float>{__ldg(a + m),         __ldg(a + P + m),     __ldg(a + 2 * P + m), __ldg(a + 3 * P + m),
                       __ldg(a + 4 * P + m), __ldg(a + 5 * P + m), __ldg(a + 6 * P + m), __ldg(a + 7 * P + m)};
}
__device__ __forceinline__ void stcf8(float* a, long long P, long long m, const Cons<float>& u) {
    a[m] = u.rho; a[P + m] = u.E; a[2 * P + m] = u.mx; a[3 * P + m] = u.my;
    a[4 * P + m] = u.mz; a[5 * P + m] = u.Bx; a[6 * P + m] = u.By; a[7 * P + m] = u.Bz;
}
__device__ __forceinline__ Prim<float> f32_prim8(const Prim<double>& w) {
    return Prim<float>{(float)w.rho, (float)w.p,  (float)w.vx, (float)w.vy,
                       (float)w.vz,  (float)w.Bx, (float)w.By, (float)w.Bz};
}

// K1: half states along x, y, z (MUSCL with the face-B source terms, the
// normal component from the faces) and the body E of w, cells [-2, n+1]^3.
// Launch bounds: three CTAs per SM spilled the MUSCL and HLLD kernels; two
// CTAs (128 registers) keep them in registers.
__global__ void __launch_bounds__(256, 2) k_m3m_halfstates(Mhd3DArgs A, Mx3M X) {
    __shared__ int s;
    if (h3_skip(A.ctl, &s)) return;
    int i, j, k;
    if (!m3_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, -2, 1, A.G, i, j, k)) return;
    const double dt = *(const volatile double*)&A.ctl->t1;
    const double dt_dx = dt / A.sa.dx, dt_dy = dt / A.sa.dy, dt_dz = dt / A.sa.dz;
    const Geo& G = A.G;
    const Geo& F = A.FG;
    const long long P = G.plane, FP = F.plane, SP = X.plane;
    auto W = [&](int a, int b, int c) { return f32_prim8(m3_ld_prim(A.w, P, gidx3(G, a, b, c))); };
    const long long f = gidx3(F, i, j, k);
    const double bx0 = m3_ld(A.B, f), bx1 = m3_ld(A.B, gidx3(F, i + 1, j, k));
    const double by0 = m3_ld(A.B, FP + f), by1 = m3_ld(A.B, FP + gidx3(F, i, j + 1, k));
    const double bz0 = m3_ld(A.B, 2 * FP + f), bz1 = m3_ld(A.B, 2 * FP + gidx3(F, i, j, k + 1));
    const float dBx = (float)((bx1 - bx0) * dt_dx), dBy = (float)((by1 - by0) * dt_dy), dBz = (float)((bz1 - bz0) * dt_dz);
    const Prim<double> w64 = m3_ld_prim(A.w, P, gidx3(G, i, j, k));
    const Prim<float> wc = f32_prim8(w64);
    int fo = 0;
    Prim<float> L, R;
    fo += !muscl_mixed<true>(A.sa.limiter, W(i - 1, j, k), L, wc, R, W(i + 1, j, k), (float)dt_dx, dBx, dBy, dBz);
    L.Bx = (float)bx0;
    R.Bx = (float)bx1;
    stf8(m3m_hs(X, 0, 0), SP, f, L);
    stf8(m3m_hs(X, 0, 1), SP, f, R);
    {
        Prim<float> a = W(i, j - 1, k), c = wc, b = W(i, j + 1, k);
        swap_xy(a); swap_xy(c); swap_xy(b);
        fo += !muscl_mixed<true>(A.sa.limiter, a, L, c, R, b, (float)dt_dy, dBy, dBx, dBz);
        swap_xy(L); swap_xy(R);
        L.By = (float)by0;
        R.By = (float)by1;
        stf8(m3m_hs(X, 1, 0), SP, f, L);
        stf8(m3m_hs(X, 1, 1), SP, f, R);
    }
    {
        Prim<float> a = W(i, j, k - 1), c = wc, b = W(i, j, k + 1);
        swap_xz(a); swap_xz(c); swap_xz(b);
        fo += !muscl_mixed<true>(A.sa.limiter, a, L, c, R, b, (float)dt_dz, dBz, dBy, dBx);
        swap_xz(L); swap_xz(R);
        L.Bz = (float)bz0;
        R.Bz = (float)bz1;
        stf8(m3m_hs(X, 2, 0), SP, f, L);
        stf8(m3m_hs(X, 2, 1), SP, f, R);
    }
    store_v3(A.S.er, SP, f, body_e(w64));
    warp_add_stat(&A.ctl->muscl_first_order, fo);
}

template <int SOLVER, int AX>
__device__ __forceinline__ void m3m_face_flux(const Mhd3DArgs& A, const Mx3M& X, int i, int j, int k, float dtn,
                                              FaceStats* st) {
    const Geo& F = A.FG;
    const long long SP = X.plane;
    const int di = AX == 0, dj = AX == 1, dk = AX == 2;
    const Prim<float> L = ldf8(m3m_hs(X, AX, 1), SP, gidx3(F, i - di, j - dj, k - dk));
    const Prim<float> R = ldf8(m3m_hs(X, AX, 0), SP, gidx3(F, i, j, k));
    Cons<float> Fl;
    face_flux_mixed<true, SOLVER, AX>(L, R, dtn, exact_opts(A.sa), Fl, st);
    stcf8(m3m_flux(X, AX), SP, gidx3(F, i, j, k), Fl);
}

// K2 (box [-2, n+1]^3) and K5 (box [-1, n]^3).
template <int SOLVER, bool FINAL>
__global__ void __launch_bounds__(256, SOLVER == RS_HLLD ? 2 : 3) k_m3m_fluxes(Mhd3DArgs A, Mx3M X) {
    __shared__ int s;
    if (h3_skip(A.ctl, &s)) return;
    int i, j, k;
    const int lo = FINAL ? -1 : -2, hi = FINAL ? 0 : 1;
    if (!m3_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, lo, hi, A.G, i, j, k)) return;
    const double dt = *(const volatile double*)&A.ctl->t1;
    const int f0 = FINAL ? 0 : -1;
    FaceStats st{};
    if (i >= f0) m3m_face_flux<SOLVER, 0>(A, X, i, j, k, (float)(dt / A.sa.dx), &st);
    if (j >= f0) m3m_face_flux<SOLVER, 1>(A, X, i, j, k, (float)(dt / A.sa.dy), &st);
    if (k >= f0) m3m_face_flux<SOLVER, 2>(A, X, i, j, k, (float)(dt / A.sa.dz), &st);
    warp_add_stat(&A.ctl->hlld_to_hlle, st.hlld_to_hlle);
}

// Edge E (CT::computeElectric 3D + CT::upwindElectric 3D) in FP64 from the
// FP32 fluxes, against the FP64 body E eref.
__device__ __forceinline__ V3 m3m_edge_e(const Mhd3DArgs& A, const Mx3M& X, const double* __restrict__ eref, int i,
                                         int j, int k) {
    const Geo& F = A.FG;
    const long long SP = X.plane;
    auto Xf = [&](int a, int b, int c, int q) { return (double)__ldg(X.fx + q * SP + gidx3(F, a, b, c)); };
    auto Yf = [&](int a, int b, int c, int q) { return (double)__ldg(X.fy + q * SP + gidx3(F, a, b, c)); };
    auto Zf = [&](int a, int b, int c, int q) { return (double)__ldg(X.fz + q * SP + gidx3(F, a, b, c)); };
    auto ER = [&](int a, int b, int c) { return m3_ld_v3(eref, SP, gidx3(F, a, b, c)); };
    // flux planes: 0 rho, 1 E, 2-4 momentum, 5 Bx, 6 By, 7 Bz
    V3 e;
    e.x = (Zf(i, j - 1, k, 6) - Yf(i, j, k - 1, 7) + Zf(i, j, k, 6) - Yf(i, j, k, 7)) * 0.25;
    e.y = (Xf(i, j, k - 1, 7) - Zf(i - 1, j, k, 5) + Xf(i, j, k, 7) - Zf(i, j, k, 5)) * 0.25;
    e.z = (Yf(i - 1, j, k, 5) - Xf(i, j - 1, k, 6) + Yf(i, j, k, 5) - Xf(i, j, k, 6)) * 0.25;
    const V3 r000 = ER(i, j, k), r100 = ER(i - 1, j, k), r010 = ER(i, j - 1, k), r001 = ER(i, j, k - 1);
    const V3 r101 = ER(i - 1, j, k - 1), r110 = ER(i - 1, j - 1, k), r011 = ER(i, j - 1, k - 1);
    e.y += upcorr(Xf(i, j, k, 0), -Zf(i - 1, j, k, 5), -Zf(i, j, k, 5), r100.y, r000.y);
    e.y += upcorr(Xf(i, j, k - 1, 0), -Zf(i - 1, j, k, 5), -Zf(i, j, k, 5), r101.y, r001.y);
    e.z += upcorr(Xf(i, j, k, 0), Yf(i - 1, j, k, 5), Yf(i, j, k, 5), r100.z, r000.z);
    e.z += upcorr(Xf(i, j - 1, k, 0), Yf(i - 1, j, k, 5), Yf(i, j, k, 5), r110.z, r010.z);
    e.x += upcorr(Yf(i, j, k, 0), Zf(i, j - 1, k, 6), Zf(i, j, k, 6), r010.x, r000.x);
    e.x += upcorr(Yf(i, j, k - 1, 0), Zf(i, j - 1, k, 6), Zf(i, j, k, 6), r011.x, r001.x);
    e.z += upcorr(Yf(i, j, k, 0), -Xf(i, j - 1, k, 6), -Xf(i, j, k, 6), r010.z, r000.z);
    e.z += upcorr(Yf(i - 1, j, k, 0), -Xf(i, j - 1, k, 6), -Xf(i, j, k, 6), r110.z, r100.z);
    e.x += upcorr(Zf(i, j, k, 0), -Yf(i, j, k - 1, 7), -Yf(i, j, k, 7), r001.x, r000.x);
    e.x += upcorr(Zf(i, j - 1, k, 0), -Yf(i, j, k - 1, 7), -Yf(i, j, k, 7), r011.x, r010.x);
    e.y += upcorr(Zf(i, j, k, 0), Xf(i, j, k - 1, 7), Xf(i, j, k, 7), r001.y, r000.y);
    e.y += upcorr(Zf(i - 1, j, k, 0), Xf(i, j, k - 1, 7), Xf(i, j, k, 7), r101.y, r100.y);
    return e;
}

// K3 (edges [-1, n+1]^3, against the body E of w) and K6 (edges [0, n]^3,
// against the half-step body E).
template <bool FINAL>
__global__ void k_m3m_edges(Mhd3DArgs A, Mx3M X) {
    __shared__ int s;
    if (h3_skip(A.ctl, &s)) return;
    int i, j, k;
    if (!m3_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, FINAL ? 0 : -1, FINAL ? 0 : 1, A.G, i, j, k)) return;
    store_v3(A.S.e0, A.S.plane, gidx3(A.FG, i, j, k), m3m_edge_e(A, X, FINAL ? A.S.eh : A.S.er, i, j, k));
}

// K4: half-step faces (Faraday at dt/2, FP64), the half-step cell (FP64
// accumulation of the FP32 predictor fluxes) with its body E, and the CTU
// corrections of the six half states in FP32 with the energies in FP64.
__global__ void __launch_bounds__(256, 2) k_m3m_half(Mhd3DArgs A, Mx3M X) {
    __shared__ int s;
    if (h3_skip(A.ctl, &s)) return;
    int i, j, k;
    if (!m3_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, -1, 0, A.G, i, j, k)) return;
    const double dt = *(const volatile double*)&A.ctl->t1;
    const double dt_dx = dt / A.sa.dx, dt_dy = dt / A.sa.dy, dt_dz = dt / A.sa.dz;
    const double hdx = 0.5 * dt_dx, hdy = 0.5 * dt_dy, hdz = 0.5 * dt_dz;
    const Geo& G = A.G;
    const Geo& F = A.FG;
    const long long P = G.plane, FP = F.plane, SP = X.plane;
    const long long m = gidx3(F, i, j, k);
    const M3Faces h = m3_faraday(A, i, j, k, hdx, hdy, hdz);
    const Prim<double> W64 = m3_ld_prim(A.w, P, gidx3(G, i, j, k));
    const Cons<float> px0 = ldcf8(X.fx, SP, m), px1 = ldcf8(X.fx, SP, gidx3(F, i + 1, j, k));
    const Cons<float> py0 = ldcf8(X.fy, SP, m), py1 = ldcf8(X.fy, SP, gidx3(F, i, j + 1, k));
    const Cons<float> pz0 = ldcf8(X.fz, SP, m), pz1 = ldcf8(X.fz, SP, gidx3(F, i, j, k + 1));
    {
        // applyFluxes g=1 at dt/2 (Unsplit.cpp:272-288), computeBodyFields, bodyElectric
        Cons<double> U = to_cons64<true>(W64);
        U = c_add<true>(U, c_mul<true>(c_sub<true>(cvt<double>(px0), cvt<double>(px1)), hdx));
        U = c_add<true>(U, c_mul<true>(c_sub<true>(cvt<double>(py0), cvt<double>(py1)), hdy));
        U = c_add<true>(U, c_mul<true>(c_sub<true>(cvt<double>(pz0), cvt<double>(pz1)), hdz));
        if (!is_finite<true>(U)) record_error(A.ctl, ST_NAN, m);
        Prim<double> wh = to_prim64<true>(U);
        wh = body_field(wh, (h.bx0 + h.bx1) * 0.5, (h.by0 + h.by1) * 0.5, (h.bz0 + h.bz1) * 0.5, A.sa.ct_energy);
        store_v3(A.S.eh, SP, m, body_e(wh));
    }
    // CTU corrections (CTU.cpp:66-129)
    const float dBx = (float)((m3_ld(A.B, gidx3(F, i + 1, j, k)) - m3_ld(A.B, m)) * dt_dx);
    const float dBy = (float)((m3_ld(A.B, FP + gidx3(F, i, j + 1, k)) - m3_ld(A.B, FP + m)) * dt_dy);
    const float dBz = (float)((m3_ld(A.B, 2 * FP + gidx3(F, i, j, k + 1)) - m3_ld(A.B, 2 * FP + m)) * dt_dz);
    const Prim<float> W = f32_prim8(W64);
    const float fdx = (float)dt_dx, fdy = (float)dt_dy, fdz = (float)dt_dz;
    const float e8 = (float)k1_8pi;
    auto E0 = [&](int a, int b, int c) { return m3_ld_v3(A.S.e0, A.S.plane, gidx3(F, a, b, c)); };
    auto apply = [&](int axis, Cons<float> corr, double bl, double br) {
        float* pl = m3m_hs(X, axis, 0);
        float* pr = m3m_hs(X, axis, 1);
        const Prim<float> sL = ldf8_rw(pl, SP, m), sR = ldf8_rw(pr, SP, m);
        Cons<float> uL = c_add<true>(to_cons<true>(sL), corr);
        Cons<float> uR = c_add<true>(to_cons<true>(sR), corr);
        if (axis == 0) { uL.Bx = (float)bl; uR.Bx = (float)br; }
        else if (axis == 1) { uL.By = (float)bl; uR.By = (float)br; }
        else { uL.Bz = (float)bl; uR.Bz = (float)br; }
        stf8(pl, SP, m, prim_from<true>(uL, energy64<true>(sL) + (double)corr.E));
        stf8(pr, SP, m, prim_from<true>(uR, energy64<true>(sR) + (double)corr.E));
    };
    {   // x states
        Cons<float> corr = c_mul<true>(c_add<true>(c_mul<true>(c_sub<true>(py0, py1), fdy),
                                                    c_mul<true>(c_sub<true>(pz0, pz1), fdz)), 0.5f);
        corr.Bx = corr.By = corr.Bz = 0.f;
        const float lim_y = lim_minmod(-dBz, dBx), lim_z = lim_minmod(-dBy, dBx);
        corr.E += e8 * (W.By * W.vy * lim_y + W.Bz * W.vz * lim_z);
        corr.By = (float)(-0.25 * dt_dz * (E0(i, j, k + 1).x - E0(i, j, k).x + E0(i, j + 1, k + 1).x - E0(i, j + 1, k).x)) +
                  0.5f * W.vy * lim_y;
        corr.Bz = (float)(0.25 * dt_dy * (E0(i, j + 1, k).x - E0(i, j, k).x + E0(i, j + 1, k + 1).x - E0(i, j, k + 1).x)) +
                  0.5f * W.vz * lim_z;
        apply(0, corr, h.bx0, h.bx1);
    }
    {   // y states
        Cons<float> corr = c_mul<true>(c_add<true>(c_mul<true>(c_sub<true>(px0, px1), fdx),
                                                    c_mul<true>(c_sub<true>(pz0, pz1), fdz)), 0.5f);
        corr.Bx = corr.By = corr.Bz = 0.f;
        const float lim_x = lim_minmod(-dBz, dBy), lim_z = lim_minmod(-dBx, dBy);
        corr.E += e8 * (W.Bx * W.vx * lim_x + W.Bz * W.vz * lim_z);
        corr.Bx = (float)(0.25 * dt_dz * (E0(i, j, k + 1).y - E0(i, j, k).y + E0(i + 1, j, k + 1).y - E0(i + 1, j, k).y)) +
                  0.5f * W.vx * lim_x;
        corr.Bz = (float)(-0.25 * dt_dx * (E0(i + 1, j, k).y - E0(i, j, k).y + E0(i + 1, j, k + 1).y - E0(i, j, k + 1).y)) +
                  0.5f * W.vz * lim_z;
        apply(1, corr, h.by0, h.by1);
    }
    {   // z states
        Cons<float> corr = c_mul<true>(c_add<true>(c_mul<true>(c_sub<true>(px0, px1), fdx),
                                                    c_mul<true>(c_sub<true>(py0, py1), fdy)), 0.5f);
        corr.Bx = corr.By = corr.Bz = 0.f;
        const float lim_x = lim_minmod(-dBy, dBz), lim_y = lim_minmod(-dBx, dBz);
        corr.E += e8 * (W.Bx * W.vx * lim_x + W.By * W.vy * lim_y);
        corr.Bx = (float)(-0.25 * dt_dy * (E0(i, j + 1, k).z - E0(i, j, k).z + E0(i + 1, j + 1, k).z - E0(i + 1, j, k).z)) +
                  0.5f * W.vx * lim_x;
        corr.By = (float)(0.25 * dt_dx * (E0(i + 1, j, k).z - E0(i, j, k).z + E0(i + 1, j + 1, k).z - E0(i, j + 1, k).z)) +
                  0.5f * W.vy * lim_y;
        apply(2, corr, h.bz0, h.bz1);
    }
}

// K7: interior cells: FP64 update with the FP32 final fluxes, Faraday on the
// faces the cell owns (FP64), face -> cell B with the energy gate,
// physicality, CFL speed.
__global__ void __launch_bounds__(256) k_m3m_update(Mhd3DArgs A, Mx3M X) {
    __shared__ int s;
    __shared__ double red[32];
    if (h3_skip(A.ctl, &s)) return;
    int i = 0, j = 0, k = 0;
    const bool in = m3_cell(blockIdx.x * (long long)blockDim.x + threadIdx.x, 0, -1, A.G, i, j, k);
    double vmax = 0.0;
    if (in) {
        const double dt = *(const volatile double*)&A.ctl->t1;
        const double d[3] = {dt / A.sa.dx, dt / A.sa.dy, dt / A.sa.dz};
        const Geo& G = A.G;
        const Geo& F = A.FG;
        const long long P = G.plane, FP = F.plane, SP = X.plane;
        const int nx = G.n[0], ny = G.n[1], nz = G.n[2];
        const long long mc = gidx3(G, i, j, k), mf = gidx3(F, i, j, k);
        const M3Faces b = m3_faraday(A, i, j, k, d[0], d[1], d[2]);
        Cons<double> U = to_cons64<true>(m3_ld_prim(A.w, P, mc));
        const long long up[3] = {gidx3(F, i + 1, j, k), gidx3(F, i, j + 1, k), gidx3(F, i, j, k + 1)};
        double* u8[8] = {&U.rho, &U.E, &U.mx, &U.my, &U.mz, &U.Bx, &U.By, &U.Bz};
#pragma unroll
        for (int ax = 0; ax < 3; ax++) {
            const float* Fl = m3m_flux(X, ax);
#pragma unroll
            for (int q = 0; q < 8; q++)
                *u8[q] += ((double)__ldg(Fl + q * SP + mf) - (double)__ldg(Fl + q * SP + up[ax])) * d[ax];
        }
        if (!is_finite<true>(U)) record_error(A.ctl, ST_NAN, mc);
        Prim<double> nw = body_field(to_prim64<true>(U), (b.bx0 + b.bx1) * 0.5, (b.by0 + b.by1) * 0.5,
                                     (b.bz0 + b.bz1) * 0.5, A.sa.ct_energy);
        if (!is_physical<true>(nw)) record_error(A.ctl, ST_UNPHYSICAL, mc);
        store_prim<true>(A.wout, P, mc, nw);
        A.Bout[mf] = b.bx0;
        A.Bout[FP + mf] = b.by0;
        A.Bout[2 * FP + mf] = b.bz0;
        if (i == nx - 1) A.Bout[gidx3(F, nx, j, k)] = b.bx1;
        if (j == ny - 1) A.Bout[FP + gidx3(F, i, ny, k)] = b.by1;
        if (k == nz - 1) A.Bout[2 * FP + gidx3(F, i, j, nz)] = b.bz1;
        vmax = cfl_speed_mx<true>(nw, A.sa.cfl, A.sa.dx, A.sa.dy, A.sa.dz);
    }
    vmax = block_max(vmax, red);
    if (threadIdx.x == 0) atomic_max_speed(&A.ctl->vmax[A.sa.slot_out], vmax);
}

template <int SOLVER>
int go(const Geo& G, const Geo& FG, const double* w, double* wout, const double* B, double* Bout, const Mhd3DScratch& S,
       StepCtl* ctl, const StepArgs& sa, cudaStream_t st) {
    Mhd3DArgs A{G, FG, w, wout, B, Bout, S, ctl, sa};
    const Mx3M X{reinterpret_cast<float*>(S.hs), reinterpret_cast<float*>(S.fx), reinterpret_cast<float*>(S.fy),
                 reinterpret_cast<float*>(S.fz), S.plane};
    auto blocks = [&](int lo, int hi) {
        const long long n = (long long)(G.n[0] + hi - lo + 1) * (G.n[1] + hi - lo + 1) * (G.n[2] + hi - lo + 1);
        return (int)((n + 255) / 256);
    };
    if (cudaMemcpyAsync(wout, w, sizeof(double) * 8 * G.plane, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return 1;
    if (cudaMemcpyAsync(Bout, B, sizeof(double) * 3 * FG.plane, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return 1;
    k_m3m_halfstates<<<blocks(-2, 1), 256, 0, st>>>(A, X);
    k_m3m_fluxes<SOLVER, false><<<blocks(-2, 1), 256, 0, st>>>(A, X);
    k_m3m_edges<false><<<blocks(-1, 1), 256, 0, st>>>(A, X);
    k_m3m_half<<<blocks(-1, 0), 256, 0, st>>>(A, X);
    k_m3m_fluxes<SOLVER, true><<<blocks(-1, 0), 256, 0, st>>>(A, X);
    k_m3m_edges<true><<<blocks(0, 0), 256, 0, st>>>(A, X);
    k_m3m_update<<<blocks(0, -1), 256, 0, st>>>(A, X);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace

int launch_step3d_mhd_mixed(int solver, const Geo& G, const Geo& FG, const double* w, double* wout, const double* B,
                            double* Bout, const Mhd3DScratch& S, StepCtl* ctl, const StepArgs& sa, cudaStream_t st) {
    switch (solver) {
        case RS_HLL: return go<RS_HLL>(G, FG, w, wout, B, Bout, S, ctl, sa, st);
        case RS_HLLE: return go<RS_HLLE>(G, FG, w, wout, B, Bout, S, ctl, sa, st);
        default: return go<RS_HLLD>(G, FG, w, wout, B, Bout, S, ctl, sa, st);
    }
}

}  // namespace dgpu
