// Fused mixed FP32/FP64 2D MHD CTU + CT step: the whole step in one kernel.
//
// A CTA owns a strip of TJ output columns and a segment of rows, and marches
// down the segment R rows at a time. Each iteration runs every phase of the
// step on R new rows, each phase a fixed number of rows ahead of the one that
// consumes it:
//   S0 load w (FP64 -> FP32) and its body E           rows a+3 .. a+R+2
//   S1 MUSCL-Hancock half states (x and y)            rows a+2 .. a+R+1
//   S2 predictor fluxes (x faces, y faces)            rows a+2 .. a+R+1
//   S3 predictor corner E                             rows a+2 .. a+R+1
//   S4 half step: CT half update of the faces, the
//      half-step cells and their body E, the CTU
//      corrections of the half states (in place)      rows a+1 .. a+R
//   S5 final fluxes                                   rows a+1 .. a+R
//   S6 final corner E                                 rows a+1 .. a+R
//   S7 conservative update + Faraday + cell B          rows a   .. a+R-1
// so every intermediate is produced once, lives in a shared-memory ring of
// R+1 or R+2 rows and never goes to HBM: the step reads the state and face B
// and writes them back (plus re-reads of recently loaded rows, which hit L2).
// Only the strip's side columns are computed twice (by both neighbouring
// strips): two extra columns per side for the half states, fewer for the
// later phases. Iterations before the segment fill the rings.
//
// The arithmetic of every phase is that of step_mhd_mixed.cuh (FP32
// reconstruction, limiters, Riemann fluxes and CTU corrections; FP64 energies
// and pressure recovery, half-step and final updates, corner E and Faraday),
// and every phase covers exactly the reference's index ranges
// (ctu_sweep_MHD 2D, CTU.cpp:133-203; computeFlux_X/Y, Unsplit.cpp:58-60;
// CT::computeElectric / upwindElectric, Electric.cpp:24-74; CT::Faraday,
// B_fields.cpp:21-40; applyFluxes, Unsplit.cpp:256-270): the segment and strip
// bounds clip each phase's rows and columns to those ranges at the grid edges.
#pragma once

#include "step_mhd_mixed.cuh"

namespace dgpu {

// Strips of kFuseTJ columns marching kFuseR rows per iteration, kFuseNT threads.
// Each phase's items per iteration (rows x its column window) against the
// 256 threads: with 28 columns every phase fills its last round of threads
// well (S2 504 and S5 472 solves: two rounds each; S3, S6, S7 one round),
// where 32 columns left rounds of 24 to 56 items in five phases. Measured on
// Orszag-Tang 1024^2: 0.432 ms per step against 0.496 ms with 32 columns
// (24 columns: 0.518 ms; 6 rows x 32 columns: 0.462 ms).
constexpr int kFuseTJ = 28, kFuseR = 8, kFuseNT = 256;

template <int TJ, int R>
struct FusedMhdSmem {
    static constexpr int KW = R + 2;  // rows of w (FP32) and its body E
    static constexpr int KH = R + 2;  // rows of half states
    static constexpr int K1 = R + 1;  // rows of every other ring
    // columns of each ring and the global column of its first entry (from j0)
    static constexpr int CW = TJ + 6, OW = -3;    // w
    static constexpr int CH = TJ + 4, OH = -2;    // body E of w, half states, predictor x fluxes
    static constexpr int CY = TJ + 3, OY = -1;    // predictor y fluxes, predictor corner E
    static constexpr int CC = TJ + 2, OC = -1;    // half-step body E, final x fluxes
    static constexpr int CF = TJ + 1, OF = 0;     // final y fluxes, final corner E
    float w[KW][8][CW];
    float er[KW][3][CH];
    float hs[KH][32][CH];    // per cell: xL 0-7, xR 8-15, yL 16-23, yR 24-31 (rho, p, vx, vy, vz, Bx, By, Bz)
    float px[K1][8][CH];     // predictor x-face fluxes (rho, E, mx, my, mz, Bx, By, Bz)
    float py[K1][8][CY];
    float e0[K1][3][CY];
    float eh[K1][3][CC];
    float fx[K1][8][CC];
    float fy[K1][8][CF];
    float ec[K1][3][CF];
    double red[32];
    int skip;
};

template <int K>
__device__ __forceinline__ int ring(int r) {
    return (r + 64 * K) % K;  // rows are >= -3
}

template <int TJ, int R>
__device__ __forceinline__ Prim<float> fm_hs(const FusedMhdSmem<TJ, R>& S, int row, int k, int c) {
    const int s = ring<FusedMhdSmem<TJ, R>::KH>(row);
    const int b = 8 * k;
    return Prim<float>{S.hs[s][b][c],     S.hs[s][b + 1][c], S.hs[s][b + 2][c], S.hs[s][b + 3][c],
                       S.hs[s][b + 4][c], S.hs[s][b + 5][c], S.hs[s][b + 6][c], S.hs[s][b + 7][c]};
}
template <int TJ, int R>
__device__ __forceinline__ void fm_put_hs(FusedMhdSmem<TJ, R>& S, int row, int k, int c, const Prim<float>& p) {
    const int s = ring<FusedMhdSmem<TJ, R>::KH>(row);
    const int b = 8 * k;
    S.hs[s][b][c] = p.rho; S.hs[s][b + 1][c] = p.p; S.hs[s][b + 2][c] = p.vx; S.hs[s][b + 3][c] = p.vy;
    S.hs[s][b + 4][c] = p.vz; S.hs[s][b + 5][c] = p.Bx; S.hs[s][b + 6][c] = p.By; S.hs[s][b + 7][c] = p.Bz;
}
template <int C>
__device__ __forceinline__ void fm_put8(float (*a)[C], int c, const Cons<float>& u) {
    a[0][c] = u.rho; a[1][c] = u.E; a[2][c] = u.mx; a[3][c] = u.my; a[4][c] = u.mz;
    a[5][c] = u.Bx; a[6][c] = u.By; a[7][c] = u.Bz;
}
template <int C>
__device__ __forceinline__ Cons<double> fm_get8(const float (*a)[C], int c) {
    Cons<double> u;
    u.rho = a[0][c]; u.E = a[1][c]; u.mx = a[2][c]; u.my = a[3][c]; u.mz = a[4][c];
    u.Bx = a[5][c]; u.By = a[6][c]; u.Bz = a[7][c];
    return u;
}
template <int C>
__device__ __forceinline__ void fm_put3(float (*a)[C], int c, const V3& v) {
    a[0][c] = (float)v.x; a[1][c] = (float)v.y; a[2][c] = (float)v.z;
}
template <int C>
__device__ __forceinline__ V3 fm_get3(const float (*a)[C], int c) {
    return V3{a[0][c], a[1][c], a[2][c]};
}

// corner_e_mx (step_mhd_mixed.cuh) on ring entries: FX(row, col, comp) and
// FY(row, col, comp) read the x / y face fluxes, ER(row, col) the body E.
template <class FXf, class FYf, class ERf>
__device__ __forceinline__ V3 fm_corner_e(int i, int j, FXf FX, FYf FY, ERf ER) {
    V3 e;
    e.x = -FY(i, j, 7);
    e.y = FX(i, j, 7);
    e.z = (FY(i - 1, j, 5) - FX(i, j - 1, 6) + FY(i, j, 5) - FX(i, j, 6)) * 0.25;
    const V3 r00 = ER(i, j), r10 = ER(i - 1, j), r01 = ER(i, j - 1), r11 = ER(i - 1, j - 1);
    e.z += upcorr(FX(i, j, 0), FY(i - 1, j, 5), FY(i, j, 5), r10.z, r00.z);
    e.z += upcorr(FX(i, j - 1, 0), FY(i - 1, j, 5), FY(i, j, 5), r11.z, r01.z);
    e.z += upcorr(FY(i, j, 0), -FX(i, j - 1, 6), -FX(i, j, 6), r01.z, r00.z);
    e.z += upcorr(FY(i - 1, j, 0), -FX(i, j - 1, 6), -FX(i, j, 6), r11.z, r10.z);
    e.x += 0.25 * (-2 * FY(i, j, 7) - r00.x - r01.x);
    e.y += 0.25 * (2 * FX(i, j, 7) - r00.y - r10.y);
    return e;
}

// Rows [lo, hi) of a phase at iteration a: [a + off, a + R + off) clipped to
// the rows the segment [sb, se) needs from it, [first, se + off). The march
// starts at a = sb - kFill(R), early enough that the filling iterations reach
// every phase's first row (w is needed from sb - 3 at offset 3).
struct RowSpan {
    int lo, hi;
};
template <int R>
__device__ __forceinline__ RowSpan span_of(int a, int se, int off, int first) {
    RowSpan s;
    s.hi = min(a + R + off, se + off);
    s.lo = max(a + off, first);
    return s;
}
template <int R>
constexpr int kFill = R * ((6 + R - 1) / R);

// The step of one strip (columns from strip * TJ) and one segment (rows from
// seg * seg_rows) of one grid, run by the calling CTA; `cta` of `ctas` is the
// CTA's place among all CTAs stepping this grid (they share the ghost-frame
// copy). CTA-uniform early returns only.
template <int SOLVER, int TJ, int R, int NT>
__device__ __forceinline__ void mhd2d_fused_body(const Geo& G, const Geo& FG, const double* __restrict__ w,
                                                 double* __restrict__ wout, const double* __restrict__ B,
                                                 double* __restrict__ Bout, StepCtl* ctl, const StepArgs& sa,
                                                 int seg_rows, int strip, int seg, long long cta, long long ctas,
                                                 FusedMhdSmem<TJ, R>& S) {
    using S_t = FusedMhdSmem<TJ, R>;
    if (mhd_skip(ctl, &S.skip)) return;
    // The ghost frame of the output buffers (every point the update does not
    // write) is copied from the inputs by all CTAs, before any returns early.
    mhd2d_copy_frame(G, FG, w, wout, B, Bout, 0, mhd2d_frame_points(G.n[0], G.n[1], G.g), cta * NT + threadIdx.x,
                     ctas * NT);

    const int nx = G.n[0], ny = G.n[1];
    const long long P = G.plane, FP = FG.plane;
    const int j0 = strip * TJ;
    const int sb = seg * seg_rows, se = min(sb + seg_rows, nx);
    if (sb >= se) return;
    const double dt = *(const volatile double*)&ctl->t1;
    const double dt_dx = dt / sa.dx, dt_dy = dt / sa.dy, hdx = 0.5 * dt_dx, hdy = 0.5 * dt_dy;
    const float fdx = (float)dt_dx, fdy = (float)dt_dy;
    const ExactOpts eo = exact_opts(sa);
    FaceStats st{};
    int fo = 0;
    double vmax = 0.0;

    // column windows of each phase, clipped to the reference's ranges
    const int cw_lo = max(j0 - 3, -3), cw_hi = min(j0 + TJ + 3, ny + 3);   // w
    const int ch_lo = max(j0 - 2, -2), ch_hi = min(j0 + TJ + 2, ny + 2);   // half states, x predictor, body E of w
    const int cy_lo = max(j0 - 1, -1), cy_hi = min(j0 + TJ + 2, ny + 2);   // y predictor faces, predictor corners
    const int cc_lo = max(j0 - 1, -1), cc_hi = min(j0 + TJ + 1, ny + 1);   // half-step cells, final x faces
    const int cf_lo = max(j0, 0), cf_hi = min(j0 + TJ + 1, ny + 1);        // final y faces, final corners
    const int cu_hi = min(j0 + TJ, ny);                                       // updated cells

    auto gF = [&](int i, int j) { return gidx2(FG, i, j); };

    for (int a = sb - kFill<R>; a < se; a += R) {
        // ---- S0: w rows (FP64 -> FP32 ring) and the body E of w
        {
            const RowSpan rs = span_of<R>(a, se, 3, sb - 3);
            const int n = (rs.hi - rs.lo) * S_t::CW;
            for (int t = threadIdx.x; t < n; t += NT) {
                const int i = rs.lo + t / S_t::CW, c = t % S_t::CW, j = j0 + S_t::OW + c;
                if (j < cw_lo || j >= cw_hi) continue;
                const Prim<double> q = load_prim<true>(w, P, gidx2(G, i, j));
                const int s = ring<S_t::KW>(i);
                S.w[s][0][c] = (float)q.rho; S.w[s][1][c] = (float)q.p; S.w[s][2][c] = (float)q.vx;
                S.w[s][3][c] = (float)q.vy; S.w[s][4][c] = (float)q.vz; S.w[s][5][c] = (float)q.Bx;
                S.w[s][6][c] = (float)q.By; S.w[s][7][c] = (float)q.Bz;
                const int ce = c + S_t::OW - S_t::OH;
                if (j >= ch_lo && j < ch_hi && ce >= 0 && ce < S_t::CH) fm_put3(S.er[s], ce, body_e(q));
            }
        }
        __syncthreads();
        // ---- S1: half states, one item per (cell, direction): x items first
        {
            const RowSpan rs = span_of<R>(a, se, 2, sb - 2);
            const int nc = (rs.hi - rs.lo) * S_t::CH;
            for (int t = threadIdx.x; t < 2 * nc; t += NT) {
                const bool yd = t >= nc;
                const int q = yd ? t - nc : t;
                const int i = rs.lo + q / S_t::CH, c = q % S_t::CH, j = j0 + S_t::OH + c;
                if (j < ch_lo || j >= ch_hi) continue;
                const int cw = c + S_t::OH - S_t::OW;
                auto W = [&](int ii, int cc) {
                    const int s = ring<S_t::KW>(ii);
                    return Prim<float>{S.w[s][0][cc], S.w[s][1][cc], S.w[s][2][cc], S.w[s][3][cc],
                                       S.w[s][4][cc], S.w[s][5][cc], S.w[s][6][cc], S.w[s][7][cc]};
                };
                const double bx0 = B[gF(i, j)], bx1 = B[gF(i + 1, j)];
                const double by0 = B[FP + gF(i, j)], by1 = B[FP + gF(i, j + 1)];
                const float dBx = (float)((bx1 - bx0) * dt_dx), dBy = (float)((by1 - by0) * dt_dy);
                Prim<float> l = yd ? W(i, cw - 1) : W(i - 1, cw), wc = W(i, cw), r = yd ? W(i, cw + 1) : W(i + 1, cw);
                if (yd) { swap_xy(l); swap_xy(wc); swap_xy(r); }
                Prim<float> L, Rr;
                // y: the swapped source terms, dB.y from the x faces and dB.x from the y faces
                fo += !muscl_mixed<true>(sa.limiter, l, L, wc, Rr, r, yd ? fdy : fdx, yd ? dBy : dBx, yd ? dBx : dBy, 0.f);
                if (yd) {
                    swap_xy(L); swap_xy(Rr);
                    L.By = (float)by0;
                    Rr.By = (float)by1;
                } else {
                    L.Bx = (float)bx0;
                    Rr.Bx = (float)bx1;
                }
                fm_put_hs(S, i, yd ? 2 : 0, c, L);
                fm_put_hs(S, i, yd ? 3 : 1, c, Rr);
            }
        }
        __syncthreads();
        // ---- S2: predictor fluxes, x faces (rows from sb-1) then y faces (rows
        // from sb-2), one Riemann code path: y faces solve on swapped states
        {
            const RowSpan rx = span_of<R>(a, se, 2, sb - 1), ry = span_of<R>(a, se, 2, sb - 2);
            const int nxf = (rx.hi - rx.lo) * S_t::CH, nyf = (ry.hi - ry.lo) * S_t::CY;
            for (int t = threadIdx.x; t < nxf + nyf; t += NT) {
                const bool yd = t >= nxf;
                const int q = yd ? t - nxf : t;
                const int C = yd ? S_t::CY : S_t::CH;
                const int i = (yd ? ry.lo : rx.lo) + q / C, c = q % C;
                const int j = j0 + (yd ? S_t::OY : S_t::OH) + c;
                if (yd ? (j < cy_lo || j >= cy_hi) : (j < ch_lo || j >= ch_hi)) continue;
                const int ch = j - j0 - S_t::OH;  // half-state column of cell j
                Prim<float> L = yd ? fm_hs(S, i, 3, ch - 1) : fm_hs(S, i - 1, 1, ch);
                Prim<float> Rr = yd ? fm_hs(S, i, 2, ch) : fm_hs(S, i, 0, ch);
                if (yd) { swap_xy(L); swap_xy(Rr); }
                Cons<float> Fl;
                face_flux_mixed<true, SOLVER, 0>(L, Rr, yd ? fdy : fdx, eo, Fl, &st);
                if (yd) {
                    swap_xy(Fl);
                    fm_put8(S.py[ring<S_t::K1>(i)], c, Fl);
                } else {
                    fm_put8(S.px[ring<S_t::K1>(i)], c, Fl);
                }
            }
        }
        __syncthreads();
        // ---- S3: predictor corner E against the body E of w
        {
            const RowSpan rs = span_of<R>(a, se, 2, sb - 1);
            const int n = (rs.hi - rs.lo) * S_t::CY;
            for (int t = threadIdx.x; t < n; t += NT) {
                const int i = rs.lo + t / S_t::CY, c = t % S_t::CY, j = j0 + S_t::OY + c;
                if (j < cy_lo || j >= cy_hi) continue;
                auto FX = [&](int ii, int jj, int k) {
                    return (double)S.px[ring<S_t::K1>(ii)][k][jj - j0 - S_t::OH];
                };
                auto FY = [&](int ii, int jj, int k) {
                    return (double)S.py[ring<S_t::K1>(ii)][k][jj - j0 - S_t::OY];
                };
                auto ER = [&](int ii, int jj) { return fm_get3(S.er[ring<S_t::KW>(ii)], jj - j0 - S_t::OH); };
                fm_put3(S.e0[ring<S_t::K1>(i)], c, fm_corner_e(i, j, FX, FY, ER));
            }
        }
        __syncthreads();
        // ---- S4: half step and CTU corrections (mx_half of step_mhd_mixed.cuh),
        // three items per cell: the x half states' correction, the y half
        // states' correction (one code path on selected operands), the
        // half-step cell's body E
        {
            const RowSpan rs = span_of<R>(a, se, 1, sb - 1);
            const int nc = (rs.hi - rs.lo) * S_t::CC;
            for (int t = threadIdx.x; t < 3 * nc; t += NT) {
                const int kind = t / nc, q = t - kind * nc;
                const int i = rs.lo + q / S_t::CC, c = q % S_t::CC, j = j0 + S_t::OC + c;
                if (j < cc_lo || j >= cc_hi) continue;
                const int cy = j - j0 - S_t::OY, ch = j - j0 - S_t::OH;
                auto E0 = [&](int ii, int cc) { return fm_get3(S.e0[ring<S_t::K1>(ii)], cc); };
                const V3 e00 = E0(i, cy), e10 = E0(i + 1, cy), e01 = E0(i, cy + 1), e11 = E0(i + 1, cy + 1);
                const long long m = gF(i, j);
                const double bx0 = B[m], bx1 = B[gF(i + 1, j)], by0 = B[FP + m], by1 = B[FP + gF(i, j + 1)];
                const double bxh0 = bx0 - (e01.z - e00.z) * hdy;
                const double bxh1 = bx1 - (e11.z - e10.z) * hdy;
                const double byh0 = by0 - -(e10.z - e00.z) * hdx;
                const double byh1 = by1 - -(e11.z - e01.z) * hdx;
                const long long mc = gidx2(G, i, j);
                if (kind == 2) {
                    const double bzh = B[2 * FP + m] - ((e10.y - e00.y) * hdx - (e01.x - e00.x) * hdy);
                    const Prim<double> W = load_prim<true>(w, P, mc);
                    const Cons<double> px0 = fm_get8(S.px[ring<S_t::K1>(i)], ch), px1 = fm_get8(S.px[ring<S_t::K1>(i + 1)], ch);
                    const Cons<double> py0 = fm_get8(S.py[ring<S_t::K1>(i)], cy), py1 = fm_get8(S.py[ring<S_t::K1>(i)], cy + 1);
                    Cons<double> U = to_cons64<true>(W);
                    U = c_add<true>(U, c_mul<true>(c_sub<true>(px0, px1), hdx));
                    U = c_add<true>(U, c_mul<true>(c_sub<true>(py0, py1), hdy));
                    if (!is_finite<true>(U)) record_error(ctl, ST_NAN, m);
                    Prim<double> wh = to_prim64<true>(U);
                    wh = body_field64(wh, (bxh0 + bxh1) * 0.5, (byh0 + byh1) * 0.5, bzh, sa.ct_energy);
                    fm_put3(S.eh[ring<S_t::K1>(i)], c, body_e(wh));
                    continue;
                }
                const bool yd = kind == 1;
                const double Wvz = w[4 * P + mc], WBz = w[7 * P + mc];
                const double dBx = (bx1 - bx0) * dt_dx, dBy = (by1 - by0) * dt_dy;
                // x half states: the y fluxes' difference; y half states: the x fluxes'
                const Cons<double> p0 = yd ? fm_get8(S.px[ring<S_t::K1>(i)], ch) : fm_get8(S.py[ring<S_t::K1>(i)], cy);
                const Cons<double> p1 = yd ? fm_get8(S.px[ring<S_t::K1>(i + 1)], ch) : fm_get8(S.py[ring<S_t::K1>(i)], cy + 1);
                Cons<double> corr = c_mul<true>(c_mul<true>(c_sub<true>(p0, p1), 0.5), yd ? dt_dx : dt_dy);
                corr.Bx = corr.By = corr.Bz = 0;
                const double lim_z = yd ? lim_minmod(-dBx, dBy) : lim_minmod(-dBy, dBx);
                corr.E += k1_8pi * (WBz * Wvz * lim_z);
                corr.Bz = yd ? -0.5 * dt_dx * (e10.y - e00.y) + 0.5 * Wvz * lim_z
                             : 0.5 * dt_dy * (e01.x - e00.x) + 0.5 * Wvz * lim_z;
                const int k = yd ? 2 : 0;
                const Prim<float> hl = fm_hs(S, i, k, ch), hr = fm_hs(S, i, k + 1, ch);
                const Cons<float> cf = cvt<float>(corr);
                Cons<float> ul = c_add<true>(to_cons<true>(hl), cf), ur = c_add<true>(to_cons<true>(hr), cf);
                if (yd) { ul.By = (float)byh0; ur.By = (float)byh1; }
                else { ul.Bx = (float)bxh0; ur.Bx = (float)bxh1; }
                fm_put_hs(S, i, k, ch, prim_from<true>(ul, energy64<true>(hl) + corr.E));
                fm_put_hs(S, i, k + 1, ch, prim_from<true>(ur, energy64<true>(hr) + corr.E));
            }
        }
        __syncthreads();
        // ---- S5: final fluxes, x faces (rows from sb) then y faces (rows from
        // sb-1), one Riemann code path as in S2
        {
            const RowSpan rx = span_of<R>(a, se, 1, sb), ry = span_of<R>(a, se, 1, sb - 1);
            const int nxf = (rx.hi - rx.lo) * S_t::CC, nyf = (ry.hi - ry.lo) * S_t::CF;
            for (int t = threadIdx.x; t < nxf + nyf; t += NT) {
                const bool yd = t >= nxf;
                const int q = yd ? t - nxf : t;
                const int C = yd ? S_t::CF : S_t::CC;
                const int i = (yd ? ry.lo : rx.lo) + q / C, c = q % C;
                const int j = j0 + (yd ? S_t::OF : S_t::OC) + c;
                if (yd ? (j < cf_lo || j >= cf_hi) : (j < cc_lo || j >= cc_hi)) continue;
                const int ch = j - j0 - S_t::OH;
                Prim<float> L = yd ? fm_hs(S, i, 3, ch - 1) : fm_hs(S, i - 1, 1, ch);
                Prim<float> Rr = yd ? fm_hs(S, i, 2, ch) : fm_hs(S, i, 0, ch);
                if (yd) { swap_xy(L); swap_xy(Rr); }
                Cons<float> Fl;
                face_flux_mixed<true, SOLVER, 0>(L, Rr, yd ? fdy : fdx, eo, Fl, &st);
                if (yd) {
                    swap_xy(Fl);
                    fm_put8(S.fy[ring<S_t::K1>(i)], c, Fl);
                } else {
                    fm_put8(S.fx[ring<S_t::K1>(i)], c, Fl);
                }
            }
        }
        __syncthreads();
        // ---- S6: final corner E against the half-step body E
        {
            const RowSpan rs = span_of<R>(a, se, 1, sb);
            const int n = (rs.hi - rs.lo) * S_t::CF;
            for (int t = threadIdx.x; t < n; t += NT) {
                const int i = rs.lo + t / S_t::CF, c = t % S_t::CF, j = j0 + S_t::OF + c;
                if (j < cf_lo || j >= cf_hi) continue;
                auto FX = [&](int ii, int jj, int k) {
                    return (double)S.fx[ring<S_t::K1>(ii)][k][jj - j0 - S_t::OC];
                };
                auto FY = [&](int ii, int jj, int k) {
                    return (double)S.fy[ring<S_t::K1>(ii)][k][jj - j0 - S_t::OF];
                };
                auto ER = [&](int ii, int jj) { return fm_get3(S.eh[ring<S_t::K1>(ii)], jj - j0 - S_t::OC); };
                fm_put3(S.ec[ring<S_t::K1>(i)], c, fm_corner_e(i, j, FX, FY, ER));
            }
        }
        __syncthreads();
        // ---- S7: update + Faraday + cell B (mx_update of step_mhd_mixed.cuh)
        {
            const RowSpan rs = span_of<R>(a, se, 0, sb);
            const int n = (rs.hi - rs.lo) * TJ;
            for (int t = threadIdx.x; t < n; t += NT) {
                const int i = rs.lo + t / TJ, c = t % TJ, j = j0 + c;
                if (j >= cu_hi) continue;
                auto E = [&](int ii, int cc) { return fm_get3(S.ec[ring<S_t::K1>(ii)], cc); };
                const V3 e00 = E(i, c), e10 = E(i + 1, c), e01 = E(i, c + 1), e11 = E(i + 1, c + 1);
                const long long mf = gF(i, j), mc = gidx2(G, i, j);
                const double bx0 = B[mf] - (e01.z - e00.z) * dt_dy;
                const double bx1 = B[gF(i + 1, j)] - (e11.z - e10.z) * dt_dy;
                const double by0 = B[FP + mf] - -(e10.z - e00.z) * dt_dx;
                const double by1 = B[FP + gF(i, j + 1)] - -(e11.z - e01.z) * dt_dx;
                const double bz = B[2 * FP + mf] - ((e10.y - e00.y) * dt_dx - (e01.x - e00.x) * dt_dy);
                const int cx = j - j0 - S_t::OC;
                Cons<double> U = to_cons64<true>(load_prim<true>(w, P, mc));
                U = c_add<true>(U, c_mul<true>(c_sub<true>(fm_get8(S.fx[ring<S_t::K1>(i)], cx),
                                                           fm_get8(S.fx[ring<S_t::K1>(i + 1)], cx)), dt_dx));
                U = c_add<true>(U, c_mul<true>(c_sub<true>(fm_get8(S.fy[ring<S_t::K1>(i)], c),
                                                           fm_get8(S.fy[ring<S_t::K1>(i)], c + 1)), dt_dy));
                if (!is_finite<true>(U)) record_error(ctl, ST_NAN, mc);
                Prim<double> nw = body_field64(to_prim64<true>(U), (bx0 + bx1) * 0.5, (by0 + by1) * 0.5, bz, sa.ct_energy);
                if (!is_physical<true>(nw)) record_error(ctl, ST_UNPHYSICAL, mc);
                store_prim<true>(wout, P, mc, nw);
                Bout[mf] = bx0;
                Bout[FP + mf] = by0;
                Bout[2 * FP + mf] = bz;
                if (i == nx - 1) Bout[gF(nx, j)] = bx1;
                if (j == ny - 1) Bout[FP + gF(i, ny)] = by1;
                vmax = speed_max(vmax, cfl_speed_mx<true>(nw, sa.cfl, sa.dx, sa.dy, 0.0));
            }
        }
        __syncthreads();
    }
    warp_add_stat(&ctl->muscl_first_order, fo);
    warp_add_stat(&ctl->hlld_to_hlle, st.hlld_to_hlle);
    vmax = block_max(vmax, S.red);
    if (threadIdx.x == 0) atomic_max_speed(&ctl->vmax[sa.slot_out], vmax);
}

// The single-grid step: a strip per blockIdx.x, a segment per blockIdx.y.
template <int SOLVER, int TJ, int R, int NT>
__global__ void __launch_bounds__(NT, 2) k_mhd2d_fused_mixed(Geo G, Geo FG, const double* __restrict__ w,
                                                          double* __restrict__ wout, const double* __restrict__ B,
                                                          double* __restrict__ Bout, StepCtl* ctl, StepArgs sa,
                                                          int seg_rows) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto& S = *reinterpret_cast<FusedMhdSmem<TJ, R>*>(smem_raw);
    mhd2d_fused_body<SOLVER, TJ, R, NT>(G, FG, w, wout, B, Bout, ctl, sa, seg_rows, blockIdx.x, blockIdx.y,
                                        (long long)blockIdx.y * gridDim.x + blockIdx.x,
                                        (long long)gridDim.x * gridDim.y, S);
}

}  // namespace dgpu
