// Mixed-precision building blocks: FP32 reconstruction and flux arithmetic,
// FP64 where stability needs it.
//
// A half state is an FP32 primitive state. Whenever a state is rebuilt from
// conservative variables (the MUSCL-Hancock predictor, the CTU transverse
// correction), its total energy is accumulated in FP64 from the FP64 energy of
// the state it started from, and the pressure is recovered in FP64:
//   p = (gamma - 1) (E - |m|^2 / 2 rho)
// so the subtraction of kinetic from total energy does not lose the FP32
// mantissa in high-Mach cells. Everything else (slopes, limiters, fluxes,
// wave speeds, the Riemann solves) runs in FP32.
#pragma once

#include "recon.cuh"
#include "riemann.cuh"

namespace dgpu {

// The FP64 arithmetic of the mixed path is not held to bit parity, so it
// divides by neither gamma - 1 nor a density: it multiplies by the constant
// 1 / (gamma - 1) and by the density's correctly rounded reciprocal
// (__drcp_rn), which costs fewer FP64 instructions than an IEEE division.
constexpr double kInvGm1 = 1.0 / kGm1;

// FP64 energy of a primitive state (PrimitiveState::energy in FP64).
template <bool MHD, class R>
__device__ __forceinline__ double energy64_of(const Prim<R>& w) {
    const double rho = w.rho, vx = w.vx, vy = w.vy, vz = w.vz;
    double E = (double)w.p * kInvGm1 + (0.5 * rho) * (vx * vx + vy * vy + vz * vz);
    if constexpr (MHD) {
        const double bx = w.Bx, by = w.By, bz = w.Bz;
        E += (bx * bx + by * by + bz * bz) * k1_8pi;
    }
    return E;
}
template <bool MHD>
__device__ __forceinline__ double energy64(const Prim<float>& w) {
    return energy64_of<MHD>(w);
}

// ConservativeState <-> PrimitiveState in FP64 for the mixed path's committed
// state (same formulas as to_cons / to_prim, divisions replaced as above).
template <bool MHD>
__device__ __forceinline__ Cons<double> to_cons64(const Prim<double>& w) {
    Cons<double> u;
    u.rho = w.rho;
    u.mx = w.vx * w.rho;
    u.my = w.vy * w.rho;
    u.mz = w.vz * w.rho;
    u.E = energy64_of<MHD>(w);
    if constexpr (MHD) { u.Bx = w.Bx; u.By = w.By; u.Bz = w.Bz; }
    else { u.Bx = u.By = u.Bz = 0; }
    return u;
}
template <bool MHD>
__device__ __forceinline__ Prim<double> to_prim64(const Cons<double>& u) {
    const double inv = __drcp_rn(u.rho);
    Prim<double> w;
    w.rho = u.rho;
    w.vx = u.mx * inv;
    w.vy = u.my * inv;
    w.vz = u.mz * inv;
    double Eth = u.E - (u.mx * u.mx + u.my * u.my + u.mz * u.mz) * (0.5 * inv);
    if constexpr (MHD) {
        Eth -= (u.Bx * u.Bx + u.By * u.By + u.Bz * u.Bz) * k1_8pi;
        w.Bx = u.Bx; w.By = u.By; w.Bz = u.Bz;
    } else {
        w.Bx = w.By = w.Bz = 0;
    }
    w.p = kGm1 * Eth;
    return w;
}

// CFL signal speed of a committed cell (CFL.cpp:28-84: max or sum over the
// axes of (|v| + a) / dL) evaluated in FP32 for the forms CFL_MAX and CFL_ADD:
// the mixed path's time step is its own, and the FP32 speed is within ~1e-7
// of the FP64 one; the p-norm form keeps the FP64 function.
template <bool MHD>
__device__ __forceinline__ double cfl_speed_mx(const Prim<double>& W64, int cfl, double dx, double dy, double dz) {
    if (cfl != 0 && cfl != 1) return cfl_speed<MHD>(W64, cfl, dx, dy, dz);
    const Prim<float> W = cvt<float>(W64);
    float a;
    if constexpr (MHD) a = fast_speed_max(W);
    else a = sound_speed(W);
    float speed = 0.f;
    if (dx > 1e-14) speed = (fabsf(W.vx) + a) / (float)dx;
    if (dy > 1e-14) speed = cfl ? speed + (fabsf(W.vy) + a) / (float)dy : smax(speed, (fabsf(W.vy) + a) / (float)dy);
    if (dz > 1e-14) speed = cfl ? speed + (fabsf(W.vz) + a) / (float)dz : smax(speed, (fabsf(W.vz) + a) / (float)dz);
    return speed;
}
// The 1D grids' speed |v.x| + a (CFL.cpp:88-105) in FP32.
template <bool MHD>
__device__ __forceinline__ double cfl_speed_1d_mx(const Prim<double>& W64) {
    const Prim<float> W = cvt<float>(W64);
    float a;
    if constexpr (MHD) a = fast_speed_max(W);
    else a = sound_speed(W);
    return fabsf(W.vx) + a;
}

// Primitive state from FP32 momenta / density and an FP64 total energy,
// pressure recovered in FP64. The velocities are the momenta times the FP64
// reciprocal of the density that the pressure recovery computes anyway,
// rounded once to FP32: the mixed translation units are built with
// approximate FP32 division, whose rounding errors do not cancel over many
// steps. On the 1024^2 shear layer they carried the transverse velocity's
// relative L1 after 2000 steps to 3.4e-4; these velocities and the rounded
// reciprocals of the HLLC star state below bring it to 7.5e-5 (IEEE FP32
// division throughout: 7.2e-5) and 9.9e-6 after 25 steps, at 1.7 % of the
// step's time over approximate division.
template <bool MHD>
__device__ __forceinline__ Prim<float> prim_from(const Cons<float>& u, double E64) {
    Prim<float> w;
    w.rho = u.rho;
    const double rho = u.rho, mx = u.mx, my = u.my, mz = u.mz;
    const double inv = __drcp_rn(rho);
    w.vx = (float)(mx * inv);
    w.vy = (float)(my * inv);
    w.vz = (float)(mz * inv);
    double Eth = E64 - (mx * mx + my * my + mz * mz) * (0.5 * inv);
    if constexpr (MHD) {
        const double bx = u.Bx, by = u.By, bz = u.Bz;
        Eth -= (bx * bx + by * by + bz * bz) * k1_8pi;
        w.Bx = u.Bx; w.By = u.By; w.Bz = u.Bz;
    } else {
        w.Bx = w.By = w.Bz = 0.f;
    }
    w.p = (float)(kGm1 * Eth);
    return w;
}

// MUSCL-Hancock in FP32 (TVD::MUSCL, MUSCL.cpp:16-61) with the predictor's
// energy kept in FP64. Returns true when second order was kept.
template <bool MHD>
__device__ __forceinline__ bool muscl_mixed(int lim, const Prim<float>& wL, Prim<float>& outL, const Prim<float>& wC,
                                            Prim<float>& outR, const Prim<float>& wR, float dt_dL, float dBx, float dBy,
                                            float dBz) {
    Prim<float> dW, L, R;
    dW.rho = limit1(lim, wC.rho - wL.rho, wR.rho - wC.rho);
    dW.vx = limit1(lim, wC.vx - wL.vx, wR.vx - wC.vx);
    dW.vy = limit1(lim, wC.vy - wL.vy, wR.vy - wC.vy);
    dW.vz = limit1(lim, wC.vz - wL.vz, wR.vz - wC.vz);
    dW.p = limit1(lim, wC.p - wL.p, wR.p - wC.p);
    L.rho = wC.rho - 0.5f * dW.rho;  R.rho = wC.rho + 0.5f * dW.rho;
    L.vx = wC.vx - 0.5f * dW.vx;     R.vx = wC.vx + 0.5f * dW.vx;
    L.vy = wC.vy - 0.5f * dW.vy;     R.vy = wC.vy + 0.5f * dW.vy;
    L.vz = wC.vz - 0.5f * dW.vz;     R.vz = wC.vz + 0.5f * dW.vz;
    L.p = wC.p - 0.5f * dW.p;        R.p = wC.p + 0.5f * dW.p;
    if constexpr (MHD) {
        dW.Bx = limit1(lim, wC.Bx - wL.Bx, wR.Bx - wC.Bx);
        dW.By = limit1(lim, wC.By - wL.By, wR.By - wC.By);
        dW.Bz = limit1(lim, wC.Bz - wL.Bz, wR.Bz - wC.Bz);
        L.Bx = wC.Bx - 0.5f * dW.Bx;  R.Bx = wC.Bx + 0.5f * dW.Bx;
        L.By = wC.By - 0.5f * dW.By;  R.By = wC.By + 0.5f * dW.By;
        L.Bz = wC.Bz - 0.5f * dW.Bz;  R.Bz = wC.Bz + 0.5f * dW.Bz;
    } else {
        L.Bx = L.By = L.Bz = R.Bx = R.By = R.Bz = 0.f;
    }
    const Cons<float> UL = to_cons<MHD>(L), UR = to_cons<MHD>(R);
    Cons<float> corr = c_mul<MHD>(c_sub<MHD>(cons_flux<MHD>(UR, R.vx, R.vy, R.vz), cons_flux<MHD>(UL, L.vx, L.vy, L.vz)),
                                  0.5f * dt_dL);
    if constexpr (MHD) {
        const float a_s = (R.Bx - L.Bx) * dt_dL;
        const float vy = 0.5f * (L.vy + R.vy), vz = 0.5f * (L.vz + R.vz);
        const float dBy_ = 0.5f * wC.vy * lim_minmod(dBx, -dBy) - 0.5f * vy * a_s;
        const float dBz_ = 0.5f * wC.vz * lim_minmod(dBx, -dBz) - 0.5f * vz * a_s;
        corr.By -= dBy_;
        corr.Bz -= dBz_;
        corr.E -= float(k1_4pi) * (wC.By * dBy_ + wC.Bz * dBz_);
    }
    outL = prim_from<MHD>(c_sub<MHD>(UL, corr), energy64<MHD>(L) - (double)corr.E);
    outR = prim_from<MHD>(c_sub<MHD>(UR, corr), energy64<MHD>(R) - (double)corr.E);
    if (is_physical<MHD>(outL) && is_physical<MHD>(outR)) return true;
    outL = wC;
    outR = wC;
    return false;
}

// s = prim(cons(s) - tr) with the energy accumulated in FP64 (correctState).
template <bool MHD>
__device__ __forceinline__ Prim<float> correct_mixed(const Prim<float>& s, const Cons<float>& tr) {
    return prim_from<MHD>(c_sub<MHD>(to_cons<MHD>(s), tr), energy64<MHD>(s) - (double)tr.E);
}

// Riemann dispatch in FP32. The hydro physicality pivot runs in FP32; when it
// fires, the exact solver runs in FP64 on the same states (the rare path).
template <bool MHD, int SOLVER, int AX>
__device__ __forceinline__ bool face_flux_mixed(Prim<float> L, Prim<float> R, float dt_dL, ExactOpts eo, Cons<float>& F,
                                                FaceStats* st) {
    swap_axis<AX>(L);
    swap_axis<AX>(R);
    bool ok = true;
    if constexpr (MHD) {
        if constexpr (SOLVER == RS_HLL) F = hll<true>(L, R);
        else if constexpr (SOLVER == RS_HLLE) F = hlle<true>(L, R);
        else F = hlld(L, R, st);
    } else {
        if constexpr (SOLVER == RS_HLL) F = hll<false>(L, R);
        else if constexpr (SOLVER == RS_HLLE) F = hlle<false>(L, R);
        else if constexpr (SOLVER == RS_ROE) F = roe(L, R);
        else if constexpr (SOLVER == RS_EXACT) F = cvt<float>(exact_flux_default(cvt<double>(L), cvt<double>(R), eo, st));
        else F = hllc(L, R);
        if (dt_dL > 0.f) {
            const Cons<float> UL = to_cons<false>(L), UR = to_cons<false>(R);
            if (!(is_physical<false>(c_sub<false>(UL, c_mul<false>(F, dt_dL))) &&
                  is_physical<false>(c_add<false>(UR, c_mul<false>(F, dt_dL))))) {
                if (st) st->pivot_exact++;
                const Prim<double> Ld = cvt<double>(L), Rd = cvt<double>(R);
                const Cons<double> Fd = exact_flux_default(Ld, Rd, eo, st);
                const double h = dt_dL;
                const Cons<double> ULd = to_cons<false>(Ld), URd = to_cons<false>(Rd);
                ok = is_physical<false>(c_sub<false>(ULd, c_mul<false>(Fd, h))) &&
                     is_physical<false>(c_add<false>(URd, c_mul<false>(Fd, h)));
                F = cvt<float>(Fd);
            }
        }
    }
    swap_axis<AX>(F);
    return ok;
}

// ---------------------------------------------------------------------------
// Pressure offset (hydro). The FP32 rounding of an absolute pressure p enters
// the normal-momentum flux rho u^2 + p at |p| * 2^-24, which is large next to
// a small transverse velocity's momentum. A tile therefore carries every FP32
// pressure as an offset dp = p - ref from a tile-wide FP64 reference (the
// smallest pressure the tile loads, so |dp| <= |p|), and the normal-momentum
// fluxes it computes are rho u^2 + dp: the reference is the same for both faces
// of every cell the tile updates and cancels exactly in the FP64 flux
// differences. Wave speeds, energies and the physicality checks use the
// absolute pressure ref + dp.

// Absolute FP32 view of an offset state.
__device__ __forceinline__ Prim<float> abs_p(Prim<float> w, float ref_f) {
    w.p = ref_f + w.p;
    return w;
}

// FP64 energy of an offset state.
__device__ __forceinline__ double energy64_off(const Prim<float>& w, double ref) {
    Prim<double> d = cvt<double>(w);
    d.p = ref + d.p;
    return energy64_of<false>(d);
}

// Offset primitive state from FP32 momenta / density and an FP64 total energy;
// *phys: the state is finite with positive density and FP64 pressure.
__device__ __forceinline__ Prim<float> prim_from_off(const Cons<float>& u, double E64, double ref, bool* phys) {
    Prim<float> w;
    w.rho = u.rho;
    const double rho = u.rho, mx = u.mx, my = u.my, mz = u.mz;
    const double inv = __drcp_rn(rho);
    w.vx = (float)(mx * inv);
    w.vy = (float)(my * inv);
    w.vz = (float)(mz * inv);
    const double p = kGm1 * (E64 - (mx * mx + my * my + mz * mz) * (0.5 * inv));
    w.p = (float)(p - ref);
    w.Bx = w.By = w.Bz = 0.f;
    if (phys)
        *phys = sfinite(w.rho) && sfinite(w.vx) && sfinite(w.vy) && sfinite(w.vz) && sfinite(p) && w.rho > 0.f &&
                p > 0.0;
    return w;
}

// muscl_mixed<false> on offset states: slopes and faces of dp, the predictor's
// normal-momentum flux difference on dp, energies in FP64 on ref + dp.
__device__ __forceinline__ bool muscl_off(int lim, const Prim<float>& wL, Prim<float>& outL, const Prim<float>& wC,
                                          Prim<float>& outR, const Prim<float>& wR, float dt_dL, double ref,
                                          float ref_f) {
    Prim<float> dW, L, R;
    dW.rho = limit1(lim, wC.rho - wL.rho, wR.rho - wC.rho);
    dW.vx = limit1(lim, wC.vx - wL.vx, wR.vx - wC.vx);
    dW.vy = limit1(lim, wC.vy - wL.vy, wR.vy - wC.vy);
    dW.vz = limit1(lim, wC.vz - wL.vz, wR.vz - wC.vz);
    dW.p = limit1(lim, wC.p - wL.p, wR.p - wC.p);
    L.rho = wC.rho - 0.5f * dW.rho;  R.rho = wC.rho + 0.5f * dW.rho;
    L.vx = wC.vx - 0.5f * dW.vx;     R.vx = wC.vx + 0.5f * dW.vx;
    L.vy = wC.vy - 0.5f * dW.vy;     R.vy = wC.vy + 0.5f * dW.vy;
    L.vz = wC.vz - 0.5f * dW.vz;     R.vz = wC.vz + 0.5f * dW.vz;
    L.p = wC.p - 0.5f * dW.p;        R.p = wC.p + 0.5f * dW.p;
    L.Bx = L.By = L.Bz = R.Bx = R.By = R.Bz = 0.f;
    const Prim<float> La = abs_p(L, ref_f), Ra = abs_p(R, ref_f);
    const Cons<float> UL = to_cons<false>(La), UR = to_cons<false>(Ra);
    const float h = 0.5f * dt_dL;
    Cons<float> corr = c_mul<false>(c_sub<false>(cons_flux<false>(UR, Ra.vx, Ra.vy, Ra.vz),
                                                 cons_flux<false>(UL, La.vx, La.vy, La.vz)), h);
    corr.mx = ((UR.mx * Ra.vx + R.p) - (UL.mx * La.vx + L.p)) * h;
    bool okL, okR;
    outL = prim_from_off(c_sub<false>(UL, corr), energy64_off(L, ref) - (double)corr.E, ref, &okL);
    outR = prim_from_off(c_sub<false>(UR, corr), energy64_off(R, ref) - (double)corr.E, ref, &okR);
    if (okL && okR) return true;
    outL = wC;
    outR = wC;
    return false;
}

// correct_mixed<false> on an offset state.
__device__ __forceinline__ Prim<float> correct_off(const Prim<float>& s, const Cons<float>& tr, double ref, float ref_f) {
    return prim_from_off(c_sub<false>(to_cons<false>(abs_p(s, ref_f)), tr), energy64_off(s, ref) - (double)tr.E, ref,
                         nullptr);
}

// Riemann::HLLC (HLL.cpp:103-132) in FP32 on offset states: wave speeds and the
// star energy from the absolute pressures, the normal-momentum flux on dp
// (F.mx is the flux minus ref). The contact speed and the star state divide
// by way of correctly rounded reciprocals (see prim_from).
__device__ __forceinline__ Cons<float> hllc_off(const Prim<float>& L, const Prim<float>& Rt, float ref_f) {
    const Prim<float> La = abs_p(L, ref_f), Ra = abs_p(Rt, ref_f);
    const Prim<float> M = roe_avg<false>(La, Ra);
    const float aL = sound_speed(La), aR = sound_speed(Ra), aM = sound_speed(M);
    const float sl = smin(La.vx - aL, M.vx - aM);
    const float sr = smax(Ra.vx + aR, M.vx + aM);
    if (sl >= 0.f) {
        Cons<float> F = prim_flux<false>(La);
        F.mx = (La.rho * La.vx) * La.vx + L.p;
        return F;
    }
    if (sr <= 0.f) {
        Cons<float> F = prim_flux<false>(Ra);
        F.mx = (Ra.rho * Ra.vx) * Ra.vx + Rt.p;
        return F;
    }
    const float _pr = Rt.p + Ra.rho * Ra.vx * (Ra.vx - sr), _pl = L.p + La.rho * La.vx * (La.vx - sl);
    const float sc = (_pr - _pl) * __frcp_rn(Ra.rho * (Ra.vx - sr) - La.rho * (La.vx - sl));
    const bool left = sc > 0.f;
    const Prim<float>& X = left ? La : Ra;
    const float dpx = left ? L.p : Rt.p;
    const float sx = left ? sl : sr;
    const Cons<float> UX = to_cons<false>(X);
    Cons<float> U = c_mul<false>(c_mul<false>(UX, sx - X.vx), __frcp_rn(sx - sc));
    U.mx = U.rho * sc;
    U.E += U.rho * (sc - X.vx) * (sc + X.p * __frcp_rn(X.rho * (sx - X.vx)));
    Cons<float> F = c_add<false>(cons_flux<false>(UX, X.vx, X.vy, X.vz), c_mul<false>(c_sub<false>(U, UX), sx));
    F.mx = (UX.mx * X.vx + dpx) + (U.mx - UX.mx) * sx;
    return F;
}

// face_flux_mixed<false, SOLVER, AX> on offset states. With HLLC the normal
// momentum flux comes back minus ref (ref_f / ref: the tile's reference); the
// other solvers run on the absolute FP32 states, which the caller pairs with a
// zero reference.
template <int SOLVER, int AX>
__device__ __forceinline__ bool face_flux_off(Prim<float> L, Prim<float> R, float dt_dL, ExactOpts eo, Cons<float>& F,
                                              FaceStats* st, double ref, float ref_f) {
    if constexpr (SOLVER != RS_HLLC) {
        return face_flux_mixed<false, SOLVER, AX>(abs_p(L, ref_f), abs_p(R, ref_f), dt_dL, eo, F, st);
    } else {
        swap_axis<AX>(L);
        swap_axis<AX>(R);
        bool ok = true;
        F = hllc_off(L, R, ref_f);
        if (dt_dL > 0.f) {
            const Prim<float> La = abs_p(L, ref_f), Ra = abs_p(R, ref_f);
            Cons<float> Ft = F;
            Ft.mx += ref_f;
            const Cons<float> UL = to_cons<false>(La), UR = to_cons<false>(Ra);
            if (!(is_physical<false>(c_sub<false>(UL, c_mul<false>(Ft, dt_dL))) &&
                  is_physical<false>(c_add<false>(UR, c_mul<false>(Ft, dt_dL))))) {
                if (st) st->pivot_exact++;
                Prim<double> Ld = cvt<double>(L), Rd = cvt<double>(R);
                Ld.p = ref + Ld.p;
                Rd.p = ref + Rd.p;
                const Cons<double> Fd = exact_flux_default(Ld, Rd, eo, st);
                const double h = dt_dL;
                const Cons<double> ULd = to_cons<false>(Ld), URd = to_cons<false>(Rd);
                ok = is_physical<false>(c_sub<false>(ULd, c_mul<false>(Fd, h))) &&
                     is_physical<false>(c_add<false>(URd, c_mul<false>(Fd, h)));
                F = cvt<float>(Fd);
                F.mx = (float)(Fd.mx - ref);
            }
        }
        swap_axis<AX>(F);
        return ok;
    }
}

}  // namespace dgpu
