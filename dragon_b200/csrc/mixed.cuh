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

// FP64 energy of an FP32 primitive state (PrimitiveState::energy in FP64).
template <bool MHD>
__device__ __forceinline__ double energy64(const Prim<float>& w) {
    return energy<MHD>(cvt<double>(w));
}

// Primitive state from FP32 momenta / density and an FP64 total energy,
// pressure recovered in FP64.
template <bool MHD>
__device__ __forceinline__ Prim<float> prim_from(const Cons<float>& u, double E64) {
    Prim<float> w;
    w.rho = u.rho;
    w.vx = u.mx / u.rho;
    w.vy = u.my / u.rho;
    w.vz = u.mz / u.rho;
    const double rho = u.rho, mx = u.mx, my = u.my, mz = u.mz;
    double Eth = E64 - (mx * mx + my * my + mz * mz) / (2.0 * rho);
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

}  // namespace dgpu
