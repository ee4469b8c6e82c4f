// TVD limiters and MUSCL-Hancock reconstruction for the device path.
// Operand order follows DRAGON/Hydro/Reconstruction/Limiters.cpp and
// MUSCL.cpp so FP64 results match the reference bit for bit.
#pragma once

#include "fluid.cuh"

namespace dgpu {

enum Limiter : int { LIM_MINMOD = 0, LIM_MC = 1, LIM_VANLEER = 2, LIM_SUPERBEE = 3, LIM_VANALBADA = 4 };

// Limiters.cpp:44-47
template <class R> DHD R lim_minmod(R a, R b) {
    if (a * b <= R(0)) return R(0);
    return (sabs(a) < sabs(b)) ? a : b;
}
// Limiters.cpp:68-73
template <class R> DHD R lim_mc(R a, R b) {
    if (a * b <= R(0)) return R(0);
    R c = sabs(a + b);
    if (c < R(4) * sabs(a) && c < R(4) * sabs(b)) return a < R(0) ? -c / R(2) : c / R(2);
    return R(2) * lim_minmod(a, b);
}
// Limiters.cpp:94-97
template <class R> DHD R lim_vanleer(R a, R b) {
    if (a * b <= R(0)) return R(0);
    return R(2) * a * b / (a + b);
}
// Limiters.cpp:118-124
template <class R> DHD R lim_superbee(R a, R b) {
    if (a * b <= R(0)) return R(0);
    R aa = sabs(a), bb = sabs(b);
    R s1 = smin(R(2) * aa, bb), s2 = smin(aa, R(2) * bb);
    R mag = smax(s1, s2);
    return a < R(0) ? -mag : mag;
}
// Limiters.cpp:144-147
template <class R> DHD R lim_vanalbada(R a, R b) {
    if (a * b <= R(0)) return R(0);
    return a * b * (a + b) / (a * a + b * b);
}
// TVD::limit dispatch (Limiters.cpp:17-39); unknown values fall back to minmod.
template <class R> DHD R limit1(int lim, R a, R b) {
    switch (lim) {
        case LIM_MC: return lim_mc(a, b);
        case LIM_VANLEER: return lim_vanleer(a, b);
        case LIM_SUPERBEE: return lim_superbee(a, b);
        case LIM_VANALBADA: return lim_vanalbada(a, b);
        default: return lim_minmod(a, b);
    }
}

// TVD::MUSCL (MUSCL.cpp:16-61): limited primitive slopes, half-width spatial
// states, then the half-dt predictor in conservative variables; falls back to
// first order when either predicted state is unphysical. dB carries the
// face-B divergence terms of the MHD source (zero for hydro).
// Returns true when the second-order states were kept.
template <bool MHD, class R>
DHD bool muscl(int lim, const Prim<R>& wL, Prim<R>& outL, const Prim<R>& wC, Prim<R>& outR,
               const Prim<R>& wR, R dt_dL, R dBx, R dBy, R dBz) {
    Prim<R> dW, L, Rr;
    dW.rho = limit1(lim, wC.rho - wL.rho, wR.rho - wC.rho);
    dW.vx = limit1(lim, wC.vx - wL.vx, wR.vx - wC.vx);
    dW.vy = limit1(lim, wC.vy - wL.vy, wR.vy - wC.vy);
    dW.vz = limit1(lim, wC.vz - wL.vz, wR.vz - wC.vz);
    dW.p = limit1(lim, wC.p - wL.p, wR.p - wC.p);
    L.rho = wC.rho - R(0.5) * dW.rho;
    Rr.rho = wC.rho + R(0.5) * dW.rho;
    L.vx = wC.vx - dW.vx * R(0.5);
    L.vy = wC.vy - dW.vy * R(0.5);
    L.vz = wC.vz - dW.vz * R(0.5);
    Rr.vx = wC.vx + dW.vx * R(0.5);
    Rr.vy = wC.vy + dW.vy * R(0.5);
    Rr.vz = wC.vz + dW.vz * R(0.5);
    L.p = wC.p - R(0.5) * dW.p;
    Rr.p = wC.p + R(0.5) * dW.p;
    if constexpr (MHD) {
        dW.Bx = limit1(lim, wC.Bx - wL.Bx, wR.Bx - wC.Bx);
        dW.By = limit1(lim, wC.By - wL.By, wR.By - wC.By);
        dW.Bz = limit1(lim, wC.Bz - wL.Bz, wR.Bz - wC.Bz);
        L.Bx = wC.Bx - dW.Bx * R(0.5);
        L.By = wC.By - dW.By * R(0.5);
        L.Bz = wC.Bz - dW.Bz * R(0.5);
        Rr.Bx = wC.Bx + dW.Bx * R(0.5);
        Rr.By = wC.By + dW.By * R(0.5);
        Rr.Bz = wC.Bz + dW.Bz * R(0.5);
    } else {
        L.Bx = L.By = L.Bz = Rr.Bx = Rr.By = Rr.Bz = R(0);
    }

    Cons<R> UL = to_cons<MHD>(L), UR = to_cons<MHD>(Rr);
    Cons<R> corr = c_mul<MHD>(c_sub<MHD>(cons_flux<MHD>(UR, Rr.vx, Rr.vy, Rr.vz),
                                         cons_flux<MHD>(UL, L.vx, L.vy, L.vz)),
                              R(0.5) * dt_dL);
    if constexpr (MHD) {
        const R a_s = (Rr.Bx - L.Bx) * dt_dL;
        const R vy = R(0.5) * (L.vy + Rr.vy), vz = R(0.5) * (L.vz + Rr.vz);
        const R dBy_ = R(0.5) * wC.vy * lim_minmod(dBx, -dBy) - R(0.5) * vy * a_s;
        const R dBz_ = R(0.5) * wC.vz * lim_minmod(dBx, -dBz) - R(0.5) * vz * a_s;
        corr.By -= dBy_;
        corr.Bz -= dBz_;
        corr.E -= R(k1_4pi) * (wC.By * dBy_ + wC.Bz * dBz_);
    }
    outL = to_prim<MHD>(c_sub<MHD>(UL, corr));
    outR = to_prim<MHD>(c_sub<MHD>(UR, corr));
    if (is_physical<MHD>(outL) && is_physical<MHD>(outR)) return true;
    outL = wC;
    outR = wC;
    return false;
}

}  // namespace dgpu
