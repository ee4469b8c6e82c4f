// Per-cell state arithmetic for the device path: primitive/conservative
// states, the ideal-gas EOS, x-fluxes, wave speeds and physicality tests.
//
// Every expression keeps the operand order of DRAGON's FluidElement
// (DRAGON/FluidElement/FluidElement.cpp, Arithmetic.cpp) so that, compiled
// without FMA contraction, the FP64 results are bit-identical to the
// reference's. The header is plain C++ so the same functions can be compiled
// for the host by the CPU test suite.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define DHD __host__ __device__ __forceinline__
#else
#define DHD inline
#endif

namespace dgpu {

// ---------------------------------------------------------------------------
// Constants: the same constant expressions as DRAGON/Constants.h:18-39, so
// each derived value carries identical rounding.
constexpr double kGamma = 5.0 / 3.0;
constexpr double kGm1 = kGamma - 1.0;
constexpr double k1_4pi = 0.25 / M_PI;
constexpr double k1_8pi = 0.125 / M_PI;
constexpr double k8pi = 8 * M_PI;
constexpr double kGm1_2G = (kGamma - 1.0) / (2.0 * kGamma);
constexpr double kGp1_2G = (kGamma + 1.0) / (2.0 * kGamma);
constexpr double k2G_Gm1 = 2.0 * kGamma / (kGamma - 1.0);
constexpr double kGm1_2 = (kGamma - 1.0) / 2.0;
constexpr double k2_Gm1 = 2.0 / (kGamma - 1.0);
constexpr double k2_Gp1 = 2.0 / (kGamma + 1.0);
constexpr double kGm1_Gp1 = (kGamma - 1.0) / (kGamma + 1.0);
constexpr double kGinv = 1.0 / kGamma;

// sqrt(4*pi); sqrt is correctly rounded on both host and device.
DHD double sq4pi() { return sqrt(4.0 * M_PI); }

// std::min / std::max semantics (first argument wins ties, NaN in the second
// argument is ignored by max and taken by min), as the reference uses them.
template <class R> DHD R smin(R a, R b) { return (b < a) ? b : a; }
template <class R> DHD R smax(R a, R b) { return (a < b) ? b : a; }
template <class R> DHD R sabs(R a) { return fabs(a); }
template <class R> DHD bool sfinite(R a) { return isfinite(a); }

// ---------------------------------------------------------------------------
// States. B is present in the struct for both physics modes; hydro code never
// touches it (every use sits under `if constexpr (MHD)`), so it costs no
// registers there.
template <class R>
struct Prim {
    R rho, p, vx, vy, vz, Bx, By, Bz;
};
template <class R>
struct Cons {
    R rho, E, mx, my, mz, Bx, By, Bz;
};

template <class R> DHD Prim<R> zero_prim() { return Prim<R>{0, 0, 0, 0, 0, 0, 0, 0}; }
template <class R> DHD Cons<R> zero_cons() { return Cons<R>{0, 0, 0, 0, 0, 0, 0, 0}; }

template <class R> DHD R dot3(R ax, R ay, R az, R bx, R by, R bz) { return ax * bx + ay * by + az * bz; }

// PrimitiveState::energy (FluidElement.cpp:53-59)
template <bool MHD, class R>
DHD R energy(const Prim<R>& w) {
    R E = w.p / R(kGm1) + (w.rho / R(2)) * dot3(w.vx, w.vy, w.vz, w.vx, w.vy, w.vz);
    if constexpr (MHD) E += dot3(w.Bx, w.By, w.Bz, w.Bx, w.By, w.Bz) * R(k1_8pi);
    return E;
}
// ConservativeState::pressure (FluidElement.cpp:60-66)
template <bool MHD, class R>
DHD R pressure(const Cons<R>& u) {
    R Eth = u.E - dot3(u.mx, u.my, u.mz, u.mx, u.my, u.mz) / (R(2) * u.rho);
    if constexpr (MHD) Eth -= dot3(u.Bx, u.By, u.Bz, u.Bx, u.By, u.Bz) * R(k1_8pi);
    return R(kGm1) * Eth;
}
// ConservativeState(PrimitiveState) (FluidElement.cpp:35-42)
template <bool MHD, class R>
DHD Cons<R> to_cons(const Prim<R>& w) {
    Cons<R> u;
    u.rho = w.rho;
    u.mx = w.vx * w.rho;
    u.my = w.vy * w.rho;
    u.mz = w.vz * w.rho;
    u.E = energy<MHD>(w);
    if constexpr (MHD) { u.Bx = w.Bx; u.By = w.By; u.Bz = w.Bz; }
    else { u.Bx = 0; u.By = 0; u.Bz = 0; }
    return u;
}
// PrimitiveState(ConservativeState) (FluidElement.cpp:44-51)
template <bool MHD, class R>
DHD Prim<R> to_prim(const Cons<R>& u) {
    Prim<R> w;
    w.rho = u.rho;
    w.vx = u.mx / u.rho;
    w.vy = u.my / u.rho;
    w.vz = u.mz / u.rho;
    w.p = pressure<MHD>(u);
    if constexpr (MHD) { w.Bx = u.Bx; w.By = u.By; w.Bz = u.Bz; }
    else { w.Bx = 0; w.By = 0; w.Bz = 0; }
    return w;
}
// PrimitiveState::enthalpy (FluidElement.cpp:69-75)
template <bool MHD, class R>
DHD R enthalpy(const Prim<R>& w) {
    R h = energy<MHD>(w) + w.p;
    if constexpr (MHD) h += dot3(w.Bx, w.By, w.Bz, w.Bx, w.By, w.Bz) * R(k1_8pi);
    return h / w.rho;
}

// Physicality (FluidElement.cpp:82-96)
template <bool MHD, class R>
DHD bool is_physical(const Prim<R>& w) {
    if constexpr (MHD) {
        if (!(sfinite(w.Bx) && sfinite(w.By) && sfinite(w.Bz))) return false;
    }
    return sfinite(w.rho) && sfinite(w.vx) && sfinite(w.vy) && sfinite(w.vz) && sfinite(w.p) &&
           w.rho > R(0) && w.p > R(0);
}
template <bool MHD, class R>
DHD bool is_finite(const Cons<R>& u) {
    if constexpr (MHD) {
        if (!(sfinite(u.Bx) && sfinite(u.By) && sfinite(u.Bz))) return false;
    }
    return sfinite(u.rho) && sfinite(u.mx) && sfinite(u.my) && sfinite(u.mz) && sfinite(u.E);
}
template <bool MHD, class R>
DHD bool is_physical(const Cons<R>& u) {
    return is_finite<MHD>(u) && u.rho > R(0) && pressure<MHD>(u) > R(0);
}

// Wave speeds (FluidElement.cpp:99-120). pow(x,2) in the reference is folded
// to x*x by the compiler, so x*x is used here.
template <class R> DHD R sound_speed(const Prim<R>& w) { return sqrt(R(kGamma) * w.p / w.rho); }
template <class R>
DHD R alfven_speed(const Prim<R>& w) {
    return sqrt(dot3(w.Bx, w.By, w.Bz, w.Bx, w.By, w.Bz) / w.rho) / R(sq4pi());
}
template <class R>
DHD R fast_speed(const Prim<R>& w, R Bk) {
    R c = sound_speed(w), a = alfven_speed(w);
    R c2 = c * c, a2 = a * a, ak2 = (Bk * Bk / w.rho) * R(k1_4pi);
    R s = c2 + a2;
    R disc = smax(R(0), (s * s) * R(0.25) - ak2 * c2);
    return sqrt((c2 + a2) * R(0.5) + sqrt(disc));
}
template <class R> DHD R fast_speed_x(const Prim<R>& w) { return fast_speed(w, w.Bx); }
template <class R>
DHD R fast_speed_max(const Prim<R>& w) {
    R Bk;
    if (w.Bx * w.Bx < w.By * w.By) Bk = (w.Bx * w.Bx < w.Bz * w.Bz) ? w.Bx : w.Bz;
    else Bk = (w.By * w.By < w.Bz * w.Bz) ? w.By : w.Bz;
    return fast_speed(w, Bk);
}

// ConservativeState::flux(vec3 v) (FluidElement.cpp:133-155)
template <bool MHD, class R>
DHD Cons<R> cons_flux(const Cons<R>& u, R vx, R vy, R vz) {
    Cons<R> F;
    R p = pressure<MHD>(u);
    F.rho = u.mx;
    F.mx = u.mx * vx;
    F.my = u.my * vx;
    F.mz = u.mz * vx;
    F.mx += p;
    F.E = (u.E + p) * vx;
    if constexpr (MHD) {
        R pmag = dot3(u.Bx, u.By, u.Bz, u.Bx, u.By, u.Bz) * R(k1_8pi);
        F.mx += pmag;
        F.E += pmag * vx;
        R tx = (u.Bx * u.Bx) * R(k1_4pi);
        R ty = (u.By * u.Bx) * R(k1_4pi);
        R tz = (u.Bz * u.Bx) * R(k1_4pi);
        F.mx -= tx;
        F.my -= ty;
        F.mz -= tz;
        F.E -= dot3(vx, vy, vz, tx, ty, tz);
        F.By = u.By * vx - vy * u.Bx;
        F.Bz = u.Bz * vx - vz * u.Bx;
        F.Bx = 0;
    } else {
        F.Bx = 0; F.By = 0; F.Bz = 0;
    }
    return F;
}
// PrimitiveState::flux (FluidElement.cpp:132)
template <bool MHD, class R>
DHD Cons<R> prim_flux(const Prim<R>& w) {
    return cons_flux<MHD>(to_cons<MHD>(w), w.vx, w.vy, w.vz);
}
// ConservativeState::flux() (FluidElement.cpp:133-140)
template <bool MHD, class R>
DHD Cons<R> cons_flux_self(const Cons<R>& u) {
    if constexpr (MHD) return cons_flux<MHD>(u, u.mx / u.rho, u.my / u.rho, u.mz / u.rho);
    else return cons_flux<MHD>(u, u.mx / u.rho, R(0), R(0));
}

// Componentwise conservative arithmetic (Arithmetic.cpp:14-128).
template <bool MHD, class R>
DHD Cons<R> c_add(const Cons<R>& a, const Cons<R>& b) {
    Cons<R> r{a.rho + b.rho, a.E + b.E, a.mx + b.mx, a.my + b.my, a.mz + b.mz, 0, 0, 0};
    if constexpr (MHD) { r.Bx = a.Bx + b.Bx; r.By = a.By + b.By; r.Bz = a.Bz + b.Bz; }
    return r;
}
template <bool MHD, class R>
DHD Cons<R> c_sub(const Cons<R>& a, const Cons<R>& b) {
    Cons<R> r{a.rho - b.rho, a.E - b.E, a.mx - b.mx, a.my - b.my, a.mz - b.mz, 0, 0, 0};
    if constexpr (MHD) { r.Bx = a.Bx - b.Bx; r.By = a.By - b.By; r.Bz = a.Bz - b.Bz; }
    return r;
}
template <bool MHD, class R>
DHD Cons<R> c_mul(const Cons<R>& a, R s) {
    Cons<R> r{a.rho * s, a.E * s, a.mx * s, a.my * s, a.mz * s, 0, 0, 0};
    if constexpr (MHD) { r.Bx = a.Bx * s; r.By = a.By * s; r.Bz = a.Bz * s; }
    return r;
}
template <bool MHD, class R>
DHD Cons<R> c_div(const Cons<R>& a, R s) {
    Cons<R> r{a.rho / s, a.E / s, a.mx / s, a.my / s, a.mz / s, 0, 0, 0};
    if constexpr (MHD) { r.Bx = a.Bx / s; r.By = a.By / s; r.Bz = a.Bz / s; }
    return r;
}

// Axis swaps (FluidElement.cpp:170-240): the solvers always work along x.
template <class R> DHD void swap_xy(Prim<R>& w) {
    R t = w.vx; w.vx = w.vy; w.vy = t;
    t = w.Bx; w.Bx = w.By; w.By = t;
}
template <class R> DHD void swap_xz(Prim<R>& w) {
    R t = w.vx; w.vx = w.vz; w.vz = t;
    t = w.Bx; w.Bx = w.Bz; w.Bz = t;
}
template <class R> DHD void swap_xy(Cons<R>& u) {
    R t = u.mx; u.mx = u.my; u.my = t;
    t = u.Bx; u.Bx = u.By; u.By = t;
}
template <class R> DHD void swap_xz(Cons<R>& u) {
    R t = u.mx; u.mx = u.mz; u.mz = t;
    t = u.Bx; u.Bx = u.Bz; u.Bz = t;
}
// Swap selected by axis: 0 = none, 1 = XY, 2 = XZ.
template <int AX, class S> DHD void swap_axis(S& s) {
    if constexpr (AX == 1) swap_xy(s);
    else if constexpr (AX == 2) swap_xz(s);
}

// Precision conversion between storage (FP64) and compute types.
template <class R, class S> DHD Prim<R> cvt(const Prim<S>& a) {
    return Prim<R>{R(a.rho), R(a.p), R(a.vx), R(a.vy), R(a.vz), R(a.Bx), R(a.By), R(a.Bz)};
}
template <class R, class S> DHD Cons<R> cvt(const Cons<S>& a) {
    return Cons<R>{R(a.rho), R(a.E), R(a.mx), R(a.my), R(a.mz), R(a.Bx), R(a.By), R(a.Bz)};
}

}  // namespace dgpu
