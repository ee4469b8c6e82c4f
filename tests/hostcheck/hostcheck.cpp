// CPU build of the device path's per-cell and per-face functions
// (dragon_b200/csrc/*.cuh) for the CPU test suite. The CUDA kernels run these
// same functions on the GPU; compiling them with g++ and -ffp-contract=off lets
// the CPU tests check operand order against the reference bit for bit before
// any GPU run. Not part of the product: nothing outside tests/ loads it.
#include "../../dragon_b200/csrc/fluid.cuh"
#include "../../dragon_b200/csrc/frame.cuh"
#include "../../dragon_b200/csrc/recon.cuh"
#include "../../dragon_b200/csrc/riemann.cuh"

using namespace dgpu;

#ifdef HC_MHD
constexpr bool M = true;
constexpr int NF = 8;
#else
constexpr bool M = false;
constexpr int NF = 5;
#endif

static Prim<double> P(const double* a) {
    Prim<double> w = zero_prim<double>();
    w.rho = a[0]; w.p = a[1]; w.vx = a[2]; w.vy = a[3]; w.vz = a[4];
    if (M) { w.Bx = a[5]; w.By = a[6]; w.Bz = a[7]; }
    return w;
}
static void Pout(const Prim<double>& w, double* a) {
    a[0] = w.rho; a[1] = w.p; a[2] = w.vx; a[3] = w.vy; a[4] = w.vz;
    if (M) { a[5] = w.Bx; a[6] = w.By; a[7] = w.Bz; }
}
static Cons<double> C(const double* a) {
    Cons<double> u = zero_cons<double>();
    u.rho = a[0]; u.E = a[1]; u.mx = a[2]; u.my = a[3]; u.mz = a[4];
    if (M) { u.Bx = a[5]; u.By = a[6]; u.Bz = a[7]; }
    return u;
}
static void Cout(const Cons<double>& u, double* a) {
    a[0] = u.rho; a[1] = u.E; a[2] = u.mx; a[3] = u.my; a[4] = u.mz;
    if (M) { a[5] = u.Bx; a[6] = u.By; a[7] = u.Bz; }
}

template <int S, int AX>
static int flux_t(const double* l, const double* r, double dt, double* out) {
    Cons<double> F;
    ExactOpts eo{6, 1e-12};
    bool ok = face_flux<M, S, AX, double>(P(l), P(r), dt, eo, F, nullptr);
    Cout(F, out);
    return ok ? 0 : 1;
}
template <int S>
static int flux_ax(int ax, const double* l, const double* r, double dt, double* out) {
    if (ax == 0) return flux_t<S, 0>(l, r, dt, out);
    if (ax == 1) return flux_t<S, 1>(l, r, dt, out);
    return flux_t<S, 2>(l, r, dt, out);
}

extern "C" {
#ifndef HC_MHD
double hc_analytic_guess(const double* l, const double* r) { return analytic_guess(P(l), P(r)); }
// Exact flux along x with a star-pressure guess policy (learned: null or
// {learned guess, analytic guess}); stats receives
// newton_iters, exact_calls, trrs, cap_hits, guess_rejects, judge_reruns.
void hc_exact_flux_guess(const double* l, const double* r, int mode, int max_iters, const double* learned,
                         double* out, int* stats) {
    FaceStats st{};
    ExactOpts eo{max_iters, 1e-12, mode, NewtonLog{}};
    const LearnedGuess<double> lg{learned ? learned[0] : 0.0, learned ? learned[1] : 0.0, -1};
    Cout(exact_flux_default(P(l), P(r), eo, &st, learned ? &lg : nullptr), out);
    const int v[6] = {st.newton_iters, st.exact_calls, st.trrs, st.cap_hits, st.guess_rejects, st.judge_reruns};
    for (int i = 0; i < 6; i++) stats[i] = v[i];
}
#endif
int hc_nfields(void) { return NF; }
// Ghost-frame enumeration of the 2D MHD step (frame.cuh): point k of the frame
// of box b (bi0, bi1, bj0, bj1) inside range r (lo_i, hi_i, lo_j, hi_j).
int hc_frame_point(long long k, const int* r, const int* b, int* ij) {
    return frame_point(k, r[0], r[1], r[2], r[3], b[0], b[1], b[2], b[3], ij[0], ij[1]) ? 1 : 0;
}
long long hc_frame_count(const int* r, const int* b) { return frame_count(r[0], r[1], r[2], r[3], b[0], b[1], b[2], b[3]); }
long long hc_mhd2d_frame_points(long long nx, long long ny, long long g) { return mhd2d_frame_points(nx, ny, g); }
void hc_prim_to_cons(const double* w, double* u) { Cout(to_cons<M>(P(w)), u); }
void hc_cons_to_prim(const double* u, double* w) { Pout(to_prim<M>(C(u)), w); }
void hc_prim_flux(const double* w, double* f) { Cout(prim_flux<M>(P(w)), f); }
double hc_limiter(int kind, double a, double b) { return limit1(kind, a, b); }
void hc_muscl(int lim, const double* wl, const double* wc, const double* wr, double dt_dL, const double* dB,
              double* L, double* R) {
    Prim<double> oL, oR;
    muscl<M>(lim, P(wl), oL, P(wc), oR, P(wr), dt_dL, dB[0], dB[1], dB[2]);
    Pout(oL, L);
    Pout(oR, R);
}
// solver uses the dispatch ids of the runtime switch (Flux.cpp:17-74).
int hc_riemann_flux(int solver, const double* l, const double* r, double dt, int ax, double* out) {
#ifdef HC_MHD
    switch (solver) {
        case RS_HLL: return flux_ax<RS_HLL>(ax, l, r, dt, out);
        case RS_HLLE: return flux_ax<RS_HLLE>(ax, l, r, dt, out);
        default: return flux_ax<RS_HLLD>(ax, l, r, dt, out);
    }
#else
    switch (solver) {
        case RS_HLLX:
        case RS_HLLC: return flux_ax<RS_HLLC>(ax, l, r, dt, out);
        case RS_HLL: return flux_ax<RS_HLL>(ax, l, r, dt, out);
        case RS_HLLE: return flux_ax<RS_HLLE>(ax, l, r, dt, out);
        case RS_ROE: return flux_ax<RS_ROE>(ax, l, r, dt, out);
        default: return flux_ax<RS_EXACT>(ax, l, r, dt, out);
    }
#endif
}
double hc_fast_speed_max(const double* w) { return fast_speed_max(P(w)); }
}
