// Riemann solvers for the device path: HLL, HLLE, HLLC, HLLD, Roe (with the
// Harten-Hyman fix) and the exact solver, plus DRAGON's physicality
// verify-and-fallback pivot. Operand order follows
// DRAGON/Hydro/Riemann/{HLL,HLLD,Roe,Exact,Flux}.cpp.
#pragma once

#include "fluid.cuh"

#ifdef __CUDACC__
#include <cooperative_groups.h>
#endif

namespace dgpu {

// Solver ids match DRAGON/Config.h:39-50 (RIEMANN_*).
enum Solver : int { RS_EXACT = 0, RS_HLL = 1, RS_HLLC = 2, RS_HLLD = 3, RS_HLLE = 4, RS_HLLX = 5, RS_ROE = 6 };

// Counters a face solve can bump (fallback statistics).
struct FaceStats {
    int pivot_exact;   // verify failed, exact solver taken (Flux.cpp:88-93)
    int hlld_to_hlle;  // HLLD star state unphysical, HLLE taken (HLLD.cpp:77-79)
    int newton_iters;  // exact solver Newton iterations
    int exact_calls;   // exact solver star-pressure solves
    int trrs;          // two-rarefaction closed forms
    int cap_hits;      // Newton stopped by the iteration cap before the tolerance
    int guess_rejects; // Newton solves whose learned guess was unusable: analytic guess used
    int judge_reruns;  // learned guess hit the cap: solve rerun from the analytic guess
};

// Starting point of the star-pressure Newton iteration. GUESS_MEAN is the
// reference's (pL + pR) / 2 (Exact.cpp:47); GUESS_ANALYTIC is the adaptive
// PVRS / two-rarefaction / two-shock choice; GUESS_LEARNED takes the network's
// value, with the analytic guess as fallback when that value is unusable and
// as judge when the iteration from it hits the cap. GUESS_PERFECT is a
// measurement arm, not a solver option: the start is the converged star
// pressure of a first solve that is not counted, times (1 +- guess_err), or
// the reference's mean where that takes no more iterations, so its
// iteration count is the floor any guess of that accuracy with a fallback to
// the mean can reach.
enum GuessMode : int { GUESS_MEAN = 0, GUESS_ANALYTIC = 1, GUESS_LEARNED = 2, GUESS_PERFECT = 3 };

// Converged Newton solves recorded as training samples for the learned guess:
// kNewtonLogCols doubles per row (face-normal frame).
constexpr int kNewtonLogCols = 8;  // rhoL, vxL, pL, rhoR, vxR, pR, p*, iterations
struct NewtonLog {
    double* rows;                  // null: logging off
    unsigned long long* count;     // converged solves seen
    long long cap;                 // rows available
    int stride;                    // keep every stride-th solve (>= 1)
};

struct ExactOpts {
    int max_iters;     // ExactRiemann_MaxIters (Config.h:44); <= 0 means no cap
    double tol;        // ExactRiemann_Tolerance (Config.h:43)
    int guess;         // GuessMode
    NewtonLog log;
    double guess_err;  // GUESS_PERFECT: relative error given to the converged star pressure (0: none)
};

// HLL::roeAvg (HLL.cpp:21-37)
template <bool MHD, class R>
DHD Prim<R> roe_avg(const Prim<R>& L, const Prim<R>& Rt) {
    R sql = sqrt(L.rho), sqr = sqrt(Rt.rho);
    R _sql = sql / (sql + sqr), _sqr = sqr / (sql + sqr);
    Prim<R> w = zero_prim<R>();
    w.rho = sql * sqr;
    w.vx = L.vx * _sql + Rt.vx * _sqr;
    w.vy = L.vy * _sql + Rt.vy * _sqr;
    w.vz = L.vz * _sql + Rt.vz * _sqr;
    if constexpr (MHD) {
        w.Bx = L.Bx * _sql + Rt.Bx * _sqr;
        w.By = L.By * _sql + Rt.By * _sqr;
        w.Bz = L.Bz * _sql + Rt.Bz * _sqr;
    }
    R _H = _sql * enthalpy<MHD>(L) + _sqr * enthalpy<MHD>(Rt);
    R _a2 = R(kGm1) * (_H - dot3(w.vx, w.vy, w.vz, w.vx, w.vy, w.vz) / R(2));
    w.p = _a2 * w.rho / R(kGamma);
    return w;
}

// Riemann::HLL(SL,SR) (HLL.cpp:87-96)
template <bool MHD, class R>
DHD Cons<R> hll_speeds(const Prim<R>& L, const Prim<R>& Rt, R sl, R sr) {
    if (sl >= R(0)) return prim_flux<MHD>(L);
    if (sr <= R(0)) return prim_flux<MHD>(Rt);
    Cons<R> UL = to_cons<MHD>(L), UR = to_cons<MHD>(Rt);
    Cons<R> FL = cons_flux<MHD>(UL, L.vx, L.vy, L.vz);
    Cons<R> FR = cons_flux<MHD>(UR, Rt.vx, Rt.vy, Rt.vz);
    Cons<R> num = c_add<MHD>(c_sub<MHD>(c_mul<MHD>(FL, sr), c_mul<MHD>(FR, sl)),
                             c_mul<MHD>(c_sub<MHD>(UR, UL), sl * sr));
    return c_div<MHD>(num, sr - sl);
}

// Riemann::HLL (HLL.cpp:42-60). L and Rt are modified like the reference's
// member states (normal B averaged in MHD).
template <bool MHD, class R>
DHD Cons<R> hll(Prim<R>& L, Prim<R>& Rt) {
    Prim<R> M = roe_avg<MHD>(L, Rt);
    R aL, aR, aM;
    if constexpr (MHD) {
        R Bx = (L.Bx + Rt.Bx) / R(2);
        L.Bx = Bx; Rt.Bx = Bx;
        aL = fast_speed_x(L); aR = fast_speed_x(Rt); aM = fast_speed_x(M);
    } else {
        aL = sound_speed(L); aR = sound_speed(Rt); aM = sound_speed(M);
    }
    R SL = smin(L.vx - aL, M.vx - aM);
    R SR = smax(Rt.vx + aR, M.vx + aM);
    return hll_speeds<MHD>(L, Rt, SL, SR);
}

// Riemann::HLLE (HLL.cpp:61-84)
template <bool MHD, class R>
DHD Cons<R> hlle(Prim<R>& L, Prim<R>& Rt) {
    R sql = sqrt(L.rho), sqr = sqrt(Rt.rho);
    R _sql = sql / (sql + sqr), _sqr = sqr / (sql + sqr);
    R aL, aR;
    if constexpr (MHD) {
        R Bx = (L.Bx + Rt.Bx) / R(2);
        L.Bx = Bx; Rt.Bx = Bx;
        aL = fast_speed_x(L); aR = fast_speed_x(Rt);
    } else {
        aL = sound_speed(L); aR = sound_speed(Rt);
    }
    R _v = (Rt.vx - L.vx) / (sql + sqr);
    R d = (_sql * aL * aL + _sqr * aR * aR) + R(0.5) * (sql * sqr) * _v * _v;
    d = sqrt(d);
    R u = _sql * L.vx + _sqr * Rt.vx;
    R SL = smin(L.vx - aL, u - d);
    R SR = smax(Rt.vx + aR, u + d);
    return hll_speeds<MHD>(L, Rt, SL, SR);
}

// Riemann::HLLC(SL,SR) (HLL.cpp:115-132), hydro only.
template <class R>
DHD Cons<R> hllc_speeds(const Prim<R>& L, const Prim<R>& Rt, R sl, R sr) {
    if (sl >= R(0)) return prim_flux<false>(L);
    if (sr <= R(0)) return prim_flux<false>(Rt);
    R _pr = Rt.p + Rt.rho * Rt.vx * (Rt.vx - sr), _pl = L.p + L.rho * L.vx * (L.vx - sl);
    R sc = (_pr - _pl) / (Rt.rho * (Rt.vx - sr) - L.rho * (L.vx - sl));
    const Prim<R>& X = (sc > R(0)) ? L : Rt;
    R sx = sc > R(0) ? sl : sr;
    Cons<R> UX = to_cons<false>(X);
    Cons<R> U = c_div<false>(c_mul<false>(UX, sx - X.vx), sx - sc);
    U.mx = U.rho * sc;
    U.E += U.rho * (sc - X.vx) * (sc + X.p / (X.rho * (sx - X.vx)));
    return c_add<false>(cons_flux<false>(UX, X.vx, X.vy, X.vz), c_mul<false>(c_sub<false>(U, UX), sx));
}
// Riemann::HLLC (HLL.cpp:103-113)
template <class R>
DHD Cons<R> hllc(const Prim<R>& L, const Prim<R>& Rt) {
    Prim<R> M = roe_avg<false>(L, Rt);
    R aL = sound_speed(L), aR = sound_speed(Rt), aM = sound_speed(M);
    R SL = smin(L.vx - aL, M.vx - aM);
    R SR = smax(Rt.vx + aR, M.vx + aM);
    return hllc_speeds(L, Rt, SL, SR);
}

// Riemann::Roe with the Harten-Hyman entropy fix (Roe.cpp:19-96), hydro only.
template <class R>
DHD Cons<R> roe(const Prim<R>& L, const Prim<R>& Rt) {
    R sql = sqrt(L.rho), sqr = sqrt(Rt.rho);
    R _sql = sql / (sql + sqr), _sqr = sqr / (sql + sqr);
    R _rho = sql * sqr;
    R vx = L.vx * _sql + Rt.vx * _sqr;
    R vy = L.vy * _sql + Rt.vy * _sqr;
    R vz = L.vz * _sql + Rt.vz * _sqr;
    R _H = _sql * enthalpy<false>(L) + _sqr * enthalpy<false>(Rt);
    R V2 = dot3(vx, vy, vz, vx, vy, vz);
    R _a = sqrt(R(kGm1) * (_H - V2 / R(2)));
    R lambda[5] = {vx - _a, vx, vx, vx, vx + _a};
    // Eigenvectors K1..K5 (Roe.cpp:19-50) as conservative states.
    Cons<R> K[5];
    K[0] = Cons<R>{R(1), _H - vx * _a, vx - _a, vy - R(0), vz - R(0), 0, 0, 0};
    K[1] = Cons<R>{R(1), V2 / R(2), vx, vy, vz, 0, 0, 0};
    K[2] = Cons<R>{R(0), vy, R(0), R(1), R(0), 0, 0, 0};
    K[3] = Cons<R>{R(0), vz, R(0), R(0), R(1), 0, 0, 0};
    K[4] = Cons<R>{R(1), _H + vx * _a, vx + _a, vy + R(0), vz + R(0), 0, 0, 0};
    Cons<R> UL = to_cons<false>(L), UR = to_cons<false>(Rt);
    R alpha[5] = {((Rt.p - L.p) - _rho * _a * (Rt.vx - L.vx)) / (R(2) * _a * _a),
                  (Rt.rho - L.rho) - (Rt.p - L.p) / (_a * _a), _rho * (Rt.vy - L.vy), _rho * (Rt.vz - L.vz),
                  ((Rt.p - L.p) + _rho * _a * (Rt.vx - L.vx)) / (R(2) * _a * _a)};
    {
        Cons<R> SL = c_add<false>(UL, c_mul<false>(K[0], alpha[0]));
        R aL = sqrt(R(kGamma) * L.p / L.rho), aSL = sqrt(R(kGamma) * pressure<false>(SL) / SL.rho);
        R lambdaL = L.vx - aL, lambdaLS = SL.mx / SL.rho - aSL;
        if (lambdaL < R(0) && lambdaLS > R(0)) {
            R _lambda = lambdaL * (lambda[0] - lambdaLS) / (lambdaL - lambdaLS);
            return c_add<false>(cons_flux<false>(UL, L.vx, L.vy, L.vz), c_mul<false>(K[0], _lambda * alpha[0]));
        }
        Cons<R> SR = c_sub<false>(UR, c_mul<false>(K[4], alpha[4]));
        R aR = sqrt(R(kGamma) * Rt.p / Rt.rho), aSR = sqrt(R(kGamma) * pressure<false>(SR) / SR.rho);
        R lambdaR = Rt.vx + aR, lambdaRS = SR.mx / SR.rho + aSR;
        if (lambdaR > R(0) && lambdaRS < R(0)) {
            R _lambda = lambdaR * (lambda[4] - lambdaRS) / (lambdaR - lambdaRS);
            return c_sub<false>(cons_flux<false>(UR, Rt.vx, Rt.vy, Rt.vz), c_mul<false>(K[4], _lambda * alpha[4]));
        }
    }
    Cons<R> F = c_add<false>(cons_flux<false>(UL, L.vx, L.vy, L.vz), cons_flux<false>(UR, Rt.vx, Rt.vy, Rt.vz));
    for (int i = 0; i < 5; i++) F = c_sub<false>(F, c_mul<false>(K[i], alpha[i] * sabs(lambda[i])));
    return c_div<false>(F, R(2));
}

// ---------------------------------------------------------------------------
// Exact solver (Exact.cpp). Hydro only.

// Riemann::f (Exact.cpp:27-34)
template <class R> DHD R exact_f(R p, const Prim<R>& w) {
    if (p > w.p) {
        R A = R(k2_Gp1) / w.rho, B = R(kGm1_Gp1) * w.p;
        return (p - w.p) * sqrt(A / (B + p));
    }
    return R(k2_Gm1) * sound_speed(w) * (pow(p / w.p, R(kGm1_2G)) - R(1));
}
// df (Exact.cpp:35-42)
template <class R> DHD R exact_df(R p, const Prim<R>& w) {
    if (p > w.p) {
        R A = R(k2_Gp1) / w.rho, B = R(kGm1_Gp1) * w.p;
        return sqrt(A / (p + B)) * (R(1) - (p - w.p) / (R(2) * (B + p)));
    }
    return pow(p / w.p, -R(kGp1_2G)) / (w.rho * sound_speed(w));
}
// Riemann::exact_StarRho (Exact.cpp:87-90)
template <class R> DHD R exact_star_rho(const Prim<R>& w, R p) {
    if (p > w.p) return w.rho * (p + R(kGm1_Gp1) * w.p) / (R(kGm1_Gp1) * p + w.p);
    return w.rho * pow(p / w.p, R(kGinv));
}

// Star region of an exact solution; sL/sR as in RiemannSolution (Riemann.hpp:86-105).
template <class R>
struct ExactSolution {
    Prim<R> wL, wR, sL, sR;
};

#ifdef __CUDACC__
// Appends one converged solve to the sample log. The lanes of a warp that
// reach this together reserve their slots with one atomic.
__device__ __forceinline__ void newton_log_push(const NewtonLog& lg, double rl, double ul, double pl, double rr,
                                                double ur, double pr, double ps, int n) {
    namespace cg = cooperative_groups;
    cg::coalesced_group grp = cg::coalesced_threads();
    unsigned long long base = 0;
    if (grp.thread_rank() == 0) base = atomicAdd(lg.count, (unsigned long long)grp.size());
    base = grp.shfl(base, 0);
    const unsigned long long idx = base + grp.thread_rank();
    if (idx % (unsigned long long)lg.stride != 0) return;
    const unsigned long long row = idx / (unsigned long long)lg.stride;
    if (row >= (unsigned long long)lg.cap) return;
    double* r = lg.rows + row * kNewtonLogCols;
    r[0] = rl; r[1] = ul; r[2] = pl; r[3] = rr; r[4] = ur; r[5] = pr; r[6] = ps; r[7] = n;
}
#endif

constexpr int kPerfectGuessCap = 200;  // iterations of GUESS_PERFECT's uncounted first solve

// Riemann::exact_StarP (Exact.cpp:71-84): Newton from pGuess, step clamp
// 0.8 p, stop on relative change <= tol or after max_iters iterations.
// *converged tells whether the tolerance (not the cap) ended the iteration.
template <class R>
DHD R exact_star_p(const Prim<R>& L, const Prim<R>& Rt, R pGuess, ExactOpts o, FaceStats* st, bool* converged,
                   int* iterations = nullptr) {
    R pStar = pGuess, CHA = R(1);
    int iters = o.max_iters;
    int n = 0;
    do {
        R fp = exact_f(pStar, L) + exact_f(pStar, Rt) + Rt.vx - L.vx;
        R dfdp = exact_df(pStar, L) + exact_df(pStar, Rt);
        R delta = smin(fp / dfdp, R(0.8) * pStar);
        pStar -= delta;
        CHA = sabs(delta / (pStar + delta / R(2)));
        n++;
    } while (CHA > R(o.tol) && --iters != 0);
    const bool conv = !(CHA > R(o.tol));
    if (st) { st->newton_iters += n; st->exact_calls += 1; st->cap_hits += !conv; }
#ifdef __CUDA_ARCH__
    // only well-posed solves become samples: the reference also runs the
    // solver on unphysical corrected states of a step that is then retried
    if (conv && o.log.rows && pStar > R(0) && sfinite(pStar) && L.rho > R(0) && L.p > R(0) && Rt.rho > R(0) &&
        Rt.p > R(0) && sfinite(L.rho + L.p + L.vx + Rt.rho + Rt.p + Rt.vx))
        newton_log_push(o.log, L.rho, L.vx, L.p, Rt.rho, Rt.vx, Rt.p, pStar, n);
#endif
    *converged = conv;
    if (iterations) *iterations = n;
    return pStar;
}

// Adaptive analytic star-pressure guess (Toro, Riemann Solvers and Numerical
// Methods for Fluid Dynamics, 3rd ed., sec. 9.5.1, with Q = 2): the
// primitive-variable (PVRS) estimate when the pressure ratio is small and the
// estimate lies between the data pressures, the two-rarefaction estimate when
// it falls below both, the two-shock estimate linearised at PVRS otherwise.
// An unusable value (vacuum-generating data) gives the reference's mean.
template <class R>
DHD R analytic_guess(const Prim<R>& L, const Prim<R>& Rt) {
    const R aL = sound_speed(L), aR = sound_speed(Rt);
    const R du = Rt.vx - L.vx;
    const R mean = (L.p + Rt.p) / R(2);
    const R ppv = smax(R(0), mean - R(0.125) * du * (L.rho + Rt.rho) * (aL + aR));
    const R pmin = smin(L.p, Rt.p), pmax = smax(L.p, Rt.p);
    R g;
    if (pmax / pmin <= R(2) && pmin <= ppv && ppv <= pmax) {
        g = ppv;
    } else if (ppv < pmin) {
        const R z = R(kGm1_2G);
        g = pow((aL + aR - R(kGm1_2) * du) / (aL / pow(L.p, z) + aR / pow(Rt.p, z)), R(k2G_Gm1));
    } else {
        const R gL = sqrt(R(k2_Gp1) / L.rho / (ppv + R(kGm1_Gp1) * L.p));
        const R gR = sqrt(R(k2_Gp1) / Rt.rho / (ppv + R(kGm1_Gp1) * Rt.p));
        g = (gL * L.p + gR * Rt.p - du) / (gL + gR);
    }
    return (g > R(0) && sfinite(g)) ? g : mean;
}

// The network's guess for one face, evaluated by the caller (GUESS_LEARNED):
// guess, the analytic guess, and the two-rarefaction decision when the caller
// already made it (-1: not made).
template <class R>
struct LearnedGuess {
    R guess;
    R analytic;
    int trrs;
};

// The two-rarefaction early-out test of Riemann::exact (Exact.cpp:52-53).
template <class R>
DHD bool exact_is_trrs(const Prim<R>& L, const Prim<R>& Rt) {
    R p_min = smin(L.p, Rt.p);
    return exact_f(p_min, L) + exact_f(p_min, Rt) + Rt.vx - L.vx >= R(0);
}

// Riemann::exact(pGuess) including the two-rarefaction early-out (Exact.cpp:47-69)
// and Riemann::TRRS (Exact.cpp:96-113). The Newton start follows o.guess and
// is formed only when Newton runs: the reference's mean, the analytic guess,
// or the learned one (with the analytic guess as fallback when it is
// unusable and as judge, rerunning the solve, when it hits the cap).
template <class R>
DHD ExactSolution<R> exact_solve(const Prim<R>& L, const Prim<R>& Rt, ExactOpts o, FaceStats* st,
                                 const LearnedGuess<R>* learned = nullptr) {
    ExactSolution<R> s;
    s.wL = L;
    s.wR = Rt;
    s.sL = zero_prim<R>();
    s.sR = zero_prim<R>();
    s.sL.vx = L.vx; s.sL.vy = L.vy; s.sL.vz = L.vz;
    s.sR.vx = Rt.vx; s.sR.vy = Rt.vy; s.sR.vz = Rt.vz;
    const bool trrs = (learned && learned->trrs >= 0) ? learned->trrs != 0 : exact_is_trrs(L, Rt);
    if (trrs) {
        if (st) st->trrs += 1;
        R aL = sound_speed(L), aR = sound_speed(Rt);
        R _LR = pow(L.p / Rt.p, R(kGm1_2G)) * aR / aL;
        s.sL.vx = (_LR * L.vx + Rt.vx + R(k2_Gm1) * (_LR * aL - aR)) / (_LR + R(1));
        s.sR.vx = s.sL.vx;
        s.sL.p = L.p * pow(R(1) - R(kGm1_2) * (s.sL.vx - L.vx) / aL, R(k2G_Gm1));
        s.sR.p = s.sL.p;
        s.sL.rho = L.rho * pow(s.sL.p / L.p, R(kGinv));
        s.sR.rho = Rt.rho * pow(s.sR.p / Rt.p, R(kGinv));
        return s;
    }
    R pGuess, judge = R(0);
    if (o.guess == GUESS_MEAN) {
        pGuess = (L.p + Rt.p) / R(2);
    } else if (o.guess == GUESS_PERFECT) {
        // uncounted dry runs: the converged star pressure, the iterations from
        // it with the given relative error and from the mean guess; the counted
        // solve starts from whichever needs fewer (a gate that knows the answer)
        ExactOpts q = o;
        q.max_iters = kPerfectGuessCap;
        q.log.rows = nullptr;
        bool c0, c1, c2;
        int n_mean = 0, n_err = 0;
        const R mean = (L.p + Rt.p) / R(2);
        const R p0 = exact_star_p(L, Rt, mean, q, nullptr, &c0);
        const R e = R(o.guess_err);
        const R pe = (c0 && p0 > R(0) && sfinite(p0)) ? p0 * (R(1) + (L.p >= Rt.p ? e : -e)) : mean;
        ExactOpts d = o;
        d.log.rows = nullptr;
        exact_star_p(L, Rt, mean, d, nullptr, &c1, &n_mean);
        exact_star_p(L, Rt, pe, d, nullptr, &c2, &n_err);
        pGuess = (c2 && (!c1 || n_err < n_mean)) ? pe : mean;
    } else if (o.guess != GUESS_LEARNED || !learned) {
        pGuess = analytic_guess(L, Rt);
    } else if (learned->guess > R(0) && sfinite(learned->guess)) {
        pGuess = learned->guess;
        judge = learned->analytic;
    } else {
        pGuess = learned->analytic;
        if (st) st->guess_rejects++;
    }
    bool conv;
    R p = exact_star_p(L, Rt, pGuess, o, st, &conv);
    if (!conv && judge > R(0)) {
        if (st) st->judge_reruns++;
        p = exact_star_p(L, Rt, judge, o, st, &conv);
    }
    s.sL.p = p;
    s.sR.p = p;
    // Riemann::exact_StarV (Exact.cpp:85-86)
    s.sL.vx = (L.vx + Rt.vx + exact_f(p, Rt) - exact_f(p, L)) / R(2);
    s.sR.vx = s.sL.vx;
    s.sL.rho = exact_star_rho(L, p);
    s.sR.rho = exact_star_rho(Rt, p);
    return s;
}

// RiemannSolution::mirror (Exact.cpp:165-180)
template <class R> DHD void exact_mirror(ExactSolution<R>& s) {
    Prim<R> t = s.wL; s.wL = s.wR; s.wR = t;
    t = s.sL; s.sL = s.sR; s.sR = t;
    s.wL.vx *= R(-1); s.wR.vx *= R(-1); s.sL.vx *= R(-1); s.sR.vx *= R(-1);
}

// RiemannSolution::sample (Exact.cpp:122-163)
template <class R>
DHD Prim<R> exact_sample(ExactSolution<R> s, R x_t) {
    if (sabs(s.sR.vx - x_t) < R(1e-12)) {
        R sql = sqrt(s.sL.rho), sqr = sqrt(s.sR.rho);
        Cons<R> a = c_mul<false>(to_cons<false>(s.sL), sql);
        Cons<R> b = c_mul<false>(to_cons<false>(s.sR), sqr);
        return to_prim<false>(c_div<false>(c_add<false>(a, b), sql + sqr));
    }
    bool isLeft = x_t < s.sR.vx;
    if (isLeft) { exact_mirror(s); x_t = -x_t; }
    R a = sound_speed(s.wR);
    int zone;
    if (s.sR.p > s.wR.p) {
        R scale = sqrt(R(kGp1_2G) * s.sR.p / s.wR.p + R(kGm1_2G));
        zone = ((x_t - s.wR.vx) > scale * a) ? 1 : 3;
    } else {
        if ((x_t - s.wR.vx) > a) zone = 1;
        else if ((x_t - s.sR.vx) > a) zone = 2;
        else if ((x_t - s.sR.vx) > a * pow(s.sR.p / s.wR.p, R(kGm1_2G))) zone = 2;
        else zone = 3;
    }
    Prim<R> state;
    if (zone == 1) state = s.wR;
    else if (zone == 3) state = s.sR;
    else {
        state = s.wR;
        R scale = R(k2_Gp1) - R(kGm1_Gp1) * (s.wR.vx - x_t) / a;
        state.rho *= pow(scale, R(k2_Gm1));
        state.p *= pow(scale, R(k2G_Gm1));
        state.vx = R(k2_Gp1) * (x_t - a + s.wR.vx * R(kGm1_2));
    }
    if (isLeft) state.vx *= R(-1);
    return state;
}

// Riemann::exact().flux() (Exact.cpp:115-120) with the configured guess.
template <class R>
DHD Cons<R> exact_flux_default(const Prim<R>& L, const Prim<R>& Rt, ExactOpts o, FaceStats* st,
                               const LearnedGuess<R>* learned = nullptr) {
    ExactSolution<R> s = exact_solve(L, Rt, o, st, learned);
    Prim<R> w = exact_sample(s, R(0));
    return prim_flux<false>(w);
}

// ---------------------------------------------------------------------------
// HLLD (HLLD.cpp), MHD only, in DRAGON's Gaussian units.

// compute_outer_star (HLLD.cpp:21-37)
template <class R>
DHD void hlld_outer_star(Cons<R>& usK, const Prim<R>& K, R _xK, R SK, R SM, R pT, R Bx) {
    R Bx2_4pi = (Bx * Bx) * R(k1_4pi);
    R denom = _xK * (SK - SM) - Bx2_4pi;
    bool degen = sabs(denom) < R(1e-12);
    if (degen) { usK.Bx = K.Bx; usK.By = K.By; usK.Bz = K.Bz; }
    else {
        // K.B * (num) / denom: vector times scalar, then divided (HLLD.cpp:26)
        R num = _xK * (SK - K.vx) - Bx2_4pi;
        usK.Bx = (K.Bx * num) / denom; usK.By = (K.By * num) / denom; usK.Bz = (K.Bz * num) / denom;
    }
    usK.Bx = Bx;
    R vsx, vsy, vsz;
    if (degen) { vsx = K.vx - R(0); vsy = K.vy - R(0); vsz = K.vz - R(0); }
    else {
        // K.B * Bx * (SM - K.v.x) / denom * _1_4pi, left to right (HLLD.cpp:29)
        R d = SM - K.vx;
        vsx = K.vx - (((K.Bx * Bx) * d) / denom) * R(k1_4pi);
        vsy = K.vy - (((K.By * Bx) * d) / denom) * R(k1_4pi);
        vsz = K.vz - (((K.Bz * Bx) * d) / denom) * R(k1_4pi);
    }
    vsx = SM;
    usK.mx = vsx * usK.rho;
    usK.my = vsy * usK.rho;
    usK.mz = vsz * usK.rho;
    usK.E = energy<true>(K) * (SK - K.vx);
    usK.E += pT * SM - (K.p + dot3(K.Bx, K.By, K.Bz, K.Bx, K.By, K.Bz) * R(k1_8pi)) * K.vx;
    usK.E += Bx * (dot3(K.vx, K.vy, K.vz, K.Bx, K.By, K.Bz) - dot3(vsx, vsy, vsz, usK.Bx, usK.By, usK.Bz)) * R(k1_4pi);
    usK.E /= (SK - SM);
}

// compute_outer_star_zero_B (HLLD.cpp:137-150)
template <class R>
DHD void hlld_outer_star_zero_b(Cons<R>& usK, const Prim<R>& K, R SK, R SM, R pT) {
    if (sabs(SK - SM) < R(1e-12)) { usK.Bx = K.Bx; usK.By = K.By; usK.Bz = K.Bz; }
    else {
        R num = SK - K.vx, den = SK - SM;
        usK.Bx = (K.Bx * num) / den; usK.By = (K.By * num) / den; usK.Bz = (K.Bz * num) / den;
    }
    usK.Bx = 0;
    usK.mx = SM * usK.rho;
    usK.my = K.vy * usK.rho;
    usK.mz = K.vz * usK.rho;
    usK.E = energy<true>(K) * (SK - K.vx);
    usK.E += pT * SM - (K.p + dot3(K.Bx, K.By, K.Bz, K.Bx, K.By, K.Bz) * R(k1_8pi)) * K.vx;
    usK.E /= (SK - SM);
}

// Riemann::HLLD_zero_B (HLLD.cpp:152-205); falls back to HLLE like the reference.
template <class R>
DHD Cons<R> hlld_zero_b(Prim<R>& L, Prim<R>& Rt, R SL, R SR, FaceStats* st) {
    R pTL = L.p + dot3(L.Bx, L.By, L.Bz, L.Bx, L.By, L.Bz) * R(k1_8pi);
    R pTR = Rt.p + dot3(Rt.Bx, Rt.By, Rt.Bz, Rt.Bx, Rt.By, Rt.Bz) * R(k1_8pi);
    R _xL = L.rho * (SL - L.vx), _xR = Rt.rho * (SR - Rt.vx);
    R SM = ((_xR * Rt.vx - _xL * L.vx) - (pTR - pTL)) / (_xR - _xL);
    Cons<R> usL = zero_cons<R>(), usR = zero_cons<R>();
    usL.rho = _xL / (SL - SM);
    usR.rho = _xR / (SR - SM);
    Cons<R> FsL = zero_cons<R>(), FsR = zero_cons<R>();
    Prim<R> wsL = zero_prim<R>(), wsR = zero_prim<R>();
    R pT = (_xR * pTL - _xL * pTR + _xL * _xR * (Rt.vx - L.vx)) / (_xR - _xL);
    if (SM >= R(0)) {
        hlld_outer_star_zero_b(usL, L, SL, SM, pT);
        wsL.rho = usL.rho;
        wsL.vx = usL.mx / usL.rho; wsL.vy = usL.my / usL.rho; wsL.vz = usL.mz / usL.rho;
        wsL.Bx = usL.Bx; wsL.By = usL.By; wsL.Bz = usL.Bz;
        wsL.p = pT - dot3(wsL.Bx, wsL.By, wsL.Bz, wsL.Bx, wsL.By, wsL.Bz) * R(k1_8pi);
        if (!is_physical<true>(wsL) || !is_finite<true>(usL)) { if (st) st->hlld_to_hlle++; return hlle<true>(L, Rt); }
        FsL = c_add<true>(prim_flux<true>(L), c_mul<true>(c_sub<true>(usL, to_cons<true>(L)), SL));
        FsL.Bx = 0;
    }
    if (SM <= R(0)) {
        hlld_outer_star_zero_b(usR, Rt, SR, SM, pT);
        wsR.rho = usR.rho;
        wsR.vx = usR.mx / usR.rho; wsR.vy = usR.my / usR.rho; wsR.vz = usR.mz / usR.rho;
        wsR.Bx = usR.Bx; wsR.By = usR.By; wsR.Bz = usR.Bz;
        wsR.p = pT - dot3(wsR.Bx, wsR.By, wsR.Bz, wsR.Bx, wsR.By, wsR.Bz) * R(k1_8pi);
        if (!is_physical<true>(wsR) || !is_finite<true>(usR)) { if (st) st->hlld_to_hlle++; return hlle<true>(L, Rt); }
        FsR = c_add<true>(prim_flux<true>(Rt), c_mul<true>(c_sub<true>(usR, to_cons<true>(Rt)), SR));
        FsR.Bx = 0;
    }
    if (SM > R(0)) return FsL;
    if (SM < R(0)) return FsR;
    R sql = sqrt(wsL.rho), sqr = sqrt(wsR.rho);
    R _sql = sql / (sql + sqr), _sqr = sqr / (sql + sqr);
    return c_add<true>(c_mul<true>(FsL, _sql), c_mul<true>(FsR, _sqr));
}

// Riemann::HLLD (HLLD.cpp:38-133)
template <class R>
DHD Cons<R> hlld(Prim<R>& L, Prim<R>& Rt, FaceStats* st) {
    R Bx = (L.Bx + Rt.Bx) / R(2);
    L.Bx = Bx; Rt.Bx = Bx;
    R cl = fast_speed_x(L), cr = fast_speed_x(Rt);
    R SL = smin(L.vx - cl, Rt.vx - cr);
    if (SL >= R(0)) return prim_flux<true>(L);
    R SR = smax(L.vx + cl, Rt.vx + cr);
    if (SR <= R(0)) return prim_flux<true>(Rt);

    // floor 1e-100 as in HLLD.cpp:50; FP32 has no such number, so it floors at
    // 1e-30 and takes a zero normal field to the zero-field branch explicitly
    // (in FP64 Bx == 0 already satisfies the test).
    const R floor_b2 = sizeof(R) == sizeof(double) ? R(1e-100) : R(1e-30);
    R cutoff = smax(dot3(L.Bx, L.By, L.Bz, L.Bx, L.By, L.Bz) + dot3(Rt.Bx, Rt.By, Rt.Bz, Rt.Bx, Rt.By, Rt.Bz), floor_b2);
    if (Bx * Bx < R(1e-12) * cutoff || Bx == R(0)) return hlld_zero_b(L, Rt, SL, SR, st);

    R pTL = L.p + dot3(L.Bx, L.By, L.Bz, L.Bx, L.By, L.Bz) * R(k1_8pi);
    R pTR = Rt.p + dot3(Rt.Bx, Rt.By, Rt.Bz, Rt.Bx, Rt.By, Rt.Bz) * R(k1_8pi);
    R _xL = L.rho * (SL - L.vx), _xR = Rt.rho * (SR - Rt.vx);
    R SM = ((_xR * Rt.vx - _xL * L.vx) - (pTR - pTL)) / (_xR - _xL);

    Cons<R> usL = zero_cons<R>(), usR = zero_cons<R>();
    usL.rho = _xL / (SL - SM);
    R SsL = SM - sabs(Bx) / (R(sq4pi()) * sqrt(usL.rho));
    usR.rho = _xR / (SR - SM);
    R SsR = SM + sabs(Bx) / (R(sq4pi()) * sqrt(usR.rho));

    Cons<R> FsL = zero_cons<R>(), FsR = zero_cons<R>();
    Prim<R> wsL = zero_prim<R>(), wsR = zero_prim<R>();
    R pT = (_xR * pTL - _xL * pTR + _xL * _xR * (Rt.vx - L.vx)) / (_xR - _xL);

    if (SsR >= R(0)) {
        hlld_outer_star(usL, L, _xL, SL, SM, pT, Bx);
        wsL.rho = usL.rho;
        wsL.vx = usL.mx / usL.rho; wsL.vy = usL.my / usL.rho; wsL.vz = usL.mz / usL.rho;
        wsL.Bx = usL.Bx; wsL.By = usL.By; wsL.Bz = usL.Bz;
        wsL.p = pT - dot3(wsL.Bx, wsL.By, wsL.Bz, wsL.Bx, wsL.By, wsL.Bz) * R(k1_8pi);
        if (!is_physical<true>(wsL) || !is_physical<true>(usL)) { if (st) st->hlld_to_hlle++; return hlle<true>(L, Rt); }
        FsL = c_add<true>(prim_flux<true>(L), c_mul<true>(c_sub<true>(usL, to_cons<true>(L)), SL));
        FsL.Bx = 0;
    }
    if (SsL <= R(0)) {
        hlld_outer_star(usR, Rt, _xR, SR, SM, pT, Bx);
        wsR.rho = usR.rho;
        wsR.vx = usR.mx / usR.rho; wsR.vy = usR.my / usR.rho; wsR.vz = usR.mz / usR.rho;
        wsR.Bx = usR.Bx; wsR.By = usR.By; wsR.Bz = usR.Bz;
        wsR.p = pT - dot3(wsR.Bx, wsR.By, wsR.Bz, wsR.Bx, wsR.By, wsR.Bz) * R(k1_8pi);
        if (!is_physical<true>(wsR) || !is_physical<true>(usR)) { if (st) st->hlld_to_hlle++; return hlle<true>(L, Rt); }
        FsR = c_add<true>(prim_flux<true>(Rt), c_mul<true>(c_sub<true>(usR, to_cons<true>(Rt)), SR));
        FsR.Bx = 0;
    }
    if (SsL >= R(0)) return FsL;
    if (SsR <= R(0)) return FsR;

    const Prim<R>& ws = SM >= R(0) ? wsL : wsR;
    R sqL = sqrt(wsL.rho), sqR = sqrt(wsR.rho);
    R _sqL = sqL / (sqL + sqR), _sqR = sqR / (sqL + sqR);
    R sbx = Bx > R(0) ? R(sq4pi()) : (Bx < R(0) ? -R(sq4pi()) : R(0));
    Cons<R> uss = zero_cons<R>();
    Prim<R> wss = zero_prim<R>();
    wss.rho = ws.rho;
    uss.rho = wss.rho;
    // wss.v = _sqL*wsL.v + _sqR*wsR.v + (sbx*(usR.B - usL.B)*_1_4pi)/(sqL+sqR)
    wss.vx = (wsL.vx * _sqL + wsR.vx * _sqR) + ((usR.Bx - usL.Bx) * sbx * R(k1_4pi)) / (sqL + sqR);
    wss.vy = (wsL.vy * _sqL + wsR.vy * _sqR) + ((usR.By - usL.By) * sbx * R(k1_4pi)) / (sqL + sqR);
    wss.vz = (wsL.vz * _sqL + wsR.vz * _sqR) + ((usR.Bz - usL.Bz) * sbx * R(k1_4pi)) / (sqL + sqR);
    wss.vx = SM;
    uss.mx = wss.vx * uss.rho;
    uss.my = wss.vy * uss.rho;
    uss.mz = wss.vz * uss.rho;
    // wss.B = _sqL*usR.B + _sqR*usL.B + sbx*(wsR.v - wsL.v)*sqL*sqR/(sqL+sqR)
    wss.Bx = (usR.Bx * _sqL + usL.Bx * _sqR) + ((wsR.vx - wsL.vx) * sbx * sqL * sqR) / (sqL + sqR);
    wss.By = (usR.By * _sqL + usL.By * _sqR) + ((wsR.vy - wsL.vy) * sbx * sqL * sqR) / (sqL + sqR);
    wss.Bz = (usR.Bz * _sqL + usL.Bz * _sqR) + ((wsR.vz - wsL.vz) * sbx * sqL * sqR) / (sqL + sqR);
    wss.Bx = Bx;
    uss.Bx = wss.Bx; uss.By = wss.By; uss.Bz = wss.Bz;
    R dE = sbx * (dot3(ws.vx, ws.vy, ws.vz, ws.Bx, ws.By, ws.Bz) - dot3(wss.vx, wss.vy, wss.vz, wss.Bx, wss.By, wss.Bz)) *
           R(k1_4pi) * sqrt(wss.rho);
    uss.E = SM >= R(0) ? usL.E - dE : usR.E + dE;
    wss.p = pT - dot3(wss.Bx, wss.By, wss.Bz, wss.Bx, wss.By, wss.Bz) * R(k1_8pi);
    if (!is_physical<true>(wss) || !is_finite<true>(uss)) { if (st) st->hlld_to_hlle++; return hlle<true>(L, Rt); }
    if (SM >= R(0)) return c_add<true>(FsL, c_mul<true>(c_sub<true>(uss, usL), SsL));
    return c_add<true>(FsR, c_mul<true>(c_sub<true>(uss, usR), SsR));
}

// ---------------------------------------------------------------------------
// Dispatch with the verify-and-fallback pivot (Flux.cpp:17-97) for a face
// along x. dt_dx > 0 enables the hydro physicality check. Returns false when
// the reference would throw (no physical flux found).
template <bool MHD, int SOLVER, class R>
DHD bool face_flux_x(Prim<R> L, Prim<R> Rt, R dt_dx, ExactOpts eo, Cons<R>& F, FaceStats* st,
                     const LearnedGuess<R>* learned = nullptr) {
    if constexpr (MHD) {
        if constexpr (SOLVER == RS_HLL) F = hll<true>(L, Rt);
        else if constexpr (SOLVER == RS_HLLE) F = hlle<true>(L, Rt);
        else F = hlld(L, Rt, st);
        return true;
    } else {
        if constexpr (SOLVER == RS_HLL) F = hll<false>(L, Rt);
        else if constexpr (SOLVER == RS_HLLE) F = hlle<false>(L, Rt);
        else if constexpr (SOLVER == RS_ROE) F = roe(L, Rt);
        else if constexpr (SOLVER == RS_EXACT) F = exact_flux_default(L, Rt, eo, st, learned);
        else F = hllc(L, Rt);
        if (!(dt_dx > R(0))) return true;
        // verify_and_fallback (Flux.cpp:77-97); Riemann_ExactFallback_Parameter = 1
        Cons<R> UL = to_cons<false>(L), UR = to_cons<false>(Rt);
        if (is_physical<false>(c_sub<false>(UL, c_mul<false>(F, dt_dx))) &&
            is_physical<false>(c_add<false>(UR, c_mul<false>(F, dt_dx))))
            return true;
        if (st) st->pivot_exact++;
        F = exact_flux_default(L, Rt, eo, st);
        if (is_physical<false>(c_sub<false>(UL, c_mul<false>(F, dt_dx))) &&
            is_physical<false>(c_add<false>(UR, c_mul<false>(F, dt_dx))))
            return true;
        return false;
    }
}

// Riemann::flux_X/Y/Z (Flux.cpp:101-115): swap the normal axis into x, solve,
// swap the flux back. AX: 0 = x, 1 = y, 2 = z.
template <bool MHD, int SOLVER, int AX, class R>
DHD bool face_flux(Prim<R> L, Prim<R> Rt, R dt_dL, ExactOpts eo, Cons<R>& F, FaceStats* st,
                   const LearnedGuess<R>* learned = nullptr) {
    swap_axis<AX>(L);
    swap_axis<AX>(Rt);
    bool ok = face_flux_x<MHD, SOLVER>(L, Rt, dt_dL, eo, F, st, learned);
    swap_axis<AX>(F);
    return ok;
}

}  // namespace dgpu
