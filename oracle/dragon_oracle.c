/*
 * dragon_oracle.c — CPU restatement of DRAGON's unsplit Godunov update.
 *
 * TEST INFRASTRUCTURE ONLY (see dragon_oracle.h): the parity oracle, pinned
 * bit for bit against the reference library (oracle/_ref) by the CPU tests.
 * Each function names the reference function it restates (file:line within
 * the DRAGON tree). Compiled with -ffp-contract=off; expressions keep the
 * reference's operand order so results are identical, not merely close.
 */
#include "dragon_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef ORACLE_MHD
#define MHD 1
#define NF 8
#else
#define MHD 0
#define NF 5
#endif

/* ------------------------------------------------------------------------- */
/* Constants (DRAGON/Constants.h:18-39) and switches (DRAGON/Config.h)         */

#define GAMMA (5.0 / 3.0)
static const double kGm1 = GAMMA - 1.0;
static const double k1_4pi = 0.25 / M_PI;
static const double k1_8pi = 0.125 / M_PI;
static const double kGm1_2G = (GAMMA - 1.0) / (2.0 * GAMMA);
static const double kGp1_2G = (GAMMA + 1.0) / (2.0 * GAMMA);
static const double k2G_Gm1 = 2.0 * GAMMA / (GAMMA - 1.0);
static const double kGm1_2 = (GAMMA - 1.0) / 2.0;
static const double k2_Gm1 = 2.0 / (GAMMA - 1.0);
static const double k2_Gp1 = 2.0 / (GAMMA + 1.0);
static const double kGm1_Gp1 = (GAMMA - 1.0) / (GAMMA + 1.0);
static const double kGinv = 1.0 / GAMMA;
static double sq4pi(void) { return sqrt(4.0 * M_PI); }

enum { R_EXACT = 0, R_HLL = 1, R_HLLC = 2, R_HLLD = 3, R_HLLE = 4, R_HLLX = 5, R_ROE = 6 };
enum { L_MINMOD = 0, L_MC = 1, L_VANLEER = 2, L_SUPERBEE = 3, L_VANALBADA = 4 };

static struct {
    int riemann, limiter, cfl, ct_energy, exact_max_iters;
    double exact_tol, cfl_coeff, tol;
} O = {R_HLLX, L_MC, 1, 2, 6, 1e-12, 0.3, 1e-14};

void ora_set_options(int riemann, int limiter, int cfl, int ct_energy, int exact_max_iters, double exact_tol,
                     double cfl_coeff, double timestep_tol) {
    O.riemann = riemann;
    O.limiter = limiter;
    O.cfl = cfl;
    O.ct_energy = ct_energy;
    O.exact_max_iters = exact_max_iters;
    O.exact_tol = exact_tol;
    O.cfl_coeff = cfl_coeff;
    O.tol = timestep_tol;
}
int ora_nfields(void) { return NF; }

/* The reference signals failures with exceptions; here a flag set by the
 * failing function and checked by the step before it commits. */
static int g_fail;

/* std::min / std::max */
static double smin(double a, double b) { return (b < a) ? b : a; }
static double smax(double a, double b) { return (a < b) ? b : a; }

/* ------------------------------------------------------------------------- */
/* FluidElement (DRAGON/FluidElement/FluidElement.cpp, Arithmetic.cpp)         */

typedef struct { double x, y, z; } vec_t;
typedef struct { double rho, p; vec_t v; vec_t B; } prim_t;
typedef struct { double rho, E; vec_t m; vec_t B; } cons_t;

static double dot(vec_t a, vec_t b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static vec_t vscale(vec_t a, double s) { vec_t r = {a.x * s, a.y * s, a.z * s}; return r; }
static vec_t vdiv(vec_t a, double s) { vec_t r = {a.x / s, a.y / s, a.z / s}; return r; }
static vec_t vadd(vec_t a, vec_t b) { vec_t r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static vec_t vsub(vec_t a, vec_t b) { vec_t r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static vec_t vzero(void) { vec_t r = {0, 0, 0}; return r; }
/* cross (Arithmetic.cpp:95-101) */
static vec_t cross(vec_t u, vec_t v) {
    vec_t w;
    w.x = u.y * v.z - u.z * v.y;
    w.y = u.z * v.x - u.x * v.z;
    w.z = u.x * v.y - u.y * v.x;
    return w;
}
static prim_t pzero(void) { prim_t w; memset(&w, 0, sizeof w); return w; }
static cons_t czero(void) { cons_t u; memset(&u, 0, sizeof u); return u; }

/* PrimitiveState::energy (FluidElement.cpp:53-59) */
static double energy(prim_t w) {
    double E = w.p / (GAMMA - 1.0) + (w.rho / 2) * dot(w.v, w.v);
#if MHD
    E += dot(w.B, w.B) * k1_8pi;
#endif
    return E;
}
/* ConservativeState::pressure (FluidElement.cpp:60-66) */
static double pressure(cons_t u) {
    double Et = u.E - dot(u.m, u.m) / (2 * u.rho);
#if MHD
    Et -= dot(u.B, u.B) * k1_8pi;
#endif
    return (GAMMA - 1.0) * Et;
}
/* ConservativeState(PrimitiveState) (FluidElement.cpp:35-42) */
static cons_t p2c(prim_t w) {
    cons_t u = czero();
    u.rho = w.rho;
    u.m = vscale(w.v, w.rho);
    u.E = energy(w);
#if MHD
    u.B = w.B;
#endif
    return u;
}
/* PrimitiveState(ConservativeState) (FluidElement.cpp:44-51) */
static prim_t c2p(cons_t u) {
    prim_t w = pzero();
    w.rho = u.rho;
    w.v = vdiv(u.m, u.rho);
    w.p = pressure(u);
#if MHD
    w.B = u.B;
#endif
    return w;
}
/* PrimitiveState::enthalpy (FluidElement.cpp:69-75) */
static double enthalpy(prim_t w) {
    double h = energy(w) + w.p;
#if MHD
    h += dot(w.B, w.B) * k1_8pi;
#endif
    return h / w.rho;
}
static int vfinite(vec_t v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }
/* isPhysical / isFinite (FluidElement.cpp:82-96) */
static int pphys(prim_t w) {
#if MHD
    if (!vfinite(w.B)) return 0;
#endif
    return isfinite(w.rho) && vfinite(w.v) && isfinite(w.p) && w.rho > 0.0 && w.p > 0.0;
}
static int cfin(cons_t u) {
#if MHD
    if (!vfinite(u.B)) return 0;
#endif
    return isfinite(u.rho) && vfinite(u.m) && isfinite(u.E);
}
static int cphys(cons_t u) { return cfin(u) && u.rho > 0.0 && pressure(u) > 0.0; }

/* wave speeds (FluidElement.cpp:99-120); the compiler folds pow(x,2) to x*x */
static double cs(prim_t w) { return sqrt(GAMMA * w.p / w.rho); }
#if MHD
static double calf(prim_t w) { return sqrt(dot(w.B, w.B) / w.rho) / sq4pi(); }
static double cfast_k(prim_t w, double Bk) {
    double c = cs(w), a = calf(w), c2 = c * c, a2 = a * a, ak2 = (Bk * Bk / w.rho) * k1_4pi;
    double disc = smax(0.0, (c2 + a2) * (c2 + a2) * 0.25 - ak2 * c2);
    return sqrt((c2 + a2) * 0.5 + sqrt(disc));
}
static double cfast(prim_t w) { return cfast_k(w, w.B.x); }
static double cfast_max(prim_t w) {
    double Bk;
    if (w.B.x * w.B.x < w.B.y * w.B.y) Bk = (w.B.x * w.B.x < w.B.z * w.B.z) ? w.B.x : w.B.z;
    else Bk = (w.B.y * w.B.y < w.B.z * w.B.z) ? w.B.y : w.B.z;
    return cfast_k(w, Bk);
}
#endif

/* ConservativeState::flux(vec3 v) (FluidElement.cpp:133-155) */
static cons_t cflux(cons_t u, vec_t v) {
    cons_t F = czero();
    double p = pressure(u);
    F.rho = u.m.x;
    F.m = vscale(u.m, v.x);
    F.m.x += p;
    F.E = (u.E + p) * v.x;
#if MHD
    double pmag = dot(u.B, u.B) * k1_8pi;
    F.m.x += pmag;
    F.E += pmag * v.x;
    vec_t ten = vscale(vscale(u.B, u.B.x), k1_4pi);
    F.m = vsub(F.m, ten);
    F.E -= dot(v, ten);
    F.B = vsub(vscale(u.B, v.x), vscale(v, u.B.x));
    F.B.x = 0;
#endif
    return F;
}
static cons_t pflux(prim_t w) { return cflux(p2c(w), w.v); }

static cons_t cadd(cons_t a, cons_t b) {
    a.rho += b.rho; a.m = vadd(a.m, b.m); a.E += b.E;
#if MHD
    a.B = vadd(a.B, b.B);
#endif
    return a;
}
static cons_t csub(cons_t a, cons_t b) {
    a.rho -= b.rho; a.m = vsub(a.m, b.m); a.E -= b.E;
#if MHD
    a.B = vsub(a.B, b.B);
#endif
    return a;
}
static cons_t cmul(cons_t a, double s) {
    a.rho *= s; a.m = vscale(a.m, s); a.E *= s;
#if MHD
    a.B = vscale(a.B, s);
#endif
    return a;
}
static cons_t cdivs(cons_t a, double s) {
    a.rho /= s; a.m = vdiv(a.m, s); a.E /= s;
#if MHD
    a.B = vdiv(a.B, s);
#endif
    return a;
}
/* PrimitiveState += ConservativeState (FluidElement.cpp:157-162) */
static prim_t padd(prim_t w, cons_t d) { return c2p(cadd(p2c(w), d)); }

static void vswapxy(vec_t* v) { double t = v->x; v->x = v->y; v->y = t; }
static void vswapxz(vec_t* v) { double t = v->x; v->x = v->z; v->z = t; }
static void pswap(prim_t* w, int ax) {
    if (ax == 1) { vswapxy(&w->v); vswapxy(&w->B); }
    else if (ax == 2) { vswapxz(&w->v); vswapxz(&w->B); }
}
static void cswap(cons_t* u, int ax) {
    if (ax == 1) { vswapxy(&u->m); vswapxy(&u->B); }
    else if (ax == 2) { vswapxz(&u->m); vswapxz(&u->B); }
}

/* ------------------------------------------------------------------------- */
/* Limiters and MUSCL-Hancock (Hydro/Reconstruction/Limiters.cpp, MUSCL.cpp)   */

static double minmod(double a, double b) {
    if (a * b <= 0) return 0;
    return (fabs(a) < fabs(b)) ? a : b;
}
static double lim_mc(double a, double b) {
    if (a * b <= 0) return 0;
    double c = fabs(a + b);
    if (c < 4 * fabs(a) && c < 4 * fabs(b)) return a < 0 ? -c / 2 : c / 2;
    return 2 * minmod(a, b);
}
static double lim_vanleer(double a, double b) {
    if (a * b <= 0) return 0;
    return 2 * a * b / (a + b);
}
static double lim_superbee(double a, double b) {
    if (a * b <= 0) return 0;
    double aa = fabs(a), bb = fabs(b);
    double s1 = smin(2 * aa, bb), s2 = smin(aa, 2 * bb);
    double mag = smax(s1, s2);
    return a < 0 ? -mag : mag;
}
static double lim_vanalbada(double a, double b) {
    if (a * b <= 0) return 0;
    return a * b * (a + b) / (a * a + b * b);
}
/* TVD::limit (Limiters.cpp:17-39) */
static double limit(double a, double b) {
    switch (O.limiter) {
        case L_MC: return lim_mc(a, b);
        case L_VANLEER: return lim_vanleer(a, b);
        case L_SUPERBEE: return lim_superbee(a, b);
        case L_VANALBADA: return lim_vanalbada(a, b);
        default: return minmod(a, b);
    }
}
double ora_limiter(int kind, double a, double b) {
    int keep = O.limiter;
    O.limiter = kind;
    double r = limit(a, b);
    O.limiter = keep;
    return r;
}
static vec_t vlimit(vec_t a, vec_t b) { vec_t r = {limit(a.x, b.x), limit(a.y, b.y), limit(a.z, b.z)}; return r; }

/* TVD::MUSCL (MUSCL.cpp:16-61) */
static void muscl(prim_t wL, prim_t* oL, prim_t wC, prim_t* oR, prim_t wR, double dt_dL, vec_t dB) {
    prim_t dW = pzero(), L = pzero(), R = pzero();
    dW.rho = limit(wC.rho - wL.rho, wR.rho - wC.rho);
    dW.v = vlimit(vsub(wC.v, wL.v), vsub(wR.v, wC.v));
    dW.p = limit(wC.p - wL.p, wR.p - wC.p);
#if MHD
    dW.B = vlimit(vsub(wC.B, wL.B), vsub(wR.B, wC.B));
#endif
    L.rho = wC.rho - 0.5 * dW.rho;
    R.rho = wC.rho + 0.5 * dW.rho;
    L.v = vsub(wC.v, vscale(dW.v, 0.5));
    R.v = vadd(wC.v, vscale(dW.v, 0.5));
    L.p = wC.p - 0.5 * dW.p;
    R.p = wC.p + 0.5 * dW.p;
#if MHD
    L.B = vsub(wC.B, vscale(dW.B, 0.5));
    R.B = vadd(wC.B, vscale(dW.B, 0.5));
#endif
    cons_t UL = p2c(L), UR = p2c(R);
    cons_t corr = cmul(csub(cflux(UR, R.v), cflux(UL, L.v)), 0.5 * dt_dL);
#if MHD
    const double a_s = (R.B.x - L.B.x) * dt_dL;
    const double vy = 0.5 * (L.v.y + R.v.y), vz = 0.5 * (L.v.z + R.v.z);
    const double dBy_ = 0.5 * wC.v.y * minmod(dB.x, -dB.y) - 0.5 * vy * a_s;
    const double dBz_ = 0.5 * wC.v.z * minmod(dB.x, -dB.z) - 0.5 * vz * a_s;
    corr.B.y -= dBy_;
    corr.B.z -= dBz_;
    corr.E -= k1_4pi * (wC.B.y * dBy_ + wC.B.z * dBz_);
#else
    (void)dB;
#endif
    *oL = c2p(csub(UL, corr));
    *oR = c2p(csub(UR, corr));
    if (pphys(*oL) && pphys(*oR)) return;
    *oL = wC;
    *oR = wC;
}

/* ------------------------------------------------------------------------- */
/* Riemann solvers (Hydro/Riemann/HLL.cpp, HLLD.cpp, Roe.cpp, Exact.cpp)        */

typedef struct { prim_t L, R; } rp_t;  /* struct Riemann: solvers may edit L/R (normal B) */

/* HLL::roeAvg (HLL.cpp:21-37) */
static prim_t roe_avg(prim_t L, prim_t R) {
    double sql = sqrt(L.rho), sqr = sqrt(R.rho);
    double _sql = sql / (sql + sqr), _sqr = sqr / (sql + sqr);
    prim_t w = pzero();
    w.rho = sql * sqr;
    w.v = vadd(vscale(L.v, _sql), vscale(R.v, _sqr));
#if MHD
    w.B = vadd(vscale(L.B, _sql), vscale(R.B, _sqr));
#endif
    double H = _sql * enthalpy(L) + _sqr * enthalpy(R);
    double a2 = (GAMMA - 1) * (H - dot(w.v, w.v) / 2);
    w.p = a2 * w.rho / GAMMA;
    return w;
}
/* Riemann::HLL(SL,SR) (HLL.cpp:87-96) */
static cons_t hll_s(rp_t* r, double sl, double sr) {
    if (sl >= 0) return cflux(p2c(r->L), r->L.v);
    if (sr <= 0) return cflux(p2c(r->R), r->R.v);
    cons_t UL = p2c(r->L), UR = p2c(r->R);
    cons_t FL = cflux(UL, r->L.v), FR = cflux(UR, r->R.v);
    return cdivs(cadd(csub(cmul(FL, sr), cmul(FR, sl)), cmul(csub(UR, UL), sl * sr)), sr - sl);
}
/* Riemann::HLL (HLL.cpp:42-60) */
static cons_t hll(rp_t* r) {
    prim_t M = roe_avg(r->L, r->R);
#if MHD
    double Bx = (r->L.B.x + r->R.B.x) / 2;
    r->L.B.x = Bx; r->R.B.x = Bx;
    double aL = cfast(r->L), aR = cfast(r->R), aM = cfast(M);
#else
    double aL = cs(r->L), aR = cs(r->R), aM = cs(M);
#endif
    double SL = smin(r->L.v.x - aL, M.v.x - aM);
    double SR = smax(r->R.v.x + aR, M.v.x + aM);
    return hll_s(r, SL, SR);
}
/* Riemann::HLLE (HLL.cpp:61-84) */
static cons_t hlle(rp_t* r) {
    double sql = sqrt(r->L.rho), sqr = sqrt(r->R.rho);
    double _sql = sql / (sql + sqr), _sqr = sqr / (sql + sqr);
#if MHD
    double Bx = (r->L.B.x + r->R.B.x) / 2;
    r->L.B.x = Bx; r->R.B.x = Bx;
    double aL = cfast(r->L), aR = cfast(r->R);
#else
    double aL = cs(r->L), aR = cs(r->R);
#endif
    double _v = (r->R.v.x - r->L.v.x) / (sql + sqr);
    double d = (_sql * aL * aL + _sqr * aR * aR) + 0.5 * (sql * sqr) * _v * _v;
    d = sqrt(d);
    double u = _sql * r->L.v.x + _sqr * r->R.v.x;
    double SL = smin(r->L.v.x - aL, u - d);
    double SR = smax(r->R.v.x + aR, u + d);
    return hll_s(r, SL, SR);
}

#if !MHD
/* Riemann::HLLC (HLL.cpp:103-132) */
static cons_t hllc(rp_t* r) {
    prim_t L = r->L, R = r->R;
    prim_t M = roe_avg(L, R);
    double aL = cs(L), aR = cs(R), aM = cs(M);
    double sl = smin(L.v.x - aL, M.v.x - aM);
    double sr = smax(R.v.x + aR, M.v.x + aM);
    if (sl >= 0) return pflux(L);
    if (sr <= 0) return pflux(R);
    double _pr = R.p + R.rho * R.v.x * (R.v.x - sr), _pl = L.p + L.rho * L.v.x * (L.v.x - sl);
    double sc = (_pr - _pl) / (R.rho * (R.v.x - sr) - L.rho * (L.v.x - sl));
    prim_t X = (sc > 0 ? L : R);
    double sx = sc > 0 ? sl : sr;
    cons_t UX = p2c(X);
    cons_t U = cdivs(cmul(UX, sx - X.v.x), sx - sc);
    U.m.x = U.rho * sc;
    U.E += U.rho * (sc - X.v.x) * (sc + X.p / (X.rho * (sx - X.v.x)));
    return cadd(cflux(UX, X.v), cmul(csub(U, UX), sx));
}

/* Riemann::Roe with Harten-Hyman (Roe.cpp:19-96) */
static cons_t ck(double rho, double E, double mx, double my, double mz) {
    cons_t K = czero();
    K.rho = rho; K.E = E; K.m.x = mx; K.m.y = my; K.m.z = mz;
    return K;
}
static cons_t roe(rp_t* r) {
    prim_t L = r->L, R = r->R;
    double sql = sqrt(L.rho), sqr = sqrt(R.rho);
    double _sql = sql / (sql + sqr), _sqr = sqr / (sql + sqr);
    double _rho = sql * sqr;
    vec_t v = vadd(vscale(L.v, _sql), vscale(R.v, _sqr));
    double H = _sql * enthalpy(L) + _sqr * enthalpy(R);
    double a = sqrt((GAMMA - 1) * (H - dot(v, v) / 2));
    double lambda[5] = {v.x - a, v.x, v.x, v.x, v.x + a};
    double V2 = dot(v, v);
    cons_t K[5] = {ck(1, H - v.x * a, v.x - a, v.y - 0, v.z - 0), ck(1, V2 / 2, v.x, v.y, v.z),
                   ck(0, v.y, 0, 1, 0), ck(0, v.z, 0, 0, 1), ck(1, H + v.x * a, v.x + a, v.y + 0, v.z + 0)};
    cons_t UL = p2c(L), UR = p2c(R);
    double alpha[5] = {((R.p - L.p) - _rho * a * (R.v.x - L.v.x)) / (2 * a * a),
                       (R.rho - L.rho) - (R.p - L.p) / (a * a), _rho * (R.v.y - L.v.y), _rho * (R.v.z - L.v.z),
                       ((R.p - L.p) + _rho * a * (R.v.x - L.v.x)) / (2 * a * a)};
    cons_t SL = cadd(UL, cmul(K[0], alpha[0]));
    double aL = sqrt(GAMMA * L.p / L.rho), aSL = sqrt(GAMMA * pressure(SL) / SL.rho);
    double lL = L.v.x - aL, lLS = SL.m.x / SL.rho - aSL;
    if (lL < 0 && lLS > 0) {
        double lam = lL * (lambda[0] - lLS) / (lL - lLS);
        return cadd(cflux(UL, L.v), cmul(K[0], lam * alpha[0]));
    }
    cons_t SR = csub(UR, cmul(K[4], alpha[4]));
    double aR = sqrt(GAMMA * R.p / R.rho), aSR = sqrt(GAMMA * pressure(SR) / SR.rho);
    double lR = R.v.x + aR, lRS = SR.m.x / SR.rho + aSR;
    if (lR > 0 && lRS < 0) {
        double lam = lR * (lambda[4] - lRS) / (lR - lRS);
        return csub(cflux(UR, R.v), cmul(K[4], lam * alpha[4]));
    }
    cons_t F = cadd(cflux(UL, L.v), cflux(UR, R.v));
    for (int i = 0; i < 5; i++) F = csub(F, cmul(K[i], alpha[i] * fabs(lambda[i])));
    return cdivs(F, 2);
}

/* Exact solver (Exact.cpp:18-180) */
static double ex_f(double p, prim_t w) {
    if (p > w.p) {
        double A = k2_Gp1 / w.rho, B = kGm1_Gp1 * w.p;
        return (p - w.p) * sqrt(A / (B + p));
    }
    return k2_Gm1 * cs(w) * (pow(p / w.p, kGm1_2G) - 1);
}
static double ex_df(double p, prim_t w) {
    if (p > w.p) {
        double A = k2_Gp1 / w.rho, B = kGm1_Gp1 * w.p;
        return sqrt(A / (p + B)) * (1 - (p - w.p) / (2 * (B + p)));
    }
    return pow(p / w.p, -kGp1_2G) / (w.rho * cs(w));
}
static double ex_rho(prim_t w, double p) {
    if (p > w.p) return w.rho * (p + kGm1_Gp1 * w.p) / (kGm1_Gp1 * p + w.p);
    return w.rho * pow(p / w.p, kGinv);
}
typedef struct { prim_t wL, wR, sL, sR; } sol_t;
static int g_newton_iters;
/* Optional record of every Newton-branch solve: (rhoL, vxL, pL, rhoR, vxR, pR,
 * p*, iterations; negative when the cap, not the tolerance, ended it) per row. Test infrastructure for the learned-guess sample
 * log; off unless ora_exact_log_start was called. */
static double* g_log_buf;
static long g_log_cap, g_log_n;

static sol_t exact_solve(prim_t L, prim_t R, double pGuess) {
    sol_t s;
    s.wL = L; s.wR = R;
    s.sL = pzero(); s.sR = pzero();
    s.sL.v = L.v; s.sR.v = R.v;
    g_newton_iters = 0;
    double p_min = smin(L.p, R.p);
    if (ex_f(p_min, L) + ex_f(p_min, R) + R.v.x - L.v.x >= 0) { /* TRRS (Exact.cpp:96-113) */
        double aL = cs(L), aR = cs(R);
        double LR = pow(L.p / R.p, kGm1_2G) * aR / aL;
        s.sL.v.x = (LR * L.v.x + R.v.x + k2_Gm1 * (LR * aL - aR)) / (LR + 1);
        s.sR.v.x = s.sL.v.x;
        s.sL.p = L.p * pow(1 - kGm1_2 * (s.sL.v.x - L.v.x) / aL, k2G_Gm1);
        s.sR.p = s.sL.p;
        s.sL.rho = L.rho * pow(s.sL.p / L.p, kGinv);
        s.sR.rho = R.rho * pow(s.sR.p / R.p, kGinv);
        return s;
    }
    /* exact_StarP (Exact.cpp:71-84) */
    double p = pGuess, CHA = 1;
    int iters = O.exact_max_iters;
    do {
        double fp = ex_f(p, L) + ex_f(p, R) + R.v.x - L.v.x;
        double dfdp = ex_df(p, L) + ex_df(p, R);
        double delta = smin(fp / dfdp, 0.8 * p);
        p -= delta;
        CHA = fabs(delta / (p + delta / 2));
        g_newton_iters++;
    } while (CHA > O.exact_tol && --iters != 0);
    if (g_log_buf) {
        if (g_log_n < g_log_cap) {
            double* row = g_log_buf + 8 * g_log_n;
            row[0] = L.rho; row[1] = L.v.x; row[2] = L.p;
            row[3] = R.rho; row[4] = R.v.x; row[5] = R.p;
            row[6] = p; row[7] = (CHA > O.exact_tol) ? -g_newton_iters : g_newton_iters;
        }
        g_log_n++;
    }
    s.sL.p = p;
    s.sR.p = p;
    s.sL.v.x = (L.v.x + R.v.x + ex_f(p, R) - ex_f(p, L)) / 2.0;
    s.sR.v.x = s.sL.v.x;
    s.sL.rho = ex_rho(L, p);
    s.sR.rho = ex_rho(R, p);
    return s;
}
static void ex_mirror(sol_t* s) {
    prim_t t = s->wL; s->wL = s->wR; s->wR = t;
    t = s->sL; s->sL = s->sR; s->sR = t;
    s->wL.v.x *= -1; s->wR.v.x *= -1; s->sL.v.x *= -1; s->sR.v.x *= -1;
}
/* RiemannSolution::sample (Exact.cpp:122-163) */
static prim_t ex_sample(sol_t s, double x_t) {
    if (fabs(s.sR.v.x - x_t) < 1e-12) {
        double sql = sqrt(s.sL.rho), sqr = sqrt(s.sR.rho);
        return c2p(cdivs(cadd(cmul(p2c(s.sL), sql), cmul(p2c(s.sR), sqr)), sql + sqr));
    }
    int isLeft = x_t < s.sR.v.x;
    if (isLeft) { ex_mirror(&s); x_t = -x_t; }
    double a = cs(s.wR);
    int zone;
    if (s.sR.p > s.wR.p) {
        double scale = sqrt(kGp1_2G * s.sR.p / s.wR.p + kGm1_2G);
        zone = ((x_t - s.wR.v.x) > scale * a) ? 1 : 3;
    } else {
        if ((x_t - s.wR.v.x) > a) zone = 1;
        else if ((x_t - s.sR.v.x) > a) zone = 2;
        else if ((x_t - s.sR.v.x) > a * pow(s.sR.p / s.wR.p, kGm1_2G)) zone = 2;
        else zone = 3;
    }
    prim_t st;
    if (zone == 1) st = s.wR;
    else if (zone == 3) st = s.sR;
    else {
        st = s.wR;
        double scale = k2_Gp1 - kGm1_Gp1 * (s.wR.v.x - x_t) / a;
        st.rho *= pow(scale, k2_Gm1);
        st.p *= pow(scale, k2G_Gm1);
        st.v.x = k2_Gp1 * (x_t - a + s.wR.v.x * kGm1_2);
    }
    if (isLeft) st.v.x *= -1;
    return st;
}
static cons_t exact_flux(rp_t* r) {
    sol_t s = exact_solve(r->L, r->R, (r->L.p + r->R.p) / 2.0);
    return pflux(ex_sample(s, 0));
}
#endif /* !MHD */

#if MHD
/* compute_outer_star (HLLD.cpp:21-37) */
static void outer_star(cons_t* us, prim_t K, double xK, double SK, double SM, double pT, double Bx) {
    double Bx2 = (Bx * Bx) * k1_4pi;
    double den = xK * (SK - SM) - Bx2;
    us->B = (fabs(den) < 1e-12) ? K.B : vdiv(vscale(K.B, xK * (SK - K.v.x) - Bx2), den);
    us->B.x = Bx;
    vec_t vs = vsub(K.v, fabs(den) < 1e-12 ? vzero() : vscale(vdiv(vscale(vscale(K.B, Bx), SM - K.v.x), den), k1_4pi));
    vs.x = SM;
    us->m = vscale(vs, us->rho);
    us->E = energy(K) * (SK - K.v.x);
    us->E += pT * SM - (K.p + dot(K.B, K.B) * k1_8pi) * K.v.x;
    us->E += Bx * (dot(K.v, K.B) - dot(vs, us->B)) * k1_4pi;
    us->E /= (SK - SM);
}
/* compute_outer_star_zero_B (HLLD.cpp:137-150) */
static void outer_star0(cons_t* us, prim_t K, double SK, double SM, double pT) {
    us->B = (fabs(SK - SM) < 1e-12) ? K.B : vdiv(vscale(K.B, SK - K.v.x), SK - SM);
    us->B.x = 0;
    vec_t vs = K.v;
    vs.x = SM;
    us->m = vscale(vs, us->rho);
    us->E = energy(K) * (SK - K.v.x);
    us->E += pT * SM - (K.p + dot(K.B, K.B) * k1_8pi) * K.v.x;
    us->E /= (SK - SM);
}
/* Riemann::HLLD_zero_B (HLLD.cpp:152-205) */
static cons_t hlld0(rp_t* r, double SL, double SR) {
    prim_t L = r->L, R = r->R;
    double pTL = L.p + dot(L.B, L.B) * k1_8pi, pTR = R.p + dot(R.B, R.B) * k1_8pi;
    double xL = L.rho * (SL - L.v.x), xR = R.rho * (SR - R.v.x);
    double SM = ((xR * R.v.x - xL * L.v.x) - (pTR - pTL)) / (xR - xL);
    cons_t usL = czero(), usR = czero();
    usL.rho = xL / (SL - SM);
    usR.rho = xR / (SR - SM);
    cons_t FsL = czero(), FsR = czero();
    prim_t wsL = pzero(), wsR = pzero();
    double pT = (xR * pTL - xL * pTR + xL * xR * (R.v.x - L.v.x)) / (xR - xL);
    if (SM >= 0) {
        outer_star0(&usL, L, SL, SM, pT);
        wsL.rho = usL.rho; wsL.v = vdiv(usL.m, usL.rho); wsL.B = usL.B;
        wsL.p = pT - dot(wsL.B, wsL.B) * k1_8pi;
        if (!pphys(wsL) || !cfin(usL)) return hlle(r);
        FsL = cadd(pflux(L), cmul(csub(usL, p2c(L)), SL));
        FsL.B.x = 0;
    }
    if (SM <= 0) {
        outer_star0(&usR, R, SR, SM, pT);
        wsR.rho = usR.rho; wsR.v = vdiv(usR.m, usR.rho); wsR.B = usR.B;
        wsR.p = pT - dot(wsR.B, wsR.B) * k1_8pi;
        if (!pphys(wsR) || !cfin(usR)) return hlle(r);
        FsR = cadd(pflux(R), cmul(csub(usR, p2c(R)), SR));
        FsR.B.x = 0;
    }
    if (SM > 0) return FsL;
    if (SM < 0) return FsR;
    double sql = sqrt(wsL.rho), sqr = sqrt(wsR.rho);
    double _sql = sql / (sql + sqr), _sqr = sqr / (sql + sqr);
    return cadd(cmul(FsL, _sql), cmul(FsR, _sqr));
}
/* Riemann::HLLD (HLLD.cpp:38-133) */
static cons_t hlld(rp_t* r) {
    double Bx = (r->L.B.x + r->R.B.x) / 2;
    r->L.B.x = Bx; r->R.B.x = Bx;
    prim_t L = r->L, R = r->R;
    double cl = cfast(L), cr = cfast(R);
    double SL = smin(L.v.x - cl, R.v.x - cr);
    if (SL >= 0) return pflux(L);
    double SR = smax(L.v.x + cl, R.v.x + cr);
    if (SR <= 0) return pflux(R);
    double cutoff = smax(dot(L.B, L.B) + dot(R.B, R.B), 1e-100);
    if (Bx * Bx < 1e-12 * cutoff) return hlld0(r, SL, SR);
    double pTL = L.p + dot(L.B, L.B) * k1_8pi, pTR = R.p + dot(R.B, R.B) * k1_8pi;
    double xL = L.rho * (SL - L.v.x), xR = R.rho * (SR - R.v.x);
    double SM = ((xR * R.v.x - xL * L.v.x) - (pTR - pTL)) / (xR - xL);
    cons_t usL = czero(), usR = czero();
    usL.rho = xL / (SL - SM);
    double SsL = SM - fabs(Bx) / (sq4pi() * sqrt(usL.rho));
    usR.rho = xR / (SR - SM);
    double SsR = SM + fabs(Bx) / (sq4pi() * sqrt(usR.rho));
    cons_t FsL = czero(), FsR = czero();
    prim_t wsL = pzero(), wsR = pzero();
    double pT = (xR * pTL - xL * pTR + xL * xR * (R.v.x - L.v.x)) / (xR - xL);
    if (SsR >= 0) {
        outer_star(&usL, L, xL, SL, SM, pT, Bx);
        wsL.rho = usL.rho; wsL.v = vdiv(usL.m, usL.rho); wsL.B = usL.B;
        wsL.p = pT - dot(wsL.B, wsL.B) * k1_8pi;
        if (!pphys(wsL) || !cphys(usL)) return hlle(r);
        FsL = cadd(pflux(L), cmul(csub(usL, p2c(L)), SL));
        FsL.B.x = 0;
    }
    if (SsL <= 0) {
        outer_star(&usR, R, xR, SR, SM, pT, Bx);
        wsR.rho = usR.rho; wsR.v = vdiv(usR.m, usR.rho); wsR.B = usR.B;
        wsR.p = pT - dot(wsR.B, wsR.B) * k1_8pi;
        if (!pphys(wsR) || !cphys(usR)) return hlle(r);
        FsR = cadd(pflux(R), cmul(csub(usR, p2c(R)), SR));
        FsR.B.x = 0;
    }
    if (SsL >= 0) return FsL;
    if (SsR <= 0) return FsR;
    prim_t ws = SM >= 0 ? wsL : wsR;
    double sqL = sqrt(wsL.rho), sqR = sqrt(wsR.rho);
    double _sqL = sqL / (sqL + sqR), _sqR = sqR / (sqL + sqR);
    double sbx = Bx > 0 ? sq4pi() : (Bx < 0 ? -sq4pi() : 0);
    cons_t uss = czero();
    prim_t wss = pzero();
    wss.rho = ws.rho;
    uss.rho = wss.rho;
    wss.v = vadd(vadd(vscale(wsL.v, _sqL), vscale(wsR.v, _sqR)),
                 vdiv(vscale(vscale(vsub(usR.B, usL.B), sbx), k1_4pi), sqL + sqR));
    wss.v.x = SM;
    uss.m = vscale(wss.v, uss.rho);
    wss.B = vadd(vadd(vscale(usR.B, _sqL), vscale(usL.B, _sqR)),
                 vdiv(vscale(vscale(vscale(vsub(wsR.v, wsL.v), sbx), sqL), sqR), sqL + sqR));
    wss.B.x = Bx;
    uss.B = wss.B;
    double dE = sbx * (dot(ws.v, ws.B) - dot(wss.v, wss.B)) * k1_4pi * sqrt(wss.rho);
    uss.E = SM >= 0 ? usL.E - dE : usR.E + dE;
    wss.p = pT - dot(wss.B, wss.B) * k1_8pi;
    if (!pphys(wss) || !cfin(uss)) return hlle(r);
    if (SM >= 0) return cadd(FsL, cmul(csub(uss, usL), SsL));
    return cadd(FsR, cmul(csub(uss, usR), SsR));
}
#endif

/* Riemann::flux with verify_and_fallback (Flux.cpp:17-97) */
static cons_t rflux(rp_t* r, double dt_dx) {
    cons_t F;
#if MHD
    switch (O.riemann) {
        case R_HLL: F = hll(r); break;
        case R_HLLE: F = hlle(r); break;
        default: F = hlld(r); break;
    }
    (void)dt_dx;
#else
    switch (O.riemann) {
        case R_HLLX:
        case R_HLLC: F = hllc(r); break;
        case R_HLL: F = hll(r); break;
        case R_HLLE: F = hlle(r); break;
        case R_ROE: F = roe(r); break;
        default: F = exact_flux(r); break;
    }
    if (dt_dx > 0) {
        cons_t UL = p2c(r->L), UR = p2c(r->R);
        if (cphys(csub(UL, cmul(F, dt_dx))) && cphys(cadd(UR, cmul(F, dt_dx)))) return F;
        F = exact_flux(r);
        if (cphys(csub(UL, cmul(F, dt_dx))) && cphys(cadd(UR, cmul(F, dt_dx)))) return F;
        g_fail = 1;
    }
#endif
    return F;
}
/* Riemann::flux_X/Y/Z (Flux.cpp:101-115) */
static cons_t rflux_ax(prim_t L, prim_t R, double dt, int ax) {
    rp_t r = {L, R};
    pswap(&r.L, ax);
    pswap(&r.R, ax);
    cons_t F = rflux(&r, dt);
    cswap(&F, ax);
    return F;
}

/* ------------------------------------------------------------------------- */
/* Arrays (Hydro/ExtendedArray/ExtendedArray.hpp): padded, last index fastest   */

typedef struct { int dim, n[3], g; size_t ny, nz; } shape_t;
static shape_t mkshape(int dim, int nx, int ny, int nz, int g) {
    shape_t s;
    s.dim = dim; s.n[0] = nx; s.n[1] = ny; s.n[2] = nz; s.g = g;
    s.ny = dim >= 2 ? (size_t)(ny + 2 * g) : 1;
    s.nz = dim >= 3 ? (size_t)(nz + 2 * g) : 1;
    return s;
}
static size_t shape_count(shape_t s) { return (size_t)(s.n[0] + 2 * s.g) * s.ny * s.nz; }
static size_t IX(shape_t s, int i, int j, int k) {
    if (s.dim == 1) return (size_t)(i + s.g);
    if (s.dim == 2) return (size_t)(i + s.g) * s.ny + (size_t)(j + s.g);
    return ((size_t)(i + s.g) * s.ny + (size_t)(j + s.g)) * s.nz + (size_t)(k + s.g);
}

struct ora_grid {
    int dim, n[3], g;
    double d[3];
    shape_t cs, fs;   /* cells, faces (n+1) */
    prim_t* w;
    vec_t* B;
    int nbc;
    struct { int type, faces, corners; prim_t st; } bc[32];
};

ora_grid* ora_grid_new(int dim, int nx, int ny, int nz, double dx, double dy, double dz, int ghosts) {
    ora_grid* G = (ora_grid*)calloc(1, sizeof(ora_grid));
    G->dim = dim;
    G->n[0] = nx; G->n[1] = dim >= 2 ? ny : 1; G->n[2] = dim >= 3 ? nz : 1;
    G->d[0] = dx; G->d[1] = dim >= 2 ? dy : 0; G->d[2] = dim >= 3 ? dz : 0;
    /* validGhosts (Splitting.cpp:23-31) */
    int gmin = MHD ? 3 : 2;
    G->g = ghosts > gmin ? ghosts : gmin;
    G->cs = mkshape(dim, G->n[0], G->n[1], G->n[2], G->g);
    G->fs = mkshape(dim, G->n[0] + 1, G->n[1] + 1, G->n[2] + 1, G->g);
    G->w = (prim_t*)calloc(shape_count(G->cs), sizeof(prim_t));
    if (MHD && dim >= 2) G->B = (vec_t*)calloc(shape_count(G->fs), sizeof(vec_t));
    return G;
}
void ora_grid_free(ora_grid* G) {
    if (!G) return;
    free(G->w);
    free(G->B);
    free(G);
}
int ora_grid_ghosts(const ora_grid* G) { return G->g; }

static void put_prim(prim_t w, double* a) {
    a[0] = w.rho; a[1] = w.p; a[2] = w.v.x; a[3] = w.v.y; a[4] = w.v.z;
#if MHD
    a[5] = w.B.x; a[6] = w.B.y; a[7] = w.B.z;
#endif
}
static prim_t get_prim(const double* a) {
    prim_t w = pzero();
    w.rho = a[0]; w.p = a[1]; w.v.x = a[2]; w.v.y = a[3]; w.v.z = a[4];
#if MHD
    w.B.x = a[5]; w.B.y = a[6]; w.B.z = a[7];
#endif
    return w;
}
void ora_grid_set_prim(ora_grid* G, const double* a) {
    size_t n = shape_count(G->cs);
    for (size_t m = 0; m < n; m++) G->w[m] = get_prim(a + m * NF);
}
void ora_grid_get_prim(const ora_grid* G, double* a) {
    size_t n = shape_count(G->cs);
    for (size_t m = 0; m < n; m++) put_prim(G->w[m], a + m * NF);
}
void ora_grid_set_faceB(ora_grid* G, const double* a) {
    if (!G->B) return;
    size_t n = shape_count(G->fs);
    for (size_t m = 0; m < n; m++) { G->B[m].x = a[3 * m]; G->B[m].y = a[3 * m + 1]; G->B[m].z = a[3 * m + 2]; }
}
void ora_grid_get_faceB(const ora_grid* G, double* a) {
    if (!G->B) return;
    size_t n = shape_count(G->fs);
    for (size_t m = 0; m < n; m++) { a[3 * m] = G->B[m].x; a[3 * m + 1] = G->B[m].y; a[3 * m + 2] = G->B[m].z; }
}

#define W2(G, i, j) (G)->w[IX((G)->cs, i, j, 0)]
#define W3(G, i, j, k) (G)->w[IX((G)->cs, i, j, k)]
#define B2(G, i, j) (G)->B[IX((G)->fs, i, j, 0)]
#define B3(G, i, j, k) (G)->B[IX((G)->fs, i, j, k)]

/* ------------------------------------------------------------------------- */
/* Boundaries (Boundary/BoundaryTypes, BoundaryList.hpp:79-104)                 */

enum { BC_OUT = 0, BC_GATED = 1, BC_FIXED = 2, BC_REFL = 3, BC_PER = 4, BC_IGN = 5 };
#define XN 1
#define XP 2
#define YN 4
#define YP 8
#define ZN 16
#define ZP 32

void ora_boundary_clear(ora_grid* G) { G->nbc = 0; }
int ora_boundary_add(ora_grid* G, int type, int faces, int corners, const double* state) {
    if (G->nbc >= 32 || type < 0 || type > 5) return 1;
    if (type == BC_PER) { /* Periodic.cpp:14-15 */
        int f = 0;
        if (faces & (XN | XP)) f |= XN | XP;
        if (faces & (YN | YP)) f |= YN | YP;
        if (faces & (ZN | ZP)) f |= ZN | ZP;
        faces = f;
    }
    G->bc[G->nbc].type = type;
    G->bc[G->nbc].faces = faces;
    G->bc[G->nbc].corners = corners;
    G->bc[G->nbc].st = state ? get_prim(state) : pzero();
    G->nbc++;
    return 0;
}

/* Generic cell copy along axis a for one ghost layer of one face. */
static int *AXV(int* q, int a) { return &q[a]; }

/* Outflow / Gated / Fixed / Reflective / Periodic cell ghosts, in the
 * reference's face order (X-, X+, Y-, Y+, Z-, Z+). */
static void bc_cells(ora_grid* G, int type, int faces, int corners, prim_t st) {
    const int dim = G->dim, ng = G->g;
    if (type == BC_IGN) return;
    for (int a = 0; a < dim; a++) {
        int neg = faces & (1 << (2 * a)), pos = faces & (1 << (2 * a + 1));
        if (type == BC_PER) { if (!(neg || pos)) continue; }
        int t[2] = {-1, -1}, nt = 0;
        for (int b = 0; b < dim; b++) if (b != a) t[nt++] = b;
        int lo0 = 0, hi0 = 1, lo1 = 0, hi1 = 1;
        if (nt > 0) { lo0 = corners ? -ng : 0; hi0 = corners ? G->n[t[0]] + ng : G->n[t[0]]; }
        if (nt > 1) { lo1 = corners ? -ng : 0; hi1 = corners ? G->n[t[1]] + ng : G->n[t[1]]; }
        const int na = G->n[a];
        for (int side = 0; side < 2; side++) {
            if (type == BC_PER) { if (side == 1) break; }  /* periodic does both sides per layer */
            else if (side == 0 ? !neg : !pos) continue;
            for (int c0 = lo0; c0 < hi0; c0++)
                for (int c1 = lo1; c1 < hi1; c1++)
                    for (int gl = 1; gl <= ng; gl++) {
                        int q[3] = {0, 0, 0}, s[3] = {0, 0, 0};
                        if (nt > 0) q[t[0]] = s[t[0]] = c0;
                        if (nt > 1) q[t[1]] = s[t[1]] = c1;
                        if (type == BC_PER) {
                            q[a] = -gl; s[a] = na - gl;
                            W3(G, q[0], q[1], q[2]) = W3(G, s[0], s[1], s[2]);
                            q[a] = na - 1 + gl; s[a] = gl - 1;
                            W3(G, q[0], q[1], q[2]) = W3(G, s[0], s[1], s[2]);
                            continue;
                        }
                        *AXV(q, a) = side == 0 ? -gl : na - 1 + gl;
                        if (type == BC_REFL) *AXV(s, a) = side == 0 ? gl - 1 : na - gl;
                        else *AXV(s, a) = side == 0 ? 0 : na - 1;
                        prim_t v = (type == BC_FIXED) ? st : W3(G, s[0], s[1], s[2]);
                        double* vn = a == 0 ? &v.v.x : (a == 1 ? &v.v.y : &v.v.z);
                        if (type == BC_GATED) {
                            if (side == 0 && *vn > 0) *vn = 0;
                            if (side == 1 && *vn < 0) *vn = 0;
                        } else if (type == BC_REFL) {
                            *vn *= -1;
#if MHD
                            v.B = vscale(v.B, -1);
                            if (a == 0) v.B.x *= -1; else if (a == 1) v.B.y *= -1; else v.B.z *= -1;
#endif
                        }
                        W3(G, q[0], q[1], q[2]) = v;
                    }
        }
    }
}

#if MHD
static double* bcomp(vec_t* v, int a) { return a == 0 ? &v->x : (a == 1 ? &v->y : &v->z); }
/* Face-B ghosts (Outflow.cpp:78-117,188-258; Reflective.cpp:99-137,233-300;
 * Periodic.cpp:311-331,371-405; Fixed.cpp:372-406,472-532). */
static void bc_faces(ora_grid* G, int type, int faces, int corners, prim_t st) {
    const int dim = G->dim, ng = G->g;
    if (type == BC_IGN) return;
    for (int a = 0; a < dim; a++) {
        int neg = faces & (1 << (2 * a)), pos = faces & (1 << (2 * a + 1));
        int t[2] = {-1, -1}, nt = 0;
        for (int b = 0; b < dim; b++) if (b != a) t[nt++] = b;
        int lo0 = corners ? -ng : 0, hi0 = corners ? G->n[t[0]] + ng : G->n[t[0]];
        int lo1 = 0, hi1 = 0;
        if (nt > 1) { lo1 = corners ? -ng : 0; hi1 = corners ? G->n[t[1]] + ng : G->n[t[1]]; }
        const int na = G->n[a];
        int tr0 = a == 0 ? 1 : 0, tr1 = a == 2 ? 1 : 2;
        for (int side = 0; side < 2; side++) {
            if (type == BC_PER) { if (side == 1 || !(neg || pos)) break; }
            else if (side == 0 ? !neg : !pos) continue;
            for (int c0 = lo0; c0 <= hi0; c0++)
                for (int c1 = lo1; c1 <= hi1; c1++) {
#define FB(ia) (*(q[a] = (ia), q[t[0]] = c0, (nt > 1 ? q[t[1]] = c1 : 0), &B3(G, q[0], q[1], q[2])))
                    int q[3] = {0, 0, 0};
                    if (type == BC_OUT || type == BC_GATED) {
                        if (side == 0) {
                            for (int gl = 1; gl <= ng; gl++) {
                                vec_t b0 = FB(0);
                                FB(-gl) = b0;
                                double v1 = *bcomp(&FB(-gl + 1), a), v2 = *bcomp(&FB(-gl + 2), a);
                                *bcomp(&FB(-gl), a) = 2 * v1 - v2;
                            }
                        } else {
                            vec_t bm = FB(na - 1);
                            *bcomp(&FB(na), tr0) = *bcomp(&bm, tr0);
                            *bcomp(&FB(na), tr1) = *bcomp(&bm, tr1);
                            for (int gl = 1; gl <= ng; gl++) {
                                vec_t bn = FB(na);
                                FB(na + gl) = bn;
                                double v1 = *bcomp(&FB(na + gl - 1), a), v2 = *bcomp(&FB(na + gl - 2), a);
                                *bcomp(&FB(na + gl), a) = 2 * v1 - v2;
                            }
                        }
                    } else if (type == BC_REFL) {
                        if (side == 0) {
                            for (int gl = 1; gl <= ng; gl++) {
                                vec_t s = vscale(FB(gl - 1), -1);
                                double nrm = *bcomp(&FB(gl), a);
                                FB(-gl) = s;
                                *bcomp(&FB(-gl), a) = nrm;
                            }
                        } else {
                            vec_t s0 = vscale(FB(na - 1), -1);
                            FB(na) = s0;
                            for (int gl = 1; gl <= ng; gl++) {
                                vec_t s = vscale(FB(na - gl - 1), -1);
                                double nrm = *bcomp(&FB(na - gl), a);
                                FB(na + gl) = s;
                                *bcomp(&FB(na + gl), a) = nrm;
                            }
                        }
                    } else if (type == BC_PER) {
                        for (int gl = 1; gl <= ng; gl++) {
                            vec_t s1 = FB(na - gl);
                            FB(-gl) = s1;
                            vec_t s2 = FB(gl - 1);
                            FB(na - 1 + gl) = s2;
                        }
                    } else if (type == BC_FIXED) {
                        if (side == 0) {
                            *bcomp(&FB(0), a) = *bcomp(&st.B, a);
                            for (int gl = 1; gl <= ng; gl++) FB(-gl) = st.B;
                        } else {
                            for (int gl = 0; gl < ng; gl++) FB(na + gl) = st.B;
                        }
                    }
#undef FB
                }
        }
    }
}
#endif

/* BoundaryList::apply: implicit Outflow over uncovered faces, then the list. */
void ora_boundary_apply(ora_grid* G) {
    int unc = XN | XP | YN | YP | ZN | ZP;
    for (int e = 0; e < G->nbc; e++) unc &= ~G->bc[e].faces;
    if (unc) {
        bc_cells(G, BC_OUT, unc, 1, pzero());
#if MHD
        if (G->dim >= 2) bc_faces(G, BC_OUT, unc, 1, pzero());
#endif
    }
    for (int e = 0; e < G->nbc; e++) {
        bc_cells(G, G->bc[e].type, G->bc[e].faces, G->bc[e].corners, G->bc[e].st);
#if MHD
        if (G->dim >= 2) bc_faces(G, G->bc[e].type, G->bc[e].faces, G->bc[e].corners, G->bc[e].st);
#endif
    }
}

/* ------------------------------------------------------------------------- */
/* CFL (Hydro/CFL/CFL.cpp:28-137)                                               */

static double sig_a(prim_t W) {
#if MHD
    return cfast_max(W);
#else
    return cs(W);
#endif
}
static double cfl_speed(prim_t W, double dx, double dy, double dz) {
    double a = sig_a(W), speed = 0;
    if (O.cfl == 0) {
        if (dx > 1e-14) speed = (fabs(W.v.x) + a) / dx;
        if (dy > 1e-14) speed = smax(speed, (fabs(W.v.y) + a) / dy);
        if (dz > 1e-14) speed = smax(speed, (fabs(W.v.z) + a) / dz);
    } else if (O.cfl == 1) {
        if (dx > 1e-14) speed = (fabs(W.v.x) + a) / dx;
        if (dy > 1e-14) speed += (fabs(W.v.y) + a) / dy;
        if (dz > 1e-14) speed += (fabs(W.v.z) + a) / dz;
    } else {
        double p = O.cfl;
        if (dx > 1e-14) speed = pow((fabs(W.v.x) + a) / dx, p);
        if (dy > 1e-14) speed += pow((fabs(W.v.y) + a) / dy, p);
        if (dz > 1e-14) speed += pow((fabs(W.v.z) + a) / dz, p);
        speed = pow(speed, 1.0 / p);
    }
    return speed;
}
int ora_cfl_time(ora_grid* G, double* dt) {
    double m = 0;
    if (G->dim == 1) {
        for (int i = -1; i < G->n[0] + 1; i++) {
            prim_t W = G->w[IX(G->cs, i, 0, 0)];
            m = smax(m, fabs(W.v.x) + sig_a(W));
        }
        if (m <= 0) return 2;
        *dt = O.cfl_coeff * G->d[0] / m;
        return 0;
    }
    int kl = G->dim == 3 ? -1 : 0, kh = G->dim == 3 ? G->n[2] + 1 : 1;
    for (int i = -1; i < G->n[0] + 1; i++)
        for (int j = -1; j < G->n[1] + 1; j++)
            for (int k = kl; k < kh; k++) m = smax(m, cfl_speed(W3(G, i, j, k), G->d[0], G->d[1], G->d[2]));
    if (m <= 0) return 2;
    *dt = O.cfl_coeff / m;
    return 0;
}

/* ------------------------------------------------------------------------- */
/* 1D step (Godunov::sweep + Grid1D::unsplit_step, Splitting.cpp:67-115)        */

static int step1d(ora_grid* G, double dt) {
    const int n = G->n[0], g = G->g;
    const double dt_dx = dt / G->d[0];
    size_t cnt = shape_count(G->cs);
    prim_t* w = (prim_t*)malloc(cnt * sizeof(prim_t));
    memcpy(w, G->w, cnt * sizeof(prim_t));
#define WW(i) w[(i) + g]
    vec_t z = vzero();
    prim_t LR = WW(-g), RL, RR;
    muscl(WW(-g), &RL, WW(-g + 1), &RR, WW(-g + 2), dt_dx, z);
    cons_t fL = rflux_ax(LR, RL, dt_dx, 0), fR;
    for (int i = -g + 1; i < n + g - 1; i++) {
        LR = RR;
        if (i + 2 < n + g) muscl(WW(i), &RL, WW(i + 1), &RR, WW(i + 2), dt_dx, z);
        else RL = WW(i + 1);
        fR = rflux_ax(LR, RL, dt_dx, 0);
        WW(i) = padd(WW(i), cmul(csub(fL, fR), dt_dx));
        fL = fR;
    }
    LR = RR;
    RL = WW(n + g - 1);
    fR = rflux_ax(LR, RL, dt_dx, 0);
    WW(n + g - 2) = padd(WW(n + g - 2), cmul(csub(fL, fR), dt_dx));
    int bad = g_fail;
    for (int i = 0; i < n && !bad; i++)
        if (!pphys(WW(i))) bad = 1;
#undef WW
    if (!bad) memcpy(G->w, w, cnt * sizeof(prim_t));
    free(w);
    return bad;
}

/* ------------------------------------------------------------------------- */
/* 2D unsplit step (Unsplit.cpp:28-111, 210-225, 256-270, 292-342; CTU.cpp:133-278) */

typedef struct { shape_t s; prim_t* a; } parr;
typedef struct { shape_t s; cons_t* a; } carr;
typedef struct { shape_t s; vec_t* a; } varr;
static parr pnew(shape_t s) { parr r = {s, (prim_t*)calloc(shape_count(s), sizeof(prim_t))}; return r; }
static carr cnew(shape_t s) { carr r = {s, (cons_t*)calloc(shape_count(s), sizeof(cons_t))}; return r; }
static varr vnew(shape_t s) { varr r = {s, (vec_t*)calloc(shape_count(s), sizeof(vec_t))}; return r; }
#define A2(A, i, j) (A).a[IX((A).s, i, j, 0)]
#define A3(A, i, j, k) (A).a[IX((A).s, i, j, k)]

/* computeHalfStates_X/Y (Unsplit.cpp:292-342) with copyFaceFields (B_fields.cpp:166-183) */
static void halfstates2d(ora_grid* G, parr L, parr R, int ax, double dt) {
    const int nx = G->n[0], ny = G->n[1], g = G->g;
    const double dt_dx = dt / G->d[0], dt_dy = dt / G->d[1];
    if (ax == 0) {
        for (int i = -g + 1; i < nx + g - 1; i++)
            for (int j = -g; j < ny + g; j++) {
                vec_t dB = vzero();
#if MHD
                dB.x = (B2(G, i + 1, j).x - B2(G, i, j).x) * dt_dx;
                dB.y = (B2(G, i, j + 1).y - B2(G, i, j).y) * dt_dy;
#endif
                muscl(W2(G, i - 1, j), &A2(L, i, j), W2(G, i, j), &A2(R, i, j), W2(G, i + 1, j), dt_dx, dB);
            }
        for (int j = -g; j < ny + g; j++) {
            A2(L, -g, j) = W2(G, -g, j); A2(R, -g, j) = W2(G, -g, j);
            A2(L, nx - 1 + g, j) = W2(G, nx - 1 + g, j); A2(R, nx - 1 + g, j) = W2(G, nx - 1 + g, j);
        }
#if MHD
        for (int i = -g; i < nx + g; i++)
            for (int j = -g; j < ny + g; j++) { A2(L, i, j).B.x = B2(G, i, j).x; A2(R, i, j).B.x = B2(G, i + 1, j).x; }
#endif
    } else {
        for (int i = -g; i < nx + g; i++)
            for (int j = -g + 1; j < ny + g - 1; j++) {
                vec_t dB = vzero();
#if MHD
                dB.y = (B2(G, i + 1, j).x - B2(G, i, j).x) * dt_dx;
                dB.x = (B2(G, i, j + 1).y - B2(G, i, j).y) * dt_dy;
#endif
                prim_t wl = W2(G, i, j - 1), wc = W2(G, i, j), wr = W2(G, i, j + 1);
                pswap(&wl, 1); pswap(&wc, 1); pswap(&wr, 1);
                muscl(wl, &A2(L, i, j), wc, &A2(R, i, j), wr, dt_dy, dB);
                pswap(&A2(L, i, j), 1); pswap(&A2(R, i, j), 1);
            }
        for (int i = -g; i < nx + g; i++) {
            A2(L, i, -g) = W2(G, i, -g); A2(R, i, -g) = W2(G, i, -g);
            A2(L, i, ny - 1 + g) = W2(G, i, ny - 1 + g); A2(R, i, ny - 1 + g) = W2(G, i, ny - 1 + g);
        }
#if MHD
        for (int i = -g; i < nx + g; i++)
            for (int j = -g; j < ny + g; j++) { A2(L, i, j).B.y = B2(G, i, j).y; A2(R, i, j).B.y = B2(G, i, j + 1).y; }
#endif
    }
}
/* computeFlux_X / computeFlux_Y (Unsplit.cpp:210-225) */
static void flux2d(parr L, parr R, carr F, int ax, int x0, int x1, int y0, int y1, double dt) {
    if (ax == 0) {
        for (int i = x0; i <= x1; i++)
            for (int j = y0; j < y1; j++) A2(F, i, j) = rflux_ax(A2(R, i - 1, j), A2(L, i, j), dt, 0);
    } else {
        for (int i = x0; i < x1; i++)
            for (int j = y0; j <= y1; j++) A2(F, i, j) = rflux_ax(A2(R, i, j - 1), A2(L, i, j), dt, 1);
    }
}
/* applyFluxes (Unsplit.cpp:256-270) */
static void apply2d(ora_grid* G, parr wn, carr FX, carr FY, double dt_dx, double dt_dy, int g) {
    const int nx = G->n[0], ny = G->n[1];
    memcpy(wn.a, G->w, shape_count(G->cs) * sizeof(prim_t));
    for (int i = -g; i < nx + g; i++)
        for (int j = -g; j < ny + g; j++) {
            cons_t U = p2c(W2(G, i, j));
            U = cadd(U, cmul(csub(A2(FX, i, j), A2(FX, i + 1, j)), dt_dx));
            U = cadd(U, cmul(csub(A2(FY, i, j), A2(FY, i, j + 1)), dt_dy));
            A2(wn, i, j) = c2p(U);
            if (!cfin(U)) g_fail = 1;
        }
}

#if MHD
static int should_protect(prim_t w);
static void body_fields2d(ora_grid* G, varr Bf, parr wn);
#endif

#if !MHD
/* correctState (CTU.cpp:264-278) */
static void correct2d(parr L, parr R, carr F, double dt_dL, int dim, int nx, int ny) {
    const int isX = dim % 2 == 0, isY = dim % 2 == 1;
    for (int i = -isY; i < nx + isY; i++)
        for (int j = -isX; j < ny + isX; j++) {
            cons_t tr = cmul(csub(A2(F, i + isX, j + isY), A2(F, i, j)), dt_dL);
            A2(L, i, j) = c2p(csub(p2c(A2(L, i, j)), tr));
            A2(R, i, j) = c2p(csub(p2c(A2(R, i, j)), tr));
        }
}
#endif

#if MHD
/* CT::computeElectric 2D (Electric.cpp:24-33) */
static void electric2d(varr E, carr FX, carr FY, int g, int nx, int ny) {
    for (int i = -g; i <= nx + g; i++)
        for (int j = -g; j <= ny + g; j++) {
            A2(E, i, j).x = -A2(FY, i, j).B.z;
            A2(E, i, j).y = A2(FX, i, j).B.z;
            A2(E, i, j).z = (A2(FY, i - 1, j).B.x - A2(FX, i, j - 1).B.y + A2(FY, i, j).B.x - A2(FX, i, j).B.y) * 0.25;
        }
}
/* upwindCorr (Electric.cpp:52-57) */
static double upcorr(double m, double em, double ep, double rm, double rp) {
    if (m > 1e-18) return 0.25 * (em - rm);
    if (m < -1e-18) return 0.25 * (ep - rp);
    return 0.125 * (em + ep - rm - rp);
}
/* CT::upwindElectric 2D (Electric.cpp:59-74) */
static void upwind2d(varr E, carr FX, carr FY, varr Er, int g, int nx, int ny) {
    for (int i = -g; i <= nx + g; i++)
        for (int j = -g; j <= ny + g; j++) {
            vec_t* e = &A2(E, i, j);
            e->z += upcorr(A2(FX, i, j).rho, A2(FY, i - 1, j).B.x, A2(FY, i, j).B.x, A2(Er, i - 1, j).z, A2(Er, i, j).z);
            e->z += upcorr(A2(FX, i, j - 1).rho, A2(FY, i - 1, j).B.x, A2(FY, i, j).B.x, A2(Er, i - 1, j - 1).z,
                           A2(Er, i, j - 1).z);
            e->z += upcorr(A2(FY, i, j).rho, -A2(FX, i, j - 1).B.y, -A2(FX, i, j).B.y, A2(Er, i, j - 1).z, A2(Er, i, j).z);
            e->z += upcorr(A2(FY, i - 1, j).rho, -A2(FX, i, j - 1).B.y, -A2(FX, i, j).B.y, A2(Er, i - 1, j - 1).z,
                           A2(Er, i - 1, j).z);
            e->x += 0.25 * (-2 * A2(FY, i, j).B.z - A2(Er, i, j).x - A2(Er, i, j - 1).x);
            e->y += 0.25 * (2 * A2(FX, i, j).B.z - A2(Er, i, j).y - A2(Er, i - 1, j).y);
        }
}
/* CT::bodyElectric 2D (Electric.cpp:108-115) */
static void bodyE2d(parr w, varr E, int g, int nx, int ny) {
    for (int i = -g - 1; i <= nx + g; i++)
        for (int j = -g - 1; j <= ny + g; j++) A2(E, i, j) = cross(A2(w, i, j).B, A2(w, i, j).v);
}
/* CT::Faraday 2D (B_fields.cpp:21-40) */
static void faraday2d(varr E, varr Bf, double dt_dx, double dt_dy, int g, int nx, int ny) {
    for (int i = -g; i <= nx + g; i++)
        for (int j = -g; j < ny + g; j++) A2(Bf, i, j).x -= (A2(E, i, j + 1).z - A2(E, i, j).z) * dt_dy;
    for (int i = -g; i < nx + g; i++)
        for (int j = -g; j <= ny + g; j++) A2(Bf, i, j).y -= -(A2(E, i + 1, j).z - A2(E, i, j).z) * dt_dx;
    for (int i = -g; i < nx + g; i++)
        for (int j = -g; j < ny + g; j++)
            A2(Bf, i, j).z -= (A2(E, i + 1, j).y - A2(E, i, j).y) * dt_dx - (A2(E, i, j + 1).x - A2(E, i, j).x) * dt_dy;
}
/* CT::shouldProtectThermal (B_fields.cpp:91-114): the compile-time BETA_GATED
 * form, beta = 8 pi p / B^2 */
static int should_protect(prim_t w) {
    switch (O.ct_energy) {
        case 0: return 0;
        case 1: return 1;
        default: {
            double B2 = dot(w.B, w.B);
            if (B2 == 0) return 0;
            double beta = 8 * M_PI * w.p / dot(w.B, w.B);
            return beta <= 0.1;
        }
    }
}
/* CT::computeBodyField(s) 2D (B_fields.cpp:70-79,129-136) */
static void body_fields2d(ora_grid* G, varr Bf, parr wn) {
    const int nx = G->n[0], ny = G->n[1], ng = G->g;
    for (int i = -ng; i < nx + ng; i++)
        for (int j = -ng; j < ny + ng; j++) {
            vec_t b = {(A2(Bf, i, j).x + A2(Bf, i + 1, j).x) * 0.5, (A2(Bf, i, j).y + A2(Bf, i, j + 1).y) * 0.5,
                       A2(Bf, i, j).z};
            if (!should_protect(A2(wn, i, j))) {
                cons_t U = p2c(A2(wn, i, j));
                U.B = b;
                A2(wn, i, j) = c2p(U);
            } else {
                A2(wn, i, j).B = b;
            }
        }
}
#endif

static int step2d(ora_grid* G, double dt) {
    const int nx = G->n[0], ny = G->n[1];
    const double dt_dx = dt / G->d[0], dt_dy = dt / G->d[1];
    shape_t cs = G->cs;
    parr xL = pnew(cs), xR = pnew(cs), yL = pnew(cs), yR = pnew(cs), wn = pnew(cs);
    carr FX = cnew(cs), FY = cnew(cs);
    g_fail = 0;
    halfstates2d(G, xL, xR, 0, dt);
    halfstates2d(G, yL, yR, 1, dt);
#if !MHD
    { /* ctu_sweep_hydro (CTU.cpp:206-218) */
        carr PX = cnew(cs), PY = cnew(cs);
        flux2d(xL, xR, PX, 0, 0, nx, -1, ny + 1, dt_dx);
        flux2d(yL, yR, PY, 1, -1, nx + 1, 0, ny, dt_dy);
        correct2d(xL, xR, PY, 0.5 * dt_dy, 1, nx, ny);
        correct2d(yL, yR, PX, 0.5 * dt_dx, 0, nx, ny);
        free(PX.a); free(PY.a);
    }
    flux2d(xL, xR, FX, 0, 0, nx, 0, ny, dt_dx);
    flux2d(yL, yR, FY, 1, 0, nx, 0, ny, dt_dy);
    apply2d(G, wn, FX, FY, dt_dx, dt_dy, 0);
    varr Bn = {G->fs, NULL};
#else
    varr Ehalf = vnew(G->fs);
    { /* ctu_sweep_MHD 2D (CTU.cpp:133-203) */
        carr PX = cnew(cs), PY = cnew(cs);
        flux2d(xL, xR, PX, 0, -1, nx + 1, -2, ny + 2, dt_dx);
        flux2d(yL, yR, PY, 1, -2, nx + 2, -1, ny + 1, dt_dy);
        varr Bh = vnew(G->fs), E0 = vnew(G->fs);
        electric2d(E0, PX, PY, 1, nx, ny);
        parr wcur = {cs, G->w};
        bodyE2d(wcur, Ehalf, 1, nx, ny);
        upwind2d(E0, PX, PY, Ehalf, 1, nx, ny);
        memcpy(Bh.a, G->B, shape_count(G->fs) * sizeof(vec_t));
        faraday2d(E0, Bh, 0.5 * dt_dx, 0.5 * dt_dy, 1, nx, ny);
        parr wh = pnew(cs);
        apply2d(G, wh, PX, PY, 0.5 * dt_dx, 0.5 * dt_dy, 1);
        body_fields2d(G, Bh, wh);
        bodyE2d(wh, Ehalf, 0, nx, ny);
        free(wh.a);
        for (int i = -1; i < nx + 1; i++)
            for (int j = -1; j < ny + 1; j++) {
                double dBx = (B2(G, i + 1, j).x - B2(G, i, j).x) * dt_dx;
                double dBy = (B2(G, i, j + 1).y - B2(G, i, j).y) * dt_dy;
                prim_t W = W2(G, i, j);
                cons_t corr = cmul(cmul(csub(A2(PY, i, j), A2(PY, i, j + 1)), 0.5), dt_dy);
                corr.B = vzero();
                double lim_z = minmod(-dBy, dBx);
                corr.E += k1_8pi * (W.B.z * W.v.z * lim_z);
                corr.B.z = 0.5 * dt_dy * (A2(E0, i, j + 1).x - A2(E0, i, j).x) + 0.5 * W.v.z * lim_z;
                cons_t uL = cadd(p2c(A2(xL, i, j)), corr), uR = cadd(p2c(A2(xR, i, j)), corr);
                uL.B.x = A2(Bh, i, j).x;
                uR.B.x = A2(Bh, i + 1, j).x;
                A2(xL, i, j) = c2p(uL);
                A2(xR, i, j) = c2p(uR);

                corr = cmul(cmul(csub(A2(PX, i, j), A2(PX, i + 1, j)), 0.5), dt_dx);
                corr.B = vzero();
                lim_z = minmod(-dBx, dBy);
                corr.E += k1_8pi * (W.B.z * W.v.z * lim_z);
                corr.B.z = -0.5 * dt_dx * (A2(E0, i + 1, j).y - A2(E0, i, j).y) + 0.5 * W.v.z * lim_z;
                uL = cadd(p2c(A2(yL, i, j)), corr);
                uR = cadd(p2c(A2(yR, i, j)), corr);
                uL.B.y = A2(Bh, i, j).y;
                uR.B.y = A2(Bh, i, j + 1).y;
                A2(yL, i, j) = c2p(uL);
                A2(yR, i, j) = c2p(uR);
            }
        free(PX.a); free(PY.a); free(Bh.a); free(E0.a);
    }
    flux2d(xL, xR, FX, 0, 0, nx, -1, ny + 1, dt_dx);
    flux2d(yL, yR, FY, 1, -1, nx + 1, 0, ny, dt_dy);
    apply2d(G, wn, FX, FY, dt_dx, dt_dy, 0);
    varr E = vnew(G->fs), Bn = vnew(G->fs);
    electric2d(E, FX, FY, 0, nx, ny);
    upwind2d(E, FX, FY, Ehalf, 0, nx, ny);
    memcpy(Bn.a, G->B, shape_count(G->fs) * sizeof(vec_t));
    faraday2d(E, Bn, dt_dx, dt_dy, 0, nx, ny);
    body_fields2d(G, Bn, wn);
    free(E.a); free(Ehalf.a);
#endif
    int bad = g_fail;
    for (int i = 0; i < nx && !bad; i++)
        for (int j = 0; j < ny && !bad; j++)
            if (!pphys(A2(wn, i, j))) bad = 1;
    if (!bad) {
        for (int i = 0; i < nx; i++)
            for (int j = 0; j < ny; j++) W2(G, i, j) = A2(wn, i, j);
#if MHD
        for (int i = 0; i < nx + 1; i++)
            for (int j = 0; j < ny + 1; j++) B2(G, i, j) = A2(Bn, i, j);
#endif
    }
#if MHD
    free(Bn.a);
#else
    (void)Bn;
#endif
    free(xL.a); free(xR.a); free(yL.a); free(yR.a); free(wn.a); free(FX.a); free(FY.a);
    return bad;
}

/* ------------------------------------------------------------------------- */
/* 3D unsplit step (Unsplit.cpp:115-206, 226-254, 272-288, 344-436; CTU.cpp)   */

static void halfstates3d(ora_grid* G, parr L, parr R, int ax, double dt) {
    const int nx = G->n[0], ny = G->n[1], nz = G->n[2], g = G->g;
    const double dt_dx = dt / G->d[0], dt_dy = dt / G->d[1], dt_dz = dt / G->d[2];
    const double dts[3] = {dt_dx, dt_dy, dt_dz};
    int lo[3] = {-g, -g, -g}, hi[3] = {nx + g, ny + g, nz + g};
    lo[ax] += 1;
    hi[ax] -= 1;
    for (int i = lo[0]; i < hi[0]; i++)
        for (int j = lo[1]; j < hi[1]; j++)
            for (int k = lo[2]; k < hi[2]; k++) {
                vec_t dB = vzero();
#if MHD
                double bx = (B3(G, i + 1, j, k).x - B3(G, i, j, k).x) * dt_dx;
                double by = (B3(G, i, j + 1, k).y - B3(G, i, j, k).y) * dt_dy;
                double bz = (B3(G, i, j, k + 1).z - B3(G, i, j, k).z) * dt_dz;
                if (ax == 0) { dB.x = bx; dB.y = by; dB.z = bz; }
                else if (ax == 1) { dB.y = bx; dB.x = by; dB.z = bz; }
                else { dB.z = bx; dB.y = by; dB.x = bz; }
#endif
                int di = ax == 0, dj = ax == 1, dk = ax == 2;
                prim_t wl = W3(G, i - di, j - dj, k - dk), wc = W3(G, i, j, k), wr = W3(G, i + di, j + dj, k + dk);
                pswap(&wl, ax); pswap(&wc, ax); pswap(&wr, ax);
                muscl(wl, &A3(L, i, j, k), wc, &A3(R, i, j, k), wr, dts[ax], dB);
                pswap(&A3(L, i, j, k), ax); pswap(&A3(R, i, j, k), ax);
            }
    /* leftmost / rightmost ghosts */
    int e0 = -g, e1 = G->n[ax] - 1 + g;
    int l2[3] = {-g, -g, -g}, h2[3] = {nx + g, ny + g, nz + g};
    l2[ax] = 0; h2[ax] = 1;
    for (int i = l2[0]; i < h2[0]; i++)
        for (int j = l2[1]; j < h2[1]; j++)
            for (int k = l2[2]; k < h2[2]; k++) {
                int q[3] = {i, j, k};
                q[ax] = e0;
                A3(L, q[0], q[1], q[2]) = W3(G, q[0], q[1], q[2]);
                A3(R, q[0], q[1], q[2]) = W3(G, q[0], q[1], q[2]);
                q[ax] = e1;
                A3(L, q[0], q[1], q[2]) = W3(G, q[0], q[1], q[2]);
                A3(R, q[0], q[1], q[2]) = W3(G, q[0], q[1], q[2]);
            }
#if MHD
    for (int i = -g; i < nx + g; i++)
        for (int j = -g; j < ny + g; j++)
            for (int k = -g; k < nz + g; k++) {
                if (ax == 0) { A3(L, i, j, k).B.x = B3(G, i, j, k).x; A3(R, i, j, k).B.x = B3(G, i + 1, j, k).x; }
                else if (ax == 1) { A3(L, i, j, k).B.y = B3(G, i, j, k).y; A3(R, i, j, k).B.y = B3(G, i, j + 1, k).y; }
                else { A3(L, i, j, k).B.z = B3(G, i, j, k).z; A3(R, i, j, k).B.z = B3(G, i, j, k + 1).z; }
            }
#endif
}
/* computeFlux_X/Y/Z 3D (Unsplit.cpp:226-254): ranges [lo, hi) with the normal
 * axis inclusive of hi */
static void flux3d(parr L, parr R, carr F, int ax, const int* lo, const int* hi, double dt) {
    int h[3] = {hi[0], hi[1], hi[2]};
    h[ax] += 1;
    for (int i = lo[0]; i < h[0]; i++)
        for (int j = lo[1]; j < h[1]; j++)
            for (int k = lo[2]; k < h[2]; k++) {
                int di = ax == 0, dj = ax == 1, dk = ax == 2;
                A3(F, i, j, k) = rflux_ax(A3(R, i - di, j - dj, k - dk), A3(L, i, j, k), dt, ax);
            }
}
static void apply3d(ora_grid* G, parr wn, carr FX, carr FY, carr FZ, double dx_, double dy_, double dz_, int g) {
    const int nx = G->n[0], ny = G->n[1], nz = G->n[2];
    memcpy(wn.a, G->w, shape_count(G->cs) * sizeof(prim_t));
    for (int i = -g; i < nx + g; i++)
        for (int j = -g; j < ny + g; j++)
            for (int k = -g; k < nz + g; k++) {
                cons_t U = p2c(W3(G, i, j, k));
                U = cadd(U, cmul(csub(A3(FX, i, j, k), A3(FX, i + 1, j, k)), dx_));
                U = cadd(U, cmul(csub(A3(FY, i, j, k), A3(FY, i, j + 1, k)), dy_));
                U = cadd(U, cmul(csub(A3(FZ, i, j, k), A3(FZ, i, j, k + 1)), dz_));
                A3(wn, i, j, k) = c2p(U);
                if (!cfin(U)) g_fail = 1;
            }
}

#if !MHD
/* correctState 3D (CTU.cpp:280-301) */
static void correct3d(parr L, parr R, carr F, double dt_dL, int sd, int fd, const int* n) {
    int isF[3] = {fd == 0, fd == 1, fd == 2}, isS[3] = {sd == 0, sd == 1, sd == 2};
    for (int i = -isS[0]; i < n[0] + isS[0]; i++)
        for (int j = -isS[1]; j < n[1] + isS[1]; j++)
            for (int k = -isS[2]; k < n[2] + isS[2]; k++) {
                cons_t tr = cmul(csub(A3(F, i + isF[0], j + isF[1], k + isF[2]), A3(F, i, j, k)), dt_dL);
                A3(L, i, j, k) = c2p(csub(p2c(A3(L, i, j, k)), tr));
                A3(R, i, j, k) = c2p(csub(p2c(A3(R, i, j, k)), tr));
            }
}
/* computeCTUFlux_X/Y/Z (CTU.cpp:306-370): normal axis ax, transverse flux T
 * along axis td with weight dtT; output F along ax with dt_n. */
static void ctuflux3d(parr L, parr R, carr T, carr F, int ax, int td, double dt_n, double dtT, const int* n) {
    int isT[3] = {td == 0, td == 1, td == 2};
    int lo[3], hi[3];
    for (int a = 0; a < 3; a++) {
        if (a == ax) { lo[a] = 0; hi[a] = n[a]; }
        else { lo[a] = -1 + isT[a]; hi[a] = n[a] + 1 - isT[a]; }
    }
    int o1 = ax == 0 ? 1 : 0, o2 = ax == 2 ? 1 : 2;  /* the two other axes, in loop order */
    for (int a1 = lo[o1]; a1 < hi[o1]; a1++)
        for (int a2 = lo[o2]; a2 < hi[o2]; a2++) {
            int q[3];
            q[o1] = a1; q[o2] = a2; q[ax] = lo[ax] - 1;
            int t[3] = {q[0] + isT[0], q[1] + isT[1], q[2] + isT[2]};
            prim_t __L = c2p(csub(p2c(A3(R, q[0], q[1], q[2])),
                                  cmul(csub(A3(T, t[0], t[1], t[2]), A3(T, q[0], q[1], q[2])), dtT)));
            for (int m = lo[ax]; m <= hi[ax]; m++) {
                q[ax] = m;
                t[0] = q[0] + isT[0]; t[1] = q[1] + isT[1]; t[2] = q[2] + isT[2];
                cons_t tr = cmul(csub(A3(T, t[0], t[1], t[2]), A3(T, q[0], q[1], q[2])), dtT);
                prim_t __R = c2p(csub(p2c(A3(L, q[0], q[1], q[2])), tr));
                A3(F, q[0], q[1], q[2]) = rflux_ax(__L, __R, dt_n, ax);
                __L = c2p(csub(p2c(A3(R, q[0], q[1], q[2])), tr));
            }
        }
}
#endif

#if MHD
/* CT for 3D (Electric.cpp:35-47,76-100,116-125; B_fields.cpp:41-66,80-89,137-149) */
static void electric3d(varr E, carr FX, carr FY, carr FZ, int g, const int* n) {
    for (int i = -g; i <= n[0] + g; i++)
        for (int j = -g; j <= n[1] + g; j++)
            for (int k = -g; k <= n[2] + g; k++) {
                A3(E, i, j, k).x = (A3(FZ, i, j - 1, k).B.y - A3(FY, i, j, k - 1).B.z + A3(FZ, i, j, k).B.y -
                                    A3(FY, i, j, k).B.z) * 0.25;
                A3(E, i, j, k).y = (A3(FX, i, j, k - 1).B.z - A3(FZ, i - 1, j, k).B.x + A3(FX, i, j, k).B.z -
                                    A3(FZ, i, j, k).B.x) * 0.25;
                A3(E, i, j, k).z = (A3(FY, i - 1, j, k).B.x - A3(FX, i, j - 1, k).B.y + A3(FY, i, j, k).B.x -
                                    A3(FX, i, j, k).B.y) * 0.25;
            }
}
static void upwind3d(varr E, carr FX, carr FY, carr FZ, varr Er, int g, const int* n) {
    for (int i = -g; i <= n[0] + g; i++)
        for (int j = -g; j <= n[1] + g; j++)
            for (int k = -g; k <= n[2] + g; k++) {
                vec_t* e = &A3(E, i, j, k);
                e->y += upcorr(A3(FX, i, j, k).rho, -A3(FZ, i - 1, j, k).B.x, -A3(FZ, i, j, k).B.x, A3(Er, i - 1, j, k).y,
                               A3(Er, i, j, k).y);
                e->y += upcorr(A3(FX, i, j, k - 1).rho, -A3(FZ, i - 1, j, k).B.x, -A3(FZ, i, j, k).B.x,
                               A3(Er, i - 1, j, k - 1).y, A3(Er, i, j, k - 1).y);
                e->z += upcorr(A3(FX, i, j, k).rho, A3(FY, i - 1, j, k).B.x, A3(FY, i, j, k).B.x, A3(Er, i - 1, j, k).z,
                               A3(Er, i, j, k).z);
                e->z += upcorr(A3(FX, i, j - 1, k).rho, A3(FY, i - 1, j, k).B.x, A3(FY, i, j, k).B.x,
                               A3(Er, i - 1, j - 1, k).z, A3(Er, i, j - 1, k).z);
                e->x += upcorr(A3(FY, i, j, k).rho, A3(FZ, i, j - 1, k).B.y, A3(FZ, i, j, k).B.y, A3(Er, i, j - 1, k).x,
                               A3(Er, i, j, k).x);
                e->x += upcorr(A3(FY, i, j, k - 1).rho, A3(FZ, i, j - 1, k).B.y, A3(FZ, i, j, k).B.y,
                               A3(Er, i, j - 1, k - 1).x, A3(Er, i, j, k - 1).x);
                e->z += upcorr(A3(FY, i, j, k).rho, -A3(FX, i, j - 1, k).B.y, -A3(FX, i, j, k).B.y, A3(Er, i, j - 1, k).z,
                               A3(Er, i, j, k).z);
                e->z += upcorr(A3(FY, i - 1, j, k).rho, -A3(FX, i, j - 1, k).B.y, -A3(FX, i, j, k).B.y,
                               A3(Er, i - 1, j - 1, k).z, A3(Er, i - 1, j, k).z);
                e->x += upcorr(A3(FZ, i, j, k).rho, -A3(FY, i, j, k - 1).B.z, -A3(FY, i, j, k).B.z, A3(Er, i, j, k - 1).x,
                               A3(Er, i, j, k).x);
                e->x += upcorr(A3(FZ, i, j - 1, k).rho, -A3(FY, i, j, k - 1).B.z, -A3(FY, i, j, k).B.z,
                               A3(Er, i, j - 1, k - 1).x, A3(Er, i, j - 1, k).x);
                e->y += upcorr(A3(FZ, i, j, k).rho, A3(FX, i, j, k - 1).B.z, A3(FX, i, j, k).B.z, A3(Er, i, j, k - 1).y,
                               A3(Er, i, j, k).y);
                e->y += upcorr(A3(FZ, i - 1, j, k).rho, A3(FX, i, j, k - 1).B.z, A3(FX, i, j, k).B.z,
                               A3(Er, i - 1, j, k - 1).y, A3(Er, i - 1, j, k).y);
            }
}
static void bodyE3d(parr w, varr E, int g, const int* n) {
    for (int i = -g - 1; i <= n[0] + g; i++)
        for (int j = -g - 1; j <= n[1] + g; j++)
            for (int k = -g - 1; k <= n[2] + g; k++) A3(E, i, j, k) = cross(A3(w, i, j, k).B, A3(w, i, j, k).v);
}
static void faraday3d(varr E, varr Bf, double dx_, double dy_, double dz_, int g, const int* n) {
    for (int i = -g; i <= n[0] + g; i++)
        for (int j = -g; j < n[1] + g; j++)
            for (int k = -g; k < n[2] + g; k++)
                A3(Bf, i, j, k).x -= (A3(E, i, j + 1, k).z - A3(E, i, j, k).z) * dy_ -
                                     (A3(E, i, j, k + 1).y - A3(E, i, j, k).y) * dz_;
    for (int i = -g; i < n[0] + g; i++)
        for (int j = -g; j <= n[1] + g; j++)
            for (int k = -g; k < n[2] + g; k++)
                A3(Bf, i, j, k).y -= (A3(E, i, j, k + 1).x - A3(E, i, j, k).x) * dz_ -
                                     (A3(E, i + 1, j, k).z - A3(E, i, j, k).z) * dx_;
    for (int i = -g; i < n[0] + g; i++)
        for (int j = -g; j < n[1] + g; j++)
            for (int k = -g; k <= n[2] + g; k++)
                A3(Bf, i, j, k).z -= (A3(E, i + 1, j, k).y - A3(E, i, j, k).y) * dx_ -
                                     (A3(E, i, j + 1, k).x - A3(E, i, j, k).x) * dy_;
}
static void body_fields3d(ora_grid* G, varr Bf, parr wn) {
    const int ng = G->g;
    for (int i = -ng; i < G->n[0] + ng; i++)
        for (int j = -ng; j < G->n[1] + ng; j++)
            for (int k = -ng; k < G->n[2] + ng; k++) {
                vec_t c = A3(Bf, i, j, k);
                vec_t o = {A3(Bf, i + 1, j, k).x, A3(Bf, i, j + 1, k).y, A3(Bf, i, j, k + 1).z};
                vec_t b = vscale(vadd(c, o), 0.5);
                if (!should_protect(A3(wn, i, j, k))) {
                    cons_t U = p2c(A3(wn, i, j, k));
                    U.B = b;
                    A3(wn, i, j, k) = c2p(U);
                } else {
                    A3(wn, i, j, k).B = b;
                }
            }
}
#endif

static int step3d(ora_grid* G, double dt) {
    const int* n = G->n;
    const int nx = n[0], ny = n[1], nz = n[2];
    const double dt_dx = dt / G->d[0], dt_dy = dt / G->d[1], dt_dz = dt / G->d[2];
    shape_t cs = G->cs;
    parr xL = pnew(cs), xR = pnew(cs), yL = pnew(cs), yR = pnew(cs), zL = pnew(cs), zR = pnew(cs), wn = pnew(cs);
    carr FX = cnew(cs), FY = cnew(cs), FZ = cnew(cs);
    g_fail = 0;
    halfstates3d(G, xL, xR, 0, dt);
    halfstates3d(G, yL, yR, 1, dt);
    halfstates3d(G, zL, zR, 2, dt);
#if !MHD
    { /* ctu_sweep_hydro 3D (CTU.cpp:222-261) */
        carr PX = cnew(cs), PY = cnew(cs), PZ = cnew(cs), Q3 = cnew(cs), Q4 = cnew(cs);
        int lx[3] = {0, -1, -1}, hx[3] = {nx, ny + 1, nz + 1};
        int ly[3] = {-1, 0, -1}, hy[3] = {nx + 1, ny, nz + 1};
        int lz[3] = {-1, -1, 0}, hz[3] = {nx + 1, ny + 1, nz};
        flux3d(xL, xR, PX, 0, lx, hx, dt_dx);
        flux3d(yL, yR, PY, 1, ly, hy, dt_dy);
        flux3d(zL, zR, PZ, 2, lz, hz, dt_dz);
        carr FXz = Q3, FYz = Q4;
        ctuflux3d(xL, xR, PZ, FXz, 0, 2, dt_dx, dt_dz / 3.0, n);
        ctuflux3d(yL, yR, PZ, FYz, 1, 2, dt_dy, dt_dz / 3.0, n);
        carr FXy = PZ;  /* PZ is consumed: reused like the reference */
        ctuflux3d(xL, xR, PY, FXy, 0, 1, dt_dx, dt_dy / 3.0, n);
        carr FZy = cnew(cs);
        ctuflux3d(zL, zR, PY, FZy, 2, 1, dt_dz, dt_dy / 3.0, n);
        correct3d(xL, xR, FYz, 0.5 * dt_dy, 0, 1, n);
        correct3d(xL, xR, FZy, 0.5 * dt_dz, 0, 2, n);
        carr FYx = FYz, FZx = FZy;
        ctuflux3d(yL, yR, PX, FYx, 1, 0, dt_dy, dt_dx / 3.0, n);
        ctuflux3d(zL, zR, PX, FZx, 2, 0, dt_dz, dt_dx / 3.0, n);
        correct3d(yL, yR, FXz, 0.5 * dt_dx, 1, 0, n);
        correct3d(yL, yR, FZx, 0.5 * dt_dz, 1, 2, n);
        correct3d(zL, zR, FXy, 0.5 * dt_dx, 2, 0, n);
        correct3d(zL, zR, FYx, 0.5 * dt_dy, 2, 1, n);
        free(PX.a); free(PY.a); free(PZ.a); free(Q3.a); free(Q4.a); free(FZy.a);
    }
    {
        int l[3] = {0, 0, 0}, h[3] = {nx, ny, nz};
        flux3d(xL, xR, FX, 0, l, h, dt_dx);
        flux3d(yL, yR, FY, 1, l, h, dt_dy);
        flux3d(zL, zR, FZ, 2, l, h, dt_dz);
    }
    apply3d(G, wn, FX, FY, FZ, dt_dx, dt_dy, dt_dz, 0);
#else
    varr Ehalf = vnew(G->fs);
    { /* ctu_sweep_MHD 3D (CTU.cpp:34-130) */
        carr PX = cnew(cs), PY = cnew(cs), PZ = cnew(cs);
        /* computeFlux_X/Y/Z ranges of CTU.cpp:42-44 (normal axis inclusive) */
        int lx[3] = {-1, -2, -2}, hx[3] = {nx + 1, ny + 2, nz + 2};
        int ly[3] = {-2, -1, -2}, hy[3] = {nx + 2, ny + 1, nz + 2};
        int lz[3] = {-2, -2, -1}, hz[3] = {nx + 2, ny + 2, nz + 1};
        flux3d(xL, xR, PX, 0, lx, hx, dt_dx);
        flux3d(yL, yR, PY, 1, ly, hy, dt_dy);
        flux3d(zL, zR, PZ, 2, lz, hz, dt_dz);
        varr Bh = vnew(G->fs), E0 = vnew(G->fs);
        electric3d(E0, PX, PY, PZ, 1, n);
        parr wcur = {cs, G->w};
        bodyE3d(wcur, Ehalf, 1, n);
        upwind3d(E0, PX, PY, PZ, Ehalf, 1, n);
        memcpy(Bh.a, G->B, shape_count(G->fs) * sizeof(vec_t));
        faraday3d(E0, Bh, 0.5 * dt_dx, 0.5 * dt_dy, 0.5 * dt_dz, 1, n);
        parr wh = pnew(cs);
        apply3d(G, wh, PX, PY, PZ, 0.5 * dt_dx, 0.5 * dt_dy, 0.5 * dt_dz, 1);
        body_fields3d(G, Bh, wh);
        bodyE3d(wh, Ehalf, 0, n);
        free(wh.a);
        for (int i = -1; i < nx + 1; i++)
            for (int j = -1; j < ny + 1; j++)
                for (int k = -1; k < nz + 1; k++) {
                    double dBx = (B3(G, i + 1, j, k).x - B3(G, i, j, k).x) * dt_dx;
                    double dBy = (B3(G, i, j + 1, k).y - B3(G, i, j, k).y) * dt_dy;
                    double dBz = (B3(G, i, j, k + 1).z - B3(G, i, j, k).z) * dt_dz;
                    prim_t W = W3(G, i, j, k);
                    cons_t corr = cmul(cadd(cmul(csub(A3(PY, i, j, k), A3(PY, i, j + 1, k)), dt_dy),
                                            cmul(csub(A3(PZ, i, j, k), A3(PZ, i, j, k + 1)), dt_dz)), 0.5);
                    corr.B = vzero();
                    double lim_y = minmod(-dBz, dBx), lim_z = minmod(-dBy, dBx);
                    corr.E += k1_8pi * (W.B.y * W.v.y * lim_y + W.B.z * W.v.z * lim_z);
                    corr.B.y = -0.25 * dt_dz *
                                   (A3(E0, i, j, k + 1).x - A3(E0, i, j, k).x + A3(E0, i, j + 1, k + 1).x -
                                    A3(E0, i, j + 1, k).x) + 0.5 * W.v.y * lim_y;
                    corr.B.z = 0.25 * dt_dy *
                                   (A3(E0, i, j + 1, k).x - A3(E0, i, j, k).x + A3(E0, i, j + 1, k + 1).x -
                                    A3(E0, i, j, k + 1).x) + 0.5 * W.v.z * lim_z;
                    cons_t uL = cadd(p2c(A3(xL, i, j, k)), corr), uR = cadd(p2c(A3(xR, i, j, k)), corr);
                    uL.B.x = A3(Bh, i, j, k).x;
                    uR.B.x = A3(Bh, i + 1, j, k).x;
                    A3(xL, i, j, k) = c2p(uL);
                    A3(xR, i, j, k) = c2p(uR);

                    corr = cmul(cadd(cmul(csub(A3(PX, i, j, k), A3(PX, i + 1, j, k)), dt_dx),
                                     cmul(csub(A3(PZ, i, j, k), A3(PZ, i, j, k + 1)), dt_dz)), 0.5);
                    corr.B = vzero();
                    double lim_x = minmod(-dBz, dBy);
                    lim_z = minmod(-dBx, dBy);
                    corr.E += k1_8pi * (W.B.x * W.v.x * lim_x + W.B.z * W.v.z * lim_z);
                    corr.B.x = 0.25 * dt_dz *
                                   (A3(E0, i, j, k + 1).y - A3(E0, i, j, k).y + A3(E0, i + 1, j, k + 1).y -
                                    A3(E0, i + 1, j, k).y) + 0.5 * W.v.x * lim_x;
                    corr.B.z = -0.25 * dt_dx *
                                   (A3(E0, i + 1, j, k).y - A3(E0, i, j, k).y + A3(E0, i + 1, j, k + 1).y -
                                    A3(E0, i, j, k + 1).y) + 0.5 * W.v.z * lim_z;
                    uL = cadd(p2c(A3(yL, i, j, k)), corr);
                    uR = cadd(p2c(A3(yR, i, j, k)), corr);
                    uL.B.y = A3(Bh, i, j, k).y;
                    uR.B.y = A3(Bh, i, j + 1, k).y;
                    A3(yL, i, j, k) = c2p(uL);
                    A3(yR, i, j, k) = c2p(uR);

                    corr = cmul(cadd(cmul(csub(A3(PX, i, j, k), A3(PX, i + 1, j, k)), dt_dx),
                                     cmul(csub(A3(PY, i, j, k), A3(PY, i, j + 1, k)), dt_dy)), 0.5);
                    corr.B = vzero();
                    lim_x = minmod(-dBy, dBz);
                    lim_y = minmod(-dBx, dBz);
                    corr.E += k1_8pi * (W.B.x * W.v.x * lim_x + W.B.y * W.v.y * lim_y);
                    corr.B.x = -0.25 * dt_dy *
                                   (A3(E0, i, j + 1, k).z - A3(E0, i, j, k).z + A3(E0, i + 1, j + 1, k).z -
                                    A3(E0, i + 1, j, k).z) + 0.5 * W.v.x * lim_x;
                    corr.B.y = 0.25 * dt_dx *
                                   (A3(E0, i + 1, j, k).z - A3(E0, i, j, k).z + A3(E0, i + 1, j + 1, k).z -
                                    A3(E0, i, j + 1, k).z) + 0.5 * W.v.y * lim_y;
                    uL = cadd(p2c(A3(zL, i, j, k)), corr);
                    uR = cadd(p2c(A3(zR, i, j, k)), corr);
                    uL.B.z = A3(Bh, i, j, k).z;
                    uR.B.z = A3(Bh, i, j, k + 1).z;
                    A3(zL, i, j, k) = c2p(uL);
                    A3(zR, i, j, k) = c2p(uR);
                }
        free(PX.a); free(PY.a); free(PZ.a); free(Bh.a); free(E0.a);
    }
    {
        flux3d(xL, xR, FX, 0, (int[]){0, -1, -1}, (int[]){nx, ny + 1, nz + 1}, dt_dx);
        flux3d(yL, yR, FY, 1, (int[]){-1, 0, -1}, (int[]){nx + 1, ny, nz + 1}, dt_dy);
        flux3d(zL, zR, FZ, 2, (int[]){-1, -1, 0}, (int[]){nx + 1, ny + 1, nz}, dt_dz);
    }
    apply3d(G, wn, FX, FY, FZ, dt_dx, dt_dy, dt_dz, 0);
    varr E = vnew(G->fs), Bn = vnew(G->fs);
    electric3d(E, FX, FY, FZ, 0, n);
    upwind3d(E, FX, FY, FZ, Ehalf, 0, n);
    memcpy(Bn.a, G->B, shape_count(G->fs) * sizeof(vec_t));
    faraday3d(E, Bn, dt_dx, dt_dy, dt_dz, 0, n);
    body_fields3d(G, Bn, wn);
    free(E.a); free(Ehalf.a);
#endif
    int bad = g_fail;
    for (int i = 0; i < nx && !bad; i++)
        for (int j = 0; j < ny && !bad; j++)
            for (int k = 0; k < nz && !bad; k++)
                if (!pphys(A3(wn, i, j, k))) bad = 1;
    if (!bad) {
        for (int i = 0; i < nx; i++)
            for (int j = 0; j < ny; j++)
                for (int k = 0; k < nz; k++) W3(G, i, j, k) = A3(wn, i, j, k);
#if MHD
        for (int i = 0; i < nx + 1; i++)
            for (int j = 0; j < ny + 1; j++)
                for (int k = 0; k < nz + 1; k++) B3(G, i, j, k) = A3(Bn, i, j, k);
#endif
    }
#if MHD
    free(Bn.a);
#endif
    free(xL.a); free(xR.a); free(yL.a); free(yR.a); free(zL.a); free(zR.a); free(wn.a);
    free(FX.a); free(FY.a); free(FZ.a);
    return bad;
}

/* ------------------------------------------------------------------------- */
/* Grid::unsplit_step / advance_unsplit / initialize_B_fields                  */

int ora_unsplit_step(ora_grid* G, double dt) {
    g_fail = 0;
    if (G->dim == 1) return step1d(G, dt);
    if (G->dim == 2) return step2d(G, dt);
    return step3d(G, dt);
}

/* Grid::advance_unsplit (CFL.cpp:188-213); the reference exits the process
 * where this returns 3. */
int ora_advance(ora_grid* G, double dt, int check_cfl, int* steps, int* retries) {
    int ns = 0, nr = 0;
    while (dt > O.tol) {
        ora_boundary_apply(G);
        double t1 = dt;
        if (check_cfl) {
            double c;
            if (ora_cfl_time(G, &c)) return 2;
            t1 = smin(dt, c);
        }
        for (;;) {
            if (ora_unsplit_step(G, t1) == 0) break;
            nr++;
            t1 *= 0.5;
            if (t1 < O.tol) return 3;
        }
        ns++;
        dt -= t1;
    }
    if (steps) *steps = ns;
    if (retries) *retries = nr;
    return 0;
}

int ora_initialize_B_fields(ora_grid* G) {
#if MHD
    if (G->dim < 2) return 1;
    ora_boundary_apply(G);
    const int ng = G->g;
    if (G->dim == 2) {
        for (int i = -ng; i < G->n[0] + ng; i++)
            for (int j = -ng; j < G->n[1] + ng; j++) {
                vec_t b = {(B2(G, i, j).x + B2(G, i + 1, j).x) * 0.5, (B2(G, i, j).y + B2(G, i, j + 1).y) * 0.5,
                           B2(G, i, j).z};
                W2(G, i, j).B = b;
            }
    } else {
        for (int i = -ng; i < G->n[0] + ng; i++)
            for (int j = -ng; j < G->n[1] + ng; j++)
                for (int k = -ng; k < G->n[2] + ng; k++) {
                    vec_t o = {B3(G, i + 1, j, k).x, B3(G, i, j + 1, k).y, B3(G, i, j, k + 1).z};
                    W3(G, i, j, k).B = vscale(vadd(B3(G, i, j, k), o), 0.5);
                }
    }
    return 0;
#else
    (void)G;
    return 1;
#endif
}

/* ------------------------------------------------------------------------- */
/* Unit-level entry points                                                      */

void ora_muscl(const double* wl, const double* wc, const double* wr, double dt_dL, const double* dB, double* L,
               double* R) {
    prim_t oL, oR;
    vec_t b = {dB[0], dB[1], dB[2]};
    muscl(get_prim(wl), &oL, get_prim(wc), &oR, get_prim(wr), dt_dL, b);
    put_prim(oL, L);
    put_prim(oR, R);
}
static void put_cons(cons_t u, double* a) {
    a[0] = u.rho; a[1] = u.E; a[2] = u.m.x; a[3] = u.m.y; a[4] = u.m.z;
#if MHD
    a[5] = u.B.x; a[6] = u.B.y; a[7] = u.B.z;
#endif
}
int ora_riemann_flux(int solver, const double* l, const double* r, double dt_dx, int axis, double* out) {
    int keep = O.riemann;
    O.riemann = solver;
    g_fail = 0;
    cons_t F = rflux_ax(get_prim(l), get_prim(r), dt_dx, axis);
    O.riemann = keep;
    put_cons(F, out);
    return g_fail;
}
void ora_exact_log_start(double* buf, long cap) {
#if !MHD
    g_log_buf = buf;
    g_log_cap = cap;
    g_log_n = 0;
#else
    (void)buf; (void)cap;
#endif
}
long ora_exact_log_stop(void) {
#if !MHD
    g_log_buf = 0;
    return g_log_n;
#else
    return 0;
#endif
}
void ora_exact_star(const double* l, const double* r, double pGuess, double* sl, double* sr, int* iters) {
#if !MHD
    prim_t L = get_prim(l), R = get_prim(r);
    sol_t s = exact_solve(L, R, pGuess > 0 ? pGuess : (L.p + R.p) / 2.0);
    put_prim(s.sL, sl);
    put_prim(s.sR, sr);
    if (iters) *iters = g_newton_iters;
#else
    (void)l; (void)r; (void)pGuess; (void)sl; (void)sr;
    if (iters) *iters = 0;
#endif
}
