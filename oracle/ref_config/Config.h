// Switch surface used to compile the DRAGON reference as the parity oracle.
//
// The reference keeps its switches in DRAGON/Config.h as preprocessor
// definitions and constants (DRAGON/Config.h:18-110). This header defines the
// same names, with the values the oracle needs, so that the reference's own
// sources compile unchanged when this directory comes first on the include
// path. Differences from the shipped header, all deliberate:
//   * MHD is chosen by the build (-DORACLE_MHD), giving one hydro and one MHD
//     library, exactly as the reference needs two builds.
//   * The Riemann solver, limiter and CFL variant are CHOOSE_RUNTIME so one
//     library serves every configuration; the reference's runtime globals
//     (DRAGON/Config.h:97-110) are defined below and set through the shim.
//   * The CT energy mode is the shipped compile-time BETA_GATED unless
//     -DORACLE_CT_RUNTIME is given (then it is a runtime global too). The two
//     forms of the beta gate round differently (DRAGON/MHD/B_fields.cpp:96-112),
//     so the compile-time form is the one parity is pinned on.
//   * core_count is a runtime integer (DistGrid.cpp:44,63-64,90-92 only read
//     it), so the CPU baseline can match the host it runs on.
#ifndef DRAGON_ORACLE_CONFIG_H
#define DRAGON_ORACLE_CONFIG_H

#include <string>

#define CHOOSE_RUNTIME -1

namespace CONFIG {

#ifdef ORACLE_MHD
#define MHD
#endif

#define CT_CONSV_TOTAL_E 0
#define CT_CONSV_THERMAL 1
#define CT_CONSV_BETA_GATED 2
constexpr double CT_Energy_Beta = 0.1;
#ifdef ORACLE_CT_RUNTIME
#define CT_ENERGY_CONSV CHOOSE_RUNTIME
#else
#define CT_ENERGY_CONSV CT_CONSV_BETA_GATED
#endif

#define DIMENSION_UNSPLIT
#define CTU

#define RIEMANN_EXACT 0
#define Exact_Rarefactions_Check
constexpr double ExactRiemann_Tolerance = 1E-12;
constexpr int ExactRiemann_MaxIters = 6;
#define RIEMANN_HLL 1
#define RIEMANN_HLLC 2
#define RIEMANN_HLLD 3
#define HLLD_PHYSICAL_SAFETY
#define RIEMANN_HLLE 4
#define RIEMANN_HLLX 5
#define RIEMANN_ROE 6
#define Harten_Hyman
#define RIEMANN_DEFAULT CHOOSE_RUNTIME

#ifndef MHD
#define RIEMANN_VERIFY_FALLBACK
constexpr double Riemann_ExactFallback_Parameter = 1.0;
#endif

constexpr double final_time = 1000.0;
constexpr double dt = 1.0;
constexpr double CFL_coeff = 0.3;
constexpr double Timestep_Tolerance = 1e-14;

#define CFL_ADD 1
#define CFL_MAX 0
#define CFL_CALCULATION CHOOSE_RUNTIME

#define MUSCL_Hancock
#define LIMITER_MINMOD 0
#define LIMITER_MC 1
#define LIMITER_VANLEER 2
#define LIMITER_SUPERBEE 3
#define LIMITER_VANALBADA 4
#define MUSCL_DEFAULT_LIMITER CHOOSE_RUNTIME

inline int core_count = 1;

inline int riemann_choice = RIEMANN_HLLX;
inline int limiter_choice = LIMITER_MC;
inline int cfl_choice = CFL_ADD;
#if CT_ENERGY_CONSV == CHOOSE_RUNTIME
inline int CT_energy_choice = CT_CONSV_BETA_GATED;
#endif
}

#endif
