/*
 * dragon_learned.h — learned star-pressure guess for the exact Riemann solver.
 *
 * The reference's exact solver starts its Newton iteration for the star
 * pressure from (pL + pR) / 2 (Hydro/Riemann/Exact.cpp:47) and already takes
 * the guess as a parameter (Riemann::exact(double pGuess),
 * Hydro/Riemann/Riemann.hpp:54). This interface adds, with no counterpart in
 * the reference:
 *   - a per-grid log of converged Newton solves (the training samples),
 *   - a small network trained on the GPU that predicts ln(p_star / p_analytic)
 *     from the face's normalised left/right states,
 *   - the grid option dragon_config.exact_guess = 2, under which the 3D exact
 *     solver starts from the network's guess, keeps the analytic guess as
 *     fallback (unusable output) and judge (cap hit: rerun from it), and still
 *     iterates to ExactRiemann_Tolerance.
 *
 * Network: 6 -> 32 -> 32 -> 1, ReLU, BF16 weights and activations, FP32
 * accumulation; inference is warp-level tensor-core MMA inside the flux
 * kernels. Parameters travel as DRAGON_MLP_PARAMS floats:
 *   [0, 192)     W1 (32 x 6, row-major [out][in])     [192, 224)   b1
 *   [224, 1248)  W2 (32 x 32)                         [1248, 1280) b2
 *   [1280, 1312) W3 (1 x 32)                          1312         b3
 *   [1313, 1319) feature means    [1319, 1325) feature standard deviations
 *   1325 target mean, 1326 target standard deviation, 1327 gate: |ln(p_star / p_a)|
 *   predictions at or below the gate keep the analytic guess unchanged.
 * Features of a face (normal frame): ln(rhoL/rho_m), ln(pL/p_m), (uL-u_m)/c_m,
 * ln(rhoR/rho_m), ln(pR/p_m), (uR-u_m)/c_m with geometric means rho_m, p_m,
 * u_m the mean velocity and c_m = sqrt(gamma p_m / rho_m).
 *
 * All calls return DRAGON_GPU_OK or an error code (dragon_gpu_last_error()).
 */
#ifndef DRAGON_LEARNED_H
#define DRAGON_LEARNED_H

#include "dragon_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

#define DRAGON_MLP_INPUTS 6
#define DRAGON_MLP_HIDDEN 32
#define DRAGON_MLP_WEIGHTS 1313
#define DRAGON_MLP_PARAMS 1328
/* one logged solve: rhoL, vxL, pL, rhoR, vxR, pR, p*, Newton iterations */
#define DRAGON_NEWTON_LOG_COLS 8

/* Exact-solver counters accumulated over every step of a grid. */
typedef struct dragon_newton_stats {
    unsigned long long exact_calls;    /* star-pressure Newton solves */
    unsigned long long newton_iters;   /* Newton iterations (Exact.cpp:71-84) */
    unsigned long long trrs;           /* two-rarefaction closed forms (no Newton) */
    unsigned long long cap_hits;       /* solves stopped by ExactRiemann_MaxIters */
    unsigned long long guess_rejects;  /* learned guess unusable, analytic used */
    unsigned long long judge_reruns;   /* learned start hit the cap, rerun from the analytic guess */
    unsigned long long pivots_exact;   /* verify_and_fallback pivots to the exact solver */
    unsigned long long log_seen;       /* converged solves offered to the log */
    unsigned long long log_stored;     /* rows stored in the log */
} dragon_newton_stats;

int dragon_gpu_newton_stats(dragon_grid* g, dragon_newton_stats* out, int reset);

/* Starts (or restarts, clearing it) the grid's log of converged Newton
 * solves: keeps every stride-th solve up to capacity rows in device memory.
 * capacity 0 stops logging and frees the log. */
int dragon_gpu_newton_log_enable(dragon_grid* g, long long capacity, int stride);
/* Copies up to max_rows stored rows to host memory. */
int dragon_gpu_newton_log_read(dragon_grid* g, double* host_rows, long long max_rows, long long* n_out);
/* Device address of the stored rows (valid until the log is restarted). */
int dragon_gpu_newton_log_device(dragon_grid* g, const double** rows, long long* n_stored);

typedef struct dragon_mlp dragon_mlp;

/* A network with He-uniform weights from seed, zero biases, identity
 * normalisation and gate 0, plus an empty training set, on the current device. */
int dragon_gpu_mlp_create(unsigned long long seed, dragon_mlp** out);
int dragon_gpu_mlp_destroy(dragon_mlp* m);
/* Parameters in the layout above (n = DRAGON_MLP_PARAMS). Loading resets the
 * optimiser state. */
int dragon_gpu_mlp_load(dragon_mlp* m, const float* params, int n);
int dragon_gpu_mlp_save(dragon_mlp* m, float* params, int n);

/* Appends n log rows (device or host memory) to the training set. */
int dragon_gpu_mlp_add_samples(dragon_mlp* m, const double* rows, long long n, int rows_on_device);
long long dragon_gpu_mlp_sample_count(const dragon_mlp* m);
int dragon_gpu_mlp_clear_samples(dragon_mlp* m);
/* Sets feature and target normalisation to the training set's mean / std. */
int dragon_gpu_mlp_fit_normalisation(dragon_mlp* m);
/* Raw features (n x 6) and targets ln(p_star / p_analytic) of samples [first, first+n). */
int dragon_gpu_mlp_features(dragon_mlp* m, long long first, long long n, float* x, float* t);

/* Loss 0.5 mean((y - t_n)^2) over samples [first, first+n) in normalised
 * target units, and its gradient w.r.t. the DRAGON_MLP_WEIGHTS weights
 * (through the BF16 rounding points as identities). No update. */
int dragon_gpu_mlp_gradient(dragon_mlp* m, long long first, long long n, float* grad, float* loss);
/* steps of Adam (beta 0.9 / 0.999) on minibatches of batch samples drawn from
 * the training set with a counter-based hash of (seed, step); loss receives
 * the last minibatch's loss. */
int dragon_gpu_mlp_train(dragon_mlp* m, int steps, int batch, float lr, float* loss);
/* RMS error of the predicted ln(p_star / p_analytic) over samples [first, first+n). */
int dragon_gpu_mlp_evaluate(dragon_mlp* m, long long first, long long n, float* rmse);
int dragon_gpu_mlp_set_gate(dragon_mlp* m, float gate);

/* Tensor-core inference on n faces given as rows rhoL, vxL, pL, rhoR, vxR, pR
 * (host memory): learned guess, analytic guess and raw network output. Any
 * output pointer may be NULL. */
int dragon_gpu_mlp_guess(dragon_mlp* m, const double* pairs, long long n, double* guess, double* analytic,
                         float* y);

/* Copies the network into the grid (used when exact_guess = 2). */
int dragon_gpu_grid_set_mlp(dragon_grid* g, const dragon_mlp* m);

#ifdef __cplusplus
}
#endif

#endif /* DRAGON_LEARNED_H */
