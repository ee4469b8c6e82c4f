// Strang-split step (Grid2D/3D::split_step, Splitting.cpp:118-217): each
// split step is a sequence of one-dimensional Godunov sweeps
// (Godunov::sweep, Splitting.cpp:67-95) along every grid line of one axis,
// ghost lines included, each preceded by the boundary fill. A sweep kernel
// covers a tile of TL lines x TC cells; the axis along which memory is
// contiguous is the fast index of the tile, so loads coalesce whichever
// axis is swept. Velocities are swapped into the sweep axis on load and back
// on store (swappedXY / swappedXZ). Per line the arithmetic is the 1D sweep's
// (raw outermost ghosts as end states, every cell but the two outermost
// updated, the second zero-flux round trip on cell np-2).
#pragma once

#include "grid.cuh"
#include "recon.cuh"
#include "riemann.cuh"

namespace dgpu {

// CTA-uniform skip once the step failed or the advance is done.
__device__ __forceinline__ bool cta_should_skip_sweep(const StepCtl* ctl, int* s_flag) {
    if (threadIdx.x == 0) *s_flag = *(const volatile int*)&ctl->err | *(const volatile int*)&ctl->done;
    __syncthreads();
    return *s_flag != 0;
}

// Tile shapes on 256 threads: a tile's half states (TL x (TC + 2)) fill one
// round of threads and its faces (TL x (TC + 1)) nearly one, where 8 x 32 and
// 32 x 8 tiles ran both phases in two rounds (272 to 320 items).
template <int DIM, int AX>
struct SweepShape {
    static constexpr bool kPosFast = AX == DIM - 1;  // the swept axis is the contiguous one
    static constexpr int TL = kPosFast ? 8 : 32;     // lines per tile
    static constexpr int TC = kPosFast ? 30 : 6;     // cells per line per tile
    static constexpr size_t kSmem = sizeof(double) * 5 * TL * ((TC + 4) + 2 * (TC + 2) + (TC + 1));
};

// Padded element index of position p on line L of the sweep along AX.
template <int DIM, int AX>
__device__ __forceinline__ long long sweep_elem(const Geo& G, long long L, int p) {
    if constexpr (DIM == 2) {
        const int t = (int)L;  // the other axis
        return AX == 0 ? (long long)p * G.pitch + t : (long long)t * G.pitch + p;
    } else {
        // transverse axes t0 < t1, t1 fastest
        constexpr int T0 = AX == 0 ? 1 : 0, T1 = AX == 2 ? 1 : 2;
        const int e1 = G.ext[T1];
        const int c1 = (int)(L % e1), c0 = (int)(L / e1);
        int q[3];
        q[AX] = p;
        q[T0] = c0;
        q[T1] = c1;
        return (long long)q[0] * G.pitch2 + (long long)q[1] * G.pitch + q[2];
    }
}

template <int SOLVER, int DIM, int AX>
__global__ void __launch_bounds__(256) k_sweep(Geo G, const double* __restrict__ win, double* __restrict__ wout,
                                               StepCtl* ctl, StepArgs sa, double factor) {
    using Sh = SweepShape<DIM, AX>;
    constexpr int TL = Sh::TL, TC = Sh::TC;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sw = reinterpret_cast<double*>(smem_raw);       // [5][TL][TC+4]
    double* sL = sw + 5 * TL * (TC + 4);                    // [5][TL][TC+2]
    double* sR = sL + 5 * TL * (TC + 2);
    double* sF = sR + 5 * TL * (TC + 2);                    // [5][TL][TC+1]
    __shared__ int s_skip;
    if (cta_should_skip_sweep(ctl, &s_skip)) return;

    const int np = G.ext[AX];
    long long nlines = 1;
#pragma unroll
    for (int b = 0; b < DIM; b++)
        if (b != AX) nlines *= G.ext[b];
    const int p0 = blockIdx.x * TC;
    const long long L0 = (long long)blockIdx.y * TL;
    const long long PL = G.plane;
    const double dL = AX == 0 ? sa.dx : AX == 1 ? sa.dy : sa.dz;
    // advanceX(dt / 2) or advanceX(dt): the sweep's dt, then dt / dL (Splitting.cpp:225-236)
    const double dt = (factor == 0.5) ? *(volatile double*)&ctl->t1 / 2 : *(volatile double*)&ctl->t1;
    const double dt_dx = dt / dL;
    const ExactOpts eo = exact_opts(sa);
    FaceStats st{};

    // (line l, local cell c) of item q in a tile W cells wide, contiguous axis fastest
    auto decode = [&](int q, int W, int& l, int& c) {
        if constexpr (Sh::kPosFast) { l = q / W; c = q % W; }
        else { l = q % TL; c = q / TL; }
    };
    auto W_at = [&](int l, int q) {
        Prim<double> r;
        r.rho = sw[(0 * TL + l) * (TC + 4) + q];
        r.p = sw[(1 * TL + l) * (TC + 4) + q];
        r.vx = sw[(2 * TL + l) * (TC + 4) + q];
        r.vy = sw[(3 * TL + l) * (TC + 4) + q];
        r.vz = sw[(4 * TL + l) * (TC + 4) + q];
        r.Bx = r.By = r.Bz = 0;
        return r;
    };
    auto put_hs = [&](double* a, int l, int q, const Prim<double>& r) {
        a[(0 * TL + l) * (TC + 2) + q] = r.rho;
        a[(1 * TL + l) * (TC + 2) + q] = r.p;
        a[(2 * TL + l) * (TC + 2) + q] = r.vx;
        a[(3 * TL + l) * (TC + 2) + q] = r.vy;
        a[(4 * TL + l) * (TC + 2) + q] = r.vz;
    };
    auto get_hs = [&](const double* a, int l, int q) {
        Prim<double> r;
        r.rho = a[(0 * TL + l) * (TC + 2) + q];
        r.p = a[(1 * TL + l) * (TC + 2) + q];
        r.vx = a[(2 * TL + l) * (TC + 2) + q];
        r.vy = a[(3 * TL + l) * (TC + 2) + q];
        r.vz = a[(4 * TL + l) * (TC + 2) + q];
        r.Bx = r.By = r.Bz = 0;
        return r;
    };

    // load cells p in [p0-2, p0+TC+2), velocities in the sweep frame
    for (int q = threadIdx.x; q < TL * (TC + 4); q += blockDim.x) {
        int l, c;
        decode(q, TC + 4, l, c);
        const int p = p0 - 2 + c;
        const long long L = L0 + l;
        if (L < nlines && p >= 0 && p < np) {
            const long long m = sweep_elem<DIM, AX>(G, L, p);
            Prim<double> r = load_prim<false>(win, PL, m);
            swap_axis<AX>(r);
            sw[(0 * TL + l) * (TC + 4) + c] = r.rho;
            sw[(1 * TL + l) * (TC + 4) + c] = r.p;
            sw[(2 * TL + l) * (TC + 4) + c] = r.vx;
            sw[(3 * TL + l) * (TC + 4) + c] = r.vy;
            sw[(4 * TL + l) * (TC + 4) + c] = r.vz;
        }
    }
    __syncthreads();
    // half states of cells p in [p0-1, p0+TC]; local index c = p - p0 + 1
    for (int q = threadIdx.x; q < TL * (TC + 2); q += blockDim.x) {
        int l, c;
        decode(q, TC + 2, l, c);
        const int p = p0 - 1 + c;
        if (L0 + l < nlines && p >= 1 && p <= np - 2) {
            Prim<double> oL, oR;
            muscl<false>(sa.limiter, W_at(l, c), oL, W_at(l, c + 1), oR, W_at(l, c + 2), dt_dx, 0.0, 0.0, 0.0);
            put_hs(sL, l, c, oL);
            put_hs(sR, l, c, oR);
        }
    }
    __syncthreads();
    // faces p in [p0-1, p0+TC-1] between cells p and p+1; local index c = p - p0 + 1
    for (int q = threadIdx.x; q < TL * (TC + 1); q += blockDim.x) {
        int l, c;
        decode(q, TC + 1, l, c);
        const int p = p0 - 1 + c;
        const long long L = L0 + l;
        if (L >= nlines || p < 0 || p > np - 2) continue;
        const Prim<double> Lf = (p == 0) ? W_at(l, c + 1) : get_hs(sR, l, c);
        const Prim<double> Rf = (p + 1 == np - 1) ? W_at(l, c + 2) : get_hs(sL, l, c + 1);
        Cons<double> F;
        if (!face_flux_x<false, SOLVER>(Lf, Rf, dt_dx, eo, F, &st)) record_error(ctl, ST_FINAL_FLUX, sweep_elem<DIM, AX>(G, L, p));
        sF[(0 * TL + l) * (TC + 1) + c] = F.rho;
        sF[(1 * TL + l) * (TC + 1) + c] = F.E;
        sF[(2 * TL + l) * (TC + 1) + c] = F.mx;
        sF[(3 * TL + l) * (TC + 1) + c] = F.my;
        sF[(4 * TL + l) * (TC + 1) + c] = F.mz;
    }
    __syncthreads();
    auto fget = [&](int l, int c) {
        Cons<double> u;
        u.rho = sF[(0 * TL + l) * (TC + 1) + c];
        u.E = sF[(1 * TL + l) * (TC + 1) + c];
        u.mx = sF[(2 * TL + l) * (TC + 1) + c];
        u.my = sF[(3 * TL + l) * (TC + 1) + c];
        u.mz = sF[(4 * TL + l) * (TC + 1) + c];
        u.Bx = u.By = u.Bz = 0;
        return u;
    };
    // update cells p in [p0, p0+TC): w[p] += (F[p-1/2] - F[p+1/2]) dt/dL, written back in the grid frame
    for (int q = threadIdx.x; q < TL * TC; q += blockDim.x) {
        int l, c;
        decode(q, TC, l, c);
        const int p = p0 + c;
        const long long L = L0 + l;
        if (L >= nlines || p >= np) continue;
        Prim<double> nw = W_at(l, c + 2);
        if (p >= 1 && p <= np - 2) {
            const Cons<double> fl = fget(l, c), fr = fget(l, c + 1);
            nw = to_prim<false>(c_add<false>(to_cons<false>(nw), c_mul<false>(c_sub<false>(fl, fr), dt_dx)));
            if (p == np - 2) nw = to_prim<false>(c_add<false>(to_cons<false>(nw), c_mul<false>(c_sub<false>(fr, fr), dt_dx)));
        }
        swap_axis<AX>(nw);
        store_prim<false>(wout, PL, sweep_elem<DIM, AX>(G, L, p), nw);
    }
    if (st.pivot_exact) atomicAdd(&ctl->pivots_exact, (unsigned long long)st.pivot_exact);
    if (st.newton_iters) atomicAdd(&ctl->newton_iters, (unsigned long long)st.newton_iters);
    if (st.exact_calls) atomicAdd(&ctl->exact_calls, (unsigned long long)st.exact_calls);
    if (st.trrs) atomicAdd(&ctl->trrs, (unsigned long long)st.trrs);
    if (st.cap_hits) atomicAdd(&ctl->cap_hits, (unsigned long long)st.cap_hits);
}

template <int SOLVER, int DIM, int AX>
inline int launch_sweep_t(const Geo& G, const double* win, double* wout, StepCtl* ctl, const StepArgs& sa, double factor,
                          cudaStream_t st) {
    using Sh = SweepShape<DIM, AX>;
    long long nlines = 1;
    for (int b = 0; b < DIM; b++)
        if (b != AX) nlines *= G.ext[b];
    const dim3 grid((G.ext[AX] + Sh::TC - 1) / Sh::TC, (unsigned)((nlines + Sh::TL - 1) / Sh::TL));
    if (cudaFuncSetAttribute(k_sweep<SOLVER, DIM, AX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Sh::kSmem) !=
        cudaSuccess)
        return 1;
    k_sweep<SOLVER, DIM, AX><<<grid, 256, Sh::kSmem, st>>>(G, win, wout, ctl, sa, factor);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace dgpu
