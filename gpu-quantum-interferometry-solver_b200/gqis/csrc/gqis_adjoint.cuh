// gqis_adjoint.cuh - discrete adjoint of the fixed-step RK4 sweep (FP64), with checkpoints.
//
// For every point the kernel returns J = <O>_avg (the right-endpoint time average of the
// forward sweep, as the mean output) or, with FINAL, J = <O> at the last step (as the final output),
// and dJ/dtheta for the P parameters of the emitted adjoint
// struct A (runtime constants and/or the sweep parameters). The gradient is the exact derivative
// of the discrete RK4 map (reverse-mode linearisation of gqfixed::RK4 with its stage times):
//   1. forward: RK4 from the initial state, storing the state every C steps (checkpoints);
//   2. per segment, last to first: recompute the segment's step-start states from its checkpoint;
//   3. backward through the segment's steps, for step y_n -> y_{n+1} with stages k_1..k_4:
//        kb_1 = h/6 lam, kb_2 = kb_3 = h/3 lam, kb_4 = h/6 lam, lam_n = lam_{n+1}
//        stage s = 4..1 (input u_s, time t_s):  ub = J(u_s, t_s)^T kb_s;
//        theta_b += (dF/dtheta)(u_s, t_s)^T kb_s;  lam_n += ub;  kb_{s-1} += c_s ub
//      (u_2 = y + h/2 k_1, u_3 = y + h/2 k_2, u_4 = y + h k_3) and lam_m += w dO/dy for the
//      averaged states m > warmup (w = 1 / (N - warmup)); with FINAL only lam_N = dO/dy(y_N).
// The forward and the recomputation share rk4_step, so the recomputed states are bit-identical.
// Functions of time alone (the model's and the adjoint struct's time_funcs, e.g. cos(w t)) come from a
// per-warp table of the stage times of kAdjChunk steps, filled by the warp's lanes together, as in
// gqfixed::RK4; the passes refill it as they move forward or backward through the steps.
// Scratch (caller-provided, gqis_adjoint_scratch_bytes): checkpoints and one segment of states
// per point, laid out [slot][component][point] so a warp's accesses coalesce.
#pragma once

#include "gqis_common.cuh"

namespace gqadjoint {

template <class M>
struct Step {
    static constexpr int S = M::S;
    using PC = PointCtx<M, FormFP64>;

    // Stage times of step n (k_1 reuses the drives of the previous step's end, as gqfixed::RK4).
    __device__ __forceinline__ static void times(const gqis_sweep_desc& d, int n, double tk[4]) {
        const double dt = d.dt, h2 = dt * 0.5;
        const double t_mid = ((double)n + 0.5) * dt;
        tk[0] = d.t_in + ((n == 0) ? 0.0 : (((double)(n - 1) + 0.5) * dt + h2));
        tk[1] = d.t_in + t_mid;
        tk[2] = d.t_in + t_mid;
        tk[3] = d.t_in + (t_mid + h2);
    }

    // Drives at time t: from the functions of time Tf (the table) where the model has any.
    __device__ __forceinline__ static void drives(const PC& pc, double t, const double* Tf, double* Dr) {
        if constexpr (M::NTF > 0) {
            pc.drives_tf(t, Tf, Dr);
        } else {
            pc.drives(t, Dr);
        }
    }

    // One RK4 step with the forward kernel's rounding; optionally returns the stage inputs. tf0, tf1,
    // tf3: the model's functions of time at the step's start, midpoint and end.
    __device__ __forceinline__ static void rk4_step(const PC& pc, const gqis_sweep_desc& d, int n, double* y,
                                                    double (*u)[S], const double* tf0, const double* tf1,
                                                    const double* tf3) {
        const double dt = d.dt, h2 = dt * 0.5, h6 = dt / 6.0;
        double tk[4], k[S], yt[S], acc[S], Dr[M::NDRV];
        times(d, n, tk);
        drives(pc, tk[0], tf0, Dr);
        pc.rhs(y, Dr, k);
#pragma unroll
        for (int i = 0; i < S; ++i) {
            if (u) u[0][i] = y[i];
            yt[i] = fma(h2, k[i], y[i]);
            acc[i] = k[i];
            if (u) u[1][i] = yt[i];
        }
        drives(pc, tk[1], tf1, Dr);
        pc.rhs(yt, Dr, k);
#pragma unroll
        for (int i = 0; i < S; ++i) {
            yt[i] = fma(h2, k[i], y[i]);
            acc[i] = fma(2.0, k[i], acc[i]);
            if (u) u[2][i] = yt[i];
        }
        pc.rhs(yt, Dr, k);
        drives(pc, tk[3], tf3, Dr);
#pragma unroll
        for (int i = 0; i < S; ++i) {
            yt[i] = fma(dt, k[i], y[i]);
            acc[i] = fma(2.0, k[i], acc[i]);
            if (u) u[3][i] = yt[i];
        }
        pc.rhs(yt, Dr, k);
#pragma unroll
        for (int i = 0; i < S; ++i) {
            acc[i] += k[i];
            y[i] = fma(h6, acc[i], y[i]);
        }
    }
};

constexpr int kAdjChunk = 16;  // steps per table fill

// Table entries e = 3 i + kind (step nb + i; kind 0: start, 1: midpoint, 2: end) of the functions of
// time, the model's (M::NTF) then the adjoint's (A::NTF), computed by the warp's active lanes. Not
// inlined: its FP64 transcendental code stays out of the integration loops' registers.
template <class M, class A>
__device__ __noinline__ void fill_adjoint_table(const gqis_sweep_desc& d, int nb, int rank, int nlanes,
                                                const double* Cd, const double* Ca, double* tab) {
    constexpr int W = M::NTF + A::NTF;
    for (int e = rank; e < 3 * kAdjChunk; e += nlanes) {
        double tk[4];
        Step<M>::times(d, nb + e / 3, tk);
        const int kind = e % 3;
        const double t = kind == 0 ? tk[0] : (kind == 1 ? tk[1] : tk[3]);
        if constexpr (M::NTF > 0) M::time_funcs(t, Cd, tab + e * W);
        if constexpr (A::NTF > 0) A::time_funcs(t, Ca, tab + e * W + M::NTF);
    }
}

template <class M, class A, int FINAL>
__global__ void __launch_bounds__(GQ_BLOCK) adjoint_rk4_kernel(const gqis_adjoint_desc a) {
    constexpr int S = M::S;
    constexpr int P = A::P;
    using St = Step<M>;
    const gqis_sweep_desc& d = a.sweep;
    const int64_t local = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (local >= d.point_count) return;
    const int64_t npts = d.point_count;
    const int N = d.num_steps, W = d.warmup_steps, CE = a.checkpoint_every;
    const int nck = (N + CE - 1) / CE;
    double* ck = a.scratch;                                   // [nck][S][npts]
    double* seg = a.scratch + (size_t)nck * S * npts;         // [CE][S][npts]

    typename St::PC pc;
    pc.load(d, d.point_begin + local);
    const double X = pc.Xd, Yv = pc.Yd;
    const double* C = a.adjoint_consts;
    const double dt = d.dt;
    const double w = FINAL ? 1.0 : 1.0 / (double)(N - W);

    // per-warp table of the functions of time (lanes of this warp past the grid's end have exited)
    constexpr int TW = M::NTF + A::NTF;
    __shared__ double tf_tab[TW > 0 ? GQ_BLOCK / 32 : 1][TW > 0 ? 3 * kAdjChunk * TW : 1];
    double* const tab = tf_tab[TW > 0 ? (threadIdx.x >> 5) : 0];
    const int lane = threadIdx.x & 31;
    const int64_t valid = npts - (local - lane);
    const unsigned warp_mask = valid >= 32 ? 0xffffffffu : ((1u << valid) - 1u);
    const int rank = __popc(warp_mask & ((1u << lane) - 1u)), nlanes = __popc(warp_mask);
    int cb = -(1 << 30);  // first step of the table's block
    // entry of step n, kind 0 / 1 / 2 (start / midpoint / end); `up`: the pass moves forward in n
    auto tf_at = [&](int n, int kind, bool up) -> const double* {
        if constexpr (TW > 0) {
            if (n < cb || n >= cb + kAdjChunk) {
                const int nb = up ? n : (n >= kAdjChunk - 1 ? n - (kAdjChunk - 1) : 0);
                __syncwarp(warp_mask);  // the previous block is consumed
                fill_adjoint_table<M, A>(d, nb, rank, nlanes, pc.Cd, C, tab);
                __syncwarp(warp_mask);
                cb = nb;
            }
            return tab + (3 * (n - cb) + kind) * TW;
        } else {
            return nullptr;
        }
    };

    // ---- 1. forward with checkpoints
    double y[S];
    pc.init(d, local, y);
    double obs_sum = 0.0, obs_im = 0.0;
    for (int n = 0; n < N; ++n) {
        if (n % CE == 0) {
#pragma unroll
            for (int i = 0; i < S; ++i) ck[((size_t)(n / CE) * S + i) * npts + local] = y[i];
        }
        St::rk4_step(pc, d, n, y, nullptr, tf_at(n, 0, true), tf_at(n, 1, true), tf_at(n, 2, true));
        if (FINAL ? (n == N - 1) : (n >= W)) {
            double tk[4], Dr[M::NDRV], re, im;
            St::times(d, n, tk);
            St::drives(pc, tk[3], tf_at(n, 2, true), Dr);
            pc.observe(y, Dr, re, im);
            obs_sum += re;
            obs_im = im;
        }
    }
    double* res = static_cast<double*>(d.results);
    res[2 * (size_t)local] = FINAL ? obs_sum : obs_sum * w;
    res[2 * (size_t)local + 1] = FINAL ? obs_im : 0.0;
    double ynext[S];  // y_{n+1} while stepping back through step n
#pragma unroll
    for (int i = 0; i < S; ++i) ynext[i] = y[i];

    // ---- 2./3. backward, segment by segment
    double lam[S], tb[P > 0 ? P : 1];
#pragma unroll
    for (int i = 0; i < S; ++i) lam[i] = 0.0;
#pragma unroll
    for (int m = 0; m < P; ++m) tb[m] = 0.0;
    for (int c = nck - 1; c >= 0; --c) {
        const int n0 = c * CE;
        const int n1 = (n0 + CE < N) ? n0 + CE : N;
        if (c + 1 < nck) {
#pragma unroll
            for (int i = 0; i < S; ++i) ynext[i] = ck[((size_t)(c + 1) * S + i) * npts + local];
        }
#pragma unroll
        for (int i = 0; i < S; ++i) y[i] = ck[((size_t)c * S + i) * npts + local];
        for (int n = n0; n < n1; ++n) {
#pragma unroll
            for (int i = 0; i < S; ++i) seg[((size_t)(n - n0) * S + i) * npts + local] = y[i];
            if (n + 1 < n1) St::rk4_step(pc, d, n, y, nullptr, tf_at(n, 0, true), tf_at(n, 1, true), tf_at(n, 2, true));
        }
        for (int n = n1 - 1; n >= n0; --n) {
            double tk[4];
            St::times(d, n, tk);
            const double* tfe = tf_at(n, 2, false);  // this step's end: the model's, then the adjoint's
            const double* tfa[4] = {tf_at(n, 0, false), tf_at(n, 1, false), tf_at(n, 1, false), tfe};
            if (FINAL ? (n == N - 1) : (n >= W)) {  // seed of the output at y_{n+1}
                double Da[A::ND > 0 ? A::ND : 1], g[S];
                A::drives(tk[3], TW > 0 ? tfe + M::NTF : nullptr, X, Yv, C, Da);
                A::dobs(ynext, Da, X, Yv, C, g);
#pragma unroll
                for (int i = 0; i < S; ++i) lam[i] = fma(w, g[i], lam[i]);
            }
#pragma unroll
            for (int i = 0; i < S; ++i) y[i] = seg[((size_t)(n - n0) * S + i) * npts + local];
            double u[4][S];
#pragma unroll
            for (int i = 0; i < S; ++i) ynext[i] = y[i];  // y_n is y_{n+1} of the next iteration
            St::rk4_step(pc, d, n, y, u, tfa[0], tfa[1], tfe);
            const double h2 = dt * 0.5, h6 = dt / 6.0;
            const double cw[4] = {h6, 2.0 * h6, 2.0 * h6, h6};
            const double cs[4] = {0.0, h2, h2, dt};
            double kbs[4][S];
#pragma unroll
            for (int s = 0; s < 4; ++s)
#pragma unroll
                for (int i = 0; i < S; ++i) kbs[s][i] = cw[s] * lam[i];
#pragma unroll
            for (int s = 3; s >= 0; --s) {
                double Da[A::ND > 0 ? A::ND : 1], dDa[A::ND * P > 0 ? A::ND * P : 1], ub[S];
                const double* tfs = TW > 0 ? tfa[s] + M::NTF : nullptr;
                A::drives(tk[s], tfs, X, Yv, C, Da);
                A::ddrives(tk[s], tfs, X, Yv, C, dDa);
                A::jt(u[s], kbs[s], Da, X, Yv, C, ub);
                A::fparam(u[s], kbs[s], Da, dDa, X, Yv, C, tb);
#pragma unroll
                for (int i = 0; i < S; ++i) {
                    lam[i] += ub[i];
                    if (s > 0) kbs[s - 1][i] = fma(cs[s], ub[i], kbs[s - 1][i]);
                }
            }
        }
    }
#pragma unroll
    for (int m = 0; m < P; ++m) a.grad[(size_t)local * P + m] = tb[m];
}

}  // namespace gqadjoint
