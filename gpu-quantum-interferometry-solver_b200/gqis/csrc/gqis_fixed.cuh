// gqis_fixed.cuh - fixed-step sweep kernels: one parameter point per thread, the reduced
// state in registers, inputs read once, one result (or trace row) written per point.
//
// Step structure and output timing follow the reference integrators (gqis/cuda_solvers.py):
//   RK4 (:470-517): k1 pipelined from the end of the previous step, drives at t+dt/2 and t+dt;
//   explicit RK with a tableau (:48-224, :227-369; dp5, tsit5, anas5, alshina6, dop853):
//       drives at t + c_s dt for every stage, then at t + dt when c_last != 1;
//   LSRK4 2N-storage (:520-607): residual = a_s residual + dt f, y += b_s residual;
//   AB5 (:609-702): four RK4 start steps, then the five-step Adams-Bashforth formula.
// The observable / trace is recorded after every step with the drives at the step end.
#pragma once

#include "gqis_common.cuh"

namespace gqfixed {

// State updates go through F::accumulate(y, c, a, h): a plain FMA in the FP64 form, a
// compensated FP32 update (running correction c, h applied as hi + lo) in the FP32 form.

// ------------------------------------------------------------------- classical RK4
// Functions of time alone at the stage times of steps step .. step + kTimes/2 - 1 (entry 2s: the
// step's midpoint, entry 2s + 1: its end, computed as in RK4::run), entries split over the warp's
// lanes. Not inlined: its FP64 transcendental code would otherwise raise the register count of
// the whole integration loop; it runs once per kTimes/2 steps.
template <class M, int kTimes>
// (dt and t_in are passed by value: a reference to the launch descriptor would force the kernels
// to copy their descriptor parameter to local memory.)
__device__ __noinline__ void fill_time_table(double dt, double t_in, int step, int rank, int nlanes,
                                             const double* Cd, double* tab) {
    const double dt2d = dt * 0.5;
    for (int e = rank; e < kTimes; e += nlanes) {
        double te = ((double)(step + (e >> 1)) + 0.5) * dt;
        if (e & 1) te += dt2d;
        M::time_funcs(t_in + te, Cd, tab + e * M::NTF);
    }
}

struct RK4 {
    template <class M, class F, int OUT, int TRACE>
    __device__ __forceinline__ static void run(const gqis_sweep_desc& d, int64_t local, int64_t p) {
        using R = typename F::real;
        constexpr int S = M::S;
        PointCtx<M, F> pc;
        pc.load(d, p);
        R y[S], c[S], k[S], yt[S], acc[S], Dr[M::NDRV];
        pc.init(d, local, y);
#pragma unroll
        for (int i = 0; i < S; ++i) c[i] = (R)0;
        Recorder<M, F, OUT, TRACE> rec;
        rec.begin(d);

        const double dt = d.dt;
        const double dt2d = dt * 0.5;
        const R h = (R)dt, h2 = (R)dt2d;
        const Coef<R> h6 = Coef<R>::make(dt / 6.0);
        // Functions of time alone (M::NTF of them) are the same for every point: each warp evaluates
        // them for the stage times of kChunk steps at once into shared memory (lanes of the warp past
        // the end of the grid have exited, so the warp synchronises only its remaining lanes).
        // Only for small models (S <= 35, N <= 6): there the drive's transcendental functions are a
        // visible share of a step; larger reduced models spill, and the table-fill call inside the loop
        // costs them more than it saves (measured at N = 8: 148 vs 110 ms in FP64).
        constexpr int kChunk = 16, kTimes = 2 * kChunk;
        constexpr int NTF = (M::S <= 35) ? M::NTF : 0;
        __shared__ double tf_table[NTF > 0 ? GQ_BLOCK / 32 : 1][NTF > 0 ? kTimes * NTF : 1];
        double* const tab = tf_table[NTF > 0 ? (threadIdx.x >> 5) : 0];
        const int lane = threadIdx.x & 31;
        const int64_t valid = d.point_count - (local - lane);  // lanes of this warp inside the grid
        const unsigned warp_mask = valid >= 32 ? 0xffffffffu : ((1u << valid) - 1u);
        const int rank = __popc(warp_mask & ((1u << lane) - 1u)), nlanes = __popc(warp_mask);
        pc.drives(d.t_in + 0.0, Dr);
        pc.rhs(y, Dr, k);
        for (int step = 0; step < d.num_steps; ++step) {
            double t_mid = ((double)step + 0.5) * dt;
            const int slot = step % kChunk;
            if constexpr (NTF > 0) {
                if (slot == 0) {
                    __syncwarp(warp_mask);  // the previous chunk is consumed
                    fill_time_table<M, kTimes>(d.dt, d.t_in, step, rank, nlanes, pc.Cd, tab);
                    __syncwarp(warp_mask);
                }
                pc.drives_tf(d.t_in + t_mid, tab + (2 * slot) * NTF, Dr);
            } else {
                pc.drives(d.t_in + t_mid, Dr);
            }
#pragma unroll
            for (int i = 0; i < S; ++i) {
                yt[i] = fma(h2, k[i], y[i]);
                acc[i] = k[i];
            }
            pc.rhs(yt, Dr, k);
#pragma unroll
            for (int i = 0; i < S; ++i) {
                yt[i] = fma(h2, k[i], y[i]);
                acc[i] = fma((R)2, k[i], acc[i]);
            }
            pc.rhs(yt, Dr, k);
            t_mid += dt2d;
            if constexpr (NTF > 0) {
                pc.drives_tf(d.t_in + t_mid, tab + (2 * slot + 1) * NTF, Dr);
            } else {
                pc.drives(d.t_in + t_mid, Dr);
            }
#pragma unroll
            for (int i = 0; i < S; ++i) {
                yt[i] = fma(h, k[i], y[i]);
                acc[i] = fma((R)2, k[i], acc[i]);
            }
            pc.rhs(yt, Dr, k);
#pragma unroll
            for (int i = 0; i < S; ++i) {
                acc[i] += k[i];
                F::accumulate(y[i], c[i], acc[i], h6);
            }
            if (step + 1 < d.num_steps) pc.rhs(y, Dr, k);
            rec.step(d, pc, local, step, y, Dr);
        }
        rec.finish(d, pc, local, y, Dr);
    }
};

// ------------------------------------------------------ explicit RK from a tableau T
// T provides NS, c(i), a(i, j, w), b(i, w) as constexpr-foldable functions; w is the
// per-launch fitted parameter (solver_params[0]) used by anas5 and ignored by the others.
template <class T>
struct ExplicitRK {
    template <class M, class F, int OUT, int TRACE>
    __device__ __forceinline__ static void run(const gqis_sweep_desc& d, int64_t local, int64_t p) {
        using R = typename F::real;
        constexpr int S = M::S;
        constexpr int NS = T::NS;
        PointCtx<M, F> pc;
        pc.load(d, p);
        R y[S], c[S], yt[S], Dr[M::NDRV];
        R k[NS][S];
        pc.init(d, local, y);
#pragma unroll
        for (int i = 0; i < S; ++i) c[i] = (R)0;
        Recorder<M, F, OUT, TRACE> rec;
        rec.begin(d);

        const double w = d.solver_params[0];
        const double dt = d.dt;
        const R h = (R)dt;
        const Coef<R> hc = Coef<R>::make(dt);
        pc.drives(d.t_in + 0.0, Dr);
        pc.rhs(y, Dr, k[0]);
        for (int step = 0; step < d.num_steps; ++step) {
            const double t0 = (double)step * dt;
#pragma unroll
            for (int s = 1; s < NS; ++s) {
#pragma unroll
                for (int i = 0; i < S; ++i) {
                    R acc = (R)0;
#pragma unroll
                    for (int j = 0; j < s; ++j) {
                        if (T::nonzero_a(s, j)) acc = fma((R)T::a(s, j, w), k[j][i], acc);
                    }
                    yt[i] = fma(h, acc, y[i]);
                }
                if (T::c(s) != T::c(s - 1) || s == 1) pc.drives(d.t_in + fma(T::c(s), dt, t0), Dr);
                pc.rhs(yt, Dr, k[s]);
            }
#pragma unroll
            for (int i = 0; i < S; ++i) {
                R acc = (R)0;
#pragma unroll
                for (int j = 0; j < NS; ++j) {
                    if (T::nonzero_b(j)) acc = fma((R)T::b(j, w), k[j][i], acc);
                }
                F::accumulate(y[i], c[i], acc, hc);
            }
            if (T::c(NS - 1) != 1.0) pc.drives(d.t_in + (t0 + dt), Dr);
            if (step + 1 < d.num_steps) pc.rhs(y, Dr, k[0]);
            rec.step(d, pc, local, step, y, Dr);
        }
        rec.finish(d, pc, local, y, Dr);
    }
};

// ----------------------------------------- Carpenter-Kennedy five-stage 2N-storage RK4
// Coefficients: Carpenter & Kennedy (1994), NASA TM-109112, the (5,4) 2N-storage scheme.
struct LowStorageRK4 {
    __host__ __device__ static constexpr double A(int s) {
        constexpr double v[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                                 -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
        return v[s];
    }
    __host__ __device__ static constexpr double B(int s) {
        constexpr double v[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                                 1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                                 2277821191437.0 / 14882151754819.0};
        return v[s];
    }
    __host__ __device__ static constexpr double C(int s) {
        constexpr double v[5] = {0.0, 1432997174477.0 / 9575080441755.0, 2526269341429.0 / 6820363962896.0,
                                 2006345519317.0 / 3224310063776.0, 2802321613138.0 / 2924317926251.0};
        return v[s];
    }
    template <class M, class F, int OUT, int TRACE>
    __device__ __forceinline__ static void run(const gqis_sweep_desc& d, int64_t local, int64_t p) {
        using R = typename F::real;
        constexpr int S = M::S;
        PointCtx<M, F> pc;
        pc.load(d, p);
        R y[S], c[S], k[S], res[S], Dr[M::NDRV];
        pc.init(d, local, y);
#pragma unroll
        for (int i = 0; i < S; ++i) c[i] = (R)0;
        Recorder<M, F, OUT, TRACE> rec;
        rec.begin(d);
        const double dt = d.dt;
        const R h = (R)dt;
        pc.drives(d.t_in + 0.0, Dr);
        for (int step = 0; step < d.num_steps; ++step) {
            const double t0 = (double)step * dt;
#pragma unroll
            for (int s = 0; s < 5; ++s) {
                if (s > 0) pc.drives(d.t_in + fma(C(s), dt, t0), Dr);
                pc.rhs(y, Dr, k);
                const Coef<R> bs = Coef<R>::make(B(s));
#pragma unroll
                for (int i = 0; i < S; ++i) {
                    res[i] = (s == 0) ? h * k[i] : fma((R)A(s), res[i], h * k[i]);
                    F::accumulate(y[i], c[i], res[i], bs);
                }
            }
            pc.drives(d.t_in + (t0 + dt), Dr);
            rec.step(d, pc, local, step, y, Dr);
        }
        rec.finish(d, pc, local, y, Dr);
    }
};

// ------------------------------------------------ five-step Adams-Bashforth with RK4 start
struct AdamsBashforth5 {
    template <class M, class F, int OUT, int TRACE>
    __device__ __forceinline__ static void run(const gqis_sweep_desc& d, int64_t local, int64_t p) {
        using R = typename F::real;
        constexpr int S = M::S;
        PointCtx<M, F> pc;
        pc.load(d, p);
        // f[0] is the newest derivative f_n, f[4] the oldest f_{n-4}.
        R y[S], c[S], yt[S], acc[S], kt[S], f[5][S], Dr[M::NDRV];
        pc.init(d, local, y);
#pragma unroll
        for (int i = 0; i < S; ++i) c[i] = (R)0;
        Recorder<M, F, OUT, TRACE> rec;
        rec.begin(d);
        const double dt = d.dt;
        const R h = (R)dt, h2 = (R)(dt * 0.5);
        const Coef<R> h6 = Coef<R>::make(dt / 6.0), hc = Coef<R>::make(dt);
        pc.drives(d.t_in + 0.0, Dr);
        pc.rhs(y, Dr, f[0]);
        int step = 0;
        for (; step < d.num_steps && step < 4; ++step) {  // RK4 start steps
            const double t0 = (double)step * dt;
            pc.drives(d.t_in + fma(0.5, dt, t0), Dr);
#pragma unroll
            for (int i = 0; i < S; ++i) {
                yt[i] = fma(h2, f[0][i], y[i]);
                acc[i] = f[0][i];
            }
            pc.rhs(yt, Dr, kt);
#pragma unroll
            for (int i = 0; i < S; ++i) {
                yt[i] = fma(h2, kt[i], y[i]);
                acc[i] = fma((R)2, kt[i], acc[i]);
            }
            pc.rhs(yt, Dr, kt);
#pragma unroll
            for (int i = 0; i < S; ++i) {
                yt[i] = fma(h, kt[i], y[i]);
                acc[i] = fma((R)2, kt[i], acc[i]);
            }
            pc.drives(d.t_in + (t0 + dt), Dr);
            pc.rhs(yt, Dr, kt);
#pragma unroll
            for (int i = 0; i < S; ++i) {
                acc[i] += kt[i];
                F::accumulate(y[i], c[i], acc[i], h6);
            }
#pragma unroll
            for (int j = 4; j > 0; --j)
#pragma unroll
                for (int i = 0; i < S; ++i) f[j][i] = f[j - 1][i];
            if (step + 1 < d.num_steps) pc.rhs(y, Dr, f[0]);
            rec.step(d, pc, local, step, y, Dr);
        }
        const R b0 = (R)(1901.0 / 720.0), b1 = (R)(-1387.0 / 360.0), b2 = (R)(109.0 / 30.0),
                b3 = (R)(-637.0 / 360.0), b4 = (R)(251.0 / 720.0);
        for (; step < d.num_steps; ++step) {
            const double t0 = (double)step * dt;
#pragma unroll
            for (int i = 0; i < S; ++i) {
                R s = (R)0;
                s = fma(b0, f[0][i], s);
                s = fma(b1, f[1][i], s);
                s = fma(b2, f[2][i], s);
                s = fma(b3, f[3][i], s);
                s = fma(b4, f[4][i], s);
                F::accumulate(y[i], c[i], s, hc);
            }
            pc.drives(d.t_in + (t0 + dt), Dr);
#pragma unroll
            for (int j = 4; j > 0; --j)
#pragma unroll
                for (int i = 0; i < S; ++i) f[j][i] = f[j - 1][i];
            if (step + 1 < d.num_steps) pc.rhs(y, Dr, f[0]);
            rec.step(d, pc, local, step, y, Dr);
        }
        rec.finish(d, pc, local, y, Dr);
    }
};

template <class Solver, class M, class F, int OUT, int TRACE>
__global__ void __launch_bounds__(GQ_BLOCK, GQ_MIN_BLOCKS) sweep_fixed_kernel(const gqis_sweep_desc d) {
    const int64_t local = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (local >= d.point_count) return;
    Solver::template run<M, F, OUT, TRACE>(d, local, d.point_begin + local);
}

// A batch: item i covers threads [starts[i], starts[i + 1]), a whole number of warps (threads past
// the item's points return), so each warp integrates points of one item and its time table serves
// them all.
template <class Solver, class M, class F, int OUT, int TRACE>
__global__ void __launch_bounds__(GQ_BLOCK, GQ_MIN_BLOCKS)
    sweep_fixed_batch_kernel(const __grid_constant__ BatchParams b) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= b.starts[b.count]) return;
    const int i = batch_item(b, g);  // the same for the whole warp
    const gqis_sweep_desc& d = b.items[i];
    const int64_t local = g - b.starts[i];
    if (local >= d.point_count) return;
    Solver::template run<M, F, OUT, TRACE>(d, local, d.point_begin + local);
}

}  // namespace gqfixed
