// gqis_adaptive.cuh - adaptive sweep kernels (Tsit5 5(4) and DOP853 8(5,3)) in a persistent,
// work-stealing grid.
//
// Each lane owns one parameter point at a time and advances it by one step attempt per loop
// iteration; a lane whose point is finished takes the next point index from a device counter
// (one warp-aggregated atomicAdd per refill). Lanes of a warp therefore stay busy although
// their points need very different numbers of steps, instead of idling until the slowest point
// of a fixed thread-to-point assignment ends. Every point's arithmetic depends only on its own
// data, so results do not depend on the schedule.
//
// Output semantics follow the reference adaptive solver (gqis/cuda_solvers.py:731-908,
// gqis/solver.py:2154-2174): steps adapt inside each uniform tlist interval and the last step
// of an interval ends on its output time; MEAN is the trapezoid time average over the
// accepted steps after warmup, weighted by step length; traces are taken at interval ends;
// more than max_substeps attempts in one interval makes the point's result NaN. Time, the
// error norm and the step-size controller are FP64 in both forms. After a rejection the FSAL
// derivative of the step start is kept (the reference recomputes the same value).
#pragma once

#include "gqis_common.cuh"

namespace gqadaptive {

// ------------------------------------------------------------------ Tsit5 (FSAL, 7 evals)
// Tableau T: c(i), a(i,j), b(i), e(i) (e = b - b_hat, index 6 weights f(y_new)).
template <class T>
struct Tsit5Pair {
    static constexpr int NS = 6;
    static constexpr double kExponent = -0.2;   // error ~ h^5
    static constexpr double kMinFactor = 0.2, kMaxFactor = 5.0, kSafety = 0.9;
    static constexpr bool kNoGrowthAfterReject = false;

    template <class M, class F>
    __device__ __forceinline__ static double attempt(const PointCtx<M, F>& pc, double t_abs, double hs,
                                                     const typename F::real* y, const typename F::real* k1,
                                                     typename F::real* y_new, typename F::real* k_next,
                                                     typename F::real* Dr, double rtol, double atol) {
        using R = typename F::real;
        constexpr int S = M::S;
        R k[NS][S], yt[S];
        const R h = (R)hs;
#pragma unroll
        for (int i = 0; i < S; ++i) k[0][i] = k1[i];
#pragma unroll
        for (int s = 1; s < NS; ++s) {
#pragma unroll
            for (int i = 0; i < S; ++i) {
                R acc = (R)0;
#pragma unroll
                for (int j = 0; j < s; ++j) acc = fma((R)T::a(s, j), k[j][i], acc);
                yt[i] = fma(h, acc, y[i]);
            }
            pc.drives(t_abs + T::c(s) * hs, Dr);
            pc.rhs(yt, Dr, k[s]);
        }
#pragma unroll
        for (int i = 0; i < S; ++i) {
            R acc = (R)0;
#pragma unroll
            for (int j = 0; j < NS; ++j) acc = fma((R)T::b(j), k[j][i], acc);
            y_new[i] = fma(h, acc, y[i]);
        }
        pc.rhs(y_new, Dr, k_next);  // c6 = 1: the drives are already at t + hs
        double sum = 0.0;
#pragma unroll
        for (int i = 0; i < S; ++i) {
            double e = T::e(6) * (double)k_next[i];
#pragma unroll
            for (int j = 0; j < NS; ++j) e = fma(T::e(j), (double)k[j][i], e);
            e *= hs;
            const double sc = fma(rtol, fmax(fabs((double)y[i]), fabs((double)y_new[i])), atol);
            const double r = e / sc;
            sum = fma(r, r, sum);
        }
        return sqrt(sum / (double)S);
    }
};

// ------------------------------------------------------- DOP853 (12 stages + f(y_new))
// Hairer, Norsett & Wanner, "Solving ODEs I", DOP853: 8th-order main formula, error from the
// 5th- and 3rd-order embedded estimates combined as err5^2 / sqrt(err5^2 + 0.01 err3^2).
// Tableau T: c(i), a(i,j), b(i), e5(i), e3(i) for i < 12.
template <class T>
struct Dop853Pair {
    static constexpr int NS = 12;
    static constexpr double kExponent = -1.0 / 8.0;
    static constexpr double kMinFactor = 0.2, kMaxFactor = 10.0, kSafety = 0.9;
    static constexpr bool kNoGrowthAfterReject = true;

    template <class M, class F>
    __device__ __forceinline__ static double attempt(const PointCtx<M, F>& pc, double t_abs, double hs,
                                                     const typename F::real* y, const typename F::real* k1,
                                                     typename F::real* y_new, typename F::real* k_next,
                                                     typename F::real* Dr, double rtol, double atol) {
        using R = typename F::real;
        constexpr int S = M::S;
        R k[NS][S], yt[S];
        const R h = (R)hs;
#pragma unroll
        for (int i = 0; i < S; ++i) k[0][i] = k1[i];
#pragma unroll
        for (int s = 1; s < NS; ++s) {
#pragma unroll
            for (int i = 0; i < S; ++i) {
                R acc = (R)0;
#pragma unroll
                for (int j = 0; j < s; ++j)
                    if (T::a(s, j) != 0.0) acc = fma((R)T::a(s, j), k[j][i], acc);
                yt[i] = fma(h, acc, y[i]);
            }
            pc.drives(t_abs + T::c(s) * hs, Dr);
            pc.rhs(yt, Dr, k[s]);
        }
        double e5 = 0.0, e3 = 0.0;
#pragma unroll
        for (int i = 0; i < S; ++i) {
            R acc = (R)0;
            double x5 = 0.0, x3 = 0.0;
#pragma unroll
            for (int j = 0; j < NS; ++j) {
                if (T::b(j) != 0.0) acc = fma((R)T::b(j), k[j][i], acc);
                if (T::e5(j) != 0.0) x5 = fma(T::e5(j), (double)k[j][i], x5);
                if (T::e3(j) != 0.0) x3 = fma(T::e3(j), (double)k[j][i], x3);
            }
            y_new[i] = fma(h, acc, y[i]);
            const double sc = fma(rtol, fmax(fabs((double)y[i]), fabs((double)y_new[i])), atol);
            x5 /= sc;
            x3 /= sc;
            e5 = fma(x5, x5, e5);
            e3 = fma(x3, x3, e3);
        }
        if (T::c(NS - 1) != 1.0) pc.drives(t_abs + hs, Dr);
        pc.rhs(y_new, Dr, k_next);
        if (e5 == 0.0 && e3 == 0.0) return 0.0;
        return fabs(hs) * e5 / sqrt((e5 + 0.01 * e3) * (double)S);
    }
};

// -------------------------------------------------------------- per-lane point state
template <class Pair, class M, class F, int OUT, int TRACE>
struct Lane {
    using R = typename F::real;
    static constexpr int S = M::S;
    PointCtx<M, F> pc;
    int64_t local;
    R y[S], k1[S], y_prev[S], Dr[M::NDRV];
    double h, tau;
    int step, substeps, accepted, rejected, next_sample, sample;
    bool rejected_last;
    double re_sum, im_sum;  // trapezoid time average (FP64 in both forms)
    double state_sum[OUT == GQIS_OUT_MEAN_STATE ? S : 1];
    R obs_re_prev, obs_im_prev;

    __device__ __forceinline__ void start(const gqis_sweep_desc& d, int64_t loc) {
        local = loc;
        pc.load(d, d.point_begin + loc);
        pc.init(d, loc, y);
        pc.drives(d.t_in + 0.0, Dr);
        pc.rhs(y, Dr, k1);
        h = d.dt;
        tau = 0.0;
        step = 0;
        substeps = 0;
        accepted = rejected = 0;
        next_sample = d.trace_offset;
        sample = 0;
        rejected_last = false;
        re_sum = 0.0;
        im_sum = 0.0;
        if constexpr (OUT == GQIS_OUT_MEAN_STATE) {
#pragma unroll
            for (int i = 0; i < S; ++i) state_sum[i] = 0.0;
        }
        if constexpr (OUT == GQIS_OUT_MEAN) pc.observe(y, Dr, obs_re_prev, obs_im_prev);
    }

    __device__ __forceinline__ void record_trace(const gqis_sweep_desc& d) {
        if constexpr (TRACE != GQIS_TRACE_NONE) {
            if (step == next_sample) {
                if (sample < d.num_trace) {
                    R* tr = static_cast<R*>(d.trace);
                    if constexpr (TRACE == GQIS_TRACE_OBSERVABLE) {
                        R re, im;
                        pc.observe(y, Dr, re, im);
                        const size_t o = ((size_t)local * d.num_trace + sample) * 2;
                        tr[o] = re;
                        tr[o + 1] = im;
                    } else {
                        const size_t o = ((size_t)local * d.num_trace + sample) * S;
#pragma unroll
                        for (int i = 0; i < S; ++i) tr[o + i] = y[i];
                    }
                }
                ++sample;
                next_sample += d.trace_stride;
            }
        }
    }

    __device__ __forceinline__ void finish(const gqis_sweep_desc& d, bool failed) {
        R* out = static_cast<R*>(d.results);
        const R nan = (R)__longlong_as_double(0x7ff8000000000000LL);
        if constexpr (OUT == GQIS_OUT_MEAN) {
            out[2 * (size_t)local] = failed ? nan : (R)re_sum;
            out[2 * (size_t)local + 1] = failed ? nan : (R)im_sum;
        } else if constexpr (OUT == GQIS_OUT_FINAL) {
            R re, im;
            pc.observe(y, Dr, re, im);
            out[2 * (size_t)local] = failed ? nan : re;
            out[2 * (size_t)local + 1] = failed ? nan : im;
        } else if constexpr (OUT == GQIS_OUT_FINAL_STATE) {
#pragma unroll
            for (int i = 0; i < S; ++i) out[(size_t)local * S + i] = failed ? nan : y[i];
        } else {
#pragma unroll
            for (int i = 0; i < S; ++i) out[(size_t)local * S + i] = failed ? nan : (R)state_sum[i];
        }
        if (d.step_counts) {
            d.step_counts[2 * (size_t)local] = accepted;
            d.step_counts[2 * (size_t)local + 1] = rejected;
        }
    }

    // One step attempt; returns true when the point is finished.
    __device__ __forceinline__ bool advance(const gqis_sweep_desc& d, double rtol, double atol, int max_substeps,
                                            double inv_avg_time) {
        const double dt_out = d.dt;
        const double remaining = dt_out - tau;
        const bool last = h * 1.01 >= remaining;
        const double hs = last ? remaining : h;
        const double t_abs = d.t_in + fma((double)step, dt_out, tau);
        R y_new[S], k_next[S];
        const double err = Pair::template attempt<M, F>(pc, t_abs, hs, y, k1, y_new, k_next, Dr, rtol, atol);
        double factor = Pair::kSafety * pow(err, Pair::kExponent);
        factor = fmin(Pair::kMaxFactor, fmax(Pair::kMinFactor, factor));  // NaN error -> min factor
        bool interval_done = false;
        if (err <= 1.0) {
            ++accepted;
            if (Pair::kNoGrowthAfterReject && rejected_last) factor = fmin(1.0, factor);
            rejected_last = false;
            const double wgt = 0.5 * hs * inv_avg_time;  // trapezoid weight of this step
            if constexpr (OUT == GQIS_OUT_MEAN) {
                R re, im;
                pc.observe(y_new, Dr, re, im);
                if (step >= d.warmup_steps) {
                    re_sum = fma(wgt, (double)re + (double)obs_re_prev, re_sum);
                    im_sum = fma(wgt, (double)im + (double)obs_im_prev, im_sum);
                }
                obs_re_prev = re;
                obs_im_prev = im;
            }
            if constexpr (OUT == GQIS_OUT_MEAN_STATE) {
                if (step >= d.warmup_steps) {
#pragma unroll
                    for (int i = 0; i < S; ++i) state_sum[i] = fma(wgt, (double)y_new[i] + (double)y[i], state_sum[i]);
                }
            }
#pragma unroll
            for (int i = 0; i < S; ++i) {
                y[i] = y_new[i];
                k1[i] = k_next[i];
            }
            tau = last ? dt_out : tau + hs;
            h = last ? fmax(h, hs * factor) : hs * factor;
            interval_done = last;
        } else {
            ++rejected;
            rejected_last = true;
            h = hs * factor;
        }
        if (++substeps > max_substeps) {
            const R nan = (R)__longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
            for (int i = 0; i < S; ++i) y[i] = nan;
            record_trace(d);
            finish(d, true);
            return true;
        }
        if (interval_done) {
            record_trace(d);
            ++step;
            tau = 0.0;
            substeps = 0;
            if (step >= d.num_steps) {
                finish(d, false);
                return true;
            }
        }
        return false;
    }
};

// GQ_STATIC_SCHEDULE=1 builds the classic one-point-per-thread schedule instead (grid = all
// points, no refill), kept for measuring what the work stealing gains.
#ifndef GQ_STATIC_SCHEDULE
#define GQ_STATIC_SCHEDULE 0
#endif

template <class Pair, class M, class F, int OUT, int TRACE>
__global__ void __launch_bounds__(GQ_BLOCK, GQ_MIN_BLOCKS) sweep_adaptive_kernel(const gqis_sweep_desc d) {
    const unsigned lane_id = threadIdx.x & 31u;
    const double rtol = d.solver_params[0], atol = d.solver_params[1];
    const int max_substeps = (int)d.solver_params[2];
    const double inv_avg_time = 1.0 / ((double)(d.num_steps - d.warmup_steps) * d.dt);
    Lane<Pair, M, F, OUT, TRACE> L;
    bool active = false, exhausted = false;
#if GQ_STATIC_SCHEDULE
    {
        const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (idx < d.point_count) {
            L.start(d, idx);
            active = true;
        }
        exhausted = true;
        (void)lane_id;
    }
#endif
    for (;;) {
        const unsigned need = __ballot_sync(0xffffffffu, !active && !exhausted);
        if (need) {
            const int leader = __ffs(need) - 1;
            unsigned base = 0;
            if ((int)lane_id == leader) base = atomicAdd(d.work_counter, (unsigned)__popc(need));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (!active && !exhausted) {
                const unsigned rank = __popc(need & ((1u << lane_id) - 1u));
                const int64_t idx = (int64_t)base + rank;
                if (idx < d.point_count) {
                    L.start(d, idx);
                    active = true;
                } else {
                    exhausted = true;
                }
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        if (active && L.advance(d, rtol, atol, max_substeps, inv_avg_time)) active = false;
    }
}

// A batch: lanes take global point indices from the batch's one counter, so points of every item
// share the persistent grid (a lane that finishes a point of one item may continue with a point of
// another). Each lane keeps its item's descriptor; points are integrated exactly as in a launch of
// their own.
template <class Pair, class M, class F, int OUT, int TRACE>
__global__ void __launch_bounds__(GQ_BLOCK, GQ_MIN_BLOCKS)
    sweep_adaptive_batch_kernel(const __grid_constant__ BatchParams b) {
    // lanes of a warp work on different items: their descriptors are read from shared memory
    __shared__ gqis_sweep_desc items[GQIS_BATCH_MAX];
    {
        const int words = b.count * (int)(sizeof(gqis_sweep_desc) / sizeof(uint32_t));
        const uint32_t* src = reinterpret_cast<const uint32_t*>(b.items);
        uint32_t* dst = reinterpret_cast<uint32_t*>(items);
        for (int w = threadIdx.x; w < words; w += blockDim.x) dst[w] = src[w];
        __syncthreads();
    }
    const unsigned lane_id = threadIdx.x & 31u;
    const int64_t total = b.starts[b.count];
    Lane<Pair, M, F, OUT, TRACE> L;
    const gqis_sweep_desc* dp = items;
    double rtol = 0.0, atol = 0.0, inv_avg_time = 0.0;
    int max_substeps = 0;
    bool active = false, exhausted = false;
    for (;;) {
        const unsigned need = __ballot_sync(0xffffffffu, !active && !exhausted);
        if (need) {
            const int leader = __ffs(need) - 1;
            unsigned base = 0;
            if ((int)lane_id == leader) base = atomicAdd(b.counter, (unsigned)__popc(need));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (!active && !exhausted) {
                const int64_t g = (int64_t)base + __popc(need & ((1u << lane_id) - 1u));
                if (g < total) {
                    const int i = batch_item(b, g);
                    dp = items + i;
                    rtol = dp->solver_params[0];
                    atol = dp->solver_params[1];
                    max_substeps = (int)dp->solver_params[2];
                    inv_avg_time = 1.0 / ((double)(dp->num_steps - dp->warmup_steps) * dp->dt);
                    L.start(*dp, g - b.starts[i]);
                    active = true;
                } else {
                    exhausted = true;
                }
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        if (active && L.advance(*dp, rtol, atol, max_substeps, inv_avg_time)) active = false;
    }
}

}  // namespace gqadaptive
