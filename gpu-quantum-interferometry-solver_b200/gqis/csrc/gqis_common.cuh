// gqis_common.cuh - precision forms, math wrappers and per-point output recording shared by
// every sweep kernel. sm_100a only; included by the per-model translation unit that the
// Python front end generates (model struct + this template library).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "gqis_b200.h"

#ifndef GQ_BLOCK
#define GQ_BLOCK 128
#endif
#ifndef GQ_MIN_BLOCKS
#define GQ_MIN_BLOCKS 1
#endif
#ifndef GQ_FAST_TRIG
#define GQ_FAST_TRIG 0
#endif

// ---------------------------------------------------------------------------------------
// gq:: math entry points used by the emitted model code. Overloads pick the float or double
// CUDA math function from the argument type, so model text written once serves both forms.
// ---------------------------------------------------------------------------------------
namespace gq {
#define GQ_UNARY(name, fname)                                                        \
    __device__ __forceinline__ float name(float x) { return ::fname(x); }            \
    __device__ __forceinline__ double name(double x) { return ::name(x); }
GQ_UNARY(sqrt, sqrtf)
GQ_UNARY(cbrt, cbrtf)
GQ_UNARY(sin, sinf)
GQ_UNARY(cos, cosf)
GQ_UNARY(tan, tanf)
GQ_UNARY(asin, asinf)
GQ_UNARY(acos, acosf)
GQ_UNARY(atan, atanf)
GQ_UNARY(sinh, sinhf)
GQ_UNARY(cosh, coshf)
GQ_UNARY(tanh, tanhf)
GQ_UNARY(asinh, asinhf)
GQ_UNARY(acosh, acoshf)
GQ_UNARY(atanh, atanhf)
GQ_UNARY(exp, expf)
GQ_UNARY(expm1, expm1f)
GQ_UNARY(log, logf)
GQ_UNARY(log1p, log1pf)
GQ_UNARY(log10, log10f)
GQ_UNARY(log2, log2f)
GQ_UNARY(fabs, fabsf)
GQ_UNARY(floor, floorf)
GQ_UNARY(ceil, ceilf)
GQ_UNARY(erf, erff)
GQ_UNARY(erfc, erfcf)
GQ_UNARY(tgamma, tgammaf)
GQ_UNARY(lgamma, lgammaf)
#undef GQ_UNARY
#define GQ_BINARY(name, fname)                                                              \
    __device__ __forceinline__ float name(float x, float y) { return ::fname(x, y); }       \
    __device__ __forceinline__ double name(double x, double y) { return ::name(x, y); }     \
    __device__ __forceinline__ double name(double x, float y) { return ::name(x, (double)y); } \
    __device__ __forceinline__ double name(float x, double y) { return ::name((double)x, y); }
GQ_BINARY(pow, powf)
GQ_BINARY(atan2, atan2f)
GQ_BINARY(fmax, fmaxf)
GQ_BINARY(fmin, fminf)
GQ_BINARY(hypot, hypotf)
#undef GQ_BINARY
__device__ __forceinline__ float pow(float x, int n) { return ::powf(x, (float)n); }
__device__ __forceinline__ double pow(double x, int n) { return ::pow(x, (double)n); }

// x**n for small integer n as a product chain (exact-order multiplications, no pow()).
template <int n, class T>
__device__ __forceinline__ T ipow(T x) {
    T r = x;
#pragma unroll
    for (int i = 1; i < n; ++i) r = r * x;
    return r;
}
}  // namespace gq

// ---------------------------------------------------------------------------------------
// Phase reduction for the FP32 form: a periodic function of an FP64 phase is evaluated as
// f(r) with r = x - 2*pi*k, k = rint(x / 2pi), using a two-part 2*pi (Cody-Waite reduction);
// r then fits FP32 without losing the phase accuracy that an FP32 t * omega would lose.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ float gq_reduce_2pi(double x) {
    const double k = rint(x * 0.15915494309189533577);   // 1 / (2 pi)
    double r = fma(-k, 6.2831853071795862320, x);        // 2 pi rounded to double
    r = fma(-k, 2.4492935982947064e-16, r);             // 2 pi minus its double rounding
    return (float)r;
}

// A step-size coefficient split into a rounded part and its rounding error, so an FP32 form
// can apply the FP64 value of h/6 (a systematic FP32 rounding of h/6 biases every step).
template <class R>
struct Coef {
    R hi, lo;
    __device__ __forceinline__ static Coef make(double v) {
        Coef c;
        c.hi = (R)v;
        c.lo = (R)(v - (double)c.hi);
        return c;
    }
};

// Plain FP64 form: the parity form. Everything is double; the time average is a plain
// running sum as in the reference kernel (N_Level_Kernel.cu:104, gqis/solver.py:2144-2152).
struct FormFP64 {
    using real = double;
    static constexpr int id = GQIS_FORM_FP64;
    static constexpr bool kCompensated = false;
    __device__ __forceinline__ static double sin(double x) { return ::sin(x); }
    __device__ __forceinline__ static double cos(double x) { return ::cos(x); }
    __device__ __forceinline__ static double tan(double x) { return ::tan(x); }
    // y += h * a (c unused)
    __device__ __forceinline__ static void accumulate(double& y, double& c, double a, Coef<double> h) {
        (void)c;
        y = fma(h.hi, a, y);
    }
    struct Sum {
        double s = 0.0;
        __device__ __forceinline__ void add(double v) { s += v; }
        __device__ __forceinline__ double value() const { return s; }
    };
};

// FP32 form: state, stages and RHS in FP32 with three FP64-grade ingredients:
//  * the state update y += h*a is compensated (Kahan): y carries a running FP32 correction c,
//    and h is applied as hi + lo, so neither the per-step rounding of y nor a rounded h/6
//    accumulates over 10^4 steps (without them the map error is ~1e-6, with them ~1e-7);
//  * time and the drive phase are FP64; the phase is reduced to [-pi, pi] before FP32 sin/cos;
//  * the running time average is a compensated FP32 sum flushed into FP64 every 256 steps.
struct FormFP32 {
    using real = float;
    static constexpr int id = GQIS_FORM_FP32;
    static constexpr bool kCompensated = true;
#if GQ_FAST_TRIG
    // Hardware sin/cos on the reduced phase |r| <= pi: absolute error below 2^-21.4.
    __device__ __forceinline__ static float sin(double x) { return __sinf(gq_reduce_2pi(x)); }
    __device__ __forceinline__ static float cos(double x) { return __cosf(gq_reduce_2pi(x)); }
#else
    __device__ __forceinline__ static float sin(double x) { return ::sinf(gq_reduce_2pi(x)); }
    __device__ __forceinline__ static float cos(double x) { return ::cosf(gq_reduce_2pi(x)); }
#endif
    __device__ __forceinline__ static float tan(double x) { return ::tanf(gq_reduce_2pi(x)); }
    __device__ __forceinline__ static float sin(float x) { return ::sinf(x); }
    __device__ __forceinline__ static float cos(float x) { return ::cosf(x); }
    __device__ __forceinline__ static float tan(float x) { return ::tanf(x); }
    __device__ __forceinline__ static void accumulate(float& y, float& c, float a, Coef<float> h) {
        // Kahan update with h * a - c formed by two FMAs (h to ~FP64 accuracy as hi + lo). Without the
        // compensation the four-level 2048^2 x 8000 map is 10% faster but 2.5e-6 off the FP64 form.
        const float v = fmaf(a, h.hi, fmaf(a, h.lo, -c));
        const float s = y + v;
        c = (s - y) - v;
        y = s;
    }
    struct Sum {
        double total = 0.0;
        float s = 0.0f, c = 0.0f;
        int n = 0;
        __device__ __forceinline__ void add(float v) {
            const float u = v - c;
            const float t = s + u;
            c = (t - s) - u;
            s = t;
            if (++n == 256) {
                total += (double)s - (double)c;
                s = c = 0.0f;
                n = 0;
            }
        }
        __device__ __forceinline__ double value() const { return total + ((double)s - (double)c); }
    };
};

// ---------------------------------------------------------------------------------------
// Batches (gqis_sweep_launch_batch): up to GQIS_BATCH_MAX launches of one module in one grid.
// The descriptors travel as the kernel's parameter (a __grid_constant__ struct of ~13 KB), so a
// batch needs no device scratch and no copy. Item i owns the global work indices
// [starts[i], starts[i + 1]) - threads of the fixed-step kernels (padded to whole warps, so that
// a warp never mixes items), point pairs of the packed kernel (padded likewise), points of the
// persistent adaptive kernels; starts[count] is the total.
// ---------------------------------------------------------------------------------------
struct BatchParams {
    int32_t count;
    uint32_t* counter;  // adaptive kernels: the batch's zeroed work-stealing counter
    int64_t starts[GQIS_BATCH_MAX + 1];
    gqis_sweep_desc items[GQIS_BATCH_MAX];
};

// The item whose range holds global index g (0 <= g < starts[count]): binary search.
__device__ __forceinline__ int batch_item(const BatchParams& b, int64_t g) {
    int lo = 0, hi = b.count;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (b.starts[mid] <= g) lo = mid;
        else hi = mid;
    }
    return lo;
}

// ---------------------------------------------------------------------------------------
// Per-point context: sweep parameters, constants and static terms in FP64 (for drives) and
// in the form's type (for the RHS and the observable).
// ---------------------------------------------------------------------------------------
template <class M, class F>
struct PointCtx {
    using R = typename F::real;
    double Xd, Yd;
    R X, Y;
    double Cd[M::NCONST];
    R Cr[M::NCONST];
    double Sd[M::NSTAT];
    R Sr[M::NSTAT];

    __device__ __forceinline__ void load(const gqis_sweep_desc& d, int64_t p) {
        const int ix = (int)(p / d.num_y);
        const int iy = (int)(p - (int64_t)ix * d.num_y);
        Xd = d.par_x[ix];
        Yd = d.par_y[iy];
        X = (R)Xd;
        Y = (R)Yd;
#pragma unroll
        for (int i = 0; i < M::NCONST; ++i) {
            Cd[i] = d.consts ? __ldg(d.consts + i) : 0.0;
            Cr[i] = (R)Cd[i];
        }
#pragma unroll
        for (int i = 0; i < M::NSTAT; ++i) Sd[i] = 0.0;
        M::statics(Xd, Yd, Sd, Cd);
#pragma unroll
        for (int i = 0; i < M::NSTAT; ++i) Sr[i] = (R)Sd[i];
    }

    __device__ __forceinline__ void drives(double t_abs, R* Dr) const {
        M::template drives<F>(Xd, Yd, t_abs, X, Y, Dr, Sd, Sr, Cd, Cr);
    }

    // drives with the model's functions of time alone (M::time_funcs at t_abs) given in Tf
    __device__ __forceinline__ void drives_tf(double t_abs, const double* Tf, R* Dr) const {
        M::template drives_tf<F>(Xd, Yd, t_abs, X, Y, Dr, Sd, Sr, Cd, Cr, Tf);
    }

    __device__ __forceinline__ void rhs(const R* y, const R* Dr, R* dy) const {
        M::rhs(y, X, Y, Dr, Sr, dy, Cr);
    }

    __device__ __forceinline__ void observe(const R* y, const R* Dr, R& re, R& im) const {
        M::observe(y, X, Y, Dr, Sr, Cr, re, im);
    }

    __device__ __forceinline__ void init(const gqis_sweep_desc& d, int64_t local, R* y) const {
        if constexpr (M::kInitFromArray) {
            const R* src = static_cast<const R*>(d.rho0) + (size_t)local * M::S;
#pragma unroll
            for (int i = 0; i < M::S; ++i) y[i] = src[i];
        } else {
            double y0[M::S];
#pragma unroll
            for (int i = 0; i < M::S; ++i) y0[i] = 0.0;
            M::init(y0, Xd, Yd, Cd);
#pragma unroll
            for (int i = 0; i < M::S; ++i) y[i] = (R)y0[i];
        }
    }
};

// ---------------------------------------------------------------------------------------
// Output recording for fixed-step solvers: called once after every step with the state and
// the drives at the end of the step (gqis/solver.py:2126-2196 semantics).
// ---------------------------------------------------------------------------------------
template <class M, class F, int OUT, int TRACE>
struct Recorder {
    using R = typename F::real;
    typename F::Sum re_sum, im_sum;
    double state_sum[OUT == GQIS_OUT_MEAN_STATE ? M::S : 1];
    int next_sample;
    int sample;

    __device__ __forceinline__ void begin(const gqis_sweep_desc& d) {
        if constexpr (OUT == GQIS_OUT_MEAN_STATE) {
#pragma unroll
            for (int i = 0; i < M::S; ++i) state_sum[i] = 0.0;
        }
        next_sample = d.trace_offset;
        sample = 0;
    }

    __device__ __forceinline__ void step(const gqis_sweep_desc& d, const PointCtx<M, F>& pc, int64_t local,
                                         int step_index, const R* y, const R* Dr) {
        if constexpr (OUT == GQIS_OUT_MEAN) {
            if (step_index >= d.warmup_steps) {
                R re, im;
                pc.observe(y, Dr, re, im);
                re_sum.add(re);
                im_sum.add(im);
            }
        }
        if constexpr (OUT == GQIS_OUT_MEAN_STATE) {
            if (step_index >= d.warmup_steps) {
#pragma unroll
                for (int i = 0; i < M::S; ++i) state_sum[i] += (double)y[i];
            }
        }
        if constexpr (TRACE != GQIS_TRACE_NONE) {
            if (step_index == next_sample) {
                if (sample < d.num_trace) {
                    R* tr = static_cast<R*>(d.trace);
                    if constexpr (TRACE == GQIS_TRACE_OBSERVABLE) {
                        R re, im;
                        pc.observe(y, Dr, re, im);
                        const size_t o = ((size_t)local * d.num_trace + sample) * 2;
                        tr[o] = re;
                        tr[o + 1] = im;
                    } else {
                        const size_t o = ((size_t)local * d.num_trace + sample) * M::S;
#pragma unroll
                        for (int i = 0; i < M::S; ++i) tr[o + i] = y[i];
                    }
                }
                ++sample;
                next_sample += d.trace_stride;
            }
        }
    }

    __device__ __forceinline__ void finish(const gqis_sweep_desc& d, const PointCtx<M, F>& pc, int64_t local,
                                           const R* y, const R* Dr) {
        R* out = static_cast<R*>(d.results);
        if constexpr (OUT == GQIS_OUT_MEAN) {
            const double inv = 1.0 / (double)(d.num_steps - d.warmup_steps);
            out[2 * (size_t)local] = (R)(re_sum.value() * inv);
            out[2 * (size_t)local + 1] = (R)(im_sum.value() * inv);
        } else if constexpr (OUT == GQIS_OUT_FINAL) {
            R re, im;
            pc.observe(y, Dr, re, im);
            out[2 * (size_t)local] = re;
            out[2 * (size_t)local + 1] = im;
        } else if constexpr (OUT == GQIS_OUT_FINAL_STATE) {
#pragma unroll
            for (int i = 0; i < M::S; ++i) out[(size_t)local * M::S + i] = y[i];
        } else {
            const double n = (double)(d.num_steps - d.warmup_steps);
#pragma unroll
            for (int i = 0; i < M::S; ++i) out[(size_t)local * M::S + i] = (R)(state_sum[i] / n);
        }
    }
};
