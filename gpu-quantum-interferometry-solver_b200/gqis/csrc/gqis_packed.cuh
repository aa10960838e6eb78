// gqis_packed.cuh - the FP32 form with two parameter points per thread in packed FP32 arithmetic.
//
// Blackwell executes one fma/add/mul.rn.f32x2 instruction on a pair of FP32 lanes. A thread that
// integrates two points with the same instruction stream (the points differ only in data) issues
// each FP32 operation once for both, so the issue slots that bound the one-point-per-thread FP32
// sweep are halved while the FMA pipe does the same work. Per point, the arithmetic is the scalar
// FP32 form's: the same RHS terms, stage formulas, compensated state update and compensated time
// average; FP64 time, drives and the per-warp table of time functions are shared code.
//
// The model's RHS/observable templates (gqis_common.cuh, emitted per model) are instantiated with
// R = gq::f32x2. A product a*b is kept unevaluated (gq::m2) until it meets an addition, so
// "x + a*b" becomes one fma.rn.f32x2 as nvcc's contraction makes it one FFMA in the scalar form.
#pragma once

#include "gqis_common.cuh"
#include "gqis_f32x2.cuh"

namespace gq {

struct m2;

// Two FP32 values, one per point of the thread's pair.
struct f32x2 {
    float2 v;
    f32x2() = default;
    __device__ __forceinline__ f32x2(float2 a) : v(a) {}
    __device__ __forceinline__ f32x2(float a, float b) : v(make_float2(a, b)) {}
    __device__ __forceinline__ f32x2(double s) : v(make_float2((float)s, (float)s)) {}
    __device__ __forceinline__ f32x2(float s) : v(make_float2(s, s)) {}
    __device__ __forceinline__ f32x2(int s) : v(make_float2((float)s, (float)s)) {}
    __device__ __forceinline__ f32x2(const m2& p);
    __device__ __forceinline__ f32x2& operator+=(const f32x2& o) {
        v = f2_add(v, o.v);
        return *this;
    }
    __device__ __forceinline__ f32x2& operator-=(const f32x2& o) {
        v = f2_sub(v, o.v);
        return *this;
    }
    __device__ __forceinline__ f32x2& operator*=(const f32x2& o) {
        v = f2_mul(v, o.v);
        return *this;
    }
};

// A pending product a*b.
struct m2 {
    float2 a, b;
};
__device__ __forceinline__ f32x2::f32x2(const m2& p) : v(f2_mul(p.a, p.b)) {}

__device__ __forceinline__ m2 operator*(const f32x2& x, const f32x2& y) { return m2{x.v, y.v}; }
__device__ __forceinline__ m2 operator*(const m2& p, const f32x2& y) { return m2{f2_mul(p.a, p.b), y.v}; }
__device__ __forceinline__ m2 operator*(const f32x2& x, const m2& p) { return m2{x.v, f2_mul(p.a, p.b)}; }
__device__ __forceinline__ m2 operator*(const m2& p, const m2& q) { return m2{f2_mul(p.a, p.b), f2_mul(q.a, q.b)}; }

__device__ __forceinline__ f32x2 operator+(const f32x2& x, const f32x2& y) { return f32x2(f2_add(x.v, y.v)); }
__device__ __forceinline__ f32x2 operator-(const f32x2& x, const f32x2& y) { return f32x2(f2_sub(x.v, y.v)); }
__device__ __forceinline__ f32x2 operator+(const f32x2& x, const m2& p) { return f32x2(f2_fma(p.a, p.b, x.v)); }
__device__ __forceinline__ f32x2 operator+(const m2& p, const f32x2& x) { return f32x2(f2_fma(p.a, p.b, x.v)); }
__device__ __forceinline__ f32x2 operator-(const f32x2& x, const m2& p) { return f32x2(f2_fma(f2_neg(p.a), p.b, x.v)); }
__device__ __forceinline__ f32x2 operator-(const m2& p, const f32x2& x) { return f32x2(f2_fma(p.a, p.b, f2_neg(x.v))); }
__device__ __forceinline__ f32x2 operator+(const m2& p, const m2& q) { return f32x2(f2_fma(q.a, q.b, f2_mul(p.a, p.b))); }
__device__ __forceinline__ f32x2 operator-(const m2& p, const m2& q) {
    return f32x2(f2_fma(f2_neg(q.a), q.b, f2_mul(p.a, p.b)));
}
__device__ __forceinline__ f32x2 operator-(const f32x2& x) { return f32x2(f2_neg(x.v)); }
__device__ __forceinline__ m2 operator-(const m2& p) { return m2{f2_neg(p.a), p.b}; }
__device__ __forceinline__ f32x2 operator/(const f32x2& x, const f32x2& y) {
    return f32x2(x.v.x / y.v.x, x.v.y / y.v.y);
}
__device__ __forceinline__ f32x2 operator/(const m2& p, const f32x2& y) { return f32x2(p) / y; }
__device__ __forceinline__ f32x2 operator/(const f32x2& x, const m2& q) { return x / f32x2(q); }
__device__ __forceinline__ f32x2 operator/(const m2& p, const m2& q) { return f32x2(p) / f32x2(q); }

// Math functions of the model text, lane by lane.
#define GQ_PACKED_UNARY(name, fname) \
    __device__ __forceinline__ f32x2 name(const f32x2& x) { return f32x2(::fname(x.v.x), ::fname(x.v.y)); }
GQ_PACKED_UNARY(sqrt, sqrtf)
GQ_PACKED_UNARY(cbrt, cbrtf)
GQ_PACKED_UNARY(sin, sinf)
GQ_PACKED_UNARY(cos, cosf)
GQ_PACKED_UNARY(tan, tanf)
GQ_PACKED_UNARY(asin, asinf)
GQ_PACKED_UNARY(acos, acosf)
GQ_PACKED_UNARY(atan, atanf)
GQ_PACKED_UNARY(sinh, sinhf)
GQ_PACKED_UNARY(cosh, coshf)
GQ_PACKED_UNARY(tanh, tanhf)
GQ_PACKED_UNARY(asinh, asinhf)
GQ_PACKED_UNARY(acosh, acoshf)
GQ_PACKED_UNARY(atanh, atanhf)
GQ_PACKED_UNARY(exp, expf)
GQ_PACKED_UNARY(expm1, expm1f)
GQ_PACKED_UNARY(log, logf)
GQ_PACKED_UNARY(log1p, log1pf)
GQ_PACKED_UNARY(log10, log10f)
GQ_PACKED_UNARY(log2, log2f)
GQ_PACKED_UNARY(fabs, fabsf)
GQ_PACKED_UNARY(floor, floorf)
GQ_PACKED_UNARY(ceil, ceilf)
GQ_PACKED_UNARY(erf, erff)
GQ_PACKED_UNARY(erfc, erfcf)
GQ_PACKED_UNARY(tgamma, tgammaf)
GQ_PACKED_UNARY(lgamma, lgammaf)
#undef GQ_PACKED_UNARY
__device__ __forceinline__ f32x2 sqrt(const m2& p) { return sqrt(f32x2(p)); }
#define GQ_PACKED_BINARY(name, fname)                                     \
    __device__ __forceinline__ f32x2 name(const f32x2& x, const f32x2& y) { \
        return f32x2(::fname(x.v.x, y.v.x), ::fname(x.v.y, y.v.y));         \
    }
GQ_PACKED_BINARY(pow, powf)
GQ_PACKED_BINARY(atan2, atan2f)
GQ_PACKED_BINARY(fmax, fmaxf)
GQ_PACKED_BINARY(fmin, fminf)
GQ_PACKED_BINARY(hypot, hypotf)
#undef GQ_PACKED_BINARY
__device__ __forceinline__ f32x2 pow(const f32x2& x, int n) { return pow(x, f32x2((float)n)); }

}  // namespace gq

// The FP32 form for a pair of points: same rounding steps per point as FormFP32.
struct FormFP32x2 {
    using real = gq::f32x2;
    using scalar_form = FormFP32;
    static constexpr int id = GQIS_FORM_FP32;

    // Compensated y += h*a per lane with the correction kept negated (cn = -c): gq::f2_kahan.
    __device__ __forceinline__ static void accumulate(gq::f32x2& y, gq::f32x2& cn, const gq::f32x2& a,
                                                      float2 h_hi, float2 h_lo) {
        gq::f2_kahan(y.v, cn.v, a.v, h_hi, h_lo);
    }

    // Compensated running sum per lane, flushed into FP64 every 256 terms (FormFP32::Sum per lane).
    struct Sum {
        double total0 = 0.0, total1 = 0.0;
        float2 s = make_float2(0.0f, 0.0f), cn = make_float2(0.0f, 0.0f);  // cn = -(FormFP32::Sum::c)
        int n = 0;
        __device__ __forceinline__ void add(const gq::f32x2& v) {
            const float2 u = gq::f2_add(v.v, cn);
            const float2 t = gq::f2_add(s, u);
            cn = gq::f2_sub(u, gq::f2_sub(t, s));
            s = t;
            if (++n == 256) {
                total0 += (double)s.x + (double)cn.x;
                total1 += (double)s.y + (double)cn.y;
                s = cn = make_float2(0.0f, 0.0f);
                n = 0;
            }
        }
        __device__ __forceinline__ double value(int lane) const {
            return lane == 0 ? total0 + ((double)s.x + (double)cn.x) : total1 + ((double)s.y + (double)cn.y);
        }
    };
};

namespace gqpacked {

using gq::f32x2;

// Sweep parameters, constants and static terms of a pair of points: FP64 per point (drives), packed
// FP32 for the RHS and observable.
template <class M>
struct PairCtx {
    double Xd[2], Yd[2];
    float Xs[2], Ys[2];
    f32x2 X, Y;
    double Cd[M::NCONST];
    float Cs[M::NCONST];
    f32x2 Cr[M::NCONST];
    double Sd[2][M::NSTAT];
    float Ss[2][M::NSTAT];
    f32x2 Sr[M::NSTAT];

    __device__ __forceinline__ void load(const gqis_sweep_desc& d, const int64_t p[2]) {
#pragma unroll
        for (int i = 0; i < M::NCONST; ++i) {
            Cd[i] = d.consts ? __ldg(d.consts + i) : 0.0;
            Cs[i] = (float)Cd[i];
            Cr[i] = f32x2(Cs[i]);
        }
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            const int ix = (int)(p[l] / d.num_y);
            const int iy = (int)(p[l] - (int64_t)ix * d.num_y);
            Xd[l] = d.par_x[ix];
            Yd[l] = d.par_y[iy];
            Xs[l] = (float)Xd[l];
            Ys[l] = (float)Yd[l];
#pragma unroll
            for (int i = 0; i < M::NSTAT; ++i) Sd[l][i] = 0.0;
            M::statics(Xd[l], Yd[l], Sd[l], Cd);
#pragma unroll
            for (int i = 0; i < M::NSTAT; ++i) Ss[l][i] = (float)Sd[l][i];
        }
        X = f32x2(Xs[0], Xs[1]);
        Y = f32x2(Ys[0], Ys[1]);
#pragma unroll
        for (int i = 0; i < M::NSTAT; ++i) Sr[i] = f32x2(Ss[0][i], Ss[1][i]);
    }

    // Drives of both points at one stage time: FP64 per point, each value rounded to FP32 once.
    __device__ __forceinline__ void drives(double t_abs, f32x2* Dr) const {
        float D0[M::NDRV], D1[M::NDRV];
        M::template drives<FormFP32>(Xd[0], Yd[0], t_abs, Xs[0], Ys[0], D0, Sd[0], Ss[0], Cd, Cs);
        M::template drives<FormFP32>(Xd[1], Yd[1], t_abs, Xs[1], Ys[1], D1, Sd[1], Ss[1], Cd, Cs);
#pragma unroll
        for (int k = 0; k < M::NDRV; ++k) Dr[k] = f32x2(D0[k], D1[k]);
    }

    __device__ __forceinline__ void drives_tf(double t_abs, const double* Tf, f32x2* Dr) const {
        float D0[M::NDRV], D1[M::NDRV];
        M::template drives_tf<FormFP32>(Xd[0], Yd[0], t_abs, Xs[0], Ys[0], D0, Sd[0], Ss[0], Cd, Cs, Tf);
        M::template drives_tf<FormFP32>(Xd[1], Yd[1], t_abs, Xs[1], Ys[1], D1, Sd[1], Ss[1], Cd, Cs, Tf);
#pragma unroll
        for (int k = 0; k < M::NDRV; ++k) Dr[k] = f32x2(D0[k], D1[k]);
    }

    __device__ __forceinline__ void rhs(const f32x2* y, const f32x2* Dr, f32x2* dy) const {
        M::rhs(y, X, Y, Dr, Sr, dy, Cr);
    }

    __device__ __forceinline__ void observe(const f32x2* y, const f32x2* Dr, f32x2& re, f32x2& im) const {
        M::observe(y, X, Y, Dr, Sr, Cr, re, im);
    }

    __device__ __forceinline__ void init(const gqis_sweep_desc& d, const int64_t local[2], f32x2* y) const {
        if constexpr (M::kInitFromArray) {
            const float* src0 = static_cast<const float*>(d.rho0) + (size_t)local[0] * M::S;
            const float* src1 = static_cast<const float*>(d.rho0) + (size_t)local[1] * M::S;
#pragma unroll
            for (int i = 0; i < M::S; ++i) y[i] = f32x2(src0[i], src1[i]);
        } else {
            double y0[M::S], y1[M::S];
#pragma unroll
            for (int i = 0; i < M::S; ++i) y0[i] = y1[i] = 0.0;
            M::init(y0, Xd[0], Yd[0], Cd);
            M::init(y1, Xd[1], Yd[1], Cd);
#pragma unroll
            for (int i = 0; i < M::S; ++i) y[i] = f32x2((float)y0[i], (float)y1[i]);
        }
    }
};

// Output recording for a pair (Recorder of gqis_common.cuh, lane by lane). valid[1] is false for the
// duplicate second point of a grid with an odd number of points: it computes, but writes nothing.
template <class M, int OUT, int TRACE>
struct PairRecorder {
    typename FormFP32x2::Sum re_sum, im_sum;
    double state_sum[OUT == GQIS_OUT_MEAN_STATE ? 2 : 1][OUT == GQIS_OUT_MEAN_STATE ? M::S : 1];
    int next_sample;
    int sample;

    __device__ __forceinline__ void begin(const gqis_sweep_desc& d) {
        if constexpr (OUT == GQIS_OUT_MEAN_STATE) {
#pragma unroll
            for (int i = 0; i < M::S; ++i) state_sum[0][i] = state_sum[1][i] = 0.0;
        }
        next_sample = d.trace_offset;
        sample = 0;
    }

    __device__ __forceinline__ void step(const gqis_sweep_desc& d, const PairCtx<M>& pc, const int64_t local[2],
                                         bool second_valid, int step_index, const f32x2* y, const f32x2* Dr) {
        if constexpr (OUT == GQIS_OUT_MEAN) {
            if (step_index >= d.warmup_steps) {
                f32x2 re, im;
                pc.observe(y, Dr, re, im);
                re_sum.add(re);
                im_sum.add(im);
            }
        }
        if constexpr (OUT == GQIS_OUT_MEAN_STATE) {
            if (step_index >= d.warmup_steps) {
#pragma unroll
                for (int i = 0; i < M::S; ++i) {
                    state_sum[0][i] += (double)y[i].v.x;
                    state_sum[1][i] += (double)y[i].v.y;
                }
            }
        }
        if constexpr (TRACE != GQIS_TRACE_NONE) {
            if (step_index == next_sample) {
                if (sample < d.num_trace) {
                    float* tr = static_cast<float*>(d.trace);
                    if constexpr (TRACE == GQIS_TRACE_OBSERVABLE) {
                        f32x2 re, im;
                        pc.observe(y, Dr, re, im);
                        const size_t o0 = ((size_t)local[0] * d.num_trace + sample) * 2;
                        tr[o0] = re.v.x;
                        tr[o0 + 1] = im.v.x;
                        if (second_valid) {
                            const size_t o1 = ((size_t)local[1] * d.num_trace + sample) * 2;
                            tr[o1] = re.v.y;
                            tr[o1 + 1] = im.v.y;
                        }
                    } else {
                        const size_t o0 = ((size_t)local[0] * d.num_trace + sample) * M::S;
                        const size_t o1 = ((size_t)local[1] * d.num_trace + sample) * M::S;
#pragma unroll
                        for (int i = 0; i < M::S; ++i) tr[o0 + i] = y[i].v.x;
                        if (second_valid) {
#pragma unroll
                            for (int i = 0; i < M::S; ++i) tr[o1 + i] = y[i].v.y;
                        }
                    }
                }
                ++sample;
                next_sample += d.trace_stride;
            }
        }
    }

    __device__ __forceinline__ void finish(const gqis_sweep_desc& d, const PairCtx<M>& pc, const int64_t local[2],
                                           bool second_valid, const f32x2* y, const f32x2* Dr) {
        float* out = static_cast<float*>(d.results);
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            if (l == 1 && !second_valid) break;
            const size_t p = (size_t)local[l];
            if constexpr (OUT == GQIS_OUT_MEAN) {
                const double inv = 1.0 / (double)(d.num_steps - d.warmup_steps);
                out[2 * p] = (float)(re_sum.value(l) * inv);
                out[2 * p + 1] = (float)(im_sum.value(l) * inv);
            } else if constexpr (OUT == GQIS_OUT_FINAL) {
                f32x2 re, im;
                pc.observe(y, Dr, re, im);
                out[2 * p] = l ? re.v.y : re.v.x;
                out[2 * p + 1] = l ? im.v.y : im.v.x;
            } else if constexpr (OUT == GQIS_OUT_FINAL_STATE) {
#pragma unroll
                for (int i = 0; i < M::S; ++i) out[p * M::S + i] = l ? y[i].v.y : y[i].v.x;
            } else {
                const double n = (double)(d.num_steps - d.warmup_steps);
#pragma unroll
                for (int i = 0; i < M::S; ++i) out[p * M::S + i] = (float)(state_sum[l][i] / n);
            }
        }
    }
};

// Classical RK4 (gqfixed::RK4's step structure and time table) on a pair of points.
struct RK4x2 {
    template <class M, int OUT, int TRACE>
    __device__ __forceinline__ static void run(const gqis_sweep_desc& d, int64_t pair, int64_t pair_count) {
        constexpr int S = M::S;
        const int64_t local[2] = {2 * pair, (2 * pair + 1 < d.point_count) ? 2 * pair + 1 : 2 * pair};
        const bool second_valid = 2 * pair + 1 < d.point_count;
        const int64_t p[2] = {d.point_begin + local[0], d.point_begin + local[1]};
        PairCtx<M> pc;
        pc.load(d, p);
        f32x2 y[S], cn[S], k[S], yt[S], acc[S], Dr[M::NDRV];
        pc.init(d, local, y);
#pragma unroll
        for (int i = 0; i < S; ++i) cn[i] = f32x2(0.0f);
        PairRecorder<M, OUT, TRACE> rec;
        rec.begin(d);

        const double dt = d.dt;
        const double dt2d = dt * 0.5;
        const float2 h = make_float2((float)dt, (float)dt), h2 = make_float2((float)dt2d, (float)dt2d);
        const Coef<float> h6 = Coef<float>::make(dt / 6.0);
        const float2 h6hi = make_float2(h6.hi, h6.hi), h6lo = make_float2(h6.lo, h6.lo);
        const float2 two = make_float2(2.0f, 2.0f);
        // functions of time alone: one table per warp for the stage times of kChunk steps
        constexpr int kChunk = 16, kTimes = 2 * kChunk;
        constexpr int NTF = (M::S <= 35) ? M::NTF : 0;
        __shared__ double tf_table[NTF > 0 ? GQ_BLOCK / 32 : 1][NTF > 0 ? kTimes * NTF : 1];
        double* const tab = tf_table[NTF > 0 ? (threadIdx.x >> 5) : 0];
        const int lane = threadIdx.x & 31;
        const int64_t valid = pair_count - (pair - lane);  // lanes of this warp inside the grid
        const unsigned warp_mask = valid >= 32 ? 0xffffffffu : ((1u << valid) - 1u);
        const int rank = __popc(warp_mask & ((1u << lane) - 1u)), nlanes = __popc(warp_mask);
        pc.drives(d.t_in + 0.0, Dr);
        pc.rhs(y, Dr, k);
        for (int step = 0; step < d.num_steps; ++step) {
            double t_mid = ((double)step + 0.5) * dt;
            const int slot = step % kChunk;
            if constexpr (NTF > 0) {
                if (slot == 0) {
                    __syncwarp(warp_mask);
                    gqfixed::fill_time_table<M, kTimes>(d.dt, d.t_in, step, rank, nlanes, pc.Cd, tab);
                    __syncwarp(warp_mask);
                }
                pc.drives_tf(d.t_in + t_mid, tab + (2 * slot) * NTF, Dr);
            } else {
                pc.drives(d.t_in + t_mid, Dr);
            }
#pragma unroll
            for (int i = 0; i < S; ++i) {
                yt[i].v = gq::f2_fma(h2, k[i].v, y[i].v);
                acc[i] = k[i];
            }
            pc.rhs(yt, Dr, k);
#pragma unroll
            for (int i = 0; i < S; ++i) {
                yt[i].v = gq::f2_fma(h2, k[i].v, y[i].v);
                acc[i].v = gq::f2_fma(two, k[i].v, acc[i].v);
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
                yt[i].v = gq::f2_fma(h, k[i].v, y[i].v);
                acc[i].v = gq::f2_fma(two, k[i].v, acc[i].v);
            }
            pc.rhs(yt, Dr, k);
#pragma unroll
            for (int i = 0; i < S; ++i) {
                acc[i].v = gq::f2_add(acc[i].v, k[i].v);
                FormFP32x2::accumulate(y[i], cn[i], acc[i], h6hi, h6lo);
            }
            if (step + 1 < d.num_steps) pc.rhs(y, Dr, k);
            rec.step(d, pc, local, second_valid, step, y, Dr);
        }
        rec.finish(d, pc, local, second_valid, y, Dr);
    }
};

// One thread per pair of consecutive points: local points 2q and 2q + 1 of the launch.
template <class M, int OUT, int TRACE>
__global__ void __launch_bounds__(GQ_BLOCK, GQ_MIN_BLOCKS) sweep_pair_kernel(const gqis_sweep_desc d) {
    const int64_t pair = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t pair_count = (d.point_count + 1) / 2;
    if (pair >= pair_count) return;
    RK4x2::run<M, OUT, TRACE>(d, pair, pair_count);
}

// A batch: item i covers pairs [starts[i], starts[i + 1]), a whole number of warps of pairs.
template <class M, int OUT, int TRACE>
__global__ void __launch_bounds__(GQ_BLOCK, GQ_MIN_BLOCKS)
    sweep_pair_batch_kernel(const __grid_constant__ BatchParams b) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= b.starts[b.count]) return;
    const int i = batch_item(b, g);  // the same for the whole warp
    const gqis_sweep_desc& d = b.items[i];
    const int64_t pair = g - b.starts[i];
    const int64_t pair_count = (d.point_count + 1) / 2;
    if (pair >= pair_count) return;
    RK4x2::run<M, OUT, TRACE>(d, pair, pair_count);
}

}  // namespace gqpacked
