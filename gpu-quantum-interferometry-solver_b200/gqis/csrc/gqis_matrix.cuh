// gqis_matrix.cuh - density-matrix form of the Lindblad sweep for larger Hilbert spaces.
//
// The reduced one-point-per-thread kernels keep N*N-1 reals per point in registers and spill
// from N ~ 16 on (the N = 16 reduced RHS has ~30k operations over 255 states). Here one CTA
// integrates one parameter point; rho (N x N complex, N padded to the model's tile) is spread
// over the CTA's threads as register tiles of TR x TC elements, and the RHS is
//     d rho/dt = -i (K - K^dag) + J(rho),   K = H_eff(t) rho,
//     H_eff(t) = Heff0 + sum_k c_k(t) M_k + sum_g c_g(t) diag(v_g),
//     Heff0 = H0 - i/2 sum_L L^dag L   (constant-rate collapse operators),
//     J(rho)_e = W_e rho_e + sum_q coef_q [c_rate(q)] rho_src(q)   (the L rho L^dag terms),
// which is the master equation of gqis/solver.py:452-457 written with rho H^dag = (H rho)^dag
// (rho is Hermitian). The constant operators Heff0, M_k, v_g, W, the jump list, O and rho0 are
// model data baked into the module (struct MM of the generated source); the coefficients
// c(t) = MM::coef(t, X, Y, consts) are evaluated in FP64 at each stage time.
// The RK4 stage structure, stage times, right-endpoint mean and FP32-form compensated update
// are those of gqfixed::RK4. The mean of <O> is accumulated in FP64 per thread as the thread's
// part of Tr(O rho) (linear in rho), so no per-step reduction is needed.
#pragma once

#include "gqis_common.cuh"

namespace gqmatrix {

template <class R>
struct Cx {
    R re, im;
};

// Complex entry i of an interleaved (re, im) array, one 8- or 16-byte load (the module's arrays
// are 16-byte aligned).
__device__ __forceinline__ Cx<float> ldc(const float* __restrict__ p, int i) {
    const float2 v = __ldg(reinterpret_cast<const float2*>(p) + i);
    return {v.x, v.y};
}
__device__ __forceinline__ Cx<double> ldc(const double* __restrict__ p, int i) {
    const double2 v = __ldg(reinterpret_cast<const double2*>(p) + i);
    return {v.x, v.y};
}

template <class R>
__device__ __forceinline__ void cmac(Cx<R>& acc, Cx<R> a, Cx<R> x) {  // acc += a * x
    acc.re = fma(a.re, x.re, fma(-a.im, x.im, acc.re));
    acc.im = fma(a.re, x.im, fma(a.im, x.re, acc.im));
}

// Dynamic shared memory of the kernel: the stage input (two buffers, or one and a barrier more per
// stage), K (rows padded by one) and H(t) = Heff0 + sum_k c_k(t) M_k (rows padded by one), formed once
// per coefficient time instead of by every thread that reads an entry. Layouts in order of
// preference, the first that fits one CTA (227 KB): two buffers + H, one buffer + H, two buffers.
constexpr size_t kSmemLimit = 232448;
template <class MM, class R>
constexpr size_t smem_layout_bytes(int buffers, bool with_h) {
    return ((size_t)buffers * MM::N * MM::N + (size_t)(with_h ? 2 : 1) * MM::N * (MM::N + 1)) * sizeof(Cx<R>);
}
template <class MM, class R>
constexpr bool h_in_smem() {
    return smem_layout_bytes<MM, R>(1, true) <= kSmemLimit;
}
template <class MM, class R>
constexpr int stage_buffers() {
    return (smem_layout_bytes<MM, R>(2, true) <= kSmemLimit || !h_in_smem<MM, R>()) ? 2 : 1;
}
template <class MM, class R>
constexpr size_t smem_bytes() {
    return smem_layout_bytes<MM, R>(stage_buffers<MM, R>(), h_in_smem<MM, R>());
}

template <class MM, class F, int OUT, int TRACE>
__global__ void __launch_bounds__(MM::THREADS) matrix_rk4_kernel(const gqis_sweep_desc d) {
    using R = typename F::real;
    constexpr int N = MM::N, NN = N * N, TR = MM::TR, TC = MM::TC, COLT = N / TC, LD = N + 1;
    constexpr int NO = MM::NO;
    static_assert((N / TR) * COLT == MM::THREADS && MM::THREADS % 32 == 0, "tile layout");
    extern __shared__ __align__(16) unsigned char gq_smem[];
    constexpr bool kHs = h_in_smem<MM, R>();
    constexpr int NB = stage_buffers<MM, R>();
    Cx<R>* const bufs = reinterpret_cast<Cx<R>*>(gq_smem);  // [NB][NN]
    Cx<R>* const Ks = bufs + NB * NN;                        // [N][LD]
    Cx<R>* const Hs = Ks + N * LD;                           // [N][LD] H(t), if kHs

    const int64_t local = blockIdx.x;
    const int64_t p = d.point_begin + local;
    const int ix = (int)(p / d.num_y);
    const int iy = (int)(p - (int64_t)ix * d.num_y);
    const double Xd = d.par_x[ix], Yd = d.par_y[iy];
    double Cd[MM::NCONST];
#pragma unroll
    for (int i = 0; i < MM::NCONST; ++i) Cd[i] = d.consts ? __ldg(d.consts + i) : 0.0;
    const int tid = threadIdx.x;
    const int r0 = (tid / COLT) * TR, c0 = (tid % COLT) * TC;

    Cx<R> y[TR][TC], k[TR][TC], acc[TR][TC];
    R cre[TR][TC], cim[TR][TC];  // compensation terms of the FP32 form's update
    // ---- initial state: the model's rho0, or the reduced layout of gqis/solver.py:202-250
    double pop_last = 1.0;
    if constexpr (MM::kInitFromArray) {
        const R* src = static_cast<const R*>(d.rho0) + (size_t)local * MM::S;
        for (int i = 0; i < NO - 1; ++i) pop_last -= (double)src[i];
    }
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
        for (int b = 0; b < TC; ++b) {
            const int i = r0 + a, j = c0 + b;
            Cx<R> v = {(R)0, (R)0};
            if constexpr (MM::kInitFromArray) {
                const R* src = static_cast<const R*>(d.rho0) + (size_t)local * MM::S;
                if (i < NO && j < NO) {
                    if (i == j) {
                        v.re = (i < NO - 1) ? src[i] : (R)pop_last;
                    } else {
                        const int lo = i < j ? i : j, hi = i < j ? j : i;
                        const int slot = NO - 1 + 2 * (lo * NO - (lo * (lo + 1)) / 2 + (hi - lo - 1));
                        v.re = src[slot];
                        v.im = (i < j) ? src[slot + 1] : -src[slot + 1];
                    }
                }
            } else {
                const Cx<double> r = ldc(MM::rho0(), i * N + j);
                v = {(R)r.re, (R)r.im};
            }
            y[a][b] = v;
            cre[a][b] = cim[a][b] = (R)0;
        }

    double c[MM::NCOEF > 0 ? MM::NCOEF : 1];
    R cr[MM::NCOEF > 0 ? MM::NCOEF : 1];
    // H(t) entry e of the current coefficients, with the same operations wherever it is formed
    auto h_entry = [&](int e) {
        Cx<R> h = ldc(MM::heff(), e);
#pragma unroll
        for (int q = 0; q < MM::ND; ++q) {
            const Cx<R> dq = ldc(MM::dense(q), e);
            h.re = fma(cr[q], dq.re, h.re);
            h.im = fma(cr[q], dq.im, h.im);
        }
        return h;
    };
    // Coefficients at time t; with kHs also H(t) into shared memory. Called between stages: the last
    // reads of Hs (the previous stage's products) precede that stage's K barrier, and the next
    // stage's products follow its first barrier.
    auto coef = [&](double t) {
        MM::coef(t, Xd, Yd, Cd, c);
#pragma unroll
        for (int q = 0; q < MM::NCOEF; ++q) cr[q] = (R)c[q];
        if constexpr (kHs) {
            for (int e = tid; e < NN; e += MM::THREADS) Hs[(e / N) * LD + e % N] = h_entry(e);
        }
    };

    // k = f(rho) for the stage input in buffer `bi` (written by every thread before the call).
    auto rhs = [&](int bi) {
        const Cx<R>* __restrict__ rt = bufs + (NB > 1 ? bi : 0) * NN;
        __syncthreads();  // stage input complete; previous readers of Ks are done
        Cx<R> kt[TR][TC];
#pragma unroll
        for (int a = 0; a < TR; ++a)
#pragma unroll
            for (int b = 0; b < TC; ++b) kt[a][b] = {(R)0, (R)0};
#pragma unroll 4
        for (int m = 0; m < N; ++m) {
            Cx<R> col[TC];
#pragma unroll
            for (int b = 0; b < TC; ++b) col[b] = rt[m * N + c0 + b];
#pragma unroll
            for (int a = 0; a < TR; ++a) {
                const Cx<R> h = kHs ? Hs[(r0 + a) * LD + m] : h_entry((r0 + a) * N + m);
#pragma unroll
                for (int b = 0; b < TC; ++b) cmac(kt[a][b], h, col[b]);
            }
        }
        if constexpr (MM::NG > 0) {
#pragma unroll
            for (int a = 0; a < TR; ++a) {
                Cx<R> dv = {(R)0, (R)0};
#pragma unroll
                for (int g = 0; g < MM::NG; ++g) {
                    const Cx<R> v = ldc(MM::diag(g), r0 + a);
                    dv.re = fma(cr[MM::ND + g], v.re, dv.re);
                    dv.im = fma(cr[MM::ND + g], v.im, dv.im);
                }
#pragma unroll
                for (int b = 0; b < TC; ++b) cmac(kt[a][b], dv, rt[(r0 + a) * N + c0 + b]);
            }
        }
#pragma unroll
        for (int a = 0; a < TR; ++a)
#pragma unroll
            for (int b = 0; b < TC; ++b) Ks[(r0 + a) * LD + c0 + b] = kt[a][b];
        __syncthreads();  // K complete
#pragma unroll
        for (int a = 0; a < TR; ++a)
#pragma unroll
            for (int b = 0; b < TC; ++b) {
                const int i = r0 + a, j = c0 + b, e = i * N + j;
                const Cx<R> kij = Ks[i * LD + j], kji = Ks[j * LD + i];
                Cx<R> o = {kij.im + kji.im, kji.re - kij.re};  // -i (K_ij - conj(K_ji))
                cmac(o, ldc(MM::wjump(), e), rt[e]);
                if constexpr (MM::NJ > 0) {
                    const int q1 = __ldg(MM::jbegin() + e + 1);
                    for (int q = __ldg(MM::jbegin() + e); q < q1; ++q) {
                        Cx<R> w = ldc(MM::jcoef(), q);
                        const int rate = __ldg(MM::jrate() + q);
                        if (rate >= 0) {
                            w.re *= cr[rate];
                            w.im *= cr[rate];
                        }
                        cmac(o, w, rt[__ldg(MM::jsrc() + q)]);
                    }
                }
                k[a][b] = o;
            }
    };

    auto write_stage = [&](int bi, R s) {  // buffer bi <- y + s k
        if constexpr (NB == 1) __syncthreads();  // the previous stage input is no longer read
        Cx<R>* __restrict__ w = bufs + (NB > 1 ? bi : 0) * NN;
#pragma unroll
        for (int a = 0; a < TR; ++a)
#pragma unroll
            for (int b = 0; b < TC; ++b)
                w[(r0 + a) * N + c0 + b] = {fma(s, k[a][b].re, y[a][b].re), fma(s, k[a][b].im, y[a][b].im)};
    };

    // This thread's part of Tr(O rho) = sum_ij O_ji rho_ij, in FP64.
    auto observe = [&](double& ore, double& oim) {
#pragma unroll
        for (int a = 0; a < TR; ++a)
#pragma unroll
            for (int b = 0; b < TC; ++b) {
                const Cx<double> o = ldc(MM::obs_t(), (r0 + a) * N + c0 + b);
                const double xr = (double)y[a][b].re, xi = (double)y[a][b].im;
                ore = fma(o.re, xr, fma(-o.im, xi, ore));
                oim = fma(o.re, xi, fma(o.im, xr, oim));
            }
    };

    // Sum of (re, im) over the CTA, valid in thread 0 (the callers are uniform over the CTA; the
    // buffer is reused only after further barriers).
    __shared__ double red[2][MM::THREADS / 32];
    auto cta_sum = [&](double& re, double& im) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            re += __shfl_xor_sync(0xffffffffu, re, off);
            im += __shfl_xor_sync(0xffffffffu, im, off);
        }
        if ((tid & 31) == 0) {
            red[0][tid >> 5] = re;
            red[1][tid >> 5] = im;
        }
        __syncthreads();
        if (tid == 0) {
            re = im = 0.0;
            for (int w = 0; w < MM::THREADS / 32; ++w) {
                re += red[0][w];
                im += red[1][w];
            }
        }
    };

    const double dt = d.dt, dt2d = dt * 0.5;
    const R h = (R)dt, h2 = (R)dt2d;
    const Coef<R> h6 = Coef<R>::make(dt / 6.0);
    double osum_re = 0.0, osum_im = 0.0;
    int next_sample = d.trace_offset, sample = 0;  // observable trace, as the Recorder of gqfixed
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
        for (int b = 0; b < TC; ++b) k[a][b] = {(R)0, (R)0};
    int cur = 0;
    write_stage(0, (R)0);
    coef(d.t_in + 0.0);
    rhs(0);
    for (int step = 0; step < d.num_steps; ++step) {
        double t_mid = ((double)step + 0.5) * dt;
#pragma unroll
        for (int a = 0; a < TR; ++a)
#pragma unroll
            for (int b = 0; b < TC; ++b) acc[a][b] = k[a][b];
        write_stage(cur ^ 1, h2);
        cur ^= 1;
        coef(d.t_in + t_mid);
        rhs(cur);
#pragma unroll
        for (int a = 0; a < TR; ++a)
#pragma unroll
            for (int b = 0; b < TC; ++b)
                acc[a][b] = {fma((R)2, k[a][b].re, acc[a][b].re), fma((R)2, k[a][b].im, acc[a][b].im)};
        write_stage(cur ^ 1, h2);
        cur ^= 1;
        rhs(cur);
        t_mid += dt2d;
#pragma unroll
        for (int a = 0; a < TR; ++a)
#pragma unroll
            for (int b = 0; b < TC; ++b)
                acc[a][b] = {fma((R)2, k[a][b].re, acc[a][b].re), fma((R)2, k[a][b].im, acc[a][b].im)};
        write_stage(cur ^ 1, h);
        cur ^= 1;
        coef(d.t_in + t_mid);
        rhs(cur);
#pragma unroll
        for (int a = 0; a < TR; ++a)
#pragma unroll
            for (int b = 0; b < TC; ++b) {
                acc[a][b].re += k[a][b].re;
                acc[a][b].im += k[a][b].im;
                F::accumulate(y[a][b].re, cre[a][b], acc[a][b].re, h6);
                F::accumulate(y[a][b].im, cim[a][b], acc[a][b].im, h6);
            }
        if (OUT == GQIS_OUT_MEAN && step >= d.warmup_steps) observe(osum_re, osum_im);
        if constexpr (TRACE == GQIS_TRACE_OBSERVABLE) {
            if (step == next_sample) {
                double tre = 0.0, tim = 0.0;
                observe(tre, tim);
                cta_sum(tre, tim);
                if (tid == 0 && sample < d.num_trace) {
                    R* tr = static_cast<R*>(d.trace) + ((size_t)local * d.num_trace + sample) * 2;
                    tr[0] = (R)tre;
                    tr[1] = (R)tim;
                }
                ++sample;
                next_sample += d.trace_stride;
            }
        }
        if (step + 1 < d.num_steps) {  // k1 of the next step, at this step's end time
            write_stage(cur ^ 1, (R)0);
            cur ^= 1;
            rhs(cur);
        }
    }

    R* out = static_cast<R*>(d.results);
    if constexpr (OUT == GQIS_OUT_FINAL_STATE) {
#pragma unroll
        for (int a = 0; a < TR; ++a)
#pragma unroll
            for (int b = 0; b < TC; ++b) {
                const int i = r0 + a, j = c0 + b;
                R* dst = out + (size_t)local * MM::S;
                if (i == j && i < NO - 1) {
                    dst[i] = y[a][b].re;
                } else if (i < j && j < NO) {
                    const int slot = NO - 1 + 2 * (i * NO - (i * (i + 1)) / 2 + (j - i - 1));
                    dst[slot] = y[a][b].re;
                    dst[slot + 1] = y[a][b].im;
                }
            }
    } else {
        if constexpr (OUT == GQIS_OUT_FINAL) observe(osum_re, osum_im);
        cta_sum(osum_re, osum_im);
        if (tid == 0) {
            double sr = osum_re, si = osum_im;
            if constexpr (OUT == GQIS_OUT_MEAN) {
                const double inv = 1.0 / (double)(d.num_steps - d.warmup_steps);
                sr *= inv;
                si *= inv;
            }
            out[2 * (size_t)local] = (R)sr;
            out[2 * (size_t)local + 1] = (R)si;
        }
    }
}

}  // namespace gqmatrix
