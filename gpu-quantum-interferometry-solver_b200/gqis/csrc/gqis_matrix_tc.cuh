// gqis_matrix_tc.cuh - density-matrix Lindblad sweep on the sm_100a tensor cores (tcgen05).
//
// Same master equation, RK4 stage structure and outputs as gqis_matrix.cuh (the CUDA-core
// form), with the operator products on the tensor cores. One CTA integrates a tile of
// P = 128 / N points (N = padded dimension 8, 16 or 32); the tile is one M = 128 MMA:
//
//   row r = p*N + j  (point p of the tile, column j of its rho)  = tensor-memory lane r
//   A[r][k]   = Re rho_p[k][j] (k < N),  Im rho_p[k-N][j] (k >= N)        (tensor memory)
//   B[k][col] = real embedding of T_q^T for the operator terms           (shared memory)
//               T_0 = Heff0, T_q = M_q (dense, q = 1..ND), T_{ND+g} = diag(v_g) (g = 1..NG)
//               col = (2q + c) N + n, c = 0 (Re) / 1 (Im)
//   D[r][col] = Re/Im (T_q rho_p)[n][j]                                    (tensor memory)
//
// One MMA chain gives every point's T_q rho at once; the epilogue forms K = sum_q c_q(t) T_q rho
// with the point's FP64-evaluated coefficients (c_0 = 1), -i (K - K^dag) through a transposed
// read of K in shared memory, the jump terms, and the RK4 combination, and writes the next stage
// input back into A. Operands are split TF32 (x = hi + lo, both TF32), three MMAs per K step
// (hi*hi + hi*lo + lo*hi) with FP32 accumulation; the state is FP32 with the FP32 form's
// compensated update, time and coefficients FP64, the mean of <O> FP64.
//
// Thread t: lane r = t % 128 (warp quadrant r / 32), rows n0 = 8 (t / 128) .. n0 + 7 of column j.
// Diagonal operator terms go through the MMA (kDiagInMma, small N) or the epilogue (larger N,
// where the MMA is the longer part of a stage). Coefficients are evaluated once per point and
// stage time by one thread and shared through shared memory. Jump terms come from per-thread
// lists (the module's tcj_* tables) whose sources are populations rho_aa, shared through shared
// memory when the stage input is written, or the thread's own element (element-wise terms on
// coherences, kOwnTerms); those and the diagonal terms done in the epilogue read the stage input
// back from A (hi + lo).
// One thread polls the MMA's mbarrier (bounded); the CTA meets it at a barrier. On give-up the
// CTA writes NaN outputs, waits (bounded) for the MMA in flight, frees its tensor memory and
// returns.
#pragma once

#include <type_traits>

#include "gqis_matrix.cuh"
#include "gqis_tcgen05.cuh"

namespace gqmatrix_tc {

using gqmatrix::Cx;
using gqmatrix::ldc;

constexpr uint32_t kMaxPolls = 1u << 20;  // mbarrier polls before a wait gives up

template <class MM>
struct TcShape {
    static constexpr int N = MM::N;
    static constexpr int P = 128 / N;         // points per tile
    static constexpr int E = 8;               // rows of a column per thread
    static constexpr int H = N / E;           // threads per column
    static constexpr int THREADS = 128 * H;
    static constexpr int MIN_CTAS = 65536 / (THREADS * 128);  // keeps <= 128 registers per thread
    static constexpr int NGM = MM::kDiagInMma ? MM::NG : 0;  // diagonal terms done by the MMA
    static constexpr int NT = 1 + MM::ND + NGM;      // operator terms in B
    static constexpr int NMMA = 2 * N * NT;   // B / D columns
    static constexpr int KDIM = 2 * N;        // real-embedded inner dimension
    static constexpr int KCH = KDIM / 8;      // MMA K steps of 8 TF32
    static constexpr int NC = MM::NCOEF > 0 ? MM::NCOEF : 1;
    static constexpr int COL_D = 0, COL_AHI = NMMA, COL_ALO = NMMA + KDIM;
    static constexpr int COLS_USED = NMMA + 2 * KDIM;
    static constexpr int TMEM_COLS = COLS_USED <= 32 ? 32 : COLS_USED <= 64 ? 64 : COLS_USED <= 128 ? 128
                                   : COLS_USED <= 256 ? 256 : 512;
    static constexpr int LDK = N + 1;         // padded column stride of the K buffer
    // shared memory layout (bytes)
    static constexpr size_t B_BYTES = (size_t)NMMA * KDIM * 4;
    static constexpr size_t OFF_BHI = 0, OFF_BLO = B_BYTES;
    static constexpr size_t OFF_K = 2 * B_BYTES;
    static constexpr size_t K_BYTES = (size_t)P * N * LDK * 8;
    static constexpr size_t OFF_RD = OFF_K + K_BYTES;           // [2][P*N] populations of the stage input
    static constexpr size_t RD_BYTES = 2 * (size_t)P * N * 4;
    static constexpr size_t OFF_CS = OFF_RD + RD_BYTES;         // [2][P][NC] coefficients
    static constexpr size_t CS_BYTES = 2 * (size_t)P * NC * 4;
    static constexpr size_t OFF_RED = (OFF_CS + CS_BYTES + 7) / 8 * 8;
    static constexpr size_t RED_BYTES = 2 * (size_t)H * P * 8;
    static constexpr size_t OFF_MISC = OFF_RED + RED_BYTES;
    static constexpr size_t NEEDED = OFF_MISC + 64;
    // At most 512 / TMEM_COLS CTAs can hold tensor memory on one SM: pad the shared memory so that
    // no more CTAs fit (228 KB per SM, 1 KB reserved per CTA) and no allocation ever waits.
    static constexpr int MAX_CTAS = 512 / TMEM_COLS;
    static constexpr size_t FLOOR = 233472 / (MAX_CTAS + 1) + 1;
    static constexpr size_t SMEM = ((NEEDED > FLOOR ? NEEDED : FLOOR) + 1023) / 1024 * 1024;
    static_assert(N == 8 || N == 16 || N == 32, "tensor-core form: padded dimension 8, 16 or 32");
    static_assert(NMMA % 16 == 0 && NMMA <= 256, "MMA N dimension");
    static_assert(COLS_USED <= 512, "tensor memory columns");
    static_assert(SMEM <= 232448, "shared memory per CTA");
    static_assert(MIN_CTAS >= 1, "threads");
};

// Byte offset of B element (col, k) in the K-major no-swizzle layout: per K step of 8, rows in
// groups of 8 (256 bytes: two 8 x 16-byte core matrices for the K halves).
template <class T>
__device__ __forceinline__ uint32_t b_offset(int col, int k) {
    return (uint32_t)((k >> 3) * (T::NMMA * 32) + (col >> 3) * 256 + ((k & 7) >> 2) * 128 + (col & 7) * 16 + (k & 3) * 4);
}

// TF32 rounding (nearest, ties away from zero) of a finite FP32 number with integer operations:
// add half a unit of the 10-bit mantissa's last place to the magnitude, clear the 13 dropped bits.
__device__ __forceinline__ float tf32_round(float x) {
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

template <class MM, int OUT, int TRACE>
__global__ void __launch_bounds__(TcShape<MM>::THREADS, TcShape<MM>::MIN_CTAS) matrix_tc_kernel(const gqis_sweep_desc d) {
    using T = TcShape<MM>;
    using F = FormFP32;
    constexpr int N = T::N, P = T::P, E = T::E, LDK = T::LDK, NO = MM::NO, NC = T::NC;
    static_assert(std::is_same<typename MM::real, float>::value, "tensor-core form uses FP32 model data");
    extern __shared__ __align__(1024) unsigned char gq_smem[];
    float* const bhi = reinterpret_cast<float*>(gq_smem + T::OFF_BHI);
    float* const blo = reinterpret_cast<float*>(gq_smem + T::OFF_BLO);
    Cx<float>* const kbuf = reinterpret_cast<Cx<float>*>(gq_smem + T::OFF_K);
    float* const rdiag = reinterpret_cast<float*>(gq_smem + T::OFF_RD);
    float* const cs = reinterpret_cast<float*>(gq_smem + T::OFF_CS);
    double* const red = reinterpret_cast<double*>(gq_smem + T::OFF_RED);
    uint64_t* const bar = reinterpret_cast<uint64_t*>(gq_smem + T::OFF_MISC);
    uint32_t* const tslot = reinterpret_cast<uint32_t*>(gq_smem + T::OFF_MISC + 8);

    const int tid = threadIdx.x;
    const int r = tid & 127;
    const int hh = tid >> 7;
    const int p = r / N, j = r % N;
    const int n0 = hh * E;
    const int warp = tid >> 5;
    const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
    const bool lead = (j == 0) && (hh == 0);  // evaluates the point's coefficients

    const int64_t local = (int64_t)blockIdx.x * P + p;
    const bool active = local < d.point_count;
    const int64_t lp = active ? local : d.point_count - 1;  // idle rows integrate a copy of the last point
    const int64_t gp = d.point_begin + lp;
    const int ix = (int)(gp / d.num_y);
    const int iy = (int)(gp - (int64_t)ix * d.num_y);
    const double Xd = d.par_x[ix], Yd = d.par_y[iy];

    // ---- B = split-TF32 real embedding of the operator terms; mbarrier; tensor memory
    for (int e = tid; e < T::NMMA * T::KDIM; e += T::THREADS) {
        const int col = e / T::KDIM, k = e % T::KDIM;
        const int q = col / (2 * N), c = (col / N) & 1, n = col % N;
        const int m = k % N;
        const bool imag_in = k >= N;
        float tr, ti;
        if (q <= MM::ND) {  // Heff0 and the dense terms; then the diagonal terms (NGM of them)
            const float* op = (q == 0) ? MM::heff() : MM::dense(q - 1);
            tr = __ldg(op + 2 * (n * N + m));
            ti = __ldg(op + 2 * (n * N + m) + 1);
        } else {
            const float* v = MM::diag(q - 1 - MM::ND);
            tr = (n == m) ? __ldg(v + 2 * n) : 0.f;
            ti = (n == m) ? __ldg(v + 2 * n + 1) : 0.f;
        }
        const float val = (c == 0) ? (imag_in ? -ti : tr) : (imag_in ? tr : ti);
        const float hi = tf32_round(val);
        const float lo = tf32_round(val - hi);
        const uint32_t off = b_offset<T>(col, k) >> 2;
        bhi[off] = hi;
        blo[off] = lo;
    }
    gqtc::fence_proxy_async_smem();
    if (tid == 0) gqtc::mbar_init(bar, 1);
    if (warp == 0) {
        gqtc::tmem_alloc(tslot, T::TMEM_COLS);
        gqtc::tmem_relinquish();
    }
    gqtc::fence_before_sync();
    __syncthreads();
    gqtc::fence_after_sync();
    const uint32_t tbase = *tslot;
    const uint32_t t_d = tbase + T::COL_D + lane_base;
    const uint32_t t_ahi = tbase + T::COL_AHI + lane_base;
    const uint32_t t_alo = tbase + T::COL_ALO + lane_base;
    const uint32_t idesc = gqtc::idesc_tf32_m128(T::NMMA);
    const uint32_t b_hi_addr = gqtc::smem_u32(bhi), b_lo_addr = gqtc::smem_u32(blo);

    // ---- state: rows n0..n0+7 of column j, FP32 with compensation
    float yre[E], yim[E], cre[E], cim[E], are[E], aim[E];
    {
        double pop_last = 1.0;
        if constexpr (MM::kInitFromArray) {
            const float* src = static_cast<const float*>(d.rho0) + (size_t)lp * MM::S;
            for (int i = 0; i < NO - 1; ++i) pop_last -= (double)src[i];
        }
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int n = n0 + e;
            float vr = 0.f, vi = 0.f;
            if constexpr (MM::kInitFromArray) {
                const float* src = static_cast<const float*>(d.rho0) + (size_t)lp * MM::S;
                if (n < NO && j < NO) {
                    if (n == j) {
                        vr = (n < NO - 1) ? src[n] : (float)pop_last;
                    } else {
                        const int lo = n < j ? n : j, hi = n < j ? j : n;
                        const int slot = NO - 1 + 2 * (lo * NO - (lo * (lo + 1)) / 2 + (hi - lo - 1));
                        vr = src[slot];
                        vi = (n < j) ? src[slot + 1] : -src[slot + 1];
                    }
                }
            } else {
                const Cx<double> v = ldc(MM::rho0(), n * N + j);
                vr = (float)v.re;
                vi = (float)v.im;
            }
            yre[e] = vr;
            yim[e] = vi;
            cre[e] = cim[e] = 0.f;
            are[e] = aim[e] = 0.f;
        }
    }
    const int jl = j * T::H + hh;  // this thread's jump list
    const int jcount = __ldg(MM::tcj_count() + jl);

    // coefficients of the point at time t into slot `v` (lead thread only)
    auto coef = [&](double t, int v) {
        if (lead) {
            double Cd[MM::NCONST], c[NC];
#pragma unroll
            for (int i = 0; i < MM::NCONST; ++i) Cd[i] = d.consts ? __ldg(d.consts + i) : 0.0;
            MM::coef(t, Xd, Yd, Cd, c);
#pragma unroll
            for (int q = 0; q < MM::NCOEF; ++q) cs[(v * P + p) * NC + q] = (float)c[q];
        }
    };

    // stage input u = y + s k -> A (hi / lo TF32 parts); populations -> rdiag[slot]
    auto write_stage = [&](float s, const float (&kre)[E], const float (&kim)[E], int slot) {
        float hr[E], hi_[E], lr[E], li[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const float ur = fmaf(s, kre[e], yre[e]), ui = fmaf(s, kim[e], yim[e]);
            hr[e] = tf32_round(ur);
            hi_[e] = tf32_round(ui);
            lr[e] = ur - hr[e];  // |lo| <= 2^-11 |u|; its TF32 read loses at most 2^-21 |u|
            li[e] = ui - hi_[e];
            if (n0 + e == j) rdiag[slot * P * N + p * N + j] = ur;
        }
        gqtc::tmem_st8(t_ahi + n0, hr);
        gqtc::tmem_st8(t_ahi + N + n0, hi_);
        gqtc::tmem_st8(t_alo + n0, lr);
        gqtc::tmem_st8(t_alo + N + n0, li);
    };

    uint32_t phase = 0;
    // k = f(u) for the stage input in A; false when the MMA wait gave up (uniform over the CTA).
    auto eval = [&](float (&kre)[E], float (&kim)[E], int slot, int v) -> bool {
        gqtc::tmem_wait_st();
        gqtc::fence_before_sync();
        __syncthreads();  // stage input complete in A; coefficients and populations written
        if (tid == 0) {
            gqtc::fence_after_sync();
#pragma unroll
            for (int kc = 0; kc < T::KCH; ++kc) {
                const uint32_t boff = (uint32_t)(kc * T::NMMA * 32);
                const uint64_t dh = gqtc::smem_desc_kmajor(b_hi_addr + boff, 128, 256);
                const uint64_t dl = gqtc::smem_desc_kmajor(b_lo_addr + boff, 128, 256);
                gqtc::mma_tf32_ts(tbase + T::COL_D, tbase + T::COL_AHI + 8 * kc, dh, idesc, kc > 0 ? 1u : 0u);
                gqtc::mma_tf32_ts(tbase + T::COL_D, tbase + T::COL_AHI + 8 * kc, dl, idesc, 1u);
                gqtc::mma_tf32_ts(tbase + T::COL_D, tbase + T::COL_ALO + 8 * kc, dh, idesc, 1u);
            }
            gqtc::mma_commit(bar);
        }
        float cq[T::NT];  // the point's coefficients of the operator terms (c_0 = 1)
        cq[0] = 1.f;
#pragma unroll
        for (int q = 1; q < T::NT; ++q) cq[q] = cs[(v * P + p) * NC + (q - 1)];
        // one thread polls the mbarrier; the others wait at the barrier instead of spinning
        const bool ok = (tid != 0) || gqtc::mbar_wait_bounded(bar, phase, kMaxPolls);
        if (__syncthreads_or(!ok)) return false;  // MMA complete (or given up, uniformly)
        phase ^= 1u;
        gqtc::fence_after_sync();
        float Kr[E], Ki[E];
#pragma unroll
        for (int q = 0; q < T::NT; ++q) {
            float a[8], b[8];
            gqtc::tmem_ld8(t_d + (2 * q) * N + n0, a);
            gqtc::tmem_ld8(t_d + (2 * q + 1) * N + n0, b);
            gqtc::tmem_wait_ld();
#pragma unroll
            for (int e = 0; e < E; ++e) {
                Kr[e] = (q == 0) ? a[e] : fmaf(cq[q], a[e], Kr[e]);
                Ki[e] = (q == 0) ? b[e] : fmaf(cq[q], b[e], Ki[e]);
            }
        }
        float ur[E], ui[E];
        if constexpr (MM::kOwnTerms || (T::NGM < MM::NG)) {  // terms that need the stage input itself
            float a[8], b[8], c2[8], d2[8];
            gqtc::tmem_ld8(t_ahi + n0, a);
            gqtc::tmem_ld8(t_ahi + N + n0, b);
            gqtc::tmem_ld8(t_alo + n0, c2);
            gqtc::tmem_ld8(t_alo + N + n0, d2);
            gqtc::tmem_wait_ld();
#pragma unroll
            for (int e = 0; e < E; ++e) {
                ur[e] = a[e] + c2[e];
                ui[e] = b[e] + d2[e];
            }
        }
        if constexpr (T::NGM < MM::NG) {  // diagonal terms in the epilogue: K += (sum_g c_g v_g[n]) u[n][j]
#pragma unroll
            for (int e = 0; e < E; ++e) {
                Cx<float> dv = {0.f, 0.f};
#pragma unroll
                for (int g = 0; g < MM::NG; ++g) {
                    const Cx<float> vg = ldc(MM::diag(g), n0 + e);
                    const float cg = cs[(v * P + p) * NC + MM::ND + g];
                    dv.re = fmaf(cg, vg.re, dv.re);
                    dv.im = fmaf(cg, vg.im, dv.im);
                }
                Kr[e] = fmaf(dv.re, ur[e], fmaf(-dv.im, ui[e], Kr[e]));
                Ki[e] = fmaf(dv.re, ui[e], fmaf(dv.im, ur[e], Ki[e]));
            }
        }
#pragma unroll
        for (int e = 0; e < E; ++e) kbuf[(p * N + j) * LDK + n0 + e] = {Kr[e], Ki[e]};
        __syncthreads();  // K complete
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int n = n0 + e;
            const Cx<float> kt = kbuf[(p * N + n) * LDK + j];  // K[j][n]
            kre[e] = Ki[e] + kt.im;                             // -i (K[n][j] - conj(K[j][n]))
            kim[e] = kt.re - Kr[e];
        }
        // jump terms of this thread: population rho_aa of the stage input into row e
        float jre = 0.f, jim = 0.f;
        for (int q = 0; q < jcount; ++q) {
            const int idx = jl * MM::TCJ_MAX + q;
            const int rate = __ldg(MM::tcj_rate() + idx);
            Cx<float> w = ldc(MM::tcj_coef(), idx);
            if (rate >= 0) {
                const float cr = cs[(v * P + p) * NC + rate];
                w.re *= cr;
                w.im *= cr;
            }
            const int a = __ldg(MM::tcj_a() + idx);
            if constexpr (MM::kJumpsOnDiagonal && !MM::kOwnTerms) {
                const float x = rdiag[slot * P * N + p * N + a];
                jre = fmaf(w.re, x, jre);
                jim = fmaf(w.im, x, jim);
            } else {
                const int e = __ldg(MM::tcj_e() + idx);
                const float x = (a >= 0) ? rdiag[slot * P * N + p * N + a] : 0.f;
#pragma unroll
                for (int ee = 0; ee < E; ++ee)
                    if (ee == e) {
                        Cx<float> src = {x, 0.f};  // a population, or the element itself (a < 0)
                        if constexpr (MM::kOwnTerms) {
                            if (a < 0) src = {ur[ee], ui[ee]};
                        }
                        kre[ee] = fmaf(w.re, src.re, fmaf(-w.im, src.im, kre[ee]));
                        kim[ee] = fmaf(w.re, src.im, fmaf(w.im, src.re, kim[ee]));
                    }
            }
        }
        if constexpr (MM::kJumpsOnDiagonal) {
#pragma unroll
            for (int e = 0; e < E; ++e)
                if (n0 + e == j) {
                    kre[e] += jre;
                    kim[e] += jim;
                }
        }
        return true;
    };

    const double dt = d.dt, dt2d = dt * 0.5;
    const float h = (float)dt, h2 = (float)dt2d;
    const Coef<float> h6 = Coef<float>::make(dt / 6.0);
    double osum_re = 0.0, osum_im = 0.0;
    // Sum of (re, im) over the threads of point p, valid in its lead thread: over the N columns (lanes
    // p*N .. p*N+N-1 of a warp), then over the H row blocks through shared memory. Uniform over the CTA.
    auto point_sum = [&](double& re, double& im) {
#pragma unroll
        for (int off = N / 2; off > 0; off >>= 1) {
            re += __shfl_xor_sync(0xffffffffu, re, off);
            im += __shfl_xor_sync(0xffffffffu, im, off);
        }
        if (j == 0) {
            red[(0 * T::H + hh) * P + p] = re;
            red[(1 * T::H + hh) * P + p] = im;
        }
        __syncthreads();
        if (lead) {
            re = im = 0.0;
            for (int g = 0; g < T::H; ++g) {
                re += red[(0 * T::H + g) * P + p];
                im += red[(1 * T::H + g) * P + p];
            }
        }
    };
    int next_sample = d.trace_offset, sample = 0;  // observable trace, as the Recorder of gqfixed
    auto observe = [&]() {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const Cx<double> o = ldc(MM::obs_t(), (n0 + e) * N + j);
            const double xr = (double)yre[e], xi = (double)yim[e];
            osum_re = fma(o.re, xr, fma(-o.im, xi, osum_re));
            osum_im = fma(o.re, xi, fma(o.im, xr, osum_im));
        }
    };

    // Evaluations it = 4 n + s (step n, stage s). Stage times: s = 0 at the previous step's end
    // (t_in + 0 for n = 0), s = 1, 2 at t_mid = (n + 1/2) dt, s = 3 at t_mid + dt/2 - the times and
    // roundings of gqfixed::RK4. Coefficients change at it = 0 and at s = 1, 3 (version cv).
    bool failed = false;
    {
        float kre[E], kim[E];
#pragma unroll
        for (int e = 0; e < E; ++e) kre[e] = kim[e] = 0.f;
        int cv = 0;
        coef(d.t_in + 0.0, cv);
        write_stage(0.f, kre, kim, 0);
        const int total = 4 * d.num_steps;
        for (int it = 0; it < total; ++it) {
            const int step = it >> 2, s = it & 3;
            if (!eval(kre, kim, it & 1, cv)) {
                failed = true;
                break;
            }
            const int nslot = (it + 1) & 1;
            if (s == 3) {
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    are[e] += kre[e];
                    aim[e] += kim[e];
                    F::accumulate(yre[e], cre[e], are[e], h6);
                    F::accumulate(yim[e], cim[e], aim[e], h6);
                }
                if (OUT == GQIS_OUT_MEAN && step >= d.warmup_steps) observe();
                if constexpr (TRACE == GQIS_TRACE_OBSERVABLE) {
                    if (step == next_sample) {
                        double s_re = osum_re, s_im = osum_im;  // observe() adds into osum: keep it
                        osum_re = osum_im = 0.0;
                        observe();
                        double tre = osum_re, tim = osum_im;
                        osum_re = s_re;
                        osum_im = s_im;
                        point_sum(tre, tim);
                        if (lead && active && sample < d.num_trace) {
                            float* tr = static_cast<float*>(d.trace) + ((size_t)local * d.num_trace + sample) * 2;
                            tr[0] = (float)tre;
                            tr[1] = (float)tim;
                        }
                        ++sample;
                        next_sample += d.trace_stride;
                    }
                }
                if (step + 1 == d.num_steps) break;
#pragma unroll
                for (int e = 0; e < E; ++e) kre[e] = kim[e] = 0.f;
                write_stage(0.f, kre, kim, nslot);  // input of the next step's k1 (same time)
            } else {
                const double t_mid = ((double)step + 0.5) * dt;
                if (s == 0) {
#pragma unroll
                    for (int e = 0; e < E; ++e) {
                        are[e] = kre[e];
                        aim[e] = kim[e];
                    }
                    cv ^= 1;
                    coef(d.t_in + t_mid, cv);
                } else {
#pragma unroll
                    for (int e = 0; e < E; ++e) {
                        are[e] = fmaf(2.f, kre[e], are[e]);
                        aim[e] = fmaf(2.f, kim[e], aim[e]);
                    }
                    if (s == 2) {
                        cv ^= 1;
                        coef(d.t_in + (t_mid + dt2d), cv);
                    }
                }
                write_stage(s == 2 ? h : h2, kre, kim, nslot);
            }
        }
    }

    float* out = static_cast<float*>(d.results);
    if (failed) {
        // the MMA of the last phase did not signal: wait once more (bounded), mark the tile's outputs
        gqtc::mbar_wait_bounded(bar, phase, kMaxPolls);
        if (active && lead) {
            const int width = (OUT == GQIS_OUT_FINAL_STATE) ? MM::S : 2;
            for (int i = 0; i < width; ++i) out[(size_t)local * width + i] = __int_as_float(0x7fc00000);
        }
    } else if constexpr (OUT == GQIS_OUT_FINAL_STATE) {
        if (active) {
            float* dst = out + (size_t)local * MM::S;
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int n = n0 + e;
                if (n == j && n < NO - 1) {
                    dst[n] = yre[e];
                } else if (n < j && j < NO) {
                    const int slot = NO - 1 + 2 * (n * NO - (n * (n + 1)) / 2 + (j - n - 1));
                    dst[slot] = yre[e];
                    dst[slot + 1] = yim[e];
                }
            }
        }
    } else {
        if constexpr (OUT == GQIS_OUT_FINAL) observe();
        point_sum(osum_re, osum_im);
        if (lead && active) {
            double sr = osum_re, si = osum_im;
            if constexpr (OUT == GQIS_OUT_MEAN) {
                const double inv = 1.0 / (double)(d.num_steps - d.warmup_steps);
                sr *= inv;
                si *= inv;
            }
            out[2 * (size_t)local] = (float)sr;
            out[2 * (size_t)local + 1] = (float)si;
        }
    }
    gqtc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        gqtc::fence_after_sync();
        gqtc::tmem_dealloc(tbase, T::TMEM_COLS);
    }
}

}  // namespace gqmatrix_tc
