// gqis_matrix_tc.cuh - density-matrix Lindblad sweep on the sm_100a tensor cores (tcgen05).
//
// Same master equation, RK4 stage structure and outputs as gqis_matrix.cuh (the CUDA-core
// form), with the operator products on the tensor cores. A tile of P = 128 / N points
// (N = padded dimension 8, 16, 32 or 64) is one M = 128 MMA:
//
//   row r = p*N + j  (point p of the tile, column j of its rho)  = tensor-memory lane r
//   A[r][k]   = Re rho_p[m][j] (k = 2m),  Im rho_p[m][j] (k = 2m + 1)     (tensor memory, column m)
//   B[k][col] = real embedding of T_q^T for the operator terms           (shared memory)
//               T_0 = Heff0, T_q = M_q (dense, q = 1..ND), T_{ND+g} = diag(v_g) (g = 1..NG)
//               col = 2 NH q + 2 (n - nb) + c, c = 0 (Im) / 1 (Re)
//   D[r][col] = Im/Re (T_q rho_p)[n][j]                                    (tensor memory)
//
// Real and imaginary parts sit in adjacent D columns (and in one A column as two FP16), so one 32x32b
// load or store moves a thread's E complex elements, on which the epilogue computes in packed FP32
// (one f32x2 instruction per complex element; each lane rounds as the scalar instruction).
//
// Up to N = 32 one CTA holds the tile (NH = N rows n of every column, nb = 0). At N = 64 the
// tile's state does not fit one SM's registers, so a cluster of CL = 2 CTAs shares it: CTA c owns
// rows n in [nb, nb + NH), nb = c NH, NH = N / 2, of every column, multiplies with the B columns of
// its rows only, and both CTAs keep the whole stage input in A. Each stage the CTAs swap their
// halves of the stage input and the parts of K the other one reads transposed through distributed
// shared memory: st.async stores into the partner's buffer that count their bytes on the partner's
// mbarrier (one per buffer), on which one thread of the receiving CTA waits (bounded); no cluster-wide
// barrier inside the integration loop.
//
// One MMA chain gives every point's T_q rho at once; the epilogue forms K = sum_q c_q(t) T_q rho
// with the point's FP64-evaluated coefficients (c_0 = 1), -i (K - K^dag) through a transposed
// read of K in shared memory, the jump terms, and the RK4 combination, and writes the next stage
// input back into A. Operands are split FP16 (x = hi + lo, both FP16, 22 significant bits as a split
// TF32 pair), scaled by powers of two (A by 2^12, each operator term so that its largest entry is in
// [2^12, 2^13)) that the epilogue undoes exactly; kind::f16 MMAs (K = 16, twice the K of kind::tf32 per
// instruction at the same cycles), three per K step (hi*hi + hi*lo + lo*hi) with FP32 accumulation.
// The state is FP32 with the FP32 form's compensated update, time and coefficients FP64, the mean of
// <O> FP64.
//
// Thread t: lane r = t % 128 (warp quadrant r / 32), rows n0 = nb + E (t / 128) .. n0 + E - 1 of column j
// (E = 8 rows per thread; the emitter may choose 4).
// Diagonal operator terms go through the MMA (kDiagInMma, wherever the MMA is wide enough) or the
// epilogue (their per-point sums formed while the MMA runs). Coefficients are evaluated in FP64 for every point
// and stage time of KB steps at once, spread over all threads while an MMA runs, into a
// double-buffered table in shared memory. Jump terms come from per-thread
// lists (the module's tcj_* tables) whose sources are populations rho_aa, shared through shared
// memory when the stage input is written, or the thread's own element (element-wise terms on
// coherences, kOwnTerms); those and the diagonal terms done in the epilogue read the stage input
// back from A (hi + lo).
// Every thread polls the MMA's mbarrier (bounded; in a cluster one thread, and the CTA meets it at a
// barrier); a give-up is made uniform over the CTA at the next barrier. On give-up the
// CTA writes NaN outputs, waits (bounded) for the MMA in flight, frees its tensor memory and returns.
// A CTA of a cluster instead stops using the tensor cores but keeps exchanging (zeros) to the end of
// the loop, so its partner never waits in vain; the two tell each other at one cluster barrier after
// the loop, and both write NaN. A CTA whose exchange wait gives up stops waiting altogether.
#pragma once

#include <cuda_fp16.h>

#include <type_traits>

#include "gqis_f32x2.cuh"
#include "gqis_matrix.cuh"
#include "gqis_tcgen05.cuh"

namespace gqmatrix_tc {

using gqmatrix::Cx;
using gqmatrix::ldc;
using gq::f2_add;
using gq::f2_fma;
using gq::f2_sub;

// mbarrier polls before an in-loop wait (MMA completion, partner's bytes) gives up. A build can
// lower it (-DGQ_TC_MAX_POLLS=0 makes every such wait give up at once, which tests the give-up
// path); the final wait for an MMA still in flight keeps the full limit, so no MMA writes tensor
// memory after the kernel freed it.
#ifndef GQ_TC_MAX_POLLS
#define GQ_TC_MAX_POLLS (1u << 20)
#endif
constexpr uint32_t kMaxPolls = GQ_TC_MAX_POLLS;
constexpr uint32_t kDrainPolls = 1u << 20;

// Tensor-memory columns an allocation of `used` columns takes (a power of two, at least 32).
__host__ __device__ constexpr int tmem_alloc_cols(int used) {
    return used <= 32 ? 32 : used <= 64 ? 64 : used <= 128 ? 128 : used <= 256 ? 256 : 512;
}

template <class MM>
struct TcShape {
    static constexpr int N = MM::N;
    static constexpr int CL = MM::TC_CL;      // CTAs per tile (cluster size, chosen by the model emitter)
    static constexpr int NH = N / CL;         // rows n of every column held by one CTA
    static constexpr int P = 128 / N;         // points per tile
    static constexpr int E = MM::TC_E;        // rows of a column per thread (4 or 8, chosen by the emitter)
    static constexpr int H = NH / E;          // threads per column in one CTA
    static constexpr int THREADS = 128 * H;
    static constexpr int MIN_CTAS = 65536 / (THREADS * (E == 8 ? 128 : 64));  // registers per thread: 128 / 64
    static constexpr int NGM = MM::kDiagInMma ? MM::NG : 0;  // diagonal terms done by the MMA
    static constexpr int NT = 1 + MM::ND + NGM;      // operator terms in B
    static constexpr int NMMA = 2 * NH * NT;  // B / D columns
    static constexpr int KDIM = 2 * N;        // real-embedded inner dimension
    static constexpr int KCH = KDIM / 16;     // MMA K steps of 16 FP16
    static constexpr int NC = MM::NCOEF > 0 ? MM::NCOEF : 1;
    static constexpr int CG = N > 32 ? N / 32 : 1;  // warps spanned by one column set (point sums)
    static constexpr int KB = 8;              // steps per block of the coefficient table
    static constexpr int TS = 3 * KB;         // table slots per block: start, midpoint and end of each step
    // A: one 32-bit column per row m of the stage input, (Re, Im) as two FP16 (K elements 2m, 2m + 1)
    static constexpr int COL_D = 0, COL_AHI = NMMA, COL_ALO = NMMA + N;
    static constexpr int COLS_USED = NMMA + 2 * N;
    static constexpr int A_SCALE_EXP = 12;  // A = 2^12 u: |u| <= 16 stays below the FP16 maximum
    static constexpr uint32_t KSTEP_BYTES = 2u * NMMA * 32u;  // B of one K step: NMMA hi rows, then NMMA lo rows
    static constexpr int TMEM_COLS = tmem_alloc_cols(COLS_USED);
    static constexpr int LDK = N + 2;         // padded column stride of the K buffer (16-byte rows, no conflicts)
    static_assert(2 * E <= 16, "one 32x32b.x16 tensor-memory access per operand pair block");
    // shared memory layout (bytes)
    static constexpr size_t B_BYTES = (size_t)NMMA * KDIM * 2;  // one of the two FP16 parts
    static constexpr size_t OFF_B = 0;
    static constexpr size_t OFF_K = 2 * B_BYTES;
    static constexpr size_t K_BYTES = (size_t)P * NH * LDK * 8;  // K[j][n] for the CTA's rows n, every j
    static constexpr size_t OFF_X = OFF_K + K_BYTES;            // [P][H][E/2][N] x 2 the partner's stage input
    static constexpr size_t X_BYTES = CL > 1 ? (size_t)P * H * E * N * 8 : 0;
    static constexpr uint32_t KX_BYTES = (uint32_t)(P * NH * NH * 8);  // K entries the partner sends per stage
    static constexpr size_t OFF_RD = OFF_X + X_BYTES;           // [2][P*N] populations of the stage input
    static constexpr size_t RD_BYTES = 2 * (size_t)P * N * 4;
    static constexpr size_t OFF_CS = OFF_RD + RD_BYTES;         // [2][TS][P][NC] coefficient table
    static constexpr size_t CS_BYTES = 2 * (size_t)TS * P * NC * 4;
    static constexpr size_t OFF_RED = (OFF_CS + CS_BYTES + 7) / 8 * 8;
    static constexpr size_t RED_BYTES = 2 * (size_t)H * CG * P * 8 + 2 * (size_t)P * 8;  // + the partner's sums
    static constexpr size_t OFF_DV = OFF_RED + RED_BYTES;       // [P][N] sum_g c_g v_g[n] of the stage
    static constexpr size_t DV_BYTES = (NGM < MM::NG) ? (size_t)P * N * 8 : 0;
    static constexpr size_t OFF_MISC = OFF_DV + DV_BYTES;       // mbarriers, tensor-memory slot, failure flag
    static constexpr size_t NEEDED = OFF_MISC + 128;  // + the terms' largest B entries (bits), at + 64
    // At most 512 / TMEM_COLS CTAs can hold tensor memory on one SM: pad the shared memory so that
    // no more CTAs fit (228 KB per SM, 1 KB reserved per CTA) and no allocation ever waits.
    static constexpr int MAX_CTAS = 512 / TMEM_COLS;
    static constexpr size_t FLOOR = 233472 / (MAX_CTAS + 1) + 1;
    static constexpr size_t SMEM = ((NEEDED > FLOOR ? NEEDED : FLOOR) + 1023) / 1024 * 1024;
    static_assert(N == 8 || N == 16 || N == 32 || N == 64, "tensor-core form: padded dimension 8, 16, 32 or 64");
    static_assert(CL == 1 || CL == 2, "one or two CTAs per tile");
    static_assert((E == 4 || E == 8) && H >= 1 && NH % E == 0, "rows per thread");
    static_assert(NMMA % 16 == 0 && NMMA <= 256, "MMA N dimension");
    static_assert(COLS_USED <= 512, "tensor memory columns");
    static_assert(SMEM <= 232448, "shared memory per CTA");
    static_assert(MIN_CTAS >= 1, "threads");
    static_assert(NT <= 16, "operator terms (64 bytes of maxima)");
};

// Byte offset of B element (col, k) of FP16 part `part` (0 hi, 1 lo) in the K-major no-swizzle layout:
// per K step of 16 the hi rows, then the lo rows, in groups of 8 (256 bytes: two 8 x 16-byte core
// matrices for the K halves).
template <class T>
__device__ __forceinline__ uint32_t b_offset(int col, int k, int part) {
    return (uint32_t)((k >> 4) * T::KSTEP_BYTES + part * (T::NMMA * 32) + (col >> 3) * 256 + ((k & 15) >> 3) * 128 +
                      (col & 7) * 16 + (k & 7) * 2);
}

// Split FP16 of a scaled value x (|x| < 65504): hi = x rounded to FP16, lo = the exact remainder rounded
// to FP16, both packed as one 32-bit word per lane pair; hi + lo keeps 22 significant bits (as a split
// TF32 pair) down to |x| ~ 2^-3, and an absolute 2^-25 below.
__device__ __forceinline__ void split_f16(float2 x, uint32_t& hi, uint32_t& lo) {
    const __half2 h = __float22half2_rn(x);
    const __half2 l = __float22half2_rn(f2_sub(x, __half22float2(h)));
    hi = *reinterpret_cast<const uint32_t*>(&h);
    lo = *reinterpret_cast<const uint32_t*>(&l);
}
// (hi + lo) of a split pair, unscaled by 2^-A_SCALE_EXP
__device__ __forceinline__ float2 join_f16(uint32_t hi, uint32_t lo, float unscale) {
    const float2 h = __half22float2(*reinterpret_cast<const __half2*>(&hi));
    const float2 l = __half22float2(*reinterpret_cast<const __half2*>(&lo));
    return gq::f2_mul(f2_add(h, l), make_float2(unscale, unscale));
}

template <class MM, int OUT, int TRACE>
__global__ void __launch_bounds__(TcShape<MM>::THREADS, TcShape<MM>::MIN_CTAS) matrix_tc_kernel(const gqis_sweep_desc d) {
    using T = TcShape<MM>;
    constexpr int N = T::N, P = T::P, E = T::E, LDK = T::LDK, NO = MM::NO, NC = T::NC, NH = T::NH, H = T::H;
    static_assert(std::is_same<typename MM::real, float>::value, "tensor-core form uses FP32 model data");
    extern __shared__ __align__(1024) unsigned char gq_smem[];
    float2* const kbuf = reinterpret_cast<float2*>(gq_smem + T::OFF_K);  // (Im, Re) of K[n][j]
    float2* const xbuf = reinterpret_cast<float2*>(gq_smem + T::OFF_X);
    float* const rdiag = reinterpret_cast<float*>(gq_smem + T::OFF_RD);
    float* const cs = reinterpret_cast<float*>(gq_smem + T::OFF_CS);
    double* const red = reinterpret_cast<double*>(gq_smem + T::OFF_RED);
    Cx<float>* const dvs = reinterpret_cast<Cx<float>*>(gq_smem + T::OFF_DV);
    uint64_t* const bar = reinterpret_cast<uint64_t*>(gq_smem + T::OFF_MISC);
    uint32_t* const tslot = reinterpret_cast<uint32_t*>(gq_smem + T::OFF_MISC + 8);
    uint32_t* const fail_flag = reinterpret_cast<uint32_t*>(gq_smem + T::OFF_MISC + 12);  // set by the partner
    uint64_t* const xbar = reinterpret_cast<uint64_t*>(gq_smem + T::OFF_MISC + 16);  // partner's stage input in
    uint64_t* const kbar = reinterpret_cast<uint64_t*>(gq_smem + T::OFF_MISC + 24);  // partner's K entries in

    const int tid = threadIdx.x;
    const int r = tid & 127;
    const int hh = tid >> 7;
    const int p = r / N, j = r % N;
    const int crank = T::CL > 1 ? (int)gqtc::cluster_ctarank() : 0;
    const int nb = crank * NH;   // first row of this CTA
    const int n0 = nb + hh * E;  // first row of this thread
    const int warp = tid >> 5;
    const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
    const bool lead = (j == 0) && (hh == 0);  // holds the point's sums (in each CTA)

    const int64_t tile = (int64_t)(blockIdx.x / T::CL);
    const int64_t local = tile * P + p;
    const bool active = local < d.point_count;
    const int64_t lp = active ? local : d.point_count - 1;  // idle rows integrate a copy of the last point

    // ---- B = split-FP16 real embedding of the operator terms, each term scaled by a power of two that
    // puts its largest entry in [2^12, 2^13); mbarrier; tensor memory
    auto b_entry = [&](int col, int k) -> float {
        const int q = col / (2 * NH), n = nb + (col % (2 * NH)) / 2;
        const bool re_out = (col & 1) != 0;  // output columns (Im, Re) of row n
        const int m = k >> 1;
        const bool imag_in = (k & 1) != 0;   // input columns (Re, Im) of row m
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
        // Re out = sum Tr Re rho - Ti Im rho; Im out = sum Ti Re rho + Tr Im rho
        return re_out ? (imag_in ? -ti : tr) : (imag_in ? tr : ti);
    };
    uint32_t* const bmax = reinterpret_cast<uint32_t*>(gq_smem + T::OFF_MISC + 64);  // largest |entry| of
    // each term (FP32 bits: non-negative floats order as unsigned integers)
    if (tid < T::NT) bmax[tid] = 0u;
    __syncthreads();
    for (int e = tid; e < T::NMMA * T::KDIM; e += T::THREADS) {
        const int col = e / T::KDIM;
        atomicMax(&bmax[col / (2 * NH)], __float_as_uint(fabsf(b_entry(col, e % T::KDIM))));
    }
    __syncthreads();
    // 2^-(A scale + term scale): D_q back to the units of T_q rho (exact: powers of two)
    auto term_exp = [&](int q) -> int {
        const uint32_t bits = bmax[q];
        if (bits == 0u) return 0;
        const int ex = (int)((bits >> 23) & 0xFFu) - 127;  // floor(log2 max) of a normal number
        return min(max(12 - ex, -24), 40);
    };
    __half* const bsm = reinterpret_cast<__half*>(gq_smem + T::OFF_B);
    for (int e = tid; e < T::NMMA * T::KDIM; e += T::THREADS) {
        const int col = e / T::KDIM, k = e % T::KDIM;
        const float val = ldexpf(b_entry(col, k), term_exp(col / (2 * NH)));
        const __half hi = __float2half_rn(val);
        const __half lo = __float2half_rn(val - __half2float(hi));
        bsm[b_offset<T>(col, k, 0) >> 1] = hi;
        bsm[b_offset<T>(col, k, 1) >> 1] = lo;
    }
    float unscale[T::NT];
#pragma unroll
    for (int q = 0; q < T::NT; ++q) unscale[q] = ldexpf(1.f, -(T::A_SCALE_EXP + term_exp(q)));
    gqtc::fence_proxy_async_smem();
    if (tid == 0) {
        gqtc::mbar_init(bar, 1);
        *fail_flag = 0u;
        if constexpr (T::CL > 1) {
            gqtc::mbar_init(xbar, 1);
            gqtc::mbar_init(kbar, 1);
        }
    }
    if (warp == 0) {
        gqtc::tmem_alloc(tslot, T::TMEM_COLS);
        gqtc::tmem_relinquish();
    }
    gqtc::fence_before_sync();
    __syncthreads();
    gqtc::fence_after_sync();
    // The partner CTA's buffers (distributed shared memory) are mapped where they are used (one mapa
    // each, which keeps no address live across the loop); both CTAs run before either writes there.
    const uint32_t peer = (uint32_t)(crank ^ 1);
    if constexpr (T::CL > 1) gqtc::cluster_sync();
    const uint32_t tbase = *tslot;
    const uint32_t t_d = tbase + T::COL_D + lane_base;
    const uint32_t t_ahi = tbase + T::COL_AHI + lane_base;
    const uint32_t t_alo = tbase + T::COL_ALO + lane_base;
    const uint32_t idesc = gqtc::idesc_f16_m128(T::NMMA);
    // B descriptor of K step 0; K step kc and the lo part are fixed offsets in its 14-bit address field
    // (shared-memory addresses stay below 2^18 bytes)
    const uint64_t bdesc0 = gqtc::smem_desc_kmajor(gqtc::smem_u32(bsm), 128, 256);

    // ---- state: rows n0 .. n0 + E - 1 of column j as (Re, Im) pairs, FP32 with compensation (kept
    // negated), and the RK4 sum of the step's stages
    float2 y[E], cn[E], acc[E];
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
            y[e] = make_float2(vr, vi);
            cn[e] = acc[e] = make_float2(0.f, 0.f);
        }
    }
    const int jl = j * (N / E) + n0 / E;  // this thread's jump list (column j, row block n0 / 8)
    const int jcount = __ldg(MM::tcj_count() + jl);
    // every jump term feeds a diagonal element from a population: all of them are summed while the MMA runs
    constexpr bool kJumpsEarly = MM::kJumpsOnDiagonal && !MM::kOwnTerms;

    const double dt = d.dt, dt2d = dt * 0.5;
    // Coefficient table of block b (steps b KB .. b KB + KB - 1) into buffer b & 1: for every point of
    // the tile and step n the coefficients at the stage times of gqfixed::RK4 - slot 3 i: the step's
    // start (t_in + 0 for n = 0, else the previous step's end), 3 i + 1: t_mid = (n + 1/2) dt,
    // 3 i + 2: t_mid + dt/2. All threads share the work; a thread evaluates at most a few entries.
    auto fill_table = [&](int b) {
        for (int idx = tid; idx < T::TS * P; idx += T::THREADS) {
            const int slot = idx / P, pp = idx - slot * P;
            const int n = b * T::KB + slot / 3, kind = slot % 3;
            double t;
            if (kind == 0)
                t = (n == 0) ? d.t_in + 0.0 : d.t_in + ((((double)(n - 1) + 0.5) * dt) + dt2d);
            else if (kind == 1)
                t = d.t_in + ((double)n + 0.5) * dt;
            else
                t = d.t_in + ((((double)n + 0.5) * dt) + dt2d);
            int64_t lq = tile * P + pp;
            if (lq >= d.point_count) lq = d.point_count - 1;
            const int64_t gq = d.point_begin + lq;
            const int qx = (int)(gq / d.num_y);
            const int qy = (int)(gq - (int64_t)qx * d.num_y);
            double Cd[MM::NCONST], c[NC];
#pragma unroll
            for (int i = 0; i < MM::NCONST; ++i) Cd[i] = d.consts ? __ldg(d.consts + i) : 0.0;
            MM::coef(t, __ldg(d.par_x + qx), __ldg(d.par_y + qy), Cd, c);
#pragma unroll
            for (int q = 0; q < MM::NCOEF; ++q) cs[(((b & 1) * T::TS + slot) * P + pp) * NC + q] = (float)c[q];
        }
    };

    // stage input u = y + s k -> A (2^12 u as hi / lo FP16 parts, one column per row); populations ->
    // rdiag[slot]; in a cluster also into the partner's exchange buffer (its rows of A are this CTA's rows)
    const float2 a_scale = make_float2((float)(1 << T::A_SCALE_EXP), (float)(1 << T::A_SCALE_EXP));
    const float a_unscale = 1.f / (float)(1 << T::A_SCALE_EXP);
    auto write_stage = [&](float s, const float2 (&k)[E], int slot) {
        float hv[E], lv[E];
        const float2 s2 = make_float2(s, s);
        float2 prev = make_float2(0.f, 0.f);  // the previous row's stage input
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const float2 u = f2_fma(s2, k[e], y[e]);
            uint32_t hb, lb;
            split_f16(gq::f2_mul(u, a_scale), hb, lb);
            hv[e] = __uint_as_float(hb);
            lv[e] = __uint_as_float(lb);
            if (n0 + e == j) rdiag[slot * P * N + p * N + j] = u.x;
            if constexpr (T::CL > 1) {  // rows e - 1, e as one 16-byte remote store
                if (e & 1)
                    gqtc::st_async_v4(gqtc::cluster_peer_u32(xbuf, peer) +
                                          (uint32_t)((((p * H + hh) * (E / 2) + e / 2) * N + j) * 16),
                                      prev.x, prev.y, u.x, u.y, gqtc::cluster_peer_u32(xbar, peer));
            }
            prev = u;
        }
        gqtc::tmem_st<E>(t_ahi + n0, hv);
        gqtc::tmem_st<E>(t_alo + n0, lv);
    };

    uint32_t phase = 0, xphase = 0, kphase = 0;
    bool failed = false;    // the tile's results are lost (uniform over the CTA)
    bool mma_lost = false;  // an MMA wait gave up: that MMA may still be in flight
    bool dead = false;      // an exchange wait gave up: no more waits (cluster CTAs)
    // Waits (one thread, bounded) until the partner's bytes of this phase are in (expecting `bytes`).
    auto exchange_wait = [&](uint64_t* xb, uint32_t& ph, uint32_t bytes) {
        bool ok = true;
        if (tid == 0 && !dead) {
            gqtc::mbar_arrive_expect_tx(xb, bytes);
            ok = gqtc::mbar_wait_bounded(xb, ph, kMaxPolls);
        }
        if (__syncthreads_or(!ok)) {
            dead = true;
            failed = true;
        }
        ph ^= 1u;
    };
    // k = f(u) for the stage input in A with the coefficients of table entry v; false when the MMA wait
    // gave up (one CTA; uniform over it). While the MMA runs, the threads fill the coefficient table of
    // block `fill` (if >= 0).
    auto eval = [&](float2 (&k)[E], int slot, int v, int fill) -> bool {
        if constexpr (T::CL > 1) {
            exchange_wait(xbar, xphase, (uint32_t)T::X_BYTES);  // the partner's half of the stage input
            const int mb = (crank ^ 1) * NH + hh * E;
            const float4* xs = reinterpret_cast<const float4*>(xbuf) + (p * H + hh) * (E / 2) * N + j;
            float hv[E], lv[E];  // rows mb .. mb + E - 1, split as in write_stage
#pragma unroll
            for (int e2 = 0; e2 < E / 2; ++e2) {
                const float4 u = xs[e2 * N];
                const float2 u0 = make_float2(u.x, u.y), u1 = make_float2(u.z, u.w);
                uint32_t h0, l0, h1, l1;
                split_f16(gq::f2_mul(u0, a_scale), h0, l0);
                split_f16(gq::f2_mul(u1, a_scale), h1, l1);
                hv[2 * e2] = __uint_as_float(h0);
                hv[2 * e2 + 1] = __uint_as_float(h1);
                lv[2 * e2] = __uint_as_float(l0);
                lv[2 * e2 + 1] = __uint_as_float(l1);
                if (mb + 2 * e2 == j) rdiag[slot * P * N + p * N + j] = u0.x;
                if (mb + 2 * e2 + 1 == j) rdiag[slot * P * N + p * N + j] = u1.x;
            }
            gqtc::tmem_st<E>(t_ahi + mb, hv);
            gqtc::tmem_st<E>(t_alo + mb, lv);
        }
        gqtc::tmem_wait_st();
        gqtc::fence_before_sync();
        __syncthreads();  // stage input complete in A; coefficients and populations written
        if (tid == 0 && !failed) {
            gqtc::fence_after_sync();
#pragma unroll
            for (int kc = 0; kc < T::KCH; ++kc) {
                const uint64_t dh = bdesc0 + (uint64_t)((kc * T::KSTEP_BYTES) >> 4);
                const uint64_t dl = dh + (uint64_t)((T::NMMA * 32) >> 4);
                // K step kc: rows m = 8 kc .. 8 kc + 7 of the stage input, 8 columns of A
                gqtc::mma_f16_ts(tbase + T::COL_D, tbase + T::COL_AHI + 8 * kc, dh, idesc, kc > 0 ? 1u : 0u);
                gqtc::mma_f16_ts(tbase + T::COL_D, tbase + T::COL_AHI + 8 * kc, dl, idesc, 1u);
                gqtc::mma_f16_ts(tbase + T::COL_D, tbase + T::COL_ALO + 8 * kc, dh, idesc, 1u);
            }
            gqtc::mma_commit(bar);
        }
        if (fill >= 0) fill_table(fill);  // the other buffer was last read a block ago
        float cq[T::NT];  // the point's coefficients of the operator terms (c_0 = 1)
        cq[0] = 1.f;
#pragma unroll
        for (int q = 1; q < T::NT; ++q) cq[q] = cs[(v * P + p) * NC + (q - 1)];
        // While the MMA runs: what needs no MMA result. The jump terms from populations (those of the
        // stage input are in rdiag since the barrier above) and the diagonal terms' coefficients.
        float jre = 0.f, jim = 0.f;
        if constexpr (kJumpsEarly) {
            // Every entry of the padded list (padding: weight 0, population 0), unrolled, so that all
            // loads issue at once: the thread that issued the MMAs polls for them right after this.
#pragma unroll
            for (int q = 0; q < MM::TCJ_MAX; ++q) {
                const int idx = jl * MM::TCJ_MAX + q;
                const int rate = __ldg(MM::tcj_rate() + idx);
                const Cx<float> w = ldc(MM::tcj_coef(), idx);
                const float cr = (rate >= 0) ? cs[(v * P + p) * NC + (rate >= 0 ? rate : 0)] : 1.f;
                const float x = rdiag[slot * P * N + p * N + __ldg(MM::tcj_a() + idx)];
                jre = fmaf(w.re * cr, x, jre);
                jim = fmaf(w.im * cr, x, jim);
            }
        }
        if constexpr (T::NGM < MM::NG) {  // every point's sum_g c_g v_g[n], read after the barrier below
            for (int idx = tid; idx < P * N; idx += T::THREADS) {
                const int pp = idx / N, n = idx - pp * N;
                Cx<float> dv = {0.f, 0.f};
#pragma unroll
                for (int g = 0; g < MM::NG; ++g) {
                    const Cx<float> vg = ldc(MM::diag(g), n);
                    const float cg = cs[(v * P + pp) * NC + MM::ND + g];
                    dv.re = fmaf(cg, vg.re, dv.re);
                    dv.im = fmaf(cg, vg.im, dv.im);
                }
                dvs[idx] = dv;
            }
        }
        // One CTA per tile: every thread waits for the MMA itself (bounded), so each warp starts its
        // epilogue as soon as the MMA has completed; a give-up is made uniform over the warp at once (the
        // tensor-memory loads below are warp-aligned) and over the CTA at the K barrier. In a cluster one
        // thread polls and the CTA meets at a barrier.
        const bool ok = (T::CL == 1 || tid == 0) ? (failed || gqtc::mbar_wait_bounded(bar, phase, kMaxPolls)) : true;
        const bool bad = T::CL == 1 ? __any_sync(0xffffffffu, !ok) : __syncthreads_or(!ok);
        if constexpr (T::CL == 1 && T::NGM < MM::NG) __syncthreads();  // every point's dvs written
        if (bad) {
            failed = true;
            mma_lost = true;
        }
        float2 W[E];  // (Im, Re) of K[n][j] = sum_q c_q (T_q rho)[n][j] for the thread's rows n
        float2 U[E];  // (Re, Im) of the stage input u[n][j], where a term needs it
#pragma unroll
        for (int e = 0; e < E; ++e) W[e] = U[e] = make_float2(0.f, 0.f);
        if (!failed) {  // (a cluster CTA that gave up sends zeros)
            phase ^= 1u;
            gqtc::fence_after_sync();
#pragma unroll
            for (int q = 0; q < T::NT; ++q) {
                float dq[2 * E];
                gqtc::tmem_ld<2 * E>(t_d + 2 * (q * NH + (n0 - nb)), dq);
                gqtc::tmem_wait_ld();
                const float cu = cq[q] * unscale[q];  // D_q is 2^(A scale + term scale) T_q u
                const float2 c2 = make_float2(cu, cu);
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const float2 d2 = make_float2(dq[2 * e], dq[2 * e + 1]);
                    W[e] = (q == 0) ? gq::f2_mul(c2, d2) : f2_fma(c2, d2, W[e]);
                }
            }
            if constexpr (MM::kOwnTerms || (T::NGM < MM::NG)) {  // terms that need the stage input itself
                float a[E], b[E];
                gqtc::tmem_ld<E>(t_ahi + n0, a);
                gqtc::tmem_ld<E>(t_alo + n0, b);
                gqtc::tmem_wait_ld();
#pragma unroll
                for (int e = 0; e < E; ++e) U[e] = join_f16(__float_as_uint(a[e]), __float_as_uint(b[e]), a_unscale);
            }
            if constexpr (T::NGM < MM::NG) {  // diagonal terms in the epilogue: K += (sum_g c_g v_g[n]) u[n][j]
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const Cx<float> dv = dvs[p * N + n0 + e];
                    // Re K += dv.re ur - dv.im ui, Im K += dv.re ui + dv.im ur (the dv.im products first)
                    W[e] = f2_fma(make_float2(dv.im, -dv.im), U[e], W[e]);
                    W[e] = f2_fma(make_float2(dv.re, dv.re), make_float2(U[e].y, U[e].x), W[e]);
                }
            }
        }  // !failed
        {
            // K[n][j] for the rows n of this thread goes to the CTA that reads row j of K transposed
            // (16-byte stores: LDK even, n0 a multiple of 8)
            const int kdst = j / NH;
            const int kidx = (p * NH + (j - kdst * NH)) * LDK + n0;
            if (T::CL > 1 && kdst != crank) {
                const uint32_t ka = gqtc::cluster_peer_u32(kbuf, peer) + (uint32_t)kidx * 8u;
                const uint32_t kb = gqtc::cluster_peer_u32(kbar, peer);
#pragma unroll
                for (int e = 0; e < E; e += 2)
                    gqtc::st_async_v4(ka + 8u * e, W[e].x, W[e].y, W[e + 1].x, W[e + 1].y, kb);
            } else {
                float4* const kb = reinterpret_cast<float4*>(kbuf + kidx);
#pragma unroll
                for (int e = 0; e < E; e += 2) kb[e / 2] = make_float4(W[e].x, W[e].y, W[e + 1].x, W[e + 1].y);
            }
        }
        if constexpr (T::CL > 1) {
            exchange_wait(kbar, kphase, T::KX_BYTES);  // the partner's K entries; this CTA's own ones
        } else {
            if (__syncthreads_or(bad)) return false;  // K complete (or an MMA wait gave up in some warp)
        }
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const float2 kt = kbuf[(p * NH + (n0 - nb + e)) * LDK + j];  // (Im, Re) of K[j][n], n = n0 + e
            // -i (K[n][j] - conj(K[j][n])) = (Im K[n][j] + Im K[j][n], Re K[j][n] - Re K[n][j])
            k[e] = f2_fma(W[e], make_float2(1.f, -1.f), kt);
        }
        // the other jump terms of this thread: population rho_aa of the stage input, or the element
        // itself, into row e
        for (int q = 0; q < (kJumpsEarly ? 0 : jcount); ++q) {
            const int idx = jl * MM::TCJ_MAX + q;
            const int rate = __ldg(MM::tcj_rate() + idx);
            Cx<float> w = ldc(MM::tcj_coef(), idx);
            if (rate >= 0) {
                const float cr = cs[(v * P + p) * NC + rate];
                w.re *= cr;
                w.im *= cr;
            }
            const int a = __ldg(MM::tcj_a() + idx);
            const int e = __ldg(MM::tcj_e() + idx);
            const float x = (a >= 0) ? rdiag[slot * P * N + p * N + a] : 0.f;
#pragma unroll
            for (int ee = 0; ee < E; ++ee)
                if (ee == e) {
                    float2 src = make_float2(x, 0.f);  // a population, or the element itself (a < 0)
                    if constexpr (MM::kOwnTerms) {
                        if (a < 0) src = U[ee];
                    }
                    // Re k += w.re src.re - w.im src.im, Im k += w.re src.im + w.im src.re (w.im first)
                    k[ee] = f2_fma(make_float2(-w.im, w.im), make_float2(src.y, src.x), k[ee]);
                    k[ee] = f2_fma(make_float2(w.re, w.re), src, k[ee]);
                }
        }
        if constexpr (MM::kJumpsOnDiagonal) {
            const float2 jv = make_float2(jre, jim);
#pragma unroll
            for (int e = 0; e < E; ++e)
                if (n0 + e == j) k[e] = f2_add(k[e], jv);
        }
        return true;
    };

    const float h = (float)dt, h2 = (float)dt2d;
    const Coef<float> h6 = Coef<float>::make(dt / 6.0);
    const float2 h6_hi = make_float2(h6.hi, h6.hi), h6_lo = make_float2(h6.lo, h6.lo);
    double osum_re = 0.0, osum_im = 0.0;
    // Sum of (re, im) over the threads of point p, valid in its lead thread (of cluster rank 0): over
    // the point's columns in a warp (lanes p*N .. of at most 32), then over the row blocks and warps
    // through shared memory, then over the cluster. Uniform over the CTA (the cluster); the barrier
    // in front keeps a previous call's reads of the sums apart from this call's writes.
    auto point_sum = [&](double& re, double& im) {
        if constexpr (T::CL > 1) {
            gqtc::cluster_sync();
        } else {
            __syncthreads();
        }
        constexpr int W = N < 32 ? N : 32;  // columns of the point in one warp
#pragma unroll
        for (int off = W / 2; off > 0; off >>= 1) {
            re += __shfl_xor_sync(0xffffffffu, re, off);
            im += __shfl_xor_sync(0xffffffffu, im, off);
        }
        constexpr int NR = T::H * T::CG;  // partial sums of a point: row blocks x warps of columns
        if (j % W == 0) {
            red[(0 * NR + hh * T::CG + j / W) * P + p] = re;
            red[(1 * NR + hh * T::CG + j / W) * P + p] = im;
        }
        __syncthreads();
        if (lead) {
            re = im = 0.0;
            for (int g = 0; g < NR; ++g) {
                re += red[(0 * NR + g) * P + p];
                im += red[(1 * NR + g) * P + p];
            }
        }
        if constexpr (T::CL > 1) {
            constexpr int PS = 2 * T::H * T::CG * P;  // the partner's sums
            if (lead && crank == 1) {
                double* const red_peer = gqtc::cluster_peer(red, peer);
                red_peer[PS + 2 * p] = re;
                red_peer[PS + 2 * p + 1] = im;
            }
            gqtc::cluster_sync();
            if (lead && crank == 0) {
                re += red[PS + 2 * p];
                im += red[PS + 2 * p + 1];
            }
        }
    };
    int next_sample = d.trace_offset, sample = 0;  // observable trace, as the Recorder of gqfixed
    auto observe = [&]() {
        if constexpr (MM::kObsDiagonal) {
            // A diagonal observable: only the thread holding its column's diagonal element has a nonzero
            // entry (the others would add exact zeros); it picks that element as the sum of the rows
            // weighted 1 (that row) and 0 (the others), which reproduces it exactly and needs no
            // indexed access to the state, and adds one product, the general loop's operations on it.
            if (n0 <= j && j < n0 + E) {
                float2 yd = make_float2(0.f, 0.f);
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const float w = (j - n0 == e) ? 1.f : 0.f;
                    yd = f2_fma(make_float2(w, w), y[e], yd);
                }
                const Cx<double> o = ldc(MM::obs_t(), j * N + j);
                const double xr = (double)yd.x, xi = (double)yd.y;
                osum_re = fma(o.re, xr, fma(-o.im, xi, osum_re));
                osum_im = fma(o.re, xi, fma(o.im, xr, osum_im));
            }
        } else {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const Cx<double> o = ldc(MM::obs_t(), (n0 + e) * N + j);
                const double xr = (double)y[e].x, xi = (double)y[e].y;
                osum_re = fma(o.re, xr, fma(-o.im, xi, osum_re));
                osum_im = fma(o.re, xi, fma(o.im, xr, osum_im));
            }
        }
    };

    // Evaluations it = 4 n + s (step n, stage s). Stage times: s = 0 at the previous step's end
    // (t_in + 0 for n = 0), s = 1, 2 at t_mid = (n + 1/2) dt, s = 3 at t_mid + dt/2 - the times and
    // roundings of gqfixed::RK4, whose coefficients come from the table (block step / KB). The next
    // block's table is filled during the MMA of stage 1 of a block's last step.
    {
        float2 k[E];
#pragma unroll
        for (int e = 0; e < E; ++e) k[e] = make_float2(0.f, 0.f);
        fill_table(0);
        write_stage(0.f, k, 0);
        const int total = 4 * d.num_steps;
        for (int it = 0; it < total; ++it) {
            const int step = it >> 2, s = it & 3;
            const int sb = step % T::KB;
            const int ver = ((step / T::KB) & 1) * T::TS + 3 * sb + (s == 0 ? 0 : (s == 3 ? 2 : 1));
            const int fill = (s == 1 && sb == T::KB - 1) ? step / T::KB + 1 : -1;
            if (!eval(k, it & 1, ver, fill)) {  // (a single CTA only)
                failed = true;
                mma_lost = true;
                break;
            }
            const int nslot = (it + 1) & 1;
            if (s == 3) {
#pragma unroll
                for (int e = 0; e < E; ++e) {  // FormFP32::accumulate on both parts
                    acc[e] = f2_add(acc[e], k[e]);
                    gq::f2_kahan(y[e], cn[e], acc[e], h6_hi, h6_lo);
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
                        if (lead && active && crank == 0 && sample < d.num_trace) {
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
                for (int e = 0; e < E; ++e) k[e] = make_float2(0.f, 0.f);
                write_stage(0.f, k, nslot);  // input of the next step's k1 (same time)
            } else {
                if (s == 0) {
#pragma unroll
                    for (int e = 0; e < E; ++e) acc[e] = k[e];
                } else {
#pragma unroll
                    for (int e = 0; e < E; ++e) acc[e] = f2_fma(make_float2(2.f, 2.f), k[e], acc[e]);
                }
                write_stage(s == 2 ? h : h2, k, nslot);
            }
        }
    }

    if constexpr (T::CL > 1) {  // a failure of either CTA fails the tile (one cluster barrier, both CTAs)
        if (tid == 0 && failed) *gqtc::cluster_peer(fail_flag, peer) = 1u;
        gqtc::cluster_sync();
        if (*reinterpret_cast<volatile uint32_t*>(fail_flag) != 0u) failed = true;
    }
    float* out = static_cast<float*>(d.results);
    if (failed) {
        // an MMA that did not signal: wait once more for it (bounded); mark the tile's outputs
        if (mma_lost && tid == 0) gqtc::mbar_wait_bounded(bar, phase, kDrainPolls);
        if (active && lead && crank == 0) {
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
                    dst[n] = y[e].x;
                } else if (n < j && j < NO) {
                    const int slot = NO - 1 + 2 * (n * NO - (n * (n + 1)) / 2 + (j - n - 1));
                    dst[slot] = y[e].x;
                    dst[slot + 1] = y[e].y;
                }
            }
        }
    } else {
        if constexpr (OUT == GQIS_OUT_FINAL) observe();
        point_sum(osum_re, osum_im);
        if (lead && active && crank == 0) {
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
    if constexpr (T::CL > 1) gqtc::cluster_sync();  // no access to the partner's memory after this
    if (warp == 0) {
        gqtc::fence_after_sync();
        gqtc::tmem_dealloc(tbase, T::TMEM_COLS);
    }
}

}  // namespace gqmatrix_tc
