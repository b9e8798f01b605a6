// build_device.cuh -- the per-tile banded solve shared by the builder kernel and the fused
// builder + evaluator kernel.
//
// A thread block owns a tile of TL batch lines and keeps the whole right-hand side of those lines
// in shared memory (rows x TL doubles, lines contiguous), so each sample is read from HBM once and
// each coefficient written once. The rows are brought in with asynchronous global->shared copies
// (cp.async), all in flight at once. Inside the tile every line is cut into NC chunks; a
// (line, chunk) thread runs the banded LU sweeps of its chunk. The dependence between chunks is a
// short carry vector (kl values forward, ku values backward) that is linear in the chunk's incoming
// carry with a transfer matrix fixed by the factors (precomputed on the host), so each sweep runs
// in three phases:
//   A: every chunk sweeps with a zero incoming carry and records its outgoing carry;
//   B: a log-depth scan over the chunks chains the carries through products of transfer matrices;
//   C: every chunk sweeps again from its true carry and writes its rows.
// Periodic systems add a border of k rows/cols (Schur complement; the 2x2 block solve of
// splines_linear_problem_2x2_blocks.cpp:274-298) applied in shared memory.
#pragma once

#include <type_traits>

#include "check_bounds.cuh"
#include "ddcb_internal.hpp"

namespace ddcb {

struct BuildArgs
{
    SolveTables t;
    RhsMap r;
    int raw;            // 1: plain multi-RHS solve (rows in = rows out, no rotation)
    int64_t nlines;
    const double* vals;
    Lines lv;
    const double* dlo;
    Lines llo;
    const double* dhi;
    Lines lhi;
    double* out;
    Lines lo;
    int nct;            // chunk threads per line (block = TL * nct)
    int pair16;         // vals: adjacent line pairs are 16-byte aligned and contiguous
    int pair16_out;     // out: the same for the coefficient output
    int64_t line_base;  // first line of the block's tile; < 0: blockIdx.x * TL
};

// First line of the block's tile.
template <int TL>
__device__ __forceinline__ int64_t tile_line0(BuildArgs const& args)
{
    return args.line_base >= 0 ? args.line_base : (int64_t)blockIdx.x * TL;
}


__device__ __forceinline__ int64_t line_offset(Lines const& L, int64_t b)
{
    return (b / L.inner) * L.outer_stride + (b % L.inner);
}

__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gmem_src)
{
    unsigned const s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem_src) : "memory");
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src)
{
    unsigned const s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }


__device__ __forceinline__ double2 fma2(double a, double2 y, double2 w)
{
    return make_double2(fma(a, y.x, w.x), fma(a, y.y, w.y));
}
__device__ __forceinline__ float2 fma2(float a, float2 y, float2 w) { return make_float2(fmaf(a, y.x, w.x), fmaf(a, y.y, w.y)); }
__device__ __forceinline__ double2 mul2(double2 v, double d) { return make_double2(v.x * d, v.y * d); }
__device__ __forceinline__ float2 mul2(float2 v, float d) { return make_float2(v.x * d, v.y * d); }
__device__ __forceinline__ double2 add2(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 sub2(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// the same on a single line (a tile of one line: no partner)
__device__ __forceinline__ double fma2(double a, double y, double w) { return fma(a, y, w); }
__device__ __forceinline__ float fma2(float a, float y, float w) { return fmaf(a, y, w); }
__device__ __forceinline__ double mul2(double v, double d) { return v * d; }
__device__ __forceinline__ float mul2(float v, float d) { return v * d; }
__device__ __forceinline__ double add2(double a, double b) { return a + b; }
__device__ __forceinline__ float add2(float a, float b) { return a + b; }
__device__ __forceinline__ double sub2(double a, double b) { return a - b; }
__device__ __forceinline__ float sub2(float a, float b) { return a - b; }

// The factor tables in the arithmetic type R of a solve: the FP64 tables, or their FP32 copies
// (the FP32 solves of the refinement mode).
template <class R>
struct Fac;
template <>
struct Fac<double>
{
    using V = double2;
    __device__ static V zero() { return make_double2(0.0, 0.0); }
    __device__ static const double* Lf(SolveTables const& t) { return t.Lf; }
    __device__ static const double* Uf(SolveTables const& t) { return t.Uf; }
    __device__ static const double* PhiF(SolveTables const& t) { return t.PhiF; }
    __device__ static const double* PhiB(SolveTables const& t) { return t.PhiB; }
    __device__ static const double* lam(SolveTables const& t) { return t.lam_val; }
    __device__ static const double* Sinv(SolveTables const& t) { return t.Sinv; }
    __device__ static const double* Qg(SolveTables const& t) { return t.Qg; }
};
template <>
struct Fac<float>
{
    using V = float2;
    __device__ static V zero() { return make_float2(0.f, 0.f); }
    __device__ static const float* Lf(SolveTables const& t) { return t.f32.Lf; }
    __device__ static const float* Uf(SolveTables const& t) { return t.f32.Uf; }
    __device__ static const float* PhiF(SolveTables const& t) { return t.f32.PhiF; }
    __device__ static const float* PhiB(SolveTables const& t) { return t.f32.PhiB; }
    __device__ static const float* lam(SolveTables const& t) { return t.f32.lam_val; }
    __device__ static const float* Sinv(SolveTables const& t) { return t.f32.Sinv; }
    __device__ static const float* Qg(SolveTables const& t) { return t.f32.Qg; }
};

// What a thread's chunk works on: a pair of lines (V = Fac<R>::V, 2 lanes), or the one line of a
// single-line tile (V = R).
template <class R, int TL>
using Lanes = typename std::conditional<TL % 2 == 0, typename Fac<R>::V, R>::type;
template <class V>
__device__ __forceinline__ V zero_of() { return V {}; }

// Forward sweep with L (and the row interchanges when PIV) over rows [a, e) (chunk c) of a line
// pair (or of the single line); T2 points at the pair's column (row j at T2[j*P]). w[0..KL-1] hold rows a..a+KL-1 on
// entry. Phase A (WRITE false) reads rows beyond e from the tile, which nothing has written yet.
// Phase C (WRITE true) writes rows a..e-1; without interchanges rows beyond e only feed the next
// chunk's rows, so they are not read; with interchanges they come from the halo copy.
template <class R, class V, int KL, bool PIV, bool WRITE, int UNR>
__device__ __forceinline__ void fwd_sweep(SolveTables const& t, V* T2, int P, int a, int e, int c, V* w, const V* halo,
                                          int hstride)
{
    R const* __restrict__ Lf = Fac<R>::Lf(t);
    int const lim = (WRITE && !PIV) ? e : t.m; // fill rows below lim are read
    int const qs = factor_stride(t);
#pragma unroll UNR
    for (int j = a; j < e; ++j) {
        int const rr = j + KL;
        V fill = zero_of<V>();
        if (rr < e) fill = T2[rr * P];
        else if (rr < lim) fill = (WRITE && PIV) ? halo[(rr - e) * hstride] : T2[rr * P];
        w[KL] = fill;
        if (PIV) {
            int const pv = __ldg(t.piv + piv_index(t, j, a, c));
#pragma unroll
            for (int q = 1; q <= KL; ++q)
                if (pv == q) {
                    V const s = w[0];
                    w[0] = w[q];
                    w[q] = s;
                }
        }
        V const y = w[0];
        if (WRITE) T2[j * P] = y;
        R const* L = Lf + factor_base(t, j, a, c, KL);
#pragma unroll
        for (int q = 1; q <= KL; ++q) w[q] = fma2(-__ldg(L + (q - 1) * qs), y, w[q]);
#pragma unroll
        for (int q = 0; q < KL; ++q) w[q] = w[q + 1];
    }
}

// Backward sweep with U over rows e-1 .. a (chunk c) of a line pair; z[0..KU-1] hold the solution
// rows e .. e+KU-1 (the carry from the chunk below) on entry.
template <class R, class V, int KU, bool WRITE, int UNR>
__device__ __forceinline__ void bwd_sweep(SolveTables const& t, V* T2, int P, int a, int e, int c, V* z)
{
    R const* __restrict__ Uf = Fac<R>::Uf(t);
    int const qs = factor_stride(t);
#pragma unroll UNR
    for (int j = e - 1; j >= a; --j) {
        R const* U = Uf + factor_base(t, j, a, c, KU + 1);
        V s = T2[j * P];
#pragma unroll
        for (int q = 1; q <= KU; ++q) s = fma2(-__ldg(U + q * qs), z[q - 1], s);
        V const x = mul2(s, __ldg(U));
        if (WRITE) T2[j * P] = x;
#pragma unroll
        for (int q = KU - 1; q >= 1; --q) z[q] = z[q - 1];
        z[0] = x;
    }
}

// Log-depth (Kogge-Stone) scan of the chunk carries of a line pair (carry of chunk c, entry q at
// C2[(c*KC + q)*P]). On entry carry[c] holds chunk c's outgoing carry for a zero incoming carry;
// on exit it holds the true outgoing carry. Forward: chunk c's carry flows into c+1,
// out(c) = Phi_c out(c-1) + hat(c); step k adds P(k,c) y(c-2^k). Backward: the carry flows from
// c+1 into c with Q(k,c) y(c+2^k). Every thread of the block takes part in the barriers; threads
// of chunk c < NC do the arithmetic.
template <class R, class V, int K, int KC, bool FWD, bool PRE_OK = true>
__device__ __forceinline__ void carry_scan(const R* __restrict__ Pm, V* C2, int P, int nscan, int NC, int c)
{
    V y[K];
    bool const act = c < NC;
    if (act) {
#pragma unroll
        for (int q = 0; q < K; ++q) y[q] = C2[(c * KC + q) * P];
    }
    for (int k = 0; k < nscan; ++k) {
        int const nb = FWD ? c - (1 << k) : c + (1 << k);
        bool const has = act && (FWD ? nb >= 0 : nb < NC);
        V v[K];
        // the matrix is read before the barrier (its loads overlap the wait) when it is small and
        // the caller can spare the registers
        constexpr bool PRE = PRE_OK && K <= 4;
        R mk[PRE ? K * K : 1];
        if (has) {
            if constexpr (PRE) {
#pragma unroll
                for (int q = 0; q < K * K; ++q) mk[q] = __ldg(Pm + (k * K * K + q) * NC + c);
            }
#pragma unroll
            for (int q = 0; q < K; ++q) v[q] = C2[(nb * KC + q) * P];
        }
        __syncthreads();
        if (has) {
#pragma unroll
            for (int r = 0; r < K; ++r) {
                V s = y[r];
#pragma unroll
                for (int q = 0; q < K; ++q) {
                    R const mrq = PRE ? mk[PRE ? r * K + q : 0] : __ldg(Pm + (k * K * K + r * K + q) * NC + c);
                    s = fma2(mrq, v[q], s);
                }
                y[r] = s;
            }
#pragma unroll
            for (int q = 0; q < K; ++q) C2[(c * KC + q) * P] = y[q];
        }
        __syncthreads();
    }
}

// Shared-memory doubles of one tile: the rows, the carries, the halo rows (row interchanges only)
// and the border scratch.
__host__ __device__ inline size_t tile_doubles(SolveTables const& t, int TL, int KL, int KU)
{
    int const KC = KL > KU ? KL : KU;
    return (size_t)t.n * TL + (size_t)t.nchunk * KC * TL + (t.pivot ? (size_t)t.nchunk * KL * TL : 0) + (size_t)t.k * TL;
}

// Largest tile width in {TL, TL/2, ..., 2} whose shared memory (bytes(width)) fits in the
// device's per-block opt-in limit; TL itself when none does (the launch then reports it).
template <class Bytes>
inline int fit_tile_lines(int TL, Bytes bytes)
{
    int dev = 0, optin = 0;
    DDCB_CUDA_CHECK(cudaGetDevice(&dev));
    DDCB_CUDA_CHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    for (int w = TL; w >= 2; w /= 2)
        if (bytes(w) <= size_t(optin)) return w;
    return TL;
}

// Steps 2-4 of a solve on a tile already in shared memory (T[j*TL + l] = right-hand side row j of
// line l, in the arithmetic type R): forward and backward sweeps, border correction. A thread owns
// one chunk of a pair of lines (paired shared-memory accesses; each factor load serves both
// lines), or of the one line of a TL = 1 tile. The carries, halo and border scratch follow the n
// rows (tile_doubles elements of R in all). On return (after a barrier) T holds the solution.
// Every thread of the block must call it; TL is even or 1, and the block has at least
// nchunk * max(TL / 2, 1) threads.
// UNR0 (0: the default) sets the rows unrolled per sweep step; PRE lets the carry scans load their
// transfer matrices before each barrier (K x K registers more).
template <int TL, int KL, int KU, class R = double, int UNR0 = 0, bool PRE = true>
__device__ __forceinline__ void solve_in_tile(SolveTables const& t, int /*nct*/, R* smem)
{
    static_assert(TL % 2 == 0 || TL == 1, "the solve works on line pairs, or on one line");
    using V = Lanes<R, TL>;
    constexpr int P = TL % 2 == 0 ? TL / 2 : 1;
    constexpr int KC = KL > KU ? KL : KU;
    // rows unrolled per sweep step: 4 by default; a single line pair is not unrolled, which keeps
    // its kernels free of spills
    constexpr int UNR = UNR0 > 0 ? UNR0 : (TL >= 4 ? 4 : 1);
    int const n = t.n, m = t.m, k = t.k;
    int const NC = t.nchunk;
    int const tid = threadIdx.x;
    int const p = tid % P;
    int const c = tid / P;
    int const nthr = blockDim.x / P;                     // threads per pair
    V* const T2 = reinterpret_cast<V*>(smem) + p;        // n rows, stride P
    V* const carry = T2 + (size_t)n * P;                 // NC x KC rows
    V* const halo = carry + (size_t)NC * KC * P;         // NC x KL rows (row interchanges only)
    V* const btmp = halo + (t.pivot ? (size_t)NC * KL * P : 0); // k rows
    V const zero = zero_of<V>();

    int a = 0, e = 0;
    if (c < NC) {
        a = c * t.chunk_len + 2 * max(0, c - t.chunk_split);
        e = (c == NC - 1) ? m : a + t.chunk_len + (c >= t.chunk_split ? 2 : 0);
    }

    // ---- 2. forward sweep with L (and the row interchanges) ----
    if (m > 0) {
        if (c < NC) {
            V w[KL + 1];
#pragma unroll
            for (int q = 0; q < KL; ++q) w[q] = (a + q < m) ? T2[(a + q) * P] : zero;
            if (t.pivot) fwd_sweep<R, V, KL, true, false, UNR>(t, T2, P, a, e, c, w, nullptr, 0);
            else fwd_sweep<R, V, KL, false, false, UNR>(t, T2, P, a, e, c, w, nullptr, 0);
#pragma unroll
            for (int q = 0; q < KL; ++q) {
                V const orig = (e + q < m) ? T2[(e + q) * P] : zero;
                carry[(c * KC + q) * P] = sub2(w[q], orig);
                if (t.pivot) halo[(c * KL + q) * P] = orig;
            }
        }
        __syncthreads();
        carry_scan<R, V, KL, KC, true, PRE>(Fac<R>::PhiF(t), carry, P, t.nscan_f, NC, c);
        if (c < NC) {
            V w[KL + 1];
#pragma unroll
            for (int q = 0; q < KL; ++q) {
                V v = (a + q < m) ? T2[(a + q) * P] : zero;
                if (c > 0 && a + q < m) v = add2(v, carry[((c - 1) * KC + q) * P]);
                w[q] = v;
            }
            if (t.pivot) fwd_sweep<R, V, KL, true, true, UNR>(t, T2, P, a, e, c, w, halo + (size_t)c * KL * P, P);
            else fwd_sweep<R, V, KL, false, true, UNR>(t, T2, P, a, e, c, w, nullptr, 0);
        }
        __syncthreads();

        // ---- 3. backward sweep with U ----
        if (c < NC) {
            V z[KU];
#pragma unroll
            for (int q = 0; q < KU; ++q) z[q] = zero;
            bwd_sweep<R, V, KU, false, UNR>(t, T2, P, a, e, c, z);
#pragma unroll
            for (int q = 0; q < KU; ++q) carry[(c * KC + q) * P] = z[q];
        }
        __syncthreads();
        carry_scan<R, V, KU, KC, false, PRE>(Fac<R>::PhiB(t), carry, P, t.nscan_b, NC, c);
        if (c < NC) {
            V z[KU];
#pragma unroll
            for (int q = 0; q < KU; ++q) z[q] = (c + 1 < NC) ? carry[((c + 1) * KC + q) * P] : zero;
            bwd_sweep<R, V, KU, true, UNR>(t, T2, P, a, e, c, z);
        }
        __syncthreads();
    }

    // ---- 4. border: x2 = S^-1 (b2 - lambda x'), x1 = x' - (Q^-1 gamma) x2 ----
    if (k > 0) {
        R const* lam = Fac<R>::lam(t);
        R const* Sinv = Fac<R>::Sinv(t);
        R const* Qg = Fac<R>::Qg(t);
        for (int r = c; r < k; r += nthr) {
            V s = T2[(m + r) * P];
            int const q1 = __ldg(t.lam_row + r + 1);
            for (int q = __ldg(t.lam_row + r); q < q1; ++q) s = fma2(-__ldg(lam + q), T2[__ldg(t.lam_col + q) * P], s);
            btmp[r * P] = s;
        }
        __syncthreads();
        for (int r = c; r < k; r += nthr) {
            V s = zero;
            for (int q = 0; q < k; ++q) s = fma2(__ldg(Sinv + r * k + q), btmp[q * P], s);
            T2[(m + r) * P] = s;
        }
        __syncthreads();
        int const nq = t.qg_lo + t.qg_hi;
        for (int q = c; q < nq; q += nthr) {
            int const i = q < t.qg_lo ? q : m - t.qg_hi + (q - t.qg_lo);
            V s = T2[i * P];
            for (int r = 0; r < k; ++r) s = fma2(-__ldg(Qg + (size_t)q * k + r), T2[(m + r) * P], s);
            T2[i * P] = s;
        }
        __syncthreads();
    }
}

// Right-hand side value of tile row r of a line (the value the gather below places there): a
// sample, a dx-scaled Hermite derivative, or 0.
__device__ __forceinline__ double rhs_row(BuildArgs const& args, int r, int64_t line)
{
    RhsMap const& R = args.r;
    int const n = args.t.n;
    int const v0 = (args.raw || R.periodic) ? 0 : R.nbe_lo;
    int const v1 = (args.raw || R.periodic) ? n : R.nbe_lo + R.npoints;
    int sr = r + R.lrot;
    sr -= (sr >= n) ? n : 0;
    if (sr >= v0 && sr < v1) return args.vals[(int64_t)DDCB_INDEX(sr - v0, v1 - v0) * args.lv.stride + line_offset(args.lv, line)];
    if (sr < R.nbe_lo) return sr < R.nbv_lo ? args.dlo[sr * args.llo.stride + line_offset(args.llo, line)] * R.dxpow_lo[sr] : 0.0;
    int const i = sr - (n - R.nbe_hi);
    return i < R.nbv_hi ? args.dhi[i * args.lhi.stride + line_offset(args.lhi, line)] * R.dxpow_hi[i] : 0.0;
}

// Step 1 of a build: gather the right-hand side rows of the tile (spline_builder.hpp:952-1052).
// Tile row r holds system row (r + lrot) mod n; values arrive by async copies, Hermite rows are
// scaled by dx^k. Ends with a barrier.
template <int TL>
__device__ __forceinline__ void gather_tile(BuildArgs const& args, double* T)
{
    RhsMap const& R = args.r;
    int const n = args.t.n;
    int const nct = args.nct;
    int const tid = threadIdx.x;
    int const v0 = (args.raw || R.periodic) ? 0 : R.nbe_lo;
    int const v1 = (args.raw || R.periodic) ? n : R.nbe_lo + R.npoints;

    // ---- 1. gather the right-hand side: tile row r holds system row (r + lrot) mod n; values
    //         arrive by async copies, Hermite rows are scaled by dx^k ----
    // Rows that are not samples: dx-scaled Hermite derivatives, or 0.
    auto other_row = [&](int sr, int64_t line) -> double {
        if (sr < R.nbe_lo) return sr < R.nbv_lo ? args.dlo[sr * args.llo.stride + line_offset(args.llo, line)] * R.dxpow_lo[sr] : 0.0;
        int const i = sr - (n - R.nbe_hi);
        return i < R.nbv_hi ? args.dhi[i * args.lhi.stride + line_offset(args.lhi, line)] * R.dxpow_hi[i] : 0.0;
    };
    if (TL % 2 == 0 && args.pair16) {
        // two adjacent lines per 16-byte copy, which bypasses L1 (cp.async.cg) and so leaves the
        // solve tables resident there
        constexpr int HP = TL / 2 > 0 ? TL / 2 : 1; // line pairs of the tile (TL even here)
        int const p = tid % HP;
        int const c2 = tid / HP;
        int64_t const line = tile_line0<TL>(args) + 2 * p;
        bool const live0 = line < args.nlines, live1 = line + 1 < args.nlines;
        int64_t const ov = live0 ? line_offset(args.lv, line) : 0;
        for (int r = c2; r < n; r += 2 * nct) {
            int sr = r + R.lrot;
            sr -= (sr >= n) ? n : 0;
            double* dst = T + r * TL + 2 * p;
            if (sr >= v0 && sr < v1) {
                if (live1) {
                    cp_async16(dst, args.vals + (int64_t)DDCB_INDEX(sr - v0, v1 - v0) * args.lv.stride + ov);
                } else {
                    dst[0] = live0 ? args.vals[(int64_t)(sr - v0) * args.lv.stride + ov] : 0.0;
                    dst[1] = 0.0;
                }
            } else {
                dst[0] = live0 ? other_row(sr, line) : 0.0;
                dst[1] = live1 ? other_row(sr, line + 1) : 0.0;
            }
        }
    } else {
        int const l = tid % TL;
        int const c = tid / TL;
        int64_t const line = tile_line0<TL>(args) + l;
        bool const live = line < args.nlines;
        int64_t const ov = live ? line_offset(args.lv, line) : 0;
        for (int r = c; r < n; r += nct) {
            int sr = r + R.lrot;
            sr -= (sr >= n) ? n : 0;
            if (live && sr >= v0 && sr < v1) cp_async8(T + r * TL + l, args.vals + (int64_t)DDCB_INDEX(sr - v0, v1 - v0) * args.lv.stride + ov);
            else T[r * TL + l] = live && !(sr >= v0 && sr < v1) ? other_row(sr, line) : 0.0;
        }
    }
    cp_async_wait_all();
    __syncthreads();
}

// Steps 1-4 of a build. On return (after a barrier) T[j*TL + l] holds solution column j of line l,
// for j < n.
template <int TL, int KL, int KU, int UNR0 = 0>
__device__ __forceinline__ void solve_tile(BuildArgs const& args, double* smem)
{
    gather_tile<TL>(args, smem);
    solve_in_tile<TL, KL, KU, double, UNR0>(args.t, args.nct, smem);
}

// Tile row holding output row b: the solution of tile column j belongs to B-spline
// (j + srot) mod n (srot combines the periodic offset of spline_builder.hpp:619-658 with the
// rotation of the boundary blocks), and periodic rows n.. repeat rows 0.. (spline_builder.hpp:1073-1100).
__device__ __forceinline__ int coef_row(RhsMap const& R, int n, int b)
{
    int r = (b >= n ? b - n : b) - R.srot;
    r += (r < 0) ? n : 0;
    r -= (r >= n) ? n : 0;
    return r;
}

// Step 5: store the coefficients of the tile (streaming stores: the output is not read again by
// this kernel).
template <int TL>
__device__ __forceinline__ void store_tile(BuildArgs const& args, const double* T)
{
    int const n = args.t.n;
    int const tid = threadIdx.x;
    int const rows = args.raw ? n : args.r.size;
    if (TL % 2 == 0 && args.pair16_out) {
        constexpr int HP = TL / 2 > 0 ? TL / 2 : 1; // line pairs of the tile (TL even here)
        int const p = tid % HP;
        int const c2 = tid / HP;
        int64_t const line = tile_line0<TL>(args) + 2 * p;
        if (line >= args.nlines) return;
        int64_t const oo = line_offset(args.lo, line);
        bool const live1 = line + 1 < args.nlines;
        for (int r = c2; r < rows; r += 2 * args.nct) {
            double2 const v = *reinterpret_cast<const double2*>(T + DDCB_INDEX(coef_row(args.r, n, r), n) * TL + 2 * p);
            double* dst = args.out + r * args.lo.stride + oo;
            if (live1) __stcs(reinterpret_cast<double2*>(dst), v);
            else __stcs(dst, v.x);
        }
        return;
    }
    int const l = tid % TL;
    int const c = tid / TL;
    int64_t const line = tile_line0<TL>(args) + l;
    if (line >= args.nlines) return;
    int64_t const oo = line_offset(args.lo, line);
    for (int r = c; r < rows; r += args.nct) __stcs(args.out + r * args.lo.stride + oo, T[DDCB_INDEX(coef_row(args.r, n, r), n) * TL + l]);
}

} // namespace ddcb
