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
};

__device__ __forceinline__ int64_t line_offset(Lines const& L, int64_t b)
{
    return (b / L.inner) * L.outer_stride + (b % L.inner);
}

__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gmem_src)
{
    unsigned const s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem_src) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Shared-memory doubles of one tile: the rows, the carries, the halo rows and the border scratch.
__host__ __device__ inline size_t tile_doubles(SolveTables const& t, int TL, int KL, int KU)
{
    int const KC = KL > KU ? KL : KU;
    return (size_t)t.n * TL + (size_t)t.nchunk * KC * TL + (size_t)t.nchunk * KL * TL + (size_t)t.k * TL;
}

template <int KL, bool PIV>
__device__ __forceinline__ void fwd_sweep(SolveTables const& t, double* T, int TL, int l, int a, int e, double* w,
                                          bool write, const double* halo, int hstride)
{
    int const m = t.m;
    for (int j = a; j < e; ++j) {
        int const rr = j + KL;
        double fill;
        if (rr < e) fill = T[rr * TL + l];
        else if (rr < m) fill = halo ? halo[(rr - e) * hstride] : T[rr * TL + l];
        else fill = 0.0;
        w[KL] = fill;
        if (PIV) {
            int const p = __ldg(t.piv + j);
#pragma unroll
            for (int q = 1; q <= KL; ++q)
                if (p == q) {
                    double const s = w[0];
                    w[0] = w[q];
                    w[q] = s;
                }
        }
        double const y = w[0];
        if (write) T[j * TL + l] = y;
        double const* L = t.Lf + (size_t)j * KL;
#pragma unroll
        for (int q = 1; q <= KL; ++q) w[q] = fma(-__ldg(L + q - 1), y, w[q]);
#pragma unroll
        for (int q = 0; q < KL; ++q) w[q] = w[q + 1];
    }
}

template <int KU>
__device__ __forceinline__ void bwd_sweep(SolveTables const& t, double* T, int TL, int l, int a, int e, double* z, bool write)
{
    for (int j = e - 1; j >= a; --j) {
        double const* U = t.Uf + (size_t)j * (KU + 1);
        double s = T[j * TL + l];
#pragma unroll
        for (int q = 1; q <= KU; ++q) s = fma(-__ldg(U + q), z[q - 1], s);
        double const x = s * __ldg(U);
        if (write) T[j * TL + l] = x;
#pragma unroll
        for (int q = KU - 1; q >= 1; --q) z[q] = z[q - 1];
        z[0] = x;
    }
}

// Log-depth (Kogge-Stone) scan of the chunk carries. On entry carry[c] holds chunk c's outgoing
// carry for a zero incoming carry; on exit it holds the true outgoing carry. Forward: chunk c's
// carry flows into c+1, out(c) = Phi_c out(c-1) + hat(c); step k adds P(k,c) y(c-2^k). Backward:
// the carry flows from c+1 into c with Q(k,c) y(c+2^k). Every thread of the block takes part in the
// barriers; threads of chunk c < NC do the arithmetic.
template <int K, int KC, int TL, bool FWD>
__device__ __forceinline__ void carry_scan(const double* __restrict__ P, double* carry, int nscan, int NC, int c, int l)
{
    double y[K];
    bool const act = c < NC;
    if (act) {
#pragma unroll
        for (int q = 0; q < K; ++q) y[q] = carry[(c * KC + q) * TL + l];
    }
    for (int k = 0; k < nscan; ++k) {
        int const nb = FWD ? c - (1 << k) : c + (1 << k);
        bool const has = act && (FWD ? nb >= 0 : nb < NC);
        double v[K];
        if (has) {
#pragma unroll
            for (int q = 0; q < K; ++q) v[q] = carry[(nb * KC + q) * TL + l];
        }
        __syncthreads();
        if (has) {
            double const* M = P + ((size_t)k * NC + c) * K * K;
#pragma unroll
            for (int r = 0; r < K; ++r) {
                double s = y[r];
#pragma unroll
                for (int q = 0; q < K; ++q) s = fma(__ldg(M + r * K + q), v[q], s);
                y[r] = s;
            }
#pragma unroll
            for (int q = 0; q < K; ++q) carry[(c * KC + q) * TL + l] = y[q];
        }
        __syncthreads();
    }
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
    int const l = tid % TL;
    int const c = tid / TL;
    int64_t const line = (int64_t)blockIdx.x * TL + l;
    bool const live = line < args.nlines;

    // ---- 1. gather the right-hand side: tile row r holds system row (r + lrot) mod n; values
    //         arrive by async copies, Hermite rows are scaled by dx^k ----
    {
        int64_t const ov = live ? line_offset(args.lv, line) : 0;
        int const v0 = (args.raw || R.periodic) ? 0 : R.nbe_lo;
        int const v1 = (args.raw || R.periodic) ? n : R.nbe_lo + R.npoints;
        for (int r = c; r < n; r += nct) {
            int sr = r + R.lrot;
            sr -= (sr >= n) ? n : 0;
            if (live && sr >= v0 && sr < v1) {
                cp_async8(T + r * TL + l, args.vals + (int64_t)(sr - v0) * args.lv.stride + ov);
            } else {
                double v = 0.0;
                if (live && sr < R.nbe_lo) {
                    if (sr < R.nbv_lo) v = args.dlo[sr * args.llo.stride + line_offset(args.llo, line)] * R.dxpow_lo[sr];
                } else if (live && sr >= v1) {
                    int const i = sr - (n - R.nbe_hi);
                    if (i < R.nbv_hi) v = args.dhi[i * args.lhi.stride + line_offset(args.lhi, line)] * R.dxpow_hi[i];
                }
                T[r * TL + l] = v;
            }
        }
        cp_async_wait_all();
    }
    __syncthreads();
}

// Steps 2-4 of a solve on a tile already in shared memory (T[j*TL + l] = right-hand side row j of
// line l): forward and backward sweeps, border correction. On return (after a barrier) T holds the
// solution. Every thread of the block must call it.
template <int TL, int KL, int KU>
__device__ __forceinline__ void solve_in_tile(SolveTables const& t, int nct, double* smem)
{
    constexpr int KC = KL > KU ? KL : KU;
    int const n = t.n, m = t.m, k = t.k;
    int const NC = t.nchunk;
    double* T = smem;                              // n x TL
    double* carry = T + (size_t)n * TL;            // NC x KC x TL
    double* halo = carry + (size_t)NC * KC * TL;   // NC x KL x TL
    double* btmp = halo + (size_t)NC * KL * TL;    // k x TL
    int const tid = threadIdx.x;
    int const l = tid % TL;
    int const c = tid / TL;

    int a = 0, e = 0;
    if (c < NC) {
        a = c * t.chunk_len;
        e = (c == NC - 1) ? m : a + t.chunk_len;
    }

    // ---- 2. forward sweep with L (and the row interchanges) ----
    if (m > 0) {
        if (c < NC) {
            double w[KL + 1];
#pragma unroll
            for (int q = 0; q < KL; ++q) w[q] = (a + q < m) ? T[(a + q) * TL + l] : 0.0;
            if (t.pivot) fwd_sweep<KL, true>(t, T, TL, l, a, e, w, false, nullptr, 0);
            else fwd_sweep<KL, false>(t, T, TL, l, a, e, w, false, nullptr, 0);
#pragma unroll
            for (int q = 0; q < KL; ++q) {
                double const orig = (e + q < m) ? T[(e + q) * TL + l] : 0.0;
                carry[(c * KC + q) * TL + l] = w[q] - orig;
                halo[(c * KL + q) * TL + l] = orig;
            }
        }
        __syncthreads();
        carry_scan<KL, KC, TL, true>(t.PhiF, carry, t.nscan, NC, c, l);
        if (c < NC) {
            double w[KL + 1];
#pragma unroll
            for (int q = 0; q < KL; ++q)
                w[q] = (a + q < m) ? T[(a + q) * TL + l] + (c > 0 ? carry[((c - 1) * KC + q) * TL + l] : 0.0) : 0.0;
            if (t.pivot) fwd_sweep<KL, true>(t, T, TL, l, a, e, w, true, halo + (size_t)c * KL * TL + l, TL);
            else fwd_sweep<KL, false>(t, T, TL, l, a, e, w, true, halo + (size_t)c * KL * TL + l, TL);
        }
        __syncthreads();

        // ---- 3. backward sweep with U ----
        if (c < NC) {
            double z[KU];
#pragma unroll
            for (int q = 0; q < KU; ++q) z[q] = 0.0;
            bwd_sweep<KU>(t, T, TL, l, a, e, z, false);
#pragma unroll
            for (int q = 0; q < KU; ++q) carry[(c * KC + q) * TL + l] = z[q];
        }
        __syncthreads();
        carry_scan<KU, KC, TL, false>(t.PhiB, carry, t.nscan, NC, c, l);
        if (c < NC) {
            double z[KU];
#pragma unroll
            for (int q = 0; q < KU; ++q) z[q] = (c + 1 < NC) ? carry[((c + 1) * KC + q) * TL + l] : 0.0;
            bwd_sweep<KU>(t, T, TL, l, a, e, z, true);
        }
        __syncthreads();
    }

    // ---- 4. border: x2 = S^-1 (b2 - lambda x'), x1 = x' - (Q^-1 gamma) x2 ----
    if (k > 0) {
        // border row r is handled by chunk thread r of the line
        for (int r = c; r < k; r += nct) {
            double s = T[(m + r) * TL + l];
            int const q1 = __ldg(t.lam_row + r + 1);
            for (int q = __ldg(t.lam_row + r); q < q1; ++q) s = fma(-__ldg(t.lam_val + q), T[__ldg(t.lam_col + q) * TL + l], s);
            btmp[r * TL + l] = s;
        }
        __syncthreads();
        for (int r = c; r < k; r += nct) {
            double s = 0.0;
            for (int q = 0; q < k; ++q) s = fma(__ldg(t.Sinv + r * k + q), btmp[q * TL + l], s);
            T[(m + r) * TL + l] = s;
        }
        __syncthreads();
        int const nq = t.qg_lo + t.qg_hi;
        for (int q = c; q < nq; q += nct) {
            int const i = q < t.qg_lo ? q : m - t.qg_hi + (q - t.qg_lo);
            double s = T[i * TL + l];
            for (int r = 0; r < k; ++r) s = fma(-__ldg(t.Qg + (size_t)q * k + r), T[(m + r) * TL + l], s);
            T[i * TL + l] = s;
        }
        __syncthreads();
    }
}

// Steps 1-4 of a build. On return (after a barrier) T[j*TL + l] holds solution column j of line l,
// for j < n.
template <int TL, int KL, int KU>
__device__ __forceinline__ void solve_tile(BuildArgs const& args, double* smem)
{
    gather_tile<TL>(args, smem);
    solve_in_tile<TL, KL, KU>(args.t, args.nct, smem);
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

// Step 5: store the coefficients of the tile.
template <int TL>
__device__ __forceinline__ void store_tile(BuildArgs const& args, const double* T)
{
    int const n = args.t.n;
    int const tid = threadIdx.x;
    int const l = tid % TL;
    int const c = tid / TL;
    int64_t const line = (int64_t)blockIdx.x * TL + l;
    if (line >= args.nlines) return;
    int64_t const oo = line_offset(args.lo, line);
    int const rows = args.raw ? n : args.r.size;
    for (int r = c; r < rows; r += args.nct) args.out[r * args.lo.stride + oo] = T[coef_row(args.r, n, r) * TL + l];
}

} // namespace ddcb
