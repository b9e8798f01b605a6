// build_kernels.cu -- batched spline interpolation solve (SplineBuilder::operator(),
// spline_builder.hpp:896-1101) as one kernel per call.
//
// Design (B200): a thread block owns a tile of TL batch lines and keeps the whole right-hand side
// of those lines in shared memory (rows x TL doubles, lines contiguous), so each sample is read
// from HBM once and each coefficient written once. Inside the tile every line is cut into NC
// chunks; a (line, chunk) thread runs the banded LU sweeps of its chunk. The dependence between
// chunks is a short carry vector (kl values forward, ku values backward) that is linear in the
// chunk's incoming carry with a transfer matrix fixed by the factors (precomputed on the host), so
// each sweep runs in three phases:
//   A: every chunk sweeps with a zero incoming carry and records its outgoing carry;
//   B: one thread per line chains the carries through the transfer matrices;
//   C: every chunk sweeps again from its true carry and writes its rows.
// Periodic systems add a border of k rows/cols (Schur complement, 2x2 block solve of
// splines_linear_problem_2x2_blocks.cpp:274-298) applied in shared memory before the coefficients
// are stored with the periodic offset rotation and duplicated rows (spline_builder.hpp:1061-1100).
#include <algorithm>

#include "ddcb_internal.hpp"

namespace ddcb {

namespace {

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
__device__ __forceinline__ void bwd_sweep(SolveTables const& t, double* T, int TL, int l, int a, int e, double* z,
                                          bool write)
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

template <int TL, int KL, int KU>
__global__ void __launch_bounds__(1024) build_kernel(const __grid_constant__ BuildArgs args)
{
    extern __shared__ double smem[];
    SolveTables const& t = args.t;
    RhsMap const& R = args.r;
    constexpr int KC = KL > KU ? KL : KU;
    int const n = t.n, m = t.m, k = t.k;
    int const NC = t.nchunk;
    int const nct = args.nct;
    double* T = smem;                              // n x TL
    double* carry = T + (size_t)n * TL;            // NC x KC x TL
    double* halo = carry + (size_t)NC * KC * TL;   // NC x KL x TL
    double* btmp = halo + (size_t)NC * KL * TL;    // k x TL

    int const tid = threadIdx.x;
    int const l = tid % TL;
    int const c = tid / TL;
    int64_t const line = (int64_t)blockIdx.x * TL + l;
    bool const live = line < args.nlines;

    // ---- 1. gather the right-hand side rows of this tile (spline_builder.hpp:952-1052) ----
    {
        int64_t const ov = live ? line_offset(args.lv, line) : 0;
        int64_t const olo = (live && args.dlo) ? line_offset(args.llo, line) : 0;
        int64_t const ohi = (live && args.dhi) ? line_offset(args.lhi, line) : 0;
        for (int r = c; r < n; r += nct) {
            double v = 0.0;
            if (live) {
                if (args.raw || R.periodic) {
                    v = args.vals[r * args.lv.stride + ov];
                } else if (r < R.nbe_lo) {
                    if (r < R.nbv_lo) v = args.dlo[r * args.llo.stride + olo] * R.dxpow_lo[r];
                } else if (r < R.nbe_lo + R.npoints) {
                    v = args.vals[(int64_t)(r - R.nbe_lo) * args.lv.stride + ov];
                } else {
                    int const i = r - (n - R.nbe_hi);
                    if (i < R.nbv_hi) v = args.dhi[i * args.lhi.stride + ohi] * R.dxpow_hi[i];
                }
            }
            T[r * TL + l] = v;
        }
    }
    __syncthreads();

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
        if (c == 0) {
            double cin[KL];
#pragma unroll
            for (int q = 0; q < KL; ++q) cin[q] = 0.0;
            for (int cc = 0; cc < NC; ++cc) {
                double hat[KL];
#pragma unroll
                for (int q = 0; q < KL; ++q) {
                    hat[q] = carry[(cc * KC + q) * TL + l];
                    carry[(cc * KC + q) * TL + l] = cin[q];
                }
                double const* P = t.PhiF + (size_t)cc * KL * KL;
#pragma unroll
                for (int r = 0; r < KL; ++r) {
                    double s = hat[r];
#pragma unroll
                    for (int q = 0; q < KL; ++q) s = fma(__ldg(P + r * KL + q), cin[q], s);
                    hat[r] = s;
                }
#pragma unroll
                for (int q = 0; q < KL; ++q) cin[q] = hat[q];
            }
        }
        __syncthreads();
        if (c < NC) {
            double w[KL + 1];
#pragma unroll
            for (int q = 0; q < KL; ++q) w[q] = (a + q < m) ? T[(a + q) * TL + l] + carry[(c * KC + q) * TL + l] : 0.0;
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
        if (c == 0) {
            double cin[KU];
#pragma unroll
            for (int q = 0; q < KU; ++q) cin[q] = 0.0;
            for (int cc = NC - 1; cc >= 0; --cc) {
                double hat[KU];
#pragma unroll
                for (int q = 0; q < KU; ++q) {
                    hat[q] = carry[(cc * KC + q) * TL + l];
                    carry[(cc * KC + q) * TL + l] = cin[q];
                }
                double const* P = t.PhiB + (size_t)cc * KU * KU;
#pragma unroll
                for (int r = 0; r < KU; ++r) {
                    double s = hat[r];
#pragma unroll
                    for (int q = 0; q < KU; ++q) s = fma(__ldg(P + r * KU + q), cin[q], s);
                    hat[r] = s;
                }
#pragma unroll
                for (int q = 0; q < KU; ++q) cin[q] = hat[q];
            }
        }
        __syncthreads();
        if (c < NC) {
            double z[KU];
#pragma unroll
            for (int q = 0; q < KU; ++q) z[q] = carry[(c * KC + q) * TL + l];
            bwd_sweep<KU>(t, T, TL, l, a, e, z, true);
        }
        __syncthreads();
    }

    // ---- 4. border: x2 = S^-1 (b2 - lambda x'), x1 = x' - (Q^-1 gamma) x2 ----
    if (k > 0) {
        if (c == 0) {
            for (int r = 0; r < k; ++r) btmp[r * TL + l] = T[(m + r) * TL + l];
            for (int q = 0; q < t.lam_nnz; ++q)
                btmp[__ldg(t.lam_row + q) * TL + l] -= __ldg(t.lam_val + q) * T[__ldg(t.lam_col + q) * TL + l];
            for (int r = 0; r < k; ++r) {
                double s = 0.0;
                for (int q = 0; q < k; ++q) s = fma(__ldg(t.Sinv + r * k + q), btmp[q * TL + l], s);
                T[(m + r) * TL + l] = s;
            }
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

    // ---- 5. store: coefficient row r holds the solution of column ((r mod n) - offset) mod n ----
    if (live) {
        int64_t const oo = line_offset(args.lo, line);
        int const rows = args.raw ? n : R.size;
        for (int r = c; r < rows; r += nct) {
            int src = r;
            if (!args.raw && R.periodic) {
                src = (r % n) - R.offset;
                src = ((src % n) + n) % n;
            }
            args.out[r * args.lo.stride + oo] = T[src * TL + l];
        }
    }
}

size_t smem_bytes(SolveTables const& t, int TL, int KL, int KU)
{
    int const KC = std::max(KL, KU);
    return sizeof(double) * ((size_t)t.n * TL + (size_t)t.nchunk * KC * TL + (size_t)t.nchunk * KL * TL + (size_t)t.k * TL);
}

template <int TL, int KL, int KU>
void launch_tl(BuildArgs const& args, cudaStream_t s)
{
    int const nct = args.nct;
    size_t const sm = smem_bytes(args.t, TL, KL, KU);
    int dev = 0, optin = 0;
    DDCB_CUDA_CHECK(cudaGetDevice(&dev));
    DDCB_CUDA_CHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (sm > size_t(optin))
        throw Error(DDCB_ERR_UNSUPPORTED, "line tile of " + std::to_string(sm) + " bytes exceeds shared memory (" + std::to_string(optin)
                                              + "); use fewer tile lines");
    auto kern = build_kernel<TL, KL, KU>;
    if (sm > 48 * 1024) DDCB_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    int64_t const grid = (args.nlines + TL - 1) / TL;
    kern<<<dim3((unsigned)grid), dim3(TL * nct), sm, s>>>(args);
    DDCB_CUDA_CHECK(cudaGetLastError());
}

template <int KL, int KU>
void launch_k(BuildArgs const& args, int TL, cudaStream_t s)
{
    switch (TL) {
    case 1: launch_tl<1, KL, KU>(args, s); break;
    case 4: launch_tl<4, KL, KU>(args, s); break;
    case 8: launch_tl<8, KL, KU>(args, s); break;
    default: throw Error(DDCB_ERR_UNSUPPORTED, "tile_lines must be 1, 4 or 8");
    }
}

void dispatch(BuildArgs const& args, int TL, cudaStream_t s)
{
    int const kl = args.t.kl, ku = args.t.ku;
    // the plan pads kl/ku up to one of these shapes (plan.cpp: padded_bandwidths)
    if (kl == 1 && ku == 1) launch_k<1, 1>(args, TL, s);
    else if (kl == 1 && ku == 2) launch_k<1, 2>(args, TL, s);
    else if (kl == 1 && ku == 4) launch_k<1, 4>(args, TL, s);
    else if (kl == 2 && ku == 2) launch_k<2, 2>(args, TL, s);
    else if (kl == 2 && ku == 4) launch_k<2, 4>(args, TL, s);
    else if (kl == 4 && ku == 4) launch_k<4, 4>(args, TL, s);
    else if (kl == 4 && ku == 8) launch_k<4, 8>(args, TL, s);
    else throw Error(DDCB_ERR_UNSUPPORTED, "band shape kl=" + std::to_string(kl) + " ku=" + std::to_string(ku) + " has no kernel");
}

int pick_nct(SolveTables const& t, int TL)
{
    // chunk threads per line: enough for the sweeps, a multiple of 32/TL, 128..1024 threads
    int nct = std::max(t.nchunk, 1);
    int const warp_mult = std::max(1, 32 / TL);
    nct = (nct + warp_mult - 1) / warp_mult * warp_mult;
    while (nct * TL < 128) nct += warp_mult;
    while (nct * TL > 1024) nct -= warp_mult;
    return nct;
}

} // namespace

void launch_build(Builder const& b, double* coefs, Lines const& lc, double const* vals, Lines const& lv,
                  double const* dlo, Lines const& llo, double const* dhi, Lines const& lhi, cudaStream_t s)
{
    BuildArgs args {};
    args.t = b.tables;
    args.r = b.rhs;
    args.raw = 0;
    args.nlines = lv.nlines();
    args.vals = vals;
    args.lv = lv;
    args.dlo = dlo;
    args.llo = llo;
    args.dhi = dhi;
    args.lhi = lhi;
    args.out = coefs;
    args.lo = lc;
    args.nct = pick_nct(b.tables, b.tile_lines);
    if (args.nlines == 0) return;
    dispatch(args, b.tile_lines, s);
}

void launch_solve_multirhs(Builder const& b, double* rhs, long ld, long nrhs, bool transpose, cudaStream_t s)
{
    BuildArgs args {};
    args.t = transpose ? b.tables_t : b.tables;
    args.r = b.rhs;
    args.raw = 1;
    args.nlines = nrhs;
    Lines L {b.n, ld, nrhs, 1, 0};
    args.vals = rhs;
    args.lv = L;
    args.out = rhs;
    args.lo = L;
    args.nct = pick_nct(args.t, b.tile_lines);
    if (nrhs == 0) return;
    dispatch(args, b.tile_lines, s);
}

} // namespace ddcb
