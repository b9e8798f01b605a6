// adjoint_kernels.cu -- reverse-mode derivatives of the builder and the evaluator.
//
// The builder is linear in its inputs: coefs = P A^-1 R (vals, dx^k derivs), with R placing the
// samples and the dx-scaled Hermite derivatives into the rows of the system
// (spline_builder.hpp:952-1052), A the collocation matrix and P the periodic offset rotation and
// duplication of the solution (spline_builder.hpp:1061-1100). Its adjoint
//   g_vals = R^T A^-T P^T g_coefs
// folds the cotangents of the duplicated coefficients back onto their originals, solves with A^T
// (the plan's factorisation of the transposed system: the transposed solve of
// splines_linear_problem_2x2_blocks.cpp:292-297 and splines_linear_problem_band.cpp:147-157) and
// hands each tile row back to the sample or the derivative it came from.
//
// The evaluator y = sum_i c[jmin+i] B_i(x) has the adjoint g_c[jmin+i] += g_y B_i(x) and
// g_x = g_y s'(x): a scatter-add of basis-weighted cotangents into a shared-memory tile of the
// line's coefficients, and the spline derivative for the coordinate. Basis values are recomputed
// from the coordinates, never stored by the forward pass.
//
// The fused kernel runs both for the loss of a build + evaluate step: the scattered cotangents land
// directly in the tile of the transposed solve, so neither g_coefs nor the coefficients' tile
// round-trips through HBM.
#include <algorithm>
#include <type_traits>

#include "build_device.cuh"
#include "eval_device.cuh"

namespace ddcb {

namespace {

constexpr int kAdjThreads = 512;

// Cotangent tile rows of B-spline jmin + i: the coefficient row itself (RowsDirect) or the column
// of the solve it came from (RowsRotated, the inverse of coef_row; duplicates fold automatically).
struct RowsDirect
{
    __device__ __forceinline__ int row0(int jmin) const { return jmin; }
    __device__ __forceinline__ int row(int r0, int i) const { return r0 + i; }
};

struct RowsRotated
{
    int n;
    int offset;
    __device__ __forceinline__ int row0(int jmin) const
    {
        int r = jmin - offset;
        r += (r < 0) ? n : 0;
        r -= (r >= n) ? n : 0;
        return r;
    }
    __device__ __forceinline__ int row(int r0, int i) const
    {
        int r = r0 + i;
        return r - ((r >= n) ? n : 0);
    }
};

struct AdjointArgs
{
    SolveTables t;          // factorisation of A^T
    RhsMap r;
    int64_t nlines;
    int nct;
    const double* gc;       // cotangents of the coefficients (size rows)
    Lines lgc;
    double* gv;             // cotangents of the samples (npoints rows)
    Lines lgv;
    double* gdlo;           // cotangents of the lower / upper Hermite derivatives (nbv rows), or NULL
    Lines lglo;
    double* gdhi;
    Lines lghi;
    int pair_in;            // g_coefs: adjacent line pairs 16-byte aligned and contiguous
    int pair_out;           // g_vals: the same
};

// P^T: tile row j (column j of the solve) collects the cotangents of every coefficient row b with
// coef_row(b) = j, i.e. b = (j + srot) mod n, + n, ... below size. The first occurrence of each
// row arrives by async copies (two lines per 16-byte copy where aligned); the few periodic
// duplicates (rows n .. size-1) are added after. Ends with a barrier.
template <int TL>
__device__ __forceinline__ void gather_adjoint(AdjointArgs const& a, double* T)
{
    int const n = a.t.n;
    int const size = a.r.size;
    int const tid = threadIdx.x;
    if (TL % 2 == 0 && a.pair_in) {
        int const p = tid % (TL / 2);
        int const c2 = tid / (TL / 2);
        int const step = blockDim.x / (TL / 2);
        int64_t const line = (int64_t)blockIdx.x * TL + 2 * p;
        bool const live0 = line < a.nlines, live1 = line + 1 < a.nlines;
        int64_t const og = live0 ? line_offset(a.lgc, line) : 0;
        for (int j = c2; j < n; j += step) {
            int b = j + a.r.srot;
            b -= (b >= n) ? n : 0;
            double* dst = T + j * TL + 2 * p;
            if (live1) cp_async16(dst, a.gc + b * a.lgc.stride + og);
            else {
                dst[0] = live0 ? a.gc[b * a.lgc.stride + og] : 0.0;
                dst[1] = 0.0;
            }
        }
    } else {
        int const l = tid % TL;
        int const c = tid / TL;
        int64_t const line = (int64_t)blockIdx.x * TL + l;
        bool const live = line < a.nlines;
        int64_t const og = live ? line_offset(a.lgc, line) : 0;
        for (int j = c; j < n; j += a.nct) {
            int b = j + a.r.srot;
            b -= (b >= n) ? n : 0;
            if (live) cp_async8(T + j * TL + l, a.gc + b * a.lgc.stride + og);
            else T[j * TL + l] = 0.0;
        }
    }
    cp_async_wait_all();
    __syncthreads();
    if (size > n) {
        int const l = tid % TL;
        int const c = tid / TL;
        int64_t const line = (int64_t)blockIdx.x * TL + l;
        if (line < a.nlines) {
            int64_t const og = line_offset(a.lgc, line);
            for (int b = n + c; b < size; b += a.nct) {
                int j = (b - n) - a.r.srot; // row of the first occurrence, b - n
                j += (j < 0) ? n : 0;
                T[j * TL + l] += a.gc[b * a.lgc.stride + og];
            }
        }
        __syncthreads();
    }
}

// R^T: tile row i of the transposed solve is the cotangent of system row (i + lrot) mod n: a
// sample, or a Hermite derivative (times the dx^k the forward pass scaled it by). Samples leave by
// streaming stores, two lines per 16-byte store where aligned.
template <int TL>
__device__ __forceinline__ void store_adjoint(AdjointArgs const& a, const double* T)
{
    RhsMap const& R = a.r;
    int const n = a.t.n;
    int const tid = threadIdx.x;
    int const v0 = R.periodic ? 0 : R.nbe_lo;
    int const v1 = R.periodic ? n : R.nbe_lo + R.npoints;
    if (TL % 2 == 0 && a.pair_out) {
        int const p = tid % (TL / 2);
        int const c2 = tid / (TL / 2);
        int const step = blockDim.x / (TL / 2);
        int64_t const line = (int64_t)blockIdx.x * TL + 2 * p;
        if (line < a.nlines) {
            bool const live1 = line + 1 < a.nlines;
            int64_t const ov = line_offset(a.lgv, line);
            for (int i = c2; i < n; i += step) {
                int sr = i + R.lrot;
                sr -= (sr >= n) ? n : 0;
                if (sr < v0 || sr >= v1) continue;
                double2 const g = *reinterpret_cast<const double2*>(T + i * TL + 2 * p);
                double* dst = a.gv + (int64_t)(sr - v0) * a.lgv.stride + ov;
                if (live1) __stcs(reinterpret_cast<double2*>(dst), g);
                else __stcs(dst, g.x);
            }
        }
    }
    int const l = tid % TL;
    int const c = tid / TL;
    int64_t const line = (int64_t)blockIdx.x * TL + l;
    if (line >= a.nlines) return;
    int64_t const ov = line_offset(a.lgv, line);
    for (int i = c; i < n; i += a.nct) {
        int sr = i + R.lrot;
        sr -= (sr >= n) ? n : 0;
        double const g = T[i * TL + l];
        if (sr >= v0 && sr < v1) {
            if (!(TL % 2 == 0 && a.pair_out)) __stcs(a.gv + (int64_t)(sr - v0) * a.lgv.stride + ov, g);
        } else if (sr < v0) {
            if (sr < R.nbv_lo && a.gdlo) a.gdlo[sr * a.lglo.stride + line_offset(a.lglo, line)] = g * R.dxpow_lo[sr];
        } else {
            int const q = sr - (n - R.nbe_hi);
            if (q < R.nbv_hi && a.gdhi) a.gdhi[q * a.lghi.stride + line_offset(a.lghi, line)] = g * R.dxpow_hi[q];
        }
    }
}

template <int TL, int KL, int KU>
__global__ void __launch_bounds__(1024) build_adjoint_kernel(const __grid_constant__ AdjointArgs a)
{
    extern __shared__ __align__(16) double smem[];
    gather_adjoint<TL>(a, smem);
    solve_in_tile<TL, KL, KU>(a.t, a.nct, smem);
    store_adjoint<TL>(a, smem);
}

struct EvalAdjointArgs
{
    EvalBasis eb;
    int ex_lo, ex_hi;
    int64_t nlines;
    int size;               // coefficient rows
    const double* coords;
    Lines lx;
    const double* coefs;    // needed for g_coords only
    Lines lc;
    int coef_pairs;         // coefs: adjacent line pairs 16-byte aligned and contiguous
    const double* gy;       // cotangents of the evaluated values
    Lines lgy;
    double* gc;             // out: cotangents of the coefficients (standalone kernel)
    Lines lgc;
    double* gx;             // out: cotangents of the coordinates, or NULL
    Lines lgx;
};

// The knot pairs (non-uniform bases) into shared memory, as async copies.
template <bool UNI>
__device__ __forceinline__ void load_knot_pairs(EvalAdjointArgs const& a, double2* K)
{
    if (!UNI)
        for (int i = threadIdx.x; i < a.eb.nk - 1; i += blockDim.x) cp_async16(K + i, a.eb.kpairs + i);
}

// The coefficient tile of the block's TLE lines into C (row r of line l at C[r*TLE + l]), as async
// copies: two lines per 16-byte copy where the layout allows.
template <int TLE>
__device__ __forceinline__ void load_coef_tile(EvalAdjointArgs const& a, double* C)
{
    int const tid = threadIdx.x;
    if (TLE % 2 == 0 && a.coef_pairs) {
        int const p = tid % (TLE / 2);
        int const c2 = tid / (TLE / 2);
        int const step = blockDim.x / (TLE / 2);
        int64_t const l0 = (int64_t)blockIdx.x * TLE + 2 * p;
        if (l0 + 1 < a.nlines) {
            int64_t const oc = line_offset(a.lc, l0);
            for (int r = c2; r < a.size; r += step) cp_async16(C + r * TLE + 2 * p, a.coefs + r * a.lc.stride + oc);
        } else if (l0 < a.nlines) {
            int64_t const oc = line_offset(a.lc, l0);
            for (int r = c2; r < a.size; r += step) cp_async8(C + r * TLE + 2 * p, a.coefs + r * a.lc.stride + oc);
        }
        return;
    }
    int const l = tid % TLE;
    int const c = tid / TLE;
    int const step = blockDim.x / TLE;
    int64_t const line = (int64_t)blockIdx.x * TLE + l;
    if (line >= a.nlines) return;
    int64_t const oc = line_offset(a.lc, line);
    for (int r = c; r < a.size; r += step) cp_async8(C + r * TLE + l, a.coefs + r * a.lc.stride + oc);
}

// dy/dx of one evaluated point: s'(x) for a value (ORDER 0) with the boundary handling of
// eval_value_bc (0 outside the domain, where null and constant extrapolation do not move with x),
// or the next derivative for a derivative (ORDER 1, no boundary handling).
template <int D, int ORDER, bool UNI, class Acc>
__device__ __forceinline__ double point_dydx(EvalBasis const& eb, double x, Acc const& C)
{
    if constexpr (ORDER == 0) {
        if (eb.b.periodic) x = periodic_wrap(eb.b, x);
        else if (x < eb.b.rmin || x > eb.b.rmax) return 0.0;
        return eval_deriv_no_bc<D, 1, UNI>(eb, x, C);
    } else if constexpr (ORDER + 1 <= D) {
        return eval_deriv_no_bc<D, ORDER + 1, UNI>(eb, x, C);
    } else {
        return 0.0;
    }
}

// Phase 1 of an evaluator adjoint: g_x = g_y * dy/dx for the points of the thread's line, with the
// line's coefficients in the shared tile C.
template <int D, int TLE, int ORDER, bool UNI>
__device__ __forceinline__ void coord_cotangents(EvalAdjointArgs const& a, EvalBasis const& eb, const double* C)
{
    int const tid = threadIdx.x;
    int const l = tid % TLE;
    int const c = tid / TLE;
    int const nct = blockDim.x / TLE;
    int64_t const line = (int64_t)blockIdx.x * TLE + l;
    if (line >= a.nlines) return;
    int64_t const ox = line_offset(a.lx, line);
    int64_t const og = line_offset(a.lgy, line);
    int64_t const oxo = line_offset(a.lgx, line);
    CoefDirect const acc {C + l, TLE};
    constexpr int U = 8; // points in flight per thread
    int64_t const m = a.lx.n;
    int const npt = m > c ? int((m - c + nct - 1) / nct) : 0;
    for (int q0 = 0; q0 < npt; q0 += U) {
        double xs[U], gs[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            int64_t const p = c + int64_t(q0 + u) * nct;
            xs[u] = (q0 + u < npt) ? a.coords[p * a.lx.stride + ox] : 0.0;
            gs[u] = (q0 + u < npt) ? a.gy[p * a.lgy.stride + og] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (q0 + u < npt)
                __stcs(a.gx + (c + int64_t(q0 + u) * nct) * a.lgx.stride + oxo, gs[u] * point_dydx<D, ORDER, UNI>(eb, xs[u], acc));
    }
}

// Phase 2: scatter g_y * dy/dc into the cotangent tile G (rows from Rows). The coordinates and
// cotangents are read a second time; the block read them just before, so they come from L2.
template <int D, int TLE, int ORDER, bool UNI, class Rows>
__device__ __forceinline__ void scatter_points(EvalAdjointArgs const& a, EvalBasis const& eb, double* G, Rows const& rows)
{
    int const tid = threadIdx.x;
    int const l = tid % TLE;
    int const c = tid / TLE;
    int const nct = blockDim.x / TLE;
    int64_t const line = (int64_t)blockIdx.x * TLE + l;
    if (line >= a.nlines) return;
    int64_t const ox = line_offset(a.lx, line);
    int64_t const og = line_offset(a.lgy, line);
    CoefDirect const none {nullptr, 0};
    constexpr int U = 8;
    int64_t const m = a.lx.n;
    int const npt = m > c ? int((m - c + nct - 1) / nct) : 0;
    for (int q0 = 0; q0 < npt; q0 += U) {
        double xs[U], gs[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            int64_t const p = c + int64_t(q0 + u) * nct;
            xs[u] = (q0 + u < npt) ? __ldcs(a.coords + p * a.lx.stride + ox) : 0.0;
            gs[u] = (q0 + u < npt) ? __ldcs(a.gy + p * a.lgy.stride + og) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (q0 + u >= npt) continue;
            double w[D + 1], unused;
            int const jmin = point_adjoint<D, ORDER, UNI>(eb, a.ex_lo, a.ex_hi, xs[u], none, false, w, unused);
            if (jmin >= 0) {
                int const r0 = rows.row0(DDCB_INDEX(jmin, eb.b.ncells));
#pragma unroll
                for (int i = 0; i < D + 1; ++i) atomicAdd(G + rows.row(r0, i) * TLE + l, gs[u] * w[i]);
            }
        }
    }
}

// Evaluator adjoint. One shared tile serves twice: first as the coefficient tile for g_x, then as
// the cotangent tile the scatter accumulates into.
template <int D, int TLE, int ORDER, bool UNI>
__global__ void __launch_bounds__(kAdjThreads) eval_adjoint_kernel(const __grid_constant__ EvalAdjointArgs a)
{
    extern __shared__ __align__(16) double smem[];
    double* G = smem;                                                  // size x TLE
    double2* K = reinterpret_cast<double2*>(smem + (((size_t)a.size * TLE + 1) & ~size_t(1)));
    load_knot_pairs<UNI>(a, K);
    if (a.gx) load_coef_tile<TLE>(a, G);
    cp_async_wait_all();
    __syncthreads();
    EvalBasis eb = a.eb;
    if (!UNI) eb.kpairs = K;
    if (a.gx) {
        coord_cotangents<D, TLE, ORDER, UNI>(a, eb, G);
        __syncthreads();
    }
    for (int i = threadIdx.x; i < a.size * TLE; i += blockDim.x) G[i] = 0.0;
    __syncthreads();
    scatter_points<D, TLE, ORDER, UNI>(a, eb, G, RowsDirect {});
    __syncthreads();
    int const l = threadIdx.x % TLE;
    int const c = threadIdx.x / TLE;
    int const nct = blockDim.x / TLE;
    int64_t const line = (int64_t)blockIdx.x * TLE + l;
    if (line >= a.nlines) return;
    int64_t const og = line_offset(a.lgc, line);
    for (int r = c; r < a.size; r += nct) __stcs(a.gc + r * a.lgc.stride + og, G[r * TLE + l]);
}

// Doubles of the fused kernel's shared tile: the solve tile, or the coefficient tile if larger.
__host__ __device__ inline size_t fused_tile_doubles(SolveTables const& t, int size, int TL, int KL, int KU)
{
    size_t const td = tile_doubles(t, TL, KL, KU);
    size_t const tc = (size_t)size * TL;
    return ((td > tc ? td : tc) + 1) & ~size_t(1);
}

// Backward of build + evaluate: g_x from the coefficient tile, then the scatter into the
// transposed solve's tile (the same shared memory), the solve with A^T and the sample cotangents.
template <int TL, int KL, int KU, int D, int ORDER, bool UNI>
__global__ void __launch_bounds__(1024) build_eval_adjoint_kernel(const __grid_constant__ AdjointArgs a,
                                                                  const __grid_constant__ EvalAdjointArgs ea)
{
    extern __shared__ __align__(16) double smem[];
    double* T = smem;
    double2* K = reinterpret_cast<double2*>(smem + fused_tile_doubles(a.t, ea.size, TL, KL, KU));
    load_knot_pairs<UNI>(ea, K);
    if (ea.gx) load_coef_tile<TL>(ea, T);
    cp_async_wait_all();
    __syncthreads();
    EvalBasis eb = ea.eb;
    if (!UNI) eb.kpairs = K;
    if (ea.gx) {
        coord_cotangents<D, TL, ORDER, UNI>(ea, eb, T);
        __syncthreads();
    }
    for (int i = threadIdx.x; i < a.t.n * TL; i += blockDim.x) T[i] = 0.0;
    __syncthreads();
    scatter_points<D, TL, ORDER, UNI>(ea, eb, T, RowsRotated {a.t.n, a.r.srot});
    __syncthreads();
    solve_in_tile<TL, KL, KU>(a.t, a.nct, smem);
    store_adjoint<TL>(a, smem);
}

int adj_nct(SolveTables const& t, int TL, int min_threads)
{
    int nct = std::max(t.nchunk, 1);
    int const warp_mult = std::max(1, 32 / TL);
    nct = (nct + warp_mult - 1) / warp_mult * warp_mult;
    while (nct * TL < min_threads) nct += warp_mult;
    while (nct * TL > 1024) nct -= warp_mult;
    return nct;
}

size_t optin_smem()
{
    int dev = 0, optin = 0;
    DDCB_CUDA_CHECK(cudaGetDevice(&dev));
    DDCB_CUDA_CHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    return size_t(optin);
}

template <class Kern>
void set_smem(Kern k, size_t sm)
{
    if (sm > 48 * 1024) DDCB_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
}

template <int TL, int KL, int KU>
void launch_build_adjoint_tl(AdjointArgs const& a, cudaStream_t s)
{
    size_t const sm = sizeof(double) * tile_doubles(a.t, TL, KL, KU);
    if (sm > optin_smem()) throw Error(DDCB_ERR_UNSUPPORTED, "adjoint line tile exceeds shared memory; use fewer tile lines");
    auto kern = build_adjoint_kernel<TL, KL, KU>;
    set_smem(kern, sm);
    kern<<<dim3((unsigned)((a.nlines + TL - 1) / TL)), dim3(TL * a.nct), sm, s>>>(a);
    DDCB_CUDA_CHECK(cudaGetLastError());
}

template <int KL, int KU>
void launch_build_adjoint_k(AdjointArgs const& a, int TL, cudaStream_t s)
{
    switch (TL) {
    case 2: launch_build_adjoint_tl<2, KL, KU>(a, s); break;
    case 4: launch_build_adjoint_tl<4, KL, KU>(a, s); break;
    case 8: launch_build_adjoint_tl<8, KL, KU>(a, s); break;
    default: throw Error(DDCB_ERR_UNSUPPORTED, "tile_lines must be 2, 4 or 8");
    }
}

void dispatch_build_adjoint(AdjointArgs const& a, int TL, cudaStream_t s)
{
    int const kl = a.t.kl, ku = a.t.ku;
    // the band shapes the plan pads both the system and its transpose to (plan.cpp, HostSolve::analyse)
    if (kl == 1 && ku == 1) launch_build_adjoint_k<1, 1>(a, TL, s);
    else if (kl == 1 && ku == 2) launch_build_adjoint_k<1, 2>(a, TL, s);
    else if (kl == 2 && ku == 2) launch_build_adjoint_k<2, 2>(a, TL, s);
    else if (kl == 3 && ku == 3) launch_build_adjoint_k<3, 3>(a, TL, s);
    else if (kl == 1 && ku == 4) launch_build_adjoint_k<1, 4>(a, TL, s);
    else if (kl == 2 && ku == 4) launch_build_adjoint_k<2, 4>(a, TL, s);
    else if (kl == 4 && ku == 4) launch_build_adjoint_k<4, 4>(a, TL, s);
    else if (kl == 3 && ku == 6) launch_build_adjoint_k<3, 6>(a, TL, s);
    else if (kl == 1 && ku == 8) launch_build_adjoint_k<1, 8>(a, TL, s);
    else if (kl == 2 && ku == 8) launch_build_adjoint_k<2, 8>(a, TL, s);
    else if (kl == 4 && ku == 8) launch_build_adjoint_k<4, 8>(a, TL, s);
    else throw Error(DDCB_ERR_UNSUPPORTED, "band shape kl=" + std::to_string(kl) + " ku=" + std::to_string(ku) + " has no adjoint kernel");
}

AdjointArgs make_adjoint_args(Builder const& b, const double* gc, Lines const& lgc, double* gv, Lines const& lgv,
                              double* gdlo, Lines const& lglo, double* gdhi, Lines const& lghi)
{
    AdjointArgs a {};
    a.t = b.tables_t;
    a.r = b.rhs;
    a.nlines = lgv.nlines();
    a.gc = gc;
    a.lgc = lgc;
    a.gv = gv;
    a.lgv = lgv;
    a.gdlo = gdlo;
    a.lglo = lglo;
    a.gdhi = gdhi;
    a.lghi = lghi;
    a.pair_in = gc != nullptr && line_pairs_aligned(gc, lgc);
    a.pair_out = line_pairs_aligned(gv, lgv);
    return a;
}

EvalAdjointArgs make_eval_adjoint_args(Evaluator const& e, double const* coords, Lines const& lx, double const* coefs,
                                       Lines const& lc, double const* gy, Lines const& lgy, double* gc, Lines const& lgc,
                                       double* gx, Lines const& lgx)
{
    EvalAdjointArgs a {};
    a.eb = e.eb;
    a.ex_lo = e.ex_lo;
    a.ex_hi = e.ex_hi;
    a.nlines = lx.nlines();
    a.size = int(e.basis.size());
    a.coords = coords;
    a.lx = lx;
    a.coefs = coefs;
    a.lc = lc;
    a.coef_pairs = coefs != nullptr && line_pairs_aligned(coefs, lc);
    a.gy = gy;
    a.lgy = lgy;
    a.gc = gc;
    a.lgc = lgc;
    a.gx = gx;
    a.lgx = lgx;
    return a;
}

size_t eval_adjoint_smem(EvalAdjointArgs const& a, int TLE, bool uni)
{
    return sizeof(double) * (((size_t)a.size * TLE + 1) & ~size_t(1)) + (uni ? 0 : sizeof(double2) * (size_t)a.eb.nk);
}

template <int D, int TLE, bool UNI>
void launch_eval_adjoint_d(EvalAdjointArgs const& a, int order, cudaStream_t s)
{
    size_t const sm = eval_adjoint_smem(a, TLE, UNI);
    dim3 grid((unsigned)((a.nlines + TLE - 1) / TLE)), block(kAdjThreads);
    if (order == 0) {
        auto k = eval_adjoint_kernel<D, TLE, 0, UNI>;
        set_smem(k, sm);
        k<<<grid, block, sm, s>>>(a);
    } else {
        auto k = eval_adjoint_kernel<D, TLE, 1, UNI>;
        set_smem(k, sm);
        k<<<grid, block, sm, s>>>(a);
    }
    DDCB_CUDA_CHECK(cudaGetLastError());
}

template <int TLE>
void launch_eval_adjoint_tle(EvalAdjointArgs const& a, int order, cudaStream_t s)
{
    bool const uni = a.eb.b.uniform != 0;
    switch (a.eb.b.degree) {
    case 1: uni ? launch_eval_adjoint_d<1, TLE, true>(a, order, s) : launch_eval_adjoint_d<1, TLE, false>(a, order, s); break;
    case 2: uni ? launch_eval_adjoint_d<2, TLE, true>(a, order, s) : launch_eval_adjoint_d<2, TLE, false>(a, order, s); break;
    case 3: uni ? launch_eval_adjoint_d<3, TLE, true>(a, order, s) : launch_eval_adjoint_d<3, TLE, false>(a, order, s); break;
    case 4: uni ? launch_eval_adjoint_d<4, TLE, true>(a, order, s) : launch_eval_adjoint_d<4, TLE, false>(a, order, s); break;
    case 5: uni ? launch_eval_adjoint_d<5, TLE, true>(a, order, s) : launch_eval_adjoint_d<5, TLE, false>(a, order, s); break;
    default: throw Error(DDCB_ERR_UNSUPPORTED, "degree must be in 1..5");
    }
}

template <int KL, int KU, int D, int ORDER, bool UNI>
bool launch_fused5(AdjointArgs const& a, EvalAdjointArgs const& ea, cudaStream_t s)
{
    constexpr int TL = 8;
    size_t const sm = sizeof(double) * fused_tile_doubles(a.t, ea.size, TL, KL, KU) + (UNI ? 0 : sizeof(double2) * (size_t)ea.eb.nk);
    if (sm > optin_smem()) return false;
    auto kern = build_eval_adjoint_kernel<TL, KL, KU, D, ORDER, UNI>;
    set_smem(kern, sm);
    kern<<<dim3((unsigned)((a.nlines + TL - 1) / TL)), dim3(TL * a.nct), sm, s>>>(a, ea);
    DDCB_CUDA_CHECK(cudaGetLastError());
    return true;
}

template <int KL, int KU, int D>
bool launch_fused_ord(AdjointArgs const& a, EvalAdjointArgs const& ea, int order, cudaStream_t s)
{
    bool const uni = ea.eb.b.uniform != 0;
    if (order == 0) return uni ? launch_fused5<KL, KU, D, 0, true>(a, ea, s) : launch_fused5<KL, KU, D, 0, false>(a, ea, s);
    if (order == 1) return uni ? launch_fused5<KL, KU, D, 1, true>(a, ea, s) : launch_fused5<KL, KU, D, 1, false>(a, ea, s);
    return false;
}

template <int KL, int KU>
bool launch_fused_deg(AdjointArgs const& a, EvalAdjointArgs const& ea, int order, cudaStream_t s)
{
    switch (ea.eb.b.degree) {
    case 1: return launch_fused_ord<KL, KU, 1>(a, ea, order, s);
    case 2: return launch_fused_ord<KL, KU, 2>(a, ea, order, s);
    case 3: return launch_fused_ord<KL, KU, 3>(a, ea, order, s);
    case 4: return launch_fused_ord<KL, KU, 4>(a, ea, order, s);
    case 5: return launch_fused_ord<KL, KU, 5>(a, ea, order, s);
    default: return false;
    }
}

} // namespace

void launch_build_adjoint(Builder const& b, double const* gc, Lines const& lgc, double* gv, Lines const& lgv,
                          double* gdlo, Lines const& lglo, double* gdhi, Lines const& lghi, cudaStream_t s)
{
    AdjointArgs a = make_adjoint_args(b, gc, lgc, gv, lgv, gdlo, lglo, gdhi, lghi);
    if (a.nlines == 0) return;
    int const TL = fit_tile_lines(std::min(b.tile_lines, 8), [&](int w) { return sizeof(double) * tile_doubles(a.t, w, a.t.kl, a.t.ku); });
    a.nct = adj_nct(a.t, TL, 128);
    dispatch_build_adjoint(a, TL, s);
}

void launch_eval_adjoint(Evaluator const& e, int order, double const* coords, Lines const& lx, double const* coefs,
                         Lines const& lc, double const* gy, Lines const& lgy, double* gc, Lines const& lgc, double* gx,
                         Lines const& lgx, cudaStream_t s)
{
    EvalAdjointArgs a = make_eval_adjoint_args(e, coords, lx, coefs, lc, gy, lgy, gc, lgc, gx, lgx);
    if (a.nlines == 0) return;
    // eight lines per block: the shared tile of a 1000-row line takes under a third of an SM
    if (eval_adjoint_smem(a, 8, a.eb.b.uniform != 0) <= optin_smem()) launch_eval_adjoint_tle<8>(a, order, s);
    else if (eval_adjoint_smem(a, 4, a.eb.b.uniform != 0) <= optin_smem()) launch_eval_adjoint_tle<4>(a, order, s);
    else if (eval_adjoint_smem(a, 1, a.eb.b.uniform != 0) <= optin_smem()) launch_eval_adjoint_tle<1>(a, order, s);
    else throw Error(DDCB_ERR_UNSUPPORTED, "coefficient tile of the evaluator adjoint exceeds shared memory");
}

bool launch_build_eval_adjoint(Builder const& b, Evaluator const& e, int order, double const* coords, Lines const& lx,
                               double const* coefs, Lines const& lc, double const* gy, Lines const& lgy, double* gv,
                               Lines const& lgv, double* gdlo, Lines const& lglo, double* gdhi, Lines const& lghi,
                               double* gx, Lines const& lgx, cudaStream_t s)
{
    if (lgv.nlines() == 0) return true;
    bool fused = false;
    if (b.tile_lines == 8) {
        AdjointArgs a = make_adjoint_args(b, nullptr, Lines {}, gv, lgv, gdlo, lglo, gdhi, lghi);
        a.nct = adj_nct(a.t, 8, kAdjThreads);
        EvalAdjointArgs ea = make_eval_adjoint_args(e, coords, lx, coefs, lc, gy, lgy, nullptr, Lines {}, gx, lgx);
        int const kl = a.t.kl, ku = a.t.ku;
        if (kl == 1 && ku == 1) fused = launch_fused_deg<1, 1>(a, ea, order, s);
        else if (kl == 2 && ku == 2) fused = launch_fused_deg<2, 2>(a, ea, order, s);
        else if (kl == 3 && ku == 3) fused = launch_fused_deg<3, 3>(a, ea, order, s);
        else if (kl == 4 && ku == 4) fused = launch_fused_deg<4, 4>(a, ea, order, s);
    }
    if (!fused) {
        // two kernels through a stream-ordered cotangent buffer of the coefficients
        int64_t const nl = lgv.nlines();
        int64_t const size = int64_t(b.basis.size());
        double* gc = nullptr;
        DDCB_CUDA_CHECK(cudaMallocAsync(reinterpret_cast<void**>(&gc), sizeof(double) * size_t(size * nl), s));
        Lines const lgc {size, nl, nl, 1, 0};
        try {
            launch_eval_adjoint(e, order, coords, lx, coefs, lc, gy, lgy, gc, lgc, gx, lgx, s);
            launch_build_adjoint(b, gc, lgc, gv, lgv, gdlo, lglo, gdhi, lghi, s);
        } catch (...) {
            cudaFreeAsync(gc, s);
            throw;
        }
        DDCB_CUDA_CHECK(cudaFreeAsync(gc, s));
    }
    return fused;
}

} // namespace ddcb
