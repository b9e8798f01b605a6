// eval_device.cuh -- device-side point evaluation of a spline from a coefficient tile.
//
// Uniform bases need no tables: the cell comes from a scaled offset and the basis from the
// uniform Cox-de Boor triangle. Non-uniform bases read the knots around the cell as (t_i, t_i+1)
// pairs from shared memory (16-byte loads). Values and first derivatives divide by the knot
// differences, one division per level of the triangle (batched inversion); higher derivatives and
// the adjoints take the knot-span inverses from a small table built with the evaluator.
#pragma once

#include "bspline_math.cuh"
#include "check_bounds.cuh"

namespace ddcb {

// Everything the kernels need to locate a point and evaluate the basis.
struct EvalBasis
{
    BasisDesc b;              // b.knots: device knots
    const double2* kpairs;    // nk-1 pairs (t_i, t_i+1): device copy, or shared-memory copy in a kernel
    const double* inv_span;   // degree x nk: inv_span[(len-1)*nk + i] = 1/(t[i+len] - t[i]) (0 if empty);
                              // global memory, or a shared-memory copy in a kernel (plain loads)
    const double2* lut;       // nbucket entries {split, c0}: c0 the cell (knot index) holding the
                              // bucket start, split the first knot inside the bucket (+inf if none);
                              // device copy, or shared-memory copy in a kernel
    int nbucket;
    double bucket_scale;      // nbucket / (rmax - rmin)
    int nk;                   // number of knots
};

#if defined(__CUDACC__)

// Coefficient access of one line. row0(jmin) gives the row of B-spline jmin; get(row0, i) the
// coefficient of B-spline jmin + i.
// CoefDirect: coefficients in basis order, row b at C[b*cs].
struct CoefDirect
{
    const double* C;
    int cs;
    __device__ __forceinline__ int row0(int jmin) const { return jmin; }
    __device__ __forceinline__ double get(int r0, int i) const { return C[(r0 + i) * cs]; }
};

// CoefRotated: coefficients still in the builder's column order inside its tile: B-spline b lives
// in column ((b mod n) - offset) mod n (spline_builder.hpp:1061-1100).
struct CoefRotated
{
    const double* C;
    int cs;
    int n;
    int offset;
    __device__ __forceinline__ int row0(int jmin) const
    {
        int r = jmin - offset;
        r += (r < 0) ? n : 0;
        r -= (r >= n) ? n : 0;
        return r;
    }
    __device__ __forceinline__ double get(int r0, int i) const
    {
        int r = r0 + i;
        r -= (r >= n) ? n : 0;
        return C[r * cs];
    }
};

// CoefGlobal: coefficients in basis order in global memory (row b at C[b*cs]), read through the
// read-only cache.
struct CoefGlobal
{
    const double* C;
    int64_t cs;
    __device__ __forceinline__ int row0(int jmin) const { return jmin; }
    __device__ __forceinline__ double get(int r0, int i) const { return __ldg(C + (int64_t)(r0 + i) * cs); }
};

// First guess of the cell of x as a knot index (the cell [t_c, t_c+1) with t_c <= x < t_c+1), with
// the end rules of bsplines_non_uniform.hpp:666-695: the bucket's start cell, plus one past the
// bucket's inner knot. Exact when the bucket holds at most one knot (the table is built with
// buckets no wider than the narrowest cell, up to a size cap) and x is not within rounding of a
// bucket edge; nonuniform_walk finishes it otherwise.
__device__ __forceinline__ int nonuniform_guess(EvalBasis const& eb, double x)
{
    int const d = eb.b.degree;
    if (x <= eb.b.rmin) return d;
    if (x >= eb.b.rmax) return d + eb.b.ncells - 1;
    int bk = static_cast<int>((x - eb.b.rmin) * eb.bucket_scale);
    bk = bk < 0 ? 0 : (bk >= eb.nbucket ? eb.nbucket - 1 : bk);
    double2 const e = eb.lut[bk];
    return static_cast<int>(e.y) + (x >= e.x ? 1 : 0);
}

// Whether c is the cell of x, given tc = t_c and tc1 = t_c+1.
__device__ __forceinline__ bool nonuniform_is_cell(EvalBasis const& eb, double x, int c, double tc, double tc1)
{
    int const d = eb.b.degree;
    return (c == d || x >= tc) && (c == d + eb.b.ncells - 1 || x < tc1);
}

// The cell of x in [d, last], walking over the knot pairs from the guess c.
__device__ __forceinline__ int nonuniform_walk_pairs(const double2* kpairs, int d, int last, double x, int c)
{
    double2 p = kpairs[c];
    while (c < last && x >= p.y) p = kpairs[++c];
    while (c > d && x < p.x) p = kpairs[--c];
    return c;
}

__device__ __forceinline__ int nonuniform_walk(EvalBasis const& eb, double x, int c)
{
    return nonuniform_walk_pairs(eb.kpairs, eb.b.degree, eb.b.degree + eb.b.ncells - 1, x, c);
}

// Cell of x: the guess, checked against its knot pair (equal to bisection for any mesh).
__device__ __forceinline__ int nonuniform_locate(EvalBasis const& eb, double x)
{
    int const c = nonuniform_guess(eb, x);
    double2 const p = eb.kpairs[DDCB_INDEX(c, eb.nk - 1)];
    return nonuniform_is_cell(eb, x, c, p.x, p.y) ? c : nonuniform_walk(eb, x, c);
}

// The 2P knots t[c-P+1 .. c+P] around cell c (P >= 1), by P pair loads.
template <int P>
__device__ __forceinline__ void load_knots(EvalBasis const& eb, int c, double* kn)
{
#pragma unroll
    for (int q = 0; q < P; ++q) {
        double2 const p = eb.kpairs[DDCB_INDEX(c - P + 1 + 2 * q, eb.nk - 1)];
        kn[2 * q] = p.x;
        kn[2 * q + 1] = p.y;
    }
}

// The cell of x and its 2P knots t[c-P+1 .. c+P] (P >= 1): the guess's knots hold t_c and t_c+1,
// which check it; a wrong guess is walked to the cell and its knots reloaded.
template <int P>
__device__ __forceinline__ int locate_load_knots(EvalBasis const& eb, double x, double* kn)
{
    int c = nonuniform_guess(eb, x);
    load_knots<P>(eb, c, kn);
    if (!nonuniform_is_cell(eb, x, c, kn[P - 1], kn[P])) {
        c = nonuniform_walk(eb, x, c);
        load_knots<P>(eb, c, kn);
    }
    return c;
}

// Non-uniform Cox-de Boor values of degree P on cell c (bsplines_non_uniform.hpp:459-497), with
// the knot-span inverses read from the span table (ispan = inv_span + c: entry (j, r) is
// 1/(t[c+r+1] - t[c+r-j]) at ispan[j*nk + r - j]).
template <int P>
__device__ __forceinline__ void nonuniform_values_span(const double* kn, const double* ispan, int nk, double x, double* v)
{
    double left[P + 1], right[P + 1];
    v[0] = 1.0;
#pragma unroll
    for (int j = 0; j < P; ++j) {
        left[j] = x - kn[P - 1 - j];  // x - t[c-j]
        right[j] = kn[P + j] - x;     // t[c+j+1] - x
        double saved = 0.0;
#pragma unroll
        for (int r = 0; r < j + 1; ++r) {
            double const temp = v[r] * ispan[j * nk + r - j];
            v[r] = saved + right[r] * temp;
            saved = left[j - r] * temp;
        }
        v[j + 1] = saved;
    }
}

// As nonuniform_values_span, also returning the degree P-1 values of the same cell (the level
// before the last of the triangle), which the spline derivative needs.
template <int P>
__device__ __forceinline__ void nonuniform_values_span2(const double* kn, const double* ispan, int nk, double x, double* v,
                                                        double* vprev)
{
    double left[P + 1], right[P + 1];
    v[0] = 1.0;
    if (P == 1) vprev[0] = 1.0;
#pragma unroll
    for (int j = 0; j < P; ++j) {
        left[j] = x - kn[P - 1 - j];
        right[j] = kn[P + j] - x;
        double saved = 0.0;
#pragma unroll
        for (int r = 0; r < j + 1; ++r) {
            double const temp = v[r] * ispan[j * nk + r - j];
            v[r] = saved + right[r] * temp;
            saved = left[j - r] * temp;
        }
        v[j + 1] = saved;
        if (j == P - 2) {
#pragma unroll
            for (int r = 0; r < P; ++r) vprev[r] = v[r];
        }
    }
}

// 1/d for a positive normal d: the hardware approximation (rcp.approx.ftz.f64) refined by two
// Newton-Raphson steps r <- r + r (1 - d r) (quadratic convergence: the approximation's ~20 bits
// become more than the 53 of a double; within an ulp or two of the rounded quotient), without the
// special-case path of an IEEE division. Used for knot differences, which are positive and far from
// the range limits.
__device__ __forceinline__ double recip_newton(double d)
{
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
    double e = fma(-d, r, 1.0);
    r = fma(r, e, r);
    e = fma(-d, r, 1.0);
    return fma(r, e, r);
}

// Non-uniform Cox-de Boor values of degree P on the cell whose knots are kn (the layout of
// nonuniform_values_span), dividing by the knot differences themselves: the j+1 denominators of
// level j are inverted together with one division (prefix products, then one reciprocal, then
// back-substitution of the products). Every denominator t[c+r+1] - t[c+r-j] spans the cell
// [t_c, t_c+1), which is never empty (break points strictly increase), so no guard is needed even
// where boundary knots repeat. The products hold at most P knot differences, so they stay in FP64
// range for spacings between 1e-60 and 1e60 of the coordinate unit.
template <int P>
__device__ __forceinline__ void nonuniform_values_div(const double* kn, double x, double* v)
{
    double left[P + 1], right[P + 1];
    v[0] = 1.0;
#pragma unroll
    for (int j = 0; j < P; ++j) {
        left[j] = x - kn[P - 1 - j];
        right[j] = kn[P + j] - x;
        double d[P], pre[P], inv_d[P];
#pragma unroll
        for (int r = 0; r <= j; ++r) {
            double const den = kn[P + r] - kn[P - 1 - j + r];
            d[r] = den;
            pre[r] = r == 0 ? d[0] : pre[r - 1] * d[r];
        }
        double inv = recip_newton(pre[j]);
#pragma unroll
        for (int r = j; r >= 1; --r) {
            inv_d[r] = inv * pre[r - 1];
            inv *= d[r];
        }
        inv_d[0] = inv;
        double saved = 0.0;
#pragma unroll
        for (int r = 0; r < j + 1; ++r) {
            double const temp = v[r] * inv_d[r];
            v[r] = saved + right[r] * temp;
            saved = left[j - r] * temp;
        }
        v[j + 1] = saved;
    }
}

// s'(x) on the non-uniform cell ck (spline_evaluator.hpp:357-478 for order 1): the 2D knots around
// the cell give both the degree-(D-1) basis and the divided-difference factors
// D / (t[ck+i] - t[ck-D+i]), i = 1..D, computed here rather than read from the span table. Each of
// these spans contains the cell, so none is empty.
template <int D, class Acc>
__device__ __forceinline__ double nonuniform_deriv1(EvalBasis const& eb, double x, Acc const& C)
{
    constexpr int P = D - 1;
    double kn[2 * D]; // t[ck-D+1 .. ck+D]
    int const ck = locate_load_knots<D>(eb, x, kn);
    double v[P + 1];
    if constexpr (P > 0) nonuniform_values_div<P>(kn + 1, x, v);
    else v[0] = 1.0;
    double d[D], pre[D], f[D + 1];
#pragma unroll
    for (int i = 1; i <= D; ++i) {
        double const den = kn[D - 1 + i] - kn[i - 1];
        d[i - 1] = den;
        pre[i - 1] = i == 1 ? d[0] : pre[i - 2] * d[i - 1];
    }
    double inv = double(D) / pre[D - 1];
#pragma unroll
    for (int i = D; i >= 2; --i) {
        f[i] = inv * pre[i - 2];
        inv *= d[i - 1];
    }
    f[1] = inv;
    int const r0 = C.row0(DDCB_INDEX(ck - D, eb.b.ncells));
    double y = 0.0;
    double cprev = C.get(r0, 0);
#pragma unroll
    for (int r = 0; r < P + 1; ++r) {
        double const ci = C.get(r0, r + 1);
        y = fma((ci - cprev) * f[r + 1], v[r], y);
        cprev = ci;
    }
    return y;
}

// s'(x) on a non-uniform basis from the derivative spline's coefficients: Acc holds
// d_j = D (c_j - c_{j-1}) / (t_{j+D} - t_j), the coefficients of s' on the degree-(D-1) B-splines
// (de Boor, "A Practical Guide to Splines", X.(15)), so a point needs the 2(D-1) knots around its
// cell and the degree-(D-1) basis only: no divided-difference factors, one knot pair fewer than
// nonuniform_deriv1. D >= 2.
template <int D, class Acc>
__device__ __forceinline__ double nonuniform_deriv1_dcoef(EvalBasis const& eb, double x, Acc const& C)
{
    constexpr int P = D - 1;
    double kn[2 * P]; // t[ck-P+1 .. ck+P]
    int const ck = locate_load_knots<P>(eb, x, kn);
    double v[P + 1];
    nonuniform_values_div<P>(kn, x, v);
    int const r0 = C.row0(DDCB_INDEX(ck - D, eb.b.ncells) + 1);
    double y = 0.0;
#pragma unroll
    for (int r = 0; r < P + 1; ++r) y = fma(C.get(r0, r), v[r], y);
    return y;
}

// s(x) without boundary handling (spline_evaluator.hpp:556-605).
template <int D, bool UNI, class Acc>
__device__ __forceinline__ double eval_value_no_bc(EvalBasis const& eb, double x, Acc const& C)
{
    double v[D + 1];
    int jmin;
    if (UNI) {
        double off;
        jmin = uniform_cell(eb.b, x, off);
        uniform_values_t<D>(off, v);
    } else {
        double kn[2 * D];
        jmin = locate_load_knots<D>(eb, x, kn) - D;
        nonuniform_values_div<D>(kn, x, v);
    }
    int const r0 = C.row0(DDCB_INDEX(jmin, eb.b.ncells));
    double y = 0.0;
#pragma unroll
    for (int i = 0; i < D + 1; ++i) y = fma(C.get(r0, i), v[i], y);
    return y;
}

// s(x) with the periodic wrap or the extrapolation rules (spline_evaluator.hpp:529-554,
// null_extrapolation_rule.hpp:14-26, constant_extrapolation_rule.hpp:27-52 evaluated at the
// domain end).
template <int D, bool UNI, class Acc>
__device__ __forceinline__ double eval_value_bc(EvalBasis const& eb, int ex_lo, int ex_hi, double x, Acc const& C)
{
    if (eb.b.periodic) {
        x = periodic_wrap(eb.b, x);
    } else {
        if (x < eb.b.rmin) {
            if (ex_lo == 1) return 0.0;
            x = eb.b.rmin;
        } else if (x > eb.b.rmax) {
            if (ex_hi == 1) return 0.0;
            x = eb.b.rmax;
        }
    }
    return eval_value_no_bc<D, UNI>(eb, x, C);
}

// d^ORDER s / dx^ORDER at x (spline_evaluator.hpp:388-430, no boundary handling): ORDER rounds of
// divided differences of the D+1 coefficients of the cell (the derivative spline, de Boor,
// "A Practical Guide to Splines", X.(15)), then the degree-(D-ORDER) basis.
template <int D, int ORDER, bool UNI, class Acc>
__device__ __forceinline__ double eval_deriv_no_bc(EvalBasis const& eb, double x, Acc const& C)
{
    constexpr int P = D - ORDER;
    double cc[D + 1];
    double v[P + 1];
    int jmin;
    if constexpr (!UNI && ORDER == 1) {
        return nonuniform_deriv1<D>(eb, x, C);
    }
    if (UNI) {
        double off;
        jmin = uniform_cell(eb.b, x, off);
        uniform_values_t<P>(off, v);
    } else {
        int const ck = nonuniform_locate(eb, x);
        jmin = ck - D;
        if constexpr (P > 0) {
            double kn[2 * P];
            load_knots<P>(eb, ck, kn);
            nonuniform_values_span<P>(kn, eb.inv_span + ck, eb.nk, x, v);
        } else {
            v[0] = 1.0;
        }
    }
    const double* dspan = eb.inv_span + jmin; // 1/(t[jmin+i+len] - t[jmin+i]) at dspan[(len-1)*nk + i]
    int const r0 = C.row0(DDCB_INDEX(jmin, eb.b.ncells));
#pragma unroll
    for (int i = 0; i < D + 1; ++i) cc[i] = C.get(r0, i);
#pragma unroll
    for (int k = 1; k <= ORDER; ++k) {
#pragma unroll
        for (int i = D; i >= k; --i) {
            if (UNI) cc[i] = (cc[i] - cc[i - 1]) * eb.b.inv_step;
            else cc[i] = double(D - k + 1) * (cc[i] - cc[i - 1]) * dspan[(D - k) * eb.nk + i];
        }
    }
    double y = 0.0;
#pragma unroll
    for (int r = 0; r < P + 1; ++r) y = fma(cc[ORDER + r], v[r], y);
    return y;
}

// Value (ORDER 0, with boundary handling) or ORDER-th derivative (no boundary handling).
template <int D, int ORDER, bool UNI, class Acc>
__device__ __forceinline__ double eval_point(EvalBasis const& eb, int ex_lo, int ex_hi, double x, Acc const& C)
{
    if constexpr (ORDER == 0) return eval_value_bc<D, UNI>(eb, ex_lo, ex_hi, x, C);
    else return eval_deriv_no_bc<D, ORDER, UNI>(eb, x, C);
}

#endif // __CUDACC__

} // namespace ddcb

namespace ddcb {

#if defined(__CUDACC__)

// Values of the ORDER-th derivative of the D+1 non-zero degree-D B-splines at x (the quantity the
// reference takes from eval_basis_and_n_derivs, bsplines_*.hpp); returns the first B-spline index.
// The degree-(D-ORDER) basis is raised back to degree D with the transpose of the derivative
// differencing: d/dx B_{i,p} = p/(t_{i+p}-t_i) B_{i,p-1} - p/(t_{i+p+1}-t_{i+1}) B_{i+1,p-1}.
template <int D, int ORDER, bool UNI>
__device__ __forceinline__ int basis_derivs(EvalBasis const& eb, double x, double* val)
{
    constexpr int P = D - ORDER;
    double w[D + 2];
    int jmin;
    if (UNI) {
        double off;
        jmin = uniform_cell(eb.b, x, off);
        uniform_values_t<P>(off, w + ORDER);
    } else {
        int const ck = nonuniform_locate(eb, x);
        jmin = ck - D;
        if constexpr (P > 0) {
            double kn[2 * P];
            load_knots<P>(eb, ck, kn);
            nonuniform_values_span<P>(kn, eb.inv_span + ck, eb.nk, x, w + ORDER);
        } else {
            w[ORDER] = 1.0;
        }
    }
    // w[i] holds the value for B-spline jmin + i of the current degree, for i in [k, D]
#pragma unroll
    for (int k = ORDER; k >= 1; --k) {
        // degree p = D-k+1 from degree D-k: entries i in [k-1, D]
        int constexpr dummy = 0;
        (void)dummy;
        double nw[D + 2];
#pragma unroll
        for (int i = 0; i <= D; ++i) nw[i] = 0.0;
#pragma unroll
        for (int i = k - 1; i <= D; ++i) {
            double const a = (i >= k) ? w[i] : 0.0;       // B_{i, p-1}
            double const b = (i + 1 <= D) ? w[i + 1] : 0.0; // B_{i+1, p-1}
            double fa, fb;
            if (UNI) {
                fa = eb.b.inv_step;
                fb = eb.b.inv_step;
            } else {
                int const p = D - k + 1;
                fa = double(p) * eb.inv_span[(p - 1) * eb.nk + jmin + i];
                fb = double(p) * eb.inv_span[(p - 1) * eb.nk + jmin + i + 1];
            }
            nw[i] = fa * a - fb * ((i + 1 <= D && i + 1 >= k) ? b : 0.0);
        }
#pragma unroll
        for (int i = 0; i <= D; ++i) w[i] = nw[i];
    }
#pragma unroll
    for (int i = 0; i <= D; ++i) val[i] = w[i];
    return jmin;
}

// Reverse mode of one evaluated point. For y = s(x) (ORDER 0, with the boundary handling of
// eval_value_bc) or y = s'(x) (ORDER 1, no boundary handling), returns the first B-spline index
// jmin and the weights wts[i] = dy/dc[jmin+i] (the B-spline values, or their derivatives), and sets
// dydx = dy/dx (s'(x) or s''(x); 0 where y does not depend on x). Returns -1 when y is identically
// 0 there (null extrapolation). dydx is computed only when want_dx is set.
template <int D, int ORDER, bool UNI, class Acc>
__device__ __forceinline__ int point_adjoint(EvalBasis const& eb, int ex_lo, int ex_hi, double x, Acc const& C,
                                             bool want_dx, double* wts, double& dydx)
{
    dydx = 0.0;
    if constexpr (ORDER == 0) {
        bool fixed = false; // y does not move with x (constant extrapolation)
        if (eb.b.periodic) {
            x = periodic_wrap(eb.b, x);
        } else if (x < eb.b.rmin) {
            if (ex_lo == 1) return -1;
            x = eb.b.rmin;
            fixed = true;
        } else if (x > eb.b.rmax) {
            if (ex_hi == 1) return -1;
            x = eb.b.rmax;
            fixed = true;
        }
        double vp[D > 1 ? D : 1];
        int jmin;
        if (UNI) {
            double off;
            jmin = uniform_cell(eb.b, x, off);
            uniform_values_t<D>(off, wts);
            uniform_values_t<D - 1>(off, vp);
        } else {
            int const ck = nonuniform_locate(eb, x);
            jmin = ck - D;
            double kn[2 * D];
            load_knots<D>(eb, ck, kn);
            nonuniform_values_span2<D>(kn, eb.inv_span + ck, eb.nk, x, wts, vp);
        }
        if (want_dx && !fixed) {
            // s'(x) = sum_r cc[r+1] B_{jmin+1+r, D-1}(x), cc the first divided differences
            int const r0 = C.row0(DDCB_INDEX(jmin, eb.b.ncells));
            double cprev = C.get(r0, 0);
            double y = 0.0;
#pragma unroll
            for (int i = 1; i <= D; ++i) {
                double const ci = C.get(r0, i);
                double const f = UNI ? eb.b.inv_step : double(D) * eb.inv_span[(D - 1) * eb.nk + jmin + i];
                y = fma((ci - cprev) * f, vp[i - 1], y);
                cprev = ci;
            }
            dydx = y;
        }
        return jmin;
    } else {
        int const jmin = basis_derivs<D, ORDER, UNI>(eb, x, wts);
        if constexpr (ORDER + 1 <= D) {
            if (want_dx) dydx = eval_deriv_no_bc<D, ORDER + 1, UNI>(eb, x, C);
        }
        return jmin;
    }
}

#endif

} // namespace ddcb
