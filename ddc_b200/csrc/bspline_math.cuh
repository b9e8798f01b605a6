// bspline_math.cuh -- B-spline basis evaluation shared by the host plan code and the kernels.
//
// The algorithms are the published ones the reference also uses, so their steps are alike:
//   * Cox-de Boor triangle for the degree+1 non-zero basis values (de Boor, "A Practical Guide to
//     Splines", B-spline recurrence), in the uniform form of bsplines_uniform.hpp:392-426 and the
//     left/right-difference form of bsplines_non_uniform.hpp:459-497;
//   * values plus n derivatives by Algorithm A2.3 of Piegl & Tiller, "The NURBS Book"
//     (bsplines_uniform.hpp:473-564, bsplines_non_uniform.hpp:559-664);
//   * cell location: scaled offset for uniform knots (bsplines_uniform.hpp:566-595), bisection over
//     the break points for non-uniform ones (bsplines_non_uniform.hpp:666-695).
// Keeping the same operation order keeps results within a few ulps of the reference's.
#pragma once

#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define DDCB_HD __host__ __device__ __forceinline__
#else
#define DDCB_HD inline
#endif

namespace ddcb {

constexpr int kMaxDegree = 7;

// Plain description of a basis, valid on host or device depending on where `knots` points.
struct BasisDesc
{
    int degree;
    int periodic;
    int uniform;
    int ncells;
    double rmin;
    double rmax;
    double length;
    double step;     // uniform knot spacing
    double inv_step; // 1/step, as the reference computes it (bsplines_uniform.hpp:366-369)
    const double* knots; // non-uniform: ncells + 1 + 2*degree knots, knot k at knots[k]
};

// bsplines_uniform.hpp:566-595. Returns the cell index and sets offset in [0,1].
DDCB_HD int uniform_cell(BasisDesc const& b, double x, double& offset)
{
    int icell;
    if (x <= b.rmin) {
        icell = 0;
        offset = 0.0;
    } else if (x >= b.rmax) {
        icell = b.ncells - 1;
        offset = 1.0;
    } else {
        offset = (x - b.rmin) * b.inv_step;
        icell = static_cast<int>(offset);
        offset = offset - icell;
        // The reference maps icell == ncells with a zero offset to the last cell. The scaled
        // offset can also round to just above ncells for x a few ulps below rmax; that point is
        // the end of the last cell too (the reference would index past its coefficients there).
        if (icell >= b.ncells) {
            icell = b.ncells - 1;
            offset = 1.0;
        }
    }
    return icell;
}

// bsplines_non_uniform.hpp:666-695. Returns the knot index of the cell start (in [d, d+ncells)).
DDCB_HD int nonuniform_cell(BasisDesc const& b, double x)
{
    int const d = b.degree;
    if (x <= b.rmin) return d;
    if (x >= b.rmax) return d + b.ncells - 1;
    int low = d, high = d + b.ncells;
    int icell = low + (high - low) / 2;
    while (x < b.knots[icell] || x >= b.knots[icell + 1]) {
        if (x < b.knots[icell]) high = icell;
        else low = icell;
        icell = low + (high - low) / 2;
    }
    return icell;
}

// Uniform Cox-de Boor values from the cell offset (deg+1 values).
DDCB_HD void uniform_values(int deg, double offset, double* v)
{
    v[0] = 1.0;
    for (int j = 1; j <= deg; ++j) {
        double xx = -offset;
        double saved = 0.0;
        for (int r = 0; r < j; ++r) {
            xx += 1.0;
            double const temp = v[r] / j;
            v[r] = saved + xx * temp;
            saved = (j - xx) * temp;
        }
        v[j] = saved;
    }
}

// Non-uniform Cox-de Boor values in the cell starting at knot `icell`.
DDCB_HD void nonuniform_values(BasisDesc const& b, int deg, int icell, double x, double* v)
{
    double left[kMaxDegree + 1], right[kMaxDegree + 1];
    v[0] = 1.0;
    for (int j = 0; j < deg; ++j) {
        left[j] = x - b.knots[icell - j];
        right[j] = b.knots[icell + j + 1] - x;
        double saved = 0.0;
        for (int r = 0; r < j + 1; ++r) {
            double const temp = v[r] / (right[r] + left[j - r]);
            v[r] = saved + right[r] * temp;
            saved = left[j - r] * temp;
        }
        v[j + 1] = saved;
    }
}

// Values of the degree+1 non-zero B-splines at x; returns the index of the first one.
DDCB_HD int eval_basis(BasisDesc const& b, double x, double* v)
{
    if (b.uniform) {
        double offset;
        int const jmin = uniform_cell(b, x, offset);
        uniform_values(b.degree, offset, v);
        return jmin;
    }
    int const icell = nonuniform_cell(b, x);
    nonuniform_values(b, b.degree, icell, x, v);
    return icell - b.degree;
}

// Values and derivatives up to order n (A2.3). out[i*(n+1)+k] = k-th derivative of B_{jmin+i}.
DDCB_HD int eval_basis_and_n_derivs(BasisDesc const& b, double x, int n, double* out)
{
    int const d = b.degree;
    int const nc = n + 1;
    double ndu[kMaxDegree + 1][kMaxDegree + 1];
    double a[kMaxDegree + 1][2];
    int jmin;
    bool const uni = b.uniform != 0;
    if (uni) {
        double offset;
        jmin = uniform_cell(b, x, offset);
        ndu[0][0] = 1.0;
        for (int j = 1; j < d + 1; ++j) {
            double xx = -offset;
            double saved = 0.0;
            for (int r = 0; r < j; ++r) {
                xx += 1.0;
                double const temp = ndu[j - 1][r] / j;
                ndu[j][r] = saved + xx * temp;
                saved = (j - xx) * temp;
            }
            ndu[j][j] = saved;
        }
    } else {
        int const icell = nonuniform_cell(b, x);
        jmin = icell - d;
        double left[kMaxDegree + 1], right[kMaxDegree + 1];
        ndu[0][0] = 1.0;
        for (int j = 0; j < d; ++j) {
            left[j] = x - b.knots[icell - j];
            right[j] = b.knots[icell + j + 1] - x;
            double saved = 0.0;
            for (int r = 0; r < j + 1; ++r) {
                ndu[r][j + 1] = 1.0 / (right[r] + left[j - r]);
                double const temp = ndu[j][r] * ndu[r][j + 1];
                ndu[j + 1][r] = saved + right[r] * temp;
                saved = left[j - r] * temp;
            }
            ndu[j + 1][j + 1] = saved;
        }
    }
    for (int i = 0; i < d + 1; ++i) out[i * nc] = ndu[d][i];
    for (int r = 0; r < d + 1; ++r) {
        int s1 = 0, s2 = 1;
        a[0][0] = 1.0;
        for (int k = 1; k < n + 1; ++k) {
            double dd = 0.0;
            int const rk = r - k;
            int const pk = d - k;
            // uniform knots: every knot difference is one step, so the inverse differences are
            // 1/(pk+1) in units of the step; non-uniform: saved inverses in ndu's lower triangle
            if (r >= k) {
                a[0][s2] = uni ? a[0][s1] / (pk + 1) : a[0][s1] * ndu[rk][pk + 1];
                dd = a[0][s2] * ndu[pk][rk];
            }
            int const j1 = rk > -1 ? 1 : (-rk);
            int const j2 = (r - 1) <= pk ? k : (d - r + 1);
            for (int j = j1; j < j2; ++j) {
                a[j][s2] = uni ? (a[j][s1] - a[j - 1][s1]) / (pk + 1) : (a[j][s1] - a[j - 1][s1]) * ndu[rk + j][pk + 1];
                dd += a[j][s2] * ndu[pk][rk + j];
            }
            if (r <= pk) {
                a[k][s2] = uni ? -a[k - 1][s1] / (pk + 1) : -a[k - 1][s1] * ndu[r][pk + 1];
                dd += a[k][s2] * ndu[pk][r];
            }
            out[r * nc + k] = dd;
            int const t = s1;
            s1 = s2;
            s2 = t;
        }
    }
    if (uni) {
        double f = d * b.inv_step;
        for (int k = 1; k < n + 1; ++k) {
            for (int i = 0; i < d + 1; ++i) out[i * nc + k] *= f;
            f *= (d - k) * b.inv_step;
        }
    } else {
        int rr = d;
        for (int k = 1; k < n + 1; ++k) {
            for (int i = 0; i < d + 1; ++i) out[i * nc + k] *= rr;
            rr *= d - k;
        }
    }
    return jmin;
}

// Periodic wrap of the evaluator (spline_evaluator.hpp:537-543): only outside [rmin, rmax].
DDCB_HD double periodic_wrap(BasisDesc const& b, double x)
{
    if (x < b.rmin || x > b.rmax) x -= floor((x - b.rmin) / b.length) * b.length;
    return x;
}

} // namespace ddcb

namespace ddcb {

// ---- compile-time-degree device forms used by the kernels ------------------------------------

// Uniform Cox-de Boor values of degree P from the cell offset; the divisions by the small integer
// j are multiplications by its rounded reciprocal.
template <int P>
DDCB_HD void uniform_values_t(double offset, double* v)
{
    v[0] = 1.0;
#pragma unroll
    for (int j = 1; j <= P; ++j) {
        double const inv_j = 1.0 / j;
        double xx = -offset;
        double saved = 0.0;
#pragma unroll
        for (int r = 0; r < j; ++r) {
            xx += 1.0;
            double const temp = v[r] * inv_j;
            v[r] = saved + xx * temp;
            saved = (j - xx) * temp;
        }
        v[j] = saved;
    }
}

// Non-uniform Cox-de Boor values of degree P in the cell starting at knot icell, with the knot
// span inverses read from inv_span[(len-1)*nk + first_knot] = 1/(t[first+len] - t[first]).
template <int P>
DDCB_HD void nonuniform_values_t(const double* knots, const double* inv_span, int nk, int icell, double x, double* v)
{
    double left[P + 1], right[P + 1];
    v[0] = 1.0;
#pragma unroll
    for (int j = 0; j < P; ++j) {
        left[j] = x - knots[icell - j];
        right[j] = knots[icell + j + 1] - x;
        double saved = 0.0;
#pragma unroll
        for (int r = 0; r < j + 1; ++r) {
            double const temp = v[r] * inv_span[j * nk + icell + r - j];
            v[r] = saved + right[r] * temp;
            saved = left[j - r] * temp;
        }
        v[j + 1] = saved;
    }
}

} // namespace ddcb
