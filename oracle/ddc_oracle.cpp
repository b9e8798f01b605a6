// ddc_oracle.cpp -- CPU restatement of DDC's batched spline builder/evaluator (TEST INFRASTRUCTURE).
//
// This file is the parity oracle and the timed CPU baseline ("port") of the reference hot path:
// ddc::SplineBuilder / ddc::SplineEvaluator (CExA-project/ddc v0.15.1). It is NOT part of the
// product: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / --impl reference
// legs may load it. The product (ddc_b200/) never links or calls it.
//
// Parity status: the reference cannot be compiled here (it needs Kokkos, Kokkos-Kernels, LAPACKE
// and Ginkgo, none of which exist in the image), so this restatement is pinned against
//   * the reference's own known-answer tests, restated in tests/test_oracle_known_answers.py
//     (partition of unity, polynomial exactness, Tikhomirov error bounds, A*inv(A)=I on the
//     reference's deterministic test matrices), and
//   * an independent implementation of the same mathematics (scipy.interpolate / LAPACK via
//     scipy.linalg.lapack), through the golden fixtures in tests/golden/.
// No golden output of the reference itself exists (the reference ships none and cannot run here).
//
// Every routine cites the reference file:line it restates. LAPACK / Kokkos-Kernels routines that
// the reference calls (dpttrf, dpbtrf, dgbtrf, dgetrf and the batched Serial*trs solves) are
// restated from their published unblocked algorithms.
//
// Layout convention of every batched array here: (row, line) row-major, line index contiguous,
// i.e. element (i, b) at ptr[i * B + b] -- DDC's (x, batch) layout_right ordering.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace oracle {

enum Closure { PERIODIC = 0, HERMITE = 1, HOMOGENEOUS_HERMITE = 2, GREVILLE = 3 };
enum Extrap { EX_PERIODIC = 0, EX_NULL = 1, EX_CONSTANT = 2 };

// spline_builder_closures.hpp:43-55
static int n_boundary_equations(int bc, int degree)
{
    if (bc == PERIODIC || bc == GREVILLE) return 0;
    return degree / 2;
}

// math_tools.hpp:61-65 (modulo with floor)
static long modulo(long x, long y)
{
    return x - y * static_cast<long>(std::floor(double(x) / double(y)));
}

// math_tools.hpp:67-75
static double ipow(double a, int i)
{
    double r = 1.0;
    for (int j = 0; j < i; ++j) r *= a;
    return r;
}

// ------------------------------------------------------------------------------------------------
// B-spline bases: bsplines_uniform.hpp and bsplines_non_uniform.hpp
// ------------------------------------------------------------------------------------------------
struct BSplines
{
    int degree = 3;
    bool periodic = false;
    bool uniform = true;
    long ncells_ = 0;
    // uniform: knot k has coordinate origin + k*step (uniform_point_sampling.hpp:124-128,
    // ghosted init uniform_point_sampling.hpp:170-192, bsplines_uniform.hpp:145-155)
    double origin = 0.0, step = 1.0;
    // non-uniform: explicit knot vector (bsplines_non_uniform.hpp:414-457)
    std::vector<double> knots;

    long ncells() const { return ncells_; }
    long nbasis() const { return ncells_ + (periodic ? 0 : degree); } // bsplines_uniform.hpp:339-342
    long size() const { return ncells_ + degree; }                     // bsplines_uniform.hpp:309-312
    double knot(long k) const { return uniform ? origin + double(k) * step : knots[k]; }
    double rmin() const { return knot(degree); }
    double rmax() const { return knot(degree + ncells_); }
    double length() const { return rmax() - rmin(); }

    // bsplines_uniform.hpp:566-595
    void get_icell_and_offset(long& icell, double& offset, double x) const
    {
        double const inv_dx = 1.0 / step;
        if (x <= rmin()) {
            icell = 0;
            offset = 0.0;
        } else if (x >= rmax()) {
            icell = ncells_ - 1;
            offset = 1.0;
        } else {
            offset = (x - rmin()) * inv_dx;
            icell = static_cast<long>(offset);
            offset = offset - double(icell);
            if (icell == ncells_ && offset == 0.0) {
                icell = ncells_ - 1;
                offset = 1.0;
            }
        }
    }

    // bsplines_non_uniform.hpp:666-695 (returns the knot index of the cell start)
    long find_cell_start(double x) const
    {
        long const front = degree, back = degree + ncells_;
        if (x <= rmin()) return front;
        if (x >= rmax()) return back - 1;
        long low = front, high = back;
        long icell = low + (high - low) / 2;
        while (x < knots[icell] || x >= knots[icell + 1]) {
            if (x < knots[icell]) high = icell;
            else low = icell;
            icell = low + (high - low) / 2;
        }
        return icell;
    }

    // Values of the deg+1 non-zero B-splines of degree `deg` at x; returns jmin.
    // Uniform: bsplines_uniform.hpp:392-426 (deg may exceed degree, used by integrals.hpp:78-82).
    // Non-uniform: bsplines_non_uniform.hpp:459-497.
    long eval_basis(double* values, double x, int deg) const
    {
        if (uniform) {
            long jmin;
            double offset;
            get_icell_and_offset(jmin, offset, x);
            values[0] = 1.0;
            for (int j = 1; j <= deg; ++j) {
                double xx = -offset;
                double saved = 0.0;
                for (int r = 0; r < j; ++r) {
                    xx += 1;
                    double const temp = values[r] / j;
                    values[r] = saved + xx * temp;
                    saved = (j - xx) * temp;
                }
                values[j] = saved;
            }
            return jmin;
        }
        long const icell = find_cell_start(x);
        double left[8], right[8];
        values[0] = 1.0;
        for (int j = 0; j < deg; ++j) {
            left[j] = x - knots[icell - j];
            right[j] = knots[icell + j + 1] - x;
            double saved = 0.0;
            for (int r = 0; r < j + 1; ++r) {
                double const temp = values[r] / (right[r] + left[j - r]);
                values[r] = saved + right[r] * temp;
                saved = left[j - r] * temp;
            }
            values[j + 1] = saved;
        }
        return icell - degree;
    }

    // Values and n derivatives (NURBS book A2.3). derivs is (degree+1) x (n+1) row-major:
    // derivs[i*(n+1)+k] = k-th derivative of B_{jmin+i}.
    // Uniform: bsplines_uniform.hpp:473-564; non-uniform: bsplines_non_uniform.hpp:559-664.
    long eval_basis_and_n_derivs(double* derivs, double x, int n) const
    {
        int const d = degree;
        int const nc = n + 1;
        double ndu[8][8];
        double a[8][2];
        long jmin;
        if (uniform) {
            double offset;
            get_icell_and_offset(jmin, offset, x);
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
            for (int i = 0; i < d + 1; ++i) derivs[i * nc + 0] = ndu[d][i];
            for (int r = 0; r < d + 1; ++r) {
                int s1 = 0, s2 = 1;
                a[0][0] = 1.0;
                for (int k = 1; k < n + 1; ++k) {
                    double dd = 0.0;
                    int const rk = r - k;
                    int const pk = d - k;
                    if (r >= k) {
                        a[0][s2] = a[0][s1] / (pk + 1);
                        dd = a[0][s2] * ndu[pk][rk];
                    }
                    int const j1 = rk > -1 ? 1 : (-rk);
                    int const j2 = (r - 1) <= pk ? k : (d - r + 1);
                    for (int j = j1; j < j2; ++j) {
                        a[j][s2] = (a[j][s1] - a[j - 1][s1]) / (pk + 1);
                        dd += a[j][s2] * ndu[pk][rk + j];
                    }
                    if (r <= pk) {
                        a[k][s2] = -a[k - 1][s1] / (pk + 1);
                        dd += a[k][s2] * ndu[pk][r];
                    }
                    derivs[r * nc + k] = dd;
                    std::swap(s1, s2);
                }
            }
            double const inv_dx = 1.0 / step;
            double dfac = d * inv_dx;
            for (int k = 1; k < n + 1; ++k) {
                for (int i = 0; i < d + 1; ++i) derivs[i * nc + k] *= dfac;
                dfac *= (d - k) * inv_dx;
            }
            return jmin;
        }
        long const icell = find_cell_start(x);
        double left[8], right[8];
        ndu[0][0] = 1.0;
        for (int j = 0; j < d; ++j) {
            left[j] = x - knots[icell - j];
            right[j] = knots[icell + j + 1] - x;
            double saved = 0.0;
            for (int r = 0; r < j + 1; ++r) {
                ndu[r][j + 1] = 1.0 / (right[r] + left[j - r]);
                double const temp = ndu[j][r] * ndu[r][j + 1];
                ndu[j + 1][r] = saved + right[r] * temp;
                saved = left[j - r] * temp;
            }
            ndu[j + 1][j + 1] = saved;
        }
        for (int j = 0; j < d + 1; ++j) derivs[j * nc + 0] = ndu[d][j];
        for (int r = 0; r < d + 1; ++r) {
            int s1 = 0, s2 = 1;
            a[0][0] = 1.0;
            for (int k = 1; k < n + 1; ++k) {
                double dd = 0.0;
                int const rk = r - k;
                int const pk = d - k;
                if (r >= k) {
                    a[0][s2] = a[0][s1] * ndu[rk][pk + 1];
                    dd = a[0][s2] * ndu[pk][rk];
                }
                int const j1 = rk > -1 ? 1 : (-rk);
                int const j2 = (r - 1) <= pk ? k : (d - r + 1);
                for (int j = j1; j < j2; ++j) {
                    a[j][s2] = (a[j][s1] - a[j - 1][s1]) * ndu[rk + j][pk + 1];
                    dd += a[j][s2] * ndu[pk][rk + j];
                }
                if (r <= pk) {
                    a[k][s2] = -a[k - 1][s1] * ndu[r][pk + 1];
                    dd += a[k][s2] * ndu[pk][r];
                }
                derivs[r * nc + k] = dd;
                std::swap(s1, s2);
            }
        }
        int rr = d;
        for (int k = 1; k < n + 1; ++k) {
            for (int i = 0; i < d + 1; ++i) derivs[i * nc + k] *= rr;
            rr *= d - k;
        }
        return icell - degree;
    }

    // Integrals of every B-spline over the domain, size() entries (periodic duplicates get 0).
    // integrals.hpp:30-101 (uniform), :110-153 (non-uniform).
    void integrals(double* out) const
    {
        long const sz = size();
        if (uniform) {
            if (periodic) {
                for (long i = 0; i < nbasis(); ++i) out[i] = step;
                for (long i = nbasis(); i < sz; ++i) out[i] = 0.0;
            } else {
                for (long i = degree; i < sz - degree; ++i) out[i] = step;
                double edge[10];
                eval_basis(edge, rmin(), degree + 1);
                double d_eval = 0.0;
                for (int k = 0; k < degree + 2; ++k) d_eval += edge[k];
                for (int i = 0; i < degree; ++i) {
                    double c_eval = 0.0;
                    for (int k = 0; k < degree - i; ++k) c_eval += edge[k];
                    double const v = step * (d_eval - c_eval);
                    out[i] = v;
                    out[sz - 1 - i] = v;
                }
            }
            return;
        }
        double const inv_deg = 1.0 / (degree + 1);
        for (long i = 0; i < nbasis(); ++i) out[i] = (knots[i + degree + 1] - knots[i]) * inv_deg;
        for (long i = nbasis(); i < sz; ++i) out[i] = 0.0;
    }
};

static std::unique_ptr<BSplines> make_uniform(int degree, bool periodic, double a, double b, long ncells)
{
    auto bs = std::make_unique<BSplines>();
    bs->degree = degree;
    bs->periodic = periodic;
    bs->uniform = true;
    bs->ncells_ = ncells;
    // uniform_point_sampling.hpp:179-181: step = (b-a)/(n-1), origin = a - ghosts*step
    double const step = (b - a) / double(ncells);
    bs->step = step;
    bs->origin = a - double(degree) * step;
    return bs;
}

static std::unique_ptr<BSplines> make_non_uniform(int degree, bool periodic, double const* breaks, long nbreaks)
{
    auto bs = std::make_unique<BSplines>();
    bs->degree = degree;
    bs->periodic = periodic;
    bs->uniform = false;
    bs->ncells_ = nbreaks - 1;
    std::vector<double>& k = bs->knots;
    k.assign(nbreaks + 2 * degree, 0.0);
    for (long i = 0; i < nbreaks; ++i) k[degree + i] = breaks[i];
    double const rmin = k[degree];
    double const rmax = k[nbreaks + degree - 1];
    long const nc = nbreaks - 1;
    if (periodic) {
        double const period = rmax - rmin;
        for (int i = 1; i < degree + 1; ++i) {
            k[degree - i] = k[degree + nc - i] - period;
            k[degree + nc + i] = k[degree + i] + period;
        }
    } else {
        for (int i = 1; i < degree + 1; ++i) {
            k[degree - i] = rmin;
            k[degree + nbreaks - 1 + i] = rmax;
        }
    }
    return bs;
}

// ------------------------------------------------------------------------------------------------
// Interpolation points: greville_interpolation_points.hpp:47-269
// ------------------------------------------------------------------------------------------------
static std::vector<double> greville_points(BSplines const& bs, int bc_lo, int bc_hi)
{
    int const d = bs.degree;
    int const nbe_min = n_boundary_equations(bc_lo, d);
    int const nbe_max = n_boundary_equations(bc_hi, d);
    int const nbe = nbe_min + nbe_max;
    long const npoints = bs.nbasis() - nbe;
    std::vector<double> pts;
    bool const uniform_sampling = bs.uniform && ((nbe_min != 0 && nbe_max != 0) || bs.periodic);
    if (bs.uniform) {
        // uniform_greville_points (:47-69)
        double const shift = (d % 2 == 0) ? 0.5 : 0.0;
        double const dx = (bs.rmax() - bs.rmin()) / double(bs.ncells());
        if (uniform_sampling) {
            // UniformPointSampling(origin = rmin + shift*dx, step = dx): coordinate(i) = origin + i*dx
            double const o = bs.rmin() + shift * dx;
            pts.resize(npoints);
            for (long i = 0; i < npoints; ++i) pts[i] = o + double(i) * dx;
            return pts;
        }
        // Intermediate uniform sampling (:171-228): points_wo_bcs.coordinate(i) = o + i*dx
        double const o = bs.rmin() + shift * dx;
        auto wo = [&](long i) { return o + double(i) * dx; };
        pts.assign(npoints, 0.0);
        long const n_break_points = bs.ncells() + 1;
        if (bc_lo == GREVILLE) {
            for (int i = 0; i < d / 2 + 1; ++i) {
                pts[i] = (d - i) * bs.rmin();
                // knots get_last_support_knot(i) - i .. (exclusive end at last support knot)
                long const last = i + d + 1;
                for (long k = last - i; k < last; ++k) pts[i] += bs.knot(k);
                pts[i] /= d;
            }
        } else {
            pts[0] = wo(0);
        }
        long const n_start = (bc_lo == GREVILLE) ? d / 2 + 1 : 1;
        long const domain_size = n_break_points - 2;
        for (long ip = 1; ip < 1 + domain_size; ++ip) pts[ip - 1 + n_start] = wo(ip);
        if (bc_hi == GREVILLE) {
            for (int i = 0; i < d / 2 + 1; ++i) {
                pts[npoints - 1 - i] = (d - i) * bs.rmax();
                long const spline_idx = bs.nbasis() - 1 - i;
                long const first = spline_idx + 1; // get_first_support_knot(spline_idx) + 1
                for (long k = first; k < first + i; ++k) pts[npoints - 1 - i] += bs.knot(k);
                pts[npoints - 1 - i] /= d;
            }
        } else {
            pts[npoints - 1] = wo(bs.ncells() - 1 + d % 2);
        }
        return pts;
    }
    // non_uniform_greville_points (:72-132)
    long const nb = bs.nbasis();
    long const n_greville = bs.periodic ? nb + 1 : nb;
    std::vector<double> g(n_greville, 0.0);
    for (long ib = 0; ib < nb; ++ib) {
        g[ib] = 0.0;
        for (long k = ib + 1; k < ib + 1 + d; ++k) g[ib] += bs.knot(k);
        g[ib] /= d;
    }
    if (bs.periodic) {
        std::vector<double> temp(d);
        long np = 0;
        while (g[np] < bs.rmin()) {
            temp[np] = g[np] + bs.length();
            ++np;
        }
        for (long i = 0; i < nb - np; ++i) g[i] = g[i + np];
        for (long i = 0; i < np; ++i) g[nb - np + i] = temp[i];
        g[n_greville - 1] = g[0] + bs.length();
    }
    if (nbe == 0) {
        // The sampling holds n_greville points; the interpolation domain takes the first npoints.
        pts.assign(g.begin(), g.begin() + npoints);
        return pts;
    }
    pts.resize(g.size() - nbe);
    for (size_t i = 0; i < pts.size(); ++i) pts[i] = g[i + nbe_min];
    return pts;
}

// ------------------------------------------------------------------------------------------------
// Linear problems: splines_linear_problem*.{hpp,cpp}
// solve(b, ld, ncols, transpose): b is rows x ncols with row stride ld (LayoutRight MultiRHS,
// splines_linear_problem.hpp:27), columns solved independently (thread per column).
// ------------------------------------------------------------------------------------------------
struct LinearProblem
{
    long n;
    explicit LinearProblem(long n_) : n(n_) {}
    virtual ~LinearProblem() = default;
    virtual double get(long i, long j) const = 0;
    virtual void set(long i, long j, double v) = 0;
    virtual void setup() = 0;
    virtual void solve_col(double* b, long ld, bool transpose) const = 0;
    virtual long required_rows() const { return n; }
    virtual void solve(double* b, long ld, long ncols, bool transpose, int nthreads) const
    {
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (long c = 0; c < ncols; ++c) solve_col(b + c, ld, transpose);
    }
};

// splines_linear_problem_dense.cpp:34-130: dgetrf (partial pivoting) + SerialGetrs
struct Dense : LinearProblem
{
    std::vector<double> a;
    std::vector<long> ipiv;
    explicit Dense(long n_) : LinearProblem(n_), a(n_ * n_, 0.0), ipiv(n_, 0) {}
    double get(long i, long j) const override { return a[i * n + j]; }
    void set(long i, long j, double v) override { a[i * n + j] = v; }
    void setup() override
    {
        for (long j = 0; j < n; ++j) {
            long p = j;
            double amax = std::fabs(a[j * n + j]);
            for (long i = j + 1; i < n; ++i) {
                if (std::fabs(a[i * n + j]) > amax) {
                    amax = std::fabs(a[i * n + j]);
                    p = i;
                }
            }
            ipiv[j] = p;
            if (a[p * n + j] == 0.0)
                throw std::runtime_error("LAPACKE_dgetrf failed with error code " + std::to_string(j + 1));
            if (p != j)
                for (long k = 0; k < n; ++k) std::swap(a[j * n + k], a[p * n + k]);
            double const inv = 1.0 / a[j * n + j];
            for (long i = j + 1; i < n; ++i) a[i * n + j] *= inv;
            for (long i = j + 1; i < n; ++i) {
                double const l = a[i * n + j];
                if (l != 0.0)
                    for (long k = j + 1; k < n; ++k) a[i * n + k] -= l * a[j * n + k];
            }
        }
    }
    void solve_col(double* b, long ld, bool transpose) const override
    {
        if (n == 0) return;
        auto B = [&](long i) -> double& { return b[i * ld]; };
        if (!transpose) {
            for (long i = 0; i < n; ++i)
                if (ipiv[i] != i) std::swap(B(i), B(ipiv[i]));
            for (long i = 0; i < n; ++i)
                for (long k = 0; k < i; ++k) B(i) -= a[i * n + k] * B(k);
            for (long i = n - 1; i >= 0; --i) {
                for (long k = i + 1; k < n; ++k) B(i) -= a[i * n + k] * B(k);
                B(i) /= a[i * n + i];
            }
        } else {
            for (long i = 0; i < n; ++i) {
                for (long k = 0; k < i; ++k) B(i) -= a[k * n + i] * B(k);
                B(i) /= a[i * n + i];
            }
            for (long i = n - 1; i >= 0; --i)
                for (long k = i + 1; k < n; ++k) B(i) -= a[k * n + i] * B(k);
            for (long i = n - 1; i >= 0; --i)
                if (ipiv[i] != i) std::swap(B(i), B(ipiv[i]));
        }
    }
};

// splines_linear_problem_band.cpp:30-170: dgbtrf (partial pivoting, storage (2kl+ku+1) x n,
// band_storage_row_index = kl+ku+i-j) + SerialGbtrs
struct Band : LinearProblem
{
    long kl, ku;
    std::vector<double> q; // (2kl+ku+1) x n
    std::vector<long> ipiv;
    Band(long n_, long kl_, long ku_) : LinearProblem(n_), kl(kl_), ku(ku_), q((2 * kl_ + ku_ + 1) * n_, 0.0), ipiv(n_, 0) {}
    double& Q(long r, long j) { return q[r * n + j]; }
    double Q(long r, long j) const { return q[r * n + j]; }
    bool in_band(long i, long j) const { return i >= std::max(0L, j - ku) && i < std::min(n, j + kl + 1); }
    double get(long i, long j) const override { return in_band(i, j) ? Q(kl + ku + i - j, j) : 0.0; }
    void set(long i, long j, double v) override
    {
        if (in_band(i, j)) Q(kl + ku + i - j, j) = v;
        // out-of-band entries are dropped (band.cpp:95-97 asserts they are < 1e-15)
    }
    // element (i, j) of the working array in dgbtf2 coordinates: row kv + i - j, kv = ku + kl
    double& W(long i, long j) { return Q(kl + ku + i - j, j); }
    void setup() override
    {
        // Unblocked dgbtf2. The fill-in rows 0..kl-1 of the storage start zeroed.
        long const kv = ku + kl;
        (void)kv;
        long ju = 0;
        for (long j = 0; j < n; ++j) {
            long const km = std::min(kl, n - 1 - j);
            long jp = 0;
            double amax = std::fabs(W(j, j));
            for (long t = 1; t <= km; ++t) {
                if (std::fabs(W(j + t, j)) > amax) {
                    amax = std::fabs(W(j + t, j));
                    jp = t;
                }
            }
            ipiv[j] = j + jp;
            if (W(j + jp, j) == 0.0)
                throw std::runtime_error("LAPACKE_dgbtrf failed with error code " + std::to_string(j + 1));
            ju = std::max(ju, std::min(j + ku + jp, n - 1));
            if (jp != 0)
                for (long c = j; c <= ju; ++c) std::swap(W(j, c), W(j + jp, c));
            if (km > 0) {
                double const inv = 1.0 / W(j, j);
                for (long t = 1; t <= km; ++t) W(j + t, j) *= inv;
                for (long c = j + 1; c <= ju; ++c) {
                    double const u = W(j, c);
                    if (u != 0.0)
                        for (long t = 1; t <= km; ++t) W(j + t, c) -= W(j + t, j) * u;
                }
            }
        }
    }
    void solve_col(double* b, long ld, bool transpose) const override
    {
        auto B = [&](long i) -> double& { return b[i * ld]; };
        long const kd = kl + ku; // storage row of the diagonal
        auto Wc = [&](long i, long j) { return Q(kd + i - j, j); };
        if (!transpose) {
            // L: for each column j apply the interchange, then the rank-1 update (dgbtrs)
            if (kl > 0)
                for (long j = 0; j < n - 1; ++j) {
                    long const lm = std::min(kl, n - j - 1);
                    long const l = ipiv[j];
                    if (l != j) std::swap(B(l), B(j));
                    for (long t = 1; t <= lm; ++t) B(j + t) -= Wc(j + t, j) * B(j);
                }
            // U: upper band with kl+ku superdiagonals (dtbsv upper, no transpose)
            for (long j = n - 1; j >= 0; --j) {
                B(j) /= Wc(j, j);
                double const t = B(j);
                long const i0 = std::max(0L, j - kd);
                for (long i = j - 1; i >= i0; --i) B(i) -= Wc(i, j) * t;
            }
        } else {
            // U^T (dtbsv upper, transpose)
            for (long j = 0; j < n; ++j) {
                double t = B(j);
                long const i0 = std::max(0L, j - kd);
                for (long i = i0; i < j; ++i) t -= Wc(i, j) * B(i);
                B(j) = t / Wc(j, j);
            }
            // L^T with interchanges in reverse order
            if (kl > 0)
                for (long j = n - 2; j >= 0; --j) {
                    long const lm = std::min(kl, n - j - 1);
                    for (long t = 1; t <= lm; ++t) B(j) -= Wc(j + t, j) * B(j + t);
                    long const l = ipiv[j];
                    if (l != j) std::swap(B(l), B(j));
                }
        }
    }
};

// splines_linear_problem_pds_band.cpp:30-120: dpbtrf('L') + SerialPbtrs (lower)
struct PDSBand : LinearProblem
{
    long kd;
    std::vector<double> q; // (kd+1) x n, q[(j-i)*n + i] = A(i,j) for i<=j
    PDSBand(long n_, long kd_) : LinearProblem(n_), kd(kd_), q((kd_ + 1) * n_, 0.0) {}
    double get(long i, long j) const override
    {
        if (i > j) std::swap(i, j);
        return (j - i <= kd) ? q[(j - i) * n + i] : 0.0;
    }
    void set(long i, long j, double v) override
    {
        if (i > j) std::swap(i, j);
        if (j - i <= kd) q[(j - i) * n + i] = v;
    }
    // Lower factor L(i, j), i >= j, stored at q[(i-j)*n + j]
    double& L(long i, long j) { return q[(i - j) * n + j]; }
    double L(long i, long j) const { return q[(i - j) * n + j]; }
    void setup() override
    {
        for (long j = 0; j < n; ++j) {
            double ajj = L(j, j);
            if (ajj <= 0.0)
                throw std::runtime_error("LAPACKE_dpbtrf failed with error code " + std::to_string(j + 1));
            ajj = std::sqrt(ajj);
            L(j, j) = ajj;
            long const kn = std::min(kd, n - 1 - j);
            double const inv = 1.0 / ajj;
            for (long t = 1; t <= kn; ++t) L(j + t, j) *= inv;
            for (long c = 1; c <= kn; ++c)
                for (long r = c; r <= kn; ++r) L(j + r, j + c) -= L(j + r, j) * L(j + c, j);
        }
    }
    void solve_col(double* b, long ld, bool) const override
    {
        auto B = [&](long i) -> double& { return b[i * ld]; };
        for (long i = 0; i < n; ++i) {
            double t = B(i);
            for (long k = std::max(0L, i - kd); k < i; ++k) t -= L(i, k) * B(k);
            B(i) = t / L(i, i);
        }
        for (long i = n - 1; i >= 0; --i) {
            double t = B(i);
            for (long k = i + 1; k <= std::min(n - 1, i + kd); ++k) t -= L(k, i) * B(k);
            B(i) = t / L(i, i);
        }
    }
};

// splines_linear_problem_pds_tridiag.cpp:30-113: dpttrf + SerialPttrs
struct PDSTridiag : LinearProblem
{
    std::vector<double> d, e;
    explicit PDSTridiag(long n_) : LinearProblem(n_), d(n_, 0.0), e(n_, 0.0) {}
    double get(long i, long j) const override
    {
        if (i > j) std::swap(i, j);
        if (j == i) return d[i];
        if (j == i + 1) return e[i];
        return 0.0;
    }
    void set(long i, long j, double v) override
    {
        if (i > j) std::swap(i, j);
        if (j == i) d[i] = v;
        else if (j == i + 1) e[i] = v;
    }
    void setup() override
    {
        for (long i = 0; i < n - 1; ++i) {
            if (d[i] <= 0.0)
                throw std::runtime_error("LAPACKE_dpttrf failed with error code " + std::to_string(i + 1));
            double const ei = e[i];
            e[i] = ei / d[i];
            d[i + 1] -= e[i] * ei;
        }
        if (n > 0 && d[n - 1] <= 0.0)
            throw std::runtime_error("LAPACKE_dpttrf failed with error code " + std::to_string(n));
    }
    void solve_col(double* b, long ld, bool) const override
    {
        auto B = [&](long i) -> double& { return b[i * ld]; };
        for (long i = 1; i < n; ++i) B(i) -= e[i - 1] * B(i - 1);
        B(n - 1) /= d[n - 1];
        for (long i = n - 2; i >= 0; --i) B(i) = B(i) / d[i] - B(i + 1) * e[i];
    }
};

// splines_linear_problem_2x2_blocks.cpp:75-298: [[Q, gamma],[lambda, delta]] with Schur complement
struct Blocks2x2 : LinearProblem
{
    std::unique_ptr<LinearProblem> tl;   // Q
    std::unique_ptr<Dense> br;           // delta, then delta - lambda Q^-1 gamma
    long nq;
    std::vector<double> tr;              // gamma (nq x nb), then Q^-1 gamma
    std::vector<double> bl;              // lambda (nb x nq)
    struct Coo { std::vector<long> r, c; std::vector<double> v; };
    Coo tr_coo, bl_coo;
    Blocks2x2(long n_, std::unique_ptr<LinearProblem> q)
        : LinearProblem(n_), tl(std::move(q)), nq(0)
    {
        nq = tl->n;
        br.reset(new Dense(n - nq));
        tr.assign(nq * (n - nq), 0.0);
        bl.assign((n - nq) * nq, 0.0);
    }
    long nb() const { return n - nq; }
    double get(long i, long j) const override
    {
        if (i < nq && j < nq) return tl->get(i, j);
        if (i >= nq && j >= nq) return br->get(i - nq, j - nq);
        if (j >= nq) return tr[i * nb() + (j - nq)];
        return bl[(i - nq) * nq + j];
    }
    void set(long i, long j, double v) override
    {
        if (i < nq && j < nq) tl->set(i, j, v);
        else if (i >= nq && j >= nq) br->set(i - nq, j - nq, v);
        else if (j >= nq) tr[i * nb() + (j - nq)] = v;
        else bl[(i - nq) * nq + j] = v;
    }
    // dense2coo with tol 1e-14 (2x2_blocks.cpp:146-190, default tol in 2x2_blocks.hpp:90)
    static Coo dense2coo(std::vector<double> const& m, long rows, long cols, double tol = 1e-14)
    {
        Coo c;
        for (long i = 0; i < rows; ++i)
            for (long j = 0; j < cols; ++j)
                if (std::fabs(m[i * cols + j]) >= tol) {
                    c.r.push_back(i);
                    c.c.push_back(j);
                    c.v.push_back(m[i * cols + j]);
                }
        return c;
    }
    void setup() override
    {
        tl->setup();
        if (nb() > 0) tl->solve(tr.data(), nb(), nb(), false, 1);
        tr_coo = dense2coo(tr, nq, nb());
        bl_coo = dense2coo(bl, nb(), nq);
        // compute_schur_complement (2x2_blocks.cpp:192-210)
        for (long i = 0; i < nb(); ++i)
            for (long j = 0; j < nb(); ++j) {
                double val = 0.0;
                for (long l = 0; l < nq; ++l) val += bl[i * nq + l] * tr[l * nb() + j];
                br->set(i, j, br->get(i, j) - val);
            }
        br->setup();
    }
    // spdm_minus1_1 (2x2_blocks.cpp:236-272) on one column
    static void spdm(Coo const& op, double const* x, double* y, long ld, bool transpose)
    {
        for (size_t k = 0; k < op.v.size(); ++k) {
            if (!transpose) y[op.r[k] * ld] -= op.v[k] * x[op.c[k] * ld];
            else y[op.c[k] * ld] -= op.v[k] * x[op.r[k] * ld];
        }
    }
    void solve_col(double* b, long ld, bool transpose) const override
    {
        double* b1 = b;
        double* b2 = b + nq * ld;
        if (!transpose) {
            tl->solve_col(b1, ld, false);
            spdm(bl_coo, b1, b2, ld, false);
            br->solve_col(b2, ld, false);
            spdm(tr_coo, b2, b1, ld, false);
        } else {
            spdm(tr_coo, b1, b2, ld, true);
            br->solve_col(b2, ld, true);
            spdm(bl_coo, b2, b1, ld, true);
            tl->solve_col(b1, ld, true);
        }
    }
    // The reference launches each step as its own batched kernel (thread per column); the
    // per-column fusion here computes identical arithmetic.
};

// splines_linear_problem_3x3_blocks.cpp:18-151: top rows/cols moved behind the centre block
struct Blocks3x3 : Blocks2x2
{
    long top;
    Blocks3x3(long n_, long top_, std::unique_ptr<LinearProblem> center)
        : Blocks2x2(n_, std::move(center)), top(top_) {}
    void adjust(long& i, long& j) const
    {
        if (i < top) i += nq;
        else if (i < top + nq) i -= top;
        if (j < top) j += nq;
        else if (j < top + nq) j -= top;
    }
    double get(long i, long j) const override
    {
        adjust(i, j);
        return Blocks2x2::get(i, j);
    }
    void set(long i, long j, double v) override
    {
        adjust(i, j);
        Blocks2x2::set(i, j, v);
    }
    long required_rows() const override { return n + top; }
    void solve_col(double* b, long ld, bool transpose) const override
    {
        // interchange_rows_from_3_to_2_blocks_rhs (:66-98)
        long const bot = n - top - nq;
        std::vector<double> buf(std::max(bot, top));
        for (long i = 0; i < bot; ++i) buf[i] = b[(top + nq + i) * ld];
        for (long i = 0; i < bot; ++i) b[(2 * top + nq + i) * ld] = buf[i];
        for (long i = 0; i < top; ++i) b[(top + nq + i) * ld] = b[i * ld];
        Blocks2x2::solve_col(b + top * ld, ld, transpose);
        // interchange_rows_from_2_to_3_blocks_rhs (:100-128)
        for (long i = 0; i < top; ++i) b[i * ld] = b[(top + nq + i) * ld];
        for (long i = 0; i < bot; ++i) buf[i] = b[(2 * top + nq + i) * ld];
        for (long i = 0; i < bot; ++i) b[(top + nq + i) * ld] = buf[i];
    }
};

// splines_linear_problem_maker.hpp:56-76
static std::unique_ptr<LinearProblem> make_new_band(long n, long kl, long ku, bool pds)
{
    if (kl == ku && kl == 1 && pds) return std::make_unique<PDSTridiag>(n);
    if (kl == ku && pds) return std::make_unique<PDSBand>(n, kl);
    if (2 * kl + ku + 1 >= n) return std::make_unique<Dense>(n);
    return std::make_unique<Band>(n, kl, ku);
}

// splines_linear_problem_maker.hpp:92-111
static std::unique_ptr<LinearProblem> make_block_with_band_main(long n, long kl, long ku, bool pds, long bottom, long top)
{
    long const main = n - top - bottom;
    auto mb = make_new_band(main, kl, ku, pds);
    if (top == 0) return std::make_unique<Blocks2x2>(n, std::move(mb));
    return std::make_unique<Blocks3x3>(n, top, std::move(mb));
}

// splines_linear_problem_maker.hpp:129-146
static std::unique_ptr<LinearProblem> make_periodic_band(long n, long kl, long ku, bool pds)
{
    long const bottom = std::max(kl, ku);
    long const top = n - bottom;
    if (bottom * (n + top) + (2 * kl + ku + 1) * top >= n * n) return std::make_unique<Dense>(n);
    return make_block_with_band_main(n, kl, ku, pds, bottom, 0);
}

// ------------------------------------------------------------------------------------------------
// SplineBuilder: spline_builder.hpp
// ------------------------------------------------------------------------------------------------
struct Builder
{
    BSplines const* bs;
    std::vector<double> points;
    int bc_lo, bc_hi;
    int nbe_lo, nbe_hi, nbv_lo, nbv_hi;
    int odd;
    long offset = 0;
    double dx;
    std::unique_ptr<LinearProblem> mat;
    std::string structure;
    std::vector<double> assembled; // dense copy of the assembled matrix (for tests)

    Builder(BSplines const* b, double const* pts, long npts, int lo, int hi)
        : bs(b), points(pts, pts + npts), bc_lo(lo), bc_hi(hi)
    {
        int const d = bs->degree;
        if ((lo == PERIODIC) != (hi == PERIODIC)) throw std::runtime_error("Incompatible closure relations");
        if (bs->periodic != (lo == PERIODIC)) throw std::runtime_error("Closure relations do not match the periodicity of the B-splines");
        nbe_lo = n_boundary_equations(lo, d);
        nbe_hi = n_boundary_equations(hi, d);
        nbv_lo = (lo == HOMOGENEOUS_HERMITE) ? 0 : nbe_lo;
        nbv_hi = (hi == HOMOGENEOUS_HERMITE) ? 0 : nbe_hi;
        odd = d % 2;
        dx = (bs->rmax() - bs->rmin()) / double(bs->ncells()); // spline_builder.hpp:233-234
        check_valid_grid();
        compute_offset();
        // block sizes (spline_builder.hpp:241-253, 668-709)
        int upper_block, lower_block;
        if (bs->uniform) {
            upper_block = block_uniform(lo, nbe_lo);
            lower_block = block_uniform(hi, nbe_hi);
        } else {
            upper_block = block_non_uniform(lo, nbe_lo);
            lower_block = block_non_uniform(hi, nbe_hi);
        }
        // allocate_matrix LAPACK branch (spline_builder.hpp:740-763)
        long const ubw = bs->uniform ? d / 2 : d - 1;
        long const nb = bs->nbasis();
        if (bs->periodic) mat = make_periodic_band(nb, ubw, ubw, bs->uniform);
        else mat = make_block_with_band_main(nb, ubw, ubw, bs->uniform, lower_block, upper_block);
        describe();
        build_matrix_system();
        assembled.assign(nb * nb, 0.0);
        for (long i = 0; i < nb; ++i)
            for (long j = 0; j < nb; ++j) assembled[i * nb + j] = mat->get(i, j);
        mat->setup();
    }

    void describe()
    {
        structure = describe_lp(mat.get());
    }
    static std::string describe_lp(LinearProblem const* p)
    {
        if (auto q = dynamic_cast<Blocks3x3 const*>(p))
            return "3x3(top=" + std::to_string(q->top) + ",bottom=" + std::to_string(q->nb() - q->top) + ",Q=" + describe_lp(q->tl.get()) + ")";
        if (auto q = dynamic_cast<Blocks2x2 const*>(p))
            return "2x2(bottom=" + std::to_string(q->nb()) + ",Q=" + describe_lp(q->tl.get()) + ")";
        if (dynamic_cast<PDSTridiag const*>(p)) return "PDSTridiag(" + std::to_string(p->n) + ")";
        if (auto q = dynamic_cast<PDSBand const*>(p)) return "PDSBand(" + std::to_string(p->n) + ",kd=" + std::to_string(q->kd) + ")";
        if (auto q = dynamic_cast<Band const*>(p)) return "Band(" + std::to_string(p->n) + ",kl=" + std::to_string(q->kl) + ",ku=" + std::to_string(q->ku) + ")";
        if (dynamic_cast<Dense const*>(p)) return "Dense(" + std::to_string(p->n) + ")";
        return "?";
    }

    // spline_builder.hpp:668-685
    int block_uniform(int bc, int nbc) const
    {
        if (bc == PERIODIC) return bs->degree / 2;
        if (bc == HERMITE || bc == HOMOGENEOUS_HERMITE) return nbc;
        return bs->degree - 1; // GREVILLE
    }
    // spline_builder.hpp:695-709
    int block_non_uniform(int bc, int nbc) const
    {
        if (bc == PERIODIC || bc == GREVILLE) return bs->degree - 1;
        return nbc + 1; // HERMITE, HOMOGENEOUS_HERMITE
    }

    // spline_builder.hpp:1244-1317
    void check_valid_grid()
    {
        long const expected = bs->nbasis() - nbe_lo - nbe_hi;
        if (long(points.size()) != expected)
            throw std::runtime_error("Incorrect number of points supplied to NonUniformInterpolationPoints. (Received : "
                                     + std::to_string(points.size()) + ", expected : " + std::to_string(expected));
        int n_in_cell = 0;
        long cell_end = bs->degree + 1; // knot index of break_point_domain.front() + 1
        auto check = [&](int npc, long cend) {
            if (npc > bs->degree + 1) {
                long const failed = cend - bs->degree;
                throw std::runtime_error("The spline problem is overconstrained. There are " + std::to_string(npc)
                                         + " points in the " + std::to_string(failed) + "-th cell.");
            }
        };
        for (double p : points) {
            double const ce = bs->knot(cell_end);
            if (p > ce) {
                check(n_in_cell, cell_end);
                n_in_cell = 1;
                cell_end += 1;
            } else if (p == ce) {
                check(n_in_cell + 1, cell_end);
                n_in_cell = 1;
                cell_end += 1;
            } else {
                n_in_cell += 1;
            }
        }
        check(n_in_cell, cell_end);
    }

    // spline_builder.hpp:619-658
    void compute_offset()
    {
        offset = 0;
        if (!bs->periodic) return;
        int const d = bs->degree;
        double values[10];
        long const jmin = bs->eval_basis(values, points[d], d);
        if (d % 2 == 0) {
            offset = jmin - 0 + d / 2 - d;
        } else {
            int const mid = d / 2;
            offset = jmin - 0 + (values[mid] > values[mid + 1] ? mid : mid + 1) - d;
        }
    }

    // spline_builder.hpp:784-886
    void build_matrix_system()
    {
        int const d = bs->degree;
        long const nb = bs->nbasis();
        int const nc = d / 2 + 1;
        if (bc_lo == HERMITE || bc_lo == HOMOGENEOUS_HERMITE) {
            std::vector<double> derivs((d + 1) * nc, 0.0);
            bs->eval_basis_and_n_derivs(derivs.data(), bs->rmin(), nbe_lo);
            // the reference's derivs span is (d+1) x (d/2+1); A2.3 fills columns 0..nbe
            std::vector<double> dv((d + 1) * nc, 0.0);
            for (int i = 0; i < d + 1; ++i)
                for (int k = 0; k <= nbe_lo; ++k) dv[i * nc + k] = derivs[i * (nbe_lo + 1) + k];
            for (int i = 0; i < d + 1; ++i)
                for (int j = 1; j < nc; ++j) dv[i * nc + j] *= ipow(dx, j);
            for (int i = 0; i < nbe_lo; ++i)
                for (int j = 0; j < d; ++j) mat->set(i, j, dv[j * nc + i + odd]);
        }
        double values[10];
        for (size_t ix = 0; ix < points.size(); ++ix) {
            long const jmin = bs->eval_basis(values, points[ix], d);
            for (int s = 0; s < d + 1; ++s) {
                long const j = modulo(jmin - offset + s, nb);
                mat->set(long(ix) + nbe_lo, j, values[s]);
            }
        }
        if (bc_hi == HERMITE || bc_hi == HOMOGENEOUS_HERMITE) {
            std::vector<double> derivs((d + 1) * (nbe_hi + 1), 0.0);
            bs->eval_basis_and_n_derivs(derivs.data(), bs->rmax(), nbe_hi);
            std::vector<double> dv((d + 1) * nc, 0.0);
            for (int i = 0; i < d + 1; ++i)
                for (int k = 0; k <= nbe_hi; ++k) dv[i * nc + k] = derivs[i * (nbe_hi + 1) + k];
            for (int i = 0; i < d + 1; ++i)
                for (int j = 1; j < nc; ++j) dv[i * nc + j] *= ipow(dx, j);
            long const i0 = nb - nbe_hi;
            long const j0 = nb - d;
            for (int j = 0; j < d; ++j)
                for (int i = 0; i < nbe_hi; ++i) mat->set(i0 + i, j0 + j, dv[(j + 1) * nc + i + odd]);
        }
    }

    // SplineBuilder::operator() (spline_builder.hpp:896-1101), reference schedule:
    // copy passes K1/K2, transposed scratch K3, batched solve, transpose back K10, periodic
    // duplication K11, each a full pass parallel over lines. Arrays in (row, line) layout.
    void build(double* spline, double const* vals, double const* dlo, double const* dhi, long B, int nthreads) const
    {
        if (B == 0) return;
        int const d = bs->degree;
        long const nb = bs->nbasis();
        long const np = long(points.size());
        long const off = offset;
        // K1 lower Hermite rows
        if (bc_lo == HERMITE) {
#pragma omp parallel for num_threads(nthreads) schedule(static)
            for (long j = 0; j < B; ++j)
                for (int i = 0; i < nbe_lo; ++i) spline[i * B + j] = dlo[i * B + j] * ipow(dx, i + odd);
        } else if (bc_lo == HOMOGENEOUS_HERMITE) {
            for (int i = 0; i < nbe_lo; ++i) std::fill(spline + i * B, spline + (i + 1) * B, 0.0);
        }
        // K2 zero the offset rows, copy the values
        for (long i = 0; i < off; ++i) std::fill(spline + (nbe_lo + i) * B, spline + (nbe_lo + i + 1) * B, 0.0);
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (long i = 0; i < np; ++i) std::memcpy(spline + (nbe_lo + off + i) * B, vals + i * B, sizeof(double) * B);
        // K1 upper Hermite rows
        if (bc_hi == HERMITE) {
#pragma omp parallel for num_threads(nthreads) schedule(static)
            for (long j = 0; j < B; ++j)
                for (int i = 0; i < nbe_hi; ++i) spline[(nb - nbe_hi + i) * B + j] = dhi[i * B + j] * ipow(dx, i + odd);
        } else if (bc_hi == HOMOGENEOUS_HERMITE) {
            for (int i = 0; i < nbe_hi; ++i) std::fill(spline + (nb - nbe_hi + i) * B, spline + (nb - nbe_hi + i + 1) * B, 0.0);
        }
        // K3 per-call scratch, transpose (a shifted copy in this layout)
        long const rows = mat->required_rows();
        std::vector<double> tr(size_t(rows) * size_t(B), 0.0);
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (long j = 0; j < B; ++j)
            for (long i = 0; i < nb; ++i) tr[i * B + j] = spline[(i + off) * B + j];
        // batched solve, thread per column
        mat->solve(tr.data(), B, B, false, nthreads);
        // K10 transpose back
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (long j = 0; j < B; ++j)
            for (long i = 0; i < nb; ++i) spline[(i + off) * B + j] = tr[i * B + j];
        // K11 periodic duplication
        if (bs->periodic) {
#pragma omp parallel for num_threads(nthreads) schedule(static)
            for (long j = 0; j < B; ++j) {
                if (off != 0) {
                    for (long i = 0; i < off; ++i) spline[i * B + j] = spline[(nb + i) * B + j];
                    for (long i = off; i < d; ++i) spline[(nb + i) * B + j] = spline[i * B + j];
                }
                for (long i = 0; i < d; ++i) spline[(nb + i) * B + j] = spline[i * B + j];
            }
        }
    }

    // quadrature_coefficients (spline_builder.hpp:1103-1234): solve A^T q = integrals
    void quadrature(double* qlo, double* q, double* qhi) const
    {
        long const nb = bs->nbasis();
        std::vector<double> ints(bs->size());
        bs->integrals(ints.data());
        std::vector<double> rhs(mat->required_rows(), 0.0);
        for (long i = 0; i < mat->n; ++i) rhs[i] = ints[i];
        mat->solve_col(rhs.data(), 1, true);
        for (int i = 0; i < nbv_lo; ++i) qlo[i] = rhs[i] * ipow(dx, i + odd);
        long const ncoef = nb - nbv_lo - nbv_hi;
        for (long i = 0; i < ncoef; ++i) q[i] = rhs[nbv_lo + i];
        for (int i = 0; i < nbv_hi; ++i) qhi[i] = rhs[nbv_lo + ncoef + i] * ipow(dx, i + odd);
    }
};

// ------------------------------------------------------------------------------------------------
// SplineEvaluator: spline_evaluator.hpp:257-605 and the extrapolation rules
// ------------------------------------------------------------------------------------------------
// eval_no_bc (spline_evaluator.hpp:556-605); coefs of one line with stride ld
static double eval_no_bc(BSplines const& bs, int order, double x, double const* c, long ld)
{
    int const d = bs.degree;
    double vals[10];
    long jmin;
    if (order == 0) {
        jmin = bs.eval_basis(vals, x, d);
    } else {
        double derivs[10 * 10];
        jmin = bs.eval_basis_and_n_derivs(derivs, x, order);
        for (int i = 0; i < d + 1; ++i) vals[i] = derivs[i * (order + 1) + order];
    }
    double y = 0.0;
    for (int i = 0; i < d + 1; ++i) y += c[(jmin + i) * ld] * vals[i];
    return y;
}

// eval (spline_evaluator.hpp:529-554) with periodic wrap / extrapolation rules
// (null_extrapolation_rule.hpp:14-26, constant_extrapolation_rule.hpp:27-52)
static double eval_bc(BSplines const& bs, int ex_lo, int ex_hi, double x, double const* c, long ld)
{
    if (bs.periodic) {
        if (x < bs.rmin() || x > bs.rmax()) x -= std::floor((x - bs.rmin()) / bs.length()) * bs.length();
    } else {
        if (x < bs.rmin()) {
            if (ex_lo == EX_NULL) return 0.0;
            return eval_no_bc(bs, 0, bs.rmin(), c, ld);
        }
        if (x > bs.rmax()) {
            if (ex_hi == EX_NULL) return 0.0;
            return eval_no_bc(bs, 0, bs.rmax(), c, ld);
        }
    }
    return eval_no_bc(bs, 0, x, c, ld);
}

// ------------------------------------------------------------------------------------------------
// 2D tensor-product builder/evaluator: spline_builder_2d.hpp:526-651, spline_evaluator_2d.hpp
// Arrays (x1, x2, batch) row-major, batch contiguous.
// ------------------------------------------------------------------------------------------------
static double eval2d_no_bc(BSplines const& b1, BSplines const& b2, int o1, int o2, double x1, double x2,
                           double const* c, long ld1, long ld2)
{
    double v1[10], v2[10];
    long j1, j2;
    int const d1 = b1.degree, d2 = b2.degree;
    if (o1 == 0) j1 = b1.eval_basis(v1, x1, d1);
    else {
        double t[100];
        j1 = b1.eval_basis_and_n_derivs(t, x1, o1);
        for (int i = 0; i < d1 + 1; ++i) v1[i] = t[i * (o1 + 1) + o1];
    }
    if (o2 == 0) j2 = b2.eval_basis(v2, x2, d2);
    else {
        double t[100];
        j2 = b2.eval_basis_and_n_derivs(t, x2, o2);
        for (int i = 0; i < d2 + 1; ++i) v2[i] = t[i * (o2 + 1) + o2];
    }
    double y = 0.0;
    for (int i = 0; i < d1 + 1; ++i)
        for (int j = 0; j < d2 + 1; ++j) y += c[(j1 + i) * ld1 + (j2 + j) * ld2] * v1[i] * v2[j];
    return y;
}

static double eval2d_bc(BSplines const& b1, BSplines const& b2, int ex1lo, int ex1hi, int ex2lo, int ex2hi,
                        double x1, double x2, double const* c, long ld1, long ld2)
{
    if (b1.periodic && (x1 < b1.rmin() || x1 > b1.rmax())) x1 -= std::floor((x1 - b1.rmin()) / b1.length()) * b1.length();
    if (b2.periodic && (x2 < b2.rmin() || x2 > b2.rmax())) x2 -= std::floor((x2 - b2.rmin()) / b2.length()) * b2.length();
    // constant_extrapolation_rule.hpp:143-193: evaluate at the boundary in the interest dim,
    // clamp (non-periodic) or keep (periodic) the other coordinate.
    auto clamp = [](double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); };
    if (!b1.periodic) {
        if (x1 < b1.rmin()) {
            if (ex1lo == EX_NULL) return 0.0;
            double const y2 = b2.periodic ? x2 : clamp(x2, b2.rmin(), b2.rmax());
            return eval2d_no_bc(b1, b2, 0, 0, b1.rmin(), y2, c, ld1, ld2);
        }
        if (x1 > b1.rmax()) {
            if (ex1hi == EX_NULL) return 0.0;
            double const y2 = b2.periodic ? x2 : clamp(x2, b2.rmin(), b2.rmax());
            return eval2d_no_bc(b1, b2, 0, 0, b1.rmax(), y2, c, ld1, ld2);
        }
    }
    if (!b2.periodic) {
        if (x2 < b2.rmin()) {
            if (ex2lo == EX_NULL) return 0.0;
            double const y1 = b1.periodic ? x1 : clamp(x1, b1.rmin(), b1.rmax());
            return eval2d_no_bc(b1, b2, 0, 0, y1, b2.rmin(), c, ld1, ld2);
        }
        if (x2 > b2.rmax()) {
            if (ex2hi == EX_NULL) return 0.0;
            double const y1 = b1.periodic ? x1 : clamp(x1, b1.rmin(), b1.rmax());
            return eval2d_no_bc(b1, b2, 0, 0, y1, b2.rmax(), c, ld1, ld2);
        }
    }
    return eval2d_no_bc(b1, b2, 0, 0, x1, x2, c, ld1, ld2);
}

} // namespace oracle

// ================================================================================================
// C interface (ctypes). Errors: functions returning a handle return nullptr and write the
// message into orc_last_error().
// ================================================================================================
using namespace oracle;

static thread_local std::string g_err;

extern "C" {

char const* orc_last_error() { return g_err.c_str(); }

void* orc_bsplines_uniform(int degree, int periodic, double rmin, double rmax, long ncells)
{
    try {
        if (degree < 1 || degree > 7 || ncells < 1 || !(rmin < rmax)) throw std::runtime_error("invalid uniform B-spline parameters");
        return make_uniform(degree, periodic != 0, rmin, rmax, ncells).release();
    } catch (std::exception const& e) {
        g_err = e.what();
        return nullptr;
    }
}

void* orc_bsplines_non_uniform(int degree, int periodic, double const* breaks, long nbreaks)
{
    try {
        if (degree < 1 || degree > 7 || nbreaks < 2) throw std::runtime_error("invalid non-uniform B-spline parameters");
        return make_non_uniform(degree, periodic != 0, breaks, nbreaks).release();
    } catch (std::exception const& e) {
        g_err = e.what();
        return nullptr;
    }
}

void orc_bsplines_free(void* p) { delete static_cast<BSplines*>(p); }

// info: [degree, periodic, uniform, ncells, nbasis, size]; rminmax: [rmin, rmax]
void orc_bsplines_info(void* p, long* info, double* rminmax)
{
    auto* bs = static_cast<BSplines*>(p);
    info[0] = bs->degree;
    info[1] = bs->periodic;
    info[2] = bs->uniform;
    info[3] = bs->ncells();
    info[4] = bs->nbasis();
    info[5] = bs->size();
    rminmax[0] = bs->rmin();
    rminmax[1] = bs->rmax();
}

double orc_knot(void* p, long k) { return static_cast<BSplines*>(p)->knot(k); }

long orc_eval_basis(void* p, double x, double* vals)
{
    auto* bs = static_cast<BSplines*>(p);
    return bs->eval_basis(vals, x, bs->degree);
}

long orc_eval_basis_and_n_derivs(void* p, double x, int n, double* out)
{
    return static_cast<BSplines*>(p)->eval_basis_and_n_derivs(out, x, n);
}

void orc_integrals(void* p, double* out) { static_cast<BSplines*>(p)->integrals(out); }

long orc_greville(void* p, int lo, int hi, double* out, long cap)
{
    try {
        auto pts = greville_points(*static_cast<BSplines*>(p), lo, hi);
        if (long(pts.size()) > cap) return -1;
        std::copy(pts.begin(), pts.end(), out);
        return long(pts.size());
    } catch (std::exception const& e) {
        g_err = e.what();
        return -1;
    }
}

void* orc_builder_create(void* bsp, double const* pts, long npts, int lo, int hi)
{
    try {
        return new Builder(static_cast<BSplines*>(bsp), pts, npts, lo, hi);
    } catch (std::exception const& e) {
        g_err = e.what();
        return nullptr;
    }
}

void orc_builder_free(void* p) { delete static_cast<Builder*>(p); }

// info: [offset, nbe_lo, nbe_hi, nbv_lo, nbv_hi, required_rows, npoints]
void orc_builder_info(void* p, long* info, double* dx)
{
    auto* b = static_cast<Builder*>(p);
    info[0] = b->offset;
    info[1] = b->nbe_lo;
    info[2] = b->nbe_hi;
    info[3] = b->nbv_lo;
    info[4] = b->nbv_hi;
    info[5] = b->mat->required_rows();
    info[6] = long(b->points.size());
    *dx = b->dx;
}

long orc_builder_structure(void* p, char* out, long cap)
{
    auto* b = static_cast<Builder*>(p);
    long const n = std::min<long>(cap - 1, long(b->structure.size()));
    std::memcpy(out, b->structure.data(), n);
    out[n] = 0;
    return n;
}

void orc_builder_matrix(void* p, double* out)
{
    auto* b = static_cast<Builder*>(p);
    std::copy(b->assembled.begin(), b->assembled.end(), out);
}

void orc_build(void* p, double* spline, double const* vals, double const* dlo, double const* dhi, long B, int nthreads)
{
    static_cast<Builder*>(p)->build(spline, vals, dlo, dhi, B, nthreads);
}

// In-place solve of rhs (required_rows x B) through the builder's linear problem.
void orc_solve(void* p, double* rhs, long B, int transpose, int nthreads)
{
    auto* b = static_cast<Builder*>(p);
    b->mat->solve(rhs, B, B, transpose != 0, nthreads);
}

void orc_quadrature(void* p, double* qlo, double* q, double* qhi) { static_cast<Builder*>(p)->quadrature(qlo, q, qhi); }

// Batched evaluation: coords/out (m x B), coefs (size x B). order<0: eval with BCs, else deriv.
void orc_eval(void* bsp, int order, int ex_lo, int ex_hi, double const* coords, double const* coefs, double* out,
              long m, long B, int nthreads)
{
    auto const& bs = *static_cast<BSplines*>(bsp);
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (long j = 0; j < B; ++j)
        for (long i = 0; i < m; ++i) {
            double const x = coords[i * B + j];
            out[i * B + j] = order < 0 ? eval_bc(bs, ex_lo, ex_hi, x, coefs + j, B) : eval_no_bc(bs, order, x, coefs + j, B);
        }
}

// integrate (spline_evaluator.hpp:493-526): out[j] = sum_i coefs[i, j] * integral(B_i)
void orc_integrate(void* bsp, double const* coefs, double* out, long B, int nthreads)
{
    auto const& bs = *static_cast<BSplines*>(bsp);
    std::vector<double> ints(bs.size());
    bs.integrals(ints.data());
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (long j = 0; j < B; ++j) {
        double s = 0.0;
        for (long i = 0; i < bs.size(); ++i) s += coefs[i * B + j] * ints[i];
        out[j] = s;
    }
}

// 2D builder (spline_builder_2d.hpp:526-651). Layout (x1, x2, batch), batch contiguous.
//   vals:     (np1, np2, B)
//   dmin1/dmax1: (nbv1, np2, B) derivs in dim1;  dmin2/dmax2: (np1, nbv2, B) derivs in dim2
//   mixed (4 corners): (nbv1, nbv2, B)
//   spline:   (size1, size2, B)
void orc_build2d(void* p1, void* p2, double* spline, double const* vals, double const* dmin1, double const* dmax1,
                 double const* dmin2, double const* dmax2, double const* m11, double const* m21, double const* m12,
                 double const* m22, long B, int nthreads)
{
    auto* b1 = static_cast<Builder*>(p1);
    auto* b2 = static_cast<Builder*>(p2);
    long const s1 = b1->bs->size();
    long const s2 = b2->bs->size();
    long const np2 = long(b2->points.size());
    int const nbv2lo = b2->nbv_lo, nbv2hi = b2->nbv_hi;
    // builder1 runs on lines along x1 with batch (x2, B) flattened: (np1, np2*B) layout matches.
    std::vector<double> spline1(size_t(s1) * np2 * B, 0.0);
    b1->build(spline1.data(), vals, dmin1, dmax1, np2 * B, nthreads);
    std::vector<double> s1dmin, s1dmax;
    if (b2->bc_lo == HERMITE) {
        s1dmin.assign(size_t(s1) * nbv2lo * B, 0.0);
        b1->build(s1dmin.data(), dmin2, m11, m21, nbv2lo * B, nthreads);
    }
    if (b2->bc_hi == HERMITE) {
        s1dmax.assign(size_t(s1) * nbv2hi * B, 0.0);
        b1->build(s1dmax.data(), dmax2, m12, m22, nbv2hi * B, nthreads);
    }
    // builder2 on lines along x2: for each x1-coefficient row r, a (np2, B) slab.
    for (long r = 0; r < s1; ++r) {
        b2->build(spline + r * s2 * B, spline1.data() + r * np2 * B,
                  s1dmin.empty() ? nullptr : s1dmin.data() + r * nbv2lo * B,
                  s1dmax.empty() ? nullptr : s1dmax.data() + r * nbv2hi * B, B, nthreads);
    }
}

// 2D evaluation: coords1/coords2/out (n1, n2, B) flattened as (m, B) with m = n1*n2 points per
// field; coefs (size1, size2, B). order1/order2 < 0 means value with boundary handling.
void orc_eval2d(void* bs1p, void* bs2p, int o1, int o2, int ex1lo, int ex1hi, int ex2lo, int ex2hi,
                double const* c1, double const* c2, double const* coefs, double* out, long m, long B, int nthreads)
{
    auto const& b1 = *static_cast<BSplines*>(bs1p);
    auto const& b2 = *static_cast<BSplines*>(bs2p);
    long const s2 = b2.size();
    long const ld2 = B, ld1 = s2 * B;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (long j = 0; j < B; ++j)
        for (long i = 0; i < m; ++i) {
            double const x1 = c1[i * B + j], x2 = c2[i * B + j];
            out[i * B + j] = (o1 < 0) ? eval2d_bc(b1, b2, ex1lo, ex1hi, ex2lo, ex2hi, x1, x2, coefs + j, ld1, ld2)
                                      : eval2d_no_bc(b1, b2, o1, o2, x1, x2, coefs + j, ld1, ld2);
        }
}

// Reference linear problems on a user matrix (tests/splines/splines_linear_problem.cpp).
// kind: 0 dense, 1 band(kl,ku), 2 pds band(kl), 3 pds tridiag, 4 maker band(kl,ku,pds),
//       5 block band main (kl,ku,pds,bottom,top), 6 periodic band (kl,ku,pds)
void* orc_lp_create(int kind, long n, long kl, long ku, int pds, long bottom, long top)
{
    try {
        LinearProblem* p = nullptr;
        switch (kind) {
        case 0: p = new Dense(n); break;
        case 1: p = new Band(n, kl, ku); break;
        case 2: p = new PDSBand(n, kl); break;
        case 3: p = new PDSTridiag(n); break;
        case 4: p = make_new_band(n, kl, ku, pds != 0).release(); break;
        case 5: p = make_block_with_band_main(n, kl, ku, pds != 0, bottom, top).release(); break;
        case 6: p = make_periodic_band(n, kl, ku, pds != 0).release(); break;
        case 7: p = new Blocks2x2(n, std::make_unique<Dense>(n - bottom)); break;
        case 8: p = new Blocks3x3(n, top, std::make_unique<Dense>(n - bottom - top)); break;
        default: throw std::runtime_error("unknown linear problem kind");
        }
        return p;
    } catch (std::exception const& e) {
        g_err = e.what();
        return nullptr;
    }
}
void orc_lp_free(void* p) { delete static_cast<LinearProblem*>(p); }
void orc_lp_set(void* p, long i, long j, double v) { static_cast<LinearProblem*>(p)->set(i, j, v); }
double orc_lp_get(void* p, long i, long j) { return static_cast<LinearProblem*>(p)->get(i, j); }
long orc_lp_required_rows(void* p) { return static_cast<LinearProblem*>(p)->required_rows(); }
int orc_lp_setup(void* p)
{
    try {
        static_cast<LinearProblem*>(p)->setup();
        return 0;
    } catch (std::exception const& e) {
        g_err = e.what();
        return 1;
    }
}
void orc_lp_solve(void* p, double* b, long ncols, int transpose)
{
    static_cast<LinearProblem*>(p)->solve(b, ncols, ncols, transpose != 0, 1);
}
long orc_lp_describe(void* p, char* out, long cap)
{
    std::string const s = Builder::describe_lp(static_cast<LinearProblem*>(p));
    long const n = std::min<long>(cap - 1, long(s.size()));
    std::memcpy(out, s.data(), n);
    out[n] = 0;
    return n;
}

int orc_max_threads()
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

} // extern "C"
