// ddcb.hpp -- C++ face of the C-ABI in ddcb.h, with the reference's class names and argument order
// (ddc::SplineBuilder, ddc::SplineEvaluator, ddc::SplineBuilder2D; src/ddc/kernels/splines/),
// for host code that keeps DDC's calling shape while the work runs in libddcb.so.
//
// The classes own their handles (move-only, like SplineBuilder, spline_builder.hpp:352-372) and
// turn every failing status into std::runtime_error carrying the library's message, the error
// type the reference throws at construction (spline_builder.hpp:227-260). Data are device pointers
// with a ddcb_lines layout; `lines_xb` and `lines_bx` build the two common ones. An adapter that
// owns DDC ChunkSpans fills the layout from the span's extents and strides.
#pragma once

#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "ddcb.h"

namespace ddcb {

inline void check(ddcb_status s)
{
    if (s != DDCB_SUCCESS) throw std::runtime_error(std::string(ddcb_status_string(s)) + ": " + ddcb_last_error_message());
}

// (x, batch) row-major: the dimension of interest first, nbatch contiguous lines.
inline ddcb_lines lines_xb(int64_t n, int64_t nbatch) { return ddcb_lines {n, nbatch, nbatch, 1, 0}; }
// (batch, x) row-major: one line per row of n contiguous values.
inline ddcb_lines lines_bx(int64_t n, int64_t nbatch) { return ddcb_lines {n, 1, 1, nbatch, n}; }

enum class SplineBuilderClosure { PERIODIC = DDCB_PERIODIC, HERMITE = DDCB_HERMITE,
                                  HOMOGENEOUS_HERMITE = DDCB_HOMOGENEOUS_HERMITE, GREVILLE = DDCB_GREVILLE };
enum class Extrapolation { PERIODIC = DDCB_EXTRAP_PERIODIC, NULL_VALUE = DDCB_EXTRAP_NULL, CONSTANT = DDCB_EXTRAP_CONSTANT };

template <class H, ddcb_status (*Destroy)(H)>
class Handle
{
public:
    Handle() = default;
    explicit Handle(H h) : m_h(h) {}
    Handle(Handle const&) = delete;
    Handle& operator=(Handle const&) = delete;
    Handle(Handle&& o) noexcept : m_h(std::exchange(o.m_h, nullptr)) {}
    Handle& operator=(Handle&& o) noexcept
    {
        if (this != &o) {
            reset();
            m_h = std::exchange(o.m_h, nullptr);
        }
        return *this;
    }
    ~Handle() { reset(); }
    H get() const { return m_h; }

private:
    void reset()
    {
        if (m_h) Destroy(m_h);
        m_h = nullptr;
    }
    H m_h = nullptr;
};

// UniformBSplines / NonUniformBSplines (bsplines_uniform.hpp, bsplines_non_uniform.hpp).
class BSplines
{
public:
    static BSplines uniform(int degree, bool periodic, double rmin, double rmax, int64_t ncells)
    {
        ddcb_bsplines h = nullptr;
        check(ddcb_bsplines_create_uniform(degree, periodic ? 1 : 0, rmin, rmax, ncells, &h));
        return BSplines(h);
    }
    static BSplines non_uniform(int degree, bool periodic, std::vector<double> const& breaks)
    {
        ddcb_bsplines h = nullptr;
        check(ddcb_bsplines_create_non_uniform(degree, periodic ? 1 : 0, breaks.data(), int64_t(breaks.size()), &h));
        return BSplines(h);
    }
    ddcb_bsplines get() const { return m_h.get(); }
    ddcb_bsplines_info info() const
    {
        ddcb_bsplines_info i {};
        check(ddcb_bsplines_get_info(get(), &i));
        return i;
    }
    // GrevilleInterpolationPoints<BSplines, lo, hi>::get_sampling() (greville_interpolation_points.hpp)
    std::vector<double> greville_points(SplineBuilderClosure lo, SplineBuilderClosure hi) const
    {
        std::vector<double> pts(size_t(info().nbasis + 2));
        int64_t n = 0;
        check(ddcb_greville_points(get(), ddcb_closure(lo), ddcb_closure(hi), pts.data(), int64_t(pts.size()), &n));
        pts.resize(size_t(n));
        return pts;
    }

private:
    explicit BSplines(ddcb_bsplines h) : m_h(h) {}
    Handle<ddcb_bsplines, ddcb_bsplines_destroy> m_h;
};

// SplineBuilder<ExecSpace, MemorySpace, BSplines, InterpolationDDim, lo, hi, Solver>
// (spline_builder.hpp:57-65); the device plan lives on the CUDA device current at construction.
class SplineBuilder
{
public:
    SplineBuilder(BSplines const& bs, SplineBuilderClosure lo, SplineBuilderClosure hi, ddcb_builder_options const* options = nullptr)
        : SplineBuilder(bs, bs.greville_points(lo, hi), lo, hi, options)
    {
    }
    SplineBuilder(BSplines const& bs, std::vector<double> const& interpolation_points, SplineBuilderClosure lo,
                  SplineBuilderClosure hi, ddcb_builder_options const* options = nullptr)
    {
        ddcb_builder h = nullptr;
        check(ddcb_builder_create(bs.get(), interpolation_points.data(), int64_t(interpolation_points.size()), ddcb_closure(lo),
                                  ddcb_closure(hi), options, &h));
        m_h = Handle<ddcb_builder, ddcb_builder_destroy>(h);
    }
    ddcb_builder get() const { return m_h.get(); }
    ddcb_builder_info info() const
    {
        ddcb_builder_info i {};
        check(ddcb_builder_get_info(get(), &i));
        return i;
    }
    // operator()(spline, vals, derivs_xmin, derivs_xmax) (spline_builder.hpp:538-557)
    void operator()(double* spline, ddcb_lines spline_layout, double const* vals, ddcb_lines vals_layout,
                    double const* derivs_xmin = nullptr, ddcb_lines derivs_xmin_layout = {}, double const* derivs_xmax = nullptr,
                    ddcb_lines derivs_xmax_layout = {}, ddcb_stream stream = nullptr) const
    {
        check(ddcb_build(get(), spline, spline_layout, vals, vals_layout, derivs_xmin, derivs_xmin_layout, derivs_xmax,
                         derivs_xmax_layout, stream));
    }
    // quadrature_coefficients() (spline_builder.hpp:1103-1234): (lower derivatives, values, upper derivatives)
    void quadrature_coefficients(std::vector<double>& q_lo, std::vector<double>& q, std::vector<double>& q_hi) const
    {
        ddcb_builder_info const i = info();
        q_lo.assign(size_t(i.nbv_lo) + 1, 0.0);
        q.assign(size_t(i.nbasis - i.nbv_lo - i.nbv_hi), 0.0);
        q_hi.assign(size_t(i.nbv_hi) + 1, 0.0);
        check(ddcb_quadrature_coefficients(get(), q_lo.data(), q.data(), q_hi.data()));
        q_lo.resize(size_t(i.nbv_lo));
        q_hi.resize(size_t(i.nbv_hi));
    }

private:
    Handle<ddcb_builder, ddcb_builder_destroy> m_h;
};

// SplineEvaluator<ExecSpace, MemorySpace, BSplines, EvaluationDDim, LowerRule, UpperRule>
// (spline_evaluator.hpp:160-186).
class SplineEvaluator
{
public:
    SplineEvaluator(BSplines const& bs, Extrapolation lo = Extrapolation::NULL_VALUE, Extrapolation hi = Extrapolation::NULL_VALUE)
    {
        ddcb_evaluator h = nullptr;
        check(ddcb_evaluator_create(bs.get(), ddcb_extrapolation(lo), ddcb_extrapolation(hi), &h));
        m_h = Handle<ddcb_evaluator, ddcb_evaluator_destroy>(h);
    }
    ddcb_evaluator get() const { return m_h.get(); }
    // operator()(spline_eval, coords_eval, spline_coef) (spline_evaluator.hpp:257-294)
    void operator()(double* spline_eval, ddcb_lines eval_layout, double const* coords_eval, ddcb_lines coords_layout,
                    double const* spline_coef, ddcb_lines coef_layout, ddcb_stream stream = nullptr) const
    {
        check(ddcb_eval(get(), spline_eval, eval_layout, coords_eval, coords_layout, spline_coef, coef_layout, stream));
    }
    // deriv(order, spline_eval, coords_eval, spline_coef) (spline_evaluator.hpp:357-478)
    void deriv(int order, double* spline_eval, ddcb_lines eval_layout, double const* coords_eval, ddcb_lines coords_layout,
               double const* spline_coef, ddcb_lines coef_layout, ddcb_stream stream = nullptr) const
    {
        check(ddcb_eval_deriv(get(), order, spline_eval, eval_layout, coords_eval, coords_layout, spline_coef, coef_layout, stream));
    }
    // integrate(integrals, spline_coef) (spline_evaluator.hpp:493-526)
    void integrate(double* integrals, int64_t integrals_outer_stride, double const* spline_coef, ddcb_lines coef_layout,
                   ddcb_stream stream = nullptr) const
    {
        check(ddcb_integrate(get(), integrals, integrals_outer_stride, spline_coef, coef_layout, stream));
    }

private:
    Handle<ddcb_evaluator, ddcb_evaluator_destroy> m_h;
};

// The build + evaluate step on HOST arrays, batch slices of the copies overlapping the kernels
// (ddcb_host_pipeline_*): what a DDC user writes around SplineBuilder and SplineEvaluator with
// ddc::parallel_deepcopy, pipelined. order 0 evaluates values, k >= 1 the k-th derivative. The
// builder and evaluator must outlive the pipeline.
class HostPipeline
{
public:
    HostPipeline(SplineBuilder const& b, SplineEvaluator const& e, int order, int64_t npoints, int64_t slice_lines = 4096)
    {
        ddcb_host_pipeline h = nullptr;
        check(ddcb_host_pipeline_create(b.get(), e.get(), order, npoints, slice_lines, &h));
        m_h = Handle<ddcb_host_pipeline, ddcb_host_pipeline_destroy>(h);
    }
    ddcb_host_pipeline get() const { return m_h.get(); }
    // Queued on `stream`; synchronize it before reading out (and coefs, when given).
    void operator()(double const* vals, ddcb_lines vals_layout, double const* coords, ddcb_lines coords_layout, double* out,
                    ddcb_lines out_layout, double const* derivs_lo = nullptr, ddcb_lines derivs_lo_layout = {},
                    double const* derivs_hi = nullptr, ddcb_lines derivs_hi_layout = {}, double* coefs = nullptr,
                    ddcb_lines coefs_layout = {}, ddcb_stream stream = nullptr) const
    {
        check(ddcb_host_pipeline_run(get(), vals, vals_layout, derivs_lo, derivs_lo_layout, derivs_hi, derivs_hi_layout, coords,
                                     coords_layout, out, out_layout, coefs, coefs_layout, stream));
    }

private:
    Handle<ddcb_host_pipeline, ddcb_host_pipeline_destroy> m_h;
};

} // namespace ddcb
