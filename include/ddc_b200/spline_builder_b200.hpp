// spline_builder_b200.hpp -- DDC's SplineBuilder with SplineSolver::B200 and a B200 SplineEvaluator,
// over the C-ABI of ddcb.h.
//
// Selecting the path: DDC's solver enum (src/ddc/kernels/splines/spline_builder.hpp:36-39) gains one
// member, `B200`, and this header provides the partial specialisation
//     ddc::SplineBuilder<ExecSpace, MemorySpace, BSplines, InterpolationDDim, Lower, Upper,
//                        ddc::SplineSolver::B200>
// with the public interface of the primary template (spline_builder.hpp:57-557, 1103-1234): the
// same member types and constants, constructors, domain helpers, operator() and
// quadrature_coefficients. Code written against ddc::SplineBuilder switches to the B200 kernels by
// changing its Solver template argument; the coefficients it produces have DDC's layout, so DDC's
// own SplineEvaluator keeps working on them. ddc_b200::SplineEvaluator has SplineEvaluator's
// template parameters (spline_evaluator.hpp:40-186) and runs the evaluation on the GPU too.
//
// Data: every ChunkSpan is described to the library by ddcb_lines (lines_of below) from its
// allocation mdspan's extents and strides; any dimension order works as long as the batch
// dimensions that follow the dimension of interest are contiguous (DDC's layout_right), or the
// dimension of interest itself is (layout_left-like single lines). Work is queued on the CUDA
// stream of the execution space instance (Kokkos::Cuda::cuda_stream()) when it has one, else on
// the default stream, and is asynchronous like the Kokkos kernels it replaces. Failures throw
// std::runtime_error with the library's message, as the reference does at construction.
//
// Not covered: constant extrapolation at a position other than the domain ends (the library's
// constant rule evaluates at rmin / rmax, which is how DDC's examples and tests construct it).
#pragma once

#include <cstddef>
#include <optional>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#include <ddc/ddc.hpp>
#include <ddc/kernels/splines.hpp>

#include "../ddcb.h"

namespace ddc_b200 {

inline void check(ddcb_status s)
{
    if (s != DDCB_SUCCESS) throw std::runtime_error(ddcb_last_error_message());
}

// The CUDA stream of an execution space instance (Kokkos::Cuda), or the default stream.
template <class ExecSpace>
ddcb_stream stream_of(ExecSpace const& es)
{
    if constexpr (requires { es.cuda_stream(); }) return reinterpret_cast<ddcb_stream>(es.cuda_stream());
    else return nullptr;
}

// The ddcb_lines of a ChunkSpan whose dimension of interest is DDim: every other dimension is a
// batch dimension, flattened in the span's dimension order. The trailing batch dimensions that are
// contiguous form the `inner` part; the remaining ones must be regularly strided (`outer`).
template <class DDim, class Span>
ddcb_lines lines_of(Span const& span)
{
    using Dom = decltype(span.domain());
    constexpr std::size_t R = Dom::rank();
    constexpr std::size_t r = ddc::type_seq_rank_v<DDim, ddc::to_type_seq_t<Dom>>;
    static_assert(r < R, "the span does not have the dimension of interest");
    auto const md = span.allocation_mdspan();
    ddcb_lines l {};
    l.n = int64_t(md.extent(r));
    l.stride = int64_t(md.stride(r));
    // batch dimensions in order, skipping extents of 1 (their strides are irrelevant)
    std::vector<std::pair<int64_t, int64_t>> b; // (extent, stride)
    for (std::size_t d = 0; d < R; ++d)
        if (d != r && md.extent(d) != 1) b.emplace_back(int64_t(md.extent(d)), int64_t(md.stride(d)));
    // inner: the longest trailing run with unit stride at the end and packed strides above it
    std::size_t k = b.size();
    int64_t inner = 1;
    while (k > 0 && b[k - 1].second == inner) {
        inner *= b[k - 1].first;
        --k;
    }
    // outer: the leading dimensions must chain regularly
    int64_t outer = 1, ostride = k > 0 ? b[k - 1].second : 0;
    for (std::size_t d = k; d-- > 0;) {
        if (b[d].second != ostride * outer)
            throw std::runtime_error("ddc_b200: the batch dimensions of this span are not regularly strided");
        outer *= b[d].first;
    }
    l.inner = inner;
    l.outer = outer;
    l.outer_stride = outer > 1 ? ostride : 0;
    if (md.extent(r) == 0 || l.inner * l.outer == 0) l.inner = l.outer = 0;
    return l;
}

// The coordinates of the points of a 1D discrete domain (the interpolation points of a builder).
template <class DDim>
std::vector<double> interpolation_points_of(ddc::DiscreteDomain<DDim> const& dom)
{
    std::vector<double> pts;
    for (auto const e : dom) pts.push_back(double(ddc::coordinate(e)));
    return pts;
}

// The break points of a non-uniform B-spline dimension (NonUniformBSplines::break_point_domain).
template <class BSplines>
std::vector<double> break_points_of()
{
    std::vector<double> br;
    for (auto const e : ddc::discrete_space<BSplines>().break_point_domain()) br.push_back(double(ddc::coordinate(e)));
    return br;
}

// The library's basis for a DDC B-spline dimension (owned).
template <class BSplines>
class Basis
{
    ddcb_bsplines h_ = nullptr;

public:
    Basis()
    {
        auto const& bs = ddc::discrete_space<BSplines>();
        int const deg = int(BSplines::degree()), per = BSplines::is_periodic() ? 1 : 0;
        if constexpr (BSplines::is_uniform()) {
            check(ddcb_bsplines_create_uniform(deg, per, double(bs.rmin()), double(bs.rmax()), int64_t(bs.ncells()), &h_));
        } else {
            std::vector<double> const br = break_points_of<BSplines>();
            check(ddcb_bsplines_create_non_uniform(deg, per, br.data(), int64_t(br.size()), &h_));
        }
    }
    Basis(Basis const&) = delete;
    Basis& operator=(Basis const&) = delete;
    Basis(Basis&& o) noexcept : h_(std::exchange(o.h_, nullptr)) {}
    Basis& operator=(Basis&& o) noexcept
    {
        std::swap(h_, o.h_);
        return *this;
    }
    ~Basis()
    {
        if (h_) ddcb_bsplines_destroy(h_);
    }
    ddcb_bsplines get() const { return h_; }
};

constexpr ddcb_closure closure_of(ddc::SplineBuilderClosure c)
{
    switch (c) {
    case ddc::SplineBuilderClosure::PERIODIC: return DDCB_PERIODIC;
    case ddc::SplineBuilderClosure::HERMITE: return DDCB_HERMITE;
    case ddc::SplineBuilderClosure::HOMOGENEOUS_HERMITE: return DDCB_HOMOGENEOUS_HERMITE;
    default: return DDCB_GREVILLE;
    }
}

// n_boundary_equations (spline_builder_closures.hpp:43-55).
constexpr int n_boundary_equations(ddc::SplineBuilderClosure c, std::size_t degree)
{
    return (c == ddc::SplineBuilderClosure::HERMITE || c == ddc::SplineBuilderClosure::HOMOGENEOUS_HERMITE) ? int(degree / 2) : 0;
}

// The library's rule for a DDC extrapolation rule type.
template <class Rule>
struct extrapolation_of;
template <class... D>
struct extrapolation_of<ddc::PeriodicExtrapolationRule<D...>>
{
    static constexpr ddcb_extrapolation value = DDCB_EXTRAP_PERIODIC;
};
template <>
struct extrapolation_of<ddc::NullExtrapolationRule>
{
    static constexpr ddcb_extrapolation value = DDCB_EXTRAP_NULL;
};
template <class... D>
struct extrapolation_of<ddc::ConstantExtrapolationRule<D...>>
{
    static constexpr ddcb_extrapolation value = DDCB_EXTRAP_CONSTANT;
};

// SplineEvaluator<ExecSpace, MemorySpace, BSplines, EvaluationDDim, LowerExtrapolationRule,
// UpperExtrapolationRule> (spline_evaluator.hpp:40-526) on the GPU: operator(), deriv and
// integrate over batched ChunkSpans.
template <class ExecSpace, class MemorySpace, class BSplines, class EvaluationDDim, class LowerExtrapolationRule,
          class UpperExtrapolationRule>
class SplineEvaluator
{
public:
    using exec_space = ExecSpace;
    using memory_space = MemorySpace;
    using continuous_dimension_type = typename BSplines::continuous_dimension_type;
    using evaluation_discrete_dimension_type = EvaluationDDim;
    using bsplines_type = BSplines;
    using lower_extrapolation_rule_type = LowerExtrapolationRule;
    using upper_extrapolation_rule_type = UpperExtrapolationRule;
    template <class BatchedInterpolationDDom>
    using batched_spline_domain_type = ddc::replace_dim_of_t<BatchedInterpolationDDom, EvaluationDDim, BSplines>;

private:
    LowerExtrapolationRule m_lower;
    UpperExtrapolationRule m_upper;
    Basis<BSplines> m_basis;
    ddcb_evaluator m_e = nullptr;

public:
    explicit SplineEvaluator(LowerExtrapolationRule const& lower, UpperExtrapolationRule const& upper)
        : m_lower(lower), m_upper(upper)
    {
        check(ddcb_evaluator_create(m_basis.get(), extrapolation_of<LowerExtrapolationRule>::value,
                                    extrapolation_of<UpperExtrapolationRule>::value, &m_e));
    }
    SplineEvaluator(SplineEvaluator const&) = delete;
    SplineEvaluator& operator=(SplineEvaluator const&) = delete;
    SplineEvaluator(SplineEvaluator&& o) noexcept
        : m_lower(o.m_lower), m_upper(o.m_upper), m_basis(std::move(o.m_basis)), m_e(std::exchange(o.m_e, nullptr))
    {
    }
    ~SplineEvaluator()
    {
        if (m_e) ddcb_evaluator_destroy(m_e);
    }
    LowerExtrapolationRule lower_extrapolation_rule() const { return m_lower; }
    UpperExtrapolationRule upper_extrapolation_rule() const { return m_upper; }

    // operator()(spline_eval, coords_eval, spline_coef) (spline_evaluator.hpp:257-294). Coordinates
    // may carry several continuous dimensions; the one of this evaluator is read with its stride.
    template <class Layout1, class Layout2, class Layout3, class BatchedInterpolationDDom, class... CoordsDims>
    void operator()(ddc::ChunkSpan<double, BatchedInterpolationDDom, Layout1, memory_space> const& spline_eval,
                    ddc::ChunkSpan<ddc::Coordinate<CoordsDims...> const, BatchedInterpolationDDom, Layout2, memory_space> const& coords_eval,
                    ddc::ChunkSpan<double const, batched_spline_domain_type<BatchedInterpolationDDom>, Layout3, memory_space> const& spline_coef,
                    ExecSpace const& es = ExecSpace()) const
    {
        auto [x, lx] = coords_lines(coords_eval);
        check(ddcb_eval(m_e, spline_eval.data_handle(), lines_of<EvaluationDDim>(spline_eval), x, lx,
                        spline_coef.data_handle(), lines_of<BSplines>(spline_coef), stream_of(es)));
    }

    // deriv(DiscreteElement<Deriv<X>>(order), spline_eval, coords_eval, spline_coef)
    // (spline_evaluator.hpp:388-430).
    template <class DElem, class Layout1, class Layout2, class Layout3, class BatchedInterpolationDDom, class... CoordsDims>
    void deriv(DElem const& deriv_order, ddc::ChunkSpan<double, BatchedInterpolationDDom, Layout1, memory_space> const& spline_eval,
               ddc::ChunkSpan<ddc::Coordinate<CoordsDims...> const, BatchedInterpolationDDom, Layout2, memory_space> const& coords_eval,
               ddc::ChunkSpan<double const, batched_spline_domain_type<BatchedInterpolationDDom>, Layout3, memory_space> const& spline_coef,
               ExecSpace const& es = ExecSpace()) const
    {
        auto [x, lx] = coords_lines(coords_eval);
        check(ddcb_eval_deriv(m_e, int32_t(deriv_order.uid()), spline_eval.data_handle(),
                              lines_of<EvaluationDDim>(spline_eval), x, lx, spline_coef.data_handle(),
                              lines_of<BSplines>(spline_coef), stream_of(es)));
    }

    // integrate(integrals, spline_coef) (spline_evaluator.hpp:493-526): integrals over the batch
    // domain, contiguous.
    template <class Layout1, class Layout2, class BatchDDom, class BatchedSplineDDom>
    void integrate(ddc::ChunkSpan<double, BatchDDom, Layout1, memory_space> const& integrals,
                   ddc::ChunkSpan<double const, BatchedSplineDDom, Layout2, memory_space> const& spline_coef,
                   ExecSpace const& es = ExecSpace()) const
    {
        ddcb_lines const lc = lines_of<BSplines>(spline_coef);
        check(ddcb_integrate(m_e, integrals.data_handle(), lc.inner, spline_coef.data_handle(), lc, stream_of(es)));
    }

private:
    template <class Span>
    static auto coords_lines(Span const& coords)
    {
        using C = std::remove_const_t<std::remove_pointer_t<decltype(coords.data_handle())>>;
        constexpr int ncomp = int(sizeof(C) / sizeof(double));
        static_assert(sizeof(C) == ncomp * sizeof(double), "coordinates must be doubles");
        int comp = 0;
        if constexpr (ncomp > 1) comp = coordinate_rank<C>::value;
        ddcb_lines l = lines_of<EvaluationDDim>(coords);
        l.stride *= ncomp;
        l.outer_stride *= ncomp;
        if (ncomp > 1 && l.inner > 1)
            throw std::runtime_error("ddc_b200: multi-dimensional coordinates need a unit-extent inner batch");
        return std::pair {reinterpret_cast<double const*>(coords.data_handle()) + comp, l};
    }
    template <class C>
    struct coordinate_rank;
    template <class... CD>
    struct coordinate_rank<ddc::Coordinate<CD...>>
    {
        static constexpr int value = int(ddc::type_seq_rank_v<continuous_dimension_type, ddc::detail::TypeSeq<CD...>>);
    };
};

} // namespace ddc_b200

namespace ddc {

// SplineBuilder with Solver = SplineSolver::B200: the interface of spline_builder.hpp:57-557 and
// quadrature_coefficients (:1103-1234), with the plan and the solves in libddcb.
template <class ExecSpace, class MemorySpace, class BSplines, class InterpolationDDim, SplineBuilderClosure SBCLower,
          SplineBuilderClosure SBCUpper>
class SplineBuilder<ExecSpace, MemorySpace, BSplines, InterpolationDDim, SBCLower, SBCUpper, SplineSolver::B200>
{
    static_assert((BSplines::is_periodic() && SBCLower == SplineBuilderClosure::PERIODIC && SBCUpper == SplineBuilderClosure::PERIODIC)
                  || (!BSplines::is_periodic() && SBCLower != SplineBuilderClosure::PERIODIC
                      && SBCUpper != SplineBuilderClosure::PERIODIC));

public:
    using exec_space = ExecSpace;
    using memory_space = MemorySpace;
    using continuous_dimension_type = typename InterpolationDDim::continuous_dimension_type;
    using interpolation_discrete_dimension_type = InterpolationDDim;
    using bsplines_type = BSplines;
    using deriv_type = ddc::Deriv<continuous_dimension_type>;
    using interpolation_domain_type = ddc::DiscreteDomain<interpolation_discrete_dimension_type>;
    template <class BatchedInterpolationDDom>
    using batched_interpolation_domain_type = BatchedInterpolationDDom;
    template <class BatchedInterpolationDDom>
    using batch_domain_type = ddc::remove_dims_of_t<BatchedInterpolationDDom, interpolation_discrete_dimension_type>;
    template <class BatchedInterpolationDDom>
    using batched_spline_domain_type = ddc::replace_dim_of_t<BatchedInterpolationDDom, interpolation_discrete_dimension_type, bsplines_type>;
    template <class BatchedInterpolationDDom>
    using batched_derivs_domain_type = ddc::replace_dim_of_t<BatchedInterpolationDDom, interpolation_discrete_dimension_type, deriv_type>;

    static constexpr bool s_odd = BSplines::degree() % 2;
    static constexpr int s_nbe_xmin = ddc_b200::n_boundary_equations(SBCLower, BSplines::degree());
    static constexpr int s_nbe_xmax = ddc_b200::n_boundary_equations(SBCUpper, BSplines::degree());
    static constexpr int s_nbv_xmin = SBCLower == SplineBuilderClosure::HOMOGENEOUS_HERMITE ? 0 : s_nbe_xmin;
    static constexpr int s_nbv_xmax = SBCUpper == SplineBuilderClosure::HOMOGENEOUS_HERMITE ? 0 : s_nbe_xmax;
    static constexpr SplineBuilderClosure s_sbc_xmin = SBCLower;
    static constexpr SplineBuilderClosure s_sbc_xmax = SBCUpper;
    static constexpr SplineSolver s_spline_solver = SplineSolver::B200;

private:
    interpolation_domain_type m_interpolation_domain;
    ddc_b200::Basis<BSplines> m_basis;
    ddcb_builder m_b = nullptr;
    std::string m_label;

public:
    // SplineBuilder(label, interpolation_domain, cols_per_chunk, preconditioner_max_block_size)
    // (spline_builder.hpp:227-260): the two Ginkgo tuning arguments are accepted and unused.
    explicit SplineBuilder(std::string label, interpolation_domain_type const& interpolation_domain,
                           std::optional<std::size_t> = std::nullopt, std::optional<unsigned int> = std::nullopt)
        : m_interpolation_domain(interpolation_domain), m_label(std::move(label))
    {
        std::vector<double> const pts = ddc_b200::interpolation_points_of(interpolation_domain);
        ddcb_builder_options opts {DDCB_FP64, 2, 0, 0, 0.0};
        ddcb_status const s = ddcb_builder_create(m_basis.get(), pts.data(), int64_t(pts.size()), ddc_b200::closure_of(SBCLower),
                                                  ddc_b200::closure_of(SBCUpper), &opts, &m_b);
        ddc_b200::check(s);
    }
    explicit SplineBuilder(interpolation_domain_type const& interpolation_domain, std::optional<std::size_t> cols = std::nullopt,
                           std::optional<unsigned int> pre = std::nullopt)
        : SplineBuilder("no-label", interpolation_domain, cols, pre)
    {
    }
    template <class BatchedInterpolationDDom>
        requires(!std::is_same_v<BatchedInterpolationDDom, interpolation_domain_type>)
    explicit SplineBuilder(BatchedInterpolationDDom const& batched_interpolation_domain, std::optional<std::size_t> cols = std::nullopt,
                           std::optional<unsigned int> pre = std::nullopt)
        : SplineBuilder("no-label", interpolation_domain_type(batched_interpolation_domain), cols, pre)
    {
    }
    SplineBuilder(SplineBuilder const&) = delete;
    SplineBuilder& operator=(SplineBuilder const&) = delete;
    SplineBuilder(SplineBuilder&& o) noexcept
        : m_interpolation_domain(o.m_interpolation_domain)
        , m_basis(std::move(o.m_basis))
        , m_b(std::exchange(o.m_b, nullptr))
        , m_label(std::move(o.m_label))
    {
    }
    ~SplineBuilder()
    {
        if (m_b) ddcb_builder_destroy(m_b);
    }

    interpolation_domain_type interpolation_domain() const noexcept { return m_interpolation_domain; }
    template <class BatchedInterpolationDDom>
    BatchedInterpolationDDom batched_interpolation_domain(BatchedInterpolationDDom const& d) const noexcept
    {
        return d;
    }
    template <class BatchedInterpolationDDom>
    batch_domain_type<BatchedInterpolationDDom> batch_domain(BatchedInterpolationDDom const& d) const noexcept
    {
        return ddc::remove_dims_of<interpolation_discrete_dimension_type>(d);
    }
    ddc::DiscreteDomain<bsplines_type> spline_domain() const noexcept { return ddc::discrete_space<bsplines_type>().full_domain(); }
    template <class BatchedInterpolationDDom>
    batched_spline_domain_type<BatchedInterpolationDDom> batched_spline_domain(BatchedInterpolationDDom const& d) const noexcept
    {
        return ddc::replace_dim_of<interpolation_discrete_dimension_type, bsplines_type>(d, spline_domain());
    }

    // operator()(spline, vals, derivs_xmin, derivs_xmax) (spline_builder.hpp:538-557, 896-1101).
    template <class Layout, class BatchedInterpolationDDom>
    void operator()(ddc::ChunkSpan<double, batched_spline_domain_type<BatchedInterpolationDDom>, Layout, memory_space> spline,
                    ddc::ChunkSpan<double const, BatchedInterpolationDDom, Layout, memory_space> vals,
                    std::optional<ddc::ChunkSpan<double const, batched_derivs_domain_type<BatchedInterpolationDDom>, Layout, memory_space>>
                            derivs_xmin = std::nullopt,
                    std::optional<ddc::ChunkSpan<double const, batched_derivs_domain_type<BatchedInterpolationDDom>, Layout, memory_space>>
                            derivs_xmax = std::nullopt,
                    ExecSpace const& es = ExecSpace()) const
    {
        ddcb_lines const none {0, 1, 0, 0, 0};
        ddcb_lines const llo = derivs_xmin ? ddc_b200::lines_of<deriv_type>(*derivs_xmin) : none;
        ddcb_lines const lhi = derivs_xmax ? ddc_b200::lines_of<deriv_type>(*derivs_xmax) : none;
        ddc_b200::check(ddcb_build(m_b, spline.data_handle(), ddc_b200::lines_of<bsplines_type>(spline), vals.data_handle(),
                                   ddc_b200::lines_of<interpolation_discrete_dimension_type>(vals),
                                   derivs_xmin ? derivs_xmin->data_handle() : nullptr, llo,
                                   derivs_xmax ? derivs_xmax->data_handle() : nullptr, lhi, ddc_b200::stream_of(es)));
    }

    // quadrature_coefficients() (spline_builder.hpp:1103-1234), as host vectors
    // (q_derivs_xmin, q, q_derivs_xmax), the Hermite parts scaled by dx^k.
    std::tuple<std::vector<double>, std::vector<double>, std::vector<double>> quadrature_coefficients() const
    {
        ddcb_builder_info info {};
        ddc_b200::check(ddcb_builder_get_info(m_b, &info));
        std::vector<double> qlo(std::size_t(info.nbv_lo)), q(std::size_t(info.nbasis - info.nbv_lo - info.nbv_hi)),
                qhi(std::size_t(info.nbv_hi));
        ddc_b200::check(ddcb_quadrature_coefficients(m_b, qlo.data(), q.data(), qhi.data()));
        return {std::move(qlo), std::move(q), std::move(qhi)};
    }

    // The library's builder handle (for the other calls of ddcb.h on the same plan).
    ddcb_builder handle() const noexcept { return m_b; }
};

} // namespace ddc
