// Stand-in for DDC's splines header (src/ddc/kernels/splines/): the closure and solver enums, with
// the solver enum carrying the B200 member that the adapter's integration adds, the extrapolation
// rule types, and uniform / non-uniform B-spline dimensions whose discrete spaces the tests fill.
// Test infrastructure only.
#pragma once

#include <cstddef>
#include <vector>

#include <ddc/ddc.hpp>

namespace ddc {

enum class SplineBuilderClosure { PERIODIC, HERMITE, HOMOGENEOUS_HERMITE, GREVILLE };

// spline_builder.hpp:36-39 with the one added member
enum class SplineSolver { GINKGO, LAPACK, B200 };

// the primary template (spline_builder.hpp:57-65); only the B200 specialisation is defined here
template <class ExecSpace, class MemorySpace, class BSplines, class InterpolationDDim, SplineBuilderClosure SBCLower,
          SplineBuilderClosure SBCUpper, SplineSolver Solver>
class SplineBuilder;

template <class... Dims>
struct PeriodicExtrapolationRule
{
};
struct NullExtrapolationRule
{
};
template <class... Dims>
struct ConstantExtrapolationRule
{
};

template <class CDim, std::size_t D, bool Periodic>
struct UniformBSplinesMock
{
    using continuous_dimension_type = CDim;
    static constexpr std::size_t degree() { return D; }
    static constexpr bool is_periodic() { return Periodic; }
    static constexpr bool is_uniform() { return true; }
};
template <class CDim, std::size_t D, bool Periodic>
struct NonUniformBSplinesMock
{
    using continuous_dimension_type = CDim;
    static constexpr std::size_t degree() { return D; }
    static constexpr bool is_periodic() { return Periodic; }
    static constexpr bool is_uniform() { return false; }
};

} // namespace ddc
