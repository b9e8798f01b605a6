// Compile-and-run check of include/ddc_b200/spline_builder_b200.hpp against the DDC-surface mock:
// ddc::SplineBuilder<..., ddc::SplineSolver::B200> and ddc_b200::SplineEvaluator on ChunkSpans of
// the characteristics-advection shape (x, y) and of the transposed order (y, x) must give exactly
// the coefficients and values of direct ddcb_build / ddcb_eval calls. Uniform periodic cubic (the
// example's basis) and non-uniform quintic with Hermite closures (derivative spans).
// Exit 0: all equal; 1: a difference; 2: a library error; 77: no CUDA device (compile-only use).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include <cuda_runtime.h>

#include <ddc_b200/spline_builder_b200.hpp>

struct X
{
};

template <class Self, std::size_t N>
struct PointsImpl
{
    std::vector<double> pts;
    double coordinate(std::ptrdiff_t i) const { return pts[std::size_t(i)]; }
};

// ---- periodic uniform cubic on [0, 1), 12 cells ----
struct BSplinesP : ddc::UniformBSplinesMock<X, 3, true>
{
    struct Impl
    {
        double rmin() const { return 0.0; }
        double rmax() const { return 1.0; }
        std::size_t ncells() const { return 12; }
        ddc::DiscreteDomain<BSplinesP> full_domain() const
        {
            return ddc::DiscreteDomain<BSplinesP>(ddc::DiscreteElement<BSplinesP>(0), ddc::DiscreteVector<BSplinesP>(15));
        }
    };
};
struct DDimXP
{
    using continuous_dimension_type = X;
    using Impl = PointsImpl<DDimXP, 0>;
};

// ---- non-uniform quintic on [0, 1], 10 cells, Hermite closures ----
struct Knots
{
    using continuous_dimension_type = X;
    using Impl = PointsImpl<Knots, 1>;
};
struct BSplinesH : ddc::NonUniformBSplinesMock<X, 5, false>
{
    struct Impl
    {
        ddc::DiscreteDomain<Knots> break_point_domain() const
        {
            return ddc::DiscreteDomain<Knots>(ddc::DiscreteElement<Knots>(0), ddc::DiscreteVector<Knots>(11));
        }
        ddc::DiscreteDomain<BSplinesH> full_domain() const
        {
            return ddc::DiscreteDomain<BSplinesH>(ddc::DiscreteElement<BSplinesH>(0), ddc::DiscreteVector<BSplinesH>(15));
        }
    };
};
struct DDimXH
{
    using continuous_dimension_type = X;
    using Impl = PointsImpl<DDimXH, 2>;
};
struct DDimY
{
};

using Exec = Kokkos::DefaultExecutionSpace;
using Mem = Exec::memory_space;

static int g_fail = 0;

static std::vector<double> dev_to_host(double const* d, std::size_t n)
{
    std::vector<double> h(n);
    cudaMemcpy(h.data(), d, n * sizeof(double), cudaMemcpyDeviceToHost);
    return h;
}
static double* host_to_dev(std::vector<double> const& h)
{
    double* d = nullptr;
    cudaMalloc(&d, h.size() * sizeof(double));
    cudaMemcpy(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice);
    return d;
}
static void expect_equal(char const* what, std::vector<double> const& a, std::vector<double> const& b)
{
    if (a.size() != b.size() || std::memcmp(a.data(), b.data(), a.size() * sizeof(double)) != 0) {
        std::printf("DIFFERENT: %s\n", what);
        g_fail = 1;
    } else {
        std::printf("equal: %s\n", what);
    }
}

static std::vector<double> greville(ddcb_bsplines b, ddcb_closure lo, ddcb_closure hi)
{
    int64_t n = 0;
    ddc_b200::check(ddcb_greville_points(b, lo, hi, nullptr, 0, &n));
    std::vector<double> p(std::size_t(n), 0.0);
    ddc_b200::check(ddcb_greville_points(b, lo, hi, p.data(), n, &n));
    return p;
}

// (x, y) layout: build + evaluate through the adapter and directly, on ny lines.
template <class BS, class DX, ddc::SplineBuilderClosure CL, class LowerRule, class UpperRule>
static void run_case(char const* name, std::size_t ny, LowerRule lr, UpperRule ur)
{
    using Builder = ddc::SplineBuilder<Exec, Mem, BS, DX, CL, CL, ddc::SplineSolver::B200>;
    std::size_t const np = ddc::discrete_space<DX>().pts.size();
    ddc::DiscreteDomain<DX> const xdom(ddc::DiscreteElement<DX>(0), ddc::DiscreteVector<DX>(std::ptrdiff_t(np)));
    ddc::DiscreteDomain<DDimY> const ydom(ddc::DiscreteElement<DDimY>(0), ddc::DiscreteVector<DDimY>(std::ptrdiff_t(ny)));
    ddc::DiscreteDomain<DX, DDimY> const mesh(xdom, ydom);
    Builder const builder(mesh);
    std::size_t const nc = ddc::discrete_space<BS>().full_domain().size();
    std::mt19937_64 rng(42);
    std::uniform_real_distribution<double> u(-1.0, 1.0), ux(-0.2, 1.2);
    std::vector<double> hv(np * ny), hx(np * ny), hlo(std::size_t(Builder::s_nbv_xmin) * ny), hhi(std::size_t(Builder::s_nbv_xmax) * ny);
    for (auto& v : hv) v = u(rng);
    for (auto& v : hx) v = ux(rng);
    for (auto& v : hlo) v = u(rng);
    for (auto& v : hhi) v = u(rng);
    double *dv = host_to_dev(hv), *dx = host_to_dev(hx), *dlo = hlo.empty() ? nullptr : host_to_dev(hlo),
           *dhi = hhi.empty() ? nullptr : host_to_dev(hhi);
    double *dc1 = nullptr, *dc2 = nullptr, *dy1 = nullptr, *dy2 = nullptr;
    cudaMalloc(&dc1, nc * ny * sizeof(double));
    cudaMalloc(&dc2, nc * ny * sizeof(double));
    cudaMalloc(&dy1, np * ny * sizeof(double));
    cudaMalloc(&dy2, np * ny * sizeof(double));
    // through the adapter
    auto const sdom = builder.batched_spline_domain(mesh);
    ddc::ChunkSpan<double, std::remove_const_t<decltype(sdom)>> coef(dc1, sdom);
    ddc::ChunkSpan<double const, ddc::DiscreteDomain<DX, DDimY>> vals(dv, mesh);
    using Deriv = typename Builder::deriv_type;
    ddc::DiscreteDomain<Deriv, DDimY> const dlo_dom(
            ddc::DiscreteDomain<Deriv>(ddc::DiscreteElement<Deriv>(1), ddc::DiscreteVector<Deriv>(Builder::s_nbv_xmin)), ydom);
    ddc::DiscreteDomain<Deriv, DDimY> const dhi_dom(
            ddc::DiscreteDomain<Deriv>(ddc::DiscreteElement<Deriv>(1), ddc::DiscreteVector<Deriv>(Builder::s_nbv_xmax)), ydom);
    if constexpr (CL == ddc::SplineBuilderClosure::HERMITE)
        builder(coef, vals, std::optional(ddc::ChunkSpan<double const, ddc::DiscreteDomain<Deriv, DDimY>>(dlo, dlo_dom)),
                std::optional(ddc::ChunkSpan<double const, ddc::DiscreteDomain<Deriv, DDimY>>(dhi, dhi_dom)));
    else
        builder(coef, vals);
    ddc_b200::SplineEvaluator<Exec, Mem, BS, DX, LowerRule, UpperRule> const evaluator(lr, ur);
    ddc::ChunkSpan<double, ddc::DiscreteDomain<DX, DDimY>> out(dy1, mesh);
    ddc::ChunkSpan<ddc::Coordinate<X> const, ddc::DiscreteDomain<DX, DDimY>> coords(reinterpret_cast<ddc::Coordinate<X> const*>(dx), mesh);
    evaluator(out, coords, coef.span_cview());
    // directly through the C-ABI
    ddcb_lines const lv {int64_t(np), int64_t(ny), int64_t(ny), 1, 0}, lc {int64_t(nc), int64_t(ny), int64_t(ny), 1, 0};
    ddcb_lines const llo {Builder::s_nbv_xmin, int64_t(ny), int64_t(ny), 1, 0}, lhi {Builder::s_nbv_xmax, int64_t(ny), int64_t(ny), 1, 0};
    ddcb_lines const none {0, 1, 0, 0, 0};
    ddc_b200::check(ddcb_build(builder.handle(), dc2, lc, dv, lv, dlo, dlo ? llo : none, dhi, dhi ? lhi : none, nullptr));
    ddc_b200::Basis<BS> basis;
    ddcb_evaluator e = nullptr;
    ddc_b200::check(ddcb_evaluator_create(basis.get(), ddc_b200::extrapolation_of<LowerRule>::value,
                                          ddc_b200::extrapolation_of<UpperRule>::value, &e));
    ddc_b200::check(ddcb_eval(e, dy2, lv, dx, lv, dc2, lc, nullptr));
    cudaDeviceSynchronize();
    std::printf("%s:\n", name);
    expect_equal("coefficients (x, y)", dev_to_host(dc1, nc * ny), dev_to_host(dc2, nc * ny));
    expect_equal("values (x, y)", dev_to_host(dy1, np * ny), dev_to_host(dy2, np * ny));
    // the transposed order (y, x): one contiguous line per y
    ddc::DiscreteDomain<DDimY, DX> const tmesh(ydom, xdom);
    std::vector<double> hvt(np * ny);
    for (std::size_t i = 0; i < np; ++i)
        for (std::size_t j = 0; j < ny; ++j) hvt[j * np + i] = hv[i * ny + j];
    double* dvt = host_to_dev(hvt);
    double* dct = nullptr;
    cudaMalloc(&dct, nc * ny * sizeof(double));
    auto const tsdom = builder.batched_spline_domain(tmesh);
    ddc::ChunkSpan<double, std::remove_const_t<decltype(tsdom)>> tcoef(dct, tsdom);
    if constexpr (CL != ddc::SplineBuilderClosure::HERMITE) {
        builder(tcoef, ddc::ChunkSpan<double const, ddc::DiscreteDomain<DDimY, DX>>(dvt, tmesh));
        cudaDeviceSynchronize();
        std::vector<double> ct = dev_to_host(dct, nc * ny), c = dev_to_host(dc2, nc * ny), back(nc * ny);
        for (std::size_t i = 0; i < nc; ++i)
            for (std::size_t j = 0; j < ny; ++j) back[i * ny + j] = ct[j * nc + i];
        // the two layouts run different tile paths; both are FP64 solves of the same systems
        double err = 0.0, mx = 0.0;
        for (std::size_t k = 0; k < back.size(); ++k) {
            err = std::fmax(err, std::fabs(back[k] - c[k]));
            mx = std::fmax(mx, std::fabs(c[k]));
        }
        std::printf("%s: coefficients (y, x) vs (x, y), max rel diff %.3g\n", err / mx <= 1e-13 ? "equal" : "DIFFERENT", err / mx);
        if (err / mx > 1e-13) g_fail = 1;
    }
    ddcb_evaluator_destroy(e);
    for (double* p : {dv, dx, dlo, dhi, dc1, dc2, dy1, dy2, dvt, dct})
        if (p) cudaFree(p);
}

int main()
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        std::printf("no CUDA device\n");
        return 77;
    }
    try {
        {
            ddcb_bsplines b = nullptr;
            ddc_b200::check(ddcb_bsplines_create_uniform(3, 1, 0.0, 1.0, 12, &b));
            ddc::discrete_space<DDimXP>().pts = greville(b, DDCB_PERIODIC, DDCB_PERIODIC);
            ddcb_bsplines_destroy(b);
        }
        {
            std::vector<double> br(11);
            for (int i = 0; i <= 10; ++i) br[i] = i / 10.0 + ((i > 0 && i < 10) ? 0.02 * std::sin(3.0 * i) : 0.0);
            ddc::discrete_space<Knots>().pts = br;
            ddcb_bsplines b = nullptr;
            ddc_b200::check(ddcb_bsplines_create_non_uniform(5, 0, br.data(), 11, &b));
            ddc::discrete_space<DDimXH>().pts = greville(b, DDCB_HERMITE, DDCB_HERMITE);
            ddcb_bsplines_destroy(b);
        }
        run_case<BSplinesP, DDimXP, ddc::SplineBuilderClosure::PERIODIC>("periodic uniform cubic", 37,
                                                                         ddc::PeriodicExtrapolationRule<X>(),
                                                                         ddc::PeriodicExtrapolationRule<X>());
        run_case<BSplinesH, DDimXH, ddc::SplineBuilderClosure::HERMITE>("non-uniform quintic Hermite", 20,
                                                                        ddc::ConstantExtrapolationRule<X>(),
                                                                        ddc::NullExtrapolationRule());
    } catch (std::exception const& ex) {
        std::printf("library error: %s\n", ex.what());
        return 2;
    }
    std::printf("%s\n", g_fail ? "FAILED" : "ALL EQUAL");
    return g_fail;
}
