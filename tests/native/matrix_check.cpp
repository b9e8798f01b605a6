// Host-side check that the builder plan solves the reference's system: for every degree,
// uniform / non-uniform / periodic basis, closure pair and several sizes, the plan's assembled
// matrix (reference row and column order, after the symmetric storage of uniform centre blocks)
// equals the oracle's restatement of the reference's SplineBuilder matrix entry by entry, up to
// entries below 1e-15 that either side keeps or drops. Links the plan (included) and the oracle
// library (test infrastructure). No CUDA call is made.
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "../../ddc_b200/csrc/plan.cpp"

extern "C" {
void* orc_bsplines_uniform(int degree, int periodic, double rmin, double rmax, long ncells);
void* orc_bsplines_non_uniform(int degree, int periodic, double const* breaks, long nbreaks);
void orc_bsplines_free(void* p);
void* orc_builder_create(void* bsp, double const* pts, long npts, int lo, int hi);
void orc_builder_free(void* p);
void orc_builder_matrix(void* p, double* out);
}

int main()
{
    int failures = 0, cases = 0;
    std::mt19937_64 rng(777);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    int const bcs[][2] = {{0, 0}, {1, 1}, {3, 3}, {1, 3}, {3, 1}, {2, 2}};
    for (int d = 1; d <= 5; ++d)
        for (int uni = 0; uni < 2; ++uni)
            for (auto const& bc : bcs)
                for (int nc : {7, 12, 40, 129, 429}) {
                    bool const per = bc[0] == 0;
                    ddcb::Basis b;
                    std::vector<double> br(nc + 1);
                    double const h = 1.0 / nc;
                    for (int i = 0; i <= nc; ++i) br[i] = i * h + ((i > 0 && i < nc) ? 0.3 * h * U(rng) : 0.0);
                    void* ob = nullptr;
                    if (uni) {
                        ddcb::make_uniform_basis(b, d, per, 0.0, 1.0, nc);
                        ob = orc_bsplines_uniform(d, per, 0.0, 1.0, nc);
                    } else {
                        ddcb::make_non_uniform_basis(b, d, per, br.data(), nc + 1);
                        ob = orc_bsplines_non_uniform(d, per, br.data(), nc + 1);
                    }
                    auto pts = ddcb::greville_points(b, bc[0], bc[1]);
                    ddcb_builder_options opt {0, 2, 8, 16, 0.0};
                    ddcb::Builder* bl = nullptr;
                    void* obl = nullptr;
                    try {
                        bl = ddcb::create_builder_host(b, pts.data(), long(pts.size()), bc[0], bc[1], &opt);
                        obl = orc_builder_create(ob, pts.data(), long(pts.size()), bc[0], bc[1]);
                    } catch (std::exception const& e) {
                        std::printf("FAIL create d=%d uni=%d bc=%d,%d nc=%d: %s\n", d, uni, bc[0], bc[1], nc, e.what());
                        ++failures;
                        continue;
                    }
                    long const n = bl->n;
                    std::vector<double> A(size_t(n * n));
                    orc_builder_matrix(obl, A.data());
                    auto const& rows = static_cast<ddcb::BuilderPrivate*>(bl->host_private)->ref_rows;
                    double worst = 0.0;
                    for (long i = 0; i < n; ++i)
                        for (long j = 0; j < n; ++j) {
                            auto it = rows[i].find(j);
                            double const p = it == rows[i].end() ? 0.0 : it->second, o = A[size_t(i * n + j)];
                            if (std::fabs(p) < 1e-15 && std::fabs(o) < 1e-15) continue;
                            worst = std::fmax(worst, std::fabs(p - o));
                        }
                    ++cases;
                    bool const bad = !(worst == 0.0);
                    if (bad) ++failures;
                    if (bad || std::getenv("MATRIX_CHECK_VERBOSE"))
                        std::printf("%s d=%d uni=%d bc=%d,%d nc=%d max|plan - oracle| = %.3e\n", bad ? "FAIL" : "ok", d, uni,
                                    bc[0], bc[1], nc, worst);
                    orc_builder_free(obl);
                    orc_bsplines_free(ob);
                    ddcb::destroy_builder(bl);
                }
    std::printf("matrix_check: %d cases, %d failures\n", cases, failures);
    return failures ? 1 : 0;
}
