// Host-side check of the builder plan: for many bases, closures and sizes, the device solve's
// steps (chunked sweeps, log-depth carry scan, border correction), emulated on the host with the
// very tables the kernels receive, reproduce the direct banded solve. Prints one line per case
// and exits non-zero if any case exceeds the tolerance. No CUDA call is made.
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "../../ddc_b200/csrc/ddcb_internal.hpp"

int main()
{
    int failures = 0, cases = 0;
    std::mt19937_64 rng(12345);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    int const bcs[][2] = {{0, 0}, {1, 1}, {3, 3}, {1, 3}, {3, 1}, {2, 2}};
    for (int d = 1; d <= 5; ++d)
        for (int uni = 0; uni < 2; ++uni)
            for (auto const& bc : bcs)
                for (int nc : {9, 17, 40, 101, 300})
                    for (int chunks : {4, 32}) {
                        bool const per = bc[0] == 0;
                        ddcb::Basis b;
                        if (uni) ddcb::make_uniform_basis(b, d, per, 0.0, 1.0, nc);
                        else {
                            std::vector<double> br(nc + 1);
                            double const h = 1.0 / nc;
                            for (int i = 0; i <= nc; ++i) br[i] = i * h + ((i > 0 && i < nc) ? 0.3 * h * U(rng) : 0.0);
                            ddcb::make_non_uniform_basis(b, d, per, br.data(), nc + 1);
                        }
                        auto pts = ddcb::greville_points(b, bc[0], bc[1]);
                        ddcb_builder_options opt {0, 2, 8, chunks};
                        ddcb::Builder* bl = nullptr;
                        try {
                            bl = ddcb::create_builder_host(b, pts.data(), long(pts.size()), bc[0], bc[1], &opt);
                        } catch (std::exception const& e) {
                            std::printf("FAIL create d=%d uni=%d bc=%d,%d nc=%d: %s\n", d, uni, bc[0], bc[1], nc, e.what());
                            ++failures;
                            continue;
                        }
                        {
                            std::vector<double> vals(bl->points.size()), dlo(8), dhi(8);
                            for (auto& v : vals) v = U(rng);
                            for (auto& v : dlo) v = U(rng);
                            for (auto& v : dhi) v = U(rng);
                            double const err = ddcb::emulate_build(*bl, vals.data(), dlo.data(), dhi.data());
                            ++cases;
                            // the dense reference and the banded solve agree to cond(A)*eps
                            bool const bad = !(err <= 1e-11);
                            if (bad) ++failures;
                            if (bad || std::getenv("PLAN_CHECK_VERBOSE"))
                                std::printf("%s build d=%d uni=%d bc=%d,%d nc=%d chunks=%d err=%.3e %s\n", bad ? "FAIL" : "ok", d,
                                            uni, bc[0], bc[1], nc, chunks, err, bl->structure.c_str());
                        }
                        for (int tr = 0; tr < 2; ++tr) {
                            std::vector<double> rhs(bl->n);
                            for (auto& v : rhs) v = U(rng);
                            double const err = ddcb::emulate_device_solve(*bl, rhs.data(), tr != 0);
                            ++cases;
                            bool const bad = !(err <= 1e-12);
                            if (bad) ++failures;
                            if (bad || std::getenv("PLAN_CHECK_VERBOSE"))
                                std::printf("%s d=%d uni=%d bc=%d,%d nc=%d chunks=%d tr=%d err=%.3e %s\n", bad ? "FAIL" : "ok", d,
                                            uni, bc[0], bc[1], nc, chunks, tr, err, bl->structure.c_str());
                        }
                        ddcb::destroy_builder(bl);
                    }
    // Adversarial meshes for the plan's no-pivoting decision: strongly graded cells (widths over six
    // decades), one near-degenerate cell, alternating wide and narrow cells, and a long domain
    // whose Hermite rows carry large dx^k scale factors. The device steps must still match the
    // dense solve with partial pivoting.
    for (int d = 1; d <= 5; ++d)
        for (int kind = 0; kind < 4; ++kind)
            for (auto const& bc : bcs)
                for (int chunks : {4, 32}) {
                    bool const per = bc[0] == 0;
                    int const nc = 60;
                    std::vector<double> w(nc);
                    for (int i = 0; i < nc; ++i) {
                        if (kind == 0) w[i] = std::pow(1e6, double(i) / (nc - 1));
                        else if (kind == 1) w[i] = i == nc / 2 ? 1e-9 : 1.0;
                        else if (kind == 2) w[i] = i % 2 ? 1e-3 : 1.0;
                        else w[i] = 1.0 + 0.3 * U(rng);
                    }
                    double const length = kind == 3 ? 1e4 : 1.0;
                    double tot = 0.0;
                    for (double v : w) tot += v;
                    std::vector<double> br(nc + 1, 0.0);
                    for (int i = 0; i < nc; ++i) br[i + 1] = br[i] + w[i] * length / tot;
                    br[nc] = length;
                    ddcb::Basis b;
                    ddcb::make_non_uniform_basis(b, d, per, br.data(), nc + 1);
                    auto pts = ddcb::greville_points(b, bc[0], bc[1]);
                    ddcb_builder_options opt {0, 2, 8, chunks};
                    ddcb::Builder* bl = nullptr;
                    try {
                        bl = ddcb::create_builder_host(b, pts.data(), long(pts.size()), bc[0], bc[1], &opt);
                    } catch (std::exception const& e) {
                        std::printf("FAIL create adversarial kind=%d d=%d bc=%d,%d: %s\n", kind, d, bc[0], bc[1], e.what());
                        ++failures;
                        continue;
                    }
                    std::vector<double> vals(bl->points.size()), dlo(8), dhi(8);
                    for (auto& v : vals) v = U(rng);
                    for (auto& v : dlo) v = U(rng);
                    for (auto& v : dhi) v = U(rng);
                    double const err = ddcb::emulate_build(*bl, vals.data(), dlo.data(), dhi.data());
                    ++cases;
                    bool const bad = !(err <= 1e-11);
                    if (bad) ++failures;
                    if (bad || std::getenv("PLAN_CHECK_VERBOSE"))
                        std::printf("%s adversarial kind=%d d=%d bc=%d,%d chunks=%d err=%.3e %s\n", bad ? "FAIL" : "ok", kind, d,
                                    bc[0], bc[1], chunks, err, bl->structure.c_str());
                    ddcb::destroy_builder(bl);
                }
    std::printf("plan_check: %d cases, %d failures\n", cases, failures);
    return failures ? 1 : 0;
}
