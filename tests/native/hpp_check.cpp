// Compile-and-run check of include/ddcb.hpp on a machine without a GPU: the basis and its Greville
// points are host objects; creating a builder needs a CUDA device, so without one the C++ wrapper
// must report the library's error as std::runtime_error.
#include <cstdio>
#include <stdexcept>

#include "../../include/ddcb.hpp"

int main()
{
    auto bs = ddcb::BSplines::uniform(3, true, 0.0, 1.0, 1000);
    auto pts = bs.greville_points(ddcb::SplineBuilderClosure::PERIODIC, ddcb::SplineBuilderClosure::PERIODIC);
    if (pts.size() != 1000 || bs.info().size != 1003) {
        std::printf("FAIL greville %zu size %lld\n", pts.size(), (long long)bs.info().size);
        return 1;
    }
    auto moved = std::move(bs);
    try {
        ddcb::SplineBuilder b(moved, ddcb::SplineBuilderClosure::PERIODIC, ddcb::SplineBuilderClosure::PERIODIC);
        ddcb::SplineEvaluator ev(moved);
        ddcb::HostPipeline pipe(b, ev, 0, 16, 64);
        std::printf("OK builder created (a GPU is present): nbasis %lld\n", (long long)b.info().nbasis);
    } catch (std::runtime_error const& e) {
        std::printf("OK runtime_error: %s\n", e.what());
    }
    try {
        ddcb::BSplines::non_uniform(3, false, {0.0, 0.5, 0.2, 1.0});
        std::printf("FAIL unsorted breaks accepted\n");
        return 1;
    } catch (std::runtime_error const& e) {
        std::printf("OK bad grid: %s\n", e.what());
    }
    return 0;
}
