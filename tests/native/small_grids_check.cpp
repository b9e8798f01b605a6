// Host-side sweep of the builder plan over tiny grids: 1..15 cells, degrees 1..5, periodic /
// Hermite / Greville closures, uniform and non-uniform meshes. Every grid is either planned or
// refused with an ddcb::Error (a periodic basis needs more cells than its degree); none may read or
// write outside its arrays (the test compiles this file with AddressSanitizer and
// UndefinedBehaviorSanitizer). Prints the number of planned and refused grids.
#include <cstdio>
#include <vector>

#include "../../ddc_b200/csrc/ddcb_internal.hpp"

int main()
{
    int planned = 0, refused = 0, wrong = 0;
    int const closures[] = {DDCB_PERIODIC, DDCB_HERMITE, DDCB_GREVILLE};
    for (int uni = 0; uni < 2; ++uni)
        for (int c : closures)
            for (int d = 1; d <= 5; ++d)
                for (int nc = 1; nc < 16; ++nc) {
                    bool const per = c == DDCB_PERIODIC;
                    ddcb::Basis b;
                    if (uni) ddcb::make_uniform_basis(b, d, per, 0.0, 2.0, nc);
                    else {
                        std::vector<double> br(nc + 1);
                        for (int i = 0; i <= nc; ++i) br[i] = 2.0 * i / nc + (i > 0 && i < nc ? 0.1 / nc * ((i % 3) - 1) : 0.0);
                        ddcb::make_non_uniform_basis(b, d, per, br.data(), nc + 1);
                    }
                    try {
                        auto pts = ddcb::greville_points(b, c, c);
                        ddcb_builder_options opt {0, 2, 8, 0, 0.0};
                        ddcb::Builder* bl = ddcb::create_builder_host(b, pts.data(), long(pts.size()), c, c, &opt);
                        ddcb::destroy_builder(bl);
                        ++planned;
                        if (per && nc <= d) ++wrong;
                    } catch (ddcb::Error const&) {
                        ++refused;
                        if (!(per && nc <= d)) ++wrong;
                    }
                }
    std::printf("small_grids_check: %d planned, %d refused, %d unexpected\n", planned, refused, wrong);
    return wrong ? 1 : 0;
}
