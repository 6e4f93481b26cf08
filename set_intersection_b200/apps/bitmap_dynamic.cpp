// bitmap_dynamic: drop-in for the reference's `bitmap_dynamic` executable (src/bitmap_dynamic.cu:21-238): same
// flags, same result file; the counts come from libsi_b200.so.
#include "app_common.hpp"

int main(int argc, char** argv) {
    const si_app::Spec spec{"bitmap_dynamic", "GPU dynamic bitmap intersection (bitmap_dynamic)", SI_TECH_BITMAP, si_app::Kind::Sorted, {"blocks", "threads", "partition"}, {"warp"}};
    return si_app::run(spec, argc, argv);
}
