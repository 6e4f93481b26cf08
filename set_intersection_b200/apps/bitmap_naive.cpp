// bitmap_naive: drop-in for the reference's `bitmap_naive` executable (src/bitmap_naive.cu:17-151): same
// flags, same result file; the counts come from libsi_b200.so.
#include "app_common.hpp"

int main(int argc, char** argv) {
    const si_app::Spec spec{"bitmap_naive", "GPU naive bitmap intersection (bitmap_naive)", SI_TECH_BITMAP_NAIVE, si_app::Kind::Dense, {"blocks", "threads"}, {}};
    return si_app::run(spec, argc, argv);
}
