// hi: drop-in for the reference's `hi` executable (src/hi.cu:47-293): same
// flags, same result file; the counts come from libsi_b200.so.
#include "app_common.hpp"

int main(int argc, char** argv) {
    const si_app::Spec spec{"hi", "GPU hash intersection (hi)", SI_TECH_HI, si_app::Kind::Sorted, {"blocks", "threads", "partition", "buckets", "bucket-size"}, {"warp", "path"}};
    return si_app::run(spec, argc, argv);
}
