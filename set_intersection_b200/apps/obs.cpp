// obs: drop-in for the reference's `obs` executable (src/obs.cu:38-273): same
// flags, same result file; the counts come from libsi_b200.so.
#include "app_common.hpp"

int main(int argc, char** argv) {
    const si_app::Spec spec{"obs", "GPU optimized binary search (obs)", SI_TECH_OBS, si_app::Kind::Sorted, {"blocks", "threads", "partition"}, {"warp", "path"}};
    return si_app::run(spec, argc, argv);
}
