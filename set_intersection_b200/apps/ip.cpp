// ip: drop-in for the reference's `ip` executable (src/ip.cu:14-205): same
// flags, same result file; the counts come from libsi_b200.so.
#include "app_common.hpp"

int main(int argc, char** argv) {
    const si_app::Spec spec{"ip", "GPU intersect path (ip)", SI_TECH_IP, si_app::Kind::Sorted, {"blocks", "threads", "partition"}, {}};
    return si_app::run(spec, argc, argv);
}
