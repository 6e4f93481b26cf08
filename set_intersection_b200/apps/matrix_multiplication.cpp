// matrix_multiplication: drop-in for the reference's `matrix_multiplication` executable (src/matrix_multiplication.cu:14-208): same
// flags, same result file; the counts come from libsi_b200.so.
#include "app_common.hpp"

int main(int argc, char** argv) {
    const si_app::Spec spec{"matrix_multiplication", "GPU matrix multiplication intersection (mm, tensor cores)", SI_TECH_MM, si_app::Kind::Dense, {"partition"}, {}};
    return si_app::run(spec, argc, argv);
}
