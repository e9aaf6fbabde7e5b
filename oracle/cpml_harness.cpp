// cpml_harness.cpp — times the reference's CPU split-field PML program
// (3DCPUwithPML_3DArray_GridIncludePMLandOrder/, "CPML" below) as shipped,
// single-threaded, for the CPU baseline of the measurement.  Test and
// measurement infrastructure only; nothing of the product links it.
//
// The reference sources are compiled where they lie (oracle/Makefile puts
// their directory on the include path).  Its destructor
// (CPML/ElasticWaveEquation3D.cpp:43-46) calls the two-argument member
// declaration macro DEF_3D_VelocityStress with five arguments, which no
// compiler accepts; the class header is included first, with the macro as
// the reference defines it, and the macro is then redefined to take any
// number of arguments and expand to nothing before the .cpp is included, so
// those four destructor lines vanish (the arrays are released at exit).
// Nothing else of the reference changes.
//
// The timed loop is the body of CPML's propagate() (CPML/ElasticWaveEquation3D.cpp:53-85)
// without its file and console output: loadSeismicSource, velocityUpdate,
// stressUpdate per step, after calculateDamping.
//
//   cpml_bench <interior edge> <pml> <steps> <ftz 0|1>
// prints: cells=<updated cells per step> steps=<timed steps> seconds=<wall time>
#include "ElasticWaveEquation3D.h"
#undef DEF_3D_VelocityStress
#define DEF_3D_VelocityStress(...)
#include "ElasticWaveEquation3D.cpp"

#include <xmmintrin.h>

#include <chrono>
#include <cstdlib>

int main(int argc, char **argv) {
    const int n = argc > 1 ? std::atoi(argv[1]) : 101;
    const int pml = argc > 2 ? std::atoi(argv[2]) : 10;
    const int steps = argc > 3 ? std::atoi(argv[3]) : 10;
    const bool ftz = argc > 4 && std::atoi(argv[4]) != 0;
    if (n < 8 || pml < 1 || steps < 1) return 2;
    if (ftz) _mm_setcsr(_mm_getcsr() | 0x8040);   // flush-to-zero and denormals-are-zero
    GRID grid = {n, n, n};
    SOURCELOCATION src = {0};
    src.x = grid.xLength / 2 + pml + ORDER / 2;   // the reference main.cpp's source cell
    src.y = grid.yLength / 2 + pml + ORDER / 2;
    src.z = grid.zLength / 2 + pml + ORDER / 2;
    const int N = n + 2 * pml + ORDER;
    DEF_3D_POINTER(float, buoyancy);
    DEF_3D_POINTER(float, lambda);
    DEF_3D_POINTER(float, mu);
    ALLOCATE_3D(float, buoyancy, N, N, N);
    ALLOCATE_3D(float, lambda, N, N, N);
    ALLOCATE_3D(float, mu, N, N, N);
    // the reference main.cpp's homogeneous medium: rho 2500, velocity Vs
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j)
            for (int k = 0; k < N; ++k) {
                buoyancy[i][j][k] = 1.0f / 2500.0f;
                lambda[i][j][k] = 2500.0f * Vs * Vs;
                mu[i][j][k] = 2500.0f * Vs * Vs / 3.0f;
            }
    ElasticWaveEquation3D ewq(grid, steps + 1, pml, buoyancy, lambda, mu, src);
    ewq.calculateDamping();
    ewq.loadSeismicSource(0);   // one untimed step
    ewq.velocityUpdate();
    ewq.stressUpdate();
    const auto t0 = std::chrono::steady_clock::now();
    for (int it = 1; it <= steps; ++it) {
        ewq.loadSeismicSource(it);
        ewq.velocityUpdate();
        ewq.stressUpdate();
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const long long cells = (long long)(n + 2 * pml) * (n + 2 * pml) * (n + 2 * pml);
    std::printf("cells=%lld steps=%d seconds=%.6f\n", cells, steps, secs);
    return 0;
}
