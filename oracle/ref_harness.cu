// ref_harness.cu — drives the REFERENCE single-GPU PML program as an oracle pin.
//
// TEST INFRASTRUCTURE ONLY (see oracle/sgfd_oracle.cpp).  oracle/Makefile
// compiles this file together with the reference's own, unmodified
// 3DGPUwithPML_1DArraySingleGPU_optimization/ElasticWaveEquation.cu, taken
// from where it lies, into oracle/_ref/ref_opt.  It constructs the
// reference's ElasticWaveEquation class (OPT/ElasticWaveEquation.h:17-60) and
// advances it through the class's own propagate()/sourceFunction()
// (OPT/ElasticWaveEquation.cu:184-204), exactly as run() does
// (OPT/ElasticWaveEquation.cu:140-182), minus run()'s per-step console line and
// its text snapshots (whose "surf XOY" slice reads past the end of the field,
// OPT/ElasticWaveEquation.cu:895).  It then writes the station trace and the
// nine wavefields in binary so tests can compare them at full precision.
//
// Case file (little-endian): int32 magic 0x43464753 ("SGFC"), int32 version 1,
// int32 nx ny nz pml nt sx sy sz rx ry rz medium_kind, float dt dx dy dz f0,
// float coef[5]; medium_kind 0: float b[n], lambda[n], mu[n] follow;
// medium_kind 1: float rho vp vs follow (homogeneous).
// Output file: float station[nt], then vx vy vz txx tyy tzz txy txz tyz (n each).
// stdout: one line "ref_opt steps=<nt> cells=<computed> ms=<device ms>".

#include "ElasticWaveEquation.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

static void die(const char *m) { std::fprintf(stderr, "ref_harness: %s\n", m); std::exit(2); }

int main(int argc, char **argv) {
    if (argc != 3) die("usage: ref_opt <case.bin> <out.bin>");
    FILE *fp = std::fopen(argv[1], "rb");
    if (!fp) die("cannot open case file");
    int32_t hdr[14];
    float fl[10];
    if (std::fread(hdr, 4, 14, fp) != 14 || hdr[0] != 0x43464753 || hdr[1] != 1) die("bad case header");
    if (std::fread(fl, 4, 10, fp) != 10) die("bad case header");
    const int nx = hdr[2], ny = hdr[3], nz = hdr[4], pml = hdr[5], nt = hdr[6];
    if (nx < 11 || ny < 11 || nz < 11 || nt < 1) die("bad sizes");
    const size_t n = (size_t)nx * ny * nz;
    if (n * sizeof(float) >= (size_t)1 << 31) die("grid too large for the reference's int memsize");

    GRID grid = {nx, ny, nz};
    Delta delta = {fl[0], fl[1], fl[2], fl[3]};
    const float f0 = fl[4];
    SOURCELOCATION src = {hdr[7], hdr[8], hdr[9]};
    STATIONLOCATION sta = {hdr[10], hdr[11], hdr[12]};
    DifferenceCoefficient dc;
    for (int i = 0; i < 5; ++i) dc.diff_coef[i] = fl[5 + i];

    Medium medCPU;
    ALLOCATE_3D_Medium(medCPU);
    if (hdr[13] == 0) {
        if (std::fread(medCPU.buoyancy, 4, n, fp) != n || std::fread(medCPU.lambda, 4, n, fp) != n ||
            std::fread(medCPU.mu, 4, n, fp) != n)
            die("short medium");
    } else {
        float h[3];
        if (std::fread(h, 4, 3, fp) != 3) die("short homogeneous medium");
        const double rho = h[0], vp = h[1], vs = h[2];
        for (size_t i = 0; i < n; ++i) {
            medCPU.buoyancy[i] = (float)(1.0 / rho);
            medCPU.mu[i] = (float)(rho * vs * vs);
            medCPU.lambda[i] = (float)(rho * (vp * vp - 2.0 * vs * vs));
        }
    }
    std::fclose(fp);

    // Launch shape of the reference driver (CON/main.cu:59-61).
    dim3 blocksPerGrid((nx + 31) / 32, (ny + 15) / 16, nz);
    dim3 threadsPerBlock(32, 16);
    GPUDim gpuDim = {blocksPerGrid, threadsPerBlock};

    ElasticWaveEquation ewq(nt, gpuDim, pml, grid, delta, medCPU, src, sta, dc, f0);

    // Medium upload, as run() does (OPT/ElasticWaveEquation.cu:143-147).
    const size_t bytes = n * sizeof(float);
    CHECK(cudaMemcpy(ewq.medGPU.buoyancy, medCPU.buoyancy, bytes, cudaMemcpyHostToDevice));
    CHECK(cudaMemcpy(ewq.medGPU.lambda, medCPU.lambda, bytes, cudaMemcpyHostToDevice));
    CHECK(cudaMemcpy(ewq.medGPU.mu, medCPU.mu, bytes, cudaMemcpyHostToDevice));

    cudaEvent_t e0, e1;
    CHECK(cudaEventCreate(&e0));
    CHECK(cudaEventCreate(&e1));
    CHECK(cudaEventRecord(e0));
    for (int it = 0; it < nt; ++it) ewq.propagate(it, ewq.sourceFunction(it));
    CHECK(cudaEventRecord(e1));
    CHECK(cudaEventSynchronize(e1));
    float ms = 0;
    CHECK(cudaEventElapsedTime(&ms, e0, e1));

    CHECK(cudaMemcpy(ewq.stationDataCPU, ewq.stationDataGPU, nt * sizeof(float), cudaMemcpyDeviceToHost));
    FILE *out = std::fopen(argv[2], "wb");
    if (!out) die("cannot open output");
    std::fwrite(ewq.stationDataCPU, 4, nt, out);
    float *fields[9] = {ewq.vsGPU.velocityX, ewq.vsGPU.velocityY, ewq.vsGPU.velocityZ,
                        ewq.vsGPU.stressXX,  ewq.vsGPU.stressYY,  ewq.vsGPU.stressZZ,
                        ewq.vsGPU.stressXY,  ewq.vsGPU.stressXZ,  ewq.vsGPU.stressYZ};
    std::vector<float> host(n);
    for (int k = 0; k < 9; ++k) {
        CHECK(cudaMemcpy(host.data(), fields[k], bytes, cudaMemcpyDeviceToHost));
        std::fwrite(host.data(), 4, n, out);
    }
    std::fclose(out);
    const long long computed = (long long)(nx - 10) * (ny - 10) * (nz - 10);
    std::printf("ref_opt steps=%d cells=%lld ms=%.4f\n", nt, computed, ms);
    DELETE_3D_Medium(medCPU);
    return 0;
}
