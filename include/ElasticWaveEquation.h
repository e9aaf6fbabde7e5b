/*
 * ElasticWaveEquation.h — the reference's solver class, re-implemented as a
 * host-side wrapper over the C ABI of libsgfd.so (include/sgfd.h).
 *
 * Drop-in for 3DGPUwithPML_1DArraySingleGPU_optimization/ElasticWaveEquation.h:
 * the constructor, the methods and the public members keep the reference's
 * names and signatures (ElasticWaveEquation.h:17-60), so the reference driver
 * main.cu compiles and runs unchanged against this header (link -lsgfd).
 *
 * Behaviour kept from the reference:
 *   - sourceFunction(it) is the reference Ricker wavelet
 *     (ElasticWaveEquation.cu:184-189);
 *   - propagate(it, s) adds dt*dt*s to txx, tyy, tzz at the source, updates
 *     velocities then stresses, and records txx at the station
 *     (ElasticWaveEquation.cu:191-232);
 *   - run() uploads the medium, steps timeLength times printing
 *     "Time Iterator: it", writes the txx slice files every 100 steps from
 *     step 500 on, then writes stationData.txt (ElasticWaveEquation.cu:140-182);
 *   - snapShootSlice / snapShootVolum / stationDataOutput write the same file
 *     names and value orders (ElasticWaveEquation.cu:843-960).  The
 *     reference's "surf XOY" slice indexes past the end of the field
 *     (ElasticWaveEquation.cu:895); here it holds the plane z =
 *     CalculateAreaEndZ that the loop intends.
 *   - the rounding is the reference's (SGFD_ARITH_REF), and its two index
 *     quirks are kept (SGFD_QUIRKS_REF).
 * Differences by design:
 *   - device state belongs to the sgfd handle (padded rows, compact PML
 *     splits), so vsGPU, medGPU, stationDataGPU and the vsPMLCPU split
 *     pointers are null; fields reach the host through vsCPU;
 *   - gpuDim is accepted and ignored: launch shapes are the library's;
 *   - CUDA errors print a message and exit(1), as the reference's CHECK does.
 */
#ifndef ELASTIC_WAVE_EQUATION_H
#define ELASTIC_WAVE_EQUATION_H

#include "sgfd.h"          /* first: ElasticMacro.h defines short macros (R, tau, order) */
#include "ElasticMacro.h"

class ElasticWaveEquation
{
public:
    VelocityStress vsGPU;
    VelocityStress vsCPU;

    int timeLength;
    GRID grid; Delta delta; Medium medGPU; Medium medCPU;
    DifferenceCoefficient dc;
    float mainFrequncy;

    GPUDim gpuDim;
    int pml;

    VelocityStressPML vsPMLCPU[26];

    SOURCELOCATION sourceLocationCPU;
    STATIONLOCATION stationLocationCPU;

    float *stationDataCPU;
    float *stationDataGPU;

    ElasticWaveEquation(
        int timeLength, GPUDim gpuDim, int pml,
        GRID grid, Delta delta, Medium medCPU,
        SOURCELOCATION sourceLocation, STATIONLOCATION stationLocationCPU,
        DifferenceCoefficient dc,
        float mainFrequncy );
    ~ElasticWaveEquation();
    ElasticWaveEquation(const ElasticWaveEquation &) = delete;
    ElasticWaveEquation &operator=(const ElasticWaveEquation &) = delete;

    void propagate( int timeIndex, float sourceValue );
    float sourceFunction( int timeIndex );
    void snapShootVolum(int it);
    void snapShootSlice(int it);
    void run();
    void calStartEndPoint( );
    void vsPMLCPUTovsPML( );
    void stationLocationCPUTostationLocationGPU();
    void sourceLocationCPUTosourceLocationGPU();
    void stationDataOutput();

    /* The libsgfd handle behind this object (not in the reference). */
    sgfd_solver *handle() const { return solver_; }

private:
    sgfd_solver *solver_;
    bool mediumUploaded_;
    void check(int status, const char *what);
    void downloadField(int field, float *dst);
};

#endif /* ELASTIC_WAVE_EQUATION_H */
