// ElasticWaveEquation.cpp — the reference's solver class as a host-side
// wrapper over the C ABI (include/sgfd.h).  See include/ElasticWaveEquation.h
// for what is kept from 3DGPUwithPML_1DArraySingleGPU_optimization/ and what
// differs.  Compiled into libsgfd.so.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/ElasticWaveEquation.h"

void ElasticWaveEquation::check(int status, const char *what) {
    if (status == SGFD_OK) return;
    std::fprintf(stderr, "ElasticWaveEquation: %s failed (%d): %s\n", what, status,
                 solver_ ? sgfd_last_error(solver_) : sgfd_global_error());
    std::exit(1);   // the reference's CHECK exits too (common.h:6-16)
}

ElasticWaveEquation::ElasticWaveEquation(int timeLength, GPUDim gpuDim, int pml, GRID grid, Delta delta,
                                         Medium medCPU, SOURCELOCATION sourceLocationCPU,
                                         STATIONLOCATION stationLocationCPU, DifferenceCoefficient dc,
                                         float mainFrequncy)
    : timeLength(timeLength), grid(grid), delta(delta), medCPU(medCPU), dc(dc), mainFrequncy(mainFrequncy),
      gpuDim(gpuDim), pml(pml), sourceLocationCPU(sourceLocationCPU), stationLocationCPU(stationLocationCPU),
      solver_(nullptr), mediumUploaded_(false) {
    const size_t n = (size_t)grid.xLength * grid.yLength * grid.zLength;
    std::memset(&vsGPU, 0, sizeof vsGPU);
    std::memset(&medGPU, 0, sizeof medGPU);
    std::memset(vsPMLCPU, 0, sizeof vsPMLCPU);
    stationDataCPU = new float[timeLength > 0 ? timeLength : 1]();
    stationDataGPU = nullptr;

    calStartEndPoint();
    ALLOCATE_3D_VelocityStress(vsCPU, n);
    // region extents, as the reference sizes its split arrays (ElasticWaveEquation.cu:34-41)
    for (int i = 0; i < nAREA; ++i) {
        vsPMLCPU[i].xLength = vsPMLCPU[i].endX - vsPMLCPU[i].startX + 1;
        vsPMLCPU[i].yLength = vsPMLCPU[i].endY - vsPMLCPU[i].startY + 1;
        vsPMLCPU[i].zLength = vsPMLCPU[i].endZ - vsPMLCPU[i].startZ + 1;
    }

    sgfd_config c;
    sgfd_config_default(&c);
    c.nx = grid.xLength;
    c.ny = grid.yLength;
    c.nz = grid.zLength;
    c.pml = pml;
    c.dt = delta.t;
    c.dx = delta.x;
    c.dy = delta.y;
    c.dz = delta.z;
    for (int i = 0; i < ORDER / 2; ++i) c.coef[i] = dc.diff_coef[i];
    c.damping = SGFD_DAMP_REFGPU;
    c.quirks = SGFD_QUIRKS_REF;
    c.arith = SGFD_ARITH_REF;
    check(sgfd_create(&c, &solver_), "sgfd_create");
    vsPMLCPUTovsPML();
    sourceLocationCPUTosourceLocationGPU();
    stationLocationCPUTostationLocationGPU();
}

ElasticWaveEquation::~ElasticWaveEquation() {
    sgfd_destroy(solver_);
    DELETE_3D_VelocityStress(vsCPU);
    delete[] stationDataCPU;
}

// The 26-region table of the PML shell (ElasticWaveEquation.cu:47-108): for
// each axis a region covers the low band [5, 5+pml), the interior
// [5+pml, n-5-pml) or the high band [n-5-pml, n-5).
void ElasticWaveEquation::calStartEndPoint() {
    const int lo[3] = {START, START, START};
    const int a[3] = {CalculateAreaStart, CalculateAreaStart, CalculateAreaStart};
    const int b[3] = {CalculateAreaEndX, CalculateAreaEndY, CalculateAreaEndZ};
    const int hi[3] = {EndX, EndY, EndZ};
    // band per axis: 0 = low PML band, 1 = interior, 2 = high PML band
    auto set = [&](int id, int bx, int by, int bz) {
        const int band[3] = {bx, by, bz};
        int s[3], e[3];
        for (int k = 0; k < 3; ++k) {
            s[k] = band[k] == 0 ? lo[k] : band[k] == 1 ? a[k] : b[k];
            e[k] = band[k] == 0 ? a[k] : band[k] == 1 ? b[k] : hi[k];
        }
        vsPMLCPU[id].startX = s[0]; vsPMLCPU[id].startY = s[1]; vsPMLCPU[id].startZ = s[2];
        vsPMLCPU[id].endX = e[0]; vsPMLCPU[id].endY = e[1]; vsPMLCPU[id].endZ = e[2];
    };
    set(VERTEX0, 0, 0, 0); set(VERTEX1, 0, 0, 2); set(VERTEX2, 0, 2, 0); set(VERTEX3, 0, 2, 2);
    set(VERTEX4, 2, 0, 0); set(VERTEX5, 2, 0, 2); set(VERTEX6, 2, 2, 0); set(VERTEX7, 2, 2, 2);
    set(SURFACE0, 0, 1, 1); set(SURFACE1, 2, 1, 1); set(SURFACE2, 1, 0, 1);
    set(SURFACE3, 1, 2, 1); set(SURFACE4, 1, 1, 0); set(SURFACE5, 1, 1, 2);
    set(EDGE0, 0, 0, 1); set(EDGE1, 0, 2, 1); set(EDGE2, 0, 1, 0); set(EDGE3, 0, 1, 2);
    set(EDGE4, 2, 0, 1); set(EDGE5, 2, 2, 1); set(EDGE6, 2, 1, 0); set(EDGE7, 2, 1, 2);
    set(EDGE8, 1, 0, 0); set(EDGE9, 1, 0, 2); set(EDGE10, 1, 2, 0); set(EDGE11, 1, 2, 2);
}

// The split-field state is implied by pml inside libsgfd; nothing to upload.
void ElasticWaveEquation::vsPMLCPUTovsPML() {}

void ElasticWaveEquation::sourceLocationCPUTosourceLocationGPU() {
    check(sgfd_set_source(solver_, sourceLocationCPU.x, sourceLocationCPU.y, sourceLocationCPU.z), "set source");
}

void ElasticWaveEquation::stationLocationCPUTostationLocationGPU() {
    const int32_t xyz[3] = {stationLocationCPU.x, stationLocationCPU.y, stationLocationCPU.z};
    const int32_t comp = SGFD_TXX;   // the reference station records txx
    check(sgfd_set_receivers(solver_, 1, xyz, &comp, timeLength > 0 ? timeLength : 1), "set station");
}

float ElasticWaveEquation::sourceFunction(int timeIndex) {
    return sgfd_ricker_ref(mainFrequncy, delta.t, timeIndex);
}

void ElasticWaveEquation::propagate(int timeIndex, float sourceValue) {
    if (!mediumUploaded_) {
        check(sgfd_set_medium(solver_, medCPU.buoyancy, medCPU.lambda, medCPU.mu), "medium upload");
        mediumUploaded_ = true;
    }
    check(sgfd_step(solver_, timeIndex, sourceValue), "propagate");
}

void ElasticWaveEquation::downloadField(int field, float *dst) {
    check(sgfd_get_field(solver_, field, dst), "field download");
}

void ElasticWaveEquation::run() {
    check(sgfd_set_medium(solver_, medCPU.buoyancy, medCPU.lambda, medCPU.mu), "medium upload");
    mediumUploaded_ = true;
    for (int it = 0; it < timeLength; it++) {
        cout << "Time Iterator: " << it << endl;
        const float sourceValue = sourceFunction(it);
        propagate(it, sourceValue);
        if (it % 100 == 0 && it >= 500) {
            downloadField(SGFD_TXX, vsCPU.stressXX);
            snapShootSlice(it);
        }
    }
    check(sgfd_get_traces(solver_, stationDataCPU), "station download");
    stationDataOutput();
}

// txx slices through the source (YoZ, XoZ, XOY) and through the inner faces
// of the high PML bands ("surf"), one value per line
// (ElasticWaveEquation.cu:843-909).
void ElasticWaveEquation::snapShootSlice(int it) {
    const char *names[6] = {"snapshotSliceXX_YoZ_%d.txt", "snapshotSliceXX_XoZ_%d.txt", "snapshotSliceXX_XOY_%d.txt",
                            "surfSliceXX_YoZ_%d.txt", "surfSliceXX_XoZ_%d.txt", "surfSliceXX_XOY_%d.txt"};
    ofstream f[6];
    for (int k = 0; k < 6; ++k) {
        char name[128];
        std::snprintf(name, sizeof name, names[k], it);
        f[k].open(name);
    }
    const float *txx = vsCPU.stressXX;
    const int sx = sourceLocationCPU.x, sy = sourceLocationCPU.y, sz = sourceLocationCPU.z;
    const int ex = CalculateAreaEndX, ey = CalculateAreaEndY, ez = CalculateAreaEndZ;
    for (int iz = 0; iz < grid.zLength; ++iz)
        for (int iy = 0; iy < grid.yLength; ++iy) {
            f[0] << txx[INDEX(sx, iy, iz)] << endl;
            f[3] << txx[INDEX(ex, iy, iz)] << endl;
        }
    for (int iz = 0; iz < grid.zLength; ++iz)
        for (int ix = 0; ix < grid.xLength; ++ix) {
            f[1] << txx[INDEX(ix, sy, iz)] << endl;
            f[4] << txx[INDEX(ix, ey, iz)] << endl;
        }
    for (int iy = 0; iy < grid.yLength; ++iy)
        for (int ix = 0; ix < grid.xLength; ++ix) {
            f[2] << txx[INDEX(ix, iy, sz)] << endl;
            f[5] << txx[INDEX(ix, iy, ez)] << endl;
        }
}

// txx over the computed region, x fastest, one value per line
// (ElasticWaveEquation.cu:911-948).  Like the reference it writes vsCPU as it is.
void ElasticWaveEquation::snapShootVolum(int it) {
    char name[128];
    std::snprintf(name, sizeof name, "snapshot_%d_%d.txt", 0, it);
    cout << name << endl;
    ofstream f(name);
    for (int iz = order; iz < grid.zLength - order; iz++)
        for (int iy = order; iy < grid.yLength - order; iy++)
            for (int ix = order; ix < grid.xLength - order; ix++) f << vsCPU.stressXX[INDEX(ix, iy, iz)] << endl;
}

void ElasticWaveEquation::stationDataOutput() {
    ofstream f("stationData.txt");
    for (int i = 0; i < timeLength; ++i) f << stationDataCPU[i] << endl;
}
