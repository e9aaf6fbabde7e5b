/*
 * ElasticMacro.h — source-compatible stand-in for the reference's parameter
 * header (3DGPUwithPML_1DArraySingleGPU_optimization/ElasticMacro.h).
 *
 * A program written against the reference (its main.cu) compiles unchanged
 * against this header and ElasticWaveEquation.h; the solver behind them is
 * libsgfd.so (include/sgfd.h).  Kept from the reference, with the same names
 * and values because user code refers to them:
 *   - the standard headers and `using namespace std` that main.cu relies on
 *     (it calls cout, pow and time unqualified; ElasticMacro.h:9-17);
 *   - the constants PI, R, tau, ORDER, order, nAREA (ElasticMacro.h:19-28);
 *   - the INDEX, DAMPING, region-bound and medium-average macros
 *     (ElasticMacro.h:22-41, 106-119), which expand against variables named
 *     `grid` and `pml` in scope, as in the reference;
 *   - the region ids VERTEX0..EDGE11 (ElasticMacro.h:77-102);
 *   - the host allocation macros ALLOCATE_3D_Medium / DELETE_3D_Medium and
 *     ALLOCATE_3D_VelocityStress / DELETE_3D_VelocityStress
 *     (ElasticMacro.h:200-218, 271-295);
 *   - the plain structs GRID, Delta, VelocityStress, VelocityStressPML,
 *     Medium, DifferenceCoefficient, GPUDim, SOURCELOCATION, STATIONLOCATION
 *     (ElasticMacro.h:300-401).
 * Not kept: the CUDA allocation macros and the PML update macros, which in
 * the reference are the kernels' implementation, not part of its interface.
 */
#ifndef ELASTIC_MACRO_H
#define ELASTIC_MACRO_H

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iostream>
#include <memory.h>
#include <vector_types.h>   /* dim3 for GPUDim */
using namespace std;

#define PI 3.1415926f
#define R 0.001f
#define tau 4.3f
#define INDEX( ix, iy, iz ) (ix) + (iy) * grid.xLength + (iz) * grid.yLength * grid.xLength
#define ORDER 10
#define order 5
#define DAMPING0( V, pml, delta ) tau * V / ( delta ) * ( 8.0f / 15.0f - 0.03f * ( pml ) + 1.0f / 1500.0f * ( ( pml ) * ( pml ) ) )
#define DAMPING( V, i, pml, delta ) DAMPING0( V, pml, delta ) * powf( ( i ) * 1.0f / ( ( pml ) * 1.0f ), 2 )
#define nAREA 26

#define START order
#define CalculateAreaStart order + pml
#define CalculateAreaEndX grid.xLength - order - pml
#define CalculateAreaEndY grid.yLength - order - pml
#define CalculateAreaEndZ grid.zLength - order - pml
#define EndX grid.xLength - order
#define EndY grid.yLength - order
#define EndZ grid.zLength - order

#define AreaCondition( ix, iy, iz, start_x, start_y, start_z, end_x, end_y, end_z ) \
    ( start_x <= ix && ix < end_x ) && ( start_y <= iy && iy < end_y ) && ( start_z <= iz && iz < end_z )

/* PML region ids: 8 vertices, 6 surfaces, 12 edges of the absorbing shell. */
#define VERTEX0 0
#define VERTEX1 1
#define VERTEX2 2
#define VERTEX3 3
#define VERTEX4 4
#define VERTEX5 5
#define VERTEX6 6
#define VERTEX7 7
#define SURFACE0 8
#define SURFACE1 9
#define SURFACE2 10
#define SURFACE3 11
#define SURFACE4 12
#define SURFACE5 13
#define EDGE0 14
#define EDGE1 15
#define EDGE2 16
#define EDGE3 17
#define EDGE4 18
#define EDGE5 19
#define EDGE6 20
#define EDGE7 21
#define EDGE8 22
#define EDGE9 23
#define EDGE10 24
#define EDGE11 25

/* Staggered-grid medium averages: 2-point buoyancy, 4-point harmonic mu. */
#define BUOYANCYBAR( buoyancy1, buoyancy2 ) ( ( buoyancy1 + buoyancy2 ) / 2 )
#define BUOYANCYBARX( buoyancy, ix, iy, iz ) BUOYANCYBAR( buoyancy[INDEX( ix, iy, iz )], buoyancy[INDEX( ix + 1, iy, iz )] )
#define BUOYANCYBARY( buoyancy, ix, iy, iz ) BUOYANCYBAR( buoyancy[INDEX( ix, iy, iz )], buoyancy[INDEX( ix, iy + 1, iz )] )
#define BUOYANCYBARZ( buoyancy, ix, iy, iz ) BUOYANCYBAR( buoyancy[INDEX( ix, iy, iz )], buoyancy[INDEX( ix, iy, iz + 1 )] )
#define MUBAR( mu1, mu2, mu3, mu4 ) ( 4.0f / ( 1 / mu1 + 1 / mu2 + 1 / mu3 + 1 / mu4 ) )
#define MUBARXY( mu, ix, iy, iz ) \
    MUBAR( mu[INDEX( ix, iy, iz )], mu[INDEX( ix + 1, iy, iz )], mu[INDEX( ix, iy + 1, iz )], mu[INDEX( ix + 1, iy + 1, iz )] )
/* The reference's txz average takes mu[ix+1, iy+1, iz] as its fourth point
 * (ElasticMacro.h:116-117); the solver reproduces it with SGFD_QUIRKS_REF. */
#define MUBARXZ( mu, ix, iy, iz ) \
    MUBAR( mu[INDEX( ix, iy, iz )], mu[INDEX( ix + 1, iy, iz )], mu[INDEX( ix, iy, iz + 1 )], mu[INDEX( ix + 1, iy + 1, iz )] )
#define MUBARYZ( mu, ix, iy, iz ) \
    MUBAR( mu[INDEX( ix, iy, iz )], mu[INDEX( ix, iy + 1, iz )], mu[INDEX( ix, iy, iz + 1 )], mu[INDEX( ix, iy + 1, iz + 1 )] )

/* Host allocations (the reference's main.cu uses the Medium pair). */
#define ALLOCATE_3D_Medium( med ) \
    med.buoyancy = new float[ (size_t)grid.xLength * grid.yLength * grid.zLength ]; \
    med.lambda   = new float[ (size_t)grid.xLength * grid.yLength * grid.zLength ]; \
    med.mu       = new float[ (size_t)grid.xLength * grid.yLength * grid.zLength ];

#define DELETE_3D_Medium( med ) \
    delete [] med.buoyancy; \
    delete [] med.lambda; \
    delete [] med.mu;

#define ALLOCATE_3D_VelocityStress( vs, n ) \
    vs.stressXX  = new float[ n ](); vs.stressYY = new float[ n ](); vs.stressZZ = new float[ n ](); \
    vs.stressXY  = new float[ n ](); vs.stressXZ = new float[ n ](); vs.stressYZ = new float[ n ](); \
    vs.velocityX = new float[ n ](); vs.velocityY = new float[ n ](); vs.velocityZ = new float[ n ]();

#define DELETE_3D_VelocityStress( vs ) \
    delete[] vs.stressXX; delete[] vs.stressYY; delete[] vs.stressZZ; \
    delete[] vs.stressXY; delete[] vs.stressXZ; delete[] vs.stressYZ; \
    delete[] vs.velocityX; delete[] vs.velocityY; delete[] vs.velocityZ;

typedef struct SOURCELOCATION { int x; int y; int z; } SOURCELOCATION;
typedef struct GRID { int xLength; int yLength; int zLength; } GRID;
typedef struct Delta { float t; float x; float y; float z; } Delta;

typedef struct VelocityStress {
    float *stressXX;
    float *stressYY;
    float *stressZZ;
    float *stressXY;
    float *stressXZ;
    float *stressYZ;
    float *velocityX;
    float *velocityY;
    float *velocityZ;
} VelocityStress;

/* One PML region: its split fields and its [start, end) box.  With
 * libsgfd the split state lives in the solver's compact PML array, so the
 * pointers stay null; the bounds are filled as the reference fills them. */
typedef struct VelocityStressPML {
    float *stressXXx, *stressXXy, *stressXXz;
    float *stressYYx, *stressYYy, *stressYYz;
    float *stressZZx, *stressZZy, *stressZZz;
    float *stressXYx, *stressXYy;
    float *stressXZx, *stressXZz;
    float *stressYZy, *stressYZz;
    float *velocityXx, *velocityXy, *velocityXz;
    float *velocityYx, *velocityYy, *velocityYz;
    float *velocityZx, *velocityZy, *velocityZz;
    int startX, startY, startZ;
    int endX, endY, endZ;
    int xLength, yLength, zLength;
} VelocityStressPML;

typedef struct Medium { float *buoyancy; float *lambda; float *mu; } Medium;
typedef struct DifferenceCoefficient { float diff_coef[ORDER / 2]; } DifferenceCoefficient;
typedef struct GPUDim { dim3 blocksPerGrid; dim3 threadsPerBlock; } GPUDim;
typedef struct STATIONLOCATION { int x; int y; int z; } STATIONLOCATION;

#endif /* ELASTIC_MACRO_H */
