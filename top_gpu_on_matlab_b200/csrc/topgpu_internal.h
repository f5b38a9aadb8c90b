// topgpu_internal.h -- shared internal declarations of libtopgpu.so.
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include "topgpu.h"

namespace topgpu {

void set_error(const char *fmt, ...);

// Local node d-offsets (dy, dx, dz) of the eight element corners in the
// reference's eNodMat column order (TOP_GPU.m:2083-2090): column j of an
// element with base voxel (ey, ex, ez) is node (ey+dy, ex+dx, ez+dz).
constexpr int kCornerDY[8] = {1, 1, 0, 0, 1, 1, 0, 0};
constexpr int kCornerDX[8] = {0, 1, 1, 0, 0, 1, 1, 0};
constexpr int kCornerDZ[8] = {0, 0, 0, 0, 1, 1, 1, 1};

struct MeshLevel {
    int resX = 0, resY = 0, resZ = 0;   // element grid
    int span = 0;                       // coarsening factor to this level (0 on level 0)
    int64_t Ne = 0, Nn = 0, nInt = 0;
    std::vector<int32_t> eleMapBack, eleMapForward, eNodMat, nodMapBack, nodMapForward;
    std::vector<int32_t> nodesOnBoundary, elementsOnBoundary;
    std::vector<int32_t> elementUpwardMap, transferMat, solidNodeMap;
    std::vector<double> transferMatCoeffi, RI;
    std::vector<int32_t> nodeCount;     // active elements incident to each node
    double Ke[576];
    int64_t gridNodes() const { return int64_t(resX + 1) * (resY + 1) * (resZ + 1); }
    int64_t gridElems() const { return int64_t(resX) * resY * resZ; }
};

}  // namespace topgpu

struct top_mesh {
    int nely = 0, nelx = 0, nelz = 0, control = 0, superElement = 0;
    double nu = 0.3, cellSize = 1.0;
    std::vector<topgpu::MeshLevel> L;
    // boundary conditions (empty until apply_bc / apply_optcase)
    bool hasBC = false;
    int64_t nFix = 0;
    std::vector<int32_t> fixingCond;     // [nFix x 4] col-major
    int nLoads = 0;
    std::vector<double> F;               // [3Nn x nLoads]
    std::vector<double> weights;
    std::vector<int32_t> mapUniqueKes, eleWithFixedDOFs;
    std::vector<double> uniqueKesFree, uniqueKesFixed;
    std::vector<uint8_t> nodeFixed;      // level-0 compact nodes: bit c = component c fixed
    std::vector<double> I_mat;           // super-element sub-voxel stiffnesses [576 x 64]
    // .TopVoxel models: passive elements (compact, ascending) and the file's
    // per-voxel densities (file order; empty when the file has none)
    std::vector<int32_t> passiveElements;
    std::vector<double> densityLayout;
};

namespace topgpu {
// child slot -> position of the child inside its coarse cell, following the
// reference's sub-element lists (TOP_GPU.m:1938-2017)
void child_slot_position(int span, int slot, int *ly, int *lx, int *lz);
// trilinear weight of coarse corner j at fine position (ly,lx,lz) of a span-s cell
double trilinear_weight(int span, int ly, int lx, int lz, int j);
// Galerkin prolongation block P_s (24x24 col-major) of child slot s
void child_prolongation(int span, int slot, double *P);
}  // namespace topgpu
