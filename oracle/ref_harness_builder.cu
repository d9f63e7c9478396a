// ref_harness_builder.cu -- single-face boundary-condition builder for the
// reference program (test infrastructure, compiled by ref_build.py into the
// reference build in place of its builder file; never part of libvlbm).
//
// It implements the reference's builder hook, gpuBuildBoundaryConditions and
// gpuSchSpecial (boundaryConditionsBuilder.h:21-22, boundaryConditionsHandler.h:52-58),
// with the NodeTypeMap setters of structs/nodeTypeMap.h, so that one face of the
// lattice carries a boundary scheme none of the reference's builder files puts
// there (velocity Zou-He on the west, east, front and back faces, pressure
// Zou-He with a chosen density):
//
//   HARNESS_FACE    direction code of the face under test (NORTH .. BACK)
//   HARNESS_SCHEME  its scheme (BC_SCHEME_VEL_ZOUHE or BC_SCHEME_PRES_ZOUHE)
//
// The face carries value index 1: UX_BC[1] on west/east, UZ_BC[1] on
// front/back, UY_BC[1] on north/south for velocity; RHO_BC[1] for pressure.
// Half-way bounce-back walls close the two faces normal to y (to z when the
// face under test is north or south) and win on the shared edges; the
// remaining axes are periodic.  oracle.harness_map writes the same words.
#include "boundaryConditionsBuilder.h"

#if !defined(HARNESS_FACE) || !defined(HARNESS_SCHEME)
#error "HARNESS_FACE and HARNESS_SCHEME must be defined"
#endif

__global__
void gpuBuildBoundaryConditions(NodeTypeMap* const gpuMapBC, int gpuNumber)
{
    const unsigned int x = threadIdx.x + blockDim.x * blockIdx.x;
    const unsigned int y = threadIdx.y + blockDim.y * blockIdx.y;
    const unsigned int z = threadIdx.z + blockDim.z * blockIdx.z;
    if (x >= NX || y >= NY || z >= NZ)
        return;
    const unsigned int zg = z + NZ * gpuNumber;
    NodeTypeMap& m = gpuMapBC[idxScalar(x, y, z)];
    m.setIsUsed(true);
    m.setSavePostCol(false);
    m.setSchemeBC(BC_NULL);
    m.setGeometry(CONCAVE);
    m.setUxIdx(0);
    m.setUyIdx(0);
    m.setUzIdx(0);
    m.setRhoIdx(0);

    const int face = HARNESS_FACE;
    const bool wallsInZ = (face == NORTH || face == SOUTH);
    // walls first: they take the edges they share with the face under test
    if (wallsInZ) {
        if (zg == 0) { m.setSchemeBC(BC_SCHEME_BOUNCE_BACK); m.setDirection(BACK); return; }
        if (zg == NZ_TOTAL - 1) { m.setSchemeBC(BC_SCHEME_BOUNCE_BACK); m.setDirection(FRONT); return; }
    } else {
        if (y == 0) { m.setSchemeBC(BC_SCHEME_BOUNCE_BACK); m.setDirection(SOUTH); return; }
        if (y == NY - 1) { m.setSchemeBC(BC_SCHEME_BOUNCE_BACK); m.setDirection(NORTH); return; }
    }
    bool onFace = false;
    switch (face) {
    case NORTH: onFace = (y == NY - 1); break;
    case SOUTH: onFace = (y == 0); break;
    case WEST: onFace = (x == 0); break;
    case EAST: onFace = (x == NX - 1); break;
    case FRONT: onFace = (zg == NZ_TOTAL - 1); break;
    case BACK: onFace = (zg == 0); break;
    default: break;
    }
    if (!onFace)
        return;
    m.setSchemeBC(HARNESS_SCHEME);
    m.setDirection(face);
    if (HARNESS_SCHEME == BC_SCHEME_PRES_ZOUHE) {
        m.setRhoIdx(1);
    } else if (face == WEST || face == EAST) {
        m.setUxIdx(1);
    } else if (face == FRONT || face == BACK) {
        m.setUzIdx(1);
    } else {
        m.setUyIdx(1);
    }
}


__device__
void gpuSchSpecial(NodeTypeMap* gpuNT,
    dfloat* fPostStream,
    dfloat* fPostCol,
    const short unsigned int x,
    const short unsigned int y,
    const short unsigned int z)
{
    // the harness places no special-scheme node
}
