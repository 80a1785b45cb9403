// CBCTSinMatPolyForwardProjGrid.cpp — see CBCTSinMatPolyForwardProjGrid.h.
#include "CBCTSinMatPolyForwardProjGrid.h"

#include <iostream>
#include <stdexcept>

CBCTSinMatPolyForwardProjGrid::~CBCTSinMatPolyForwardProjGrid() = default;

// CBCTSinMatPolyForwardProjGrid.cpp:13-145: density projection once, then all
// energies; here one fused pass.
void CBCTSinMatPolyForwardProjGrid::computePolyForwProj()
{
    std::cout << "single-material forward projection with grid ====>>>>" << std::endl;
    runDeviceProjection(true, true, true);
    saveAll(true);
}

// CBCTSinMatPolyForwardProjGrid.cpp:147-267.
void CBCTSinMatPolyForwardProjGrid::computePolyForwProjNoResponse()
{
    std::cout << "single-material forward projection with grid, no detector response ====>>>>" << std::endl;
    runDeviceProjection(true, false, true);
    saveAll(false);
}

// CBCTSinMatPolyForwardProjGrid.cpp:269-388: the same outputs as
// computePolyForwProj, with per-view focal-spot offsets (computeFoSpOffset)
// shifting each view's sampling and re-aligning its projection.
void CBCTSinMatPolyForwardProjGrid::computePolyForwProjFoSp()
{
    std::cout << "single-material forward projection with grid, focal spot ====>>>>" << std::endl;
    computeFoSpOffset();
    focalSpot_ = true;
    try {
        runDeviceProjection(true, true, true);
    } catch (...) {
        focalSpot_ = false;
        throw;
    }
    focalSpot_ = false;
    saveAll(true);
}
