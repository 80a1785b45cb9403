// CBCTSinMatPolyForwardProjNoGrid.cpp — see CBCTSinMatPolyForwardProjNoGrid.h.
#include "CBCTSinMatPolyForwardProjNoGrid.h"

#include <iostream>
#include <stdexcept>

CBCTSinMatPolyForwardProjNoGrid::~CBCTSinMatPolyForwardProjNoGrid() = default;

// CBCTSinMatPolyForwardProjNoGrid.cpp:10-111.
void CBCTSinMatPolyForwardProjNoGrid::computePolyForwProj()
{
    std::cout << "single-material forward projection without grid ====>>>>" << std::endl;
    runDeviceProjection(false, true, true);
    saveAll(true);
}

// CBCTSinMatPolyForwardProjNoGrid.cpp:113-214.
void CBCTSinMatPolyForwardProjNoGrid::computePolyForwProjNoResponse()
{
    std::cout << "single-material forward projection without grid, no detector response ====>>>>" << std::endl;
    runDeviceProjection(false, false, true);
    saveAll(false);
}

// CBCTSinMatPolyForwardProjNoGrid.cpp:216-331: the same outputs as
// computePolyForwProj, with per-view focal-spot offsets (computeFoSpOffset)
// shifting each view's sampling and re-aligning its projection.
void CBCTSinMatPolyForwardProjNoGrid::computePolyForwProjFoSp()
{
    std::cout << "single-material forward projection without grid, focal spot ====>>>>" << std::endl;
    computeFoSpOffset();
    focalSpot_ = true;
    try {
        runDeviceProjection(false, true, true);
    } catch (...) {
        focalSpot_ = false;
        throw;
    }
    focalSpot_ = false;
    saveAll(true);
}
