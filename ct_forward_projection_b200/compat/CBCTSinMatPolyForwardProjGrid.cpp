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

void CBCTSinMatPolyForwardProjGrid::computePolyForwProjFoSp()
{
    throw std::runtime_error("the focal-spot path is unreachable in the reference and not rebuilt");
}
