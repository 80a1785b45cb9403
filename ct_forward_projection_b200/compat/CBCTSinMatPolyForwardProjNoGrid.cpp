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

void CBCTSinMatPolyForwardProjNoGrid::computePolyForwProjFoSp()
{
    throw std::runtime_error("the focal-spot path is unreachable in the reference and not rebuilt");
}
