// CBCTPolyForwardProjNoGrid.cpp — see CBCTPolyForwardProjNoGrid.h.
#include "CBCTPolyForwardProjNoGrid.h"

#include <iostream>

CBCTPolyForwardProjNoGrid::CBCTPolyForwardProjNoGrid(CTScanParas p, FilePath f, const PhantomMaterial m)
    : CBCTPolyForwardProjGrid(p, GridInfo(), f, m)
{
}

CBCTPolyForwardProjNoGrid::~CBCTPolyForwardProjNoGrid() = default;

void CBCTPolyForwardProjNoGrid::computePolyForwProj()
{
    std::cout << "forward projection without grid ====>>>>" << std::endl;
    runDeviceProjection(false, true, false);
    saveAll(false);
}

// I0 only (CBCTPolyForwardProjNoGrid.cpp:188-264).
void CBCTPolyForwardProjNoGrid::testI0()
{
    runFlatField(false, true);
    creatOutputFolder();
    saveI0();
}

void CBCTPolyForwardProjNoGrid::initGridInfo() {}

// One energy's flat field without grid (CBCTPolyForwardProjNoGrid.cpp:290-299).
void CBCTPolyForwardProjNoGrid::addI0()
{
    for (size_t k = 0; k < nPix(); k++)
        h_mForwardProj.I0[k] += (float)mCTScanParas.I0Val * mCTScanSystemInfo.spectrumVal * h_mForwardProj.detResponse[k];
}

void CBCTPolyForwardProjNoGrid::addI0NoResponse()
{
    for (size_t k = 0; k < nPix(); k++) h_mForwardProj.I0[k] += (float)mCTScanParas.I0Val * mCTScanSystemInfo.spectrumVal;
}
