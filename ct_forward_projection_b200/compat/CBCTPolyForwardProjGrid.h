// CBCTPolyForwardProjGrid.h — multi-material projector with anti-scatter grid,
// the interface of the reference's Source/CBCTPolyForwardProjGrid.h:11-44.
#pragma once

#include <vector>

#include "CBCTForwardProj.h"
#include "Grid.h"

class CBCTPolyForwardProjGrid : public CBCTForwardProj {
public:
    CBCTPolyForwardProjGrid(CTScanParas inCTScanParas, GridInfo inGridInfo, FilePath inFileInfo,
                            const PhantomMaterial inPhantomMaterial);
    ~CBCTPolyForwardProjGrid();

    virtual void computePolyForwProj();
    virtual void testI0();
    virtual void initGridInfo();
    virtual void saveIandIAbsorb();
    virtual void addI0();
    virtual void addI0NoResponse();
    virtual void saveI0();
    virtual void readPhantom();
    virtual void showProcessInfo();
    virtual void showProcessInfoNoResponse();
    virtual void scatterSimulGrid();
    virtual void saveProj();

public:
    Grid* mGrid = nullptr;
    GridAndDetectorSystem mGridAndDetectorSystem;
    std::vector<size_t> gridPeriodIndex;

protected:
    const char* tag() const override { return "Grid"; }
    void saveAll(bool withResponseSample);
};
