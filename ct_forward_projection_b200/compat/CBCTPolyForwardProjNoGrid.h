// CBCTPolyForwardProjNoGrid.h — multi-material projector without grid, the
// interface of the reference's Source/CBCTPolyForwardProjNoGrid.h:9-36.
#pragma once

#include "CBCTPolyForwardProjGrid.h"

class CBCTPolyForwardProjNoGrid : public CBCTPolyForwardProjGrid {
public:
    CBCTPolyForwardProjNoGrid(CTScanParas inCTScanParas, FilePath inFileInfo, const PhantomMaterial inPhantomMaterial);
    ~CBCTPolyForwardProjNoGrid();

    virtual void computePolyForwProj();
    virtual void testI0();
    virtual void initGridInfo();
    virtual void addI0();
    virtual void addI0NoResponse();

protected:
    const char* tag() const override { return "NoGrid"; }
};
