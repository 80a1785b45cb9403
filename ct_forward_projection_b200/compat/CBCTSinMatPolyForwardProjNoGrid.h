// CBCTSinMatPolyForwardProjNoGrid.h — single-material projector without grid,
// the interface of the reference's Source/CBCTSinMatPolyForwardProjNoGrid.h:3-17.
#pragma once

#include "CBCTPolyForwardProjNoGrid.h"

class CBCTSinMatPolyForwardProjNoGrid : private CBCTPolyForwardProjNoGrid {
public:
    CBCTSinMatPolyForwardProjNoGrid(CTScanParas inCTScanParas, FilePath inFileInfo,
                                    const PhantomMaterial inPhantomMaterial)
        : CBCTPolyForwardProjNoGrid(inCTScanParas, inFileInfo, inPhantomMaterial)
    {
    }
    ~CBCTSinMatPolyForwardProjNoGrid();

    virtual void computePolyForwProj();
    void computePolyForwProjNoResponse();
    // Unreachable in the reference and not rebuilt; throws.
    void computePolyForwProjFoSp();

    using CBCTForwardProj::I;
    using CBCTForwardProj::IAbsorb;
    using CBCTForwardProj::IPolyenergetic;
    using CBCTForwardProj::IPolyenergeticAbsorb;
    using CBCTForwardProj::h_mForwardProj;
    using CBCTForwardProj::aDetResponse;
};
