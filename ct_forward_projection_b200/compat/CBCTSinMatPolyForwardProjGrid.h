// CBCTSinMatPolyForwardProjGrid.h — single-material projector with grid, the
// interface of the reference's Source/CBCTSinMatPolyForwardProjGrid.h:5-21
// (private inheritance, as there).
#pragma once

#include "CBCTPolyForwardProjGrid.h"

class CBCTSinMatPolyForwardProjGrid : private CBCTPolyForwardProjGrid {
public:
    CBCTSinMatPolyForwardProjGrid(CTScanParas inCTScanParas, GridInfo inGridInfo, FilePath inFileInfo,
                                  const PhantomMaterial inphantomMaterial)
        : CBCTPolyForwardProjGrid(inCTScanParas, inGridInfo, inFileInfo, inphantomMaterial)
    {
    }
    ~CBCTSinMatPolyForwardProjGrid();

    virtual void computePolyForwProj();
    void computePolyForwProjNoResponse();
    // The focal-spot path is unreachable in the reference
    // (ForwardProjection.cpp:20-84) and not rebuilt; throws.
    void computePolyForwProjFoSp();

    // Results, read-only access for callers of the private base.
    using CBCTForwardProj::I;
    using CBCTForwardProj::IAbsorb;
    using CBCTForwardProj::IPolyenergetic;
    using CBCTForwardProj::IPolyenergeticAbsorb;
    using CBCTForwardProj::h_mForwardProj;
    using CBCTForwardProj::aDetResponse;
};
