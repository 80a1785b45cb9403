// ForwardProjection.h — reads Config/ScanSetting.ini and Config/OutPutFolder.ini
// and runs the selected projector, the interface of the reference's
// Source/ForwardProjection.h:11-65.
#pragma once

#include <string>

#include "CBCTPolyForwardProjGrid.h"
#include "CBCTPolyForwardProjNoGrid.h"
#include "CBCTSinMatPolyForwardProjGrid.h"
#include "CBCTSinMatPolyForwardProjNoGrid.h"
#include "DataType.h"
#include "InitFile.h"

class ForwardProjection {
public:
    ForwardProjection() = default;
    ~ForwardProjection();

    // ForwardProjection::run (ForwardProjection.cpp:20-84): the IsTestI0 /
    // IsDetResponse / IsGrid / IsSingleMaterial dispatch.  Throws
    // std::runtime_error on a bad or missing configuration entry or file, and
    // for the multi-material no-response combinations, which the reference
    // silently skips (ForwardProjection.cpp:61-64, 72-75).
    void run();

    // Directory holding Config/ (default: the working directory).
    std::string baseDir = ".";

private:
    void forwardPolyProjGrid();
    void forwardSinMatPolyProjGrid();
    void forwardSinMatPolyProjGridNoResponse();
    void forwardPolyProjNoGrid();
    void forwardSinMatPolyProjNoGrid();
    void forwardSinMatPolyProjNoGridNoResponse();
    void forwarProjNoGridTestI0();

    void _getCTScanConfig();
    void _getCTScanGridConfig();
    void _getCTScanDetResponseConfig();
    void _getOutputFolderConfig();

    CTScanParas mCTScanParas;
    GridInfo mGridInfo;
    FilePath mFilePath;
    CInitFile mCInitFile;
    int _isTestI0 = 0;
    int _isDetResponse = 0;
    int _isGrid = 0;
    int _isSingleMaterial = 0;
    PhantomMaterial _mPhantomMaterial;
};
