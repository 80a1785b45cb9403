// DataType.h — the parameter and buffer structs of the projector's C++ API,
// with the fields, names and units of the reference's Source/DataType.h:19-180
// so that code written against the reference's classes compiles unchanged.
#pragma once

#include <cstddef>
#include <string>

#define DELETEARR(arrP)      \
    if (arrP != nullptr) {   \
        delete[] arrP;       \
        arrP = nullptr;      \
    }

#define DELETE(var)          \
    if (var != nullptr) {    \
        delete var;          \
        var = nullptr;       \
    }

typedef unsigned char uint8;
typedef unsigned int uint32;

// Scintillator (DataType.h:23-30).
struct ScintilltorInfo {
    std::string scintillatorName;
    float scintillatorDensity = 0;        // g/cm^3
    float scintillatorThickness = 0;      // mm
    float scintillatorThicknessErr = 0;   // mm
    float detResponseFactor = 0;          // photoelectric conversion factor
};

// Scan parameters (DataType.h:33-55).
struct CTScanParas {
    size_t pNumX = 0, pNumY = 0, pNumZ = 0;       // phantom voxels
    float pLengthX = 0, pLengthY = 0, pLengthZ = 0;  // mm
    size_t projNum = 0;                            // views
    size_t dNumU = 0, dNumV = 0;                   // detector columns, rows
    float sod = 0, sdd = 0;                        // mm
    int rotatedDirection = 1;
    float dSize = 0;                               // detector pitch, mm
    size_t I0Val = 0;                              // photons before weighting
    float focalSpotSize = 0;                       // mm
    int spectrumStep = 1;
    int specEnergyNum = 0;                         // energy bins, e <-> (e+1) keV
    ScintilltorInfo mScintilltorInfo;
};

// Focused anti-scatter grid (DataType.h:57-75).
struct GridInfo {
    int interspcaceWidth = 0;   // um
    int gridStripsWidth = 0;    // um
    float h = 0;                // mm
    float FD = 0;               // mm
    std::string gridStripMaterial;
    float gridStripDensity = 0;
    std::string gridStripMAPath;
    std::string interspaceMaterial;
    float interspaceDensity = 0;
    std::string interspaceMAPath;
    float gridStripLinearAtten = 0;     // 1/mm
    float interspaceLinearAtten = 0;    // 1/mm
};

// Derived quantities (DataType.h:78-111), filled by computeParas.
struct CTScanSystemInfo {
    float totalTime = 0.0f;
    int rotatedDirection = 1;
    float thetaStep = 0, dHalfLU = 0, dHalfLV = 0, FOVR = 0, FOVH = 0;
    float pHalfX = 0, pHalfY = 0, pHalfZ = 0;
    float pSizeX = 0, pSizeY = 0, pSizeZ = 0;
    float dx = 0, dy = 0, dz = 0;
    size_t intNum = 0;
    float spectrumVal = 0;
    float phantomMAtten = 0;
};

// Sample coordinates of the reference's GPU layer (DataType.h:120-125).  The
// ctfp kernels compute coordinates per sample and keep none; the struct is
// kept for source compatibility.
struct Coordinate {
    float *imgIntX = nullptr, *imgIntY = nullptr, *imgIntZ = nullptr;
};

// Host buffers of one simulation (DataType.h:128-146).
struct PolyForwardProj {
    uint8* phantomStructure = nullptr;
    float* phantom = nullptr;              // density (single material) or per-energy mu (reference)
    float* phantomMassAtten = nullptr;
    float* spectrumNormal = nullptr;
    float* grid = nullptr;                 // [dNumU] grid transmission of the current energy
    float* gridLinearAtten = nullptr;      // [E] 1/mm
    float* interspaceLinearAtten = nullptr;
    float *I = nullptr, *I0 = nullptr, *IAbsorb = nullptr;
    float* proj = nullptr;
    float* scintillatorLineAtten = nullptr;     // [E] 1/mm
    float* scintillatorPerThickness = nullptr;  // [V*U] mm
    float* detResponse = nullptr;               // [V*U] current energy
    float *foSpOffsetU = nullptr, *foSpOffsetV = nullptr;
};
typedef PolyForwardProj ForwardProj;

// Paths (DataType.h:149-158).
struct FilePath {
    std::string spectrumPath;
    std::string gridPath;
    std::string phantomPath;
    std::string phantomMAttenPath;
    std::string outputFolder;
    std::string scintillatorPath;
    std::string convKernelGridPath;
};

// Materials of a label phantom (DataType.h:161-168).
struct PhantomMaterial {
    int materialNum = 0;
    std::string structureMarkPath;
    float* density = nullptr;
    std::string* massAttenPath = nullptr;
};

enum ScanMode { TestI0, GridNoResponse, GridResponse, NoGridNoResponse, NoGridResponse };
