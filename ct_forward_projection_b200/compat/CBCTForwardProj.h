// CBCTForwardProj.h — base of the drop-in projector classes, with the public
// interface of the reference's Source/CBCTForwardProj.h:10-100 (virtual
// hooks, public data members holding the results after computePolyForwProj).
//
// Where the reference loops energies on the host and launches two kernels per
// view and energy (CBCTPolyForwardProjGrid.cpp:159-177), these classes build
// all energies' tables on the device and run one ctfp_forward for all views
// and energies (include/ctfp.h), then floor to uint32 and form proj on the
// device.  Errors throw std::runtime_error; the reference printed a message
// and called exit() (e.g. CBCTForwardProj.cpp:155-160), which only the CLI
// (ForwardProjection::run's caller) does here.
//
// The sampler follows the environment variable CTFP_INTERP: "texture"
// (default: the reference's hardware tex3D), "texemu" (its exact software
// emulation) or "trilinear" (exact FP32 trilinear at FP64 coordinates).
// CTFP_SKIP_EMPTY=1 turns on empty-space skipping (ctfp_plan_set_skip_empty).
#pragma once

#include <filesystem>
#include <string>
#include <vector>

#include "DataType.h"
#include "PhantomObject.h"

class CBCTForwardProj {
public:
    CBCTForwardProj();
    virtual ~CBCTForwardProj() = 0;

    virtual void computePolyForwProj() = 0;

    virtual void computeParas();
    virtual void initGridInfo() = 0;

    virtual void addIandIAbsorb();
    virtual void convertIandIAbsorbDt();
    virtual void saveIandIAbsorb() = 0;

    virtual void testI0() = 0;
    virtual void addStandardI0(float& I0Standard);

    virtual void addI0() = 0;
    virtual void saveI0() = 0;

    virtual void computePerScinThinckness();
    virtual void updateDetResponse();

    virtual void computeFoSpOffset();

    virtual void readSpecrtumNorm();
    virtual void readGridMassAttu();
    virtual void readScintillatorMassAttu();
    virtual void getADetResponse();
    virtual void saveADetResponse();

    virtual void readPhantom() = 0;

    virtual void showScanSystemInfo();
    virtual void showGridmInfo();
    virtual void showProcessInfo() = 0;

    virtual void computeProj();
    virtual void saveProj() = 0;

    virtual void creatOutputFolder();
    virtual void _removeOutputFolder();

    virtual void scatterSimulGrid() = 0;

public:
    PhantomObject* mPhantomObject = nullptr;

    CTScanSystemInfo mCTScanSystemInfo;
    CTScanParas mCTScanParas;
    Coordinate d_mCoordinate;
    PolyForwardProj h_mForwardProj;
    PolyForwardProj d_mForwardProj;
    FilePath mFilePath;

    PhantomMaterial _mPhantomMaterial;

    GridInfo mGridInfo;

    size_t specIndex = 0;

    float* I = nullptr;                       // [P][V][U] sum over energies
    uint32* IPolyenergetic = nullptr;         // floor(I)
    float* IAbsorb = nullptr;
    uint32* IPolyenergeticAbsorb = nullptr;
    float* IEScatter = nullptr;
    float* aDetResponse = nullptr;            // detResponse at flat index (U+V)/2 per energy

protected:
    // The whole simulation through the C ABI: tables for every energy, one
    // fused forward, device floor/log; fills I, IAbsorb, IPolyenergetic,
    // IPolyenergeticAbsorb, h_mForwardProj.I0 and h_mForwardProj.proj.
    void runDeviceProjection(bool grid, bool response, bool singleMaterial);
    // Flat-field only (TestI0 mode): h_mForwardProj.I0.
    void runFlatField(bool grid, bool response);
    // Output file tag, "Grid" or "NoGrid".
    virtual const char* tag() const = 0;
    void writeRaw(const std::string& name, const void* data, size_t bytes) const;
    size_t nRays() const { return mCTScanParas.dNumU * mCTScanParas.dNumV * mCTScanParas.projNum; }
    size_t nPix() const { return mCTScanParas.dNumU * mCTScanParas.dNumV; }
    void freeResults();

    bool focalSpot_ = false;         // runDeviceProjection applies h_mForwardProj.foSpOffset{U,V}
    std::vector<float> gridTable_;   // [E][U] grid transmission
    std::vector<float> detTable_;    // [E][V][U] detector response
};
