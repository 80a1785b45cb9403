// CBCTPolyForwardProjGrid.cpp — see CBCTPolyForwardProjGrid.h.
#include "CBCTPolyForwardProjGrid.h"

#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>

CBCTPolyForwardProjGrid::CBCTPolyForwardProjGrid(CTScanParas p, GridInfo g, FilePath f, const PhantomMaterial m)
{
    mCTScanParas = p;
    mCTScanParas.spectrumStep = 1;  // CBCTPolyForwardProjGrid.cpp:40
    mGridInfo = g;
    mFilePath = f;
    _mPhantomMaterial = m;
}

CBCTPolyForwardProjGrid::~CBCTPolyForwardProjGrid() { DELETE(mGrid); }

void CBCTPolyForwardProjGrid::computePolyForwProj()
{
    std::cout << "forward projection with grid ====>>>>" << std::endl;
    runDeviceProjection(true, true, false);
    saveAll(false);
}

void CBCTPolyForwardProjGrid::saveAll(bool withResponseSample)
{
    creatOutputFolder();
    saveIandIAbsorb();
    saveI0();
    if (withResponseSample) saveADetResponse();
    saveProj();
}

void CBCTPolyForwardProjGrid::testI0()
{
    runFlatField(true, true);
    creatOutputFolder();
    saveI0();
}

// GridInfo -> GridAndDetectorSystem (CBCTPolyForwardProjGrid.cpp:287-308).
void CBCTPolyForwardProjGrid::initGridInfo()
{
    mGridAndDetectorSystem.angleNums = mCTScanParas.projNum;
    mGridAndDetectorSystem.dNums = mCTScanParas.dNumU;
    mGridAndDetectorSystem.dSize = mCTScanParas.dSize * 1000;
    mGridAndDetectorSystem.FD = mGridInfo.FD;
    mGridAndDetectorSystem.h = mGridInfo.h;
    mGridAndDetectorSystem.gridStripsWidth = mGridInfo.gridStripsWidth;
    mGridAndDetectorSystem.interspcaceWidth = mGridInfo.interspcaceWidth;
    mGridAndDetectorSystem.gridStripMaterial = mGridInfo.gridStripMaterial;
    mGridAndDetectorSystem.interspaceMaterial = mGridInfo.interspaceMaterial;
    mGridAndDetectorSystem.gridStripDensity = mGridInfo.gridStripDensity;
    mGridAndDetectorSystem.interspaceDensity = mGridInfo.interspaceDensity;
    mGridAndDetectorSystem.gridStripMAPath = mGridInfo.gridStripMAPath;
    mGridAndDetectorSystem.interspaceMAPath = mGridInfo.interspaceMAPath;
    mGridAndDetectorSystem.mI0Photons = mCTScanParas.I0Val;
    mGridAndDetectorSystem.gridStripLinearAtten = mGridInfo.gridStripLinearAtten;
    mGridAndDetectorSystem.interspaceLinearAtten = mGridInfo.interspaceLinearAtten;
}

void CBCTPolyForwardProjGrid::saveIandIAbsorb()
{
    const std::string dims = std::to_string(mCTScanParas.dNumU) + "x" + std::to_string(mCTScanParas.dNumV) + "x" +
                             std::to_string(mCTScanParas.projNum);
    writeRaw(std::string("PhoImgPro_") + tag() + "_" + dims + "_uint32.raw", IPolyenergetic, nRays() * sizeof(uint32));
    writeRaw(std::string("PhoImgAbsorb_") + tag() + "_" + dims + "_uint32.raw", IPolyenergeticAbsorb,
             nRays() * sizeof(uint32));
}

// One energy's flat field, FP32 (CBCTPolyForwardProjGrid.cpp:330-339).
void CBCTPolyForwardProjGrid::addI0()
{
    for (size_t i = 0; i < mCTScanParas.dNumV; i++)
        for (size_t j = 0; j < mCTScanParas.dNumU; j++)
            h_mForwardProj.I0[i * mCTScanParas.dNumU + j] += (float)mCTScanParas.I0Val * mCTScanSystemInfo.spectrumVal *
                                                             h_mForwardProj.grid[j] *
                                                             h_mForwardProj.detResponse[i * mCTScanParas.dNumU + j];
}

void CBCTPolyForwardProjGrid::addI0NoResponse()
{
    for (size_t i = 0; i < mCTScanParas.dNumV; i++)
        for (size_t j = 0; j < mCTScanParas.dNumU; j++)
            h_mForwardProj.I0[i * mCTScanParas.dNumU + j] +=
                (float)mCTScanParas.I0Val * mCTScanSystemInfo.spectrumVal * h_mForwardProj.grid[j];
}

void CBCTPolyForwardProjGrid::saveI0()
{
    writeRaw(std::string("BgImgPro_") + tag() + "_" + std::to_string(mCTScanParas.dNumU) + "x" +
                 std::to_string(mCTScanParas.dNumV) + "_float.raw",
             h_mForwardProj.I0, nPix() * sizeof(float));
}

// Per-energy linear-attenuation volumes of an earlier input format
// (CBCTPolyForwardProjGrid.cpp:365-382): <phantomPath>_<E>keV.raw.
void CBCTPolyForwardProjGrid::readPhantom()
{
    const size_t n = mCTScanParas.pNumX * mCTScanParas.pNumY * mCTScanParas.pNumZ;
    const std::string path = mFilePath.phantomPath + "_" + std::to_string((specIndex + 1) * mCTScanParas.spectrumStep) +
                             "keV.raw";
    std::ifstream ifs(path, std::ios::in | std::ios::binary);
    if (!ifs) throw std::runtime_error("cannot open " + path);
    if (!h_mForwardProj.phantom) h_mForwardProj.phantom = new float[n];
    ifs.read(reinterpret_cast<char*>(h_mForwardProj.phantom), (std::streamsize)(n * sizeof(float)));
}

void CBCTPolyForwardProjGrid::showProcessInfo()
{
    std::cout << (specIndex + 1) * mCTScanParas.spectrumStep << " keV" << std::endl;
}

void CBCTPolyForwardProjGrid::showProcessInfoNoResponse() { showProcessInfo(); }

void CBCTPolyForwardProjGrid::scatterSimulGrid() {}

void CBCTPolyForwardProjGrid::saveProj()
{
    writeRaw(std::string("Projection_") + tag() + "_" + std::to_string(mCTScanParas.dNumU) + "x" +
                 std::to_string(mCTScanParas.dNumV) + "x" + std::to_string(mCTScanParas.projNum) + "_float.raw",
             h_mForwardProj.proj, nRays() * sizeof(float));
}
