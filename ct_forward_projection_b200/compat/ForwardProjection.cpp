// ForwardProjection.cpp — see ForwardProjection.h.  Keys, sections and the
// missing-entry sentinels follow the reference's parser
// (ForwardProjection.cpp:197-419); paths in the INI are relative to baseDir.
#include "ForwardProjection.h"

#include <filesystem>
#include <stdexcept>

namespace {
void require(bool ok, const char* what)
{
    if (!ok) throw std::runtime_error(what);
}
}  // namespace

ForwardProjection::~ForwardProjection()
{
    DELETEARR(_mPhantomMaterial.density);
    DELETEARR(_mPhantomMaterial.massAttenPath);
}

void ForwardProjection::run()
{
    _getCTScanConfig();
    _getOutputFolderConfig();
    if (_isTestI0) {
        forwarProjNoGridTestI0();
        return;
    }
    if (_isDetResponse) {
        if (_isGrid) {
            if (_isSingleMaterial) forwardSinMatPolyProjGrid();
            else forwardPolyProjGrid();
        } else {
            if (_isSingleMaterial) forwardSinMatPolyProjNoGrid();
            else forwardPolyProjNoGrid();
        }
    } else {
        require(_isSingleMaterial != 0,
                "IsDetResponse=0 with IsSingleMaterial=0 has no projector (the reference does nothing for it)");
        if (_isGrid) forwardSinMatPolyProjGridNoResponse();
        else forwardSinMatPolyProjNoGridNoResponse();
    }
}

void ForwardProjection::forwardPolyProjGrid()
{
    _getCTScanGridConfig();
    _getCTScanDetResponseConfig();
    CBCTPolyForwardProjGrid p(mCTScanParas, mGridInfo, mFilePath, _mPhantomMaterial);
    p.computePolyForwProj();
}

void ForwardProjection::forwardSinMatPolyProjGrid()
{
    _getCTScanGridConfig();
    _getCTScanDetResponseConfig();
    CBCTSinMatPolyForwardProjGrid p(mCTScanParas, mGridInfo, mFilePath, _mPhantomMaterial);
    p.computePolyForwProj();
}

void ForwardProjection::forwardSinMatPolyProjGridNoResponse()
{
    _getCTScanGridConfig();
    CBCTSinMatPolyForwardProjGrid p(mCTScanParas, mGridInfo, mFilePath, _mPhantomMaterial);
    p.computePolyForwProjNoResponse();
}

void ForwardProjection::forwardPolyProjNoGrid()
{
    _getCTScanDetResponseConfig();
    CBCTPolyForwardProjNoGrid p(mCTScanParas, mFilePath, _mPhantomMaterial);
    p.computePolyForwProj();
}

void ForwardProjection::forwardSinMatPolyProjNoGrid()
{
    _getCTScanDetResponseConfig();
    CBCTSinMatPolyForwardProjNoGrid p(mCTScanParas, mFilePath, _mPhantomMaterial);
    p.computePolyForwProj();
}

void ForwardProjection::forwardSinMatPolyProjNoGridNoResponse()
{
    CBCTSinMatPolyForwardProjNoGrid p(mCTScanParas, mFilePath, _mPhantomMaterial);
    p.computePolyForwProjNoResponse();
}

void ForwardProjection::forwarProjNoGridTestI0()
{
    _getCTScanDetResponseConfig();
    CBCTPolyForwardProjNoGrid p(mCTScanParas, mFilePath, _mPhantomMaterial);
    p.testI0();
}

void ForwardProjection::_getCTScanConfig()
{
    mCInitFile.GetFileName((baseDir + "/Config/ScanSetting.ini").c_str());
    const char* s = "ScanPara";
    mCInitFile.GetEntryValue(s, "IsTestI0", -100, _isTestI0);
    mCInitFile.GetEntryValue(s, "IsDetResponse", -100, _isDetResponse);
    mCInitFile.GetEntryValue(s, "IsGrid", -100, _isGrid);
    mCInitFile.GetEntryValue(s, "IsSingleMaterial", -100, _isSingleMaterial);
    mCInitFile.GetEntryValue(s, "SDD", -100.0f, mCTScanParas.sdd);
    mCInitFile.GetEntryValue(s, "SOD", -100.0f, mCTScanParas.sod);
    const bool views = mCInitFile.GetEntryValue(s, "ScanAngleNum", (size_t)0, mCTScanParas.projNum);
    mCInitFile.GetEntryValue(s, "RotatedDirection", -100, mCTScanParas.rotatedDirection);
    require(_isTestI0 != -100 && _isDetResponse != -100 && _isGrid != -100 && _isSingleMaterial != -100 &&
                mCTScanParas.sdd >= 0 && mCTScanParas.sod >= 0 && views && mCTScanParas.rotatedDirection != -100,
            "bad [ScanPara] entries in ScanSetting.ini");

    s = "RaySource";
    const bool photons = mCInitFile.GetEntryValue(s, "Photons", (size_t)0, mCTScanParas.I0Val);
    mCInitFile.GetEntryValue(s, "SpecEnergyNum", -100, mCTScanParas.specEnergyNum);
    mCInitFile.GetEntryValue(s, "SpectrumPath", "null", mFilePath.spectrumPath);
    require(photons && mCTScanParas.specEnergyNum > 0 && mFilePath.spectrumPath != "null",
            "bad [RaySource] entries in ScanSetting.ini");
    mFilePath.spectrumPath = baseDir + "/" + mFilePath.spectrumPath;

    s = "PhantomVox";
    bool ok = mCInitFile.GetEntryValue(s, "PNumX", (size_t)0, mCTScanParas.pNumX);
    ok &= (bool)mCInitFile.GetEntryValue(s, "PNumY", (size_t)0, mCTScanParas.pNumY);
    ok &= (bool)mCInitFile.GetEntryValue(s, "PNumZ", (size_t)0, mCTScanParas.pNumZ);
    require(ok, "bad phantom voxel counts in ScanSetting.ini");
    mCInitFile.GetEntryValue(s, "PLengthX", -100.0f, mCTScanParas.pLengthX);
    mCInitFile.GetEntryValue(s, "PLengthY", -100.0f, mCTScanParas.pLengthY);
    mCInitFile.GetEntryValue(s, "PLengthZ", -100.0f, mCTScanParas.pLengthZ);
    require(mCTScanParas.pLengthX >= 0 && mCTScanParas.pLengthY >= 0 && mCTScanParas.pLengthZ >= 0,
            "bad phantom size in ScanSetting.ini");

    s = "Detector";
    ok = mCInitFile.GetEntryValue(s, "DNumU", (size_t)0, mCTScanParas.dNumU);
    ok &= (bool)mCInitFile.GetEntryValue(s, "DNumV", (size_t)0, mCTScanParas.dNumV);
    mCInitFile.GetEntryValue(s, "DSize", -100.0f, mCTScanParas.dSize);
    require(ok && mCTScanParas.dSize >= 0, "bad [Detector] entries in ScanSetting.ini");

    s = "PhantomMaterial";
    mCInitFile.GetEntryValue(s, "MaterialNum", -100, _mPhantomMaterial.materialNum);
    mCInitFile.GetEntryValue(s, "StructureMarkPath", "null", _mPhantomMaterial.structureMarkPath);
    require(_mPhantomMaterial.materialNum > 0 && _mPhantomMaterial.structureMarkPath != "null",
            "bad [PhantomMaterial] entries in ScanSetting.ini");
    _mPhantomMaterial.structureMarkPath = baseDir + "/" + _mPhantomMaterial.structureMarkPath;
    DELETEARR(_mPhantomMaterial.density);
    DELETEARR(_mPhantomMaterial.massAttenPath);
    _mPhantomMaterial.density = new float[(size_t)_mPhantomMaterial.materialNum];
    _mPhantomMaterial.massAttenPath = new std::string[(size_t)_mPhantomMaterial.materialNum];
    for (int i = 0; i < _mPhantomMaterial.materialNum; i++) {
        const std::string dk = "Density" + std::to_string(i + 1), mk = "MassAttenPath" + std::to_string(i + 1);
        mCInitFile.GetEntryValue(s, dk.c_str(), -100.0f, _mPhantomMaterial.density[i]);
        mCInitFile.GetEntryValue(s, mk.c_str(), "null", _mPhantomMaterial.massAttenPath[i]);
        require(_mPhantomMaterial.density[i] >= 0 && _mPhantomMaterial.massAttenPath[i] != "null",
                "bad material density or attenuation path in ScanSetting.ini");
        _mPhantomMaterial.massAttenPath[i] = baseDir + "/" + _mPhantomMaterial.massAttenPath[i];
    }
}

void ForwardProjection::_getCTScanGridConfig()
{
    const char* s = "PostGrid";
    mCInitFile.GetEntryValue(s, "FD", -100.0f, mGridInfo.FD);
    mCInitFile.GetEntryValue(s, "Height", -100.0f, mGridInfo.h);
    mCInitFile.GetEntryValue(s, "GridStripsWidth", -100, mGridInfo.gridStripsWidth);
    mCInitFile.GetEntryValue(s, "InterspcaceWidth", -100, mGridInfo.interspcaceWidth);
    mCInitFile.GetEntryValue(s, "GridStripMaterial", "null", mGridInfo.gridStripMaterial);
    mCInitFile.GetEntryValue(s, "InterspaceMaterial", "null", mGridInfo.interspaceMaterial);
    mCInitFile.GetEntryValue(s, "GridStripDensity", -100.0f, mGridInfo.gridStripDensity);
    mCInitFile.GetEntryValue(s, "InterspaceDensity", -100.0f, mGridInfo.interspaceDensity);
    mCInitFile.GetEntryValue(s, "GridStripMAPath", "null", mGridInfo.gridStripMAPath);
    mCInitFile.GetEntryValue(s, "InterspaceMAPath", "null", mGridInfo.interspaceMAPath);
    require(mGridInfo.FD >= 0 && mGridInfo.h >= 0 && mGridInfo.gridStripsWidth >= 0 &&
                mGridInfo.interspcaceWidth >= 0 && mGridInfo.interspaceMaterial != "null" &&
                mGridInfo.gridStripMaterial != "null" && mGridInfo.gridStripDensity >= 0 &&
                mGridInfo.interspaceDensity >= 0 && mGridInfo.gridStripMAPath != "null" &&
                mGridInfo.interspaceMAPath != "null",
            "bad [PostGrid] entries in ScanSetting.ini");
    mGridInfo.gridStripMAPath = baseDir + "/" + mGridInfo.gridStripMAPath;
    mGridInfo.interspaceMAPath = baseDir + "/" + mGridInfo.interspaceMAPath;
}

void ForwardProjection::_getCTScanDetResponseConfig()
{
    const char* s = "Scintillator";
    ScintilltorInfo& sc = mCTScanParas.mScintilltorInfo;
    mCInitFile.GetEntryValue(s, "Density", -100.0f, sc.scintillatorDensity);
    mCInitFile.GetEntryValue(s, "Thickness", -100.0f, sc.scintillatorThickness);
    mCInitFile.GetEntryValue(s, "ThicknessErr", -100.0f, sc.scintillatorThicknessErr);
    mCInitFile.GetEntryValue(s, "PhotoelectConverFactor", -100.0f, sc.detResponseFactor);
    mCInitFile.GetEntryValue(s, "ScintillatorMAPath", "null", mFilePath.scintillatorPath);
    require(sc.scintillatorDensity >= 0 && sc.scintillatorThickness >= 0 && sc.scintillatorThicknessErr >= 0 &&
                sc.detResponseFactor >= 0 && sc.detResponseFactor <= 1 && mFilePath.scintillatorPath != "null",
            "bad [Scintillator] entries in ScanSetting.ini");
    mFilePath.scintillatorPath = baseDir + "/" + mFilePath.scintillatorPath;
}

// The reference opens Config/OutputFolder.ini while it ships
// Config/OutPutFolder.ini (ForwardProjection.cpp:376); both names are tried.
void ForwardProjection::_getOutputFolderConfig()
{
    CInitFile f;
    const std::string a = baseDir + "/Config/OutputFolder.ini", b = baseDir + "/Config/OutPutFolder.ini";
    f.GetFileName(std::filesystem::exists(a) ? a.c_str() : b.c_str());
    const char* section = _isTestI0 ? "NoGridResponseTestI0"
                          : _isGrid ? (_isDetResponse ? "GridResponse" : "GridNoResponse")
                                    : (_isDetResponse ? "NoGridResponse" : "NoGridNoResponse");
    f.GetEntryValue(section, "OutFolder", "null", mFilePath.outputFolder);
    require(mFilePath.outputFolder != "null", "missing OutFolder in OutPutFolder.ini");
    mFilePath.outputFolder = baseDir + "/" + mFilePath.outputFolder;
}
