// CBCTForwardProj.cpp — see CBCTForwardProj.h.
#include "CBCTForwardProj.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <stdexcept>

#include "ctfp.h"

namespace {

#define CTFP_CHECK(call)                                                                           \
    do {                                                                                           \
        ctfp_status st_ = (call);                                                                  \
        if (st_ != CTFP_OK) throw std::runtime_error(std::string(#call) + ": " + ctfp_last_error_string()); \
    } while (0)

#define CUDA_CHECK(call)                                                                           \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Device buffers of one run, freed on scope exit.
struct DeviceBuffers {
    std::vector<void*> ptrs;
    template <typename T>
    T* alloc(size_t n)
    {
        void* p = nullptr;
        CUDA_CHECK(cudaMalloc(&p, n * sizeof(T) + 16));
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
    ~DeviceBuffers()
    {
        for (void* p : ptrs) cudaFree(p);
    }
};

struct PlanGuard {
    ctfp_plan* p = nullptr;
    ~PlanGuard() { ctfp_plan_destroy(p); }
};

int interp_from_env()
{
    const char* e = std::getenv("CTFP_INTERP");
    if (!e || !*e || std::strcmp(e, "texture") == 0) return CTFP_INTERP_TEXTURE;
    if (std::strcmp(e, "texemu") == 0) return CTFP_INTERP_TEXEMU;
    if (std::strcmp(e, "trilinear") == 0) return CTFP_INTERP_TRILINEAR;
    throw std::runtime_error(std::string("CTFP_INTERP must be texture, texemu or trilinear, not ") + e);
}

// Reads the first n values of a one-column table (one value per line).
std::vector<float> read_table(const std::string& path, int n, const char* what)
{
    std::ifstream ifs(path);
    if (!ifs) throw std::runtime_error(std::string("cannot open ") + what + " " + path);
    std::vector<float> v((size_t)n, 0.0f);
    int i = 0;
    float buf;
    while (i < n && ifs >> buf) v[(size_t)i++] = buf;
    if (i < n) throw std::runtime_error(std::string(what) + " " + path + " has fewer than SpecEnergyNum rows");
    return v;
}

// MSVC CRT rand() (the reference was built with it): state * 214013 + 2531011.

}  // namespace

CBCTForwardProj::CBCTForwardProj() = default;
CBCTForwardProj::~CBCTForwardProj() { freeResults(); }

void CBCTForwardProj::freeResults()
{
    DELETEARR(h_mForwardProj.grid);
    DELETEARR(h_mForwardProj.I);
    DELETEARR(h_mForwardProj.I0);
    DELETEARR(h_mForwardProj.phantom);
    DELETEARR(h_mForwardProj.phantomMassAtten);
    DELETEARR(h_mForwardProj.spectrumNormal);
    DELETEARR(h_mForwardProj.IAbsorb);
    DELETEARR(h_mForwardProj.detResponse);
    DELETEARR(h_mForwardProj.gridLinearAtten);
    DELETEARR(h_mForwardProj.interspaceLinearAtten);
    DELETEARR(h_mForwardProj.scintillatorLineAtten);
    DELETEARR(h_mForwardProj.scintillatorPerThickness);
    DELETEARR(h_mForwardProj.proj);
    DELETEARR(h_mForwardProj.foSpOffsetU);
    DELETEARR(h_mForwardProj.foSpOffsetV);
    DELETEARR(I);
    DELETEARR(IPolyenergetic);
    DELETEARR(IAbsorb);
    DELETEARR(IPolyenergeticAbsorb);
    DELETEARR(IEScatter);
    DELETEARR(aDetResponse);
    DELETE(mPhantomObject);
}

// CBCTForwardProj::computeParas (CBCTForwardProj.cpp:23-62) through ctfp_compute_paras.
void CBCTForwardProj::computeParas()
{
    ctfp_geometry g{};
    g.pNumX = (int64_t)mCTScanParas.pNumX; g.pNumY = (int64_t)mCTScanParas.pNumY; g.pNumZ = (int64_t)mCTScanParas.pNumZ;
    g.pLengthX = mCTScanParas.pLengthX; g.pLengthY = mCTScanParas.pLengthY; g.pLengthZ = mCTScanParas.pLengthZ;
    g.projNum = (int64_t)mCTScanParas.projNum;
    g.dNumU = (int64_t)mCTScanParas.dNumU; g.dNumV = (int64_t)mCTScanParas.dNumV;
    g.dSize = mCTScanParas.dSize; g.sod = mCTScanParas.sod; g.sdd = mCTScanParas.sdd;
    g.rotatedDirection = mCTScanParas.rotatedDirection;
    ctfp_system_info s{};
    CTFP_CHECK(ctfp_compute_paras(&g, &s));
    CTScanSystemInfo& o = mCTScanSystemInfo;
    o.rotatedDirection = mCTScanParas.rotatedDirection;
    o.thetaStep = s.thetaStep; o.dHalfLU = s.dHalfLU; o.dHalfLV = s.dHalfLV; o.FOVR = s.FOVR; o.FOVH = s.FOVH;
    o.pHalfX = s.pHalfX; o.pHalfY = s.pHalfY; o.pHalfZ = s.pHalfZ;
    o.pSizeX = s.pSizeX; o.pSizeY = s.pSizeY; o.pSizeZ = s.pSizeZ;
    o.dx = s.dx; o.dy = s.dy; o.dz = s.dz;
    o.intNum = (size_t)s.intNum;
}

// Host energy sums of per-energy results (CBCTForwardProj.cpp:65-76), for
// callers that accumulate h_mForwardProj.I / IAbsorb themselves.
void CBCTForwardProj::addIandIAbsorb()
{
    if (!I || !IAbsorb || !h_mForwardProj.I || !h_mForwardProj.IAbsorb) return;
    for (size_t i = 0; i < nRays(); i++) I[i] += h_mForwardProj.I[i];
    for (size_t i = 0; i < nRays(); i++) IAbsorb[i] += h_mForwardProj.IAbsorb[i];
}

// floor to uint32 (CBCTForwardProj.cpp:79-90).
void CBCTForwardProj::convertIandIAbsorbDt()
{
    if (!IPolyenergetic) IPolyenergetic = new uint32[nRays()];
    if (!IPolyenergeticAbsorb) IPolyenergeticAbsorb = new uint32[nRays()];
    for (size_t i = 0; i < nRays(); i++) IPolyenergetic[i] = (uint32)floorf(I[i]);
    for (size_t i = 0; i < nRays(); i++) IPolyenergeticAbsorb[i] = (uint32)floorf(IAbsorb[i]);
}

// I0 of the nominal scintillator thickness for one energy (CBCTForwardProj.cpp:92-95).
void CBCTForwardProj::addStandardI0(float& I0Standard)
{
    I0Standard += (float)mCTScanParas.I0Val * mCTScanSystemInfo.spectrumVal *
                  mCTScanParas.mScintilltorInfo.detResponseFactor *
                  (1 - expf(-h_mForwardProj.scintillatorLineAtten[specIndex] *
                            mCTScanParas.mScintilltorInfo.scintillatorThickness));
}

// Per-pixel CsI thickness, srand(100) + MSVC rand() (CBCTForwardProj.cpp:99-111).
void CBCTForwardProj::computePerScinThinckness()
{
    if (!h_mForwardProj.scintillatorPerThickness) h_mForwardProj.scintillatorPerThickness = new float[nPix()];
    CTFP_CHECK(ctfp_scintillator_thickness((int64_t)nPix(), mCTScanParas.mScintilltorInfo.scintillatorThickness,
                                           mCTScanParas.mScintilltorInfo.scintillatorThicknessErr,
                                           h_mForwardProj.scintillatorPerThickness));
}

// Detector response of the current energy (CBCTForwardProj.cpp:114-120).
void CBCTForwardProj::updateDetResponse()
{
    if (!h_mForwardProj.detResponse) h_mForwardProj.detResponse = new float[nPix()];
    for (size_t i = 0; i < nPix(); i++)
        h_mForwardProj.detResponse[i] =
            mCTScanParas.mScintilltorInfo.detResponseFactor *
            (1 - expf(-h_mForwardProj.scintillatorLineAtten[specIndex] * h_mForwardProj.scintillatorPerThickness[i]));
}

// Per-view focal-spot offsets (CBCTForwardProj.cpp:122-148), mm.
void CBCTForwardProj::computeFoSpOffset()
{
    if (!h_mForwardProj.foSpOffsetU) h_mForwardProj.foSpOffsetU = new float[mCTScanParas.projNum];
    if (!h_mForwardProj.foSpOffsetV) h_mForwardProj.foSpOffsetV = new float[mCTScanParas.projNum];
    CTFP_CHECK(ctfp_focal_spot_offsets((int64_t)mCTScanParas.projNum, mCTScanParas.focalSpotSize,
                                       h_mForwardProj.foSpOffsetU, h_mForwardProj.foSpOffsetV));
}

// Normalised spectrum, SpecEnergyNum values (CBCTForwardProj.cpp:150-171).
void CBCTForwardProj::readSpecrtumNorm()
{
    const std::vector<float> v = read_table(mFilePath.spectrumPath, mCTScanParas.specEnergyNum, "spectrum");
    DELETEARR(h_mForwardProj.spectrumNormal);
    h_mForwardProj.spectrumNormal = new float[v.size()];
    std::memcpy(h_mForwardProj.spectrumNormal, v.data(), v.size() * sizeof(float));
}

// Grid strip / interspace mass attenuation -> 1/mm (CBCTForwardProj.cpp:174-225).
void CBCTForwardProj::readGridMassAttu()
{
    const int E = mCTScanParas.specEnergyNum;
    const std::vector<float> s = read_table(mGridInfo.gridStripMAPath, E, "grid strip attenuation table");
    const std::vector<float> i = read_table(mGridInfo.interspaceMAPath, E, "grid interspace attenuation table");
    DELETEARR(h_mForwardProj.gridLinearAtten);
    DELETEARR(h_mForwardProj.interspaceLinearAtten);
    h_mForwardProj.gridLinearAtten = new float[(size_t)E];
    h_mForwardProj.interspaceLinearAtten = new float[(size_t)E];
    for (int e = 0; e < E; e++) {
        h_mForwardProj.gridLinearAtten[e] = s[(size_t)e] * mGridInfo.gridStripDensity / 10;
        h_mForwardProj.interspaceLinearAtten[e] = i[(size_t)e] * mGridInfo.interspaceDensity / 10;
    }
}

// CsI mass attenuation -> 1/mm (CBCTForwardProj.cpp:228-252).
void CBCTForwardProj::readScintillatorMassAttu()
{
    const int E = mCTScanParas.specEnergyNum;
    const std::vector<float> v = read_table(mFilePath.scintillatorPath, E, "scintillator attenuation table");
    DELETEARR(h_mForwardProj.scintillatorLineAtten);
    h_mForwardProj.scintillatorLineAtten = new float[(size_t)E];
    for (int e = 0; e < E; e++)
        h_mForwardProj.scintillatorLineAtten[e] = v[(size_t)e] * mCTScanParas.mScintilltorInfo.scintillatorDensity / 10;
}

// Response of the pixel at flat index (U + V) / 2 (CBCTForwardProj.cpp:255-258).
void CBCTForwardProj::getADetResponse()
{
    if (!aDetResponse) aDetResponse = new float[(size_t)mCTScanParas.specEnergyNum];
    aDetResponse[specIndex] = h_mForwardProj.detResponse[(mCTScanParas.dNumU + mCTScanParas.dNumV) / 2];
}

void CBCTForwardProj::saveADetResponse()
{
    std::filesystem::create_directories(mFilePath.outputFolder);
    std::ofstream ofs(mFilePath.outputFolder + "/ADetResponse.txt");
    if (!ofs) throw std::runtime_error("cannot write " + mFilePath.outputFolder + "/ADetResponse.txt");
    for (int e = 0; e < mCTScanParas.specEnergyNum; e++) ofs << aDetResponse[e] << std::endl;
}

void CBCTForwardProj::showScanSystemInfo()
{
    std::cout << "detector " << mCTScanParas.dNumU << " x " << mCTScanParas.dNumV << " @ " << mCTScanParas.dSize
              << " mm, SDD " << mCTScanParas.sdd << " mm, SOD " << mCTScanParas.sod << " mm, FOV "
              << 2 * mCTScanSystemInfo.FOVR << " x " << 2 * mCTScanSystemInfo.FOVH << " mm, voxel "
              << mCTScanSystemInfo.pSizeX << " x " << mCTScanSystemInfo.pSizeY << " x " << mCTScanSystemInfo.pSizeZ
              << " mm, photons " << mCTScanParas.I0Val << std::endl;
}

void CBCTForwardProj::showGridmInfo()
{
    std::cout << "grid " << mGridInfo.gridStripMaterial << "/" << mGridInfo.interspaceMaterial << ", period "
              << mGridInfo.gridStripsWidth + mGridInfo.interspcaceWidth << " um (strip " << mGridInfo.gridStripsWidth
              << ", interspace " << mGridInfo.interspcaceWidth << "), h " << mGridInfo.h << " mm, FD " << mGridInfo.FD
              << " mm" << std::endl;
}

// proj = logf(I0 / floor(I)) on the host (CBCTForwardProj.cpp:376-387).
void CBCTForwardProj::computeProj()
{
    if (!h_mForwardProj.proj) h_mForwardProj.proj = new float[nRays()];
    for (size_t j = 0; j < mCTScanParas.projNum; j++)
        for (size_t i = 0; i < nPix(); i++)
            h_mForwardProj.proj[j * nPix() + i] = logf(h_mForwardProj.I0[i] / IPolyenergetic[j * nPix() + i]);
}

void CBCTForwardProj::creatOutputFolder()
{
    if (std::filesystem::exists(mFilePath.outputFolder)) _removeOutputFolder();
    std::filesystem::create_directories(mFilePath.outputFolder);
}

void CBCTForwardProj::_removeOutputFolder() { std::filesystem::remove_all(mFilePath.outputFolder); }

void CBCTForwardProj::writeRaw(const std::string& name, const void* data, size_t bytes) const
{
    const std::string path = mFilePath.outputFolder + "/" + name;
    std::ofstream ofs(path, std::ios::out | std::ios::binary);
    if (!ofs) throw std::runtime_error("cannot write " + path);
    ofs.write(static_cast<const char*>(data), (std::streamsize)bytes);
}

void CBCTForwardProj::runDeviceProjection(bool grid, bool response, bool single)
{
    computeParas();
    readSpecrtumNorm();
    DELETE(mPhantomObject);
    mPhantomObject = new PhantomObject(mCTScanParas, _mPhantomMaterial);
    mPhantomObject->readData();
    if (response) {
        computePerScinThinckness();
        readScintillatorMassAttu();
    }
    if (grid) {
        readGridMassAttu();
        initGridInfo();
    }
    const int E = mCTScanParas.specEnergyNum;
    const size_t U = mCTScanParas.dNumU, V = mCTScanParas.dNumV, P = mCTScanParas.projNum;
    const size_t npix = U * V, nray = npix * P, nvox = mPhantomObject->voxels();
    const int M = single ? 1 : _mPhantomMaterial.materialNum;
    if (M < 1 || M > CTFP_MAX_MATERIALS) throw std::runtime_error("MaterialNum must be 1..4");

    ctfp_geometry g{};
    g.pNumX = (int64_t)mCTScanParas.pNumX; g.pNumY = (int64_t)mCTScanParas.pNumY; g.pNumZ = (int64_t)mCTScanParas.pNumZ;
    g.pLengthX = mCTScanParas.pLengthX; g.pLengthY = mCTScanParas.pLengthY; g.pLengthZ = mCTScanParas.pLengthZ;
    g.projNum = (int64_t)P; g.dNumU = (int64_t)U; g.dNumV = (int64_t)V;
    g.dSize = mCTScanParas.dSize; g.sod = mCTScanParas.sod; g.sdd = mCTScanParas.sdd;
    g.rotatedDirection = mCTScanParas.rotatedDirection;

    PlanGuard plan;
    CTFP_CHECK(ctfp_plan_create(&g, M, interp_from_env(), 0, &plan.p));
    if (const char* sk = std::getenv("CTFP_SKIP_EMPTY"))
        if (sk[0] == '1') CTFP_CHECK(ctfp_plan_set_skip_empty(plan.p, 1));
    if (focalSpot_)
        CTFP_CHECK(ctfp_plan_set_focal_spot(plan.p, h_mForwardProj.foSpOffsetU, h_mForwardProj.foSpOffsetV));
    DeviceBuffers db;

    // density maps: label -> rho_m (multi-material), label * density[0] (single)
    float* vols[CTFP_MAX_MATERIALS] = {};
    for (int m = 0; m < M; m++) vols[m] = db.alloc<float>(nvox);
    if (single) {
        std::vector<float> rho(nvox);
        mPhantomObject->computeDesity(rho.data());
        CUDA_CHECK(cudaMemcpy(vols[0], rho.data(), nvox * sizeof(float), cudaMemcpyHostToDevice));
    } else {
        uint8_t* d_lab = db.alloc<uint8_t>(nvox);
        CUDA_CHECK(cudaMemcpy(d_lab, mPhantomObject->structure(), nvox, cudaMemcpyHostToDevice));
        CTFP_CHECK(ctfp_labels_to_density(d_lab, (int64_t)nvox, M, _mPhantomMaterial.density, vols, nullptr));
    }
    // attenuation per density, 1/mm per g/cm^3 (PhantomObject.cpp:56, 62)
    std::vector<float> mu((size_t)E * M);
    for (int e = 0; e < E; e++)
        for (int m = 0; m < M; m++) mu[(size_t)e * M + m] = mPhantomObject->massAtten((size_t)e, m) / 10.f;
    // grid transmission [E][U] and detector response [E][V][U], built on the device
    gridTable_.clear();
    detTable_.clear();
    if (grid) {
        float* d_grid = db.alloc<float>((size_t)E * U);
        ctfp_grid_params gp{mGridInfo.gridStripsWidth, mGridInfo.interspcaceWidth, mGridInfo.h, mGridInfo.FD};
        CTFP_CHECK(ctfp_build_grid_table(&g, &gp, E, h_mForwardProj.gridLinearAtten,
                                         h_mForwardProj.interspaceLinearAtten, CTFP_GRID_COLUMN, d_grid, nullptr));
        gridTable_.resize((size_t)E * U);
        CUDA_CHECK(cudaMemcpy(gridTable_.data(), d_grid, gridTable_.size() * sizeof(float), cudaMemcpyDeviceToHost));
    }
    if (response) {
        float* d_thick = db.alloc<float>(npix);
        float* d_det = db.alloc<float>((size_t)E * npix);
        CUDA_CHECK(cudaMemcpy(d_thick, h_mForwardProj.scintillatorPerThickness, npix * sizeof(float),
                              cudaMemcpyHostToDevice));
        CTFP_CHECK(ctfp_build_det_response(E, (int64_t)npix, h_mForwardProj.scintillatorLineAtten, d_thick,
                                           mCTScanParas.mScintilltorInfo.detResponseFactor, d_det, nullptr));
        detTable_.resize((size_t)E * npix);
        CUDA_CHECK(cudaMemcpy(detTable_.data(), d_det, detTable_.size() * sizeof(float), cudaMemcpyDeviceToHost));
    }
    CTFP_CHECK(ctfp_set_spectral_tables(plan.p, E, h_mForwardProj.spectrumNormal, mu.data(),
                                        grid ? gridTable_.data() : nullptr, grid ? CTFP_GRID_COLUMN : CTFP_GRID_NONE,
                                        response ? detTable_.data() : nullptr, (float)mCTScanParas.I0Val));

    float* d_I = db.alloc<float>(nray);
    float* d_A = db.alloc<float>(nray);
    float* d_I0 = db.alloc<float>(npix);
    uint32_t* d_Ip = db.alloc<uint32_t>(nray);
    uint32_t* d_Ap = db.alloc<uint32_t>(nray);
    float* d_proj = db.alloc<float>(nray);
    CTFP_CHECK(ctfp_forward(plan.p, vols, d_I, d_A, d_I0, nullptr, nullptr));
    CTFP_CHECK(ctfp_finalize_counts((int64_t)npix, (int64_t)P, d_I, d_A, d_I0, d_Ip, d_Ap, d_proj, nullptr));

    DELETEARR(I); DELETEARR(IAbsorb); DELETEARR(IPolyenergetic); DELETEARR(IPolyenergeticAbsorb);
    DELETEARR(h_mForwardProj.I0); DELETEARR(h_mForwardProj.proj);
    I = new float[nray];
    IAbsorb = new float[nray];
    IPolyenergetic = new uint32[nray];
    IPolyenergeticAbsorb = new uint32[nray];
    h_mForwardProj.I0 = new float[npix];
    h_mForwardProj.proj = new float[nray];
    CUDA_CHECK(cudaMemcpy(I, d_I, nray * sizeof(float), cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(IAbsorb, d_A, nray * sizeof(float), cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(IPolyenergetic, d_Ip, nray * sizeof(uint32), cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(IPolyenergeticAbsorb, d_Ap, nray * sizeof(uint32), cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(h_mForwardProj.I0, d_I0, npix * sizeof(float), cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(h_mForwardProj.proj, d_proj, nray * sizeof(float), cudaMemcpyDeviceToHost));

    // per-energy views the reference leaves behind: response sample, last energy's tables
    if (response) {
        DELETEARR(aDetResponse);
        aDetResponse = new float[(size_t)E];
        for (int e = 0; e < E; e++) aDetResponse[e] = detTable_[(size_t)e * npix + (U + V) / 2];
        DELETEARR(h_mForwardProj.detResponse);
        h_mForwardProj.detResponse = new float[npix];
        std::memcpy(h_mForwardProj.detResponse, &detTable_[(size_t)(E - 1) * npix], npix * sizeof(float));
    }
    if (grid) {
        DELETEARR(h_mForwardProj.grid);
        h_mForwardProj.grid = new float[U];
        std::memcpy(h_mForwardProj.grid, &gridTable_[(size_t)(E - 1) * U], U * sizeof(float));
    }
    specIndex = (size_t)E;
}

void CBCTForwardProj::runFlatField(bool grid, bool response)
{
    computeParas();
    readSpecrtumNorm();
    if (response) {
        computePerScinThinckness();
        readScintillatorMassAttu();
    }
    if (grid) {
        readGridMassAttu();
        initGridInfo();
    }
    const int E = mCTScanParas.specEnergyNum;
    const size_t U = mCTScanParas.dNumU;
    DELETEARR(h_mForwardProj.I0);
    h_mForwardProj.I0 = new float[nPix()]();
    std::vector<float> gtab;
    if (grid) {
        ctfp_geometry g{};
        g.pNumX = g.pNumY = g.pNumZ = 1;
        g.pLengthX = g.pLengthY = g.pLengthZ = 1.0f;
        g.projNum = 1; g.dNumU = (int64_t)U; g.dNumV = (int64_t)mCTScanParas.dNumV;
        g.dSize = mCTScanParas.dSize; g.sod = mCTScanParas.sod; g.sdd = mCTScanParas.sdd; g.rotatedDirection = 1;
        DeviceBuffers db;
        float* d_grid = db.alloc<float>((size_t)E * U);
        ctfp_grid_params gp{mGridInfo.gridStripsWidth, mGridInfo.interspcaceWidth, mGridInfo.h, mGridInfo.FD};
        CTFP_CHECK(ctfp_build_grid_table(&g, &gp, E, h_mForwardProj.gridLinearAtten,
                                         h_mForwardProj.interspaceLinearAtten, CTFP_GRID_COLUMN, d_grid, nullptr));
        gtab.resize((size_t)E * U);
        CUDA_CHECK(cudaMemcpy(gtab.data(), d_grid, gtab.size() * sizeof(float), cudaMemcpyDeviceToHost));
    }
    float I0Standard = 0.0f;
    // FP32 sums in energy order, as addI0 / addStandardI0 (CBCTPolyForwardProjNoGrid.cpp:290-299)
    for (specIndex = 0; specIndex < (size_t)E; specIndex++) {
        mCTScanSystemInfo.spectrumVal = h_mForwardProj.spectrumNormal[specIndex];
        if (response) updateDetResponse();
        for (size_t k = 0; k < nPix(); k++) {
            float w = (float)mCTScanParas.I0Val * mCTScanSystemInfo.spectrumVal;
            if (grid) w = w * gtab[specIndex * U + k % U];
            if (response) w = w * h_mForwardProj.detResponse[k];
            h_mForwardProj.I0[k] += w;
        }
        if (response) addStandardI0(I0Standard);
    }
    std::cout << "I0 at the nominal scintillator thickness " << mCTScanParas.mScintilltorInfo.scintillatorThickness
              << " mm: " << I0Standard << std::endl;
}
