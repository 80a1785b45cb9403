// PhantomObject.h — label phantom and per-material attenuation tables, the
// interface of the reference's Source/PhantomObject.h:9-47.
#pragma once

#include <string>
#include <vector>

#include "DataType.h"

class PhantomObject {
public:
    PhantomObject(const CTScanParas mCTScanParas, const PhantomMaterial mPhantomMaterial);
    ~PhantomObject();

    // Reads the uint8 label volume (StructureMarkPath) and the mass-attenuation
    // tables (one value per line, line e = (e+1) keV; PhantomObject.cpp:75-131).
    // Throws std::runtime_error when a file cannot be read.
    void readData();

    // mu(x) = massAtten[e][label-1] * density[label-1] / 10 in 1/mm, 0 for label 0
    // (PhantomObject.cpp:38-58).
    void updataLineAtten(float* lineAttenCoef, size_t specIndex);
    // massAtten[e][0] / 10 (PhantomObject.cpp:60-63).
    void updataMassAtten(float& massAttenCoef, size_t specIndex);
    // density(x) = label(x) * density[0] (PhantomObject.cpp:65-71).
    void computeDesity(float* density);

    const uint8* structure() const { return _structureMark.data(); }
    size_t voxels() const { return _pNumX * _pNumY * _pNumZ; }
    int materials() const { return _mPhantomMaterial.materialNum; }
    float massAtten(size_t specIndex, int material) const { return _massAttenCoef[specIndex][(size_t)material]; }
    float density(int material) const { return _mPhantomMaterial.density[material]; }

private:
    void _readPhantomStructure();
    void _readMassAtten();

    PhantomMaterial _mPhantomMaterial;
    std::vector<uint8> _structureMark;
    std::vector<std::vector<float>> _massAttenCoef;  // [energy][material]
    int _specEnergyNum;
    size_t _pNumX, _pNumY, _pNumZ;
};
