// PhantomObject.cpp — see PhantomObject.h.
#include "PhantomObject.h"

#include <fstream>
#include <iostream>
#include <stdexcept>

PhantomObject::PhantomObject(const CTScanParas p, const PhantomMaterial m)
    : _mPhantomMaterial(m), _specEnergyNum(p.specEnergyNum), _pNumX(p.pNumX), _pNumY(p.pNumY), _pNumZ(p.pNumZ)
{
}

PhantomObject::~PhantomObject() = default;

void PhantomObject::readData()
{
    _readPhantomStructure();
    _readMassAtten();
}

void PhantomObject::_readPhantomStructure()
{
    _structureMark.assign(voxels(), 0);
    std::ifstream ifs(_mPhantomMaterial.structureMarkPath, std::ios::in | std::ios::binary);
    if (!ifs) throw std::runtime_error("cannot open phantom structure file " + _mPhantomMaterial.structureMarkPath);
    ifs.read(reinterpret_cast<char*>(_structureMark.data()), (std::streamsize)voxels());
    if ((size_t)ifs.gcount() != voxels())
        throw std::runtime_error("phantom structure file " + _mPhantomMaterial.structureMarkPath + " is truncated");
}

void PhantomObject::_readMassAtten()
{
    const int M = _mPhantomMaterial.materialNum;
    _massAttenCoef.assign((size_t)_specEnergyNum, std::vector<float>((size_t)M, 0.0f));
    for (int m = 0; m < M; m++) {
        const std::string& path = _mPhantomMaterial.massAttenPath[m];
        std::ifstream ifs(path);
        if (!ifs) throw std::runtime_error("cannot open mass attenuation table of material " + std::to_string(m + 1) +
                                           ": " + path);
        int e = 0;
        float buf;
        while (e < _specEnergyNum && ifs >> buf) _massAttenCoef[(size_t)e++][(size_t)m] = buf;
        if (e < _specEnergyNum)
            throw std::runtime_error("mass attenuation table " + path + " has fewer than SpecEnergyNum rows");
    }
}

void PhantomObject::updataLineAtten(float* out, size_t e)
{
    for (size_t i = 0; i < voxels(); i++) {
        const int lab = _structureMark[i];
        out[i] = (lab >= 1 && lab <= _mPhantomMaterial.materialNum)
                     ? _massAttenCoef[e][(size_t)lab - 1] * _mPhantomMaterial.density[lab - 1] / 10.f
                     : 0.0f;
    }
}

void PhantomObject::updataMassAtten(float& out, size_t e) { out = _massAttenCoef[e][0] / 10.f; }

void PhantomObject::computeDesity(float* density)
{
    for (size_t i = 0; i < voxels(); i++) density[i] = _structureMark[i] * _mPhantomMaterial.density[0];
}
