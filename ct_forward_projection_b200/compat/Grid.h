// Grid.h — focused anti-scatter grid, the interface of the reference's
// Source/Grid.h:42-158.  The transmission per detector column is computed on
// the device by ctfp_build_grid_table (include/ctfp.h).
#pragma once

#include <cstddef>
#include <string>
#include <vector>

struct GridAndDetectorSystem {
    size_t dNums = 0;           // detector columns
    float dSize = 0;            // um
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
    float gridStripLinearAtten = 0;    // 1/mm
    float interspaceLinearAtten = 0;   // 1/mm
    size_t mI0Photons = 0;
    size_t angleNums = 0;
};

class Grid {
public:
    explicit Grid(GridAndDetectorSystem sys);
    Grid(float* gridOutput, GridAndDetectorSystem sys);
    ~Grid();
    Grid(const Grid&) = delete;
    Grid& operator=(const Grid&) = delete;

    // Prepares the discretisation (Grid.cpp:373-405).
    void defGrid();
    // Writes the column transmission for one energy into the output array
    // (Grid.cpp:408-443); attenuation in 1/mm.
    void updataGrid(float gridStripLinearAtten, float interspaceLinearAtten);
    // The reference writes a period index to a fixed path and discards it
    // (Grid.cpp:642); nothing to compute here.
    void getPeriodIncex(std::vector<size_t>& gridPeriodIndex) { gridPeriodIndex.clear(); }

private:
    GridAndDetectorSystem sys_;
    float* grid_ = nullptr;      // host output, dNums
    float* d_grid_ = nullptr;    // device scratch, dNums
};
