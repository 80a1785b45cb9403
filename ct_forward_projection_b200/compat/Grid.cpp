// Grid.cpp — see Grid.h.
#include "Grid.h"

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "ctfp.h"

Grid::Grid(GridAndDetectorSystem sys) : sys_(sys) {}
Grid::Grid(float* out, GridAndDetectorSystem sys) : sys_(sys), grid_(out) {}
Grid::~Grid()
{
    if (d_grid_) cudaFree(d_grid_);
}

void Grid::defGrid()
{
    if (!d_grid_ && cudaMalloc(&d_grid_, sizeof(float) * sys_.dNums) != cudaSuccess)
        throw std::runtime_error("Grid: device allocation failed");
}

void Grid::updataGrid(float mu_strip, float mu_inter)
{
    defGrid();
    ctfp_geometry g{};
    g.pNumX = g.pNumY = g.pNumZ = 1;
    g.pLengthX = g.pLengthY = g.pLengthZ = 1.0f;
    g.projNum = 1;
    g.dNumU = (int64_t)sys_.dNums;
    g.dNumV = 1;
    g.dSize = sys_.dSize / 1000.0f;  // um -> mm
    g.sod = 1.0f;
    g.sdd = 2.0f;
    g.rotatedDirection = 1;
    ctfp_grid_params gp{sys_.gridStripsWidth, sys_.interspcaceWidth, sys_.h, sys_.FD};
    if (ctfp_build_grid_table(&g, &gp, 1, &mu_strip, &mu_inter, CTFP_GRID_COLUMN, d_grid_, nullptr) != CTFP_OK)
        throw std::runtime_error(std::string("Grid::updataGrid: ") + ctfp_last_error_string());
    if (grid_ && cudaMemcpy(grid_, d_grid_, sizeof(float) * sys_.dNums, cudaMemcpyDeviceToHost) != cudaSuccess)
        throw std::runtime_error("Grid::updataGrid: copy failed");
}
