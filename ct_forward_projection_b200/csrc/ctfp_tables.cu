// ctfp_tables.cu — table builders on the device: anti-scatter grid
// transmission, scintillator response, label-map ingestion; and the seeded
// scintillator thickness on the host.
//
// The reference builds these on the host once per energy: the grid over
// dNumU * dSize one-micron units with one expf each (Grid.cpp:90-270), the
// detector response over U*V pixels (CBCTForwardProj.cpp:114-120), and the
// multi-material attenuation volume over N^3 voxels (PhantomObject.cpp:38-58).
#include <cmath>
#include <cstring>
#include <string>

#include "../../include/ctfp.h"
#include "ctfp_device.cuh"

namespace ctfp {
void set_last_error(const std::string& msg);  // ctfp_api.cu
}

namespace {

ctfp_status tfail(ctfp_status st, const std::string& m)
{
    ctfp::set_last_error(m);
    return st;
}

// One focused-grid problem in micron units (Grid.cpp:36-63, 373-386).
struct GridUnits {
    long long N;      // discrete 1-um units across the detector, dNumU * dSize
    int dSize;        // um per detector column
    int sw, iw, period;
    float h, FD;      // um
    long long c;      // N / 2
    long long start;  // first unit (counting leftwards) of the periodic region
    int uOdd, iOdd;
    float ms, mi;     // per-um attenuation of strip and interspace at one energy
};

// Unit height h/FD * sqrt(FD^2 + d^2 + y^2), d from the grid centre
// (Grid.cpp:76-87); y = 0 reproduces the reference.
__device__ __forceinline__ float unit_height(const GridUnits& gu, long long j, float y)
{
    const float dc = (float)((double)j + 0.5 - (double)((float)gu.N / 2));
    return gu.h / gu.FD * sqrtf(gu.FD * gu.FD + dc * dc + y * y);
}

// Sum of the 1-um unit transmissions over the mirrored-index range
// [jlo, jhi]: the closed form of the fill loops of createDiscreteGrid_u{E,O}d{E,O}
// (Grid.cpp:90-270).  Units j > start form the central interspace half-gap,
// each with its own height (Grid.cpp:93-96, 137-141, 181-184, 226-230); below
// it the pattern repeats with period sw + iw counted leftwards from start:
// strip units with their own heights (Grid.cpp:107), interspace units with the
// height of their period's first unit (Grid.cpp:115).  Interspace units of one
// period therefore share one transmission, and each run of them contributes its
// length times that value.
__device__ double sum_units(const GridUnits& gu, long long jlo, long long jhi, float y)
{
    double sum = 0.0;
    long long j = jhi;
    // central half-gap (j > start), own unit heights
    for (; j >= jlo && j > gu.start; j--) sum += (double)expf(-gu.mi * unit_height(gu, j, y));
    while (j >= jlo) {
        const long long k = gu.start - j;
        const long long q = k / gu.period, r = k % gu.period;
        if (r < gu.sw) {
            // strip units of this period, down to the strip's end or jlo
            const long long jend = max(jlo, j - (gu.sw - 1 - r));
            for (; j >= jend; j--) sum += (double)expf(-gu.ms * unit_height(gu, j, y));
        } else {
            // interspace units of this period share one transmission
            const long long jend = max(jlo, j - (gu.period - 1 - r));
            const float t = expf(-gu.mi * unit_height(gu, gu.start - q * gu.period, y));
            sum += (double)t * (double)(j - jend + 1);
            j = jend - 1;
        }
    }
    return sum;
}

// First unit of the mirrored (right) half and the mirror image of a unit
// there, per parity case (Grid.cpp:126-129, 170-173, 214-217, 260-263).
__device__ __forceinline__ long long mirror_start(const GridUnits& gu)
{
    return (!gu.uOdd && !gu.iOdd) ? gu.c : gu.c + 1;
}
__device__ __forceinline__ long long mirror_of(const GridUnits& gu, long long i)
{
    return ((!gu.uOdd && !gu.iOdd) || (gu.uOdd && gu.iOdd)) ? gu.N - i - 1 : gu.N - i;
}

__global__ void k_grid(GridUnits gu, int E, const float* __restrict__ mus, const float* __restrict__ mui, int U,
                       int V, int layout, float dHalfLV_um, float dSize_um, float* out)
{
    const long long per_e = layout == CTFP_GRID_PIXEL ? (long long)U * V : (long long)U;
    const long long n = per_e * E;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int e = (int)(t / per_e);
        const long long rem = t % per_e;
        const int u = (int)(rem % U);
        const int v = (int)(rem / U);
        GridUnits g = gu;
        g.ms = mus[e] / 1000.0f;  // 1/mm -> 1/um (Grid.cpp:410)
        g.mi = mui[e] / 1000.0f;  // (Grid.cpp:411)
        float y = 0.f;
        if (layout == CTFP_GRID_PIXEL) y = dHalfLV_um - dSize_um / 2 - (float)v * dSize_um;
        // binning1D: mean over the pixel's units, accumulated in double
        // (Grid.cpp:299-306); units left of the mirror map to themselves,
        // units right of it to their mirror images
        const long long i0 = (long long)u * gu.dSize, i1 = i0 + gu.dSize - 1;
        const long long m = mirror_start(g);
        double sum = 0.0;
        if (i0 < m) sum += sum_units(g, i0, min(i1, m - 1), y);
        if (i1 >= m) sum += sum_units(g, mirror_of(g, i1), mirror_of(g, max(i0, m)), y);
        out[t] = (float)(sum / (double)gu.dSize);
    }
}

__global__ void k_det_response(int E, long long n_pix, const float* __restrict__ mu, const float* __restrict__ thick,
                               float factor, float* out)
{
    const long long n = n_pix * E;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int e = (int)(t / n_pix);
        const long long k = t % n_pix;
        out[t] = factor * (1.0f - expf(-mu[e] * thick[k]));
    }
}

struct DensityParams {
    float* out[ctfp::kMaxM];
    float density[ctfp::kMaxM];
};

__global__ void k_labels(const uint8_t* __restrict__ labels, long long n, int M, DensityParams dp)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int lab = labels[t];
        for (int m = 0; m < M; m++) dp.out[m][t] = (lab == m + 1) ? dp.density[m] : 0.0f;
    }
}

unsigned blocks_for(long long n)
{
    long long nb = (n + 255) / 256;
    if (nb > 148 * 32) nb = 148 * 32;
    return (unsigned)(nb < 1 ? 1 : nb);
}

}  // namespace

extern "C" {

ctfp_status ctfp_build_grid_table(const ctfp_geometry* g, const ctfp_grid_params* grid, int32_t E,
                                  const float* mu_strip, const float* mu_inter, int32_t layout, float* out,
                                  void* stream)
{
    if (!g || !grid || !mu_strip || !mu_inter || !out) return tfail(CTFP_INVALID_ARG, "NULL argument");
    if (E < 1 || E > CTFP_MAX_ENERGIES) return tfail(CTFP_INVALID_ARG, "n_energies out of range");
    if (layout != CTFP_GRID_COLUMN && layout != CTFP_GRID_PIXEL) return tfail(CTFP_INVALID_ARG, "bad layout");
    if (grid->gridStripsWidth <= 0 || grid->interspaceWidth <= 0 || !(grid->h > 0.f) || !(grid->FD > 0.f))
        return tfail(CTFP_INVALID_ARG, "grid widths, h and FD must be positive");
    if (g->dNumU <= 0 || g->dNumV <= 0 || !(g->dSize > 0.f)) return tfail(CTFP_INVALID_ARG, "bad detector");
    GridUnits gu;
    std::memset(&gu, 0, sizeof(gu));
    // dSize in um as the reference truncates it (CBCTPolyForwardProjGrid.cpp:291 into size_t Grid::dSize)
    const float dsz_um = g->dSize * 1000;
    gu.dSize = (int)dsz_um;
    if (gu.dSize < 1) return tfail(CTFP_INVALID_ARG, "dSize below 1 um");
    gu.N = (long long)g->dNumU * gu.dSize;
    gu.sw = grid->gridStripsWidth;
    gu.iw = grid->interspaceWidth;
    gu.period = gu.sw + gu.iw;
    gu.h = grid->h * 1000;
    gu.FD = grid->FD * 1000;
    gu.c = gu.N / 2;
    gu.uOdd = (int)(gu.N % 2);
    gu.iOdd = gu.iw % 2;
    if (gu.N < (long long)gu.iw + 2) return tfail(CTFP_INVALID_ARG, "detector narrower than the central interspace");
    if (!gu.uOdd) gu.start = gu.c - 1 - gu.iw / 2;
    else gu.start = gu.iOdd ? gu.c - 1 - gu.iw / 2 : gu.c - gu.iw / 2;
    float *dms = nullptr, *dmi = nullptr;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMalloc(&dms, sizeof(float) * E);
    if (e == cudaSuccess) e = cudaMalloc(&dmi, sizeof(float) * E);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dms, mu_strip, sizeof(float) * E, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dmi, mu_inter, sizeof(float) * E, cudaMemcpyHostToDevice, s);
    const float dHalfLV = (float)g->dNumV * g->dSize / 2;
    const long long n = (long long)E * g->dNumU * (layout == CTFP_GRID_PIXEL ? g->dNumV : 1);
    if (e == cudaSuccess) {
        k_grid<<<blocks_for(n), 256, 0, s>>>(gu, E, dms, dmi, (int)g->dNumU, (int)g->dNumV, layout, dHalfLV * 1000,
                                             dsz_um, out);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(dms);
    cudaFree(dmi);
    if (e != cudaSuccess) return tfail(CTFP_CUDA_ERROR, std::string("ctfp_build_grid_table: ") + cudaGetErrorString(e));
    return CTFP_OK;
}

ctfp_status ctfp_scintillator_thickness(int64_t n_pix, float thickness, float thickness_err, float* out)
{
    if (n_pix < 0 || !out) return tfail(CTFP_INVALID_ARG, "bad argument");
    if (!(thickness_err >= 0.f)) return tfail(CTFP_INVALID_ARG, "thickness_err must be non-negative");
    // srand(100); MSVC rand(): state = state * 214013 + 2531011, (state >> 16) & 0x7fff
    uint32_t state = 100u;
    const int beg = (int)(-thickness_err * 10000);
    const int endd = (int)(thickness_err * 10000);
    for (int64_t i = 0; i < n_pix; i++) {
        state = state * 214013u + 2531011u;
        const int r = (int)((state >> 16) & 0x7fffu);
        const float err = -thickness_err + (float)(r % (endd - beg + 1)) / 10000.0f;
        out[i] = thickness + err;
    }
    return CTFP_OK;
}

ctfp_status ctfp_build_det_response(int32_t E, int64_t n_pix, const float* mu_scint, const float* thickness,
                                    float factor, float* out, void* stream)
{
    if (E < 1 || E > CTFP_MAX_ENERGIES || n_pix < 0 || !mu_scint || !thickness || !out)
        return tfail(CTFP_INVALID_ARG, "bad argument");
    cudaStream_t s = (cudaStream_t)stream;
    float* dmu = nullptr;
    cudaError_t e = cudaMalloc(&dmu, sizeof(float) * E);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dmu, mu_scint, sizeof(float) * E, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && n_pix > 0) {
        k_det_response<<<blocks_for(n_pix * E), 256, 0, s>>>(E, n_pix, dmu, thickness, factor, out);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(dmu);
    if (e != cudaSuccess) return tfail(CTFP_CUDA_ERROR, std::string("ctfp_build_det_response: ") + cudaGetErrorString(e));
    return CTFP_OK;
}

ctfp_status ctfp_labels_to_density(const uint8_t* labels, int64_t n_vox, int32_t M, const float* density,
                                   float* const* out, void* stream)
{
    if (!labels || !density || !out || n_vox < 0 || M < 1 || M > CTFP_MAX_MATERIALS)
        return tfail(CTFP_INVALID_ARG, "bad argument");
    DensityParams dp;
    std::memset(&dp, 0, sizeof(dp));
    for (int m = 0; m < M; m++) {
        if (!out[m]) return tfail(CTFP_INVALID_ARG, "output pointer is NULL");
        dp.out[m] = out[m];
        dp.density[m] = density[m];
    }
    if (n_vox > 0) k_labels<<<blocks_for(n_vox), 256, 0, (cudaStream_t)stream>>>(labels, n_vox, M, dp);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return tfail(CTFP_CUDA_ERROR, std::string("ctfp_labels_to_density: ") + cudaGetErrorString(e));
    return CTFP_OK;
}

}  // extern "C"
