// ctfp_kernels.cuh — kernel parameter blocks and launcher declarations.
#pragma once

#include "ctfp_device.cuh"

namespace ctfp {

// One problem as the march kernels see it.
struct MarchParams {
    GeomParams g;
    const float* vol[kMaxM];          // material densities [nz][ny][nx]
    cudaTextureObject_t tex[kMaxM];   // same volumes as 3D textures (TEXTURE mode)
    cudaTextureObject_t ltex[kMaxM];  // same volumes as layered 2D textures (SAMPLER_LAYERED)
    cudaTextureObject_t xtex[kMaxM];  // SAMPLER_AXIS: layered along x (layer x, texel (y, z))
    cudaTextureObject_t ytex[kMaxM];  // SAMPLER_AXIS: layered along y (layer y, texel (x, z))
    float* L;                         // [P][V][U][M] path integrals (out, may be null)
    const float* Lin;                 // [P][V][U][M] path integrals (in, epilogue/adjoint)
    float* I;                         // [P][V][U] (may be null)
    float* IAbs;                      // [P][V][U] (may be null)
    const float* W;                   // [E][V][U] energy weights I0Val*S*G*D
    const float* mu;                  // [E][M] attenuation per density, 1/mm per g/cm^3
    const float* gI;                  // [P][V][U] dLoss/dI (adjoint)
    const float* gIAbs;               // [P][V][U] dLoss/dIAbsorb (adjoint, may be null)
    float* gvol[kMaxM];               // gradient volumes (adjoint)
    float4* gexp[kMaxM];              // face-expanded gradient accumulators (adjoint), see AxisScatter
    int E;
    int view0;                        // first view of this launch
    int n_views;                      // views in this launch
    int views_per_cta;                // views each CTA marches for its pixel tile
    int out_view0;                    // view stored at index 0 of I, IAbs, L, Lin, gI, gIAbs (0: full arrays)
    const uint8_t* occ;               // empty-space skipping: brick occupancy (null: march every sample)
    int occ_x, occ_y;                 // bricks along x, y (see launch_occupancy)
    unsigned* status;                 // plan-owned word; kCtfpStatusWaitTimeout is or-ed in when a bounded wait ran out
    int wait_limit;                   // polls of a TMA completion before a CTA gives up on staging
};

// Bits of the plan's device status word (ctfp_plan_check_status; the same
// values as CTFP_STATUS_* in ctfp.h).  WaitTimeout: a CTA gave up waiting for
// a TMA load and read the volume instead (outputs correct).  ExitWaitTimeout:
// the CTA's bounded wait at exit for that load ran out as well, so the copy may
// have landed in shared memory another CTA owned (outputs not trusted).
constexpr unsigned kCtfpStatusWaitTimeout = 1u;
constexpr unsigned kCtfpStatusExitWaitTimeout = 2u;

// Bricks of kOccShift^2 voxels per axis for empty-space skipping.  Brick
// (bx, by, bz) is marked when any material has a non-zero voxel in
// [8b - 1, 8b + 7] on every axis: exactly the voxels a footprint with base
// corner ix in [8b - 1, 8b + 6] (brick of ix + 1) can read.
constexpr int kOccShift = 3;
inline int occ_dim(int n) { return ((n + 1) >> kOccShift) + 1; }

struct LaunchShape {
    int tile_u = 16, tile_v = 8, views_per_cta = 2;
    int min_ctas = 4;  // register cap of the forward march: 65536 / (256 * min_ctas) per thread
};

// Launchers; all return cudaGetLastError() of the launch.  sampler selects
// SAMPLER_GLOBAL or SAMPLER_LAYERED for the software interp modes.
cudaError_t launch_forward(const MarchParams& prm, int M, int interp, int sampler, bool do_spectral,
                           const LaunchShape& ls, cudaStream_t st);
cudaError_t launch_spectral_from_L(const MarchParams& prm, int M, cudaStream_t st);
// Adjoint scatter into the face-expanded accumulators prm.gexp (zeroed by
// the caller), followed by launch_fold into prm.gvol.
cudaError_t launch_backward(const MarchParams& prm, int M, int interp, bool from_gL, const LaunchShape& ls,
                            cudaStream_t st);
cudaError_t launch_fold(const MarchParams& prm, int M, cudaStream_t st);
// Elements (float4) of one material's face-expanded accumulator (face_elems).
size_t expanded_elems(const GeomParams& g);
cudaError_t launch_weights(const float* spectrum, const float* grid, int grid_layout, const float* det,
                           float I0Val, int E, int U, int V, float* W, float* I0, cudaStream_t st);
cudaError_t launch_finalize(int64_t n_pix, int64_t n_views, const float* I, const float* IAbs, const float* I0,
                            uint32_t* Ipoly, uint32_t* IAbsPoly, float* proj, cudaStream_t st);
cudaError_t launch_sample_points(const float* vol, cudaTextureObject_t tex, int nx, int ny, int nz, int interp,
                                 const float* pts, int64_t n, float* out, cudaStream_t st);
cudaError_t launch_count_support(const GeomParams& g, unsigned long long* out, cudaStream_t st);
// Focal-spot re-alignment of compact line-integral images [n_views][V][U][M]
// of views view0.. (interp selects exact or texture-unit bilinear weights).
cudaError_t launch_shift_views(const float* in, float* out, const GeomParams& g, int M, int interp, int view0,
                               int n_views, cudaStream_t st);
// SAMPLER_AXIS: writes one volume [nz][ny][nx] into its x-layered copy
// (surface xs: texture layer x + 1, texel (y, z)) and its y-layered copy (ys:
// texture layer y + 1, texel (x, z)).
cudaError_t launch_axis_fill(const float* vol, int nx, int ny, int nz, cudaSurfaceObject_t xs, cudaSurfaceObject_t ys,
                             cudaStream_t st);
// The axis march's texture quad-gathers over every view of a problem, with the
// launch shape's tile and lane layout: out[0] += quads, out[1] += samples.
cudaError_t launch_axis_gather_count(const GeomParams& g, int interp, const LaunchShape& ls, unsigned long long* out,
                                     cudaStream_t st);
// Zeros the pad layers (0 and the last) of both copies; once per array.
cudaError_t launch_axis_zero_pads(int nx, int ny, int nz, cudaSurfaceObject_t xs, cudaSurfaceObject_t ys,
                                  cudaStream_t st);
// Fills occ [occ_dim(nz)][occ_dim(ny)][occ_dim(nx)] from the M volumes
// (vol: host array of M device pointers; occ is zeroed first).
cudaError_t launch_occupancy(const float* const* vol, int M, int nx, int ny, int nz, uint8_t* occ, cudaStream_t st);

}  // namespace ctfp
