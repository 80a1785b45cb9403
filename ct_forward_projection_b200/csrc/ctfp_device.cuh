// ctfp_device.cuh — device-side geometry and sampling shared by the march
// kernels (forward, line integrals, adjoint, batched).
//
// Geometry restates the reference's per-sample coordinate pipeline
// (Source/CUDAFun/CBCTPolyProjGPU.cu:1813-1848 ray direction and t_i,
// :1915-1920 rotation, axis flips and the +0.5 texture offset), but folds it
// into one affine map per ray and axis, c(i) = a + b*i, evaluated in FP64 once
// per ray.  Per sample the coordinate is one FP64 FMA per axis,
// so the 3*K*U*V coordinate buffers and the K*U*V sample buffer of the
// reference (CBCTPolyProjGPU.cu:498-517, 557) do not exist.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ctfp {

enum { INTERP_TRILINEAR = 0, INTERP_TEXEMU = 1, INTERP_TEXTURE = 2 };
constexpr int kMaxM = 4;

// Scalar geometry shared by every ray of one problem.
struct GeomParams {
    int nx, ny, nz;          // voxels
    int U, V, P;             // detector columns, rows, views
    int K;                   // samples per ray (intNum)
    float dHalfLU, dHalfLV, dSize, sod, sdd, FOVR, dx;
    float pHalfX, pHalfY, pHalfZ, pSizeX, pSizeY, pSizeZ;
    const double2* trig;     // per view (cos, sin) of the FP32 view angle
};

// One ray's sample segment: coordinates c(i) = a + b*i in FP64, evaluated
// for i in [i0, i1).  Samples outside [i0, i1) have every trilinear corner
// outside the volume and contribute exactly 0.  FP64 coordinates keep the
// trilinear weights accurate to FP32 rounding relative to themselves, which a
// ray grazing the volume (weights ~1e-4) needs for 1e-5 relative accuracy.
struct RaySeg {
    double ax, ay, az;
    double bx, by, bz;
    int i0, i1;
};

// Clip i to the open interval where lo < a + b*i < hi, intersected with
// [i0, i1).  Conservative by one sample on each side; exactness comes from
// the border handling in the samplers.
__device__ __forceinline__ void clip_axis(double a, double b, double lo, double hi, int& i0, int& i1)
{
    if (fabs(b) < 1e-12) {
        if (!(a > lo && a < hi)) { i1 = i0; }
        return;
    }
    double t0 = (lo - a) / b, t1 = (hi - a) / b;
    double tmin = fmin(t0, t1), tmax = fmax(t0, t1);
    double f0 = floor(tmin) - 1.0, f1 = ceil(tmax) + 2.0;
    if (f0 > (double)i0) i0 = (f0 > 2e9) ? 2000000000 : (int)f0;
    if (f1 < (double)i1) i1 = (f1 < -2e9) ? -2000000000 : (int)f1;
}

__device__ __forceinline__ RaySeg ray_segment(const GeomParams& g, int p, int v, int u)
{
    const double dsz = g.dSize, sdd = g.sdd, sod = g.sod;
    // detector cell centre, index 0 at +dHalf (CBCTPolyProjGPU.cu:1813-1814)
    const double detU = (double)g.dHalfLU - dsz / 2 - (double)u * dsz;
    const double detV = (double)g.dHalfLV - dsz / 2 - (double)v * dsz;
    const double R = sqrt(sdd * sdd + detU * detU + detV * detV);
    // direction cosines as the reference forms them (.cu:1825-1829):
    // (cosG*cosB, cosG*sinB, sinG), which is not (sdd, detU, detV)/R
    const double sinG = detV / R;
    const double cosG = sqrt(sdd * sdd + detU * detU) / R;
    const double sinB = detU / R;
    const double cosB = sqrt(sdd * sdd + detV * detV) / R;
    const double A = cosG * cosB, B = cosG * sinB, C = sinG;
    const double t0 = sod - (double)g.FOVR + (double)g.dx / 2, dt = g.dx;  // .cu:1846
    const double2 cs = g.trig[p];
    const double cth = cs.x, sth = cs.y;
    // tu = X cos - Y sin + pHalfX; tv = -(X sin + Y cos) + pHalfY; tw = -Z + pHalfZ
    const double ku = A * cth - B * sth, cu = -sod * cth + (double)g.pHalfX;
    const double kv = -(A * sth + B * cth), cv = sod * sth + (double)g.pHalfY;
    const double kw = -C, cw = (double)g.pHalfZ;
    const double ax = (ku * t0 + cu) / g.pSizeX, bx = ku * dt / g.pSizeX;
    const double ay = (kv * t0 + cv) / g.pSizeY, by = kv * dt / g.pSizeY;
    const double az = (kw * t0 + cw) / g.pSizeZ, bz = kw * dt / g.pSizeZ;
    RaySeg s;
    s.i0 = 0;
    s.i1 = g.K;
    clip_axis(ax, bx, -1.0, (double)g.nx, s.i0, s.i1);
    clip_axis(ay, by, -1.0, (double)g.ny, s.i0, s.i1);
    clip_axis(az, bz, -1.0, (double)g.nz, s.i0, s.i1);
    if (s.i1 < s.i0) s.i1 = s.i0;
    s.ax = ax; s.ay = ay; s.az = az;
    s.bx = bx; s.by = by; s.bz = bz;
    return s;
}

// Trilinear footprint of one sample: base corner and weights.
struct Corner {
    int ix, iy, iz;
    float wx, wy, wz;
};

// Weight of the texture unit's linear filter for x_B = x - 0.5, where x is the
// FP32 coordinate handed to tex3D: the fraction held with 8 fractional bits.
__device__ __forceinline__ float tex_weight(float xb, float fl)
{
    return floorf((xb - fl) * 256.0f + 0.5f) * (1.0f / 256.0f);
}

// Footprint at the FP64 coordinate (cx, cy, cz).  TRILINEAR: exact fraction
// of the FP64 coordinate, rounded once to FP32.  TEXEMU: the texture unit's
// view of the FP32 coordinate float(c + 0.5) that tex3D receives.
template <int MODE>
__device__ __forceinline__ Corner corner_of(double cx, double cy, double cz)
{
    Corner c;
    if (MODE == INTERP_TRILINEAR) {
        const double fx = floor(cx), fy = floor(cy), fz = floor(cz);
        c.ix = (int)fx; c.iy = (int)fy; c.iz = (int)fz;
        c.wx = (float)(cx - fx); c.wy = (float)(cy - fy); c.wz = (float)(cz - fz);
    } else {
        const float xb = (float)(cx + 0.5) - 0.5f, yb = (float)(cy + 0.5) - 0.5f, zb = (float)(cz + 0.5) - 0.5f;
        const float fx = floorf(xb), fy = floorf(yb), fz = floorf(zb);
        c.ix = (int)fx; c.iy = (int)fy; c.iz = (int)fz;
        c.wx = tex_weight(xb, fx);
        c.wy = tex_weight(yb, fy);
        c.wz = tex_weight(zb, fz);
    }
    return c;
}

__device__ __forceinline__ float lerpf(float a, float b, float w) { return fmaf(w, b - a, a); }

// Loads the 8 corners of M volumes for one footprint and interpolates.
// Corners outside the volume read as 0 (cudaAddressModeBorder, .cu:2200-2202).
template <int M>
__device__ __forceinline__ void gather_interp(const float* const* __restrict__ vol, int nx, int ny, int nz,
                                              const Corner& c, float* out)
{
    const int nxy = nx * ny;
    const bool interior = (unsigned)c.ix < (unsigned)(nx - 1) && (unsigned)c.iy < (unsigned)(ny - 1) &&
                          (unsigned)c.iz < (unsigned)(nz - 1);
    const int base = (c.iz * ny + c.iy) * nx + c.ix;
    if (interior) {
#pragma unroll
        for (int m = 0; m < M; m++) {
            const float* __restrict__ q = vol[m] + base;
            const float v000 = __ldg(q), v100 = __ldg(q + 1);
            const float v010 = __ldg(q + nx), v110 = __ldg(q + nx + 1);
            const float v001 = __ldg(q + nxy), v101 = __ldg(q + nxy + 1);
            const float v011 = __ldg(q + nxy + nx), v111 = __ldg(q + nxy + nx + 1);
            const float a0 = lerpf(v000, v100, c.wx), a1 = lerpf(v010, v110, c.wx);
            const float a2 = lerpf(v001, v101, c.wx), a3 = lerpf(v011, v111, c.wx);
            out[m] = lerpf(lerpf(a0, a1, c.wy), lerpf(a2, a3, c.wy), c.wz);
        }
    } else {
        const bool x0 = (unsigned)c.ix < (unsigned)nx, x1 = (unsigned)(c.ix + 1) < (unsigned)nx;
        const bool y0 = (unsigned)c.iy < (unsigned)ny, y1 = (unsigned)(c.iy + 1) < (unsigned)ny;
        const bool z0 = (unsigned)c.iz < (unsigned)nz, z1 = (unsigned)(c.iz + 1) < (unsigned)nz;
#pragma unroll
        for (int m = 0; m < M; m++) {
            const float* __restrict__ q = vol[m];
            const float v000 = (x0 && y0 && z0) ? __ldg(q + base) : 0.f;
            const float v100 = (x1 && y0 && z0) ? __ldg(q + base + 1) : 0.f;
            const float v010 = (x0 && y1 && z0) ? __ldg(q + base + nx) : 0.f;
            const float v110 = (x1 && y1 && z0) ? __ldg(q + base + nx + 1) : 0.f;
            const float v001 = (x0 && y0 && z1) ? __ldg(q + base + nxy) : 0.f;
            const float v101 = (x1 && y0 && z1) ? __ldg(q + base + nxy + 1) : 0.f;
            const float v011 = (x0 && y1 && z1) ? __ldg(q + base + nxy + nx) : 0.f;
            const float v111 = (x1 && y1 && z1) ? __ldg(q + base + nxy + nx + 1) : 0.f;
            const float a0 = lerpf(v000, v100, c.wx), a1 = lerpf(v010, v110, c.wx);
            const float a2 = lerpf(v001, v101, c.wx), a3 = lerpf(v011, v111, c.wx);
            out[m] = lerpf(lerpf(a0, a1, c.wy), lerpf(a2, a3, c.wy), c.wz);
        }
    }
}

// Scatters w * g[m] into the 8 corners of M gradient volumes (transposed
// trilinear weights), skipping corners outside the volume.
template <int M>
__device__ __forceinline__ void scatter_interp(float* const* __restrict__ gvol, int nx, int ny, int nz,
                                               const Corner& c, const float* g)
{
    const int nxy = nx * ny;
    const int base = (c.iz * ny + c.iy) * nx + c.ix;
    const float ux = 1.f - c.wx, uy = 1.f - c.wy, uz = 1.f - c.wz;
    const float w[8] = {ux * uy * uz, c.wx * uy * uz, ux * c.wy * uz, c.wx * c.wy * uz,
                        ux * uy * c.wz, c.wx * uy * c.wz, ux * c.wy * c.wz, c.wx * c.wy * c.wz};
    const int off[8] = {0, 1, nx, nx + 1, nxy, nxy + 1, nxy + nx, nxy + nx + 1};
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int x = c.ix + (k & 1), y = c.iy + ((k >> 1) & 1), z = c.iz + ((k >> 2) & 1);
        if ((unsigned)x < (unsigned)nx && (unsigned)y < (unsigned)ny && (unsigned)z < (unsigned)nz) {
#pragma unroll
            for (int m = 0; m < M; m++) atomicAdd(gvol[m] + base + off[k], w[k] * g[m]);
        }
    }
}

// Compensated (Kahan) accumulation, FP32.
__device__ __forceinline__ void kahan_add(float& s, float& c, float x)
{
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

}  // namespace ctfp
