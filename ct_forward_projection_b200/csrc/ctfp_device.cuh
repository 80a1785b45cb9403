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

#include <climits>
#include <cuda_runtime.h>
#include <stdint.h>

namespace ctfp {

enum { INTERP_TRILINEAR = 0, INTERP_TEXEMU = 1, INTERP_TEXTURE = 2 };
// Where the software samplers (TRILINEAR, TEXEMU) read their 8 corners.
// The values are those of ctfp_sampler (include/ctfp.h).
enum { SAMPLER_GLOBAL = 1, SAMPLER_LAYERED = 2, SAMPLER_BRICK = 3, SAMPLER_AXIS = 4 };
// Kernel-internal: the layered sampler with empty-space skipping.
enum { SAMPLER_LAYERED_SKIP = 16 };
constexpr int kMaxM = 4;

// Scalar geometry shared by every ray of one problem.
struct GeomParams {
    int nx, ny, nz;          // voxels
    int U, V, P;             // detector columns, rows, views
    int K;                   // samples per ray (intNum)
    float dHalfLU, dHalfLV, dSize, sod, sdd, FOVR, dx;
    float pHalfX, pHalfY, pHalfZ, pSizeX, pSizeY, pSizeZ;
    float rpSizeX, rpSizeY, rpSizeZ;  // 1 / pSize rounded to FP32 (div_rn_recip)
    const double2* trig;     // per view (cos, sin) of the FP32 view angle
    const float2* trigf;     // the same, rounded to FP32 (compat samplers)
    const float2* fspot;     // per view focal-spot offset (u, v) in mm, or null
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
    // focal-spot offset: added to the rotated y and the z coordinate
    // (transformFocalSpotKernel, CBCTPolyProjGPU.cu:1943-1944)
    double fu = 0.0, fv = 0.0;
    if (g.fspot) {
        const float2 f = g.fspot[p];
        fu = f.x;
        fv = f.y;
    }
    // tu = X cos - Y sin + pHalfX; tv = -(X sin + Y cos) + pHalfY; tw = -Z + pHalfZ
    const double ku = A * cth - B * sth, cu = -sod * cth + (double)g.pHalfX;
    const double kv = -(A * sth + B * cth), cv = sod * sth + (double)g.pHalfY + fu;
    const double kw = -C, cw = (double)g.pHalfZ + fv;
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

// The reference's own FP32 sample coordinates, for the samplers that
// reproduce its texture fetch (TEXEMU, TEXTURE): the FP32 operations of
// computeIntPointCoordinatesKernel and transformKernel
// (CBCTPolyProjGPU.cu:1813-1848, 1915-1920), with explicit IEEE intrinsics so
// every rounding is fixed, cos/sin of the FP32 view angle correctly rounded,
// and fused multiply-adds where the reference's build fuses them (determined
// from its outputs on grazing rays): detU/detV = fma(-u, dSize, dHalf - dSize/2),
// t = fma(i, dx, t0), X = fma(cosG cosB, t, -sod), tu = fma(X, c, -(Y s)) +
// pHalfX, tv = -fma(X, s, Y c) + pHalfY.  Rays that graze the volume have path
// integrals that move by percents with 1e-5-voxel coordinate changes, so only
// this arithmetic reproduces the reference's outputs there.
struct RayRef32 {
    float cgcb, cgsb, sinG;  // direction cosines (.cu:1825-1829, 1846-1848)
    float c, s;              // cos, sin of the view angle
    float t0;                // sod - FOVR + dx / 2
    float fu, fv;            // focal-spot offset of the view (0 without one), mm
};

__device__ __forceinline__ RayRef32 ray_ref32(const GeomParams& g, int p, int v, int u)
{
    const float half = __fdiv_rn(g.dSize, 2.0f);
    const float detU = __fmaf_rn(-(float)u, g.dSize, __fsub_rn(g.dHalfLU, half));
    const float detV = __fmaf_rn(-(float)v, g.dSize, __fsub_rn(g.dHalfLV, half));
    const float s2 = __fmul_rn(g.sdd, g.sdd), u2 = __fmul_rn(detU, detU), v2 = __fmul_rn(detV, detV);
    const float R = __fsqrt_rn(__fadd_rn(__fadd_rn(s2, u2), v2));
    RayRef32 r;
    r.sinG = __fdiv_rn(detV, R);
    const float cosG = __fdiv_rn(__fsqrt_rn(__fadd_rn(s2, u2)), R);
    const float sinB = __fdiv_rn(detU, R);
    const float cosB = __fdiv_rn(__fsqrt_rn(__fadd_rn(s2, v2)), R);
    r.cgcb = __fmul_rn(cosG, cosB);
    r.cgsb = __fmul_rn(cosG, sinB);
    const float2 cs = g.trigf[p];
    r.c = cs.x;
    r.s = cs.y;
    r.t0 = __fadd_rn(__fsub_rn(g.sod, g.FOVR), __fdiv_rn(g.dx, 2.0f));
    r.fu = 0.f;
    r.fv = 0.f;
    if (g.fspot) {
        const float2 f = g.fspot[p];
        r.fu = f.x;
        r.fv = f.y;
    }
    return r;
}

// x / y correctly rounded to FP32, given r = 1 / y correctly rounded to FP32
// (a per-plan constant here): two correction steps after Markstein (P. W.
// Markstein, "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Develop. 34(1), 1990; the theorem in Muller et al.,
// "Handbook of Floating-Point Arithmetic", on the correction q + (x - q y) r).
// With r within half an ulp of 1 / y, q0 = x r is within 1.5 ulp of x / y; the
// remainder x - q y is exact in one fused multiply-add, so the first step
// leaves q1 within an ulp, and from there the second step's result is the
// correctly rounded quotient (quotients and divisors away from the overflow
// and subnormal ranges).  Checked bit for bit against the IEEE division on the
// device (ctfp_check_division).
__device__ __forceinline__ float div_rn_recip(float x, float y, float r)
{
    const float q0 = __fmul_rn(x, r);
    const float q1 = __fmaf_rn(__fmaf_rn(-q0, y, x), r, q0);
    return __fmaf_rn(__fmaf_rn(-q1, y, x), r, q1);
}

// tex3D coordinates (voxel index + 0.5) of sample i.  The division by the
// voxel size is the IEEE one either way; RECIP forms it with div_rn_recip.
// Both give the same bits: the texture emulation's march runs 8.5 % faster
// with RECIP (65.5 against 71.6 ms on the 256^3 two-material grid workload),
// the hardware-texture march 3 % slower (57.2 against 55.5 ms), so the tex3D
// paths pass RECIP = false.
template <bool RECIP = true>
__device__ __forceinline__ float3 ref32_coords(const GeomParams& g, const RayRef32& r, int i)
{
    const float t = __fmaf_rn((float)i, g.dx, r.t0);
    const float X = __fmaf_rn(r.cgcb, t, -g.sod);
    const float Y = __fmul_rn(r.cgsb, t);
    const float Z = __fmul_rn(r.sinG, t);
    const float tu = __fadd_rn(__fmaf_rn(X, r.c, -__fmul_rn(Y, r.s)), g.pHalfX);
    // + the focal-spot offset, added last as in CBCTPolyProjGPU.cu:1943-1944
    // (adding 0 leaves the coordinate unchanged)
    const float tv = __fadd_rn(__fadd_rn(-__fmaf_rn(X, r.s, __fmul_rn(Y, r.c)), g.pHalfY), r.fu);
    const float tw = __fadd_rn(__fadd_rn(-Z, g.pHalfZ), r.fv);
    if (!RECIP)
        return make_float3(__fadd_rn(__fdiv_rn(tu, g.pSizeX), 0.5f), __fadd_rn(__fdiv_rn(tv, g.pSizeY), 0.5f),
                           __fadd_rn(__fdiv_rn(tw, g.pSizeZ), 0.5f));
    return make_float3(__fadd_rn(div_rn_recip(tu, g.pSizeX, g.rpSizeX), 0.5f),
                       __fadd_rn(div_rn_recip(tv, g.pSizeY, g.rpSizeY), 0.5f),
                       __fadd_rn(div_rn_recip(tw, g.pSizeZ, g.rpSizeZ), 0.5f));
}

// Trilinear footprint of one sample: base corner, the weights of the upper
// corners (w) and of the lower corners (u = 1 - w).  Both are formed before
// rounding to FP32, so a corner weight near 0 on either side keeps its
// relative accuracy (1 - w computed from a rounded w near 1 would not).
struct Corner {
    int ix, iy, iz;
    float tx, ty;    // ix + 1, iy + 1 as FP32: the gather coordinate of the layered sampler
    float wx, wy, wz;
    float ux, uy, uz;
    int qx, qy, qz;  // TEXEMU: the texture unit's 8-bit fractions (0..255)
};

// k / 256 for 0 <= k < 2^23 without a conversion instruction: the bits of
// 2^15 + k / 256 (whose ulp is 1/256) minus 2^15, both steps exact.
__device__ __forceinline__ float q8_to_float(int k) { return __int_as_float(0x47000000 + k) - 32768.0f; }

// The texture unit's 8 corner weights (in 1/256) for 8-bit fractions A (x),
// B (y), C (z), measured on the B200 with single-corner tex3D probes (exact
// over 3e4 random points): per z slice with Z = C or 256 - C, the x split
// p1 = round_half_up(A Z / 256), p0 = Z - p1; then the y split of each,
// upper-y weight round_half_up(B p1 / 256) for x = 1 and round_half_down(B p0 /
// 256) for x = 0, lower-y weight the remainder.  Weights always sum to 256.
// Index k = dz*4 + dy*2 + dx.
__device__ __forceinline__ void texunit_weights(int A, int B, int C, float* w)
{
#pragma unroll
    for (int dz = 0; dz < 2; dz++) {
        const int Z = dz ? C : 256 - C;
        const int p1 = (A * Z + 128) >> 8;
        const int p0 = Z - p1;
        const int w11 = (B * p1 + 128) >> 8;
        const int w01 = (B * p0 + 127) >> 8;
        w[dz * 4 + 0] = q8_to_float(p0 - w01);
        w[dz * 4 + 1] = q8_to_float(p1 - w11);
        w[dz * 4 + 2] = q8_to_float(w01);
        w[dz * 4 + 3] = q8_to_float(w11);
    }
}

// Interpolates the 8 corner values v[k] (k = dz*4 + dy*2 + dx).
template <int MODE>
__device__ __forceinline__ float interp8(const Corner& c, const float* v)
{
    if (MODE == 1 /* INTERP_TEXEMU */) {
        float w[8];
        texunit_weights(c.qx, c.qy, c.qz, w);
        float s = w[0] * v[0];
#pragma unroll
        for (int k = 1; k < 8; k++) s = fmaf(w[k], v[k], s);
        return s;
    }
    const float a0 = fmaf(v[1], c.wx, v[0] * c.ux), a1 = fmaf(v[3], c.wx, v[2] * c.ux);
    const float a2 = fmaf(v[5], c.wx, v[4] * c.ux), a3 = fmaf(v[7], c.wx, v[6] * c.ux);
    const float b0 = fmaf(a1, c.wy, a0 * c.uy), b1 = fmaf(a3, c.wy, a2 * c.uy);
    return fmaf(b1, c.wz, b0 * c.uz);
}

// The texture unit's fixed-point coordinate for the FP32 coordinate x handed
// to tex3D: X = round_half_up((x - 0.5) * 256); base texel X >> 8, fraction
// X & 255 in 1/256 (measured on the B200 with in-bounds tex3D sweeps and
// single-corner probes: exact over 3e5 + 3e4 points, edges included).
// x * 256 - 127.5 is exact in FP32 for |x| < 2^15.  (A round-down add of
// 1.5 * 2^23 in place of floorf and the conversion ran the texture emulation
// 1 % slower.)
__device__ __forceinline__ int tex_fixed(float x) { return (int)floorf(fmaf(x, 256.0f, -127.5f)); }

// The two weights of one axis from the exact FP64 fraction f in [0, 1): the
// smaller of f and 1 - f (both exact in FP64) is rounded once to FP32 and the
// larger is formed from it in FP32, which is accurate in absolute terms and
// so relative to a value >= 1/2.  One conversion per axis.
__device__ __forceinline__ void frac_pair(double f, float& w, float& u)
{
    const bool lo = f < 0.5;
    const float sm = (float)(lo ? f : 1.0 - f);
    const float bg = 1.0f - sm;
    w = lo ? sm : bg;
    u = lo ? bg : sm;
}

// Texture-unit footprint at the FP32 tex3D coordinate (x, y, z) = index + 0.5.
__device__ __forceinline__ Corner corner_tex(float3 x)
{
    Corner c = {};
    const int X = tex_fixed(x.x), Y = tex_fixed(x.y), Z = tex_fixed(x.z);
    c.ix = X >> 8; c.iy = Y >> 8; c.iz = Z >> 8;
    c.tx = (float)(c.ix + 1); c.ty = (float)(c.iy + 1);
    c.qx = X & 255; c.qy = Y & 255; c.qz = Z & 255;
    return c;
}

// Base index and the two weights of one axis at the FP64 coordinate x: base
// b = floor(x), fraction f = x - b, upper weight w = f and lower weight
// u = 1 - f, each rounded once from FP64 to FP32.  1 - f is exact in FP64 for
// f >= 1/2 (and within 2^-53 of the true value, near 1, otherwise), so both
// weights keep their FP32 relative accuracy however close to 0 either is.
// The floor comes from one FP64 add rounded down: x + 1.5 * 2^52 lands on the
// integer grid of that binade at 1.5 * 2^52 + floor(x) (|x| < 2^51), whose low
// word is floor(x) in two's complement and whose difference with 1.5 * 2^52
// is floor(x) exactly.  (A floor() and an add for the index ran the
// 256^3 two-material forward 4.4 % slower: 50.75 against 48.54 ms.)
__device__ __forceinline__ int axis_weights(double x, float& w, float& u)
{
    const double t = __dadd_rd(x, 6755399441055744.0);
    const double f = x - (t - 6755399441055744.0);
    w = __double2float_rn(f);
    u = __double2float_rn(1.0 - f);
    return __double2loint(t);
}

// (float)n for -3 <= n < 2^23 - 3 without a conversion instruction: the bits
// of 2^23 + (n + 3) as a float, minus 2^23 + 3 (exact).
__device__ __forceinline__ float small_int_to_float(int n)
{
    return __int_as_float(0x4B000000 | (n + 3)) - 8388611.0f;
}

// Footprint at the FP64 coordinate (cx, cy, cz).  TRILINEAR: exact fraction
// of the FP64 coordinate, rounded once to FP32 (axis_weights).  TEXEMU: the
// texture unit's fixed-point view of the FP32 coordinate float(c + 0.5) that
// tex3D receives.
template <int MODE>
__device__ __forceinline__ Corner corner_of(double cx, double cy, double cz)
{
    Corner c = {};
    if (MODE == INTERP_TRILINEAR) {
        c.ix = axis_weights(cx, c.wx, c.ux);
        c.iy = axis_weights(cy, c.wy, c.uy);
        c.iz = axis_weights(cz, c.wz, c.uz);
        c.tx = small_int_to_float(c.ix + 1); c.ty = small_int_to_float(c.iy + 1);
    } else {
        const int X = tex_fixed((float)(cx + 0.5)), Y = tex_fixed((float)(cy + 0.5)), Z = tex_fixed((float)(cz + 0.5));
        c.ix = X >> 8; c.iy = Y >> 8; c.iz = Z >> 8;
        c.qx = X & 255; c.qy = Y & 255; c.qz = Z & 255;
    }
    return c;
}


// Loads the 8 corners (k = dz*4 + dy*2 + dx) of M volumes for one footprint
// from the caller's linear volumes.  Corners outside the volume read as 0
// (cudaAddressModeBorder, CBCTPolyProjGPU.cu:2200-2202).
template <int M>
__device__ __forceinline__ void load8_global(const float* const* __restrict__ vol, int nx, int ny, int nz,
                                             const Corner& c, float (*v)[8])
{
    const int nxy = nx * ny;
    const bool interior = (unsigned)c.ix < (unsigned)(nx - 1) && (unsigned)c.iy < (unsigned)(ny - 1) &&
                          (unsigned)c.iz < (unsigned)(nz - 1);
    const int base = (c.iz * ny + c.iy) * nx + c.ix;
    if (interior) {
#pragma unroll
        for (int m = 0; m < M; m++) {
            const float* __restrict__ q = vol[m] + base;
            v[m][0] = __ldg(q); v[m][1] = __ldg(q + 1); v[m][2] = __ldg(q + nx); v[m][3] = __ldg(q + nx + 1);
            v[m][4] = __ldg(q + nxy); v[m][5] = __ldg(q + nxy + 1);
            v[m][6] = __ldg(q + nxy + nx); v[m][7] = __ldg(q + nxy + nx + 1);
        }
    } else {
        const bool x0 = (unsigned)c.ix < (unsigned)nx, x1 = (unsigned)(c.ix + 1) < (unsigned)nx;
        const bool y0 = (unsigned)c.iy < (unsigned)ny, y1 = (unsigned)(c.iy + 1) < (unsigned)ny;
        const bool z0 = (unsigned)c.iz < (unsigned)nz, z1 = (unsigned)(c.iz + 1) < (unsigned)nz;
#pragma unroll
        for (int m = 0; m < M; m++) {
            const float* __restrict__ q = vol[m];
            v[m][0] = (x0 && y0 && z0) ? __ldg(q + base) : 0.f;
            v[m][1] = (x1 && y0 && z0) ? __ldg(q + base + 1) : 0.f;
            v[m][2] = (x0 && y1 && z0) ? __ldg(q + base + nx) : 0.f;
            v[m][3] = (x1 && y1 && z0) ? __ldg(q + base + nx + 1) : 0.f;
            v[m][4] = (x0 && y0 && z1) ? __ldg(q + base + nxy) : 0.f;
            v[m][5] = (x1 && y0 && z1) ? __ldg(q + base + nxy + 1) : 0.f;
            v[m][6] = (x0 && y1 && z1) ? __ldg(q + base + nxy + nx) : 0.f;
            v[m][7] = (x1 && y1 && z1) ? __ldg(q + base + nxy + nx + 1) : 0.f;
        }
    }
}

// Loads the 8 corners and interpolates (global sampler).
template <int M, int MODE>
__device__ __forceinline__ void gather_interp(const float* const* __restrict__ vol, int nx, int ny, int nz,
                                              const Corner& c, float* out)
{
    float v[M][8];
    load8_global<M>(vol, nx, ny, nz, c, v);
#pragma unroll
    for (int m = 0; m < M; m++) out[m] = interp8<MODE>(c, v[m]);
}

// Four texels of the 2x2 footprint with lower corner (ix, iy) in one layer
// of a layered 2D texture (tld4, PTX "texture gather").  The coordinate is the
// footprint's centre, (x, y) = (ix + 1, iy + 1) (x_B = ix + 0.5), so the unit's
// own 8-bit coordinate rounding cannot move the footprint.  Returned in gather order:
// x = (ix, iy+1), y = (ix+1, iy+1), z = (ix+1, iy), w = (ix, iy).  Border
// addressing reads 0 outside the layer.
__device__ __forceinline__ float4 gather_layer(cudaTextureObject_t t, int layer, float x, float y)
{
    float4 r;
    asm("tld4.r.a2d.v4.f32.f32 {%0, %1, %2, %3}, [%4, {%5, %6, %7, %8}];"
        : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
        : "l"(t), "r"(layer), "f"(x), "f"(y), "f"(y));
    return r;
}

// gather_layer for gathers issued under a condition: a volatile asm is not
// executed more often than the source says, so the compiler cannot turn the
// conditional gather into an unconditional one plus a select (which would
// spend the texture unit's time on every lane, the work a skipped gather saves).
__device__ __forceinline__ float4 gather_layer_cond(cudaTextureObject_t t, int layer, float x, float y)
{
    float4 r;
    asm volatile("tld4.r.a2d.v4.f32.f32 {%0, %1, %2, %3}, [%4, {%5, %6, %7, %8}];"
                 : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
                 : "l"(t), "r"(layer), "f"(x), "f"(y), "f"(y));
    return r;
}

// The 8 corners of M volumes held as layered 2D textures (one layer per z
// slice): two gathers per material.  Layers outside [0, nz) read as 0 here,
// since layer indices are clamped, not bordered, by the unit.
template <int M>
__device__ __forceinline__ void load8_layered(const cudaTextureObject_t* ltex, int nz, const Corner& c, float (*v)[8])
{
    const bool z0ok = (unsigned)c.iz < (unsigned)nz, z1ok = (unsigned)(c.iz + 1) < (unsigned)nz;
    const int l0 = z0ok ? c.iz : 0, l1 = z1ok ? c.iz + 1 : 0;
#pragma unroll
    for (int m = 0; m < M; m++) {
        float4 a = gather_layer(ltex[m], l0, c.tx, c.ty);
        float4 b = gather_layer(ltex[m], l1, c.tx, c.ty);
        if (!z0ok) a = make_float4(0.f, 0.f, 0.f, 0.f);
        if (!z1ok) b = make_float4(0.f, 0.f, 0.f, 0.f);
        v[m][0] = a.w; v[m][1] = a.z; v[m][2] = a.x; v[m][3] = a.y;
        v[m][4] = b.w; v[m][5] = b.z; v[m][6] = b.x; v[m][7] = b.y;
    }
}

// Loads the 8 corners and interpolates (layered sampler).
template <int M, int MODE>
__device__ __forceinline__ void gather4_interp(const cudaTextureObject_t* ltex, int nz, const Corner& c, float* out)
{
    float v[M][8];
    load8_layered<M>(ltex, nz, c, v);
#pragma unroll
    for (int m = 0; m < M; m++) out[m] = interp8<MODE>(c, v[m]);
}

// One 16-byte vector reduction into global memory (the adjoint's accumulators).
__device__ __forceinline__ void red_add_v4(float4* p, float a, float b, float c, float d)
{
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a), "f"(b), "f"(c), "f"(d)
                 : "memory");
}


// exp(-a) and 1 - exp(-a), each to a few ulp relative.  For |a| < 1/4 the
// absorbed fraction is the Taylor series 1 - exp(-a) = a (1 - a/2 + a^2/6 -
// a^3/24 + a^4/120 - a^5/720 + a^6/5040), whose first omitted term is below
// 2e-9 of it, so a thin ray's absorption keeps its relative accuracy, and the
// transmission is its complement; otherwise the transmission is
// exp2f(-a log2 e) and the absorption its complement, at most a factor 4.5 of
// cancellation.  Every spectral epilogue (plan forward, batch, no-allocation
// forward) uses this one function.
__device__ __forceinline__ void transmit(float a, float& ex, float& om)
{
    if (fabsf(a) < 0.25f) {
        float q = fmaf(a, 1.0f / 5040.0f, -1.0f / 720.0f);
        q = fmaf(a, q, 1.0f / 120.0f);
        q = fmaf(a, q, -1.0f / 24.0f);
        q = fmaf(a, q, 1.0f / 6.0f);
        q = fmaf(a, q, -0.5f);
        q = fmaf(a, q, 1.0f);
        om = a * q;
        ex = 1.0f - om;
    } else {
        ex = exp2f(a * -1.44269504088896341f);
        om = 1.0f - ex;
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

// K2: I = sum_e W_e exp(-sum_m mu_em L_m), IAbs = sum_e W_e (1 - exp(...)).
// The energy sums are split over 4 accumulators (energy e into e mod 4) and
// combined pairwise: each takes about E / 4 positive terms, so the sum's
// relative rounding error stays below (E / 4 + 2) ulp with one fused
// multiply-add per term and output.
template <int M>
__device__ __forceinline__ void spectral_term(const float* s_mu, int e, const float* __restrict__ Wp, int64_t npix,
                                              const float* L, float& sI, float& sA)
{
    float att = 0.f;
#pragma unroll
    for (int m = 0; m < M; m++) att = fmaf(s_mu[e * M + m], L[m], att);
    const float w = __ldg(Wp + (int64_t)e * npix);
    float ex, om;
    transmit(att, ex, om);
    sI = fmaf(w, ex, sI);
    sA = fmaf(w, om, sA);
}

template <int M>
__device__ __forceinline__ void spectral(const float* s_mu, int E, const float* __restrict__ W, int64_t pix,
                                         int64_t npix, const float* L, float& I, float& IAbs)
{
    float sI[4] = {0.f, 0.f, 0.f, 0.f}, sA[4] = {0.f, 0.f, 0.f, 0.f};
    const float* Wp = W + pix;
    int e = 0;
    // 8 energies per step (8 table loads in flight; 0.5 % of the 256^3
    // two-material forward against 4), accumulator k & 3 taking energy e + k:
    // every accumulator sums the same energies in the same order as with
    // steps of 4, so the sums do not change
    for (; e + 8 <= E; e += 8) {
#pragma unroll
        for (int k = 0; k < 8; k++) spectral_term<M>(s_mu, e + k, Wp, npix, L, sI[k & 3], sA[k & 3]);
    }
    for (; e + 4 <= E; e += 4) {
#pragma unroll
        for (int k = 0; k < 4; k++) spectral_term<M>(s_mu, e + k, Wp, npix, L, sI[k], sA[k]);
    }
    for (; e < E; e++) spectral_term<M>(s_mu, e, Wp, npix, L, sI[0], sA[0]);
    I = (sI[0] + sI[1]) + (sI[2] + sI[3]);
    IAbs = (sA[0] + sA[1]) + (sA[2] + sA[3]);
}

// The fused forward + loss + adjoint's epilogue: I as spectral() forms it
// (the same terms in the same order, so the batch's I equals the plain
// forward's), and S_m = sum_e mu_em W_e exp(-a_e), the derivative -dI/dL_m.
template <int M>
__device__ __forceinline__ void spectral_adjoint_term(const float* s_mu, int e, const float* __restrict__ Wp,
                                                      int64_t npix, const float* L, float& sI, float* S)
{
    float att = 0.f;
#pragma unroll
    for (int m = 0; m < M; m++) att = fmaf(s_mu[e * M + m], L[m], att);
    const float w = __ldg(Wp + (int64_t)e * npix);
    float ex, om;
    transmit(att, ex, om);
    sI = fmaf(w, ex, sI);
    const float Ie = w * ex;
#pragma unroll
    for (int m = 0; m < M; m++) S[m] = fmaf(s_mu[e * M + m], Ie, S[m]);
}

template <int M>
__device__ __forceinline__ void spectral_adjoint(const float* s_mu, int E, const float* __restrict__ W, int64_t pix,
                                                 int64_t npix, const float* L, float& I, float* S)
{
    float sI[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int m = 0; m < M; m++) S[m] = 0.f;
    const float* Wp = W + pix;
    int e = 0;
    // the steps of spectral(): the same order for sI, and S in energy order
    for (; e + 8 <= E; e += 8) {
#pragma unroll
        for (int k = 0; k < 8; k++) spectral_adjoint_term<M>(s_mu, e + k, Wp, npix, L, sI[k & 3], S);
    }
    for (; e + 4 <= E; e += 4) {
#pragma unroll
        for (int k = 0; k < 4; k++) spectral_adjoint_term<M>(s_mu, e + k, Wp, npix, L, sI[k], S);
    }
    for (; e < E; e++) spectral_adjoint_term<M>(s_mu, e, Wp, npix, L, sI[0], S);
    I = (sI[0] + sI[1]) + (sI[2] + sI[3]);
}

}  // namespace ctfp
