// ctfp_axis.cuh — the axis sampler's ray march (SAMPLER_AXIS), shared by the
// plan kernels (k_forward_axis) and the batched persistent kernels.
#pragma once

#include "ctfp_device.cuh"

namespace ctfp {

// Brick occupancy for empty-space skipping as a march reads it: bricks of
// 2^shift voxels per axis, occ_x x occ_y per z layer of bricks.
struct OccView {
    const uint8_t* occ;
    int occ_x, occ_y, nx, ny, nz, shift;
    // whether the footprint with base corner c can read a non-zero voxel;
    // bases outside [-1, n - 1] read only the border
    __device__ __forceinline__ bool occupied(const Corner& c) const
    {
        const unsigned x = (unsigned)(c.ix + 1), y = (unsigned)(c.iy + 1), z = (unsigned)(c.iz + 1);
        if (x > (unsigned)nx || y > (unsigned)ny || z > (unsigned)nz) return false;
        const size_t b = ((size_t)(z >> shift) * occ_y + (y >> shift)) * occ_x + (x >> shift);
        return __ldg(occ + b) != 0;
    }
};

// ---------------------------------------------------------------------------
// Axis sampler (SAMPLER_AXIS).  A view whose central ray runs mostly along x
// reads the copies layered along x (layer = x index, texel (y, z)); any other
// view reads the copies layered along y (layer = y, texel (x, z)).  A sample's
// footprint is then two 2x2 gathers, layers L and L + 1, at the in-layer base
// (a, b).  Consecutive samples lie half a voxel apart, mostly along the layer
// axis, so a sample usually has the previous sample's footprint or the same
// in-layer base one layer on.  Each ray keeps two gathers per material in
// registers, slot 0 for the even and slot 1 for the odd layer of its current
// pair, and a sample fetches only a slot whose layer or base changed: nothing,
// one layer (the other slot keeps its layer), or both when the in-layer base
// moved.  Which slot is the lower layer depends on L's parity, which selects
// the layer-axis weights rather than moving values between registers.  The
// texture unit spends its time per active quad of 4 lanes, so the lane layout
// (k_forward_axis) puts each quad on 4 adjacent detector rows of one column:
// their rays cross layer and in-layer cell boundaries at nearly the same
// samples and skip their gathers together.  The copies carry one zero layer
// before and after the volume (texture layer = layer + 1), and the unit clamps
// layer indices, so a footprint overhanging the volume reads zeros there with
// no test.

// The gathers one ray holds: the layers in slot 0 (even) and slot 1 (odd)
// and their in-layer base; the sentinel layer matches no footprint (bases are
// >= -2).  fetch() takes the next footprint (lower layer lc, in-layer base
// (a, b)), says which slots must be fetched (their texture layers are e0 + 1
// and e1 + 1: layer 0 of a copy is its zero pad) and holds the new pair.
struct AxisHold {
    int h0 = -1000000000, h1 = -1000000000, ca = 0, cb = 0;
    __device__ __forceinline__ void fetch(int lc, int a, int b, int& e0, int& e1, bool& n0, bool& n1)
    {
        const int par = lc & 1;
        e0 = lc + par;       // the even layer of {lc, lc + 1}
        e1 = lc + 1 - par;   // the odd one
        const bool base = (a == ca) & (b == cb);
        n0 = !(base & (h0 == e0));
        n1 = !(base & (h1 == e1));
        h0 = e0;
        h1 = e1;
        ca = a;
        cb = b;
    }
};

// The footprint of sample i in the axis sampler's terms: lower layer, in-layer
// base and the corner (TRILINEAR: from the stepped FP64 coordinates).
template <int MODE>
__device__ __forceinline__ Corner axis_corner(const GeomParams& g, const RayRef32& r, int i, double& cx, double& cy,
                                              double& cz, const RaySeg& s)
{
    if (MODE == INTERP_TRILINEAR) {
        const Corner c = corner_of<INTERP_TRILINEAR>(cx, cy, cz);
        cx += s.bx;
        cy += s.by;
        cz += s.bz;
        return c;
    }
    return corner_tex(ref32_coords(g, r, i));
}

// L_m for one ray with the axis sampler (AX 0: layered along x, 1: along y).
// Each ray is marched on its own (from its own first sample), so its result
// does not depend on the launch shape.  (Stepping a warp's lanes through
// common sample indices instead, from the earliest entry to the latest exit
// among them, measured 3 % slower on poly_grid_256: the extra iterations
// cost more than the gathers the tighter lockstep saves.)
template <int M, int MODE, int AX, bool SKIP>
__device__ __forceinline__ void march_ray_axis(const GeomParams& g, const cudaTextureObject_t* xtex,
                                               const cudaTextureObject_t* ytex, const OccView& occ, int p, int v,
                                               int u, float* L)
{
    const RaySeg s = ray_segment(g, p, v, u);
    RayRef32 r;
    if (MODE != INTERP_TRILINEAR) r = ray_ref32(g, p, v, u);
    const cudaTextureObject_t* tx = AX == 0 ? xtex : ytex;
    float acc[M], cmp[M];
    float4 q0[M], q1[M];  // slot 0: the even layer of the pair, slot 1: the odd one
#pragma unroll
    for (int m = 0; m < M; m++) {
        acc[m] = 0.f;
        cmp[m] = 0.f;
        q0[m] = q1[m] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    AxisHold hold;
    // FP64 coordinates stepped by one sample (c += b: within 1e-10 voxel of
    // a + b i over any ray); samples summed in blocks of kBlock in FP32, the
    // block sums compensated (Kahan)
    double cx = fma((double)s.i0, s.bx, s.ax), cy = fma((double)s.i0, s.by, s.ay), cz = fma((double)s.i0, s.bz, s.az);
    constexpr int kBlock = 16;
    for (int ib = s.i0; ib < s.i1; ib += kBlock) {
    const int ie = min(ib + kBlock, s.i1);
    float blk[M];
#pragma unroll
    for (int m = 0; m < M; m++) blk[m] = 0.f;
#pragma unroll 2
    for (int i = ib; i < ie; i++) {
        const Corner c = axis_corner<MODE>(g, r, i, cx, cy, cz, s);
        if (SKIP && !occ.occupied(c)) continue;
        const int lc = AX == 0 ? c.ix : c.iy;
        const int a = AX == 0 ? c.iy : c.ix;
        const int b = c.iz;
        const int par = lc & 1;
        int e0, e1;
        bool n0, n1;
        hold.fetch(lc, a, b, e0, e1, n0, n1);
        const float fa = small_int_to_float(a + 1), fb = small_int_to_float(b + 1);
        if (n0) {
#pragma unroll
            for (int m = 0; m < M; m++) q0[m] = gather_layer_cond(tx[m], e0 + 1, fa, fb);
        }
        if (n1) {
#pragma unroll
            for (int m = 0; m < M; m++) q1[m] = gather_layer_cond(tx[m], e1 + 1, fa, fb);
        }
        if (MODE == INTERP_TRILINEAR) {
            // weights of the lower and upper layer, assigned to the slots by
            // parity; each gather's in-layer value as a dot product with the
            // four in-layer weight products (shared by the materials and both
            // slots; tld4 order: x = (a, b+1), y = (a+1, b+1), z = (a+1, b),
            // w = (a, b)), the slots' layer weights folded into the block sum
            const float wl = AX == 0 ? c.ux : c.uy, wh = AX == 0 ? c.wx : c.wy;
            const float w0 = par ? wh : wl, w1 = par ? wl : wh;
            const float ua = AX == 0 ? c.uy : c.ux, wa = AX == 0 ? c.wy : c.wx;
            const float p00 = ua * c.uz, p10 = wa * c.uz, p01 = ua * c.wz, p11 = wa * c.wz;
#pragma unroll
            for (int m = 0; m < M; m++) {
                const float s0 = fmaf(q0[m].y, p11, fmaf(q0[m].x, p01, fmaf(q0[m].z, p10, q0[m].w * p00)));
                const float s1 = fmaf(q1[m].y, p11, fmaf(q1[m].x, p01, fmaf(q1[m].z, p10, q1[m].w * p00)));
                blk[m] = fmaf(s1, w1, fmaf(s0, w0, blk[m]));
            }
        } else {
            // the texture unit's 8 weights (k = dz*4 + dy*2 + dx); the layer
            // axis is bit 0 of k (x) or bit 1 (y); slot 0 is the lower layer
            // when par = 0
            float w[8];
            texunit_weights(c.qx, c.qy, c.qz, w);
            constexpr int lb = AX == 0 ? 1 : 2;  // the layer bit of k
            constexpr int ab = AX == 0 ? 2 : 1;  // the in-layer axis bit of k
            float g0[4], g1[4];  // weights of slot 0 / slot 1 texels (a, b), (a+1, b), (a, b+1), (a+1, b+1)
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int k = (j & 2 ? 4 : 0) + (j & 1 ? ab : 0);
                g0[j] = par ? w[k + lb] : w[k];
                g1[j] = par ? w[k] : w[k + lb];
            }
#pragma unroll
            for (int m = 0; m < M; m++) {
                float v = g0[0] * q0[m].w;
                v = fmaf(g0[1], q0[m].z, v);
                v = fmaf(g0[2], q0[m].x, v);
                v = fmaf(g0[3], q0[m].y, v);
                v = fmaf(g1[0], q1[m].w, v);
                v = fmaf(g1[1], q1[m].z, v);
                v = fmaf(g1[2], q1[m].x, v);
                v = fmaf(g1[3], q1[m].y, v);
                blk[m] += v;
            }
        }
    }
#pragma unroll
    for (int m = 0; m < M; m++) kahan_add(acc[m], cmp[m], blk[m]);
    }
#pragma unroll
    for (int m = 0; m < M; m++) L[m] = g.dx * (acc[m] - cmp[m]);
}

// The gathers the axis march of one ray issues, as the texture unit sees
// them: the warp's lanes run the march loop in step, lane k at iteration j on
// its own sample i0_k + j, and per iteration and slot the lane quads with a
// lane that fetches are counted (out[0], per material), with the lanes'
// samples (out[1], per material).  The first lane of warp_mask returns the
// warp's totals.  Same footprints and hold logic as march_ray_axis.
template <int MODE, int AX>
__device__ __forceinline__ void count_ray_axis(const GeomParams& g, int p, int v, int u, unsigned warp_mask,
                                               unsigned long long* out)
{
    const RaySeg s = ray_segment(g, p, v, u);
    RayRef32 r;
    if (MODE != INTERP_TRILINEAR) r = ray_ref32(g, p, v, u);
    const int len = s.i1 - s.i0;
    const int wlen = __reduce_max_sync(warp_mask, len > 0 ? len : 0);
    double cx = fma((double)s.i0, s.bx, s.ax), cy = fma((double)s.i0, s.by, s.ay), cz = fma((double)s.i0, s.bz, s.az);
    AxisHold hold;
    unsigned long long quads = 0, samples = 0;
    for (int j = 0; j < wlen; j++) {
        bool n0 = false, n1 = false;
        if (j < len) {
            const Corner c = axis_corner<MODE>(g, r, s.i0 + j, cx, cy, cz, s);
            int e0, e1;
            hold.fetch(AX == 0 ? c.ix : c.iy, AX == 0 ? c.iy : c.ix, c.iz, e0, e1, n0, n1);
            samples++;
        }
        // quads with a fetching lane: OR the 4 lanes of each quad onto its first lane
        unsigned b0 = __ballot_sync(warp_mask, n0), b1 = __ballot_sync(warp_mask, n1);
        b0 = (b0 | (b0 >> 1) | (b0 >> 2) | (b0 >> 3)) & 0x11111111u;
        b1 = (b1 | (b1 >> 1) | (b1 >> 2) | (b1 >> 3)) & 0x11111111u;
        quads += (unsigned long long)(__popc(b0) + __popc(b1));
    }
    samples = __reduce_add_sync(warp_mask, (unsigned)samples);
    out[0] = quads;
    out[1] = samples;
}

// ---------------------------------------------------------------------------
// Adjoint accumulators, face-expanded along the march axis.  One float4 array
// per material holds two blocks: the x-face block, cells (x, z + 1, y + 1) of
// nx x (nz + 1) x (ny + 1), then the y-face block, cells (y, z + 1, x + 1) of
// ny x (nz + 1) x (nx + 1).  Cell (layer l, in-layer base a, z base b) of a
// block holds the contributions to the 2 x 2 face of layer l with lower corner
// (a, b): components (a, b), (a + 1, b), (a, b + 1), (a + 1, b + 1).  Views
// marched along x scatter into the x-face block, the others into the y-face
// block; face_fold sums both blocks into each voxel.
__host__ __device__ __forceinline__ size_t xface_elems(int nx, int ny, int nz)
{
    return (size_t)nx * (size_t)(nz + 1) * (size_t)(ny + 1);
}
__host__ __device__ __forceinline__ size_t face_elems(int nx, int ny, int nz)
{
    return xface_elems(nx, ny, nz) + (size_t)ny * (size_t)(nz + 1) * (size_t)(nx + 1);
}
template <int AX>
__device__ __forceinline__ size_t face_index(int nx, int ny, int nz, int l, int a, int b)
{
    if (AX == 0) return ((size_t)l * (size_t)(nz + 1) + (size_t)(b + 1)) * (size_t)(ny + 1) + (size_t)(a + 1);
    return xface_elems(nx, ny, nz) +
           ((size_t)l * (size_t)(nz + 1) + (size_t)(b + 1)) * (size_t)(nx + 1) + (size_t)(a + 1);
}

// The gradient contribution of every face cell that touches voxel (x, y, z).
__device__ __forceinline__ float face_fold(const float4* __restrict__ e, int nx, int ny, int nz, int x, int y, int z)
{
    // x faces of layer x: bases (y, z), (y - 1, z), (y, z - 1), (y - 1, z - 1)
    const float4* ex = e + face_index<0>(nx, ny, nz, x, 0, 0) - (size_t)(ny + 1) - 1;  // the (a, b) = (-1, -1) cell
    const size_t row = (size_t)(ny + 1);
    const float sx = (ex[(size_t)(z + 1) * row + (y + 1)].x + ex[(size_t)(z + 1) * row + y].y) +
                     (ex[(size_t)z * row + (y + 1)].z + ex[(size_t)z * row + y].w);
    const float4* ey = e + face_index<1>(nx, ny, nz, y, 0, 0) - (size_t)(nx + 1) - 1;
    const size_t rowy = (size_t)(nx + 1);
    const float sy = (ey[(size_t)(z + 1) * rowy + (x + 1)].x + ey[(size_t)(z + 1) * rowy + x].y) +
                     (ey[(size_t)z * rowy + (x + 1)].z + ey[(size_t)z * rowy + x].w);
    return sx + sy;
}

// Adjoint of one ray's march, accumulated per face of the march axis (AX):
// the face weights a sample gives its lower layer and its upper layer are
// summed in slot 0 (the even layer of the pair) and slot 1 (the odd one), as
// the forward holds its gathers; a slot is flushed -- one 16-byte vector
// reduction per material, its sums times the ray's dLoss/dL_m -- when its
// layer or the in-layer base changes, and at the end of the ray.  Consecutive
// samples keep their base and advance a layer on every second sample or so,
// so a slot collects two or three samples per flush.  Layers and bases outside
// the volume touch no voxel and are not flushed.
template <int M, int AX>
struct AxisScatter {
    int h0 = -1000000000, h1 = -1000000000, ca = 0, cb = 0;
    float s0[4] = {0.f, 0.f, 0.f, 0.f}, s1[4] = {0.f, 0.f, 0.f, 0.f};

    __device__ __forceinline__ void flush(float4* const* __restrict__ acc, int nx, int ny, int nz, int l,
                                          const float* sv, const float* g) const
    {
        const int nl = AX == 0 ? nx : ny, na = AX == 0 ? ny : nx;
        if ((unsigned)l >= (unsigned)nl || ca < -1 || ca >= na || cb < -1 || cb >= nz) return;
        const size_t k = face_index<AX>(nx, ny, nz, l, ca, cb);
#pragma unroll
        for (int m = 0; m < M; m++) red_add_v4(acc[m] + k, sv[0] * g[m], sv[1] * g[m], sv[2] * g[m], sv[3] * g[m]);
    }

    // Moves the slots to footprint c (flushing a slot whose layer or base
    // changes); returns the parity of c's lower layer.
    __device__ __forceinline__ int step(float4* const* __restrict__ acc, int nx, int ny, int nz, const Corner& c,
                                        const float* g)
    {
        const int lc = AX == 0 ? c.ix : c.iy, a = AX == 0 ? c.iy : c.ix, b = c.iz;
        const int par = lc & 1;
        const int e0 = lc + par, e1 = lc + 1 - par;
        const bool base = (a == ca) & (b == cb);
        if (!(base & (h0 == e0))) {
            flush(acc, nx, ny, nz, h0, s0, g);
#pragma unroll
            for (int j = 0; j < 4; j++) s0[j] = 0.f;
        }
        if (!(base & (h1 == e1))) {
            flush(acc, nx, ny, nz, h1, s1, g);
#pragma unroll
            for (int j = 0; j < 4; j++) s1[j] = 0.f;
        }
        h0 = e0;
        h1 = e1;
        ca = a;
        cb = b;
        return par;
    }

    // TRILINEAR: the sample's face weights straight from its axis weights:
    // the four in-layer products (a, b), (a + 1, b), (a, b + 1), (a + 1, b + 1)
    // times the layer weight of each slot (the lower layer's in the slot of
    // its parity).  The same products as the 8 trilinear weights, with the
    // layer axis's weight applied last.
    __device__ __forceinline__ void add_trilinear(float4* const* __restrict__ acc, int nx, int ny, int nz,
                                                  const Corner& c, const float* g)
    {
        const int par = step(acc, nx, ny, nz, c, g);
        const float ua = AX == 0 ? c.uy : c.ux, wa = AX == 0 ? c.wy : c.wx;
        const float wl = AX == 0 ? c.ux : c.uy, wh = AX == 0 ? c.wx : c.wy;
        const float w0 = par ? wh : wl, w1 = par ? wl : wh;
        const float p[4] = {ua * c.uz, wa * c.uz, ua * c.wz, wa * c.wz};
#pragma unroll
        for (int j = 0; j < 4; j++) {
            s0[j] = fmaf(p[j], w0, s0[j]);
            s1[j] = fmaf(p[j], w1, s1[j]);
        }
    }

    // The sample with footprint c and its 8 transposed weights w[k]
    // (k = dz*4 + dy*2 + dx).
    __device__ __forceinline__ void add(float4* const* __restrict__ acc, int nx, int ny, int nz, const Corner& c,
                                        const float* w, const float* g)
    {
        const int par = step(acc, nx, ny, nz, c, g);
        constexpr int lb = AX == 0 ? 1 : 2;  // the layer bit of k
        constexpr int ab = AX == 0 ? 2 : 1;  // the in-layer axis bit of k
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int k = (j & 2 ? 4 : 0) + (j & 1 ? ab : 0);
            s0[j] += par ? w[k + lb] : w[k];
            s1[j] += par ? w[k] : w[k + lb];
        }
    }

    __device__ __forceinline__ void finish(float4* const* __restrict__ acc, int nx, int ny, int nz, const float* g)
    {
        flush(acc, nx, ny, nz, h0, s0, g);
        flush(acc, nx, ny, nz, h1, s1, g);
    }
};

// The 8 transposed weights of a footprint (k = dz*4 + dy*2 + dx): the
// trilinear products, or the texture unit's weights (TEXEMU).
template <int MODE>
__device__ __forceinline__ void corner_weights(const Corner& c, float* w)
{
    if (MODE == INTERP_TEXEMU) {
        texunit_weights(c.qx, c.qy, c.qz, w);
    } else {
        const float uy_uz = c.uy * c.uz, wy_uz = c.wy * c.uz, uy_wz = c.uy * c.wz, wy_wz = c.wy * c.wz;
        w[0] = c.ux * uy_uz; w[1] = c.wx * uy_uz; w[2] = c.ux * wy_uz; w[3] = c.wx * wy_uz;
        w[4] = c.ux * uy_wz; w[5] = c.wx * uy_wz; w[6] = c.ux * wy_wz; w[7] = c.wx * wy_wz;
    }
}

// The adjoint scatter of one ray: the transposed weights of the march's
// samples (FP64 coordinates for TRILINEAR, the reference's FP32 coordinates
// and the texture unit's weights otherwise) into the face accumulators of the
// view's march axis, scaled by g[m] = dLoss/dL_m times dx.  For M <= 2 the
// sample loops are unrolled by 2: the poly_grid_256 forward + adjoint step ran
// 1.0 ms and the fused step 1.6 ms faster than with them rolled; the
// 4-material adjoint of large_4mat_512 ran 2.6 % slower unrolled.
template <int M, int MODE>
__device__ __forceinline__ void scatter_ray_axis(const GeomParams& gp, float4* const* __restrict__ acc, int p, int v,
                                                 int u, const float* g, bool axis_x)
{
    const RaySeg s = ray_segment(gp, p, v, u);
    RayRef32 r;
    if (MODE != INTERP_TRILINEAR) r = ray_ref32(gp, p, v, u);
    double cx = fma((double)s.i0, s.bx, s.ax), cy = fma((double)s.i0, s.by, s.ay), cz = fma((double)s.i0, s.bz, s.az);
    float w[8];
    if (axis_x) {
        AxisScatter<M, 0> run;
#pragma unroll(M <= 2 ? 2 : 1)
        for (int i = s.i0; i < s.i1; i++) {
            const Corner c = axis_corner<MODE>(gp, r, i, cx, cy, cz, s);
            if (MODE == INTERP_TRILINEAR) {
                run.add_trilinear(acc, gp.nx, gp.ny, gp.nz, c, g);
            } else {
                corner_weights<MODE>(c, w);
                run.add(acc, gp.nx, gp.ny, gp.nz, c, w, g);
            }
        }
        run.finish(acc, gp.nx, gp.ny, gp.nz, g);
    } else {
        AxisScatter<M, 1> run;
#pragma unroll(M <= 2 ? 2 : 1)
        for (int i = s.i0; i < s.i1; i++) {
            const Corner c = axis_corner<MODE>(gp, r, i, cx, cy, cz, s);
            if (MODE == INTERP_TRILINEAR) {
                run.add_trilinear(acc, gp.nx, gp.ny, gp.nz, c, g);
            } else {
                corner_weights<MODE>(c, w);
                run.add(acc, gp.nx, gp.ny, gp.nz, c, w, g);
            }
        }
        run.finish(acc, gp.nx, gp.ny, gp.nz, g);
    }
}

// Whether view p reads the x-layered copies: its central ray (direction
// (cos th, -sin th) in the volume's x-y plane) advances at least as many x
// voxels as y voxels per step.
__device__ __forceinline__ bool axis_is_x(const GeomParams& g, int p)
{
    const double2 cs = g.trig[p];
    return fabs(cs.x) * (double)g.pSizeY >= fabs(cs.y) * (double)g.pSizeX;
}

}  // namespace ctfp
