// ctfp_kernels.cu — the march kernels (K1 ray march fused with the K2
// spectral epilogue), the adjoint scatter, and small helper kernels.
//
// K1+K2 replaces, for every (view, pixel) ray, the reference's
//   transformKernel (CBCTPolyProjGPU.cu:1902-1924)  K*U*V samples to HBM per view
//   forward*Kernel  (CBCTPolyProjGPU.cu:1980-2169)  per-ray sum + Beer-Lambert per energy
//   host energy loop (CBCTPolyForwardProjGrid.cpp:159-177, CBCTForwardProj.cpp:65-76)
// with one pass: samples stay in registers, each material is marched once for
// all energies (sum_m mu[e][m] * L_m equals the reference's per-energy
// mu_E-volume integral because trilinear interpolation is linear in the voxel
// values), and the energy sum runs on the device in compensated FP32.
#include <cuda.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "ctfp_axis.cuh"
#include "ctfp_kernels.cuh"

namespace ctfp {

namespace {

template <int M, int SAMPLER>
__device__ __forceinline__ void load_corners(const MarchParams& prm, const Corner& c, float (*v)[8])
{
    if (SAMPLER == SAMPLER_LAYERED || SAMPLER == SAMPLER_LAYERED_SKIP) load8_layered<M>(prm.ltex, prm.g.nz, c, v);
    else load8_global<M>(prm.vol, prm.g.nx, prm.g.ny, prm.g.nz, c, v);
}

// Whether the footprint with base corner c can read a non-zero voxel (brick
// occupancy); bases outside [-1, n - 1] read only the border.
__device__ __forceinline__ bool footprint_occupied(const MarchParams& prm, const Corner& c)
{
    const unsigned x = (unsigned)(c.ix + 1), y = (unsigned)(c.iy + 1), z = (unsigned)(c.iz + 1);
    if (x > (unsigned)prm.g.nx || y > (unsigned)prm.g.ny || z > (unsigned)prm.g.nz) return false;
    const size_t b = ((size_t)(z >> kOccShift) * prm.occ_y + (y >> kOccShift)) * prm.occ_x + (x >> kOccShift);
    return __ldg(prm.occ + b) != 0;
}

// One sample of a software-interpolated march: fetch the footprint,
// interpolate, accumulate.  With empty-space skipping, a footprint inside an
// all-zero brick contributes exactly zero and is not fetched.
template <int M, int MODE, int SAMPLER>
__device__ __forceinline__ void sample_acc(const MarchParams& prm, const Corner& c, float* acc, float* cmp)
{
    if (SAMPLER == SAMPLER_LAYERED_SKIP && !footprint_occupied(prm, c)) return;
    float v[M][8];
    load_corners<M, SAMPLER>(prm, c, v);
#pragma unroll
    for (int m = 0; m < M; m++) kahan_add(acc[m], cmp[m], interp8<MODE>(c, v[m]));
}

// L_m for one ray, compensated FP32 sum times dx.  TRILINEAR samples at FP64
// coordinates; the compat samplers at the reference's FP32 coordinates.
template <int M, int MODE, int SAMPLER>
__device__ __forceinline__ void march_ray(const MarchParams& prm, int p, int v, int u, float* L)
{
    const RaySeg s = ray_segment(prm.g, p, v, u);
    float acc[M], cmp[M];
#pragma unroll
    for (int m = 0; m < M; m++) { acc[m] = 0.f; cmp[m] = 0.f; }
    if (MODE == INTERP_TRILINEAR) {
#pragma unroll 2
        for (int i = s.i0; i < s.i1; i++) {
            const double t = (double)i;
            sample_acc<M, MODE, SAMPLER>(
                prm, corner_of<INTERP_TRILINEAR>(fma(t, s.bx, s.ax), fma(t, s.by, s.ay), fma(t, s.bz, s.az)), acc, cmp);
        }
    } else if (MODE == INTERP_TEXTURE) {
        // the reference's own fetch: tex3D on a border/linear texture
        const RayRef32 r = ray_ref32(prm.g, p, v, u);
#pragma unroll 2
        for (int i = s.i0; i < s.i1; i++) {
            const float3 x = ref32_coords<false>(prm.g, r, i);
            // with empty-space skipping: the unit's own footprint (base texel
            // of its fixed-point coordinate) in an all-zero brick filters to 0
            if (SAMPLER == SAMPLER_LAYERED_SKIP && !footprint_occupied(prm, corner_tex(x))) continue;
#pragma unroll
            for (int m = 0; m < M; m++) kahan_add(acc[m], cmp[m], tex3D<float>(prm.tex[m], x.x, x.y, x.z));
        }
    } else {
        const RayRef32 r = ray_ref32(prm.g, p, v, u);
#pragma unroll 2
        for (int i = s.i0; i < s.i1; i++) sample_acc<M, MODE, SAMPLER>(prm, corner_tex(ref32_coords(prm.g, r, i)), acc, cmp);
    }
#pragma unroll
    for (int m = 0; m < M; m++) L[m] = prm.g.dx * (acc[m] - cmp[m]);
}

__device__ __forceinline__ void load_mu(float* s_mu, const float* mu, int n)
{
    const int nt = blockDim.x * blockDim.y;
    for (int k = threadIdx.y * blockDim.x + threadIdx.x; k < n; k += nt) s_mu[k] = mu[k];
    __syncthreads();
}

template <int M>
__device__ __forceinline__ void store_L(float* L, int64_t ray, const float* l)
{
    float* q = L + ray * M;
    if (M == 4) {
        *reinterpret_cast<float4*>(q) = make_float4(l[0], l[1], l[2], l[3]);
    } else if (M == 2) {
        *reinterpret_cast<float2*>(q) = make_float2(l[0], l[1]);
    } else {
#pragma unroll
        for (int m = 0; m < M; m++) q[m] = l[m];
    }
}

template <int M>
__device__ __forceinline__ void load_L(const float* L, int64_t ray, float* l)
{
    const float* q = L + ray * M;
    if (M == 4) {
        const float4 a = *reinterpret_cast<const float4*>(q);
        l[0] = a.x; l[1] = a.y; l[2] = a.z; l[3] = a.w;
    } else if (M == 2) {
        const float2 a = *reinterpret_cast<const float2*>(q);
        l[0] = a.x; l[1] = a.y;
    } else {
#pragma unroll
        for (int m = 0; m < M; m++) l[m] = q[m];
    }
}

// K1+K2. Grid: x = pixel tiles along u, y = along v, z = view groups.
template <int M, int MODE, int SAMPLER, bool SPECTRAL, int MINB>
__global__ void __launch_bounds__(256, MINB) k_forward(const MarchParams prm)
{
    extern __shared__ float s_mu[];
    if (SPECTRAL) load_mu(s_mu, prm.mu, prm.E * M);
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y * blockDim.y + threadIdx.y;
    if (u >= prm.g.U || v >= prm.g.V) return;
    const int64_t npix = (int64_t)prm.g.U * prm.g.V;
    const int64_t pix = (int64_t)v * prm.g.U + u;
    const int pend = prm.view0 + prm.n_views;
    for (int k = 0; k < prm.views_per_cta; k++) {
        const int p = prm.view0 + blockIdx.z * prm.views_per_cta + k;
        if (p >= pend) break;
        float L[M];
        march_ray<M, MODE, SAMPLER>(prm, p, v, u, L);
        const int64_t ray = (int64_t)(p - prm.out_view0) * npix + pix;
        if (prm.L) store_L<M>(prm.L, ray, L);
        if (SPECTRAL) {
            float I, A;
            spectral<M>(s_mu, prm.E, prm.W, pix, npix, L, I, A);
            if (prm.I) prm.I[ray] = I;
            if (prm.IAbs) prm.IAbs[ray] = A;
        }
    }
}

// K1+K2 with the axis sampler.  One-dimensional CTAs of tile_u * tile_v
// threads (tile_v a multiple of 4) cover a tile_u x tile_v pixel tile: lane
// quads run down 4 detector rows of one column, so a warp covers 8 columns x
// 4 rows.  Grid: x = pixel tiles along u, y = along v, z = view groups.
template <int M, int MODE, bool SKIP, bool SPECTRAL, int MINB>
__global__ void __launch_bounds__(256, MINB) k_forward_axis(const MarchParams prm, int tile_u, int warp_rows)
{
    extern __shared__ float s_mu[];
    if (SPECTRAL) load_mu(s_mu, prm.mu, prm.E * M);
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int tile_v = (int)blockDim.x / tile_u;
    // a warp covers wcols columns x warp_rows rows, lane quads down 4 rows
    const int wcols = 32 / warp_rows, warps_u = tile_u / wcols;
    const int col = (lane >> 2) % wcols, row = 4 * ((lane >> 2) / wcols) + (lane & 3);
    const int u = blockIdx.x * tile_u + (w % warps_u) * wcols + col;
    const int v = blockIdx.y * tile_v + (w / warps_u) * warp_rows + row;
    if (u >= prm.g.U || v >= prm.g.V) return;
    const int64_t npix = (int64_t)prm.g.U * prm.g.V;
    const int64_t pix = (int64_t)v * prm.g.U + u;
    const int pend = prm.view0 + prm.n_views;
    for (int k = 0; k < prm.views_per_cta; k++) {
        const int p = prm.view0 + blockIdx.z * prm.views_per_cta + k;
        if (p >= pend) break;
        float L[M];
        const OccView ov{prm.occ, prm.occ_x, prm.occ_y, prm.g.nx, prm.g.ny, prm.g.nz, kOccShift};
        if (axis_is_x(prm.g, p)) march_ray_axis<M, MODE, 0, SKIP>(prm.g, prm.xtex, prm.ytex, ov, p, v, u, L);
        else march_ray_axis<M, MODE, 1, SKIP>(prm.g, prm.xtex, prm.ytex, ov, p, v, u, L);
        const int64_t ray = (int64_t)(p - prm.out_view0) * npix + pix;
        if (prm.L) store_L<M>(prm.L, ray, L);
        if (SPECTRAL) {
            float I, A;
            spectral<M>(s_mu, prm.E, prm.W, pix, npix, L, I, A);
            if (prm.I) prm.I[ray] = I;
            if (prm.IAbs) prm.IAbs[ray] = A;
        }
    }
}

// Texture quad-gathers of the axis march (count_ray_axis) over every view,
// with k_forward_axis's CTA tile and lane layout; out[0] += quads, out[1] +=
// samples.  Grid: x = pixel tiles along u, y = along v, z = views.
template <int MODE>
__global__ void __launch_bounds__(256) k_axis_gather_count(const GeomParams g, int tile_u, int warp_rows,
                                                           unsigned long long* out)
{
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int tile_v = (int)blockDim.x / tile_u;
    const int wcols = 32 / warp_rows, warps_u = tile_u / wcols;
    const int col = (lane >> 2) % wcols, row = 4 * ((lane >> 2) / wcols) + (lane & 3);
    const int u = blockIdx.x * tile_u + (w % warps_u) * wcols + col;
    const int v = blockIdx.y * tile_v + (w / warps_u) * warp_rows + row;
    const bool valid = u < g.U && v < g.V;
    const unsigned warp_mask = __ballot_sync(0xffffffffu, valid);
    if (!valid) return;
    const int p = blockIdx.z;
    unsigned long long r[2];
    if (axis_is_x(g, p)) count_ray_axis<MODE, 0>(g, p, v, u, warp_mask, r);
    else count_ray_axis<MODE, 1>(g, p, v, u, warp_mask, r);
    if (lane == __ffs(warp_mask) - 1) {
        atomicAdd(out, r[0]);
        atomicAdd(out + 1, r[1]);
    }
}

// The x- and y-layered copies of one volume, through a 32 x 32 (x, y) tile
// of one z slice in shared memory so that both copies are written along their
// texel rows; voxel layer l is texture layer l + 1 (layer 0 and the last
// layer are zeros, k_axis_zero_layers).  Block (32, 8); grid (ceil(nx / 32),
// ceil(ny / 32), nz).
__global__ void __launch_bounds__(256) k_axis_fill(const float* __restrict__ vol, int nx, int ny,
                                                   cudaSurfaceObject_t xs, cudaSurfaceObject_t ys)
{
    __shared__ float t[32][33];
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32, z = blockIdx.z;
    const int tx = threadIdx.x;
    for (int ty = threadIdx.y; ty < 32; ty += 8) {
        const int x = x0 + tx, y = y0 + ty;
        t[ty][tx] = (x < nx && y < ny) ? __ldg(vol + ((size_t)z * ny + y) * nx + x) : 0.f;
    }
    __syncthreads();
    for (int ty = threadIdx.y; ty < 32; ty += 8) {
        {
            const int x = x0 + tx, y = y0 + ty;  // y-layered: layer y, texel (x, z)
            if (x < nx && y < ny) surf2DLayeredwrite(t[ty][tx], ys, x * (int)sizeof(float), z, y + 1);
        }
        {
            const int y = y0 + tx, x = x0 + ty;  // x-layered: layer x, texel (y, z)
            if (x < nx && y < ny) surf2DLayeredwrite(t[tx][ty], xs, y * (int)sizeof(float), z, x + 1);
        }
    }
}

// Zeros texture layer `layer` (width x height texels) of a layered surface.
__global__ void k_axis_zero_layer(cudaSurfaceObject_t sf, int width, int height, int layer)
{
    const int n = width * height;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        surf2DLayeredwrite(0.0f, sf, (k % width) * (int)sizeof(float), k / width, layer);
}

template <int M>
__global__ void __launch_bounds__(256) k_spectral_from_L(const MarchParams prm)
{
    extern __shared__ float s_mu[];
    load_mu(s_mu, prm.mu, prm.E * M);
    const int64_t npix = (int64_t)prm.g.U * prm.g.V;
    const int64_t nray = npix * prm.g.P;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x * blockDim.y;
    for (int64_t ray = (int64_t)blockIdx.x * blockDim.x * blockDim.y + threadIdx.y * blockDim.x + threadIdx.x;
         ray < nray; ray += stride) {
        float L[M];
        load_L<M>(prm.Lin, ray, L);
        float I, A;
        spectral<M>(s_mu, prm.E, prm.W, ray % npix, npix, L, I, A);
        if (prm.I) prm.I[ray] = I;
        if (prm.IAbs) prm.IAbs[ray] = A;
    }
}

// Adjoint: spectral-weight recompute from the checkpoint, then the matched
// ray march scattering the transposed trilinear weights with vector
// reductions.  FROM_GL: the input is dLoss/dL directly (transpose of the line
// integrals).
//
// Grid: x = pixel tiles along u, y = view groups, z = pixel tiles along v, so
// that the CTAs resident at any time cover one band of detector rows for many
// views.  The rays of a row band cross a thin z-slab of the volume (the cone
// angle is small), so the accumulator cells they reduce into stay in L2; with
// views outermost every view would sweep the whole accumulator through DRAM.
// Register cap for 4 CTAs of 256 threads (64 registers, ~40 B of spills): the
// poly_grid_256 adjoint 0.8 ms faster than at 3 CTAs (76 registers, none).
template <int M, int MODE, bool FROM_GL>
__global__ void __launch_bounds__(256, 4) k_backward(const MarchParams prm)
{
    extern __shared__ float s_mu[];
    if (!FROM_GL) load_mu(s_mu, prm.mu, prm.E * M);
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.z * blockDim.y + threadIdx.y;
    if (u >= prm.g.U || v >= prm.g.V) return;
    const int64_t npix = (int64_t)prm.g.U * prm.g.V;
    const int64_t pix = (int64_t)v * prm.g.U + u;
    const int pend = prm.view0 + prm.n_views;
    for (int k = 0; k < prm.views_per_cta; k++) {
        const int p = prm.view0 + blockIdx.y * prm.views_per_cta + k;
        if (p >= pend) break;
        const int64_t ray = (int64_t)(p - prm.out_view0) * npix + pix;
        float g[M];
        if (FROM_GL) {
            load_L<M>(prm.Lin, ray, g);
#pragma unroll
            for (int m = 0; m < M; m++) g[m] *= prm.g.dx;
        } else {
            float L[M], S[M];
            load_L<M>(prm.Lin, ray, L);
#pragma unroll
            for (int m = 0; m < M; m++) S[m] = 0.f;
            // the spectral weights as the forward formed them (transmit, the
            // same order), so S matches the fused kernels' exactly
            for (int e = 0; e < prm.E; e++) {
                float att = 0.f;
#pragma unroll
                for (int m = 0; m < M; m++) att = fmaf(s_mu[e * M + m], L[m], att);
                float ex, om;
                transmit(att, ex, om);
                const float Ie = __ldg(prm.W + (int64_t)e * npix + pix) * ex;
#pragma unroll
                for (int m = 0; m < M; m++) S[m] = fmaf(s_mu[e * M + m], Ie, S[m]);
            }
            const float gd = ((prm.gIAbs ? prm.gIAbs[ray] : 0.f) - (prm.gI ? prm.gI[ray] : 0.f)) * prm.g.dx;
#pragma unroll
            for (int m = 0; m < M; m++) g[m] = gd * S[m];
        }
        bool any = false;
#pragma unroll
        for (int m = 0; m < M; m++) any |= (g[m] != 0.f);
        if (!any) continue;
        // the transposed weights of the forward's sampler (for the texture
        // modes, the texture unit's, at the reference's FP32 coordinates)
        scatter_ray_axis<M, MODE == INTERP_TRILINEAR ? INTERP_TRILINEAR : INTERP_TEXEMU>(
            prm.g, prm.gexp, p, v, u, g, axis_is_x(prm.g, p));
    }
}

// Sums the face accumulators of both march axes into the gradient volumes
// (face_fold).  One streaming pass.
template <int M>
__global__ void k_fold(const MarchParams prm)
{
    const int nx = prm.g.nx, ny = prm.g.ny, nz = prm.g.nz;
    const int64_t n = (int64_t)nx * ny * nz;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(k % nx), y = (int)((k / nx) % ny), z = (int)(k / ((int64_t)nx * ny));
#pragma unroll
        for (int m = 0; m < M; m++) prm.gvol[m][k] += face_fold(prm.gexp[m], nx, ny, nz, x, y, z);
    }
}

// W[e][k] = ((I0Val * S_e) * G_e) * D_e in the reference's multiplication order
// (CBCTPolyProjGPU.cu:1994); I0[k] = the sum over e (CBCTPolyForwardProjGrid.cpp:330-339).
__global__ void k_weights(const float* __restrict__ S, const float* __restrict__ G, int grid_layout,
                          const float* __restrict__ D, float I0Val, int E, int U, int V, float* W, float* I0)
{
    const int64_t npix = (int64_t)U * V;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < npix; k += (int64_t)gridDim.x * blockDim.x) {
        const int u = (int)(k % U);
        // the spectral epilogue's summation order (energy e into accumulator
        // e mod 4, E rounded down to a multiple of 4 first, the rest into
        // accumulator 0, combined pairwise), so that a ray with no attenuation
        // gives exactly I0
        float s[4] = {0.f, 0.f, 0.f, 0.f};
        const int E4 = E & ~3;
        for (int e = 0; e < E; e++) {
            float w = I0Val * S[e];
            if (grid_layout == 1) w = w * G[(int64_t)e * U + u];
            if (grid_layout == 2) w = w * G[(int64_t)e * npix + k];
            if (D) w = w * D[(int64_t)e * npix + k];
            W[(int64_t)e * npix + k] = w;
            const int a = e < E4 ? (e & 3) : 0;
            if (a == 0) s[0] += w;
            else if (a == 1) s[1] += w;
            else if (a == 2) s[2] += w;
            else s[3] += w;
        }
        I0[k] = (s[0] + s[1]) + (s[2] + s[3]);
    }
}

// Ipoly = (uint32)floorf(I); proj = logf(I0 / Ipoly) (CBCTForwardProj.cpp:79-90, 376-387).
__global__ void k_finalize(int64_t n_pix, int64_t n, const float* __restrict__ I, const float* __restrict__ IAbs,
                           const float* __restrict__ I0, uint32_t* Ipoly, uint32_t* IAbsPoly, float* proj)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        if (I) {
            const uint32_t ip = (uint32_t)floorf(I[k]);
            if (Ipoly) Ipoly[k] = ip;
            if (proj && I0) proj[k] = logf(I0[k % n_pix] / (float)ip);
        }
        if (IAbs && IAbsPoly) IAbsPoly[k] = (uint32_t)floorf(IAbs[k]);
    }
}

__global__ void k_sample_points(const float* vol, cudaTextureObject_t tex, int nx, int ny, int nz, int interp,
                                const float* pts, int64_t n, float* out)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const double cx = pts[3 * k], cy = pts[3 * k + 1], cz = pts[3 * k + 2];
        float val;
        if (interp == INTERP_TEXTURE) {
            val = tex3D<float>(tex, (float)(cx + 0.5), (float)(cy + 0.5), (float)(cz + 0.5));
        } else {
            const float* vp[1] = {vol};
            if (interp == INTERP_TEXEMU)
                gather_interp<1, INTERP_TEXEMU>(vp, nx, ny, nz, corner_of<INTERP_TEXEMU>(cx, cy, cz), &val);
            else
                gather_interp<1, INTERP_TRILINEAR>(vp, nx, ny, nz, corner_of<INTERP_TRILINEAR>(cx, cy, cz), &val);
        }
        out[k] = val;
    }
}

// Exact count of samples whose trilinear footprint touches the volume.
__global__ void k_count_support(const GeomParams g, unsigned long long* out)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y * blockDim.y + threadIdx.y;
    unsigned long long n = 0;
    if (u < g.U && v < g.V) {
        for (int p = blockIdx.z; p < g.P; p += gridDim.z) {
            const RaySeg s = ray_segment(g, p, v, u);
            for (int i = s.i0; i < s.i1; i++) {
                const double t = (double)i;
                const double cx = fma(t, s.bx, s.ax), cy = fma(t, s.by, s.ay), cz = fma(t, s.bz, s.az);
                n += (cx > -1.0 && cy > -1.0 && cz > -1.0 && cx < (double)g.nx && cy < (double)g.ny &&
                      cz < (double)g.nz);
            }
        }
    }
    // warp reduce then one atomic per warp
    for (int o = 16; o > 0; o >>= 1) n += __shfl_down_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, n);
}

// ---------------------------------------------------------------------------
// Brick sampler: the CTA stages, for every segment of kBS consecutive samples,
// the box of voxels its ray bundle crosses in shared memory, and each sample
// reads its 8 corners from there (LDS) instead of through the texture unit.
// Rays of one CTA step through the same sample indices, so at any index their
// samples lie on a small patch: kBU x kBV rays about one voxel apart, swept
// kBS/2 voxels along the rays per segment.  The box origin and fit are
// computed per segment from the rays' first and last footprints (FP64
// coordinates are affine in the sample index, so their floors are monotone;
// the FP32 compat coordinates get a one-voxel margin).  A segment whose box
// does not fit, and any sample outside the box, reads the caller's volume
// instead, so the result never depends on the fit.
constexpr int kBU = 8, kBV = 16;             // rays per CTA: u x v
constexpr int kBX = 16, kBY = 16, kBZ = 20;  // box, voxels
constexpr int kBXp = 17;                     // row pitch (floats)
constexpr int kBZp = 296;                    // slice pitch: 17 * 16 + 24 = 8 (mod 32 banks)
constexpr int kBS = 16;                      // samples per segment
constexpr int kBoxFloats = kBZp * kBZ;       // one material's box

template <int MODE>
__device__ __forceinline__ Corner corner_at(const MarchParams& prm, const RaySeg& s, const RayRef32& r, int i)
{
    if (MODE == INTERP_TRILINEAR) {
        const double t = (double)i;
        return corner_of<INTERP_TRILINEAR>(fma(t, s.bx, s.ax), fma(t, s.by, s.ay), fma(t, s.bz, s.az));
    }
    return corner_tex(ref32_coords(prm.g, r, i));
}

template <int M, int MODE, bool SPECTRAL, int MINB>
__global__ void __launch_bounds__(kBU * kBV, MINB) k_forward_brick(const MarchParams prm)
{
    extern __shared__ float smem[];
    float* s_box = smem;                   // [M][kBZ][kBY][kBXp] (slices kBZp apart)
    float* s_mu = smem + M * kBoxFloats;   // [E][M]
    __shared__ int s_red[8];
    if (SPECTRAL) load_mu(s_mu, prm.mu, prm.E * M);
    const int tid = threadIdx.y * kBU + threadIdx.x;
    const int u = blockIdx.x * kBU + threadIdx.x;
    const int v = blockIdx.y * kBV + threadIdx.y;
    const bool live = u < prm.g.U && v < prm.g.V;
    const int64_t npix = (int64_t)prm.g.U * prm.g.V;
    const int64_t pix = (int64_t)v * prm.g.U + u;
    const int pend = prm.view0 + prm.n_views;
    constexpr int margin = MODE == INTERP_TRILINEAR ? 0 : 1;
    for (int k = 0; k < prm.views_per_cta; k++) {
        const int p = prm.view0 + blockIdx.z * prm.views_per_cta + k;
        if (p >= pend) break;
        RaySeg s;
        s.i0 = s.i1 = 0;
        if (live) s = ray_segment(prm.g, p, v, u);
        RayRef32 r;
        if (MODE != INTERP_TRILINEAR && live) r = ray_ref32(prm.g, p, v, u);
        if (tid == 0) {
            s_red[0] = INT_MAX;
            s_red[1] = INT_MIN;
        }
        __syncthreads();
        if (s.i1 > s.i0) {
            atomicMin(&s_red[0], s.i0);
            atomicMax(&s_red[1], s.i1);
        }
        __syncthreads();
        const int I0 = s_red[0], I1 = s_red[1];
        __syncthreads();
        float acc[M], cmp[M];
#pragma unroll
        for (int m = 0; m < M; m++) { acc[m] = 0.f; cmp[m] = 0.f; }
        for (int seg = I0; seg < I1; seg += kBS) {
            const int a0 = max(seg, s.i0), a1 = min(min(seg + kBS, I1), s.i1);
            if (tid == 0) {
                s_red[0] = s_red[1] = s_red[2] = INT_MAX;
                s_red[3] = s_red[4] = s_red[5] = INT_MIN;
            }
            __syncthreads();
            if (a0 < a1) {
                const Corner c0 = corner_at<MODE>(prm, s, r, a0), c1 = corner_at<MODE>(prm, s, r, a1 - 1);
                atomicMin(&s_red[0], min(c0.ix, c1.ix) - margin);
                atomicMin(&s_red[1], min(c0.iy, c1.iy) - margin);
                atomicMin(&s_red[2], min(c0.iz, c1.iz) - margin);
                atomicMax(&s_red[3], max(c0.ix, c1.ix) + margin);
                atomicMax(&s_red[4], max(c0.iy, c1.iy) + margin);
                atomicMax(&s_red[5], max(c0.iz, c1.iz) + margin);
            }
            __syncthreads();
            const int ox = s_red[0], oy = s_red[1], oz = s_red[2];
            const bool fits = s_red[3] >= ox && s_red[3] + 1 - ox < kBX && s_red[4] + 1 - oy < kBY &&
                              s_red[5] + 1 - oz < kBZ;
            if (fits) {
                // stage the box; voxels outside the volume read as 0 (border)
                const int nx = prm.g.nx, ny = prm.g.ny, nz = prm.g.nz;
                for (int idx = tid; idx < kBX * kBY * kBZ; idx += kBU * kBV) {
                    const int x = idx % kBX, y = (idx / kBX) % kBY, z = idx / (kBX * kBY);
                    const int gx = ox + x, gy = oy + y, gz = oz + z;
                    const bool in = (unsigned)gx < (unsigned)nx && (unsigned)gy < (unsigned)ny &&
                                    (unsigned)gz < (unsigned)nz;
                    const int64_t off = ((int64_t)gz * ny + gy) * nx + gx;
                    const int so = z * kBZp + y * kBXp + x;
#pragma unroll
                    for (int m = 0; m < M; m++) s_box[m * kBoxFloats + so] = in ? __ldg(prm.vol[m] + off) : 0.f;
                }
            }
            __syncthreads();
            for (int i = a0; i < a1; i++) {
                const Corner c = corner_at<MODE>(prm, s, r, i);
                const int bx = c.ix - ox, by = c.iy - oy, bz = c.iz - oz;
                float cv[M][8];
                if (fits && (unsigned)bx < (unsigned)(kBX - 1) && (unsigned)by < (unsigned)(kBY - 1) &&
                    (unsigned)bz < (unsigned)(kBZ - 1)) {
                    const int b = bz * kBZp + by * kBXp + bx;
#pragma unroll
                    for (int m = 0; m < M; m++) {
                        const float* q = s_box + m * kBoxFloats + b;
                        cv[m][0] = q[0]; cv[m][1] = q[1]; cv[m][2] = q[kBXp]; cv[m][3] = q[kBXp + 1];
                        cv[m][4] = q[kBZp]; cv[m][5] = q[kBZp + 1]; cv[m][6] = q[kBZp + kBXp];
                        cv[m][7] = q[kBZp + kBXp + 1];
                    }
                } else {
                    load8_global<M>(prm.vol, prm.g.nx, prm.g.ny, prm.g.nz, c, cv);
                }
#pragma unroll
                for (int m = 0; m < M; m++) kahan_add(acc[m], cmp[m], interp8<MODE>(c, cv[m]));
            }
            __syncthreads();
        }
        if (!live) continue;
        float L[M];
#pragma unroll
        for (int m = 0; m < M; m++) L[m] = prm.g.dx * (acc[m] - cmp[m]);
        const int64_t ray = (int64_t)(p - prm.out_view0) * npix + pix;
        if (prm.L) store_L<M>(prm.L, ray, L);
        if (SPECTRAL) {
            float I, A;
            spectral<M>(s_mu, prm.E, prm.W, pix, npix, L, I, A);
            if (prm.I) prm.I[ray] = I;
            if (prm.IAbs) prm.IAbs[ray] = A;
        }
    }
}

// ---------------------------------------------------------------------------
// Brick sampler with TMA staging: the same boxes, the same fit rule and the
// same reads as k_forward_brick, but each box is one tensor load per material
// (cp.async.bulk.tensor.3d, issued by one thread, completion counted on an
// mbarrier) instead of 128 threads' scalar loads.  The box's x origin is
// rounded down to a multiple of 4 voxels, because a tiled tensor load must
// start on a 16-byte boundary in x, so kTX = 16 + 3 + 1 columns are staged;
// y and z start at the box origin, and voxels outside the volume (negative or
// past the end) arrive as zeros, the texture border.  The dense box layout is
// the one TMA writes: rows of kTX floats, slices of kTX * kBY floats.
//
// Every wait is bounded: thread 0 issues, all threads poll the mbarrier at
// most prm.wait_limit times; when any gives up, the CTA reads that segment and
// all later ones from the volume (same results), ors kCtfpStatusWaitTimeout
// into the plan's status word, and before exiting waits, again bounded, for
// the load still in flight so that it cannot land in shared memory the CTA no
// longer owns; when that exit wait runs out as well, it ors
// kCtfpStatusExitWaitTimeout, an error (outputs not trusted).
constexpr int kTX = 20;
constexpr int kTRow = kTX, kTSlice = kTX * kBY;
constexpr int kTBoxFloats = kTSlice * kBZ;  // 6400 floats = 25600 bytes, a multiple of 128
constexpr int kExitPolls = 1 << 22;

struct BrickMaps {
    CUtensorMap tm[kMaxM];
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded poll of one mbarrier phase; true when it completed.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int limit)
{
    for (int k = 0; k < limit; k++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tma_load_box(float* dst, const CUtensorMap* tm, int x, int y, int z, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

template <int M, int MODE, bool SPECTRAL, int MINB>
__global__ void __launch_bounds__(kBU * kBV, MINB)
    k_forward_brick_tma(const MarchParams prm, const __grid_constant__ BrickMaps maps)
{
    extern __shared__ unsigned char smem_raw[];
    float* s_box = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    float* s_mu = s_box + M * kTBoxFloats;  // [E][M]
    __shared__ int s_red[8];
    __shared__ __align__(8) uint64_t s_bar;
    const int tid = threadIdx.y * kBU + threadIdx.x;
    if (tid == 0) mbar_init(&s_bar, 1);
    if (SPECTRAL) load_mu(s_mu, prm.mu, prm.E * M);
    __syncthreads();
    uint32_t phase = 0;
    bool staging = true;   // CTA-uniform: false once a wait ran out
    bool in_flight = false;  // CTA-uniform: a load whose completion was not seen
    const int u = blockIdx.x * kBU + threadIdx.x;
    const int v = blockIdx.y * kBV + threadIdx.y;
    const bool live = u < prm.g.U && v < prm.g.V;
    const int64_t npix = (int64_t)prm.g.U * prm.g.V;
    const int64_t pix = (int64_t)v * prm.g.U + u;
    const int pend = prm.view0 + prm.n_views;
    constexpr int margin = MODE == INTERP_TRILINEAR ? 0 : 1;
    for (int k = 0; k < prm.views_per_cta; k++) {
        const int p = prm.view0 + blockIdx.z * prm.views_per_cta + k;
        if (p >= pend) break;
        RaySeg s;
        s.i0 = s.i1 = 0;
        if (live) s = ray_segment(prm.g, p, v, u);
        RayRef32 r;
        if (MODE != INTERP_TRILINEAR && live) r = ray_ref32(prm.g, p, v, u);
        if (tid == 0) {
            s_red[0] = INT_MAX;
            s_red[1] = INT_MIN;
        }
        __syncthreads();
        if (s.i1 > s.i0) {
            atomicMin(&s_red[0], s.i0);
            atomicMax(&s_red[1], s.i1);
        }
        __syncthreads();
        const int I0 = s_red[0], I1 = s_red[1];
        __syncthreads();
        float acc[M], cmp[M];
#pragma unroll
        for (int m = 0; m < M; m++) { acc[m] = 0.f; cmp[m] = 0.f; }
        for (int seg = I0; seg < I1; seg += kBS) {
            const int a0 = max(seg, s.i0), a1 = min(min(seg + kBS, I1), s.i1);
            if (tid == 0) {
                s_red[0] = s_red[1] = s_red[2] = INT_MAX;
                s_red[3] = s_red[4] = s_red[5] = INT_MIN;
            }
            __syncthreads();
            if (a0 < a1) {
                const Corner c0 = corner_at<MODE>(prm, s, r, a0), c1 = corner_at<MODE>(prm, s, r, a1 - 1);
                atomicMin(&s_red[0], min(c0.ix, c1.ix) - margin);
                atomicMin(&s_red[1], min(c0.iy, c1.iy) - margin);
                atomicMin(&s_red[2], min(c0.iz, c1.iz) - margin);
                atomicMax(&s_red[3], max(c0.ix, c1.ix) + margin);
                atomicMax(&s_red[4], max(c0.iy, c1.iy) + margin);
                atomicMax(&s_red[5], max(c0.iz, c1.iz) + margin);
            }
            __syncthreads();
            const int ox = s_red[0], oy = s_red[1], oz = s_red[2];
            bool fits = staging && s_red[3] >= ox && s_red[3] + 1 - ox < kBX && s_red[4] + 1 - oy < kBY &&
                        s_red[5] + 1 - oz < kBZ;
            const int ox4 = ox & ~3;  // floor to a multiple of 4: the load starts on a 16-byte boundary
            if (fits) {
                if (tid == 0) {
                    mbar_expect_tx(&s_bar, (uint32_t)(M * kTBoxFloats * sizeof(float)));
#pragma unroll
                    for (int m = 0; m < M; m++) tma_load_box(s_box + m * kTBoxFloats, &maps.tm[m], ox4, oy, oz, &s_bar);
                }
                const bool done = mbar_wait_bounded(&s_bar, phase, prm.wait_limit);
                if (__syncthreads_and(done)) {
                    phase ^= 1u;
                } else {
                    // give up staging in this CTA; the load may still land
                    staging = false;
                    in_flight = true;
                    fits = false;
                    if (tid == 0 && prm.status) atomicOr(prm.status, kCtfpStatusWaitTimeout);
                }
            }
            const int dxa = ox - ox4;
            for (int i = a0; i < a1; i++) {
                const Corner c = corner_at<MODE>(prm, s, r, i);
                const int bx = c.ix - ox, by = c.iy - oy, bz = c.iz - oz;
                float cv[M][8];
                if (fits && (unsigned)bx < (unsigned)(kBX - 1) && (unsigned)by < (unsigned)(kBY - 1) &&
                    (unsigned)bz < (unsigned)(kBZ - 1)) {
                    const int b = bz * kTSlice + by * kTRow + bx + dxa;
#pragma unroll
                    for (int m = 0; m < M; m++) {
                        const float* q = s_box + m * kTBoxFloats + b;
                        cv[m][0] = q[0]; cv[m][1] = q[1]; cv[m][2] = q[kTRow]; cv[m][3] = q[kTRow + 1];
                        cv[m][4] = q[kTSlice]; cv[m][5] = q[kTSlice + 1]; cv[m][6] = q[kTSlice + kTRow];
                        cv[m][7] = q[kTSlice + kTRow + 1];
                    }
                } else {
                    load8_global<M>(prm.vol, prm.g.nx, prm.g.ny, prm.g.nz, c, cv);
                }
#pragma unroll
                for (int m = 0; m < M; m++) kahan_add(acc[m], cmp[m], interp8<MODE>(c, cv[m]));
            }
            __syncthreads();  // the box is read; the next segment may overwrite it
        }
        if (!live) continue;
        float L[M];
#pragma unroll
        for (int m = 0; m < M; m++) L[m] = prm.g.dx * (acc[m] - cmp[m]);
        const int64_t ray = (int64_t)(p - prm.out_view0) * npix + pix;
        if (prm.L) store_L<M>(prm.L, ray, L);
        if (SPECTRAL) {
            float I, A;
            spectral<M>(s_mu, prm.E, prm.W, pix, npix, L, I, A);
            if (prm.I) prm.I[ray] = I;
            if (prm.IAbs) prm.IAbs[ray] = A;
        }
    }
    // a load given up on may still be writing the box: wait for it (bounded)
    // before the CTA's shared memory is released; if that wait runs out too,
    // the copy may land in shared memory another CTA then owns, which the
    // plan's status word reports as an error (kCtfpStatusExitWaitTimeout)
    if (in_flight) {
        const bool landed = mbar_wait_bounded(&s_bar, phase, kExitPolls);
        if (!landed && tid == 0 && prm.status) atomicOr(prm.status, kCtfpStatusExitWaitTimeout);
    }
}

// The dynamic shared-memory opt-in is per device and per kernel; plans on
// other threads may get here at the same time (setting it twice is harmless).
template <typename K>
cudaError_t opt_in_smem(K kernel, std::atomic<unsigned long long>& done)
{
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && (done.load() >> dev & 1ull)) return cudaSuccess;
    const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e == cudaSuccess && dev < 64) done.fetch_or(1ull << dev);
    return e;
}

template <int M, int MODE, bool SPEC>
cudaError_t brick_launch(const MarchParams& prm, const BrickMaps* maps, dim3 grid, size_t smem_loads, size_t smem_tma,
                         cudaStream_t st)
{
    static std::atomic<unsigned long long> set_loads{0}, set_tma{0};
    if (maps) {
        const cudaError_t e = opt_in_smem(k_forward_brick_tma<M, MODE, SPEC, 4>, set_tma);
        if (e != cudaSuccess) return e;
        k_forward_brick_tma<M, MODE, SPEC, 4><<<grid, dim3(kBU, kBV), smem_tma, st>>>(prm, *maps);
    } else {
        const cudaError_t e = opt_in_smem(k_forward_brick<M, MODE, SPEC, 4>, set_loads);
        if (e != cudaSuccess) return e;
        k_forward_brick<M, MODE, SPEC, 4><<<grid, dim3(kBU, kBV), smem_loads, st>>>(prm);
    }
    return cudaGetLastError();
}

template <int M>
cudaError_t brick_dispatch(const MarchParams& prm, int interp, bool spec, const BrickMaps* maps, dim3 grid,
                           size_t smem_loads, size_t smem_tma, cudaStream_t st)
{
    if (interp == INTERP_TRILINEAR)
        return spec ? brick_launch<M, INTERP_TRILINEAR, true>(prm, maps, grid, smem_loads, smem_tma, st)
                    : brick_launch<M, INTERP_TRILINEAR, false>(prm, maps, grid, smem_loads, smem_tma, st);
    if (interp == INTERP_TEXEMU)
        return spec ? brick_launch<M, INTERP_TEXEMU, true>(prm, maps, grid, smem_loads, smem_tma, st)
                    : brick_launch<M, INTERP_TEXEMU, false>(prm, maps, grid, smem_loads, smem_tma, st);
    return cudaErrorInvalidValue;
}

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
// (no link-time dependency on libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled()
{
    static std::once_flag once;
    static EncodeTiledFn fn = nullptr;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(f);
    });
    return fn;
}

// Tensor maps of the M volumes for the TMA-staged boxes, when the volumes
// allow them: rows of a multiple of 16 bytes (pNumX % 4 == 0) and every base
// address on a 16-byte boundary.  False: stage with plain loads.
bool brick_maps(const MarchParams& prm, int M, BrickMaps& bm)
{
    const char* mode = std::getenv("CTFP_BRICK_STAGING");
    if (mode && std::strcmp(mode, "loads") == 0) return false;
    const EncodeTiledFn fn = encode_tiled();
    if (!fn) return false;
    const int nx = prm.g.nx, ny = prm.g.ny, nz = prm.g.nz;
    if (nx % 4 != 0) return false;
    std::memset(&bm, 0, sizeof(bm));
    for (int m = 0; m < M; m++) {
        if (reinterpret_cast<uintptr_t>(prm.vol[m]) % 16 != 0) return false;
        const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
        const cuuint64_t strides[2] = {(cuuint64_t)nx * sizeof(float), (cuuint64_t)nx * ny * sizeof(float)};
        const cuuint32_t box[3] = {(cuuint32_t)kTX, (cuuint32_t)kBY, (cuuint32_t)kBZ};
        const cuuint32_t estride[3] = {1, 1, 1};
        if (fn(&bm.tm[m], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(prm.vol[m]), dims, strides, box,
               estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    }
    return true;
}

template <int M, int MODE, int SAMPLER, int MINB>
cudaError_t fwd_launch(const MarchParams& prm, bool spec, dim3 grid, dim3 block, size_t smem, cudaStream_t st)
{
    if (spec) k_forward<M, MODE, SAMPLER, true, MINB><<<grid, block, smem, st>>>(prm);
    else k_forward<M, MODE, SAMPLER, false, MINB><<<grid, block, 0, st>>>(prm);
    return cudaGetLastError();
}

template <int M, int MODE, int SAMPLER>
cudaError_t fwd_dispatch_spec(const MarchParams& prm, bool spec, int minb, dim3 grid, dim3 block, size_t smem,
                              cudaStream_t st)
{
    switch (minb) {
        case 3: return fwd_launch<M, MODE, SAMPLER, 3>(prm, spec, grid, block, smem, st);
        case 4:
        case 5: return fwd_launch<M, MODE, SAMPLER, 4>(prm, spec, grid, block, smem, st);
        default: return fwd_launch<M, MODE, SAMPLER, 2>(prm, spec, grid, block, smem, st);
    }
}

template <int M>
cudaError_t fwd_dispatch_mode(const MarchParams& prm, int interp, int sampler, bool spec, int minb, dim3 grid,
                              dim3 block, size_t smem, cudaStream_t st)
{
    const bool lay = sampler == SAMPLER_LAYERED;
    switch (interp) {
        case INTERP_TRILINEAR:
            if (lay && prm.occ)
                return fwd_dispatch_spec<M, INTERP_TRILINEAR, SAMPLER_LAYERED_SKIP>(prm, spec, minb, grid, block, smem, st);
            return lay ? fwd_dispatch_spec<M, INTERP_TRILINEAR, SAMPLER_LAYERED>(prm, spec, minb, grid, block, smem, st)
                       : fwd_dispatch_spec<M, INTERP_TRILINEAR, SAMPLER_GLOBAL>(prm, spec, minb, grid, block, smem, st);
        case INTERP_TEXEMU:
            if (lay && prm.occ)
                return fwd_dispatch_spec<M, INTERP_TEXEMU, SAMPLER_LAYERED_SKIP>(prm, spec, minb, grid, block, smem, st);
            return lay ? fwd_dispatch_spec<M, INTERP_TEXEMU, SAMPLER_LAYERED>(prm, spec, minb, grid, block, smem, st)
                       : fwd_dispatch_spec<M, INTERP_TEXEMU, SAMPLER_GLOBAL>(prm, spec, minb, grid, block, smem, st);
        case INTERP_TEXTURE:
            if (prm.occ)
                return fwd_dispatch_spec<M, INTERP_TEXTURE, SAMPLER_LAYERED_SKIP>(prm, spec, minb, grid, block, smem, st);
            return fwd_dispatch_spec<M, INTERP_TEXTURE, SAMPLER_GLOBAL>(prm, spec, minb, grid, block, smem, st);
    }
    return cudaErrorInvalidValue;
}

// Rows of the detector a warp of the axis kernel covers (32 / rows columns):
// 8 rows x 4 columns measured 1-2 % faster than 4 x 8 and 16 x 2 on
// poly_grid_256 (53.6 against 54.1 and 54.5 ms).
constexpr int kAxisWarpRows = 8;

template <int M, int MODE, bool SKIP, int MINB>
cudaError_t axis_launch(const MarchParams& prm, bool spec, int tile_u, dim3 grid, dim3 block, size_t smem,
                        cudaStream_t st)
{
    int wr = kAxisWarpRows;
    const int tile_v = (int)block.x / tile_u;
    if (tile_u % (32 / wr) != 0 || tile_v % wr != 0) wr = 4;
    if (spec) k_forward_axis<M, MODE, SKIP, true, MINB><<<grid, block, smem, st>>>(prm, tile_u, wr);
    else k_forward_axis<M, MODE, SKIP, false, MINB><<<grid, block, 0, st>>>(prm, tile_u, wr);
    return cudaGetLastError();
}

template <int M, int MODE, bool SKIP>
cudaError_t axis_dispatch_minb(const MarchParams& prm, bool spec, int minb, int tile_u, dim3 grid, dim3 block,
                               size_t smem, cudaStream_t st)
{
    switch (minb) {
        case 3: return axis_launch<M, MODE, SKIP, 3>(prm, spec, tile_u, grid, block, smem, st);
        case 4: return axis_launch<M, MODE, SKIP, 4>(prm, spec, tile_u, grid, block, smem, st);
        case 5: return axis_launch<M, MODE, SKIP, 5>(prm, spec, tile_u, grid, block, smem, st);
        default: return axis_launch<M, MODE, SKIP, 2>(prm, spec, tile_u, grid, block, smem, st);
    }
}

template <int M>
cudaError_t axis_dispatch(const MarchParams& prm, int interp, bool spec, int minb, int tile_u, dim3 grid,
                          dim3 block, size_t smem, cudaStream_t st)
{
    const bool skip = prm.occ != nullptr;
    if (interp == INTERP_TRILINEAR)
        return skip ? axis_dispatch_minb<M, INTERP_TRILINEAR, true>(prm, spec, minb, tile_u, grid, block, smem, st)
                    : axis_dispatch_minb<M, INTERP_TRILINEAR, false>(prm, spec, minb, tile_u, grid, block, smem, st);
    if (interp == INTERP_TEXEMU)
        return skip ? axis_dispatch_minb<M, INTERP_TEXEMU, true>(prm, spec, minb, tile_u, grid, block, smem, st)
                    : axis_dispatch_minb<M, INTERP_TEXEMU, false>(prm, spec, minb, tile_u, grid, block, smem, st);
    return cudaErrorInvalidValue;
}

template <int M>
cudaError_t bwd_dispatch(const MarchParams& prm, int interp, bool from_gL, dim3 grid, dim3 block, size_t smem,
                         cudaStream_t st)
{
    const bool tri = interp == INTERP_TRILINEAR;
    if (from_gL) {
        if (tri) k_backward<M, INTERP_TRILINEAR, true><<<grid, block, 0, st>>>(prm);
        else k_backward<M, INTERP_TEXEMU, true><<<grid, block, 0, st>>>(prm);
    } else {
        if (tri) k_backward<M, INTERP_TRILINEAR, false><<<grid, block, smem, st>>>(prm);
        else k_backward<M, INTERP_TEXEMU, false><<<grid, block, smem, st>>>(prm);
    }
    return cudaGetLastError();
}

dim3 march_grid(const MarchParams& prm, const LaunchShape& ls)
{
    return dim3((prm.g.U + ls.tile_u - 1) / ls.tile_u, (prm.g.V + ls.tile_v - 1) / ls.tile_v,
                (prm.n_views + ls.views_per_cta - 1) / ls.views_per_cta);
}

}  // namespace

namespace {

// One launch over prm.n_views views (at most 65535 view groups: grid.z).
cudaError_t launch_forward_once(const MarchParams& prm, int M, int interp, int sampler, bool do_spectral,
                                const LaunchShape& ls, cudaStream_t st)
{
    if (sampler == SAMPLER_BRICK && interp != INTERP_TEXTURE) {
        const dim3 grid((prm.g.U + kBU - 1) / kBU, (prm.g.V + kBV - 1) / kBV,
                        (prm.n_views + ls.views_per_cta - 1) / ls.views_per_cta);
        if (grid.z == 0) return cudaSuccess;
        const size_t mu_floats = do_spectral ? (size_t)prm.E * M : 0;
        const size_t smem = sizeof(float) * ((size_t)M * kBoxFloats + mu_floats);
        const size_t smem_tma = 128 + sizeof(float) * ((size_t)M * kTBoxFloats + mu_floats);  // + alignment slack
        BrickMaps bm;
        const BrickMaps* maps = brick_maps(prm, M, bm) ? &bm : nullptr;
        switch (M) {
            case 1: return brick_dispatch<1>(prm, interp, do_spectral, maps, grid, smem, smem_tma, st);
            case 2: return brick_dispatch<2>(prm, interp, do_spectral, maps, grid, smem, smem_tma, st);
            case 3: return brick_dispatch<3>(prm, interp, do_spectral, maps, grid, smem, smem_tma, st);
            case 4: return brick_dispatch<4>(prm, interp, do_spectral, maps, grid, smem, smem_tma, st);
        }
        return cudaErrorInvalidValue;
    }
    if (sampler == SAMPLER_AXIS && interp != INTERP_TEXTURE) {
        // lane quads run down 4 detector rows and a warp covers 8 columns:
        // tiles whose height is not a multiple of 4, or whose width is not a
        // multiple of 8, use 16 x 16
        LaunchShape as = ls;
        if (as.tile_v % 4 != 0 || as.tile_u % 8 != 0 || as.tile_u * as.tile_v > 256 ||
            (as.tile_u * as.tile_v) % 32 != 0) {
            as.tile_u = 16;
            as.tile_v = 16;
        }
        const dim3 block(as.tile_u * as.tile_v), grid = march_grid(prm, as);
        const size_t smem = do_spectral ? sizeof(float) * (size_t)prm.E * M : 0;
        if (grid.x == 0 || grid.y == 0 || grid.z == 0) return cudaSuccess;
        switch (M) {
            case 1: return axis_dispatch<1>(prm, interp, do_spectral, as.min_ctas, as.tile_u, grid, block, smem, st);
            case 2: return axis_dispatch<2>(prm, interp, do_spectral, as.min_ctas, as.tile_u, grid, block, smem, st);
            case 3: return axis_dispatch<3>(prm, interp, do_spectral, as.min_ctas, as.tile_u, grid, block, smem, st);
            case 4: return axis_dispatch<4>(prm, interp, do_spectral, as.min_ctas, as.tile_u, grid, block, smem, st);
        }
        return cudaErrorInvalidValue;
    }
    const dim3 block(ls.tile_u, ls.tile_v), grid = march_grid(prm, ls);
    const size_t smem = do_spectral ? sizeof(float) * (size_t)prm.E * M : 0;
    if (grid.x == 0 || grid.y == 0 || grid.z == 0) return cudaSuccess;
    switch (M) {
        case 1: return fwd_dispatch_mode<1>(prm, interp, sampler, do_spectral, ls.min_ctas, grid, block, smem, st);
        case 2: return fwd_dispatch_mode<2>(prm, interp, sampler, do_spectral, ls.min_ctas, grid, block, smem, st);
        case 3: return fwd_dispatch_mode<3>(prm, interp, sampler, do_spectral, ls.min_ctas, grid, block, smem, st);
        case 4: return fwd_dispatch_mode<4>(prm, interp, sampler, do_spectral, ls.min_ctas, grid, block, smem, st);
    }
    return cudaErrorInvalidValue;
}

}  // namespace

cudaError_t launch_forward(const MarchParams& prm_in, int M, int interp, int sampler, bool do_spectral,
                           const LaunchShape& ls, cudaStream_t st)
{
    // view groups run along grid.z, at most 65535 per launch
    const int vpc = ls.views_per_cta;
    const int max_views = 65535 * vpc;
    for (int v0 = 0; v0 < prm_in.n_views; v0 += max_views) {
        MarchParams prm = prm_in;
        prm.views_per_cta = vpc;
        prm.view0 = prm_in.view0 + v0;
        prm.n_views = std::min(max_views, prm_in.n_views - v0);
        const cudaError_t e = launch_forward_once(prm, M, interp, sampler, do_spectral, ls, st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_axis_gather_count(const GeomParams& g, int interp, const LaunchShape& ls, unsigned long long* out,
                                     cudaStream_t st)
{
    LaunchShape as = ls;
    if (as.tile_v % 4 != 0 || as.tile_u % 8 != 0 || as.tile_u * as.tile_v > 256 || (as.tile_u * as.tile_v) % 32 != 0) {
        as.tile_u = 16;
        as.tile_v = 16;
    }
    int wr = kAxisWarpRows;
    if (as.tile_u % (32 / wr) != 0 || as.tile_v % wr != 0) wr = 4;
    for (int p0 = 0; p0 < g.P; p0 += 65535) {
        GeomParams gv = g;
        const int n = std::min(65535, g.P - p0);
        gv.trig = g.trig + p0;  // views p0 .. p0 + n - 1 as views 0 .. n - 1
        gv.trigf = g.trigf + p0;
        if (g.fspot) gv.fspot = g.fspot + p0;
        gv.P = n;
        const dim3 grid((g.U + as.tile_u - 1) / as.tile_u, (g.V + as.tile_v - 1) / as.tile_v, n);
        if (interp == INTERP_TRILINEAR) k_axis_gather_count<INTERP_TRILINEAR><<<grid, as.tile_u * as.tile_v, 0, st>>>(gv, as.tile_u, wr, out);
        else k_axis_gather_count<INTERP_TEXEMU><<<grid, as.tile_u * as.tile_v, 0, st>>>(gv, as.tile_u, wr, out);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_axis_zero_pads(int nx, int ny, int nz, cudaSurfaceObject_t xs, cudaSurfaceObject_t ys,
                                  cudaStream_t st)
{
    // x-layered: texels (y, z), layers 0 and nx + 1; y-layered: texels (x, z), layers 0 and ny + 1
    k_axis_zero_layer<<<64, 256, 0, st>>>(xs, ny, nz, 0);
    k_axis_zero_layer<<<64, 256, 0, st>>>(xs, ny, nz, nx + 1);
    k_axis_zero_layer<<<64, 256, 0, st>>>(ys, nx, nz, 0);
    k_axis_zero_layer<<<64, 256, 0, st>>>(ys, nx, nz, ny + 1);
    return cudaGetLastError();
}

cudaError_t launch_axis_fill(const float* vol, int nx, int ny, int nz, cudaSurfaceObject_t xs, cudaSurfaceObject_t ys,
                             cudaStream_t st)
{
    const dim3 grid((nx + 31) / 32, (ny + 31) / 32, nz);
    if (grid.x == 0 || grid.y == 0 || grid.z == 0) return cudaSuccess;
    k_axis_fill<<<grid, dim3(32, 8), 0, st>>>(vol, nx, ny, xs, ys);
    return cudaGetLastError();
}

cudaError_t launch_spectral_from_L(const MarchParams& prm, int M, cudaStream_t st)
{
    const dim3 block(256, 1);
    const int64_t nray = (int64_t)prm.g.U * prm.g.V * prm.g.P;
    int64_t nb = (nray + 255) / 256;
    if (nb > 148 * 64) nb = 148 * 64;
    if (nb == 0) return cudaSuccess;
    const size_t smem = sizeof(float) * (size_t)prm.E * M;
    switch (M) {
        case 1: k_spectral_from_L<1><<<(unsigned)nb, block, smem, st>>>(prm); break;
        case 2: k_spectral_from_L<2><<<(unsigned)nb, block, smem, st>>>(prm); break;
        case 3: k_spectral_from_L<3><<<(unsigned)nb, block, smem, st>>>(prm); break;
        case 4: k_spectral_from_L<4><<<(unsigned)nb, block, smem, st>>>(prm); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_backward(const MarchParams& prm_in, int M, int interp, bool from_gL, const LaunchShape& ls,
                            cudaStream_t st)
{
    const dim3 block(ls.tile_u, ls.tile_v);
    const size_t smem = sizeof(float) * (size_t)prm_in.E * M;
    // row bands outermost (grid.z), views in grid.y: at most 65535 view
    // groups per launch
    const int vpc = ls.views_per_cta;
    const int max_views = 65535 * vpc;
    for (int v0 = 0; v0 < prm_in.n_views; v0 += max_views) {
        MarchParams prm = prm_in;
        prm.views_per_cta = vpc;
        prm.view0 = prm_in.view0 + v0;
        prm.n_views = std::min(max_views, prm_in.n_views - v0);
        const dim3 grid((prm.g.U + ls.tile_u - 1) / ls.tile_u, (prm.n_views + vpc - 1) / vpc,
                        (prm.g.V + ls.tile_v - 1) / ls.tile_v);
        if (grid.x == 0 || grid.y == 0 || grid.z == 0) return cudaSuccess;
        cudaError_t e = cudaErrorInvalidValue;
        switch (M) {
            case 1: e = bwd_dispatch<1>(prm, interp, from_gL, grid, block, smem, st); break;
            case 2: e = bwd_dispatch<2>(prm, interp, from_gL, grid, block, smem, st); break;
            case 3: e = bwd_dispatch<3>(prm, interp, from_gL, grid, block, smem, st); break;
            case 4: e = bwd_dispatch<4>(prm, interp, from_gL, grid, block, smem, st); break;
        }
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

size_t expanded_elems(const GeomParams& g) { return face_elems(g.nx, g.ny, g.nz); }

cudaError_t launch_fold(const MarchParams& prm, int M, cudaStream_t st)
{
    const int64_t n = (int64_t)prm.g.nx * prm.g.ny * prm.g.nz;
    int64_t nb = (n + 255) / 256;
    if (nb > 148 * 16) nb = 148 * 16;
    switch (M) {
        case 1: k_fold<1><<<(unsigned)nb, 256, 0, st>>>(prm); break;
        case 2: k_fold<2><<<(unsigned)nb, 256, 0, st>>>(prm); break;
        case 3: k_fold<3><<<(unsigned)nb, 256, 0, st>>>(prm); break;
        case 4: k_fold<4><<<(unsigned)nb, 256, 0, st>>>(prm); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_weights(const float* spectrum, const float* grid, int grid_layout, const float* det, float I0Val,
                           int E, int U, int V, float* W, float* I0, cudaStream_t st)
{
    const int64_t npix = (int64_t)U * V;
    int64_t nb = (npix + 255) / 256;
    if (nb > 148 * 32) nb = 148 * 32;
    if (nb == 0) return cudaSuccess;
    k_weights<<<(unsigned)nb, 256, 0, st>>>(spectrum, grid, grid_layout, det, I0Val, E, U, V, W, I0);
    return cudaGetLastError();
}

cudaError_t launch_finalize(int64_t n_pix, int64_t n_views, const float* I, const float* IAbs, const float* I0,
                            uint32_t* Ipoly, uint32_t* IAbsPoly, float* proj, cudaStream_t st)
{
    const int64_t n = n_pix * n_views;
    int64_t nb = (n + 255) / 256;
    if (nb > 148 * 32) nb = 148 * 32;
    if (nb == 0) return cudaSuccess;
    k_finalize<<<(unsigned)nb, 256, 0, st>>>(n_pix, n, I, IAbs, I0, Ipoly, IAbsPoly, proj);
    return cudaGetLastError();
}

cudaError_t launch_sample_points(const float* vol, cudaTextureObject_t tex, int nx, int ny, int nz, int interp,
                                 const float* pts, int64_t n, float* out, cudaStream_t st)
{
    int64_t nb = (n + 255) / 256;
    if (nb > 148 * 32) nb = 148 * 32;
    if (nb == 0) return cudaSuccess;
    k_sample_points<<<(unsigned)nb, 256, 0, st>>>(vol, tex, nx, ny, nz, interp, pts, n, out);
    return cudaGetLastError();
}

namespace {

// One thread per voxel: a non-zero voxel marks every brick whose dilated
// range [8b - 1, 8b + 7] holds it (b = (x + 1) >> 3, and b - 1 when x + 1 is a
// multiple of 8), per axis.  Concurrent stores all write 1.
struct VolPtrs {
    const float* p[kMaxM];
};

__global__ void k_occupancy(const VolPtrs vol, int M, int nx, int ny, int nz, int ox, int oy, uint8_t* occ)
{
    const int64_t n = (int64_t)nx * ny * nz;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        bool any = false;
        for (int m = 0; m < M; m++) any |= __ldg(vol.p[m] + k) != 0.f;
        if (!any) continue;
        const int x = (int)(k % nx), y = (int)((k / nx) % ny), z = (int)(k / ((int64_t)nx * ny));
        const int bx = (x + 1) >> kOccShift, by = (y + 1) >> kOccShift, bz = (z + 1) >> kOccShift;
        const int lx = ((x + 1) & ((1 << kOccShift) - 1)) == 0 && bx > 0;
        const int ly = ((y + 1) & ((1 << kOccShift) - 1)) == 0 && by > 0;
        const int lz = ((z + 1) & ((1 << kOccShift) - 1)) == 0 && bz > 0;
        for (int dz = 0; dz <= lz; dz++)
            for (int dy = 0; dy <= ly; dy++)
                for (int dx = 0; dx <= lx; dx++)
                    occ[((size_t)(bz - dz) * oy + (by - dy)) * ox + (bx - dx)] = 1;
    }
}

}  // namespace

namespace {

// Focal-spot re-alignment of the line-integral images (projOffsetMatchKernel,
// CBCTPolyProjGPU.cu:1956-1978): out[p][v][u][m] = in[p] sampled at
// (u + offU[p] / dSize, v + offV[p] / dSize), bilinear, 0 outside the image.
// The compat modes reproduce the texture unit (8-bit weights at the FP32
// coordinate u + offU/dSize + 0.5 it receives); TRILINEAR interpolates
// exactly at the FP64 position.
template <int M, int MODE>
__global__ void k_shift_views(const float* __restrict__ in, float* __restrict__ out, const float2* __restrict__ fspot,
                              int U, int V, float dSize, int view0, int n_views)
{
    const int64_t npix = (int64_t)U * V;
    const int64_t n = npix * n_views;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = t / npix, pix = t % npix;
        const int u = (int)(pix % U), v = (int)(pix / U);
        const float2 f = fspot[view0 + k];
        int ix, iy;
        float w[4];  // (ix, iy), (ix + 1, iy), (ix, iy + 1), (ix + 1, iy + 1)
        if (MODE == INTERP_TRILINEAR) {
            const double cx = (double)u + (double)f.x / (double)dSize, cy = (double)v + (double)f.y / (double)dSize;
            const double fx = floor(cx), fy = floor(cy);
            ix = (int)fx;
            iy = (int)fy;
            float wx, ux, wy, uy;
            frac_pair(cx - fx, wx, ux);
            frac_pair(cy - fy, wy, uy);
            w[0] = ux * uy; w[1] = wx * uy; w[2] = ux * wy; w[3] = wx * wy;
        } else {
            const float x = __fadd_rn(__fadd_rn((float)u, __fdiv_rn(f.x, dSize)), 0.5f);
            const float y = __fadd_rn(__fadd_rn((float)v, __fdiv_rn(f.y, dSize)), 0.5f);
            const int X = tex_fixed(x), Y = tex_fixed(y);
            ix = X >> 8;
            iy = Y >> 8;
            float w8[8];
            texunit_weights(X & 255, Y & 255, 0, w8);  // the view coordinate p + 0.5 has fraction 0
            w[0] = w8[0]; w[1] = w8[1]; w[2] = w8[2]; w[3] = w8[3];
        }
        const float* src = in + k * npix * M;
        float acc[M];
#pragma unroll
        for (int m = 0; m < M; m++) acc[m] = 0.f;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int x = ix + (c & 1), y = iy + (c >> 1);
            if ((unsigned)x >= (unsigned)U || (unsigned)y >= (unsigned)V) continue;
            const float* q = src + ((int64_t)y * U + x) * M;
#pragma unroll
            for (int m = 0; m < M; m++) acc[m] = fmaf(w[c], __ldg(q + m), acc[m]);
        }
        float* d = out + t * M;
#pragma unroll
        for (int m = 0; m < M; m++) d[m] = acc[m];
    }
}

template <int MODE>
cudaError_t shift_dispatch(int M, const float* in, float* out, const float2* fspot, int U, int V, float dSize,
                           int view0, int n_views, unsigned nb, cudaStream_t st)
{
    switch (M) {
        case 1: k_shift_views<1, MODE><<<nb, 256, 0, st>>>(in, out, fspot, U, V, dSize, view0, n_views); break;
        case 2: k_shift_views<2, MODE><<<nb, 256, 0, st>>>(in, out, fspot, U, V, dSize, view0, n_views); break;
        case 3: k_shift_views<3, MODE><<<nb, 256, 0, st>>>(in, out, fspot, U, V, dSize, view0, n_views); break;
        case 4: k_shift_views<4, MODE><<<nb, 256, 0, st>>>(in, out, fspot, U, V, dSize, view0, n_views); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_shift_views(const float* in, float* out, const GeomParams& g, int M, int interp, int view0,
                               int n_views, cudaStream_t st)
{
    if (!g.fspot) return cudaErrorInvalidValue;
    const int64_t n = (int64_t)g.U * g.V * n_views;
    if (n == 0) return cudaSuccess;
    int64_t nb = (n + 255) / 256;
    if (nb > 148 * 32) nb = 148 * 32;
    if (interp == INTERP_TRILINEAR)
        return shift_dispatch<INTERP_TRILINEAR>(M, in, out, g.fspot, g.U, g.V, g.dSize, view0, n_views, (unsigned)nb, st);
    return shift_dispatch<INTERP_TEXEMU>(M, in, out, g.fspot, g.U, g.V, g.dSize, view0, n_views, (unsigned)nb, st);
}

cudaError_t launch_occupancy(const float* const* vol, int M, int nx, int ny, int nz, uint8_t* occ, cudaStream_t st)
{
    const int ox = occ_dim(nx), oy = occ_dim(ny), oz = occ_dim(nz);
    cudaError_t e = cudaMemsetAsync(occ, 0, (size_t)ox * oy * oz, st);
    if (e != cudaSuccess) return e;
    VolPtrs vp = {};
    for (int m = 0; m < M && m < kMaxM; m++) vp.p[m] = vol[m];
    const int64_t n = (int64_t)nx * ny * nz;
    int64_t nb = (n + 255) / 256;
    if (nb > 148 * 32) nb = 148 * 32;
    k_occupancy<<<(unsigned)nb, 256, 0, st>>>(vp, M, nx, ny, nz, ox, oy, occ);
    return cudaGetLastError();
}

cudaError_t launch_count_support(const GeomParams& g, unsigned long long* out, cudaStream_t st)
{
    const dim3 block(32, 8);
    int gz = g.P < 64 ? g.P : 64;
    const dim3 grid((g.U + 31) / 32, (g.V + 7) / 8, gz > 0 ? gz : 1);
    if (g.P == 0 || g.U == 0 || g.V == 0) return cudaSuccess;
    k_count_support<<<grid, block, 0, st>>>(g, out);
    return cudaGetLastError();
}

}  // namespace ctfp
