// ctfp_batch.cu — the batched form: many independent problems (their own
// geometry, materials, spectra, view counts) run by persistent kernels over a
// device work queue, the whole call replayed as one CUDA graph.  No reference
// counterpart.
//
// Work unit = (item, view, 8 x 8 pixel tile): the 64 rays of one CTA, whose
// neighbouring rays share texture-cache lines.  Items are grouped by material
// count and sampler mode (one kernel instantiation each, so every group runs
// with the registers its own march needs); within a group they are queued
// largest first (rays x samples x materials), and every CTA takes the next
// unit from the group's counter (atomicAdd, no waits), so long problems start
// early and short ones fill the tail.
//
// Two kinds of call: the forward (march + spectral epilogue, optional
// checkpoint) and the fused forward + loss + adjoint, which for every ray
// marches, forms I, the loss term (log I - log I_target)^2 and its gradient,
// recomputes the spectral weights, and marches again scattering into the
// corner-expanded accumulators; a fold kernel then adds the accumulators into
// the gradients.
#include <algorithm>
#include <cstring>
#include <new>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/ctfp.h"
#include "ctfp_axis.cuh"
#include "ctfp_kernels.cuh"

namespace ctfp {
void set_last_error(const std::string& msg);
const GeomParams& plan_geom(const ctfp_plan* p);
int plan_materials(const ctfp_plan* p);
int plan_interp(const ctfp_plan* p);
int plan_sampler(const ctfp_plan* p);
int plan_device(const ctfp_plan* p);
int plan_energies(const ctfp_plan* p);
const float* plan_mu(const ctfp_plan* p);
const float* plan_W(const ctfp_plan* p);
cudaTextureObject_t plan_ltex(const ctfp_plan* p, int m);
cudaTextureObject_t plan_xtex(const ctfp_plan* p, int m);
cudaTextureObject_t plan_ytex(const ctfp_plan* p, int m);
cudaTextureObject_t plan_tex(const ctfp_plan* p, int m);
ctfp_status plan_upload(ctfp_plan* p, const float* const* volumes, cudaStream_t st);
}  // namespace ctfp

using namespace ctfp;

namespace {

// Threads of a persistent CTA, per kind of call, and the default rays and
// views of a work unit.  Forward: 128 threads, units of one view of a 128-ray
// tile (8 x 16 by default), the plain forward kernel's CTA: with the item's
// texture handles warp-uniform (item_tex) a one-item batch runs the 36-view
// poly_grid_256 case in 5.79 ms against 5.81 for the plain kernel, and 5.90
// and 6.22 ms with units of 2 and 4 views.  Fused forward + adjoint: 64
// threads, one view of a 64-ray tile (8 x 8), measured 3 % faster than
// 128-thread units (more CTAs in flight per SM for the scatter).
template <bool ADJOINT>
struct BatchShape {
    static constexpr int threads = ADJOINT ? 64 : 128;
    static constexpr int warps = threads / 32;
};
constexpr int kTU = 8, kTV = 8;  // the fused kernel's default tile; the forward's is 8 x 16
constexpr int kVPU[2] = {1, 1};  // default views per unit: forward, fused forward + adjoint
constexpr int kMaxVPU = 8;
inline int kind_threads(int kind) { return kind ? BatchShape<true>::threads : BatchShape<false>::threads; }

// One item as the persistent kernels see it.  The pointer fields are refreshed
// per call.
struct ItemDesc {
    GeomParams g;
    cudaTextureObject_t ltex[kMaxM];   // layered textures (TRILINEAR, TEXEMU)
    cudaTextureObject_t xtex[kMaxM];   // the axis sampler's x- and y-layered copies (TRILINEAR, TEXEMU)
    cudaTextureObject_t ytex[kMaxM];
    cudaTextureObject_t tex[kMaxM];    // 3D textures (TEXTURE: the reference's own sampler)
    const float* mu;   // [E][M]
    const float* W;    // [E][V][U]
    int M, E, interp;
    int tiles_u, tiles_v;
    int vgroups;       // groups of views per unit: ceil(P / views per unit)
    long long unit0;   // first unit of this item in the batch's numbering
    long long units;
    // per call
    float* I;
    float* IAbs;
    float* L;
    const float* I_target;
    float* gvol[kMaxM];
    float4* gexp[kMaxM];
    float* loss;       // device scalar accumulated with atomicAdd
};

// One group: items [first, first + count) of the table, units [begin, end).
struct GroupArgs {
    const ItemDesc* items;
    int first, count;
    long long begin, end;
    unsigned long long* counter;
    int tu_shift;  // rays of a unit tile: (1 << tu_shift) x (threads >> tu_shift)
    int vpu;       // views per unit
};

__device__ __forceinline__ int find_item(const GroupArgs& a, long long unit)
{
    int lo = a.first, hi = a.first + a.count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (a.items[mid].unit0 <= unit) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// The texture handles of the current item, read once per work unit through
// warp reductions of their two halves.  Every lane of a CTA holds the same
// item, but a value loaded from the item table is not known to be warp-uniform
// to the compiler, which must then assume a different texture per lane at
// every gather; the reductions' results are uniform by construction.  (All 32
// lanes of the warp execute this.)
template <int M>
struct ItemTex {
    cudaTextureObject_t x[M], y[M], l[M], t[M];
};
__device__ __forceinline__ cudaTextureObject_t warp_uniform(cudaTextureObject_t h)
{
    const unsigned lo = __reduce_min_sync(0xffffffffu, (unsigned)h);
    const unsigned hi = __reduce_min_sync(0xffffffffu, (unsigned)(h >> 32));
    return ((cudaTextureObject_t)hi << 32) | lo;
}
template <int M, int MODE, bool AXIS>
__device__ __forceinline__ ItemTex<M> item_tex(const ItemDesc& it)
{
    ItemTex<M> r;
#pragma unroll
    for (int m = 0; m < M; m++) {
        r.x[m] = r.y[m] = r.l[m] = r.t[m] = 0;
        if (MODE == INTERP_TEXTURE) {
            r.t[m] = warp_uniform(it.tex[m]);
        } else if (AXIS) {
            r.x[m] = warp_uniform(it.xtex[m]);
            r.y[m] = warp_uniform(it.ytex[m]);
        } else {
            r.l[m] = warp_uniform(it.ltex[m]);
        }
    }
    return r;
}

template <int MODE>
__device__ __forceinline__ Corner batch_corner(const ItemDesc& it, const RaySeg& s, const RayRef32& r, int i)
{
    if (MODE == INTERP_TRILINEAR) {
        const double t = (double)i;
        return corner_of<INTERP_TRILINEAR>(fma(t, s.bx, s.ax), fma(t, s.by, s.ay), fma(t, s.bz, s.az));
    }
    return corner_tex(ref32_coords(it.g, r, i));
}

// Path integrals of one ray: the axis sampler (AXIS), the layered sampler, or
// in TEXTURE mode the hardware tex3D at the reference's FP32 coordinates (as
// k_forward).
template <int M, int MODE, bool AXIS>
__device__ __forceinline__ void batch_march(const ItemDesc& it, const ItemTex<M>& tx, const RaySeg& s,
                                            const RayRef32& r, int p, int v, int u, float* L)
{
    if (AXIS && MODE != INTERP_TEXTURE) {
        const OccView none{nullptr, 0, 0, 0, 0, 0, 0};
        constexpr int AM = MODE == INTERP_TEXTURE ? INTERP_TEXEMU : MODE;  // (not instantiated for TEXTURE)
        if (axis_is_x(it.g, p)) march_ray_axis<M, AM, 0, false>(it.g, tx.x, tx.y, none, p, v, u, L);
        else march_ray_axis<M, AM, 1, false>(it.g, tx.x, tx.y, none, p, v, u, L);
        return;
    }
    float acc[M], cmp[M];
#pragma unroll
    for (int m = 0; m < M; m++) { acc[m] = 0.f; cmp[m] = 0.f; }
    if (MODE == INTERP_TEXTURE) {
#pragma unroll 2
        for (int i = s.i0; i < s.i1; i++) {
            const float3 x = ref32_coords<false>(it.g, r, i);
#pragma unroll
            for (int m = 0; m < M; m++) kahan_add(acc[m], cmp[m], tex3D<float>(tx.t[m], x.x, x.y, x.z));
        }
#pragma unroll
        for (int m = 0; m < M; m++) L[m] = it.g.dx * (acc[m] - cmp[m]);
        return;
    }
#pragma unroll 2
    for (int i = s.i0; i < s.i1; i++) {
        const Corner c = batch_corner<MODE>(it, s, r, i);
        float v[M][8];
        load8_layered<M>(tx.l, it.g.nz, c, v);
#pragma unroll
        for (int m = 0; m < M; m++) kahan_add(acc[m], cmp[m], interp8<MODE>(c, v[m]));
    }
#pragma unroll
    for (int m = 0; m < M; m++) L[m] = it.g.dx * (acc[m] - cmp[m]);
}



// One ray.  ADJOINT: the fused forward + loss + adjoint; returns the ray's
// loss term.
template <int M, int MODE, bool ADJOINT, bool AXIS>
__device__ __forceinline__ float process_ray(const ItemDesc& it, const ItemTex<M>& tx, const float* s_mu, int p, int v,
                                             int u)
{
    const int64_t npix = (int64_t)it.g.U * it.g.V;
    const int64_t pix = (int64_t)v * it.g.U + u;
    const int64_t ray = (int64_t)p * npix + pix;
    const RaySeg s = ray_segment(it.g, p, v, u);
    RayRef32 r;
    if (MODE != INTERP_TRILINEAR) r = ray_ref32(it.g, p, v, u);
    float L[M];
    batch_march<M, MODE, AXIS>(it, tx, s, r, p, v, u, L);
    // the plain forward's epilogue (spectral / spectral_adjoint), so the
    // batch's I equals ctfp_forward's for the same path integrals
    if (!ADJOINT) {
        float I, A;
        spectral<M>(s_mu, it.E, it.W, pix, npix, L, I, A);
        if (it.I) it.I[ray] = I;
        if (it.IAbs) it.IAbs[ray] = A;
        if (it.L) {
#pragma unroll
            for (int m = 0; m < M; m++) it.L[ray * M + m] = L[m];
        }
        return 0.f;
    }
    float I, S[M];
    spectral_adjoint<M>(s_mu, it.E, it.W, pix, npix, L, I, S);
    if (it.I) it.I[ray] = I;
    // loss (log I - log T)^2: dLoss/dI = 2 (log I - log T) / I, dI/dL_m = -S_m
    if (!(I > 0.f)) return 0.f;
    const float res = logf(I) - logf(it.I_target[ray]);
    const float gI = 2.0f * res / I;
    float g[M];
    bool any = false;
#pragma unroll
    for (int m = 0; m < M; m++) {
        g[m] = -gI * S[m] * it.g.dx;
        any |= g[m] != 0.f;
    }
    // TEXTURE: the transpose of the texture unit's weights, which the
    // emulation reproduces exactly (as ctfp_backward does for such a plan)
    if (any)
        scatter_ray_axis<M, MODE == INTERP_TRILINEAR ? INTERP_TRILINEAR : INTERP_TEXEMU>(it.g, it.gexp, p, v, u, g,
                                                                                          axis_is_x(it.g, p));
    return res * res;
}

// CTAs per SM the kernels are compiled for (their register caps: 65536 /
// (threads * minb)).  Forward, trilinear: 8 CTAs of 128 threads, 64
// registers, the plain forward kernel's cap, for every material count: with
// the texture handles in uniform registers the 3-material batch forward ran
// the 3-material problems of the 48-problem batch 3.7 % slower than their
// plain calls at this cap, and 9 % and 15 % slower at 6 and 5 CTAs (80 and
// 96 registers).  Fused forward + adjoint (64-thread CTAs): it carries the
// scatter's run accumulators on top of the march; 14 CTAs (72 registers) for
// M <= 2 and 12 (80) for more materials ran the 48-problem fused step 1.7 %
// faster than 12 and 10 CTAs, and as fast as 16 (64 registers, spills).  The
// texture emulation's FP32 reference coordinates take more registers than the
// FP64 trilinear ones.
template <bool ADJOINT, int M, int MODE, bool AXIS>
struct BatchBudget {
    static constexpr int minb = MODE == INTERP_TRILINEAR
                                    ? (ADJOINT ? (M <= 2 ? 14 : 12) : 8)
                                    : (ADJOINT ? (M <= 2 ? 10 : 8) : (M <= 2 ? 6 : 5));
};

// MULTI: units of more than one view (a.vpu > 1), marched one view after the
// other; the one-view kernel has no view loop, whose live state cost the fused
// axis kernel 3 % on the 48-problem batch.
template <int M, int MODE, bool ADJOINT, bool AXIS, bool MULTI>
__global__ void __launch_bounds__(BatchShape<ADJOINT>::threads, BatchBudget<ADJOINT, M, MODE, AXIS>::minb)
    k_batch(const GroupArgs a)
{
    constexpr int kThreads = BatchShape<ADJOINT>::threads, kWarps = BatchShape<ADJOINT>::warps;
    __shared__ float s_mu[CTFP_MAX_ENERGIES * M];
    __shared__ float s_loss[kWarps];
    // the current unit as thread 0 decoded it: item, first view, tile column
    // and row, and whether the item changed.  Every thread re-reads these
    // (volatile) where it needs them, so none of them is held in a register
    // across a ray's march.
    __shared__ int s_end, s_item, s_new, s_p, s_tu, s_tv;
    // the current item and its unit range (thread 0): the units a CTA takes
    // mostly fall in one item, so the item search runs only when the item
    // changes
    __shared__ int s_cached;
    __shared__ long long s_cbegin, s_cend;
    if (threadIdx.x == 0) {
        s_cached = -1;
        s_cbegin = s_cend = 0;
    }
    for (;;) {
        __syncthreads();  // the previous unit is done with s_mu, s_loss and the unit fields
        if (threadIdx.x == 0) {
            const long long unit = a.begin + (long long)atomicAdd(a.counter, 1ull);
            s_end = unit >= a.end;
            if (unit < a.end) {
                const int cached = s_cached;
                const int k = (unit >= s_cbegin && unit < s_cend) ? cached : find_item(a, unit);
                const ItemDesc& it = a.items[k];
                s_new = k != cached;
                s_cached = k;
                s_cbegin = it.unit0;
                s_cend = it.unit0 + it.units;
                // unit order within an item.  Forward: view group, then tile
                // row, then tile column.  Adjoint: tile row, then view group,
                // then tile column, so that the CTAs resident at any time work
                // on one band of detector rows over many views: those rays
                // cross a thin z-slab of the volume, whose accumulator cells
                // then stay in L2.
                const long long local = unit - it.unit0;
                if (ADJOINT) {
                    const long long band_units = (long long)it.vgroups * it.tiles_u;
                    const int rem = (int)(local % band_units);
                    s_tv = (int)(local / band_units);
                    s_p = rem / it.tiles_u;
                    s_tu = rem % it.tiles_u;
                } else {
                    const int tiles = it.tiles_u * it.tiles_v;
                    const int t = (int)(local % tiles);
                    s_p = (int)(local / tiles);
                    s_tv = t / it.tiles_u;
                    s_tu = t % it.tiles_u;
                }
                s_item = k;
            }
        }
        __syncthreads();
        if (*(volatile int*)&s_end) break;
        const ItemDesc* const itp = a.items + *(volatile int*)&s_item;
        if (*(volatile int*)&s_new) {
            for (int j = threadIdx.x; j < itp->E * M; j += kThreads) s_mu[j] = itp->mu[j];
            __syncthreads();
        }
        const ItemTex<M> tx = item_tex<M, MODE, AXIS>(*itp);
        float loss = 0.f;
#pragma unroll 1
        for (int k = 0; k < (MULTI ? a.vpu : 1); k++) {
            const ItemDesc& it = a.items[*(volatile int*)&s_item];
            // this thread's ray within the unit's tile
            const int tile_u = 1 << a.tu_shift, tile_v = kThreads >> a.tu_shift;
            int du, dv;
            if (AXIS && tile_v % 4 == 0 && tile_u <= kThreads / 4) {
                // the axis sampler's lane quads run down 4 detector rows
                const int q = threadIdx.x >> 2;
                du = q % tile_u;
                dv = 4 * (q / tile_u) + (threadIdx.x & 3);
            } else {
                du = threadIdx.x & (tile_u - 1);
                dv = threadIdx.x >> a.tu_shift;
            }
            const int u = *(volatile int*)&s_tu * tile_u + du;
            const int v = *(volatile int*)&s_tv * tile_v + dv;
            const int pk = *(volatile int*)&s_p * (MULTI ? a.vpu : 1) + k;
            if (u < it.g.U && v < it.g.V && pk < it.g.P) loss += process_ray<M, MODE, ADJOINT, AXIS>(it, tx, s_mu, pk, v, u);
        }
        if (ADJOINT) {
            const ItemDesc& it = a.items[*(volatile int*)&s_item];
            if (it.loss) {
                const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
                for (int o = 16; o > 0; o >>= 1) loss += __shfl_down_sync(0xffffffffu, loss, o);
                if (lane == 0) s_loss[warp] = loss;
                __syncthreads();
                if (threadIdx.x == 0) {
                    float t = 0.f;
                    for (int w = 0; w < kWarps; w++) t += s_loss[w];
                    atomicAdd(it.loss, t);
                }
            }
        }
    }
}

// Folds every item's corner-expanded accumulators into its gradients.
__global__ void k_batch_fold(const ItemDesc* items, int n_items, const long long* vox0, long long total)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = n_items - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (vox0[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        const ItemDesc& it = items[lo];
        const long long k = t - vox0[lo];
        const int nx = it.g.nx, ny = it.g.ny, nz = it.g.nz;
        const int x = (int)(k % nx), y = (int)((k / nx) % ny), z = (int)(k / ((long long)nx * ny));
        for (int m = 0; m < it.M; m++) it.gvol[m][k] += face_fold(it.gexp[m], nx, ny, nz, x, y, z);
    }
}

using KernelFn = void (*)(GroupArgs);

template <int M, bool ADJOINT, bool MULTI>
KernelFn kernel_for_m(int interp, bool axis)
{
    if (interp == INTERP_TRILINEAR)
        return axis ? k_batch<M, INTERP_TRILINEAR, ADJOINT, true, MULTI>
                    : k_batch<M, INTERP_TRILINEAR, ADJOINT, false, MULTI>;
    if (interp == INTERP_TEXEMU)
        return axis ? k_batch<M, INTERP_TEXEMU, ADJOINT, true, MULTI> : k_batch<M, INTERP_TEXEMU, ADJOINT, false, MULTI>;
    return k_batch<M, INTERP_TEXTURE, ADJOINT, false, MULTI>;
}

template <bool ADJOINT, bool MULTI>
KernelFn kernel_for_v(int M, int interp, bool axis)
{
    switch (M) {
        case 1: return kernel_for_m<1, ADJOINT, MULTI>(interp, axis);
        case 2: return kernel_for_m<2, ADJOINT, MULTI>(interp, axis);
        case 3: return kernel_for_m<3, ADJOINT, MULTI>(interp, axis);
        default: return kernel_for_m<4, ADJOINT, MULTI>(interp, axis);
    }
}

// The kernel of one kind of call for units of vpu views (both variants have
// the same register budget, hence the same persistent grid).
template <bool ADJOINT>
KernelFn kernel_for(int M, int interp, bool axis, int vpu = 1)
{
    return vpu > 1 ? kernel_for_v<ADJOINT, true>(M, interp, axis) : kernel_for_v<ADJOINT, false>(M, interp, axis);
}

}  // namespace

struct ctfp_batch {
    int n = 0;
    int device = 0;
    // rays and views of a work unit, per kind of call (0: forward, 1: forward
    // + adjoint), set by ctfp_batch_set_shape and ctfp_batch_set_views or
    // tuned per kind by ctfp_batch_autotune
    int tile_u[2] = {kTU, kTU}, tile_v[2] = {2 * kTV, kTV};
    int vpu[2] = {kVPU[0], kVPU[1]};
    int laid_out = -1;  // the kind the units are currently laid out for
    std::vector<ctfp_plan*> plans;
    std::vector<int> order;            // item slot -> plan index (grouped, cost order within a group)
    std::vector<bool> item_axis;       // slot -> the plan marches the axis sampler's copies
    std::vector<long long> vox0;       // first voxel of each slot in the fold's flat index
    std::vector<ItemDesc> items;       // tables of the current call
    struct Group {
        int M, interp, axis, first, count;
        long long begin, end;
        int grid[2];                   // persistent grid: forward, forward + adjoint
    };
    std::vector<Group> groups;
    ItemDesc* d_items[2] = {nullptr, nullptr};  // device tables of the forward, forward + adjoint graphs
    long long* d_vox0 = nullptr;
    long long total_units = 0, total_vox = 0;
    unsigned long long* d_counter = nullptr;    // one per group
    float4* d_gexp = nullptr;          // all items' accumulators, contiguous
    size_t gexp_elems = 0;
    std::vector<size_t> gexp_off;      // [slot][m]
    cudaStream_t capture = nullptr;    // private stream the graphs are recorded on
    // one graph per kind, valid for the tables, volume pointers and loss
    // pointer it was recorded with; it runs in the order of the stream it is
    // launched on
    struct Graph {
        cudaGraphExec_t exec = nullptr;
        std::vector<ItemDesc> items;
        std::vector<const float*> vols;
        float* loss = nullptr;
    } graph[2];
};

namespace {

ctfp_status bfail(ctfp_status st, const std::string& m)
{
    ctfp::set_last_error(m);
    return st;
}

#define BATCH_CUDA(call)                                                                                  \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess)                                                                            \
            return bfail(e_ == cudaErrorMemoryAllocation ? CTFP_OOM : CTFP_CUDA_ERROR,                    \
                         std::string(#call) + ": " + cudaGetErrorString(e_));                             \
    } while (0)

// Records one call's stream work: volume uploads, counters, accumulators, the
// persistent kernel of every group, the fold.
ctfp_status record(ctfp_batch* b, bool adjoint, const std::vector<const float*>& vols, float* loss, cudaStream_t st,
                   int tune_div = 0)
{
    size_t off = 0;
    for (int s = 0; s < b->n && tune_div == 0; s++) {
        ctfp_plan* p = b->plans[(size_t)b->order[(size_t)s]];
        ctfp_status rs = plan_upload(p, vols.data() + off, st);
        if (rs != CTFP_OK) return rs;
        off += (size_t)b->items[(size_t)s].M;
    }
    BATCH_CUDA(cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned long long) * b->groups.size(), st));
    if (adjoint) {
        // (tuning leaves the accumulators as they are: a real call zeroes them)
        if (tune_div == 0) BATCH_CUDA(cudaMemsetAsync(b->d_gexp, 0, b->gexp_elems * sizeof(float4), st));
        if (loss) BATCH_CUDA(cudaMemsetAsync(loss, 0, sizeof(float) * (size_t)b->n, st));
    }
    const ItemDesc* table = b->d_items[adjoint ? 1 : 0];
    for (size_t gi = 0; gi < b->groups.size(); gi++) {
        const ctfp_batch::Group& G = b->groups[gi];
        // tuning runs the first 1/tune_div of each group's queue: its largest items
        const long long end = tune_div > 0 ? G.begin + std::max(1LL, (G.end - G.begin) / tune_div) : G.end;
        GroupArgs a{table, G.first, G.count, G.begin, end, b->d_counter + gi,
                    __builtin_ctz((unsigned)b->tile_u[adjoint ? 1 : 0]), b->vpu[adjoint ? 1 : 0]};
        const int vpu = b->vpu[adjoint ? 1 : 0];
        KernelFn fn = adjoint ? kernel_for<true>(G.M, G.interp, G.axis, vpu)
                              : kernel_for<false>(G.M, G.interp, G.axis, vpu);
        fn<<<G.grid[adjoint ? 1 : 0], kind_threads(adjoint ? 1 : 0), 0, st>>>(a);
        BATCH_CUDA(cudaGetLastError());
    }
    if (adjoint && tune_div == 0) {
        long long nb = (b->total_vox + 255) / 256;
        if (nb > 148 * 16) nb = 148 * 16;
        k_batch_fold<<<(unsigned)std::max<long long>(nb, 1), 256, 0, st>>>(table, b->n, b->d_vox0, b->total_vox);
        BATCH_CUDA(cudaGetLastError());
    }
    return CTFP_OK;
}

// Replays the graph of this kind on st, recording it first (on the batch's
// private stream: the caller's may be the legacy default stream, which cannot
// be captured) when the tables, the volume pointers or the loss pointer differ
// from its recording.
ctfp_status run(ctfp_batch* b, bool adjoint, const std::vector<const float*>& vols, float* loss, cudaStream_t st)
{
    ctfp_batch::Graph& G = b->graph[adjoint ? 1 : 0];
    const bool same = G.exec && G.loss == loss && G.vols == vols &&
                      std::memcmp(G.items.data(), b->items.data(), sizeof(ItemDesc) * (size_t)b->n) == 0;
    if (!same) {
        if (G.exec) cudaGraphExecDestroy(G.exec);
        G.exec = nullptr;
        // the device table changes only here, after the stream's earlier work
        BATCH_CUDA(cudaStreamSynchronize(st));
        BATCH_CUDA(cudaMemcpy(b->d_items[adjoint ? 1 : 0], b->items.data(), sizeof(ItemDesc) * (size_t)b->n,
                              cudaMemcpyHostToDevice));
        cudaGraph_t gr = nullptr;
        BATCH_CUDA(cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeThreadLocal));
        const ctfp_status rs = record(b, adjoint, vols, loss, b->capture);
        const cudaError_t e = cudaStreamEndCapture(b->capture, &gr);
        if (rs != CTFP_OK) {
            if (gr) cudaGraphDestroy(gr);
            return rs;
        }
        if (e != cudaSuccess) return bfail(CTFP_CUDA_ERROR, std::string("graph capture: ") + cudaGetErrorString(e));
        const cudaError_t ei = cudaGraphInstantiate(&G.exec, gr, 0);
        cudaGraphDestroy(gr);
        if (ei != cudaSuccess) {
            G.exec = nullptr;
            return bfail(CTFP_CUDA_ERROR, std::string("graph instantiate: ") + cudaGetErrorString(ei));
        }
        G.items = b->items;
        G.vols = vols;
        G.loss = loss;
    }
    BATCH_CUDA(cudaGraphLaunch(G.exec, st));
    return CTFP_OK;
}

struct DevScope {
    int prev = -1;
    explicit DevScope(int d)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != d) cudaSetDevice(d);
    }
    ~DevScope()
    {
        int c = -1;
        if (prev >= 0 && cudaGetDevice(&c) == cudaSuccess && c != prev) cudaSetDevice(prev);
    }
};

bool batchable(const ctfp_plan* p)
{
    return (plan_interp(p) == INTERP_TEXTURE || plan_sampler(p) == SAMPLER_LAYERED ||
            plan_sampler(p) == SAMPLER_AXIS) &&
           !plan_geom(p).fspot;
}

// Whether the item marches the axis sampler's copies.
bool uses_axis(const ctfp_plan* p) { return plan_interp(p) != INTERP_TEXTURE && plan_sampler(p) == SAMPLER_AXIS; }

// Unit counts and queue ranges for the unit shape of one kind of call: item s
// holds tiles_u x tiles_v x ceil(P / views per unit) units, numbered after the
// items before it.
void layout_units(ctfp_batch* b, int kind)
{
    b->laid_out = kind;
    long long unit = 0;
    size_t gi = 0;
    for (int s = 0; s < b->n; s++) {
        const GeomParams& g = plan_geom(b->plans[(size_t)b->order[(size_t)s]]);
        ItemDesc& it = b->items[(size_t)s];
        while (gi + 1 < b->groups.size() && s >= b->groups[gi + 1].first) gi++;
        if (s == b->groups[gi].first) b->groups[gi].begin = unit;
        it.unit0 = unit;
        it.units = (long long)((g.U + b->tile_u[kind] - 1) / b->tile_u[kind]) *
                   ((g.V + b->tile_v[kind] - 1) / b->tile_v[kind]) * ((g.P + b->vpu[kind] - 1) / b->vpu[kind]);
        unit += it.units;
        b->groups[gi].end = unit;
    }
    b->total_units = unit;
}

// Fills the per-call tables from the plans' current state, with the units
// laid out for this kind of call.
ctfp_status fill_items(ctfp_batch* b, int kind)
{
    if (b->laid_out != kind) layout_units(b, kind);
    for (int s = 0; s < b->n; s++) {
        ctfp_plan* p = b->plans[(size_t)b->order[(size_t)s]];
        if (!batchable(p))
            return bfail(CTFP_UNSUPPORTED,
                         "batched items need the axis or layered sampler (or CTFP_INTERP_TEXTURE) and no focal spot");
        if (plan_energies(p) < 1) return bfail(CTFP_NOT_READY, "spectral tables not set for an item");
        ItemDesc& it = b->items[(size_t)s];
        const long long unit0 = it.unit0, units = it.units;
        const int M = it.M, interp = it.interp;
        const bool axis = b->item_axis[(size_t)s];
        if (plan_materials(p) != M || plan_interp(p) != interp || uses_axis(p) != axis)
            return bfail(CTFP_INVALID_ARG, "a plan's sampler mode changed after ctfp_batch_create");
        std::memset(&it, 0, sizeof(it));
        it.g = plan_geom(p);
        it.M = M;
        it.E = plan_energies(p);
        it.interp = interp;
        it.mu = plan_mu(p);
        it.W = plan_W(p);
        for (int m = 0; m < it.M; m++) {
            it.ltex[m] = plan_ltex(p, m);
            it.xtex[m] = plan_xtex(p, m);
            it.ytex[m] = plan_ytex(p, m);
            it.tex[m] = plan_tex(p, m);
            it.gexp[m] = b->d_gexp + b->gexp_off[(size_t)s * kMaxM + m];
        }
        it.tiles_u = (it.g.U + b->tile_u[kind] - 1) / b->tile_u[kind];
        it.tiles_v = (it.g.V + b->tile_v[kind] - 1) / b->tile_v[kind];
        it.vgroups = (it.g.P + b->vpu[kind] - 1) / b->vpu[kind];
        it.unit0 = unit0;
        it.units = units;
    }
    return CTFP_OK;
}

}  // namespace

extern "C" {

ctfp_status ctfp_batch_create(int32_t n_items, ctfp_plan* const* plans, ctfp_batch** out)
{
    if (!out) return bfail(CTFP_INVALID_ARG, "out is NULL");
    *out = nullptr;
    if (!plans || n_items < 1) return bfail(CTFP_INVALID_ARG, "need at least one plan");
    for (int i = 0; i < n_items; i++)
        if (!plans[i]) return bfail(CTFP_INVALID_ARG, "plan is NULL");
    const int dev = plan_device(plans[0]);
    for (int i = 0; i < n_items; i++) {
        if (plan_device(plans[i]) != dev) return bfail(CTFP_INVALID_ARG, "plans must share one device");
        if (!batchable(plans[i]))
            return bfail(CTFP_UNSUPPORTED,
                         "batched items need the axis or layered sampler (or CTFP_INTERP_TEXTURE) and no focal spot");
        if (plan_energies(plans[i]) < 1) return bfail(CTFP_NOT_READY, "spectral tables not set for an item");
    }
    DevScope ds(dev);
    ctfp_batch* b = new (std::nothrow) ctfp_batch();
    if (!b) return bfail(CTFP_OOM, "host allocation failed");
    b->n = n_items;
    b->device = dev;
    b->plans.assign(plans, plans + n_items);
    // group by (materials, mode), groups by total cost; within a group cost
    // order (rays x samples x materials), largest first: the queue hands out
    // units in this order (longest-processing-time-first list scheduling)
    std::vector<double> cost((size_t)n_items);
    for (int i = 0; i < n_items; i++) {
        const GeomParams& g = plan_geom(plans[i]);
        cost[(size_t)i] = (double)g.U * g.V * g.P * g.K * plan_materials(plans[i]);
    }
    auto gkey = [&](int i) {
        return (plan_materials(plans[i]) * 4 + plan_interp(plans[i])) * 2 + (uses_axis(plans[i]) ? 1 : 0);
    };
    std::vector<double> gcost(64, 0.0);
    for (int i = 0; i < n_items; i++) gcost[(size_t)gkey(i)] += cost[(size_t)i];
    b->order.resize((size_t)n_items);
    std::iota(b->order.begin(), b->order.end(), 0);
    std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) {
        const int gx = gkey(x), gy = gkey(y);
        if (gx != gy) return gcost[(size_t)gx] != gcost[(size_t)gy] ? gcost[(size_t)gx] > gcost[(size_t)gy] : gx < gy;
        return cost[(size_t)x] > cost[(size_t)y];
    });
    b->items.resize((size_t)n_items);
    b->item_axis.resize((size_t)n_items);
    b->vox0.resize((size_t)n_items);
    b->gexp_off.assign((size_t)n_items * kMaxM, 0);
    long long unit = 0, vox = 0;
    size_t gexp = 0;
    for (int s = 0; s < n_items; s++) {
        ctfp_plan* p = plans[b->order[(size_t)s]];
        const GeomParams& g = plan_geom(p);
        ItemDesc& it = b->items[(size_t)s];
        it.M = plan_materials(p);
        it.interp = plan_interp(p);
        const int ax = uses_axis(p) ? 1 : 0;
        b->item_axis[(size_t)s] = ax != 0;
        if (b->groups.empty() || b->groups.back().M != it.M || b->groups.back().interp != it.interp ||
            b->groups.back().axis != ax)
            b->groups.push_back({it.M, it.interp, ax, s, 0, unit, unit, {0, 0}});
        b->groups.back().count++;
        b->vox0[(size_t)s] = vox;
        vox += (long long)g.nx * g.ny * g.nz;
        for (int m = 0; m < it.M; m++) {
            b->gexp_off[(size_t)s * kMaxM + m] = gexp;
            gexp += expanded_elems(g);
        }
    }
    layout_units(b, 0);
    b->total_vox = vox;
    b->gexp_elems = gexp;
    cudaError_t e = cudaMalloc(&b->d_items[0], sizeof(ItemDesc) * (size_t)n_items);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_items[1], sizeof(ItemDesc) * (size_t)n_items);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_vox0, sizeof(long long) * (size_t)n_items);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_counter, sizeof(unsigned long long) * b->groups.size());
    if (e == cudaSuccess) e = cudaMalloc(&b->d_gexp, sizeof(float4) * gexp);
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_vox0, b->vox0.data(), sizeof(long long) * (size_t)n_items, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking);
    int nsm = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    for (ctfp_batch::Group& G : b->groups) {
        for (int k = 0; k < 2 && e == cudaSuccess; k++) {
            int per = 0;
            KernelFn fn = k ? kernel_for<true>(G.M, G.interp, G.axis) : kernel_for<false>(G.M, G.interp, G.axis);
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, kind_threads(k), 0);
            G.grid[k] = std::max(1, per) * std::max(1, nsm);
        }
    }
    if (e != cudaSuccess) {
        ctfp_batch_destroy(b);
        return bfail(e == cudaErrorMemoryAllocation ? CTFP_OOM : CTFP_CUDA_ERROR,
                     std::string("ctfp_batch_create: ") + cudaGetErrorString(e));
    }
    ctfp_status rs = fill_items(b, 0);
    if (rs != CTFP_OK) {
        ctfp_batch_destroy(b);
        return rs;
    }
    *out = b;
    return CTFP_OK;
}

ctfp_status ctfp_batch_destroy(ctfp_batch* b)
{
    if (!b) return CTFP_OK;
    DevScope ds(b->device);
    for (int i = 0; i < 2; i++)
        if (b->graph[i].exec) cudaGraphExecDestroy(b->graph[i].exec);
    cudaFree(b->d_items[0]);
    cudaFree(b->d_items[1]);
    cudaFree(b->d_vox0);
    cudaFree(b->d_counter);
    cudaFree(b->d_gexp);
    if (b->capture) cudaStreamDestroy(b->capture);
    delete b;
    return CTFP_OK;
}

ctfp_status ctfp_batch_forward(ctfp_batch* b, const float* const* const* volumes, float* const* I,
                               float* const* IAbsorb, float* const* L_ckpt, void* stream)
{
    if (!b) return bfail(CTFP_INVALID_ARG, "batch is NULL");
    if (!volumes || !I) return bfail(CTFP_INVALID_ARG, "volumes and I are required");
    DevScope ds(b->device);
    ctfp_status rs = fill_items(b, 0);
    if (rs != CTFP_OK) return rs;
    std::vector<const float*> vols;
    for (int s = 0; s < b->n; s++) {
        const int k = b->order[(size_t)s];
        ItemDesc& it = b->items[(size_t)s];
        if (!volumes[k] || !I[k]) return bfail(CTFP_INVALID_ARG, "NULL volume list or I for an item");
        for (int m = 0; m < it.M; m++) vols.push_back(volumes[k][m]);
        it.I = I[k];
        it.IAbs = IAbsorb ? IAbsorb[k] : nullptr;
        it.L = L_ckpt ? L_ckpt[k] : nullptr;
    }
    return run(b, false, vols, nullptr, (cudaStream_t)stream);
}

ctfp_status ctfp_batch_forward_adjoint(ctfp_batch* b, const float* const* const* volumes,
                                       const float* const* I_target, float* const* I, float* const* const* g_volumes,
                                       float* loss, void* stream)
{
    if (!b) return bfail(CTFP_INVALID_ARG, "batch is NULL");
    if (!volumes || !I_target || !g_volumes) return bfail(CTFP_INVALID_ARG, "volumes, I_target, g_volumes are required");
    DevScope ds(b->device);
    ctfp_status rs = fill_items(b, 1);
    if (rs != CTFP_OK) return rs;
    std::vector<const float*> vols;
    for (int s = 0; s < b->n; s++) {
        const int k = b->order[(size_t)s];
        ItemDesc& it = b->items[(size_t)s];
        if (!volumes[k] || !I_target[k] || !g_volumes[k])
            return bfail(CTFP_INVALID_ARG, "NULL volume list, target or gradient list for an item");
        for (int m = 0; m < it.M; m++) {
            if (!g_volumes[k][m]) return bfail(CTFP_INVALID_ARG, "NULL gradient volume");
            vols.push_back(volumes[k][m]);
            it.gvol[m] = g_volumes[k][m];
        }
        it.I = I ? I[k] : nullptr;
        it.I_target = I_target[k];
        it.loss = loss ? loss + k : nullptr;
    }
    return run(b, true, vols, loss, (cudaStream_t)stream);
}

ctfp_status ctfp_batch_set_shape(ctfp_batch* b, int32_t tile_u, int32_t tile_v)
{
    if (!b) return bfail(CTFP_INVALID_ARG, "batch is NULL");
    if (tile_u < 1 || tile_v < 1 || tile_u * tile_v != BatchShape<true>::threads || (tile_u & (tile_u - 1)) != 0)
        return bfail(CTFP_INVALID_ARG, "tile_u x tile_v must be 64 rays, tile_u a power of two");
    DevScope ds(b->device);
    // graphs recorded with the old queue may still be running
    BATCH_CUDA(cudaDeviceSynchronize());
    for (ctfp_batch::Graph& G : b->graph) {
        if (G.exec) cudaGraphExecDestroy(G.exec);
        G.exec = nullptr;
    }
    b->tile_u[0] = b->tile_u[1] = tile_u;
    b->tile_v[0] = 2 * tile_v;  // the forward's 128-ray tile: the same tile, twice as high
    b->tile_v[1] = tile_v;
    layout_units(b, 0);
    return CTFP_OK;
}

ctfp_status ctfp_batch_set_views(ctfp_batch* b, int32_t fwd_views, int32_t adj_views)
{
    if (!b) return bfail(CTFP_INVALID_ARG, "batch is NULL");
    if (fwd_views < 1 || fwd_views > kMaxVPU || adj_views < 1 || adj_views > kMaxVPU)
        return bfail(CTFP_INVALID_ARG, "views per work unit must be in [1, 8]");
    DevScope ds(b->device);
    BATCH_CUDA(cudaDeviceSynchronize());
    for (ctfp_batch::Graph& G : b->graph) {
        if (G.exec) cudaGraphExecDestroy(G.exec);
        G.exec = nullptr;
    }
    b->vpu[0] = fwd_views;
    b->vpu[1] = adj_views;
    layout_units(b, 0);
    return CTFP_OK;
}

ctfp_status ctfp_batch_get_views(const ctfp_batch* b, int32_t* fwd_views, int32_t* adj_views)
{
    if (!b) return bfail(CTFP_INVALID_ARG, "batch is NULL");
    if (fwd_views) *fwd_views = b->vpu[0];
    if (adj_views) *adj_views = b->vpu[1];
    return CTFP_OK;
}

ctfp_status ctfp_batch_autotune(ctfp_batch* b, const float* const* const* volumes, const float* const* I_target,
                                ctfp_launch_shape* out, void* stream)
{
    if (!b) return bfail(CTFP_INVALID_ARG, "batch is NULL");
    if (!volumes || !I_target) return bfail(CTFP_INVALID_ARG, "volumes and I_target are required");
    DevScope ds(b->device);
    cudaStream_t st = (cudaStream_t)stream;
    std::vector<const float*> vols;
    for (int s = 0; s < b->n; s++) {
        const int k = b->order[(size_t)s];
        if (!volumes[k] || !I_target[k]) return bfail(CTFP_INVALID_ARG, "NULL volume list or target for an item");
        for (int m = 0; m < b->items[(size_t)s].M; m++) vols.push_back(volumes[k][m]);
    }
    // the volumes once into the plans' arrays; the candidates then time only
    // their kernels, on the first eighth of every group's queue
    size_t off = 0;
    for (int s = 0; s < b->n; s++) {
        ctfp_status rs = plan_upload(b->plans[(size_t)b->order[(size_t)s]], vols.data() + off, st);
        if (rs != CTFP_OK) return rs;
        off += (size_t)b->items[(size_t)s].M;
    }
    float* loss = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    BATCH_CUDA(cudaMalloc(&loss, sizeof(float) * (size_t)b->n));
    struct Freer {
        float* p;
        cudaEvent_t a, c;
        ~Freer()
        {
            cudaFree(p);
            if (a) cudaEventDestroy(a);
            if (c) cudaEventDestroy(c);
        }
    } freer{loss, nullptr, nullptr};
    BATCH_CUDA(cudaEventCreate(&e0));
    freer.a = e0;
    BATCH_CUDA(cudaEventCreate(&e1));
    freer.c = e1;
    // 64-ray tiles; the forward's candidates are the same tiles twice as high
    static const int shapes[][2] = {{8, 8}, {16, 4}, {4, 16}, {32, 2}, {2, 32}};
    const int nshapes = (int)(sizeof(shapes) / sizeof(shapes[0]));
    static const int views[] = {1, 2, 4};
    const int nviews = (int)(sizeof(views) / sizeof(views[0]));
    // times one candidate unit shape of one kind on its own kernel
    auto time_shape = [&](int kind, int c, int vpu, float& ms) -> ctfp_status {
        b->tile_u[kind] = shapes[c][0];
        b->tile_v[kind] = shapes[c][1] * (kind ? 1 : 2);
        b->vpu[kind] = vpu;
        layout_units(b, kind);
        ctfp_status rs = fill_items(b, kind);
        if (rs != CTFP_OK) return rs;
        for (int s = 0; s < b->n; s++) {
            ItemDesc& it = b->items[(size_t)s];
            it.I_target = I_target[b->order[(size_t)s]];
            it.loss = kind ? loss + b->order[(size_t)s] : nullptr;
            it.I = nullptr;  // the forward's outputs go nowhere while tuning
            it.IAbs = nullptr;
            it.L = nullptr;
        }
        BATCH_CUDA(cudaStreamSynchronize(st));
        BATCH_CUDA(cudaMemcpy(b->d_items[kind], b->items.data(), sizeof(ItemDesc) * (size_t)b->n,
                              cudaMemcpyHostToDevice));
        rs = record(b, kind == 1, vols, kind ? loss : nullptr, st, 8);  // warm-up
        if (rs != CTFP_OK) return rs;
        BATCH_CUDA(cudaEventRecord(e0, st));
        rs = record(b, kind == 1, vols, kind ? loss : nullptr, st, 8);
        if (rs != CTFP_OK) return rs;
        BATCH_CUDA(cudaEventRecord(e1, st));
        BATCH_CUDA(cudaEventSynchronize(e1));
        BATCH_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return CTFP_OK;
    };
    int best[2] = {-1, -1}, best_vpu[2] = {b->vpu[0], b->vpu[1]};
    float best_ms[2] = {0.f, 0.f};
    // each kind of call on its own kernel, the forward, then the fused forward
    // + adjoint: the tiles at the kind's current views per unit, then the
    // views per unit with the fastest tile
    for (int kind = 0; kind < 2; kind++) {
        const int vpu0 = b->vpu[kind];
        for (int c = 0; c < nshapes; c++) {
            float ms = 0.f;
            const ctfp_status rs = time_shape(kind, c, vpu0, ms);
            if (rs != CTFP_OK) return rs;
            if (best[kind] < 0 || ms < best_ms[kind]) {
                best[kind] = c;
                best_ms[kind] = ms;
            }
        }
        for (int j = 0; j < nviews; j++) {
            if (views[j] == vpu0) continue;
            float ms = 0.f;
            const ctfp_status rs = time_shape(kind, best[kind], views[j], ms);
            if (rs != CTFP_OK) return rs;
            if (ms < best_ms[kind]) {
                best_vpu[kind] = views[j];
                best_ms[kind] = ms;
            }
        }
    }
    // graphs recorded with the old queues may still be running
    BATCH_CUDA(cudaDeviceSynchronize());
    for (ctfp_batch::Graph& G : b->graph) {
        if (G.exec) cudaGraphExecDestroy(G.exec);
        G.exec = nullptr;
    }
    for (int kind = 0; kind < 2; kind++) {
        b->tile_u[kind] = shapes[best[kind]][0];
        b->tile_v[kind] = shapes[best[kind]][1] * (kind ? 1 : 2);
        b->vpu[kind] = best_vpu[kind];
    }
    layout_units(b, 0);
    if (out) {
        out->tile_u = shapes[best[1]][0];
        out->tile_v = shapes[best[1]][1];
        out->views_per_cta = best_vpu[1];
        out->min_ctas_per_sm = 0;
        out->ms = best_ms[1];
        out->from_cache = 0;
    }
    return CTFP_OK;
}

ctfp_status ctfp_batch_get_shapes(const ctfp_batch* b, int32_t* fwd_tile_u, int32_t* fwd_tile_v,
                                  int32_t* adj_tile_u, int32_t* adj_tile_v)
{
    if (!b) return bfail(CTFP_INVALID_ARG, "batch is NULL");
    if (fwd_tile_u) *fwd_tile_u = b->tile_u[0];
    if (fwd_tile_v) *fwd_tile_v = b->tile_v[0];
    if (adj_tile_u) *adj_tile_u = b->tile_u[1];
    if (adj_tile_v) *adj_tile_v = b->tile_v[1];
    return CTFP_OK;
}

ctfp_status ctfp_batch_info(const ctfp_batch* b, int64_t* total_units, int32_t* grid_forward, int32_t* grid_adjoint)
{
    if (!b) return bfail(CTFP_INVALID_ARG, "batch is NULL");
    if (total_units) *total_units = b->total_units;
    int g0 = 0, g1 = 0;
    for (const ctfp_batch::Group& G : b->groups) {
        g0 = std::max(g0, G.grid[0]);
        g1 = std::max(g1, G.grid[1]);
    }
    if (grid_forward) *grid_forward = g0;
    if (grid_adjoint) *grid_adjoint = g1;
    return CTFP_OK;
}

}  // extern "C"
