// ctfp_api.cu — the extern "C" boundary declared in include/ctfp.h.
//
// Ownership: the caller owns every buffer it passes (volumes, outputs,
// checkpoints, gradients).  A plan owns its tables (view trigonometry, energy
// weights W[E][V][U], flat field I0, attenuation table) and, in texture mode,
// one cudaArray + texture object per material.  No call resets the device and
// none exits: every failure is a ctfp_status plus a per-thread message.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/ctfp.h"
#include "ctfp_kernels.cuh"

using namespace ctfp;

struct ctfp_plan {
    ctfp_geometry geom{};
    ctfp_system_info info{};
    int M = 0;
    int interp = 0;
    int device = 0;
    GeomParams gp{};
    double2* d_trig = nullptr;  // [P] (cos, sin) of the FP32 view angles
    float2* d_trigf = nullptr;  // [P] the same rounded to FP32 (compat samplers)
    // spectral tables
    int E = 0;
    bool spectral_ready = false;
    float* d_mu = nullptr;  // [E][M]
    float* d_W = nullptr;   // [E][V][U]
    float* d_I0 = nullptr;  // [V][U]
    // texture mode
    cudaArray_t arr[kMaxM] = {};
    cudaTextureObject_t tex[kMaxM] = {};
    // layered-gather sampler for the software modes
    int sampler = SAMPLER_LAYERED;
    cudaArray_t larr[kMaxM] = {};
    cudaTextureObject_t ltex[kMaxM] = {};
    // axis sampler: copies layered along x and along y, written through surfaces
    cudaArray_t xarr[kMaxM] = {}, yarr[kMaxM] = {};
    cudaTextureObject_t xtex[kMaxM] = {}, ytex[kMaxM] = {};
    cudaSurfaceObject_t xsurf[kMaxM] = {}, ysurf[kMaxM] = {};
    LaunchShape shape{};
    unsigned long long* d_count = nullptr;
    // empty-space skipping (off by default): brick occupancy, rebuilt from the
    // volumes at every call
    bool skip_empty = false;
    uint8_t* d_occ = nullptr;
    // device status word written by kernels whose bounded waits ran out
    unsigned* d_status = nullptr;
    // focal spot (off unless set): per-view offsets, and the march's raw
    // line integrals before the re-alignment (grown on demand)
    float2* d_fspot = nullptr;
    float* d_fs_raw = nullptr;
    size_t fs_raw_elems = 0;
    float* d_fs_L = nullptr;
    size_t fs_L_elems = 0;
    // corner-expanded adjoint accumulators (allocated on first backward)
    float4* d_gexp[kMaxM] = {};
    // staging for ctfp_forward_host
    float* h2d_vol[kMaxM] = {};
    float* d2h_I = nullptr;
    float* d2h_IAbs = nullptr;
    // ctfp_forward_host pipelining: results of finished view chunks go back
    // on a second stream while later chunks are marched; the chunks alternate
    // between the caller's stream and march_stream, so each chunk's last wave
    // of CTAs overlaps the next chunk's first
    cudaStream_t copy_stream = nullptr;
    cudaStream_t march_stream = nullptr;
    cudaEvent_t prepared = nullptr;
    cudaEvent_t chunk_done[16] = {};
    cudaEvent_t copies_done = nullptr;
};

namespace {

thread_local std::string g_last_error;

ctfp_status fail(ctfp_status st, const std::string& msg)
{
    g_last_error = msg;
    return st;
}

ctfp_status cuda_fail(cudaError_t e, const char* what)
{
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? CTFP_OOM : CTFP_CUDA_ERROR;
}

#define CTFP_CUDA(call)                                   \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

// Keeps the caller's current device and switches to the plan's for one call.
struct DeviceScope {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceScope(int dev)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) err = cudaSetDevice(dev);
    }
    ~DeviceScope()
    {
        if (prev >= 0) {
            int cur = -1;
            if (cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
        }
    }
};

ctfp_status check_geometry(const ctfp_geometry* g)
{
    if (!g) return fail(CTFP_INVALID_ARG, "geometry is NULL");
    if (g->pNumX <= 0 || g->pNumY <= 0 || g->pNumZ <= 0)
        return fail(CTFP_INVALID_ARG, "pNumX/pNumY/pNumZ must be positive");
    if ((double)g->pNumX * (double)g->pNumY * (double)g->pNumZ >= 2147483647.0)
        return fail(CTFP_UNSUPPORTED, "volume must hold fewer than 2^31 voxels");
    if (!(g->pLengthX > 0.f && g->pLengthY > 0.f && g->pLengthZ > 0.f))
        return fail(CTFP_INVALID_ARG, "pLengthX/pLengthY/pLengthZ must be positive");
    if (g->projNum <= 0 || g->projNum > 1000000) return fail(CTFP_INVALID_ARG, "projNum out of range");
    if (g->dNumU <= 0 || g->dNumV <= 0 || g->dNumU > 65535 || g->dNumV > 65535)
        return fail(CTFP_INVALID_ARG, "dNumU/dNumV out of range");
    if (!(g->dSize > 0.f)) return fail(CTFP_INVALID_ARG, "dSize must be positive");
    if (!(g->sod > 0.f) || !(g->sdd > g->sod)) return fail(CTFP_INVALID_ARG, "need 0 < sod < sdd");
    if (g->rotatedDirection != 1 && g->rotatedDirection != -1)
        return fail(CTFP_INVALID_ARG, "rotatedDirection must be +1 or -1");
    if (g->reserved != 0) return fail(CTFP_INVALID_ARG, "reserved must be 0");
    return CTFP_OK;
}

void compute_paras(const ctfp_geometry* g, ctfp_system_info* s)
{
    // CBCTForwardProj::computeParas (CBCTForwardProj.cpp:28-60), FP32 in the
    // reference's order. Every product is stored through a volatile float
    // before it is added, so no multiply-add contraction changes the result.
    std::memset(s, 0, sizeof(*s));
    volatile float t;
    s->thetaStep = (float)360 / (float)g->projNum;
    s->dHalfLU = (float)g->dNumU * g->dSize / 2;
    s->dHalfLV = (float)g->dNumV * g->dSize / 2;
    t = s->dHalfLU * s->dHalfLU;
    volatile float t2 = g->sdd * g->sdd;
    float rad = sqrtf(t + t2);
    t = g->sod * s->dHalfLU;
    s->FOVR = t / rad;
    t = (g->sod - s->FOVR) * s->dHalfLV;
    s->FOVH = t / g->sdd;
    s->pSizeX = g->pLengthX / (float)g->pNumX;
    s->pSizeY = g->pLengthY / (float)g->pNumY;
    s->pSizeZ = g->pLengthZ / (float)g->pNumZ;
    s->pHalfX = g->pLengthX / 2;
    s->pHalfY = g->pLengthY / 2;
    s->pHalfZ = g->pLengthZ / 2;
    s->dx = (float)(0.5 * s->pSizeX);
    s->dy = (float)(0.5 * s->pSizeY);
    s->dz = (float)(0.5 * s->pSizeZ);
    t = 2 * s->FOVR;
    s->intNum = (int64_t)roundf(t / s->dx);
}

float view_angle(const ctfp_geometry* g, const ctfp_system_info* s, int64_t p)
{
    // CBCTPolyProjGPU.cu:51 with PI = acosf(-1) (CBCTPolyProjGPU.cuh:21). The
    // reference's size_t product wraps for rotatedDirection = -1 and gives every
    // view the same angle; the intended signed angle is used instead.
    volatile float a = (float)p * s->thetaStep;
    a = a / 180.0f;
    a = a * acosf(-1.0f);
    return g->rotatedDirection < 0 ? -a : a;
}

bool valid_interp(int i) { return i == INTERP_TRILINEAR || i == INTERP_TEXEMU || i == INTERP_TEXTURE; }

ctfp_status make_textures(ctfp_plan* p)
{
    cudaChannelFormatDesc cd = cudaCreateChannelDesc<float>();
    cudaExtent ext = make_cudaExtent((size_t)p->geom.pNumX, (size_t)p->geom.pNumY, (size_t)p->geom.pNumZ);
    for (int m = 0; m < p->M; m++) {
        if (p->arr[m]) continue;
        CTFP_CUDA(cudaMalloc3DArray(&p->arr[m], &cd, ext));
        cudaResourceDesc rd;
        std::memset(&rd, 0, sizeof(rd));
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = p->arr[m];
        cudaTextureDesc td;
        std::memset(&td, 0, sizeof(td));
        td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
        td.filterMode = cudaFilterModeLinear;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 0;
        CTFP_CUDA(cudaCreateTextureObject(&p->tex[m], &rd, &td, nullptr));
    }
    return CTFP_OK;
}

// One layered 2D array per material (a layer per z slice), read by tld4.
ctfp_status make_layered(ctfp_plan* p)
{
    cudaChannelFormatDesc cd = cudaCreateChannelDesc<float>();
    cudaExtent ext = make_cudaExtent((size_t)p->geom.pNumX, (size_t)p->geom.pNumY, (size_t)p->geom.pNumZ);
    for (int m = 0; m < p->M; m++) {
        if (p->larr[m]) continue;
        CTFP_CUDA(cudaMalloc3DArray(&p->larr[m], &cd, ext, cudaArrayLayered));
        cudaResourceDesc rd;
        std::memset(&rd, 0, sizeof(rd));
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = p->larr[m];
        cudaTextureDesc td;
        std::memset(&td, 0, sizeof(td));
        td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
        td.filterMode = cudaFilterModePoint;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 0;
        CTFP_CUDA(cudaCreateTextureObject(&p->ltex[m], &rd, &td, nullptr));
    }
    return CTFP_OK;
}

// Layered array (width x height texels, `layers` layers) with a point-filter,
// border-addressed texture object and a surface object for writing it.
ctfp_status make_layered_rw(size_t width, size_t height, size_t layers, cudaArray_t& arr, cudaTextureObject_t& tex,
                            cudaSurfaceObject_t& surf)
{
    cudaChannelFormatDesc cd = cudaCreateChannelDesc<float>();
    CTFP_CUDA(cudaMalloc3DArray(&arr, &cd, make_cudaExtent(width, height, layers),
                                cudaArrayLayered | cudaArraySurfaceLoadStore));
    cudaResourceDesc rd;
    std::memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td;
    std::memset(&td, 0, sizeof(td));
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
    td.filterMode = cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    CTFP_CUDA(cudaCreateTextureObject(&tex, &rd, &td, nullptr));
    CTFP_CUDA(cudaCreateSurfaceObject(&surf, &rd));
    return CTFP_OK;
}

// The axis sampler's two copies per material: layered along x (texels
// (y, z), texture layer x + 1) and along y (texels (x, z), layer y + 1), each
// with a zero layer before and after the volume.
ctfp_status make_axis(ctfp_plan* p)
{
    const size_t nx = (size_t)p->geom.pNumX, ny = (size_t)p->geom.pNumY, nz = (size_t)p->geom.pNumZ;
    for (int m = 0; m < p->M; m++) {
        if (p->xarr[m]) continue;
        ctfp_status st = make_layered_rw(ny, nz, nx + 2, p->xarr[m], p->xtex[m], p->xsurf[m]);
        if (st == CTFP_OK) st = make_layered_rw(nx, nz, ny + 2, p->yarr[m], p->ytex[m], p->ysurf[m]);
        if (st != CTFP_OK) return st;
        CTFP_CUDA(launch_axis_zero_pads((int)nx, (int)ny, (int)nz, p->xsurf[m], p->ysurf[m], 0));
        CTFP_CUDA(cudaStreamSynchronize(0));
    }
    return CTFP_OK;
}

// two pad layers each: at most 2046 voxel layers along x and y
bool axis_fits(const ctfp_geometry& g) { return g.pNumX <= 2046 && g.pNumY <= 2046 && g.pNumZ <= 32768; }

void free_textures(ctfp_plan* p)
{
    for (int m = 0; m < kMaxM; m++) {
        if (p->xsurf[m]) cudaDestroySurfaceObject(p->xsurf[m]);
        if (p->ysurf[m]) cudaDestroySurfaceObject(p->ysurf[m]);
        if (p->xtex[m]) cudaDestroyTextureObject(p->xtex[m]);
        if (p->ytex[m]) cudaDestroyTextureObject(p->ytex[m]);
        if (p->xarr[m]) cudaFreeArray(p->xarr[m]);
        if (p->yarr[m]) cudaFreeArray(p->yarr[m]);
        p->xsurf[m] = p->ysurf[m] = 0;
        p->xtex[m] = p->ytex[m] = 0;
        p->xarr[m] = p->yarr[m] = nullptr;
        if (p->tex[m]) cudaDestroyTextureObject(p->tex[m]);
        if (p->arr[m]) cudaFreeArray(p->arr[m]);
        if (p->ltex[m]) cudaDestroyTextureObject(p->ltex[m]);
        if (p->larr[m]) cudaFreeArray(p->larr[m]);
        p->tex[m] = 0;
        p->arr[m] = nullptr;
        p->ltex[m] = 0;
        p->larr[m] = nullptr;
    }
}

bool uses_layered(const ctfp_plan* p) { return p->interp != INTERP_TEXTURE && p->sampler == SAMPLER_LAYERED; }
bool uses_axis(const ctfp_plan* p) { return p->interp != INTERP_TEXTURE && p->sampler == SAMPLER_AXIS; }

// Refreshes the plan's arrays (3D for TEXTURE, layered for the layered
// sampler) from the caller's linear volumes; no-op for the global sampler.
ctfp_status upload_textures(ctfp_plan* p, const float* const* volumes, cudaStream_t st)
{
    const bool tex3d = p->interp == INTERP_TEXTURE;
    if (uses_axis(p)) {
        for (int m = 0; m < p->M; m++)
            CTFP_CUDA(launch_axis_fill(volumes[m], (int)p->geom.pNumX, (int)p->geom.pNumY, (int)p->geom.pNumZ,
                                       p->xsurf[m], p->ysurf[m], st));
        return CTFP_OK;
    }
    if (!tex3d && !uses_layered(p)) return CTFP_OK;
    for (int m = 0; m < p->M; m++) {
        cudaMemcpy3DParms cp;
        std::memset(&cp, 0, sizeof(cp));
        cp.srcPtr = make_cudaPitchedPtr((void*)volumes[m], (size_t)p->geom.pNumX * sizeof(float),
                                        (size_t)p->geom.pNumX, (size_t)p->geom.pNumY);
        cp.dstArray = tex3d ? p->arr[m] : p->larr[m];
        cp.extent = make_cudaExtent((size_t)p->geom.pNumX, (size_t)p->geom.pNumY, (size_t)p->geom.pNumZ);
        cp.kind = cudaMemcpyDeviceToDevice;
        CTFP_CUDA(cudaMemcpy3DAsync(&cp, st));
    }
    return CTFP_OK;
}

// Polls of a TMA completion before a CTA of the TMA-staged brick sampler gives
// up staging (a completion normally takes a few microseconds; the default
// bounds the wait near a millisecond).  CTFP_WAIT_LIMIT overrides it.
int wait_limit()
{
    const char* e = std::getenv("CTFP_WAIT_LIMIT");
    if (e && *e) return std::max(0, std::atoi(e));
    return 1 << 16;
}

MarchParams base_params(const ctfp_plan* p)
{
    MarchParams prm;
    std::memset(&prm, 0, sizeof(prm));
    prm.g = p->gp;
    prm.E = p->E;
    prm.mu = p->d_mu;
    prm.W = p->d_W;
    prm.view0 = 0;
    prm.n_views = (int)p->geom.projNum;
    for (int m = 0; m < kMaxM; m++) {
        prm.tex[m] = p->tex[m];
        prm.ltex[m] = p->ltex[m];
        prm.xtex[m] = p->xtex[m];
        prm.ytex[m] = p->ytex[m];
    }
    if (p->skip_empty && p->d_occ) {
        prm.occ = p->d_occ;
        prm.occ_x = occ_dim(p->gp.nx);
        prm.occ_y = occ_dim(p->gp.ny);
    }
    prm.status = p->d_status;
    prm.wait_limit = wait_limit();
    return prm;
}

// Device scratch of at least n floats, grown on demand.
ctfp_status ensure_scratch(float*& ptr, size_t& have, size_t n)
{
    if (n <= have) return CTFP_OK;
    cudaFree(ptr);
    ptr = nullptr;
    have = 0;
    CTFP_CUDA(cudaMalloc(&ptr, n * sizeof(float)));
    have = n;
    return CTFP_OK;
}

// The march over views [view0, view0 + n) with a focal spot: raw line
// integrals into plan scratch, then the re-alignment into L (compact).
ctfp_status focal_spot_march(ctfp_plan* p, MarchParams prm, int64_t view0, int64_t n, float* L, cudaStream_t s)
{
    const size_t elems = (size_t)n * p->geom.dNumU * p->geom.dNumV * p->M;
    ctfp_status st = ensure_scratch(p->d_fs_raw, p->fs_raw_elems, elems);
    if (st != CTFP_OK) return st;
    prm.view0 = (int)view0;
    prm.n_views = (int)n;
    prm.out_view0 = (int)view0;
    prm.L = p->d_fs_raw;
    prm.I = nullptr;
    prm.IAbs = nullptr;
    prm.occ = nullptr;  // the image shift reads neighbouring rays: march them all
    CTFP_CUDA(launch_forward(prm, p->M, p->interp, p->sampler, false, p->shape, s));
    CTFP_CUDA(launch_shift_views(p->d_fs_raw, L, p->gp, p->M, p->interp, (int)view0, (int)n, s));
    return CTFP_OK;
}

// Sampler copies of the caller's volumes and, with empty-space skipping, the
// brick occupancy, on stream st.
ctfp_status prepare_volumes(ctfp_plan* p, const float* const* volumes, cudaStream_t st)
{
    ctfp_status rs = upload_textures(p, volumes, st);
    if (rs != CTFP_OK) return rs;
    if (p->skip_empty && p->d_occ)
        CTFP_CUDA(launch_occupancy(volumes, p->M, p->gp.nx, p->gp.ny, p->gp.nz, p->d_occ, st));
    return CTFP_OK;
}

// Zeroed corner-expanded accumulators for one adjoint launch.
ctfp_status prepare_expanded(ctfp_plan* p, MarchParams& prm, cudaStream_t st)
{
    const size_t n = expanded_elems(p->gp);
    for (int m = 0; m < p->M; m++) {
        if (!p->d_gexp[m]) CTFP_CUDA(cudaMalloc(&p->d_gexp[m], n * sizeof(float4)));
        CTFP_CUDA(cudaMemsetAsync(p->d_gexp[m], 0, n * sizeof(float4), st));
        prm.gexp[m] = p->d_gexp[m];
    }
    return CTFP_OK;
}

ctfp_status check_volumes(const ctfp_plan* p, const float* const* volumes)
{
    if (!volumes) return fail(CTFP_INVALID_ARG, "volumes is NULL");
    for (int m = 0; m < p->M; m++)
        if (!volumes[m]) return fail(CTFP_INVALID_ARG, "volume pointer is NULL");
    return CTFP_OK;
}

}  // namespace

extern "C" {

const char* ctfp_last_error_string(void) { return g_last_error.c_str(); }

ctfp_status ctfp_plan_check_status(ctfp_plan* p, uint32_t* flags)
{
    if (!p) return fail(CTFP_INVALID_ARG, "plan is NULL");
    DeviceScope ds(p->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "cudaSetDevice");
    CTFP_CUDA(cudaDeviceSynchronize());
    unsigned v = 0;
    CTFP_CUDA(cudaMemcpy(&v, p->d_status, sizeof(v), cudaMemcpyDeviceToHost));
    CTFP_CUDA(cudaMemset(p->d_status, 0, sizeof(v)));
    if (flags) *flags = v;
    if (v & kCtfpStatusExitWaitTimeout)
        return fail(CTFP_CUDA_ERROR,
                    "a TMA-staged brick load was still in flight when its CTA exited: outputs since the last check "
                    "and the shared memory of CTAs resident with it may be corrupt");
    if (v & kCtfpStatusWaitTimeout)
        return fail(CTFP_TIMEOUT, "a TMA-staged brick wait ran out; those samples were read from the volume");
    return CTFP_OK;
}

const char* ctfp_version(void) { return "ctfp 0.1.0 (sm_100a)"; }

ctfp_status ctfp_compute_paras(const ctfp_geometry* g, ctfp_system_info* out)
{
    ctfp_status st = check_geometry(g);
    if (st != CTFP_OK) return st;
    if (!out) return fail(CTFP_INVALID_ARG, "out is NULL");
    compute_paras(g, out);
    return CTFP_OK;
}

ctfp_status ctfp_view_angle(const ctfp_geometry* g, int64_t view, float* angle)
{
    ctfp_status st = check_geometry(g);
    if (st != CTFP_OK) return st;
    if (!angle || view < 0 || view >= g->projNum) return fail(CTFP_INVALID_ARG, "bad view or NULL angle");
    ctfp_system_info s;
    compute_paras(g, &s);
    *angle = view_angle(g, &s, view);
    return CTFP_OK;
}

ctfp_status ctfp_plan_create(const ctfp_geometry* g, int32_t n_materials, int32_t interp, int32_t device,
                             ctfp_plan** out)
{
    if (!out) return fail(CTFP_INVALID_ARG, "out is NULL");
    *out = nullptr;
    ctfp_status st = check_geometry(g);
    if (st != CTFP_OK) return st;
    if (n_materials < 1 || n_materials > CTFP_MAX_MATERIALS)
        return fail(CTFP_INVALID_ARG, "n_materials must be in [1, 4]");
    if (!valid_interp(interp)) return fail(CTFP_INVALID_ARG, "unknown interp mode");
    ctfp_system_info info;
    compute_paras(g, &info);
    if (info.intNum <= 0 || info.intNum > 100000000) return fail(CTFP_INVALID_ARG, "intNum out of range");
    DeviceScope ds(device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "cudaSetDevice");
    ctfp_plan* p = new (std::nothrow) ctfp_plan();
    if (!p) return fail(CTFP_OOM, "host allocation failed");
    p->geom = *g;
    p->info = info;
    p->M = n_materials;
    p->interp = interp;
    p->device = device;
    GeomParams& gp = p->gp;
    gp.nx = (int)g->pNumX; gp.ny = (int)g->pNumY; gp.nz = (int)g->pNumZ;
    gp.U = (int)g->dNumU; gp.V = (int)g->dNumV; gp.P = (int)g->projNum;
    gp.K = (int)info.intNum;
    gp.dHalfLU = info.dHalfLU; gp.dHalfLV = info.dHalfLV; gp.dSize = g->dSize;
    gp.sod = g->sod; gp.sdd = g->sdd; gp.FOVR = info.FOVR; gp.dx = info.dx;
    gp.pHalfX = info.pHalfX; gp.pHalfY = info.pHalfY; gp.pHalfZ = info.pHalfZ;
    gp.pSizeX = info.pSizeX; gp.pSizeY = info.pSizeY; gp.pSizeZ = info.pSizeZ;
    gp.rpSizeX = 1.0f / info.pSizeX; gp.rpSizeY = 1.0f / info.pSizeY; gp.rpSizeZ = 1.0f / info.pSizeZ;
    std::vector<double2> trig((size_t)g->projNum);
    std::vector<float2> trigf((size_t)g->projNum);
    for (int64_t k = 0; k < g->projNum; k++) {
        const double a = (double)view_angle(g, &info, k);
        trig[(size_t)k] = make_double2(std::cos(a), std::sin(a));
        trigf[(size_t)k] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    cudaError_t e = cudaMalloc(&p->d_trig, sizeof(double2) * trig.size());
    if (e == cudaSuccess) e = cudaMemcpy(p->d_trig, trig.data(), sizeof(double2) * trig.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_trigf, sizeof(float2) * trigf.size());
    if (e == cudaSuccess)
        e = cudaMemcpy(p->d_trigf, trigf.data(), sizeof(float2) * trigf.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_count, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&p->d_status, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(p->d_status, 0, sizeof(unsigned));
    if (e != cudaSuccess) {
        ctfp_plan_destroy(p);
        return cuda_fail(e, "plan allocation");
    }
    gp.trig = p->d_trig;
    gp.trigf = p->d_trigf;
    // default corner source: the axis sampler (fastest measured); layered
    // textures hold at most 2048 layers, so past its limits the z-layered
    // sampler, past those the caller's volumes
    p->sampler = axis_fits(*g) ? SAMPLER_AXIS : (g->pNumZ <= 2048 ? SAMPLER_LAYERED : SAMPLER_GLOBAL);
    if (uses_layered(p) || uses_axis(p)) {
        st = uses_axis(p) ? make_axis(p) : make_layered(p);
        if (st != CTFP_OK) {
            std::string msg = g_last_error;
            ctfp_plan_destroy(p);
            return fail(st, msg);
        }
    }
    if (interp == INTERP_TEXTURE) {
        st = make_textures(p);
        if (st != CTFP_OK) {
            std::string msg = g_last_error;
            ctfp_plan_destroy(p);
            return fail(st, msg);
        }
    }
    *out = p;
    return CTFP_OK;
}

ctfp_status ctfp_plan_destroy(ctfp_plan* p)
{
    if (!p) return CTFP_OK;
    DeviceScope ds(p->device);
    free_textures(p);
    cudaFree(p->d_trig);
    cudaFree(p->d_trigf);
    cudaFree(p->d_mu);
    cudaFree(p->d_W);
    cudaFree(p->d_I0);
    cudaFree(p->d_count);
    for (int m = 0; m < kMaxM; m++) cudaFree(p->h2d_vol[m]);
    for (int m = 0; m < kMaxM; m++) cudaFree(p->d_gexp[m]);
    cudaFree(p->d_occ);
    cudaFree(p->d_status);
    for (cudaEvent_t& e : p->chunk_done)
        if (e) cudaEventDestroy(e);
    if (p->copies_done) cudaEventDestroy(p->copies_done);
    if (p->prepared) cudaEventDestroy(p->prepared);
    if (p->copy_stream) cudaStreamDestroy(p->copy_stream);
    if (p->march_stream) cudaStreamDestroy(p->march_stream);
    cudaFree(p->d_fspot);
    cudaFree(p->d_fs_raw);
    cudaFree(p->d_fs_L);
    cudaFree(p->d2h_I);
    cudaFree(p->d2h_IAbs);
    delete p;
    return CTFP_OK;
}

ctfp_status ctfp_plan_get_system_info(const ctfp_plan* p, ctfp_system_info* out)
{
    if (!p || !out) return fail(CTFP_INVALID_ARG, "NULL argument");
    *out = p->info;
    return CTFP_OK;
}

ctfp_status ctfp_plan_set_interp(ctfp_plan* p, int32_t interp)
{
    if (!p) return fail(CTFP_INVALID_ARG, "plan is NULL");
    if (!valid_interp(interp)) return fail(CTFP_INVALID_ARG, "unknown interp mode");
    DeviceScope ds(p->device);
    if (interp == INTERP_TEXTURE) {
        ctfp_status st = make_textures(p);
        if (st != CTFP_OK) return st;
    }
    p->interp = interp;
    if (uses_layered(p)) return make_layered(p);
    if (uses_axis(p)) return make_axis(p);
    return CTFP_OK;
}

ctfp_status ctfp_plan_set_sampler(ctfp_plan* p, int32_t sampler)
{
    if (!p) return fail(CTFP_INVALID_ARG, "plan is NULL");
    if (sampler != CTFP_SAMPLER_GLOBAL && sampler != CTFP_SAMPLER_LAYERED && sampler != CTFP_SAMPLER_BRICK &&
        sampler != CTFP_SAMPLER_AXIS)
        return fail(CTFP_INVALID_ARG, "unknown sampler");
    if (sampler == CTFP_SAMPLER_LAYERED && p->geom.pNumZ > 2048)
        return fail(CTFP_UNSUPPORTED, "layered sampler holds at most 2048 z slices");
    if (sampler == CTFP_SAMPLER_AXIS && !axis_fits(p->geom))
        return fail(CTFP_UNSUPPORTED, "axis sampler needs pNumX, pNumY <= 2046 and pNumZ <= 32768");
    DeviceScope ds(p->device);
    p->sampler = sampler;
    if (uses_layered(p)) return make_layered(p);
    if (uses_axis(p)) return make_axis(p);
    return CTFP_OK;
}

ctfp_status ctfp_set_spectral_tables(ctfp_plan* p, int32_t E, const float* spectrum, const float* mu,
                                     const float* grid, int32_t grid_layout, const float* det_response, float I0Val)
{
    if (!p) return fail(CTFP_INVALID_ARG, "plan is NULL");
    if (E < 1 || E > CTFP_MAX_ENERGIES) return fail(CTFP_INVALID_ARG, "n_energies must be in [1, 256]");
    if (!spectrum || !mu) return fail(CTFP_INVALID_ARG, "spectrum and mu are required");
    if (grid_layout < 0 || grid_layout > 2) return fail(CTFP_INVALID_ARG, "unknown grid layout");
    if (grid_layout != 0 && !grid) return fail(CTFP_INVALID_ARG, "grid table is NULL");
    if (!(I0Val >= 0.f)) return fail(CTFP_INVALID_ARG, "I0Val must be non-negative");
    DeviceScope ds(p->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "cudaSetDevice");
    const int64_t U = p->geom.dNumU, V = p->geom.dNumV, npix = U * V;
    const size_t nG = grid_layout == 1 ? (size_t)E * U : grid_layout == 2 ? (size_t)E * npix : 0;
    const size_t nD = det_response ? (size_t)E * npix : 0;
    float *dS = nullptr, *dG = nullptr, *dD = nullptr;
    cudaFree(p->d_mu); p->d_mu = nullptr;
    cudaFree(p->d_W); p->d_W = nullptr;
    cudaFree(p->d_I0); p->d_I0 = nullptr;
    p->spectral_ready = false;
    cudaError_t e = cudaMalloc(&p->d_mu, sizeof(float) * (size_t)E * p->M);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_W, sizeof(float) * (size_t)E * npix);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_I0, sizeof(float) * (size_t)npix);
    if (e == cudaSuccess) e = cudaMalloc(&dS, sizeof(float) * (size_t)E);
    if (e == cudaSuccess && nG) e = cudaMalloc(&dG, sizeof(float) * nG);
    if (e == cudaSuccess && nD) e = cudaMalloc(&dD, sizeof(float) * nD);
    if (e == cudaSuccess) e = cudaMemcpy(p->d_mu, mu, sizeof(float) * (size_t)E * p->M, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dS, spectrum, sizeof(float) * (size_t)E, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nG) e = cudaMemcpy(dG, grid, sizeof(float) * nG, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nD) e = cudaMemcpy(dD, det_response, sizeof(float) * nD, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launch_weights(dS, dG, grid_layout, dD, I0Val, E, (int)U, (int)V, p->d_W, p->d_I0, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaFree(dS);
    cudaFree(dG);
    cudaFree(dD);
    if (e != cudaSuccess) return cuda_fail(e, "ctfp_set_spectral_tables");
    p->E = E;
    p->spectral_ready = true;
    return CTFP_OK;
}

ctfp_status ctfp_line_integrals(ctfp_plan* p, const float* const* volumes, float* L, void* stream)
{
    if (!p) return fail(CTFP_INVALID_ARG, "plan is NULL");
    ctfp_status st = check_volumes(p, volumes);
    if (st != CTFP_OK) return st;
    if (!L) return fail(CTFP_INVALID_ARG, "L is NULL");
    DeviceScope ds(p->device);
    cudaStream_t s = (cudaStream_t)stream;
    MarchParams prm = base_params(p);
    for (int m = 0; m < p->M; m++) prm.vol[m] = volumes[m];
    prm.L = L;
    st = prepare_volumes(p, volumes, s);
    if (st != CTFP_OK) return st;
    if (p->gp.fspot) return focal_spot_march(p, prm, 0, p->geom.projNum, L, s);
    CTFP_CUDA(launch_forward(prm, p->M, p->interp, p->sampler, false, p->shape, s));
    return CTFP_OK;
}

// The fused forward over views [view0, view0 + n_views); outputs hold those
// views from index 0 when compact, else are full [projNum] arrays.
static ctfp_status forward_range(ctfp_plan* p, const float* const* volumes, int64_t view0, int64_t n_views,
                                 bool compact, float* I, float* IAbsorb, float* I0, float* L_ckpt, void* stream,
                                 bool prepare = true)
{
    if (!p) return fail(CTFP_INVALID_ARG, "plan is NULL");
    ctfp_status st = check_volumes(p, volumes);
    if (st != CTFP_OK) return st;
    if (!p->spectral_ready) return fail(CTFP_NOT_READY, "spectral tables not set");
    if (view0 < 0 || n_views < 0 || view0 + n_views > p->geom.projNum)
        return fail(CTFP_INVALID_ARG, "view range outside [0, projNum)");
    DeviceScope ds(p->device);
    cudaStream_t s = (cudaStream_t)stream;
    MarchParams prm = base_params(p);
    for (int m = 0; m < p->M; m++) prm.vol[m] = volumes[m];
    prm.I = I;
    prm.IAbs = IAbsorb;
    prm.L = L_ckpt;
    prm.view0 = (int)view0;
    prm.n_views = (int)n_views;
    prm.out_view0 = compact ? (int)view0 : 0;
    if (prepare) {
        st = prepare_volumes(p, volumes, s);
        if (st != CTFP_OK) return st;
    }
    if (n_views > 0 && p->gp.fspot) {
        // focal spot: march, re-align the line-integral images, then the
        // spectral epilogue on the re-aligned integrals
        const int64_t npix = p->geom.dNumU * p->geom.dNumV;
        const int64_t skip = compact ? 0 : view0;
        float* Ldst = L_ckpt ? L_ckpt + skip * npix * p->M : nullptr;
        if (!Ldst) {
            st = ensure_scratch(p->d_fs_L, p->fs_L_elems, (size_t)n_views * npix * p->M);
            if (st != CTFP_OK) return st;
            Ldst = p->d_fs_L;
        }
        st = focal_spot_march(p, prm, view0, n_views, Ldst, s);
        if (st != CTFP_OK) return st;
        MarchParams sp = base_params(p);
        sp.g.P = (int)n_views;
        sp.Lin = Ldst;
        sp.I = I ? I + skip * npix : nullptr;
        sp.IAbs = IAbsorb ? IAbsorb + skip * npix : nullptr;
        CTFP_CUDA(launch_spectral_from_L(sp, p->M, s));
    } else if (n_views > 0) {
        CTFP_CUDA(launch_forward(prm, p->M, p->interp, p->sampler, true, p->shape, s));
    }
    if (I0)
        CTFP_CUDA(cudaMemcpyAsync(I0, p->d_I0, sizeof(float) * (size_t)(p->geom.dNumU * p->geom.dNumV),
                                  cudaMemcpyDeviceToDevice, s));
    return CTFP_OK;
}

ctfp_status ctfp_forward(ctfp_plan* p, const float* const* volumes, float* I, float* IAbsorb, float* I0,
                         float* L_ckpt, void* stream)
{
    return forward_range(p, volumes, 0, p ? p->geom.projNum : 0, false, I, IAbsorb, I0, L_ckpt, stream);
}

ctfp_status ctfp_forward_views(ctfp_plan* p, const float* const* volumes, int64_t view0, int64_t n_views, float* I,
                               float* IAbsorb, float* I0, float* L_ckpt, void* stream)
{
    return forward_range(p, volumes, view0, n_views, true, I, IAbsorb, I0, L_ckpt, stream);
}

ctfp_status ctfp_forward_host(ctfp_plan* p, const float* const* host_volumes, float* host_I, float* host_IAbsorb,
                              float* host_I0, void* stream)
{
    if (!p) return fail(CTFP_INVALID_ARG, "plan is NULL");
    ctfp_status st = check_volumes(p, host_volumes);
    if (st != CTFP_OK) return st;
    if (!host_I || !host_IAbsorb) return fail(CTFP_INVALID_ARG, "host_I and host_IAbsorb are required");
    if (!p->spectral_ready) return fail(CTFP_NOT_READY, "spectral tables not set");
    DeviceScope ds(p->device);
    cudaStream_t s = (cudaStream_t)stream;
    const size_t nvox = (size_t)p->geom.pNumX * p->geom.pNumY * p->geom.pNumZ;
    const size_t nray = (size_t)p->geom.projNum * p->geom.dNumU * p->geom.dNumV;
    for (int m = 0; m < p->M; m++)
        if (!p->h2d_vol[m]) CTFP_CUDA(cudaMalloc(&p->h2d_vol[m], nvox * sizeof(float)));
    if (!p->d2h_I) CTFP_CUDA(cudaMalloc(&p->d2h_I, nray * sizeof(float)));
    if (!p->d2h_IAbs) CTFP_CUDA(cudaMalloc(&p->d2h_IAbs, nray * sizeof(float)));
    const int kChunks = (int)(sizeof(p->chunk_done) / sizeof(p->chunk_done[0]));
    if (!p->copy_stream) CTFP_CUDA(cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking));
    if (!p->march_stream) CTFP_CUDA(cudaStreamCreateWithFlags(&p->march_stream, cudaStreamNonBlocking));
    for (cudaEvent_t& e : p->chunk_done)
        if (!e) CTFP_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    if (!p->copies_done) CTFP_CUDA(cudaEventCreateWithFlags(&p->copies_done, cudaEventDisableTiming));
    if (!p->prepared) CTFP_CUDA(cudaEventCreateWithFlags(&p->prepared, cudaEventDisableTiming));
    const float* dv[kMaxM] = {};
    for (int m = 0; m < p->M; m++) {
        CTFP_CUDA(cudaMemcpyAsync(p->h2d_vol[m], host_volumes[m], nvox * sizeof(float), cudaMemcpyHostToDevice, s));
        dv[m] = p->h2d_vol[m];
    }
    st = prepare_volumes(p, dv, s);
    if (st != CTFP_OK) return st;
    // the views in up to kChunks contiguous chunks: chunk c's results are
    // copied back on the copy stream while chunk c + 1 is marched.  Chunks
    // alternate between s and march_stream (they write disjoint views and
    // only read the prepared volumes); the focal-spot march shares one
    // scratch buffer between chunks, so it keeps them all on s.
    CTFP_CUDA(cudaEventRecord(p->prepared, s));
    // on every return, nothing of this call is left running on the plan's own
    // streams (an error part-way must not leave copies into the caller's
    // host buffers in flight)
    struct Drain {
        ctfp_plan* p;
        ~Drain()
        {
            cudaStreamSynchronize(p->march_stream);
            cudaStreamSynchronize(p->copy_stream);
        }
    } drain{p};
    const bool two = !p->gp.fspot;
    if (two) CTFP_CUDA(cudaStreamWaitEvent(p->march_stream, p->prepared, 0));
    // The last chunk's copy is the one the march cannot hide, so it is made a
    // quarter of the others: P - n_last views in kChunks - 1 chunks, then n_last.
    const int64_t P = p->geom.projNum, npix = p->geom.dNumU * p->geom.dNumV;
    const int64_t n_last = P >= 2 * kChunks ? std::max<int64_t>(1, (P + kChunks - 1) / kChunks / 4) : 0;
    const int64_t per = (P - n_last + kChunks - 2) / (kChunks - 1);
    int c = 0;
    for (int64_t v0 = 0; v0 < P; c++) {
        const int64_t n = v0 + per <= P - n_last ? per : (v0 < P - n_last ? P - n_last - v0 : P - v0);
        const int64_t v_start = v0;
        v0 += n;
        cudaStream_t cs = (two && (c & 1)) ? p->march_stream : s;
        st = forward_range(p, dv, v_start, n, false, p->d2h_I, p->d2h_IAbs, nullptr, nullptr, cs, false);
        if (st != CTFP_OK) return st;
        CTFP_CUDA(cudaEventRecord(p->chunk_done[c], cs));
        CTFP_CUDA(cudaStreamWaitEvent(p->copy_stream, p->chunk_done[c], 0));
        const size_t off = (size_t)(v_start * npix), bytes = (size_t)(n * npix) * sizeof(float);
        CTFP_CUDA(cudaMemcpyAsync(host_I + off, p->d2h_I + off, bytes, cudaMemcpyDeviceToHost, p->copy_stream));
        CTFP_CUDA(cudaMemcpyAsync(host_IAbsorb + off, p->d2h_IAbs + off, bytes, cudaMemcpyDeviceToHost,
                                  p->copy_stream));
    }
    if (host_I0)
        CTFP_CUDA(cudaMemcpyAsync(host_I0, p->d_I0, sizeof(float) * (size_t)npix, cudaMemcpyDeviceToHost,
                                  p->copy_stream));
    CTFP_CUDA(cudaEventRecord(p->copies_done, p->copy_stream));
    CTFP_CUDA(cudaStreamWaitEvent(s, p->copies_done, 0));
    CTFP_CUDA(cudaStreamSynchronize(s));
    return CTFP_OK;
}

ctfp_status ctfp_spectral_from_L(ctfp_plan* p, const float* L, float* I, float* IAbsorb, void* stream)
{
    if (!p || !L) return fail(CTFP_INVALID_ARG, "NULL argument");
    if (!p->spectral_ready) return fail(CTFP_NOT_READY, "spectral tables not set");
    DeviceScope ds(p->device);
    MarchParams prm = base_params(p);
    prm.Lin = L;
    prm.I = I;
    prm.IAbs = IAbsorb;
    CTFP_CUDA(launch_spectral_from_L(prm, p->M, (cudaStream_t)stream));
    return CTFP_OK;
}

ctfp_status ctfp_finalize_counts(int64_t n_pix, int64_t n_views, const float* I, const float* IAbsorb,
                                 const float* I0, uint32_t* Ipoly, uint32_t* IAbsPoly, float* proj, void* stream)
{
    if (n_pix < 0 || n_views < 0) return fail(CTFP_INVALID_ARG, "negative size");
    if (proj && (!I0 || !I)) return fail(CTFP_INVALID_ARG, "proj needs I and I0");
    CTFP_CUDA(launch_finalize(n_pix, n_views, I, IAbsorb, I0, Ipoly, IAbsPoly, proj, (cudaStream_t)stream));
    return CTFP_OK;
}

static ctfp_status backward_range(ctfp_plan* p, const float* L_ckpt, const float* gI, const float* gIAbsorb,
                                  int64_t view0, int64_t n_views, bool compact, float* const* g_volumes, void* stream)
{
    if (!p || !L_ckpt || !g_volumes) return fail(CTFP_INVALID_ARG, "NULL argument");
    if (!gI && !gIAbsorb) return fail(CTFP_INVALID_ARG, "need gI or gIAbsorb");
    if (!p->spectral_ready) return fail(CTFP_NOT_READY, "spectral tables not set");
    if (view0 < 0 || n_views < 0 || view0 + n_views > p->geom.projNum)
        return fail(CTFP_INVALID_ARG, "view range outside [0, projNum)");
    for (int m = 0; m < p->M; m++)
        if (!g_volumes[m]) return fail(CTFP_INVALID_ARG, "gradient volume pointer is NULL");
    if (p->gp.fspot) return fail(CTFP_UNSUPPORTED, "the adjoint does not model a focal spot");
    DeviceScope ds(p->device);
    MarchParams prm = base_params(p);
    prm.Lin = L_ckpt;
    prm.gI = gI;
    prm.gIAbs = gIAbsorb;
    prm.view0 = (int)view0;
    prm.n_views = (int)n_views;
    prm.out_view0 = compact ? (int)view0 : 0;
    for (int m = 0; m < p->M; m++) prm.gvol[m] = g_volumes[m];
    if (n_views == 0) return CTFP_OK;
    cudaStream_t s = (cudaStream_t)stream;
    ctfp_status st = prepare_expanded(p, prm, s);
    if (st != CTFP_OK) return st;
    CTFP_CUDA(launch_backward(prm, p->M, p->interp, false, p->shape, s));
    CTFP_CUDA(launch_fold(prm, p->M, s));
    return CTFP_OK;
}

ctfp_status ctfp_backward(ctfp_plan* p, const float* L_ckpt, const float* gI, const float* gIAbsorb,
                          float* const* g_volumes, void* stream)
{
    return backward_range(p, L_ckpt, gI, gIAbsorb, 0, p ? p->geom.projNum : 0, false, g_volumes, stream);
}

ctfp_status ctfp_backward_views(ctfp_plan* p, const float* L_ckpt, const float* gI, const float* gIAbsorb,
                                int64_t view0, int64_t n_views, float* const* g_volumes, void* stream)
{
    return backward_range(p, L_ckpt, gI, gIAbsorb, view0, n_views, true, g_volumes, stream);
}

ctfp_status ctfp_line_integrals_adjoint(ctfp_plan* p, const float* gL, float* const* g_volumes, void* stream)
{
    if (!p || !gL || !g_volumes) return fail(CTFP_INVALID_ARG, "NULL argument");
    for (int m = 0; m < p->M; m++)
        if (!g_volumes[m]) return fail(CTFP_INVALID_ARG, "gradient volume pointer is NULL");
    if (p->gp.fspot) return fail(CTFP_UNSUPPORTED, "the adjoint does not model a focal spot");
    DeviceScope ds(p->device);
    MarchParams prm = base_params(p);
    prm.Lin = gL;
    for (int m = 0; m < p->M; m++) prm.gvol[m] = g_volumes[m];
    cudaStream_t s = (cudaStream_t)stream;
    ctfp_status st = prepare_expanded(p, prm, s);
    if (st != CTFP_OK) return st;
    CTFP_CUDA(launch_backward(prm, p->M, p->interp, true, p->shape, s));
    CTFP_CUDA(launch_fold(prm, p->M, s));
    return CTFP_OK;
}

ctfp_status ctfp_sample_volume(const float* volume, int64_t nx, int64_t ny, int64_t nz, int32_t interp,
                               const float* points, int64_t n, float* out, void* stream)
{
    if (!volume || !points || !out || n < 0) return fail(CTFP_INVALID_ARG, "bad argument");
    if (nx <= 0 || ny <= 0 || nz <= 0 || (double)nx * ny * nz >= 2147483647.0)
        return fail(CTFP_INVALID_ARG, "bad volume size");
    if (!valid_interp(interp)) return fail(CTFP_INVALID_ARG, "unknown interp mode");
    cudaStream_t s = (cudaStream_t)stream;
    cudaArray_t arr = nullptr;
    cudaTextureObject_t tex = 0;
    if (interp == INTERP_TEXTURE) {
        cudaChannelFormatDesc cd = cudaCreateChannelDesc<float>();
        cudaExtent ext = make_cudaExtent((size_t)nx, (size_t)ny, (size_t)nz);
        CTFP_CUDA(cudaMalloc3DArray(&arr, &cd, ext));
        cudaMemcpy3DParms cp;
        std::memset(&cp, 0, sizeof(cp));
        cp.srcPtr = make_cudaPitchedPtr((void*)volume, (size_t)nx * sizeof(float), (size_t)nx, (size_t)ny);
        cp.dstArray = arr;
        cp.extent = ext;
        cp.kind = cudaMemcpyDeviceToDevice;
        cudaError_t e = cudaMemcpy3DAsync(&cp, s);
        cudaResourceDesc rd;
        std::memset(&rd, 0, sizeof(rd));
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = arr;
        cudaTextureDesc td;
        std::memset(&td, 0, sizeof(td));
        td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
        td.filterMode = cudaFilterModeLinear;
        td.readMode = cudaReadModeElementType;
        if (e == cudaSuccess) e = cudaCreateTextureObject(&tex, &rd, &td, nullptr);
        if (e != cudaSuccess) {
            cudaFreeArray(arr);
            return cuda_fail(e, "texture setup");
        }
    }
    cudaError_t e = launch_sample_points(volume, tex, (int)nx, (int)ny, (int)nz, interp, points, n, out, s);
    if (interp == INTERP_TEXTURE) {
        cudaError_t e2 = cudaStreamSynchronize(s);
        if (e == cudaSuccess) e = e2;
        cudaDestroyTextureObject(tex);
        cudaFreeArray(arr);
    }
    if (e != cudaSuccess) return cuda_fail(e, "ctfp_sample_volume");
    return CTFP_OK;
}

ctfp_status ctfp_axis_gather_count(ctfp_plan* p, double* quad_gathers_per_sample)
{
    if (!p || !quad_gathers_per_sample) return fail(CTFP_INVALID_ARG, "NULL argument");
    if (p->interp == INTERP_TEXTURE) return fail(CTFP_UNSUPPORTED, "the hardware texture mode has no gathers");
    DeviceScope ds(p->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "cudaSetDevice");
    unsigned long long* d = nullptr;
    CTFP_CUDA(cudaMalloc(&d, 2 * sizeof(unsigned long long)));
    unsigned long long h[2] = {0, 0};
    cudaError_t e = cudaMemset(d, 0, 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = launch_axis_gather_count(p->gp, p->interp, p->shape, d, 0);
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(e, "ctfp_axis_gather_count");
    *quad_gathers_per_sample = h[1] ? (double)h[0] / (double)h[1] : 0.0;
    return CTFP_OK;
}

ctfp_status ctfp_count_support_samples(ctfp_plan* p, int64_t* out)
{
    if (!p || !out) return fail(CTFP_INVALID_ARG, "NULL argument");
    DeviceScope ds(p->device);
    CTFP_CUDA(cudaMemset(p->d_count, 0, sizeof(unsigned long long)));
    CTFP_CUDA(launch_count_support(p->gp, p->d_count, 0));
    unsigned long long h = 0;
    CTFP_CUDA(cudaMemcpy(&h, p->d_count, sizeof(h), cudaMemcpyDeviceToHost));
    *out = (int64_t)h;
    return CTFP_OK;
}

}  // extern "C"

// Internal accessors for the other translation units.
namespace ctfp {
void set_last_error(const std::string& msg) { g_last_error = msg; }
const GeomParams& plan_geom(const ctfp_plan* p) { return p->gp; }
int plan_materials(const ctfp_plan* p) { return p->M; }
int plan_interp(const ctfp_plan* p) { return p->interp; }
int plan_sampler(const ctfp_plan* p) { return p->sampler; }
int plan_device(const ctfp_plan* p) { return p->device; }
int plan_energies(const ctfp_plan* p) { return p->spectral_ready ? p->E : 0; }
const float* plan_mu(const ctfp_plan* p) { return p->d_mu; }
const float* plan_W(const ctfp_plan* p) { return p->d_W; }
LaunchShape& plan_shape(ctfp_plan* p) { return p->shape; }
cudaTextureObject_t plan_ltex(const ctfp_plan* p, int m) { return p->ltex[m]; }
cudaTextureObject_t plan_xtex(const ctfp_plan* p, int m) { return p->xtex[m]; }
cudaTextureObject_t plan_ytex(const ctfp_plan* p, int m) { return p->ytex[m]; }
cudaTextureObject_t plan_tex(const ctfp_plan* p, int m) { return p->tex[m]; }
MarchParams plan_march_params(const ctfp_plan* p) { return base_params(p); }
const ctfp_geometry& plan_geometry(const ctfp_plan* p) { return p->geom; }
// Copies the caller's volumes into the plan's sampler arrays (layered or 3D) on stream st.
ctfp_status plan_upload(ctfp_plan* p, const float* const* volumes, cudaStream_t st)
{
    ctfp_status s = check_volumes(p, volumes);
    if (s != CTFP_OK) return s;
    return prepare_volumes(p, volumes, st);
}
}  // namespace ctfp

extern "C" ctfp_status ctfp_plan_set_focal_spot(ctfp_plan* p, const float* offset_u, const float* offset_v)
{
    if (!p) return fail(CTFP_INVALID_ARG, "plan is NULL");
    if (!offset_u != !offset_v) return fail(CTFP_INVALID_ARG, "give both offset arrays or neither");
    DeviceScope ds(p->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "cudaSetDevice");
    if (!offset_u) {
        p->gp.fspot = nullptr;
        return CTFP_OK;
    }
    const size_t P = (size_t)p->geom.projNum;
    std::vector<float2> f(P);
    for (size_t k = 0; k < P; k++) {
        if (!std::isfinite(offset_u[k]) || !std::isfinite(offset_v[k]))
            return fail(CTFP_INVALID_ARG, "focal-spot offsets must be finite");
        f[k] = make_float2(offset_u[k], offset_v[k]);
    }
    if (!p->d_fspot) CTFP_CUDA(cudaMalloc(&p->d_fspot, sizeof(float2) * P));
    CTFP_CUDA(cudaMemcpy(p->d_fspot, f.data(), sizeof(float2) * P, cudaMemcpyHostToDevice));
    p->gp.fspot = p->d_fspot;
    return CTFP_OK;
}

extern "C" ctfp_status ctfp_focal_spot_offsets(int64_t n_views, float focal_spot_size, float* offset_u,
                                               float* offset_v)
{
    if (n_views < 0 || !offset_u || !offset_v) return fail(CTFP_INVALID_ARG, "bad argument");
    if (!(focal_spot_size >= 0.f)) return fail(CTFP_INVALID_ARG, "focal_spot_size must be non-negative");
    // CBCTForwardProj::computeFoSpOffset (CBCTForwardProj.cpp:122-148): srand(10),
    // MSVC rand() (state * 214013 + 2531011, bits 16-30), offsets on a 1e-4 mm
    // lattice across the spot [-r, r), redrawn while u^2 + v^2 > pi * r^2 (the
    // reference's test: pi r^2, not r^2)
    uint32_t state = 10u;
    auto next = [&state]() {
        state = state * 214013u + 2531011u;
        return (int)((state >> 16) & 0x7fffu);
    };
    const float radius = focal_spot_size / 2.0f;
    const int size = (int)(focal_spot_size * 10000);
    const float pi = acosf(-1.0f);
    for (int64_t k = 0; k < n_views; k++) {
        float du = 0.f, dv = 0.f;
        if (size > 0) {
            const float bound = pi * radius * radius;
            do {
                du = -radius + (float)(next() % size) / 10000.0f;
                dv = -radius + (float)(next() % size) / 10000.0f;
            } while (du * du + dv * dv > bound);
        }
        offset_u[k] = du;
        offset_v[k] = dv;
    }
    return CTFP_OK;
}

extern "C" ctfp_status ctfp_plan_set_skip_empty(ctfp_plan* p, int32_t enable)
{
    if (!p) return fail(CTFP_INVALID_ARG, "plan is NULL");
    DeviceScope ds(p->device);
    if (ds.err != cudaSuccess) return cuda_fail(ds.err, "cudaSetDevice");
    if (enable && !p->d_occ) {
        const size_t n = (size_t)occ_dim(p->gp.nx) * occ_dim(p->gp.ny) * occ_dim(p->gp.nz);
        CTFP_CUDA(cudaMalloc(&p->d_occ, n));
    }
    p->skip_empty = enable != 0;
    return CTFP_OK;
}

extern "C" ctfp_status ctfp_plan_set_launch_shape(ctfp_plan* p, int32_t tile_u, int32_t tile_v, int32_t views_per_cta,
                                                  int32_t min_ctas_per_sm)
{
    if (!p) return fail(CTFP_INVALID_ARG, "plan is NULL");
    if (tile_u < 1 || tile_v < 1 || tile_u * tile_v > 256 || (tile_u * tile_v) % 32 != 0 || views_per_cta < 1)
        return fail(CTFP_INVALID_ARG, "tile_u*tile_v must be a multiple of 32 and at most 256");
    if (min_ctas_per_sm < 2 || min_ctas_per_sm > 5)
        return fail(CTFP_INVALID_ARG, "min_ctas_per_sm must be 2, 3, 4 or 5 (5: the axis sampler only; others use 4)");
    if (tile_u * tile_v * min_ctas_per_sm > 2048)
        return fail(CTFP_INVALID_ARG, "tile_u*tile_v*min_ctas_per_sm exceeds 2048 threads per SM");
    p->shape.tile_u = tile_u;
    p->shape.tile_v = tile_v;
    p->shape.views_per_cta = views_per_cta;
    p->shape.min_ctas = min_ctas_per_sm;
    return CTFP_OK;
}
