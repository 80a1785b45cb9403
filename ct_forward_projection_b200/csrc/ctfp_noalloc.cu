// ctfp_noalloc.cu — ctfp_forward_noalloc: the fused forward projection for
// callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc at all: a reconstruction loop that runs
// inside a host framework owning every byte of device memory through its own
// pool, a real-time pipeline that may not allocate after start-up, or a
// process sharing a GPU under a fixed memory budget.  ctfp_forward needs a plan,
// and a plan allocates its tables.  This entry point takes every input and
// output from the caller and keeps the little scratch it needs (per-view
// trigonometry, the attenuation and spectrum tables) in a fixed file-scope
// device array, so it allocates nothing.  The energy weights I0Val*S*G*D are
// formed per ray from the caller's grid and detector tables instead of being
// tabulated.
//
// The scratch array is shared by every call on a device and keeps the last
// call's contents; calls whose kernels overlap on the GPU (two streams, two
// threads) race on it.  Every call rewrites all of the scratch it reads, so
// nothing has to start at zero.  The array is part of the library's module:
// every GPU that loads libctfp.so holds it until the process exits.
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ctfp.h"
#include "ctfp_device.cuh"

namespace ctfp {
void set_last_error(const std::string& msg);  // ctfp_api.cu
}

using namespace ctfp;

namespace {

// Layout of the scratch array: view trigonometry in FP64 and FP32, then
// attenuation, then spectrum.  CTFP_NOALLOC_SCRATCH_BYTES is the stated
// maximum size.
constexpr size_t kTrigBytes = sizeof(double2) * CTFP_NOALLOC_MAX_VIEWS + sizeof(float2) * CTFP_NOALLOC_MAX_VIEWS;
constexpr size_t kTrigfOffset = sizeof(double2) * CTFP_NOALLOC_MAX_VIEWS;
constexpr size_t kMuBytes = sizeof(float) * CTFP_MAX_ENERGIES * CTFP_MAX_MATERIALS;
constexpr size_t kSpecBytes = sizeof(float) * CTFP_MAX_ENERGIES;
static_assert(kTrigBytes + kMuBytes + kSpecBytes <= CTFP_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds its size");

static __device__ __align__(256) unsigned char g_noalloc_scratch[CTFP_NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch, looked up once per device with that
// device current.  Host code may not use the symbol itself as an address.
std::mutex g_scratch_mu;
std::vector<void*> g_scratch_ptr;

ctfp_status nfail(ctfp_status st, const std::string& m)
{
    ctfp::set_last_error(m);
    return st;
}

struct NoallocParams {
    GeomParams g;
    const float* vol[kMaxM];
    const float* S;       // scratch [E]
    const float* mu;      // scratch [E][M]
    const float* G;       // caller, device: NULL, [E][U] or [E][V][U]
    const float* D;       // caller, device: NULL or [E][V][U]
    int grid_layout;
    float I0Val;
    int E;
    float* I;
    float* IAbs;
    float* I0;
};

__device__ __forceinline__ float weight_of(const NoallocParams& q, int e, int u, int64_t pix, int64_t npix)
{
    // the reference's multiplication order: ((I0Val * S) * G) * D
    float w = q.I0Val * q.S[e];
    if (q.grid_layout == CTFP_GRID_COLUMN) w = w * __ldg(q.G + (int64_t)e * q.g.U + u);
    if (q.grid_layout == CTFP_GRID_PIXEL) w = w * __ldg(q.G + (int64_t)e * npix + pix);
    if (q.D) w = w * __ldg(q.D + (int64_t)e * npix + pix);
    return w;
}

template <int M, int MODE>
__global__ void __launch_bounds__(256) k_forward_noalloc(const NoallocParams q)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y * blockDim.y + threadIdx.y;
    const int p = blockIdx.z;
    if (u >= q.g.U || v >= q.g.V) return;
    const int64_t npix = (int64_t)q.g.U * q.g.V;
    const int64_t pix = (int64_t)v * q.g.U + u;
    const RaySeg s = ray_segment(q.g, p, v, u);
    float acc[M], cmp[M];
#pragma unroll
    for (int m = 0; m < M; m++) { acc[m] = 0.f; cmp[m] = 0.f; }
    // the same sample positions as ctfp_forward: FP64 for TRILINEAR, the
    // reference's FP32 coordinates for the texture-unit emulation
    const RayRef32 r = ray_ref32(q.g, p, v, u);
    for (int i = s.i0; i < s.i1; i++) {
        const double t = (double)i;
        const Corner c = MODE == INTERP_TRILINEAR
                             ? corner_of<INTERP_TRILINEAR>(fma(t, s.bx, s.ax), fma(t, s.by, s.ay), fma(t, s.bz, s.az))
                             : corner_tex(ref32_coords(q.g, r, i));
        float val[M];
        gather_interp<M, MODE>(q.vol, q.g.nx, q.g.ny, q.g.nz, c, val);
#pragma unroll
        for (int m = 0; m < M; m++) kahan_add(acc[m], cmp[m], val[m]);
    }
    float L[M];
#pragma unroll
    for (int m = 0; m < M; m++) L[m] = q.g.dx * (acc[m] - cmp[m]);
    float sI = 0.f, cI = 0.f, sA = 0.f, cA = 0.f;
    for (int e = 0; e < q.E; e++) {
        float att = 0.f;
#pragma unroll
        for (int m = 0; m < M; m++) att = fmaf(q.mu[e * M + m], L[m], att);
        const float w = weight_of(q, e, u, pix, npix);
        float ex, om;
        transmit(att, ex, om);
        kahan_add(sI, cI, w * ex);
        kahan_add(sA, cA, w * om);
    }
    const int64_t ray = (int64_t)p * npix + pix;
    q.I[ray] = sI - cI;
    q.IAbs[ray] = sA - cA;
}

__global__ void k_flat_field_noalloc(const NoallocParams q)
{
    const int64_t npix = (int64_t)q.g.U * q.g.V;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < npix; k += (int64_t)gridDim.x * blockDim.x) {
        float s = 0.f, c = 0.f;
        for (int e = 0; e < q.E; e++) kahan_add(s, c, weight_of(q, e, (int)(k % q.g.U), k, npix));
        q.I0[k] = s - c;
    }
}

template <int M>
cudaError_t launch_m(const NoallocParams& q, int interp, dim3 grid, dim3 block, cudaStream_t st)
{
    if (interp == INTERP_TRILINEAR) k_forward_noalloc<M, INTERP_TRILINEAR><<<grid, block, 0, st>>>(q);
    else k_forward_noalloc<M, INTERP_TEXEMU><<<grid, block, 0, st>>>(q);
    return cudaGetLastError();
}

// FP32 view angle as the reference's launchers compute it (CBCTPolyProjGPU.cu:51).
float angle_of(const ctfp_geometry* g, const ctfp_system_info& s, int64_t p)
{
    volatile float a = (float)p * s.thetaStep;
    a = a / 180.0f;
    a = a * acosf(-1.0f);
    return g->rotatedDirection < 0 ? -a : a;
}

}  // namespace

extern "C" ctfp_status ctfp_forward_noalloc(const ctfp_geometry* g, int32_t n_materials, int32_t interp,
                                            int32_t n_energies, const float* spectrum, const float* mu,
                                            const float* grid, int32_t grid_layout, const float* det_response,
                                            float I0Val, const float* const* volumes, float* I, float* IAbsorb,
                                            float* I0, void* stream)
{
    ctfp_system_info info;
    ctfp_status st = ctfp_compute_paras(g, &info);  // validates the geometry
    if (st != CTFP_OK) return st;
    if (n_materials < 1 || n_materials > CTFP_MAX_MATERIALS)
        return nfail(CTFP_INVALID_ARG, "ctfp_forward_noalloc: n_materials must be in [1, 4]");
    if (interp != INTERP_TRILINEAR && interp != INTERP_TEXEMU)
        return nfail(CTFP_UNSUPPORTED, "ctfp_forward_noalloc: only CTFP_INTERP_TRILINEAR and CTFP_INTERP_TEXEMU "
                                       "(the hardware texture needs a cudaArray, i.e. an allocation)");
    if (g->projNum > CTFP_NOALLOC_MAX_VIEWS)
        return nfail(CTFP_INVALID_ARG, "ctfp_forward_noalloc: projNum " + std::to_string(g->projNum) +
                                           " exceeds CTFP_NOALLOC_MAX_VIEWS (" +
                                           std::to_string(CTFP_NOALLOC_MAX_VIEWS) + ")");
    if (n_energies < 1 || n_energies > CTFP_MAX_ENERGIES)
        return nfail(CTFP_INVALID_ARG, "ctfp_forward_noalloc: n_energies must be in [1, " +
                                           std::to_string(CTFP_MAX_ENERGIES) + "]");
    if (!spectrum || !mu || !volumes || !I || !IAbsorb)
        return nfail(CTFP_INVALID_ARG, "ctfp_forward_noalloc: spectrum, mu, volumes, I and IAbsorb are required");
    if (grid_layout < 0 || grid_layout > 2 || (grid_layout != 0 && !grid))
        return nfail(CTFP_INVALID_ARG, "ctfp_forward_noalloc: bad grid layout or NULL grid");
    for (int m = 0; m < n_materials; m++)
        if (!volumes[m]) return nfail(CTFP_INVALID_ARG, "ctfp_forward_noalloc: volume pointer is NULL");
    if (info.intNum <= 0 || info.intNum > 100000000)
        return nfail(CTFP_INVALID_ARG, "ctfp_forward_noalloc: intNum out of range");

    // every call copies its host tables (spectrum, mu, the views'
    // trigonometry) from pageable host memory, which a stream capture cannot
    // record: refuse a capturing stream before anything is issued
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing((cudaStream_t)stream, &cap);
    if (e != cudaSuccess) return nfail(CTFP_CUDA_ERROR, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(e));
    if (cap != cudaStreamCaptureStatusNone)
        return nfail(CTFP_UNSUPPORTED, "ctfp_forward_noalloc: the stream is capturing (its host-table copies cannot "
                                       "be recorded in a graph)");
    int dev = 0;
    e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return nfail(CTFP_CUDA_ERROR, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    unsigned char* scratch = nullptr;
    {
        // set-up, once per device, with that device current
        std::lock_guard<std::mutex> lk(g_scratch_mu);
        if ((size_t)dev >= g_scratch_ptr.size()) g_scratch_ptr.resize((size_t)dev + 1, nullptr);
        if (!g_scratch_ptr[(size_t)dev]) {
            void* ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess || !ptr)
                return nfail(CTFP_CUDA_ERROR, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") +
                                                  cudaGetErrorString(e));
            g_scratch_ptr[(size_t)dev] = ptr;
        }
        scratch = (unsigned char*)g_scratch_ptr[(size_t)dev];
    }

    // tables into the scratch (pageable host sources are staged by the copy
    // before cudaMemcpyAsync returns, so these vectors may go out of scope)
    const int64_t P = g->projNum, E = n_energies, M = n_materials;
    std::vector<double2> trig((size_t)P);
    std::vector<float2> trigf((size_t)P);
    for (int64_t k = 0; k < P; k++) {
        const double a = (double)angle_of(g, info, k);
        trig[(size_t)k] = make_double2(std::cos(a), std::sin(a));
        trigf[(size_t)k] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    cudaStream_t s = (cudaStream_t)stream;
    double2* d_trig = (double2*)scratch;
    float2* d_trigf = (float2*)(scratch + kTrigfOffset);
    float* d_mu = (float*)(scratch + kTrigBytes);
    float* d_S = (float*)(scratch + kTrigBytes + kMuBytes);
    e = cudaMemcpyAsync(d_trig, trig.data(), sizeof(double2) * (size_t)P, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_trigf, trigf.data(), sizeof(float2) * (size_t)P, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_mu, mu, sizeof(float) * (size_t)(E * M), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_S, spectrum, sizeof(float) * (size_t)E, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return nfail(CTFP_CUDA_ERROR, std::string("ctfp_forward_noalloc tables: ") + cudaGetErrorString(e));

    NoallocParams q;
    std::memset(&q, 0, sizeof(q));
    GeomParams& gp = q.g;
    gp.nx = (int)g->pNumX; gp.ny = (int)g->pNumY; gp.nz = (int)g->pNumZ;
    gp.U = (int)g->dNumU; gp.V = (int)g->dNumV; gp.P = (int)g->projNum;
    gp.K = (int)info.intNum;
    gp.dHalfLU = info.dHalfLU; gp.dHalfLV = info.dHalfLV; gp.dSize = g->dSize;
    gp.sod = g->sod; gp.sdd = g->sdd; gp.FOVR = info.FOVR; gp.dx = info.dx;
    gp.pHalfX = info.pHalfX; gp.pHalfY = info.pHalfY; gp.pHalfZ = info.pHalfZ;
    gp.pSizeX = info.pSizeX; gp.pSizeY = info.pSizeY; gp.pSizeZ = info.pSizeZ;
    gp.rpSizeX = 1.0f / info.pSizeX; gp.rpSizeY = 1.0f / info.pSizeY; gp.rpSizeZ = 1.0f / info.pSizeZ;
    gp.trig = d_trig;
    gp.trigf = d_trigf;
    for (int m = 0; m < M; m++) q.vol[m] = volumes[m];
    q.S = d_S;
    q.mu = d_mu;
    q.G = grid_layout ? grid : nullptr;
    q.grid_layout = grid_layout;
    q.D = det_response;
    q.I0Val = I0Val;
    q.E = (int)E;
    q.I = I;
    q.IAbs = IAbsorb;
    q.I0 = I0;

    const dim3 block(32, 8), grd((gp.U + 31) / 32, (gp.V + 7) / 8, (unsigned)P);
    switch (M) {
        case 1: e = launch_m<1>(q, interp, grd, block, s); break;
        case 2: e = launch_m<2>(q, interp, grd, block, s); break;
        case 3: e = launch_m<3>(q, interp, grd, block, s); break;
        default: e = launch_m<4>(q, interp, grd, block, s); break;
    }
    if (e == cudaSuccess && I0) {
        const int64_t npix = (int64_t)gp.U * gp.V;
        int64_t nb = (npix + 255) / 256;
        if (nb > 148 * 8) nb = 148 * 8;
        k_flat_field_noalloc<<<(unsigned)nb, 256, 0, s>>>(q);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return nfail(CTFP_CUDA_ERROR, std::string("ctfp_forward_noalloc: ") + cudaGetErrorString(e));
    return CTFP_OK;
}
