// ctfp_diag.cu — the sampler roofline: the peak rate at which this device's
// texture path delivers trilinear footprints when nothing else limits it.
// No reference counterpart.
//
// The march reads each voxel-sample's 8 corners either with two 4-texel
// gathers (tld4) from a layered 2D texture (CTFP_SAMPLER_LAYERED) or with one
// filtered tex3D fetch (CTFP_INTERP_TEXTURE).  The kernels here issue only
// those fetches, from a texture small enough to stay in the L1 texture cache,
// with the same warp shape as the march (neighbouring lanes on neighbouring
// texels) and full occupancy, so their rate is the unit's ceiling for the
// march's access pattern; the march's own rate divided by it is its fraction
// of the texture roofline.
#include <string>

#include "../../include/ctfp.h"
#include "ctfp_kernels.cuh"

namespace ctfp {
void set_last_error(const std::string& msg);
}

using namespace ctfp;

namespace {

constexpr int kDim = 32, kLayers = 8, kIters = 2048;

// Compares div_rn_recip(x, y, r) with the IEEE division x / y bit for bit on
// n pseudo-random x per thread block sweep: x = +-(1 + m 2^-23) 2^e with a
// uniformly random 23-bit m and e in [-20, 20], from a SplitMix64 stream.
__global__ void __launch_bounds__(256) k_check_division(float y, float r, long long n, unsigned long long seed,
                                                        unsigned long long* mismatches)
{
    unsigned long long bad = 0;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(k + 1);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        const unsigned m = (unsigned)z & 0x7FFFFFu;
        const int e = (int)((z >> 23) % 41ull) - 20;
        const unsigned sign = (unsigned)(z >> 63) << 31;
        const float x = __uint_as_float(sign | ((unsigned)(e + 127) << 23) | m);
        const float q = __fdiv_rn(x, y);
        const float d = div_rn_recip(x, y, r);
        bad += __float_as_uint(q) != __float_as_uint(d);
    }
    if (bad) atomicAdd(mismatches, bad);
}

// One voxel-sample per iteration and thread: two gathers (layers l, l + 1).
__global__ void __launch_bounds__(256) k_peak_gather(cudaTextureObject_t t, float* out)
{
    const int lane = threadIdx.x & 31;
    float acc = 0.f;
    float x = 1.0f + (float)(lane & 7) + (float)(blockIdx.x & 7);
    float y = 1.0f + (float)(lane >> 3) + (float)(threadIdx.x >> 5);
#pragma unroll 4
    for (int i = 0; i < kIters; i++) {
        const int l = i & (kLayers - 2);
        const float4 a = gather_layer(t, l, x, y);
        const float4 b = gather_layer(t, l + 1, x, y);
        acc += (a.x + a.y) + (a.z + a.w) + (b.x + b.y) + (b.z + b.w);
        x = x >= (float)(kDim - 9) ? 1.0f : x + 1.0f;
        y = y >= (float)(kDim - 9) ? 1.0f : y + 0.5f;
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

// One voxel-sample per iteration and thread: one filtered tex3D fetch.
__global__ void __launch_bounds__(256) k_peak_tex3d(cudaTextureObject_t t, float* out)
{
    const int lane = threadIdx.x & 31;
    float acc = 0.f;
    float x = 1.3f + (float)(lane & 7) + (float)(blockIdx.x & 7);
    float y = 1.7f + (float)(lane >> 3) + (float)(threadIdx.x >> 5);
    float z = 1.1f;
#pragma unroll 4
    for (int i = 0; i < kIters; i++) {
        acc += tex3D<float>(t, x, y, z);
        x = x >= (float)(kDim - 9) ? 1.3f : x + 0.93f;
        y = y >= (float)(kDim - 9) ? 1.7f : y + 0.41f;
        z = z >= (float)(kLayers - 2) ? 1.1f : z + 0.12f;
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

}  // namespace

extern "C" ctfp_status ctfp_sampler_peak(int32_t device, int32_t kind, double* voxel_samples_per_s)
{
    if (!voxel_samples_per_s || (kind != CTFP_SAMPLER_LAYERED && kind != 0)) {
        set_last_error("kind must be CTFP_SAMPLER_LAYERED or 0 (hardware tex3D)");
        return CTFP_INVALID_ARG;
    }
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != device && cudaSetDevice(device) != cudaSuccess) {
        set_last_error("cudaSetDevice failed");
        return CTFP_CUDA_ERROR;
    }
    cudaArray_t arr = nullptr;
    cudaTextureObject_t tex = 0;
    float* out = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int nsm = 0;
    ctfp_status rs = CTFP_OK;
    std::string where;
    auto ok = [&](cudaError_t e, const char* w) {
        if (e != cudaSuccess && rs == CTFP_OK) {
            rs = CTFP_CUDA_ERROR;
            where = std::string(w) + ": " + cudaGetErrorString(e);
        }
        return rs == CTFP_OK;
    };
    cudaChannelFormatDesc cd = cudaCreateChannelDesc<float>();
    const bool layered = kind == CTFP_SAMPLER_LAYERED;
    ok(cudaMalloc3DArray(&arr, &cd, make_cudaExtent(kDim, kDim, kLayers), layered ? cudaArrayLayered : 0),
       "cudaMalloc3DArray");
    if (rs == CTFP_OK) {
        cudaResourceDesc rd = {};
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = arr;
        cudaTextureDesc td = {};
        td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
        td.filterMode = layered ? cudaFilterModePoint : cudaFilterModeLinear;
        td.readMode = cudaReadModeElementType;
        ok(cudaCreateTextureObject(&tex, &rd, &td, nullptr), "cudaCreateTextureObject");
    }
    ok(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");
    const int blocks = nsm * 8, threads = 256;
    ok(cudaMalloc(&out, sizeof(float) * (size_t)blocks * threads), "cudaMalloc");
    ok(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
    ok(cudaEventCreate(&e0), "cudaEventCreate");
    ok(cudaEventCreate(&e1), "cudaEventCreate");
    float best = 1e30f;
    for (int rep = 0; rep < 4 && rs == CTFP_OK; rep++) {
        ok(cudaEventRecord(e0, st), "cudaEventRecord");
        if (layered) k_peak_gather<<<blocks, threads, 0, st>>>(tex, out);
        else k_peak_tex3d<<<blocks, threads, 0, st>>>(tex, out);
        ok(cudaGetLastError(), "launch");
        ok(cudaEventRecord(e1, st), "cudaEventRecord");
        ok(cudaEventSynchronize(e1), "cudaEventSynchronize");
        float ms = 0.f;
        ok(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
        if (rep > 0 && ms < best) best = ms;  // the first launch warms up
    }
    if (rs == CTFP_OK) *voxel_samples_per_s = (double)blocks * threads * kIters / (best * 1e-3);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    cudaFree(out);
    if (tex) cudaDestroyTextureObject(tex);
    if (arr) cudaFreeArray(arr);
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
    if (rs != CTFP_OK) set_last_error(where);
    return rs;
}

extern "C" ctfp_status ctfp_check_division(int32_t device, float divisor, int64_t n, uint64_t seed,
                                           int64_t* mismatches)
{
    if (!mismatches || n < 0 || !(divisor > 0.f) || divisor > 1e30f) {
        set_last_error("ctfp_check_division: needs a positive finite divisor, n >= 0 and an output");
        return CTFP_INVALID_ARG;
    }
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != device) cudaSetDevice(device);
    unsigned long long* d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(d, 0, sizeof(unsigned long long));
    const float r = 1.0f / divisor;  // the reciprocal the plans store (rpSize)
    if (e == cudaSuccess) {
        k_check_division<<<148 * 8, 256>>>(divisor, r, (long long)n, (unsigned long long)seed, d);
        e = cudaGetLastError();
    }
    unsigned long long h = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
    if (d) cudaFree(d);
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
    if (e != cudaSuccess) {
        set_last_error(std::string("ctfp_check_division: ") + cudaGetErrorString(e));
        return CTFP_CUDA_ERROR;
    }
    *mismatches = (int64_t)h;
    return CTFP_OK;
}
