// ctfp_autotune.cu — picks the forward kernel's launch shape for a plan by
// timing candidates on the device.  No reference counterpart: the reference
// launches fixed 8 x 8 x 8 / 8 x 8 blocks (Source/CUDAFun/CBCTPolyProjGPU.cuh:22-24,
// CBCTPolyProjGPU.cu:41-45).
//
// Search: stage 1 times every tile (8 x 8 ... 64 x 4) at every register cap
// (2, 3, 4 CTAs per SM) with 2 views per CTA; stage 2 times the three best
// with 1, 2 and 4 views per CTA.  Each candidate runs the fused forward over
// four chunks of views spread round the rotation (the sampling pattern changes
// with the angle) launched concurrently on four streams, once to warm up and
// twice timed with CUDA events; the fastest total wins.  Results are cached
// per process under a key of the geometry, materials, sampler, energies and
// device name, and optionally in
// the text file named by CTFP_TUNE_CACHE (one "key tile_u tile_v views
// min_ctas ms" line per entry), which later processes read.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/ctfp.h"
#include "ctfp_kernels.cuh"

namespace ctfp {
void set_last_error(const std::string& msg);
const GeomParams& plan_geom(const ctfp_plan* p);
const ctfp_geometry& plan_geometry(const ctfp_plan* p);
int plan_materials(const ctfp_plan* p);
int plan_interp(const ctfp_plan* p);
int plan_sampler(const ctfp_plan* p);
int plan_device(const ctfp_plan* p);
int plan_energies(const ctfp_plan* p);
LaunchShape& plan_shape(ctfp_plan* p);
MarchParams plan_march_params(const ctfp_plan* p);
ctfp_status plan_upload(ctfp_plan* p, const float* const* volumes, cudaStream_t st);
}  // namespace ctfp

using namespace ctfp;

namespace {

struct Entry {
    LaunchShape shape;
    float ms;
};

std::mutex g_mu;
std::map<std::string, Entry> g_cache;
bool g_file_read = false;

ctfp_status tfail(ctfp_status st, const std::string& m)
{
    ctfp::set_last_error(m);
    return st;
}

std::string cache_key(const ctfp_plan* p, int n_sample)
{
    const ctfp_geometry& g = plan_geometry(p);
    cudaDeviceProp prop;
    std::string dev = "unknown";
    if (cudaGetDeviceProperties(&prop, plan_device(p)) == cudaSuccess) dev = prop.name;
    for (char& c : dev)
        if (c == ' ') c = '_';
    std::ostringstream k;
    k << dev << "|" << g.pNumX << "x" << g.pNumY << "x" << g.pNumZ << "|" << g.pLengthX << "," << g.pLengthY << ","
      << g.pLengthZ << "|P" << g.projNum << "|" << g.dNumU << "x" << g.dNumV << "@" << g.dSize << "|" << g.sod << ","
      << g.sdd << "|M" << plan_materials(p) << "|i" << plan_interp(p) << "|s" << plan_sampler(p) << "|E"
      << plan_energies(p) << "|n" << n_sample;
    return k.str();
}

void read_file_cache()
{
    if (g_file_read) return;
    g_file_read = true;
    const char* path = std::getenv("CTFP_TUNE_CACHE");
    if (!path || !*path) return;
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream in(line);
        std::string key;
        Entry e;
        if (in >> key >> e.shape.tile_u >> e.shape.tile_v >> e.shape.views_per_cta >> e.shape.min_ctas >> e.ms)
            g_cache[key] = e;
    }
}

void append_file_cache(const std::string& key, const Entry& e)
{
    const char* path = std::getenv("CTFP_TUNE_CACHE");
    if (!path || !*path) return;
    std::ofstream f(path, std::ios::app);
    f << key << " " << e.shape.tile_u << " " << e.shape.tile_v << " " << e.shape.views_per_cta << " "
      << e.shape.min_ctas << " " << e.ms << "\n";
}

bool valid_shape(const LaunchShape& s)
{
    const int t = s.tile_u * s.tile_v;
    return t >= 32 && t <= 256 && t % 32 == 0 && s.views_per_cta >= 1 && s.min_ctas >= 2 && s.min_ctas <= 5 &&
           t * s.min_ctas <= 2048;
}

// Streams and events of one tuning run: the view chunks of a candidate run
// concurrently, one per stream, so the sample ends in one partial wave of
// CTAs rather than one per chunk (a chunk of a few waves run alone ends in a
// partial wave that weighs more for CTAs of more views, which made short
// samples favour 1 view per CTA).
struct ChunkStreams {
    cudaStream_t s[4] = {};
    cudaEvent_t fork = nullptr, join[4] = {};
    ~ChunkStreams()
    {
        for (cudaStream_t x : s)
            if (x) cudaStreamDestroy(x);
        for (cudaEvent_t x : join)
            if (x) cudaEventDestroy(x);
        if (fork) cudaEventDestroy(fork);
    }
    cudaError_t create()
    {
        cudaError_t e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
        for (int k = 0; k < 4 && e == cudaSuccess; k++) {
            e = cudaStreamCreateWithFlags(&s[k], cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&join[k], cudaEventDisableTiming);
        }
        return e;
    }
};

// Total time of one candidate over the view chunks (ms), or a negative value
// on a launch error.
float time_shape(const MarchParams& base, int M, int interp, int sampler, const LaunchShape& ls,
                 const std::vector<std::pair<int, int>>& chunks, cudaEvent_t e0, cudaEvent_t e1, cudaStream_t st,
                 ChunkStreams& cs, int reps)
{
    auto run_all = [&]() -> cudaError_t {
        // every chunk stream starts after the work already on st, and st
        // continues after all of them
        cudaError_t e = cudaEventRecord(cs.fork, st);
        for (size_t k = 0; k < chunks.size() && e == cudaSuccess; k++) {
            cudaStream_t sk = cs.s[k % 4];
            e = cudaStreamWaitEvent(sk, cs.fork, 0);
            MarchParams prm = base;
            prm.view0 = chunks[k].first;
            prm.n_views = chunks[k].second;
            if (e == cudaSuccess) e = launch_forward(prm, M, interp, sampler, true, ls, sk);
            if (e == cudaSuccess) e = cudaEventRecord(cs.join[k % 4], sk);
        }
        for (size_t k = 0; k < chunks.size() && k < 4 && e == cudaSuccess; k++)
            e = cudaStreamWaitEvent(st, cs.join[k], 0);
        return e;
    };
    if (run_all() != cudaSuccess) return -1.f;
    if (cudaEventRecord(e0, st) != cudaSuccess) return -1.f;
    for (int r = 0; r < reps; r++)
        if (run_all() != cudaSuccess) return -1.f;
    if (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) return -1.f;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) return -1.f;
    return ms / (float)reps;
}

}  // namespace

extern "C" ctfp_status ctfp_plan_autotune(ctfp_plan* p, const float* const* volumes, float* I, float* IAbsorb,
                                          int32_t n_sample_views, ctfp_launch_shape* out, void* stream)
{
    if (!p) return tfail(CTFP_INVALID_ARG, "plan is NULL");
    if (!volumes || !I) return tfail(CTFP_INVALID_ARG, "volumes and I are required");
    if (plan_energies(p) < 1) return tfail(CTFP_NOT_READY, "spectral tables not set");
    const GeomParams& g = plan_geom(p);
    int n = n_sample_views > 0 ? n_sample_views : 64;
    n = std::min(n, g.P);
    const std::string key = cache_key(p, n);
    {
        std::lock_guard<std::mutex> lk(g_mu);
        read_file_cache();
        auto it = g_cache.find(key);
        if (it != g_cache.end() && valid_shape(it->second.shape)) {
            plan_shape(p) = it->second.shape;
            if (out) {
                out->tile_u = it->second.shape.tile_u;
                out->tile_v = it->second.shape.tile_v;
                out->views_per_cta = it->second.shape.views_per_cta;
                out->min_ctas_per_sm = it->second.shape.min_ctas;
                out->ms = it->second.ms;
                out->from_cache = 1;
            }
            return CTFP_OK;
        }
    }
    int prev_dev = -1;
    cudaGetDevice(&prev_dev);
    if (prev_dev != plan_device(p)) cudaSetDevice(plan_device(p));
    cudaStream_t st = (cudaStream_t)stream;
    ctfp_status rs = plan_upload(p, volumes, st);
    // four chunks spread round the rotation
    std::vector<std::pair<int, int>> chunks;
    const int nch = std::min(4, n);
    for (int c = 0; c < nch; c++) {
        const int len = n / nch + (c < n % nch ? 1 : 0);
        const int v0 = (int)((long long)c * g.P / nch);
        chunks.emplace_back(v0, std::min(len, g.P - v0));
    }
    MarchParams base = plan_march_params(p);
    for (int m = 0; m < plan_materials(p); m++) base.vol[m] = volumes[m];
    base.I = I;
    base.IAbs = IAbsorb;
    const int M = plan_materials(p), interp = plan_interp(p), sampler = plan_sampler(p);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ChunkStreams cs;
    Entry best{plan_shape(p), -1.f};
    if (rs == CTFP_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess ||
                          cs.create() != cudaSuccess))
        rs = tfail(CTFP_CUDA_ERROR, "cudaEventCreate / cudaStreamCreate failed");
    if (rs == CTFP_OK) {
        static const int tiles[][2] = {{16, 8}, {32, 4}, {8, 16}, {64, 2}, {16, 16}, {32, 8}, {8, 32}, {64, 4},
                                       {8, 8},  {16, 4}};
        std::vector<Entry> stage1;
        for (const auto& t : tiles)
            for (int minb = 2; minb <= 4; minb++) {
                LaunchShape ls{t[0], t[1], 2, minb};
                if (!valid_shape(ls)) continue;
                const float ms = time_shape(base, M, interp, sampler, ls, chunks, e0, e1, st, cs, 2);
                if (ms < 0.f) {
                    rs = tfail(CTFP_CUDA_ERROR, std::string("autotune launch: ") + cudaGetErrorString(cudaGetLastError()));
                    break;
                }
                stage1.push_back({ls, ms});
            }
        if (rs == CTFP_OK && !stage1.empty()) {
            std::sort(stage1.begin(), stage1.end(), [](const Entry& a, const Entry& b) { return a.ms < b.ms; });
            best = stage1[0];
            const size_t top = std::min<size_t>(3, stage1.size());
            for (size_t i = 0; i < top && rs == CTFP_OK; i++)
                for (int vpc : {1, 4}) {
                    LaunchShape ls = stage1[i].shape;
                    ls.views_per_cta = vpc;
                    const float ms = time_shape(base, M, interp, sampler, ls, chunks, e0, e1, st, cs, 2);
                    if (ms < 0.f) {
                        rs = tfail(CTFP_CUDA_ERROR, "autotune launch failed");
                        break;
                    }
                    if (ms < best.ms) best = {ls, ms};
                }
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (prev_dev >= 0 && prev_dev != plan_device(p)) cudaSetDevice(prev_dev);
    if (rs != CTFP_OK) return rs;
    plan_shape(p) = best.shape;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_cache[key] = best;
        append_file_cache(key, best);
    }
    if (out) {
        out->tile_u = best.shape.tile_u;
        out->tile_v = best.shape.tile_v;
        out->views_per_cta = best.shape.views_per_cta;
        out->min_ctas_per_sm = best.shape.min_ctas;
        out->ms = best.ms;
        out->from_cache = 0;
    }
    return CTFP_OK;
}
