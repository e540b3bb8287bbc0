// tune.cu -- schedule autotuner with an on-disk cache.
//
// For a length n and a batch size, the planner's best few candidates (by
// heuristic score) are timed on the current device through launch_fft --
// the same path a real call takes, fixed-size and pipelined kernels included
// -- on synthetic data, and the fastest is kept. Results are cached per
// (device name, n, batch bucket, width/thread constraints) in memory and in
// a text file so a process pays for tuning once per machine.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <tuple>

#include "fft_engine.h"
#include "plan.h"

namespace fftb200 {

namespace {

std::mutex g_tmu;
std::map<std::string, EnginePlan> g_tuned;
bool g_loaded = false;

std::string cache_path()
{
    if (const char* p = getenv("FFTLIB_B200_TUNE_CACHE")) return p;
    const char* home = getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/fftlib_b200_tune.txt";
}

uint32_t bucket(uint32_t batch)
{
    uint32_t b = 1;
    while (b < batch && b < (1u << 20)) b <<= 2;
    return b;
}

std::string key_of(const char* dev, uint32_t n, uint32_t batch, int emaxOnly, uint32_t maxT)
{
    std::ostringstream os;
    os << dev << "|" << n << "|" << bucket(batch) << "|" << emaxOnly << "|" << maxT;
    return os.str();
}

// line: <key> <emax> <T> <P> <R0> ... <R(P-1)>
void load_cache()
{
    if (g_loaded) return;
    g_loaded = true;
    FILE* f = fopen(cache_path().c_str(), "r");
    if (!f) return;
    char line[512];
    while (fgets(line, sizeof(line), f)) {
        std::istringstream is(line);
        std::string key;
        EnginePlan e;
        if (!(is >> key >> e.emax >> e.T >> e.P) || e.P < 1 || e.P > kMaxPasses) continue;
        uint32_t prod = 1;
        bool ok = true;
        for (int i = 0; i < e.P; ++i) ok = ok && (is >> e.R[i]) && e.R[i] > 0, prod *= (uint32_t)e.R[i];
        const size_t bar = key.find('|');
        if (!ok || bar == std::string::npos) continue;
        e.n = (uint32_t)strtoul(key.c_str() + bar + 1, nullptr, 10);
        if (prod != e.n) continue;
        g_tuned[key] = e;
    }
    fclose(f);
}

void append_cache(const std::string& key, const EnginePlan& e)
{
    const std::string path = cache_path();
    const size_t slash = path.rfind('/');
    if (slash != std::string::npos) mkdir(path.substr(0, slash).c_str(), 0755); // best effort
    FILE* f = fopen(path.c_str(), "a");
    if (!f) return;
    fprintf(f, "%s %d %u %d", key.c_str(), e.emax, e.T, e.P);
    for (int i = 0; i < e.P; ++i) fprintf(f, " %d", e.R[i]);
    fprintf(f, "\n");
    fclose(f);
}

__global__ void k_fill(float2* x, size_t count, uint32_t seed)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    uint32_t h = (uint32_t)i * 2654435761u ^ seed;
    h ^= h >> 15;
    h *= 2246822519u;
    h ^= h >> 13;
    x[i] = make_float2((float)(h & 0xFFFF) / 32768.0f - 1.0f, (float)(h >> 16) / 32768.0f - 1.0f);
}

// Average milliseconds of one launch of schedule e over `batch` transforms.
float time_candidate(const EnginePlan& e, float2* x, float2* y, uint32_t batch, cudaStream_t s, bool* ok)
{
    *ok = false;
    float2* tw = nullptr;
    if (make_pass_table(&tw, e, s) != cudaSuccess) {
        cudaGetLastError();
        return 0.f;
    }
    FftArgs a = engine_args(e, tw);
    a.err = error_word().dev;
    a.in = x;
    a.out = y;
    a.batch = batch;
    a.inBatch = e.n;
    a.inElem = 1;
    a.outBatch = e.n;
    a.outElem = 1;
    finalize_launch(a, e, true, true);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float ms = 0.f;
    cudaError_t err = launch_fft(a, e.emax, s); // warm-up
    if (err == cudaSuccess) {
        cudaEventRecord(e0, s);
        const int reps = 5;
        for (int r = 0; r < reps && err == cudaSuccess; ++r) err = launch_fft(a, e.emax, s);
        cudaEventRecord(e1, s);
        if (err == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess) {
            cudaEventElapsedTime(&ms, e0, e1);
            ms /= reps;
            *ok = true;
        }
    }
    if (err != cudaSuccess) cudaGetLastError();
    cudaStreamSynchronize(s);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(tw);
    return ms;
}

} // namespace

bool autotune_enabled()
{
    const char* v = getenv("FFTLIB_B200_AUTOTUNE");
    return v && *v && strcmp(v, "0") != 0;
}

bool tune_schedule(uint32_t n, uint32_t batch, int emaxOnly, uint32_t maxT, EnginePlan* out, ScheduleTimer timer)
{
    if (!timer) timer = &time_candidate;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return false;
    std::string devName(prop.name);
    std::replace(devName.begin(), devName.end(), ' ', '_');
    const std::string key = key_of(devName.c_str(), n, batch, emaxOnly, maxT);
    std::lock_guard<std::mutex> lock(g_tmu);
    load_cache();
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) {
        *out = it->second;
        return true;
    }
    std::vector<EnginePlan> cands = engine_candidates(n, emaxOnly, maxT);
    if (cands.empty()) return false;
    if (cands.size() > 4) cands.resize(4);
    // enough work to time: at least ~32 MB of data, at most 256 MB
    const size_t per = (size_t)n * sizeof(float2);
    size_t tb = std::max<size_t>(batch, (32u << 20) / per);
    tb = std::min<size_t>(tb, std::max<size_t>(1, (256u << 20) / per));
    float2 *x = nullptr, *y = nullptr;
    cudaStream_t s = nullptr;
    if (cudaMalloc(&x, per * tb) != cudaSuccess || cudaMalloc(&y, per * tb) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
        cudaFree(x);
        cudaFree(y);
        cudaGetLastError();
        return false;
    }
    const size_t count = (size_t)n * tb;
    k_fill<<<(unsigned)((count + 255) / 256), 256, 0, s>>>(x, count, 12345u);
    float best = 0.f;
    int bestIdx = -1;
    for (size_t i = 0; i < cands.size(); ++i) {
        bool ok = false;
        const float ms = timer(cands[i], x, y, (uint32_t)tb, s, &ok);
        if (ok && (bestIdx < 0 || ms < best)) {
            best = ms;
            bestIdx = (int)i;
        }
    }
    cudaStreamDestroy(s);
    cudaFree(x);
    cudaFree(y);
    if (bestIdx < 0) return false;
    *out = cands[(size_t)bestIdx];
    g_tuned[key] = *out;
    append_cache(key, *out);
    return true;
}

} // namespace fftb200
