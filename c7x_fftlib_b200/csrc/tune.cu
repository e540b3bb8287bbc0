// tune.cu -- autotuners with an on-disk cache.
//
// Two users: the mixed-length kernel (tune_schedule: the radix schedule of
// each length group, timed through the mixed kernel itself) and the batched
// entry points (tune_batched for FP32 c2c / ifft / r2c / c2r: radix
// schedule, transforms per CTA, persistent kernel or not and its CTA count;
// tune_i16 for the int16 kernel: threads per transform, hence transforms per
// CTA, and CTA count). Candidates are timed with CUDA events on synthetic
// data through the launch sequence a real call takes, and the fastest is
// kept per (device name, length, batch bucket, kind and dtype) in memory and
// in a text file ($FFTLIB_B200_TUNE_CACHE, default
// $HOME/.cache/fftlib_b200_tune.txt), so a process pays for tuning once per
// machine. A cached entry is used only if it is still one of the current
// candidates, so a stale or edited file cannot select a launch that does not
// exist.
//
// The reference factors each length into its radix stages once, at _init
// (src/fft_c7x/FFTLIB_fft1dBatched_i32fc_c32fc_o32fc/c7504/
// FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_ci.cpp:99-118); the tuner takes that
// decision by measurement instead of by rule, at the same point.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "FFTLIB_types.h"
#include "fft_engine.h"
#include "fft_i16.h"
#include "plan.h"

extern "C" FFTLIB_STATUS FFTLIB_b200_tw_gen_i16_device(int16_t* pW, uint32_t numPoints, void* stream);

namespace fftb200 {

namespace {

// ---- cache: one line per entry, "<key> <value tokens>" -----------------------

std::mutex g_tmu;
std::map<std::string, std::string> g_cache;
std::string g_loadedPath;
bool g_loaded = false;

std::string cache_path()
{
    if (const char* p = getenv("FFTLIB_B200_TUNE_CACHE")) return p;
    const char* home = getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/fftlib_b200_tune.txt";
}

// (Re)reads the file when the cache path is new to this process.
void load_cache()
{
    const std::string path = cache_path();
    if (g_loaded && path == g_loadedPath) return;
    g_cache.clear();
    g_loaded = true;
    g_loadedPath = path;
    FILE* f = fopen(path.c_str(), "r");
    if (!f) return;
    char line[512];
    while (fgets(line, sizeof(line), f)) {
        std::string l(line);
        while (!l.empty() && (l.back() == '\n' || l.back() == '\r' || l.back() == ' ')) l.pop_back();
        const size_t sp = l.find(' ');
        if (sp == std::string::npos || sp == 0) continue;
        g_cache[l.substr(0, sp)] = l.substr(sp + 1);
    }
    fclose(f);
}

bool cache_get(const std::string& key, std::string* value)
{
    load_cache();
    auto it = g_cache.find(key);
    if (it == g_cache.end()) return false;
    *value = it->second;
    return true;
}

void cache_put(const std::string& key, const std::string& value)
{
    g_cache[key] = value;
    const std::string path = g_loadedPath;
    const size_t slash = path.rfind('/');
    if (slash != std::string::npos) mkdir(path.substr(0, slash).c_str(), 0755); // best effort
    FILE* f = fopen(path.c_str(), "a");
    if (!f) return;
    fprintf(f, "%s %s\n", key.c_str(), value.c_str());
    fclose(f);
}

bool device_of(int* dev, cudaDeviceProp* prop)
{
    return cudaGetDevice(dev) == cudaSuccess && cudaGetDeviceProperties(prop, *dev) == cudaSuccess;
}

// key: <device name>|<n>|<batch bucket>|<tag>
std::string key_of(const cudaDeviceProp& prop, uint32_t n, uint32_t batch, const std::string& tag)
{
    std::string dev(prop.name);
    std::replace(dev.begin(), dev.end(), ' ', '_');
    std::ostringstream os;
    os << dev << "|" << n << "|" << tune_bucket(batch) << "|" << tag;
    return os.str();
}

std::string encode(const EnginePlan& e)
{
    std::ostringstream os;
    os << e.emax << " " << e.T << " " << e.P;
    for (int i = 0; i < e.P; ++i) os << " " << e.R[i];
    return os.str();
}

bool same_schedule(const EnginePlan& a, const EnginePlan& b)
{
    if (a.n != b.n || a.emax != b.emax || a.T != b.T || a.P != b.P) return false;
    for (int i = 0; i < a.P; ++i)
        if (a.R[i] != b.R[i]) return false;
    return true;
}

// A schedule from `is`, accepted only if it is one of `cands`.
bool decode(std::istream& is, uint32_t n, const std::vector<EnginePlan>& cands, EnginePlan* out)
{
    EnginePlan e;
    e.n = n;
    if (!(is >> e.emax >> e.T >> e.P) || e.P < 1 || e.P > kMaxPasses) return false;
    for (int i = 0; i < e.P; ++i)
        if (!(is >> e.R[i])) return false;
    for (const EnginePlan& c : cands)
        if (same_schedule(c, e)) {
            *out = c;
            return true;
        }
    return false;
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

__global__ void k_fill_i16(short2* x, size_t count, uint32_t seed)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    uint32_t h = (uint32_t)i * 2654435761u ^ seed;
    h ^= h >> 15;
    h *= 2246822519u;
    h ^= h >> 13;
    x[i] = make_short2((short)((int)(h & 0xFFF) - 2048), (short)((int)((h >> 16) & 0xFFF) - 2048));
}

// Average milliseconds of one call of `run` on stream s: one warm-up call,
// then enough repetitions for about 2 ms of work (5 to 200).
template <class Run>
float time_runs(Run run, cudaStream_t s, bool* ok)
{
    *ok = false;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess) return 0.f;
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return 0.f;
    }
    float ms = 0.f;
    cudaError_t err = run();
    if (err == cudaSuccess) err = cudaEventRecord(e0, s);
    if (err == cudaSuccess) err = run();
    if (err == cudaSuccess) err = cudaEventRecord(e1, s);
    if (err == cudaSuccess) err = cudaEventSynchronize(e1);
    float one = 0.f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&one, e0, e1);
    int reps = 5;
    if (err == cudaSuccess && one > 0.f) reps = std::max(5, std::min(200, (int)(2.0f / one)));
    if (err == cudaSuccess) err = cudaEventRecord(e0, s);
    for (int r = 0; r < reps && err == cudaSuccess; ++r) err = run();
    if (err == cudaSuccess) err = cudaEventRecord(e1, s);
    if (err == cudaSuccess) err = cudaEventSynchronize(e1);
    if (err == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess && !take_device_error()) {
        ms /= (float)reps;
        *ok = true;
    }
    if (err != cudaSuccess) cudaGetLastError();
    cudaStreamSynchronize(s);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms;
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
    const float ms = time_runs([&] { return launch_fft(a, e.emax, s); }, s, ok);
    cudaFree(tw);
    return ms;
}

// Device buffers of a timing run, released on scope exit.
struct TuneBuffers {
    std::vector<void*> ptrs;
    cudaStream_t s = nullptr;
    bool ok = true;
    void* alloc(size_t bytes)
    {
        void* p = nullptr;
        if (ok && cudaMalloc(&p, std::max<size_t>(bytes, 16)) != cudaSuccess) {
            cudaGetLastError();
            ok = false;
            p = nullptr;
        }
        if (p) ptrs.push_back(p);
        return p;
    }
    ~TuneBuffers()
    {
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
        for (void* p : ptrs) cudaFree(p);
    }
};

// The batched FP32 launch choices worth timing for length n, best guess
// first: the planner's top three schedules and every other schedule of n
// that has a fixed-size kernel; for a fixed-size schedule whose persistent
// pipelined kernel takes this kind, that kernel with all resident CTAs, with
// 1 and 2 per SM, and the one-tile-per-CTA kernel; for the others the
// planner's transforms per CTA and half as many.
std::vector<BatchedChoice> batched_candidates(uint32_t n, int kind, int mode, int sms)
{
    std::vector<EnginePlan> all = engine_candidates(n);
    std::vector<EnginePlan> scheds;
    for (size_t i = 0; i < all.size() && scheds.size() < 3; ++i) scheds.push_back(all[i]);
    for (const StaticEntry& st : static_schedules()) {
        if (st.n != n) continue;
        EnginePlan e;
        e.n = n;
        e.emax = st.emax;
        e.T = st.T;
        e.P = st.P;
        for (int i = 0; i < st.P; ++i) e.R[i] = st.R[i];
        bool seen = false;
        for (const EnginePlan& s : scheds) seen = seen || same_schedule(s, e);
        if (!seen) scheds.push_back(e);
    }
    // the pipelined kernel's row conditions (launch_fft)
    const bool kindPipes = kind == TUNE_C2C || kind == TUNE_IFFT || (kind == TUNE_R2C && n % 2u == 0) ||
                           (kind == TUNE_C2R && mode == 0 && n % 2u == 0 && n >= 64u);
    std::vector<BatchedChoice> out;
    for (const EnginePlan& e : scheds) {
        BatchedChoice c;
        c.eng = e;
        const bool fixed = static_max_threads(n, e.emax, e.T, e.P, e.R) != 0;
        const int resident = fixed ? static_pipelined_resident(n, e.emax, e.T, e.P, e.R) : 0;
        if (fixed && resident > 0 && kindPipes) {
            out.push_back(c);
            for (int k = 1; k <= 2 && k < resident; ++k) {
                c.gridCap = (uint32_t)(k * sms);
                out.push_back(c);
            }
            c.gridCap = 0;
            c.noPipe = true;
            out.push_back(c);
        } else {
            out.push_back(c);
            const uint32_t m = e.T >= 128u ? 1u : 256u / e.T;
            if (m >= 2u) {
                c.tileM = m / 2u;
                out.push_back(c);
            }
        }
    }
    return out;
}

std::string batched_tag(int kind, int mode)
{
    static const char* const names[] = {"c2c", "ifft", "r2c", "c2r"};
    std::string t = std::string(names[kind & 3]) + ":f32";
    if (kind == TUNE_R2C || kind == TUNE_C2R) t += ":m" + std::to_string(mode);
    return t;
}

std::string encode(const BatchedChoice& c)
{
    return encode(c.eng) + " " + std::to_string(c.gridCap) + " " + std::to_string(c.tileM) + " " +
           (c.noPipe ? "1" : "0");
}

bool same_choice(const BatchedChoice& a, const BatchedChoice& b)
{
    return same_schedule(a.eng, b.eng) && a.gridCap == b.gridCap && a.tileM == b.tileM && a.noPipe == b.noPipe;
}

// Milliseconds of one call of `kind` over `batch` transforms with choice c.
float time_batched(const ComplexPlan* base, const BatchedChoice& c, int kind, int mode, void* x, void* y,
                   void* scratch, uint32_t batch, cudaStream_t s, bool* ok)
{
    *ok = false;
    ComplexPlan t = *base;
    t.eng = c.eng;
    t.gridCap = c.gridCap;
    t.tileM = c.tileM;
    t.noPipe = c.noPipe;
    t.tw = nullptr;
    if (make_pass_table(&t.tw, t.eng, s) != cudaSuccess) {
        cudaGetLastError();
        return 0.f;
    }
    const float ms = time_runs(
        [&]() -> cudaError_t {
            switch (kind) {
            case TUNE_C2C: return run_c2c(&t, (float2*)x, (float2*)y, batch, false, s);
            case TUNE_IFFT: return run_c2c(&t, (float2*)x, (float2*)y, batch, true, s);
            case TUNE_R2C: return run_r2c(&t, (float*)x, (float2*)scratch, (float2*)y, batch, mode, s);
            default: return run_c2r(&t, (const float2*)x, (float2*)scratch, (float*)y, batch, mode, s);
            }
        },
        s, ok);
    cudaStreamSynchronize(s);
    cudaFree(t.tw);
    return ms;
}

// ---- int16 -------------------------------------------------------------------

// Threads per transform of the int16 kernel worth timing: the launcher's
// default first, then twice and half as many, each a power of two up to 256
// that leaves the CTA's shared memory (the Q15 table as 32-bit pairs plus
// 256 / tg padded transforms) within 227 KB.
std::vector<uint32_t> i16_tg_candidates(uint32_t n)
{
    std::vector<uint32_t> out;
    const uint32_t def = i16_default_tg(n);
    for (uint32_t tg : {def, 2u * def, def / 2u})
        if (tg >= 1u && tg <= i16_max_tg(n) && i16_smem_bytes(n, tg, i16_prefetch(n, tg, 3u)) <= 227u * 1024u &&
            std::find(out.begin(), out.end(), tg) == out.end())
            out.push_back(tg);
    return out;
}

// $FFTLIB_B200_TUNE_VERBOSE set to a non-zero value: every timed candidate
// is reported on stderr.
bool tune_verbose()
{
    const char* v = getenv("FFTLIB_B200_TUNE_VERBOSE");
    return v && *v && strcmp(v, "0") != 0;
}

} // namespace

uint32_t tune_bucket(uint32_t batch)
{
    uint32_t b = 1;
    while (b < batch && b < (1u << 20)) b <<= 2;
    return b;
}

bool autotune_enabled()
{
    const char* v = getenv("FFTLIB_B200_AUTOTUNE");
    return v && *v && strcmp(v, "0") != 0;
}

bool tune_schedule(uint32_t n, uint32_t batch, int emaxOnly, uint32_t maxT, EnginePlan* out, ScheduleTimer timer)
{
    if (!timer) timer = &time_candidate;
    int dev = 0;
    cudaDeviceProp prop;
    if (!device_of(&dev, &prop)) return false;
    const std::string key =
        key_of(prop, n, batch, "mixed:e" + std::to_string(emaxOnly) + ":t" + std::to_string(maxT));
    std::vector<EnginePlan> cands = engine_candidates(n, emaxOnly, maxT);
    if (cands.empty()) return false;
    if (cands.size() > 4) cands.resize(4);
    std::lock_guard<std::mutex> lock(g_tmu);
    std::string val;
    if (cache_get(key, &val)) {
        std::istringstream is(val);
        if (decode(is, n, cands, out)) return true;
    }
    // enough work to time: at least ~32 MB of data, at most 256 MB
    const size_t per = (size_t)n * sizeof(float2);
    size_t tb = std::max<size_t>(batch, (32u << 20) / per);
    tb = std::min<size_t>(tb, std::max<size_t>(1, (256u << 20) / per));
    TuneBuffers b;
    float2* x = (float2*)b.alloc(per * tb);
    float2* y = (float2*)b.alloc(per * tb);
    if (!b.ok || cudaStreamCreateWithFlags(&b.s, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const size_t count = (size_t)n * tb;
    k_fill<<<(unsigned)((count + 255) / 256), 256, 0, b.s>>>(x, count, 12345u);
    float best = 0.f;
    int bestIdx = -1;
    for (size_t i = 0; i < cands.size(); ++i) {
        bool ok = false;
        const float ms = timer(cands[i], x, y, (uint32_t)tb, b.s, &ok);
        if (ok && (bestIdx < 0 || ms < best)) {
            best = ms;
            bestIdx = (int)i;
        }
    }
    if (bestIdx < 0) return false;
    *out = cands[(size_t)bestIdx];
    cache_put(key, encode(*out));
    return true;
}

bool tune_batched(const ComplexPlan* base, int kind, int mode, uint32_t batch, BatchedChoice* out)
{
    if (base->multiPass || kind < TUNE_C2C || kind > TUNE_C2R) return false;
    const uint32_t n = base->n;
    int dev = 0;
    cudaDeviceProp prop;
    if (!device_of(&dev, &prop)) return false;
    const std::vector<BatchedChoice> cands = batched_candidates(n, kind, mode, prop.multiProcessorCount);
    if (cands.empty()) return false;
    const std::string key = key_of(prop, n, batch, batched_tag(kind, mode));
    std::lock_guard<std::mutex> lock(g_tmu);
    std::string val;
    if (cache_get(key, &val)) {
        std::istringstream is(val);
        BatchedChoice c;
        int np = 0;
        std::vector<EnginePlan> schedules;
        for (const BatchedChoice& k : cands) schedules.push_back(k.eng);
        if (decode(is, n, schedules, &c.eng) && (is >> c.gridCap >> c.tileM >> np)) {
            c.noPipe = np != 0;
            for (const BatchedChoice& k : cands)
                if (same_choice(k, c)) {
                    *out = k;
                    return true;
                }
        }
    }
    // the batch of the call (about 16 MB of transforms at least, 256 MB at most)
    const bool real = kind == TUNE_R2C || kind == TUNE_C2R;
    const size_t per = (size_t)(real ? 2u * n + 2u : n) * sizeof(float2);  // widest row of either side
    size_t tb = std::max<size_t>(std::max(batch, 1u), (16u << 20) / per);
    tb = std::min<size_t>(tb, std::max<size_t>(1, (256u << 20) / per));
    TuneBuffers b;
    void* x = b.alloc(per * tb);
    void* y = b.alloc(per * tb);
    void* scratch = real ? b.alloc((size_t)n * sizeof(float2) * tb) : nullptr;
    if (!b.ok || cudaStreamCreateWithFlags(&b.s, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const size_t count = per * tb / sizeof(float2);
    k_fill<<<(unsigned)((count + 255) / 256), 256, 0, b.s>>>((float2*)x, count, 12345u);
    float best = 0.f;
    int bestIdx = -1;
    const bool verbose = tune_verbose();
    for (size_t i = 0; i < cands.size(); ++i) {
        bool ok = false;
        const float ms = time_batched(base, cands[i], kind, mode, x, y, scratch, (uint32_t)tb, b.s, &ok);
        if (verbose)
            fprintf(stderr, "fftlib_b200 tune %s: %s -> %s\n", key.c_str(), encode(cands[i]).c_str(),
                    ok ? (std::to_string(ms * 1e3f) + " us").c_str() : "failed");
        if (ok && (bestIdx < 0 || ms < best)) {
            best = ms;
            bestIdx = (int)i;
        }
    }
    if (bestIdx < 0) return false;
    *out = cands[(size_t)bestIdx];
    cache_put(key, encode(*out));
    return true;
}

bool tune_i16(uint32_t n, uint32_t batch, I16Choice* out)
{
    if (n < 16u || n > 16384u || (n & (n - 1u))) return false;
    int dev = 0;
    cudaDeviceProp prop;
    if (!device_of(&dev, &prop)) return false;
    const int sms = prop.multiProcessorCount;
    std::vector<I16Choice> cands;
    for (uint32_t tg : i16_tg_candidates(n)) {
        const int resident = i16_resident(n, tg, 3u);
        cands.push_back(I16Choice{tg, 0u, 3u});
        for (int k = 1; k <= 2 && k < resident; ++k) cands.push_back(I16Choice{tg, (uint32_t)(k * sms), 3u});
        // the 64-register build, when shared memory lets a fourth CTA in
        if (i16_resident(n, tg, 4u) > resident) cands.push_back(I16Choice{tg, 0u, 4u});
    }
    if (cands.empty()) return false;
    const std::string key = key_of(prop, n, batch, "c2c:i16");
    std::lock_guard<std::mutex> lock(g_tmu);
    std::string val;
    if (cache_get(key, &val)) {
        std::istringstream is(val);
        I16Choice c{};
        if (is >> c.tg >> c.gridCap >> c.minBlocks)
            for (const I16Choice& k : cands)
                if (k.tg == c.tg && k.gridCap == c.gridCap && k.minBlocks == c.minBlocks) {
                    *out = k;
                    return true;
                }
    }
    const size_t per = (size_t)n * 2u * sizeof(int16_t);
    size_t tb = std::max<size_t>(std::max(batch, 1u), (16u << 20) / per);
    tb = std::min<size_t>(tb, std::max<size_t>(1, (256u << 20) / per));
    TuneBuffers b;
    short2* x = (short2*)b.alloc(per * tb);
    short2* y = (short2*)b.alloc(per * tb);
    int16_t* w = (int16_t*)b.alloc((size_t)n * 2u * sizeof(int16_t));
    uint32_t* sh = (uint32_t*)b.alloc(8u * sizeof(uint32_t));
    if (!b.ok || cudaStreamCreateWithFlags(&b.s, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const uint32_t ones[8] = {1u, 1u, 1u, 1u, 1u, 1u, 1u, 1u};
    if (FFTLIB_b200_tw_gen_i16_device(w, n, b.s) != FFTLIB_SUCCESS ||
        cudaMemcpyAsync(sh, ones, sizeof(ones), cudaMemcpyHostToDevice, b.s) != cudaSuccess ||
        cudaStreamSynchronize(b.s) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const size_t count = (size_t)n * tb;
    k_fill_i16<<<(unsigned)((count + 255) / 256), 256, 0, b.s>>>(x, count, 12345u);
    float best = 0.f;
    int bestIdx = -1;
    const bool verbose = tune_verbose();
    for (size_t i = 0; i < cands.size(); ++i) {
        bool ok = false;
        const I16Choice c = cands[i];
        const float ms = time_runs(
            [&] {
                return launch_fft_i16((const int16_t*)x, (int16_t*)y, w, sh, n, (uint32_t)tb, b.s, c.tg, c.gridCap,
                                      c.minBlocks);
            },
            b.s, &ok);
        if (verbose)
            fprintf(stderr, "fftlib_b200 tune %s: %u %u %u -> %s\n", key.c_str(), c.tg, c.gridCap, c.minBlocks,
                    ok ? (std::to_string(ms * 1e3f) + " us").c_str() : "failed");
        if (ok && (bestIdx < 0 || ms < best)) {
            best = ms;
            bestIdx = (int)i;
        }
    }
    if (bestIdx < 0) return false;
    *out = cands[(size_t)bestIdx];
    cache_put(key, std::to_string(out->tg) + " " + std::to_string(out->gridCap) + " " +
                       std::to_string(out->minBlocks));
    return true;
}

} // namespace fftb200
