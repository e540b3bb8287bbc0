// plan.cu -- FP32 FFT planning, plan cache and launch sequences.
#include "plan.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <sstream>

#include "fft_engine.h"
#include "fft_split.h"

namespace fftb200 {

bool is_235(uint32_t n)
{
    if (n == 0) return false;
    while (n % 2u == 0u) n /= 2u;
    while (n % 3u == 0u) n /= 3u;
    while (n % 5u == 0u) n /= 5u;
    return n == 1u;
}

namespace {

// In-register DFT sizes the engine carries (2^a 3^b 5^c up to 32).
const int kRadices[] = {32, 30, 27, 25, 24, 20, 18, 16, 15, 12, 10, 9, 8, 6, 5, 4, 3, 2};
const int kEmax[] = {8, 16, 32};

int min_radix(int emax) { return emax >= 32 ? 8 : 1; }

void enumerate(uint32_t rem, int maxIdx, std::vector<int>& cur, std::vector<std::vector<int>>& out,
               size_t maxLen)
{
    if (rem == 1u) {
        out.push_back(cur);
        return;
    }
    if (cur.size() >= maxLen) return;
    for (int i = maxIdx; i < (int)(sizeof(kRadices) / sizeof(int)); ++i) {
        const int r = kRadices[i];
        if (rem % (uint32_t)r) continue;
        cur.push_back(r);
        enumerate(rem / (uint32_t)r, i, cur, out, maxLen);
        cur.pop_back();
    }
}

// Score a radix sequence on an engine width: each pass is one shared-memory
// round trip; idle butterfly slots and wider register files cost extra.
bool evaluate(uint32_t n, const int* seq, int len, int emax, EnginePlan* e, bool pipelined = false)
{
    // widths without a runtime-engine instantiation (the mixed-batch kernel's)
    // are capped by the caller's maxT instead
    const int maxT = engine_max_threads(emax) ? engine_max_threads(emax) : 1024;
    if (len > kMaxPasses) return false;
    uint32_t T = 1;
    for (int i = 0; i < len; ++i) {
        const int r = seq[i];
        if (r > emax || r < min_radix(emax)) return false;
        const uint32_t nb = n / (uint32_t)r;
        const uint32_t bmax = (uint32_t)(emax / r);
        T = std::max(T, (nb + bmax - 1) / bmax);
    }
    if ((int)T > maxT) return false;
    double score = 0.0;
    for (int i = 0; i < len; ++i) {
        const uint32_t nb = n / (uint32_t)seq[i];
        const uint32_t b = (nb + T - 1) / T;
        const double util = (double)nb / (double)(T * b);
        score += 1.0 + 0.5 * (1.0 / util - 1.0);
    }
    // measured on B200: the 32-wide engine (90-115 registers per thread)
    // runs at about a third of the 16-wide one's throughput, so it is kept
    // for lengths nothing narrower can plan
    score += emax == 32 ? 2.5 : emax == 16 ? 0.15 : 0.0;
    // a one-pass schedule cannot run in the bulk-copy pipelined kernel (its
    // first pass is its last): at N = 8 and 16 it measured 2.7 TB/s, at 9,
    // 10 and 12 2.1 TB/s, against 4.2-4.3 TB/s for the two-pass pipelined
    // N = 18, 20, so from N = 8 up two-pass schedules win
    if (pipelined && len == 1 && n >= 8u) score += 1.5;
    e->n = n;
    e->emax = emax;
    e->T = T;
    e->P = len;
    for (int i = 0; i < len; ++i) e->R[i] = seq[i];
    e->score = score;
    return true;
}

} // namespace

std::vector<EnginePlan> engine_candidates(uint32_t n, int emaxOnly, uint32_t maxT)
{
    std::vector<EnginePlan> out;
    if (!is_235(n)) return out;
    if (n == 1u) {
        EnginePlan e;
        e.n = 1;
        e.emax = 8;
        e.T = 1;
        e.P = 1;
        e.R[0] = 1;
        out.push_back(e);
        return out;
    }
    std::vector<std::vector<int>> seqs;
    std::vector<int> cur;
    enumerate(n, 0, cur, seqs, kMaxPasses);
    for (const auto& s : seqs) {
        const int only[1] = {emaxOnly};
        for (int emax : (emaxOnly ? std::vector<int>(only, only + 1) : std::vector<int>(kEmax, kEmax + 3))) {
            EnginePlan e;
            if (evaluate(n, s.data(), (int)s.size(), emax, &e, emaxOnly == 0) && (!maxT || e.T <= maxT))
                out.push_back(e);
        }
    }
    std::stable_sort(out.begin(), out.end(),
                     [](const EnginePlan& a, const EnginePlan& b) { return a.score < b.score; });
    return out;
}

namespace {

// Depth-first search over non-increasing radix sequences, keeping only the
// best schedule (no heap allocation).
void search_best(uint32_t n, uint32_t rem, int maxIdx, int* seq, int len, EnginePlan* best, bool* found)
{
    if (rem == 1u) {
        for (int emax : kEmax) {
            EnginePlan e;
            if (evaluate(n, seq, len, emax, &e, true) && (!*found || e.score < best->score)) {
                *best = e;
                *found = true;
            }
        }
        return;
    }
    if (len >= kMaxPasses) return;
    for (int i = maxIdx; i < (int)(sizeof(kRadices) / sizeof(int)); ++i) {
        const int r = kRadices[i];
        if (rem % (uint32_t)r) continue;
        seq[len] = r;
        search_best(n, rem / (uint32_t)r, i, seq, len + 1, best, found);
    }
}

} // namespace

bool plan_engine(uint32_t n, EnginePlan* out)
{
    if (n == 0 || n > kMaxSingleN || !is_235(n)) return false;
    if (n == 1u) {
        EnginePlan e;
        e.n = 1;
        e.emax = 8;
        e.T = 1;
        e.P = 1;
        e.R[0] = 1;
        *out = e;
        return true;
    }
    // a fixed-size schedule measured faster than the heuristic's pick
    for (const StaticEntry& st : static_schedules()) {
        if (st.n != n || !st.preferred) continue;
        EnginePlan e;
        e.n = n;
        e.emax = st.emax;
        e.T = st.T;
        e.P = st.P;
        for (int i = 0; i < st.P; ++i) e.R[i] = st.R[i];
        *out = e;
        return true;
    }
    int seq[kMaxPasses];
    bool found = false;
    EnginePlan best;
    search_best(n, n, 0, seq, 0, &best, &found);
    if (found) *out = best;
    return found;
}

std::string describe(const EnginePlan& e)
{
    std::ostringstream os;
    os << "N=" << e.n << " E=" << e.emax << " T=" << e.T << " radices=";
    for (int p = 0; p < e.P; ++p) os << (p ? "x" : "") << e.R[p];
    return os.str();
}

const ErrorWord& error_word()
{
    static std::mutex mu;
    static ErrorWord words[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        static ErrorWord none;
        return none;
    }
    std::lock_guard<std::mutex> lock(mu);
    ErrorWord& w = words[dev];
    if (!w.dev) {
        void* h = nullptr;
        if (cudaHostAlloc(&h, sizeof(uint32_t), cudaHostAllocMapped) == cudaSuccess) {
            *(volatile uint32_t*)h = 0;
            void* d = nullptr;
            if (cudaHostGetDevicePointer(&d, h, 0) == cudaSuccess) {
                w.host = (volatile uint32_t*)h;
                w.dev = (uint32_t*)d;
            } else {
                cudaFreeHost(h);
                cudaGetLastError();
            }
        } else {
            cudaGetLastError();
        }
    }
    return w;
}

uint32_t take_device_error()
{
    const ErrorWord& w = error_word();
    if (!w.host) return 0;
    const uint32_t v = *w.host;
    if (v) *w.host = 0;
    return v;
}

FftArgs engine_args(const EnginePlan& e, const float2* tw)
{
    FftArgs a{};
    a.tw = tw;
    a.N = e.n;
    a.T = e.T;
    a.P = (uint32_t)e.P;
    uint32_t ns = 1, off = 0;
    for (int p = 0; p < e.P; ++p) {
        const uint32_t r = (uint32_t)e.R[p];
        a.pass[p].R = (int32_t)r;
        a.pass[p].Ns = ns;
        a.pass[p].nsMagic = fastdiv_magic(ns);
        a.pass[p].stride = e.n / r;
        a.pass[p].twOffset = off;
        if (p > 0) off += (r - 1u) * ns;
        ns *= r;
    }
    a.scale = 1.0f;
    a.nMagic = fastdiv_magic(e.n);
    a.slen = smem_len(e.n);
    a.inCount = e.n;
    a.inMagic = a.nMagic;
    a.ioMode = IO_C2C;
    return a;
}

void finalize_launch(FftArgs& a, const EnginePlan& e, bool contiguousIn, bool contiguousOut)
{
    const uint32_t maxT = (uint32_t)engine_max_threads(e.emax);
    uint32_t M;
    if (a.batchMinor) {
        M = std::max(1u, std::min(16u, maxT / e.T));
    } else {
        // T >= 128: one transform per CTA (the pipelined kernels' shape)
        M = e.T >= 128u ? 1u : 256u / e.T;
        M = std::max(1u, std::min(M, maxT / e.T));
    }
    const uint32_t bytesPer = a.slen * (uint32_t)sizeof(float2);
    M = std::min(M, std::max(1u, (64u * 1024u) / bytesPer));
    M = std::max(1u, std::min(M, a.batch));
    a.M = M;
    a.staged = (!a.batchMinor && e.T < 8u && contiguousIn && (contiguousOut || a.ioMode == IO_R2C_SPLIT)) ? 1 : 0;
}

// ---------------------------------------------------------------------------
// plan cache
// ---------------------------------------------------------------------------

namespace {

std::mutex g_mu;
std::map<std::pair<int, uint32_t>, ComplexPlan*> g_plans;

cudaError_t make_table(float2** p, uint32_t n, uint32_t count, cudaStream_t s)
{
    cudaError_t e = cudaMalloc((void**)p, sizeof(float2) * std::max(count, 1u));
    if (e != cudaSuccess) return e;
    return launch_twiddle(*p, n, count, s);
}

} // namespace

// Per-pass twiddle blocks of a single-kernel schedule (see PassInfo).
cudaError_t make_pass_table(float2** p, const EnginePlan& e, cudaStream_t s)
{
    TwiddlePasses tp{};
    uint32_t ns = 1, off = 0;
    for (int i = 0; i < e.P; ++i) {
        const uint32_t r = (uint32_t)e.R[i];
        if (i > 0) {
            tp.R[tp.P] = r;
            tp.Ns[tp.P] = ns;
            tp.off[tp.P] = off;
            tp.P++;
            off += (r - 1u) * ns;
        }
        ns *= r;
    }
    tp.total = off;
    cudaError_t err = cudaMalloc((void**)p, sizeof(float2) * std::max(off, 1u));
    if (err != cudaSuccess) return err;
    return launch_twiddle_passes(*p, tp, s);
}

namespace {

// Largest divisor of x that is at most cap.
uint32_t largest_divisor(uint32_t x, uint32_t cap)
{
    for (uint32_t d = std::min(x, cap); d > 1u; --d)
        if (x % d == 0u) return d;
    return 1u;
}

void split_dfs(uint32_t rest, int left, uint32_t* cur, int depth, double* best, int* bestG, uint32_t* bestR)
{
    if (left == 0) {
        if (rest != 1u) return;
        // balanced first (the largest radix bounds the tile size), then runs:
        // pass i >= 1 tiles its columns in runs of a divisor of the product
        // of the radices before it
        uint32_t mx = 0, ns = 1;
        double runs = 0.0;
        for (int i = 0; i < depth; ++i) {
            mx = std::max(mx, cur[i]);
            if (i > 0) runs += 16.0 / (double)largest_divisor(ns, 16u);
            ns *= cur[i];
        }
        const double score = (double)mx + runs;
        if (score < *best) {
            *best = score;
            *bestG = depth;
            for (int i = 0; i < depth; ++i) bestR[i] = cur[i];
        }
        return;
    }
    for (uint32_t d = 2; d <= std::min(rest, kMaxGlobalRadix); ++d) {
        if (rest % d) continue;  // every divisor of a 2^a 3^b 5^c length is a single-kernel length
        cur[depth] = d;
        split_dfs(rest / d, left - 1, cur, depth + 1, best, bestG, bestR);
    }
}

} // namespace

bool split_global(uint32_t n, int* G, uint32_t* R)
{
    if (!is_235(n)) return false;
    for (int g = 2; g <= kMaxGlobal; ++g) {
        uint32_t cur[kMaxGlobal];
        double best = 1e300;
        int bestG = 0;
        split_dfs(n, g, cur, 0, &best, &bestG, R);
        if (bestG) {
            *G = bestG;
            return true;
        }
    }
    return false;
}

ComplexPlan* get_complex_plan(uint32_t n, bool needSplit, cudaError_t* err)
{
    *err = cudaSuccess;
    if (!is_235(n)) {
        *err = cudaErrorInvalidValue;
        return nullptr;
    }
    int dev = 0;
    if ((*err = cudaGetDevice(&dev)) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lock(g_mu);
    ComplexPlan*& slot = g_plans[{dev, n}];
    cudaStream_t s = cudaStreamPerThread;
    if (!slot) {
        ComplexPlan* p = new ComplexPlan();
        p->device = dev;
        p->n = n;
        cudaDeviceGetAttribute(&p->sms, cudaDevAttrMultiProcessorCount, dev);
        if (n <= kMaxSingleN && plan_engine(n, &p->eng)) {
            *err = make_pass_table(&p->tw, p->eng, s);
        } else if (split_global(n, &p->G, p->R)) {
            p->multiPass = true;
            // W_n^p = twLo[p mod L] twHi[p / L], L the power of two at or above sqrt(n)
            uint32_t bits = 0;
            while ((1ull << (2 * bits)) < n) ++bits;
            p->twLoBits = bits;
            const uint32_t lo = 1u << bits, hi = (n + lo - 1u) / lo;
            *err = make_table(&p->twLo, n, lo, s);
            if (*err == cudaSuccess) {
                *err = cudaMalloc((void**)&p->twHi, sizeof(float2) * hi);
                if (*err == cudaSuccess) *err = launch_twiddle(p->twHi, n, hi, s, lo);
            }
            for (int g = 0; g < p->G && *err == cudaSuccess; ++g) {
                plan_engine(p->R[g], &p->engG[g]);
                *err = make_pass_table(&p->twG[g], p->engG[g], s);
            }
        } else {
            *err = cudaErrorInvalidValue;
        }
        if (*err == cudaSuccess) *err = cudaStreamSynchronize(s);
        if (*err != cudaSuccess) {
            cudaFree(p->tw);
            for (float2* t : p->twG) cudaFree(t);
            cudaFree(p->twLo);
            cudaFree(p->twHi);
            delete p;
            g_plans.erase({dev, n});
            return nullptr;
        }
        slot = p;
    }
    if (needSplit && !slot->twSplit) {
        *err = make_table(&slot->twSplit, 2u * n, n, s);
        if (*err == cudaSuccess) *err = cudaStreamSynchronize(s);
        if (*err != cudaSuccess) {
            cudaFree(slot->twSplit);
            slot->twSplit = nullptr;
            return nullptr;
        }
    }
    return slot;
}

namespace {

// Tuned plans and the real kinds' own schedules, per (device, length and
// choice).
std::map<std::pair<int, std::string>, ComplexPlan*> g_tuned_plans;

std::string choice_key(uint32_t n, const BatchedChoice& c)
{
    return std::to_string(n) + " " + describe(c.eng) + " g" + std::to_string(c.gridCap) + " m" +
           std::to_string(c.tileM) + (c.noPipe ? " np" : "");
}

void free_plan(ComplexPlan* p)
{
    cudaSetDevice(p->device);
    cudaFree(p->tw);
    for (float2* t : p->twG) cudaFree(t);
    cudaFree(p->twLo);
    cudaFree(p->twHi);
    cudaFree(p->twSplit);
    delete p;
}

} // namespace

namespace {

const StaticEntry* static_of(const EnginePlan& e)
{
    for (const StaticEntry& st : static_schedules()) {
        if (st.n != e.n || st.emax != e.emax || st.T != e.T || st.P != e.P) continue;
        bool same = true;
        for (int i = 0; i < e.P; ++i) same = same && st.R[i] == e.R[i];
        if (same) return &st;
    }
    return nullptr;
}

// Without the autotuner, the real kinds take a fixed-size schedule of the
// same length whose pipelined kernel runs their split in registers (the
// first pass for c2r with inMode 0, the last for r2c) when the planner's
// does not and one is registered (e.g. 8 x 16 x 16 beside 16 x 16 x 8 for
// h = 2048).
bool real_kind_schedule(const ComplexPlan* base, int kind, int mode, BatchedChoice* c)
{
    const bool wantFirst = kind == TUNE_C2R && mode == 0, wantLast = kind == TUNE_R2C;
    if (!wantFirst && !wantLast) return false;
    const StaticEntry* cur = static_of(base->eng);
    if (cur && ((wantFirst && cur->mirrorFirst) || (wantLast && cur->mirrorLast))) return false;
    for (const StaticEntry& st : static_schedules()) {
        if (st.n != base->n || !((wantFirst && st.mirrorFirst) || (wantLast && st.mirrorLast))) continue;
        EnginePlan e;
        e.n = st.n;
        e.emax = st.emax;
        e.T = st.T;
        e.P = st.P;
        for (int i = 0; i < st.P; ++i) e.R[i] = st.R[i];
        c->eng = e;
        return true;
    }
    return false;
}

} // namespace

ComplexPlan* get_batched_plan(uint32_t n, bool needSplit, int kind, int mode, uint32_t batch, cudaError_t* err)
{
    ComplexPlan* base = get_complex_plan(n, needSplit, err);
    if (!base || base->multiPass) return base;
    BatchedChoice c;
    const bool tuned = autotune_enabled() && tune_batched(base, kind, mode, batch, &c);
    if (!tuned && !real_kind_schedule(base, kind, mode, &c)) return base;
    std::lock_guard<std::mutex> lock(g_mu);
    ComplexPlan*& slot = g_tuned_plans[{base->device, choice_key(n, c) + (tuned ? " tuned" : "")}];
    cudaStream_t s = cudaStreamPerThread;
    if (!slot) {
        ComplexPlan* p = new ComplexPlan();
        p->device = base->device;
        p->sms = base->sms;
        p->n = n;
        p->eng = c.eng;
        p->gridCap = c.gridCap;
        p->tileM = c.tileM;
        p->noPipe = c.noPipe;
        p->tuned = tuned;
        *err = make_pass_table(&p->tw, p->eng, s);
        if (*err == cudaSuccess) *err = cudaStreamSynchronize(s);
        if (*err != cudaSuccess) {
            free_plan(p);
            g_tuned_plans.erase({base->device, choice_key(n, c) + (tuned ? " tuned" : "")});
            return nullptr;
        }
        slot = p;
    }
    if (needSplit && !slot->twSplit) {
        *err = make_table(&slot->twSplit, 2u * n, n, s);
        if (*err == cudaSuccess) *err = cudaStreamSynchronize(s);
        if (*err != cudaSuccess) {
            cudaFree(slot->twSplit);
            slot->twSplit = nullptr;
            return nullptr;
        }
    }
    return slot;
}

std::string describe_plan(const ComplexPlan* p)
{
    if (p->multiPass) {
        std::string s = "planner: global passes";
        for (int g = 0; g < p->G; ++g)
            s += (g ? " x " : " ") + std::to_string(p->R[g]) + " [" + describe(p->engG[g]) + "]";
        return s;
    }
    const EnginePlan& e = p->eng;
    if (small_fft_length(p->n)) return std::string(p->tuned ? "tuned: " : "planner: ") + "N=" + std::to_string(p->n) +
                                      " (c2c: one transform per thread; real kinds: " + describe(e) + ")";
    const bool fixed = static_max_threads(p->n, e.emax, e.T, e.P, e.R) != 0;
    const bool pipe = fixed && !p->noPipe && static_pipelined_resident(p->n, e.emax, e.T, e.P, e.R) > 0;
    std::string s = std::string(p->tuned ? "tuned: " : "planner: ") + describe(e);
    s += fixed ? (pipe ? " (fixed-size pipelined kernel" : " (fixed-size kernel") : " (runtime-radix engine";
    if (pipe && p->gridCap) s += ", " + std::to_string(p->gridCap) + " CTAs";
    if (!pipe && p->tileM) s += ", " + std::to_string(p->tileM) + " transforms per CTA";
    return s + ")";
}

void release_all_plans()
{
    std::lock_guard<std::mutex> lock(g_mu);
    int cur = 0;
    cudaGetDevice(&cur);
    for (auto& kv : g_plans)
        if (kv.second) free_plan(kv.second);
    for (auto& kv : g_tuned_plans)
        if (kv.second) free_plan(kv.second);
    g_plans.clear();
    g_tuned_plans.clear();
    cudaSetDevice(cur);
}

// ---------------------------------------------------------------------------
// launch sequences
// ---------------------------------------------------------------------------

namespace {

constexpr uint32_t kMaxSmemBytes = 227u * 1024u;

// Staged tile of one global pass: M columns of one channel (M divides
// perCh, and ns when ns > 1, so a tile never straddles a channel or an
// output group), loaded and stored as runs of M adjacent values through
// shared memory and computed Mc columns at a time within the kernel's thread
// limit (the fixed-size kernel's when the schedule has one). M is the
// largest such divisor up to 16 that leaves two CTAs per SM room in shared
// memory, smaller (not below 4) where that leaves fewer than 2 tiles per SM.
void tile_global(FftArgs& a, const EnginePlan& e, uint32_t perCh, uint32_t ns, int sms)
{
    a.staged = 1;
    a.batchMinor = 0;
    a.perCh = perCh;
    a.slen = smem_len(e.n);
    a.inCount = e.n;
    a.inMagic = fastdiv_magic(e.n);
    const uint32_t bytesPer = a.slen * (uint32_t)sizeof(float2);
    const uint32_t mMax = std::max(1u, std::min(16u, kMaxSmemBytes / 2u / bytesPer));
    const uint32_t want = 2u * (uint32_t)std::max(sms, 1);
    uint32_t M = 1;
    for (uint32_t d = mMax; d >= 1u; --d) {
        if (perCh % d || (ns > 1u && ns % d)) continue;
        if (M == 1u) M = d;                    // the largest valid tile
        if (d >= 4u && a.batch / d >= want) {  // prefer one that fills the device
            M = d;
            break;
        }
        if (d < 4u) break;
    }
    const int st = static_max_threads(e.n, e.emax, e.T, e.P, e.R);
    const uint32_t cap = st ? (uint32_t)st : (uint32_t)engine_max_threads(e.emax);
    uint32_t Mc = 1;
    for (uint32_t d = M; d >= 1u; --d) {
        if (M % d == 0u && e.T * d <= cap) {
            Mc = d;
            break;
        }
    }
    a.M = M;
    a.Mc = Mc;
    a.mMagic = fastdiv_magic(M);
}

// Complex transform of `batch` rows of length n of `in` into `out` by G
// global Stockham passes, one launch each for the whole batch. Pass g (radix
// R, ns = product of the radices before it) runs the R-point sub-transform
// of every column j < n/R: inputs in[j + q n/R], q < R, times
// W_{ns R}^{q (j mod ns)} (pass g > 0), outputs to
// out[(j / ns) ns R + (j mod ns) + q ns]. Both sides move runs of adjacent
// columns; the last pass (ns = n/R) writes where it reads, so it may run in
// place. Passes alternate between out and in (in is overwritten when G > 2)
// and the last one lands in out.
cudaError_t run_global(const ComplexPlan* p, float2* in, float2* out, uint32_t batch, bool inverse, cudaStream_t s)
{
    const uint32_t n = p->n;
    const float2* src = in;
    uint32_t ns = 1;
    for (int g = 0; g < p->G; ++g) {
        const uint32_t R = p->R[g], cols = n / R;
        float2* dst = (g % 2 == 0 || g + 1 == p->G) ? out : in;
        FftArgs a = engine_args(p->engG[g], p->twG[g]);
        a.err = error_word().dev;
        a.in = src;
        a.out = dst;
        a.batch = batch * cols;
        a.inChStride = a.outChStride = n;
        a.inBatch = 1;
        a.inElem = cols;
        a.outBatch = 1;
        a.outElem = ns;
        a.outGroup = ns;
        a.outGroupStride = (int64_t)ns * R;
        if (g > 0) {
            a.twLo = p->twLo;
            a.twHi = p->twHi;
            a.twLoBits = p->twLoBits;
            a.twNs = ns;
            a.twStep = n / (ns * R);
        }
        a.conjIn = (g == 0 && inverse) ? 1 : 0;
        if (g + 1 == p->G) {
            a.conjOut = inverse ? 1 : 0;
            a.scale = inverse ? 1.0f / (float)n : 1.0f;
        }
        tile_global(a, p->engG[g], cols, ns, p->sms);
        cudaError_t e = launch_fft(a, p->engG[g].emax, s);
        if (e != cudaSuccess) return e;
        src = dst;
        ns *= R;
    }
    return cudaSuccess;
}

} // namespace

namespace {

// The plan's launch choices on top of finalize_launch's (tileM only lowers
// the transforms per CTA, so the tile still fits where the planner's did).
void apply_choice(FftArgs& a, const ComplexPlan* p)
{
    a.gridCap = p->gridCap;
    a.noPipe = p->noPipe ? 1u : 0u;
    if (p->tileM && p->tileM < a.M) a.M = p->tileM;
}

} // namespace

cudaError_t run_c2c(const ComplexPlan* p, float2* in, float2* out, uint32_t batch, bool inverse, cudaStream_t s,
                    uint32_t gridCap, bool overlapPrev)
{
    if (batch == 0) return cudaSuccess;
    if (p->multiPass) return run_global(p, in, out, batch, inverse, s);
    const uint32_t n = p->n;
    FftArgs a = engine_args(p->eng, p->tw);
    a.err = error_word().dev;
    a.in = in;
    a.out = out;
    a.batch = batch;
    a.inBatch = n;
    a.inElem = 1;
    a.outBatch = n;
    a.outElem = 1;
    a.conjIn = a.conjOut = inverse ? 1 : 0;
    a.scale = inverse ? 1.0f / (float)n : 1.0f;
    finalize_launch(a, p->eng, true, true);
    apply_choice(a, p);
    if (gridCap) a.gridCap = gridCap;
    a.overlapPrev = overlapPrev ? 1u : 0u;
    return launch_fft(a, p->eng.emax, s);
}

cudaError_t run_r2c(const ComplexPlan* p, float* x, float2* scratch, float2* y, uint32_t batch, int outmode,
                    cudaStream_t s)
{
    if (batch == 0) return cudaSuccess;
    const uint32_t h = p->n;
    if (p->multiPass) {
        if (!scratch) return cudaErrorInvalidValue;
        cudaError_t e = run_global(p, (float2*)x, scratch, batch, false, s);
        if (e != cudaSuccess) return e;
        return launch_r2c_post(scratch, y, p->twSplit, h, batch, outmode, s);
    }
    FftArgs a = engine_args(p->eng, p->tw);
    a.err = error_word().dev;
    a.in = (const float2*)x;
    a.out = y;
    a.batch = batch;
    a.inBatch = h;
    a.inElem = 1;
    a.outBatch = outmode ? 2u * h : h + 1u;
    a.outElem = 1;
    a.ioMode = IO_R2C_SPLIT;
    a.realMode = outmode ? 1 : 0;
    a.twSplit = p->twSplit;
    finalize_launch(a, p->eng, true, false);
    apply_choice(a, p);
    return launch_fft(a, p->eng.emax, s);
}

namespace {

// The single-kernel c2r stages a whole input row (inCount bins) in the
// transform's shared-memory region; the full spectrum (inMode 1) of the
// longest single-kernel lengths does not fit in one CTA's 227 KB.
bool c2r_staged_fits(uint32_t h, uint32_t inCount)
{
    return (size_t)smem_len(std::max(h, inCount)) * sizeof(float2) <= 227u * 1024u;
}

} // namespace

bool c2r_needs_scratch(const ComplexPlan* p, int inmode)
{
    const uint32_t h = p->n;
    return p->multiPass || !c2r_staged_fits(h, inmode ? 2u * h : h + 1u);
}

cudaError_t run_c2r(const ComplexPlan* p, const float2* x, float2* scratch, float* y, uint32_t batch, int inmode,
                    cudaStream_t s)
{
    if (batch == 0) return cudaSuccess;
    const uint32_t h = p->n;
    const uint32_t inCount = inmode ? 2u * h : h + 1u;
    if (!p->multiPass && !c2r_staged_fits(h, inCount)) {
        // split as a pre-pass into the work buffer, then the plain inverse
        if (!scratch) return cudaErrorInvalidValue;
        cudaError_t e = launch_c2r_pre(x, scratch, p->twSplit, h, batch, inmode, s);
        if (e != cudaSuccess) return e;
        return run_c2c(p, scratch, (float2*)y, batch, true, s);
    }
    if (p->multiPass) {
        if (!scratch) return cudaErrorInvalidValue;
        cudaError_t e = launch_c2r_pre(x, scratch, p->twSplit, h, batch, inmode, s);
        if (e != cudaSuccess) return e;
        return run_global(p, scratch, (float2*)y, batch, true, s);
    }
    FftArgs a = engine_args(p->eng, p->tw);
    a.err = error_word().dev;
    a.in = x;
    a.out = (float2*)y;
    a.batch = batch;
    a.inBatch = inCount;
    a.inElem = 1;
    a.outBatch = h;
    a.outElem = 1;
    a.ioMode = IO_C2R_SPLIT;
    a.realMode = inmode ? 1 : 0;
    a.twSplit = p->twSplit;
    a.conjIn = a.conjOut = 1;
    a.scale = 1.0f / (float)h;
    a.inCount = inCount;
    a.inMagic = fastdiv_magic(inCount);
    a.slen = smem_len(std::max(h, inCount));
    finalize_launch(a, p->eng, true, true);
    apply_choice(a, p);
    return launch_fft(a, p->eng.emax, s);
}

} // namespace fftb200
