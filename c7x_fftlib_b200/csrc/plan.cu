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
    // first pass is its last): at N = 8 and 16 it measured 2.7 TB/s, so the
    // two-pass schedules with fixed-size pipelined kernels (4x2, 8x2) win
    if (pipelined && len == 1 && (n == 8u || n == 16u)) score += 1.5;
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

// n = n1 * n2 with n1 <= n2, n1 as close to sqrt(n) as possible, both with
// single-kernel schedules.
bool split_four_step(uint32_t n, uint32_t* n1, uint32_t* n2)
{
    const uint32_t root = (uint32_t)std::sqrt((double)n);
    for (uint32_t d = root + 1; d >= 2; --d) {
        if (n % d) continue;
        const uint32_t e = n / d;
        if (d > e || e > kMaxSingleN) continue;
        EnginePlan a, b;
        if (plan_engine(d, &a) && plan_engine(e, &b)) {
            *n1 = d;
            *n2 = e;
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
        if (n <= kMaxSingleN && plan_engine(n, &p->eng)) {
            EnginePlan tuned;
            if (autotune_enabled() && tune_schedule(n, 4096, 0, 0, &tuned)) p->eng = tuned;
            *err = make_pass_table(&p->tw, p->eng, s);
        } else if (split_four_step(n, &p->n1, &p->n2)) {
            p->fourStep = true;
            plan_engine(p->n1, &p->eng1);
            plan_engine(p->n2, &p->eng2);
            *err = make_table(&p->tw, n, n, s);
            if (*err == cudaSuccess) *err = make_pass_table(&p->tw1, p->eng1, s);
            if (*err == cudaSuccess) *err = make_pass_table(&p->tw2, p->eng2, s);
        } else {
            *err = cudaErrorInvalidValue;
        }
        if (*err == cudaSuccess) *err = cudaStreamSynchronize(s);
        if (*err != cudaSuccess) {
            cudaFree(p->tw);
            cudaFree(p->tw1);
            cudaFree(p->tw2);
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

void release_all_plans()
{
    std::lock_guard<std::mutex> lock(g_mu);
    int cur = 0;
    cudaGetDevice(&cur);
    for (auto& kv : g_plans) {
        ComplexPlan* p = kv.second;
        if (!p) continue;
        cudaSetDevice(p->device);
        cudaFree(p->tw);
        cudaFree(p->tw1);
        cudaFree(p->tw2);
        cudaFree(p->twSplit);
        delete p;
    }
    g_plans.clear();
    cudaSetDevice(cur);
}

// ---------------------------------------------------------------------------
// launch sequences
// ---------------------------------------------------------------------------

namespace {

// Four-step complex transform of each length-n row of `in` (overwritten)
// into `out`: columns of the n1 x n2 view first (W_n fused into their
// store), then rows, whose outputs land transposed at k1 + n1 * k2.
cudaError_t run_four_step(const ComplexPlan* p, float2* in, float2* out, uint32_t batch, bool inverse,
                          cudaStream_t s)
{
    const uint32_t n = p->n, n1 = p->n1, n2 = p->n2;
    for (uint32_t c = 0; c < batch; ++c) {
        float2* x = in + (size_t)c * n;
        float2* y = out + (size_t)c * n;
        FftArgs a = engine_args(p->eng1, p->tw1);
        a.err = error_word().dev;
        a.in = x;
        a.out = x;
        a.batch = n2;
        a.inBatch = 1;
        a.inElem = n2;
        a.outBatch = 1;
        a.outElem = n2;
        a.batchMinor = 1;
        a.conjIn = inverse ? 1 : 0;
        a.twBig = p->tw;
        a.bigN = n;
        finalize_launch(a, p->eng1, false, false);
        cudaError_t e = launch_fft(a, p->eng1.emax, s);
        if (e != cudaSuccess) return e;

        FftArgs b = engine_args(p->eng2, p->tw2);
        b.err = error_word().dev;
        b.in = x;
        b.out = y;
        b.batch = n1;
        b.inBatch = n2;
        b.inElem = 1;
        b.outBatch = 1;
        b.outElem = n1;
        b.conjOut = inverse ? 1 : 0;
        b.scale = inverse ? 1.0f / (float)n : 1.0f;
        finalize_launch(b, p->eng2, false, false);
        e = launch_fft(b, p->eng2.emax, s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

} // namespace

cudaError_t run_c2c(const ComplexPlan* p, float2* in, float2* out, uint32_t batch, bool inverse, cudaStream_t s)
{
    if (batch == 0) return cudaSuccess;
    if (p->fourStep) return run_four_step(p, in, out, batch, inverse, s);
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
    return launch_fft(a, p->eng.emax, s);
}

cudaError_t run_r2c(const ComplexPlan* p, float* x, float2* scratch, float2* y, uint32_t batch, int outmode,
                    cudaStream_t s)
{
    if (batch == 0) return cudaSuccess;
    const uint32_t h = p->n;
    if (p->fourStep) {
        if (!scratch) return cudaErrorInvalidValue;
        cudaError_t e = run_four_step(p, (float2*)x, scratch, batch, false, s);
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
    return p->fourStep || !c2r_staged_fits(h, inmode ? 2u * h : h + 1u);
}

cudaError_t run_c2r(const ComplexPlan* p, const float2* x, float2* scratch, float* y, uint32_t batch, int inmode,
                    cudaStream_t s)
{
    if (batch == 0) return cudaSuccess;
    const uint32_t h = p->n;
    const uint32_t inCount = inmode ? 2u * h : h + 1u;
    if (!p->fourStep && !c2r_staged_fits(h, inCount)) {
        // split as a pre-pass into the work buffer, then the plain inverse
        if (!scratch) return cudaErrorInvalidValue;
        cudaError_t e = launch_c2r_pre(x, scratch, p->twSplit, h, batch, inmode, s);
        if (e != cudaSuccess) return e;
        return run_c2c(p, scratch, (float2*)y, batch, true, s);
    }
    if (p->fourStep) {
        if (!scratch) return cudaErrorInvalidValue;
        cudaError_t e = launch_c2r_pre(x, scratch, p->twSplit, h, batch, inmode, s);
        if (e != cudaSuccess) return e;
        return run_four_step(p, scratch, (float2*)y, batch, true, s);
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
    return launch_fft(a, p->eng.emax, s);
}

} // namespace fftb200
