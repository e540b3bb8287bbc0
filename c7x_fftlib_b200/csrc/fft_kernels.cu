// fft_kernels.cu -- dispatch over the FP32 engine instantiations and the
// FP64 twiddle-table generator.
#include "fft_engine.h"

namespace fftb200 {

template <int EMAX, int MAXT>
cudaError_t launch_generic(const FftArgs& a, cudaStream_t s);
extern template cudaError_t launch_generic<8, 1024>(const FftArgs&, cudaStream_t);
extern template cudaError_t launch_generic<16, 512>(const FftArgs&, cudaStream_t);
extern template cudaError_t launch_generic<32, 512>(const FftArgs&, cudaStream_t);

// W[i] = exp(-2 pi i (i stride mod n) / n) for i < count, evaluated in FP64
// with the angle reduced exactly in integers (sincospi of 2 r / n,
// r = i stride mod n) and rounded once to FP32.
__global__ void k_twiddle_f64(float2* __restrict__ w, uint32_t n, uint32_t count, uint32_t stride)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const uint32_t r = (uint32_t)(((uint64_t)i * stride) % n);
    double s, c;
    sincospi(2.0 * (double)r / (double)n, &s, &c);
    w[i] = make_float2((float)c, (float)(-s));
}

// Per-pass blocks: the angle 2 pi (q k mod Ns R) / (Ns R) is reduced
// exactly in integers before the FP64 sincospi.
__global__ void k_twiddle_passes(float2* __restrict__ w, const TwiddlePasses tp)
{
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= tp.total) return;
    uint32_t p = 0;
    while (p + 1 < tp.P && e >= tp.off[p + 1]) ++p;
    const uint32_t l = e - tp.off[p];
    const uint32_t ns = tp.Ns[p], m = ns * tp.R[p];
    const uint32_t q = l / ns + 1u, k = l % ns;
    const uint32_t r = (uint32_t)(((uint64_t)q * k) % m);
    double s, c;
    sincospi(2.0 * (double)r / (double)m, &s, &c);
    w[e] = make_float2((float)c, (float)(-s));
}

int engine_max_threads(int emax)
{
    switch (emax) {
    case 8: return 1024;
    case 16: return 512;
    case 32: return 512;
    default: return 0;
    }
}

void register_static_a(std::vector<StaticEntry>& out);
void register_static_b(std::vector<StaticEntry>& out);
void register_static_c(std::vector<StaticEntry>& out);
void register_static_d(std::vector<StaticEntry>& out);
void register_static_e(std::vector<StaticEntry>& out);
void register_static_f(std::vector<StaticEntry>& out);
void register_static_g(std::vector<StaticEntry>& out);
void register_static_h(std::vector<StaticEntry>& out);
void register_static_i(std::vector<StaticEntry>& out);
void register_static_j(std::vector<StaticEntry>& out);
void register_static_k(std::vector<StaticEntry>& out);
void register_static_l(std::vector<StaticEntry>& out);
void register_static_m(std::vector<StaticEntry>& out);
void register_static_n(std::vector<StaticEntry>& out);
void register_static_o(std::vector<StaticEntry>& out);
void register_static_p(std::vector<StaticEntry>& out);
void register_static_q(std::vector<StaticEntry>& out);
void register_static_r(std::vector<StaticEntry>& out);

const std::vector<StaticEntry>& static_schedules()
{
    static const std::vector<StaticEntry> table = [] {
        std::vector<StaticEntry> t;
        register_static_a(t);
        register_static_b(t);
        register_static_c(t);
        register_static_d(t);
        register_static_e(t);
        register_static_f(t);
        register_static_g(t);
        register_static_h(t);
        register_static_i(t);
        register_static_j(t);
        register_static_k(t);
        register_static_l(t);
        register_static_m(t);
        register_static_n(t);
        register_static_o(t);
        register_static_p(t);
        register_static_q(t);
        register_static_r(t);
        return t;
    }();
    return table;
}

namespace {
const StaticEntry* find_static(const FftArgs& a, int emax)
{
    for (const StaticEntry& e : static_schedules()) {
        if (e.n != a.N || e.emax != emax || e.T != a.T || e.P != (int)a.P) continue;
        bool same = true;
        for (int p = 0; p < e.P; ++p) same = same && (e.R[p] == a.pass[p].R);
        if (same && a.T * tile_group(a) <= (uint32_t)e.maxThreads) return &e;
    }
    return nullptr;
}
} // namespace

int static_max_threads(uint32_t n, int emax, uint32_t T, int P, const int* R)
{
    for (const StaticEntry& e : static_schedules()) {
        if (e.n != n || e.emax != emax || e.T != T || e.P != P) continue;
        bool same = true;
        for (int p = 0; p < P; ++p) same = same && (e.R[p] == R[p]);
        if (same) return e.maxThreads;
    }
    return 0;
}

int static_pipelined_resident(uint32_t n, int emax, uint32_t T, int P, const int* R)
{
    for (const StaticEntry& e : static_schedules()) {
        if (e.n != n || e.emax != emax || e.T != T || e.P != P) continue;
        bool same = true;
        for (int p = 0; p < P; ++p) same = same && (e.R[p] == R[p]);
        if (same) return e.residentPipelined[IO_C2C] ? e.residentPipelined[IO_C2C]() : 0;
    }
    return 0;
}

cudaError_t launch_fft(const FftArgs& a, int emax, cudaStream_t s)
{
    if (a.batch == 0) return cudaSuccess;
    if (small_fft_eligible(a)) return launch_fft_small(a, s);
    if (const StaticEntry* st = find_static(a, emax)) {
        // the pipelined kernel brings whole tiles in with bulk copies, so the
        // static kernel's staged I/O (for transforms of few threads) is moot
        // inputs: rows of N (c2c, r2c) or N + 1 bins (c2r inMode 0, which
        // the stage holds beside its padded exchange layout for N >= 64)
        const bool rowsOk = ((a.ioMode == IO_C2C || a.ioMode == IO_R2C_SPLIT) && a.inBatch == (int64_t)a.N) ||
                            (a.ioMode == IO_C2R_SPLIT && !a.realMode && a.inBatch == (int64_t)a.N + 1 && a.N >= 64u);
        const auto pipe = a.ioMode >= 0 && a.ioMode <= IO_C2R_SPLIT ? st->launchPipelined[a.ioMode] : nullptr;
        const bool pipelinable = pipe && !a.noPipe && a.err && rowsOk && !a.batchMinor && !a.perCh &&
                                 a.inElem == 1 && a.outElem == 1 && ((uintptr_t)a.in & 15u) == 0;
        if (pipelinable) {
            FftArgs b = a;
            b.staged = 0;
            return pipe(b, s);
        }
        return st->launch(a, s);
    }
    switch (emax) {
    case 8: return launch_generic<8, 1024>(a, s);
    case 16: return launch_generic<16, 512>(a, s);
    case 32: return launch_generic<32, 512>(a, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_twiddle_passes(float2* w, const TwiddlePasses& tp, cudaStream_t s)
{
    if (tp.total == 0) return cudaSuccess;
    k_twiddle_passes<<<(tp.total + 255) / 256, 256, 0, s>>>(w, tp);
    return cudaGetLastError();
}

cudaError_t launch_twiddle(float2* w, uint32_t n, uint32_t count, cudaStream_t s, uint32_t stride)
{
    if (count == 0) return cudaSuccess;
    k_twiddle_f64<<<(count + 255) / 256, 256, 0, s>>>(w, n, count, stride);
    return cudaGetLastError();
}

} // namespace fftb200
