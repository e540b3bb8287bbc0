/*
 * fftlib_caller.c -- a plain C program that uses libfftlib_b200.so the way an
 * FFTLIB application does: it includes <fftlib.h>, links the library and
 * calls the reference's entry points with host buffers, in the reference test
 * drivers' order (_checkParams / _init / _kernel for the batched kernels,
 * test/fft_c7x/FFTLIB_fft1dBatched_i32fc_c32fc_o32fc/FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_d.c:205-216;
 * getHandleSize / getSizes / twGen / init_checkParams / init /
 * exec_checkParams / exec for the DFT coordinator,
 * test/fft_c7xmma/FFTLIB_FFT_fft_ixX_cxX_oxX/FFTLIB_FFT_fft_ixX_cxX_oxX_d.c:39-154).
 *
 *   fftlib_caller layout        struct sizes and offsets, enum values
 *   fftlib_caller checkparams   the c2c / ifft checkParams coverage cases
 *                               1000-1011 (..._d.c:370-534); no GPU needed
 *   fftlib_caller run DIR       transforms on the GPU; inputs and outputs
 *                               are written to DIR as raw little-endian
 *                               arrays for the test to compare with the oracle
 *
 * Test infrastructure: built and run by tests/test_c_caller.py.
 */
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <fftlib.h>

static int failures = 0;

#define EXPECT_OK(call)                                                                        \
    do {                                                                                       \
        FFTLIB_STATUS st_ = (call);                                                            \
        if (st_ != FFTLIB_SUCCESS) {                                                           \
            fprintf(stderr, "%s:%d: %s returned %d (%s)\n", __FILE__, __LINE__, #call, (int)st_, \
                    FFTLIB_b200_lastError());                                                  \
            failures++;                                                                        \
        }                                                                                      \
    } while (0)

/* deterministic inputs: a 64-bit LCG */
static uint64_t lcg_state = 0x9E3779B97F4A7C15ull;
static uint32_t lcg_next(void)
{
    lcg_state = lcg_state * 6364136223846793005ull + 1442695040888963407ull;
    return (uint32_t)(lcg_state >> 32);
}
static float uniform_pm1(void) { return (float)((double)lcg_next() / 4294967296.0 * 2.0 - 1.0); }

static void *xmalloc(size_t bytes)
{
    void *p = NULL;
    if (posix_memalign(&p, 64, bytes ? bytes : 64) != 0) {
        fprintf(stderr, "out of host memory\n");
        exit(2);
    }
    memset(p, 0, bytes ? bytes : 64);
    return p;
}

static void dump(const char *dir, const char *name, const void *p, size_t bytes)
{
    char path[1024];
    snprintf(path, sizeof path, "%s/%s", dir, name);
    FILE *f = fopen(path, "wb");
    if (!f || fwrite(p, 1, bytes, f) != bytes) {
        fprintf(stderr, "cannot write %s\n", path);
        failures++;
    }
    if (f) fclose(f);
}

/* ---- layout ------------------------------------------------------------- */

static int layout(void)
{
    printf("sizeof_bufParams1D %zu\n", sizeof(FFTLIB_bufParams1D_t));
    printf("offset_bufParams1D_dim_x %zu\n", offsetof(FFTLIB_bufParams1D_t, dim_x));
    printf("sizeof_bufParams2D %zu\n", sizeof(FFTLIB_bufParams2D_t));
    printf("sizeof_mma_initargs %zu\n", sizeof(FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs));
    printf("offset_mma_fftSize %zu\n", offsetof(FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs, fftSize));
    printf("offset_mma_shiftVector %zu\n", offsetof(FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs, shiftVector));
    printf("sizeof_status %zu\n", sizeof(FFTLIB_STATUS));
    printf("FFTLIB_FLOAT32 %d\n", (int)FFTLIB_FLOAT32);
    printf("FFTLIB_INT16 %d\n", (int)FFTLIB_INT16);
    printf("FFTLIB_UINT32 %d\n", (int)FFTLIB_UINT32);
    printf("FFTLIB_ERR_NULL_POINTER %d\n", (int)FFTLIB_ERR_NULL_POINTER);
    printf("FFTLIB_ERR_NOT_IMPLEMENTED %d\n", (int)FFTLIB_ERR_NOT_IMPLEMENTED);
    printf("FFTLIB_FUNCTION_OPTIMIZED %d\n", (int)FFTLIB_FUNCTION_OPTIMIZED);
    printf("PBLOCK_C2C %d\n", (int)FFTLIB_FFT1DBATCHED_I32FC_C32FC_O32FC_PBLOCK_SIZE);
    printf("PBLOCK_I16 %d\n", (int)FFTLIB_FFT1DBATCHED_I16SC_C16SC_O16SC_PBLOCK_SIZE);
    return 0;
}

/* ---- checkParams coverage cases ----------------------------------------- */

typedef FFTLIB_STATUS (*check_fn)(FFTLIB_F32 *, FFTLIB_bufParams1D_t *, FFTLIB_F32 *, FFTLIB_bufParams1D_t *,
                                  FFTLIB_F32 *, FFTLIB_bufParams1D_t *, uint32_t, uint32_t, void *);
typedef FFTLIB_STATUS (*check_cn_fn)(FFTLIB_F32 *, FFTLIB_bufParams1D_t *, FFTLIB_F32 *, FFTLIB_bufParams1D_t *,
                                     FFTLIB_F32 *, FFTLIB_bufParams1D_t *, uint32_t, uint32_t);

static void coverage(const char *name, check_fn opt, check_cn_fn cn, void *pBlockMem)
{
    const uint32_t n0 = 64, ch0 = 4;
    for (int tc = 1000; tc <= 1011; ++tc) {
        uint32_t n = n0, ch = ch0;
        const uint32_t dim = ch * n * 2;
        FFTLIB_F32 *X = (FFTLIB_F32 *)xmalloc((dim + 4) * sizeof(FFTLIB_F32));
        FFTLIB_F32 *W = (FFTLIB_F32 *)xmalloc(2 * n * sizeof(FFTLIB_F32));
        FFTLIB_F32 *Y = (FFTLIB_F32 *)xmalloc(dim * sizeof(FFTLIB_F32));
        FFTLIB_bufParams1D_t bX = {FFTLIB_FLOAT32, dim}, bW = {FFTLIB_FLOAT32, 2 * n}, bY = {FFTLIB_FLOAT32, dim};
        FFTLIB_F32 *pX = X, *pW = W, *pY = Y;
        void *pBlock = pBlockMem;
        switch (tc) {
        case 1000: pX = NULL; break;
        case 1001: pW = NULL; break;
        case 1002: pY = NULL; break;
        case 1003: pBlock = NULL; break;
        case 1004: bY.dim_x = dim / 2; break;
        case 1005: bW.dim_x = n; break;
        case 1006: bX.data_type = FFTLIB_UINT32; break;
        case 1007: bW.data_type = FFTLIB_UINT32; break;
        case 1008: bY.data_type = FFTLIB_UINT32; break;
        case 1009: pX = X + 1; break; /* 4 bytes off a 16-byte boundary */
        case 1010:
        case 1011:
            n = tc == 1010 ? 7 : 30;
            ch = 1;
            bX.dim_x = bY.dim_x = ch * n * 2;
            bW.dim_x = 2 * n;
            break;
        }
        const FFTLIB_STATUS so = opt(pX, &bX, pW, &bW, pY, &bY, n, ch, pBlock);
        const FFTLIB_STATUS sc = cn(pX, &bX, pW, &bW, pY, &bY, n, ch);
        printf("%s %d %d %d\n", name, tc, (int)so, (int)sc);
        free(X);
        free(W);
        free(Y);
    }
}

static int checkparams(void)
{
    static uint8_t pb[FFTLIB_FFT1DBATCHED_I32FC_C32FC_O32FC_PBLOCK_SIZE];
    static uint8_t pbi[FFTLIB_IFFT1DBATCHED_I32FC_C32FC_O32FC_PBLOCK_SIZE];
    coverage("c2c", FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_checkParams, FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_checkParams_cn,
             pb);
    coverage("ifft", FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc_checkParams,
             FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc_checkParams_cn, pbi);
    return 0;
}

/* ---- transforms (GPU) --------------------------------------------------- */

static void run_c2c(const char *dir, int inverse, uint32_t n, uint32_t ch)
{
    static uint8_t pBlock[FFTLIB_FFT1DBATCHED_I32FC_C32FC_O32FC_PBLOCK_SIZE];
    const uint32_t dim = 2 * n * ch;
    FFTLIB_F32 *X = (FFTLIB_F32 *)xmalloc(dim * sizeof(FFTLIB_F32));
    FFTLIB_F32 *W = (FFTLIB_F32 *)xmalloc(2 * n * sizeof(FFTLIB_F32));
    FFTLIB_F32 *Y = (FFTLIB_F32 *)xmalloc(dim * sizeof(FFTLIB_F32));
    for (uint32_t i = 0; i < dim; ++i) X[i] = uniform_pm1();
    char name[64];
    snprintf(name, sizeof name, "%s_%u_%u_in.f32", inverse ? "ifft" : "c2c", n, ch);
    dump(dir, name, X, dim * sizeof(FFTLIB_F32)); /* before the call: pX may be clobbered */
    FFTLIB_b200_tw_gen_c2c(W, n);
    FFTLIB_bufParams1D_t bX = {FFTLIB_FLOAT32, dim}, bW = {FFTLIB_FLOAT32, 2 * n}, bY = {FFTLIB_FLOAT32, dim};
    if (inverse) {
        EXPECT_OK(FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc_checkParams(X, &bX, W, &bW, Y, &bY, n, ch, pBlock));
        EXPECT_OK(FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc_init(X, &bX, W, &bW, Y, &bY, n, ch, pBlock));
        EXPECT_OK(FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc_kernel(X, &bX, W, &bW, Y, &bY, n, ch, pBlock));
    } else {
        EXPECT_OK(FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_checkParams(X, &bX, W, &bW, Y, &bY, n, ch, pBlock));
        EXPECT_OK(FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_init(X, &bX, W, &bW, Y, &bY, n, ch, pBlock));
        EXPECT_OK(FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_kernel(X, &bX, W, &bW, Y, &bY, n, ch, pBlock));
    }
    snprintf(name, sizeof name, "%s_%u_%u_out.f32", inverse ? "ifft" : "c2c", n, ch);
    dump(dir, name, Y, dim * sizeof(FFTLIB_F32));
    free(X);
    free(W);
    free(Y);
}

static void run_r2c_c2r(const char *dir, uint32_t n, uint32_t ch)
{
    static uint8_t pbR[FFTLIB_FFT1DBATCHED_I32F_C32FC_O32FC_PBLOCK_SIZE];
    static uint8_t pbC[FFTLIB_IFFT1DBATCHED_I32FC_C32FC_O32F_PBLOCK_SIZE];
    const uint32_t nb = n / 2 + 1; /* outmode / inMode 0: n/2 + 1 bins */
    FFTLIB_F32 *X = (FFTLIB_F32 *)xmalloc(n * ch * sizeof(FFTLIB_F32));
    FFTLIB_F32 *W = (FFTLIB_F32 *)xmalloc(n * sizeof(FFTLIB_F32));
    FFTLIB_F32 *Sf = (FFTLIB_F32 *)xmalloc(2 * n * sizeof(FFTLIB_F32));
    FFTLIB_F32 *Xf = (FFTLIB_F32 *)xmalloc((n + 2) * 2 * ch * sizeof(FFTLIB_F32));
    FFTLIB_F32 *Y = (FFTLIB_F32 *)xmalloc(2 * nb * ch * sizeof(FFTLIB_F32));
    FFTLIB_F32 *Yc = (FFTLIB_F32 *)xmalloc(2 * nb * ch * sizeof(FFTLIB_F32));
    FFTLIB_F32 *Z = (FFTLIB_F32 *)xmalloc(n * ch * sizeof(FFTLIB_F32));
    for (uint32_t i = 0; i < n * ch; ++i) X[i] = uniform_pm1();
    dump(dir, "r2c_in.f32", X, n * ch * sizeof(FFTLIB_F32));
    FFTLIB_bufParams1D_t b = {FFTLIB_FLOAT32, n * ch};
    tw_gen_r2c(W, (int32_t)n);
    split_factor_gen_r2c(Sf, (int32_t)n);
    EXPECT_OK(FFTLIB_fft1dBatched_i32f_c32fc_o32fc_init(X, &b, W, &b, Xf, &b, Sf, &b, Y, &b, n, ch, 0, pbR));
    EXPECT_OK(FFTLIB_fft1dBatched_i32f_c32fc_o32fc_kernel(X, &b, W, &b, Xf, &b, Sf, &b, Y, &b, n, ch, 0, pbR));
    dump(dir, "r2c_out.f32", Y, 2 * nb * ch * sizeof(FFTLIB_F32));
    memcpy(Yc, Y, 2 * nb * ch * sizeof(FFTLIB_F32));
    ifft_c2r_tw_gen(W, (int32_t)n);
    ifft_c2r_split_factor_gen(Sf, (int32_t)n);
    EXPECT_OK(FFTLIB_ifft1dBatched_i32fc_c32fc_o32f_init(Yc, &b, W, &b, Xf, &b, Sf, &b, Z, &b, n, ch, 0, pbC));
    EXPECT_OK(FFTLIB_ifft1dBatched_i32fc_c32fc_o32f_kernel(Yc, &b, W, &b, Xf, &b, Sf, &b, Z, &b, n, ch, 0, pbC));
    dump(dir, "c2r_out.f32", Z, n * ch * sizeof(FFTLIB_F32));
    free(X);
    free(W);
    free(Sf);
    free(Xf);
    free(Y);
    free(Yc);
    free(Z);
}

static void run_i16(const char *dir, uint32_t n, uint32_t ch)
{
    static uint8_t pBlock[FFTLIB_FFT1DBATCHED_I16SC_C16SC_O16SC_PBLOCK_SIZE];
    const uint32_t dim = 2 * n * ch;
    int16_t *X = (int16_t *)xmalloc(dim * sizeof(int16_t));
    int16_t *W = (int16_t *)xmalloc(2 * n * sizeof(int16_t));
    int16_t *Y = (int16_t *)xmalloc(dim * sizeof(int16_t));
    uint32_t shift[5] = {2, 2, 2, 2, 2};
    for (uint32_t i = 0; i < dim; ++i) X[i] = (int16_t)((int32_t)(lcg_next() % 4096u) - 2048);
    dump(dir, "i16_in.i16", X, dim * sizeof(int16_t));
    FFTLIB_b200_tw_gen_i16(W, n);
    FFTLIB_bufParams1D_t bX = {FFTLIB_INT16, dim}, bW = {FFTLIB_INT16, 2 * n}, bS = {FFTLIB_UINT32, 5};
    EXPECT_OK(FFTLIB_fft1dBatched_i16sc_c16sc_o16sc_checkParams(X, &bX, W, &bW, Y, &bX, shift, &bS, n, ch, pBlock));
    EXPECT_OK(FFTLIB_fft1dBatched_i16sc_c16sc_o16sc_init(X, &bX, W, &bW, Y, &bX, shift, &bS, n, ch, pBlock));
    EXPECT_OK(FFTLIB_fft1dBatched_i16sc_c16sc_o16sc_kernel(X, &bX, W, &bW, Y, &bX, shift, &bS, n, ch, pBlock));
    dump(dir, "i16_out.i16", Y, dim * sizeof(int16_t));
    free(X);
    free(W);
    free(Y);
}

/* The DFT coordinator in the reference driver's order. */
static void run_mma(const char *dir, const char *tag, uint32_t dataType, uint32_t n, uint32_t batch, uint32_t shift0)
{
    FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs args;
    memset(&args, 0, sizeof args);
    args.funcStyle = FFTLIB_FUNCTION_OPTIMIZED;
    args.fftSize = n;
    args.batchSize = batch;
    args.interleave = 1;
    for (int k = 0; k < FFTLIB_FFT_FFT_IXX_CXX_OXX_NUMSHIFTS; ++k) args.shiftVector[k] = k ? 0 : shift0;
    const int32_t handleSize = FFTLIB_FFT_fft_ixX_cxX_oxX_getHandleSize(&args);
    FFTLIB_kernelHandle handle = xmalloc((size_t)handleSize);
    FFTLIB_bufParams1D_t bX = {dataType, 0}, bW = {dataType, 0}, bY = {dataType, 0};
    EXPECT_OK(FFTLIB_FFT_fft_ixX_cxX_oxX_getSizes(&args, &bX, &bW, &bY));
    const size_t es = (size_t)FFTLIB_sizeof(dataType);
    void *pX = xmalloc(bX.dim_x * es), *pW = xmalloc(bW.dim_x * es), *pY = xmalloc(bY.dim_x * es);
    for (uint32_t i = 0; i < bX.dim_x; ++i) {
        if (dataType == FFTLIB_FLOAT32) ((float *)pX)[i] = uniform_pm1();
        else ((int16_t *)pX)[i] = (int16_t)(lcg_next() & 0xFFFFu);
    }
    char name[64];
    snprintf(name, sizeof name, "mma_%s_in.bin", tag);
    dump(dir, name, pX, bX.dim_x * es);
    EXPECT_OK(FFTLIB_FFT_fft_ixX_cxX_oxX_twGen(&args, pW, &bW));
    EXPECT_OK(FFTLIB_FFT_fft_ixX_cxX_oxX_init_checkParams(handle, &bX, &bW, &bY, &args));
    EXPECT_OK(FFTLIB_FFT_fft_ixX_cxX_oxX_init(handle, &bX, &bW, &bY, &args));
    EXPECT_OK(FFTLIB_FFT_fft_ixX_cxX_oxX_exec_checkParams(handle, pX, pW, pY));
    EXPECT_OK(FFTLIB_FFT_fft_ixX_cxX_oxX_exec(handle, pX, pW, pY));
    printf("mma_%s path %d\n", tag, (int)FFTLIB_b200_FFT_fft_path(handle));
    snprintf(name, sizeof name, "mma_%s_out.bin", tag);
    dump(dir, name, pY, bY.dim_x * es);
    free(pX);
    free(pW);
    free(pY);
    free(handle);
}

static int run(const char *dir)
{
    run_c2c(dir, 0, 256, 16);   /* the reference's CPU configuration */
    run_c2c(dir, 0, 4096, 64);
    run_c2c(dir, 1, 960, 5);
    run_c2c(dir, 0, 31250, 2);  /* global passes, pX used as work buffer */
    run_r2c_c2r(dir, 4096, 8);
    run_i16(dir, 1024, 32);
    run_mma(dir, "f32_256", FFTLIB_FLOAT32, 256, 300, 0);
    run_mma(dir, "i16_32", FFTLIB_INT16, 32, 100, 12);
    printf("failures %d\n", failures);
    return failures ? 1 : 0;
}

int main(int argc, char **argv)
{
    if (argc >= 2 && !strcmp(argv[1], "layout")) return layout();
    if (argc >= 2 && !strcmp(argv[1], "checkparams")) return checkparams();
    if (argc >= 3 && !strcmp(argv[1], "run")) return run(argv[2]);
    fprintf(stderr, "usage: %s layout | checkparams | run DIR\n", argv[0]);
    return 2;
}
