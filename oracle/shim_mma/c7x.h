/* Host stand-in for the TI C7000 compiler's <c7x.h>, for compiling the
 * reference's natural-C (_cn) DFT-coordinator and LINALG sources with g++.
 * They include it through src/common/FFTLIB_types.h and use from it only
 * the arithmetic shift helpers below; the rest are opaque names that
 * declarations of the optimized kernels mention. Test infrastructure. */
#ifndef ORACLE_SHIM_MMA_C7X_H
#define ORACLE_SHIM_MMA_C7X_H

#include <stdint.h>

#ifndef SE_PARAM_SIZE
#define SE_PARAM_SIZE 64
#endif
#ifndef SA_PARAM_SIZE
#define SA_PARAM_SIZE 64
#endif

namespace c7x {
struct uchar_vec { uint8_t v[64]; };
struct ushort_vec { uint16_t v[32]; };
} // namespace c7x

struct __HWA_CONFIG_REG_v1 { uint8_t v[64]; };
struct __HWA_OFFSET_REG { uint8_t v[64]; };
struct __SE_TEMPLATE_v1 { uint8_t v[64]; };
struct __SA_TEMPLATE_v1 { uint8_t v[64]; };
struct uchar64 { uint8_t v[64]; };

/* arithmetic (signed) and logical (unsigned) shifts */
static inline int32_t __shift_right(int32_t a, uint32_t s) { return a >> s; }
static inline int64_t __shift_right(int64_t a, uint32_t s) { return a >> s; }
static inline uint32_t __shift_right(uint32_t a, uint32_t s) { return a >> s; }
static inline uint64_t __shift_right(uint64_t a, uint32_t s) { return a >> s; }
static inline int32_t __shift_left(int32_t a, uint32_t s) { return (int32_t)((uint32_t)a << s); }
static inline int64_t __shift_left(int64_t a, uint32_t s) { return (int64_t)((uint64_t)a << s); }
static inline uint32_t __shift_left(uint32_t a, uint32_t s) { return a << s; }
static inline uint64_t __shift_left(uint64_t a, uint32_t s) { return a << s; }

#endif
