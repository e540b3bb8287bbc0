/*
 * FFTLIB_types.h -- ABI types of the FFTLIB C API, for libfftlib_b200.so.
 *
 * Names and numeric values are those of the reference library so existing
 * FFTLIB callers compile and link unchanged:
 *   status codes          src/common/FFTLIB_types.h:168-211
 *   FFTLIB_F32 / _D64     src/common/FFTLIB_types.h:164-165
 *   kernel handle         src/common/FFTLIB_types.h:213
 *   function style        src/common/FFTLIB_types.h:216-221
 *   data types            src/common/FFTLIB_bufParams.h:22-42
 *   1-D buffer params     src/common/FFTLIB_bufParams.h:62-67
 *   FFTLIB_sizeof         src/common/FFTLIB_bufParams.h:121
 * Nothing here depends on CUDA.
 */
#ifndef FFTLIB_B200_TYPES_H_
#define FFTLIB_B200_TYPES_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double FFTLIB_D64;
typedef float  FFTLIB_F32;

typedef enum {
   FFTLIB_SUCCESS                      = 0,
   FFTLIB_ERR_FAILURE                  = 1,
   FFTLIB_ERR_INVALID_VALUE            = 2,
   FFTLIB_ERR_INVALID_TYPE             = 3,
   FFTLIB_ERR_INVALID_DIMENSION        = 4,
   FFTLIB_ERR_NULL_POINTER             = 5,
   FFTLIB_ERR_NOT_IMPLEMENTED          = 6,
   FFTLIB_ERR_NOT_EQUAL_WIDTH_STRIDE   = 7,
   FFTLIB_ERR_NOT_ALIGNED_PTRS_STRIDES = 8,
   FFTLIB_ERR_NOT_ALIGNED_WIDTHS       = 9,
   FFTLIB_ERR_BUFFER_TOO_SMALL         = 10,
   FFTLIB_ERR_INVALID_ACTIVATION       = 11,
   FFTLIB_ERR_INVALID_SHIFT            = 12,
   FFTLIB_ERROR_MAX                    = 13,
   FFTLIB_ERR_INVALID_OUTMODE          = 14,
   FFTLIB_ERR_MATRIX_MATRIX_MULTIPLY_UNSUPPORTED_INPUT_TYPE                  = 10000,
   FFTLIB_ERR_MATRIX_MATRIX_MULTIPLY_UNSUPPORTED_OUTPUT_TYPE                 = 10001,
   FFTLIB_ERR_MATRIX_MATRIX_MULTIPLY_UNSUPPORTED_TYPE_COMBINATION            = 10002,
   FFTLIB_ERR_MATRIX_MATRIX_MULTIPLY_ACCUMULATE_UNSUPPORTED_INPUT_TYPE       = 11000,
   FFTLIB_ERR_MATRIX_MATRIX_MULTIPLY_ACCUMULATE_UNSUPPORTED_OUTPUT_TYPE      = 11001,
   FFTLIB_ERR_MATRIX_MATRIX_MULTIPLY_ACCUMULATE_UNSUPPORTED_TYPE_COMBINATION = 11002,
   FFTLIB_ERR_MATRIX_TRANSPOSE_UNSUPPORTED_INPUT_TYPE                        = 12000,
   FFTLIB_ERR_MATRIX_TRANSPOSE_UNSUPPORTED_OUTPUT_TYPE                       = 12001,
   FFTLIB_ERR_MATRIX_TRANSPOSE_UNSUPPORTED_TYPE_COMBINATION                  = 12002,
   FFTLIB_ERR_POINTWISE_MATRIX_MATRIX_MULTIPLY_UNSUPPORTED_INPUT_TYPE        = 13000,
   FFTLIB_ERR_POINTWISE_MATRIX_MATRIX_MULTIPLY_UNSUPPORTED_OUTPUT_TYPE       = 13001,
   FFTLIB_ERR_POINTWISE_MATRIX_MATRIX_MULTIPLY_UNSUPPORTED_TYPE_COMBINATION  = 13002
} FFTLIB_STATUS_NAME;

typedef FFTLIB_STATUS_NAME FFTLIB_STATUS;

typedef void *FFTLIB_kernelHandle;

typedef enum {
   FFTLIB_FUNCTION_NATC = 0,
   FFTLIB_FUNCTION_OPTIMIZED,
   FFTLIB_FUNCTION_MAX = 128
} FFTLIB_FUNCTION_STYLE;

typedef enum _FFTLIB_data_type_e {
   FFTLIB_INT8    = 0,
   FFTLIB_INT16   = 1,
   FFTLIB_INT32   = 2,
   FFTLIB_INT64   = 3,
   FFTLIB_INT128  = 4,
   FFTLIB_UINT8   = 5,
   FFTLIB_UINT16  = 6,
   FFTLIB_UINT24  = 7,
   FFTLIB_UINT32  = 8,
   FFTLIB_UINT64  = 9,
   FFTLIB_UINT128 = 10,
   FFTLIB_FLOAT16 = 11,
   FFTLIB_FLOAT32 = 12,
   FFTLIB_FLOAT64 = 13
} FFTLIB_data_type_e;

typedef struct {
   uint32_t data_type; /* FFTLIB_data_type_e */
   uint32_t dim_x;     /* width in elements */
} FFTLIB_bufParams1D_t;

/* reference: src/common/FFTLIB_bufParams.h:69-78 */
typedef struct {
   uint32_t data_type; /* FFTLIB_data_type_e */
   uint32_t dim_x;     /* width in elements */
   uint32_t dim_y;     /* height in elements */
   int32_t stride_y;   /* row stride in bytes */
} FFTLIB_bufParams2D_t;

/* Bytes per element of a FFTLIB_data_type_e value. */
static inline int32_t FFTLIB_sizeof(uint32_t type)
{
   switch (type) {
   case FFTLIB_INT8: case FFTLIB_UINT8: return 1;
   case FFTLIB_INT16: case FFTLIB_UINT16: case FFTLIB_FLOAT16: return 2;
   case FFTLIB_UINT24: return 3;
   case FFTLIB_INT32: case FFTLIB_UINT32: case FFTLIB_FLOAT32: return 4;
   case FFTLIB_INT64: case FFTLIB_UINT64: case FFTLIB_FLOAT64: return 8;
   case FFTLIB_INT128: case FFTLIB_UINT128: return 16;
   default: return 1;
   }
}

/* The reference sizes its pBlock buffers in units of the C7x streaming-engine
 * parameter block (SE_PARAM_SIZE, 64 bytes on C7x, defined by the TI
 * compiler's c7x.h). libfftlib_b200 keeps the same macro so that the
 * *_PBLOCK_SIZE expressions are unchanged; its plan record needs 64 bytes. */
#ifndef SE_PARAM_SIZE
#define SE_PARAM_SIZE 64
#endif

#ifdef __cplusplus
}
#endif

#endif /* FFTLIB_B200_TYPES_H_ */
