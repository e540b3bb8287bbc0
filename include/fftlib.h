/*
 * fftlib.h -- umbrella header of libfftlib_b200.so, in place of the
 * reference's src/fftlib.h.
 */
#ifndef FFTLIB_B200_FFTLIB_H_
#define FFTLIB_B200_FFTLIB_H_

#include "fftlib_b200/FFTLIB_types.h"
#include "fftlib_b200/fft_c7x.h"
#include "fftlib_b200/fft1d_c7x.h"
#include "fftlib_b200/fft_c7xmma.h"
#include "fftlib_b200/fft_c7xmma_variants.h"
#include "fftlib_b200/linalg_c7xmma.h"
#include "fftlib_b200/fftlib_b200_ext.h"

#endif
