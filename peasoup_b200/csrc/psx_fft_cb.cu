// psx_fft_cb.cu -- cuFFT load callback that performs the acceleration
// resample gather inside the batched R2C transform, so the resampled
// series is never written to memory.  Compiled to LTO IR and handed to
// cuFFT with cufftXtSetJITCallback (see psx_fft.cu).
//
// Element `offset` of a batched R2C input with distance N belongs to
// trial t = offset / N, sample i = offset - t*N; the callback returns the
// dereddened series at the resampleII read index of (i, k_t), the same
// index psx_resampleII computes (reference src/kernels.cu:321-324).
#include <cufftXt.h>
#include "psx_device.cuh"
#include "psx_fft_cb.h"

extern "C" __device__ cufftReal psx_resample_load(void* dataIn, unsigned long long offset,
                                                  void* callerInfo, void* sharedPointer)
{
    const psx_resample_cb_info* info = static_cast<const psx_resample_cb_info*>(callerInfo);
    const unsigned long long q = offset >> info->shift;
    const unsigned long long t = info->three ? (unsigned long long)((unsigned)q / 3u) : q;
    const unsigned long long i = offset - t * info->n;
    return psx::gather_at(info->series, psx::resampleII_index(i, info->ktab[t], info->size),
                          info->n);
}
