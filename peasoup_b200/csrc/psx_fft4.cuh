// psx_fft4.cuh -- the batched search's own forward transform: for each
// acceleration trial, the complex DFT of length M = N/2 of the resampled
// series read as interleaved pairs, z[m] = x'[2m] + i x'[2m+1], in two
// passes over HBM (four-step split M = R * C, R = 1024 or 768), with the
// resample gather done by the first pass's loads; and the unpack +
// interbin + normalise pass that reads its transposed output.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>

namespace psx {


struct Fft4Plan {
    size_t n = 0;      // real samples N
    unsigned R = 1024; // rows of the four-step split: 768 for 3 * 2^k, 1024
                       // up to N = 2^25, 2048 at 2^26, 4096 at 2^27
    unsigned C = 0;    // row length of the second pass (M / R)
    int logc = 0;
    float2* d_tab = nullptr;  // twiddle tables (offsets below, in float2)
    size_t tab_len = 0;
    unsigned offA2 = 0, offA3 = 0, offQ = 0, offP = 0, offB = 0, offRv = 0, offRk = 0;

    // N = 2^19 .. 2^27 (R = 1024, 2048, 4096) or 3 * 2^17 .. 3 * 2^23
    // (R = 768), i.e. C = 2^8 .. 2^14.
    static bool supported(size_t n);
    static unsigned rows_for(size_t n);
    // float2 entries of the twiddle tables of a plan for n
    static size_t table_floats2(size_t n);
    int create(size_t n);
    void destroy();
    ~Fft4Plan() { destroy(); }

    // ntrials transforms: trial t gathers series[resampleII index of
    // ktab[t]] (the resampleII read index in FP64, as the resample kernel
    // forms it) and leaves Z = DFT_M(z) transposed:
    //   zt[t * zpitch + k1 * C + k2] = Z[k1 + R * k2].
    // y (ypitch complex elements per trial, >= M) holds the intermediate.
    int exec(const float* series, const double* ktab, int ntrials, float2* y, size_t ypitch,
             float2* zt, size_t zpitch, cudaStream_t s) const;
    // The two passes of exec on their own (pass 1: gather + column
    // transforms into y; pass 2: row transforms of y into zt).
    // trow (optional): trial t gathers series + trow[t] * xpitch instead
    // (trials of several series in one launch)
    int exec_cols(const float* series, const double* ktab, int ntrials, float2* y,
                  size_t ypitch, cudaStream_t s, const unsigned* trow = nullptr,
                  size_t xpitch = 0) const;
    int exec_rows(const float2* y, size_t ypitch, int ntrials, float2* zt, size_t zpitch,
                  cudaStream_t s) const;
    // The N samples pass 1 gathers for one trial (ktab[0]), written to out
    // in series order instead of being transformed (the debug tap).
    int dump_gather(const float* series, const double* ktab, float* out, cudaStream_t s) const;

    // Real spectrum bins 0..M of each trial from zt, interbinned and
    // normalised with stat[3] (mean*N) and stat[4] (std*N), written at
    // p + t * ppitch.
    // trow (optional): trial t's statistics at stat + 8 * trow[t]
    int form(const float2* zt, size_t zpitch, int ntrials, float* p, size_t ppitch,
             const float* stat, cudaStream_t s, const unsigned* trow = nullptr) const;

private:
    template <int R, bool DUMP>
    static void launch_cols(const Fft4Plan& f, const float* series, const double* ktab,
                            int ntrials, float2* y, size_t ypitch, cudaStream_t s,
                            const unsigned* trow, size_t xpitch);
};

}  // namespace psx
