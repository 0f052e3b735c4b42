// ffter.hpp -- unnormalised transforms of the drop-in API (reference
// include/transforms/ffter.hpp: CuFFTer :8-31, CuFFTerC2C :33-53,
// CuFFTerR2C :54-80, CuFFTerC2R :82-110) over psx_fft_plan_*.
#pragma once
#include <cufft.h>
#include "peasoup_b200.h"
#include "utils/exceptions.hpp"

class CuFFTer {
protected:
    psx_fft_plan* plan;
    unsigned int size;
    psx_stream_t stream;
    CuFFTer(unsigned int n, long long batch, int kind, psx_stream_t s)
        : plan(nullptr), size(n), stream(s)
    {
        ErrorChecker::check(psx_fft_plan_create(&plan, n, batch, kind), "CuFFTer");
    }

public:
    double get_resolution(float tsamp) { return 1.0 / (size * tsamp); }
    virtual unsigned int get_output_size() { return size / 2 + 1; }
    virtual ~CuFFTer()
    {
        if (plan) psx_fft_plan_destroy(plan);
    }
    CuFFTer(const CuFFTer&) = delete;
    CuFFTer& operator=(const CuFFTer&) = delete;
};

class CuFFTerC2C : public CuFFTer {
public:
    explicit CuFFTerC2C(unsigned int n, unsigned int batch = 1, psx_stream_t s = nullptr)
        : CuFFTer(n, batch, PSX_FFT_C2C, s)
    {
    }
    unsigned int get_output_size() override { return size; }
    // direction CUFFT_FORWARD or CUFFT_INVERSE, unnormalised, as cufftExecC2C
    void execute(cufftComplex* input, cufftComplex* output, int direction)
    {
        ErrorChecker::check(psx_fft_exec_c2c(plan, input, output, direction, stream),
                            "CuFFTerC2C::execute");
    }
};

class CuFFTerR2C : public CuFFTer {
public:
    explicit CuFFTerR2C(unsigned int n, long long batch = 1, psx_stream_t s = nullptr)
        : CuFFTer(n, batch, PSX_FFT_R2C, s)
    {
    }
    void execute(float* tim, cufftComplex* fseries)
    {
        ErrorChecker::check(psx_fft_exec(plan, tim, fseries, stream), "CuFFTerR2C::execute");
    }
};

class CuFFTerC2R : public CuFFTer {
public:
    explicit CuFFTerC2R(unsigned int n, long long batch = 1, psx_stream_t s = nullptr)
        : CuFFTer(n, batch, PSX_FFT_C2R, s)
    {
    }
    unsigned int get_output_size() override { return size; }
    void execute(cufftComplex* input, float* output)
    {
        ErrorChecker::check(psx_fft_exec(plan, input, output, stream), "CuFFTerC2R::execute");
    }
};
