// psx_fft.cu -- cuFFT plans for the search: plain R2C/C2R plans (the
// drop-in CuFFTerR2C / CuFFTerC2R), batched R2C plans and the complex
// transforms of the batched trials.
#include <cufft.h>
#include <cufftXt.h>
#include <cuda_runtime.h>
#include <cstring>
#include "psx_common.cuh"
#include "psx_fft.cuh"

namespace psx {

const char* cufft_name(cufftResult r)
{
    switch (r) {
    case CUFFT_SUCCESS: return "CUFFT_SUCCESS";
    case CUFFT_INVALID_PLAN: return "CUFFT_INVALID_PLAN";
    case CUFFT_ALLOC_FAILED: return "CUFFT_ALLOC_FAILED";
    case CUFFT_INVALID_VALUE: return "CUFFT_INVALID_VALUE";
    case CUFFT_INTERNAL_ERROR: return "CUFFT_INTERNAL_ERROR";
    case CUFFT_EXEC_FAILED: return "CUFFT_EXEC_FAILED";
    case CUFFT_SETUP_FAILED: return "CUFFT_SETUP_FAILED";
    case CUFFT_INVALID_SIZE: return "CUFFT_INVALID_SIZE";
    case CUFFT_NOT_SUPPORTED: return "CUFFT_NOT_SUPPORTED";
    default: return "cuFFT error";
    }
}

static int fft_status(cufftResult r, const char* where)
{
    if (r == CUFFT_SUCCESS) return PSX_OK;
    set_error("%s: %s (%d)", where, cufft_name(r), (int)r);
    return PSX_ERR_CUFFT;
}

bool fft_size_supported(size_t n)
{
    if (n < 16 || (n & 1)) return false;
    size_t m = n;
    while ((m & 1) == 0) m >>= 1;
    return m == 1 || m == 3;
}

int FftPlan::create(size_t n_, long long batch_, int kind_, size_t in_dist, size_t out_dist)
{
    destroy();
    if (!fft_size_supported(n_) || batch_ < 1) {
        set_error("fft plan: unsupported size %zu (2^k or 3*2^k, >= 16) or batch %lld", n_, batch_);
        return PSX_ERR_INVALID;
    }
    n = n_;
    batch = batch_;
    kind = kind_;
    PSX_TRY(fft_status(cufftCreate(&h), "cufftCreate"));
    have = true;
    const size_t nb = n / 2 + 1;
    if (in_dist == 0) in_dist = kind == PSX_FFT_R2C ? n : kind == kFftC2C ? n : nb;
    if (out_dist == 0) out_dist = kind == PSX_FFT_R2C ? nb : n;
    long long dims[1] = {(long long)n};
    long long inembed[1] = {(long long)in_dist};
    long long onembed[1] = {(long long)out_dist};
    const cufftType type = kind == PSX_FFT_R2C ? CUFFT_R2C : kind == kFftC2C ? CUFFT_C2C : CUFFT_C2R;
    PSX_TRY(fft_status(cufftMakePlanMany64(h, 1, dims, inembed, 1, (long long)in_dist, onembed, 1,
                                           (long long)out_dist, type, batch, &work_bytes),
                       "cufftMakePlanMany64"));
    return PSX_OK;
}

void FftPlan::destroy()
{
    if (have) cufftDestroy(h);
    have = false;
}

int FftPlan::exec(const void* in, void* out, cudaStream_t s)
{
    if (!have) {
        set_error("fft plan not created");
        return PSX_ERR_INVALID;
    }
    PSX_TRY(fft_status(cufftSetStream(h, s), "cufftSetStream"));
    if (kind == PSX_FFT_R2C)
        return fft_status(cufftExecR2C(h, (cufftReal*)const_cast<void*>(in), (cufftComplex*)out),
                          "cufftExecR2C");
    if (kind == kFftC2C)
        return fft_status(cufftExecC2C(h, (cufftComplex*)const_cast<void*>(in), (cufftComplex*)out,
                                       CUFFT_FORWARD),
                          "cufftExecC2C");
    return fft_status(cufftExecC2R(h, (cufftComplex*)const_cast<void*>(in), (cufftReal*)out),
                      "cufftExecC2R");
}

int FftPlan::exec_c2c(const void* in, void* out, int direction, cudaStream_t s)
{
    if (!have || kind != kFftC2C) {
        set_error("fft exec_c2c: not a complex plan");
        return PSX_ERR_INVALID;
    }
    if (direction != CUFFT_FORWARD && direction != CUFFT_INVERSE) {
        set_error("fft exec_c2c: direction must be -1 (forward) or +1 (inverse)");
        return PSX_ERR_INVALID;
    }
    PSX_TRY(fft_status(cufftSetStream(h, s), "cufftSetStream"));
    return fft_status(cufftExecC2C(h, (cufftComplex*)const_cast<void*>(in), (cufftComplex*)out,
                                   direction),
                      "cufftExecC2C");
}

}  // namespace psx

struct psx_fft_plan {
    psx::FftPlan p;
};

extern "C" {

int psx_fft_plan_create(psx_fft_plan** plan, size_t size, long long batch, int kind)
{
    psx::clear_error();
    if (!plan || (kind != PSX_FFT_R2C && kind != PSX_FFT_C2R && kind != PSX_FFT_C2C)) {
        psx::set_error("fft_plan_create: bad arguments");
        return PSX_ERR_INVALID;
    }
    *plan = nullptr;
    psx_fft_plan* p = new (std::nothrow) psx_fft_plan;
    if (!p) return PSX_ERR_ALLOC;
    int rc = kind == PSX_FFT_C2C ? p->p.create(size, batch, psx::kFftC2C, size, size)
                                 : p->p.create(size, batch, kind, 0, 0);
    if (rc != PSX_OK) {
        delete p;
        return rc;
    }
    *plan = p;
    return PSX_OK;
}

int psx_fft_exec(psx_fft_plan* plan, const void* d_in, void* d_out, psx_stream_t stream)
{
    psx::clear_error();
    if (!plan || !d_in || !d_out) {
        psx::set_error("fft_exec: bad arguments");
        return PSX_ERR_INVALID;
    }
    if (plan->p.kind == psx::kFftC2C) {
        psx::set_error("fft_exec: a complex plan needs psx_fft_exec_c2c (a direction)");
        return PSX_ERR_INVALID;
    }
    return plan->p.exec(d_in, d_out, psx::cs(stream));
}

int psx_fft_exec_c2c(psx_fft_plan* plan, const void* d_in, void* d_out, int direction,
                     psx_stream_t stream)
{
    psx::clear_error();
    if (!plan || !d_in || !d_out) {
        psx::set_error("fft_exec_c2c: bad arguments");
        return PSX_ERR_INVALID;
    }
    return plan->p.exec_c2c(d_in, d_out, direction, psx::cs(stream));
}

int psx_fft_plan_destroy(psx_fft_plan* plan)
{
    psx::clear_error();
    delete plan;
    return PSX_OK;
}

}  // extern "C"
