// psx_search.cu -- the per-DM acceleration search engine behind
// psx_search_dm / psx_search_block: the body of the reference's DM loop
// (src/pipeline_multi.cu:161-294) re-organised for a B200.
//
// Per DM (prologue, once, no host round trip):
//   copy in -> baseline removal (device-side do/while, up to four passes
//   before the host takes over) -> zero padding -> R2C -> amplitude ->
//   5/25/125-bin running median fused with the division of the spectrum ->
//   birdie zapping -> interbin statistics (device-resident mean*N, std*N)
//   -> C2R into the resident dereddened series.
// Per acceleration trial (the hot loop), in launch groups of `batch`:
//   resample gather -> R2C (one batched cuFFT; by default the library's
//   two-pass transform with the gather in its first pass) -> k_form_norm
//   (interbin + normalise in one pass) -> k_harm_tiles (fractional harmonic
//   sums + threshold + warp-aggregated compaction of every (trial, fold,
//   bin, S/N) above threshold).  The trial schedule of a DM can be captured
//   as one CUDA graph.  Nothing per trial goes to the host: the records of
//   a DM come back in one copy, and the host clusters them
//   (peakfinder.hpp:72-94), forms frequencies and distils them
//   (distiller.hpp) while the GPU already runs the next DM (two record
//   slots, psx_search_block).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <vector>
#include "psx_common.cuh"
#include "psx_device.cuh"
#include "psx_fft.cuh"
#include "psx_fft4.cuh"
#include "psx_harm.cuh"
#include "psx_host.h"
#include "psx_stages.cuh"

namespace psx {

// Host threads that cluster and distil one DM's records trial by trial.
// run(fn) calls fn on every worker and on the calling thread and returns
// when all have returned; fn pulls its own work items.  Each worker takes
// part in every run: the next run starts only after all of the previous
// one's calls have returned.
class WorkPool {
public:
    explicit WorkPool(int workers)
    {
        for (int i = 0; i < workers; ++i) th_.emplace_back([this] { loop(); });
    }
    ~WorkPool()
    {
        {
            std::lock_guard<std::mutex> g(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : th_) t.join();
    }
    void run(const std::function<void()>& fn)
    {
        {
            std::lock_guard<std::mutex> g(m_);
            fn_ = &fn;
            pending_ = (int)th_.size();
            ++gen_;
        }
        cv_.notify_all();
        fn();
        std::unique_lock<std::mutex> g(m_);
        done_.wait(g, [this] { return pending_ == 0; });
        fn_ = nullptr;
    }

private:
    void loop()
    {
        int seen = 0;
        for (;;) {
            const std::function<void()>* f;
            {
                std::unique_lock<std::mutex> g(m_);
                cv_.wait(g, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
                f = fn_;
            }
            (*f)();
            std::lock_guard<std::mutex> g(m_);
            if (--pending_ == 0) done_.notify_one();
        }
    }
    std::vector<std::thread> th_;
    std::mutex m_;
    std::condition_variable cv_, done_;
    const std::function<void()>* fn_ = nullptr;
    int pending_ = 0, gen_ = 0;
    bool stop_ = false;
};

// ------------------------------------------------------------ kernels
// Interbinned amplitude normalised with the DM's statistics
// (reference src/kernels.cu:238-259 then :496-507), for `rows` spectra.
// Two bins per thread from one 128-bit load; the previous bin of the
// pair's first element is a cached scalar load.
__global__ void __launch_bounds__(256) k_form_norm(const float* __restrict__ X, size_t xpitch,
                                                   float* __restrict__ p, size_t ppitch,
                                                   unsigned nbins, const float* __restrict__ stat)
{
    const float meanN = stat[3], stdN = stat[4];
    const float* x = X + (size_t)blockIdx.y * xpitch;
    float* o = p + (size_t)blockIdx.y * ppitch;
    const unsigned npairs = nbins / 2;
    const unsigned stride = gridDim.x * blockDim.x;
    for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < npairs; q += stride) {
        const float4 v = reinterpret_cast<const float4*>(x)[q];
        float rl = 0.f, il = 0.f;
        if (q > 0) {
            rl = x[4 * q - 2];
            il = x[4 * q - 1];
        }
        float2 r;
        r.x = normalise(interbin(v.x, v.y, rl, il), meanN, stdN);
        r.y = normalise(interbin(v.z, v.w, v.x, v.y), meanN, stdN);
        reinterpret_cast<float2*>(o)[q] = r;
    }
    if ((nbins & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        const unsigned k = nbins - 1;
        const float rl = k ? x[2 * k - 2] : 0.f, il = k ? x[2 * k - 1] : 0.f;
        o[k] = normalise(interbin(x[2 * k], x[2 * k + 1], rl, il), meanN, stdN);
    }
}

// The real spectrum of a length-N series from the complex transform Z of
// length M = N/2 of z[n] = x[2n] + i x[2n+1] (the series read as interleaved
// pairs), unpacked, interbinned and normalised in one pass: for j and M - j
//   X[j]   = ((ar + u) + i (ai - v)) / 2,  X[M-j] = ((ar - u) + i (-ai - v)) / 2
// with Z[j] = (zr, zi), Z[M-j] = (wr, wi), ar = zr + wr, ai = zi - wi,
// br = zr - wr, bi = zi + wi, u = c bi - s br, v = s bi + c br and
// (c, s) = (cos, sin)(pi j / M).  It is the step cuFFT's R2C runs after its
// complex passes, merged with the interbinning and normalisation of the
// reference (src/kernels.cu:238-259, :496-507) that come next.  Each thread
// takes the four bins k0..k0+3 (k0 = 4q) and their mirrors M-k0-3..M-k0;
// the previous bin each interbin value needs is one more unpacked pair.
// M is a multiple of 8; thread 0 also forms bin M/2.
__device__ __forceinline__ void unpack_pair(const float2* __restrict__ z, unsigned M, unsigned j,
                                            float inv_m, float2& lo, float2& hi)
{
    const float2 a = z[j], w = z[j ? M - j : 0];
    const float ar = a.x + w.x, ai = a.y - w.y, br = a.x - w.x, bi = a.y + w.y;
    float sn, cs;
    sincospif((float)j * inv_m, &sn, &cs);
    const float u = cs * bi - sn * br, v = sn * bi + cs * br;
    lo = make_float2(0.5f * (ar + u), 0.5f * (ai - v));
    hi = make_float2(0.5f * (ar - u), 0.5f * (-ai - v));
}

// (cos, sin)(pi d / M) for d = -1 .. 4, rounded once from double: the
// twiddles of a thread's six pairs are W(k0) times these.
struct TwSteps {
    float2 w[6];
};

__global__ void __launch_bounds__(256) k_unpack_form_norm(const float* __restrict__ Zf, size_t zpitch,
                                                          float* __restrict__ p, size_t ppitch,
                                                          unsigned M, float inv_m, TwSteps steps,
                                                          const float* __restrict__ stat)
{
    const float meanN = stat[3], stdN = stat[4];
    const float2* z = reinterpret_cast<const float2*>(Zf) + (size_t)blockIdx.y * zpitch;
    float* o = p + (size_t)blockIdx.y * ppitch;
    const unsigned Q = M / 8;
    const unsigned stride = gridDim.x * blockDim.x;
    for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < Q; q += stride) {
        const unsigned k0 = 4 * q;
        // Z[k0-1+t] and Z[(M-(k0-1+t)) mod M], t = 0..5: the four interior
        // pairs of each side with two 128-bit loads (k0 and M-k0-4 are even)
        float2 zl[6], zh[6];
        const float4* z4 = reinterpret_cast<const float4*>(z);
        const float4 l0 = z4[k0 / 2], l1 = z4[k0 / 2 + 1];
        const float4 h0 = z4[(M - k0 - 4) / 2], h1 = z4[(M - k0 - 4) / 2 + 1];
        zl[1] = make_float2(l0.x, l0.y);
        zl[2] = make_float2(l0.z, l0.w);
        zl[3] = make_float2(l1.x, l1.y);
        zl[4] = make_float2(l1.z, l1.w);
        zl[5] = z[k0 + 4];
        zh[5] = make_float2(h0.x, h0.y);  // Z[M-k0-4]
        zh[4] = make_float2(h0.z, h0.w);  // Z[M-k0-3]
        zh[3] = make_float2(h1.x, h1.y);  // Z[M-k0-2]
        zh[2] = make_float2(h1.z, h1.w);  // Z[M-k0-1]
        if (k0 == 0) {
            zl[0] = zh[0] = make_float2(0.f, 0.f);
            zh[1] = zl[1];  // j = 0 is its own mirror
        } else {
            zl[0] = z[k0 - 1];
            zh[0] = z[M - k0 + 1];
            zh[1] = z[M - k0];
        }
        float2 lo[6], hi[6];  // X[k0-1+t], X[M-(k0-1+t)]
        float s0, c0;
        sincospif((float)k0 * inv_m, &s0, &c0);  // one call per thread
#pragma unroll
        for (int t = 0; t < 6; ++t) {
            const float2 a = zl[t], w = zh[t];
            const float ar = a.x + w.x, ai = a.y - w.y, br = a.x - w.x, bi = a.y + w.y;
            const float2 d = steps.w[t];  // angle of pair k0-1+t = angle(k0) + angle(t-1)
            const float cs = c0 * d.x - s0 * d.y, sn = s0 * d.x + c0 * d.y;
            const float u = cs * bi - sn * br, v = sn * bi + cs * br;
            lo[t] = make_float2(0.5f * (ar + u), 0.5f * (ai - v));
            hi[t] = make_float2(0.5f * (ar - u), 0.5f * (-ai - v));
        }
        if (k0 == 0) lo[0] = make_float2(0.f, 0.f);  // X[-1] := 0; hi[0] is not used
        float4 r;
        r.x = normalise(interbin(lo[1].x, lo[1].y, lo[0].x, lo[0].y), meanN, stdN);
        r.y = normalise(interbin(lo[2].x, lo[2].y, lo[1].x, lo[1].y), meanN, stdN);
        r.z = normalise(interbin(lo[3].x, lo[3].y, lo[2].x, lo[2].y), meanN, stdN);
        r.w = normalise(interbin(lo[4].x, lo[4].y, lo[3].x, lo[3].y), meanN, stdN);
        reinterpret_cast<float4*>(o)[q] = r;
        // bins M - k0 - t use X[M - k0 - t] (hi[t+1]) and X[M - k0 - t - 1] (hi[t+2])
#pragma unroll
        for (int t = 0; t < 4; ++t)
            o[M - k0 - t] = normalise(interbin(hi[t + 1].x, hi[t + 1].y, hi[t + 2].x, hi[t + 2].y),
                                      meanN, stdN);
        if (q == 0) {  // bin M/2 (its own mirror) with bin M/2 - 1
            float2 a, b, c, d;
            unpack_pair(z, M, M / 2, inv_m, a, b);
            unpack_pair(z, M, M / 2 - 1, inv_m, c, d);
            o[M / 2] = normalise(interbin(a.x, a.y, c.x, c.y), meanN, stdN);
        }
    }
}

// Fused harmonic sums + threshold + compaction: tile shapes and launcher.
// Persistent grid of MINB CTAs per SM, each one producer warp plus NC
// consumer threads and kHarmStages shared stages of a T-bin tile and its
// fractional windows.  The shapes below are the autotuner's choices
// (psx_search_config::harm_shape); shape 4 is the default.  Shapes 6 and 7
// stage every window for 3 or 2 trials at once with 2D tensor copies
// (k_harm_rows, one CTA per SM, NC consumers per trial).
constexpr int kHarmStages = 2;

struct HarmShape {
    int T, NC, minb;
    bool ool;  // exact pass out of line
    int rows;  // trials per item (multi-row kernel), 0 for k_harm_tiles
};
constexpr HarmShape kHarmShapes[] = {
    {512, 128, 3, true, 0},   // 1
    {512, 256, 3, true, 0},   // 2
    {256, 128, 6, true, 0},   // 3
    {512, 256, 3, false, 0},  // 4
    {256, 128, 6, false, 0},  // 5
    {512, 128, 1, true, 3},   // 6
    {512, 128, 1, true, 2},   // 7
};
static_assert(sizeof(kHarmShapes) / sizeof(kHarmShapes[0]) == PSX_HARM_SHAPES, "shape table");
constexpr int kHarmDefaultShape = 4;

template <int F, int SH>
struct HarmKernel {
    static constexpr HarmShape S = kHarmShapes[SH];
    static constexpr size_t smem_bytes()
    {
        return (size_t)kHarmStages * sizeof(float) * harm_smem_floats(F, S.T);
    }
    static int configure()
    {
        return cuda_status(cudaFuncSetAttribute(k_harm_tiles<F, S.T, S.NC, S.minb, S.ool>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)smem_bytes()),
                           "harmonic-sum kernel attribute");
    }
    static int launch(const float* p, size_t ppitch, unsigned row_len, const PeakParams& pp,
                      int trial0, int rows, int4* rec, unsigned* counter, unsigned cap,
                      cudaStream_t s)
    {
        const unsigned ntiles = (pp.hi - pp.lo + S.T - 1) / S.T;
        const unsigned items = ntiles * (unsigned)rows;
        const unsigned grid = std::min(items, (unsigned)(sm_count() * S.minb));
        k_harm_tiles<F, S.T, S.NC, S.minb, S.ool><<<grid, S.NC + 32, smem_bytes(), s>>>(
            p, ppitch, row_len, pp, trial0, rows, ntiles, rec, counter, cap);
        return launch_status("harmonic-sum kernel");
    }
};

// The multi-row kernel (shapes 6 and 7): ROWS trials per item.
template <int F, int SH>
struct HarmRowsKernel {
    static constexpr HarmShape S = kHarmShapes[SH];
    static constexpr size_t smem_bytes()
    {
        return (size_t)kHarmStages * sizeof(float) * rows_stage_floats(F, S.T, S.rows);
    }
    static int configure()
    {
        return cuda_status(cudaFuncSetAttribute(k_harm_rows<F, S.T, S.NC, S.rows>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)smem_bytes()),
                           "harmonic-sum kernel attribute");
    }
    static int launch(const HarmMaps* maps, const PeakParams& pp, int trial0, int rows, int4* rec,
                      unsigned* counter, unsigned cap, cudaStream_t s)
    {
        if (!maps) {
            set_error("harmonic-sum kernel: shape %d needs the instance's tensor maps", SH + 1);
            return PSX_ERR_INVALID;
        }
        const unsigned ntiles = (pp.hi - pp.lo + S.T - 1) / S.T;
        const unsigned items = ntiles * (((unsigned)rows + S.rows - 1) / S.rows);
        const unsigned grid = std::min(items, (unsigned)sm_count());
        k_harm_rows<F, S.T, S.NC, S.rows><<<grid, S.rows * S.NC + 32, smem_bytes(), s>>>(
            *maps, pp, trial0, rows, ntiles, rec, counter, cap);
        return launch_status("harmonic-sum kernel");
    }
};

template <int F>
static int configure_harm_f()
{
    int rc = PSX_OK;
    if (rc == PSX_OK) rc = HarmRowsKernel<F, 5>::configure();
    if (rc == PSX_OK) rc = HarmRowsKernel<F, 6>::configure();
    if (rc == PSX_OK) rc = HarmKernel<F, 0>::configure();
    if (rc == PSX_OK) rc = HarmKernel<F, 1>::configure();
    if (rc == PSX_OK) rc = HarmKernel<F, 2>::configure();
    if (rc == PSX_OK) rc = HarmKernel<F, 3>::configure();
    if (rc == PSX_OK) rc = HarmKernel<F, 4>::configure();
    return rc;
}

// Opts every shape of the kernel for F folds into its dynamic shared
// memory (once per device, before any launch or capture).
static int configure_harm(int F)
{
    switch (F) {
    case 0: return configure_harm_f<0>();
    case 1: return configure_harm_f<1>();
    case 2: return configure_harm_f<2>();
    case 3: return configure_harm_f<3>();
    case 4: return configure_harm_f<4>();
    default: return configure_harm_f<5>();
    }
}

template <int F>
static int launch_harm_f(int shape, const float* p, size_t ppitch, unsigned row_len,
                         const PeakParams& pp, int trial0, int rows, int4* rec, unsigned* counter,
                         unsigned cap, cudaStream_t s, const HarmMaps* maps)
{
    switch (shape) {
    case 6: return HarmRowsKernel<F, 5>::launch(maps, pp, trial0, rows, rec, counter, cap, s);
    case 7: return HarmRowsKernel<F, 6>::launch(maps, pp, trial0, rows, rec, counter, cap, s);
    case 2: return HarmKernel<F, 1>::launch(p, ppitch, row_len, pp, trial0, rows, rec, counter, cap, s);
    case 3: return HarmKernel<F, 2>::launch(p, ppitch, row_len, pp, trial0, rows, rec, counter, cap, s);
    case 4: return HarmKernel<F, 3>::launch(p, ppitch, row_len, pp, trial0, rows, rec, counter, cap, s);
    case 5: return HarmKernel<F, 4>::launch(p, ppitch, row_len, pp, trial0, rows, rec, counter, cap, s);
    default: return HarmKernel<F, 0>::launch(p, ppitch, row_len, pp, trial0, rows, rec, counter, cap, s);
    }
}

static int launch_harm(int F, int shape, const float* p, size_t ppitch, unsigned row_len,
                       const PeakParams& pp, int trial0, int rows, int4* rec, unsigned* counter,
                       unsigned cap, cudaStream_t s, const HarmMaps* maps = nullptr)
{
    switch (F) {
    case 0: return launch_harm_f<0>(shape, p, ppitch, row_len, pp, trial0, rows, rec, counter, cap, s, maps);
    case 1: return launch_harm_f<1>(shape, p, ppitch, row_len, pp, trial0, rows, rec, counter, cap, s, maps);
    case 2: return launch_harm_f<2>(shape, p, ppitch, row_len, pp, trial0, rows, rec, counter, cap, s, maps);
    case 3: return launch_harm_f<3>(shape, p, ppitch, row_len, pp, trial0, rows, rec, counter, cap, s, maps);
    case 4: return launch_harm_f<4>(shape, p, ppitch, row_len, pp, trial0, rows, rec, counter, cap, s, maps);
    default: return launch_harm_f<5>(shape, p, ppitch, row_len, pp, trial0, rows, rec, counter, cap, s, maps);
    }
}

constexpr int kDeviceBaselinePasses = 4;

// Grouped prologue: DM trials per group by default, the largest transform
// it applies to by default, and the most acceleration trials per DM trial
// (averaged over a call) for which the default groups.  Measured on B200
// with 1-3 trials per DM trial: 4 rows take the per-DM cost from 89 to
// 55 us at 2^19 points and from 93 to 65 us at 2^20 (8 and 16 rows a
// little less), 150 to 141 us at 2^22, nothing at 2^23, where the
// prologue's launches are long enough to fill the device on their own.
// With many trials per DM trial the trials outweigh the prologue and the
// two slots' overlap already hides it.
constexpr int kGroupRowsDefault = 4;
constexpr int kGroupRowsMax = 16;
constexpr size_t kGroupMaxPoints = (size_t)1 << 22;
constexpr double kGroupMaxTrials = 32.0;

// Rows of the group sets an instance of this configuration may use (0: it
// never groups).
static int group_rows_for(const psx_search_config* c)
{
    if (c->mode != PSX_MODE_BATCHED || c->group_dms == 1) return 0;
    if (c->group_dms >= 2) return c->group_dms;
    return c->fft_size <= kGroupMaxPoints ? kGroupRowsDefault : 0;
}

// Tensor maps of a spectrum buffer of `rows` rows of `pitch` floats for
// the multi-row harmonic kernel: the rows as 8-byte elements, one map per
// window width 32 (c + 1) floats, boxes [width, box_rows]; out-of-bounds
// elements read as zero.  cuTensorMapEncodeTiled comes from the driver
// through the runtime's entry-point query.
static int encode_harm_maps(const float* buf, size_t pitch, int rows, int box_rows, HarmMaps* out)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn) {
            (void)cudaGetLastError();
            set_error("cuTensorMapEncodeTiled is not available from the driver");
            return PSX_ERR_CUDA;
        }
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    if ((pitch & 3) || (reinterpret_cast<uintptr_t>(buf) & 15) || rows < 1) {
        set_error("harmonic maps: pitch must be a multiple of 4 floats and the buffer 16-byte aligned");
        return PSX_ERR_INVALID;
    }
    for (int c = 0; c < kHarmWidthClasses; ++c) {
        const cuuint64_t dims[2] = {(cuuint64_t)(pitch / 2), (cuuint64_t)rows};
        const cuuint64_t strides[1] = {(cuuint64_t)(pitch * sizeof(float))};
        const cuuint32_t box[2] = {(cuuint32_t)(16 * (c + 1)), (cuuint32_t)box_rows};
        const cuuint32_t estr[2] = {1, 1};
        const CUresult r = encode(&out->m[c], CU_TENSOR_MAP_DATA_TYPE_INT64, 2,
                                  const_cast<float*>(buf), dims, strides, box, estr,
                                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) {
            set_error("cuTensorMapEncodeTiled failed (%d) for the harmonic maps", (int)r);
            return PSX_ERR_CUDA;
        }
    }
    return PSX_OK;
}

}  // namespace psx

using namespace psx;

namespace {

size_t round_up(size_t v, size_t m) { return (v + m - 1) / m * m; }

double ms_since(std::chrono::steady_clock::time_point t)
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}

// Untuned trials per launch group: about 2^28 samples (1 GB of resampled
// series) per group, 1..32; cuFFT's batched transforms get faster with the
// batch up to that size on B200 (psx_autotune picks per configuration).
int default_batch(size_t n)
{
    size_t b = ((size_t)1 << 28) / n;
    if (b < 1) b = 1;
    if (b > 32) b = 32;
    size_t p = 1;
    while (p * 2 <= b) p *= 2;
    return (int)p;
}

// Per-DM state that must not be shared by two DMs in flight.
struct Slot {
    int4* d_rec = nullptr;
    // [0] hits, [1] kernel error, [2] baseline still active after the device
    // passes, [3] passes; [4] the loop's start flag, [5] pass counter, [6..]
    // the flag each device pass leaves for the next
    unsigned* d_count = nullptr;
    size_t rec_cap = 0;
    int4* h_rec = nullptr;
    unsigned* h_count = nullptr;
    double* d_ktab = nullptr;
    double* h_ktab = nullptr;
    size_t ktab_cap = 0;
    cudaEvent_t done = nullptr;
    cudaEvent_t copied = nullptr;
    std::vector<cudaEvent_t> ev;  // profiling: prologue start/end, trials start, 4 per launch group
    // The DM's resident dereddened series and the prologue's scratch, one
    // set per slot: the prologue of the next DM runs on this slot's own
    // stream while the previous DM's trials run on the compute stream.
    float* d_tim = nullptr;
    float* d_Xp = nullptr;    // prologue spectrum (Bp complex)
    void* d_med = nullptr;
    double2* d_part = nullptr;
    double* d_sums = nullptr;
    float* d_stat = nullptr;  // interbin statistics: [3] mean*N, [4] std*N
    float* d_mean = nullptr;
    FftPlan* r2c = nullptr;   // batch-1 plans of the prologue
    FftPlan* c2r = nullptr;
    cudaStream_t pst = nullptr;
    cudaEvent_t ready = nullptr;  // prologue complete (on pst)
    // job
    std::vector<float> accs;
    const float* series = nullptr;
    size_t nsamps = 0;
    bool on_device = false;
    bool host_baseline = false;
    float dm = 0.f;
    int dm_idx = 0;
    int groups = 0;
    int launches = 0;
    int ffts = 0;
    bool profiled = false;
    // a slot of a group set: its device buffers are rows of the set's
    // arrays (not freed on their own), its prologue stream is the set's
    bool grouped = false;
};

// Grouped prologue (DM trials with few acceleration trials): G slots whose
// per-DM buffers are rows of contiguous arrays, so that the prologues of G
// DM trials run as one batch -- batched cuFFT plans and row-indexed
// kernels -- instead of G sequences of small launches.
struct GroupSet {
    std::vector<Slot> slots;  // G slots
    float* tim = nullptr;     // G x N dereddened series
    float* Xp = nullptr;      // G x 2 Bp prologue spectra
    float* med = nullptr;     // G x med_floats median scratch
    double2* part = nullptr;  // G x 2 nb partial sums
    double* sums = nullptr;   // G x 2
    float* stat = nullptr;    // G x 8
    unsigned* count = nullptr;  // G x 16 counters and flags
    float* mean = nullptr;    // G x 2
    FftPlan r2c, c2r;         // batch-G plans over the rows
    // Trial schedule spanning the chunk's DM trials (two-pass transform):
    // the trials of all its DM trials in one list (DM trial i's at
    // [off[i], off[i+1])), each with its factor and its series row, and one
    // record buffer for the chunk.
    int4* d_rec = nullptr;
    int4* h_rec = nullptr;
    size_t rec_cap = 0;
    unsigned* d_cnt = nullptr;  // [0] hits, [1] staging error
    unsigned* h_cnt = nullptr;  // d_cnt's two words, then the rows' 16 counters each
    double* d_ktab = nullptr;
    double* h_ktab = nullptr;
    unsigned* d_trow = nullptr;
    unsigned* h_trow = nullptr;
    size_t tab_cap = 0;
    cudaEvent_t done = nullptr;
    std::vector<int> off;
    int groups = 0, launches = 0;
};

struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
    int launches = 0, ffts = 0, groups = 0;
};

}  // namespace

struct psx_search {
    psx_search_config cfg{};
    std::vector<float> bf, bw;
    size_t N = 0, B = 0, Bp = 0;
    int F = 0;
    int batch = 1;
    int harm_shape = 1;
    int lanes = 1;               // streams the launch groups alternate over
    int device = 0;
    cudaStream_t st = nullptr;   // compute (lane 0)
    cudaStream_t st2 = nullptr;  // lane 1
    cudaStream_t cst = nullptr;  // record copies
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    bool own_stream = false;
    // Scheduling priority (a server's hint, psx_search_set_priority): set 0
    // holds the streams made at creation, set 1 the same streams at the
    // device's greatest priority (made on first use); the set in use is
    // swapped at a DM boundary, the new streams waiting for the old ones.
    cudaStream_t set_st[2] = {nullptr, nullptr}, set_st2[2] = {nullptr, nullptr};
    cudaStream_t set_pst[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    cudaEvent_t ev_switch[4] = {nullptr, nullptr, nullptr, nullptr};
    int prio_cur = 0;
    std::atomic<int> prio_want{0};
    double bin_width = 0.0;
    float bin_width_f = 0.f;
    float tobs = 0.f;
    PeakParams pk{};
    float factor[6] = {0, 0, 0, 0, 0, 0};

    // trial buffers of each lane (lane 0 also serves the plain path and the
    // debug tap); d_tr/d_X/d_p alias lane 0
    float* d_trl[2] = {nullptr, nullptr};
    float* d_Xl[2] = {nullptr, nullptr};
    float* d_pl[2] = {nullptr, nullptr};
    HarmMaps hmaps[2] = {};  // per lane: the spectra as boxes of the multi-row shape's rows
    float* d_tr = nullptr;
    float* d_X = nullptr;
    float* d_p = nullptr;
    float* d_bf = nullptr;
    float* d_bw = nullptr;
    size_t bird_cap = 0;  // entries d_bf / d_bw hold
    float* h_mean = nullptr;
    TwSteps tw_steps{};  // unit rotations of the fused unpack kernel

    Slot slot[2];
    // grouped prologue (0 = off): two sets of kGroupRows slots, used in turn
    int group_rows = 0;
    size_t med_floats = 0;
    GroupSet gset[2];
    FftPlan r2c1;                      // plain-mode trials and the debug tap
    Fft4Plan f4;                       // the hand-written transform (fft_form 3)
    bool use_f4 = false;
    cudaEvent_t call_start = nullptr;  // compute-stream position at a call's start
    std::map<int, FftPlan*> r2cb[2];  // batched plans per lane, by batch
    std::map<long long, GraphEntry> graphs;
    std::map<long long, int> capture_failures;

    Slot* last_dm = nullptr;  // the slot of the last DM trial finished (debug tap)
    bool profile = false;
    psx_search_profile prof{};
    psx_search_info info{};
    int nthreads = 1;
    std::unique_ptr<WorkPool> pool;  // nthreads - 1 workers, made on first use

    ~psx_search() { release(); }

    void drop_graphs()
    {
        for (auto& g : graphs) cudaGraphExecDestroy(g.second.exec);
        graphs.clear();
    }

    int apply_priority();

    void release()
    {
        if (prio_cur == 1) {  // back to the creation streams, then drop set 1
            for (cudaStream_t q : {st, st2, slot[0].pst, slot[1].pst})
                if (q) cudaStreamSynchronize(q);
            st = set_st[0];
            st2 = set_st2[0];
            slot[0].pst = set_pst[0][0];
            slot[1].pst = set_pst[0][1];
            prio_cur = 0;
        }
        for (cudaStream_t q : {set_st[1], set_st2[1], set_pst[1][0], set_pst[1][1]})
            if (q) {
                cudaStreamSynchronize(q);
                cudaStreamDestroy(q);
            }
        set_st[1] = set_st2[1] = set_pst[1][0] = set_pst[1][1] = nullptr;
        for (cudaEvent_t& e : ev_switch) {
            if (e) cudaEventDestroy(e);
            e = nullptr;
        }
        if (st) cudaStreamSynchronize(st);
        if (cst) cudaStreamSynchronize(cst);
        drop_graphs();
        if (st2) cudaStreamSynchronize(st2);
        for (auto& m : r2cb) {
            for (auto& p : m) delete p.second;
            m.clear();
        }
        r2c1.destroy();
        void* dev[] = {d_trl[0], d_Xl[0], d_pl[0], d_trl[1], d_Xl[1], d_pl[1], d_bf, d_bw};
        for (void* q : dev)
            if (q) cudaFree(q);
        for (int l = 0; l < 2; ++l) d_trl[l] = d_Xl[l] = d_pl[l] = nullptr;
        d_tr = d_X = d_p = d_bf = d_bw = nullptr;
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        ev_fork = ev_join = nullptr;
        if (call_start) cudaEventDestroy(call_start);
        call_start = nullptr;
        if (h_mean) cudaFreeHost(h_mean);
        h_mean = nullptr;
        last_dm = nullptr;
        free_groups();
        for (Slot& s : slot) {
            if (s.d_rec) cudaFree(s.d_rec);
            if (s.d_count) cudaFree(s.d_count);
            if (s.d_ktab) cudaFree(s.d_ktab);
            if (s.h_rec) cudaFreeHost(s.h_rec);
            if (s.h_count) cudaFreeHost(s.h_count);
            if (s.h_ktab) cudaFreeHost(s.h_ktab);
            if (s.done) cudaEventDestroy(s.done);
            if (s.copied) cudaEventDestroy(s.copied);
            for (cudaEvent_t e : s.ev) cudaEventDestroy(e);
            if (s.pst) cudaStreamSynchronize(s.pst);
            void* sdev[] = {s.d_tim, s.d_Xp, s.d_med, s.d_part, s.d_sums, s.d_stat,
                            s.d_mean};
            for (void* q : sdev)
                if (q) cudaFree(q);
            delete s.r2c;
            delete s.c2r;
            if (s.ready) cudaEventDestroy(s.ready);
            if (s.pst) cudaStreamDestroy(s.pst);
            s = Slot();
        }
        if (cst) cudaStreamDestroy(cst);
        cst = nullptr;
        if (st2) cudaStreamDestroy(st2);
        st2 = nullptr;
        if (own_stream && st) cudaStreamDestroy(st);
        st = nullptr;
        own_stream = false;
    }

    bool batched() const { return cfg.mode == PSX_MODE_BATCHED; }
    // batched trials through the hand-written two-pass transform (resample
    // gather in its first pass) + the unpack kernel of its transposed output
    bool fft4() const { return use_f4; }
    // batched trials through cuFFT's complex transform + fused unpack kernel
    bool fused_form() const { return batched() && cfg.fft_form != 2 && !use_f4; }

    int get_plan(int b, FftPlan** out, int lane = 0);
    int grow_records(Slot& s, size_t need);
    int grow_ktab(Slot& s, size_t need);
    int ensure_events(Slot& s, int groups);
    int prologue(Slot& s);
    int prologue_group(GroupSet& g, int count, cudaStream_t ps);
    int prep(Slot& s, const float* series, size_t nsamps, bool on_device, float dm, int dm_idx);
    int enqueue_trials(Slot& s);
    int alloc_groups();
    int alloc_groups_sets();
    void free_groups();
    // launch groups spanning a chunk's DM trials: the two-pass path with one
    // lane and no stage profiling (which times each DM trial's groups)
    bool span_mode() const { return use_f4 && lanes == 1 && !profile; }
    int grow_span_records(GroupSet& g, size_t need);
    int grow_span_tables(GroupSet& g, size_t need);
    int trials_span(GroupSet& g, int cnt);
    int group_rows_for_call(const float* dms, int ndm) const;
    int trials_enqueue(Slot& s, int nacc);
    int trials_range(Slot& s, int t_begin, int t_end, bool reset);
    int run_trials(Slot& s, int nacc);
    int enqueue(Slot& s, const float* series, size_t nsamps, bool on_device, float dm,
                int dm_idx);
    // The records of one DM trial, copied out of its slot so that the slot
    // can take the next DM trial while they are distilled.
    struct DmRecords {
        std::vector<int4> recs;
        std::vector<float> accs;
        float dm = 0.f;
        int dm_idx = 0;
    };
    int finish(Slot& s, DmRecords& job);
    int finish_span(GroupSet& g, int cnt, std::vector<DmRecords>& jobs);
    void collect(const DmRecords& job, int output, std::vector<psx_candidate>& out,
                 std::vector<int>& nassoc, std::vector<int>& trial_of);
    void read_profile(Slot& s);
};

int psx_search::get_plan(int b, FftPlan** out, int lane)
{
    auto it = r2cb[lane].find(b);
    if (it != r2cb[lane].end()) {
        *out = it->second;
        return PSX_OK;
    }
    FftPlan* p = new (std::nothrow) FftPlan;
    if (!p) return PSX_ERR_ALLOC;
    // fused form: a complex transform of length N/2 over the series read as
    // interleaved pairs (row distances in complex elements)
    int rc = fused_form() ? p->create(N / 2, b, kFftC2C, N / 2, Bp)
                          : p->create(N, b, PSX_FFT_R2C, N, Bp);
    if (rc != PSX_OK) {
        delete p;
        return rc;
    }
    r2cb[lane][b] = p;
    *out = p;
    return PSX_OK;
}

// Swaps in the stream set of the wanted priority (at a DM boundary): the
// new streams first wait for everything queued on the old ones.  Only for
// an instance that owns its streams.
int psx_search::apply_priority()
{
    const int want = prio_want.load(std::memory_order_relaxed) ? 1 : 0;
    if (want == prio_cur || !own_stream) return PSX_OK;
    if (!set_st[1]) {
        int pri_lo = 0, pri_hi = 0;
        PSX_CUDA(cudaDeviceGetStreamPriorityRange(&pri_lo, &pri_hi));
        PSX_CUDA(cudaStreamCreateWithPriority(&set_st[1], cudaStreamNonBlocking, pri_hi));
        if (set_st2[0])
            PSX_CUDA(cudaStreamCreateWithPriority(&set_st2[1], cudaStreamNonBlocking, pri_hi));
        for (int k = 0; k < 2; ++k)
            PSX_CUDA(cudaStreamCreateWithPriority(&set_pst[1][k], cudaStreamNonBlocking, pri_hi));
        for (cudaEvent_t& e : ev_switch)
            if (!e) PSX_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    cudaStream_t from[4] = {st, st2, slot[0].pst, slot[1].pst};
    cudaStream_t to[4] = {set_st[want], set_st2[want], set_pst[want][0], set_pst[want][1]};
    for (int k = 0; k < 4; ++k) {
        if (!from[k] || !to[k]) continue;
        PSX_CUDA(cudaEventRecord(ev_switch[k], from[k]));
        PSX_CUDA(cudaStreamWaitEvent(to[k], ev_switch[k], 0));
    }
    st = set_st[want];
    st2 = set_st2[want];
    slot[0].pst = set_pst[want][0];
    slot[1].pst = set_pst[want][1];
    prio_cur = want;
    return PSX_OK;
}

int psx_search::grow_records(Slot& s, size_t need)
{
    if (need <= s.rec_cap) return PSX_OK;
    const size_t cap = round_up(need + need / 4, 4096);
    PSX_CUDA(cudaStreamSynchronize(st));
    PSX_CUDA(cudaStreamSynchronize(cst));
    if (s.d_rec) cudaFree(s.d_rec);
    if (s.h_rec) cudaFreeHost(s.h_rec);
    s.d_rec = nullptr;
    s.h_rec = nullptr;
    s.rec_cap = 0;
    PSX_CUDA(cudaMalloc(&s.d_rec, sizeof(int4) * cap));
    PSX_CUDA(cudaMallocHost(&s.h_rec, sizeof(int4) * cap));
    s.rec_cap = cap;
    drop_graphs();  // captured schedules hold the old buffer
    return PSX_OK;
}

int psx_search::grow_ktab(Slot& s, size_t need)
{
    if (need <= s.ktab_cap) return PSX_OK;
    const size_t cap = round_up(need + need / 2, 256);
    PSX_CUDA(cudaStreamSynchronize(st));
    if (s.d_ktab) cudaFree(s.d_ktab);
    if (s.h_ktab) cudaFreeHost(s.h_ktab);
    s.d_ktab = nullptr;
    s.h_ktab = nullptr;
    s.ktab_cap = 0;
    PSX_CUDA(cudaMalloc(&s.d_ktab, sizeof(double) * cap));
    PSX_CUDA(cudaMallocHost(&s.h_ktab, sizeof(double) * cap));
    s.ktab_cap = cap;
    drop_graphs();
    return PSX_OK;
}

int psx_search::ensure_events(Slot& s, int groups)
{
    const size_t need = 3 + 4 * (size_t)groups;
    while (s.ev.size() < need) {
        cudaEvent_t e;
        PSX_CUDA(cudaEventCreate(&e));
        s.ev.push_back(e);
    }
    return PSX_OK;
}

// src/pipeline_multi.cu:170-238 for one series, on the slot's own stream.
// It starts once the caller's work queued before this call (call_start)
// and the slot's previous DM (whose trials read s.d_tim) are done, and
// records s.ready; the trials wait for s.ready on the compute stream.  So
// the prologue of DM d+1 runs alongside the trials of DM d.
int psx_search::prologue(Slot& s)
{
    if (!s.r2c) {  // a grouped slot run on its own (a retry): batch-1 plans on first need
        s.r2c = new (std::nothrow) FftPlan;
        s.c2r = new (std::nothrow) FftPlan;
        if (!s.r2c || !s.c2r) return PSX_ERR_ALLOC;
        PSX_TRY(s.r2c->create(N, 1, PSX_FFT_R2C, 0, 0));
        PSX_TRY(s.c2r->create(N, 1, PSX_FFT_C2R, 0, 0));
    }
    cudaStream_t ps = s.pst;
    PSX_CUDA(cudaStreamWaitEvent(ps, call_start, 0));
    PSX_CUDA(cudaStreamWaitEvent(ps, s.done, 0));
    if (s.profiled) PSX_CUDA(cudaEventRecord(s.ev[0], ps));
    const size_t ncopy = std::min(s.nsamps, N);
    // a device series 16-byte aligned is copied by the first baseline pass
    const bool fused_copy =
        s.on_device && !s.host_baseline && (reinterpret_cast<uintptr_t>(s.series) & 15u) == 0;
    if (!fused_copy)
        PSX_CUDA(cudaMemcpyAsync(s.d_tim, s.series, sizeof(float) * ncopy,
                                 s.on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                 ps));
    // baseline removal over the copied samples (timeseries.hpp:282-287,
    // src/kernels.cu:463-479)
    const int nb = reduction_blocks();
    if (!s.host_baseline) {
        // sums of the series, then per pass one kernel: the mean of the
        // previous sums, the subtraction and the new sums (which alternate
        // between the two halves of d_part); passes after convergence
        // return at once
        unsigned* st = s.d_count + 4;  // [0] start flag, [1] passes
        if (fused_copy)
            PSX_TRY(launch_partials_v4(s.series, ncopy, s.d_part, s.d_tim, st, ps));
        else
            PSX_TRY(launch_partials_v4(s.d_tim, ncopy, s.d_part, nullptr, st, ps));
        ++s.launches;
        for (int pass = 0; pass < kDeviceBaselinePasses; ++pass) {
            const bool last = pass == kDeviceBaselinePasses - 1;
            PSX_TRY(launch_baseline_pass_v4(
                s.d_tim, ncopy, s.d_part + (pass & 1) * nb, s.d_part + ((pass + 1) & 1) * nb,
                pass == 0 ? st : s.d_count + 6 + pass - 1, s.d_count + 6 + pass, st + 1,
                last ? s.d_count + 2 : nullptr, last ? s.d_count + 3 : nullptr, ps));
            ++s.launches;
        }
    } else {
        int count = 0;
        float mean = 0.f;
        do {
            PSX_TRY(remove_baseline_pass(s.d_tim, ncopy, s.d_part, s.d_sums, s.d_mean, ps));
            s.launches += 4;
            PSX_CUDA(cudaMemcpyAsync(h_mean, s.d_mean, sizeof(float), cudaMemcpyDeviceToHost, ps));
            PSX_CUDA(cudaStreamSynchronize(ps));
            mean = *h_mean;
            if (count++ > 100) break;
        } while (std::fabs(mean) > 5e-7 * (double)ncopy);
    }
    // zero padding (pipeline_multi.cu:179-187)
    if (ncopy < N) {
        PSX_TRY(launch_fill(s.d_tim + ncopy, N - ncopy, 0.f, ps));
        ++s.launches;
    }
    PSX_TRY(s.r2c->exec(s.d_tim, s.d_Xp, ps));
    ++s.ffts;
    // amplitude spectrum (spectrumformer.hpp:16-22)
    // amplitudes, their 5/25/125-bin medians, and the division by the
    // spliced median (spectrumformer.hpp:16-22, dereddener.hpp:41-66)
    PSX_TRY(launch_running_median_spectrum(s.d_Xp, B, bin_width, cfg.boundary_5_freq,
                                           cfg.boundary_25_freq, s.d_med, ps));
    s.launches += 2;
    if (!bf.empty()) {
        PSX_TRY(launch_zap(s.d_Xp, d_bf, d_bw, bin_width_f, bf.size(), B, ps));
        ++s.launches;
    }
    // interbin statistics (pipeline_multi.cu:230-234) -> mean*N, std*N
    PSX_TRY(launch_interbin_stats_v4(s.d_Xp, B, s.d_part, s.d_sums, s.d_stat, (float)N, ps));
    s.launches += 2;
    PSX_TRY(s.c2r->exec(s.d_Xp, s.d_tim, ps));
    ++s.ffts;
    if (s.profiled) PSX_CUDA(cudaEventRecord(s.ev[1], ps));
    PSX_CUDA(cudaEventRecord(s.ready, ps));
    return PSX_OK;
}

int psx_search::grow_span_records(GroupSet& g, size_t need)
{
    if (need <= g.rec_cap) return PSX_OK;
    const size_t cap = round_up(need + need / 4, 4096);
    PSX_CUDA(cudaStreamSynchronize(st));
    PSX_CUDA(cudaStreamSynchronize(cst));
    if (g.d_rec) cudaFree(g.d_rec);
    if (g.h_rec) cudaFreeHost(g.h_rec);
    g.d_rec = g.h_rec = nullptr;
    g.rec_cap = 0;
    PSX_CUDA(cudaMalloc(&g.d_rec, sizeof(int4) * cap));
    PSX_CUDA(cudaMallocHost(&g.h_rec, sizeof(int4) * cap));
    g.rec_cap = cap;
    return PSX_OK;
}

int psx_search::grow_span_tables(GroupSet& g, size_t need)
{
    if (need <= g.tab_cap) return PSX_OK;
    const size_t cap = round_up(need + need / 4, 256);
    PSX_CUDA(cudaStreamSynchronize(st));
    for (void* q : {(void*)g.d_ktab, (void*)g.d_trow})
        if (q) cudaFree(q);
    for (void* q : {(void*)g.h_ktab, (void*)g.h_trow})
        if (q) cudaFreeHost(q);
    g.d_ktab = g.h_ktab = nullptr;
    g.d_trow = g.h_trow = nullptr;
    g.tab_cap = 0;
    PSX_CUDA(cudaMalloc((void**)&g.d_ktab, sizeof(double) * cap));
    PSX_CUDA(cudaMalloc((void**)&g.d_trow, sizeof(unsigned) * cap));
    PSX_CUDA(cudaMallocHost(&g.h_ktab, sizeof(double) * cap));
    PSX_CUDA(cudaMallocHost(&g.h_trow, sizeof(unsigned) * cap));
    g.tab_cap = cap;
    return PSX_OK;
}

// The trials of a chunk's cnt DM trials (prologues queued, factors in the
// slots) as one list in launch groups of `batch` that run across DM-trial
// boundaries: pass 1 gathers each trial from its own series row, the unpack
// normalises it with its own row's statistics, and the harmonic kernel's
// records carry the trial's index in the list.  On the compute stream;
// records g.done and every slot's done.
int psx_search::trials_span(GroupSet& g, int cnt)
{
    const int T = g.off[cnt];
    for (int i = 0; i < cnt; ++i) {
        Slot& sl = g.slots[i];
        PSX_CUDA(cudaStreamWaitEvent(st, sl.ready, 0));
        // each slot keeps its own factors too (the debug tap reads them)
        PSX_CUDA(cudaMemcpyAsync(sl.d_ktab, sl.h_ktab, sizeof(double) * sl.accs.size(),
                                 cudaMemcpyHostToDevice, st));
    }
    PSX_CUDA(cudaMemcpyAsync(g.d_ktab, g.h_ktab, sizeof(double) * T, cudaMemcpyHostToDevice, st));
    PSX_CUDA(cudaMemcpyAsync(g.d_trow, g.h_trow, sizeof(unsigned) * T, cudaMemcpyHostToDevice, st));
    PSX_CUDA(cudaMemsetAsync(g.d_cnt, 0, sizeof(unsigned) * 2, st));
    const bool span = pk.hi > pk.lo;
    float* tr = d_trl[0];
    float* X = d_Xl[0];
    float* pp = d_pl[0];
    g.groups = 0;
    g.launches = 0;
    for (int t0 = 0; t0 < T;) {
        const int b = std::min(batch, T - t0);
        PSX_TRY(f4.exec_cols(g.tim, g.d_ktab + t0, b, reinterpret_cast<float2*>(tr), N / 2, st,
                             g.d_trow + t0, N));
        PSX_TRY(f4.exec_rows(reinterpret_cast<const float2*>(tr), N / 2, b,
                             reinterpret_cast<float2*>(X), Bp, st));
        PSX_TRY(f4.form(reinterpret_cast<const float2*>(X), Bp, b, pp, Bp, g.stat, st,
                        g.d_trow + t0));
        g.launches += 3;
        if (span) {  // as trials_range: leftover trials on the single-row shape
            const int rows = kHarmShapes[harm_shape - 1].rows;
            const int rem = rows > 1 ? b % rows : 0, bm = b - rem;
            if (bm > 0) {
                PSX_TRY(launch_harm(F, harm_shape, pp, Bp, (unsigned)Bp, pk, t0, bm, g.d_rec,
                                    g.d_cnt, (unsigned)g.rec_cap, st, &hmaps[0]));
                ++g.launches;
            }
            if (rem > 0) {
                PSX_TRY(launch_harm(F, kHarmDefaultShape, pp + (size_t)bm * Bp, Bp, (unsigned)Bp,
                                    pk, t0 + bm, rem, g.d_rec, g.d_cnt, (unsigned)g.rec_cap, st));
                ++g.launches;
            }
        }
        t0 += b;
        ++g.groups;
    }
    // the hit counter, and every row's prologue counters (baseline flags)
    PSX_CUDA(cudaMemcpyAsync(g.h_cnt, g.d_cnt, sizeof(unsigned) * 2, cudaMemcpyDeviceToHost, st));
    PSX_CUDA(cudaMemcpyAsync(g.h_cnt + 2, g.count, sizeof(unsigned) * 16 * (size_t)cnt,
                             cudaMemcpyDeviceToHost, st));
    PSX_CUDA(cudaEventRecord(g.done, st));
    for (int i = 0; i < cnt; ++i) PSX_CUDA(cudaEventRecord(g.slots[i].done, st));
    return PSX_OK;
}

// Waits for a spanning chunk, grows its record buffer and runs its trials
// again if they overflowed it, and splits the records into one job per DM
// trial (trial indices back to each DM trial's own); a DM trial whose
// baseline needed more passes than the device loop makes runs again alone
// through the per-DM path with the host loop.
int psx_search::finish_span(GroupSet& g, int cnt, std::vector<DmRecords>& jobs)
{
    for (int attempt = 0;; ++attempt) {
        const auto t_wait = std::chrono::steady_clock::now();
        PSX_CUDA(cudaEventSynchronize(g.done));
        prof.host_wait_ms += ms_since(t_wait);
        if (g.h_cnt[1] != 0) {
            set_error("search: harmonic-sum staging did not complete (status 0x%x)", g.h_cnt[1]);
            return PSX_ERR_CUDA;
        }
        if (g.h_cnt[0] <= g.rec_cap) break;
        if (attempt == 2) {
            set_error("search: could not complete DM trials %d..", g.slots[0].dm_idx);
            return PSX_ERR_OVERFLOW;
        }
        PSX_TRY(grow_span_records(g, g.h_cnt[0]));
        PSX_TRY(trials_span(g, cnt));
    }
    const size_t nrec = g.h_cnt[0];
    if (nrec) {
        PSX_CUDA(cudaStreamWaitEvent(cst, g.done, 0));
        PSX_CUDA(cudaMemcpyAsync(g.h_rec, g.d_rec, sizeof(int4) * nrec, cudaMemcpyDeviceToHost,
                                 cst));
        PSX_CUDA(cudaStreamSynchronize(cst));
    }
    jobs.assign(cnt, DmRecords{});
    for (int i = 0; i < cnt; ++i) {
        const Slot& sl = g.slots[i];
        jobs[i].accs = sl.accs;
        jobs[i].dm = sl.dm;
        jobs[i].dm_idx = sl.dm_idx;
    }
    for (size_t r = 0; r < nrec; ++r) {
        int4 q = g.h_rec[r];
        if (q.x < 0 || q.x >= g.off[cnt]) continue;
        const int i = (int)(std::upper_bound(g.off.begin(), g.off.begin() + cnt + 1, q.x) -
                            g.off.begin()) - 1;
        q.x -= g.off[i];
        jobs[i].recs.push_back(q);
    }
    const int T = g.off[cnt];
    info.ntrials += T;
    info.nbatches += g.groups;
    info.kernel_launches += g.launches + g.slots[0].launches;
    info.fft_launches += g.slots[0].ffts;
    info.above_threshold += (long long)nrec;
    for (int i = 0; i < cnt; ++i) {
        const unsigned* c = g.h_cnt + 2 + 16 * (size_t)i;
        Slot& sl = g.slots[i];
        info.baseline_passes = (int)c[3];
        if (c[2] != 0) {  // rare: the baseline loop needs the host
            info.ntrials -= (int)sl.accs.size();
            info.above_threshold -= (long long)jobs[i].recs.size();
            sl.host_baseline = true;
            PSX_TRY(enqueue(sl, sl.series, sl.nsamps, sl.on_device, sl.dm, sl.dm_idx));
            PSX_TRY(finish(sl, jobs[i]));
        }
    }
    last_dm = &g.slots[cnt - 1];
    return PSX_OK;
}

// Group sets, made when the instance is created (where its configuration
// can group): per set, the per-DM
// buffers of G slots as rows of contiguous arrays (row strides N, 2 Bp,
// the median scratch, 2 nb, 2, 8, 16 and 2 elements), the batch-G plans
// of the prologue's transforms, and per slot its own record buffer, factor
// table, pinned counters and events.
int psx_search::alloc_groups()
{
    if (!gset[0].slots.empty()) return PSX_OK;
    const int rc = alloc_groups_sets();
    if (rc != PSX_OK) free_groups();  // nothing half-made stays for the next call
    return rc;
}

int psx_search::alloc_groups_sets()
{
    const int G = group_rows_for(&cfg);
    if (G < 2) return PSX_OK;
    const size_t nb = (size_t)reduction_blocks();
    med_floats = median_scratch_bytes(B) / sizeof(float);
    for (GroupSet& g : gset) {
        PSX_CUDA(cudaMalloc((void**)&g.tim, sizeof(float) * N * G));
        PSX_CUDA(cudaMalloc((void**)&g.Xp, sizeof(float) * 2 * Bp * G));
        PSX_CUDA(cudaMalloc((void**)&g.med, sizeof(float) * med_floats * G));
        PSX_CUDA(cudaMalloc((void**)&g.part, sizeof(double2) * 2 * nb * G));
        PSX_CUDA(cudaMalloc((void**)&g.sums, sizeof(double) * 2 * G));
        PSX_CUDA(cudaMalloc((void**)&g.stat, sizeof(float) * 8 * G));
        PSX_CUDA(cudaMalloc((void**)&g.count, sizeof(unsigned) * 16 * G));
        PSX_CUDA(cudaMalloc((void**)&g.mean, sizeof(float) * 2 * G));
        // rows past a call's last DM trial are transformed too (the plans
        // hold G rows): they start as zeros, never as uninitialised memory
        PSX_CUDA(cudaMemsetAsync(g.tim, 0, sizeof(float) * N * G, st));
        PSX_CUDA(cudaMemsetAsync(g.Xp, 0, sizeof(float) * 2 * Bp * G, st));
        PSX_TRY(g.r2c.create(N, G, PSX_FFT_R2C, N, Bp));
        PSX_TRY(g.c2r.create(N, G, PSX_FFT_C2R, Bp, N));
        if (use_f4) {  // the spanning trial schedule's counters and event
            PSX_CUDA(cudaMalloc((void**)&g.d_cnt, sizeof(unsigned) * 4));
            PSX_CUDA(cudaMallocHost(&g.h_cnt, sizeof(unsigned) * (2 + 16 * (size_t)G)));
            PSX_CUDA(cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming));
            PSX_TRY(grow_span_records(g, (size_t)1 << 20));
            PSX_TRY(grow_span_tables(g, 256));
        }
        g.slots.resize(G);
        for (int i = 0; i < G; ++i) {
            Slot& sl = g.slots[i];
            sl.grouped = true;
            sl.d_tim = g.tim + (size_t)i * N;
            sl.d_Xp = g.Xp + (size_t)i * 2 * Bp;
            sl.d_med = g.med + (size_t)i * med_floats;
            sl.d_part = g.part + (size_t)i * 2 * nb;
            sl.d_sums = g.sums + 2 * i;
            sl.d_stat = g.stat + 8 * i;
            sl.d_count = g.count + 16 * i;
            sl.d_mean = g.mean + 2 * i;
            PSX_CUDA(cudaMallocHost(&sl.h_count, sizeof(unsigned) * 4));
            PSX_CUDA(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
            PSX_CUDA(cudaEventCreateWithFlags(&sl.copied, cudaEventDisableTiming));
            PSX_CUDA(cudaEventCreateWithFlags(&sl.ready, cudaEventDisableTiming));
            PSX_TRY(grow_records(sl, (size_t)1 << 18));
            PSX_TRY(grow_ktab(sl, 64));
        }
    }
    PSX_CUDA(cudaStreamSynchronize(st));
    return PSX_OK;
}

void psx_search::free_groups()
{
    for (Slot& s : slot)
        if (s.pst) cudaStreamSynchronize(s.pst);
    for (GroupSet& g : gset) {
        for (Slot& s : g.slots) {
            if (s.d_rec) cudaFree(s.d_rec);
            if (s.d_ktab) cudaFree(s.d_ktab);
            if (s.h_rec) cudaFreeHost(s.h_rec);
            if (s.h_count) cudaFreeHost(s.h_count);
            if (s.h_ktab) cudaFreeHost(s.h_ktab);
            for (cudaEvent_t e : {s.done, s.copied, s.ready})
                if (e) cudaEventDestroy(e);
            for (cudaEvent_t e : s.ev) cudaEventDestroy(e);
            delete s.r2c;  // batch-1 plans of a retried DM trial, if any
            delete s.c2r;
        }
        g.slots.clear();
        for (void* q : {(void*)g.d_rec, (void*)g.d_cnt, (void*)g.d_ktab, (void*)g.d_trow})
            if (q) cudaFree(q);
        for (void* q : {(void*)g.h_rec, (void*)g.h_cnt, (void*)g.h_ktab, (void*)g.h_trow})
            if (q) cudaFreeHost(q);
        if (g.done) cudaEventDestroy(g.done);
        g.d_rec = g.h_rec = nullptr;
        g.d_cnt = g.h_cnt = g.d_trow = g.h_trow = nullptr;
        g.d_ktab = g.h_ktab = nullptr;
        g.rec_cap = g.tab_cap = 0;
        g.done = nullptr;
        void* dev[] = {g.tim, g.Xp, g.med, g.part, g.sums, g.stat, g.count, g.mean};
        for (void* q : dev)
            if (q) cudaFree(q);
        g.tim = g.Xp = g.med = g.stat = g.mean = nullptr;
        g.part = nullptr;
        g.sums = nullptr;
        g.count = nullptr;
        g.r2c.destroy();
        g.c2r.destroy();
    }
}

// Rows per grouped prologue for a call over these DM trials (0: one
// prologue per DM trial).  A call groups when it has more DM trials than a
// group holds; by default also only when its DM trials average at most
// kGroupMaxTrials acceleration trials.
int psx_search::group_rows_for_call(const float* dms, int ndm) const
{
    const int G = group_rows_for(&cfg);
    if (G < 2 || ndm <= G) return 0;
    if (cfg.group_dms >= 2) return G;
    const psx_search_config& c = cfg;
    double total = 0.0;
    for (int d = 0; d < ndm; ++d)
        total += (double)accel_list(c.acc_lo, c.acc_hi, c.acc_tol, c.acc_pulse_width, N, c.tsamp,
                                    c.cfreq_hz, c.ch_bw_hz, dms[d], c.cdm)
                     .size();
    return total <= kGroupMaxTrials * ndm ? G : 0;
}

// The prologues of the first `count` slots of a group set as one batch:
// each launch of prologue() becomes one launch over `count` rows (grid y =
// row) that computes every row exactly as the single-row launch computes
// it, and the two transforms run as batch-G plans.  On stream ps, after the
// caller's work queued before the call and after every slot of the set is
// done with its previous DM trial; records each slot's ready.
int psx_search::prologue_group(GroupSet& g, int count, cudaStream_t ps)
{
    PSX_CUDA(cudaStreamWaitEvent(ps, call_start, 0));
    for (Slot& sl : g.slots) PSX_CUDA(cudaStreamWaitEvent(ps, sl.done, 0));
    Slot& s0 = g.slots[0];
    if (s0.profiled) PSX_CUDA(cudaEventRecord(s0.ev[0], ps));
    const size_t ncopy = std::min(s0.nsamps, N);  // one length for every series of a call
    for (int i = 0; i < count; ++i) {
        Slot& sl = g.slots[i];
        sl.pst = ps;
        PSX_CUDA(cudaMemcpyAsync(sl.d_tim, sl.series, sizeof(float) * ncopy,
                                 sl.on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                 ps));
    }
    // baseline removal (timeseries.hpp:282-287, src/kernels.cu:463-479):
    // the device loop of prologue(), row by row
    const size_t nb = (size_t)reduction_blocks(), pst_ = 2 * nb;
    unsigned* c = g.count;
    PSX_TRY(launch_partials_rows(g.tim, ncopy, N, count, g.part, pst_, c + 4, 16, ps));
    for (int pass = 0; pass < kDeviceBaselinePasses; ++pass) {
        const bool last = pass == kDeviceBaselinePasses - 1;
        PSX_TRY(launch_baseline_pass_rows(
            g.tim, ncopy, N, count, g.part + (pass & 1) * nb, g.part + ((pass + 1) & 1) * nb, pst_,
            pass == 0 ? c + 4 : c + 6 + pass - 1, c + 6 + pass, c + 5, last ? c + 2 : nullptr,
            last ? c + 3 : nullptr, 16, ps));
    }
    // zero padding (pipeline_multi.cu:179-187)
    if (ncopy < N) PSX_TRY(launch_fill_rows(g.tim + ncopy, N - ncopy, N, count, 0.f, ps));
    PSX_TRY(g.r2c.exec(g.tim, g.Xp, ps));
    // amplitudes, medians and dereddening (spectrumformer.hpp:16-22,
    // dereddener.hpp:41-66), zapping, interbin statistics
    // (pipeline_multi.cu:230-234), inverse transform
    PSX_TRY(launch_running_median_spectrum_rows(g.Xp, 2 * Bp, count, B, bin_width,
                                                cfg.boundary_5_freq, cfg.boundary_25_freq, g.med,
                                                med_floats, ps));
    if (!bf.empty())
        PSX_TRY(launch_zap_rows(g.Xp, 2 * Bp, count, d_bf, d_bw, bin_width_f, bf.size(), B, ps));
    PSX_TRY(launch_interbin_stats_rows(g.Xp, 2 * Bp, count, B, g.part, pst_, g.sums, 2, g.stat, 8,
                                       (float)N, ps));
    PSX_TRY(g.c2r.exec(g.Xp, g.tim, ps));
    const int launches = 5 + (ncopy < N ? 1 : 0) + 2 + (bf.empty() ? 0 : 1) + 2;
    for (int i = 0; i < count; ++i) {
        Slot& sl = g.slots[i];
        // the batch's launches and transforms are counted once, on row 0
        sl.launches += i == 0 ? launches : 0;
        sl.ffts += i == 0 ? 2 : 0;
        // profiling: the batch's span is row 0's prologue, the other rows
        // get an empty one
        if (sl.profiled) {
            if (i) PSX_CUDA(cudaEventRecord(sl.ev[0], ps));
            PSX_CUDA(cudaEventRecord(sl.ev[1], ps));
        }
        PSX_CUDA(cudaEventRecord(sl.ready, ps));
    }
    return PSX_OK;
}

// Trials of the launch group starting at t0: `batch` while that many are
// left; the rest as one group with the two-pass transform (any group size
// works there), else in power-of-two groups (the cuFFT plans exist for
// powers of two only).
static int group_size(int nacc, int t0, int batch, bool any_size)
{
    int b = batch;
    if (any_size) return std::min(b, nacc - t0);
    while (b > nacc - t0) b >>= 1;
    return b;
}

// Enqueues every acceleration trial of the DM (k factors already in
// s.d_ktab) plus the reset of the record counter.
int psx_search::trials_enqueue(Slot& s, int nacc)
{
    s.groups = 0;
    return trials_range(s, 0, nacc, true);
}

// Enqueues trials [t_begin, t_end) of the DM in launch groups (numbered on
// from s.groups), after the reset of the record counter when `reset`.
int psx_search::trials_range(Slot& s, int t_begin, int nacc, bool reset)
{
    if (reset) {
        PSX_CUDA(cudaMemsetAsync(s.d_count, 0, sizeof(unsigned) * 2, st));
        if (s.profiled) PSX_CUDA(cudaEventRecord(s.ev[2], st));
    }
    const unsigned T = 256;
    const unsigned span = pk.hi > pk.lo ? pk.hi - pk.lo : 0;
    // launch groups alternate over the lanes; lane 1 starts after the
    // counter reset and lane 0 waits for lane 1 at the end (fork / join,
    // also inside a graph capture)
    const int L = batched() ? lanes : 1;
    if (L > 1) {
        PSX_CUDA(cudaEventRecord(ev_fork, st));
        PSX_CUDA(cudaStreamWaitEvent(st2, ev_fork, 0));
    }
    int t0 = t_begin, g = s.groups;
    while (t0 < nacc) {
        const int lane = g % L;
        cudaStream_t ls = lane ? st2 : st;
        float* tr = d_trl[lane];
        float* X = d_Xl[lane];
        float* pp = d_pl[lane];
        int b = 1;
        if (fft4()) {
            // resample gather + transform in two passes; the profile times
            // the first pass (which does the gather) as the resample stage
            b = group_size(nacc, t0, batch, true);
            PSX_TRY(f4.exec_cols(s.d_tim, s.d_ktab + t0, b, reinterpret_cast<float2*>(tr), N / 2,
                                 ls));
            if (s.profiled) PSX_CUDA(cudaEventRecord(s.ev[3 + 4 * g], ls));
            PSX_TRY(f4.exec_rows(reinterpret_cast<const float2*>(tr), N / 2, b,
                                 reinterpret_cast<float2*>(X), Bp, ls));
            s.launches += 2;
        } else if (batched()) {
            b = batch;
            while (b > nacc - t0) b >>= 1;
            FftPlan* plan = nullptr;
            PSX_TRY(get_plan(b, &plan, lane));
            PSX_TRY(launch_resample(s.d_tim, tr, N, s.d_ktab + t0, 0.0, b, N, false, ls));
            ++s.launches;
            if (s.profiled) PSX_CUDA(cudaEventRecord(s.ev[3 + 4 * g], ls));
            PSX_TRY(plan->exec(tr, X, ls));
            ++s.ffts;
        } else {
            PSX_TRY(launch_resample(s.d_tim, tr, N, s.d_ktab + t0, 0.0, 1, N, false, ls));
            ++s.launches;
            if (s.profiled) PSX_CUDA(cudaEventRecord(s.ev[3 + 4 * g], ls));
            PSX_TRY(r2c1.exec(tr, X, ls));
            ++s.ffts;
        }
        if (s.profiled) PSX_CUDA(cudaEventRecord(s.ev[3 + 4 * g + 1], ls));
        if (fft4()) {
            PSX_TRY(f4.form(reinterpret_cast<const float2*>(X), Bp, b, pp, Bp, s.d_stat, ls));
        } else if (fused_form()) {
            const unsigned M = (unsigned)(N / 2);
            dim3 gu(grid_for(M / 8, T, 4), (unsigned)b);
            k_unpack_form_norm<<<gu, T, 0, ls>>>(X, Bp, pp, Bp, M, 1.0f / (float)M, tw_steps,
                                                 s.d_stat);
        } else {
            dim3 gf(grid_for(B / 2 + 1, T, 4), (unsigned)b);
            k_form_norm<<<gf, T, 0, ls>>>(X, 2 * Bp, pp, Bp, (unsigned)B, s.d_stat);
        }
        ++s.launches;
        PSX_TRY(launch_status("form kernel"));
        if (s.profiled) PSX_CUDA(cudaEventRecord(s.ev[3 + 4 * g + 2], ls));
        if (span) {
            // A multi-row shape stages `rows` trials per tile; the group's
            // last b % rows trials go to the single-row default shape
            // instead of a tile padded with unused rows (every shape gives
            // the same records).
            const int rows = kHarmShapes[harm_shape - 1].rows;
            const int rem = rows > 1 ? b % rows : 0, bm = b - rem;
            if (bm > 0) {
                PSX_TRY(launch_harm(F, harm_shape, pp, Bp, (unsigned)Bp, pk, t0, bm, s.d_rec,
                                    s.d_count, (unsigned)s.rec_cap, ls, &hmaps[lane]));
                ++s.launches;
            }
            if (rem > 0) {
                PSX_TRY(launch_harm(F, kHarmDefaultShape, pp + (size_t)bm * Bp, Bp, (unsigned)Bp,
                                    pk, t0 + bm, rem, s.d_rec, s.d_count, (unsigned)s.rec_cap, ls));
                ++s.launches;
            }
        }
        if (s.profiled) PSX_CUDA(cudaEventRecord(s.ev[3 + 4 * g + 3], ls));
        t0 += b;
        ++g;
    }
    if (L > 1) {
        PSX_CUDA(cudaEventRecord(ev_join, st2));
        PSX_CUDA(cudaStreamWaitEvent(st, ev_join, 0));
    }
    s.groups = g;
    return PSX_OK;
}

static int count_groups(int nacc, bool batched, int batch, bool any_size)
{
    if (!batched) return nacc;
    int t0 = 0, g = 0;
    while (t0 < nacc) {
        t0 += group_size(nacc, t0, batch, any_size);
        ++g;
    }
    return g;
}

int psx_search::run_trials(Slot& s, int nacc)
{
    // events recorded inside a graph carry no timestamps: profiling runs
    // the schedule without capture
    // (a grouped slot's schedule is launched directly: graphs are keyed by
    // the two regular slots' buffers)
    const bool graph = batched() && cfg.use_graph && !s.profiled && !s.grouped;
    if (s.profiled) PSX_TRY(ensure_events(s, count_groups(nacc, batched(), batch, fft4())));
    if (!graph) return trials_enqueue(s, nacc);
    // One lane: the graph holds the counter reset and the full launch groups
    // and is keyed by their number, which neighbouring DM trials share (the
    // trial count changes slowly with DM), so few graphs are captured; the
    // shorter tail groups are launched directly after it.  Two lanes: one
    // graph per trial count.
    const int upto = lanes == 1 ? (nacc / batch) * batch : nacc;
    if (upto == 0) return trials_enqueue(s, nacc);
    const long long key = ((long long)upto << 2) | ((&s == &slot[1]) ? 2 : 0);
    auto it = graphs.find(key);
    auto tail = [&]() -> int {
        if (upto >= nacc) return PSX_OK;
        return trials_range(s, upto, nacc, false);
    };
    if (it == graphs.end() && capture_failures[key] >= 2) return trials_enqueue(s, nacc);
    if (it == graphs.end()) {
        // cuFFT plans must exist before capture (creation allocates); the
        // two-pass transform has none
        if (!fft4())
            for (int l = 0; l < lanes; ++l)
                for (int b = batch; b >= 1; b >>= 1) {
                    FftPlan* p = nullptr;
                    PSX_TRY(get_plan(b, &p, l));
                }
        const int l0 = s.launches, f0 = s.ffts;
        PSX_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        int rc = trials_enqueue(s, upto);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (rc != PSX_OK || e != cudaSuccess) {
            // A capture can be invalidated from outside this instance (in a
            // multi-threaded host, e.g. by a kernel module loaded on first
            // use while the capture is open).  Nothing captured has run:
            // launch the same schedule directly and try capturing next time.
            if (g) cudaGraphDestroy(g);
            (void)cudaGetLastError();  // capture errors are not sticky
            clear_error();
            s.launches = l0;
            s.ffts = f0;
            ++info.capture_fallbacks;
            ++capture_failures[key];  // after two, this schedule is not captured again
            return trials_enqueue(s, nacc);
        }
        GraphEntry ge;
        e = cudaGraphInstantiate(&ge.exec, g, 0);
        cudaGraphDestroy(g);
        PSX_CUDA(e);
        ge.launches = s.launches - l0;
        ge.ffts = s.ffts - f0;
        ge.groups = s.groups;
        s.launches = l0;
        s.ffts = f0;
        it = graphs.emplace(key, ge).first;
    }
    PSX_CUDA(cudaGraphLaunch(it->second.exec, st));
    s.launches += it->second.launches;
    s.ffts += it->second.ffts;
    s.groups = it->second.groups;
    PSX_TRY(tail());
    return PSX_OK;
}

// The host half of one DM trial's set-up: its job fields, acceleration list
// and factors, and the profiling events it needs.
int psx_search::prep(Slot& s, const float* series, size_t nsamps, bool on_device, float dm,
                     int dm_idx)
{
    const psx_search_config& c = cfg;
    s.series = series;
    s.nsamps = nsamps;
    s.on_device = on_device;
    s.dm = dm;
    s.dm_idx = dm_idx;
    s.launches = 0;
    s.ffts = 0;
    s.groups = 0;
    s.profiled = profile;
    s.accs = accel_list(c.acc_lo, c.acc_hi, c.acc_tol, c.acc_pulse_width, N, c.tsamp, c.cfreq_hz,
                        c.ch_bw_hz, dm, c.cdm);
    const int nacc = (int)s.accs.size();
    PSX_TRY(grow_ktab(s, (size_t)nacc));
    for (int t = 0; t < nacc; ++t) s.h_ktab[t] = accel_fact(s.accs[t], c.tsamp);
    if (s.profiled) PSX_TRY(ensure_events(s, count_groups(nacc, batched(), batch, fft4())));
    return PSX_OK;
}

// The trials of a DM trial whose prologue is queued (s.ready): its factors,
// the trial schedule, the hit counter's copy back and s.done.
int psx_search::enqueue_trials(Slot& s)
{
    const int nacc = (int)s.accs.size();
    PSX_CUDA(cudaStreamWaitEvent(st, s.ready, 0));
    PSX_CUDA(cudaMemcpyAsync(s.d_ktab, s.h_ktab, sizeof(double) * nacc, cudaMemcpyHostToDevice, st));
    PSX_TRY(run_trials(s, nacc));
    PSX_CUDA(cudaMemcpyAsync(s.h_count, s.d_count, sizeof(unsigned) * 4, cudaMemcpyDeviceToHost, st));
    PSX_CUDA(cudaEventRecord(s.done, st));
    return PSX_OK;
}

int psx_search::enqueue(Slot& s, const float* series, size_t nsamps, bool on_device, float dm,
                        int dm_idx)
{
    const auto t_host = std::chrono::steady_clock::now();
    PSX_TRY(apply_priority());
    PSX_TRY(prep(s, series, nsamps, on_device, dm, dm_idx));
    PSX_TRY(prologue(s));
    PSX_TRY(enqueue_trials(s));
    prof.host_enqueue_ms += ms_since(t_host);
    return PSX_OK;
}

void psx_search::read_profile(Slot& s)
{
    if (!s.profiled) return;
    auto span = [&](cudaEvent_t a, cudaEvent_t b, double& acc) {
        float ms = 0.f;
        const cudaError_t e = cudaEventElapsedTime(&ms, a, b);
        if (e == cudaSuccess) {
            acc += ms;
        } else {
            ++prof.event_errors;
            prof.last_event_error = (int)e;
        }
    };
    span(s.ev[0], s.ev[1], prof.prologue_ms);
    for (int g = 0; g < s.groups; ++g) {
        // the previous group of the same lane (or the start of the trials)
        const int L = batched() ? lanes : 1;
        cudaEvent_t prev = g < L ? s.ev[2] : s.ev[3 + 4 * (g - L) + 3];
        cudaEvent_t* e = &s.ev[3 + 4 * g];
        span(prev, e[0], prof.resample_ms);
        span(e[0], e[1], prof.fft_ms);
        span(e[1], e[2], prof.form_ms);
        span(e[2], e[3], prof.harm_ms);
    }
    prof.groups += s.groups;
    prof.trials += (long long)s.accs.size();
    prof.dms += 1;
    cudaGetLastError();
}

// Host side of one DM: bucket the records by (trial, fold), order each
// bucket by bin (the order the reference's copy_if leaves them in),
// cluster (peakfinder.hpp:72-94), form candidate frequencies, distil per
// trial (pipeline_multi.cu:283-289) and optionally per DM (:294).
void psx_search::collect(const DmRecords& job, int output, std::vector<psx_candidate>& out,
                         std::vector<int>& nassoc, std::vector<int>& trial_of)
{
    const int nacc = (int)job.accs.size();
    const size_t nrec = job.recs.size();
    const int nf = F + 1;
    const size_t nkeys = (size_t)nacc * nf;
    std::vector<unsigned> off(nkeys + 1, 0);
    for (size_t r = 0; r < nrec; ++r) {
        const int4 q = job.recs[r];
        if (q.x >= 0 && q.x < nacc && q.y >= 0 && q.y < nf) ++off[(size_t)q.x * nf + q.y + 1];
    }
    for (size_t k = 0; k < nkeys; ++k) off[k + 1] += off[k];
    std::vector<std::pair<int, float>> items(off[nkeys]);
    {
        std::vector<unsigned> pos(off.begin(), off.end() - 1);
        for (size_t r = 0; r < nrec; ++r) {
            const int4 q = job.recs[r];
            if (q.x < 0 || q.x >= nacc || q.y < 0 || q.y >= nf) continue;
            float v;
            std::memcpy(&v, &q.w, sizeof v);
            items[pos[(size_t)q.x * nf + q.y]++] = std::make_pair(q.z, v);
        }
    }
    // per-trial work in parallel when there is enough of it
    std::vector<std::vector<psx_candidate>> per(nacc);
    auto work = [&](int t_begin, int t_end) {
        std::vector<int> idx, pidx;
        std::vector<float> snr, psnr;
        std::vector<psx_candidate> tc;
        for (int t = t_begin; t < t_end; ++t) {
            tc.clear();
            for (int h = 0; h < nf; ++h) {
                const size_t k = (size_t)t * nf + h;
                auto b = items.begin() + off[k], e = items.begin() + off[k + 1];
                if (b == e) continue;
                std::sort(b, e, [](const std::pair<int, float>& x, const std::pair<int, float>& y) {
                    return x.first < y.first;
                });
                const size_t n = (size_t)(e - b);
                idx.resize(n);
                snr.resize(n);
                for (size_t i = 0; i < n; ++i) {
                    idx[i] = b[i].first;
                    snr[i] = b[i].second;
                }
                pidx.resize(n);
                psnr.resize(n);
                const size_t np = unique_peaks(idx.data(), snr.data(), n, cfg.min_gap, pidx.data(),
                                               psnr.data());
                for (size_t i = 0; i < np; ++i)
                    tc.push_back(psx_candidate{job.dm, job.dm_idx, job.accs[t], h, psnr[i],
                                               (float)pidx[i] * factor[h]});
            }
            if (tc.empty()) continue;
            const size_t keep = distill(PSX_DISTILL_HARMONIC, tc.data(), tc.size(), cfg.freq_tol,
                                        cfg.max_harm, tobs, 0, 1, nullptr);
            per[t].assign(tc.begin(), tc.begin() + keep);
        }
    };
    // trials in parallel once a DM has enough records to pay for waking the
    // pool (about 1 us per thread against ~0.1 us of host work per record)
    if (nrec > 1024 && nacc > 1 && nthreads > 1) {
        if (!pool) pool.reset(new WorkPool(nthreads - 1));
        std::atomic<int> next{0};
        const int chunk = std::max(1, nacc / (nthreads * 4));
        const std::function<void()> fn = [&] {
            for (;;) {
                const int b = next.fetch_add(chunk);
                if (b >= nacc) break;
                work(b, std::min(nacc, b + chunk));
            }
        };
        pool->run(fn);
    } else {
        work(0, nacc);
    }
    out.clear();
    nassoc.clear();
    trial_of.clear();
    for (int t = 0; t < nacc; ++t)
        for (const psx_candidate& c : per[t]) {
            out.push_back(c);
            trial_of.push_back(t);
        }
    if (output == PSX_OUT_DM_FOREST && !out.empty()) {
        // AccelerationDistiller(tobs, freq_tol, keep_related) keeping trees
        // (pipeline_multi.cu:149, 294): the trial survivors are leaves
        std::vector<int> ones(out.size(), 1);
        std::vector<psx_candidate> f(out.size() * 2);
        std::vector<int> fs(f.size());
        size_t nn = 0;
        int rc = psx_distill_forest(PSX_DISTILL_ACCEL, out.data(), ones.data(), out.size(),
                                    cfg.freq_tol, cfg.max_harm, tobs, 1, 1, f.data(), fs.data(),
                                    f.size(), &nn, nullptr);
        if (rc == PSX_ERR_OVERFLOW) {
            f.resize(nn);
            fs.resize(nn);
            rc = psx_distill_forest(PSX_DISTILL_ACCEL, out.data(), ones.data(), out.size(),
                                    cfg.freq_tol, cfg.max_harm, tobs, 1, 1, f.data(), fs.data(),
                                    f.size(), &nn, nullptr);
        }
        f.resize(nn);
        fs.resize(nn);
        trial_of.assign(nn, -1);
        for (size_t k = 0; k < nn; ++k) {
            auto it = std::lower_bound(job.accs.begin(), job.accs.end(), f[k].acc);
            if (it != job.accs.end() && *it == f[k].acc) trial_of[k] = (int)(it - job.accs.begin());
        }
        out.swap(f);
        nassoc.swap(fs);
    } else if (output == PSX_OUT_DM && !out.empty()) {
        std::vector<psx_candidate> c = out;
        nassoc.assign(c.size(), 0);
        const size_t keep = distill(PSX_DISTILL_ACCEL, c.data(), c.size(), cfg.freq_tol,
                                    cfg.max_harm, tobs, 1, 1, nassoc.data());
        c.resize(keep);
        nassoc.resize(keep);
        trial_of.assign(keep, -1);
        for (size_t k = 0; k < keep; ++k) {
            auto it = std::lower_bound(job.accs.begin(), job.accs.end(), c[k].acc);
            if (it != job.accs.end() && *it == c[k].acc) trial_of[k] = (int)(it - job.accs.begin());
        }
        out.swap(c);
    } else {
        nassoc.assign(out.size(), 0);
    }
}

int psx_search::finish(Slot& s, DmRecords& job)
{
    for (int attempt = 0; attempt < 3; ++attempt) {
        const auto t_wait = std::chrono::steady_clock::now();
        PSX_CUDA(cudaEventSynchronize(s.done));
        prof.host_wait_ms += ms_since(t_wait);
        const size_t hits = s.h_count[0];
        if (s.h_count[1] != 0) {
            set_error("search: harmonic-sum staging did not complete (status 0x%x)", s.h_count[1]);
            return PSX_ERR_CUDA;
        }
        const bool baseline_pending = !s.host_baseline && s.h_count[2] != 0;
        if (hits <= s.rec_cap && !baseline_pending) break;
        // Rare: more hits than the record slot holds, or a baseline that
        // needed more passes than the device loop makes.  Run the DM again
        // (after everything queued so far) with a larger slot / the host
        // loop; the result is as if it had run once.
        if (hits > s.rec_cap) PSX_TRY(grow_records(s, hits));
        if (baseline_pending) s.host_baseline = true;
        if (attempt == 2) {
            set_error("search: could not complete DM %d", s.dm_idx);
            return PSX_ERR_OVERFLOW;
        }
        PSX_TRY(enqueue(s, s.series, s.nsamps, s.on_device, s.dm, s.dm_idx));
    }
    const size_t nrec = s.h_count[0];
    info.baseline_passes = s.host_baseline ? -1 : (int)s.h_count[3];
    s.host_baseline = false;
    if (nrec) {
        PSX_CUDA(cudaStreamWaitEvent(cst, s.done, 0));
        PSX_CUDA(cudaMemcpyAsync(s.h_rec, s.d_rec, sizeof(int4) * nrec, cudaMemcpyDeviceToHost, cst));
        PSX_CUDA(cudaEventRecord(s.copied, cst));
        PSX_CUDA(cudaEventSynchronize(s.copied));
    }
    read_profile(s);
    info.ntrials += (int)s.accs.size();
    info.nbatches += s.groups;
    info.kernel_launches += s.launches;
    info.fft_launches += s.ffts;
    info.above_threshold += (long long)nrec;
    job.recs.assign(s.h_rec, s.h_rec + nrec);
    job.accs = s.accs;
    job.dm = s.dm;
    job.dm_idx = s.dm_idx;
    return PSX_OK;
}

extern "C" {

void psx_search_config_defaults(psx_search_config* c, size_t fft_size, float tsamp)
{
    if (!c) return;
    std::memset(c, 0, sizeof *c);
    c->fft_size = fft_size;
    c->tsamp = tsamp;
    c->cdm = 0.0f;
    c->acc_lo = 0.0f;
    c->acc_hi = 0.0f;
    c->acc_tol = 1.10f;
    c->acc_pulse_width = 64e-6f;
    c->cfreq_hz = 1475.12e6f;
    c->ch_bw_hz = 1.09e6f;
    c->nharmonics = 4;
    c->min_snr = 9.0f;
    c->min_freq = 0.1f;
    c->max_freq = 1100.0f;
    c->min_gap = 30;
    c->freq_tol = 0.0001f;
    c->max_harm = 16.0f;
    c->boundary_5_freq = 0.05f;
    c->boundary_25_freq = 0.5f;
    c->mode = PSX_MODE_BATCHED;
    c->batch = 0;
    c->use_fft_callback = 0;
    c->use_graph = 1;
    c->harm_shape = 0;
    c->lanes = 0;
    c->fft_form = 0;
}

static int effective_batch(const psx_search_config* c);

static int check_config(const psx_search_config* c)
{
    if (!c) {
        set_error("search: null config");
        return PSX_ERR_INVALID;
    }
    if (!fft_size_supported(c->fft_size) || c->fft_size < 1024 || c->fft_size > ((size_t)1 << 28)) {
        set_error("search: fft_size %zu must be 2^k or 3*2^k within [1024, 2^28]", c->fft_size);
        return PSX_ERR_INVALID;
    }
    if (!(c->tsamp > 0.f)) {
        set_error("search: tsamp must be positive");
        return PSX_ERR_INVALID;
    }
    if (c->nharmonics < 0 || c->nharmonics > 5) {
        set_error("search: nharmonics must be 0..5 (the reference sums at most 5 folds)");
        return PSX_ERR_INVALID;
    }
    if (c->mode != PSX_MODE_PLAIN && c->mode != PSX_MODE_BATCHED) {
        set_error("search: unknown mode %d", c->mode);
        return PSX_ERR_INVALID;
    }
    if (c->use_fft_callback) {
        set_error("search: the resample inside cuFFT (use_fft_callback) is not available: cuFFT "
                  "11.4 of CUDA 12.9 cannot plan LTO load callbacks on sm_100; the two-pass "
                  "transform (fft_form 3) gathers the resampled series in its first pass");
        return PSX_ERR_UNSUPPORTED;
    }
    if (c->batch < 0 || c->batch > 1024) {
        set_error("search: batch must be 0..1024");
        return PSX_ERR_INVALID;
    }
    if (c->fft_form < 0 || c->fft_form > 3) {
        set_error("search: fft_form must be 0..3");
        return PSX_ERR_INVALID;
    }
    if (c->fft_form == 3 && (c->mode != PSX_MODE_BATCHED || !Fft4Plan::supported(c->fft_size))) {
        set_error("search: fft_form 3 needs the batched mode and "
                  "fft_size 2^19 .. 2^27 or 3 * 2^17 .. 3 * 2^23");
        return PSX_ERR_INVALID;
    }
    if (c->lanes < 0 || c->lanes > 2) {
        set_error("search: lanes must be 0..2");
        return PSX_ERR_INVALID;
    }
    if (c->group_dms < 0 || c->group_dms > kGroupRowsMax) {
        set_error("search: group_dms must be 0..%d", kGroupRowsMax);
        return PSX_ERR_INVALID;
    }
    if (c->harm_shape < 0 || c->harm_shape > PSX_HARM_SHAPES) {
        set_error("search: harm_shape must be 0..%d", PSX_HARM_SHAPES);
        return PSX_ERR_INVALID;
    }
    if (c->harm_shape > 0 && kHarmShapes[c->harm_shape - 1].rows > 0 &&
        (c->mode != PSX_MODE_BATCHED || effective_batch(c) < kHarmShapes[c->harm_shape - 1].rows)) {
        set_error("search: harm_shape %d stages %d trials per tile and needs the batched mode "
                  "with at least that many trials per launch group",
                  c->harm_shape, kHarmShapes[c->harm_shape - 1].rows);
        return PSX_ERR_INVALID;
    }
    if (c->nbirdies && (!c->birdie_freqs || !c->birdie_widths)) {
        set_error("search: birdie arrays missing");
        return PSX_ERR_INVALID;
    }
    if (c->acc_hi < c->acc_lo) {
        set_error("search: acc_hi < acc_lo");
        return PSX_ERR_INVALID;
    }
    return PSX_OK;
}

static int effective_form(const psx_search_config* c);

// Trials per launch group: the configured count (or the default), rounded
// down to a power of two where cuFFT plans carry the trials (they exist for
// powers of two only); the two-pass transform takes any count.
static int effective_batch(const psx_search_config* c)
{
    if (c->mode != PSX_MODE_BATCHED) return 1;
    int b = c->batch ? c->batch : default_batch(c->fft_size);
    if (effective_form(c) == 3) return b;
    int p = 1;
    while (p * 2 <= b) p *= 2;
    return p;
}

// Transform path of the trials: 3 = the hand-written two-pass transform,
// 1 = cuFFT's complex transform + the fused unpack kernel, 2 = the
// reference's real transform (also plain mode).
static int effective_form(const psx_search_config* c)
{
    if (c->mode != PSX_MODE_BATCHED || c->fft_form == 2) return 2;
    if (c->fft_form == 3 || (c->fft_form == 0 && Fft4Plan::supported(c->fft_size))) return 3;
    return 1;
}

static int effective_lanes(const psx_search_config* c)
{
    if (c->mode != PSX_MODE_BATCHED) return 1;
    // one lane by default: measured on B200 at 2^23, a second lane did not
    // raise throughput (the persistent harmonic grid already fills every SM)
    return c->lanes ? c->lanes : 1;
}

size_t psx_search_footprint(const psx_search_config* c)
{
    if (check_config(c) != PSX_OK) return 0;
    const size_t N = c->fft_size, B = N / 2 + 1, Bp = round_up(B, 64);
    const size_t b = (size_t)effective_batch(c);
    const size_t L = (size_t)effective_lanes(c);
    size_t bytes = 0;
    bytes += 2 * sizeof(float) * (N + 2 * Bp);        // per slot: series, prologue spectrum
    bytes += 2 * median_scratch_bytes(B);
    bytes += L * sizeof(float) * N * b;               // resampled series, per lane
    bytes += L * sizeof(float) * 2 * Bp * b;          // complex spectra, per lane
    bytes += L * sizeof(float) * Bp * b;              // normalised spectra, per lane
    bytes += 2 * sizeof(int4) * ((size_t)1 << 20);    // two initial record slots
    // cuFFT work areas: about one transform's worth per batched plan size and
    // lane (none with the two-pass transform, which has twiddle tables
    // instead), plus the batch-1 plans of the two slots' prologues and the
    // plain path
    if (effective_form(c) == 3)
        bytes += sizeof(float) * 2 * Bp * 6 + sizeof(float2) * Fft4Plan::table_floats2(N);
    else
        bytes += sizeof(float) * 2 * Bp * (2 * b * L + 6);
    // two group sets of G rows (made with the instance): series,
    // prologue spectra, median scratch, each slot's first record buffer, and
    // about one batch's worth of transform work area per batch-G plan
    const size_t G = (size_t)group_rows_for(c);
    if (G >= 2)
        bytes += 2 * G *
                     (sizeof(float) * (N + 2 * Bp) + median_scratch_bytes(B) +
                      sizeof(int4) * ((size_t)1 << 18) + 2 * sizeof(float) * 2 * Bp) +
                 // the spanning schedule's first record buffer per set
                 (effective_form(c) == 3 ? 2 * sizeof(int4) * ((size_t)1 << 20) : 0);
    return bytes;
}

// Host-side state of an instance derived from its configuration: the
// birdie list, transform sizes, tobs and bin width (floats, as at
// pipeline_multi.cu:126-128), the search ranges of every fold
// (peakfinder.hpp:78-83) and the fast-pass vote level.  Shared by
// psx_search_create and psx_search_retarget.
static void host_setup(psx_search* s, const psx_search_config* cfg)
{
    s->cfg = *cfg;
    s->bf.clear();
    s->bw.clear();
    if (cfg->nbirdies) {
        s->bf.assign(cfg->birdie_freqs, cfg->birdie_freqs + cfg->nbirdies);
        s->bw.assign(cfg->birdie_widths, cfg->birdie_widths + cfg->nbirdies);
    }
    s->cfg.birdie_freqs = nullptr;
    s->cfg.birdie_widths = nullptr;
    s->N = cfg->fft_size;
    s->B = s->N / 2 + 1;
    s->Bp = round_up(s->B, 64);
    s->F = cfg->nharmonics;
    s->batch = effective_batch(cfg);
    s->lanes = effective_lanes(cfg);
    s->harm_shape = cfg->harm_shape ? cfg->harm_shape : kHarmDefaultShape;
    s->use_f4 = effective_form(cfg) == 3;
    {
        const double M = (double)(s->N / 2), pi = 3.14159265358979323846;
        for (int t = 0; t < 6; ++t)
            s->tw_steps.w[t] = make_float2((float)std::cos(pi * (t - 1) / M),
                                           (float)std::sin(pi * (t - 1) / M));
    }
    unsigned hc = std::thread::hardware_concurrency();
    s->nthreads = (int)std::max(1u, std::min(8u, hc ? hc : 1u));
    // pipeline_multi.cu:126-128: tobs and bin width are floats
    s->tobs = (float)s->N * cfg->tsamp;
    s->bin_width_f = (float)(1.0 / (double)s->tobs);
    s->bin_width = (double)s->bin_width_f;
    // search ranges of every fold (peakfinder.hpp:78-83)
    unsigned lo = 0xffffffffu, hi = 0;
    for (int h = 0; h <= 5; ++h) {
        int st, en;
        float fac;
        peak_range((unsigned)s->B, s->bin_width, h, cfg->min_freq, cfg->max_freq, &st, &en, &fac);
        if (st < 0) st = 0;
        if (en > (int)s->B) en = (int)s->B;
        if (h > s->F) {
            st = 0;
            en = 0;
        }
        s->pk.start[h] = st;
        s->pk.end[h] = en;
        s->factor[h] = fac;
        if (en > st) {
            lo = std::min(lo, (unsigned)st);
            hi = std::max(hi, (unsigned)en);
        }
    }
    s->pk.lo = hi > lo ? (lo & ~127u) : 0;
    s->pk.hi = hi > lo ? hi : 0;
    s->pk.thresh = cfg->min_snr;
    s->pk.vote = cfg->min_snr - std::fabs(cfg->min_snr) * 0x1p-20f;
    s->pk.wait_limit = kHarmWaitLimit;
    s->pk.flags = 0;
}

int psx_search_create(const psx_search_config* cfg, psx_search** out)
{
    clear_error();
    if (!out) return PSX_ERR_INVALID;
    *out = nullptr;
    PSX_TRY(check_config(cfg));
    psx_search* s = new (std::nothrow) psx_search;
    if (!s) return PSX_ERR_ALLOC;
    host_setup(s, cfg);

    int rc = PSX_OK;
    auto fail = [&](int code) {
        delete s;
        return code;
    };
    if ((rc = cuda_status(cudaGetDevice(&s->device), "cudaGetDevice")) != PSX_OK) return fail(rc);
    if ((rc = configure_harm(s->F)) != PSX_OK) return fail(rc);
    if ((rc = cuda_status(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking),
                          "cudaStreamCreate")) != PSX_OK)
        return fail(rc);
    s->own_stream = true;
    if ((rc = cuda_status(cudaStreamCreateWithFlags(&s->cst, cudaStreamNonBlocking),
                          "cudaStreamCreate")) != PSX_OK)
        return fail(rc);
    const size_t N = s->N, Bp = s->Bp;
    const size_t b = (size_t)s->batch;
    const int nb = reduction_blocks();
#define ALLOC(ptr, bytes)                                                        \
    if ((rc = cuda_status(cudaMalloc((void**)&(ptr), (bytes)), "cudaMalloc")) != \
        PSX_OK)                                                                  \
        return fail(rc == PSX_ERR_CUDA ? PSX_ERR_ALLOC : rc);
    for (int l = 0; l < s->lanes; ++l) {
        ALLOC(s->d_trl[l], sizeof(float) * N * b);
        ALLOC(s->d_Xl[l], sizeof(float) * 2 * Bp * b);
        ALLOC(s->d_pl[l], sizeof(float) * Bp * b);
    }
    s->d_tr = s->d_trl[0];
    s->d_X = s->d_Xl[0];
    s->d_p = s->d_pl[0];
    if (kHarmShapes[s->harm_shape - 1].rows > 0)
        for (int l = 0; l < s->lanes; ++l)
            if ((rc = encode_harm_maps(s->d_pl[l], Bp, (int)b, kHarmShapes[s->harm_shape - 1].rows,
                                       &s->hmaps[l])) != PSX_OK)
                return fail(rc);
    for (Slot& sl : s->slot) {
        ALLOC(sl.d_count, sizeof(unsigned) * 16);
        ALLOC(sl.d_tim, sizeof(float) * N);
        ALLOC(sl.d_Xp, sizeof(float) * 2 * Bp);
        ALLOC(sl.d_med, median_scratch_bytes(s->B));
        ALLOC(sl.d_part, sizeof(double2) * 2 * nb);  // two halves: baseline passes alternate
        ALLOC(sl.d_sums, sizeof(double) * 2);
        ALLOC(sl.d_stat, sizeof(float) * 8);
        ALLOC(sl.d_mean, sizeof(float) * 2);
    }
    if (!s->bf.empty()) {
        ALLOC(s->d_bf, sizeof(float) * s->bf.size());
        ALLOC(s->d_bw, sizeof(float) * s->bw.size());
        s->bird_cap = s->bf.size();
    }
#undef ALLOC
    if (cudaMallocHost(&s->h_mean, sizeof(float) * 4) != cudaSuccess) return fail(PSX_ERR_ALLOC);
    for (Slot& sl : s->slot) {
        if (cudaMallocHost(&sl.h_count, sizeof(unsigned) * 4) != cudaSuccess)
            return fail(PSX_ERR_ALLOC);
        if (cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&sl.copied, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&sl.ready, cudaEventDisableTiming) != cudaSuccess)
            return fail(PSX_ERR_CUDA);
        if ((rc = cuda_status(cudaStreamCreateWithFlags(&sl.pst, cudaStreamNonBlocking),
                              "cudaStreamCreate")) != PSX_OK)
            return fail(rc);
        sl.r2c = new (std::nothrow) FftPlan;
        sl.c2r = new (std::nothrow) FftPlan;
        if (!sl.r2c || !sl.c2r) return fail(PSX_ERR_ALLOC);
        if ((rc = sl.r2c->create(N, 1, PSX_FFT_R2C, 0, 0)) != PSX_OK) return fail(rc);
        if ((rc = sl.c2r->create(N, 1, PSX_FFT_C2R, 0, 0)) != PSX_OK) return fail(rc);
        if ((rc = s->grow_records(sl, (size_t)1 << 20)) != PSX_OK) return fail(rc);
        if ((rc = s->grow_ktab(sl, 1024)) != PSX_OK) return fail(rc);
    }
    if (!s->bf.empty()) {
        cudaMemcpy(s->d_bf, s->bf.data(), sizeof(float) * s->bf.size(), cudaMemcpyHostToDevice);
        cudaMemcpy(s->d_bw, s->bw.data(), sizeof(float) * s->bw.size(), cudaMemcpyHostToDevice);
    }
    // zero the padded tails once so no uninitialised memory is ever read
    for (int l = 0; l < s->lanes; ++l) {
        cudaMemsetAsync(s->d_Xl[l], 0, sizeof(float) * 2 * Bp * b, s->st);
        cudaMemsetAsync(s->d_pl[l], 0, sizeof(float) * Bp * b, s->st);
    }
    if (s->lanes > 1) {
        if ((rc = cuda_status(cudaStreamCreateWithFlags(&s->st2, cudaStreamNonBlocking),
                              "cudaStreamCreate")) != PSX_OK)
            return fail(rc);
        if (cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming) != cudaSuccess)
            return fail(PSX_ERR_CUDA);
    }
    for (Slot& sl : s->slot) {
        cudaMemsetAsync(sl.d_Xp, 0, sizeof(float) * 2 * Bp, s->st);
    }
    if (cudaEventCreateWithFlags(&s->call_start, cudaEventDisableTiming) != cudaSuccess)
        return fail(PSX_ERR_CUDA);
    if ((rc = s->r2c1.create(N, 1, PSX_FFT_R2C, 0, 0)) != PSX_OK) return fail(rc);
    if (s->fft4()) {
        if ((rc = s->f4.create(N)) != PSX_OK) return fail(rc);
    } else if (s->batched()) {
        FftPlan* p = nullptr;
        for (int l = 0; l < s->lanes; ++l)
            if ((rc = s->get_plan(s->batch, &p, l)) != PSX_OK) return fail(rc);
    }
    if ((rc = cuda_status(cudaStreamSynchronize(s->st), "search create")) != PSX_OK)
        return fail(rc);
    s->info.batch = s->batch;
    s->info.harm_shape = s->harm_shape;
    s->info.fft_callback = 0;
    s->info.fft_form = effective_form(cfg);
    s->set_st[0] = s->st;
    s->set_st2[0] = s->st2;
    for (int k = 0; k < 2; ++k) s->set_pst[0][k] = s->slot[k].pst;
    // group sets made now (their bytes are in the footprint), so a call
    // that groups does not pay for them on first use
    if ((rc = s->alloc_groups()) != PSX_OK) return fail(rc);
    *out = s;
    return PSX_OK;
}

int psx_search_destroy(psx_search* s)
{
    clear_error();
    if (!s) return PSX_OK;
    delete s;
    return PSX_OK;
}

int psx_harmonic_peaks(const float* d_spec, size_t pitch, size_t nbins, int rows, int nharms,
                       const int* h_start, const int* h_end, float thresh, int* d_records,
                       size_t cap, size_t* h_count, unsigned wait_limit, unsigned flags,
                       psx_stream_t stream)
{
    clear_error();
    if (!d_spec || !h_start || !h_end || !h_count || rows < 1 || nharms < 0 || nharms > 5 ||
        nbins == 0 || nbins > 0x7fffffffu || pitch < nbins || (cap && !d_records) ||
        (pitch & 3u) || (reinterpret_cast<uintptr_t>(d_spec) & 15u)) {
        set_error("harmonic_peaks: bad arguments (nharms 0..5, pitch >= nbins and a multiple of "
                  "4, spectra 16-byte aligned)");
        return PSX_ERR_INVALID;
    }
    *h_count = 0;
    PeakParams pk{};
    unsigned lo = 0xffffffffu, hi = 0;
    for (int h = 0; h <= 5; ++h) {
        int st = h <= nharms ? std::max(0, h_start[h]) : 0;
        int en = h <= nharms ? std::min((int)nbins, h_end[h]) : 0;
        if (en < st) en = st;
        pk.start[h] = st;
        pk.end[h] = en;
        if (en > st) {
            lo = std::min(lo, (unsigned)st);
            hi = std::max(hi, (unsigned)en);
        }
    }
    if (hi <= lo) return PSX_OK;  // empty search ranges
    pk.lo = lo & ~127u;
    pk.hi = hi;
    pk.thresh = thresh;
    pk.vote = thresh - std::fabs(thresh) * 0x1p-20f;
    pk.wait_limit = wait_limit ? wait_limit : kHarmWaitLimit;
    pk.flags = flags;
    cudaStream_t cs_ = cs(stream);
    PSX_TRY(configure_harm(nharms));
    unsigned* d_counter = nullptr;
    PSX_CUDA(cudaMallocAsync((void**)&d_counter, sizeof(unsigned) * 2, cs_));
    int rc = cuda_status(cudaMemsetAsync(d_counter, 0, sizeof(unsigned) * 2, cs_), "memset");
    if (rc == PSX_OK)
        rc = launch_harm(nharms, kHarmDefaultShape, d_spec, pitch, (unsigned)nbins, pk, 0, rows,
                         reinterpret_cast<int4*>(d_records), d_counter, (unsigned)cap, cs_);
    unsigned hcnt[2] = {0, 0};
    if (rc == PSX_OK)
        rc = cuda_status(cudaMemcpyAsync(hcnt, d_counter, sizeof hcnt, cudaMemcpyDeviceToHost, cs_),
                         "harmonic_peaks copy");
    cudaFreeAsync(d_counter, cs_);
    if (rc == PSX_OK) rc = cuda_status(cudaStreamSynchronize(cs_), "harmonic_peaks");
    if (rc != PSX_OK) return rc;
    if (hcnt[1] != 0) {
        set_error("harmonic_peaks: a staging wait ran out after %u polls (status 0x%x)",
                  pk.wait_limit, hcnt[1]);
        return PSX_ERR_CUDA;
    }
    *h_count = hcnt[0];
    if (hcnt[0] > cap) {
        set_error("harmonic_peaks: %u hits, buffer holds %zu", hcnt[0], cap);
        return PSX_ERR_OVERFLOW;
    }
    return PSX_OK;
}

int psx_search_retarget(psx_search* s, const psx_search_config* cfg)
{
    clear_error();
    if (!s) {
        set_error("search_retarget: null instance");
        return PSX_ERR_INVALID;
    }
    PSX_TRY(check_config(cfg));
    const int shape = cfg->harm_shape ? cfg->harm_shape : kHarmDefaultShape;
    if (cfg->fft_size != s->N || cfg->mode != s->cfg.mode ||
        effective_batch(cfg) != s->batch || shape != s->harm_shape ||
        effective_lanes(cfg) != s->lanes ||
        effective_form(cfg) != effective_form(&s->cfg) ||
        group_rows_for(cfg) != group_rows_for(&s->cfg)) {
        set_error("search_retarget: fft_size, mode, batch, harmonic shape, lanes, "
                  "transform path and prologue grouping must match the instance");
        return PSX_ERR_INVALID;
    }
    PSX_CUDA(cudaSetDevice(s->device));
    // work queued with the old parameters finishes first
    PSX_CUDA(cudaStreamSynchronize(s->st));
    PSX_CUDA(cudaStreamSynchronize(s->cst));
    for (Slot& sl : s->slot) PSX_CUDA(cudaStreamSynchronize(sl.pst));
    // the fold count only selects the harmonic kernel's instantiation (no
    // buffer depends on it): opt that one into its shared memory
    PSX_TRY(configure_harm(cfg->nharmonics));
    host_setup(s, cfg);
    if (s->bf.size() > s->bird_cap) {
        cudaFree(s->d_bf);
        cudaFree(s->d_bw);
        s->d_bf = s->d_bw = nullptr;
        s->bird_cap = 0;
        PSX_CUDA(cudaMalloc((void**)&s->d_bf, sizeof(float) * s->bf.size()));
        PSX_CUDA(cudaMalloc((void**)&s->d_bw, sizeof(float) * s->bw.size()));
        s->bird_cap = s->bf.size();
    }
    if (!s->bf.empty()) {
        PSX_CUDA(cudaMemcpy(s->d_bf, s->bf.data(), sizeof(float) * s->bf.size(),
                            cudaMemcpyHostToDevice));
        PSX_CUDA(cudaMemcpy(s->d_bw, s->bw.data(), sizeof(float) * s->bw.size(),
                            cudaMemcpyHostToDevice));
    }
    // captured schedules hold the old search ranges by value
    s->drop_graphs();
    return PSX_OK;
}

int psx_search_set_stream(psx_search* s, psx_stream_t stream)
{
    clear_error();
    if (!s) return PSX_ERR_INVALID;
    // the creation streams first (priorities apply to owned streams only)
    s->prio_want.store(0);
    PSX_TRY(s->apply_priority());
    PSX_CUDA(cudaStreamSynchronize(s->st));
    if (s->own_stream) cudaStreamDestroy(s->st);
    s->own_stream = false;
    s->st = cs(stream);
    s->set_st[0] = s->st;
    return PSX_OK;
}

int psx_search_set_priority(psx_search* s, int high)
{
    if (!s) return PSX_ERR_INVALID;
    s->prio_want.store(high ? 1 : 0, std::memory_order_relaxed);
    return PSX_OK;
}

int psx_search_set_profile(psx_search* s, int on)
{
    if (!s) return PSX_ERR_INVALID;
    s->profile = on != 0;
    return PSX_OK;
}

int psx_search_get_profile(psx_search* s, psx_search_profile* out, int reset)
{
    if (!s || !out) return PSX_ERR_INVALID;
    *out = s->prof;
    if (reset) s->prof = psx_search_profile{};
    return PSX_OK;
}

int psx_search_block(psx_search* s, const float* const* series, size_t nsamps,
                     int series_on_device, const float* dms, const int* dm_idx, int ndm,
                     int output, psx_candidate* h_out, int* h_nassoc, int* h_trial, int* h_dm,
                     size_t cap, size_t* n_out)
{
    clear_error();
    if (!s || !series || !dms || !n_out || ndm <= 0 || nsamps == 0 ||
        (output != PSX_OUT_TRIAL && output != PSX_OUT_DM && output != PSX_OUT_DM_FOREST)) {
        set_error("search: bad arguments");
        return PSX_ERR_INVALID;
    }
    for (int d = 0; d < ndm; ++d)
        if (!series[d]) {
            set_error("search: null series %d", d);
            return PSX_ERR_INVALID;
        }
    *n_out = 0;
    PSX_CUDA(cudaSetDevice(s->device));
    const int bp = s->info.batch, cbk = s->info.fft_callback;
    s->info = psx_search_info{};
    s->info.batch = bp;
    s->info.fft_callback = cbk;
    s->info.harm_shape = s->harm_shape;
    s->info.fft_form = effective_form(&s->cfg);
    s->info.graph = s->batched() && s->cfg.use_graph && !s->profile ? 1 : 0;
    // prologues wait for the caller's work queued on the compute stream so far
    PSX_CUDA(cudaEventRecord(s->call_start, s->st));
    std::vector<psx_candidate> all;
    std::vector<int> all_na, all_tr, all_dm;
    // DM d's records are distilled (collect) on a collector thread while
    // this thread queues DM d+2: with few acceleration trials per DM trial
    // the host's distillation would otherwise leave the device idle.  Jobs
    // are taken in DM order, so the output order is that of the loop.
    std::mutex jmu;
    std::condition_variable jcv;
    std::deque<std::pair<int, psx_search::DmRecords>> jobs;
    bool jobs_closed = false;
    auto take = [&](int d, psx_search::DmRecords& job) {
        std::vector<psx_candidate> out;
        std::vector<int> na, tr;
        const auto t0 = std::chrono::steady_clock::now();
        s->collect(job, output, out, na, tr);
        s->prof.host_collect_ms += ms_since(t0);
        all.insert(all.end(), out.begin(), out.end());
        all_na.insert(all_na.end(), na.begin(), na.end());
        all_tr.insert(all_tr.end(), tr.begin(), tr.end());
        all_dm.insert(all_dm.end(), out.size(), d);
    };
    std::thread collector;
    if (ndm > 1)
        collector = std::thread([&] {
            for (;;) {
                std::pair<int, psx_search::DmRecords> j;
                {
                    std::unique_lock<std::mutex> lock(jmu);
                    jcv.wait(lock, [&] { return jobs_closed || !jobs.empty(); });
                    if (jobs.empty()) return;
                    j = std::move(jobs.front());
                    jobs.pop_front();
                }
                take(j.first, j.second);
            }
        });
    // (no early return from here until the collector is joined)
    auto push_job = [&](int d, psx_search::DmRecords& job) {
        if (ndm == 1) {
            take(d, job);
        } else {
            std::lock_guard<std::mutex> lock(jmu);
            jobs.emplace_back(d, std::move(job));
            jcv.notify_one();
        }
    };
    auto finish_dm = [&](int d, Slot& sl) -> int {
        s->last_dm = &sl;
        psx_search::DmRecords job;
        const int r = s->finish(sl, job);
        if (r != PSX_OK) return r;
        push_job(d, job);
        return PSX_OK;
    };
    const bool on_dev = series_on_device != 0;
    const int G = s->group_rows_for_call(dms, ndm);
    int rc = PSX_OK;
    if (G) {
        // Grouped prologues: chunks of G DM trials alternate between the two
        // group sets; chunk c + 1's batched prologue (on slot (c + 1) & 1's
        // stream) runs while chunk c's trials run, as the per-DM slots do.
        // With the two-pass transform the chunk's trials also run as one
        // list, in launch groups across its DM trials (trials_span).
        rc = s->alloc_groups();
        const int nchunks = (ndm + G - 1) / G;
        const bool spanning = s->span_mode();
        auto enqueue_chunk = [&](int c) -> int {
            const auto t_host = std::chrono::steady_clock::now();
            GroupSet& g = s->gset[c & 1];
            const int d0 = c * G, cnt = std::min(G, ndm - d0);
            PSX_TRY(s->apply_priority());
            for (int i = 0; i < cnt; ++i)
                PSX_TRY(s->prep(g.slots[i], series[d0 + i], nsamps, on_dev, dms[d0 + i],
                                dm_idx ? dm_idx[d0 + i] : d0 + i));
            PSX_TRY(s->prologue_group(g, cnt, s->slot[c & 1].pst));
            if (spanning) {
                g.off.assign((size_t)cnt + 1, 0);
                for (int i = 0; i < cnt; ++i) g.off[i + 1] = g.off[i] + (int)g.slots[i].accs.size();
                PSX_TRY(s->grow_span_tables(g, (size_t)g.off[cnt]));
                for (int i = 0; i < cnt; ++i)
                    for (int t = g.off[i]; t < g.off[i + 1]; ++t) {
                        g.h_ktab[t] = g.slots[i].h_ktab[t - g.off[i]];
                        g.h_trow[t] = (unsigned)i;
                    }
                PSX_TRY(s->trials_span(g, cnt));
            } else {
                for (int i = 0; i < cnt; ++i) PSX_TRY(s->enqueue_trials(g.slots[i]));
            }
            s->prof.host_enqueue_ms += ms_since(t_host);
            return PSX_OK;
        };
        if (rc == PSX_OK) rc = enqueue_chunk(0);
        for (int c = 0; c < nchunks && rc == PSX_OK; ++c) {
            if (c + 1 < nchunks) rc = enqueue_chunk(c + 1);
            const int d0 = c * G, cnt = std::min(G, ndm - d0);
            if (spanning && rc == PSX_OK) {
                std::vector<psx_search::DmRecords> cj;
                rc = s->finish_span(s->gset[c & 1], cnt, cj);
                for (int i = 0; i < cnt && rc == PSX_OK; ++i) push_job(d0 + i, cj[i]);
            } else {
                for (int i = 0; i < cnt && rc == PSX_OK; ++i)
                    rc = finish_dm(d0 + i, s->gset[c & 1].slots[i]);
            }
        }
        s->info.group_dms = G;
    } else {
        rc = s->enqueue(s->slot[0], series[0], nsamps, on_dev, dms[0], dm_idx ? dm_idx[0] : 0);
        for (int d = 0; d < ndm && rc == PSX_OK; ++d) {
            if (d + 1 < ndm)
                rc = s->enqueue(s->slot[(d + 1) & 1], series[d + 1], nsamps, on_dev, dms[d + 1],
                                dm_idx ? dm_idx[d + 1] : d + 1);
            if (rc == PSX_OK) rc = finish_dm(d, s->slot[d & 1]);
        }
    }
    if (collector.joinable()) {
        {
            std::lock_guard<std::mutex> lock(jmu);
            jobs_closed = true;
            if (rc != PSX_OK) jobs.clear();
        }
        jcv.notify_one();
        collector.join();
    }
    if (rc != PSX_OK) {
        cudaStreamSynchronize(s->st);
        cudaStreamSynchronize(s->cst);
        return rc;
    }
    *n_out = all.size();
    if (all.size() > cap || (!h_out && !all.empty())) {
        set_error("search: %zu candidates, buffer holds %zu", all.size(), cap);
        return PSX_ERR_OVERFLOW;
    }
    if (!all.empty()) std::memcpy(h_out, all.data(), sizeof(psx_candidate) * all.size());
    for (size_t k = 0; k < all.size(); ++k) {
        if (h_nassoc) h_nassoc[k] = all_na[k];
        if (h_trial) h_trial[k] = all_tr[k];
        if (h_dm) h_dm[k] = all_dm[k];
    }
    return PSX_OK;
}

int psx_search_dm(psx_search* s, const float* series, size_t nsamps, int series_on_device,
                  float dm, int dm_idx, int output, psx_candidate* h_out, int* h_nassoc,
                  int* h_trial, size_t cap, size_t* n_out)
{
    const float* one[1] = {series};
    return psx_search_block(s, one, nsamps, series_on_device, &dm, &dm_idx, 1, output, h_out,
                            h_nassoc, h_trial, nullptr, cap, n_out);
}

int psx_search_last_info(const psx_search* s, psx_search_info* info)
{
    if (!s || !info) return PSX_ERR_INVALID;
    *info = s->info;
    return PSX_OK;
}

int psx_search_debug_tap(psx_search* s, int trial, float* h_tim_dered, float* h_tim_r,
                         float* h_pspec, float* h_norm2)
{
    clear_error();
    if (!s) return PSX_ERR_INVALID;
    // the dereddened series on the device is the last DM's
    Slot& sl = s->last_dm ? *s->last_dm : s->slot[0];
    const std::vector<float>& accs = sl.accs;
    if (h_tim_dered)
        PSX_CUDA(cudaMemcpyAsync(h_tim_dered, sl.d_tim, sizeof(float) * s->N,
                                 cudaMemcpyDeviceToHost, s->st));
    if (h_norm2)
        PSX_CUDA(cudaMemcpyAsync(h_norm2, sl.d_stat + 3, sizeof(float) * 2, cudaMemcpyDeviceToHost,
                                 s->st));
    if (h_tim_r || h_pspec) {
        if (trial < 0 || trial >= (int)accs.size()) {
            set_error("debug_tap: trial %d out of range", trial);
            return PSX_ERR_INVALID;
        }
        if (s->fft4())  // what the trials' own pass 1 gathers
            PSX_TRY(s->f4.dump_gather(sl.d_tim, sl.d_ktab + trial, s->d_tr, s->st));
        else
            PSX_TRY(launch_resample(sl.d_tim, s->d_tr, s->N, nullptr,
                                    accel_fact(accs[trial], s->cfg.tsamp), 1, s->N, false,
                                    s->st));
        if (h_tim_r)
            PSX_CUDA(cudaMemcpyAsync(h_tim_r, s->d_tr, sizeof(float) * s->N,
                                     cudaMemcpyDeviceToHost, s->st));
        if (h_pspec && s->fft4()) {
            // the trials' own path: gather + two-pass transform + unpack
            PSX_TRY(s->f4.exec(sl.d_tim, sl.d_ktab + trial, 1, reinterpret_cast<float2*>(s->d_tr),
                               s->N / 2, reinterpret_cast<float2*>(s->d_X), s->Bp, s->st));
            PSX_TRY(s->f4.form(reinterpret_cast<const float2*>(s->d_X), s->Bp, 1, s->d_p, s->Bp,
                               sl.d_stat, s->st));
            PSX_CUDA(cudaMemcpyAsync(h_pspec, s->d_p, sizeof(float) * s->B,
                                     cudaMemcpyDeviceToHost, s->st));
        } else if (h_pspec && s->fused_form()) {
            // the trials' own path: complex transform + fused unpack
            FftPlan* plan = nullptr;
            PSX_TRY(s->get_plan(1, &plan, 0));
            PSX_TRY(plan->exec(s->d_tr, s->d_X, s->st));
            const unsigned M = (unsigned)(s->N / 2);
            dim3 gu(grid_for(M / 8, 256, 4), 1);
            k_unpack_form_norm<<<gu, 256, 0, s->st>>>(s->d_X, s->Bp, s->d_p, s->Bp, M,
                                                      1.0f / (float)M, s->tw_steps, sl.d_stat);
            PSX_TRY(launch_status("debug tap"));
            PSX_CUDA(cudaMemcpyAsync(h_pspec, s->d_p, sizeof(float) * s->B,
                                     cudaMemcpyDeviceToHost, s->st));
        } else if (h_pspec) {
            PSX_TRY(s->r2c1.exec(s->d_tr, s->d_X, s->st));
            dim3 gf(grid_for(s->B / 2 + 1, 256, 4), 1);
            k_form_norm<<<gf, 256, 0, s->st>>>(s->d_X, 2 * s->Bp, s->d_p, s->Bp, (unsigned)s->B,
                                               sl.d_stat);
            PSX_TRY(launch_status("debug tap"));
            PSX_CUDA(cudaMemcpyAsync(h_pspec, s->d_p, sizeof(float) * s->B,
                                     cudaMemcpyDeviceToHost, s->st));
        }
    }
    return cuda_status(cudaStreamSynchronize(s->st), "debug tap");
}

}  // extern "C"
