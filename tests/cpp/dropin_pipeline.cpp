// dropin_pipeline.cpp -- one DM trial searched through the C++ drop-in
// transform classes (include/transforms, include/utils, include/data_types)
// in the call order of the reference's DM loop
// (src/pipeline_multi.cu:161-294), one stage per call.  Used by the GPU
// tests to show that code written against the reference's transform API
// runs unchanged on libpeasoup_b200 and finds the same candidates as the
// fused engine (psx_search_dm, plain schedule).
//
// usage: dropin_pipeline series.f32 nsamps fft_size tsamp dm acc_lo acc_hi
//                        nharm min_snr zapfile|- out.bin
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>
#include <cufft.h>
#include "data_types/candidates.hpp"
#include "data_types/fourierseries.hpp"
#include "data_types/timeseries.hpp"
#include "transforms/birdiezapper.hpp"
#include "transforms/dereddener.hpp"
#include "transforms/distiller.hpp"
#include "transforms/ffter.hpp"
#include "transforms/harmonicfolder.hpp"
#include "transforms/peakfinder.hpp"
#include "transforms/resampler.hpp"
#include "transforms/spectrumformer.hpp"
#include "transforms/spectrumnormaliser.hpp"
#include "utils/stats.hpp"
#include "utils/utils.hpp"

// The other classes a reference translation unit may name: CuFFTerC2C
// (a forward and inverse round trip gives n times the input) and the
// 8-bit host series of ReusableDeviceTimeSeries (converted exactly).
// Returns 0 when both hold.
static int check_other_classes()
{
    const unsigned n = 1024;
    std::vector<cufftComplex> z(n), back(n);
    for (unsigned i = 0; i < n; ++i) z[i] = cufftComplex{std::sin(0.37f * i), std::cos(1.3f * i)};
    cufftComplex* d = nullptr;
    if (cudaMalloc(&d, sizeof(cufftComplex) * n) != cudaSuccess) return 5;
    cudaMemcpy(d, z.data(), sizeof(cufftComplex) * n, cudaMemcpyHostToDevice);
    {
        CuFFTerC2C c2c(n);
        c2c.execute(d, d, CUFFT_FORWARD);
        c2c.execute(d, d, CUFFT_INVERSE);
    }
    cudaMemcpy(back.data(), d, sizeof(cufftComplex) * n, cudaMemcpyDeviceToHost);
    cudaFree(d);
    for (unsigned i = 0; i < n; ++i)
        if (std::fabs(back[i].x - n * z[i].x) > 1e-3f * n || std::fabs(back[i].y - n * z[i].y) > 1e-3f * n)
            return 6;
    std::vector<uint8_t> u8(n);
    for (unsigned i = 0; i < n; ++i) u8[i] = (uint8_t)(i * 37u);
    TimeSeries<uint8_t> host_u8(u8.data(), n, 64e-6f);
    ReusableDeviceTimeSeries<float, uint8_t> d_u8(n);
    d_u8.copy_from_host(host_u8);
    std::vector<float> f(n);
    cudaMemcpy(f.data(), d_u8.get_data(), sizeof(float) * n, cudaMemcpyDeviceToHost);
    for (unsigned i = 0; i < n; ++i)
        if (f[i] != (float)u8[i]) return 7;
    return 0;
}

int main(int argc, char** argv)
{
    if (argc != 12) {
        std::fprintf(stderr, "usage: %s series nsamps fft_size tsamp dm acc_lo acc_hi nharm "
                             "min_snr zapfile out\n", argv[0]);
        return 2;
    }
    const std::size_t nsamps = std::strtoull(argv[2], nullptr, 10);
    const unsigned size = (unsigned)std::strtoul(argv[3], nullptr, 10);
    const float tsamp = std::strtof(argv[4], nullptr), dm = std::strtof(argv[5], nullptr);
    const float acc_lo = std::strtof(argv[6], nullptr), acc_hi = std::strtof(argv[7], nullptr);
    const int nharm = std::atoi(argv[8]);
    const float min_snr = std::strtof(argv[9], nullptr);
    const std::string zapfile = argv[10];
    std::vector<float> host(nsamps);
    {
        std::ifstream f(argv[1], std::ios::binary);
        f.read((char*)host.data(), sizeof(float) * nsamps);
        if (!f) return 3;
    }
    try {
        if (int rc = check_other_classes()) {
            std::fprintf(stderr, "drop-in class check failed (%d)\n", rc);
            return rc;
        }
        // set-up, as the worker thread does once
        const float tobs = size * tsamp;
        const float bin_width = 1.0 / tobs;
        DeviceFourierSeries<cufftComplex> d_fseries(size / 2 + 1, bin_width);
        ReusableDeviceTimeSeries<float, float> d_tim(size);
        DeviceTimeSeries<float> d_tim_r(size);
        DevicePowerSpectrum<float> pspec(d_fseries);
        CuFFTerR2C r2c(size);
        CuFFTerC2R c2r(size);
        TimeDomainResampler resampler;
        Dereddener rednoise(size / 2 + 1);
        SpectrumFormer former;
        PeakFinder cand_finder(min_snr, 0.1f, 1100.0f, size);
        HarmonicSums<float> sums(pspec, nharm);
        HarmonicFolder harm_folder(sums);
        HarmonicDistiller harm_finder(1e-4f, 16.0f, false);
        AccelerationDistiller acc_still(tobs, 1e-4f, true);
        Zapper* bzap = zapfile != "-" ? new Zapper(zapfile) : nullptr;
        AccelerationPlan acc_plan(acc_lo, acc_hi, 1.10f, 64e-6f, size, tsamp, 1475.12e6f, 1.09e6f);

        // one DM trial
        DedispersedTimeSeries<float> tim(host.data(), nsamps, tsamp, dm);
        d_tim.copy_from_host(tim);
        d_tim.remove_baseline(nsamps < size ? nsamps : size);
        if (size > nsamps) d_tim.fill(nsamps, size, 0);
        std::vector<float> acc_list;
        acc_plan.generate_accel_list(dm, 0.0f, acc_list);
        r2c.execute(d_tim.get_data(), d_fseries.get_data());
        former.form(d_fseries, pspec);
        rednoise.calculate_median(pspec);
        rednoise.deredden(d_fseries);
        if (bzap) bzap->zap(d_fseries);
        former.form_interpolated(d_fseries, pspec);
        float mean, rms, std_;
        stats::stats<float>(pspec.get_data(), size / 2 + 1, &mean, &rms, &std_);
        c2r.execute(d_fseries.get_data(), d_tim.get_data());
        SpectrumNormaliser norm(mean, std_, size);
        CandidateCollection accel_trial_cands;
        for (size_t jj = 0; jj < acc_list.size(); ++jj) {
            resampler.resampleII(d_tim, d_tim_r, size, acc_list[jj]);
            r2c.execute(d_tim_r.get_data(), d_fseries.get_data());
            former.form_interpolated(d_fseries, pspec);
            norm.normalise(pspec);
            harm_folder.fold(pspec);
            SpectrumCandidates trial_cands(dm, 0, acc_list[jj]);
            cand_finder.find_candidates(pspec, trial_cands);
            cand_finder.find_candidates(sums, trial_cands);
            accel_trial_cands.append(harm_finder.distill(trial_cands.cands));
        }
        std::vector<Candidate> dm_cands = acc_still.distill(accel_trial_cands.cands);
        delete bzap;
        std::ofstream out(argv[11], std::ios::binary);
        for (const Candidate& c : dm_cands) {
            CandidatePOD p{c.dm, c.dm_idx, c.acc, c.nh, c.snr, c.freq};
            out.write((const char*)&p, sizeof p);
        }
        std::printf("%zu candidates from %zu trials\n", dm_cands.size(), acc_list.size());
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
