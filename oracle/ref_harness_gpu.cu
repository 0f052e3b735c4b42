/*
 * ref_harness_gpu.cu -- drives the reference's OWN CUDA implementation of
 * the acceleration-search path (its src/kernels.cu, include/transforms/*
 * and the unmodified Worker class of src/pipeline_multi.cu) from plain
 * host buffers, so that tests can compare the new implementation with the
 * reference on the same GPU and the same inputs.
 *
 * TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile from the reference
 * sources where they lie (nothing is copied) into oracle/_ref/; never
 * linked by the product.  Every entry point copies its inputs to the
 * device, calls the reference API, and copies the results back; the
 * reference synchronises the device after every launch itself.
 *
 * Peasoup's main() is renamed at compile time (-Dmain=...) so that the
 * file defining Worker and DMDispenser can be included whole.
 */
#include <cstdio>
#include <functional>
#include <cstring>
#include <string>
#include <vector>
#include <iostream>
#include <sstream>
#include <map>
#include <chrono>
#include <thrust/device_vector.h>
#include <data_types/fourierseries.hpp>
#include <data_types/timeseries.hpp>
#include <transforms/ffter.hpp>
#include <kernels/kernels.h>
#include <kernels/defaults.h>
#include <utils/utils.hpp>
#include <utils/exceptions.hpp>
/* The running-median buffer is a private member of the reference's
   Dereddener; expose it to this harness only. */
#define private public
#include <transforms/dereddener.hpp>
#undef private
#include "src/pipeline_multi.cu"

namespace {

template <class T>
T* dev_alloc(size_t n)
{
    T* p = nullptr;
    if (cudaMalloc((void**)&p, sizeof(T) * (n ? n : 1)) != cudaSuccess) return nullptr;
    return p;
}

int guarded(const std::function<void()>& f)
{
    try {
        f();
    } catch (const std::exception& e) {
        std::fprintf(stderr, "reference harness: %s\n", e.what());
        return 1;
    }
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

/* ReusableDeviceTimeSeries<float, X>::copy_from_host (timeseries.hpp:
   352-361): the host->device copy of n 8-bit samples and the reference's
   conversion_kernel (src/kernels.cu:1171-1200); X = unsigned char or char,
   the two 8-bit types the reference instantiates. */
template <class X>
int copy_from_host_8bit(const X* in, float* out, size_t n)
{
    return guarded([&] {
        ReusableDeviceTimeSeries<float, X> d(n);
        TimeSeries<X> host(const_cast<X*>(in), n, 64e-6f);
        d.copy_from_host(host);
        cudaMemcpy(out, d.get_data(), sizeof(float) * n, cudaMemcpyDeviceToHost);
    });
}

}  // namespace

extern "C" {

typedef struct {
    float dm;
    int dm_idx;
    float acc;
    int nh;
    float snr;
    float freq;
} ref_candidate;

/* TimeDomainResampler::resampleII (resampler.hpp:26-31). */
int ref_resampleII(const float* in, float* out, size_t n, float acc, float tsamp)
{
    return guarded([&] {
        DeviceTimeSeries<float> a(n), b(n);
        a.set_tsamp(tsamp);
        cudaMemcpy(a.get_data(), in, sizeof(float) * n, cudaMemcpyHostToDevice);
        TimeDomainResampler r;
        r.resampleII(a, b, (unsigned)n, acc);
        cudaMemcpy(out, b.get_data(), sizeof(float) * n, cudaMemcpyDeviceToHost);
    });
}

int ref_copy_from_host_u8(const unsigned char* in, float* out, size_t n)
{
    return copy_from_host_8bit<unsigned char>(in, out, n);
}

int ref_copy_from_host_i8(const char* in, float* out, size_t n)
{
    return copy_from_host_8bit<char>(in, out, n);
}

/* TimeDomainResampler::resample (resampler.hpp:19-24). */
int ref_resample(const float* in, float* out, size_t n, float acc, float tsamp)
{
    return guarded([&] {
        DeviceTimeSeries<float> a(n), b(n);
        a.set_tsamp(tsamp);
        cudaMemcpy(a.get_data(), in, sizeof(float) * n, cudaMemcpyHostToDevice);
        TimeDomainResampler r;
        r.resample(a, b, (unsigned)n, acc);
        cudaMemcpy(out, b.get_data(), sizeof(float) * n, cudaMemcpyDeviceToHost);
    });
}

/* CuFFTerR2C::execute (ffter.hpp:54-80). */
int ref_fft_r2c(const float* in, size_t n, float* out_c)
{
    return guarded([&] {
        size_t nb = n / 2 + 1;
        float* d_in = dev_alloc<float>(n);
        cufftComplex* d_out = dev_alloc<cufftComplex>(nb);
        cudaMemcpy(d_in, in, sizeof(float) * n, cudaMemcpyHostToDevice);
        {
            CuFFTerR2C fft((unsigned)n);
            fft.execute(d_in, d_out);
            cudaDeviceSynchronize();
        }
        cudaMemcpy(out_c, d_out, sizeof(cufftComplex) * nb, cudaMemcpyDeviceToHost);
        cudaFree(d_in);
        cudaFree(d_out);
    });
}

/* CuFFTerC2R::execute (ffter.hpp:82-110). */
int ref_fft_c2r(const float* in_c, size_t n, float* out)
{
    return guarded([&] {
        size_t nb = n / 2 + 1;
        cufftComplex* d_in = dev_alloc<cufftComplex>(nb);
        float* d_out = dev_alloc<float>(n);
        cudaMemcpy(d_in, in_c, sizeof(cufftComplex) * nb, cudaMemcpyHostToDevice);
        {
            CuFFTerC2R fft((unsigned)n);
            fft.execute(d_in, d_out);
            cudaDeviceSynchronize();
        }
        cudaMemcpy(out, d_out, sizeof(float) * n, cudaMemcpyDeviceToHost);
        cudaFree(d_in);
        cudaFree(d_out);
    });
}

/* SpectrumFormer::form / form_interpolated (spectrumformer.hpp:8-22). */
int ref_form(const float* in_c, size_t nbins, int interbin, float* out)
{
    return guarded([&] {
        DeviceFourierSeries<cufftComplex> fs((unsigned)nbins, 1.0);
        DevicePowerSpectrum<float> ps(fs);
        cudaMemcpy(fs.get_data(), in_c, sizeof(cufftComplex) * nbins, cudaMemcpyHostToDevice);
        SpectrumFormer f;
        if (interbin) f.form_interpolated(fs, ps); else f.form(fs, ps);
        cudaMemcpy(out, ps.get_data(), sizeof(float) * nbins, cudaMemcpyDeviceToHost);
    });
}

/* Dereddener::calculate_median (dereddener.hpp:41-62); returns the
   spliced running median. */
int ref_running_median(const float* powers, size_t nbins, double bin_width, float* median)
{
    return guarded([&] {
        DevicePowerSpectrum<float> ps((unsigned)nbins, bin_width);
        cudaMemcpy(ps.get_data(), powers, sizeof(float) * nbins, cudaMemcpyHostToDevice);
        Dereddener d((unsigned)nbins);
        d.calculate_median(ps);
        cudaMemcpy(median, d.median, sizeof(float) * nbins, cudaMemcpyDeviceToHost);
    });
}

/* calculate_median on `powers` followed by Dereddener::deredden of the
   complex series X (in place). */
int ref_deredden(float* X, const float* powers, size_t nbins, double bin_width)
{
    return guarded([&] {
        DevicePowerSpectrum<float> ps((unsigned)nbins, bin_width);
        DeviceFourierSeries<cufftComplex> fs((unsigned)nbins, bin_width);
        cudaMemcpy(ps.get_data(), powers, sizeof(float) * nbins, cudaMemcpyHostToDevice);
        cudaMemcpy(fs.get_data(), X, sizeof(cufftComplex) * nbins, cudaMemcpyHostToDevice);
        Dereddener d((unsigned)nbins);
        d.calculate_median(ps);
        d.deredden(fs);
        cudaMemcpy(X, fs.get_data(), sizeof(cufftComplex) * nbins, cudaMemcpyDeviceToHost);
    });
}

/* Zapper(zapfile).zap (birdiezapper.hpp:29-65), X in place. */
int ref_zap(float* X, size_t nbins, double bin_width, const char* zapfile)
{
    return guarded([&] {
        DeviceFourierSeries<cufftComplex> fs((unsigned)nbins, bin_width);
        cudaMemcpy(fs.get_data(), X, sizeof(cufftComplex) * nbins, cudaMemcpyHostToDevice);
        Zapper z{std::string(zapfile)};
        z.zap(fs);
        cudaDeviceSynchronize();
        cudaMemcpy(X, fs.get_data(), sizeof(cufftComplex) * nbins, cudaMemcpyDeviceToHost);
    });
}

/* stats::stats (stats.hpp:25-33). */
int ref_stats(const float* x, size_t n, float* mean, float* rms, float* sd)
{
    return guarded([&] {
        float* d = dev_alloc<float>(n);
        cudaMemcpy(d, x, sizeof(float) * n, cudaMemcpyHostToDevice);
        stats::stats<float>(d, (unsigned)n, mean, rms, sd);
        cudaFree(d);
    });
}

/* stats::normalise (stats.hpp:35-40), in place. */
int ref_normalise(float* x, size_t n, float mean, float sd)
{
    return guarded([&] {
        float* d = dev_alloc<float>(n);
        cudaMemcpy(d, x, sizeof(float) * n, cudaMemcpyHostToDevice);
        stats::normalise(d, mean, sd, (unsigned)n);
        cudaMemcpy(x, d, sizeof(float) * n, cudaMemcpyDeviceToHost);
        cudaFree(d);
    });
}

/* DeviceTimeSeries::remove_baseline (timeseries.hpp:282-287), in place. */
int ref_remove_baseline(float* x, size_t n)
{
    return guarded([&] {
        DeviceTimeSeries<float> t(n);
        cudaMemcpy(t.get_data(), x, sizeof(float) * n, cudaMemcpyHostToDevice);
        t.remove_baseline(n);
        cudaMemcpy(x, t.get_data(), sizeof(float) * n, cudaMemcpyDeviceToHost);
    });
}

/* HarmonicSums + HarmonicFolder::fold (fourierseries.hpp:162-188,
   harmonicfolder.hpp:8-45); out holds nfolds spectra of n bins. */
int ref_harmonic_sums(const float* in, size_t n, int nfolds, float* out)
{
    return guarded([&] {
        DevicePowerSpectrum<float> ps((unsigned)n, 1.0);
        cudaMemcpy(ps.get_data(), in, sizeof(float) * n, cudaMemcpyHostToDevice);
        HarmonicSums<float> sums(ps, (unsigned)nfolds);
        HarmonicFolder folder(sums);
        folder.fold(ps);
        for (int h = 0; h < nfolds; ++h)
            cudaMemcpy(out + (size_t)h * n, sums[h]->get_data(), sizeof(float) * n,
                       cudaMemcpyDeviceToHost);
    });
}

/* PeakFinder::find_candidates on one spectrum with harmonic number nh
   (peakfinder.hpp:72-94). */
int ref_find_candidates(const float* spec, size_t nbins, double bin_width, int nh,
                        float thresh, float min_freq, float max_freq, int min_gap,
                        float* snr, float* freq, size_t cap, size_t* n)
{
    return guarded([&] {
        DevicePowerSpectrum<float> ps((unsigned)nbins, bin_width, (unsigned)nh);
        cudaMemcpy(ps.get_data(), spec, sizeof(float) * nbins, cudaMemcpyHostToDevice);
        PeakFinder pf(thresh, min_freq, max_freq, (unsigned)(2 * (nbins - 1)), min_gap);
        SpectrumCandidates sc(0.0f, 0, 0.0f);
        pf.find_candidates(ps, sc);
        *n = sc.cands.size();
        for (size_t i = 0; i < sc.cands.size() && i < cap; ++i) {
            snr[i] = sc.cands[i].snr;
            freq[i] = sc.cands[i].freq;
        }
    });
}

/* Search parameters of the Worker (the CmdLineOptions fields it reads). */
typedef struct {
    float cdm;
    float acc_start, acc_end, acc_tol, acc_pulse_width_us;
    float cfreq_hz, ch_bw_hz;
    int nharmonics;
    float min_snr, min_freq, max_freq;
    int max_harm;
    float freq_tol;
    const char* zapfile; /* "" or NULL for none */
} ref_search_args;

/* Runs the reference's unmodified Worker::start (pipeline_multi.cu:111-303)
   over `ndm` dedispersed series of `nsamps` samples with transform length
   `fft_size`, exactly as peasoup's main() sets it up
   (pipeline_multi.cu:412-421, 523-535).  Writes the per-DM
   acceleration-distilled candidates and, for each, its count of associated
   candidates (Candidate::count_assoc). */
static void flatten_tree(Candidate& c, std::vector<ref_candidate>& out, std::vector<int>& sizes)
{
    const size_t at = out.size();
    out.push_back(ref_candidate{c.dm, c.dm_idx, c.acc, c.nh, c.snr, c.freq});
    sizes.push_back(0);
    for (size_t k = 0; k < c.assoc.size(); ++k) flatten_tree(c.assoc[k], out, sizes);
    sizes[at] = (int)(out.size() - at);
}

static int worker_search(const float* series, size_t ndm, size_t nsamps, float tsamp,
                         const float* dms, size_t fft_size, const ref_search_args* a,
                         ref_candidate* out, int* nassoc, int* sizes_out, size_t cap,
                         size_t* n_out, double* start_seconds = nullptr)
{
    return guarded([&] {
        DispersionTrials<float> trials(tsamp);
        std::vector<float> dm_list(dms, dms + ndm);
        trials.resize(nsamps, dm_list);
        std::memcpy(trials.get_data_ptr(), series, sizeof(float) * ndm * nsamps);
        DMDispenser dispenser(trials);
        CmdLineOptions args;
        args.zapfilename = a->zapfile ? a->zapfile : "";
        args.verbose = false;
        args.cdm = a->cdm;
        args.acc_start = a->acc_start;
        args.acc_end = a->acc_end;
        args.acc_tol = a->acc_tol;
        args.acc_pulse_width = a->acc_pulse_width_us;
        args.boundary_5_freq = 0.05f;
        args.boundary_25_freq = 0.5f;
        args.nharmonics = a->nharmonics;
        args.min_snr = a->min_snr;
        args.min_freq = a->min_freq;
        args.max_freq = a->max_freq;
        args.max_harm = a->max_harm;
        args.freq_tol = a->freq_tol;
        AccelerationPlan plan(args.acc_start, args.acc_end, args.acc_tol,
                              args.acc_pulse_width * 1e-6, fft_size, tsamp,
                              a->cfreq_hz, a->ch_bw_hz);
        Worker w(trials, dispenser, plan, args, (unsigned)fft_size, 0);
        const auto t0 = std::chrono::steady_clock::now();
        w.start();
        if (start_seconds)
            *start_seconds =
                std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::vector<Candidate>& c = w.dm_trial_cands.cands;
        if (sizes_out) {
            // the candidates with their association trees, as a forest
            std::vector<ref_candidate> f;
            std::vector<int> fs;
            for (size_t i = 0; i < c.size(); ++i) flatten_tree(c[i], f, fs);
            *n_out = f.size();
            for (size_t i = 0; i < f.size() && i < cap; ++i) {
                out[i] = f[i];
                sizes_out[i] = fs[i];
            }
            return;
        }
        *n_out = c.size();
        for (size_t i = 0; i < c.size() && i < cap; ++i) {
            out[i] = ref_candidate{c[i].dm, c[i].dm_idx, c[i].acc, c[i].nh, c[i].snr, c[i].freq};
            if (nassoc) nassoc[i] = c[i].count_assoc();
        }
    });
}

int ref_worker_search(const float* series, size_t ndm, size_t nsamps, float tsamp,
                      const float* dms, size_t fft_size, const ref_search_args* a,
                      ref_candidate* out, int* nassoc, size_t cap, size_t* n_out)
{
    return worker_search(series, ndm, nsamps, tsamp, dms, fft_size, a, out, nassoc, nullptr, cap,
                         n_out);
}

/* The same run, also returning the wall time of Worker::start alone (the
   worker's own set-up of transforms and plans, every DM trial's host->device
   copy, prologue and acceleration trials; every launch there is followed by
   a device synchronisation, so wall time is device time).  The staging copy
   of the series into the reference's DispersionTrials container is outside
   it: in the reference's program that container is the dedisperser's
   output. */
int ref_worker_search_timed(const float* series, size_t ndm, size_t nsamps, float tsamp,
                            const float* dms, size_t fft_size, const ref_search_args* a,
                            ref_candidate* out, int* nassoc, size_t cap, size_t* n_out,
                            double* start_seconds)
{
    return worker_search(series, ndm, nsamps, tsamp, dms, fft_size, a, out, nassoc, nullptr, cap,
                         n_out, start_seconds);
}

/* The same run; its per-DM candidates with their association trees as a
   forest (nodes depth first, subtree sizes). */
int ref_worker_search_forest(const float* series, size_t ndm, size_t nsamps, float tsamp,
                             const float* dms, size_t fft_size, const ref_search_args* a,
                             ref_candidate* out, int* sizes, size_t cap, size_t* n_out)
{
    return worker_search(series, ndm, nsamps, tsamp, dms, fft_size, a, out, nullptr, sizes, cap,
                         n_out);
}

}  // extern "C"

/* DispersionTrials::write_timeseries_to_file (include/data_types/
   timeseries.hpp:520-594) as the reference's main calls it for a dump
   (src/pipeline_multi.cu:505-512): series `idx` of a block of ndm series of
   nsamps samples, under `outdir` with the file stem `stem`.  hd holds
   src_raj, src_dej, tstart, tsamp, fch1, foff; hi holds telescope_id,
   machine_id, nchans.  Host code only (no device call). */
extern "C" int ref_write_timeseries(const char* outdir, const char* stem, const float* data,
                                    size_t nsamps, const float* dms, size_t ndm, size_t idx,
                                    const double* hd, const int* hi, const char* source_name)
{
    try {
        DispersionTrials<float> trials((float)hd[3]);
        std::vector<float> dl(dms, dms + ndm);
        trials.resize(nsamps, dl);
        std::memcpy(trials.get_data_ptr(), data, sizeof(float) * nsamps * ndm);
        SigprocHeader h;
        h.src_raj = hd[0];
        h.src_dej = hd[1];
        h.tstart = hd[2];
        h.tsamp = hd[3];
        h.fch1 = hd[4];
        h.foff = hd[5];
        h.telescope_id = hi[0];
        h.machine_id = hi[1];
        h.nchans = hi[2];
        h.source_name = source_name;
        trials.write_timeseries_to_file(outdir, stem, idx, h);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
