/* orc_dedisp.c -- CPU restatement of the producer side of the search:
 * SIGPROC sample unpacking and direct incoherent dedispersion.
 *
 * TEST INFRASTRUCTURE ONLY (tests/, smoke(), bench.py's CPU legs).
 *
 * The reference dedisperses through the external dedisp library
 * (include/transforms/dedisperser.hpp:23-188: dedisp_create_plan_multi,
 * dedisp_generate_dm_list, dedisp_set_killmask, dedisp_execute with
 * 32-bit output).  dedisp (github.com/vishnubk/dedisp, an unpinned clone
 * of its HEAD in the reference's Dockerfile:34-37) is not present, so this
 * file restates the published algorithm (Barsdell et al. 2012, MNRAS 422,
 * 379: direct dedispersion over a per-channel delay table; DM spacing
 * from the smearing budget of Cordes & McLaughlin 2003) in plain loops:
 *
 *   delay_c   = K/dt * (f_c^-2 - f_0^-2),  f_c = fch1 + c*foff (MHz),
 *               K = 4.15e3 s MHz^2 cm^3/pc, float arithmetic;
 *   D(d, c)   = round-half-even(float(dm_d * delay_c));
 *   out[d][t] = map( sum over live channels c of x_c[t + D(d, c)] ),
 *               t < nsamps - max_delay,
 *   max_delay = floor(float(dm_max * delay_last) + 0.5).
 *
 * The channel sum is an exact integer.  `map` is the identity (raw) or
 * (sum - nchans*m/2) * 1/(m*sqrt(nchans)) + 1/2 with m = 2^nbits - 1,
 * each step one IEEE single operation (this file is compiled with
 * -ffp-contract=off).  The search downstream removes the baseline and
 * normalises its spectrum, so it sees any affine map alike up to
 * rounding.  Parity against dedisp itself is unpinned (absent library);
 * the known answers are the tutorial filterbank's pulsar (P = 250 ms at
 * DM 30, example_data/tutorial.fil) and planted dispersed pulses.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>

/* Channel c of one SIGPROC sample row.  Rows hold nchans*nbits/8 bytes;
 * below 8 bits the first channel sits in the least significant bits of
 * its byte; 16-bit samples are little-endian. */
unsigned orc_sigproc_value(const uint8_t* row, size_t c, int nbits)
{
    if (nbits == 8) return row[c];
    if (nbits == 16) return (unsigned)row[2 * c] | ((unsigned)row[2 * c + 1] << 8);
    size_t bit = c * (size_t)nbits;
    unsigned mask = (1u << nbits) - 1u;
    return (row[bit >> 3] >> (bit & 7)) & mask;
}

void orc_delay_table(size_t nchans, float tsamp, float fch1, float foff, float* out)
{
    const double k_dm = 4.15e3;
    for (size_t c = 0; c < nchans; ++c) {
        float inv_f = 1.0f / (fch1 + (float)c * foff);
        float inv_0 = 1.0f / fch1;
        float diff = inv_f * inv_f - inv_0 * inv_0;
        out[c] = (float)(k_dm / (double)tsamp * (double)diff);
    }
}

/* DM trials from dm_start upwards until one reaches dm_end.  Each next
 * DM x is the root of
 *   tsamp^2 + w^2 + a^2 x^2 + b^2 (x - p)^2 = tol^2 (tsamp^2 + w^2 + a^2 p^2)
 * (times in microseconds): the width at x, with the smearing across one
 * channel a*x and the smearing b*(x - p) of the DM step across a quarter
 * of the band, equals tol times the width at the previous trial p.
 * a = 8.3 us * foff / f^3 per unit DM at the centre frequency f (GHz),
 * b = a * nchans / 4.  The list is kept in float; each step starts from
 * the stored value. */
size_t orc_dm_list(size_t nchans, float tsamp, float fch1, float foff, float dm_start,
                   float dm_end, float width_us, float tol, float* out, size_t cap)
{
    double ts = (double)tsamp * 1e6;
    double f = ((double)fch1 + ((double)(nchans / 2) - 0.5) * (double)foff) * 1e-3;
    double t2 = (double)tol * (double)tol;
    double a = 8.3 * (double)foff / (f * f * f);
    double a2 = a * a;
    double b2 = a2 * ((double)(nchans * nchans) / 16.0);
    double c = (ts * ts + (double)width_us * (double)width_us) * (t2 - 1.0);
    size_t n = 0;
    float prev = dm_start;
    if (cap > 0) out[0] = prev;
    n = 1;
    while (prev < dm_end) {
        double p = (double)prev;
        double k = c + t2 * a2 * p * p;
        double x = (b2 * p + sqrt(-a2 * b2 * p * p + (a2 + b2) * k)) / (a2 + b2);
        prev = (float)x;
        if (n < cap) out[n] = prev;
        ++n;
        if (n > 100000000) break;
    }
    return n;
}

size_t orc_max_delay(const float* delays, size_t nchans, const float* dms, size_t ndm)
{
    float dm_max = 0.0f;
    for (size_t d = 0; d < ndm; ++d)
        if (d == 0 || dms[d] > dm_max) dm_max = dms[d];
    float prod = dm_max * delays[nchans - 1];
    return (size_t)floor((double)prod + 0.5);
}

void orc_map_constants(size_t nchans, int nbits, float* mid, float* scale)
{
    double m = (double)((1u << nbits) - 1u);
    *mid = (float)(0.5 * (double)nchans * m);
    *scale = (float)(1.0 / (m * sqrt((double)nchans)));
}

/* rows: nsamps SIGPROC rows; out: ndm rows of out_pitch floats, the first
 * nsamps - max_delay of each written.  killmask may be NULL (all live). */
int orc_dedisperse(const uint8_t* rows, size_t nsamps, size_t nchans, int nbits,
                   const float* delays, const float* dms, size_t ndm, const int* killmask,
                   int raw, float* out, size_t out_pitch)
{
    size_t row_bytes = nchans * (size_t)nbits / 8;
    size_t max_delay = orc_max_delay(delays, nchans, dms, ndm);
    if (max_delay >= nsamps) return -1;
    size_t nout = nsamps - max_delay;
    float mid, scale;
    orc_map_constants(nchans, nbits, &mid, &scale);
    for (size_t d = 0; d < ndm; ++d) {
        for (size_t t = 0; t < nout; ++t) {
            uint64_t sum = 0;
            for (size_t c = 0; c < nchans; ++c) {
                if (killmask && !killmask[c]) continue;
                float p = dms[d] * delays[c];
                long sh = lrintf(p);
                sum += orc_sigproc_value(rows + (t + (size_t)sh) * row_bytes, c, nbits);
            }
            float v = (float)sum;
            if (!raw) {
                v = v - mid;
                v = v * scale;
                v = v + 0.5f;
            }
            out[d * out_pitch + t] = v;
        }
    }
    return 0;
}
