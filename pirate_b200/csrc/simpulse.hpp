// simpulse.hpp -- simulated dispersed, scattered FRB pulses on a (frequency, time) grid, for injection
// into the dedisperser's input.
//
// Replaces pirate::simpulse::SinglePulse (include/pirate/simpulse.hpp:40-119, src_lib/simpulse.cpp),
// itself the 'single_pulse' part of the standalone simpulse library. Same pulse model and
// parameters:
// - Each channel [nu_lo, nu_hi]'s profile is a Gaussian (intrinsic_width), convolved with the
//   channel's dispersion smearing (a boxcar of the delay difference across the channel) and with a
//   one-sided exponential of the scattering time at the channel centre.
// - The spectrum goes as (nu / nu_0)^spectral_index, nu_0 the band centre.
// - The whole pulse is scaled so that sum over samples of (value^2 / channel variance) = snr^2.
// The profile is synthesised in the Fourier domain on internal_nt points spanning the channel's
// support, turned into a cumulative distribution, and integrated over each output sample. pirate
// uses MKL for the inverse FFT; here a radix-2 Cooley-Tukey transform of this file's own does it.

#pragma once

#include <string>
#include <vector>

namespace pb2 {

// Dispersion delay in seconds of a pulse of dispersion measure dm (pc cm^-3) at freq_mhz, with
// pirate's K_DM = 4.148808e6 ms MHz^2 per pc cm^-3 (include/pirate/constants.hpp:49).
double dispersion_delay(double dm, double freq_mhz);

// Scattering time in seconds at freq_mhz for scattering measure sm (the scattering time in ms at
// 1 GHz), scaling as freq^-4 (include/pirate/constants.hpp:50).
double scattering_time(double sm, double freq_mhz);

struct SinglePulseParams
{
    double dm = -1.0;                               // pc cm^-3
    double sm = -1.0;                               // scattering time in ms at 1 GHz
    double intrinsic_width = -1.0;                  // Gaussian width, seconds
    double spectral_index = -1000.0;
    double undispersed_arrival_time_sec = -1.0e6;   // arrival time at infinite frequency
    double time_sample_ms = -10.0;
    double snr = -1.0;                              // matched-filter SNR
    std::vector<double> freq_edges_mhz;             // nfreq + 1, strictly increasing, > 0
    std::vector<double> freq_variances;             // nfreq, > 0
    double subband_freq_lo_mhz = 0.0;               // only channels overlapping the subband get samples
    double subband_freq_hi_mhz = 1.0e9;
    long internal_nt = 1024;                        // synthesis points per channel, a power of two >= 64
};

struct SinglePulse
{
    SinglePulseParams params;
    long nfreq = 0;

    // Sparse pulse on the sample grid where sample i spans [i*dt, (i+1)*dt] seconds: channel f
    // (low to high frequency) has freq_nt[f] samples starting at index freq_it0[f], stored at
    // sparse_data[freq_sd_off[f] ...]. Indices may be negative. Channels outside the subband have
    // freq_nt = 0 and freq_it0 = it_start. it_start / it_end bound every channel's samples.
    std::vector<long> freq_it0, freq_nt, freq_sd_off;
    std::vector<float> sparse_data;
    long it_start = 0, it_end = 0;

    explicit SinglePulse(const SinglePulseParams &p);

    // out[f * row_stride + (i - out_it0)] += weight * pulse(f, i) for every pulse sample, on an array of
    // nfreq rows spanning samples [out_it0, out_it0 + out_nt), which must cover [it_start, it_end).
    void add_to_timestream(float *out, long out_nfreq, long out_nt, long row_stride, long out_it0, float weight) const;

    // Moves the pulse by delta_it samples (and its undispersed arrival time by delta_it samples).
    void shift_samples(long delta_it);

    std::string str() const;
};

// In-place radix-2 complex transform of n = 2^k points, x[m] <- sum_j x[j] exp(sign * 2 pi i j m / n),
// unnormalised (re and im interleaved: x[2j], x[2j+1]).
void fft_radix2(double *x, long n, int sign);

}  // namespace pb2
