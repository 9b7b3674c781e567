// simpulse.cpp -- simulated FRB pulses (model and citations in simpulse.hpp).

#include "simpulse.hpp"

#include <algorithm>
#include <cmath>
#include <complex>
#include <limits>
#include <sstream>
#include <stdexcept>

namespace pb2 {

namespace {

constexpr double kDm = 4.148808e6;               // ms MHz^2 per pc cm^-3 (include/pirate/constants.hpp:49)
constexpr double kScatteringIndex = 4.0;         // include/pirate/constants.hpp:50

[[noreturn]] void fail(const std::string &msg) { throw std::runtime_error("SinglePulse: " + msg); }

// Radix-2 decimation-in-time transform with a twiddle table built once per size.
struct Radix2
{
    long n = 0;
    int logn = 0;
    std::vector<double> c, s;      // cos, sin of 2 pi j / n, j < n/2

    explicit Radix2(long n_) : n(n_)
    {
        if (n < 2 || (n & (n - 1)))
            throw std::runtime_error("fft_radix2: n must be a power of two >= 2");
        while ((1L << logn) < n) logn++;
        c.resize(n / 2);
        s.resize(n / 2);
        for (long j = 0; j < n / 2; j++) {
            const double a = 2.0 * M_PI * (double) j / (double) n;
            c[j] = std::cos(a);
            s[j] = std::sin(a);
        }
    }

    void apply(double *x, int sign) const
    {
        for (long i = 0, j = 0; i < n; i++) {          // bit-reversal permutation
            if (i < j) {
                std::swap(x[2 * i], x[2 * j]);
                std::swap(x[2 * i + 1], x[2 * j + 1]);
            }
            long m = n >> 1;
            while (m >= 1 && (j & m)) { j ^= m; m >>= 1; }
            j |= m;
        }
        for (long len = 2; len <= n; len <<= 1) {
            const long half = len / 2, step = n / len;
            for (long i = 0; i < n; i += len)
                for (long k = 0; k < half; k++) {
                    const double wr = c[k * step], wi = sign * s[k * step];
                    double *u = x + 2 * (i + k), *v = x + 2 * (i + k + half);
                    const double tr = v[0] * wr - v[1] * wi, ti = v[0] * wi + v[1] * wr;
                    v[0] = u[0] - tr; v[1] = u[1] - ti;
                    u[0] += tr; u[1] += ti;
                }
        }
    }
};

double sinc(double x) { return (x * x > 1.0e-100) ? std::sin(x) / x : 1.0; }

// Linear interpolation of the normalised cumulative profile cum[0..N] at s in sample units.
double cum_at(const std::vector<double> &cum, long N, double s)
{
    if (s < 1.0e-10) return 0.0;
    if (s > N - 1.0e-10) return cum[N];
    const long i = (long) s;
    const double f = s - (double) i;
    return (1.0 - f) * cum[i] + f * cum[i + 1];
}

}  // namespace

void fft_radix2(double *x, long n, int sign)
{
    Radix2(n).apply(x, sign >= 0 ? 1 : -1);
}

double dispersion_delay(double dm, double freq_mhz)
{
    if (!(dm >= 0.0) || !(freq_mhz > 0.0)) fail("dispersion_delay needs dm >= 0 and freq > 0");
    return 1.0e-3 * kDm * dm / (freq_mhz * freq_mhz);
}

double scattering_time(double sm, double freq_mhz)
{
    if (!(sm >= 0.0) || !(freq_mhz > 0.0)) fail("scattering_time needs sm >= 0 and freq > 0");
    return 1.0e-3 * sm / std::pow(freq_mhz / 1000.0, kScatteringIndex);
}

SinglePulse::SinglePulse(const SinglePulseParams &p) : params(p)
{
    const std::vector<double> &edges = p.freq_edges_mhz;
    nfreq = (long) edges.size() - 1;
    if (nfreq < 1) fail("freq_edges_MHz needs at least two edges");
    if (!(edges[0] > 0.0)) fail("frequency edges must be positive");
    for (long i = 0; i < nfreq; i++)
        if (!(edges[i] < edges[i + 1])) fail("freq_edges_MHz must be strictly increasing");
    if ((long) p.freq_variances.size() != nfreq) fail("freq_variances must have one entry per channel");
    for (double v : p.freq_variances)
        if (!(v > 0.0)) fail("freq_variances must be > 0");
    const long N = p.internal_nt;
    if (N < 64 || (N & (N - 1))) fail("internal_nt must be a power of two >= 64");
    if (!(p.dm >= 0.0)) fail("dm is negative or unset");
    if (!(p.sm >= 0.0)) fail("sm is negative or unset");
    if (!(p.intrinsic_width >= 0.0)) fail("intrinsic_width is negative or unset");
    if (!(p.spectral_index > -1000.0)) fail("spectral_index is unset");
    if (!(p.undispersed_arrival_time_sec > -1.0e6)) fail("undispersed_arrival_time_sec is unset");
    if (!(p.time_sample_ms > 0.0)) fail("time_sample_ms is negative or unset");
    if (!(p.snr >= 0.0)) fail("snr is negative or unset");
    if (!(p.subband_freq_lo_mhz < p.subband_freq_hi_mhz)) fail("subband_freq_lo_MHz must be < subband_freq_hi_MHz");
    if (p.subband_freq_hi_mhz <= edges[0] || p.subband_freq_lo_mhz >= edges[nfreq])
        fail("the subband does not overlap the frequency band");
    if (p.dm == 0.0 && p.sm == 0.0 && p.intrinsic_width == 0.0)
        fail("a delta-function pulse (dm = sm = intrinsic_width = 0) is not supported");

    const double dt = 1.0e-3 * p.time_sample_ms;
    const double nu0 = 0.5 * (edges[0] + edges[nfreq]);
    const long nfft = 2 * N;
    const Radix2 fft(nfft);
    std::vector<double> buf(2 * nfft), cum(N + 1);
    std::vector<float> data;
    double snr_sq = 0.0;

    freq_it0.assign(nfreq, 0);
    freq_nt.assign(nfreq, 0);
    freq_sd_off.assign(nfreq, 0);
    it_start = std::numeric_limits<long>::max();
    it_end = std::numeric_limits<long>::min();
    long total = 0;

    for (long f = 0; f < nfreq; f++) {
        const double lo = edges[f], hi = edges[f + 1];
        freq_sd_off[f] = total;
        if (hi <= p.subband_freq_lo_mhz || lo >= p.subband_freq_hi_mhz)
            continue;
        const double nuc = 0.5 * (lo + hi);
        const double d0 = dispersion_delay(p.dm, hi), d1 = dispersion_delay(p.dm, lo);
        const double dmw = d1 - d0;
        const double ts = scattering_time(p.sm, nuc);
        // Support of the channel's profile: the smearing window, padded by 10% of it, 4 Gaussian
        // widths each side, one scattering time before and ten after.
        const double t0 = d0 - 0.1 * dmw - 4.0 * p.intrinsic_width - ts;
        const double t1 = d1 + 0.1 * dmw + 4.0 * p.intrinsic_width + 10.0 * ts;
        if (!(t0 < t1)) fail("empty pulse support");
        // Profile at t_i = t0 + (i + 1/2)(t1 - t0)/N, i < N: centre of the smearing window relative to t_0.
        const double tcen = 0.5 * (d0 + d1) - (t0 + (t1 - t0) / (2.0 * N));
        const double wt = std::pow(nuc / nu0, p.spectral_index);

        // Conjugate-even spectrum on nfft points (period 2(t1 - t0), so the profile does not wrap),
        // then the inverse transform.
        const double om0 = 2.0 * M_PI * (double) N / (double) nfft / (t1 - t0);
        for (long j = 0; j <= N; j++) {
            const double om = om0 * (double) j;
            std::complex<double> z = std::exp(-0.5 * (p.intrinsic_width * om) * (p.intrinsic_width * om));
            z *= sinc(0.5 * dmw * om);
            z /= std::complex<double>(1.0, ts * om);
            z *= std::complex<double>(std::cos(tcen * om), -std::sin(tcen * om));
            if (j == 0 || j == N) z = std::complex<double>(z.real(), 0.0);
            buf[2 * j] = z.real();
            buf[2 * j + 1] = z.imag();
            if (j > 0 && j < N) {
                buf[2 * (nfft - j)] = z.real();
                buf[2 * (nfft - j) + 1] = -z.imag();
            }
        }
        fft.apply(buf.data(), +1);

        cum[0] = 0.0;
        for (long i = 0; i < N; i++)
            cum[i + 1] = cum[i] + std::max(buf[2 * i], 0.0);
        if (!(cum[N] > 0.0)) {
            std::ostringstream ss;
            ss << "channel " << f << " produced a degenerate profile (no positive samples)";
            fail(ss.str());
        }
        for (long i = 0; i <= N; i++)
            cum[i] /= cum[N];

        const double pt0 = p.undispersed_arrival_time_sec + t0, pt1 = p.undispersed_arrival_time_sec + t1;
        const long i0 = (long) std::floor(pt0 / dt), i1 = (long) std::ceil(pt1 / dt);
        freq_it0[f] = i0;
        freq_nt[f] = i1 - i0;
        total += i1 - i0;
        it_start = std::min(it_start, i0);
        it_end = std::max(it_end, i1);
        const double amp = wt / dt, var = p.freq_variances[f];
        for (long it = i0; it < i1; it++) {
            const double a = cum_at(cum, N, N * ((double) it * dt - pt0) / (t1 - t0));
            const double b = cum_at(cum, N, N * ((double) (it + 1) * dt - pt0) / (t1 - t0));
            const double v = amp * (b - a);
            data.push_back((float) v);
            snr_sq += v * v / var;
        }
    }
    if (total <= 0) fail("the pulse has no samples");
    for (long f = 0; f < nfreq; f++)
        if (freq_nt[f] == 0) freq_it0[f] = it_start;
    if (!(snr_sq > 0.0)) fail("the pulse has zero energy");
    const double scale = p.snr / std::sqrt(snr_sq);
    sparse_data.resize(total);
    for (long k = 0; k < total; k++)
        sparse_data[k] = (float) ((double) data[k] * scale);
}

void SinglePulse::add_to_timestream(float *out, long out_nfreq, long out_nt, long row_stride, long out_it0, float weight) const
{
    if (!out) fail("add_to_timestream: null array");
    if (out_nfreq != nfreq) fail("add_to_timestream: the array must have one row per channel");
    if (out_nt <= 0 || row_stride < out_nt) fail("add_to_timestream: bad array shape");
    if (out_it0 > it_start || out_it0 + out_nt < it_end) {
        std::ostringstream ss;
        ss << "add_to_timestream: the array spans samples [" << out_it0 << ", " << out_it0 + out_nt
           << "), which does not cover the pulse's range [" << it_start << ", " << it_end << ")";
        fail(ss.str());
    }
    for (long f = 0; f < nfreq; f++) {
        float *row = out + f * row_stride + (freq_it0[f] - out_it0);
        const float *src = sparse_data.data() + freq_sd_off[f];
        for (long j = 0; j < freq_nt[f]; j++)
            row[j] += weight * src[j];
    }
}

void SinglePulse::shift_samples(long delta_it)
{
    for (long &i : freq_it0) i += delta_it;
    it_start += delta_it;
    it_end += delta_it;
    params.undispersed_arrival_time_sec += 1.0e-3 * (double) delta_it * params.time_sample_ms;
}

std::string SinglePulse::str() const
{
    std::ostringstream ss;
    ss << "SinglePulse(nfreq=" << nfreq << ", freq=[" << params.freq_edges_mhz.front() << ", "
       << params.freq_edges_mhz.back() << "] MHz, dm=" << params.dm << ", sm=" << params.sm
       << ", intrinsic_width=" << params.intrinsic_width << ", spectral_index=" << params.spectral_index
       << ", undispersed_arrival_time=" << params.undispersed_arrival_time_sec << " s, snr=" << params.snr
       << ", time_sample_ms=" << params.time_sample_ms << ", samples=[" << it_start << ", " << it_end << "))";
    return ss.str();
}

}  // namespace pb2
