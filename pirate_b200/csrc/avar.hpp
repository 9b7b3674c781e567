// avar.hpp -- analytic variances of the peak finder's trials, and the SNR weights made from them.
//
// Replaces pirate's PfAvarApproximation (include/pirate/PfVariance.hpp:86-120,
// src_lib/PfVariance.cpp:236-366; the python original is pirate_frb/slow_avar/PfVariance.py:465-640)
// and the non-random branch of PeakFindingKernelParams::fill_host_weights
// (src_lib/PeakFindingKernel.cu:606-692). GpuDedisperser::fill_analytic_weights
// (src_lib/GpuDedisperser.cpp:1162-1238) is built on these two.
//
// The model (pirate's approximation). Input channel i carries white noise of variance v_i. Tree
// gridding spreads it over the tree channels c it overlaps, with weights g_c (overlap lengths on the
// channel map). After k butterfly levels, the row (band F, delay d) of the partial tree holds, for
// that channel, a sum of deltas g_c 2^(-k/2) at integer times tau_k(c, d), c in band F. The variance
// of that row after profile kernel p (autocorrelation A_p) is
//
//     v_i 2^-k [ sum_c g_c^2 A_p(0) + 2 sum_{c<c'} g_c g_c' A_p(|tau_k(c,d) - tau_k(c',d)|) ].
//
// A tree with weight-DM downsampling 2^L and rank r uses the level k = r - L (k = r - L + 1 and the
// upper half of the delays for a downsampled primary tree). The variances of its 2^L bands are
// averaged into the 2^R peak-finding frequency bands and then into the tree's subbands. Channels
// split between bands (correlations across bands) are neglected, which is the approximation.

#pragma once

#include <vector>

#include "plan.hpp"

namespace pb2 {

// Autocorrelation A_p(lag) = sum_t h_p[t] h_p[t+lag] of the first P peak-finding profile kernels:
// p = 0 is one sample; level l (w = 2^l) adds ones(2w), [1/2 x w, 1 x w, 1/2 x w] and
// [1/2 x w, 1 x 2w, 1/2 x w] (pirate_frb/slow_avar/PfVariance.py:31-44).
struct PfProfileAutocorr
{
    long P = 0;
    std::vector<long> len;                  // kernel length per profile (A_p(lag) = 0 for lag >= len)
    std::vector<std::vector<double>> A;     // A[p][lag], lag < len[p]

    explicit PfProfileAutocorr(long P);
    double at(long p, long lag) const { return (lag < len[p]) ? A[p][lag] : 0.0; }
};

// Per tree: variance[(n * ndm_wt + d) * P + p] for subband n < N, weight-DM index d < ndm_wt and
// profile p < P, the shape of pirate's PfAvarApproximation::tree_variance[itree] (N, ndm_wt, P).
// freq_variances: nfreq values, each > 0. Throws std::runtime_error on bad arguments, or if a
// variance comes out non-positive.
std::vector<std::vector<double>> pf_analytic_variances(const DedispersionPlan &plan, const double *freq_variances, long nfreq);

// One beam's weights of tree t in the dedisperser's layout (ndm_wt, nt_wt, P, N):
// w[d, t, p, n] = 1 / sqrt(float(variance[n, d, p])), the same for every time t.
std::vector<float> pf_weights_from_variances(const DedispersionTree &t, const std::vector<double> &variance);

}  // namespace pb2
