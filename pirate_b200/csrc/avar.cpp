// avar.cpp -- analytic peak-finding variances and weights (model and citations in avar.hpp).
//
// pirate computes the variances by propagating a compressed time series per input channel through
// the tree levels (SparseTile / SparseTileTriple, src_lib/SparseTile.cpp) and autocorrelating it
// (PfVarianceConvolver::variance, src_lib/PfVariance.cpp:75-100). Here the same quantity is
// evaluated in closed form. For one input channel, a partial-tree row is a handful of deltas at
// known integer delays, so its autocorrelation is a sum over channel pairs. The delays of the
// channels in a band differ only through the steps of the top m delay bits, where m is the number
// of low channel-index bits in which the band's channels differ. So each band costs 2^m evaluations
// of a few channel pairs, and its variance is stored against that m-bit delay prefix.
// Floating-point sums run in a different order than pirate's, so values agree to rounding
// (relative 1e-15), not bitwise.

#include "avar.hpp"

#include <algorithm>
#include <cmath>
#include <sstream>
#include <stdexcept>

namespace pb2 {

PfProfileAutocorr::PfProfileAutocorr(long P_) : P(P_)
{
    if (P < 1 || (P - 1) % 3 != 0)
        throw std::runtime_error("PfProfileAutocorr: nprofiles must be 1 + 3 * (number of boxcar levels)");
    std::vector<std::vector<double>> h{{1.0}};
    for (long l = 0; 3 * l + 1 < P; l++) {
        const long w = 1L << l;
        std::vector<double> box(2 * w, 1.0), tri(3 * w, 1.0), trap(4 * w, 1.0);
        for (long i = 0; i < w; i++) {
            tri[i] = tri[2 * w + i] = 0.5;
            trap[i] = trap[3 * w + i] = 0.5;
        }
        h.push_back(box);
        h.push_back(tri);
        h.push_back(trap);
    }
    len.resize(P);
    A.resize(P);
    for (long p = 0; p < P; p++) {
        const long n = (long)h[p].size();
        len[p] = n;
        A[p].assign(n, 0.0);
        for (long lag = 0; lag < n; lag++)
            for (long t = 0; t + lag < n; t++)
                A[p][lag] += h[p][t] * h[p][t + lag];
    }
}

namespace {

int bit_length(unsigned long x) { return x ? 64 - __builtin_clzl(x) : 0; }

// Per-tree state of the sweep over input channels.
struct TreeModel
{
    long R = 0, L = 0, P = 0, N = 0;
    long kk = 0;          // bits of the weight-DM index (ndm_wt = 2^kk)
    long klevel = 0;      // tree level whose rows the tree's variances come from
    bool upper = false;   // downsampled primary tree: upper half of the level-klevel delays
    std::vector<long> flo, fhi;
    // acc[f][mm]: (2^mm, P) row-major sums, for peak-finding band f < 2^R, of contributions that
    // depend on the weight-DM index d only through its top mm bits.
    std::vector<std::vector<std::vector<double>>> acc;
};

struct Level
{
    long k = 0, Lmax = 0, P = 0;
    std::vector<long> trees;
};

}  // namespace

std::vector<std::vector<double>> pf_analytic_variances(const DedispersionPlan &plan, const double *fv, long nfreq)
{
    if (nfreq != plan.nfreq) {
        std::ostringstream ss;
        ss << "PfAvarApproximation: freq_variances has length " << nfreq << ", expected nfreq=" << plan.nfreq;
        throw std::runtime_error(ss.str());
    }
    if (!fv)
        throw std::runtime_error("PfAvarApproximation: freq_variances is null");
    for (long i = 0; i < nfreq; i++) {
        if (!(fv[i] > 0.0)) {
            std::ostringstream ss;
            ss << "PfAvarApproximation: freq_variances[" << i << "] = " << fv[i] << " must be > 0";
            throw std::runtime_error(ss.str());
        }
    }

    const long nchan = pow2(plan.config.toplevel_tree_rank);
    const std::vector<double> cm = plan.config.make_channel_map();   // decreasing; channel c spans [cm[c+1], cm[c]]
    const long ntrees = plan.ntrees;

    std::vector<TreeModel> tm(ntrees);
    std::vector<Level> levels;
    long Pmax = 1;
    for (long t = 0; t < ntrees; t++) {
        const DedispersionTree &tr = plan.trees[t];
        TreeModel &M = tm[t];
        const long r = tr.total_rank();
        M.R = tr.frequency_subbands.pf_rank;
        M.L = integer_log2(tr.pf.wt_dm_downsampling);
        M.P = tr.nprofiles;
        M.N = tr.frequency_subbands.N;
        M.upper = tr.primary_tree_index > 0;
        if (!(0 <= M.R && M.R <= M.L && M.L <= r)) {
            std::ostringstream ss;
            ss << "PfAvarApproximation: tree " << t << " needs 0 <= pf_rank (" << M.R << ") <= log2(wt_dm_downsampling) ("
               << M.L << ") <= tree rank (" << r << ")";
            throw std::runtime_error(ss.str());
        }
        M.kk = r - M.L;
        M.klevel = M.kk + (M.upper ? 1 : 0);
        if (tr.ndm_wt != pow2(M.kk))
            throw std::runtime_error("PfAvarApproximation: ndm_wt != 2^(tree rank - log2(wt_dm_downsampling))");
        M.flo = tr.frequency_subbands.n_to_flo;
        M.fhi = tr.frequency_subbands.n_to_fhi;
        M.acc.assign(pow2(M.R), std::vector<std::vector<double>>(M.kk + 1));
        for (auto &af : M.acc)
            for (long mm = 0; mm <= M.kk; mm++)
                af[mm].assign(pow2(mm) * M.P, 0.0);
        Pmax = std::max(Pmax, M.P);

        auto it = std::find_if(levels.begin(), levels.end(), [&](const Level &v) { return v.k == M.klevel; });
        if (it == levels.end()) {
            levels.push_back(Level());
            it = levels.end() - 1;
            it->k = M.klevel;
        }
        it->Lmax = std::max(it->Lmax, M.L);
        it->P = std::max(it->P, M.P);
        it->trees.push_back(t);
    }

    const PfProfileAutocorr ac(Pmax);
    std::vector<double> g, var;
    std::vector<long> tau;

    for (long i = 0; i < nfreq; i++) {
        // Tree channels overlapped by input channel i, i.e. by the index interval [i, i+1]:
        // c0 = first c with cm[c+1] < i+1, c1 = first c with cm[c] <= i.
        const double lo = (double)i, hi = (double)(i + 1);
        const long c0 = std::partition_point(cm.begin() + 1, cm.end(), [&](double x) { return x >= hi; }) - (cm.begin() + 1);
        const long c1 = std::partition_point(cm.begin(), cm.end() - 1, [&](double x) { return x > lo; }) - cm.begin();
        if (c0 >= c1) {
            std::ostringstream ss;
            ss << "PfAvarApproximation: input channel " << i << " overlaps no tree channel";
            throw std::runtime_error(ss.str());
        }
        g.resize(c1 - c0);
        for (long c = c0; c < c1; c++)
            g[c - c0] = std::max(0.0, std::min(cm[c], hi) - std::max(cm[c + 1], lo));

        for (const Level &lev : levels) {
            const long k = lev.k, P = lev.P;
            const double norm_k = std::ldexp(1.0, -(int)k);
            for (long F = c0 >> k; F <= ((c1 - 1) >> k) && F < pow2(lev.Lmax); F++) {
                const long a = std::max(c0, F << k), b = std::min(c1, (F + 1) << k) - 1;
                const int m = bit_length((unsigned long)(a ^ b));
                const long nj = pow2(m), nc = b - a + 1;
                var.assign(nj * P, 0.0);
                tau.resize(nc);
                for (long j = 0; j < nj; j++) {
                    // Relative delay of each channel for delay prefix j: at level s < m, the lower
                    // (even) channel of a pair is delayed by the step d_{s+1} - d_s of the delay,
                    // d_s = top s bits; levels >= m delay every channel of the band alike.
                    for (long q = 0; q < nc; q++) {
                        const long c = a + q;
                        long ts = 0;
                        for (int s = 0; s < m; s++)
                            if (!((c >> s) & 1))
                                ts += (j >> (m - s - 1)) - (j >> (m - s));
                        tau[q] = ts;
                    }
                    double *vj = &var[j * P];
                    for (long q = 0; q < nc; q++) {
                        const double gq = g[a + q - c0];
                        if (gq == 0.0)
                            continue;
                        for (long p = 0; p < P; p++)
                            vj[p] += gq * gq * ac.A[p][0];
                        for (long q2 = q + 1; q2 < nc; q2++) {
                            const double g2 = g[a + q2 - c0];
                            if (g2 == 0.0)
                                continue;
                            const long lag = std::labs(tau[q] - tau[q2]);
                            const double cross = 2.0 * gq * g2;
                            for (long p = 0; p < P; p++)
                                vj[p] += cross * ac.at(p, lag);
                        }
                    }
                    for (long p = 0; p < P; p++)
                        vj[p] *= norm_k;
                }

                for (long t : lev.trees) {
                    TreeModel &M = tm[t];
                    if (F >= pow2(M.L))
                        continue;
                    const long f = F >> (M.L - M.R);
                    const double s = std::ldexp(fv[i], -(int)(M.L - M.R));
                    if (!M.upper) {
                        double *dst = M.acc[f][m].data();
                        for (long j = 0; j < nj; j++)
                            for (long p = 0; p < M.P; p++)
                                dst[j * M.P + p] += s * var[j * P + p];
                    } else if (m == 0) {
                        double *dst = M.acc[f][0].data();
                        for (long p = 0; p < M.P; p++)
                            dst[p] += s * var[p];
                    } else {
                        // upper half: the top delay bit is 1 and dropped
                        const long h = nj / 2;
                        double *dst = M.acc[f][m - 1].data();
                        for (long j = h; j < nj; j++)
                            for (long p = 0; p < M.P; p++)
                                dst[(j - h) * M.P + p] += s * var[j * P + p];
                    }
                }
            }
        }
    }

    // Per tree and subband n: the mean over n's peak-finding bands, expanded over the weight-DM index.
    std::vector<std::vector<double>> out(ntrees);
    for (long t = 0; t < ntrees; t++) {
        const TreeModel &M = tm[t];
        const long nd = pow2(M.kk), P = M.P;
        out[t].assign(M.N * nd * P, 0.0);
        for (long n = 0; n < M.N; n++) {
            const double inv = 1.0 / (double)(M.fhi[n] - M.flo[n]);
            double *dst = &out[t][n * nd * P];
            for (long f = M.flo[n]; f < M.fhi[n]; f++)
                for (long mm = 0; mm <= M.kk; mm++) {
                    const double *src = M.acc[f][mm].data();
                    for (long d = 0; d < nd; d++) {
                        const double *row = src + (d >> (M.kk - mm)) * P;
                        for (long p = 0; p < P; p++)
                            dst[d * P + p] += inv * row[p];
                    }
                }
        }
        for (size_t e = 0; e < out[t].size(); e++) {
            if (!(out[t][e] > 0.0)) {
                std::ostringstream ss;
                ss << "PfAvarApproximation: tree " << t << " has a non-positive variance " << out[t][e]
                   << " at (n, d, p) = (" << e / (nd * P) << ", " << (e / P) % nd << ", " << e % P << ")";
                throw std::runtime_error(ss.str());
            }
        }
    }
    return out;
}

std::vector<float> pf_weights_from_variances(const DedispersionTree &t, const std::vector<double> &var)
{
    const long D = t.ndm_wt, T = t.nt_wt, P = t.nprofiles, N = t.frequency_subbands.N;
    if ((long)var.size() != N * D * P)
        throw std::runtime_error("pf_weights_from_variances: variance array has the wrong size");
    // base[d][n][p] = 1/sqrt of the variance rounded to float (pirate: rsqrtf(variances[n,d,p])).
    std::vector<float> base(D * N * P);
    for (long n = 0; n < N; n++)
        for (long d = 0; d < D; d++)
            for (long p = 0; p < P; p++) {
                const double v = var[(n * D + d) * P + p];
                if (!(v > 0.0))
                    throw std::runtime_error("pf_weights_from_variances: variances must be > 0");
                base[(d * N + n) * P + p] = (float)(1.0 / std::sqrt((double)(float)v));
            }
    std::vector<float> out(D * T * P * N);
    float *o = out.data();
    for (long d = 0; d < D; d++)
        for (long it = 0; it < T; it++)
            for (long p = 0; p < P; p++)
                for (long n = 0; n < N; n++)
                    *o++ = base[(d * N + n) * P + p];
    return out;
}

}  // namespace pb2
