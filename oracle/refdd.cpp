// oracle/refdd.cpp -- CPU ORACLE (test infrastructure only; never linked into the product).
//
// A restatement, templated on the arithmetic type Real (float = bitwise twin of the reference's
// fp32 CPU path, double = FP64 oracle), of pirate's CPU reference dedisperser:
//
//   FrequencySubbands           src_lib/FrequencySubbands.cpp:32-70,162-204
//   channel map / delay maps    src_lib/DedispersionConfig.cpp:62-193,239-250
//   plan (trees, ranks, pf)     src_lib/DedispersionPlan.cpp:29-146,246-342
//   bit_reverse, rb_lag,
//   downsample_{time,freq},
//   dedispersion_delay,
//   dedisperse_non_incremental  src_lib/utils.cpp:189-344
//   ReferenceLagbuf             src_lib/ReferenceLagbuf.cpp:46-127
//   ReferenceTree               src_lib/ReferenceTree.cpp:21-345
//   ReferenceTreeGridding       src_lib/TreeGriddingKernel.cu:62-102
//   ReferenceLaggedDownsampling src_lib/ReferenceLaggedDownsamplingKernel.cpp:27-139
//   ReferenceDedispersionKernel src_lib/DedispersionKernel.cu:219-300 (ring buffers disabled)
//   ReferencePeakFindingKernel  src_lib/PeakFindingKernel.cu:197-560 (apply, eval_tokens)
//   bare pf weights             src_lib/PeakFindingKernel.cu:606-692, src_lib/PfVariance.cpp:74-98
//   ReferenceDedisperser0/1     src_lib/ReferenceDedisperser.cpp:50-455
//
// Self-tests ported from the reference (ReferenceTree::test_basics / test_subbands,
// ReferenceLagbuf::test_random) are exposed through the C API at the bottom of this file.
//
// Parity of this restatement is pinned by those self-tests (brute-force sums against
// dedispersion_delay(), subband trees against independent sub-trees, incremental lags against
// one-shot shifts), by sophistication 0 == sophistication 1 (two independently structured
// algorithms), and by the plan fields of the reference's own configs/example_dedispersion_plan.yml.
// The reference itself cannot be compiled here (it needs ksgpu, yaml-cpp, MKL).
//
// Build with -ffp-contract=off so that a*b+c is never fused: the fp32 instantiation then performs
// exactly the reference's sequence of fp32 roundings.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace orc {

using std::vector;
using std::runtime_error;

#define ORC_ASSERT(cond) do { if (!(cond)) throw runtime_error(std::string("oracle assert failed: ") + #cond + " (" + std::to_string(__LINE__) + ")"); } while (0)

static inline long pow2(long n) { ORC_ASSERT(n >= 0 && n <= 40); return 1L << n; }

static inline bool is_pow2(long n) { return (n > 0) && !(n & (n-1)); }

static inline int ilog2(long n)
{
    ORC_ASSERT(is_pow2(n));
    int p = 0;
    while ((1L << p) < n) p++;
    return p;
}

static inline long xdiv(long m, long n) { ORC_ASSERT(n > 0 && m >= 0 && (m % n) == 0); return m / n; }

// utils.cpp:189
static int bit_reverse(int i, int nbits)
{
    ORC_ASSERT(nbits >= 0 && nbits <= 30 && i >= 0 && i < (1 << nbits));
    int j = 0;
    for (int b = 0; b < nbits; b++) { j = (j << 1) | (i & 1); i >>= 1; }
    return j;
}

// utils.cpp:224 -- lag between stage-1 output row (freq_coarse, dm_brev) and the stage-2 tree.
static long rb_lag(long freq_coarse, long dm_brev, long stage1_rank, long stage2_rank, bool uflag)
{
    long ndm = pow2(stage1_rank), nfreq = pow2(stage2_rank);
    ORC_ASSERT(freq_coarse >= 0 && freq_coarse < nfreq && dm_brev >= 0 && dm_brev < ndm);
    long dm = bit_reverse(dm_brev, stage1_rank) + (uflag ? ndm : 0);
    return (nfreq - 1 - freq_coarse) * dm;
}

// utils.cpp:288 -- total delay of (freq, dm_brev) in a rank-r tree.
static long dedispersion_delay(int rank, long freq, long dm_brev)
{
    long delay = 0, delay0 = 0;
    for (int r = 0; r < rank; r++) {
        long d = (dm_brev & 1) ? (delay0 + 1) : delay0;
        delay += (freq & 1) ? 0 : d;
        delay0 += d;
        dm_brev >>= 1;
        freq >>= 1;
    }
    return delay;
}


// -------------------------------------------------------------------------------------------------
// FrequencySubbands (FrequencySubbands.cpp:32-70, 162-204)


struct Subbands
{
    vector<long> counts;
    long pf_rank = -1, N = 0, M = 0;
    vector<long> m_to_n, m_to_d, n_to_flo, n_to_fhi, n_to_mbase;

    static void validate(const vector<long> &c)
    {
        ORC_ASSERT(c.size() > 0 && c.size() <= 5);
        long pr = c.size() - 1;
        ORC_ASSERT(c[pr] == 1);
        for (long l = 0; l <= pr; l++) {
            long mx = (l > 0) ? (pow2(pr + 1 - l) - 1) : pow2(pr);
            ORC_ASSERT(c[l] >= 0 && c[l] <= mx);
        }
    }

    Subbands() : Subbands(vector<long>{1}) { }

    explicit Subbands(const vector<long> &c) : counts(c)
    {
        validate(c);
        pf_rank = c.size() - 1;
        for (long l = 0; l <= pf_rank; l++) {
            for (long b = 0; b < c[l]; b++) {
                long s = pow2(std::max(l - 1, 0L));
                n_to_flo.push_back(b * s);
                n_to_fhi.push_back(b * s + pow2(l));
                n_to_mbase.push_back(M);
                for (long d = 0; d < pow2(l); d++) { m_to_n.push_back(N); m_to_d.push_back(d); }
                M += pow2(l);
                N += 1;
            }
        }
    }

    long m_to_flo(long m) const { return n_to_flo.at(m_to_n.at(m)); }
    long m_to_fhi(long m) const { return n_to_fhi.at(m_to_n.at(m)); }

    // FrequencySubbands.cpp:162
    static vector<long> restrict_counts(const vector<long> &c, long et_level, long new_pf_rank)
    {
        validate(c);
        long src_rank = c.size() - 1;
        long early_rank = std::max(src_rank - et_level, 0L);
        vector<long> ec(early_rank + 1, 0);
        ec[early_rank] = 1;
        for (long l = 0; l < early_rank; l++) {
            long mx = (l > 0) ? (pow2(early_rank + 1 - l) - 1) : pow2(early_rank);
            ec[l] = std::min(c[l], mx);
        }
        vector<long> dc(new_pf_rank + 1, 0);
        dc[new_pf_rank] = 1;
        for (long l = 0; l < new_pf_rank; l++) {
            long sl = l - new_pf_rank + early_rank;
            if (sl < 0 || ec[sl] == 0) dc[l] = 0;
            else if (sl == 0 && l > 0) dc[l] = 2 * ec[sl] - 1;
            else if (sl > 0 && l == 0) dc[l] = ec[sl] / 2 + 1;
            else dc[l] = ec[sl];
        }
        validate(dc);
        return dc;
    }
};


// -------------------------------------------------------------------------------------------------
// Config and plan (DedispersionConfig.cpp, DedispersionPlan.cpp:29-146)


struct PrimaryTree { long num_early_triggers, max_width, dm_downsampling, time_downsampling, wt_dm_downsampling, wt_time_downsampling; };

struct Config
{
    vector<long> zone_nfreq;
    vector<double> zone_freq_edges;
    double time_sample_ms = 1.0;
    long toplevel_tree_rank = 0;
    long time_samples_per_chunk = 0;
    long nbits = 32;                    // storage dtype width (32 or 16); sets nelts_per_segment
    vector<long> subband_counts;
    vector<PrimaryTree> primary_trees;
    long beams_per_gpu = 0, beams_per_batch = 0;

    long nfreq() const { long s = 0; for (long n : zone_nfreq) s += n; return s; }

    // DedispersionConfig.cpp:62
    double frequency_to_index(double freq) const
    {
        double fmin = zone_freq_edges.front(), fmax = zone_freq_edges.back();
        freq = std::min(std::max(freq, fmin), fmax);
        double off = 0;
        for (size_t i = 0; i < zone_nfreq.size(); i++) {
            double f0 = zone_freq_edges[i], f1 = zone_freq_edges[i+1];
            if (freq <= f1) { off += (freq - f0) / (f1 - f0) * zone_nfreq[i]; break; }
            off += zone_nfreq[i];
        }
        return std::min(std::max(off, 0.0), double(nfreq()));
    }

    // DedispersionConfig.cpp:135
    double delay_to_frequency(double delay) const
    {
        double flo = zone_freq_edges.front(), fhi = zone_freq_edges.back();
        double ntree = pow2(toplevel_tree_rank);
        delay = std::min(std::max(delay, 0.0), ntree);
        double scale = ntree / (1.0/(flo*flo) - 1.0/(fhi*fhi));
        return 1.0 / sqrt(delay/scale + 1.0/(fhi*fhi));
    }

    // DedispersionConfig.cpp:239
    vector<double> channel_map() const
    {
        long nchan = pow2(toplevel_tree_rank);
        vector<double> cm(nchan + 1);
        for (long n = 0; n <= nchan; n++)
            cm[n] = frequency_to_index(delay_to_frequency(n));
        return cm;
    }
};


struct TreeInfo
{
    long ipri, et_level, amb_rank, dd_rank, nt_ds;
    vector<long> sb_counts;
    long max_width, dm_ds, time_ds, wt_dm_ds, wt_time_ds;
    long Dcore, nprofiles, ndm_out, ndm_wt, nt_out, nt_wt;
    long total_rank() const { return amb_rank + dd_rank; }
};


struct Plan
{
    Config config;
    long nt_in = 0, npri = 0, nelts_per_segment = 0;
    vector<long> stage1_dd_rank, stage1_amb_rank;
    vector<TreeInfo> trees;

    // Dcore is the peak finder's time granularity (a kernel choice in the reference, taken from
    // its kernel registry; its production kernels use min(Dout, 8), makefile_helper.py:321).
    Plan(const Config &c, long dcore_max) : config(c)
    {
        nt_in = c.time_samples_per_chunk;
        npri = c.primary_trees.size();
        nelts_per_segment = 1024 / c.nbits;
        ORC_ASSERT(npri >= 1 && npri <= 7);
        ORC_ASSERT(c.toplevel_tree_rank >= 1 && c.toplevel_tree_rank <= 16);
        ORC_ASSERT((nt_in % (nelts_per_segment * pow2(npri - 1))) == 0);

        for (long ipri = 0; ipri < npri; ipri++) {
            long ptr = ipri ? (c.toplevel_tree_rank - 1) : c.toplevel_tree_rank;
            long s1dd = ptr / 2, s1amb = ptr - s1dd;
            stage1_dd_rank.push_back(s1dd);
            stage1_amb_rank.push_back(s1amb);
            const PrimaryTree &pt = c.primary_trees[ipri];

            for (long et = pt.num_early_triggers; et >= 0; et--) {
                TreeInfo t;
                t.ipri = ipri; t.et_level = et;
                t.amb_rank = s1dd; t.dd_rank = s1amb - et;
                t.nt_ds = xdiv(nt_in, pow2(ipri));
                ORC_ASSERT(t.dd_rank >= 1);
                long pf_rank = (t.dd_rank + 1) / 2;
                t.sb_counts = Subbands::restrict_counts(c.subband_counts, et, pf_rank);
                t.max_width = pt.max_width;
                t.dm_ds = pt.dm_downsampling ? pt.dm_downsampling : pow2(pf_rank);
                t.time_ds = pt.time_downsampling ? pt.time_downsampling : t.dm_ds;
                t.wt_dm_ds = pt.wt_dm_downsampling;
                t.wt_time_ds = pt.wt_time_downsampling;
                t.nprofiles = 1 + 3 * ilog2(t.max_width);
                t.ndm_out = xdiv(pow2(t.total_rank()), t.dm_ds);
                t.ndm_wt = xdiv(pow2(t.total_rank()), t.wt_dm_ds);
                t.nt_out = xdiv(t.nt_ds, t.time_ds);
                t.nt_wt = xdiv(t.nt_ds, t.wt_time_ds);
                t.Dcore = std::min(t.time_ds, dcore_max);
                trees.push_back(t);
            }
        }
    }
};


// -------------------------------------------------------------------------------------------------
// ReferenceLagbuf (ReferenceLagbuf.cpp:46-127): per-row incremental delay of (nrows, ntime) data.


template<typename R>
struct Lagbuf
{
    vector<int> lags;
    long ntime;
    vector<R> pstate;
    vector<R> tmp;

    Lagbuf(const vector<int> &lags_, long ntime_) : lags(lags_), ntime(ntime_)
    {
        long n = 0;
        for (int l : lags) { ORC_ASSERT(l >= 0); n += l; }
        pstate.assign(n, R(0));
        tmp.resize(ntime);
    }

    // data: (nrows, ntime), row stride 'rs'. Row i is replaced by its lags[i]-delayed version.
    void apply(R *data, long rs)
    {
        R *ps = pstate.data();
        for (size_t i = 0; i < lags.size(); i++) {
            long lag = lags[i];
            if (lag <= 0) continue;
            R *d = data + i * rs;
            long n = std::min(lag, ntime);
            // (ps | d) concatenated, then split at ntime: output = first ntime, state = last lag.
            memcpy(tmp.data(), d + (ntime - n), n * sizeof(R));
            memmove(d + n, d, (ntime - n) * sizeof(R));
            memcpy(d, ps, n * sizeof(R));
            memmove(ps, ps + n, (lag - n) * sizeof(R));
            memcpy(ps + (lag - n), tmp.data(), n * sizeof(R));
            ps += lag;
        }
    }
};


// -------------------------------------------------------------------------------------------------
// ReferenceTree (ReferenceTree.cpp:21-345)


template<typename R>
struct RefTree
{
    long B, amb_rank, dd_rank, T, S;
    Subbands fs;
    long Dpf;
    vector<R> pstate;
    vector<R> scratch;
    std::unique_ptr<Lagbuf<R>> final_lagbuf;

    RefTree(long B_, long amb_, long dd_, long T_, long S_, const vector<long> &counts)
        : B(B_), amb_rank(amb_), dd_rank(dd_), T(T_), S(S_), fs(counts)
    {
        ORC_ASSERT(B > 0 && amb_rank >= 0 && dd_rank >= 0 && T > 0 && S > 0);
        ORC_ASSERT(fs.pf_rank <= dd_rank);
        Dpf = pow2(amb_rank + dd_rank - fs.pf_rank);
        scratch.assign(S * (T + pow2(dd_rank) + 1), R(0));

        // Subband outputs are delayed so that all subbands of one DM line up (ReferenceTree.cpp:41-50).
        vector<int> fl(B * Dpf * fs.M);
        for (long b = 0; b < B; b++)
            for (long dpf = 0; dpf < Dpf; dpf++)
                for (long m = 0; m < fs.M; m++) {
                    long ff = pow2(fs.pf_rank) - fs.m_to_fhi(m);
                    long dd = dpf & (pow2(dd_rank - fs.pf_rank) - 1);
                    fl[(b * Dpf + dpf) * fs.M + m] = ff * dd * S;
                }
        final_lagbuf.reset(new Lagbuf<R>(fl, T * S));
    }

    // buf: (B, 2^amb, 2^dd, T*S) contiguous, dedispersed in place (row index -> bit-reversed dm).
    // out: (B, Dpf, M, T*S) contiguous subband outputs, or nullptr if M == 1.
    void dedisperse(R *buf, R *out)
    {
        long A = pow2(amb_rank), D = pow2(dd_rank), TS = T * S;
        ORC_ASSERT(out || fs.M == 1);
        long ps = 0;
        for (long b = 0; b < B; b++) {
            for (long a = 0; a < A; a++) {
                R *bufp = buf + ((b * A + a) * D) * TS;
                R *outp = nullptr;
                if (out) {
                    long pfdm = long(bit_reverse(a, amb_rank)) << (dd_rank - fs.pf_rank);
                    outp = out + ((b * Dpf + pfdm) * fs.M) * TS;
                }
                ps = dd2(bufp, TS, outp, fs.M * TS, TS, ps);
            }
        }
        if (out)
            final_lagbuf->apply(out, TS);
        ORC_ASSERT(ps == (long) pstate.size());
    }

    long dd2(R *bufp, long bstr, R *outp, long odstr, long omstr, long ps)
    {
        long TS = T * S, pf_rank = fs.pf_rank, pf_ndm = pow2(dd_rank - pf_rank), mcurr = 0;

        for (long r = 0; r <= dd_rank; r++) {
            long nf_in = pow2(dd_rank - r), ndm_in = pow2(r);

            if (outp && r == dd_rank - pf_rank) {
                // pf level 0: unstaggered bands are a transposed copy of the current rows.
                long pf_ns = fs.counts.at(0);
                ORC_ASSERT(nf_in == pow2(pf_rank) && ndm_in == pf_ndm);
                for (long dm_in = 0; dm_in < ndm_in; dm_in++) {
                    long dbr = bit_reverse(dm_in, r);
                    for (long pfs = 0; pfs < pf_ns; pfs++) {
                        const R *src = bufp + (pfs * ndm_in + dbr) * bstr;
                        R *dst = outp + dm_in * odstr + pfs * omstr;
                        memcpy(dst, src, TS * sizeof(R));
                    }
                }
                mcurr += pf_ns;
            }

            if (r >= dd_rank) break;

            long pf_level = r + pf_rank - dd_rank + 1;
            if (outp && pf_level > 0) {
                // Staggered bands at pf_level: extra butterflies over band pairs (pfs, pfs+1).
                long pf_ns = fs.counts.at(pf_level), pf_nd2 = pow2(pf_level - 1);
                ORC_ASSERT(ndm_in == pf_ndm * pf_nd2);
                for (long pf_dm = 0; pf_dm < pf_ndm; pf_dm++) {
                    for (long d2 = 0; d2 < pf_nd2; d2++) {
                        long dm_in = pf_dm * pf_nd2 + d2;
                        long dbr = bit_reverse(dm_in, r);
                        for (long pfs = 0; pfs < pf_ns; pfs++) {
                            R *src = bufp + (pfs * ndm_in + dbr) * bstr;
                            long m = mcurr + pfs * (2 * pf_nd2) + 2 * d2;
                            R *dst = outp + pf_dm * odstr + m * omstr;
                            ps = dd1(dst, omstr, src, ndm_in * bstr, ps, dm_in);
                        }
                    }
                }
                mcurr += pf_ns * 2 * pf_nd2;
            }

            long nf_out = nf_in / 2, ndm_out = 2 * ndm_in;
            for (long fo = 0; fo < nf_out; fo++) {
                for (long dbr = 0; dbr < ndm_in; dbr++) {
                    long dm_in = bit_reverse(dbr, r);
                    R *p = bufp + (fo * ndm_out + dbr) * bstr;
                    ps = dd1(p, ndm_in * bstr, p, ndm_in * bstr, ps, dm_in);
                }
            }
        }
        ORC_ASSERT(mcurr == (outp ? fs.M : 0));
        return ps;
    }

    // One butterfly: dst0[t] = (src0[t-lag] + src1[t])/sqrt2, dst1[t] = (src0[t-lag-1] + src1[t])/sqrt2,
    // with lags in units of S-element time samples and (lag+1)*S elements of history in pstate.
    long dd1(R *dst, long dstr, const R *src, long sstr, long ps, long lag)
    {
        const R rsqrt2 = R(0.7071067811865476);
        long TS = T * S;
        if (ps + (lag + 1) * S > (long) pstate.size())
            pstate.resize(ps + (lag + 1) * S, R(0));
        R *st = pstate.data() + ps;
        R *tmp = scratch.data();
        ORC_ASSERT((long) scratch.size() >= (T + lag + 1) * S);
        memcpy(tmp, st, (lag + 1) * S * sizeof(R));
        memcpy(tmp + (lag + 1) * S, src, TS * sizeof(R));
        memcpy(st, tmp + TS, (lag + 1) * S * sizeof(R));
        for (long ts = TS - 1; ts >= 0; ts--) {
            R x0 = tmp[ts], x1 = tmp[ts + S], y = src[sstr + ts];
            dst[ts] = rsqrt2 * (x1 + y);
            dst[dstr + ts] = rsqrt2 * (x0 + y);
        }
        return ps + (lag + 1) * S;
    }
};


// utils.cpp:300 -- one-shot (non-incremental) dedispersion of a (nfreq, ninner) array in place.
template<typename R>
static void dedisperse_non_incremental(R *arr, long nfreq, long ninner, long nspec)
{
    const R rsqrt2 = R(0.7071067811865476);
    int rank = ilog2(nfreq);
    for (int r = 0; r < rank; r++) {
        long pr = pow2(r);
        for (long i = 0; i < nfreq; i += 2 * pr) {
            for (long j = 0; j < pr; j++) {
                R *row0 = arr + (i + j) * ninner;
                R *row1 = row0 + pr * ninner;
                long lag1 = bit_reverse(j, r) * nspec, lag0 = lag1 + nspec;
                for (long k = ninner - 1; k >= 0; k--) {
                    R x0 = (k >= lag0) ? row0[k - lag0] : R(0);
                    R x1 = (k >= lag1) ? row0[k - lag1] : R(0);
                    R y = row1[k];
                    row0[k] = rsqrt2 * (x1 + y);
                    row1[k] = rsqrt2 * (x0 + y);
                }
            }
        }
    }
}


// -------------------------------------------------------------------------------------------------
// Tree gridding (TreeGriddingKernel.cu:62-102)


template<typename R>
struct Gridding
{
    long F, N, T;
    vector<double> cm;
    Gridding(const vector<double> &cm_, long F_, long T_) : F(F_), N(cm_.size() - 1), T(T_), cm(cm_) { }

    void apply(R *out, const float *in, long B) const
    {
        for (long b = 0; b < B; b++) {
            R *op = out + b * N * T;
            const float *ip = in + b * F * T;
            for (long i = 0; i < N * T; i++) op[i] = R(0);
            for (long n = 0; n < N; n++) {
                double f0 = cm[n + 1], f1 = cm[n];
                long if0 = std::max(long(f0), 0L), if1 = std::min(long(f1) + 1, F);
                for (long f = if0; f < if1; f++) {
                    double flo = std::max(f0, double(f)), fhi = std::min(f1, double(f) + 1);
                    double w = std::max(fhi - flo, 0.0);
                    R wr = R(float(w));   // the reference grids with float(w)
                    for (long t = 0; t < T; t++)
                        op[n * T + t] += wr * R(ip[f * T + t]);
                }
            }
        }
    }
};


// -------------------------------------------------------------------------------------------------
// Lagged downsampling (ReferenceLaggedDownsamplingKernel.cpp:27-139)


template<typename R>
struct LaggedDownsampler
{
    long r, s, npri, nb, ntime, nbatches;
    vector<std::unique_ptr<Lagbuf<R>>> small, large;   // per batch
    std::unique_ptr<LaggedDownsampler<R>> next;

    LaggedDownsampler(long r_, long out_dd_rank, long npri_, long nb_, long ntime_, long nbatches_)
        : r(r_), s(out_dd_rank + 1), npri(npri_), nb(nb_), ntime(ntime_), nbatches(nbatches_)
    {
        if (npri <= 1) return;
        long nt2 = xdiv(ntime, 2);
        vector<int> sl(nb * pow2(r)), ll(nb * pow2(r - 1));
        for (long i = 0; i < nb * pow2(r); i++) sl[i] = (i & 1) ? 0 : 1;
        for (long i = 0; i < nb * pow2(r - s); i++)
            for (long j = 0; j < pow2(s - 1); j++)
                ll[i * pow2(s - 1) + j] = pow2(s - 1) - j - 1;
        for (long i = 0; i < nbatches; i++) {
            small.emplace_back(new Lagbuf<R>(sl, nt2));
            large.emplace_back(new Lagbuf<R>(ll, nt2));
        }
        if (npri > 2)
            next.reset(new LaggedDownsampler<R>(r, out_dd_rank, npri - 1, nb, nt2, nbatches));
    }

    // in: (nb, 2^r, ntime); outs[k]: (nb, 2^(r-1), ntime/2^(k+1)) for k = 0..npri-2.
    void apply(const R *in, R *const *outs, long ibatch)
    {
        if (npri <= 1) return;
        const R w = R(0.7071067811865476);
        long nt2 = ntime / 2, nrow = nb * pow2(r);
        vector<R> ds(nrow * nt2), ds2;
        for (long c = 0; c < nrow; c++)
            for (long t = 0; t < nt2; t++)
                ds[c * nt2 + t] = w * (in[c * ntime + 2 * t] + in[c * ntime + 2 * t + 1]);
        ds2 = ds;
        small[ibatch]->apply(ds2.data(), nt2);
        R *out = outs[0];
        for (long c = 0; c < nrow / 2; c++)
            for (long t = 0; t < nt2; t++)
                out[c * nt2 + t] = w * (ds2[(2 * c) * nt2 + t] + ds2[(2 * c + 1) * nt2 + t]);
        large[ibatch]->apply(out, nt2);
        if (npri > 2)
            next->apply(ds.data(), outs + 1, ibatch);
    }
};


// -------------------------------------------------------------------------------------------------
// Peak finder (PeakFindingKernel.cu:197-560)


template<typename R>
struct PeakFinder
{
    long B, D, M, N, nt_in, nt_out, ndm_wt, nt_wt, Wmax, Dcore, total_beams;
    Subbands fs;
    long Dout, nbatches, P, tpad, L, expected_ibatch = 0;
    vector<long> tdt, tnt, tiout, tnout, tsout;
    vector<vector<R>> tmp;   // per level, (B, D, M, tnt[l])
    vector<R> pstate;        // (total_beams, D, M, tpad)

    PeakFinder(const TreeInfo &t, long B_, long total_beams_)
        : B(B_), D(t.ndm_out), nt_in(t.nt_ds), nt_out(t.nt_out), ndm_wt(t.ndm_wt), nt_wt(t.nt_wt),
          Wmax(t.max_width), Dcore(t.Dcore), total_beams(total_beams_), fs(t.sb_counts)
    {
        M = fs.M; N = fs.N;
        nbatches = xdiv(total_beams, B);
        P = 3 * ilog2(Wmax) + 1;
        Dout = xdiv(nt_in, nt_out);
        ORC_ASSERT(is_pow2(Dcore) && (Dout % Dcore) == 0);
        tpad = std::max(2 * Wmax, 4L);
        L = std::max(ilog2(Wmax), 1);
        pstate.assign(total_beams * D * M * tpad, R(0));
        for (long l = 0; l < L; l++) {
            long dt = std::min(Dcore, pow2(l));
            long nt = xdiv(nt_in + tpad - pow2(l), dt) + 1;
            tdt.push_back(dt); tnt.push_back(nt);
            tnout.push_back(xdiv(Dout, dt));
            tsout.push_back(xdiv(pow2(l), dt));
            tiout.push_back(xdiv(tpad + dt - pow2(l), dt));
            tmp.emplace_back(B * D * M * nt, R(0));
        }
    }

    static inline void upd(R &mx, uint32_t &am, R val, uint32_t tok)
    {
        am = (val > mx) ? tok : am;
        mx = std::max(mx, val);
    }

    // in: (B, D, M, nt_in); wt: (B, ndm_wt, nt_wt, P, N); outputs (B, D, nt_out).
    void apply(R *out_max, uint32_t *out_argmax, const R *in, const float *wt, long ibatch)
    {
        ORC_ASSERT(ibatch == expected_ibatch);
        expected_ibatch = (ibatch + 1) % nbatches;
        long b0 = ibatch * B, t1 = std::min(tpad, nt_in), t0 = tpad - t1;

        for (long b = 0; b < B; b++)
            for (long d = 0; d < D; d++)
                for (long m = 0; m < M; m++) {
                    R *dst = &tmp[0][((b * D + d) * M + m) * tnt[0]];
                    R *ps = &pstate[(((b0 + b) * D + d) * M + m) * tpad];
                    const R *src = in + ((b * D + d) * M + m) * nt_in;
                    for (long t = 0; t < tpad; t++) dst[t] = ps[t];
                    for (long t = 0; t < nt_in; t++) dst[t + tpad] = src[t];
                    for (long t = 0; t < t0; t++) ps[t] = ps[t + nt_in];
                    for (long t = 0; t < t1; t++) ps[t + t0] = src[t + nt_in - t1];
                }

        for (long l = 0; l + 1 < L; l++) {
            long ns = tnt[l], nd = tnt[l + 1];
            long rr = xdiv(tdt[l + 1], tdt[l]), ss = xdiv(pow2(l), tdt[l]);
            ORC_ASSERT(rr * (nd - 1) + ss == ns - 1);
            for (long i = 0; i < B * D * M; i++) {
                R *dst = &tmp[l + 1][i * nd];
                const R *src = &tmp[l][i * ns];
                for (long t = 0; t < nd; t++) dst[t] = src[rr * t] + src[rr * t + ss];
            }
        }

        long Wds = xdiv(D, ndm_wt), Tds = xdiv(nt_out, nt_wt);
        for (long b = 0; b < B; b++)
            for (long d = 0; d < D; d++)
                for (long tout = 0; tout < nt_out; tout++) {
                    const float *wp = wt + (((b * ndm_wt + d / Wds) * nt_wt + tout / Tds) * P) * N;
                    R mx = R(-1.0e30f);
                    uint32_t am = ~0u;
                    for (long l = 0; l < L; l++) {
                        const R *ti = &tmp[l][((b * D + d) * M) * tnt[l]];
                        long mstr = tnt[l], dt = tdt[l], ns = tnout[l], S = tsout[l], I = tiout[l];
                        for (long m = 0; m < M; m++) {
                            long n = fs.m_to_n[m];
                            R w0 = l ? R(0) : R(wp[n]);
                            R w1 = (P > 1) ? R(wp[(3 * l + 1) * N + n]) : R(0);
                            R w2 = (P > 1) ? R(wp[(3 * l + 2) * N + n]) : R(0);
                            R w3 = (P > 1) ? R(wp[(3 * l + 3) * N + n]) : R(0);
                            for (long is = 0; is < ns; is++) {
                                long j = m * mstr + I + tout * ns + is;
                                R x0 = ti[j - 3 * S], x1 = ti[j - 2 * S], x2 = ti[j - S], x3 = ti[j];
                                uint32_t tk0 = (uint32_t(m) << 16) | uint32_t(is * dt);
                                R y0 = x3;
                                R y1 = x2 + x3;
                                R y2 = R(0.5f) * x1 + x2 + R(0.5f) * x3;
                                R y3 = R(0.5f) * x0 + x1 + x2 + R(0.5f) * x3;
                                if (l == 0) upd(mx, am, w0 * y0, tk0);
                                if (P > 1) {
                                    upd(mx, am, w1 * y1, tk0 | uint32_t((3 * l + 1) << 8));
                                    upd(mx, am, w2 * y2, tk0 | uint32_t((3 * l + 2) << 8));
                                    upd(mx, am, w3 * y3, tk0 | uint32_t((3 * l + 3) << 8));
                                }
                            }
                        }
                    }
                    out_max[(b * D + d) * nt_out + tout] = mx;
                    out_argmax[(b * D + d) * nt_out + tout] = am;
                }
    }

    // Re-evaluates one trial per output element, selected by 'tokens' (PeakFindingKernel.cu:467).
    // Returns 0 on success, or -1 if a token is malformed.
    int eval_tokens(R *out, const uint32_t *tokens, const float *wt) const
    {
        long Wds = xdiv(D, ndm_wt), Tds = xdiv(nt_out, nt_wt);
        for (long b = 0; b < B; b++)
            for (long d = 0; d < D; d++)
                for (long tout = 0; tout < nt_out; tout++) {
                    uint32_t tk = tokens[(b * D + d) * nt_out + tout];
                    long m = (tk >> 16) & 0xffff, p = (tk >> 8) & 0xff, t = tk & 0xff;
                    if (m >= M || p >= P || t >= Dout) return -1;
                    long l = p ? (p - 1) / 3 : 0, q = p - 3 * l;
                    long dt = tdt[l], is = t / dt;
                    if (t != is * dt) return -1;
                    long n = fs.m_to_n[m];
                    R w = R(wt[(((b * ndm_wt + d / Wds) * nt_wt + tout / Tds) * P + p) * N + n]);
                    long j = ((b * D + d) * M + m) * tnt[l] + tiout[l] + tout * tnout[l] + is, S = tsout[l];
                    const vector<R> &ti = tmp[l];
                    R x0 = ti[j - 3 * S], x1 = ti[j - 2 * S], x2 = ti[j - S], x3 = ti[j];
                    R y;
                    if (q == 0) y = x3;
                    else if (q == 1) y = x2 + x3;
                    else if (q == 2) y = R(0.5f) * x1 + x2 + R(0.5f) * x3;
                    else y = R(0.5f) * x0 + x1 + x2 + R(0.5f) * x3;
                    out[(b * D + d) * nt_out + tout] = w * y;
                }
        return 0;
    }
};


// -------------------------------------------------------------------------------------------------
// ReferenceDedispersionKernel (DedispersionKernel.cu:219-300), with ring buffers disabled.
// Operates on a contiguous (B, 2^amb, 2^dd, T) buffer: optional residual lags, then the tree.


template<typename R>
struct DdKernel
{
    long B, amb_rank, dd_rank, T, nbatches, nt_per_segment;
    bool apply_rlags, downsampled;
    vector<std::unique_ptr<RefTree<R>>> trees;
    vector<std::unique_ptr<Lagbuf<R>>> rlags;

    DdKernel(long B_, long amb, long dd, long T_, long total_beams, const vector<long> &counts,
             bool rl, bool ds, long nps)
        : B(B_), amb_rank(amb), dd_rank(dd), T(T_), nt_per_segment(nps), apply_rlags(rl), downsampled(ds)
    {
        nbatches = xdiv(total_beams, B);
        for (long i = 0; i < nbatches; i++)
            trees.emplace_back(new RefTree<R>(B, amb, dd, T, 1, counts));
        if (rl) {
            long A = pow2(amb), F = pow2(dd);
            vector<int> lg(B * A * F);
            for (long b = 0; b < B; b++)
                for (long a = 0; a < A; a++)
                    for (long f = 0; f < F; f++)
                        lg[(b * A + a) * F + f] = rb_lag(f, a, amb, dd, ds) % nt_per_segment;
            for (long i = 0; i < nbatches; i++)
                rlags.emplace_back(new Lagbuf<R>(lg, T));
        }
    }

    void apply(R *dd, R *sb_out, long ibatch)
    {
        if (apply_rlags) rlags[ibatch]->apply(dd, T);
        trees[ibatch]->dedisperse(dd, sb_out);
    }
};


// -------------------------------------------------------------------------------------------------
// ReferenceDedisperser0/1 (ReferenceDedisperser.cpp:50-455)


template<typename R>
struct Dedisperser
{
    Plan plan;
    int sophistication;
    long B, F, nt_in, total_beams, nbatches, ntrees, npri, rtop;
    std::unique_ptr<Gridding<R>> grid;
    vector<std::unique_ptr<PeakFinder<R>>> pfs;
    vector<vector<R>> sb;        // per tree PF input (B, ndm_out, M, nt_ds)

    // sophistication 0
    vector<vector<R>> ds_inputs;                         // per primary tree (B, 2^rtop, nt/2^p)
    vector<std::unique_ptr<RefTree<R>>> trees0;          // nbatches * ntrees
    vector<vector<R>> sb0;                               // per tree (B, ndm_ref, M, nt)

    // sophistication 1
    std::unique_ptr<LaggedDownsampler<R>> lds;
    vector<vector<R>> s1buf;                             // per primary tree (B, 2^rank_p, nt_p)
    vector<std::unique_ptr<DdKernel<R>>> s1k, s2k;
    vector<std::unique_ptr<Lagbuf<R>>> s2lags;           // nbatches * ntrees
    vector<vector<R>> s2buf;

    Dedisperser(const Plan &p, int soph) : plan(p), sophistication(soph)
    {
        const Config &c = plan.config;
        B = c.beams_per_batch; F = c.nfreq(); nt_in = plan.nt_in; total_beams = c.beams_per_gpu;
        nbatches = xdiv(total_beams, B); ntrees = plan.trees.size(); npri = plan.npri;
        rtop = c.toplevel_tree_rank;
        grid.reset(new Gridding<R>(c.channel_map(), F, nt_in));
        for (const TreeInfo &t : plan.trees) {
            pfs.emplace_back(new PeakFinder<R>(t, B, total_beams));
            Subbands fs(t.sb_counts);
            sb.emplace_back(B * t.ndm_out * fs.M * t.nt_ds, R(0));
        }

        if (soph == 0) {
            for (long ip = 0; ip < npri; ip++)
                ds_inputs.emplace_back(B * pow2(rtop) * xdiv(nt_in, pow2(ip)), R(0));
            for (long ib = 0; ib < nbatches; ib++)
                for (const TreeInfo &t : plan.trees) {
                    long rr = t.total_rank() + (t.ipri > 0 ? 1 : 0);
                    trees0.emplace_back(new RefTree<R>(B, 0, rr, t.nt_ds, 1, t.sb_counts));
                }
            for (const TreeInfo &t : plan.trees) {
                long rr = t.total_rank() + (t.ipri > 0 ? 1 : 0);
                Subbands fs(t.sb_counts);
                sb0.emplace_back(B * pow2(rr - fs.pf_rank) * fs.M * t.nt_ds, R(0));
            }
        }
        else if (soph == 1) {
            long odr = (npri > 1) ? plan.stage1_dd_rank[1] : 0;
            lds.reset(new LaggedDownsampler<R>(rtop, odr, npri, B, nt_in, nbatches));
            for (long ip = 0; ip < npri; ip++) {
                long rk = plan.stage1_dd_rank[ip] + plan.stage1_amb_rank[ip];
                long nt = xdiv(nt_in, pow2(ip));
                s1buf.emplace_back(B * pow2(rk) * nt, R(0));
                s1k.emplace_back(new DdKernel<R>(B, plan.stage1_amb_rank[ip], plan.stage1_dd_rank[ip], nt,
                                                 total_beams, {1}, false, ip > 0, plan.nelts_per_segment));
            }
            for (const TreeInfo &t : plan.trees)
                s2k.emplace_back(new DdKernel<R>(B, t.amb_rank, t.dd_rank, t.nt_ds, total_beams, t.sb_counts,
                                                 true, t.ipri > 0, plan.nelts_per_segment));
            long S = plan.nelts_per_segment;
            for (long ib = 0; ib < nbatches; ib++)
                for (const TreeInfo &t : plan.trees) {
                    long rank = t.total_rank();
                    vector<int> lg(B * pow2(rank));
                    for (long fc = 0; fc < pow2(t.dd_rank); fc++)
                        for (long db = 0; db < pow2(t.amb_rank); db++) {
                            long row = fc * pow2(t.amb_rank) + db;
                            long lag = rb_lag(fc, db, t.amb_rank, t.dd_rank, t.ipri > 0);
                            for (long b = 0; b < B; b++) lg[b * pow2(rank) + row] = (lag / S) * S;
                        }
                    s2lags.emplace_back(new Lagbuf<R>(lg, t.nt_ds));
                }
            for (const TreeInfo &t : plan.trees)
                s2buf.emplace_back(B * pow2(t.total_rank()) * t.nt_ds, R(0));
        }
        else
            throw runtime_error("oracle: sophistication must be 0 or 1");
    }

    // Tree-domain input (ReferenceDedisperser with tree_domain_input, src_lib/ReferenceDedisperser.cpp:205-213,
    // 388-396): 'in' is already gridded, (B, 2^rtop, nt_in), and step 0 is a copy.
    void load_tree_domain(R *dst, const float *in) const
    {
        for (long i = 0; i < B * pow2(rtop) * nt_in; i++)
            dst[i] = R(in[i]);
    }

    // in: (B, F, nt_in) float, or (B, 2^rtop, nt_in) with tree_domain; wts[itree]: (B, ndm_wt, nt_wt, P, N);
    // outputs (B, ndm_out, nt_out).
    void dedisperse(long ibatch, const float *in, const float *const *wts, R *const *omax, uint32_t *const *oarg,
                    bool tree_domain = false)
    {
        if (sophistication == 0) {
            if (tree_domain)
                load_tree_domain(ds_inputs[0].data(), in);
            else
                grid->apply(ds_inputs[0].data(), in, B);
            for (long ip = 1; ip < npri; ip++) {
                const R w = R(0.7071067811865476);
                long ntd = xdiv(nt_in, pow2(ip));
                const R *src = ds_inputs[ip - 1].data();
                R *dst = ds_inputs[ip].data();
                for (long c = 0; c < B * pow2(rtop); c++)
                    for (long t = 0; t < ntd; t++)
                        dst[c * ntd + t] = w * (src[c * 2 * ntd + 2 * t] + src[c * 2 * ntd + 2 * t + 1]);
            }
            for (long it = 0; it < ntrees; it++) {
                const TreeInfo &t = plan.trees[it];
                long rr = t.total_rank() + (t.ipri > 0 ? 1 : 0);
                long nt = t.nt_ds;
                vector<R> dd(B * pow2(rr) * nt);
                for (long b = 0; b < B; b++)
                    memcpy(&dd[b * pow2(rr) * nt], &ds_inputs[t.ipri][b * pow2(rtop) * nt], pow2(rr) * nt * sizeof(R));
                trees0[ibatch * ntrees + it]->dedisperse(dd.data(), sb0[it].data());
                Subbands fs(t.sb_counts);
                long ndmr = pow2(rr - fs.pf_rank), slab = fs.M * nt;
                const R *src = sb0[it].data();
                R *dst = sb[it].data();
                for (long b = 0; b < B; b++) {
                    long d0 = (t.ipri > 0) ? ndmr / 2 : 0;
                    memcpy(dst + b * t.ndm_out * slab, src + (b * ndmr + d0) * slab, t.ndm_out * slab * sizeof(R));
                }
                pfs[it]->apply(omax[it], oarg[it], sb[it].data(), wts[it], ibatch);
            }
            return;
        }

        if (tree_domain)
            load_tree_domain(s1buf[0].data(), in);
        else
            grid->apply(s1buf[0].data(), in, B);
        vector<R *> louts;
        for (long ip = 1; ip < npri; ip++) louts.push_back(s1buf[ip].data());
        lds->apply(s1buf[0].data(), louts.data(), ibatch);

        for (long ip = 0; ip < npri; ip++)
            s1k[ip]->apply(s1buf[ip].data(), nullptr, ibatch);

        for (long it = 0; it < ntrees; it++) {
            const TreeInfo &t = plan.trees[it];
            long rank = t.total_rank();
            long rk1 = plan.stage1_dd_rank[t.ipri] + plan.stage1_amb_rank[t.ipri];
            long nt = t.nt_ds;
            R *dst = s2buf[it].data();
            for (long b = 0; b < B; b++)
                memcpy(dst + b * pow2(rank) * nt, &s1buf[t.ipri][b * pow2(rk1) * nt], pow2(rank) * nt * sizeof(R));
            s2lags[ibatch * ntrees + it]->apply(dst, nt);

            // (B, 2^dd, 2^amb, T) -> transposed (B, 2^amb, 2^dd, T) for the stage-2 tree.
            long A2 = pow2(t.amb_rank), D2 = pow2(t.dd_rank);
            vector<R> tr(B * A2 * D2 * nt);
            for (long b = 0; b < B; b++)
                for (long f = 0; f < D2; f++)
                    for (long a = 0; a < A2; a++)
                        memcpy(&tr[((b * A2 + a) * D2 + f) * nt], dst + ((b * D2 + f) * A2 + a) * nt, nt * sizeof(R));
            s2k[it]->apply(tr.data(), sb[it].data(), ibatch);
            pfs[it]->apply(omax[it], oarg[it], sb[it].data(), wts[it], ibatch);
        }
    }
};


// -------------------------------------------------------------------------------------------------
// Ported reference self-tests (deterministic seeds instead of the reference's global RNG).


struct Rng
{
    std::mt19937_64 g;
    explicit Rng(uint64_t s) : g(s) { }
    long randint(long lo, long hi) { return std::uniform_int_distribution<long>(lo, hi - 1)(g); }
    double uniform(double lo, double hi) { return std::uniform_real_distribution<double>(lo, hi)(g); }
};

// ReferenceTree::test_basics (ReferenceTree.cpp:354-462): incremental tree == one-shot tree, and
// one-shot entries == brute-force sums over dedispersion_delay(). Returns max |difference|.
template<typename R>
static double test_tree_basics(uint64_t seed, long N, long B, long T, long S, long amb_rank, long dd_rank)
{
    Rng rng(seed);
    long A = pow2(amb_rank), D = pow2(dd_rank), NTS = N * T * S;
    vector<R> in(B * A * D * NTS);
    for (R &x : in) x = R(rng.uniform(-1, 1));

    vector<R> out_dni(in.size());
    vector<R> tmp(D * NTS);
    for (long b = 0; b < B; b++)
        for (long a = 0; a < A; a++) {
            memcpy(tmp.data(), &in[(b * A + a) * D * NTS], D * NTS * sizeof(R));
            dedisperse_non_incremental(tmp.data(), D, NTS, S);
            memcpy(&out_dni[(b * A + a) * D * NTS], tmp.data(), D * NTS * sizeof(R));
        }

    double maxerr = 0;
    for (int e = 0; e < 10; e++) {
        long b = rng.randint(0, B), a = rng.randint(0, A), t = rng.randint(0, N * T), dmb = rng.randint(0, D);
        R w = R(1) / std::sqrt(R(D));
        for (long s = 0; s < S; s++) {
            R acc = 0;
            for (long f = 0; f < D; f++) {
                long t0 = t - dedispersion_delay(dd_rank, f, dmb);
                if (t0 >= 0) acc += w * in[((b * A + a) * D + f) * NTS + t0 * S + s];
            }
            R got = out_dni[((b * A + a) * D + dmb) * NTS + t * S + s];
            maxerr = std::max(maxerr, double(std::fabs(got - acc)));
        }
    }

    RefTree<R> tree(B, amb_rank, dd_rank, T, S, {1});
    vector<R> chunk(B * A * D * T * S);
    for (long ic = 0; ic < N; ic++) {
        for (long i = 0; i < B * A * D; i++)
            memcpy(&chunk[i * T * S], &in[i * NTS + ic * T * S], T * S * sizeof(R));
        tree.dedisperse(chunk.data(), nullptr);
        for (long i = 0; i < B * A * D; i++)
            for (long k = 0; k < T * S; k++)
                maxerr = std::max(maxerr, double(std::fabs(chunk[i * T * S + k] - out_dni[i * NTS + ic * T * S + k])));
    }
    return maxerr;
}

// ReferenceTree::test_subbands (ReferenceTree.cpp:471-631): subband outputs == independent sub-trees.
template<typename R>
static double test_tree_subbands(uint64_t seed, const vector<long> &counts, long nchunks, long B, long T, long S,
                                 long amb_rank, long dd_rank)
{
    Rng rng(seed);
    Subbands fs(counts);
    ORC_ASSERT(dd_rank >= fs.pf_rank);
    long N = fs.N, M = fs.M, pf_rank = fs.pf_rank;
    long A = pow2(amb_rank), Din = pow2(dd_rank), Dpf = pow2(amb_rank + dd_rank - pf_rank), TS = T * S;

    RefTree<R> big(B, amb_rank, dd_rank, T, S, counts);
    vector<std::unique_ptr<RefTree<R>>> subs;
    for (long n = 0; n < N; n++) {
        long sz = (fs.n_to_fhi[n] - fs.n_to_flo[n]) << (dd_rank - pf_rank);
        subs.emplace_back(new RefTree<R>(B, amb_rank, ilog2(sz), T, S, {1}));
    }
    Lagbuf<R> lb(big.final_lagbuf->lags, TS);

    vector<R> in(B * A * Din * TS), buf(in.size()), out(B * Dpf * M * TS), out2(out.size());
    double maxerr = 0;
    for (long ic = 0; ic < nchunks; ic++) {
        for (R &x : in) x = R(rng.uniform(-1, 1));
        buf = in;
        big.dedisperse(buf.data(), out.data());
        for (long n = 0; n < N; n++) {
            long flo = fs.n_to_flo[n] << (dd_rank - pf_rank), fhi = fs.n_to_fhi[n] << (dd_rank - pf_rank);
            long lev = ilog2(fs.n_to_fhi[n] - fs.n_to_flo[n]);
            long sz = fhi - flo, srk = ilog2(sz);
            vector<R> dd(B * A * sz * TS);
            for (long b = 0; b < B; b++)
                for (long a = 0; a < A; a++)
                    memcpy(&dd[(b * A + a) * sz * TS], &in[((b * A + a) * Din + flo) * TS], sz * TS * sizeof(R));
            subs[n]->dedisperse(dd.data(), nullptr);
            for (long b = 0; b < B; b++)
                for (long a = 0; a < A; a++) {
                    long dmc = bit_reverse(a, amb_rank);
                    for (long d = 0; d < sz; d++) {
                        long dmf = bit_reverse(d, srk);
                        long dpf = (dmc << (dd_rank - pf_rank)) + (dmf >> lev);
                        long m = fs.n_to_mbase[n] + (dmf & (pow2(lev) - 1));
                        memcpy(&out2[((b * Dpf + dpf) * M + m) * TS], &dd[((b * A + a) * sz + d) * TS], TS * sizeof(R));
                    }
                }
            if (n == N - 1) {
                // Full band is last: the big tree's in-place output equals the full-band sub-tree.
                ORC_ASSERT(fs.n_to_flo[n] == 0 && fs.n_to_fhi[n] == pow2(pf_rank));
                for (size_t i = 0; i < buf.size(); i++)
                    maxerr = std::max(maxerr, double(std::fabs(buf[i] - dd[i])));
            }
        }
        lb.apply(out2.data(), TS);
        for (size_t i = 0; i < out.size(); i++)
            maxerr = std::max(maxerr, double(std::fabs(out[i] - out2[i])));
    }
    return maxerr;
}

// ReferenceLagbuf::test_random (ReferenceLagbuf.cpp:136-236): incremental == one-shot shift.
template<typename R>
static double test_lagbuf(uint64_t seed, long nrows, long nchunks, long ntime, long maxlag)
{
    Rng rng(seed);
    vector<int> lags(nrows);
    for (int &l : lags) l = int(rng.randint(0, maxlag + 1));
    Lagbuf<R> lb(lags, ntime);
    vector<R> all(nrows * nchunks * ntime);
    for (R &x : all) x = R(rng.uniform(-1, 1));
    vector<R> chunk(nrows * ntime);
    double maxerr = 0;
    for (long ic = 0; ic < nchunks; ic++) {
        for (long i = 0; i < nrows; i++)
            memcpy(&chunk[i * ntime], &all[(i * nchunks + ic) * ntime], ntime * sizeof(R));
        lb.apply(chunk.data(), ntime);
        for (long i = 0; i < nrows; i++)
            for (long t = 0; t < ntime; t++) {
                long ta = ic * ntime + t - lags[i];
                R expect = (ta >= 0) ? all[i * nchunks * ntime + ta] : R(0);
                maxerr = std::max(maxerr, double(std::fabs(chunk[i * ntime + t] - expect)));
            }
    }
    return maxerr;
}

}  // namespace orc


// -------------------------------------------------------------------------------------------------
// C API (ctypes)


using namespace orc;

// IEEE binary16 -> binary32, exact (every half is a float): sign, 5-bit exponent (bias 15), 10-bit
// fraction; subnormals are normalized, infinities and NaNs keep their class.
static float orc_half_to_float(uint16_t h)
{
    const uint32_t sign = uint32_t(h >> 15) << 31;
    const uint32_t e = (h >> 10) & 0x1f, frac = h & 0x3ff;
    uint32_t bits;
    if (e == 0x1f) {
        bits = sign | 0x7f800000u | (frac << 13);
    } else if (e != 0) {
        bits = sign | ((e - 15 + 127) << 23) | (frac << 13);
    } else if (frac == 0) {
        bits = sign;
    } else {
        int ee = -14;                 // value = frac * 2^-24 = 1.f * 2^(ee)
        uint32_t m = frac;
        while (!(m & 0x400)) { m <<= 1; ee--; }
        bits = sign | (uint32_t(ee + 127) << 23) | ((m & 0x3ff) << 13);
    }
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

// ReferenceDequantizationKernel::apply (src_lib/GpuDequantizationKernel.cu:326-380): int4 data
// (low nibble = even sample), one fp16 (scale, offset) pair per 256 samples of a (beam, freq) row,
// out = 0 for the sentinel -8, else scale * value + offset in fp32 (a multiply, then an add).
static void orc_dequantize_impl(const uint8_t *data, const uint16_t *scoff, float *out, long nbeams, long nfreq, long ntime)
{
    const long nchunks = ntime / 256;
    for (long row = 0; row < nbeams * nfreq; row++) {
        for (long c = 0; c < nchunks; c++) {
            const long pair = row * nchunks + c;
            const float scale = orc_half_to_float(scoff[2 * pair]), offset = orc_half_to_float(scoff[2 * pair + 1]);
            for (long it = 0; it < 256; it++) {
                const long i = (row * nchunks + c) * 256 + it;
                const uint8_t byte = data[i / 2];
                const int nib = (i % 2 == 0) ? (byte & 0x0f) : ((byte >> 4) & 0x0f);
                const int value = (nib >= 8) ? (nib - 16) : nib;
                const float prod = scale * float(value);
                out[i] = (value == -8) ? 0.0f : (prod + offset);
            }
        }
    }
}

struct orc_handle
{
    int real_bits;
    std::unique_ptr<Plan> plan;
    std::unique_ptr<Dedisperser<float>> d32;
    std::unique_ptr<Dedisperser<double>> d64;
};

static thread_local std::string orc_err;

extern "C" {

const char *orc_last_error() { return orc_err.c_str(); }

int orc_dequantize(const uint8_t *data, const uint16_t *scales_offsets, float *out, long nbeams, long nfreq, long ntime)
{
    if (ntime % 256) { orc_err = "orc_dequantize: ntime must be a multiple of 256"; return -1; }
    orc_dequantize_impl(data, scales_offsets, out, nbeams, nfreq, ntime);
    return 0;
}

float orc_half_to_float_c(uint16_t h) { return orc_half_to_float(h); }

// Primary tree i: ptrees[6*i .. 6*i+5] = (num_early_triggers, max_width, dm_downsampling,
// time_downsampling, wt_dm_downsampling, wt_time_downsampling).
void *orc_create(int nzones, const long *zone_nfreq, const double *zone_freq_edges, double time_sample_ms,
                 long toplevel_tree_rank, long time_samples_per_chunk, long nbits,
                 int nsb, const long *subband_counts, int npri, const long *ptrees,
                 long beams_per_gpu, long beams_per_batch, long dcore_max, int sophistication, int real_bits)
{
    try {
        Config c;
        c.zone_nfreq.assign(zone_nfreq, zone_nfreq + nzones);
        c.zone_freq_edges.assign(zone_freq_edges, zone_freq_edges + nzones + 1);
        c.time_sample_ms = time_sample_ms;
        c.toplevel_tree_rank = toplevel_tree_rank;
        c.time_samples_per_chunk = time_samples_per_chunk;
        c.nbits = nbits;
        c.subband_counts.assign(subband_counts, subband_counts + nsb);
        for (int i = 0; i < npri; i++) {
            const long *p = ptrees + 6 * i;
            c.primary_trees.push_back({p[0], p[1], p[2], p[3], p[4], p[5]});
        }
        c.beams_per_gpu = beams_per_gpu;
        c.beams_per_batch = beams_per_batch;
        orc_handle *h = new orc_handle;
        h->real_bits = real_bits;
        h->plan.reset(new Plan(c, dcore_max));
        if (real_bits == 32) h->d32.reset(new Dedisperser<float>(*h->plan, sophistication));
        else if (real_bits == 64) h->d64.reset(new Dedisperser<double>(*h->plan, sophistication));
        else throw runtime_error("real_bits must be 32 or 64");
        return h;
    } catch (std::exception &e) { orc_err = e.what(); return nullptr; }
}

void orc_destroy(void *h) { delete (orc_handle *) h; }

long orc_ntrees(void *h) { return ((orc_handle *) h)->plan->trees.size(); }

// info[16] = ipri, et_level, amb_rank, dd_rank, nt_ds, ndm_out, nt_out, ndm_wt, nt_wt, nprofiles,
//            N, M, Dcore, max_width, pf_rank, time_ds
int orc_tree_info(void *hv, long itree, long *info)
{
    orc_handle *h = (orc_handle *) hv;
    if (itree < 0 || itree >= (long) h->plan->trees.size()) return -1;
    const TreeInfo &t = h->plan->trees[itree];
    Subbands fs(t.sb_counts);
    long v[16] = { t.ipri, t.et_level, t.amb_rank, t.dd_rank, t.nt_ds, t.ndm_out, t.nt_out, t.ndm_wt, t.nt_wt,
                   t.nprofiles, fs.N, fs.M, t.Dcore, t.max_width, fs.pf_rank, t.time_ds };
    memcpy(info, v, sizeof(v));
    return 0;
}

// Channel map of the plan's tree gridding (length 2^rank + 1).
int orc_channel_map(void *hv, double *out)
{
    orc_handle *h = (orc_handle *) hv;
    vector<double> cm = h->plan->config.channel_map();
    memcpy(out, cm.data(), cm.size() * sizeof(double));
    return 0;
}

// Outputs are written as double regardless of the oracle's arithmetic type. tree_domain != 0: 'in' is
// tree-domain input (B, 2^toplevel_tree_rank, nt_in) instead of (B, nfreq, nt_in).
int orc_dedisperse(void *hv, long ibatch, const float *in, const float *const *wts, double *const *omax,
                   uint32_t *const *oarg, int tree_domain)
{
    try {
        orc_handle *h = (orc_handle *) hv;
        long nt = h->plan->trees.size();
        if (h->real_bits == 64) {
            h->d64->dedisperse(ibatch, in, wts, omax, oarg, tree_domain != 0);
            return 0;
        }
        vector<vector<float>> tmp(nt);
        vector<float *> ptrs(nt);
        for (long i = 0; i < nt; i++) {
            const TreeInfo &t = h->plan->trees[i];
            tmp[i].resize(h->plan->config.beams_per_batch * t.ndm_out * t.nt_out);
            ptrs[i] = tmp[i].data();
        }
        h->d32->dedisperse(ibatch, in, wts, ptrs.data(), oarg, tree_domain != 0);
        for (long i = 0; i < nt; i++)
            for (size_t k = 0; k < tmp[i].size(); k++)
                omax[i][k] = tmp[i][k];
        return 0;
    } catch (std::exception &e) { orc_err = e.what(); return -1; }
}

// Evaluates argmax tokens against the most recent dedisperse() call of tree 'itree'.
int orc_eval_tokens(void *hv, long itree, const uint32_t *tokens, const float *wt, double *out)
{
    try {
        orc_handle *h = (orc_handle *) hv;
        if (h->real_bits == 64) return h->d64->pfs.at(itree)->eval_tokens(out, tokens, wt);
        const PeakFinder<float> &pf = *h->d32->pfs.at(itree);
        vector<float> tmp(pf.B * pf.D * pf.nt_out);
        int rc = pf.eval_tokens(tmp.data(), tokens, wt);
        for (size_t k = 0; k < tmp.size(); k++) out[k] = tmp[k];
        return rc;
    } catch (std::exception &e) { orc_err = e.what(); return -1; }
}

// Stage-0 gridded output of the most recent call (sophistication 1 only), shape (B, 2^rank, nt).
int orc_gridded(void *hv, double *out)
{
    orc_handle *h = (orc_handle *) hv;
    if (h->real_bits == 64) { const auto &v = h->d64->s1buf.at(0); std::copy(v.begin(), v.end(), out); }
    else { const auto &v = h->d32->s1buf.at(0); std::copy(v.begin(), v.end(), out); }
    return 0;
}

// Peak-finder input (subband array) of tree 'itree' from the most recent call, (B, ndm_out, M, nt_ds).
int orc_pf_input(void *hv, long itree, double *out)
{
    orc_handle *h = (orc_handle *) hv;
    if (h->real_bits == 64) { const auto &v = h->d64->sb.at(itree); std::copy(v.begin(), v.end(), out); }
    else { const auto &v = h->d32->sb.at(itree); std::copy(v.begin(), v.end(), out); }
    return 0;
}

double orc_test_tree_basics(uint64_t seed, long N, long B, long T, long S, long amb, long dd, int real_bits)
{
    try {
        return (real_bits == 64) ? test_tree_basics<double>(seed, N, B, T, S, amb, dd)
                                 : test_tree_basics<float>(seed, N, B, T, S, amb, dd);
    } catch (std::exception &e) { orc_err = e.what(); return -1; }
}

double orc_test_tree_subbands(uint64_t seed, int nsb, const long *counts, long nchunks, long B, long T, long S,
                              long amb, long dd, int real_bits)
{
    try {
        vector<long> c(counts, counts + nsb);
        return (real_bits == 64) ? test_tree_subbands<double>(seed, c, nchunks, B, T, S, amb, dd)
                                 : test_tree_subbands<float>(seed, c, nchunks, B, T, S, amb, dd);
    } catch (std::exception &e) { orc_err = e.what(); return -1; }
}

double orc_test_lagbuf(uint64_t seed, long nrows, long nchunks, long ntime, long maxlag)
{
    try { return test_lagbuf<float>(seed, nrows, nchunks, ntime, maxlag); }
    catch (std::exception &e) { orc_err = e.what(); return -1; }
}

// Subband bookkeeping for tests: fills m_to_n, m_to_d (length M) and n_to_flo, n_to_fhi (length N).
int orc_subbands(int nsb, const long *counts, long *NM, long *m_to_n, long *m_to_d, long *n_to_flo, long *n_to_fhi)
{
    try {
        Subbands fs(vector<long>(counts, counts + nsb));
        NM[0] = fs.N; NM[1] = fs.M;
        if (m_to_n) for (long m = 0; m < fs.M; m++) { m_to_n[m] = fs.m_to_n[m]; m_to_d[m] = fs.m_to_d[m]; }
        if (n_to_flo) for (long n = 0; n < fs.N; n++) { n_to_flo[n] = fs.n_to_flo[n]; n_to_fhi[n] = fs.n_to_fhi[n]; }
        return 0;
    } catch (std::exception &e) { orc_err = e.what(); return -1; }
}

int orc_restrict_subbands(int nsb, const long *counts, long et_level, long new_pf_rank, long *out)
{
    try {
        vector<long> r = Subbands::restrict_counts(vector<long>(counts, counts + nsb), et_level, new_pf_rank);
        for (size_t i = 0; i < r.size(); i++) out[i] = r[i];
        return (int) r.size();
    } catch (std::exception &e) { orc_err = e.what(); return -1; }
}

}  // extern "C"
