// plan.cpp -- config parsing/validation and plan construction (see plan.hpp for reference citations).

#include "plan.hpp"
#include "yaml_lite.hpp"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <stdexcept>

namespace pb2 {

using std::runtime_error;
using std::string;
using std::vector;

#define PB2_REQUIRE(cond, msg) do { if (!(cond)) { std::stringstream _ss; _ss << msg; throw runtime_error(_ss.str()); } } while (0)

static constexpr int max_tree_rank = 16;         // include/pirate/constants.hpp:206
static constexpr int max_primary_trees = 7;      // include/pirate/constants.hpp:207
static constexpr int max_pf_width = 32;          // include/pirate/constants.hpp:208
static constexpr int max_peak_finding_rank = 4;  // include/pirate/constants.hpp:209
static constexpr double k_dm = 4.148808e6;       // include/pirate/constants.hpp:49
static constexpr long max_dcore = 8;             // production peak-finder granularity (makefile_helper.py:321)


string dtype_str(Dtype d)
{
    switch (d) {
    case Dtype::f32: return "float32";
    case Dtype::f16: return "float16";
    case Dtype::bf16: return "bfloat16";
    }
    return "?";
}

Dtype dtype_from_str(const string &s)
{
    if (s == "float32") return Dtype::f32;
    if (s == "float16") return Dtype::f16;
    if (s == "bfloat16") return Dtype::bf16;
    throw runtime_error("DedispersionConfig: invalid dtype '" + s + "' (expected float32, float16 or bfloat16)");
}

int integer_log2(long n)
{
    PB2_REQUIRE(is_pow2(n), "integer_log2: " << n << " is not a power of two");
    int p = 0;
    while ((1L << p) < n) p++;
    return p;
}

int bit_reverse(int i, int nbits)
{
    int j = 0;
    for (int b = 0; b < nbits; b++) { j = (j << 1) | (i & 1); i >>= 1; }
    return j;
}

// src_lib/utils.cpp:224
long rb_lag(long freq_coarse, long dm_brev, long stage1_rank, long stage2_rank, bool uflag)
{
    long ndm = pow2(stage1_rank), nfreq = pow2(stage2_rank);
    PB2_REQUIRE(freq_coarse >= 0 && freq_coarse < nfreq && dm_brev >= 0 && dm_brev < ndm, "rb_lag: bad index");
    long dm = bit_reverse(dm_brev, stage1_rank) + (uflag ? ndm : 0);
    return (nfreq - 1 - freq_coarse) * dm;
}


// -------------------------------------------------------------------------------------------------
// FrequencySubbands (src_lib/FrequencySubbands.cpp:32-216)


void FrequencySubbands::validate_subband_counts(const vector<long> &c)
{
    PB2_REQUIRE(c.size() > 0, "FrequencySubbands: empty subband_counts");
    long pr = c.size() - 1;
    PB2_REQUIRE(c[pr] == 1, "FrequencySubbands: last subband count must be 1 (the full band)");
    PB2_REQUIRE(pr <= max_peak_finding_rank, "FrequencySubbands: max allowed pf_rank is " << max_peak_finding_rank);
    for (long l = 0; l <= pr; l++) {
        long mx = (l > 0) ? (pow2(pr + 1 - l) - 1) : pow2(pr);
        PB2_REQUIRE(c[l] >= 0 && c[l] <= mx, "FrequencySubbands: subband_counts[" << l << "]=" << c[l] << " out of range [0," << mx << "]");
    }
}

FrequencySubbands::FrequencySubbands(const vector<long> &c) : subband_counts(c)
{
    validate_subband_counts(c);
    pf_rank = c.size() - 1;
    for (long l = 0; l <= pf_rank; l++)
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

FrequencySubbands::FrequencySubbands(const vector<long> &c, double fmin_, double fmax_) : FrequencySubbands(c)
{
    fmin = fmin_;
    fmax = fmax_;
    long nf = pow2(pf_rank) + 1;
    double a = pow(fmax, -2.0), b = pow(fmin, -2.0);
    for (long f = 0; f < nf; f++)
        f_to_freq.push_back(pow(a + (double(f) / double(nf - 1)) * (b - a), -0.5));
}

vector<long> FrequencySubbands::restrict_subband_counts(const vector<long> &c, long et_level, long new_pf_rank)
{
    validate_subband_counts(c);
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
    validate_subband_counts(dc);
    return dc;
}


// -------------------------------------------------------------------------------------------------
// DedispersionConfig (src_lib/DedispersionConfig.cpp)


long DedispersionConfig::get_total_nfreq() const
{
    long s = 0;
    for (long n : zone_nfreq) s += n;
    return s;
}

int DedispersionConfig::get_nelts_per_segment() const
{
    return 1024 / dtype_nbits(dtype);   // one 128-byte cache line
}

double DedispersionConfig::frequency_to_index(double freq) const
{
    double fmin = zone_freq_edges.front(), fmax = zone_freq_edges.back();
    double eps = 1.0e-5 * (fmax - fmin);
    PB2_REQUIRE(freq >= fmin - eps && freq <= fmax + eps,
                "DedispersionConfig::frequency_to_index(): frequency " << freq << " is out of range [" << fmin << ", " << fmax << "]");
    freq = std::min(std::max(freq, fmin), fmax);
    double off = 0;
    for (size_t i = 0; i < zone_nfreq.size(); i++) {
        double f0 = zone_freq_edges[i], f1 = zone_freq_edges[i + 1];
        if (freq <= f1) { off += (freq - f0) / (f1 - f0) * zone_nfreq[i]; break; }
        off += zone_nfreq[i];
    }
    return std::min(std::max(off, 0.0), double(get_total_nfreq()));
}

double DedispersionConfig::index_to_frequency(double index) const
{
    double tot = get_total_nfreq(), eps = 1.0e-5 * tot;
    PB2_REQUIRE(index >= -eps && index <= tot + eps, "DedispersionConfig::index_to_frequency(): index " << index << " is out of range [0, " << tot << "]");
    index = std::min(std::max(index, 0.0), tot);
    double off = 0;
    for (size_t i = 0; i < zone_nfreq.size(); i++) {
        double next = off + zone_nfreq[i];
        if (index <= next) {
            double frac = (index - off) / zone_nfreq[i];
            return zone_freq_edges[i] + frac * (zone_freq_edges[i + 1] - zone_freq_edges[i]);
        }
        off = next;
    }
    return zone_freq_edges.back();
}

double DedispersionConfig::delay_to_frequency(double delay) const
{
    double flo = zone_freq_edges.front(), fhi = zone_freq_edges.back();
    double ntree = pow2(toplevel_tree_rank), eps = 1.0e-5 * ntree;
    PB2_REQUIRE(delay >= -eps && delay <= ntree + eps, "DedispersionConfig::delay_to_frequency(): delay " << delay << " is out of range [0, " << ntree << "]");
    delay = std::min(std::max(delay, 0.0), ntree);
    double scale = ntree / (1.0 / (flo * flo) - 1.0 / (fhi * fhi));
    return 1.0 / sqrt(delay / scale + 1.0 / (fhi * fhi));
}

double DedispersionConfig::frequency_to_delay(double freq) const
{
    double flo = zone_freq_edges.front(), fhi = zone_freq_edges.back();
    double ntree = pow2(toplevel_tree_rank), eps = 1.0e-5 * (fhi - flo);
    PB2_REQUIRE(freq >= flo - eps && freq <= fhi + eps, "DedispersionConfig::frequency_to_delay(): frequency " << freq << " is out of range");
    freq = std::min(std::max(freq, flo), fhi);
    double d = 1.0 / (freq * freq), dlo = 1.0 / (flo * flo), dhi = 1.0 / (fhi * fhi);
    return ntree * (d - dhi) / (dlo - dhi);
}

double DedispersionConfig::dm_per_unit_delay() const
{
    double flo = zone_freq_edges.front(), fhi = zone_freq_edges.back();
    return time_sample_ms / (k_dm * (1.0 / (flo * flo) - 1.0 / (fhi * fhi)));
}

vector<double> DedispersionConfig::make_channel_map() const
{
    long nchan = pow2(toplevel_tree_rank);
    vector<double> cm(nchan + 1);
    for (long n = 0; n <= nchan; n++)
        cm[n] = frequency_to_index(delay_to_frequency(n));
    return cm;
}

// src_lib/DedispersionConfig.cpp:333-435, plus the B200 kernels' own limits.
void DedispersionConfig::validate() const
{
    PB2_REQUIRE(toplevel_tree_rank > 0, "DedispersionConfig: toplevel_tree_rank must be > 0");
    PB2_REQUIRE(primary_trees.size() > 0, "DedispersionConfig: primary_trees must be nonempty");
    PB2_REQUIRE(time_samples_per_chunk > 0, "DedispersionConfig: time_samples_per_chunk must be > 0");
    PB2_REQUIRE(time_sample_ms > 0, "DedispersionConfig: time_sample_ms must be > 0");
    PB2_REQUIRE(beams_per_gpu > 0 && beams_per_batch > 0 && num_active_batches > 0, "DedispersionConfig: beam counts must be > 0");
    PB2_REQUIRE(toplevel_tree_rank <= max_tree_rank, "DedispersionConfig: toplevel_tree_rank must be <= " << max_tree_rank);
    PB2_REQUIRE(num_primary_trees() <= max_primary_trees, "DedispersionConfig: at most " << max_primary_trees << " primary trees");
    PB2_REQUIRE(zone_nfreq.size() > 0 && zone_freq_edges.size() == zone_nfreq.size() + 1, "DedispersionConfig: zone_freq_edges must have length len(zone_nfreq)+1");
    for (long n : zone_nfreq) PB2_REQUIRE(n > 0, "DedispersionConfig: zone_nfreq entries must be > 0");
    for (size_t i = 0; i + 1 < zone_freq_edges.size(); i++)
        PB2_REQUIRE(zone_freq_edges[i] > 0 && zone_freq_edges[i] < zone_freq_edges[i + 1], "DedispersionConfig: zone_freq_edges must be positive and increasing");

    int nps = get_nelts_per_segment();
    long min_nt = nps * pow2(num_primary_trees() - 1);
    PB2_REQUIRE(time_samples_per_chunk % min_nt == 0, "DedispersionConfig: time_samples_per_chunk=" << time_samples_per_chunk
                << " must be a multiple of " << min_nt << " (this value depends on dtype and the number of primary trees)");
    PB2_REQUIRE(beams_per_gpu % beams_per_batch == 0, "DedispersionConfig: beams_per_gpu must be a multiple of beams_per_batch");
    PB2_REQUIRE(num_active_batches * beams_per_batch <= beams_per_gpu, "DedispersionConfig: num_active_batches * beams_per_batch must be <= beams_per_gpu");
    PB2_REQUIRE(max_gpu_clag >= 0 && future_write_max_samples >= 0, "DedispersionConfig: max_gpu_clag and future_write_max_samples must be >= 0");
    FrequencySubbands::validate_subband_counts(frequency_subband_counts);

    for (long ipri = 0; ipri < num_primary_trees(); ipri++) {
        const PrimaryTree &pt = primary_trees[ipri];
        long ptr = ipri ? (toplevel_tree_rank - 1) : toplevel_tree_rank;
        long s1dd = ptr / 2;
        PB2_REQUIRE(pt.num_early_triggers >= 0 && pt.num_early_triggers <= ptr - s1dd,
                    "DedispersionConfig: num_early_triggers[" << ipri << "] must be in [0," << (ptr - s1dd) << "]");
        PB2_REQUIRE(pt.max_width > 0 && is_pow2(pt.max_width) && pt.max_width <= max_pf_width,
                    "DedispersionConfig: max_width[" << ipri << "] must be a power of two <= " << max_pf_width);
        PB2_REQUIRE(pt.wt_dm_downsampling > 0 && is_pow2(pt.wt_dm_downsampling), "DedispersionConfig: wt_dm_downsampling must be a power of two");
        PB2_REQUIRE(pt.wt_time_downsampling > 0 && is_pow2(pt.wt_time_downsampling), "DedispersionConfig: wt_time_downsampling must be a power of two");
        long min_rank = ptr - pt.num_early_triggers;
        PB2_REQUIRE(pt.wt_dm_downsampling <= pow2(min_rank), "DedispersionConfig: wt_dm_downsampling[" << ipri << "]=" << pt.wt_dm_downsampling
                    << " must be <= " << pow2(min_rank) << ". This upper bound is set by the smallest tree at primary_tree_index=" << ipri << " (i.e. the earliest trigger).");
        if (pt.dm_downsampling > 0)
            PB2_REQUIRE(is_pow2(pt.dm_downsampling) && pt.wt_dm_downsampling >= pt.dm_downsampling, "DedispersionConfig: bad dm_downsampling");
        if (pt.time_downsampling > 0)
            PB2_REQUIRE(is_pow2(pt.time_downsampling) && pt.wt_time_downsampling >= pt.time_downsampling, "DedispersionConfig: bad time_downsampling");
    }
}

static string fmt_double(double x)
{
    std::stringstream ss;
    ss << std::setprecision(17) << x;
    return ss.str();
}

template<typename T>
static string flow_list(const vector<T> &v)
{
    std::stringstream ss;
    ss << "[";
    for (size_t i = 0; i < v.size(); i++) ss << (i ? ", " : "") << v[i];
    ss << "]";
    return ss.str();
}

string DedispersionConfig::to_yaml_string() const
{
    validate();
    std::stringstream ss;
    vector<string> edges;
    for (double e : zone_freq_edges) edges.push_back(fmt_double(e));
    ss << "zone_nfreq: " << flow_list(zone_nfreq) << "\n"
       << "zone_freq_edges: " << flow_list(edges) << "\n"
       << "time_sample_ms: " << fmt_double(time_sample_ms) << "\n"
       << "toplevel_tree_rank: " << toplevel_tree_rank << "\n"
       << "time_samples_per_chunk: " << time_samples_per_chunk << "\n"
       << "dtype: " << dtype_str(dtype) << "\n"
       << "frequency_subband_counts: " << flow_list(frequency_subband_counts) << "\n"
       << "primary_trees:\n";
    for (const PrimaryTree &p : primary_trees)
        ss << "  - {num_early_triggers: " << p.num_early_triggers << ", max_width: " << p.max_width
           << ", dm_downsampling: " << p.dm_downsampling << ", time_downsampling: " << p.time_downsampling
           << ", wt_dm_downsampling: " << p.wt_dm_downsampling << ", wt_time_downsampling: " << p.wt_time_downsampling << "}\n";
    ss << "beams_per_gpu: " << beams_per_gpu << "\n"
       << "beams_per_batch: " << beams_per_batch << "\n"
       << "num_active_batches: " << num_active_batches << "\n"
       << "future_write_max_samples: " << future_write_max_samples << "\n"
       << "max_gpu_clag: " << max_gpu_clag << "\n";
    return ss.str();
}

static const yaml::Node *req(const yaml::Node *m, const string &k, const string &name)
{
    const yaml::Node *n = m->get(k);
    PB2_REQUIRE(n, name << ": missing required key '" << k << "'");
    return n;
}

static long as_long(const yaml::Node *n, const string &what)
{
    PB2_REQUIRE(n && n->kind == yaml::Node::Scalar, what << ": expected an integer");
    char *end = nullptr;
    long v = strtol(n->scalar.c_str(), &end, 10);
    PB2_REQUIRE(end && *end == 0 && !n->scalar.empty(), what << ": expected an integer, got '" << n->scalar << "'");
    return v;
}

static double as_double(const yaml::Node *n, const string &what)
{
    PB2_REQUIRE(n && n->kind == yaml::Node::Scalar, what << ": expected a number");
    char *end = nullptr;
    double v = strtod(n->scalar.c_str(), &end);
    PB2_REQUIRE(end && *end == 0 && !n->scalar.empty(), what << ": expected a number, got '" << n->scalar << "'");
    return v;
}

template<typename T, typename F>
static vector<T> as_vec(const yaml::Node *n, const string &what, F conv)
{
    PB2_REQUIRE(n && n->kind == yaml::Node::Seq, what << ": expected a list");
    vector<T> v;
    for (auto &e : n->seq) v.push_back(conv(e.get(), what));
    return v;
}

// src_lib/DedispersionConfig.cpp:651-735 (same keys, same old-syntax errors, same unknown-key check).
DedispersionConfig DedispersionConfig::from_yaml_string(const string &text, const string &name)
{
    yaml::NodeP root = yaml::parse(text, name);
    PB2_REQUIRE(root->kind == yaml::Node::Map, name << ": top level must be a mapping");
    const yaml::Node *f = root.get();
    if (f->get("tree_rank"))
        throw runtime_error(name + ": key 'tree_rank' is from an old config syntax -- it has been renamed to 'toplevel_tree_rank' (same meaning).");
    for (const char *k : {"peak_finding_params", "early_triggers", "num_downsampling_levels"})
        if (f->get(k))
            throw runtime_error(name + ": key '" + k + "' is from an old config syntax. The keys 'peak_finding_params', "
                                "'early_triggers', and 'num_downsampling_levels' have been replaced by 'primary_trees'.");

    static const vector<string> known = {"zone_nfreq", "zone_freq_edges", "time_sample_ms", "toplevel_tree_rank",
        "time_samples_per_chunk", "dtype", "beams_per_gpu", "beams_per_batch", "num_active_batches",
        "future_write_max_samples", "max_gpu_clag", "frequency_subband_counts", "primary_trees"};
    for (auto &kv : f->map)
        PB2_REQUIRE(std::find(known.begin(), known.end(), kv.first) != known.end(), name << ": invalid key '" << kv.first << "'");

    DedispersionConfig c;
    c.zone_nfreq = as_vec<long>(req(f, "zone_nfreq", name), "zone_nfreq", as_long);
    c.zone_freq_edges = as_vec<double>(req(f, "zone_freq_edges", name), "zone_freq_edges", as_double);
    c.time_sample_ms = as_double(req(f, "time_sample_ms", name), "time_sample_ms");
    c.toplevel_tree_rank = as_long(req(f, "toplevel_tree_rank", name), "toplevel_tree_rank");
    c.time_samples_per_chunk = as_long(req(f, "time_samples_per_chunk", name), "time_samples_per_chunk");
    const yaml::Node *dt = req(f, "dtype", name);
    PB2_REQUIRE(dt->kind == yaml::Node::Scalar, name << ": dtype must be a string");
    c.dtype = dtype_from_str(dt->scalar);
    c.beams_per_gpu = as_long(req(f, "beams_per_gpu", name), "beams_per_gpu");
    c.beams_per_batch = as_long(req(f, "beams_per_batch", name), "beams_per_batch");
    c.num_active_batches = as_long(req(f, "num_active_batches", name), "num_active_batches");
    c.future_write_max_samples = as_long(req(f, "future_write_max_samples", name), "future_write_max_samples");
    if (f->get("max_gpu_clag")) c.max_gpu_clag = as_long(f->get("max_gpu_clag"), "max_gpu_clag");
    c.frequency_subband_counts = as_vec<long>(req(f, "frequency_subband_counts", name), "frequency_subband_counts", as_long);

    const yaml::Node *pts = req(f, "primary_trees", name);
    PB2_REQUIRE(pts->kind == yaml::Node::Seq, name << ": primary_trees must be a list");
    static const vector<string> pknown = {"num_early_triggers", "max_width", "dm_downsampling", "time_downsampling",
                                          "wt_dm_downsampling", "wt_time_downsampling"};
    for (auto &pn : pts->seq) {
        PB2_REQUIRE(pn->kind == yaml::Node::Map, name << ": each primary_trees entry must be a mapping");
        for (auto &kv : pn->map)
            PB2_REQUIRE(std::find(pknown.begin(), pknown.end(), kv.first) != pknown.end(), name << ": invalid key '" << kv.first << "' in primary_trees");
        PrimaryTree p;
        p.num_early_triggers = as_long(req(pn.get(), "num_early_triggers", name), "num_early_triggers");
        p.max_width = as_long(req(pn.get(), "max_width", name), "max_width");
        p.dm_downsampling = pn->get("dm_downsampling") ? as_long(pn->get("dm_downsampling"), "dm_downsampling") : 0;
        p.time_downsampling = pn->get("time_downsampling") ? as_long(pn->get("time_downsampling"), "time_downsampling") : 0;
        p.wt_dm_downsampling = as_long(req(pn.get(), "wt_dm_downsampling", name), "wt_dm_downsampling");
        p.wt_time_downsampling = as_long(req(pn.get(), "wt_time_downsampling", name), "wt_time_downsampling");
        c.primary_trees.push_back(p);
    }
    c.validate();
    return c;
}

DedispersionConfig DedispersionConfig::from_yaml(const string &filename)
{
    std::ifstream f(filename);
    PB2_REQUIRE(f.good(), "DedispersionConfig::from_yaml(): could not open '" << filename << "'");
    std::stringstream ss;
    ss << f.rdbuf();
    return from_yaml_string(ss.str(), filename);
}


// -------------------------------------------------------------------------------------------------
// DedispersionPlan (src_lib/DedispersionPlan.cpp:29-146)


DedispersionPlan::DedispersionPlan(const DedispersionConfig &cfg) : config(cfg)
{
    config.validate();
    dtype = config.dtype;
    nfreq = config.get_total_nfreq();
    nt_in = config.time_samples_per_chunk;
    num_primary_trees = config.num_primary_trees();
    beams_per_gpu = config.beams_per_gpu;
    beams_per_batch = config.beams_per_batch;
    num_active_batches = config.num_active_batches;
    nbits = dtype_nbits(dtype);
    nelts_per_segment = config.get_nelts_per_segment();
    nbytes_per_segment = 128;

    for (long ipri = 0; ipri < num_primary_trees; ipri++) {
        int ptr = ipri ? (config.toplevel_tree_rank - 1) : config.toplevel_tree_rank;
        int s1dd = ptr / 2, s1amb = ptr - s1dd;
        stage1_dd_rank.push_back(s1dd);
        stage1_amb_rank.push_back(s1amb);
        long net = config.primary_trees[ipri].num_early_triggers;

        for (long et = net; et >= 0; et--) {
            DedispersionTree t;
            t.primary_tree_index = ipri;
            t.early_trigger_level = et;
            t.amb_rank = s1dd;
            t.dd_rank = s1amb - et;
            t.nt_ds = nt_in / pow2(ipri);
            PB2_REQUIRE(t.dd_rank >= 1, "DedispersionPlan: tree dd_rank must be >= 1");
            long tot_rank = t.total_rank();
            long pf_rank = (t.dd_rank + 1) / 2;
            double fmin = config.delay_to_frequency(pow2(config.toplevel_tree_rank - et));
            double fmax = config.zone_freq_edges.back();
            vector<long> sc = FrequencySubbands::restrict_subband_counts(config.frequency_subband_counts, et, pf_rank);
            t.frequency_subbands = FrequencySubbands(sc, fmin, fmax);
            t.pf = config.primary_trees[ipri];
            if (t.pf.dm_downsampling == 0) t.pf.dm_downsampling = pow2(pf_rank);
            if (t.pf.time_downsampling == 0) t.pf.time_downsampling = t.pf.dm_downsampling;

            // The stage-2 subband tree emits one output row per (coarse dm, multiplet), i.e. its DM
            // axis is downsampled by exactly 2^pf_rank; pirate's reference dedisperser has the same
            // requirement (ReferenceDedispersionKernel::_check_sb_out, DedispersionKernel.cu:338).
            PB2_REQUIRE(t.pf.dm_downsampling == pow2(pf_rank), "DedispersionPlan: dm_downsampling[" << ipri << "]=" << t.pf.dm_downsampling
                        << " must be 0 or 2^pf_rank=" << pow2(pf_rank));
            PB2_REQUIRE(t.pf.dm_downsampling <= t.pf.wt_dm_downsampling && t.pf.wt_dm_downsampling <= pow2(tot_rank), "DedispersionPlan: bad wt_dm_downsampling");
            PB2_REQUIRE(t.pf.time_downsampling <= t.pf.wt_time_downsampling && t.pf.wt_time_downsampling <= t.nt_ds, "DedispersionPlan: bad wt_time_downsampling");
            PB2_REQUIRE(t.nt_ds % t.pf.wt_time_downsampling == 0, "DedispersionPlan: nt_ds must be divisible by wt_time_downsampling");
            PB2_REQUIRE(t.pf.time_downsampling <= 64, "DedispersionPlan: time_downsampling must be <= 64 (B200 peak finder window)");

            t.nprofiles = 1 + 3 * integer_log2(t.pf.max_width);
            t.ndm_out = pow2(tot_rank) / t.pf.dm_downsampling;
            t.ndm_wt = pow2(tot_rank) / t.pf.wt_dm_downsampling;
            t.nt_out = t.nt_ds / t.pf.time_downsampling;
            t.nt_wt = t.nt_ds / t.pf.wt_time_downsampling;
            t.Dcore = std::min(t.pf.time_downsampling, max_dcore);
            double dm0 = config.dm_per_unit_delay() * pow2(config.toplevel_tree_rank);
            t.dm_min = dm0 * ((ipri > 0) ? pow2(ipri - 1) : 0);
            t.dm_max = dm0 * pow2(ipri);
            t.trigger_frequency = fmin;
            trees.push_back(t);
        }
    }
    ntrees = trees.size();

    max_row_lag.resize(num_primary_trees);
    for (long ipri = 0; ipri < num_primary_trees; ipri++)
        max_row_lag[ipri].assign(pow2(stage1_dd_rank[ipri] + stage1_amb_rank[ipri]), 0);
    for (const DedispersionTree &t : trees) {
        long ip = t.primary_tree_index;
        for (long a = 0; a < pow2(t.dd_rank); a++)
            for (long d = 0; d < pow2(t.amb_rank); d++) {
                long row = a * pow2(t.amb_rank) + d;
                max_row_lag[ip][row] = std::max(max_row_lag[ip][row], rb_lag(a, d, t.amb_rank, t.dd_rank, ip > 0));
            }
    }
}

// src_lib/DedispersionPlan.cpp:481-540
void DedispersionPlan::decode_argmax(uint32_t token, long itree, long idm, long it,
                                     long &fmin, long &fmax, long &tlo, long &thi, long &p) const
{
    PB2_REQUIRE(itree >= 0 && itree < ntrees, "decode_argmax: itree out of range");
    const DedispersionTree &tr = trees[itree];
    const FrequencySubbands &fs = tr.frequency_subbands;
    PB2_REQUIRE(idm >= 0 && idm < tr.ndm_out, "decode_argmax: idm out of range");
    PB2_REQUIRE(it >= 0 && it < tr.nt_out, "decode_argmax: itime out of range");
    long Dout = tr.nt_ds / tr.nt_out;
    long m = (token >> 16) & 0xffff;
    p = (token >> 8) & 0xff;
    long t = token & 0xff;
    PB2_REQUIRE(m < fs.M, "decode_argmax: bad token (m out of range)");
    PB2_REQUIRE(p < tr.nprofiles, "decode_argmax: bad token (p out of range)");
    PB2_REQUIRE(t < Dout, "decode_argmax: bad token (t out of range)");
    long lpf = p ? (p - 1) / 3 : 0;
    long dt = std::min(tr.Dcore, pow2(lpf));
    PB2_REQUIRE(t % dt == 0, "decode_argmax: bad token (t not a multiple of dt)");
    long n = fs.m_to_n[m], dfine = fs.m_to_d[m];
    long flo = fs.n_to_flo[n], fhi = fs.n_to_fhi[n];
    long lsb = integer_log2(fhi - flo);
    long ipri = tr.primary_tree_index;
    long rr = tr.total_rank() + ((ipri > 0) ? 1 : 0);
    long G = pow2(rr - fs.pf_rank);
    fmin = flo * G;
    fmax = fhi * G - 1;
    long dhi = idm + ((ipri > 0) ? tr.ndm_out : 0);
    long Tpf = it * Dout + t + dt - 1;
    long thi_ds = Tpf - (pow2(fs.pf_rank) - fhi) * dhi;
    long tlo_ds = thi_ds - (dhi * pow2(lsb) + dfine);
    thi = (thi_ds + 1) << ipri;
    tlo = (tlo_ds + 1) << ipri;
}

// src_lib/DedispersionPlan.cpp:544-611
void DedispersionPlan::decode_argmax2(long itree, long fmin, long fmax, long tlo, long thi, long p,
                                      double &freq_lo, double &freq_hi, double &dm, double &timestamp, double &width) const
{
    PB2_REQUIRE(itree >= 0 && itree < ntrees, "decode_argmax2: itree out of range");
    long ntree = pow2(config.toplevel_tree_rank);
    long ipri = trees[itree].primary_tree_index;
    PB2_REQUIRE(fmin >= 0 && fmin < fmax && fmax < ntree && tlo <= thi && p >= 0 && p < trees[itree].nprofiles, "decode_argmax2: bad arguments");
    double dslope = double(thi - tlo) / double(fmax - fmin);
    long pdiv = p / 3, pmod = p - 3 * pdiv;
    double pw, psh;
    if (p == 0) { pw = 1.0 * (1 << ipri); psh = 0.5 * (1 << ipri); }
    else if (pmod == 1) { pw = 1.0 * (1 << (ipri + pdiv + 1)); psh = 0.5 * (1 << (ipri + pdiv + 1)); }
    else if (pmod == 2) { pw = 2.0 * (1 << (ipri + pdiv)); psh = 1.5 * (1 << (ipri + pdiv)); }
    else { pw = 3.0 * (1 << (ipri + pdiv - 1)); psh = 2.0 * (1 << (ipri + pdiv - 1)); }
    freq_lo = config.delay_to_frequency(fmax + 1);
    freq_hi = config.delay_to_frequency(fmin);
    dm = dslope * ntree * config.dm_per_unit_delay();
    timestamp = thi + dslope * (ntree - 0.5 - fmax) - psh;
    width = pw;
}

// src_lib/DedispersionPlan.cpp:634-657
vector<long> DedispersionPlan::compute_steady_state_it0(long itree) const
{
    PB2_REQUIRE(itree >= 0 && itree < ntrees, "compute_steady_state_it0: itree out of range");
    const DedispersionTree &tr = trees[itree];
    long p = tr.primary_tree_index, e = tr.early_trigger_level;
    long T_ds = tr.pf.time_downsampling, D_ds = tr.pf.dm_downsampling, Wmax = tr.pf.max_width;
    long d_lo = (p > 0) ? pow2(config.toplevel_tree_rank + p - 1) : 0;
    long d0 = d_lo / pow2(e + p);
    vector<long> ret(tr.ndm_out);
    for (long idm = 0; idm < tr.ndm_out; idm++) {
        long dmax = d0 + (idm + 1) * D_ds - 1;
        ret[idm] = (dmax + 4 * Wmax + T_ds - 1) / T_ds;
    }
    return ret;
}

string DedispersionPlan::to_yaml_string() const
{
    std::stringstream ss;
    ss << "dtype: " << dtype_str(dtype) << "\n"
       << "nfreq: " << nfreq << "\n"
       << "nt_in: " << nt_in << "\n"
       << "toplevel_tree_rank: " << config.toplevel_tree_rank << "\n"
       << "num_primary_trees: " << num_primary_trees << "\n"
       << "beams_per_gpu: " << beams_per_gpu << "\n"
       << "beams_per_batch: " << beams_per_batch << "\n"
       << "num_active_batches: " << num_active_batches << "\n"
       << "stage1_dd_rank: " << flow_list(stage1_dd_rank) << "\n"
       << "stage1_amb_rank: " << flow_list(stage1_amb_rank) << "\n"
       << "ntrees: " << ntrees << "\n"
       << "trees:\n";
    for (long i = 0; i < ntrees; i++) {
        const DedispersionTree &t = trees[i];
        ss << "  - tree_index: " << i << "\n"
           << "    ndm_out: " << t.ndm_out << "\n"
           << "    nt_out: " << t.nt_out << "\n"
           << "    dm_min: " << fmt_double(t.dm_min) << "\n"
           << "    dm_max: " << fmt_double(t.dm_max) << "\n"
           << "    trigger_frequency: " << fmt_double(t.trigger_frequency) << "\n"
           << "    primary_tree_index: " << t.primary_tree_index << "\n"
           << "    early_trigger_level: " << t.early_trigger_level << "\n"
           << "    amb_rank: " << t.amb_rank << "\n"
           << "    dd_rank: " << t.dd_rank << "\n"
           << "    nt_ds: " << t.nt_ds << "\n"
           << "    max_width: " << t.pf.max_width << "\n"
           << "    dm_downsampling: " << t.pf.dm_downsampling << "\n"
           << "    time_downsampling: " << t.pf.time_downsampling << "\n"
           << "    Dcore: " << t.Dcore << "\n"
           << "    nprofiles: " << t.nprofiles << "\n"
           << "    wt_dm_downsampling: " << t.pf.wt_dm_downsampling << "\n"
           << "    wt_time_downsampling: " << t.pf.wt_time_downsampling << "\n"
           << "    ndm_wt: " << t.ndm_wt << "\n"
           << "    nt_wt: " << t.nt_wt << "\n"
           << "    frequency_subband_counts: " << flow_list(t.frequency_subbands.subband_counts) << "\n";
    }
    long N = 0;
    for (const DedispersionTree &t : trees) N += t.ndm_out * t.nt_out;
    double T = 1.0e-3 * config.time_samples_per_chunk * config.time_sample_ms;
    double gbps = 1.0e-9 * N * beams_per_gpu * (4 + nbits / 8) / T;
    ss << "dedispersion_outputs: " << std::fixed << std::setprecision(3) << gbps << " GB/s\n";
    return ss.str();
}

}  // namespace pb2
