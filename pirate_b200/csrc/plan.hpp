// plan.hpp -- DedispersionConfig / FrequencySubbands / DedispersionPlan for the B200 dedisperser.
//
// Same YAML schema, validation rules and derived quantities as pirate's
//   include/pirate/DedispersionConfig.hpp:21-194   (config, channel map, delay maps)
//   include/pirate/FrequencySubbands.hpp:22-100     (subbands / multiplets)
//   include/pirate/DedispersionTree.hpp:19-59       (per-output-tree shapes)
//   include/pirate/DedispersionPlan.hpp:33-225      (plan, decode_argmax, steady-state)
// The plan does not build pirate's MegaRingbuf: lag storage is laid out by the GPU dedisperser
// (one delay line per stage-1 output row, see dedisperser.cu).

#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace pb2 {

enum class Dtype : int { f32 = 0, f16 = 1, bf16 = 2 };

std::string dtype_str(Dtype d);
Dtype dtype_from_str(const std::string &s);
inline int dtype_nbits(Dtype d) { return (d == Dtype::f32) ? 32 : 16; }

inline long pow2(long n) { return 1L << n; }
inline bool is_pow2(long n) { return (n > 0) && !(n & (n - 1)); }
int integer_log2(long n);
int bit_reverse(int i, int nbits);
long rb_lag(long freq_coarse, long dm_brev, long stage1_rank, long stage2_rank, bool uflag);

struct FrequencySubbands
{
    std::vector<long> subband_counts;
    long pf_rank = -1, N = 0, M = 0;
    std::vector<long> m_to_n, m_to_d, n_to_flo, n_to_fhi, n_to_mbase;
    std::vector<double> f_to_freq;
    double fmin = 0, fmax = 0;

    FrequencySubbands() : FrequencySubbands(std::vector<long>{1}) { }
    explicit FrequencySubbands(const std::vector<long> &counts);
    FrequencySubbands(const std::vector<long> &counts, double fmin, double fmax);

    long m_to_flo(long m) const { return n_to_flo.at(m_to_n.at(m)); }
    long m_to_fhi(long m) const { return n_to_fhi.at(m_to_n.at(m)); }

    static void validate_subband_counts(const std::vector<long> &counts);
    static std::vector<long> restrict_subband_counts(const std::vector<long> &counts, long et_level, long new_pf_rank);
};

struct PrimaryTree
{
    long num_early_triggers = 0;
    long max_width = 0;
    long dm_downsampling = 0;
    long time_downsampling = 0;
    long wt_dm_downsampling = 0;
    long wt_time_downsampling = 0;
};

struct DedispersionConfig
{
    std::vector<long> zone_nfreq;
    std::vector<double> zone_freq_edges;
    double time_sample_ms = 0.0;
    long toplevel_tree_rank = -1;
    long time_samples_per_chunk = 0;
    Dtype dtype = Dtype::f32;
    std::vector<long> frequency_subband_counts;
    std::vector<PrimaryTree> primary_trees;
    long beams_per_gpu = 0;
    long beams_per_batch = 0;
    long num_active_batches = 0;
    long future_write_max_samples = 0;
    long max_gpu_clag = 10000;

    long num_primary_trees() const { return primary_trees.size(); }
    long get_total_nfreq() const;
    int get_nelts_per_segment() const;

    void validate() const;
    std::string to_yaml_string() const;
    static DedispersionConfig from_yaml_string(const std::string &text, const std::string &name = "config");
    static DedispersionConfig from_yaml(const std::string &filename);

    double frequency_to_index(double freq) const;
    double index_to_frequency(double index) const;
    double delay_to_frequency(double delay) const;
    double frequency_to_delay(double freq) const;
    double dm_per_unit_delay() const;
    std::vector<double> make_channel_map() const;
};

struct DedispersionTree
{
    int primary_tree_index = -1;
    int early_trigger_level = -1;
    int amb_rank = 0;
    int dd_rank = 0;
    int nt_ds = 0;
    long total_rank() const { return amb_rank + dd_rank; }

    FrequencySubbands frequency_subbands;
    PrimaryTree pf;
    long Dcore = 0;
    long nprofiles = 0;
    long ndm_out = 0, ndm_wt = 0, nt_out = 0, nt_wt = 0;
    double dm_min = 0, dm_max = 0, trigger_frequency = 0;
};

struct DedispersionPlan
{
    DedispersionConfig config;
    Dtype dtype = Dtype::f32;
    long nfreq = 0, nt_in = 0, num_primary_trees = 0, beams_per_gpu = 0, beams_per_batch = 0,
         num_active_batches = 0, nbits = 0;
    std::vector<long> stage1_dd_rank, stage1_amb_rank;
    long ntrees = 0;
    std::vector<DedispersionTree> trees;
    int nelts_per_segment = 0;
    int nbytes_per_segment = 0;

    // Largest lag (in tree samples) of stage-1 output row (a, dm_brev) over the stage-2 trees that
    // read it, per primary tree; row index a * 2^stage1_dd_rank + dm_brev.
    std::vector<std::vector<long>> max_row_lag;

    explicit DedispersionPlan(const DedispersionConfig &config);

    void decode_argmax(uint32_t token, long itree, long idm, long it,
                       long &fmin, long &fmax, long &tlo, long &thi, long &p) const;
    void decode_argmax2(long itree, long fmin, long fmax, long tlo, long thi, long p,
                        double &freq_lo, double &freq_hi, double &dm, double &timestamp, double &width) const;
    std::vector<long> compute_steady_state_it0(long itree) const;
    std::string to_yaml_string() const;
};

}  // namespace pb2
