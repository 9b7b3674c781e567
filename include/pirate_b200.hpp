// pirate_b200.hpp -- C++ classes with pirate's names and calling conventions over the C ABI of
// pirate_b200.h (header only; link libpirate_b200.so).
//
// They replace, for a caller of pirate's dedispersion path:
//   pirate::DedispersionConfig   include/pirate/DedispersionConfig.hpp:21-194 (from_yaml, to_yaml_string)
//   pirate::DedispersionPlan     include/pirate/DedispersionPlan.hpp:33-225 (trees, decode_argmax)
//   pirate::GpuDedisperser       include/pirate/Dedisperser.hpp:45-254 (create, allocate, acquire_input,
//                                release_input_and_launch_dd_kernels, acquire_output -> Outputs by value,
//                                release_output, fill_all_weights, fill_analytic_weights, stop, time)
// Errors are thrown as std::runtime_error carrying the library's message, as pirate's xassert does.
// Streams are cudaStream_t values passed as void * (nullptr: the legacy default stream), so this
// header needs no CUDA headers.

#ifndef PIRATE_B200_HPP
#define PIRATE_B200_HPP

#include "pirate_b200.h"

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace pirate_b200 {

inline void check(int rc)
{
    if (rc != 0) throw std::runtime_error(pb2_last_error());
}

class DedispersionConfig
{
public:
    static DedispersionConfig from_yaml(const std::string &path)
    {
        pb2_config *c = nullptr;
        check(pb2_config_from_yaml(path.c_str(), &c));
        return DedispersionConfig(c);
    }
    static DedispersionConfig from_yaml_string(const std::string &text)
    {
        pb2_config *c = nullptr;
        check(pb2_config_from_yaml_string(text.c_str(), &c));
        return DedispersionConfig(c);
    }
    std::string to_yaml_string() const
    {
        long need = 0;
        check(pb2_config_to_yaml(h.get(), nullptr, 0, &need));
        std::vector<char> buf(need);
        check(pb2_config_to_yaml(h.get(), buf.data(), need, &need));
        return std::string(buf.data());
    }
    double dm_per_unit_delay() const
    {
        double d = 0;
        check(pb2_config_dm_per_unit_delay(h.get(), &d));
        return d;
    }
    const pb2_config *handle() const { return h.get(); }

private:
    explicit DedispersionConfig(pb2_config *c) : h(c, pb2_config_destroy) {}
    std::shared_ptr<pb2_config> h;
};

class DedispersionPlan
{
public:
    explicit DedispersionPlan(const DedispersionConfig &config)
    {
        pb2_plan *p = nullptr;
        check(pb2_plan_create(config.handle(), &p));
        h.reset(p, pb2_plan_destroy);
        long n = 0;
        check(pb2_plan_ntrees(p, &n));
        trees.resize(n);
        for (long i = 0; i < n; i++) check(pb2_plan_tree_info(p, i, &trees[i]));
        ntrees = n;
    }

    long ntrees = 0;
    std::vector<pb2_tree_info> trees;   // the fields of pirate's DedispersionTree

    // decode_argmax (src_lib/DedispersionPlan.cpp:481): token + (itree, idm, itime) -> (fmin, fmax, tlo, thi, p).
    void decode_argmax(uint32_t token, long itree, long idm, long itime, long &fmin, long &fmax, long &tlo,
                       long &thi, long &p) const
    {
        long o[5];
        check(pb2_plan_decode_argmax(h.get(), token, itree, idm, itime, o));
        fmin = o[0]; fmax = o[1]; tlo = o[2]; thi = o[3]; p = o[4];
    }
    const pb2_plan *handle() const { return h.get(); }

private:
    std::shared_ptr<pb2_plan> h;
};

class GpuDedisperser
{
public:
    // GpuDedisperser::Params (include/pirate/Dedisperser.hpp:47-86), without the stream pool (internal).
    struct Params
    {
        int cuda_device_id = 0;
        long num_consumers = 1;
        long nbatches_out = 0;         // 0 -> num_active_batches
        long nbatches_wt = 0;          // 0 -> nbatches_out
        long initial_chunk = 0;
        bool synchronous = false;
        long release_timeout_ms = 0;   // 0 -> 60 s
    };

    // GpuDedisperser::Outputs (include/pirate/Dedisperser.hpp:98-125): device pointers per tree.
    struct Outputs
    {
        int dtype = 0;   // 0 float32, 1 float16, 2 bfloat16
        long nbeams = 0, ichunk_zero_based = 0, ichunk_fpga_based = 0, ibeam = 0;
        std::vector<long> ndm_out, nt_out;
        std::vector<void *> out_max;
        std::vector<uint32_t *> out_argmax;
    };

    static std::shared_ptr<GpuDedisperser> create(const DedispersionPlan &plan, const Params &params)
    {
        return std::shared_ptr<GpuDedisperser>(new GpuDedisperser(plan, params));
    }

    GpuDedisperser(const GpuDedisperser &) = delete;
    GpuDedisperser &operator=(const GpuDedisperser &) = delete;
    ~GpuDedisperser() { pb2_dd_destroy(h); }

    void allocate() { check(pb2_dd_allocate(h)); }

    // The input slot (beams_per_batch, nfreq, nt_in) in the config's dtype; shape3 receives the shape.
    void *acquire_input(long seq_id, void *stream, long *shape3 = nullptr)
    {
        void *p = nullptr;
        long s[3];
        check(pb2_dd_acquire_input(h, seq_id, stream, &p, shape3 ? shape3 : s));
        return p;
    }
    void release_input_and_launch_dd_kernels(long seq_id, void *stream) { check(pb2_dd_release_input(h, seq_id, stream)); }

    Outputs acquire_output(long consumer_id, long seq_id, void *stream, bool sync = false)
    {
        pb2_outputs o;
        check(pb2_dd_acquire_output(h, consumer_id, seq_id, stream, sync ? 1 : 0, &o));
        Outputs r;
        r.dtype = o.dtype;
        r.nbeams = o.nbeams;
        r.ichunk_zero_based = o.ichunk_zero_based;
        r.ichunk_fpga_based = o.ichunk_fpga_based;
        r.ibeam = o.ibeam;
        for (long i = 0; i < o.ntrees; i++) {
            r.ndm_out.push_back(o.ndm_out[i]);
            r.nt_out.push_back(o.nt_out[i]);
            r.out_max.push_back(o.out_max[i]);
            r.out_argmax.push_back(o.out_argmax[i]);
        }
        return r;
    }
    void release_output(long consumer_id, long seq_id, void *stream) { check(pb2_dd_release_output(h, consumer_id, seq_id, stream)); }

    // Host weights (nbatches_wt, beams_per_batch, ndm_wt, nt_wt, nprofiles, N) of tree itree.
    void fill_all_weights(long itree, const float *host, long nelts) { check(pb2_dd_fill_weights(h, itree, host, nelts)); }
    void fill_analytic_weights(const std::vector<double> &freq_variances)
    {
        check(pb2_dd_fill_analytic_weights(h, freq_variances.data(), long(freq_variances.size())));
    }
    void stop() { check(pb2_dd_stop(h)); }
    // GpuDedisperser::time (src_lib/GpuDedisperser.cpp:1573-1665): the real-time beams of each of
    // niterations int4 batches copied from pinned host memory, dedispersed and consumed (element 0 is 0).
    std::vector<double> time(long niterations)
    {
        std::vector<double> rtb(niterations > 0 ? niterations : 0);
        check(pb2_dd_time(h, niterations, rtb.data()));
        return rtb;
    }
    long device_bytes() const
    {
        long n = 0;
        check(pb2_dd_device_bytes(h, &n));
        return n;
    }

private:
    GpuDedisperser(const DedispersionPlan &plan, const Params &p)
    {
        pb2_dd_params q;
        q.cuda_device_id = p.cuda_device_id;
        q.nbatches_out = p.nbatches_out;
        q.nbatches_wt = p.nbatches_wt;
        q.num_consumers = p.num_consumers;
        q.synchronous = p.synchronous ? 1 : 0;
        q.initial_chunk = p.initial_chunk;
        q.release_timeout_ms = p.release_timeout_ms;
        check(pb2_dd_create(plan.handle(), &q, &h));
    }
    pb2_dedisperser *h = nullptr;
};

}  // namespace pirate_b200

#endif
