// A C++ caller of the dedispersion path through include/pirate_b200.hpp (pirate's GpuDedisperser
// calling convention over the C ABI), used by tests/test_cpp_caller.py.
//
//   dd_cpp CONFIG.yml --plan                         prints the plan's trees (no GPU needed)
//   dd_cpp CONFIG.yml NSEQ IN.bin WT.bin OUT.bin     dedisperses NSEQ batches (float32 config):
//       IN.bin  NSEQ inputs (beams_per_batch, nfreq, nt_in) float32, in seq_id order
//       WT.bin  per tree, (nbatches_wt, beams_per_batch, ndm_wt, nt_wt, nprofiles, N) float32
//       OUT.bin per seq_id and tree: out_max (beams, ndm_out, nt_out) float32, then out_argmax uint32

#include "pirate_b200.hpp"

#include <cuda_runtime_api.h>

#include <cstdio>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

using namespace pirate_b200;

static std::vector<char> read_file(const std::string &path)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open " + path);
    return std::vector<char>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

static void cuda(cudaError_t e)
{
    if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
}

int main(int argc, char **argv)
{
    try {
        if (argc < 3) throw std::runtime_error("usage: dd_cpp CONFIG.yml --plan | NSEQ IN.bin WT.bin OUT.bin");
        std::vector<char> yml = read_file(argv[1]);
        yml.push_back(0);
        DedispersionConfig cfg = DedispersionConfig::from_yaml_string(yml.data());
        DedispersionPlan plan(cfg);
        if (std::string(argv[2]) == "--plan") {
            std::cout << "ntrees " << plan.ntrees << "\n";
            for (const pb2_tree_info &t : plan.trees)
                std::cout << "tree " << t.primary_tree_index << " " << t.early_trigger_level << " " << t.ndm_out << " "
                          << t.nt_out << " " << t.nprofiles << " " << t.Dcore << "\n";
            return 0;
        }
        if (argc < 6) throw std::runtime_error("usage: dd_cpp CONFIG.yml NSEQ IN.bin WT.bin OUT.bin");
        const long nseq = std::stol(argv[2]);
        std::vector<char> in = read_file(argv[3]), wt = read_file(argv[4]);

        GpuDedisperser::Params params;
        params.num_consumers = 1;
        auto dd = GpuDedisperser::create(plan, params);
        dd->allocate();
        // The weight file holds, tree after tree, nslots = nbatches_wt * beams_per_batch slots of each
        // tree's per-beam weights (ndm_wt * nt_wt * nprofiles * N floats).
        long per_beam_total = 0;
        for (const pb2_tree_info &t : plan.trees) per_beam_total += t.ndm_wt * t.nt_wt * t.nprofiles * t.nsubbands;
        const long nslots = long(wt.size() / sizeof(float)) / per_beam_total;
        size_t wo = 0;
        for (long i = 0; i < plan.ntrees; i++) {
            const pb2_tree_info &t = plan.trees[i];
            const long n = nslots * t.ndm_wt * t.nt_wt * t.nprofiles * t.nsubbands;
            dd->fill_all_weights(i, (const float *) (wt.data() + wo), n);
            wo += size_t(n) * sizeof(float);
        }
        std::ofstream out(argv[5], std::ios::binary);
        size_t io = 0;
        for (long seq = 0; seq < nseq; seq++) {
            long shape[3];
            void *x = dd->acquire_input(seq, nullptr, shape);
            size_t nb = size_t(shape[0] * shape[1] * shape[2]) * sizeof(float);
            cuda(cudaMemcpy(x, in.data() + io, nb, cudaMemcpyHostToDevice));
            io += nb;
            dd->release_input_and_launch_dd_kernels(seq, nullptr);
            GpuDedisperser::Outputs o = dd->acquire_output(0, seq, nullptr, true);
            for (size_t i = 0; i < o.out_max.size(); i++) {
                size_t n = size_t(o.nbeams * o.ndm_out[i] * o.nt_out[i]);
                std::vector<float> m(n);
                std::vector<uint32_t> a(n);
                cuda(cudaMemcpy(m.data(), o.out_max[i], n * sizeof(float), cudaMemcpyDeviceToHost));
                cuda(cudaMemcpy(a.data(), o.out_argmax[i], n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
                out.write((const char *) m.data(), n * sizeof(float));
                out.write((const char *) a.data(), n * sizeof(uint32_t));
            }
            dd->release_output(0, seq, nullptr);
        }
        return 0;
    } catch (std::exception &e) {
        std::fprintf(stderr, "dd_cpp: %s\n", e.what());
        return 1;
    }
}
