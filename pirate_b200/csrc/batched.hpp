// batched.hpp -- many beams with uneven plans in one CUDA graph per chunk.
//
// pirate runs one GpuDedisperser per plan and interleaves batches over a pool of compute streams
// (src_lib/GpuDedisperser.cpp:990-1000). Here a BatchedDedisperser holds one group per plan (tree rank,
// number of primary trees, beams), each a GpuDedisperser whose beams form a single batch, and runs one
// chunk of every group as ONE CUDA graph launch: the groups' kernel sequences are captured once, as
// parallel branches (or one serial chain), and replayed every chunk. Every kernel reads the chunk index
// from a device counter that the graph's last node advances, so the same executable graph serves every
// chunk without parameter updates. A project autotuner times the schedule choices (per group: merged or
// per-tree stage-2 grids, peak-finding kernel variant, gridding block size; and branch concurrency)
// with CUDA events on the replayed graph and keeps the fastest.

#pragma once

#include "dedisperser.hpp"

#include <memory>
#include <string>
#include <vector>

namespace pb2 {

class BatchedDedisperser
{
public:
    BatchedDedisperser(const std::vector<DedispersionPlan> &plans, int cuda_device_id);
    ~BatchedDedisperser();
    BatchedDedisperser(const BatchedDedisperser &) = delete;
    BatchedDedisperser &operator=(const BatchedDedisperser &) = delete;

    // Allocates every group (device memory zeroed) and the chunk counter.
    void allocate();
    long ngroups() const { return long(groups.size()); }
    GpuDedisperser &group(long g);

    // Schedule: per-group tuning and whether the groups' branches run concurrently. Invalidates the graph.
    void set_schedule(const std::vector<GroupTuning> &tuning, bool concurrent);
    // One chunk of every group: one graph launch on 'stream' (the graph is captured on first use).
    // Inputs: each group's input slot 0 (group(g).input_ptr(0)), written before the call on 'stream'
    // or ordered before it; outputs: group(g).outputs_ptr(0), valid after the call on 'stream'.
    void step(cudaStream_t stream);
    long chunks_done() const { return nsteps; }
    // Zeroes every group's state and the chunk counter (a fresh stream of chunks), keeping the graph.
    void reset(cudaStream_t stream);
    // Times 'reps' replays per candidate schedule (after one warm-up replay each), keeps the fastest,
    // resets the state, and returns a JSON record of the candidates and the choice.
    std::string autotune(int reps);
    // Device time of 'n' steps on 'stream' (CUDA events), in ms per step.
    double time_steps(int n, cudaStream_t stream);
    // Kernel launches per step (graph nodes that are kernels).
    long kernels_per_step() const { return nkernels; }

private:
    void build_graph();
    void drop_graph();

    int device = 0;
    std::vector<DedispersionPlan> plans;
    std::vector<std::unique_ptr<GpuDedisperser>> groups;
    std::vector<GroupTuning> tuning;
    bool concurrent = true;
    long *ctr = nullptr;                  // device chunk counter
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cap = nullptr;           // capture origin
    std::vector<cudaStream_t> branch;     // one per group
    cudaEvent_t ev_fork = nullptr;
    std::vector<cudaEvent_t> ev_join;
    long nsteps = 0, nkernels = 0;
    bool allocated = false;
};

}  // namespace pb2
