// batched.cu -- BatchedDedisperser (see batched.hpp).

#include "batched.hpp"

#include <chrono>
#include <sstream>
#include <stdexcept>

namespace pb2 {

#define BD_CHECK(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) \
    throw std::runtime_error(std::string("BatchedDedisperser: " #x ": ") + cudaGetErrorString(_e)); } while (0)

__global__ void advance_counter_kernel(long *ctr)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) ctr[0] += 1;
}

BatchedDedisperser::BatchedDedisperser(const std::vector<DedispersionPlan> &plans_, int dev) : device(dev), plans(plans_)
{
    if (plans.empty()) throw std::runtime_error("BatchedDedisperser: no plans");
    for (const DedispersionPlan &p : plans) {
        if (p.beams_per_gpu != p.beams_per_batch)
            throw std::runtime_error("BatchedDedisperser: each group's beams must form one batch (beams_per_gpu == beams_per_batch)");
        GpuDedisperser::Params gp;
        gp.cuda_device_id = dev;
        gp.num_consumers = 0;
        gp.nbatches_out = 1;
        gp.nbatches_wt = 1;
        groups.emplace_back(new GpuDedisperser(p, gp));
    }
    tuning.assign(groups.size(), GroupTuning());
}

BatchedDedisperser::~BatchedDedisperser()
{
    cudaSetDevice(device);
    drop_graph();
    if (cap) cudaStreamSynchronize(cap);
    for (cudaStream_t s : branch) if (s) { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
    if (cap) cudaStreamDestroy(cap);
    if (ev_fork) cudaEventDestroy(ev_fork);
    for (cudaEvent_t e : ev_join) if (e) cudaEventDestroy(e);
    if (ctr) cudaFree(ctr);
}

GpuDedisperser &BatchedDedisperser::group(long g)
{
    if (g < 0 || g >= long(groups.size())) throw std::runtime_error("BatchedDedisperser: group index out of range");
    return *groups[g];
}

void BatchedDedisperser::allocate()
{
    if (allocated) throw std::runtime_error("BatchedDedisperser::allocate() called twice");
    BD_CHECK(cudaSetDevice(device));
    for (auto &g : groups) g->allocate();
    BD_CHECK(cudaMalloc(&ctr, sizeof(long)));
    BD_CHECK(cudaMemset(ctr, 0, sizeof(long)));
    BD_CHECK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    branch.resize(groups.size());
    ev_join.resize(groups.size());
    for (size_t i = 0; i < groups.size(); i++) {
        BD_CHECK(cudaStreamCreateWithFlags(&branch[i], cudaStreamNonBlocking));
        BD_CHECK(cudaEventCreateWithFlags(&ev_join[i], cudaEventDisableTiming));
    }
    BD_CHECK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    BD_CHECK(cudaDeviceSynchronize());
    allocated = true;
}

void BatchedDedisperser::drop_graph()
{
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
}

void BatchedDedisperser::set_schedule(const std::vector<GroupTuning> &t, bool conc)
{
    if (t.size() != groups.size()) throw std::runtime_error("BatchedDedisperser::set_schedule: one tuning per group");
    for (const GroupTuning &x : t)
        if (x.grid_block < 32 || x.grid_block > 512) throw std::runtime_error("BatchedDedisperser::set_schedule: grid_block out of [32, 512]");
    BD_CHECK(cudaSetDevice(device));
    drop_graph();
    tuning = t;
    concurrent = conc;
}

void BatchedDedisperser::build_graph()
{
    BD_CHECK(cudaSetDevice(device));
    drop_graph();
    BD_CHECK(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    try {
        if (concurrent) {
            BD_CHECK(cudaEventRecord(ev_fork, cap));
            for (size_t i = 0; i < groups.size(); i++) {
                BD_CHECK(cudaStreamWaitEvent(branch[i], ev_fork, 0));
                groups[i]->enqueue_chunk(branch[i], ctr, tuning[i]);
                BD_CHECK(cudaEventRecord(ev_join[i], branch[i]));
                BD_CHECK(cudaStreamWaitEvent(cap, ev_join[i], 0));
            }
        } else {
            for (size_t i = 0; i < groups.size(); i++) groups[i]->enqueue_chunk(cap, ctr, tuning[i]);
        }
        advance_counter_kernel<<<1, 32, 0, cap>>>(ctr);
        BD_CHECK(cudaGetLastError());
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(cap, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    BD_CHECK(cudaStreamEndCapture(cap, &graph));
    BD_CHECK(cudaGraphInstantiate(&exec, graph, 0));
    size_t n = 0;
    BD_CHECK(cudaGraphGetNodes(graph, nullptr, &n));
    std::vector<cudaGraphNode_t> nodes(n);
    BD_CHECK(cudaGraphGetNodes(graph, nodes.data(), &n));
    nkernels = 0;
    for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType ty;
        BD_CHECK(cudaGraphNodeGetType(nd, &ty));
        if (ty == cudaGraphNodeTypeKernel) nkernels++;
    }
}

void BatchedDedisperser::step(cudaStream_t stream)
{
    if (!allocated) throw std::runtime_error("BatchedDedisperser::step(): allocate() was not called");
    BD_CHECK(cudaSetDevice(device));
    if (!exec) build_graph();
    BD_CHECK(cudaGraphLaunch(exec, stream));
    nsteps++;
}

void BatchedDedisperser::reset(cudaStream_t stream)
{
    BD_CHECK(cudaSetDevice(device));
    for (auto &g : groups) g->zero_state(stream);
    BD_CHECK(cudaMemsetAsync(ctr, 0, sizeof(long), stream));
    BD_CHECK(cudaStreamSynchronize(stream));
    nsteps = 0;
}

double BatchedDedisperser::time_steps(int n, cudaStream_t stream)
{
    if (n < 1) throw std::runtime_error("BatchedDedisperser::time_steps: n must be >= 1");
    cudaEvent_t e0, e1;
    BD_CHECK(cudaEventCreate(&e0));
    BD_CHECK(cudaEventCreate(&e1));
    BD_CHECK(cudaEventRecord(e0, stream));
    for (int i = 0; i < n; i++) step(stream);
    BD_CHECK(cudaEventRecord(e1, stream));
    BD_CHECK(cudaEventSynchronize(e1));
    float ms = 0;
    BD_CHECK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms / n;
}

std::string BatchedDedisperser::autotune(int reps)
{
    if (!allocated) throw std::runtime_error("BatchedDedisperser::autotune(): allocate() was not called");
    if (reps < 1) throw std::runtime_error("BatchedDedisperser::autotune(): reps must be >= 1");
    BD_CHECK(cudaSetDevice(device));
    cudaStream_t s = cap;
    std::ostringstream js;
    js << "{\"candidates\": [";
    // Coordinate descent: start from the defaults with concurrent branches; for each group and knob, try
    // the alternatives with the other choices fixed and keep any that is faster; then the concurrency.
    std::vector<GroupTuning> best = tuning;
    bool best_conc = true;
    auto measure = [&](const std::vector<GroupTuning> &t, bool conc) {
        set_schedule(t, conc);
        step(s);                          // capture and warm up
        BD_CHECK(cudaStreamSynchronize(s));
        return time_steps(reps, s);
    };
    bool first = true;
    auto record = [&](const char *what, long g, double ms) {
        js << (first ? "" : ", ") << "{\"try\": \"" << what << "\", \"group\": " << g << ", \"ms\": " << ms << "}";
        first = false;
    };
    double best_ms = measure(best, best_conc);
    record("defaults", -1, best_ms);
    for (size_t g = 0; g < groups.size(); g++) {
        for (int knob = 0; knob < 3; knob++) {
            std::vector<std::vector<GroupTuning>> alts;
            if (knob == 0) { auto t = best; t[g].merge_stage2 = !t[g].merge_stage2; alts.push_back(t); }
            if (knob == 1) { auto t = best; t[g].pf_general = !t[g].pf_general; alts.push_back(t); }
            if (knob == 2) for (int gb : {64, 256, 512}) if (gb != best[g].grid_block) { auto t = best; t[g].grid_block = gb; alts.push_back(t); }
            for (auto &t : alts) {
                double ms = measure(t, best_conc);
                const char *names[3] = {"merge_stage2", "pf_general", "grid_block"};
                record(names[knob], long(g), ms);
                if (ms < best_ms * 0.995) { best_ms = ms; best = t; }
            }
        }
    }
    if (groups.size() > 1) {
        double ms = measure(best, !best_conc);
        record("concurrent", -1, ms);
        if (ms < best_ms * 0.995) { best_ms = ms; best_conc = !best_conc; }
    }
    set_schedule(best, best_conc);
    reset(s);
    js << "], \"chosen\": {\"concurrent\": " << (best_conc ? "true" : "false") << ", \"ms_per_step\": " << best_ms << ", \"groups\": [";
    for (size_t g = 0; g < groups.size(); g++)
        js << (g ? ", " : "") << "{\"merge_stage2\": " << (best[g].merge_stage2 ? "true" : "false") << ", \"pf_general\": "
           << (best[g].pf_general ? "true" : "false") << ", \"grid_block\": " << best[g].grid_block << "}";
    js << "]}}";
    return js.str();
}

}  // namespace pb2
