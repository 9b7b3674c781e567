// Minimal stand-in for ksgpu's KernelTimer (oracle/_ref build only; never used by the CPU path).
#ifndef _KSGPU_SHIM_KERNEL_TIMER_HPP
#define _KSGPU_SHIM_KERNEL_TIMER_HPP

#include <stdexcept>
#include <cuda_runtime.h>

namespace ksgpu {

struct KernelTimer
{
    int niterations = 0, nstreams = 0, istream = 0, curr_iteration = 0;
    cudaStream_t stream = nullptr;
    double dt = 0;
    KernelTimer(int niter, int nstr) : niterations(niter), nstreams(nstr)
    {
        throw std::runtime_error("ksgpu shim: KernelTimer is not supported (host-only reference build)");
    }
    bool next() { return false; }
    bool warmed_up = false;
};

}  // namespace ksgpu

#endif
