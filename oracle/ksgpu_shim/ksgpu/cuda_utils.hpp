// Minimal stand-in for ksgpu's cuda_utils.hpp (oracle/_ref build only). The reference CPU path makes
// no CUDA calls; CUDA_CALL throws on any error so a stray call fails loudly.
#ifndef _KSGPU_SHIM_CUDA_UTILS_HPP
#define _KSGPU_SHIM_CUDA_UTILS_HPP

#include <memory>
#include <stdexcept>
#include <string>
#include <cuda_runtime.h>
#include "xassert.hpp"

#define CUDA_CALL(x) do { cudaError_t _err = (x); if (_err != cudaSuccess) \
    throw std::runtime_error(std::string("CUDA call failed: " #x ": ") + cudaGetErrorString(_err)); } while (0)
#define CUDA_PEEK(msg) CUDA_CALL(cudaPeekAtLastError())

namespace ksgpu {

struct CudaStreamWrapper
{
    std::shared_ptr<CUstream_st> p;
    CudaStreamWrapper() {}
    static CudaStreamWrapper create(int = 0)
    {
        throw std::runtime_error("ksgpu shim: CUDA streams are not supported (host-only reference build)");
    }
    operator cudaStream_t() const { return p.get(); }
    cudaStream_t get() const { return p.get(); }
};

// Sets the current device for a scope. The host-only reference build never selects a device.
struct CudaSetDevice
{
    explicit CudaSetDevice(int)
    {
        throw std::runtime_error("ksgpu shim: CUDA devices are not supported (host-only reference build)");
    }
};

inline std::runtime_error make_cuda_exception(cudaError_t err, const char *what, const char *file, int line)
{
    return std::runtime_error(std::string(file) + ":" + std::to_string(line) + ": " + what + " failed: " + cudaGetErrorString(err));
}

inline void assign_kernel_dims(dim3 &nblocks, dim3 &nthreads, long nx, long ny, long nz, int nthreads_per_block = 128, bool = false)
{
    nthreads = dim3(unsigned(nthreads_per_block), 1, 1);
    nblocks = dim3(unsigned((nx + nthreads_per_block - 1) / nthreads_per_block), unsigned(ny), unsigned(nz));
}

}  // namespace ksgpu

#endif
