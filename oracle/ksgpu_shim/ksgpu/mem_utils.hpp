// Minimal stand-in for ksgpu's mem_utils.hpp (oracle/_ref build only): host allocation lives in
// Array.hpp (af_alloc, _af_alloc).
#ifndef _KSGPU_SHIM_MEM_UTILS_HPP
#define _KSGPU_SHIM_MEM_UTILS_HPP
#include "Array.hpp"
#include "cuda_utils.hpp"
#endif
