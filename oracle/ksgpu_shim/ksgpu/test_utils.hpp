// Minimal stand-in for ksgpu's test_utils.hpp (oracle/_ref build only).
#ifndef _KSGPU_SHIM_TEST_UTILS_HPP
#define _KSGPU_SHIM_TEST_UTILS_HPP

#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>
#include "Array.hpp"
#include "rand_utils.hpp"

namespace ksgpu {

// Strides for 'shape' whose innermost 'ncontig' axes are contiguous and whose other axes have
// random padding.
inline std::vector<long> make_random_strides(const std::vector<long> &shape, int ncontig = 0, int nalign = 1)
{
    int nd = int(shape.size());
    std::vector<long> s(nd);
    long n = 1;
    for (int d = nd - 1; d >= 0; d--) {
        if (nd - 1 - d >= ncontig && shape[d] > 1) n += rand_int(0, 3) * std::max(nalign, 1);
        s[d] = n;
        n *= std::max(shape[d], 1L);
    }
    return s;
}
inline std::vector<long> make_random_strides(std::initializer_list<long> shape, int ncontig = 0, int nalign = 1)
{
    return make_random_strides(std::vector<long>(shape), ncontig, nalign);
}

}  // namespace ksgpu

#endif
