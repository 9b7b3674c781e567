// Minimal stand-in for ksgpu's rand_utils.hpp (oracle/_ref build only): a process-wide mt19937 and
// the few random helpers that pirate's reference sources call.
#ifndef _KSGPU_SHIM_RAND_UTILS_HPP
#define _KSGPU_SHIM_RAND_UTILS_HPP

#include <algorithm>
#include <cmath>
#include <random>
#include <vector>
#include "xassert.hpp"

namespace ksgpu {

inline std::mt19937 &default_rng()
{
    static std::mt19937 rng(20240601u);
    return rng;
}

// Uniform integer in [lo, hi).
inline long rand_int(long lo, long hi, std::mt19937 &rng = default_rng())
{
    xassert(lo < hi);
    return std::uniform_int_distribution<long>(lo, hi - 1)(rng);
}

inline double rand_uniform(double lo = 0.0, double hi = 1.0, std::mt19937 &rng = default_rng())
{
    return std::uniform_real_distribution<double>(lo, hi)(rng);
}
inline float rand_uniform(float lo, float hi, std::mt19937 &rng)
{
    return float(std::uniform_real_distribution<double>(lo, hi)(rng));
}

inline bool rand_bool(std::mt19937 &rng = default_rng()) { return rand_int(0, 2, rng) != 0; }

inline std::vector<long> rand_int_vec(long n, long lo, long hi, std::mt19937 &rng = default_rng())
{
    std::vector<long> v(n);
    for (long i = 0; i < n; i++) v[i] = rand_int(lo, hi, rng);
    return v;
}

inline std::vector<double> rand_uniform_vec(long n, double lo = 0.0, double hi = 1.0, std::mt19937 &rng = default_rng())
{
    std::vector<double> v(n);
    for (long i = 0; i < n; i++) v[i] = rand_uniform(lo, hi, rng);
    return v;
}

template<typename T>
inline void randomly_permute(std::vector<T> &v, std::mt19937 &rng = default_rng())
{
    std::shuffle(v.begin(), v.end(), rng);
}

template<typename T>
inline T rand_element(const std::vector<T> &v, std::mt19937 &rng = default_rng())
{
    xassert(!v.empty());
    return v[rand_int(0, long(v.size()), rng)];
}

// n random positive integers whose product is at most maxprod.
inline std::vector<long> random_integers_with_bounded_product(int n, long maxprod, std::mt19937 &rng = default_rng())
{
    xassert(n > 0 && maxprod > 0);
    std::vector<long> ret(n, 1);
    double budget = std::log(double(maxprod));
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::shuffle(order.begin(), order.end(), rng);
    for (int k = 0; k < n; k++) {
        double share = std::uniform_real_distribution<double>(0, budget)(rng) * (k == n - 1 ? 1.0 : 0.7);
        long v = std::max(1L, long(std::exp(share)));
        ret[order[k]] = v;
        budget -= std::log(double(v));
        if (budget < 0) budget = 0;
    }
    long p = 1;
    for (long v : ret) p *= v;
    xassert(p <= maxprod);
    return ret;
}

}  // namespace ksgpu

#endif
