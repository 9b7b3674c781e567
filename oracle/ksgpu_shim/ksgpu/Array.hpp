// Minimal stand-in for ksgpu::Array (oracle/_ref build only). ksgpu is not vendored with pirate, so
// this header provides the subset of its strided N-dimensional array that pirate's CPU reference
// sources use: host allocation (af_uhost/af_rhost, af_zero), element access, slicing, reshaping
// views, transposition, copies between arrays of equal shape, and dtype-erased Array<void> views.
// Device arrays are not supported: the reference CPU path never needs them.
#ifndef _KSGPU_SHIM_ARRAY_HPP
#define _KSGPU_SHIM_ARRAY_HPP

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <iostream>
#include <memory>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "Dtype.hpp"
#include "xassert.hpp"
#include "rand_utils.hpp"
#include <cuda_runtime.h>

namespace ksgpu {

static constexpr int ArrayMaxDim = 8;

enum : int {
    af_gpu = 0x01, af_uhost = 0x02, af_rhost = 0x04, af_unified = 0x08,
    af_zero = 0x10, af_random = 0x20, af_guard = 0x40,
    af_mmap_small = 0x100, af_mmap_huge = 0x200, af_mmap_try_huge = 0x400, af_verbose = 0x800
};
static constexpr int af_location_flags = af_gpu | af_uhost | af_rhost | af_unified;

inline bool af_on_host(int f) { return (f & (af_uhost | af_rhost | af_unified)) != 0; }
inline bool af_on_gpu(int f) { return (f & (af_gpu | af_unified)) != 0; }

// Host allocation with 128-byte alignment. af_zero clears; af_random fills with random bytes.
inline std::shared_ptr<void> af_alloc(long nbytes, int aflags)
{
    if (nbytes < 0) throw std::runtime_error("ksgpu::af_alloc: negative size");
    if ((aflags & af_gpu) && !(aflags & af_unified))
        throw std::runtime_error("ksgpu shim: device allocation is not supported (host-only reference build)");
    size_t n = size_t((nbytes + 127) / 128 * 128);
    if (n == 0) n = 128;
    void *p = std::aligned_alloc(128, n);
    if (!p) throw std::runtime_error("ksgpu::af_alloc: out of memory");
    if (aflags & (af_zero | af_random))
        memset(p, 0, n);   // af_random arrays are then filled by _randomize_elements()
    return std::shared_ptr<void>(p, [](void *q) { std::free(q); });
}

inline std::vector<long> make_contiguous_strides(const std::vector<long> &shape)
{
    std::vector<long> s(shape.size());
    long n = 1;
    for (int d = int(shape.size()) - 1; d >= 0; d--) { s[d] = n; n *= std::max(shape[d], 1L); }
    return s;
}

template<typename T>
struct Array
{
    using elt_ref = typename std::add_lvalue_reference<T>::type;

    T *data = nullptr;
    int ndim = 0;
    long shape[ArrayMaxDim] = {};
    long size = 0;
    long strides[ArrayMaxDim] = {};
    std::shared_ptr<void> base;
    int aflags = 0;
    Dtype dtype;

    Array() { if constexpr (!std::is_void_v<T>) dtype = Dtype::native<T>(); }

    Array(int nd, const long *shp, int flags) { _init(_native_or_fail(), nd, shp, nullptr, flags); }
    Array(int nd, const long *shp, const long *str, int flags) { _init(_native_or_fail(), nd, shp, str, flags); }
    Array(const std::vector<long> &shp, int flags) { _init(_native_or_fail(), int(shp.size()), shp.data(), nullptr, flags); }
    Array(std::initializer_list<long> shp, int flags) { _init(_native_or_fail(), int(shp.size()), shp.begin(), nullptr, flags); }
    Array(const std::vector<long> &shp, const std::vector<long> &str, int flags)
    {
        xassert(shp.size() == str.size());
        _init(_native_or_fail(), int(shp.size()), shp.data(), str.data(), flags);
    }
    Array(std::initializer_list<long> shp, std::initializer_list<long> str, int flags)
    {
        xassert(shp.size() == str.size());
        _init(_native_or_fail(), int(shp.size()), shp.begin(), str.begin(), flags);
    }
    Array(const Dtype &dt, int nd, const long *shp, int flags) { _init(_checked(dt), nd, shp, nullptr, flags); }
    Array(const Dtype &dt, const std::vector<long> &shp, int flags) { _init(_checked(dt), int(shp.size()), shp.data(), nullptr, flags); }
    Array(const Dtype &dt, std::initializer_list<long> shp, int flags) { _init(_checked(dt), int(shp.size()), shp.begin(), nullptr, flags); }
    Array(const Dtype &dt, const std::vector<long> &shp, const std::vector<long> &str, int flags)
    {
        xassert(shp.size() == str.size());
        _init(_checked(dt), int(shp.size()), shp.data(), str.data(), flags);
    }

    // A typed array is usable wherever an Array<void> (lvalue) is expected: the layouts agree.
    operator Array<void> &() { return *reinterpret_cast<Array<void> *>(this); }
    operator const Array<void> &() const { return *reinterpret_cast<const Array<void> *>(this); }

    // Typed arrays from Array<void> (dtype checked).
    template<typename U, typename = std::enable_if_t<std::is_void_v<U> && !std::is_void_v<T>>>
    Array(const Array<U> &x)
    {
        _check_dtype<T>(x.dtype, "ksgpu::Array conversion");
        _copy_header(x);
        data = (T *) x.data;
    }

    template<typename U>
    Array<U> cast(const char *where = "ksgpu::Array::cast") const
    {
        _check_dtype<U>(dtype, where);
        Array<U> r;
        r._copy_header(*this);
        r.data = (U *) data;
        return r;
    }
    template<typename U> Array<U> template_cast(const char *where = "ksgpu::Array::template_cast") const { return cast<U>(where); }

    template<typename U>
    void _copy_header(const Array<U> &x)
    {
        ndim = x.ndim; size = x.size; base = x.base; aflags = x.aflags; dtype = x.dtype;
        for (int d = 0; d < ArrayMaxDim; d++) { shape[d] = x.shape[d]; strides[d] = x.strides[d]; }
    }

    long itemsize() const { return dtype.nbits / 8; }
    bool on_host() const { return (aflags & af_gpu) == 0 || (aflags & af_unified); }
    bool on_gpu() const { return af_on_gpu(aflags); }
    bool is_allocated() const { return bool(base) || data != nullptr; }

    int get_ncontig() const
    {
        int nc = 0;
        long expect = 1;
        for (int d = ndim - 1; d >= 0; d--) {
            if (shape[d] != 1 && strides[d] != expect) break;
            nc++;
            expect *= shape[d];
        }
        return nc;
    }
    bool is_fully_contiguous() const { return get_ncontig() == ndim; }

    bool shape_equals(int nd, const long *shp) const
    {
        if (nd != ndim) return false;
        for (int d = 0; d < nd; d++) if (shape[d] != shp[d]) return false;
        return true;
    }
    bool shape_equals(const std::vector<long> &shp) const { return shape_equals(int(shp.size()), shp.data()); }
    bool shape_equals(std::initializer_list<long> shp) const { return shape_equals(int(shp.size()), shp.begin()); }
    template<typename U> bool shape_equals(const Array<U> &x) const { return shape_equals(x.ndim, x.shape); }

    static std::string _tup(int nd, const long *v)
    {
        std::stringstream ss;
        ss << "(";
        for (int d = 0; d < nd; d++) ss << (d ? "," : "") << v[d];
        ss << ")";
        return ss.str();
    }
    bool strides_equal(int nd, const long *str) const
    {
        if (nd != ndim) return false;
        for (int d = 0; d < nd; d++) if (shape[d] > 1 && strides[d] != str[d]) return false;
        return true;
    }
    bool strides_equal(const std::vector<long> &str) const { return strides_equal(int(str.size()), str.data()); }
    bool strides_equal(std::initializer_list<long> str) const { return strides_equal(int(str.size()), str.begin()); }

    std::string shape_str() const { return _tup(ndim, shape); }
    std::string stride_str() const { return _tup(ndim, strides); }
    std::vector<long> shape_vec() const { return std::vector<long>(shape, shape + ndim); }
    std::vector<long> stride_vec() const { return std::vector<long>(strides, strides + ndim); }

    long _offset(int nd, const long *ix) const
    {
        if (nd != ndim) throw std::runtime_error("ksgpu::Array::at(): wrong number of indices for shape " + shape_str());
        long o = 0;
        for (int d = 0; d < nd; d++) {
            if (ix[d] < 0 || ix[d] >= shape[d])
                throw std::runtime_error("ksgpu::Array::at(): index " + _tup(nd, ix) + " out of range for shape " + shape_str());
            o += ix[d] * strides[d];
        }
        return o;
    }
    elt_ref at(std::initializer_list<long> ix) const { return _elt(_offset(int(ix.size()), ix.begin())); }
    elt_ref at(const std::vector<long> &ix) const { return _elt(_offset(int(ix.size()), ix.data())); }

    Array slice(int axis, long ix) const
    {
        if (axis < 0 || axis >= ndim || ix < 0 || ix >= shape[axis])
            throw std::runtime_error("ksgpu::Array::slice(): bad axis/index for shape " + shape_str());
        Array r = *this;
        r.data = _advance(ix * strides[axis]);
        for (int d = axis; d < ndim - 1; d++) { r.shape[d] = shape[d + 1]; r.strides[d] = strides[d + 1]; }
        r.ndim = ndim - 1;
        r.shape[r.ndim] = 0; r.strides[r.ndim] = 0;
        r._set_size();
        return r;
    }
    Array slice(int axis, long start, long stop) const
    {
        if (axis < 0 || axis >= ndim || start < 0 || stop < start || stop > shape[axis])
            throw std::runtime_error("ksgpu::Array::slice(): bad range for shape " + shape_str());
        Array r = *this;
        r.data = _advance(start * strides[axis]);
        r.shape[axis] = stop - start;
        r._set_size();
        return r;
    }

    // A view with a new shape over the same elements in C order; throws if the strides do not allow it.
    Array reshape(int nd, const long *shp) const
    {
        long n = 1;
        for (int d = 0; d < nd; d++) n *= shp[d];
        if (n != size)
            throw std::runtime_error("ksgpu::Array::reshape(): size mismatch " + shape_str() + " -> " + _tup(nd, shp));
        Array r = *this;
        r.ndim = nd;
        for (int d = 0; d < ArrayMaxDim; d++) { r.shape[d] = (d < nd) ? shp[d] : 0; r.strides[d] = 0; }
        if (size == 0) {
            std::vector<long> s = make_contiguous_strides(std::vector<long>(shp, shp + nd));
            for (int d = 0; d < nd; d++) r.strides[d] = s[d];
            return r;
        }
        // Drop length-1 axes of the source, then match groups of axes with equal products.
        std::vector<long> os, ost;
        for (int d = 0; d < ndim; d++) if (shape[d] != 1) { os.push_back(shape[d]); ost.push_back(strides[d]); }
        size_t i = 0;
        int j = 0;
        while (j < nd) {
            if (shp[j] == 1) { r.strides[j] = 1; j++; continue; }
            // group: source axes [i0, i) and target axes [j0, j)
            size_t i0 = i;
            int j0 = j;
            long pi = os[i++], pj = shp[j++];
            while (pi != pj) {
                if (pi < pj) pi *= os[i++];
                else pj *= shp[j++];
            }
            for (size_t k = i0; k + 1 < i; k++)
                if (ost[k] != ost[k + 1] * os[k + 1])
                    throw std::runtime_error("ksgpu::Array::reshape(): strides " + stride_str() + " of shape " + shape_str() + " do not allow shape " + _tup(nd, shp));
            long s = ost[i - 1];
            for (int k = j - 1; k >= j0; k--) { r.strides[k] = s; s *= shp[k]; }
        }
        return r;
    }
    Array reshape(const std::vector<long> &shp) const { return reshape(int(shp.size()), shp.data()); }
    Array reshape(std::initializer_list<long> shp) const { return reshape(int(shp.size()), shp.begin()); }

    Array transpose(const std::vector<int> &perm) const
    {
        if (int(perm.size()) != ndim) throw std::runtime_error("ksgpu::Array::transpose(): wrong permutation length");
        Array r = *this;
        std::vector<bool> seen(ndim, false);
        for (int d = 0; d < ndim; d++) {
            int p = perm[d];
            if (p < 0 || p >= ndim || seen[p]) throw std::runtime_error("ksgpu::Array::transpose(): invalid permutation");
            seen[p] = true;
            r.shape[d] = shape[p];
            r.strides[d] = strides[p];
        }
        return r;
    }
    Array transpose(std::initializer_list<int> perm) const { return transpose(std::vector<int>(perm)); }

    // Elementwise copy from an array of the same shape and dtype (any strides).
    template<typename U>
    void fill(const Array<U> &src) const
    {
        if (!shape_equals(src.ndim, src.shape))
            throw std::runtime_error("ksgpu::Array::fill(): shape mismatch " + shape_str() + " vs " + src.shape_str());
        if (dtype != src.dtype)
            throw std::runtime_error("ksgpu::Array::fill(): dtype mismatch " + dtype.str() + " vs " + src.dtype.str());
        if (!on_host() || !src.on_host())
            throw std::runtime_error("ksgpu shim: fill() supports host arrays only");
        if (size == 0) return;
        _copy_rec(0, (char *) data, (const char *) src.data, src.strides);
    }

    // Multi-index iteration in C order: for (auto ix = a.ix_start(); a.ix_valid(ix); a.ix_next(ix)).
    std::vector<long> ix_start() const { return std::vector<long>(ndim, 0); }
    bool ix_valid(const std::vector<long> &ix) const { return size > 0 && ndim > 0 && ix[0] < shape[0]; }
    void ix_next(std::vector<long> &ix) const
    {
        for (int d = ndim - 1; d >= 0; d--) {
            if (++ix[d] < shape[d]) return;
            if (d > 0) ix[d] = 0;
        }
    }

    // Fills a float array with uniform random values in [-1, 1].
    void randomize() const
    {
        if constexpr (std::is_same_v<T, float> || std::is_same_v<T, double>) {
            std::mt19937 &rng = _rng();
            std::uniform_real_distribution<double> u(-1.0, 1.0);
            for (auto ix = ix_start(); ix_valid(ix); ix_next(ix)) at(ix) = T(u(rng));
        }
        else throw std::runtime_error("ksgpu shim: randomize() supports float arrays only");
    }
    static std::mt19937 &_rng() { static std::mt19937 r(987654321u); return r; }

    void set_zero() const
    {
        if (size == 0) return;
        Array z = Array(dtype, shape_vec(), af_uhost | af_zero);
        fill(z);
    }

    Array clone() const
    {
        Array r(dtype, shape_vec(), af_uhost);
        r.fill(*this);
        return r;
    }
    Array clone(int flags) const
    {
        Array r(dtype, shape_vec(), flags);
        r.fill(*this);
        return r;
    }

    Array to_host(bool = true) const
    {
        if (!on_host()) throw std::runtime_error("ksgpu shim: device arrays are not supported");
        return *this;
    }
    Array to_gpu(cudaStream_t = nullptr) const
    {
        throw std::runtime_error("ksgpu shim: device arrays are not supported (host-only reference build)");
    }

    // Converts elements to another dtype (float16/32/64, signed/unsigned integers).
    Array<void> convert(const Dtype &dst_dtype) const
    {
        Array<void> r(dst_dtype, shape_vec(), af_uhost);
        Array<void> src = *this;
        std::vector<long> ix(ndim, 0);
        for (long n = 0; n < size; n++) {
            long so = 0, dofs = 0;
            for (int d = 0; d < ndim; d++) { so += ix[d] * strides[d]; dofs += ix[d] * r.strides[d]; }
            _store((char *) r.data + dofs * r.itemsize(), dst_dtype, _load((const char *) data + so * itemsize(), dtype));
            for (int d = ndim - 1; d >= 0; d--) { if (++ix[d] < shape[d]) break; ix[d] = 0; }
        }
        return r;
    }
    template<typename U> Array<U> convert() const { return convert(Dtype::native<U>()).template cast<U>(); }

    static double _load(const char *p, const Dtype &dt)
    {
        if (dt == Dtype(df_float, 32)) return *(const float *) p;
        if (dt == Dtype(df_float, 64)) return *(const double *) p;
        if (dt == Dtype(df_float, 16)) return double(__half2float(*(const __half *) p));
        if (dt == Dtype(df_int, 32)) return *(const int *) p;
        if (dt == Dtype(df_uint, 32)) return *(const unsigned int *) p;
        if (dt == Dtype(df_int, 64)) return double(*(const long *) p);
        if (dt == Dtype(df_uint, 8)) return *(const unsigned char *) p;
        throw std::runtime_error("ksgpu shim: convert() from " + dt.str() + " is not supported");
    }
    static void _store(char *p, const Dtype &dt, double v)
    {
        if (dt == Dtype(df_float, 32)) *(float *) p = float(v);
        else if (dt == Dtype(df_float, 64)) *(double *) p = v;
        else if (dt == Dtype(df_float, 16)) *(__half *) p = __float2half_rn(float(v));
        else if (dt == Dtype(df_int, 32)) *(int *) p = int(v);
        else if (dt == Dtype(df_uint, 32)) *(unsigned int *) p = (unsigned int) v;
        else if (dt == Dtype(df_int, 64)) *(long *) p = long(v);
        else if (dt == Dtype(df_uint, 8)) *(unsigned char *) p = (unsigned char) v;
        else throw std::runtime_error("ksgpu shim: convert() to " + dt.str() + " is not supported");
    }

    // ---- internals ----
    static Dtype _native_or_fail()
    {
        if constexpr (std::is_void_v<T>) throw std::runtime_error("ksgpu::Array<void>: a dtype is required");
        else return Dtype::native<T>();
    }
    static Dtype _checked(const Dtype &dt) { _check_dtype<T>(dt, "ksgpu::Array constructor"); return dt; }

    void _set_size()
    {
        size = 1;
        for (int d = 0; d < ndim; d++) size *= shape[d];
        if (ndim == 0) size = 0;
    }

    void _init(const Dtype &dt, int nd, const long *shp, const long *str, int flags)
    {
        if (nd < 0 || nd > ArrayMaxDim) throw std::runtime_error("ksgpu::Array: bad ndim");
        if (dt.nbits == 0 || dt.nbits % 8) throw std::runtime_error("ksgpu::Array: bad dtype " + dt.str());
        dtype = dt;
        ndim = nd;
        aflags = flags & af_location_flags;
        for (int d = 0; d < nd; d++) {
            if (shp[d] < 0) throw std::runtime_error("ksgpu::Array: negative shape");
            shape[d] = shp[d];
        }
        _set_size();
        std::vector<long> s = str ? std::vector<long>(str, str + nd) : make_contiguous_strides(std::vector<long>(shp, shp + nd));
        long span = 1;
        for (int d = 0; d < nd; d++) {
            if (s[d] < 0) throw std::runtime_error("ksgpu::Array: negative strides are not supported");
            strides[d] = s[d];
            if (shape[d] > 0) span += (shape[d] - 1) * s[d];
        }
        if (size == 0) span = 0;
        base = af_alloc(span * (dt.nbits / 8), flags);
        data = (T *) base.get();
        if (flags & af_random) _randomize_elements();
    }

    // af_random: floating-point elements uniform in [-1, 1], integer elements uniform in [0, 100).
    void _randomize_elements() const
    {
        std::mt19937 &rng = default_rng();
        std::uniform_real_distribution<double> u(-1.0, 1.0);
        std::vector<long> ix(ndim, 0);
        for (long n = 0; n < size; n++) {
            long o = 0;
            for (int d = 0; d < ndim; d++) o += ix[d] * strides[d];
            char *p = (char *) data + o * (dtype.nbits / 8);
            _store(p, dtype, (dtype.flags & df_float) ? u(rng) : double(rand_int(0, 100, rng)));
            for (int d = ndim - 1; d >= 0; d--) { if (++ix[d] < shape[d]) break; ix[d] = 0; }
        }
    }

    T *_advance(long nelts) const { return (T *) ((char *) data + nelts * (dtype.nbits / 8)); }
    elt_ref _elt(long o) const
    {
        if constexpr (std::is_void_v<T>) throw std::runtime_error("ksgpu::Array<void>::at() is not available");
        else return data[o];
    }

    void _copy_rec(int d, char *dst, const char *src, const long *sstr) const
    {
        long es = dtype.nbits / 8;
        if (d == ndim - 1) {
            if (strides[d] == 1 && sstr[d] == 1) { memmove(dst, src, shape[d] * es); return; }
            for (long i = 0; i < shape[d]; i++) memmove(dst + i * strides[d] * es, src + i * sstr[d] * es, es);
            return;
        }
        for (long i = 0; i < shape[d]; i++)
            _copy_rec(d + 1, dst + i * strides[d] * es, src + i * sstr[d] * es, sstr);
    }
};

// Initializes every member of 'arr' except 'data' and 'base' (allocating them too if 'allocate'),
// and returns the number of elements that an allocation must span.
inline long _array_init_dchecked(Array<void> &arr, const Dtype &dtype, int ndim, const long *shape, const long *strides,
                                 int aflags, bool allocate)
{
    Array<void> tmp(dtype, std::vector<long>(), af_uhost);   // dtype checks only
    if (ndim < 0 || ndim > ArrayMaxDim) throw std::runtime_error("ksgpu::_array_init_dchecked: bad ndim");
    arr = Array<void>();
    arr.dtype = dtype;
    arr.ndim = ndim;
    arr.aflags = aflags & af_location_flags;
    std::vector<long> shp(shape, shape + ndim);
    std::vector<long> str = strides ? std::vector<long>(strides, strides + ndim) : make_contiguous_strides(shp);
    long span = 1;
    for (int d = 0; d < ndim; d++) {
        if (shp[d] < 0 || str[d] < 0) throw std::runtime_error("ksgpu::_array_init_dchecked: negative shape or stride");
        arr.shape[d] = shp[d];
        arr.strides[d] = str[d];
        if (shp[d] > 0) span += (shp[d] - 1) * str[d];
    }
    arr._set_size();
    if (arr.size == 0) span = 0;
    if (allocate && span > 0) {
        arr.base = af_alloc(span * (dtype.nbits / 8), aflags);
        arr.data = arr.base.get();
        if (aflags & af_random) arr._randomize_elements();
    }
    return span;
}

// Throws if two arrays of equal shape differ by more than epsabs + epsrel * |b| anywhere.
template<typename T, typename U>
inline double assert_arrays_equal(const Array<T> &a, const Array<U> &b, const std::string &na, const std::string &nb,
                                  const std::vector<std::string> &axis_names, float epsabs = 3.0e-5f, float epsrel = 1.0e-5f,
                                  long = 0, bool = false)
{
    xassert(a.shape_equals(b.ndim, b.shape));
    xassert(int(axis_names.size()) == a.ndim);
    Array<double> ad = Array<void>(a).convert(Dtype::native<double>()).template cast<double>();
    Array<double> bd = Array<void>(b).convert(Dtype::native<double>()).template cast<double>();
    double maxdiff = 0;
    for (long i = 0; i < ad.size; i++) {
        double x = ad.data[i], y = bd.data[i];
        double d = std::fabs(x - y);
        if (!(d <= epsabs + epsrel * std::fabs(y)) && !(std::isnan(x) && std::isnan(y))) {
            std::stringstream ss;
            ss << "assert_arrays_equal: " << na << " and " << nb << " differ at flat index " << i << ": " << x << " vs " << y;
            throw std::runtime_error(ss.str());
        }
        if (d > maxdiff) maxdiff = d;
    }
    return maxdiff;
}

inline std::shared_ptr<void> _af_alloc(const Dtype &dtype, long nelts, int aflags)
{
    return af_alloc((nelts * dtype.nbits + 7) / 8, aflags);
}

inline void _check_array_invariants_except_dtype(const Array<void> &arr, const char *where)
{
    if (arr.ndim < 0 || arr.ndim > ArrayMaxDim) throw std::runtime_error(std::string(where) + ": bad ndim");
    if (arr.size > 0 && !arr.data) throw std::runtime_error(std::string(where) + ": null data");
}

}  // namespace ksgpu

#endif
