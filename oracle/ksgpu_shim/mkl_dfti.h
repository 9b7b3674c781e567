// Minimal stand-in for MKL's DFTI interface (MKL is not installed here), for the oracle/_ref build
// only: the one transform pirate's simpulse.cpp uses, a 1-d double-precision complex-to-real backward
// DFT of a conjugate-even (n/2 + 1)-entry input ("CCE" storage), out-of-place and unnormalized:
//   x[j] = sum_{k=0}^{n-1} X[k] exp(+2 pi i j k / n),  X[n-k] = conj(X[k]).
// Computed as a complex radix-2 Cooley-Tukey transform of the Hermitian-completed input when n is a
// power of two, and as a direct sum otherwise.
#ifndef _MKL_DFTI_SHIM_H
#define _MKL_DFTI_SHIM_H

#include <cmath>
#include <complex>
#include <vector>

typedef long MKL_LONG;

enum DFTI_CONFIG_PARAM { DFTI_PRECISION, DFTI_FORWARD_DOMAIN, DFTI_CONJUGATE_EVEN_STORAGE, DFTI_PLACEMENT };
enum DFTI_CONFIG_VALUE { DFTI_SINGLE, DFTI_DOUBLE, DFTI_REAL, DFTI_COMPLEX, DFTI_COMPLEX_COMPLEX, DFTI_COMPLEX_REAL,
                         DFTI_INPLACE, DFTI_NOT_INPLACE };
enum { DFTI_NO_ERROR = 0, DFTI_BAD_DESCRIPTOR = 1, DFTI_UNIMPLEMENTED = 2 };

struct DFTI_DESCRIPTOR
{
    long n = 0;
    bool real_double = false, cce = false, not_inplace = false, committed = false;
};
typedef DFTI_DESCRIPTOR *DFTI_DESCRIPTOR_HANDLE;

inline long DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE *h, DFTI_CONFIG_VALUE prec, DFTI_CONFIG_VALUE dom, long dim, long n)
{
    if (prec != DFTI_DOUBLE || dom != DFTI_REAL || dim != 1 || n < 1) return DFTI_UNIMPLEMENTED;
    *h = new DFTI_DESCRIPTOR;
    (*h)->n = n;
    (*h)->real_double = true;
    return DFTI_NO_ERROR;
}

inline long DftiSetValue(DFTI_DESCRIPTOR_HANDLE h, DFTI_CONFIG_PARAM p, DFTI_CONFIG_VALUE v)
{
    if (!h) return DFTI_BAD_DESCRIPTOR;
    if (p == DFTI_CONJUGATE_EVEN_STORAGE && v == DFTI_COMPLEX_COMPLEX) { h->cce = true; return DFTI_NO_ERROR; }
    if (p == DFTI_PLACEMENT && v == DFTI_NOT_INPLACE) { h->not_inplace = true; return DFTI_NO_ERROR; }
    return DFTI_UNIMPLEMENTED;
}

inline long DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE h)
{
    if (!h || !h->cce || !h->not_inplace) return DFTI_UNIMPLEMENTED;
    h->committed = true;
    return DFTI_NO_ERROR;
}

inline long DftiComputeBackward(DFTI_DESCRIPTOR_HANDLE h, void *in, void *out)
{
    if (!h || !h->committed) return DFTI_BAD_DESCRIPTOR;
    typedef std::complex<double> cd;
    const long n = h->n;
    const cd *X = (const cd *) in;
    double *x = (double *) out;
    std::vector<cd> a(n);
    for (long k = 0; k <= n / 2; k++) a[k] = X[k];
    for (long k = n / 2 + 1; k < n; k++) a[k] = std::conj(X[n - k]);
    if ((n & (n - 1)) == 0) {
        // bit-reversal permutation, then iterative butterflies with the +i sign
        for (long i = 1, j = 0; i < n; i++) {
            long bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) std::swap(a[i], a[j]);
        }
        for (long len = 2; len <= n; len <<= 1) {
            const double ang = 2.0 * M_PI / double(len);
            for (long i = 0; i < n; i += len)
                for (long k = 0; k < len / 2; k++) {
                    cd w(std::cos(ang * k), std::sin(ang * k));
                    cd u = a[i + k], v = a[i + k + len / 2] * w;
                    a[i + k] = u + v;
                    a[i + k + len / 2] = u - v;
                }
        }
        for (long j = 0; j < n; j++) x[j] = a[j].real();
    }
    else {
        for (long j = 0; j < n; j++) {
            cd s = 0;
            for (long k = 0; k < n; k++) s += a[k] * std::polar(1.0, 2.0 * M_PI * double((j * k) % n) / double(n));
            x[j] = s.real();
        }
    }
    return DFTI_NO_ERROR;
}

inline long DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE *h)
{
    delete *h;
    *h = nullptr;
    return DFTI_NO_ERROR;
}

inline bool DftiErrorClass(long status, long cls) { return status == cls; }
inline const char *DftiErrorMessage(long status) { return status == DFTI_NO_ERROR ? "no error" : "DFTI stand-in: unsupported call"; }

#endif
