// fixscale.h -- the scale of the deterministic mode's integer node sums
// (fixpoint.cuh), in plain C++ so that host code and host tests use the same
// functions as the kernels.
#pragma once
#include <cmath>
#include <cstring>

#ifdef __CUDACC__
#define DMPM_FIX_HD __host__ __device__ __forceinline__
#else
#define DMPM_FIX_HD inline
#endif

namespace dmpm {

// bound slots (one unsigned float bit pattern each)
enum : int { FIXB_MOMENTUM = 0, FIXB_MASS = 1, FIXB_ADJ = 2, FIXB_RASTER = 3, FIXB_SLOTS = 4 };

DMPM_FIX_HD float fix_bits_to_float(unsigned b) {
    float f;
    memcpy(&f, &b, sizeof(f));
    return f;
}

// k for a pass over n particles whose contributions are bounded by the float
// with bit pattern cbits; clamped to [-126, 126] so that 2^k and 2^-k are
// normal floats (a non-finite bound gives -126: the pass's inputs were not
// finite, which the kernels that made them report)
DMPM_FIX_HD int fix_exponent(unsigned cbits, long long n) {
    const float c = fix_bits_to_float(cbits);
    int e = 0;
    if (!(c <= 3.4e38f)) return -126;
    if (c > 0.f) {
        (void)frexpf(c, &e);  // c = f 2^e, f in [0.5, 1): c < 2^e
    } else {
        e = -126;  // no contribution is nonzero
    }
    int b = 0;
    while (b < 62 && (1ll << b) < n) b++;
    int k = 61 - e - b;
    if (k > 126) k = 126;
    if (k < -126) k = -126;
    return k;
}

// 2^k as a float, k in [-126, 127]
DMPM_FIX_HD float fix_pow2(int k) {
    const unsigned b = (unsigned)(k + 127) << 23;
    return fix_bits_to_float(b);
}

}  // namespace dmpm
