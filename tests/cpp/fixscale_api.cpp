// fixscale_api.cpp -- C wrappers over csrc/fixscale.h (the scale of the
// deterministic mode's integer node sums) for tests/test_fixpoint_host.py.
// Test infrastructure only.
#include <cstdint>
#include "fixscale.h"

extern "C" int fx_exponent(unsigned cbits, long long n) { return dmpm::fix_exponent(cbits, n); }
extern "C" float fx_pow2(int k) { return dmpm::fix_pow2(k); }

// Sum n float contributions the way the kernels do: each rounded once to
// round(x 2^k) (round half to even, as __float2ll_rn) and added as int64
// (wrapping, as the 64-bit atomics do); back to float as __ll2float_rn(sum) 2^-k.
// order[] gives the order of the adds.  Returns the float node value.
extern "C" float fx_sum(const float* x, const int* order, long long n, int k, long long* isum) {
    const float s = dmpm::fix_pow2(k);
    unsigned long long acc = 0;
    for (long long i = 0; i < n; i++) {
        const float v = x[order[i]] * s;
        const long long q = (long long)std::nearbyint((double)v);  // v is a float: exact in double
        acc += (unsigned long long)q;
    }
    *isum = (long long)acc;
    return (float)(long long)acc * dmpm::fix_pow2(-k);
}
