// fastdiv.h -- unsigned 32-bit division by a run-time invariant divisor with a
// multiply-high and two shifts (Granlund & Montgomery, "Division by invariant
// integers using multiplication", PLDI 1994, Figure 4.1).  Exact for all
// 32-bit numerators.
#pragma once
#include <stdint.h>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

namespace glsm {

struct FastDiv {
    unsigned d, m;
    int s1, s2;
};

inline FastDiv make_fastdiv(unsigned d) {
    FastDiv f;
    f.d = d ? d : 1;
    int l = 0;
    while ((1ull << l) < f.d) l++;
    f.m = (unsigned)(((1ull << 32) * ((1ull << l) - f.d)) / f.d + 1);
    f.s1 = l ? 1 : 0;
    f.s2 = l ? l - 1 : 0;
    return f;
}

__host__ __device__ __forceinline__ unsigned fdiv(unsigned n, const FastDiv& f) {
#ifdef __CUDA_ARCH__
    const unsigned t = __umulhi(n, f.m);
#else
    const unsigned t = (unsigned)(((unsigned long long)n * f.m) >> 32);
#endif
    return (t + ((n - t) >> f.s1)) >> f.s2;
}

}  // namespace glsm
