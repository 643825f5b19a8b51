// d3q19.cuh -- the D3Q19 velocity set in the reference's direction order
// (rest, 6 faces, then the xy, xz, yz diagonals; src/fluid.cu:202-215), as
// constexpr functions so that fully unrolled loops fold them to immediates.
#pragma once

namespace glsm {

__host__ __device__ __forceinline__ constexpr int qcx(int q) {
    return (q == 1 || q == 7 || q == 10 || q == 11 || q == 14) ? 1
           : (q == 2 || q == 8 || q == 9 || q == 12 || q == 13) ? -1
                                                                  : 0;
}
__host__ __device__ __forceinline__ constexpr int qcy(int q) {
    return (q == 3 || q == 7 || q == 8 || q == 15 || q == 16) ? 1
           : (q == 4 || q == 9 || q == 10 || q == 17 || q == 18) ? -1
                                                                   : 0;
}
__host__ __device__ __forceinline__ constexpr int qcz(int q) {
    return (q == 5 || q == 11 || q == 12 || q == 15 || q == 18) ? 1
           : (q == 6 || q == 13 || q == 14 || q == 16 || q == 17) ? -1
                                                                    : 0;
}
// opposite direction: faces pair (1,2),(3,4),(5,6); diagonals pair within
// groups of four as (7,9),(8,10),(11,13),(12,14),(15,17),(16,18)
__host__ __device__ __forceinline__ constexpr int qopp(int q) {
    return q == 0 ? 0 : (q <= 6 ? ((q & 1) ? q + 1 : q - 1) : 7 + ((q - 7) / 4) * 4 + (((q - 7) % 4) + 2) % 4);
}
__host__ __device__ __forceinline__ constexpr float qw(int q) {
    return q == 0 ? 1.0f / 3.0f : (q <= 6 ? 1.0f / 18.0f : 1.0f / 36.0f);
}

static_assert(qopp(7) == 9 && qopp(10) == 8 && qopp(13) == 11 && qopp(16) == 18 && qopp(5) == 6, "opp table");
static_assert(qcx(qopp(11)) == -1 && qcz(qopp(11)) == -1, "opp reverses");

}  // namespace glsm
