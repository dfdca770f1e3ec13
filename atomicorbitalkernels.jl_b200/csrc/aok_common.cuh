// aok_common.cuh -- device helpers shared by the overlap and orbital kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "aok.h"

namespace aok {

constexpr int kMaxL = AOK_MAX_L;
constexpr int kTileB = 32;          // batch elements per tile (one per lane)
constexpr int kMaxPanels = 16;
constexpr int kMaxShells = 64;

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }

// Cartesian component c of a shell of momentum l, in the reference's order
// (kernels_2c.jl:201-217): for x = l..0, for z = 0..l-x: (x, y = l-x-z, z).
// Closed form (no loops, so unrolled call sites fold instantly): with
// n = l - x, the first component of that x is n(n+1)/2, so
// n = #{t >= 1 : t(t+1)/2 <= c} and z = c - n(n+1)/2.
__host__ __device__ constexpr int cart_n(int c) {
    return (c >= 1) + (c >= 3) + (c >= 6) + (c >= 10) + (c >= 15) + (c >= 21);
}
__host__ __device__ constexpr int cart_x(int l, int c) { return l - cart_n(c); }
__host__ __device__ constexpr int cart_z(int l, int c) { return c - cart_n(c) * (cart_n(c) + 1) / 2; }
__host__ __device__ constexpr int cart_y(int l, int c) { return l - cart_x(l, c) - cart_z(l, c); }

// Accumulator elements per work item (register budget); larger shell-pair
// blocks are split into chunks of output elements.
__host__ __device__ constexpr int max_elems() { return 36; }
__host__ __device__ constexpr int nchunks(int ne) { return (ne + max_elems() - 1) / max_elems(); }

// Error-free sum a + b = s + e (Knuth TwoSum).
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
    s = a + b;
    float bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

// Primitive-pair record of one (species pair, shell pair): everything that
// does not depend on the geometry, computed once per call in FP64.
//   w    = c_a c_b (pi/p)^{3/2}
//   mu   = a b / p (FP64 record); mu log2(e) as hi + lo (FP32 record)
//   ra   = a/p,  rb = b/p,  oo2p = 1/(2p), flush = row length (non-zero ket coefficients).
struct PPf {
    float w, mu_hi, mu_lo, ra, rb, oo2p, flush, pad;
};
struct PPd {
    double w, mu, ra, rb, oo2p, flush, pad0, pad1;
};
template <typename FT> struct PPT;
template <> struct PPT<float> { using type = PPf; };
template <> struct PPT<double> { using type = PPd; };

// Work item: a shell pair (sa, sb), or a chunk of its output elements.
struct Item {
    int16_t cls;    // la*4 + lb
    int16_t chunk;
    int16_t sa, sb;
};

struct Panels {
    int n;                          // number of panels
    int col0[kMaxPanels + 1];       // first output column of each panel (+ N)
    int item0[kMaxPanels + 1];      // first item of each panel in the item list
};

}  // namespace aok
