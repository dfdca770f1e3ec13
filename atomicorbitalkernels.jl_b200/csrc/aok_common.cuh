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
constexpr int kMaxPairs = 256;     // species pairs (NZ <= 16)

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialisation may start while its predecessor in the stream still runs;
// pdl_wait() blocks until that predecessor has completed and its writes are
// visible (a no-op for a kernel launched without the attribute), and
// pdl_trigger() lets the successor's launch begin before this kernel ends.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Cartesian component c of a shell of momentum l, in the reference's order
// (kernels_2c.jl:102-119): for x = l..0, for z = 0..l-x: (x, y = l-x-z, z).
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

// 2^x with the hardware approximation (MUFU ex2, flushes subnormal results).
__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Error-free sum a + b = s + e (Knuth TwoSum).
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
    s = a + b;
    float bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

// Primitive-pair record of one (species pair, shell pair) of class (la, lb):
// everything that does not depend on the geometry, computed once per call in
// FP64.  With p = a + b, w = c_a c_b (pi/p)^{3/2} and the moment slots
// (al, be) used by the class (al <= la, be <= lb, (la - al) + (lb - be) even,
// ga = (la + lb - al - be) / 2), in slot order:
//   FP32:  w rb^al ra^be q^ga per slot;  mu log2(e) as hi, lo;  row length
//          (the slot values first, so that pairs of them are aligned register
//          pairs for the paired FMA)
//   FP64:  mu;                    row length;  w rb^al ra^be q^ga per slot
// (ra = a/p, rb = b/p, q = 1/2p), padded to whole 16-byte words.  The row
// length is the number of non-zero ket coefficients: records form rows of
// equal length, one per bra primitive.
__host__ __device__ constexpr int md_nv(int la, int lb) {
    return ((la + 1) * (lb + 1) + (((la + lb) & 1) == 0 ? 1 : 0)) / 2;
}
__host__ __device__ constexpr int rec_words16_f32(int la, int lb) { return (3 + md_nv(la, lb) + 3) / 4; }
__host__ __device__ constexpr int rec_words16_f64(int la, int lb) { return (2 + md_nv(la, lb) + 1) / 2; }
constexpr int kRecMaxBytesF32 = 16 * rec_words16_f32(kMaxL, kMaxL);
constexpr int kRecMaxBytesF64 = 16 * rec_words16_f64(kMaxL, kMaxL);
static_assert(md_nv(3, 3) == 8 && md_nv(2, 3) == 6 && md_nv(1, 1) == 2 && md_nv(0, 1) == 1, "moment slots");

// Work item: a shell pair (sa, sb).
struct Item {
    int16_t cls;    // la*4 + lb
    int16_t chunk;  // 2C forward execution order: the item's primitive-pair count
    int16_t sa, sb;
};

// 2C forward stage images.  Per species pair, the records of the items in
// execution order are cut into chunks that fit the kernel's shared-memory
// stage; a chunk is [one ExecItem per item, padded to 16 bytes][the items'
// records].  A segment is a run of items of one panel inside one chunk.
struct __align__(8) ExecItem {
    int16_t cls;  // la*4 + lb
    int16_t n;    // primitive pairs (records)
    int16_t rec;  // 16-byte offset of the item's first record in the stage
    int16_t dst;  // element offset of the block's (0,0) entry in a lane's slab
};
struct __align__(8) Seg {
    int it0, it1;  // items [it0, it1) of the pair's execution order
    int ibase;     // first item of the chunk: its ExecItem opens the stage
    int off;       // 16-byte offset of the chunk in the packed array
    int n16;       // chunk size, 16-byte words
    int pn;        // panel, + kSegPanelEnd when the segment closes the panel
};
constexpr int kSegPanelEnd = 256;

struct Panels {
    int n;                          // number of panels
    int col0[kMaxPanels + 1];       // first output column of each panel (+ N)
    int item0[kMaxPanels + 1];      // first item of each panel in the item list
};

}  // namespace aok
