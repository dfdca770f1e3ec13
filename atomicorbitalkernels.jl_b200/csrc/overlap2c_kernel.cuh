// overlap2c_kernel.cuh -- the persistent 2-center overlap kernel, templated
// on the element type; instantiated once per precision (overlap2c_f32.cu,
// overlap2c_f64.cu) so the two builds compile in parallel.  See overlap2c.cu
// for the design notes.
#pragma once

#include <cstring>

#include "aok_internal.h"
#include "md2c.cuh"

namespace aok {

// 256 threads per CTA; CTAs per SM (the plan's fwd_ctas): FP32 2 (registers
// <= 128), or 3 for bases of <= 2 primitives per shell (<= 80 registers: the
// few f-f items spill a little, the many cheap items gain latency hiding);
// FP64 1, or 2 for such bases.
constexpr int kThreadsF32 = 256;
constexpr int kThreadsF64 = 256;

// --------------------------------------------------------------------------
// Geometry per lane.
// --------------------------------------------------------------------------
template <typename FT> struct Geo;
template <> struct Geo<float> {
    float AB[3];
    float R2, R2lo;
};
template <> struct Geo<double> {
    double AB[3];
    double R2;
};

__device__ __forceinline__ void load_geo(Geo<float>& g, const float* A, const float* B, float s, bool use_s) {
    double R2 = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float a = A[c], b = B[c];
        if (use_s) {
            a = a * s;
            b = b * s;
        }
        double d = (double)a - (double)b;  // exact
        g.AB[c] = (float)d;
        R2 += d * d;
    }
    g.R2 = (float)R2;
    g.R2lo = (float)(R2 - (double)g.R2);
}
__device__ __forceinline__ void load_geo(Geo<double>& g, const double* A, const double* B, double s, bool use_s) {
    double R2 = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double a = A[c], b = B[c];
        if (use_s) {
            a = a * s;
            b = b * s;
        }
        double d = a - b;
        g.AB[c] = d;
        R2 += d * d;
    }
    g.R2 = R2;
}

// --------------------------------------------------------------------------
// Shared-memory record access (the warp stages an item's records first).
// --------------------------------------------------------------------------
__device__ __forceinline__ float4 lds128(uint32_t a) {
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
    return v;
}
__device__ __forceinline__ double2 lds128d(uint32_t a) {
    double2 v;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a));
    return v;
}

// Zero block (a shell pair with no primitive pair: an absent shell).
template <int LA, int LB, typename FT>
__device__ __forceinline__ void md_zero(FT* dst, int N) {
#pragma unroll
    for (int j = 0; j < ncart(LB); ++j)
#pragma unroll
        for (int i = 0; i < ncart(LA); ++i) dst[j * N + i] = FT(0);
}

// --------------------------------------------------------------------------
// One work item (shell pair) for one lane (batch element): FP32C.
// rec: shared-memory address of the item's n records (class-sized, see
// aok_common.cuh), ip-major in rows of equal length.  dst points at the
// block's (0,0) element inside this lane's slab; element (i, j) of the block
// lives at dst[j*N + i].  Moment m += exp(-mu R^2) * (w mono_m); the partial
// sums of a row are folded into (hi, lo) with TwoSum at the end of the row.
// --------------------------------------------------------------------------
__device__ __forceinline__ float lds32(uint32_t a) {
    float v;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
    return v;
}

// One primitive pair (n == 1): the moments are the record's slot values times
// its exponential; no loop and no compensation are needed.
template <int LA, int LB>
__device__ __forceinline__ void run_item1_body(uint32_t rec, const Geo<float> g, float* dst, int N) {
    constexpr int NM = (LA + 1) * (LB + 1), NV = md_nv(LA, LB), R16 = rec_words16_f32(LA, LB);
    float r[4 * R16];
#pragma unroll
    for (int w = 0; w < R16; ++w) {
        const float4 v = lds128(rec + 16u * w);
        r[4 * w] = v.x;
        r[4 * w + 1] = v.y;
        r[4 * w + 2] = v.z;
        r[4 * w + 3] = v.w;
    }
    const float m0 = r[NV], m1 = r[NV + 1];
    const float xh = m0 * g.R2;
    const float xl = fmaf(m0, g.R2, -xh) + fmaf(m1, g.R2, m0 * g.R2lo);
    const float e = ex2_approx(-xh) * fmaf(-0.6931471805599453f, xl, 1.f);
    float M[NM];
    int j = 0;
#pragma unroll
    for (int al = 0; al <= LA; ++al)
#pragma unroll
        for (int be = 0; be <= LB; ++be) {
            M[al * (LB + 1) + be] = 0.f;
            if (MdTab<LA, LB>::used(al, be)) {
                M[al * (LB + 1) + be] = e * r[j];
                ++j;
            }
        }
    md_transform<LA, LB, float>(M, g.AB, dst, N);
}

template <int LA, int LB>
__device__ __forceinline__ void run_item_body(uint32_t rec, int n, const Geo<float> g, float* dst, int N) {
    constexpr int NM = (LA + 1) * (LB + 1), NV = md_nv(LA, LB), NP = (NV + 1) / 2, R16 = rec_words16_f32(LA, LB);
    if (n == 0) {
        md_zero<LA, LB, float>(dst, N);
        return;
    }
    // moment sums in slot order: hi + lo per slot, and the current row's partial
    // sums as pairs (slots 2i, 2i+1; for odd NV the last pair's second half is unused)
    float hi[NV], lo[NV];
    float2 part[NP];
#pragma unroll
    for (int j = 0; j < NV; ++j) hi[j] = lo[j] = 0.f;
#pragma unroll
    for (int i = 0; i < NP; ++i) part[i] = make_float2(0.f, 0.f);
    const int rowlen = (int)lds32(rec + 4u * (NV + 2));
    for (int q0 = 0; q0 < n; q0 += rowlen) {
        for (int q = q0; q < q0 + rowlen; ++q) {
            float r[4 * R16];
#pragma unroll
            for (int w = 0; w < R16; ++w) {
                const float4 v = lds128(rec + 16u * (R16 * q + w));
                r[4 * w] = v.x;
                r[4 * w + 1] = v.y;
                r[4 * w + 2] = v.z;
                r[4 * w + 3] = v.w;
            }
            // exp(-mu R^2) = 2^-(mu2 R^2), argument in double-float (mu2 = hi + lo):
            // 2^-(xh + xl) = 2^-xh (1 - ln2 xl) to first order in |xl| < 2^-20 xh
            const float m0 = r[NV], m1 = r[NV + 1];
            const float xh = m0 * g.R2;
            const float xl = fmaf(m0, g.R2, -xh) + fmaf(m1, g.R2, m0 * g.R2lo);
            const float e = ex2_approx(-xh) * fmaf(-0.6931471805599453f, xl, 1.f);
            const float2 ee = make_float2(e, e);
#pragma unroll
            for (int i = 0; i < NP; ++i) part[i] = __ffma2_rn(ee, make_float2(r[2 * i], r[2 * i + 1]), part[i]);
        }
        if (q0 == 0) {  // the first row opens the sums exactly
#pragma unroll
            for (int j = 0; j < NV; ++j) hi[j] = (j & 1) ? part[j / 2].y : part[j / 2].x;
        } else {
#pragma unroll
            for (int j = 0; j < NV; ++j) {
                float s, e;
                two_sum(hi[j], (j & 1) ? part[j / 2].y : part[j / 2].x, s, e);
                hi[j] = s;
                lo[j] += e;
            }
        }
#pragma unroll
        for (int i = 0; i < NP; ++i) part[i] = make_float2(0.f, 0.f);
    }
    float M[NM];
    int j = 0;
#pragma unroll
    for (int al = 0; al <= LA; ++al)
#pragma unroll
        for (int be = 0; be <= LB; ++be) {
            M[al * (LB + 1) + be] = 0.f;
            if (MdTab<LA, LB>::used(al, be)) {
                M[al * (LB + 1) + be] = hi[j] + lo[j];
                ++j;
            }
        }
    md_transform<LA, LB, float>(M, g.AB, dst, N);
}

// FP64, one primitive pair: no loop.
template <int LA, int LB>
__device__ __forceinline__ void run_item1_body(uint32_t rec, const Geo<double> g, double* dst, int N) {
    constexpr int NM = (LA + 1) * (LB + 1), R16 = rec_words16_f64(LA, LB);
    double r[2 * R16];
#pragma unroll
    for (int w = 0; w < R16; ++w) {
        const double2 v = lds128d(rec + 16u * w);
        r[2 * w] = v.x;
        r[2 * w + 1] = v.y;
    }
    const double e = exp(-r[0] * g.R2);
    double mom[NM];
    int j = 0;
#pragma unroll
    for (int al = 0; al <= LA; ++al)
#pragma unroll
        for (int be = 0; be <= LB; ++be) {
            mom[al * (LB + 1) + be] = 0.0;
            if (MdTab<LA, LB>::used(al, be)) {
                mom[al * (LB + 1) + be] = e * r[2 + j];
                ++j;
            }
        }
    md_transform<LA, LB, double>(mom, g.AB, dst, N);
}

// FP64 variant: plain double accumulation, records from shared memory.
template <int LA, int LB>
__device__ __forceinline__ void run_item_body(uint32_t rec, int n, const Geo<double> g, double* dst, int N) {
    constexpr int NM = (LA + 1) * (LB + 1), R16 = rec_words16_f64(LA, LB);
    if (n == 0) {
        md_zero<LA, LB, double>(dst, N);
        return;
    }
    double mom[NM];
#pragma unroll
    for (int m = 0; m < NM; ++m) mom[m] = 0.0;
    for (int q = 0; q < n; ++q) {
        double r[2 * R16];
#pragma unroll
        for (int w = 0; w < R16; ++w) {
            const double2 v = lds128d(rec + 16u * (R16 * q + w));
            r[2 * w] = v.x;
            r[2 * w + 1] = v.y;
        }
        const double e = exp(-r[0] * g.R2);
        int j = 0;
#pragma unroll
        for (int al = 0; al <= LA; ++al)
#pragma unroll
            for (int be = 0; be <= LB; ++be)
                if (MdTab<LA, LB>::used(al, be)) {
                    mom[al * (LB + 1) + be] = fma(e, r[2 + j], mom[al * (LB + 1) + be]);
                    ++j;
                }
    }
    md_transform<LA, LB, double>(mom, g.AB, dst, N);
}

template <int LA, int LB, typename FT>
__device__ __noinline__ void run_item(uint32_t rec, int n, const Geo<FT> g, FT* dst, int N) {
    run_item_body<LA, LB>(rec, n, g, dst, N);
}

// Classes with l <= 1 on both sides run inline, and an item of one
// primitive pair takes the loop-free routine: for these few-output blocks a call
// and the loop cost more than the arithmetic.  The other classes run as calls
// (one copy of each class's code, so the kernel keeps its register budget and
// the instruction cache holds the loop).
template <int LA, int LB>
__device__ __forceinline__ void run_class(uint32_t rec, int n, const Geo<float>& g, float* dst, int N) {
    if constexpr (LA <= 1 && LB <= 1) {
        if (n == 1)
            run_item1_body<LA, LB>(rec, g, dst, N);
        else
            run_item_body<LA, LB>(rec, n, g, dst, N);
    } else {
        run_item<LA, LB, float>(rec, n, g, dst, N);
    }
}
template <int LA, int LB>
__device__ __forceinline__ void run_class(uint32_t rec, int n, const Geo<double>& g, double* dst, int N) {
    if constexpr (LA <= 1 && LB <= 1) {
        if (n == 1)
            run_item1_body<LA, LB>(rec, g, dst, N);
        else
            run_item_body<LA, LB>(rec, n, g, dst, N);
    } else {
        run_item<LA, LB, double>(rec, n, g, dst, N);
    }
}

template <typename FT>
__device__ __forceinline__ void dispatch(int cls, uint32_t pp, int n, const Geo<FT>& g, FT* dst, int N) {
    switch (cls) {
#define AOK_CASE(LA, LB) \
    case (LA) * 4 + (LB): run_class<LA, LB>(pp, n, g, dst, N); break;
        AOK_CASE(0, 0) AOK_CASE(0, 1) AOK_CASE(0, 2) AOK_CASE(0, 3)
        AOK_CASE(1, 0) AOK_CASE(1, 1) AOK_CASE(1, 2) AOK_CASE(1, 3)
        AOK_CASE(2, 0) AOK_CASE(2, 1) AOK_CASE(2, 2) AOK_CASE(2, 3)
        AOK_CASE(3, 0) AOK_CASE(3, 1) AOK_CASE(3, 2) AOK_CASE(3, 3)
#undef AOK_CASE
        default: break;
    }
}

template <typename FT>
struct Ov2Params {
    FT* out;
    const FT* posA;
    const FT* posB;
    FT scale;
    int use_scale;
    const float4* pk;     // stage images: per species pair, chunks of [ExecItem...][records]
    const Seg* segs;      // per species pair: seg_stride segments
    const int* nseg;      // segments per species pair
    int seg_stride;
    const int* perm;
    const int4* tiles;
    const int* ntiles;
    unsigned* counter;
    Panels panels;
    int N, slab_stride;
    unsigned stage_offset;  // byte offset of the stage in dynamic shared memory
};

// Copy n16 16-byte words of a packed chunk into the stage, all threads, four
// loads in flight per thread.
template <int THREADS>
__device__ __forceinline__ void stage_chunk(float4* dst, const float4* __restrict__ src, int n16) {
    int i = threadIdx.x;
    for (; i + 3 * THREADS < n16; i += 4 * THREADS) {
        const float4 v0 = __ldg(src + i), v1 = __ldg(src + i + THREADS), v2 = __ldg(src + i + 2 * THREADS),
                     v3 = __ldg(src + i + 3 * THREADS);
        dst[i] = v0;
        dst[i + THREADS] = v1;
        dst[i + 2 * THREADS] = v2;
        dst[i + 3 * THREADS] = v3;
    }
    for (; i < n16; i += THREADS) dst[i] = __ldg(src + i);
}

// Geometry of the tile's 32 lanes (zero geometry for lanes past the tile's end)
// and each lane's batch element (b).
template <typename FT>
__device__ __forceinline__ void tile_geo(Geo<FT>& g, int& b, const Ov2Params<FT>& P, int start, int cnt, int lane) {
    b = 0;
    if (lane < cnt) {
        b = P.perm[start + lane];
        load_geo(g, P.posA + 3 * (size_t)b, P.posB + 3 * (size_t)b, P.scale, P.use_scale != 0);
    } else {
        const FT z[3] = {FT(0), FT(0), FT(0)};
        load_geo(g, z, z, P.scale, false);
    }
}

// Persistent CTAs take tiles (<= 32 batch elements of one species pair, one per
// lane) from a global queue.  Per tile the CTA walks the pair's segments: the
// warps take the segment's items from a shared counter and run them on the
// staged chunk, writing their blocks into the lane's slab of the current panel;
// at a panel's end the CTA streams the slab out.  A chunk is copied into the
// stage only when it is not there already (consecutive tiles of one species
// pair whose records fit one chunk stage them once).  The next tile is
// claimed when the last segment starts, and its geometry and first chunk are
// fetched while the last panel streams out, so a tile starts without a wait.
template <typename FT, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB) k_overlap2c(const __grid_constant__ Ov2Params<FT> P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FT* slab = reinterpret_cast<FT*>(smem_raw);
    float4* stage = reinterpret_cast<float4*>(smem_raw + P.stage_offset);
    const ExecItem* sitems = reinterpret_cast<const ExecItem*>(stage);
    const uint32_t stage_saddr = (uint32_t)__cvta_generic_to_shared(stage);
    __shared__ int s_tile, s_cnt;
    __shared__ int4 s_td;
    __shared__ Geo<FT> s_geo[32];
    __shared__ int s_b[2][32];  // batch element of each lane, double-buffered across tiles
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = THREADS / 32;
    const int ntiles = *P.ntiles;
    int staged = -1;  // packed offset of the chunk in the stage (the same in every thread)
    // prologue: the first tile, its geometry and its first chunk
    if (threadIdx.x == 0) {
        s_tile = (int)atomicAdd(P.counter, 1u);
        s_cnt = 0;
    }
    __syncthreads();
    int tile = s_tile;
    if (tile < ntiles) {
        const int4 td = P.tiles[tile];
        if (warp == NW - 1) {
            Geo<FT> g;
            int b;
            tile_geo(g, b, P, td.y, td.z, lane);
            s_geo[lane] = g;
            s_b[0][lane] = b;
            if (lane == 0) s_td = td;
        }
        const Seg S0 = P.segs[(size_t)td.x * P.seg_stride];
        stage_chunk<THREADS>(stage, P.pk + S0.off, S0.n16);
        staged = S0.off;
    }
    __syncthreads();
    int buf = 0;  // s_b buffer of the current tile
    while (tile < ntiles) {
        const int4 td = s_td;
        const int pair = td.x, cnt = td.z;
        const Geo<FT> g = s_geo[lane];
        const Seg* segs = P.segs + (size_t)pair * P.seg_stride;
        const int nseg = P.nseg[pair];
        FT* sl = slab + (size_t)lane * P.slab_stride;
        int next = ntiles;
        Seg S = segs[0];
        for (int k = 0; k < nseg; ++k) {
            if (k == nseg - 1 && threadIdx.x == 0) s_tile = (int)atomicAdd(P.counter, 1u);
            for (;;) {
                int it = 0;
                if (lane == 0) it = atomicAdd(&s_cnt, 1);
                it = __shfl_sync(0xffffffffu, it, 0) + S.it0;
                if (it >= S.it1) break;
                const ExecItem e = sitems[it - S.ibase];
                dispatch(e.cls, stage_saddr + 16u * (uint32_t)e.rec, e.n, g, sl + e.dst, P.N);
            }
            const Seg Sn = k + 1 < nseg ? segs[k + 1] : S;
            __syncthreads();
            int4 tdn = make_int4(0, 0, 0, 0);
            if (k == nseg - 1) {
                next = s_tile;
                if (next < ntiles) {
                    tdn = P.tiles[next];
                    if (warp == NW - 1) {  // the next tile's geometry, ahead of this warp's share of the stores
                        Geo<FT> gn;
                        int bn;
                        tile_geo(gn, bn, P, tdn.y, tdn.z, lane);
                        s_geo[lane] = gn;
                        s_b[buf ^ 1][lane] = bn;
                        if (lane == 0) s_td = tdn;
                    }
                }
            }
            if (S.pn >= kSegPanelEnd) {  // the panel is complete: stream the slab out
                const int pn = S.pn - kSegPanelEnd;
                const int col0 = P.panels.col0[pn];
                const int len = (P.panels.col0[pn + 1] - col0) * P.N;
                for (int bl = warp; bl < cnt; bl += NW) {
                    const int bg = s_b[buf][bl];
                    FT* o = P.out + (size_t)bg * P.N * P.N + (size_t)col0 * P.N;
                    const FT* s = slab + (size_t)bl * P.slab_stride;
                    int e = lane;
                    for (; e + 96 < len; e += 128) {  // four loads in flight, streaming stores
                        const FT v0 = s[e], v1 = s[e + 32], v2 = s[e + 64], v3 = s[e + 96];
                        __stcs(o + e, v0);
                        __stcs(o + e + 32, v1);
                        __stcs(o + e + 64, v2);
                        __stcs(o + e + 96, v3);
                    }
                    for (; e < len; e += 32) __stcs(o + e, s[e]);
                }
            }
            if (k + 1 < nseg) {
                if (Sn.off != staged) {
                    stage_chunk<THREADS>(stage, P.pk + Sn.off, Sn.n16);
                    staged = Sn.off;
                }
            } else if (next < ntiles) {
                const Seg S0 = P.segs[(size_t)tdn.x * P.seg_stride];
                if (S0.off != staged) {
                    stage_chunk<THREADS>(stage, P.pk + S0.off, S0.n16);
                    staged = S0.off;
                }
            }
            if (threadIdx.x == 0) s_cnt = 0;
            __syncthreads();
            S = Sn;
        }
        tile = next;
        buf ^= 1;
    }
}

template <typename FT, int THREADS, int MINB>
inline int launch_ov2(aok_plan* p, void* out, const void* posA, const void* posB, double lengthscale,
                      cudaStream_t s) {
    Ov2Params<FT> P;
    memset(&P, 0, sizeof(P));
    P.out = (FT*)out;
    P.posA = (const FT*)posA;
    P.posB = (const FT*)posB;
    P.scale = (FT)lengthscale;
    P.use_scale = (FT)lengthscale != FT(1);
    P.pk = (const float4*)p->d_pk;
    P.segs = p->d_segs;
    P.nseg = p->d_nseg;
    P.seg_stride = p->seg_stride;
    P.perm = p->d_perm;
    P.tiles = p->d_tiles;
    P.ntiles = p->d_ntiles;
    P.counter = p->d_counter;
    P.panels = p->panels;
    P.N = (int)p->N;
    P.slab_stride = (int)p->slab_stride;
    const size_t slab = (p->smem_bytes + 15) / 16 * 16;
    P.stage_offset = (unsigned)slab;
    const size_t smem = slab + p->stage_bytes;
    auto kern = k_overlap2c<FT, THREADS, MINB>;
    const int st = kernel_prepare((const void*)kern, smem, THREADS, nullptr);
    if (st != AOK_OK) return st;
    timing_begin(p, s);
    kern<<<p->num_sms * MINB, THREADS, smem, s>>>(P);
    timing_end(p, s);
    return cuda_status(cudaGetLastError(), "k_overlap2c");
}


}  // namespace aok
