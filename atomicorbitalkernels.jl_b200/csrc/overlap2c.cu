// overlap2c.cu -- batched 2-center Cartesian-Gaussian overlap, sm_100a.
//
// Replaces batch_S_orbital_kernel! (src/integrals/orbital/overlap_2c.jl:15-131)
// and batch_S_kernel! (src/integrals/kernels_2c.jl:11-125).
//
// Pipeline per call (all stream-ordered, no host synchronisation):
//   k_pack2c    per species pair: the execution order of the shell pairs and
//               their geometry-free primitive-pair records (FP64-computed),
//               compacted to the non-zero-coefficient pairs in the
//               reference's (ip, jp) order and packed with item headers in
//               execution order into chunks that fit the forward kernel's
//               shared-memory stage.
//   k_bin_*     counting sort of the batch by species pair; tiles of 32
//               batch elements of one species pair; resets the work counter.
//   k_overlap2c persistent kernel (two CTAs per SM for FP32, one for FP64)
//               draining the tile queue (overlap2c_kernel.cuh).
//               Lane = batch element, so a warp runs one shell pair for 32
//               geometries with identical control flow.  Per shell pair the
//               primitive-pair loop accumulates the <= 8 moments
//               exp(-mu R^2) w rb^al ra^be q^ga (one FMA each), and the
//               compile-time geometry terms of the class (md2c.cuh) turn them
//               into the block once.  Records come from the shared-memory
//               stage; blocks go into a shared-memory slab holding complete
//               output columns of 32 batch elements, which is then streamed
//               out with coalesced stores (each batch element's (N,N) matrix
//               is contiguous in the reference layout).
//
// The reference's l >= 2 stride aliasing (block element lin = c1 + (2la+1)*c2,
// read back as blk[i + nbf_a*j], kernels_2c.jl:99-124) is reproduced at
// compile time in the term tables.
//
// FP32C precision: FP32 arithmetic on FP64-computed records; the Gaussian
// prefactor exp(-mu R^2) uses a double-float argument (mu log2 e and R^2 each
// carried as hi + lo), and the moments are summed per bra row in FP32 and
// folded into the running sums with TwoSum at each row's end.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "aok_internal.h"
#include "md2c.cuh"

namespace aok {

#define AOK_TRY_ST(x)                  \
    do {                               \
        int _st = (x);                 \
        if (_st != AOK_OK) return _st; \
    } while (0)

constexpr double kPi = 3.14159265358979323846;

// --------------------------------------------------------------------------
// GaussianBasis path: flat per-shell primitive lists -> padded (ns, K) tables.
// --------------------------------------------------------------------------
template <typename FT>
__global__ void k_gb_pad(FT* __restrict__ zeta, FT* __restrict__ coef, const int64_t* __restrict__ nprim,
                         const int64_t* __restrict__ off, const FT* __restrict__ c, const FT* __restrict__ a,
                         int ns, int K, int* err) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= ns * K) return;
    int s = q % ns, k = q / ns;
    int64_t n = nprim[s];
    if (n > K || n < 0) atomicCAS(err, 0, AOK_ERR_INVALID);
    if (k < n && k < K) {
        zeta[q] = a[off[s] + k];
        coef[q] = c[off[s] + k];
    } else {
        zeta[q] = FT(1);
        coef[q] = FT(0);
    }
}

// --------------------------------------------------------------------------
// Primitive-pair records.
// --------------------------------------------------------------------------
// w rb^al ra^be q^ga for the class's moment slots, in slot order, written as
// out[j] (converted to FT) as they are formed; returns the slot count.
template <typename FT>
__device__ __forceinline__ int fill_monos(FT* out, int la, int lb, double w, double ra, double rb, double q) {
    int j = 0;
    for (int al = 0; al <= la; ++al)
        for (int be = 0; be <= lb; ++be) {
            if (((la - al) + (lb - be)) & 1) continue;
            double v = w;
            for (int k = 0; k < al; ++k) v *= rb;
            for (int k = 0; k < be; ++k) v *= ra;
            for (int k = 0; k < (la + lb - al - be) / 2; ++k) v *= q;
            out[j++] = (FT)v;
        }
    return j;
}

__device__ __forceinline__ void fill_pp(float* r, int la, int lb, double ca, double cb, double aa, double ab,
                                        int rowlen) {
    const double p = aa + ab, ip = 1.0 / p;
    const double x = kPi * ip;
    const double log2e = 1.4426950408889634074;
    const double mu2 = ((aa * ab) * ip) * log2e;  // exponent in base 2
    const int nv = fill_monos(r, la, lb, ca * cb * (x * sqrt(x)), aa * ip, ab * ip, 0.5 * ip);
    r[nv] = (float)mu2;
    r[nv + 1] = (float)(mu2 - (double)r[nv]);
    r[nv + 2] = (float)rowlen;
    for (int j = 3 + nv; j < 4 * rec_words16_f32(la, lb); ++j) r[j] = 0.f;
}
__device__ __forceinline__ void fill_pp(double* r, int la, int lb, double ca, double cb, double aa, double ab,
                                        int rowlen) {
    const double p = aa + ab;
    const double x = kPi / p;
    const int nv = fill_monos(r + 2, la, lb, ca * cb * (x * sqrt(x)), aa / p, ab / p, 0.5 / p);
    r[0] = aa * ab / p;
    r[1] = (double)rowlen;
    for (int j = 2 + nv; j < 2 * rec_words16_f64(la, lb); ++j) r[j] = 0.0;
}
template <typename FT> __host__ __device__ constexpr int rec_words16(int la, int lb);
template <> __host__ __device__ constexpr int rec_words16<float>(int la, int lb) { return rec_words16_f32(la, lb); }
template <> __host__ __device__ constexpr int rec_words16<double>(int la, int lb) { return rec_words16_f64(la, lb); }

// --------------------------------------------------------------------------
// Execution order, records and stage images of one species pair.
//
// Primitive pairs: those with non-zero coefficients on both sides, na * nb
// per shell pair, in the reference's (ip, jp) order (ip-major); each record
// carries nb as its row length.
//
// Order: within each panel, heavier classes first (warps that run
// concurrently share the class's code in the instruction cache), and inside a
// class the items with more primitive pairs first (longest-processing-time
// order for the warps' dynamic queue); rank sort in shared memory, or the
// static order for bases of more than kOrderMax items.
//
// Stage images: the items, in that order, are cut greedily into chunks of at
// most stage16 16-byte words, each laid out as [ExecItem per item, padded to
// 16 bytes][the items' records]; the segments are the runs of items of one
// panel inside one chunk.  The cut is a binary search per chunk over the
// prefix sums of the record sizes.  The host sizes the stage to hold the
// largest item, so every chunk holds at least one.
//
// Grid (species pairs, parts): every CTA of a pair sorts and cuts (cheap,
// identical results); part 0 writes the segments; the parts share the record
// computation, one warp per item, lanes over the K x K primitive grid with a
// ballot compaction.  Dynamic shared memory: pack2c_smem(nitems) bytes.
// --------------------------------------------------------------------------
constexpr int kOrderMax = 2048;
// Per species pair, after the NZ*NZ stage images in the same allocation: the key of
// the last k_pack2c build (stage size, non-zero counts of the bra and ket species'
// shells; all ones until the first build), then per item of the execution order the
// item and the 16-byte word at which its records start.
constexpr int kPackKeyStride = 4 + 2 * kMaxShells;
static_assert(sizeof(Item) == sizeof(long long), "an item is loaded as one 8-byte word");
size_t pack2c_cache_bytes(size_t npairs, int nitems) {
    return npairs * (sizeof(int) * kPackKeyStride + (sizeof(Item) + sizeof(int)) * (size_t)nitems);
}

size_t pack2c_smem(int nitems) { return (size_t)28 * nitems + 16; }
int pack2c_parts(int nitems) { return std::min(16, std::max(1, (nitems + 15) / 16)); }

template <typename FT>
__global__ void __launch_bounds__(256) k_pack2c(float4* __restrict__ pk, Seg* __restrict__ segs,
                                                int* __restrict__ nseg, const Item* __restrict__ items,
                                                const FT* __restrict__ zeta, const FT* __restrict__ coef,
                                                Panels panels, const int* __restrict__ boff, int nitems, int ns,
                                                int K, int NZ, int N, int stage16, int pair16, int seg_stride,
                                                int* __restrict__ pkey, Item* __restrict__ citems,
                                                int* __restrict__ cdst) {
    extern __shared__ unsigned long long psm64[];
    unsigned long long* key = psm64;                               // nitems
    Item* sorted = reinterpret_cast<Item*>(psm64 + nitems);        // nitems; chunk = primitive pairs
    int* P = reinterpret_cast<int*>(psm64 + 2 * (size_t)nitems);   // nitems + 1: exclusive prefix, record words
    int* cst = P + nitems + 1;                                     // first item of chunk j (+ nitems)
    int* chd = cst + nitems + 1;                                   // header words before chunk j
    __shared__ int s_item0[kMaxPanels + 1], s_col0[kMaxPanels + 1], s_boff[kMaxShells + 1];
    __shared__ int s_nnz[2][kMaxShells];
    __shared__ int s_wsum[8], s_nch;
    const int pair = blockIdx.x, ga = pair / NZ, gb = pair % NZ;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = 8;
    const int npan = panels.n;
    pdl_wait();  // coef may come from the k_compile_coef launched just before
    if (tid <= npan) {
        s_item0[tid] = panels.item0[tid];
        s_col0[tid] = panels.col0[tid];
    }
    if (tid <= ns) s_boff[tid] = boff[tid];
    for (int i = tid; i < 2 * ns; i += blockDim.x) {
        const int sh = i % ns, g = i < ns ? ga : gb;
        int c = 0;
        for (int k = 0; k < K; ++k) c += coef[sh + ns * (k + K * g)] != FT(0);
        s_nnz[i / ns][sh] = c;
    }
    __syncthreads();
    // the primitive-pair records of item `it` at `out` (compacted non-zero pairs, (ip, jp) order)
    auto write_records = [&](const Item it, FT* out) {
        const int la = it.cls >> 2, lb = it.cls & 3;
        const int words = rec_words16<FT>(la, lb) * (16 / (int)sizeof(FT));
        const int nb = s_nnz[1][it.sb];
        int n = 0;
        for (int e0 = 0; e0 < K * K; e0 += 32) {
            const int e = e0 + lane;
            const int ip = e / K, jp = e % K;
            double ca = 0.0, cb = 0.0, aa = 0.0, ab = 0.0;
            if (e < K * K) {
                ca = (double)coef[it.sa + ns * (ip + K * ga)];
                cb = (double)coef[it.sb + ns * (jp + K * gb)];
                aa = (double)zeta[it.sa + ns * (ip + K * ga)];
                ab = (double)zeta[it.sb + ns * (jp + K * gb)];
            }
            const bool valid = (e < K * K) && ca != 0.0 && cb != 0.0;
            const unsigned m = __ballot_sync(0xffffffffu, valid);
            if (valid) fill_pp(out + (size_t)(n + __popc(m & ((1u << lane) - 1u))) * words, la, lb, ca, cb, aa, ab, nb);
            n += __popc(m);
        }
    };
    // Everything but the record values (order, chunks, headers, segments) follows from
    // the stage size and the non-zero counts of the two species' shells.  When they
    // equal the key of the last build for this pair, the headers and segments in place
    // stand and only the records are rewritten, at the offsets cached with the key.
    int* bkey = pkey + (size_t)pair * kPackKeyStride;
    {
        int same = tid != 0 || __ldcg(bkey) == stage16;
        for (int i = tid; i < 2 * ns; i += blockDim.x) same &= __ldcg(bkey + 1 + i) == s_nnz[i / ns][i % ns];
        if (__syncthreads_and(same)) {
            __threadfence();
            for (int i = blockIdx.y * NW + warp; i < nitems; i += gridDim.y * NW) {
                const long long w = __ldcg(reinterpret_cast<const long long*>(citems) + (size_t)pair * nitems + i);
                Item it;
                memcpy(&it, &w, sizeof(Item));
                const int d16 = __ldcg(cdst + (size_t)pair * nitems + i);
                write_records(it, reinterpret_cast<FT*>(pk + (size_t)pair * pair16 + d16));
            }
            return;
        }
    }
    auto panel_of = [&](int i) {
        int pn = 0;
        while (pn + 1 < npan && i >= s_item0[pn + 1]) ++pn;
        return pn;
    };
    for (int i = tid; i < nitems; i += blockDim.x) {
        Item it = items[i];
        const int n = s_nnz[0][it.sa] * s_nnz[1][it.sb];
        it.chunk = (int16_t)n;
        sorted[i] = it;
        const int la = it.cls >> 2, lb = it.cls & 3;
        key[i] = ((unsigned long long)panel_of(i) << 48) |
                 ((unsigned long long)(0xFFFF - md_terms(la, lb)) << 32) |
                 ((unsigned long long)(0xFFFF - n) << 16) | (unsigned long long)it.cls;
    }
    __syncthreads();
    if (nitems <= kOrderMax) {
        Item mine[kOrderMax / 256];
        int rank[kOrderMax / 256];
#pragma unroll
        for (int t = 0; t < kOrderMax / 256; ++t) {
            const int i = tid + 256 * t;
            rank[t] = -1;
            if (i < nitems) {
                const unsigned long long ki = key[i];
                int r = 0;
                for (int j = 0; j < nitems; ++j) {
                    const unsigned long long kj = key[j];
                    r += (kj < ki) || (kj == ki && j < i);
                }
                rank[t] = r;
                mine[t] = sorted[i];
            }
        }
        __syncthreads();
#pragma unroll
        for (int t = 0; t < kOrderMax / 256; ++t)
            if (rank[t] >= 0) sorted[rank[t]] = mine[t];
        __syncthreads();
    }
    // record words per item and their exclusive prefix (block scan)
    {
        const int per = (nitems + 255) / 256;
        const int i0 = min(nitems, tid * per), i1 = min(nitems, i0 + per);
        int sum = 0;
        for (int i = i0; i < i1; ++i) {
            const int w = (int)sorted[i].chunk * rec_words16<FT>(sorted[i].cls >> 2, sorted[i].cls & 3);
            P[i] = w;
            sum += w;
        }
        int incl = sum;
        for (int d = 1; d < 32; d <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += v;
        }
        if (lane == 31) s_wsum[warp] = incl;
        __syncthreads();
        int run = incl - sum;
        for (int w = 0; w < warp; ++w) run += s_wsum[w];
        for (int i = i0; i < i1; ++i) {
            const int w = P[i];
            P[i] = run;
            run += w;
        }
        if (tid == 255) P[nitems] = run;
    }
    __syncthreads();
    if (tid == 0) {
        int nch = 0, c0 = 0, h = 0;
        while (c0 < nitems) {
            cst[nch] = c0;
            chd[nch] = h;
            int lo = c0 + 1, hi = nitems;  // the largest c1 whose chunk [c0, c1) fits
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if ((mid - c0 + 1) / 2 + P[mid] - P[c0] <= stage16) lo = mid;
                else hi = mid - 1;
            }
            h += (lo - c0 + 1) / 2;
            c0 = lo;
            ++nch;
        }
        cst[nch] = nitems;
        chd[nch] = h;
        s_nch = nch;
        if (blockIdx.y == 0) {
            Seg* sg = segs + (size_t)pair * seg_stride;
            int nout = 0;
            for (int j = 0; j < nch; ++j) {
                const int a0 = cst[j], a1 = cst[j + 1];
                const int off = pair * pair16 + P[a0] + chd[j];
                const int n16 = (a1 - a0 + 1) / 2 + P[a1] - P[a0];
                for (int a = a0; a < a1;) {  // split the chunk at panel starts
                    const int pn = panel_of(a);
                    const int b = min(a1, s_item0[pn + 1]);
                    sg[nout++] = Seg{a, b, a0, off, n16, pn + (b == s_item0[pn + 1] ? kSegPanelEnd : 0)};
                    a = b;
                }
            }
            nseg[pair] = nout;
        }
    }
    __syncthreads();
    const int nch = s_nch;
    if (blockIdx.y == 0) {  // the cache for the next call: order and record offsets, then the key
        for (int i = tid; i < nitems; i += blockDim.x) {
            int lo = 0, hi = nch - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (cst[mid] <= i) lo = mid;
                else hi = mid - 1;
            }
            citems[(size_t)pair * nitems + i] = sorted[i];
            cdst[(size_t)pair * nitems + i] = chd[lo] + (cst[lo + 1] - cst[lo] + 1) / 2 + P[i];
        }
        __threadfence();
        __syncthreads();
        for (int i = tid; i < 2 * ns; i += blockDim.x) bkey[1 + i] = s_nnz[i / ns][i % ns];
        if (tid == 0) bkey[0] = stage16;
    }
    for (int i = blockIdx.y * NW + warp; i < nitems; i += gridDim.y * NW) {
        const Item it = sorted[i];
        int lo = 0, hi = nch - 1;  // chunk j with cst[j] <= i < cst[j + 1]
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (cst[mid] <= i) lo = mid;
            else hi = mid - 1;
        }
        const int a0 = cst[lo], a1 = cst[lo + 1];
        float4* cbase = pk + (size_t)pair * pair16 + P[a0] + chd[lo];
        const int r0 = (a1 - a0 + 1) / 2 + P[i] - P[a0];
        if (lane == 0) {
            const int pn = panel_of(i);
            ExecItem e;
            e.cls = it.cls;
            e.n = it.chunk;
            e.rec = (int16_t)r0;
            e.dst = (int16_t)((s_boff[it.sb] - s_col0[pn]) * N + s_boff[it.sa]);
            reinterpret_cast<ExecItem*>(cbase)[i - a0] = e;
        }
        write_records(it, reinterpret_cast<FT*>(cbase + r0));
    }
}

// --------------------------------------------------------------------------
// Species-pair bins: multi-block counting sort in two launches, no waiting.
//   k_bin_count    per block: histogram of its chunk of the batch
//   k_bin_scatter  per block: reads every block's histogram (at most 512
//                  blocks x NZ^2 keys), derives its own offsets, scatters its
//                  chunk stably (so the permutation is reproducible), and
//                  writes every nblk-th entry of the tile table (tiles of
//                  <= 32 elements of one key); block 0 also sets the tile
//                  count and resets the work-queue counter.
// k_bin_identity replaces both for single-species batches.
// --------------------------------------------------------------------------
constexpr int kBinThreads = 256;
constexpr int kBinMaxBlocks = kBinMaxBlocksHost;

// Key of element b: (a - 1) NZ + (c - 1) for a pair, ((a - 1) NZ + (c - 1)) NZ + (d - 1)
// for a triple (sidxC given); -1 past the end or for a species index outside 1..NZ.
__device__ __forceinline__ int pair_key(const int64_t* sidxA, const int64_t* sidxB, const int64_t* sidxC, int b,
                                        int B, int NZ, int* err) {
    if (b >= B) return -1;
    int64_t a = sidxA ? sidxA[b] : 1, c = sidxB ? sidxB[b] : 1, d = sidxC ? sidxC[b] : 1;
    if (a < 1 || a > NZ || c < 1 || c > NZ || d < 1 || d > NZ) {
        if (err) atomicCAS(err, 0, AOK_ERR_SPECIES);
        return -1;
    }
    const int k = (int)((a - 1) * NZ + (c - 1));
    return sidxC ? k * NZ + (int)(d - 1) : k;
}

// zeros for the three values of a left-out element (see BinBufs::zero3)
__device__ __forceinline__ void zero_three(void* zero3, int bytes, int b) {
    if (bytes == 8) {
        double* d = (double*)zero3 + 3 * (size_t)b;
        d[0] = d[1] = d[2] = 0.0;
    } else {
        float* f = (float*)zero3 + 3 * (size_t)b;
        f[0] = f[1] = f[2] = 0.0f;
    }
}

__global__ void __launch_bounds__(kBinThreads) k_bin_count(const int64_t* __restrict__ sidxA,
                                                            const int64_t* __restrict__ sidxB,
                                                            const int64_t* __restrict__ sidxC, int B, int NZ, int np,
                                                            int chunk, int* __restrict__ blockhist,
                                                            int* __restrict__ err, void* zero3, void* zero3b,
                                                            int zero3_bytes) {
    __shared__ int hist[kMaxPairs];
    for (int k = threadIdx.x; k < np; k += blockDim.x) hist[k] = 0;
    __syncthreads();
    const int c0 = blockIdx.x * chunk, c1 = min(B, c0 + chunk);
    for (int b = c0 + threadIdx.x; b < c1; b += blockDim.x) {
        const int key = pair_key(sidxA, sidxB, sidxC, b, c1, NZ, err);
        if (key >= 0) {
            atomicAdd(&hist[key], 1);
        } else {  // b < c1: a bad species index
            if (zero3) zero_three(zero3, zero3_bytes, b);
            if (zero3b) zero_three(zero3b, zero3_bytes, b);
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < np; k += blockDim.x) blockhist[(size_t)blockIdx.x * np + k] = hist[k];
}

constexpr int kBinWarps = kBinThreads / 32;
__global__ void __launch_bounds__(kBinThreads) k_bin_scatter(const int64_t* __restrict__ sidxA,
                                                              const int64_t* __restrict__ sidxB,
                                                              const int64_t* __restrict__ sidxC, int B, int NZ,
                                                              int np, int chunk, const int* __restrict__ blockhist,
                                                              int* __restrict__ perm, int4* __restrict__ tiles,
                                                              int* __restrict__ ntiles, int* __restrict__ tbase_out,
                                                              unsigned* __restrict__ counter, int* __restrict__ err) {
    __shared__ int wcount[kBinWarps][kMaxPairs];
    __shared__ int before[kMaxPairs], tot[kMaxPairs], base[kMaxPairs], tbase[kMaxPairs + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nblk = gridDim.x, me = blockIdx.x;
    // per key: elements in earlier blocks, and the total (integer sums, so the
    // order of the shared atomics does not matter)
    for (int k = threadIdx.x; k < np; k += blockDim.x) {
        before[k] = 0;
        tot[k] = 0;
    }
    __syncthreads();
    if (np <= (int)blockDim.x) {
        // thread t sums key t % np over blocks t / np, t / np + stride, ... in
        // registers, then one shared atomic per thread and key
        const int k = threadIdx.x % np, r0 = threadIdx.x / np, stride = blockDim.x / np;
        if (r0 < stride) {
            int tt = 0, b4 = 0;
            for (int blk = r0; blk < nblk; blk += stride) {
                const int v = blockhist[(size_t)blk * np + k];
                tt += v;
                if (blk < me) b4 += v;
            }
            if (tt) atomicAdd(&tot[k], tt);
            if (b4) atomicAdd(&before[k], b4);
        }
    } else {
        for (int i = threadIdx.x; i < nblk * np; i += blockDim.x) {
            const int k = i % np, blk = i / np;
            const int v = blockhist[i];
            if (v) {
                atomicAdd(&tot[k], v);
                if (blk < me) atomicAdd(&before[k], v);
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0, tacc = 0;
        for (int q = 0; q < np; ++q) {
            base[q] = acc;
            tbase[q] = tacc;
            acc += tot[q];
            tacc += (tot[q] + kTileB - 1) / kTileB;
        }
        tbase[np] = tacc;
        if (me == 0) {
            *ntiles = tacc;
            *counter = 0u;
        }
    }
    __syncthreads();
    if (me == 0)
        for (int q = threadIdx.x; q <= np; q += blockDim.x) tbase_out[q] = tbase[q];
    // tiles: this block writes tiles me, me + nblk, ...
    for (int t = me + (int)threadIdx.x * nblk; t < tbase[np]; t += blockDim.x * nblk) {
        int k = 0;
        while (tbase[k + 1] <= t) ++k;
        const int off = (t - tbase[k]) * kTileB;
        tiles[t] = make_int4(k, base[k] + off, min(kTileB, tot[k] - off), 0);
    }
    // stable scatter of this block's chunk: warp w owns a contiguous sub-range
    const int sub = (chunk + kBinWarps - 1) / kBinWarps;
    const int c0 = me * chunk + warp * sub;
    const int c1 = min(min(B, (me + 1) * chunk), c0 + sub);
    for (int k = lane; k < np; k += 32) wcount[warp][k] = 0;
    __syncwarp();
    for (int b0 = c0; b0 < c1; b0 += 32) {
        const int key = pair_key(sidxA, sidxB, sidxC, b0 + lane, c1, NZ, err);
        const unsigned peers = __match_any_sync(0xffffffffu, key);
        if (key >= 0 && lane == __ffs(peers) - 1) wcount[warp][key] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    for (int k = threadIdx.x; k < np; k += blockDim.x) {
        int acc = base[k] + before[k];
        for (int w = 0; w < kBinWarps; ++w) {
            const int v = wcount[w][k];
            wcount[w][k] = acc;
            acc += v;
        }
    }
    __syncthreads();
    for (int b0 = c0; b0 < c1; b0 += 32) {
        const int b = b0 + lane;
        const int key = pair_key(sidxA, sidxB, sidxC, b, c1, NZ, err);
        const unsigned peers = __match_any_sync(0xffffffffu, key);
        if (key >= 0) perm[wcount[warp][key] + __popc(peers & ((1u << lane) - 1u))] = b;
        __syncwarp();
        if (key >= 0 && lane == __ffs(peers) - 1) wcount[warp][key] += __popc(peers);
        __syncwarp();
    }
}

// Single species (or no indices): every element in key 0, in batch order.  The
// indices that are given are still range-checked (a bad one sets *err; the
// element stays in the bin, and the kernels that read the index themselves
// leave it out).
__global__ void k_bin_identity(int B, int np, int* __restrict__ perm, int4* __restrict__ tiles,
                               int* __restrict__ ntiles, int* __restrict__ tbase, unsigned* __restrict__ counter,
                               const int64_t* __restrict__ sidxA, const int64_t* __restrict__ sidxB,
                               const int64_t* __restrict__ sidxC, int NZ, int* __restrict__ err) {
    pdl_trigger();  // a programmatic successor may launch now (it waits for this grid's end)
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    const int nt = (B + kTileB - 1) / kTileB;
    if (b < B && (sidxA || sidxB || sidxC)) (void)pair_key(sidxA, sidxB, sidxC, b, B, NZ, err);
    if (b < B) perm[b] = b;
    if (b * kTileB < B) tiles[b] = make_int4(0, b * kTileB, min(kTileB, B - b * kTileB), 0);
    if (b <= np) tbase[b] = b == 0 ? 0 : nt;  // every element is in species pair 0
    if (b == 0) {
        *ntiles = nt;
        *counter = 0u;
    }
}

// --------------------------------------------------------------------------
// Host side: schedule and launchers.
// --------------------------------------------------------------------------

static size_t npairs_of(const aok_plan* p) { return (size_t)(p->NZ * p->NZ); }

static void free_schedule(aok_plan* p) {
    void** bufs[] = {(void**)&p->d_pk, (void**)&p->d_segs, (void**)&p->d_nseg, (void**)&p->d_items,
                     (void**)&p->d_blockhist};
    for (void** b : bufs)
        if (*b) {
            cudaFree(*b);
            *b = nullptr;
        }
    if (p->gexec) {  // kernel parameters of the captured chain change with the schedule
        cudaGraphExecDestroy(p->gexec);
        p->gexec = nullptr;
    }
}

int setup_overlap2c_schedule(aok_plan* p, int ctas, size_t stage_req) {
    const int ns = (int)p->ns, N = (int)p->N;
    const bool f64 = p->prec == AOK_PREC_F64;
    const size_t fsz = f64 ? sizeof(double) : sizeof(float);
    free_schedule(p);
    // Stage images (k_pack2c): a species pair's records fill at most pair16
    // 16-byte words (every primitive pair present, plus item headers and
    // padding); the stage holds one chunk and at least the largest item.
    const size_t K2 = (size_t)p->K * p->K;
    size_t pair16 = 2 * (size_t)ns * ns;
    for (int a = 0; a < ns; ++a)
        for (int b = 0; b < ns; ++b) {
            const int la = (int)p->ls[a], lb = (int)p->ls[b];
            pair16 += K2 * (size_t)(f64 ? rec_words16_f64(la, lb) : rec_words16_f32(la, lb));
        }
    const size_t one_item = 16 + K2 * (f64 ? kRecMaxBytesF64 : kRecMaxBytesF32);
    const size_t stage_pref = stage_req ? stage_req : (size_t)(f64 ? 48 : 24) * 1024;
    const size_t stage = (std::max(one_item, std::min(stage_pref, pair16 * 16)) + 15) / 16 * 16;
    if (stage > (size_t)200 * 1024)
        return set_error(AOK_ERR_UNSUPPORTED, "too many primitives per shell for the 2C stage");
    // FP32: two CTAs per SM, three for bases of <= 2 primitives per shell;
    // FP64: one, two for such bases.  The slab shares the CTA's shared memory
    // with the stage; a basis whose widest shell column would not fit falls back
    // to one CTA per SM.
    const bool few = p->K <= 2;
    p->fwd_ctas = ctas ? ctas : f64 ? (few ? 2 : 1) : (few ? 3 : 2);
    if (f64 ? (p->fwd_ctas < 1 || p->fwd_ctas > 2) : (p->fwd_ctas < 2 || p->fwd_ctas > 3))
        return set_error(AOK_ERR_INVALID, "2C forward: unsupported CTAs per SM");
    const size_t cap = p->fwd_ctas == 3 ? (size_t)72 * 1024 : p->fwd_ctas == 2 ? (size_t)112 * 1024 : (size_t)224 * 1024;
    size_t budget = p->fwd_ctas == 1 ? std::min((size_t)120 * 1024, (size_t)224 * 1024 - stage)
                                     : cap - std::min(stage, cap);
    {
        size_t widest = 0;
        for (int s = 0; s < ns; ++s) widest = std::max(widest, (size_t)ncart((int)p->ls[s]));
        const size_t need = ((size_t)N * widest + 1) * kTileB * fsz;
        if (budget < need) budget = (size_t)224 * 1024 - stage;
    }
    // panels: consecutive ket shells whose column range fits the slab budget
    std::vector<int> pcols{0};
    std::vector<int> pshell{0};
    int width = 0;
    auto stride_for = [&](int w) {
        size_t s = (size_t)N * w;
        if (s % 2 == 0) s += 1;  // odd stride: conflict-free lane-per-slab stores
        return s;
    };
    for (int s = 0; s < ns; ++s) {
        int nb = ncart((int)p->ls[s]);
        if (width > 0 && stride_for(width + nb) * kTileB * fsz > budget) {
            pcols.push_back(pcols.back() + width);
            pshell.push_back(s);
            width = 0;
        }
        width += nb;
    }
    pcols.push_back(pcols.back() + width);
    pshell.push_back(ns);
    const int npan = (int)pcols.size() - 1;
    if (npan > kMaxPanels) return set_error(AOK_ERR_UNSUPPORTED, "basis too large for the panel schedule");
    size_t maxw = 0;
    for (int i = 0; i < npan; ++i) maxw = std::max(maxw, (size_t)(pcols[i + 1] - pcols[i]));
    p->slab_stride = stride_for((int)maxw);
    p->smem_bytes = p->slab_stride * kTileB * fsz;
    p->stage_bytes = stage;
    if ((p->smem_bytes + 15) / 16 * 16 + stage > 227 * 1024)
        return set_error(AOK_ERR_UNSUPPORTED, "a single shell column exceeds the shared-memory slab");
    // items per panel, heaviest first
    std::vector<Item> items;
    p->panels.n = npan;
    for (int pn = 0; pn < npan; ++pn) {
        p->panels.col0[pn] = pcols[pn];
        p->panels.item0[pn] = (int)items.size();
        std::vector<std::pair<double, Item>> v;
        for (int sb = pshell[pn]; sb < pshell[pn + 1]; ++sb)
            for (int sa = 0; sa < ns; ++sa) {
                int la = (int)p->ls[sa], lb = (int)p->ls[sb];
                Item it{(int16_t)(la * 4 + lb), (int16_t)0, (int16_t)sa, (int16_t)sb};
                v.push_back({(double)md_terms(la, lb), it});
            }
        std::stable_sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
        for (auto& x : v) items.push_back(x.second);
    }
    p->panels.col0[npan] = pcols[npan];
    p->panels.item0[npan] = (int)items.size();
    p->nitems = (int)items.size();
    if (pair16 * npairs_of(p) >= ((size_t)1 << 31))
        return set_error(AOK_ERR_UNSUPPORTED, "basis too large for the 2C stage images");
    p->pair16 = (int)pair16;
    p->seg_stride = p->nitems + npan;
    const size_t npairs = (size_t)(p->NZ * p->NZ);
    cudaError_t e = cudaMalloc(&p->d_pk, 16 * pair16 * npairs + pack2c_cache_bytes(npairs, (int)items.size()));
    if (e != cudaSuccess) return cuda_status(e, "cudaMalloc(pk)");
    e = cudaMemset((char*)p->d_pk + 16 * pair16 * npairs, 0xFF, sizeof(int) * kPackKeyStride * npairs);
    if (e != cudaSuccess) return cuda_status(e, "cudaMemset(pack keys)");
    e = cudaMalloc(&p->d_segs, sizeof(Seg) * p->seg_stride * npairs);
    if (e != cudaSuccess) return cuda_status(e, "cudaMalloc(segs)");
    e = cudaMalloc(&p->d_nseg, sizeof(int) * npairs);
    if (e != cudaSuccess) return cuda_status(e, "cudaMalloc(nseg)");
    e = cudaMalloc(&p->d_items, sizeof(Item) * items.size());
    if (e != cudaSuccess) return cuda_status(e, "cudaMalloc(items)");
    if (pack2c_smem((int)items.size()) > 48 * 1024) {
        const int smem = (int)pack2c_smem((int)items.size());
        if ((e = cudaFuncSetAttribute(k_pack2c<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) !=
                cudaSuccess ||
            (e = cudaFuncSetAttribute(k_pack2c<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) !=
                cudaSuccess)
            return cuda_status(e, "cudaFuncSetAttribute(k_pack2c)");
    }
    p->max_bin_blocks = kBinMaxBlocks;
    e = cudaMalloc(&p->d_blockhist, sizeof(int) * p->max_bin_blocks * bin_keys_max(p->NZ));
    if (e != cudaSuccess) return cuda_status(e, "cudaMalloc(blockhist)");
    e = cudaMemcpy(p->d_items, items.data(), sizeof(Item) * items.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_status(e, "cudaMemcpy(items)");
    return AOK_OK;
}

int launch_gb_pad(aok_plan* p, const int64_t* nprim, const int64_t* prim_offset, const void* coef,
                  const void* alpha, cudaStream_t s) {
    int n = (int)(p->ns * p->K);
    int th = 128, bl = (n + th - 1) / th;
    if (p->prec == AOK_PREC_F64)
        k_gb_pad<double><<<bl, th, 0, s>>>((double*)p->d_gb_zeta, (double*)p->d_gb_coef, nprim, prim_offset,
                                           (const double*)coef, (const double*)alpha, (int)p->ns, (int)p->K,
                                           p->d_err);
    else
        k_gb_pad<float><<<bl, th, 0, s>>>((float*)p->d_gb_zeta, (float*)p->d_gb_coef, nprim, prim_offset,
                                          (const float*)coef, (const float*)alpha, (int)p->ns, (int)p->K,
                                          p->d_err);
    return cuda_status(cudaGetLastError(), "k_gb_pad");
}

int launch_prep2c(aok_plan* p, const void* zeta, const void* coef, cudaStream_t s, bool pdl) {
    const dim3 grid((unsigned)(p->NZ * p->NZ), (unsigned)pack2c_parts(p->nitems));
    const size_t smem = pack2c_smem(p->nitems);
    const int stage16 = (int)(p->stage_bytes / 16);
    const size_t npairs = npairs_of(p);
    int* pkey = (int*)((char*)p->d_pk + 16 * (size_t)p->pair16 * npairs);
    Item* citems = (Item*)(pkey + kPackKeyStride * npairs);
    int* cdst = (int*)(citems + npairs * (size_t)p->nitems);
    auto go = [&](auto kern, auto zt, auto cf) {
        if (pdl)
            return launch_pdl(kern, grid, dim3(256), smem, s, (float4*)p->d_pk, p->d_segs, p->d_nseg,
                              (const Item*)p->d_items, zt, cf, p->panels, (const int*)p->d_boff, p->nitems, (int)p->ns,
                              (int)p->K, (int)p->NZ, (int)p->N, stage16, p->pair16, p->seg_stride, pkey, citems, cdst);
        kern<<<grid, 256, smem, s>>>((float4*)p->d_pk, p->d_segs, p->d_nseg, p->d_items, zt, cf, p->panels, p->d_boff,
                                     p->nitems, (int)p->ns, (int)p->K, (int)p->NZ, (int)p->N, stage16, p->pair16,
                                     p->seg_stride, pkey, citems, cdst);
        return cudaGetLastError();
    };
    const cudaError_t e = p->prec == AOK_PREC_F64
                              ? go(k_pack2c<double>, (const double*)zeta, (const double*)coef)
                              : go(k_pack2c<float>, (const float*)zeta, (const float*)coef);
    return cuda_status(e, "k_pack2c");
}

int launch_bin3_into(const BinBufs& bb, const int64_t* sidxA, const int64_t* sidxB, const int64_t* sidxC,
                     int64_t B, int NZ, cudaStream_t s) {
    const int np = sidxC ? NZ * NZ * NZ : NZ * NZ;
    // blocks of >= 512 elements; at most 512 blocks, and few enough that each
    // block's read of all block histograms stays <= 16K entries
    const int maxb = std::min(kBinMaxBlocks, std::max(128, 16384 / np));
    const int chunk = (int)std::max<int64_t>(512, (B + maxb - 1) / maxb);
    const int nblk = (int)((B + chunk - 1) / chunk);
    if (NZ == 1 || (!sidxA && !sidxB && !sidxC)) {
        k_bin_identity<<<(int)((std::max<int64_t>(B, np + 1) + 255) / 256), 256, 0, s>>>(
            (int)B, np, bb.perm, bb.tiles, bb.ntiles, bb.tbase, bb.counter, sidxA, sidxB, sidxC, NZ, bb.err);
        return cuda_status(cudaGetLastError(), "k_bin_identity");
    }
    k_bin_count<<<nblk, kBinThreads, 0, s>>>(sidxA, sidxB, sidxC, (int)B, NZ, np, chunk, bb.blockhist, bb.err,
                                             bb.zero3, bb.zero3b, bb.zero3_bytes);
    AOK_TRY_ST(cuda_status(cudaGetLastError(), "k_bin_count"));
    k_bin_scatter<<<nblk, kBinThreads, 0, s>>>(sidxA, sidxB, sidxC, (int)B, NZ, np, chunk, bb.blockhist, bb.perm,
                                               bb.tiles, bb.ntiles, bb.tbase, bb.counter, bb.err);
    return cuda_status(cudaGetLastError(), "k_bin_scatter");
}

int launch_bin_into(const BinBufs& bb, const int64_t* sidxA, const int64_t* sidxB, int64_t B, int NZ,
                    cudaStream_t s) {
    return launch_bin3_into(bb, sidxA, sidxB, nullptr, B, NZ, s);
}

int launch_bin(aok_plan* p, const int64_t* sidxA, const int64_t* sidxB, int64_t B, cudaStream_t s) {
    ++p->gen;  // the plan's bins change
    const BinBufs bb{p->d_perm, p->d_tiles, p->d_ntiles, p->d_tbase, p->d_counter, p->d_blockhist, p->d_err};
    return launch_bin_into(bb, sidxA, sidxB, B, (int)p->NZ, s);
}

int launch_overlap2c(aok_plan* p, void* out, const void* posA, const void* posB, int64_t B, double lengthscale,
                     cudaStream_t s) {
    (void)B;
    if (p->prec == AOK_PREC_F64) return launch_ov2_f64(p, out, posA, posB, lengthscale, s);
    return launch_ov2_f32(p, out, posA, posB, lengthscale, s);
}

}  // namespace aok
