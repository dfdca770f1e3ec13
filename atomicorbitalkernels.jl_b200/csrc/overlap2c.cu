// overlap2c.cu -- batched 2-center Cartesian-Gaussian overlap, sm_100a.
//
// Replaces batch_S_orbital_kernel! (src/integrals/orbital/overlap_2c.jl:165-281)
// and batch_S_kernel! (src/integrals/kernels_2c.jl:110-224).
//
// Pipeline per call (all stream-ordered, no host synchronisation):
//   k_prep2c    one warp per (species pair, shell pair): the geometry-free
//               primitive-pair records (w, mu, a/p, b/p, 1/2p) in FP64,
//               compacted to the non-zero-coefficient pairs in the
//               reference's (ip, jp) order.
//   k_order2c   per species pair, the execution order of the work items.
//   k_bin_*     counting sort of the batch by species pair; tiles of 32
//               batch elements of one species pair; resets the work counter.
//   k_overlap2c persistent kernel (two CTAs per SM for FP32, one for FP64)
//               draining the tile queue.
//               Lane = batch element, so a warp runs one shell pair for 32
//               geometries with identical control flow.  Shell-pair classes
//               (la, lb) are compile-time specialised: the 1-D overlap
//               tables E^x_ij (Obara-Saika form of the MD t=0 coefficients)
//               and the block accumulators live in registers.  Blocks are
//               written into a shared-memory slab holding complete output
//               columns of 32 batch elements, which is then streamed out
//               with fully coalesced stores (each batch element's (N,N) slab
//               is contiguous in the reference layout).
//
// The reference's l >= 2 stride aliasing (block element lin = c1 + (2la+1)*c2,
// read back as blk[i + nbf_a*j], kernels_2c.jl:209-223) is reproduced at
// compile time: component pair (c1, c2) accumulates into element
// lin = c1 + (2la+1) c2 of the (nbf_a, nbf_b) block.
//
// FP32C precision: FP32 arithmetic; the Gaussian prefactor exp(-mu R^2) uses
// a double-float argument (mu and R^2 each carried as hi + lo), and the
// primitive-pair sum is accumulated per ip row in FP32 and folded into the
// running block sum with TwoSum whenever ip changes; the rounding errors are
// collected in the shared-memory slab and added at the end.
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
// w rb^al ra^be q^ga for the class's moment slots, in slot order.
__device__ __forceinline__ int fill_monos(double* wm, int la, int lb, double w, double ra, double rb, double q) {
    int j = 0;
    for (int al = 0; al <= la; ++al)
        for (int be = 0; be <= lb; ++be) {
            if (((la - al) + (lb - be)) & 1) continue;
            double v = w;
            for (int k = 0; k < al; ++k) v *= rb;
            for (int k = 0; k < be; ++k) v *= ra;
            for (int k = 0; k < (la + lb - al - be) / 2; ++k) v *= q;
            wm[j++] = v;
        }
    return j;
}

__device__ __forceinline__ void fill_pp(float* r, int la, int lb, double ca, double cb, double aa, double ab,
                                        int rowlen) {
    const double p = aa + ab, ip = 1.0 / p;
    const double x = kPi * ip;
    const double log2e = 1.4426950408889634074;
    const double mu2 = ((aa * ab) * ip) * log2e;  // exponent in base 2
    double wm[8];
    const int nv = fill_monos(wm, la, lb, ca * cb * (x * sqrt(x)), aa * ip, ab * ip, 0.5 * ip);
    r[0] = (float)mu2;
    r[1] = (float)(mu2 - (double)r[0]);
    r[2] = (float)rowlen;
    for (int j = 0; j < nv; ++j) r[3 + j] = (float)wm[j];
    for (int j = 3 + nv; j < 4 * rec_words16_f32(la, lb); ++j) r[j] = 0.f;
}
__device__ __forceinline__ void fill_pp(double* r, int la, int lb, double ca, double cb, double aa, double ab,
                                        int rowlen) {
    const double p = aa + ab;
    const double x = kPi / p;
    double wm[8];
    const int nv = fill_monos(wm, la, lb, ca * cb * (x * sqrt(x)), aa / p, ab / p, 0.5 / p);
    r[0] = aa * ab / p;
    r[1] = (double)rowlen;
    for (int j = 0; j < nv; ++j) r[2 + j] = wm[j];
    for (int j = 2 + nv; j < 2 * rec_words16_f64(la, lb); ++j) r[j] = 0.0;
}
template <typename FT> __host__ __device__ constexpr int rec_words16(int la, int lb);
template <> __host__ __device__ constexpr int rec_words16<float>(int la, int lb) { return rec_words16_f32(la, lb); }
template <> __host__ __device__ constexpr int rec_words16<double>(int la, int lb) { return rec_words16_f64(la, lb); }

// One warp per (species pair, shell pair); lanes sweep the K x K primitive
// grid in ip-major order and compact the non-zero-coefficient pairs with a
// ballot, preserving the reference's (ip, jp) summation order.  Records of a
// shell pair are contiguous at the class's record size, starting at the
// shell pair's region of K*K maximum-size records.
template <typename FT>
__global__ void k_prep2c(FT* __restrict__ pp, int* __restrict__ npp, const FT* __restrict__ zeta,
                         const FT* __restrict__ coef, const int* __restrict__ ls, int ns, int K, int NZ) {
    const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (q >= NZ * NZ * ns * ns) return;
    int sb = q % ns;
    int t = q / ns;
    int sa = t % ns;
    t /= ns;
    int gb = t % NZ, ga = t / NZ;
    const int la = ls[sa], lb = ls[sb];
    constexpr int kMaxWords = sizeof(FT) == 4 ? kRecMaxBytesF32 / 4 : kRecMaxBytesF64 / 8;
    const int words = rec_words16<FT>(la, lb) * (16 / (int)sizeof(FT));
    FT* out = pp + (size_t)q * K * K * kMaxWords;
    int n = 0;
    // every row (ip with a non-zero coefficient) holds the same jp set
    int nb = 0;
    for (int jp = 0; jp < K; ++jp) nb += coef[sb + ns * (jp + K * gb)] != FT(0);
    for (int e0 = 0; e0 < K * K; e0 += 32) {
        const int e = e0 + lane;
        const int ip = e / K, jp = e % K;
        double ca = 0.0, cb = 0.0, aa = 0.0, ab = 0.0;
        if (e < K * K) {
            ca = (double)coef[sa + ns * (ip + K * ga)];
            cb = (double)coef[sb + ns * (jp + K * gb)];
            aa = (double)zeta[sa + ns * (ip + K * ga)];
            ab = (double)zeta[sb + ns * (jp + K * gb)];
        }
        const bool valid = (e < K * K) && ca != 0.0 && cb != 0.0;
        const unsigned m = __ballot_sync(0xffffffffu, valid);
        if (valid) fill_pp(out + (size_t)(n + __popc(m & ((1u << lane) - 1u))) * words, la, lb, ca, cb, aa, ab, nb);
        n += __popc(m);
    }
    if (lane == 0) npp[q] = n;
}

// --------------------------------------------------------------------------
// Execution order of the work items of one species pair (each item carries its
// number of primitive pairs in `chunk`): within each panel,
// heavier classes first (warps that run concurrently share the class's code
// in the instruction cache), and inside a class the items with more primitive
// pairs first (longest-processing-time order for the warps' dynamic queue).
// One CTA per species pair, rank sort in shared memory.
// --------------------------------------------------------------------------
constexpr int kOrderMax = 2048;


__global__ void __launch_bounds__(256) k_order2c(Item* __restrict__ order, const Item* __restrict__ items,
                                                 const int* __restrict__ npp, Panels panels, int nitems, int ns) {
    __shared__ unsigned long long key[kOrderMax];
    const int pair = blockIdx.x;
    Item* out = order + (size_t)pair * nitems;
    if (nitems > kOrderMax) {  // very large bases: keep the static order
        for (int i = threadIdx.x; i < nitems; i += blockDim.x) {
            Item o = items[i];
            o.chunk = (int16_t)min(npp[((size_t)pair * ns + o.sa) * ns + o.sb], 32767);
            out[i] = o;
        }
        return;
    }
    for (int i = threadIdx.x; i < nitems; i += blockDim.x) {
        const Item it = items[i];
        int pn = 0;
        while (pn + 1 < panels.n && i >= panels.item0[pn + 1]) ++pn;
        // heavy classes first (terms of the geometry transform), grouped by class
        // so that the warps of a CTA mostly run the same code; then by primitive pairs
        const int la = it.cls >> 2, lb = it.cls & 3;
        const int n = npp[((size_t)pair * ns + it.sa) * ns + it.sb];
        const unsigned long long k = ((unsigned long long)pn << 48) |
                                     ((unsigned long long)(0xFFFF - md_terms(la, lb)) << 32) |
                                     ((unsigned long long)(0xFFFF - min(n, 0xFFFF)) << 16) |
                                     (unsigned long long)it.cls;
        key[i] = (k << 0);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nitems; i += blockDim.x) {
        const unsigned long long ki = key[i];
        int r = 0;
        for (int j = 0; j < nitems; ++j) {
            const unsigned long long kj = key[j];
            r += (kj < ki) || (kj == ki && j < i);
        }
        Item o = items[i];
        o.chunk = (int16_t)min(npp[((size_t)pair * ns + o.sa) * ns + o.sb], 32767);
        out[r] = o;
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

__device__ __forceinline__ int pair_key(const int64_t* sidxA, const int64_t* sidxB, int b, int B, int NZ, int* err) {
    if (b >= B) return -1;
    int64_t a = sidxA ? sidxA[b] : 1, c = sidxB ? sidxB[b] : 1;
    if (a < 1 || a > NZ || c < 1 || c > NZ) {
        if (err) atomicCAS(err, 0, AOK_ERR_SPECIES);
        return -1;
    }
    return (int)((a - 1) * NZ + (c - 1));
}

__global__ void __launch_bounds__(kBinThreads) k_bin_count(const int64_t* __restrict__ sidxA,
                                                            const int64_t* __restrict__ sidxB, int B, int NZ,
                                                            int chunk, int* __restrict__ blockhist,
                                                            int* __restrict__ err) {
    __shared__ int hist[kMaxPairs];
    const int np = NZ * NZ;
    for (int k = threadIdx.x; k < np; k += blockDim.x) hist[k] = 0;
    __syncthreads();
    const int c0 = blockIdx.x * chunk, c1 = min(B, c0 + chunk);
    for (int b = c0 + threadIdx.x; b < c1; b += blockDim.x) {
        const int key = pair_key(sidxA, sidxB, b, c1, NZ, err);
        if (key >= 0) atomicAdd(&hist[key], 1);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < np; k += blockDim.x) blockhist[(size_t)blockIdx.x * np + k] = hist[k];
}

constexpr int kBinWarps = kBinThreads / 32;
__global__ void __launch_bounds__(kBinThreads) k_bin_scatter(const int64_t* __restrict__ sidxA,
                                                              const int64_t* __restrict__ sidxB, int B, int NZ,
                                                              int chunk, const int* __restrict__ blockhist,
                                                              int* __restrict__ perm, int4* __restrict__ tiles,
                                                              int* __restrict__ ntiles, int* __restrict__ tbase_out,
                                                              unsigned* __restrict__ counter, int* __restrict__ err) {
    __shared__ int wcount[kBinWarps][kMaxPairs];
    __shared__ int before[kMaxPairs], tot[kMaxPairs], base[kMaxPairs], tbase[kMaxPairs + 1];
    const int np = NZ * NZ, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
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
        const int key = pair_key(sidxA, sidxB, b0 + lane, c1, NZ, err);
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
        const int key = pair_key(sidxA, sidxB, b, c1, NZ, err);
        const unsigned peers = __match_any_sync(0xffffffffu, key);
        if (key >= 0) perm[wcount[warp][key] + __popc(peers & ((1u << lane) - 1u))] = b;
        __syncwarp();
        if (key >= 0 && lane == __ffs(peers) - 1) wcount[warp][key] += __popc(peers);
        __syncwarp();
    }
}

__global__ void k_bin_identity(int B, int np, int* __restrict__ perm, int4* __restrict__ tiles,
                               int* __restrict__ ntiles, int* __restrict__ tbase, unsigned* __restrict__ counter) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    const int nt = (B + kTileB - 1) / kTileB;
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

int setup_overlap2c_schedule(aok_plan* p) {
    const int ns = (int)p->ns, N = (int)p->N;
    const size_t fsz = p->prec == AOK_PREC_F64 ? sizeof(double) : sizeof(float);
    // FP32: two CTAs per SM; FP64: one.  The slab shares the CTA's shared memory
    // with the per-warp record buffers (K*K maximum-size records per warp); a
    // basis whose widest shell column would not fit falls back to one CTA per SM.
    const size_t recbuf = (size_t)8 * p->K * p->K * (p->prec == AOK_PREC_F64 ? kRecMaxBytesF64 : kRecMaxBytesF32);
    size_t budget = p->prec == AOK_PREC_F64 ? (size_t)120 * 1024
                                            : (size_t)112 * 1024 - std::min(recbuf, (size_t)112 * 1024);
    {
        size_t widest = 0;
        for (int s = 0; s < ns; ++s) widest = std::max(widest, (size_t)ncart((int)p->ls[s]));
        const size_t need = ((size_t)N * widest + 1) * kTileB * fsz;
        if (budget < need) budget = (size_t)224 * 1024 - std::min(recbuf, (size_t)224 * 1024);
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
    if (p->smem_bytes > 227 * 1024)
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
    cudaError_t e = cudaMalloc(&p->d_items, sizeof(Item) * items.size());
    if (e != cudaSuccess) return cuda_status(e, "cudaMalloc(items)");
    e = cudaMalloc(&p->d_order, sizeof(Item) * items.size() * p->NZ * p->NZ);
    if (e != cudaSuccess) return cuda_status(e, "cudaMalloc(order)");
    p->max_bin_blocks = kBinMaxBlocks;
    e = cudaMalloc(&p->d_blockhist, sizeof(int) * p->max_bin_blocks * p->NZ * p->NZ);
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

int launch_prep2c(aok_plan* p, const void* zeta, const void* coef, cudaStream_t s) {
    int n = (int)(p->NZ * p->NZ * p->ns * p->ns);
    int th = 128, bl = (n * 32 + th - 1) / th;
    if (p->prec == AOK_PREC_F64)
        k_prep2c<double><<<bl, th, 0, s>>>((double*)p->d_pp, p->d_npp, (const double*)zeta, (const double*)coef,
                                           p->d_ls, (int)p->ns, (int)p->K, (int)p->NZ);
    else
        k_prep2c<float><<<bl, th, 0, s>>>((float*)p->d_pp, p->d_npp, (const float*)zeta, (const float*)coef,
                                          p->d_ls, (int)p->ns, (int)p->K, (int)p->NZ);
    AOK_TRY_ST(cuda_status(cudaGetLastError(), "k_prep2c"));
    k_order2c<<<(int)(p->NZ * p->NZ), 256, 0, s>>>(p->d_order, p->d_items, p->d_npp, p->panels, p->nitems,
                                                  (int)p->ns);
    return cuda_status(cudaGetLastError(), "k_order2c");
}

int launch_bin_into(const BinBufs& bb, const int64_t* sidxA, const int64_t* sidxB, int64_t B, int NZ,
                    cudaStream_t s) {
    // blocks of >= 512 elements; at most 512 blocks, and few enough that each
    // block's read of all block histograms stays <= 16K entries
    const int maxb = std::min(kBinMaxBlocks, std::max(128, 16384 / (NZ * NZ)));
    const int chunk = (int)std::max<int64_t>(512, (B + maxb - 1) / maxb);
    const int nblk = (int)((B + chunk - 1) / chunk);
    if (NZ == 1 || (!sidxA && !sidxB)) {
        const int np = NZ * NZ;
        k_bin_identity<<<(int)((std::max<int64_t>(B, np + 1) + 255) / 256), 256, 0, s>>>(
            (int)B, np, bb.perm, bb.tiles, bb.ntiles, bb.tbase, bb.counter);
        return cuda_status(cudaGetLastError(), "k_bin_identity");
    }
    k_bin_count<<<nblk, kBinThreads, 0, s>>>(sidxA, sidxB, (int)B, NZ, chunk, bb.blockhist, bb.err);
    AOK_TRY_ST(cuda_status(cudaGetLastError(), "k_bin_count"));
    k_bin_scatter<<<nblk, kBinThreads, 0, s>>>(sidxA, sidxB, (int)B, NZ, chunk, bb.blockhist, bb.perm, bb.tiles,
                                               bb.ntiles, bb.tbase, bb.counter, bb.err);
    return cuda_status(cudaGetLastError(), "k_bin_scatter");
}

int launch_bin(aok_plan* p, const int64_t* sidxA, const int64_t* sidxB, int64_t B, cudaStream_t s) {
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
