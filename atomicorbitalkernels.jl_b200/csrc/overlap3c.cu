// overlap3c.cu -- 3-center overlap host side: the compact primitive lists, the
// item list, and the aok_overlap3c_gb / aok_overlap3c entry points.  The kernel is in
// overlap3c_kernel.cuh (one instantiation per precision: overlap3c_f32.cu,
// overlap3c_f64.cu).
#include <algorithm>
#include <cstring>
#include <vector>

#include "overlap3c_kernel.cuh"

namespace aok {

// The primitives of every (species g, shell s): the non-zero-coefficient slots of
// the padded (ns,K,NZ) tables, compacted in slot order into pz/pc at (g ns + s) K,
// and their number pn[g ns + s] (also into spn, shared).  One warp per (shell,
// species), lanes over the slots.
template <typename FT>
__device__ __forceinline__ void prim3c_padded(FT* __restrict__ pz, FT* __restrict__ pc, int* __restrict__ pn,
                                              int* spn, const FT* __restrict__ zeta, const FT* __restrict__ coef,
                                              int ns, int K, int NZ) {
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int t = threadIdx.x >> 5; t < ns * NZ; t += nw) {
        const int sh = t % ns, g = t / ns;
        int n = 0;
        for (int k0 = 0; k0 < K; k0 += 32) {
            const int k = k0 + lane;
            const size_t o = (size_t)sh + (size_t)ns * (k + (size_t)K * g);
            const FT c = k < K ? coef[o] : FT(0);
            const unsigned m = __ballot_sync(0xffffffffu, c != FT(0));
            if (c != FT(0)) {
                const int at = n + __popc(m & ((1u << lane) - 1u));
                pz[(size_t)t * K + at] = zeta[o];
                pc[(size_t)t * K + at] = c;
            }
            n += __popc(m);
        }
        if (lane == 0) {
            pn[t] = n;
            spn[t] = n;
        }
    }
}

// The same lists from CompiledBasis-style flat tables (one species): shell s has
// nprim[s] primitives at prim_offset[s] (0-based); counts outside 0..K are flagged
// (AOK_ERR_INVALID in err) and read as 0.
template <typename FT>
__device__ __forceinline__ void prim3c_flat(FT* __restrict__ pz, FT* __restrict__ pc, int* __restrict__ pn, int* spn,
                                            const int64_t* __restrict__ nprim, const int64_t* __restrict__ off,
                                            const FT* __restrict__ coef, const FT* __restrict__ alpha, int ns, int K,
                                            int* __restrict__ err) {
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int t = threadIdx.x >> 5; t < ns; t += nw) {
        int64_t mm = nprim[t];
        if (mm < 0 || mm > K) {
            if (lane == 0) atomicCAS(err, 0, AOK_ERR_INVALID);
            mm = 0;
        }
        const int64_t o0 = off[t];
        int n = 0;
        for (int k0 = 0; k0 < (int)mm; k0 += 32) {
            const int k = k0 + lane;
            const FT c = k < (int)mm ? coef[o0 + k] : FT(0);
            const unsigned m = __ballot_sync(0xffffffffu, c != FT(0));
            if (c != FT(0)) {
                const int at = n + __popc(m & ((1u << lane) - 1u));
                pz[(size_t)t * K + at] = alpha[o0 + k];
                pc[(size_t)t * K + at] = c;
            }
            n += __popc(m);
        }
        if (lane == 0) {
            pn[t] = n;
            spn[t] = n;
        }
    }
}

// Per call, one CTA: the item order of the kernel's unit queue and its cut into
// segments.  Items that run the same code (one shell-triple class and page
// chunk; all f-shell classes share one routine) are kept together, so that the
// warps in flight at any time run few distinct routines and the instruction
// cache holds them; the groups are ordered by their heaviest item, heaviest
// first, and the items inside a group heaviest first, so the queue ends with
// cheap work.  Cost = primitive triples (the largest count over the species per
// shell) x (the exponential + E tables + the chunk's products) + a fixed part per
// item and per output; the f-shell classes (run-time loops, FP64 tables) count
// four times.
// Rank sort in shared memory.  The ordered list is then cut into segments of
// about total / G cost, G = target_units / tiles (a warp takes a whole segment
// of one tile per unit); an item that costs more than that is a segment alone.
// More than kOrder3Max items keep the static order, one item per segment.
// segs: the nseg + 1 segment bounds, then nseg at [n + 1] and H at [n + 2].
constexpr int kOrder3Max = 2048;
constexpr int kOrder3Threads = 256;
constexpr int kOrder3Per = kOrder3Max / kOrder3Threads;
constexpr int kCodes3 = 27 * 8 + 1;  // (class, chunk) codes of the specialised classes, + one for the f shells

__device__ __forceinline__ int code3(const Item3& it) {
    return it.cls >= kClsF3 ? kCodes3 - 1 : it.cls * 8 + it.chunk;
}

// Inclusive scan of one value per thread over the kOrder3Threads threads.
__device__ __forceinline__ long long block_scan3(long long v, long long* wtot) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    if (lane == 31) wtot[w] = v;
    __syncthreads();
    if (w == 0) {
        long long t = lane < kOrder3Threads / 32 ? wtot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long u = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += u;
        }
        if (lane < kOrder3Threads / 32) wtot[lane] = t;
    }
    __syncthreads();
    if (w > 0) v += wtot[w - 1];
    __syncthreads();
    return v;
}

__device__ __forceinline__ void order3c_body(Item3* __restrict__ order, int* __restrict__ segs,
                                             const Item3* __restrict__ items, const int* pn, int ntiles, int n,
                                             int ns, int NZ, int target_units) {
    __shared__ unsigned long long ikey[kOrder3Max], gkey[kOrder3Max];
    __shared__ int cst[kOrder3Max];
    __shared__ int gmax[kCodes3];
    __shared__ long long wtot[kOrder3Threads / 32];
    if (n > kOrder3Max) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            order[i] = items[i];
            segs[i] = i;
        }
        if (threadIdx.x == 0) {
            segs[n] = n;
            segs[n + 1] = n;
            segs[n + 2] = 0;
        }
        return;
    }
    for (int c = threadIdx.x; c < kCodes3; c += blockDim.x) gmax[c] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const Item3 it = items[i];
        const bool f = it.cls >= kClsF3;
        const int c = f ? it.cls - kClsF3 : it.cls;
        const int la = f ? c >> 4 : c / 9, lb = f ? (c >> 2) & 3 : (c / 3) % 3, lc = f ? c & 3 : c % 3;
        const int ppc = pages_per_chunk3(la, lb);
        const int pages = min(ppc, ncart(lc) - it.chunk * ppc);
        const long long per = 40 + 12LL * (la + 1) * (lb + 1) * (lc + 1) + 2LL * ncart(la) * ncart(lb) * pages;
        int na = 0, nb = 0, nc = 0;  // primitive counts, the largest over the species
        for (int g = 0; g < NZ; ++g) {
            na = max(na, pn[g * ns + it.sa]);
            nb = max(nb, pn[g * ns + it.sb]);
            nc = max(nc, pn[g * ns + it.sc]);
        }
        long long cost = (long long)na * nb * nc * per * (f ? 4 : 1) + 100 + 8LL * ncart(la) * ncart(lb) * pages;
        cost = min(cost, (long long)0x7FFFFFFF);
        cst[i] = (int)cost;
        // ascending = heaviest first; equal costs by routine, then by position
        ikey[i] = ((unsigned long long)(0x7FFFFFFF - cost) << 32) | ((unsigned)code3(it) << 12) | (unsigned)i;
        atomicMax(&gmax[code3(it)], (int)cost);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int ci = code3(items[i]);
        gkey[i] = ((unsigned long long)(0x7FFFFFFF - gmax[ci]) << 32) | (unsigned)ci;
    }
    __syncthreads();
    int rank[kOrder3Per], rcost[kOrder3Per], rcls[kOrder3Per];
#pragma unroll
    for (int k = 0; k < kOrder3Per; ++k) {
        const int i = threadIdx.x + k * kOrder3Threads;
        rank[k] = -1;
        if (i >= n) continue;
        const unsigned long long gi = gkey[i], ki = ikey[i];
        int r = 0;
        for (int j = 0; j < n; ++j) {
            const unsigned long long gj = gkey[j];
            r += gj < gi || (gj == gi && ikey[j] < ki);
        }
        const Item3 it = items[i];
        order[r] = it;
        rank[k] = r;
        rcost[k] = cst[i];
        rcls[k] = it.cls;
    }
    __syncthreads();
    // the costs and classes in queue order (cst and gkey are free again)
    int* qcls = reinterpret_cast<int*>(gkey);
#pragma unroll
    for (int k = 0; k < kOrder3Per; ++k)
        if (rank[k] >= 0) {
            cst[rank[k]] = rcost[k];
            qcls[rank[k]] = rcls[k];
        }
    __syncthreads();
    // exclusive cost prefix of this thread's kOrder3Per consecutive positions
    const int r0 = threadIdx.x * kOrder3Per;
    long long tsum = 0;
#pragma unroll
    for (int k = 0; k < kOrder3Per; ++k)
        if (r0 + k < n) tsum += cst[r0 + k];
    const long long incl = block_scan3(tsum, wtot);
    __shared__ long long total_s;
    if (threadIdx.x == kOrder3Threads - 1) total_s = incl;
    __syncthreads();
    const long long total = total_s;
    const long long G = max(1LL, min((long long)n, (long long)target_units / max(ntiles, 1)));
    const long long C = max(1LL, (total + G - 1) / G);
    // a segment starts at r when a multiple of C lies in (prefix(r - 1), prefix(r)], or next to an item of cost >= C
    long long P = incl - tsum;
    unsigned flags = 0u;
    int cnt = 0;
#pragma unroll
    for (int k = 0; k < kOrder3Per; ++k) {
        const int r = r0 + k;
        if (r >= n) break;
        bool start = r == 0;
        if (!start) {
            const long long pc = cst[r - 1];
            start = (P / C) != ((P - pc) / C) || pc >= C || cst[r] >= C;
        }
        if (start) {
            flags |= 1u << k;
            ++cnt;
        }
        P += cst[r];
    }
    const long long pos_incl = block_scan3(cnt, wtot);
    int pos = (int)(pos_incl - cnt);
#pragma unroll
    for (int k = 0; k < kOrder3Per; ++k)
        if (flags & (1u << k)) segs[pos++] = r0 + k;
    if (threadIdx.x == kOrder3Threads - 1) {
        segs[pos_incl] = n;
        segs[n + 1] = (int)pos_incl;
    }
    // H: the leading items of cost >= 2C with blocks of <= kSplitM3 elements (each a
    // segment alone), whose records the CTA's warps share for one tile per unit
    if (threadIdx.x == 0) {
        int h = 0;
        while (h < n && cst[h] >= 2 * C) {
            const int cls = qcls[h];
            if (cls >= kClsF3) break;
            const int la = cls / 9, lb = (cls / 3) % 3, lc = cls % 3;
            if (ncart(la) * ncart(lb) * ncart(lc) > kSplitM3) break;
            ++h;
        }
        segs[n + 2] = h;
    }
}

// One CTA per call ahead of the kernel: the compact primitive lists (from the padded
// tables, or from flat GaussianBasis-style tables when nprim is given), then the
// queue order and its segments.  It needs no binning result (the segment count uses
// the tile count of the batch, ntiles = ceil(B / 32)), so on the species-aware path it
// runs on the plan's side stream while the batch is binned; on the single-species path
// it follows the one-launch identity binning programmatically on the caller's stream
// and waits for the bins only before it ends.
// The order and the segments are a function of (n, ntiles, target_units) and the
// primitive counts alone, and key[] holds those of the last build: when they match
// (the usual case, a fixed basis over many batches) the sort and the cut are skipped
// and the buffers from that build stand.  A miss rebuilds them and then the key.
template <typename FT>
__global__ void __launch_bounds__(kOrder3Threads) k_prep3c(FT* __restrict__ pz, FT* __restrict__ pc,
                                                           int* __restrict__ pn, const FT* __restrict__ zeta,
                                                           const FT* __restrict__ coef, const int64_t* __restrict__ nprim,
                                                           const int64_t* __restrict__ off, int* __restrict__ err,
                                                           Item3* __restrict__ order, int* __restrict__ segs,
                                                           int* __restrict__ key, const Item3* __restrict__ items,
                                                           int ntiles, int n, int ns, int K, int NZ, int target_units) {
    __shared__ int spn[kMaxShells * 6];
    pdl_trigger();  // the kernel may launch now; it waits for this grid's end
    if (nprim)
        prim3c_flat<FT>(pz, pc, pn, spn, nprim, off, coef, zeta, ns, K, err);
    else
        prim3c_padded<FT>(pz, pc, pn, spn, zeta, coef, ns, K, NZ);
    __syncthreads();
    const int nc = nprim ? ns : ns * NZ;
    int same = threadIdx.x != 0 || (key[0] == n && key[1] == ntiles && key[2] == target_units && key[3] == nc);
    for (int t = threadIdx.x; t < nc; t += blockDim.x) same &= key[4 + t] == spn[t];
    if (__syncthreads_and(same)) {
        pdl_wait();  // launched after the bins: they are complete once this grid is
        return;
    }
    order3c_body(order, segs, items, spn, ntiles, n, ns, NZ, target_units);
    for (int t = threadIdx.x; t < nc; t += blockDim.x) key[4 + t] = spn[t];
    if (threadIdx.x == 0) {
        key[0] = n;
        key[1] = ntiles;
        key[2] = target_units;
        key[3] = nc;
    }
    pdl_wait();
}

int setup_overlap3c_schedule(aok_plan* p) {
    if (p->d_items3) return AOK_OK;
    if (p->NZ * p->NZ * p->NZ > kMaxPairs)
        return set_error(AOK_ERR_UNSUPPORTED, "3C overlap: more than 6 species (NZ^3 > 256 species triples)");
    if (p->Lmax > kMaxL3) return set_error(AOK_ERR_UNSUPPORTED, "3C overlap: shells above l = 3");
    const int ns = (int)p->ns;
    // every (shell triple, page chunk), statically ordered by class cost
    std::vector<std::pair<int, Item3>> v;
    for (int sc = 0; sc < ns; ++sc)
        for (int sa = 0; sa < ns; ++sa)
            for (int sb = 0; sb < ns; ++sb) {
                const int la = (int)p->ls[sa], lb = (int)p->ls[sb], lc = (int)p->ls[sc];
                const int ppc = pages_per_chunk3(la, lb), nch = nchunks3(la, lb, lc);
                for (int c = 0; c < nch; ++c) {
                    const int pages = std::min(ppc, ncart(lc) - c * ppc);
                    const int cost = (la + 1) * (lb + 1) * (lc + 1) * 12 + 2 * ncart(la) * ncart(lb) * pages;
                    const bool f = std::max(la, std::max(lb, lc)) > kMaxL3Spec;
                    const int cls = f ? kClsF3 + la * 16 + lb * 4 + lc : la * 9 + lb * 3 + lc;
                    v.push_back({f ? 4 * cost : cost,
                                 Item3{(int16_t)cls, (int16_t)c, (int16_t)sa, (int16_t)sb, (int16_t)sc, 0}});
                }
            }
    std::stable_sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    std::vector<Item3> items;
    for (auto& x : v) items.push_back(x.second);
    p->nitems3 = (int)items.size();
    const size_t fsz = p->prec == AOK_PREC_F64 ? sizeof(double) : sizeof(float);
    cudaError_t e;
    if ((e = cudaMalloc(&p->d_items3, sizeof(Item3) * items.size())) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(items3)");
    if ((e = cudaMalloc(&p->d_order3, sizeof(Item3) * items.size())) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(order3)");
    if ((e = cudaMalloc(&p->d_segs3, sizeof(int) * (items.size() + 3))) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(segs3)");
    if ((e = cudaMemcpy(p->d_items3, items.data(), sizeof(Item3) * items.size(), cudaMemcpyHostToDevice)) !=
        cudaSuccess)
        return cuda_status(e, "cudaMemcpy(items3)");
    // compact primitive lists: zeta then coef, each ns*K*NZ, and the ns*NZ lengths
    if ((e = cudaMalloc(&p->d_pp3, 2 * fsz * (size_t)(ns * p->K * p->NZ))) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(prim3)");
    if ((e = cudaMalloc(&p->d_npp3, sizeof(int) * (size_t)(ns * p->NZ))) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(nprim3)");
    // the schedule key of k_prep3c: all ones (n = -1) matches no call, so the first builds
    const size_t kbytes = sizeof(int) * (size_t)(4 + ns * p->NZ);
    if ((e = cudaMalloc(&p->d_key3, kbytes)) != cudaSuccess) return cuda_status(e, "cudaMalloc(key3)");
    if ((e = cudaMemset(p->d_key3, 0xFF, kbytes)) != cudaSuccess) return cuda_status(e, "cudaMemset(key3)");
    return AOK_OK;
}

// The kernel's unit counter (32 bits, each warp claims one past the end) must not
// wrap: at most nitems x (B / 32 + one partial tile per key) units (a segment holds
// at least one item).
static int check_units3(const aok_plan* p, int64_t B, const char* who) {
    if ((int64_t)p->nitems3 * ((B + 31) / 32 + bin_keys_max(p->NZ) + 1) >= ((int64_t)1 << 31))
        return set_error(AOK_ERR_LENGTH, std::string(who) + ": too many (shell triple, tile) units; split the batch");
    return AOK_OK;
}

// The 3C prep for B elements on stream `side` (see k_prep3c): the compact primitive
// lists of the padded (zeta, coef) tables, or of the flat tables when nprim is given
// (zeta = alpha), and the per-call item order and segments.  pdl: launched with
// programmatic serialisation right after the binning on the same stream.
static int launch_prep3c(aok_plan* p, const void* zeta, const void* coef, const int64_t* nprim,
                         const int64_t* prim_offset, int64_t B, cudaStream_t side, bool pdl) {
    const size_t nt = (size_t)(p->ns * p->K * p->NZ);
    // FP32: about eight (segment, tile) pairs per resident warp (three CTAs of four warps
    // per SM); FP64: about one item per segment
    const int target_units = p->prec == AOK_PREC_F64 ? (1 << 30) : p->num_sms * 3 * (kThreads3 / 32) * 8;
    const int ntiles = (int)std::min<int64_t>((B + 31) / 32, 1 << 30);
    auto go = [&](auto kern, auto pz, auto zt, auto cf) {
        if (pdl)
            return launch_pdl(kern, dim3(1), dim3(kOrder3Threads), 0, side, pz, pz + nt, p->d_npp3, zt, cf, nprim,
                              prim_offset, p->d_err, (Item3*)p->d_order3, p->d_segs3, p->d_key3,
                              (const Item3*)p->d_items3, ntiles, p->nitems3, (int)p->ns, (int)p->K, (int)p->NZ,
                              target_units);
        kern<<<1, kOrder3Threads, 0, side>>>(pz, pz + nt, p->d_npp3, zt, cf, nprim, prim_offset, p->d_err,
                                             (Item3*)p->d_order3, p->d_segs3, p->d_key3, (const Item3*)p->d_items3,
                                             ntiles, p->nitems3, (int)p->ns, (int)p->K, (int)p->NZ, target_units);
        return cudaGetLastError();
    };
    const cudaError_t e = p->prec == AOK_PREC_F64
                              ? go(k_prep3c<double>, (double*)p->d_pp3, (const double*)zeta, (const double*)coef)
                              : go(k_prep3c<float>, (float*)p->d_pp3, (const float*)zeta, (const float*)coef);
    return cuda_status(e, "k_prep3c");
}

// The 3C overlap: the prep on the plan's side stream while `bin` bins the batch on s,
// then the kernel over the plan's bins once both are done; with `chain` (a one-launch
// binning) all three on s, the prep and the kernel launched programmatically.
template <typename Bin>
static int launch_overlap3c(aok_plan* p, void* out, const void* zeta, const void* coef, const int64_t* nprim,
                            const int64_t* prim_offset, const void* posA, const void* posB, const void* posC,
                            int64_t B, double lengthscale, cudaStream_t s, Bin bin, bool chain) {
    int st;
    if (chain) {
        // one stream: the (one-launch) binning, then the prep and the kernel, each launched
        // programmatically so that its launch overlaps its predecessor
        if ((st = bin()) != AOK_OK) return st;
        if ((st = launch_prep3c(p, zeta, coef, nprim, prim_offset, B, s, true)) != AOK_OK) return st;
    } else {
        if ((st = cuda_status(cudaEventRecord(p->ev_fork, s), "cudaEventRecord")) != AOK_OK) return st;
        if ((st = cuda_status(cudaStreamWaitEvent(p->side, p->ev_fork, 0), "cudaStreamWaitEvent")) != AOK_OK)
            return st;
        if ((st = launch_prep3c(p, zeta, coef, nprim, prim_offset, B, p->side, false)) != AOK_OK) return st;
        if ((st = cuda_status(cudaEventRecord(p->ev_join, p->side), "cudaEventRecord")) != AOK_OK) return st;
        if ((st = bin()) != AOK_OK) return st;
        if ((st = cuda_status(cudaStreamWaitEvent(s, p->ev_join, 0), "cudaStreamWaitEvent")) != AOK_OK) return st;
    }
    if (p->prec == AOK_PREC_F64) return launch_ov3_f64(p, out, posA, posB, posC, lengthscale, s, chain);
    return launch_ov3_f32(p, out, posA, posB, posC, lengthscale, s, chain);
}

}  // namespace aok

using namespace aok;

extern "C" int aok_overlap3c_gb(aok_plan* p, void* out, const int64_t* nprim, const int64_t* prim_offset,
                                const void* coef, const void* alpha, const void* posA, const void* posB,
                                const void* posC, int64_t B, void* stream) {
    if (!p) return set_error(AOK_ERR_INVALID, "aok_overlap3c_gb: null plan");
    if (p->NZ != 1) return set_error(AOK_ERR_INVALID, "aok_overlap3c_gb: plan must have NZ = 1");
    if (B < 0) return set_error(AOK_ERR_INVALID, "aok_overlap3c_gb: negative batch");
    if (B > p->max_batch) return set_error(AOK_ERR_LENGTH, "aok_overlap3c_gb: batch exceeds the plan's max_batch");
    int st = setup_overlap3c_schedule(p);
    if (st != AOK_OK) return st;
    if (B == 0) return AOK_OK;
    if (!out || !nprim || !prim_offset || !coef || !alpha || !posA || !posB || !posC)
        return set_error(AOK_ERR_INVALID, "aok_overlap3c_gb: null pointer");
    if ((st = check_units3(p, B, "aok_overlap3c_gb")) != AOK_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    return launch_overlap3c(p, out, alpha, coef, nprim, prim_offset, posA, posB, posC, B, 1.0, s,
                            [&] { return launch_bin(p, nullptr, nullptr, B, s); }, true);
}

extern "C" int aok_overlap3c(aok_plan* p, void* out, const void* zeta, const void* coef, const void* posA,
                             const void* posB, const void* posC, const int64_t* sidxA, const int64_t* sidxB,
                             const int64_t* sidxC, int64_t B, double lengthscale, void* stream) {
    static const char* who = "aok_overlap3c";
    if (!p) return set_error(AOK_ERR_INVALID, std::string(who) + ": null plan");
    if (B < 0) return set_error(AOK_ERR_INVALID, std::string(who) + ": negative batch");
    if (B > p->max_batch) return set_error(AOK_ERR_LENGTH, std::string(who) + ": batch exceeds the plan's max_batch");
    int st = setup_overlap3c_schedule(p);
    if (st != AOK_OK) return st;
    if (B == 0) return AOK_OK;
    if (!out || !zeta || !coef || !posA || !posB || !posC || !sidxA || !sidxB || !sidxC)
        return set_error(AOK_ERR_INVALID, std::string(who) + ": null pointer");
    if ((st = check_units3(p, B, who)) != AOK_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    ++p->gen;  // the plan's bins change
    const BinBufs bb{p->d_perm, p->d_tiles, p->d_ntiles, p->d_tbase, p->d_counter, p->d_blockhist, p->d_err};
    return launch_overlap3c(p, out, zeta, coef, nullptr, nullptr, posA, posB, posC, B, lengthscale, s,
                            [&] { return launch_bin3_into(bb, sidxA, sidxB, sidxC, B, (int)p->NZ, s); }, false);
}
