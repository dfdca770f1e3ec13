// overlap2c.cu -- batched 2-center Cartesian-Gaussian overlap, sm_100a.
//
// Replaces batch_S_orbital_kernel! (src/integrals/orbital/overlap_2c.jl:165-281)
// and batch_S_kernel! (src/integrals/kernels_2c.jl:110-224).
//
// Pipeline per call (all stream-ordered, no host synchronisation):
//   k_prep2c    one thread per (species pair, shell pair): the geometry-free
//               primitive-pair records (w, mu, a/p, b/p, 1/2p) in FP64,
//               compacted to the non-zero-coefficient pairs in the
//               reference's (ip, jp) order.
//   k_bin       counting sort of the batch by species pair; tiles of 32
//               batch elements of one species pair; resets the work counter.
//   k_overlap2c persistent kernel, one CTA per SM, draining the tile queue.
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
// running block sum with TwoSum; the rounding errors are collected in the
// shared-memory slab and added at the end.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "aok_internal.h"

namespace aok {

constexpr double kPi = 3.14159265358979323846;
constexpr int kThreadsF32 = 512;
constexpr int kThreadsF64 = 256;

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
__device__ __forceinline__ void fill_pp(PPf& r, double ca, double cb, double aa, double ab) {
    double p = aa + ab;
    double x = kPi / p;
    double mu = aa * ab / p;
    r.w = (float)(ca * cb * (x * sqrt(x)));
    r.mu_hi = (float)mu;
    r.mu_lo = (float)(mu - (double)r.mu_hi);
    r.ra = (float)(aa / p);
    r.rb = (float)(ab / p);
    r.oo2p = (float)(0.5 / p);
    r.flush = 0.f;
    r.pad = 0.f;
}
__device__ __forceinline__ void fill_pp(PPd& r, double ca, double cb, double aa, double ab) {
    double p = aa + ab;
    double x = kPi / p;
    r.w = ca * cb * (x * sqrt(x));
    r.mu = aa * ab / p;
    r.ra = aa / p;
    r.rb = ab / p;
    r.oo2p = 0.5 / p;
    r.flush = 0.0;
    r.pad0 = r.pad1 = 0.0;
}

template <typename FT>
__global__ void k_prep2c(typename PPT<FT>::type* __restrict__ pp, int* __restrict__ npp,
                         const FT* __restrict__ zeta, const FT* __restrict__ coef, int ns, int K, int NZ) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= NZ * NZ * ns * ns) return;
    int sb = q % ns;
    int t = q / ns;
    int sa = t % ns;
    t /= ns;
    int gb = t % NZ, ga = t / NZ;
    auto* out = pp + (size_t)q * K * K;
    int n = 0;
    for (int ip = 0; ip < K; ++ip) {
        double ca = (double)coef[sa + ns * (ip + K * ga)];
        if (ca == 0.0) continue;
        double aa = (double)zeta[sa + ns * (ip + K * ga)];
        int row0 = n;
        for (int jp = 0; jp < K; ++jp) {
            double cb = (double)coef[sb + ns * (jp + K * gb)];
            if (cb == 0.0) continue;
            double ab = (double)zeta[sb + ns * (jp + K * gb)];
            fill_pp(out[n], ca, cb, aa, ab);
            ++n;
        }
        if (n > row0) out[n - 1].flush = 1;
    }
    npp[q] = n;
}

// --------------------------------------------------------------------------
// Species-pair bins (single CTA counting sort).
// --------------------------------------------------------------------------
constexpr int kBinThreads = 1024;
constexpr int kMaxPairs = 256;

__global__ void __launch_bounds__(kBinThreads) k_bin(const int64_t* __restrict__ sidxA,
                                                      const int64_t* __restrict__ sidxB, int B, int NZ,
                                                      int* __restrict__ perm, int4* __restrict__ tiles,
                                                      int* __restrict__ ntiles, unsigned* __restrict__ counter,
                                                      int* __restrict__ err) {
    __shared__ int hist[kMaxPairs], cursor[kMaxPairs], tbase[kMaxPairs + 1], base[kMaxPairs];
    const int np = NZ * NZ;
    for (int k = threadIdx.x; k < np; k += blockDim.x) hist[k] = 0;
    __syncthreads();
    for (int b = threadIdx.x; b < B; b += blockDim.x) {
        int64_t a = sidxA ? sidxA[b] : 1, c = sidxB ? sidxB[b] : 1;
        if (a < 1 || a > NZ || c < 1 || c > NZ) {
            atomicCAS(err, 0, AOK_ERR_SPECIES);
            continue;
        }
        atomicAdd(&hist[(a - 1) * NZ + (c - 1)], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0, tacc = 0;
        for (int k = 0; k < np; ++k) {
            base[k] = acc;
            cursor[k] = acc;
            tbase[k] = tacc;
            acc += hist[k];
            tacc += (hist[k] + kTileB - 1) / kTileB;
        }
        tbase[np] = tacc;
        *ntiles = tacc;
        *counter = 0u;
    }
    __syncthreads();
    for (int b = threadIdx.x; b < B; b += blockDim.x) {
        int64_t a = sidxA ? sidxA[b] : 1, c = sidxB ? sidxB[b] : 1;
        if (a < 1 || a > NZ || c < 1 || c > NZ) continue;
        int pos = atomicAdd(&cursor[(a - 1) * NZ + (c - 1)], 1);
        perm[pos] = b;
    }
    for (int k = threadIdx.x; k < np; k += blockDim.x) {
        int n = hist[k];
        for (int t = 0; t * kTileB < n; ++t)
            tiles[tbase[k] + t] = make_int4(k, base[k] + t * kTileB, min(kTileB, n - t * kTileB), 0);
    }
}

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
// 1-D overlap table E[i][j] = E_0^{ij} (McMurchie-Davidson t = 0 coefficient,
// built with the Obara-Saika form of the recursion, HJO eq. 9.5.6-9.5.7 with
// E_1^{ij} = (i E_0^{i-1,j} + j E_0^{i,j-1}) / 2p):
//   E[i+1][j] = PA E[i][j] + (i E[i-1][j] + j E[i][j-1]) / 2p
//   E[i][j+1] = PB E[i][j] + (i E[i-1][j] + j E[i][j-1]) / 2p
// PA = -(b/p) AB and PB = (a/p) AB are formed directly (no P - A cancellation).
// --------------------------------------------------------------------------
template <int LA, int LB, typename FT>
__device__ __forceinline__ void build_E(FT (&E)[LA + 1][LB + 1], FT PA, FT PB, FT oo2p, FT e00) {
    E[0][0] = e00;
#pragma unroll
    for (int i = 1; i <= LA; ++i) {
        if (i >= 2)
            E[i][0] = PA * E[i - 1][0] + oo2p * (FT(i - 1) * E[i - 2][0]);
        else
            E[i][0] = PA * E[i - 1][0];
    }
#pragma unroll
    for (int j = 1; j <= LB; ++j) {
        if (j >= 2)
            E[0][j] = PB * E[0][j - 1] + oo2p * (FT(j - 1) * E[0][j - 2]);
        else
            E[0][j] = PB * E[0][j - 1];
#pragma unroll
        for (int i = 1; i <= LA; ++i) {
            FT c = FT(j) * E[i - 1][j - 1];
            if (i >= 2) c = c + FT(i - 1) * E[i - 2][j];
            E[i][j] = PA * E[i - 1][j] + oo2p * c;
        }
    }
}

template <int LA, int LB>
struct ClassInfo {
    static constexpr int NA = ncart(LA), NB = ncart(LB), NE = NA * NB, N1 = 2 * LA + 1;
    static constexpr int NCH = nchunks(NE);
};

// --------------------------------------------------------------------------
// One work item for one lane (batch element): FP32C.
// dst points at the block's (0,0) element inside this lane's slab; element
// (i, j) of the block lives at dst[j*N + i].
// --------------------------------------------------------------------------
template <int LA, int LB, int C>
__device__ __noinline__ void run_item(const PPf* __restrict__ pp, int n, const Geo<float> g, float* dst, int N) {
    using CI = ClassInfo<LA, LB>;
    constexpr int L0 = C * CI::NE / CI::NCH, L1 = (C + 1) * CI::NE / CI::NCH, M = L1 - L0;
    float hi[M], part[M];
#pragma unroll
    for (int m = 0; m < M; ++m) {
        hi[m] = 0.f;
        part[m] = 0.f;
        dst[((L0 + m) / CI::NA) * N + (L0 + m) % CI::NA] = 0.f;
    }
    for (int q = 0; q < n; ++q) {
        const float4 r0 = __ldg(reinterpret_cast<const float4*>(pp + q));
        const float4 r1 = __ldg(reinterpret_cast<const float4*>(pp + q) + 1);
        const float w = r0.x, mu_hi = r0.y, mu_lo = r0.z, ra = r0.w, rb = r1.x, oo2p = r1.y, flush = r1.z;
        // exp(-mu R^2) with the argument in double-float
        const float xh = mu_hi * g.R2;
        const float xl = fmaf(mu_hi, g.R2, -xh) + fmaf(mu_lo, g.R2, mu_hi * g.R2lo);
        const float e00 = (expf(-xh) * (1.f - xl)) * w;
        float Ex[LA + 1][LB + 1], Ey[LA + 1][LB + 1], Ez[LA + 1][LB + 1];
        build_E<LA, LB, float>(Ex, -rb * g.AB[0], ra * g.AB[0], oo2p, e00);
        build_E<LA, LB, float>(Ey, -rb * g.AB[1], ra * g.AB[1], oo2p, 1.f);
        build_E<LA, LB, float>(Ez, -rb * g.AB[2], ra * g.AB[2], oo2p, 1.f);
#pragma unroll
        for (int c2 = 0; c2 < CI::NB; ++c2)
#pragma unroll
            for (int c1 = 0; c1 < CI::NA; ++c1) {
                const int lin = c1 + CI::N1 * c2;
                if (lin >= L0 && lin < L1) {
                    const float yz = Ey[cart_y(LA, c1)][cart_y(LB, c2)] * Ez[cart_z(LA, c1)][cart_z(LB, c2)];
                    part[lin - L0] = fmaf(Ex[cart_x(LA, c1)][cart_x(LB, c2)], yz, part[lin - L0]);
                }
            }
        if (flush != 0.f) {
#pragma unroll
            for (int m = 0; m < M; ++m) {
                float s, e;
                two_sum(hi[m], part[m], s, e);
                hi[m] = s;
                part[m] = 0.f;
                dst[((L0 + m) / CI::NA) * N + (L0 + m) % CI::NA] += e;
            }
        }
    }
#pragma unroll
    for (int m = 0; m < M; ++m) {
        float* d = dst + ((L0 + m) / CI::NA) * N + (L0 + m) % CI::NA;
        *d = hi[m] + *d;
    }
}

// FP64 variant: plain double accumulation.
template <int LA, int LB, int C>
__device__ __noinline__ void run_item(const PPd* __restrict__ pp, int n, const Geo<double> g, double* dst, int N) {
    using CI = ClassInfo<LA, LB>;
    constexpr int L0 = C * CI::NE / CI::NCH, L1 = (C + 1) * CI::NE / CI::NCH, M = L1 - L0;
    double acc[M];
#pragma unroll
    for (int m = 0; m < M; ++m) acc[m] = 0.0;
    for (int q = 0; q < n; ++q) {
        const double2 r0 = __ldg(reinterpret_cast<const double2*>(pp + q));
        const double2 r1 = __ldg(reinterpret_cast<const double2*>(pp + q) + 1);
        const double r2w = __ldg(reinterpret_cast<const double*>(pp + q) + 4);
        const double w = r0.x, mu = r0.y, ra = r1.x, rb = r1.y, oo2p = r2w;
        const double e00 = exp(-mu * g.R2) * w;
        double Ex[LA + 1][LB + 1], Ey[LA + 1][LB + 1], Ez[LA + 1][LB + 1];
        build_E<LA, LB, double>(Ex, -rb * g.AB[0], ra * g.AB[0], oo2p, e00);
        build_E<LA, LB, double>(Ey, -rb * g.AB[1], ra * g.AB[1], oo2p, 1.0);
        build_E<LA, LB, double>(Ez, -rb * g.AB[2], ra * g.AB[2], oo2p, 1.0);
#pragma unroll
        for (int c2 = 0; c2 < CI::NB; ++c2)
#pragma unroll
            for (int c1 = 0; c1 < CI::NA; ++c1) {
                const int lin = c1 + CI::N1 * c2;
                if (lin >= L0 && lin < L1) {
                    const double yz = Ey[cart_y(LA, c1)][cart_y(LB, c2)] * Ez[cart_z(LA, c1)][cart_z(LB, c2)];
                    acc[lin - L0] = fma(Ex[cart_x(LA, c1)][cart_x(LB, c2)], yz, acc[lin - L0]);
                }
            }
    }
#pragma unroll
    for (int m = 0; m < M; ++m) dst[((L0 + m) / CI::NA) * N + (L0 + m) % CI::NA] = acc[m];
}

template <typename PP, typename FT, int LA, int LB>
__device__ __forceinline__ void run_chunks(int chunk, const PP* pp, int n, const Geo<FT>& g, FT* dst, int N) {
    constexpr int NCH = ClassInfo<LA, LB>::NCH;
    if constexpr (NCH == 1) {
        run_item<LA, LB, 0>(pp, n, g, dst, N);
    } else if constexpr (NCH == 2) {
        if (chunk == 0) run_item<LA, LB, 0>(pp, n, g, dst, N);
        else run_item<LA, LB, 1>(pp, n, g, dst, N);
    } else {
        static_assert(NCH == 3, "chunk count");
        if (chunk == 0) run_item<LA, LB, 0>(pp, n, g, dst, N);
        else if (chunk == 1) run_item<LA, LB, 1>(pp, n, g, dst, N);
        else run_item<LA, LB, 2>(pp, n, g, dst, N);
    }
}

template <typename PP, typename FT>
__device__ __forceinline__ void dispatch(int cls, int chunk, const PP* pp, int n, const Geo<FT>& g, FT* dst, int N) {
    switch (cls) {
#define AOK_CASE(LA, LB) \
    case (LA) * 4 + (LB): run_chunks<PP, FT, LA, LB>(chunk, pp, n, g, dst, N); break;
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
    const typename PPT<FT>::type* pp;
    const int* npp;
    const int* perm;
    const int4* tiles;
    const int* ntiles;
    unsigned* counter;
    const Item* items;
    Panels panels;
    int ns, K, N, slab_stride;
    int boff[kMaxShells + 1];
};

template <typename FT, int THREADS>
__global__ void __launch_bounds__(THREADS, 1) k_overlap2c(const __grid_constant__ Ov2Params<FT> P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FT* slab = reinterpret_cast<FT*>(smem_raw);
    __shared__ int s_tile;
    __shared__ int s_next[kMaxPanels];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = THREADS / 32;
    const int ntiles = *P.ntiles;
    for (;;) {
        if (threadIdx.x == 0) {
            s_tile = (int)atomicAdd(P.counter, 1u);
            for (int i = 0; i < P.panels.n; ++i) s_next[i] = 0;
        }
        __syncthreads();
        const int tile = s_tile;
        if (tile >= ntiles) break;
        const int4 td = P.tiles[tile];
        const int pair = td.x, start = td.y, cnt = td.z;
        Geo<FT> g;
        if (lane < cnt) {
            const int b = P.perm[start + lane];
            load_geo(g, P.posA + 3 * (size_t)b, P.posB + 3 * (size_t)b, P.scale, P.use_scale != 0);
        } else {
            const FT z[3] = {FT(0), FT(0), FT(0)};
            load_geo(g, z, z, P.scale, false);
        }
        FT* sl = slab + (size_t)lane * P.slab_stride;
        for (int pn = 0; pn < P.panels.n; ++pn) {
            const int col0 = P.panels.col0[pn];
            const int i0 = P.panels.item0[pn], i1 = P.panels.item0[pn + 1];
            for (;;) {
                int it = 0;
                if (lane == 0) it = atomicAdd(&s_next[pn], 1);
                it = __shfl_sync(0xffffffffu, it, 0) + i0;
                if (it >= i1) break;
                const Item wi = P.items[it];
                const int q = (pair * P.ns + wi.sa) * P.ns + wi.sb;
                const int n = __ldg(P.npp + q);
                FT* dst = sl + (size_t)(P.boff[wi.sb] - col0) * P.N + P.boff[wi.sa];
                dispatch(wi.cls, wi.chunk, P.pp + (size_t)q * P.K * P.K, n, g, dst, P.N);
            }
            __syncthreads();
            const int len = (P.panels.col0[pn + 1] - col0) * P.N;
            for (int bl = warp; bl < cnt; bl += NW) {
                const int bg = P.perm[start + bl];
                FT* o = P.out + (size_t)bg * P.N * P.N + (size_t)col0 * P.N;
                const FT* s = slab + (size_t)bl * P.slab_stride;
                for (int e = lane; e < len; e += 32) o[e] = s[e];
            }
            __syncthreads();
        }
    }
}

// --------------------------------------------------------------------------
// Host side: schedule and launchers.
// --------------------------------------------------------------------------
static double class_cost(int la, int lb, int elems) {
    // per primitive pair: setup + three 1-D tables + contraction of `elems`
    return 24.0 + 12.0 * (la + 1) * (lb + 1) + 2.0 * elems;
}

int setup_overlap2c_schedule(aok_plan* p) {
    const int ns = (int)p->ns, N = (int)p->N;
    const size_t fsz = p->prec == AOK_PREC_F64 ? sizeof(double) : sizeof(float);
    const size_t budget = 200 * 1024;
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
                int ne = ncart(la) * ncart(lb), nch = nchunks(ne);
                for (int c = 0; c < nch; ++c) {
                    int e = (c + 1) * ne / nch - c * ne / nch;
                    Item it{(int16_t)(la * 4 + lb), (int16_t)c, (int16_t)sa, (int16_t)sb};
                    v.push_back({class_cost(la, lb, e), it});
                }
            }
        std::stable_sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
        for (auto& x : v) items.push_back(x.second);
    }
    p->panels.col0[npan] = pcols[npan];
    p->panels.item0[npan] = (int)items.size();
    p->nitems = (int)items.size();
    cudaError_t e = cudaMalloc(&p->d_items, sizeof(Item) * items.size());
    if (e != cudaSuccess) return cuda_status(e, "cudaMalloc(items)");
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
    int th = 64, bl = (n + th - 1) / th;
    if (p->prec == AOK_PREC_F64)
        k_prep2c<double><<<bl, th, 0, s>>>((PPd*)p->d_pp, p->d_npp, (const double*)zeta, (const double*)coef,
                                           (int)p->ns, (int)p->K, (int)p->NZ);
    else
        k_prep2c<float><<<bl, th, 0, s>>>((PPf*)p->d_pp, p->d_npp, (const float*)zeta, (const float*)coef,
                                          (int)p->ns, (int)p->K, (int)p->NZ);
    return cuda_status(cudaGetLastError(), "k_prep2c");
}

int launch_bin(aok_plan* p, const int64_t* sidxA, const int64_t* sidxB, int64_t B, cudaStream_t s) {
    k_bin<<<1, kBinThreads, 0, s>>>(sidxA, sidxB, (int)B, (int)p->NZ, p->d_perm, p->d_tiles, p->d_ntiles,
                                    p->d_counter, p->d_err);
    return cuda_status(cudaGetLastError(), "k_bin");
}

template <typename FT, int THREADS>
static int launch_ov2(aok_plan* p, void* out, const void* posA, const void* posB, double lengthscale,
                      cudaStream_t s) {
    Ov2Params<FT> P;
    memset(&P, 0, sizeof(P));
    P.out = (FT*)out;
    P.posA = (const FT*)posA;
    P.posB = (const FT*)posB;
    P.scale = (FT)lengthscale;
    P.use_scale = (FT)lengthscale != FT(1);
    P.pp = (const typename PPT<FT>::type*)p->d_pp;
    P.npp = p->d_npp;
    P.perm = p->d_perm;
    P.tiles = p->d_tiles;
    P.ntiles = p->d_ntiles;
    P.counter = p->d_counter;
    P.items = p->d_items;
    P.panels = p->panels;
    P.ns = (int)p->ns;
    P.K = (int)p->K;
    P.N = (int)p->N;
    P.slab_stride = (int)p->slab_stride;
    for (int i = 0; i <= p->ns; ++i) P.boff[i] = (int)p->boff[i];
    auto kern = k_overlap2c<FT, THREADS>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->smem_bytes);
    if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(k_overlap2c)");
    timing_begin(p, s);
    kern<<<p->num_sms, THREADS, p->smem_bytes, s>>>(P);
    timing_end(p, s);
    return cuda_status(cudaGetLastError(), "k_overlap2c");
}

int launch_overlap2c(aok_plan* p, void* out, const void* posA, const void* posB, int64_t B, double lengthscale,
                     cudaStream_t s) {
    (void)B;
    if (p->prec == AOK_PREC_F64) return launch_ov2<double, kThreadsF64>(p, out, posA, posB, lengthscale, s);
    return launch_ov2<float, kThreadsF32>(p, out, posA, posB, lengthscale, s);
}

}  // namespace aok
