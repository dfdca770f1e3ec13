// overlap2c_bwd.cuh -- (zeta, D) pullback of the species-aware 2C overlap, sm_100a.
//
// Replaces batch_S_orbital_pb_kernel! + _overlap_pb_coef_alpha
// (src/integrals/orbital/overlap_2c_grad.jl:71-242) and, chained with
// k_compile_coef_pb, pullback_ps (overlap_2c_grad.jl:296-304).
//
// Per primitive pair (ip, jp) of a shell pair and batch element the reference
// accumulates (overlap_2c_grad.jl:173-212), with g the cotangent read back
// through the same aliased lin -> (i, j) map as the forward:
//   Bsum = sum_c g_c E_prod,   dcoef[sa,ip] += cb pref0 Bsum,  dcoef[sb,jp] += ca pref0 Bsum
//   dalpha[sa,ip] += ca cb d/dalpha_a (pref0 E_prod) . g,  and symmetrically for jp.
// The reference evaluates d/dalpha through raised-momentum tables to l+2.
// Here the cotangent block is first contracted with the geometry into
// cotangent moments G (md2c.cuh, the transpose of the forward transform), so
// that per primitive pair Bsum = sum G mono(ra, rb, q) and the exponent
// derivatives follow from the chain rule on (ra, rb, q) and
//   d log(pref0 exp(-mu R^2))/da = -3/(2p) - R^2 (b/p)^2   (and a <-> b).
//
// Padded slots whose exponent equals that of an earlier zero slot of the same
// shell are listed once; k_pb_reduce copies the first one's (bitwise equal)
// value to the others.
// Padded slots are not skipped (as in the reference): a pair with exactly one
// zero coefficient still feeds the zero slot's dcoef (value-only work).  In
// the full parameter pullback, pairs whose zero slot belongs to an absent
// shell (all coefficients zero) are dropped, because the normalisation
// pullback discards that shell (overlap_2c_grad.jl:262); the kernel-level
// pullback keeps them, so its dcoef matches the reference slot for slot.
// Pairs with both coefficients zero contribute 0.
//
// Deterministic, no global atomics: each work item's per-lane slot sums are
// added over the 32 lanes in lane order and stored per item; after a tile,
// its CTA sums the items in their fixed order into the tile's row (FP64);
// k_pb_reduce sums the tile rows in tile order.  With the stable species-pair
// binning the tile contents, and so every partial, are reproducible.
#pragma once

#include "overlap2c_kernel.cuh"

namespace aok {

// Geometry-free record of a backward primitive pair (FP64-computed).
struct PBf {
    float pref0, ca, cb, mu_hi, mu_lo, ra, rb, oo2p, ip, jp, side, pad[5];
};
struct PBd {
    double pref0, ca, cb, mu, ra, rb, oo2p, ip, jp, side, pad[6];
};
template <typename FT> struct PBT;
template <> struct PBT<float> { using type = PBf; };
template <> struct PBT<double> { using type = PBd; };

__device__ __forceinline__ void fill_pb(PBf& r, double ca, double cb, double aa, double ab, int ip, int jp,
                                        int side) {
    const double p = aa + ab, x = 3.14159265358979323846 / p;
    const double mu2 = (aa * ab / p) * 1.4426950408889634074;
    r.pref0 = (float)(x * sqrt(x));
    r.ca = (float)ca;
    r.cb = (float)cb;
    r.mu_hi = (float)mu2;
    r.mu_lo = (float)(mu2 - (double)r.mu_hi);
    r.ra = (float)(aa / p);
    r.rb = (float)(ab / p);
    r.oo2p = (float)(0.5 / p);
    r.ip = (float)ip;
    r.jp = (float)jp;
    r.side = (float)side;
}
__device__ __forceinline__ void fill_pb(PBd& r, double ca, double cb, double aa, double ab, int ip, int jp,
                                        int side) {
    const double p = aa + ab, x = 3.14159265358979323846 / p;
    r.pref0 = x * sqrt(x);
    r.ca = ca;
    r.cb = cb;
    r.mu = aa * ab / p;
    r.ra = aa / p;
    r.rb = ab / p;
    r.oo2p = 0.5 / p;
    r.ip = ip;
    r.jp = jp;
    r.side = side;
}

// One warp per (species pair, shell pair): `full` list (both coefficients
// non-zero) and `val` list (one zero coefficient on a present shell; side 0:
// the zero slot is (sa, ip), side 1: (sb, jp)).
template <typename FT>
__global__ void k_prep_pb(typename PBT<FT>::type* __restrict__ full, typename PBT<FT>::type* __restrict__ val,
                          int2* __restrict__ counts, const FT* __restrict__ zeta, const FT* __restrict__ coef, int ns,
                          int K, int NZ, int keep_absent) {
    const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (q >= NZ * NZ * ns * ns) return;
    const int sb = q % ns;
    int t = q / ns;
    const int sa = t % ns;
    t /= ns;
    const int gb = t % NZ, ga = t / NZ;
    bool pa = false, pbk = false;
    for (int k = lane; k < K; k += 32) {
        pa |= coef[sa + ns * (k + K * ga)] != FT(0);
        pbk |= coef[sb + ns * (k + K * gb)] != FT(0);
    }
    const bool presA = keep_absent || __any_sync(0xffffffffu, pa);
    const bool presB = keep_absent || __any_sync(0xffffffffu, pbk);
    auto* of = full + (size_t)q * K * K;
    auto* ov = val + (size_t)q * K * K;
    int nf = 0, nv = 0;
    for (int e0 = 0; e0 < K * K; e0 += 32) {
        const int e = e0 + lane;
        const int ip = e / K, jp = e % K;
        double ca = 0.0, cb = 0.0, aa = 1.0, ab = 1.0;
        if (e < K * K) {
            ca = (double)coef[sa + ns * (ip + K * ga)];
            cb = (double)coef[sb + ns * (jp + K * gb)];
            aa = (double)zeta[sa + ns * (ip + K * ga)];
            ab = (double)zeta[sb + ns * (jp + K * gb)];
        }
        const bool in = e < K * K;
        const bool isf = in && ca != 0.0 && cb != 0.0;
        bool isv = in && ((ca == 0.0 && cb != 0.0 && presA) || (cb == 0.0 && ca != 0.0 && presB));
        if (isv) {
            // a zero slot whose exponent equals that of an earlier zero slot of the
            // same shell receives bitwise the same dcoef: k_pb_reduce copies it
            const int z = ca == 0.0 ? ip : jp, sz = ca == 0.0 ? sa : sb, gz = ca == 0.0 ? ga : gb;
            const FT zz = zeta[sz + ns * (z + K * gz)];
            for (int k = 0; k < z; ++k)
                if (coef[sz + ns * (k + K * gz)] == FT(0) && zeta[sz + ns * (k + K * gz)] == zz) isv = false;
        }
        const unsigned mf = __ballot_sync(0xffffffffu, isf), mv = __ballot_sync(0xffffffffu, isv);
        const unsigned lt = (1u << lane) - 1u;
        if (isf) fill_pb(of[nf + __popc(mf & lt)], ca, cb, aa, ab, ip, jp, 0);
        if (isv) fill_pb(ov[nv + __popc(mv & lt)], ca, cb, aa, ab, ip, jp, ca == 0.0 ? 0 : 1);
        nf += __popc(mf);
        nv += __popc(mv);
    }
    if (lane == 0) counts[q] = make_int2(nf, nv);
}

// ---------------------------------------------------------------------------
// Per primitive pair, from the cotangent moments G (md2c.cuh):
//   T0 = sum G mono,  Ta = (1/2q) d/da sum G mono,  Tb = (1/2q) d/db sum G mono
// with mono = rb^al ra^be q^ga and, by the chain rule on (ra, rb, q),
//   d mono/da = 2q [-(al + ga) mono + be rb^{al+1} ra^{be-1} q^ga]
//   d mono/db = 2q [al rb^{al-1} ra^{be+1} q^ga - (be + ga) mono].
// ---------------------------------------------------------------------------
template <int LA, int LB, typename FT, bool DERIV>
__device__ __forceinline__ void md_dual(const FT (&G)[(LA + 1) * (LB + 1)], FT ra, FT rb, FT q, FT& T0, FT& Ta,
                                        FT& Tb) {
    constexpr int W = LA + LB;
    FT rbp[LA + 2], rap[LB + 2], qp[W / 2 + 1];
    rbp[0] = FT(1);
#pragma unroll
    for (int k = 1; k <= LA + 1; ++k) rbp[k] = rbp[k - 1] * rb;
    rap[0] = FT(1);
#pragma unroll
    for (int k = 1; k <= LB + 1; ++k) rap[k] = rap[k - 1] * ra;
    qp[0] = FT(1);
#pragma unroll
    for (int k = 1; k <= W / 2; ++k) qp[k] = qp[k - 1] * q;
    T0 = Ta = Tb = FT(0);
#pragma unroll
    for (int al = 0; al <= LA; ++al)
#pragma unroll
        for (int be = 0; be <= LB; ++be)
            if (MdTab<LA, LB>::used(al, be)) {
                const int ga = (W - al - be) / 2;
                const FT Gm = G[al * (LB + 1) + be];
                const FT mono = (rbp[al] * rap[be]) * qp[ga];
                T0 = fma(Gm, mono, T0);
                if (DERIV) {
                    FT da = FT(-(al + ga)) * mono, db = FT(-(be + ga)) * mono;
                    if (be > 0) da = fma(FT(be), (rbp[al + 1] * rap[be - 1]) * qp[ga], da);
                    if (al > 0) db = fma(FT(al), (rbp[al - 1] * rap[be + 1]) * qp[ga], db);
                    Ta = fma(Gm, da, Ta);
                    Tb = fma(Gm, db, Tb);
                }
            }
}

template <typename FT> struct PBLoad;
template <> struct PBLoad<float> {
    float pref0, ca, cb, mu_hi, mu_lo, ra, rb, oo2p;
    int ip, jp, side;
    __device__ __forceinline__ void load(const PBf* r) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(r));
        const float4 b = __ldg(reinterpret_cast<const float4*>(r) + 1);
        const float4 c = __ldg(reinterpret_cast<const float4*>(r) + 2);
        pref0 = a.x; ca = a.y; cb = a.z; mu_hi = a.w;
        mu_lo = b.x; ra = b.y; rb = b.z; oo2p = b.w;
        ip = (int)c.x; jp = (int)c.y; side = (int)c.z;
    }
    // pref0 * exp(-mu R^2)
    __device__ __forceinline__ float pref(const Geo<float>& g) const {
        const float xh = mu_hi * g.R2;
        const float xl = fmaf(mu_hi, g.R2, -xh) + fmaf(mu_lo, g.R2, mu_hi * g.R2lo);
        return (exp2f(-xh) * fmaf(-0.6931471805599453f, xl, 1.f)) * pref0;
    }
};
template <> struct PBLoad<double> {
    double pref0, ca, cb, mu, ra, rb, oo2p;
    int ip, jp, side;
    __device__ __forceinline__ void load(const PBd* r) {
        const double2 a = __ldg(reinterpret_cast<const double2*>(r));
        const double2 b = __ldg(reinterpret_cast<const double2*>(r) + 1);
        const double2 c = __ldg(reinterpret_cast<const double2*>(r) + 2);
        const double2 d = __ldg(reinterpret_cast<const double2*>(r) + 3);
        const double2 e = __ldg(reinterpret_cast<const double2*>(r) + 4);
        pref0 = a.x; ca = a.y; cb = b.x; mu = b.y; ra = c.x; rb = c.y; oo2p = d.x;
        ip = (int)d.y; jp = (int)e.x; side = (int)e.y;
    }
    __device__ __forceinline__ double pref(const Geo<double>& g) const { return exp(-mu * g.R2) * pref0; }
};

// Per-lane slot accumulators of the current item live in shared memory:
// acc[(side*2 + kind)*K + k][lane], row stride 33 (conflict-free column sums).
template <typename FT>
__device__ __forceinline__ FT& acc_at(FT* acc, int row, int lane) {
    return acc[row * 33 + lane];
}

// One work item (shell pair) for one lane: FT = float or double.
template <typename FT, int LA, int LB>
__device__ __noinline__ void pb_item(const typename PBT<FT>::type* __restrict__ pf, int nf,
                                     const typename PBT<FT>::type* __restrict__ pv, int nv, const Geo<FT> g,
                                     const FT* gslab, int N, FT* acc, int K, int lane) {
    if (nf == 0 && nv == 0) return;  // absent shell: nothing to add
    FT G[(LA + 1) * (LB + 1)];
    md_cotangent<LA, LB, FT>(G, g.AB, gslab, N);
    // full pairs: value + both exponent derivatives
    for (int q = 0; q < nf; ++q) {
        PBLoad<FT> r;
        r.load(pf + q);
        const FT P = r.pref(g);  // pref0 exp(-mu R^2)
        FT T0, Ta, Tb;
        md_dual<LA, LB, FT, true>(G, r.ra, r.rb, r.oo2p, T0, Ta, Tb);
        const FT two_q = FT(2) * r.oo2p, kpre = FT(-3) * r.oo2p;  // -3/(2p)
        const FT ka = kpre - g.R2 * (r.rb * r.rb), kb = kpre - g.R2 * (r.ra * r.ra);
        const FT V = P * T0, cab = r.ca * r.cb * P;
        acc_at(acc, 0 * K + r.ip, lane) += r.cb * V;
        acc_at(acc, 1 * K + r.ip, lane) += cab * fma(two_q, Ta, ka * T0);
        acc_at(acc, 2 * K + r.jp, lane) += r.ca * V;
        acc_at(acc, 3 * K + r.jp, lane) += cab * fma(two_q, Tb, kb * T0);
    }
    // one-zero pairs: the zero slot's dcoef only
    for (int q = 0; q < nv; ++q) {
        PBLoad<FT> r;
        r.load(pv + q);
        const FT P = r.pref(g);
        FT T0, Ta, Tb;
        md_dual<LA, LB, FT, false>(G, r.ra, r.rb, r.oo2p, T0, Ta, Tb);
        if (r.side == 0)
            acc_at(acc, 0 * K + r.ip, lane) += r.cb * (P * T0);
        else
            acc_at(acc, 2 * K + r.jp, lane) += r.ca * (P * T0);
    }
}

template <typename FT>
__device__ __forceinline__ void pb_dispatch(int cls, const typename PBT<FT>::type* pf, int nf,
                                            const typename PBT<FT>::type* pv, int nv, const Geo<FT>& g,
                                            const FT* gs, int N, FT* acc, int K, int lane) {
    switch (cls) {
#define AOK_PB_CASE(LA, LB) \
    case (LA) * 4 + (LB): pb_item<FT, LA, LB>(pf, nf, pv, nv, g, gs, N, acc, K, lane); break;
        AOK_PB_CASE(0, 0) AOK_PB_CASE(0, 1) AOK_PB_CASE(0, 2) AOK_PB_CASE(0, 3)
        AOK_PB_CASE(1, 0) AOK_PB_CASE(1, 1) AOK_PB_CASE(1, 2) AOK_PB_CASE(1, 3)
        AOK_PB_CASE(2, 0) AOK_PB_CASE(2, 1) AOK_PB_CASE(2, 2) AOK_PB_CASE(2, 3)
        AOK_PB_CASE(3, 0) AOK_PB_CASE(3, 1) AOK_PB_CASE(3, 2) AOK_PB_CASE(3, 3)
#undef AOK_PB_CASE
        default: break;
    }
}

template <typename FT>
struct PbParams {
    const FT* dS;
    const FT* posA;
    const FT* posB;
    FT scale;
    int use_scale;
    const typename PBT<FT>::type* pf;
    const typename PBT<FT>::type* pv;
    const int2* counts;
    const int* perm;
    const int4* tiles;
    const int* ntiles;
    unsigned* counter;
    const Item* items;
    int nitems;
    Panels panels;
    const int* order_id;  // static item id of each position of `items`
    const int* csr;       // per (side, shell): static item ids, ascending
    double* itemacc;      // [gridDim.x][nitems][4K], indexed by static item id
    double* tilerows;     // [tile][4 * ns * K]: (side, kind, shell, k)
    int ns, K, NZ, N, slab_stride;
    int boff[kMaxShells + 1];
    int csr_off[2 * (kMaxShells + 1)];
};

template <typename FT, int THREADS>
__global__ void __launch_bounds__(THREADS, 1) k_overlap2c_pb(const __grid_constant__ PbParams<FT> P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NW = THREADS / 32;
    FT* slab = reinterpret_cast<FT*>(smem_raw);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    FT* acc = slab + (size_t)kTileB * P.slab_stride + (size_t)warp * (4 * P.K) * 33;
    __shared__ int s_tile;
    __shared__ int s_next[kMaxPanels];
    const int K4 = 4 * P.K;
    double* iacc = P.itemacc + (size_t)blockIdx.x * P.nitems * K4;
    for (int i = lane; i < K4 * 33; i += 32) acc[i] = FT(0);
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
        const FT* sl = slab + (size_t)lane * P.slab_stride;
        const Item* order = P.items + (size_t)pair * P.nitems;
        for (int pn = 0; pn < P.panels.n; ++pn) {
            const int col0 = P.panels.col0[pn];
            const int len = (P.panels.col0[pn + 1] - col0) * P.N;
            // stage the panel of dS for the tile's batch elements (coalesced);
            // lanes past the tile's end see zeros
            for (int bl = warp; bl < kTileB; bl += NW) {
                FT* s = slab + (size_t)bl * P.slab_stride;
                if (bl < cnt) {
                    const FT* src = P.dS + (size_t)P.perm[start + bl] * P.N * P.N + (size_t)col0 * P.N;
                    for (int e = lane; e < len; e += 32) s[e] = src[e];
                } else {
                    for (int e = lane; e < len; e += 32) s[e] = FT(0);
                }
            }
            __syncthreads();
            const int i0 = P.panels.item0[pn], i1 = P.panels.item0[pn + 1];
            for (;;) {
                int it = 0;
                if (lane == 0) it = atomicAdd(&s_next[pn], 1);
                it = __shfl_sync(0xffffffffu, it, 0) + i0;
                if (it >= i1) break;
                const Item wi = order[it];
                const int sid = P.order_id[(size_t)pair * P.nitems + it];
                const int q = (pair * P.ns + wi.sa) * P.ns + wi.sb;
                const int2 n = P.counts[q];
                const FT* gs = sl + (size_t)(P.boff[wi.sb] - col0) * P.N + P.boff[wi.sa];
                pb_dispatch<FT>(wi.cls, P.pf + (size_t)q * P.K * P.K, n.x, P.pv + (size_t)q * P.K * P.K, n.y, g, gs,
                                P.N, acc, P.K, lane);
                __syncwarp();
                // the item's slot sums over the 32 lanes, in lane order
                for (int r = lane; r < K4; r += 32) {
                    double sum = 0.0;
                    for (int l = 0; l < 32; ++l) sum += (double)acc[r * 33 + l];
                    iacc[(size_t)sid * K4 + r] = sum;
                }
                __syncwarp();
                for (int i = lane; i < K4 * 33; i += 32) acc[i] = FT(0);
                __syncwarp();
            }
            __syncthreads();
        }
        // the tile's row: the items of each (side, shell) summed in static id order
        double* trow = P.tilerows + (size_t)tile * 4 * P.ns * P.K;
        for (int t = threadIdx.x; t < 4 * P.ns * P.K; t += blockDim.x) {
            const int k = t % P.K, s = (t / P.K) % P.ns, sk = t / (P.K * P.ns);  // sk = side*2 + kind
            const int side = sk >> 1;
            const int c0 = P.csr_off[side * (P.ns + 1) + s], c1 = P.csr_off[side * (P.ns + 1) + s + 1];
            double sum = 0.0;
            for (int c = c0; c < c1; ++c) sum += iacc[(size_t)P.csr[c] * K4 + sk * P.K + k];
            trow[t] = sum;
        }
    }
}

// Fixed-order sum of the tile rows: out[kind][(s, k, sigma)].
// Grid (column groups of 32, NZ): lane = column (kind, s, k) of species sigma,
// warp w sums tiles w, w + NW, ... in order (both sides), and warp 0 adds the
// NW partials in warp order, so the result does not depend on scheduling.
constexpr int kPbReduceThreads = 512;

template <typename FT>
__global__ void __launch_bounds__(kPbReduceThreads) k_pb_reduce(FT* __restrict__ dcoef, FT* __restrict__ dalpha,
                                                                const double* __restrict__ tilerows,
                                                                const int4* __restrict__ tiles,
                                                                const int* __restrict__ ntiles,
                                                                const FT* __restrict__ zeta,
                                                                const FT* __restrict__ coef, int ns, int K, int NZ) {
    constexpr int NW = kPbReduceThreads / 32;
    __shared__ double part[NW][33];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int sigma = blockIdx.y, SK = ns * K;
    const int col = blockIdx.x * 32 + lane;  // kind * SK + s * K + k
    const bool valid = col < 2 * SK;
    const int kind = valid ? col / SK : 0, s = valid ? (col % SK) / K : 0;
    int k = valid ? col % K : 0;
    const int slot = s + ns * (k + K * sigma);
    if (valid && kind == 0 && coef[slot] == FT(0)) {
        // zero slots with equal exponents share the first one's value (k_prep_pb
        // lists the first only)
        const FT z = zeta[slot];
        for (int k2 = 0; k2 < k; ++k2) {
            const int o = s + ns * (k2 + K * sigma);
            if (coef[o] == FT(0) && zeta[o] == z) {
                k = k2;
                break;
            }
        }
    }
    const int nt = *ntiles, R = 4 * SK;
    const int c0 = (0 * 2 + kind) * SK + s * K + k, c1 = (1 * 2 + kind) * SK + s * K + k;
    double sum = 0.0;
    if (valid) {
        for (int tile = warp; tile < nt; tile += NW) {
            const int pair = tiles[tile].x;
            const double* row = tilerows + (size_t)tile * R;
            if (pair / NZ == sigma) sum += row[c0];
            if (pair % NZ == sigma) sum += row[c1];
        }
    }
    part[warp][lane] = sum;
    __syncthreads();
    if (warp == 0 && valid) {
        double tot = 0.0;
        for (int w = 0; w < NW; ++w) tot += part[w][lane];
        const int out = s + ns * (((col % SK) % K) + K * sigma);
        if (kind == 0) dcoef[out] = (FT)tot;
        else dalpha[out] = (FT)tot;
    }
}

constexpr int kPbThreadsF32 = 512;
constexpr int kPbThreadsF64 = 256;

template <typename FT, int THREADS>
inline int launch_pb(aok_plan* p, void* dcoef, void* dalpha, const void* dS, const void* zeta, const void* coef,
                     const void* posA, const void* posB, double lengthscale, cudaStream_t s) {
    constexpr int NW = THREADS / 32;
    PbParams<FT> P;
    memset(&P, 0, sizeof(P));
    P.dS = (const FT*)dS;
    P.posA = (const FT*)posA;
    P.posB = (const FT*)posB;
    P.scale = (FT)lengthscale;
    P.use_scale = (FT)lengthscale != FT(1);
    P.pf = (const typename PBT<FT>::type*)p->d_pb_full;
    P.pv = (const typename PBT<FT>::type*)p->d_pb_val;
    P.counts = p->d_pb_counts;
    P.perm = p->d_perm;
    P.tiles = p->d_tiles;
    P.ntiles = p->d_ntiles;
    P.counter = p->d_counter;
    P.items = p->d_order;
    P.nitems = p->nitems;
    P.panels = p->panels;
    P.order_id = p->d_order_id;
    P.csr = p->d_pb_csr;
    for (size_t i = 0; i < p->pb_csr_off.size(); ++i) P.csr_off[i] = p->pb_csr_off[i];
    P.itemacc = (double*)p->d_partials;
    P.tilerows = (double*)p->d_tilerows;
    P.ns = (int)p->ns;
    P.K = (int)p->K;
    P.NZ = (int)p->NZ;
    P.N = (int)p->N;
    P.slab_stride = (int)p->slab_stride;
    for (int i = 0; i <= p->ns; ++i) P.boff[i] = (int)p->boff[i];
    const size_t smem = sizeof(FT) * ((size_t)kTileB * p->slab_stride + (size_t)NW * 4 * p->K * 33);
    if (smem > 227 * 1024) return set_error(AOK_ERR_UNSUPPORTED, "pullback: shared-memory budget exceeded");
    auto kern = k_overlap2c_pb<FT, THREADS>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(k_overlap2c_pb)");
    const int grid = p->num_sms;
    timing_begin(p, s);
    kern<<<grid, THREADS, smem, s>>>(P);
    timing_end(p, s);
    AOK_TRY_PB(cuda_status(cudaGetLastError(), "k_overlap2c_pb"));
    const dim3 rgrid((unsigned)((2 * p->ns * p->K + 31) / 32), (unsigned)p->NZ);
    k_pb_reduce<FT><<<rgrid, kPbReduceThreads, 0, s>>>((FT*)dcoef, (FT*)dalpha, (const double*)p->d_tilerows,
                                                       p->d_tiles, p->d_ntiles, (const FT*)zeta,
                                                       (const FT*)coef, (int)p->ns, (int)p->K, (int)p->NZ);
    return cuda_status(cudaGetLastError(), "k_pb_reduce");
}

}  // namespace aok
