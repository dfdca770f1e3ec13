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
// The reference evaluates d/dalpha through raised-momentum tables to l+2; here
// the same derivative is taken in forward mode on the t = 0 recursion:
//   d(pref0 F T)/d a = pref0 F [(-3/(2p) - R^2 (b/p)^2) T + dT/da],
// with F = exp(-mu R^2), T = E^x E^y E^z, dPA/da = dPB/da = (b/p) AB / p,
// dPA/db = dPB/db = -(a/p) AB / p, d(k/2p)/da = d(k/2p)/db = -(k/2p)/p.
// The contraction with g is factored per axis: H^x[i][j] = sum over
// components with x powers (i, j) of g E^y E^z (and H^y, H^z), so that
// Bsum = sum E^x H^x and the derivative = sum_axes sum dE H.
//
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
        const bool isv = in && ((ca == 0.0 && cb != 0.0 && presA) || (cb == 0.0 && ca != 0.0 && presB));
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
// Per-axis tables.
// ---------------------------------------------------------------------------
// H^x[i][j] (and H^y, H^z) from the cotangent values g of the item's chunk.
template <int LA, int LB, int L0, int L1, typename FT>
__device__ __forceinline__ void build_H(FT (&Hx)[LA + 1][LB + 1], FT (&Hy)[LA + 1][LB + 1], FT (&Hz)[LA + 1][LB + 1],
                                        const FT (&Ex)[LA + 1][LB + 1], const FT (&Ey)[LA + 1][LB + 1],
                                        const FT (&Ez)[LA + 1][LB + 1], const FT* g, bool need_yz) {
    using CI = ClassInfo<LA, LB>;
#pragma unroll
    for (int i = 0; i <= LA; ++i)
#pragma unroll
        for (int j = 0; j <= LB; ++j) Hx[i][j] = Hy[i][j] = Hz[i][j] = FT(0);
#pragma unroll
    for (int c2 = 0; c2 < CI::NB; ++c2)
#pragma unroll
        for (int c1 = 0; c1 < CI::NA; ++c1) {
            const int lin = c1 + CI::N1 * c2;
            if (lin >= L0 && lin < L1) {
                const int x1 = cart_x(LA, c1), x2 = cart_x(LB, c2), y1 = cart_y(LA, c1), y2 = cart_y(LB, c2),
                          z1 = cart_z(LA, c1), z2 = cart_z(LB, c2);
                const FT gv = g[lin - L0];
                Hx[x1][x2] += gv * (Ey[y1][y2] * Ez[z1][z2]);
                if (need_yz) {
                    const FT gx = gv * Ex[x1][x2];
                    Hy[y1][y2] += gx * Ez[z1][z2];
                    Hz[z1][z2] += gx * Ey[y1][y2];
                }
            }
        }
}

// sum_ij dE/da[i][j] H[i][j] and sum_ij dE/db[i][j] H[i][j] for one axis, by
// forward-mode differentiation of the build_E recursion.
template <int LA, int LB, typename FT>
__device__ __forceinline__ void dual_sums(const FT (&E)[LA + 1][LB + 1], const FT (&H)[LA + 1][LB + 1], FT PA, FT PB,
                                          const FT (&O)[4], FT invp, FT ua, FT ub, FT& Sa, FT& Sb) {
    FT Da[LA + 1][LB + 1], Db[LA + 1][LB + 1];
    Da[0][0] = FT(0);
    Db[0][0] = FT(0);
#pragma unroll
    for (int i = 1; i <= LA; ++i) {
        FT c = FT(0), da = ua * E[i - 1][0] + PA * Da[i - 1][0], db = ub * E[i - 1][0] + PA * Db[i - 1][0];
        if (i >= 2) {
            c = O[i - 1] * E[i - 2][0];
            da += O[i - 1] * Da[i - 2][0];
            db += O[i - 1] * Db[i - 2][0];
        }
        Da[i][0] = da - c * invp;
        Db[i][0] = db - c * invp;
    }
#pragma unroll
    for (int j = 1; j <= LB; ++j) {
        {
            FT c = FT(0), da = ua * E[0][j - 1] + PB * Da[0][j - 1], db = ub * E[0][j - 1] + PB * Db[0][j - 1];
            if (j >= 2) {
                c = O[j - 1] * E[0][j - 2];
                da += O[j - 1] * Da[0][j - 2];
                db += O[j - 1] * Db[0][j - 2];
            }
            Da[0][j] = da - c * invp;
            Db[0][j] = db - c * invp;
        }
#pragma unroll
        for (int i = 1; i <= LA; ++i) {
            FT c = O[j] * E[i - 1][j - 1];
            FT da = ua * E[i - 1][j] + PA * Da[i - 1][j] + O[j] * Da[i - 1][j - 1];
            FT db = ub * E[i - 1][j] + PA * Db[i - 1][j] + O[j] * Db[i - 1][j - 1];
            if (i >= 2) {
                c += O[i - 1] * E[i - 2][j];
                da += O[i - 1] * Da[i - 2][j];
                db += O[i - 1] * Db[i - 2][j];
            }
            Da[i][j] = da - c * invp;
            Db[i][j] = db - c * invp;
        }
    }
#pragma unroll
    for (int i = 0; i <= LA; ++i)
#pragma unroll
        for (int j = 0; j <= LB; ++j) {
            Sa += Da[i][j] * H[i][j];
            Sb += Db[i][j] * H[i][j];
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

// One work item (shell-pair chunk) for one lane: FT = float or double.
template <typename FT, int LA, int LB, int C>
__device__ __noinline__ void pb_item(const typename PBT<FT>::type* __restrict__ pf, int nf,
                                     const typename PBT<FT>::type* __restrict__ pv, int nv, const Geo<FT> g,
                                     const FT* gslab, int N, FT* acc, int K, int lane) {
    using CI = ClassInfo<LA, LB>;
    constexpr int L0 = C * CI::NE / CI::NCH, L1 = (C + 1) * CI::NE / CI::NCH, M = L1 - L0;
    FT gv[M];
#pragma unroll
    for (int m = 0; m < M; ++m) gv[m] = gslab[((L0 + m) / CI::NA) * N + (L0 + m) % CI::NA];
    // full pairs: value + both exponent derivatives
    for (int q = 0; q < nf; ++q) {
        PBLoad<FT> r;
        r.load(pf + q);
        const FT P = r.pref(g);
        const FT O[4] = {FT(0), r.oo2p, FT(2) * r.oo2p, FT(3) * r.oo2p};
        const FT invp = FT(2) * r.oo2p;
        FT PA[3], PB[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            PA[a] = -r.rb * g.AB[a];
            PB[a] = r.ra * g.AB[a];
        }
        FT Ex[LA + 1][LB + 1], Ey[LA + 1][LB + 1], Ez[LA + 1][LB + 1];
        build_E<LA, LB, FT>(Ex, PA[0], PB[0], O, FT(1));
        build_E<LA, LB, FT>(Ey, PA[1], PB[1], O, FT(1));
        build_E<LA, LB, FT>(Ez, PA[2], PB[2], O, FT(1));
        FT Hx[LA + 1][LB + 1], Hy[LA + 1][LB + 1], Hz[LA + 1][LB + 1];
        build_H<LA, LB, L0, L1, FT>(Hx, Hy, Hz, Ex, Ey, Ez, gv, true);
        FT Bs = FT(0);
#pragma unroll
        for (int i = 0; i <= LA; ++i)
#pragma unroll
            for (int j = 0; j <= LB; ++j) Bs += Ex[i][j] * Hx[i][j];
        FT Ba = FT(0), Bb = FT(0);
        if (LA + LB > 0) {
            dual_sums<LA, LB, FT>(Ex, Hx, PA[0], PB[0], O, invp, r.rb * g.AB[0] * invp, -r.ra * g.AB[0] * invp, Ba, Bb);
            dual_sums<LA, LB, FT>(Ey, Hy, PA[1], PB[1], O, invp, r.rb * g.AB[1] * invp, -r.ra * g.AB[1] * invp, Ba, Bb);
            dual_sums<LA, LB, FT>(Ez, Hz, PA[2], PB[2], O, invp, r.rb * g.AB[2] * invp, -r.ra * g.AB[2] * invp, Ba, Bb);
        }
        const FT kpre = FT(-3) * r.oo2p;  // -3/(2p)
        const FT ka = kpre - g.R2 * (r.rb * r.rb), kb = kpre - g.R2 * (r.ra * r.ra);
        const FT PBs = P * Bs, cab = r.ca * r.cb * P;
        acc_at(acc, 0 * K + r.ip, lane) += r.cb * PBs;
        acc_at(acc, 1 * K + r.ip, lane) += cab * (ka * Bs + Ba);
        acc_at(acc, 2 * K + r.jp, lane) += r.ca * PBs;
        acc_at(acc, 3 * K + r.jp, lane) += cab * (kb * Bs + Bb);
    }
    // one-zero pairs: the zero slot's dcoef only
    for (int q = 0; q < nv; ++q) {
        PBLoad<FT> r;
        r.load(pv + q);
        const FT P = r.pref(g);
        const FT O[4] = {FT(0), r.oo2p, FT(2) * r.oo2p, FT(3) * r.oo2p};
        FT Ex[LA + 1][LB + 1], Ey[LA + 1][LB + 1], Ez[LA + 1][LB + 1];
        build_E<LA, LB, FT>(Ex, -r.rb * g.AB[0], r.ra * g.AB[0], O, FT(1));
        build_E<LA, LB, FT>(Ey, -r.rb * g.AB[1], r.ra * g.AB[1], O, FT(1));
        build_E<LA, LB, FT>(Ez, -r.rb * g.AB[2], r.ra * g.AB[2], O, FT(1));
        FT Hx[LA + 1][LB + 1], Hy[LA + 1][LB + 1], Hz[LA + 1][LB + 1];
        build_H<LA, LB, L0, L1, FT>(Hx, Hy, Hz, Ex, Ey, Ez, gv, false);
        FT Bs = FT(0);
#pragma unroll
        for (int i = 0; i <= LA; ++i)
#pragma unroll
            for (int j = 0; j <= LB; ++j) Bs += Ex[i][j] * Hx[i][j];
        if (r.side == 0)
            acc_at(acc, 0 * K + r.ip, lane) += r.cb * (P * Bs);
        else
            acc_at(acc, 2 * K + r.jp, lane) += r.ca * (P * Bs);
    }
}

template <typename FT, int LA, int LB>
__device__ __forceinline__ void pb_chunks(int chunk, const typename PBT<FT>::type* pf, int nf,
                                          const typename PBT<FT>::type* pv, int nv, const Geo<FT>& g, const FT* gs,
                                          int N, FT* acc, int K, int lane) {
    constexpr int NCH = ClassInfo<LA, LB>::NCH;
    if constexpr (NCH == 1) {
        pb_item<FT, LA, LB, 0>(pf, nf, pv, nv, g, gs, N, acc, K, lane);
    } else if constexpr (NCH == 2) {
        if (chunk == 0) pb_item<FT, LA, LB, 0>(pf, nf, pv, nv, g, gs, N, acc, K, lane);
        else pb_item<FT, LA, LB, 1>(pf, nf, pv, nv, g, gs, N, acc, K, lane);
    } else {
        if (chunk == 0) pb_item<FT, LA, LB, 0>(pf, nf, pv, nv, g, gs, N, acc, K, lane);
        else if (chunk == 1) pb_item<FT, LA, LB, 1>(pf, nf, pv, nv, g, gs, N, acc, K, lane);
        else pb_item<FT, LA, LB, 2>(pf, nf, pv, nv, g, gs, N, acc, K, lane);
    }
}

template <typename FT>
__device__ __forceinline__ void pb_dispatch(int cls, int chunk, const typename PBT<FT>::type* pf, int nf,
                                            const typename PBT<FT>::type* pv, int nv, const Geo<FT>& g,
                                            const FT* gs, int N, FT* acc, int K, int lane) {
    switch (cls) {
#define AOK_PB_CASE(LA, LB) \
    case (LA) * 4 + (LB): pb_chunks<FT, LA, LB>(chunk, pf, nf, pv, nv, g, gs, N, acc, K, lane); break;
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
    double* itemacc;   // [gridDim.x][nitems][4K]
    double* tilerows;  // [tile][4 * ns * K]: (side, kind, shell, k)
    int ns, K, NZ, N, slab_stride;
    int boff[kMaxShells + 1];
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
                const int q = (pair * P.ns + wi.sa) * P.ns + wi.sb;
                const int2 n = P.counts[q];
                const FT* gs = sl + (size_t)(P.boff[wi.sb] - col0) * P.N + P.boff[wi.sa];
                pb_dispatch<FT>(wi.cls, wi.chunk, P.pf + (size_t)q * P.K * P.K, n.x, P.pv + (size_t)q * P.K * P.K,
                                n.y, g, gs, P.N, acc, P.K, lane);
                __syncwarp();
                // the item's slot sums over the 32 lanes, in lane order
                for (int r = lane; r < K4; r += 32) {
                    double sum = 0.0;
                    for (int l = 0; l < 32; ++l) sum += (double)acc[r * 33 + l];
                    iacc[(size_t)it * K4 + r] = sum;
                }
                __syncwarp();
                for (int i = lane; i < K4 * 33; i += 32) acc[i] = FT(0);
                __syncwarp();
            }
            __syncthreads();
        }
        // the tile's row: items summed in their fixed order
        double* trow = P.tilerows + (size_t)tile * 4 * P.ns * P.K;
        for (int t = threadIdx.x; t < 4 * P.ns * P.K; t += blockDim.x) {
            const int k = t % P.K, s = (t / P.K) % P.ns, sk = t / (P.K * P.ns);  // sk = side*2 + kind
            const int side = sk >> 1, kind = sk & 1;
            double sum = 0.0;
            for (int i = 0; i < P.nitems; ++i) {
                const Item wi = order[i];
                if ((side == 0 ? wi.sa : wi.sb) == s) sum += iacc[(size_t)i * K4 + (side * 2 + kind) * P.K + k];
            }
            trow[t] = sum;
        }
    }
}

// Fixed-order sum of the tile rows: out[kind][(s, k, sigma)].
template <typename FT>
__global__ void k_pb_reduce(FT* __restrict__ dcoef, FT* __restrict__ dalpha, const double* __restrict__ tilerows,
                            const int4* __restrict__ tiles, const int* __restrict__ ntiles, int ns, int K, int NZ) {
    const int S = ns * K * NZ;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * S) return;
    const int kind = t / S, slot = t % S;
    const int s = slot % ns, k = (slot / ns) % K, sigma = slot / (ns * K);
    const int nt = *ntiles, R = 4 * ns * K;
    double sum = 0.0;
    for (int tile = 0; tile < nt; ++tile) {
        const int pair = tiles[tile].x;
        const double* row = tilerows + (size_t)tile * R;
        if (pair / NZ == sigma) sum += row[((0 * 2 + kind) * ns + s) * K + k];
        if (pair % NZ == sigma) sum += row[((1 * 2 + kind) * ns + s) * K + k];
    }
    if (kind == 0) dcoef[slot] = (FT)sum;
    else dalpha[slot] = (FT)sum;
}

constexpr int kPbThreadsF32 = 512;
constexpr int kPbThreadsF64 = 256;

template <typename FT, int THREADS>
inline int launch_pb(aok_plan* p, void* dcoef, void* dalpha, const void* dS, const void* posA, const void* posB,
                     double lengthscale, cudaStream_t s) {
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
    const int S = (int)(p->ns * p->K * p->NZ);
    k_pb_reduce<FT><<<(2 * S + 127) / 128, 128, 0, s>>>((FT*)dcoef, (FT*)dalpha, (const double*)p->d_tilerows,
                                                       p->d_tiles, p->d_ntiles, (int)p->ns, (int)p->K,
                                                       (int)p->NZ);
    return cuda_status(cudaGetLastError(), "k_pb_reduce");
}

}  // namespace aok
