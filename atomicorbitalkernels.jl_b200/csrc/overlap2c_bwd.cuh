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
// Padded slots are not skipped (as in the reference): a pair with exactly one
// zero coefficient still feeds the zero slot's dcoef (value-only work).  A zero
// slot whose exponent equals that of an earlier zero slot of the same shell is
// listed once; k_pb_reduce copies the first one's (bitwise equal) value to the
// others.  In the full parameter pullback, pairs whose zero slot belongs to an
// absent shell (all coefficients zero) are dropped, because the normalisation
// pullback discards that shell (overlap_2c_grad.jl:262); the kernel-level
// pullback keeps them, so its dcoef matches the reference slot for slot.
//
// Records of a (species pair, shell pair), all row-structured:
//   full   na rows (bra primitives with c_a != 0) x nb columns (c_b != 0)
//   valA   nza rows (listed zero bra slots) x nb columns: feeds dcoef of the row
//   valB   nzb rows (listed zero ket slots) x na columns: feeds dcoef of the row
// Within a row the bra-side sums stay in registers; the ket-side sums of the
// full list go to a small per-lane shared-memory column buffer.  Row and column
// sums are added over the warp's 32 lanes by a fixed butterfly.
//
// Deterministic, no global atomics: items are assigned to warps statically
// (item i of a panel to warp i mod NW), each warp adds its sums into its own
// FP64 row of (side, kind, shell, k) slots in item order, the tile's row is the
// sum of the warp rows in warp order, and k_pb_reduce sums the tile rows in
// tile order.  With the stable species-pair binning every partial is
// reproducible.
#pragma once

#include "overlap2c_kernel.cuh"

namespace aok {

// Geometry-free record of a backward primitive pair (FP64-computed).  `idx`
// packs ip + 256 jp.
struct PBf {
    float mu_hi, mu_lo, pref0, ca, cb, ra, rb, oo2p, idx, pad[3];
};
struct PBd {
    double mu, pref0, ca, cb, ra, rb, oo2p, idx, pad[2];
};
template <typename FT> struct PBT;
template <> struct PBT<float> { using type = PBf; };
template <> struct PBT<double> { using type = PBd; };
static_assert(sizeof(PBf) == 48 && sizeof(PBd) == 80, "record sizes (whole 16-byte words)");

__device__ __forceinline__ void fill_pb(PBf& r, double ca, double cb, double aa, double ab, int ip, int jp) {
    const double p = aa + ab, x = 3.14159265358979323846 / p;
    const double mu2 = (aa * ab / p) * 1.4426950408889634074;
    r.mu_hi = (float)mu2;
    r.mu_lo = (float)(mu2 - (double)r.mu_hi);
    r.pref0 = (float)(x * sqrt(x));
    r.ca = (float)ca;
    r.cb = (float)cb;
    r.ra = (float)(aa / p);
    r.rb = (float)(ab / p);
    r.oo2p = (float)(0.5 / p);
    r.idx = (float)(ip + 256 * jp);
    r.pad[0] = r.pad[1] = r.pad[2] = 0.f;
}
__device__ __forceinline__ void fill_pb(PBd& r, double ca, double cb, double aa, double ab, int ip, int jp) {
    const double p = aa + ab, x = 3.14159265358979323846 / p;
    r.mu = aa * ab / p;
    r.pref0 = x * sqrt(x);
    r.ca = ca;
    r.cb = cb;
    r.ra = aa / p;
    r.rb = ab / p;
    r.oo2p = 0.5 / p;
    r.idx = (double)(ip + 256 * jp);
    r.pad[0] = r.pad[1] = 0.0;
}

// One warp per (species pair, shell pair): the three row-structured lists in
// one region of K*K records, counts (na, nb, nza, nzb).  The per-slot flags
// (non-zero; listed zero slot) of both shells go to shared memory first, so
// that every record's ranks are O(K) shared-memory reads.
constexpr int kPrepPbWarps = 4;

template <typename FT>
__global__ void __launch_bounds__(32 * kPrepPbWarps)
    k_prep_pb(typename PBT<FT>::type* __restrict__ rec, int4* __restrict__ counts, const FT* __restrict__ zeta,
              const FT* __restrict__ coef, int ns, int K, int NZ, int keep_absent) {
    extern __shared__ unsigned char flags_raw[];  // [warp][4][K]: nzA, lsA, nzB, lsB
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q = blockIdx.x * kPrepPbWarps + warp;
    if (q >= NZ * NZ * ns * ns) return;
    unsigned char* nzA = flags_raw + (size_t)warp * 4 * K;
    unsigned char *lsA = nzA + K, *nzB = nzA + 2 * K, *lsB = nzA + 3 * K;
    const int sb = q % ns;
    int t = q / ns;
    const int sa = t % ns;
    t /= ns;
    const int gb = t % NZ, ga = t / NZ;
    const FT* ca_ = coef + ns * K * ga + sa;  // ca_[ns * k]
    const FT* cb_ = coef + ns * K * gb + sb;
    const FT* za_ = zeta + ns * K * ga + sa;
    const FT* zb_ = zeta + ns * K * gb + sb;
    // a zero slot is listed iff no earlier zero slot of the shell has its exponent
    for (int k = lane; k < K; k += 32) {
        const bool za0 = ca_[ns * k] == FT(0), zb0 = cb_[ns * k] == FT(0);
        bool la = za0, lb = zb0;
        for (int k2 = 0; k2 < k; ++k2) {
            if (la && ca_[ns * k2] == FT(0) && za_[ns * k2] == za_[ns * k]) la = false;
            if (lb && cb_[ns * k2] == FT(0) && zb_[ns * k2] == zb_[ns * k]) lb = false;
        }
        nzA[k] = !za0;
        nzB[k] = !zb0;
        lsA[k] = la;
        lsB[k] = lb;
    }
    __syncwarp();
    int na = 0, nb = 0, nla = 0, nlb = 0;
    for (int k = 0; k < K; ++k) {
        na += nzA[k];
        nb += nzB[k];
        nla += lsA[k];
        nlb += lsB[k];
    }
    const int nza = (keep_absent || na > 0) ? nla : 0;
    const int nzb = (keep_absent || nb > 0) ? nlb : 0;
    auto* out = rec + (size_t)q * K * K;
    for (int e = lane; e < K * K; e += 32) {
        const int ip = e / K, jp = e % K;
        int rka = 0, rkb = 0, rza = 0, rzb = 0;  // ranks among non-zero / listed slots
        for (int k = 0; k < ip; ++k) {
            rka += nzA[k];
            rza += lsA[k];
        }
        for (int k = 0; k < jp; ++k) {
            rkb += nzB[k];
            rzb += lsB[k];
        }
        int slot = -1;
        if (nzA[ip] && nzB[jp]) slot = rka * nb + rkb;
        else if (nzB[jp] && lsA[ip] && rza < nza) slot = na * nb + rza * nb + rkb;
        else if (nzA[ip] && lsB[jp] && rzb < nzb) slot = na * nb + nza * nb + rzb * na + rka;
        if (slot >= 0)
            fill_pb(out[slot], (double)ca_[ns * ip], (double)cb_[ns * jp], (double)za_[ns * ip],
                    (double)zb_[ns * jp], ip, jp);
    }
    if (lane == 0) counts[q] = make_int4(na, nb, nza, nzb);
}

// Warps per pullback CTA and the largest item list k_pb_assign sorts.
constexpr int kPbWarps = 8;
constexpr int kAssignMax = 2048;

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

// Record fields from shared memory.
template <typename FT> struct PBLoad;
template <> struct PBLoad<float> {
    float mu_hi, mu_lo, pref0, ca, cb, ra, rb, oo2p;
    int idx;
    __device__ __forceinline__ void load(uint32_t a) {
        const float4 x = lds128(a), y = lds128(a + 16u), z = lds128(a + 32u);
        mu_hi = x.x; mu_lo = x.y; pref0 = x.z; ca = x.w;
        cb = y.x; ra = y.y; rb = y.z; oo2p = y.w;
        idx = (int)z.x;
    }
    // pref0 * exp(-mu R^2), argument in double-float (as the forward)
    __device__ __forceinline__ float pref(const Geo<float>& g) const {
        const float xh = mu_hi * g.R2;
        const float xl = fmaf(mu_hi, g.R2, -xh) + fmaf(mu_lo, g.R2, mu_hi * g.R2lo);
        return (ex2_approx(-xh) * fmaf(-0.6931471805599453f, xl, 1.f)) * pref0;
    }
};
template <> struct PBLoad<double> {
    double mu, pref0, ca, cb, ra, rb, oo2p;
    int idx;
    __device__ __forceinline__ void load(uint32_t a) {
        const double2 x = lds128d(a), y = lds128d(a + 16u), z = lds128d(a + 32u), w = lds128d(a + 48u);
        mu = x.x; pref0 = x.y; ca = y.x; cb = y.y; ra = z.x; rb = z.y; oo2p = w.x;
        idx = (int)w.y;
    }
    __device__ __forceinline__ double pref(const Geo<double>& g) const { return exp(-mu * g.R2) * pref0; }
};

template <typename FT>
__device__ __forceinline__ FT warp_sum(FT v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// One work item (shell pair) for one lane.  rec: shared-memory address of the
// item's records; n = (na, nb, nza, nzb); colbuf: this warp's ket-side column
// sums [2][K][33]; wrow: this warp's FP64 row, slot ((side*2 + kind)*ns + s)*K + k.
template <typename FT, int LA, int LB>
__device__ __noinline__ void pb_item(uint32_t rec, int4 n, const Geo<FT> g, const FT* gslab, int N, FT* colbuf,
                                     double* wrow, int ns, int K, int sa, int sb, int lane) {
    constexpr int RB = sizeof(typename PBT<FT>::type);
    const int na = n.x, nb = n.y, nza = n.z, nzb = n.w;
    if (na * nb + nza * nb + nzb * na == 0) return;  // absent shell: nothing to add
    FT G[(LA + 1) * (LB + 1)];
    md_cotangent<LA, LB, FT>(G, g.AB, gslab, N);
    const int SK = ns * K;
    // full list: value + both exponent derivatives
    for (int r = 0; r < na; ++r) {
        FT a0 = FT(0), a1 = FT(0);
        int ip = 0;
        for (int c = 0; c < nb; ++c) {
            PBLoad<FT> R;
            R.load(rec + (uint32_t)(RB * (r * nb + c)));
            const FT P = R.pref(g);  // pref0 exp(-mu R^2)
            FT T0, Ta, Tb;
            md_dual<LA, LB, FT, true>(G, R.ra, R.rb, R.oo2p, T0, Ta, Tb);
            const FT two_q = FT(2) * R.oo2p, kpre = FT(-3) * R.oo2p;  // -3/(2p)
            const FT ka = kpre - g.R2 * (R.rb * R.rb), kb = kpre - g.R2 * (R.ra * R.ra);
            const FT V = P * T0, cab = R.ca * R.cb * P;
            a0 += R.cb * V;
            a1 += cab * fma(two_q, Ta, ka * T0);
            colbuf[(0 * K + c) * 33 + lane] += R.ca * V;
            colbuf[(1 * K + c) * 33 + lane] += cab * fma(two_q, Tb, kb * T0);
            ip = R.idx & 255;
        }
        a0 = warp_sum(a0);
        a1 = warp_sum(a1);
        if (lane == 0) {
            wrow[(0 * 2 + 0) * SK + sa * K + ip] += (double)a0;
            wrow[(0 * 2 + 1) * SK + sa * K + ip] += (double)a1;
        }
    }
    if (na > 0) {
        __syncwarp();
        for (int c = 0; c < nb; ++c) {
            const FT s0 = warp_sum(colbuf[(0 * K + c) * 33 + lane]), s1 = warp_sum(colbuf[(1 * K + c) * 33 + lane]);
            colbuf[(0 * K + c) * 33 + lane] = FT(0);
            colbuf[(1 * K + c) * 33 + lane] = FT(0);
            PBLoad<FT> R;
            R.load(rec + (uint32_t)(RB * c));
            if (lane == 0) {
                const int jp = R.idx >> 8;
                wrow[(1 * 2 + 0) * SK + sb * K + jp] += (double)s0;
                wrow[(1 * 2 + 1) * SK + sb * K + jp] += (double)s1;
            }
        }
        __syncwarp();
    }
    // listed zero bra slots: dcoef of the row's slot only
    uint32_t base = rec + (uint32_t)(RB * na * nb);
    for (int r = 0; r < nza; ++r) {
        FT a0 = FT(0);
        int ip = 0;
        for (int c = 0; c < nb; ++c) {
            PBLoad<FT> R;
            R.load(base + (uint32_t)(RB * (r * nb + c)));
            FT T0, Ta, Tb;
            md_dual<LA, LB, FT, false>(G, R.ra, R.rb, R.oo2p, T0, Ta, Tb);
            a0 += R.cb * (R.pref(g) * T0);
            ip = R.idx & 255;
        }
        a0 = warp_sum(a0);
        if (lane == 0 && nb > 0) wrow[(0 * 2 + 0) * SK + sa * K + ip] += (double)a0;
    }
    // listed zero ket slots
    base += (uint32_t)(RB * nza * nb);
    for (int r = 0; r < nzb; ++r) {
        FT b0 = FT(0);
        int jp = 0;
        for (int c = 0; c < na; ++c) {
            PBLoad<FT> R;
            R.load(base + (uint32_t)(RB * (r * na + c)));
            FT T0, Ta, Tb;
            md_dual<LA, LB, FT, false>(G, R.ra, R.rb, R.oo2p, T0, Ta, Tb);
            b0 += R.ca * (R.pref(g) * T0);
            jp = R.idx >> 8;
        }
        b0 = warp_sum(b0);
        if (lane == 0 && na > 0) wrow[(1 * 2 + 0) * SK + sb * K + jp] += (double)b0;
    }
}

template <typename FT>
__device__ __forceinline__ void pb_dispatch(int cls, uint32_t rec, int4 n, const Geo<FT>& g, const FT* gs, int N,
                                            FT* colbuf, double* wrow, int ns, int K, int sa, int sb, int lane) {
    switch (cls) {
#define AOK_PB_CASE(LA, LB) \
    case (LA) * 4 + (LB): pb_item<FT, LA, LB>(rec, n, g, gs, N, colbuf, wrow, ns, K, sa, sb, lane); break;
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
    const FT* zeros;   // N*N zeros: the cotangent seen by lanes past a tile's end
    const FT* posA;
    const FT* posB;
    FT scale;
    int use_scale;
    const typename PBT<FT>::type* rec;
    const int4* counts;
    const int* perm;
    const int4* tiles;
    const int* ntiles;
    unsigned* counter;
    const Item* items;    // per pair: items grouped by warp (k_pb_assign)
    const int* woff;      // per pair: kPbWarps + 1 offsets
    int nitems;
    double* grows;     // per (CTA, warp) rows in global memory when they do not fit in shared memory
    double* tilerows;  // [tile][4 * ns * K]: (side, kind, shell, k)
    int ns, K, NZ, N;
    unsigned col_offset, row_offset;  // byte offsets in dynamic shared memory (records at 0)
    int boff[kMaxShells + 1];
};

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Persistent kernel over tiles (32 batch elements of one species pair).  Each
// lane reads its cotangent blocks directly from global memory (contiguous runs
// of a block column), so there is no shared panel and no barrier inside a
// tile.  Each warp runs its own list of the pair's items (k_pb_assign); the
// next item's records are copied into shared memory (cp.async,
// double-buffered) while the current one runs.
template <typename FT, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB) k_overlap2c_pb(const __grid_constant__ PbParams<FT> P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NW = THREADS / 32;
    constexpr int REC = sizeof(typename PBT<FT>::type), REC16 = REC / 16;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int R = 4 * P.ns * P.K, KK = P.K * P.K;
    // two record buffers per warp
    const uint32_t rec0 = (uint32_t)__cvta_generic_to_shared(smem_raw) + (uint32_t)(2 * warp * KK * REC);
    FT* colbuf = reinterpret_cast<FT*>(smem_raw + P.col_offset) + (size_t)warp * 2 * P.K * 33;
    double* rows = P.grows ? P.grows + (size_t)blockIdx.x * NW * R : reinterpret_cast<double*>(smem_raw + P.row_offset);
    double* wrow = rows + (size_t)warp * R;
    __shared__ int s_tile;
    for (int i = lane; i < 2 * P.K * 33; i += 32) colbuf[i] = FT(0);
    const int ntiles = *P.ntiles;
    for (;;) {
        if (threadIdx.x == 0) s_tile = (int)atomicAdd(P.counter, 1u);
        __syncthreads();
        const int tile = s_tile;
        if (tile >= ntiles) break;
        for (int i = lane; i < R; i += 32) wrow[i] = 0.0;
        __syncwarp();
        const int4 td = P.tiles[tile];
        const int pair = td.x, start = td.y, cnt = td.z;
        Geo<FT> g;
        const FT* gbase = P.zeros;
        if (lane < cnt) {
            const int b = P.perm[start + lane];
            load_geo(g, P.posA + 3 * (size_t)b, P.posB + 3 * (size_t)b, P.scale, P.use_scale != 0);
            gbase = P.dS + (size_t)b * P.N * P.N;
        } else {
            const FT z[3] = {FT(0), FT(0), FT(0)};
            load_geo(g, z, z, P.scale, false);
        }
        const Item* order = P.items + (size_t)pair * P.nitems;
        const int w0 = P.woff[pair * (kPbWarps + 1) + warp], w1 = P.woff[pair * (kPbWarps + 1) + warp + 1];
        auto issue = [&](int it, uint32_t dst) {
            const Item wi = order[it];
            const int q = (pair * P.ns + wi.sa) * P.ns + wi.sb;
            const int4 n = P.counts[q];
            const int nrec = n.x * n.y + n.z * n.y + n.w * n.x;
            const float4* src = reinterpret_cast<const float4*>(P.rec + (size_t)q * KK);
            for (int i = lane; i < nrec * REC16; i += 32) cp_async16(dst + 16u * i, src + i);
        };
        int k = 0;
        if (w0 < w1) issue(w0, rec0);
        cp_async_commit();
        for (int it = w0; it < w1; ++it, ++k) {
            const uint32_t cur = rec0 + (uint32_t)((k & 1) * KK * REC);
            if (it + 1 < w1) issue(it + 1, rec0 + (uint32_t)(((k + 1) & 1) * KK * REC));
            cp_async_commit();
            cp_async_wait<1>();
            __syncwarp();
            const Item wi = order[it];
            const int q = (pair * P.ns + wi.sa) * P.ns + wi.sb;
            const FT* gs = gbase + (size_t)P.boff[wi.sb] * P.N + P.boff[wi.sa];
            pb_dispatch<FT>(wi.cls, cur, P.counts[q], g, gs, P.N, colbuf, wrow, P.ns, P.K, wi.sa, wi.sb, lane);
            __syncwarp();
        }
        cp_async_wait<0>();
        __syncthreads();
        // the tile's row: the warp rows summed in warp order
        double* trow = P.tilerows + (size_t)tile * R;
        for (int t = threadIdx.x; t < R; t += blockDim.x) {
            double sum = 0.0;
            for (int w = 0; w < NW; ++w) sum += rows[(size_t)w * R + t];
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
        // four tiles' loads in flight at a time; the additions stay in tile order
        int tile = warp;
        for (; tile + 3 * NW < nt; tile += 4 * NW) {
            double v[8];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int pair = tiles[tile + u * NW].x;
                const double* row = tilerows + (size_t)(tile + u * NW) * R;
                v[2 * u] = pair / NZ == sigma ? row[c0] : 0.0;
                v[2 * u + 1] = pair % NZ == sigma ? row[c1] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) sum += v[u];
        }
        for (; tile < nt; tile += NW) {
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

constexpr int kPbThreadsF32 = 32 * kPbWarps;  // two CTAs per SM
constexpr int kPbThreadsF64 = 32 * kPbWarps;  // one CTA per SM
template <typename FT> constexpr int pb_min_blocks() { return sizeof(FT) == 4 ? 2 : 1; }

template <typename FT, int THREADS>
inline int launch_pb(aok_plan* p, void* dcoef, void* dalpha, const void* dS, const void* zeta, const void* coef,
                     const void* posA, const void* posB, double lengthscale, cudaStream_t s) {
    constexpr int NW = THREADS / 32;
    constexpr int MINB = pb_min_blocks<FT>();
    PbParams<FT> P;
    memset(&P, 0, sizeof(P));
    P.dS = (const FT*)dS;
    P.zeros = (const FT*)p->d_pb_zeros;
    P.posA = (const FT*)posA;
    P.posB = (const FT*)posB;
    P.scale = (FT)lengthscale;
    P.use_scale = (FT)lengthscale != FT(1);
    P.rec = (const typename PBT<FT>::type*)p->d_pb_rec;
    P.counts = p->d_pb_counts;
    P.perm = p->d_perm;
    P.tiles = p->d_tiles;
    P.ntiles = p->d_ntiles;
    P.counter = p->d_counter;
    P.items = p->d_pb_order;
    P.woff = p->d_pb_woff;
    P.nitems = p->nitems;
    P.tilerows = (double*)p->d_tilerows;
    P.ns = (int)p->ns;
    P.K = (int)p->K;
    P.NZ = (int)p->NZ;
    P.N = (int)p->N;
    for (int i = 0; i <= p->ns; ++i) P.boff[i] = (int)p->boff[i];
    // dynamic shared memory: record buffers (2 per warp) | column buffers | warp rows
    auto up16 = [](size_t x) { return (x + 15) / 16 * 16; };
    const size_t recs = up16((size_t)NW * 2 * p->K * p->K * sizeof(typename PBT<FT>::type));
    const size_t cols = up16((size_t)NW * 2 * p->K * 33 * sizeof(FT));
    const size_t rows = (size_t)NW * 4 * p->ns * p->K * sizeof(double);
    const size_t cap = (size_t)(MINB == 2 ? 112 : 224) * 1024;
    P.col_offset = (unsigned)recs;
    P.row_offset = (unsigned)(recs + cols);
    size_t smem = recs + cols + rows;
    if (smem > cap) {  // warp rows in global memory instead
        smem = recs + cols;
        if (smem > 227 * 1024) return set_error(AOK_ERR_UNSUPPORTED, "pullback: shared-memory budget exceeded");
        P.grows = (double*)p->d_partials;
    }
    auto kern = k_overlap2c_pb<FT, THREADS, MINB>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(k_overlap2c_pb)");
    const int grid = p->num_sms * MINB;
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
