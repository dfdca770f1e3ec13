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
// Records of a (species pair, shell pair), in one region of K*K records:
//   full   na x nb pairs (c_a != 0, c_b != 0): value and both exponent derivatives
//   valA   nza x nb pairs (listed zero bra slots): dcoef of the bra slot
//   valB   nzb x na pairs (listed zero ket slots): dcoef of the ket slot
//
// Record-parallel evaluation.  A work unit is (species pair, shell pair, chunk
// of 8 tiles = 256 batch elements, group of <= 32 records).  For each 32 batch
// elements the warp first puts lane = element and computes the cotangent
// moments G_m(b) (md2c.cuh) into shared memory; then lane = record and the
// warp loops over the elements accumulating
//   S0_m = sum_b exp(-mu R_b^2) G_m(b),   S1_m = sum_b exp(-mu R_b^2) R_b^2 G_m(b),
// (records fewer than 32 are replicated over the lanes, each copy taking every
// r-th element; the copies are added by a fixed butterfly).  Everything that
// depends on the primitive pair only (monomials, their exponent derivatives,
// coefficients, pref0) is applied once per record and unit:
//   V = pref0 sum_m mono_m S0_m,
//   dV/da = pref0 [2q sum_m dmono_m/da' S0_m - 3q sum mono S0 - rb^2 sum mono S1].
// Each unit writes its (dcoef, dalpha) for the bra and ket slots to its own
// FP64 partial row; k_pb_reduce sums the partial rows in a fixed order, so
// the result does not depend on which warp ran which unit.
#pragma once

#include "compile_coef.cuh"
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

constexpr int kPbWarps = 8;        // warps per pullback CTA
constexpr int kPbChunkTiles = 8;   // tiles (of 32 batch elements) per work unit

template <typename FT>
__device__ __forceinline__ FT warp_sum_from(FT v, int first) {
    // butterfly over the lane bits >= log2(first): adds the copies of a record
    for (int o = first; o < 32; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Record fields, loaded by the lane that owns the record.
template <typename FT> struct PBLoad;
template <> struct PBLoad<float> {
    float mu_hi, mu_lo, pref0, ca, cb, ra, rb, oo2p;
    int idx;
    __device__ __forceinline__ void load(const PBf* r) {
        const float4 x = __ldg(reinterpret_cast<const float4*>(r)), y = __ldg(reinterpret_cast<const float4*>(r) + 1),
                     z = __ldg(reinterpret_cast<const float4*>(r) + 2);
        mu_hi = x.x; mu_lo = x.y; pref0 = x.z; ca = x.w;
        cb = y.x; ra = y.y; rb = y.z; oo2p = y.w;
        idx = (int)z.x;
    }
    __device__ __forceinline__ void zero() { mu_hi = mu_lo = pref0 = ca = cb = ra = rb = oo2p = 0.f; idx = 0; }
    // exp(-mu R^2) with the argument in double-float (as the forward)
    __device__ __forceinline__ float ex(float R2, float R2lo) const {
        const float xh = mu_hi * R2;
        const float xl = fmaf(mu_hi, R2, -xh) + fmaf(mu_lo, R2, mu_hi * R2lo);
        return ex2_approx(-xh) * fmaf(-0.6931471805599453f, xl, 1.f);
    }
};
template <> struct PBLoad<double> {
    double mu, pref0, ca, cb, ra, rb, oo2p;
    int idx;
    __device__ __forceinline__ void load(const PBd* r) {
        mu = r->mu; pref0 = r->pref0; ca = r->ca; cb = r->cb; ra = r->ra; rb = r->rb; oo2p = r->oo2p;
        idx = (int)r->idx;
    }
    __device__ __forceinline__ void zero() { mu = pref0 = ca = cb = ra = rb = oo2p = 0.0; idx = 0; }
    __device__ __forceinline__ double ex(double R2, double) const { return exp(-mu * R2); }
};

template <typename FT>
struct PbParams {
    const FT* dS;
    const FT* dS2;         // non-null: the cotangent is dS - dS2 (scaled by alpha in the reductions)
    const FT* posA;
    const FT* posB;
    FT scale;
    int use_scale;
    const typename PBT<FT>::type* rec;
    const int4* counts;
    const int* perm;
    const int4* tiles;
    const int* tbase;      // first tile of each species pair (np + 1)
    unsigned* counter;     // unit queue
    const Item* items;     // static pullback item list, heaviest classes first
    int nitems, np, gmax;  // gmax: record groups per item (ceil(K*K / 32))
    double* partial;       // [unit][4][K]: bra dcoef, bra dalpha, ket dcoef, ket dalpha
    int ns, K, NZ, N;
    int boff[kMaxShells + 1];
};

// Per-warp shared memory: the 32 elements' cotangent moments and R^2, and the
// records' results for the slot sums.
// FP32 rows of G are 16-byte aligned (read as float4 broadcasts); FP64 rows
// keep an odd stride.
template <typename FT> constexpr int pb_gstride() { return sizeof(FT) == 4 ? 12 : 9; }
template <typename FT>
struct __align__(16) PbWarpSmem {
    FT G[32][pb_gstride<FT>()];  // used moment slots (<= 8) per element
    FT R2[32], R2lo[32];
    FT val[32][4];
    int slotA[32], slotB[32];
};

template <typename FT>
struct Sums4 {
    FT a0, a1, b0, b1;  // bra dcoef, bra dalpha, ket dcoef, ket dalpha of slot k = lane
};

// One unit: records [32 g, 32 g + ng) of item (sa, sb) over elements
// perm[e0, e1).  Lanes k < K return the unit's sums for slot k.
template <typename FT, int LA, int LB>
__device__ __noinline__ Sums4<FT> pb_unit(const PbParams<FT>& P, PbWarpSmem<FT>& W, int q, int4 n, int sa, int sb,
                                          int g, int e0, int e1, int lane) {
    constexpr int NM = (LA + 1) * (LB + 1), NV = md_nv(LA, LB);
    const int na = n.x, nb = n.y, nza = n.z, nzb = n.w;
    const int nrec = na * nb + nza * nb + nzb * na;
    const int ng = min(32, nrec - 32 * g);
    int npad = 1;
    while (npad < ng) npad <<= 1;
    const int reps = 32 / npad;
    const int r = 32 * g + (lane & (npad - 1)), rep = lane / npad;
    const bool own = (lane & (npad - 1)) < ng;
    PBLoad<FT> R;
    if (own) R.load(P.rec + (size_t)q * P.K * P.K + r);
    else R.zero();
    FT S0[NM], S1[NM];
#pragma unroll
    for (int m = 0; m < NM; ++m) S0[m] = S1[m] = FT(0);
    float2 S01[NV];  // FP32: (S0, S1) of the used slots as pairs, one paired FMA per slot
#pragma unroll
    for (int j = 0; j < NV; ++j) S01[j] = make_float2(0.f, 0.f);
    // each lane's batch element of the next 32, loaded one round ahead
    int bnext = e0 + lane < e1 ? P.perm[e0 + lane] : 0;
    for (int c0 = e0; c0 < e1; c0 += 32) {
        // phase A: lane = element; cotangent moments of its block
        {
            const int e = c0 + lane;
            const int b = bnext;
            if (c0 + 32 + lane < e1) bnext = P.perm[c0 + 32 + lane];
            FT G[NM];
            FT R2 = FT(0), R2lo = FT(0);
            if (e < e1) {
                Geo<FT> geo;
                load_geo(geo, P.posA + 3 * (size_t)b, P.posB + 3 * (size_t)b, P.scale, P.use_scale != 0);
                const size_t go = (size_t)b * P.N * P.N + (size_t)P.boff[sb] * P.N + P.boff[sa];
                if (P.dS2)
                    md_cotangent_diff<LA, LB, FT>(G, geo.AB, P.dS + go, P.dS2 + go, P.N);
                else
                    md_cotangent<LA, LB, FT>(G, geo.AB, P.dS + go, P.N);
                R2 = geo.R2;
                if constexpr (sizeof(FT) == 4) R2lo = geo.R2lo;
            } else {
#pragma unroll
                for (int m = 0; m < NM; ++m) G[m] = FT(0);
            }
            int j = 0;
#pragma unroll
            for (int al = 0; al <= LA; ++al)
#pragma unroll
                for (int be = 0; be <= LB; ++be)
                    if (MdTab<LA, LB>::used(al, be)) W.G[lane][j++] = G[al * (LB + 1) + be];
            W.R2[lane] = R2;
            W.R2lo[lane] = R2lo;
        }
        __syncwarp();
        // phase B: lane = record (copy `rep` of it takes elements rep, rep + reps, ...)
        const int ne = min(32, e1 - c0);
        if constexpr (sizeof(FT) == 4) {
            for (int t = rep; t < ne; t += reps) {
                const float x = R.ex(W.R2[t], W.R2lo[t]);
                const float2 xx = make_float2(x, x * W.R2[t]);
                float gv[4 * ((NV + 3) / 4)];
#pragma unroll
                for (int w = 0; w < (NV + 3) / 4; ++w) {
                    const float4 v = *reinterpret_cast<const float4*>(&W.G[t][4 * w]);
                    gv[4 * w] = v.x;
                    gv[4 * w + 1] = v.y;
                    gv[4 * w + 2] = v.z;
                    gv[4 * w + 3] = v.w;
                }
#pragma unroll
                for (int j = 0; j < NV; ++j) S01[j] = __ffma2_rn(xx, make_float2(gv[j], gv[j]), S01[j]);
            }
        } else {
            for (int t = rep; t < ne; t += reps) {
                const FT x = R.ex(W.R2[t], W.R2lo[t]);
                const FT xr = x * W.R2[t];
                int j = 0;
#pragma unroll
                for (int al = 0; al <= LA; ++al)
#pragma unroll
                    for (int be = 0; be <= LB; ++be)
                        if (MdTab<LA, LB>::used(al, be)) {
                            const FT Gm = W.G[t][j++];
                            S0[al * (LB + 1) + be] = fma(x, Gm, S0[al * (LB + 1) + be]);
                            S1[al * (LB + 1) + be] = fma(xr, Gm, S1[al * (LB + 1) + be]);
                        }
            }
        }
        __syncwarp();
    }
    if constexpr (sizeof(FT) == 4) {
        int j = 0;
#pragma unroll
        for (int al = 0; al <= LA; ++al)
#pragma unroll
            for (int be = 0; be <= LB; ++be)
                if (MdTab<LA, LB>::used(al, be)) {
                    S0[al * (LB + 1) + be] = S01[j].x;
                    S1[al * (LB + 1) + be] = S01[j].y;
                    ++j;
                }
    }
    (void)NV;
#pragma unroll
    for (int m = 0; m < NM; ++m) {
        S0[m] = warp_sum_from(S0[m], npad);
        S1[m] = warp_sum_from(S1[m], npad);
    }
    // per record: geometry-free factors, once
    FT vA0 = FT(0), vA1 = FT(0), vB0 = FT(0), vB1 = FT(0);
    int slotA = -1, slotB = -1;
    if (own && rep == 0) {
        FT T0, Ta, Tb, U, u1, u2;
        md_dual<LA, LB, FT, true>(S0, R.ra, R.rb, R.oo2p, T0, Ta, Tb);
        md_dual<LA, LB, FT, false>(S1, R.ra, R.rb, R.oo2p, U, u1, u2);
        const FT V = R.pref0 * T0;
        const int ip = R.idx & 255, jp = R.idx >> 8;
        if (r < na * nb) {
            const FT two_q = FT(2) * R.oo2p, m3q = FT(-3) * R.oo2p, cab = R.ca * R.cb * R.pref0;
            vA0 = R.cb * V;
            vA1 = cab * (two_q * Ta + m3q * T0 - (R.rb * R.rb) * U);
            vB0 = R.ca * V;
            vB1 = cab * (two_q * Tb + m3q * T0 - (R.ra * R.ra) * U);
            slotA = ip;
            slotB = jp;
        } else if (r < na * nb + nza * nb) {
            vA0 = R.cb * V;
            slotA = ip;
        } else {
            vB0 = R.ca * V;
            slotB = jp;
        }
    }
    W.val[lane][0] = vA0;
    W.val[lane][1] = vA1;
    W.val[lane][2] = vB0;
    W.val[lane][3] = vB1;
    W.slotA[lane] = slotA;
    W.slotB[lane] = slotB;
    __syncwarp();
    Sums4<FT> res{FT(0), FT(0), FT(0), FT(0)};
    if (lane < P.K) {
        for (int l = 0; l < npad; ++l) {
            if (W.slotA[l] == lane) {
                res.a0 += W.val[l][0];
                res.a1 += W.val[l][1];
            }
            if (W.slotB[l] == lane) {
                res.b0 += W.val[l][2];
                res.b1 += W.val[l][3];
            }
        }
    }
    __syncwarp();
    return res;
}

template <typename FT>
__device__ __forceinline__ Sums4<FT> pb_dispatch(int cls, const PbParams<FT>& P, PbWarpSmem<FT>& W, int q, int4 n,
                                                 int sa, int sb, int g, int e0, int e1, int lane) {
    switch (cls) {
#define AOK_PB_CASE(LA, LB) \
    case (LA) * 4 + (LB): return pb_unit<FT, LA, LB>(P, W, q, n, sa, sb, g, e0, e1, lane);
        AOK_PB_CASE(0, 0) AOK_PB_CASE(0, 1) AOK_PB_CASE(0, 2) AOK_PB_CASE(0, 3)
        AOK_PB_CASE(1, 0) AOK_PB_CASE(1, 1) AOK_PB_CASE(1, 2) AOK_PB_CASE(1, 3)
        AOK_PB_CASE(2, 0) AOK_PB_CASE(2, 1) AOK_PB_CASE(2, 2) AOK_PB_CASE(2, 3)
        AOK_PB_CASE(3, 0) AOK_PB_CASE(3, 1) AOK_PB_CASE(3, 2) AOK_PB_CASE(3, 3)
#undef AOK_PB_CASE
        default: return Sums4<FT>{FT(0), FT(0), FT(0), FT(0)};
    }
}

// Unit numbering.  Species pair k has nch_k = ceil(tiles_k / kPbChunkTiles)
// chunks; chpre = prefix of nch over the pairs (NCH = total).
//   storage id:  ((chpre[k] + j) * nitems + i) * gmax + g
//   queue order: item i outermost (heaviest classes first), then (k, j), then g.
__device__ __forceinline__ int pb_nch(const int* tbase, int k) {
    return (tbase[k + 1] - tbase[k] + kPbChunkTiles - 1) / kPbChunkTiles;
}

template <typename FT, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB) k_overlap2c_pb(const __grid_constant__ PbParams<FT> P) {
    pdl_trigger();  // the unit sums may launch now (they wait for this grid's end)
    constexpr int NW = THREADS / 32;
    __shared__ int chpre[kMaxPairs + 1];
    __shared__ PbWarpSmem<FT> wsm[NW];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int k = 0; k < P.np; ++k) {
            chpre[k] = acc;
            acc += pb_nch(P.tbase, k);
        }
        chpre[P.np] = acc;
    }
    __syncthreads();
    const int NCH = chpre[P.np];
    // 32-bit unit numbers: the partial rows of all units fit in device memory,
    // so there are far fewer than 2^32 of them
    const unsigned total = (unsigned)NCH * (unsigned)P.nitems * (unsigned)P.gmax;
    for (;;) {
        unsigned u = 0;
        if (lane == 0) u = atomicAdd(P.counter, 1u);
        u = __shfl_sync(0xffffffffu, u, 0);
        if (u >= total) break;
        const int g = (int)(u % (unsigned)P.gmax);
        const unsigned kj_i = u / (unsigned)P.gmax;
        const int i = (int)(kj_i / (unsigned)NCH), kj = (int)(kj_i % (unsigned)NCH);
        int k = 0;
        while (chpre[k + 1] <= kj) ++k;
        const int j = kj - chpre[k];
        const Item wi = P.items[i];
        const int q = (k * P.ns + wi.sa) * P.ns + wi.sb;
        const int4 n = P.counts[q];
        const int nrec = n.x * n.y + n.z * n.y + n.w * n.x;
        if (32 * g >= nrec) continue;  // empty unit: k_pb_reduce skips it
        const int t0 = P.tbase[k] + j * kPbChunkTiles, t1 = min(t0 + kPbChunkTiles, P.tbase[k + 1]);
        const int e0 = P.tiles[t0].y, e1 = P.tiles[t1 - 1].y + P.tiles[t1 - 1].z;
        const Sums4<FT> res = pb_dispatch<FT>(wi.cls, P, wsm[warp], q, n, wi.sa, wi.sb, g, e0, e1, lane);
        if (lane < P.K) {
            double* out = P.partial + ((((size_t)(chpre[k] + j) * P.nitems + i) * P.gmax + g) * 4) * P.K;
            out[0 * P.K + lane] = (double)res.a0;
            out[1 * P.K + lane] = (double)res.a1;
            out[2 * P.K + lane] = (double)res.b0;
            out[3 * P.K + lane] = (double)res.b1;
        }
    }
}

// Fixed-order sums of the unit partials, in two stages.
// k_pb_sum_units: one warp per (species pair k, item i); lane = (value, slot);
// sums the item's units over chunks, then record groups (empty units
// skipped), eight loads in flight, into rows[k][i][4][K] (zeros for an item
// without records or a species pair without batch elements).
static __global__ void k_pb_sum_units(double* __restrict__ rows, const double* __restrict__ partial,
                                      const int4* __restrict__ counts, const int* __restrict__ tbase,
                                      const Item* __restrict__ items, int ns, int K, int np, int nitems, int gmax) {
    pdl_trigger();
    const int lane = threadIdx.x & 31;
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (wid >= np * nitems) return;
    const int k = wid / nitems, i = wid % nitems;
    int chbase = 0;  // chunks of the earlier species pairs (integer sum: order-free)
    for (int k2 = lane; k2 < k; k2 += 32) chbase += pb_nch(tbase, k2);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) chbase += __shfl_xor_sync(0xffffffffu, chbase, o);
    const int nch = pb_nch(tbase, k);
    const Item wi = items[i];
    const int4 n = counts[((size_t)k * ns + wi.sa) * ns + wi.sb];
    const int ng = (n.x * n.y + n.z * n.y + n.w * n.x + 31) / 32;
    const int nu = nch * ng;
    // the bins, counts and items above were complete before the pullback kernel started;
    // only the partial rows below come from it
    pdl_wait();
    double* out = rows + ((size_t)k * nitems + i) * 4 * K;
    for (int c = lane; c < 4 * K; c += 32) {
        double sum = 0.0;
        for (int u0 = 0; u0 < nu; u0 += 8) {
            double v[8];
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                const int u = u0 + t, j = u / ng, g = u % ng;
                v[t] = u < nu ? partial[((((size_t)(chbase + j) * nitems + i) * gmax + g) * 4) * K + c] : 0.0;
            }
#pragma unroll
            for (int t = 0; t < 8; ++t) sum += v[t];
        }
        out[c] = sum;
    }
}

// Sum of one output slot (kind, shell s, primitive kk, species sigma) over the
// (side, species pair, other shell) rows, by one warp: lanes take the rows in
// a fixed strided order and a fixed butterfly adds the lanes, so the result
// is reproducible.  Zero slots with equal exponents take the first one's
// value (k_prep_pb lists the first only).
template <typename FT>
__device__ __forceinline__ double pb_slot_sum(const double* __restrict__ rows, const int* __restrict__ itemidx,
                                              const FT* __restrict__ zeta, const FT* __restrict__ coef, int ns,
                                              int K, int NZ, int nitems, int kind, int s, int kk, int sigma,
                                              int lane) {
    const int slot = s + ns * (kk + K * sigma);
    if (kind == 0 && coef[slot] == FT(0)) {
        const FT z = zeta[slot];
        for (int k2 = 0; k2 < kk; ++k2) {
            const int o = s + ns * (k2 + K * sigma);
            if (coef[o] == FT(0) && zeta[o] == z) {
                kk = k2;
                break;
            }
        }
    }
    double sum = 0.0;
    for (int w = lane; w < 2 * NZ * ns; w += 32) {
        const int side = w / (NZ * ns), other = (w / ns) % NZ, o = w % ns;
        const int k = side == 0 ? sigma * NZ + other : other * NZ + sigma;
        const int i = side == 0 ? itemidx[s * ns + o] : itemidx[o * ns + s];
        sum += rows[((size_t)k * nitems + i) * 4 * K + (side * 2 + kind) * K + kk];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    return sum;
}

// Kernel-level pullback: one warp per output slot, (dcoef, dalpha).
template <typename FT>
__global__ void k_pb_reduce(FT* __restrict__ dcoef, FT* __restrict__ dalpha, const double* __restrict__ rows,
                            const int* __restrict__ itemidx, const FT* __restrict__ zeta, const FT* __restrict__ coef,
                            int ns, int K, int NZ, int nitems, double alpha) {
    pdl_wait();
    const int lane = threadIdx.x & 31;
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int S = ns * K * NZ;
    if (wid >= 2 * S) return;
    const int kind = wid / S, slot = wid % S;
    const int s = slot % ns, kk = (slot / ns) % K, sigma = slot / (ns * K);
    const double sum =
        alpha * pb_slot_sum<FT>(rows, itemidx, zeta, coef, ns, K, NZ, nitems, kind, s, kk, sigma, lane);
    if (lane == 0) {
        if (kind == 0) dcoef[slot] = (FT)sum;
        else dalpha[slot] = (FT)sum;
    }
}

// Parameter pullback: one CTA per (shell, species).  Its warps sum the 2K
// slots of the shell (as k_pb_reduce, kept in FP64), then warp 0 applies the
// VJP of the contraction normalisation (compile_coef.cuh) -> (dD, dzeta).
template <typename FT>
__global__ void k_pb_reduce_ps(FT* __restrict__ dD, FT* __restrict__ dz, const double* __restrict__ rows,
                               const int* __restrict__ itemidx, const FT* __restrict__ zeta,
                               const FT* __restrict__ coef, const FT* __restrict__ D, const int* __restrict__ ls,
                               int ns, int K, int NZ, int nitems, double alpha) {
    extern __shared__ double red[];  // dcoef[K], dalpha[K], VJP terms [2][K*K]
    __shared__ double s_nsq;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int s = blockIdx.x % ns, sigma = blockIdx.x / ns;
    const size_t base = (size_t)s + (size_t)ns * K * sigma;
    if (warp == 0) {  // the parameter-only half of the VJP, beside the slot sums
        const double nsq = coef_vjp_prepare<FT>(zeta, D, red + 2 * K, base, ns, K, ls[s], lane);
        if (lane == 0) s_nsq = nsq;
    }
    pdl_wait();  // the parameter-only half above overlaps the unit sums
    for (int w = warp - 1; w >= 0 && w < 2 * K; w += nw - 1) {
        const double v = pb_slot_sum<FT>(rows, itemidx, zeta, coef, ns, K, NZ, nitems, w / K, s, w % K, sigma, lane);
        if (lane == 0) red[w] = alpha * v;  // the pullback is linear in the cotangent
    }
    __syncthreads();
    if (warp == 0)
        coef_vjp_finish<FT>(
            dD, dz, [&](int i) { return red[i]; }, [&](int i) { return red[K + i]; }, D, red + 2 * K, s_nsq, base,
            ns, K, ls[s], lane);
}

constexpr int kPbThreadsF32 = 32 * kPbWarps;  // two CTAs per SM
constexpr int kPbThreadsF64 = 32 * kPbWarps;  // one CTA per SM
template <typename FT> constexpr int pb_min_blocks() { return sizeof(FT) == 4 ? 2 : 1; }

// Launches the pullback kernel and its reductions.  D == nullptr: kernel-level
// pullback, out0/out1 = (dcoef, dalpha).  Otherwise the parameter pullback,
// out0/out1 = (dD, dzeta).  The cotangent is dS, or alpha (dS - dS2) when dS2 is
// given (alpha scales the reduced gradients).
template <typename FT, int THREADS>
inline int launch_pb(aok_plan* p, void* out0, void* out1, const void* dS, const void* dS2, double alpha,
                     const void* zeta, const void* coef, const void* D, const void* posA, const void* posB,
                     double lengthscale, cudaStream_t s, unsigned* counter) {
    constexpr int MINB = pb_min_blocks<FT>();
    PbParams<FT> P;
    memset(&P, 0, sizeof(P));
    P.dS = (const FT*)dS;
    P.dS2 = (const FT*)dS2;
    P.posA = (const FT*)posA;
    P.posB = (const FT*)posB;
    P.scale = (FT)lengthscale;
    P.use_scale = (FT)lengthscale != FT(1);
    P.rec = (const typename PBT<FT>::type*)p->d_pb_rec;
    P.counts = p->d_pb_counts;
    P.perm = p->d_perm;
    P.tiles = p->d_tiles;
    P.tbase = p->d_tbase;
    P.counter = counter;
    P.items = p->d_pb_items;
    P.nitems = p->nitems;
    P.np = (int)(p->NZ * p->NZ);
    P.gmax = (int)((p->K * p->K + 31) / 32);
    P.partial = (double*)p->d_partials;
    P.ns = (int)p->ns;
    P.K = (int)p->K;
    P.NZ = (int)p->NZ;
    P.N = (int)p->N;
    for (int i = 0; i <= p->ns; ++i) P.boff[i] = (int)p->boff[i];
    auto kern = k_overlap2c_pb<FT, THREADS, MINB>;
    timing_begin(p, s);
    kern<<<p->num_sms * MINB, THREADS, 0, s>>>(P);
    timing_end(p, s);
    AOK_TRY_PB(cuda_status(cudaGetLastError(), "k_overlap2c_pb"));
    const int nw1 = P.np * p->nitems;
    // the two reductions start with programmatic serialisation (pdl_wait before their first read)
    AOK_TRY_PB(cuda_status(launch_pdl(k_pb_sum_units, dim3((nw1 * 32 + 255) / 256), dim3(256), 0, s,
                                      (double*)p->d_pb_rows, (const double*)p->d_partials,
                                      (const int4*)p->d_pb_counts, (const int*)p->d_tbase,
                                      (const Item*)p->d_pb_items, (int)p->ns, (int)p->K, P.np, p->nitems, P.gmax),
                           "k_pb_sum_units"));
    if (D) {
        const size_t sm = sizeof(double) * (2 * p->K + 2 * p->K * p->K);
        if (sm > 48 * 1024) return set_error(AOK_ERR_UNSUPPORTED, "pullback: K too large");
        // one warp per slot sum (2K of them) plus the VJP warp, as far as the kernel's
        // registers allow in one CTA (the kernel loops over the slots otherwise)
        static int max_thr = 0;
        if (max_thr == 0) {
            cudaFuncAttributes fa;
            max_thr = cudaFuncGetAttributes(&fa, k_pb_reduce_ps<FT>) == cudaSuccess ? fa.maxThreadsPerBlock : 256;
        }
        const int want = 32 * (int)(2 * p->K + 1), cap = max_thr / 32 * 32;
        const unsigned thr = (unsigned)(want < cap ? want : cap < 64 ? 64 : cap);
        return cuda_status(launch_pdl(k_pb_reduce_ps<FT>, dim3((unsigned)(p->ns * p->NZ)), dim3(thr), sm, s,
                                      (FT*)out0, (FT*)out1, (const double*)p->d_pb_rows,
                                      (const int*)p->d_pb_itemidx, (const FT*)zeta, (const FT*)coef, (const FT*)D,
                                      (const int*)p->d_ls, (int)p->ns, (int)p->K, (int)p->NZ, p->nitems, alpha),
                           "k_pb_reduce_ps");
    }
    const int S = (int)(p->ns * p->K * p->NZ);
    return cuda_status(launch_pdl(k_pb_reduce<FT>, dim3((2 * S * 32 + 255) / 256), dim3(256), 0, s, (FT*)out0,
                                  (FT*)out1, (const double*)p->d_pb_rows, (const int*)p->d_pb_itemidx,
                                  (const FT*)zeta, (const FT*)coef, (int)p->ns, (int)p->K, (int)p->NZ, p->nitems,
                                  alpha),
                       "k_pb_reduce");
}

}  // namespace aok
