// overlap2c_dpos.cu -- position pullback of the species-aware 2C overlap, sm_100a.
//
// No counterpart in the reference: its rrule of batch_overlap returns no
// tangent for the positions (overlap_2c_grad.jl:309-318), and position
// gradients of the overlap are listed as not implemented.  Given the
// cotangent dS (N,N,B), this computes dA_b = sum_{mu,nu} dS[mu,nu,b] dS_{mu nu}/dA_b
// and dB_b (3,B).
//
// In the moment formulation (md2c.cuh) a shell-pair block depends on the
// geometry only through AB = A - B:
//   S_c = sum_m coef_{c,m}(AB) M_m,   M_m = sum_pp w exp(-mu R^2) mono_m,  R^2 = |AB|^2,
// so, with N_m = sum_pp mu w exp(-mu R^2) mono_m (one more FMA per slot),
//   dS_c/dAB = sum_m (d coef_{c,m}/dAB) M_m - 2 AB sum_m coef_{c,m} N_m,
// and dS/dA = dS/dAB, dS/dB = -dS/dAB.  Contracted with the cotangent g of the
// block, the derivative terms are the same compile-time term tables as the
// forward transform (each term an integer times X^px Y^py Z^pz), with one
// power differentiated per axis.  The reference's aliased block layout is
// inside the tables, so the result is the gradient of exactly what the forward
// writes.
//
// Scheduling: the batch is binned by species pair (tiles of 32 elements of one
// pair, as the forward); a CTA of 8 warps takes a tile, lane = batch element.
// The warps take the pair's shell pairs round-robin from a list ordered
// heaviest class first; each lane accumulates its element's dAB over its
// warp's shell pairs, and the 8 warp partials are added in warp order, so the
// result does not depend on scheduling.  Records (FP64-computed, per
// (species pair, shell pair), only pairs with both coefficients non-zero):
// mu and w rb^al ra^be q^ga per used moment slot.
#include <algorithm>
#include <vector>

#include "md2c.cuh"
#include "overlap2c_kernel.cuh"
#include "aok_internal.h"

namespace aok {

struct DPf {
    float mu_hi, mu_lo, mu, pad;  // mu log2(e) as hi + lo (the exponent), mu (the N moment)
    float v[8];                   // w rb^al ra^be q^ga per used slot
};
struct DPd {
    double mu, pad;
    double v[8];
};
template <typename FT> struct DPT;
template <> struct DPT<float> { using type = DPf; };
template <> struct DPT<double> { using type = DPd; };
static_assert(sizeof(DPf) == 48 && sizeof(DPd) == 80, "record sizes (whole 16-byte words)");

__device__ __forceinline__ void dp_set_mu(DPf& r, double mu) {
    const double m2 = mu * 1.4426950408889634074;
    r.mu_hi = (float)m2;
    r.mu_lo = (float)(m2 - (double)r.mu_hi);
    r.mu = (float)mu;
    r.pad = 0.f;
}
__device__ __forceinline__ void dp_set_mu(DPd& r, double mu) {
    r.mu = mu;
    r.pad = 0.0;
}

// One warp per (species pair, shell pair) q = ((ga NZ + gb) ns + sa) ns + sb:
// the records of its primitive pairs with both coefficients non-zero, in
// (ip, jp) order, and their count.
template <typename FT>
__global__ void __launch_bounds__(128) k_prep_dpos(typename DPT<FT>::type* __restrict__ rec, int* __restrict__ counts,
                                                   const FT* __restrict__ zeta, const FT* __restrict__ coef,
                                                   const int* __restrict__ ls, int ns, int K, int NZ) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q = blockIdx.x * 4 + warp;
    if (q >= NZ * NZ * ns * ns) return;
    const int sb = q % ns;
    int t = q / ns;
    const int sa = t % ns;
    t /= ns;
    const int gb = t % NZ, ga = t / NZ;
    const FT* ca_ = coef + (size_t)ns * K * ga + sa;  // ca_[ns * k]
    const FT* cb_ = coef + (size_t)ns * K * gb + sb;
    const FT* za_ = zeta + (size_t)ns * K * ga + sa;
    const FT* zb_ = zeta + (size_t)ns * K * gb + sb;
    const int la = ls[sa], lb = ls[sb];
    int na = 0, nb = 0;
    for (int k = 0; k < K; ++k) {
        na += ca_[ns * k] != FT(0);
        nb += cb_[ns * k] != FT(0);
    }
    auto* out = rec + (size_t)q * K * K;
    for (int e = lane; e < K * K; e += 32) {
        const int ip = e / K, jp = e % K;
        if (ca_[ns * ip] == FT(0) || cb_[ns * jp] == FT(0)) continue;
        int rka = 0, rkb = 0;
        for (int k = 0; k < ip; ++k) rka += ca_[ns * k] != FT(0);
        for (int k = 0; k < jp; ++k) rkb += cb_[ns * k] != FT(0);
        const double a = (double)za_[ns * ip], b = (double)zb_[ns * jp];
        const double p = a + b, x = 3.14159265358979323846 / p;
        const double w = (double)ca_[ns * ip] * (double)cb_[ns * jp] * (x * sqrt(x));
        const double ra = a / p, rb = b / p, qq = 0.5 / p;
        typename DPT<FT>::type r;
        dp_set_mu(r, a * b / p);
        int j = 0;
        for (int al = 0; al <= la; ++al)
            for (int be = 0; be <= lb; ++be)
                if ((((la - al) + (lb - be)) & 1) == 0) {
                    const int gm = (la + lb - al - be) / 2;
                    double m = w;
                    for (int i = 0; i < al; ++i) m *= rb;
                    for (int i = 0; i < be; ++i) m *= ra;
                    for (int i = 0; i < gm; ++i) m *= qq;
                    r.v[j++] = (FT)m;
                }
        for (; j < 8; ++j) r.v[j] = FT(0);
        out[rka * nb + rkb] = r;
    }
    if (lane == 0) counts[q] = na * nb;
}

template <typename FT>
struct DposParams {
    const FT* dS;
    const FT* posA;
    const FT* posB;
    FT* dA;
    FT* dB;
    FT scale;
    int use_scale;
    const typename DPT<FT>::type* rec;
    const int* counts;
    const int* perm;
    const int4* tiles;
    const int* ntiles;
    unsigned* counter;
    const Item* items;
    int nitems, ns, K, NZ, N;
    int boff[kMaxShells + 1];
};

constexpr int kDposWarps = 8;

// exp(-mu R^2) of a record, and mu
__device__ __forceinline__ float dp_exp(const DPf* r, float R2, float R2lo, float& mu) {
    const float4 h = __ldg(reinterpret_cast<const float4*>(r));
    mu = h.z;
    const float xh = h.x * R2;
    const float xl = fmaf(h.x, R2, -xh) + fmaf(h.y, R2, h.x * R2lo);
    return ex2_approx(-xh) * fmaf(-0.6931471805599453f, xl, 1.f);
}
__device__ __forceinline__ double dp_exp(const DPd* r, double R2, double, double& mu) {
    mu = __ldg(&r->mu);
    return exp(-mu * R2);
}

// The gradient of one shell pair's block for this lane's element, added to acc.
template <typename FT, int LA, int LB>
__device__ __noinline__ void dpos_item(const typename DPT<FT>::type* __restrict__ rec, int nrec, const Geo<FT>& geo,
                                       const FT* __restrict__ gs, int N, bool valid, double (&acc)[3]) {
    using TB = MdTab<LA, LB>;
    constexpr int NM = TB::NM, NV = md_nv(LA, LB);
    FT R2lo = FT(0);
    if constexpr (sizeof(FT) == 4) R2lo = geo.R2lo;
    FT Mv[NV], Nv[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) Mv[j] = Nv[j] = FT(0);
    for (int r = 0; r < nrec; ++r) {
        FT mu;
        const FT e = dp_exp(rec + r, geo.R2, R2lo, mu);
        const FT em = e * mu;
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            const FT v = __ldg(&rec[r].v[j]);
            Mv[j] = fma(e, v, Mv[j]);
            Nv[j] = fma(em, v, Nv[j]);
        }
    }
    if (!valid) return;
    FT M[NM], Nm[NM];
    {
        int j = 0;
#pragma unroll
        for (int al = 0; al <= LA; ++al)
#pragma unroll
            for (int be = 0; be <= LB; ++be) {
                const int m = al * (LB + 1) + be;
                if (TB::used(al, be)) {
                    M[m] = Mv[j];
                    Nm[m] = Nv[j];
                    ++j;
                } else {
                    M[m] = Nm[m] = FT(0);
                }
            }
    }
    constexpr auto tb = TB::make();
    FT xp[3][TB::W + 1], dxp[3][TB::W + 1];
    md_powers<TB::W, FT>(xp, geo.AB);
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        dxp[t][0] = FT(0);
#pragma unroll
        for (int k = 1; k <= TB::W; ++k) dxp[t][k] = FT(k) * xp[t][k - 1];
    }
    FT ax = FT(0), ay = FT(0), az = FT(0), an = FT(0), gv = FT(0);
#pragma unroll
    for (int i = 0; i < TB::T; ++i) {
        const MdTerm e = tb.t[i];
        if (i == 0 || tb.t[i - 1].lin != e.lin) gv = gs[(e.lin / TB::NA) * N + e.lin % TB::NA];
        if (e.cst != 0) {
            const FT t = FT(e.cst) * gv;
            const FT X = xp[0][e.px], Y = xp[1][e.py], Z = xp[2][e.pz];
            const FT tm = t * M[e.m];
            if (e.px) ax = fma(tm, dxp[0][e.px] * (Y * Z), ax);
            if (e.py) ay = fma(tm, (X * dxp[1][e.py]) * Z, ay);
            if (e.pz) az = fma(tm, (X * Y) * dxp[2][e.pz], az);
            an = fma(t * Nm[e.m], (X * Y) * Z, an);
        }
    }
    acc[0] += (double)ax - 2.0 * (double)geo.AB[0] * (double)an;
    acc[1] += (double)ay - 2.0 * (double)geo.AB[1] * (double)an;
    acc[2] += (double)az - 2.0 * (double)geo.AB[2] * (double)an;
}

template <typename FT>
__device__ __forceinline__ void dpos_dispatch(int cls, const typename DPT<FT>::type* rec, int nrec, const Geo<FT>& geo,
                                              const FT* gs, int N, bool valid, double (&acc)[3]) {
    switch (cls) {
#define AOK_DPOS_CASE(LA, LB) \
    case (LA) * 4 + (LB): dpos_item<FT, LA, LB>(rec, nrec, geo, gs, N, valid, acc); break;
        AOK_DPOS_CASE(0, 0) AOK_DPOS_CASE(0, 1) AOK_DPOS_CASE(0, 2) AOK_DPOS_CASE(0, 3)
        AOK_DPOS_CASE(1, 0) AOK_DPOS_CASE(1, 1) AOK_DPOS_CASE(1, 2) AOK_DPOS_CASE(1, 3)
        AOK_DPOS_CASE(2, 0) AOK_DPOS_CASE(2, 1) AOK_DPOS_CASE(2, 2) AOK_DPOS_CASE(2, 3)
        AOK_DPOS_CASE(3, 0) AOK_DPOS_CASE(3, 1) AOK_DPOS_CASE(3, 2) AOK_DPOS_CASE(3, 3)
#undef AOK_DPOS_CASE
        default: break;
    }
}

// FP32: two CTAs per SM (<= 128 registers); FP64: one
template <typename FT>
__global__ void __launch_bounds__(32 * kDposWarps, sizeof(FT) == 4 ? 2 : 1)
    k_overlap2c_dpos(const __grid_constant__ DposParams<FT> P) {
    __shared__ double part[kDposWarps][3][32];
    __shared__ int s_tile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ntiles = *P.ntiles;
    for (;;) {
        if (threadIdx.x == 0) s_tile = (int)atomicAdd(P.counter, 1u);
        __syncthreads();
        const int t = s_tile;
        if (t >= ntiles) break;
        const int4 tl = P.tiles[t];  // (species pair, first element in perm, count)
        const int k = tl.x;
        const bool valid = lane < tl.z;
        const int b = P.perm[tl.y + (valid ? lane : 0)];
        Geo<FT> geo;
        load_geo(geo, P.posA + 3 * (size_t)b, P.posB + 3 * (size_t)b, P.scale, P.use_scale != 0);
        const FT* gs0 = P.dS + (size_t)b * P.N * P.N;
        double acc[3] = {0.0, 0.0, 0.0};
        for (int i = warp; i < P.nitems; i += kDposWarps) {
            const Item wi = P.items[i];
            const int q = (k * P.ns + wi.sa) * P.ns + wi.sb;
            const int nrec = P.counts[q];
            if (nrec == 0) continue;
            const FT* gs = gs0 + (size_t)P.boff[wi.sb] * P.N + P.boff[wi.sa];
            dpos_dispatch<FT>(wi.cls, P.rec + (size_t)q * P.K * P.K, nrec, geo, gs, P.N, valid, acc);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) part[warp][c][lane] = acc[c];
        __syncthreads();
        if (warp == 0 && valid) {
            const double sc = P.use_scale ? (double)P.scale : 1.0;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double s = 0.0;
#pragma unroll
                for (int w = 0; w < kDposWarps; ++w) s += part[w][c][lane];
                if (P.dA) P.dA[3 * (size_t)b + c] = (FT)(sc * s);
                if (P.dB) P.dB[3 * (size_t)b + c] = (FT)(-sc * s);
            }
        }
        __syncthreads();  // part and s_tile are reused by the next tile
    }
}

static int ensure_dpos_buffers(aok_plan* p) {
    if (p->d_dpos_rec) return AOK_OK;
    const int ns = (int)p->ns;
    const size_t npair = (size_t)(p->NZ * p->NZ * ns * ns);
    const size_t rsz = p->prec == AOK_PREC_F64 ? sizeof(DPd) : sizeof(DPf);
    cudaError_t e;
    if ((e = cudaMalloc(&p->d_dpos_rec, npair * p->K * p->K * rsz)) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(dpos_rec)");
    if ((e = cudaMalloc(&p->d_dpos_counts, sizeof(int) * npair)) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(dpos_counts)");
    // one item per shell pair, heaviest classes first (round-robin over the warps)
    std::vector<std::pair<int, Item>> v;
    for (int sa = 0; sa < ns; ++sa)
        for (int sb = 0; sb < ns; ++sb) {
            const int la = (int)p->ls[sa], lb = (int)p->ls[sb];
            v.push_back({md_terms(la, lb), Item{(int16_t)(la * 4 + lb), 0, (int16_t)sa, (int16_t)sb}});
        }
    std::stable_sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    std::vector<Item> items;
    for (auto& x : v) items.push_back(x.second);
    if ((e = cudaMalloc(&p->d_dpos_items, sizeof(Item) * items.size())) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(dpos_items)");
    return cuda_status(cudaMemcpy(p->d_dpos_items, items.data(), sizeof(Item) * items.size(), cudaMemcpyHostToDevice),
                       "cudaMemcpy(dpos_items)");
}

template <typename FT>
static int launch_dpos_T(aok_plan* p, void* dA, void* dB, const void* dS, const void* posA, const void* posB,
                         double lengthscale, cudaStream_t s) {
    DposParams<FT> P;
    memset(&P, 0, sizeof(P));
    P.dS = (const FT*)dS;
    P.posA = (const FT*)posA;
    P.posB = (const FT*)posB;
    P.dA = (FT*)dA;
    P.dB = (FT*)dB;
    P.scale = (FT)lengthscale;
    P.use_scale = (FT)lengthscale != FT(1);
    P.rec = (const typename DPT<FT>::type*)p->d_dpos_rec;
    P.counts = p->d_dpos_counts;
    P.perm = p->d_perm;
    P.tiles = p->d_tiles;
    P.ntiles = p->d_ntiles;
    P.counter = p->d_counter;
    P.items = p->d_dpos_items;
    P.nitems = (int)(p->ns * p->ns);
    P.ns = (int)p->ns;
    P.K = (int)p->K;
    P.NZ = (int)p->NZ;
    P.N = (int)p->N;
    for (int i = 0; i <= p->ns; ++i) P.boff[i] = (int)p->boff[i];
    auto kern = k_overlap2c_dpos<FT>;
    int occ = 0;
    AOK_TRY_PB(kernel_prepare((const void*)kern, 0, 32 * kDposWarps, &occ));
    const int grid = std::max(1, std::min(p->max_tiles, p->num_sms * std::max(occ, 1)));
    timing_begin(p, s);
    kern<<<grid, 32 * kDposWarps, 0, s>>>(P);
    timing_end(p, s);
    return cuda_status(cudaGetLastError(), "k_overlap2c_dpos");
}

// The position pullback after argument checks: records on the plan's side
// stream while the batch is binned (pairs with a bad species index are left
// out and their dA, dB zeroed), then the kernel.
int launch_overlap2c_dpos(aok_plan* p, void* dA, void* dB, const void* dS, const void* zeta, const void* coef,
                          const int64_t* sidxA, const int64_t* sidxB, const void* posA, const void* posB, int64_t B,
                          double lengthscale, cudaStream_t s) {
    AOK_TRY_PB(ensure_dpos_buffers(p));
    AOK_TRY_PB(cuda_status(cudaEventRecord(p->ev_fork, s), "cudaEventRecord"));
    AOK_TRY_PB(cuda_status(cudaStreamWaitEvent(p->side, p->ev_fork, 0), "cudaStreamWaitEvent"));
    const int nq = (int)(p->NZ * p->NZ * p->ns * p->ns);
    if (p->prec == AOK_PREC_F64)
        k_prep_dpos<double><<<(nq + 3) / 4, 128, 0, p->side>>>((DPd*)p->d_dpos_rec, p->d_dpos_counts,
                                                               (const double*)zeta, (const double*)coef, p->d_ls,
                                                               (int)p->ns, (int)p->K, (int)p->NZ);
    else
        k_prep_dpos<float><<<(nq + 3) / 4, 128, 0, p->side>>>((DPf*)p->d_dpos_rec, p->d_dpos_counts,
                                                              (const float*)zeta, (const float*)coef, p->d_ls,
                                                              (int)p->ns, (int)p->K, (int)p->NZ);
    AOK_TRY_PB(cuda_status(cudaGetLastError(), "k_prep_dpos"));
    AOK_TRY_PB(cuda_status(cudaEventRecord(p->ev_join, p->side), "cudaEventRecord"));
    ++p->gen;  // the plan's bins change
    BinBufs bb{p->d_perm, p->d_tiles, p->d_ntiles, p->d_tbase, p->d_counter, p->d_blockhist, p->d_err};
    bb.zero3 = dA;
    bb.zero3b = dB;
    bb.zero3_bytes = p->prec == AOK_PREC_F64 ? 8 : 4;
    AOK_TRY_PB(launch_bin_into(bb, sidxA, sidxB, B, (int)p->NZ, s));
    AOK_TRY_PB(cuda_status(cudaStreamWaitEvent(s, p->ev_join, 0), "cudaStreamWaitEvent"));
    if (p->prec == AOK_PREC_F64) return launch_dpos_T<double>(p, dA, dB, dS, posA, posB, lengthscale, s);
    return launch_dpos_T<float>(p, dA, dB, dS, posA, posB, lengthscale, s);
}

}  // namespace aok
