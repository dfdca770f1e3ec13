// compile_coef.cuh -- device helpers of the contraction normalisation
// (cartesian_gto_basis.jl:74-120) and its VJP (overlap_2c_grad.jl:251-286),
// shared by k_compile_coef[_pb] and the fused pullback reduction.
#pragma once

#include "aok_internal.h"

namespace aok {

__device__ __forceinline__ double cart_dfac(int n) {
    double p = 1.0;
    for (int k = n; k > 1; k -= 2) p *= k;
    return p;
}

__device__ __forceinline__ double norm_c(int l) {
    const double pi15 = 5.568327996831707845;  // pi^{3/2}
    return (pi15 * (l == 0 ? 1.0 : cart_dfac(2 * l - 1))) / (double)(1 << l);
}

// x^(l + 3/2) = x^(l+1) * sqrt(x)
__device__ __forceinline__ double pow_l32(double x, int l) {
    double r = x;
    for (int i = 0; i < l; ++i) r *= x;
    return r * sqrt(x);
}

// sum_ij D_i D_j / (z_i + z_j)^(l+3/2) over one (shell, species): lanes split
// the K x K terms, then a fixed-order butterfly reduction.
template <typename FT>
__device__ __forceinline__ double warp_normsum(const FT* __restrict__ zeta, const FT* __restrict__ D, size_t base,
                                               int ns, int K, int l, int lane) {
    double acc = 0.0;
    for (int e = lane; e < K * K; e += 32) {
        const int i = e / K, j = e % K;
        const double Di = (double)D[base + (size_t)ns * i], Dj = (double)D[base + (size_t)ns * j];
        const double zz = (double)zeta[base + (size_t)ns * i] + (double)zeta[base + (size_t)ns * j];
        acc += (Di * Dj) / pow_l32(zz, l);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    return acc;
}

// VJP of coef = D / sqrt(normsq) for one (shell, species), run by one warp:
//   dD_m = dcoef_m / n - g_m dot / (2 n^3),  dz_m = dalpha_m - h_m dot / (2 n^3)
// dcoef(i), dalpha(i): callables giving the incoming cotangents (double);
// tg: 2*K*K doubles of this warp's shared memory.  The K*K terms
// D_j / (z_m + z_j)^e (and the same over (z_m + z_j)) are spread over the
// lanes; lane m adds row m in order j = 0..K-1.
// The parameter-only half of the VJP below: normsq = c * sum_ij ..., and the K*K
// terms D_j / (z_m + z_j)^e (tg) and the same over (z_m + z_j) (th), in this
// warp's shared memory.  Returns normsq.
template <typename FT>
__device__ __forceinline__ double coef_vjp_prepare(const FT* __restrict__ zeta, const FT* __restrict__ D, double* tg,
                                                   size_t base, int ns, int K, int l, int lane) {
    auto Dv = [&](int i) { return (double)D[base + (size_t)ns * i]; };
    auto zv = [&](int i) { return (double)zeta[base + (size_t)ns * i]; };
    const double nsq = norm_c(l) * warp_normsum(zeta, D, base, ns, K, l, lane);
    double* th = tg + K * K;
    for (int e2 = lane; e2 < K * K; e2 += 32) {
        const int m = e2 / K, j = e2 % K;
        const double den = zv(m) + zv(j);
        const double p = pow_l32(den, l);
        tg[e2] = Dv(j) / p;
        th[e2] = Dv(j) / (p * den);
    }
    __syncwarp();
    return nsq;
}

// The cotangent half: dD_m = dcoef_m / n - g_m dot / (2 n^3),  dz_m = dalpha_m - h_m dot / (2 n^3).
// dcoef(i), dalpha(i): callables giving the incoming cotangents (double); tg and nsq
// from coef_vjp_prepare (same warp, or after a barrier).  Lane m adds row m in order
// j = 0..K-1.
template <typename FT, typename DC, typename DA>
__device__ __forceinline__ void coef_vjp_finish(FT* __restrict__ dD, FT* __restrict__ dz, DC dcoef, DA dalpha,
                                                const FT* __restrict__ D, const double* tg, double nsq, size_t base,
                                                int ns, int K, int l, int lane) {
    const double e = (double)l + 1.5;
    const double c = norm_c(l);
    auto Dv = [&](int i) { return (double)D[base + (size_t)ns * i]; };
    double dot = 0.0;
    for (int i = lane; i < K; i += 32) dot += dcoef(i) * Dv(i);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
    if (!(nsq > 0.0)) {
        for (int m = lane; m < K; m += 32) {
            size_t o = base + (size_t)ns * m;
            dD[o] = FT(0);
            dz[o] = (FT)dalpha(m);
        }
        return;
    }
    const double n = sqrt(nsq);
    const double s2n3 = dot / (2.0 * ((n * n) * n));
    const double* th = tg + K * K;
    for (int m = lane; m < K; m += 32) {
        double gm = 0.0, hm = 0.0;
        for (int j = 0; j < K; ++j) {
            gm += tg[m * K + j];
            hm += th[m * K + j];
        }
        gm *= 2.0 * c;
        hm *= ((-2.0 * c) * e) * Dv(m);
        const size_t o = base + (size_t)ns * m;
        dD[o] = (FT)(dcoef(m) / n - gm * s2n3);
        dz[o] = (FT)(dalpha(m) - hm * s2n3);
    }
}

// VJP of coef = D / sqrt(normsq) for one (shell, species), run by one warp
// (coef_vjp_prepare, then coef_vjp_finish); tg: 2*K*K doubles of this warp's
// shared memory.
template <typename FT, typename DC, typename DA>
__device__ __forceinline__ void coef_vjp_warp(FT* __restrict__ dD, FT* __restrict__ dz, DC dcoef, DA dalpha,
                                              const FT* __restrict__ zeta, const FT* __restrict__ D, double* tg,
                                              size_t base, int ns, int K, int l, int lane) {
    const double nsq = coef_vjp_prepare<FT>(zeta, D, tg, base, ns, K, l, lane);
    coef_vjp_finish<FT>(dD, dz, dcoef, dalpha, D, tg, nsq, base, ns, K, l, lane);
}

}  // namespace aok
