// compile_coef.cu -- spherical -> Cartesian contraction normalisation and its VJP
// on the device, so a (zeta, D) gradient step never leaves the GPU.
//
// Replaces _cart_normsq / _compile_coef (src/integrals/orbital/cartesian_gto_basis.jl:74-120)
// and _compile_coef_pb (src/integrals/orbital/overlap_2c_grad.jl:251-286):
//   normsq = c sum_ij D_i D_j / (z_i + z_j)^e,  c = pi^{3/2} (2l-1)!! / 2^l,  e = l + 3/2
//   coef   = D / sqrt(normsq)            (zero when normsq <= 0: absent shell)
//   dD_m   = dcoef_m / n - g_m dot / (2 n^3),  g_m = 2c sum_j D_j / (z_m+z_j)^e
//   dz_m   = -h_m dot / (2 n^3),  h_m = -2c e D_m sum_j D_j / (z_m+z_j)^{e+1}
// with dot = sum_i dcoef_i D_i and n = sqrt(normsq).  One warp per
// (shell, species).  All arithmetic is FP64 (also for FP32 data: these are
// the primitive normalisation constants).
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

// one warp per (shell, species)
template <typename FT>
__global__ void k_compile_coef(FT* __restrict__ coef, const FT* __restrict__ zeta, const FT* __restrict__ D,
                               const int* __restrict__ ls, int ns, int K, int NZ) {
    const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (q >= ns * NZ) return;
    const int s = q % ns, g = q / ns;
    const int l = ls[s];
    const size_t base = (size_t)s + (size_t)ns * K * g;
    const double nsq = norm_c(l) * warp_normsum(zeta, D, base, ns, K, l, lane);
    const double n = nsq > 0.0 ? sqrt(nsq) : 0.0;
    for (int m = lane; m < K; m += 32)
        coef[base + (size_t)ns * m] = nsq > 0.0 ? (FT)((double)D[base + (size_t)ns * m] / n) : FT(0);
}

// one warp per (shell, species): the K*K terms D_j / (z_m + z_j)^e (and the
// same over (z_m + z_j)) are spread over the lanes, then lane m adds row m in
// order j = 0..K-1
template <typename FT>
__global__ void k_compile_coef_pb(FT* __restrict__ dD, FT* __restrict__ dz, const FT* __restrict__ dcoef,
                                  const FT* __restrict__ zeta, const FT* __restrict__ D,
                                  const FT* __restrict__ dalpha_add, const int* __restrict__ ls, int ns, int K,
                                  int NZ) {
    const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (q >= ns * NZ) return;
    const int s = q % ns, g = q / ns;
    const int l = ls[s];
    const double e = (double)l + 1.5;
    const double c = norm_c(l);
    const size_t base = (size_t)s + (size_t)ns * K * g;
    auto Dv = [&](int i) { return (double)D[base + (size_t)ns * i]; };
    auto zv = [&](int i) { return (double)zeta[base + (size_t)ns * i]; };
    const double nsq = c * warp_normsum(zeta, D, base, ns, K, l, lane);
    double dot = 0.0;
    for (int i = lane; i < K; i += 32) dot += (double)dcoef[base + (size_t)ns * i] * Dv(i);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
    if (!(nsq > 0.0)) {
        for (int m = lane; m < K; m += 32) {
            size_t o = base + (size_t)ns * m;
            dD[o] = FT(0);
            dz[o] = dalpha_add ? dalpha_add[o] : FT(0);
        }
        return;
    }
    const double n = sqrt(nsq);
    const double s2n3 = dot / (2.0 * ((n * n) * n));
    extern __shared__ double terms[];  // per warp: [2][K*K]
    double* tg = terms + (size_t)(threadIdx.x >> 5) * 2 * K * K;
    double* th = tg + K * K;
    for (int e2 = lane; e2 < K * K; e2 += 32) {
        const int m = e2 / K, j = e2 % K;
        const double den = zv(m) + zv(j);
        const double p = pow_l32(den, l);
        tg[e2] = Dv(j) / p;
        th[e2] = Dv(j) / (p * den);
    }
    __syncwarp();
    for (int m = lane; m < K; m += 32) {
        double gm = 0.0, hm = 0.0;
        for (int j = 0; j < K; ++j) {
            gm += tg[m * K + j];
            hm += th[m * K + j];
        }
        gm *= 2.0 * c;
        hm *= ((-2.0 * c) * e) * Dv(m);
        const size_t o = base + (size_t)ns * m;
        dD[o] = (FT)((double)dcoef[o] / n - gm * s2n3);
        const double dzn = -hm * s2n3;
        dz[o] = dalpha_add ? (FT)((double)dalpha_add[o] + dzn) : (FT)dzn;
    }
}

int launch_compile_coef(aok_plan* p, void* coef, const void* zeta, const void* D, cudaStream_t s) {
    int n = (int)(p->ns * p->NZ), th = 128, bl = (n * 32 + th - 1) / th;
    if (p->prec == AOK_PREC_F64)
        k_compile_coef<double><<<bl, th, 0, s>>>((double*)coef, (const double*)zeta, (const double*)D, p->d_ls,
                                                 (int)p->ns, (int)p->K, (int)p->NZ);
    else
        k_compile_coef<float><<<bl, th, 0, s>>>((float*)coef, (const float*)zeta, (const float*)D, p->d_ls,
                                                (int)p->ns, (int)p->K, (int)p->NZ);
    return cuda_status(cudaGetLastError(), "k_compile_coef");
}

int launch_compile_coef_pb(aok_plan* p, void* dD, void* dzeta, const void* dcoef, const void* zeta, const void* D,
                           const void* dalpha_add, cudaStream_t s) {
    int n = (int)(p->ns * p->NZ), th = 128, bl = (n * 32 + th - 1) / th;
    const size_t sm = sizeof(double) * (th / 32) * 2 * p->K * p->K;
    if (sm > 48 * 1024) return set_error(AOK_ERR_UNSUPPORTED, "compile_coef pullback: K too large");
    if (p->prec == AOK_PREC_F64)
        k_compile_coef_pb<double><<<bl, th, sm, s>>>((double*)dD, (double*)dzeta, (const double*)dcoef,
                                                    (const double*)zeta, (const double*)D,
                                                    (const double*)dalpha_add, p->d_ls, (int)p->ns, (int)p->K,
                                                    (int)p->NZ);
    else
        k_compile_coef_pb<float><<<bl, th, sm, s>>>((float*)dD, (float*)dzeta, (const float*)dcoef,
                                                   (const float*)zeta, (const float*)D, (const float*)dalpha_add,
                                                   p->d_ls, (int)p->ns, (int)p->K, (int)p->NZ);
    return cuda_status(cudaGetLastError(), "k_compile_coef_pb");
}

}  // namespace aok

using namespace aok;

extern "C" int aok_compile_coef(aok_plan* p, void* coef, const void* zeta, const void* D, void* stream) {
    if (!p || !coef || !zeta || !D) return set_error(AOK_ERR_INVALID, "aok_compile_coef: null pointer");
    return launch_compile_coef(p, coef, zeta, D, (cudaStream_t)stream);
}

extern "C" int aok_compile_coef_pullback(aok_plan* p, void* dD, void* dzeta, const void* dcoef, const void* zeta,
                                         const void* D, void* stream) {
    if (!p || !dD || !dzeta || !dcoef || !zeta || !D)
        return set_error(AOK_ERR_INVALID, "aok_compile_coef_pullback: null pointer");
    return launch_compile_coef_pb(p, dD, dzeta, dcoef, zeta, D, nullptr, (cudaStream_t)stream);
}
