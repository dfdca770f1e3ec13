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
#include "compile_coef.cuh"

namespace aok {

// one warp per (shell, species)
template <typename FT>
__global__ void k_compile_coef(FT* __restrict__ coef, const FT* __restrict__ zeta, const FT* __restrict__ D,
                               const int* __restrict__ ls, int ns, int K, int NZ) {
    pdl_trigger();  // the record packing may launch now (it waits for this grid's end)
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

// one warp per (shell, species)
template <typename FT>
__global__ void k_compile_coef_pb(FT* __restrict__ dD, FT* __restrict__ dz, const FT* __restrict__ dcoef,
                                  const FT* __restrict__ zeta, const FT* __restrict__ D,
                                  const FT* __restrict__ dalpha_add, const int* __restrict__ ls, int ns, int K,
                                  int NZ) {
    const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (q >= ns * NZ) return;
    const int s = q % ns, g = q / ns;
    const size_t base = (size_t)s + (size_t)ns * K * g;
    extern __shared__ double terms[];  // per warp: [2][K*K]
    coef_vjp_warp<FT>(
        dD, dz, [&](int i) { return (double)dcoef[base + (size_t)ns * i]; },
        [&](int i) { return dalpha_add ? (double)dalpha_add[base + (size_t)ns * i] : 0.0; }, zeta, D,
        terms + (size_t)(threadIdx.x >> 5) * 2 * K * K, base, ns, K, ls[s], lane);
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
