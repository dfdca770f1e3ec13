// overlap2c_bwd.cu -- pullback host side: record lists, buffers, dispatch to
// the per-precision kernels (overlap2c_bwd_f32.cu, overlap2c_bwd_f64.cu).
#include "overlap2c_bwd.cuh"

namespace aok {

int launch_prep_pb(aok_plan* p, const void* zeta, const void* coef, int keep_absent, cudaStream_t s) {
    const int n = (int)(p->NZ * p->NZ * p->ns * p->ns);
    const int th = 128, bl = (n * 32 + th - 1) / th;
    if (p->prec == AOK_PREC_F64)
        k_prep_pb<double><<<bl, th, 0, s>>>((PBd*)p->d_pb_full, (PBd*)p->d_pb_val, p->d_pb_counts,
                                            (const double*)zeta, (const double*)coef, (int)p->ns, (int)p->K,
                                            (int)p->NZ, keep_absent);
    else
        k_prep_pb<float><<<bl, th, 0, s>>>((PBf*)p->d_pb_full, (PBf*)p->d_pb_val, p->d_pb_counts,
                                           (const float*)zeta, (const float*)coef, (int)p->ns, (int)p->K,
                                           (int)p->NZ, keep_absent);
    return cuda_status(cudaGetLastError(), "k_prep_pb");
}

int ensure_pb_buffers(aok_plan* p) {
    if (p->d_pb_full) return AOK_OK;
    const size_t n = (size_t)(p->NZ * p->NZ * p->ns * p->ns) * p->K * p->K;
    const size_t rec = p->prec == AOK_PREC_F64 ? sizeof(PBd) : sizeof(PBf);
    const int NW = (p->prec == AOK_PREC_F64 ? kPbThreadsF64 : kPbThreadsF32) / 32;
    const size_t S = (size_t)(p->ns * p->K * p->NZ);
    cudaError_t e;
    if ((e = cudaMalloc(&p->d_pb_full, n * rec)) != cudaSuccess) return cuda_status(e, "cudaMalloc(pb_full)");
    if ((e = cudaMalloc(&p->d_pb_val, n * rec)) != cudaSuccess) return cuda_status(e, "cudaMalloc(pb_val)");
    if ((e = cudaMalloc(&p->d_pb_counts, sizeof(int2) * (size_t)(p->NZ * p->NZ * p->ns * p->ns))) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(pb_counts)");
    (void)NW;
    (void)S;
    if ((e = cudaMalloc(&p->d_partials, sizeof(double) * 4 * p->K * (size_t)p->nitems * p->num_sms)) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(itemacc)");
    if ((e = cudaMalloc(&p->d_tilerows, sizeof(double) * 4 * p->ns * p->K * (size_t)p->max_tiles)) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(tilerows)");
    return AOK_OK;
}

int launch_overlap2c_pb(aok_plan* p, void* dcoef, void* dalpha, const void* dS, const void* zeta, const void* coef,
                        const void* posA, const void* posB, int64_t B, double lengthscale, int keep_absent,
                        cudaStream_t s) {
    (void)B;
    AOK_TRY_PB(ensure_pb_buffers(p));
    AOK_TRY_PB(launch_prep_pb(p, zeta, coef, keep_absent, s));
    if (p->prec == AOK_PREC_F64) return launch_pb_f64(p, dcoef, dalpha, dS, zeta, coef, posA, posB, lengthscale, s);
    return launch_pb_f32(p, dcoef, dalpha, dS, zeta, coef, posA, posB, lengthscale, s);
}

}  // namespace aok
