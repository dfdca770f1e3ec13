// measure.cu -- measurement aid: the FMA-pipe throughput of this GPU (FP32, FP32
// paired, FP64), against which the compute-bound kernels' pipe use is quoted.
// A kernel of independent FMA chains on every SM, timed with CUDA events.
#include <string>

#include "aok_internal.h"

namespace aok {

namespace {
__device__ float g_sink_f;
__device__ double g_sink_d;
constexpr int kChains = 8;
constexpr int kFmaThreads = 256;
constexpr int kFmaIters = 4096;

template <typename T>
__global__ void __launch_bounds__(kFmaThreads) k_fma_chain(int iters, T b, T c) {
    T a[kChains];
#pragma unroll
    for (int i = 0; i < kChains; ++i) a[i] = T(threadIdx.x + i) * T(1e-3);
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int i = 0; i < kChains; ++i) a[i] = fma(a[i], b, c);
    T s = T(0);
#pragma unroll
    for (int i = 0; i < kChains; ++i) s += a[i];
    if (s == T(-1)) {  // never true: keeps the chains alive
        if constexpr (sizeof(T) == 4) g_sink_f = s;
        else g_sink_d = s;
    }
}

__global__ void __launch_bounds__(kFmaThreads) k_ffma2_chain(int iters, float b, float c) {
    float2 a[kChains];
#pragma unroll
    for (int i = 0; i < kChains; ++i) a[i] = make_float2((threadIdx.x + i) * 1e-3f, (threadIdx.x - i) * 1e-3f);
    const float2 bb = make_float2(b, b), cc = make_float2(c, c);
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int i = 0; i < kChains; ++i) a[i] = __ffma2_rn(a[i], bb, cc);
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < kChains; ++i) s += a[i].x + a[i].y;
    if (s == -1.f) g_sink_f = s;
}
}  // namespace

}  // namespace aok

using namespace aok;

extern "C" int aok_measure_fma_peak(int precision, int paired, double* tflops, void* stream) {
    if (!tflops) return set_error(AOK_ERR_INVALID, "aok_measure_fma_peak: null pointer");
    if (precision != AOK_PREC_F64 && precision != AOK_PREC_F32C)
        return set_error(AOK_ERR_INVALID, "aok_measure_fma_peak: unknown precision");
    cudaStream_t s = (cudaStream_t)stream;
    int dev = 0, sms = 0;
    int st = cuda_status(cudaGetDevice(&dev), "cudaGetDevice");
    if (st != AOK_OK) return st;
    if ((st = cuda_status(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute")) !=
        AOK_OK)
        return st;
    const int grid = sms * 8;
    auto launch = [&]() {
        if (precision == AOK_PREC_F64) k_fma_chain<double><<<grid, kFmaThreads, 0, s>>>(kFmaIters, 0.999999, 1e-7);
        else if (paired) k_ffma2_chain<<<grid, kFmaThreads, 0, s>>>(kFmaIters, 0.999999f, 1e-7f);
        else k_fma_chain<float><<<grid, kFmaThreads, 0, s>>>(kFmaIters, 0.999999f, 1e-7f);
        return cuda_status(cudaGetLastError(), "k_fma_chain");
    };
    if ((st = launch()) != AOK_OK) return st;  // warm-up
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if ((st = cuda_status(cudaEventCreate(&e0), "cudaEventCreate")) != AOK_OK) return st;
    if ((st = cuda_status(cudaEventCreate(&e1), "cudaEventCreate")) != AOK_OK) {
        cudaEventDestroy(e0);
        return st;
    }
    constexpr int kReps = 5;
    float ms = 0.f;
    st = cuda_status(cudaEventRecord(e0, s), "cudaEventRecord");
    for (int r = 0; r < kReps && st == AOK_OK; ++r) st = launch();
    if (st == AOK_OK) st = cuda_status(cudaEventRecord(e1, s), "cudaEventRecord");
    if (st == AOK_OK) st = cuda_status(cudaEventSynchronize(e1), "cudaEventSynchronize");
    if (st == AOK_OK) st = cuda_status(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != AOK_OK) return st;
    const double flops = 2.0 * (paired && precision != AOK_PREC_F64 ? 2.0 : 1.0) * kChains * (double)kFmaIters *
                         kFmaThreads * (double)grid * kReps;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return AOK_OK;
}
