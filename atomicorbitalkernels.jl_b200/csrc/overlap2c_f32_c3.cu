// overlap2c_f32_c3.cu -- float instantiation of the 2-center overlap kernel,
// three CTAs per SM (bases of few primitives per shell).
#include "overlap2c_kernel.cuh"

namespace aok {

int launch_ov2_f32_c3(aok_plan* p, void* out, const void* posA, const void* posB, double lengthscale,
                      cudaStream_t s) {
    return launch_ov2<float, kThreadsF32, 3>(p, out, posA, posB, lengthscale, s);
}

}  // namespace aok
