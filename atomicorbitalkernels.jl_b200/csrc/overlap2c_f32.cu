// overlap2c_f32.cu -- float instantiation of the 2-center overlap kernel,
// two CTAs per SM (three: overlap2c_f32_c3.cu).
#include "overlap2c_kernel.cuh"

namespace aok {

int launch_ov2_f32_c3(aok_plan* p, void* out, const void* posA, const void* posB, double lengthscale,
                      cudaStream_t s);

int launch_ov2_f32(aok_plan* p, void* out, const void* posA, const void* posB, double lengthscale,
                   cudaStream_t s) {
    if (p->fwd_ctas == 3) return launch_ov2_f32_c3(p, out, posA, posB, lengthscale, s);
    return launch_ov2<float, kThreadsF32, 2>(p, out, posA, posB, lengthscale, s);
}

}  // namespace aok
