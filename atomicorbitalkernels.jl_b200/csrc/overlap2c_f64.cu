// overlap2c_f64.cu -- double instantiation of the 2-center overlap kernel,
// one CTA per SM (two: overlap2c_f64_c2.cu).
#include "overlap2c_kernel.cuh"

namespace aok {

int launch_ov2_f64_c2(aok_plan* p, void* out, const void* posA, const void* posB, double lengthscale,
                      cudaStream_t s);

int launch_ov2_f64(aok_plan* p, void* out, const void* posA, const void* posB, double lengthscale,
                   cudaStream_t s) {
    if (p->fwd_ctas == 2) return launch_ov2_f64_c2(p, out, posA, posB, lengthscale, s);
    return launch_ov2<double, kThreadsF64, 1>(p, out, posA, posB, lengthscale, s);
}

}  // namespace aok
