// overlap2c_f64_c2.cu -- double instantiation of the 2-center overlap kernel,
// two CTAs per SM (bases of few primitives per shell).
#include "overlap2c_kernel.cuh"

namespace aok {

int launch_ov2_f64_c2(aok_plan* p, void* out, const void* posA, const void* posB, double lengthscale,
                      cudaStream_t s) {
    return launch_ov2<double, kThreadsF64, 2>(p, out, posA, posB, lengthscale, s);
}

}  // namespace aok
