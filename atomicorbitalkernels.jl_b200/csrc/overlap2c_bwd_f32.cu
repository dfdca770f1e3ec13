// overlap2c_bwd_f32.cu -- float instantiation of the 2C pullback kernel.
#include "overlap2c_bwd.cuh"

namespace aok {

int launch_pb_f32(aok_plan* p, void* out0, void* out1, const void* dS, const void* dS2, double alpha,
                  const void* zeta, const void* coef, const void* D, const void* posA, const void* posB,
                  double lengthscale, cudaStream_t s, unsigned* counter) {
    return launch_pb<float, kPbThreadsF32>(p, out0, out1, dS, dS2, alpha, zeta, coef, D, posA, posB,
                                                    lengthscale, s, counter);
}

}  // namespace aok
