// overlap2c_bwd_f32.cu -- float instantiation of the 2C pullback kernel.
#include "overlap2c_bwd.cuh"

namespace aok {

int launch_pb_f32(aok_plan* p, void* dcoef, void* dalpha, const void* dS, const void* zeta, const void* coef,
                  const void* posA, const void* posB,
                  double lengthscale, cudaStream_t s) {
    return launch_pb<float, kPbThreadsF32>(p, dcoef, dalpha, dS, zeta, coef, posA, posB, lengthscale, s);
}

}  // namespace aok
