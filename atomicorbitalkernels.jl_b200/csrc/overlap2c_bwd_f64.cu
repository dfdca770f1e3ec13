// overlap2c_bwd_f64.cu -- double instantiation of the 2C pullback kernel.
#include "overlap2c_bwd.cuh"

namespace aok {

int launch_pb_f64(aok_plan* p, void* dcoef, void* dalpha, const void* dS, const void* zeta, const void* coef,
                  const void* posA, const void* posB,
                  double lengthscale, cudaStream_t s) {
    return launch_pb<double, kPbThreadsF64>(p, dcoef, dalpha, dS, zeta, coef, posA, posB, lengthscale, s);
}

}  // namespace aok
