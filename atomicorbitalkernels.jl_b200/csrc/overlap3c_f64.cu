// overlap3c_f64.cu -- double instantiation of the 3-center overlap kernel.
#include "overlap3c_kernel.cuh"

namespace aok {

int launch_ov3_f64(aok_plan* p, void* out, const void* posA, const void* posB, const void* posC, double lengthscale,
                   cudaStream_t s, bool pdl) {
    if (p->Lmax > kMaxL3Spec) return launch_ov3<double, true>(p, out, posA, posB, posC, lengthscale, s, pdl);
    return launch_ov3<double, false>(p, out, posA, posB, posC, lengthscale, s, pdl);
}

}  // namespace aok
