// overlap3c_f32.cu -- float instantiation of the 3-center overlap kernel.
#include "overlap3c_kernel.cuh"

namespace aok {

int launch_ov3_f32(aok_plan* p, void* out, const void* posA, const void* posB, const void* posC, double lengthscale,
                   cudaStream_t s, bool pdl) {
    if (p->Lmax > kMaxL3Spec) return launch_ov3<float, true>(p, out, posA, posB, posC, lengthscale, s, pdl);
    return launch_ov3<float, false>(p, out, posA, posB, posC, lengthscale, s, pdl);
}

}  // namespace aok
