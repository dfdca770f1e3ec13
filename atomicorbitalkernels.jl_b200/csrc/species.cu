// species.cu -- species labels -> species-axis indices on the device, replacing the
// host lookup _cgto_species_index / _cgto_sidx (src/integrals/orbital/overlap_2c.jl:148-158)
// so that a batch's labels need no host round trip before the 2C kernels.
#include "aok_internal.h"

namespace aok {

struct SpeciesList {
    int64_t z[kMaxPairs];  // the plan's species labels in order (NZ <= 16 in practice)
    int n;
};

__global__ void k_species_index(int64_t* __restrict__ sidx, const int64_t* __restrict__ label, int64_t n,
                                const __grid_constant__ SpeciesList zl, int* err) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t s = label[i];
    int64_t sigma = 0;  // first match, 1-based (0: not in the list)
    for (int k = 0; k < zl.n; ++k)
        if (zl.z[k] == s) {
            sigma = k + 1;
            break;
        }
    if (sigma == 0) atomicCAS(err, 0, AOK_ERR_SPECIES);
    sidx[i] = sigma;
}

}  // namespace aok

using namespace aok;

extern "C" int aok_species_index(aok_plan* p, int64_t* sidx, const int64_t* label, int64_t n,
                                 const int64_t* zlist, void* stream) {
    if (!p) return set_error(AOK_ERR_INVALID, "aok_species_index: null plan");
    if (n < 0) return set_error(AOK_ERR_INVALID, "aok_species_index: negative length");
    if (n == 0) return AOK_OK;
    if (!sidx || !label || !zlist) return set_error(AOK_ERR_INVALID, "aok_species_index: null pointer");
    if (p->NZ > kMaxPairs) return set_error(AOK_ERR_UNSUPPORTED, "aok_species_index: too many species");
    SpeciesList zl{};
    zl.n = (int)p->NZ;
    for (int k = 0; k < zl.n; ++k) zl.z[k] = zlist[k];
    const int th = 256;
    const int64_t bl = (n + th - 1) / th;
    k_species_index<<<(unsigned)bl, th, 0, (cudaStream_t)stream>>>(sidx, label, n, zl, p->d_err);
    return cuda_status(cudaGetLastError(), "k_species_index");
}
