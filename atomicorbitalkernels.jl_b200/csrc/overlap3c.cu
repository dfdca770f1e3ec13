// overlap3c.cu -- 3-center overlap host side: primitive-triple records, the
// item list, and the aok_overlap3c_gb entry point.  The kernel is in
// overlap3c_kernel.cuh (one instantiation per precision: overlap3c_f32.cu,
// overlap3c_f64.cu).
#include <algorithm>
#include <cstring>
#include <vector>

#include "overlap3c_kernel.cuh"

namespace aok {

__device__ __forceinline__ void fill_pt(PTf& r, double ca, double cb, double cc, double a, double b, double c, int grp) {
    const double q = a + b + c, x = 3.14159265358979323846 / q, l2e = 1.4426950408889634074;
    const double kab = a * b / q * l2e, kac = a * c / q * l2e, kbc = b * c / q * l2e;
    r.w = (float)(ca * cb * cc * (x * sqrt(x)));
    r.kab_hi = (float)kab;
    r.kab_lo = (float)(kab - (double)r.kab_hi);
    r.kac_hi = (float)kac;
    r.kac_lo = (float)(kac - (double)r.kac_hi);
    r.kbc_hi = (float)kbc;
    r.kbc_lo = (float)(kbc - (double)r.kbc_hi);
    r.ra = (float)(a / q);
    r.rb = (float)(b / q);
    r.rc = (float)(c / q);
    r.oo2q = (float)(0.5 / q);
    r.grp = (float)grp;
}
__device__ __forceinline__ void fill_pt(PTd& r, double ca, double cb, double cc, double a, double b, double c, int) {
    const double q = a + b + c, x = 3.14159265358979323846 / q;
    r.w = ca * cb * cc * (x * sqrt(x));
    r.kab = a * b / q;
    r.kac = a * c / q;
    r.kbc = b * c / q;
    r.ra = a / q;
    r.rb = b / q;
    r.rc = c / q;
    r.oo2q = 0.5 / q;
}

// One warp per shell triple; lanes sweep the K^3 grid in (ip, jp, kp) order
// and compact the non-zero-coefficient triples (ballot), preserving order.
template <typename FT>
__global__ void k_prep3c(typename PTT<FT>::type* __restrict__ pp, int* __restrict__ npp, const FT* __restrict__ zeta,
                         const FT* __restrict__ coef, int ns, int K) {
    const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (q >= ns * ns * ns) return;
    const int sc = q % ns, sb = (q / ns) % ns, sa = q / (ns * ns);
    auto* out = pp + (size_t)q * K * K * K;
    int n = 0;
    const int K3 = K * K * K;
    for (int e0 = 0; e0 < K3; e0 += 32) {
        const int e = e0 + lane;
        const int ip = e / (K * K), jp = (e / K) % K, kp = e % K;
        double ca = 0, cb = 0, cc = 0, a = 1, b = 1, c = 1;
        if (e < K3) {
            ca = (double)coef[sa + ns * ip];
            cb = (double)coef[sb + ns * jp];
            cc = (double)coef[sc + ns * kp];
            a = (double)zeta[sa + ns * ip];
            b = (double)zeta[sb + ns * jp];
            c = (double)zeta[sc + ns * kp];
        }
        const bool valid = e < K3 && ca != 0.0 && cb != 0.0 && cc != 0.0;
        const unsigned m = __ballot_sync(0xffffffffu, valid);
        if (valid) fill_pt(out[n + __popc(m & ((1u << lane) - 1u))], ca, cb, cc, a, b, c, ip * K + jp);
        n += __popc(m);
    }
    if (lane == 0) npp[q] = n;
}

// Per call, one CTA: the items sorted by estimated cost, heaviest first, so
// that the kernel's unit queue (item-major) ends with cheap items.  Cost =
// primitive triples x (E tables + the chunk's products) + a fixed part per
// item; the f-shell classes (run-time loops, FP64 tables) count four times.
// Rank sort in shared memory; more than kOrder3Max items keep the static order.
constexpr int kOrder3Max = 2048;

__global__ void __launch_bounds__(256) k_order3c(Item3* __restrict__ order, const Item3* __restrict__ items,
                                                 const int* __restrict__ npp, int n, int ns) {
    __shared__ unsigned long long key[kOrder3Max];
    if (n > kOrder3Max) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) order[i] = items[i];
        return;
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const Item3 it = items[i];
        const bool f = it.cls >= kClsF3;
        const int c = f ? it.cls - kClsF3 : it.cls;
        const int la = f ? c >> 4 : c / 9, lb = f ? (c >> 2) & 3 : (c / 3) % 3, lc = f ? c & 3 : c % 3;
        const int ppc = pages_per_chunk3(la, lb);
        const int pages = min(ppc, ncart(lc) - it.chunk * ppc);
        const long long per = 12LL * (la + 1) * (lb + 1) * (lc + 1) + 2LL * ncart(la) * ncart(lb) * pages;
        long long cost = (long long)npp[(it.sa * ns + it.sb) * ns + it.sc] * per * (f ? 4 : 1) + 64;
        cost = min(cost, (long long)0x7FFFFFFF);
        key[i] = ((unsigned long long)(0x7FFFFFFF - cost) << 32) | (unsigned)i;  // ascending key = descending cost
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const unsigned long long ki = key[i];
        int r = 0;
        for (int j = 0; j < n; ++j) r += key[j] < ki;
        order[r] = items[i];
    }
}

int setup_overlap3c_schedule(aok_plan* p) {
    if (p->d_items3) return AOK_OK;
    if (p->NZ != 1) return set_error(AOK_ERR_INVALID, "aok_overlap3c_gb: plan must have NZ = 1");
    if (p->Lmax > kMaxL3) return set_error(AOK_ERR_UNSUPPORTED, "aok_overlap3c_gb: shells above l = 3");
    const int ns = (int)p->ns;
    // every (shell triple, page chunk), statically ordered by class cost
    std::vector<std::pair<int, Item3>> v;
    for (int sc = 0; sc < ns; ++sc)
        for (int sa = 0; sa < ns; ++sa)
            for (int sb = 0; sb < ns; ++sb) {
                const int la = (int)p->ls[sa], lb = (int)p->ls[sb], lc = (int)p->ls[sc];
                const int ppc = pages_per_chunk3(la, lb), nch = nchunks3(la, lb, lc);
                for (int c = 0; c < nch; ++c) {
                    const int pages = std::min(ppc, ncart(lc) - c * ppc);
                    const int cost = (la + 1) * (lb + 1) * (lc + 1) * 12 + 2 * ncart(la) * ncart(lb) * pages;
                    const bool f = std::max(la, std::max(lb, lc)) > kMaxL3Spec;
                    const int cls = f ? kClsF3 + la * 16 + lb * 4 + lc : la * 9 + lb * 3 + lc;
                    v.push_back({f ? 4 * cost : cost,
                                 Item3{(int16_t)cls, (int16_t)c, (int16_t)sa, (int16_t)sb, (int16_t)sc, 0}});
                }
            }
    std::stable_sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    std::vector<Item3> items;
    for (auto& x : v) items.push_back(x.second);
    p->nitems3 = (int)items.size();
    const size_t nrec = (size_t)ns * ns * ns * p->K * p->K * p->K;
    const size_t rec = p->prec == AOK_PREC_F64 ? sizeof(PTd) : sizeof(PTf);
    cudaError_t e;
    if ((e = cudaMalloc(&p->d_items3, sizeof(Item3) * items.size())) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(items3)");
    if ((e = cudaMalloc(&p->d_order3, sizeof(Item3) * items.size())) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(order3)");
    if ((e = cudaMemcpy(p->d_items3, items.data(), sizeof(Item3) * items.size(), cudaMemcpyHostToDevice)) !=
        cudaSuccess)
        return cuda_status(e, "cudaMemcpy(items3)");
    if ((e = cudaMalloc(&p->d_pp3, nrec * rec)) != cudaSuccess) return cuda_status(e, "cudaMalloc(pp3)");
    if ((e = cudaMalloc(&p->d_npp3, sizeof(int) * (size_t)ns * ns * ns)) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(npp3)");
    return AOK_OK;
}

int launch_overlap3c(aok_plan* p, void* out, const void* posA, const void* posB, const void* posC, int64_t B,
                     cudaStream_t s) {
    (void)B;
    const int n = (int)(p->ns * p->ns * p->ns), th = 128, bl = (n * 32 + th - 1) / th;
    if (p->prec == AOK_PREC_F64)
        k_prep3c<double><<<bl, th, 0, s>>>((PTd*)p->d_pp3, p->d_npp3, (const double*)p->d_gb_zeta,
                                           (const double*)p->d_gb_coef, (int)p->ns, (int)p->K);
    else
        k_prep3c<float><<<bl, th, 0, s>>>((PTf*)p->d_pp3, p->d_npp3, (const float*)p->d_gb_zeta,
                                          (const float*)p->d_gb_coef, (int)p->ns, (int)p->K);
    int st = cuda_status(cudaGetLastError(), "k_prep3c");
    if (st != AOK_OK) return st;
    k_order3c<<<1, 256, 0, s>>>((Item3*)p->d_order3, (const Item3*)p->d_items3, p->d_npp3, p->nitems3, (int)p->ns);
    if ((st = cuda_status(cudaGetLastError(), "k_order3c")) != AOK_OK) return st;
    if (p->prec == AOK_PREC_F64) return launch_ov3_f64(p, out, posA, posB, posC, s);
    return launch_ov3_f32(p, out, posA, posB, posC, s);
}

}  // namespace aok

using namespace aok;

extern "C" int aok_overlap3c_gb(aok_plan* p, void* out, const int64_t* nprim, const int64_t* prim_offset,
                                const void* coef, const void* alpha, const void* posA, const void* posB,
                                const void* posC, int64_t B, void* stream) {
    if (!p) return set_error(AOK_ERR_INVALID, "aok_overlap3c_gb: null plan");
    if (B < 0) return set_error(AOK_ERR_INVALID, "aok_overlap3c_gb: negative batch");
    if (B > p->max_batch) return set_error(AOK_ERR_LENGTH, "aok_overlap3c_gb: batch exceeds the plan's max_batch");
    int st = setup_overlap3c_schedule(p);
    if (st != AOK_OK) return st;
    if (B == 0) return AOK_OK;
    if (!out || !nprim || !prim_offset || !coef || !alpha || !posA || !posB || !posC)
        return set_error(AOK_ERR_INVALID, "aok_overlap3c_gb: null pointer");
    cudaStream_t s = (cudaStream_t)stream;
    if ((st = launch_gb_pad(p, nprim, prim_offset, coef, alpha, s)) != AOK_OK) return st;
    if ((st = launch_bin(p, nullptr, nullptr, B, s)) != AOK_OK) return st;
    return launch_overlap3c(p, out, posA, posB, posC, B, s);
}
