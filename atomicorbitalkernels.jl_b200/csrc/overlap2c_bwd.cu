// overlap2c_bwd.cu -- pullback host side: record lists, buffers, dispatch to
// the per-precision kernels (overlap2c_bwd_f32.cu, overlap2c_bwd_f64.cu).
#include "overlap2c_bwd.cuh"

namespace aok {

// Work assignment of one species pair to the NW warps of a pullback CTA: the
// items sorted by class (heavy first, so the warps run the same code at about
// the same time) and estimated cost, then assigned greedily to the least
// loaded warp (longest-processing-time rule).  Deterministic: ties go to the
// lower warp.  out: the pair's items grouped by warp, in sorted order;
// woff: NW + 1 offsets.
__device__ __forceinline__ int pb_item_cost(int cls, int4 n) {
    const int la = cls >> 2, lb = cls & 3, nv = md_nv(la, lb);
    const int full = n.x * n.y, val = n.z * n.y + n.w * n.x;
    if (full + val == 0) return 8;
    return 100 + 5 * md_terms(la, lb) / 2 + full * (45 + 12 * nv) + val * (30 + 4 * nv);
}

__global__ void __launch_bounds__(256) k_pb_assign(Item* __restrict__ out, int* __restrict__ woff,
                                                   const Item* __restrict__ items, const int4* __restrict__ counts,
                                                   int nitems, int ns) {
    __shared__ unsigned long long key[kAssignMax];
    __shared__ short sorted[kAssignMax];
    __shared__ unsigned char owner[kAssignMax];
    __shared__ int cost[kAssignMax];
    const int pair = blockIdx.x;
    const int n = min(nitems, kAssignMax);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const Item it = items[i];
        const int c = pb_item_cost(it.cls, counts[((size_t)pair * ns + it.sa) * ns + it.sb]);
        cost[i] = c;
        const int la = it.cls >> 2, lb = it.cls & 3;
        key[i] = ((unsigned long long)(0xFFFF - md_terms(la, lb)) << 48) |
                 ((unsigned long long)(0x7FFFFFFF - c) << 16) | (unsigned long long)it.cls;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const unsigned long long ki = key[i];
        int r = 0;
        for (int j = 0; j < n; ++j) {
            const unsigned long long kj = key[j];
            r += (kj < ki) || (kj == ki && j < i);
        }
        sorted[r] = (short)i;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        long long load[kPbWarps];  // fully unrolled: stays in registers
#pragma unroll
        for (int v = 0; v < kPbWarps; ++v) load[v] = 0;
        for (int r = 0; r < n; ++r) {
            int w = 0;
            long long best = load[0];
#pragma unroll
            for (int v = 1; v < kPbWarps; ++v)
                if (load[v] < best) {
                    best = load[v];
                    w = v;
                }
            owner[r] = (unsigned char)w;
            const int c = cost[sorted[r]];
#pragma unroll
            for (int v = 0; v < kPbWarps; ++v)
                if (v == w) load[v] += c;
        }
    }
    __syncthreads();
    if (threadIdx.x < kPbWarps) {
        const int w = threadIdx.x;
        int before = 0, pos = 0;
        for (int r = 0; r < n; ++r) before += owner[r] < w;
        woff[pair * (kPbWarps + 1) + w] = before;
        if (w == kPbWarps - 1) woff[pair * (kPbWarps + 1) + kPbWarps] = n;
        Item* o = out + (size_t)pair * nitems + before;
        for (int r = 0; r < n; ++r)
            if (owner[r] == w) o[pos++] = items[sorted[r]];
    }
}


int launch_prep_pb(aok_plan* p, const void* zeta, const void* coef, int keep_absent, cudaStream_t s) {
    const int n = (int)(p->NZ * p->NZ * p->ns * p->ns);
    const int bl = (n + kPrepPbWarps - 1) / kPrepPbWarps;
    const size_t sm = (size_t)kPrepPbWarps * 4 * p->K;
    if (p->prec == AOK_PREC_F64)
        k_prep_pb<double><<<bl, 32 * kPrepPbWarps, sm, s>>>((PBd*)p->d_pb_rec, p->d_pb_counts, (const double*)zeta,
                                                            (const double*)coef, (int)p->ns, (int)p->K, (int)p->NZ,
                                                            keep_absent);
    else
        k_prep_pb<float><<<bl, 32 * kPrepPbWarps, sm, s>>>((PBf*)p->d_pb_rec, p->d_pb_counts, (const float*)zeta,
                                                           (const float*)coef, (int)p->ns, (int)p->K, (int)p->NZ,
                                                           keep_absent);
    AOK_TRY_PB(cuda_status(cudaGetLastError(), "k_prep_pb"));
    if (p->nitems > kAssignMax) return set_error(AOK_ERR_UNSUPPORTED, "pullback: too many shell pairs");
    k_pb_assign<<<(int)(p->NZ * p->NZ), 256, 0, s>>>(p->d_pb_order, p->d_pb_woff, p->d_items, p->d_pb_counts,
                                                    p->nitems, (int)p->ns);
    return cuda_status(cudaGetLastError(), "k_pb_assign");
}

int ensure_pb_buffers(aok_plan* p) {
    if (p->d_pb_rec) return AOK_OK;
    const size_t npair = (size_t)(p->NZ * p->NZ * p->ns * p->ns);
    const size_t rec = p->prec == AOK_PREC_F64 ? sizeof(PBd) : sizeof(PBf);
    const int NW = (p->prec == AOK_PREC_F64 ? kPbThreadsF64 : kPbThreadsF32) / 32;
    cudaError_t e;
    if ((e = cudaMalloc(&p->d_pb_rec, npair * p->K * p->K * rec)) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(pb_rec)");
    if ((e = cudaMalloc(&p->d_pb_counts, sizeof(int4) * npair)) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(pb_counts)");
    if ((e = cudaMalloc(&p->d_pb_order, sizeof(Item) * p->nitems * p->NZ * p->NZ)) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(pb_order)");
    if ((e = cudaMalloc(&p->d_pb_woff, sizeof(int) * (kPbWarps + 1) * p->NZ * p->NZ)) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(pb_woff)");
    // warp rows in global memory (used only when they do not fit in shared memory)
    const size_t ctas = (size_t)p->num_sms * (p->prec == AOK_PREC_F64 ? 1 : 2);
    if ((e = cudaMalloc(&p->d_partials, sizeof(double) * 4 * p->ns * p->K * (size_t)NW * ctas)) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(pb_rows)");
    const size_t fsz = p->prec == AOK_PREC_F64 ? sizeof(double) : sizeof(float);
    if ((e = cudaMalloc(&p->d_pb_zeros, fsz * p->N * p->N)) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(pb_zeros)");
    if ((e = cudaMemset(p->d_pb_zeros, 0, fsz * p->N * p->N)) != cudaSuccess)
        return cuda_status(e, "cudaMemset(pb_zeros)");
    if ((e = cudaMalloc(&p->d_tilerows, sizeof(double) * 4 * p->ns * p->K * (size_t)p->max_tiles)) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(tilerows)");
    return AOK_OK;
}

int launch_overlap2c_pb(aok_plan* p, void* dcoef, void* dalpha, const void* dS, const void* zeta, const void* coef,
                        const void* posA, const void* posB, int64_t B, double lengthscale, int keep_absent,
                        cudaStream_t s) {
    (void)B;
    AOK_TRY_PB(ensure_pb_buffers(p));
    AOK_TRY_PB(launch_prep_pb(p, zeta, coef, keep_absent, s));
    if (p->prec == AOK_PREC_F64) return launch_pb_f64(p, dcoef, dalpha, dS, zeta, coef, posA, posB, lengthscale, s);
    return launch_pb_f32(p, dcoef, dalpha, dS, zeta, coef, posA, posB, lengthscale, s);
}

}  // namespace aok
