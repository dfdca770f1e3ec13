// overlap2c_bwd.cu -- pullback host side: record lists, buffers, dispatch to
// the per-precision kernels (overlap2c_bwd_f32.cu, overlap2c_bwd_f64.cu).
#include <algorithm>
#include <vector>

#include "overlap2c_bwd.cuh"

namespace aok {

int launch_prep_pb(aok_plan* p, const void* zeta, const void* coef, int keep_absent, cudaStream_t s) {
    ++p->gen;  // the pullback records change
    const int n = (int)(p->NZ * p->NZ * p->ns * p->ns);
    const int bl = (n + kPrepPbWarps - 1) / kPrepPbWarps;
    const size_t sm = (size_t)kPrepPbWarps * 4 * p->K;
    if (p->prec == AOK_PREC_F64)
        k_prep_pb<double><<<bl, 32 * kPrepPbWarps, sm, s>>>(
            (PBd*)p->d_pb_rec, p->d_pb_counts, (const double*)zeta, (const double*)coef, (int)p->ns, (int)p->K,
            (int)p->NZ, keep_absent);
    else
        k_prep_pb<float><<<bl, 32 * kPrepPbWarps, sm, s>>>(
            (PBf*)p->d_pb_rec, p->d_pb_counts, (const float*)zeta, (const float*)coef, (int)p->ns, (int)p->K,
            (int)p->NZ, keep_absent);
    return cuda_status(cudaGetLastError(), "k_prep_pb");
}

int ensure_pb_buffers(aok_plan* p) {
    if (p->d_pb_rec) return AOK_OK;
    const int ns = (int)p->ns;
    const size_t npair = (size_t)(p->NZ * p->NZ * ns * ns);
    const size_t rec = p->prec == AOK_PREC_F64 ? sizeof(PBd) : sizeof(PBf);
    cudaError_t e;
    if ((e = cudaMalloc(&p->d_pb_rec, npair * p->K * p->K * rec)) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(pb_rec)");
    if ((e = cudaMalloc(&p->d_pb_counts, sizeof(int4) * npair)) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(pb_counts)");
    // static item list (one item per shell pair), heaviest classes first
    std::vector<std::pair<int, Item>> v;
    for (int sa = 0; sa < ns; ++sa)
        for (int sb = 0; sb < ns; ++sb) {
            const int la = (int)p->ls[sa], lb = (int)p->ls[sb];
            v.push_back({md_terms(la, lb), Item{(int16_t)(la * 4 + lb), 0, (int16_t)sa, (int16_t)sb}});
        }
    std::stable_sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    std::vector<Item> items;
    std::vector<int> idx((size_t)ns * ns);
    for (size_t i = 0; i < v.size(); ++i) {
        items.push_back(v[i].second);
        idx[(size_t)v[i].second.sa * ns + v[i].second.sb] = (int)i;
    }
    if ((e = cudaMalloc(&p->d_pb_items, sizeof(Item) * items.size())) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(pb_items)");
    if ((e = cudaMemcpy(p->d_pb_items, items.data(), sizeof(Item) * items.size(), cudaMemcpyHostToDevice)) !=
        cudaSuccess)
        return cuda_status(e, "cudaMemcpy(pb_items)");
    if ((e = cudaMalloc(&p->d_pb_itemidx, sizeof(int) * idx.size())) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(pb_itemidx)");
    if ((e = cudaMemcpy(p->d_pb_itemidx, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice)) !=
        cudaSuccess)
        return cuda_status(e, "cudaMemcpy(pb_itemidx)");
    // unit partials: chunks (each species pair rounds up) x items x record groups x 4 x K
    const size_t nch = (size_t)(p->max_tiles + kPbChunkTiles - 1) / kPbChunkTiles + (size_t)(p->NZ * p->NZ);
    const size_t gmax = (size_t)((p->K * p->K + 31) / 32);
    if (nch * items.size() * gmax >= ((size_t)1 << 31))
        return set_error(AOK_ERR_UNSUPPORTED, "pullback: too many work units (batch x shell pairs)");
    if ((e = cudaMalloc(&p->d_partials, sizeof(double) * nch * items.size() * gmax * 4 * p->K)) != cudaSuccess)
        return cuda_status(e, "cudaMalloc(pb_partials)");
    if ((e = cudaMalloc(&p->d_pb_rows, sizeof(double) * (size_t)(p->NZ * p->NZ) * items.size() * 4 * p->K)) !=
        cudaSuccess)
        return cuda_status(e, "cudaMalloc(pb_rows)");
    return AOK_OK;
}

// The pullback after argument checks: the record lists (for the parameter
// pullback after compiling the coefficients from D) are built on the plan's
// side stream while the batch is binned on the caller's stream; then the
// record-parallel kernel and its reductions.  D == nullptr: kernel-level
// pullback (out0, out1) = (dcoef, dalpha) from `coef`; otherwise
// (out0, out1) = (dD, dzeta) and `coef` is ignored.
int launch_overlap2c_pb(aok_plan* p, void* out0, void* out1, const void* dS, const void* zeta, const void* coef,
                        const void* D, const int64_t* sidxA, const int64_t* sidxB, const void* posA,
                        const void* posB, int64_t B, double lengthscale, int keep_absent, cudaStream_t s) {
    AOK_TRY_PB(ensure_pb_buffers(p));
    if (D) coef = p->d_coef_scratch;
    AOK_TRY_PB(cuda_status(cudaEventRecord(p->ev_fork, s), "cudaEventRecord"));
    AOK_TRY_PB(cuda_status(cudaStreamWaitEvent(p->side, p->ev_fork, 0), "cudaStreamWaitEvent"));
    if (D) AOK_TRY_PB(launch_compile_coef(p, p->d_coef_scratch, zeta, D, p->side));
    AOK_TRY_PB(launch_prep_pb(p, zeta, coef, keep_absent, p->side));
    AOK_TRY_PB(cuda_status(cudaEventRecord(p->ev_join, p->side), "cudaEventRecord"));
    AOK_TRY_PB(launch_bin(p, sidxA, sidxB, B, s));
    AOK_TRY_PB(cuda_status(cudaStreamWaitEvent(s, p->ev_join, 0), "cudaStreamWaitEvent"));
    if (p->prec == AOK_PREC_F64)
        return launch_pb_f64(p, out0, out1, dS, nullptr, 1.0, zeta, coef, D, posA, posB, lengthscale, s,
                             p->d_counter);
    return launch_pb_f32(p, out0, out1, dS, nullptr, 1.0, zeta, coef, D, posA, posB, lengthscale, s,
                         p->d_counter);
}

// The pullback of an rrule forward (aok_overlap2c_rrule): its bins and its
// pullback records (prepared on the side stream, ev_pb) are reused; its kernel
// claims units from the plan's second work counter, which the rrule forward reset
// on the side stream (the first one is the forward kernel's).  The cotangent is dS, or
// alpha (dS - dS2) when dS2 is given.
int launch_pb_prepared(aok_plan* p, void* out0, void* out1, const void* dS, const void* dS2, double alpha,
                       const void* zeta, const void* D, const void* posA, const void* posB, double lengthscale,
                       cudaStream_t s) {
    AOK_TRY_PB(cuda_status(cudaStreamWaitEvent(s, p->ev_pb, 0), "cudaStreamWaitEvent"));
    if (p->prec == AOK_PREC_F64)
        return launch_pb_f64(p, out0, out1, dS, dS2, alpha, zeta, p->d_coef_scratch, D, posA, posB, lengthscale,
                             s, p->d_counter + 1);
    return launch_pb_f32(p, out0, out1, dS, dS2, alpha, zeta, p->d_coef_scratch, D, posA, posB, lengthscale, s,
                         p->d_counter + 1);
}

}  // namespace aok
