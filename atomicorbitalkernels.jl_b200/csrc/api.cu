// api.cu -- the C ABI declared in include/aok.h: plans, validation, error
// reporting, and the entry points that chain the kernels on the caller's stream.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>

#include <map>
#include <tuple>
#include <mutex>
#include <string>

#include "aok_internal.h"

namespace aok {

int kernel_prepare(const void* k, size_t smem, int threads, int* occ) {
    static std::mutex mu;
    static std::map<std::tuple<int, const void*, int, size_t>, int> occs;
    static std::map<std::pair<int, const void*>, size_t> limit;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetDevice");
    std::lock_guard<std::mutex> lock(mu);
    const auto key = std::make_tuple(dev, k, threads, smem);
    const auto it = occs.find(key);
    if (it != occs.end()) {
        if (occ) *occ = it->second;
        return AOK_OK;
    }
    size_t& lim = limit[std::make_pair(dev, k)];
    if (smem > lim) {  // once per (device, kernel) and larger size
        if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess)
            return cuda_status(e, "cudaFuncSetAttribute");
        lim = smem;
    }
    int n = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, threads, smem)) != cudaSuccess)
        return cuda_status(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    occs[key] = n;
    if (occ) *occ = n;
    return AOK_OK;
}

}  // namespace aok


namespace aok {

static thread_local std::string g_last_error;

int set_error(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return AOK_OK;
    return set_error(AOK_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
static int dmalloc(T** p, size_t n, const char* what) {
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
    return cuda_status(e, what);
}

static int dmalloc_bytes(void** p, size_t n, const char* what) {
    if (n == 0) n = 16;
    cudaError_t e = cudaMalloc(p, n);
    return cuda_status(e, what);
}

static void dfree(void* p) {
    if (p) cudaFree(p);
}

void timing_begin(aok_plan* p, cudaStream_t s) {
    if (p->ev.empty() || 2 * p->ev_used + 1 >= (int)p->ev.size()) return;
    cudaEventRecord(p->ev[2 * p->ev_used], s);
}

void timing_end(aok_plan* p, cudaStream_t s) {
    if (p->ev.empty() || 2 * p->ev_used + 1 >= (int)p->ev.size()) return;
    cudaEventRecord(p->ev[2 * p->ev_used + 1], s);
    p->ev_used++;
}

}  // namespace aok

using namespace aok;

#define AOK_TRY(x)                      \
    do {                                \
        int _st = (x);                  \
        if (_st != AOK_OK) return _st;  \
    } while (0)

extern "C" {

const char* aok_last_error(void) { return g_last_error.c_str(); }

const char* aok_version(void) { return "aok_b200 0.1.0 (sm_100a)"; }

int aok_plan_create(aok_plan** plan, int64_t nshells, const int64_t* ls, int64_t K, int64_t NZ, int precision,
                    int64_t max_batch) {
    if (!plan || !ls) return set_error(AOK_ERR_INVALID, "aok_plan_create: null pointer");
    *plan = nullptr;
    if (nshells <= 0 || K <= 0 || NZ <= 0 || max_batch < 0)
        return set_error(AOK_ERR_INVALID, "aok_plan_create: nshells, K, NZ must be positive");
    if (precision != AOK_PREC_F64 && precision != AOK_PREC_F32C)
        return set_error(AOK_ERR_INVALID, "aok_plan_create: unknown precision");
    if (nshells > kMaxShells) return set_error(AOK_ERR_UNSUPPORTED, "aok_plan_create: more than 64 shells");
    if (NZ * NZ > 256) return set_error(AOK_ERR_UNSUPPORTED, "aok_plan_create: more than 16 species");
    if (K > 128) return set_error(AOK_ERR_UNSUPPORTED, "aok_plan_create: more than 128 primitives per shell");
    if (max_batch > (int64_t)0x7fffffff - 64)
        return set_error(AOK_ERR_UNSUPPORTED, "aok_plan_create: batch larger than 2^31");
    for (int64_t s = 0; s < nshells; ++s)
        if (ls[s] < 0 || ls[s] > AOK_MAX_L)
            return set_error(AOK_ERR_UNSUPPORTED,
                             "aok_plan_create: shell angular momentum outside 0..3 (compiled classes)");
    aok_plan* p = new aok_plan();
    p->ns = nshells;
    p->K = K;
    p->NZ = NZ;
    p->prec = precision;
    p->max_batch = max_batch;
    p->ls.assign(ls, ls + nshells);
    p->boff.assign(nshells + 1, 0);
    for (int64_t s = 0; s < nshells; ++s) {
        p->boff[s + 1] = p->boff[s] + ncart((int)ls[s]);
        p->Lmax = std::max(p->Lmax, (int)ls[s]);
    }
    p->N = p->boff[nshells];
    int st = AOK_OK;
    auto fail = [&](int code) {
        aok_plan_destroy(p);
        return code;
    };
    if ((st = cuda_status(cudaGetDevice(&p->device), "cudaGetDevice")) != AOK_OK) return fail(st);
    if ((st = cuda_status(cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, p->device),
                          "cudaDeviceGetAttribute")) != AOK_OK)
        return fail(st);
    const size_t fsz = precision == AOK_PREC_F64 ? sizeof(double) : sizeof(float);
    p->max_tiles = (int)((max_batch + kTileB - 1) / kTileB + bin_keys_max(NZ) + 1);
    std::vector<int> ls32(nshells), boff32(nshells + 1);
    for (int64_t s = 0; s < nshells; ++s) ls32[s] = (int)ls[s];
    for (int64_t s = 0; s <= nshells; ++s) boff32[s] = (int)p->boff[s];
    if ((st = dmalloc(&p->d_ls, nshells, "cudaMalloc(ls)")) ||
        (st = dmalloc(&p->d_boff, nshells + 1, "cudaMalloc(boff)")) ||
        (st = dmalloc(&p->d_perm, (size_t)max_batch, "cudaMalloc(perm)")) ||
        (st = dmalloc(&p->d_tiles, (size_t)p->max_tiles, "cudaMalloc(tiles)")) ||
        (st = dmalloc(&p->d_ntiles, 1, "cudaMalloc(ntiles)")) ||
        (st = dmalloc(&p->d_tbase, (size_t)(bin_keys_max(NZ) + 1), "cudaMalloc(tbase)")) ||
        (st = dmalloc(&p->d_counter, 2, "cudaMalloc(counter)")) ||
        (st = dmalloc(&p->d_err, 1, "cudaMalloc(err)")) ||
        (st = dmalloc_bytes(&p->d_gb_zeta, (size_t)(nshells * K) * fsz, "cudaMalloc(gb_zeta)")) ||
        (st = dmalloc_bytes(&p->d_gb_coef, (size_t)(nshells * K) * fsz, "cudaMalloc(gb_coef)")) ||
        (st = dmalloc_bytes(&p->d_coef_scratch, (size_t)(nshells * K * NZ) * fsz, "cudaMalloc(coef)")))
        return fail(st);
    if ((st = cuda_status(cudaMemcpy(p->d_ls, ls32.data(), sizeof(int) * nshells, cudaMemcpyHostToDevice),
                          "cudaMemcpy(ls)")) ||
        (st = cuda_status(cudaMemcpy(p->d_boff, boff32.data(), sizeof(int) * (nshells + 1), cudaMemcpyHostToDevice),
                          "cudaMemcpy(boff)")) ||
        (st = cuda_status(cudaMemset(p->d_err, 0, sizeof(int)), "cudaMemset(err)")))
        return fail(st);
    if ((st = setup_overlap2c_schedule(p)) != AOK_OK) return fail(st);
    if ((st = cuda_status(cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking), "cudaStreamCreate")) ||
        (st = cuda_status(cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming), "cudaEventCreate")) ||
        (st = cuda_status(cudaEventCreateWithFlags(&p->ev_join, cudaEventDisableTiming), "cudaEventCreate")))
        return fail(st);
    *plan = p;
    return AOK_OK;
}

int aok_plan_destroy(aok_plan* p) {
    if (!p) return AOK_OK;
    void* bufs[] = {p->d_ls,        p->d_boff,      p->d_perm,
                    p->d_tiles,     p->d_ntiles,    p->d_tbase,     p->d_counter,    p->d_err,
                    p->d_items,     p->d_blockhist, p->d_gb_zeta,    p->d_gb_coef,
                    p->d_pb_rec,    p->d_pb_counts, p->d_pb_items,  p->d_pb_itemidx, p->d_pb_rows,
                    p->d_partials,  p->d_coef_scratch, p->d_pp3,    p->d_npp3,       p->d_items3,    p->d_order3,    p->d_segs3,     p->d_key3,
                    p->d_pk,        p->d_segs,      p->d_nseg,      p->d_dpos_rec,   p->d_dpos_counts,
                    p->d_dpos_items};
    for (void* b : bufs) dfree(b);
    if (p->gexec) cudaGraphExecDestroy(p->gexec);
    if (p->cap) cudaStreamDestroy(p->cap);
    for (cudaEvent_t e : p->ev) cudaEventDestroy(e);
    if (p->ev_fork) cudaEventDestroy(p->ev_fork);
    if (p->ev_join) cudaEventDestroy(p->ev_join);
    if (p->ev_pb) cudaEventDestroy(p->ev_pb);
    if (p->side) cudaStreamDestroy(p->side);
    delete p;
    return AOK_OK;
}

int aok_plan_nbf(const aok_plan* p, int64_t* nbf_total) {
    if (!p || !nbf_total) return set_error(AOK_ERR_INVALID, "aok_plan_nbf: null pointer");
    *nbf_total = p->N;
    return AOK_OK;
}

int aok_plan_check(aok_plan* p, void* stream) {
    if (!p) return set_error(AOK_ERR_INVALID, "aok_plan_check: null plan");
    cudaStream_t s = (cudaStream_t)stream;
    AOK_TRY(cuda_status(cudaStreamSynchronize(s), "cudaStreamSynchronize"));
    int h = 0;
    AOK_TRY(cuda_status(cudaMemcpy(&h, p->d_err, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy(err)"));
    AOK_TRY(cuda_status(cudaMemset(p->d_err, 0, sizeof(int)), "cudaMemset(err)"));
    if (h == AOK_ERR_SPECIES) return set_error(h, "species index outside 1..NZ");
    if (h != 0) return set_error(h, "device-side validation failed");
    return AOK_OK;
}

int aok_plan_timing_enable(aok_plan* p, int capacity) {
    if (!p || capacity < 0) return set_error(AOK_ERR_INVALID, "aok_plan_timing_enable: bad argument");
    for (cudaEvent_t e : p->ev) cudaEventDestroy(e);
    p->ev.clear();
    p->ev_used = 0;
    for (int i = 0; i < 2 * capacity; ++i) {
        cudaEvent_t e;
        AOK_TRY(cuda_status(cudaEventCreate(&e), "cudaEventCreate"));
        p->ev.push_back(e);
    }
    return AOK_OK;
}

int aok_plan_timing_read(aok_plan* p, double* total_ms, int64_t* launches) {
    if (!p || !total_ms || !launches) return set_error(AOK_ERR_INVALID, "aok_plan_timing_read: null pointer");
    double tot = 0.0;
    for (int i = 0; i < p->ev_used; ++i) {
        AOK_TRY(cuda_status(cudaEventSynchronize(p->ev[2 * i + 1]), "cudaEventSynchronize"));
        float ms = 0.f;
        AOK_TRY(cuda_status(cudaEventElapsedTime(&ms, p->ev[2 * i], p->ev[2 * i + 1]), "cudaEventElapsedTime"));
        tot += ms;
    }
    *total_ms = tot;
    *launches = p->ev_used;
    p->ev_used = 0;
    return AOK_OK;
}

static int check_batch(aok_plan* p, int64_t B, const char* who) {
    if (B < 0) return set_error(AOK_ERR_INVALID, std::string(who) + ": negative batch");
    if (B > p->max_batch)
        return set_error(AOK_ERR_LENGTH, std::string(who) + ": batch exceeds the plan's max_batch");
    return AOK_OK;
}

// The fixed-basis forward from the plan's CUDA graph: captured on the plan's
// capture stream (thread-local mode), instantiated once, updated in place when
// the arguments change (re-instantiated if the update is refused), launched on
// the caller's stream.
static int overlap2c_graph(aok_plan* p, void* out, const void* posA, const void* posB, const int64_t* sidxA,
                           const int64_t* sidxB, int64_t B, double lengthscale, cudaStream_t s) {
    const aok_plan::GraphKey k{out, posA, posB, sidxA, sidxB, B, lengthscale};
    const aok_plan::GraphKey& o = p->gkey;
    const bool same = p->gexec && o.out == k.out && o.posA == k.posA && o.posB == k.posB && o.sidxA == k.sidxA &&
                      o.sidxB == k.sidxB && o.B == k.B && o.lengthscale == k.lengthscale;
    if (!same) {
        if (!p->cap) AOK_TRY(cuda_status(cudaStreamCreateWithFlags(&p->cap, cudaStreamNonBlocking), "cudaStreamCreate"));
        AOK_TRY(cuda_status(cudaStreamBeginCapture(p->cap, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture"));
        int st = launch_bin(p, sidxA, sidxB, B, p->cap);
        if (st == AOK_OK) st = launch_overlap2c(p, out, posA, posB, B, lengthscale, p->cap);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(p->cap, &g);
        if (st != AOK_OK || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return st != AOK_OK ? st : cuda_status(e, "cudaStreamEndCapture");
        }
        if (p->gexec) {
            cudaGraphExecUpdateResultInfo info;
            if (cudaGraphExecUpdate(p->gexec, g, &info) != cudaSuccess) {
                (void)cudaGetLastError();
                cudaGraphExecDestroy(p->gexec);
                p->gexec = nullptr;
            }
        }
        cudaError_t ei = cudaSuccess;
        if (!p->gexec) ei = cudaGraphInstantiate(&p->gexec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            p->gexec = nullptr;
            return cuda_status(ei, "cudaGraphInstantiate");
        }
        p->gkey = k;
    }
    ++p->gen;  // the replayed chain rebins
    return cuda_status(cudaGraphLaunch(p->gexec, s), "cudaGraphLaunch");
}

int aok_overlap2c(aok_plan* p, void* out, const void* zeta, const void* coef, const void* posA, const void* posB,
                  const int64_t* sidxA, const int64_t* sidxB, int64_t B, double lengthscale, void* stream) {
    if (!p) return set_error(AOK_ERR_INVALID, "aok_overlap2c: null plan");
    AOK_TRY(check_batch(p, B, "aok_overlap2c"));
    if (B == 0) return AOK_OK;
    if (!out || !posA || !posB || !sidxA || !sidxB || (!zeta) != (!coef))
        return set_error(AOK_ERR_INVALID, "aok_overlap2c: null pointer");
    cudaStream_t s = (cudaStream_t)stream;
    if (zeta && coef) {
        // record preparation on the side stream, concurrent with the binning
        p->basis_set = false;
        AOK_TRY(cuda_status(cudaEventRecord(p->ev_fork, s), "cudaEventRecord"));
        AOK_TRY(cuda_status(cudaStreamWaitEvent(p->side, p->ev_fork, 0), "cudaStreamWaitEvent"));
        AOK_TRY(launch_prep2c(p, zeta, coef, p->side));
        AOK_TRY(cuda_status(cudaEventRecord(p->ev_join, p->side), "cudaEventRecord"));
        AOK_TRY(launch_bin(p, sidxA, sidxB, B, s));
        AOK_TRY(cuda_status(cudaStreamWaitEvent(s, p->ev_join, 0), "cudaStreamWaitEvent"));
    } else {
        if (!p->basis_set) return set_error(AOK_ERR_INVALID, "aok_overlap2c: no zeta/coef and no aok_plan_set_basis");
        if (p->graph_on && p->ev.empty()) return overlap2c_graph(p, out, posA, posB, sidxA, sidxB, B, lengthscale, s);
        AOK_TRY(launch_bin(p, sidxA, sidxB, B, s));
    }
    return launch_overlap2c(p, out, posA, posB, B, lengthscale, s);
}

// Shapes chosen by aok_plan_autotune, per (precision, shells, K, NZ, non-zero
// coefficient pattern, B).
namespace {
struct TuneChoice {
    int ctas;
    size_t stage;
};
std::mutex g_tune_mu;
std::map<std::string, TuneChoice> g_tune_cache;
}  // namespace

int aok_plan_autotune(aok_plan* p, void* out, const void* zeta, const void* coef, const void* posA,
                      const void* posB, const int64_t* sidxA, const int64_t* sidxB, int64_t B, double lengthscale,
                      void* stream, int64_t* choice) {
    if (!p) return set_error(AOK_ERR_INVALID, "aok_plan_autotune: null plan");
    AOK_TRY(check_batch(p, B, "aok_plan_autotune"));
    if (!out || !zeta || !coef || !posA || !posB || !sidxA || !sidxB || B == 0)
        return set_error(AOK_ERR_INVALID, "aok_plan_autotune: null pointer or empty batch");
    cudaStream_t s = (cudaStream_t)stream;
    const bool f64 = p->prec == AOK_PREC_F64;
    // key: precision, shells, K, NZ, non-zero coefficient pattern, B
    const size_t nc = (size_t)(p->ns * p->K * p->NZ);
    std::vector<unsigned char> c(nc * (f64 ? 8 : 4));
    AOK_TRY(cuda_status(cudaMemcpyAsync(c.data(), coef, c.size(), cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync"));
    AOK_TRY(cuda_status(cudaStreamSynchronize(s), "cudaStreamSynchronize"));
    std::string key = std::to_string(p->prec) + "|" + std::to_string(p->K) + "|" + std::to_string(p->NZ) + "|" +
                      std::to_string(B) + "|";
    for (int64_t l : p->ls) key += (char)('0' + l);
    key += "|";
    for (size_t i = 0; i < nc; ++i) {
        const double v = f64 ? ((const double*)c.data())[i] : (double)((const float*)c.data())[i];
        key += v != 0.0 ? '1' : '0';
    }
    auto apply = [&](int ctas, size_t stage) -> int {
        AOK_TRY(setup_overlap2c_schedule(p, ctas, stage));
        AOK_TRY(launch_prep2c(p, zeta, coef, s));
        p->basis_set = true;
        return AOK_OK;
    };
    auto forward = [&]() -> int {
        AOK_TRY(launch_bin(p, sidxA, sidxB, B, s));
        return launch_overlap2c(p, out, posA, posB, B, lengthscale, s);
    };
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            AOK_TRY(apply(it->second.ctas, it->second.stage));
            AOK_TRY(forward());
            if (choice) {
                choice[0] = p->fwd_ctas;
                choice[1] = (int64_t)p->stage_bytes;
                choice[2] = 1;
            }
            return cuda_status(cudaStreamSynchronize(s), "cudaStreamSynchronize");
        }
    }
    std::vector<int> ctas = f64 ? std::vector<int>{1, 2} : std::vector<int>{2, 3};
    std::vector<size_t> stages = f64 ? std::vector<size_t>{48 * 1024, 80 * 1024}
                                     : std::vector<size_t>{24 * 1024, 40 * 1024};
    std::vector<cudaEvent_t> ev0(p->ev);
    p->ev.clear();  // direct launches, no measurement events of the plan
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int st = cuda_status(cudaEventCreate(&e0), "cudaEventCreate");
    if (st == AOK_OK) st = cuda_status(cudaEventCreate(&e1), "cudaEventCreate");
    float best = -1.f;
    TuneChoice bestc{0, 0};
    for (int ct : ctas)
        for (size_t sb : stages) {
            if (st != AOK_OK) break;
            if (apply(ct, sb) != AOK_OK) continue;  // shape does not fit this basis
            if (forward() != AOK_OK || forward() != AOK_OK) continue;
            // the faster of two timed batches of kReps forwards
            constexpr int kReps = 6;
            float ms = -1.f;
            for (int round = 0; round < 2 && st == AOK_OK; ++round) {
                st = cuda_status(cudaEventRecord(e0, s), "cudaEventRecord");
                for (int r = 0; r < kReps && st == AOK_OK; ++r) st = forward();
                if (st == AOK_OK) st = cuda_status(cudaEventRecord(e1, s), "cudaEventRecord");
                if (st == AOK_OK) st = cuda_status(cudaEventSynchronize(e1), "cudaEventSynchronize");
                float t = 0.f;
                if (st == AOK_OK) st = cuda_status(cudaEventElapsedTime(&t, e0, e1), "cudaEventElapsedTime");
                if (st == AOK_OK && (ms < 0.f || t < ms)) ms = t;
            }
            if (st == AOK_OK && (best < 0.f || ms < best)) {
                best = ms;
                bestc = TuneChoice{p->fwd_ctas, p->stage_bytes};
            }
        }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    p->ev = ev0;
    if (st != AOK_OK || best < 0.f) {  // leave the plan with its default shape
        const int st2 = setup_overlap2c_schedule(p);
        p->basis_set = false;
        if (st != AOK_OK) return st;
        if (st2 != AOK_OK) return st2;
        return set_error(AOK_ERR_UNSUPPORTED, "aok_plan_autotune: no launch shape fits this basis");
    }
    AOK_TRY(apply(bestc.ctas, bestc.stage));
    AOK_TRY(forward());
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[key] = bestc;
    }
    if (choice) {
        choice[0] = p->fwd_ctas;
        choice[1] = (int64_t)p->stage_bytes;
        choice[2] = 0;
    }
    return cuda_status(cudaStreamSynchronize(s), "cudaStreamSynchronize");
}

int aok_plan_set_graph(aok_plan* p, int enable) {
    if (!p) return set_error(AOK_ERR_INVALID, "aok_plan_set_graph: null plan");
    p->graph_on = enable != 0;
    return AOK_OK;
}

int aok_plan_set_basis(aok_plan* p, const void* zeta, const void* coef, void* stream) {
    if (!p || !zeta || !coef) return set_error(AOK_ERR_INVALID, "aok_plan_set_basis: null pointer");
    AOK_TRY(launch_prep2c(p, zeta, coef, (cudaStream_t)stream));
    p->basis_set = true;
    return AOK_OK;
}

int aok_overlap2c_gb(aok_plan* p, void* out, const int64_t* nprim, const int64_t* prim_offset, const void* coef,
                     const void* alpha, const void* posA, const void* posB, int64_t B, void* stream) {
    if (!p) return set_error(AOK_ERR_INVALID, "aok_overlap2c_gb: null plan");
    if (p->NZ != 1) return set_error(AOK_ERR_INVALID, "aok_overlap2c_gb: plan must have NZ = 1");
    AOK_TRY(check_batch(p, B, "aok_overlap2c_gb"));
    if (B == 0) return AOK_OK;
    if (!out || !nprim || !prim_offset || !coef || !alpha || !posA || !posB)
        return set_error(AOK_ERR_INVALID, "aok_overlap2c_gb: null pointer");
    cudaStream_t s = (cudaStream_t)stream;
    p->basis_set = false;
    AOK_TRY(launch_gb_pad(p, nprim, prim_offset, coef, alpha, s));
    AOK_TRY(launch_prep2c(p, p->d_gb_zeta, p->d_gb_coef, s));
    AOK_TRY(launch_bin(p, nullptr, nullptr, B, s));
    return launch_overlap2c(p, out, posA, posB, B, 1.0, s);
}

static int overlap2c_pullback(aok_plan* p, void* out0, void* out1, const void* dS, const void* zeta,
                              const void* coef, const void* D, const void* posA, const void* posB,
                              const int64_t* sidxA, const int64_t* sidxB, int64_t B, double lengthscale,
                              int keep_absent, void* stream, const char* who) {
    AOK_TRY(check_batch(p, B, who));
    cudaStream_t s = (cudaStream_t)stream;
    const size_t fsz = p->prec == AOK_PREC_F64 ? sizeof(double) : sizeof(float);
    if (B == 0) {  // no pairs: zero gradients
        AOK_TRY(cuda_status(cudaMemsetAsync(out0, 0, fsz * p->ns * p->K * p->NZ, s), "cudaMemsetAsync"));
        return cuda_status(cudaMemsetAsync(out1, 0, fsz * p->ns * p->K * p->NZ, s), "cudaMemsetAsync");
    }
    if (!dS || !posA || !posB || !sidxA || !sidxB)
        return set_error(AOK_ERR_INVALID, std::string(who) + ": null pointer");
    return launch_overlap2c_pb(p, out0, out1, dS, zeta, coef, D, sidxA, sidxB, posA, posB, B, lengthscale,
                               keep_absent, s);
}

int aok_overlap2c_pullback(aok_plan* p, void* dcoef, void* dalpha, const void* dS, const void* zeta,
                           const void* coef, const void* posA, const void* posB, const int64_t* sidxA,
                           const int64_t* sidxB, int64_t B, double lengthscale, void* stream) {
    if (!p) return set_error(AOK_ERR_INVALID, "aok_overlap2c_pullback: null plan");
    if (!dcoef || !dalpha || !zeta || !coef) return set_error(AOK_ERR_INVALID, "aok_overlap2c_pullback: null pointer");
    return overlap2c_pullback(p, dcoef, dalpha, dS, zeta, coef, nullptr, posA, posB, sidxA, sidxB, B, lengthscale, 1,
                              stream, "aok_overlap2c_pullback");
}

int aok_overlap2c_position_pullback(aok_plan* p, void* dA, void* dB, const void* dS, const void* zeta,
                                    const void* coef, const void* posA, const void* posB, const int64_t* sidxA,
                                    const int64_t* sidxB, int64_t B, double lengthscale, void* stream) {
    static const char* who = "aok_overlap2c_position_pullback";
    if (!p) return set_error(AOK_ERR_INVALID, std::string(who) + ": null plan");
    if (!dA && !dB) return set_error(AOK_ERR_INVALID, std::string(who) + ": dA and dB are both null");
    AOK_TRY(check_batch(p, B, who));
    if (B == 0) return AOK_OK;
    if (!dS || !zeta || !coef || !posA || !posB || !sidxA || !sidxB)
        return set_error(AOK_ERR_INVALID, std::string(who) + ": null pointer");
    return launch_overlap2c_dpos(p, dA, dB, dS, zeta, coef, sidxA, sidxB, posA, posB, B, lengthscale,
                                 (cudaStream_t)stream);
}

int aok_overlap2c_rrule(aok_plan* p, void* out, const void* zeta, const void* D, const void* posA, const void* posB,
                        const int64_t* sidxA, const int64_t* sidxB, int64_t B, double lengthscale, void* stream) {
    if (!p) return set_error(AOK_ERR_INVALID, "aok_overlap2c_rrule: null plan");
    AOK_TRY(check_batch(p, B, "aok_overlap2c_rrule"));
    p->rgen = 0;
    if (B == 0) return AOK_OK;
    if (!out || !zeta || !D || !posA || !posB || !sidxA || !sidxB)
        return set_error(AOK_ERR_INVALID, "aok_overlap2c_rrule: null pointer");
    cudaStream_t s = (cudaStream_t)stream;
    AOK_TRY(ensure_pb_buffers(p));
    if (!p->ev_pb)
        AOK_TRY(cuda_status(cudaEventCreateWithFlags(&p->ev_pb, cudaEventDisableTiming), "cudaEventCreate"));
    p->basis_set = false;
    void* coef = p->d_coef_scratch;
    // side stream: coef, the forward records, then (while the overlap kernel runs) the pullback records
    AOK_TRY(cuda_status(cudaEventRecord(p->ev_fork, s), "cudaEventRecord"));
    AOK_TRY(cuda_status(cudaStreamWaitEvent(p->side, p->ev_fork, 0), "cudaStreamWaitEvent"));
    AOK_TRY(launch_compile_coef(p, coef, zeta, D, p->side));
    AOK_TRY(launch_prep2c(p, zeta, coef, p->side, true));
    AOK_TRY(cuda_status(cudaEventRecord(p->ev_join, p->side), "cudaEventRecord"));
    // the pullback kernel's work counter (the forward kernel uses the first one)
    AOK_TRY(cuda_status(cudaMemsetAsync(p->d_counter + 1, 0, sizeof(unsigned), p->side), "cudaMemsetAsync"));
    AOK_TRY(launch_prep_pb(p, zeta, coef, 0, p->side));
    AOK_TRY(cuda_status(cudaEventRecord(p->ev_pb, p->side), "cudaEventRecord"));
    AOK_TRY(launch_bin(p, sidxA, sidxB, B, s));
    AOK_TRY(cuda_status(cudaStreamWaitEvent(s, p->ev_join, 0), "cudaStreamWaitEvent"));
    AOK_TRY(launch_overlap2c(p, out, posA, posB, B, lengthscale, s));
    p->rkey = aok_plan::RruleKey{zeta, D, posA, posB, sidxA, sidxB, B, lengthscale};
    p->rgen = p->gen;
    return AOK_OK;
}

// The rrule pullback with the cotangent dS, or alpha (dS - dS2) when dS2 is given.
static int pullback_ps_rrule(aok_plan* p, void* dzeta, void* dD, const void* dS, const void* dS2, double alpha,
                             const void* zeta, const void* D, const void* posA, const void* posB,
                             const int64_t* sidxA, const int64_t* sidxB, int64_t B, double lengthscale, void* stream,
                             const char* who) {
    if (!p) return set_error(AOK_ERR_INVALID, std::string(who) + ": null plan");
    if (!dzeta || !dD || !zeta || !D) return set_error(AOK_ERR_INVALID, std::string(who) + ": null pointer");
    AOK_TRY(check_batch(p, B, who));
    cudaStream_t s = (cudaStream_t)stream;
    if (B == 0) {
        const size_t fsz = p->prec == AOK_PREC_F64 ? sizeof(double) : sizeof(float);
        AOK_TRY(cuda_status(cudaMemsetAsync(dD, 0, fsz * p->ns * p->K * p->NZ, s), "cudaMemsetAsync"));
        return cuda_status(cudaMemsetAsync(dzeta, 0, fsz * p->ns * p->K * p->NZ, s), "cudaMemsetAsync");
    }
    if (!dS || !posA || !posB || !sidxA || !sidxB) return set_error(AOK_ERR_INVALID, std::string(who) + ": null pointer");
    const aok_plan::RruleKey& k = p->rkey;
    const bool match = p->rgen != 0 && p->rgen == p->gen && k.zeta == zeta && k.D == D && k.posA == posA &&
                       k.posB == posB && k.sidxA == sidxA && k.sidxB == sidxB && k.B == B &&
                       k.lengthscale == lengthscale;
    if (!match)
        return set_error(AOK_ERR_INVALID, std::string(who) + ": no matching aok_overlap2c_rrule on this plan "
                                                             "(other arguments, or another 2C call in between)");
    return launch_pb_prepared(p, dD, dzeta, dS, dS2, alpha, zeta, D, posA, posB, lengthscale, s);
}

int aok_overlap_pullback_ps_rrule(aok_plan* p, void* dzeta, void* dD, const void* dS, const void* zeta,
                                  const void* D, const void* posA, const void* posB, const int64_t* sidxA,
                                  const int64_t* sidxB, int64_t B, double lengthscale, void* stream) {
    return pullback_ps_rrule(p, dzeta, dD, dS, nullptr, 1.0, zeta, D, posA, posB, sidxA, sidxB, B, lengthscale,
                             stream, "aok_overlap_pullback_ps_rrule");
}

int aok_overlap_pullback_ps_rrule_residual(aok_plan* p, void* dzeta, void* dD, const void* S, const void* T,
                                           double alpha, const void* zeta, const void* D, const void* posA,
                                           const void* posB, const int64_t* sidxA, const int64_t* sidxB, int64_t B,
                                           double lengthscale, void* stream) {
    static const char* who = "aok_overlap_pullback_ps_rrule_residual";
    if (B > 0 && (!S || !T)) return set_error(AOK_ERR_INVALID, std::string(who) + ": null pointer");
    return pullback_ps_rrule(p, dzeta, dD, S, T, alpha, zeta, D, posA, posB, sidxA, sidxB, B, lengthscale, stream,
                             who);
}

int aok_overlap_pullback_ps(aok_plan* p, void* dzeta, void* dD, const void* dS, const void* zeta, const void* D,
                            const void* posA, const void* posB, const int64_t* sidxA, const int64_t* sidxB,
                            int64_t B, double lengthscale, void* stream) {
    if (!p) return set_error(AOK_ERR_INVALID, "aok_overlap_pullback_ps: null plan");
    if (!dzeta || !dD || !zeta || !D) return set_error(AOK_ERR_INVALID, "aok_overlap_pullback_ps: null pointer");
    return overlap2c_pullback(p, dD, dzeta, dS, zeta, nullptr, D, posA, posB, sidxA, sidxB, B, lengthscale, 0, stream,
                              "aok_overlap_pullback_ps");
}

}  // extern "C"
