// aok_internal.h -- host-side plan objects and kernel launchers (not part of the ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "aok.h"
#include "aok_common.cuh"

struct aok_plan {
    int64_t ns = 0, K = 0, NZ = 0, N = 0, max_batch = 0;
    int Lmax = 0;
    int prec = AOK_PREC_F64;
    int device = 0;
    int num_sms = 0;
    std::vector<int64_t> ls, boff;
    // shell tables on the device
    int* d_ls = nullptr;             // ns
    int* d_boff = nullptr;           // ns+1
    // species-pair bins: permutation, tiles, tile count, work counter
    int* d_perm = nullptr;
    int4* d_tiles = nullptr;
    int* d_ntiles = nullptr;
    int* d_tbase = nullptr;          // first tile of each species pair (NZ*NZ + 1)
    unsigned* d_counter = nullptr;   // work counters: [0] binning-reset kernels, [1] the rrule pullback
    int max_tiles = 0;
    // device error word (AOK_ERR_* of the first fault a kernel met)
    int* d_err = nullptr;
    // 2C forward schedule
    aok::Item* d_items = nullptr;    // static item list (nitems), panel-major
    int nitems = 0;
    // stage images of the forward kernel (k_pack2c): packed chunks and segments
    void* d_pk = nullptr;            // NZ*NZ regions of pair16 16-byte words
    aok::Seg* d_segs = nullptr;      // NZ*NZ regions of seg_stride segments
    int* d_nseg = nullptr;           // segments per species pair
    int pair16 = 0, seg_stride = 0;
    size_t stage_bytes = 0;          // shared-memory stage of the forward kernel
    int fwd_ctas = 2;                // forward kernel CTAs per SM
    // multi-block binning scratch
    int* d_blockhist = nullptr;      // nblk * NZ*NZ
    int max_bin_blocks = 0;
    aok::Panels panels{};
    size_t slab_stride = 0;          // elements per batch slot in the panel buffer
    size_t smem_bytes = 0;
    // GaussianBasis-path padded tables (ns*K)
    void* d_gb_zeta = nullptr;
    void* d_gb_coef = nullptr;
    // pullback: primitive-pair lists, per-warp FP64 partial rows, scratch coef
    void* d_pb_rec = nullptr;        // pullback records: per (species pair, shell pair) K*K
    int4* d_pb_counts = nullptr;     // (na, nb, nza, nzb) per (species pair, shell pair)
    aok::Item* d_pb_items = nullptr; // pullback items (one per shell pair), heaviest classes first
    int* d_pb_itemidx = nullptr;     // (sa, sb) -> position in d_pb_items
    void* d_pb_rows = nullptr;       // per (species pair, item): unit sums (FP64, 4*K)
    void* d_partials = nullptr;      // per-CTA item sums
    int max_blocks = 0;
    void* d_coef_scratch = nullptr;  // ns*K*NZ
    // position pullback (overlap2c_dpos.cu): records per (species pair, shell pair), their
    // counts, and the shell-pair list heaviest class first
    void* d_dpos_rec = nullptr;
    int* d_dpos_counts = nullptr;
    aok::Item* d_dpos_items = nullptr;
    // 3C schedule (overlap3c.cu)
    void* d_pp3 = nullptr;
    int* d_npp3 = nullptr;
    void* d_items3 = nullptr;
    void* d_order3 = nullptr;        // per call: the items in queue order (k_prep3c)
    int* d_segs3 = nullptr;          // per call: segment starts in d_order3 (nitems3 + 1), then the count
    int* d_key3 = nullptr;           // what d_order3/d_segs3 were built from: (n, tiles, target, counts)
    int nitems3 = 0;
    // graph mode of the fixed-basis forward (aok_plan_set_graph): the instantiated
    // launch chain, the arguments it was captured with, a private capture stream
    bool graph_on = false;
    cudaGraphExec_t gexec = nullptr;
    cudaStream_t cap = nullptr;
    struct GraphKey {
        void* out;
        const void *posA, *posB;
        const int64_t *sidxA, *sidxB;
        int64_t B;
        double lengthscale;
    } gkey{};
    // rrule state (aok_overlap2c_rrule -> aok_overlap_pullback_ps_rrule): the
    // arguments of the forward, the generation of the plan's bins and pullback
    // records it left, and the event after its pullback-record preparation
    struct RruleKey {
        const void *zeta, *D, *posA, *posB;
        const int64_t *sidxA, *sidxB;
        int64_t B;
        double lengthscale;
    } rkey{};
    uint64_t gen = 0;        // bumped by every call that rebins or rebuilds pullback records
    uint64_t rgen = 0;       // the generation an rrule forward left (0: none)
    cudaEvent_t ev_pb = nullptr;
    // side stream for the record preparation (forked/joined with events)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    bool basis_set = false;          // records fixed by aok_plan_set_basis
    // optional event pairs around the dominant kernel (measurement aid)
    std::vector<cudaEvent_t> ev;
    int ev_used = 0;
};

struct aok_orbitals {
    int64_t nRad = 0, K = 0, NZ = 0, nOrb = 0;
    int L = 0;
    int radial = AOK_RADIAL_GAUSSIAN;
    int prec = AOK_PREC_F64;
    int device = 0;
    int num_sms = 0;
    std::vector<int64_t> poly, iR, iY;
    int* d_poly = nullptr;
    int* d_iR = nullptr;
    int* d_iY = nullptr;
    void* d_partials = nullptr;
    int max_blocks = 0;
    int* d_err = nullptr;
    // slot-parallel pullback: points binned by species, unit partial rows
    int64_t epb_ucap = 0;
    void* d_epb_partial = nullptr;
};

namespace aok {

#define AOK_TRY_PB(x)                  \
    do {                               \
        int _st = (x);                 \
        if (_st != AOK_OK) return _st; \
    } while (0)

// error helpers (api.cu)
int set_error(int code, const std::string& msg);
int cuda_status(cudaError_t e, const char* what);

// timing aid (api.cu): record the pair's first/second event on `s`
void timing_begin(aok_plan* p, cudaStream_t s);
void timing_end(aok_plan* p, cudaStream_t s);

// launchers (overlap2c.cu)
// pdl: launched with programmatic serialisation after k_compile_coef on the same stream
int launch_prep2c(aok_plan* p, const void* zeta, const void* coef, cudaStream_t s, bool pdl = false);

// Launch of `k` with programmatic stream serialisation (see pdl_wait / pdl_trigger).
template <typename... Exp, typename... Act>
cudaError_t launch_pdl(void (*k)(Exp...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Act&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, static_cast<Act&&>(args)...);
}
// Counting sort of a batch by species key (stable), tiles of 32 elements of
// one key, and the first tile of each key.  Buffers: perm (B), tiles
// (B/32 + NZ^2 + 1), tbase (NZ^2 + 1), blockhist (kBinMaxBlocksHost * NZ^2).
// An element with a species index outside 1..NZ sets *err and is left out of
// the bins; when zero3 (zero3b) is set, its three values zero3[3b..3b+2]
// (elements of zero3_bytes bytes, e.g. a position gradient) are written as zeros.
struct BinBufs {
    int* perm;
    int4* tiles;
    int* ntiles;
    int* tbase;
    unsigned* counter;
    int* blockhist;
    int* err;
    void* zero3 = nullptr;
    void* zero3b = nullptr;
    int zero3_bytes = 0;
};
constexpr int kBinMaxBlocksHost = 512;
int launch_bin_into(const BinBufs& bb, const int64_t* sidxA, const int64_t* sidxB, int64_t B, int NZ,
                    cudaStream_t s);
int launch_bin(aok_plan* p, const int64_t* sidxA, const int64_t* sidxB, int64_t B, cudaStream_t s);
// Binning by species triple (sidxC given): keys ((a-1) NZ + (b-1)) NZ + (c-1), NZ^3 <= 256.
int launch_bin3_into(const BinBufs& bb, const int64_t* sidxA, const int64_t* sidxB, const int64_t* sidxC,
                     int64_t B, int NZ, cudaStream_t s);
// Keys a plan's bin buffers are sized for: species triples when NZ^3 fits the
// binning's 256 keys (the species-aware 3C overlap), species pairs otherwise.
inline int64_t bin_keys_max(int64_t NZ) { return NZ * NZ * NZ <= 256 ? NZ * NZ * NZ : NZ * NZ; }
int launch_pb_prepared(aok_plan* p, void* out0, void* out1, const void* dS, const void* dS2, double alpha,
                       const void* zeta, const void* D, const void* posA, const void* posB, double lengthscale,
                       cudaStream_t s);
int ensure_pb_buffers(aok_plan* p);
int launch_overlap2c_dpos(aok_plan* p, void* dA, void* dB, const void* dS, const void* zeta, const void* coef,
                          const int64_t* sidxA, const int64_t* sidxB, const void* posA, const void* posB, int64_t B,
                          double lengthscale, cudaStream_t s);
int launch_prep_pb(aok_plan* p, const void* zeta, const void* coef, int keep_absent, cudaStream_t s);
int launch_overlap2c(aok_plan* p, void* out, const void* posA, const void* posB, int64_t B,
                     double lengthscale, cudaStream_t s);
int launch_gb_pad(aok_plan* p, const int64_t* nprim, const int64_t* prim_offset, const void* coef,
                  const void* alpha, cudaStream_t s);
// ctas = 0, stage_req = 0: the defaults (see overlap2c.cu).
int setup_overlap2c_schedule(aok_plan* p, int ctas = 0, size_t stage_req = 0);
int launch_ov2_f32(aok_plan* p, void* out, const void* posA, const void* posB, double lengthscale, cudaStream_t s);
int launch_ov2_f64(aok_plan* p, void* out, const void* posA, const void* posB, double lengthscale, cudaStream_t s);

// compile_coef.cu
int launch_compile_coef(aok_plan* p, void* coef, const void* zeta, const void* D, cudaStream_t s);
int launch_compile_coef_pb(aok_plan* p, void* dD, void* dzeta, const void* dcoef, const void* zeta,
                           const void* D, const void* dalpha_add, cudaStream_t s);

// overlap2c_bwd*.cu
int launch_pb_f32(aok_plan* p, void* out0, void* out1, const void* dS, const void* dS2, double alpha,
                  const void* zeta, const void* coef, const void* D, const void* posA, const void* posB,
                  double lengthscale, cudaStream_t s, unsigned* counter);
int launch_pb_f64(aok_plan* p, void* out0, void* out1, const void* dS, const void* dS2, double alpha,
                  const void* zeta, const void* coef, const void* D, const void* posA, const void* posB,
                  double lengthscale, cudaStream_t s, unsigned* counter);
int launch_overlap2c_pb(aok_plan* p, void* out0, void* out1, const void* dS, const void* zeta, const void* coef,
                        const void* D, const int64_t* sidxA, const int64_t* sidxB, const void* posA,
                        const void* posB, int64_t B, double lengthscale, int keep_absent, cudaStream_t s);

// api.cu: a kernel's dynamic shared-memory limit (raised when a launch needs more
// than the default) and its resident blocks per SM for (threads, smem bytes) on the
// current device (occ may be null).  Both are kept per (device, kernel, threads,
// smem), so a repeated launch shape costs one map lookup instead of driver calls.
int kernel_prepare(const void* k, size_t smem, int threads, int* occ);

// overlap3c.cu
int setup_overlap3c_schedule(aok_plan* p);
// pdl: launched with programmatic serialisation after the prep on the same stream
int launch_ov3_f32(aok_plan* p, void* out, const void* posA, const void* posB, const void* posC, double lengthscale,
                   cudaStream_t s, bool pdl);
int launch_ov3_f64(aok_plan* p, void* out, const void* posA, const void* posB, const void* posC, double lengthscale,
                   cudaStream_t s, bool pdl);

// orbitals.cu
int launch_evaluate(aok_orbitals* o, void* P, void* dP, const void* X, const int64_t* sidx,
                    const void* zeta, const void* D, int64_t nX, double lengthscale, cudaStream_t s);
int launch_evaluate_pb(aok_orbitals* o, void* dX, void* dzeta, void* dD, const void* dP,
                       const void* X, const int64_t* sidx, const void* zeta, const void* D,
                       int64_t nX, double lengthscale, cudaStream_t s);

}  // namespace aok
