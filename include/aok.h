/*
 * aok.h -- C ABI of libaok_b200.so, the sm_100a kernels behind the
 * AtomicOrbitalKernels.jl hot path (v0.0.4 API).
 *
 * Every entry point takes plain device pointers and sizes, runs stream-ordered
 * on the caller's cudaStream_t (passed as void*, NULL = legacy default
 * stream), never synchronises the device, never aborts, throws or prints, and
 * returns an int status (AOK_OK = 0).  On failure aok_last_error() returns a
 * thread-local message.  The caller owns every array; a plan owns only its
 * scratch tables (primitive-pair lists, the species-pair bins, the work-queue
 * counter) and the device error word.
 *
 * Layouts are the reference's column-major (Julia) layouts:
 *   positions (3,B)                  pos[c + 3*b]
 *   2C output (N,N,B)                out[i + N*(j + N*b)]
 *   3C output (N,N,N,B)              out[i + N*(j + N*(k + N*b))]
 *   per-species tables (ns,K,NZ)     t[s + ns*(k + K*sigma)]
 *   orbital values (nX,nOrb)         P[j + nX*i]
 *   orbital gradients (3,nX,nOrb)    dP[c + 3*(j + nX*i)]   (SVector{3} per entry)
 *   species indices                  int64, 1-based (as produced in Julia)
 * The element type of every floating-point array is double for
 * AOK_PREC_F64 and float for AOK_PREC_F32C.
 */
#ifndef AOK_H
#define AOK_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AOK_OK 0
#define AOK_ERR_INVALID 1      /* null pointer, negative size, bad enum       */
#define AOK_ERR_UNSUPPORTED 2  /* angular momentum / size beyond the kernels   */
#define AOK_ERR_CUDA 3         /* CUDA runtime error (message has the detail)  */
#define AOK_ERR_SPECIES 4      /* species index outside 1..NZ                  */
#define AOK_ERR_LENGTH 5       /* inconsistent lengths                         */
#define AOK_ERR_TIMEOUT 6      /* a bounded device-side wait gave up           */

#define AOK_PREC_F64 0         /* all-FP64 kernels                             */
#define AOK_PREC_F32C 1        /* FP32 arithmetic, compensated accumulation    */

#define AOK_RADIAL_GAUSSIAN 0  /* R = sum D exp(-zeta r^2)                     */
#define AOK_RADIAL_SLATER 1    /* R = r^poly sum D exp(-zeta r)                */

#define AOK_MAX_L 3            /* highest shell angular momentum compiled      */

typedef struct aok_plan aok_plan;        /* overlap plan (2C and 3C)          */
typedef struct aok_orbitals aok_orbitals;/* orbital-evaluation plan           */
typedef struct aok_radials aok_radials;  /* radial-layer plan                 */

/* Thread-local message for the last failing call on this thread (no reference
 * counterpart: the Julia extension raises error(aok_last_error()) with it). */
const char* aok_last_error(void);
/* Library version string (no reference counterpart). */
const char* aok_version(void);

/*
 * Overlap plan for a shell structure shared by all species: ls[nshells]
 * (host array) and K primitive slots per shell, NZ species.  Mirrors the
 * param-free part of compile_basis, _compile_struct
 * (src/integrals/orbital/cartesian_gto_basis.jl:88-104) and, with NZ = 1 and
 * K = max nprim, CompiledBasis (src/integrals/compiled_basis.jl:36-99).
 * max_batch bounds B for the 2C entry points (scratch is sized by it).
 */
int aok_plan_create(aok_plan** plan, int64_t nshells, const int64_t* ls, int64_t K,
                    int64_t NZ, int precision, int64_t max_batch);
int aok_plan_destroy(aok_plan* plan);
/* nbf_total of the plan's shell structure (basis.nbf_total,
 * src/integrals/orbital/cartesian_gto_basis.jl:42). */
int aok_plan_nbf(const aok_plan* plan, int64_t* nbf_total);
/* Synchronises `stream`, then reports (and clears) the plan's device error
 * word: AOK_ERR_SPECIES if a kernel met a species index outside 1..NZ.  The
 * device half of the unknown-species error of _cgto_species_index
 * (src/integrals/orbital/overlap_2c.jl:148-154). */
int aok_plan_check(aok_plan* plan, void* stream);
/* Measurement aid (no reference counterpart): when enabled, every call
 * records a CUDA event pair around its dominant kernel (up to `capacity`
 * pairs); aok_plan_timing_read synchronises those events and returns the
 * summed kernel time and the number of timed launches, then resets. */
int aok_plan_timing_enable(aok_plan* plan, int capacity);
int aok_plan_timing_read(aok_plan* plan, double* total_ms, int64_t* launches);
/* Measurement aid (no reference counterpart): the FMA-pipe throughput of the
 * current GPU in TFLOP/s, FP32 (precision AOK_PREC_F32C; paired != 0 uses the
 * paired FP32 FMA) or FP64, from a kernel of independent FMA chains on every SM
 * timed with CUDA events on `stream` (synchronises it).  The denominator for
 * the pipe use of compute-bound kernels. */
int aok_measure_fma_peak(int precision, int paired, double* tflops, void* stream);

/*
 * coef = D / sqrt(normsq) per shell and species on the device.
 * Replaces _compile_coef / _cart_normsq
 * (src/integrals/orbital/cartesian_gto_basis.jl:74-83, 110-120).
 * zeta, D, coef: (ns,K,NZ).
 */
int aok_compile_coef(aok_plan* plan, void* coef, const void* zeta, const void* D, void* stream);

/*
 * Fixes the plan's basis parameters: the geometry-free primitive-pair records
 * (and their execution order) are computed once from zeta, coef (ns,K,NZ) and
 * kept in the plan.  This is the device half of compile_basis
 * (src/integrals/orbital/cartesian_gto_basis.jl:138-146): later aok_overlap2c
 * calls given zeta = coef = NULL use these records, as batch_overlap! uses a
 * compiled CartesianGTOBasis.  Calling it again replaces the parameters.
 */
int aok_plan_set_basis(aok_plan* plan, const void* zeta, const void* coef, void* stream);
/*
 * Graph mode for a fixed basis (no reference counterpart; the launch form of
 * batch_overlap! on a compiled basis).  enable != 0: aok_overlap2c calls with
 * zeta = coef = NULL replay their launch chain (species-pair binning + the
 * overlap kernel) from one instantiated CUDA graph per plan, captured on the
 * first call and re-captured (graph update) when out, the positions, the
 * species indices, B or lengthscale change.  While timing is enabled
 * (aok_plan_timing_enable) calls launch directly.  Default: disabled.
 */
int aok_plan_set_graph(aok_plan* plan, int enable);
/*
 * Autotuner of the 2C forward's launch shape (no reference counterpart).  Times
 * aok_overlap2c on these inputs under each candidate shape (CTAs per SM; size
 * of the shared-memory record stage, which trades against the output slab),
 * keeps the fastest in the plan, and caches it process-wide under (precision,
 * shell structure, K, NZ, pattern of non-zero coefficients, B): a later call
 * with the same key applies the cached shape without timing.  Leaves the basis
 * fixed as aok_plan_set_basis(zeta, coef) does and out holding the forward.
 * Synchronises `stream`.  choice (may be NULL) receives {CTAs per SM, stage
 * bytes, 1 if taken from the cache else 0}.
 */
int aok_plan_autotune(aok_plan* plan, void* out, const void* zeta, const void* coef,
                      const void* posA, const void* posB, const int64_t* sidxA,
                      const int64_t* sidxB, int64_t B, double lengthscale, void* stream,
                      int64_t* choice);

/*
 * Batched 2-center overlap, species-aware Cartesian basis.
 * Replaces batch_S_orbital_kernel! + batch_overlap!(out, ::CartesianGTOBasis, XA, XB)
 * (src/integrals/orbital/overlap_2c.jl:15-131, 171-197).
 * out (N,N,B); zeta, coef (ns,K,NZ); posA, posB (3,B) in the basis's input
 * unit (multiplied by lengthscale on the device, overlap_2c.jl:184-185);
 * sidxA, sidxB (B) 1-based.  Zero-coefficient primitive pairs are skipped.
 * zeta = coef = NULL uses the parameters fixed by aok_plan_set_basis.
 */
int aok_overlap2c(aok_plan* plan, void* out, const void* zeta, const void* coef,
                  const void* posA, const void* posB, const int64_t* sidxA,
                  const int64_t* sidxB, int64_t B, double lengthscale, void* stream);
/*
 * Species labels -> 1-based species indices on the device.  Replaces the host
 * lookup _cgto_species_index / _cgto_sidx (src/integrals/orbital/overlap_2c.jl:148-158):
 * sidx[i] = first k + 1 with zlist[k] == label[i].  label, sidx: device int64 (n);
 * zlist: host int64 (the plan's NZ labels in basis order).  A label not in the
 * list gets 0 and sets the plan's error word (AOK_ERR_SPECIES from
 * aok_plan_check), as the 2C entry points do for an index outside 1..NZ.
 */
int aok_species_index(aok_plan* plan, int64_t* sidx, const int64_t* label, int64_t n,
                      const int64_t* zlist, void* stream);

/*
 * Batched 2-center overlap, GaussianBasis path (NZ = 1 plan, K = max nprim).
 * Replaces batch_S_kernel! + batch_overlap!(out, ::CompiledBasis, posA, posB)
 * (src/integrals/kernels_2c.jl:11-163).  nprim (ns), prim_offset (ns+1):
 * device int64; coef, alpha: flat per-primitive (prim_offset[ns]); posA,
 * posB (3,B) already in Bohr (the reference's to_bohr runs on the host,
 * src/integrals/units.jl:28-35).
 */
int aok_overlap2c_gb(aok_plan* plan, void* out, const int64_t* nprim,
                     const int64_t* prim_offset, const void* coef, const void* alpha,
                     const void* posA, const void* posB, int64_t B, void* stream);

/*
 * Batched 3-center overlap, GaussianBasis path (NZ = 1 plan).
 * Replaces batch_V_kernel! + batch_overlap_3c! (src/integrals/kernels_3c.jl:12-200).
 * out (N,N,N,B); posA, posB, posC (3,B) in Bohr.  Shells up to l = 3, at most
 * 64 shells; no limit on N beyond the output's size.
 */
int aok_overlap3c_gb(aok_plan* plan, void* out, const int64_t* nprim,
                     const int64_t* prim_offset, const void* coef, const void* alpha,
                     const void* posA, const void* posB, const void* posC, int64_t B,
                     void* stream);
/*
 * Batched 3-center overlap on the species-aware (orbital) path: no reference
 * counterpart (the reference computes the 3C overlap for a CompiledBasis only,
 * src/integrals/kernels_3c.jl:183-222, and lists the orbital-path 3C overlap as
 * not implemented).  Centre A of element b uses species sidxA[b] (1-based), and
 * so on, with the padded (ns,K,NZ) zeta, coef of aok_overlap2c and its
 * zero-coefficient skip; positions (3,B) times lengthscale.  out (N,N,N,B) in
 * the reference's aliased 3C block layout.  NZ^3 <= 256 (at most 6 species);
 * elements are binned by species triple.  A species index outside 1..NZ sets
 * the plan's error word (aok_plan_check) and the element's slab is not written.
 */
int aok_overlap3c(aok_plan* plan, void* out, const void* zeta, const void* coef, const void* posA,
                  const void* posB, const void* posC, const int64_t* sidxA, const int64_t* sidxB,
                  const int64_t* sidxC, int64_t B, double lengthscale, void* stream);

/*
 * Kernel pullback of the species-aware 2C overlap: dcoef and dalpha
 * (= d/dzeta through the kernel), both (ns,K,NZ), from the cotangent dS (N,N,B).
 * Replaces batch_S_orbital_pb_kernel! + _overlap_pb_coef_alpha
 * (src/integrals/orbital/overlap_2c_grad.jl:71-242).  Padded slots are not
 * skipped (as in the reference).  Deterministic: per-block partials and a
 * fixed-order second-stage reduction, no global atomics.
 */
int aok_overlap2c_pullback(aok_plan* plan, void* dcoef, void* dalpha, const void* dS,
                           const void* zeta, const void* coef, const void* posA,
                           const void* posB, const int64_t* sidxA, const int64_t* sidxB,
                           int64_t B, double lengthscale, void* stream);

/*
 * Position pullback of the species-aware 2C overlap (no reference counterpart:
 * the reference's rrule returns no position tangent and lists position
 * gradients of the overlap as not implemented).  From the cotangent dS (N,N,B)
 * of aok_overlap2c's output, dA, dB (3,B) = sum dS * dS/dA, sum dS * dS/dB with
 * respect to the input positions (the lengthscale factor included); either may
 * be NULL.  The overlap depends on A - B only, so dB = -dA.  zeta, coef,
 * positions and species indices as aok_overlap2c.  Deterministic (fixed-order
 * sums, no atomics on data).  A pair whose species index is outside 1..NZ gets
 * dA = dB = 0 and sets the plan's error word (aok_plan_check).
 */
int aok_overlap2c_position_pullback(aok_plan* plan, void* dA, void* dB, const void* dS, const void* zeta,
                                    const void* coef, const void* posA, const void* posB,
                                    const int64_t* sidxA, const int64_t* sidxB, int64_t B,
                                    double lengthscale, void* stream);

/*
 * Closed-form VJP of the normalisation: (dD, dzeta_norm) from dcoef.
 * Replaces _compile_coef_pb (src/integrals/orbital/overlap_2c_grad.jl:251-286).
 */
int aok_compile_coef_pullback(aok_plan* plan, void* dD, void* dzeta, const void* dcoef,
                              const void* zeta, const void* D, void* stream);

/*
 * Full parameter pullback of the differentiable overlap:
 * dzeta = dalpha + dzeta_norm, dD, from dS.  Replaces pullback_ps(dS, orb, XA, XB, ps, st)
 * (src/integrals/orbital/overlap_2c_grad.jl:296-304); zeta, D are ps.Rnl.
 */
int aok_overlap_pullback_ps(aok_plan* plan, void* dzeta, void* dD, const void* dS,
                            const void* zeta, const void* D, const void* posA,
                            const void* posB, const int64_t* sidxA, const int64_t* sidxB,
                            int64_t B, double lengthscale, void* stream);

/*
 * The two halves of rrule(batch_overlap, orb, XA, XB, ps, st)
 * (src/integrals/orbital/overlap_2c_grad.jl:309-318) with the pullback's
 * preparation moved into the forward.  aok_overlap2c_rrule computes coef from
 * (zeta, D) as compile_basis does, writes S = batch_overlap(orb, XA, XB, ps, st)
 * into out, and, on the plan's side stream while the overlap kernel runs,
 * prepares the pullback's primitive-pair records; it keeps the species binning.
 * aok_overlap_pullback_ps_rrule then returns (dzeta, dD) as aok_overlap_pullback_ps
 * would, without compiling, preparing or binning again.  It must follow the
 * forward on the same plan with the same zeta, D, posA, posB, sidxA, sidxB, B and
 * lengthscale, and with no other 2C call on the plan in between; otherwise it
 * returns AOK_ERR_INVALID.  The caller keeps the inputs unchanged in between.
 */
int aok_overlap2c_rrule(aok_plan* plan, void* out, const void* zeta, const void* D,
                        const void* posA, const void* posB, const int64_t* sidxA,
                        const int64_t* sidxB, int64_t B, double lengthscale, void* stream);
int aok_overlap_pullback_ps_rrule(aok_plan* plan, void* dzeta, void* dD, const void* dS,
                                  const void* zeta, const void* D, const void* posA,
                                  const void* posB, const int64_t* sidxA, const int64_t* sidxB,
                                  int64_t B, double lengthscale, void* stream);
/*
 * The rrule pullback for a squared-residual loss, with the cotangent formed on
 * the fly: dS = alpha * (S - T), S the forward's output and T a target of the
 * same layout (N,N,B) -- the gradient of (alpha/2) * sum (S - T)^2, e.g.
 * alpha = 2 for L = sum (S - T)^2.  Same conditions and results as
 * aok_overlap_pullback_ps_rrule given that dS, without writing or reading dS
 * (the difference is taken in the kernel that reads the cotangent, alpha is
 * applied to the reduced gradient).  It fuses the loss's cotangent into the
 * pullback of rrule(batch_overlap, ...) (src/integrals/orbital/overlap_2c_grad.jl:309-318).
 */
int aok_overlap_pullback_ps_rrule_residual(aok_plan* plan, void* dzeta, void* dD, const void* S,
                                           const void* T, double alpha, const void* zeta,
                                           const void* D, const void* posA, const void* posB,
                                           const int64_t* sidxA, const int64_t* sidxB, int64_t B,
                                           double lengthscale, void* stream);

/*
 * Orbital-evaluation plan: radial spec (nRad radials, K slots, NZ species,
 * poly[nRad] radial powers), orbital index maps iR, iY (nOrb, 1-based),
 * harmonics up to L.  Mirrors AtomicOrbitals' state
 * (src/orbitals/atomicorbitals.jl:31-75, 90-98) and GaussianTypeRadials /
 * SlaterTypeRadials (src/orbitals/gtostoradials.jl:14-46).
 */
int aok_orbitals_create(aok_orbitals** orb, int64_t nRad, int64_t K, int64_t NZ,
                        const int64_t* poly, int64_t nOrb, const int64_t* iR,
                        const int64_t* iY, int64_t L, int radial_kind, int precision);
int aok_orbitals_destroy(aok_orbitals* orb);
/* Synchronises `stream`, then reports (and clears) the orbitals' device error
 * word: AOK_ERR_SPECIES if aok_evaluate, aok_evaluate_ed or
 * aok_evaluate_pullback met a species index outside 1..NZ.  No memory outside
 * the arguments is touched for such a point: the forward evaluates it as
 * species 1 (its values are not meaningful); the pullback gives it dX = 0 and
 * leaves it out of the (zeta, D) gradient.  The device half of the
 * reference's unknown-species error (_cgto_species_index,
 * src/integrals/orbital/overlap_2c.jl:148-158) for callers that pass device
 * species indices unchecked. */
int aok_orbitals_check(aok_orbitals* orb, void* stream);

/*
 * P (nX,nOrb) = R_{iR} * Z_{iY} at positions X (3,nX) times lengthscale.
 * Replaces evaluate(basis, Rs, sidx, ps, st) (src/orbitals/atomicorbitals.jl:148-162):
 * _rnl_val_ka!, SpheriCart.compute and _aorb_val_ka! fused in one kernel.
 */
int aok_evaluate(aok_orbitals* orb, void* P, const void* X, const int64_t* sidx,
                 const void* zeta, const void* D, int64_t nX, double lengthscale,
                 void* stream);

/*
 * P and dP (3,nX,nOrb) (gradient w.r.t. the input coordinates, including the
 * lengthscale factor).  Replaces evaluate_ed(basis, Rs, sidx, ps, st)
 * (src/orbitals/atomicorbitals.jl:192-210): _rnl_ed_ka!,
 * SpheriCart.compute_with_gradients, _aorb_ed_ka! and `dRnlm .*= s` fused.
 */
int aok_evaluate_ed(aok_orbitals* orb, void* P, void* dP, const void* X,
                    const int64_t* sidx, const void* zeta, const void* D, int64_t nX,
                    double lengthscale, void* stream);

/*
 * Pullback of evaluate: dX (3,nX) (may be NULL) and dzeta, dD (nRad,K,NZ)
 * (may be NULL together) from dP (nX,nOrb).  Replaces the rrule pullback
 * (src/orbitals/atomicorbitals.jl:249-316: _aorb_pbx_ka!, _aorb_pbrad_ka!,
 * and the radial pullback_ps, src/orbitals/gtostoradials.jl:232-267),
 * recomputing R, Z and their gradients instead of reading stored ones.
 * Deterministic (per-block partials, fixed-order reduction).
 */
int aok_evaluate_pullback(aok_orbitals* orb, void* dX, void* dzeta, void* dD,
                          const void* dP, const void* X, const int64_t* sidx,
                          const void* zeta, const void* D, int64_t nX, double lengthscale,
                          void* stream);

/*
 * The radial layer on its own: GaussianTypeRadials / SlaterTypeRadials with
 * nRad radials of K primitive slots for NZ species and radial powers poly[nRad]
 * (host array; the layer's state st.poly, src/orbitals/gtostoradials.jl:14-46,
 * 103-113).  Values are R[j,k] = r_j^poly[k] sum_m D[k,m,s_j] exp(-zeta[k,m,s_j] f(r_j))
 * with f(r) = r^2 (Gaussian) or r (Slater).
 */
int aok_radials_create(aok_radials** rad, int64_t nRad, int64_t K, int64_t NZ, const int64_t* poly,
                       int radial_kind, int precision);
int aok_radials_destroy(aok_radials* rad);
/* Synchronises `stream`, then reports (and clears) the plan's device error word:
 * AOK_ERR_SPECIES if a radial call met a species index outside 1..NZ (the device
 * half of _z2i's unknown-species error, src/orbitals/gtostoradials.jl:58-62).  Such
 * a point is evaluated as species 1 by the forward and left out of the pullback. */
int aok_radials_check(aok_radials* rad, void* stream);
/*
 * R (nX,nRad) and, when dR is not NULL, dR/dr (nX,nRad) at the radii r (nX) for
 * species indices sidx (nX, 1-based); zeta, D are ps.zeta, ps.D (nRad,K,NZ).
 * Replaces evaluate / evaluate_ed(basis::GSRadials, r, sidx, ps, st)
 * (src/orbitals/gtostoradials.jl:117-185: _rnl_val_ka!, _rnl_ed_ka!).
 */
int aok_radials_evaluate(aok_radials* rad, void* R, void* dR, const void* r, const int64_t* sidx,
                         const void* zeta, const void* D, int64_t nX, void* stream);
/*
 * Parameter pullback of the radial layer: dzeta, dD (nRad,K,NZ) from the
 * cotangent dRin (nX,nRad) of R.  Replaces pullback_ps(dR, basis::GSRadials, r,
 * sidx, ps, st) (src/orbitals/gtostoradials.jl:232-267, _gtostoradials_pb_ka!):
 * units of consecutive points are reduced per species and (radial, primitive)
 * slot into per-unit FP64 partial rows summed in a fixed order (deterministic,
 * no atomics on data).
 */
int aok_radials_pullback(aok_radials* rad, void* dzeta, void* dD, const void* dRin, const void* r,
                         const int64_t* sidx, const void* zeta, const void* D, int64_t nX, void* stream);

/*
 * Allocation-free variant of aok_evaluate_pullback.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory when
 * they need the pullback -- a host framework that owns the whole device
 * through its own pooling allocator, or a service that reserves its memory at
 * start-up and must not grow afterwards.  It takes the orbital description by
 * value (host arrays poly[nRad], iR[nOrb], iY[nOrb], 1-based maps as in
 * aok_orbitals_create) instead of a plan, and allocates nothing: its scratch
 * (index maps, error word, per-block FP64 partial rows) is one static device
 * array of AOK_NOALLOC_SCRATCH_BYTES that every GPU loading the library keeps
 * until the process exits.  Limits: nRad <= 64, nOrb <= 256, K <= 64,
 * NZ <= 64, nX < 2^31, and, when the (zeta, D) gradient is asked for,
 * 4096 + 16 * nRad*K*NZ * ceil(nX / 128) bytes must fit the scratch (a
 * dX-only call needs no partial rows); larger requests return
 * AOK_ERR_UNSUPPORTED with the sizes in the message.  The first call on a
 * device looks up the array's device address (make it before any stream
 * capture).  All calls share the array and overwrite it, so calls that may
 * overlap on the GPU race and must be serialised by the caller.  Arguments
 * and results otherwise as aok_evaluate_pullback: a point whose species index
 * is outside 1..NZ gets dX = 0, adds nothing to (dzeta, dD), and sets the
 * scratch's error word, which aok_evaluate_pullback_noalloc_check reports.
 */
#define AOK_NOALLOC_SCRATCH_BYTES (8u << 20)
int aok_evaluate_pullback_noalloc(int64_t nRad, int64_t K, int64_t NZ, const int64_t* poly,
                                  int64_t nOrb, const int64_t* iR, const int64_t* iY, int64_t L,
                                  int radial_kind, int precision, void* dX, void* dzeta,
                                  void* dD, const void* dP, const void* X, const int64_t* sidx,
                                  const void* zeta, const void* D, int64_t nX,
                                  double lengthscale, void* stream);
/* The error report of aok_evaluate_pullback_noalloc (no reference counterpart;
 * its role is that of aok_orbitals_check): synchronises `stream`, then reads
 * and clears the static scratch's error word on the current device and returns
 * AOK_ERR_SPECIES if the allocation-free pullback met a species index outside
 * 1..NZ since the last check.  Each allocation-free call clears the word when
 * it starts, so check after the call and before the next one.  Allocates
 * nothing; AOK_OK if no allocation-free call has run on the device. */
int aok_evaluate_pullback_noalloc_check(void* stream);

#ifdef __cplusplus
}
#endif

#endif /* AOK_H */
