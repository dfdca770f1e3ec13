// orbitals.cu -- fused atomic-orbital evaluation phi_i = R_{iR[i]}(r) Z_{iY[i]}(r)
// with spatial gradients, and its pullback, sm_100a.
//
// Replaces, in one kernel per call:
//   _rnl_val_ka! / _rnl_ed_ka!        src/orbitals/gtostoradials.jl:117-153
//   SpheriCart compute[_with_gradients] (called at atomicorbitals.jl:155,200)
//   _aorb_val_ka! / _aorb_ed_ka!      src/orbitals/atomicorbitals.jl:110-125
//   `r = norm.(Rs)`, `s .* Rs`, `dRnlm .*= s`   atomicorbitals.jl:138-141,153,198,208
// and for the pullback
//   _aorb_pbx_ka!                     atomicorbitals.jl:283-299
//   _aorb_pbrad_ka! + radial pullback atomicorbitals.jl:249-267, gtostoradials.jl:232-267
//
// One thread per point: the radials (per-species zeta, D staged in shared
// memory), the real solid harmonics Z_lm and their gradients (compile-time
// L, recursion in registers), then the products written straight to the
// reference layouts P[j + nX*i] and dP[c + 3*(j + nX*i)] (coalesced per
// orbital).  The per-thread R, dR, Z, dZ live in shared memory so the
// orbital index maps iR/iY can be arbitrary.
//
// Real solid harmonics (L2-normalised on the unit sphere, index l^2+l+m):
//   Z_l0 = F_l0 Q_l^0,  Z_l,+m = sqrt2 F_lm Q_l^m C_m,  Z_l,-m = sqrt2 F_lm Q_l^m S_m,
//   F_lm = sqrt((2l+1)/(4 pi) (l-m)!/(l+m)!),  C_m + i S_m = (x + i y)^m,
//   Q_m^m = (2m-1)!!,  Q_{m+1}^m = (2m+1) z Q_m^m,
//   Q_l^m = ((2l-1) z Q_{l-1}^m - (l+m-1) r^2 Q_{l-2}^m) / (l - m),
// no Condon-Shortley phase (Z_1,-1 : Z_1,0 : Z_1,1 = y : z : x).
//
// The parameter pullback is deterministic: each warp reduces its 32 points'
// contributions per species with a fixed butterfly, warps are summed in order
// into a per-block FP64 row, and the rows are summed in block order.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "aok_internal.h"

namespace aok {

constexpr int kEvalThreads = 128;
constexpr int kEvalMaxL = 4;
constexpr int kMaxY = (kEvalMaxL + 1) * (kEvalMaxL + 1);

struct EvalParams {
    void* P;          // (nX, nOrb)
    void* dP;         // (3, nX, nOrb) or null
    const void* X;    // (3, nX)
    const int64_t* sidx;
    const void* zeta; // (nRad, K, NZ)
    const void* D;
    const int* poly;  // (nRad)
    const int* iR;    // (nOrb) 0-based
    const int* iY;    // (nOrb) 0-based
    int* err;
    long long nX;
    int nRad, K, NZ, nOrb, slater;
    double scale;
    double F[kMaxY];  // F_lm by index l^2+l+m (m >= 0 entries used)
    // pullback only
    const void* dPin; // (nX, nOrb)
    void* dX;         // (3, nX) or null
    double* rows;     // [block][2 * nRad*K*NZ] or null
};

// Rounding-pinned arithmetic for the values (R, Z, r): the compiler may not fuse
// these into an FMA, so a value is computed by the same operations whether or
// not the kernel also forms gradients (evaluate and evaluate_ed agree bitwise).
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
template <typename FT>
__device__ __forceinline__ FT norm3(FT x, FT y, FT z) {
    return sqrt(fma_rn(x, x, fma_rn(y, y, mul_rn(z, z))));
}

// value + gradient
template <typename FT> struct D4 {
    FT v, x, y, z;
};
template <typename FT>
__device__ __forceinline__ D4<FT> dmul(const D4<FT>& a, const D4<FT>& b) {
    return {mul_rn(a.v, b.v), a.x * b.v + a.v * b.x, a.y * b.v + a.v * b.y, a.z * b.v + a.v * b.z};
}
template <typename FT>
__device__ __forceinline__ D4<FT> dlin(FT ca, const D4<FT>& a, FT cb, const D4<FT>& b) {
    return {fma_rn(ca, a.v, mul_rn(cb, b.v)), ca * a.x + cb * b.x, ca * a.y + cb * b.y, ca * a.z + cb * b.z};
}

// Z_lm and gradients for l <= L at (x, y, z), written to Z[idx], G[3*idx + c].
// The convention is SpheriCart's (Bigi, Fraux, Browning, Ceriotti, J. Chem. Phys.
// 159, 064802 (2023), Sec. II), the harmonics the reference's SolidHarmonics
// evaluates: Z_l^m = F_l^|m| Q_l^|m| {s_|m|, 1/sqrt2, c_m} with
// F_l^m = (-1)^m sqrt((2l+1)/(2pi) (l-m)!/(l+m)!) and Q_m^m = (-1)^m (2m-1)!!.
// The two (-1)^m cancel, so here both are dropped: Q_m^m = (2m-1)!! and the
// m != 0 factor is sqrt(2) F_lm with F_lm = sqrt((2l+1)/(4pi) (l-m)!/(l+m)!).
template <typename FT, int L>
__device__ __forceinline__ void solid_harmonics(FT x, FT y, FT z, const double* F, FT* Zs, FT* Gs, int stride) {
    const D4<FT> X{x, FT(1), FT(0), FT(0)}, Y{y, FT(0), FT(1), FT(0)}, Zd{z, FT(0), FT(0), FT(1)};
    const D4<FT> r2{fma_rn(x, x, fma_rn(y, y, mul_rn(z, z))), FT(2) * x, FT(2) * y, FT(2) * z};
    D4<FT> C[L + 1], S[L + 1];
    C[0] = {FT(1), FT(0), FT(0), FT(0)};
    S[0] = {FT(0), FT(0), FT(0), FT(0)};
#pragma unroll
    for (int m = 0; m < L; ++m) {
        C[m + 1] = dlin(FT(1), dmul(X, C[m]), FT(-1), dmul(Y, S[m]));
        S[m + 1] = dlin(FT(1), dmul(X, S[m]), FT(1), dmul(Y, C[m]));
    }
#pragma unroll
    for (int m = 0; m <= L; ++m) {
        D4<FT> q2{FT(0), FT(0), FT(0), FT(0)}, q1{FT(0), FT(0), FT(0), FT(0)};
        FT dfac = FT(1);
        for (int k = 2 * m - 1; k > 1; k -= 2) dfac *= FT(k);
        D4<FT> q{dfac, FT(0), FT(0), FT(0)};  // Q_m^m
#pragma unroll
        for (int l = m; l <= L; ++l) {
            if (l == m + 1) {
                q = dmul(D4<FT>{mul_rn(FT(2 * m + 1), z), FT(0), FT(0), FT(2 * m + 1)}, q1);
            } else if (l >= m + 2) {
                const D4<FT> a = dmul(D4<FT>{mul_rn(FT(2 * l - 1), z), FT(0), FT(0), FT(2 * l - 1)}, q1);
                const D4<FT> b = dmul(D4<FT>{mul_rn(FT(l + m - 1), r2.v), FT(l + m - 1) * r2.x, FT(l + m - 1) * r2.y,
                                             FT(l + m - 1) * r2.z},
                                      q2);
                const FT inv = FT(1) / FT(l - m);
                q = dlin(inv, a, -inv, b);
            }
            const int i0 = l * l + l;
            if (m == 0) {
                const FT f = (FT)F[i0];
                Zs[i0 * stride] = mul_rn(f, q.v);
                Gs[(3 * i0 + 0) * stride] = f * q.x;
                Gs[(3 * i0 + 1) * stride] = f * q.y;
                Gs[(3 * i0 + 2) * stride] = f * q.z;
            } else {
                const FT f = (FT)(1.4142135623730951 * F[i0 + m]);
                const D4<FT> pc = dmul(q, C[m]), ps = dmul(q, S[m]);
                Zs[(i0 + m) * stride] = mul_rn(f, pc.v);
                Gs[(3 * (i0 + m) + 0) * stride] = f * pc.x;
                Gs[(3 * (i0 + m) + 1) * stride] = f * pc.y;
                Gs[(3 * (i0 + m) + 2) * stride] = f * pc.z;
                Zs[(i0 - m) * stride] = mul_rn(f, ps.v);
                Gs[(3 * (i0 - m) + 0) * stride] = f * ps.x;
                Gs[(3 * (i0 - m) + 1) * stride] = f * ps.y;
                Gs[(3 * (i0 - m) + 2) * stride] = f * ps.z;
            }
            q2 = q1;
            q1 = q;
        }
    }
}

// Radial k at r for species sg: R = r^p sum_m D e^{-zeta f(r)}, dR/dr.
// FP32 sums use TwoSum compensation over the K terms.
// exp(-zeta f): FP32 as 2^{-(zeta log2 e) f} with zl = zeta log2(e) computed in
// FP64 and rounded once (relative error ~1e-7 (1 + zeta f)); FP64 plain exp.
__device__ __forceinline__ float exp_neg(float z, float zl, float f) {
    (void)z;
    return ex2_approx(-zl * f);
}
__device__ __forceinline__ double exp_neg(double z, double zl, double f) {
    (void)zl;
    return exp(-z * f);
}

// Words (of FT) of the per-(radial, species) primitive counts that follow the tables.
__host__ __device__ constexpr int count_words(int nRad, int NZ, int fsz) { return (nRad * NZ * 4 + fsz - 1) / fsz; }

// Primitives of radial k, species sg, up to the last non-zero D: the trailing ones
// (padding of shorter contractions) add exact zeros to R and dR, so they are skipped.
template <typename FT>
__device__ __forceinline__ int radial_count(const FT* D, int k, int sg, int nRad, int K) {
    int mk = K;
    while (mk > 0 && D[k + nRad * (mk - 1 + K * sg)] == FT(0)) --mk;
    return mk;
}

// (zeta, D, zeta log2 e) of primitive slot o: three separate shared-memory
// tables, or one packed entry per slot (one 16-byte load in FP32).
template <typename FT>
struct SepTab {
    const FT *z, *D, *l;
    __device__ __forceinline__ void get(int o, int, FT& zo, FT& Do, FT& lo) const {
        zo = z[o];
        Do = D[o];
        lo = l[o];
    }
};
struct __align__(16) Pk64 {
    double z, D, l, pad;
};
template <typename FT> struct PkEntry;
template <> struct PkEntry<float> { using type = float4; };
template <> struct PkEntry<double> { using type = Pk64; };
// Packed entries: species sg's block of nRad*K slots starts at sg (nRad*K + 1), one
// spare entry per species, so lanes of different species read different banks.
template <typename FT>
struct PkTab {
    const typename PkEntry<FT>::type* p;
    __device__ __forceinline__ void get(int o, int sg, FT& zo, FT& Do, FT& lo) const {
        const auto t = p[o + sg];
        if constexpr (sizeof(FT) == 4) {
            zo = t.x;
            Do = t.y;
            lo = t.z;
        } else {
            zo = t.z;
            Do = t.D;
            lo = t.l;
        }
    }
};
template <typename FT>
__device__ __forceinline__ typename PkEntry<FT>::type pk_entry(FT z, FT D, FT l) {
    typename PkEntry<FT>::type e;
    if constexpr (sizeof(FT) == 4) {
        e = make_float4(z, D, l, 0.f);
    } else {
        e.z = z;
        e.D = D;
        e.l = l;
        e.pad = 0.0;
    }
    return e;
}

template <typename FT, typename Tab>
__device__ __forceinline__ void radial_t(const Tab& tb, const int* sn, int k, int sg, int nRad, int K, int p,
                                         int slater, FT r, FT& R, FT& dR) {
    const FT f = slater ? r : r * r;
    const FT df = slater ? FT(1) : FT(2) * r;
    FT s = FT(0), se = FT(0), ds = FT(0);
    const int mk = sn[k + nRad * sg];
    for (int m = 0; m < mk; ++m) {
        const int o = k + nRad * (m + K * sg);
        FT z, D, zl;
        tb.get(o, sg, z, D, zl);
        const FT a = mul_rn(D, exp_neg(z, zl, f));
        if constexpr (sizeof(FT) == 4) {
            const float t = s + a, bb = t - s;
            se += (s - (t - bb)) + (a - bb);
            s = t;
        } else {
            s = add_rn(s, a);
        }
        ds += (-z * df) * a;
    }
    s += se;
    FT rp = FT(1);
    for (int i = 0; i < p; ++i) rp *= r;
    FT drp = FT(0);
    if (p > 0) {
        drp = FT(p);
        for (int i = 0; i < p - 1; ++i) drp *= r;
    }
    R = mul_rn(rp, s);
    dR = drp * s + rp * ds;
}

template <typename FT>
__device__ __forceinline__ void radial(const FT* sz, const FT* sD, const FT* sl, const int* sn, int k, int sg,
                                       int nRad, int K, int p, int slater, FT r, FT& R, FT& dR) {
    radial_t<FT>(SepTab<FT>{sz, sD, sl}, sn, k, sg, nRad, K, p, slater, r, R, dR);
}

// shared layout: zeta, D tables, then per-thread R, dR (nRad), Z (nY), G (3 nY)
template <typename FT>
struct EvalSmem {
    FT* sz;
    FT* sD;
    FT* sl;  // zeta log2(e)
    int* sn; // primitive counts per (radial, species), radial_count
    FT* R;
    FT* dR;
    FT* Z;
    FT* G;
};
template <typename FT>
__device__ __forceinline__ EvalSmem<FT> eval_smem(unsigned char* raw, int ntab, int nRad, int NZ, int nY) {
    EvalSmem<FT> s;
    FT* p = reinterpret_cast<FT*>(raw);
    s.sz = p;
    s.sD = p + ntab;
    s.sl = p + 2 * ntab;
    s.sn = reinterpret_cast<int*>(p + 3 * ntab);
    p += 3 * ntab + count_words(nRad, NZ, (int)sizeof(FT));
    s.R = p;
    p += nRad * kEvalThreads;
    s.dR = p;
    p += nRad * kEvalThreads;
    s.Z = p;
    p += nY * kEvalThreads;
    s.G = p;
    return s;
}

template <typename FT, int L, bool GRAD>
__global__ void __launch_bounds__(kEvalThreads) k_evaluate(const __grid_constant__ EvalParams P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int nY = (L + 1) * (L + 1);
    const int ntab = P.nRad * P.K * P.NZ;
    EvalSmem<FT> S = eval_smem<FT>(smem_raw, ntab, P.nRad, P.NZ, nY);
    for (int i = threadIdx.x; i < ntab; i += blockDim.x) {
        S.sz[i] = ((const FT*)P.zeta)[i];
        S.sD[i] = ((const FT*)P.D)[i];
        S.sl[i] = (FT)((double)((const FT*)P.zeta)[i] * 1.4426950408889634074);
    }
    for (int i = threadIdx.x; i < P.nRad * P.NZ; i += blockDim.x)
        S.sn[i] = radial_count((const FT*)P.D, i % P.nRad, i / P.nRad, P.nRad, P.K);
    __syncthreads();
    // the blocks stay resident and stride over the points, so each stages the tables once
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < P.nX;
         j += (long long)gridDim.x * blockDim.x) {
        const int t = threadIdx.x;
        const FT* X = (const FT*)P.X;
        FT x = X[3 * j], y = X[3 * j + 1], z = X[3 * j + 2];
        const FT sc = (FT)P.scale;
        if (sc != FT(1)) {
            x = sc * x;
            y = sc * y;
            z = sc * z;
        }
        const FT r = norm3(x, y, z);
        int sg = (int)P.sidx[j] - 1;
        if (sg < 0 || sg >= P.NZ) {
            atomicCAS(P.err, 0, AOK_ERR_SPECIES);
            sg = 0;
        }
        for (int k = 0; k < P.nRad; ++k) {
            FT R, dR;
            radial<FT>(S.sz, S.sD, S.sl, S.sn, k, sg, P.nRad, P.K, P.poly[k], P.slater, r, R, dR);
            S.R[k * kEvalThreads + t] = R;
            S.dR[k * kEvalThreads + t] = dR;
        }
        solid_harmonics<FT, L>(x, y, z, P.F, S.Z + t, S.G + t, kEvalThreads);
        FT* Pout = (FT*)P.P;
        FT* dPout = (FT*)P.dP;
        const FT ux = x / r, uy = y / r, uz = z / r;  // X[j] / r[j] (NaN at r = 0, as the reference)
        for (int i = 0; i < P.nOrb; ++i) {
            const int k = P.iR[i], yi = P.iY[i];
            const FT rn = S.R[k * kEvalThreads + t], yl = S.Z[yi * kEvalThreads + t];
            Pout[j + P.nX * i] = rn * yl;
            if (GRAD) {
                const FT dr = S.dR[k * kEvalThreads + t];
                FT* o = dPout + 3 * (j + P.nX * i);
                FT gx = (dr * ux) * yl + rn * S.G[(3 * yi + 0) * kEvalThreads + t];
                FT gy = (dr * uy) * yl + rn * S.G[(3 * yi + 1) * kEvalThreads + t];
                FT gz = (dr * uz) * yl + rn * S.G[(3 * yi + 2) * kEvalThreads + t];
                if (sc != FT(1)) {
                    gx *= sc;
                    gy *= sc;
                    gz *= sc;
                }
                o[0] = gx;
                o[1] = gy;
                o[2] = gz;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Forward with the harmonics in registers (L <= 3, each (radial, harmonic) pair
// used by at most one orbital).  The orbital maps are turned into a table
// otab[k * nY + yi] -> orbital (or -1) held in the kernel's parameter space, so
// that the loop over radials k (run time) nests an unrolled loop over the
// harmonics yi (compile time): Z[yi], G[yi] stay in registers and R_k, dR_k
// are used as soon as they are formed.  Compared with k_evaluate this drops
// the per-thread shared-memory round trip of R, dR, Z, G and the per-orbital
// map loads; the table entries are warp-uniform constant-bank reads.
// ---------------------------------------------------------------------------
constexpr int kRegMaxRad = 64;
constexpr int kRegMaxL = 3;
struct EvalRegParams {
    EvalParams E;
    int16_t otab[kRegMaxRad * (kRegMaxL + 1) * (kRegMaxL + 1)];
    int8_t poly[kRegMaxRad];
    // block maps (BLK): radial k feeds the 2l+1 orbitals ob[k] .. ob[k] + 2l, in
    // harmonic order l^2 .. l^2 + 2l, with l = lk[k] (-1: a radial no orbital uses)
    int8_t lk[kRegMaxRad];
    int16_t ob[kRegMaxRad];
};

// The orbitals of one radial under block maps: 2 LL + 1 outputs, harmonic and
// orbital indices known at compile time relative to the block's start.
template <typename FT, int LL, int L, bool GRAD>
__device__ __forceinline__ void emit_block(FT R, FT dR, FT ux, FT uy, FT uz, FT sc, const FT (&Z)[(L + 1) * (L + 1)],
                                           const FT (&G)[3 * (L + 1) * (L + 1)], FT* Pout, FT* dPout, long long j,
                                           long long nX, int o0) {
    if constexpr (LL <= L) {
#pragma unroll
        for (int m = 0; m <= 2 * LL; ++m) {
            const int yi = LL * LL + m;
            const long long at = j + nX * (o0 + m);
            Pout[at] = R * Z[yi];
            if (GRAD) {
                FT gx = (dR * ux) * Z[yi] + R * G[3 * yi + 0];
                FT gy = (dR * uy) * Z[yi] + R * G[3 * yi + 1];
                FT gz = (dR * uz) * Z[yi] + R * G[3 * yi + 2];
                if (sc != FT(1)) {
                    gx *= sc;
                    gy *= sc;
                    gz *= sc;
                }
                FT* op = dPout + 3 * at;
                op[0] = gx;
                op[1] = gy;
                op[2] = gz;
            }
        }
    }
}

template <typename FT, int L, bool GRAD, bool BLK = false>
__global__ void __launch_bounds__(kEvalThreads) k_evaluate_reg(const __grid_constant__ EvalRegParams Q) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const EvalParams& P = Q.E;
    constexpr int nY = (L + 1) * (L + 1);
    const int ntab = P.nRad * P.K * P.NZ;
    auto* pk = reinterpret_cast<typename PkEntry<FT>::type*>(smem_raw);  // (zeta, D, zeta log2 e) per slot
    int* sn = reinterpret_cast<int*>(pk + ntab + P.NZ);
    const int nsl = P.nRad * P.K;
    for (int i = threadIdx.x; i < ntab; i += blockDim.x) {
        const FT z = ((const FT*)P.zeta)[i];
        pk[i + i / nsl] = pk_entry<FT>(z, ((const FT*)P.D)[i], (FT)((double)z * 1.4426950408889634074));
    }
    for (int i = threadIdx.x; i < P.nRad * P.NZ; i += blockDim.x)
        sn[i] = radial_count((const FT*)P.D, i % P.nRad, i / P.nRad, P.nRad, P.K);
    __syncthreads();
    FT* Pout = (FT*)P.P;
    FT* dPout = (FT*)P.dP;
    const FT sc = (FT)P.scale;
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < P.nX;
         j += (long long)gridDim.x * blockDim.x) {
        const FT* X = (const FT*)P.X;
        FT x = X[3 * j], y = X[3 * j + 1], z = X[3 * j + 2];
        if (sc != FT(1)) {
            x = sc * x;
            y = sc * y;
            z = sc * z;
        }
        const FT r = norm3(x, y, z);
        int sg = (int)P.sidx[j] - 1;
        if (sg < 0 || sg >= P.NZ) {
            atomicCAS(P.err, 0, AOK_ERR_SPECIES);
            sg = 0;
        }
        FT Z[nY], G[3 * nY];
        solid_harmonics<FT, L>(x, y, z, P.F, Z, G, 1);
        const FT ux = x / r, uy = y / r, uz = z / r;  // X[j] / r[j] (NaN at r = 0, as the reference)
        if constexpr (BLK) {
            for (int k = 0; k < P.nRad; ++k) {
                const int l = Q.lk[k];
                if (l < 0) continue;
                FT R, dR;
                radial_t<FT>(PkTab<FT>{pk}, sn, k, sg, P.nRad, P.K, Q.poly[k], P.slater, r, R, dR);
                const int o0 = Q.ob[k];
                switch (l) {
                    case 0: emit_block<FT, 0, L, GRAD>(R, dR, ux, uy, uz, sc, Z, G, Pout, dPout, j, P.nX, o0); break;
                    case 1: emit_block<FT, 1, L, GRAD>(R, dR, ux, uy, uz, sc, Z, G, Pout, dPout, j, P.nX, o0); break;
                    case 2: emit_block<FT, 2, L, GRAD>(R, dR, ux, uy, uz, sc, Z, G, Pout, dPout, j, P.nX, o0); break;
                    default: emit_block<FT, 3, L, GRAD>(R, dR, ux, uy, uz, sc, Z, G, Pout, dPout, j, P.nX, o0); break;
                }
            }
        } else {
            for (int k = 0; k < P.nRad; ++k) {
                FT R, dR;
                radial_t<FT>(PkTab<FT>{pk}, sn, k, sg, P.nRad, P.K, Q.poly[k], P.slater, r, R, dR);
#pragma unroll
                for (int yi = 0; yi < nY; ++yi) {
                    const int o = Q.otab[k * nY + yi];
                    if (o < 0) continue;
                    Pout[j + P.nX * o] = R * Z[yi];
                    if (GRAD) {
                        FT gx = (dR * ux) * Z[yi] + R * G[3 * yi + 0];
                        FT gy = (dR * uy) * Z[yi] + R * G[3 * yi + 1];
                        FT gz = (dR * uz) * Z[yi] + R * G[3 * yi + 2];
                        if (sc != FT(1)) {
                            gx *= sc;
                            gy *= sc;
                            gz *= sc;
                        }
                        FT* op = dPout + 3 * (j + P.nX * o);
                        op[0] = gx;
                        op[1] = gy;
                        op[2] = gz;
                    }
                }
            }
        }
    }
}

// Pullback: dX (optional) and per-block rows of (dD, dzeta) partials.
template <typename FT, int L>
__global__ void __launch_bounds__(kEvalThreads) k_evaluate_pb(const __grid_constant__ EvalParams P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int nY = (L + 1) * (L + 1);
    constexpr int NW = kEvalThreads / 32;
    const int ntab = P.nRad * P.K * P.NZ;
    EvalSmem<FT> S = eval_smem<FT>(smem_raw, ntab, P.nRad, P.NZ, nY);
    // per-warp FP64 accumulators [warp][2][ntab] after the per-thread scratch
    double* wacc = reinterpret_cast<double*>(
        smem_raw + (((size_t)3 * ntab + count_words(P.nRad, P.NZ, (int)sizeof(FT)) +
                     (size_t)(2 * P.nRad + 4 * nY) * kEvalThreads) * sizeof(FT) + 7) / 8 * 8);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < ntab; i += blockDim.x) {
        S.sz[i] = ((const FT*)P.zeta)[i];
        S.sD[i] = ((const FT*)P.D)[i];
        S.sl[i] = (FT)((double)((const FT*)P.zeta)[i] * 1.4426950408889634074);
    }
    for (int i = threadIdx.x; i < P.nRad * P.NZ; i += blockDim.x)
        S.sn[i] = radial_count((const FT*)P.D, i % P.nRad, i / P.nRad, P.nRad, P.K);
    for (int i = threadIdx.x; i < NW * 2 * ntab; i += blockDim.x) wacc[i] = 0.0;
    __syncthreads();
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = j < P.nX;
    const int t = threadIdx.x;
    FT x = FT(0), y = FT(0), z = FT(1);
    int sg = -1;
    if (valid) {
        const FT* X = (const FT*)P.X;
        x = X[3 * j];
        y = X[3 * j + 1];
        z = X[3 * j + 2];
        const FT sc = (FT)P.scale;
        if (sc != FT(1)) {
            x = sc * x;
            y = sc * y;
            z = sc * z;
        }
        sg = (int)P.sidx[j] - 1;
        if (sg < 0 || sg >= P.NZ) {
            atomicCAS(P.err, 0, AOK_ERR_SPECIES);
            sg = -1;
        }
    }
    const FT r = norm3(x, y, z);
    const int sgc = sg < 0 ? 0 : sg;
    for (int k = 0; k < P.nRad; ++k) {
        FT R, dR;
        radial<FT>(S.sz, S.sD, S.sl, S.sn, k, sgc, P.nRad, P.K, P.poly[k], P.slater, r, R, dR);
        S.R[k * kEvalThreads + t] = R;
        S.dR[k * kEvalThreads + t] = dR;
    }
    solid_harmonics<FT, L>(x, y, z, P.F, S.Z + t, S.G + t, kEvalThreads);
    const FT* dPin = (const FT*)P.dPin;
    // dX = sum_i dP[j,i] grad phi_i ; dRad[k] = sum_{i: iR = k} dP[j,i] Z_iY  (reuses the dR slots' neighbour)
    FT ax = FT(0), ay = FT(0), az = FT(0);
    const FT ux = x / r, uy = y / r, uz = z / r;
    // accumulate dRad into S.R after dX is done: first pass dX
    if (valid && P.dX) {
        // a point with a species index outside 1..NZ (sg = -1) gets dX = 0
        for (int i = 0; i < (sg >= 0 ? P.nOrb : 0); ++i) {
            const int k = P.iR[i], yi = P.iY[i];
            const FT g = dPin[j + P.nX * i];
            const FT rn = S.R[k * kEvalThreads + t], yl = S.Z[yi * kEvalThreads + t];
            const FT dr = S.dR[k * kEvalThreads + t];
            ax += g * ((dr * ux) * yl + rn * S.G[(3 * yi + 0) * kEvalThreads + t]);
            ay += g * ((dr * uy) * yl + rn * S.G[(3 * yi + 1) * kEvalThreads + t]);
            az += g * ((dr * uz) * yl + rn * S.G[(3 * yi + 2) * kEvalThreads + t]);
        }
        const FT sc = (FT)P.scale;
        FT* dX = (FT*)P.dX;
        dX[3 * j] = sc != FT(1) ? ax * sc : ax;
        dX[3 * j + 1] = sc != FT(1) ? ay * sc : ay;
        dX[3 * j + 2] = sc != FT(1) ? az * sc : az;
    }
    if (!P.rows) return;
    // dRad[k] into S.dR (radial derivative no longer needed)
    for (int k = 0; k < P.nRad; ++k) S.dR[k * kEvalThreads + t] = FT(0);
    if (valid)
        for (int i = 0; i < P.nOrb; ++i) {
            const int k = P.iR[i], yi = P.iY[i];
            S.dR[k * kEvalThreads + t] += dPin[j + P.nX * i] * S.Z[yi * kEvalThreads + t];
        }
    // per (k, m): contributions of this point to its species' slot, reduced over the warp per species
    const FT f = P.slater ? r : r * r;
    for (int k = 0; k < P.nRad; ++k) {
        const int p = P.poly[k];
        FT rp = FT(1);
        for (int i = 0; i < p; ++i) rp *= r;
        const FT gg = S.dR[k * kEvalThreads + t] * rp;
        for (int m = 0; m < P.K; ++m) {
            FT cD = FT(0), cZ = FT(0);
            if (sg >= 0) {
                const int o = k + P.nRad * (m + P.K * sg);
                const FT a = exp_neg(S.sz[o], S.sl[o], f);
                cD = gg * a;
                cZ = ((gg * S.sD[o]) * a) * (-f);
            }
            for (int s = 0; s < P.NZ; ++s) {
                double vD = (sg == s) ? (double)cD : 0.0, vZ = (sg == s) ? (double)cZ : 0.0;
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    vD += __shfl_xor_sync(0xffffffffu, vD, off);
                    vZ += __shfl_xor_sync(0xffffffffu, vZ, off);
                }
                if (lane == 0) {
                    const int o = k + P.nRad * (m + P.K * s);
                    wacc[(size_t)warp * 2 * ntab + o] += vD;
                    wacc[(size_t)warp * 2 * ntab + ntab + o] += vZ;
                }
            }
        }
    }
    __syncthreads();
    double* row = P.rows + (size_t)blockIdx.x * 2 * ntab;
    for (int i = threadIdx.x; i < 2 * ntab; i += blockDim.x) {
        double sum = 0.0;
        for (int w = 0; w < NW; ++w) sum += wacc[(size_t)w * 2 * ntab + i];
        row[i] = sum;
    }
}

// ---------------------------------------------------------------------------
// Slot-parallel parameter pullback (used by aok_evaluate_pullback).
//
// A work unit is kEpbUnit = 32 consecutive points in the caller's order, dealt
// statically to the warps; four blocks of 8 warps per SM (<= 64 registers).  For
// each 32 points the warp first puts lane = point: radials (of the point's own species), harmonics, dX, and the radial
// cotangents gg_k = r^p_k sum_{i: iR[i] = k} dP[j,i] Z_{iY[i]} and f(r) into
// shared memory (the dP rows and positions are read coalesced).  Then, per
// species sigma present among the 32 points (a ballot), lane = slot (k, m) of
// sigma and the warp loops over those points in order:
//   dD[k,m,sigma]    += gg_k exp(-zeta f),
//   dzeta[k,m,sigma] += -D gg_k exp(-zeta f) f        (gtostoradials.jl:232-253),
// into the warp's per-unit accumulators (shared memory, one per (sigma, slot)),
// with no cross-lane reduction.  Each warp adds its units' sums into FP64
// running sums, each block writes its warps' sums in warp order as one partial
// row, and k_epb_reduce adds the rows in order, so the result is reproducible
// and does not depend on how the points' species are mixed.  A point with a species
// index outside 1..NZ gets dX = 0, is left out of every species, and sets the
// error word.
// ---------------------------------------------------------------------------
constexpr int kEpbUnit = 32;      // consecutive points per unit
constexpr int kEpbMaxGroups = 4;  // slots per species <= 128

struct EpbParams {
    EvalParams E;
    double* partial;    // [2][NZ][nRad*K][ucap]: dD, dzeta per (species, slot), units contiguous
    int ucap;           // row length of partial (at least the grid)
    int wwords;         // per-warp shared-memory words (of FT): scratch + accumulators
    int nrows;          // host side: the rows written (one per block of the launch)
    // register path (REG): (radial, harmonic) -> orbital table and radial powers
    int16_t otab[kRegMaxRad * (kRegMaxL + 1) * (kRegMaxL + 1)];
    int8_t poly[kRegMaxRad];
    // and, for block maps (blk != 0), each radial's l and first orbital (block_maps)
    int blk;
    int8_t lk[kRegMaxRad];
    int16_t ob[kRegMaxRad];
};

// Point phase of the register pullback under block maps: radial k's 2 LL + 1
// orbitals o0 + m with harmonics LL^2 + m; adds their dX terms and returns the
// radial cotangent sum_m dP[j, o0 + m] Z[LL^2 + m].
template <typename FT, int LL, int L>
__device__ __forceinline__ FT pb_block(FT Rk, FT dRk, FT ux, FT uy, FT uz, const FT (&Z)[(L + 1) * (L + 1)],
                                       const FT (&G)[3 * (L + 1) * (L + 1)], const FT* dPin, long long j,
                                       long long nX, int o0, FT& ax, FT& ay, FT& az) {
    FT gk = FT(0);
    if constexpr (LL <= L) {
#pragma unroll
        for (int m = 0; m <= 2 * LL; ++m) {
            const int yi = LL * LL + m;
            const FT g = dPin[j + nX * (o0 + m)];
            ax += g * ((dRk * ux) * Z[yi] + Rk * G[3 * yi + 0]);
            ay += g * ((dRk * uy) * Z[yi] + Rk * G[3 * yi + 1]);
            az += g * ((dRk * uz) * Z[yi] + Rk * G[3 * yi + 2]);
            gk += g * Z[yi];
        }
    }
    return gk;
}

// per-warp shared-memory scratch of the slot-parallel pullback (floats of FT):
// R, dR [nRad][32], Z [nY][32], G [3 nY][32], gg [nRad][kGgRow], f [32].  The
// radial cotangents' rows are padded to 33 words: in the slot phase the lanes read
// column t of different rows k, which a 32-word row would put in one bank.
constexpr int kGgRow = 33;
__host__ __device__ constexpr size_t epb_warp_words(int nRad, int nY) {
    return (size_t)(2 * nRad + 4 * nY + 1) * 32 + (size_t)nRad * kGgRow;
}
// the register path keeps only gg [nRad][kGgRow] and f [32]
__host__ __device__ constexpr size_t epb_warp_words_reg(int nRad) { return (size_t)nRad * kGgRow + 32; }
// Integer words after the (zeta, D, zeta log2 e) tables, in FT words: the primitive
// counts [nRad NZ], each species' representative slots [NZ][nRad K] and their counts [NZ].
__host__ __device__ constexpr int epb_int_words(int nRad, int K, int NZ, int fsz) {
    return (int)(((size_t)nRad * NZ + (size_t)NZ * nRad * K + NZ) * 4 + fsz - 1) / fsz;
}
// then the unit's accumulators [2][NZ][nRad*K]
__host__ __device__ constexpr size_t epb_acc_words(int nRad, int K, int NZ) { return (size_t)2 * NZ * nRad * K; }

// RAD: the radial layer's own pullback (gtostoradials.jl:232-267): X holds the
// radii r (nX), dPin the cotangent of R (nX, nRad), so gg_k = dR[j,k] r^p_k and
// there are no harmonics and no dX.
// REG (L <= 3, unique orbital maps): phase A keeps the harmonics and the current
// radial in registers and walks the (radial, harmonic) -> orbital table (as
// k_evaluate_reg), so a warp's shared memory holds only gg and f(r).
template <typename FT, int L, bool RAD = false, bool REG = false>
__global__ void __launch_bounds__(256, 4) k_evaluate_pbs(const __grid_constant__ EpbParams Q) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int nY = (L + 1) * (L + 1);
    const EvalParams& P = Q.E;
    const int ntab = P.nRad * P.K * P.NZ, nslot = P.nRad * P.K, NZ = P.NZ;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    auto* pk = reinterpret_cast<typename PkEntry<FT>::type*>(smem_raw);  // (zeta, D, zeta log2 e), species-padded
    const PkTab<FT> tb{pk};
    int* sn = reinterpret_cast<int*>(pk + ntab + NZ);
    int* srep = sn + P.nRad * P.NZ;  // [NZ][nslot]: each species' representative slots, in slot order
    int* snrep = srep + NZ * nslot;  // [NZ]: their number
    FT* wbase = reinterpret_cast<FT*>(pk + ntab + NZ) + epb_int_words(P.nRad, P.K, P.NZ, (int)sizeof(FT)) +
                (size_t)warp * Q.wwords;
    FT *R = wbase, *dR = R + 32 * P.nRad, *Z = dR + 32 * P.nRad, *G = Z + 32 * nY,
       *gg = REG ? wbase : G + 96 * nY, *fv = gg + kGgRow * P.nRad, *acc = fv + 32;
    // each warp's FP64 running sums over its units, after all warps' scratch
    const int nacc = 2 * NZ * nslot;
    double* wacc_all = reinterpret_cast<double*>(
        (reinterpret_cast<uintptr_t>(wbase - (size_t)warp * Q.wwords + (size_t)nw * Q.wwords) + 7) & ~(uintptr_t)7);
    double* wacc = wacc_all + (size_t)warp * nacc;
    for (int i = lane; i < nacc; i += 32) wacc[i] = 0.0;
    for (int i = threadIdx.x; i < ntab; i += blockDim.x) {
        const FT z = ((const FT*)P.zeta)[i];
        pk[i + i / nslot] = pk_entry<FT>(z, ((const FT*)P.D)[i], (FT)((double)z * 1.4426950408889634074));
    }
    for (int i = threadIdx.x; i < P.nRad * P.NZ; i += blockDim.x)
        sn[i] = radial_count((const FT*)P.D, i % P.nRad, i / P.nRad, P.nRad, P.K);
    __syncthreads();
    // A slot whose exponent equals that of an earlier slot of the same radial and species
    // (the padding of shorter contractions repeats one exponent) has the same sums
    // sum gg e^{-zeta f} and sum gg e^{-zeta f} f: only the first such slot, its
    // representative, is evaluated, and k_epb_reduce gives the others its sums.
    for (int sg = warp; sg < NZ; sg += nw) {
        int c = 0;
        for (int s0 = 0; s0 < nslot; s0 += 32) {
            const int s = s0 + lane;
            bool rep = false;
            if (s < nslot) {
                const int k = s % P.nRad, m = s / P.nRad;
                FT z, d, l;
                tb.get(s + nslot * sg, sg, z, d, l);
                rep = true;
                for (int m2 = 0; m2 < m && rep; ++m2) {
                    FT z2;
                    tb.get(k + P.nRad * (m2 + P.K * sg), sg, z2, d, l);
                    rep = z2 != z;
                }
            }
            const unsigned b = __ballot_sync(0xffffffffu, rep);
            if (rep) srep[sg * nslot + c + __popc(b & ((1u << lane) - 1u))] = s;
            c += __popc(b);
        }
        if (lane == 0) snrep[sg] = c;
    }
    __syncthreads();
    const long long nunits = (P.nX + kEpbUnit - 1) / kEpbUnit;
    const FT* dPin = (const FT*)P.dPin;
    const FT* Xin = (const FT*)P.X;
    const FT sc = (FT)P.scale;
    for (long long u = (long long)blockIdx.x * nw + warp; u < nunits; u += (long long)gridDim.x * nw) {
        for (int i = lane; i < 2 * NZ * nslot; i += 32) acc[i] = FT(0);
        const long long j0 = u * kEpbUnit, j1 = min(P.nX, j0 + kEpbUnit);
        for (long long c0 = j0; c0 < j1; c0 += 32) {
            // phase A: lane = point
            const long long j = c0 + lane;
            int sg = -1;
            if (j < j1) {
                sg = (int)P.sidx[j] - 1;
                if (sg < 0 || sg >= NZ) {
                    atomicCAS(P.err, 0, AOK_ERR_SPECIES);
                    sg = -1;
                    if (P.dX) {
                        FT* dX = (FT*)P.dX;
                        dX[3 * j] = dX[3 * j + 1] = dX[3 * j + 2] = FT(0);
                    }
                }
            }
            const bool valid = sg >= 0;
            const int sgr = valid ? sg : 0;  // a table row for the lanes that add nothing
            {
                FT r;
                if constexpr (RAD) {
                    r = valid ? Xin[j] : FT(0);
                    for (int k = 0; k < P.nRad; ++k) gg[k * kGgRow + lane] = valid ? dPin[j + P.nX * k] : FT(0);
                } else if constexpr (REG) {
                    FT x = FT(0), y = FT(0), z = FT(1);
                    if (valid) {
                        x = Xin[3 * j];
                        y = Xin[3 * j + 1];
                        z = Xin[3 * j + 2];
                        if (sc != FT(1)) {
                            x = sc * x;
                            y = sc * y;
                            z = sc * z;
                        }
                    }
                    r = norm3(x, y, z);
                    FT Zr[nY], Gr[3 * nY];
                    solid_harmonics<FT, L>(x, y, z, P.F, Zr, Gr, 1);
                    const FT ux = x / r, uy = y / r, uz = z / r;
                    FT ax = FT(0), ay = FT(0), az = FT(0);
                    for (int k = 0; k < P.nRad; ++k) {
                        if (Q.blk) {  // block maps: one switch on the radial's l
                            const int l = Q.lk[k];
                            FT gk = FT(0);
                            if (l >= 0 && valid) {
                                FT Rk, dRk;
                                radial_t<FT>(tb, sn, k, sgr, P.nRad, P.K, Q.poly[k], P.slater, r, Rk, dRk);
                                const int o0 = Q.ob[k];
                                switch (l) {
                                    case 0:
                                        gk = pb_block<FT, 0, L>(Rk, dRk, ux, uy, uz, Zr, Gr, dPin, j, P.nX, o0, ax,
                                                                  ay, az);
                                        break;
                                    case 1:
                                        gk = pb_block<FT, 1, L>(Rk, dRk, ux, uy, uz, Zr, Gr, dPin, j, P.nX, o0, ax,
                                                                  ay, az);
                                        break;
                                    case 2:
                                        gk = pb_block<FT, 2, L>(Rk, dRk, ux, uy, uz, Zr, Gr, dPin, j, P.nX, o0, ax,
                                                                  ay, az);
                                        break;
                                    default:
                                        gk = pb_block<FT, 3, L>(Rk, dRk, ux, uy, uz, Zr, Gr, dPin, j, P.nX, o0, ax,
                                                                  ay, az);
                                        break;
                                }
                            }
                            gg[k * kGgRow + lane] = gk;
                            continue;
                        }
                        FT Rk, dRk;
                        radial_t<FT>(tb, sn, k, sgr, P.nRad, P.K, Q.poly[k], P.slater, r, Rk, dRk);
                        FT gk = FT(0);
                        if (valid) {
#pragma unroll
                            for (int yi = 0; yi < nY; ++yi) {
                                const int o = Q.otab[k * nY + yi];
                                if (o < 0) continue;
                                const FT g = dPin[j + P.nX * o];
                                ax += g * ((dRk * ux) * Zr[yi] + Rk * Gr[3 * yi + 0]);
                                ay += g * ((dRk * uy) * Zr[yi] + Rk * Gr[3 * yi + 1]);
                                az += g * ((dRk * uz) * Zr[yi] + Rk * Gr[3 * yi + 2]);
                                gk += g * Zr[yi];
                            }
                        }
                        gg[k * kGgRow + lane] = gk;
                    }
                    if (valid && P.dX) {
                        FT* dX = (FT*)P.dX;
                        dX[3 * j] = sc != FT(1) ? ax * sc : ax;
                        dX[3 * j + 1] = sc != FT(1) ? ay * sc : ay;
                        dX[3 * j + 2] = sc != FT(1) ? az * sc : az;
                    }
                } else {
                    FT x = FT(0), y = FT(0), z = FT(1);
                    if (valid) {
                        x = Xin[3 * j];
                        y = Xin[3 * j + 1];
                        z = Xin[3 * j + 2];
                        if (sc != FT(1)) {
                            x = sc * x;
                            y = sc * y;
                            z = sc * z;
                        }
                    }
                    r = norm3(x, y, z);
                    for (int k = 0; k < P.nRad; ++k) {
                        FT Rk, dRk;
                        radial_t<FT>(tb, sn, k, sgr, P.nRad, P.K, P.poly[k], P.slater, r, Rk, dRk);
                        R[k * 32 + lane] = Rk;
                        dR[k * 32 + lane] = dRk;
                        gg[k * kGgRow + lane] = FT(0);
                    }
                    solid_harmonics<FT, L>(x, y, z, P.F, Z + lane, G + lane, 32);
                    const FT ux = x / r, uy = y / r, uz = z / r;
                    FT ax = FT(0), ay = FT(0), az = FT(0);
                    if (valid) {
                        for (int i = 0; i < P.nOrb; ++i) {
                            const int k = P.iR[i], yi = P.iY[i];
                            const FT g = dPin[j + P.nX * i];
                            const FT rn = R[k * 32 + lane], yl = Z[yi * 32 + lane], dr = dR[k * 32 + lane];
                            ax += g * ((dr * ux) * yl + rn * G[(3 * yi + 0) * 32 + lane]);
                            ay += g * ((dr * uy) * yl + rn * G[(3 * yi + 1) * 32 + lane]);
                            az += g * ((dr * uz) * yl + rn * G[(3 * yi + 2) * 32 + lane]);
                            gg[k * kGgRow + lane] += g * yl;
                        }
                        if (P.dX) {
                            FT* dX = (FT*)P.dX;
                            dX[3 * j] = sc != FT(1) ? ax * sc : ax;
                            dX[3 * j + 1] = sc != FT(1) ? ay * sc : ay;
                            dX[3 * j + 2] = sc != FT(1) ? az * sc : az;
                        }
                    }
                }
                for (int k = 0; k < P.nRad; ++k) {
                    FT rp = FT(1);
                    for (int i = 0; i < P.poly[k]; ++i) rp *= r;
                    gg[k * kGgRow + lane] *= rp;  // zero for the lanes that add nothing
                }
                fv[lane] = P.slater ? r : r * r;
            }
            __syncwarp();
            // phase B: per species present, lane = representative slot (k, m) of sigma,
            // the points in order
            for (int sigma = 0; sigma < NZ; ++sigma) {
                const unsigned msk = __ballot_sync(0xffffffffu, sg == sigma);
                if (msk == 0u) continue;
                const int nr = snrep[sigma];
#pragma unroll
                for (int g = 0; g < kEpbMaxGroups; ++g) {
                    const int rr = g * 32 + lane;
                    if (g * 32 < nr && rr < nr) {
                        const int s = srep[sigma * nslot + rr];
                        const int k = s % P.nRad;
                        FT zk, dk, zl;
                        tb.get(s + nslot * sigma, sigma, zk, dk, zl);
                        FT* aDp = acc + sigma * nslot + s;
                        FT* aZp = aDp + NZ * nslot;
                        FT aD = *aDp, aZ = *aZp;
                        unsigned m = msk;
                        while (m) {
                            const int t = __ffs(m) - 1;
                            m &= m - 1u;
                            const FT f = fv[t], w = gg[k * kGgRow + t];
                            const FT ex = exp_neg(zk, zl, f) * w;
                            aD += ex;
                            aZ = fma(ex, f, aZ);
                        }
                        *aDp = aD;
                        *aZp = aZ;
                    }
                }
            }
            __syncwarp();
        }
        // the unit's sums into the warp's FP64 running sums: sum gg e^{-zeta f} (dD), then
        // sum gg e^{-zeta f} f (dzeta = -D times its total); zero for the slots that are
        // not representatives
        for (int i = lane; i < nacc; i += 32) wacc[i] += (double)acc[i];
        __syncwarp();
    }
    // the block's partial row: its warps' sums in warp order (the units of each warp
    // are fixed by the launch shape, so the result is reproducible)
    __syncthreads();
    for (int i = threadIdx.x; i < nacc; i += blockDim.x) {
        double sum = 0.0;
        for (int w = 0; w < nw; ++w) sum += wacc_all[(size_t)w * nacc + i];
        Q.partial[(size_t)i * Q.ucap + blockIdx.x] = sum;
    }
}

// dD, dzeta of slot (k, m, sigma): one block of kEpbRedThreads per output value.
// Thread t adds the unit rows t, t + kEpbRedThreads, ... (four loads in flight);
// the threads' sums are added by a fixed tree, so the result is reproducible.
constexpr int kEpbRedThreads = 256;
template <typename FT>
__global__ void __launch_bounds__(kEpbRedThreads) k_epb_reduce(FT* __restrict__ dD, FT* __restrict__ dzeta,
                                                               const double* __restrict__ partial,
                                                               const FT* __restrict__ zeta, const FT* __restrict__ D,
                                                               int nRad, int K, int nout, int nunits, int ucap) {
    __shared__ double ws[kEpbRedThreads / 32];
    const int t = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int kind = t / nout, o = t - kind * nout;  // o = slot + nRad K species
    // the representative of slot o: the first slot of its radial and species with its exponent
    const int k = o % nRad, m = (o / nRad) % K, base = o - k - nRad * m;
    int orep = o;
    for (int m2 = 0; m2 < m; ++m2)
        if (zeta[base + k + nRad * m2] == zeta[o]) {
            orep = base + k + nRad * m2;
            break;
        }
    const double* row = partial + ((size_t)kind * nout + orep) * ucap;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int v = threadIdx.x;
    for (; v + 3 * kEpbRedThreads < nunits; v += 4 * kEpbRedThreads) {
        s0 += row[v];
        s1 += row[v + kEpbRedThreads];
        s2 += row[v + 2 * kEpbRedThreads];
        s3 += row[v + 3 * kEpbRedThreads];
    }
    for (; v < nunits; v += kEpbRedThreads) s0 += row[v];
    double sum = (s0 + s1) + (s2 + s3);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off);
    if (lane == 0) ws[warp] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < kEpbRedThreads / 32; ++w) tot += ws[w];
        if (kind == 0) dD[o] = (FT)tot;
        else dzeta[o] = (FT)(-(double)D[o] * tot);
    }
}

// the partial rows of one slot-parallel pullback call, summed (k_epb_reduce)
static int launch_epb_reduce(aok_orbitals* o, void* dD, void* dzeta, const EpbParams& Q, cudaStream_t s) {
    const int nout = (int)(o->nRad * o->K * o->NZ), nunits = Q.nrows;
    const int nRad = (int)o->nRad, K = (int)o->K;
    if (o->prec == AOK_PREC_F64)
        k_epb_reduce<double><<<2 * nout, kEpbRedThreads, 0, s>>>((double*)dD, (double*)dzeta, Q.partial,
                                                                  (const double*)Q.E.zeta, (const double*)Q.E.D,
                                                                  nRad, K, nout, nunits, Q.ucap);
    else
        k_epb_reduce<float><<<2 * nout, kEpbRedThreads, 0, s>>>((float*)dD, (float*)dzeta, Q.partial,
                                                                 (const float*)Q.E.zeta, (const float*)Q.E.D, nRad,
                                                                 K, nout, nunits, Q.ucap);
    return cuda_status(cudaGetLastError(), "k_epb_reduce");
}

template <typename FT>
__global__ void k_eval_reduce(FT* __restrict__ dD, FT* __restrict__ dzeta, const double* __restrict__ rows, int nrows,
                              int ntab) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * ntab) return;
    double s = 0.0;
    for (int r = 0; r < nrows; ++r) s += rows[(size_t)r * 2 * ntab + t];
    if (t < ntab) dD[t] = (FT)s;
    else dzeta[t - ntab] = (FT)s;
}

// ---------------------------------------------------------------------------
// The radial layer on its own (GaussianTypeRadials / SlaterTypeRadials
// evaluate and evaluate_ed, gtostoradials.jl:117-185): R[j,k] (nX, nRad) and
// dR/dr from the radii r (nX) and species indices.  One thread per point; the
// blocks stay resident and stride over the points, staging the (zeta, D)
// tables and the per-(radial, species) primitive counts once.  A point's
// nRad values go to nRad columns, so the stores of a warp are coalesced per
// column.  A species index outside 1..NZ sets the error word and the point is
// evaluated as species 1 (as in evaluate).
// ---------------------------------------------------------------------------
template <typename FT, bool ED>
__global__ void __launch_bounds__(kEvalThreads) k_radials(const __grid_constant__ EvalParams P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ntab = P.nRad * P.K * P.NZ;
    FT* sz = reinterpret_cast<FT*>(smem_raw);
    FT* sD = sz + ntab;
    FT* sl = sD + ntab;
    int* sn = reinterpret_cast<int*>(sl + ntab);
    for (int i = threadIdx.x; i < ntab; i += blockDim.x) {
        sz[i] = ((const FT*)P.zeta)[i];
        sD[i] = ((const FT*)P.D)[i];
        sl[i] = (FT)((double)((const FT*)P.zeta)[i] * 1.4426950408889634074);
    }
    for (int i = threadIdx.x; i < P.nRad * P.NZ; i += blockDim.x)
        sn[i] = radial_count((const FT*)P.D, i % P.nRad, i / P.nRad, P.nRad, P.K);
    __syncthreads();
    const FT* rin = (const FT*)P.X;
    FT* Rout = (FT*)P.P;
    FT* dRout = (FT*)P.dP;
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < P.nX;
         j += (long long)gridDim.x * blockDim.x) {
        const FT r = rin[j];
        int sg = (int)P.sidx[j] - 1;
        if (sg < 0 || sg >= P.NZ) {
            atomicCAS(P.err, 0, AOK_ERR_SPECIES);
            sg = 0;
        }
        for (int k = 0; k < P.nRad; ++k) {
            FT R, dR;
            radial<FT>(sz, sD, sl, sn, k, sg, P.nRad, P.K, P.poly[k], P.slater, r, R, dR);
            __stcs(Rout + j + P.nX * k, R);
            if constexpr (ED) __stcs(dRout + j + P.nX * k, dR);
        }
    }
}

static size_t eval_smem_bytes(const aok_orbitals* o, bool pb) {
    const size_t fsz = o->prec == AOK_PREC_F64 ? 8 : 4;
    const int nY = (o->L + 1) * (o->L + 1);
    const size_t ntab = (size_t)(o->nRad * o->K * o->NZ);
    size_t b = (3 * ntab + (size_t)count_words((int)o->nRad, (int)o->NZ, (int)fsz) +
                (size_t)(2 * o->nRad + 4 * nY) * kEvalThreads) * fsz;
    if (pb) b = (b + 7) / 8 * 8 + (size_t)(kEvalThreads / 32) * 2 * ntab * 8;
    return b;
}

template <typename FT, int L>
static int launch_eval_L(aok_orbitals* o, EvalParams& P, bool grad, bool pb, cudaStream_t s) {
    const size_t smem = eval_smem_bytes(o, pb);
    if (smem > 227 * 1024) return set_error(AOK_ERR_UNSUPPORTED, "evaluate: basis too large for shared memory");
    int grid = (int)((P.nX + kEvalThreads - 1) / kEvalThreads);
    if (pb) {
        auto k = k_evaluate_pb<FT, L>;
        AOK_TRY_PB(kernel_prepare((const void*)k, smem, kEvalThreads, nullptr));
        k<<<grid, kEvalThreads, smem, s>>>(P);
        return cuda_status(cudaGetLastError(), "k_evaluate_pb");
    }
    // resident blocks striding over the points (k_evaluate)
    auto k = grad ? k_evaluate<FT, L, true> : k_evaluate<FT, L, false>;
    int occ = 0;
    AOK_TRY_PB(kernel_prepare((const void*)k, smem, kEvalThreads, &occ));
    grid = std::max(1, std::min(grid, o->num_sms * std::max(occ, 1)));
    k<<<grid, kEvalThreads, smem, s>>>(P);
    return cuda_status(cudaGetLastError(), "k_evaluate");
}

template <typename FT>
static int launch_eval_T(aok_orbitals* o, EvalParams& P, bool grad, bool pb, cudaStream_t s) {
    switch (o->L) {
        case 0: return launch_eval_L<FT, 0>(o, P, grad, pb, s);
        case 1: return launch_eval_L<FT, 1>(o, P, grad, pb, s);
        case 2: return launch_eval_L<FT, 2>(o, P, grad, pb, s);
        case 3: return launch_eval_L<FT, 3>(o, P, grad, pb, s);
        case 4: return launch_eval_L<FT, 4>(o, P, grad, pb, s);
        default: return set_error(AOK_ERR_UNSUPPORTED, "evaluate: harmonics above l = 4");
    }
}

static void fill_params(aok_orbitals* o, EvalParams& P, const void* X, const int64_t* sidx, const void* zeta,
                        const void* D, int64_t nX, double lengthscale) {
    memset(&P, 0, sizeof(P));
    P.X = X;
    P.sidx = sidx;
    P.zeta = zeta;
    P.D = D;
    P.poly = o->d_poly;
    P.iR = o->d_iR;
    P.iY = o->d_iY;
    P.err = o->d_err;
    P.nX = nX;
    P.nRad = (int)o->nRad;
    P.K = (int)o->K;
    P.NZ = (int)o->NZ;
    P.nOrb = (int)o->nOrb;
    P.slater = o->radial == AOK_RADIAL_SLATER;
    P.scale = lengthscale;
    for (int l = 0; l <= o->L; ++l)
        for (int m = 0; m <= l; ++m) {
            double fac = 1.0;
            for (int q = l - m + 1; q <= l + m; ++q) fac /= (double)q;
            P.F[l * l + l + m] = std::sqrt((2.0 * l + 1.0) / (4.0 * 3.14159265358979323846) * fac);
        }
}

// Block maps: every radial k that any orbital uses feeds exactly the 2l+1
// orbitals ob[k] .. ob[k] + 2l, in harmonic order l^2 .. l^2 + 2l (the layout
// the reference's AtomicOrbitals builds, atomicorbitals.jl:56-75).  Fills lk, ob.
static bool block_maps(const aok_orbitals* o, int8_t* lk, int16_t* ob) {
    if (o->nRad > kRegMaxRad) return false;
    for (int64_t k = 0; k < o->nRad; ++k) {
        lk[k] = -1;
        ob[k] = 0;
    }
    std::vector<int> cnt((size_t)o->nRad, 0);
    for (int64_t i = 0; i < o->nOrb; ++i) {
        const int64_t k = o->iR[i] - 1, yi = o->iY[i] - 1;
        int& c = cnt[(size_t)k];
        if (c == 0) {  // the radial's first orbital opens its block at m = 0
            int l = 0;
            while ((l + 1) * (l + 1) <= yi) ++l;
            if (yi != l * l || l > kRegMaxL || i > 32767) return false;
            lk[k] = (int8_t)l;
            ob[k] = (int16_t)i;
        } else if (i != ob[k] + c || yi != lk[k] * lk[k] + c || c > 2 * lk[k]) {
            return false;
        }
        ++c;
    }
    for (int64_t k = 0; k < o->nRad; ++k)
        if (cnt[(size_t)k] != 0 && cnt[(size_t)k] != 2 * lk[k] + 1) return false;
    return true;
}

// The register-path forward when the maps allow it (L <= 3, nRad <= 64, each
// (radial, harmonic) pair at most once, radial powers < 128); returns -1 otherwise.
template <typename FT, int L>
static int launch_eval_reg_L(aok_orbitals* o, const EvalParams& P, bool grad, cudaStream_t s) {
    constexpr int nY = (L + 1) * (L + 1);
    EvalRegParams Q;
    memset(&Q, 0, sizeof(Q));
    Q.E = P;
    for (int i = 0; i < kRegMaxRad * (kRegMaxL + 1) * (kRegMaxL + 1); ++i) Q.otab[i] = -1;
    for (int64_t i = 0; i < o->nOrb; ++i) {
        const int64_t k = o->iR[i] - 1, yi = o->iY[i] - 1;
        int16_t& e = Q.otab[k * nY + yi];
        if (e >= 0) return -1;  // a repeated (radial, harmonic) pair: the general kernel
        e = (int16_t)i;
    }
    for (int64_t k = 0; k < o->nRad; ++k) {
        if (o->poly[k] > 127) return -1;
        Q.poly[k] = (int8_t)o->poly[k];
    }
    const bool blk = block_maps(o, Q.lk, Q.ob);
    const size_t fsz = sizeof(FT);
    const size_t smem =
        (4 * (size_t)(o->nRad * o->K * o->NZ + o->NZ) + count_words((int)o->nRad, (int)o->NZ, (int)fsz)) * fsz;
    if (smem > 227 * 1024) return -1;
    void* k = blk ? (grad ? (void*)k_evaluate_reg<FT, L, true, true> : (void*)k_evaluate_reg<FT, L, false, true>)
                  : (grad ? (void*)k_evaluate_reg<FT, L, true> : (void*)k_evaluate_reg<FT, L, false>);
    int occ = 0;
    AOK_TRY_PB(kernel_prepare(k, smem, kEvalThreads, &occ));
    const int grid = (int)std::max<int64_t>(
        1, std::min<int64_t>((P.nX + kEvalThreads - 1) / kEvalThreads, (int64_t)o->num_sms * std::max(occ, 1)));
    void* args[] = {&Q};
    return cuda_status(cudaLaunchKernel(k, dim3(grid), dim3(kEvalThreads), args, smem, s), "k_evaluate_reg");
}

template <typename FT>
static int launch_eval_reg(aok_orbitals* o, const EvalParams& P, bool grad, cudaStream_t s) {
    if (o->nRad > kRegMaxRad) return -1;
    switch (o->L) {
        case 0: return launch_eval_reg_L<FT, 0>(o, P, grad, s);
        case 1: return launch_eval_reg_L<FT, 1>(o, P, grad, s);
        case 2: return launch_eval_reg_L<FT, 2>(o, P, grad, s);
        case 3: return launch_eval_reg_L<FT, 3>(o, P, grad, s);
        default: return -1;
    }
}

int launch_evaluate(aok_orbitals* o, void* Pv, void* dP, const void* X, const int64_t* sidx, const void* zeta,
                    const void* D, int64_t nX, double lengthscale, cudaStream_t s) {
    EvalParams P;
    fill_params(o, P, X, sidx, zeta, D, nX, lengthscale);
    P.P = Pv;
    P.dP = dP;
    const int st = o->prec == AOK_PREC_F64 ? launch_eval_reg<double>(o, P, dP != nullptr, s)
                                           : launch_eval_reg<float>(o, P, dP != nullptr, s);
    if (st != -1) return st;
    if (o->prec == AOK_PREC_F64) return launch_eval_T<double>(o, P, dP != nullptr, false, s);
    return launch_eval_T<float>(o, P, dP != nullptr, false, s);
}

// partial rows of the slot-parallel pullback: one per block of a launch, so at most
// one per unit and at most 8 per SM (its blocks are at least 256 threads)
static int ensure_epb_buffers(aok_orbitals* o, int64_t nX) {
    const int64_t units = std::min<int64_t>((nX + kEpbUnit - 1) / kEpbUnit, (int64_t)o->num_sms * 8);
    if (units <= o->epb_ucap && o->d_epb_partial) return AOK_OK;
    if (o->d_epb_partial) cudaFree(o->d_epb_partial);
    o->d_epb_partial = nullptr;
    o->epb_ucap = 0;
    cudaError_t e = cudaMalloc(&o->d_epb_partial, sizeof(double) * (size_t)units * 2 * o->nRad * o->K * o->NZ);
    if (e != cudaSuccess) return cuda_status(e, "cudaMalloc(evaluate pullback rows)");
    o->epb_ucap = units;
    return AOK_OK;
}

// Blocks of the slot-parallel pullback: as many warps (up to 8) as the per-warp
// shared memory allows, and the resident blocks per SM from the occupancy query.
static int launch_epb_kernel(aok_orbitals* o, const void* k, EpbParams& Q, size_t tab, size_t wbytes,
                             cudaStream_t s, const char* what) {
    // per warp: the FT scratch and accumulators, then (after all warps' scratch) its FP64 sums
    const size_t wd = sizeof(double) * epb_acc_words((int)o->nRad, (int)o->K, (int)o->NZ);
    int nw = 8;
    while (nw > 1 && tab + nw * (wbytes + wd) + 8 > 227 * 1024) --nw;
    const size_t smem = tab + nw * (wbytes + wd) + 8;
    if (smem > 227 * 1024) return set_error(AOK_ERR_UNSUPPORTED, std::string(what) + ": basis too large");
    int occ = 0;
    AOK_TRY_PB(kernel_prepare(k, smem, 32 * nw, &occ));
    Q.wwords = (int)(wbytes / (o->prec == AOK_PREC_F64 ? 8 : 4));
    const int64_t units = (Q.E.nX + kEpbUnit - 1) / kEpbUnit;
    const int64_t want = (units + nw - 1) / nw;
    // one partial row per block: no more blocks than the rows allocated
    const int grid = (int)std::max<int64_t>(
        1, std::min<int64_t>(std::min<int64_t>(want, (int64_t)o->num_sms * std::max(occ, 1)), Q.ucap));
    Q.nrows = grid;
    void* args[] = {&Q};
    return cuda_status(cudaLaunchKernel(k, dim3(grid), dim3(32 * nw), args, smem, s), what);
}

template <typename FT, int L>
static int launch_epb_L(aok_orbitals* o, EpbParams& Q, cudaStream_t s) {
    constexpr int nY = (L + 1) * (L + 1);
    const size_t fsz = sizeof(FT);
    const size_t tab =
        (4 * (size_t)(o->nRad * o->K * o->NZ + o->NZ) + epb_int_words((int)o->nRad, (int)o->K, (int)o->NZ, (int)fsz)) *
        fsz;
    const size_t accw = epb_acc_words((int)o->nRad, (int)o->K, (int)o->NZ);
    if constexpr (L <= kRegMaxL) {
        // the register path when every (radial, harmonic) pair is used at most once
        bool ok = o->nRad <= kRegMaxRad;
        for (int i = 0; ok && i < kRegMaxRad * nY; ++i) Q.otab[i] = -1;
        for (int64_t i = 0; ok && i < o->nOrb; ++i) {
            int16_t& e = Q.otab[(o->iR[i] - 1) * nY + (o->iY[i] - 1)];
            if (e >= 0) ok = false;
            else e = (int16_t)i;
        }
        for (int64_t k = 0; ok && k < o->nRad; ++k) {
            if (o->poly[k] > 127) ok = false;
            else Q.poly[k] = (int8_t)o->poly[k];
        }
        Q.blk = ok && block_maps(o, Q.lk, Q.ob) ? 1 : 0;
        const size_t wbytes = (epb_warp_words_reg((int)o->nRad) + accw) * fsz;
        if (ok && tab + wbytes <= 227 * 1024)
            return launch_epb_kernel(o, (const void*)k_evaluate_pbs<FT, L, false, true>, Q, tab, wbytes, s,
                                     "k_evaluate_pbs");
    }
    const size_t wbytes = (epb_warp_words((int)o->nRad, nY) + accw) * fsz;
    return launch_epb_kernel(o, (const void*)k_evaluate_pbs<FT, L>, Q, tab, wbytes, s, "k_evaluate_pbs");
}

template <typename FT>
static int launch_epb_T(aok_orbitals* o, EpbParams& Q, cudaStream_t s) {
    switch (o->L) {
        case 0: return launch_epb_L<FT, 0>(o, Q, s);
        case 1: return launch_epb_L<FT, 1>(o, Q, s);
        case 2: return launch_epb_L<FT, 2>(o, Q, s);
        case 3: return launch_epb_L<FT, 3>(o, Q, s);
        case 4: return launch_epb_L<FT, 4>(o, Q, s);
        default: return set_error(AOK_ERR_UNSUPPORTED, "evaluate: harmonics above l = 4");
    }
}

int launch_evaluate_pb(aok_orbitals* o, void* dX, void* dzeta, void* dD, const void* dPin, const void* X,
                       const int64_t* sidx, const void* zeta, const void* D, int64_t nX, double lengthscale,
                       cudaStream_t s) {
    EvalParams P;
    fill_params(o, P, X, sidx, zeta, D, nX, lengthscale);
    P.dPin = dPin;
    P.dX = dX;
    const int nslot = (int)(o->nRad * o->K);
    if (dzeta && dD && nslot <= 32 * kEpbMaxGroups) {
        // slot-parallel: units of consecutive points, lanes = (radial, primitive) slots per species
        AOK_TRY_PB(ensure_epb_buffers(o, nX));
        EpbParams Q;
        memset(&Q, 0, sizeof(Q));
        Q.E = P;
        Q.partial = (double*)o->d_epb_partial;
        Q.ucap = (int)o->epb_ucap;
        const int st = o->prec == AOK_PREC_F64 ? launch_epb_T<double>(o, Q, s) : launch_epb_T<float>(o, Q, s);
        if (st != AOK_ERR_UNSUPPORTED) {
            AOK_TRY_PB(st);
            return launch_epb_reduce(o, dD, dzeta, Q, s);
        }
        // a basis whose per-warp scratch does not fit: the per-block-rows kernel below
    }
    const int grid = (int)((nX + kEvalThreads - 1) / kEvalThreads);
    const int ntab = (int)(o->nRad * o->K * o->NZ);
    if (dzeta && dD) {
        if (grid > o->max_blocks) {
            if (o->d_partials) cudaFree(o->d_partials);
            o->d_partials = nullptr;
            cudaError_t e = cudaMalloc(&o->d_partials, sizeof(double) * 2 * ntab * (size_t)grid);
            if (e != cudaSuccess) return cuda_status(e, "cudaMalloc(evaluate partials)");
            o->max_blocks = grid;
        }
        P.rows = (double*)o->d_partials;
    }
    int st = o->prec == AOK_PREC_F64 ? launch_eval_T<double>(o, P, true, true, s)
                                     : launch_eval_T<float>(o, P, true, true, s);
    if (st != AOK_OK || !P.rows) return st;
    if (o->prec == AOK_PREC_F64)
        k_eval_reduce<double><<<(2 * ntab + 127) / 128, 128, 0, s>>>((double*)dD, (double*)dzeta, P.rows, grid, ntab);
    else
        k_eval_reduce<float><<<(2 * ntab + 127) / 128, 128, 0, s>>>((float*)dD, (float*)dzeta, P.rows, grid, ntab);
    return cuda_status(cudaGetLastError(), "k_eval_reduce");
}

// radial layer forward: R (and dR) at the radii r
int launch_radials(aok_orbitals* o, void* R, void* dR, const void* r, const int64_t* sidx, const void* zeta,
                   const void* D, int64_t nX, cudaStream_t s) {
    EvalParams P;
    fill_params(o, P, r, sidx, zeta, D, nX, 1.0);
    P.P = R;
    P.dP = dR;
    const size_t fsz = o->prec == AOK_PREC_F64 ? 8 : 4;
    const size_t smem = (3 * (size_t)(o->nRad * o->K * o->NZ) + count_words((int)o->nRad, (int)o->NZ, (int)fsz)) * fsz;
    if (smem > 227 * 1024) return set_error(AOK_ERR_UNSUPPORTED, "radials: basis too large for shared memory");
    void* k;
    if (o->prec == AOK_PREC_F64) k = dR ? (void*)k_radials<double, true> : (void*)k_radials<double, false>;
    else k = dR ? (void*)k_radials<float, true> : (void*)k_radials<float, false>;
    int occ = 0;
    AOK_TRY_PB(kernel_prepare(k, smem, kEvalThreads, &occ));
    const int grid = (int)std::max<int64_t>(
        1, std::min<int64_t>((nX + kEvalThreads - 1) / kEvalThreads, (int64_t)o->num_sms * std::max(occ, 1)));
    void* args[] = {&P};
    return cuda_status(cudaLaunchKernel(k, dim3(grid), dim3(kEvalThreads), args, smem, s), "k_radials");
}

// radial layer pullback: (dzeta, dD) from dR (nX, nRad), slot-parallel over species-binned points
int launch_radials_pb(aok_orbitals* o, void* dzeta, void* dD, const void* dRin, const void* r, const int64_t* sidx,
                      const void* zeta, const void* D, int64_t nX, cudaStream_t s) {
    EvalParams P;
    fill_params(o, P, r, sidx, zeta, D, nX, 1.0);
    P.dPin = dRin;
    const int nslot = (int)(o->nRad * o->K);
    if (nslot > 32 * kEpbMaxGroups)
        return set_error(AOK_ERR_UNSUPPORTED, "radials pullback: more than 128 (radial, primitive) slots");
    AOK_TRY_PB(ensure_epb_buffers(o, nX));
    EpbParams Q;
    memset(&Q, 0, sizeof(Q));
    Q.E = P;
    Q.partial = (double*)o->d_epb_partial;
    Q.ucap = (int)o->epb_ucap;
    const size_t fsz = o->prec == AOK_PREC_F64 ? 8 : 4;
    const size_t tab =
        (4 * (size_t)(o->nRad * o->K * o->NZ + o->NZ) + epb_int_words((int)o->nRad, (int)o->K, (int)o->NZ, (int)fsz)) *
        fsz;
    const size_t wbytes =
        (epb_warp_words((int)o->nRad, 1) + epb_acc_words((int)o->nRad, (int)o->K, (int)o->NZ)) * fsz;
    const void* k = o->prec == AOK_PREC_F64 ? (const void*)k_evaluate_pbs<double, 0, true>
                                            : (const void*)k_evaluate_pbs<float, 0, true>;
    AOK_TRY_PB(launch_epb_kernel(o, k, Q, tab, wbytes, s, "k_evaluate_pbs (radial)"));
    return launch_epb_reduce(o, dD, dzeta, Q, s);
}

}  // namespace aok

using namespace aok;

extern "C" {

int aok_orbitals_create(aok_orbitals** out, int64_t nRad, int64_t K, int64_t NZ, const int64_t* poly, int64_t nOrb,
                        const int64_t* iR, const int64_t* iY, int64_t L, int radial_kind, int precision) {
    if (!out || !poly || !iR || !iY) return set_error(AOK_ERR_INVALID, "aok_orbitals_create: null pointer");
    *out = nullptr;
    if (nRad <= 0 || K <= 0 || NZ <= 0 || nOrb <= 0 || L < 0)
        return set_error(AOK_ERR_INVALID, "aok_orbitals_create: sizes must be positive");
    if (L > kEvalMaxL) return set_error(AOK_ERR_UNSUPPORTED, "aok_orbitals_create: harmonics above l = 4");
    if (radial_kind != AOK_RADIAL_GAUSSIAN && radial_kind != AOK_RADIAL_SLATER)
        return set_error(AOK_ERR_INVALID, "aok_orbitals_create: unknown radial kind");
    if (precision != AOK_PREC_F64 && precision != AOK_PREC_F32C)
        return set_error(AOK_ERR_INVALID, "aok_orbitals_create: unknown precision");
    const int64_t nY = (L + 1) * (L + 1);
    std::vector<int> p32(nRad), r32(nOrb), y32(nOrb);
    for (int64_t k = 0; k < nRad; ++k) {
        if (poly[k] < 0 || poly[k] > 64) return set_error(AOK_ERR_INVALID, "aok_orbitals_create: bad radial power");
        p32[k] = (int)poly[k];
    }
    for (int64_t i = 0; i < nOrb; ++i) {
        if (iR[i] < 1 || iR[i] > nRad || iY[i] < 1 || iY[i] > nY)
            return set_error(AOK_ERR_INVALID, "aok_orbitals_create: orbital index map out of range");
        r32[i] = (int)(iR[i] - 1);
        y32[i] = (int)(iY[i] - 1);
    }
    aok_orbitals* o = new aok_orbitals();
    o->nRad = nRad;
    o->K = K;
    o->NZ = NZ;
    o->nOrb = nOrb;
    o->L = (int)L;
    o->radial = radial_kind;
    o->prec = precision;
    o->poly.assign(poly, poly + nRad);
    o->iR.assign(iR, iR + nOrb);
    o->iY.assign(iY, iY + nOrb);
    auto fail = [&](int code) {
        aok_orbitals_destroy(o);
        return code;
    };
    int st;
    if ((st = cuda_status(cudaGetDevice(&o->device), "cudaGetDevice"))) return fail(st);
    if ((st = cuda_status(cudaDeviceGetAttribute(&o->num_sms, cudaDevAttrMultiProcessorCount, o->device),
                          "cudaDeviceGetAttribute")))
        return fail(st);
    if ((st = cuda_status(cudaMalloc(&o->d_poly, sizeof(int) * nRad), "cudaMalloc(poly)")) ||
        (st = cuda_status(cudaMalloc(&o->d_iR, sizeof(int) * nOrb), "cudaMalloc(iR)")) ||
        (st = cuda_status(cudaMalloc(&o->d_iY, sizeof(int) * nOrb), "cudaMalloc(iY)")) ||
        (st = cuda_status(cudaMalloc(&o->d_err, sizeof(int)), "cudaMalloc(err)")))
        return fail(st);
    if ((st = cuda_status(cudaMemcpy(o->d_poly, p32.data(), sizeof(int) * nRad, cudaMemcpyHostToDevice), "memcpy")) ||
        (st = cuda_status(cudaMemcpy(o->d_iR, r32.data(), sizeof(int) * nOrb, cudaMemcpyHostToDevice), "memcpy")) ||
        (st = cuda_status(cudaMemcpy(o->d_iY, y32.data(), sizeof(int) * nOrb, cudaMemcpyHostToDevice), "memcpy")) ||
        (st = cuda_status(cudaMemset(o->d_err, 0, sizeof(int)), "memset")))
        return fail(st);
    if (eval_smem_bytes(o, true) > 227 * 1024)
        return fail(set_error(AOK_ERR_UNSUPPORTED, "aok_orbitals_create: basis too large for shared memory"));
    *out = o;
    return AOK_OK;
}

int aok_orbitals_destroy(aok_orbitals* o) {
    if (!o) return AOK_OK;
    void* bufs[] = {o->d_poly,        o->d_iR,          o->d_iY,          o->d_partials,      o->d_err,
                    o->d_epb_partial};
    for (void* b : bufs)
        if (b) cudaFree(b);
    delete o;
    return AOK_OK;
}

int aok_orbitals_check(aok_orbitals* o, void* stream) {
    if (!o) return set_error(AOK_ERR_INVALID, "aok_orbitals_check: null plan");
    int st = cuda_status(cudaStreamSynchronize((cudaStream_t)stream), "cudaStreamSynchronize");
    if (st != AOK_OK) return st;
    int h = 0;
    if ((st = cuda_status(cudaMemcpy(&h, o->d_err, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy(err)")))
        return st;
    if ((st = cuda_status(cudaMemset(o->d_err, 0, sizeof(int)), "cudaMemset(err)"))) return st;
    if (h == AOK_ERR_SPECIES) return set_error(h, "species index outside 1..NZ");
    if (h != 0) return set_error(h, "device-side validation failed");
    return AOK_OK;
}

int aok_evaluate(aok_orbitals* o, void* P, const void* X, const int64_t* sidx, const void* zeta, const void* D,
                 int64_t nX, double lengthscale, void* stream) {
    if (!o) return set_error(AOK_ERR_INVALID, "aok_evaluate: null plan");
    if (nX < 0) return set_error(AOK_ERR_INVALID, "aok_evaluate: negative nX");
    if (nX == 0) return AOK_OK;
    if (!P || !X || !sidx || !zeta || !D) return set_error(AOK_ERR_INVALID, "aok_evaluate: null pointer");
    return launch_evaluate(o, P, nullptr, X, sidx, zeta, D, nX, lengthscale, (cudaStream_t)stream);
}

int aok_evaluate_ed(aok_orbitals* o, void* P, void* dP, const void* X, const int64_t* sidx, const void* zeta,
                    const void* D, int64_t nX, double lengthscale, void* stream) {
    if (!o) return set_error(AOK_ERR_INVALID, "aok_evaluate_ed: null plan");
    if (nX < 0) return set_error(AOK_ERR_INVALID, "aok_evaluate_ed: negative nX");
    if (nX == 0) return AOK_OK;
    if (!P || !dP || !X || !sidx || !zeta || !D) return set_error(AOK_ERR_INVALID, "aok_evaluate_ed: null pointer");
    return launch_evaluate(o, P, dP, X, sidx, zeta, D, nX, lengthscale, (cudaStream_t)stream);
}

int aok_evaluate_pullback(aok_orbitals* o, void* dX, void* dzeta, void* dD, const void* dP, const void* X,
                          const int64_t* sidx, const void* zeta, const void* D, int64_t nX, double lengthscale,
                          void* stream) {
    if (!o) return set_error(AOK_ERR_INVALID, "aok_evaluate_pullback: null plan");
    if ((dzeta == nullptr) != (dD == nullptr))
        return set_error(AOK_ERR_INVALID, "aok_evaluate_pullback: dzeta and dD must both be given or both null");
    if (nX < 0) return set_error(AOK_ERR_INVALID, "aok_evaluate_pullback: negative nX");
    cudaStream_t s = (cudaStream_t)stream;
    const size_t fsz = o->prec == AOK_PREC_F64 ? 8 : 4;
    if (nX == 0) {
        if (dzeta) {
            int st = cuda_status(cudaMemsetAsync(dzeta, 0, fsz * o->nRad * o->K * o->NZ, s), "memset");
            if (st) return st;
            return cuda_status(cudaMemsetAsync(dD, 0, fsz * o->nRad * o->K * o->NZ, s), "memset");
        }
        return AOK_OK;
    }
    if (!dP || !X || !sidx || !zeta || !D) return set_error(AOK_ERR_INVALID, "aok_evaluate_pullback: null pointer");
    return launch_evaluate_pb(o, dX, dzeta, dD, dP, X, sidx, zeta, D, nX, lengthscale, s);
}

// ---- the radial layer (GaussianTypeRadials / SlaterTypeRadials) ----

struct aok_radials {
    aok_orbitals* o = nullptr;  // radial tables, error word and the binned-pullback buffers
};

int aok_radials_create(aok_radials** out, int64_t nRad, int64_t K, int64_t NZ, const int64_t* poly, int radial_kind,
                       int precision) {
    if (!out || !poly) return set_error(AOK_ERR_INVALID, "aok_radials_create: null pointer");
    *out = nullptr;
    const int64_t one = 1;
    aok_orbitals* o = nullptr;
    // one placeholder orbital (radial 1, Z_00): the radial layer uses only the radial half of the plan
    int st = aok_orbitals_create(&o, nRad, K, NZ, poly, 1, &one, &one, 0, radial_kind, precision);
    if (st != AOK_OK) {
        std::string m = aok_last_error();
        const std::string from = "aok_orbitals_create";
        if (m.compare(0, from.size(), from) == 0) m = "aok_radials_create" + m.substr(from.size());
        return set_error(st, m);
    }
    aok_radials* r = new aok_radials();
    r->o = o;
    *out = r;
    return AOK_OK;
}

int aok_radials_destroy(aok_radials* r) {
    if (!r) return AOK_OK;
    aok_orbitals_destroy(r->o);
    delete r;
    return AOK_OK;
}

int aok_radials_check(aok_radials* r, void* stream) {
    if (!r) return set_error(AOK_ERR_INVALID, "aok_radials_check: null plan");
    return aok_orbitals_check(r->o, stream);
}

int aok_radials_evaluate(aok_radials* r, void* R, void* dR, const void* rad, const int64_t* sidx, const void* zeta,
                         const void* D, int64_t nX, void* stream) {
    if (!r) return set_error(AOK_ERR_INVALID, "aok_radials_evaluate: null plan");
    if (nX < 0) return set_error(AOK_ERR_INVALID, "aok_radials_evaluate: negative nX");
    if (nX == 0) return AOK_OK;
    if (!R || !rad || !sidx || !zeta || !D) return set_error(AOK_ERR_INVALID, "aok_radials_evaluate: null pointer");
    return launch_radials(r->o, R, dR, rad, sidx, zeta, D, nX, (cudaStream_t)stream);
}

int aok_radials_pullback(aok_radials* r, void* dzeta, void* dD, const void* dRin, const void* rad,
                         const int64_t* sidx, const void* zeta, const void* D, int64_t nX, void* stream) {
    if (!r) return set_error(AOK_ERR_INVALID, "aok_radials_pullback: null plan");
    if (!dzeta || !dD) return set_error(AOK_ERR_INVALID, "aok_radials_pullback: null pointer");
    if (nX < 0) return set_error(AOK_ERR_INVALID, "aok_radials_pullback: negative nX");
    aok_orbitals* o = r->o;
    cudaStream_t s = (cudaStream_t)stream;
    if (nX == 0) {
        const size_t fsz = o->prec == AOK_PREC_F64 ? 8 : 4;
        int st = cuda_status(cudaMemsetAsync(dzeta, 0, fsz * o->nRad * o->K * o->NZ, s), "memset");
        if (st) return st;
        return cuda_status(cudaMemsetAsync(dD, 0, fsz * o->nRad * o->K * o->NZ, s), "memset");
    }
    if (!dRin || !rad || !sidx || !zeta || !D) return set_error(AOK_ERR_INVALID, "aok_radials_pullback: null pointer");
    return launch_radials_pb(o, dzeta, dD, dRin, rad, sidx, zeta, D, nX, s);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free evaluate pullback.
//
// Some callers cannot allocate device memory when they need this pullback:
// a host framework that owns the whole device through its own pooling
// allocator (and forbids allocations behind its back), or a long-running
// service that reserves its memory at start-up and must not grow later.
// aok_evaluate_pullback allocates twice (the aok_orbitals plan and, on
// first use, its per-block partial rows); this variant needs neither: the
// index maps, the device error word and the per-block FP64 partial rows live
// in one file-scope device array of kNoAllocScratchBytes (8 MiB) that every
// GPU which loads the library holds until the process exits.
//
// The array's host-side name is not a device address, so the first call on
// each device looks up the real address with cudaGetSymbolAddress (with that
// device current) and caches it; make that first call before any stream
// capture.  Every call shares the one array and overwrites it (the error word
// is cleared by each call, every partial row is rewritten), so calls that can
// overlap on the GPU -- on different streams, or on the same device from
// different threads without ordering -- race on it and must be serialised by
// the caller.
// ---------------------------------------------------------------------------
#include <mutex>

namespace aok {

constexpr size_t kNoAllocScratchBytes = (size_t)8 << 20;
constexpr int kNoAllocMaxRad = 64;
constexpr int kNoAllocMaxOrb = 256;
constexpr int kNoAllocMaxK = 64;
constexpr int kNoAllocMaxNZ = 64;
constexpr size_t kNoAllocMapsOffset = 256;        // after the error word
constexpr size_t kNoAllocRowsOffset = 4096;       // after the index maps
static_assert(kNoAllocMapsOffset + sizeof(int) * (kNoAllocMaxRad + 2 * kNoAllocMaxOrb) <= kNoAllocRowsOffset,
              "index maps overflow their region");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static std::mutex g_noalloc_mu;
static void* g_noalloc_ptr[256];

struct NoAllocMaps {
    int nRad, nOrb;
    int poly[kNoAllocMaxRad];
    int iR[kNoAllocMaxOrb];
    int iY[kNoAllocMaxOrb];
};

// copies the index maps (kernel parameters) into the scratch and clears the error word
__global__ void k_noalloc_setup(const __grid_constant__ NoAllocMaps m, unsigned char* scratch) {
    int* err = reinterpret_cast<int*>(scratch);
    int* maps = reinterpret_cast<int*>(scratch + kNoAllocMapsOffset);
    if (threadIdx.x == 0) *err = 0;
    for (int i = threadIdx.x; i < m.nRad; i += blockDim.x) maps[i] = m.poly[i];
    for (int i = threadIdx.x; i < m.nOrb; i += blockDim.x) {
        maps[kNoAllocMaxRad + i] = m.iR[i];
        maps[kNoAllocMaxRad + kNoAllocMaxOrb + i] = m.iY[i];
    }
}

static int noalloc_scratch(unsigned char** out) {
    int dev = 0;
    int st = cuda_status(cudaGetDevice(&dev), "cudaGetDevice");
    if (st != AOK_OK) return st;
    if (dev < 0 || dev >= 256) return set_error(AOK_ERR_UNSUPPORTED, "aok_evaluate_pullback_noalloc: device id");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        st = cuda_status(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(noalloc scratch)");
        if (st != AOK_OK) return st;
        g_noalloc_ptr[dev] = p;
    }
    *out = (unsigned char*)g_noalloc_ptr[dev];
    return AOK_OK;
}

}  // namespace aok

// Reads and clears the scratch's error word on the current device (after
// synchronising `stream`): AOK_ERR_SPECIES if the last allocation-free
// pullback met a species index outside 1..NZ.  Allocates nothing.
extern "C" int aok_evaluate_pullback_noalloc_check(void* stream) {
    using namespace aok;
    int dev = 0;
    int st = cuda_status(cudaGetDevice(&dev), "cudaGetDevice");
    if (st != AOK_OK) return st;
    if (dev < 0 || dev >= 256) return set_error(AOK_ERR_UNSUPPORTED, "aok_evaluate_pullback_noalloc_check: device id");
    unsigned char* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        scratch = (unsigned char*)g_noalloc_ptr[dev];
    }
    if (!scratch) return AOK_OK;  // no allocation-free call has run on this device
    if ((st = cuda_status(cudaStreamSynchronize((cudaStream_t)stream), "cudaStreamSynchronize"))) return st;
    int h = 0;
    if ((st = cuda_status(cudaMemcpy(&h, scratch, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy(err)")))
        return st;
    if ((st = cuda_status(cudaMemset(scratch, 0, sizeof(int)), "cudaMemset(err)"))) return st;
    if (h == AOK_ERR_SPECIES) return set_error(h, "species index outside 1..NZ");
    if (h != 0) return set_error(h, "device-side validation failed");
    return AOK_OK;
}

extern "C" int aok_evaluate_pullback_noalloc(int64_t nRad, int64_t K, int64_t NZ, const int64_t* poly, int64_t nOrb,
                                             const int64_t* iR, const int64_t* iY, int64_t L, int radial_kind,
                                             int precision, void* dX, void* dzeta, void* dD, const void* dP,
                                             const void* X, const int64_t* sidx, const void* zeta, const void* D,
                                             int64_t nX, double lengthscale, void* stream) {
    using namespace aok;
    const char* who = "aok_evaluate_pullback_noalloc";
    if (!poly || !iR || !iY) return set_error(AOK_ERR_INVALID, std::string(who) + ": null pointer");
    if (nRad <= 0 || K <= 0 || NZ <= 0 || nOrb <= 0 || L < 0 || nX < 0)
        return set_error(AOK_ERR_INVALID, std::string(who) + ": sizes must be positive");
    if (L > kEvalMaxL) return set_error(AOK_ERR_UNSUPPORTED, std::string(who) + ": harmonics above l = 4");
    if (radial_kind != AOK_RADIAL_GAUSSIAN && radial_kind != AOK_RADIAL_SLATER)
        return set_error(AOK_ERR_INVALID, std::string(who) + ": unknown radial kind");
    if (precision != AOK_PREC_F64 && precision != AOK_PREC_F32C)
        return set_error(AOK_ERR_INVALID, std::string(who) + ": unknown precision");
    if ((dzeta == nullptr) != (dD == nullptr))
        return set_error(AOK_ERR_INVALID, std::string(who) + ": dzeta and dD must both be given or both null");
    if (nRad > kNoAllocMaxRad || nOrb > kNoAllocMaxOrb)
        return set_error(AOK_ERR_UNSUPPORTED, std::string(who) + ": more than 64 radials or 256 orbitals");
    // bounded before any product is formed, so nRad*K*NZ and the scratch size cannot wrap
    if (K > kNoAllocMaxK || NZ > kNoAllocMaxNZ)
        return set_error(AOK_ERR_UNSUPPORTED, std::string(who) + ": more than 64 primitive slots or 64 species");
    if (nX > (int64_t)INT32_MAX)
        return set_error(AOK_ERR_UNSUPPORTED, std::string(who) + ": nX above 2^31 - 1");
    const int64_t nY = (L + 1) * (L + 1);
    NoAllocMaps maps;
    memset(&maps, 0, sizeof(maps));
    maps.nRad = (int)nRad;
    maps.nOrb = (int)nOrb;
    for (int64_t k = 0; k < nRad; ++k) {
        if (poly[k] < 0 || poly[k] > 64) return set_error(AOK_ERR_INVALID, std::string(who) + ": bad radial power");
        maps.poly[k] = (int)poly[k];
    }
    for (int64_t i = 0; i < nOrb; ++i) {
        if (iR[i] < 1 || iR[i] > nRad || iY[i] < 1 || iY[i] > nY)
            return set_error(AOK_ERR_INVALID, std::string(who) + ": orbital index map out of range");
        maps.iR[i] = (int)(iR[i] - 1);
        maps.iY[i] = (int)(iY[i] - 1);
    }
    const int64_t ntab = nRad * K * NZ;  // <= 64^3
    const int64_t grid = (nX + kEvalThreads - 1) / kEvalThreads;
    // the partial rows are needed only for the (zeta, D) gradient; a dX-only call
    // uses the index maps and the error word alone
    const size_t need = kNoAllocRowsOffset + (dzeta ? sizeof(double) * 2 * (size_t)ntab * (size_t)grid : 0);
    if (need > kNoAllocScratchBytes)
        return set_error(AOK_ERR_UNSUPPORTED,
                         std::string(who) + ": nX = " + std::to_string(nX) + " needs " + std::to_string(need) +
                             " bytes of scratch; the static scratch holds " +
                             std::to_string(kNoAllocScratchBytes) + " (use aok_evaluate_pullback)");
    cudaStream_t s = (cudaStream_t)stream;
    const size_t fsz = precision == AOK_PREC_F64 ? 8 : 4;
    if (nX == 0) {
        if (dzeta) {
            int st = cuda_status(cudaMemsetAsync(dzeta, 0, fsz * ntab, s), "memset");
            if (st) return st;
            return cuda_status(cudaMemsetAsync(dD, 0, fsz * ntab, s), "memset");
        }
        return AOK_OK;
    }
    if (!dP || !X || !sidx || !zeta || !D) return set_error(AOK_ERR_INVALID, std::string(who) + ": null pointer");
    unsigned char* scratch = nullptr;
    int st = noalloc_scratch(&scratch);
    if (st != AOK_OK) return st;
    // a plan-shaped descriptor on the stack whose tables point into the scratch
    aok_orbitals o;
    o.nRad = nRad;
    o.K = K;
    o.NZ = NZ;
    o.nOrb = nOrb;
    o.L = (int)L;
    o.radial = radial_kind;
    o.prec = precision;
    int* mp = reinterpret_cast<int*>(scratch + kNoAllocMapsOffset);
    o.d_poly = mp;
    o.d_iR = mp + kNoAllocMaxRad;
    o.d_iY = mp + kNoAllocMaxRad + kNoAllocMaxOrb;
    o.d_err = reinterpret_cast<int*>(scratch);
    if (eval_smem_bytes(&o, true) > 227 * 1024)
        return set_error(AOK_ERR_UNSUPPORTED, std::string(who) + ": basis too large for shared memory");
    k_noalloc_setup<<<1, 256, 0, s>>>(maps, scratch);
    st = cuda_status(cudaGetLastError(), "k_noalloc_setup");
    if (st != AOK_OK) return st;
    EvalParams P;
    fill_params(&o, P, X, sidx, zeta, D, nX, lengthscale);
    P.dPin = dP;
    P.dX = dX;
    P.rows = dzeta ? reinterpret_cast<double*>(scratch + kNoAllocRowsOffset) : nullptr;
    st = precision == AOK_PREC_F64 ? launch_eval_T<double>(&o, P, true, true, s)
                                   : launch_eval_T<float>(&o, P, true, true, s);
    if (st != AOK_OK || !P.rows) return st;
    if (precision == AOK_PREC_F64)
        k_eval_reduce<double><<<(int)((2 * ntab + 127) / 128), 128, 0, s>>>((double*)dD, (double*)dzeta, P.rows,
                                                                          (int)grid, (int)ntab);
    else
        k_eval_reduce<float><<<(int)((2 * ntab + 127) / 128), 128, 0, s>>>((float*)dD, (float*)dzeta, P.rows,
                                                                         (int)grid, (int)ntab);
    return cuda_status(cudaGetLastError(), "k_eval_reduce");
}
