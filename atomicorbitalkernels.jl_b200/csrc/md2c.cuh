// md2c.cuh -- 2-center overlap by primitive-pair moments (early contraction).
//
// With p = a + b, ra = a/p, rb = b/p, q = 1/(2p) and X = A_x - B_x, the
// McMurchie-Davidson t = 0 coefficient of the 1-D overlap (the quantity the
// reference builds recursively, Reference/ecoeffs.jl and
// src/integrals/kernels_2c.jl:57-97) has the closed form obtained by
// expanding x_A = x_P + PA, x_B = x_P + PB about the Gaussian product centre,
// with PA = -rb X, PB = ra X and int x_P^n exp(-p x_P^2) = (n-1)!! q^{n/2}
// sqrt(pi/p) for even n:
//
//   E_0^{ij} = sum_{k<=i, l<=j, k+l even} C(i,k) C(j,l) (-1)^{i-k}
//              X^{(i-k)+(j-l)} rb^{i-k} ra^{j-l} (k+l-1)!! q^{(k+l)/2}.
//
// For a Cartesian component pair the product over the three axes is a sum of
// monomials rb^al ra^be q^ga with al <= la, be <= lb and al + be + 2 ga = la + lb,
// whose coefficients depend on the geometry only.  So a shell-pair block is
//
//   S_c = sum_{al,be} coef_{c,al,be}(AB) * M_{al,be},
//   M_{al,be} = sum over primitive pairs of w exp(-mu R^2) rb^al ra^be q^ga,
//
// i.e. the primitive-pair loop accumulates (la+1)(lb+1)/2 moments (8 for f-f)
// and the geometry is applied once per shell pair.  The coefficient tables are
// generated at compile time (MdTab); each term is an integer constant times
// X^px Y^py Z^pz.  The pullback uses the transpose: cotangent moments
// G_{al,be} = sum_c g_c coef_{c,al,be}, then per primitive pair
// dS/dcoef ~ sum G mono and the exponent derivatives from the chain rule on
// (ra, rb, q):  d ra/da = 2q rb, d rb/da = -2q rb, d q/da = -2q^2 (and
// symmetrically in b), plus d log(w exp(-mu R^2))/da = -3q - R^2 rb^2.
#pragma once

#include "aok_common.cuh"

namespace aok {

constexpr int md_binom(int n, int k) {
    int r = 1;
    for (int i = 0; i < k; ++i) r = r * (n - i) / (i + 1);
    return r;
}
constexpr int md_dfact_m1(int n) {  // (n-1)!! for even n >= 0
    int r = 1;
    for (int v = n - 1; v > 0; v -= 2) r *= v;
    return r;
}

struct MdTerm {
    short lin;          // block element (reference's aliased index c1 + (2la+1) c2)
    signed char m;      // moment slot al*(lb+1) + be
    signed char px, py, pz;
    short cst;          // 0: placeholder of an element no component maps to
};

// Terms of every block element of class (LA, LB), ordered by element.
template <int LA, int LB>
struct MdTab {
    static constexpr int NA = ncart(LA), NB = ncart(LB), N1 = 2 * LA + 1, NE = NA * NB;
    static constexpr int NM = (LA + 1) * (LB + 1), W = LA + LB;
    template <bool FILL>
    static constexpr int gen(MdTerm* out) {
        int n = 0;
        for (int lin = 0; lin < NE; ++lin) {
            bool any = false;
            for (int c2 = 0; c2 < NB; ++c2) {
                const int c1 = lin - N1 * c2;
                if (c1 < 0 || c1 >= NA) continue;
                any = true;
                const int x1 = cart_x(LA, c1), y1 = cart_y(LA, c1), z1 = cart_z(LA, c1);
                const int x2 = cart_x(LB, c2), y2 = cart_y(LB, c2), z2 = cart_z(LB, c2);
                for (int kx = 0; kx <= x1; ++kx)
                    for (int lx = 0; lx <= x2; ++lx) {
                        if ((kx + lx) & 1) continue;
                        for (int ky = 0; ky <= y1; ++ky)
                            for (int ly = 0; ly <= y2; ++ly) {
                                if ((ky + ly) & 1) continue;
                                for (int kz = 0; kz <= z1; ++kz)
                                    for (int lz = 0; lz <= z2; ++lz) {
                                        if ((kz + lz) & 1) continue;
                                        const int al = (x1 - kx) + (y1 - ky) + (z1 - kz);
                                        const int be = (x2 - lx) + (y2 - ly) + (z2 - lz);
                                        const int c = ((al & 1) ? -1 : 1) * md_binom(x1, kx) * md_binom(x2, lx) *
                                                      md_dfact_m1(kx + lx) * md_binom(y1, ky) * md_binom(y2, ly) *
                                                      md_dfact_m1(ky + ly) * md_binom(z1, kz) * md_binom(z2, lz) *
                                                      md_dfact_m1(kz + lz);
                                        if (FILL)
                                            out[n] = MdTerm{(short)lin, (signed char)(al * (LB + 1) + be),
                                                            (signed char)(x1 - kx + x2 - lx),
                                                            (signed char)(y1 - ky + y2 - ly),
                                                            (signed char)(z1 - kz + z2 - lz), (short)c};
                                        ++n;
                                    }
                            }
                    }
            }
            if (!any) {
                if (FILL) out[n] = MdTerm{(short)lin, 0, 0, 0, 0, 0};
                ++n;
            }
        }
        return n;
    }
    static constexpr int T = gen<false>(nullptr);
    struct Arr {
        MdTerm t[T];
    };
    static constexpr Arr make() {
        Arr a{};
        gen<true>(a.t);
        return a;
    }
    // moment slot (al, be) is used iff (LA - al) + (LB - be) is even
    static constexpr bool used(int al, int be) { return (((LA - al) + (LB - be)) & 1) == 0; }
};

// Number of terms of class (la, lb) (scheduling cost model).
__host__ __device__ constexpr int md_terms(int la, int lb) {
    // symmetric in (la, lb); written as a branch chain so device code needs no table
    return la > lb ? md_terms(lb, la)
           : la == 0 ? (lb == 0 ? 1 : lb == 1 ? 3 : lb == 2 ? 9 : 19)
           : la == 1 ? (lb == 1 ? 12 : lb == 2 ? 36 : 84)
           : la == 2 ? (lb == 2 ? 111 : 261)
                     : 632;
}
static_assert(md_terms(3, 1) == 84 && md_terms(2, 2) == 111 && md_terms(0, 3) == 19, "term counts");
// table size = terms + one placeholder per block element no component maps to
static_assert(MdTab<3, 3>::T == 632 + 27, "f-f term count");
static_assert(MdTab<2, 2>::T == 111 + 5, "d-d term count");
static_assert(MdTab<1, 3>::T == 84, "p-f term count");

// X^k for k = 0..W per axis.
template <int W, typename FT>
__device__ __forceinline__ void md_powers(FT (&xp)[3][W + 1], const FT (&AB)[3]) {
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        xp[t][0] = FT(1);
#pragma unroll
        for (int k = 1; k <= W; ++k) xp[t][k] = xp[t][k - 1] * AB[t];
    }
}

// Forward transform: block elements from the moments, written to
// dst[(lin / NA) * N + lin % NA] (each element once).
template <int LA, int LB, typename FT>
__device__ __forceinline__ void md_transform(const FT (&M)[(LA + 1) * (LB + 1)], const FT (&AB)[3], FT* dst, int N) {
    using TB = MdTab<LA, LB>;
    constexpr auto tb = TB::make();
    FT xp[3][TB::W + 1];
    md_powers<TB::W, FT>(xp, AB);
    FT v = FT(0);
#pragma unroll
    for (int i = 0; i < TB::T; ++i) {
        const MdTerm e = tb.t[i];
        if (e.cst != 0) v = fma(FT(e.cst) * ((xp[0][e.px] * xp[1][e.py]) * xp[2][e.pz]), M[e.m], v);
        if (i == TB::T - 1 || tb.t[i + 1].lin != e.lin) {
            dst[(e.lin / TB::NA) * N + e.lin % TB::NA] = v;
            v = FT(0);
        }
    }
}

// Transposed transform: cotangent moments G from the block's cotangent g
// (read at the same aliased positions as the forward writes).
template <int LA, int LB, typename FT>
__device__ __forceinline__ void md_cotangent(FT (&G)[(LA + 1) * (LB + 1)], const FT (&AB)[3], const FT* g, int N) {
    using TB = MdTab<LA, LB>;
    constexpr auto tb = TB::make();
    FT xp[3][TB::W + 1];
    md_powers<TB::W, FT>(xp, AB);
#pragma unroll
    for (int m = 0; m < TB::NM; ++m) G[m] = FT(0);
    FT gv = FT(0);
#pragma unroll
    for (int i = 0; i < TB::T; ++i) {
        const MdTerm e = tb.t[i];
        if (i == 0 || tb.t[i - 1].lin != e.lin) gv = g[(e.lin / TB::NA) * N + e.lin % TB::NA];
        if (e.cst != 0) G[e.m] = fma(gv * ((xp[0][e.px] * xp[1][e.py]) * xp[2][e.pz]), FT(e.cst), G[e.m]);
    }
}

// The same with the cotangent given as the difference g = a - b of two arrays
// (read at the same positions): the cotangent of a squared-residual loss without
// materialising it (its scale is applied to the final gradient).
template <int LA, int LB, typename FT>
__device__ __forceinline__ void md_cotangent_diff(FT (&G)[(LA + 1) * (LB + 1)], const FT (&AB)[3], const FT* a,
                                                  const FT* b, int N) {
    using TB = MdTab<LA, LB>;
    constexpr auto tb = TB::make();
    FT xp[3][TB::W + 1];
    md_powers<TB::W, FT>(xp, AB);
#pragma unroll
    for (int m = 0; m < TB::NM; ++m) G[m] = FT(0);
    FT gv = FT(0);
#pragma unroll
    for (int i = 0; i < TB::T; ++i) {
        const MdTerm e = tb.t[i];
        if (i == 0 || tb.t[i - 1].lin != e.lin) {
            const int o = (e.lin / TB::NA) * N + e.lin % TB::NA;
            gv = a[o] - b[o];
        }
        if (e.cst != 0) G[e.m] = fma(gv * ((xp[0][e.px] * xp[1][e.py]) * xp[2][e.pz]), FT(e.cst), G[e.m]);
    }
}

}  // namespace aok
