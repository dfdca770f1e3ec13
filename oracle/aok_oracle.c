/*
 * aok_oracle.c -- CPU FP64 restatement of the reference's hot-path algorithms.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA library is
 * compared against; the product path never links, loads or calls it.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
 *
 * Each routine restates one reference routine (AtomicOrbitalKernels.jl v0.0.4)
 * and keeps its operation order (no FMA contraction: build with
 * -ffp-contract=off), so that results agree with the reference's Float64 CPU
 * path to rounding.  Layouts are the reference's column-major (Julia) layouts:
 *
 *   positions (3,B)            pos[c + 3*b]
 *   2C output (N,N,B)          out[i + N*(j + N*b)]
 *   3C output (N,N,N,B)        out[i + N*(j + N*(k + N*b))]
 *   per-species tables (ns,K,NZ)  t[s + ns*(k + K*sigma)]
 *   species indices            1-based (Julia convention)
 *
 * Parity pins (tests/test_oracle.py): the reference's known-answer tests
 * (s/s closed form, shell-pair symmetry, analytic single-atom overlap,
 * directional-derivative identities, absent-species zero gradient) plus an
 * mpmath quadrature spot check and central finite differences.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

static int set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    return nthreads;
#else
    (void)nthreads;
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* McMurchie-Davidson 2-center E table, one axis.                            */
/* Follows kernels_2c.jl:57-97 (same recursion in overlap_2c.jl:64-104      */
/* and overlap_2c_grad.jl:132-166).  1-based indices as in the reference:    */
/* E[t, i, j] with t in 1..TM, i in 1..IM, j in 1..JM.                        */
/* ------------------------------------------------------------------------ */
#define E2(t, i, j) E[((t) - 1) + TM * (((i) - 1) + IM * ((j) - 1))]

static void md_E2(double* E, int TM, int IM, int la1, int lb1,
                  double PA, double PB, double AB, double mu, double oo2p) {
    for (int jb = 1; jb <= lb1; ++jb)
        for (int ia = 1; ia <= la1; ++ia) {
            int ab = ia + jb;
            if (ab <= TM) E2(ab, ia, jb) = 0.0;
            if (ab + 1 <= TM) E2(ab + 1, ia, jb) = 0.0;
        }
    E2(1, 1, 1) = exp(((-mu) * AB) * AB);
    for (int i = 2; i <= la1; ++i) {
        E2(1, i, 1) = PA * E2(1, i - 1, 1) + E2(2, i - 1, 1);
        for (int t = 2; t <= i; ++t)
            E2(t, i, 1) = (PA * E2(t, i - 1, 1) + (double)t * E2(t + 1, i - 1, 1)) +
                          oo2p * E2(t - 1, i - 1, 1);
    }
    for (int j = 2; j <= lb1; ++j) {
        E2(1, 1, j) = PB * E2(1, 1, j - 1) + E2(2, 1, j - 1);
        for (int t = 2; t <= j; ++t)
            E2(t, 1, j) = (PB * E2(t, 1, j - 1) + (double)t * E2(t + 1, 1, j - 1)) +
                          oo2p * E2(t - 1, 1, j - 1);
        for (int i = 2; i <= la1; ++i) {
            E2(1, i, j) = PA * E2(1, i - 1, j) + E2(2, i - 1, j);
            for (int t = 2; t <= i + j - 1; ++t)
                E2(t, i, j) = (PA * E2(t, i - 1, j) + (double)t * E2(t + 1, i - 1, j)) +
                              oo2p * E2(t - 1, i - 1, j);
        }
    }
}

/* One primitive pair accumulated into the aliased shell-pair block.
 * Contraction order and the N1 = 2*l_a+1 linear stride follow
 * kernels_2c.jl:99-119 (= overlap_2c.jl:106-126).                           */
static void contract2(double* blk, const double* Ex, const double* Ey, const double* Ez,
                      int TM, int IM, int la, int lb, double prefac) {
    const double* E;
    int N1 = 2 * la + 1;
    int index1 = 1;
    for (int ll1 = la; ll1 >= 0; --ll1)
        for (int n1 = 0; n1 <= la - ll1; ++n1) {
            int m1 = la - ll1 - n1;
            int index2 = 1;
            for (int ll2 = lb; ll2 >= 0; --ll2)
                for (int n2 = 0; n2 <= lb - ll2; ++n2) {
                    int m2 = lb - ll2 - n2;
                    int lin = index1 + N1 * (index2 - 1);
                    double ex, ey, ez;
                    E = Ex; ex = E2(1, ll1 + 1, ll2 + 1);
                    E = Ey; ey = E2(1, m1 + 1, m2 + 1);
                    E = Ez; ez = E2(1, n1 + 1, n2 + 1);
                    blk[lin - 1] += ((ex * ey) * ez) * prefac;
                    index2 += 1;
                }
            index1 += 1;
        }
}

static int lmax_of(const int64_t* ls, int64_t ns) {
    int L = 0;
    for (int64_t s = 0; s < ns; ++s) if ((int)ls[s] > L) L = (int)ls[s];
    return L;
}

/* Shared body of both 2-center kernels: primitives come from per-shell lists
 * (pointer + count) chosen by the caller.  skip_zero reproduces the orbital
 * kernel's `(ca == 0 || cb == 0) && continue` (overlap_2c.jl:202).           */
static void s2_block(double* out, int64_t N, int64_t b,
                     int la, int lb, int64_t row_off, int64_t col_off,
                     const double* ca_v, const double* aa_v, int64_t na, int64_t sa_stride,
                     const double* cb_v, const double* ab_v, int64_t nb, int64_t sb_stride,
                     const double* A, const double* B_, int skip_zero,
                     double* Ebuf, int TM, int IM, double* blk) {
    int nbf_a = (la + 1) * (la + 2) / 2, nbf_b = (lb + 1) * (lb + 2) / 2;
    for (int k = 0; k < nbf_a * nbf_b; ++k) blk[k] = 0.0;
    double* Ex = Ebuf;
    double* Ey = Ebuf + TM * IM * IM;
    double* Ez = Ebuf + 2 * TM * IM * IM;
    for (int64_t ip = 0; ip < na; ++ip)
        for (int64_t jp = 0; jp < nb; ++jp) {
            double ca = ca_v[ip * sa_stride], cb = cb_v[jp * sb_stride];
            if (skip_zero && (ca == 0.0 || cb == 0.0)) continue;
            double aa = aa_v[ip * sa_stride], ab = ab_v[jp * sb_stride];
            double p = aa + ab;
            double Px = (aa * A[0] + ab * B_[0]) / p;
            double Py = (aa * A[1] + ab * B_[1]) / p;
            double Pz = (aa * A[2] + ab * B_[2]) / p;
            double mu = aa * ab / p;
            double oo2p = 0.5 / p;
            double prefac = ca * cb * pow(M_PI / p, 1.5);
            double P3[3] = {Px, Py, Pz};
            for (int ax = 0; ax < 3; ++ax) {
                double ABx = A[ax] - B_[ax];
                double PA = P3[ax] - A[ax];
                double PB = P3[ax] - B_[ax];
                md_E2(Ebuf + ax * TM * IM * IM, TM, IM, la + 1, lb + 1, PA, PB, ABx, mu, oo2p);
            }
            contract2(blk, Ex, Ey, Ez, TM, IM, la, lb, prefac);
        }
    for (int j = 0; j < nbf_b; ++j)
        for (int i = 0; i < nbf_a; ++i)
            out[(row_off + i) + N * ((col_off + j) + N * b)] = blk[i + nbf_a * j];
}

/* batch_S_kernel! + batch_overlap! (kernels_2c.jl:11-163): GaussianBasis path.
 * Positions are in Bohr (the Unitful conversion happens above this layer).  */
int aokor_overlap2c_gb(double* out, int64_t ns, const int64_t* ls, const int64_t* nprim,
                       const int64_t* prim_off, const double* coef, const double* alpha,
                       const double* posA, const double* posB, int64_t B, int nthreads) {
    int L = lmax_of(ls, ns);
    int TM = 2 * L + 2, IM = L + 1;
    int64_t* boff = (int64_t*)malloc(sizeof(int64_t) * (size_t)(ns + 1));
    boff[0] = 0;
    for (int64_t s = 0; s < ns; ++s) boff[s + 1] = boff[s] + (ls[s] + 1) * (ls[s] + 2) / 2;
    int64_t N = boff[ns];
    memset(out, 0, sizeof(double) * (size_t)(N * N * B));
    int nt = set_threads(nthreads);
    (void)nt;
#pragma omp parallel num_threads(nt)
    {
        double* Ebuf = (double*)malloc(sizeof(double) * (size_t)(3 * TM * IM * IM));
        double* blk = (double*)malloc(sizeof(double) * (size_t)(((L + 1) * (L + 2) / 2) * ((L + 1) * (L + 2) / 2)));
#pragma omp for schedule(static)
        for (int64_t b = 0; b < B; ++b)
            for (int64_t sa = 0; sa < ns; ++sa)
                for (int64_t sb = 0; sb < ns; ++sb)
                    s2_block(out, N, b, (int)ls[sa], (int)ls[sb], boff[sa], boff[sb],
                             coef + prim_off[sa], alpha + prim_off[sa], nprim[sa], 1,
                             coef + prim_off[sb], alpha + prim_off[sb], nprim[sb], 1,
                             posA + 3 * b, posB + 3 * b, 0, Ebuf, TM, IM, blk);
        free(Ebuf);
        free(blk);
    }
    free(boff);
    return 0;
}

/* batch_S_orbital_kernel! + batch_overlap! (overlap_2c.jl:15-131,171-197):
 * species-indexed padded primitives, zero-coef skip, 1-based sidx.
 * lengthscale multiplies positions as in overlap_2c.jl:184-185.             */
int aokor_overlap2c_orb(double* out, int64_t ns, int64_t K, int64_t NZ, const int64_t* ls,
                        const double* coef, const double* zeta,
                        const int64_t* sidxA, const int64_t* sidxB,
                        const double* posA, const double* posB, int64_t B,
                        double lengthscale, int nthreads) {
    for (int64_t b = 0; b < B; ++b)
        if (sidxA[b] < 1 || sidxA[b] > NZ || sidxB[b] < 1 || sidxB[b] > NZ) return 4;
    int L = lmax_of(ls, ns);
    int TM = 2 * L + 2, IM = L + 1;
    int64_t* boff = (int64_t*)malloc(sizeof(int64_t) * (size_t)(ns + 1));
    boff[0] = 0;
    for (int64_t s = 0; s < ns; ++s) boff[s + 1] = boff[s] + (ls[s] + 1) * (ls[s] + 2) / 2;
    int64_t N = boff[ns];
    memset(out, 0, sizeof(double) * (size_t)(N * N * B));
    int nt = set_threads(nthreads);
    (void)nt;
#pragma omp parallel num_threads(nt)
    {
        double* Ebuf = (double*)malloc(sizeof(double) * (size_t)(3 * TM * IM * IM));
        double* blk = (double*)malloc(sizeof(double) * (size_t)(((L + 1) * (L + 2) / 2) * ((L + 1) * (L + 2) / 2)));
        double A[3], Bv[3];
#pragma omp for schedule(static)
        for (int64_t b = 0; b < B; ++b) {
            int64_t sa_ = sidxA[b] - 1, sb_ = sidxB[b] - 1;
            for (int c = 0; c < 3; ++c) {
                A[c] = posA[3 * b + c];
                Bv[c] = posB[3 * b + c];
                if (lengthscale != 1.0) { A[c] *= lengthscale; Bv[c] *= lengthscale; }
            }
            for (int64_t s_a = 0; s_a < ns; ++s_a)
                for (int64_t s_b = 0; s_b < ns; ++s_b)
                    s2_block(out, N, b, (int)ls[s_a], (int)ls[s_b], boff[s_a], boff[s_b],
                             coef + s_a + ns * K * sa_, zeta + s_a + ns * K * sa_, K, ns,
                             coef + s_b + ns * K * sb_, zeta + s_b + ns * K * sb_, K, ns,
                             A, Bv, 1, Ebuf, TM, IM, blk);
        }
        free(Ebuf);
        free(blk);
    }
    free(boff);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Position pullback of the orbital-path 2C overlap (no reference            */
/* counterpart; the reference has no position gradient of the overlap).     */
/* Independent of the product's moment formulation: each Cartesian Gaussian  */
/* is differentiated itself,                                                 */
/*   d/dA_x [x_A^i exp(-a x_A^2)] = 2a x_A^{i+1} exp(-a x_A^2) - i x_A^{i-1} exp(-a x_A^2), */
/* (and with b, j for B), and the 1-D overlaps of the raised and lowered     */
/* powers come from the same E-table recursion as the forward (tables to    */
/* l+1 on each side).  The derivative blocks are placed with the forward's   */
/* aliased lin = c1 + (2la+1) c2 layout and read back through the shell's    */
/* nbf strides, so dA[c,b] = sum dS . dOut/dA_c exactly as the forward       */
/* writes Out.  dA, dB (3,B); dS (N,N,B).                                    */
/* ------------------------------------------------------------------------ */
static double e0(const double* E, int TM, int IM, int i, int j) {
    /* E^{ij}_0 with 0-based powers; 0 for a negative power */
    if (i < 0 || j < 0) return 0.0;
    return E2(1, i + 1, j + 1);
}

int aokor_overlap2c_orb_dpos(double* dA, double* dB, const double* dS, int64_t ns, int64_t K, int64_t NZ,
                             const int64_t* ls, const double* coef, const double* zeta,
                             const int64_t* sidxA, const int64_t* sidxB,
                             const double* posA, const double* posB, int64_t B,
                             double lengthscale, int nthreads) {
    for (int64_t b = 0; b < B; ++b)
        if (sidxA[b] < 1 || sidxA[b] > NZ || sidxB[b] < 1 || sidxB[b] > NZ) return 4;
    int L = lmax_of(ls, ns);
    int TM = 2 * L + 4, IM = L + 2;
    int64_t* boff = (int64_t*)malloc(sizeof(int64_t) * (size_t)(ns + 1));
    boff[0] = 0;
    for (int64_t s = 0; s < ns; ++s) boff[s + 1] = boff[s] + (ls[s] + 1) * (ls[s] + 2) / 2;
    int64_t N = boff[ns];
    int nt = set_threads(nthreads);
    (void)nt;
    int nc = (L + 1) * (L + 2) / 2;
#pragma omp parallel num_threads(nt)
    {
        double* Ebuf = (double*)malloc(sizeof(double) * (size_t)(3 * TM * IM * IM));
        double* blkA = (double*)malloc(sizeof(double) * (size_t)(3 * nc * nc));
        double* blkB = (double*)malloc(sizeof(double) * (size_t)(3 * nc * nc));
#pragma omp for schedule(static)
        for (int64_t b = 0; b < B; ++b) {
            int64_t ga = sidxA[b] - 1, gb = sidxB[b] - 1;
            double A[3], Bv[3], ga3[3] = {0, 0, 0}, gb3[3] = {0, 0, 0};
            for (int c = 0; c < 3; ++c) {
                A[c] = posA[3 * b + c];
                Bv[c] = posB[3 * b + c];
                if (lengthscale != 1.0) { A[c] *= lengthscale; Bv[c] *= lengthscale; }
            }
            for (int64_t sa = 0; sa < ns; ++sa)
                for (int64_t sb = 0; sb < ns; ++sb) {
                    int la = (int)ls[sa], lb = (int)ls[sb];
                    int nbf_a = (la + 1) * (la + 2) / 2, nbf_b = (lb + 1) * (lb + 2) / 2;
                    int N1 = 2 * la + 1;
                    for (int k = 0; k < 3 * nc * nc; ++k) { blkA[k] = 0.0; blkB[k] = 0.0; }
                    for (int64_t ip = 0; ip < K; ++ip)
                        for (int64_t jp = 0; jp < K; ++jp) {
                            double ca = coef[sa + ns * (ip + K * ga)], cb = coef[sb + ns * (jp + K * gb)];
                            if (ca == 0.0 || cb == 0.0) continue;
                            double aa = zeta[sa + ns * (ip + K * ga)], ab = zeta[sb + ns * (jp + K * gb)];
                            double p = aa + ab;
                            double mu = aa * ab / p, oo2p = 0.5 / p;
                            double prefac = ca * cb * pow(M_PI / p, 1.5);
                            for (int ax = 0; ax < 3; ++ax) {
                                double Px = (aa * A[ax] + ab * Bv[ax]) / p;
                                md_E2(Ebuf + ax * TM * IM * IM, TM, IM, la + 2, lb + 2, Px - A[ax], Px - Bv[ax],
                                      A[ax] - Bv[ax], mu, oo2p);
                            }
                            /* component pairs in the forward's order (kernels_2c.jl:102-119) */
                            int index1 = 1;
                            for (int ll1 = la; ll1 >= 0; --ll1)
                                for (int n1 = 0; n1 <= la - ll1; ++n1) {
                                    int m1 = la - ll1 - n1;
                                    int pa[3] = {ll1, m1, n1};
                                    int index2 = 1;
                                    for (int ll2 = lb; ll2 >= 0; --ll2)
                                        for (int n2 = 0; n2 <= lb - ll2; ++n2) {
                                            int m2 = lb - ll2 - n2;
                                            int pb[3] = {ll2, m2, n2};
                                            int lin = index1 + N1 * (index2 - 1);
                                            double f[3], fa[3], fb[3];
                                            for (int ax = 0; ax < 3; ++ax) {
                                                const double* E = Ebuf + ax * TM * IM * IM;
                                                int i = pa[ax], j = pb[ax];
                                                f[ax] = e0(E, TM, IM, i, j);
                                                fa[ax] = 2.0 * aa * e0(E, TM, IM, i + 1, j) - i * e0(E, TM, IM, i - 1, j);
                                                fb[ax] = 2.0 * ab * e0(E, TM, IM, i, j + 1) - j * e0(E, TM, IM, i, j - 1);
                                            }
                                            for (int c = 0; c < 3; ++c) {
                                                double oa = 1.0, ob = 1.0;
                                                for (int ax = 0; ax < 3; ++ax) {
                                                    oa *= (ax == c) ? fa[ax] : f[ax];
                                                    ob *= (ax == c) ? fb[ax] : f[ax];
                                                }
                                                blkA[c * nc * nc + lin - 1] += oa * prefac;
                                                blkB[c * nc * nc + lin - 1] += ob * prefac;
                                            }
                                            index2 += 1;
                                        }
                                    index1 += 1;
                                }
                        }
                    for (int j = 0; j < nbf_b; ++j)
                        for (int i = 0; i < nbf_a; ++i) {
                            double g = dS[(boff[sa] + i) + N * ((boff[sb] + j) + N * b)];
                            for (int c = 0; c < 3; ++c) {
                                ga3[c] += g * blkA[c * nc * nc + i + nbf_a * j];
                                gb3[c] += g * blkB[c * nc * nc + i + nbf_a * j];
                            }
                        }
                }
            for (int c = 0; c < 3; ++c) {
                dA[3 * b + c] = lengthscale * ga3[c];
                dB[3 * b + c] = lengthscale * gb3[c];
            }
        }
        free(Ebuf);
        free(blkA);
        free(blkB);
    }
    free(boff);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* 3-center overlap: batch_V_kernel! (kernels_3c.jl:12-162).                 */
/* E3[t, i, j, k], TM = 3Lmax+3.  The table is zeroed in full per primitive  */
/* triple and axis; for l <= 3 this equals the reference's partial zeroing   */
/* (its extra t-entries never reach t = 1), for l >= 4 the reference reads   */
/* uninitialised entries and has no defined value to match.                 */
/* ------------------------------------------------------------------------ */
#define E3I(t, i, j, k) E[((t) - 1) + TM * (((i) - 1) + IM * (((j) - 1) + IM * ((k) - 1)))]

static void md_E3(double* E, int TM, int IM, int la1, int lb1, int lc1,
                  double QA, double QB, double QC, double e0, double oo2q) {
    memset(E, 0, sizeof(double) * (size_t)(TM * IM * IM * IM));
    E3I(1, 1, 1, 1) = e0;
    for (int i = 2; i <= la1; ++i) {
        E3I(1, i, 1, 1) = QA * E3I(1, i - 1, 1, 1) + E3I(2, i - 1, 1, 1);
        for (int t = 2; t <= i; ++t)
            E3I(t, i, 1, 1) = (QA * E3I(t, i - 1, 1, 1) + (double)t * E3I(t + 1, i - 1, 1, 1)) +
                              oo2q * E3I(t - 1, i - 1, 1, 1);
    }
    for (int j = 2; j <= lb1; ++j) {
        E3I(1, 1, j, 1) = QB * E3I(1, 1, j - 1, 1) + E3I(2, 1, j - 1, 1);
        for (int t = 2; t <= j; ++t)
            E3I(t, 1, j, 1) = (QB * E3I(t, 1, j - 1, 1) + (double)t * E3I(t + 1, 1, j - 1, 1)) +
                              oo2q * E3I(t - 1, 1, j - 1, 1);
        for (int i = 2; i <= la1; ++i) {
            E3I(1, i, j, 1) = QA * E3I(1, i - 1, j, 1) + E3I(2, i - 1, j, 1);
            for (int t = 2; t <= i + j - 1; ++t)
                E3I(t, i, j, 1) = (QA * E3I(t, i - 1, j, 1) + (double)t * E3I(t + 1, i - 1, j, 1)) +
                                  oo2q * E3I(t - 1, i - 1, j, 1);
        }
    }
    for (int k = 2; k <= lc1; ++k) {
        E3I(1, 1, 1, k) = QC * E3I(1, 1, 1, k - 1) + E3I(2, 1, 1, k - 1);
        for (int t = 2; t <= k; ++t)
            E3I(t, 1, 1, k) = (QC * E3I(t, 1, 1, k - 1) + (double)t * E3I(t + 1, 1, 1, k - 1)) +
                              oo2q * E3I(t - 1, 1, 1, k - 1);
        for (int j = 2; j <= lb1; ++j) {
            E3I(1, 1, j, k) = QB * E3I(1, 1, j - 1, k) + E3I(2, 1, j - 1, k);
            for (int t = 2; t <= j + k - 1; ++t)
                E3I(t, 1, j, k) = (QB * E3I(t, 1, j - 1, k) + (double)t * E3I(t + 1, 1, j - 1, k)) +
                                  oo2q * E3I(t - 1, 1, j - 1, k);
        }
        for (int j = 1; j <= lb1; ++j)
            for (int i = 2; i <= la1; ++i) {
                E3I(1, i, j, k) = QA * E3I(1, i - 1, j, k) + E3I(2, i - 1, j, k);
                for (int t = 2; t <= i + j + k - 1; ++t) {
                    if (t + 1 > TM) {  /* only reachable for l >= 4 */
                        E3I(t, i, j, k) = QA * E3I(t, i - 1, j, k) + oo2q * E3I(t - 1, i - 1, j, k);
                        continue;
                    }
                    E3I(t, i, j, k) = (QA * E3I(t, i - 1, j, k) + (double)t * E3I(t + 1, i - 1, j, k)) +
                                      oo2q * E3I(t - 1, i - 1, j, k);
                }
            }
    }
}

/* One shell-triple block of one batch element: the primitive loop and the  */
/* aliased contraction of batch_V_kernel! (kernels_3c.jl:12-162).  Each     */
/* centre's primitives come as (coef, alpha) lists with a stride; with      */
/* skip_zero a triple with a zero coefficient is skipped (the orbital path, */
/* padded slots).  Ebuf: 3 * TM*IM^3, blk: NBF^3 doubles.                   */
static void v3_block(double* out, int64_t N, int64_t b, const int64_t* ls, const int64_t* boff,
                     int64_t s_a, int64_t s_b, int64_t s_c,
                     const double* ca_v, const double* aa_v, int64_t na, int64_t sta,
                     const double* cb_v, const double* ab_v, int64_t nb, int64_t stb,
                     const double* cc_v, const double* ac_v, int64_t nc, int64_t stc,
                     const double* A, const double* Bp, const double* C, int skip_zero,
                     double* Ebuf, int TM, int IM, double* blk) {
    size_t esz = (size_t)(TM * IM * IM * IM);
    int la = (int)ls[s_a], lb = (int)ls[s_b], lc = (int)ls[s_c];
    int nbf_a = (la + 1) * (la + 2) / 2, nbf_b = (lb + 1) * (lb + 2) / 2,
        nbf_c = (lc + 1) * (lc + 2) / 2;
    int N1 = 2 * la + 1, N2 = 2 * lb + 1;
    for (int q = 0; q < nbf_a * nbf_b * nbf_c; ++q) blk[q] = 0.0;
    for (int64_t ip = 0; ip < na; ++ip)
        for (int64_t jp = 0; jp < nb; ++jp)
            for (int64_t kp = 0; kp < nc; ++kp) {
                double ca = ca_v[ip * sta], aa = aa_v[ip * sta];
                double cb = cb_v[jp * stb], ab = ab_v[jp * stb];
                double cc = cc_v[kp * stc], ac = ac_v[kp * stc];
                if (skip_zero && (ca == 0.0 || cb == 0.0 || cc == 0.0)) continue;
                double p = aa + ab;
                double P[3], Q[3];
                for (int c = 0; c < 3; ++c) P[c] = (aa * A[c] + ab * Bp[c]) / p;
                double q = p + ac;
                for (int c = 0; c < 3; ++c) Q[c] = (p * P[c] + ac * C[c]) / q;
                double mu = aa * ab / p;
                double nu = p * ac / q;
                double oo2q = 0.5 / q;
                double prefac = ca * cb * cc * pow(M_PI / q, 1.5);
                for (int ax = 0; ax < 3; ++ax) {
                    double AB = A[ax] - Bp[ax];
                    double PC = P[ax] - C[ax];
                    double QA = Q[ax] - A[ax];
                    double QB = Q[ax] - Bp[ax];
                    double QC = Q[ax] - C[ax];
                    double e0 = exp((((-mu) * AB) * AB) - ((nu * PC) * PC));
                    md_E3(Ebuf + ax * esz, TM, IM, la + 1, lb + 1, lc + 1, QA, QB, QC, e0, oo2q);
                }
                const double* E;
                int index1 = 1;
                for (int ll1 = la; ll1 >= 0; --ll1)
                    for (int n1 = 0; n1 <= la - ll1; ++n1) {
                        int m1 = la - ll1 - n1;
                        int index2 = 1;
                        for (int ll2 = lb; ll2 >= 0; --ll2)
                            for (int n2 = 0; n2 <= lb - ll2; ++n2) {
                                int m2 = lb - ll2 - n2;
                                int index3 = 1;
                                for (int ll3 = lc; ll3 >= 0; --ll3)
                                    for (int n3 = 0; n3 <= lc - ll3; ++n3) {
                                        int m3 = lc - ll3 - n3;
                                        int lin = index1 + N1 * (index2 - 1) + N1 * N2 * (index3 - 1);
                                        double ex, ey, ez;
                                        E = Ebuf;           ex = E3I(1, ll1 + 1, ll2 + 1, ll3 + 1);
                                        E = Ebuf + esz;     ey = E3I(1, m1 + 1, m2 + 1, m3 + 1);
                                        E = Ebuf + 2 * esz; ez = E3I(1, n1 + 1, n2 + 1, n3 + 1);
                                        blk[lin - 1] += ((ex * ey) * ez) * prefac;
                                        index3 += 1;
                                    }
                                index2 += 1;
                            }
                        index1 += 1;
                    }
            }
    for (int kk = 0; kk < nbf_c; ++kk)
        for (int jj = 0; jj < nbf_b; ++jj)
            for (int ii = 0; ii < nbf_a; ++ii)
                out[(boff[s_a] + ii) + N * ((boff[s_b] + jj) + N * ((boff[s_c] + kk) + N * b))] =
                    blk[ii + nbf_a * jj + nbf_a * nbf_b * kk];
}

int aokor_overlap3c_gb(double* out, int64_t ns, const int64_t* ls, const int64_t* nprim,
                       const int64_t* prim_off, const double* coef, const double* alpha,
                       const double* posA, const double* posB, const double* posC,
                       int64_t B, int nthreads) {
    int L = lmax_of(ls, ns);
    int TM = 3 * L + 3, IM = L + 1;
    int NBF = (L + 1) * (L + 2) / 2;
    int64_t* boff = (int64_t*)malloc(sizeof(int64_t) * (size_t)(ns + 1));
    boff[0] = 0;
    for (int64_t s = 0; s < ns; ++s) boff[s + 1] = boff[s] + (ls[s] + 1) * (ls[s] + 2) / 2;
    int64_t N = boff[ns];
    memset(out, 0, sizeof(double) * (size_t)(N * N * N * B));
    int nt = set_threads(nthreads);
    (void)nt;
#pragma omp parallel num_threads(nt)
    {
        size_t esz = (size_t)(TM * IM * IM * IM);
        double* Ebuf = (double*)malloc(sizeof(double) * 3 * esz);
        double* blk = (double*)malloc(sizeof(double) * (size_t)(NBF * NBF * NBF));
#pragma omp for schedule(static)
        for (int64_t b = 0; b < B; ++b)
            for (int64_t s_a = 0; s_a < ns; ++s_a)
                for (int64_t s_b = 0; s_b < ns; ++s_b)
                    for (int64_t s_c = 0; s_c < ns; ++s_c)
                        v3_block(out, N, b, ls, boff, s_a, s_b, s_c,
                                 coef + prim_off[s_a], alpha + prim_off[s_a], nprim[s_a], 1,
                                 coef + prim_off[s_b], alpha + prim_off[s_b], nprim[s_b], 1,
                                 coef + prim_off[s_c], alpha + prim_off[s_c], nprim[s_c], 1,
                                 posA + 3 * b, posB + 3 * b, posC + 3 * b, 0, Ebuf, TM, IM, blk);
        free(Ebuf);
        free(blk);
    }
    free(boff);
    return 0;
}

/* 3C overlap on the species-aware (orbital) path -- no reference counterpart */
/* (the reference has the 3C kernel for CompiledBasis only): centre A of     */
/* element b uses species sidxA[b] (1-based), and so on, with the padded     */
/* (ns,K,NZ) tables of the 2C orbital path and its zero-coefficient skip;    */
/* positions multiplied by lengthscale.  Returns 4 on a bad species index.   */
int aokor_overlap3c_orb(double* out, int64_t ns, int64_t K, int64_t NZ, const int64_t* ls,
                        const double* coef, const double* zeta, const int64_t* sidxA,
                        const int64_t* sidxB, const int64_t* sidxC, const double* posA,
                        const double* posB, const double* posC, int64_t B, double lengthscale,
                        int nthreads) {
    for (int64_t b = 0; b < B; ++b)
        if (sidxA[b] < 1 || sidxA[b] > NZ || sidxB[b] < 1 || sidxB[b] > NZ || sidxC[b] < 1 || sidxC[b] > NZ)
            return 4;
    int L = lmax_of(ls, ns);
    int TM = 3 * L + 3, IM = L + 1;
    int NBF = (L + 1) * (L + 2) / 2;
    int64_t* boff = (int64_t*)malloc(sizeof(int64_t) * (size_t)(ns + 1));
    boff[0] = 0;
    for (int64_t s = 0; s < ns; ++s) boff[s + 1] = boff[s] + (ls[s] + 1) * (ls[s] + 2) / 2;
    int64_t N = boff[ns];
    memset(out, 0, sizeof(double) * (size_t)(N * N * N * B));
    int nt = set_threads(nthreads);
    (void)nt;
#pragma omp parallel num_threads(nt)
    {
        size_t esz = (size_t)(TM * IM * IM * IM);
        double* Ebuf = (double*)malloc(sizeof(double) * 3 * esz);
        double* blk = (double*)malloc(sizeof(double) * (size_t)(NBF * NBF * NBF));
#pragma omp for schedule(static)
        for (int64_t b = 0; b < B; ++b) {
            int64_t ga = sidxA[b] - 1, gb = sidxB[b] - 1, gc = sidxC[b] - 1;
            double A[3], Bv[3], C[3];
            for (int c = 0; c < 3; ++c) {
                A[c] = posA[3 * b + c];
                Bv[c] = posB[3 * b + c];
                C[c] = posC[3 * b + c];
                if (lengthscale != 1.0) { A[c] *= lengthscale; Bv[c] *= lengthscale; C[c] *= lengthscale; }
            }
            for (int64_t s_a = 0; s_a < ns; ++s_a)
                for (int64_t s_b = 0; s_b < ns; ++s_b)
                    for (int64_t s_c = 0; s_c < ns; ++s_c)
                        v3_block(out, N, b, ls, boff, s_a, s_b, s_c,
                                 coef + s_a + ns * K * ga, zeta + s_a + ns * K * ga, K, ns,
                                 coef + s_b + ns * K * gb, zeta + s_b + ns * K * gb, K, ns,
                                 coef + s_c + ns * K * gc, zeta + s_c + ns * K * gc, K, ns,
                                 A, Bv, C, 1, Ebuf, TM, IM, blk);
        }
        free(Ebuf);
        free(blk);
    }
    free(boff);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* 2C overlap pullback: batch_S_orbital_pb_kernel! (overlap_2c_grad.jl:71-  */
/* 214).  E to l+2, no zero skip, aliased readback of dS.  Accumulation is  */
/* sequential (b, s_a, s_b, ip, jp); with nthreads > 1 each thread owns a   */
/* partial that is summed in thread order.                                   */
/* ------------------------------------------------------------------------ */
int aokor_overlap2c_orb_pb(double* dcoef, double* dalpha, const double* dS,
                           int64_t ns, int64_t K, int64_t NZ, const int64_t* ls,
                           const double* coef, const double* zeta,
                           const int64_t* sidxA, const int64_t* sidxB,
                           const double* posA, const double* posB, int64_t B,
                           double lengthscale, int nthreads) {
    for (int64_t b = 0; b < B; ++b)
        if (sidxA[b] < 1 || sidxA[b] > NZ || sidxB[b] < 1 || sidxB[b] > NZ) return 4;
    int L = lmax_of(ls, ns);
    int Lr = L + 2;
    int TM = 2 * Lr + 2, IM = Lr + 1;
    int64_t* boff = (int64_t*)malloc(sizeof(int64_t) * (size_t)(ns + 1));
    boff[0] = 0;
    for (int64_t s = 0; s < ns; ++s) boff[s + 1] = boff[s] + (ls[s] + 1) * (ls[s] + 2) / 2;
    int64_t N = boff[ns];
    int64_t nslot = ns * K * NZ;
    int nt = set_threads(nthreads);
    double* part = (double*)calloc((size_t)(2 * nslot * nt), sizeof(double));
#pragma omp parallel num_threads(nt)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double* pc = part + (size_t)(2 * nslot * tid);
        double* pa = pc + nslot;
        double* E = (double*)malloc(sizeof(double) * (size_t)(3 * TM * IM * IM));
#pragma omp for schedule(static)
        for (int64_t b = 0; b < B; ++b) {
            int64_t sga = sidxA[b] - 1, sgb = sidxB[b] - 1;
            double A[3], Bv[3];
            for (int c = 0; c < 3; ++c) {
                A[c] = posA[3 * b + c];
                Bv[c] = posB[3 * b + c];
                if (lengthscale != 1.0) { A[c] *= lengthscale; Bv[c] *= lengthscale; }
            }
            for (int64_t s_a = 0; s_a < ns; ++s_a)
                for (int64_t s_b = 0; s_b < ns; ++s_b) {
                    int la = (int)ls[s_a], lb = (int)ls[s_b];
                    int nbf_a = (la + 1) * (la + 2) / 2;
                    int N1 = 2 * la + 1;
                    int64_t row_off = boff[s_a], col_off = boff[s_b];
                    for (int64_t ip = 0; ip < K; ++ip)
                        for (int64_t jp = 0; jp < K; ++jp) {
                            int64_t ia = s_a + ns * (ip + K * sga), ib = s_b + ns * (jp + K * sgb);
                            double ca = coef[ia], cb = coef[ib];
                            double aa = zeta[ia], ab = zeta[ib];
                            double p = aa + ab;
                            double P[3];
                            for (int c = 0; c < 3; ++c) P[c] = (aa * A[c] + ab * Bv[c]) / p;
                            double mu = aa * ab / p;
                            double oo2p = 0.5 / p;
                            double pref0 = pow(M_PI / p, 1.5);
                            for (int ax = 0; ax < 3; ++ax)
                                md_E2(E + ax * TM * IM * IM, TM, IM, la + 3, lb + 3,
                                      P[ax] - A[ax], P[ax] - Bv[ax], A[ax] - Bv[ax], mu, oo2p);
                            const double* Ex = E;
                            const double* Ey = E + TM * IM * IM;
                            const double* Ez = E + 2 * TM * IM * IM;
                            double Bsum = 0.0, Aa = 0.0, Ab = 0.0;
                            int index1 = 1;
                            for (int ll1 = la; ll1 >= 0; --ll1)
                                for (int n1 = 0; n1 <= la - ll1; ++n1) {
                                    int m1 = la - ll1 - n1;
                                    int index2 = 1;
                                    for (int ll2 = lb; ll2 >= 0; --ll2)
                                        for (int n2 = 0; n2 <= lb - ll2; ++n2) {
                                            int m2 = lb - ll2 - n2;
                                            int lin = index1 + N1 * (index2 - 1);
                                            int i = (lin - 1) % nbf_a + 1;
                                            int j = (lin - 1) / nbf_a + 1;
                                            double g = dS[(row_off + i - 1) + N * ((col_off + j - 1) + N * b)];
                                            const double* E_;
                                            double ex, ey, ez, exa, eya, eza, exb, eyb, ezb;
#define EE(T, a, bb) (E_ = (T), E_[((1) - 1) + TM * (((a) - 1) + IM * ((bb) - 1))])
                                            ex = EE(Ex, ll1 + 1, ll2 + 1);
                                            ey = EE(Ey, m1 + 1, m2 + 1);
                                            ez = EE(Ez, n1 + 1, n2 + 1);
                                            exa = EE(Ex, ll1 + 3, ll2 + 1);
                                            eya = EE(Ey, m1 + 3, m2 + 1);
                                            eza = EE(Ez, n1 + 3, n2 + 1);
                                            exb = EE(Ex, ll1 + 1, ll2 + 3);
                                            eyb = EE(Ey, m1 + 1, m2 + 3);
                                            ezb = EE(Ez, n1 + 1, n2 + 3);
#undef EE
                                            double Eprod = (ex * ey) * ez;
                                            double dGa = -((((exa * ey) * ez) + ((ex * eya) * ez)) + ((ex * ey) * eza));
                                            double dGb = -((((exb * ey) * ez) + ((ex * eyb) * ez)) + ((ex * ey) * ezb));
                                            Bsum += g * Eprod;
                                            Aa += g * dGa;
                                            Ab += g * dGb;
                                            index2 += 1;
                                        }
                                    index1 += 1;
                                }
                            pc[ia] += (cb * pref0) * Bsum;
                            pc[ib] += (ca * pref0) * Bsum;
                            pa[ia] += ((ca * cb) * pref0) * Aa;
                            pa[ib] += ((ca * cb) * pref0) * Ab;
                        }
                }
        }
        free(E);
    }
    for (int64_t q = 0; q < nslot; ++q) { dcoef[q] = 0.0; dalpha[q] = 0.0; }
    for (int t = 0; t < nt; ++t)
        for (int64_t q = 0; q < nslot; ++q) {
            dcoef[q] += part[(size_t)(2 * nslot * t) + q];
            dalpha[q] += part[(size_t)(2 * nslot * t + nslot) + q];
        }
    free(part);
    free(boff);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Spherical -> Cartesian normalisation: _cart_dfac, _cart_normsq,           */
/* _compile_coef (cartesian_gto_basis.jl:69-120) and its closed-form VJP     */
/* _compile_coef_pb (overlap_2c_grad.jl:251-286).                            */
/* ------------------------------------------------------------------------ */
static double cart_dfac(int n) {
    double p = 1.0;
    int k = n;
    while (k > 1) { p *= k; k -= 2; }
    return p;
}

static double cart_normsq(const double* D, const double* z, int64_t K, int64_t stride, int l) {
    double df = pow(M_PI, 1.5) * (l == 0 ? 1.0 : cart_dfac(2 * l - 1));
    double e = (double)l + 1.5;
    double s = 0.0;
    for (int64_t i = 0; i < K; ++i)
        for (int64_t j = 0; j < K; ++j)
            s += (D[i * stride] * D[j * stride]) / pow(z[i * stride] + z[j * stride], e);
    return (df / pow(2.0, l)) * s;
}

void aokor_compile_coef(double* coef, const double* zeta, const double* D, const int64_t* ls,
                        int64_t ns, int64_t K, int64_t NZ) {
    for (int64_t q = 0; q < ns * K * NZ; ++q) coef[q] = 0.0;
    for (int64_t sg = 0; sg < NZ; ++sg)
        for (int64_t k = 0; k < ns; ++k) {
            int64_t base = k + ns * K * sg;
            double nsq = cart_normsq(D + base, zeta + base, K, ns, (int)ls[k]);
            if (nsq > 0) {
                double n = sqrt(nsq);
                for (int64_t m = 0; m < K; ++m) coef[base + ns * m] = D[base + ns * m] / n;
            }
        }
}

void aokor_compile_coef_pb(double* dD, double* dzeta, const double* dcoef, const double* zeta,
                           const double* D, const int64_t* ls, int64_t ns, int64_t K, int64_t NZ) {
    for (int64_t q = 0; q < ns * K * NZ; ++q) { dD[q] = 0.0; dzeta[q] = 0.0; }
    for (int64_t sg = 0; sg < NZ; ++sg)
        for (int64_t k = 0; k < ns; ++k) {
            int l = (int)ls[k];
            int64_t base = k + ns * K * sg;
            const double* Dk = D + base;
            const double* zk = zeta + base;
            const double* gk = dcoef + base;
            double nsq = cart_normsq(Dk, zk, K, ns, l);
            if (!(nsq > 0)) continue;
            double n = sqrt(nsq);
            double c = (pow(M_PI, 1.5) * (l == 0 ? 1.0 : cart_dfac(2 * l - 1))) / pow(2.0, l);
            double e = (double)l + 1.5;
            double dotcD = 0.0;
            for (int64_t i = 0; i < K; ++i) dotcD += gk[i * ns] * Dk[i * ns];
            double s2n3 = dotcD / (2.0 * ((n * n) * n));
            for (int64_t m = 0; m < K; ++m) {
                double gm = 0.0, hm = 0.0;
                for (int64_t j = 0; j < K; ++j) {
                    double den = zk[m * ns] + zk[j * ns];
                    gm += Dk[j * ns] / pow(den, e);
                    hm += Dk[j * ns] / pow(den, e + 1.0);
                }
                gm *= 2.0 * c;
                hm *= ((-2.0 * c) * e) * Dk[m * ns];
                dD[base + ns * m] = gk[m * ns] / n - gm * s2n3;
                dzeta[base + ns * m] = -hm * s2n3;
            }
        }
}

/* ------------------------------------------------------------------------ */
/* Radial bases: _rnl_val_ka! / _rnl_ed_ka! (gtostoradials.jl:117-153).      */
/* R (nX,nRad), dR (nX,nRad) or NULL; slater selects f(r) = r, else r^2.     */
/* ------------------------------------------------------------------------ */
static double ipow(double x, int64_t n) {
    double r = 1.0;
    for (int64_t i = 0; i < n; ++i) r *= x;
    return r;
}

void aokor_radials(double* R, double* dR, const double* r, const int64_t* sidx,
                   const double* zeta, const double* D, const int64_t* poly,
                   int64_t nX, int64_t nRad, int64_t K, int64_t NZ, int slater) {
    (void)NZ;
    for (int64_t k = 0; k < nRad; ++k)
        for (int64_t i = 0; i < nX; ++i) {
            int64_t sg = sidx[i] - 1;
            double ri = r[i];
            double fx = slater ? ri : ri * ri;
            double dfx = slater ? 1.0 : 2.0 * ri;
            double s = 0.0, ds = 0.0;
            for (int64_t m = 0; m < K; ++m) {
                double z = zeta[k + nRad * (m + K * sg)];
                double a = D[k + nRad * (m + K * sg)] * exp((-z) * fx);
                s += a;
                ds += ((-z) * dfx) * a;
            }
            int64_t p = poly[k];
            double rp = ipow(ri, p);
            double drp = (p == 0) ? 0.0 : (double)p * ipow(ri, p - 1);
            R[i + nX * k] = rp * s;
            if (dR) dR[i + nX * k] = drp * s + rp * ds;
        }
}

/* ------------------------------------------------------------------------ */
/* Real solid harmonics Z_lm(r) = r^l Y_lm(r^), L2-normalised on the unit    */
/* sphere, index l^2+l+m (0-based), the layout SpheriCart's SolidHarmonics   */
/* uses (test_gaussianbasis.jl:40).  Restated from the definition:           */
/*   Z_l0 = F_l0 Q_l^0,  Z_l,+m = sqrt2 F_lm Q_l^m C_m,  Z_l,-m = sqrt2 F_lm Q_l^m S_m */
/*   F_lm = sqrt((2l+1)/(4pi) (l-m)!/(l+m)!),  C_m + i S_m = (x + i y)^m,     */
/*   Q_m^m = (2m-1)!!, Q_{m+1}^m = (2m+1) z Q_m^m,                            */
/*   Q_l^m = ((2l-1) z Q_{l-1}^m - (l+m-1) r^2 Q_{l-2}^m) / (l-m)            */
/* (no Condon-Shortley phase: Z_1,-1 : Z_1,0 : Z_1,1 = y : z : x).  This is  */
/* SpheriCart's definition (Bigi et al., J. Chem. Phys. 159, 064802 (2023),  */
/* Sec. II) with its two (-1)^m factors, in F_l^m and in Q_m^m, cancelled.   */
/* Gradients by forward-mode dual numbers (value + 3 partials).              */
/* ------------------------------------------------------------------------ */
typedef struct { double v, x, y, z; } d4;
static d4 d4c(double v) { d4 r = {v, 0, 0, 0}; return r; }
static d4 d4add(d4 a, d4 b) { d4 r = {a.v + b.v, a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static d4 d4sub(d4 a, d4 b) { d4 r = {a.v - b.v, a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static d4 d4mul(d4 a, d4 b) {
    d4 r = {a.v * b.v, a.x * b.v + a.v * b.x, a.y * b.v + a.v * b.y, a.z * b.v + a.v * b.z};
    return r;
}
static d4 d4scale(d4 a, double s) { d4 r = {a.v * s, a.x * s, a.y * s, a.z * s}; return r; }

#define SH_LMAX 8
void aokor_solid_harmonics(double* Z, double* dZ, const double* X, int64_t nX, int L) {
    int nY = (L + 1) * (L + 1);
    for (int64_t j = 0; j < nX; ++j) {
        d4 x = {X[3 * j], 1, 0, 0}, y = {X[3 * j + 1], 0, 1, 0}, z = {X[3 * j + 2], 0, 0, 1};
        d4 r2 = d4add(d4add(d4mul(x, x), d4mul(y, y)), d4mul(z, z));
        d4 C[SH_LMAX + 1], S[SH_LMAX + 1];
        C[0] = d4c(1.0);
        S[0] = d4c(0.0);
        for (int m = 0; m < L; ++m) {
            C[m + 1] = d4sub(d4mul(x, C[m]), d4mul(y, S[m]));
            S[m + 1] = d4add(d4mul(x, S[m]), d4mul(y, C[m]));
        }
        d4 Q[SH_LMAX + 1][SH_LMAX + 1];
        for (int m = 0; m <= L; ++m) {
            Q[m][m] = d4c(cart_dfac(2 * m - 1));
            if (m + 1 <= L) Q[m + 1][m] = d4mul(d4scale(z, (double)(2 * m + 1)), Q[m][m]);
            for (int l = m + 2; l <= L; ++l)
                Q[l][m] = d4scale(d4sub(d4mul(d4scale(z, (double)(2 * l - 1)), Q[l - 1][m]),
                                        d4mul(d4scale(r2, (double)(l + m - 1)), Q[l - 2][m])),
                                  1.0 / (double)(l - m));
        }
        for (int l = 0; l <= L; ++l) {
            for (int m = 0; m <= l; ++m) {
                double fac = 1.0;  /* (l-m)!/(l+m)! */
                for (int q = l - m + 1; q <= l + m; ++q) fac /= (double)q;
                double F = sqrt((2.0 * l + 1.0) / (4.0 * M_PI) * fac);
                if (m == 0) {
                    d4 v = d4scale(Q[l][0], F);
                    int idx = l * l + l;
                    Z[j + nX * idx] = v.v;
                    if (dZ) { dZ[3 * (j + nX * idx)] = v.x; dZ[3 * (j + nX * idx) + 1] = v.y; dZ[3 * (j + nX * idx) + 2] = v.z; }
                } else {
                    d4 vp = d4scale(d4mul(Q[l][m], C[m]), sqrt(2.0) * F);
                    d4 vm = d4scale(d4mul(Q[l][m], S[m]), sqrt(2.0) * F);
                    int ip = l * l + l + m, im = l * l + l - m;
                    Z[j + nX * ip] = vp.v;
                    Z[j + nX * im] = vm.v;
                    if (dZ) {
                        dZ[3 * (j + nX * ip)] = vp.x; dZ[3 * (j + nX * ip) + 1] = vp.y; dZ[3 * (j + nX * ip) + 2] = vp.z;
                        dZ[3 * (j + nX * im)] = vm.x; dZ[3 * (j + nX * im) + 1] = vm.y; dZ[3 * (j + nX * im) + 2] = vm.z;
                    }
                }
            }
        }
        (void)nY;
    }
}

/* ------------------------------------------------------------------------ */
/* Atomic orbitals: evaluate_ed (atomicorbitals.jl:192-210, _aorb_ed_ka!    */
/* :115-125).  X (3,nX) input-unit positions, iR/iY 1-based (nOrb).          */
/* P (nX,nOrb); dP (3,nX,nOrb) or NULL.                                       */
/* ------------------------------------------------------------------------ */
void aokor_evaluate_ed(double* P, double* dP, const double* X, const int64_t* sidx,
                       const double* zeta, const double* D, const int64_t* poly,
                       const int64_t* iR, const int64_t* iY, int64_t nX, int64_t nRad,
                       int64_t K, int64_t NZ, int64_t nOrb, int L, int slater,
                       double lengthscale, int nthreads) {
    int nY = (L + 1) * (L + 1);
    int nt = set_threads(nthreads);
    (void)nt;
    const int64_t CH = 256;
#pragma omp parallel num_threads(nt)
    {
        double* Xs = (double*)malloc(sizeof(double) * 3 * CH);
        double* r = (double*)malloc(sizeof(double) * CH);
        double* R = (double*)malloc(sizeof(double) * CH * nRad);
        double* dR = (double*)malloc(sizeof(double) * CH * nRad);
        double* Y = (double*)malloc(sizeof(double) * CH * nY);
        double* dY = (double*)malloc(sizeof(double) * 3 * CH * nY);
#pragma omp for schedule(static)
        for (int64_t c0 = 0; c0 < nX; c0 += CH) {
            int64_t n = (nX - c0 < CH) ? nX - c0 : CH;
            for (int64_t j = 0; j < n; ++j) {
                for (int c = 0; c < 3; ++c) {
                    double v = X[3 * (c0 + j) + c];
                    Xs[3 * j + c] = (lengthscale == 1.0) ? v : lengthscale * v;
                }
                r[j] = sqrt(Xs[3 * j] * Xs[3 * j] + Xs[3 * j + 1] * Xs[3 * j + 1] + Xs[3 * j + 2] * Xs[3 * j + 2]);
            }
            aokor_radials(R, dR, r, sidx + c0, zeta, D, poly, n, nRad, K, NZ, slater);
            aokor_solid_harmonics(Y, dY, Xs, n, L);
            for (int64_t i = 0; i < nOrb; ++i) {
                int64_t k = iR[i] - 1, y = iY[i] - 1;
                for (int64_t j = 0; j < n; ++j) {
                    double rn = R[j + n * k], yl = Y[j + n * y];
                    P[(c0 + j) + nX * i] = rn * yl;
                    if (dP) {
                        for (int c = 0; c < 3; ++c) {
                            double drj = Xs[3 * j + c] / r[j];
                            double v = (dR[j + n * k] * drj) * yl + rn * dY[3 * (j + n * y) + c];
                            if (lengthscale != 1.0) v *= lengthscale;
                            dP[3 * ((c0 + j) + nX * i) + c] = v;
                        }
                    }
                }
            }
        }
        free(Xs); free(r); free(R); free(dR); free(Y); free(dY);
    }
}

/* Radial-layer parameter pullback: the segmented reduction of              */
/* _gtostoradials_pb_ka! and pullback_ps (gtostoradials.jl:232-267), one     */
/* accumulator per (species, radial, primitive) slot over the points of that */
/* species.  dzeta, dD (nRad,K,NZ); dRv (nX,nRad) is the cotangent of R.     */
void aokor_radials_pb(double* dzeta, double* dD, const double* dRv, const double* r,
                      const int64_t* sidx, const double* zeta, const double* D,
                      const int64_t* poly, int64_t nX, int64_t nRad, int64_t K, int64_t NZ,
                      int slater) {
    for (int64_t q = 0; q < nRad * K * NZ; ++q) { dzeta[q] = 0.0; dD[q] = 0.0; }
    for (int64_t sg = 0; sg < NZ; ++sg)
        for (int64_t k = 0; k < nRad; ++k)
            for (int64_t m = 0; m < K; ++m) {
                int64_t slot = k + nRad * (m + K * sg);
                double zkm = zeta[slot], Dkm = D[slot];
                double pz = 0.0, pD = 0.0;
                for (int64_t i = 0; i < nX; ++i) {
                    if (sidx[i] - 1 != sg) continue;
                    double ri = r[i];
                    double fx = slater ? ri : ri * ri;
                    double a = exp((-zkm) * fx);
                    double gg = dRv[i + nX * k] * ipow(ri, poly[k]);
                    pD += gg * a;
                    pz += ((gg * Dkm) * a) * (-fx);
                }
                dD[slot] = pD;
                dzeta[slot] = pz;
            }
}

/* Parameter pullback of evaluate: pullback_ps (atomicorbitals.jl:254-267),  */
/* _aorb_pbrad_ka! (:249-252) and the radial segmented pullback              */
/* (gtostoradials.jl:232-267).  dzeta, dD (nRad,K,NZ); dP (nX,nOrb).         */
void aokor_evaluate_pb(double* dzeta, double* dD, const double* dPv, const double* X,
                       const int64_t* sidx, const double* zeta, const double* D,
                       const int64_t* poly, const int64_t* iR, const int64_t* iY,
                       int64_t nX, int64_t nRad, int64_t K, int64_t NZ, int64_t nOrb, int L,
                       int slater, double lengthscale) {
    int nY = (L + 1) * (L + 1);
    double* Xs = (double*)malloc(sizeof(double) * 3 * (size_t)nX);
    double* r = (double*)malloc(sizeof(double) * (size_t)nX);
    double* Y = (double*)malloc(sizeof(double) * (size_t)(nX * nY));
    double* dR = (double*)calloc((size_t)(nX * nRad), sizeof(double));
    for (int64_t j = 0; j < nX; ++j) {
        for (int c = 0; c < 3; ++c) {
            double v = X[3 * j + c];
            Xs[3 * j + c] = (lengthscale == 1.0) ? v : lengthscale * v;
        }
        r[j] = sqrt(Xs[3 * j] * Xs[3 * j] + Xs[3 * j + 1] * Xs[3 * j + 1] + Xs[3 * j + 2] * Xs[3 * j + 2]);
    }
    aokor_solid_harmonics(Y, NULL, Xs, nX, L);
    for (int64_t i = 0; i < nOrb; ++i)
        for (int64_t j = 0; j < nX; ++j)
            dR[j + nX * (iR[i] - 1)] += dPv[j + nX * i] * Y[j + nX * (iY[i] - 1)];
    aokor_radials_pb(dzeta, dD, dR, r, sidx, zeta, D, poly, nX, nRad, K, NZ, slater);
    free(Xs); free(r); free(Y); free(dR);
}

/* Position pullback: _aorb_pbx_ka! (atomicorbitals.jl:283-290).  dX (3,nX). */
void aokor_evaluate_pbx(double* dX, const double* dPv, const double* dPhi, int64_t nX, int64_t nOrb) {
    for (int64_t j = 0; j < nX; ++j)
        for (int c = 0; c < 3; ++c) {
            double acc = 0.0;
            for (int64_t i = 0; i < nOrb; ++i) acc += dPv[j + nX * i] * dPhi[3 * (j + nX * i) + c];
            dX[3 * j + c] = acc;
        }
}
