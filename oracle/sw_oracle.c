/*
 * ORACLE — test infrastructure only.  Nothing in the product imports, links or
 * calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, and only as the checker.
 *
 * CPU restatement of the ForceConstants.jl Stillinger-Weber path with the
 * AutoDiffCalculator (reference paths relative to the ForceConstants.jl root):
 *
 *   StillingerWeberSilicon, Φ₂, Φ₃_si     src/interactions/SW.jl:29-83
 *   third_order!(IFC3, sys, ::SW, ::AutoDiffCalculator)
 *                                          src/autodiff/third_order_AD.jl:71-170
 *   set_third_order_terms!/_alt! scatter  src/autodiff/third_order_AD.jl:180-224
 *   second_order!(IFC2, sys, ::SW, ::AutoDiffCalculator)
 *                                          src/autodiff/second_order_AD.jl:40-110
 *   ASR!, apply_tols!, nearest_mirror!     (shared with lj_oracle.c)
 *
 * Block derivatives.  The reference differentiates the SW energy
 * automatically (FastDifferentiation-generated kernels with cosθ₀ written as
 * -0.333333333333, and a run-time Symbolics kernel for the iik block with the
 * potential's exact cosθ₀ = -1/3).  This file computes the same derivatives
 * with exact third-order hyper-dual arithmetic (three nilpotent directions,
 * the ε1ε2ε3 coefficient is the mixed third partial), with cosθ₀ chosen per
 * block family like the reference (cos0[0] for the generated families, cos0[1]
 * for iik).  Built with -DSW_BLOCKS_FROM_REFERENCE (into oracle/_ref/) it uses
 * the reference's own generated kernels instead, translated to C by
 * oracle/translate_sw_ref.py; that build pins this one.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

void oracle_nearest_mirror(double r[3], const double box[3]);
void oracle_asr3(double* psi, int64_t N);
void oracle_asr2(double* ifc2, int64_t N);
void oracle_apply_tols(double* arr, int64_t len, double tol);

/* SW.jl:29-44, LAMMPS Si.sw parameters, derived constants in Float64 as there. */
static const double SW_EPS = 2.1683, SW_SIGMA = 2.0951, SW_A = 1.80, SW_LAMBDA = 21.0, SW_GAMMA = 1.20;
static const double SW_AA = 7.049556277, SW_BB = 0.6022245584, SW_P = 4.0, SW_Q = 0.0;

double oracle_sw_rcut(void) { return SW_A * SW_SIGMA; }

#ifndef SW_BLOCKS_FROM_REFERENCE
/* ---------------------------------------------------------------- hyper-dual */
typedef struct { double f, e1, e2, e3, e12, e13, e23, e123; } hd;

static hd hd_c(double c) { hd r = {c, 0, 0, 0, 0, 0, 0, 0}; return r; }
static hd hd_add(hd a, hd b) {
    hd r = {a.f + b.f, a.e1 + b.e1, a.e2 + b.e2, a.e3 + b.e3, a.e12 + b.e12, a.e13 + b.e13, a.e23 + b.e23,
            a.e123 + b.e123};
    return r;
}
static hd hd_sub(hd a, hd b) {
    hd r = {a.f - b.f, a.e1 - b.e1, a.e2 - b.e2, a.e3 - b.e3, a.e12 - b.e12, a.e13 - b.e13, a.e23 - b.e23,
            a.e123 - b.e123};
    return r;
}
static hd hd_mul(hd a, hd b) {
    hd r;
    r.f = a.f * b.f;
    r.e1 = a.f * b.e1 + a.e1 * b.f;
    r.e2 = a.f * b.e2 + a.e2 * b.f;
    r.e3 = a.f * b.e3 + a.e3 * b.f;
    r.e12 = a.f * b.e12 + a.e1 * b.e2 + a.e2 * b.e1 + a.e12 * b.f;
    r.e13 = a.f * b.e13 + a.e1 * b.e3 + a.e3 * b.e1 + a.e13 * b.f;
    r.e23 = a.f * b.e23 + a.e2 * b.e3 + a.e3 * b.e2 + a.e23 * b.f;
    r.e123 = a.f * b.e123 + a.e1 * b.e23 + a.e2 * b.e13 + a.e3 * b.e12 + a.e12 * b.e3 + a.e13 * b.e2 +
             a.e23 * b.e1 + a.e123 * b.f;
    return r;
}
/* g(x) with g', g'', g''' at x.f */
static hd hd_fun(hd x, double g, double g1, double g2, double g3) {
    hd r;
    r.f = g;
    r.e1 = g1 * x.e1;
    r.e2 = g1 * x.e2;
    r.e3 = g1 * x.e3;
    r.e12 = g1 * x.e12 + g2 * x.e1 * x.e2;
    r.e13 = g1 * x.e13 + g2 * x.e1 * x.e3;
    r.e23 = g1 * x.e23 + g2 * x.e2 * x.e3;
    r.e123 = g1 * x.e123 + g2 * (x.e1 * x.e23 + x.e2 * x.e13 + x.e3 * x.e12) + g3 * x.e1 * x.e2 * x.e3;
    return r;
}
static hd hd_exp(hd x) { double e = exp(x.f); return hd_fun(x, e, e, e, e); }
static hd hd_sqrt(hd x) {
    double s = sqrt(x.f);
    return hd_fun(x, s, 0.5 / s, -0.25 / (x.f * s), 0.375 / (x.f * x.f * s));
}
static hd hd_inv(hd x) {
    double i = 1.0 / x.f;
    return hd_fun(x, i, -i * i, 2.0 * i * i * i, -6.0 * i * i * i * i);
}
static hd hd_div(hd a, hd b) { return hd_mul(a, hd_inv(b)); }

/* SW.jl:76-78 with r = |x| (q = 0 ⇒ (σ/r)^q = 1). */
static hd sw_phi2(const hd x[3]) {
    hd r = hd_sqrt(hd_add(hd_add(hd_mul(x[0], x[0]), hd_mul(x[1], x[1])), hd_mul(x[2], x[2])));
    hd sr = hd_div(hd_c(SW_SIGMA), r);
    hd sr2 = hd_mul(sr, sr);
    hd srp = hd_mul(sr2, sr2); /* (σ/r)^4 */
    (void)SW_P;
    (void)SW_Q;
    hd t = hd_sub(hd_mul(hd_c(SW_BB), srp), hd_c(1.0));
    hd ex = hd_exp(hd_div(hd_c(SW_SIGMA), hd_sub(r, hd_c(SW_A * SW_SIGMA))));
    return hd_mul(hd_mul(hd_c(SW_AA * SW_EPS), t), ex);
}

/* SW.jl:68-73,81-83 from 9 absolute coordinates [r_i; r_j; r_k]. */
static hd sw_phi3(const hd x[9], double cos0) {
    hd u[3], v[3];
    for (int d = 0; d < 3; ++d) {
        u[d] = hd_sub(x[d], x[3 + d]);
        v[d] = hd_sub(x[d], x[6 + d]);
    }
    hd ru = hd_sqrt(hd_add(hd_add(hd_mul(u[0], u[0]), hd_mul(u[1], u[1])), hd_mul(u[2], u[2])));
    hd rv = hd_sqrt(hd_add(hd_add(hd_mul(v[0], v[0]), hd_mul(v[1], v[1])), hd_mul(v[2], v[2])));
    hd dot = hd_add(hd_add(hd_mul(u[0], v[0]), hd_mul(u[1], v[1])), hd_mul(u[2], v[2]));
    hd c = hd_div(dot, hd_mul(ru, rv));
    hd d = hd_sub(c, hd_c(cos0));
    const double rc = SW_A * SW_SIGMA, gs = SW_SIGMA * SW_GAMMA, le = SW_EPS * SW_LAMBDA;
    hd e1 = hd_exp(hd_div(hd_c(gs), hd_sub(ru, hd_c(rc))));
    hd e2 = hd_exp(hd_div(hd_c(gs), hd_sub(rv, hd_c(rc))));
    return hd_mul(hd_mul(hd_mul(hd_c(le), hd_mul(d, d)), e1), e2);
}

/* ∂³h/∂(X_a)∂(Y_b)∂(Z_c) for atoms X,Y,Z ∈ {0:i, 1:j, 2:k}; block[a+3b+9c]. */
static void block3(const double r9[9], int X, int Y, int Z, double cos0, double* out) {
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            for (int c = 0; c < 3; ++c) {
                hd x[9];
                for (int q = 0; q < 9; ++q) x[q] = hd_c(r9[q]);
                x[3 * X + a].e1 = 1.0;
                x[3 * Y + b].e2 = 1.0;
                x[3 * Z + c].e3 = 1.0;
                out[a + 3 * b + 9 * c] = sw_phi3(x, cos0).e123;
            }
}

static void block2(const double r9[9], int X, int Y, double cos0, double* out) {
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            hd x[9];
            for (int q = 0; q < 9; ++q) x[q] = hd_c(r9[q]);
            x[3 * X + a].e1 = 1.0;
            x[3 * Y + b].e2 = 1.0;
            out[a + 3 * b] = sw_phi3(x, cos0).e12;
        }
}

void oracle_sw_pair_block3(const double r3[3], double* out) {
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            for (int c = 0; c < 3; ++c) {
                hd x[3] = {hd_c(r3[0]), hd_c(r3[1]), hd_c(r3[2])};
                x[a].e1 = 1.0;
                x[b].e2 = 1.0;
                x[c].e3 = 1.0;
                out[a + 3 * b + 9 * c] = sw_phi2(x).e123;
            }
}

void oracle_sw_pair_block2(const double r3[3], double* out) {
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            hd x[3] = {hd_c(r3[0]), hd_c(r3[1]), hd_c(r3[2])};
            x[a].e1 = 1.0;
            x[b].e2 = 1.0;
            out[a + 3 * b] = sw_phi2(x).e12;
        }
}

/* out: 7 blocks of 27 in the order iij, ijj, iik, ikk, jjk, jkk, ijk. */
void oracle_sw_triplet_blocks(const double r9[9], const double cos0[2], double* out) {
    block3(r9, 0, 0, 1, cos0[0], out + 0 * 27);  /* iij */
    block3(r9, 0, 1, 1, cos0[0], out + 1 * 27);  /* ijj */
    block3(r9, 0, 0, 2, cos0[1], out + 2 * 27);  /* iik (run-time Symbolics, exact cosθ₀) */
    block3(r9, 0, 2, 2, cos0[0], out + 3 * 27);  /* ikk */
    block3(r9, 1, 1, 2, cos0[0], out + 4 * 27);  /* jjk */
    block3(r9, 1, 2, 2, cos0[0], out + 5 * 27);  /* jkk */
    block3(r9, 0, 1, 2, cos0[0], out + 6 * 27);  /* ijk */
}

/* out: 3 blocks of 9: ij, ik, jk (second_order_AD.jl:80-95). */
void oracle_sw_triplet_blocks2(const double r9[9], const double cos0[2], double* out) {
    block2(r9, 0, 1, cos0[0], out + 0);
    block2(r9, 0, 2, cos0[0], out + 9);
    block2(r9, 1, 2, cos0[0], out + 18);
}
#else
/* ------------------------------------------- the reference's own kernels */
void ref_H3_exec_ij(const double* x, double* out);
void ref_H3_exec_iij(const double* x, double* out);
void ref_H3_exec_ijj(const double* x, double* out);
void ref_H3_exec_iik(const double* x, double* out);
void ref_H3_exec_ikk(const double* x, double* out);
void ref_H3_exec_jjk(const double* x, double* out);
void ref_H3_exec_jkk(const double* x, double* out);
void ref_H3_exec_ijk(const double* x, double* out);
void ref_H2_exec_pair(const double* x, double* out);
void ref_H2_exec_ij(const double* x, double* out);
void ref_H2_exec_ik(const double* x, double* out);
void ref_H2_exec_jk(const double* x, double* out);

void oracle_sw_pair_block3(const double r3[3], double* out) { ref_H3_exec_ij(r3, out); }
void oracle_sw_pair_block2(const double r3[3], double* out) { ref_H2_exec_pair(r3, out); }
void oracle_sw_triplet_blocks(const double r9[9], const double cos0[2], double* out) {
    (void)cos0;
    ref_H3_exec_iij(r9, out + 0 * 27);
    ref_H3_exec_ijj(r9, out + 1 * 27);
    ref_H3_exec_iik(r9, out + 2 * 27);
    ref_H3_exec_ikk(r9, out + 3 * 27);
    ref_H3_exec_jjk(r9, out + 4 * 27);
    ref_H3_exec_jkk(r9, out + 5 * 27);
    ref_H3_exec_ijk(r9, out + 6 * 27);
}
void oracle_sw_triplet_blocks2(const double r9[9], const double cos0[2], double* out) {
    (void)cos0;
    ref_H2_exec_ij(r9, out + 0);
    ref_H2_exec_ik(r9, out + 9);
    ref_H2_exec_jk(r9, out + 18);
}
#endif

/* ------------------------------------------------ scatter helpers (:180-224) */
#define P3(x, y, z) psi[(x) + n * ((y) + n * (int64_t)(z))]

/* permutedims(B, p)[i1,i2,i3] = B[a1,a2,a3] with a_{p[m]} = i_m (Julia). */
static double perm_get(const double* B, const int p[3], int i1, int i2, int i3) {
    int a[3];
    a[p[0] - 1] = i1;
    a[p[1] - 1] = i2;
    a[p[2] - 1] = i3;
    return B[a[0] + 3 * a[1] + 9 * a[2]];
}

static void add_block(double* psi, int64_t n, int64_t A, int64_t B, int64_t C, const double* blk, int p1, int p2,
                      int p3, double sign) {
    const int p[3] = {p1, p2, p3};
    for (int c = 0; c < 3; ++c)
        for (int b = 0; b < 3; ++b)
            for (int a = 0; a < 3; ++a) P3(3 * A + a, 3 * B + b, 3 * C + c) += sign * perm_get(blk, p, a, b, c);
}

/* set_third_order_terms!(arr, rng1, rng2, block) — 3-argument form */
static void set3_plain(double* psi, int64_t n, int64_t r1, int64_t r2, const double* blk, double sign) {
    add_block(psi, n, r1, r1, r2, blk, 1, 2, 3, sign);
    add_block(psi, n, r1, r2, r1, blk, 1, 2, 3, sign);
    add_block(psi, n, r2, r1, r1, blk, 1, 2, 3, sign);
}
/* aab form */
static void set3_aab(double* psi, int64_t n, int64_t r1, int64_t r2, const double* blk) {
    add_block(psi, n, r1, r1, r2, blk, 1, 2, 3, 1.0);
    add_block(psi, n, r1, r2, r1, blk, 1, 3, 2, 1.0);
    add_block(psi, n, r2, r1, r1, blk, 3, 2, 1, 1.0);
}
/* abb form (set_third_order_terms_alt!) */
static void set3_abb(double* psi, int64_t n, int64_t r1, int64_t r2, const double* blk) {
    add_block(psi, n, r2, r1, r1, blk, 1, 2, 3, 1.0);
    add_block(psi, n, r1, r2, r1, blk, 2, 1, 3, 1.0);
    add_block(psi, n, r1, r1, r2, blk, 3, 2, 1, 1.0);
}
/* abc form */
static void set3_abc(double* psi, int64_t n, int64_t r1, int64_t r2, int64_t r3, const double* blk) {
    add_block(psi, n, r1, r2, r3, blk, 1, 2, 3, 1.0);
    add_block(psi, n, r1, r3, r2, blk, 1, 3, 2, 1.0);
    add_block(psi, n, r2, r1, r3, blk, 2, 1, 3, 1.0);
    add_block(psi, n, r2, r3, r1, blk, 2, 3, 1, 1.0);
    add_block(psi, n, r3, r1, r2, blk, 3, 1, 2, 1.0);
    add_block(psi, n, r3, r2, r1, blk, 3, 2, 1, 1.0);
}

static void mirror_vec(const double* pos, const double box[3], int64_t i, int64_t j, double r[3]) {
    for (int d = 0; d < 3; ++d) r[d] = pos[3 * i + d] - pos[3 * j + d];
    oracle_nearest_mirror(r, box);
}

/* third_order_AD.jl:71-170 (serial, as the reference), then ASR; then
 * apply_tols! (ifc.jl:29).  Returns -1 when the force-constant cutoff exceeds
 * the SW cutoff (third_order_AD.jl:74). */
int oracle_third_order_sw(const double* pos, int64_t N, const double box[3], const double cos0[2], double r_cut,
                          double tol, double* psi) {
    if (!(r_cut <= oracle_sw_rcut())) return -1;
    const int64_t n = 3 * N;
    memset(psi, 0, sizeof(double) * (size_t)(n * n * n));
    const double rc2 = r_cut * r_cut;
    double blk[7 * 27], pb[27], r_arr[9];
    for (int64_t i = 0; i < N; ++i) {
        for (int64_t j = 0; j < N; ++j) {
            if (i == j) continue;
            double rij[3];
            mirror_vec(pos, box, i, j, rij);
            double dij = rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2];
            if (!(dij < rc2)) continue;
            if (j > i) {
                oracle_sw_pair_block3(rij, pb);
                set3_plain(psi, n, i, j, pb, -1.0);
                set3_plain(psi, n, j, i, pb, 1.0);
            }
            for (int64_t k = j + 1; k < N; ++k) {
                if (k == i) continue;
                double rik[3];
                mirror_vec(pos, box, i, k, rik);
                double dik = rik[0] * rik[0] + rik[1] * rik[1] + rik[2] * rik[2];
                if (!(dik < rc2)) continue;
                for (int d = 0; d < 3; ++d) {
                    r_arr[d] = pos[3 * i + d];
                    r_arr[3 + d] = pos[3 * i + d] - rij[d];
                    r_arr[6 + d] = pos[3 * i + d] - rik[d];
                }
                oracle_sw_triplet_blocks(r_arr, cos0, blk);
                set3_aab(psi, n, i, j, blk + 0 * 27);   /* iij */
                set3_abb(psi, n, j, i, blk + 1 * 27);   /* ijj */
                set3_aab(psi, n, i, k, blk + 2 * 27);   /* iik */
                set3_abb(psi, n, k, i, blk + 3 * 27);   /* ikk */
                set3_aab(psi, n, j, k, blk + 4 * 27);   /* jjk */
                set3_abb(psi, n, k, j, blk + 5 * 27);   /* jkk */
                set3_abc(psi, n, i, j, k, blk + 6 * 27); /* ijk */
            }
        }
    }
    oracle_asr3(psi, N);
    oracle_apply_tols(psi, n * n * n, tol);
    return 0;
}

/* second_order_AD.jl:40-110, then ASR!(IFC2) and apply_tols! (ifc.jl:3-18). */
int oracle_second_order_sw(const double* pos, int64_t N, const double box[3], const double cos0[2], double r_cut,
                           double tol, double* ifc2) {
    if (!(r_cut <= oracle_sw_rcut())) return -1;
    const int64_t n = 3 * N;
    memset(ifc2, 0, sizeof(double) * (size_t)(n * n));
    const double rc2 = r_cut * r_cut;
    double b2[27], pb[9], r_arr[9];
#define I2(x, y) ifc2[(x) + n * (int64_t)(y)]
    for (int64_t i = 0; i < N; ++i) {
        for (int64_t j = 0; j < N; ++j) {
            if (i == j) continue;
            double rij[3];
            mirror_vec(pos, box, i, j, rij);
            double dij = rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2];
            if (!(dij < rc2)) continue;
            if (j > i) {
                oracle_sw_pair_block2(rij, pb);
                for (int b = 0; b < 3; ++b)
                    for (int a = 0; a < 3; ++a) {
                        I2(3 * i + a, 3 * j + b) += -pb[a + 3 * b];
                        I2(3 * j + a, 3 * i + b) += -pb[a + 3 * b];
                    }
            }
            for (int64_t k = j + 1; k < N; ++k) {
                if (k == i) continue;
                double rik[3];
                mirror_vec(pos, box, i, k, rik);
                double dik = rik[0] * rik[0] + rik[1] * rik[1] + rik[2] * rik[2];
                if (!(dik < rc2)) continue;
                for (int d = 0; d < 3; ++d) {
                    r_arr[d] = pos[3 * i + d];
                    r_arr[3 + d] = pos[3 * i + d] - rij[d];
                    r_arr[6 + d] = pos[3 * i + d] - rik[d];
                }
                oracle_sw_triplet_blocks2(r_arr, cos0, b2);
                const int64_t at[3][2] = {{i, j}, {i, k}, {j, k}};
                for (int q = 0; q < 3; ++q)
                    for (int b = 0; b < 3; ++b)
                        for (int a = 0; a < 3; ++a) {
                            I2(3 * at[q][0] + a, 3 * at[q][1] + b) += b2[9 * q + a + 3 * b];
                            I2(3 * at[q][1] + a, 3 * at[q][0] + b) += b2[9 * q + b + 3 * a];
                        }
            }
        }
    }
#undef I2
    oracle_asr2(ifc2, N);
    oracle_apply_tols(ifc2, n * n, tol);
    return 0;
}
