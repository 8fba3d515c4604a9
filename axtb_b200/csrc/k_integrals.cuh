// Shell-pair integrals over contracted Gaussians: overlap, dipole and traceless quadrupole
// blocks (Obara-Saika moment recursion about the ket centre, Cartesian-to-spherical transform)
// with the core Hamiltonian scaling, and their derivatives with respect to the ket centre
// contracted on the fly with the density, energy-weighted density and SCF potentials for the
// nuclear gradient. Follows crates/axtb/src/integrals.rs:28-367 (S, D, Q), 400-521 (ket
// derivatives), 991-1006 (shift to the bra) and crates/axtb/src/hamiltonian.rs:77-94 (H0),
// 101-223 (gradient). One thread per atom pair; blocks are written straight into the AO
// matrices (each element has exactly one writer), gradient pieces into a per-pair buffer. In the
// gradient each shell pair runs in a function templated on its two angular momenta (a switch per
// pair), so the Cartesian accumulators have compile-time sizes and stay in registers for s and p
// shells (at most 168 registers a thread: three CTAs of 128 per SM); d-shell pairs, in their own
// non-inlined functions, spill what does not fit. The S, D, Q kernel keeps the generic loops: the
// same templating there gave the integrals other last bits (the compiler fuses the recursion's
// products differently once the angular momenta are constants), and those bits steer a few
// chaotic SCFs that axtb's records pin.
#pragma once
#include "common.cuh"
#include "k_geometry.cuh"

namespace axg {

struct Shl {
    int l, np;
    double a[MAXPRIM], c[MAXPRIM];
};

__device__ __forceinline__ void load_shell(const Batch& B, int s, Shl& sh) {
    sh.l = B.s_l[s];
    sh.np = B.s_np[s];
    for (int p = 0; p < MAXPRIM; p++) {
        sh.a[p] = B.s_alpha[s * MAXPRIM + p];
        sh.c[p] = B.s_coeff[s * MAXPRIM + p];
    }
}

__device__ __forceinline__ int ncart(int l) { return (l + 1) * (l + 2) / 2; }
__device__ __forceinline__ int nsph(int l) { return 2 * l + 1; }

// Cartesian exponents in the order x^lx y^ly z^lz with lx descending, then ly descending
__device__ __forceinline__ void cart_exp(int l, int c, int e[3]) {
    int k = 0;
    for (int lx = l; lx >= 0; lx--)
        for (int ly = l - lx; ly >= 0; ly--) {
            if (k == c) {
                e[0] = lx;
                e[1] = ly;
                e[2] = l - lx - ly;
                return;
            }
            k++;
        }
}

// Cartesian-to-spherical factor T_l[m][c] (m: -l..l; p: y, z, x)
__device__ __forceinline__ double sph_t(int l, int m, int c) {
    if (l == 0) return 1.0;
    if (l == 1) return (m == 0 && c == 1) || (m == 1 && c == 2) || (m == 2 && c == 0) ? 1.0 : 0.0;
    const double s3 = 1.7320508075688772, s3_4 = 0.8660254037844386;
    switch (m * 6 + c) {
        case 0 * 6 + 1: return s3;
        case 1 * 6 + 4: return s3;
        case 2 * 6 + 0: return -0.5;
        case 2 * 6 + 3: return -0.5;
        case 2 * 6 + 5: return 1.0;
        case 3 * 6 + 2: return s3;
        case 4 * 6 + 0: return s3_4;
        case 4 * 6 + 3: return -s3_4;
        default: return 0.0;
    }
}

// one-dimensional Obara-Saika table t[a][b] = int (x-A)^a (x-B)^b (unscaled) for a <= LA, b <= LB
template <int LA, int LB>
__device__ __forceinline__ void os_1d(double rpa, double rpb, double h, double (&t)[LA + 1][LB + 1]) {
    t[0][0] = 1.0;
    if constexpr (LA >= 1) {
        t[1][0] = rpa;
#pragma unroll
        for (int i = 1; i < LA; i++) t[i + 1][0] = rpa * t[i][0] + i * h * t[i - 1][0];
    }
    if constexpr (LB >= 1) {
        t[0][1] = rpb;
#pragma unroll
        for (int i = 1; i <= LA; i++) t[i][1] = rpb * t[i][0] + i * h * t[i - 1][0];
#pragma unroll
        for (int j = 1; j < LB; j++) {
            t[0][j + 1] = rpb * t[0][j] + j * h * t[0][j - 1];
#pragma unroll
            for (int i = 1; i <= LA; i++) t[i][j + 1] = rpb * t[i][j] + h * (i * t[i - 1][j] + j * t[i][j - 1]);
        }
    }
}

// the same table for runtime la, lb (the S, D, Q integrals: their bits steer a few chaotic SCFs,
// so they keep this form)
__device__ __forceinline__ void os_1d(int la, int lb, double rpa, double rpb, double h, double t[6][6]) {
    t[0][0] = 1.0;
    if (la >= 1) {
        t[1][0] = rpa;
        for (int i = 1; i < la; i++) t[i + 1][0] = rpa * t[i][0] + i * h * t[i - 1][0];
    }
    if (lb >= 1) {
        t[0][1] = rpb;
        for (int i = 1; i <= la; i++) t[i][1] = rpb * t[i][0] + i * h * t[i - 1][0];
        for (int j = 1; j < lb; j++) {
            t[0][j + 1] = rpb * t[0][j] + j * h * t[0][j - 1];
            for (int i = 1; i <= la; i++) t[i][j + 1] = rpb * t[i][j] + h * (i * t[i - 1][j] + j * t[i][j - 1]);
        }
    }
}

__device__ __forceinline__ void traceless6(double* q) {
    double tr = 0.5 * (q[0] + q[2] + q[5]);
    q[0] = 1.5 * q[0] - tr;
    q[1] *= 1.5;
    q[2] = 1.5 * q[2] - tr;
    q[3] *= 1.5;
    q[4] *= 1.5;
    q[5] = 1.5 * q[5] - tr;
}

__device__ __forceinline__ bool prim_pref(double ai, double aj, double r2, double intcut, double& oab, double& pre) {
    double eab = ai + aj;
    oab = 1.0 / eab;
    double est = ai * aj * r2 * oab;
    if (est > intcut) return false;
    const double sqrtpi3 = 5.568327996831708;  // pi^(3/2)
    double so = sqrt(oab);
    pre = exp(-est) * sqrtpi3 * (so * so * so);
    return true;
}

__device__ __forceinline__ bool pair_screened(double a, double b, double r2, double intcut) {
    return a * b * r2 / (a + b) > intcut * (1.0 + 1e-10);
}

// S, D (about R_i) and traceless Q (about R_i) of (bra cj at R_j, ket ci at R_i), vec = R_i - R_j.
// Outputs in spherical order, block index jm + nsph(lj)*im.
__device__ void multipole_block(const Shl& cj, const Shl& ci, const double vec[3], double intcut, double* s, double* d,
                                double* q) {
    double r2 = vec[0] * vec[0] + vec[1] * vec[1] + vec[2] * vec[2];
    int li = ci.l, lj = cj.l, ncj = ncart(lj), nci = ncart(li);
    double cart[36][10];
    for (int p = 0; p < ncj * nci; p++)
        for (int x = 0; x < 10; x++) cart[p][x] = 0.0;
    double t[3][6][6];
    for (int ip = 0; ip < ci.np; ip++)
        for (int jp = 0; jp < cj.np; jp++) {
            double ai = ci.a[ip], aj = cj.a[jp], oab, pre;
            if (!prim_pref(ai, aj, r2, intcut, oab, pre)) continue;
            for (int k = 0; k < 3; k++) os_1d(li + 2, lj, -vec[k] * aj * oab, vec[k] * ai * oab, 0.5 * oab, t[k]);
            double cc = ci.c[ip] * cj.c[jp] * pre;
            for (int ic = 0; ic < nci; ic++) {
                int ea[3];
                cart_exp(li, ic, ea);
                for (int jc = 0; jc < ncj; jc++) {
                    int eb[3];
                    cart_exp(lj, jc, eb);
                    double v[3][3];
                    for (int k = 0; k < 3; k++)
                        for (int mm = 0; mm < 3; mm++) v[k][mm] = t[k][ea[k] + mm][eb[k]];
                    double* c = cart[jc + ncj * ic];
                    c[0] += cc * v[0][0] * v[1][0] * v[2][0];
                    c[1] += cc * v[0][1] * v[1][0] * v[2][0];
                    c[2] += cc * v[0][0] * v[1][1] * v[2][0];
                    c[3] += cc * v[0][0] * v[1][0] * v[2][1];
                    c[4] += cc * v[0][2] * v[1][0] * v[2][0];
                    c[5] += cc * v[0][1] * v[1][1] * v[2][0];
                    c[6] += cc * v[0][0] * v[1][2] * v[2][0];
                    c[7] += cc * v[0][1] * v[1][0] * v[2][1];
                    c[8] += cc * v[0][0] * v[1][1] * v[2][1];
                    c[9] += cc * v[0][0] * v[1][0] * v[2][2];
                }
            }
        }
    int nsj = nsph(lj), nsi = nsph(li);
    for (int im = 0; im < nsi; im++)
        for (int jm = 0; jm < nsj; jm++) {
            double o[10];
            for (int x = 0; x < 10; x++) o[x] = 0.0;
            for (int ic = 0; ic < nci; ic++) {
                double ti = sph_t(li, im, ic);
                if (ti == 0.0) continue;
                for (int jc = 0; jc < ncj; jc++) {
                    double tj = sph_t(lj, jm, jc);
                    if (tj == 0.0) continue;
                    for (int x = 0; x < 10; x++) o[x] += tj * ti * cart[jc + ncj * ic][x];
                }
            }
            int k = jm + nsj * im;
            s[k] = o[0];
            for (int x = 0; x < 3; x++) d[3 * k + x] = o[1 + x];
            double qq[6] = {o[4], o[5], o[6], o[7], o[8], o[9]};
            traceless6(qq);
            for (int x = 0; x < 6; x++) q[6 * k + x] = qq[x];
        }
}

__device__ __forceinline__ void shift_bra(const double vec[3], double s, const double* di, const double* qi, double* dj,
                                          double* qj) {
    for (int k = 0; k < 3; k++) dj[k] = di[k] + vec[k] * s;
    qj[0] = 2.0 * vec[0] * di[0] + vec[0] * vec[0] * s;
    qj[1] = vec[0] * di[1] + vec[1] * di[0] + vec[0] * vec[1] * s;
    qj[2] = 2.0 * vec[1] * di[1] + vec[1] * vec[1] * s;
    qj[3] = vec[0] * di[2] + vec[2] * di[0] + vec[0] * vec[2] * s;
    qj[4] = vec[1] * di[2] + vec[2] * di[1] + vec[1] * vec[2] * s;
    qj[5] = 2.0 * vec[2] * di[2] + vec[2] * vec[2] * s;
    traceless6(qj);
    for (int k = 0; k < 6; k++) qj[k] += qi[k];
}

__device__ __forceinline__ double kshell(int k, int l) {
    const double KD[3] = {1.85, 2.23, 2.23};
    if ((k == 2 && (l == 0 || l == 1)) || (l == 2 && (k == 0 || k == 1))) return 2.0;
    return (KD[l] + KD[k]) / 2.0;
}
// H0 scaling of (bra shell sj on atom aj, ket shell si on atom ai): crates/axtb/src/gfn2.rs:73-89
__device__ __forceinline__ double hscale(const Batch& B, int sj, int aj, int si, int ai) {
    double den = sq(B.a_en[aj] - B.a_en[ai]);
    double za = B.s_slater[sj], zb = B.s_slater[si];
    double zij = sqrt(2.0 * sqrt(za * zb) / (za + zb));
    return zij * (kshell(B.s_l[si], B.s_l[sj]) * (1.0 + 2.0e-2 * den));
}

// pair index with the diagonal: p = i(i+1)/2 + j, j <= i
__device__ __forceinline__ void unpack_pair_diag(long long p, int& i, int& j) {
    int ii = (int)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
    while ((long long)(ii + 1) * (ii + 2) / 2 <= p) ii++;
    while ((long long)ii * (ii + 1) / 2 > p) ii--;
    i = ii;
    j = (int)(p - (long long)ii * (ii + 1) / 2);
}
__device__ __forceinline__ void unpack_pair(long long p, int& i, int& j) {  // p = i(i-1)/2 + j, j < i
    unpack_pair_diag(p, i, j);  // i(i+1)/2 + j form of p gives (i', j'); convert
    // p = i(i-1)/2 + j with j < i  <=>  p = (i-1)i/2 + j, i.e. diagonal form with row i-1, col j <= i-1
    i = i + 1;
}

// S, H0, D, Q of every atom pair (i >= j) of every molecule; m_pd0 = offsets of the pairs with
// diagonal (sum of nat(nat+1)/2)
__global__ void k_integrals(Batch B, State S, const long long* m_pd0, long long npd) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= npd) return;
    int m = find_mol(m_pd0, B.nmol, g);
    int li, lj;
    unpack_pair_diag(g - m_pd0[m], li, lj);
    int ia = B.m_at0[m] + li, ja = B.m_at0[m] + lj;
    int n = B.m_nao[m], ao0 = B.m_ao0[m];
    long long mat = B.m_mat0[m], nn = B.nnT;
    double vec[3];
    dvec(S.xyz, ia, ja, vec);
    double r2 = vec[0] * vec[0] + vec[1] * vec[1] + vec[2] * vec[2];
    bool onsite = ia == ja;
    // atom pairs beyond the conventions' distance cutoff (tblite) or screened by their exponents
    if (!onsite && (r2 > B.m_paircut2[m] || pair_screened(B.a_amin[ia], B.a_amin[ja], r2, B.intcut))) return;
    double rr = onsite ? 0.0 : sqrt(sqrt(r2) / (B.a_rad[ja] + B.a_rad[ia]));
    double s[25], d[75], q[150];
    Shl ci, cj;
    for (int si = B.a_sh0[ia]; si < B.a_sh0[ia] + B.a_nsh[ia]; si++) {
        load_shell(B, si, ci);
        for (int sj = B.a_sh0[ja]; sj < B.a_sh0[ja] + B.a_nsh[ja]; sj++) {
            if (!onsite && pair_screened(B.s_amin[si], B.s_amin[sj], r2, B.intcut)) continue;
            load_shell(B, sj, cj);
            multipole_block(cj, ci, vec, B.intcut, s, d, q);
            double hij;
            if (onsite) hij = 0.5 * (S.se[si] + S.se[sj]);
            else {
                double shp = (1.0 + B.s_shpoly[si] * rr) * (1.0 + B.s_shpoly[sj] * rr);
                hij = 0.5 * (S.se[si] + S.se[sj]) * hscale(B, sj, ja, si, ia) * shp;
            }
            int nsj = nsph(cj.l);
            for (int im = 0; im < nsph(ci.l); im++)
                for (int jm = 0; jm < nsj; jm++) {
                    int k = jm + nsj * im;
                    int mu = B.s_ao0[sj] + jm - ao0, nu = B.s_ao0[si] + im - ao0;
                    long long e1 = mat + mu + (long long)nu * n;
                    S.S[e1] = s[k];
                    S.H0[e1] = s[k] * hij;
                    for (int x = 0; x < 3; x++) S.D[x * nn + e1] = d[3 * k + x];
                    for (int x = 0; x < 6; x++) S.Q[x * nn + e1] = q[6 * k + x];
                    if (!onsite) {
                        double dj[3], qj[6];
                        shift_bra(vec, s[k], &d[3 * k], &q[6 * k], dj, qj);
                        long long e2 = mat + nu + (long long)mu * n;
                        S.S[e2] = s[k];
                        S.H0[e2] = s[k] * hij;
                        for (int x = 0; x < 3; x++) S.D[x * nn + e2] = dj[x];
                        for (int x = 0; x < 6; x++) S.Q[x * nn + e2] = qj[x];
                    }
                }
        }
    }
}

// One shell pair's part of k_h0_gradient (shell si of angular momentum LI on atom i, sj of LJ on
// atom j): compile-time sizes keep the Cartesian weights and accumulators in registers for s and p
// shells; the operations of the generic loop in the same order (the compiler may fuse other
// products: the gradient agrees to round-off)
template <int LI, int LJ>
__device__ __noinline__ void shell_pair_h0_gradient(const Batch& B, const State& S, const Shl& ci, const Shl& cj, int si, int sj,
                                       int ia, int ja, const double vec[3], double r2, double rr, int n, int ao0,
                                       long long mat, const double* vdi, const double* vdj, const double* vqi,
                                       const double* vqj, double dg[3], double& dcni, double& dcnj) {
    constexpr int NCI = (LI + 1) * (LI + 2) / 2, NCJ = (LJ + 1) * (LJ + 2) / 2;
    constexpr int NSI = 2 * LI + 1, NSJ = 2 * LJ + 1;
    const int MOM[10][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0},
                            {1, 1, 0}, {0, 2, 0}, {1, 0, 1}, {0, 1, 1}, {0, 0, 2}};
    const int AB[6][2] = {{0, 0}, {0, 1}, {1, 1}, {0, 2}, {1, 2}, {2, 2}};
    // shell-pair factors of H0
    double shpi = 1.0 + B.s_shpoly[si] * rr, shpj = 1.0 + B.s_shpoly[sj] * rr;
    double shp = shpi * shpj;
    double dshp = (shpi * B.s_shpoly[sj] + shpj * B.s_shpoly[si]) * 0.5 * rr / r2;
    double dsv[3] = {dshp / shp * vec[0], dshp / shp * vec[1], dshp / shp * vec[2]};
    double hs = hscale(B, sj, ja, si, ia) * shp;
    double hij = 0.5 * (S.se[si] + S.se[sj]) * hs;
    double dhdcni = S.dsedcn[si] * hs, dhdcnj = S.dsedcn[sj] * hs;
    // The contraction is linear in the integrals of each AO pair, and its multipole part uses the
    // same potentials for all of them: the spherical transform moves onto three Cartesian weights
    // (P, the overlap-derivative factor, 2 P h), so the integrals are accumulated as they are made
    // instead of held per Cartesian pair.
    double wp[NCI * NCJ], ws[NCI * NCJ], wh[NCI * NCJ];
#pragma unroll
    for (int c = 0; c < NCI * NCJ; c++) wp[c] = ws[c] = wh[c] = 0.0;
#pragma unroll
    for (int im = 0; im < NSI; im++)
#pragma unroll
        for (int jm = 0; jm < NSJ; jm++) {
            int mu = B.s_ao0[sj] + jm - ao0, nu = B.s_ao0[si] + im - ao0;
            long long e1 = mat + mu + (long long)nu * n;
            double pij = S.P[e1], hpij = pij * hij;
            int amu = B.s_ao0[sj] + jm, anu = B.s_ao0[si] + im;
            double vmu = S.vsh[B.o_sh[amu]] + S.vat[B.o_at[amu]];
            double vnu = S.vsh[B.o_sh[anu]] + S.vat[B.o_at[anu]];
            double sval = -pij * (vmu + vnu) + 2.0 * hpij - 2.0 * S.W[e1];
#pragma unroll
            for (int ic = 0; ic < NCI; ic++) {
                double ti = sph_t(LI, im, ic);
                if (ti == 0.0) continue;
#pragma unroll
                for (int jc = 0; jc < NCJ; jc++) {
                    double tj = sph_t(LJ, jm, jc);
                    if (tj == 0.0) continue;
                    double f = tj * ti;
                    int c = jc + NCJ * ic;
                    wp[c] += f * pij;
                    ws[c] += f * sval;
                    wh[c] += f * (2.0 * hpij);
                }
            }
        }
    // weighted Cartesian values [s, d_j(3), m_j(6)] and R_i derivatives (moments about R_j): av, ad
    // with the P weights; sds = the overlap derivative with its factor; sh = the overlap with 2 P h
    double av[10], ad[30], sds[3] = {0.0, 0.0, 0.0}, sh = 0.0;
#pragma unroll
    for (int x = 0; x < 10; x++) av[x] = 0.0;
#pragma unroll
    for (int x = 0; x < 30; x++) ad[x] = 0.0;
    double t[3][LI + 2][LJ + 3];
    for (int ip = 0; ip < ci.np; ip++) {
        double ai2 = 2.0 * ci.a[ip];
        for (int jp = 0; jp < cj.np; jp++) {
            double ai = ci.a[ip], aj = cj.a[jp], oab, pre;
            if (!prim_pref(ai, aj, r2, B.intcut, oab, pre)) continue;
#pragma unroll
            for (int k = 0; k < 3; k++) os_1d<LI + 1, LJ + 2>(-vec[k] * aj * oab, vec[k] * ai * oab, 0.5 * oab, t[k]);
            double cc = ci.c[ip] * cj.c[jp] * pre;
#pragma unroll
            for (int ic = 0; ic < NCI; ic++) {
                int ea[3];
                cart_exp(LI, ic, ea);
#pragma unroll
                for (int jc = 0; jc < NCJ; jc++) {
                    int c = jc + NCJ * ic;
                    double fp = cc * wp[c], fs = cc * ws[c], fh = cc * wh[c];
                    int eb[3];
                    cart_exp(LJ, jc, eb);
                    double v[3][3], gg[3][3];
#pragma unroll
                    for (int k = 0; k < 3; k++)
#pragma unroll
                        for (int mm = 0; mm < 3; mm++) {
                            v[k][mm] = t[k][ea[k]][eb[k] + mm];
                            double x = ai2 * t[k][ea[k] + 1][eb[k] + mm];
                            if (ea[k] > 0) x -= ea[k] * t[k][ea[k] - 1][eb[k] + mm];
                            gg[k][mm] = x;
                        }
#pragma unroll
                    for (int nq = 0; nq < 10; nq++) {
                        double X = v[0][MOM[nq][0]], Y = v[1][MOM[nq][1]], Zz = v[2][MOM[nq][2]];
                        double d0 = gg[0][MOM[nq][0]] * Y * Zz, d1 = X * gg[1][MOM[nq][1]] * Zz;
                        double d2 = X * Y * gg[2][MOM[nq][2]], xyz = X * Y * Zz;
                        av[nq] += fp * xyz;
                        ad[3 * nq] += fp * d0;
                        ad[3 * nq + 1] += fp * d1;
                        ad[3 * nq + 2] += fp * d2;
                        if (nq == 0) {
                            sds[0] += fs * d0;
                            sds[1] += fs * d1;
                            sds[2] += fs * d2;
                            sh += fh * xyz;
                        }
                    }
                }
            }
        }
    }
    // the multipole part: moments about R_i from those about R_j, traceless quadrupoles,
    // contracted with the atomic dipole and quadrupole potentials
    double s = av[0];
    double djv[3] = {av[1], av[2], av[3]};
    double ds[3] = {ad[0], ad[1], ad[2]};
    double ddj[3][3], dmj[3][6], ddi[3][3], dmi[3][6];
#pragma unroll
    for (int k = 0; k < 3; k++) {
#pragma unroll
        for (int c = 0; c < 3; c++) ddj[k][c] = ad[3 * (1 + c) + k];
#pragma unroll
        for (int c = 0; c < 6; c++) dmj[k][c] = ad[3 * (4 + c) + k];
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
#pragma unroll
        for (int c = 0; c < 3; c++) ddi[k][c] = ddj[k][c] - vec[c] * ds[k];
        ddi[k][k] -= s;
#pragma unroll
        for (int nq = 0; nq < 6; nq++) {
            int a_ = AB[nq][0], b_ = AB[nq][1];
            double x = dmj[k][nq] - vec[a_] * ddj[k][b_] - vec[b_] * ddj[k][a_] + vec[a_] * vec[b_] * ds[k];
            if (a_ == k) x += -djv[b_] + vec[b_] * s;
            if (b_ == k) x += -djv[a_] + vec[a_] * s;
            dmi[k][nq] = x;
        }
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        traceless6(dmi[k]);
        traceless6(dmj[k]);
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        double mp = 0.0;
#pragma unroll
        for (int c = 0; c < 3; c++) mp += ddi[k][c] * vdi[c] + ddj[k][c] * vdj[c];
#pragma unroll
        for (int c = 0; c < 6; c++) mp += dmi[k][c] * vqi[c] + dmj[k][c] * vqj[c];
        dg[k] += sds[k] + sh * dsv[k] - mp;
    }
    dcni += dhdcni * s;
    dcnj += dhdcnj * s;
}

// Nuclear gradient of the one-electron energy per atom pair (i > j): dE/dR_i (= -dE/dR_j) and
// the CN derivatives of both atoms, from the ket-centre derivatives of S, D, Q contracted with
// P, W, the AO charge potential and the atomic multipole potentials (crates/axtb/src/hamiltonian.rs:101-223).
// out[pair*5 + (0..2)] = dg, [3] = dE/dCN_i, [4] = dE/dCN_j
__global__ void __launch_bounds__(128, 3) k_h0_gradient(Batch B, State S, const long long* m_pair0, long long np, double* out) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= np) return;
    int m = find_mol(m_pair0, B.nmol, g);
    int li, lj;
    unpack_pair(g - m_pair0[m], li, lj);
    int ia = B.m_at0[m] + li, ja = B.m_at0[m] + lj;
    int n = B.m_nao[m], ao0 = B.m_ao0[m];
    long long mat = B.m_mat0[m];
    double* o = out + g * 5;
    for (int x = 0; x < 5; x++) o[x] = 0.0;
    double vec[3];
    dvec(S.xyz, ia, ja, vec);
    double r2 = vec[0] * vec[0] + vec[1] * vec[1] + vec[2] * vec[2];
    if (r2 > B.m_paircut2[m] || pair_screened(B.a_amin[ia], B.a_amin[ja], r2, B.intcut) || r2 < DBL_EPSILON) return;
    double rr = sqrt(sqrt(r2) / (B.a_rad[ja] + B.a_rad[ia]));
    const double* vdi = S.vdp + 3 * ia;
    const double* vdj = S.vdp + 3 * ja;
    const double* vqi = S.vqp + 6 * ia;
    const double* vqj = S.vqp + 6 * ja;
    double dg[3] = {0, 0, 0}, dcni = 0.0, dcnj = 0.0;
    Shl ci, cj;
    for (int si = B.a_sh0[ia]; si < B.a_sh0[ia] + B.a_nsh[ia]; si++) {
        load_shell(B, si, ci);
        for (int sj = B.a_sh0[ja]; sj < B.a_sh0[ja] + B.a_nsh[ja]; sj++) {
            if (pair_screened(B.s_amin[si], B.s_amin[sj], r2, B.intcut)) continue;
            load_shell(B, sj, cj);
            switch (ci.l * 3 + cj.l) {
#define AXG_H0G(L1, L2) \
    shell_pair_h0_gradient<L1, L2>(B, S, ci, cj, si, sj, ia, ja, vec, r2, rr, n, ao0, mat, vdi, vdj, vqi, vqj, dg, dcni, dcnj)
                case 0: AXG_H0G(0, 0); break;
                case 1: AXG_H0G(0, 1); break;
                case 2: AXG_H0G(0, 2); break;
                case 3: AXG_H0G(1, 0); break;
                case 4: AXG_H0G(1, 1); break;
                case 5: AXG_H0G(1, 2); break;
                case 6: AXG_H0G(2, 0); break;
                case 7: AXG_H0G(2, 1); break;
                default: AXG_H0G(2, 2); break;
#undef AXG_H0G
            }
        }
    }
    o[0] = dg[0];
    o[1] = dg[1];
    o[2] = dg[2];
    o[3] = dcni;
    o[4] = dcnj;
}

}  // namespace axg
