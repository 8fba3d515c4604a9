// TEST INFRASTRUCTURE - NOT PART OF THE PRODUCT.
//
// CPU FP64 restatement of the GFN2-xTB energy + analytic nuclear gradient of axtb
// (default "axtb" conventions, crates/axtb/src/conventions.rs:244-268), written from the
// reference's algorithm, one function per reference routine, each citing the file:line it
// follows (paths relative to the axtb checkout). It is the parity checker of the CUDA path and
// the CPU baseline of bench.py; nothing in the product links it.
//
// Dense eigenproblems: the reference uses faer 0.22.6 (Cholesky, Householder
// tridiagonalisation, dsterf/dstein-style occupied-only eigenvectors; not vendored). Here the
// same mathematically unique quantities (all eigenvalues, the occupied subspace) come from a
// Cholesky reduction and Householder tridiagonalisation + implicit QL (EISPACK tred2/tql2), or
// from an optional LAPACK found at run time; energies agree to round-off either way.
#include "gfn2_oracle.h"

#include <dlfcn.h>

#include <algorithm>
#include <array>
#include <cstdlib>
#include <cctype>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../axtb_b200/csrc/params/gfn2_tables.h"
#include "../axtb_b200/csrc/params/solvation_tables.h"

using namespace gfn2tab;
using std::vector;

namespace {

// ---- constants: crates/base/src/units.rs:18-24, 53-88
const double PI = 3.14159265358979323846;
const double AUTOAA = 5.29177210544e-11 * 1e10;
const double AATOAU = 1.0 / AUTOAA;
const double KB_HARTREE = 3.1668115634564e-6;
const double PLANCK_2018 = 6.62607015e-34;
const double ME_2018 = 9.1093837015e-31;
const double C_LIGHT = 299792458.0;
const double ALPHA_2018 = 7.2973525693e-3;
const double HBAR_2018 = PLANCK_2018 / (2.0 * PI);
const double BOHR_M_2018 = HBAR_2018 / (ME_2018 * C_LIGHT * ALPHA_2018);
const double MCTC_AATOAU = 1.0 / (BOHR_M_2018 * 1e10);

struct Fail : std::runtime_error {
    int code;
    Fail(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Atomic radii (Angstrom) of mctc-lib; crates/axtb/src/param/element_data.rs:60-92.
const double ATOMIC_RAD_AA_TAB[118] = {
    0.32, 0.37, 1.30, 0.99, 0.84, 0.75, 0.71, 0.64, 0.60, 0.62, 1.60, 1.40, 1.24, 1.14, 1.09,
    1.04, 1.00, 1.01, 2.00, 1.74, 1.59, 1.48, 1.44, 1.30, 1.29, 1.24, 1.18, 1.17, 1.22, 1.20,
    1.23, 1.20, 1.20, 1.18, 1.17, 1.16, 2.15, 1.90, 1.76, 1.64, 1.56, 1.46, 1.38, 1.36, 1.34,
    1.30, 1.36, 1.40, 1.42, 1.40, 1.40, 1.37, 1.36, 1.36, 2.38, 2.06, 1.94, 1.84, 1.90, 1.88,
    1.86, 1.85, 1.83, 1.82, 1.81, 1.80, 1.79, 1.77, 1.77, 1.78, 1.74, 1.64, 1.58, 1.50, 1.41,
    1.36, 1.32, 1.30, 1.30, 1.32, 1.44, 1.45, 1.50, 1.42, 1.48, 1.46, 2.42, 2.11, 2.01, 1.90,
    1.84, 1.83, 1.80, 1.80, 1.73, 1.68, 1.68, 1.68, 1.65, 1.67, 1.73, 1.76, 1.61, 1.57, 1.49,
    1.43, 1.41, 1.34, 1.29, 1.28, 1.21, 1.22, 1.36, 1.43, 1.62, 1.75, 1.65, 1.57};
double ATOMIC_RAD_AA(int z) { return ATOMIC_RAD_AA_TAB[z - 1]; }

// ---- element radii of the axtb conventions: crates/axtb/src/param/mod.rs:39-48
double rcov_codata(int z) { return 4.0 / 3.0 * (COVALENT_RAD_2009_AA[z - 1] * AATOAU); }
double atomic_rad_codata(int z) { return ATOMIC_RAD_AA(z) * AATOAU; }
// mctc-lib radii of the EEQ guess CN: crates/axtb/src/param/element_data.rs:15-24,94-103
double rcov_mctc(int z) { return 4.0 / 3.0 * (MCTC_AATOAU * COVALENT_RAD_2009_AA[z - 1]); }
// mctc-lib's atomic radii in bohr (tblite): crates/axtb/src/param/element_data.rs:26-58
double atomic_rad_mctc(int z) { return MCTC_AATOAU * ATOMIC_RAD_AA(z); }

// ---- conventions (crates/axtb/src/conventions.rs:150-353): the settings that differ between
// axtb's default conventions, the xtb 6.8.0 program's and tblite 0.8.0's. Not restated: the
// xtb 6.7.1 row; the per-triple ATM order and the full eigensolver of the program conventions
// (the same numbers up to round-off as the pair sums and the occupied-only solve used here).
const double KB_XTB_TBLITE = 3.166808578545117e-06;  // crates/base/src/units.rs:81
struct Conv {
    int id = 0;                    // 0 axtb, 1 xtb (6.8.0), 2 tblite (0.8.0)
    double kb = KB_HARTREE;        // Boltzmann constant of the electronic temperature
    double aufbau_max_etemp = 0.0; // up to this temperature (K) no Fermi smearing
    bool eeq_guess = true;         // EEQ start (tblite: zero charges)
    double eeq_cn_cut = 25.0, eeq_cap = 8.0;  // EEQ-guess CN cutoff; log cap (<= 0: none)
    double cn_cut = 40.0, rep_cut = 40.0;     // GFN2 CN and repulsion cutoffs
    double d4_cn_cut = 40.0, d2_cut = 72.0, d2_w = 1.0, d3_cut = 40.0, d3_w = 1.0;
    bool output_aes = false;       // gradient with the AES potentials of the output moments
    int default_mixer = 0;         // 0 auto, 1 Broyden
};
thread_local Conv g_conv;

Conv make_conv(int id) {
    Conv c;
    c.id = id;
    if (id == 0) return c;
    // xtb 6.8.0 and tblite 0.8.0: conventions.rs:274-298 and 326-350
    c.kb = KB_XTB_TBLITE;
    c.cn_cut = c.rep_cut = 25.0;
    c.d4_cn_cut = 30.0;  // RealspaceCutoff::TBLITE_GFN2, crates/d4/src/disp.rs:44-47
    c.d2_cut = 50.0;
    c.d3_cut = 25.0;
    c.d2_w = c.d3_w = 0.05;
    c.default_mixer = 1;
    if (id == 1) {
        c.aufbau_max_etemp = 0.1;
        c.eeq_cn_cut = 40.0;  // the xtb program's guess CN: its D4 radii, 40 bohr, no cap
        c.eeq_cap = 0.0;
        c.output_aes = true;
    } else {
        c.eeq_guess = false;
    }
    return c;
}
// element tables of the conventions
double conv_en(int z) { return g_conv.id == 1 ? XTB_PAULING_EN[z - 1] : PAULING_EN[z - 1]; }
double conv_atomic_rad(int z) {
    return g_conv.id == 1 ? XTB_ATOMIC_RAD[z - 1] : g_conv.id == 2 ? atomic_rad_mctc(z) : atomic_rad_codata(z);
}
double conv_cn_rcov(int z) {
    return g_conv.id == 1 ? XTB_COVALENT_RAD_D3[z - 1] : g_conv.id == 2 ? rcov_mctc(z) : rcov_codata(z);
}
double conv_d4_rcov(int z) {
    return g_conv.id == 1 ? XTB_D4_RCOV[z - 1] : g_conv.id == 2 ? rcov_mctc(z) : rcov_codata(z);
}
double conv_d4_en(int z) { return g_conv.id == 1 ? XTB_D4_EN[z - 1] : PAULING_EN[z - 1]; }
double conv_eeq_rcov(int z) { return g_conv.id == 1 ? XTB_D4_RCOV[z - 1] : rcov_mctc(z); }
// tblite's screening threshold (crates/axtb/src/basis.rs:140-143)
double integral_cutoff_tblite(double acc) {
    acc = std::min(std::max(acc, 1.0e-4), 1.0e3);
    return std::min(std::max(25.0 - 10.0 * std::log10(acc), 5.0), 25.0);
}


inline double sq(double x) { return x * x; }

// ============================================================================ molecule, basis
struct Shell {
    int l = 0, np = 0;
    double a[6] = {0}, c[6] = {0};
    double amin = 0;
};

// STO-nG expansion with tblite's primitive normalisation: crates/axtb/src/basis.rs:20-81,
// crates/base/src/math.rs:134-138.
Shell slater_to_gauss(int ng, int n, int l, double zeta) {
    if ((n > 5 || n <= l) && !(n == 6 && ng == 6)) throw Fail(1, "STO-NG: unsupported n, l");
    int ityp;
    switch (l) {
        case 0: ityp = n; break;
        case 1: ityp = 4 + n; break;
        case 2: ityp = 7 + n; break;
        default: throw Fail(1, "STO-NG: l > 2 not in GFN2");
    }
    ityp -= 1;
    Shell s;
    s.l = l;
    s.np = ng;
    double z2 = zeta * zeta;
    auto fill = [&](const double* a, const double* c) {
        for (int i = 0; i < ng; i++) {
            s.a[i] = a[i] * z2;
            s.c[i] = c[i];
        }
    };
    switch (ng) {
        case 1: s.a[0] = P_ALPHA1[ityp] * z2; s.c[0] = 1.0; break;
        case 2: fill(P_ALPHA2[ityp], P_COEFF2[ityp]); break;
        case 3: fill(P_ALPHA3[ityp], P_COEFF3[ityp]); break;
        case 4: fill(P_ALPHA4[ityp], P_COEFF4[ityp]); break;
        case 5: fill(P_ALPHA5[ityp], P_COEFF5[ityp]); break;
        case 6:
            if (n == 6) {
                if (l == 0) fill(P_ALPHA_6S, P_COEFF_6S);
                else if (l == 1) fill(P_ALPHA_6P, P_COEFF_6P);
                else throw Fail(1, "STO-6G n=6 only for s and p");
            } else {
                fill(P_ALPHA6[ityp], P_COEFF6[ityp]);
            }
            break;
        default: throw Fail(1, "STO-NG: unsupported primitive count");
    }
    static const double DFACT[5] = {1.0, 1.0, 3.0, 15.0, 105.0};
    for (int i = 0; i < ng; i++) {
        double top = 2.0 / PI;
        double r = std::sqrt(4.0 * s.a[i]);
        double pw = 1.0;
        for (int k = 0; k < l; k++) pw *= r;
        s.c[i] *= std::pow(top * s.a[i], 0.75) * pw / std::sqrt(DFACT[l]);
    }
    s.amin = INFINITY;
    for (int i = 0; i < ng; i++) s.amin = std::min(s.amin, s.a[i]);
    return s;
}

struct Mol {
    int nat = 0;
    vector<int> Z;
    vector<double> xyz;  // nat*3
    double charge = 0;
    int uhf = -1;
    vector<int> species, id;  // species by first appearance (crates/base/src/molecule.rs:35-60)
    const double* R(int i) const { return &xyz[3 * i]; }
};

struct Basis {
    int nsh = 0, nao = 0;
    vector<Shell> sh;            // per shell (basis order)
    vector<int> sh2at, iao_sh, ish_at, nsh_at, iao_at, nao_at, ao2at, ao2sh;
    vector<double> amin_at;
    double intcut = 25.0;
    double pair_cut2 = INFINITY;  // squared atom-pair distance cutoff of the integrals
};

// crates/axtb/src/gfn2.rs:34-56 and crates/axtb/src/basis.rs:165-229
Basis build_basis(const Mol& m, double acc) {
    Basis b;
    for (int iat = 0; iat < m.nat; iat++) {
        int z = m.Z[iat];
        if (z > 86) throw Fail(2, "GFN2-xTB: unsupported element");
        b.ish_at.push_back(b.nsh);
        b.iao_at.push_back(b.nao);
        b.nsh_at.push_back(NSHELL[z - 1]);
        double amin = INFINITY;
        for (int ish = 0; ish < NSHELL[z - 1]; ish++) {
            Shell s = slater_to_gauss(NUMBER_OF_PRIMITIVES[z - 1][ish], PRINCIPAL_QUANTUM_NUMBER[z - 1][ish],
                                      ANG_SHELL[z - 1][ish], SLATER_EXPONENT[z - 1][ish]);
            b.sh.push_back(s);
            b.sh2at.push_back(iat);
            b.iao_sh.push_back(b.nao);
            for (int k = 0; k < 2 * s.l + 1; k++) {
                b.ao2at.push_back(iat);
                b.ao2sh.push_back(b.nsh);
            }
            b.nao += 2 * s.l + 1;
            b.nsh++;
            amin = std::min(amin, s.amin);
        }
        b.nao_at.push_back(b.nao - b.iao_at[iat]);
        b.amin_at.push_back(amin);
    }
    // primitive screening (crates/axtb/src/gfn2.rs:58-62): axtb the xtb program's threshold
    // (crates/axtb/src/basis.rs:135-137), xtb 6.8.0 tblite's at the SCF accuracy, tblite tblite's at
    // accuracy 1; tblite also leaves out atom pairs beyond sqrt(2 cut(acc) / min alpha), at most
    // 40 bohr (crates/axtb/src/basis.rs:247-249)
    if (g_conv.id == 0) b.intcut = std::max(25.0 - 10.0 * std::log10(acc), 20.0);
    else if (g_conv.id == 1) b.intcut = integral_cutoff_tblite(acc);
    else b.intcut = integral_cutoff_tblite(1.0);
    b.pair_cut2 = INFINITY;
    if (g_conv.id == 2) {
        double amin = INFINITY;
        for (double a : b.amin_at) amin = std::min(amin, a);
        double pc = std::min(std::sqrt(2.0 * integral_cutoff_tblite(acc) / amin), 40.0);
        b.pair_cut2 = pc * pc;
    }
    return b;
}

// ============================================================================ integrals
// Obara-Saika moment tables, Cartesian-to-spherical transform and the multipole blocks:
// crates/axtb/src/integrals.rs:28-127 (tables), 132-179 (spherical), 216-241 (screening),
// 277-367 (S, D, Q), 400-521 (ket derivatives), 991-1006 (shift to the bra).
const int MT = 8;

int ncart(int l) { return (l + 1) * (l + 2) / 2; }
int nsph(int l) { return 2 * l + 1; }

void cart_exp(int l, int out[][3]) {
    int k = 0;
    for (int lx = l; lx >= 0; lx--)
        for (int ly = l - lx; ly >= 0; ly--) {
            out[k][0] = lx;
            out[k][1] = ly;
            out[k][2] = l - lx - ly;
            k++;
        }
}

// T[m][c] for l = 0..2 (nsph x ncart, row-major)
void sph_trafo(int l, double* T) {
    if (l == 0) {
        T[0] = 1.0;
    } else if (l == 1) {
        const double t[9] = {0, 1, 0, 0, 0, 1, 1, 0, 0};
        std::memcpy(T, t, sizeof t);
    } else {
        double s3 = std::sqrt(3.0), s3_4 = s3 * 0.5;
        const double t[30] = {0.0, s3,  0.0, 0.0,   0.0, 0.0,  //
                              0.0, 0.0, 0.0, 0.0,   s3,  0.0,  //
                              -0.5, 0.0, 0.0, -0.5, 0.0, 1.0,  //
                              0.0, 0.0, s3,  0.0,   0.0, 0.0,  //
                              s3_4, 0.0, 0.0, -s3_4, 0.0, 0.0};
        std::memcpy(T, t, sizeof t);
    }
}

void build_1d(int la, int lb, const double rpa[3], const double rpb[3], double oab, double t[3][MT][MT]) {
    double h = 0.5 * oab;
    for (int k = 0; k < 3; k++) {
        auto& tk = t[k];
        tk[0][0] = 1.0;
        if (la >= 1) {
            tk[1][0] = rpa[k];
            for (int i = 1; i < la; i++) tk[i + 1][0] = rpa[k] * tk[i][0] + i * h * tk[i - 1][0];
        }
        if (lb >= 1) {
            tk[0][1] = rpb[k];
            for (int i = 1; i <= la; i++) tk[i][1] = rpb[k] * tk[i][0] + i * h * tk[i - 1][0];
            for (int j = 1; j < lb; j++) {
                tk[0][j + 1] = rpb[k] * tk[0][j] + j * h * tk[0][j - 1];
                for (int i = 1; i <= la; i++)
                    tk[i][j + 1] = rpb[k] * tk[i][j] + h * (i * tk[i - 1][j] + j * tk[i][j - 1]);
            }
        }
    }
}

// cart[(jc + ncj*ic)*N + x] -> out[(jm + nsj*im)*N + x]
void to_spherical(int lj, int li, int N, const double* cart, double* out) {
    int ncj = ncart(lj), nci = ncart(li), nsj = nsph(lj), nsi = nsph(li);
    double Tj[30], Ti[30];
    sph_trafo(lj, Tj);
    sph_trafo(li, Ti);
    vector<double> tmp(nsj * nci * N, 0.0);
    for (int ic = 0; ic < nci; ic++)
        for (int jm = 0; jm < nsj; jm++)
            for (int jc = 0; jc < ncj; jc++) {
                double t = Tj[jm * ncj + jc];
                if (t == 0.0) continue;
                for (int x = 0; x < N; x++) tmp[(jm + nsj * ic) * N + x] += t * cart[(jc + ncj * ic) * N + x];
            }
    for (int i = 0; i < nsj * nsi * N; i++) out[i] = 0.0;
    for (int im = 0; im < nsi; im++)
        for (int jm = 0; jm < nsj; jm++)
            for (int ic = 0; ic < nci; ic++) {
                double t = Ti[im * nci + ic];
                if (t == 0.0) continue;
                for (int x = 0; x < N; x++) out[(jm + nsj * im) * N + x] += t * tmp[(jm + nsj * ic) * N + x];
            }
}

bool pair_screened(double a, double b, double r2, double intcut) { return a * b * r2 / (a + b) > intcut * (1.0 + 1e-10); }

bool prefactor(double ai, double aj, double r2, double intcut, double& oab, double& pre) {
    double eab = ai + aj;
    oab = 1.0 / eab;
    double est = ai * aj * r2 * oab;
    if (est > intcut) return false;
    double sp = std::sqrt(PI);
    double sqrtpi3 = sp * sp * sp;
    double so = std::sqrt(oab);
    pre = std::exp(-est) * sqrtpi3 * (so * so * so);
    return true;
}

void traceless(double* q) {
    double tr = 0.5 * (q[0] + q[2] + q[5]);
    q[0] = 1.5 * q[0] - tr;
    q[1] *= 1.5;
    q[2] = 1.5 * q[2] - tr;
    q[3] *= 1.5;
    q[4] *= 1.5;
    q[5] = 1.5 * q[5] - tr;
}

// S, D, Q blocks of (bra cj on R_j, ket ci on R_i), vec = R_i - R_j; moments about R_i.
// block index jm + nsph(lj)*im; d[blk*3+k], q[blk*6+k]
void multipole(const Shell& cj, const Shell& ci, const double vec[3], double intcut, double* s, double* d, double* q) {
    double r2 = vec[0] * vec[0] + vec[1] * vec[1] + vec[2] * vec[2];
    int li = ci.l, lj = cj.l;
    int ei[6][3], ej[6][3];
    cart_exp(li, ei);
    cart_exp(lj, ej);
    int ncj = ncart(lj), nci = ncart(li);
    double cart[36 * 10];
    std::memset(cart, 0, sizeof cart);
    double t[3][MT][MT];
    for (int ip = 0; ip < ci.np; ip++)
        for (int jp = 0; jp < cj.np; jp++) {
            double ai = ci.a[ip], aj = cj.a[jp], oab, pre;
            if (!prefactor(ai, aj, r2, intcut, oab, pre)) continue;
            double rpi[3] = {-vec[0] * aj * oab, -vec[1] * aj * oab, -vec[2] * aj * oab};
            double rpj[3] = {vec[0] * ai * oab, vec[1] * ai * oab, vec[2] * ai * oab};
            build_1d(li + 2, lj, rpi, rpj, oab, t);
            double cc = ci.c[ip] * cj.c[jp] * pre;
            for (int ic = 0; ic < nci; ic++)
                for (int jc = 0; jc < ncj; jc++) {
                    const int* a = ei[ic];
                    const int* b = ej[jc];
                    double v[3][3];
                    for (int k = 0; k < 3; k++)
                        for (int m = 0; m < 3; m++) v[k][m] = t[k][a[k] + m][b[k]];
                    double* c = &cart[(jc + ncj * ic) * 10];
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
    double sph[25 * 10];
    to_spherical(lj, li, 10, cart, sph);
    int nb = nsph(lj) * nsph(li);
    for (int k = 0; k < nb; k++) {
        const double* c = &sph[k * 10];
        s[k] = c[0];
        for (int x = 0; x < 3; x++) d[k * 3 + x] = c[1 + x];
        double qq[6] = {c[4], c[5], c[6], c[7], c[8], c[9]};
        traceless(qq);
        for (int x = 0; x < 6; x++) q[k * 6 + x] = qq[x];
    }
}

// moments about R_i -> about R_j = R_i - vec (crates/axtb/src/integrals.rs:991-1006)
void shift_to_bra(const double vec[3], double s, const double* di, const double* qi, double* dj, double* qj) {
    for (int k = 0; k < 3; k++) dj[k] = di[k] + vec[k] * s;
    qj[0] = 2.0 * vec[0] * di[0] + vec[0] * vec[0] * s;
    qj[1] = vec[0] * di[1] + vec[1] * di[0] + vec[0] * vec[1] * s;
    qj[2] = 2.0 * vec[1] * di[1] + vec[1] * vec[1] * s;
    qj[3] = vec[0] * di[2] + vec[2] * di[0] + vec[0] * vec[2] * s;
    qj[4] = vec[1] * di[2] + vec[2] * di[1] + vec[1] * vec[2] * s;
    qj[5] = 2.0 * vec[2] * di[2] + vec[2] * vec[2] * s;
    traceless(qj);
    for (int k = 0; k < 6; k++) qj[k] += qi[k];
}

struct MGrad {
    double s[25], ds[25][3], ddi[25][3][3], ddj[25][3][3], dqi[25][3][6], dqj[25][3][6];
};

// ket-centre derivatives of S, D, Q (crates/axtb/src/integrals.rs:400-521)
void multipole_grad(const Shell& cj, const Shell& ci, const double vec[3], double intcut, MGrad& out) {
    double r2 = vec[0] * vec[0] + vec[1] * vec[1] + vec[2] * vec[2];
    int li = ci.l, lj = cj.l;
    int ei[6][3], ej[6][3];
    cart_exp(li, ei);
    cart_exp(lj, ej);
    int ncj = ncart(lj), nci = ncart(li);
    const int NV = 10;
    static const int MOM[10][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0},
                                   {1, 1, 0}, {0, 2, 0}, {1, 0, 1}, {0, 1, 1}, {0, 0, 2}};
    double val[36 * NV], der[36 * 3 * NV];
    std::memset(val, 0, sizeof val);
    std::memset(der, 0, sizeof der);
    double t[3][MT][MT];
    for (int ip = 0; ip < ci.np; ip++) {
        double ai2 = 2.0 * ci.a[ip];
        for (int jp = 0; jp < cj.np; jp++) {
            double ai = ci.a[ip], aj = cj.a[jp], oab, pre;
            if (!prefactor(ai, aj, r2, intcut, oab, pre)) continue;
            double rpi[3] = {-vec[0] * aj * oab, -vec[1] * aj * oab, -vec[2] * aj * oab};
            double rpj[3] = {vec[0] * ai * oab, vec[1] * ai * oab, vec[2] * ai * oab};
            build_1d(li + 1, lj + 2, rpi, rpj, oab, t);
            double cc = ci.c[ip] * cj.c[jp] * pre;
            for (int ic = 0; ic < nci; ic++)
                for (int jc = 0; jc < ncj; jc++) {
                    const int* a = ei[ic];
                    const int* b = ej[jc];
                    double v[3][3], g[3][3];
                    for (int k = 0; k < 3; k++)
                        for (int m = 0; m < 3; m++) {
                            v[k][m] = t[k][a[k]][b[k] + m];
                            g[k][m] = ai2 * t[k][a[k] + 1][b[k] + m];
                            if (a[k] > 0) g[k][m] -= a[k] * t[k][a[k] - 1][b[k] + m];
                        }
                    double* vc = &val[(jc + ncj * ic) * NV];
                    double* dc = &der[(jc + ncj * ic) * 3 * NV];
                    for (int n = 0; n < NV; n++) {
                        const int* mm = MOM[n];
                        double x = v[0][mm[0]], y = v[1][mm[1]], z = v[2][mm[2]];
                        vc[n] += cc * x * y * z;
                        dc[3 * n] += cc * g[0][mm[0]] * y * z;
                        dc[3 * n + 1] += cc * x * g[1][mm[1]] * z;
                        dc[3 * n + 2] += cc * x * y * g[2][mm[2]];
                    }
                }
        }
    }
    double sval[25 * NV], sder[25 * 3 * NV];
    to_spherical(lj, li, NV, val, sval);
    to_spherical(lj, li, 3 * NV, der, sder);
    static const int AB[6][2] = {{0, 0}, {0, 1}, {1, 1}, {0, 2}, {1, 2}, {2, 2}};
    int nb = nsph(lj) * nsph(li);
    for (int blk = 0; blk < nb; blk++) {
        const double* v = &sval[blk * NV];
        const double* dv = &sder[blk * 3 * NV];
        double s = v[0];
        double dj[3] = {v[1], v[2], v[3]};
        double ds[3] = {dv[0], dv[1], dv[2]};
        out.s[blk] = s;
        for (int k = 0; k < 3; k++) out.ds[blk][k] = ds[k];
        double ddj[3][3], dmj[3][6], ddi[3][3], dmi[3][6];
        for (int k = 0; k < 3; k++) {
            for (int c = 0; c < 3; c++) ddj[k][c] = dv[3 * (1 + c) + k];
            for (int c = 0; c < 6; c++) dmj[k][c] = dv[3 * (4 + c) + k];
        }
        for (int k = 0; k < 3; k++) {
            for (int c = 0; c < 3; c++) ddi[k][c] = ddj[k][c] - vec[c] * ds[k];
            ddi[k][k] -= s;
            for (int n = 0; n < 6; n++) {
                int a = AB[n][0], b = AB[n][1];
                double x = dmj[k][n] - vec[a] * ddj[k][b] - vec[b] * ddj[k][a] + vec[a] * vec[b] * ds[k];
                if (a == k) x += -dj[b] + vec[b] * s;
                if (b == k) x += -dj[a] + vec[a] * s;
                dmi[k][n] = x;
            }
        }
        for (int k = 0; k < 3; k++) {
            traceless(dmi[k]);
            traceless(dmj[k]);
        }
        std::memcpy(out.ddi[blk], ddi, sizeof ddi);
        std::memcpy(out.ddj[blk], ddj, sizeof ddj);
        std::memcpy(out.dqi[blk], dmi, sizeof dmi);
        std::memcpy(out.dqj[blk], dmj, sizeof dmj);
    }
}

// ============================================================================ model setup
struct Model {
    Mol m;
    Basis b;
    // H0 (crates/axtb/src/gfn2.rs:58-90)
    vector<double> selfenergy, kcn, shpoly, refocc;  // per shell
    vector<double> rad;                               // per atom
    vector<double> cn_rcov;                           // per atom (GFN2 CN radii)
    // hscale for shell pairs: function
    vector<double> hardness, gam3;  // per shell
    // AES (crates/axtb/src/gfn2.rs:102-113, coulomb.rs:357-360)
    vector<double> dkernel, qkernel, aes_rad, aes_vcn;  // per atom
    // repulsion (crates/axtb/src/gfn2.rs:114-116)
    vector<double> rep_alpha, rep_zeff;
};

double kshell(int k, int l) {
    static const double KDIAG[5] = {1.85, 2.23, 2.23, 2.23, 2.23};
    if ((k == 2 && (l == 0 || l == 1)) || (l == 2 && (k == 0 || k == 1))) return 2.0;
    return (KDIAG[l] + KDIAG[k]) / 2.0;
}

// hscale[jsp][isp][jsh][ish] of crates/axtb/src/gfn2.rs:73-89 for bra shell (zj, jsh), ket (zi, ish)
double hscale(int zj, int jsh, int zi, int ish) {
    double den = sq(conv_en(zj) - conv_en(zi));
    int jl = ANG_SHELL[zj - 1][jsh], il = ANG_SHELL[zi - 1][ish];
    double za = SLATER_EXPONENT[zj - 1][jsh], zb = SLATER_EXPONENT[zi - 1][ish];
    double zij = std::pow(2.0 * std::sqrt(za * zb) / (za + zb), 0.5);
    double enp = 1.0 + 2.0e-2 * den;
    double km = kshell(il, jl) * enp;
    return zij * km;
}

Model build_model(const Mol& m, double acc) {
    Model md;
    md.m = m;
    md.b = build_basis(m, acc);
    const Basis& b = md.b;
    static const double SHELL_HUBBARD_DERIVS[5] = {1.0, 0.5, 0.25, 0.25, 0.25};
    for (int s = 0; s < b.nsh; s++) {
        int iat = b.sh2at[s], z = m.Z[iat], ish = s - b.ish_at[iat], l = ANG_SHELL[z - 1][ish];
        md.selfenergy.push_back(P_SELFENERGY[z - 1][ish]);
        md.kcn.push_back(P_KCN[z - 1][l]);
        md.shpoly.push_back(P_SHPOLY[z - 1][l]);
        md.refocc.push_back(REFERENCE_OCC[z - 1][l]);
        md.hardness.push_back(HUBBARD_PARAMETER[z - 1] * SHELL_HUBBARD[z - 1][l]);
        md.gam3.push_back(P_HUBBARD_DERIVS[z - 1] * SHELL_HUBBARD_DERIVS[l]);
    }
    for (int i = 0; i < m.nat; i++) {
        int z = m.Z[i];
        md.rad.push_back(conv_atomic_rad(z));
        md.cn_rcov.push_back(conv_cn_rcov(z));
        md.dkernel.push_back(P_DKERNEL[z - 1]);
        md.qkernel.push_back(P_QKERNEL[z - 1]);
        md.aes_rad.push_back(P_RAD[z - 1]);
        md.aes_vcn.push_back(P_VCN[z - 1]);
        md.rep_alpha.push_back(REP_ALPHA[z - 1]);
        md.rep_zeff.push_back(REP_ZEFF[z - 1]);
    }
    return md;
}

// ============================================================================ GFN2 CN
// double-exponential count, crates/base/src/ncoord.rs:59-121, model axtb/src/ncoord.rs:28-33
double exp_count(double k, double r, double r0) { return 1.0 / (1.0 + std::exp(-k * (r0 / r - 1.0))); }
double exp_dcount(double k, double r, double r0) {
    double e = std::exp(-k * (r0 / r - 1.0));
    return (-k * r0 * e) / (std::pow(r, 2.0) * std::pow(e + 1.0, 2.0));
}
double dexp_count(double r, double rc) { return exp_count(10.0, r, rc) * exp_count(20.0, r, rc + 2.0); }
double dexp_dcount(double r, double rc) {
    return exp_dcount(10.0, r, rc) * exp_count(20.0, r, rc + 2.0) + exp_count(10.0, r, rc) * exp_dcount(20.0, r, rc + 2.0);
}

#define CN_CUTOFF (g_conv.cn_cut)  // conventions.rs:251, 285, 339

vector<double> gfn2_cn(const Model& md) {
    const Mol& m = md.m;
    vector<double> cn(m.nat, 0.0);
    for (int i = 0; i < m.nat; i++)
        for (int j = 0; j < i; j++) {
            double v[3] = {m.R(i)[0] - m.R(j)[0], m.R(i)[1] - m.R(j)[1], m.R(i)[2] - m.R(j)[2]};
            double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            if (r2 > CN_CUTOFF * CN_CUTOFF || r2 < 1e-12) continue;
            double c = dexp_count(std::sqrt(r2), md.cn_rcov[i] + md.cn_rcov[j]);
            cn[i] += c;
            cn[j] += c;
        }
    return cn;
}

// chain rule sum_A dE/dCN_A dCN_A/dR (crates/base/src/ncoord.rs:486-519, Scaled order)
void gfn2_cn_grad(const Model& md, const vector<double>& dedcn, vector<double>& g) {
    const Mol& m = md.m;
    for (int i = 0; i < m.nat; i++)
        for (int j = 0; j < i; j++) {
            double s = dedcn[i] + dedcn[j];
            double v[3] = {m.R(i)[0] - m.R(j)[0], m.R(i)[1] - m.R(j)[1], m.R(i)[2] - m.R(j)[2]};
            double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            if (r2 > CN_CUTOFF * CN_CUTOFF || r2 < 1e-12) continue;
            double r = std::sqrt(r2);
            double d = dexp_dcount(r, md.cn_rcov[i] + md.cn_rcov[j]);
            double t = d * s / r;
            for (int k = 0; k < 3; k++) {
                g[3 * i + k] += t * v[k];
                g[3 * j + k] -= t * v[k];
            }
        }
}

// ============================================================================ AO matrices
struct Ints {
    int n = 0;
    vector<double> S, H0, D[3], Q[6];
};

// crates/axtb/src/hamiltonian.rs:42-54 (self energies) and 77-94 (H0), ao.rs:195-291
Ints build_ints(const Model& md, const vector<double>& se) {
    const Mol& m = md.m;
    const Basis& b = md.b;
    int n = b.nao;
    Ints I;
    I.n = n;
    I.S.assign((size_t)n * n, 0.0);
    I.H0.assign((size_t)n * n, 0.0);
    for (int k = 0; k < 3; k++) I.D[k].assign((size_t)n * n, 0.0);
    for (int k = 0; k < 6; k++) I.Q[k].assign((size_t)n * n, 0.0);
    auto at = [n](vector<double>& M, int r, int c) -> double& { return M[(size_t)r + (size_t)c * n]; };
    double s[25], d[75], q[150];
    for (int iat = 0; iat < m.nat; iat++) {
        for (int jat = 0; jat <= iat; jat++) {
            double vec[3] = {m.R(iat)[0] - m.R(jat)[0], m.R(iat)[1] - m.R(jat)[1], m.R(iat)[2] - m.R(jat)[2]};
            double r2 = vec[0] * vec[0] + vec[1] * vec[1] + vec[2] * vec[2];
            bool onsite = iat == jat;
            if (!onsite && (r2 > b.pair_cut2 || pair_screened(b.amin_at[iat], b.amin_at[jat], r2, b.intcut))) continue;
            double rr = onsite ? 0.0 : std::sqrt(std::sqrt(r2) / (md.rad[jat] + md.rad[iat]));
            for (int ish = 0; ish < b.nsh_at[iat]; ish++) {
                int si = b.ish_at[iat] + ish;
                const Shell& ci = b.sh[si];
                for (int jsh = 0; jsh < b.nsh_at[jat]; jsh++) {
                    int sj = b.ish_at[jat] + jsh;
                    const Shell& cj = b.sh[sj];
                    if (!onsite && pair_screened(ci.amin, cj.amin, r2, b.intcut)) continue;
                    multipole(cj, ci, vec, b.intcut, s, d, q);
                    double hij;
                    if (onsite) {
                        hij = 0.5 * (se[si] + se[sj]);
                    } else {
                        double shp = (1.0 + md.shpoly[si] * rr) * (1.0 + md.shpoly[sj] * rr);
                        hij = 0.5 * (se[si] + se[sj]) * hscale(m.Z[jat], jsh, m.Z[iat], ish) * shp;
                    }
                    int nj = nsph(cj.l);
                    for (int im = 0; im < nsph(ci.l); im++)
                        for (int jm = 0; jm < nj; jm++) {
                            int ij = jm + nj * im;
                            int mu = b.iao_sh[sj] + jm, nu = b.iao_sh[si] + im;
                            at(I.S, mu, nu) = s[ij];
                            at(I.H0, mu, nu) = s[ij] * hij;
                            for (int k = 0; k < 3; k++) at(I.D[k], mu, nu) = d[ij * 3 + k];
                            for (int k = 0; k < 6; k++) at(I.Q[k], mu, nu) = q[ij * 6 + k];
                            if (!onsite) {
                                double dj[3], qj[6];
                                shift_to_bra(vec, s[ij], &d[ij * 3], &q[ij * 6], dj, qj);
                                at(I.S, nu, mu) = s[ij];
                                at(I.H0, nu, mu) = s[ij] * hij;
                                for (int k = 0; k < 3; k++) at(I.D[k], nu, mu) = dj[k];
                                for (int k = 0; k < 6; k++) at(I.Q[k], nu, mu) = qj[k];
                            }
                        }
                }
            }
        }
    }
    return I;
}

// ============================================================================ electrostatics
// ES2 gamma (crates/axtb/src/coulomb.rs:61-119), g = 2
vector<double> es2_gamma(const Model& md) {
    const Mol& m = md.m;
    const Basis& b = md.b;
    int nsh = b.nsh;
    vector<double> g((size_t)nsh * nsh);
    for (int iat = 0; iat < m.nat; iat++)
        for (int jat = 0; jat <= iat; jat++) {
            double v[3] = {m.R(jat)[0] - m.R(iat)[0], m.R(jat)[1] - m.R(iat)[1], m.R(jat)[2] - m.R(iat)[2]};
            double r1g = std::pow(std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]), 2.0);
            for (int ish = 0; ish < b.nsh_at[iat]; ish++) {
                int jmax = iat == jat ? ish + 1 : b.nsh_at[jat];
                for (int jsh = 0; jsh < jmax; jsh++) {
                    int a = b.ish_at[iat] + ish, c = b.ish_at[jat] + jsh;
                    double eta = 0.5 * (md.hardness[a] + md.hardness[c]);
                    double val = iat == jat ? eta : 1.0 / std::pow(r1g + std::pow(eta, -2.0), 1.0 / 2.0);
                    g[(size_t)a * nsh + c] = val;
                    g[(size_t)c * nsh + a] = val;
                }
            }
        }
    return g;
}

// ES2 gradient (crates/axtb/src/coulomb.rs:123-169)
void es2_grad(const Model& md, const vector<double>& qsh, vector<double>& g) {
    const Mol& m = md.m;
    const Basis& b = md.b;
    for (int iat = 1; iat < m.nat; iat++)
        for (int jat = 0; jat < iat; jat++) {
            double v[3] = {m.R(iat)[0] - m.R(jat)[0], m.R(iat)[1] - m.R(jat)[1], m.R(iat)[2] - m.R(jat)[2]};
            double r1 = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            double dg = 0.0;
            for (int ish = 0; ish < b.nsh_at[iat]; ish++)
                for (int jsh = 0; jsh < b.nsh_at[jat]; jsh++) {
                    int a = b.ish_at[iat] + ish, c = b.ish_at[jat] + jsh;
                    double eta = 0.5 * (md.hardness[a] + md.hardness[c]);
                    double dtmp = 1.0 / (std::pow(r1, 2.0) + std::pow(eta, -2.0));
                    dtmp = -std::pow(r1, 0.0) * dtmp * std::pow(dtmp, 0.5);
                    dg += dtmp * qsh[a] * qsh[c];
                }
            for (int k = 0; k < 3; k++) {
                g[3 * iat + k] += dg * v[k];
                g[3 * jat + k] -= dg * v[k];
            }
        }
}

// AES (damped multipoles), crates/axtb/src/coulomb.rs:357-397 (cache), 407-502 (potentials),
// 668-731 (energy), 896-1001 (gradient)
const double QSCALE[6] = {1.0, 2.0, 1.0, 2.0, 2.0, 1.0};
struct AesCache {
    vector<double> mrad, dmrdcn, g3, g5;  // g3, g5 packed (i, j < i) at i(i-1)/2 + j
};
inline size_t pidx(int i, int j) { return (size_t)i * (i - 1) / 2 + j; }

AesCache aes_cache(const Model& md, const vector<double>& cn) {
    const Mol& m = md.m;
    AesCache c;
    const double shift = 1.2, kexp = 4.0, rmax = 5.0;
    for (int i = 0; i < m.nat; i++) {
        double arg = cn[i] - md.aes_vcn[i] - shift;
        double t1 = std::exp(-kexp * arg);
        double t2 = (rmax - md.aes_rad[i]) / (1.0 + t1);
        c.mrad.push_back(md.aes_rad[i] + t2);
        c.dmrdcn.push_back(-t2 * kexp * t1 / (1.0 + t1));
    }
    size_t np = (size_t)m.nat * (m.nat > 0 ? m.nat - 1 : 0) / 2;
    c.g3.assign(np, 0.0);
    c.g5.assign(np, 0.0);
    for (int i = 1; i < m.nat; i++)
        for (int j = 0; j < i; j++) {
            double v[3] = {m.R(i)[0] - m.R(j)[0], m.R(i)[1] - m.R(j)[1], m.R(i)[2] - m.R(j)[2]};
            double r1 = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            double g1 = 1.0 / r1, g3 = g1 * g1 * g1, g5 = g3 * g1 * g1;
            double rr = 0.5 * (c.mrad[j] + c.mrad[i]) * g1;
            double f3 = 1.0 / (1.0 + 6.0 * std::pow(rr, 3.0));
            double f5 = 1.0 / (1.0 + 6.0 * std::pow(rr, 4.0));
            c.g3[pidx(i, j)] = g3 * f3;
            c.g5[pidx(i, j)] = g5 * f5;
        }
    return c;
}

void aes_potential(const Model& md, const AesCache& c, const vector<double>& qat, const vector<double>& dp,
                   const vector<double>& qp, vector<double>& vat, vector<double>& vdp, vector<double>& vqp) {
    const Mol& m = md.m;
    for (int a = 0; a < m.nat; a++) {
        double va = 0.0, vd[3] = {0, 0, 0}, vq[6] = {0, 0, 0, 0, 0, 0};
        for (int b = 0; b < m.nat; b++) {
            if (b == a) continue;
            size_t p = pidx(std::max(a, b), std::min(a, b));
            double w[3] = {m.R(a)[0] - m.R(b)[0], m.R(a)[1] - m.R(b)[1], m.R(a)[2] - m.R(b)[2]};
            double g3 = c.g3[p], g5 = c.g5[p];
            double r2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
            double tc[6] = {w[0] * w[0], w[0] * w[1], w[1] * w[1], w[0] * w[2], w[1] * w[2], w[2] * w[2]};
            const double* mb = &dp[3 * b];
            double mbw = mb[0] * w[0] + mb[1] * w[1] + mb[2] * w[2];
            va += mbw * g3;
            for (int k = 0; k < 3; k++) vd[k] -= w[k] * g3 * qat[b];
            for (int k = 0; k < 3; k++) vd[k] += g5 * (r2 * mb[k] - 3.0 * w[k] * mbw);
            double thb = 0.0;
            for (int k = 0; k < 6; k++) {
                double t = QSCALE[k] * tc[k] * g5;
                vq[k] += t * qat[b];
                thb += t * qp[6 * b + k];
            }
            va += thb;
        }
        vat[a] += va;
        for (int k = 0; k < 3; k++) vdp[3 * a + k] += vd[k] + 2.0 * md.dkernel[a] * dp[3 * a + k];
        for (int k = 0; k < 6; k++) vqp[6 * a + k] += vq[k] + 2.0 * md.qkernel[a] * qp[6 * a + k] * QSCALE[k];
    }
}

double aes_energy(const Model& md, const AesCache& c, const vector<double>& qat, const vector<double>& dp,
                  const vector<double>& qp) {
    const Mol& m = md.m;
    double e = 0.0;
    for (int i = 1; i < m.nat; i++)
        for (int j = 0; j < i; j++) {
            size_t p = pidx(i, j);
            double g3 = c.g3[p], g5 = c.g5[p];
            double v[3] = {m.R(i)[0] - m.R(j)[0], m.R(i)[1] - m.R(j)[1], m.R(i)[2] - m.R(j)[2]};
            double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            const double *di = &dp[3 * i], *dj = &dp[3 * j];
            double miv = di[0] * v[0] + di[1] * v[1] + di[2] * v[2];
            double mjv = dj[0] * v[0] + dj[1] * v[1] + dj[2] * v[2];
            double ep = (qat[i] * mjv - qat[j] * miv) * g3;
            ep += g5 * (r2 * (di[0] * dj[0] + di[1] * dj[1] + di[2] * dj[2]) - 3.0 * miv * mjv);
            double tc[6] = {v[0] * v[0], v[0] * v[1], v[1] * v[1], v[0] * v[2], v[1] * v[2], v[2] * v[2]};
            for (int k = 0; k < 6; k++) ep += QSCALE[k] * tc[k] * g5 * (qat[j] * qp[6 * i + k] + qat[i] * qp[6 * j + k]);
            e += ep;
        }
    for (int i = 0; i < m.nat; i++) {
        const double* di = &dp[3 * i];
        e += md.dkernel[i] * (di[0] * di[0] + di[1] * di[1] + di[2] * di[2]);
        double qq = 0.0;
        for (int k = 0; k < 6; k++) qq += QSCALE[k] * qp[6 * i + k] * qp[6 * i + k];
        e += md.qkernel[i] * qq;
    }
    return e;
}

void aes_grad(const Model& md, const AesCache& c, const vector<double>& qat, const vector<double>& dp,
              const vector<double>& qp, vector<double>& g, vector<double>& dedcn) {
    const Mol& m = md.m;
    const double kdmp3 = 3.0, kdmp5 = 4.0;
    vector<double> dedr(m.nat, 0.0);
    for (int iat = 1; iat < m.nat; iat++)
        for (int jat = 0; jat < iat; jat++) {
            double rr = 0.5 * (c.mrad[iat] + c.mrad[jat]);
            double vec[3] = {m.R(jat)[0] - m.R(iat)[0], m.R(jat)[1] - m.R(iat)[1], m.R(jat)[2] - m.R(iat)[2]};
            double r2 = vec[0] * vec[0] + vec[1] * vec[1] + vec[2] * vec[2];
            double r1 = std::sqrt(r2);
            double g1 = 1.0 / r1, g3 = g1 * g1 * g1, g5 = g3 * g1 * g1, g7 = g5 * g1 * g1;
            double fdmp3 = 1.0 / (1.0 + 6.0 * std::pow(rr * g1, kdmp3));
            double ddmp3 = -3.0 * g5 * fdmp3 - kdmp3 * fdmp3 * (fdmp3 - 1.0) * g5;
            double fdmp5 = 1.0 / (1.0 + 6.0 * std::pow(rr * g1, kdmp5));
            double ddmp5 = -5.0 * fdmp5 - kdmp5 * (fdmp5 * fdmp5 - fdmp5);
            double qi = qat[iat], qj = qat[jat];
            const double *di = &dp[3 * iat], *dj = &dp[3 * jat];
            double dpiqj = (vec[0] * di[0] + vec[1] * di[1] + vec[2] * di[2]) * qj;
            double qidpj = (vec[0] * dj[0] + vec[1] * dj[1] + vec[2] * dj[2]) * qi;
            double fddr = 3.0 * (dpiqj - qidpj) * kdmp3 * fdmp3 * g3 * (fdmp3 / rr) * std::pow(rr * g1, kdmp3);
            double dg[3];
            for (int k = 0; k < 3; k++) dg[k] = -ddmp3 * vec[k] * (dpiqj - qidpj) + fdmp3 * g3 * (qi * dj[k] - qj * di[k]);
            double dpidpj = dj[0] * di[0] + dj[1] * di[1] + dj[2] * di[2];
            double dpiv = di[0] * vec[0] + di[1] * vec[1] + di[2] * vec[2];
            double dpjv = dj[0] * vec[0] + dj[1] * vec[1] + dj[2] * vec[2];
            double edd = dpidpj * r2 - 3.0 * dpjv * dpiv;
            fddr += 3.0 * edd * kdmp5 * fdmp5 * g5 * (fdmp5 / rr) * std::pow(rr * g1, kdmp5);
            for (int k = 0; k < 3; k++)
                dg[k] += -2.0 * fdmp5 * g5 * dpidpj * vec[k] + 3.0 * fdmp5 * g5 * (dpiv * dj[k] + dpjv * di[k]) -
                         edd * ddmp5 * g7 * vec[k];
            const double *ti = &qp[6 * iat], *tj = &qp[6 * jat];
            double eq = 2.0 * (qj * ti[1] + tj[1] * qi) * vec[0] * vec[1] + 2.0 * (qj * ti[3] + tj[3] * qi) * vec[0] * vec[2] +
                        2.0 * (qj * ti[4] + tj[4] * qi) * vec[1] * vec[2] + (qj * ti[0] + tj[0] * qi) * vec[0] * vec[0] +
                        (qj * ti[2] + tj[2] * qi) * vec[1] * vec[1] + (qj * ti[5] + tj[5] * qi) * vec[2] * vec[2];
            fddr += eq * 3.0 * kdmp5 * fdmp5 * g5 * fdmp5 / rr * std::pow(rr * g1, kdmp5);
            double tvj[3] = {vec[0] * tj[0] + vec[1] * tj[1] + vec[2] * tj[3], vec[0] * tj[1] + vec[1] * tj[2] + vec[2] * tj[4],
                             vec[0] * tj[3] + vec[1] * tj[4] + vec[2] * tj[5]};
            double tvi[3] = {vec[0] * ti[0] + vec[1] * ti[1] + vec[2] * ti[3], vec[0] * ti[1] + vec[1] * ti[2] + vec[2] * ti[4],
                             vec[0] * ti[3] + vec[1] * ti[4] + vec[2] * ti[5]};
            for (int k = 0; k < 3; k++)
                dg[k] += -eq * ddmp5 * g7 * vec[k] - 2.0 * fdmp5 * g5 * qi * tvj[k] - 2.0 * fdmp5 * g5 * qj * tvi[k];
            dedr[iat] += fddr;
            dedr[jat] += fddr;
            for (int k = 0; k < 3; k++) {
                g[3 * iat + k] += dg[k];
                g[3 * jat + k] -= dg[k];
            }
        }
    for (int i = 0; i < m.nat; i++) dedcn[i] += dedr[i] * c.dmrdcn[i];
}

// ============================================================================ repulsion
// crates/axtb/src/repulsion.rs:19-73; cutoff 40 bohr (conventions.rs:252)
double repulsion(const Model& md, vector<double>* g) {
    const Mol& m = md.m;
    double e = 0.0;
    const double cutoff = g_conv.rep_cut;
    for (int i = 0; i < m.nat; i++)
        for (int j = 0; j < i; j++) {
            double v[3] = {m.R(i)[0] - m.R(j)[0], m.R(i)[1] - m.R(j)[1], m.R(i)[2] - m.R(j)[2]};
            double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            if (r2 > cutoff * cutoff || r2 < 1e-12) continue;
            double r1 = std::sqrt(r2);
            double kexp = (m.Z[i] > 2 || m.Z[j] > 2) ? 1.5 : 1.0;
            double alpha = std::sqrt(md.rep_alpha[j] * md.rep_alpha[i]);
            double r1k = std::pow(r1, kexp);
            double exa = std::exp(-alpha * r1k);
            double r1r = std::pow(r1, 1.0);
            double de = md.rep_zeff[j] * md.rep_zeff[i] * exa / r1r;
            e += de;
            if (g) {
                double f = -(alpha * r1k * kexp + 1.0) * de / r2;
                for (int k = 0; k < 3; k++) {
                    (*g)[3 * i + k] += f * v[k];
                    (*g)[3 * j + k] -= f * v[k];
                }
            }
        }
    return e;
}

// ============================================================================ D4
// model: crates/d4/src/model.rs (zeta 86-105, trapezoid 113-138, ngw 140-151, reference alpha
// 160-195, C6 table 197-217, weights 474-570, pair C6 577-631); dispersion:
// crates/d4/src/disp.rs (two-body 274-334, energy/potential 380-455, gradient 460-484,
// three-body 490-512 / 614-734); CN crates/d4/src/ncoord.rs with axtb's radii and cutoffs
// (conventions.rs:255-258: CN 40, two-body 72 width 1, three-body 40 width 1).
const int MAXREF = 7, NFREQ = 23;
const double D4_GA = 3.0, D4_GC = 2.0, D4_WF = 6.0;
const double S6 = 1.0, S8 = 2.7, S9 = 5.0, A1 = 0.52, A2 = 5.0, ALP = 16.0;
#define D4_CN_CUT (g_conv.d4_cn_cut)
#define D2_CUT (g_conv.d2_cut)
#define D2_W (g_conv.d2_w)
#define D3_CUT (g_conv.d3_cut)
#define D3_W (g_conv.d3_w)

double zeta_f(double a, double c, double qref, double qmod) {
    if (qmod < 0.0) return std::exp(a);
    return std::exp(a * (1.0 - std::exp(c * (1.0 - qref / qmod))));
}
void zeta_df(double a, double c, double qref, double qmod, double& z, double& dz) {
    if (qmod < 0.0) {
        z = std::exp(a);
        dz = 0.0;
        return;
    }
    double e = std::exp(c * (1.0 - qref / qmod));
    z = std::exp(a * (1.0 - e));
    dz = -((a * c * e * z * qref) / (qmod * qmod));
}

const double FREQ[NFREQ] = {0.000001, 0.050000, 0.100000, 0.200000, 0.300000, 0.400000, 0.500000, 0.600000,
                            0.700000, 0.800000, 0.900000, 1.000000, 1.200000, 1.400000, 1.600000, 1.800000,
                            2.000000, 2.500000, 3.000000, 4.000000, 5.000000, 7.500000, 10.00000};

struct D4 {
    int nat = 0, nsp = 0;
    vector<int> id, spZ;
    vector<int> nref;
    vector<std::array<int, MAXREF>> ngw;
    vector<std::array<double, MAXREF>> refcn, refq;
    vector<double> zeff, eta, r4r2, rcov, en;
    vector<double> c6ref;  // [isp*nsp+jsp][7][7]
    vector<double> rr, r0;
    vector<double> cn;
    bool off = false;  // Options::dispersion = false: the term is left out (crates/axtb/src/lib.rs:185-187)
    // two-body pair list (i > j)
    vector<int> pi, pj;
    vector<double> pe, pg;
    double c6(int isp, int jsp, int a, int b) const { return c6ref[((size_t)(isp * nsp + jsp) * MAXREF + a) * MAXREF + b]; }
};

double trapzd(const double* pol) {
    double w[NFREQ];
    w[0] = 0.5 * (FREQ[1] - FREQ[0]);
    for (int k = 1; k < NFREQ - 1; k++) w[k] = 0.5 * ((FREQ[k] - FREQ[k - 1]) + (FREQ[k + 1] - FREQ[k]));
    w[NFREQ - 1] = 0.5 * (FREQ[NFREQ - 1] - FREQ[NFREQ - 2]);
    double s = 0.0;
    for (int k = 0; k < NFREQ; k++) s += pol[k] * w[k];
    return s;
}

double en_factor(double ei, double ej) {
    const double K4 = 4.10451, K5 = 19.08857, K6 = 2.0 * (11.28174 * 11.28174);
    double x = std::fabs(ei - ej) + K5;
    return K4 * std::exp(-((x * x) / K6));
}
double erf_count(double r, double rc) { return 0.5 * (1.0 + std::erf(-((7.5 * (r - rc)) / rc))); }
double erf_dcount(double r, double rc) {
    const double SQRTPI = 1.7724538509055159;
    double e = 7.5 * (r - rc) / rc;
    return -(7.5 * std::exp(-(e * e))) / (SQRTPI * rc);
}

void smooth_cutoff(double r, double cutoff, double width, double& sw, double& dsw) {
    if (width <= 0.0 || cutoff <= 0.0) {
        sw = 1.0;
        dsw = 0.0;
        return;
    }
    double w = std::min(width, cutoff), inner = cutoff - w;
    if (r <= inner) {
        sw = 1.0;
        dsw = 0.0;
    } else if (r >= cutoff) {
        sw = 0.0;
        dsw = 0.0;
    } else {
        double x = (cutoff - r) / w, x2 = x * x;
        sw = (x2 * x) * (10.0 + x * (-15.0 + 6.0 * x));
        double omx = 1.0 - x;
        dsw = -((30.0 * x2 * (omx * omx)) / w);
    }
}

D4 d4_setup(const Mol& m) {
    D4 d;
    d.nat = m.nat;
    d.id = m.id;
    d.spZ = m.species;
    d.nsp = (int)m.species.size();
    for (int isp = 0; isp < d.nsp; isp++) {
        int z = d.spZ[isp];
        if (z > 103) throw Fail(2, "D4: unsupported element");
        int nr = REFN[z - 1];
        d.nref.push_back(nr);
        // reference Gaussian weights count (crates/d4/src/model.rs:140-158)
        int cnc[20] = {0};
        cnc[0] = 1;
        auto icn = [](double x) { long v = std::lround(x); return (int)std::min(19L, std::max(0L, v)); };
        for (int r = 0; r < nr; r++) cnc[icn(REFCN[z - 1][r])] += 1;
        std::array<int, MAXREF> ngw;
        ngw.fill(1);
        for (int r = 0; r < nr; r++) {
            int c = cnc[icn(REFCN[z - 1][r])];
            ngw[r] = c * (c + 1) / 2;
        }
        d.ngw.push_back(ngw);
        std::array<double, MAXREF> rc{}, rq{};
        for (int r = 0; r < nr; r++) {
            rc[r] = REFCOVCN[z - 1][r];
            rq[r] = REFQ_GFN2[z - 1][r];
        }
        d.refcn.push_back(rc);
        d.refq.push_back(rq);
        d.zeff.push_back(EFFECTIVE_NUCLEAR_CHARGE[z - 1]);
        d.eta.push_back(CHEMICAL_HARDNESS[z - 1]);
        d.r4r2.push_back(std::sqrt(0.5 * (R4_OVER_R2[z - 1] * std::sqrt((double)z))));
        d.rcov.push_back(conv_d4_rcov(z));
        d.en.push_back(conv_d4_en(z));
    }
    // reference polarisabilities and C6 table
    vector<double> aiw((size_t)d.nsp * MAXREF * NFREQ, 0.0);
    for (int isp = 0; isp < d.nsp; isp++) {
        int z = d.spZ[isp];
        for (int ir = 0; ir < d.nref[isp]; ir++) {
            int is = REFSYS[z - 1][ir];
            if (is == 0) continue;
            double iz = EFFECTIVE_NUCLEAR_CHARGE[is - 1];
            double gam = CHEMICAL_HARDNESS[is - 1] * D4_GC;
            double zv = zeta_f(D4_GA, gam, iz, REFH_GFN2[z - 1][ir] + iz);
            double asc = ASCALE[z - 1][ir], hc = HCOUNT[z - 1][ir];
            for (int k = 0; k < NFREQ; k++) {
                double a = SSCALE[is - 1] * SECAIW[is - 1][k] * zv;
                double v = asc * (ALPHAIW[z - 1][ir][k] - hc * a);
                aiw[((size_t)isp * MAXREF + ir) * NFREQ + k] = v > 0.0 ? v : 0.0;
            }
        }
    }
    d.c6ref.assign((size_t)d.nsp * d.nsp * MAXREF * MAXREF, 0.0);
    double prod[NFREQ];
    for (int isp = 0; isp < d.nsp; isp++)
        for (int jsp = 0; jsp <= isp; jsp++)
            for (int ir = 0; ir < d.nref[isp]; ir++)
                for (int jr = 0; jr < d.nref[jsp]; jr++) {
                    for (int k = 0; k < NFREQ; k++)
                        prod[k] = aiw[((size_t)isp * MAXREF + ir) * NFREQ + k] * aiw[((size_t)jsp * MAXREF + jr) * NFREQ + k];
                    double c6 = 3.0 / PI * trapzd(prod);
                    d.c6ref[((size_t)(jsp * d.nsp + isp) * MAXREF + jr) * MAXREF + ir] = c6;
                    d.c6ref[((size_t)(isp * d.nsp + jsp) * MAXREF + ir) * MAXREF + jr] = c6;
                }
    d.rr.assign((size_t)d.nsp * d.nsp, 0.0);
    d.r0.assign((size_t)d.nsp * d.nsp, 0.0);
    for (int a = 0; a < d.nsp; a++)
        for (int b = 0; b < d.nsp; b++) {
            double v = 3.0 * d.r4r2[a] * d.r4r2[b];
            d.rr[a * d.nsp + b] = v;
            d.r0[a * d.nsp + b] = A1 * std::sqrt(v) + A2;
        }
    // D4 CN
    d.cn.assign(m.nat, 0.0);
    for (int i = 0; i < m.nat; i++)
        for (int j = 0; j < i; j++) {
            double v[3] = {m.R(i)[0] - m.R(j)[0], m.R(i)[1] - m.R(j)[1], m.R(i)[2] - m.R(j)[2]};
            double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            if (r2 > D4_CN_CUT * D4_CN_CUT || r2 < 1e-12) continue;
            double c = en_factor(d.en[d.id[i]], d.en[d.id[j]]) * erf_count(std::sqrt(r2), d.rcov[d.id[i]] + d.rcov[d.id[j]]);
            d.cn[i] += c;
            d.cn[j] += c;
        }
    // two-body pair list with the damped 1/r^6 + 1/r^8 factors
    for (int i = 0; i < m.nat; i++)
        for (int j = 0; j < i; j++) {
            double v[3] = {m.R(i)[0] - m.R(j)[0], m.R(i)[1] - m.R(j)[1], m.R(i)[2] - m.R(j)[2]};
            double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            if (r2 > D2_CUT * D2_CUT || r2 < DBL_EPSILON) continue;
            double r = std::sqrt(r2), sw, dsw;
            smooth_cutoff(r, D2_CUT, D2_W, sw, dsw);
            if (sw <= 0.0) continue;
            int k = d.id[i] * d.nsp + d.id[j];
            double rrij = d.rr[k], r0ij = d.r0[k];
            double r0_2 = r0ij * r0ij, r0_3 = r0_2 * r0ij;
            double t6 = 1.0 / ((r2 * r2) * r2 + r0_3 * r0_3);
            double r0_4 = r0_2 * r0_2;
            double t8 = 1.0 / ((r2 * r2) * (r2 * r2) + r0_4 * r0_4);
            double d6 = -(6.0 * (r2 * r2) * (t6 * t6));
            double d8 = -(8.0 * ((r2 * r2) * r2) * (t8 * t8));
            double e0 = S6 * t6 + S8 * rrij * t8;
            double g0 = S6 * d6 + S8 * rrij * d8;
            d.pi.push_back(i);
            d.pj.push_back(j);
            d.pe.push_back(sw * e0);
            d.pg.push_back(sw * g0 + dsw * e0 / r);
        }
    return d;
}

// reference weights (crates/d4/src/model.rs:474-570)
void d4_weights(const D4& d, const vector<double>& q, vector<double>& gw, vector<double>* dgwdcn,
                vector<double>* dgwdq) {
    gw.assign((size_t)d.nat * MAXREF, 0.0);
    if (dgwdcn) dgwdcn->assign((size_t)d.nat * MAXREF, 0.0);
    if (dgwdq) dgwdq->assign((size_t)d.nat * MAXREF, 0.0);
    double eps_norm = std::sqrt(DBL_MIN);
    for (int iat = 0; iat < d.nat; iat++) {
        int isp = d.id[iat], nr = d.nref[isp];
        double zi = d.zeff[isp], gi = d.eta[isp] * D4_GC, cni = d.cn[iat];
        const auto& refcn = d.refcn[isp];
        const auto& ngw = d.ngw[isp];
        double norm = 0.0, dnorm = 0.0;
        for (int r = 0; r < nr; r++)
            for (int igw = 1; igw <= ngw[r]; igw++) {
                double wf = igw * D4_WF, dd = cni - refcn[r];
                double g = std::exp(-(wf * (dd * dd)));
                norm += g;
                dnorm += 2.0 * wf * (refcn[r] - cni) * g;
            }
        norm = std::fabs(norm) > eps_norm ? 1.0 / norm : 0.0;
        double maxcn = -INFINITY;
        for (int r = 0; r < nr; r++) maxcn = std::max(maxcn, refcn[r]);
        for (int r = 0; r < nr; r++) {
            double expw = 0.0, expd = 0.0;
            for (int igw = 1; igw <= ngw[r]; igw++) {
                double wf = igw * D4_WF, dd = cni - refcn[r];
                double g = std::exp(-(wf * (dd * dd)));
                expw += g;
                expd += 2.0 * wf * (refcn[r] - cni) * g;
            }
            double gwk = expw * norm;
            if (!std::isfinite(gwk) || norm == 0.0) gwk = std::fabs(maxcn - refcn[r]) < 1e-12 ? 1.0 : 0.0;
            double qref = d.refq[isp][r] + zi, qmod = q[iat] + zi;
            double z, dz;
            zeta_df(D4_GA, gi, qref, qmod, z, dz);
            gw[(size_t)iat * MAXREF + r] = gwk * z;
            if (dgwdq) (*dgwdq)[(size_t)iat * MAXREF + r] = gwk * dz;
            if (dgwdcn) {
                double dgwk = norm * (expd - expw * dnorm * norm);
                if (!std::isfinite(dgwk) || norm == 0.0) dgwk = 0.0;
                (*dgwdcn)[(size_t)iat * MAXREF + r] = dgwk * z;
            }
        }
    }
}

void pair_c6(const D4& d, int i, int j, const vector<double>& gw, const vector<double>* dgw, double& c6, double& di,
             double& dj) {
    int isp = d.id[i], jsp = d.id[j];
    c6 = di = dj = 0.0;
    for (int a = 0; a < d.nref[isp]; a++)
        for (int b = 0; b < d.nref[jsp]; b++) {
            double r = d.c6(isp, jsp, a, b);
            c6 += gw[(size_t)i * MAXREF + a] * gw[(size_t)j * MAXREF + b] * r;
            if (dgw) {
                di += (*dgw)[(size_t)i * MAXREF + a] * gw[(size_t)j * MAXREF + b] * r;
                dj += gw[(size_t)i * MAXREF + a] * (*dgw)[(size_t)j * MAXREF + b] * r;
            }
        }
}

// D4 CN chain rule (crates/d4/src/ncoord.rs:56-70; Jacobian order, zero weights skipped)
void d4_cn_grad(const D4& d, const Mol& m, const vector<double>& dedcn, vector<double>& g) {
    for (int i = 0; i < m.nat; i++)
        for (int j = 0; j < i; j++) {
            double s = dedcn[i] + dedcn[j];
            if (s == 0.0) continue;
            double v[3] = {m.R(i)[0] - m.R(j)[0], m.R(i)[1] - m.R(j)[1], m.R(i)[2] - m.R(j)[2]};
            double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            if (r2 > D4_CN_CUT * D4_CN_CUT || r2 < 1e-12) continue;
            double r = std::sqrt(r2);
            double dc = en_factor(d.en[d.id[i]], d.en[d.id[j]]) * erf_dcount(r, d.rcov[d.id[i]] + d.rcov[d.id[j]]);
            for (int k = 0; k < 3; k++) {
                double t = dc * v[k] / r * s;
                g[3 * i + k] += t;
                g[3 * j + k] -= t;
            }
        }
}

// two-body energy and dE/dq (crates/d4/src/disp.rs:380-455)
double d4_energy(const D4& d, const vector<double>& q, vector<double>* vat) {
    vector<double> gw, dgwdq;
    d4_weights(d, q, gw, nullptr, vat ? &dgwdq : nullptr);
    double e = 0.0;
    for (size_t p = 0; p < d.pi.size(); p++) {
        double c6, di, dj;
        pair_c6(d, d.pi[p], d.pj[p], gw, vat ? &dgwdq : nullptr, c6, di, dj);
        e += -(c6 * d.pe[p]);
        if (vat) {
            (*vat)[d.pi[p]] -= di * d.pe[p];
            (*vat)[d.pj[p]] -= dj * d.pe[p];
        }
    }
    return e;
}

// two-body gradient at fixed charges (crates/d4/src/disp.rs:460-484)
void d4_grad(const D4& d, const Mol& m, const vector<double>& q, vector<double>& g) {
    vector<double> gw, dgwdcn;
    d4_weights(d, q, gw, &dgwdcn, nullptr);
    vector<double> dedcn(d.nat, 0.0);
    for (size_t p = 0; p < d.pi.size(); p++) {
        int i = d.pi[p], j = d.pj[p];
        double c6, dci, dcj;
        pair_c6(d, i, j, gw, &dgwdcn, c6, dci, dcj);
        dedcn[i] -= dci * d.pe[p];
        dedcn[j] -= dcj * d.pe[p];
        for (int k = 0; k < 3; k++) {
            double dg = -c6 * d.pg[p] * (m.R(i)[k] - m.R(j)[k]);
            g[3 * i + k] += dg;
            g[3 * j + k] -= dg;
        }
    }
    d4_cn_grad(d, m, dedcn, g);
}

// Axilrod-Teller-Muto three-body term at q = 0 with rational damping, smooth cutoff and
// the CN chain rule (crates/d4/src/disp.rs:490-512 with the triple kernel 735-913 and the
// pair-sum order 614-734 of the axtb conventions; the sum here runs over triples i > j > k).
double d4_atm(const D4& d, const Mol& m, vector<double>* g) {
    int n = m.nat;
    vector<double> q0(n, 0.0), gw, dgwdcn;
    d4_weights(d, q0, gw, &dgwdcn, nullptr);
    // pair table (dense) of r2, sw, dsw/r, t, c6, dlnc6/dcn
    vector<double> R2((size_t)n * n), SW((size_t)n * n, 0.0), DSWR((size_t)n * n), T((size_t)n * n), C6((size_t)n * n),
        QL((size_t)n * n, 0.0);
    const double alp3 = ALP / 3.0;
    for (int a = 0; a < n; a++)
        for (int b = 0; b < a; b++) {
            double v[3] = {m.R(b)[0] - m.R(a)[0], m.R(b)[1] - m.R(a)[1], m.R(b)[2] - m.R(a)[2]};
            double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            if (r2 > D3_CUT * D3_CUT || r2 < DBL_EPSILON) continue;
            double r = std::sqrt(r2), sw, dsw;
            smooth_cutoff(r, D3_CUT, D3_W, sw, dsw);
            double r0 = d.r0[d.id[b] * d.nsp + d.id[a]];
            double c6, dca, dcb;
            pair_c6(d, a, b, gw, &dgwdcn, c6, dca, dcb);
            double t = std::pow(r0 / r, alp3);
            for (auto [x, y] : {std::pair<int, int>{a, b}, std::pair<int, int>{b, a}}) {
                size_t k = (size_t)x * n + y;
                R2[k] = r2;
                SW[k] = sw;
                DSWR[k] = dsw / r;
                T[k] = t;
                C6[k] = c6;
            }
            QL[(size_t)a * n + b] = c6 != 0.0 ? dca / c6 : 0.0;  // dln C6_ab / dCN_a
            QL[(size_t)b * n + a] = c6 != 0.0 ? dcb / c6 : 0.0;  // dln C6_ab / dCN_b
        }
    double etot = 0.0;
    vector<double> dedcn(n, 0.0);
    for (int i = 0; i < n; i++)
        for (int j = 0; j < i; j++) {
            size_t ij = (size_t)i * n + j;
            if (SW[ij] <= 0.0) continue;
            for (int k = 0; k < j; k++) {
                size_t ik = (size_t)i * n + k, jk = (size_t)j * n + k;
                double sw = SW[ij] * SW[ik] * SW[jk];
                if (sw <= 0.0) continue;
                double c9 = -(S9 * std::sqrt(std::fabs(C6[ij] * C6[ik] * C6[jk])));
                double r2ij = R2[ij], r2ik = R2[ik], r2jk = R2[jk];
                double r1 = std::sqrt(r2ij * r2ik * r2jk);
                double ir3 = 1.0 / (r1 * r1 * r1), ir5 = ir3 / (r1 * r1);
                double rpow = T[ij] * T[ik] * T[jk];
                double fdmp = 1.0 / (1.0 + 6.0 * rpow);
                double ang = 0.375 * (r2ij + r2jk - r2ik) * (r2ij - r2jk + r2ik) * (-r2ij + r2jk + r2ik) * ir5 + ir3;
                double de0 = ang * fdmp * c9;
                etot += -de0 * sw;
                if (!g) continue;
                double dfdmp = -(2.0 * ALP * rpow * (fdmp * fdmp));
                auto dang_of = [&](double a, double b, double c) {  // d ang / d r2_a * (-r2_a)... per dftd4
                    return -((0.375 * (a * a * a + (a * a) * (b + c) + a * (3.0 * (b * b) + 2.0 * b * c + 3.0 * (c * c)) -
                                       5.0 * ((b - c) * (b - c)) * (b + c))) *
                             ir5);
                };
                double swc9 = sw * c9;
                double fij = swc9 * (-(dang_of(r2ij, r2jk, r2ik) * fdmp) + ang * dfdmp) / r2ij - de0 * DSWR[ij] * SW[ik] * SW[jk];
                double fik = swc9 * (-(dang_of(r2ik, r2jk, r2ij) * fdmp) + ang * dfdmp) / r2ik - de0 * DSWR[ik] * SW[ij] * SW[jk];
                double fjk = swc9 * (-(dang_of(r2jk, r2ik, r2ij) * fdmp) + ang * dfdmp) / r2jk - de0 * DSWR[jk] * SW[ij] * SW[ik];
                for (int x = 0; x < 3; x++) {
                    double vij = m.R(j)[x] - m.R(i)[x], vik = m.R(k)[x] - m.R(i)[x], vjk = m.R(k)[x] - m.R(j)[x];
                    (*g)[3 * i + x] -= fij * vij + fik * vik;
                    (*g)[3 * j + x] += fij * vij - fjk * vjk;
                    (*g)[3 * k + x] += fik * vik + fjk * vjk;
                }
                double h = 0.5 * de0 * sw;
                dedcn[i] -= h * (QL[ij] + QL[ik]);
                dedcn[j] -= h * (QL[(size_t)j * n + i] + QL[jk]);
                dedcn[k] -= h * (QL[(size_t)k * n + i] + QL[(size_t)k * n + j]);
            }
        }
    if (g) d4_cn_grad(d, m, dedcn, *g);
    return etot;
}

// ============================================================================ EEQ start
// crates/axtb/src/eeq.rs:43-77 (multicharge CN with log cap 8, 25 bohr; bordered system)
vector<double> eeq_charges(const Mol& m) {
    int n = m.nat;
    for (int z : m.Z)
        if (z > 103) throw Fail(2, "EEQ: unsupported element");
    vector<double> cn(n, 0.0);
    for (int i = 0; i < n; i++)
        for (int j = 0; j < i; j++) {
            double v[3] = {m.R(i)[0] - m.R(j)[0], m.R(i)[1] - m.R(j)[1], m.R(i)[2] - m.R(j)[2]};
            double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            if (r2 > g_conv.eeq_cn_cut * g_conv.eeq_cn_cut || r2 < 1e-12) continue;
            double c = erf_count(std::sqrt(r2), conv_eeq_rcov(m.Z[i]) + conv_eeq_rcov(m.Z[j]));
            cn[i] += c;
            cn[j] += c;
        }
    const double cap = g_conv.eeq_cap;
    if (cap > 0.0)
        for (double& c : cn) c = std::log(1.0 + std::exp(cap)) - std::log(std::exp(cap - c) + 1.0);
    int N = n + 1;
    vector<double> A((size_t)N * N, 0.0), x(N);
    double sqrt2pi = std::sqrt(2.0 / PI);
    for (int i = 0; i < n; i++) {
        int zi = m.Z[i] - 1;
        A[(size_t)i * N + i] = EEQ_ETA[zi] + sqrt2pi / EEQ_RAD[zi];
        for (int j = 0; j < i; j++) {
            int zj = m.Z[j] - 1;
            double v[3] = {m.R(i)[0] - m.R(j)[0], m.R(i)[1] - m.R(j)[1], m.R(i)[2] - m.R(j)[2]};
            double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            double gam = 1.0 / (EEQ_RAD[zi] * EEQ_RAD[zi] + EEQ_RAD[zj] * EEQ_RAD[zj]);
            double val = std::erf(std::sqrt(r2 * gam)) / std::sqrt(r2);
            A[(size_t)i * N + j] = val;
            A[(size_t)j * N + i] = val;
        }
        A[(size_t)i * N + n] = 1.0;
        A[(size_t)n * N + i] = 1.0;
        x[i] = -EEQ_CHI[zi] + EEQ_KCNCHI[zi] / std::sqrt(cn[i] + 1e-14) * cn[i];
    }
    x[n] = m.charge;
    // LU with partial pivoting
    vector<int> piv(N);
    for (int k = 0; k < N; k++) {
        int p = k;
        for (int i = k + 1; i < N; i++)
            if (std::fabs(A[(size_t)i * N + k]) > std::fabs(A[(size_t)p * N + k])) p = i;
        if (A[(size_t)p * N + k] == 0.0) throw Fail(4, "EEQ singular");
        if (p != k) {
            for (int c = 0; c < N; c++) std::swap(A[(size_t)k * N + c], A[(size_t)p * N + c]);
            std::swap(x[k], x[p]);
        }
        for (int i = k + 1; i < N; i++) {
            double f = A[(size_t)i * N + k] / A[(size_t)k * N + k];
            if (f == 0.0) continue;
            for (int c = k; c < N; c++) A[(size_t)i * N + c] -= f * A[(size_t)k * N + c];
            x[i] -= f * x[k];
        }
    }
    for (int k = N - 1; k >= 0; k--) {
        double s = x[k];
        for (int c = k + 1; c < N; c++) s -= A[(size_t)k * N + c] * x[c];
        x[k] = s / A[(size_t)k * N + k];
    }
    x.resize(n);
    for (double v : x)
        if (!std::isfinite(v)) throw Fail(4, "EEQ charges are not finite");
    return x;
}

// ============================================================================ eigensolver
// Symmetric tridiagonalisation with accumulated transformations (EISPACK tred2) and implicit
// QL with Wilkinson shifts (tql2); A is n x n row-major, replaced by the eigenvectors (column k
// of the row-major array = eigenvector k); eigenvalues ascending.
void tred2_tql2(int n, vector<double>& a, vector<double>& d) {
    d.assign(n, 0.0);
    vector<double> e(n, 0.0);
    auto A = [&](int i, int j) -> double& { return a[(size_t)i * n + j]; };
    for (int i = n - 1; i > 0; i--) {
        int l = i - 1;
        double h = 0.0, scale = 0.0;
        if (l > 0) {
            for (int k = 0; k <= l; k++) scale += std::fabs(A(i, k));
            if (scale == 0.0) {
                e[i] = A(i, l);
            } else {
                for (int k = 0; k <= l; k++) {
                    A(i, k) /= scale;
                    h += A(i, k) * A(i, k);
                }
                double f = A(i, l);
                double g = f >= 0.0 ? -std::sqrt(h) : std::sqrt(h);
                e[i] = scale * g;
                h -= f * g;
                A(i, l) = f - g;
                f = 0.0;
                for (int j = 0; j <= l; j++) {
                    A(j, i) = A(i, j) / h;
                    g = 0.0;
                    for (int k = 0; k <= j; k++) g += A(j, k) * A(i, k);
                    for (int k = j + 1; k <= l; k++) g += A(k, j) * A(i, k);
                    e[j] = g / h;
                    f += e[j] * A(i, j);
                }
                double hh = f / (h + h);
                for (int j = 0; j <= l; j++) {
                    f = A(i, j);
                    e[j] = g = e[j] - hh * f;
                    for (int k = 0; k <= j; k++) A(j, k) -= (f * e[k] + g * A(i, k));
                }
            }
        } else {
            e[i] = A(i, l);
        }
        d[i] = h;
    }
    d[0] = 0.0;
    e[0] = 0.0;
    for (int i = 0; i < n; i++) {
        int l = i - 1;
        if (d[i] != 0.0) {
            for (int j = 0; j <= l; j++) {
                double g = 0.0;
                for (int k = 0; k <= l; k++) g += A(i, k) * A(k, j);
                for (int k = 0; k <= l; k++) A(k, j) -= g * A(k, i);
            }
        }
        d[i] = A(i, i);
        A(i, i) = 1.0;
        for (int j = 0; j <= l; j++) A(j, i) = A(i, j) = 0.0;
    }
    for (int i = 1; i < n; i++) e[i - 1] = e[i];
    e[n - 1] = 0.0;
    for (int l = 0; l < n; l++) {
        int iter = 0, m;
        do {
            for (m = l; m < n - 1; m++) {
                double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
                if (std::fabs(e[m]) <= DBL_EPSILON * dd) break;
            }
            if (m != l) {
                if (iter++ == 60) throw Fail(4, "QL iteration did not converge");
                double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
                double r = std::hypot(g, 1.0);
                g = d[m] - d[l] + e[l] / (g + (g >= 0.0 ? std::fabs(r) : -std::fabs(r)));
                double s = 1.0, c = 1.0, p = 0.0;
                int i;
                for (i = m - 1; i >= l; i--) {
                    double f = s * e[i], b = c * e[i];
                    e[i + 1] = (r = std::hypot(f, g));
                    if (r == 0.0) {
                        d[i + 1] -= p;
                        e[m] = 0.0;
                        break;
                    }
                    s = f / r;
                    c = g / r;
                    g = d[i + 1] - p;
                    r = (d[i] - g) * s + 2.0 * c * b;
                    d[i + 1] = g + (p = s * r);
                    g = c * r - b;
                    for (int k = 0; k < n; k++) {
                        f = A(k, i + 1);
                        A(k, i + 1) = s * A(k, i) + c * f;
                        A(k, i) = c * A(k, i) - s * f;
                    }
                }
                if (r == 0.0 && i >= l) continue;
                d[l] -= p;
                e[l] = g;
                e[m] = 0.0;
            }
        } while (m != l);
    }
    // sort ascending
    vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return d[x] < d[y]; });
    vector<double> d2(n), a2((size_t)n * n);
    for (int c = 0; c < n; c++) {
        d2[c] = d[order[c]];
        for (int r = 0; r < n; r++) a2[(size_t)r * n + c] = a[(size_t)r * n + order[c]];
    }
    d.swap(d2);
    a.swap(a2);
}

// optional LAPACK from the image (scipy's OpenBLAS build), for the timed CPU baseline
struct Lapack {
    typedef void (*potrf_t)(const char*, const int*, double*, const int*, int*);
    typedef void (*sygst_t)(const int*, const char*, const int*, double*, const int*, const double*, const int*, int*);
    typedef void (*syevd_t)(const char*, const char*, const int*, double*, const int*, double*, double*, const int*, int*,
                            const int*, int*);
    typedef void (*trsm_t)(const char*, const char*, const char*, const char*, const int*, const int*, const double*,
                           const double*, const int*, double*, const int*);
    typedef void (*setthreads_t)(int);
    potrf_t potrf = nullptr;
    sygst_t sygst = nullptr;
    syevd_t syevd = nullptr;
    trsm_t trsm = nullptr;
    setthreads_t setthreads = nullptr;
    bool ok = false;
};

const Lapack& lapack() {
    static Lapack L = [] {
        Lapack l;
        const char* env = std::getenv("AXTB_ORACLE_LAPACK");
        if (!env) return l;
        void* h = dlopen(env, RTLD_NOW | RTLD_LOCAL);
        if (!h) return l;
        l.potrf = (Lapack::potrf_t)dlsym(h, "scipy_dpotrf_");
        l.sygst = (Lapack::sygst_t)dlsym(h, "scipy_dsygst_");
        l.syevd = (Lapack::syevd_t)dlsym(h, "scipy_dsyevd_");
        l.trsm = (Lapack::trsm_t)dlsym(h, "scipy_dtrsm_");
        l.setthreads = (Lapack::setthreads_t)dlsym(h, "scipy_openblas_set_num_threads");
        l.ok = l.potrf && l.sygst && l.syevd && l.trsm;
        return l;
    }();
    return L;
}

// F C = S C e with S = L L^T: F' = L^-1 F L^-T, eigenpairs of F', C = L^-T U
// (crates/base/src/linalg/eigen.rs:72-113, 213-296)
struct GenEig {
    int n = 0;
    vector<double> L;  // row-major lower triangle
    bool use_lapack = false;
    vector<double> Lcm;  // column-major factor for LAPACK
    void init(const vector<double>& S, int nn, bool lap) {
        n = nn;
        use_lapack = lap && lapack().ok;
        if (use_lapack) {
            Lcm = S;
            int info = 0;
            char lo = 'L';
            lapack().potrf(&lo, &n, Lcm.data(), &n, &info);
            if (info != 0) throw Fail(4, "overlap matrix is not positive definite");
            return;
        }
        L.assign((size_t)n * n, 0.0);
        for (int j = 0; j < n; j++) {
            double s = S[(size_t)j + (size_t)j * n];
            for (int k = 0; k < j; k++) s -= L[(size_t)j * n + k] * L[(size_t)j * n + k];
            if (!(s > 0.0)) throw Fail(4, "overlap matrix is not positive definite");
            double ljj = std::sqrt(s);
            L[(size_t)j * n + j] = ljj;
            for (int i = j + 1; i < n; i++) {
                double t = S[(size_t)i + (size_t)j * n];
                for (int k = 0; k < j; k++) t -= L[(size_t)i * n + k] * L[(size_t)j * n + k];
                L[(size_t)i * n + j] = t / ljj;
            }
        }
    }
    // F column-major symmetric; eps all n eigenvalues; C column-major n x n (columns eigvecs)
    void solve(const vector<double>& F, vector<double>& eps, vector<double>& C) {
        if (use_lapack) {
            vector<double> A = F;
            int itype = 1, info = 0;
            char lo = 'L', jv = 'V';
            lapack().sygst(&itype, &lo, &n, A.data(), &n, Lcm.data(), &n, &info);
            eps.assign(n, 0.0);
            int lwork = -1, liwork = -1, iw = 0;
            double wq = 0;
            lapack().syevd(&jv, &lo, &n, A.data(), &n, eps.data(), &wq, &lwork, &iw, &liwork, &info);
            lwork = (int)wq;
            liwork = iw;
            vector<double> work(lwork);
            vector<int> iwork(liwork);
            lapack().syevd(&jv, &lo, &n, A.data(), &n, eps.data(), work.data(), &lwork, iwork.data(), &liwork, &info);
            if (info != 0) throw Fail(4, "LAPACK eigensolver failed");
            char side = 'L', tr = 'T', nu = 'N';
            double one = 1.0;
            lapack().trsm(&side, &lo, &tr, &nu, &n, &n, &one, Lcm.data(), &n, A.data(), &n);
            C.swap(A);
            return;
        }
        // X = L^-1 F (column by column), F' = L^-1 X^T (symmetric)
        vector<double> X((size_t)n * n), Fp((size_t)n * n);
        for (int c = 0; c < n; c++)
            for (int i = 0; i < n; i++) {
                double t = F[(size_t)i + (size_t)c * n];
                for (int k = 0; k < i; k++) t -= L[(size_t)i * n + k] * X[(size_t)k * n + c];
                X[(size_t)i * n + c] = t / L[(size_t)i * n + i];
            }
        // Fp = L^-1 X^T: row-major Fp[i][c] = (L^-1 (X^T)[:,c])_i, (X^T)[k][c] = X[c][k]
        for (int c = 0; c < n; c++)
            for (int i = 0; i < n; i++) {
                double t = X[(size_t)c * n + i];
                for (int k = 0; k < i; k++) t -= L[(size_t)i * n + k] * Fp[(size_t)k * n + c];
                Fp[(size_t)i * n + c] = t / L[(size_t)i * n + i];
            }
        for (int i = 0; i < n; i++)
            for (int j = 0; j < i; j++) {
                double v = 0.5 * (Fp[(size_t)i * n + j] + Fp[(size_t)j * n + i]);
                Fp[(size_t)i * n + j] = Fp[(size_t)j * n + i] = v;
            }
        tred2_tql2(n, Fp, eps);  // Fp row-major: column k = eigenvector k
        // C = L^-T U: back substitution per column
        C.assign((size_t)n * n, 0.0);
        for (int c = 0; c < n; c++)
            for (int i = n - 1; i >= 0; i--) {
                double t = Fp[(size_t)i * n + c];
                for (int k = i + 1; k < n; k++) t -= L[(size_t)k * n + i] * C[(size_t)k + (size_t)c * n];
                C[(size_t)i + (size_t)c * n] = t / L[(size_t)i * n + i];
            }
    }
};

// ============================================================================ occupations
// crates/base/src/occupations.rs:58-128 (aufbau, fermi, tblite filling), 179 (entropy)
int aufbau(double nel, vector<double>& occ) {
    int n = (int)occ.size();
    int full = (int)std::floor(nel);
    for (int i = 0; i < n; i++) occ[i] = i < full ? 1.0 : 0.0;
    double rem = std::fmod(nel, 1.0);
    if (full < n) occ[full] = rem;
    return full + (rem > 0.5 ? 1 : 0);
}

bool fill_tblite(double nel, double kt, const vector<double>& emo, vector<double>& occ, double& ef_used) {
    int homo = aufbau(nel, occ);
    if (!(nel > 0.0 && kt > 0.0)) return false;
    int nao = (int)emo.size();
    double sqrttiny = std::sqrt(DBL_MIN);
    int i0 = std::max(homo, 1) - 1;
    int i1 = std::min(homo + 1, nao) - 1;
    double ef = 0.5 * (emo[i0] + emo[i1]);
    ef_used = ef;
    const double tol = 1e5 * DBL_EPSILON;
    for (int it = 0; it < 200; it++) {
        double total = 0.0, dtotal = 0.0;
        ef_used = ef;
        for (int i = 0; i < nao; i++) {
            double arg = (emo[i] - ef) / kt, f, df;
            if (arg > 50.0) {
                f = 0.0;
                df = 0.0;
            } else if (arg < -50.0) {
                f = 1.0;
                df = 0.0;
            } else {
                f = 1.0 / (std::exp(arg) + 1.0);
                df = -f * (1.0 - f) / kt;
            }
            occ[i] = f;
            total += f;
            dtotal -= df;
        }
        if (std::fabs(nel - total) <= tol) break;
        if (dtotal > sqrttiny) ef += (nel - total) / dtotal;
        else break;
    }
    return true;
}

double entropy_tblite(const vector<double>& occ, double kt) {
    double s = 0.0;
    for (double o : occ) s += std::log(std::pow(o, o) * std::pow(1.0 - o, 1.0 - o));
    return s * kt;
}

// ============================================================================ solvation
// Implicit solvation (ALPB, GBSA) of crates/solvation/src as a charge-dependent SCF term
// (crates/axtb/src/solvation.rs:40-110): setup lib.rs:389-497, geometry lib.rs:553-627 (Born
// radii born.rs:103-157, surface sasa.rs:31-240, kernel kernel.rs:28-66, shape kernel.rs:163-196),
// energy and potential lib.rs:636-690, gradient lib.rs:692-712 (kernel.rs:70-160, born.rs:160-216,
// kernel.rs:198-238). axtb's and tblite's conventions use its corrected variant (CODATA 2022
// radii and constants), the xtb 6.8.0 conventions xtb's (mctc-lib's bohr factor and xtb's
// constants in the free-energy shift); both recompute r1 for every pair of the Born integral.
const double HARTREE_TO_KCAL_PER_MOL = 4.3597447222060e-18 * 6.02214076e23 / 4184.0;  // units.rs:37
const double IDEAL_GAS_MOL_VOLUME_EXACT = 6.02214076e23 * 1.380649e-23 * 298.15 / 1.0e5 * 1.0e3;  // lib.rs:128
const double XTB680_AATOAU = 1.0 / 5.29177210904492434e-1;  // units.rs:88

struct Solv {
    int nat = 0;
    bool alpb = false, lhb = false;
    double keps = 0, alpbet = 0, c1 = 0, gshift = 0, lrcut = 0, srcut = 0, w = 0, ah0 = 0, ah1 = 0, ah3 = 0;
    vector<double> vdwr, rho, svdw, vdwsa, t1, t2, wrp, gamsasa, hbmag;
    // geometry
    vector<double> brad, dbrad, sasa, hbw, dhbdw, B, dsdr;
    double adet = 0.0;
    vector<vector<int>> nb;                       // SASA neighbours of each atom, ascending
    vector<vector<std::array<double, 3>>> nbg;   // d sasa_i / d R_j per neighbour
    vector<std::array<double, 3>> selfg;          // d sasa_i / d R_i
};

// free-energy shift of a reference state (lib.rs:277-306): 0 gsolv, 1 bar1M, 2 reference
double solv_state_shift(int state, double temp, double density, double mass, double kb, double vm) {
    using namespace solvtab;
    if (state == 0) return 0.0;
    double s = std::log(vm * temp / AMBIENT_TEMPERATURE);
    if (state == 2) s += std::log(density / REF_DENSITY * REF_MOLECULAR_MASS / mass);
    return temp * kb * s;
}

// the parameter set of a solvent name (lib.rs:255-272: lower case, xtb's aliases, the model's table)
const solvtab::SolventParam* solv_lookup(const char* name, bool alpb) {
    using namespace solvtab;
    std::string s(name ? name : "");
    size_t a = s.find_first_not_of(" \t\n"), b = s.find_last_not_of(" \t\n");
    s = a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
    for (char& c : s) c = (char)std::tolower((unsigned char)c);
    for (const auto& al : ALIASES)
        if (s == al.alias) {
            s = al.name;
            break;
        }
    if (alpb) {
        for (const auto& t : ALPB_SOLVENTS)
            if (s == t.name) return &PARAMS[t.param];
    } else {
        for (const auto& t : GBSA_SOLVENTS)
            if (s == t.name) return &PARAMS[t.param];
    }
    return nullptr;
}

Solv solv_setup(const Mol& m, int model, const char* solvent, int state) {
    using namespace solvtab;
    Solv sv;
    sv.nat = m.nat;
    sv.alpb = model == 0;
    for (int z : m.Z)
        if (z > NELEM) throw Fail(1, "solvation: unsupported element");
    const SolventParam* p = solv_lookup(solvent, sv.alpb);
    if (!p) throw Fail(1, "solvation: unknown solvent");
    bool xtb = g_conv.id == 1;
    double aatoau = xtb ? XTB680_AATOAU : AATOAU;
    const double temp = DEFAULT_TEMPERATURE;
    sv.gshift = xtb ? p->gshift * (1.0 / AUTOKCAL) + solv_state_shift(state, temp, p->rhos, p->smass, KB, IDEAL_GAS_MOL_VOLUME)
                    : p->gshift / HARTREE_TO_KCAL_PER_MOL +
                          solv_state_shift(state, temp, p->rhos, p->smass, KB_HARTREE, IDEAL_GAS_MOL_VOLUME_EXACT);
    double eps = p->epsv;
    sv.c1 = p->c1;
    double offset = p->soset * 0.1 * aatoau, probe = p->rprobe * aatoau;
    bool any_hb = false;
    for (double t : p->tmp) any_hb = any_hb || std::fabs(t) > 1.0e-3;
    sv.alpbet = sv.alpb ? ALPB_ALPHA / eps : 0.0;
    sv.keps = (1.0 / eps - 1.0) / (1.0 + sv.alpbet);
    sv.lrcut = LRCUT_AA * aatoau;
    double w = SMOOTH_W_AA * aatoau, w3 = w * (w * w);
    sv.w = w;
    sv.ah0 = 0.5;
    sv.ah1 = 3.0 / (4.0 * w);
    sv.ah3 = -1.0 / (4.0 * w3);
    double maxsa = -INFINITY;
    for (int z : m.Z) {
        int iz = z - 1;
        double rvdw = aatoau * VDW_RAD_D3_AA[iz];
        sv.vdwr.push_back(rvdw);
        sv.rho.push_back(rvdw * p->sx[iz]);
        sv.svdw.push_back(rvdw - offset);
        double rsa = rvdw + probe;
        sv.vdwsa.push_back(rsa);
        maxsa = std::max(maxsa, rsa);
        sv.t1.push_back((rsa - w) * (rsa - w));
        sv.t2.push_back((rsa + w) * (rsa + w));
        double r = rsa + w;
        double wr = (0.25 / w + 3.0 * sv.ah3 * (0.2 * r * r - 0.5 * r * rsa + rsa * rsa / 3.0)) * r * r * r;
        r = rsa - w;
        wr -= (0.25 / w + 3.0 * sv.ah3 * (0.2 * r * r - 0.5 * r * rsa + rsa * rsa / 3.0)) * r * r * r;
        sv.wrp.push_back(wr);
        sv.gamsasa.push_back(p->gamscale[iz] * (4.0 * PI) * SURFACE_TENSION);
        sv.hbmag.push_back(any_hb ? -(p->tmp[iz] * p->tmp[iz]) * (1.0 / AUTOKCAL) : 0.0);
        if (sv.hbmag.back() < 0.0) sv.lhb = true;
    }
    sv.srcut = 2.0 * (w + maxsa) + SRCUT_AA * aatoau;
    return sv;
}

// one pair of the Born integral (born.rs:13-96): the contributions to psi_i and psi_j and their
// derivatives over r; r1 = 1/r for every pair
struct PsiC {
    bool on = false;
    double g = 0.0, dg = 0.0;
};
inline PsiC psi_nonoverlap(double r, double rho, double r1) {
    double ap = r + rho, am = r - rho, ab = ap * am, rhab = rho / ab;
    double lnab = 0.5 * std::log(am / ap) * r1;
    return {true, rhab + lnab, -2.0 * rhab / ab + (rhab - lnab) * r1 * r1};
}
inline PsiC psi_overlap(double r, double rho, double rvdw) {
    double r1 = 1.0 / r, r12 = 0.5 * r1, r24 = r12 * r12;
    double ap = r + rho, am = r - rho, rh1 = 1.0 / rvdw, rhr1 = 1.0 / ap, aprh1 = ap * rh1;
    double lnab = std::log(aprh1);
    double g = rh1 - rhr1 + r12 * (0.5 * am * (rhr1 - rh1 * aprh1) - lnab);
    double dg = rhr1 * rhr1 * (1.0 - 0.25 * am * r1 * (1.0 + aprh1 * aprh1)) + rho * r24 * (rhr1 - rh1 * aprh1) +
                r12 * (r1 * lnab - rhr1);
    return {true, g, dg * r1};
}
void psi_pair(double r, double rhoi, double rhoj, double rvi, double rvj, PsiC& ci, PsiC& cj) {
    double r1 = 1.0 / r;
    bool ovij = !(r >= rvi + rhoj), ovji = !(r >= rhoi + rvj);
    ci = PsiC{};
    cj = PsiC{};
    if (!ovij && !ovji) {
        ci = psi_nonoverlap(r, rhoj, r1);
        cj = std::fabs(rhoi - rhoj) < 1.0e-8 ? ci : psi_nonoverlap(r, rhoi, r1);
    } else if (!ovij && ovji) {
        ci = psi_nonoverlap(r, rhoj, r1);
        if (r + rhoi > rvj) cj = psi_overlap(r, rhoi, rvj);
    } else if (ovij && !ovji) {
        if (r + rhoj > rvi) ci = psi_overlap(r, rhoj, rvi);
        cj = psi_nonoverlap(r, rhoi, r1);
    } else {
        if (r + rhoj > rvi) ci = psi_overlap(r, rhoj, rvi);
        if (r + rhoi > rvj) cj = psi_overlap(r, rhoi, rvj);
    }
}

double adet_inertia(const Mol& m, const vector<double>& rad, double in[3][3], double center[3]) {
    const double TOF = 2.0 / 5.0;
    double tot = 0.0;
    center[0] = center[1] = center[2] = 0.0;
    for (int i = 0; i < m.nat; i++) {
        double r3 = rad[i] * rad[i] * rad[i];
        tot += r3;
        for (int k = 0; k < 3; k++) center[k] += m.R(i)[k] * r3;
    }
    for (int k = 0; k < 3; k++) center[k] /= tot;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) in[a][b] = 0.0;
    for (int i = 0; i < m.nat; i++) {
        double r2 = rad[i] * rad[i], r3 = r2 * rad[i];
        double v[3] = {m.R(i)[0] - center[0], m.R(i)[1] - center[1], m.R(i)[2] - center[2]};
        double d2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        double diag = r3 * (d2 + TOF * r2);
        for (int k = 0; k < 3; k++) in[k][k] += diag;
        for (int c = 0; c < 3; c++)
            for (int r = 0; r < 3; r++) in[r][c] -= r3 * v[c] * v[r];
    }
    return tot;
}
double det3(const double a[3][3]) {
    return a[0][0] * a[1][1] * a[2][2] - a[0][0] * a[1][2] * a[2][1] - a[0][1] * a[1][0] * a[2][2] +
           a[0][1] * a[1][2] * a[2][0] + a[0][2] * a[1][0] * a[2][1] - a[0][2] * a[1][1] * a[2][0];
}

void solv_geometry(Solv& sv, const Mol& m) {
    using namespace solvtab;
    int n = m.nat;
    auto dist = [&](int i, int j, double v[3]) {
        for (int k = 0; k < 3; k++) v[k] = m.R(i)[k] - m.R(j)[k];
        return v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    };
    // Born radii (GBOBC-II)
    sv.brad.assign(n, 0.0);
    sv.dbrad.assign(n, 0.0);
    vector<double>& psi = sv.brad;
    double lr2 = sv.lrcut * sv.lrcut;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < i; j++) {
            double v[3], d2 = dist(i, j, v);
            if (!(d2 < lr2)) continue;
            PsiC ci, cj;
            psi_pair(std::sqrt(d2), sv.rho[i], sv.rho[j], sv.vdwr[i], sv.vdwr[j], ci, cj);
            if (ci.on) psi[i] += ci.g;
            if (cj.on) psi[j] += cj.g;
        }
    for (int i = 0; i < n; i++) {
        double br = psi[i], s1 = 1.0 / sv.svdw[i], v1 = 1.0 / sv.vdwr[i], s2 = 0.5 * sv.svdw[i];
        br *= s2;
        double arg2 = br * (OBC_GAMMA * br - OBC_BETA);
        double arg = br * (OBC_ALPHA + arg2);
        arg2 = 2.0 * arg2 + OBC_ALPHA + OBC_GAMMA * br * br;
        double th = std::tanh(arg), ch = std::cosh(arg);
        double out = 1.0 / (s1 - v1 * th) * sv.c1;
        double dpsi = ch * (s1 - v1 * th);
        dpsi = s2 * v1 * arg2 / (dpsi * dpsi) * sv.c1;
        psi[i] = out;
        sv.dbrad[i] = dpsi;
    }
    // surface areas and their derivatives
    sv.nb.assign(n, {});
    double sr2 = sv.srcut * sv.srcut;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < i; j++) {
            double v[3], d2 = dist(i, j, v);
            double rmax = sv.vdwsa[i] + sv.vdwsa[j] + sv.w + 1.0e-6;
            if (d2 < sr2 && d2 < rmax * rmax) {
                sv.nb[i].push_back(j);
                sv.nb[j].push_back(i);
            }
        }
    for (auto& l : sv.nb) std::sort(l.begin(), l.end());
    sv.sasa.assign(n, 0.0);
    sv.selfg.assign(n, {0.0, 0.0, 0.0});
    sv.nbg.assign(n, {});
    for (int i = 0; i < n; i++) {
        const vector<int>& nl = sv.nb[i];
        int nno = (int)nl.size();
        vector<std::array<double, 3>> grads(nno, {0.0, 0.0, 0.0});
        vector<double> tj2(nno);
        vector<int> gi(nno);
        vector<std::array<double, 3>> gs(nno);
        std::array<double, 3> gself = {0.0, 0.0, 0.0};
        double sasai = 0.0, rsa = sv.vdwsa[i];
        for (int ip = 0; ip < 230; ip++) {
            const double* g = LEBEDEV_230[ip];
            double xp[3] = {m.R(i)[0] + rsa * g[0], m.R(i)[1] + rsa * g[1], m.R(i)[2] + rsa * g[2]};
            bool buried = false;
            for (int s = 0; s < nno; s++) {
                int j = nl[s];
                double dx = xp[0] - m.R(j)[0], dy = xp[1] - m.R(j)[1], dz = xp[2] - m.R(j)[2];
                tj2[s] = dx * dx + dy * dy + dz * dz;
                buried = buried || tj2[s] <= sv.t1[j];
            }
            if (buried) continue;
            int nni = 0;
            double sasap = 1.0;
            for (int s = 0; s < nno; s++) {
                int j = nl[s];
                if (!(tj2[s] < sv.t2[j])) continue;
                double tj[3] = {xp[0] - m.R(j)[0], xp[1] - m.R(j)[1], xp[2] - m.R(j)[2]};
                double sq = std::sqrt(tj2[s]), uj = sq - sv.vdwsa[j], ah3uj2 = sv.ah3 * uj * uj;
                double ds = sv.ah1 + 3.0 * ah3uj2;
                double sij = sv.ah0 + (sv.ah1 + ah3uj2) * uj;
                if (1.0 < sij) sij = 1.0;
                if (0.0 > sij) sij = 0.0;
                if (sij < DBL_MIN) {
                    sasap = 0.0;
                    break;
                }
                sasap *= sij;
                ds /= sij * sq;
                gi[nni] = s;
                gs[nni] = {ds * tj[0], ds * tj[1], ds * tj[2]};
                nni++;
            }
            if (sasap > TOLSESP) {
                double wsa = g[3] * sv.wrp[i] * sasap;
                sasai += wsa;
                for (int q = 0; q < nni; q++)
                    for (int k = 0; k < 3; k++) {
                        double d = wsa * gs[q][k];
                        gself[k] += d;
                        grads[gi[q]][k] -= d;
                    }
            }
        }
        sv.sasa[i] = sasai;
        sv.selfg[i] = gself;
        sv.nbg[i] = grads;
    }
    sv.dsdr.assign(3 * n, 0.0);
    for (int i = 0; i < n; i++) {
        double c = sv.gamsasa[i];
        if (c == 0.0) continue;
        for (int k = 0; k < 3; k++) sv.dsdr[3 * i + k] += sv.selfg[i][k] * c;
        for (size_t s = 0; s < sv.nb[i].size(); s++)
            for (int k = 0; k < 3; k++) sv.dsdr[3 * sv.nb[i][s] + k] += sv.nbg[i][s][k] * c;
    }
    sv.hbw.assign(n, 0.0);
    sv.dhbdw.assign(n, 0.0);
    if (sv.lhb)
        for (int i = 0; i < n; i++) {
            double smaxd = 1.0 / (sv.vdwsa[i] * sv.vdwsa[i]);
            sv.hbw[i] = sv.hbmag[i] * (sv.sasa[i] * smaxd);
            sv.dhbdw[i] = sv.hbmag[i] * smaxd;
        }
    sv.adet = 0.0;
    if (sv.alpbet > 0.0) {
        double in[3][3], c[3];
        double tot = adet_inertia(m, sv.vdwr, in, c);
        sv.adet = std::sqrt(std::pow(det3(in), 1.0 / 3.0) / ((2.0 / 5.0) * tot));
    }
    // Born matrix: P16 (ALPB) or Still (GBSA) kernel, H-bond diagonal, ALPB shape term
    sv.B.assign((size_t)n * n, 0.0);
    const double zo16 = ZETA_P16 / 16.0;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < i; j++) {
            double v[3], r = std::sqrt(dist(i, j, v)), val;
            if (sv.alpb) {
                double ab = std::sqrt(sv.brad[i] * sv.brad[j]);
                double arg = ab / (ab + zo16 * r);
                arg *= arg;
                arg *= arg;
                arg *= arg;
                arg *= arg;
                val = sv.keps * (1.0 / (r + ab * arg));
            } else {
                double r2 = r * r, aa = sv.brad[i] * sv.brad[j], dd = 0.25 * r2 / aa;
                val = sv.keps * (1.0 / std::sqrt(r2 + aa * std::exp(-dd)));
            }
            sv.B[(size_t)i * n + j] = sv.B[(size_t)j * n + i] = val;
        }
    for (int i = 0; i < n; i++) sv.B[(size_t)i * n + i] = sv.keps * (1.0 / sv.brad[i]);
    if (sv.lhb)
        for (int i = 0; i < n; i++) sv.B[(size_t)i * n + i] += 2.0 * sv.hbw[i];
    if (sv.alpbet > 0.0) {
        double shift = sv.keps * sv.alpbet / sv.adet;
        for (double& x : sv.B) x += shift;
    }
}

// dot product with four interleaved partial sums (lib.rs:742-758)
double dot4(const double* a, const double* b, int n) {
    double acc[4] = {0, 0, 0, 0};
    int n4 = n / 4 * 4;
    for (int i = 0; i < n4; i += 4)
        for (int k = 0; k < 4; k++) acc[k] += a[i + k] * b[i + k];
    double s = (acc[0] + acc[1]) + (acc[2] + acc[3]);
    for (int i = n4; i < n; i++) s += a[i] * b[i];
    return s;
}

// fixed part: surface term and shift (lib.rs:636-652)
double solv_fixed(const Solv& sv, vector<double>* g) {
    double e = 0.0, shift = sv.gshift / sv.nat;
    for (int i = 0; i < sv.nat; i++) e += sv.sasa[i] * sv.gamsasa[i] + shift;
    if (g)
        for (int k = 0; k < 3 * sv.nat; k++) (*g)[k] += sv.dsdr[k];
    return e;
}
// charge-dependent energy 1/2 q^T B q (lib.rs:654-664) and potential B q (lib.rs:666-675)
double solv_energy(const Solv& sv, const vector<double>& q) {
    double e = 0.0;
    for (int i = 0; i < sv.nat; i++) e += q[i] * (0.5 * dot4(&sv.B[(size_t)i * sv.nat], q.data(), sv.nat));
    return e;
}
void solv_potential(const Solv& sv, const vector<double>& q, vector<double>& vat) {
    for (int i = 0; i < sv.nat; i++) vat[i] += dot4(&sv.B[(size_t)i * sv.nat], q.data(), sv.nat);
}

// explicit gradient of 1/2 q^T B q at fixed charges (lib.rs:692-712)
void solv_gradient(const Solv& sv, const Mol& m, const vector<double>& q, vector<double>& grad) {
    int n = sv.nat;
    vector<double> dedbr(n, 0.0);
    const double zo16 = solvtab::ZETA_P16 / 16.0;
    for (int i = 0; i < n; i++) {
        double gi[3] = {0, 0, 0}, di = 0.0;
        for (int j = 0; j < i; j++) {
            double v[3] = {m.R(i)[0] - m.R(j)[0], m.R(i)[1] - m.R(j)[1], m.R(i)[2] - m.R(j)[2]};
            double r = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]), qq = q[i] * q[j];
            if (sv.alpb) {
                double ab = std::sqrt(sv.brad[i] * sv.brad[j]);
                double a1 = ab / (ab + zo16 * r), a16 = a1 * a1;
                a16 *= a16;
                a16 *= a16;
                a16 *= a16;
                double fgb = r + ab * a16, dfgb = 1.0 / fgb, dfgb2 = dfgb * dfgb;
                double ap = (1.0 - solvtab::ZETA_P16 * a1 * a16) * dfgb2;
                for (int k = 0; k < 3; k++) {
                    double dg = ap * v[k] * sv.keps / r * qq;
                    gi[k] -= dg;
                    grad[3 * j + k] += dg;
                }
                double bp = -0.5 * (r * solvtab::ZETA_P16 / ab * a1 + 1.0) / ab * a16 * dfgb2;
                di += sv.brad[j] * bp * sv.keps * qq;
                dedbr[j] += sv.brad[i] * bp * sv.keps * qq;
            } else {
                double r2 = r * r, aa = sv.brad[i] * sv.brad[j], dd = 0.25 * r2 / aa, expd = std::exp(-dd);
                double fgb2 = r2 + aa * expd, dfgb2 = 1.0 / fgb2, dfgb = std::sqrt(dfgb2);
                double dfgb3 = dfgb2 * dfgb * sv.keps, ap = (1.0 - 0.25 * expd) * dfgb3;
                for (int k = 0; k < 3; k++) {
                    double dr = ap * v[k];
                    gi[k] -= dr * qq;
                    grad[3 * j + k] += dr * qq;
                }
                double bp = -0.5 * expd * (1.0 + dd) * dfgb3;
                di += sv.brad[j] * bp * qq;
                dedbr[j] += sv.brad[i] * bp * qq;
            }
        }
        for (int k = 0; k < 3; k++) grad[3 * i + k] += gi[k];
        dedbr[i] += di;
    }
    for (int i = 0; i < n; i++) {
        double bp = 1.0 / sv.brad[i], qq = q[i] * bp;
        dedbr[i] += -0.5 * sv.keps * qq * bp * q[i];
    }
    // Born radii chain: sum_i (dE/dbrad_i dbrad_i/dpsi_i) dpsi_i/dR
    for (int i = 0; i < n; i++) dedbr[i] *= sv.dbrad[i];
    double lr2 = sv.lrcut * sv.lrcut;
    for (int i = 0; i < n; i++) {
        double gi[3] = {0, 0, 0};
        for (int j = 0; j < i; j++) {
            double v[3] = {m.R(i)[0] - m.R(j)[0], m.R(i)[1] - m.R(j)[1], m.R(i)[2] - m.R(j)[2]};
            double d2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            if (!(d2 < lr2)) continue;
            PsiC ci, cj;
            psi_pair(std::sqrt(d2), sv.rho[i], sv.rho[j], sv.vdwr[i], sv.vdwr[j], ci, cj);
            double s = 0.0;
            if (ci.on) s += dedbr[i] * ci.dg;
            if (cj.on) s += dedbr[j] * cj.dg;
            if (s != 0.0)
                for (int k = 0; k < 3; k++) {
                    gi[k] += s * v[k];
                    grad[3 * j + k] -= s * v[k];
                }
        }
        for (int k = 0; k < 3; k++) grad[3 * i + k] += gi[k];
    }
    // H-bond term through the surface
    if (sv.lhb)
        for (int i = 0; i < n; i++) {
            double c = sv.dhbdw[i] * q[i] * q[i];
            if (c == 0.0) continue;
            for (int k = 0; k < 3; k++) grad[3 * i + k] += sv.selfg[i][k] * c;
            for (size_t s = 0; s < sv.nb[i].size(); s++)
                for (int k = 0; k < 3; k++) grad[3 * sv.nb[i][s] + k] += sv.nbg[i][s][k] * c;
        }
    // ALPB shape term (kernel.rs:198-238)
    if (sv.alpbet > 0.0) {
        double qt = 0.0;
        for (double x : q) qt += x;
        double in[3][3], c[3];
        double tot = adet_inertia(m, sv.vdwr, in, c);
        double adet = std::sqrt(std::pow(det3(in), 1.0 / 3.0) / ((2.0 / 5.0) * tot));
        double t2 = tot * tot, a2 = adet * adet;
        double fa = 250.0 / (48.0 * (t2 * tot) * ((a2 * a2) * adet));
        double fb = -0.5 * sv.keps * sv.alpbet * (qt * qt) / a2;
        auto f = [&](double x) { return x * fa * fb; };
        double xy = in[0][1] * in[2][2] - in[0][2] * in[1][2];
        double xz = in[0][2] * in[1][1] - in[0][1] * in[2][1];
        double yz = in[0][0] * in[1][2] - in[0][1] * in[0][2];
        double xx = in[0][0] * (in[1][1] + in[2][2]) - in[0][1] * in[0][1] - in[0][2] * in[0][2];
        double yy = in[1][1] * (in[0][0] + in[2][2]) - in[0][1] * in[0][1] - in[1][2] * in[1][2];
        double zz = in[2][2] * (in[0][0] + in[1][1]) - in[0][2] * in[0][2] - in[1][2] * in[1][2];
        double d[3][3] = {{f(xx), f(xy), f(xz)}, {f(xy), f(yy), f(yz)}, {f(xz), f(yz), f(zz)}};
        for (int i = 0; i < n; i++) {
            double r3 = sv.vdwr[i] * sv.vdwr[i] * sv.vdwr[i];
            double v[3] = {m.R(i)[0] - c[0], m.R(i)[1] - c[1], m.R(i)[2] - c[2]};
            for (int k = 0; k < 3; k++) grad[3 * i + k] += r3 * (d[k][0] * v[0] + d[k][1] * v[1] + d[k][2] * v[2]);
        }
    }
}

// ============================================================================ Broyden
// modified Broyden mixing of crates/axtb/src/scf/mixing.rs:185-338 (memory = max_iter) with
// Gauss elimination crates/base/src/linalg/lu.rs:81-112
// sequential dot product (crates/base/src/math.rs:69-71)
double dot_seq(const vector<double>& x, const vector<double>& y) {
    double s = -0.0;
    for (size_t i = 0; i < x.size(); i++) s += x[i] * y[i];
    return s;
}

// a mixer of the packed SCC variables (crates/axtb/src/scf/mixing.rs:27-39 VectorMixer): the
// SCF writes the input q_in it built the Fock matrix from and the residual dq = out - q_in, and
// next() replaces q_in by the next input (false: the mixer failed)
struct VMix {
    vector<double> q_in, dq;
    explicit VMix(int n) : q_in(n), dq(n) {}
    virtual ~VMix() = default;
    virtual bool next() = 0;
};

struct Broyden : VMix {
    int n, memory, iter = 0;
    double damp;
    vector<vector<double>> df, u, a;
    vector<double> omega, qlast, dqlast;
    Broyden(int n_, int mem, double d) : VMix(n_), n(n_), memory(std::max(mem, 1)), damp(d), qlast(n_), dqlast(n_) {}
    static double dot(const vector<double>& x, const vector<double>& y) { return dot_seq(x, y); }
    bool next() override {
        iter++;
        if (iter == 1) {
            dqlast = dq;
            qlast = q_in;
            for (int i = 0; i < n; i++) q_in[i] += damp * dq[i];
            return true;
        }
        int itn = iter - 1;
        int it1 = (itn - 1) % memory;
        int nhist = std::min(memory, itn);
        int first = itn + 1 > memory ? itn + 1 - memory : 1;
        vector<int> hist(nhist);
        for (int ih = 0; ih < nhist; ih++) hist[ih] = (first + ih - 1) % memory;
        const double OMEGA0 = 0.01, MINW = 1.0, MAXW = 100000.0, WFAC = 0.01;
        if (it1 == (int)df.size()) {
            df.push_back(vector<double>(n, 0.0));
            u.push_back(vector<double>(n, 0.0));
            omega.push_back(0.0);
            for (auto& row : a) row.push_back(0.0);
            a.push_back(vector<double>(df.size(), 0.0));
        }
        double norm = std::sqrt(dot(dq, dq));
        omega[it1] = norm > WFAC / MAXW ? WFAC / norm : MAXW;
        if (omega[it1] < MINW) omega[it1] = MINW;
        for (int i = 0; i < n; i++) df[it1][i] = dq[i] - dqlast[i];
        double inv = 1.0 / std::max(std::sqrt(dot(df[it1], df[it1])), DBL_EPSILON);
        for (double& x : df[it1]) x *= inv;
        vector<double> c(nhist);
        vector<vector<double>> beta(nhist, vector<double>(nhist));
        for (int ih = 0; ih < nhist; ih++) {
            int i = hist[ih];
            c[ih] = omega[i] * dot(df[i], dq);
            for (int j : hist) a[i][j] = dot(df[i], df[j]);
        }
        for (int ih = 0; ih < nhist; ih++) {
            for (int jh = 0; jh < nhist; jh++) beta[ih][jh] = omega[hist[ih]] * omega[hist[jh]] * a[hist[ih]][hist[jh]];
            beta[ih][ih] += OMEGA0 * OMEGA0;
        }
        // Gauss elimination with the last largest pivot
        for (int col = 0; col < nhist; col++) {
            int piv = col;
            for (int i = col + 1; i < nhist; i++)
                if (std::fabs(beta[i][col]) >= std::fabs(beta[piv][col])) piv = i;
            if (beta[piv][col] == 0.0) return false;
            std::swap(beta[col], beta[piv]);
            std::swap(c[col], c[piv]);
            for (int row = col + 1; row < nhist; row++) {
                double f = beta[row][col] / beta[col][col];
                if (f != 0.0) {
                    for (int k = col; k < nhist; k++) beta[row][k] -= f * beta[col][k];
                    c[row] -= f * c[col];
                }
            }
        }
        for (int col = nhist - 1; col >= 0; col--) {
            double s = c[col];
            for (int k = col + 1; k < nhist; k++) s -= beta[col][k] * c[k];
            c[col] = s / beta[col][col];
        }
        for (int k = 0; k < n; k++) u[it1][k] = damp * df[it1][k] + inv * (q_in[k] - qlast[k]);
        dqlast = dq;
        qlast = q_in;
        for (int k = 0; k < n; k++) q_in[k] += damp * dq[k];
        for (int ih = 0; ih < nhist; ih++) {
            int i = hist[ih];
            double f = omega[i] * c[ih];
            for (int k = 0; k < n; k++) q_in[k] -= f * u[i][k];
        }
        return true;
    }
};

// ============================================================================ DIIS
// Pulay (DIIS / Anderson) mixing with restarts (crates/axtb/src/scf/mixing.rs:342-525): the
// constants of :342-357, next() of :414-458 and the coefficients of :466-525.
const int DIIS_SIZE = 30;
const double DIIS_DEPENDENCE = 1e-2;
const int DIIS_STALL = 12;
const double DIIS_RESTART_GROWTH = 1e3, DIIS_RESTART_FLOOR = 0.1;

// c minimising |sum_i c_i r_i| with sum_i c_i = 1, from min_g |r_n - sum_j g_j (r_n - r_j)|:
// the differences to the newest residual are orthonormalised newest first by modified
// Gram-Schmidt until one keeps less than DIIS_DEPENDENCE of its norm; R g = Q^T r_n is solved by
// back substitution, c_j = g_j for the kept j and c_n = 1 - sum g
vector<double> diis_coefficients(const std::deque<vector<double>>& r) {
    int m = (int)r.size();
    const vector<double>& last = r[m - 1];
    size_t n = last.size();
    vector<vector<double>> basis, rcol;
    vector<int> kept;
    for (int j = m - 2; j >= 0; j--) {
        vector<double> d(n);
        for (size_t k = 0; k < n; k++) d[k] = last[k] - r[j][k];
        double norm0 = std::sqrt(dot_seq(d, d));
        if (std::isnan(norm0) || norm0 <= 0.0) break;
        vector<double> col(basis.size() + 1, 0.0);
        for (size_t l = 0; l < basis.size(); l++) {
            double h = dot_seq(basis[l], d);
            col[l] = h;
            for (size_t k = 0; k < n; k++) d[k] -= h * basis[l][k];
        }
        double nr = std::sqrt(dot_seq(d, d));
        if (nr < DIIS_DEPENDENCE * norm0) break;
        col[basis.size()] = nr;
        for (double& x : d) x /= nr;
        basis.push_back(std::move(d));
        rcol.push_back(std::move(col));
        kept.push_back(j);
    }
    int p = (int)basis.size();
    vector<double> g(p, 0.0);
    for (int l = p - 1; l >= 0; l--) {
        double v = dot_seq(basis[l], last);
        for (int k = l + 1; k < p; k++) v -= rcol[k][l] * g[k];
        g[l] = v / rcol[l][l];
    }
    vector<double> c(m, 0.0);
    c[m - 1] = 1.0;
    for (int l = 0; l < p; l++) {
        c[kept[l]] += g[l];
        c[m - 1] -= g[l];
    }
    return c;
}

struct Diis : VMix {
    double damp;
    std::deque<vector<double>> hq, hr;
    bool have_best = false;
    double best_norm = 0.0;
    vector<double> best_q, best_r;
    int since_best = 0;
    Diis(int n, double d) : VMix(n), damp(d) {}
    bool next() override {
        double norm = std::sqrt(dot_seq(dq, dq));
        if (!std::isfinite(norm)) return false;
        if (have_best) {
            bool diverging = norm > DIIS_RESTART_GROWTH * best_norm && norm > DIIS_RESTART_FLOOR;
            if (diverging || since_best >= DIIS_STALL) {
                // restart from the best iterate with half the damping
                since_best = 0;
                hq.clear();
                hr.clear();
                damp *= 0.5;
                for (size_t k = 0; k < best_q.size(); k++) q_in[k] = best_q[k] + damp * best_r[k];
                return true;
            }
        }
        if (!have_best || norm < best_norm) {
            have_best = true;
            best_norm = norm;
            best_q = q_in;
            best_r = dq;
            since_best = 0;
        } else {
            since_best++;
        }
        if ((int)hq.size() == DIIS_SIZE) {
            hq.pop_front();
            hr.pop_front();
        }
        hq.push_back(q_in);
        hr.push_back(dq);
        vector<double> c = diis_coefficients(hr);
        for (size_t k = 0; k < q_in.size(); k++) {
            double x = 0.0;
            for (size_t i = 0; i < c.size(); i++)
                if (c[i] != 0.0) x += c[i] * (hq[i][k] + damp * hr[i][k]);
            q_in[k] = x;
        }
        return true;
    }
};

// ============================================================================ single point
const double SQRT2 = 1.4142135623730951;
const bool QOFF[6] = {false, true, false, true, true, false};

struct Moments {
    vector<double> qsh, qat, dp, qp;
};

void qat_from_qsh(const Basis& b, int nat, const vector<double>& qsh, vector<double>& qat) {
    qat.assign(nat, 0.0);
    for (int s = 0; s < b.nsh; s++) qat[b.sh2at[s]] += qsh[s];
}

void pack(const Moments& m, int nsh, int nat, vector<double>& v) {
    v.assign(nsh + 9 * nat, 0.0);
    for (int s = 0; s < nsh; s++) v[s] = m.qsh[s];
    for (int a = 0; a < nat; a++) {
        for (int c = 0; c < 3; c++) v[nsh + 3 * a + c] = m.dp[3 * a + c];
        for (int c = 0; c < 6; c++) v[nsh + 3 * nat + 6 * a + c] = m.qp[6 * a + c] * (QOFF[c] ? SQRT2 : 1.0);
    }
}
void unpack(const vector<double>& v, const Basis& b, int nat, Moments& m) {
    int nsh = b.nsh;
    m.qsh.assign(v.begin(), v.begin() + nsh);
    m.dp.assign(3 * nat, 0.0);
    m.qp.assign(6 * nat, 0.0);
    for (int a = 0; a < nat; a++) {
        for (int c = 0; c < 3; c++) m.dp[3 * a + c] = v[nsh + 3 * a + c];
        for (int c = 0; c < 6; c++) m.qp[6 * a + c] = v[nsh + 3 * nat + 6 * a + c] / (QOFF[c] ? SQRT2 : 1.0);
    }
    qat_from_qsh(b, nat, m.qsh, m.qat);
}

struct Pot {
    vector<double> vsh, vat, vdp, vqp;
};

int run(OracleRun* R) {
    Mol m;
    m.nat = R->nat;
    if (m.nat <= 0) throw Fail(1, "molecule has no atoms");
    m.Z.assign(R->numbers, R->numbers + m.nat);
    m.xyz.assign(R->positions, R->positions + 3 * m.nat);
    m.charge = R->charge;
    m.uhf = R->uhf;
    for (int z : m.Z) {
        if (z <= 0 || z > 118) throw Fail(1, "invalid atomic number");
        auto it = std::find(m.species.begin(), m.species.end(), z);
        if (it == m.species.end()) {
            m.species.push_back(z);
            m.id.push_back((int)m.species.size() - 1);
        } else {
            m.id.push_back((int)(it - m.species.begin()));
        }
    }
    double acc = R->accuracy;
    if (!(acc > 0.0)) throw Fail(1, "accuracy must be positive");
    if (R->conventions < 0 || R->conventions > 2) throw Fail(1, "unknown conventions (axtb, xtb or tblite)");
    g_conv = make_conv(R->conventions);
    int mixer_kind = R->mixer < 0 ? g_conv.default_mixer : R->mixer;
    if (mixer_kind > 2) throw Fail(1, "unknown SCF mixer (auto, broyden or diis)");
    Model md = build_model(m, acc);
    const Basis& b = md.b;
    int nat = m.nat, nsh = b.nsh, nao = b.nao;
    R->nsh = nsh;
    R->nao = nao;
    // electrons (crates/axtb/src/xtb.rs:1178-1212)
    double nref = 0.0;
    for (double x : md.refocc) nref += x;
    double nocc = nref - m.charge;
    long nel_int = std::lround(nocc);
    long nuhf = m.uhf >= 0 ? m.uhf : ((nel_int % 2) + 2) % 2;
    if (m.uhf >= 0 && (m.uhf % 2) != ((nel_int % 2) + 2) % 2) throw Fail(1, "electrons and unpaired electrons incompatible");
    if (nocc < 0.0 || nuhf > nocc) throw Fail(1, "impossible electron count");
    double nalpha = (nocc + nuhf) / 2.0, nbeta = (nocc - nuhf) / 2.0;
    if (nalpha > nao + 1e-9) throw Fail(1, "too many electrons for the basis");
    // aufbau occupations up to the conventions' temperature (crates/axtb/src/xtb.rs:462)
    double kt = R->etemp <= g_conv.aufbau_max_etemp ? 0.0 : R->etemp * g_conv.kb;

    // geometry: CN, self energies, gamma, AES cache, D4 (crates/axtb/src/xtb.rs:275-292)
    vector<double> cn = gfn2_cn(md);
    vector<double> se(nsh), dsedcn(nsh);
    for (int s = 0; s < nsh; s++) {
        se[s] = md.selfenergy[s] - md.kcn[s] * cn[b.sh2at[s]];
        dsedcn[s] = -md.kcn[s];
    }
    vector<double> gam = es2_gamma(md);
    AesCache ac = aes_cache(md, cn);
    D4 d4 = d4_setup(m);
    d4.off = R->no_dispersion != 0;
    bool wantg = R->want_gradient != 0;
    vector<double> grad(3 * nat, 0.0), dedcn(nat, 0.0);
    double e_rep = repulsion(md, wantg ? &grad : nullptr);
    double e_atm = d4.off ? 0.0 : d4_atm(d4, m, wantg ? &grad : nullptr);
    // implicit solvation: geometry part, surface energy and shift (crates/axtb/src/solvation.rs:66-75)
    bool solv = R->solv_model >= 0;
    Solv sv;
    double e_solv_fixed = 0.0;
    if (solv) {
        if (R->solv_model > 1 || R->solv_state < 0 || R->solv_state > 2) throw Fail(1, "solvation: unknown model or state");
        sv = solv_setup(m, R->solv_model, R->solvent, R->solv_state);
        solv_geometry(sv, m);
        e_solv_fixed = solv_fixed(sv, wantg ? &grad : nullptr);
    }
    Ints I = build_ints(md, se);
    GenEig eig;
    eig.init(I.S, nao, R->eig_backend == 1);
    if (eig.use_lapack && lapack().setthreads) lapack().setthreads(R->lapack_threads > 0 ? R->lapack_threads : 1);

    // start: EEQ charges split over shells by reference occupation (xtb.rs:522-549)
    Moments st;
    st.qsh.assign(nsh, 0.0);
    st.dp.assign(3 * nat, 0.0);
    st.qp.assign(6 * nat, 0.0);
    if (g_conv.eeq_guess) {
        vector<double> q = eeq_charges(m);
        for (int iat = 0; iat < nat; iat++) {
            int is = b.ish_at[iat], ns = b.nsh_at[iat];
            double tot = 0.0;
            for (int k = 0; k < ns; k++) tot += md.refocc[is + k];
            for (int k = 0; k < ns; k++) st.qsh[is + k] = tot > 0.0 ? q[iat] * md.refocc[is + k] / tot : 0.0;
        }
    }
    qat_from_qsh(b, nat, st.qsh, st.qat);

    int ndim = nsh + 9 * nat;
    const double econv = 1e-6 * acc, pconv = 2e-5 * acc;
    Pot pot;
    vector<double> F((size_t)nao * nao), C, emo, occa(nao), occb(nao), focc(nao), P((size_t)nao * nao);
    int kocc = 0;
    double ts = 0.0, elast = 0.0;
    double terms[8] = {0};
    Moments out;
    bool converged = false;
    int iters = 0, iters_all = 0;
    double esolv_last = 0.0;
    vector<double> packed, q_last;  // q_last: the last input of the last attempt
    // the attempts of the mixer plan (crates/axtb/src/scf/mixing.rs:163-199, run by
    // crates/axtb/src/xtb.rs:590-645): auto = Broyden, then DIIS from the start guess with its own
    // max_iter; a failed mixer or a lost Fermi level gives way to the next attempt and ends the
    // last one with its error (non-finite values end the single point at once)
    const int plan_auto[2] = {1, 2}, plan_broyden[1] = {1}, plan_diis[1] = {2};
    const int* plan = mixer_kind == 1 ? plan_broyden : mixer_kind == 2 ? plan_diis : plan_auto;
    int nplan = mixer_kind == 0 ? 2 : 1;
    for (int ia = 0; ia < nplan && !converged; ia++) {
        bool last_attempt = ia + 1 == nplan;
        std::unique_ptr<VMix> mixer;
        if (plan[ia] == 1) mixer.reset(new Broyden(ndim, R->max_iter, 0.4));
        else mixer.reset(new Diis(ndim, 0.4));
        VMix& mix = *mixer;
        Moments state = st;
        elast = 0.0;
        iters = 0;
        for (int iter = 1; iter <= R->max_iter; iter++) {
            if (iter > 1) {
                if (!mix.next()) {
                    if (last_attempt) throw Fail(4, plan[ia] == 1 ? "Broyden mixing failed" : "DIIS mixing failed");
                    break;
                }
                unpack(mix.q_in, b, nat, state);
            }
            iters = iter;
            // potentials (xtb.rs:316-340)
            pot.vsh.assign(nsh, 0.0);
            pot.vat.assign(nat, 0.0);
            pot.vdp.assign(3 * nat, 0.0);
            pot.vqp.assign(6 * nat, 0.0);
            for (int a = 0; a < nsh; a++) {
                double s = 0.0;
                for (int c = 0; c < nsh; c++) s += gam[(size_t)a * nsh + c] * state.qsh[c];
                pot.vsh[a] += s;
            }
            for (int a = 0; a < nsh; a++) pot.vsh[a] += state.qsh[a] * state.qsh[a] * md.gam3[a];
            aes_potential(md, ac, state.qat, state.dp, state.qp, pot.vat, pot.vdp, pot.vqp);
            if (!d4.off) d4_energy(d4, state.qat, &pot.vat);
            if (solv) solv_potential(sv, state.qat, pot.vat);
            // Fock (crates/axtb/src/scf/fock.rs:22-104)
            vector<double> B((size_t)nao * nao);
            for (int nu = 0; nu < nao; nu++) {
                int at = b.ao2at[nu];
                double v = pot.vsh[b.ao2sh[nu]] + pot.vat[at];
                for (int mu = 0; mu < nao; mu++) {
                    size_t k = (size_t)mu + (size_t)nu * nao;
                    double x = I.S[k] * v;
                    for (int c = 0; c < 3; c++) x += I.D[c][k] * pot.vdp[3 * at + c];
                    for (int c = 0; c < 6; c++) x += I.Q[c][k] * pot.vqp[6 * at + c];
                    B[k] = x;
                }
            }
            for (int nu = 0; nu < nao; nu++)
                for (int mu = 0; mu < nao; mu++) {
                    size_t k = (size_t)mu + (size_t)nu * nao;
                    F[k] = I.H0[k] - 0.5 * (B[k] + B[(size_t)nu + (size_t)mu * nao]);
                    if (!std::isfinite(F[k])) throw Fail(4, "non-finite Fock matrix");
                }
            pack(state, nsh, nat, mix.q_in);
            // diagonalize + fill (xtb.rs:997-1031)
            eig.solve(F, emo, C);
            double efa = 0, efb = 0;
            fill_tblite(nalpha, kt, emo, occa, efa);
            fill_tblite(nbeta, kt, emo, occb, efb);
            kocc = 0;
            for (int i = nao - 1; i >= 0; i--)
                if (occa[i] + occb[i] > 1e-16) {
                    kocc = i + 1;
                    break;
                }
            double pa = 0, pb = 0;
            for (int i = 0; i < nao; i++) {
                pa += occa[i];
                pb += occb[i];
            }
            if (std::fabs(pa - nalpha) > 1e-6 || std::fabs(pb - nbeta) > 1e-6) {
                if (last_attempt) throw Fail(4, "Fermi level not found");
                break;
            }
            ts = entropy_tblite(occa, kt) + entropy_tblite(occb, kt);
            for (int i = 0; i < nao; i++) focc[i] = occa[i] + occb[i];
            // density (occupied columns)
            std::fill(P.begin(), P.end(), 0.0);
            for (int k = 0; k < kocc; k++) {
                double f = focc[k];
                const double* c = &C[(size_t)k * nao];
                for (int nu = 0; nu < nao; nu++) {
                    double fc = f * c[nu];
                    for (int mu = 0; mu < nao; mu++) P[(size_t)mu + (size_t)nu * nao] += c[mu] * fc;
                }
            }
            // Mulliken (crates/axtb/src/scf/mulliken.rs:19-59)
            out.qsh.assign(md.refocc.begin(), md.refocc.end());
            out.dp.assign(3 * nat, 0.0);
            out.qp.assign(6 * nat, 0.0);
            for (int nu = 0; nu < nao; nu++) {
                int at = b.ao2at[nu];
                double r0 = 0.0, r[9] = {0};
                for (int mu = 0; mu < nao; mu++) {
                    size_t k = (size_t)mu + (size_t)nu * nao;
                    r0 += P[k] * I.S[k];
                    for (int c = 0; c < 3; c++) r[c] += P[k] * I.D[c][k];
                    for (int c = 0; c < 6; c++) r[3 + c] += P[k] * I.Q[c][k];
                }
                out.qsh[b.ao2sh[nu]] -= r0;
                for (int c = 0; c < 3; c++) out.dp[3 * at + c] -= r[c];
                for (int c = 0; c < 6; c++) out.qp[6 * at + c] -= r[3 + c];
            }
            qat_from_qsh(b, nat, out.qsh, out.qat);
            pack(out, nsh, nat, packed);
            for (int i = 0; i < ndim; i++) mix.dq[i] = packed[i] - mix.q_in[i];
            // energy (xtb.rs:1058-1146)
            double e2 = 0.0;
            for (int a = 0; a < nsh; a++) {
                double v = 0.0;
                for (int c = 0; c < nsh; c++) v += gam[(size_t)a * nsh + c] * out.qsh[c];
                e2 += 0.5 * out.qsh[a] * v;
            }
            double e3 = 0.0;
            for (int a = 0; a < nsh; a++) e3 += out.qsh[a] * out.qsh[a] * out.qsh[a] * md.gam3[a] / 3.0;
            double eaes = aes_energy(md, ac, out.qat, out.dp, out.qp);
            double edisp = d4.off ? 0.0 : d4_energy(d4, out.qat, nullptr);
            // band energy column by column, the columns' dots summed in order (xtb.rs:1130-1133)
            double band = 0.0;
            for (int nu = 0; nu < nao; nu++) {
                double col = 0.0;
                for (int mu = 0; mu < nao; mu++) col += I.H0[(size_t)mu + (size_t)nu * nao] * P[(size_t)mu + (size_t)nu * nao];
                band += col;
            }
            double esolv = solv ? solv_energy(sv, out.qat) : 0.0;
            esolv_last = esolv;
            double energy = e2 + e3 + eaes + edisp + ts + band + esolv;
            if (!std::isfinite(energy)) throw Fail(4, "non-finite energy");
            double res = 0.0;
            for (double x : mix.dq) res += x * x;
            res = std::sqrt(res / ndim);
            double de = energy - elast;
            elast = energy;
            terms[2] = energy;
            terms[3] = e2;
            terms[4] = e3;
            terms[5] = eaes;
            terms[1] = edisp;
            terms[6] = ts;
            terms[7] = band;
            if (std::fabs(de) < econv && res < pconv) {
                converged = true;
                break;
            }
        }
        iters_all += iters;
        R->mixer_used = plan[ia] == 1 ? 0 : (mixer_kind == 0 ? 2 : 1);
        q_last = mix.q_in;
    }
    // iterations of the converged attempt; of all attempts when none converged (xtb.rs:624-645)
    R->iterations = converged ? iters : iters_all;
    R->converged = converged;
    terms[0] = e_rep;
    terms[1] += e_atm;
    double energy = e_rep + e_atm + terms[2] + e_solv_fixed;
    R->e_solvation = e_solv_fixed + esolv_last;
    if (R->energy) *R->energy = energy;
    if (R->terms) std::memcpy(R->terms, terms, sizeof terms);
    if (R->qat) std::copy(out.qat.begin(), out.qat.end(), R->qat);
    if (R->qsh) std::copy(out.qsh.begin(), out.qsh.end(), R->qsh);
    if (R->dpat) std::copy(out.dp.begin(), out.dp.end(), R->dpat);
    if (R->qpat) std::copy(out.qp.begin(), out.qp.end(), R->qpat);
    if (R->emo) std::copy(emo.begin(), emo.end(), R->emo);
    if (R->focc) std::copy(focc.begin(), focc.end(), R->focc);
    if (R->density) std::copy(P.begin(), P.end(), R->density);
    if (R->dipole) {
        for (int k = 0; k < 3; k++) {
            double s = 0.0;
            for (int i = 0; i < nat; i++) s += out.qat[i] * m.R(i)[k] + out.dp[3 * i + k];
            R->dipole[k] = s;
        }
    }
    vector<double> W;
    if (wantg || R->wdensity) {
        W.assign((size_t)nao * nao, 0.0);
        for (int k = 0; k < kocc; k++) {
            double f = focc[k] * emo[k];
            const double* c = &C[(size_t)k * nao];
            for (int nu = 0; nu < nao; nu++) {
                double fc = f * c[nu];
                for (int mu = 0; mu < nao; mu++) W[(size_t)mu + (size_t)nu * nao] += c[mu] * fc;
            }
        }
        if (R->wdensity) std::copy(W.begin(), W.end(), R->wdensity);
    }
    if (!converged) throw Fail(3, "SCF not converged");
    if (wantg) {
        // add_scc_gradient (crates/axtb/src/xtb.rs:346-387) with the output moments and the
        // potentials of the last Fock matrix (SccGradient::Output); the xtb 6.8.0 conventions take
        // the dipole and quadrupole potentials of the output moments and shift the atom potential
        // by the AES atom potential of the output moments minus that of the last input
        // (SccGradient::OutputAes, crates/axtb/src/xtb.rs:700-722)
        if (g_conv.output_aes) {
            Moments in;
            unpack(q_last, b, nat, in);
            vector<double> ai(nat, 0.0), di(3 * nat, 0.0), qi(6 * nat, 0.0);
            vector<double> ao(nat, 0.0), dout(3 * nat, 0.0), qout(6 * nat, 0.0);
            aes_potential(md, ac, in.qat, in.dp, in.qp, ai, di, qi);
            aes_potential(md, ac, out.qat, out.dp, out.qp, ao, dout, qout);
            pot.vdp = dout;
            pot.vqp = qout;
            for (int i = 0; i < nat; i++) pot.vat[i] += ao[i] - ai[i];
        }
        es2_grad(md, out.qsh, grad);
        aes_grad(md, ac, out.qat, out.dp, out.qp, grad, dedcn);
        if (!d4.off) d4_grad(d4, m, out.qat, grad);
        if (solv) solv_gradient(sv, m, out.qat, grad);
        // H0/S/D/Q derivative contraction (crates/axtb/src/hamiltonian.rs:101-223)
        vector<double> vao(nao);
        for (int mu = 0; mu < nao; mu++) vao[mu] = pot.vsh[b.ao2sh[mu]] + pot.vat[b.ao2at[mu]];
        MGrad gr;
        for (int iat = 0; iat < nat; iat++) {
            int zi = m.Z[iat];
            for (int jat = 0; jat < iat; jat++) {
                int zj = m.Z[jat];
                double vec[3] = {m.R(iat)[0] - m.R(jat)[0], m.R(iat)[1] - m.R(jat)[1], m.R(iat)[2] - m.R(jat)[2]};
                double r2 = vec[0] * vec[0] + vec[1] * vec[1] + vec[2] * vec[2];
                if (r2 > b.pair_cut2 || pair_screened(b.amin_at[iat], b.amin_at[jat], r2, b.intcut)) continue;
                if (r2 < DBL_EPSILON) continue;
                double rr = std::sqrt(std::sqrt(r2) / (md.rad[jat] + md.rad[iat]));
                double dg[3] = {0, 0, 0}, dcni = 0.0, dcnj = 0.0;
                for (int ish = 0; ish < b.nsh_at[iat]; ish++) {
                    int si = b.ish_at[iat] + ish;
                    const Shell& ci = b.sh[si];
                    for (int jsh = 0; jsh < b.nsh_at[jat]; jsh++) {
                        int sj = b.ish_at[jat] + jsh;
                        const Shell& cj = b.sh[sj];
                        if (pair_screened(ci.amin, cj.amin, r2, b.intcut)) continue;
                        multipole_grad(cj, ci, vec, b.intcut, gr);
                        double shpi = 1.0 + md.shpoly[si] * rr, shpj = 1.0 + md.shpoly[sj] * rr;
                        double shp = shpi * shpj;
                        double dshp = (shpi * md.shpoly[sj] + shpj * md.shpoly[si]) * 0.5 * rr / r2;
                        double dsv[3] = {dshp / shp * vec[0], dshp / shp * vec[1], dshp / shp * vec[2]};
                        double hs = hscale(zj, jsh, zi, ish) * shp;
                        double hij = 0.5 * (se[si] + se[sj]) * hs;
                        double dhdcni = dsedcn[si] * hs, dhdcnj = dsedcn[sj] * hs;
                        int nj = nsph(cj.l);
                        for (int im = 0; im < nsph(ci.l); im++)
                            for (int jm = 0; jm < nj; jm++) {
                                int ij = jm + nj * im;
                                int mu = b.iao_sh[sj] + jm, nu = b.iao_sh[si] + im;
                                size_t k = (size_t)mu + (size_t)nu * nao;
                                double pij = P[k], hpij = pij * hij;
                                double sval = -pij * (vao[mu] + vao[nu]) + 2.0 * hpij - 2.0 * W[k];
                                for (int x = 0; x < 3; x++) {
                                    double mp = 0.0;
                                    for (int c = 0; c < 3; c++)
                                        mp += gr.ddi[ij][x][c] * pot.vdp[3 * iat + c] + gr.ddj[ij][x][c] * pot.vdp[3 * jat + c];
                                    for (int c = 0; c < 6; c++)
                                        mp += gr.dqi[ij][x][c] * pot.vqp[6 * iat + c] + gr.dqj[ij][x][c] * pot.vqp[6 * jat + c];
                                    dg[x] += sval * gr.ds[ij][x] + 2.0 * hpij * gr.s[ij] * dsv[x] - pij * mp;
                                }
                                dcni += dhdcni * pij * gr.s[ij];
                                dcnj += dhdcnj * pij * gr.s[ij];
                            }
                    }
                }
                dedcn[iat] += dcni;
                dedcn[jat] += dcnj;
                for (int x = 0; x < 3; x++) {
                    grad[3 * iat + x] += dg[x];
                    grad[3 * jat + x] -= dg[x];
                }
            }
            for (int ish = 0; ish < b.nsh_at[iat]; ish++) {
                int s = b.ish_at[iat] + ish, ii = b.iao_sh[s];
                double dc = 0.0;
                for (int k = 0; k < 2 * b.sh[s].l + 1; k++) dc += dsedcn[s] * P[(size_t)(ii + k) * (nao + 1)];
                dedcn[iat] += dc;
            }
        }
        gfn2_cn_grad(md, dedcn, grad);
        if (R->gradient) std::copy(grad.begin(), grad.end(), R->gradient);
    }
    return 0;
}

}  // namespace

extern "C" int oracle_sizes(int nat, const int* numbers, int* nsh, int* nao) {
    int s = 0, a = 0;
    for (int i = 0; i < nat; i++) {
        int z = numbers[i];
        if (z < 1 || z > 86) return -1;
        s += NSHELL[z - 1];
        for (int k = 0; k < NSHELL[z - 1]; k++) a += 2 * ANG_SHELL[z - 1][k] + 1;
    }
    *nsh = s;
    *nao = a;
    return 0;
}

extern "C" int oracle_singlepoint(OracleRun* R) {
    R->error[0] = 0;
    R->iterations = 0;
    R->converged = 0;
    R->mixer_used = 0;
    R->e_solvation = 0.0;
    try {
        return run(R);
    } catch (const Fail& f) {
        std::snprintf(R->error, sizeof R->error, "%s", f.what());
        return f.code;
    } catch (const std::exception& e) {
        std::snprintf(R->error, sizeof R->error, "%s", e.what());
        return 4;
    }
}

// the DIIS mixer alone, for its own tests (crates/axtb/src/scf/mixing.rs:583-652): coefficients
// of m residuals of length n (row i = r_i, oldest first)
extern "C" void oracle_diis_coefficients(int m, int n, const double* r, double* c) {
    std::deque<vector<double>> h;
    for (int i = 0; i < m; i++) h.emplace_back(r + (size_t)i * n, r + (size_t)(i + 1) * n);
    vector<double> v = diis_coefficients(h);
    std::copy(v.begin(), v.end(), c);
}

// DIIS on the linear fixed point q = diag(eig) q + b from q = 0: steps until the RMS residual is
// below tol (or -1 after max_steps, or -2 when the mixer failed); the last input in q
extern "C" int oracle_diis_linear(int n, const double* eig, const double* b, double damp, double tol, int max_steps,
                                  double* q) {
    Diis mix(n, damp);
    for (int step = 0;; step++) {
        double rr = 0.0;
        for (int k = 0; k < n; k++) {
            mix.dq[k] = eig[k] * mix.q_in[k] + b[k] - mix.q_in[k];
            rr += mix.dq[k] * mix.dq[k];
        }
        std::copy(mix.q_in.begin(), mix.q_in.end(), q);
        if (std::sqrt(rr / n) < tol) return step;
        if (step == max_steps) return -1;
        if (!mix.next()) return -2;
    }
}

extern "C" int oracle_integrals(int nat, const int* numbers, const double* positions, double acc, double* cn_out,
                                double* S, double* H0, double* D, double* Q) {
    try {
        g_conv = make_conv(0);
        Mol m;
        m.nat = nat;
        m.Z.assign(numbers, numbers + nat);
        m.xyz.assign(positions, positions + 3 * nat);
        for (int z : m.Z) {
            auto it = std::find(m.species.begin(), m.species.end(), z);
            if (it == m.species.end()) {
                m.species.push_back(z);
                m.id.push_back((int)m.species.size() - 1);
            } else {
                m.id.push_back((int)(it - m.species.begin()));
            }
        }
        Model md = build_model(m, acc);
        vector<double> cn = gfn2_cn(md);
        if (cn_out) std::copy(cn.begin(), cn.end(), cn_out);
        vector<double> se(md.b.nsh);
        for (int s = 0; s < md.b.nsh; s++) se[s] = md.selfenergy[s] - md.kcn[s] * cn[md.b.sh2at[s]];
        Ints I = build_ints(md, se);
        size_t nn = (size_t)I.n * I.n;
        if (S) std::copy(I.S.begin(), I.S.end(), S);
        if (H0) std::copy(I.H0.begin(), I.H0.end(), H0);
        if (D)
            for (int k = 0; k < 3; k++) std::copy(I.D[k].begin(), I.D[k].end(), D + k * nn);
        if (Q)
            for (int k = 0; k < 6; k++) std::copy(I.Q[k].begin(), I.Q[k].end(), Q + k * nn);
        return 0;
    } catch (const Fail& f) {
        return f.code;
    }
}
