// Device-side layout of a batch of molecules and small helpers shared by the kernels.
//
// Every quantity of every molecule lives in one flat array per kind, indexed globally:
// atoms, shells and AOs of molecule m start at m_at0[m], m_sh0[m], m_ao0[m]; its dense AO
// matrices (column-major, leading dimension nao_m) start at m_mat0[m] in each matrix plane;
// its SCC vector (nsh + 9 nat entries) at m_vec0[m]; its atom pairs (i > j, packed
// i(i-1)/2 + j) at m_pair0[m]. Kernels take global work indices and find their molecule
// through these offsets, so one launch serves one molecule or thousands.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace axg {

constexpr int MAXPRIM = 6;
constexpr int MAXREF = 7;
constexpr int NFREQ = 23;

// Status bits of one molecule (per-molecule word on the device)
enum : int {
    ST_NOT_PD = 1,         // overlap (or EEQ) matrix not positive definite
    ST_NONFINITE = 2,      // non-finite energy
    ST_FERMI = 4,          // electrons not placed by the Fermi search
    ST_MIXER = 8,          // mixer failed (Broyden system singular, non-finite DIIS residual)
    ST_INVIT = 16,         // inverse iteration produced a non-finite vector
    ST_HISTORY = 32,       // Broyden history capacity exhausted
    ST_TIMEOUT = 64,       // a bounded device wait gave up
    ST_FOCK = 128,         // non-finite Fock matrix
    ST_SOLV = 256,         // an atom has more SASA neighbours than the solvation lists hold
};

struct Batch {
    int nmol, natT, nshT, naoT;
    long long nnT;      // sum of nao^2
    long long npairT;   // sum of nat(nat-1)/2
    long long nvecT;    // sum of SCC vector lengths
    int nsp;            // distinct elements in the batch (D4 tables)
    int hist_cap;       // Broyden history slots per molecule (the span holds at least DIIS's)
    // molecules
    const int *m_nat, *m_nsh, *m_nao, *m_at0, *m_sh0, *m_ao0, *m_dim;
    const long long *m_mat0, *m_vec0, *m_pair0, *m_hist0;
    const long long* m_gam0;          // per-molecule offsets of the shell gamma matrices (sum nsh^2)
    const double *m_nalpha, *m_nbeta, *m_charge;
    // atoms
    const int *a_Z, *a_mol, *a_sh0, *a_nsh, *a_ao0, *a_sp;
    const double *a_rcov;      // GFN2 CN covalent radius (bohr)
    const double *a_rad;       // H0 shell-polynomial atomic radius (bohr)
    const double *a_amin;      // smallest primitive exponent of the atom
    const double *a_rcov_eeq;  // EEQ-guess CN covalent radius (bohr)
    const double *a_en;        // Pauling EN
    const double *a_aes_rad, *a_aes_vcn, *a_dk, *a_qk;  // AES parameters
    const double *a_rep_alpha, *a_rep_zeff;
    const double *a_eeq_chi, *a_eeq_eta, *a_eeq_kcn, *a_eeq_rad;
    // shells
    const int *s_l, *s_np, *s_at, *s_ao0, *s_ish, *s_mol;
    const double *s_alpha, *s_coeff;  // [shell][MAXPRIM]
    const double *s_amin, *s_se0, *s_kcn, *s_shpoly, *s_refocc, *s_hard, *s_gam3, *s_slater;
    const int *s_Z;
    // AOs
    const int *o_sh, *o_at;
    // D4 species tables (batch species = distinct elements)
    const int *sp_nref, *sp_ngw;      // nref[nsp], ngw[nsp][MAXREF]
    const double *sp_refcn, *sp_refq, *sp_zeff, *sp_gi, *sp_rcov, *sp_en;  // per species (x MAXREF)
    const double *sp_c6ref;           // [nsp*nsp][MAXREF][MAXREF]
    const double *sp_rr, *sp_r0;      // [nsp*nsp]
    double intcut;                    // primitive screening threshold
    double kt;                        // electronic kT (Eh)
    double damping;
    double econv, pconv;
    int max_iter;
    // real-space cutoffs (bohr) of the conventions (crates/axtb/src/conventions.rs:150-353): GFN2
    // CN, repulsion, D4 CN, D4 two-body and three-body with their smooth-switch widths, EEQ-guess
    // CN with its log cap (<= 0: none); squared atom-pair cutoff of the integrals per molecule
    double cn_cut, rep_cut, d4_cn_cut, d2_cut, d2_w, d3_cut, d3_w, eeq_cn_cut, eeq_cap;
    const double* m_paircut2;
    int output_aes;  // 1: gradient with the AES potentials of the output moments (xtb 6.8.0)
    // implicit solvation (crates/solvation): on, ALPB (else GBSA), model scalars, per-atom
    // radii, surface and H-bond parameters, per-molecule SASA neighbour cutoff
    int solv, sv_alpb;
    double sv_keps, sv_alpbet, sv_c1, sv_lrcut, sv_w, sv_ah0, sv_ah1, sv_ah3, sv_gshift;
    const double *sv_vdwr, *sv_rho, *sv_svdw, *sv_vdwsa, *sv_t1, *sv_t2, *sv_wrp, *sv_gam, *sv_hbmag;
    const double* sv_srcut;
    int split;                        // 1: basis-transform and W GEMMs in split precision
    int disp;                         // 0: the D4 term is left out (Options::dispersion = false)
    int band_max;                     // one-CTA molecules below this many AOs reduce to tridiagonal form in two stages
    int chase_max;                    // ... with stage 2 in its own launch (k_chase) up to this many AOs (0: none)
};

// per-geometry and per-iteration device state
struct State {
    double* xyz;          // natT*3
    // geometry intermediates
    double *cn, *se, *dsedcn, *mrad, *dmrdcn, *cn_d4, *cn_eeq;
    // AO matrices: planes of nnT doubles
    double *S, *H0, *D, *Q;  // D: 3 planes, Q: 6 planes
    double *Linv;
    double *F, *Fp, *Z, *C, *P, *W;
    double *scr1, *scr2, *scr3;  // nnT each: inverse-iteration / back-transform scratch
    unsigned char* piv;          // nnT
    double *emo, *focc;          // naoT
    double* focc_a;              // naoT: alpha occupations (NULL: not kept)
    double* efermi;              // 2 nmol: alpha and beta Fermi levels (NaN: aufbau filling; NULL: not kept)
    double *dtri, *etri, *tau;   // naoT: tridiagonal and Householder factors
    int* kocc;                   // nmol
    // SCC moments (input = mixed, output = Mulliken)
    double *qsh_in, *qat_in, *dp_in, *qp_in;
    double *qsh_out, *qat_out, *dp_out, *qp_out;
    double *vsh, *vat, *vdp, *vqp;  // potentials of the last Fock build
    double *gw, *dgw;               // D4 weights and their charge (or CN) derivatives [natT][MAXREF]
    double *ao_part;                // naoT * 11: per-AO column dots (S, D3, Q6, H0)
    // mixer
    double *q_in, *dq, *qlast, *dqlast, *df, *u, *amat, *omega;  // vecs; df/u: hist x vec
    int* iter;                      // nmol: mixer iteration counter
    double* diis;                   // nmol*8: DIIS scalars
    double* start;                  // nshT + 10 natT: start moments (qsh; qat, dp, qp per atom)
    int* mix_used;                  // nmol: 0 Broyden, 1 DIIS, 2 DIIS after Broyden
    int* niter_prev;                // nmol: iterations of an earlier attempt
    int* have_guess;                // nmol: 1 when the molecule's output moments are a converged start
    int* retry;                     // nmol: molecules that run again from the fresh guess
    // per molecule scalars
    double *energy, *elast, *de, *res, *ts, *e_fixed;  // nmol
    double* terms;     // nmol*8
    int* status;       // nmol
    int* conv;         // nmol: 1 converged, 0 running
    int* active;       // nmol: 1 while the SCF runs
    int* niter;        // nmol: SCF iterations done
    double *grad, *dedcn, *dedcn_d4;  // natT*3, natT, natT
    double* pair_buf;  // npairT*8: per atom-pair gradient partials
    double* e_atom;    // natT
    double* mol_cyc;   // nmol: SM cycles of each molecule's last eigen phase (profiling runs)
    double* e_terms;   // natT*5: ES2, ES3, AES, D4 two-body, band per atom
    // implicit solvation: Born radii and dbrad/dpsi, surface areas, H-bond weights and their
    // surface derivative factors, self surface derivatives (natT*3), dE/dpsi, A_det per molecule,
    // SASA neighbour lists (natT*SOLV_MAXNB) and counts
    double *sv_brad, *sv_dbrad, *sv_sasa, *sv_hbw, *sv_dhbdw, *sv_selfg, *sv_dedbr, *sv_adet;
    double *sv_eatom, *sv_emol;  // solvation energy per atom (last iteration) and per molecule
    int *sv_nb, *sv_nbn;
    // cooperative scratch
    double* red;       // reduction partials (grid-size * 8)
    double* eeq_A;     // EEQ system matrices (sum (nat)^2)
    double* gam;       // shell gamma matrices of the geometry, per molecule nsh x nsh (row s, column t)
    long long* m_eeq0;
};

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double sq(double x) { return x * x; }

// molecule owning global work index g, given ascending per-molecule start offsets
__device__ __forceinline__ int find_mol(const long long* off, int nmol, long long g) {
    int lo = 0, hi = nmol - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

}  // namespace axg
