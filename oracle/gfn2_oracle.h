/* TEST INFRASTRUCTURE - NOT PART OF THE PRODUCT.
 *
 * CPU FP64 restatement of axtb's GFN2-xTB energy + analytic gradient single point in its
 * default ("axtb") conventions and its xtb 6.8.0 and tblite 0.8.0 conventions, used only as the parity checker of the CUDA path (tests/,
 * __graft_entry__.smoke) and as the timed CPU baseline of bench.py. Parity of this restatement
 * is pinned against the reference's own recorded results (tests/golden, generated from
 * axtb tests/reference_matrix/results.json: absolute energies, energy terms, charges and
 * dipoles of axtb 0.1.0 at SCF accuracy 1e-6) and against central finite differences of its
 * own energy for the gradient (the reference's tests/consistency.rs check). */
#pragma once
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    /* inputs */
    int nat;
    const int* numbers;      /* atomic numbers, nat */
    const double* positions; /* bohr, nat*3 row-major */
    double charge;
    int uhf;                 /* -1: default (nel mod 2) */
    double accuracy;         /* SCF accuracy multiplier (1.0 = xtb default) */
    double etemp;            /* K */
    int max_iter;
    int want_gradient;
    int eig_backend;         /* 0: builtin Householder/QL, 1: dlopen'ed LAPACK when found */
    int lapack_threads;      /* threads of the LAPACK backend (0 = library default) */
    int mixer;               /* -1: the conventions' mixer; 0: auto (Broyden, then DIIS from the
                                start guess), 1: Broyden, 2: DIIS */
    int conventions;         /* 0: axtb (default), 1: the xtb 6.8.0 program's, 2: tblite 0.8.0's */
    int solv_model;          /* implicit solvation: -1 none, 0 ALPB, 1 GBSA */
    const char* solvent;     /* solvent name (xtb's names and aliases) */
    int solv_state;          /* reference state: 0 gsolv, 1 bar1M, 2 reference */
    int no_dispersion;       /* 1: leave the D4 term out (Options::dispersion = false,
                                crates/axtb/src/lib.rs:185-187); 0: with it (default) */
    /* outputs (caller-allocated; any may be NULL) */
    double* energy;
    double* gradient;        /* nat*3 */
    double* qat;             /* nat */
    double* qsh;             /* nsh */
    double* dpat;            /* nat*3 */
    double* qpat;            /* nat*6 */
    double* dipole;          /* 3 */
    double* terms;           /* 8: repulsion, dispersion, electronic, isotropic_es,
                                third_order, anisotropic, entropy, band */
    double* emo;             /* nao orbital energies */
    double* focc;            /* nao occupations */
    double* density;         /* nao*nao, column-major */
    double* wdensity;        /* nao*nao */
    double e_solvation;      /* the solvation term (its surface, shift and polar parts), Eh */
    int iterations;          /* of the converged attempt; of all attempts when none converged */
    int converged;
    int mixer_used;          /* mixer of the last attempt: 0 Broyden, 1 DIIS, 2 DIIS after Broyden (auto) */
    int nsh, nao;
    char error[256];
} OracleRun;

/* Number of shells and AOs of a molecule (negative on an unsupported element). */
int oracle_sizes(int nat, const int* numbers, int* nsh, int* nao);

/* Full single point; returns 0 on success, a nonzero status (1 input, 2 unsupported element,
 * 3 SCF not converged, 4 numerical) otherwise, with a message in run->error. */
int oracle_singlepoint(OracleRun* run);

/* Intermediates of one geometry (for kernel-level parity): GFN2 coordination numbers (nat),
 * overlap, core Hamiltonian, dipole (3) and quadrupole (6) matrices (nao*nao column-major,
 * any pointer may be NULL) at SCF accuracy acc. */
int oracle_integrals(int nat, const int* numbers, const double* positions, double acc,
                     double* cn, double* S, double* H0, double* D, double* Q);

/* The DIIS mixer alone: Pulay coefficients of m residuals of length n (row-major, oldest
 * first) into c (m); and DIIS on the linear fixed point q = diag(eig) q + b from q = 0, returning
 * the steps until the RMS residual is below tol (-1: not within max_steps, -2: mixer failed)
 * with the last input in q (n). */
void oracle_diis_coefficients(int m, int n, const double* r, double* c);
int oracle_diis_linear(int n, const double* eig, const double* b, double damp, double tol, int max_steps,
                       double* q);

#ifdef __cplusplus
}
#endif
