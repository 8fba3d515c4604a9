/* axtb_gpu.h - C ABI of the B200 (sm_100a) GFN2-xTB energy + gradient engine.
 *
 * Drop-in boundary for axtb's GFN2-xTB single point. The reference interface each entry point
 * replaces (paths in the axtb repository):
 *
 *   axtb_gpu_create       axtb::Calculator::new(Hamiltonian::Gfn2, numbers, positions, charge,
 *                         uhf, Options) -- crates/axtb/src/calculator.rs:92-128, with the
 *                         molecule checks of crates/base/src/molecule.rs:35-60 and the SCF
 *                         option checks of crates/axtb/src/xtb.rs:1159-1174
 *   axtb_gpu_singlepoint  Method::singlepoint(&mut self, positions, &Want) --
 *                         crates/base/src/method/mod.rs:62, impl crates/axtb/src/calculator.rs:387-395
 *                         (the warm start from the previous geometry's moments,
 *                         calculator.rs:194-206), returning the SinglePoint fields of
 *                         crates/base/src/method/results.rs:39-57
 *   axtb_gpu_batch        no reference counterpart (axtb runs one calculation per process or
 *                         per Session lineage, crates/driver/src/calculator.rs:258-277): many
 *                         independent single points in one device pass
 *   axtb_gpu_destroy      Drop of the calculator
 *   axtb_gpu_last_error   the message of crates/base/src/error.rs:8-24 Error values
 *
 * Status codes mirror the reference's Error kinds (crates/base/src/error.rs:8-24).
 * Nothing here aborts, traps or hangs: device loops are bounded by max_iter and report a
 * status. All pointers are host pointers unless stated; outputs are caller-allocated and no
 * pointer is retained after a call returns. A handle is used by one thread at a time.
 */
#ifndef AXTB_GPU_H
#define AXTB_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum AxtbStatus {
    AXTB_OK = 0,
    AXTB_ERR_INPUT = 1,               /* Error::Input */
    AXTB_ERR_UNSUPPORTED_ELEMENT = 2, /* Error::UnsupportedElement */
    AXTB_ERR_SCF_NOT_CONVERGED = 3,   /* Error::ScfNotConverged {iterations, energy_change, residual} */
    AXTB_ERR_NUMERICAL = 4,           /* Error::Numerical (non-finite values, lost Fermi level, ...) */
    AXTB_ERR_DEVICE = 5,              /* CUDA error or missing device (no CPU fallback exists) */
};

/* Options (crates/axtb/src/lib.rs:92-133 Options and ScfSettings; defaults of
 * crates/axtb/src/xtb.rs:101-106). Fill with axtb_gpu_default_options. */
typedef struct AxtbOptions {
    double accuracy;   /* SCF accuracy multiplier (thresholds 1e-6*acc Eh and 2e-5*acc e); 1.0 */
    double etemp;      /* electronic temperature, K; 300 */
    int32_t max_iter;  /* iterations of the SCF; 250 */
    double damping;    /* Broyden damping, (0, 1]; 0.4 */
    int32_t guess;     /* 0: EEQ charges (default), 1: neutral atoms */
    int32_t precision; /* 0: FP64 throughout (default); 1: split precision: the basis-transform
                          (F' = L^-1 F L^-T) and energy-weighted-density GEMMs as BF16 tensor-core
                          products of three-part split operands (FP32-level accuracy); eigensolver,
                          C, P, mixer and sums stay FP64. For SCC accuracy >= ~1e-3; tighter
                          settings ask for energy changes below its rounding floor. */
    int32_t device;    /* CUDA device ordinal; 0 */
    int32_t mixer;     /* SCC mixer (crates/axtb/src/scf/mixing.rs:81-94 MixerKind): -1 the
                          conventions' (default: auto for axtb, Broyden for xtb and tblite); 0 auto
                          (modified Broyden; a molecule it leaves unconverged, with a failed mixer or
                          a lost Fermi level starts again from its start moments with DIIS and
                          another max_iter iterations), 1 Broyden alone, 2 DIIS alone */
    int32_t conventions; /* crates/axtb/src/conventions.rs Conventions: 0 axtb (default), 1 the xtb
                          6.8.0 program's (its element tables, 25/30/50/25 bohr cutoffs, tblite's
                          screening, aufbau up to 0.1 K, its EEQ-start CN, the gradient with the
                          AES potentials of the output moments), 2 tblite 0.8.0's (mctc-lib radii,
                          the same cutoffs, atom-pair integral cutoff, zero-charge start) */
    int32_t solvation;   /* implicit solvation (crates/axtb/src/solvation.rs, crates/solvation): -1 none
                          (default), 0 ALPB, 1 GBSA; GFN2-xTB parameters of xtb, the corrected variant in
                          the axtb and tblite conventions, xtb's in the xtb conventions */
    const char* solvent; /* the solvent, by xtb's names and aliases (case-insensitive); read during
                          axtb_gpu_create / axtb_gpu_batch_create only */
    int32_t solvation_state; /* reference state of the solvation free energy: 0 gsolv (default),
                          1 bar1M, 2 reference */
    int32_t dispersion;  /* 1 (default): with the D4 dispersion term; 0: without it (Options::dispersion,
                          crates/axtb/src/lib.rs:106-107, 185-187: for validation only) */
    int32_t band_max_nao; /* schedule of the dense algebra (no reference counterpart; results agree to
                          round-off either way): molecules of 34 AOs up to below this many use the
                          two-stage tridiagonal reduction, the others the one-stage one; -1 the default (64;
                          axtb_b200.autotune measures the crossover on a device) */
    int32_t grid_min_nao; /* molecules from this many AOs run their dense algebra on the whole GPU,
                          the rest one per CTA; -1 the default (1024) */
} AxtbOptions;

/* Results of one single point (crates/base/src/method/results.rs:39-57). Array members are
 * caller-allocated and may be NULL when not wanted. */
typedef struct AxtbResult {
    double energy;          /* total energy, Eh */
    double* gradient;       /* nat*3, Eh/bohr (written when the gradient is requested) */
    double* charges;        /* nat Mulliken atomic charges */
    double* dipole;         /* 3, e*bohr */
    double* qsh;            /* nsh shell charges */
    double* dpat;           /* nat*3 atomic dipoles */
    double* qpat;           /* nat*6 atomic quadrupoles (xx, xy, yy, xz, yz, zz) */
    double terms[8];        /* repulsion, dispersion, electronic, isotropic_es, third_order,
                               anisotropic, entropy, band */
    int32_t iterations;     /* SCF iterations of the converged attempt (of all attempts on failure) */
    int32_t converged;      /* 1 when converged */
    int32_t status;         /* AxtbStatus of this molecule */
    double energy_change;   /* last |dE| (ScfNotConverged payload) */
    double residual;        /* last residual norm (ScfNotConverged payload) */
    int32_t mixer_used;     /* mixer of the result (ScfResult::mixer_used): 0 Broyden, 1 DIIS,
                               2 DIIS after Broyden did not converge ("diis-fallback") */
    double solvation;       /* the solvation term (surface, shift and polar parts; part of the
                               electronic subtotal as in crates/axtb/src/calculator.rs:301-316); 0 without */
    /* the electronic structure (Electronic of crates/base/src/method/results.rs:77-142) */
    double* emo;            /* nao orbital energies (Eh), ascending: every level (OrbitalLevels::energies) */
    double* focc;           /* nao occupations of both spins together (0..2) */
    double* focc_alpha;     /* nao alpha occupations (beta = focc - focc_alpha) */
    double fermi_levels[2]; /* alpha and beta Fermi levels (Eh); NaN where the occupations are the
                               aufbau filling (0 K, or no electrons of that spin) */
    double electronic_temperature; /* K of the occupations; 0 where they are the aufbau filling */
    int32_t nao;            /* basis functions: the length of emo, focc, focc_alpha */
    int32_t warm_start;     /* 1: the SCF of the result started from previous or given moments
                               (ScfReport::start "previous"), 0: from the guess */
    int32_t fallback_iterations; /* iterations of the Broyden attempt that the DIIS fallback replaced
                               (mixer_used 2; ScfReport::attempts), 0 otherwise */
    double timings[4];      /* wall time (s) of the device pass the result came from: set-up
                               (geometry, integrals, overlap factorisation, guess), scf, gradient,
                               total (SinglePoint::timings; a batch reports the batch's pass) */
} AxtbResult;

/* One molecule of a batch: atomic numbers, positions (bohr, nat*3 row-major), charge and the
 * number of unpaired electrons (-1 for the default, nel mod 2). */
typedef struct AxtbMol {
    int32_t nat;
    const int32_t* numbers;
    const double* positions;
    double charge;
    int32_t uhf;
} AxtbMol;

typedef struct AxtbHandle AxtbHandle;
typedef struct AxtbBatch AxtbBatch;

void axtb_gpu_default_options(AxtbOptions* opts);

/* Sizes of a molecule's basis (shells and AOs); AXTB_ERR_UNSUPPORTED_ELEMENT past Rn. */
int axtb_gpu_basis_size(const int32_t* numbers, int32_t nat, int32_t* nsh, int32_t* nao);

/* Calculator for one molecule (axtb::Calculator::new). The positions set the first geometry
 * checked; singlepoint takes the positions of each call. */
int axtb_gpu_create(const int32_t* numbers, int32_t nat, double charge, int32_t uhf, const AxtbOptions* opts,
                    AxtbHandle** out);

/* E (+ gradient when want_gradient) at `positions` (host, bohr, nat*3). The SCF starts from the
 * previous call's converged moments when there is one, and once more from the EEQ guess when
 * that start fails (crates/axtb/src/calculator.rs:194-206). */
int axtb_gpu_singlepoint(AxtbHandle* h, const double* positions, int32_t want_gradient, AxtbResult* out);

/* The SCC moments the calculator's next SCF starts from: shell charges (nsh), atomic dipoles
 * (nat*3) and atomic quadrupoles (nat*6, xx, xy, yy, xz, yz, zz) -- the converged moments of its
 * last successful single point, or the ones given to it (Method::wavefunction,
 * crates/axtb/src/calculator.rs:413-423). Any output may be NULL. AXTB_ERR_INPUT when it has none
 * (before the first converged single point, or after a failed one: reset_wavefunction). */
int axtb_gpu_get_moments(const AxtbHandle* h, double* qsh, double* dpat, double* qpat);

/* Start the next SCF from these moments (sizes as above; another calculator's or another
 * program's converged moments): given = 1 is Method::set_wavefunction, given = 0 is
 * Method::set_history(Some) (crates/axtb/src/calculator.rs:425-442; this calculator always reuses
 * previous moments, so the two start the same way). qsh = NULL forgets them
 * (set_history(None)). The single point that starts from them still runs once more from the
 * guess when it does not converge. */
int axtb_gpu_set_moments(AxtbHandle* h, const double* qsh, const double* dpat, const double* qpat, int32_t given);

void axtb_gpu_destroy(AxtbHandle* h);

/* Message of the last failed call on `h` (or of the last failed handle-less call when h is
 * NULL); returns the message length. */
int axtb_gpu_last_error(const AxtbHandle* h, char* buf, size_t len);

/* Many independent single points in one device pass. `outs[i]` receives molecule i's results,
 * `status[i]` its AxtbStatus (also outs[i].status). Returns AXTB_OK when the pass ran (per-
 * molecule failures are reported in status), an error code otherwise. */
int axtb_gpu_batch(const AxtbMol* mols, int32_t nmol, const AxtbOptions* opts, int32_t want_gradient,
                   AxtbResult* outs, int32_t* status);

/* Reusable batch: set up once for a list of molecules (their numbers, charges, spins and a
 * first geometry), then run it on new positions. axtb_gpu_batch_run takes host positions
 * (all molecules' nat*3 arrays concatenated in batch order); axtb_gpu_batch_run_device takes
 * a DEVICE pointer to the same layout and writes energies (nmol) and, with want_gradient,
 * gradients (same layout as the positions) to DEVICE pointers, on the batch's stream. */
int axtb_gpu_batch_create(const AxtbMol* mols, int32_t nmol, const AxtbOptions* opts, AxtbBatch** out);
int axtb_gpu_batch_run(AxtbBatch* b, const double* positions, int32_t want_gradient, AxtbResult* outs,
                       int32_t* status);
int axtb_gpu_batch_run_device(AxtbBatch* b, const double* d_positions, int32_t want_gradient, double* d_energy,
                              double* d_gradient, int32_t* status);
/* Restarts across runs (a trajectory of geometries): with enable = 1, every later run starts
 * each molecule from its converged moments of the previous run (a molecule without them from
 * the guess), and a molecule that then ends unconverged runs once more from the guess, as each
 * molecule's axtb::Calculator does under Restart::Previous (crates/axtb/src/calculator.rs:185-206,
 * crates/base/src/method/retry.rs:150-158). enable = 2 is the same without the second run from
 * the guess: a molecule whose warm start does not converge reports the failure, as the displaced
 * points of axtb's numerical Hessian do (crates/axtb/src/calculator.rs:273-284). enable = 0 (the
 * default) forgets the moments. Every call forgets the moments of the previous run. */
int axtb_gpu_batch_set_restart(AxtbBatch* b, int32_t enable);
/* Molecule mol's converged output moments of the last run (sizes as for axtb_gpu_get_moments;
 * any output may be NULL); AXTB_ERR_INPUT when it did not converge. */
int axtb_gpu_batch_get_moments(AxtbBatch* b, int32_t mol, double* qsh, double* dpat, double* qpat);
/* Start molecule mol of the next run from these moments (a session lineage's previous moments,
 * or the reference point of a Hessian's displacements); turns restarts on (enable = 1 unless
 * axtb_gpu_batch_set_restart chose 2 before). */
int axtb_gpu_batch_set_moments(AxtbBatch* b, int32_t mol, const double* qsh, const double* dpat, const double* qpat);
/* The CUDA stream (cudaStream_t) the batch runs on, for callers that time or order work. */
void* axtb_gpu_batch_stream(AxtbBatch* b);
/* Number of kernels the last run launched (counted on the host at each launch). */
int64_t axtb_gpu_batch_launches(const AxtbBatch* b);
void axtb_gpu_batch_destroy(AxtbBatch* b);

/* Orbital energies, Fermi occupations and density matrix of one molecule from its Fock matrix
 * and overlap matrix (FC = SCe with Fermi smearing at kT for nalpha + nbeta electrons), without
 * allocating any device memory. No counterpart in the reference: it is for callers that cannot
 * call cudaMalloc, e.g. code inside another framework's stream-ordered memory pool or under a
 * fixed device-memory budget, where an allocation would fail or would synchronise the device.
 * All scratch lives in one array in the library's device image: 4.89 MiB, held by every GPU
 * that loads the library until the process exits, which limits nao to 256.
 * Inputs d_fock and d_overlap (nao*nao, column-major) and outputs d_emo, d_focc (nao) and
 * d_density (nao*nao) are device pointers the caller allocates; d_status (optional, device)
 * receives the molecule's status bits (0 = ok). The work is queued on `stream` (a
 * cudaStream_t; NULL = the legacy default stream) and the call returns without waiting.
 * The first call on a device looks the array's device address up; make that first call before
 * any stream capture. Calls share the one array: calls that overlap on the GPU (other streams,
 * other host threads) race and must be ordered by the caller. Returns AXTB_ERR_INPUT for nao
 * outside 1..256 or bad arguments, AXTB_ERR_DEVICE when the launch fails. */
int axtb_gpu_density_static(const double* d_fock, const double* d_overlap, int32_t nao, double nalpha, double nbeta,
                            double kt, double* d_emo, double* d_focc, double* d_density, int32_t* d_status,
                            void* stream);

#ifdef __cplusplus
}
#endif

#endif /* AXTB_GPU_H */
