/* axtb_gpu_debug.h - introspection of a batch after axtb_gpu_batch_run, for kernel-level
 * parity tests. No reference counterpart: axtb's own unit tests reach the same intermediates
 * through crate-internal functions (coordination numbers crates/axtb/src/ncoord.rs:39,
 * AO matrices crates/axtb/src/hamiltonian.rs:77-94, density crates/axtb/src/xtb.rs:1033-1038).
 */
#ifndef AXTB_GPU_DEBUG_H
#define AXTB_GPU_DEBUG_H

#include "axtb_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

enum AxtbDebugQuantity {
    AXTB_DBG_CN = 0,          /* nat GFN2 coordination numbers */
    AXTB_DBG_OVERLAP = 1,     /* nao*nao overlap, column-major */
    AXTB_DBG_H0 = 2,          /* nao*nao core Hamiltonian */
    AXTB_DBG_DIPOLE = 3,      /* 3 planes of nao*nao dipole integrals (about the column AO's atom) */
    AXTB_DBG_QUADRUPOLE = 4,  /* 6 planes of nao*nao traceless quadrupole integrals */
    AXTB_DBG_DENSITY = 5,     /* nao*nao density of the last iteration */
    AXTB_DBG_FOCK = 6,        /* nao*nao last Fock matrix */
    AXTB_DBG_EMO = 7,         /* nao orbital energies */
    AXTB_DBG_FOCC = 8,        /* nao occupations */
    AXTB_DBG_WDENSITY = 9,    /* nao*nao energy-weighted density (after a gradient run) */
    AXTB_DBG_EEQ = 10,        /* nat EEQ start charges */
    AXTB_DBG_LINV = 11,       /* nao*nao inverse Cholesky factor of the overlap */
    AXTB_DBG_EIGEN_CYCLES = 12, /* 1 value: SM clock cycles of the molecule's last eigen phase
                                   (runs with profiling on; 0 otherwise) */
    AXTB_DBG_STATUS_BITS = 13,  /* 1 value: the molecule's raw status bits of its last attempt
                                   (1 overlap/EEQ not positive definite, 2 non-finite energy,
                                   4 Fermi level lost, 8 mixer failed, 16 non-finite
                                   inverse-iteration vector, 32 Broyden history full, 64 a
                                   bounded device wait gave up, 128 non-finite Fock matrix) */
};

/* Per-kernel timing: with profiling on, every kernel launch of a run is bracketed by CUDA
 * events on the batch's stream; axtb_gpu_batch_profile writes a JSON object with, per kernel,
 * launches, milliseconds, algorithmic FLOPs and bytes, plus the host<->device bytes of the
 * public-API runs. Enabling resets the counters. Returns the JSON length. */
int axtb_gpu_batch_set_profiling(AxtbBatch* b, int32_t enable);
int axtb_gpu_batch_profile(const AxtbBatch* b, char* buf, size_t len);

/* Copy quantity `what` of molecule `mol` of the last run into host memory `out`. */
int axtb_gpu_batch_debug(AxtbBatch* b, int32_t mol, int32_t what, double* out);

#ifdef __cplusplus
}
#endif

#endif /* AXTB_GPU_DEBUG_H */
