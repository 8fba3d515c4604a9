// The cooperative per-molecule dense algebra kernel. Large molecules (team = the whole grid)
// are processed first, one after the other; then every CTA works through its own list of small
// molecules (team = that CTA). Phases:
//   PH_OVERLAP  Cholesky of S and L^-1 (once per geometry; crates/base/src/linalg/eigen.rs:72-113)
//   PH_EEQ      EEQ start charges from the Cholesky factor of the EEQ matrix
//               (crates/axtb/src/eeq.rs:43-77, bordered system solved by its Schur complement)
//   PH_EIGEN    F' = L^-1 F L^-T, eigenvalues, tblite Fermi filling, occupied eigenvectors,
//               C = L^-T Q Z and P = C f C^T (crates/axtb/src/xtb.rs:997-1038); for a molecule
//               whose band is chased on chip (k_chase) only F' and stage 1 of the reduction
//   PH_EIGEN_TAIL  the rest of those molecules' eigen phase, after k_chase
//   PH_WDENS    W = C (f e) C^T (crates/axtb/src/xtb.rs:688-696)
//   PH_LEVELS   the orbital energies above the ones the SCF needed, from the last tridiagonal
//               matrix (all levels, as the reference's eigensolver returns them for the result)
#pragma once
#include "common.cuh"
#include "team_la.cuh"
#include "team_band.cuh"

namespace axg {

enum { PH_OVERLAP = 0, PH_EEQ = 1, PH_EIGEN = 2, PH_WDENS = 3, PH_LEVELS = 4, PH_EIGEN_TAIL = 5 };

struct TeamPlan {
    const int* big;        // molecules run by the whole grid
    int nbig;
    const int* small_off;  // per CTA: range into small_list
    const int* small_list;
    const int* head_off;   // the same for PH_EIGEN (balanced on its own cost model) ...
    const int* head_list;
    const int* tail_off;   // ... and for PH_EIGEN_TAIL
    const int* tail_list;
    const long long* m_wk0;   // per-molecule workspace offsets into wk
    double* wk;
    const long long* m_sq0;   // per-molecule nat^2 offsets (EEQ planes)
    double* eeq_rhs;          // natT
    double* eeq_q;            // natT: EEQ charges
    long long eeq_plane;      // size of one EEQ plane (sum nat^2)
    int cycles;               // 1: accumulate per-phase SM cycles of mol_eigen into g_team_cycles
};

// per-phase cycle counters of the eigen phase (g_team_cycles, instrumentation read by the profiler)
#define TEAM_PHASE(k)                                                  \
    do {                                                               \
        if (P.cycles && t.tid() == 0) {                                \
            long long now__ = clock64();                               \
            atomicAdd(&g_team_cycles[k], (unsigned long long)(now__ - t0__)); \
            t0__ = now__;                                              \
        }                                                              \
    } while (0)

__device__ void mol_overlap(const Team& t, const Batch& B, State& S, const TeamPlan& P, int m) {
    int n = B.m_nao[m];
    long long mat = B.m_mat0[m];
    double* L = S.scr1 + mat;
    for (long long e = t.tid(); e < (long long)n * n; e += t.nthreads()) L[e] = S.S[mat + e];
    t.sync();
    double* tmp = P.wk + P.m_wk0[m];
    bool ok = team_cholesky(t, L, n, n, tmp);
    if (!ok && t.tid() == 0) atomicOr(&S.status[m], ST_NOT_PD);
    team_trinv(t, L, n, S.Linv + mat, n, n, tmp);
}

__device__ void mol_eeq(const Team& t, const Batch& B, State& S, const TeamPlan& P, int m) {
    int n = B.m_nat[m], a0 = B.m_at0[m];
    long long o = P.m_sq0[m];
    double* A = S.eeq_A + o;
    double* Li = S.eeq_A + P.eeq_plane + o;
    double* Ji = S.eeq_A + 2 * P.eeq_plane + o;
    double* tmp = P.wk + P.m_wk0[m];
    bool ok = team_cholesky(t, A, n, n, tmp);
    team_trinv(t, A, n, Li, n, n, tmp);
    // J^-1 = L^-T L^-1
    team_gemm(t, true, false, n, n, n, 1.0, Li, n, Li, n, 0.0, Ji, n);
    t.sync();
    // a = J^-1 x, b = J^-1 1 (J^-1 symmetric: row i = column i)
    double sa = 0.0, sb = 0.0;
    for (int i = t.tid(); i < n; i += t.nthreads()) {
        double va = 0.0, vb = 0.0;
        for (int c = 0; c < n; c++) {
            double j = Ji[c + (long long)i * n];
            va += j * P.eeq_rhs[a0 + c];
            vb += j;
        }
        P.eeq_q[a0 + i] = va;
        tmp[i] = vb;
        sa += va;
        sb += vb;
    }
    sa = team_sum(t, sa, S.red);
    sb = team_sum(t, sb, S.red);
    double lam = (sa - B.m_charge[m]) / sb;
    for (int i = t.tid(); i < n; i += t.nthreads()) {
        double q = P.eeq_q[a0 + i] - lam * tmp[i];
        if (!ok || !isfinite(q)) q = 0.0;  // neutral-atom start when the EEQ system fails
        P.eeq_q[a0 + i] = q;
    }
    t.sync();
}

// tblite Fermi filling of both spins (warp 0 of the team's first CTA): focc = f_alpha + f_beta,
// kocc, -TS; *more = 1 when only kc levels are true eigenvalues (kc < n) and level kc - 1 still
// holds more than 1e-16 electrons of either spin. Ends with a team barrier.
__device__ void mol_fermi(const Team& t, const Batch& B, State& S, int m, const double* emo, int n, double* focc,
                          double* occb, int kc, double* more) {
    if (t.rank == 0 && threadIdx.x < 32) {
        double efa, efb;
        warp_fill(B.m_nalpha[m], B.kt, emo, n, focc, &efa);
        warp_fill(B.m_nbeta[m], B.kt, emo, n, occb, &efb);
        int lane = threadIdx.x;
        double pa = 0.0, pb = 0.0, ts = 0.0, flast = 0.0;
        int kl = 0;
        double* falpha = S.focc_a ? S.focc_a + B.m_ao0[m] : nullptr;
        for (int i = lane; i < n; i += 32) {
            double fa = focc[i], fb = occb[i];
            if (falpha) falpha[i] = fa;
            pa += fa;
            pb += fb;
            if (B.kt > 0.0) ts += log(pow(fa, fa) * pow(1.0 - fa, 1.0 - fa)) + log(pow(fb, fb) * pow(1.0 - fb, 1.0 - fb));
            if (i == kc - 1) flast = fmax(fa, fb);
            double f = fa + fb;
            focc[i] = f;
            if (f > 1e-16) kl = max(kl, i + 1);
        }
        pa = warp_sum(pa);
        pb = warp_sum(pb);
        ts = warp_sum(ts);
        for (int o = 16; o > 0; o >>= 1) {
            kl = max(kl, __shfl_xor_sync(0xffffffffu, kl, o));
            flast = fmax(flast, __shfl_xor_sync(0xffffffffu, flast, o));
        }
        if (lane == 0) {
            S.kocc[m] = kl;
            S.ts[m] = ts * B.kt;
            if (S.efermi) {  // the Fermi levels, NaN where the filling is aufbau (0 K, no electrons)
                bool fa = B.kt > 0.0 && B.m_nalpha[m] > 0.0, fb = B.kt > 0.0 && B.m_nbeta[m] > 0.0;
                S.efermi[2 * m] = fa ? efa : __longlong_as_double(0x7ff8000000000000LL);
                S.efermi[2 * m + 1] = fb ? efb : __longlong_as_double(0x7ff8000000000000LL);
            }
            *more = (kc < n && flast > 1e-16) ? 1.0 : 0.0;
            if (fabs(pa - B.m_nalpha[m]) > 1e-6 || fabs(pb - B.m_nbeta[m]) > 1e-6) atomicOr(&S.status[m], ST_FERMI);
        }
    }
    t.sync();
}

// the two-stage reduction needs a band stage: a matrix of at most BW + 1 rows already is a band,
// and the one-stage path keeps the bits that small chaotic SCFs follow
__device__ __forceinline__ bool two_stage(const Team& t, const Batch& B, int n) {
    return !t.global && n > BW + 1 && n < B.band_max;
}
// stage 2 of the two-stage reduction in its own launch with the band in shared memory (k_chase)
__device__ __forceinline__ bool chased_on_chip(const Team& t, const Batch& B, int n) {
    return two_stage(t, B, n) && n <= B.chase_max;
}

// after_chase: the part after k_chase of a molecule whose bulge chasing ran on chip (from its
// tridiagonal matrix on); otherwise the whole eigen phase, or for such a molecule the part before
// GRID_ROWS: the whole-grid instance (k_team_grid), whose tridiagonal reduction sums the symv rows
// warp by warp (grid_symv_combine); k_team and the allocation-free entry point use the other
template <bool GRID_ROWS = false>
__device__ void mol_eigen(const Team& t, const Batch& B, State& S, const TeamPlan& P, int m, bool after_chase) {
    int n = B.m_nao[m], ao0 = B.m_ao0[m];
    long long mat = B.m_mat0[m];
    double* wk = P.wk + P.m_wk0[m];
    double* Linv = S.Linv + mat;
    double* X = S.scr1 + mat;
    double* Fp = S.Fp + mat;
    long long t0__ = clock64(), tstart = t0__;
    double* d = S.dtri + ao0;
    double* e = S.etri + ao0;
    double* tau = S.tau + ao0;
    const int nsl = symv_slots(n);
    const bool band = two_stage(t, B, n);
    if (!after_chase) {
    // F' = L^-1 F L^-T (L^-1 is lower triangular; F' is symmetric and only its lower triangle is
    // used: the tiles on and below the diagonal are computed)
    // split precision for the basis transform only: an error there perturbs F', whose exactly
    // orthonormal FP64 eigenvectors move the variational energy at second order; C and P stay
    // FP64 (rounding in P would break its idempotency and enter the energy at first order)
    const int sp = B.split ? GEMM_SPLIT : 0;
    team_gemm(t, false, false, n, n, n, 1.0, Linv, n, S.F + mat, n, 0.0, X, n, GEMM_A_LOWER | sp);
    t.sync();
    team_gemm(t, false, true, n, n, n, 1.0, X, n, Linv, n, 0.0, Fp, n, GEMM_B_UPPER | GEMM_LOWER_TILES | sp);
    t.sync();
    TEAM_PHASE(0);
    double* vbuf = wk;
    double* pbuf = wk + n;
    double* ppart = wk + 2 * n;
    if (band) {
        // one CTA: two-stage reduction (dense -> band on GEMMs, band -> tridiagonal by bulge
        // chasing), the stage-2 reflectors in the W plane (free until the gradient's W)
        team_sy2sb(t, Fp, n, n, tau, wk);
        TEAM_PHASE(16);
        if (n <= B.chase_max) {  // stage 2 and the rest in the next two launches
            if (P.cycles && t.tid() == 0) S.mol_cyc[m] = (double)(clock64() - tstart);
            return;
        }
        team_sb2st(t, Fp, n, n, d, e, wk, S.W + mat);
        TEAM_PHASE(17);
    } else {
        double* Vp = wk + 2 * n + (long long)nsl * n;  // the back-transform's vb area (64 n)
        team_tridiag_blocked<GRID_ROWS>(t, Fp, n, n, d, e, tau, Vp, Vp + (long long)NBP * n, vbuf, pbuf, ppart, S.red,
                                        P.cycles != 0);
        if (P.cycles && t.tid() == 0) t0__ = clock64();  // the tridiagonal's parts were counted in 8..13
    }
    TEAM_PHASE(1);
    }
    double* emo = S.emo + ao0;
    // eigenvalues: the lowest ceil(n_occ) + a margin first; the levels above get the Gershgorin
    // bound (occupation exactly 0 at any sensible kT). If the highest computed level still holds
    // more than 1e-16 electrons (small gap, high temperature), the rest are computed and the
    // filling is redone, so every level with f > 1e-16 is a true eigenvalue.
    team_gershgorin(t, d, e, n, wk);
    int kc = min(n, (int)ceil(fmax(B.m_nalpha[m], B.m_nbeta[m])) + max(16, n / 16));
    team_bisect(t, d, e, n, emo, wk, 0, kc);
    for (int q = kc + t.tid(); q < n; q += t.nthreads()) emo[q] = wk[1];
    t.sync();
    TEAM_PHASE(2);
    double* focc = S.focc + ao0;
    double* occb = wk + 8;  // n entries
    mol_fermi(t, B, S, m, emo, n, focc, occb, kc, wk + 3);
    if (wk[3] != 0.0) {
        team_bisect(t, d, e, n, emo, wk, kc, n);
        TEAM_PHASE(2);
        mol_fermi(t, B, S, m, emo, n, focc, occb, n, wk + 3);
    }
    TEAM_PHASE(3);
    int k = S.kocc[m];
    double* Zm = S.Z + mat;
    team_invit(t, d, e, emo, n, k, Zm, n, S.scr1 + mat, S.scr2 + mat, S.scr3 + mat, S.piv + mat, S.P + mat, &S.status[m]);
    TEAM_PHASE(4);
    // back-transform: vb (n x 64), tb, gm (64 x 64), y, y2 (64 x k)
    double* vb = wk + 2 * n + (long long)nsl * n;
    double* tb = vb + 64LL * n;
    double* gm = tb + 64 * 64;
    double* y = gm + 64 * 64;
    double* y2 = y + 64LL * n;
    if (band) {
        team_apply_q2(t, n, k, Zm, n, S.W + mat, wk);
        TEAM_PHASE(18);
        team_apply_q1(t, Fp, n, n, k, Zm, n, wk);
        TEAM_PHASE(19);
    } else {
        team_backtransform(t, Fp, n, tau, n, k, Zm, n, vb, tb, gm, y, y2);
    }
    TEAM_PHASE(5);
    // C = L^-T Z'; P = (C f) C^T
    double* Cm = S.C + mat;
    team_gemm(t, true, false, n, k, n, 1.0, Linv, n, Zm, n, 0.0, Cm, n, GEMM_A_UPPER);
    t.sync();
    TEAM_PHASE(6);
    double* Cf = S.scr1 + mat;
    for (long long q = t.tid(); q < (long long)n * k; q += t.nthreads()) Cf[q] = Cm[q] * focc[q / n];
    t.sync();
    team_gemm(t, false, true, n, n, k, 1.0, Cf, n, Cm, n, 0.0, S.P + mat, n, GEMM_LOWER_TILES);
    t.sync();
    team_mirror_lower(t, S.P + mat, n, 0, n);
    t.sync();
    TEAM_PHASE(7);
    if (P.cycles && t.tid() == 0) {
        double c = (double)(clock64() - tstart);
        if (after_chase) S.mol_cyc[m] += c;  // after the part before and the chase
        else S.mol_cyc[m] = c;
    }
}

__device__ void mol_wdens(const Team& t, const Batch& B, State& S, const TeamPlan& P, int m) {
    int n = B.m_nao[m], ao0 = B.m_ao0[m], k = S.kocc[m];
    long long mat = B.m_mat0[m];
    double* Cm = S.C + mat;
    double* Cf = S.scr1 + mat;
    for (long long q = t.tid(); q < (long long)n * k; q += t.nthreads()) {
        int c = (int)(q / n);
        Cf[q] = Cm[q] * (S.focc[ao0 + c] * S.emo[ao0 + c]);
    }
    t.sync();
    team_gemm(t, false, true, n, n, k, 1.0, Cf, n, Cm, n, 0.0, S.W + mat, n, GEMM_LOWER_TILES | (B.split ? GEMM_SPLIT : 0));
    t.sync();
    team_mirror_lower(t, S.W + mat, n, 0, n);
    t.sync();
}

// Every orbital energy of the last eigen phase: the SCF bisects only the lowest
// ceil(n_occ) + max(16, n/16) levels of the tridiagonal matrix (or all of them), the rest
// holding the Gershgorin bound; this bisects the rest of the same (d, e).
__device__ void mol_levels(const Team& t, const Batch& B, State& S, const TeamPlan& P, int m) {
    int n = B.m_nao[m], ao0 = B.m_ao0[m];
    double* wk = P.wk + P.m_wk0[m];
    const double* d = S.dtri + ao0;
    const double* e = S.etri + ao0;
    int kc = min(n, (int)ceil(fmax(B.m_nalpha[m], B.m_nbeta[m])) + max(16, n / 16));
    if (kc >= n) return;
    team_gershgorin(t, d, e, n, wk);
    team_bisect(t, d, e, n, S.emo + ao0, wk, kc, n);
}

__device__ __forceinline__ bool phase_wants(const State& S, int phase, int m) {
    if (phase == PH_EIGEN || phase == PH_EIGEN_TAIL) return S.active[m] != 0;
    if (phase == PH_WDENS) return S.conv[m] != 0;
    return true;
}

template <bool GRID_ROWS>
__device__ void run_mol(const Team& t, const Batch& B, State& S, const TeamPlan& P, int phase, int m) {
    switch (phase) {
        case PH_OVERLAP: mol_overlap(t, B, S, P, m); break;
        case PH_EEQ: mol_eeq(t, B, S, P, m); break;
        case PH_EIGEN:
        case PH_EIGEN_TAIL:
            if (phase == PH_EIGEN || chased_on_chip(t, B, B.m_nao[m])) mol_eigen<GRID_ROWS>(t, B, S, P, m, phase == PH_EIGEN_TAIL);
            break;
        case PH_WDENS: mol_wdens(t, B, S, P, m); break;
        case PH_LEVELS: mol_levels(t, B, S, P, m); break;
    }
}

__global__ void __launch_bounds__(TEAM_THREADS, 2) k_team(Batch B, State S, TeamPlan P, int phase) {
    if (threadIdx.x == 0) s_team_gen = 0;
    __syncthreads();
    Team g{(int)blockIdx.x, (int)gridDim.x, true};
    for (int i = 0; i < P.nbig; i++) {
        int m = P.big[i];
        if (phase_wants(S, phase, m)) run_mol<false>(g, B, S, P, phase, m);  // uniform across the grid
    }
    Team one{0, 1, false};
    const int* off = phase == PH_EIGEN ? P.head_off : phase == PH_EIGEN_TAIL ? P.tail_off : P.small_off;
    const int* list = phase == PH_EIGEN ? P.head_list : phase == PH_EIGEN_TAIL ? P.tail_list : P.small_list;
    for (int i = off[blockIdx.x]; i < off[blockIdx.x + 1]; i++) {
        int m = list[i];
        if (phase_wants(S, phase, m)) run_mol<false>(one, B, S, P, phase, m);
    }
}

// The whole-grid molecules (P.big) of a phase, one after the other on the whole cooperative grid.
// A batch that holds such molecules runs this launch first and then k_team for the rest (with
// nbig = 0): the grid path gets its own instance of the dense algebra, and the one-CTA path's
// kernel is compiled without the grid-only code.
__global__ void __launch_bounds__(TEAM_THREADS, 2) k_team_grid(Batch B, State S, TeamPlan P, int phase) {
    if (threadIdx.x == 0) s_team_gen = 0;
    __syncthreads();
    Team g{(int)blockIdx.x, (int)gridDim.x, true};
    for (int i = 0; i < P.nbig; i++) {
        int m = P.big[i];
        if (phase_wants(S, phase, m)) run_mol<true>(g, B, S, P, phase, m);  // uniform across the grid
    }
}

}  // namespace axg
