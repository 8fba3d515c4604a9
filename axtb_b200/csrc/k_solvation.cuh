// Implicit solvation (ALPB, GBSA) of crates/solvation/src as a charge-dependent SCF term
// (crates/axtb/src/solvation.rs:40-110). Per geometry: SASA neighbour lists, Born radii (GBOBC-II,
// born.rs:103-157), smoothed surface areas on the 230-point Lebedev grid (sasa.rs:31-240) and the
// ALPB shape descriptor (kernel.rs:163-196). Per SCF iteration: the potential B q of the input
// charges and the energy q_i (B q)_i / 2 of the output charges with the Born matrix B evaluated
// pair by pair (P16 or Still kernel, kernel.rs:28-66, H-bond diagonal, ALPB shape term). After the
// SCF: the explicit gradient at fixed charges (kernel.rs:70-160, born.rs:160-216, the surface
// derivatives contracted with surface tension and H-bond weights, kernel.rs:198-238). Every atom's
// result has one writer and a fixed summation order: runs reproduce bit for bit.
#pragma once
#include "common.cuh"
#include "k_geometry.cuh"
#include "params/solvation_tables.h"

namespace axg {

constexpr int SOLV_MAXNB = 512;  // SASA neighbours an atom may have (more: ST_SOLV)
__constant__ double c_lebedev[230][4];

// ---- Born radii: one pair of the integral, atom `hi` > atom `lo` in the reference's order
struct PsiTerm {
    bool on;
    double g, dg;
};
__device__ __forceinline__ PsiTerm psi_nonoverlap(double r, double rho, double r1) {
    double ap = r + rho, am = r - rho, ab = ap * am, rhab = rho / ab;
    double lnab = 0.5 * log(am / ap) * r1;
    return {true, rhab + lnab, -2.0 * rhab / ab + (rhab - lnab) * r1 * r1};
}
__device__ __forceinline__ PsiTerm psi_overlap(double r, double rho, double rvdw) {
    double r1 = 1.0 / r, r12 = 0.5 * r1, r24 = r12 * r12;
    double ap = r + rho, am = r - rho, rh1 = 1.0 / rvdw, rhr1 = 1.0 / ap, aprh1 = ap * rh1;
    double lnab = log(aprh1);
    double g = rh1 - rhr1 + r12 * (0.5 * am * (rhr1 - rh1 * aprh1) - lnab);
    double dg = rhr1 * rhr1 * (1.0 - 0.25 * am * r1 * (1.0 + aprh1 * aprh1)) + rho * r24 * (rhr1 - rh1 * aprh1) +
                r12 * (r1 * lnab - rhr1);
    return {true, g, dg * r1};
}
// the four overlap cases of the pair (hi, lo): ci to psi_hi, cj to psi_lo (r1 = 1/r for every pair)
__device__ __forceinline__ void psi_pair(const Batch& B, int hi, int lo, double r, PsiTerm& ci, PsiTerm& cj) {
    double rhoi = B.sv_rho[hi], rhoj = B.sv_rho[lo], rvi = B.sv_vdwr[hi], rvj = B.sv_vdwr[lo];
    double r1 = 1.0 / r;
    bool ovij = !(r >= rvi + rhoj), ovji = !(r >= rhoi + rvj);
    ci = {false, 0.0, 0.0};
    cj = {false, 0.0, 0.0};
    if (!ovij && !ovji) {
        ci = psi_nonoverlap(r, rhoj, r1);
        cj = fabs(rhoi - rhoj) < 1.0e-8 ? ci : psi_nonoverlap(r, rhoi, r1);
    } else if (!ovij) {
        ci = psi_nonoverlap(r, rhoj, r1);
        if (r + rhoi > rvj) cj = psi_overlap(r, rhoi, rvj);
    } else if (!ovji) {
        if (r + rhoj > rvi) ci = psi_overlap(r, rhoj, rvi);
        cj = psi_nonoverlap(r, rhoi, r1);
    } else {
        if (r + rhoj > rvi) ci = psi_overlap(r, rhoj, rvi);
        if (r + rhoi > rvj) cj = psi_overlap(r, rhoi, rvj);
    }
}

// Born radii and dbrad/dpsi; warp per atom (lanes over the molecule's other atoms)
__global__ void k_solv_born(Batch B, State S) {
    int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (a >= B.natT) return;
    AtomView mv = mol_atoms(B, a);
    double lr2 = B.sv_lrcut * B.sv_lrcut, psi = 0.0;
    for (int b = mv.i0 + lane; b < mv.i0 + mv.n; b += 32) {
        if (b == a) continue;
        double v[3];
        dvec(S.xyz, a, b, v);
        double d2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        if (!(d2 < lr2)) continue;
        PsiTerm ci, cj;
        if (a > b) {
            psi_pair(B, a, b, sqrt(d2), ci, cj);
            if (ci.on) psi += ci.g;
        } else {
            psi_pair(B, b, a, sqrt(d2), ci, cj);
            if (cj.on) psi += cj.g;
        }
    }
    psi = warp_sum(psi);
    if (lane == 0) {
        double s1 = 1.0 / B.sv_svdw[a], v1 = 1.0 / B.sv_vdwr[a], s2 = 0.5 * B.sv_svdw[a];
        double br = psi * s2;
        double arg2 = br * (solvtab::OBC_GAMMA * br - solvtab::OBC_BETA);
        double arg = br * (solvtab::OBC_ALPHA + arg2);
        arg2 = 2.0 * arg2 + solvtab::OBC_ALPHA + solvtab::OBC_GAMMA * br * br;
        double th = tanh(arg), ch = cosh(arg);
        S.sv_brad[a] = 1.0 / (s1 - v1 * th) * B.sv_c1;
        double dpsi = ch * (s1 - v1 * th);
        S.sv_dbrad[a] = s2 * v1 * arg2 / (dpsi * dpsi) * B.sv_c1;
    }
}

// SASA neighbours (ascending) of each atom: r < srcut and r < R_sa,i + R_sa,j + w (sasa.rs:31-70)
__device__ __forceinline__ bool sasa_near(const Batch& B, const State& S, int i, int j, int m) {
    double v[3];
    dvec(S.xyz, i, j, v);
    double d2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    double rmax = B.sv_vdwsa[i] + B.sv_vdwsa[j] + B.sv_w + 1.0e-6;
    return d2 < B.sv_srcut[m] * B.sv_srcut[m] && d2 < rmax * rmax;
}
__global__ void k_solv_neighbours(Batch B, State S) {
    int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (a >= B.natT) return;
    AtomView mv = mol_atoms(B, a);
    int* out = S.sv_nb + (long long)a * SOLV_MAXNB;
    int cnt = 0;
    for (int base = mv.i0; base < mv.i0 + mv.n; base += 32) {
        int b = base + lane;
        bool take = b < mv.i0 + mv.n && b != a && sasa_near(B, S, a, b, mv.m);
        unsigned mask = __ballot_sync(0xffffffffu, take);
        int pos = cnt + __popc(mask & ((1u << lane) - 1u));
        if (take && pos < SOLV_MAXNB) out[pos] = b;
        cnt += __popc(mask);
    }
    if (lane == 0) {
        S.sv_nbn[a] = min(cnt, SOLV_MAXNB);
        if (cnt > SOLV_MAXNB) atomicOr(&S.status[mv.m], ST_SOLV);
    }
}

// the smoothed surface function of grid point xp of atom i (sasa.rs:150-200): its product over
// the neighbours, and for neighbour `want` (or -1) the factor of the derivative g (tj times
// dsasa_ij / (sasa_ij |tj|)); false when the point is buried or below the weight threshold
__device__ __forceinline__ bool sasa_point(const Batch& B, const State& S, int i, const double xp[3], int want,
                                           double& sasap, double gw[3], double gself[3], double wsa_scale) {
    const int* nb = S.sv_nb + (long long)i * SOLV_MAXNB;
    int nno = S.sv_nbn[i];
    for (int s = 0; s < nno; s++) {
        int j = nb[s];
        double dx = xp[0] - S.xyz[3 * j], dy = xp[1] - S.xyz[3 * j + 1], dz = xp[2] - S.xyz[3 * j + 2];
        if (dx * dx + dy * dy + dz * dz <= B.sv_t1[j]) return false;
    }
    sasap = 1.0;
    for (int s = 0; s < nno; s++) {
        int j = nb[s];
        double tj[3] = {xp[0] - S.xyz[3 * j], xp[1] - S.xyz[3 * j + 1], xp[2] - S.xyz[3 * j + 2]};
        double tj2 = tj[0] * tj[0] + tj[1] * tj[1] + tj[2] * tj[2];
        if (!(tj2 < B.sv_t2[j])) continue;
        double sq = sqrt(tj2), uj = sq - B.sv_vdwsa[j], ah3uj2 = B.sv_ah3 * uj * uj;
        double sij = B.sv_ah0 + (B.sv_ah1 + ah3uj2) * uj;
        if (1.0 < sij) sij = 1.0;
        if (0.0 > sij) sij = 0.0;
        if (sij < DBL_MIN) return false;
        sasap *= sij;
    }
    if (!(sasap > solvtab::TOLSESP)) return false;
    // derivative factors (a second pass: the weight needs the whole product)
    for (int s = 0; s < nno; s++) {
        int j = nb[s];
        double tj[3] = {xp[0] - S.xyz[3 * j], xp[1] - S.xyz[3 * j + 1], xp[2] - S.xyz[3 * j + 2]};
        double tj2 = tj[0] * tj[0] + tj[1] * tj[1] + tj[2] * tj[2];
        if (!(tj2 < B.sv_t2[j])) continue;
        double sq = sqrt(tj2), uj = sq - B.sv_vdwsa[j], ah3uj2 = B.sv_ah3 * uj * uj;
        double ds = B.sv_ah1 + 3.0 * ah3uj2;
        double sij = B.sv_ah0 + (B.sv_ah1 + ah3uj2) * uj;
        if (1.0 < sij) sij = 1.0;
        if (0.0 > sij) sij = 0.0;
        ds /= sij * sq;
        double wsa = wsa_scale * sasap;
        for (int k = 0; k < 3; k++) {
            double d = wsa * (ds * tj[k]);
            if (gself) gself[k] += d;
            if (j == want) gw[k] -= d;
        }
    }
    return true;
}

// surface areas, their self derivatives, H-bond weights; warp per atom, lanes over grid points
__global__ void k_solv_sasa(Batch B, State S) {
    int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (a >= B.natT) return;
    double rsa = B.sv_vdwsa[a], wr = B.sv_wrp[a];
    const double* xa = S.xyz + 3 * a;
    double sasa = 0.0, gself[3] = {0.0, 0.0, 0.0};
    for (int p = lane; p < 230; p += 32) {
        const double* g = c_lebedev[p];
        double xp[3] = {xa[0] + rsa * g[0], xa[1] + rsa * g[1], xa[2] + rsa * g[2]};
        double sasap, dummy[3];
        if (!sasa_point(B, S, a, xp, -1, sasap, dummy, gself, g[3] * wr)) continue;
        sasa += g[3] * wr * sasap;
    }
    sasa = warp_sum(sasa);
    for (int k = 0; k < 3; k++) gself[k] = warp_sum(gself[k]);
    if (lane == 0) {
        S.sv_sasa[a] = sasa;
        for (int k = 0; k < 3; k++) S.sv_selfg[3 * a + k] = gself[k];
        double smaxd = 1.0 / (B.sv_vdwsa[a] * B.sv_vdwsa[a]);
        S.sv_hbw[a] = B.sv_hbmag[a] * (sasa * smaxd);
        S.sv_dhbdw[a] = B.sv_hbmag[a] * smaxd;
    }
}

// ALPB shape descriptor A_det per molecule (kernel.rs:107-164); one CTA per molecule, thread 0
__device__ double solv_inertia(const Batch& B, const State& S, int a0, int n, double in[3][3], double c[3]) {
    const double TOF = 2.0 / 5.0;
    double tot = 0.0;
    c[0] = c[1] = c[2] = 0.0;
    for (int i = a0; i < a0 + n; i++) {
        double r = B.sv_vdwr[i], r3 = r * r * r;
        tot += r3;
        for (int k = 0; k < 3; k++) c[k] += S.xyz[3 * i + k] * r3;
    }
    for (int k = 0; k < 3; k++) c[k] /= tot;
    for (int x = 0; x < 3; x++)
        for (int y = 0; y < 3; y++) in[x][y] = 0.0;
    for (int i = a0; i < a0 + n; i++) {
        double r = B.sv_vdwr[i], r2 = r * r, r3 = r2 * r;
        double v[3] = {S.xyz[3 * i] - c[0], S.xyz[3 * i + 1] - c[1], S.xyz[3 * i + 2] - c[2]};
        double d2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        double diag = r3 * (d2 + TOF * r2);
        for (int k = 0; k < 3; k++) in[k][k] += diag;
        for (int col = 0; col < 3; col++)
            for (int row = 0; row < 3; row++) in[row][col] -= r3 * v[col] * v[row];
    }
    return tot;
}
__device__ __forceinline__ double solv_det3(const double a[3][3]) {
    return a[0][0] * a[1][1] * a[2][2] - a[0][0] * a[1][2] * a[2][1] - a[0][1] * a[1][0] * a[2][2] +
           a[0][1] * a[1][2] * a[2][0] + a[0][2] * a[1][0] * a[2][1] - a[0][2] * a[1][1] * a[2][0];
}
__global__ void k_solv_adet(Batch B, State S) {
    int m = blockIdx.x;
    if (m >= B.nmol || threadIdx.x != 0) return;
    double in[3][3], c[3];
    double tot = solv_inertia(B, S, B.m_at0[m], B.m_nat[m], in, c);
    S.sv_adet[m] = B.sv_alpbet > 0.0 ? sqrt(pow(solv_det3(in), 1.0 / 3.0) / ((2.0 / 5.0) * tot)) : 0.0;
}

// Born matrix element B_ij (i != j) without the shape term
__device__ __forceinline__ double born_pair(const Batch& B, double r, double bi, double bj) {
    if (B.sv_alpb) {
        double ab = sqrt(bi * bj);
        double arg = ab / (ab + (solvtab::ZETA_P16 / 16.0) * r);
        arg *= arg;
        arg *= arg;
        arg *= arg;
        arg *= arg;
        return B.sv_keps * (1.0 / (r + ab * arg));
    }
    double r2 = r * r, aa = bi * bj, dd = 0.25 * r2 / aa;
    return B.sv_keps * (1.0 / sqrt(r2 + aa * exp(-dd)));
}

// (B q)_a for charges q; warp per atom, lanes over the molecule's atoms
__device__ __forceinline__ double born_row(const Batch& B, const State& S, int a, const AtomView& mv, const double* q,
                                           int lane) {
    double v = 0.0, qt = 0.0;
    for (int b = mv.i0 + lane; b < mv.i0 + mv.n; b += 32) {
        qt += q[b];
        if (b == a) continue;
        double w[3];
        dvec(S.xyz, a, b, w);
        v += born_pair(B, sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]), S.sv_brad[a], S.sv_brad[b]) * q[b];
    }
    v = warp_sum(v);
    qt = warp_sum(qt);
    v += (B.sv_keps * (1.0 / S.sv_brad[a]) + 2.0 * S.sv_hbw[a]) * q[a];
    if (B.sv_alpbet > 0.0) v += B.sv_keps * B.sv_alpbet / S.sv_adet[mv.m] * qt;
    return v;
}

// potential of the input charges added to the atom potential (after k_potentials)
__global__ void k_solv_potential(Batch B, State S) {
    int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (a >= B.natT) return;
    AtomView mv = mol_atoms(B, a);
    if (S.active[mv.m] == 0) return;
    double v = born_row(B, S, a, mv, S.qat_in, lane);
    if (lane == 0) S.vat[a] += v;
}

// energy of the output charges plus the fixed surface and shift energies, added to the atom's
// electronic energy (after k_energy)
__global__ void k_solv_energy(Batch B, State S) {
    int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (a >= B.natT) return;
    AtomView mv = mol_atoms(B, a);
    if (S.active[mv.m] == 0) return;
    double v = born_row(B, S, a, mv, S.qat_out, lane);
    if (lane == 0) {
        double q = S.qat_out[a];
        double e = q * (0.5 * v) + S.sv_sasa[a] * B.sv_gam[a] + B.sv_gshift / mv.n;
        S.e_atom[a] += e;
        S.sv_eatom[a] = e;
    }
}

// gradient: direct pair terms of 1/2 q^T B q at fixed Born radii and dE/dbrad (times dbrad/dpsi)
__global__ void k_solv_grad_kernel(Batch B, State S) {
    int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (a >= B.natT) return;
    AtomView mv = mol_atoms(B, a);
    const double* q = S.qat_out;
    double g[3] = {0.0, 0.0, 0.0}, de = 0.0, ba = S.sv_brad[a], keps = B.sv_keps;
    for (int b = mv.i0 + lane; b < mv.i0 + mv.n; b += 32) {
        if (b == a) continue;
        double v[3];
        dvec(S.xyz, a, b, v);
        double r = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]), qq = q[a] * q[b], bb = S.sv_brad[b];
        if (B.sv_alpb) {
            double ab = sqrt(ba * bb);
            double a1 = ab / (ab + (solvtab::ZETA_P16 / 16.0) * r), a16 = a1 * a1;
            a16 *= a16;
            a16 *= a16;
            a16 *= a16;
            double dfgb = 1.0 / (r + ab * a16), dfgb2 = dfgb * dfgb;
            double ap = (1.0 - solvtab::ZETA_P16 * a1 * a16) * dfgb2;
            for (int k = 0; k < 3; k++) g[k] -= ap * v[k] * keps / r * qq;
            double bp = -0.5 * (r * solvtab::ZETA_P16 / ab * a1 + 1.0) / ab * a16 * dfgb2;
            de += bb * bp * keps * qq;
        } else {
            double r2 = r * r, aa = ba * bb, dd = 0.25 * r2 / aa, expd = exp(-dd);
            double dfgb2 = 1.0 / (r2 + aa * expd), dfgb = sqrt(dfgb2), dfgb3 = dfgb2 * dfgb * keps;
            double ap = (1.0 - 0.25 * expd) * dfgb3;
            for (int k = 0; k < 3; k++) g[k] -= ap * v[k] * qq;
            de += bb * (-0.5 * expd * (1.0 + dd) * dfgb3) * qq;
        }
    }
    for (int k = 0; k < 3; k++) g[k] = warp_sum(g[k]);
    de = warp_sum(de);
    if (lane == 0) {
        for (int k = 0; k < 3; k++) S.grad[3 * a + k] += g[k];
        double bp = 1.0 / ba, qq = q[a] * bp;
        de += -0.5 * keps * qq * bp * q[a];
        S.sv_dedbr[a] = de * S.sv_dbrad[a];
    }
}

// gradient through the Born radii: sum over pairs of (f_hi dg_hi + f_lo dg_lo) (R_hi - R_lo)
__global__ void k_solv_grad_psi(Batch B, State S) {
    int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (a >= B.natT) return;
    AtomView mv = mol_atoms(B, a);
    double lr2 = B.sv_lrcut * B.sv_lrcut, g[3] = {0.0, 0.0, 0.0};
    for (int b = mv.i0 + lane; b < mv.i0 + mv.n; b += 32) {
        if (b == a) continue;
        double v[3];
        dvec(S.xyz, a, b, v);
        double d2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        if (!(d2 < lr2)) continue;
        int hi = max(a, b), lo = min(a, b);
        PsiTerm ci, cj;
        psi_pair(B, hi, lo, sqrt(d2), ci, cj);
        double s = 0.0;
        if (ci.on) s += S.sv_dedbr[hi] * ci.dg;
        if (cj.on) s += S.sv_dedbr[lo] * cj.dg;
        for (int k = 0; k < 3; k++) g[k] += s * v[k];
    }
    for (int k = 0; k < 3; k++) g[k] = warp_sum(g[k]);
    if (lane == 0)
        for (int k = 0; k < 3; k++) S.grad[3 * a + k] += g[k];
}

// gradient of the surface terms: sum_i c_i d sasa_i / d R_a with c_i = gamma_i + dhbdw_i q_i^2
// (surface tension and H-bond weight); the neighbours' parts recomputed point by point;
// warp per receiving atom a, lanes over grid points
__global__ void k_solv_grad_surface(Batch B, State S) {
    int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (a >= B.natT) return;
    const double* q = S.qat_out;
    double g[3] = {0.0, 0.0, 0.0};
    const int* nb = S.sv_nb + (long long)a * SOLV_MAXNB;
    int nno = S.sv_nbn[a];
    for (int s = 0; s < nno; s++) {
        int i = nb[s];
        double ci = B.sv_gam[i] + S.sv_dhbdw[i] * q[i] * q[i];
        if (ci == 0.0) continue;
        double rsa = B.sv_vdwsa[i], wr = B.sv_wrp[i];
        const double* xi = S.xyz + 3 * i;
        double gi[3] = {0.0, 0.0, 0.0};
        for (int p = lane; p < 230; p += 32) {
            const double* gp = c_lebedev[p];
            double xp[3] = {xi[0] + rsa * gp[0], xi[1] + rsa * gp[1], xi[2] + rsa * gp[2]};
            double sasap;
            sasa_point(B, S, i, xp, a, sasap, gi, nullptr, gp[3] * wr);
        }
        for (int k = 0; k < 3; k++) g[k] += gi[k] * ci;
    }
    for (int k = 0; k < 3; k++) g[k] = warp_sum(g[k]);
    if (lane == 0) {
        double ca = B.sv_gam[a] + S.sv_dhbdw[a] * q[a] * q[a];
        for (int k = 0; k < 3; k++) S.grad[3 * a + k] += g[k] + S.sv_selfg[3 * a + k] * ca;
    }
}

// gradient of the ALPB shape term 1/2 keps alpbet / A_det (sum q)^2; one CTA per molecule
__global__ void k_solv_grad_adet(Batch B, State S) {
    int m = blockIdx.x;
    if (m >= B.nmol || B.sv_alpbet <= 0.0) return;
    int a0 = B.m_at0[m], n = B.m_nat[m];
    __shared__ double d[3][3], c[3];
    if (threadIdx.x == 0) {
        double qt = 0.0;
        for (int i = a0; i < a0 + n; i++) qt += S.qat_out[i];
        double in[3][3];
        double tot = solv_inertia(B, S, a0, n, in, c);
        double adet = sqrt(pow(solv_det3(in), 1.0 / 3.0) / ((2.0 / 5.0) * tot));
        double t2 = tot * tot, a2 = adet * adet;
        double fa = 250.0 / (48.0 * (t2 * tot) * ((a2 * a2) * adet));
        double fb = -0.5 * B.sv_keps * B.sv_alpbet * (qt * qt) / a2;
        double xy = in[0][1] * in[2][2] - in[0][2] * in[1][2];
        double xz = in[0][2] * in[1][1] - in[0][1] * in[2][1];
        double yz = in[0][0] * in[1][2] - in[0][1] * in[0][2];
        double xx = in[0][0] * (in[1][1] + in[2][2]) - in[0][1] * in[0][1] - in[0][2] * in[0][2];
        double yy = in[1][1] * (in[0][0] + in[2][2]) - in[0][1] * in[0][1] - in[1][2] * in[1][2];
        double zz = in[2][2] * (in[0][0] + in[1][1]) - in[0][2] * in[0][2] - in[1][2] * in[1][2];
        double e[3][3] = {{xx, xy, xz}, {xy, yy, yz}, {xz, yz, zz}};
        for (int x = 0; x < 3; x++)
            for (int y = 0; y < 3; y++) d[x][y] = e[x][y] * fa * fb;
    }
    __syncthreads();
    for (int i = a0 + threadIdx.x; i < a0 + n; i += blockDim.x) {
        double r = B.sv_vdwr[i], r3 = r * r * r;
        double v[3] = {S.xyz[3 * i] - c[0], S.xyz[3 * i + 1] - c[1], S.xyz[3 * i + 2] - c[2]};
        for (int k = 0; k < 3; k++) S.grad[3 * i + k] += r3 * (d[k][0] * v[0] + d[k][1] * v[1] + d[k][2] * v[2]);
    }
}

}  // namespace axg
