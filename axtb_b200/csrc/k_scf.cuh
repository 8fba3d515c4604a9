// Kernels of one SCF iteration over a batch (inactive molecules skip their work):
// potentials of the input moments (ES2, ES3, AES2, self-consistent D4), the Fock matrix,
// Mulliken moments of the new density with the band energy, the energy of the output moments,
// and the convergence test with the next input by modified Broyden or DIIS mixing. Then the
// pair terms of the gradient.
#pragma once
#include "common.cuh"
#include "k_geometry.cuh"
#include "k_integrals.cuh"

namespace axg {

constexpr double SQRT2 = 1.4142135623730951;
__constant__ double QSCALE[6] = {1.0, 2.0, 1.0, 2.0, 2.0, 1.0};
__constant__ int QOFF[6] = {0, 1, 0, 1, 1, 0};

__device__ __forceinline__ bool mol_active(const State& S, int m) { return S.active[m] != 0; }

// ES2 kernel element (crates/axtb/src/coulomb.rs:61-119, g = 2); same atom: eta
__device__ __forceinline__ double gamma_el(const Batch& B, const double* x, int sa, int sb) {
    int a = B.s_at[sa], b = B.s_at[sb];
    double eta = 0.5 * (B.s_hard[sa] + B.s_hard[sb]);
    if (a == b) return eta;
    double v[3];
    dvec(x, a, b, v);
    double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    return 1.0 / sqrt(r2 + 1.0 / (eta * eta));
}

// the shell gamma matrix of each molecule's geometry (crates/axtb/src/coulomb.rs:61-119), made once
// per run and read by every SCC iteration's potentials and energies: thread per element
__global__ void k_gamma(Batch B, State S, long long ngam) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ngam) return;
    int m = find_mol(B.m_gam0, B.nmol, g);
    int nsh = B.m_nsh[m], sh0 = B.m_sh0[m];
    long long l = g - B.m_gam0[m];
    int s = (int)(l / nsh), t = (int)(l - (long long)s * nsh);
    S.gam[g] = gamma_el(B, S.xyz, sh0 + s, sh0 + t);
}

// AES pair factors g3 = f3/r^3, g5 = f5/r^5 (crates/axtb/src/coulomb.rs:382-394)
__device__ __forceinline__ void aes_g35(const State& S, int a, int b, double r2, double& g3, double& g5) {
    double r1 = sqrt(r2), g1 = 1.0 / r1;
    double gg3 = g1 * g1 * g1, gg5 = gg3 * g1 * g1;
    double rr = 0.5 * (S.mrad[b] + S.mrad[a]) * g1;
    double rr3 = rr * rr * rr;
    g3 = gg3 * (1.0 / (1.0 + 6.0 * rr3));
    g5 = gg5 * (1.0 / (1.0 + 6.0 * rr3 * rr));
}

// AES potential terms of partner b at atom a (crates/axtb/src/coulomb.rs:407-502) for the moments
// (qat, dp, qp), w = R_a - R_b: added to the atom, dipole and quadrupole potentials of a
__device__ __forceinline__ void aes_pair_potential(const State& S, int a, int b, const double* qat, const double* dp,
                                                   const double* qp, const double w[3], double r2, double& va,
                                                   double vd[3], double vq[6]) {
    double g3, g5;
    aes_g35(S, a, b, r2, g3, g5);
    const double* mb = dp + 3 * b;
    double qb = qat[b];
    double mbw = mb[0] * w[0] + mb[1] * w[1] + mb[2] * w[2];
    va += mbw * g3;
    for (int k = 0; k < 3; k++) vd[k] += -w[k] * g3 * qb + g5 * (r2 * mb[k] - 3.0 * w[k] * mbw);
    double tc[6] = {w[0] * w[0], w[0] * w[1], w[1] * w[1], w[0] * w[2], w[1] * w[2], w[2] * w[2]};
    double thb = 0.0;
    for (int k = 0; k < 6; k++) {
        double t = QSCALE[k] * tc[k] * g5;
        vq[k] += t * qb;
        thb += t * qp[6 * b + k];
    }
    va += thb;
}

// potentials of the input moments: warp per atom (shell potentials of the atom's shells, atom,
// dipole and quadrupole potentials); crates/axtb/src/xtb.rs:316-340 with coulomb.rs:407-502,
// 1006-1021, 1141-1143 and crates/d4/src/disp.rs:420-455
__global__ void k_potentials(Batch B, State S) {
    int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (a >= B.natT) return;
    AtomView mv = mol_atoms(B, a);
    if (!mol_active(S, mv.m)) return;
    const double* x = S.xyz;
    int sh0 = B.m_sh0[mv.m], nsh = B.m_nsh[mv.m];
    // ES2 + ES3 for the shells of atom a
    for (int s = B.a_sh0[a]; s < B.a_sh0[a] + B.a_nsh[a]; s++) {
        double v = 0.0;
        const double* gs = S.gam + B.m_gam0[mv.m] + (long long)(s - sh0) * nsh - sh0;
        for (int t = sh0 + lane; t < sh0 + nsh; t += 32) v += gs[t] * S.qsh_in[t];
        v = warp_sum(v);
        if (lane == 0) S.vsh[s] = v + S.qsh_in[s] * S.qsh_in[s] * B.s_gam3[s];
    }
    // AES and D4 atom potentials
    double va = 0.0, vd[3] = {0, 0, 0}, vq[6] = {0, 0, 0, 0, 0, 0};
    int spa = B.a_sp[a];
    for (int b = mv.i0 + lane; b < mv.i0 + mv.n; b += 32) {
        if (b == a) continue;
        double w[3];
        dvec(x, a, b, w);
        double r2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
        aes_pair_potential(S, a, b, S.qat_in, S.dp_in, S.qp_in, w, r2, va, vd, vq);
        // D4: -dC6/dq_a * pair factor
        double pe, pg;
        if (d4_pair(B, spa, B.a_sp[b], r2, pe, pg)) {
            double c6, da, db;
            pair_c6(B, S, a, b, c6, da, db);
            va -= da * pe;
        }
    }
    va = warp_sum(va);
    for (int k = 0; k < 3; k++) vd[k] = warp_sum(vd[k]);
    for (int k = 0; k < 6; k++) vq[k] = warp_sum(vq[k]);
    if (lane == 0) {
        S.vat[a] = va;
        for (int k = 0; k < 3; k++) S.vdp[3 * a + k] = vd[k] + 2.0 * B.a_dk[a] * S.dp_in[3 * a + k];
        for (int k = 0; k < 6; k++) S.vqp[6 * a + k] = vq[k] + 2.0 * B.a_qk[a] * S.qp_in[6 * a + k] * QSCALE[k];
    }
}

// potentials of the gradient in the xtb 6.8.0 conventions (SccGradient::OutputAes,
// crates/axtb/src/xtb.rs:700-722): the dipole and quadrupole potentials of the output moments,
// and the atom potential of the last Fock matrix shifted by the AES atom potential of the output
// moments minus that of the last input moments; warp per atom
__global__ void k_gradient_potentials_aes(Batch B, State S) {
    int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (a >= B.natT) return;
    AtomView mv = mol_atoms(B, a);
    const double* x = S.xyz;
    double vo = 0.0, vi = 0.0, vd[3] = {0, 0, 0}, vq[6] = {0, 0, 0, 0, 0, 0};
    double vdi[3] = {0, 0, 0}, vqi[6] = {0, 0, 0, 0, 0, 0};
    for (int b = mv.i0 + lane; b < mv.i0 + mv.n; b += 32) {
        if (b == a) continue;
        double w[3];
        dvec(x, a, b, w);
        double r2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
        aes_pair_potential(S, a, b, S.qat_out, S.dp_out, S.qp_out, w, r2, vo, vd, vq);
        aes_pair_potential(S, a, b, S.qat_in, S.dp_in, S.qp_in, w, r2, vi, vdi, vqi);
    }
    vo = warp_sum(vo);
    vi = warp_sum(vi);
    for (int k = 0; k < 3; k++) vd[k] = warp_sum(vd[k]);
    for (int k = 0; k < 6; k++) vq[k] = warp_sum(vq[k]);
    if (lane == 0) {
        S.vat[a] += vo - vi;
        for (int k = 0; k < 3; k++) S.vdp[3 * a + k] = vd[k] + 2.0 * B.a_dk[a] * S.dp_out[3 * a + k];
        for (int k = 0; k < 6; k++) S.vqp[6 * a + k] = vq[k] + 2.0 * B.a_qk[a] * S.qp_out[6 * a + k] * QSCALE[k];
    }
}

// Fock matrix F = H0 - (B + B^T)/2, B(mu,nu) = S v_ao(nu) + D.v_d(A_nu) + Q.v_q(A_nu)
// (crates/axtb/src/scf/fock.rs:22-104). One 32x32 tile per CTA (32x8 threads), the transposed
// half of each pair of elements staged through shared memory.
__device__ __forceinline__ double bterm(const Batch& B, const State& S, long long e, int ao_col) {
    int at = B.o_at[ao_col];
    double v = S.vsh[B.o_sh[ao_col]] + S.vat[at];
    long long nn = B.nnT;
    double x = S.S[e] * v;
    for (int k = 0; k < 3; k++) x += S.D[k * nn + e] * S.vdp[3 * at + k];
    for (int k = 0; k < 6; k++) x += S.Q[k * nn + e] * S.vqp[6 * at + k];
    return x;
}

// F = H0 - (B + B^T)/2 by pairs of 32 x 32 tiles (I, J) and (J, I), I >= J: each element's B
// term is formed once (both tiles' B in shared memory), each matrix read once and F written once
__global__ void k_fock(Batch B, State S, const long long* m_tile0, long long ntiles) {
    __shared__ double ba[32][33], bb[32][33];  // ba[b][a] = B(I + a, J + b), bb[b][a] = B(J + a, I + b)
    long long tile = blockIdx.x;
    if (tile >= ntiles) return;
    int m = find_mol(m_tile0, B.nmol, tile);
    if (!mol_active(S, m)) return;
    int n = B.m_nao[m], ao0 = B.m_ao0[m];
    long long lt = tile - m_tile0[m];
    // lt = I (I + 1) / 2 + J, J <= I
    int ti = (int)((sqrt(8.0 * (double)lt + 1.0) - 1.0) * 0.5);
    while ((long long)(ti + 1) * (ti + 2) / 2 <= lt) ti++;
    while ((long long)ti * (ti + 1) / 2 > lt) ti--;
    int tj = (int)(lt - (long long)ti * (ti + 1) / 2);
    const bool diag = ti == tj;
    long long mat = B.m_mat0[m];
    int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int b = ty; b < 32; b += 8) {
        int row = ti * 32 + tx, col = tj * 32 + b;
        ba[b][tx] = (row < n && col < n) ? bterm(B, S, mat + row + (long long)col * n, ao0 + col) : 0.0;
        if (!diag) {
            int row2 = tj * 32 + tx, col2 = ti * 32 + b;
            bb[b][tx] = (row2 < n && col2 < n) ? bterm(B, S, mat + row2 + (long long)col2 * n, ao0 + col2) : 0.0;
        }
    }
    __syncthreads();
    // tile (I, J): B^T from the other tile (the diagonal tile from itself)
    for (int b = ty; b < 32; b += 8) {
        int row = ti * 32 + tx, col = tj * 32 + b;
        if (row >= n || col >= n) continue;
        long long e = mat + row + (long long)col * n;
        double f = S.H0[e] - 0.5 * (ba[b][tx] + (diag ? ba[tx][b] : bb[tx][b]));
        if (!isfinite(f)) atomicOr(&S.status[m], ST_FOCK);
        S.F[e] = f;
    }
    if (diag) return;
    for (int b = ty; b < 32; b += 8) {
        int row = tj * 32 + tx, col = ti * 32 + b;
        if (row >= n || col >= n) continue;
        long long e = mat + row + (long long)col * n;
        double f = S.H0[e] - 0.5 * (bb[b][tx] + ba[tx][b]);
        if (!isfinite(f)) atomicOr(&S.status[m], ST_FOCK);
        S.F[e] = f;
    }
}

// Mulliken column dots (crates/axtb/src/scf/mulliken.rs:19-59) and the band energy column
// (crates/axtb/src/xtb.rs:1129-1135): warp per AO column; out[nu*11 + k]
__global__ void k_mulliken(Batch B, State S) {
    int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (g >= B.naoT) return;
    int at = B.o_at[g], m = B.a_mol[at];
    if (!mol_active(S, m)) return;
    int n = B.m_nao[m], nu = g - B.m_ao0[m];
    long long col = B.m_mat0[m] + (long long)nu * n, nn = B.nnT;
    double r[11];
    for (int k = 0; k < 11; k++) r[k] = 0.0;
    for (int mu = lane; mu < n; mu += 32) {
        long long e = col + mu;
        double p = S.P[e];
        r[0] += p * S.S[e];
        for (int k = 0; k < 3; k++) r[1 + k] += p * S.D[k * nn + e];
        for (int k = 0; k < 6; k++) r[4 + k] += p * S.Q[k * nn + e];
        r[10] += p * S.H0[e];
    }
    for (int k = 0; k < 11; k++) r[k] = warp_sum(r[k]);
    if (lane == 0)
        for (int k = 0; k < 11; k++) S.ao_part[(long long)g * 11 + k] = r[k];
}

// output moments from the column dots: thread per atom (its shells and AOs in order)
__global__ void k_moments(Batch B, State S) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= B.natT) return;
    int m = B.a_mol[a];
    if (!mol_active(S, m)) return;
    double dp[3] = {0, 0, 0}, qp[6] = {0, 0, 0, 0, 0, 0}, qa = 0.0, band = 0.0;
    for (int s = B.a_sh0[a]; s < B.a_sh0[a] + B.a_nsh[a]; s++) {
        double q = B.s_refocc[s];
        for (int o = B.s_ao0[s]; o < B.s_ao0[s] + 2 * B.s_l[s] + 1; o++) {
            const double* r = S.ao_part + (long long)o * 11;
            q -= r[0];
            for (int k = 0; k < 3; k++) dp[k] -= r[1 + k];
            for (int k = 0; k < 6; k++) qp[k] -= r[4 + k];
            band += r[10];
        }
        S.qsh_out[s] = q;
        qa += q;
    }
    S.qat_out[a] = qa;
    for (int k = 0; k < 3; k++) S.dp_out[3 * a + k] = dp[k];
    for (int k = 0; k < 6; k++) S.qp_out[6 * a + k] = qp[k];
    S.e_atom[a] = band;  // band part of the atom's electronic energy; the rest is added next
    S.e_terms[5 * a + 4] = band;
}

// electronic energy per atom of the output moments (crates/axtb/src/xtb.rs:1058-1146): ES2 and
// ES3 of its shells, half of its AES pair energies plus its on-site AES, half of its D4
// two-body pair energies (weights at the output charges), plus the band part from k_moments
__global__ void k_energy(Batch B, State S) {
    int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (a >= B.natT) return;
    AtomView mv = mol_atoms(B, a);
    if (!mol_active(S, mv.m)) return;
    const double* x = S.xyz;
    int sh0 = B.m_sh0[mv.m], nsh = B.m_nsh[mv.m];
    double e = 0.0, e2 = 0.0, e3 = 0.0, eaes = 0.0, ed = 0.0;
    for (int s = B.a_sh0[a]; s < B.a_sh0[a] + B.a_nsh[a]; s++) {
        double v = 0.0;
        const double* gs = S.gam + B.m_gam0[mv.m] + (long long)(s - sh0) * nsh - sh0;
        for (int t = sh0 + lane; t < sh0 + nsh; t += 32) v += gs[t] * S.qsh_out[t];
        v = warp_sum(v);
        double q = S.qsh_out[s];
        e2 += 0.5 * q * v;
        e3 += q * q * q * B.s_gam3[s] / 3.0;
    }
    int spa = B.a_sp[a];
    const double* di = S.dp_out + 3 * a;
    const double* ti = S.qp_out + 6 * a;
    double qi = S.qat_out[a];
    for (int b = mv.i0 + lane; b < mv.i0 + mv.n; b += 32) {
        if (b == a) continue;
        double v[3];
        dvec(x, a, b, v);
        double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        double g3, g5;
        aes_g35(S, a, b, r2, g3, g5);
        const double* dj = S.dp_out + 3 * b;
        const double* tj = S.qp_out + 6 * b;
        double qj = S.qat_out[b];
        double miv = di[0] * v[0] + di[1] * v[1] + di[2] * v[2];
        double mjv = dj[0] * v[0] + dj[1] * v[1] + dj[2] * v[2];
        double ep = (qi * mjv - qj * miv) * g3;
        ep += g5 * (r2 * (di[0] * dj[0] + di[1] * dj[1] + di[2] * dj[2]) - 3.0 * miv * mjv);
        double tc[6] = {v[0] * v[0], v[0] * v[1], v[1] * v[1], v[0] * v[2], v[1] * v[2], v[2] * v[2]};
        for (int k = 0; k < 6; k++) ep += QSCALE[k] * tc[k] * g5 * (qj * ti[k] + qi * tj[k]);
        eaes += 0.5 * ep;
        double pe, pg;
        if (d4_pair(B, spa, B.a_sp[b], r2, pe, pg)) {
            double c6, da, db;
            pair_c6(B, S, a, b, c6, da, db);
            ed -= 0.5 * c6 * pe;
        }
    }
    eaes = warp_sum(eaes);
    ed = warp_sum(ed);
    if (lane == 0) {
        double qq = 0.0;
        for (int k = 0; k < 6; k++) qq += QSCALE[k] * ti[k] * ti[k];
        eaes += B.a_dk[a] * (di[0] * di[0] + di[1] * di[1] + di[2] * di[2]) + B.a_qk[a] * qq;
        e = e2 + e3 + eaes + ed;
        S.e_atom[a] += e;
        // term pieces per atom (reduced per molecule in k_broyden)
        S.e_terms[5 * a + 0] = e2;
        S.e_terms[5 * a + 1] = e3;
        S.e_terms[5 * a + 2] = eaes;
        S.e_terms[5 * a + 3] = ed;
    }
}

// ----------------------------------------------------------------------------- Broyden
__device__ double cta_sum(double v) {
    __shared__ double red[32];
    __shared__ double out;
    v = warp_sum(v);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) s += red[k];
        out = s;
    }
    __syncthreads();
    return out;
}

__device__ __forceinline__ void pack_moment(const Batch& B, int m, const double* qsh, const double* dp, const double* qp,
                                            double* v, int tid, int nthr) {
    int nsh = B.m_nsh[m], nat = B.m_nat[m], s0 = B.m_sh0[m], a0 = B.m_at0[m];
    for (int i = tid; i < nsh + 9 * nat; i += nthr) {
        double x;
        if (i < nsh) x = qsh[s0 + i];
        else if (i < nsh + 3 * nat) x = dp[3 * a0 + (i - nsh)];
        else {
            int r = i - nsh - 3 * nat, c = r % 6;
            x = qp[6 * a0 + r] * (QOFF[c] ? SQRT2 : 1.0);
        }
        v[i] = x;
    }
}

// energy assembly, residual and convergence test of one SCF iteration
// (crates/axtb/src/scf/convergence.rs:99-130, crates/axtb/src/scf/driver.rs:263-290) for the CTA
// of molecule m; true when the molecule's SCF attempt ends here (converged, failed or out of
// iterations) and no mixing step follows
__device__ bool scf_iteration_end(const Batch& B, const State& S, int m) {
    int tid = threadIdx.x, nthr = blockDim.x;
    int dim = B.m_dim[m], nat = B.m_nat[m], a0 = B.m_at0[m];
    long long v0 = B.m_vec0[m];
    double* q_in = S.q_in + v0;
    double* dq = S.dq + v0;
    // energy and terms (sums in atom order per thread stripe, reduced deterministically)
    double e = 0.0, t2 = 0.0, t3 = 0.0, ta = 0.0, td = 0.0, tb = 0.0;
    for (int a = tid; a < nat; a += nthr) {
        e += S.e_atom[a0 + a];
        t2 += S.e_terms[5 * (a0 + a) + 0];
        t3 += S.e_terms[5 * (a0 + a) + 1];
        ta += S.e_terms[5 * (a0 + a) + 2];
        td += S.e_terms[5 * (a0 + a) + 3];
        tb += S.e_terms[5 * (a0 + a) + 4];
    }
    e = cta_sum(e) + S.ts[m];
    if (B.solv) {  // the solvation term (crates/axtb/src/calculator.rs:314)
        double es = 0.0;
        for (int a = tid; a < nat; a += nthr) es += S.sv_eatom[a0 + a];
        es = cta_sum(es);
        if (tid == 0) S.sv_emol[m] = es;
    }
    t2 = cta_sum(t2);
    t3 = cta_sum(t3);
    ta = cta_sum(ta);
    td = cta_sum(td);
    tb = cta_sum(tb);
    // residual dq = pack(out) - q_in
    pack_moment(B, m, S.qsh_out, S.dp_out, S.qp_out, dq, tid, nthr);
    __syncthreads();
    double rr = 0.0;
    for (int i = tid; i < dim; i += nthr) {
        dq[i] -= q_in[i];
        rr += dq[i] * dq[i];
    }
    rr = cta_sum(rr);
    __shared__ int s_done;
    if (tid == 0) {
        double res = sqrt(rr / dim);
        double de = e - S.elast[m];
        S.elast[m] = e;
        S.energy[m] = e;
        S.de[m] = de;
        S.res[m] = res;
        double* tm = S.terms + 8 * m;
        tm[2] = e;
        tm[3] = t2;
        tm[4] = t3;
        tm[5] = ta;
        tm[1] = td;
        tm[6] = S.ts[m];
        tm[7] = tb;
        int it = ++S.niter[m];
        if (!isfinite(e)) S.status[m] |= ST_NONFINITE;
        bool ok = fabs(de) < B.econv && res < B.pconv;
        s_done = 0;
        if (S.status[m] != 0) {
            S.active[m] = 0;
            s_done = 1;
        } else if (ok) {
            S.conv[m] = 1;
            S.active[m] = 0;
            s_done = 1;
        } else if (it >= B.max_iter) {
            S.active[m] = 0;
            s_done = 1;
        }
    }
    __syncthreads();
    return s_done != 0;
}

// the new input q_in into the input moments (and re-packed, as the reference packs the state it
// unpacked: crates/axtb/src/scf/driver.rs:225-229)
__device__ void unpack_input(const Batch& B, const State& S, int m) {
    int tid = threadIdx.x, nthr = blockDim.x;
    int dim = B.m_dim[m], nat = B.m_nat[m], a0 = B.m_at0[m];
    double* q_in = S.q_in + B.m_vec0[m];
    __syncthreads();
    int nsh = B.m_nsh[m], s0 = B.m_sh0[m];
    for (int i = tid; i < dim; i += nthr) {
        double x = q_in[i];
        if (i < nsh) S.qsh_in[s0 + i] = x;
        else if (i < nsh + 3 * nat) S.dp_in[3 * a0 + (i - nsh)] = x;
        else {
            int r = i - nsh - 3 * nat, c = r % 6;
            double y = x / (QOFF[c] ? SQRT2 : 1.0);
            S.qp_in[6 * a0 + r] = y;
            q_in[i] = y * (QOFF[c] ? SQRT2 : 1.0);
        }
    }
    __syncthreads();
    for (int a = tid; a < nat; a += nthr) {
        double q = 0.0;
        for (int s = B.a_sh0[a0 + a]; s < B.a_sh0[a0 + a] + B.a_nsh[a0 + a]; s++) q += S.qsh_in[s];
        S.qat_in[a0 + a] = q;
    }
}

constexpr int BROYDEN_MAX_HIST = 256;  // history slots a molecule can hold (shared solve vector)

// the iteration's end and the next input by modified Broyden mixing
// (crates/axtb/src/scf/mixing.rs:251-338 with crates/base/src/linalg/lu.rs:81-112); one CTA per
// molecule. The Gauss elimination updates the rows below the pivot in parallel, each row with
// the reference's operations in its order.
__global__ void k_broyden(Batch B, State S, int hist_cap) {
    int m = blockIdx.x;
    if (m >= B.nmol || !mol_active(S, m)) return;
    if (scf_iteration_end(B, S, m)) return;
    int tid = threadIdx.x, nthr = blockDim.x;
    int dim = B.m_dim[m];
    long long v0 = B.m_vec0[m];
    double* q_in = S.q_in + v0;
    double* dq = S.dq + v0;
    double* qlast = S.qlast + v0;
    double* dqlast = S.dqlast + v0;
    long long h0 = B.m_hist0[m];
    double* df = S.df + h0;  // hist_cap * dim
    double* u = S.u + h0;
    double* amat = S.amat + (long long)m * hist_cap * hist_cap;
    double* omega = S.omega + (long long)m * hist_cap;
    __shared__ int s_ok;
    // one thread advances the step counter; every thread reads it back
    __shared__ int s_iter;
    if (tid == 0) s_iter = ++S.iter[m];
    __syncthreads();
    int iter = s_iter;
    double alpha = B.damping;
    if (iter == 1) {
        for (int i = tid; i < dim; i += nthr) {
            dqlast[i] = dq[i];
            qlast[i] = q_in[i];
            q_in[i] += alpha * dq[i];
        }
    } else {
        int itn = iter - 1;
        int it1 = itn - 1;
        if (it1 >= hist_cap) {
            if (tid == 0) {
                S.status[m] |= ST_HISTORY;
                S.active[m] = 0;
            }
            return;
        }
        int nh = itn;  // memory = max_iter >= iterations: the whole history
        double* dfi = df + (long long)it1 * dim;
        double nr = 0.0;
        for (int i = tid; i < dim; i += nthr) nr += dq[i] * dq[i];
        nr = sqrt(cta_sum(nr));
        const double OMEGA0 = 0.01, MINW = 1.0, MAXW = 100000.0, WFAC = 0.01;
        double om = nr > WFAC / MAXW ? WFAC / nr : MAXW;
        if (om < MINW) om = MINW;
        if (tid == 0) omega[it1] = om;
        double dn = 0.0;
        for (int i = tid; i < dim; i += nthr) {
            double v = dq[i] - dqlast[i];
            dfi[i] = v;
            dn += v * v;
        }
        dn = cta_sum(dn);
        double inv = 1.0 / fmax(sqrt(dn), DBL_EPSILON);
        for (int i = tid; i < dim; i += nthr) dfi[i] *= inv;
        __syncthreads();
        // a[it1][j] = df_it1 . df_j (j <= it1), c[j] = omega_j df_j . dq
        __shared__ double cvec[BROYDEN_MAX_HIST];
        __shared__ int s_piv;
        for (int j = 0; j < nh; j++) {
            double* dfj = df + (long long)j * dim;
            double s1 = 0.0, s2 = 0.0;
            for (int i = tid; i < dim; i += nthr) {
                s1 += dfi[i] * dfj[i];
                s2 += dfj[i] * dq[i];
            }
            s1 = cta_sum(s1);
            s2 = cta_sum(s2);
            if (tid == 0) {
                amat[it1 * hist_cap + j] = s1;
                amat[j * hist_cap + it1] = s1;
                cvec[j] = s2;  // times omega below
            }
        }
        __syncthreads();
        // beta (kept in the tail of amat's slab) = omega_i omega_j a_ij + omega0^2 delta_ij
        double* bt = S.amat + (long long)B.nmol * hist_cap * hist_cap + (long long)m * hist_cap * hist_cap;
        for (int e = tid; e < nh * nh; e += nthr) {
            int i = e / nh, j = e % nh;
            double v = omega[i] * omega[j] * amat[i * hist_cap + j];
            if (i == j) v += OMEGA0 * OMEGA0;
            bt[i * hist_cap + j] = v;
        }
        __syncthreads();
        if (tid == 0) {
            s_ok = 1;
            for (int i = 0; i < nh; i++) cvec[i] *= omega[i];
        }
        // Gauss elimination with the last largest pivot
        for (int col = 0; col < nh; col++) {
            __syncthreads();
            if (tid == 0) {
                int piv = col;
                for (int i = col + 1; i < nh; i++)
                    if (fabs(bt[i * hist_cap + col]) >= fabs(bt[piv * hist_cap + col])) piv = i;
                if (bt[piv * hist_cap + col] == 0.0) s_ok = 0;
                s_piv = piv;
            }
            __syncthreads();
            if (!s_ok) break;
            int piv = s_piv;
            if (piv != col) {
                for (int k = tid; k < nh; k += nthr) {
                    double tmp = bt[col * hist_cap + k];
                    bt[col * hist_cap + k] = bt[piv * hist_cap + k];
                    bt[piv * hist_cap + k] = tmp;
                }
                if (tid == 0) {
                    double tmp = cvec[col];
                    cvec[col] = cvec[piv];
                    cvec[piv] = tmp;
                }
                __syncthreads();
            }
            const double* prow = bt + (long long)col * hist_cap;
            for (int row = col + 1 + tid; row < nh; row += nthr) {
                double* rrow = bt + (long long)row * hist_cap;
                double f = rrow[col] / prow[col];
                if (f != 0.0) {
                    for (int k = col; k < nh; k++) rrow[k] -= f * prow[k];
                    cvec[row] -= f * cvec[col];
                }
            }
        }
        __syncthreads();
        if (tid == 0 && s_ok)
            for (int col = nh - 1; col >= 0; col--) {
                double s = cvec[col];
                for (int k = col + 1; k < nh; k++) s -= bt[col * hist_cap + k] * cvec[k];
                cvec[col] = s / bt[col * hist_cap + col];
            }
        __syncthreads();
        if (!s_ok) {
            if (tid == 0) {
                S.status[m] |= ST_MIXER;
                S.active[m] = 0;
            }
            return;
        }
        double* ui = u + (long long)it1 * dim;
        for (int i = tid; i < dim; i += nthr) {
            ui[i] = alpha * dfi[i] + inv * (q_in[i] - qlast[i]);
            dqlast[i] = dq[i];
            qlast[i] = q_in[i];
            double v = q_in[i] + alpha * dq[i];
            for (int j = 0; j < nh; j++) v -= omega[j] * cvec[j] * u[(long long)j * dim + i];
            q_in[i] = v;
        }
    }
    unpack_input(B, S, m);
}

// ----------------------------------------------------------------------------- DIIS
// Pulay (DIIS, Anderson) mixing with restarts (crates/axtb/src/scf/mixing.rs:342-525). Per
// molecule, in its mixer history span (DIIS_SLOTS vectors in df and in u):
//   df slots [0, DIIS_SIZE): inputs q_i (a ring), [DIIS_SIZE, 2 DIIS_SIZE - 1): the orthonormal
//   basis of the residual differences, then the best input and its residual;
//   u slots [0, DIIS_SIZE): residuals r_i (the same ring).
// Scalars in S.diis[8 m ..]: damping, best residual norm, best seen (0/1), iterations since the
// best, history length, ring head.
constexpr int DIIS_SIZE = 30;
constexpr int DIIS_SLOTS = 2 * DIIS_SIZE + 1;
constexpr double DIIS_DEPENDENCE = 1e-2;
constexpr int DIIS_STALL = 12;
constexpr double DIIS_RESTART_GROWTH = 1e3, DIIS_RESTART_FLOOR = 0.1;

__device__ __forceinline__ void diis_reset(const Batch& B, const State& S, int m) {
    double* d = S.diis + 8 * m;
    d[0] = B.damping;
    for (int k = 1; k < 8; k++) d[k] = 0.0;
}

// the iteration's end and the next input by DIIS: the coefficients c minimise |sum c_i r_i|
// with sum c_i = 1, from the differences r_n - r_j orthonormalised newest first by modified
// Gram-Schmidt (a difference keeping less than DIIS_DEPENDENCE of its norm ends the basis) and
// R g = Q^T r_n; the next input is sum c_i (q_i + damp r_i). A residual DIIS_RESTART_GROWTH times
// the best (above DIIS_RESTART_FLOOR), or DIIS_STALL iterations without a better one, restart
// from the best input with half the damping. One CTA per molecule.
__global__ void k_diis(Batch B, State S) {
    int m = blockIdx.x;
    if (m >= B.nmol || !mol_active(S, m)) return;
    if (scf_iteration_end(B, S, m)) return;
    int tid = threadIdx.x, nthr = blockDim.x;
    int dim = B.m_dim[m];
    long long v0 = B.m_vec0[m];
    double* q_in = S.q_in + v0;
    const double* dq = S.dq + v0;
    long long h0 = B.m_hist0[m];
    double* hq = S.df + h0;                                   // input ring
    double* hr = S.u + h0;                                    // residual ring
    double* basis = S.df + h0 + (long long)DIIS_SIZE * dim;  // DIIS_SIZE - 1 basis vectors
    double* best_q = S.df + h0 + (long long)(2 * DIIS_SIZE - 1) * dim;
    double* best_r = best_q + dim;
    double* sc = S.diis + 8 * m;
    __shared__ double s_R[DIIS_SIZE][DIIS_SIZE];  // s_R[l][p]: entry l of column p of R
    __shared__ double s_c[DIIS_SIZE], s_g[DIIS_SIZE];
    __shared__ int s_kept[DIIS_SIZE];
    double nn = 0.0;
    for (int i = tid; i < dim; i += nthr) nn += dq[i] * dq[i];
    double norm = sqrt(cta_sum(nn));
    double damp = sc[0];
    bool have_best = sc[2] != 0.0;
    int since_best = (int)sc[3], count = (int)sc[4], head = (int)sc[5];
    int mode = 0;  // 0 mix, 1 restart, 2 failed (the same on every thread)
    if (!isfinite(norm)) mode = 2;
    else if (have_best && ((norm > DIIS_RESTART_GROWTH * sc[1] && norm > DIIS_RESTART_FLOOR) ||
                           since_best >= DIIS_STALL))
        mode = 1;
    __syncthreads();
    if (mode == 2) {
        if (tid == 0) {
            S.status[m] |= ST_MIXER;
            S.active[m] = 0;
        }
        return;
    }
    if (mode == 1) {
        // drop the history and restart from the best input with half the damping
        damp *= 0.5;
        for (int i = tid; i < dim; i += nthr) q_in[i] = best_q[i] + damp * best_r[i];
        if (tid == 0) {
            sc[0] = damp;
            sc[3] = 0.0;
            sc[4] = 0.0;
            sc[5] = 0.0;
        }
        unpack_input(B, S, m);
        return;
    }
    bool better = !have_best || norm < sc[1];
    if (better)
        for (int i = tid; i < dim; i += nthr) {
            best_q[i] = q_in[i];
            best_r[i] = dq[i];
        }
    since_best = better ? 0 : since_best + 1;
    // push (q_in, dq), dropping the oldest pair of a full history
    if (count == DIIS_SIZE) {
        head = (head + 1) % DIIS_SIZE;
        count--;
    }
    int slot = (head + count) % DIIS_SIZE;
    count++;
    for (int i = tid; i < dim; i += nthr) {
        hq[(long long)slot * dim + i] = q_in[i];
        hr[(long long)slot * dim + i] = dq[i];
    }
    __syncthreads();
    if (tid == 0) {
        if (better) sc[1] = norm;
        sc[2] = 1.0;
        sc[3] = since_best;
        sc[4] = count;
        sc[5] = head;
    }
    auto phys = [&](int i) { return (long long)((head + i) % DIIS_SIZE) * dim; };
    const double* last = hr + phys(count - 1);
    int p = 0;
    for (int j = count - 2; j >= 0; j--) {
        double* d = basis + (long long)p * dim;
        const double* rj = hr + phys(j);
        double a = 0.0;
        for (int i = tid; i < dim; i += nthr) {
            double v = last[i] - rj[i];
            d[i] = v;
            a += v * v;
        }
        double norm0 = sqrt(cta_sum(a));
        if (isnan(norm0) || norm0 <= 0.0) break;
        for (int l = 0; l < p; l++) {
            const double* bl = basis + (long long)l * dim;
            double h = 0.0;
            for (int i = tid; i < dim; i += nthr) h += bl[i] * d[i];
            h = cta_sum(h);
            if (tid == 0) s_R[l][p] = h;
            for (int i = tid; i < dim; i += nthr) d[i] -= h * bl[i];
        }
        double b2 = 0.0;
        for (int i = tid; i < dim; i += nthr) b2 += d[i] * d[i];
        double nr = sqrt(cta_sum(b2));
        if (nr < DIIS_DEPENDENCE * norm0) break;
        if (tid == 0) {
            s_R[p][p] = nr;
            s_kept[p] = j;
        }
        for (int i = tid; i < dim; i += nthr) d[i] /= nr;
        p++;
    }
    // R g = Q^T r_n by back substitution; c_j = g_j (kept j), c_n = 1 - sum g
    for (int l = 0; l < p; l++) {
        const double* bl = basis + (long long)l * dim;
        double h = 0.0;
        for (int i = tid; i < dim; i += nthr) h += bl[i] * last[i];
        h = cta_sum(h);
        if (tid == 0) s_g[l] = h;
    }
    if (tid == 0) {
        for (int l = p - 1; l >= 0; l--) {
            double v = s_g[l];
            for (int k = l + 1; k < p; k++) v -= s_R[l][k] * s_g[k];
            s_g[l] = v / s_R[l][l];
        }
        for (int i = 0; i < count; i++) s_c[i] = 0.0;
        s_c[count - 1] = 1.0;
        for (int l = 0; l < p; l++) {
            s_c[s_kept[l]] += s_g[l];
            s_c[count - 1] -= s_g[l];
        }
    }
    __syncthreads();
    for (int i = tid; i < dim; i += nthr) {
        double x = 0.0;
        for (int k = 0; k < count; k++) {
            double c = s_c[k];
            if (c != 0.0) x += c * (hq[phys(k) + i] + damp * hr[phys(k) + i]);
        }
        q_in[i] = x;
    }
    unpack_input(B, S, m);
}

// ----------------------------------------------------------------------------- gradient pairs
// ES2 (crates/axtb/src/coulomb.rs:123-169), AES (896-1001) and D4 two-body at fixed charges
// (crates/d4/src/disp.rs:460-484; weights and dgw/dCN at the output charges) per atom; warp per atom
__global__ void k_grad_pairs(Batch B, State S) {
    int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (a >= B.natT) return;
    AtomView mv = mol_atoms(B, a);
    if (!S.conv[mv.m]) return;
    const double* x = S.xyz;
    double g[3] = {0, 0, 0}, dedr = 0.0, dcn4 = 0.0;
    const double kdmp3 = 3.0, kdmp5 = 4.0;
    int spa = B.a_sp[a];
    for (int b = mv.i0 + lane; b < mv.i0 + mv.n; b += 32) {
        if (b == a) continue;
        double v[3];
        dvec(x, a, b, v);  // R_a - R_b
        double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        double r1 = sqrt(r2);
        // ES2
        double dg = 0.0;
        for (int s = B.a_sh0[a]; s < B.a_sh0[a] + B.a_nsh[a]; s++)
            for (int t = B.a_sh0[b]; t < B.a_sh0[b] + B.a_nsh[b]; t++) {
                double eta = 0.5 * (B.s_hard[s] + B.s_hard[t]);
                double dt = 1.0 / (r2 + 1.0 / (eta * eta));
                dt = -dt * sqrt(dt);
                dg += dt * S.qsh_out[s] * S.qsh_out[t];
            }
        for (int k = 0; k < 3; k++) g[k] += dg * v[k];
        // AES: the reference's pair (iat, jat) with vec = R_jat - R_iat; here (a, b) as (i, j)
        {
            double rr = 0.5 * (S.mrad[a] + S.mrad[b]);
            double vec[3] = {-v[0], -v[1], -v[2]};
            double g1 = 1.0 / r1, g3 = g1 * g1 * g1, g5 = g3 * g1 * g1, g7 = g5 * g1 * g1;
            double rg = rr * g1, rg3 = rg * rg * rg, rg4 = rg3 * rg;
            double fdmp3 = 1.0 / (1.0 + 6.0 * rg3);
            double ddmp3 = -3.0 * g5 * fdmp3 - kdmp3 * fdmp3 * (fdmp3 - 1.0) * g5;
            double fdmp5 = 1.0 / (1.0 + 6.0 * rg4);
            double ddmp5 = -5.0 * fdmp5 - kdmp5 * (fdmp5 * fdmp5 - fdmp5);
            double qi = S.qat_out[a], qj = S.qat_out[b];
            const double* di = S.dp_out + 3 * a;
            const double* dj = S.dp_out + 3 * b;
            double dpiqj = (vec[0] * di[0] + vec[1] * di[1] + vec[2] * di[2]) * qj;
            double qidpj = (vec[0] * dj[0] + vec[1] * dj[1] + vec[2] * dj[2]) * qi;
            double fddr = 3.0 * (dpiqj - qidpj) * kdmp3 * fdmp3 * g3 * (fdmp3 / rr) * rg3;
            double gg[3];
            for (int k = 0; k < 3; k++) gg[k] = -ddmp3 * vec[k] * (dpiqj - qidpj) + fdmp3 * g3 * (qi * dj[k] - qj * di[k]);
            double dpidpj = dj[0] * di[0] + dj[1] * di[1] + dj[2] * di[2];
            double dpiv = di[0] * vec[0] + di[1] * vec[1] + di[2] * vec[2];
            double dpjv = dj[0] * vec[0] + dj[1] * vec[1] + dj[2] * vec[2];
            double edd = dpidpj * r2 - 3.0 * dpjv * dpiv;
            fddr += 3.0 * edd * kdmp5 * fdmp5 * g5 * (fdmp5 / rr) * rg4;
            for (int k = 0; k < 3; k++)
                gg[k] += -2.0 * fdmp5 * g5 * dpidpj * vec[k] + 3.0 * fdmp5 * g5 * (dpiv * dj[k] + dpjv * di[k]) -
                         edd * ddmp5 * g7 * vec[k];
            const double* ti = S.qp_out + 6 * a;
            const double* tj = S.qp_out + 6 * b;
            double eq = 2.0 * (qj * ti[1] + tj[1] * qi) * vec[0] * vec[1] + 2.0 * (qj * ti[3] + tj[3] * qi) * vec[0] * vec[2] +
                        2.0 * (qj * ti[4] + tj[4] * qi) * vec[1] * vec[2] + (qj * ti[0] + tj[0] * qi) * vec[0] * vec[0] +
                        (qj * ti[2] + tj[2] * qi) * vec[1] * vec[1] + (qj * ti[5] + tj[5] * qi) * vec[2] * vec[2];
            fddr += eq * 3.0 * kdmp5 * fdmp5 * g5 * fdmp5 / rr * rg4;
            double tvj[3] = {vec[0] * tj[0] + vec[1] * tj[1] + vec[2] * tj[3], vec[0] * tj[1] + vec[1] * tj[2] + vec[2] * tj[4],
                             vec[0] * tj[3] + vec[1] * tj[4] + vec[2] * tj[5]};
            double tvi[3] = {vec[0] * ti[0] + vec[1] * ti[1] + vec[2] * ti[3], vec[0] * ti[1] + vec[1] * ti[2] + vec[2] * ti[4],
                             vec[0] * ti[3] + vec[1] * ti[4] + vec[2] * ti[5]};
            for (int k = 0; k < 3; k++)
                gg[k] += -eq * ddmp5 * g7 * vec[k] - 2.0 * fdmp5 * g5 * qi * tvj[k] - 2.0 * fdmp5 * g5 * qj * tvi[k];
            for (int k = 0; k < 3; k++) g[k] += gg[k];
            dedr += fddr;
        }
        // D4 two-body at the output charges (dgw = dgw/dCN)
        double pe, pg;
        if (d4_pair(B, spa, B.a_sp[b], r2, pe, pg)) {
            double c6, da, db;
            pair_c6(B, S, a, b, c6, da, db);
            dcn4 -= da * pe;
            for (int k = 0; k < 3; k++) g[k] += -c6 * pg * v[k];
        }
    }
    for (int k = 0; k < 3; k++) g[k] = warp_sum(g[k]);
    dedr = warp_sum(dedr);
    dcn4 = warp_sum(dcn4);
    if (lane == 0) {
        for (int k = 0; k < 3; k++) S.grad[3 * a + k] += g[k];
        S.dedcn[a] += dedr * S.dmrdcn[a];
        S.dedcn_d4[a] += dcn4;
    }
}

// one-electron gradient pieces gathered per atom from the per-pair buffer, plus the on-site CN
// term (crates/axtb/src/hamiltonian.rs:211-221); warp per atom
__global__ void k_h0_gather(Batch B, State S, const long long* m_pair0, const double* pairs) {
    int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (a >= B.natT) return;
    AtomView mv = mol_atoms(B, a);
    if (!S.conv[mv.m]) return;
    int la = a - mv.i0;
    double g[3] = {0, 0, 0}, dc = 0.0;
    for (int lb = lane; lb < mv.n; lb += 32) {
        if (lb == la) continue;
        if (la > lb) {
            const double* p = pairs + (m_pair0[mv.m] + (long long)la * (la - 1) / 2 + lb) * 5;
            for (int k = 0; k < 3; k++) g[k] += p[k];
            dc += p[3];
        } else {
            const double* p = pairs + (m_pair0[mv.m] + (long long)lb * (lb - 1) / 2 + la) * 5;
            for (int k = 0; k < 3; k++) g[k] -= p[k];
            dc += p[4];
        }
    }
    for (int k = 0; k < 3; k++) g[k] = warp_sum(g[k]);
    dc = warp_sum(dc);
    if (lane == 0) {
        int n = B.m_nao[mv.m];
        long long mat = B.m_mat0[mv.m];
        int ao0 = B.m_ao0[mv.m];
        for (int s = B.a_sh0[a]; s < B.a_sh0[a] + B.a_nsh[a]; s++)
            for (int o = B.s_ao0[s]; o < B.s_ao0[s] + 2 * B.s_l[s] + 1; o++) {
                int mu = o - ao0;
                dc += S.dsedcn[s] * S.P[mat + mu + (long long)mu * n];
            }
        for (int k = 0; k < 3; k++) S.grad[3 * a + k] += g[k];
        S.dedcn[a] += dc;
    }
}

// CN chain rules: GFN2 CN with dE/dCN (crates/base/src/ncoord.rs:486-519) and the D4 CN with
// its dE/dCN (crates/d4/src/ncoord.rs:56-70); warp per atom
__global__ void k_cn_chain(Batch B, State S) {
    int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (a >= B.natT) return;
    AtomView mv = mol_atoms(B, a);
    if (!S.conv[mv.m]) return;
    double g[3] = {0, 0, 0};
    int spa = B.a_sp[a];
    for (int b = mv.i0 + lane; b < mv.i0 + mv.n; b += 32) {
        if (b == a) continue;
        double v[3];
        dvec(S.xyz, a, b, v);
        double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        if (r2 < 1e-12) continue;
        double r = sqrt(r2);
        if (r2 <= B.cn_cut * B.cn_cut) {
            double d = dexp_dcount(r, B.a_rcov[a] + B.a_rcov[b]);
            double t = d * (S.dedcn[a] + S.dedcn[b]) / r;
            for (int k = 0; k < 3; k++) g[k] += t * v[k];
        }
        if (r2 <= B.d4_cn_cut * B.d4_cn_cut) {
            int spb = B.a_sp[b];
            double dc = en_factor(B.sp_en[spa], B.sp_en[spb]) * erf_dcount(r, B.sp_rcov[spa] + B.sp_rcov[spb]);
            double s = S.dedcn_d4[a] + S.dedcn_d4[b];
            for (int k = 0; k < 3; k++) g[k] += dc * v[k] / r * s;
        }
    }
    for (int k = 0; k < 3; k++) g[k] = warp_sum(g[k]);
    if (lane == 0)
        for (int k = 0; k < 3; k++) S.grad[3 * a + k] += g[k];
}

}  // namespace axg
