// Geometry-dependent kernels of one batch: coordination numbers, self energies, multipole
// radii, repulsion, D4 reference weights and the Axilrod-Teller-Muto term, the EEQ start
// system. Pair sums run one warp per atom (lanes over partner atoms of the same molecule), so
// every atom's sum is its own and no atomics are needed; each pair term is evaluated from both
// of its atoms.
#pragma once
#include "common.cuh"

namespace axg {

// ---- constants of the models; the real-space cutoffs of the conventions are Batch fields
constexpr double D4_S6 = 1.0, D4_S8 = 2.7, D4_S9 = 5.0, D4_ALP = 16.0;  // crates/d4/src/disp.rs:24
constexpr double D4_GA = 3.0, D4_WF = 6.0;  // crates/d4/src/model.rs:20-22

struct AtomView {
    int m, i0, n;  // molecule, first atom, atom count
};
__device__ __forceinline__ AtomView mol_atoms(const Batch& B, int a) {
    int m = B.a_mol[a];
    return {m, B.m_at0[m], B.m_nat[m]};
}
__device__ __forceinline__ void dvec(const double* x, int a, int b, double v[3]) {
    v[0] = x[3 * a] - x[3 * b];
    v[1] = x[3 * a + 1] - x[3 * b + 1];
    v[2] = x[3 * a + 2] - x[3 * b + 2];
}

// double-exponential count of the GFN2 CN (crates/base/src/ncoord.rs:59-121)
__device__ __forceinline__ double ecount(double k, double r, double r0) { return 1.0 / (1.0 + exp(-k * (r0 / r - 1.0))); }
__device__ __forceinline__ double edcount(double k, double r, double r0) {
    double e = exp(-k * (r0 / r - 1.0));
    return (-k * r0 * e) / (r * r * ((e + 1.0) * (e + 1.0)));
}
__device__ __forceinline__ double dexp_count(double r, double rc) { return ecount(10.0, r, rc) * ecount(20.0, r, rc + 2.0); }
__device__ __forceinline__ double dexp_dcount(double r, double rc) {
    return edcount(10.0, r, rc) * ecount(20.0, r, rc + 2.0) + ecount(10.0, r, rc) * edcount(20.0, r, rc + 2.0);
}
// error-function count (crates/base/src/ncoord.rs:123-148) and D4's EN weight (crates/d4/src/ncoord.rs:20-30)
__device__ __forceinline__ double erf_count(double r, double rc) { return 0.5 * (1.0 + erf(-((7.5 * (r - rc)) / rc))); }
__device__ __forceinline__ double erf_dcount(double r, double rc) {
    double e = 7.5 * (r - rc) / rc;
    return -(7.5 * exp(-(e * e))) / (1.7724538509055159 * rc);
}
__device__ __forceinline__ double en_factor(double ei, double ej) {
    double x = fabs(ei - ej) + 19.08857;
    return 4.10451 * exp(-((x * x) / (2.0 * (11.28174 * 11.28174))));
}
// smooth real-space switch (crates/d4/src/disp.rs:40-62)
__device__ __forceinline__ void smooth_cut(double r, double cutoff, double width, double& sw, double& dsw) {
    double w = fmin(width, cutoff), inner = cutoff - w;
    if (r <= inner) {
        sw = 1.0;
        dsw = 0.0;
    } else if (r >= cutoff) {
        sw = 0.0;
        dsw = 0.0;
    } else {
        double x = (cutoff - r) / w, x2 = x * x, omx = 1.0 - x;
        sw = (x2 * x) * (10.0 + x * (-15.0 + 6.0 * x));
        dsw = -((30.0 * x2 * (omx * omx)) / w);
    }
}

// GFN2, D4 and EEQ coordination numbers; warp per atom
__global__ void k_cn(Batch B, State S) {
    int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (a >= B.natT) return;
    AtomView mv = mol_atoms(B, a);
    const double* x = S.xyz;
    int spa = B.a_sp[a];
    double c1 = 0.0, c2 = 0.0, c3 = 0.0;
    for (int b = mv.i0 + lane; b < mv.i0 + mv.n; b += 32) {
        if (b == a) continue;
        double v[3];
        dvec(x, a, b, v);
        double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        if (r2 < 1e-12) continue;
        double r = sqrt(r2);
        if (r2 <= B.cn_cut * B.cn_cut) c1 += dexp_count(r, B.a_rcov[a] + B.a_rcov[b]);
        if (r2 <= B.d4_cn_cut * B.d4_cn_cut) {
            int spb = B.a_sp[b];
            c2 += en_factor(B.sp_en[spa], B.sp_en[spb]) * erf_count(r, B.sp_rcov[spa] + B.sp_rcov[spb]);
        }
        if (r2 <= B.eeq_cn_cut * B.eeq_cn_cut) c3 += erf_count(r, B.a_rcov_eeq[a] + B.a_rcov_eeq[b]);
    }
    c1 = warp_sum(c1);
    c2 = warp_sum(c2);
    c3 = warp_sum(c3);
    if (lane == 0) {
        S.cn[a] = c1;
        S.cn_d4[a] = c2;
        // multicharge's log cap (crates/base/src/ncoord.rs log_cap); none in the xtb conventions
        const double cap = B.eeq_cap;
        S.cn_eeq[a] = cap > 0.0 ? log(1.0 + exp(cap)) - log(exp(cap - c3) + 1.0) : c3;
    }
}

// self energies (crates/axtb/src/hamiltonian.rs:42-54) and AES radii (crates/axtb/src/coulomb.rs:368-380)
__global__ void k_selfenergy(Batch B, State S) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < B.nshT) {
        int a = B.s_at[s];
        S.se[s] = B.s_se0[s] - B.s_kcn[s] * S.cn[a];
        S.dsedcn[s] = -B.s_kcn[s];
    }
    if (s < B.natT) {
        const double shift = 1.2, kexp = 4.0, rmax = 5.0;
        double arg = S.cn[s] - B.a_aes_vcn[s] - shift;
        double t1 = exp(-kexp * arg);
        double t2 = (rmax - B.a_aes_rad[s]) / (1.0 + t1);
        S.mrad[s] = B.a_aes_rad[s] + t2;
        S.dmrdcn[s] = -t2 * kexp * t1 / (1.0 + t1);
    }
}

// repulsion energy and gradient (crates/axtb/src/repulsion.rs:44-73); warp per atom
__global__ void k_repulsion(Batch B, State S) {
    int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (a >= B.natT) return;
    AtomView mv = mol_atoms(B, a);
    double e = 0.0, g[3] = {0, 0, 0};
    int za = B.a_Z[a];
    for (int b = mv.i0 + lane; b < mv.i0 + mv.n; b += 32) {
        if (b == a) continue;
        double v[3];
        dvec(S.xyz, a, b, v);
        double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        if (r2 > B.rep_cut * B.rep_cut || r2 < 1e-12) continue;
        double r1 = sqrt(r2);
        double kexp = (za > 2 || B.a_Z[b] > 2) ? 1.5 : 1.0;
        double alpha = sqrt(B.a_rep_alpha[b] * B.a_rep_alpha[a]);
        double r1k = kexp == 1.5 ? r1 * sqrt(r1) : r1;
        double de = B.a_rep_zeff[b] * B.a_rep_zeff[a] * exp(-alpha * r1k) / r1;
        e += 0.5 * de;
        double f = -(alpha * r1k * kexp + 1.0) * de / r2;
        for (int k = 0; k < 3; k++) g[k] += f * v[k];
    }
    e = warp_sum(e);
    for (int k = 0; k < 3; k++) g[k] = warp_sum(g[k]);
    if (lane == 0) {
        S.e_atom[a] += e;
        for (int k = 0; k < 3; k++) S.grad[3 * a + k] += g[k];
    }
}

// D4 reference weights (crates/d4/src/model.rs:474-570) at charges q; mode 0: dgw = dgw/dq,
// 1: dgw = dgw/dCN, 2: no derivative. One thread per atom.
__global__ void k_d4_weights(Batch B, State S, const double* q, int mode) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= B.natT) return;
    int sp = B.a_sp[a];
    int nr = B.sp_nref[sp];
    const int* ngw = B.sp_ngw + sp * MAXREF;
    const double* refcn = B.sp_refcn + sp * MAXREF;
    const double* refq = B.sp_refq + sp * MAXREF;
    double zi = B.sp_zeff[sp], gi = B.sp_gi[sp], cni = S.cn_d4[a];
    double norm = 0.0, dnorm = 0.0;
    for (int r = 0; r < nr; r++)
        for (int ig = 1; ig <= ngw[r]; ig++) {
            double wf = ig * D4_WF, dd = cni - refcn[r];
            double g = exp(-(wf * (dd * dd)));
            norm += g;
            dnorm += 2.0 * wf * (refcn[r] - cni) * g;
        }
    norm = fabs(norm) > sqrt(DBL_MIN) ? 1.0 / norm : 0.0;
    double maxcn = -INFINITY;
    for (int r = 0; r < nr; r++) maxcn = fmax(maxcn, refcn[r]);
    for (int r = 0; r < MAXREF; r++) {
        double gw = 0.0, dg = 0.0;
        if (r < nr) {
            double expw = 0.0, expd = 0.0;
            for (int ig = 1; ig <= ngw[r]; ig++) {
                double wf = ig * D4_WF, dd = cni - refcn[r];
                double g = exp(-(wf * (dd * dd)));
                expw += g;
                expd += 2.0 * wf * (refcn[r] - cni) * g;
            }
            double gwk = expw * norm;
            if (!isfinite(gwk) || norm == 0.0) gwk = fabs(maxcn - refcn[r]) < 1e-12 ? 1.0 : 0.0;
            double qref = refq[r] + zi, qmod = q[a] + zi;
            double z, dz = 0.0;
            if (qmod < 0.0) {
                z = exp(D4_GA);
            } else {
                double e = exp(gi * (1.0 - qref / qmod));
                z = exp(D4_GA * (1.0 - e));
                dz = -((D4_GA * gi * e * z * qref) / (qmod * qmod));
            }
            gw = gwk * z;
            if (mode == 0) dg = gwk * dz;
            else if (mode == 1) {
                double dgwk = norm * (expd - expw * dnorm * norm);
                if (!isfinite(dgwk) || norm == 0.0) dgwk = 0.0;
                dg = dgwk * z;
            }
        }
        S.gw[(long long)a * MAXREF + r] = gw;
        S.dgw[(long long)a * MAXREF + r] = dg;
    }
}

// C6 of a pair and its derivatives through the weight derivatives dgw (crates/d4/src/model.rs:577-631)
__device__ __forceinline__ void pair_c6(const Batch& B, const State& S, int a, int b, double& c6, double& da, double& db) {
    int spa = B.a_sp[a], spb = B.a_sp[b];
    const double* blk = B.sp_c6ref + (long long)(spa * B.nsp + spb) * MAXREF * MAXREF;
    const double* wa = S.gw + (long long)a * MAXREF;
    const double* wb = S.gw + (long long)b * MAXREF;
    const double* ga = S.dgw + (long long)a * MAXREF;
    const double* gb = S.dgw + (long long)b * MAXREF;
    int na = B.sp_nref[spa], nb = B.sp_nref[spb];
    c6 = da = db = 0.0;
    for (int r = 0; r < na; r++)
        for (int s = 0; s < nb; s++) {
            double ref = blk[r * MAXREF + s];
            c6 += wa[r] * wb[s] * ref;
            da += ga[r] * wb[s] * ref;
            db += wa[r] * gb[s] * ref;
        }
}

// two-body damped pair factor with its smooth switch (crates/d4/src/disp.rs:298-322):
// pe (energy factor), pg (radial derivative / r); false outside the cutoff
__device__ __forceinline__ bool d4_pair(const Batch& B, int spa, int spb, double r2, double& pe, double& pg) {
    if (!B.disp || r2 > B.d2_cut * B.d2_cut || r2 < DBL_EPSILON) return false;
    double r = sqrt(r2), sw, dsw;
    smooth_cut(r, B.d2_cut, B.d2_w, sw, dsw);
    if (sw <= 0.0) return false;
    int k = spa * B.nsp + spb;
    double rr = B.sp_rr[k], r0 = B.sp_r0[k];
    double r0_2 = r0 * r0, r0_3 = r0_2 * r0, r0_4 = r0_2 * r0_2;
    double t6 = 1.0 / ((r2 * r2) * r2 + r0_3 * r0_3);
    double t8 = 1.0 / ((r2 * r2) * (r2 * r2) + r0_4 * r0_4);
    double d6 = -(6.0 * (r2 * r2) * (t6 * t6));
    double d8 = -(8.0 * ((r2 * r2) * r2) * (t8 * t8));
    double e0 = D4_S6 * t6 + D4_S8 * rr * t8;
    double g0 = D4_S6 * d6 + D4_S8 * rr * d8;
    pe = sw * e0;
    pg = sw * g0 + dsw * e0 / r;
    return true;
}

// ATM pair tables of one molecule (dense nat x nat): w = sqrt|C6| * sw, t = (r0/r)^(alp/3)
// at q = 0 (crates/d4/src/disp.rs:614-665); thread per (a, k) element
__global__ void k_atm_tables(Batch B, State S, double* wt, double* tt, const long long* m_sq0, long long nsq) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nsq) return;
    int m = find_mol(m_sq0, B.nmol, g);
    long long gi = g - m_sq0[m];
    int n = B.m_nat[m], i0 = B.m_at0[m];
    int a = i0 + (int)(gi / n), k = i0 + (int)(gi % n);
    double w = 0.0, tv = 0.0;
    if (a != k) {
        double v[3];
        dvec(S.xyz, a, k, v);
        double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        if (r2 <= B.d3_cut * B.d3_cut && r2 >= DBL_EPSILON) {
            double r = sqrt(r2), sw, dsw;
            smooth_cut(r, B.d3_cut, B.d3_w, sw, dsw);
            double c6, da, db;
            pair_c6(B, S, a, k, c6, da, db);
            w = sqrt(fabs(c6)) * sw;
            double r0 = B.sp_r0[B.a_sp[a] * B.nsp + B.a_sp[k]];
            tv = pow(r0 / r, D4_ALP / 3.0);
        }
    }
    wt[m_sq0[m] + gi] = w;
    tt[m_sq0[m] + gi] = tv;
}

// ATM in the pair-sum form of the axtb conventions (crates/d4/src/disp.rs:666-733 and its term
// kernel 920-960): for every atom pair (a, b) the sum over third atoms k of the triple's damped
// angular term (ds) and its radial derivative (gs). Both sums are symmetric in a and b, so each
// unordered pair (a > b) is summed once, by one warp with lanes over k, into pairs[2 p]; the
// gather below turns them into each atom's energy, gradient and dE/dCN.
__global__ void k_atm_pairs(Batch B, State S, const double* wt, const double* tt, const long long* m_sq0,
                            const long long* m_pair0, long long np, double* pairs) {
    long long p = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (p >= np) return;
    int m = find_mol(m_pair0, B.nmol, p);
    long long pl = p - m_pair0[m];
    int la = (int)((sqrt(8.0 * (double)pl + 1.0) + 1.0) * 0.5);  // pl = la (la - 1) / 2 + lb, lb < la
    while ((long long)la * (la - 1) / 2 > pl) la--;
    while ((long long)(la + 1) * la / 2 <= pl) la++;
    int lb = (int)(pl - (long long)la * (la - 1) / 2);
    int n = B.m_nat[m], i0 = B.m_at0[m];
    int a = i0 + la, b = i0 + lb;
    double ds = 0.0, gs = 0.0;
    double vab[3];
    dvec(S.xyz, b, a, vab);
    double r2 = vab[0] * vab[0] + vab[1] * vab[1] + vab[2] * vab[2];
    if (r2 <= B.d3_cut * B.d3_cut && r2 >= DBL_EPSILON) {
        const double* W = wt + m_sq0[m];
        const double* T = tt + m_sq0[m];
        const double alp3 = D4_ALP / 3.0;
        double ir = 1.0 / sqrt(r2), t6 = 6.0 * T[(long long)la * n + lb];
        double r2_2 = r2 * r2;
        const double* wa = W + (long long)la * n;
        const double* wb = W + (long long)lb * n;
        const double* ta = T + (long long)la * n;
        const double* tb = T + (long long)lb * n;
        for (int lk = lane; lk < n; lk += 32) {
            double c = wa[lk] * wb[lk];
            if (c == 0.0) continue;
            int k = i0 + lk;
            double vak[3], vbk[3];
            dvec(S.xyz, k, a, vak);
            dvec(S.xyz, k, b, vbk);
            double r2ak = vak[0] * vak[0] + vak[1] * vak[1] + vak[2] * vak[2];
            double r2bk = vbk[0] * vbk[0] + vbk[1] * vbk[1] + vbk[2] * vbk[2];
            double cralp = t6 * ta[lk] * tb[lk];
            double fdmp = 1.0 / (1.0 + cralp);
            double ir1 = ir * rsqrt(r2ak * r2bk);  // 1 / (r_ab r_ak r_bk)
            double rrr2 = ir1 * ir1, rrr3 = rrr2 * ir1;
            double angf = 0.375 * rrr2 * rrr3;
            double s1 = r2ak + r2bk, d1 = (r2bk - r2ak) * (r2bk - r2ak);
            double ang = angf * ((r2_2 - d1) * (s1 - r2)) + rrr3;
            double cf = c * fdmp;
            ds += ang * cf;
            double pp = r2 * (r2 * (r2 + s1) + 2.0 * (s1 * s1) + d1) - 5.0 * (d1 * s1);
            gs += cf * (angf * pp - alp3 * (cralp * fdmp) * ang);
        }
        ds = warp_sum(ds);
        gs = warp_sum(gs);
    }
    if (lane == 0) {
        pairs[2 * p] = ds;
        pairs[2 * p + 1] = gs;
    }
}

// ATM energy, gradient and dE/dCN (D4 CN) per atom from the pair sums: atom a adds, over its
// partners b, -sw d / 6, the radial force and -d sw dC6/dCN_a / (2 C6), with
// d = -s9 sqrt|C6_ab| ds. One warp per atom, lanes over partners.
__global__ void k_atm_gather(Batch B, State S, const long long* m_pair0, const double* pairs) {
    int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (a >= B.natT) return;
    AtomView mv = mol_atoms(B, a);
    int n = mv.n, la = a - mv.i0;
    double ea = 0.0, ga[3] = {0, 0, 0}, dca = 0.0;
    for (int lb = lane; lb < n; lb += 32) {
        if (lb == la) continue;
        int b = mv.i0 + lb;
        double vab[3];
        dvec(S.xyz, b, a, vab);  // R_b - R_a
        double r2 = vab[0] * vab[0] + vab[1] * vab[1] + vab[2] * vab[2];
        if (r2 > B.d3_cut * B.d3_cut || r2 < DBL_EPSILON) continue;
        double r = sqrt(r2), sw, dsw;
        smooth_cut(r, B.d3_cut, B.d3_w, sw, dsw);
        if (sw <= 0.0) continue;
        long long pl = la > lb ? (long long)la * (la - 1) / 2 + lb : (long long)lb * (lb - 1) / 2 + la;
        const double* pp = pairs + 2 * (m_pair0[mv.m] + pl);
        double ds = pp[0], gs = pp[1];
        double c6, dda, ddb;
        pair_c6(B, S, a, b, c6, dda, ddb);
        double cab = -(D4_S9 * sqrt(fabs(c6)));
        double d = ds * cab, g = gs * cab;
        double de = sw * d;
        ea -= de / 6.0;
        double f = sw * g / r2 - (dsw / r) * d;
        for (int x = 0; x < 3; x++) ga[x] -= f * vab[x];
        double qa = c6 != 0.0 ? dda / c6 : 0.0;
        dca -= 0.5 * de * qa;
    }
    ea = warp_sum(ea);
    dca = warp_sum(dca);
    for (int x = 0; x < 3; x++) ga[x] = warp_sum(ga[x]);
    if (lane == 0) {
        S.e_atom[a] += ea;
        for (int x = 0; x < 3; x++) S.grad[3 * a + x] += ga[x];
        S.dedcn_d4[a] += dca;
    }
}

// EEQ system of each molecule (crates/axtb/src/eeq.rs:43-77): J (nat x nat, column-major) and
// right-hand side x; the charge constraint is applied after the solve (Schur complement).
__global__ void k_eeq_matrix(Batch B, State S, const long long* m_sq0, double* rhs, long long nsq) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nsq) return;
    int m = find_mol(m_sq0, B.nmol, g);
    long long gi = g - m_sq0[m];
    int n = B.m_nat[m], i0 = B.m_at0[m];
    int i = (int)(gi % n), j = (int)(gi / n);
    int a = i0 + i, b = i0 + j;
    double v;
    if (i == j) {
        v = B.a_eeq_eta[a] + sqrt(2.0 / 3.14159265358979323846) / B.a_eeq_rad[a];
        double cn = S.cn_eeq[a];
        rhs[a] = -B.a_eeq_chi[a] + B.a_eeq_kcn[a] / sqrt(cn + 1e-14) * cn;
    } else {
        double d[3];
        dvec(S.xyz, a, b, d);
        double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        double gam = 1.0 / (B.a_eeq_rad[a] * B.a_eeq_rad[a] + B.a_eeq_rad[b] * B.a_eeq_rad[b]);
        v = erf(sqrt(r2 * gam)) / sqrt(r2);
    }
    S.eeq_A[m_sq0[m] + gi] = v;
}

}  // namespace axg
