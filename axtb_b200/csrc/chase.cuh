// Stage 2 of the two-stage tridiagonal reduction (band -> tridiagonal by bulge chasing) with the
// band held in shared memory: its own launch between the eigen phase's stage 1 (k_team,
// PH_EIGEN) and the rest (k_team, PH_EIGEN_TAIL).
//
// In the team kernel the band of a one-CTA molecule lives in global memory (two CTAs share an SM
// and 66 KB of shared memory each), and every time step of the chase waits on a global-memory
// round per 32 x 32 block. Here one CTA takes a whole SM (up to 227 KB of shared memory): a band
// of up to CHASE_ROWS rows (2 BW diagonals, band and bulge, 512 B per row) sits in one CTA, and
// a band of up to 2 CHASE_ROWS rows is split by rows over the two CTAs of a cluster, each warp
// reading and writing the partner's rows through distributed shared memory. No tile per warp: a
// task works on the band storage itself (the block below its window stays there until the next
// step of the sweep), so the arithmetic is that of the global-memory chase operation for
// operation and the results are the same bits.
//
// Schedule: a task (sweep j, step s) runs on a slot of three warps, one per block it updates
// (the diagonal block two-sided, the rest of the previous block below from the left, the block
// below from the right); each of the three computes the task's reflector from the same column
// (the same bits). Sweep j takes slot j mod NS (NS = 5 slots for one CTA, 10 for a cluster
// pair), sweep j+1 three time steps behind sweep j (the tasks of one time step touch disjoint
// elements), one CTA barrier (or cluster barrier) per time step. The molecules of a launch: the
// large ones on the clusters, then the others one per CTA (host-side plan, longest first).
#pragma once
#include "team_band.cuh"

namespace axg {

constexpr int CHASE_SLOTS = 5;                                   // concurrent tasks per CTA
constexpr int CHASE_WARPS = 3 * CHASE_SLOTS;                     // three warps per task
constexpr int CHASE_THREADS = 32 * CHASE_WARPS;
constexpr int CHASE_ROWS = 440;                                  // band rows per CTA
constexpr int CHASE_DYN_BYTES = CHASE_ROWS * LDB * 8;            // 225,280 B of dynamic shared memory
constexpr int CHASE_MAX_NAO = 2 * CHASE_ROWS;                    // the largest band a cluster pair holds
constexpr int CHASE_STATIC_BYTES = (CHASE_WARPS + CHASE_SLOTS) * BW * 8;  // per-warp v, per-slot w
static_assert(CHASE_DYN_BYTES + CHASE_STATIC_BYTES <= 227 * 1024, "one CTA per SM: 227 KB at most");
// three time steps between sweeps (disjoint tasks) need ceil(steps of sweep 0 / slots) <= 3
static_assert((CHASE_ROWS - 1 + BW - 1) / BW <= 3 * CHASE_SLOTS, "one CTA: at most three steps per slot");
static_assert((CHASE_MAX_NAO - 1 + BW - 1) / BW <= 3 * 2 * CHASE_SLOTS, "a pair: at most three steps per slot");

struct ChasePlan {
    const int* pair_off;   // per cluster: range into pair_list (molecules above CHASE_ROWS AOs)
    const int* pair_list;
    const int* solo_off;   // per CTA: range into solo_list
    const int* solo_list;
    int cycles;            // 1: add the chase's SM cycles to g_team_cycles[17] and the molecule's counter
};

// Band element (r, c), r >= c, r - c < LDB, at row r, slot r - c. One CTA (PAIR false) indexes
// its own shared memory. A cluster pair holds rows [0, h) in rank 0 and rows [h, n) in rank 1 and
// addresses both through the cluster's shared window (32-bit addresses, one select per row).
template <bool PAIR>
struct BandRef;

template <>
struct BandRef<false> {
    __device__ __forceinline__ double ld(int r, int c) const { return s_work[r * LDB + (r - c)]; }
    __device__ __forceinline__ void st(int r, int c, double v) const { s_work[r * LDB + (r - c)] = v; }
};

template <>
struct BandRef<true> {
    unsigned a0, a1;  // rows 0.. at a0; rows h.. at a1 (a1 - h LDB 8 bytes: row r at a1 + r LDB 8)
    int h;
    __device__ __forceinline__ unsigned addr(int r, int c) const {
        return (r < h ? a0 : a1) + (unsigned)(r * LDB + (r - c)) * 8u;
    }
    __device__ __forceinline__ double ld(int r, int c) const {
        double v;
        asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(addr(r, c)));
        return v;
    }
    __device__ __forceinline__ void st(int r, int c, double v) const {
        asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(addr(r, c)), "d"(v) : "memory");
    }
};

// One task (sweep j, step s) on the band, in place, by the three warps of a slot: role 0 the
// diagonal block (two-sided), role 1 the rest of the previous block below (from the left, step
// s > 0), role 2 the block below (from the right). The operations of warp_chase on the same
// values in the same order (the same bits). Each warp loads its block into registers first (no
// other task of the time step touches it), and the three read the column to annihilate before
// role 0 overwrites it (a barrier of the slot's 96 threads). vs: the warp's copy of the
// reflector; ws: the slot's w vector (role 0).
template <bool PAIR>
__device__ __forceinline__ void chase_task(const BandRef<PAIR>& b, int role, int slot, int n, int j, int s,
                                           double* vs, double* ws, double* refl) {
    const int lane = threadIdx.x & 31;
    const int lo = j + 1 + s * BW, hi = min(lo + BW - 1, n - 1), L = hi - lo + 1;
    const int pc = s == 0 ? j : lo - BW;  // the column to annihilate
    const int elo = hi + 1, ehi = min(hi + BW, n - 1), LE = ehi - elo + 1;
    double x = lane < L ? b.ld(lo + lane, pc) : 0.0;
    double a[BW];
    bool mine;  // this lane updates entries of the role's block
    if (role == 0) {
        mine = lane < L;
#pragma unroll
        for (int r = 0; r < BW; r++)
            a[r] = mine && r < L ? (r >= lane ? b.ld(lo + r, lo + lane) : b.ld(lo + lane, lo + r)) : 0.0;
    } else if (role == 1) {
        mine = s > 0 && lane >= 1;
#pragma unroll
        for (int r = 0; r < BW; r++) a[r] = mine && r < L ? b.ld(lo + r, pc + lane) : 0.0;
    } else {
        mine = lane < LE;
#pragma unroll
        for (int r = 0; r < BW; r++) a[r] = mine && r < L ? b.ld(elo + lane, lo + r) : 0.0;
    }
    asm volatile("bar.sync %0, 96;" ::"r"(1 + slot) : "memory");  // the column is read by all three
    double alpha = __shfl_sync(0xffffffffu, x, 0);
    double xn2 = warp_sum(lane >= 1 && lane < L ? x * x : 0.0);
    double beta, tc, scale;
    if (L < 2 || xn2 == 0.0) {
        tc = 0.0;
        beta = alpha;
        scale = 0.0;
    } else {
        beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
        tc = (beta - alpha) / beta;
        scale = 1.0 / (alpha - beta);
    }
    double v = lane == 0 ? 1.0 : (lane < L ? x * scale : 0.0);
    vs[lane] = v;
    if (role == 0) {
        double* rf = refl + band_refl_index(n, j, s) * BW;
        rf[lane] = lane == 0 ? tc : v;
        if (lane < L) b.st(lo + lane, pc, lane == 0 ? beta : 0.0);
    }
    __syncwarp();
    if (tc == 0.0) return;
    if (role == 0) {
        // the diagonal block lo..hi: y = tau D v, w = y - tau/2 (v.y) v, D -= v w^T + w v^T
        double y = 0.0;
#pragma unroll
        for (int r = 0; r < BW; r++)
            if (r < L) y = fma(a[r], vs[r], y);
        y *= tc;
        double K = -0.5 * tc * warp_sum(lane < L ? v * y : 0.0);
        ws[lane] = y + K * v;
        __syncwarp();
        if (mine) {
            const double wl = ws[lane];
#pragma unroll
            for (int r = 0; r < BW; r++)
                if (r < L && r >= lane) b.st(lo + r, lo + lane, a[r] - (vs[r] * wl + ws[r] * v));
        }

    } else if (role == 1) {
        // step s > 0: the reflector from the left on the other columns of the previous block below
        if (mine) {
            double w = 0.0;
#pragma unroll
            for (int r = 0; r < BW; r++)
                if (r < L) w = fma(vs[r], a[r], w);
            const double tw = tc * w;
#pragma unroll
            for (int r = 0; r < BW; r++)
                if (r < L) b.st(lo + r, pc + lane, a[r] - tw * vs[r]);
        }
    } else if (mine) {
        // the block below (rows elo..ehi, columns lo..hi) from the right, lane = row
        double u = 0.0;
#pragma unroll
        for (int c = 0; c < BW; c++)
            if (c < L) u = fma(a[c], vs[c], u);
        const double tu = tc * u;
#pragma unroll
        for (int c = 0; c < BW; c++)
            if (c < L) b.st(elo + lane, lo + c, a[c] - tu * vs[c]);
    }
}

__device__ __forceinline__ void cluster_barrier() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

template <bool PAIR>
__device__ __forceinline__ void chase_sync() {
    if (PAIR) cluster_barrier();
    else __syncthreads();
}

// Stage 2 of molecule m (stage 1 left the band in the lower diagonals 0..BW of F'): d, e get the
// tridiagonal matrix, the reflectors go to the W plane (band_refl_index order)
template <bool PAIR>
__device__ void chase_mol(const Batch& B, State& S, const ChasePlan& C, int m, int rank, double (*s_v)[BW],
                          double (*s_w)[BW]) {
    long long c0 = clock64();
    const int n = B.m_nao[m], ao0 = B.m_ao0[m];
    const long long mat = B.m_mat0[m];
    const double* A = S.Fp + mat;  // leading dimension n
    const int h = PAIR ? (n + 1) / 2 : n;
    BandRef<PAIR> b;
    if constexpr (PAIR) {
        unsigned self = (unsigned)__cvta_generic_to_shared(s_work), r0, r1;
        asm volatile("mapa.shared::cluster.u32 %0, %1, 0;" : "=r"(r0) : "r"(self));
        asm volatile("mapa.shared::cluster.u32 %0, %1, 1;" : "=r"(r1) : "r"(self));
        b.a0 = r0;
        b.a1 = r1 - (unsigned)(h * LDB * 8);
        b.h = h;
    }
    const int my0 = PAIR && rank == 1 ? h : 0, my1 = PAIR && rank == 0 ? h : n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int q = threadIdx.x; q < (my1 - my0) * LDB; q += blockDim.x) s_work[q] = 0.0;
    chase_sync<PAIR>();
    // the band from A's lower triangle: a warp per column of this CTA's rows, lanes down the
    // column (coalesced), element (c + BW, c) by lane 0
    for (int c = my0 + warp; c < my1; c += CHASE_WARPS) {
        const double* ac = A + (long long)c * n;
        if (c + lane < n) b.st(c + lane, c, ac[c + lane]);
        if (lane == 0 && c + BW < n) b.st(c + BW, c, ac[c + BW]);
    }
    chase_sync<PAIR>();
    double* refl = S.W + mat;
    if (n > 2) {
        const int NS = PAIR ? 2 * CHASE_SLOTS : CHASE_SLOTS;
        const int slot = warp / 3, role = warp - 3 * slot;
        const int g = (PAIR ? rank * CHASE_SLOTS : 0) + slot;
        const int S0 = band_steps(n);
        const int lam = max(3, (S0 + NS - 1) / NS);
        const int nsweep = n - 2;
        const int tend = lam * (nsweep - 1) + S0;
        for (int t = 0; t < tend; t++) {
            int jm = min(t / lam, nsweep - 1);
            int j = jm - (((jm - g) % NS) + NS) % NS;
            if (j >= 0) {
                int s = t - lam * j;
                if (s < band_steps(n - j)) chase_task<PAIR>(b, role, slot, n, j, s, s_v[warp], s_w[slot], refl);
            }
            chase_sync<PAIR>();
        }
    }
    double* d = S.dtri + ao0;
    double* e = S.etri + ao0;
    for (int i = my0 + threadIdx.x; i < my1; i += blockDim.x) {
        d[i] = b.ld(i, i);
        e[i] = i + 1 < n ? b.ld(i + 1, i) : 0.0;
    }
    chase_sync<PAIR>();  // the partner has read this CTA's rows before they are overwritten
    if (C.cycles && threadIdx.x == 0 && rank == 0) {
        // in units of a team-kernel CTA (half an SM): a whole SM counts twice, a pair four times
        double cyc = (double)(clock64() - c0) * (PAIR ? 4.0 : 2.0);
        atomicAdd(&g_team_cycles[17], (unsigned long long)cyc);
        S.mol_cyc[m] += cyc;
    }
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(CHASE_THREADS, 1)
    k_chase(Batch B, State S, ChasePlan C) {
    __shared__ double s_v[CHASE_WARPS][BW], s_w[CHASE_SLOTS][BW];
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int cid = blockIdx.x >> 1;
    for (int i = C.pair_off[cid]; i < C.pair_off[cid + 1]; i++) {
        int m = C.pair_list[i];
        if (S.active[m]) chase_mol<true>(B, S, C, m, rank, s_v, s_w);  // same on both CTAs
    }
    for (int i = C.solo_off[blockIdx.x]; i < C.solo_off[blockIdx.x + 1]; i++) {
        int m = C.solo_list[i];
        if (S.active[m]) chase_mol<false>(B, S, C, m, 0, s_v, s_w);
    }
}

}  // namespace axg
