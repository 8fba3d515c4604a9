// Two-stage reduction of a symmetric matrix to tridiagonal form, for the one-CTA teams (molecules
// below the whole-grid size): the reference diagonalises the reduced Fock matrix with faer's
// one-stage tridiagonalisation (crates/base/src/linalg/eigen.rs:213-296, tridiag.rs:55,376); the
// eigenvalues and the occupied subspace are unique, so any orthogonal reduction gives the same
// energies to round-off. The one-stage reduction streams the whole trailing matrix once per column
// (a chain of dependent load rounds from HBM, n^3/6 x 8 bytes); here:
//
//   stage 1  dense -> band of half-width BW (panels of BW columns): a Householder QR of each panel
//            below the band, then the two-sided update of the trailing matrix as DMMA GEMMs
//            (Y = A V with A read from its lower triangle, W = Y T - V (T^T V^T Y T) / 2,
//            A -= V W^T + W V^T): the n^3 work moves into GEMMs and the matrix is read ~3n/BW
//            times instead of n times;
//   stage 2  band -> tridiagonal by bulge chasing: sweep j annihilates column j below the
//            subdiagonal with a reflector on rows j+1..j+BW, and each later step s of the sweep
//            annihilates the first column of the bulge the previous reflector left below the band
//            (a reflector on rows j+1+s BW .. j+(s+1) BW) and applies it to the diagonal block
//            and the block below. Sweep j+1 runs three steps behind sweep j (the tasks at one
//            time step touch disjoint elements), one warp per sweep, the band (and its bulge, 2 BW
//            diagonals) in global memory by rows with each task's 32 x 32 blocks in the warp's
//            shared tile;
//   back     Z <- Q2 Z, then Z <- Q1 Z: the stage-2 reflectors of 32 consecutive sweeps at one
//            step form a 64 x 64 orthogonal block (explicit, applied as a GEMM to 64 rows of Z;
//            groups from the last, steps in ascending order, which respects every overlap), then
//            the stage-1 panels from the last as compact-WY blocks.
#pragma once
#include "team_la.cuh"

namespace axg {

constexpr int BW = 32;       // half-bandwidth of the intermediate band matrix
constexpr int LDB = 2 * BW;  // band storage per column: diagonals 0 .. 2 BW - 1 (band and bulge)
constexpr int BWARPS = TEAM_THREADS / 32;
static_assert(BW == 32 && BWARPS * 32 * (BW + 1) <= SMEM_WORK, "stage-2 tiles: one 32 x 33 tile per warp");
static_assert(2 * 64 * 65 <= SMEM_WORK, "two 64 x 64 stage-2 blocks fit the work area");

// Per-molecule workspace of the two-stage path (doubles), in this order: scalars (8), beta
// occupations (n), then V, Y, X (n x BW each), G/VX/M (3 BW^2), the panels' T factors
// (ceil(n/BW) BW^2), the band (LDB n), the group blocks (64^2 per step of a group), and the
// GEMM result of one block (64 n).
__host__ __device__ constexpr int band_steps(int n) { return (n - 1 + BW - 1) / BW; }
__host__ __device__ constexpr long long band_off_v(int n) { return 8LL + ((n + 7) / 8) * 8LL; }
__host__ __device__ constexpr long long band_off_y(int n) { return band_off_v(n) + (long long)BW * n; }
__host__ __device__ constexpr long long band_off_x(int n) { return band_off_y(n) + (long long)BW * n; }
__host__ __device__ constexpr long long band_off_small(int n) { return band_off_x(n) + (long long)BW * n; }
__host__ __device__ constexpr long long band_off_t(int n) { return band_off_small(n) + 3LL * BW * BW; }
__host__ __device__ constexpr long long band_off_band(int n) {
    return band_off_t(n) + (long long)((n + BW - 1) / BW) * BW * BW;
}
__host__ __device__ constexpr long long band_off_blocks(int n) { return band_off_band(n) + (long long)LDB * n; }
__host__ __device__ constexpr long long band_off_tmp(int n) {
    return band_off_blocks(n) + (long long)(band_steps(n) + 1) * 64 * 64;
}
__host__ __device__ constexpr long long band_workspace(int n) { return band_off_tmp(n) + 64LL * n; }

// Per-molecule workspace of the team kernel (doubles): the larger of the two-stage path's and the
// whole-grid path's (one-stage reduction: the column vectors, the symmetric product's slots and
// the V, W panels; the back-transformation's Vb, T, G, Y, Y2), which also covers the Cholesky's
// and the triangular inverse's (CB x CB + 1, CB x n)
__host__ __device__ constexpr long long onestage_workspace(int n) {
    return (2LL + symv_slots(n)) * (n < 64 ? 64 : n) + 64LL * (n < 64 ? 64 : n) + 2LL * 64 * 64 +
           2LL * 64 * (n < 64 ? 64 : n) + 64LL * (n < 64 ? 64 : n) + 64;
}
__host__ __device__ constexpr long long team_workspace(int n) {
    return band_workspace(n) > onestage_workspace(n) ? band_workspace(n) : onestage_workspace(n);
}

// F(x) = sum_{m=1}^{x} ceil(m / BW): stage-2 reflector (j, s) of an n x n matrix is number
// F(n-1) - F(n-1-j) + s (sweep j has ceil((n-1-j)/BW) steps); each takes BW doubles
// (tau, v_1 .. v_{BW-1}; v_0 = 1)
__host__ __device__ __forceinline__ long long band_prefix(long long x) {
    long long q = x / BW, r = x % BW;
    return BW * q * (q + 1) / 2 + r * (q + 1);
}
__host__ __device__ __forceinline__ long long band_refl_index(int n, int j, int s) {
    return band_prefix(n - 1) - band_prefix(n - 1 - j) + s;
}

// ---------------------------------------------------------------------------------- stage 1
// Householder QR of the m x nb panel P (leading dimension ld) with nr reflectors: reflector c
// acts on rows c..m-1, v_c = 1 at row c, kept below it in P; R above and on the diagonal; tau[c].
// Each reflector is also staged in shared memory; warp w updates the columns q = w (mod 8), all
// of them in one pass over the rows (their dot products together, then their updates), and the
// warp owning column c + 1 also forms its norm for the next reflector. Two CTA barriers per
// column.
__device__ void cta_panel_qr(double* P, long long ld, int m, int nb, int nr, double* tau) {
    __shared__ double s_xn2, s_alpha;
    double* sv = s_work;  // the current reflector (m values)
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int QW = (BW + BWARPS - 1) / BWARPS;  // columns per warp
    if (warp == 0) {
        double xs = 0.0;
        for (int i = 1 + lane; i < m; i += 32) xs += sq(P[i]);
        xs = warp_sum(xs);
        if (lane == 0) {
            s_xn2 = xs;
            s_alpha = P[0];
        }
    }
    __syncthreads();
    for (int c = 0; c < nr; c++) {
        double* pc = P + (long long)c * ld;
        double xn2 = s_xn2, alpha = s_alpha, beta, tc, scale;
        if (xn2 == 0.0) {
            tc = 0.0;
            beta = alpha;
            scale = 0.0;
        } else {
            beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
            tc = (beta - alpha) / beta;
            scale = 1.0 / (alpha - beta);
        }
        for (int i = c + 1 + threadIdx.x; i < m; i += blockDim.x) {
            double v = pc[i] * scale;
            pc[i] = v;
            sv[i] = v;
        }
        __syncthreads();  // v visible; every thread has read s_xn2 and s_alpha
        if (threadIdx.x == 0) {
            pc[c] = beta;
            tau[c] = tc;
        }
        int q0 = c + 1 + ((warp - (c + 1)) % BWARPS + BWARPS) % BWARPS;
        double* pq[QW];
        bool on[QW];
        double w[QW];
#pragma unroll
        for (int u = 0; u < QW; u++) {
            int q = q0 + u * BWARPS;
            on[u] = q < nb;
            pq[u] = P + (long long)(on[u] ? q : c) * ld;
            w[u] = 0.0;
        }
        if (q0 < nb) {  // uniform over the warp
#pragma unroll 4
            for (int i = c + 1 + lane; i < m; i += 32) {
                double vi = sv[i];
#pragma unroll
                for (int u = 0; u < QW; u++)
                    if (on[u]) w[u] = fma(vi, pq[u][i], w[u]);
            }
            double tw[QW];
#pragma unroll
            for (int u = 0; u < QW; u++) tw[u] = on[u] ? tc * (warp_sum(w[u]) + pq[u][c]) : 0.0;
            __syncwarp();  // every lane has read the pq[u][c]
            if (lane == 0)
#pragma unroll
                for (int u = 0; u < QW; u++)
                    if (on[u]) pq[u][c] -= tw[u];
            double xs = 0.0;  // the norm below row c + 1 of column c + 1 (owned by u = 0 when q0 = c + 1)
#pragma unroll 4
            for (int i = c + 1 + lane; i < m; i += 32) {
                double vi = sv[i];
#pragma unroll
                for (int u = 0; u < QW; u++)
                    if (on[u]) {
                        double x = pq[u][i] - tw[u] * vi;
                        pq[u][i] = x;
                        if (u == 0 && i > c + 1) xs += x * x;
                    }
            }
            if (q0 == c + 1) {
                xs = warp_sum(xs);
                __syncwarp();
                if (lane == 0) {
                    s_xn2 = xs;
                    s_alpha = pq[0][c + 1];
                }
            }
        }
        __syncthreads();
    }
}

// T (nr x nr, upper, leading dimension BW) of the compact-WY form H_0 .. H_{nr-1} = I - V T V^T
// from G = V^T V (leading dimension BW) and tau (LAPACK dlarft, forward columnwise), one warp
__device__ void warp_larft(const double* G, const double* tau, int nr, double* T) {
    int lane = threadIdx.x & 31;
    for (int q = lane; q < BW * BW; q += 32) T[q] = 0.0;
    __syncwarp();
    for (int c = 0; c < nr; c++) {
        double tc = tau[c];
        double s = 0.0;
        if (lane < c)
            for (int q = lane; q < c; q++) s += T[lane + q * BW] * G[q + c * BW];
        __syncwarp();
        if (lane < c) T[lane + c * BW] = -tc * s;
        if (lane == 0) T[c + c * BW] = tc;
        __syncwarp();
    }
}

// Stage 1 on A (n x n, lower triangle, leading dimension lda): afterwards A's diagonals 0..BW
// hold the band and the stage-1 reflectors lie below it in the panel columns (panel p: columns
// p BW .., reflector c with its unit at row p BW + BW + c); tau gets the reflector factors at the
// panel column, the T factor of panel p is kept at wk + band_off_t(n) + p BW^2.
__device__ void team_sy2sb(const Team& t, double* A, long long lda, int n, double* tau, double* wk) {
    double* V = wk + band_off_v(n);
    double* Y = wk + band_off_y(n);
    double* X = wk + band_off_x(n);
    double* G = wk + band_off_small(n);
    double* VX = G + BW * BW;
    double* M = VX + BW * BW;
    for (int p = 0;; p++) {
        int j0 = p * BW, r0 = j0 + BW, m = n - r0;
        if (m < 2) break;
        int nb = min(BW, n - j0), nr = min(nb, m - 1);
        double* P = A + r0 + (long long)j0 * lda;
        double* T = wk + band_off_t(n) + (long long)p * BW * BW;
        cta_panel_qr(P, lda, m, nb, nr, tau + j0);
        // explicit V (m x nr, leading dimension m): unit at row c, zeros above
        for (long long q = threadIdx.x; q < (long long)m * nr; q += blockDim.x) {
            int i = (int)(q % m), c = (int)(q / m);
            V[q] = i == c ? 1.0 : (i > c ? P[i + (long long)c * lda] : 0.0);
        }
        __syncthreads();
        team_gemm(t, true, false, nr, nr, m, 1.0, V, m, V, m, 0.0, G, BW);
        if (threadIdx.x < 32) warp_larft(G, tau + j0, nr, T);
        double* A22 = A + r0 + (long long)r0 * lda;
        // Y = A22 V (A22 from its lower triangle)
        team_gemm(t, false, false, m, nr, m, 1.0, A22, lda, V, m, 0.0, Y, m, GEMM_A_SYMM);
        // X = Y T; VX = V^T X; M = T^T VX; W = X - V M / 2 (in X)
        team_gemm(t, false, false, m, nr, nr, 1.0, Y, m, T, BW, 0.0, X, m, GEMM_B_UPPER);
        team_gemm(t, true, false, nr, nr, m, 1.0, V, m, X, m, 0.0, VX, BW);
        team_gemm(t, true, false, nr, nr, nr, 1.0, T, BW, VX, BW, 0.0, M, BW);
        team_gemm(t, false, false, m, nr, nr, -0.5, V, m, M, BW, 1.0, X, m);
        // A22 -= V W^T + W V^T (lower tiles)
        team_gemm(t, false, true, m, m, nr, -1.0, V, m, X, m, 1.0, A22, lda, GEMM_LOWER_TILES);
        team_gemm(t, false, true, m, m, nr, -1.0, X, m, V, m, 1.0, A22, lda, GEMM_LOWER_TILES);
    }
}

// ---------------------------------------------------------------------------------- stage 2
// band element (r, c) of the lower band storage (r >= c, r - c < LDB), stored by rows: a warp
// whose lanes take consecutive columns of one row reads and writes consecutive addresses
__device__ __forceinline__ double* band_at(double* bd, int r, int c) { return bd + (long long)r * LDB + (r - c); }

// One bulge-chasing task (sweep j, step s) by one warp with its tile Tl (32 x 33) and vector
// slots vs, ws (32 each). The tile holds, between steps of a sweep, the block below the previous
// window (after the previous reflector was applied from the right).
__device__ void warp_chase(double* bd, int n, int j, int s, double (*Tl)[BW + 1], double* vs, double* ws,
                           double* refl) {
    int lane = threadIdx.x & 31;
    int lo = j + 1 + s * BW, hi = min(lo + BW - 1, n - 1), L = hi - lo + 1;
    int pc = s == 0 ? j : lo - BW;
    int elo = hi + 1, ehi = min(hi + BW, n - 1), LE = ehi - elo + 1;  // block below (LE <= 0: none)
    // the column to annihilate: column j (s = 0) or the tile's first column
    double x = 0.0;
    if (lane < L) x = s == 0 ? *band_at(bd, lo + lane, j) : Tl[lane][0];
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
    double* rf = refl + band_refl_index(n, j, s) * BW;
    rf[lane] = lane == 0 ? tc : v;
    __syncwarp();
    if (s == 0) {
        if (lane < L) *band_at(bd, lo + lane, j) = lane == 0 ? beta : 0.0;
    } else {
        // the annihilated column, then the reflector from the left on the tile's other columns
        // (columns pc+1 .. lo-1), and the block back to the band
        if (lane < L) Tl[lane][0] = lane == 0 ? beta : 0.0;
        if (lane >= 1 && tc != 0.0) {
            double w = 0.0;
            for (int r = 0; r < L; r++) w = fma(vs[r], Tl[r][lane], w);
            double tw = tc * w;
            for (int r = 0; r < L; r++) Tl[r][lane] -= tw * vs[r];
        }
        __syncwarp();
        for (int r = 0; r < L; r++) *band_at(bd, lo + r, pc + lane) = Tl[r][lane];
    }
    if (tc == 0.0 && LE <= 0) return;
    __syncwarp();
    // the diagonal block lo..hi, two-sided: y = tau D v, w = y - tau/2 (v.y) v, D -= v w^T + w v^T
    // (loads in batches of 16 independent ones per lane)
    // the lower triangle by rows (coalesced), then mirrored in the tile
    if (lane < L) {
#pragma unroll
        for (int r0 = 0; r0 < BW; r0 += 16) {
            double tv[16];
#pragma unroll
            for (int u = 0; u < 16; u++) {
                int r = r0 + u;
                tv[u] = (r < L && r >= lane) ? *band_at(bd, lo + r, lo + lane) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 16; u++)
                if (r0 + u >= lane) Tl[r0 + u][lane] = tv[u];
        }
    }
    __syncwarp();
    if (lane < L)
        for (int c = lane + 1; c < L; c++) Tl[lane][c] = Tl[c][lane];
    __syncwarp();
    if (tc != 0.0) {
        double y = 0.0;
        if (lane < L)
            for (int r = 0; r < L; r++) y = fma(Tl[r][lane], vs[r], y);
        y *= tc;
        double K = -0.5 * tc * warp_sum(lane < L ? v * y : 0.0);
        ws[lane] = y + K * v;
        __syncwarp();
        if (lane < L) {
            double wl = ws[lane];
            for (int r = 0; r < L; r++) {  // row by row: the lanes write consecutive addresses
                double d = Tl[r][lane] - (vs[r] * wl + ws[r] * v);
                if (r >= lane) *band_at(bd, lo + r, lo + lane) = d;
            }
        }
        __syncwarp();
    }
    // the block below (rows elo..ehi, columns lo..hi) from the right; it stays in the tile
    if (LE > 0) {
        if (lane < L) {
#pragma unroll
            for (int r0 = 0; r0 < BW; r0 += 16) {
                double tv[16];
#pragma unroll
                for (int u = 0; u < 16; u++) {
                    int r = r0 + u;
                    tv[u] = r < LE ? *band_at(bd, elo + r, lo + lane) : 0.0;
                }
#pragma unroll
                for (int u = 0; u < 16; u++) Tl[r0 + u][lane] = tv[u];
            }
        }
        __syncwarp();
        if (lane < LE && tc != 0.0) {
            double u = 0.0;
            for (int c = 0; c < L; c++) u = fma(Tl[lane][c], vs[c], u);
            double tu = tc * u;
            for (int c = 0; c < L; c++) Tl[lane][c] -= tu * vs[c];
        }
        __syncwarp();
    }
}

// Stage 2 on the band kept in A's diagonals 0..BW (after team_sy2sb): d, e get the tridiagonal
// matrix; the reflectors go to refl (band_refl_index order). One CTA.
__device__ void team_sb2st(const Team& t, const double* A, long long lda, int n, double* d, double* e, double* wk,
                           double* refl) {
    __shared__ double s_v[BWARPS][BW], s_w[BWARPS][BW];
    double* bd = wk + band_off_band(n);
    for (long long q = threadIdx.x; q < (long long)LDB * n; q += blockDim.x) {
        int dg = (int)(q % LDB);
        int r = (int)(q / LDB);  // row r, diagonal dg: element (r, r - dg)
        bd[q] = (dg <= BW && r - dg >= 0) ? A[r + (long long)(r - dg) * lda] : 0.0;
    }
    __syncthreads();
    int warp = threadIdx.x >> 5;
    auto Tl = reinterpret_cast<double(*)[BW + 1]>(s_work + warp * BW * (BW + 1));
    if (n > 2) {
        const int S0 = band_steps(n);
        const int lam = max(3, (S0 + BWARPS - 1) / BWARPS);
        const int nsweep = n - 2;
        const int tend = lam * (nsweep - 1) + S0;
        for (int tau_ = 0; tau_ < tend; tau_++) {
            // this warp's sweep: the latest j = warp (mod BWARPS) started by now
            int jm = min(tau_ / lam, nsweep - 1);
            int j = jm - (((jm - warp) % BWARPS) + BWARPS) % BWARPS;
            if (j >= 0) {
                int s = tau_ - lam * j;
                if (s < band_steps(n - j)) warp_chase(bd, n, j, s, Tl, s_v[warp], s_w[warp], refl);
            }
            __syncthreads();
        }
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        d[i] = *band_at(bd, i, i);
        e[i] = i + 1 < n ? *band_at(bd, i + 1, i) : 0.0;
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------------- back
// Z <- Q2 Z (Z: n x k, leading dimension ldz) from the stage-2 reflectors, one CTA. Per group of
// 32 sweeps (from the last) and step s (ascending; this order respects every overlap), the 32
// reflectors of the group at step s form an explicit 64 x 64 orthogonal block X_s on the rows
// from J + 1 + s BW: built in shared memory (thread = column, the reflectors in order), then
// applied in place, Z[w0 : w0 + 64] <- X_s Z[w0 : w0 + 64], on the FP64 tensor cores with X_s
// kept in shared memory and Z streamed through a three-deep ring of 64 x 16 column chunks
// (cp.async; each chunk is read, multiplied and stored before the ring reuses its slot).
constexpr int Q2_XLD = 68;  // X_s row stride (doubles): conflict-free fragment loads
constexpr int Q2_ZC = 16;   // Z columns per chunk
constexpr int Q2_ZLD = 20;  // chunk row stride (doubles)
constexpr int Q2_STAGES = 3;
static_assert(64 * Q2_XLD + Q2_STAGES * 64 * Q2_ZLD <= SMEM_WORK && BW * BW <= Q2_STAGES * 64 * Q2_ZLD,
              "X_s and the chunk ring (or the staged reflectors) fit the work area");

__device__ void cta_q2_block(const double* X, double* Z, long long ldz, int rows, int k) {
    double* ring = s_work + 64 * Q2_XLD;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = warp & 3, wn = warp >> 2;  // warp tile: rows wm*16 .. +16, chunk columns wn*8 .. +8
    const int lr = lane >> 2, lc = lane & 3;
    const int nch = (k + Q2_ZC - 1) / Q2_ZC;
    auto issue = [&](int ch) {
        if (ch < nch) {
            double* st = ring + (ch % Q2_STAGES) * 64 * Q2_ZLD;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                int e = threadIdx.x + q * 256;
                int r = e & 63, c = e >> 6;
                int gc = ch * Q2_ZC + c;
                bool ok = r < rows && gc < k;
                cp_async8(st + r * Q2_ZLD + c, ok ? Z + r + (long long)gc * ldz : Z, ok);
            }
        }
        cp_async_commit();
    };
    issue(0);
    issue(1);
    for (int ch = 0; ch < nch; ch++) {
        cp_async_wait<1>();  // this thread's copies of chunk ch have landed
        __syncthreads();     // everyone's have; the slot of chunk ch - 1 is free
        issue(ch + 2);
        const double* zs = ring + (ch % Q2_STAGES) * 64 * Q2_ZLD;
        double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
        for (int kk = 0; kk < 64; kk += 4) {
            double bf = zs[(kk + lc) * Q2_ZLD + wn * 8 + lr];
#pragma unroll
            for (int i = 0; i < 2; i++) {
                double af = X[(wm * 16 + i * 8 + lr) * Q2_XLD + kk + lc];
                dmma_8x8x4(acc[i][0], acc[i][1], af, bf);
            }
        }
#pragma unroll
        for (int i = 0; i < 2; i++) {
            int r = wm * 16 + i * 8 + lr;
#pragma unroll
            for (int h = 0; h < 2; h++) {
                int gc = ch * Q2_ZC + wn * 8 + lc * 2 + h;
                if (r < rows && gc < k) Z[r + (long long)gc * ldz] = acc[i][h];
            }
        }
    }
    cp_async_wait<0>();
    __syncthreads();  // the work area is free for the next block
}

__device__ void team_apply_q2(const Team& t, int n, int k, double* Z, long long ldz, const double* refl, double* wk) {
    if (n <= 2 || k <= 0) return;
    const int nsweep = n - 2;
    double* X = s_work;  // 64 x Q2_XLD
    for (int J = ((nsweep - 1) / BW) * BW; J >= 0; J -= BW) {
        int ns = band_steps(n - J);  // steps of the group's first sweep (the longest)
        for (int s = 0; s < ns; s++) {
            int w0 = J + 1 + s * BW, rows = min(64, n - w0);
            if (rows <= 0) break;
            // the group's reflectors at step s, staged in shared memory by every thread (the
            // chunk ring's space, free until the product), tau = 0 for sweeps without the step
            double* R = s_work + 64 * Q2_XLD;
            for (int q = threadIdx.x; q < BW * BW; q += blockDim.x) {
                int j = J + q / BW;
                bool has = j < nsweep && s < band_steps(n - j);
                R[q] = has ? refl[band_refl_index(n, j, s) * BW + q % BW] : 0.0;
            }
            __syncthreads();
            // X_s = H_{J,s} H_{J+1,s} .. H_{J+31,s} on the 64 rows from w0 (thread = column)
            int col = threadIdx.x;
            if (col < 64) {
                for (int r = 0; r < 64; r++) X[r * Q2_XLD + col] = r == col ? 1.0 : 0.0;
                for (int dl = BW - 1; dl >= 0; dl--) {
                    const double* rf = R + dl * BW;
                    double tc = rf[0];
                    if (tc == 0.0) continue;
                    int lo = J + dl + 1 + s * BW, L = min(BW, n - lo);
                    int r0 = lo - w0;  // = dl
                    double w = X[r0 * Q2_XLD + col];
                    for (int r = 1; r < L; r++) w = fma(rf[r], X[(r0 + r) * Q2_XLD + col], w);
                    double tw = tc * w;
                    X[r0 * Q2_XLD + col] -= tw;
                    for (int r = 1; r < L; r++) X[(r0 + r) * Q2_XLD + col] -= tw * rf[r];
                }
            }
            __syncthreads();
            cta_q2_block(X, Z + w0, ldz, rows, k);
        }
    }
}

// Z <- Q1 Z from the stage-1 panels (from the last): Z[r0:] -= V (T (V^T Z[r0:]))
__device__ void team_apply_q1(const Team& t, const double* A, long long lda, int n, int k, double* Z, long long ldz,
                              double* wk) {
    double* V = wk + band_off_v(n);
    double* Y1 = wk + band_off_y(n);  // BW x k
    double* Y2 = wk + band_off_x(n);  // BW x k
    int np = 0;
    while (n - (np * BW + BW) >= 2) np++;
    for (int p = np - 1; p >= 0; p--) {
        int j0 = p * BW, r0 = j0 + BW, m = n - r0;
        int nb = min(BW, n - j0), nr = min(nb, m - 1);
        const double* P = A + r0 + (long long)j0 * lda;
        const double* T = wk + band_off_t(n) + (long long)p * BW * BW;
        for (long long q = threadIdx.x; q < (long long)m * nr; q += blockDim.x) {
            int i = (int)(q % m), c = (int)(q / m);
            V[q] = i == c ? 1.0 : (i > c ? P[i + (long long)c * lda] : 0.0);
        }
        __syncthreads();
        team_gemm(t, true, false, nr, k, m, 1.0, V, m, Z + r0, ldz, 0.0, Y1, BW);
        team_gemm(t, false, false, nr, k, nr, 1.0, T, BW, Y1, BW, 0.0, Y2, BW, GEMM_A_UPPER);
        team_gemm(t, false, false, m, k, nr, -1.0, V, m, Y2, BW, 1.0, Z + r0, ldz);
    }
}

}  // namespace axg
