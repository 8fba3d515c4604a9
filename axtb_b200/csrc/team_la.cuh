// Dense FP64 linear algebra run by a "team": one CTA (small molecules, many per launch, each CTA
// taking its own molecules) or the whole cooperative grid (a large molecule, every CTA at once).
// The same device functions serve both; a team barrier is __syncthreads() for one CTA and a
// grid-wide barrier for the whole grid (cooperative launch, so every CTA is resident).
//
// Matrices are column-major with an explicit leading dimension. These routines compute the
// quantities of the reference's dense algebra (crates/base/src/linalg/eigen.rs: Cholesky of S,
// the reduced matrix L^-1 F L^-T, its eigenvalues and occupied eigenvectors, C = L^-T U; and
// crates/base/src/linalg/density.rs: P = C diag(f) C^T) with B200-friendly algorithms:
// blocked right-looking Cholesky, a row-block triangular inverse on GEMMs, Householder
// tridiagonalisation with lower-triangle symmetric matrix-vector products, Sturm-count bisection
// (one thread per eigenvalue, the levels up to the Fermi level), inverse iteration for the occupied vectors (one
// thread per vector, re-orthogonalised within clusters of close eigenvalues) and the blocked
// (compact WY) back-transformation on GEMMs.
#pragma once
#include <cooperative_groups.h>
#include <cuda_bf16.h>

#include "common.cuh"

namespace axg {
namespace cg = cooperative_groups;

constexpr int TEAM_THREADS = 256;

// SM-cycle counters of the eigen phase's parts (instrumentation, read by the profiler):
// 0..7 the phases of the eigen step, 8..13 the parts of the tridiagonal reduction
constexpr int TEAM_CYCLE_SLOTS = 24;
__device__ unsigned long long g_team_cycles[TEAM_CYCLE_SLOTS];

struct Team {
    int rank;     // CTA rank in the team
    int size;     // CTAs in the team
    bool global;  // the team is the whole grid
    __device__ __forceinline__ void sync() const {
        if (global) cg::this_grid().sync();
        else __syncthreads();
    }
    __device__ __forceinline__ int tid() const { return rank * blockDim.x + threadIdx.x; }
    __device__ __forceinline__ int nthreads() const { return size * blockDim.x; }
    __device__ __forceinline__ int warp() const { return (rank * blockDim.x + threadIdx.x) >> 5; }
    __device__ __forceinline__ int nwarps() const { return (size * blockDim.x) >> 5; }
};

// Layout of the grid team's reduction buffer `gred`: the panel dot partials (64 values x at most
// PD_PARTS CTAs), then two alternating slots of one double per CTA for team_sum.
constexpr int PD_PARTS = 64;
constexpr int RED_SUM0 = 64 * PD_PARTS;
__host__ __device__ constexpr long long team_red_doubles(int grid) { return RED_SUM0 + 2LL * grid + 64; }

// Parity of the grid-team sums this CTA has made (k_team clears it at entry; every CTA makes the
// same sequence of calls, so the parity agrees across the grid).
__shared__ int s_team_gen;

// sum of p[0..n) by one warp: lane-strided partial sums (eight loads in flight per lane), then a
// butterfly; the order is fixed, so every lane and every CTA gets the same bits. p is read
// through L2 (written by other CTAs before a grid barrier).
__device__ __forceinline__ double warp_gather_sum(const double* p, int n) {
    int lane = threadIdx.x & 31;
    double s = 0.0;
    for (int k0 = 0; k0 < n; k0 += 256) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            int k = k0 + u * 32 + lane;
            v[u] = k < n ? __ldcg(p + k) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; u++) s += v[u];
    }
    return warp_sum(s);
}

// Deterministic team sum: warp sums, CTA sum in fixed warp order, then (global team) the CTA
// partials gathered by one warp in a fixed order. A grid team writes its partials into one of
// two alternating slots: a CTA that runs ahead into the next sum writes the other slot while a
// slow one still reads this one, so one grid barrier per sum suffices.
__device__ double team_sum(const Team& t, double v, double* gred) {
    __shared__ double sred[TEAM_THREADS / 32];
    __shared__ double sout, sall;
    v = warp_sum(v);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sred[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) s += sred[k];
        sout = s;
    }
    __syncthreads();
    double blk = sout;
    if (!t.global) return blk;
    double* slot = gred + RED_SUM0 + (long long)(s_team_gen & 1) * t.size;
    if (threadIdx.x == 0) slot[t.rank] = blk;
    t.sync();
    if (threadIdx.x < 32) {
        double s = warp_gather_sum(slot, t.size);
        if (threadIdx.x == 0) {
            sall = s;
            s_team_gen++;
        }
    }
    __syncthreads();
    return sall;
}

// ---------------------------------------------------------------------------------- GEMM
// C(MxN) = alpha op(A) op(B) + beta C; op(A) = A (M x K, lda) or A^T (A is K x M);
// op(B) = B (K x N, ldb) or B^T (B is N x K). 64x64 CTA tiles on FP64 tensor cores
// (mma.sync m8n8k4.f64: each of the 8 warps owns a 32x16 block of 4x2 MMA tiles), k-steps of 16
// fed through a GSTAGES-deep ring of shared-memory stages by asynchronous copies (cp.async, 8
// bytes per element, zero-filled outside the operands), so the loads of GSTAGES - 1 k-steps are
// in flight while one computes. Flags restrict the work to the non-zero part of structured
// operands (exactly: the skipped products are zero) or of symmetric results:
//   GEMM_A_LOWER  op(A) lower triangular: k <= row      GEMM_A_UPPER  op(A) upper: k >= row
//   GEMM_B_UPPER  op(B) upper triangular: k <= col      GEMM_B_LOWER  op(B) lower: k >= col
//   GEMM_LOWER_TILES  only tiles with bi >= bj
//   GEMM_A_SYMM   A is symmetric (M x M) and only its lower triangle is read: op(A)[r][k] =
//                 A[max(r,k)][min(r,k)] (ta is ignored)
// GEMM_SPLIT computes the products in split precision instead of FP64: every operand value is
// rounded to FP32 and split into three BF16 parts (x ~ h + m + l, 24 significant bits, the
// width of FP32), and A B ~ the six products of significance down to 2^-16 (Al Bh + Am Bm +
// Ah Bl, then Am Bh + Ah Bm, then Ah Bh) on the BF16 tensor cores (mma.sync m16n8k16), summed in
// FP32 within each k-step of 16 and in FP64 across k-steps; the result is stored in FP64.
constexpr int GT = 64, GK = 16, GSTAGES = 4;
enum { GEMM_A_LOWER = 1, GEMM_A_UPPER = 2, GEMM_B_UPPER = 4, GEMM_LOWER_TILES = 8, GEMM_B_LOWER = 16, GEMM_SPLIT = 32,
       GEMM_A_SYMM = 64 };

// One dynamic shared-memory work area per CTA, used in turn (never at the same time, each user
// starting and ending at a CTA barrier): the GEMM's stages, the Cholesky's diagonal block, the
// bisection's tridiagonal matrix, the band reduction's per-warp tiles and the second stage's
// back-transformation blocks.
constexpr int CB = 64;
constexpr int GSTAGE = 2 * GK * (GT + 2);  // A and B tiles of one stage
constexpr int SMEM_WORK = GSTAGES * GSTAGE;
constexpr int SMEM_WORK_BYTES = SMEM_WORK * 8;
static_assert(CB * (CB + 1) <= SMEM_WORK, "diagonal block fits the work area");
extern __shared__ __align__(16) double s_work[];

__device__ __forceinline__ void dmma_8x8x4(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// 8-byte asynchronous copy global -> shared; ok = false zero-fills the destination without a read
__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool ok) {
    unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(ok ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// two FP64 values -> three BF16 parts each (x ~ h + m + l after rounding to FP32), packed in
// pairs as mma operands (the first value in the low half)
__device__ __forceinline__ void split_pair(double a, double b, unsigned& hi, unsigned& mid, unsigned& lo) {
    float fa = (float)a, fb = (float)b;
    __nv_bfloat162 h = __floats2bfloat162_rn(fa, fb);
    float2 hf = __bfloat1622float2(h);
    float ra = fa - hf.x, rb = fb - hf.y;
    __nv_bfloat162 m = __floats2bfloat162_rn(ra, rb);
    float2 mf = __bfloat1622float2(m);
    __nv_bfloat162 l = __floats2bfloat162_rn(ra - mf.x, rb - mf.y);
    hi = *reinterpret_cast<unsigned*>(&h);
    mid = *reinterpret_cast<unsigned*>(&m);
    lo = *reinterpret_cast<unsigned*>(&l);
}

__device__ __forceinline__ void mma_bf16_16816(float* c, const unsigned* a, const unsigned* b) {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

template <bool SPLIT>
__device__ __noinline__ void team_gemm_t(const Team& t, bool ta, bool tb, int M, int N, int K, double alpha,
                                         const double* A, long long lda, const double* B, long long ldb, double beta,
                                         double* Cm, long long ldc, int flags) {
    typedef double Stage[2][GK][GT + 2];  // [A, B][k][m or n]
    Stage* stg = reinterpret_cast<Stage*>(s_work);
    if (M <= 0 || N <= 0) return;
    const bool symm = (flags & GEMM_A_SYMM) != 0;
    const int tm = (M + GT - 1) / GT, tn = (N + GT - 1) / GT, ntile = tm * tn;
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int wm = warp & 1, wn = warp >> 1;  // warp block: rows wm*32.., cols wn*16..
    int lr = lane >> 2, lc = lane & 3;
    // this CTA's tiles in order (tile = rank + i * size, upper tiles skipped for GEMM_LOWER_TILES)
    // and each tile's k range; the k-steps of all of them form one stream, so the copies of the
    // next tile's first k-steps are in flight while the current tile finishes and stores
    auto next_tile = [&](int tile) {
        for (tile += t.size; tile < ntile; tile += t.size)
            if (!((flags & GEMM_LOWER_TILES) && tile / tm > tile % tm)) break;
        return tile;
    };
    auto krange = [&](int tile, int& kb, int& nk) {
        int row0 = (tile % tm) * GT, col0 = (tile / tm) * GT;
        int k0 = 0, ke = K;
        if (flags & GEMM_A_LOWER) ke = min(ke, row0 + GT);
        if (flags & GEMM_B_UPPER) ke = min(ke, col0 + GT);
        if (flags & GEMM_A_UPPER) k0 = max(k0, (row0 / GK) * GK);
        if (flags & GEMM_B_LOWER) k0 = max(k0, (col0 / GK) * GK);
        kb = k0;
        nk = ke > k0 ? (ke - k0 + GK - 1) / GK : 1;  // an empty range: one k-step of zeros
        return ke;
    };
    int first = t.rank;
    if (first < ntile && (flags & GEMM_LOWER_TILES) && first / tm > first % tm) first = next_tile(first);
    // the copies of one k-step of `tile` into `slot`: each thread 4 elements of each operand,
    // consecutive threads along the operand's contiguous dimension; zero outside [kb, ke)
    auto issue = [&](int tile, int k0, int ke, int slot) {
        int row0 = (tile % tm) * GT, col0 = (tile / tm) * GT;
        Stage& S = stg[slot];
        // op(A) tile rows row0.., k k0..; the symmetric operand is read as stored below the
        // diagonal and transposed above it (both coalesced), element by element on the diagonal
        bool at = symm ? (k0 >= row0 + GT) : ta;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            int e = threadIdx.x + q * 256;
            int mm = at ? e / GK : e % GT, kk = at ? e % GK : e / GT;
            int gr = row0 + mm, gk = k0 + kk;
            bool ok = gr < M && gk < ke;
            long long off;
            if (symm) off = gr >= gk ? gr + (long long)gk * lda : gk + (long long)gr * lda;
            else off = ta ? gk + (long long)gr * lda : gr + (long long)gk * lda;
            cp_async8(&S[0][kk][mm], ok ? A + off : A, ok);
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            int e = threadIdx.x + q * 256;
            int nn = tb ? e % GT : e / GK, kk = tb ? e / GT : e % GK;
            int gc = col0 + nn, gk = k0 + kk;
            bool ok = gc < N && gk < ke;
            long long off = tb ? gc + (long long)gk * ldb : gk + (long long)gc * ldb;
            cp_async8(&S[1][kk][nn], ok ? B + off : B, ok);
        }
    };
    // issue cursor (runs GSTAGES - 1 k-steps ahead) and compute cursor
    int it_tile = first, it_kb = 0, it_nk = 0, it_ke = 0, it_ks = 0;
    if (it_tile < ntile) it_ke = krange(it_tile, it_kb, it_nk);
    auto issue_next = [&](int slot) {
        if (it_tile >= ntile) return;
        issue(it_tile, it_kb + it_ks * GK, it_ke, slot);
        if (++it_ks == it_nk) {
            it_tile = next_tile(it_tile);
            it_ks = 0;
            if (it_tile < ntile) it_ke = krange(it_tile, it_kb, it_nk);
        }
    };
    double acc[4][2][2];   // FP64: 4 x 2 tiles of 8 x 8 per warp
    double accf[2][2][4];  // split: 2 x 2 tiles of 16 x 8 per warp (FP64 sum of FP32 k-step partials)
    __syncthreads();  // the stages are free (the previous user is done with them)
#pragma unroll
    for (int st = 0; st < GSTAGES - 1; st++) {
        issue_next(st);
        cp_async_commit();
    }
    int f = 0;  // k-steps computed so far (the stage ring position)
    for (int tile = first; tile < ntile; tile = next_tile(tile)) {
        int kb_, nk;
        krange(tile, kb_, nk);
        int row0 = (tile % tm) * GT, col0 = (tile / tm) * GT;
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 2; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
#pragma unroll
        for (int i = 0; i < 2; i++)
#pragma unroll
            for (int j = 0; j < 2; j++)
#pragma unroll
                for (int h = 0; h < 4; h++) accf[i][j][h] = 0.0;
        for (int ks = 0; ks < nk; ks++, f++) {
            cp_async_wait<GSTAGES - 2>();  // this thread's copies of k-step f have landed
            __syncthreads();               // everyone's have; and the stage of k-step f - 1 is free
            issue_next((f + GSTAGES - 1) % GSTAGES);
            cp_async_commit();
            Stage& S = stg[f % GSTAGES];
            if constexpr (SPLIT) {
                // one k16 step: A rows g, g + 8 of each 16-row tile; k = 2 lc (+1), 2 lc + 8 (+1)
                unsigned ah[2][4], am[2][4], al[2][4], bh[2][2], bm[2][2], bl[2][2];
                const int k0s = 2 * lc;
#pragma unroll
                for (int i = 0; i < 2; i++) {
                    int r = wm * 32 + i * 16 + lr;
                    split_pair(S[0][k0s][r], S[0][k0s + 1][r], ah[i][0], am[i][0], al[i][0]);
                    split_pair(S[0][k0s][r + 8], S[0][k0s + 1][r + 8], ah[i][1], am[i][1], al[i][1]);
                    split_pair(S[0][k0s + 8][r], S[0][k0s + 9][r], ah[i][2], am[i][2], al[i][2]);
                    split_pair(S[0][k0s + 8][r + 8], S[0][k0s + 9][r + 8], ah[i][3], am[i][3], al[i][3]);
                }
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    int c = wn * 16 + j * 8 + lr;
                    split_pair(S[1][k0s][c], S[1][k0s + 1][c], bh[j][0], bm[j][0], bl[j][0]);
                    split_pair(S[1][k0s + 8][c], S[1][k0s + 9][c], bh[j][1], bm[j][1], bl[j][1]);
                }
                // per k-step partial sum in FP32, smallest terms first, added to the accumulator
#pragma unroll
                for (int i = 0; i < 2; i++)
#pragma unroll
                    for (int j = 0; j < 2; j++) {
                        float p[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                        mma_bf16_16816(p, al[i], bh[j]);
                        mma_bf16_16816(p, am[i], bm[j]);
                        mma_bf16_16816(p, ah[i], bl[j]);
                        mma_bf16_16816(p, am[i], bh[j]);
                        mma_bf16_16816(p, ah[i], bm[j]);
                        mma_bf16_16816(p, ah[i], bh[j]);
#pragma unroll
                        for (int h = 0; h < 4; h++) accf[i][j][h] += (double)p[h];
                    }
            } else {
#pragma unroll
                for (int kk = 0; kk < GK; kk += 4) {
                    double af[4], bf[2];
#pragma unroll
                    for (int i = 0; i < 4; i++) af[i] = S[0][kk + lc][wm * 32 + i * 8 + lr];
#pragma unroll
                    for (int j = 0; j < 2; j++) bf[j] = S[1][kk + lc][wn * 16 + j * 8 + lr];
#pragma unroll
                    for (int i = 0; i < 4; i++)
#pragma unroll
                        for (int j = 0; j < 2; j++) dmma_8x8x4(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
                }
            }
        }
        if constexpr (SPLIT) {
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 2; j++)
#pragma unroll
                    for (int h = 0; h < 4; h++) {
                        int gr = row0 + wm * 32 + i * 16 + lr + (h >> 1) * 8;
                        int gc = col0 + wn * 16 + j * 8 + lc * 2 + (h & 1);
                        if (gr >= M || gc >= N) continue;
                        double* dst = &Cm[gr + (long long)gc * ldc];
                        double v = alpha * accf[i][j][h];
                        *dst = beta == 0.0 ? v : v + beta * *dst;
                    }
        } else {
#pragma unroll
            for (int i = 0; i < 4; i++) {
                int gr = row0 + wm * 32 + i * 8 + lr;
                if (gr >= M) continue;
#pragma unroll
                for (int j = 0; j < 2; j++)
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        int gc = col0 + wn * 16 + j * 8 + lc * 2 + h;
                        if (gc >= N) continue;
                        double* dst = &Cm[gr + (long long)gc * ldc];
                        double v = alpha * acc[i][j][h];
                        *dst = beta == 0.0 ? v : v + beta * *dst;
                    }
            }
        }
    }
    cp_async_wait<0>();
    __syncthreads();  // the stages are free for the next user
}

__device__ __forceinline__ void team_gemm(const Team& t, bool ta, bool tb, int M, int N, int K, double alpha,
                                          const double* A, long long lda, const double* B, long long ldb, double beta,
                                          double* Cm, long long ldc, int flags = 0) {
    if (flags & GEMM_SPLIT) team_gemm_t<true>(t, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, Cm, ldc, flags);
    else team_gemm_t<false>(t, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, Cm, ldc, flags);
}

// A[c][i] = A[i][c] for i > c in the square block [r0, n)
__device__ void team_mirror_lower(const Team& t, double* A, long long lda, int r0, int n) {
    int m = n - r0;
    for (long long q = t.tid(); q < (long long)m * m; q += t.nthreads()) {
        int i = r0 + (int)(q % m), c = r0 + (int)(q / m);
        if (i < c) A[i + (long long)c * lda] = A[c + (long long)i * lda];
    }
}

// ---------------------------------------------------------------------------------- Cholesky
// Blocked right-looking Cholesky and triangular inverse in panels of CB columns. The CB x CB
// diagonal block is factored (and inverted) in shared memory by the team's first CTA; the panel
// and the trailing matrix are DMMA GEMMs: a team barrier every few GEMMs instead of two per column.
#define s_tri (*reinterpret_cast<double(*)[CB][CB + 1]>(s_work))

// the lower triangle of the nb x nb block at Bp (leading dimension ld) into s_tri (rest zero)
__device__ void cta_load_lower(const double* Bp, long long ld, int nb) {
    __syncthreads();
    for (int e = threadIdx.x; e < CB * CB; e += blockDim.x) {
        int r = e % CB, c = e / CB;
        s_tri[r][c] = (r < nb && c < nb && r >= c) ? Bp[r + (long long)c * ld] : 0.0;
    }
    __syncthreads();
}

// in-place lower Cholesky of the block in s_tri (unblocked, right-looking); false (on every
// thread) when a pivot is not positive
__device__ bool cta_potrf(int nb) {
    bool ok = true;
    for (int j = 0; j < nb; j++) {
        double p = s_tri[j][j];
        if (!(p > 0.0)) {
            ok = false;
            p = 1.0;
        }
        double ljj = sqrt(p), inv = 1.0 / ljj;
        __syncthreads();  // the pivot has been read
        for (int r = j + 1 + threadIdx.x; r < nb; r += blockDim.x) s_tri[r][j] *= inv;
        if (threadIdx.x == 0) s_tri[j][j] = ljj;
        __syncthreads();
        int m = nb - j - 1;
        for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
            int r = j + 1 + e % m, c = j + 1 + e / m;
            if (r >= c) s_tri[r][c] -= s_tri[r][j] * s_tri[c][j];
        }
        __syncthreads();
    }
    return ok;
}

// in-place inverse of the lower triangular block in s_tri (LAPACK dtrti2 order: columns from the
// last, x <- -T x / l_jj with T the already inverted trailing block)
__device__ void cta_trtri(int nb) {
    for (int j = nb - 1; j >= 0; j--) {
        double d = 1.0 / s_tri[j][j];
        int r = j + 1 + threadIdx.x;
        double y = 0.0;
        if (r < nb)
            for (int q = j + 1; q <= r; q++) y += s_tri[r][q] * s_tri[q][j];
        __syncthreads();
        if (r < nb) s_tri[r][j] = -d * y;
        if (threadIdx.x == 0) s_tri[j][j] = d;
        __syncthreads();
    }
}

// In-place lower Cholesky of the n x n SPD matrix A (the strict upper triangle is zeroed).
// Returns false (on every thread) when a pivot is not positive. scr holds CB x CB + 1 doubles.
__device__ __noinline__ bool team_cholesky(const Team& t, double* A, int n, long long lda, double* scr) {
    bool ok = true;  // kept by the first CTA, published in scr[CB * CB] at the end
    for (int k0 = 0; k0 < n; k0 += CB) {
        int nb = min(CB, n - k0), m2 = n - k0 - nb;
        double* A11 = A + k0 + (long long)k0 * lda;
        if (t.rank == 0) {
            cta_load_lower(A11, lda, nb);
            ok = cta_potrf(nb) && ok;
            for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
                int r = e % nb, c = e / nb;
                if (r >= c) A11[r + (long long)c * lda] = s_tri[r][c];
            }
            if (m2 > 0) {
                cta_trtri(nb);
                for (int e = threadIdx.x; e < CB * CB; e += blockDim.x) {
                    int r = e % CB, c = e / CB;
                    scr[e] = (r >= c) ? s_tri[r][c] : 0.0;
                }
            }
        }
        t.sync();
        if (m2 > 0) {
            double* A21 = A11 + nb;
            double* A22 = A21 + (long long)nb * lda;
            // L21 = A21 L11^-T, in place: an output tile (64 rows x nb <= 64 columns) reads only
            // its own rows of A21, all of them before its first store
            team_gemm(t, false, true, m2, nb, nb, 1.0, A21, lda, scr, CB, 0.0, A21, lda, GEMM_B_UPPER);
            t.sync();
            team_gemm(t, false, true, m2, m2, nb, -1.0, A21, lda, A21, lda, 1.0, A22, lda, GEMM_LOWER_TILES);
            t.sync();
        }
    }
    for (long long e = t.tid(); e < (long long)n * n; e += t.nthreads()) {
        int i = (int)(e % n), c = (int)(e / n);
        if (i < c) A[i + (long long)c * lda] = 0.0;
    }
    if (t.tid() == 0) scr[CB * CB] = ok ? 1.0 : 0.0;
    t.sync();
    return scr[CB * CB] != 0.0;
}

// Linv = L^-1 for lower triangular L (n x n), row blocks of CB: the diagonal block is inverted in
// shared memory, then Linv[I, 0:i0] = L_II^-1 (-L[I, 0:i0] Linv[0:i0, 0:i0]) on two GEMMs;
// `tmp` holds CB x n.
__device__ __noinline__ void team_trinv(const Team& t, const double* L, long long ldl, double* Linv, long long ldi, int n, double* tmp) {
    for (long long e = t.tid(); e < (long long)n * n; e += t.nthreads()) Linv[(e % n) + (e / n) * ldi] = 0.0;
    t.sync();
    for (int i0 = 0; i0 < n; i0 += CB) {
        int nb = min(CB, n - i0);
        double* Xii = Linv + i0 + (long long)i0 * ldi;
        if (t.rank == 0) {
            cta_load_lower(L + i0 + (long long)i0 * ldl, ldl, nb);
            cta_trtri(nb);
            for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
                int r = e % nb, c = e / nb;
                if (r >= c) Xii[r + (long long)c * ldi] = s_tri[r][c];
            }
        }
        if (i0 > 0) {
            team_gemm(t, false, false, nb, i0, i0, -1.0, L + i0, ldl, Linv, ldi, 0.0, tmp, CB, GEMM_B_LOWER);
            t.sync();  // tmp and Xii complete
            team_gemm(t, false, false, nb, i0, nb, 1.0, Xii, ldi, tmp, CB, 0.0, Linv + i0, ldi, GEMM_A_LOWER);
        }
        t.sync();
    }
}

// ---------------------------------------------------------------------------------- tridiagonal
// Householder reduction of the symmetric A (n x n) to T = Q^T A Q in panels of NBP columns (the
// LAPACK dsytrd/dlatrd scheme): d, e get the diagonal and subdiagonal, tau the reflector factors;
// reflector j (I - tau_j v v^T, v_{j+1} = 1) is kept in A[j+2:n, j]. Within a panel, column j is
// first brought up to date with the panel's earlier reflectors, its Householder vector is formed,
// and w = tau (A v - W (V^T v) - V (W^T v)) uses the trailing matrix as it was at the start of the
// panel (one read-only pass, no writes); after the panel the trailing matrix takes the rank-2*NBP
// update A -= V W^T + W V^T on GEMMs. V and W are n x NBP (leading dimension n).
constexpr int NBP = 32;

// ys[q] = V[r0:n, q] . v (q < c) and ys[c + q] = W[r0:n, q] . v, into shared memory
__device__ __noinline__ void team_panel_dots(const Team& t, const double* V, const double* W, long long ldv, const double* v, int r0,
                                int n, int c, double* ys, double* gpart) {
    static_assert(2 * NBP <= 64 && TEAM_THREADS == 256, "panel dots: at most 64 values, eight per warp");
    // no barrier first: warps that finish their symv items start here (ys was last read before
    // the previous column's team sums)
    int nq = 2 * c;
    // a grid team splits the rows over PD_PARTS CTAs only (few partials to gather afterwards)
    int parts = t.global ? min(t.size, PD_PARTS) : 1;
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (t.rank < parts) {
        int m = n - r0, per = (m + parts - 1) / parts;
        int rb0 = r0 + t.rank * per, rb1 = min(n, rb0 + per);
        // warp wid takes the vectors q = wid + 8u, all in one pass over its rows
        double s[8];
#pragma unroll
        for (int u = 0; u < 8; u++) s[u] = 0.0;
        for (int i = rb0 + lane; i < rb1; i += 32) {
            double vi = v[i];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                int q = wid + u * nw;
                if (q < nq) {
                    const double* X = q < c ? V + (long long)q * ldv : W + (long long)(q - c) * ldv;
                    s[u] = fma(X[i], vi, s[u]);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
            int q = wid + u * nw;
            double r = warp_sum(s[u]);
            if (lane == 0 && q < nq) {
                if (t.global) gpart[q * PD_PARTS + t.rank] = r;
                else ys[q] = r;
            }
        }
    }
    if (t.global) {
        t.sync();
        // warp wid gathers q = wid + 8u: lane holds parts lane and lane + 32; the butterfly gives
        // every CTA the same sum
        double g[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            int q = wid + u * nw;
            const double* gp = gpart + q * PD_PARTS;
            double a0 = (q < nq && lane < parts) ? __ldcg(gp + lane) : 0.0;
            double a1 = (q < nq && lane + 32 < parts) ? __ldcg(gp + lane + 32) : 0.0;
            g[u] = a0 + a1;
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
            int q = wid + u * nw;
            double r = warp_sum(g[u]);
            if (lane == 0 && q < nq) ys[q] = r;
        }
    }
    __syncthreads();
}

// Slots of the symv partial sums for an n x n matrix: 4 per 64-column block plus one.
__host__ __device__ constexpr int symv_slots(int n) { return 4 * ((n + 63) / 64) + 1; }

// y = A[r0:n, r0:n] v from the lower triangle only (A symmetric; the strict upper triangle is
// never read and may hold stale values). The trailing matrix is cut into 64 x 64 tiles (blocks
// counted from r0, bi >= bj) and each tile into four 16-column quarters; a warp takes a
// (tile, quarter) item, each lane two of its rows (lane, lane + 32), 32 loads in flight per lane.
// An item adds A_ic v_c to the rows of block bi and, strictly below the diagonal, A_ic v_i to its
// 16 columns (rows of block bj). Slots, per row block R (rt blocks in all): the row sums of items
// (R, bj, q) in slot 4 bj + q; the transposed sums of items (bi > R, R, q) in slot 3R + 3 + bi;
// the diagonal tile's transposed part in slot 3R + 3 + rt. Every (slot, row) is written exactly
// once, so the rows of block R sum their 3R + 4 + rt slots in a fixed order. ppart[slot * n + row];
// returns rt.
__device__ __noinline__ int team_symv_lower(const Team& t, const double* A, long long lda, int r0, int n,
                                            const double* v, double* ppart) {
    int m = n - r0;
    int rt = (m + 63) / 64;
    int nitem = 4 * (rt * (rt + 1) / 2);
    int lane = threadIdx.x & 31;
    for (int it = t.warp(); it < nitem; it += t.nwarps()) {
        int tl = it >> 2, qt = it & 3;
        // tl = bi (bi + 1) / 2 + bj
        int bi = (int)((sqrt(8.0 * tl + 1.0) - 1.0) * 0.5);
        while ((bi + 1) * (bi + 2) / 2 <= tl) bi++;
        while (bi * (bi + 1) / 2 > tl) bi--;
        int bj = tl - bi * (bi + 1) / 2;
        bool diag = bi == bj;
        int i0 = r0 + bi * 64, c0 = r0 + bj * 64, c1 = min(n, c0 + 64), cb = c0 + 16 * qt;
        int ia = i0 + lane, ib = ia + 32;
        bool oka = ia < n, okb = ib < n;
        int la = oka ? ia : n - 1, lb = okb ? ib : n - 1;
        double ra = 0.0, rb = 0.0;
        if (cb < c1) {  // uniform over the warp
            double va = oka ? v[ia] : 0.0, vb = okb ? v[ib] : 0.0;
            int tslot = 3 * bj + 3 + (diag ? rt : bi);
            double xa[16], xb[16];
#pragma unroll
            for (int u = 0; u < 16; u++) {
                const double* col = A + (long long)min(cb + u, n - 1) * lda;
                xa[u] = col[la];
                xb[u] = col[lb];
            }
            double p[16];
#pragma unroll
            for (int u = 0; u < 16; u++) {
                int c = cb + u;
                bool okc = c < c1;
                double vc = okc ? v[c] : 0.0;
                // lower triangle of the tile, rows and columns inside the matrix
                double a = (oka && okc && (!diag || ia >= c)) ? xa[u] : 0.0;
                double b = (okb && okc && (!diag || ib >= c)) ? xb[u] : 0.0;
                ra = fma(a, vc, ra);
                rb = fma(b, vc, rb);
                double ta = (diag && ia == c) ? 0.0 : a;  // transposed part: strictly below
                double tb = (diag && ib == c) ? 0.0 : b;
                p[u] = fma(tb, vb, ta * va);
            }
            // reduce-scatter of the 16 column partials over the warp: after the four halving
            // steps lane holds column u = 8 b4 + 4 b3 + 2 b2 + b1 (b_k = bit k of the lane)
            double q8[8], q4[4], q2[2];
            {
                bool h = (lane >> 4) & 1;
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    double r = __shfl_xor_sync(0xffffffffu, h ? p[k] : p[8 + k], 16);
                    q8[k] = (h ? p[8 + k] : p[k]) + r;
                }
            }
            {
                bool h = (lane >> 3) & 1;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    double r = __shfl_xor_sync(0xffffffffu, h ? q8[k] : q8[4 + k], 8);
                    q4[k] = (h ? q8[4 + k] : q8[k]) + r;
                }
            }
            {
                bool h = (lane >> 2) & 1;
#pragma unroll
                for (int k = 0; k < 2; k++) {
                    double r = __shfl_xor_sync(0xffffffffu, h ? q4[k] : q4[2 + k], 4);
                    q2[k] = (h ? q4[2 + k] : q4[k]) + r;
                }
            }
            double cs;
            {
                bool h = (lane >> 1) & 1;
                double r = __shfl_xor_sync(0xffffffffu, h ? q2[0] : q2[1], 2);
                cs = (h ? q2[1] : q2[0]) + r;
            }
            cs += __shfl_xor_sync(0xffffffffu, cs, 1);
            int cu = cb + ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 + ((lane >> 1) & 1);
            if ((lane & 1) == 0 && cu < c1) ppart[(long long)tslot * n + cu] = cs;
        }
        int rslot = 4 * bj + qt;  // written even for an empty quarter (zeros)
        if (oka) ppart[(long long)rslot * n + ia] = ra;
        if (okb) ppart[(long long)rslot * n + ib] = rb;
    }
    return rt;
}

// Grid team: the rows' symv sums, p_i = tau (sum of row i's slots - W_i. ys[0:c] - V_i. ys[c:2c]),
// into pbuf; returns this thread's part of p . v. A warp per row (rows spread over the whole
// grid), lanes over the row's slots, then lanes over the panel's c terms, with butterfly sums in
// a fixed order; a warp's rows (i, i + nwarps, i + 2 nwarps) are taken three at a time with all
// of their loads in flight together. (A one-CTA team sums each row in one thread, four slots at a
// time; for a large matrix that left the last row blocks, with hundreds of slots each, to a few
// CTAs while the rest of the grid waited.)
__device__ __noinline__ double grid_symv_combine(const Team& t, const double* ppart, int rt, int r0, int n,
                                                 const double* V, const double* W, long long ldv, const double* ys,
                                                 int c, double tj, const double* vbuf, double* pbuf) {
    constexpr int R = 3;
    int lane = threadIdx.x & 31;
    int nw = t.nwarps();
    double pv = 0.0;
    for (int i0 = r0 + t.warp(); i0 < n; i0 += R * nw) {
        int nsl[R];
        double s[R], wv[R];
        int nmax = 0;
#pragma unroll
        for (int r = 0; r < R; r++) {
            int i = i0 + r * nw;
            nsl[r] = i < n ? 3 * ((i - r0) >> 6) + 4 + rt : 0;
            nmax = max(nmax, nsl[r]);
            s[r] = 0.0;
            wv[r] = 0.0;
            if (i < n && lane < c) wv[r] = W[i + lane * ldv] * ys[lane] + V[i + lane * ldv] * ys[c + lane];
        }
        for (int k0 = 0; k0 < nmax; k0 += 256) {
            double x[R][8];
#pragma unroll
            for (int r = 0; r < R; r++) {
                const double* pp = ppart + (i0 + r * nw);
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    int k = k0 + u * 32 + lane;
                    x[r][u] = k < nsl[r] ? __ldcg(pp + (long long)k * n) : 0.0;
                }
            }
#pragma unroll
            for (int r = 0; r < R; r++)
#pragma unroll
                for (int u = 0; u < 8; u++) s[r] += x[r][u];
        }
#pragma unroll
        for (int r = 0; r < R; r++) {
            int i = i0 + r * nw;
            double sr = (warp_sum(s[r]) - warp_sum(wv[r])) * tj;
            if (lane == 0 && i < n) {
                pbuf[i] = sr;
                pv += sr * vbuf[i];
            }
        }
    }
    return pv;
}

// GRID_ROWS: the instance for whole-grid teams (t.global), with the row sums of
// grid_symv_combine; the one-CTA instance is compiled without that code, so the batch path's
// hot loop keeps its own register allocation.
template <bool GRID_ROWS>
__device__ __noinline__ void team_tridiag_blocked(const Team& t, double* A, long long lda, int n, double* d, double* e, double* tau,
                                     double* V, double* W, double* vbuf, double* pbuf, double* ppart, double* gred,
                                     bool cyc = false) {
    __shared__ double ys[64];
    const long long ldv = n;
    int nrefl = n - 2;
    long long t0 = clock64();
    auto tick = [&](int k) {
        if (cyc && t.tid() == 0) {
            long long now = clock64();
            atomicAdd(&g_team_cycles[k], (unsigned long long)(now - t0));
            t0 = now;
        }
    };
    for (int j0 = 0; j0 < nrefl; j0 += NBP) {
        int nb = min(NBP, nrefl - j0);
        for (int c = 0; c < nb; c++) {
            int j = j0 + c, r0 = j + 1;
            // (1) column j brought up to date with the panel's earlier reflectors, in the same pass
            // as the squared norm of A[r0+1:n, j] for (2) its Householder vector; the team sum's
            // barrier publishes the updated column
            double xs = 0.0;
            for (int i = j + t.tid(); i < n; i += t.nthreads()) {
                double a = A[i + (long long)j * lda];
                if (c > 0) {
                    double s = 0.0;
                    for (int q = 0; q < c; q++)
                        s += V[i + q * ldv] * W[j + q * ldv] + W[i + q * ldv] * V[j + q * ldv];
                    a -= s;
                    A[i + (long long)j * lda] = a;
                }
                if (i > r0) xs += sq(a);
            }
            tick(8);
            double xnorm2 = team_sum(t, xs, gred);
            double alpha = A[r0 + (long long)j * lda];
            double beta, tj, scale;
            if (xnorm2 == 0.0) {
                tj = 0.0;
                beta = alpha;
                scale = 0.0;
            } else {
                beta = -copysign(sqrt(alpha * alpha + xnorm2), alpha);
                tj = (beta - alpha) / beta;
                scale = 1.0 / (alpha - beta);
            }
            for (int i = r0 + t.tid(); i < n; i += t.nthreads()) {
                double v = i == r0 ? 1.0 : A[i + (long long)j * lda] * scale;
                vbuf[i] = v;
                V[i + c * ldv] = v;
                if (i > r0) A[i + (long long)j * lda] = v;
            }
            // A[r0, j] keeps alpha: the subdiagonal lives in e[j], and every thread of the team
            // reads alpha after the norm's barrier, so nothing may overwrite it before the next one
            if (t.tid() == 0) {
                e[j] = beta;
                tau[j] = tj;
                d[j] = A[j + (long long)j * lda];
            }
            t.sync();
            tick(9);
            // (3) w = tau (A v - W V^T v - V W^T v) - tau^2/2 (..) v
            if (tj != 0.0) {
                int rt = team_symv_lower(t, A, lda, r0, n, vbuf, ppart);
                tick(10);
                team_panel_dots(t, V, W, ldv, vbuf, r0, n, c, ys, gred);  // its barrier also publishes ppart
                tick(11);
                double pv = 0.0;
                bool grid_rows = false;
                if constexpr (GRID_ROWS) grid_rows = t.global;
                if (grid_rows) {
                    pv = grid_symv_combine(t, ppart, rt, r0, n, V, W, ldv, ys, c, tj, vbuf, pbuf);
                } else {
                    for (int i = r0 + t.tid(); i < n; i += t.nthreads()) {
                        int nsl = 3 * ((i - r0) >> 6) + 4 + rt;  // this row's symv slots
                        // four independent partial sums (four loads in flight), combined in a fixed order
                        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
                        const double* pp = ppart + i;
                        int ch = 0;
                        for (; ch + 3 < nsl; ch += 4) {
                            s0 += pp[(long long)ch * n];
                            s1 += pp[(long long)(ch + 1) * n];
                            s2 += pp[(long long)(ch + 2) * n];
                            s3 += pp[(long long)(ch + 3) * n];
                        }
                        for (; ch < nsl; ch++) s0 += pp[(long long)ch * n];
                        double s = (s0 + s1) + (s2 + s3);
                        for (int q = 0; q < c; q++) s -= W[i + q * ldv] * ys[q] + V[i + q * ldv] * ys[c + q];
                        s *= tj;
                        pbuf[i] = s;
                        pv += s * vbuf[i];
                    }
                }
                double dot = team_sum(t, pv, gred);
                double K = -0.5 * tj * dot;
                for (int i = r0 + t.tid(); i < n; i += t.nthreads())
                    W[i + c * ldv] = (grid_rows ? __ldcg(pbuf + i) : pbuf[i]) + K * vbuf[i];
            } else {
                for (int i = r0 + t.tid(); i < n; i += t.nthreads()) W[i + c * ldv] = 0.0;
            }
            t.sync();
            tick(12);
        }
        // (4) trailing update of rows and columns q0..n-1
        int q0 = j0 + nb, mm = n - q0;
        if (mm > 0) {
            double* Aq = A + q0 + (long long)q0 * lda;
            team_gemm(t, false, true, mm, mm, nb, -1.0, V + q0, ldv, W + q0, ldv, 1.0, Aq, lda, GEMM_LOWER_TILES);
            t.sync();
            team_gemm(t, false, true, mm, mm, nb, -1.0, W + q0, ldv, V + q0, ldv, 1.0, Aq, lda, GEMM_LOWER_TILES);
            t.sync();
            tick(13);
        }
    }
    if (t.tid() == 0) {
        if (n >= 2) {
            d[n - 2] = A[(n - 2) + (long long)(n - 2) * lda];
            e[n - 2] = A[(n - 1) + (long long)(n - 2) * lda];
            tau[n - 2] = 0.0;
        }
        d[n - 1] = A[(n - 1) + (long long)(n - 1) * lda];
        e[n - 1] = 0.0;
        tau[n - 1] = 0.0;
    }
    t.sync();
}

// number of eigenvalues of the symmetric tridiagonal (d, e) below x (Sturm sequence)
__device__ __forceinline__ int sturm_count(const double* d, const double* e, int n, double x, double pivmin) {
    int cnt = 0;
    double q = d[0] - x;
    if (fabs(q) < pivmin) q = -pivmin;
    if (q < 0.0) cnt++;
    for (int i = 1; i < n; i++) {
        q = d[i] - x - e[i - 1] * e[i - 1] / q;
        if (fabs(q) < pivmin) q = -pivmin;
        if (q < 0.0) cnt++;
    }
    return cnt;
}

// Gershgorin bounds of the symmetric tridiagonal (d, e) and the pivot floor into gbuf[0..2]
// (thread 0 of the team; the team barrier publishes them)
__device__ void team_gershgorin(const Team& t, const double* d, const double* e, int n, double* gbuf) {
    if (t.tid() == 0) {
        double lo = INFINITY, hi = -INFINITY, emax = 0.0;
        for (int i = 0; i < n; i++) {
            double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i + 1 < n ? fabs(e[i]) : 0.0);
            lo = fmin(lo, d[i] - r);
            hi = fmax(hi, d[i] + r);
            if (i + 1 < n) emax = fmax(emax, e[i] * e[i]);
        }
        double tnrm = fmax(fabs(lo), fabs(hi));
        lo -= 2.0 * DBL_EPSILON * tnrm * n + 1e-300;
        hi += 2.0 * DBL_EPSILON * tnrm * n + 1e-300;
        gbuf[0] = lo;
        gbuf[1] = hi;
        gbuf[2] = DBL_MIN * fmax(1.0, emax);
    }
    t.sync();
}

// Sturm counts of R shifts at once (independent recurrences interleaved, so the divisions of one
// hide the latency of the others), d and e^2 in shared memory
template <int R>
__device__ __forceinline__ void sturm_counts_sh(const double* sd, const double* se2, int n, const double* x,
                                                double pivmin, int* cnt) {
    double q[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
        q[r] = sd[0] - x[r];
        if (fabs(q[r]) < pivmin) q[r] = -pivmin;
        cnt[r] = q[r] < 0.0 ? 1 : 0;
    }
    for (int i = 1; i < n; i++) {
        double di = sd[i], ei = se2[i - 1];
#pragma unroll
        for (int r = 0; r < R; r++) {
            q[r] = di - x[r] - ei / q[r];
            if (fabs(q[r]) < pivmin) q[r] = -pivmin;
            cnt[r] += q[r] < 0.0 ? 1 : 0;
        }
    }
}

__device__ __forceinline__ bool bisect_done(double lo, double hi, double pivmin) {
    return hi - lo <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + pivmin;
}

// R eigenvalues per thread (k = k0 + threadIdx.x + r blockDim.x), bisection interleaved
template <int R>
__device__ void cta_bisect_ilp(const double* sd, const double* se2, int n, double* w, double glo, double ghi,
                               double pivmin, int k0, int k1) {
    double lo[R], hi[R], x[R];
    int cnt[R];
    bool live[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
        lo[r] = glo;
        hi[r] = ghi;
        live[r] = k0 + (int)threadIdx.x + r * (int)blockDim.x < k1;
    }
    for (int it = 0; it < 200; it++) {
        bool any = false;
#pragma unroll
        for (int r = 0; r < R; r++) {
            double mid = 0.5 * (lo[r] + hi[r]);
            if (live[r] && (bisect_done(lo[r], hi[r], pivmin) || mid <= lo[r] || mid >= hi[r])) live[r] = false;
            x[r] = live[r] ? mid : lo[r];
            any = any || live[r];
        }
        if (!any) break;
        sturm_counts_sh<R>(sd, se2, n, x, pivmin, cnt);
#pragma unroll
        for (int r = 0; r < R; r++) {
            int k = k0 + (int)threadIdx.x + r * (int)blockDim.x;
            if (!live[r]) continue;
            if (cnt[r] > k) hi[r] = x[r];
            else lo[r] = x[r];
        }
    }
#pragma unroll
    for (int r = 0; r < R; r++) {
        int k = k0 + (int)threadIdx.x + r * (int)blockDim.x;
        if (k < k1) w[k] = 0.5 * (lo[r] + hi[r]);
    }
}

// eigenvalues k0..k1-1 of one CTA's tridiagonal (d, e), d and e^2 staged in shared memory
__device__ void cta_bisect(const double* d, const double* e, int n, double* w, const double* gbuf, int k0, int k1) {
    double glo = gbuf[0], ghi = gbuf[1], pivmin = gbuf[2];
    double* sd = s_work;
    double* se2 = s_work + n;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        sd[i] = d[i];
        se2[i] = i + 1 < n ? e[i] * e[i] : 0.0;
    }
    __syncthreads();
    int cnt = k1 - k0, nt = blockDim.x;
    if (cnt > 0) {
        // plain bisection per level (multisection takes fewer steps for few levels, but ends on
        // other bits, and a few chaotic SCFs follow those bits)
        if (cnt <= nt) {
            cta_bisect_ilp<1>(sd, se2, n, w, glo, ghi, pivmin, k0, k1);
        } else if (cnt <= 2 * nt) {
            cta_bisect_ilp<2>(sd, se2, n, w, glo, ghi, pivmin, k0, k1);
        } else if (cnt <= 3 * nt) {
            cta_bisect_ilp<3>(sd, se2, n, w, glo, ghi, pivmin, k0, k1);
        } else {
            cta_bisect_ilp<4>(sd, se2, n, w, glo, ghi, pivmin, k0, k1);
        }
    }
    __syncthreads();
}

// eigenvalues k0..k1-1 (ascending order) by bisection, one thread per eigenvalue index; gbuf holds
// team_gershgorin's bounds. One CTA whose matrix fits the shared work area: cta_bisect.
__device__ __noinline__ void team_bisect(const Team& t, const double* d, const double* e, int n, double* w,
                                         const double* gbuf, int k0, int k1) {
    if (!t.global && 2 * n <= SMEM_WORK && k1 - k0 <= 4 * (int)blockDim.x) {
        cta_bisect(d, e, n, w, gbuf, k0, k1);
        return;
    }
    double glo = gbuf[0], ghi = gbuf[1], pivmin = gbuf[2];
    for (int k = k0 + t.tid(); k < k1; k += t.nthreads()) {
        double lo = glo, hi = ghi;
        for (int it = 0; it < 200; it++) {
            double mid = 0.5 * (lo + hi);
            if (hi - lo <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + pivmin || mid <= lo || mid >= hi) break;
            if (sturm_count(d, e, n, mid, pivmin) > k) hi = mid;
            else lo = mid;
        }
        w[k] = 0.5 * (lo + hi);
    }
    t.sync();
}

// ---------------------------------------------------------------------------------- Fermi
// tblite Fermi filling of nel electrons at kT over the ascending levels emo (one warp):
// crates/base/src/occupations.rs:58-128; returns false when kt == 0 (aufbau only).
__device__ void warp_fill(double nel, double kt, const double* emo, int n, double* occ, double* ef_out) {
    int lane = threadIdx.x & 31;
    int full = (int)floor(nel);
    double rem = fmod(nel, 1.0);
    for (int i = lane; i < n; i += 32) occ[i] = i < full ? 1.0 : (i == full ? rem : 0.0);
    int homo = full + (rem > 0.5 ? 1 : 0);
    __syncwarp();
    if (!(nel > 0.0 && kt > 0.0)) {
        *ef_out = 0.0;
        return;
    }
    int i0 = max(homo, 1) - 1, i1 = min(homo + 1, n) - 1;
    double ef = 0.5 * (emo[i0] + emo[i1]), ef_used = ef;
    const double tol = 1e5 * DBL_EPSILON, sqrttiny = sqrt(DBL_MIN);
    for (int it = 0; it < 200; it++) {
        double tot = 0.0, dtot = 0.0;
        ef_used = ef;
        for (int i = lane; i < n; i += 32) {
            double arg = (emo[i] - ef) / kt, f, df;
            if (arg > 50.0) {
                f = 0.0;
                df = 0.0;
            } else if (arg < -50.0) {
                f = 1.0;
                df = 0.0;
            } else {
                f = 1.0 / (exp(arg) + 1.0);
                df = -f * (1.0 - f) / kt;
            }
            occ[i] = f;
            tot += f;
            dtot -= df;
        }
        tot = warp_sum(tot);
        dtot = warp_sum(dtot);
        if (fabs(nel - tot) <= tol) break;
        if (dtot > sqrttiny) ef += (nel - tot) / dtot;
        else break;
    }
    __syncwarp();
    *ef_out = ef_used;
}

// ---------------------------------------------------------------------------------- inverse iteration
__device__ __forceinline__ double hash_uniform(unsigned int a, unsigned int b) {
    unsigned int h = a * 0x9E3779B1u ^ (b + 0x7F4A7C15u) * 0x85EBCA77u;
    h ^= h >> 16;
    h *= 0x7FEB352Du;
    h ^= h >> 15;
    h *= 0x846CA68Bu;
    h ^= h >> 16;
    return ((double)h / 4294967296.0) * 2.0 - 1.0;
}

// Eigenvectors of the tridiagonal (d, e) for the eigenvalues w[0..k) by inverse iteration, one
// thread per cluster of eigenvalues closer than ctol (vectors of a cluster re-orthogonalised
// against its earlier members). Two solves per vector from a hashed start: with eigenvalues
// from bisection to working precision the first solve already amplifies the wanted direction by
// ~1/eps, the second one settles it (LAPACK's dstein stops at that growth and adds one solve).
// Vector q is written to column q of V (n x k, ldv). Work planes
// u0, u1, lm (n*n each, interleaved [i*n + q]), piv (n*n bytes), x (n*n interleaved). The solves
// carry the running values in registers, so the loads of a step (factors and right-hand side)
// do not wait for the previous step's stores.
// Returns (through flag) nonzero when a vector was not finite.
__device__ __noinline__ void team_invit(const Team& t, const double* d, const double* e, const double* w, int n, int k,
                                        double* V, long long ldv, double* __restrict__ u0, double* __restrict__ u1,
                                        double* __restrict__ lm, unsigned char* __restrict__ piv,
                                        double* __restrict__ x, int* flag) {
    double tnrm = 0.0;
    for (int i = 0; i < n; i++) {
        double r = fabs(d[i]) + (i > 0 ? fabs(e[i - 1]) : 0.0) + (i + 1 < n ? fabs(e[i]) : 0.0);
        tnrm = fmax(tnrm, r);
    }
    if (tnrm == 0.0) tnrm = 1.0;
    const double ctol = 1e-6 * tnrm, pert = 10.0 * DBL_EPSILON * tnrm, pivmin = DBL_EPSILON * tnrm;
    const long long LD = n;  // interleave stride
    for (int q0 = t.tid(); q0 < k; q0 += t.nthreads()) {
        if (q0 > 0 && w[q0] - w[q0 - 1] <= ctol) continue;  // not a cluster head
        int q1 = q0 + 1;
        while (q1 < k && w[q1] - w[q1 - 1] <= ctol) q1++;
        double lam_prev = -INFINITY;
        for (int q = q0; q < q1; q++) {
            double lam = w[q];
            if (q > q0 && lam < lam_prev + pert) lam = lam_prev + pert;
            lam_prev = lam;
            // LU with partial pivoting of T - lam I; active row (ca, cb)
            double ca = d[0] - lam, cb = n > 1 ? e[0] : 0.0;
            for (int i = 0; i + 1 < n; i++) {
                double sub = e[i], a1 = d[i + 1] - lam, b1 = (i + 2 < n) ? e[i + 1] : 0.0;
                long long ix = (long long)i * LD + q;
                if (fabs(ca) >= fabs(sub)) {
                    double pv = ca;
                    if (pv == 0.0) pv = pivmin;
                    double l = sub / pv;
                    u0[ix] = pv;
                    u1[ix] = cb;
                    lm[ix] = l;
                    piv[ix] = 0;
                    ca = a1 - l * cb;
                    cb = b1;
                } else {
                    double l = ca / sub;
                    u0[ix] = sub;
                    u1[ix] = a1;
                    lm[ix] = l;
                    piv[ix] = 1;
                    ca = cb - l * a1;
                    cb = -l * b1;
                }
            }
            {
                long long ix = (long long)(n - 1) * LD + q;
                u0[ix] = (ca == 0.0) ? pivmin : ca;
            }
            for (int i = 0; i < n; i++) x[(long long)i * LD + q] = hash_uniform((unsigned)q, (unsigned)i);
            for (int iter = 0; iter < 2; iter++) {
                // forward: L with the row interchanges; cur = row i after the earlier steps
                double cur = x[q];
                for (int i = 0; i + 1 < n; i++) {
                    long long ix = (long long)i * LD + q, ix1 = ix + LD;
                    double nxt = x[ix1];
                    double xi = cur, xi1 = nxt;
                    if (piv[ix]) {
                        xi = nxt;
                        xi1 = cur;
                    }
                    x[ix] = xi;
                    cur = xi1 - lm[ix] * xi;
                }
                x[(long long)(n - 1) * LD + q] = cur;
                // backward: U with up to two superdiagonals (u2_i = e_{i+1} after an interchange)
                double xn1 = 0.0, xn2 = 0.0, mx = 0.0;
                for (int i = n - 1; i >= 0; i--) {
                    long long ix = (long long)i * LD + q;
                    double v = x[ix];
                    if (i + 1 < n) v -= u1[ix] * xn1;
                    if (i + 2 < n && piv[ix]) v -= e[i + 1] * xn2;
                    v /= u0[ix];
                    x[ix] = v;
                    xn2 = xn1;
                    xn1 = v;
                    mx = fmax(mx, fabs(v));
                }
                // scale by the largest element, orthogonalise within the cluster, normalise
                if (!(mx > 0.0) || !isfinite(mx)) {
                    atomicOr(flag, ST_INVIT);
                    mx = 1.0;
                }
                double inv = 1.0 / mx;
                for (int i = 0; i < n; i++) x[(long long)i * LD + q] *= inv;
                for (int pp = q0; pp < q; pp++) {
                    double dt = 0.0;
                    for (int i = 0; i < n; i++) dt += x[(long long)i * LD + pp] * x[(long long)i * LD + q];
                    for (int i = 0; i < n; i++) x[(long long)i * LD + q] -= dt * x[(long long)i * LD + pp];
                }
                double nr = 0.0;
                for (int i = 0; i < n; i++) nr += sq(x[(long long)i * LD + q]);
                nr = 1.0 / sqrt(nr);
                for (int i = 0; i < n; i++) x[(long long)i * LD + q] *= nr;  // later cluster members use it
            }
            for (int i = 0; i < n; i++) V[i + (long long)q * ldv] = x[(long long)i * LD + q];
        }
    }
    t.sync();
}

// Z <- Q Z for Q = H_0 H_1 ... H_{n-3} kept in A (team_tridiag_blocked), Z = V (n x k, ldv), blocked by
// 64 reflectors (compact WY: H_b..H_{b+nb-1} = I - Vb T Vb^T, T upper triangular).
// Work: vb (n x 64), tb (64 x 64), gm (64 x 64), y (64 x k), y2 (64 x k).
__device__ __noinline__ void team_backtransform(const Team& t, const double* A, long long lda, const double* tau, int n, int k,
                                   double* V, long long ldv, double* vb, double* tb, double* gm, double* y, double* y2) {
    int nrefl = n - 2;
    if (nrefl <= 0 || k <= 0) return;
    const int NB = GT;
    for (int b0 = ((nrefl - 1) / NB) * NB; b0 >= 0; b0 -= NB) {
        int jb = min(NB, nrefl - b0);
        int r0 = b0 + 1, nr = n - r0;
        // explicit Vb (nr x jb, ld nr): unit at row c, A below, zero above
        for (long long q = t.tid(); q < (long long)nr * jb; q += t.nthreads()) {
            int r = (int)(q % nr), c = (int)(q / nr);
            double v = r == c ? 1.0 : (r > c ? A[(r0 + r) + (long long)(b0 + c) * lda] : 0.0);
            vb[r + (long long)c * nr] = v;
        }
        t.sync();
        // G = Vb^T Vb (jb x jb)
        team_gemm(t, true, false, jb, jb, nr, 1.0, vb, nr, vb, nr, 0.0, gm, NB);
        t.sync();
        // T by the forward recurrence (one warp of CTA 0)
        if (t.rank == 0 && threadIdx.x < 32) {
            int lane = threadIdx.x;
            for (int q = lane; q < NB * NB; q += 32) tb[q] = 0.0;
            __syncwarp();
            for (int c = 0; c < jb; c++) {
                double tc = tau[b0 + c];
                // column c: T[0:c, c] = -tau_c T[0:c,0:c] G[0:c, c]
                for (int i = lane; i < c; i += 32) {
                    double s = 0.0;
                    for (int q = i; q < c; q++) s += tb[i + q * NB] * gm[q + c * NB];
                    tb[i + c * NB] = -tc * s;
                }
                __syncwarp();
                if (lane == 0) tb[c + c * NB] = tc;
                __syncwarp();
            }
        }
        t.sync();
        // y = Vb^T Z[r0:, :] (jb x k); y2 = T y; Z[r0:, :] -= Vb y2
        team_gemm(t, true, false, jb, k, nr, 1.0, vb, nr, V + r0, ldv, 0.0, y, NB);
        t.sync();
        team_gemm(t, false, false, jb, k, jb, 1.0, tb, NB, y, NB, 0.0, y2, NB);
        t.sync();
        team_gemm(t, false, false, nr, k, jb, -1.0, vb, nr, y2, NB, 1.0, V + r0, ldv);
        t.sync();
    }
}

}  // namespace axg
