// Building blocks of the rank-adaptive DLR kernel (parallel and BUG-rejection
// integrators, SolverCSD.jl :1726-2008 and :2011-2374).
//
// Widths: the rank entering a step is at most RA; augmented bases [X X~] hold
// up to KA = 2 RA columns. Tall factors are row-major in global memory (L2
// resident) with leading dimension KA (X, W) or RA (K, L and their projected /
// range-finder copies). Every reduction over rows goes through per-CTA partial
// buffers and a two-stage sum into the team's reduced buffer `red`, which all
// CTAs then read; small-matrix algebra is repeated bit-identically by every CTA
// in shared memory and in a per-CTA scratch area of global memory, so all CTAs
// take the same control decisions (ranks, rejections) without a broadcast.
#pragma once
#include "dlr_device.cuh"
#include "umma.cuh"
#include "wide_state.h"

// The rank-adaptive kernels are compiled twice: for the reference's 2D
// problems (four streaming pairs, namespace titus::wide) and for 3D problems
// (six pairs, the z pair appended; namespace titus::wide3, titus_adaptive3d.cu).
#ifndef TITUS_WIDE_NOPS
#define TITUS_WIDE_NOPS 4
#endif
#ifndef TITUS_WIDE_NS
#define TITUS_WIDE_NS wide
#endif

namespace titus {
namespace TITUS_WIDE_NS {

// streaming pairs (stencil L_d, P_N matrix A_d): (L2x, Ax), (L2y, Az), (L1x, |Ax|),
// (L1y, |Az|) and, for 3D problems, (L2z, Ay), (L1z, |Ay|)
constexpr int NOPS_W = TITUS_WIDE_NOPS;
constexpr bool kThreeD = NOPS_W == 6;
static_assert(NOPS_W == 4 || NOPS_W == 6, "four (2D) or six (3D) streaming pairs");

constexpr int NT = titus::NT;   // threads per CTA
constexpr int RA = titus::WIDE_RA;   // max rank entering a step
constexpr int KA = 2 * RA;      // max augmented width
constexpr int LDS = KA + 1;     // row stride of the truncation SVD's column arrays (odd: no bank conflicts)
constexpr int QW = titus::QM;   // psi leading dimension (reduced ordinates <= QW)
constexpr int TRW = 8;          // rows per staged tile (minimum layout)
constexpr int TRMAX = 512;      // rows per staged tile when the phase's free shared memory allows
constexpr int PMAXW = 2 * NOPS_W * KA * KA;   // largest reduction (BUG S-step Grams): 51200 doubles in 2D
constexpr int WORKD = 20480;    // shared work area (doubles)
constexpr int ACCW = 16384;     // accumulator chunk (doubles), inside the work area
constexpr int FLD = 10 * RA;    // feature-tile leading dimension (doubles)
constexpr int SCRW = kThreeD ? 90112 : 81920;   // per-CTA scratch (doubles, global)
constexpr int WCS = 3 * RA;     // row stride of the W-side completion coefficients

// extra device status codes (titus::ST_* holds 1..4)
constexpr int ST_LIMIT = 5;        // rank would exceed RA
constexpr int ST_UNSUPPORTED = 6;  // angular basis lost orthonormality (cannot complete)
constexpr int ST_SVD = 7;          // Jacobi SVD did not converge
constexpr int ST_REF_SHAPE = 8;    // the reference's next step raises DimensionMismatch (parallel-rejection loop)

using WideState = titus::WideState;

// Per-CTA scratch layout (offsets in doubles). r x r matrices use ld RA.
enum : int {
    SO_SC = 0,                            // stacked S C_d          (NOPS_W RA x RA)
    SO_SG = SO_SC + NOPS_W * RA * RA,     // stacked S^T G_d^T      (NOPS_W RA x RA)
    SO_SBAR = SO_SG + NOPS_W * RA * RA,   // S after the streaming / in-scattering S update (RA x RA)
    SO_SIDE = SO_SBAR + RA * RA,     // per-side blocks, SIDE_STRIDE each
};
// per-side block offsets (relative to SO_SIDE + side * SIDE_STRIDE)
enum : int {
    SS_F1 = 0,                 // Q1 = A F1 (range part), r x rho1
    SS_P1 = SS_F1 + RA * RA,   // F1 F1^T
    SS_T = SS_P1 + RA * RA,    // projection coefficients / range-finder transform
    SS_M1 = SS_T + RA * RA,    // Q1^T A (BUG: top block of X1^T X)
    SS_R0 = SS_M1 + RA * RA,   // Cholesky factor of the range-finder Gram
    SS_RI = SS_R0 + RA * RA,   // inverse Cholesky factor of C^T C (basis = C RI)
    SS_V0 = SS_RI + RA * RA,   // slow path: eigenvectors of G0
    SS_WC = SS_V0 + RA * RA,   // W-side completion coefficients (RA rows, stride WCS)
    SIDE_STRIDE = SS_WC + RA * 3 * RA,
};
constexpr int SO_XTPSI = SO_SIDE + 2 * SIDE_STRIDE;  // KA x QW   X^T psi
constexpr int SO_MTDW = SO_XTPSI + KA * QW;          // QW x KA   MRed^T diag(Dvec) W
constexpr int SO_TMP = SO_MTDW + QW * KA;            // 3 x KA x KA general temporaries
constexpr int SO_DBG = SO_TMP + 3 * KA * KA;           // KA x KA: input of the last truncation SVD
constexpr int SO_S0 = SO_DBG + KA * KA;                 // RA x RA: S entering the energy (parallel-rejection loop)
constexpr int SO_END = SO_S0 + RA * RA;
static_assert(SO_END <= SCRW, "per-CTA scratch too small");

struct WSmem {
    double S[KA * KA];     // state S (ld KA)
    double work[WORKD];    // phase-dependent union
    double vec[6 * KA + 2 * QW];
    double dmisc[32];
    int imisc[32];
    int wcand[RA];
    double wnrm[RA];
    int perm[KA];
    double sig[KA];
    unsigned long long mbar[2];   // MIXED mode: completion barriers of the two tensor-core chunk buffers
    unsigned tmem_slot;           // MIXED mode: TMEM base address written by tcgen05.alloc
};

// Per-side bookkeeping of one augmentation (identical in every CTA).
struct SideInfo {
    int rho1;      // numerical rank of the old basis (range part of Q1)
    int fast1;     // 1: Q1 = A R1^{-1} (certified); 0: Jacobi (F1 = V diag(lambda^-1/2))
    int rho2;      // numerical rank of the projected new directions
    int fast2;     // 1: certified CholQR2 path
    int need2;     // completion vectors appended after the range part of Q2
    int cand0;     // first X candidate used by Q2's completion
    double scale;  // Frobenius norm of [A B]
};

struct WCtx {
    DevProblem P;
    WideState st;
    WSmem* sm;
    double* scr;    // this CTA's scratch
    int G, b;
    int c0, c1, m0, m1;
    int r;          // current rank
    double* psi_in;
    double* psi_out;
    unsigned gen;
    int parity;
    const double* redp;  // reduced buffer of the latest reduction
    int cur_n;
    unsigned long long* prof;
    SideInfo side[2];
    int mixed;           // 1: MIXED precision (tensor-core operator Grams where the width >= 32)
    umma::TcCtx tc;      // tensor-core state (MIXED only)
};

// Widths from which the MIXED mode forms the operator Grams on the tensor cores.
constexpr int kTcMinWidth = 32;

// Rows per tile that fit `avail` doubles of shared memory at `per_row` doubles a row.
__device__ __forceinline__ int rows_fit(int avail, int per_row) {
    const int r = avail / per_row;
    return r < 1 ? 1 : (r > TRMAX ? TRMAX : r);
}

__device__ __forceinline__ bool is_bnd_w(const DevProblem& P, int c) {
    if constexpr (kThreeD) {
        // 3D: cell (i, j, k) at row (k nx + i) ny + j; boundary on any of the six faces
        const int nxy = P.nx * P.ny;
        const int k = c / nxy, rr = c - k * nxy;
        const int i = rr / P.ny, j = rr - i * P.ny;
        return k == 0 || k == P.nz - 1 || i == 0 || j == 0 || i == P.nx - 1 || j == P.ny - 1;
    } else {
        int i = c / P.ny, j = c - (c / P.ny) * P.ny;
        return i == 0 || j == 0 || i == P.nx - 1 || j == P.ny - 1;
    }
}

__device__ __forceinline__ bool wsync(WCtx& x) {
    ProfScope ps(x.prof, PF_BARRIER);
    prof_count(x.prof, PF_BARRIERS, 1ull);
    return team_sync(x.st.bar, x.st.status, x.G, x.b, x.gen, x.st.diag, x.P.spin_limit, x.P.fault_barrier);
}

__device__ __forceinline__ double* wpart(const WCtx& x, int g) {
    return x.st.part + ((size_t)x.parity * x.G + g) * PMAXW;
}

// Publish `cnt` partial entries of this CTA starting at `off` from the shared
// accumulator (chunked Gram passes publish several pieces before one reduce).
__device__ __forceinline__ void wpublish_chunk(WCtx& x, const double* acc, int off, int cnt) {
    double* dst = wpart(x, x.b) + off;
    for (int e = threadIdx.x; e < cnt; e += NT) dst[e] = acc[e];
}

// Two-stage team sum of entries [0, count) of the partials into the reduced
// buffer of the same parity (x.redp afterwards). Before the call every CTA
// published its partial with wpublish_chunk. The hook runs between the two
// barriers (used to zero X rows that other CTAs stop reading at the first
// barrier). A reduced buffer stays valid until the second reduction after it.
template <class Hook>
__device__ inline bool wreduce(WCtx& x, int count, Hook hook) {
    if (!wsync(x)) return false;
    hook();
    if (x.G == 1) {
        // one CTA: its partial is the sum; read it in place (the partial of
        // this parity is next written two reductions later, like `red`)
        x.redp = wpart(x, 0);
        x.parity ^= 1;
        return wsync(x);
    }
    {
        ProfScope ps(x.prof, PF_REDUCE);
        // CTA b sums the slice [e0, e1) over the G partials. Blocks of RCH
        // elements x RSPL partial-splits keep RSPL independent L2 loads in
        // flight per element (adjacent threads read adjacent elements); the
        // splits are combined in a fixed order, so the sum is deterministic.
        constexpr int RCH = 16, RSPL = NT / RCH;
        __shared__ double s_part[NT];
        const int per = (count + x.G - 1) / x.G;
        const int e0 = x.b * per, e1 = min(count, e0 + per);
        const double* base = x.st.part + (size_t)x.parity * x.G * PMAXW;
        double* red = x.st.red + (size_t)x.parity * PMAXW;
        const int el = threadIdx.x % RCH, sp = threadIdx.x / RCH;
        for (int eb = e0; eb < e1; eb += RCH) {
            const int e = eb + el;
            double a = 0.0;
            if (e < e1)
                for (int g = sp; g < x.G; g += RSPL) a += ldcg(base + (size_t)g * PMAXW + e);
            s_part[threadIdx.x] = a;
            __syncthreads();
            if (threadIdx.x < RCH && eb + threadIdx.x < e1) {
                double t = 0.0;
                for (int q = 0; q < RSPL; ++q) t += s_part[q * RCH + threadIdx.x];
                red[eb + threadIdx.x] = t;
            }
            __syncthreads();
        }
    }
    x.redp = x.st.red + (size_t)x.parity * PMAXW;
    x.parity ^= 1;
    return wsync(x);
}
__device__ inline bool wreduce(WCtx& x, int count) {
    return wreduce(x, count, [] {});
}

// red[off + i*n + j] -> D[i*ld + j]  (m x n)
__device__ inline void load_red(const WCtx& x, int off, int m, int n, double* D, int ld) {
    for (int e = threadIdx.x; e < m * n; e += NT) D[(e / n) * ld + e % n] = ldcg(x.redp + off + e);
    __syncthreads();
}

// ---------------------------------------------------------------- algebra ---
// C (m x n) = alpha op(A) op(B) + beta C; op(A) = A^T when ta (A stored k x m),
// op(B) = B^T when tb (B stored n x k). C must not alias A or B.
__device__ inline void g_mm(double* C, int ldc, const double* A, int lda, bool ta, const double* B, int ldb, bool tb,
                            int m, int k, int n, double alpha = 1.0, double beta = 0.0) {
    for (int e = threadIdx.x; e < m * n; e += NT) {
        const int i = e / n, j = e - (e / n) * n;
        double s = 0.0;
        for (int l = 0; l < k; ++l) {
            const double a = ta ? A[l * lda + i] : A[i * lda + l];
            const double bb = tb ? B[j * ldb + l] : B[l * ldb + j];
            s = fma(a, bb, s);
        }
        double v = alpha * s;
        if (beta != 0.0) v = fma(beta, C[i * ldc + j], v);
        C[i * ldc + j] = v;
    }
    __syncthreads();
}
__device__ inline void g_copy(double* D, int ldd, const double* A, int lda, int m, int n) {
    for (int e = threadIdx.x; e < m * n; e += NT) D[(e / n) * ldd + e % n] = A[(e / n) * lda + e % n];
    __syncthreads();
}
__device__ inline void g_zero(double* D, int ldd, int m, int n) {
    for (int e = threadIdx.x; e < m * n; e += NT) D[(e / n) * ldd + e % n] = 0.0;
    __syncthreads();
}

// ----------------------------------------------------------- row helpers ---
// Tile moves between global memory and shared memory. Loads are asynchronous
// copies (cp.async): a thread issues every copy of its share of the tile before
// waiting once, so a tile costs about one memory latency instead of one per
// element, and the data never passes through registers. Pairs of doubles move
// as 16-byte copies that bypass L1 (.cg); single doubles use 8-byte copies
// through L1 (.ca), which is safe because a CTA only loads rows that it wrote
// itself in this launch (L1 holds no other SM's data for them).
__device__ __forceinline__ double2 ldcg2(const double* p) { return __ldcg(reinterpret_cast<const double2*>(p)); }
__device__ __forceinline__ bool pairs_ok(const double* t, const double* A, int k, int c0, int lda, int ldt, int tc) {
    return ((k | c0 | lda | ldt | tc) & 1) == 0 &&
           ((reinterpret_cast<uintptr_t>(t) | reinterpret_cast<uintptr_t>(A)) & 15) == 0;
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// rows [r0, r0+nr) x cols [c0, c0+k) of A (ld lda) -> t (ld ldt) at column tc.
// On return this thread's copies have landed; the caller's __syncthreads makes
// the whole tile visible to the CTA.
__device__ __forceinline__ void wload(double* t, int ldt, int tc, const double* A, int lda, int c0, int r0, int nr,
                                      int k) {
    if (pairs_ok(t, A, k, c0, lda, ldt, tc)) {
        const int h = k >> 1;
        for (int e = threadIdx.x; e < nr * h; e += NT) {
            const int r = e / h, j = 2 * (e - r * h);
            cp_async16(t + r * ldt + tc + j, A + (size_t)(r0 + r) * lda + c0 + j);
        }
    } else {
        for (int e = threadIdx.x; e < nr * k; e += NT) {
            const int r = e / k, j = e - r * k;
            cp_async8(t + r * ldt + tc + j, A + (size_t)(r0 + r) * lda + c0 + j);
        }
    }
    cp_async_wait_all();
}
__device__ __forceinline__ void wstore(double* A, int lda, int c0, const double* t, int ldt, int tc, int r0, int nr,
                                       int k) {
    if (pairs_ok(t, A, k, c0, lda, ldt, tc)) {
        const int h = k >> 1;
        for (int e = threadIdx.x; e < nr * h; e += NT) {
            const int r = e / h, j = 2 * (e - r * h);
            *reinterpret_cast<double2*>(A + (size_t)(r0 + r) * lda + c0 + j) =
                *reinterpret_cast<const double2*>(t + r * ldt + tc + j);
        }
        return;
    }
    for (int e = threadIdx.x; e < nr * k; e += NT) {
        const int r = e / k, j = e - r * k;
        A[(size_t)(r0 + r) * lda + c0 + j] = t[r * ldt + tc + j];
    }
}

// Row products of a shared-memory tile: for rows r < nr and columns j < w,
//   epi(r, j, sum_{l < kd} A[r * lda + l] * mget(l, j))
// with one FMA chain per output in increasing l (the rounding of the plain
// per-element loop). A thread owns a micro-tile of RB rows x 2 columns: per l it
// reads RB entries of A and 2 of M for 2 RB independent FMAs, instead of two
// shared loads per dependent FMA. Threads of a warp share rows (broadcast reads
// of A) and take adjacent column pairs (consecutive entries of M).
template <int RB, class MGet, class Epi>
__device__ __forceinline__ void row_mm(int nr, int kd, int w, const double* A, int lda, MGet mget, Epi epi) {
    const int cb = (w + 1) >> 1, rbn = (nr + RB - 1) / RB;
    for (int tile = threadIdx.x; tile < rbn * cb; tile += NT) {
        const int rb = tile / cb, c2 = tile - rb * cb;
        const int r0 = rb * RB, j0 = 2 * c2;
        const bool j1 = j0 + 1 < w;
        double acc[RB][2];
#pragma unroll
        for (int i = 0; i < RB; ++i) acc[i][0] = acc[i][1] = 0.0;
        const double* ap[RB];
#pragma unroll
        for (int i = 0; i < RB; ++i) ap[i] = A + min(r0 + i, nr - 1) * lda;
        for (int l = 0; l < kd; ++l) {
            const double m0 = mget(l, j0);
            const double m1 = j1 ? mget(l, j0 + 1) : 0.0;
#pragma unroll
            for (int i = 0; i < RB; ++i) {
                const double a = ap[i][l];
                acc[i][0] = fma(a, m0, acc[i][0]);
                acc[i][1] = fma(a, m1, acc[i][1]);
            }
        }
#pragma unroll
        for (int i = 0; i < RB; ++i)
            if (r0 + i < nr) {
                epi(r0 + i, j0, acc[i][0]);
                if (j1) epi(r0 + i, j0 + 1, acc[i][1]);
            }
    }
}

// One Gram block of a feature tile: acc[off + i*wb + j] += sum_r F[r][ca+i] F[r][cb+j].
struct GBlock {
    int ca, wa, cb, wb, off;
};
// Accumulate a list of blocks over a tile of nr rows; 2x2 register tiles. The
// tiles of all blocks are flattened; each warp holds 32/G tiles in G row
// subgroups (subgroup s sums rows s, s+G, ...; lanes of a subgroup share rows,
// so their loads broadcast), G in {1, 2, 4, 8} minimising rounds x rows per
// lane. The G partial sums of a tile meet in a fixed xor butterfly: the result
// depends only on (blocks, nr), not on timing.
__device__ inline void gram_blocks(double* acc, const double* F, int ldf, int nr, const GBlock* bl, int nb) {
    int T = 0;
    for (int q = 0; q < nb; ++q) T += ((bl[q].wa + 1) >> 1) * ((bl[q].wb + 1) >> 1);
    int G = 1, best = 0x7fffffff;
    for (int g = 1; g <= 8; g <<= 1) {
        const int slots = (NT / 32) * (32 / g);
        const int cost = ((T + slots - 1) / slots) * ((nr + g - 1) / g);
        if (cost < best) {
            best = cost;
            G = g;
        }
    }
    const int L = 32 / G, slots = (NT / 32) * L;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int sg = lane / L, tl = lane - (lane / L) * L;
    for (int base = 0; base < T; base += slots) {
        int off = base + warp * L + tl;
        const bool valid = off < T;
        GBlock g{0, 2, 0, 2, 0};
        int hj = 1;
        if (valid)
            for (int q = 0; q < nb; ++q) {
                g = bl[q];
                hj = (g.wb + 1) >> 1;
                const int cnt = ((g.wa + 1) >> 1) * hj;
                if (off < cnt) break;
                off -= cnt;
            }
        const int i = 2 * (off / hj), j = 2 * (off - (off / hj) * hj);
        const bool i1 = i + 1 < g.wa, j1 = j + 1 < g.wb;
        double s00 = 0.0, s01 = 0.0, s10 = 0.0, s11 = 0.0;
        if (valid)
            for (int r = sg; r < nr; r += G) {
                const double* row = F + r * ldf;
                const double a0 = row[g.ca + i], a1 = i1 ? row[g.ca + i + 1] : 0.0;
                const double b0 = row[g.cb + j], b1 = j1 ? row[g.cb + j + 1] : 0.0;
                s00 = fma(a0, b0, s00);
                s01 = fma(a0, b1, s01);
                s10 = fma(a1, b0, s10);
                s11 = fma(a1, b1, s11);
            }
        for (int o = L; o < 32; o <<= 1) {
            s00 += __shfl_xor_sync(0xffffffffu, s00, o);
            s01 += __shfl_xor_sync(0xffffffffu, s01, o);
            s10 += __shfl_xor_sync(0xffffffffu, s10, o);
            s11 += __shfl_xor_sync(0xffffffffu, s11, o);
        }
        if (valid && sg == 0) {
            double* o = acc + g.off + i * g.wb + j;
            o[0] += s00;
            if (j1) o[1] += s01;
            if (i1) {
                o[g.wb] += s10;
                if (j1) o[g.wb + 1] += s11;
            }
        }
    }
}

}  // namespace TITUS_WIDE_NS
}  // namespace titus
