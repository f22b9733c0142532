// Rank-adaptive DLR energy loops as one persistent kernel per solve:
//   METHOD 1  SolveFirstCollisionSourceDLRParallel     (SolverCSD.jl:1726-2008)
//   METHOD 2  SolveFirstCollisionSourceDLRBUGRejection (SolverCSD.jl:2011-2374)
// with truncate! (:3369-3399) and the augmented bases qr([X K]) (:149-153).
//
// Step structure (every arrow into a reduction is one team barrier pair):
//   A   boundary inflow + first dose half-step (own cells)          -> barrier
//   B   uncollided sweep; streaming Grams X^T L_d X, W^T A_d W     -> reduce
//   C   K = X S - dE sum L_d X S C_d ; L = W S^T - dE sum A_d W S^T G_d^T,
//       with the Grams of [X K] and [W L]                         -> reduce
//   AUG Q1 = orth(X) from the Gram (certified Cholesky or Jacobi),
//       K' = (I - Q1 Q1^T)^2 K in two passes                      -> 2 reduces
//       range finder of K' (certified CholQR2, or Jacobi twice)    -> 1-2 reduces
//       X~ = [K' basis, completion] materialised in X[:, r:2r]
//   TRUNC one-sided Jacobi SVD of the 2r x 2r S, l1 tail rank, X <- [X X~] U_k
//   OS  out-scattering L = W S^T / (1 + dE D), W = orth(L), S = L^T W
//   IS  in-scattering K / L / S, augmentation, truncation (BUG: rejection test)
// Every CTA holds bit-identical small matrices, so rank and rejection
// decisions are uniform across the team.
#pragma once
#include "wide_linalg.cuh"

namespace titus {
namespace TITUS_WIDE_NS {

constexpr double kCertW = 1e5;   // ||R||_F ||R^-1||_F bound of the certified Cholesky paths
constexpr double kNullSvd = 1e-12;
__device__ __forceinline__ double raw_gram_floor(int k) { return 4.0 * k * 2.2e-16; }
constexpr double kGradedFloor = 1e-32;

__device__ __forceinline__ double* sside(const WCtx& x, int s, int off) {
    return x.scr + SO_SIDE + s * SIDE_STRIDE + off;
}

// ------------------------------------------------------------- row kernels ---
// F[r][fc + d*k + j] = (L_d A)[r0 + r][j]; zero on boundary rows (stencils.jl:26-128;
// 3D problems append L2z, L1z, the same rows with dz and the z neighbours).
__device__ inline void w_stencil(const WCtx& x, const double* A, int lda, int r0, int nr, int k, double* F, int ldf,
                                 int fc) {
    const DevProblem& P = x.P;
    const double hx = 0.5 / P.dx, hy = 0.5 / P.dy;
    const double ix = 1.0 / P.dx, iy = 1.0 / P.dy;
    for (int e = threadIdx.x; e < nr * k; e += NT) {
        const int r = e / k, j = e - (e / k) * k;
        const int c = r0 + r;
        double l2x = 0.0, l2y = 0.0, l1x = 0.0, l1y = 0.0, l2z = 0.0, l1z = 0.0;
        if (!is_bnd_w(P, c)) {
            const double* p = A + (size_t)c * lda + j;
            const double a0 = ldcg(p) * __ldg(P.rinv + c);
            const double axm = ldcg(p - (size_t)P.ny * lda) * __ldg(P.rinv + c - P.ny);
            const double axp = ldcg(p + (size_t)P.ny * lda) * __ldg(P.rinv + c + P.ny);
            const double aym = ldcg(p - lda) * __ldg(P.rinv + c - 1);
            const double ayp = ldcg(p + lda) * __ldg(P.rinv + c + 1);
            l2x = (axp - axm) * hx;
            l2y = (ayp - aym) * hy;
            l1x = a0 * ix - hx * axm - hx * axp;
            l1y = a0 * iy - hy * aym - hy * ayp;
            if constexpr (kThreeD) {
                const int nxy = P.nx * P.ny;
                const double hz = 0.5 / P.dz, iz = 1.0 / P.dz;
                const double azm = ldcg(p - (size_t)nxy * lda) * __ldg(P.rinv + c - nxy);
                const double azp = ldcg(p + (size_t)nxy * lda) * __ldg(P.rinv + c + nxy);
                l2z = (azp - azm) * hz;
                l1z = a0 * iz - hz * azm - hz * azp;
            }
        }
        double* row = F + r * ldf + fc;
        row[0 * k + j] = l2x;
        row[1 * k + j] = l2y;
        row[2 * k + j] = l1x;
        row[3 * k + j] = l1y;
        if constexpr (kThreeD) {
            row[4 * k + j] = l2z;
            row[5 * k + j] = l1z;
        }
    }
}
// F[r][fc + d*k + j] = (A_d B)[r0 + r][j] (sparse P_N operators Ax, Az, |Ax|, |Az|
// and, for 3D problems, Ay, |Ay|).
// A thread takes one (operator, row) and a group of up to SPJ consecutive
// columns: per nonzero it loads the index and value once and SPJ contiguous
// entries of B, so the loads of a row segment are independent. The sum over
// the nonzeros runs in CSR order for every column, as before.
__device__ inline void w_spmm(const WCtx& x, const double* B, int ldb, int r0, int nr, int k, double* F, int ldf,
                              int fc) {
    constexpr int SPJ = 8;
    const int ng = (k + SPJ - 1) / SPJ;
    for (int e = threadIdx.x; e < NOPS_W * nr * ng; e += NT) {
        const int d = e / (nr * ng);
        const int rem = e - d * nr * ng;
        const int r = rem / ng, g = rem - (rem / ng) * ng;
        const int j0 = g * SPJ, w = min(SPJ, k - j0);
        const Csr& A = x.P.op[d];
        const int m = r0 + r;
        double s[SPJ];
#pragma unroll
        for (int u = 0; u < SPJ; ++u) s[u] = 0.0;
        const int p1 = __ldg(A.rowptr + m + 1);
        for (int p = __ldg(A.rowptr + m); p < p1; ++p) {
            const double v = __ldg(A.val + p);
            const double* bp = B + (size_t)__ldg(A.col + p) * ldb + j0;
            double bv[SPJ];
#pragma unroll
            for (int u = 0; u < SPJ; ++u) bv[u] = u < w ? ldcg(bp + u) : 0.0;
#pragma unroll
            for (int u = 0; u < SPJ; ++u) s[u] = fma(v, bv[u], s[u]);
        }
        double* out = F + r * ldf + fc + d * k + j0;
#pragma unroll
        for (int u = 0; u < SPJ; ++u)
            if (u < w) out[u] = s[u];
    }
}

// dose += 1/2 dE (X[c,:k] v + psi[c,:] MRed[0,:]) stopping[sidx] / rho (SolverCSD.jl:990-997)
static __device__ __noinline__ void w_dose(WCtx& x, int sidx, const double* v, int k, bool zero_bnd_x) {
    const DevProblem& P = x.P;
    const double f = 0.5 * P.dE * P.stopping[sidx];
    for (int c = x.c0 + threadIdx.x; c < x.c1; c += NT) {
        double xv = 0.0;
        if (!(zero_bnd_x && is_bnd_w(P, c))) {
            // the row's entries are loaded in groups of 8 before they are summed
            const double* xr = x.st.X + (size_t)c * KA;
            for (int j0 = 0; j0 < k; j0 += 8) {
                double xl[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) xl[u] = j0 + u < k ? ldcg(xr + j0 + u) : 0.0;
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (j0 + u < k) xv = fma(xl[u], v[j0 + u], xv);
            }
        }
        const double* pr = x.psi_in + (size_t)c * QW;
        double u = 0.0;
        for (int kq = 0; kq < P.q; ++kq) u = fma(pr[kq], P.mred[kq], u);
        x.st.dose[c] += f * (xv + u) * P.rinv[c];
    }
}

// v = S W[0,:k]^T (S: shared, ld KA; W row 0 from global)
__device__ inline void sw0(WCtx& x, const double* S, int ldS, int k, double* v, double* w0) {
    for (int j = threadIdx.x; j < k; j += NT) w0[j] = ldcg(x.st.W + j);
    __syncthreads();
    for (int i = threadIdx.x; i < k; i += NT) {
        double s = 0.0;
        for (int j = 0; j < k; ++j) s = fma(S[i * ldS + j], w0[j], s);
        v[i] = s;
    }
    __syncthreads();
}

// ---- phase A: boundary inflow at energy[n-1] (PsiBeam, :977-988), first dose half-step
static __device__ __noinline__ void w_phase_A(WCtx& x, int n) {
    ProfScope ps_(x.prof, PF_PROLOGUE);
    const DevProblem& P = x.P;
    WSmem* sm = x.sm;
    const int k = x.r;
    sw0(x, sm->S, KA, k, sm->vec, sm->vec + KA);
    const double bce = P.bc_energy[n - 2];
    for (int c = x.c0 + threadIdx.x; c < x.c1; c += NT) {
        if (is_bnd_w(P, c)) {
            double* pr = x.psi_in + (size_t)c * QW;
            const double bs = bce * P.bc_space[c];
            for (int kq = 0; kq < P.q; ++kq) pr[kq] = bs * P.bc_angle[kq];
        }
    }
    __syncthreads();
    w_dose(x, n - 2, sm->vec, k, false);
}

// ---- uncollided sweep of own cells, psi_in -> psi_out (solveFluxUpwind! :388-463, :1000-1005)
static __device__ __noinline__ void w_sweep(WCtx& x, double sigma0) {
    ProfScope ps_(x.prof, PF_PROLOGUE);
    const DevProblem& P = x.P;
    const double dE = P.dE;
    const double den = 1.0 + dE * sigma0;
    const int q = P.q;
    // the per-ordinate quotients Omega_x / dx, Omega_z / dy (3D: Omega_y / dz), formed once
    __shared__ double s_cx[QW], s_cz[QW], s_cy[kThreeD ? QW : 1];
    __syncthreads();   // a previous call's readers are done
    for (int l = threadIdx.x; l < q; l += NT) {
        s_cx[l] = P.omega[l * 3 + 0] / P.dx;
        s_cz[l] = P.omega[l * 3 + 2] / P.dy;
        if constexpr (kThreeD) s_cy[l] = P.omega[l * 3 + 1] / P.dz;
    }
    __syncthreads();
    const int nxy = P.nx * P.ny;
    // four entries per thread: their upwind neighbours are loaded before any is used
    constexpr int SU = 4;
    const int cnt = (x.c1 - x.c0) * q;
    for (int b = threadIdx.x; b < cnt; b += SU * NT) {
        double pcv[SU], nxv[SU], nyv[SU], nzv[SU];
        int cv[SU], kv[SU], ncx[SU], ncy[SU], ncz[SU];
#pragma unroll
        for (int u = 0; u < SU; ++u) {
            const int e = b + u * NT;
            const int c = x.c0 + e / q, kq = e - (e / q) * q;
            cv[u] = c;
            kv[u] = kq;
            pcv[u] = nxv[u] = nyv[u] = nzv[u] = 0.0;
            ncx[u] = ncy[u] = ncz[u] = c;
            if (e < cnt) {
                pcv[u] = ldcg(x.psi_in + (size_t)c * QW + kq);
                if (!is_bnd_w(P, c)) {
                    ncx[u] = P.omega[kq * 3 + 0] >= 0.0 ? c - P.ny : c + P.ny;
                    ncy[u] = P.omega[kq * 3 + 2] >= 0.0 ? c - 1 : c + 1;
                    nxv[u] = ldcg(x.psi_in + (size_t)ncx[u] * QW + kq);
                    nyv[u] = ldcg(x.psi_in + (size_t)ncy[u] * QW + kq);
                    if constexpr (kThreeD) {
                        ncz[u] = P.omega[kq * 3 + 1] >= 0.0 ? c - nxy : c + nxy;
                        nzv[u] = ldcg(x.psi_in + (size_t)ncz[u] * QW + kq);
                    }
                }
            }
        }
#pragma unroll
        for (int u = 0; u < SU; ++u) {
            const int e = b + u * NT;
            if (e >= cnt) continue;
            const int c = cv[u], kq = kv[u];
            const double pc = pcv[u];
            double flux = 0.0;
            if (!is_bnd_w(P, c)) {
                const double ox = P.omega[kq * 3 + 0], oz = P.omega[kq * 3 + 2];
                const double f0 = pc * P.rinv[c];
                double ew, ns;
                if (ox >= 0.0) ew = f0 - nxv[u] * P.rinv[ncx[u]];
                else ew = nxv[u] * P.rinv[ncx[u]] - f0;
                if (oz >= 0.0) ns = f0 - nyv[u] * P.rinv[ncy[u]];
                else ns = nyv[u] * P.rinv[ncy[u]] - f0;
                flux = s_cx[kq] * ew + s_cz[kq] * ns;
                if constexpr (kThreeD) {
                    double tb;
                    if (P.omega[kq * 3 + 1] >= 0.0) tb = f0 - nzv[u] * P.rinv[ncz[u]];
                    else tb = nzv[u] * P.rinv[ncz[u]] - f0;
                    flux = flux + s_cy[kq] * tb;
                }
            }
            double out = (pc - dE * flux) / den;
            if (kq == 0 && P.restore[c]) out = pc;
            x.psi_out[(size_t)c * QW + kq] = out;
        }
    }
}

// ---- streaming Grams of width k over A (cells, stencils) and B (moments, P_N
// operators): acc[d k^2 ..] = A^T L_d A, acc[(NOPS_W+d) k^2 ..] = B^T A_d B.
// `cw` = width of A and B used; blocks for d in [d0, d1) only (chunking).
static __device__ __noinline__ void w_grams_pass(WCtx& x, const double* A, const double* B, int cw, int d0, int d1, int off0,
                                    double* acc, double* F, int ldf, int tr) {
    ProfScope ps_(x.prof, PF_ROWS_STREAM);
    GBlock bl[NOPS_W];
    int nb = 0;
    const int kk = cw * cw;
    for (int d = d0; d < d1; ++d) bl[nb++] = GBlock{0, cw, (d + 1) * cw, cw, (d - d0) * kk};
    for (int r0 = x.c0; r0 < x.c1; r0 += tr) {
        const int nr = min(tr, x.c1 - r0);
        wload(F, ldf, 0, A, KA, 0, r0, nr, cw);
        w_stencil(x, A, KA, r0, nr, cw, F, ldf, cw);
        __syncthreads();
        gram_blocks(acc + off0, F, ldf, nr, bl, nb);
        __syncthreads();
    }
    for (int r0 = x.m0; r0 < x.m1; r0 += tr) {
        const int nr = min(tr, x.m1 - r0);
        wload(F, ldf, 0, B, KA, 0, r0, nr, cw);
        w_spmm(x, B, KA, r0, nr, cw, F, ldf, cw);
        __syncthreads();
        gram_blocks(acc + off0 + (d1 - d0) * kk, F, ldf, nr, bl, nb);
        __syncthreads();
    }
}

// ---- MIXED precision: the same eight operator Grams on the tensor cores
// (umma.cuh). Per side, one run over the CTA's own rows stages the factor
// (N operand) and its four operator images (M operand, stacked) chunk by
// chunk straight from global memory -- the stencil / sparse products are
// formed where they are staged, in FP64 exactly as w_stencil / w_spmm form
// them -- and accumulates D[d cw + i][j] = sum_r (L_d A)[r][i] A[r][j] = G_d[j][i]
// in TMEM (FP32). The sums are written as this CTA's partial at the FP64
// layout [G_0..G_3 | C_0..C_3] (cw x cw each), ready for wreduce. Uses the
// whole shared work area as staging. Returns false if a completion wait timed
// out (device status set).
static __device__ __noinline__ bool w_grams_tc(WCtx& x, const double* A, const double* B, int cw) {
    ProfScope ps_(x.prof, PF_ROWS_STREAM);
    const umma::GramShape g = umma::gram_shape(NOPS_W * cw, cw);
    unsigned char* stage = reinterpret_cast<unsigned char*>(x.sm->work);
    double* dst = wpart(x, x.b);
    const int kk = cw * cw;
    const DevProblem& P = x.P;
    bool ok = true;
    for (int side = 0; side < 2; ++side) {
        const int r0 = side == 0 ? x.c0 : x.m0;
        const int rows = (side == 0 ? x.c1 : x.m1) - r0;
        double* out = dst + side * NOPS_W * kk;
        if (rows <= 0) {
            for (int e = threadIdx.x; e < NOPS_W * kk; e += NT) out[e] = 0.0;
            __syncthreads();
            continue;
        }
        bool run;
        if (side == 0) {
            const double hx = 0.5 / P.dx, hy = 0.5 / P.dy, ix = 1.0 / P.dx, iy = 1.0 / P.dy;
            run = umma::gram_run<NT, NOPS_W>(x.tc, g, stage, rows, true, [&](int r, int j, double* v) {
                const int c = r0 + r;
                const double* p = A + (size_t)c * KA + j;
                v[0] = ldcg(p);
                double l2x = 0.0, l2y = 0.0, l1x = 0.0, l1y = 0.0, l2z = 0.0, l1z = 0.0;
                if (!is_bnd_w(P, c)) {
                    const double a0 = v[0] * __ldg(P.rinv + c);
                    const double axm = ldcg(p - (size_t)P.ny * KA) * __ldg(P.rinv + c - P.ny);
                    const double axp = ldcg(p + (size_t)P.ny * KA) * __ldg(P.rinv + c + P.ny);
                    const double aym = ldcg(p - KA) * __ldg(P.rinv + c - 1);
                    const double ayp = ldcg(p + KA) * __ldg(P.rinv + c + 1);
                    l2x = (axp - axm) * hx;
                    l2y = (ayp - aym) * hy;
                    l1x = a0 * ix - hx * axm - hx * axp;
                    l1y = a0 * iy - hy * aym - hy * ayp;
                    if constexpr (kThreeD) {
                        const int nxy = P.nx * P.ny;
                        const double hz = 0.5 / P.dz, iz = 1.0 / P.dz;
                        const double azm = ldcg(p - (size_t)nxy * KA) * __ldg(P.rinv + c - nxy);
                        const double azp = ldcg(p + (size_t)nxy * KA) * __ldg(P.rinv + c + nxy);
                        l2z = (azp - azm) * hz;
                        l1z = a0 * iz - hz * azm - hz * azp;
                    }
                }
                v[1] = l2x;
                v[2] = l2y;
                v[3] = l1x;
                v[4] = l1y;
                if constexpr (kThreeD) {
                    v[5] = l2z;
                    v[6] = l1z;
                }
            });
        } else {
            run = umma::gram_run<NT, NOPS_W>(x.tc, g, stage, rows, true, [&](int r, int j, double* v) {
                const int m = r0 + r;
                v[0] = ldcg(B + (size_t)m * KA + j);
#pragma unroll
                for (int d = 0; d < NOPS_W; ++d) {
                    const Csr& Op = P.op[d];
                    double s = 0.0;
                    const int p1 = __ldg(Op.rowptr + m + 1);
                    for (int q = __ldg(Op.rowptr + m); q < p1; ++q)
                        s = fma(__ldg(Op.val + q), ldcg(B + (size_t)__ldg(Op.col + q) * KA + j), s);
                    v[1 + d] = s;
                }
            });
        }
        const bool fin = umma::gram_finish(x.tc);
        if (!(run && fin)) {
            ok = false;
            break;
        }
        umma::gram_read<NT>(x.tc, g, [&](int m, int n, double val) {
            const int d = m / cw, i = m - d * cw;
            out[d * kk + n * cw + i] = val;
        });
    }
    return ok;
}

// MIXED mode setup and teardown around a launch's work: warp 0 allocates the
// TMEM accumulators, thread 0 initialises the two completion barriers; at the
// end every outstanding MMA is waited for (bounded) before the TMEM is freed.
__device__ inline void tc_setup(WCtx& x) {
    x.mixed = x.P.precision == 1;
    if (!x.mixed) return;
    if (threadIdx.x < 32) umma::tmem_alloc(&x.sm->tmem_slot, umma::TMEM_COLS);
    if (threadIdx.x == 0) {
        umma::mbar_init(&x.sm->mbar[0], 1);
        umma::mbar_init(&x.sm->mbar[1], 1);
        umma::fence_mbar_init();
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    x.tc.mbar = x.sm->mbar;
    x.tc.tmem = x.sm->tmem_slot;
    x.tc.phase[0] = x.tc.phase[1] = 0u;
    x.tc.pending[0] = x.tc.pending[1] = 0;
    x.tc.status = x.st.status;
    x.tc.limit = umma::kWaitCycles;
}
__device__ inline void tc_teardown(WCtx& x) {
    if (!x.mixed) return;
    umma::gram_finish(x.tc);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    if (threadIdx.x < 32) umma::tmem_dealloc(x.tc.tmem, umma::TMEM_COLS);
}

__device__ inline void w_acc_zero(double* acc, int cnt) {
    for (int e = threadIdx.x; e < cnt; e += NT) acc[e] = 0.0;
    __syncthreads();
}

// Streaming Grams with the rank-r factors (before X[bnd,:] = 0, :1856-1859),
// published at [G_0..G_{NOPS_W-1} | C_0..C_{NOPS_W-1}] (r x r each) and reduced; X's boundary
// rows are zeroed between the barriers (:1859).
static __device__ __noinline__ bool w_stream_grams(WCtx& x) {
    ProfScope ps_(x.prof, PF_ROWS_STREAM);
    const int k = x.r;
    if (x.mixed && k >= kTcMinWidth) {
        if (!w_grams_tc(x, x.st.X, x.st.W, k)) return false;
    } else {
        double* acc = x.sm->work;
        double* F = x.sm->work + 2 * NOPS_W * k * k;
        w_acc_zero(acc, 2 * NOPS_W * k * k);
        w_grams_pass(x, x.st.X, x.st.W, k, 0, NOPS_W, 0, acc, F, (NOPS_W + 1) * k,
                     rows_fit(WORKD - 2 * NOPS_W * k * k, (NOPS_W + 1) * k));
        wpublish_chunk(x, acc, 0, 2 * NOPS_W * k * k);
    }
    return wreduce(x, 2 * NOPS_W * k * k, [&] {
        for (int c = x.c0 + threadIdx.x; c < x.c1; c += NT)
            if (is_bnd_w(x.P, c))
                for (int j = 0; j < k; ++j) x.st.X[(size_t)c * KA + j] = 0.0;
    });
}

// After the streaming Grams: SC_d = S C_d, SG_d = S^T G_d^T (stacked, rows d*k + l,
// ld k) in scratch; Sbar = S - dE sum G_d S C_d in scratch (ld RA).
static __device__ __noinline__ void w_stream_small(WCtx& x, bool want_sbar) {
    ProfScope ps_(x.prof, PF_SMALL);
    const int k = x.r;
    WSmem* sm = x.sm;
    double* Gd = sm->work;                      // NOPS_W k x k (ld k), from red
    double* Cd = sm->work + NOPS_W * RA * RA;   // NOPS_W k x k
    // k x k temporaries: shared memory in 2D; the 3D Grams leave no room there
    double* T = kThreeD ? x.scr + SO_TMP : sm->work + 2 * NOPS_W * RA * RA;
    double* U = kThreeD ? x.scr + SO_TMP + RA * RA : sm->work + (2 * NOPS_W + 1) * RA * RA;
    double* SC = x.scr + SO_SC;
    double* SG = x.scr + SO_SG;
    double* Sb = x.scr + SO_SBAR;
    load_red(x, 0, NOPS_W * k, k, Gd, k);
    load_red(x, NOPS_W * k * k, NOPS_W * k, k, Cd, k);
    for (int d = 0; d < NOPS_W; ++d) {
        const double* G = Gd + d * k * k;
        const double* C = Cd + d * k * k;
        g_mm(SC + d * k * k, k, sm->S, KA, false, C, k, false, k, k, k);         // S C_d
        g_mm(SG + d * k * k, k, sm->S, KA, true, G, k, true, k, k, k);           // S^T G_d^T
    }
    if (want_sbar) {
        g_copy(Sb, RA, sm->S, KA, k, k);
        for (int d = 0; d < NOPS_W; ++d) {
            g_mm(T, k, sm->S, KA, false, Cd + d * k * k, k, false, k, k, k);     // S C_d
            g_mm(U, k, Gd + d * k * k, k, false, T, k, false, k, k, k);          // G_d S C_d
            for (int e = threadIdx.x; e < k * k; e += NT) Sb[(e / k) * RA + e % k] -= x.P.dE * U[e];
            __syncthreads();
        }
    }
}

// ---- phase C: K and L streaming updates (:1861-1880) written to st.K / st.L,
// and the Grams of [X K] (X side) and [W L] (W side): per side three k x k
// blocks [A^T A | A^T B | B^T B] at offsets 0 and 3k^2.
static __device__ __noinline__ bool w_phase_C(WCtx& x) {
    ProfScope ps_(x.prof, PF_ROWS_STREAM);
    const int k = x.r;
    const double dE = x.P.dE;
    WSmem* sm = x.sm;
    double* acc = sm->work;                      // 6 k^2
    double* ST = sm->work + 6 * k * k;           // NOPS_W k x k stacked (SC or SG)
    double* F = ST + NOPS_W * k * k;             // tr x NOPS_W k stencil / operator outputs
    const int ldF = NOPS_W * k, ldT = 2 * k;
    const int tr = rows_fit(WORKD - (6 + NOPS_W) * k * k, ldF + ldT);
    double* T = F + tr * ldF;                    // tr x 2k feature tile [A | B]
    w_acc_zero(acc, 6 * k * k);
    const GBlock bl[3] = {{0, k, 0, k, 0}, {0, k, k, k, k * k}, {k, k, k, k, 2 * k * k}};
    // X side
    g_copy(ST, k, x.scr + SO_SC, k, NOPS_W * k, k);
    for (int r0 = x.c0; r0 < x.c1; r0 += tr) {
        const int nr = min(tr, x.c1 - r0);
        wload(T, ldT, 0, x.st.X, KA, 0, r0, nr, k);
        w_stencil(x, x.st.X, KA, r0, nr, k, F, ldF, 0);
        __syncthreads();
        // K = X S - dE (L_d X) (S C_d) stacked; the two chains of each entry are
        // formed by the same thread (same micro-tile map in both calls)
        const double* Sm = sm->S;
        row_mm<4>(nr, k, k, T, ldT, [&](int l, int j) { return Sm[l * KA + j]; },
                  [&](int r, int j, double v) { T[r * ldT + k + j] = v; });
        row_mm<4>(nr, NOPS_W * k, k, F, ldF, [&](int l, int j) { return ST[l * k + j]; },
                  [&](int r, int j, double v) { T[r * ldT + k + j] = T[r * ldT + k + j] - dE * v; });
        __syncthreads();
        wstore(x.st.K, RA, 0, T, ldT, k, r0, nr, k);
        gram_blocks(acc, T, ldT, nr, bl, 3);
        __syncthreads();
    }
    // W side
    g_copy(ST, k, x.scr + SO_SG, k, NOPS_W * k, k);
    const GBlock bw[3] = {{0, k, 0, k, 3 * k * k}, {0, k, k, k, 4 * k * k}, {k, k, k, k, 5 * k * k}};
    for (int r0 = x.m0; r0 < x.m1; r0 += tr) {
        const int nr = min(tr, x.m1 - r0);
        wload(T, ldT, 0, x.st.W, KA, 0, r0, nr, k);
        w_spmm(x, x.st.W, KA, r0, nr, k, F, ldF, 0);
        __syncthreads();
        // L = W S^T - dE (A_d W) (S^T G_d^T) stacked
        const double* Sm = sm->S;
        row_mm<4>(nr, k, k, T, ldT, [&](int l, int j) { return Sm[j * KA + l]; },
                  [&](int r, int j, double v) { T[r * ldT + k + j] = v; });
        row_mm<4>(nr, NOPS_W * k, k, F, ldF, [&](int l, int j) { return ST[l * k + j]; },
                  [&](int r, int j, double v) { T[r * ldT + k + j] = T[r * ldT + k + j] - dE * v; });
        __syncthreads();
        wstore(x.st.L, RA, 0, T, ldT, k, r0, nr, k);
        gram_blocks(acc, T, ldT, nr, bw, 3);
        __syncthreads();
    }
    wpublish_chunk(x, acc, 0, 6 * k * k);
    return wreduce(x, 6 * k * k);
}

// ------------------------------------------------------- augmentation -------
// Side s: A = X (cells, ld KA) or W (moments, ld KA); B = K or L (ld RA);
// BP = projected B; C = range-finder output.
struct SideBufs {
    double* A;
    double* B;
    double* BP;
    double* C;
    int r0, r1;
};
__device__ __forceinline__ SideBufs side_bufs(const WCtx& x, int s) {
    if (s == 0) return SideBufs{x.st.X, x.st.K, x.st.KP, x.st.CX, x.c0, x.c1};
    return SideBufs{x.st.W, x.st.L, x.st.LP, x.st.CW, x.m0, x.m1};
}

// Q1 = orth(A) from the reduced Gram blocks at `goff` (s*3k^2): certified
// Cholesky or Jacobi; T1 = P1 (A^T B) with P1 = F1 F1^T (Q1 Q1^T = A P1 A^T on
// the range part; completion vectors of the X side are orthogonal to K).
static __device__ __noinline__ void aug_prepare(WCtx& x, int s, int goff) {
    ProfScope ps_(x.prof, PF_SMALL);
    const int k = x.r;
    WSmem* sm = x.sm;
    SideInfo& si = x.side[s];
    double* G11 = sm->work;
    double* G12 = G11 + RA * RA;
    double* R = G12 + RA * RA;
    double* Ri = R + RA * RA;
    double* T = Ri + RA * RA;
    double* lam = sm->vec;
    load_red(x, goff, k, k, G11, RA);
    load_red(x, goff + k * k, k, k, G12, RA);
    // Frobenius norm of [A B]: traces of A^T A and B^T B
    double tr = 0.0;
    for (int j = 0; j < k; ++j) tr += G11[j * RA + j] + ldcg(x.redp + goff + 2 * k * k + j * k + j);
    si.scale = sqrt(fmax(tr, 0.0));
    const double tol = x.P.rank_tol;
    double rif;
    prof_count(x.prof, PF_CHOL_CALLS, 1ull);
    const double cond = w_chol(G11, RA, R, Ri, RA, k, &rif);
    double* F1 = sside(x, s, SS_F1);
    double* P1 = sside(x, s, SS_P1);
    double* M1 = sside(x, s, SS_M1);
    if (cond < kCertW && 1.0 / rif > 10.0 * tol * si.scale) {
        si.fast1 = 1;
        si.rho1 = k;
        g_copy(F1, RA, Ri, RA, k, k);
        g_copy(M1, RA, R, RA, k, k);
    } else {
        si.fast1 = 0;
        // G11 is still intact (w_chol copies). This Jacobi only separates the
        // scales (V0) for the graded Gram of A V0 that aug_q1_graded reduces;
        // G12 waits in SS_R0 for T1.
        prof_count(x.prof, PF_EIG_SWEEPS, (unsigned long long)w_eig(G11, T, RA, lam, k, x.st.status, raw_gram_floor(k), 1e-8));
        prof_count(x.prof, PF_EIG_CALLS, 1ull);
        g_copy(sside(x, s, SS_V0), RA, T, RA, k, k);
        g_copy(sside(x, s, SS_R0), RA, G12, RA, k, k);
        return;
    }
    __syncthreads();
    // P1 = F1 F1^T (only the first rho1 columns of F1 are nonzero)
    g_mm(P1, RA, F1, RA, false, F1, RA, true, k, si.rho1, k);
    // T1 = P1 G12
    g_mm(sside(x, s, SS_T), RA, P1, RA, false, G12, RA, false, k, k, k);
}

static __device__ __noinline__ void rf_pass(WCtx& x, int s, int mode, int rho, double* acc, int off);

// Rank-revealing Q1 after aug_prepare left V0 (Jacobi of A^T A) on a side:
// the Gram of A V0 is reduced from the rows, so its Jacobi (V2, lambda) resolves
// singular values of A far below sqrt(eps) ||A|| against the cut tol * scale,
// as the SVD of A does; a Gram of A alone carries rounding of eps ||A||^2 there.
// Q1 = A V diag(lambda^-1/2) on the rho1 values above the cut, V = V0 V2;
// M1 = Q1^T A = diag(lambda^1/2) V^T; P1 = F1 F1^T; T1 = P1 G12.
static __device__ __noinline__ bool aug_q1_graded(WCtx& x) {
    const int k = x.r;
    const bool slow[2] = {x.side[0].fast1 == 0, x.side[1].fast1 == 0};
    if (!slow[0] && !slow[1]) return true;
    double* acc = x.sm->work;
    w_acc_zero(acc, 2 * k * k);
    for (int s = 0; s < 2; ++s)
        if (slow[s]) rf_pass(x, s, 3, k, acc, s * k * k);
    wpublish_chunk(x, acc, 0, 2 * k * k);
    if (!wreduce(x, 2 * k * k)) return false;
    ProfScope ps_(x.prof, PF_SMALL);
    for (int s = 0; s < 2; ++s) {
        if (!slow[s]) continue;
        SideInfo& si = x.side[s];
        double* G = x.sm->work;
        double* V2 = G + RA * RA;
        double* V0 = V2 + RA * RA;
        double* lam = x.sm->vec;
        load_red(x, s * k * k, k, k, G, RA);
        prof_count(x.prof, PF_EIG_SWEEPS, (unsigned long long)w_eig(G, V2, RA, lam, k, x.st.status, kGradedFloor));
        prof_count(x.prof, PF_EIG_CALLS, 1ull);
        g_copy(V0, RA, sside(x, s, SS_V0), RA, k, k);
        const double cut = x.P.rank_tol * si.scale;
        int rho = 0;
        for (int j = 0; j < k; ++j) {
            if (sqrt(fmax(lam[j], 0.0)) > cut) rho = j + 1;
            else break;
        }
        si.rho1 = rho;
        g_mm(G, RA, V0, RA, false, V2, RA, false, k, k, k);   // V (G is free after the Jacobi)
        double* F1 = sside(x, s, SS_F1);
        double* M1 = sside(x, s, SS_M1);
        for (int e = threadIdx.x; e < k * k; e += NT) {
            const int i = e / k, j = e - (e / k) * k;
            F1[i * RA + j] = j < rho ? G[i * RA + j] / sqrt(lam[j]) : 0.0;
            M1[i * RA + j] = i < rho ? sqrt(lam[i]) * G[j * RA + i] : 0.0;
        }
        __syncthreads();
        if (s == 1 && rho < k && threadIdx.x == 0) set_status(x.st.status, ST_UNSUPPORTED);
        double* P1 = sside(x, s, SS_P1);
        g_mm(P1, RA, F1, RA, false, F1, RA, true, k, rho, k);
        g_mm(sside(x, s, SS_T), RA, P1, RA, false, sside(x, s, SS_R0), RA, false, k, k, k);
    }
    return true;
}

// BP = B - A T (T = SS_T) for own rows; acc[off..] += A^T BP (second=false) or BP^T BP (second=true)
static __device__ __noinline__ void aug_pass(WCtx& x, int s, bool second, double* acc, int off) {
    ProfScope ps_(x.prof, PF_RF_PASSES);
    const int k = x.r;
    SideBufs sb = side_bufs(x, s);
    double* T = x.sm->work + 2 * RA * RA;        // k x k (ld RA), after the 2k^2 accumulator
    double* F = T + RA * RA;                     // tr x 2k: [A | BP]
    const int ldF = 2 * k;
    const int tr = rows_fit(WORKD - 3 * RA * RA, ldF);
    g_copy(T, RA, sside(x, s, SS_T), RA, k, k);
    const GBlock bl = second ? GBlock{k, k, k, k, off} : GBlock{0, k, k, k, off};
    const double* Bsrc = second ? sb.BP : sb.B;
    for (int r0 = sb.r0; r0 < sb.r1; r0 += tr) {
        const int nr = min(tr, sb.r1 - r0);
        wload(F, ldF, 0, sb.A, KA, 0, r0, nr, k);
        wload(F, ldF, k, Bsrc, RA, 0, r0, nr, k);
        __syncthreads();
        row_mm<4>(nr, k, k, F, ldF, [&](int l, int j) { return T[l * RA + j]; },
                  [&](int r, int j, double v) { F[r * ldF + k + j] -= v; });
        __syncthreads();
        wstore(sb.BP, RA, 0, F, ldF, k, r0, nr, k);
        gram_blocks(acc, F, ldF, nr, &bl, 1);
        __syncthreads();
    }
}

// Both sides: BP = (I - Q1 Q1^T)^2 B in two passes; ends with BP^T BP reduced
// at offsets s*k^2.
static __device__ __noinline__ bool aug_project(WCtx& x) {
    const int k = x.r;
    double* acc = x.sm->work;
    w_acc_zero(acc, 2 * k * k);
    aug_pass(x, 0, false, acc, 0);
    aug_pass(x, 1, false, acc, k * k);
    wpublish_chunk(x, acc, 0, 2 * k * k);
    if (!wreduce(x, 2 * k * k)) return false;
    for (int s = 0; s < 2; ++s) {
        // T2 = P1 (A^T BP)
        double* G = x.sm->work;
        load_red(x, s * k * k, k, k, G, RA);
        g_mm(sside(x, s, SS_T), RA, sside(x, s, SS_P1), RA, false, G, RA, false, k, k, k);
    }
    w_acc_zero(acc, 2 * k * k);
    aug_pass(x, 0, true, acc, 0);
    aug_pass(x, 1, true, acc, k * k);
    wpublish_chunk(x, acc, 0, 2 * k * k);
    return wreduce(x, 2 * k * k);
}

// Row-wise triangular solve t[r,:] <- t[r,:] R^{-1} (R upper, shared, ld RA).
__device__ __forceinline__ void w_rsolve(double* t, int ldt, const double* R, int nr, int k) {
    for (int r = threadIdx.x; r < nr; r += NT) {
        double* row = t + r * ldt;
        for (int j = 0; j < k; ++j) {
            double v = row[j];
            for (int i = 0; i < j; ++i) v = fma(-row[i], R[i * RA + j], v);
            row[j] = v / R[j * RA + j];
        }
    }
}

// C = BP M (mode 0: M = R0 by row solves; mode 1: M = T (k x rho), product) for
// own rows; acc[off..] += C^T C (rho x rho), or (mode 2) (BP V0)^T (BP V0) and
// (mode 3) (A V0)^T (A V0) without storing C.
static __device__ __noinline__ void rf_pass(WCtx& x, int s, int mode, int rho, double* acc, int off) {
    ProfScope ps_(x.prof, PF_RF_PASSES);
    const int k = x.r;
    SideBufs sb = side_bufs(x, s);
    double* M = x.sm->work + 2 * RA * RA;   // k x k (ld RA), after the 2k^2 accumulator
    double* F = M + RA * RA;                // tr x 2k: [BP | out]
    const int ldF = 2 * k;
    const int tr = rows_fit(WORKD - 3 * RA * RA, ldF);
    g_copy(M, RA, sside(x, s, mode == 0 ? SS_R0 : (mode == 1 ? SS_T : SS_V0)), RA, k, mode == 1 ? rho : k);
    const int w = (mode == 1) ? rho : k;
    const GBlock bl{k, w, k, w, off};
    for (int r0 = sb.r0; r0 < sb.r1; r0 += tr) {
        const int nr = min(tr, sb.r1 - r0);
        if (mode == 3) wload(F, ldF, 0, sb.A, KA, 0, r0, nr, k);
        else wload(F, ldF, 0, sb.BP, RA, 0, r0, nr, k);
        __syncthreads();
        if (mode == 0) {
            for (int e = threadIdx.x; e < nr * k; e += NT) F[(e / k) * ldF + k + e % k] = F[(e / k) * ldF + e % k];
            __syncthreads();
            w_rsolve(F + k, ldF, M, nr, k);
        } else {
            row_mm<4>(nr, k, w, F, ldF, [&](int l, int j) { return M[l * RA + j]; },
                      [&](int r, int j, double v) { F[r * ldF + k + j] = v; });
        }
        __syncthreads();
        if (mode < 2) wstore(sb.C, RA, 0, F, ldF, k, r0, nr, w);
        gram_blocks(acc, F, ldF, nr, &bl, 1);
        __syncthreads();
    }
}

// Final step of a range finder: CholQR of C from its reduced Gram (rho x rho at
// red offset `off`) -> SS_RI.
static __device__ __noinline__ void rf_finish(WCtx& x, int s, int off) {
    const int rho = x.side[s].rho2;
    if (rho <= 0) return;
    double* G = x.sm->work;
    double* R = G + RA * RA;
    double* Ri = R + RA * RA;
    load_red(x, off, rho, rho, G, RA);
    double rif;
    prof_count(x.prof, PF_CHOL_CALLS, 1ull);
    const double cond = w_chol(G, RA, R, Ri, RA, rho, &rif);
    if (!(cond < INFINITY) && threadIdx.x == 0) {
        if (atomicCAS(x.st.status, 0, ST_CHOL_BREAKDOWN) == 0) {
            x.st.diag[0] = 10 + s;
            x.st.diag[2] = rho;
            x.st.diag[7] = x.cur_n;
        }
    }
    g_copy(sside(x, s, SS_RI), RA, Ri, RA, rho, rho);
}

// Slow path after the Gram of BP V0 was reduced at `off`: Jacobi -> V2, nu;
// rho = #{nu_j > cut}; SS_T = V0 V2[:, :rho] diag(1/nu).
static __device__ __noinline__ void rf_slow_rank(WCtx& x, int s, int off, bool plain) {
    const int k = x.r;
    SideInfo& si = x.side[s];
    double* G = x.sm->work;
    double* V2 = G + RA * RA;
    double* V0 = V2 + RA * RA;
    double* nu = x.sm->vec;
    load_red(x, off, k, k, G, RA);
    prof_count(x.prof, PF_EIG_SWEEPS, (unsigned long long)w_eig(G, V2, RA, nu, k, x.st.status, kGradedFloor));
    prof_count(x.prof, PF_EIG_CALLS, 1ull);
    g_copy(V0, RA, sside(x, s, SS_V0), RA, k, k);
    const double nu0 = sqrt(fmax(nu[0], 0.0));
    const double cut = x.P.rank_tol * (plain ? nu0 : si.scale);
    int rho = 0;
    if (!(plain && nu0 <= 0.0))
        for (int j = 0; j < k; ++j) {
            if (sqrt(fmax(nu[j], 0.0)) > cut) rho = j + 1;
            else break;
        }
    si.rho2 = rho;
    double* T = sside(x, s, SS_T);
    for (int e = threadIdx.x; e < k * rho; e += NT) {
        const int i = e / rho, j = e - (e / rho) * rho;
        double a = 0.0;
        for (int l = 0; l < k; ++l) a = fma(V0[i * RA + l], V2[l * RA + j], a);
        T[i * RA + j] = a / sqrt(nu[j]);
    }
    __syncthreads();
}

// Range finders of BP on the sides with do_side[s], after BP^T BP was reduced
// at offsets s*k^2. `plain[s]`: the rank cut is relative to the largest
// singular value of BP itself (orth), else to side[s].scale (augmentation).
//  certified path: Cholesky of BP^T BP with ||R||_F ||R^-1||_F < 1e5 (and, for
//    augmentation, sigma_min > 10 tol scale): C = BP R0^{-1} by row solves;
//  rank-revealing path: Jacobi of BP^T BP -> V0; Gram of BP V0 -> Jacobi ->
//    V2, nu; C = BP V0 V2_J / nu_J for nu_j above the cut.
// On return side[s].rho2 is set and SS_RI holds R^{-1} of the CholQR of C, so
// that the basis is C R^{-1} (rho2 columns).
static __device__ __noinline__ bool range_find(WCtx& x, const bool do_side[2], const bool plain[2]) {
    ProfScope ps_(x.prof, PF_CHOL);
    const int k = x.r;
    WSmem* sm = x.sm;
    const double tol = x.P.rank_tol;
    bool slow[2] = {false, false};
    for (int s = 0; s < 2; ++s) {
        if (!do_side[s]) continue;
        SideInfo& si = x.side[s];
        double* G = sm->work;
        double* R = G + RA * RA;
        double* Ri = R + RA * RA;
        double* V = Ri + RA * RA;
        load_red(x, s * k * k, k, k, G, RA);
        double rif;
        prof_count(x.prof, PF_CHOL_CALLS, 1ull);
    const double cond = w_chol(G, RA, R, Ri, RA, k, &rif);
        const bool ok = cond < kCertW && (plain[s] || 1.0 / rif > 10.0 * tol * si.scale);
        prof_count(x.prof, ok ? PF_RF_FAST : PF_RF_SLOW, 1ull);
        if (ok) {
            si.fast2 = 1;
            si.rho2 = k;
            g_copy(sside(x, s, SS_R0), RA, R, RA, k, k);
        } else {
            si.fast2 = 0;
            slow[s] = true;
            // first Jacobi of the rank-revealing path: it only separates scales for
            // the graded Gram of BP V0, whose Jacobi (tolerance 1e-15) fixes nu
            prof_count(x.prof, PF_EIG_SWEEPS, (unsigned long long)w_eig(G, V, RA, sm->vec, k, x.st.status, raw_gram_floor(k), 1e-8));
            prof_count(x.prof, PF_EIG_CALLS, 1ull);
            g_copy(sside(x, s, SS_V0), RA, V, RA, k, k);
        }
    }
    double* acc = sm->work;
    // pass 1: certified -> C = BP R0^{-1} and C^T C ; rank-revealing -> Gram of BP V0
    w_acc_zero(acc, 2 * k * k);
    for (int s = 0; s < 2; ++s)
        if (do_side[s]) rf_pass(x, s, x.side[s].fast2 ? 0 : 2, k, acc, s * k * k);
    wpublish_chunk(x, acc, 0, 2 * k * k);
    if (!wreduce(x, 2 * k * k)) return false;
    for (int s = 0; s < 2; ++s) {
        if (!do_side[s]) continue;
        if (!slow[s]) rf_finish(x, s, s * k * k);
        else rf_slow_rank(x, s, s * k * k, plain[s]);
    }
    if (slow[0] || slow[1]) {
        w_acc_zero(acc, 2 * k * k);
        for (int s = 0; s < 2; ++s)
            if (slow[s] && x.side[s].rho2 > 0) rf_pass(x, s, 1, x.side[s].rho2, acc, s * k * k);
        wpublish_chunk(x, acc, 0, 2 * k * k);
        if (!wreduce(x, 2 * k * k)) return false;
        for (int s = 0; s < 2; ++s)
            if (slow[s]) rf_finish(x, s, s * k * k);
    }
    __syncthreads();
    return true;
}

// W-side completion in the small space: candidates m = 0, 1, ... accepted when
// 1 - ||P[m,:]||^2 > 1/4 (a second scan, if the first runs out: > 1e-6)
// with P = [Q1 (nq1 cols, rows W[m,:] F1), Q2 (rows
// C[m,:] RI), v_1 .. v_a]; stores per accepted vector its candidate, norm and
// coefficients in SS_WC (row a, length nq1 + rho2 + a).
static __device__ __noinline__ void w_complete_side(WCtx& x, int nq1, int rho2, int need) {
    ProfScope ps_(x.prof, PF_COMPLETE);
    WSmem* sm = x.sm;
    double* wc = sside(x, 1, SS_WC);
    const double* F1 = sside(x, 1, SS_F1);
    const double* Ri = sside(x, 1, SS_RI);
    double* wrow = sm->vec;             // W[c,:] (k) then C[c,:] (rho2)
    double* prow = sm->vec + 2 * KA;    // P[c,:] (nq1 + rho2 + a <= 3 RA)
    __shared__ int s_acc, s_next, s_phase;
    const int k = x.r;
    if (threadIdx.x == 0) {
        s_acc = 0;
        s_next = 0;
        s_phase = 0;
    }
    __syncthreads();
    while (true) {
        const int acc = s_acc, it = s_next;
        if (acc >= need) break;
        if (it >= x.P.nwcomp) {
            // second scan from the first candidate with the relaxed threshold
            // (the basis nearly fills the moment space)
            if (s_phase == 0) {
                __syncthreads();
                if (threadIdx.x == 0) {
                    s_phase = 1;
                    s_next = 0;
                }
                __syncthreads();
                continue;
            }
            if (threadIdx.x == 0 && atomicCAS(x.st.status, 0, ST_COMPLETION) == 0) {
                x.st.diag[0] = 32;   // W side: candidate moments exhausted
                x.st.diag[2] = need;
                x.st.diag[3] = acc;
                x.st.diag[7] = x.cur_n;
            }
            __syncthreads();
            break;
        }
        const int c = x.P.wcomp[it];
        if (nq1 > 0)
            for (int j = threadIdx.x; j < k; j += NT) wrow[j] = ldcg(x.st.W + (size_t)c * KA + j);
        for (int j = threadIdx.x; j < rho2; j += NT) wrow[KA + j] = ldcg(x.st.CW + (size_t)c * RA + j);
        __syncthreads();
        for (int j = threadIdx.x; j < nq1 + rho2; j += NT) {
            double s = 0.0;
            if (j < nq1)
                for (int l = 0; l < k; ++l) s = fma(wrow[l], F1[l * RA + j], s);
            else
                for (int l = 0; l <= j - nq1; ++l) s = fma(wrow[KA + l], Ri[l * RA + (j - nq1)], s);
            prow[j] = s;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const int nb = nq1 + rho2;
            for (int a = 0; a < acc; ++a) {
                const double* w = wc + a * WCS;
                double v = (c == sm->wcand[a]) ? 1.0 : 0.0;
                for (int j = 0; j < nb + a; ++j) v -= prow[j] * w[j];
                prow[nb + a] = v / sm->wnrm[a];
            }
            double ss = 0.0;
            for (int j = 0; j < nb + acc; ++j) ss += prow[j] * prow[j];
            const double nv2 = 1.0 - ss;
            if (nv2 > (s_phase == 0 ? 0.25 : 1e-6)) {
                for (int j = 0; j < nb + acc; ++j) wc[acc * WCS + j] = prow[j];
                sm->wcand[acc] = c;
                sm->wnrm[acc] = sqrt(nv2);
                s_acc = acc + 1;
            }
            s_next = it + 1;
        }
        __syncthreads();
    }
}

// Materialise the new directions: A[:, k:2k] = [C RI | completion]; with
// `with_q1` also A[:, :k] = Q1 = [A F1 | completion] (BUG). Row tile t holds
// [old A (k) | Q1 (k) | X~ (k) | B (k)] per row (ld 4RA). With `acc`, the
// parallel integrator's S blocks are accumulated on the way: X side
// acc[0..k^2) += X~^T K, W side acc[k^2..2k^2) += L^T W~.
static __device__ __noinline__ void materialize_side(WCtx& x, int s, bool with_q1, double* acc) {
    ProfScope ps_(x.prof, PF_RF_PASSES);
    const int k = x.r;
    WSmem* sm = x.sm;
    SideBufs sb = side_bufs(x, s);
    const SideInfo& si = x.side[s];
    const int LT = 4 * k;                    // tile leading dimension
    const int LC = k + (k & 1);              // C-row leading dimension (even: 16-byte rows)
    double* F1 = sm->work + 2 * RA * RA;     // k x k (after the 2k^2 accumulator)
    double* Ri = F1 + RA * RA;               // rho2 x rho2
    const int tr = rows_fit(WORKD - 4 * RA * RA, LT + LC);
    double* t = Ri + RA * RA;                // tr x 4k
    double* cb = t + tr * LT;                // tr x LC (C rows)
    const GBlock blk = s == 0 ? GBlock{2 * k, k, 3 * k, k, 0} : GBlock{3 * k, k, 2 * k, k, k * k};
    g_copy(F1, RA, sside(x, s, SS_F1), RA, k, k);
    if (si.rho2 > 0) g_copy(Ri, RA, sside(x, s, SS_RI), RA, si.rho2, si.rho2);
    const double* wc = sside(x, 1, SS_WC);
    const int rho1 = si.rho1, rho2 = si.rho2;
    for (int r0 = sb.r0; r0 < sb.r1; r0 += tr) {
        const int nr = min(tr, sb.r1 - r0);
        wload(t, LT, 0, sb.A, KA, 0, r0, nr, k);
        if (acc) wload(t, LT, 3 * k, sb.B, RA, 0, r0, nr, k);
        if (rho2 > 0) wload(cb, LC, 0, sb.C, RA, 0, r0, nr, rho2);
        __syncthreads();
        // Q1 columns: range part A F1, then completion (X side only: the W side has rho1 == k)
        row_mm<4>(nr, k, rho1, t, LT, [&](int l, int j) { return F1[l * RA + j]; },
                  [&](int r, int j, double v) { t[r * LT + k + j] = v; });
        // X~ range part C RI (RI upper triangular: the terms l > j add exact zeros)
        row_mm<4>(nr, rho2, rho2, cb, LC, [&](int l, int j) { return l <= j ? Ri[l * RA + j] : 0.0; },
                  [&](int r, int j, double v) { t[r * LT + 2 * k + j] = v; });
        for (int e = threadIdx.x; e < nr * k; e += NT) {
            const int r = e / k, j = e - (e / k) * k;
            const int row = r0 + r;
            if (j >= rho1) {
                const int ci = j - rho1;
                t[r * LT + k + j] = (s == 0 && ci < x.P.nxcomp && row == x.P.xcomp[ci]) ? 1.0 : 0.0;
            }
            if (j >= rho2) {
                double xt = 0.0;
                if (s == 0) {
                    const int ci = si.cand0 + (j - rho2);
                    xt = (ci < x.P.nxcomp && row == x.P.xcomp[ci]) ? 1.0 : 0.0;
                }
                t[r * LT + 2 * k + j] = xt;
            }
        }
        __syncthreads();
        if (s == 1 && si.need2 > 0) {
            // completion vectors v_a[m] = (delta_{m,c_a} - P[m,:] w_a) / nrm_a, P = [Q1 | Q2 | v_1..]
            for (int r = threadIdx.x; r < nr; r += NT) {
                const int m = r0 + r;
                double* q1r = t + r * LT + k;           // Q1 row (k)
                double* q2r = t + r * LT + 2 * k;       // [Q2 (rho2) | v_1 ..]
                for (int a = 0; a < si.need2; ++a) {
                    const double* w = wc + a * WCS;
                    double v = (m == sm->wcand[a]) ? 1.0 : 0.0;
                    for (int j = 0; j < k; ++j) v -= q1r[j] * w[j];
                    for (int j = 0; j < rho2 + a; ++j) v -= q2r[j] * w[k + j];
                    q2r[rho2 + a] = v / sm->wnrm[a];
                }
            }
            __syncthreads();
        }
        if (with_q1) wstore(sb.A, KA, 0, t, LT, k, r0, nr, k);
        wstore(sb.A, KA, k, t, LT, 2 * k, r0, nr, k);
        if (acc) gram_blocks(acc, t, LT, nr, &blk, 1);
        __syncthreads();
    }
}

// Whole augmentation of both sides after the [A B] Grams were reduced at
// offsets 0 (X) and 3k^2 (W). Leaves the new directions in columns [k, 2k)
// (and Q1 in [0, k) with with_q1), without a closing barrier.
static __device__ __noinline__ bool augment(WCtx& x, bool with_q1, bool par_blocks) {
    const int k = x.r;
    if (2 * k > KA) {
        if (threadIdx.x == 0) set_status(x.st.status, ST_LIMIT);
        return false;
    }
    aug_prepare(x, 0, 0);
    aug_prepare(x, 1, 3 * k * k);
    if (!aug_q1_graded(x)) return false;
    if (!aug_project(x)) return false;
    const bool all[2] = {true, true};
    const bool aug[2] = {false, false};
    if (!range_find(x, all, aug)) return false;
    SideInfo& sx = x.side[0];
    sx.need2 = k - sx.rho2;
    sx.cand0 = k - sx.rho1;
    if (sx.cand0 + sx.need2 > x.P.nxcomp && threadIdx.x == 0 && atomicCAS(x.st.status, 0, ST_COMPLETION) == 0) {
        x.st.diag[0] = 31;   // X side: more completion vectors than candidate cells
        x.st.diag[2] = sx.cand0 + sx.need2;
        x.st.diag[3] = x.P.nxcomp;
        x.st.diag[7] = x.cur_n;
    }
    SideInfo& sw = x.side[1];
    sw.need2 = k - sw.rho2;
    sw.cand0 = 0;
    if (sw.need2 > 0) {
        w_complete_side(x, k, sw.rho2, sw.need2);
        // the completion read W[c, :k] of other CTAs' rows; Q1 overwrites those columns
        if (with_q1 && !wsync(x)) return false;
    }
    double* acc = par_blocks ? x.sm->work : nullptr;
    if (acc) w_acc_zero(acc, 2 * k * k);
    materialize_side(x, 0, with_q1, acc);
    materialize_side(x, 1, with_q1, acc);
    if (par_blocks) {
        // red [X~^T K (k^2) | L^T W~ (k^2)]
        wpublish_chunk(x, acc, 0, 2 * k * k);
        return wreduce(x, 2 * k * k);
    }
    return true;
}

// --------------------------------------------------------------- truncate ---
// truncate! of the m x m matrix given in transposed storage in work[0..):
// SVD, l1 tail rank (clamped to [2, settings.r]), deterministic completion of
// the kept null directions. Leaves U^T (rows perm[j]) at work[0], V^T at
// work[KA*LDS], sig/perm in shared memory; returns the kept rank (-1 if the
// team aborted).
static __device__ __noinline__ int w_truncate_svd(WCtx& x, int m) {
    ProfScope ps_(x.prof, PF_JACOBI);
    WSmem* sm = x.sm;
    double* At = sm->work;
    double* Vt = sm->work + KA * LDS;
    // keep the SVD input (transposed) for diagnostics
    g_copy(x.scr + SO_DBG, KA, At, LDS, m, m);
    const int sw = w_svd(At, Vt, LDS, m, sm->sig, sm->perm);
    if (x.prof && threadIdx.x == 0) {
        x.prof[PF_SVD_SWEEPS] += (unsigned long long)(sw > 0 ? sw : 60);
        x.prof[PF_SVD_CALLS] += 1ull;
    }
    if (sw < 0 && threadIdx.x == 0 && atomicCAS(x.st.status, 0, ST_SVD) == 0) {
        x.st.diag[0] = 20;
        x.st.diag[2] = m;
        x.st.diag[7] = x.cur_n;
    }
    // tol = theta ||D||_2^thetaIndex ; first j with |sum_{i >= j} D_i| < tol
    double nrm = 0.0;
    for (int j = 0; j < m; ++j) nrm = fma(sm->sig[j], sm->sig[j], nrm);
    const double tol = x.P.theta * pow(sqrt(nrm), x.P.theta_index);
    const int half = m / 2;
    int kk = half;
    for (int j = 1; j <= 2 * half; ++j) {
        double tail = 0.0;
        for (int i = j - 1; i < 2 * half; ++i) tail += sm->sig[i];
        if (fabs(tail) < tol) {
            kk = j;
            break;
        }
    }
    kk = min(kk, x.P.r);
    kk = max(kk, 2);
    kk = min(kk, m);
    const int rho = w_svd_complete(At, Vt, LDS, m, sm->sig, sm->perm, kk, kNullSvd, x.st.status, x.st.X, x.P.n,
                                   x.st.W, x.P.N, KA);
    if (threadIdx.x == 0 && *(volatile int*)x.st.status == ST_COMPLETION && x.st.diag[0] == 0.0) {
        x.st.diag[0] = 33;   // truncation: null directions of S not completed
        x.st.diag[2] = m;
        x.st.diag[3] = rho;
        x.st.diag[7] = x.cur_n;
    }
    // the completion read rows of X and W owned by other CTAs, which the
    // truncation then rewrites in place
    if (rho < kk && !wsync(x)) return -1;
    return kk;
}

// X <- X[:, :m] U[:, :kk], W <- W[:, :m] V[:, :kk] for own rows; S = diag(sig[:kk]).
// With dose2: dose += 1/2 dE (X_new S_new W_new[0,:]^T + psi MRed[0]) S[sidx] / rho.
// `w0` (m entries, any memory): row 0 of W before the update, needed for the
// dose because the CTA owning moment 0 overwrites it without a team barrier.
static __device__ __noinline__ void w_truncate_apply(WCtx& x, int m, int kk, int dose_sidx, const double* w0) {
    ProfScope ps_(x.prof, PF_ROWS_SCATTER);
    WSmem* sm = x.sm;
    const double* Ut = sm->work;
    const double* Vt = sm->work + KA * LDS;
    const int ldt = m;                      // m = 2k, even: 16-byte rows
    const int tr = rows_fit(WORKD - 2 * KA * LDS, 2 * ldt);
    double* t = sm->work + 2 * KA * LDS;    // tr x m
    double* o = t + tr * ldt;               // tr x m
    double* v = sm->vec;                    // diag(sig) W_new[0,:]^T
    if (dose_sidx >= 0) {
        for (int j = threadIdx.x; j < kk; j += NT) {
            double a = 0.0;
            for (int i = 0; i < m; ++i) a = fma(w0[i], Vt[sm->perm[j] * LDS + i], a);
            v[j] = sm->sig[j] * a;
        }
        __syncthreads();
    }
    for (int side = 0; side < 2; ++side) {
        double* A = side == 0 ? x.st.X : x.st.W;
        const double* B = side == 0 ? Ut : Vt;
        const int r0b = side == 0 ? x.c0 : x.m0, r1b = side == 0 ? x.c1 : x.m1;
        for (int r0 = r0b; r0 < r1b; r0 += tr) {
            const int nr = min(tr, r1b - r0);
            wload(t, ldt, 0, A, KA, 0, r0, nr, m);
            __syncthreads();
            const int* perm = sm->perm;
            row_mm<4>(nr, m, kk, t, ldt, [&](int l, int j) { return B[perm[j] * LDS + l]; },
                      [&](int r, int j, double v) { o[r * ldt + j] = v; });
            __syncthreads();
            wstore(A, KA, 0, o, ldt, 0, r0, nr, kk);
            __syncthreads();
        }
    }
    // S = diag(sig[:kk])
    for (int e = threadIdx.x; e < KA * KA; e += NT) sm->S[e] = 0.0;
    __syncthreads();
    for (int j = threadIdx.x; j < kk; j += NT) sm->S[j * KA + j] = sm->sig[j];
    __syncthreads();
    if (dose_sidx >= 0) w_dose(x, dose_sidx, v, kk, false);
    __syncthreads();
    x.r = kk;
}

// ------------------------------------------------------ scattering passes ---
// Out-scattering L = W S^T / (1 + dE D) (own moments, :1885-1890), written to
// L and LP, with L^T L at red offset k^2 (the range finder's side-1 slot); X
// side: X^T psi of the X before zeroing (:1904) at offset 2k^2.
static __device__ __noinline__ bool w_outscatter_pass(WCtx& x, const double* sig) {
    ProfScope ps_(x.prof, PF_ROWS_SCATTER);
    const int k = x.r;
    const DevProblem& P = x.P;
    WSmem* sm = x.sm;
    double* acc = sm->work;
    int ldt = max(2 * k, k + P.q);
    ldt += ldt & 1;                             // even: 16-byte rows
    const int tstart = 2 * RA * RA + RA * QW;   // after the largest accumulator
    const int tr = rows_fit(WORKD - tstart, ldt);
    double* t = sm->work + tstart;   // tr x ldt: W side [W | L], X side [X | psi]
    w_acc_zero(acc, 2 * k * k + k * P.q);
    const GBlock bl{k, k, k, k, k * k};
    for (int r0 = x.m0; r0 < x.m1; r0 += tr) {
        const int nr = min(tr, x.m1 - r0);
        wload(t, ldt, 0, x.st.W, KA, 0, r0, nr, k);
        __syncthreads();
        const double* Sm = sm->S;
        row_mm<4>(nr, k, k, t, ldt, [&](int l, int j) { return Sm[j * KA + l]; }, [&](int r, int j, double v) {
            const double D = sig[0] - sig[P.lof[r0 + r]];
            t[r * ldt + k + j] = v / (1.0 + P.dE * D);
        });
        __syncthreads();
        wstore(x.st.L, RA, 0, t, ldt, k, r0, nr, k);
        wstore(x.st.LP, RA, 0, t, ldt, k, r0, nr, k);
        gram_blocks(acc, t, ldt, nr, &bl, 1);
        __syncthreads();
    }
    const GBlock bx{0, k, k, P.q, 2 * k * k};
    for (int r0 = x.c0; r0 < x.c1; r0 += tr) {
        const int nr = min(tr, x.c1 - r0);
        wload(t, ldt, 0, x.st.X, KA, 0, r0, nr, k);
        wload(t, ldt, k, x.psi_in, QW, 0, r0, nr, P.q);
        __syncthreads();
        gram_blocks(acc, t, ldt, nr, &bx, 1);
        __syncthreads();
    }
    wpublish_chunk(x, acc, 0, 2 * k * k + k * P.q);
    if (!wreduce(x, 2 * k * k + k * P.q)) return false;
    load_red(x, 2 * k * k, k, P.q, x.scr + SO_XTPSI, QW);
    return true;
}

// W = [C RI | completion] (own moments); acc = [L^T W (k^2) | MRed^T diag(Dvec) W (q k)]
static __device__ __noinline__ bool w_outscatter_basis(WCtx& x, const double* sig) {
    ProfScope ps_(x.prof, PF_ROWS_SCATTER);
    const int k = x.r;
    const DevProblem& P = x.P;
    WSmem* sm = x.sm;
    const SideInfo& si = x.side[1];
    double* acc = sm->work;
    double* Ri = sm->work + RA * RA + RA * QW;   // after the largest accumulator
    double* t = Ri + RA * RA;           // tr x (3 RA + QW): [C | W_new | L | MRed D]
    const int ldt = 3 * RA + QW;
    const int tr = rows_fit(WORKD - (2 * RA * RA + RA * QW), ldt);
    const int rho = si.rho2;
    if (rho > 0) g_copy(Ri, RA, sside(x, 1, SS_RI), RA, rho, rho);
    w_acc_zero(acc, k * k + P.q * k);
    const double* wc = sside(x, 1, SS_WC);
    const GBlock bl[2] = {{2 * RA, k, RA, k, 0}, {3 * RA, P.q, RA, k, k * k}};
    for (int r0 = x.m0; r0 < x.m1; r0 += tr) {
        const int nr = min(tr, x.m1 - r0);
        if (rho > 0) wload(t, ldt, 0, x.st.CW, RA, 0, r0, nr, rho);
        wload(t, ldt, 2 * RA, x.st.L, RA, 0, r0, nr, k);
        for (int e = threadIdx.x; e < nr * P.q; e += NT) {
            const int r = e / P.q, kq = e - (e / P.q) * P.q;
            const int m = r0 + r;
            t[r * ldt + 3 * RA + kq] = P.mred[(size_t)m * P.q + kq] * sig[P.lof[m]];
        }
        __syncthreads();
        row_mm<4>(nr, rho, rho, t, ldt, [&](int l, int j) { return l <= j ? Ri[l * RA + j] : 0.0; },
                  [&](int r, int j, double v) { t[r * ldt + RA + j] = v; });
        __syncthreads();
        if (k > rho) {
            for (int r = threadIdx.x; r < nr; r += NT) {
                const int m = r0 + r;
                double* row = t + r * ldt + RA;
                for (int a = 0; a < k - rho; ++a) {
                    const double* w = wc + a * WCS;
                    double v = (m == sm->wcand[a]) ? 1.0 : 0.0;
                    for (int j = 0; j < rho + a; ++j) v -= row[j] * w[j];
                    row[rho + a] = v / sm->wnrm[a];
                }
            }
            __syncthreads();
        }
        wstore(x.st.W, KA, 0, t, ldt, RA, r0, nr, k);
        gram_blocks(acc, t, ldt, nr, bl, 2);
        __syncthreads();
    }
    wpublish_chunk(x, acc, 0, k * k + P.q * k);
    if (!wreduce(x, k * k + P.q * k)) return false;
    // S = L^T W ; MtDW (q x k)
    for (int e = threadIdx.x; e < KA * KA; e += NT) sm->S[e] = 0.0;
    __syncthreads();
    load_red(x, 0, k, k, sm->S, KA);
    load_red(x, k * k, P.q, k, x.scr + SO_MTDW, KA);
    return true;
}

// out-scattering (:1885-1890 / :2229-2234): L, W = orth(L) (plain range
// finder on the angular side), S = L^T W and MtDW; X^T psi of the pre-zeroing X.
static __device__ __noinline__ bool w_outscatter(WCtx& x, const double* sig) {
    const int k = x.r;
    if (!w_outscatter_pass(x, sig)) return false;
    const bool only_w[2] = {false, true};
    const bool plain[2] = {false, true};
    if (!range_find(x, only_w, plain)) return false;
    const int rho = x.side[1].rho2;
    if (k > rho) w_complete_side(x, 0, rho, k - rho);
    return w_outscatter_basis(x, sig);
}

// In-scattering K and L (:1905-1918): K = X S + dE psi MtDW (K[bnd] = 0),
// L = W S^T + dE Dvec (MRed Xtpsi^T); Grams of [X K] and [W L]. With sbar:
// Sbar = S + dE Xtpsi MtDW in scratch; with dose also the second dose
// half-step with (X, Sbar, W) before truncation (parallel integrator, :1943;
// the parallel-rejection loop takes its dose after the truncation, :2683).
static __device__ __noinline__ bool w_inscatter_KL(WCtx& x, const double* sig, bool sbar, bool dose, int dose_sidx) {
    const bool sbar_dose = sbar && dose;
    ProfScope ps_(x.prof, PF_ROWS_SCATTER);
    const int k = x.r;
    const DevProblem& P = x.P;
    WSmem* sm = x.sm;
    const double dE = P.dE;
    double* acc = sm->work;                   // 6 k^2
    double* Mt = sm->work + 6 * RA * RA;      // q x k MtDW (ld KA)
    double* Xp = Mt + QW * KA;                // k x q Xtpsi (ld QW)
    double* t = Xp + KA * QW;                 // tr x ldt: X side [X | K | psi], W side [W | L]
    const int ldt = 2 * k + P.q + ((2 * k + P.q) & 1);
    const int tr = rows_fit(WORKD - (6 * RA * RA + 2 * KA * QW), ldt);
    g_copy(Mt, KA, x.scr + SO_MTDW, KA, P.q, k);
    g_copy(Xp, QW, x.scr + SO_XTPSI, QW, k, P.q);
    double* Sb = x.scr + SO_SBAR;
    if (sbar) {
        // Sbar = S + dE Xtpsi MtDW
        for (int e = threadIdx.x; e < k * k; e += NT) {
            const int i = e / k, j = e - (e / k) * k;
            double a = 0.0;
            for (int l = 0; l < P.q; ++l) a = fma(Xp[i * QW + l], Mt[l * KA + j], a);
            Sb[i * RA + j] = sm->S[i * KA + j] + dE * a;
        }
        __syncthreads();
    }
    if (sbar_dose) {
        // v = Sbar W[0,:]^T
        double* w0 = sm->vec + KA;
        for (int j = threadIdx.x; j < k; j += NT) w0[j] = ldcg(x.st.W + j);
        __syncthreads();
        for (int i = threadIdx.x; i < k; i += NT) {
            double a = 0.0;
            for (int j = 0; j < k; ++j) a = fma(Sb[i * RA + j], w0[j], a);
            sm->vec[i] = a;
        }
        __syncthreads();
    }
    w_acc_zero(acc, 6 * k * k);
    const GBlock bl[3] = {{0, k, 0, k, 0}, {0, k, k, k, k * k}, {k, k, k, k, 2 * k * k}};
    for (int r0 = x.c0; r0 < x.c1; r0 += tr) {
        const int nr = min(tr, x.c1 - r0);
        wload(t, ldt, 0, x.st.X, KA, 0, r0, nr, k);
        wload(t, ldt, 2 * k, x.psi_in, QW, 0, r0, nr, P.q);
        __syncthreads();
        // K = X S + dE psi MtDW (zero on boundary rows), two chains per entry
        const double* Sm = sm->S;
        row_mm<4>(nr, k, k, t, ldt, [&](int l, int j) { return Sm[l * KA + j]; },
                  [&](int r, int j, double v) { t[r * ldt + k + j] = is_bnd_w(P, r0 + r) ? 0.0 : v; });
        row_mm<4>(nr, P.q, k, t + 2 * k, ldt, [&](int l, int j) { return Mt[l * KA + j]; },
                  [&](int r, int j, double v) {
                      if (!is_bnd_w(P, r0 + r)) t[r * ldt + k + j] += dE * v;
                  });
        __syncthreads();
        wstore(x.st.K, RA, 0, t, ldt, k, r0, nr, k);
        gram_blocks(acc, t, ldt, nr, bl, 3);
        __syncthreads();
    }
    if (sbar_dose) w_dose(x, dose_sidx, sm->vec, k, false);
    const GBlock bw[3] = {{0, k, 0, k, 3 * k * k}, {0, k, k, k, 4 * k * k}, {k, k, k, k, 5 * k * k}};
    for (int r0 = x.m0; r0 < x.m1; r0 += tr) {
        const int nr = min(tr, x.m1 - r0);
        wload(t, ldt, 0, x.st.W, KA, 0, r0, nr, k);
        __syncthreads();
        for (int e = threadIdx.x; e < nr * k; e += NT) {
            const int r = e / k, j = e - (e / k) * k;
            const int m = r0 + r;
            double s = 0.0;
            for (int l = 0; l < k; ++l) s = fma(t[r * ldt + l], sm->S[j * KA + l], s);
            double a = 0.0;   // (MRed Xtpsi^T)[m][j]
            for (int kq = 0; kq < P.q; ++kq) a = fma(P.mred[(size_t)m * P.q + kq], Xp[j * QW + kq], a);
            t[r * ldt + k + j] = s + dE * sig[P.lof[m]] * a;
        }
        __syncthreads();
        wstore(x.st.L, RA, 0, t, ldt, k, r0, nr, k);
        gram_blocks(acc, t, ldt, nr, bw, 3);
        __syncthreads();
    }
    wpublish_chunk(x, acc, 0, 6 * k * k);
    return wreduce(x, 6 * k * k);
}

// X[bnd,:] = 0 for own cells (only this CTA reads these rows until the next barrier)
__device__ inline void w_zero_bnd(WCtx& x) {
    const int k = x.r;
    for (int c = x.c0 + threadIdx.x; c < x.c1; c += NT)
        if (is_bnd_w(x.P, c))
            for (int j = 0; j < k; ++j) x.st.X[(size_t)c * KA + j] = 0.0;
    __syncthreads();
}

// Build the parallel integrator's augmented S (:1881-1885) in transposed
// storage at work[0]: S_new = [[Sbar, L^T W~], [X~^T K, 0]]; `par` holds
// [X~^T K | L^T W~] (k x k each) as augment() reduced them.
static __device__ __noinline__ void w_parallel_snew(WCtx& x, const double* par) {
    const int k = x.r, m = 2 * k;
    double* At = x.sm->work;
    const double* Sb = x.scr + SO_SBAR;
    for (int e = threadIdx.x; e < m * m; e += NT) {
        const int i = e / m, j = e - (e / m) * m;   // S_new[i][j] -> At[j][i]
        double v;
        if (i < k && j < k) v = Sb[i * RA + j];
        else if (i < k) v = ldcg(par + k * k + i * k + (j - k));        // (L^T W~)[i][j-k]
        else if (j < k) v = ldcg(par + (i - k) * k + j);                // (X~^T K)[i-k][j]
        else v = 0.0;
        At[j * LDS + i] = v;
    }
    __syncthreads();
}

// ------------------------------------------------ parallel-rejection loop ---
// SolveFirstCollisionSourceDLRParallelRejection (SolverCSD.jl:2376-2742): the
// parallel integrator's augmented step inside the BUG loop's rejections.

// S0 = S entering the energy, kept by every CTA (at n = 2 the out-scattering
// rewrites the aliased S0 in place, :2518, :2611, so it is taken again there).
__device__ inline void w_prej_save_s(WCtx& x) {
    const int k = x.r;
    double* S0 = x.scr + SO_S0;
    for (int e = threadIdx.x; e < k * k; e += NT) S0[(e / k) * RA + e % k] = x.sm->S[(e / k) * KA + e % k];
    __syncthreads();
}
// X0 = X entering the energy with its boundary rows zeroed (the streaming
// K-step, or at n = 2 the in-scattering K-step, zeroes the aliased X0 in
// place, :2532, :2618) and W0 = W, own rows; then S0.
static __device__ __noinline__ void w_prej_save(WCtx& x) {
    const int k = x.r;
    for (int e = threadIdx.x; e < (x.c1 - x.c0) * k; e += NT) {
        const int c = x.c0 + e / k, j = e - (e / k) * k;
        x.st.X0[(size_t)c * RA + j] = is_bnd_w(x.P, c) ? 0.0 : ldcg(x.st.X + (size_t)c * KA + j);
    }
    for (int e = threadIdx.x; e < (x.m1 - x.m0) * k; e += NT) {
        const int mo = x.m0 + e / k, j = e - (e / k) * k;
        x.st.W0[(size_t)mo * RA + j] = ldcg(x.st.W + (size_t)mo * KA + j);
    }
    w_prej_save_s(x);
}

// Streaming rejection test (:2567-2586). With X (boundary rows zeroed) in
// X[:, :k], X~ in X[:, k:2k], W in W[:, :k] and W~ in W[:, k:2k], one pass over
// the team's rows reduces [X~^T L_d X (4 k^2) | W^T A_d W~ (4 k^2) |
// [X X~]^T X (2k x k) | W^T [W W~] (k x 2k)]. Returns
// eta^2 = ||sum_d (X~^T L_d X) S (W^T A_d W~)||_F^2 with the entering S (the
// same value in every CTA), or -1 if the team aborted.
static __device__ __noinline__ double w_prej_stream_eta(WCtx& x) {
    const int k = x.r, m = 2 * k, kk = k * k;
    WSmem* sm = x.sm;
    {
        ProfScope ps_(x.prof, PF_ROWS_STREAM);
        double* acc = sm->work;   // 6 k^2 per side
        double* F = sm->work + 6 * kk;
        const int ldf = m + 4 * k;
        const int tr = rows_fit(WORKD - 6 * kk, ldf);
        GBlock bl[5];
        w_acc_zero(acc, 6 * kk);
        for (int d = 0; d < 4; ++d) bl[d] = GBlock{k, k, m + d * k, k, d * kk};   // X~^T (L_d X)
        bl[4] = GBlock{0, m, 0, k, 4 * kk};                                        // [X X~]^T X
        for (int r0 = x.c0; r0 < x.c1; r0 += tr) {
            const int nr = min(tr, x.c1 - r0);
            wload(F, ldf, 0, x.st.X, KA, 0, r0, nr, m);
            w_stencil(x, x.st.X, KA, r0, nr, k, F, ldf, m);
            __syncthreads();
            gram_blocks(acc, F, ldf, nr, bl, 5);
            __syncthreads();
        }
        wpublish_chunk(x, acc, 0, 4 * kk);
        wpublish_chunk(x, acc + 4 * kk, 8 * kk, 2 * kk);
        __syncthreads();
        w_acc_zero(acc, 6 * kk);
        for (int d = 0; d < 4; ++d) bl[d] = GBlock{0, k, m + d * k, k, d * kk};   // W^T (A_d W~)
        bl[4] = GBlock{0, k, 0, m, 4 * kk};                                        // W^T [W W~]
        for (int r0 = x.m0; r0 < x.m1; r0 += tr) {
            const int nr = min(tr, x.m1 - r0);
            wload(F, ldf, 0, x.st.W, KA, 0, r0, nr, m);
            w_spmm(x, x.st.W + k, KA, r0, nr, k, F, ldf, m);
            __syncthreads();
            gram_blocks(acc, F, ldf, nr, bl, 5);
            __syncthreads();
        }
        wpublish_chunk(x, acc, 4 * kk, 4 * kk);
        wpublish_chunk(x, acc + 4 * kk, 10 * kk, 2 * kk);
    }
    if (!wreduce(x, 12 * kk)) return -1.0;
    ProfScope ps_(x.prof, PF_SMALL);
    double* Gt = sm->work;
    double* Ct = sm->work + 4 * kk;
    double* T = sm->work + 8 * kk;
    double* U = sm->work + 9 * kk;
    double* E = sm->work + 10 * kk;
    load_red(x, 0, 4 * k, k, Gt, k);
    load_red(x, 4 * kk, 4 * k, k, Ct, k);
    g_zero(E, k, k, k);
    for (int d = 0; d < 4; ++d) {
        g_mm(T, k, Gt + d * kk, k, false, sm->S, KA, false, k, k, k);   // Gt_d S
        g_mm(U, k, T, k, false, Ct + d * kk, k, false, k, k, k);        // (Gt_d S) Ct_d
        for (int e = threadIdx.x; e < kk; e += NT) E[e] += U[e];
        __syncthreads();
    }
    double e2 = 0.0;
    for (int e = threadIdx.x; e < kk; e += NT) e2 = fma(E[e], E[e], e2);
    return cta_sum(e2);
}

// Streaming rejection (:2588-2592): S = ([X X~]^T X) S (W^T [W W~]) from the
// blocks w_prej_stream_eta reduced (still in x.redp); X and W already hold
// [X X~] and [W W~].
static __device__ __noinline__ void w_prej_expand_stream(WCtx& x) {
    ProfScope ps_(x.prof, PF_SMALL);
    const int k = x.r, m = 2 * k, kk = k * k;
    WSmem* sm = x.sm;
    double* Mu = sm->work;      // m x k
    double* Nu = Mu + m * k;    // k x m
    double* T = Nu + m * k;     // m x k: Mu S
    double* U = T + m * k;      // m x m
    load_red(x, 8 * kk, m, k, Mu, k);
    load_red(x, 10 * kk, k, m, Nu, m);
    g_mm(T, k, Mu, k, false, sm->S, KA, false, m, k, k);
    g_mm(U, m, T, k, false, Nu, m, false, m, k, m);
    for (int e = threadIdx.x; e < KA * KA; e += NT) {
        const int i = e / KA, j = e - (e / KA) * KA;
        sm->S[e] = (i < m && j < m) ? U[i * m + j] : 0.0;
    }
    __syncthreads();
}

// Scattering rejection test (:2652-2660): reduces X~^T psi (k x q),
// (MRed^T diag(Dvec) W~)^T (q x k) and row 0 of [W W~] (2k entries, written to
// w0 for the dose after the truncation). Returns eta^2 = ||X~^T psi MRed^T D W~||_F^2,
// or -1 if the team aborted.
static __device__ __noinline__ double w_prej_scatter_eta(WCtx& x, const double* sig, double* w0) {
    const int k = x.r, m = 2 * k;
    const DevProblem& P = x.P;
    WSmem* sm = x.sm;
    const int q = P.q;
    {
        ProfScope ps_(x.prof, PF_ROWS_SCATTER);
        double* acc = sm->work;   // 2 k q + m
        const int ldt = k + q + ((k + q) & 1);
        const int tstart = 2 * KA * QW + KA;
        const int tr = rows_fit(WORKD - tstart, ldt);
        double* tt = sm->work + tstart;
        w_acc_zero(acc, 2 * k * q + m);
        const GBlock bx{0, k, k, q, 0};
        for (int r0 = x.c0; r0 < x.c1; r0 += tr) {
            const int nr = min(tr, x.c1 - r0);
            wload(tt, ldt, 0, x.st.X, KA, k, r0, nr, k);
            wload(tt, ldt, k, x.psi_in, QW, 0, r0, nr, q);
            __syncthreads();
            gram_blocks(acc, tt, ldt, nr, &bx, 1);
            __syncthreads();
        }
        const GBlock bw{k, q, 0, k, k * q};
        for (int r0 = x.m0; r0 < x.m1; r0 += tr) {
            const int nr = min(tr, x.m1 - r0);
            wload(tt, ldt, 0, x.st.W, KA, k, r0, nr, k);
            for (int e = threadIdx.x; e < nr * q; e += NT) {
                const int r = e / q, kq = e - (e / q) * q;
                const int mo = r0 + r;
                tt[r * ldt + k + kq] = P.mred[(size_t)mo * q + kq] * sig[P.lof[mo]];
            }
            __syncthreads();
            gram_blocks(acc, tt, ldt, nr, &bw, 1);
            __syncthreads();
        }
        // row 0 of [W W~] travels through the reduction (only its owner adds it)
        if (x.m0 == 0 && x.m1 > 0)
            for (int j = threadIdx.x; j < m; j += NT) acc[2 * k * q + j] = ldcg(x.st.W + j);
        __syncthreads();
        wpublish_chunk(x, acc, 0, 2 * k * q + m);
    }
    if (!wreduce(x, 2 * k * q + m)) return -1.0;
    ProfScope ps_(x.prof, PF_SMALL);
    double* Xp = sm->work;         // k x q
    double* Mt = Xp + k * q;       // q x k
    load_red(x, 0, k, q, Xp, q);
    load_red(x, k * q, q, k, Mt, k);
    load_red(x, 2 * k * q, 1, m, w0, m);
    double e2 = 0.0;
    for (int e = threadIdx.x; e < k * k; e += NT) {
        const int i = e / k, j = e - (e / k) * k;
        double a = 0.0;
        for (int l = 0; l < q; ++l) a = fma(Xp[i * q + l], Mt[l * k + j], a);
        e2 = fma(a, a, e2);
    }
    return cta_sum(e2);
}

// Scattering rejection with an unchanged rank (:2662-2665): S = ([X0 X~]^T X0)
// S0 (W0^T [W0 W~]), X = [X0 X~], W = [W0 W~]. X~ and W~ sit in columns
// [k, 2k) of X and W already, so only the first k columns are replaced (own
// rows), followed by a team barrier (the next step's stencils read them).
static __device__ __noinline__ bool w_prej_expand_scatter(WCtx& x) {
    const int k = x.r, m = 2 * k;
    WSmem* sm = x.sm;
    {
        ProfScope ps_(x.prof, PF_ROWS_SCATTER);
        double* acc = sm->work;   // 2 m k
        double* t = sm->work + 2 * m * k;
        const int tr = rows_fit(WORKD - 2 * m * k, m);
        w_acc_zero(acc, 2 * m * k);
        const GBlock bx{0, m, 0, k, 0};   // [X0 X~]^T X0
        for (int r0 = x.c0; r0 < x.c1; r0 += tr) {
            const int nr = min(tr, x.c1 - r0);
            wload(t, m, 0, x.st.X0, RA, 0, r0, nr, k);
            wload(t, m, k, x.st.X, KA, k, r0, nr, k);
            __syncthreads();
            gram_blocks(acc, t, m, nr, &bx, 1);
            __syncthreads();
        }
        const GBlock bw{0, k, 0, m, m * k};   // W0^T [W0 W~]
        for (int r0 = x.m0; r0 < x.m1; r0 += tr) {
            const int nr = min(tr, x.m1 - r0);
            wload(t, m, 0, x.st.W0, RA, 0, r0, nr, k);
            wload(t, m, k, x.st.W, KA, k, r0, nr, k);
            __syncthreads();
            gram_blocks(acc, t, m, nr, &bw, 1);
            __syncthreads();
        }
        wpublish_chunk(x, acc, 0, 2 * m * k);
    }
    if (!wreduce(x, 2 * m * k)) return false;
    {
        ProfScope ps_(x.prof, PF_SMALL);
        double* Mu = sm->work;      // m x k
        double* Nu = Mu + m * k;    // k x m
        double* T = Nu + m * k;     // m x k: Mu S0
        double* U = T + m * k;      // m x m
        load_red(x, 0, m, k, Mu, k);
        load_red(x, m * k, k, m, Nu, m);
        g_mm(T, k, Mu, k, false, x.scr + SO_S0, RA, false, m, k, k);
        g_mm(U, m, T, k, false, Nu, m, false, m, k, m);
        for (int e = threadIdx.x; e < KA * KA; e += NT) {
            const int i = e / KA, j = e - (e / KA) * KA;
            sm->S[e] = (i < m && j < m) ? U[i * m + j] : 0.0;
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < (x.c1 - x.c0) * k; e += NT) {
        const int c = x.c0 + e / k, j = e - (e / k) * k;
        x.st.X[(size_t)c * KA + j] = x.st.X0[(size_t)c * RA + j];
    }
    for (int e = threadIdx.x; e < (x.m1 - x.m0) * k; e += NT) {
        const int mo = x.m0 + e / k, j = e - (e / k) * k;
        x.st.W[(size_t)mo * KA + j] = x.st.W0[(size_t)mo * RA + j];
    }
    return wsync(x);
}

// ---------------------------------------------------------------- kernel ---
// Loop state of one solve, carried into and out of energy_loop.
struct LoopState {
    int psi_idx;
    double t;
    int iters;
    int rank_sum;   // sum over the iterations of the rank entering each
    int eta_count;
    int n;          // on return: first energy index not processed
    bool aborted;
};

// The energy loop of one solve on this team (METHOD 1: n = n_begin..n_end;
// METHOD 2: the BUG while-loop with rejections; METHOD 5: the
// parallel-rejection while-loop), from the state in x / ls.
template <int METHOD>
static __device__ __noinline__ void energy_loop(WCtx& x, int n_begin, int n_end, int max_iters, LoopState& ls) {
    WSmem* sm = x.sm;
    const DevProblem& P = x.P;
    int psi_idx = ls.psi_idx;
    double t = ls.t;
    int iters = ls.iters;
    int rank_sum = ls.rank_sum;
    int eta_count = ls.eta_count;
    const double dE = P.dE;
    const int nE = P.nE;
    bool aborted = false;
    // METHOD 1 iterates n = n_begin..n_end; METHOD 2 runs the BUG while-loop
    int n = n_begin - 1;
    while (true) {
        n += 1;
        if (METHOD == TITUS_PARALLEL_ADAPTIVE) {
            if (n > n_end) break;
        } else {
            // BUG: while t < nEnergies dE (:2102); parallel rejection: (nEnergies-1) dE (:2467)
            if (!(t < (METHOD == TITUS_BUG_ADAPTIVE ? nE : nE - 1) * dE)) break;
            if (n == nE || n > n_end) break;
        }
        if (iters >= max_iters) break;
        x.cur_n = n;
        x.psi_in = psi_idx ? x.st.psi1 : x.st.psi0;
        x.psi_out = psi_idx ? x.st.psi0 : x.st.psi1;
        const double* sig = P.sigma + (size_t)(n - 1) * (P.npn + 1);
        if (METHOD != TITUS_PARALLEL_ADAPTIVE && x.b == 0 && threadIdx.x == 0 && iters < x.st.hist_cap) {
            x.st.rank_hist[iters] = x.r;
            x.st.time_hist[iters] = (double)n;   // energy index (eGrid[n-1] on the host)
        }
        ++iters;
        rank_sum += x.r;
        // ---- A, B
        const int k0 = x.r;   // rank entering the energy (parallel rejection: X0, W0, S0)
        if (METHOD == TITUS_PARALLEL_REJECTION) w_prej_save(x);
        w_phase_A(x, n);
        if (!wsync(x)) { aborted = true; break; }
        w_sweep(x, sig[0]);
        const bool stream = n > 2;
        if (stream) {
            if (!w_stream_grams(x)) { aborted = true; break; }
        } else if (!wsync(x)) {
            aborted = true;
            break;
        }
        psi_idx ^= 1;
        x.psi_in = psi_idx ? x.st.psi1 : x.st.psi0;
        if (stream) {
            const int k = x.r;
            w_stream_small(x, METHOD != TITUS_BUG_ADAPTIVE);
            if (!w_phase_C(x)) { aborted = true; break; }
            if (METHOD == TITUS_PARALLEL_REJECTION) {
                // [X X~], [W W~] (:2535, :2544); S_new from Sbar (:2549-2555); truncate! (:2558)
                if (!augment(x, false, true)) { aborted = true; break; }
                double* par = x.scr + SO_TMP;
                for (int e = threadIdx.x; e < 2 * k * k; e += NT) par[e] = ldcg(x.redp + e);
                __syncthreads();
                const double eta2 = w_prej_stream_eta(x);
                if (eta2 < 0.0) { aborted = true; break; }
                w_parallel_snew(x, par);
                const int kk = w_truncate_svd(x, 2 * k);
                if (kk < 0) { aborted = true; break; }
                bool repeat = false;
                if (kk == 2 * k && 2 * k < P.r) {
                    repeat = true;   // keep the truncation, redo this energy (n = n-1 without continue, :2561-2566)
                } else {
                    double s2 = 0.0;
                    for (int j = 0; j < kk; ++j) s2 += sm->sig[j] * sm->sig[j];
                    const double eta = sqrt(eta2);
                    const double bound = P.c_eta * P.theta * fmax(1e-7, pow(sqrt(s2), P.theta_index)) / dE;
                    if (x.b == 0 && threadIdx.x == 0 && eta_count < x.st.hist_cap) {
                        x.st.eta_hist[eta_count] = eta;
                        x.st.bound_hist[eta_count] = bound;
                    }
                    ++eta_count;
                    if (eta > bound && 2 * k < P.r) {
                        // reject: S = ([X X~]^T X) S (W^T [W W~]), rank 2k, repeat energy n (:2586-2593)
                        w_prej_expand_stream(x);
                        x.r = 2 * k;
                        n -= 1;
                        if (x.r > RA) {
                            if (threadIdx.x == 0) set_status(x.st.status, ST_LIMIT);
                            aborted = true;
                            break;
                        }
                        continue;
                    }
                }
                w_truncate_apply(x, 2 * k, kk, -1, nullptr);
                if (repeat) n -= 1;
                if (x.r > RA) {
                    if (threadIdx.x == 0) set_status(x.st.status, ST_LIMIT);
                    aborted = true;
                    break;
                }
            } else if (METHOD == TITUS_PARALLEL_ADAPTIVE) {
                if (!augment(x, false, true)) { aborted = true; break; }
                w_parallel_snew(x, x.redp);
                const int kk = w_truncate_svd(x, 2 * k);
                if (kk < 0) { aborted = true; break; }
                w_truncate_apply(x, 2 * k, kk, -1, nullptr);
                if (kk > RA) {
                    if (threadIdx.x == 0) set_status(x.st.status, ST_LIMIT);
                    aborted = true;
                    break;
                }
            } else {
                // BUG streaming: X1 = [Q1 X~], W1 = [Q1_W W~]; S = Mu S Nu^T
                if (!augment(x, true, false)) { aborted = true; break; }
                if (!wsync(x)) { aborted = true; break; }
                const int m = 2 * k;
                // S2 = blockdiag(M1 S N1^T, 0) in shared S (ld KA)
                double* T = sm->work;
                double* U = sm->work + RA * RA;
                g_mm(T, RA, sside(x, 0, SS_M1), RA, false, sm->S, KA, false, k, k, k);
                g_mm(U, RA, T, RA, false, sside(x, 1, SS_M1), RA, true, k, k, k);
                for (int e = threadIdx.x; e < KA * KA; e += NT) {
                    const int i = e / KA, j = e - (e / KA) * KA;
                    sm->S[e] = (i < k && j < k) ? U[i * RA + j] : 0.0;
                }
                __syncthreads();
                // S-step Grams with the 2k-wide bases, two operators per chunk
                double* acc = sm->work;
                const int mm = m * m;
                // operators per chunk: as many as fit with at least 16 feature rows
                int opc;
                if constexpr (kThreeD) {
                    const int fr = 16 * (NOPS_W + 1) * m;
                    opc = (12 * mm + fr <= WORKD) ? 6 : (6 * mm + fr <= WORKD) ? 3 : (4 * mm + fr <= WORKD) ? 2 : 1;
                } else {
                    opc = (8 * mm + 16 * 5 * m <= WORKD) ? 4 : ((4 * mm + 16 * 5 * m <= WORKD) ? 2 : 1);
                }
                double* F = sm->work + 2 * opc * mm;
                if (x.mixed && m >= kTcMinWidth) {
                    if (!w_grams_tc(x, x.st.X, x.st.W, m)) { aborted = true; break; }
                } else {
                    for (int d = 0; d < NOPS_W; d += opc) {
                        w_acc_zero(acc, 2 * opc * mm);
                        w_grams_pass(x, x.st.X, x.st.W, m, d, d + opc, 0, acc, F, (NOPS_W + 1) * m,
                                     rows_fit(WORKD - 2 * opc * mm, (NOPS_W + 1) * m));
                        wpublish_chunk(x, acc, d * mm, opc * mm);                        // X side G_d
                        wpublish_chunk(x, acc + opc * mm, (NOPS_W + d) * mm, opc * mm);  // W side C_d
                        __syncthreads();
                    }
                }
                if (!wreduce(x, 2 * NOPS_W * mm)) { aborted = true; break; }
                // Sup = S2 - dE sum_d G_d S2 C_d ; eta from the [k:, k:] block
                ProfScope ps_sup(x.prof, PF_SMALL);
                double* Gd = x.scr + SO_TMP;
                double* Cd = Gd + KA * KA;
                double* Tm = sm->work;                 // m x m
                double* Um = sm->work + KA * KA;       // m x m
                double* Sup = x.scr + SO_TMP + 2 * KA * KA;
                g_copy(Sup, KA, sm->S, KA, m, m);
                double* E = sm->work + 2 * KA * KA;    // k x k eta accumulator
                g_zero(E, RA, k, k);
                for (int d = 0; d < NOPS_W; ++d) {
                    load_red(x, d * mm, m, m, Gd, KA);
                    load_red(x, (NOPS_W + d) * mm, m, m, Cd, KA);
                    g_mm(Tm, KA, sm->S, KA, false, Cd, KA, false, m, m, m);
                    g_mm(Um, KA, Gd, KA, false, Tm, KA, false, m, m, m);
                    for (int e = threadIdx.x; e < m * m; e += NT) {
                        const int i = e / m, j = e - (e / m) * m;
                        Sup[i * KA + j] -= dE * Um[i * KA + j];
                        if (i >= k && j >= k) E[(i - k) * RA + (j - k)] += Um[i * KA + j];
                    }
                    __syncthreads();
                }
                double e2 = 0.0, s2p = 0.0;
                for (int e = threadIdx.x; e < k * k; e += NT) {
                    const double v = E[(e / k) * RA + e % k];
                    e2 = fma(v, v, e2);
                }
                for (int e = threadIdx.x; e < m * m; e += NT) {
                    const double v = Sup[(e / m) * KA + e % m];
                    s2p = fma(v, v, s2p);
                }
                const double eta2 = cta_sum(e2), sup2 = cta_sum(s2p);
                // truncate Sup
                double* At = sm->work;
                __syncthreads();
                for (int e = threadIdx.x; e < m * m; e += NT) {
                    const int i = e / m, j = e - (e / m) * m;
                    At[j * LDS + i] = Sup[i * KA + j];
                }
                __syncthreads();
                const int kk = w_truncate_svd(x, m);
                if (kk < 0) { aborted = true; break; }
                bool repeat = false;
                if (kk == 2 * k && 2 * k < P.r) {
                    repeat = true;   // accept the truncation, redo this energy (n = n-1 without continue)
                } else {
                    const double eta = sqrt(eta2);
                    const double bound = P.c_eta * P.theta * fmax(1e-7, pow(sqrt(sup2), P.theta_index)) / dE;
                    if (x.b == 0 && threadIdx.x == 0 && eta_count < x.st.hist_cap) {
                        x.st.eta_hist[eta_count] = eta;
                        x.st.bound_hist[eta_count] = bound;
                    }
                    ++eta_count;
                    if (eta > bound && 2 * k < P.r) {
                        // reject: keep X1, S2, W1 with rank 2k and repeat energy n
                        x.r = 2 * k;
                        n -= 1;
                        if (x.r > RA) {
                            if (threadIdx.x == 0) set_status(x.st.status, ST_LIMIT);
                            aborted = true;
                            break;
                        }
                        continue;
                    }
                }
                w_truncate_apply(x, m, kk, -1, nullptr);
                if (repeat) n -= 1;
                if (x.r > RA) {
                    if (threadIdx.x == 0) set_status(x.st.status, ST_LIMIT);
                    aborted = true;
                    break;
                }
            }
        }
        // ---- out-scattering
        if (!w_outscatter(x, sig)) { aborted = true; break; }
        if (METHOD == TITUS_PARALLEL_REJECTION && !stream) w_prej_save_s(x);   // S0 aliases S at n = 2
        // ---- in-scattering
        w_zero_bnd(x);
        {
            const int k = x.r;
            if (!w_inscatter_KL(x, sig, METHOD != TITUS_BUG_ADAPTIVE, METHOD == TITUS_PARALLEL_ADAPTIVE, n - 1)) {
                aborted = true;
                break;
            }
            if (METHOD == TITUS_PARALLEL_ADAPTIVE) {
                if (!augment(x, false, true)) { aborted = true; break; }
                w_parallel_snew(x, x.redp);
                const int kk = w_truncate_svd(x, 2 * k);
                if (kk < 0) { aborted = true; break; }
                w_truncate_apply(x, 2 * k, kk, -1, nullptr);
                if (kk > RA) {
                    if (threadIdx.x == 0) set_status(x.st.status, ST_LIMIT);
                    aborted = true;
                    break;
                }
                if (x.b == 0 && threadIdx.x == 0) {
                    if (n - 1 < x.st.hist_cap) {
                        x.st.rank_hist[n - 1] = x.r;
                        x.st.time_hist[n - 1] = t;
                    }
                }
                t += dE;
            } else if (METHOD == TITUS_PARALLEL_REJECTION) {
                // [X X~], [W W~] (:2627, :2632); S_new (:2634-2639); truncate! (:2642)
                if (!augment(x, false, true)) { aborted = true; break; }
                double* par = x.scr + SO_TMP;
                double* w0 = x.scr + SO_TMP + 2 * KA * KA;   // row 0 of [W W~] for the dose
                for (int e = threadIdx.x; e < 2 * k * k; e += NT) par[e] = ldcg(x.redp + e);
                __syncthreads();
                const double eta2 = w_prej_scatter_eta(x, sig, w0);
                if (eta2 < 0.0) { aborted = true; break; }
                w_parallel_snew(x, par);
                const int kk = w_truncate_svd(x, 2 * k);
                if (kk < 0) { aborted = true; break; }
                bool repeat = false;
                if (kk == 2 * k && 2 * k < P.r) {
                    repeat = true;   // :2645-2650, no continue
                } else {
                    double s2 = 0.0;
                    for (int j = 0; j < kk; ++j) s2 += sm->sig[j] * sm->sig[j];
                    const double eta = sqrt(eta2);
                    const double bound = P.c_eta * P.theta * fmax(1e-7, pow(sqrt(s2), P.theta_index)) / dE;
                    if (eta > bound && 2 * k < P.r) {
                        if (k0 != k) {
                            // [X0 X~] has k0 + k columns but the reference sets r = 2k; its
                            // repeated step's SNew[1:r,1:r] .= SBar (:2553) raises DimensionMismatch
                            if (threadIdx.x == 0 && atomicCAS(x.st.status, 0, ST_REF_SHAPE) == 0) {
                                x.st.diag[0] = k0;
                                x.st.diag[2] = k;
                                x.st.diag[7] = n;
                            }
                            aborted = true;
                            break;
                        }
                        if (!w_prej_expand_scatter(x)) { aborted = true; break; }
                        x.r = 2 * k;
                        n -= 1;
                        if (x.r > RA) {
                            if (threadIdx.x == 0) set_status(x.st.status, ST_LIMIT);
                            aborted = true;
                            break;
                        }
                        continue;
                    }
                }
                // the dose takes S[n] of the decremented n after a first-branch rejection (:2683)
                w_truncate_apply(x, 2 * k, kk, repeat ? n - 2 : n - 1, w0);
                if (repeat) n -= 1;
                if (x.r > RA) {
                    if (threadIdx.x == 0) set_status(x.st.status, ST_LIMIT);
                    aborted = true;
                    break;
                }
                t += dE;
            } else {
                const int m = 2 * k;
                if (!augment(x, true, false)) { aborted = true; break; }
                // Grams X1^T psi (m x q) and MRed^T D W1 (q x m) over the new bases
                double* acc = sm->work;
                const int ldt = m + P.q + (P.q & 1);     // [X1 | psi] or [W1 | MRed D]; m even
                const int tstart = 2 * KA * QW + KA;   // after the largest accumulator
                const int tr = rows_fit(WORKD - tstart, ldt);
                double* tt = sm->work + tstart;
                w_acc_zero(acc, 2 * m * P.q + m);
                const GBlock bx{0, m, m, P.q, 0};
                for (int r0 = x.c0; r0 < x.c1; r0 += tr) {
                    const int nr = min(tr, x.c1 - r0);
                    // own rows of X1 were just written by this CTA
                    wload(tt, ldt, 0, x.st.X, KA, 0, r0, nr, m);
                    wload(tt, ldt, m, x.psi_in, QW, 0, r0, nr, P.q);
                    __syncthreads();
                    gram_blocks(acc, tt, ldt, nr, &bx, 1);
                    __syncthreads();
                }
                const GBlock bw{m, P.q, 0, m, m * P.q};
                for (int r0 = x.m0; r0 < x.m1; r0 += tr) {
                    const int nr = min(tr, x.m1 - r0);
                    wload(tt, ldt, 0, x.st.W, KA, 0, r0, nr, m);
                    for (int e = threadIdx.x; e < nr * P.q; e += NT) {
                        const int r = e / P.q, kq = e - (e / P.q) * P.q;
                        const int mo = r0 + r;
                        tt[r * ldt + m + kq] = P.mred[(size_t)mo * P.q + kq] * sig[P.lof[mo]];
                    }
                    __syncthreads();
                    gram_blocks(acc, tt, ldt, nr, &bw, 1);
                    __syncthreads();
                }
                // row 0 of W1 travels through the reduction (only its owner adds it)
                if (x.m0 == 0 && x.m1 > 0)
                    for (int j = threadIdx.x; j < m; j += NT) acc[2 * m * P.q + j] = ldcg(x.st.W + j);
                __syncthreads();
                wpublish_chunk(x, acc, 0, 2 * m * P.q + m);
                if (!wreduce(x, 2 * m * P.q + m)) { aborted = true; break; }
                double* Xp = x.scr + SO_XTPSI;   // m x q (ld QW)
                double* Mt = x.scr + SO_MTDW;    // q x m (ld KA)
                load_red(x, 0, m, P.q, Xp, QW);
                load_red(x, m * P.q, P.q, m, Mt, KA);
                load_red(x, 2 * m * P.q, 1, m, x.scr + SO_TMP, KA);
                // S2 = blockdiag(M1 S N1^T, 0); Sup = S2 + dE Xtpsi MtDW
                double* T = sm->work;
                double* U = sm->work + RA * RA;
                g_mm(T, RA, sside(x, 0, SS_M1), RA, false, sm->S, KA, false, k, k, k);
                g_mm(U, RA, T, RA, false, sside(x, 1, SS_M1), RA, true, k, k, k);
                for (int e = threadIdx.x; e < KA * KA; e += NT) {
                    const int i = e / KA, j = e - (e / KA) * KA;
                    sm->S[e] = (i < k && j < k) ? U[i * RA + j] : 0.0;
                }
                __syncthreads();
                double* At = sm->work;
                for (int e = threadIdx.x; e < m * m; e += NT) {
                    const int i = e / m, j = e - (e / m) * m;
                    double a = 0.0;
                    for (int l = 0; l < P.q; ++l) a = fma(Xp[i * QW + l], Mt[l * KA + j], a);
                    At[j * LDS + i] = sm->S[i * KA + j] + dE * a;
                }
                __syncthreads();
                // eta = ||Xtpsi[k:, :] MtDW[:, k:]||_F
                double e2 = 0.0;
                for (int e = threadIdx.x; e < k * k; e += NT) {
                    const int i = k + e / k, j = k + e % k;
                    double a = 0.0;
                    for (int l = 0; l < P.q; ++l) a = fma(Xp[i * QW + l], Mt[l * KA + j], a);
                    e2 = fma(a, a, e2);
                }
                const double eta2 = cta_sum(e2);
                const int kk = w_truncate_svd(x, m);
                if (kk < 0) { aborted = true; break; }
                bool repeat = false;
                if (kk == 2 * k && 2 * k < P.r) {
                    repeat = true;
                } else {
                    double s2 = 0.0;
                    for (int j = 0; j < kk; ++j) s2 += sm->sig[j] * sm->sig[j];
                    const double eta = sqrt(eta2);
                    const double bound = P.c_eta * P.theta * fmax(1e-7, pow(sqrt(s2), P.theta_index)) / dE;
                    if (eta > bound && 2 * k < P.r) {
                        x.r = 2 * k;
                        n -= 1;
                        if (x.r > RA) {
                            if (threadIdx.x == 0) set_status(x.st.status, ST_LIMIT);
                            aborted = true;
                            break;
                        }
                        continue;
                    }
                }
                // the dose takes S[n] of the decremented n after a first-branch rejection (:2315)
                w_truncate_apply(x, m, kk, repeat ? n - 2 : n - 1, x.scr + SO_TMP);
                if (repeat) n -= 1;
                if (x.r > RA) {
                    if (threadIdx.x == 0) set_status(x.st.status, ST_LIMIT);
                    aborted = true;
                    break;
                }
                t += dE;
            }
        }
        // the truncation rewrote X and W rows without a team barrier; the next
        // step's first dose half-step reads W's row 0 owned by another CTA
        if (!wsync(x)) {
            aborted = true;
            break;
        }
    }
    ls.psi_idx = psi_idx;
    ls.t = t;
    ls.iters = iters;
    ls.rank_sum = rank_sum;
    ls.eta_count = eta_count;
    ls.n = n;
    ls.aborted = aborted;
}

template <int METHOD>
__global__ void __launch_bounds__(NT, 1)
adaptive_kernel(DevProblem P, WideState* states, int G, int n_begin, int n_end, int max_iters) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    WSmem* sm = reinterpret_cast<WSmem*>(smem_raw);
    WCtx x;
    x.P = P;
    x.G = G;
    x.b = blockIdx.x;
    x.st = states[0];
    x.sm = sm;
    x.scr = x.st.scr + (size_t)x.b * SCRW;
    x.prof = (blockIdx.x == 0) ? P.prof : nullptr;
    x.gen = 0;
    x.parity = 0;
    x.redp = x.st.red;
    x.cur_n = 0;
    prof_begin(x.prof);
    ProfScope ps_total(x.prof, PF_TOTAL);
    x.c0 = (int)((long long)x.b * P.n / G);
    x.c1 = (int)((long long)(x.b + 1) * P.n / G);
    x.m0 = (int)((long long)x.b * P.N / G);
    x.m1 = (int)((long long)(x.b + 1) * P.N / G);
    x.r = ldcg(x.st.info + 0);
    for (int e = threadIdx.x; e < KA * KA; e += NT) sm->S[e] = ldcg(x.st.S + e);
    __syncthreads();
    LoopState ls;
    ls.psi_idx = ldcg(x.st.info + 2);
    ls.t = ldcg(x.st.tvar);
    ls.iters = 0;
    ls.rank_sum = 0;
    ls.eta_count = ldcg(x.st.info + 4);
    ls.n = n_begin;
    ls.aborted = false;
    tc_setup(x);
    energy_loop<METHOD>(x, n_begin, n_end, max_iters, ls);
    tc_teardown(x);
    if (x.b == 0) {
        for (int e = threadIdx.x; e < KA * KA; e += NT) x.st.S[e] = sm->S[e];
        if (threadIdx.x == 0) {
            x.st.info[0] = x.r;
            x.st.info[1] = ls.iters;
            x.st.info[2] = ls.psi_idx;
            x.st.info[3] = ls.n;   // first energy index not processed
            x.st.info[4] = ls.eta_count;
            x.st.tvar[0] = ls.t;
        }
    }
}


// Per-spot tables of a batched launch (pencil beams with their own energy and
// entry point): the energy grid and everything indexed by it, and the beam's
// spatial profile. All spots share the phantom, the P_N operators and dE's rule.
struct SpotData {
    int nE;                    // energies of this spot's grid
    int n_end;                 // last energy index to run (parallel integrator)
    double dE;                 // its tau step
    const double* stopping;    // nE
    const double* bc_energy;   // nE
    const double* sigma;       // nE x (npn+1)
    const double* bc_space;    // n
    double* dose;              // n (output)
    int* result;               // [final rank, iterations, sum of the ranks entering the iterations]
};

// Initial factors of one spot (SolverCSD.jl:1728-1760, :2013-2050) on this
// CTA's own rows: X, W = first r0 identity columns (X's boundary rows zero),
// S = 0, psi = 0, dose = 0.
static __device__ __noinline__ void init_spot(WCtx& x, int r0) {
    const DevProblem& P = x.P;
    for (int e = threadIdx.x; e < (x.c1 - x.c0) * KA; e += NT) x.st.X[(size_t)x.c0 * KA + e] = 0.0;
    for (int e = threadIdx.x; e < (x.m1 - x.m0) * KA; e += NT) x.st.W[(size_t)x.m0 * KA + e] = 0.0;
    for (int e = threadIdx.x; e < (x.c1 - x.c0) * QW; e += NT) {
        x.st.psi0[(size_t)x.c0 * QW + e] = 0.0;
        x.st.psi1[(size_t)x.c0 * QW + e] = 0.0;
    }
    for (int c = x.c0 + threadIdx.x; c < x.c1; c += NT) x.st.dose[c] = 0.0;
    for (int e = threadIdx.x; e < KA * KA; e += NT) x.sm->S[e] = 0.0;
    __syncthreads();
    for (int j = threadIdx.x; j < r0; j += NT) {
        if (j >= x.c0 && j < x.c1) x.st.X[(size_t)j * KA + j] = is_bnd_w(P, j) ? 0.0 : 1.0;
        if (j >= x.m0 && j < x.m1) x.st.W[(size_t)j * KA + j] = 1.0;
    }
    __syncthreads();
}

// Batched solves: T teams of G CTAs take spots from a device work queue (an
// atomic counter over `order`, the spots sorted longest first) until it runs
// dry, re-initialising their factors on the device between spots. CTA 0 of a
// team draws the next index and publishes it to the team through info[6]
// and a team barrier. Each spot's dose goes to its own output buffer; a spot's
// result does not depend on which team solved it (all teams have G CTAs and
// the same reduction order). `max_steps_par` > 0 bounds the parallel
// integrator's energy index to 1 + max_steps_par.
template <int METHOD>
__global__ void __launch_bounds__(NT, 1)
adaptive_batched_kernel(DevProblem P0, WideState* states, int G, int T, const SpotData* spots, int nspots, int r0,
                        int max_iters, int max_steps_par, int* queue, const int* order) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    WSmem* sm = reinterpret_cast<WSmem*>(smem_raw);
    const int team = blockIdx.x / G;
    WCtx x;
    x.P = P0;
    x.G = G;
    x.b = blockIdx.x - team * G;
    x.st = states[team];
    x.sm = sm;
    x.scr = x.st.scr + (size_t)x.b * SCRW;
    x.prof = (blockIdx.x == 0) ? P0.prof : nullptr;
    x.gen = 0;
    x.parity = 0;
    x.redp = x.st.red;
    x.cur_n = 0;
    prof_begin(x.prof);
    ProfScope ps_total(x.prof, PF_TOTAL);
    x.c0 = (int)((long long)x.b * P0.n / G);
    x.c1 = (int)((long long)(x.b + 1) * P0.n / G);
    x.m0 = (int)((long long)x.b * P0.N / G);
    x.m1 = (int)((long long)(x.b + 1) * P0.N / G);
    __shared__ int s_next;
    tc_setup(x);
    while (true) {
        if (x.b == 0 && threadIdx.x == 0) {
            const int q = atomicAdd(queue, 1);
            s_next = q;
            if (G > 1) x.st.info[6] = q;   // read by the team after the barrier below
        }
        __syncthreads();
        if (G > 1) {
            if (!wsync(x)) break;
            if (x.b != 0 && threadIdx.x == 0) s_next = ldcg(x.st.info + 6);
            __syncthreads();
        }
        const int qi = s_next;
        if (qi >= nspots) break;
        const int sidx = order[qi];
        const SpotData sp = spots[sidx];
        x.P = P0;
        x.P.nE = sp.nE;
        x.P.dE = sp.dE;
        x.P.stopping = sp.stopping;
        x.P.bc_energy = sp.bc_energy;
        x.P.sigma = sp.sigma;
        x.P.bc_space = sp.bc_space;
        x.st.dose = sp.dose;
        init_spot(x, r0);
        x.r = r0;
        if (!wsync(x)) break;
        LoopState ls;
        ls.psi_idx = 0;
        ls.t = 0.0;
        ls.iters = 0;
        ls.rank_sum = 0;
        ls.eta_count = 0;
        ls.n = 2;
        ls.aborted = false;
        const int n_end = (METHOD == TITUS_PARALLEL_ADAPTIVE && max_steps_par > 0) ? min(sp.nE, 1 + max_steps_par)
                                                                                     : sp.n_end;
        energy_loop<METHOD>(x, 2, n_end, max_iters, ls);
        if (ls.aborted) break;
        if (x.b == 0 && threadIdx.x == 0) {
            sp.result[0] = x.r;
            sp.result[1] = ls.iters;
            sp.result[2] = ls.rank_sum;
        }
    }
    tc_teardown(x);
}

}  // namespace TITUS_WIDE_NS
}  // namespace titus
