// Persistent DLR energy-step kernel: fixed-rank integrator
// (SolverCSD.jl SolveFirstCollisionSourceDLR, :891-1120).
//
// Each energy step is a fixed sequence of phases separated by team barriers:
//   A  boundary inflow (PsiBeam, :977-988) + dose half-steps (:990-997, :1104-1111)
//   B  uncollided upwind sweep (:1000-1005, solveFluxUpwind! :388-463)
//      + streaming Grams X^T L_d X, W^T A_d W (:1022-1025, :1035-1038)
//   C  K = XS - dE sum L_d K C_d, L = WS^T - dE sum A_d L G_d^T (:1027, :1040)
//   D,E,F  rank-revealing orthonormal bases of K and L (svd!(K).U, :1029/:1042)
//   G  S-step Grams with the new bases (:1053-1063)
//   H..K out-scattering (:1066-1074)
//   L..O in-scattering K/L/S (:1076-1102)
// The range finder: Jacobi eig of A^T A -> V; Gram of A V -> Jacobi -> V2, nu;
// C = A V V2_J / nu_J materialised; CholQR on C. Directions with
// nu_j <= tol nu_0 are null; rank-deficient bases are completed with the
// candidate canonical vectors in index order (boundary cells for X, moments for W).
#pragma once
#include "dlr_device.cuh"

namespace titus {

constexpr int NSLOT = 24;

struct SmemLayout {
    double slot[NSLOT][KK];
    double ja[KK], jv[KK];
    double lamK[KM], lamL[KM];
    double acc[PMAX];
    double tA[TR * KM];
    double tL[4][TR * KM];
    double tO[TR * KM];
    double tP[TR * QM];
    double vec[4 * KM + QM];
    double wnrm[KM];
    int wcand[KM];
    int misc[8];
};

// slot indices
enum {
    SL_S = 0, SL_G0 = 1, SL_C0 = 5, SL_P0 = 9,
    SL_VK = 13, SL_VL = 14, SL_TK = 15, SL_TL = 16, SL_RK = 17, SL_RL = 18,
    SL_RIK = 19, SL_RIL = 20, SL_M = 21, SL_N = 22, SL_WC = 23
};

struct Ctx {
    DevProblem P;
    TeamState st;
    SmemLayout* sm;
    int G, b;
    int c0, c1, m0, m1;  // own cells / moments
    int k;               // current basis width (rank)
    double* psi_in;
    double* psi_out;
    double* CX;          // n x KM scratch (materialised C of the X-side range finder)
    double* CW;          // N x KM scratch
    int rhoK, rhoL;
    unsigned long long* prof;  // non-null only on the profiled CTA
    int red_mode;              // 1: reductions read the team's two-stage buffer
    unsigned gen;              // team barrier generation
    int parity;                // partial buffer in use (double-buffered)
    int cur_n;                 // energy index of the current step (diagnostics)
};

constexpr int kDirectReduceMax = 16;  // teams up to this size sum partials directly
constexpr int kBigRows = 6 * TR;      // rows per chunk when tA..tO are used as one tile

__device__ __forceinline__ bool is_bnd(const DevProblem& P, int c) {
    int i = c / P.ny, j = c - (c / P.ny) * P.ny;
    return i == 0 || j == 0 || i == P.nx - 1 || j == P.ny - 1;
}

// ------------------------------------------------------------- reductions ---
__device__ __forceinline__ void acc_zero(Ctx& x, int count) {
    for (int e = threadIdx.x; e < count; e += NT) x.sm->acc[e] = 0.0;
    __syncthreads();
}
// Partials are double-buffered by parity: a CTA may publish the next
// reduction while slower CTAs still read the previous one.
__device__ __forceinline__ double* part_base(const Ctx& x, int g) {
    return x.st.part + ((size_t)x.parity * x.G + g) * PMAX;
}
__device__ __forceinline__ void acc_publish(Ctx& x, int count) {
    x.parity ^= 1;
    double* dst = part_base(x, x.b);
    for (int e = threadIdx.x; e < count; e += NT) dst[e] = x.sm->acc[e];
}
// sum partial entries [off, off+m*n) over the team's CTAs into dst (KM stride)
__device__ inline void reduce_into(Ctx& x, int off, int m, int n, double* dst, int ld = KM) {
    ProfScope ps(x.prof, PF_REDUCE);
    if (x.red_mode) {
        for (int e = threadIdx.x; e < m * n; e += NT) dst[(e / n) * ld + e % n] = ldcg(x.st.red + off + e);
    } else {
        for (int e = threadIdx.x; e < m * n; e += NT) {
            double s = 0.0;
            for (int g = 0; g < x.G; ++g) s += ldcg(part_base(x, g) + off + e);
            dst[(e / n) * ld + e % n] = s;
        }
    }
    __syncthreads();
}

// acc[off + i*kb + j] += sum_r tA[r][i] tB[r][j]
__device__ __forceinline__ void gram_acc(double* acc, int off, const double* tA, int lda, int ka,
                                         const double* tB, int ldb, int kb, int nr) {
    for (int e = threadIdx.x; e < ka * kb; e += NT) {
        int i = e / kb, j = e - (e / kb) * kb;
        double s = 0.0;
        for (int r = 0; r < nr; ++r) s = fma(tA[r * lda + i], tB[r * ldb + j], s);
        acc[off + e] += s;
    }
}

// ------------------------------------------------------------ row helpers ---
__device__ __forceinline__ void load_rows(double* t, const double* A, int r0, int nr, int k) {
    for (int e = threadIdx.x; e < nr * k; e += NT) {
        int r = e / k, j = e - (e / k) * k;
        t[r * KM + j] = ldcg(A + (size_t)(r0 + r) * KM + j);
    }
}
__device__ __forceinline__ void store_rows(double* A, const double* t, int r0, int nr, int k) {
    for (int e = threadIdx.x; e < nr * k; e += NT) {
        int r = e / k, j = e - (e / k) * k;
        A[(size_t)(r0 + r) * KM + j] = t[r * KM + j];
    }
}
// tO[r][j] = sum_l tA[r][l] M[l][j]  (tA: nr x ka, M: ka x kb)
__device__ __forceinline__ void tile_mm(double* tO, const double* tA, const double* M, int nr, int ka, int kb) {
    for (int e = threadIdx.x; e < nr * kb; e += NT) {
        int r = e / kb, j = e - (e / kb) * kb;
        double s = 0.0;
        for (int l = 0; l < ka; ++l) s = fma(tA[r * KM + l], M[l * KM + j], s);
        tO[r * KM + j] = s;
    }
}

// Matrix-free stencils (stencils.jl:26-128) applied to rows [r0, r0+nr) of A:
// t[0] = L2x A, t[1] = L2y A, t[2] = L1x A, t[3] = L1y A; zero on boundary rows.
__device__ inline void stencil_tile(const Ctx& x, const double* A, int r0, int nr, int k, double (*t)[TR * KM]) {
    const DevProblem& P = x.P;
    const double hx = 0.5 / P.dx, hy = 0.5 / P.dy;
    for (int e = threadIdx.x; e < nr * k; e += NT) {
        int r = e / k, j = e - (e / k) * k;
        int c = r0 + r;
        double l2x = 0.0, l2y = 0.0, l1x = 0.0, l1y = 0.0;
        if (!is_bnd(P, c)) {
            double a0 = ldcg(A + (size_t)c * KM + j) * P.rinv[c];
            double axm = ldcg(A + (size_t)(c - P.ny) * KM + j) * P.rinv[c - P.ny];
            double axp = ldcg(A + (size_t)(c + P.ny) * KM + j) * P.rinv[c + P.ny];
            double aym = ldcg(A + (size_t)(c - 1) * KM + j) * P.rinv[c - 1];
            double ayp = ldcg(A + (size_t)(c + 1) * KM + j) * P.rinv[c + 1];
            l2x = (axp - axm) * hx;
            l2y = (ayp - aym) * hy;
            l1x = a0 / P.dx - hx * axm - hx * axp;
            l1y = a0 / P.dy - hy * aym - hy * ayp;
        }
        t[0][r * KM + j] = l2x;
        t[1][r * KM + j] = l2y;
        t[2][r * KM + j] = l1x;
        t[3][r * KM + j] = l1y;
    }
}

// Central stencils only (the RK4 integrator's streaming): t[0] = L2x A,
// t[1] = L2y A on rows [r0, r0+nr); zero on boundary rows.
__device__ inline void stencil2_tile(const Ctx& x, const double* A, int r0, int nr, int k, double (*t)[TR * KM]) {
    const DevProblem& P = x.P;
    const double hx = 0.5 / P.dx, hy = 0.5 / P.dy;
    for (int e = threadIdx.x; e < nr * k; e += NT) {
        int r = e / k, j = e - (e / k) * k;
        int c = r0 + r;
        double l2x = 0.0, l2y = 0.0;
        if (!is_bnd(P, c)) {
            double axm = ldcg(A + (size_t)(c - P.ny) * KM + j) * P.rinv[c - P.ny];
            double axp = ldcg(A + (size_t)(c + P.ny) * KM + j) * P.rinv[c + P.ny];
            double aym = ldcg(A + (size_t)(c - 1) * KM + j) * P.rinv[c - 1];
            double ayp = ldcg(A + (size_t)(c + 1) * KM + j) * P.rinv[c + 1];
            l2x = (axp - axm) * hx;
            l2y = (ayp - aym) * hy;
        }
        t[0][r * KM + j] = l2x;
        t[1][r * KM + j] = l2y;
    }
}

// Sparse P_N operators applied to rows [r0, r0+nr) of B (N x KM): t[d] = A_d B
// for the first `nops` operators (Ax, Az, |Ax|, |Az|).
__device__ inline void spmm_tile(const Ctx& x, const double* B, int r0, int nr, int k, double (*t)[TR * KM],
                                 int nops = NOPS) {
    for (int e = threadIdx.x; e < nops * nr * k; e += NT) {
        int d = e / (nr * k);
        int rem = e - d * nr * k;
        int r = rem / k, j = rem - (rem / k) * k;
        const Csr& A = x.P.op[d];
        int m = r0 + r;
        double s = 0.0;
        for (int p = A.rowptr[m]; p < A.rowptr[m + 1]; ++p) s = fma(A.val[p], ldcg(B + (size_t)A.col[p] * KM + j), s);
        t[d][r * KM + j] = s;
    }
}

// ----------------------------------------------------- range finder parts ---
// After G0 (Gram of A) is reduced into sm->ja: Jacobi -> V slot.
__device__ inline void rf_eig0(Ctx& x, double* V, double* lam, int k) {
    {
        ProfScope ps(x.prof, PF_JACOBI);
        jacobi_eig(x.sm->ja, x.sm->jv, lam, k, x.st.status);
    }
    sm_copy(V, x.sm->jv, k, k);
}
// After G1 (Gram of A V) in sm->ja: Jacobi -> V2 ; T1 = V V2_J diag(1/nu_J); returns rho.
__device__ inline int rf_eig1(Ctx& x, const double* V, double* T1, int k, double tol) {
    __shared__ double s_nu[KM];
    __shared__ int s_rho;
    {
        ProfScope ps(x.prof, PF_JACOBI);
        jacobi_eig(x.sm->ja, x.sm->jv, s_nu, k, x.st.status);
    }
    if (threadIdx.x == 0) {
        double nu0 = sqrt(fmax(s_nu[0], 0.0));
        int rho = 0;
        if (nu0 > 0.0) {
            for (int j = 0; j < k; ++j) {
                double nj = sqrt(fmax(s_nu[j], 0.0));
                if (nj > tol * nu0) rho = j + 1; else break;
            }
        }
        s_rho = rho;
        for (int j = 0; j < k; ++j) s_nu[j] = sqrt(fmax(s_nu[j], 0.0));
    }
    __syncthreads();
    int rho = s_rho;
    // T1 = V * V2[:, :rho] / nu
    for (int e = threadIdx.x; e < k * rho; e += NT) {
        int i = e / rho, j = e - (e / rho) * rho;
        double s = 0.0;
        for (int l = 0; l < k; ++l) s = fma(V[i * KM + l], x.sm->jv[l * KM + j], s);
        T1[i * KM + j] = s / s_nu[j];
    }
    __syncthreads();
    return rho;
}

// W-side completion in the small space (see oracle.linalg._complete):
// candidate c is accepted when 1 - ||P[c,:]||^2 > 1/4, P = [B, v_1..v_a],
// B = CW Ri. Stores per accepted vector its candidate, norm and coefficients
// w_a = P_{a-1}[c_a, :] in slot SL_WC (row a).
static __device__ __noinline__ void w_complete(Ctx& x, int rho, int need) {
    ProfScope ps(x.prof, PF_COMPLETE);
    SmemLayout* sm = x.sm;
    double* wc = sm->slot[SL_WC];
    double* Ri = sm->slot[SL_RIL];
    double* brow = sm->vec;           // B[c,:] (rho)
    __shared__ int s_acc, s_next;
    if (threadIdx.x == 0) { s_acc = 0; s_next = 0; }
    __syncthreads();
    while (true) {
        int acc = s_acc, it = s_next;
        if (acc >= need) break;
        if (it >= x.P.nwcomp || it >= NCAND) {
            if (threadIdx.x == 0) set_status(x.st.status, ST_COMPLETION);
            __syncthreads();
            break;
        }
        int c = x.P.wcomp[it];
        for (int j = threadIdx.x; j < rho; j += NT) {
            double s = 0.0;
            for (int l = 0; l <= j; ++l) s = fma(ldcg(x.CW + (size_t)c * KM + l), Ri[l * KM + j], s);
            brow[j] = s;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double* prow = sm->vec + KM;  // [B[c,:], v_1[c], ..., v_acc[c]]
            for (int j = 0; j < rho; ++j) prow[j] = brow[j];
            for (int a = 0; a < acc; ++a) {
                const double* w = wc + a * KM;
                double v = (c == sm->wcand[a]) ? 1.0 : 0.0;
                for (int j = 0; j < rho + a; ++j) v -= prow[j] * w[j];
                prow[rho + a] = v / sm->wnrm[a];
            }
            double ss = 0.0;
            for (int j = 0; j < rho + acc; ++j) ss += prow[j] * prow[j];
            double nv2 = 1.0 - ss;
            if (nv2 > 0.25) {
                for (int j = 0; j < rho + acc; ++j) wc[acc * KM + j] = prow[j];
                sm->wcand[acc] = c;
                sm->wnrm[acc] = sqrt(nv2);
                s_acc = acc + 1;
            }
            s_next = it + 1;
        }
        __syncthreads();
    }
}

// Materialise rows [r0, r0+nr) of the new W-side basis into tile t:
// columns :rho = C Ri, columns rho+a = completion vector a.
__device__ inline void w_basis_tile(Ctx& x, int r0, int nr, int rho, int need, double* t) {
    SmemLayout* sm = x.sm;
    const double* Ri = sm->slot[SL_RIL];
    load_rows(sm->tA, x.CW, r0, nr, rho);
    __syncthreads();
    for (int e = threadIdx.x; e < nr * rho; e += NT) {
        int r = e / rho, j = e - (e / rho) * rho;
        double s = 0.0;
        for (int l = 0; l <= j; ++l) s = fma(sm->tA[r * KM + l], Ri[l * KM + j], s);
        t[r * KM + j] = s;
    }
    __syncthreads();
    if (need > 0) {
        const double* wc = sm->slot[SL_WC];
        for (int r = threadIdx.x; r < nr; r += NT) {
            int m = r0 + r;
            double* row = t + r * KM;
            for (int a = 0; a < need; ++a) {
                const double* w = wc + a * KM;
                double v = (m == sm->wcand[a]) ? 1.0 : 0.0;
                for (int j = 0; j < rho + a; ++j) v -= row[j] * w[j];
                row[rho + a] = v / sm->wnrm[a];
            }
        }
        __syncthreads();
    }
}

// Materialise rows of the new X-side basis: C Ri, then completion cells.
__device__ inline void x_basis_tile(Ctx& x, int r0, int nr, int rho, int k, double* t) {
    SmemLayout* sm = x.sm;
    const double* Ri = sm->slot[SL_RIK];
    load_rows(sm->tA, x.CX, r0, nr, rho);
    __syncthreads();
    for (int e = threadIdx.x; e < nr * k; e += NT) {
        int r = e / k, j = e - (e / k) * k;
        double s;
        if (j < rho) {
            s = 0.0;
            for (int l = 0; l <= j; ++l) s = fma(sm->tA[r * KM + l], Ri[l * KM + j], s);
        } else {
            // completion failures are reported through the status flag; keep reads in bounds
            const int ci = j - rho;
            s = (ci < x.P.nxcomp && r0 + r == x.P.xcomp[ci]) ? 1.0 : 0.0;
        }
        t[r * KM + j] = s;
    }
    __syncthreads();
}

}  // namespace titus
