// Fixed-rank DLR energy loop (SolverCSD.jl SolveFirstCollisionSourceDLR :891-1120)
// as phases of one persistent kernel. See dlr_kernel.cuh for the phase map.
#pragma once
#include "dlr_kernel.cuh"
#include "limiter.cuh"

namespace titus {

__device__ __forceinline__ bool tsync(Ctx& x) {
    ProfScope ps(x.prof, PF_BARRIER);
    return team_sync(x.st.bar, x.st.status, x.G, x.b, x.gen, x.st.diag, x.P.spin_limit, x.P.fault_barrier);
}

// Publish this CTA's partial reduction of `count` entries and synchronise the
// team. Large teams add a second stage: CTA b sums slice b of the entries over
// all partials into the team's reduced buffer, then a second barrier; small
// teams let every CTA sum the partials directly (reduce_into).
__device__ inline bool publish_sync(Ctx& x, int count) {
    acc_publish(x, count);
    if (!tsync(x)) return false;
    if (x.G <= kDirectReduceMax) {
        x.red_mode = 0;
        return true;
    }
    {
        ProfScope ps(x.prof, PF_REDUCE);
        const int per = (count + x.G - 1) / x.G;
        const int e0 = x.b * per, e1 = min(count, e0 + per);
        for (int e = e0 + threadIdx.x; e < e1; e += NT) {
            double acc = 0.0;
            for (int g = 0; g < x.G; ++g) acc += ldcg(part_base(x, g) + e);
            x.st.red[e] = acc;
        }
    }
    x.red_mode = 1;
    return tsync(x);
}

// ---- phase A: (pending) second dose half-step, boundary inflow, first dose
// half-step, X[bnd,:] = 0.  Own cells only; no reduction.
// Inflow cell of the RK4 integrator's two-layer boundary condition
// (SolverCSD.jl:679-695): the second layer takes the PsiBeam value of the
// first layer's coordinates, and the x-sides (written last) win at corners.
// Returns the cell whose spatial factor applies, or -1 off the two rings.
__device__ __forceinline__ int bc2_source(const DevProblem& P, int c) {
    const int i = c / P.ny, j = c - (c / P.ny) * P.ny;
    if (i <= 1) return j;                              // (0, j)
    if (i >= P.nx - 2) return (P.nx - 1) * P.ny + j;   // (nx-1, j)
    if (j <= 1) return i * P.ny;                       // (i, 0)
    if (j >= P.ny - 2) return i * P.ny + P.ny - 1;     // (i, ny-1)
    return -1;
}

__device__ inline void phase_bc_dose(Ctx& x, int n, bool dose2_pending, bool do_bc, bool two_layer = false) {
    const DevProblem& P = x.P;
    SmemLayout* sm = x.sm;
    const int k = x.k;
    const double* S = sm->slot[SL_S];
    double* v = sm->vec;  // S W[0,:]^T
    double* w0 = sm->vec + KM;
    for (int j = threadIdx.x; j < k; j += NT) w0[j] = ldcg(x.st.W + j);
    __syncthreads();
    for (int i = threadIdx.x; i < k; i += NT) {
        double s = 0.0;
        for (int j = 0; j < k; ++j) s = fma(S[i * KM + j], w0[j], s);
        v[i] = s;
    }
    __syncthreads();
    const double dE = P.dE;
    // dose half-steps use csd.S at 1-based n-1 for both the pending second
    // half of step n-1 and the first half of step n (0-based index n-2)
    const double sd = P.stopping[n - 2];
    const double bce = P.bc_energy[n - 2];
    for (int c = x.c0 + threadIdx.x; c < x.c1; c += NT) {
        double xv = 0.0;
        for (int j = 0; j < k; ++j) xv = fma(x.st.X[(size_t)c * KM + j], v[j], xv);
        double* pr = x.psi_in + (size_t)c * QM;
        double dose = x.st.dose[c];
        if (dose2_pending) {
            double u = 0.0;
            for (int kq = 0; kq < P.q; ++kq) u = fma(pr[kq], P.mred[kq], u);
            dose += 0.5 * dE * (xv + u) * sd * P.rinv[c];
        }
        bool bnd = is_bnd(P, c);
        if (do_bc) {
            const int src = two_layer ? bc2_source(P, c) : (bnd ? c : -1);
            if (src >= 0) {
                double bs = bce * P.bc_space[src];
                for (int kq = 0; kq < P.q; ++kq) pr[kq] = bs * P.bc_angle[kq];
            }
            double u = 0.0;
            for (int kq = 0; kq < P.q; ++kq) u = fma(pr[kq], P.mred[kq], u);
            dose += 0.5 * dE * (xv + u) * sd * P.rinv[c];
            if (bnd)
                for (int j = 0; j < k; ++j) x.st.X[(size_t)c * KM + j] = 0.0;
        }
        x.st.dose[c] = dose;
    }
}

// Second-order limited flux of psi/rho at interior cell c (2 <= i < nx-2,
// 2 <= j < ny-2), ordinate kq: solveFlux! (SolverCSD.jl:295-386).
__device__ __forceinline__ double limited_flux_cell(const Ctx& x, int c, int kq) {
    const DevProblem& P = x.P;
    const double* p = x.psi_in + kq;
    auto phi = [&](int cc) { return ldcg(p + (size_t)cc * QM) * P.rinv[cc]; };
    const double ox = P.omega[kq * 3 + 0], oz = P.omega[kq * 3 + 2];
    const int sx = P.ny;
    const double f0 = phi(c);
    const bool px = ox >= 0.0, pz = oz >= 0.0;
    const double ew = titus_lim::axis_diff(px ? phi(c - 2 * sx) : 0.0, phi(c - sx), f0, phi(c + sx),
                                           px ? 0.0 : phi(c + 2 * sx), px);
    const double ns = titus_lim::axis_diff(pz ? phi(c - 2) : 0.0, phi(c - 1), f0, phi(c + 1), pz ? 0.0 : phi(c + 2), pz);
    return __dadd_rn(__dmul_rn(__ddiv_rn(ox, P.dx), ew), __dmul_rn(__ddiv_rn(oz, P.dy), ns));
}

// ---- uncollided sweep for own cells (psi_in -> psi_out). `limited`: the RK4
// integrator's second-order flux on the interior of the two outer rings (the
// reference's flux buffer stays zero on the rings, :648, :707); otherwise the
// first-order upwind flux on every non-boundary cell.
__device__ inline void sweep_cells(Ctx& x, double sigma0, bool limited = false) {
    const DevProblem& P = x.P;
    const double dE = P.dE;
    const double den = 1.0 + dE * sigma0;
    const int q = P.q;
    for (int e = threadIdx.x; e < (x.c1 - x.c0) * q; e += NT) {
        int c = x.c0 + e / q, kq = e - (e / q) * q;
        double pc = ldcg(x.psi_in + (size_t)c * QM + kq);
        double flux = 0.0;
        if (limited) {
            const int i = c / P.ny, j = c - (c / P.ny) * P.ny;
            if (i >= 2 && i < P.nx - 2 && j >= 2 && j < P.ny - 2) flux = limited_flux_cell(x, c, kq);
        } else if (!is_bnd(P, c)) {
            double ox = P.omega[kq * 3 + 0], oz = P.omega[kq * 3 + 2];
            double f0 = pc * P.rinv[c];
            double ew, ns;
            if (ox >= 0.0) ew = f0 - ldcg(x.psi_in + (size_t)(c - P.ny) * QM + kq) * P.rinv[c - P.ny];
            else ew = ldcg(x.psi_in + (size_t)(c + P.ny) * QM + kq) * P.rinv[c + P.ny] - f0;
            if (oz >= 0.0) ns = f0 - ldcg(x.psi_in + (size_t)(c - 1) * QM + kq) * P.rinv[c - 1];
            else ns = ldcg(x.psi_in + (size_t)(c + 1) * QM + kq) * P.rinv[c + 1] - f0;
            flux = (ox / P.dx) * ew + (oz / P.dy) * ns;
        }
        double out = (pc - dE * flux) / den;
        if (kq == 0 && P.restore[c]) out = pc;
        x.psi_out[(size_t)c * QM + kq] = out;
    }
}

// ---- streaming Grams X^T L_d X (own cells) and W^T A_d W (own moments):
// partial layout [G_0..G_{nops-1} | C_0..C_{nops-1}], each k x k. nops = 4:
// L2x/Ax, L2y/Az, L1x/|Ax|, L1y/|Az|; nops = 2: the central pair only.
__device__ inline void stream_grams_partial(Ctx& x, int nops = 4) {
    SmemLayout* sm = x.sm;
    const int k = x.k;
    for (int r0 = x.c0; r0 < x.c1; r0 += TR) {
        int nr = min(TR, x.c1 - r0);
        load_rows(sm->tA, x.st.X, r0, nr, k);
        if (nops == 2) stencil2_tile(x, x.st.X, r0, nr, k, sm->tL);
        else stencil_tile(x, x.st.X, r0, nr, k, sm->tL);
        __syncthreads();
        for (int d = 0; d < nops; ++d) gram_acc(sm->acc, d * k * k, sm->tA, KM, k, sm->tL[d], KM, k, nr);
        __syncthreads();
    }
    for (int r0 = x.m0; r0 < x.m1; r0 += TR) {
        int nr = min(TR, x.m1 - r0);
        load_rows(sm->tA, x.st.W, r0, nr, k);
        spmm_tile(x, x.st.W, r0, nr, k, sm->tL, nops);
        __syncthreads();
        for (int d = 0; d < nops; ++d) gram_acc(sm->acc, (nops + d) * k * k, sm->tA, KM, k, sm->tL[d], KM, k, nr);
        __syncthreads();
    }
}

// ---- range finder pass 1 (G1 = (A V)^T (A V)) on one side; A is n x k in global
__device__ inline void rf_pass_b(Ctx& x, const double* A, int r0b, int r1b, const double* V, int k, int off) {
    SmemLayout* sm = x.sm;
    for (int r0 = r0b; r0 < r1b; r0 += TR) {
        int nr = min(TR, r1b - r0);
        load_rows(sm->tA, A, r0, nr, k);
        __syncthreads();
        tile_mm(sm->tO, sm->tA, V, nr, k, k);
        __syncthreads();
        gram_acc(sm->acc, off, sm->tO, KM, k, sm->tO, KM, k, nr);
        __syncthreads();
    }
}
// ---- range finder pass 2: C = A T1 (written to Cbuf), G2 = C^T C
__device__ inline void rf_pass_c(Ctx& x, const double* A, double* Cbuf, int r0b, int r1b, const double* T1, int k,
                          int rho, int off) {
    SmemLayout* sm = x.sm;
    for (int r0 = r0b; r0 < r1b; r0 += TR) {
        int nr = min(TR, r1b - r0);
        load_rows(sm->tA, A, r0, nr, k);
        __syncthreads();
        tile_mm(sm->tO, sm->tA, T1, nr, k, rho);
        __syncthreads();
        store_rows(Cbuf, sm->tO, r0, nr, rho);
        gram_acc(sm->acc, off, sm->tO, KM, rho, sm->tO, KM, rho, nr);
        __syncthreads();
    }
}

// Range-finder pass of the fast path: Y = A R^{-1} by row-wise triangular
// solves (written to Cbuf), G = Y^T Y.
// Rows are processed in chunks of kBigRows over the contiguous tile area
// tA..tO (free during the range finder), one thread per row for the solve.
__device__ inline void rf_pass_solve(Ctx& x, const double* A, double* Cbuf, int r0b, int r1b, const double* R, int k, int off) {
    SmemLayout* sm = x.sm;
    double* big = sm->tA;
    for (int r0 = r0b; r0 < r1b; r0 += kBigRows) {
        int nr = min(kBigRows, r1b - r0);
        load_rows(big, A, r0, nr, k);
        __syncthreads();
        tile_rsolve(big, R, nullptr, nr, k);
        __syncthreads();
        store_rows(Cbuf, big, r0, nr, k);
        gram_acc(sm->acc, off, big, KM, k, big, KM, k, nr);
        __syncthreads();
    }
}

// Orthonormal bases of the numerical ranges of A_X (own cells) and A_W (own
// moments), after their Grams G0 were published at partial offsets 0 and
// (doX ? k*k : 0) and the team barrier passed. On return CX/CW hold C and
// slots SL_RIK/SL_RIL the inverse R of its CholQR, so that the basis is
// C R^{-1} (rho columns) followed by the completion vectors.
//  fast path: Cholesky of G0 with ||R||_F ||R^-1||_F < 1e5 certifies full
//    numerical rank; C = A R0^{-1} (row solves), then CholQR of C.
//  rank-revealing path: Jacobi eig of G0 -> V; Gram of A V -> Jacobi -> V2,
//    nu; C = A V V2_J / nu_J with nu_j > tol nu_0; CholQR of C.
// Returns false if the team aborted.
static __device__ __noinline__ bool range_finder(Ctx& x, const double* AX, const double* AW, bool doX, bool doW, int k) {
    SmemLayout* sm = x.sm;
    const double tol = x.P.rank_tol;
    const double kCert = 1e5;
    double cX = 0.0, cW = 0.0;
    if (doX) reduce_into(x, 0, k, k, sm->ja);
    if (doW) reduce_into(x, doX ? k * k : 0, k, k, sm->jv);
    {
        ProfScope ps(x.prof, PF_CHOL);
        dual_chol(doX, sm->ja, sm->slot[SL_RK], sm->slot[SL_RIK], k, &cX, doW, sm->jv, sm->slot[SL_RL],
                  sm->slot[SL_RIL], k, &cW, x.st.status, false);
    }
    const bool fastX = doX && cX < kCert, fastW = doW && cW < kCert;
    const bool slowX = doX && !fastX, slowW = doW && !fastW;
    if (slowX) {
        reduce_into(x, 0, k, k, sm->ja);
        rf_eig0(x, sm->slot[SL_VK], sm->lamK, k);
    }
    if (slowW) {
        reduce_into(x, doX ? k * k : 0, k, k, sm->ja);
        rf_eig0(x, sm->slot[SL_VL], sm->lamL, k);
    }
    // first pass
    {
        ProfScope ps(x.prof, PF_RF_PASSES);
        acc_zero(x, 2 * k * k);
        if (doX) {
            if (fastX) rf_pass_solve(x, AX, x.CX, x.c0, x.c1, sm->slot[SL_RK], k, 0);
            else rf_pass_b(x, AX, x.c0, x.c1, sm->slot[SL_VK], k, 0);
        }
        if (doW) {
            if (fastW) rf_pass_solve(x, AW, x.CW, x.m0, x.m1, sm->slot[SL_RL], k, k * k);
            else rf_pass_b(x, AW, x.m0, x.m1, sm->slot[SL_VL], k, k * k);
        }
    }
    if (!publish_sync(x, 2 * k * k)) return false;
    if (fastX) reduce_into(x, 0, k, k, sm->ja);
    if (fastW) reduce_into(x, k * k, k, k, sm->jv);
    if (fastX || fastW) {
        ProfScope ps(x.prof, PF_CHOL);
        dual_chol(fastX, sm->ja, sm->slot[SL_RK], sm->slot[SL_RIK], k, nullptr, fastW, sm->jv, sm->slot[SL_RL],
                  sm->slot[SL_RIL], k, nullptr, x.st.status, true, x.st.diag, 2, x.cur_n);
    }
    if (fastX) x.rhoK = k;
    if (fastW) x.rhoL = k;
    if (slowX) {
        reduce_into(x, 0, k, k, sm->ja);
        x.rhoK = rf_eig1(x, sm->slot[SL_VK], sm->slot[SL_TK], k, tol);
    }
    if (slowW) {
        reduce_into(x, k * k, k, k, sm->ja);
        x.rhoL = rf_eig1(x, sm->slot[SL_VL], sm->slot[SL_TL], k, tol);
    }
    if (slowX || slowW) {
        {
            ProfScope ps(x.prof, PF_RF_PASSES);
            acc_zero(x, 2 * k * k);
            if (slowX) rf_pass_c(x, AX, x.CX, x.c0, x.c1, sm->slot[SL_TK], k, x.rhoK, 0);
            if (slowW) rf_pass_c(x, AW, x.CW, x.m0, x.m1, sm->slot[SL_TL], k, x.rhoL, k * k);
        }
        if (!publish_sync(x, 2 * k * k)) return false;
        if (slowX) reduce_into(x, 0, x.rhoK, x.rhoK, sm->ja);
        if (slowW) reduce_into(x, k * k, x.rhoL, x.rhoL, sm->jv);
        ProfScope ps(x.prof, PF_CHOL);
        dual_chol(slowX, sm->ja, sm->slot[SL_RK], sm->slot[SL_RIK], x.rhoK, nullptr, slowW, sm->jv,
                  sm->slot[SL_RL], sm->slot[SL_RIL], x.rhoL, nullptr, x.st.status, true, x.st.diag, 3, x.cur_n);
    }
    if (x.b == 0 && threadIdx.x == 0 && x.st.diag) {
        x.st.diag[11] = (doX ? 1 : 0) + (fastX ? 2 : 0) + (doW ? 4 : 0) + (fastW ? 8 : 0);
        x.st.diag[12] = x.rhoK;
        x.st.diag[13] = x.rhoL;
    }
    if (doX && k - x.rhoK > x.P.nxcomp && threadIdx.x == 0) set_status(x.st.status, ST_COMPLETION);
    if (doW) w_complete(x, x.rhoL, k - x.rhoL);
    __syncthreads();
    return true;
}

// small: D = A S B^T (k x k) with scratch
__device__ inline void sm_asbt(double* D, const double* A, const double* S, const double* B, double* tmp, int k) {
    sm_mm(tmp, A, S, k, k, k);
    sm_mmt(D, tmp, B, k, k, k);
}

// ---- RK4 streaming of K and L (SolverCSD.jl:724-758), the RK4 ("HighOrder")
// integrator's replacement of phase C. Four stages with one team barrier after
// each of the first three: the stencils and the sparse P_N products read
// other CTAs' rows of the stage input. Stage 1 works from X and W directly,
// since L2_d (X S) C_d = (L2_d X)(S C_d) and A_d (W S^T) G_d^T = (A_d W)(S^T G_d^T).
// Slots on entry (d = 0: x, 1: y): C0+d = C_d = W^T A_d W, C0+2+d = S C_d,
// G0+d = G_d^T with G_d = X^T L2_d X, G0+2+d = S^T G_d^T.
// K side: f(Y) = -L2x Y C_0 - L2y Y C_1; KUP accumulates as the reference does
// (K + dE k1/6, then += 2 dE k2/6, += 2 dE k3/6, K = KUP + dE k4/6).
// L side: f(Y) = -Ax Y G_0^T - Az Y G_1^T; L + dE (l1 + 2 l2 + 2 l3 + l4)/6.
// On return K and L hold the new K, L and their Grams are published
// (offsets 0 and k*k) for the range finder. Returns false if the team aborted.
static __device__ __noinline__ bool rk4_stream(Ctx& x) {
    SmemLayout* sm = x.sm;
    const int k = x.k;
    const double dE = x.P.dE;
    const double* Sm = sm->slot[SL_S];
    const size_t nK = (size_t)x.P.n * KM, NK = (size_t)x.P.N * KM;
    double* KUP = x.st.Y;
    double* Ya = x.st.Y + nK;
    double* Yb = x.st.Y + 2 * nK;
    double* LUP = x.st.Z;
    double* La = x.st.Z + NK;
    double* Lb = x.st.Z + 2 * NK;
    for (int s = 1; s <= 4; ++s) {
        // stage inputs: Y2 = K + dE/2 k1 (Ya), Y3 = K + dE/2 k2 (Yb), Y4 = K + dE k3 (Ya)
        const double* Yin = (s == 3) ? Yb : Ya;
        double* Yout = (s == 2) ? Yb : Ya;
        const double* Lin = (s == 3) ? Lb : La;
        double* Lout = (s == 2) ? Lb : La;
        const double cnext = (s == 3) ? dE : 0.5 * dE;
        const double wup = (s == 1 || s == 4) ? 1.0 : 2.0;
        const double* C0 = sm->slot[SL_C0 + (s == 1 ? 2 : 0)];
        const double* C1 = sm->slot[SL_C0 + (s == 1 ? 3 : 1)];
        const double* H0 = sm->slot[SL_G0 + (s == 1 ? 2 : 0)];
        const double* H1 = sm->slot[SL_G0 + (s == 1 ? 3 : 1)];
        if (s == 4) acc_zero(x, 2 * k * k);
        {
            ProfScope ps(x.prof, PF_ROWS_STREAM);
            for (int r0 = x.c0; r0 < x.c1; r0 += TR) {
                const int nr = min(TR, x.c1 - r0);
                if (s == 1) {
                    load_rows(sm->tA, x.st.X, r0, nr, k);
                    stencil2_tile(x, x.st.X, r0, nr, k, sm->tL);
                } else {
                    stencil2_tile(x, Yin, r0, nr, k, sm->tL);
                }
                __syncthreads();
                for (int e = threadIdx.x; e < nr * k; e += NT) {
                    const int r = e / k, j = e - (e / k) * k;
                    const size_t g = (size_t)(r0 + r) * KM + j;
                    double t = 0.0;
                    for (int l = 0; l < k; ++l) t = fma(sm->tL[0][r * KM + l], C0[l * KM + j], t);
                    for (int l = 0; l < k; ++l) t = fma(sm->tL[1][r * KM + l], C1[l * KM + j], t);
                    const double kd = -t;
                    double Kv;
                    if (s == 1) {
                        Kv = 0.0;
                        for (int l = 0; l < k; ++l) Kv = fma(sm->tA[r * KM + l], Sm[l * KM + j], Kv);
                        x.st.K[g] = Kv;
                        KUP[g] = Kv + dE * kd / 6;
                    } else {
                        Kv = ldcg(x.st.K + g);
                        if (s < 4) KUP[g] = ldcg(KUP + g) + wup * dE * kd / 6;
                    }
                    if (s < 4) {
                        Yout[g] = Kv + cnext * kd;
                    } else {
                        const double Kn = ldcg(KUP + g) + dE * kd / 6;
                        sm->tO[r * KM + j] = Kn;
                    }
                }
                __syncthreads();
                if (s == 4) {
                    store_rows(x.st.K, sm->tO, r0, nr, k);
                    gram_acc(sm->acc, 0, sm->tO, KM, k, sm->tO, KM, k, nr);
                    __syncthreads();
                }
            }
            for (int r0 = x.m0; r0 < x.m1; r0 += TR) {
                const int nr = min(TR, x.m1 - r0);
                if (s == 1) {
                    load_rows(sm->tA, x.st.W, r0, nr, k);
                    spmm_tile(x, x.st.W, r0, nr, k, sm->tL, 2);
                } else {
                    spmm_tile(x, Lin, r0, nr, k, sm->tL, 2);
                }
                __syncthreads();
                for (int e = threadIdx.x; e < nr * k; e += NT) {
                    const int r = e / k, j = e - (e / k) * k;
                    const size_t g = (size_t)(r0 + r) * KM + j;
                    double t = 0.0;
                    for (int l = 0; l < k; ++l) t = fma(sm->tL[0][r * KM + l], H0[l * KM + j], t);
                    for (int l = 0; l < k; ++l) t = fma(sm->tL[1][r * KM + l], H1[l * KM + j], t);
                    const double ld = -t;
                    double Lv;
                    if (s == 1) {
                        Lv = 0.0;  // (W S^T)[r][j]
                        for (int l = 0; l < k; ++l) Lv = fma(sm->tA[r * KM + l], Sm[j * KM + l], Lv);
                        x.st.L[g] = Lv;
                        LUP[g] = ld;
                    } else {
                        Lv = ldcg(x.st.L + g);
                        if (s < 4) LUP[g] = ldcg(LUP + g) + wup * ld;
                    }
                    if (s < 4) {
                        Lout[g] = Lv + cnext * ld;
                    } else {
                        sm->tO[r * KM + j] = Lv + dE * (ldcg(LUP + g) + ld) / 6;
                    }
                }
                __syncthreads();
                if (s == 4) {
                    store_rows(x.st.L, sm->tO, r0, nr, k);
                    gram_acc(sm->acc, k * k, sm->tO, KM, k, sm->tO, KM, k, nr);
                    __syncthreads();
                }
            }
        }
        if (s < 4) {
            if (!tsync(x)) return false;
        } else if (!publish_sync(x, 2 * k * k)) {
            return false;
        }
    }
    return true;
}

// S-step of the RK4 integrator in the small space (SolverCSD.jl:776-791):
// f(Y) = -G_0 Y C_0 - G_1 Y C_1 with the new bases' Grams in slots G0+d, C0+d;
// S <- S + dE (s1 + 2 s2 + 2 s3 + s4) / 6. Every CTA computes it redundantly.
__device__ inline void rk4_small_s(Ctx& x) {
    SmemLayout* sm = x.sm;
    const int k = x.k;
    const double dE = x.P.dE;
    double* Sm = sm->slot[SL_S];
    double* Y = sm->slot[SL_P0];
    double* T1 = sm->slot[SL_P0 + 1];
    double* kv = sm->slot[SL_P0 + 2];
    double* sum = sm->slot[SL_P0 + 3];
    double* T2 = sm->slot[SL_VK];
    for (int s = 1; s <= 4; ++s) {
        const double* in = (s == 1) ? Sm : Y;
        sm_mm(T1, sm->slot[SL_G0], in, k, k, k);
        sm_mm(kv, T1, sm->slot[SL_C0], k, k, k);
        sm_mm(T1, sm->slot[SL_G0 + 1], in, k, k, k);
        sm_mm(T2, T1, sm->slot[SL_C0 + 1], k, k, k);
        const double w = (s == 1 || s == 4) ? 1.0 : 2.0;
        const double cn = (s == 3) ? dE : 0.5 * dE;
        for (int e = threadIdx.x; e < k * k; e += NT) {
            const int o = (e / k) * KM + e % k;
            const double d = -kv[o] - T2[o];
            sum[o] = (s == 1) ? d : sum[o] + w * d;
            if (s < 4) Y[o] = Sm[o] + cn * d;
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < k * k; e += NT) {
        const int o = (e / k) * KM + e % k;
        Sm[o] = Sm[o] + dE * sum[o] / 6;
    }
    __syncthreads();
}

// METHOD: 0 = fixed-rank DLR (SolveFirstCollisionSourceDLR), kHighOrder = the
// RK4 variant (SolveFirstCollisionSourceDLRHighOrder, SolverCSD.jl:588-889):
// two-layer inflow, limited second-order sweep, RK4 streaming with the
// central operators; the scattering steps are shared.
constexpr int kHighOrder = 3;

template <int METHOD>
__global__ void __launch_bounds__(NT, 1)
dlr_kernel(DevProblem P, TeamState* states, int G, int n_begin, int n_end, int dose2_pending_in) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SmemLayout* sm = reinterpret_cast<SmemLayout*>(smem_raw);
    if (P.zero_smem) {
        double* z = reinterpret_cast<double*>(smem_raw);
        for (size_t e = threadIdx.x; e < sizeof(SmemLayout) / sizeof(double); e += NT) z[e] = 0.0;
        __syncthreads();
    }
    Ctx x;
    x.P = P;
    x.G = G;
    x.b = blockIdx.x % G;
    x.st = states[blockIdx.x / G];
    x.sm = sm;
    x.prof = (blockIdx.x == 0) ? P.prof : nullptr;
    x.red_mode = 0;
    x.gen = 0;
    x.parity = 0;
    x.rhoK = x.rhoL = 0;
    x.cur_n = 0;
    prof_begin(x.prof);
    ProfScope ps_total(x.prof, PF_TOTAL);
    x.c0 = (int)((long long)x.b * P.n / G);
    x.c1 = (int)((long long)(x.b + 1) * P.n / G);
    x.m0 = (int)((long long)x.b * P.N / G);
    x.m1 = (int)((long long)(x.b + 1) * P.N / G);
    x.CX = x.st.K;          // C of the X-side range finder reuses K after K is consumed
    x.CW = x.st.L + (size_t)P.N * KM;  // W side: second half of the L allocation
    const int k = ldcg(x.st.info + 0);
    x.k = k;
    int psi_idx = ldcg(x.st.info + 2);
    for (int e = threadIdx.x; e < KK; e += NT) sm->slot[SL_S][e] = ldcg(x.st.S + e);
    __syncthreads();
    bool pending = dose2_pending_in != 0;
    int steps = 0;
    constexpr bool HO = (METHOD == kHighOrder);   // RK4 integrator (SolveFirstCollisionSourceDLRHighOrder)
    constexpr int nops = HO ? 2 : 4;               // streaming operators: central pair, or with Roe terms
    double* Sm = sm->slot[SL_S];
    for (int n = n_begin; n <= n_end; ++n) {
        x.psi_in = psi_idx ? x.st.psi1 : x.st.psi0;
        x.psi_out = psi_idx ? x.st.psi0 : x.st.psi1;
        const double* sig = P.sigma + (size_t)(n - 1) * (P.npn + 1);
        x.cur_n = n;
        const double dE = P.dE;
        // ---------------- phase A
        phase_bc_dose(x, n, pending, true, HO);
        pending = false;
        if (!tsync(x)) return;
        // ---------------- phase B: sweep + streaming Grams
        sweep_cells(x, sig[0], HO);
        const bool stream = (n > 2);
        if (stream) {
            acc_zero(x, 2 * nops * k * k);
            stream_grams_partial(x, nops);
            if (!publish_sync(x, 2 * nops * k * k)) return;
        } else if (!tsync(x)) {
            return;
        }
        psi_idx ^= 1;
        x.psi_in = psi_idx ? x.st.psi1 : x.st.psi0;  // swept psi
        if (stream && HO) {
            // C0+d = C_d, C0+2+d = S C_d, G0+d = G_d^T, G0+2+d = S^T G_d^T (d = 0, 1)
            for (int d = 0; d < 2; ++d) {
                reduce_into(x, d * k * k, k, k, sm->slot[SL_P0]);
                reduce_into(x, (2 + d) * k * k, k, k, sm->slot[SL_C0 + d]);
                sm_mm(sm->slot[SL_C0 + 2 + d], Sm, sm->slot[SL_C0 + d], k, k, k);
                for (int e = threadIdx.x; e < k * k; e += NT) {
                    int i = e / k, j = e % k;
                    sm->slot[SL_G0 + d][i * KM + j] = sm->slot[SL_P0][j * KM + i];
                    double s2 = 0.0;
                    for (int l = 0; l < k; ++l) s2 = fma(Sm[l * KM + i], sm->slot[SL_P0][j * KM + l], s2);
                    sm->slot[SL_G0 + 2 + d][i * KM + j] = s2;
                }
                __syncthreads();
            }
            // ---------------- phase C (RK4): K and L streaming updates
            if (!rk4_stream(x)) return;
        }
        if (stream && !HO) {
            for (int d = 0; d < 4; ++d) {
                reduce_into(x, d * k * k, k, k, sm->slot[SL_G0 + d]);
                reduce_into(x, (4 + d) * k * k, k, k, sm->slot[SL_C0 + d]);
            }
            // SC_d = S C_d -> slot C_d ; SG_d = S^T G_d^T -> slot G_d
            for (int d = 0; d < 4; ++d) {
                sm_mm(sm->slot[SL_P0], Sm, sm->slot[SL_C0 + d], k, k, k);
                sm_copy(sm->slot[SL_C0 + d], sm->slot[SL_P0], k, k);
                // (S^T G^T)[i][j] = sum_l S[l][i] G[j][l]
                for (int e = threadIdx.x; e < k * k; e += NT) {
                    int i = e / k, j = e % k;
                    double s = 0.0;
                    for (int l = 0; l < k; ++l) s = fma(Sm[l * KM + i], sm->slot[SL_G0 + d][j * KM + l], s);
                    sm->slot[SL_P0][i * KM + j] = s;
                }
                __syncthreads();
                sm_copy(sm->slot[SL_G0 + d], sm->slot[SL_P0], k, k);
            }
            // ---------------- phase C: K and L streaming updates
            acc_zero(x, 2 * k * k);
            for (int r0 = x.c0; r0 < x.c1; r0 += TR) {
                int nr = min(TR, x.c1 - r0);
                load_rows(sm->tA, x.st.X, r0, nr, k);
                stencil_tile(x, x.st.X, r0, nr, k, sm->tL);
                __syncthreads();
                for (int e = threadIdx.x; e < nr * k; e += NT) {
                    int r = e / k, j = e % k;
                    double s = 0.0;
                    for (int l = 0; l < k; ++l) s = fma(sm->tA[r * KM + l], Sm[l * KM + j], s);
                    double t = 0.0;
                    for (int d = 0; d < 4; ++d)
                        for (int l = 0; l < k; ++l) t = fma(sm->tL[d][r * KM + l], sm->slot[SL_C0 + d][l * KM + j], t);
                    sm->tO[r * KM + j] = s - dE * t;
                }
                __syncthreads();
                store_rows(x.st.K, sm->tO, r0, nr, k);
                gram_acc(sm->acc, 0, sm->tO, KM, k, sm->tO, KM, k, nr);
                __syncthreads();
            }
            for (int r0 = x.m0; r0 < x.m1; r0 += TR) {
                int nr = min(TR, x.m1 - r0);
                load_rows(sm->tA, x.st.W, r0, nr, k);
                spmm_tile(x, x.st.W, r0, nr, k, sm->tL);
                __syncthreads();
                for (int e = threadIdx.x; e < nr * k; e += NT) {
                    int r = e / k, j = e % k;
                    double s = 0.0;  // (W S^T)[r][j] = sum_l W[r][l] S[j][l]
                    for (int l = 0; l < k; ++l) s = fma(sm->tA[r * KM + l], Sm[j * KM + l], s);
                    double t = 0.0;
                    for (int d = 0; d < 4; ++d)
                        for (int l = 0; l < k; ++l) t = fma(sm->tL[d][r * KM + l], sm->slot[SL_G0 + d][l * KM + j], t);
                    sm->tO[r * KM + j] = s - dE * t;
                }
                __syncthreads();
                store_rows(x.st.L, sm->tO, r0, nr, k);
                gram_acc(sm->acc, k * k, sm->tO, KM, k, sm->tO, KM, k, nr);
                __syncthreads();
            }
            if (!publish_sync(x, 2 * k * k)) return;
        }
        if (stream) {
            // ---------------- phases D, E: range finders of K and L
            if (!range_finder(x, x.st.K, x.st.L, true, true, k)) return;
            // ---------------- phase F: new bases, MUp = XNew^T X, NUp = WNew^T W
            acc_zero(x, 2 * k * k);
            for (int r0 = x.c0; r0 < x.c1; r0 += TR) {
                int nr = min(TR, x.c1 - r0);
                x_basis_tile(x, r0, nr, x.rhoK, k, sm->tO);
                load_rows(sm->tA, x.st.X, r0, nr, k);
                __syncthreads();
                gram_acc(sm->acc, 0, sm->tO, KM, k, sm->tA, KM, k, nr);
                __syncthreads();
                store_rows(x.st.X, sm->tO, r0, nr, k);
                __syncthreads();
            }
            for (int r0 = x.m0; r0 < x.m1; r0 += TR) {
                int nr = min(TR, x.m1 - r0);
                w_basis_tile(x, r0, nr, x.rhoL, k - x.rhoL, sm->tO);
                load_rows(sm->tA, x.st.W, r0, nr, k);
                __syncthreads();
                gram_acc(sm->acc, k * k, sm->tO, KM, k, sm->tA, KM, k, nr);
                __syncthreads();
                store_rows(x.st.W, sm->tO, r0, nr, k);
                __syncthreads();
            }
            if (!publish_sync(x, 2 * k * k)) return;
            reduce_into(x, 0, k, k, sm->slot[SL_M]);
            reduce_into(x, k * k, k, k, sm->slot[SL_N]);
            // S1 = MUp S NUp^T -> slot S
            sm_asbt(sm->slot[SL_P0 + 1], sm->slot[SL_M], Sm, sm->slot[SL_N], sm->slot[SL_P0], k);
            sm_copy(Sm, sm->slot[SL_P0 + 1], k, k);
            // ---------------- phase G: S-step Grams with the new X, W
            acc_zero(x, 2 * nops * k * k);
            stream_grams_partial(x, nops);
            if (!publish_sync(x, 2 * nops * k * k)) return;
        }
        if (stream && HO) {
            for (int d = 0; d < 2; ++d) {
                reduce_into(x, d * k * k, k, k, sm->slot[SL_G0 + d]);
                reduce_into(x, (2 + d) * k * k, k, k, sm->slot[SL_C0 + d]);
            }
            rk4_small_s(x);
        }
        if (stream && !HO) {
            for (int d = 0; d < 4; ++d) {
                reduce_into(x, d * k * k, k, k, sm->slot[SL_G0 + d]);
                reduce_into(x, (4 + d) * k * k, k, k, sm->slot[SL_C0 + d]);
            }
            // S = S1 - dE sum_d G_d S1 C_d
            sm_zero(sm->slot[SL_P0 + 2], k, k);
            for (int d = 0; d < 4; ++d) {
                sm_mm(sm->slot[SL_P0], sm->slot[SL_G0 + d], Sm, k, k, k);
                sm_mm(sm->slot[SL_P0 + 1], sm->slot[SL_P0], sm->slot[SL_C0 + d], k, k, k);
                for (int e = threadIdx.x; e < k * k; e += NT)
                    sm->slot[SL_P0 + 2][(e / k) * KM + e % k] += sm->slot[SL_P0 + 1][(e / k) * KM + e % k];
                __syncthreads();
            }
            for (int e = threadIdx.x; e < k * k; e += NT) Sm[(e / k) * KM + e % k] -= dE * sm->slot[SL_P0 + 2][(e / k) * KM + e % k];
            __syncthreads();
        }
        // ---------------- phase H: out-scattering L (W side); P = psi^T X (X side, X[bnd]=0)
        acc_zero(x, k * k + P.q * k);
        for (int c = x.c0 + threadIdx.x; c < x.c1; c += NT)
            if (is_bnd(P, c))
                for (int j = 0; j < k; ++j) x.st.X[(size_t)c * KM + j] = 0.0;
        __syncthreads();
        for (int r0 = x.m0; r0 < x.m1; r0 += TR) {
            int nr = min(TR, x.m1 - r0);
            load_rows(sm->tA, x.st.W, r0, nr, k);
            __syncthreads();
            for (int e = threadIdx.x; e < nr * k; e += NT) {
                int r = e / k, j = e % k;
                double s = 0.0;
                for (int l = 0; l < k; ++l) s = fma(sm->tA[r * KM + l], Sm[j * KM + l], s);
                int m = r0 + r;
                double D = sig[0] - sig[P.lof[m]];
                sm->tO[r * KM + j] = s / (1.0 + dE * D);
            }
            __syncthreads();
            store_rows(x.st.L, sm->tO, r0, nr, k);
            gram_acc(sm->acc, 0, sm->tO, KM, k, sm->tO, KM, k, nr);
            __syncthreads();
        }
        for (int r0 = x.c0; r0 < x.c1; r0 += TR) {
            int nr = min(TR, x.c1 - r0);
            load_rows(sm->tA, x.st.X, r0, nr, k);
            for (int e = threadIdx.x; e < nr * P.q; e += NT)
                sm->tP[(e / P.q) * QM + e % P.q] = ldcg(x.psi_in + (size_t)(r0 + e / P.q) * QM + e % P.q);
            __syncthreads();
            gram_acc(sm->acc, k * k, sm->tP, QM, P.q, sm->tA, KM, k, nr);
            __syncthreads();
        }
        if (!publish_sync(x, k * k + P.q * k)) return;
        // keep P = psi^T X (q x k) in slot P0+3 ; G0 of L into ja via range_finder
        reduce_into(x, k * k, P.q, k, sm->slot[SL_P0 + 3]);
        // range finder expects G0 of the W side at partial offset 0 when doX is false
        if (!range_finder(x, nullptr, x.st.L, false, true, k)) return;
        // ---------------- phase K: W = basis(L); S = L^T W ; Bk = MRed^T diag(Dvec) W
        acc_zero(x, k * k + P.q * k);
        for (int r0 = x.m0; r0 < x.m1; r0 += TR) {
            int nr = min(TR, x.m1 - r0);
            w_basis_tile(x, r0, nr, x.rhoL, k - x.rhoL, sm->tO);
            load_rows(sm->tA, x.st.L, r0, nr, k);
            for (int e = threadIdx.x; e < nr * P.q; e += NT) {
                int r = e / P.q, kq = e % P.q;
                int m = r0 + r;
                sm->tP[r * QM + kq] = P.mred[(size_t)m * P.q + kq] * sig[P.lof[m]];
            }
            __syncthreads();
            gram_acc(sm->acc, 0, sm->tA, KM, k, sm->tO, KM, k, nr);
            gram_acc(sm->acc, k * k, sm->tP, QM, P.q, sm->tO, KM, k, nr);
            __syncthreads();
            store_rows(x.st.W, sm->tO, r0, nr, k);
            __syncthreads();
        }
        if (!publish_sync(x, k * k + P.q * k)) return;
        reduce_into(x, 0, k, k, Sm);
        reduce_into(x, k * k, P.q, k, sm->slot[SL_P0 + 2]);  // Bk (q x k)
        // ---------------- phase L: in-scattering K (X side) and L (W side)
        acc_zero(x, 2 * k * k);
        for (int r0 = x.c0; r0 < x.c1; r0 += TR) {
            int nr = min(TR, x.c1 - r0);
            load_rows(sm->tA, x.st.X, r0, nr, k);
            for (int e = threadIdx.x; e < nr * P.q; e += NT)
                sm->tP[(e / P.q) * QM + e % P.q] = ldcg(x.psi_in + (size_t)(r0 + e / P.q) * QM + e % P.q);
            __syncthreads();
            for (int e = threadIdx.x; e < nr * k; e += NT) {
                int r = e / k, j = e % k;
                double s = 0.0;
                if (!is_bnd(P, r0 + r)) {
                    for (int l = 0; l < k; ++l) s = fma(sm->tA[r * KM + l], Sm[l * KM + j], s);
                    double t = 0.0;
                    for (int kq = 0; kq < P.q; ++kq) t = fma(sm->tP[r * QM + kq], sm->slot[SL_P0 + 2][kq * KM + j], t);
                    s += dE * t;
                }
                sm->tO[r * KM + j] = s;
            }
            __syncthreads();
            store_rows(x.st.K, sm->tO, r0, nr, k);
            gram_acc(sm->acc, 0, sm->tO, KM, k, sm->tO, KM, k, nr);
            __syncthreads();
        }
        for (int r0 = x.m0; r0 < x.m1; r0 += TR) {
            int nr = min(TR, x.m1 - r0);
            load_rows(sm->tA, x.st.W, r0, nr, k);
            __syncthreads();
            for (int e = threadIdx.x; e < nr * k; e += NT) {
                int r = e / k, j = e % k;
                int m = r0 + r;
                double s = 0.0;
                for (int l = 0; l < k; ++l) s = fma(sm->tA[r * KM + l], Sm[j * KM + l], s);
                double t = 0.0;  // (MRed P)[m][j]
                for (int kq = 0; kq < P.q; ++kq) t = fma(P.mred[(size_t)m * P.q + kq], sm->slot[SL_P0 + 3][kq * KM + j], t);
                sm->tO[r * KM + j] = s + dE * sig[P.lof[m]] * t;
            }
            __syncthreads();
            store_rows(x.st.L, sm->tO, r0, nr, k);
            gram_acc(sm->acc, k * k, sm->tO, KM, k, sm->tO, KM, k, nr);
            __syncthreads();
        }
        if (!publish_sync(x, 2 * k * k)) return;
        if (!range_finder(x, x.st.K, x.st.L, true, true, k)) return;
        // ---------------- phase O: new bases; MUp, X^T psi, NUp, MRed^T D W
        const int offM = 0, offXp = k * k, offN = k * k + k * P.q, offB = 2 * k * k + k * P.q;
        acc_zero(x, 2 * k * k + 2 * k * P.q);
        for (int r0 = x.c0; r0 < x.c1; r0 += TR) {
            int nr = min(TR, x.c1 - r0);
            x_basis_tile(x, r0, nr, x.rhoK, k, sm->tO);
            load_rows(sm->tA, x.st.X, r0, nr, k);
            for (int e = threadIdx.x; e < nr * P.q; e += NT)
                sm->tP[(e / P.q) * QM + e % P.q] = ldcg(x.psi_in + (size_t)(r0 + e / P.q) * QM + e % P.q);
            __syncthreads();
            gram_acc(sm->acc, offM, sm->tO, KM, k, sm->tA, KM, k, nr);
            gram_acc(sm->acc, offXp, sm->tO, KM, k, sm->tP, QM, P.q, nr);
            __syncthreads();
            store_rows(x.st.X, sm->tO, r0, nr, k);
            __syncthreads();
        }
        for (int r0 = x.m0; r0 < x.m1; r0 += TR) {
            int nr = min(TR, x.m1 - r0);
            w_basis_tile(x, r0, nr, x.rhoL, k - x.rhoL, sm->tO);
            load_rows(sm->tA, x.st.W, r0, nr, k);
            for (int e = threadIdx.x; e < nr * P.q; e += NT) {
                int r = e / P.q, kq = e % P.q;
                int m = r0 + r;
                sm->tP[r * QM + kq] = P.mred[(size_t)m * P.q + kq] * sig[P.lof[m]];
            }
            __syncthreads();
            gram_acc(sm->acc, offN, sm->tO, KM, k, sm->tA, KM, k, nr);
            gram_acc(sm->acc, offB, sm->tP, QM, P.q, sm->tO, KM, k, nr);
            __syncthreads();
            store_rows(x.st.W, sm->tO, r0, nr, k);
            __syncthreads();
        }
        if (!publish_sync(x, 2 * k * k + 2 * k * P.q)) return;
        reduce_into(x, offM, k, k, sm->slot[SL_M]);
        reduce_into(x, offXp, k, P.q, sm->slot[SL_P0 + 3]);   // XNew^T psi (k x q)
        reduce_into(x, offN, k, k, sm->slot[SL_N]);
        reduce_into(x, offB, P.q, k, sm->slot[SL_P0 + 2]);    // MRed^T D WNew (q x k)
        // S = MUp S NUp^T + dE (X^T psi)(MRed^T D W)
        sm_asbt(sm->slot[SL_P0 + 1], sm->slot[SL_M], Sm, sm->slot[SL_N], sm->slot[SL_P0], k);
        sm_mm(sm->slot[SL_P0], sm->slot[SL_P0 + 3], sm->slot[SL_P0 + 2], k, P.q, k);
        for (int e = threadIdx.x; e < k * k; e += NT) {
            int i = e / k, j = e % k;
            Sm[i * KM + j] = sm->slot[SL_P0 + 1][i * KM + j] + dE * sm->slot[SL_P0][i * KM + j];
        }
        __syncthreads();
        pending = true;
        ++steps;
        if (x.b == 0 && threadIdx.x == 0 && x.st.rank_hist) x.st.rank_hist[n - 1] = k;
    }
    // final second dose half-step of the last step (phase A without inflow)
    if (pending && n_end >= n_begin) {
        x.psi_in = psi_idx ? x.st.psi1 : x.st.psi0;
        // the last step's index is n_end: its dose weight is csd.S[n_end] (1-based)
        phase_bc_dose(x, n_end + 1, true, false);
    }
    if (x.b == 0) {
        for (int e = threadIdx.x; e < KK; e += NT) x.st.S[e] = Sm[e];
        if (threadIdx.x == 0) {
            x.st.info[0] = k;
            x.st.info[1] = steps;
            x.st.info[2] = psi_idx;
            x.st.info[3] = n_end + 1;
        }
    }
}

}  // namespace titus
