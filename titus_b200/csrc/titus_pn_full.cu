// Full-rank P_N first-collision solver (SolveFirstCollisionSource,
// code/SolverCSD.jl:465-586) on the GPU.
//
// State: the collided flux u (n x N, row-major, row i*ny + j), the reduced
// ordinates psi (n x QM, ordinate fastest) and the dose. One energy step n is
// three kernels on one stream:
//   pn_psi_kernel      beam inflow at energy[n] (csd.S[n-1]), upwind sweep of
//                      the interior cells, psi <- (psi - dE flux) / (1 + dE sigma_0)
//                      (:517-545); the inflow values are formed where they are read;
//   pn_moments_kernel  W_d = u A_d for the four P_N operators (Ax, Az, |Ax|, |Az|):
//                      a CTA holds the rows of CB cells transposed in shared memory
//                      and each thread forms one column m of one operator, so every
//                      nonzero of A_d is read once per CB cells;
//   pn_stream_kernel   uTilde = u - dE (L2x W_0 + L2y W_1 + L1x W_2 + L1y W_3) with
//                      the matrix-free density-weighted stencils (stencils.jl:12-130),
//                      collision (1 + dE D)^{-1}, in-scattering dE Dvec (MReduced psi),
//                      boundary rows zero, and the dose with csd.SMid (:548-575).
// The whole sweep is captured once into a CUDA graph and launched as one unit.
// Bytes per step (FP64): pn_moments reads u and writes W (5 n N words),
// pn_stream reads u, W (4 n N, neighbours from L2) and writes u' (6 n N words).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "titus_handle.h"

using namespace titus;
using titus_host::fail;

namespace {

constexpr int PN_CB = 8;      // cells per CTA of pn_moments_kernel
constexpr int PN_NT = 256;    // threads per CTA

struct PnArgs {
    int nx, ny, n, N, q, npn, nE;
    double dx, dy, dE;
    const double* rinv;       // n
    const double* stopping;   // nE
    const double* smid;       // nE - 1
    const double* bc_energy;  // nE
    const double* bc_space;   // n
    const double* bc_angle;   // q
    const double* omega;      // q x 3
    const double* mred;       // N x q
    const double* sigma;      // nE x (npn+1)
    const int32_t* lof;       // N
    const int32_t* tp[4];     // CSR of A_d^T (rows = output moments)
    const int32_t* ti[4];
    const double* tv[4];
};

__device__ __forceinline__ bool pn_bnd(const PnArgs& a, int c) {
    const int i = c / a.ny, j = c - (c / a.ny) * a.ny;
    return i == 0 || j == 0 || i == a.nx - 1 || j == a.ny - 1;
}

// psi_out = (psi - dE flux) / (1 + dE sigma_0) for every cell and ordinate; the
// boundary cells hold the inflow PsiBeam(Omega_k, energy[n], x, y, n-1) and
// have zero flux (the reference's flux buffer is written on interior cells only).
__global__ void __launch_bounds__(PN_NT) pn_psi_kernel(PnArgs a, int n, const double* __restrict__ psi_in,
                                                       double* __restrict__ psi_out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.n * a.q) return;
    const int c = e / a.q, k = e - (e / a.q) * a.q;
    // energy factor at energy[n] with csd.S[n-1]: bc_energy holds scale exp(-sE (E0-E_k)^2) S_k rho_min
    const double bcf = a.bc_energy[n - 1] / a.stopping[n - 1] * a.stopping[n - 2];
    const double ang = a.bc_angle[k];
    auto val = [&](int cc) -> double {
        return pn_bnd(a, cc) ? bcf * a.bc_space[cc] * ang : psi_in[(size_t)cc * QM + k];
    };
    const double pc = val(c);
    double flux = 0.0;
    if (!pn_bnd(a, c)) {
        const double ox = a.omega[k * 3 + 0], oz = a.omega[k * 3 + 2];
        const double ew = ox >= 0.0 ? pc - val(c - a.ny) : val(c + a.ny) - pc;
        const double ns = oz >= 0.0 ? pc - val(c - 1) : val(c + 1) - pc;
        flux = (ox / a.dx) * ew + (oz / a.dy) * ns;
    }
    const double sig0 = a.sigma[(size_t)(n - 1) * (a.npn + 1)];
    psi_out[(size_t)c * QM + k] = (pc - a.dE * flux) / (1.0 + a.dE * sig0);
}

// W[d][c][m] = sum_p u[c][p] A_d[p][m] (A_d^T row m in CSR order).
__global__ void __launch_bounds__(PN_NT) pn_moments_kernel(PnArgs a, const double* __restrict__ u,
                                                           double* __restrict__ W) {
    extern __shared__ __align__(16) double us[];   // N x PN_CB, cells fastest
    const int c0 = blockIdx.x * PN_CB;
    const int nc = min(PN_CB, a.n - c0);
    const int N = a.N;
    for (int e = threadIdx.x; e < PN_CB * N; e += blockDim.x) {
        const int c = e / N, p = e - (e / N) * N;
        us[p * PN_CB + c] = c < nc ? __ldg(u + (size_t)(c0 + c) * N + p) : 0.0;
    }
    __syncthreads();
    for (int pm = threadIdx.x; pm < 4 * N; pm += blockDim.x) {
        const int d = pm / N, m = pm - (pm / N) * N;
        double acc[PN_CB];
#pragma unroll
        for (int c = 0; c < PN_CB; ++c) acc[c] = 0.0;
        const int q1 = __ldg(a.tp[d] + m + 1);
        for (int q = __ldg(a.tp[d] + m); q < q1; ++q) {
            const double v = __ldg(a.tv[d] + q);
            const double2* up = reinterpret_cast<const double2*>(us + __ldg(a.ti[d] + q) * PN_CB);
#pragma unroll
            for (int c2 = 0; c2 < PN_CB / 2; ++c2) {
                const double2 x = up[c2];
                acc[2 * c2] = fma(v, x.x, acc[2 * c2]);
                acc[2 * c2 + 1] = fma(v, x.y, acc[2 * c2 + 1]);
            }
        }
#pragma unroll
        for (int c = 0; c < PN_CB; ++c)
            if (c < nc) W[((size_t)d * a.n + c0 + c) * N + m] = acc[c];
    }
}

// u_out[c][m]: streaming from W, collision, in-scattering; the dose on the m = 0 thread.
__global__ void __launch_bounds__(PN_NT) pn_stream_kernel(PnArgs a, int n, const double* __restrict__ u,
                                                          const double* __restrict__ W,
                                                          const double* __restrict__ psi, double* __restrict__ u_out,
                                                          double* __restrict__ dose) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int N = a.N;
    if (e >= (size_t)a.n * N) return;
    const int c = (int)(e / N), m = (int)(e - (e / N) * N);
    if (pn_bnd(a, c)) {
        u_out[e] = 0.0;
        return;
    }
    const double dE = a.dE;
    const int xm = c - a.ny, xp = c + a.ny, ym = c - 1, yp = c + 1;
    auto w = [&](int d, int cc) { return W[((size_t)d * a.n + cc) * N + m]; };
    // stencil entries as the reference's sparse rows (columns in increasing order)
    const double hx = -1.0 / 2.0 / a.dx, hy = -1.0 / 2.0 / a.dy;
    const double l2x = (hx * a.rinv[xm]) * w(0, xm) + (-hx * a.rinv[xp]) * w(0, xp);
    const double l2y = (hy * a.rinv[ym]) * w(1, ym) + (-hy * a.rinv[yp]) * w(1, yp);
    const double l1x = (hx * a.rinv[xm]) * w(2, xm) + (2.0 / 2.0 / a.dx * a.rinv[c]) * w(2, c) +
                       (hx * a.rinv[xp]) * w(2, xp);
    const double l1y = (hy * a.rinv[ym]) * w(3, ym) + (2.0 / 2.0 / a.dy * a.rinv[c]) * w(3, c) +
                       (hy * a.rinv[yp]) * w(3, yp);
    double ut = u[e];
    ut = ut - dE * l2x;
    ut = ut - dE * l2y;
    ut = ut - dE * l1x;
    ut = ut - dE * l1y;
    const double* sg = a.sigma + (size_t)(n - 1) * (a.npn + 1);
    const double dv = sg[a.lof[m]];
    const double D = sg[0] - dv;
    const double* pr = psi + (size_t)c * QM;
    double src = 0.0;
    for (int k = 0; k < a.q; ++k) src = fma(a.mred[(size_t)m * a.q + k], pr[k], src);
    const double un = (ut + dE * dv * src) / (1.0 + dE * D);
    u_out[e] = un;
    if (m == 0) {
        double unc = 0.0;
        for (int k = 0; k < a.q; ++k) unc = fma(pr[k], a.mred[k], unc);
        const double half = (n == 2 || n == a.nE) ? 2.0 : 1.0;
        dose[c] += dE * (un + unc) * a.smid[n - 2] * a.rinv[c] / half;
    }
}

}  // namespace

struct titus_pn_state {
    double *u[2] = {nullptr, nullptr}, *W = nullptr, *psi[2] = {nullptr, nullptr}, *dose = nullptr;
    int32_t* tp[4] = {};
    int32_t* ti[4] = {};
    double* tv[4] = {};
    int cur_u = 0, cur_psi = 0;
    int steps_done = 0;
    bool have_result = false;
    cudaStream_t cap = nullptr;   // capture stream (graphs are recorded here, launched on the caller's)
    cudaGraphExec_t exec = nullptr;   // the last sweep's graph, reused while n_end is the same
    int exec_n_end = -1;
    std::vector<void*> allocs;
    // adjoint workspace (titus_dose_adjoint), sized for (checkpoints, segment length)
    double *ck_u = nullptr, *ck_psi = nullptr, *seg = nullptr, *lam[2] = {nullptr, nullptr}, *Y = nullptr,
           *psib[2] = {nullptr, nullptr}, *pw = nullptr, *g = nullptr, *grad = nullptr, *gprof = nullptr,
           *dose_scr = nullptr, *wt = nullptr, *tg = nullptr;
    int adj_nck = -1, adj_k = -1;
    std::vector<void*> adj_allocs;
    void adj_release() {
        for (void* p : adj_allocs) cudaFree(p);
        adj_allocs.clear();
        adj_nck = adj_k = -1;
    }
    ~titus_pn_state() {
        if (exec) cudaGraphExecDestroy(exec);
        adj_release();
        for (void* p : allocs) cudaFree(p);
        if (cap) cudaStreamDestroy(cap);
    }
};

namespace {

template <class T>
int pn_alloc(titus_pn_state* st, T** p, size_t count, const T* host = nullptr) {
    int rc = titus_host::upload(p, host, count);
    if (rc == TITUS_OK && *p) st->allocs.push_back((void*)*p);
    return rc;
}

// Device state and the CSR of each A_d^T, built on first use from the uploaded CSR of A_d.
int pn_ensure(titus_solver* s) {
    if (s->pn) return TITUS_OK;
    if (!s->smid) return fail(TITUS_ERR_ARG, "the full-rank P_N solver needs problem->stopping_mid (csd.SMid)");
    auto* st = new titus_pn_state();
    const size_t nN = (size_t)s->n * s->N;
    int rc;
    if ((rc = pn_alloc(st, &st->u[0], nN)) || (rc = pn_alloc(st, &st->u[1], nN)) ||
        (rc = pn_alloc(st, &st->W, 4 * nN)) || (rc = pn_alloc(st, &st->psi[0], (size_t)s->n * QM)) ||
        (rc = pn_alloc(st, &st->psi[1], (size_t)s->n * QM)) || (rc = pn_alloc(st, &st->dose, (size_t)s->n))) {
        delete st;
        return rc;
    }
    const int N = s->N;
    for (int d = 0; d < 4; ++d) {
        std::vector<int32_t> rp(N + 1);
        cudaError_t e = cudaMemcpy(rp.data(), s->P.op[d].rowptr, (N + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost);
        const int nnz = rp[N];
        std::vector<int32_t> ci(nnz);
        std::vector<double> v(nnz);
        if (e == cudaSuccess && nnz)
            e = cudaMemcpy(ci.data(), s->P.op[d].col, nnz * sizeof(int32_t), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && nnz) e = cudaMemcpy(v.data(), s->P.op[d].val, nnz * sizeof(double), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            delete st;
            return fail(TITUS_ERR_CUDA, "operator download: %s", cudaGetErrorString(e));
        }
        // transpose: row m of A^T lists (p, A[p][m]) in increasing p
        std::vector<int32_t> tp(N + 1, 0), ti(nnz);
        std::vector<double> tv(nnz);
        for (int q = 0; q < nnz; ++q) ++tp[ci[q] + 1];
        for (int m = 0; m < N; ++m) tp[m + 1] += tp[m];
        std::vector<int32_t> pos(tp.begin(), tp.end() - 1);
        for (int p = 0; p < N; ++p)
            for (int q = rp[p]; q < rp[p + 1]; ++q) {
                const int dst = pos[ci[q]]++;
                ti[dst] = p;
                tv[dst] = v[q];
            }
        if ((rc = pn_alloc(st, &st->tp[d], (size_t)N + 1, tp.data())) ||
            (rc = pn_alloc(st, &st->ti[d], (size_t)std::max(nnz, 1), ti.data())) ||
            (rc = pn_alloc(st, &st->tv[d], (size_t)std::max(nnz, 1), tv.data()))) {
            delete st;
            return rc;
        }
    }
    cudaError_t e = cudaStreamCreateWithFlags(&st->cap, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(pn_moments_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(PN_CB * N * sizeof(double)));
    if (e != cudaSuccess) {
        delete st;
        return fail(TITUS_ERR_CUDA, "full-rank solver set-up: %s", cudaGetErrorString(e));
    }
    s->pn = st;
    return TITUS_OK;
}

PnArgs pn_args(const titus_solver* s, const titus_pn_state* st) {
    const DevProblem& P = s->P;
    PnArgs a{};
    a.nx = P.nx;
    a.ny = P.ny;
    a.n = P.n;
    a.N = P.N;
    a.q = P.q;
    a.npn = P.npn;
    a.nE = P.nE;
    a.dx = P.dx;
    a.dy = P.dy;
    a.dE = P.dE;
    a.rinv = P.rinv;
    a.stopping = P.stopping;
    a.smid = s->smid;
    a.bc_energy = P.bc_energy;
    a.bc_space = P.bc_space;
    a.bc_angle = P.bc_angle;
    a.omega = P.omega;
    a.mred = P.mred;
    a.sigma = P.sigma;
    a.lof = P.lof;
    for (int d = 0; d < 4; ++d) {
        a.tp[d] = st->tp[d];
        a.ti[d] = st->ti[d];
        a.tv[d] = st->tv[d];
    }
    return a;
}

}  // namespace

void titus_host::pn_free(titus_solver* s) {
    delete s->pn;
    s->pn = nullptr;
}

extern "C" int titus_pn_full_solve_device(titus_solver_t* s, const titus_options_t* opt, void* stream_) {
    if (!s) return fail(TITUS_ERR_ARG, "solver is NULL");
    if (opt && opt->precision != TITUS_PRECISION_FP64)
        return fail(TITUS_ERR_ARG, "the full-rank P_N solver runs in FP64 only (precision %d)", opt->precision);
    if (s->nz) return titus_host::pn3_solve_device(s, opt, (cudaStream_t)stream_);
    int rc = pn_ensure(s);
    if (rc) return rc;
    titus_pn_state* st = s->pn;
    cudaStream_t stream = (cudaStream_t)stream_;
    const size_t nN = (size_t)s->n * s->N;
    int n_end = s->nE;
    if (opt && opt->max_steps > 0) n_end = std::min(n_end, 1 + opt->max_steps);
    // initial state: u = 0, psi = 0 (SetupIC is zero for the beam problems), dose = 0
    CK(cudaMemsetAsync(st->u[0], 0, nN * sizeof(double), stream));
    CK(cudaMemsetAsync(st->psi[0], 0, (size_t)s->n * QM * sizeof(double), stream));
    CK(cudaMemsetAsync(st->dose, 0, (size_t)s->n * sizeof(double), stream));
    // record the sweep into a graph on the capture stream (once per n_end), then
    // launch it on `stream`
    const PnArgs a = pn_args(s, st);
    const int cu_end = (n_end - 1) & 1, cp_end = (n_end - 1) & 1;
    if (st->exec && st->exec_n_end == n_end) {
        CK(cudaGraphLaunch(st->exec, stream));
        st->cur_u = cu_end;
        st->cur_psi = cp_end;
        st->steps_done = n_end - 1;
        st->have_result = true;
        return TITUS_OK;
    }
    if (st->exec) {
        CK(cudaStreamSynchronize(stream));   // the old graph may still be running
        cudaGraphExecDestroy(st->exec);
        st->exec = nullptr;
        st->exec_n_end = -1;
    }
    CK(cudaStreamBeginCapture(st->cap, cudaStreamCaptureModeThreadLocal));
    int cu = 0, cp = 0;
    const int gpsi = (int)((s->n * (size_t)s->q + PN_NT - 1) / PN_NT);
    const int gmom = (s->n + PN_CB - 1) / PN_CB;
    const int gst = (int)((nN + PN_NT - 1) / PN_NT);
    const size_t smem = PN_CB * (size_t)s->N * sizeof(double);
    for (int n = 2; n <= n_end; ++n) {
        pn_psi_kernel<<<gpsi, PN_NT, 0, st->cap>>>(a, n, st->psi[cp], st->psi[cp ^ 1]);
        pn_moments_kernel<<<gmom, PN_NT, smem, st->cap>>>(a, st->u[cu], st->W);
        pn_stream_kernel<<<gst, PN_NT, 0, st->cap>>>(a, n, st->u[cu], st->W, st->psi[cp ^ 1], st->u[cu ^ 1], st->dose);
        cu ^= 1;
        cp ^= 1;
    }
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(st->cap, &graph);
    if (e != cudaSuccess) return fail(TITUS_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(TITUS_ERR_CUDA, "graph instantiation: %s", cudaGetErrorString(e));
    st->exec = exec;
    st->exec_n_end = n_end;
    e = cudaGraphLaunch(exec, stream);
    if (e != cudaSuccess) return fail(TITUS_ERR_CUDA, "graph launch: %s", cudaGetErrorString(e));
    st->cur_u = cu;
    st->cur_psi = cp;
    st->steps_done = n_end - 1;
    st->have_result = true;
    return TITUS_OK;
}

extern "C" int titus_pn_full_fetch(titus_solver_t* s, double* u_out, double* dose_out, double* psi_out) {
    if (!s) return fail(TITUS_ERR_ARG, "solver is NULL");
    if (s->nz) return titus_host::pn3_fetch(s, u_out, dose_out, psi_out);
    if (!s->pn || !s->pn->have_result) return fail(TITUS_ERR_ARG, "no full-rank solve has run on this handle");
    titus_pn_state* st = s->pn;
    CK(cudaDeviceSynchronize());
    CK(cudaGetLastError());
    if (u_out) CK(cudaMemcpy(u_out, st->u[st->cur_u], (size_t)s->n * s->N * sizeof(double), cudaMemcpyDeviceToHost));
    if (dose_out) CK(cudaMemcpy(dose_out, st->dose, (size_t)s->n * sizeof(double), cudaMemcpyDeviceToHost));
    if (psi_out)
        CK(cudaMemcpy2D(psi_out, s->q * sizeof(double), st->psi[st->cur_psi], QM * sizeof(double),
                        s->q * sizeof(double), s->n, cudaMemcpyDeviceToHost));
    return TITUS_OK;
}

extern "C" int titus_pn_full_solve(titus_solver_t* s, const titus_options_t* opt, double* u_out, double* dose_out,
                                   double* psi_out) {
    int rc = titus_pn_full_solve_device(s, opt, nullptr);
    if (rc) return rc;
    return titus_pn_full_fetch(s, u_out, dose_out, psi_out);
}

// ---------------------------------------------------------------------------
// Adjoint of the full-rank sweep (titus_dose_adjoint): gradients of a dose
// objective J with respect to the cell densities and to PsiBeam's spatial
// profile, by the exact transpose of the explicit step above, run from the
// last energy step back to the first. Per backward step n (mu = P_int lambda /
// (1 + dE D) with g c_n / rho added to moment 0, c_n the dose weight):
//   pn_moments_kernel  V_d = u_{n-1} A_d from the recomputed forward state;
//   pn_adj_y_kernel    Y_d = L_d^T mu, the transposed matrix-free stencils
//                      (every entry of L_d carries 1/rho of its column cell);
//   pn_adj_psi_w_kernel  w = (psibar + P_int (dE (mu Dvec) MReduced + g c_n / rho
//                      MReduced[0,:])) / (1 + dE sigma_0), the adjoint of psi';
//   pn_adj_lam_kernel  lambda' = mu - dE sum_d Y_d A_d^T (rows of A_d, CB cells
//                      per CTA as in pn_moments_kernel) and, in the same pass,
//                      dJ/drho_c += dE / rho_c sum_{d,m} Y_d[c,m] V_d[c,m]
//                      (reduced over the CTA in a fixed order);
//   pn_adj_psi_bc_kernel  psibar_bc = w - dE F^T w, the transposed upwind sweep;
//                      on boundary cells it is the inflow's sensitivity
//                      (dJ/dprofile += psibar_bc . inflow factor), elsewhere it
//                      carries to the previous step.
// Checkpoints: (u, psi) entering every k-th step are kept from one forward
// pass; each segment of k steps is recomputed from its checkpoint into a
// k-slot buffer of u states and then run backward.
// ---------------------------------------------------------------------------
namespace {

struct AdjOps {
    const int32_t* rp[4];   // CSR of A_d (rows = output moment m of Y_d A_d^T)
    const int32_t* ci[4];
    const double* cv[4];
};

struct StepConst {
    const double* sg;   // sigma_l at energy[n]
    double cn;          // dose weight dE SMid[n-1] / (1 + (n == 2 or n == nE))
};

__device__ __forceinline__ StepConst step_const(const PnArgs& a, int n) {
    StepConst k;
    k.sg = a.sigma + (size_t)(n - 1) * (a.npn + 1);
    const double half = (n == 2 || n == a.nE) ? 2.0 : 1.0;
    k.cn = a.dE * a.smid[n - 2] / half;
    return k;
}

// mu[c][m]; zero outside the grid and on boundary cells
__device__ __forceinline__ double adj_mu(const PnArgs& a, const StepConst& k, const double* __restrict__ lam,
                                         const double* __restrict__ g, int c, int m) {
    if (c < 0 || c >= a.n || pn_bnd(a, c)) return 0.0;
    double l = lam[(size_t)c * a.N + m];
    if (m == 0) l += g[c] * k.cn * a.rinv[c];
    const double D = k.sg[0] - k.sg[a.lof[m]];
    return l / (1.0 + a.dE * D);
}

__global__ void __launch_bounds__(PN_NT) pn_adj_y_kernel(PnArgs a, int n, const double* __restrict__ lam,
                                                         const double* __restrict__ g, double* __restrict__ Y) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int N = a.N;
    if (e >= (size_t)a.n * N) return;
    const int c = (int)(e / N), m = (int)(e - (e / N) * N);
    const StepConst k = step_const(a, n);
    const double mc = adj_mu(a, k, lam, g, c, m);
    const double mxm = adj_mu(a, k, lam, g, c - a.ny, m), mxp = adj_mu(a, k, lam, g, c + a.ny, m);
    const double mym = adj_mu(a, k, lam, g, c - 1, m), myp = adj_mu(a, k, lam, g, c + 1, m);
    const double hx = -1.0 / 2.0 / a.dx, hy = -1.0 / 2.0 / a.dy, ri = a.rinv[c];
    const size_t nN = (size_t)a.n * N;
    Y[e] = ri * (hx * mxp - hx * mxm);
    Y[nN + e] = ri * (hy * myp - hy * mym);
    Y[2 * nN + e] = ri * (hx * mxp + (2.0 / 2.0 / a.dx) * mc + hx * mxm);
    Y[3 * nN + e] = ri * (hy * myp + (2.0 / 2.0 / a.dy) * mc + hy * mym);
}

__global__ void __launch_bounds__(PN_NT) pn_adj_psi_w_kernel(PnArgs a, int n, const double* __restrict__ lam,
                                                             const double* __restrict__ g,
                                                             const double* __restrict__ psib, double* __restrict__ w) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.n * a.q) return;
    const int c = e / a.q, kk = e - (e / a.q) * a.q;
    const StepConst k = step_const(a, n);
    double v = psib[(size_t)c * QM + kk];
    if (!pn_bnd(a, c)) {
        double s = 0.0;
        for (int m = 0; m < a.N; ++m) {
            const double dv = k.sg[a.lof[m]];
            s = fma(adj_mu(a, k, lam, g, c, m) * dv, a.mred[(size_t)m * a.q + kk], s);
        }
        v += a.dE * s + g[c] * k.cn * a.rinv[c] * a.mred[kk];
    }
    w[(size_t)c * QM + kk] = v / (1.0 + a.dE * k.sg[0]);
}

template <int CB>
__global__ void __launch_bounds__(PN_NT) pn_adj_lam_kernel(PnArgs a, AdjOps ops, int n, const double* __restrict__ lam,
                                                           const double* __restrict__ g, const double* __restrict__ Y,
                                                           const double* __restrict__ V, double* __restrict__ lam_out,
                                                           double* __restrict__ grad) {
    extern __shared__ __align__(16) double ys[];   // [d][k][cell] : 4 x N x CB
    __shared__ double red[PN_NT / 32][CB];
    const int c0 = blockIdx.x * CB;
    const int nc = min(CB, a.n - c0);
    const int N = a.N;
    const size_t nN = (size_t)a.n * N;
    for (int e = threadIdx.x; e < 4 * CB * N; e += blockDim.x) {
        const int d = e / (CB * N), rem = e - d * (CB * N);
        const int c = rem / N, kq = rem - c * N;
        ys[((size_t)d * N + kq) * CB + c] = c < nc ? Y[d * nN + (size_t)(c0 + c) * N + kq] : 0.0;
    }
    __syncthreads();
    const StepConst k = step_const(a, n);
    double gacc[CB];
#pragma unroll
    for (int c = 0; c < CB; ++c) gacc[c] = 0.0;
    for (int m = threadIdx.x; m < N; m += blockDim.x) {
        double acc[CB];
#pragma unroll
        for (int c = 0; c < CB; ++c) acc[c] = 0.0;
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const int q1 = __ldg(ops.rp[d] + m + 1);
            for (int q = __ldg(ops.rp[d] + m); q < q1; ++q) {
                const double v = __ldg(ops.cv[d] + q);
                const double* yp = ys + ((size_t)d * N + __ldg(ops.ci[d] + q)) * CB;
#pragma unroll
                for (int c = 0; c < CB; ++c) acc[c] = fma(v, yp[c], acc[c]);
            }
#pragma unroll
            for (int c = 0; c < CB; ++c)
                if (c < nc) gacc[c] = fma(ys[((size_t)d * N + m) * CB + c], V[d * nN + (size_t)(c0 + c) * N + m], gacc[c]);
        }
#pragma unroll
        for (int c = 0; c < CB; ++c)
            if (c < nc) lam_out[(size_t)(c0 + c) * N + m] = adj_mu(a, k, lam, g, c0 + c, m) - a.dE * acc[c];
    }
    // per-cell sums over the CTA: warp butterflies, then the warps in order
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < CB; ++c) {
        double v = gacc[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[wid][c] = v;
    }
    __syncthreads();
    if (threadIdx.x < nc) {
        double t = 0.0;
        for (int w2 = 0; w2 < PN_NT / 32; ++w2) t += red[w2][threadIdx.x];
        const int c = c0 + threadIdx.x;
        grad[c] += a.dE * a.rinv[c] * t;
    }
}

__global__ void __launch_bounds__(PN_NT) pn_adj_psi_bc_kernel(PnArgs a, int n, const double* __restrict__ w,
                                                              double* __restrict__ psib_out,
                                                              double* __restrict__ gprof) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.n) return;
    const bool bnd = pn_bnd(a, c);
    const double bcf = a.bc_energy[n - 1] / a.stopping[n - 1] * a.stopping[n - 2];
    auto W = [&](int cc, int kk) -> double { return (cc >= 0 && cc < a.n) ? w[(size_t)cc * QM + kk] : 0.0; };
    double acc = 0.0;
    for (int kk = 0; kk < a.q; ++kk) {
        const double ox = a.omega[kk * 3 + 0], oz = a.omega[kk * 3 + 2];
        const double ax = ox / a.dx, az = oz / a.dy;
        const double wc = W(c, kk);
        // transpose of the upwind differences: the cell's own row and the rows
        // of the downwind neighbours that difference against it
        double ft = (ox >= 0.0 ? ax : -ax) * wc + (oz >= 0.0 ? az : -az) * wc;
        ft += ox >= 0.0 ? -ax * W(c + a.ny, kk) : ax * W(c - a.ny, kk);
        ft += oz >= 0.0 ? -az * W(c + 1, kk) : az * W(c - 1, kk);
        const double pbc = wc - a.dE * ft;
        if (bnd) {
            acc = fma(pbc, bcf * a.bc_angle[kk], acc);
            psib_out[(size_t)c * QM + kk] = 0.0;
        } else {
            psib_out[(size_t)c * QM + kk] = pbc;
        }
    }
    if (bnd) gprof[c] += acc;
}

__global__ void pn_adj_objective_kernel(int n, const double* __restrict__ dose, const double* __restrict__ wt,
                                        const double* __restrict__ tg, double* __restrict__ g) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const double wc = wt ? wt[c] : 1.0;
    const double tc = tg ? tg[c] : 0.0;
    g[c] = 2.0 * wc * (dose[c] - tc);
}

// explicit 1/rho of the dose: dJ/drho_c -= g_c dose_c / rho_c
__global__ void pn_adj_final_kernel(int n, const double* __restrict__ rinv, const double* __restrict__ dose,
                                    const double* __restrict__ g, double* __restrict__ grad) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    grad[c] += -g[c] * dose[c] * rinv[c];
}

int adj_ensure(titus_solver* s, titus_pn_state* st, int nck, int k) {
    if (st->adj_nck == nck && st->adj_k == k) return TITUS_OK;
    st->adj_release();
    const size_t nN = (size_t)s->n * s->N, nQ = (size_t)s->n * QM, n = (size_t)s->n;
    auto al = [&](double** p, size_t count) {
        int rc = titus_host::upload(p, (const double*)nullptr, count);
        if (rc == TITUS_OK && *p) st->adj_allocs.push_back((void*)*p);
        return rc;
    };
    int rc;
    if ((rc = al(&st->ck_u, (size_t)nck * nN)) || (rc = al(&st->ck_psi, (size_t)nck * nQ)) ||
        (rc = al(&st->seg, (size_t)k * nN)) || (rc = al(&st->lam[0], nN)) || (rc = al(&st->lam[1], nN)) ||
        (rc = al(&st->Y, 4 * nN)) || (rc = al(&st->psib[0], nQ)) || (rc = al(&st->psib[1], nQ)) ||
        (rc = al(&st->pw, nQ)) || (rc = al(&st->g, n)) || (rc = al(&st->grad, n)) || (rc = al(&st->gprof, n)) ||
        (rc = al(&st->dose_scr, n)) || (rc = al(&st->wt, n)) || (rc = al(&st->tg, n))) {
        st->adj_release();
        return rc;
    }
    st->adj_nck = nck;
    st->adj_k = k;
    return TITUS_OK;
}

}  // namespace

extern "C" int titus_dose_adjoint(titus_solver_t* s, int32_t method, const titus_options_t* opt, const double* weight,
                                  const double* target, const double* dj_ddose, int32_t checkpoint_every,
                                  double* objective_out, double* dose_out, double* grad_density,
                                  double* grad_profile) {
    if (!s) return fail(TITUS_ERR_ARG, "solver is NULL");
    if (s->nz) return fail(TITUS_ERR_ARG, "titus_dose_adjoint: the adjoint runs the reference's 2D problems");
    if (method != TITUS_PN_FULL)
        return fail(TITUS_ERR_ARG, "titus_dose_adjoint: method %d has no adjoint (TITUS_PN_FULL = %d)", method,
                    TITUS_PN_FULL);
    if (opt && opt->precision != TITUS_PRECISION_FP64)
        return fail(TITUS_ERR_ARG, "the adjoint runs in FP64 only (precision %d)", opt->precision);
    if (checkpoint_every < 0) return fail(TITUS_ERR_ARG, "checkpoint_every must be >= 0 (0 = about sqrt(steps))");
    int rc = pn_ensure(s);
    if (rc) return rc;
    titus_pn_state* st = s->pn;
    const size_t n = (size_t)s->n, nN = n * s->N, nQ = n * QM;
    int n_end = s->nE;
    if (opt && opt->max_steps > 0) n_end = std::min(n_end, 1 + opt->max_steps);
    const int steps = n_end - 1;
    if (steps < 1) return fail(TITUS_ERR_ARG, "the energy grid has no step");
    int k = checkpoint_every > 0 ? checkpoint_every : (int)std::ceil(std::sqrt((double)steps));
    k = std::max(1, std::min(k, steps));
    const int nck = (steps + k - 1) / k;
    const int CB = (4 * (size_t)s->N * 8 * sizeof(double) <= 200 * 1024) ? 8 : 4;
    const size_t lam_smem = 4 * (size_t)s->N * CB * sizeof(double);
    if (lam_smem > 200 * 1024)
        return fail(TITUS_ERR_LIMIT, "titus_dose_adjoint: N = %d moments exceed the staged tile (N <= %d)", s->N,
                    (int)(200 * 1024 / (4 * 4 * sizeof(double))));
    if ((rc = adj_ensure(s, st, nck, k))) return rc;
    // objective weights / target or a given dJ/d(dose)
    if (dj_ddose) {
        CK(cudaMemcpy(st->g, dj_ddose, n * sizeof(double), cudaMemcpyHostToDevice));
    } else {
        if (weight) CK(cudaMemcpy(st->wt, weight, n * sizeof(double), cudaMemcpyHostToDevice));
        if (target) CK(cudaMemcpy(st->tg, target, n * sizeof(double), cudaMemcpyHostToDevice));
    }
    CK(cudaFuncSetAttribute(pn_adj_lam_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lam_smem));
    CK(cudaFuncSetAttribute(pn_adj_lam_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lam_smem));
    const PnArgs a = pn_args(s, st);
    AdjOps ops{};
    for (int d = 0; d < 4; ++d) {
        ops.rp[d] = s->P.op[d].rowptr;
        ops.ci[d] = s->P.op[d].col;
        ops.cv[d] = s->P.op[d].val;
    }
    cudaStream_t strm = nullptr;
    const int gpsi = (int)((n * (size_t)s->q + PN_NT - 1) / PN_NT);
    const int gmom = (s->n + PN_CB - 1) / PN_CB;
    const int gst = (int)((nN + PN_NT - 1) / PN_NT);
    const int gcell = (int)((n + PN_NT - 1) / PN_NT);
    const int glam = (s->n + CB - 1) / CB;
    const size_t msm = PN_CB * (size_t)s->N * sizeof(double);
    // forward pass with checkpoints of (u, psi) entering steps 2, 2 + k, ...
    CK(cudaMemsetAsync(st->u[0], 0, nN * sizeof(double), strm));
    CK(cudaMemsetAsync(st->psi[0], 0, nQ * sizeof(double), strm));
    CK(cudaMemsetAsync(st->dose, 0, n * sizeof(double), strm));
    int cu = 0, cp = 0;
    for (int nn = 2; nn <= n_end; ++nn) {
        if ((nn - 2) % k == 0) {
            const size_t i = (size_t)(nn - 2) / k;
            CK(cudaMemcpyAsync(st->ck_u + i * nN, st->u[cu], nN * sizeof(double), cudaMemcpyDeviceToDevice, strm));
            CK(cudaMemcpyAsync(st->ck_psi + i * nQ, st->psi[cp], nQ * sizeof(double), cudaMemcpyDeviceToDevice, strm));
        }
        pn_psi_kernel<<<gpsi, PN_NT, 0, strm>>>(a, nn, st->psi[cp], st->psi[cp ^ 1]);
        pn_moments_kernel<<<gmom, PN_NT, msm, strm>>>(a, st->u[cu], st->W);
        pn_stream_kernel<<<gst, PN_NT, 0, strm>>>(a, nn, st->u[cu], st->W, st->psi[cp ^ 1], st->u[cu ^ 1], st->dose);
        cu ^= 1;
        cp ^= 1;
    }
    CK(cudaGetLastError());
    // dJ/d(dose)
    if (!dj_ddose)
        pn_adj_objective_kernel<<<gcell, PN_NT, 0, strm>>>(s->n, st->dose, weight ? st->wt : nullptr,
                                                           target ? st->tg : nullptr, st->g);
    CK(cudaMemsetAsync(st->lam[0], 0, nN * sizeof(double), strm));
    CK(cudaMemsetAsync(st->psib[0], 0, nQ * sizeof(double), strm));
    CK(cudaMemsetAsync(st->grad, 0, n * sizeof(double), strm));
    CK(cudaMemsetAsync(st->gprof, 0, n * sizeof(double), strm));
    int cl = 0, cb = 0;
    for (int i = nck - 1; i >= 0; --i) {
        const int a0 = 2 + i * k, b0 = std::min(a0 + k - 1, n_end);
        auto useg = [&](int j) { return j == 0 ? st->ck_u + (size_t)i * nN : st->seg + (size_t)j * nN; };
        // recompute u entering steps a0 + 1 .. b0 (the dose goes to scratch)
        CK(cudaMemcpyAsync(st->psi[0], st->ck_psi + (size_t)i * nQ, nQ * sizeof(double), cudaMemcpyDeviceToDevice,
                           strm));
        int rp = 0;
        for (int j = 0; j + a0 < b0; ++j) {
            const int nn = a0 + j;
            pn_psi_kernel<<<gpsi, PN_NT, 0, strm>>>(a, nn, st->psi[rp], st->psi[rp ^ 1]);
            pn_moments_kernel<<<gmom, PN_NT, msm, strm>>>(a, useg(j), st->W);
            pn_stream_kernel<<<gst, PN_NT, 0, strm>>>(a, nn, useg(j), st->W, st->psi[rp ^ 1], useg(j + 1),
                                                      st->dose_scr);
            rp ^= 1;
        }
        // backward through the segment
        for (int nn = b0; nn >= a0; --nn) {
            pn_moments_kernel<<<gmom, PN_NT, msm, strm>>>(a, useg(nn - a0), st->W);
            pn_adj_y_kernel<<<gst, PN_NT, 0, strm>>>(a, nn, st->lam[cl], st->g, st->Y);
            pn_adj_psi_w_kernel<<<gpsi, PN_NT, 0, strm>>>(a, nn, st->lam[cl], st->g, st->psib[cb], st->pw);
            if (CB == 8)
                pn_adj_lam_kernel<8><<<glam, PN_NT, lam_smem, strm>>>(a, ops, nn, st->lam[cl], st->g, st->Y, st->W,
                                                                     st->lam[cl ^ 1], st->grad);
            else
                pn_adj_lam_kernel<4><<<glam, PN_NT, lam_smem, strm>>>(a, ops, nn, st->lam[cl], st->g, st->Y, st->W,
                                                                     st->lam[cl ^ 1], st->grad);
            pn_adj_psi_bc_kernel<<<gcell, PN_NT, 0, strm>>>(a, nn, st->pw, st->psib[cb ^ 1], st->gprof);
            cl ^= 1;
            cb ^= 1;
        }
        CK(cudaGetLastError());
    }
    pn_adj_final_kernel<<<gcell, PN_NT, 0, strm>>>(s->n, a.rinv, st->dose, st->g, st->grad);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(strm));
    std::vector<double> dose(n), gvec(n);
    CK(cudaMemcpy(dose.data(), st->dose, n * sizeof(double), cudaMemcpyDeviceToHost));
    if (dose_out) std::copy(dose.begin(), dose.end(), dose_out);
    if (grad_density) CK(cudaMemcpy(grad_density, st->grad, n * sizeof(double), cudaMemcpyDeviceToHost));
    if (grad_profile) CK(cudaMemcpy(grad_profile, st->gprof, n * sizeof(double), cudaMemcpyDeviceToHost));
    if (objective_out) {
        double J = 0.0;
        if (dj_ddose) {
            J = std::nan("");
        } else {
            for (size_t c = 0; c < n; ++c) {
                const double wc = weight ? weight[c] : 1.0, tc = target ? target[c] : 0.0;
                J += wc * (dose[c] - tc) * (dose[c] - tc);
            }
        }
        *objective_out = J;
    }
    // the forward state buffers now hold the last recomputation, not a solve's result
    st->have_result = false;
    return TITUS_OK;
}
