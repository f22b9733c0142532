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
    ~titus_pn_state() {
        if (exec) cudaGraphExecDestroy(exec);
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
