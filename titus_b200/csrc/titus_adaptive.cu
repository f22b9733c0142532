// Host side of the rank-adaptive integrators (TITUS_PARALLEL_ADAPTIVE,
// TITUS_BUG_ADAPTIVE, TITUS_PARALLEL_REJECTION): device state, initial factors,
// launch and result copy.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <string>
#include <type_traits>
#include <vector>

#include "titus_handle.h"
#include "dlr_adaptive.cuh"

// Host entry names: the 3D compilation (titus_adaptive3d.cu) appends _3d.
#ifndef TITUS_WIDE_HOST
#define TITUS_WIDE_HOST(name) name
#endif

using namespace titus;
using namespace titus::TITUS_WIDE_NS;
using titus_host::fail;

namespace {

using KernelFn = void (*)(DevProblem, WideState*, int, int, int, int);

// The energy-loop kernel of `method`. A template, so that the 3D build (BUG
// only) never instantiates the other integrators' kernels.
template <bool ThreeD>
KernelFn kernel_for(int method) {
    if constexpr (ThreeD) {
        return adaptive_kernel<TITUS_BUG_ADAPTIVE>;
    } else {
        if (method == TITUS_PARALLEL_ADAPTIVE) return adaptive_kernel<TITUS_PARALLEL_ADAPTIVE>;
        if (method == TITUS_PARALLEL_REJECTION) return adaptive_kernel<TITUS_PARALLEL_REJECTION>;
        return adaptive_kernel<TITUS_BUG_ADAPTIVE>;
    }
}

int ensure_state(titus_solver* s) {
    if (s->d_wst) return TITUS_OK;
    WideState& w = s->wst;
    const int n = s->n, N = s->N, G = s->num_sms;
    int rc;
    w.hist_cap = 4 * s->nE + 64;
    if ((rc = s->walloc(&w.X, (size_t)n * KA)) || (rc = s->walloc(&w.W, (size_t)N * KA)) ||
        (rc = s->walloc(&w.K, (size_t)n * RA)) || (rc = s->walloc(&w.KP, (size_t)n * RA)) ||
        (rc = s->walloc(&w.CX, (size_t)n * RA)) || (rc = s->walloc(&w.L, (size_t)N * RA)) ||
        (rc = s->walloc(&w.LP, (size_t)N * RA)) || (rc = s->walloc(&w.CW, (size_t)N * RA)) ||
        (rc = s->walloc(&w.psi0, (size_t)n * QW)) || (rc = s->walloc(&w.psi1, (size_t)n * QW)) ||
        (rc = s->walloc(&w.dose, (size_t)n)) || (rc = s->walloc(&w.S, (size_t)KA * KA)) ||
        (rc = s->walloc(&w.part, (size_t)2 * G * PMAXW)) || (rc = s->walloc(&w.red, (size_t)2 * PMAXW)) ||
        (rc = s->walloc(&w.scr, (size_t)G * SCRW)) || (rc = s->walloc(&w.bar, (size_t)G + 1)) ||
        (rc = s->walloc(&w.status, 1)) || (rc = s->walloc(&w.info, 8)) || (rc = s->walloc(&w.diag, 16)) ||
        (rc = s->walloc(&w.tvar, 1)) || (rc = s->walloc(&w.rank_hist, (size_t)w.hist_cap)) ||
        (rc = s->walloc(&w.time_hist, (size_t)w.hist_cap)) || (rc = s->walloc(&w.eta_hist, (size_t)w.hist_cap)) ||
        (rc = s->walloc(&w.bound_hist, (size_t)w.hist_cap)) || (rc = s->walloc(&w.X0, (size_t)n * RA)) ||
        (rc = s->walloc(&w.W0, (size_t)N * RA)))
        return rc;
    if ((rc = s->walloc(&s->d_wst, 1))) return rc;
    CK(cudaMemcpy(s->d_wst, &w, sizeof(WideState), cudaMemcpyHostToDevice));
    for (int method : {TITUS_PARALLEL_ADAPTIVE, TITUS_BUG_ADAPTIVE, TITUS_PARALLEL_REJECTION})
        CK(cudaFuncSetAttribute(kernel_for<kThreeD>(method), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(WSmem)));
    return TITUS_OK;
}

// Initial factors (SolverCSD.jl:1728-1760, :2013-2050): r0 = floor(settings.r / 2)
// identity columns, X's boundary rows zeroed, S = 0.
__global__ void wide_init_kernel(WideState* states, int n, int N, int nx, int ny, int r0, int hist_cap) {
    WideState st = states[0];
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < r0; j += gridDim.x * blockDim.x) {
        if (j < n) {
            const int i = j / ny, jj = j % ny;
            // 3D: the first r0 < nx ny rows lie in the z = 0 face
            const bool bnd = kThreeD || (i == 0 || jj == 0 || i == nx - 1 || jj == ny - 1);
            st.X[(size_t)j * KA + j] = bnd ? 0.0 : 1.0;
        }
        if (j < N) st.W[(size_t)j * KA + j] = 1.0;
    }
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < hist_cap; e += gridDim.x * blockDim.x) {
        st.rank_hist[e] = -1;
        st.time_hist[e] = 0.0;
        st.eta_hist[e] = 0.0;
        st.bound_hist[e] = 0.0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st.info[0] = r0;
        st.info[1] = 0;
        st.info[2] = 0;
        st.info[3] = 2;
        st.info[4] = 0;
        st.tvar[0] = 0.0;
    }
}

__global__ void wide_mark_rank0(WideState* states, int r0) {
    // the parallel integrator's rVec starts with r0 in every column (:1731); index 0 is never overwritten
    if (threadIdx.x == 0) states[0].rank_hist[0] = r0;
}

int init_state(titus_solver* s, int r0, int method, cudaStream_t stream) {
    WideState& w = s->wst;
    const int n = s->n, N = s->N;
    CK(cudaMemsetAsync(w.X, 0, (size_t)n * KA * sizeof(double), stream));
    CK(cudaMemsetAsync(w.W, 0, (size_t)N * KA * sizeof(double), stream));
    CK(cudaMemsetAsync(w.S, 0, (size_t)KA * KA * sizeof(double), stream));
    CK(cudaMemsetAsync(w.psi0, 0, (size_t)n * QW * sizeof(double), stream));
    CK(cudaMemsetAsync(w.psi1, 0, (size_t)n * QW * sizeof(double), stream));
    CK(cudaMemsetAsync(w.dose, 0, (size_t)n * sizeof(double), stream));
    wide_init_kernel<<<4, 256, 0, stream>>>(s->d_wst, n, N, s->P.nx, s->P.ny, r0, w.hist_cap);
    CK(cudaGetLastError());
    if (method == TITUS_PARALLEL_ADAPTIVE) {
        wide_mark_rank0<<<1, 32, 0, stream>>>(s->d_wst, r0);
        CK(cudaGetLastError());
    }
    return TITUS_OK;
}

int launch(titus_solver* s, int method, const titus_options_t* opt, int n_begin, int n_end, int max_iters,
           cudaStream_t stream) {
    int G = (opt && opt->team_ctas > 0) ? opt->team_ctas : std::min(s->num_sms, 64);
    G = std::max(1, std::min(G, s->num_sms));
    int per_sm = 0;
    const KernelFn kfun = kernel_for<kThreeD>(method);
    auto kern = (void*)kfun;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfun, TITUS_WIDE_NS::NT, sizeof(WSmem)));
    if (per_sm < 1) return fail(TITUS_ERR_CUDA, "adaptive kernel does not fit on an SM (smem %zu)", sizeof(WSmem));
    G = std::min(G, per_sm * s->num_sms);
    DevProblem P = s->P;
    if (opt && opt->rank_tol > 0) P.rank_tol = opt->rank_tol;
    P.prof = nullptr;
    P.zero_smem = 0;
    P.precision = opt ? opt->precision : TITUS_PRECISION_FP64;
    s->take_debug_hooks(P);
    if (opt && opt->profile) {
        CK(cudaMemsetAsync(s->prof, 0, PF_SLOTS * sizeof(unsigned long long), stream));
        P.prof = s->prof;
    }
    WideState& w = s->wst;
    CK(cudaMemsetAsync(w.bar, 0, (size_t)(s->num_sms + 1) * sizeof(unsigned), stream));
    CK(cudaMemsetAsync(w.status, 0, sizeof(int), stream));
    CK(cudaMemsetAsync(w.diag, 0, 16 * sizeof(double), stream));
    WideState* dst = s->d_wst;
    void* args[] = {&P, &dst, &G, &n_begin, &n_end, &max_iters};
    CK(cudaLaunchCooperativeKernel(kern, dim3(G), dim3(TITUS_WIDE_NS::NT), args, sizeof(WSmem), stream));
    s->last_G = G;
    s->wide_state_valid = 1;
    return TITUS_OK;
}

int check_status(titus_solver* s) {
    CK(cudaDeviceSynchronize());
    int status = 0;
    CK(cudaMemcpy(&status, s->wst.status, sizeof(int), cudaMemcpyDeviceToHost));
    if (status == 0) return TITUS_OK;
    double d[16];
    CK(cudaMemcpy(d, s->wst.diag, sizeof(d), cudaMemcpyDeviceToHost));
    int info[8];
    CK(cudaMemcpy(info, s->wst.info, sizeof(info), cudaMemcpyDeviceToHost));
    const char* what = status == ST_BARRIER_TIMEOUT  ? "team barrier timeout"
                       : status == ST_CHOL_BREAKDOWN ? "Cholesky breakdown"
                       : status == ST_COMPLETION     ? "basis completion ran out of candidates"
                       : status == ST_JACOBI         ? "Jacobi eigensolver did not converge"
                       : status == ST_LIMIT          ? "rank exceeds the adaptive kernel's capacity"
                       : status == ST_UNSUPPORTED    ? "angular basis not orthonormal (cannot complete)"
                       : status == ST_SVD            ? "Jacobi SVD did not converge"
                       : status == ST_REF_SHAPE
                           ? "scattering rejection after the streaming step changed the rank: the reference's next "
                             "step raises DimensionMismatch (SolverCSD.jl:2553)"
                           : "device error";
    const int code = status == ST_LIMIT ? TITUS_ERR_LIMIT : TITUS_ERR_DEVICE;
    if (status == ST_BARRIER_TIMEOUT) {
        unsigned counter = 0;
        CK(cudaMemcpy(&counter, s->wst.bar + s->last_G, sizeof(unsigned), cudaMemcpyDeviceToHost));
        return fail(code, "device status %d: %s (CTA %g at barrier %g saw %g arrivals, wanted %g; counter now %u)",
                    status, what, d[8], d[14], d[9], d[10], counter);
    }
    if (status == ST_SVD || (status == ST_COMPLETION && d[0] == 33)) {
        // statistics of the matrix handed to the SVD (CTA 0's copy)
        std::vector<double> a((size_t)KA * KA);
        CK(cudaMemcpy(a.data(), s->wst.scr + SO_DBG, a.size() * sizeof(double), cudaMemcpyDeviceToHost));
        const int m = (int)d[2];
        int nonfinite = 0, zeros = 0;
        double amax = 0.0, amin = INFINITY;
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j) {
                const double v = a[(size_t)i * KA + j];
                if (!std::isfinite(v)) ++nonfinite;
                else if (v == 0.0) ++zeros;
                else {
                    amax = std::max(amax, std::fabs(v));
                    amin = std::min(amin, std::fabs(v));
                }
            }
        std::string row;
        for (int j = 0; j < std::min(m, 8); ++j) row += std::to_string(a[j]) + " ";
        return fail(code, "device status %d: %s (m %d at step %g; input: %d non-finite, %d zeros, |a| in [%.3e, %.3e]; "
                    "column 0: %s)", status, what, m, d[7], nonfinite, zeros, amin, amax, row.c_str());
    }
    if (status == ST_REF_SHAPE)
        return fail(code, "device status %d: %s (rank %g entering energy index %g, %g after streaming)", status, what,
                    d[0], d[7], d[2]);
    return fail(code, "device status %d: %s (rank cap %d, adaptive width %d; diag %g %g %g step %g)", status, what,
                RA, KA, d[0], d[2], d[3], d[7]);
}

}  // namespace

int titus_host::TITUS_WIDE_HOST(wide_solve_device)(titus_solver* s, int method, const titus_options_t* opt, cudaStream_t stream) {
    int rc = ensure_state(s);
    if (rc) return rc;
    const int r0 = s->r / 2;
    if (r0 < 1) return fail(TITUS_ERR_ARG, "adaptive integrators need settings.r >= 2 (got %d)", s->r);
    if (r0 > RA) return fail(TITUS_ERR_LIMIT, "initial rank %d > %d", r0, RA);
    if (2 * r0 > s->N) return fail(TITUS_ERR_ARG, "augmented width %d exceeds the %d moments", 2 * r0, s->N);
    if ((rc = init_state(s, r0, method, stream))) return rc;
    int n_end = s->nE;
    int max_iters = INT_MAX;
    if (opt && opt->max_steps > 0) {
        if (method == TITUS_PARALLEL_ADAPTIVE) n_end = std::min(n_end, 1 + opt->max_steps);
        else max_iters = opt->max_steps;
    }
    return launch(s, method, opt, 2, n_end, max_iters, stream);
}

int titus_host::TITUS_WIDE_HOST(wide_solve_from)(titus_solver* s, int method, const titus_options_t* opt, int n_stop) {
    if (!s->d_wst || !s->wide_state_valid) return fail(TITUS_ERR_ARG, "no adaptive state to resume (call titus_set_state)");
    int info[8];
    CK(cudaMemcpy(info, s->wst.info, sizeof(info), cudaMemcpyDeviceToHost));
    const int n_begin = info[3];
    int n_end = std::min(n_stop, s->nE);
    int max_iters = INT_MAX;
    if (opt && opt->max_steps > 0) {
        if (method == TITUS_PARALLEL_ADAPTIVE) n_end = std::min(n_end, n_begin + opt->max_steps - 1);
        else max_iters = opt->max_steps;
    }
    if (n_end < n_begin) return fail(TITUS_ERR_ARG, "nothing to run (n_begin %d, n_stop %d)", n_begin, n_stop);
    return launch(s, method, opt, n_begin, n_end, max_iters, nullptr);
}

int titus_host::TITUS_WIDE_HOST(wide_fetch)(titus_solver* s, titus_result_t* res) {
    int rc = check_status(s);
    if (rc) return rc;
    WideState& w = s->wst;
    int info[8];
    CK(cudaMemcpy(info, w.info, sizeof(info), cudaMemcpyDeviceToHost));
    const int k = info[0];
    res->rank = k;
    res->steps_done = info[1];
    if (res->dose) CK(cudaMemcpy(res->dose, w.dose, s->n * sizeof(double), cudaMemcpyDeviceToHost));
    const int cap = res->r_cap;
    if ((res->X || res->S || res->W) && cap < k) return fail(TITUS_ERR_ARG, "r_cap %d < rank %d", cap, k);
    if (res->X)
        CK(cudaMemcpy2D(res->X, cap * sizeof(double), w.X, KA * sizeof(double), k * sizeof(double), s->n,
                        cudaMemcpyDeviceToHost));
    if (res->W)
        CK(cudaMemcpy2D(res->W, cap * sizeof(double), w.W, KA * sizeof(double), k * sizeof(double), s->N,
                        cudaMemcpyDeviceToHost));
    if (res->S)
        CK(cudaMemcpy2D(res->S, cap * sizeof(double), w.S, KA * sizeof(double), k * sizeof(double), k,
                        cudaMemcpyDeviceToHost));
    if (res->psi) {
        double* src = info[2] ? w.psi1 : w.psi0;
        CK(cudaMemcpy2D(res->psi, s->q * sizeof(double), src, QW * sizeof(double), s->q * sizeof(double), s->n,
                        cudaMemcpyDeviceToHost));
    }
    const int nh = std::min(s->nE, w.hist_cap);
    if (res->rank_history) CK(cudaMemcpy(res->rank_history, w.rank_hist, nh * sizeof(int), cudaMemcpyDeviceToHost));
    if (res->time_history) CK(cudaMemcpy(res->time_history, w.time_hist, nh * sizeof(double), cudaMemcpyDeviceToHost));
    if (res->eta_history) CK(cudaMemcpy(res->eta_history, w.eta_hist, nh * sizeof(double), cudaMemcpyDeviceToHost));
    if (res->bound_history)
        CK(cudaMemcpy(res->bound_history, w.bound_hist, nh * sizeof(double), cudaMemcpyDeviceToHost));
    return TITUS_OK;
}

int titus_host::TITUS_WIDE_HOST(wide_set_state)(titus_solver* s, int rank, const double* X, const double* S, const double* W,
                               const double* psi, const double* dose, int n_next) {
    int rc = ensure_state(s);
    if (rc) return rc;
    WideState& w = s->wst;
    CK(cudaMemset(w.X, 0, (size_t)s->n * KA * sizeof(double)));
    CK(cudaMemset(w.W, 0, (size_t)s->N * KA * sizeof(double)));
    CK(cudaMemset(w.S, 0, (size_t)KA * KA * sizeof(double)));
    CK(cudaMemcpy2D(w.X, KA * sizeof(double), X, rank * sizeof(double), rank * sizeof(double), s->n,
                    cudaMemcpyHostToDevice));
    CK(cudaMemcpy2D(w.W, KA * sizeof(double), W, rank * sizeof(double), rank * sizeof(double), s->N,
                    cudaMemcpyHostToDevice));
    CK(cudaMemcpy2D(w.S, KA * sizeof(double), S, rank * sizeof(double), rank * sizeof(double), rank,
                    cudaMemcpyHostToDevice));
    CK(cudaMemset(w.psi0, 0, (size_t)s->n * QW * sizeof(double)));
    CK(cudaMemcpy2D(w.psi0, QW * sizeof(double), psi, s->q * sizeof(double), s->q * sizeof(double), s->n,
                    cudaMemcpyHostToDevice));
    CK(cudaMemcpy(w.dose, dose, s->n * sizeof(double), cudaMemcpyHostToDevice));
    int info[8] = {rank, 0, 0, n_next, 0, 0, 0, 0};
    CK(cudaMemcpy(w.info, info, sizeof(info), cudaMemcpyHostToDevice));
    // pseudo-time after the energies 2..n_next-1 (the loop condition t < nE dE)
    const double t = (n_next - 2) * s->P.dE;
    CK(cudaMemcpy(w.tvar, &t, sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemset(w.rank_hist, 0xff, w.hist_cap * sizeof(int)));
    s->wide_state_valid = 1;
    return TITUS_OK;
}


#if TITUS_WIDE_NOPS == 4   // batched pencil beams: 2D problems
namespace {

struct DevTemps {
    std::vector<void*> ptrs;
    ~DevTemps() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <class T>
    int alloc(T** p, size_t count, const T* host = nullptr) {
        int rc = titus_host::upload(p, host, count);
        if (rc == TITUS_OK && *p) ptrs.push_back((void*)*p);
        return rc;
    }
};

int ensure_batch_states(titus_solver* s, int T, int G) {
    if (s->d_bst && s->b_teams >= T && s->b_G == G) return TITUS_OK;
    for (void* p : s->batch_allocs) cudaFree(p);
    s->batch_allocs.clear();
    s->d_bst = nullptr;
    const int n = s->n, N = s->N;
    auto al = [&](auto** p, size_t count) -> int {
        using Elem = std::remove_pointer_t<std::remove_reference_t<decltype(*p)>>;
        int rc = titus_host::upload(p, static_cast<const Elem*>(nullptr), count);
        if (rc == TITUS_OK && *p) s->batch_allocs.push_back((void*)*p);
        return rc;
    };
    int* status = nullptr;
    double* diag = nullptr;
    int rc;
    if ((rc = al(&status, 1)) || (rc = al(&diag, 16))) return rc;
    s->bst.assign(T, WideState{});
    for (int t = 0; t < T; ++t) {
        WideState& w = s->bst[t];
        if ((rc = al(&w.X, (size_t)n * KA)) || (rc = al(&w.W, (size_t)N * KA)) || (rc = al(&w.K, (size_t)n * RA)) ||
            (rc = al(&w.KP, (size_t)n * RA)) || (rc = al(&w.CX, (size_t)n * RA)) || (rc = al(&w.L, (size_t)N * RA)) ||
            (rc = al(&w.LP, (size_t)N * RA)) || (rc = al(&w.CW, (size_t)N * RA)) ||
            (rc = al(&w.psi0, (size_t)n * QW)) || (rc = al(&w.psi1, (size_t)n * QW)) ||
            (rc = al(&w.S, (size_t)KA * KA)) || (rc = al(&w.part, (size_t)2 * G * PMAXW)) ||
            (rc = al(&w.red, (size_t)2 * PMAXW)) || (rc = al(&w.scr, (size_t)G * SCRW)) ||
            (rc = al(&w.bar, (size_t)G + 1)) || (rc = al(&w.info, 8)) || (rc = al(&w.tvar, 1)))
            return rc;
        w.dose = nullptr;          // per spot
        w.status = status;         // shared: a failing team stops the batch
        w.diag = diag;
        w.rank_hist = nullptr;
        w.time_hist = w.eta_hist = w.bound_hist = nullptr;
        w.hist_cap = 0;
    }
    WideState* d = nullptr;
    if ((rc = al(&d, (size_t)T))) return rc;
    CK(cudaMemcpy(d, s->bst.data(), T * sizeof(WideState), cudaMemcpyHostToDevice));
    s->d_bst = d;
    s->b_teams = T;
    s->b_G = G;
    CK(cudaFuncSetAttribute(adaptive_batched_kernel<TITUS_PARALLEL_ADAPTIVE>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(WSmem)));
    CK(cudaFuncSetAttribute(adaptive_batched_kernel<TITUS_BUG_ADAPTIVE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)sizeof(WSmem)));
    return TITUS_OK;
}

}  // namespace

// A set of pencil beams uploaded once (titus_batch_upload): per-spot tables,
// the longest-first order, the work-queue counter and the outputs, all on the
// device, so repeated launches move no host data.
struct titus_batch {
    titus_solver* s = nullptr;
    int nspots = 0;
    DevTemps tmp;
    SpotData* d_sd = nullptr;
    double* d_dose = nullptr;
    int* d_res = nullptr;
    int* d_order = nullptr;
    int* d_queue = nullptr;
    int last_T = 0, last_G = 0;
    bool launched = false;
    std::vector<int> rank_sums;   // per spot, after the last fetch
};

int titus_host::batch_upload(titus_solver* s, int nspots, const titus_spot_t* spots, titus_batch** out) {
    *out = nullptr;
    const int n = s->n, npn1 = s->P.npn + 1;
    for (int i = 0; i < nspots; ++i) {
        const titus_spot_t& sp = spots[i];
        if (sp.n_energies < 2) return fail(TITUS_ERR_ARG, "spot %d: n_energies < 2", i);
        if (!(sp.d_e > 0) || !std::isfinite(sp.d_e)) return fail(TITUS_ERR_ARG, "spot %d: d_e must be finite and > 0", i);
        if (!sp.stopping || !sp.bc_energy || !sp.sigma || !sp.bc_space)
            return fail(TITUS_ERR_ARG, "spot %d: a table is NULL", i);
        for (int e = 0; e < sp.n_energies; ++e)
            if (!std::isfinite(sp.stopping[e]) || !std::isfinite(sp.bc_energy[e]))
                return fail(TITUS_ERR_ARG, "spot %d: stopping / bc_energy [%d] not finite", i, e);
        for (size_t e = 0; e < (size_t)sp.n_energies * npn1; ++e)
            if (!std::isfinite(sp.sigma[e])) return fail(TITUS_ERR_ARG, "spot %d: sigma[%zu] not finite", i, e);
        for (int c = 0; c < n; ++c)
            if (!std::isfinite(sp.bc_space[c])) return fail(TITUS_ERR_ARG, "spot %d: bc_space[%d] not finite", i, c);
    }
    auto* b = new titus_batch();
    b->s = s;
    b->nspots = nspots;
    auto bail = [&](int rc) {
        delete b;
        return rc;
    };
    size_t tot_e = 0;
    for (int i = 0; i < nspots; ++i) tot_e += (size_t)spots[i].n_energies;
    double *d_stop, *d_bce, *d_sig, *d_bcs;
    int rc;
    if ((rc = b->tmp.alloc(&d_stop, tot_e)) || (rc = b->tmp.alloc(&d_bce, tot_e)) ||
        (rc = b->tmp.alloc(&d_sig, tot_e * npn1)) || (rc = b->tmp.alloc(&d_bcs, (size_t)nspots * n)) ||
        (rc = b->tmp.alloc(&b->d_dose, (size_t)nspots * n)) || (rc = b->tmp.alloc(&b->d_res, (size_t)3 * nspots)) ||
        (rc = b->tmp.alloc(&b->d_queue, (size_t)1)))
        return bail(rc);
    std::vector<SpotData> sd(nspots);
    size_t off = 0;
    for (int i = 0; i < nspots; ++i) {
        const titus_spot_t& sp = spots[i];
        const int nE = sp.n_energies;
        cudaError_t e = cudaMemcpy(d_stop + off, sp.stopping, nE * sizeof(double), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(d_bce + off, sp.bc_energy, nE * sizeof(double), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(d_sig + off * npn1, sp.sigma, (size_t)nE * npn1 * sizeof(double), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(d_bcs + (size_t)i * n, sp.bc_space, n * sizeof(double), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return bail(fail(TITUS_ERR_CUDA, "spot table upload: %s", cudaGetErrorString(e)));
        SpotData& d = sd[i];
        d.nE = nE;
        d.n_end = nE;
        d.dE = sp.d_e;
        d.stopping = d_stop + off;
        d.bc_energy = d_bce + off;
        d.sigma = d_sig + off * npn1;
        d.bc_space = d_bcs + (size_t)i * n;
        d.dose = b->d_dose + (size_t)i * n;
        d.result = b->d_res + 3 * i;
        off += nE;
    }
    if ((rc = b->tmp.alloc(&b->d_sd, (size_t)nspots, sd.data()))) return bail(rc);
    // longest first: a spot's loop runs about nE iterations, so handing the
    // queue out in decreasing nE keeps the last teams from starting long spots
    std::vector<int> order(nspots);
    for (int i = 0; i < nspots; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int c) { return spots[a].n_energies > spots[c].n_energies; });
    if ((rc = b->tmp.alloc(&b->d_order, (size_t)nspots, order.data()))) return bail(rc);
    *out = b;
    return TITUS_OK;
}

int titus_host::batch_launch(titus_batch* b, int method, const titus_options_t* opt, cudaStream_t stream) {
    titus_solver* s = b->s;
    const int r0 = s->r / 2;
    if (r0 < 1) return fail(TITUS_ERR_ARG, "adaptive integrators need settings.r >= 2 (got %d)", s->r);
    if (r0 > RA) return fail(TITUS_ERR_LIMIT, "initial rank %d > %d", r0, RA);
    if (2 * r0 > s->N) return fail(TITUS_ERR_ARG, "augmented width %d exceeds the %d moments", 2 * r0, s->N);
    int G = (opt && opt->team_ctas > 0) ? opt->team_ctas : 1;
    G = std::max(1, std::min(G, s->num_sms));
    int per_sm = 0;
    auto kfun = method == TITUS_PARALLEL_ADAPTIVE ? adaptive_batched_kernel<TITUS_PARALLEL_ADAPTIVE>
                                                  : adaptive_batched_kernel<TITUS_BUG_ADAPTIVE>;
    CK(cudaFuncSetAttribute(kfun, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(WSmem)));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfun, TITUS_WIDE_NS::NT, sizeof(WSmem)));
    if (per_sm < 1) return fail(TITUS_ERR_CUDA, "batched kernel does not fit on an SM");
    const int T = std::max(1, std::min(b->nspots, per_sm * s->num_sms / G));
    int rc = ensure_batch_states(s, T, G);
    if (rc) return rc;
    // parallel integrator: max_steps bounds the energy index; BUG: the iterations
    const int max_steps = (opt && opt->max_steps > 0) ? opt->max_steps : 0;
    int max_iters = INT_MAX;
    if (method == TITUS_BUG_ADAPTIVE && max_steps > 0) max_iters = max_steps;
    for (int t = 0; t < T; ++t) CK(cudaMemsetAsync(s->bst[t].bar, 0, (size_t)(G + 1) * sizeof(unsigned), stream));
    CK(cudaMemsetAsync(s->bst[0].status, 0, sizeof(int), stream));
    CK(cudaMemsetAsync(s->bst[0].diag, 0, 16 * sizeof(double), stream));
    CK(cudaMemsetAsync(b->d_queue, 0, sizeof(int), stream));
    DevProblem P = s->P;
    if (opt && opt->rank_tol > 0) P.rank_tol = opt->rank_tol;
    P.prof = nullptr;
    P.zero_smem = 0;
    P.precision = opt ? opt->precision : TITUS_PRECISION_FP64;
    s->take_debug_hooks(P);
    if (opt && opt->profile) {
        CK(cudaMemsetAsync(s->prof, 0, PF_SLOTS * sizeof(unsigned long long), stream));
        P.prof = s->prof;
    }
    WideState* dst = s->d_bst;
    SpotData* d_sd = b->d_sd;
    int Tl = T, Gl = G, ns = b->nspots, r0l = r0, msl = (method == TITUS_PARALLEL_ADAPTIVE) ? max_steps : 0;
    int* queue = b->d_queue;
    const int* order = b->d_order;
    void* args[] = {&P, &dst, &Gl, &Tl, &d_sd, &ns, &r0l, &max_iters, &msl, &queue, &order};
    CK(cudaLaunchCooperativeKernel((void*)kfun, dim3(T * G), dim3(TITUS_WIDE_NS::NT), args, sizeof(WSmem), stream));
    b->last_T = T;
    b->last_G = G;
    b->launched = true;
    s->last_method = method;
    return TITUS_OK;
}

int titus_host::batch_fetch(titus_batch* b, double* dose_out, int32_t* rank_out, int32_t* iters_out) {
    if (!b->launched) return fail(TITUS_ERR_ARG, "batch has not been solved yet");
    titus_solver* s = b->s;
    CK(cudaDeviceSynchronize());
    int status = 0;
    CK(cudaMemcpy(&status, s->bst[0].status, sizeof(int), cudaMemcpyDeviceToHost));
    if (status != 0) {
        double d[16];
        CK(cudaMemcpy(d, s->bst[0].diag, sizeof(d), cudaMemcpyDeviceToHost));
        if (status == ST_BARRIER_TIMEOUT)
            return fail(TITUS_ERR_DEVICE,
                        "batched solve: device status %d: team barrier timeout (CTA %g at barrier %g saw %g arrivals, "
                        "wanted %g; teams %d x %d CTAs)", status, d[8], d[14], d[9], d[10], b->last_T, b->last_G);
        return fail(status == ST_LIMIT ? TITUS_ERR_LIMIT : TITUS_ERR_DEVICE,
                    "batched solve: device status %d (teams %d x %d CTAs)", status, b->last_T, b->last_G);
    }
    const int n = s->n;
    if (dose_out) CK(cudaMemcpy(dose_out, b->d_dose, (size_t)b->nspots * n * sizeof(double), cudaMemcpyDeviceToHost));
    std::vector<int> res(3 * b->nspots);
    CK(cudaMemcpy(res.data(), b->d_res, res.size() * sizeof(int), cudaMemcpyDeviceToHost));
    for (int i = 0; i < b->nspots; ++i) {
        if (rank_out) rank_out[i] = res[3 * i];
        if (iters_out) iters_out[i] = res[3 * i + 1];
    }
    b->rank_sums.assign(b->nspots, 0);
    for (int i = 0; i < b->nspots; ++i) b->rank_sums[i] = res[3 * i + 2];
    return TITUS_OK;
}

void titus_host::batch_free(titus_batch* b) { delete b; }

int titus_host::batch_rank_sums(titus_batch* b, int32_t* out) {
    if ((int)b->rank_sums.size() != b->nspots) return fail(TITUS_ERR_ARG, "fetch the batch first");
    for (int i = 0; i < b->nspots; ++i) out[i] = b->rank_sums[i];
    return TITUS_OK;
}

int titus_host::wide_solve_batched(titus_solver* s, int method, const titus_options_t* opt, int nspots,
                                   const titus_spot_t* spots, double* dose_out, int32_t* rank_out, int32_t* iters_out) {
    titus_batch* b = nullptr;
    int rc = batch_upload(s, nspots, spots, &b);
    if (rc) return rc;
    rc = batch_launch(b, method, opt, nullptr);
    if (!rc) rc = batch_fetch(b, dose_out, rank_out, iters_out);
    batch_free(b);
    return rc;
}
#endif

void titus_host::TITUS_WIDE_HOST(wide_free)(titus_solver* s) {
    for (void* p : s->wide_allocs) cudaFree(p);
    s->wide_allocs.clear();
    s->d_wst = nullptr;
    for (void* p : s->batch_allocs) cudaFree(p);
    s->batch_allocs.clear();
    s->d_bst = nullptr;
}
