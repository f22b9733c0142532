// C ABI of libtitus (include/titus.h): problem upload, device state, launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "titus_handle.h"
#include "wide_common.cuh"
#include "dlr_fixed.cuh"

using namespace titus;
using titus_host::fail;

namespace {
thread_local std::string g_last_error;
std::atomic<int> g_alloc_fault{0};
}  // namespace

int titus_host::take_alloc_fault() {
    int v = g_alloc_fault.load();
    while (v > 0 && !g_alloc_fault.compare_exchange_weak(v, v - 1)) {
    }
    return v == 1;
}

int titus_host::fail(int code, const char* fmt, ...) {
    char buf[768];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

titus_solver::~titus_solver() {
    titus_host::pn_free(this);
    titus_host::pn3_free(this);
    titus_host::wide_free(this);
    for (void* p : allocs) cudaFree(p);
}

// CSR of one P_N operator (N x N): rowptr monotone from 0, columns in range, values finite.
static int validate_csr(const int32_t* rp, const int32_t* ci, const double* v, int N, int d) {
    if (!rp || (!ci && rp[N] > 0) || (!v && rp[N] > 0)) return fail(TITUS_ERR_ARG, "operator %d CSR arrays missing", d);
    if (rp[0] != 0) return fail(TITUS_ERR_ARG, "operator %d rowptr[0] != 0", d);
    for (int m = 0; m < N; ++m)
        if (rp[m + 1] < rp[m]) return fail(TITUS_ERR_ARG, "operator %d rowptr not monotone", d);
    for (int p = 0; p < rp[N]; ++p) {
        if (ci[p] < 0 || ci[p] >= N) return fail(TITUS_ERR_ARG, "operator %d column index out of range", d);
        if (!std::isfinite(v[p])) return fail(TITUS_ERR_ARG, "operator %d value %d is not finite", d, p);
    }
    return TITUS_OK;
}

// `nz` = 0 for the reference's 2D problems; >= 3 z layers for a 3D problem
// (titus_create_3d), whose cell arrays hold nx ny nz entries.
static int validate(const titus_problem_t* pb, int nz = 0) {
    if (!pb) return fail(TITUS_ERR_ARG, "problem is NULL");
    if (pb->nx < 3 || pb->ny < 3) return fail(TITUS_ERR_ARG, "need nx, ny >= 3 (got %d, %d)", pb->nx, pb->ny);
    if ((long long)pb->nx * pb->ny * (nz ? nz : 1) > INT_MAX / 64)
        return fail(TITUS_ERR_LIMIT, "%d x %d x %d cells exceed this build's index range", pb->nx, pb->ny, nz);
    if (pb->npn < 0) return fail(TITUS_ERR_ARG, "npn < 0");
    if (pb->n_moments != (pb->npn + 1) * (pb->npn + 1))
        return fail(TITUS_ERR_ARG, "n_moments %d != (npn+1)^2", pb->n_moments);
    if (pb->n_ordinates < 1) return fail(TITUS_ERR_ARG, "n_ordinates < 1");
    if (pb->n_ordinates > std::min(QM, KM))
        return fail(TITUS_ERR_LIMIT, "n_ordinates %d > %d supported", pb->n_ordinates, std::min(QM, KM));
    if (pb->n_energies < 2) return fail(TITUS_ERR_ARG, "n_energies < 2");
    if (pb->r < 1) return fail(TITUS_ERR_ARG, "r < 1");
    if (pb->r > 2 * wide::RA)
        return fail(TITUS_ERR_LIMIT, "rank cap %d > %d supported by this build", pb->r, 2 * wide::RA);
    if (pb->r > pb->n_moments) return fail(TITUS_ERR_ARG, "r %d > n_moments %d", pb->r, pb->n_moments);
    if (!(pb->dx > 0) || !(pb->dy > 0) || !std::isfinite(pb->dx) || !std::isfinite(pb->dy))
        return fail(TITUS_ERR_ARG, "dx, dy must be finite and > 0");
    if (!std::isfinite(pb->theta) || !std::isfinite(pb->theta_index) || !std::isfinite(pb->c_eta))
        return fail(TITUS_ERR_ARG, "theta, theta_index and c_eta must be finite");
    const void* req[] = {pb->density, pb->e_trafo, pb->stopping, pb->bc_energy, pb->sigma,
                         pb->bc_space, pb->bc_angle, pb->omega, pb->m_reduced};
    for (const void* p : req)
        if (!p) return fail(TITUS_ERR_ARG, "a required problem array is NULL");
    // non-finite inputs would propagate through the whole energy loop unnoticed
    {
        const int n = pb->nx * pb->ny * (nz ? nz : 1), nE = pb->n_energies, q = pb->n_ordinates, N = pb->n_moments;
        struct Arr {
            const double* p;
            size_t count;
            const char* name;
        } arrs[] = {{pb->density, (size_t)n, "density"},
                    {pb->e_trafo, (size_t)nE, "e_trafo"},
                    {pb->stopping, (size_t)nE, "stopping"},
                    {pb->bc_energy, (size_t)nE, "bc_energy"},
                    {pb->sigma, (size_t)nE * (pb->npn + 1), "sigma"},
                    {pb->bc_space, (size_t)n, "bc_space"},
                    {pb->bc_angle, (size_t)q, "bc_angle"},
                    {pb->omega, (size_t)q * 3, "omega"},
                    {pb->m_reduced, (size_t)N * q, "m_reduced"},
                    {pb->stopping_mid, pb->stopping_mid ? (size_t)nE - 1 : 0, "stopping_mid"}};
        for (const Arr& a : arrs)
            for (size_t i = 0; i < a.count; ++i)
                if (!std::isfinite(a.p[i])) return fail(TITUS_ERR_ARG, "%s[%zu] is not finite", a.name, i);
    }
    if (pb->n_x_completion < 0 || pb->n_w_completion < 0 || pb->n_sweep_restore < 0)
        return fail(TITUS_ERR_ARG, "negative list length");
    const int n = pb->nx * pb->ny * (nz ? nz : 1);
    for (int i = 0; i < n; ++i)
        if (!(pb->density[i] > 0)) return fail(TITUS_ERR_ARG, "density must be > 0 (cell %d)", i);
    for (int i = 0; i < pb->n_x_completion; ++i)
        if (pb->x_completion[i] < 0 || pb->x_completion[i] >= n) return fail(TITUS_ERR_ARG, "x_completion out of range");
    for (int i = 0; i < pb->n_w_completion; ++i)
        if (pb->w_completion[i] < 0 || pb->w_completion[i] >= pb->n_moments)
            return fail(TITUS_ERR_ARG, "w_completion out of range");
    for (int i = 0; i < pb->n_sweep_restore; ++i)
        if (pb->sweep_restore[i] < 0 || pb->sweep_restore[i] >= n) return fail(TITUS_ERR_ARG, "sweep_restore out of range");
    for (int d = 0; d < 4; ++d)
        if (int rc = validate_csr(pb->op_rowptr[d], pb->op_col[d], pb->op_val[d], pb->n_moments, d)) return rc;
    return TITUS_OK;
}

// Uploads the problem into `s`; on any failure the caller deletes `s`, which
// releases every allocation made so far.
static int create_impl(const titus_problem_t* pb, titus_solver* s, int nz = 0) {
    int rc;
    CK(cudaGetDevice(&s->device));
    CK(cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, s->device));
    int coop = 0;
    CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, s->device));
    if (!coop) return fail(TITUS_ERR_CUDA, "device does not support cooperative launch");
    const int n = pb->nx * pb->ny * (nz ? nz : 1), N = pb->n_moments, q = pb->n_ordinates, nE = pb->n_energies;
    s->n = n;
    s->N = N;
    s->q = q;
    s->nE = nE;
    s->r = pb->r;
    DevProblem& P = s->P;
    P.nx = pb->nx;
    P.ny = pb->ny;
    P.n = n;
    P.N = N;
    P.npn = pb->npn;
    P.q = q;
    P.nE = nE;
    P.r = pb->r;
    P.dx = pb->dx;
    P.dy = pb->dy;
    P.dE = pb->e_trafo[1] - pb->e_trafo[0];
    P.theta = pb->theta;
    P.theta_index = pb->theta_index;
    P.c_eta = pb->c_eta;
    P.rank_tol = 1e-12;
    std::vector<double> rinv(n);
    for (int i = 0; i < n; ++i) rinv[i] = 1.0 / pb->density[i];
    std::vector<int32_t> lof(N);
    for (int l = 0; l <= pb->npn; ++l)
        for (int kk = -l; kk <= l; ++kk) lof[l * l + kk + l] = l;
    std::vector<uint8_t> restore(n, 0);
    for (int i = 0; i < pb->n_sweep_restore; ++i) restore[pb->sweep_restore[i]] = 1;
    double* d_rinv;
    double* d_stop;
    double* d_bce;
    double* d_sig;
    double* d_bcs;
    double* d_bca;
    double* d_om;
    double* d_mr;
    int32_t* d_lof;
    uint8_t* d_res;
    int32_t* d_xc = nullptr;
    int32_t* d_wc = nullptr;
    if ((rc = s->alloc(&d_rinv, n, rinv.data())) || (rc = s->alloc(&d_stop, nE, pb->stopping)) ||
        (rc = s->alloc(&d_bce, nE, pb->bc_energy)) ||
        (rc = s->alloc(&d_sig, (size_t)nE * (pb->npn + 1), pb->sigma)) || (rc = s->alloc(&d_bcs, n, pb->bc_space)) ||
        (rc = s->alloc(&d_bca, q, pb->bc_angle)) || (rc = s->alloc(&d_om, (size_t)q * 3, pb->omega)) ||
        (rc = s->alloc(&d_mr, (size_t)N * q, pb->m_reduced)) || (rc = s->alloc(&d_lof, N, lof.data())) ||
        (rc = s->alloc(&d_res, n, restore.data())) ||
        (rc = s->alloc(&d_xc, pb->n_x_completion, pb->x_completion)) ||
        (rc = s->alloc(&d_wc, pb->n_w_completion, pb->w_completion)))
        return rc;
    if (pb->stopping_mid && (rc = s->alloc(&s->smid, (size_t)nE - 1, pb->stopping_mid))) return rc;
    P.rinv = d_rinv;
    P.stopping = d_stop;
    P.bc_energy = d_bce;
    P.sigma = d_sig;
    P.bc_space = d_bcs;
    P.bc_angle = d_bca;
    P.omega = d_om;
    P.mred = d_mr;
    P.lof = d_lof;
    P.restore = d_res;
    P.xcomp = d_xc;
    P.nxcomp = pb->n_x_completion;
    P.wcomp = d_wc;
    P.nwcomp = pb->n_w_completion;
    for (int d = 0; d < 4; ++d) {
        const int nnz = pb->op_rowptr[d][N];
        int32_t* rp;
        int32_t* ci = nullptr;
        double* v = nullptr;
        if ((rc = s->alloc(&rp, N + 1, pb->op_rowptr[d])) || (rc = s->alloc(&ci, nnz, pb->op_col[d])) ||
            (rc = s->alloc(&v, nnz, pb->op_val[d])))
            return rc;
        P.op[d].rowptr = rp;
        P.op[d].col = ci;
        P.op[d].val = v;
    }
    // team state (one team); partial buffer sized for the largest team
    s->team_ctas = std::min(s->num_sms, 32);
    TeamState& st = s->st;
    const size_t nK = (size_t)n * KM, NK = (size_t)N * KM;
    unsigned* bar;
    int* info;
    if ((rc = s->alloc(&st.X, nK)) || (rc = s->alloc(&st.K, nK)) || (rc = s->alloc(&st.W, NK)) ||
        (rc = s->alloc(&st.L, 2 * NK)) || (rc = s->alloc(&st.psi0, (size_t)n * QM)) ||
        (rc = s->alloc(&st.psi1, (size_t)n * QM)) || (rc = s->alloc(&st.dose, n)) ||
        (rc = s->alloc(&st.S, KK)) || (rc = s->alloc(&st.part, (size_t)2 * s->num_sms * PMAX)) ||
        (rc = s->alloc(&st.red, PMAX)) ||
        (rc = s->alloc(&bar, s->num_sms + 1)) || (rc = s->alloc(&st.status, 1)) || (rc = s->alloc(&info, 4)) ||
        (rc = s->alloc(&st.rank_hist, nE)) || (rc = s->alloc(&st.diag, 16)))
        return rc;
    st.bar = bar;
    st.info = info;
    st.eta_hist = st.bound_hist = st.time_hist = nullptr;
    if ((rc = s->alloc(&s->d_st, 1))) return rc;
    if ((rc = s->alloc(&s->prof, PF_SLOTS))) return rc;
    CK(cudaMemset(s->prof, 0, PF_SLOTS * sizeof(unsigned long long)));
    CK(cudaDeviceGetAttribute(&s->clock_khz, cudaDevAttrClockRate, s->device));
    CK(cudaMemcpy(s->d_st, &st, sizeof(TeamState), cudaMemcpyHostToDevice));
    CK(cudaFuncSetAttribute(dlr_kernel<TITUS_DLR_FIXED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)sizeof(SmemLayout)));
    CK(cudaFuncSetAttribute(dlr_kernel<TITUS_DLR_HIGH_ORDER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)sizeof(SmemLayout)));
    return TITUS_OK;
}

static_assert(TITUS_DLR_HIGH_ORDER == titus::kHighOrder, "method id of the RK4 kernel");
static bool is_fixed_family(int method) { return method == TITUS_DLR_FIXED || method == TITUS_DLR_HIGH_ORDER; }
static bool is_wide_family(int method) {
    return method == TITUS_PARALLEL_ADAPTIVE || method == TITUS_BUG_ADAPTIVE || method == TITUS_PARALLEL_REJECTION;
}

// The RK4 integrator's stage buffers (3 x n x KM and 3 x N x KM), allocated on
// its first use.
static int ensure_rk4_buffers(titus_solver* s) {
    if (s->st.Y) return TITUS_OK;
    int rc;
    if ((rc = s->alloc(&s->st.Y, (size_t)3 * s->n * KM)) || (rc = s->alloc(&s->st.Z, (size_t)3 * s->N * KM))) {
        s->st.Y = s->st.Z = nullptr;   // both stay tracked in allocs and are freed with the handle
        return rc;
    }
    CK(cudaMemcpy(s->d_st, &s->st, sizeof(TeamState), cudaMemcpyHostToDevice));
    return TITUS_OK;
}

extern "C" int titus_create(const titus_problem_t* pb, titus_solver_t** out) {
    if (!out) return fail(TITUS_ERR_ARG, "out is NULL");
    *out = nullptr;
    int rc = validate(pb);
    if (rc) return rc;
    auto* s = new titus_solver();
    if ((rc = create_impl(pb, s))) {
        delete s;
        return rc;
    }
    *out = s;
    return TITUS_OK;
}

extern "C" int titus_create_3d(const titus_problem_t* pb, const titus_problem_3d_t* ext, titus_solver_t** out) {
    if (!out) return fail(TITUS_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!ext) return fail(TITUS_ERR_ARG, "3D extension is NULL");
    if (ext->nz < 3) return fail(TITUS_ERR_ARG, "need nz >= 3 (got %d)", ext->nz);
    if (!(ext->dz > 0) || !std::isfinite(ext->dz)) return fail(TITUS_ERR_ARG, "dz must be finite and > 0");
    int rc = validate(pb, ext->nz);
    if (rc) return rc;
    for (int d = 0; d < 2; ++d)
        if ((rc = validate_csr(ext->op_rowptr[d], ext->op_col[d], ext->op_val[d], pb->n_moments, 4 + d))) return rc;
    auto* s = new titus_solver();
    rc = create_impl(pb, s, ext->nz);
    for (int d = 0; d < 2 && !rc; ++d) {
        const int nnz = ext->op_rowptr[d][pb->n_moments];
        int32_t* rp = nullptr;
        int32_t* ci = nullptr;
        double* v = nullptr;
        if (!(rc = s->alloc(&rp, (size_t)pb->n_moments + 1, ext->op_rowptr[d])) &&
            !(rc = s->alloc(&ci, nnz, ext->op_col[d])) && !(rc = s->alloc(&v, nnz, ext->op_val[d])))
            s->op3[d] = Csr{rp, ci, v};
    }
    if (rc) {
        delete s;
        return rc;
    }
    s->nz = ext->nz;
    s->dz = ext->dz;
    s->P.nz = ext->nz;
    s->P.dz = ext->dz;
    s->P.op[4] = s->op3[0];
    s->P.op[5] = s->op3[1];
    *out = s;
    return TITUS_OK;
}

// A 3D handle (titus_create_3d) runs the full-rank P_N solver and the BUG
// integrator (plain and resumed); the other DLR integrators and the batched
// form run the reference's 2D problems.
static int reject_3d(const titus_solver* s, const char* what, int method = -1) {
    if (!s->nz || method == TITUS_BUG_ADAPTIVE) return TITUS_OK;
    return fail(TITUS_ERR_ARG, "%s: 3D problems run with titus_pn_full_solve or the BUG integrator (method %d)", what,
                TITUS_BUG_ADAPTIVE);
}

// Initial factors of SolverCSD.jl:931-955: X = first r identity columns with
// boundary rows zeroed, W = first r identity columns, S = 0.
__global__ void init_factors_kernel(TeamState* states, int n, int N, int nx, int ny, int r, int nE) {
    TeamState st = states[blockIdx.y];
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < r; j += gridDim.x * blockDim.x) {
        if (j < n) {
            int i = j / ny, jj = j % ny;
            bool bnd = (i == 0 || jj == 0 || i == nx - 1 || jj == ny - 1);
            st.X[(size_t)j * KM + j] = bnd ? 0.0 : 1.0;
        }
        if (j < N) st.W[(size_t)j * KM + j] = 1.0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st.info[0] = r;
        st.info[1] = 0;
        st.info[2] = 0;
        st.info[3] = 2;
    }
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nE; e += gridDim.x * blockDim.x) st.rank_hist[e] = -1;
}

// Device-side reset of one team's state (no host copies): factors, psi, dose.
static int init_state(titus_solver* s, int r, cudaStream_t stream) {
    const int n = s->n, N = s->N;
    TeamState& st = s->st;
    CK(cudaMemsetAsync(st.X, 0, (size_t)n * KM * sizeof(double), stream));
    CK(cudaMemsetAsync(st.W, 0, (size_t)N * KM * sizeof(double), stream));
    CK(cudaMemsetAsync(st.S, 0, KK * sizeof(double), stream));
    CK(cudaMemsetAsync(st.psi0, 0, (size_t)n * QM * sizeof(double), stream));
    CK(cudaMemsetAsync(st.psi1, 0, (size_t)n * QM * sizeof(double), stream));
    CK(cudaMemsetAsync(st.dose, 0, (size_t)n * sizeof(double), stream));
    init_factors_kernel<<<dim3(1, 1), 256, 0, stream>>>(s->d_st, n, N, s->P.nx, s->P.ny, r, s->nE);
    CK(cudaGetLastError());
    return TITUS_OK;
}

static int launch(titus_solver* s, int method, const titus_options_t* opt, int n_begin, int n_end, int dose2_pending,
                  cudaStream_t stream) {
    if (!is_fixed_family(method)) return fail(TITUS_ERR_ARG, "unknown method %d", method);
    if (s->r > KM)
        return fail(TITUS_ERR_LIMIT, "fixed-rank integrator: rank %d > %d supported by this build", s->r, KM);
    const bool ho = method == TITUS_DLR_HIGH_ORDER;
    if (ho && (s->P.nx < 5 || s->P.ny < 5))
        return fail(TITUS_ERR_ARG, "RK4 integrator: the limited flux needs nx, ny >= 5 (got %d x %d)", s->P.nx, s->P.ny);
    if (ho) {
        int rc = ensure_rk4_buffers(s);
        if (rc) return rc;
    }
    void* kfn = ho ? (void*)dlr_kernel<TITUS_DLR_HIGH_ORDER> : (void*)dlr_kernel<TITUS_DLR_FIXED>;
    int G = (opt && opt->team_ctas > 0) ? opt->team_ctas : s->team_ctas;
    G = std::min(G, s->num_sms);
    G = std::max(G, 1);
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, NT, sizeof(SmemLayout)));
    if (per_sm < 1) return fail(TITUS_ERR_CUDA, "kernel does not fit on an SM (smem %zu)", sizeof(SmemLayout));
    if (G > per_sm * s->num_sms) G = per_sm * s->num_sms;
    DevProblem P = s->P;
    if (opt && opt->rank_tol > 0) P.rank_tol = opt->rank_tol;
    P.prof = nullptr;
    P.zero_smem = getenv("TITUS_ZERO_SMEM") ? 1 : 0;
    s->take_debug_hooks(P);
    if (opt && opt->profile) {
        CK(cudaMemsetAsync(s->prof, 0, PF_SLOTS * sizeof(unsigned long long), stream));
        P.prof = s->prof;
    }
    CK(cudaMemsetAsync(s->st.bar, 0, (s->num_sms + 1) * sizeof(unsigned), stream));
    CK(cudaMemsetAsync(s->st.status, 0, sizeof(int), stream));
    CK(cudaMemsetAsync(s->st.diag, 0, 16 * sizeof(double), stream));
    TeamState* dst = s->d_st;
    void* args[] = {&P, &dst, &G, &n_begin, &n_end, &dose2_pending};
    CK(cudaLaunchCooperativeKernel(kfn, dim3(G), dim3(NT), args, sizeof(SmemLayout), stream));
    s->last_method = method;
    s->last_G = G;
    return TITUS_OK;
}

static int check_status(titus_solver* s) {
    CK(cudaDeviceSynchronize());
    int status = 0;
    CK(cudaMemcpy(&status, s->st.status, sizeof(int), cudaMemcpyDeviceToHost));
    if (status != 0) {
        const char* what = status == ST_BARRIER_TIMEOUT ? "team barrier timeout"
                           : status == ST_CHOL_BREAKDOWN ? "Cholesky breakdown in the range finder"
                           : status == ST_COMPLETION      ? "basis completion ran out of candidates"
                                                          : "device error";
        double d[16];
        CK(cudaMemcpy(d, s->st.diag, sizeof(d), cudaMemcpyDeviceToHost));
        if (status == ST_BARRIER_TIMEOUT) {
            unsigned counter = 0;
            CK(cudaMemcpy(&counter, s->st.bar + s->last_G, sizeof(unsigned), cudaMemcpyDeviceToHost));
            return fail(TITUS_ERR_DEVICE,
                        "device status %d: %s (CTA %g at barrier %g saw %g arrivals, wanted %g; counter now %u)",
                        status, what, d[8], d[14], d[9], d[10], counter);
        }
        if (status == ST_CHOL_BREAKDOWN)
            return fail(TITUS_ERR_DEVICE,
                        "device status %d: %s (stage %g side %g k %g pivot %g value %.3e G00 %.3e min diag %.3e step %g;"
                        " last range finder flags %g rhoK %g rhoL %g)",
                        status, what, d[0], d[1], d[2], d[3], d[4], d[5], d[6], d[7], d[11], d[12], d[13]);
        return fail(TITUS_ERR_DEVICE, "device status %d: %s", status, what);
    }
    return TITUS_OK;
}

static int end_index(const titus_solver* s, const titus_options_t* opt, int n_begin) {
    int n_end = s->nE;
    if (opt && opt->max_steps > 0) n_end = std::min(n_end, n_begin + opt->max_steps - 1);
    return n_end;
}

// precision must be a titus_precision_t; MIXED exists for the adaptive integrators only
static int check_precision(int method, const titus_options_t* opt) {
    const int p = opt ? opt->precision : TITUS_PRECISION_FP64;
    if (p != TITUS_PRECISION_FP64 && p != TITUS_PRECISION_MIXED) return fail(TITUS_ERR_ARG, "unknown precision %d", p);
    if (p == TITUS_PRECISION_MIXED && method != TITUS_PARALLEL_ADAPTIVE && method != TITUS_BUG_ADAPTIVE)
        return fail(TITUS_ERR_ARG, "MIXED precision applies to the adaptive integrators (method 1 or 2), got %d", method);
    return TITUS_OK;
}

extern "C" int titus_solve_device(titus_solver_t* s, int32_t method, const titus_options_t* opt, void* stream_) {
    if (!s) return fail(TITUS_ERR_ARG, "solver is NULL");
    if (int rc = reject_3d(s, "titus_solve", method)) return rc;
    if (int rc = check_precision(method, opt)) return rc;
    if (s->nz && opt && opt->precision != TITUS_PRECISION_FP64)
        return fail(TITUS_ERR_ARG, "3D problems run in FP64 (precision %d)", opt->precision);
    cudaStream_t stream = (cudaStream_t)stream_;
    if (is_wide_family(method)) {
        s->last_method = method;
        if (s->nz) return titus_host::wide_solve_device_3d(s, method, opt, stream);
        return titus_host::wide_solve_device(s, method, opt, stream);
    }
    if (!is_fixed_family(method)) return fail(TITUS_ERR_ARG, "unknown method %d", method);
    int rc = init_state(s, s->r, stream);
    if (rc) return rc;
    return launch(s, method, opt, 2, end_index(s, opt, 2), 0, stream);
}

extern "C" int titus_fetch(titus_solver_t* s, titus_result_t* res) {
    if (!s || !res) return fail(TITUS_ERR_ARG, "NULL argument");
    if (is_wide_family(s->last_method))
        return s->nz ? titus_host::wide_fetch_3d(s, res) : titus_host::wide_fetch(s, res);
    if (s->nz) return fail(TITUS_ERR_ARG, "titus_fetch: no DLR solve has run on this 3D handle");
    int rc = check_status(s);
    if (rc) return rc;
    int info[4];
    CK(cudaMemcpy(info, s->st.info, sizeof(info), cudaMemcpyDeviceToHost));
    const int k = info[0];
    res->rank = k;
    res->steps_done = info[1];
    if (res->dose) CK(cudaMemcpy(res->dose, s->st.dose, s->n * sizeof(double), cudaMemcpyDeviceToHost));
    const int rc_cap = res->r_cap;
    if ((res->X || res->S || res->W) && rc_cap < k) return fail(TITUS_ERR_ARG, "r_cap %d < rank %d", rc_cap, k);
    if (res->X)
        CK(cudaMemcpy2D(res->X, rc_cap * sizeof(double), s->st.X, KM * sizeof(double), k * sizeof(double), s->n,
                        cudaMemcpyDeviceToHost));
    if (res->W)
        CK(cudaMemcpy2D(res->W, rc_cap * sizeof(double), s->st.W, KM * sizeof(double), k * sizeof(double), s->N,
                        cudaMemcpyDeviceToHost));
    if (res->S)
        CK(cudaMemcpy2D(res->S, rc_cap * sizeof(double), s->st.S, KM * sizeof(double), k * sizeof(double), k,
                        cudaMemcpyDeviceToHost));
    if (res->psi) {
        double* src = info[2] ? s->st.psi1 : s->st.psi0;
        CK(cudaMemcpy2D(res->psi, s->q * sizeof(double), src, QM * sizeof(double), s->q * sizeof(double), s->n,
                        cudaMemcpyDeviceToHost));
    }
    if (res->rank_history) CK(cudaMemcpy(res->rank_history, s->st.rank_hist, s->nE * sizeof(int), cudaMemcpyDeviceToHost));
    if (res->eta_history) memset(res->eta_history, 0, s->nE * sizeof(double));
    if (res->bound_history) memset(res->bound_history, 0, s->nE * sizeof(double));
    if (res->time_history) memset(res->time_history, 0, s->nE * sizeof(double));
    return TITUS_OK;
}

extern "C" int titus_solve(titus_solver_t* s, int32_t method, const titus_options_t* opt, titus_result_t* res) {
    int rc = titus_solve_device(s, method, opt, nullptr);
    if (rc) return rc;
    return titus_fetch(s, res);
}

extern "C" int titus_solve_problem(const titus_problem_t* pb, int32_t method, const titus_options_t* opt,
                                   titus_result_t* res) {
    titus_solver_t* s = nullptr;
    int rc = titus_create(pb, &s);
    if (rc) return rc;
    rc = titus_solve(s, method, opt, res);
    titus_destroy(s);
    return rc;
}

extern "C" int titus_set_state(titus_solver_t* s, int32_t rank, const double* X, const double* S, const double* W,
                               const double* psi, const double* dose, int32_t n_next) {
    if (!s || !X || !S || !W || !psi || !dose) return fail(TITUS_ERR_ARG, "NULL argument");
    if (rank < 1 || rank > wide::RA) return fail(TITUS_ERR_LIMIT, "rank %d outside [1, %d]", rank, wide::RA);
    if (n_next < 2 || n_next > s->nE + 1) return fail(TITUS_ERR_ARG, "n_next %d outside [2, nE+1]", n_next);
    if (s->nz) return titus_host::wide_set_state_3d(s, rank, X, S, W, psi, dose, n_next);
    // the adaptive integrators' state always; the fixed-rank state when the rank fits
    int rcw = titus_host::wide_set_state(s, rank, X, S, W, psi, dose, n_next);
    if (rcw) return rcw;
    if (rank > KM) return TITUS_OK;
    TeamState& st = s->st;
    CK(cudaMemset(st.X, 0, (size_t)s->n * KM * sizeof(double)));
    CK(cudaMemset(st.W, 0, (size_t)s->N * KM * sizeof(double)));
    CK(cudaMemset(st.S, 0, KK * sizeof(double)));
    CK(cudaMemcpy2D(st.X, KM * sizeof(double), X, rank * sizeof(double), rank * sizeof(double), s->n,
                    cudaMemcpyHostToDevice));
    CK(cudaMemcpy2D(st.W, KM * sizeof(double), W, rank * sizeof(double), rank * sizeof(double), s->N,
                    cudaMemcpyHostToDevice));
    CK(cudaMemcpy2D(st.S, KM * sizeof(double), S, rank * sizeof(double), rank * sizeof(double), rank,
                    cudaMemcpyHostToDevice));
    CK(cudaMemset(st.psi0, 0, (size_t)s->n * QM * sizeof(double)));
    CK(cudaMemcpy2D(st.psi0, QM * sizeof(double), psi, s->q * sizeof(double), s->q * sizeof(double), s->n,
                    cudaMemcpyHostToDevice));
    CK(cudaMemcpy(st.dose, dose, s->n * sizeof(double), cudaMemcpyHostToDevice));
    int info[4] = {rank, 0, 0, n_next};
    CK(cudaMemcpy(st.info, info, sizeof(info), cudaMemcpyHostToDevice));
    CK(cudaMemset(st.rank_hist, 0xff, s->nE * sizeof(int)));
    return TITUS_OK;
}

extern "C" int titus_solve_from(titus_solver_t* s, int32_t method, const titus_options_t* opt, int32_t n_stop,
                                titus_result_t* res) {
    if (!s) return fail(TITUS_ERR_ARG, "solver is NULL");
    if (int rc = reject_3d(s, "titus_solve_from", method)) return rc;
    if (int rc = check_precision(method, opt)) return rc;
    if (is_wide_family(method)) {
        s->last_method = method;
        if (s->nz) {
            int rc = titus_host::wide_solve_from_3d(s, method, opt, n_stop);
            return rc ? rc : titus_host::wide_fetch_3d(s, res);
        }
        int rc = titus_host::wide_solve_from(s, method, opt, n_stop);
        if (rc) return rc;
        return titus_host::wide_fetch(s, res);
    }
    int info[4];
    CK(cudaMemcpy(info, s->st.info, sizeof(info), cudaMemcpyDeviceToHost));
    const int n_begin = info[3];
    int n_end = std::min(n_stop, end_index(s, opt, n_begin));
    if (n_end < n_begin) return fail(TITUS_ERR_ARG, "nothing to run (n_begin %d, n_stop %d)", n_begin, n_stop);
    // The state handed over by titus_set_state is taken after the second dose
    // half-step of step n_begin-1, so no dose half-step is pending.
    int rc = launch(s, method, opt, n_begin, n_end, 0, nullptr);
    if (rc) return rc;
    return titus_fetch(s, res);
}

extern "C" int titus_solve_batched(titus_solver_t* s, int32_t method, const titus_options_t* opt, int32_t nspots,
                                   const titus_spot_t* spots, double* dose_out, int32_t* rank_out, int32_t* iters_out) {
    if (!s || !spots || !dose_out) return fail(TITUS_ERR_ARG, "NULL argument");
    if (int rc = reject_3d(s, "titus_solve_batched")) return rc;
    if (method != TITUS_PARALLEL_ADAPTIVE && method != TITUS_BUG_ADAPTIVE)
        return fail(TITUS_ERR_ARG, "batched solves run the adaptive integrators (method 1 or 2), got %d", method);
    if (int rc = check_precision(method, opt)) return rc;
    if (nspots < 1) return fail(TITUS_ERR_ARG, "nspots < 1");
    s->last_method = method;
    return titus_host::wide_solve_batched(s, method, opt, nspots, spots, dose_out, rank_out, iters_out);
}

extern "C" int titus_batch_upload(titus_solver_t* s, int32_t nspots, const titus_spot_t* spots,
                                  titus_batch_t** out) {
    if (!s || !spots || !out) return fail(TITUS_ERR_ARG, "NULL argument");
    *out = nullptr;
    if (int rc = reject_3d(s, "titus_batch_upload")) return rc;
    if (nspots < 1) return fail(TITUS_ERR_ARG, "nspots < 1");
    return titus_host::batch_upload(s, nspots, spots, out);
}

extern "C" int titus_batch_solve_device(titus_batch_t* b, int32_t method, const titus_options_t* opt, void* stream) {
    if (!b) return fail(TITUS_ERR_ARG, "batch is NULL");
    if (method != TITUS_PARALLEL_ADAPTIVE && method != TITUS_BUG_ADAPTIVE)
        return fail(TITUS_ERR_ARG, "batched solves run the adaptive integrators (method 1 or 2), got %d", method);
    if (int rc = check_precision(method, opt)) return rc;
    return titus_host::batch_launch(b, method, opt, (cudaStream_t)stream);
}

extern "C" int titus_batch_fetch(titus_batch_t* b, double* dose_out, int32_t* rank_out, int32_t* iters_out) {
    if (!b) return fail(TITUS_ERR_ARG, "batch is NULL");
    return titus_host::batch_fetch(b, dose_out, rank_out, iters_out);
}

extern "C" int titus_batch_rank_sums(titus_batch_t* b, int32_t* out) {
    if (!b || !out) return fail(TITUS_ERR_ARG, "NULL argument");
    return titus_host::batch_rank_sums(b, out);
}

extern "C" void titus_batch_destroy(titus_batch_t* b) {
    if (b) titus_host::batch_free(b);
}

extern "C" void titus_destroy(titus_solver_t* s) { delete s; }

extern "C" int titus_last_error(char* buf, size_t len) {
    if (!buf || len == 0) return TITUS_ERR_ARG;
    snprintf(buf, len, "%s", g_last_error.c_str());
    return TITUS_OK;
}

extern "C" int titus_profile(titus_solver_t* s, double* ns, int32_t n) {
    if (!s || !ns || n < 0) return fail(TITUS_ERR_ARG, "NULL argument");
    unsigned long long cyc[PF_SLOTS];
    CK(cudaMemcpy(cyc, s->prof, sizeof(cyc), cudaMemcpyDeviceToHost));
    // [0, PF_COUNT): phase times (ns); then event counts: SVD sweeps, SVD calls,
    // eigensolver calls, eigensolver sweeps, Cholesky calls, rank-revealing and
    // certified range-finder sides, team barriers
    const int counters[] = {PF_SVD_SWEEPS, PF_SVD_CALLS, PF_EIG_CALLS, PF_EIG_SWEEPS, PF_CHOL_CALLS, PF_RF_SLOW,
                            PF_RF_FAST, PF_BARRIERS};
    const int nc = (int)(sizeof(counters) / sizeof(counters[0]));
    int m = 0;
    for (int i = 0; i < PF_COUNT && m < n; ++i, ++m) ns[m] = (double)cyc[i] * 1e6 / (double)s->clock_khz;
    for (int i = 0; i < nc && m < n; ++i, ++m) ns[m] = (double)cyc[counters[i]];
    return m;
}

extern "C" int titus_resume_point(titus_solver_t* s, int32_t* n_next, double* t) {
    if (!s || !n_next) return fail(TITUS_ERR_ARG, "NULL argument");
    CK(cudaDeviceSynchronize());
    if (is_wide_family(s->last_method) || (s->last_method < 0 && s->wide_state_valid)) {
        if (!s->d_wst) return fail(TITUS_ERR_ARG, "no solver state yet");
        int info[8];
        CK(cudaMemcpy(info, s->wst.info, sizeof(info), cudaMemcpyDeviceToHost));
        *n_next = info[3];
        if (t) CK(cudaMemcpy(t, s->wst.tvar, sizeof(double), cudaMemcpyDeviceToHost));
        return TITUS_OK;
    }
    int info[4];
    CK(cudaMemcpy(info, s->st.info, sizeof(info), cudaMemcpyDeviceToHost));
    *n_next = info[3];
    if (t) *t = (info[3] - 2) * s->P.dE;
    return TITUS_OK;
}

extern "C" int titus_debug_barrier_fault(titus_solver_t* s, int32_t barrier, int64_t spin_limit) {
    if (!s) return fail(TITUS_ERR_ARG, "solver is NULL");
    if (spin_limit < 0) return fail(TITUS_ERR_ARG, "spin_limit < 0");
    s->dbg_fault_barrier = barrier > 0 ? barrier : 0;
    s->dbg_spin_limit = spin_limit;
    return TITUS_OK;
}

extern "C" int titus_debug_fail_alloc(int32_t after) {
    if (after < 0) return fail(TITUS_ERR_ARG, "after < 0");
    g_alloc_fault.store(after);
    return TITUS_OK;
}

extern "C" int titus_max_rank(void) { return 2 * wide::RA; }
extern "C" int titus_max_ordinates(void) { return QM < KM ? QM : KM; }
extern "C" const char* titus_version(void) { return "titus-b200 0.1 (sm_100a, FP64)"; }
