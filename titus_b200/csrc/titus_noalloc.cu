// titus_solve_noalloc: the fixed-rank energy loop for callers that may not
// allocate device memory.
//
// Some callers cannot call cudaMalloc: their device memory belongs to a host
// framework's allocator or memory pool, or they run under a policy that forbids
// device allocation once the application has started. This entry point takes
// the problem arrays and the output buffers as device pointers the caller
// already owns, and keeps every intermediate (the working factors, the second
// psi buffer, the range-finder buffers, the partial reductions, the team
// barrier flags and the status words) in one file-scope device array of fixed
// size, kNoAllocScratchBytes. It calls no cudaMalloc, cudaFree or other
// allocating routine, host or device.
//
// Consequences for the caller:
//  * every GPU that loads libtitus.so holds this array until the process exits;
//  * all calls on a device share the array: calls that overlap on the GPU race
//    with each other, so serialise them (one call at a time per device);
//  * the array keeps the previous call's contents; everything that must start
//    at zero is cleared at the start of each call;
//  * every call looks the array's device address up with the caller's device
//    current (cudaGetSymbolAddress; nothing is cached, so concurrent first calls
//    from several host threads and a cudaDeviceReset between calls are safe);
//  * the call is synchronous: it reads e_trafo[0..1] back to the host before the
//    launch and the status words after it, then waits for `stream`;
//  * a problem fits when 913 n + 580 N + 4 nE + 73 728 G + 48 KiB <= 16 MiB
//    bytes (n cells, N moments, nE energies, G CTAs; 256-byte alignment of each
//    piece included in the constant): about 16 700 cells at P21 with G = 16.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>

#include "../../include/titus.h"
#include "dlr_fixed.cuh"

using namespace titus;

namespace {

constexpr size_t kNoAllocScratchBytes = 16u << 20;  // 16 MiB per device
constexpr int kNoAllocMaxTeam = 32;                 // CTAs per solve in this variant

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// The host-side symbol g_noalloc_scratch is only a stand-in: kernels get the
// device address that cudaGetSymbolAddress returns for the current device.

// Error text goes to the caller's buffer (no library-side storage).
struct ErrOut {
    char* buf;
    size_t len;
    int set(int code, const char* msg) const {
        if (buf && len) snprintf(buf, len, "%s", msg);
        return code;
    }
};

#define NA_CK(call)                                                                                  \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess) {                                                                     \
            if (eo.buf && eo.len) snprintf(eo.buf, eo.len, "%s: %s", #call, cudaGetErrorString(e_)); \
            return TITUS_ERR_CUDA;                                                                   \
        }                                                                                            \
    } while (0)

// Bump layout inside the scratch array (256-byte aligned pieces).
struct Carve {
    unsigned char* base;
    size_t off;
    template <class T>
    T* take(size_t count) {
        off = (off + 255) & ~size_t(255);
        T* p = reinterpret_cast<T*>(base + off);
        off += count * sizeof(T);
        return p;
    }
};

// Derived per-problem arrays: 1/density, Legendre order of each moment,
// zeroed restore mask (set afterwards from the caller's list).
__global__ void na_prep_kernel(const double* density, double* rinv, int n, int32_t* lof, int N, uint8_t* restore) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    for (int i = tid; i < n; i += stride) {
        rinv[i] = 1.0 / density[i];
        restore[i] = 0;
    }
    for (int m = tid; m < N; m += stride) {
        int l = (int)sqrt((double)m);
        while (l * l > m) --l;
        while ((l + 1) * (l + 1) <= m) ++l;
        lof[m] = l;
    }
}

__global__ void na_restore_kernel(uint8_t* restore, const int32_t* restore_list, int n_restore, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_restore; i += gridDim.x * blockDim.x) {
        const int c = restore_list[i];
        if (c >= 0 && c < n) restore[c] = 1;
    }
}

// Initial factors (first r identity columns, boundary rows of X zeroed) and loop counters.
__global__ void na_init_kernel(const TeamState* st_ptr, int n, int N, int nx, int ny, int r, int nE) {
    const TeamState st = *st_ptr;
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

// Copy the working factors (leading dimension KM / QM) to the caller's
// outputs (leading dimension r / q); psi from the buffer the loop ended in.
__global__ void na_out_kernel(const TeamState* st_ptr, int n, int N, int q, int r, double* dose, double* X,
                              double* S, double* W, double* psi) {
    const TeamState st = *st_ptr;
    const double* psrc = st.info[2] ? st.psi1 : st.psi0;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    for (int i = tid; i < n; i += stride) dose[i] = st.dose[i];
    for (long long e = tid; e < (long long)n * r; e += stride) X[e] = st.X[(e / r) * KM + e % r];
    for (long long e = tid; e < (long long)N * r; e += stride) W[e] = st.W[(e / r) * KM + e % r];
    for (int e = tid; e < r * r; e += stride) S[e] = st.S[(e / r) * KM + e % r];
    for (long long e = tid; e < (long long)n * q; e += stride) psi[e] = psrc[(e / q) * QM + e % q];
}

}  // namespace

extern "C" int titus_solve_noalloc(const titus_problem_t* pb, const titus_options_t* opt, double* dose, double* X,
                                   double* S, double* W, double* psi, int32_t* rank_out, void* stream_, char* err,
                                   size_t err_len) {
    const ErrOut eo{err, err_len};
    if (err && err_len) err[0] = '\0';
    if (!pb || !dose || !X || !S || !W || !psi) return eo.set(TITUS_ERR_ARG, "titus_solve_noalloc: NULL argument");
    if (pb->nx < 3 || pb->ny < 3) return eo.set(TITUS_ERR_ARG, "titus_solve_noalloc: need nx, ny >= 3");
    if (pb->npn < 0 || pb->n_moments != (pb->npn + 1) * (pb->npn + 1))
        return eo.set(TITUS_ERR_ARG, "titus_solve_noalloc: n_moments != (npn+1)^2");
    if (pb->n_ordinates < 1 || pb->n_ordinates > (QM < KM ? QM : KM))
        return eo.set(TITUS_ERR_LIMIT, "titus_solve_noalloc: n_ordinates outside [1, 24]");
    if (pb->r < 1 || pb->r > KM || pb->r > pb->n_moments)
        return eo.set(TITUS_ERR_LIMIT, "titus_solve_noalloc: r outside [1, min(24, n_moments)]");
    if (pb->n_energies < 2) return eo.set(TITUS_ERR_ARG, "titus_solve_noalloc: n_energies < 2");
    if (!(pb->dx > 0) || !(pb->dy > 0)) return eo.set(TITUS_ERR_ARG, "titus_solve_noalloc: dx, dy must be > 0");
    const void* req[] = {pb->density, pb->e_trafo, pb->stopping, pb->bc_energy, pb->sigma,
                         pb->bc_space, pb->bc_angle, pb->omega, pb->m_reduced};
    for (const void* p : req)
        if (!p) return eo.set(TITUS_ERR_ARG, "titus_solve_noalloc: a required problem array is NULL");
    for (int d = 0; d < 4; ++d)
        if (!pb->op_rowptr[d] || !pb->op_col[d] || !pb->op_val[d])
            return eo.set(TITUS_ERR_ARG, "titus_solve_noalloc: operator CSR arrays missing");
    if (pb->n_x_completion < 0 || pb->n_w_completion < 0 || pb->n_sweep_restore < 0)
        return eo.set(TITUS_ERR_ARG, "titus_solve_noalloc: negative list length");
    if (pb->n_sweep_restore > 0 && !pb->sweep_restore)
        return eo.set(TITUS_ERR_ARG, "titus_solve_noalloc: sweep_restore is NULL");
    if ((pb->n_x_completion > 0 && !pb->x_completion) || (pb->n_w_completion > 0 && !pb->w_completion))
        return eo.set(TITUS_ERR_ARG, "titus_solve_noalloc: completion list is NULL");
    cudaStream_t stream = (cudaStream_t)stream_;

    int dev = 0;
    NA_CK(cudaGetDevice(&dev));
    // the array's device address on this device (neither call allocates)
    void* scratch_addr = nullptr;
    NA_CK(cudaGetSymbolAddress(&scratch_addr, g_noalloc_scratch));
    if (!scratch_addr) return eo.set(TITUS_ERR_CUDA, "titus_solve_noalloc: scratch address lookup returned NULL");
    NA_CK(cudaFuncSetAttribute(dlr_kernel<TITUS_DLR_FIXED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(SmemLayout)));
    int num_sms = 0;
    NA_CK(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
    int G = (opt && opt->team_ctas > 0) ? opt->team_ctas : 16;
    if (G > kNoAllocMaxTeam) G = kNoAllocMaxTeam;
    if (G > num_sms) G = num_sms;

    const int n = pb->nx * pb->ny, N = pb->n_moments, q = pb->n_ordinates, nE = pb->n_energies;
    // carve the scratch array; reject problems that do not fit
    Carve cv{static_cast<unsigned char*>(scratch_addr), 0};
    TeamState st{};
    TeamState* d_st = cv.take<TeamState>(1);
    st.X = cv.take<double>((size_t)n * KM);
    st.K = cv.take<double>((size_t)n * KM);
    st.W = cv.take<double>((size_t)N * KM);
    st.L = cv.take<double>((size_t)2 * N * KM);
    st.psi0 = cv.take<double>((size_t)n * QM);
    st.psi1 = cv.take<double>((size_t)n * QM);
    st.dose = cv.take<double>(n);
    st.S = cv.take<double>(KK);
    st.part = cv.take<double>((size_t)2 * G * PMAX);
    st.red = cv.take<double>(PMAX);
    st.bar = cv.take<unsigned>(G + 1);
    st.status = cv.take<int>(1);
    st.info = cv.take<int>(4);
    st.rank_hist = cv.take<int>(nE);
    st.diag = cv.take<double>(16);
    st.eta_hist = st.bound_hist = st.time_hist = nullptr;
    double* rinv = cv.take<double>(n);
    int32_t* lof = cv.take<int32_t>(N);
    uint8_t* restore = cv.take<uint8_t>(n);
    if (cv.off > kNoAllocScratchBytes) {
        if (err && err_len)
            snprintf(err, err_len,
                     "titus_solve_noalloc: problem needs %zu bytes of scratch, the static array holds %zu "
                     "(reduce cells, moments or energy steps)",
                     cv.off, kNoAllocScratchBytes);
        return TITUS_ERR_LIMIT;
    }

    DevProblem P{};
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
    P.theta = pb->theta;
    P.theta_index = pb->theta_index;
    P.c_eta = pb->c_eta;
    P.rank_tol = (opt && opt->rank_tol > 0) ? opt->rank_tol : 1e-12;
    // dE = eTrafo[2] - eTrafo[1] (1-based): read the two values into stack memory
    double et[2];
    NA_CK(cudaMemcpyAsync(et, pb->e_trafo, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream));
    NA_CK(cudaStreamSynchronize(stream));
    P.dE = et[1] - et[0];
    P.rinv = rinv;
    P.stopping = pb->stopping;
    P.bc_energy = pb->bc_energy;
    P.sigma = pb->sigma;
    P.bc_space = pb->bc_space;
    P.bc_angle = pb->bc_angle;
    P.omega = pb->omega;
    P.mred = pb->m_reduced;
    P.lof = lof;
    for (int d = 0; d < 4; ++d) {
        P.op[d].rowptr = pb->op_rowptr[d];
        P.op[d].col = pb->op_col[d];
        P.op[d].val = pb->op_val[d];
    }
    P.xcomp = pb->x_completion;
    P.nxcomp = pb->n_x_completion;
    P.wcomp = pb->w_completion;
    P.nwcomp = pb->n_w_completion;
    P.restore = restore;
    P.prof = nullptr;
    P.zero_smem = 0;

    // clear what must start at zero, then derived arrays and initial factors
    NA_CK(cudaMemcpyAsync(d_st, &st, sizeof(TeamState), cudaMemcpyHostToDevice, stream));
    NA_CK(cudaMemsetAsync(st.X, 0, (size_t)n * KM * sizeof(double), stream));
    NA_CK(cudaMemsetAsync(st.W, 0, (size_t)N * KM * sizeof(double), stream));
    NA_CK(cudaMemsetAsync(st.S, 0, KK * sizeof(double), stream));
    NA_CK(cudaMemsetAsync(st.psi0, 0, (size_t)n * QM * sizeof(double), stream));
    NA_CK(cudaMemsetAsync(st.psi1, 0, (size_t)n * QM * sizeof(double), stream));
    NA_CK(cudaMemsetAsync(st.dose, 0, (size_t)n * sizeof(double), stream));
    NA_CK(cudaMemsetAsync(st.bar, 0, (G + 1) * sizeof(unsigned), stream));
    NA_CK(cudaMemsetAsync(st.status, 0, sizeof(int), stream));
    NA_CK(cudaMemsetAsync(st.diag, 0, 16 * sizeof(double), stream));
    na_prep_kernel<<<64, 256, 0, stream>>>(pb->density, rinv, n, lof, N, restore);
    NA_CK(cudaGetLastError());
    if (pb->n_sweep_restore > 0) {
        na_restore_kernel<<<8, 256, 0, stream>>>(restore, pb->sweep_restore, pb->n_sweep_restore, n);
        NA_CK(cudaGetLastError());
    }
    na_init_kernel<<<1, 256, 0, stream>>>(d_st, n, N, pb->nx, pb->ny, pb->r, nE);
    NA_CK(cudaGetLastError());

    int per_sm = 0;
    NA_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dlr_kernel<TITUS_DLR_FIXED>, NT, sizeof(SmemLayout)));
    if (per_sm < 1) return eo.set(TITUS_ERR_CUDA, "titus_solve_noalloc: kernel does not fit on an SM");
    int n_begin = 2;
    int n_end = nE;
    if (opt && opt->max_steps > 0 && n_begin + opt->max_steps - 1 < n_end) n_end = n_begin + opt->max_steps - 1;
    int pending = 0;
    void* args[] = {&P, &d_st, &G, &n_begin, &n_end, &pending};
    NA_CK(cudaLaunchCooperativeKernel((void*)dlr_kernel<TITUS_DLR_FIXED>, dim3(G), dim3(NT), args,
                                      sizeof(SmemLayout), stream));
    na_out_kernel<<<128, 256, 0, stream>>>(d_st, n, N, q, pb->r, dose, X, S, W, psi);
    NA_CK(cudaGetLastError());
    int status = 0;
    int info[4] = {0, 0, 0, 0};
    NA_CK(cudaMemcpyAsync(&status, st.status, sizeof(int), cudaMemcpyDeviceToHost, stream));
    NA_CK(cudaMemcpyAsync(info, st.info, sizeof(info), cudaMemcpyDeviceToHost, stream));
    NA_CK(cudaStreamSynchronize(stream));
    if (status != 0) {
        if (err && err_len) snprintf(err, err_len, "titus_solve_noalloc: device status %d", status);
        return TITUS_ERR_DEVICE;
    }
    if (rank_out) *rank_out = info[0];
    return TITUS_OK;
}
