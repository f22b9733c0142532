// Full-rank P_N first-collision solver on a 3D grid: the z extension of
// SolveFirstCollisionSource (code/SolverCSD.jl:465-586; the reference itself
// is 2D only). Cell (i, j, k) has row (k*nx + i)*ny + j; the boundary (ghost)
// cells are those on any face. Six streaming pairs, summed in this order:
//   (L2x, Ax), (L2y, Az), (L1x, |Ax|), (L1y, |Az|), (L2z, Ay), (L1z, |Ay|)
// -- the 2D list with the z pair appended; spatial z streams with Ay and the
// sweep's z term uses Omega_y.
//
// One energy step n is two kernels on one stream:
//   pn3_psi_kernel     beam inflow at energy[n] (csd.S[n-1]) formed where it is
//                      read, upwind sweep of the interior cells in x, y and z,
//                      psi <- (psi - dE flux) / (1 + dE sigma_0);
//   pn3_stream_kernel  uTilde = u - dE sum_d (L_d u) A_d, collision
//                      (1 + dE D)^{-1}, in-scattering dE Dvec (MReduced psi),
//                      boundary rows zero, and the dose with csd.SMid. The
//                      stencils act on cells and A_d on moments, so they
//                      commute: a CTA forms the stencil images (L_d u)[c][:]
//                      of its CB cells in shared memory from the neighbour rows
//                      of u (L2 resident: the z neighbours are one layer away),
//                      then applies the rows of A_d^T. No n x N intermediate
//                      goes through HBM: per step u is read once and u' written
//                      once (16 n N bytes), plus psi.
// The whole sweep is captured once into a CUDA graph and launched as one unit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "titus_handle.h"

using namespace titus;
using titus_host::fail;

namespace {

constexpr int P3_NT = 256;
constexpr int P3_NOP = 6;
constexpr int P3_CBM = 8;   // most cells per CTA of pn3_stream_kernel
constexpr size_t P3_SMEM_MAX = 100 * 1024;   // stencil images per CTA (two CTAs per SM)

struct Pn3Args {
    int nx, ny, nz, nxy, n, N, q, npn, nE, cb;
    double dx, dy, dz, dE;
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
    const int32_t* tp[P3_NOP];   // CSR of A_d^T (row m lists (p, A_d[p][m]) in increasing p)
    const int32_t* ti[P3_NOP];
    const double* tv[P3_NOP];
};

__device__ __forceinline__ bool p3_bnd(const Pn3Args& a, int c) {
    const int k = c / a.nxy, r = c - k * a.nxy;
    const int i = r / a.ny, j = r - i * a.ny;
    return k == 0 || k == a.nz - 1 || i == 0 || i == a.nx - 1 || j == 0 || j == a.ny - 1;
}

// psi_out = (psi - dE flux) / (1 + dE sigma_0) for every cell and ordinate; the
// boundary cells hold the inflow PsiBeam(Omega_k, energy[n], x, y, z, n-1) and
// have zero flux.
__global__ void __launch_bounds__(P3_NT) pn3_psi_kernel(Pn3Args a, int n, const double* __restrict__ psi_in,
                                                        double* __restrict__ psi_out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.n * a.q) return;
    const int c = e / a.q, k = e - (e / a.q) * a.q;
    const double bcf = a.bc_energy[n - 1] / a.stopping[n - 1] * a.stopping[n - 2];
    const double ang = a.bc_angle[k];
    auto val = [&](int cc) -> double {
        return p3_bnd(a, cc) ? bcf * a.bc_space[cc] * ang : psi_in[(size_t)cc * QM + k];
    };
    const double pc = val(c);
    double flux = 0.0;
    if (!p3_bnd(a, c)) {
        const double ox = a.omega[k * 3 + 0], oy = a.omega[k * 3 + 1], oz = a.omega[k * 3 + 2];
        const double ew = ox >= 0.0 ? pc - val(c - a.ny) : val(c + a.ny) - pc;
        const double ns = oz >= 0.0 ? pc - val(c - 1) : val(c + 1) - pc;
        const double tb = oy >= 0.0 ? pc - val(c - a.nxy) : val(c + a.nxy) - pc;
        flux = (ox / a.dx) * ew + (oz / a.dy) * ns + (oy / a.dz) * tb;
    }
    const double sig0 = a.sigma[(size_t)(n - 1) * (a.npn + 1)];
    psi_out[(size_t)c * QM + k] = (pc - a.dE * flux) / (1.0 + a.dE * sig0);
}

// u_out[c][m] for the CTA's CB consecutive cells; the dose on the m = 0 thread.
__global__ void __launch_bounds__(P3_NT) pn3_stream_kernel(Pn3Args a, int n, const double* __restrict__ u,
                                                           const double* __restrict__ psi,
                                                           double* __restrict__ u_out, double* __restrict__ dose) {
    extern __shared__ __align__(16) double img[];   // [P3_NOP][cb][N]: (L_d u)[c][p]
    const int N = a.N, cb = a.cb;
    const int c0 = blockIdx.x * cb;
    const int nc = min(cb, a.n - c0);
    // stencil entries as the reference's sparse rows (stencils.jl:26-128)
    const double hx = -1.0 / 2.0 / a.dx, hy = -1.0 / 2.0 / a.dy, hz = -1.0 / 2.0 / a.dz;
    const double gx = 2.0 / 2.0 / a.dx, gy = 2.0 / 2.0 / a.dy, gz = 2.0 / 2.0 / a.dz;
    for (int e = threadIdx.x; e < nc * N; e += blockDim.x) {
        const int cl = e / N, p = e - (e / N) * N;
        const int c = c0 + cl;
        double v[P3_NOP];
#pragma unroll
        for (int d = 0; d < P3_NOP; ++d) v[d] = 0.0;
        if (!p3_bnd(a, c)) {
            const int xm = c - a.ny, xp = c + a.ny, ym = c - 1, yp = c + 1, zm = c - a.nxy, zp = c + a.nxy;
            auto ld = [&](int cc) { return __ldg(u + (size_t)cc * N + p); };
            const double u0 = ld(c), uxm = ld(xm), uxp = ld(xp), uym = ld(ym), uyp = ld(yp), uzm = ld(zm),
                         uzp = ld(zp);
            const double rxm = __ldg(a.rinv + xm), rxp = __ldg(a.rinv + xp), rym = __ldg(a.rinv + ym),
                         ryp = __ldg(a.rinv + yp), rzm = __ldg(a.rinv + zm), rzp = __ldg(a.rinv + zp),
                         r0 = __ldg(a.rinv + c);
            v[0] = (hx * rxm) * uxm + (-hx * rxp) * uxp;
            v[1] = (hy * rym) * uym + (-hy * ryp) * uyp;
            v[2] = (hx * rxm) * uxm + (gx * r0) * u0 + (hx * rxp) * uxp;
            v[3] = (hy * rym) * uym + (gy * r0) * u0 + (hy * ryp) * uyp;
            v[4] = (hz * rzm) * uzm + (-hz * rzp) * uzp;
            v[5] = (hz * rzm) * uzm + (gz * r0) * u0 + (hz * rzp) * uzp;
        }
#pragma unroll
        for (int d = 0; d < P3_NOP; ++d) img[((size_t)d * cb + cl) * N + p] = v[d];
    }
    __syncthreads();
    const double dE = a.dE;
    const double* sg = a.sigma + (size_t)(n - 1) * (a.npn + 1);
    // a thread owns moment m for all of the CTA's cells: each nonzero of row m
    // of A_d^T is loaded once and applied to the cb cells' images (independent
    // FMAs), as in the moment-product kernel of the 2D solver
    for (int m = threadIdx.x; m < N; m += blockDim.x) {
        double ut[P3_CBM];
#pragma unroll
        for (int cl = 0; cl < P3_CBM; ++cl) ut[cl] = cl < nc ? u[(size_t)(c0 + cl) * N + m] : 0.0;
#pragma unroll
        for (int d = 0; d < P3_NOP; ++d) {
            const double* im = img + (size_t)d * cb * N;
            double sd[P3_CBM];
#pragma unroll
            for (int cl = 0; cl < P3_CBM; ++cl) sd[cl] = 0.0;
            const int q1 = __ldg(a.tp[d] + m + 1);
            for (int qq = __ldg(a.tp[d] + m); qq < q1; ++qq) {
                const double v = __ldg(a.tv[d] + qq);
                const double* col = im + __ldg(a.ti[d] + qq);
#pragma unroll
                for (int cl = 0; cl < P3_CBM; ++cl)
                    if (cl < cb) sd[cl] = fma(v, col[(size_t)cl * N], sd[cl]);
            }
#pragma unroll
            for (int cl = 0; cl < P3_CBM; ++cl) ut[cl] = ut[cl] - dE * sd[cl];
        }
        const double dv = sg[a.lof[m]];
        const double D = sg[0] - dv;
#pragma unroll
        for (int cl = 0; cl < P3_CBM; ++cl) {
            if (cl >= nc) continue;
            const int c = c0 + cl;
            const size_t ix = (size_t)c * N + m;
            if (p3_bnd(a, c)) {
                u_out[ix] = 0.0;
                continue;
            }
            const double* pr = psi + (size_t)c * QM;
            double src = 0.0;
            for (int k = 0; k < a.q; ++k) src = fma(a.mred[(size_t)m * a.q + k], pr[k], src);
            const double un = (ut[cl] + dE * dv * src) / (1.0 + dE * D);
            u_out[ix] = un;
            if (m == 0) {
                double unc = 0.0;
                for (int k = 0; k < a.q; ++k) unc = fma(pr[k], a.mred[k], unc);
                const double half = (n == 2 || n == a.nE) ? 2.0 : 1.0;
                dose[c] += dE * (un + unc) * a.smid[n - 2] * a.rinv[c] / half;
            }
        }
    }
}

}  // namespace

struct titus_pn3_state {
    double *u[2] = {nullptr, nullptr}, *psi[2] = {nullptr, nullptr}, *dose = nullptr;
    int32_t* tp[P3_NOP] = {};
    int32_t* ti[P3_NOP] = {};
    double* tv[P3_NOP] = {};
    int cb = 1;
    size_t smem = 0;
    int cur_u = 0, cur_psi = 0;
    int steps_done = 0;
    bool have_result = false;
    cudaStream_t cap = nullptr;
    cudaGraphExec_t exec = nullptr;
    int exec_n_end = -1;
    std::vector<void*> allocs;
    ~titus_pn3_state() {
        if (exec) cudaGraphExecDestroy(exec);
        for (void* p : allocs) cudaFree(p);
        if (cap) cudaStreamDestroy(cap);
    }
};

namespace {

template <class T>
int p3_alloc(titus_pn3_state* st, T** p, size_t count, const T* host = nullptr) {
    int rc = titus_host::upload(p, host, count);
    if (rc == TITUS_OK && *p) st->allocs.push_back((void*)*p);
    return rc;
}

// CSR of A^T on the device from the device CSR of A (N x N).
int p3_transpose(titus_pn3_state* st, const Csr& op, int N, int d) {
    std::vector<int32_t> rp(N + 1);
    cudaError_t e = cudaMemcpy(rp.data(), op.rowptr, (N + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost);
    const int nnz = e == cudaSuccess ? rp[N] : 0;
    std::vector<int32_t> ci(nnz);
    std::vector<double> v(nnz);
    if (e == cudaSuccess && nnz) e = cudaMemcpy(ci.data(), op.col, nnz * sizeof(int32_t), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && nnz) e = cudaMemcpy(v.data(), op.val, nnz * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(TITUS_ERR_CUDA, "operator download: %s", cudaGetErrorString(e));
    std::vector<int32_t> tp(N + 1, 0), ti(std::max(nnz, 1));
    std::vector<double> tv(std::max(nnz, 1));
    for (int q = 0; q < nnz; ++q) ++tp[ci[q] + 1];
    for (int m = 0; m < N; ++m) tp[m + 1] += tp[m];
    std::vector<int32_t> pos(tp.begin(), tp.end() - 1);
    for (int p = 0; p < N; ++p)
        for (int q = rp[p]; q < rp[p + 1]; ++q) {
            const int dst = pos[ci[q]]++;
            ti[dst] = p;
            tv[dst] = v[q];
        }
    int rc;
    if ((rc = p3_alloc(st, &st->tp[d], (size_t)N + 1, tp.data())) ||
        (rc = p3_alloc(st, &st->ti[d], ti.size(), ti.data())) || (rc = p3_alloc(st, &st->tv[d], tv.size(), tv.data())))
        return rc;
    return TITUS_OK;
}

int pn3_ensure(titus_solver* s) {
    if (s->pn3) return TITUS_OK;
    if (!s->smid) return fail(TITUS_ERR_ARG, "the full-rank P_N solver needs problem->stopping_mid (csd.SMid)");
    if ((long long)s->n * s->q >= (1LL << 31)) return fail(TITUS_ERR_LIMIT, "n * q >= 2^31");
    auto* st = new titus_pn3_state();
    const size_t nN = (size_t)s->n * s->N;
    int rc;
    if ((rc = p3_alloc(st, &st->u[0], nN)) || (rc = p3_alloc(st, &st->u[1], nN)) ||
        (rc = p3_alloc(st, &st->psi[0], (size_t)s->n * QM)) || (rc = p3_alloc(st, &st->psi[1], (size_t)s->n * QM)) ||
        (rc = p3_alloc(st, &st->dose, (size_t)s->n))) {
        delete st;
        return rc;
    }
    const Csr ops[P3_NOP] = {s->P.op[0], s->P.op[1], s->P.op[2], s->P.op[3], s->op3[0], s->op3[1]};
    for (int d = 0; d < P3_NOP; ++d)
        if ((rc = p3_transpose(st, ops[d], s->N, d))) {
            delete st;
            return rc;
        }
    // cells per CTA: as many (up to P3_CBM) as keep the six stencil images within the budget
    st->cb = P3_CBM;
    while (st->cb > 1 && (size_t)P3_NOP * st->cb * s->N * sizeof(double) > P3_SMEM_MAX) st->cb /= 2;
    st->smem = (size_t)P3_NOP * st->cb * s->N * sizeof(double);
    if (st->smem > 200 * 1024) {
        delete st;
        return fail(TITUS_ERR_LIMIT, "N = %d moments exceed the 3D solver's shared-memory tile", s->N);
    }
    cudaError_t e = cudaStreamCreateWithFlags(&st->cap, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(pn3_stream_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)st->smem);
    if (e != cudaSuccess) {
        delete st;
        return fail(TITUS_ERR_CUDA, "3D full-rank solver set-up: %s", cudaGetErrorString(e));
    }
    s->pn3 = st;
    return TITUS_OK;
}

Pn3Args pn3_args(const titus_solver* s, const titus_pn3_state* st) {
    const DevProblem& P = s->P;
    Pn3Args a{};
    a.nx = P.nx;
    a.ny = P.ny;
    a.nz = s->nz;
    a.nxy = P.nx * P.ny;
    a.n = P.n;
    a.N = P.N;
    a.q = P.q;
    a.npn = P.npn;
    a.nE = P.nE;
    a.cb = st->cb;
    a.dx = P.dx;
    a.dy = P.dy;
    a.dz = s->dz;
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
    for (int d = 0; d < P3_NOP; ++d) {
        a.tp[d] = st->tp[d];
        a.ti[d] = st->ti[d];
        a.tv[d] = st->tv[d];
    }
    return a;
}

}  // namespace

void titus_host::pn3_free(titus_solver* s) {
    delete s->pn3;
    s->pn3 = nullptr;
}

int titus_host::pn3_solve_device(titus_solver* s, const titus_options_t* opt, cudaStream_t stream) {
    int rc = pn3_ensure(s);
    if (rc) return rc;
    titus_pn3_state* st = s->pn3;
    const size_t nN = (size_t)s->n * s->N;
    int n_end = s->nE;
    if (opt && opt->max_steps > 0) n_end = std::min(n_end, 1 + opt->max_steps);
    CK(cudaMemsetAsync(st->u[0], 0, nN * sizeof(double), stream));
    CK(cudaMemsetAsync(st->psi[0], 0, (size_t)s->n * QM * sizeof(double), stream));
    CK(cudaMemsetAsync(st->dose, 0, (size_t)s->n * sizeof(double), stream));
    const int par_end = (n_end - 1) & 1;
    if (st->exec && st->exec_n_end == n_end) {
        CK(cudaGraphLaunch(st->exec, stream));
    } else {
        if (st->exec) {
            CK(cudaStreamSynchronize(stream));   // the old graph may still be running
            cudaGraphExecDestroy(st->exec);
            st->exec = nullptr;
            st->exec_n_end = -1;
        }
        const Pn3Args a = pn3_args(s, st);
        CK(cudaStreamBeginCapture(st->cap, cudaStreamCaptureModeThreadLocal));
        int cu = 0;
        const int gpsi = (int)((s->n * (size_t)s->q + P3_NT - 1) / P3_NT);
        const int gst = (s->n + st->cb - 1) / st->cb;
        for (int n = 2; n <= n_end; ++n) {
            pn3_psi_kernel<<<gpsi, P3_NT, 0, st->cap>>>(a, n, st->psi[cu], st->psi[cu ^ 1]);
            pn3_stream_kernel<<<gst, P3_NT, st->smem, st->cap>>>(a, n, st->u[cu], st->psi[cu ^ 1], st->u[cu ^ 1],
                                                                 st->dose);
            cu ^= 1;
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
        CK(cudaGraphLaunch(exec, stream));
    }
    st->cur_u = par_end;
    st->cur_psi = par_end;
    st->steps_done = n_end - 1;
    st->have_result = true;
    return TITUS_OK;
}

int titus_host::pn3_fetch(titus_solver* s, double* u_out, double* dose_out, double* psi_out) {
    if (!s->pn3 || !s->pn3->have_result) return fail(TITUS_ERR_ARG, "no full-rank solve has run on this handle");
    titus_pn3_state* st = s->pn3;
    CK(cudaDeviceSynchronize());
    CK(cudaGetLastError());
    if (u_out) CK(cudaMemcpy(u_out, st->u[st->cur_u], (size_t)s->n * s->N * sizeof(double), cudaMemcpyDeviceToHost));
    if (dose_out) CK(cudaMemcpy(dose_out, st->dose, (size_t)s->n * sizeof(double), cudaMemcpyDeviceToHost));
    if (psi_out)
        CK(cudaMemcpy2D(psi_out, s->q * sizeof(double), st->psi[st->cur_psi], QM * sizeof(double),
                        s->q * sizeof(double), s->n, cudaMemcpyDeviceToHost));
    return TITUS_OK;
}
