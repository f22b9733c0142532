// Device building blocks of the persistent DLR energy-step kernel (sm_100a, FP64).
//
// One "team" of G CTAs advances one solve. Rows of the spatial factors
// (cells, row i*ny+j) and of the angular factors (moments) are partitioned over
// the team's CTAs; every reduction over rows goes through per-CTA partial
// buffers in global memory (L2 resident) and is summed by every CTA in the
// same order, so all CTAs of a team hold bit-identical small matrices and take
// identical control-flow decisions without a broadcast step.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace titus {

constexpr int NT = 256;        // threads per CTA
constexpr int KM = 24;         // max basis width handled by this build
constexpr int QM = 32;         // max reduced ordinates
constexpr int TR = 16;         // rows per staged tile
constexpr int NOPS = 4;        // Ax, Az, |Ax|, |Az|
constexpr int KK = KM * KM;
constexpr int PMAX = 8 * KK;  // partial-reduction capacity (doubles); >= 2KK + 2 KM QM
constexpr int NCAND = 3 * KM;  // max W completion candidates examined

// status codes written by the device
constexpr int ST_OK = 0;
constexpr int ST_BARRIER_TIMEOUT = 1;
constexpr int ST_CHOL_BREAKDOWN = 2;
constexpr int ST_COMPLETION = 3;
constexpr int ST_JACOBI = 4;

struct Csr {
    const int32_t* rowptr;
    const int32_t* col;
    const double* val;
};

// Problem data resident on the device (shared by all teams).
struct DevProblem {
    int nx, ny, n, N, npn, q, nE, r;
    double dx, dy, dE, theta, theta_index, c_eta, rank_tol;
    const double* rinv;       // n: 1/density
    const double* stopping;   // nE
    const double* bc_energy;  // nE
    const double* sigma;      // nE x (npn+1)
    const double* bc_space;   // n
    const double* bc_angle;   // q
    const double* omega;      // q x 3
    const double* mred;       // N x q
    const int32_t* lof;       // N: Legendre order l of moment m
    Csr op[NOPS];
    const int32_t* xcomp; int nxcomp;
    const int32_t* wcomp; int nwcomp;
    const uint8_t* restore;   // n: 1 if ordinate-0 value is restored after the sweep
};

// Per-team device state.
struct TeamState {
    double* X;      // n x KM
    double* K;      // n x KM   (K, then C of the range finder)
    double* W;      // N x KM
    double* L;      // N x KM
    double* psi0;   // n x QM
    double* psi1;   // n x QM
    double* dose;   // n
    double* S;      // KM x KM (final S written back)
    double* part;   // G x PMAX partial reductions
    unsigned* bar;  // [0] = arrive count, [1] = generation
    int* status;    // device error flag
    int* info;      // [0]=rank, [1]=steps done, [2]=psi buffer index, [3]=next n
    int* rank_hist; // nE
    double* eta_hist;
    double* bound_hist;
    double* time_hist;
};

__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ int ldcg(const int* p) { return __ldcg(p); }
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Team barrier: arrive counter + generation, bounded spin. Returns false if the
// team's status flag is set (by this or another CTA, e.g. after a timeout).
__device__ bool team_sync(unsigned* bar, int* status, int G) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned gen = ld_acquire(bar + 1);
        __threadfence();
        unsigned arrived = atomicAdd(bar, 1u);
        if (arrived == (unsigned)(G - 1)) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            long long it = 0;
            while (ld_acquire(bar + 1) == gen) {
                if (++it > (1ll << 24)) {  // ~1-2 s with the sleep below
                    atomicExch(status, ST_BARRIER_TIMEOUT);
                    break;
                }
                if (it > 64) __nanosleep(100);
                if ((it & 1023) == 0 && ldcg(status) != 0) break;
            }
        }
        __threadfence();
        s_ok = (ldcg(status) == 0);
    }
    __syncthreads();
    return s_ok;
}

__device__ __forceinline__ void set_status(int* status, int code) {
    atomicCAS(status, 0, code);
}

// ---------------------------------------------------------------------------
// Small dense helpers on one CTA. Matrices are row-major with leading dim KM.
// ---------------------------------------------------------------------------

// C = A(mxk) * B(kxn); C must not alias A or B.
__device__ void sm_mm(double* C, const double* A, const double* B, int m, int k, int n) {
    for (int e = threadIdx.x; e < m * n; e += NT) {
        int i = e / n, j = e % n;
        double s = 0.0;
        for (int l = 0; l < k; ++l) s = fma(A[i * KM + l], B[l * KM + j], s);
        C[i * KM + j] = s;
    }
    __syncthreads();
}
// C = A(mxk) * B^T (B is n x k)
__device__ void sm_mmt(double* C, const double* A, const double* B, int m, int k, int n) {
    for (int e = threadIdx.x; e < m * n; e += NT) {
        int i = e / n, j = e % n;
        double s = 0.0;
        for (int l = 0; l < k; ++l) s = fma(A[i * KM + l], B[j * KM + l], s);
        C[i * KM + j] = s;
    }
    __syncthreads();
}
// C = A^T(mxk, A is k x m) * B(kxn)
__device__ void sm_tmm(double* C, const double* A, const double* B, int m, int k, int n) {
    for (int e = threadIdx.x; e < m * n; e += NT) {
        int i = e / n, j = e % n;
        double s = 0.0;
        for (int l = 0; l < k; ++l) s = fma(A[l * KM + i], B[l * KM + j], s);
        C[i * KM + j] = s;
    }
    __syncthreads();
}
__device__ void sm_copy(double* D, const double* A, int m, int n) {
    for (int e = threadIdx.x; e < m * n; e += NT) D[(e / n) * KM + e % n] = A[(e / n) * KM + e % n];
    __syncthreads();
}
__device__ void sm_zero(double* D, int m, int n) {
    for (int e = threadIdx.x; e < m * n; e += NT) D[(e / n) * KM + e % n] = 0.0;
    __syncthreads();
}

// Round-robin (tournament) pairing for the parallel cyclic Jacobi method:
// round t, slot s -> pair (p, q), p < q; returns false for the dummy slot.
__device__ __forceinline__ bool rr_pair(int m, int t, int s, int k, int& p, int& q) {
    // positions 0..m-1; position 0 fixed, others rotate by t
    auto at = [&](int pos) -> int {
        if (pos == 0) return 0;
        return 1 + ((pos - 1 + (m - 1) - t) % (m - 1));
    };
    int a = at(s), b = at(m - 1 - s);
    p = min(a, b);
    q = max(a, b);
    return q < k;
}

// Symmetric eigendecomposition by parallel cyclic Jacobi.
// In: A (k x k symmetric, in smem work array Aw). Out: lam[k] descending,
// V (k x k, columns eigenvectors, same order). Aw and V are smem arrays.
__device__ void jacobi_eig(double* Aw, double* V, double* lam, int k, int* status) {
    __shared__ double rc[KM / 2 + 1], rs[KM / 2 + 1];
    __shared__ int rp[KM / 2 + 1], rq[KM / 2 + 1];
    __shared__ int s_rot;
    __shared__ double s_lam[KM];
    __shared__ int s_perm[KM];
    for (int e = threadIdx.x; e < k * k; e += NT) V[(e / k) * KM + e % k] = ((e / k) == (e % k)) ? 1.0 : 0.0;
    __syncthreads();
    if (k <= 1) {
        if (threadIdx.x == 0 && k == 1) lam[0] = Aw[0];
        __syncthreads();
        return;
    }
    const int m = k + (k & 1);
    const int npairs = m / 2;
    int sweep = 0;
    for (; sweep < 40; ++sweep) {
        if (threadIdx.x == 0) s_rot = 0;
        __syncthreads();
        for (int t = 0; t < m - 1; ++t) {
            if (threadIdx.x < npairs) {
                int p, q;
                double c = 1.0, s = 0.0;
                bool valid = rr_pair(m, t, threadIdx.x, k, p, q);
                if (valid) {
                    double apq = Aw[p * KM + q];
                    double app = Aw[p * KM + p], aqq = Aw[q * KM + q];
                    if (apq != 0.0 && fabs(apq) > 1e-15 * sqrt(fabs(app * aqq))) {
                        double theta = (aqq - app) / (2.0 * apq);
                        double t_;
                        if (fabs(theta) > 1e150) t_ = 0.5 / theta;
                        else t_ = copysign(1.0, theta) / (fabs(theta) + sqrt(theta * theta + 1.0));
                        c = 1.0 / sqrt(t_ * t_ + 1.0);
                        s = t_ * c;
                        s_rot = 1;
                    }
                } else {
                    p = q = -1;
                }
                rc[threadIdx.x] = c;
                rs[threadIdx.x] = s;
                rp[threadIdx.x] = p;
                rq[threadIdx.x] = q;
            }
            __syncthreads();
            // rows: A <- J^T A
            for (int e = threadIdx.x; e < npairs * k; e += NT) {
                int pi = e / k, j = e % k;
                int p = rp[pi], q = rq[pi];
                if (p < 0) continue;
                double c = rc[pi], s = rs[pi];
                if (s == 0.0) continue;
                double ap = Aw[p * KM + j], aq = Aw[q * KM + j];
                Aw[p * KM + j] = c * ap - s * aq;
                Aw[q * KM + j] = s * ap + c * aq;
            }
            __syncthreads();
            // columns: A <- A J, V <- V J
            for (int e = threadIdx.x; e < npairs * k; e += NT) {
                int pi = e / k, i = e % k;
                int p = rp[pi], q = rq[pi];
                if (p < 0) continue;
                double c = rc[pi], s = rs[pi];
                if (s == 0.0) continue;
                double ap = Aw[i * KM + p], aq = Aw[i * KM + q];
                Aw[i * KM + p] = c * ap - s * aq;
                Aw[i * KM + q] = s * ap + c * aq;
                double vp = V[i * KM + p], vq = V[i * KM + q];
                V[i * KM + p] = c * vp - s * vq;
                V[i * KM + q] = s * vp + c * vq;
            }
            __syncthreads();
        }
        if (!s_rot) break;
    }
    (void)status;
    // sort descending (stable): rank of each eigenvalue
    for (int i = threadIdx.x; i < k; i += NT) s_lam[i] = Aw[i * KM + i];
    __syncthreads();
    for (int i = threadIdx.x; i < k; i += NT) {
        double li = s_lam[i];
        int rank = 0;
        for (int j = 0; j < k; ++j) {
            double lj = s_lam[j];
            if (lj > li || (lj == li && j < i)) ++rank;
        }
        s_perm[rank] = i;
    }
    __syncthreads();
    // permute V columns into Aw as scratch, then copy back
    for (int e = threadIdx.x; e < k * k; e += NT) {
        int i = e / k, j = e % k;
        Aw[i * KM + j] = V[i * KM + s_perm[j]];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < k * k; e += NT) V[(e / k) * KM + e % k] = Aw[(e / k) * KM + e % k];
    for (int j = threadIdx.x; j < k; j += NT) lam[j] = s_lam[s_perm[j]];
    __syncthreads();
}

// Upper Cholesky R^T R = G (k x k), then Ri = R^{-1} (upper). G in smem (read),
// R and Ri written (may alias nothing). Sets status on breakdown.
__device__ void chol_inv(const double* G, double* R, double* Ri, int k, int* status) {
    for (int e = threadIdx.x; e < k * k; e += NT) R[(e / k) * KM + e % k] = G[(e / k) * KM + e % k];
    __syncthreads();
    __shared__ double s_piv;
    for (int j = 0; j < k; ++j) {
        if (threadIdx.x == 0) {
            double d = R[j * KM + j];
            if (!(d > 0.0)) {
                set_status(status, ST_CHOL_BREAKDOWN);
                d = 1.0;
            }
            s_piv = sqrt(d);
            R[j * KM + j] = s_piv;
        }
        __syncthreads();
        for (int c = j + 1 + threadIdx.x; c < k; c += NT) R[j * KM + c] /= s_piv;
        __syncthreads();
        // trailing update on the upper triangle: R[a][b] -= R[j][a] R[j][b], a<=b
        int m = k - j - 1;
        for (int e = threadIdx.x; e < m * m; e += NT) {
            int a = j + 1 + e / m, b = j + 1 + e % m;
            if (b >= a) R[a * KM + b] -= R[j * KM + a] * R[j * KM + b];
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < k * k; e += NT) {
        int a = e / k, b = e % k;
        if (b < a) R[a * KM + b] = 0.0;
    }
    __syncthreads();
    // inverse of upper triangular R, column by column: Ri[:, c] solves R x = e_c
    for (int c = threadIdx.x; c < k; c += NT) {
        for (int a = k - 1; a >= 0; --a) {
            double s = (a == c) ? 1.0 : 0.0;
            if (a > c) s = 0.0;
            else {
                for (int b = a + 1; b <= c; ++b) s -= R[a * KM + b] * Ri[b * KM + c];
            }
            Ri[a * KM + c] = (a > c) ? 0.0 : s / R[a * KM + a];
        }
    }
    __syncthreads();
}

}  // namespace titus
