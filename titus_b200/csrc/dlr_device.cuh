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
constexpr int TR = 32;         // rows per staged tile
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
    Csr op[6];                // Ax, Az, |Ax|, |Az|; 3D problems also Ay, |Ay| (z streaming)
    const int32_t* xcomp; int nxcomp;
    const int32_t* wcomp; int nwcomp;
    const uint8_t* restore;   // n: 1 if ordinate-0 value is restored after the sweep
    unsigned long long* prof; // optional phase timers (SM cycles), recorded by CTA 0 of team 0
    int zero_smem;            // 1: clear the dynamic shared memory at kernel start
    long long spin_limit;     // polls before a team barrier gives up (0 = default, about a second)
    int fault_barrier;        // test hook: CTA 1 does not arrive at this barrier generation (<= 0: off)
    int precision;            // 0: FP64; 1: MIXED (tensor-core operator Grams, adaptive integrators)
    int nz;                   // 3D problems: z layers (cell (i, j, k) at row (k nx + i) ny + j); 0 in 2D
    double dz;                // 3D problems: z spacing
};

// Phase-timer categories (titus_profile reports them in this order).
enum ProfCat { PF_BARRIER = 0, PF_REDUCE, PF_JACOBI, PF_CHOL, PF_COMPLETE, PF_ROWS_STREAM, PF_ROWS_SCATTER,
               PF_RF_PASSES, PF_SMALL, PF_TOTAL, PF_PROLOGUE, PF_COUNT };
// event counters in the timer buffer (profiled CTA only; the buffer has PF_SLOTS entries)
constexpr int PF_SVD_SWEEPS = 12, PF_SVD_CALLS = 13;
constexpr int PF_EIG_CALLS = 16, PF_EIG_SWEEPS = 17, PF_CHOL_CALLS = 18, PF_RF_SLOW = 19, PF_RF_FAST = 20,
              PF_BARRIERS = 21;
constexpr int PF_SLOTS = 32;
__device__ __forceinline__ void prof_count(unsigned long long* p, int slot, unsigned long long v) {
    if (p && threadIdx.x == 0) p[slot] += v;
}

// Exclusive phase timers (SM cycles): time is charged to the innermost open
// scope. Slot PF_COUNT collects unscoped time (not reported), slots PF_CUR /
// PF_T hold the open category and the last timestamp; only thread 0 of the
// profiled CTA touches them.
constexpr int PF_CUR = 14, PF_T = 15;
struct ProfScope {
    unsigned long long* p;
    int cat;
    int prev;
    __device__ ProfScope(unsigned long long* p_, int c) : p(p_), cat(c), prev(PF_COUNT) {
        if (p && threadIdx.x == 0) {
            const unsigned long long now = clock64();
            prev = (int)p[PF_CUR];
            p[prev] += now - p[PF_T];
            p[PF_CUR] = (unsigned long long)c;
            p[PF_T] = now;
        }
    }
    __device__ ~ProfScope() {
        if (p && threadIdx.x == 0) {
            const unsigned long long now = clock64();
            p[cat] += now - p[PF_T];
            p[PF_CUR] = (unsigned long long)prev;
            p[PF_T] = now;
        }
    }
};
__device__ __forceinline__ void prof_begin(unsigned long long* p) {
    if (p && threadIdx.x == 0) {
        p[PF_CUR] = PF_COUNT;   // unclassified slot, not reported
        p[PF_T] = clock64();
    }
}

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
    double* part;   // 2 x G x PMAX partial reductions (double-buffered)
    double* red;    // PMAX: second-stage reduced entries (large teams)
    unsigned* bar;  // [0, G): arrival generation per CTA; [G]: release generation
    int* status;    // device error flag
    int* info;      // [0]=rank, [1]=steps done, [2]=psi buffer index, [3]=next n
    double* diag;   // 16: breakdown diagnostics (see record_breakdown)
    int* rank_hist; // nE
    double* eta_hist;
    double* bound_hist;
    double* time_hist;
    double* Y;      // 3 x n x KM: RK4 integrator stage buffers of the K-step (KUP, two stage inputs)
    double* Z;      // 3 x N x KM: the same for the L-step
};

__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ int ldcg(const int* p) { return __ldcg(p); }
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}


// Team barrier, one hop through L2: after the CTA's writes, thread 0 fences and
// adds 1 to the team's arrival counter flags[G], then waits (acquire loads)
// until the counter reaches gen * G, i.e. every CTA of the team has arrived at
// this generation. The counter runs modulo 2^32; the signed difference compares
// correctly while fewer than 2^31 arrivals separate the two values. flags[0, G)
// are not used. Every spin is bounded (`spin_limit` polls, default 2^21 with
// 200 ns sleeps: about a second); on expiry the status flag is set, the
// diagnostics record the CTA, the counter it saw and the one it waited for, and
// all CTAs leave. `fault_gen` >= 1 is a test hook: CTA 1 skips its arrival at
// that generation, so the wait runs out (the host reads the status; nothing
// faults). Returns false if the team's status flag is set.
__device__ inline bool team_sync(unsigned* flags, int* status, int G, int b, unsigned& gen, double* diag = nullptr,
                                 long long spin_limit = 0, int fault_gen = -1) {
    __shared__ int s_ok;
    const long long limit = spin_limit > 0 ? spin_limit : (1ll << 21);
    __syncthreads();
    ++gen;
    if (G == 1) {
        // a one-CTA team: __syncthreads already orders the block's global
        // writes before its later reads; only the status flag is shared
        if (threadIdx.x == 0) s_ok = (ldcg(status) == 0);
        __syncthreads();
        return s_ok;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned target = gen * (unsigned)G;
        const bool skip = (b == 1 && (int)gen == fault_gen);
        unsigned seen = skip ? ld_acquire(flags + G) : atomicAdd(flags + G, 1u) + 1u;
        long long it = 0;
        while ((int)(seen - target) < 0) {
            if (++it > limit) {
                if (atomicCAS(status, 0, ST_BARRIER_TIMEOUT) == 0 && diag) {
                    diag[8] = b;
                    diag[9] = seen;
                    diag[10] = target;
                    diag[14] = gen;
                }
                break;
            }
            if (it > 32) __nanosleep(200);
            if ((it & 255) == 0 && ldcg(status) != 0) break;
            seen = ld_acquire(flags + G);
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
__device__ inline void sm_mm(double* C, const double* A, const double* B, int m, int k, int n) {
    for (int e = threadIdx.x; e < m * n; e += NT) {
        int i = e / n, j = e % n;
        double s = 0.0;
        for (int l = 0; l < k; ++l) s = fma(A[i * KM + l], B[l * KM + j], s);
        C[i * KM + j] = s;
    }
    __syncthreads();
}
// C = A(mxk) * B^T (B is n x k)
__device__ inline void sm_mmt(double* C, const double* A, const double* B, int m, int k, int n) {
    for (int e = threadIdx.x; e < m * n; e += NT) {
        int i = e / n, j = e % n;
        double s = 0.0;
        for (int l = 0; l < k; ++l) s = fma(A[i * KM + l], B[j * KM + l], s);
        C[i * KM + j] = s;
    }
    __syncthreads();
}
// C = A^T(mxk, A is k x m) * B(kxn)
__device__ inline void sm_tmm(double* C, const double* A, const double* B, int m, int k, int n) {
    for (int e = threadIdx.x; e < m * n; e += NT) {
        int i = e / n, j = e % n;
        double s = 0.0;
        for (int l = 0; l < k; ++l) s = fma(A[l * KM + i], B[l * KM + j], s);
        C[i * KM + j] = s;
    }
    __syncthreads();
}
__device__ inline void sm_copy(double* D, const double* A, int m, int n) {
    for (int e = threadIdx.x; e < m * n; e += NT) D[(e / n) * KM + e % n] = A[(e / n) * KM + e % n];
    __syncthreads();
}
__device__ inline void sm_zero(double* D, int m, int n) {
    for (int e = threadIdx.x; e < m * n; e += NT) D[(e / n) * KM + e % n] = 0.0;
    __syncthreads();
}

// Round-robin (tournament) pairing for the parallel cyclic Jacobi method:
// round t, slot s -> pair (p, q), p < q; returns false for the dummy slot.
__device__ __forceinline__ bool rr_pair(int m, int t, int s, int k, int& p, int& q) {
    // positions 0..m-1; position 0 fixed, others rotate by t. For pos >= 1 and
    // 0 <= t <= m-2 the rotated index lies in [1, 2m-3]: one conditional
    // subtraction replaces the modulo.
    auto at = [&](int pos) -> int {
        if (pos == 0) return 0;
        int v = pos - 1 + (m - 1) - t;
        if (v >= m - 1) v -= m - 1;
        return 1 + v;
    };
    int a = at(s), b = at(m - 1 - s);
    p = min(a, b);
    q = max(a, b);
    return q < k;
}

// Symmetric eigendecomposition by parallel cyclic Jacobi.
// In: A (k x k symmetric, in smem work array Aw). Out: lam[k] descending,
// V (k x k, columns eigenvectors, same order). Aw and V are smem arrays.
static __device__ __noinline__ void jacobi_eig(double* Aw, double* V, double* lam, int k, int* status) {
    __shared__ double rc[KM / 2 + 1], rs[KM / 2 + 1];
    __shared__ int rp[KM / 2 + 1], rq[KM / 2 + 1];
    __shared__ int s_rot[2];  // per-sweep-parity flag: a reset never races a late reader
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
        const int par = sweep & 1;
        if (threadIdx.x == 0) s_rot[par] = 0;
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
                        s_rot[par] = 1;
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
        if (!s_rot[par]) break;
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

// Upper Cholesky R^T R = G (k x k, k <= KM <= 32) and Ri = R^{-1} by ONE warp:
// lane c keeps column c of R and of R^{-1} in registers (fully unrolled loops,
// so all register indices are static), row entries travel by shuffles.
// Returns ||R||_F ||R^{-1}||_F, or +inf on breakdown (non-positive pivot).
static __device__ __noinline__ double warp_chol_inv(const double* G, double* R, double* Ri, int k, int* bad_j = nullptr,
                                double* bad_d = nullptr) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    double col[KM];
    int first_bad = -1;
    double first_d = 0.0;
#pragma unroll
    for (int a = 0; a < KM; ++a) col[a] = (lane < k && a < k && a <= lane) ? G[a * KM + lane] : 0.0;
    bool ok = true;
#pragma unroll
    for (int j = 0; j < KM; ++j) {
        if (j < k) {
            double d = __shfl_sync(FULL, col[j], j);
            if (!(d > 0.0)) {
                if (ok) {
                    first_bad = j;
                    first_d = d;
                }
                ok = false;
                d = 1.0;
            }
            const double piv = sqrt(d);
            const double ip = 1.0 / piv;
            if (lane == j) col[j] = piv;
            else if (lane > j) col[j] *= ip;
#pragma unroll
            for (int a = j + 1; a < KM; ++a) {
                if (a < k) {
                    const double rja = __shfl_sync(FULL, col[j], a);
                    if (lane >= a) col[a] = fma(-rja, col[j], col[a]);
                }
            }
        }
    }
    // R to shared memory (column lane), then R^{-1} column lane by back substitution
    if (lane < k) {
#pragma unroll
        for (int a = 0; a < KM; ++a)
            if (a < k) R[a * KM + lane] = (a <= lane) ? col[a] : 0.0;
    }
    __syncwarp();
    double inv[KM];
    double nr = 0.0, ni = 0.0;
#pragma unroll
    for (int a = KM - 1; a >= 0; --a) {
        double v = 0.0;
        if (a < k && lane < k && a <= lane) {
            double t = (a == lane) ? 1.0 : 0.0;
#pragma unroll
            for (int b = a + 1; b < KM; ++b)
                if (b <= lane && b < k) t = fma(-R[a * KM + b], inv[b], t);
            v = t / R[a * KM + a];
        }
        inv[a] = v;
    }
    if (lane < k) {
#pragma unroll
        for (int a = 0; a < KM; ++a)
            if (a < k) {
                Ri[a * KM + lane] = inv[a];
                nr = fma(col[a], col[a], nr);
                ni = fma(inv[a], inv[a], ni);
            }
    }
    for (int o = 16; o > 0; o >>= 1) {
        nr += __shfl_xor_sync(FULL, nr, o);
        ni += __shfl_xor_sync(FULL, ni, o);
    }
    ok = __all_sync(FULL, ok);
    if (bad_j) *bad_j = first_bad;
    if (bad_d) *bad_d = first_d;
    return ok ? sqrt(nr) * sqrt(ni) : INFINITY;
}

// Two independent Cholesky factorisations on warps 0 and 1 concurrently
// (either may be skipped). Writes the condition estimates; sets the status
// flag on breakdown when `flag` is set.
// On breakdown with `flag`, the first CTA to fail records in diag:
// [0] stage tag, [1] side (0 = X, 1 = W), [2] k, [3] first bad pivot index,
// [4] its value, [5] G[0][0], [6] min diagonal of G, [7] energy index.
__device__ inline void record_breakdown(double* diag, int* status, int tag, int side, int k, int bj, double bd,
                                 const double* G, int n) {
    if (atomicCAS(status, 0, ST_CHOL_BREAKDOWN) == 0 && diag) {
        double mn = INFINITY;
        for (int a = 0; a < k; ++a) mn = fmin(mn, G[a * KM + a]);
        diag[0] = tag;
        diag[1] = side;
        diag[2] = k;
        diag[3] = bj;
        diag[4] = bd;
        diag[5] = k > 0 ? G[0] : 0.0;
        diag[6] = mn;
        diag[7] = n;
    }
}

__device__ inline void dual_chol(bool dx, const double* GX, double* RX, double* RiX, int kx, double* condX,
                          bool dw, const double* GW, double* RW, double* RiW, int kw, double* condW,
                          int* status, bool flag, double* diag = nullptr, int tag = 0, int n = 0) {
    __shared__ double s_c[2];
    const int w = threadIdx.x >> 5;
    if (w == 0 && dx) {
        int bj;
        double bd;
        double c = warp_chol_inv(GX, RX, RiX, kx, &bj, &bd);
        if ((threadIdx.x & 31) == 0) {
            s_c[0] = c;
            if (flag && !(c < INFINITY)) record_breakdown(diag, status, tag, 0, kx, bj, bd, GX, n);
        }
    }
    if (w == 1 && dw) {
        int bj;
        double bd;
        double c = warp_chol_inv(GW, RW, RiW, kw, &bj, &bd);
        if ((threadIdx.x & 31) == 0) {
            s_c[1] = c;
            if (flag && !(c < INFINITY)) record_breakdown(diag, status, tag, 1, kw, bj, bd, GW, n);
        }
    }
    __syncthreads();
    if (condX) *condX = dx ? s_c[0] : 0.0;
    if (condW) *condW = dw ? s_c[1] : 0.0;
}

// Row-wise triangular solve on a tile: Y[r,:] R = A[r,:] (R upper, k x k), in place.
__device__ __forceinline__ void tile_rsolve(double* t, const double* R, const double* dinv_unused, int nr, int k) {
    for (int r = threadIdx.x; r < nr; r += NT) {
        double* row = t + r * KM;
        for (int j = 0; j < k; ++j) {
            double v = row[j];
            for (int i = 0; i < j; ++i) v = fma(-row[i], R[i * KM + j], v);
            row[j] = v / R[j * KM + j];
        }
    }
}

}  // namespace titus
