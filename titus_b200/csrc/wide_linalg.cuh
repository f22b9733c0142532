// Small dense factorisations of the rank-adaptive kernel, run by one CTA on
// shared-memory matrices (row-major with an explicit leading dimension):
//   w_chol      upper Cholesky R^T R = G and R^{-1} (k <= RA)
//   w_eig       symmetric eigendecomposition, parallel cyclic Jacobi (k <= RA)
//   w_svd       one-sided (Hestenes) Jacobi SVD of an m x m matrix (m <= KA),
//               with w_svd_complete applying the deterministic rule for the
//               numerically null singular directions that truncate! keeps.
#pragma once
#include "wide_common.cuh"

namespace titus {
namespace TITUS_WIDE_NS {

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum over the CTA of one value per thread, in a fixed order (warp butterflies,
// then the warps in index order); every thread receives the same result.
static __device__ __noinline__ double cta_sum(double v) {
    __shared__ double s_w[NT / 32];
    v = warp_sum(v);
    __syncthreads();   // a previous call's readers are done with s_w
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    for (int w = 0; w < NT / 32; ++w) t += s_w[w];
    return t;
}

// Upper Cholesky of G (k x k, ld ldg, any memory) into R (shared, ld) and its
// inverse Ri (shared, ld). Returns ||R||_F ||R^{-1}||_F, or +inf on a
// non-positive pivot; *ri_f receives ||R^{-1}||_F (a bound 1/sigma_min).
static __device__ __noinline__ double w_chol(const double* G, int ldg, double* R, double* Ri, int ld, int k,
                                             double* ri_f) {
    __shared__ int s_ok;
    __shared__ double s_nr[NT / 32], s_ni[NT / 32];
    for (int e = threadIdx.x; e < k * k; e += NT) {
        const int i = e / k, j = e - (e / k) * k;
        R[i * ld + j] = (j >= i) ? G[i * ldg + j] : 0.0;
        Ri[i * ld + j] = 0.0;
    }
    if (threadIdx.x == 0) s_ok = 1;
    __syncthreads();
    for (int j = 0; j < k; ++j) {
        const double d = R[j * ld + j];
        const bool okp = d > 0.0;
        const double piv = okp ? sqrt(d) : 1.0;
        __syncthreads();
        for (int l = j + threadIdx.x; l < k; l += NT) R[j * ld + l] = (l == j) ? piv : R[j * ld + l] / piv;
        if (!okp && threadIdx.x == 0) s_ok = 0;
        __syncthreads();
        const int m = k - j - 1;
        for (int e = threadIdx.x; e < m * m; e += NT) {
            const int i = j + 1 + e / m, l = j + 1 + (e - (e / m) * m);
            if (l >= i) R[i * ld + l] = fma(-R[j * ld + i], R[j * ld + l], R[i * ld + l]);
        }
        __syncthreads();
    }
    // R^{-1}: warp w solves columns c = w, w+8, ...; lanes split each dot product
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int c = warp; c < k; c += NT / 32) {
        if (lane == 0) Ri[c * ld + c] = 1.0 / R[c * ld + c];
        __syncwarp();
        for (int a = c - 1; a >= 0; --a) {
            double s = 0.0;
            for (int bb = a + 1 + lane; bb <= c; bb += 32) s = fma(R[a * ld + bb], Ri[bb * ld + c], s);
            s = warp_sum(s);
            if (lane == 0) Ri[a * ld + c] = -s / R[a * ld + a];
            __syncwarp();
        }
    }
    __syncthreads();
    double nr = 0.0, ni = 0.0;
    for (int e = threadIdx.x; e < k * k; e += NT) {
        const int i = e / k, j = e - (e / k) * k;
        nr = fma(R[i * ld + j], R[i * ld + j], nr);
        ni = fma(Ri[i * ld + j], Ri[i * ld + j], ni);
    }
    nr = warp_sum(nr);
    ni = warp_sum(ni);
    if (lane == 0) {
        s_nr[warp] = nr;
        s_ni[warp] = ni;
    }
    __syncthreads();
    double tr = 0.0, ti = 0.0;
    for (int w = 0; w < NT / 32; ++w) {
        tr += s_nr[w];
        ti += s_ni[w];
    }
    const bool ok = s_ok != 0;
    __syncthreads();
    if (ri_f) *ri_f = ok ? sqrt(ti) : INFINITY;
    return ok ? sqrt(tr) * sqrt(ti) : INFINITY;
}

// Symmetric eigendecomposition by parallel cyclic Jacobi. A (k x k, shared,
// ld) is destroyed; V (shared, ld) receives the eigenvectors as columns, lam
// the eigenvalues, both in descending order. k <= RA.
// A pair is rotated when |a_pq| > rel_tol sqrt|a_pp a_qq| (1e-15: relative
// accuracy on graded matrices) and |a_pq| > rel_floor max_i |a_ii|. A Gram matrix formed
// in floating point carries noise of about k eps max|a_ii| that no rotation
// removes, so raw Grams use rel_floor ~ 4 k eps; graded Grams of already
// separated directions use a negligible floor.
static __device__ __noinline__ int w_eig(double* A, double* V, int ld, double* lam, int k, int* status,
                                         double rel_floor, double rel_tol = 1e-15) {
    __shared__ double rc[RA / 2 + 1], rs[RA / 2 + 1], rdp[RA / 2 + 1], rdq[RA / 2 + 1];
    __shared__ int rp[RA / 2 + 1], rq[RA / 2 + 1];
    __shared__ int s_rot[2];
    __shared__ double s_lam[RA];
    __shared__ int s_perm[RA];
    for (int e = threadIdx.x; e < k * k; e += NT) V[(e / k) * ld + e % k] = ((e / k) == (e % k)) ? 1.0 : 0.0;
    __syncthreads();
    if (k <= 1) {
        if (threadIdx.x == 0 && k == 1) lam[0] = A[0];
        __syncthreads();
        return 0;
    }
    const int m = k + (k & 1);
    const int npairs = m / 2;
    __shared__ double s_floor;
    if (threadIdx.x == 0) {
        double mx = 0.0;
        for (int i = 0; i < k; ++i) mx = fmax(mx, fabs(A[i * ld + i]));
        s_floor = rel_floor * mx;
    }
    __syncthreads();
    const double afloor = s_floor;
    bool conv = false;
    int nsw = 60;
    for (int sweep = 0; sweep < 60; ++sweep) {
        const int par = sweep & 1;
        if (threadIdx.x == 0) s_rot[par] = 0;
        __syncthreads();
        for (int t = 0; t < m - 1; ++t) {
            if (threadIdx.x < npairs) {
                int p, q;
                double c = 1.0, s = 0.0;
                if (rr_pair(m, t, threadIdx.x, k, p, q)) {
                    const double apq = A[p * ld + q];
                    const double app = A[p * ld + p], aqq = A[q * ld + q];
                    // a rotation whose angle is below eps changes nothing (|a_pq| <= eps max|a|):
                    // skipping it keeps the sweep count finite on rounding-level entries
                    if (fabs(apq) > afloor && apq * apq > rel_tol * rel_tol * fabs(app * aqq) &&
                        fabs(apq) > 4.4e-16 * fmax(fabs(app), fabs(aqq))) {
                        // t = tan of the rotation angle, the smaller root of
                        // t^2 + 2 th t - 1 = 0 with th = (aqq - app) / (2 apq), in the
                        // form t = 2 apq sgn(d) / (|d| + sqrt(d^2 + 4 apq^2)), d = aqq - app
                        const double d = aqq - app;
                        const double tt = 2.0 * apq * copysign(1.0, d) / (fabs(d) + sqrt(fma(d, d, 4.0 * apq * apq)));
                        c = rsqrt(fma(tt, tt, 1.0));
                        s = tt * c;
                        // the rotated 2x2 block in closed form (a_pq -> 0 exactly):
                        // two-sided updates leave a_pq at a few eps max|a_pp|, |a_qq|,
                        // which the next sweep would rotate again without end
                        rdp[threadIdx.x] = fma(-tt, apq, app);
                        rdq[threadIdx.x] = fma(tt, apq, aqq);
                        s_rot[par] = 1;
                    }
                } else {
                    q = -1;   // p is real, its partner the padding index: p stays put this round
                }
                rc[threadIdx.x] = c;
                rs[threadIdx.x] = s;
                rp[threadIdx.x] = p;
                rq[threadIdx.x] = q;
            }
            __syncthreads();
            // Both rotations at once: the thread owning rows {p_a, q_a} x columns
            // {p_b, q_b} reads the four entries, rotates the rows by pair a and the
            // columns by pair b (the order of the two one-sided passes) and writes
            // them back; no other thread touches them, so one barrier suffices.
            // A rotated diagonal block takes the closed form.
            for (int e = threadIdx.x; e < npairs * npairs; e += NT) {
                const int a = e / npairs, b = e - (e / npairs) * npairs;
                const double sa = rs[a], sb = rs[b];
                if (sa == 0.0 && sb == 0.0) continue;
                const int pa = rp[a], qa = rq[a], pb = rp[b], qb = rq[b];
                if (a == b) {
                    A[pa * ld + pa] = rdp[a];
                    A[qa * ld + qa] = rdq[a];
                    A[pa * ld + qa] = 0.0;
                    A[qa * ld + pa] = 0.0;
                    continue;
                }
                const double ca = rc[a], cb = rc[b];
                const double xpp = A[pa * ld + pb];
                const double xpq = qb >= 0 ? A[pa * ld + qb] : 0.0;
                const double xqp = qa >= 0 ? A[qa * ld + pb] : 0.0;
                const double xqq = (qa >= 0 && qb >= 0) ? A[qa * ld + qb] : 0.0;
                const double rpp = ca * xpp - sa * xqp, rpq = ca * xpq - sa * xqq;
                const double rqp = sa * xpp + ca * xqp, rqq = sa * xpq + ca * xqq;
                A[pa * ld + pb] = cb * rpp - sb * rpq;
                if (qb >= 0) A[pa * ld + qb] = sb * rpp + cb * rpq;
                if (qa >= 0) {
                    A[qa * ld + pb] = cb * rqp - sb * rqq;
                    if (qb >= 0) A[qa * ld + qb] = sb * rqp + cb * rqq;
                }
            }
            for (int e = threadIdx.x; e < npairs * k; e += NT) {
                const int b = e / k, i = e - (e / k) * k;
                const double sb = rs[b];
                if (sb == 0.0) continue;
                const int pb = rp[b], qb = rq[b];
                const double cb = rc[b];
                const double vp = V[i * ld + pb], vq = V[i * ld + qb];
                V[i * ld + pb] = cb * vp - sb * vq;
                V[i * ld + qb] = sb * vp + cb * vq;
            }
            __syncthreads();
        }
        if (!s_rot[par]) {
            conv = true;
            nsw = sweep + 1;
            break;
        }
    }
    if (!conv && threadIdx.x == 0) set_status(status, ST_JACOBI);
    __syncthreads();
    for (int i = threadIdx.x; i < k; i += NT) s_lam[i] = A[i * ld + i];
    __syncthreads();
    for (int i = threadIdx.x; i < k; i += NT) {
        const double li = s_lam[i];
        int rank = 0;
        for (int j = 0; j < k; ++j) {
            const double lj = s_lam[j];
            if (lj > li || (lj == li && j < i)) ++rank;
        }
        s_perm[rank] = i;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < k * k; e += NT) {
        const int i = e / k, j = e - (e / k) * k;
        A[i * ld + j] = V[i * ld + s_perm[j]];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < k * k; e += NT) V[(e / k) * ld + e % k] = A[(e / k) * ld + e % k];
    for (int j = threadIdx.x; j < k; j += NT) lam[j] = s_lam[s_perm[j]];
    __syncthreads();
    return nsw;
}

// One-sided Jacobi SVD of the m x m matrix whose column p is At[p*ld .. +m)
// (transposed storage keeps column operations on contiguous shared memory).
// On return At[p] = sigma_p u_p and Vt[p] = v_p (unsorted); sig[j] and
// perm[j] list the singular values in descending order (sigma_j = sig[j],
// column perm[j]). Returns the number of sweeps, or -1 without convergence.
static __device__ __noinline__ int w_svd(double* At, double* Vt, int ld, int m, double* sig, int* perm) {
    __shared__ int s_rot[2];
    __shared__ double s_n[KA];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int e = threadIdx.x; e < m * m; e += NT) Vt[(e / m) * ld + e % m] = ((e / m) == (e % m)) ? 1.0 : 0.0;
    __syncthreads();
    int sweeps = -1;
    // rotation threshold: a recomputed dot product of two length-m columns
    // carries rounding of about m eps |x| |y|. Columns with |x| below
    // 1e-16 ||A||_F are numerically null and not rotated. (A floor as high as
    // 1e-13 ||A||_F moves the dose by 2e-9: a column that starts tiny can
    // still carry a small kept singular direction.)
    const double ctol = 2.2e-16 * m;
    __shared__ double s_fro;
    if (threadIdx.x < 32) {
        double f = 0.0;
        for (int e = threadIdx.x; e < m * m; e += 32) f = fma(At[(e / m) * ld + e % m], At[(e / m) * ld + e % m], f);
        f = warp_sum(f);
        if (threadIdx.x == 0) s_fro = f;
    }
    __syncthreads();
    const double nfloor = 1e-32 * s_fro;
    if (m > 1) {
        const int mm = m + (m & 1);
        const int npairs = mm / 2;
        // LP lanes per pair (8 / 16 / 32), PPW = 32 / LP pairs per warp
        const int LP = m <= 24 ? 8 : (m <= 48 ? 16 : 32);
        const int PPW = 32 / LP;
        const int grp = lane / LP, gl = lane % LP;
        for (int sweep = 0; sweep < 60; ++sweep) {
            const int par = sweep & 1;
            if (threadIdx.x == 0) s_rot[par] = 0;
            __syncthreads();
            for (int t = 0; t < mm - 1; ++t) {
                // warp-uniform loop; every lane runs the shuffles
                for (int sb = warp * PPW; sb < npairs; sb += (NT / 32) * PPW) {
                    const int sidx = sb + grp;
                    int p = 0, q = 0;
                    const bool valid = sidx < npairs && rr_pair(mm, t, sidx, m, p, q);
                    double a = 0.0, bq = 0.0, g = 0.0;
                    if (valid)
                        for (int i = gl; i < m; i += LP) {
                            const double u = At[p * ld + i], v = At[q * ld + i];
                            a = fma(u, u, a);
                            bq = fma(v, v, bq);
                            g = fma(u, v, g);
                        }
                    for (int o = LP / 2; o > 0; o >>= 1) {
                        a += __shfl_xor_sync(0xffffffffu, a, o);
                        bq += __shfl_xor_sync(0xffffffffu, bq, o);
                        g += __shfl_xor_sync(0xffffffffu, g, o);
                    }
                    // skip rotations with an angle below eps (no effect on the columns)
                    if (valid && g != 0.0 && fmin(a, bq) > nfloor && g * g > ctol * ctol * a * bq &&
                        fabs(g) > 2.2e-16 * fmax(a, bq)) {
                        // t = tan of the angle orthogonalising the two columns:
                        // t = 2 g sgn(d) / (|d| + sqrt(d^2 + 4 g^2)), d = |y|^2 - |x|^2
                        const double d = bq - a;
                        const double tt = 2.0 * g * copysign(1.0, d) / (fabs(d) + sqrt(fma(d, d, 4.0 * g * g)));
                        const double c = rsqrt(fma(tt, tt, 1.0)), sn = c * tt;
                        for (int i = gl; i < m; i += LP) {
                            const double u = At[p * ld + i], v = At[q * ld + i];
                            At[p * ld + i] = c * u - sn * v;
                            At[q * ld + i] = sn * u + c * v;
                            const double vu = Vt[p * ld + i], vv = Vt[q * ld + i];
                            Vt[p * ld + i] = c * vu - sn * vv;
                            Vt[q * ld + i] = sn * vu + c * vv;
                        }
                        if (gl == 0) s_rot[par] = 1;
                    }
                }
                __syncthreads();
            }
            if (!s_rot[par]) {
                sweeps = sweep + 1;
                break;
            }
        }
    } else {
        sweeps = 0;
    }
    // singular values and descending order (stable)
    for (int p = warp; p < m; p += NT / 32) {
        double a = 0.0;
        for (int i = lane; i < m; i += 32) a = fma(At[p * ld + i], At[p * ld + i], a);
        a = warp_sum(a);
        if (lane == 0) s_n[p] = sqrt(a);
    }
    __syncthreads();
    for (int p = threadIdx.x; p < m; p += NT) {
        const double v = s_n[p];
        int rank = 0;
        for (int j = 0; j < m; ++j) {
            const double w = s_n[j];
            if (w > v || (w == v && j < p)) ++rank;
        }
        perm[rank] = p;
        sig[rank] = v;
    }
    __syncthreads();
    return sweeps;
}

// Normalise the left singular vectors of the numerical range (sigma_j >
// tol sigma_0, j < rho) and complete the directions j in [rho, kkeep) of both
// factors, which the matrix does not determine, by a rule that does not depend
// on the bases the small matrix is expressed in: candidate c is the row c of
// that basis (rowsU: the n x m spatial basis for U, rowsV: the N x m angular
// basis for V; global, ld ldr), i.e. the cell / moment indicator vector
// projected into the basis, taken in index order (then canonical vectors of
// R^m); rows with norm <= 1e-6 are skipped; two Gram-Schmidt passes against
// the columns before it; accepted when the residual keeps at least half the
// candidate's norm. When the candidates run out before every direction is
// filled (many null directions in a wide basis), a second scan from the first
// candidate accepts residuals above 1e-3 of the norm. Same rule as
// oracle.linalg._complete_rows. Returns rho.
static __device__ __noinline__ int w_svd_complete(double* At, double* Vt, int ld, int m, const double* sig,
                                                  const int* perm, int kkeep, double tol, int* status,
                                                  const double* rowsU, int nU, const double* rowsV, int nV,
                                                  int ldr) {
    __shared__ double s_v[KA];
    __shared__ double s_d[KA];
    __shared__ double s_nv, s_nu;
    __shared__ double s_n8[NT / 32];
    __shared__ int s_acc;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int rho = 0;
    if (m > 0 && sig[0] > 0.0)
        for (int j = 0; j < m; ++j) {
            if (sig[j] > tol * sig[0]) rho = j + 1;
            else break;
        }
    for (int e = threadIdx.x; e < rho * m; e += NT) {
        const int j = e / m, i = e - (e / m) * m;
        At[perm[j] * ld + i] /= sig[j];
    }
    __syncthreads();
    for (int side = 0; side < 2; ++side) {
        double* B = side == 0 ? At : Vt;
        const double* rows = side == 0 ? rowsU : rowsV;
        const int nrows = side == 0 ? nU : nV;
        int cand = 0;   // [0, nrows): basis rows; [nrows, nrows + m): canonical vectors
        int phase = 0;  // 0: keep half the candidate's norm; 1 (second scan): 1e-3 of it
        for (int j = rho; j < kkeep; ++j) {
            bool done = false;
            while (!done) {
                if (cand >= nrows + m) {
                    if (phase == 0) {
                        phase = 1;
                        cand = 0;
                        continue;
                    }
                    if (threadIdx.x == 0) set_status(status, ST_COMPLETION);
                    __syncthreads();
                    return rho;
                }
                int found = -1;
                if (cand < nrows) {
                    // next row with norm > 1e-6, eight candidates at a time (one per warp)
                    while (cand < nrows && found < 0) {
                        const int c = cand + warp;
                        double sq = 0.0;
                        if (c < nrows)
                            for (int i = lane; i < m; i += 32) {
                                const double v = ldcg(rows + (size_t)c * ldr + i);
                                sq = fma(v, v, sq);
                            }
                        sq = warp_sum(sq);
                        if (lane == 0) s_n8[warp] = (c < nrows) ? sq : -1.0;
                        __syncthreads();
                        int f = -1;
                        for (int w = 0; w < NT / 32; ++w)
                            if (s_n8[w] > 1e-12) {
                                f = w;
                                break;
                            }
                        __syncthreads();
                        if (f >= 0) {
                            found = cand + f;
                            cand = found + 1;
                        } else {
                            // stop at nrows: the canonical vectors come next, from the first
                            cand = min(cand + NT / 32, nrows);
                        }
                    }
                    if (found < 0) continue;   // rows exhausted: canonical vectors next
                    for (int i = threadIdx.x; i < m; i += NT) s_v[i] = ldcg(rows + (size_t)found * ldr + i);
                } else {
                    const int i0 = cand - nrows;
                    for (int i = threadIdx.x; i < m; i += NT) s_v[i] = (i == i0) ? 1.0 : 0.0;
                    ++cand;
                }
                __syncthreads();
                if (threadIdx.x < 32) {
                    double sq = 0.0;
                    for (int i = threadIdx.x; i < m; i += 32) sq = fma(s_v[i], s_v[i], sq);
                    sq = warp_sum(sq);
                    if (threadIdx.x == 0) s_nu = sqrt(sq);
                }
                __syncthreads();
                for (int pass = 0; pass < 2; ++pass) {
                    // d_a = B_a . v for a < j, then v -= sum_a d_a B_a
                    for (int a = warp; a < j; a += NT / 32) {
                        const double* ba = B + perm[a] * ld;
                        double sdot = 0.0;
                        for (int i = lane; i < m; i += 32) sdot = fma(ba[i], s_v[i], sdot);
                        sdot = warp_sum(sdot);
                        if (lane == 0) s_d[a] = sdot;
                    }
                    __syncthreads();
                    for (int i = threadIdx.x; i < m; i += NT) {
                        double v = s_v[i];
                        for (int a = 0; a < j; ++a) v = fma(-s_d[a], B[perm[a] * ld + i], v);
                        s_v[i] = v;
                    }
                    __syncthreads();
                }
                if (threadIdx.x < 32) {
                    double sq = 0.0;
                    for (int i = threadIdx.x; i < m; i += 32) sq = fma(s_v[i], s_v[i], sq);
                    sq = warp_sum(sq);
                    if (threadIdx.x == 0) {
                        s_nv = sqrt(sq);
                        s_acc = (s_nv > (phase == 0 ? 0.5 : 1e-3) * s_nu) ? 1 : 0;
                    }
                }
                __syncthreads();
                if (s_acc) {
                    const double nv = s_nv;
                    for (int i = threadIdx.x; i < m; i += NT) B[perm[j] * ld + i] = s_v[i] / nv;
                    done = true;
                }
                __syncthreads();
            }
        }
    }
    return rho;
}

}  // namespace TITUS_WIDE_NS
}  // namespace titus
