// Second-order limited upwind transport flux of the uncollided ordinates:
// solveFlux! (code/SolverCSD.jl:295-386) with its limiter helpers minmod and
// slopefit (:288-293), as the standalone C-ABI operator titus_limited_flux.
//
// Layout: phi and flux hold nx*ny*q doubles, cell (i, j) ordinate l at
// (i*ny + j)*q + l (the library's psi layout; i runs over x, j over y). The
// reference writes interior cells 2 <= i < nx-2, 2 <= j < ny-2 (1-based 3:N-2)
// and leaves the others as they were; so does this kernel.
//
// Each (cell, ordinate) needs the centre value and four neighbours per axis:
// offsets -2..+1 where the ordinate's component is >= 0, -1..+2 where it is
// negative. A thread owns one (j, l) pair and walks 32 rows along x: a warp
// reads 256 contiguous bytes per operand, rows shared by neighbouring blocks
// stay in L2, and DRAM sees phi once and flux once. The limiter arithmetic
// (limiter.cuh) keeps the reference's evaluation order, so the result is the
// same IEEE double as the FP64 restatement of the loop body.
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>

#include "../../include/titus.h"
#include "limiter.cuh"

namespace titus_host {
int fail(int code, const char* fmt, ...);
}

namespace {

constexpr int kFluxThreads = 256;

using titus_lim::face_neg;
using titus_lim::face_pos;

// y difference of one cell from its four neighbours (the face is not shared:
// adjacent j belong to other threads)
__device__ __forceinline__ double diff_y(double m2, double m1, double c, double p1, double p2, bool pos) {
    return titus_lim::axis_diff(m2, m1, c, p1, p2, pos);
}

constexpr int kRowsPerThread = 32;

// grid: x covers the ny*q (j, l) pairs of a row; y chunks of kRowsPerThread
// interior rows starting at row0 + kRowsPerThread*blockIdx.y. A thread walks its
// rows along x with a window of phi values, so each x face is formed once and
// each phi value along x is loaded once.
__global__ void __launch_bounds__(kFluxThreads) limited_flux_kernel(int nx, int ny, int q, int row0, double dx,
                                                                    double dy, const double* __restrict__ ox,
                                                                    const double* __restrict__ oz,
                                                                    const double* __restrict__ phi,
                                                                    double* __restrict__ flux) {
    const int t = blockIdx.x * kFluxThreads + threadIdx.x;
    const int row = ny * q;
    if (t >= row) return;
    const int j = t / q, l = t - (t / q) * q;
    if (j < 2 || j >= ny - 2) return;
    const int i0 = row0 + kRowsPerThread * (int)blockIdx.y;
    const int i1 = min(i0 + kRowsPerThread, nx - 2);
    if (i0 >= i1) return;
    const double wx = __ldg(ox + l), wz = __ldg(oz + l);
    // qReduced[q,1] / dx and qReduced[q,3] / dy, as the reference divides
    const double cx = __ddiv_rn(wx, dx), cz = __ddiv_rn(wz, dy);
    const bool px = wx >= 0.0, pz = wz >= 0.0;
    const size_t sx = (size_t)row;
    const size_t sq = (size_t)q;
    const double* p = phi + (size_t)i0 * sx + t;
    double* f = flux + (size_t)i0 * sx + t;
    // window: a = phi_{i-1}, b = phi_i, c = phi_{i+1}; H = face between i-1 and i
    double a = __ldg(p - sx), b = __ldg(p), c = __ldg(p + sx);
    double H = px ? face_pos(__ldg(p - 2 * sx), a, b) : face_neg(a, b, c);
    for (int i = i0; i < i1; ++i) {
        double Hn;
        double d = 0.0;
        if (px) {
            Hn = face_pos(a, b, c);                  // F+(i)
        } else {
            d = __ldg(p + 2 * sx);                   // phi_{i+2}
            Hn = face_neg(b, c, d);                  // F-(i+1)
        }
        const double ew = __dsub_rn(Hn, H);
        const double ns = pz ? diff_y(__ldg(p - 2 * sq), __ldg(p - sq), b, __ldg(p + sq), 0.0, true)
                             : diff_y(0.0, __ldg(p - sq), b, __ldg(p + sq), __ldg(p + 2 * sq), false);
        // qReduced[q,1] / dx * (east - west) + qReduced[q,3] / dy * (north - south)
        *f = __dadd_rn(__dmul_rn(cx, ew), __dmul_rn(cz, ns));
        H = Hn;
        a = b;
        b = c;
        c = px ? (i + 1 < i1 ? __ldg(p + 2 * sx) : 0.0) : d;   // phi_{i+2} (not needed after the last row)
        p += sx;
        f += sx;
    }
}

}  // namespace

extern "C" int titus_limited_flux(int32_t nx, int32_t ny, int32_t q, double dx, double dy, const double* omega_x,
                                  const double* omega_z, const double* phi, double* flux, void* stream) {
    using titus_host::fail;
    if (nx < 0 || ny < 0 || q < 1) return fail(TITUS_ERR_ARG, "titus_limited_flux: nx=%d ny=%d q=%d", nx, ny, q);
    if (!(dx > 0.0) || !(dy > 0.0)) return fail(TITUS_ERR_ARG, "titus_limited_flux: dx, dy must be > 0");
    if (!omega_x || !omega_z || !phi || !flux) return fail(TITUS_ERR_ARG, "titus_limited_flux: NULL pointer");
    if (nx < 5 || ny < 5) return TITUS_OK;   // no interior cell
    const long long row = (long long)ny * q;
    if (row > INT_MAX - kFluxThreads) return fail(TITUS_ERR_LIMIT, "titus_limited_flux: ny*q = %lld too large", row);
    const double* pb = phi;
    const double* fb = flux;
    const size_t total = (size_t)nx * (size_t)row;
    if (pb < fb + total && fb < pb + total)
        return fail(TITUS_ERR_ARG, "titus_limited_flux: phi and flux overlap");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const unsigned gx = (unsigned)((row + kFluxThreads - 1) / kFluxThreads);
    const long long chunks = (nx - 4 + kRowsPerThread - 1) / kRowsPerThread;
    // at most 65535 row chunks per launch (grid y limit)
    for (long long c0 = 0; c0 < chunks; c0 += 65535) {
        const unsigned gy = (unsigned)((chunks - c0) < 65535 ? (chunks - c0) : 65535);
        limited_flux_kernel<<<dim3(gx, gy), kFluxThreads, 0, st>>>(nx, ny, q, 2 + (int)(c0 * kRowsPerThread), dx, dy,
                                                                    omega_x, omega_z, phi, flux);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return fail(TITUS_ERR_CUDA, "titus_limited_flux: %s", cudaGetErrorString(e));
    }
    return TITUS_OK;
}
