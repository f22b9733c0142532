// titus_debug_tc_gram: the MIXED-precision tensor-core Gram run (umma.cuh) on
// a plain matrix, for the unit test of its layouts and synchronisation.
//
// F (rows x (nops + 1) nw, row-major) holds a factor A in columns [0, nw) and
// its nops operator images O_d A in columns [(d + 1) nw, (d + 2) nw). The call
// returns out[d][i][j] = sum_r (O_d A)[r][i] A[r][j] (nops x nw x nw) as the
// adaptive kernel's MIXED mode forms it: one CTA, chunks of 16 rows staged in
// hi/lo TF32, tcgen05 MMAs accumulating in TMEM, FP32 sums read back.
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/titus.h"
#include "umma.cuh"

namespace titus_host {
int fail(int code, const char* fmt, ...);
}

namespace {

using namespace titus::umma;
constexpr int kProbeThreads = 256;

template <int NOPS>
__global__ void __launch_bounds__(kProbeThreads, 1)
tc_gram_probe_kernel(const double* F, int rows, int nw, double* out, int* status) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ unsigned long long mbar[2];
    __shared__ uint32_t tmem_slot;
    const GramShape g = gram_shape(NOPS * nw, nw);
    if (threadIdx.x < 32) tmem_alloc(&tmem_slot, TMEM_COLS);
    if (threadIdx.x == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        fence_mbar_init();
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    TcCtx t;
    t.mbar = mbar;
    t.tmem = tmem_slot;
    t.phase[0] = t.phase[1] = 0u;
    t.pending[0] = t.pending[1] = 0;
    t.status = status;
    t.limit = kWaitCycles;
    const int ld = (NOPS + 1) * nw;
    const bool ok = gram_run<kProbeThreads, NOPS>(t, g, smem, rows, true, [&](int r, int j, double* v) {
        const double* row = F + (size_t)r * ld;
        v[0] = row[j];
#pragma unroll
        for (int d = 0; d < NOPS; ++d) v[1 + d] = row[(d + 1) * nw + j];
    });
    const bool fin = gram_finish(t);
    if (ok && fin)
        gram_read<kProbeThreads>(t, g, [&](int m, int n, double v) {
            const int d = m / nw, i = m - d * nw;
            out[((size_t)d * nw + i) * nw + n] = v;
        });
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (threadIdx.x < 32) tmem_dealloc(tmem_slot, TMEM_COLS);
}

template <int NOPS>
int launch_probe(const double* dF, int rows, int nw, double* dout, int* dst) {
    const GramShape g = {NOPS * nw, nw, (NOPS * nw + MTILE - 1) / MTILE, ((nw + 15) / 16) * 16, 0, 0, 0};
    const int m_bytes = g.mt * 2 * KSTEP_M, n_bytes = 2 * (g.np / 8) * 256;
    const int smem = 2 * 2 * (m_bytes + n_bytes);
    if (g.mt * g.np > TMEM_COLS) return titus_host::fail(TITUS_ERR_LIMIT, "titus_debug_tc_gram: accumulators exceed TMEM");
    cudaError_t e = cudaFuncSetAttribute(tc_gram_probe_kernel<NOPS>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return titus_host::fail(TITUS_ERR_CUDA, "titus_debug_tc_gram: %s", cudaGetErrorString(e));
    tc_gram_probe_kernel<NOPS><<<1, kProbeThreads, smem>>>(dF, rows, nw, dout, dst);
    e = cudaGetLastError();
    if (e != cudaSuccess) return titus_host::fail(TITUS_ERR_CUDA, "titus_debug_tc_gram: %s", cudaGetErrorString(e));
    return TITUS_OK;
}

}  // namespace

extern "C" int titus_debug_tc_gram(const double* F, int32_t rows, int32_t nw, int32_t nops, double* out) {
    using titus_host::fail;
    if (!F || !out) return fail(TITUS_ERR_ARG, "titus_debug_tc_gram: NULL pointer");
    if (rows < 1 || nw < 1 || nw > 80 || (nops != 1 && nops != 2 && nops != 4))
        return fail(TITUS_ERR_ARG, "titus_debug_tc_gram: rows %d, nw %d (1..80), nops %d (1, 2, 4)", rows, nw, nops);
    const size_t nF = (size_t)rows * (nops + 1) * nw, nO = (size_t)nops * nw * nw;
    double* dF = nullptr;
    double* dO = nullptr;
    int* dst = nullptr;
    int rc = TITUS_OK;
    cudaError_t e = cudaMalloc(&dF, nF * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&dO, nO * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&dst, sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(dF, F, nF * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(dO, 0, nO * sizeof(double));
    if (e == cudaSuccess) e = cudaMemset(dst, 0, sizeof(int));
    if (e != cudaSuccess) rc = fail(TITUS_ERR_CUDA, "titus_debug_tc_gram: %s", cudaGetErrorString(e));
    if (rc == TITUS_OK) {
        rc = nops == 1 ? launch_probe<1>(dF, rows, nw, dO, dst)
             : nops == 2 ? launch_probe<2>(dF, rows, nw, dO, dst)
                         : launch_probe<4>(dF, rows, nw, dO, dst);
    }
    if (rc == TITUS_OK) {
        e = cudaDeviceSynchronize();
        int st = 0;
        if (e == cudaSuccess) e = cudaMemcpy(&st, dst, sizeof(int), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(out, dO, nO * sizeof(double), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = fail(TITUS_ERR_CUDA, "titus_debug_tc_gram: %s", cudaGetErrorString(e));
        else if (st != 0) rc = fail(TITUS_ERR_DEVICE, "titus_debug_tc_gram: device status %d (completion wait timed out)", st);
    }
    cudaFree(dF);
    cudaFree(dO);
    cudaFree(dst);
    return rc;
}
