// 5th-generation tensor-core (tcgen05) Gram products for the MIXED precision
// mode of the rank-adaptive kernel: D = Mop^T Nop over a run of rows, where
// Mop is the rows x mw matrix of operator images (L_d A or A_d B, stacked)
// and Nop the rows x nw matrix of the factor itself, in TF32 with FP32
// accumulation in tensor memory (TMEM) and a hi/lo split of every FP64 input
// (x = hi + lo, D += hi_M hi_N + hi_M lo_N + lo_M hi_N: about 21 significant
// bits per product instead of TF32's 11).
//
// Layout. Both operands are staged K-major (the row index of the Gram is the
// MMA's K) without swizzle, in the canonical arrangement of 8-row x 16-byte
// core matrices: element (m, k) of a K-step of 8 rows sits at
//   (m / 8) * 256 + ((k % 8) / 4) * 128 + (m % 8) * 16 + (k % 4) * 4  bytes,
// i.e. LBO = 128 B between the two 16-byte K groups and SBO = 256 B between
// 8-row groups. A staged chunk holds KC = 16 rows (two K-steps) of every
// operand, hi and lo; two chunk buffers alternate so that converting chunk
// c + 1 overlaps the MMAs of chunk c. The M operand is cut into tiles of 128
// rows (cta_group::1, M = 128: row m of a tile is TMEM lane m); the N operand
// is padded to a multiple of 16. Rows of a tile beyond the operand read other
// staged data and only produce accumulator rows that are never read.
//
// Synchronisation: one elected thread issues the MMAs and commits them to the
// chunk buffer's mbarrier; every wait is bounded and reports failure instead
// of spinning forever. TMEM (TMEM_COLS columns) is allocated once per CTA by
// warp 0 at kernel start and freed at kernel exit.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace titus {
namespace umma {

constexpr int KC = 16;           // staged rows per chunk (two K-steps of 8)
constexpr int MTILE = 128;       // M rows per MMA tile
constexpr int KSTEP_M = 16 * 256;  // bytes of one K-step of a 128-row tile (16 groups of 8 rows)
constexpr int TMEM_COLS = 512;   // accumulator columns allocated per CTA
constexpr int kStatusTcTimeout = 8;  // device status: a tensor-core completion wait timed out
constexpr long long kWaitCycles = 2000000000LL;  // bound of one completion wait (about a second)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: K-major, no swizzle, LBO 128 B, SBO 256 B,
// descriptor version 1 (bits 46-47), base offset 0, layout type 0.
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr) {
    uint64_t d = static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
    d |= static_cast<uint64_t>(128 >> 4) << 16;
    d |= static_cast<uint64_t>(256 >> 4) << 32;
    d |= static_cast<uint64_t>(1) << 46;
    return d;
}

// Instruction descriptor of kind::tf32: D F32 (bits 4-5 = 1), A and B TF32
// (bits 7-9, 10-12 = 2), both K-major (bits 15, 16 = 0), N >> 3 at bits 17-22,
// M >> 4 at bits 24-28.
__device__ __forceinline__ uint32_t idesc_tf32(int M, int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
           (static_cast<uint32_t>(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrive on `mbar` once every tcgen05 operation issued so far by this thread has completed.
__device__ __forceinline__ void mma_commit(unsigned long long* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :
                 : "r"(smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(unsigned long long* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_u32(mbar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" : : : "memory");
}

// Wait for the completion of the phase with the given parity; gives up after
// `limit` SM clock cycles (about 2e9 = one second).
__device__ __forceinline__ bool mbar_wait(unsigned long long* mbar, uint32_t parity, long long limit) {
    const uint32_t addr = smem_u32(mbar);
    const long long t0 = clock64();
    while (clock64() - t0 < limit) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" : : : "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" : : : "memory"); }
// make this thread's generic-proxy shared-memory writes visible to the tensor core
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" : : : "memory"); }

// TMEM allocation by one full warp; the base address is written to *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(slot)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" : : : "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" : : "r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 accumulator columns of this thread's TMEM lane (warp
// w reads lanes 32 (w % 4) .. 32 (w % 4) + 31).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" : : : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// hi/lo split of an FP64 value into two TF32 bit patterns (the tensor core
// reads the 19 high bits of each 32-bit word).
__device__ __forceinline__ void split_tf32(double v, uint32_t& hi, uint32_t& lo) {
    const float f = static_cast<float>(v);
    const uint32_t h = __float_as_uint(f) & 0xFFFFE000u;
    hi = h;
    lo = __float_as_uint(static_cast<float>(v - static_cast<double>(__uint_as_float(h))));
}

// Byte offset of element (m, k) (k < KC) of an operand block with `groups`
// 8-row groups per K-step.
__device__ __forceinline__ int stage_off(int m, int k, int groups) {
    return (k >> 3) * groups * 256 + (m >> 3) * 256 + ((k & 7) >> 2) * 128 + (m & 7) * 16 + (k & 3) * 4;
}

// Shapes of one Gram run: the M operand (mw columns, in mt tiles of 128) and
// the N operand (nw columns padded to np, a multiple of 16 and <= 256).
// TMEM holds mt np <= TMEM_COLS accumulator columns.
struct GramShape {
    int mw, nw, mt, np;
    int m_bytes;   // one of hi / lo of the M operand per chunk: mt * 2 K-steps * KSTEP_M
    int n_bytes;   // the same for N: 2 K-steps * (np / 8) * 256
    int buf_bytes; // one chunk buffer: 2 (m_bytes + n_bytes)
};
__device__ __forceinline__ GramShape gram_shape(int mw, int nw) {
    GramShape g;
    g.mw = mw;
    g.nw = nw;
    g.mt = (mw + MTILE - 1) / MTILE;
    g.np = ((nw + 15) / 16) * 16;
    g.m_bytes = g.mt * 2 * KSTEP_M;
    g.n_bytes = 2 * (g.np / 8) * 256;
    g.buf_bytes = 2 * (g.m_bytes + g.n_bytes);
    return g;
}

// Per-CTA tensor-core context (shared memory words and the TMEM base).
struct TcCtx {
    unsigned long long* mbar;  // 2 mbarriers (one per chunk buffer)
    uint32_t tmem;      // TMEM base address
    uint32_t phase[2];  // next parity to wait for, per buffer
    int pending[2];     // 1 while a commit on that buffer has not been waited for
    int* status;        // device error flag (set on a timed-out wait)
    long long limit;    // clock cycles per wait
};

// Bounded wait for the MMAs committed on buffer `s`; every thread of the CTA
// calls it with the same state.
__device__ __forceinline__ bool tc_drain(TcCtx& t, int s) {
    if (!t.pending[s]) return true;
    const bool ok = mbar_wait(t.mbar + s, t.phase[s], t.limit);
    t.phase[s] ^= 1u;
    t.pending[s] = 0;
    if (!ok && threadIdx.x == 0) atomicExch(t.status, kStatusTcTimeout);
    return ok;
}

// Operator Gram run: the N operand is a factor A (nw columns) and the M
// operand its NOPS operator images stacked, M = [O_0 A | ... | O_{NOPS-1} A]
// (mw = NOPS nw), so D[d nw + i][j] = sum_rows (O_d A)[r][i] A[r][j]. D of M
// tile `tile` lives in TMEM columns [tile np, (tile + 1) np). row(r, j, v)
// fills v[0] = A[r][j] and v[1 + d] = (O_d A)[r][j] for row r (0-based within
// the run). The staging area must hold 2 buf_bytes bytes, 16-byte aligned.
// `first` = true starts a fresh accumulation. Returns false if a wait timed
// out (status set).
template <int NTH, int NOPS, class Row>
__device__ bool gram_run(TcCtx& t, const GramShape& g, unsigned char* stage, int rows, bool first, Row row) {
    const int nchunks = (rows + KC - 1) / KC;
    const int nw = g.nw;
    for (int c = 0; c < nchunks; ++c) {
        const int s = c & 1;
        if (!tc_drain(t, s)) return false;   // buffer s is free again
        unsigned char* buf = stage + s * g.buf_bytes;
        unsigned char* m_hi = buf;
        unsigned char* m_lo = buf + g.m_bytes;
        unsigned char* n_hi = buf + 2 * g.m_bytes;
        unsigned char* n_lo = n_hi + g.n_bytes;
        const int r0 = c * KC;
        for (int e = threadIdx.x; e < KC * nw; e += NTH) {
            const int k = e / nw, j = e - (e / nw) * nw;
            double v[NOPS + 1];
            if (r0 + k < rows) {
                row(r0 + k, j, v);
            } else {
#pragma unroll
                for (int d = 0; d <= NOPS; ++d) v[d] = 0.0;
            }
            uint32_t hi, lo;
            split_tf32(v[0], hi, lo);
            const int on = stage_off(j, k, g.np / 8);
            *reinterpret_cast<uint32_t*>(n_hi + on) = hi;
            *reinterpret_cast<uint32_t*>(n_lo + on) = lo;
#pragma unroll
            for (int d = 0; d < NOPS; ++d) {
                const int m = d * nw + j, tile = m / MTILE, ml = m - tile * MTILE;
                const int o = tile * 2 * KSTEP_M + stage_off(ml, k, 16);
                split_tf32(v[1 + d], hi, lo);
                *reinterpret_cast<uint32_t*>(m_hi + o) = hi;
                *reinterpret_cast<uint32_t*>(m_lo + o) = lo;
            }
        }
        fence_async_smem();
        fence_before_sync();
        __syncthreads();
        if (threadIdx.x == 0) {
            fence_after_sync();
            const uint32_t id = idesc_tf32(MTILE, g.np);
            const uint32_t a_hi = smem_u32(m_hi), a_lo = smem_u32(m_lo);
            const uint32_t b_hi = smem_u32(n_hi), b_lo = smem_u32(n_lo);
            for (int tile = 0; tile < g.mt; ++tile) {
                const uint32_t d = t.tmem + static_cast<uint32_t>(tile * g.np);
                for (int ks = 0; ks < 2; ++ks) {
                    const uint32_t ao = tile * 2 * KSTEP_M + ks * KSTEP_M;
                    const uint32_t bo = ks * (g.np / 8) * 256;
                    const uint32_t acc0 = (first && c == 0 && ks == 0) ? 0u : 1u;
                    mma_tf32(d, desc_kmajor(a_hi + ao), desc_kmajor(b_hi + bo), id, acc0);
                    mma_tf32(d, desc_kmajor(a_hi + ao), desc_kmajor(b_lo + bo), id, 1u);
                    mma_tf32(d, desc_kmajor(a_lo + ao), desc_kmajor(b_hi + bo), id, 1u);
                }
            }
            mma_commit(t.mbar + s);
        }
        t.pending[s] = 1;
    }
    return true;
}

// Wait for every outstanding MMA and make the accumulators readable.
__device__ __forceinline__ bool gram_finish(TcCtx& t) {
    const bool a = tc_drain(t, 0);
    const bool b = tc_drain(t, 1);
    fence_after_sync();
    return a && b;
}

// Read the accumulators back: for every valid (m < mw, n < nw) call
// out(m, n, value) with the FP32 sum. Warps w and w + 4 share TMEM lane
// quadrant w % 4 and split the 16-column groups between them.
template <int NTH, class Out>
__device__ void gram_read(const TcCtx& t, const GramShape& g, Out out) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int quad = warp & 3, half = warp >> 2, halves = NTH / 128;
    for (int tile = 0; tile < g.mt; ++tile) {
        const int m = tile * MTILE + quad * 32 + lane;
        for (int cg = half; cg < g.np / 16; cg += halves) {
            float v[16];
            tmem_ld16(t.tmem + (static_cast<uint32_t>(quad * 32) << 16) + static_cast<uint32_t>(tile * g.np + cg * 16),
                      v);
            if (m < g.mw) {
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    if (cg * 16 + i < g.nw) out(m, cg * 16 + i, static_cast<double>(v[i]));
            }
        }
    }
    fence_before_sync();
    __syncthreads();
}

}  // namespace umma
}  // namespace titus
