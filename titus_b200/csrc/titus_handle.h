// Host-side solver handle shared by the translation units of libtitus.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "../../include/titus.h"
#include "dlr_device.cuh"
#include "wide_state.h"

struct titus_solver;
struct titus_batch;
struct titus_pn_state;
struct titus_pn3_state;

namespace titus_host {

// Records the message for titus_last_error and returns `code`.
int fail(int code, const char* fmt, ...);

#define CK(call)                                                                                          \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess) return titus_host::fail(TITUS_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// Test hook (titus_debug_fail_alloc): when positive, the allocation that
// brings it to zero fails as if cudaMalloc had returned cudaErrorMemoryAllocation.
int take_alloc_fault();

template <class T>
int upload(T** dptr, const T* host, size_t count) {
    *dptr = nullptr;
    if (count == 0) return TITUS_OK;
    if (take_alloc_fault())
        return fail(TITUS_ERR_CUDA, "cudaMalloc(%zu bytes): %s (injected)", count * sizeof(T),
                    cudaGetErrorString(cudaErrorMemoryAllocation));
    CK(cudaMalloc((void**)dptr, count * sizeof(T)));
    if (host) CK(cudaMemcpy(*dptr, host, count * sizeof(T), cudaMemcpyHostToDevice));
    return TITUS_OK;
}

// rank-adaptive integrators (titus_adaptive.cu)
int wide_solve_device(titus_solver* s, int method, const titus_options_t* opt, cudaStream_t stream);
int wide_solve_from(titus_solver* s, int method, const titus_options_t* opt, int n_stop);
int wide_fetch(titus_solver* s, titus_result_t* res);
int wide_set_state(titus_solver* s, int rank, const double* X, const double* S, const double* W, const double* psi,
                   const double* dose, int n_next);
void wide_free(titus_solver* s);
// the BUG integrator on 3D problems (titus_adaptive3d.cu: the same source with six streaming pairs)
int wide_solve_device_3d(titus_solver* s, int method, const titus_options_t* opt, cudaStream_t stream);
int wide_solve_from_3d(titus_solver* s, int method, const titus_options_t* opt, int n_stop);
int wide_fetch_3d(titus_solver* s, titus_result_t* res);
int wide_set_state_3d(titus_solver* s, int rank, const double* X, const double* S, const double* W,
                      const double* psi, const double* dose, int n_next);
void wide_free_3d(titus_solver* s);
int batch_upload(titus_solver* s, int nspots, const titus_spot_t* spots, titus_batch** out);
int batch_launch(titus_batch* b, int method, const titus_options_t* opt, cudaStream_t stream);
int batch_fetch(titus_batch* b, double* dose_out, int32_t* rank_out, int32_t* iters_out);
void batch_free(titus_batch* b);
int batch_rank_sums(titus_batch* b, int32_t* out);
// full-rank P_N solver state (titus_pn_full.cu; 3D: titus_pn3d.cu)
void pn_free(titus_solver* s);
void pn3_free(titus_solver* s);
int pn3_solve_device(titus_solver* s, const titus_options_t* opt, cudaStream_t stream);
int pn3_fetch(titus_solver* s, double* u_out, double* dose_out, double* psi_out);
int wide_solve_batched(titus_solver* s, int method, const titus_options_t* opt, int nspots, const titus_spot_t* spots,
                       double* dose_out, int32_t* rank_out, int32_t* iters_out);

}  // namespace titus_host

struct titus_solver {
    titus::DevProblem P{};
    int n = 0, N = 0, q = 0, nE = 0;
    std::vector<void*> allocs;
    // fixed-rank team state
    titus::TeamState st{};
    titus::TeamState* d_st = nullptr;
    int team_ctas = 0;
    int device = 0;
    int num_sms = 0;
    int r = 0;
    int last_method = -1;
    int last_G = 0;
    unsigned long long* prof = nullptr;
    int clock_khz = 0;
    // rank-adaptive state (allocated on first use)
    titus::WideState wst{};
    titus::WideState* d_wst = nullptr;
    std::vector<void*> wide_allocs;
    // batched teams (allocated on first batched solve, grown on demand)
    std::vector<titus::WideState> bst;
    titus::WideState* d_bst = nullptr;
    int b_teams = 0, b_G = 0;
    std::vector<void*> batch_allocs;
    int wide_state_valid = 0;   // 1 after an adaptive solve or titus_set_state
    // full-rank P_N solver (allocated on first use) and csd.SMid
    titus_pn_state* pn = nullptr;
    // 3D problems (titus_create_3d): z layers, spacing, the z pair Ay / |Ay|
    // (device CSR) and the 3D full-rank solver state
    int nz = 0;
    double dz = 0.0;
    titus::Csr op3[2] = {};
    titus_pn3_state* pn3 = nullptr;
    double* smid = nullptr;
    // test hook (titus_debug_barrier_fault), consumed by the next launch
    long long dbg_spin_limit = 0;
    int dbg_fault_barrier = 0;
    void take_debug_hooks(titus::DevProblem& P) {
        P.spin_limit = dbg_spin_limit;
        P.fault_barrier = dbg_fault_barrier;
        dbg_spin_limit = 0;
        dbg_fault_barrier = 0;
    }

    template <class T>
    int alloc(T** p, size_t count, const T* host = nullptr) {
        int rc = titus_host::upload(p, host, count);
        if (rc == TITUS_OK && *p) allocs.push_back((void*)*p);
        return rc;
    }
    template <class T>
    int walloc(T** p, size_t count) {
        int rc = titus_host::upload(p, (const T*)nullptr, count);
        if (rc == TITUS_OK && *p) wide_allocs.push_back((void*)*p);
        return rc;
    }
    ~titus_solver();
};
