// Device state of one team of the rank-adaptive DLR kernels (shared by the 2D
// and 3D compilations of the kernel; the host handle holds it).
#pragma once

namespace titus {

constexpr int WIDE_RA = 40;   // max rank entering a step (augmented widths up to 2 WIDE_RA)

struct WideState {
    double* X;      // n x KA
    double* W;      // N x KA
    double* K;      // n x RA
    double* KP;     // n x RA  projected K
    double* CX;     // n x RA  range-finder C (X side)
    double* L;      // N x RA
    double* LP;     // N x RA
    double* CW;     // N x RA
    double* psi0;   // n x QW
    double* psi1;
    double* dose;   // n
    double* S;      // KA x KA (state S, written back at exit)
    double* part;   // 2 x G x PMAXW
    double* red;    // 2 x PMAXW (double-buffered with the partials)
    double* scr;    // G x SCRW per-CTA scratch
    unsigned* bar;  // G + 1 barrier flags
    int* status;
    int* info;      // [0] rank, [1] iterations, [2] psi index, [3] next n, [4] eta count
    double* diag;   // 16
    double* tvar;   // [0] pseudo-time t (BUG / parallel)
    int* rank_hist; // hist_cap
    double* time_hist;
    double* eta_hist;
    double* bound_hist;
    double* X0;     // n x RA: X entering the energy, boundary rows zeroed (parallel-rejection loop)
    double* W0;     // N x RA: W entering the energy (parallel-rejection loop)
    int hist_cap;
};

}  // namespace titus
