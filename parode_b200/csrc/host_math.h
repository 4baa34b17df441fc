// host_math.h -- host-side FP64 set-up of a solve: step counts, time vector,
// RK4 / ABM discretisation into the affine one-step map, ABM start-up.
#pragma once

#include <vector>

namespace parode {

struct SystemDesc {
    int n = 0, m = 0, p = 0;          // states, inputs, outputs (p as passed by the caller)
    bool zeroB = true, zeroC = true, zeroD = true;
    std::vector<double> A, B, C, D, x0;  // row-major FP64
    // Output channels of a solve: p, or n when C and D are both absent
    // (reference Sources/GPUFixedStepIterative.cpp:62-74,122-123).
    int out_size() const { return (zeroC && zeroD) ? n : p; }
};

// Step counts.  RK4: T = (long)((tEnd - t0)/h) + 1 (reference
// Sources/RungeKutta4thOrder.cpp:20).  ABM: scan steps counted from t0 + 3h,
// outputs = scan steps + 3 (Sources/AdamsMoulton.cpp:356-358).  Returns the
// number of outputs or -1 for an empty horizon.
long num_outputs(int solver, double t0, double tEnd, double h, long* n_scan);

// tv[1..count) from tv[0]: tv[i+1] = float(tv[i] + h), the reference's
// float time accumulation, element for element.
void time_chain(double* tv, long count, double h);
// Time vector with the reference's float accumulation
// (Sources/GPUFixedStepIterative.cpp:141-146); written as double.
void time_vector(int solver, double t0, double tEnd, double h, double* tv);
// The same values stored as float (the reference C ABI's fType arrays).
void time_vector_f(int solver, double t0, double tEnd, double h, float* tv);

// One-step affine map.  Phi is Ns x Ns (Ns = n or 4n), Bbar is n x W*m
// (W = 3 for RK4, 5 for ABM), both row-major FP64.
void discretise_rk4(int n, int m, const double* A, const double* B, double h, double* Phi, double* Bbar);
void discretise_abm(int n, int m, const double* A, const double* B, double h, double* Phi, double* Bbar);
// The same ABM map with only the last block row of Phi (n x 4n): the block
// rows above it are the exact shift (block b reads block b + 1).
void discretise_abm_last(int n, int m, const double* A, const double* B, double h, double* last, double* Bbar);

// ABM start-up: X0 = [x0; x1; x2; x3] from three classical RK4 steps with the
// nine inputs U[j] = u(t0 + j h/2), j = 0..8 (U is 9 x m, row-major)
// (reference Sources/AdamsMoulton.cpp:29-104).
void abm_startup(const SystemDesc& s, const double* U9, double h, double* X0);

}  // namespace parode
