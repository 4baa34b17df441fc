// blocked.h -- the blocked (fused) Blelloch scan for scan dimensions <= 64.
//
// The time axis is cut into blocks of B = 2^R steps.  One persistent kernel
// (the leaf) generates the inputs, forms the forcing terms, runs the R lowest
// Blelloch levels of every block in shared memory with the power-table
// matrices P_0..P_{R-1} resident on chip, records each block's aggregate,
// finishes the down-sweep from a zero root and writes y_local = C z + D u.
// The block aggregates are scanned by the same level machinery (blocks of
// blocks, FP64, seeded with the initial state), and a last pass adds the
// carried free response C Phi^j X_block to the outputs.  By linearity this is
// exactly the down-sweep seeded with the carry (x = z + Phi^j X).
#pragma once

#include <cuda_runtime.h>

namespace parode {

struct BlockedShape {
    int NP = 0;       // padded scan dimension (8, 16, 32 or 64)
    int R = 0;        // Blelloch levels per block
    int B = 0;        // block length 2^R
    int S = 0;        // steps per leaf tile (multiple of B)
    int S_items = 0;  // items per tile in the carry kernels
    size_t leaf_smem = 0, items_smem = 0;
};

// Chooses the shape for a scan dimension Ns and input width m; returns false
// when the blocked path does not apply (the level-synchronous path is used).
bool blocked_shape(int Ns, int m, int solver, BlockedShape* out);

struct LeafArgs {
    int solver = 0;       // 0 RK4, 1 ABM
    int n = 0, m = 0, p = 0;
    int zeroB = 1, zeroC = 1, zeroD = 1;
    long nScan = 0;       // scan steps
    long ntiles = 0;
    long ybase = 0;       // first output row written by the scan (0 RK4, 3 ABM)
    const double* P = nullptr;     // power table, levels x NP x NP
    const double* Bbar = nullptr;  // n x W*m
    const double* C = nullptr;     // p x n
    const double* D = nullptr;     // p x m
    const double* U = nullptr;     // input samples (when not generated)
    int gen = 0;                   // 1: sum-of-sinusoids generated on chip
    int stage = 0;                 // 1: Bbar, C, D copied to shared memory (leaf_smem includes them)
    const double* sa = nullptr;    // sinusoid a | f | phi (m x K each)
    const double* sf = nullptr;
    const double* sphi = nullptr;
    int K = 0;
    double u_base = 0, u_dt = 0;   // sample time base + dt * j
    double* Y = nullptr;           // outputs (rows ybase .. ybase + nScan)
    double* G = nullptr;           // block aggregates (ntiles*S/B x NP)
    int* status = nullptr;         // set non-zero by a device wait that gave up
};

// Mixed-precision (3xTF32 tcgen05) leaf: shared-memory bytes, or 0 when the
// shape is not supported (NP < 16 or too large).
size_t blocked_leaf_tc_bytes(const BlockedShape& sh, int n, int m, int p, int solver);
void launch_blocked_leaf_tc(const BlockedShape& sh, const LeafArgs& a, int grid, cudaStream_t s);

// Shared-memory bytes of the leaf with Bbar, C and D staged, or 0 when they
// do not fit next to the tile.
size_t blocked_leaf_stage_bytes(const BlockedShape& sh, int n, int m, int p, int solver);
void launch_blocked_leaf(const BlockedShape& sh, const LeafArgs& a, int grid, cudaStream_t s);

// Exclusive affine scan of `count` items (NP doubles each, in place) whose
// maps are (P_{base_level + R*...}, item): blocks of blocks through the level
// hierarchy, seeded with X0 at the top.  work: scratch of
// blocked_items_scratch(count) doubles.  Returns the number of launches.
long blocked_items_scratch(const BlockedShape& sh, long count);
int launch_blocked_carry(const BlockedShape& sh, double* items, long count, int base_level, const double* P,
                         const double* X0, double* work, int sms, cudaStream_t s);

// y[ybase + j] += CP[j mod B] X[j div B] for j < nScan; CP is B x p x NP.
void launch_blocked_fixup(const BlockedShape& sh, double* Y, long ybase, long nScan, int p, const double* CP,
                          const double* X, cudaStream_t s);

// P_l = P_{l-1}^2 for l in [l0, l1) (single CTA, NP <= 64), then, when CP is
// not null, CP[i] = Cext Phi^i for i < B (Cext: p x NP, the output rows of the
// scan state) by doubling with the table: CP[i + 2^k] = CP[i] P_k.
// Loads the carry kernels (items up / top / down, power tables) on the
// current device.  With lazy module loading a kernel's module is otherwise
// loaded, and its device memory mapped, at its first launch.
void preload_blocked_carry_kernels();

// Set-up of the allocation-free affine scan (noalloc.cu) on device `dev`:
// resolves its static scratch and loads its kernels, so that no later call
// maps device memory.
void noalloc_setup_device(int dev);

void launch_blocked_tables(const BlockedShape& sh, double* P, int l0, int l1, double* CP, const double* Cext, int p,
                           cudaStream_t s);

// ---------------------------------------------------------------------------
// Batched form: many independent systems of one padded dimension NP.  Each
// system is described by a LeafArgs (P holds power-table levels 0..R, G its
// block aggregates, which the chain stage turns into block carries).  Stages,
// in order: 0 tables (one CTA per system: P levels 1..R and CP), 1 leaf
// (work items = tile ranges, largest first, dealt round-robin to the CTAs),
// 2 chain (one CTA per system: X_{b+1} = P_R X_b + G_b in FP64, sequential
// over the system's blocks), 3 fix-up (y += C Phi^j X_b).
// ---------------------------------------------------------------------------

struct BatchItem {
    int sys = 0;
    int pad = 0;
    long t0 = 0, t1 = 0;  // tiles [t0, t1) of system `sys`
};

struct BatchLaunch {
    const LeafArgs* sys = nullptr;     // device, nsys entries
    int nsys = 0;
    const BatchItem* items = nullptr;  // device, nitems entries
    int nitems = 0;
    int grid = 0;                      // leaf CTAs
    int ms = 0;                        // largest m (sample staging width)
    size_t leaf_smem = 0;
    double* const* CPs = nullptr;      // device array of per-system CP tables (B x p x NP)
    const double* const* Cexts = nullptr;
    const double* const* X0s = nullptr;
    long max_blocks = 0;               // largest block count of a system
    int pmax = 1;
};

// Leaf shared memory for a batch: sample staging for the widest input and
// `stage_doubles` of staged Bbar | C | D (0 when not staged).
size_t batch_leaf_smem(const BlockedShape& sh, int ms, long stage_doubles);
void launch_batch_stage(int what, const BlockedShape& sh, const BatchLaunch& b, cudaStream_t s);

}  // namespace parode
