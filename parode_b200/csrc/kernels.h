// kernels.h -- host launchers of the device kernels (FP64 path).
#pragma once

#include <cuda_runtime.h>

#include <vector>

namespace parode {

// Samples per thread of the input-sampling kernels: one thread advances one
// channel over a run of this many consecutive samples.
constexpr int kSampleRun = 64;

// Column addressing of the batched affine-level contraction:
//   result(g, i) = sum_k P[i][k] * src(g, k) (+ acc(g, i))
// src(g,k) = src[g*src_gs + k*src_ks], acc/dst/cpy likewise with (g, i).
struct LevelArgs {
    const double* P = nullptr;
    long ldp = 0;
    int Np = 0;          // rows of P == contraction length (multiple of 8)
    long ncols = 0;
    const double* src = nullptr;
    long src_gs = 0, src_ks = 1;
    const double* acc = nullptr;  // may be null (no accumulate)
    long acc_gs = 0, acc_is = 1;
    double* dst = nullptr;
    long dst_gs = 0, dst_is = 1;
    double* cpy = nullptr;  // down-sweep: cpy(g,i) <- old src(g,i)
    long cpy_gs = 0, cpy_is = 1;
    // Mixed form only: an exact 0/1 part R of P with one 1 per row, taken out
    // of the tensor-core product and added back in FP64 (P v = R v + (P - R) v).
    // rn < 0: none; rn == 0: R = I; rn > 0: ABM companion blocks of rn rows,
    // row block b reads block min(b + rsh, 3).
    int rn = -1, rsh = 0;
    // Mixed form only: P - R pre-split into TF32 hi/lo tiles (level_split_bytes).
    const float* Ps = nullptr;
    // Mixed form only: device address of a 128-byte TMA tensor map over the
    // source columns (level_encode_src_map).
    const void* src_map = nullptr;
    // General shapes (tiled kernel only): rows of P (0: Np) and contraction
    // length (0: Np); dst_limit >= 0 drops every result whose linear offset
    // g*dst_gs + i*dst_is is at or beyond it (a ragged last column).
    int M = 0, K = 0;
    long dst_limit = -1;
    // Two-part source (tiled kernel, K-contiguous only): contraction indices
    // k >= K1 (K1 > 0, even) read src2(g, k - K1) = src2[g*src2_gs + k - K1].
    int K1 = 0;
    const double* src2 = nullptr;
    long src2_gs = 0;
    // Tiled kernel: columns g >= src_cols (> 0) read a zero source, so their
    // results are acc or 0 (a zero padding written by the same launch).
    long src_cols = 0;
    // Tensor-core kernel, test hook: non-zero makes CTA 0 withhold the
    // arrive of its first K slice, so the waits on that stage give up.
    int fault_withhold = 0;
};

// One GEMM of the mixed block-response leaf (kernels_resp_tc.cu):
// dst(g, i) = sum_k W[i][k] window_g[k] for rows i < rows of W and windows g,
// W pre-split (k_split of the LevelArgs with the same rows and K), the
// windows read from the sample planes through `maps` (two 128-byte TMA maps,
// resp_encode_plane_maps).  dst_limit >= 0 drops results at or beyond that
// linear offset (the last block's steps past the horizon).
struct RespArgs {
    const float* Ps = nullptr;
    int rows = 0, K = 0;
    long ncols = 0;
    const void* maps = nullptr;
    double* dst = nullptr;
    long dst_gs = 0, dst_is = 1, dst_limit = -1;
    int fault_withhold = 0;  // test hook, as LevelArgs::fault_withhold
};

// The initial-state part of the block-response outputs (kernels_state.cu):
// Y[b gs + r] = acc[b gs + r] + sum_k W[r ld + k] X[b NP + k] for r < M,
// b < nblocks, b gs + r < limit (limit < 0: none).  Returns false when W's
// M x NP state columns do not fit in shared memory (the caller then uses the
// tiled GEMM).
bool launch_state_out(int NP, const double* W, long ld, int M, const double* X, const double* acc, double* Y, long gs,
                      long nblocks, long limit, int sms, cudaStream_t s);

long resp_tc_tiles(const RespArgs& a);
std::vector<long> resp_tc_ranges(const std::vector<RespArgs>& ents, int ctas);
// Two tensor maps (hi plane, lo plane) of windows: row g starts at sample
// offset g * block_stride, K samples long; written to out (256 bytes; only
// the first when lo is null).
void resp_encode_plane_maps(const float* hi, const float* lo, long ncols, int K, long block_stride, void* out);
// one_pass: hi*hi only (the single-pass TF32 form; the lo planes and W's lo
// halves are not read).
void launch_resp_tc(const RespArgs* dArgs, const long* dStart, int nent, const long* dCta, int ctas, int* status,
                    bool one_pass, cudaStream_t s);

__host__ __device__ inline int level_rows(const LevelArgs& a) { return a.M > 0 ? a.M : a.Np; }
__host__ __device__ inline int level_k(const LevelArgs& a) { return a.K > 0 ? a.K : a.Np; }

// One Blelloch level over all columns (up-sweep, down-sweep or P*P).
void launch_affine_level(const LevelArgs& a, cudaStream_t s);

// dst(g, i) = sum_k P[i][k] src(g, k) (+ acc) for a general rows x K matrix P
// (a.M, a.K; K even) with the tiled FP64 DMMA kernel.
void launch_gemm_tiled(const LevelArgs& a, cudaStream_t s);

// Block response matrix of one system (kernels_br.cu): W (B p + NP rows, Kpad
// columns, row-major) maps a block's input-sample window to its zero-seeded
// local outputs (rows j p + o) and aggregate (rows B p + r).
struct ResponseArgs {
    int solver = 0, n = 0, m = 0, p = 0, NP = 0, B = 0;
    int zeroB = 1, zeroD = 1;
    const double* Phi = nullptr;   // NP x NP
    const double* Bbar = nullptr;  // n x W m
    const double* Cext = nullptr;  // p x NP (output rows of the scan state)
    const double* D = nullptr;     // p x m
    double* Wm = nullptr;          // row stride Kpad + NPstate
    int K = 0, Kpad = 0;           // window columns, padded to even
    int NPstate = 0;               // NP: also the initial-state columns (z_0 = I on them), or 0
    // launch_response_init / response_doubling_args / response_product_args /
    // launch_response_fill only, carved from one workspace of
    // response_workspace_doubles by response_workspace_carve:
    // CPt: B p x NP (CP_j = Cext Phi^j, block j at j p NP);
    // Qt: NP x B n2 (Q_k = Phi^k restricted to the n forcing columns, row-major
    //     with pitch B n2, Q_k at columns k n2, n2 = n rounded up to even);
    // BbarE: NP x WM2 (Bbar in the forcing rows, WM2 = W m rounded up to even);
    // MT: B p x WM2 (CP_L Bbar per slot), NT: NP B x WM2 (Q_L Bbar per slot).
    double* CPt = nullptr;
    double* Qt = nullptr;
    double* BbarE = nullptr;
    double* MT = nullptr;
    double* NT = nullptr;
};
// Window length (columns of W) for B steps: RK4 (2B + 1) m, ABM (B + 4) m.
int response_window(int solver, int B, int m);
void launch_block_response(const ResponseArgs* dArgs, int nsys, int max_np, int max_p, int max_kpad, cudaStream_t s);
// The same W for any NP, over many systems.  dStart[e] is entry e's first CTA
// (response_init_ctas / response_fill_ctas CTAs each, `ctas` in total).
// Order: init (CP_0, Q_0, BbarE); for l = 0 .. log2(B) - 1 the tiled GEMMs of
// response_doubling_args (P = the power table, P_l at l NP^2), which double
// the tables from 2^l to 2^(l+1) entries; the two GEMMs of
// response_product_args; then one fill.
long response_init_ctas(const ResponseArgs& a);
long response_fill_ctas(const ResponseArgs& a);
void launch_response_init(const ResponseArgs* dArgs, const long* dStart, int nent, long ctas, cudaStream_t s);
// Fills out[0..1] (N-contiguous tiled GEMMs) and returns their count (0 once 2^l >= B).
int response_doubling_args(const ResponseArgs& a, const double* P, int l, LevelArgs out[2]);
// The two GEMMs that fold the slots of Bbar into the tables (MT and NT), after the doubling.
void response_product_args(const ResponseArgs& a, LevelArgs out[2]);
size_t response_workspace_doubles(const ResponseArgs& a);
void response_workspace_carve(ResponseArgs& a, double* ws);
void launch_response_fill(const ResponseArgs* dArgs, const long* dStart, int nent, long ctas, cudaStream_t s);
// Block length 2^R of the response leaf for one system, and its cost in
// FP64-equivalent flops per step (the two GEMMs and a level-synchronous carry
// over blocks); window_weight scales the window and aggregate products (1 in
// FP64, the tensor cores' relative cost in the mixed form).
int response_log2_block(int solver, int NP, int n, int m, int p, long nScan, double window_weight, double executions,
                        double* flops_per_step);

// Exclusive scan of block aggregates for NP <= 64 (a multiple of 8),
// kernels_carry.cu: items[b] <- X_b with X_0 = X0, X_{b+1} = Q X_b + items[b],
// Q = P_{l0} (P: power table, level l at l NP^2).  Chunks of 16 per level;
// level h uses P_{l0 + 4h} .. P_{l0 + 4h + 3}, so the table must hold
// l0 + chunk_carry_table_levels(count) levels.  h0: the global index of the
// call's first chunk level (0 for a whole scan; a time-partitioned solve's top
// scan starts higher), which picks each level's form.  work:
// chunk_carry_scratch(count) NP doubles.  Returns the launches made.
int chunk_carry_levels(long count);
int chunk_carry_table_levels(long count);
long chunk_carry_scratch(long count);
int launch_chunk_carry(int NP, double* items, long count, const double* P, int l0, int h0, const double* X0,
                       double* work, cudaStream_t s);
// The same scan in its two halves, for a scan whose top level is done
// elsewhere (the time partition of one solve across devices): the up-sweep
// leaves the chunk aggregates of level h in arr[h] (h = `levels`, or while
// more than 16 items remain when levels < 0); once arr[h] holds the states
// entering its items, the down-sweep rewrites every lower level (items end as
// the states entering them).
struct ChunkLevels {
    double* arr[16] = {};
    long cnt[16] = {};
    int h = 0;
};
int launch_chunk_up(int NP, double* items, long count, const double* P, int l0, double* work, int levels,
                    ChunkLevels* L, cudaStream_t s);
int launch_chunk_down(int NP, const ChunkLevels& L, const double* P, int l0, cudaStream_t s);

// Columns of a level that can reach an output.  Column g combines the
// segments [g 2d, g 2d + d) and [g 2d + d, g 2d + 2d) of the time axis; when
// g 2d >= nScan both segments are padding: the column holds zeros in the
// up-sweep and writes only padding slots in the down-sweep, so it is skipped.
inline long sweep_columns(long nScan, long Tp, long d)
{
    const long all = Tp / (2 * d), used = (nScan + 2 * d - 1) / (2 * d);
    return used < all ? used : all;
}

// U[j*m + i] = sum_k a sin(2 pi f t_j + phi), t_j = base + dt*j, j < count.
void launch_sinusoid_samples(double* U, int m, int K, const double* a, const double* f, const double* phi,
                             double base, double dt, long count, cudaStream_t s, long joff = 0);

// The same samples written as TF32 hi / lo planes (hi = TF32(x),
// lo = TF32(x - hi), x = float(u)), the tensor-core GEMMs' operand form.
void launch_sinusoid_planes(float* hi, float* lo, int m, int K, const double* a, const double* f, const double* phi,
                            double base, double dt, long count, cudaStream_t s, long joff = 0);
// FP64 samples into those planes (n values).  lo may be null in both (hi only).
void launch_split_planes(const double* U, float* hi, float* lo, long n, cudaStream_t s);
// dst[i] = (float)src[i], i < n
void launch_to_float(const double* src, float* dst, long n, cudaStream_t s);

// The batch's discretisation on the device (kernels_disc.cu): one job per
// system, A (n x n) and B (n x m, m = 0 without B) in, the compact Phi (RK4
// n x n; ABM the last block row, n x 4n), Bbar (n x W max(m, 1), W = 3 / 5)
// and, when bbarT is set, its transpose out, with ||Phi - R||_inf into
// *delta when delta is set; work: discretise_work_doubles(n, m) doubles.  The same bits as the
// host restatement (host_math.cpp).  The products run first, as 32 x 32
// output tiles in three dependency stages (discretise_tiles lists a job's
// tiles of one stage, with the job's device pointers).
struct DiscJob {
    const double* A = nullptr;
    const double* B = nullptr;
    double* phi = nullptr;
    double* bbar = nullptr;
    double* bbarT = nullptr;
    double* work = nullptr;
    double* delta = nullptr;
    int n = 0, m = 0, solver = 0;
    double h = 0.0;
};
struct DiscTile {
    const double* X = nullptr;
    const double* Y = nullptr;
    double* Z = nullptr;
    int r = 0, k = 0, c = 0, i0 = 0, j0 = 0;
};
long discretise_work_doubles(int n, int m);
void discretise_tiles(const DiscJob& j, int stage, std::vector<DiscTile>& out);
// tiles[st] / ntiles[st]: device arrays of the stages' tiles.  parts > 1
// CTAs share each system's finish (jobs without bbarT and delta only).
void launch_discretise_batch(const DiscJob* jobs, int njobs, const DiscTile* const tiles[3], const long ntiles[3],
                             int sms, cudaStream_t s, int parts = 1);

// Scan-vector initialisation with the forcing term Gamma_k (zero padding
// for k >= T and for the components the solver leaves empty).
void launch_forcing(double* V, int Np, int n, int m, int solver, const double* Bbar, const double* U, long T,
                    long Tp, cudaStream_t s);

// y[(ybase + k)*p + o] = C x_k + D u_k for k < count (x_k = V[k*Np + xoff ..]).
void launch_output(double* Y, const double* V, int Np, int xoff, int n, int m, int p, const double* C,
                   const double* D, int zeroC, int zeroD, const double* U, int ustride, int uoff, long count,
                   long ybase, cudaStream_t s);

// dst[0..N) = src[0..N)
void launch_copy(double* dst, const double* src, long N, cudaStream_t s);

// Kernel launches made by the last call of each launcher (for accounting).
int launches_per_level();

// ---------------------------------------------------------------------------
// Batched forms (many systems per launch).  Every batched kernel takes a
// device array of jobs; blockIdx.y selects the job.
// ---------------------------------------------------------------------------

// Tiling of the level contraction: entries of one grouped launch must share
// the config id (and CW).  Ids 0..4: one CTA owns all Np rows of NC columns
// (Np <= 64 here); ids 5/6: 64 x 64 tiles with cp.async staging (Np > 64;
// 5: K-contiguous source columns, 6: N-contiguous, the power table).
struct LevelConfig {
    int id = 0;     // template configuration
    int CW = 1;     // column warps
    int NC = 0;     // columns per CTA
    size_t smem = 0;
};
// `a` as for launch_affine_level (the down-sweep with cpy set).
LevelConfig level_config(const LevelArgs& a);
// The arguments a grouped launch stores for `a` (tiled: the swapped form of
// the down-sweep, whose swap launch_swap_grouped performs beforehand).
LevelArgs level_grouped_args(const LevelArgs& a);
long level_tiles(const LevelConfig& c, const LevelArgs& stored);

// One level over nent systems: dStart (device, nent entries) holds each
// entry's first CTA; `tiles` CTAs in total; smem = max over entries.
void launch_affine_level_grouped(const LevelConfig& c, const LevelArgs* dArgs, const long* dStart, int nent,
                                 long tiles, size_t smem, cudaStream_t s);
// cpy(g, i) <-> dst(g, i) for every entry (original down-sweep arguments).
void launch_swap_grouped(const LevelArgs* dArgs, int nent, long max_elems, cudaStream_t s);

// Mixed-precision level contraction (3xTF32 tcgen05, FP64 in and out) for
// scan dimensions 72..1024 with K-contiguous sources and no in-place copy,
// or a general rows x K GEMM (M, K set; one source; dst_limit honoured).
// Grouped like launch_affine_level_grouped: dStart[e] = first tile of entry e,
// level_tc_tiles(a) tiles per entry.  A device wait that gives up sets *status.
bool level_tc_supported(const LevelArgs& a);
long level_tc_tiles(const LevelArgs& a);
// dCta: ctas + 1 tile boundaries (level_tc_ranges), one persistent CTA each.
void launch_level_tc(const LevelArgs* dArgs, const long* dStart, int nent, const long* dCta, int ctas, int* status,
                     cudaStream_t s);
std::vector<long> level_tc_ranges(const std::vector<LevelArgs>& ents, int ctas);
// Encodes into out[0..127] (host) the TMA tensor map of a's source columns:
// FP64, inner dimension Np (K), outer dimension ncols at stride src_gs, box
// 16 x 64, zero fill outside.  Throws on failure.
void level_encode_src_map(const LevelArgs& a, void* out);
// Bytes of the pre-split P - R of one level (tiles of 128 rows x 16 K, hi then lo).
size_t level_split_bytes(int Np);
// The same for a general rows x K matrix (LevelArgs M, K; no exact part: rn = -1).
size_t gemm_split_bytes(int rows, int K);
// Pre-split P - R for every entry (a.P, a.rn, a.rsh -> a.Ps); blockIdx.y = entry.
// max_elems: the largest split of an entry, in 8-byte units (sizes the grid).
void launch_level_split(const LevelArgs* dArgs, int nent, long max_elems, cudaStream_t s);

struct SampleJob {
    double* U = nullptr;
    int m = 0, K = 0;
    const double *a = nullptr, *f = nullptr, *phi = nullptr;
    double base = 0, dt = 0;
    long count = 0;
};
struct ForcingJob {
    double* V = nullptr;
    int Np = 0, n = 0, m = 0, solver = 0;
    const double* BbarT = nullptr;  // Bbar transposed: W m rows of n
    const double* U = nullptr;
    long T = 0, Tp = 0;
};
struct OutputJob {
    double* Y = nullptr;
    const double* V = nullptr;
    int Np = 0, xoff = 0, n = 0, m = 0, p = 0;
    const double *CT = nullptr, *DT = nullptr;  // C and D transposed: n (m) rows of p
    int zeroC = 1, zeroD = 1;
    const double* U = nullptr;
    int ustride = 1, uoff = 0;
    long count = 0, ybase = 0;
};
struct CopyJob {
    double* dst = nullptr;
    const double* src = nullptr;  // nullptr: fill with zeros
    long N = 0;
};
// Phi into the power table's level 0 (Np x Np, zero padded) from its compact
// staged form: RK4 the n x n matrix; ABM the last block row (n x 4n), the
// block rows above it being the exact shift (block b reads block b + 1).
struct PhiJob {
    double* dst = nullptr;
    const double* src = nullptr;
    int n = 0, Np = 0, solver = 0;
};
void launch_phi_batch(const PhiJob* dJobs, int njobs, long max_elems, cudaStream_t s);
// max_elems: the largest element count of a job (sizes the x dimension); for
// the samples, runs of 32 samples x channels (one thread each).
// max_terms: the largest term count of the jobs' inputs
void launch_samples_batch(const SampleJob* dJobs, int njobs, long max_elems, int max_terms, cudaStream_t s);
void launch_forcing_batch(const ForcingJob* dJobs, int njobs, long max_elems, cudaStream_t s);
void launch_output_batch(const OutputJob* dJobs, int njobs, long max_elems, cudaStream_t s);
void launch_copy_batch(const CopyJob* dJobs, int njobs, long max_elems, cudaStream_t s);

}  // namespace parode
