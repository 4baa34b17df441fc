/*
 * parode_ext.h -- entry points of libParODEShared.so beyond the reference ABI.
 *
 * These are additive: the reference (apatriciu/ParODE) has no counterpart
 * for the FP64 arrays, precision forms, device residency, batching or the
 * serving queue below, so each comment says which reference behaviour it
 * extends.  All functions are extern "C", take plain pointers and sizes and
 * report errors through nErr[0] (ParODEEnums.h values plus the extra codes
 * below), exactly as the reference ABI does.
 */
#ifndef PARODE_EXT_H_
#define PARODE_EXT_H_

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes beyond ParODEEnums.h (-1..-7). */
#define ParODE_InvalidInput     (-8)  /* uIndex names no registered input               */
#define ParODE_InvalidArgument  (-9)  /* a size, pointer or option value is out of range */
#define ParODE_DeviceError      (-10) /* a CUDA call failed or a device wait gave up     */

/* Precision forms of the scan. */
#define PARODE_PRECISION_FP64   0  /* plain: every sweep, the carry and the outputs in FP64  */
#define PARODE_PRECISION_MIXED  1  /* leaf sweeps in 3xTF32 on tcgen05 with FP32 accumulation;
                                      Phi, the power table, the upper levels and the carry in FP64 */
#define PARODE_PRECISION_TF32   2  /* single pass: the block-response GEMMs in one TF32 product
                                      (operands rounded to TF32, about 2^-11 relative), the carry and
                                      the initial-state part in FP64; other paths run the mixed form
                                      (the plan reports PARODE_PRECISION_MIXED for them).  Single
                                      solves only: a batch or the server runs it as the mixed form. */

/* Options (ParODE_SetOption / ParODE_GetOption). */
#define PARODE_OPT_PRECISION    1  /* PARODE_PRECISION_* used by SimulateODE (default FP64) */
#define PARODE_OPT_PATH         2  /* 0 auto, 1 level-synchronous sweeps, 2 blocked (leaf chosen by cost),
                                      3 blocked with the block-response GEMM leaf (FP64, inputs present),
                                      4 blocked with the in-block sweep leaf, 5 the general scan (the
                                      reference's pipeline: T copies of Phi composed pair by pair,
                                      scan dimensions up to 64) */
#define PARODE_OPT_LOG          3  /* non-zero: one line per solve or batch set-up on stderr; a server logs
                                      each batch's timeline (1), and its set-up phases too (2, which waits on
                                      the device between phases) */
#define PARODE_OPT_EXECUTIONS   4  /* >= 1 (default 1): solves a plan or batch made by ParODE_PlanCreate /
                                      ParODE_BatchCreate is expected to run; the block-response leaf picks
                                      its block size against the FP64 build of its tables spread over that
                                      many solves (SimulateODE and the server always use 1) */
#define PARODE_OPT_POOL_KEEP    7  /* >= 0 bytes (default 0): freed device memory that each selected device's
                                      stream-ordered pool keeps mapped (its release threshold), so that a
                                      later plan or batch of a similar size skips mapping fresh memory; needs
                                      ParODE_Init / InitWithGPUs first (-2 before).  A server sets its own
                                      device's threshold to its HBM budget. */
#define PARODE_OPT_DISCRETISE   8  /* where a batch (or a server's batch) discretises its systems:
                                      PARODE_DISCRETISE_AUTO (default: small batches on the host threads, with
                                      no device round trip; large ones on the device), _HOST or _DEVICE.  Both
                                      sides take every operation in the same order: the same bits. */
#define PARODE_DISCRETISE_AUTO   0
#define PARODE_DISCRETISE_HOST   1
#define PARODE_DISCRETISE_DEVICE 2

/* Test hooks, host side only (nothing faults on the device):
 *   PARODE_OPT_FAULT_ALLOC   k >= 0: the k-th device allocation of a solve,
 *                            batch or server from now on (0 = the next) fails
 *                            as if the device were out of memory; the call
 *                            reports -4 and later calls allocate normally.
 *                            -1 (default) disables it.
 *   PARODE_OPT_FAULT_WITHHOLD non-zero: the mixed-precision response solve's
 *                            tensor-core kernel withholds one arrive of its
 *                            first pipeline stage in its first CTA, so that
 *                            the waits on it give up after their bound (about
 *                            a second); the solve then reports -10
 *                            (DeviceError) and the device stays usable. */
#define PARODE_OPT_FAULT_ALLOC    5
#define PARODE_OPT_FAULT_WITHHOLD 6

void ParODE_SetOption(int option, long long value, int nErr[]);
long long ParODE_GetOption(int option, int nErr[]);

/* Number of outputs SimulateODE produces for (solver, tStart, tEnd, tStep):
 * RK4 floor((tEnd-tStart)/tStep)+1 (reference Sources/RungeKutta4thOrder.cpp:20),
 * ABM that count from tStart+3 tStep, plus 3 (Sources/AdamsMoulton.cpp:356-358).
 * Returns -1 for an empty horizon. */
long long ParODE_NumOutputs(int solver, double tStart, double tEnd, double tStep);

/* Registers the built-in input u_i(t) = sum_k amp[i*K+k] sin(2 pi freq[i*K+k] t + phase[i*K+k])
 * (K = nTerms) and returns its index in the same index space as RegisterInput.
 * Evaluated on the device in FP64 time; the scan kernels can generate it on chip. */
void ParODE_RegisterSinusoidInput(int nInputs, int nTerms, const double* amp, const double* freq,
                                  const double* phase, int uIndex[], int nErr[]);

/* FP64 form of SimulateODE: same arguments and layouts as the C ABI
 * (by value instead of by pointer), FP64 arrays, an explicit precision form,
 * and 64-bit step counts.  tVect may be NULL.  yVect receives
 * nSteps[0] x nOutputs values (time-major). */
void ParODE_SimulateODE_d(const double* A, const double* B, const double* C, const double* D,
                          int nInputs, int nStates, int nOutputs, int ZeroB, int ZeroC, int ZeroD,
                          int uIndex, double tStart, double tEnd, double tStep, const double* x0,
                          int solver, int precision, double* tVect, double* yVect,
                          long long nSteps[], int nErr[]);

/* ---- device-resident plans ------------------------------------------------
 * A plan holds one discretised system on the device (Phi, Bbar, C, D, the
 * initial scan state and every scan buffer), so repeated executions do no
 * host work and no allocation.  PlanCreate performs the host FP64
 * discretisation (and the ABM start-up) and the uploads; PlanExecute only
 * enqueues device work on `stream` (a cudaStream_t; NULL = the library's
 * stream) and returns without synchronising. */
typedef struct ParODE_Plan ParODE_Plan;

ParODE_Plan* ParODE_PlanCreate(const double* A, const double* B, const double* C, const double* D,
                               int nInputs, int nStates, int nOutputs, int ZeroB, int ZeroC, int ZeroD,
                               int uIndex, double tStart, double tEnd, double tStep, const double* x0,
                               int solver, int precision, int nErr[]);
/* Enqueue one solve.  yDev: device buffer of NumOutputs x nOutputs doubles,
 * or NULL to keep the result in the plan. */
void ParODE_PlanExecute(ParODE_Plan* plan, double* yDev, void* stream, int nErr[]);
/* Copy the last result to host memory (synchronises the plan's stream). */
void ParODE_PlanGetOutput(ParODE_Plan* plan, double* tVect, double* yVect, int nErr[]);
long long ParODE_PlanNumOutputs(const ParODE_Plan* plan);
int ParODE_PlanNumOutputChannels(const ParODE_Plan* plan);
/* Device kernel launches one PlanExecute enqueues (for launch accounting). */
int ParODE_PlanLaunchCount(const ParODE_Plan* plan);
/* Precision form the plan actually runs (PARODE_PRECISION_*): the mixed form
 * falls back to FP64 for shapes its tensor-core leaf does not cover, the
 * TF32 form to the mixed form off the block-response path. */
int ParODE_PlanPrecision(const ParODE_Plan* plan);
/* Sweep organisation: 1 level-synchronous, 2 blocked with the in-block sweep
 * leaf, 3 blocked with the block-response GEMM leaf. */
int ParODE_PlanPath(const ParODE_Plan* plan);
/* Response leaf geometry (path 3; zeros otherwise): info[0] block length B,
 * info[1] window columns K, info[2] padded scan dimension NP, info[3] blocks. */
void ParODE_PlanResponseShape(const ParODE_Plan* plan, long long info[4]);
void ParODE_PlanDestroy(ParODE_Plan* plan);
/* Stage timing: when enabled, PlanExecute records CUDA events between its
 * stages on the execution stream.  PlanStageTimes synchronises on the last
 * event and returns the number of stages; ms[i] receives stage i's
 * milliseconds (up to cap) and names its '\n'-separated names. */
void ParODE_PlanSetProfiling(ParODE_Plan* plan, int enable, int nErr[]);
int ParODE_PlanStageTimes(ParODE_Plan* plan, float* ms, int cap, char* names, int names_cap, int nErr[]);

/* ---- time partition of one solve across devices --------------------------
 * The reference splits one solve's horizon over its devices in proportion to
 * their compute units (Sources/RungeKutta4thOrder.cpp:96-125), up-sweeps each
 * device's part, carries the parts' totals across devices on the host and
 * down-sweeps (Sources/GPUFixedStepIterative.cpp:296-337).  Here shard
 * `shard` of `shards` is one plan on one device (one process per GPU):
 *   PlanShardUp    its inputs, block aggregates and the first k levels of
 *                  the chunked carry from a zero state, leaving info[2]
 *                  chunk aggregates of info[3] doubles in dTop (device);
 *   (the caller all-gathers every shard's dTop in shard order: NCCL or any
 *    device copy; equal devices take equal shares of the horizon)
 *   PlanShardDown  the scan of the gathered items seeded with the initial
 *                  state (every shard computes it, it is small), its own
 *                  down-sweep and outputs into yDev (NumOutputs rows: the
 *                  first 3 rows of an ABM solve are its start-up rows on
 *                  shard 0 only, then the shard's steps).
 * Block-response path only (scan dimension <= 64, inputs present).  info:
 * [0] first scan step of the shard, [1] its scan steps, [2] items per shard,
 * [3] doubles per item, [4] shards.  PlanExecute is refused on a shard plan;
 * PlanGetOutput returns the shard's slice of the horizon's time vector. */
ParODE_Plan* ParODE_PlanCreateShard(const double* A, const double* B, const double* C, const double* D,
                                    int nInputs, int nStates, int nOutputs, int ZeroB, int ZeroC, int ZeroD,
                                    int uIndex, double tStart, double tEnd, double tStep, const double* x0,
                                    int solver, int precision, int shard, int shards, int nErr[]);
void ParODE_PlanShardInfo(const ParODE_Plan* plan, long long info[5]);
void ParODE_PlanShardUp(ParODE_Plan* plan, double* dTop, void* stream, int nErr[]);
void ParODE_PlanShardDown(ParODE_Plan* plan, const double* dGathered, double* yDev, void* stream, int nErr[]);

/* ---- batches: many independent systems solved together -----------------
 * One call set-up for nSystems systems (per-system arrays of the
 * SimulateODE_d arguments; B, C, D may be NULL arrays when every system has
 * that matrix absent).  Device-resident afterwards: BatchExecute enqueues all
 * solves on `stream` with a fixed, small number of launches (systems with
 * inputs: the block-response leaf, one grouped GEMM per stage; scan dimension
 * <= 64 otherwise: batched blocked path per padded dimension; larger: one
 * grouped contraction launch per Blelloch level).  BatchCreate returns before
 * the device has finished the set-up it enqueued; BatchExecute on any stream
 * is ordered after it.  The reference has no batch entry point: it solves one
 * system per SimulateODE call (Sources/ParODE.cpp:281-337). */
typedef struct ParODE_Batch ParODE_Batch;
ParODE_Batch* ParODE_BatchCreate(int nSystems, const double* const A[], const double* const B[],
                                 const double* const C[], const double* const D[], const int nInputs[],
                                 const int nStates[], const int nOutputs[], const int ZeroB[], const int ZeroC[],
                                 const int ZeroD[], const int uIndex[], const double tStart[], const double tEnd[],
                                 const double tStep[], const double* const x0[], const int solver[], int precision,
                                 int nErr[]);
void ParODE_BatchExecute(ParODE_Batch* batch, void* stream, int nErr[]);
long long ParODE_BatchNumOutputs(const ParODE_Batch* batch, int i);
int ParODE_BatchNumOutputChannels(const ParODE_Batch* batch, int i);
/* Device pointer to system i's outputs (NumOutputs x channels doubles). */
const double* ParODE_BatchDeviceOutput(const ParODE_Batch* batch, int i);
/* Synchronises and copies system i's time vector and outputs (either may be NULL). */
void ParODE_BatchGetOutput(ParODE_Batch* batch, int i, double* tVect, double* yVect, int nErr[]);
int ParODE_BatchLaunchCount(const ParODE_Batch* batch);
int ParODE_BatchPath(const ParODE_Batch* batch, int i);
int ParODE_BatchPrecision(const ParODE_Batch* batch, int i);
/* Sum over systems of states x outputs: the state*steps of one execute. */
double ParODE_BatchStateSteps(const ParODE_Batch* batch);
void ParODE_BatchDestroy(ParODE_Batch* batch);
/* Create + execute + copy out + destroy; tVect[i] / yVect[i] are host arrays
 * sized for system i (NumOutputs), nSteps[i] receives its output count. */
void ParODE_SimulateODEBatch(int nSystems, const double* const A[], const double* const B[], const double* const C[],
                             const double* const D[], const int nInputs[], const int nStates[], const int nOutputs[],
                             const int ZeroB[], const int ZeroC[], const int ZeroD[], const int uIndex[],
                             const double tStart[], const double tEnd[], const double tStep[],
                             const double* const x0[], const int solver[], int precision, double* const tVect[],
                             double* const yVect[], long long nSteps[], int nErr[]);

/* ---- serving loop: asynchronous solves with continuous batching ---------
 * A scheduler thread admits submitted solves against an HBM budget (bytes;
 * <= 0: 150e9), batches whatever is pending (at most maxBatch systems per
 * batch, maxInflight batches on the device at once) as soon as memory and a
 * slot free up, runs each batch on its own stream so batches overlap, and
 * keeps each finished request's outputs in device memory (counted against
 * the budget) until it is collected.  ServerCreate maps part of the budget
 * (up to 32 GiB, at most half the free memory) into the device's
 * stream-ordered pool up front.  No counterpart in the reference.
 * ServerSubmit returns a request id (> 0) or a negative error code; a request
 * larger than the whole budget fails with -4.  ServerPoll returns 1 when the
 * request is finished (its outputs ready in device memory; output count and
 * channels filled in).  ServerResult copies tVect / yVect (NumOutputs x
 * channels; pinned host memory makes the copy fastest) and the latency
 * (submission to completion, ms), and releases the request and its device
 * memory.  Results that are never collected hold their share of the budget
 * until ServerDestroy.
 * ServerStats fills stats[12]: submitted, completed, failed, p50 ms, p99 ms,
 * mean ms, max ms, state*steps completed, span s (first submission to last
 * completion), peak in-flight bytes, batches, 0. */
typedef struct ParODE_Server ParODE_Server;
ParODE_Server* ParODE_ServerCreate(int precision, double hbmBudgetBytes, int maxBatch, int maxInflight, int nErr[]);
long long ParODE_ServerSubmit(ParODE_Server* srv, const double* A, const double* B, const double* C, const double* D,
                              int nInputs, int nStates, int nOutputs, int ZeroB, int ZeroC, int ZeroD, int uIndex,
                              double tStart, double tEnd, double tStep, const double* x0, int solver, int nErr[]);
int ParODE_ServerPoll(ParODE_Server* srv, long long id, long long nSteps[], int nChannels[], int nErr[]);
void ParODE_ServerResult(ParODE_Server* srv, long long id, double* tVect, double* yVect, double latencyMs[],
                         int nErr[]);
void ParODE_ServerStats(ParODE_Server* srv, double stats[], int nErr[]);
void ParODE_ServerDestroy(ParODE_Server* srv);

/* Affine scan on device data with no allocation (no counterpart in the
 * reference).  With all pointers in device memory of the current device:
 *   dX[k] = x_k for k < count, x_0 = dX0, x_{k+1} = Phi x_k + dGamma[k],
 * Phi ns x ns, dGamma count x ns, dX count x ns, all row-major FP64;
 * dGamma or dX0 may be NULL (zero).  ns in [1, 64].  Enqueued on `stream`
 * (NULL: the legacy default stream); returns after enqueueing.
 * It allocates nothing: its scratch is a static 16 MiB device array.  The
 * array's address is looked up, and the entry point's kernels loaded, once
 * per device by InitializeAllGPUs / InitializeSelectedGPUs (or by the first
 * call on a device when the library was not initialised): with lazy module
 * loading that is when the array's device memory is mapped, so initialise
 * (or make a first call) before reserving the device's memory for your own
 * pool, and before any stream capture.  The address belongs to the device's
 * primary context (not valid after cudaDeviceReset or under another context).
 * A call needs levels*NP^2 + NP + count*NP*(1 + ~1/(B-1))
 * doubles of it (NP = power of two >= max(8, ns)): count <= ~29,000 at
 * ns = 64, ~230,000 at ns = 8; larger calls fail with -4 (NotEnoughResources).
 * The scratch is shared: calls that overlap on the GPU race on it. */
void ParODE_AffineScanDevice(const double* dPhi, const double* dGamma, const double* dX0, int ns,
                             long long count, double* dX, void* stream, int nErr[]);

/* General affine scan over per-step maps on device data: x_0 = dX0 (NULL:
 * zero), x_{k+1} = dM[k] x_k + dV[k] (dV NULL: zero), dX[k] = x_k for
 * k < count; dM count x ns x ns, dV and dX count x ns, row-major FP64, device
 * memory of the current device; ns in [1, 64].  Every pair of every up-sweep
 * level is composed, matrices and vectors, as the reference's MM / MVV scan
 * kernels do (Kernels/MMKernelScanUpsweep.cl:13-56,
 * Kernels/MVVKernelScanUpsweep.cl:14-50, MVVKernelScanDownsweep.cl:14-50), so
 * the maps may differ from step to step (a time-varying system).  precision:
 * PARODE_PRECISION_FP64 (FP64 tensor cores) or PARODE_PRECISION_MIXED (the
 * matrix products in 3xTF32 on tcgen05 for ns in 17..64, the vectors in FP64).
 * Enqueued on `stream` (NULL: the legacy default stream); returns once the
 * scan is done.  Scratch (count rounded up to a power of two, times
 * ns^2 + ns doubles with ns rounded up to 8, 16, 32 or 64) comes from the
 * device's stream-ordered pool. */
void ParODE_AffineScanGeneral(const double* dM, const double* dV, const double* dX0, int ns, long long count,
                              int precision, double* dX, void* stream, int nErr[]);

/* Measured block length of the block-response leaf (no counterpart in the
 * reference, whose batch sizing is a memory formula,
 * Sources/RungeKutta4thOrder.cpp:91-144).  TuneResponseBlock times the
 * candidate block lengths 2^2 .. 2^7 on the current device for a synthetic
 * stable system of the class (solver, states, inputs, outputs, steps,
 * precision), five solves each after two warm-ups, and records the fastest;
 * plans and batches made afterwards for systems of the same class (scan
 * dimension, input and output counts rounded up to powers of two, steps to
 * the power of two above) use it.  log2B[0], msBest[0]: the choice and its
 * median solve time; msModel[0]: the untuned choice's.  Save / Load keep
 * one GPU's entries in a text file (gpuName NULL: the current device's
 * name); InitializeAllGPUs / InitializeSelectedGPUs load the file named by
 * the environment variable PARODE_TUNE_FILE when it is set. */
void ParODE_TuneResponseBlock(int solver, int nStates, int nInputs, int nOutputs, long long nSteps, int precision,
                              int log2B[], float msBest[], float msModel[], int nErr[]);
int ParODE_TuneSave(const char* path, const char* gpuName, int nErr[]);
int ParODE_TuneLoad(const char* path, const char* gpuName, int nErr[]);
void ParODE_TuneClear(void);

#ifdef __cplusplus
}
#endif

#endif /* PARODE_EXT_H_ */
