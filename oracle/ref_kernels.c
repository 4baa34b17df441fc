/* ref_kernels.c -- runs the reference's own OpenCL kernels (the Kernels/ .cl files of
 * apatriciu/ParODE, unmodified) on an OpenCL GPU, launched the way the
 * reference's scan driver launches them, in float.
 *
 * TEST INFRASTRUCTURE ONLY.  Its outputs are golden vectors that pin the CPU
 * oracle (parode_oracle.c) to the reference's own computation; the product
 * library never calls it.  It needs an OpenCL runtime with a GPU device
 * (the Khronos loader libOpenCL.so.1 and a vendor driver, e.g. selected with
 * OCL_ICD_FILENAMES); the kernel sources are staged by oracle/Makefile into
 * oracle/_ref/kernels from the reference tree.
 *
 * What it restates, with the reference file:line it follows:
 *  - the float host set-up (Phi, Bbar, ABM start-up): po_ref_discretise_f32 /
 *    po_ref_abm_startup_f32 of the oracle (Sources/RungeKutta4thOrder.cpp:14-70,
 *    Sources/AdamsMoulton.cpp:29-116,238-316), the start-up inputs from the u
 *    kernel on the device (Sources/AdamsMoulton.cpp:51-88);
 *  - tile and work-group sizes (Sources/RungeKutta4thOrder.cpp:75-89,
 *    Sources/AdamsMoulton.cpp:136-150) and the steps per batch
 *    (Sources/RungeKutta4thOrder.cpp:91-144) from the device's properties,
 *    optionally capped (argument max_batch) to exercise the host carry;
 *  - per batch: DistributeA, u, BTimesU (Sources/RungeKutta4thOrder.cpp:234-288,
 *    Sources/AdamsMoulton.cpp:403-461); the up-sweep with MM / MVV / left-leaf
 *    copies, the host FP32 carry, the down-sweep with MM / MVV / root copies,
 *    SystemOutput and the output gather (Sources/GPUFixedStepIterative.cpp:131-466);
 *  - the time vector's float accumulation (Sources/GPUFixedStepIterative.cpp:141-146).
 *
 * usage: ref_kernels <kernel dir> <case file> <output file>
 * case file (little-endian): int32 magic 0x50524b31, solver, n, m, p, zeroC,
 *   zeroD, max_batch; double t0, tEnd, h; float A[n n], B[n m], C[p n], D[p m],
 *   x0[n] (C / D omitted when flagged absent); int32 len; char ufunc[len].
 * output file: int32 T, q; float tVect[T]; float y[T q] (time-major).
 */
#include "parode_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ---- the OpenCL 1.2 entry points used, declared here (no CL headers) ---- */
typedef int32_t cl_int;
typedef uint32_t cl_uint;
typedef uint64_t cl_ulong;
typedef cl_ulong cl_bitfield;
typedef cl_uint cl_bool;
typedef struct _cl_platform_id* cl_platform_id;
typedef struct _cl_device_id* cl_device_id;
typedef struct _cl_context* cl_context;
typedef struct _cl_command_queue* cl_command_queue;
typedef struct _cl_mem* cl_mem;
typedef struct _cl_program* cl_program;
typedef struct _cl_kernel* cl_kernel;
typedef struct _cl_event* cl_event;
typedef intptr_t cl_context_properties;

#define CL_SUCCESS 0
#define CL_TRUE 1
#define CL_DEVICE_TYPE_GPU (1u << 2)
#define CL_DEVICE_MAX_COMPUTE_UNITS 0x1002
#define CL_DEVICE_MAX_WORK_GROUP_SIZE 0x1004
#define CL_DEVICE_MAX_MEM_ALLOC_SIZE 0x1010
#define CL_DEVICE_GLOBAL_MEM_SIZE 0x101F
#define CL_DEVICE_LOCAL_MEM_SIZE 0x1023
#define CL_DEVICE_NAME 0x102B
#define CL_MEM_READ_WRITE (1u << 0)
#define CL_PROGRAM_BUILD_LOG 0x1183

extern cl_int clGetPlatformIDs(cl_uint, cl_platform_id*, cl_uint*);
extern cl_int clGetDeviceIDs(cl_platform_id, cl_bitfield, cl_uint, cl_device_id*, cl_uint*);
extern cl_int clGetDeviceInfo(cl_device_id, cl_uint, size_t, void*, size_t*);
extern cl_context clCreateContext(const cl_context_properties*, cl_uint, const cl_device_id*,
                                  void (*)(const char*, const void*, size_t, void*), void*, cl_int*);
extern cl_command_queue clCreateCommandQueue(cl_context, cl_device_id, cl_bitfield, cl_int*);
extern cl_mem clCreateBuffer(cl_context, cl_bitfield, size_t, void*, cl_int*);
extern cl_program clCreateProgramWithSource(cl_context, cl_uint, const char**, const size_t*, cl_int*);
extern cl_int clBuildProgram(cl_program, cl_uint, const cl_device_id*, const char*, void (*)(cl_program, void*),
                             void*);
extern cl_int clGetProgramBuildInfo(cl_program, cl_device_id, cl_uint, size_t, void*, size_t*);
extern cl_kernel clCreateKernel(cl_program, const char*, cl_int*);
extern cl_int clSetKernelArg(cl_kernel, cl_uint, size_t, const void*);
extern cl_int clEnqueueNDRangeKernel(cl_command_queue, cl_kernel, cl_uint, const size_t*, const size_t*,
                                     const size_t*, cl_uint, const cl_event*, cl_event*);
extern cl_int clEnqueueReadBuffer(cl_command_queue, cl_mem, cl_bool, size_t, size_t, void*, cl_uint,
                                  const cl_event*, cl_event*);
extern cl_int clEnqueueWriteBuffer(cl_command_queue, cl_mem, cl_bool, size_t, size_t, const void*, cl_uint,
                                   const cl_event*, cl_event*);
extern cl_int clFinish(cl_command_queue);
extern cl_int clReleaseMemObject(cl_mem);
extern cl_int clReleaseKernel(cl_kernel);
extern cl_int clReleaseProgram(cl_program);
extern cl_int clReleaseCommandQueue(cl_command_queue);
extern cl_int clReleaseContext(cl_context);

/* ---- helpers ---- */

static void die(const char* what, int code)
{
    fprintf(stderr, "ref_kernels: %s (%d)\n", what, code);
    exit(2);
}

#define CK(call)                                   \
    do {                                           \
        cl_int rc_ = (call);                       \
        if (rc_ != CL_SUCCESS) die(#call, rc_);    \
    } while (0)

static char* read_file(const char* path, size_t* len)
{
    FILE* f = fopen(path, "rb");
    if (!f) die(path, -1);
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    char* b = (char*)malloc((size_t)n + 1);
    if (!b || fread(b, 1, (size_t)n, f) != (size_t)n) die("read", -1);
    b[n] = 0;
    fclose(f);
    if (len) *len = (size_t)n;
    return b;
}

typedef struct {
    cl_device_id dev;
    cl_context ctx;
    cl_command_queue q;
    char incl[4096];
    const char* dir;
} Cl;

/* Builds `src` with " -I <dir>" (the reference's options,
 * Sources/GPUManagement.cpp:699-706) and returns kernel `name`. */
static cl_kernel build(Cl* c, const char* src, const char* name, cl_program* prog)
{
    cl_int rc;
    size_t len = strlen(src);
    cl_program p = clCreateProgramWithSource(c->ctx, 1, &src, &len, &rc);
    if (rc != CL_SUCCESS) die("clCreateProgramWithSource", rc);
    rc = clBuildProgram(p, 1, &c->dev, c->incl, NULL, NULL);
    if (rc != CL_SUCCESS) {
        char log[16384];
        size_t got = 0;
        clGetProgramBuildInfo(p, c->dev, CL_PROGRAM_BUILD_LOG, sizeof log - 1, log, &got);
        log[got < sizeof log ? got : sizeof log - 1] = 0;
        fprintf(stderr, "build log of %s:\n%s\n", name, log);
        die("clBuildProgram", rc);
    }
    cl_kernel k = clCreateKernel(p, name, &rc);
    if (rc != CL_SUCCESS) die(name, rc);
    *prog = p;
    return k;
}

static cl_kernel build_file(Cl* c, const char* file, const char* name, cl_program* prog)
{
    char path[4096];
    snprintf(path, sizeof path, "%s/%s", c->dir, file);
    char* src = read_file(path, NULL);
    cl_kernel k = build(c, src, name, prog);
    free(src);
    return k;
}

static cl_mem buffer(Cl* c, size_t bytes)
{
    cl_int rc;
    cl_mem b = clCreateBuffer(c->ctx, CL_MEM_READ_WRITE, bytes > 0 ? bytes : 1, NULL, &rc);
    if (rc != CL_SUCCESS) die("clCreateBuffer", rc);
    return b;
}

static void arg_mem(cl_kernel k, cl_uint i, cl_mem m) { CK(clSetKernelArg(k, i, sizeof(cl_mem), &m)); }
static void arg_int(cl_kernel k, cl_uint i, int v) { CK(clSetKernelArg(k, i, sizeof(int), &v)); }
static void arg_uint(cl_kernel k, cl_uint i, unsigned v) { CK(clSetKernelArg(k, i, sizeof(unsigned), &v)); }
static void arg_float(cl_kernel k, cl_uint i, float v) { CK(clSetKernelArg(k, i, sizeof(float), &v)); }
static void arg_local(cl_kernel k, cl_uint i, size_t bytes) { CK(clSetKernelArg(k, i, bytes, NULL)); }

static void launch(Cl* c, cl_kernel k, int dims, size_t g0, size_t g1, size_t l0, size_t l1)
{
    size_t g[2] = {g0, g1}, l[2] = {l0, l1};
    CK(clEnqueueNDRangeKernel(c->q, k, (cl_uint)dims, NULL, g, l, 0, NULL, NULL));
}

static void write_buf(Cl* c, cl_mem b, size_t off, size_t bytes, const void* src)
{
    CK(clEnqueueWriteBuffer(c->q, b, CL_TRUE, off, bytes, src, 0, NULL, NULL));
}

static void read_buf(Cl* c, cl_mem b, size_t off, size_t bytes, void* dst)
{
    CK(clEnqueueReadBuffer(c->q, b, CL_TRUE, off, bytes, dst, 0, NULL, NULL));
}

/* u kernel launch (Sources/RungeKutta4thOrder.cpp:255-270): local (m, l1)
 * with l1 the first value reaching the sample count or m l1 >= 32. */
static void launch_u(Cl* c, cl_kernel ku, cl_mem U, float ts, float dt, int count, int m)
{
    arg_mem(ku, 0, U);
    arg_float(ku, 1, ts);
    arg_float(ku, 2, dt);
    arg_int(ku, 3, count);
    size_t l1 = 1;
    while (l1 < (size_t)count && l1 * (size_t)m < 32) ++l1;
    size_t blocks = ((size_t)count - 1) / l1 + 1;
    launch(c, ku, 2, blocks * (size_t)m, l1, (size_t)m, l1);
}

static long pow2_at_least(long v)
{
    long p = 1;
    while (p < v) p <<= 1;
    return p;
}

int main(int argc, char** argv)
{
    if (argc != 4) {
        fprintf(stderr, "usage: ref_kernels <kernel dir> <case file> <output file>\n");
        return 1;
    }
    /* ---- case ---- */
    size_t clen = 0;
    char* cs = read_file(argv[2], &clen);
    const char* cur = cs;
#define TAKE(ptr, bytes) (memcpy((ptr), cur, (bytes)), cur += (bytes))
    int32_t hdr[8];
    TAKE(hdr, sizeof hdr);
    if (hdr[0] != 0x50524b31) die("bad case file", hdr[0]);
    const int solver = hdr[1], n = hdr[2], m = hdr[3], pin = hdr[4], zeroC = hdr[5], zeroD = hdr[6];
    const long max_batch = hdr[7];
    double tt[3];
    TAKE(tt, sizeof tt);
    double t0 = tt[0];
    const double tEnd = tt[1], h = tt[2];
    if (n <= 0 || m <= 0 || (solver != 0 && solver != 1)) die("unsupported case (needs n > 0, inputs)", n);
    float* Af = (float*)malloc(sizeof(float) * (size_t)n * n);
    float* Bf = (float*)malloc(sizeof(float) * (size_t)n * m);
    float* Cf = (float*)calloc((size_t)(pin > 0 ? pin : 1) * n, sizeof(float));
    float* Df = (float*)calloc((size_t)(pin > 0 ? pin : 1) * m, sizeof(float));
    float* x0f = (float*)malloc(sizeof(float) * (size_t)n);
    TAKE(Af, sizeof(float) * (size_t)n * n);
    TAKE(Bf, sizeof(float) * (size_t)n * m);
    if (!zeroC) TAKE(Cf, sizeof(float) * (size_t)pin * n);
    if (!zeroD) TAKE(Df, sizeof(float) * (size_t)pin * m);
    TAKE(x0f, sizeof(float) * (size_t)n);
    int32_t ulen = 0;
    TAKE(&ulen, sizeof ulen);
    char* ufunc = (char*)malloc((size_t)ulen + 1);
    TAKE(ufunc, (size_t)ulen);
    ufunc[ulen] = 0;
    if ((size_t)(cur - cs) != clen) die("case file size", (int)(cur - cs));
#undef TAKE

    /* the oracle's system view of the float matrices (its float copies are exact) */
    double* Ad = (double*)malloc(sizeof(double) * (size_t)n * n);
    double* Bd = (double*)malloc(sizeof(double) * (size_t)n * m);
    double* Cd = (double*)malloc(sizeof(double) * (size_t)(pin > 0 ? pin : 1) * n);
    double* Dd = (double*)malloc(sizeof(double) * (size_t)(pin > 0 ? pin : 1) * m);
    double* x0d = (double*)malloc(sizeof(double) * (size_t)n);
    for (long i = 0; i < (long)n * n; ++i) Ad[i] = Af[i];
    for (long i = 0; i < (long)n * m; ++i) Bd[i] = Bf[i];
    for (long i = 0; i < (long)(pin > 0 ? pin : 1) * n; ++i) Cd[i] = Cf[i];
    for (long i = 0; i < (long)(pin > 0 ? pin : 1) * m; ++i) Dd[i] = Df[i];
    for (int i = 0; i < n; ++i) x0d[i] = x0f[i];
    po_system sys = {n, m, pin, 0, zeroC, zeroD, Ad, Bd, Cd, Dd, x0d};
    const int p = (zeroC && zeroD) ? n : pin;     /* Sources/GPUFixedStepIterative.cpp:58-125 */
    const int N = solver == 0 ? n : 4 * n;         /* scan dimension */
    const int W = solver == 0 ? 3 : 5;

    /* ---- OpenCL device ---- */
    Cl c;
    memset(&c, 0, sizeof c);
    c.dir = argv[1];
    snprintf(c.incl, sizeof c.incl, " -I %s", argv[1]);
    cl_platform_id plats[16];
    cl_uint np = 0;
    CK(clGetPlatformIDs(16, plats, &np));
    int found = 0;
    for (cl_uint i = 0; i < np && !found; ++i) {
        cl_uint nd = 0;
        if (clGetDeviceIDs(plats[i], CL_DEVICE_TYPE_GPU, 1, &c.dev, &nd) == CL_SUCCESS && nd > 0) found = 1;
    }
    if (!found) die("no OpenCL GPU device", 0);
    char dname[256] = {0};
    cl_uint cus = 0;
    size_t maxwg = 0;
    cl_ulong gmem = 0, maxalloc = 0, lmem = 0;
    CK(clGetDeviceInfo(c.dev, CL_DEVICE_NAME, sizeof dname - 1, dname, NULL));
    CK(clGetDeviceInfo(c.dev, CL_DEVICE_MAX_COMPUTE_UNITS, sizeof cus, &cus, NULL));
    CK(clGetDeviceInfo(c.dev, CL_DEVICE_MAX_WORK_GROUP_SIZE, sizeof maxwg, &maxwg, NULL));
    CK(clGetDeviceInfo(c.dev, CL_DEVICE_GLOBAL_MEM_SIZE, sizeof gmem, &gmem, NULL));
    CK(clGetDeviceInfo(c.dev, CL_DEVICE_MAX_MEM_ALLOC_SIZE, sizeof maxalloc, &maxalloc, NULL));
    CK(clGetDeviceInfo(c.dev, CL_DEVICE_LOCAL_MEM_SIZE, sizeof lmem, &lmem, NULL));
    cl_int rc;
    c.ctx = clCreateContext(NULL, 1, &c.dev, NULL, NULL, &rc);
    if (rc != CL_SUCCESS) die("clCreateContext", rc);
    c.q = clCreateCommandQueue(c.ctx, c.dev, 0, &rc);
    if (rc != CL_SUCCESS) die("clCreateCommandQueue", rc);

    /* ---- kernels: one program per file, the u program as the reference
     * assembles it (Sources/ParODE.cpp:410-466) ---- */
    cl_program pr[10];
    cl_kernel kDist = build_file(&c, "DistributeA.cl", "DistributeA", &pr[0]);
    cl_kernel kMMup = build_file(&c, "MMKernelScanUpsweep.cl", "MatrixMatrixMultiplicationKernelScanUpsweep", &pr[1]);
    cl_kernel kMVVup =
        build_file(&c, "MVVKernelScanUpsweep.cl", "MatrixTimesVectorPlusVectorKernelScanUpsweep", &pr[2]);
    cl_kernel kLeft = build_file(&c, "LeftLeafCopyKernelScanUpsweep.cl", "LeftLeafCopyKernelScanUpsweep", &pr[3]);
    cl_kernel kMMdn =
        build_file(&c, "MMKernelScanDownsweep.cl", "MatrixMatrixMultiplicationKernelScanDownsweep", &pr[4]);
    cl_kernel kMVVdn =
        build_file(&c, "MVVKernelScanDownsweep.cl", "MatrixTimesVectorPlusVectorKernelScanDownsweep", &pr[5]);
    cl_kernel kRoot = build_file(&c, "RootCopyKernelScanDownsweep.cl", "RootCopyKernelScanDownsweep", &pr[6]);
    cl_kernel kOut = build_file(&c, "SystemOutput.cl", "SystemOutputKernel", &pr[7]);
    cl_kernel kBU = solver == 0 ? build_file(&c, "BTimesURK4thOrder.cl", "BTimesURK4thOrder", &pr[8])
                                : build_file(&c, "BTimesUAdamsMoulton.cl", "BTimesUAdamsMoulton", &pr[8]);
    cl_kernel ku;
    {
        char path[4096];
        snprintf(path, sizeof path, "%s/u.cl", c.dir);
        char* ucl = read_file(path, NULL);
        size_t len = strlen("#include <FTypeDef.h>\n") + strlen(ufunc) + strlen(ucl) + 1;
        char* src = (char*)malloc(len);
        snprintf(src, len, "#include <FTypeDef.h>\n%s%s", ufunc, ucl);
        ku = build(&c, src, "u", &pr[9]);
        free(src);
        free(ucl);
    }

    /* ---- sizes (Sources/RungeKutta4thOrder.cpp:75-144, Sources/AdamsMoulton.cpp:136-206) ---- */
    size_t TS = N < 8 ? 4 : (N < 16 ? 8 : 16);
    if ((double)(2 * TS * TS * sizeof(float)) > 0.66 * (double)lmem) TS >>= 1;
    size_t colw = 1;
    while (colw < (size_t)(solver == 0 ? 3 * m : N)) colw <<= 1;
    size_t roww = maxwg / colw < (size_t)N ? maxwg / colw : (size_t)N;
    if ((double)(colw * roww * sizeof(float)) > 0.3 * (double)lmem) roww >>= 1;
    long nTotal, nSteps;
    float* tVect;
    float* Y;  /* nTotal x p, time-major */
    float X0[4 * 1024];
    if (N > 4 * 1024) die("scan dimension too large for the harness", N);
    float* U9 = NULL;
    long pre = 0;
    if (solver == 1) {
        /* start-up inputs u(t0 + j h/2), j = 0..8, by the u kernel (Sources/AdamsMoulton.cpp:51-88) */
        cl_mem U = buffer(&c, sizeof(float) * 9 * (size_t)m);
        launch_u(&c, ku, U, (float)t0, (float)(h / 2.0), 9, m);
        U9 = (float*)malloc(sizeof(float) * 9 * (size_t)m);
        read_buf(&c, U, 0, sizeof(float) * 9 * (size_t)m, U9);
        clReleaseMemObject(U);
        pre = 3;
        t0 += 3 * h; /* Sources/AdamsMoulton.cpp:356 */
    }
    nSteps = (long)((unsigned long)((tEnd - t0) / h) + 1);
    nTotal = nSteps + pre;
    tVect = (float*)malloc(sizeof(float) * (size_t)nTotal);
    Y = (float*)calloc((size_t)nTotal * p, sizeof(float));
    {
        /* Sources/GPUFixedStepIterative.cpp:141-146 (tStart here is the shifted t0) */
        for (long i = 0; i < pre; ++i) tVect[i] = (float)(t0 - (double)(pre - i) * h);
        tVect[pre] = (float)t0;
        for (long i = 1; i < nSteps; ++i) tVect[pre + i] = (float)((double)tVect[pre + i - 1] + h);
    }
    float* Phi = (float*)calloc((size_t)N * N, sizeof(float));
    float* Bb = (float*)calloc((size_t)n * W * m, sizeof(float));
    po_ref_discretise_f32(&sys, solver, h, Phi, Bb);
    if (solver == 0) {
        for (int r = 0; r < n; ++r) X0[r] = x0f[r];
    } else {
        float ypre[3 * 1024];
        if (p > 1024) die("too many outputs", p);
        po_ref_abm_startup_f32(&sys, h, U9, X0, ypre);
        memcpy(Y, ypre, sizeof(float) * 3 * (size_t)p);
    }
    /* steps per batch (one device): Sources/RungeKutta4thOrder.cpp:91-144 */
    long NSB;
    {
        unsigned long perStep = 2UL * ((unsigned long)N * N + N) * sizeof(float);
        unsigned long matStep = (unsigned long)N * N * sizeof(float);
        unsigned long gm = (unsigned long)(0.8 * (double)gmem), ma = (unsigned long)(0.8 * (double)maxalloc);
        unsigned long maxE = gm / perStep < ma / matStep ? gm / perStep : ma / matStep;
        double ratio = (double)(maxE / cus);
        long e = 1;
        while ((unsigned long)e < maxE && (double)e / (double)cus < ratio) e <<= 1;
        e >>= 1;
        if (e > nSteps) {
            long sum = e;
            while (sum >= nSteps) {
                e >>= 1;
                sum = e;
            }
            e <<= 1;
        }
        NSB = e;
        if (max_batch > 0 && NSB > max_batch) NSB = max_batch; /* a smaller device's batches */
        if (NSB <= 0) die("steps per batch", (int)NSB);
    }
    if ((double)N * N * NSB * sizeof(float) > 24e9) die("matrix buffers above 24 GB", (int)NSB);
    fprintf(stderr, "ref_kernels: %s, %u CUs; solver %d n %d m %d p %d N %d steps %ld per batch %ld; TS %zu MVV %zux%zu\n",
            dname, cus, solver, n, m, p, N, nSteps, NSB, TS, colw, roww);

    /* ---- buffers ---- */
    cl_mem Mb[2], Vb[2];
    for (int k = 0; k < 2; ++k) {
        Mb[k] = buffer(&c, sizeof(float) * (size_t)N * N * NSB);
        Vb[k] = buffer(&c, sizeof(float) * (size_t)N * NSB);
    }
    cl_mem ABar = buffer(&c, sizeof(float) * (size_t)N * N);
    cl_mem BBar = buffer(&c, sizeof(float) * (size_t)n * W * m);
    const size_t ucount = solver == 0 ? (size_t)(2 * NSB + 1) : (size_t)(NSB + 4);
    cl_mem Ub = buffer(&c, sizeof(float) * ucount * m);
    cl_mem Cb = buffer(&c, sizeof(float) * (size_t)(zeroC ? 1 : pin * n));
    cl_mem Db = buffer(&c, sizeof(float) * (size_t)(zeroD ? 1 : pin * m));
    cl_mem Yb = buffer(&c, sizeof(float) * (size_t)p * NSB);
    write_buf(&c, ABar, 0, sizeof(float) * (size_t)N * N, Phi);
    write_buf(&c, BBar, 0, sizeof(float) * (size_t)n * W * m, Bb);
    if (!zeroC) write_buf(&c, Cb, 0, sizeof(float) * (size_t)pin * n, Cf);
    if (!zeroD) write_buf(&c, Db, 0, sizeof(float) * (size_t)pin * m, Df);
    float* zeros = (float*)calloc((size_t)N * NSB, sizeof(float));

    /* accumulators (Sources/GPUFixedStepIterative.cpp:191-198) */
    float* accM = (float*)calloc((size_t)N * N, sizeof(float));
    float* accV = (float*)calloc((size_t)N, sizeof(float));
    float* bufM = (float*)malloc(sizeof(float) * (size_t)N * N);
    float* bufV = (float*)malloc(sizeof(float) * (size_t)N);
    float* tmpM = (float*)malloc(sizeof(float) * (size_t)N * N);
    float* tmpV = (float*)malloc(sizeof(float) * (size_t)N);
    for (int i = 0; i < N; ++i) {
        accV[i] = X0[i];
        accM[(long)i * N + i] = 1.0f;
    }
    const size_t stride_y = (zeroC && zeroD) ? (size_t)N : (size_t)p;
    float* outb = (float*)malloc(sizeof(float) * stride_y * NSB);
    long gidx = pre;
    const long nBatches = (nSteps - 1) / NSB + 1;
    for (long nB = 0; nB < nBatches; ++nB) {
        long steps = NSB;
        if (nB == nBatches - 1) steps = pow2_at_least(nSteps - nB * NSB);
        int src = 0, dst = 1;
        const double tsb = t0 + (double)(nB * NSB) * h;
        /* InitializeBatchData */
        arg_mem(kDist, 0, ABar);
        arg_mem(kDist, 1, Mb[src]);
        arg_int(kDist, 2, N * N);
        launch(&c, kDist, 1, TS * (size_t)steps, 0, TS, 0);
        if (solver == 0) {
            launch_u(&c, ku, Ub, (float)tsb, (float)(h / 2.0), (int)(2 * steps + 1), m);
            arg_mem(kBU, 0, BBar);
            arg_mem(kBU, 1, Ub);
            arg_mem(kBU, 2, Vb[src]);
            arg_uint(kBU, 3, (unsigned)N);
            arg_uint(kBU, 4, (unsigned)m);
            arg_local(kBU, 5, colw * roww * sizeof(float));
        } else {
            write_buf(&c, Vb[src], 0, sizeof(float) * (size_t)N * NSB, zeros);
            launch_u(&c, ku, Ub, (float)(tsb - 3 * h), (float)h, (int)(steps + 4), m);
            arg_mem(kBU, 0, BBar);
            arg_mem(kBU, 1, Ub);
            arg_mem(kBU, 2, Vb[src]);
            arg_uint(kBU, 3, (unsigned)n);
            arg_uint(kBU, 4, (unsigned)(5 * m));
            arg_uint(kBU, 5, (unsigned)m);
            arg_local(kBU, 6, colw * roww * sizeof(float));
        }
        launch(&c, kBU, 2, (size_t)steps * colw, roww, colw, roww);
        CK(clFinish(c.q));
        /* up-sweep */
        const size_t cpyM = (size_t)N * N < maxwg ? (size_t)N * N : maxwg;
        for (long d = 1; d < NSB; d <<= 1) {
            if (d >= steps) continue;
            const size_t groups = (size_t)(steps / (2 * d));
            arg_mem(kMMup, 0, Mb[src]);
            arg_mem(kMMup, 1, Mb[dst]);
            arg_int(kMMup, 2, (int)d);
            arg_int(kMMup, 3, N);
            arg_local(kMMup, 4, TS * TS * sizeof(float));
            arg_local(kMMup, 5, TS * TS * sizeof(float));
            launch(&c, kMMup, 2, TS * groups, TS, TS, TS);
            arg_mem(kMVVup, 0, Mb[src]);
            arg_mem(kMVVup, 1, Vb[src]);
            arg_mem(kMVVup, 2, Vb[dst]);
            arg_int(kMVVup, 3, (int)d);
            arg_int(kMVVup, 4, N);
            arg_local(kMVVup, 5, colw * roww * sizeof(float));
            launch(&c, kMVVup, 2, colw * groups, roww, colw, roww);
            arg_mem(kLeft, 0, Mb[src]);
            arg_mem(kLeft, 1, Mb[dst]);
            arg_int(kLeft, 2, (int)d);
            arg_int(kLeft, 3, N * N);
            launch(&c, kLeft, 1, cpyM * groups, 0, cpyM, 0);
            arg_mem(kLeft, 0, Vb[src]);
            arg_mem(kLeft, 1, Vb[dst]);
            arg_int(kLeft, 2, (int)d);
            arg_int(kLeft, 3, N);
            launch(&c, kLeft, 1, TS * groups, 0, TS, 0);
            CK(clFinish(c.q));
            src = dst;
            dst = (src + 1) % 2;
        }
        /* host carry (Sources/GPUFixedStepIterative.cpp:296-337) */
        read_buf(&c, Mb[src], sizeof(float) * (size_t)N * N * (steps - 1), sizeof(float) * (size_t)N * N, bufM);
        read_buf(&c, Vb[src], sizeof(float) * (size_t)N * (steps - 1), sizeof(float) * (size_t)N, bufV);
        memcpy(tmpM, accM, sizeof(float) * (size_t)N * N);
        memcpy(tmpV, accV, sizeof(float) * (size_t)N);
        for (int r = 0; r < N; ++r)
            for (int col = 0; col < N; ++col) {
                float s = 0.0f;
                for (int k = 0; k < N; ++k) s += bufM[(long)r * N + k] * tmpM[(long)k * N + col];
                accM[(long)r * N + col] = s;
            }
        for (int r = 0; r < N; ++r) {
            float s = 0.0f;
            for (int col = 0; col < N; ++col) s += bufM[(long)r * N + col] * tmpV[col];
            accV[r] = s + bufV[r];
        }
        write_buf(&c, Mb[src], sizeof(float) * (size_t)N * N * (steps - 1), sizeof(float) * (size_t)N * N, tmpM);
        write_buf(&c, Vb[src], sizeof(float) * (size_t)N * (steps - 1), sizeof(float) * (size_t)N, tmpV);
        /* down-sweep */
        for (long d = NSB / 2; d > 0; d >>= 1) {
            if (d >= steps) continue;
            const size_t groups = (size_t)(steps / (2 * d));
            arg_mem(kMMdn, 0, Mb[src]);
            arg_mem(kMMdn, 1, Mb[dst]);
            arg_int(kMMdn, 2, (int)d);
            arg_int(kMMdn, 3, N);
            arg_local(kMMdn, 4, TS * TS * sizeof(float));
            arg_local(kMMdn, 5, TS * TS * sizeof(float));
            launch(&c, kMMdn, 2, TS * groups, TS, TS, TS);
            arg_mem(kMVVdn, 0, Mb[src]);
            arg_mem(kMVVdn, 1, Vb[src]);
            arg_mem(kMVVdn, 2, Vb[dst]);
            arg_int(kMVVdn, 3, (int)d);
            arg_int(kMVVdn, 4, N);
            arg_local(kMVVdn, 5, colw * roww * sizeof(float));
            launch(&c, kMVVdn, 2, colw * groups, roww, colw, roww);
            arg_mem(kRoot, 0, Mb[src]);
            arg_mem(kRoot, 1, Mb[dst]);
            arg_int(kRoot, 2, (int)d);
            arg_int(kRoot, 3, N * N);
            launch(&c, kRoot, 1, cpyM * groups, 0, cpyM, 0);
            arg_mem(kRoot, 0, Vb[src]);
            arg_mem(kRoot, 1, Vb[dst]);
            arg_int(kRoot, 2, (int)d);
            arg_int(kRoot, 3, N);
            launch(&c, kRoot, 1, TS * groups, 0, TS, 0);
            CK(clFinish(c.q));
            src = dst;
            dst = (src + 1) % 2;
        }
        /* outputs (Sources/GPUFixedStepIterative.cpp:401-446) */
        if (zeroC && zeroD) {
            read_buf(&c, Vb[src], 0, sizeof(float) * (size_t)N * steps, outb);
        } else {
            const int strideX = solver == 0 ? 1 : 4, offX = solver == 0 ? 0 : 3;
            const int strideU = solver == 0 ? 2 : 1, offU = solver == 0 ? 0 : 3;
            arg_mem(kOut, 0, Cb);
            arg_mem(kOut, 1, Db);
            arg_mem(kOut, 2, Vb[src]);
            arg_mem(kOut, 3, Ub);
            arg_mem(kOut, 4, Yb);
            arg_int(kOut, 5, strideX);
            arg_int(kOut, 6, offX);
            arg_int(kOut, 7, strideU);
            arg_int(kOut, 8, offU);
            arg_int(kOut, 9, n);
            arg_int(kOut, 10, m);
            arg_int(kOut, 11, p);
            arg_int(kOut, 12, zeroC);
            arg_int(kOut, 13, zeroD);
            arg_local(kOut, 14, colw * roww * sizeof(float));
            launch(&c, kOut, 2, (size_t)steps * colw, roww, colw, roww);
            CK(clFinish(c.q));
            read_buf(&c, Yb, 0, sizeof(float) * (size_t)p * steps, outb);
        }
        for (long ii = 0; ii < steps; ++ii)
            if (gidx + ii < nTotal)
                for (int jj = 0; jj < p; ++jj) Y[(gidx + ii) * p + jj] = outb[(ii + 1) * stride_y - p + jj];
        gidx += steps;
    }

    FILE* fo = fopen(argv[3], "wb");
    if (!fo) die(argv[3], -1);
    int32_t sh[2] = {(int32_t)nTotal, (int32_t)p};
    fwrite(sh, sizeof sh, 1, fo);
    fwrite(tVect, sizeof(float), (size_t)nTotal, fo);
    fwrite(Y, sizeof(float), (size_t)nTotal * p, fo);
    fclose(fo);

    for (int k = 0; k < 2; ++k) {
        clReleaseMemObject(Mb[k]);
        clReleaseMemObject(Vb[k]);
    }
    clReleaseMemObject(ABar);
    clReleaseMemObject(BBar);
    clReleaseMemObject(Ub);
    clReleaseMemObject(Cb);
    clReleaseMemObject(Db);
    clReleaseMemObject(Yb);
    cl_kernel ks[10] = {kDist, kMMup, kMVVup, kLeft, kMMdn, kMVVdn, kRoot, kOut, kBU, ku};
    for (int i = 0; i < 10; ++i) {
        clReleaseKernel(ks[i]);
        clReleaseProgram(pr[i]);
    }
    clReleaseCommandQueue(c.q);
    clReleaseContext(c.ctx);
    return 0;
}
