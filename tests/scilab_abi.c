/* scilab_abi.c -- replays the argument layout of the reference's Scilab stub
 * for SimulateODE (SciLabInterface/ParODEInterfaceStubs.sci:84-135) against
 * libParODEShared.so, with no Scilab: a test program of tests/test_scilab_abi.py.
 *
 * Scilab keeps matrices column-major; the stub transposes A, B, C, D before
 * the call (ALocal = A.' ...) so that the library reads them row-major, asks
 * for tEnd = tStart + (nSteps - 1) tStep + 1e-4 tStep, derives the flags and
 * sizes from the matrix shapes, and receives xVect as an nOutputs x nSteps
 * column-major matrix (element (o, k) at o + nOutputs k, which is the
 * library's time-major xVect[k * nOutputs + o]).  The input is the stub
 * tests' u(t) = t for both channels (SciLabInterface/TestRK4.sce:63-74),
 * registered through RegisterInput.  tStart, tEnd and tStep are passed as the
 * C ABI declares them (double *).
 *
 * Built as C with -DC_INCLUDE, the reference's switch for C callers of its
 * header (PythonInterface/ParODESetup.py:3-11).
 *
 * usage: scilab_abi <solver> <case>   case 0: the Scilab tests' system
 * (A = -2 I, B = C = D = I, x0 = [1, -1]); case 1: a non-symmetric system
 * (A = [-2 1; 0.5 -3], B = [1 2; 0 1], C = [1 0; 0.5 1], D = [0.1 0; 0 0.2]),
 * where a missing transpose would show.  Prints nSteps, nErr, then one line
 * per step: t and the outputs.
 */
#include "ParODECInterface.h"

#include <stdio.h>
#include <stdlib.h>

/* A Scilab matrix: column-major storage of an r x c matrix. */
typedef struct {
    int r, c;
    float v[16];
} SciMat;

static float at(const SciMat* m, int i, int j) { return m->v[i + m->r * j]; }

/* The stub's A.' : a column-major matrix whose storage is the row-major
 * order of the original. */
static void transpose_for_call(const SciMat* m, float* out)
{
    for (int i = 0; i < m->r; ++i)
        for (int j = 0; j < m->c; ++j) out[i * m->c + j] = at(m, i, j);
}

int main(int argc, char** argv)
{
    int solver = argc > 1 ? atoi(argv[1]) : 0;
    int which = argc > 2 ? atoi(argv[2]) : 0;
    SciMat A, B, C, D;
    float x0[2];
    if (which == 0) {
        SciMat a = {2, 2, {-2, 0, 0, -2}}, id = {2, 2, {1, 0, 0, 1}};
        A = a;
        B = C = D = id;
        x0[0] = 1.0f;
        x0[1] = -1.0f;
    } else {
        /* column-major storage of [-2 1; 0.5 -3], [1 2; 0 1], [1 0; 0.5 1], [0.1 0; 0 0.2] */
        SciMat a = {2, 2, {-2, 0.5f, 1, -3}}, b = {2, 2, {1, 0, 2, 1}}, c = {2, 2, {1, 0.5f, 0, 1}},
               d = {2, 2, {0.1f, 0, 0, 0.2f}};
        A = a;
        B = b;
        C = c;
        D = d;
        x0[0] = 0.5f;
        x0[1] = 2.0f;
    }
    int err[1] = {0};
    InitializeAllGPUs((char*)"", (char*)"", err);
    if (err[0] != 0) {
        printf("init %d\n", err[0]);
        return 3;
    }
    char ufunc[] = "fType UFunc(fType t, int nInputIndex){\nfType fVal = nInputIndex == 0 ? t :\n"
                   "nInputIndex == 1 ? t :\n0.0;\nreturn fVal;\n}\n";
    int uIndex[1] = {-1};
    RegisterInput(ufunc, uIndex, err);
    if (err[0] != 0) {
        printf("register %d\n", err[0]);
        return 3;
    }
    /* SciLabInterface/ParODEInterfaceStubs.sci:84-135 */
    const int nSteps = 50;
    double tStart = 0.0, tStep = 0.1;
    double tEnd = tStart + (nSteps - 1) * tStep + 0.0001 * tStep;
    float Al[4], Bl[4], Cl[4], Dl[4];
    transpose_for_call(&A, Al);
    transpose_for_call(&B, Bl);
    transpose_for_call(&C, Cl);
    transpose_for_call(&D, Dl);
    int nStates = A.r, nInputs = B.c;
    int ZeroB = B.r == 0, ZeroC = C.r == 0, ZeroD = D.r == 0;
    int nOutputs = C.r != 0 ? C.r : (D.r != 0 ? D.r : nStates);
    float* tVect = (float*)calloc((size_t)nSteps, sizeof(float));
    float* xVect = (float*)calloc((size_t)nSteps * nOutputs, sizeof(float)); /* [nOutputs, nSteps] column-major */
    int nStepsLocal[1] = {0};
    SimulateODE(Al, Bl, Cl, Dl, &nInputs, &nStates, &nOutputs, &ZeroB, &ZeroC, &ZeroD, uIndex, &tStart, &tEnd,
                &tStep, x0, &solver, tVect, xVect, nStepsLocal, err);
    printf("%d %d\n", nStepsLocal[0], err[0]);
    for (int k = 0; k < nStepsLocal[0] && k < nSteps; ++k) {
        printf("%.9g", tVect[k]);
        for (int o = 0; o < nOutputs; ++o) printf(" %.9g", xVect[o + nOutputs * k]);
        printf("\n");
    }
    CloseGPUC();
    free(tVect);
    free(xVect);
    return err[0] == 0 ? 0 : 4;
}
