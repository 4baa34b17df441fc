/*
 * ParODECInterface.h -- the plain-C ABI of libParODEShared.so.
 *
 * Drop-in replacement for the reference's Include/ParODECInterface.h:27-99
 * (bodies Sources/ParODE.cpp:23-174): the same ten symbols, the same
 * signatures, the same pointer-and-size conventions and the same error
 * convention (status in nErr[0], values of ParODEEnums.h).  Existing callers
 * -- C programs, the Python module, Scilab `link`/`call` stubs
 * (SciLabInterface/ParODEInterfaceStubs.sci) -- bind to it unchanged.
 *
 * The kernel/include folder strings are accepted and ignored: every device
 * kernel is compiled into the library for sm_100a, and a registered input
 * function is compiled at run time with NVRTC.
 *
 * The library never frees caller memory.  Calls are serialised by a mutex
 * on the process-global library state.
 */
#ifndef PARODECINTERFACE_H_
#define PARODECINTERFACE_H_

#include <FTypeDef.h>

#ifdef C_INCLUDE
#define C_EXPORT extern
#else
#define C_EXPORT
#endif

#ifndef C_INCLUDE
extern "C"
{
#endif
	/* Replaces GetErrorDescription (reference ParODECInterface.h:27).
	 * Writes a NUL-terminated description of *ErrNo; the caller's buffer must
	 * hold 256 bytes (the size the reference's Python module passes). */
	C_EXPORT void GetErrorDescription(int *ErrNo, char strErrDescription[]);

	/* Replaces InitializeAllGPUs (reference ParODECInterface.h:30-32).
	 * Initialises every CUDA device of compute capability 10.x. */
	C_EXPORT void InitializeAllGPUs(char* pszKernelFolder,
			 char* pszIncludeFolder,
			 int nErr[]);

	/* Replaces GetAvailableGPUs (reference ParODECInterface.h:39).
	 * nGPUs[0] = number of ids written to GPUIds (CUDA device ordinals). */
	C_EXPORT void GetAvailableGPUs( int nGPUs[], int GPUIds[], int nErr[]);

	/* Replaces GetDeviceName (reference ParODECInterface.h:46); the caller's
	 * buffer must hold 256 bytes. */
	C_EXPORT void GetDeviceName( int *DeviceId, char strDeviceName[], int nErr[]);

	/* Replaces InitializeSelectedGPUs (reference ParODECInterface.h:54-56).
	 * Requires a prior GetAvailableGPUs, as in the reference. */
	C_EXPORT void InitializeSelectedGPUs( int *nGPUs, int GPUIds[],
				char* pszKernelFolder,
				char* pszIncludeFolder, int nErr[]);

	/* Replaces SimulateODE (reference ParODECInterface.h:61-79).
	 * A (nStates x nStates), B (nStates x nInputs), C (nOutputs x nStates),
	 * D (nOutputs x nInputs) and x0 are row-major; ZeroB/ZeroC/ZeroD = 1 marks
	 * an absent matrix.  tVect receives nSteps[0] times and xVect
	 * nSteps[0] x nOutputs values, time-major (xVect[step*nOutputs + out];
	 * nOutputs = nStates when C and D are both absent).  The scan runs in the
	 * precision selected by ParODE_SetOption (FP64 by default); results are
	 * rounded to fType on return. */
	C_EXPORT void SimulateODE(	fType A[],
					fType B[],
					fType C[],
					fType D[],
					int *nInputs,
					int *nStates,
					int *nOutputs,
					int *ZeroB,
					int *ZeroC,
					int *ZeroD,
					int *uIndex,
					double *tStart, double *tEnd, double *tStep,
					fType x0[],
					int *solver,
					fType tVect[],
					fType xVect[],
					int *nSteps,
					int nErr[]);

	/* Replaces RegisterInput (reference ParODECInterface.h:86).
	 * uFunc must define `fType UFunc(fType t, int nInputIndex)` in CUDA C++;
	 * it is compiled with NVRTC for the current device.  uIndex[0] receives
	 * the input's index (negative on error, as the reference). */
	C_EXPORT void RegisterInput(char uFunc[], int uIndex[], int nErr[]);

	/* Replaces CloseGPUC (reference ParODECInterface.h:89). */
	C_EXPORT void CloseGPUC();

	/* Replace StartTimer / StopTimer (reference ParODECInterface.h:94-99):
	 * milliseconds between the two calls, measured with CUDA events on the
	 * library's stream of the first initialised device. */
	C_EXPORT void StartTimer(int nErr[]);
	C_EXPORT void StopTimer(float fTime[], int nErr[]);
#ifndef C_INCLUDE
}
#endif

#endif /* PARODECINTERFACE_H_ */
