/* ParODEEnums.h -- solver ids and error codes of the ParODE API.
 * Values are those of the reference's Include/ParODEEnums.h:11-26; callers
 * compare against them, so they must not change. */
#ifndef PARODEENUMS_H_
#define PARODEENUMS_H_

enum SolverType {
  RUNGE_KUTTA = 0,
  ADAMS_BASHFORTH_MOULTON = 1
};

enum ErrorCode {
  ParODE_OK = 0,
  ParODE_NoGPU = -1,
  ParODE_NotInitialized = -2,
  ParODE_CouldNotCreateGPUKernels = -3,
  ParODE_NotEnoughResources = -4,
  ParODE_InvalidDeviceId = -5,
  ParODE_InvalidSystem = -6,
  ParODE_InvalidSolverType = -7
};

#endif /* PARODEENUMS_H_ */
