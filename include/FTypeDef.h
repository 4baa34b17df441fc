/* FTypeDef.h -- element type of the ParODE C ABI.
 * Same typedef as the reference's Include/FTypeDef.h:4 (float), so binaries
 * built against the reference headers link unchanged. */
#ifndef __FTYPE__
#define __FTYPE__

typedef float fType;

#endif
