/*
 * mex.h -- declarations of the subset of MATLAB's MEX / mx C API that the
 * kwave_b200 gateway uses, written for a compile check where MATLAB is not
 * installed.  Only the documented signatures are reproduced; there is no
 * implementation here.  With MATLAB present, build against MATLAB's own
 * headers instead (`mex` puts them on the include path).
 */
#ifndef KWAVE_B200_MEX_STUB_H
#define KWAVE_B200_MEX_STUB_H

#include <stdbool.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef size_t mwIndex;

typedef enum {
    mxUNKNOWN_CLASS = 0, mxCELL_CLASS, mxSTRUCT_CLASS, mxLOGICAL_CLASS, mxCHAR_CLASS, mxVOID_CLASS,
    mxDOUBLE_CLASS, mxSINGLE_CLASS, mxINT8_CLASS, mxUINT8_CLASS, mxINT16_CLASS, mxUINT16_CLASS,
    mxINT32_CLASS, mxUINT32_CLASS, mxINT64_CLASS, mxUINT64_CLASS, mxFUNCTION_CLASS
} mxClassID;

typedef enum { mxREAL = 0, mxCOMPLEX } mxComplexity;

mxArray *mxGetField(const mxArray *pm, mwIndex index, const char *fieldname);
double mxGetScalar(const mxArray *pm);
void *mxGetData(const mxArray *pm);
size_t mxGetNumberOfElements(const mxArray *pm);
size_t mxGetM(const mxArray *pm);
size_t mxGetN(const mxArray *pm);
mxClassID mxGetClassID(const mxArray *pm);
bool mxIsStruct(const mxArray *pm);
bool mxIsCell(const mxArray *pm);
bool mxIsChar(const mxArray *pm);
mxArray *mxGetCell(const mxArray *pm, mwIndex index);
char *mxArrayToString(const mxArray *array_ptr);
void mxFree(void *ptr);
mxArray *mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID classid, mxComplexity flag);
mxArray *mxCreateNumericArray(mwSize ndim, const mwSize *dims, mxClassID classid, mxComplexity flag);
mxArray *mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char **fieldnames);
int mxAddField(mxArray *pm, const char *fieldname);
void mxSetField(mxArray *pm, mwIndex index, const char *fieldname, mxArray *pvalue);
void mexErrMsgIdAndTxt(const char *errorid, const char *errormsg, ...);

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);

#ifdef __cplusplus
}
#endif

#endif /* KWAVE_B200_MEX_STUB_H */
