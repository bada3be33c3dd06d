/* Minimal declarations of the MATLAB/Octave MEX interface, only those the
 * gateway mex/ins2d_mex.cpp uses, with the signatures of the documented
 * MEX C API.  Test infrastructure: lets the CPU tests compile the gateway
 * where no MATLAB or Octave is installed (tests/test_mex_gateway.py); it is
 * never linked into the library. */
#ifndef INS2D_TEST_MEX_H
#define INS2D_TEST_MEX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef size_t mwIndex;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;
typedef enum {
  mxUNKNOWN_CLASS = 0,
  mxCELL_CLASS,
  mxSTRUCT_CLASS,
  mxLOGICAL_CLASS,
  mxCHAR_CLASS,
  mxVOID_CLASS,
  mxDOUBLE_CLASS,
  mxSINGLE_CLASS,
  mxINT8_CLASS,
  mxUINT8_CLASS,
  mxINT16_CLASS,
  mxUINT16_CLASS,
  mxINT32_CLASS,
  mxUINT32_CLASS,
  mxINT64_CLASS,
  mxUINT64_CLASS,
  mxFUNCTION_CLASS
} mxClassID;

mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity flag);
mxArray *mxCreateDoubleScalar(double value);
mxArray *mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID classid, mxComplexity flag);
mxArray *mxCreateString(const char *str);
mxArray *mxDuplicateArray(const mxArray *in);
void mxDestroyArray(mxArray *pa);
double *mxGetPr(const mxArray *pa);
void *mxGetData(const mxArray *pa);
mxArray *mxGetField(const mxArray *pa, mwIndex i, const char *fieldname);
size_t mxGetM(const mxArray *pa);
size_t mxGetNumberOfElements(const mxArray *pa);
double mxGetScalar(const mxArray *pa);
int mxGetString(const mxArray *pa, char *buf, mwSize buflen);
bool mxIsChar(const mxArray *pa);
bool mxIsEmpty(const mxArray *pa);
bool mxIsNumeric(const mxArray *pa);
bool mxIsUint64(const mxArray *pa);

int mexCallMATLAB(int nlhs, mxArray *plhs[], int nrhs, mxArray *prhs[], const char *fcn_name);
void mexErrMsgIdAndTxt(const char *identifier, const char *err_msg, ...);
void mexMakeArrayPersistent(mxArray *pa);

#ifdef __cplusplus
}
#endif

#endif
