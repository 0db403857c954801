"""The MEX gateway compiles against the C ABI header (MATLAB's MEX API is
replaced by a stub declaring the functions the gateway uses)."""
import os
import subprocess

from conftest import ROOT

STUB = r"""
#include <stddef.h>
typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef enum { mxDOUBLE_CLASS } mxClassID;
typedef enum { mxREAL } mxComplexity;
void mexErrMsgIdAndTxt(const char*, const char*, ...);
int mexAtExit(void (*)(void));
const mxArray* mxGetField(const mxArray*, size_t, const char*);
double mxGetScalar(const mxArray*);
double* mxGetPr(const mxArray*);
size_t mxGetNumberOfElements(const mxArray*);
size_t mxGetM(const mxArray*);
size_t mxGetN(const mxArray*);
void* mxMalloc(size_t);
void mxFree(void*);
mxArray* mxCreateDoubleMatrix(size_t, size_t, mxComplexity);
mxArray* mxCreateNumericArray(mwSize, const mwSize*, mxClassID, mxComplexity);
void mxDestroyArray(mxArray*);
mxArray* mxGetCell(const mxArray*, size_t);
int mxGetString(const mxArray*, char*, size_t);
"""


def test_mex_gateway_compiles(tmp_path):
    (tmp_path / "mex.h").write_text(STUB)
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-I", str(tmp_path), "-I",
                        os.path.join(ROOT, "include"), os.path.join(ROOT, "mex", "gj_mex.c")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
