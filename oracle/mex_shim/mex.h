/* A minimal stand-in for MATLAB's MEX C API, just large enough to compile the
 * reference's MEX_cptProlPatt.cpp (EMIN/MEX_EMIN) unmodified outside MATLAB.
 *
 * ORACLE TEST INFRASTRUCTURE: only oracle/ref_bridge_emin.cpp uses it, to run
 * the reference's pattern construction from oracle/_ref; nothing in the
 * chronoslab_b200 package includes it.
 *
 * An mxArray here is either a dense double matrix (column-major) or a sparse
 * double matrix in MATLAB's CSC layout (jc column pointers, ir row indices,
 * pr values).  mexErrMsgIdAndTxt throws MexError instead of unwinding to
 * MATLAB; the bridge catches it. */
#pragma once
#include <cstddef>
#include <stdexcept>
#include <string>
#include <vector>

typedef size_t mwIndex;
typedef size_t mwSize;
enum mxComplexity { mxREAL = 0 };

struct mxArray {
  bool sparse = false;
  size_t m = 0, n = 0;
  std::vector<mwIndex> jc, ir;
  std::vector<double> pr;
};

struct MexError : std::runtime_error {
  explicit MexError(const std::string &s) : std::runtime_error(s) {}
};

inline size_t mxGetM(const mxArray *a) { return a->m; }
inline size_t mxGetN(const mxArray *a) { return a->n; }
inline bool mxIsSparse(const mxArray *a) { return a->sparse; }
inline mwIndex *mxGetJc(const mxArray *a) { return const_cast<mwIndex *>(a->jc.data()); }
inline mwIndex *mxGetIr(const mxArray *a) { return const_cast<mwIndex *>(a->ir.data()); }
inline double *mxGetDoubles(const mxArray *a) { return const_cast<double *>(a->pr.data()); }
inline double mxGetScalar(const mxArray *a) { return a->pr.empty() ? 0.0 : a->pr[0]; }
inline size_t mxGetNumberOfElements(const mxArray *a) { return a->m * a->n; }

inline mxArray *mxCreateSparse(mwSize m, mwSize n, mwSize nzmax, mxComplexity) {
  mxArray *a = new mxArray;
  a->sparse = true;
  a->m = m;
  a->n = n;
  a->jc.assign(n + 1, 0);
  a->ir.assign(nzmax, 0);
  a->pr.assign(nzmax, 0.0);
  return a;
}

inline void mexErrMsgIdAndTxt(const char *id, const char *msg, ...) {
  throw MexError(std::string(id) + ": " + msg);
}

inline int mexPrintf(const char *, ...) { return 0; }

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);
