// Workspace of the batched (many right-hand sides) solve; see batch.cu.
#pragma once

#include "common.h"
#include "gmres.cuh"

namespace fftsvd {

struct BatchWorkspace {
   int ncols = 0;     // columns (a multiple of kBatchGroup)
   int capacity = 0;  // basis vectors per column
   DevBuf<double> V;  // capacity blocks of ncols x n
   DevBuf<double> H, cs, sn, g, h1, h2, y, partial, normpart, scal, factor;
   DevBuf<double> w, r, b0, x0, xout, t0, t1, t2;  // ncols x n each
   DevBuf<GivensState> st;
   DevBuf<int32_t> active;
   void ensure(int n, int cols, int cap);
};

}  // namespace fftsvd
