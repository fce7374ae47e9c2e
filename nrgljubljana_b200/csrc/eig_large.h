// eig_large.h -- internal: planner of the large-block eigensolver path.
#pragma once
#include <vector>

#include "ctx.h"

namespace nrg {

// Solves the blocks listed in `which` (orders n[b] > kSmallMaxN) on stream s:
// tridiagonalisation, divide and conquer, back-transform. Status words go to info_dev[b].
int eig_large_run(nrg_ctx* c, const std::vector<int>& which, const int* n, double* const* H, double* const* evals,
                  double* const* evecs, int* info_dev, cudaStream_t s);

}  // namespace nrg
