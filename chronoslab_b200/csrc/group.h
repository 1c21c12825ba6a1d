// Grouped solve of a batch of independent problems (group.cu): the problems'
// level operators stacked block-diagonally per level, one launch per operator
// and level for the whole batch, per-problem PCG_CJ scalars and reductions.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "hier.h"

namespace chronos {

struct GroupLevel {
  std::vector<int> S, C;     // problems smoothing at this level / whose coarsest level it is
  std::vector<int> off;      // per problem: first row of its slice in this level's vectors
  int nS = 0, nV = 0;        // rows of the smoothing problems (a prefix) / of all
  // A, G, G' (scaled by each problem's omega) over the nS rows; P: nS rows x
  // the next level's nV columns; P': the next level's nV rows x nS columns
  DMat A, G, Gt, P, Pt;
  DBuf<float> b32, x32, r32, t32;
  DBuf<double> b64, x64, r64, t64;
};

struct GroupSolve {
  int np = 0, nrows = 0, precision = CHRONOS_FP32;
  chronos_params prm{};
  std::vector<GroupLevel> lev;
  DMat A0;                                   // finest operators of all problems (FP64)
  DBuf<int> rstart, bstart;                  // per problem: rows and blocks of the vector kernels
  int nblocks = 0;
  int ncoarse_rows = 0;                      // batched coarsest solves
  DBuf<int> c_prob, c_row, c_n;
  DBuf<uintptr_t> c_W, c_b, c_x;
  DBuf<double> x, res, p, axp, pres, b, sc, part;
  DBuf<unsigned> tickets, ctl;
  cudaStream_t st = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  double g_tol = -1.0;
  int g_itmax = -1;
  ~GroupSolve();
};

// True when every problem has at least two levels and all share a precision.
bool group_supported(const std::vector<std::unique_ptr<Hier>> &h);
std::unique_ptr<GroupSolve> group_build(const std::vector<std::unique_ptr<Hier>> &h,
                                        const chronos_params &prm);
// x_h[p] holds x0 on entry and the solution on return; PCG_CJ semantics per
// problem (iterations, flag: 1 when not converged or on breakdown).
void group_solve(GroupSolve &g, const std::vector<const double *> &b_h,
                 const std::vector<double *> &x_h, int itmax, double tol, int *iters, int *flags,
                 double *seconds);

}  // namespace chronos
