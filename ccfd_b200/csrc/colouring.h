// Distance-3 colouring of the face-neighbour graph, for the coloured
// finite-difference Jacobian of buildMatrix (src/linearSolver.c:186-252).
//
// The reference obtains one Jacobian column per residual evaluation.  The
// residual of a cell depends on the states within two face-neighbour steps
// (second-order gradients and limiters of its neighbours), and a column of
// cell j is read in the rows of j and of its face neighbours; so columns of
// cells more than three steps apart can be evaluated in one residual pass.
// Any valid colouring gives the same Jacobian entries; fewer colours mean
// fewer residual evaluations.
#pragma once

#include <vector>

// Colours the cells 0..n-1 of the graph given by half-side lists
// (hs_off[n + 1], hs_nb[hs_off[n]], negative entries are boundary sides) so
// that no two cells within three steps share a colour.  The best of two
// greedy passes (cell order, and `order2` if given) is refined by a tabu
// search that removes colours while it succeeds within `budget` examined
// candidate moves (cell, colour) per attempt (deterministic: fixed seed).
// Returns the number of colours.
int ccfd_distance3_colouring(long n, const int* hs_off, const int* hs_nb, const int* order2, long budget,
                             std::vector<int>& color);

// The default budget of one colour-removal attempt for n cells (candidate
// moves examined; about 0.1 s of host time at the most).
long ccfd_colouring_budget(long n);
