// dihedral.h -- the 8-fold (dihedral) task decomposition of a whole board.
//
// The reference counts only the left-right mirror: row 0 is restricted to the
// left half and every prefix is counted twice (src/n_queens.cpp:74-113,
// src/n_queens_cuda.cu:181-183).  This decomposition uses all eight symmetries
// of the square and needs about 1.75x fewer DFS nodes for the same total.
//
// Solutions are split into three families by their border queens (the queens
// in row 0, row N-1, column 0 and column N-1):
//
//  * corner: a queen at (0,0).  The transpose of such a solution is another
//    solution (a transposed pair (i,j),(j,i) would share an anti-diagonal, so
//    no solution is its own transpose) and rotations move the corner.  The
//    representative has its row-1 queen column B1 below the row of its
//    column-1 queen.  B1 < k: the prefix bars column 1 from rows 2..B1-1,
//    weight 8.  B1 >= k: a solution and its transpose both have B1 >= k and
//    column-1 row >= k; the prefix bars column 1 from rows 2..k-1 and each
//    is counted with weight 4.
//  * class m (1 <= m <= k-1, 2m < N-1): the border queens' smallest distance
//    to a corner is m and (0,m) stands for it.  Rows 1..m-1 hold no queen in
//    column 0 or N-1, nor do rows below B2 = N-1-m, and the row N-1 queen
//    lies in [m, N-1-m].  The cells at distance m that (0,m) does not attack
//    are X1 = (m,N-1), X2 = (B2,0), X3 = (N-1,N-1-m); a quarter turn cycles
//    (0,m) -> X1 -> X3 -> X2.  Picking, among the nearest border queens,
//    those whose quarter-turn successor cell is empty makes a solution
//    canonical when X1 is empty (weight 8, or 4 when X3 is taken and X2
//    empty) or when all four cells are taken (weight 2).  The half turn maps
//    {X1 empty, X2 and X3 taken} onto {X1 and X3 taken, X2 empty}; with that
//    pairing no search needs to know X2:
//      x1 = 0 prefixes: weight 8, or 4 when the row N-1 queen is at X3;
//      x1 = 1 prefixes, twice: (A) side columns barred below row B2 and
//        (B) barred from row B2 on, both with the row N-1 queen at X3,
//        weight 2 each.
//  * rest: every border queen at distance >= k.  Only the mirror and the
//    top-bottom flip are used: the top queen at (0,a), k <= a, 2a < N-1; no
//    side-column queen in rows 1..k-1 or below N-1-k; the row N-1 queen in
//    [a, N-1-a]; weight 4, or 2 when it is at N-1-a.
//
// Below the prefix a task follows three rules, held in its class: rows beyond
// `side_row` may not use column 0 or N-1, row N-1 is masked by `last_mask`,
// and a completion weighs `w_tie` when its row N-1 queen is `tie_bit`, else
// `w`.
#pragma once

#include <stdint.h>

#include <vector>

namespace nqb {

// Same layout as nq_dihedral_class in include/n_queens_b200.h.
struct DihClass {
    int32_t side_row;
    uint32_t last_mask;
    uint32_t tie_bit;
    uint32_t w;
    uint32_t w_tie;
};

constexpr int kMaxDihClasses = 64;

// Class table of (N, k): every class of the decomposition in a fixed order,
// whether or not it gets a task.  Returns false for a bad (N, k).
bool dihedral_classes(int N, int k, std::vector<DihClass> &out);

// Tasks of (N, k) in class order, lowest column first within a class.
// Writes at most `cap` tasks (cols are on-board bits, ld/rd as the reference
// packs them) and returns the total count, or -1 for a bad (N, k).
int64_t dihedral_expand(int N, int k, uint32_t *cols, uint32_t *ld, uint32_t *rd, uint8_t *cls, int64_t cap);

}  // namespace nqb
