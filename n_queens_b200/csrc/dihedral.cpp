// dihedral.cpp -- host expander of the 8-fold decomposition (dihedral.h).
#include "dihedral.h"

namespace nqb {

namespace {

enum Family { kCornerLow, kCornerHigh, kNearest0, kNearest1, kRest };

struct Root {
    Family fam;
    int col;  // row-0 column
    int m;    // distance class (kNearest*)
    int cls;  // class index
};

bool valid(int N, int k) { return N >= 4 && N <= 31 && k >= 2 && k <= N - 2; }

uint32_t middle_cols(int N, int a) { return ((1u << (N - a)) - 1u) & ~((1u << a) - 1u); }

// Builds the class table and the list of roots (one per class) in order.
void plan(int N, int k, std::vector<DihClass> &cls, std::vector<Root> &roots) {
    const uint32_t full = (1u << N) - 1u;
    const uint32_t side = 1u | (1u << (N - 1));
    const int M = (N - 2) / 2;
    auto add = [&](Family f, int col, int m, DihClass c) {
        roots.push_back(Root{f, col, m, (int)cls.size()});
        cls.push_back(c);
    };
    add(kCornerLow, 0, 0, DihClass{N, full, 0u, 8u, 8u});
    add(kCornerHigh, 0, 0, DihClass{N, full, 0u, 4u, 4u});
    for (int m = 1; m <= k - 1 && m <= M; ++m) {
        const int b2 = N - 1 - m;
        const uint32_t x3 = 1u << (N - 1 - m);
        add(kNearest0, m, m, DihClass{b2, middle_cols(N, m) & ~side, x3, 8u, 4u});
        add(kNearest1, m, m, DihClass{b2, x3, x3, 2u, 2u});
        add(kNearest1, m, m, DihClass{b2 - 1, x3, x3, 2u, 2u});
    }
    for (int a = k; a <= M; ++a)
        add(kRest, a, 0, DihClass{N - 1 - k, middle_cols(N, a) & ~side, 1u << (N - 1 - a), 4u, 2u});
}

// Columns a prefix row may use, before the attack masks.  `b1` is the row-1
// column of a corner root (kCornerLow bars column 1 from rows 2..b1-1).
uint32_t row_mask(const Root &rt, const DihClass &c, int N, int k, int row, int b1) {
    const uint32_t side = 1u | (1u << (N - 1));
    uint32_t a = (1u << N) - 1u;
    switch (rt.fam) {
        case kCornerLow:
            a &= row == 1 ? (((1u << k) - 1u) & ~3u) : (row < b1 ? ~2u : ~0u);
            break;
        case kCornerHigh:
            a &= row == 1 ? ~((1u << k) - 1u) : ~2u;
            break;
        case kNearest0:
            if (row <= rt.m) a &= ~side;
            break;
        case kNearest1:
            if (row < rt.m) a &= ~side;
            else if (row == rt.m) a &= 1u << (N - 1);
            break;
        case kRest:
            a &= ~side;
            break;
    }
    if (row > c.side_row) a &= ~side;
    return a;
}

}  // namespace

bool dihedral_classes(int N, int k, std::vector<DihClass> &out) {
    out.clear();
    if (!valid(N, k)) return false;
    std::vector<Root> roots;
    plan(N, k, out, roots);
    return true;
}

int64_t dihedral_expand(int N, int k, uint32_t *cols, uint32_t *ld, uint32_t *rd, uint8_t *cls, int64_t cap) {
    if (!valid(N, k)) return -1;
    std::vector<DihClass> table;
    std::vector<Root> roots;
    plan(N, k, table, roots);
    int64_t n = 0;
    // Iterative walk over rows 1..k-1.  Level d holds the masks below rows
    // 0..d-1 and the columns of row d still to try.
    uint32_t sc[32], sl[32], sr[32], sf[32];
    for (const Root &rt : roots) {
        const DihClass &c = table[(size_t)rt.cls];
        const uint32_t p0 = 1u << rt.col;
        int b1 = 0;
        sc[1] = p0;
        sl[1] = p0 << 1;
        sr[1] = p0 >> 1;
        sf[1] = row_mask(rt, c, N, k, 1, b1) & ~(sc[1] | sl[1] | sr[1]);
        int d = 1;
        while (d >= 1) {
            if (sf[d] == 0) {
                --d;
                continue;
            }
            const uint32_t p = sf[d] & (0u - sf[d]);
            sf[d] ^= p;
            if (d == 1) b1 = __builtin_ctz(p);
            const uint32_t nc = sc[d] | p, nl = (sl[d] | p) << 1, nr = (sr[d] | p) >> 1;
            if (d + 1 == k) {
                if (n < cap) {
                    cols[n] = nc;
                    ld[n] = nl;
                    rd[n] = nr;
                    cls[n] = (uint8_t)rt.cls;
                }
                ++n;
                continue;
            }
            ++d;
            sc[d] = nc;
            sl[d] = nl;
            sr[d] = nr;
            sf[d] = row_mask(rt, c, N, k, d, b1) & ~(nc | nl | nr);
        }
    }
    return n;
}

}  // namespace nqb
