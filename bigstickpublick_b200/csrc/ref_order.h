// The reference's orders of haikus inside a block and of pairs inside the
// uncoupled matrix-element lists.  Host code shared by the CPU table builder
// and the GPU jump generator, so that both number SDs and pairs alike.
#pragma once

#include <cstdint>
#include <vector>

namespace bsg_order {

// Haiku order inside a block of one W (untruncated spaces have a single W
// section).  count_create_haikus (src/bbasis_haikus.f90:327-411) makes the
// haikus of nh particles from those of nh-1 in their order, appending a bit
// p > every occupied bit for p from the section's last state down; fill_blocks
// (src/bbasis_blocks.f90:474-562) keeps that order when it splits them by
// parity and Jz.  A haiku with occupied states b1 < b2 < ... < bk therefore
// comes before another when, at the first position where they differ, its
// state is the higher one; that is ascending order of the occupation mask
// with its ns bits reversed.
inline uint64_t haiku_rank(uint64_t bits, int ns) {
    uint64_t r = 0;
    for (int i = 0; i < ns; ++i)
        if (bits >> i & 1ull) r |= 1ull << (ns - 1 - i);
    return r;
}

// sortpair (src/btbme.f90:548-703): a heap sort of the generated pair list on
// M, then a heap sort of every run of equal M on parity.  Heap sort is not
// stable, so the order of pairs with equal (M, parity) is the one these exact
// sift steps leave; both passes are the textbook 1-based heap sort of
// Numerical Recipes (hpsort) on the range [s, e], with `below(x, y)` the
// relation that sends x towards the end.  The M pass sifts with the larger-M
// test reversed, which leaves M descending; the parity pass leaves parity
// index 1 (+) before 2 (-).
template <class R, class Below>
void heap_range(std::vector<R> &a, int64_t s, int64_t e, Below below) {
    auto at = [&](int64_t i) -> R & { return a[(size_t)(i - 1)]; };
    int64_t l = (e - s + 1) / 2 + s, n = e;
    while (n >= s) {
        R tmp;
        if (l > s) {
            tmp = at(--l);
        } else {
            tmp = at(n);
            at(n) = at(s);
            if (--n == s) {
                at(s) = tmp;
                break;
            }
        }
        int64_t i = l, j = l + l - (s - 1);
        while (j <= n) {
            if (j < n && below(at(j), at(j + 1))) ++j;
            if (below(tmp, at(j))) {
                at(i) = at(j);
                i = j;
                j = j + j - (s - 1);
            } else {
                j = n + 1;
            }
        }
        at(i) = tmp;
    }
}

// R has int fields M (Jz of the pair, integer) and pidx (1: +, 2: -)
template <class R>
void sortpair(std::vector<R> &a) {
    const int64_t n = (int64_t)a.size();
    if (n == 0) return;
    heap_range(a, 1, n, [](const R &x, const R &y) { return x.M > y.M; });
    int64_t i0 = 1;
    while (i0 <= n) {
        int64_t i1 = i0;
        while (i1 < n && a[(size_t)i1].M == a[(size_t)(i0 - 1)].M) ++i1;
        heap_range(a, i0, i1, [](const R &x, const R &y) { return x.pidx < y.pidx; });
        i0 = i1 + 1;
    }
}

}  // namespace bsg_order
