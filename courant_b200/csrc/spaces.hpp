// Host-side layout rule of the update kernels' thread spaces (engine.cu
// build_spaces), kept apart so that it can be tested on its own.
#pragma once

#include <vector>

namespace cb2 {

// The k axis of a node plane is cut into segments at `kb` (sorted, first 0,
// last the end of the k range); one thread moves four consecutive k, and the
// threads of a segment's rows follow one another. A segment thinner than four
// groups (kThin = 16 points by default; the tuner tries others) leaves most
// lanes of a warp on different rows, so it
// joins a neighbour, and the joined range takes its own class. rank(ks, ke):
// 2 when [ks, ke) goes to the general kernel (it reaches a z CPML slab that
// the lean kernels do not take, or holds both slab and Debye points), 1 when
// it meets a Debye box (lean Debye kernel, which also handles points outside
// the box), 0 otherwise (lean kernel). A thin segment never joins a thick
// neighbour whose rank the joined range would exceed (that would move the
// whole thick segment to a costlier kernel: a thin Debye box above a thick
// plain region stays thin); among the neighbours it may join, the one whose
// joined range is cheapest is taken (Debye, then plain, then general; the
// thinner on a tie); with none it stays as it is.
template <class Rank>
void merge_thin_segments(std::vector<int> &kb, Rank rank, int kThin = 16) {
    static const int cost[3] = {1, 0, 2};   // by rank: plain, box, slab
    for (bool changed = true; changed && kb.size() > 2;) {
        changed = false;
        for (size_t q = 0; q + 1 < kb.size(); q++) {
            if (kb[q + 1] - kb[q] >= kThin) continue;
            int best = -1, best_cost = 99, best_w = 1 << 30;   // cut to erase, its cost, the neighbour's width
            for (int side = 0; side < 2; side++) {
                if (side == 0 ? q == 0 : q + 2 >= kb.size()) continue;
                const int a = side == 0 ? kb[q - 1] : kb[q + 1], b = side == 0 ? kb[q] : kb[q + 2];
                const int nr = rank(a, b), nw = b - a;
                const int joined = rank(side == 0 ? a : kb[q], side == 0 ? kb[q + 1] : b);
                if (nw >= kThin && joined > nr) continue;
                if (cost[joined] < best_cost || (cost[joined] == best_cost && nw < best_w)) {
                    best = side == 0 ? (int)q : (int)q + 1;
                    best_cost = cost[joined];
                    best_w = nw;
                }
            }
            if (best < 0) continue;   // stays thin
            kb.erase(kb.begin() + best);
            changed = true;
            break;
        }
    }
}

}  // namespace cb2
