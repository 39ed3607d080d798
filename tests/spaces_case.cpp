// Driver of tests/test_spaces.py: k segments of merge_thin_segments for a
// column given on the command line: end, z-slab ranges and box ranges; a
// negative END means z tails (the slab is not cut and makes no segment
// general: the lean and Debye kernels take its groups), as engine.cu
// build_spaces ranks them.
// usage: spaces_case END S0 S1 B0 B1 [CUT ...]   (empty ranges: S0 = S1)
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "../courant_b200/csrc/spaces.hpp"

int main(int argc, char **argv) {
    const bool tails = atoi(argv[1]) < 0;
    const int end = abs(atoi(argv[1])), s0 = atoi(argv[2]), s1 = atoi(argv[3]), b0 = atoi(argv[4]), b1 = atoi(argv[5]);
    std::vector<int> kb{0};
    for (int q = 6; q < argc; q++) kb.push_back(atoi(argv[q]));
    kb.push_back(end);
    cb2::merge_thin_segments(kb, [&](int ks, int ke) {
        const bool zs = ke > s0 && ks < s1, box = ke > b0 && ks < b1;
        if (zs && !tails) return 2;
        return box ? 1 : 0;
    });
    for (int v : kb) printf("%d ", v);
    printf("\n");
    return 0;
}
