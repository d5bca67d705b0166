// am_chunks.hpp -- warp-chunk plans of one-thread-per-element blocks (host code).
//
// The force kernels of such blocks sum, per warp, the nodal forces of the warp's 32 units
// (elements, or split-hex half patches) on each node they share, and write one slot per
// distinct node. The plan built here tells each lane which staged entries it sums, in an
// order fixed by the connectivity's unit order and corner order alone.
#pragma once

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace am {

// Warp chunks of a Gauss block of nn-node elements run one thread per element: chunk c
// holds elements [32c, 32c + 32) in the processing order. Its distinct nodes, ranked by first
// appearance over the entry codes q = 32 a + lane (connectivity node a of the chunk's element
// lane), take logical slots ptr[c] + rank. The chunk's entries sorted by (rank, code) go nn to
// a lane, a byte each: words (32 c + l) nn/4 .. (32 c + l + 1) nn/4 - 1 of code / rank hold
// lane l's, rank 0xFF past the chunk's last element. All of it follows from the element order
// and the corner order, not from the node numbers. Fails (false) when a chunk has more than
// 254 distinct nodes, which the rank bytes cannot hold.
struct WarpChunks {
    std::vector<int32_t> ptr, nodes;
    std::vector<uint32_t> code, rank;
};
inline bool build_warp_chunks(const int32_t* conn, int64_t E, int nn, WarpChunks& t) {
    const int64_t C = (E + 31) / 32;
    const int W = nn / 4, Q = 32 * nn;
    t.ptr.assign(C + 1, 0);
    t.nodes.clear();
    t.code.assign(static_cast<size_t>(32 * W * C), 0xFFFFFFFFu);
    t.rank.assign(static_cast<size_t>(32 * W * C), 0xFFFFFFFFu);
    std::vector<int32_t> node(Q);
    std::vector<int> which(Q), count(Q + 1), fill(Q);
    for (int64_t c = 0; c < C; ++c) {
        const int64_t e0 = 32 * c;
        const int n = static_cast<int>(std::min<int64_t>(32, E - e0));
        std::fill(count.begin(), count.end(), 0);
        int nd = 0;
        for (int q = 0; q < Q; ++q) {
            which[q] = -1;
            if ((q & 31) >= n) continue;
            const int32_t v = conn[nn * (e0 + (q & 31)) + (q >> 5)];
            int k = 0;
            while (k < nd && node[k] != v) ++k;
            if (k == nd) node[nd++] = v;
            which[q] = k;
            ++count[k + 1];
        }
        if (nd > 254) return false;
        for (int k = 0; k < nd; ++k) count[k + 1] += count[k];
        for (int k = 0; k < nd; ++k) fill[k] = count[k];
        for (int q = 0; q < Q; ++q) {
            if (which[q] < 0) continue;
            const int j = fill[which[q]]++;  // sorted position: lane j / nn, entry j % nn of it
            const size_t w = static_cast<size_t>((32 * c + j / nn) * W + (j % nn) / 4);
            const int sh = 8 * (j % 4);
            t.code[w] = (t.code[w] & ~(0xFFu << sh)) | (static_cast<uint32_t>(q & 0xFF) << sh);
            t.rank[w] = (t.rank[w] & ~(0xFFu << sh)) | (static_cast<uint32_t>(which[q]) << sh);
        }
        for (int k = 0; k < nd; ++k) t.nodes.push_back(node[k]);
        t.ptr[c + 1] = t.ptr[c] + nd;
    }
    return true;
}

}  // namespace am
