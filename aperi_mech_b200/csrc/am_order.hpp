// am_order.hpp -- processing order of Gauss-element blocks (host code).
//
// The element kernels read each element's nodes and write its force slots; elements
// that share nodes should run next to each other, whatever numbering the caller's
// mesh carries. The order here depends on the mesh alone (coordinates and each
// element's own node order), so two numberings of one mesh run their elements in the
// same order, write the same slots and sum them in the same order: their results are
// bitwise identical once mapped back.
#pragma once

#include <algorithm>
#include <array>
#include <cstdint>
#include <utility>
#include <vector>

namespace am {

// Morton (z-order) key of a point: each coordinate scaled to 21 bits over the mesh's
// bounding box and the bits interleaved.
inline uint64_t spread21(uint64_t v) {
    v &= 0x1FFFFFull;
    v = (v | (v << 32)) & 0x1F00000000FFFFull;
    v = (v | (v << 16)) & 0x1F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

struct MortonFrame {
    double lo[3], scale[3];
    explicit MortonFrame(const std::vector<double>& X) {
        double hi[3];
        for (int i = 0; i < 3; ++i) lo[i] = hi[i] = X.empty() ? 0.0 : X[i];
        for (size_t k = 0; k < X.size(); ++k) {
            lo[k % 3] = std::min(lo[k % 3], X[k]);
            hi[k % 3] = std::max(hi[k % 3], X[k]);
        }
        for (int i = 0; i < 3; ++i) scale[i] = hi[i] > lo[i] ? 2097151.0 / (hi[i] - lo[i]) : 0.0;
    }
    uint64_t key(const double* x) const {
        uint64_t k = 0;
        for (int i = 0; i < 3; ++i) {
            const double q = std::min(std::max((x[i] - lo[i]) * scale[i], 0.0), 2097151.0);
            k |= spread21(static_cast<uint64_t>(q)) << i;
        }
        return k;
    }
};

// Processing order of a Gauss block (internal index -> caller's index) chosen from the
// mesh alone, so that any numbering of the same mesh gives the same order, and with it
// the same force-slot order and bitwise the same sums.
//  - Tet4: the tets are first tried as split-hex rings, found by topology: a tet
//    (c0, a, b, c3) belongs to the ring of tets sharing its first and last node; a ring
//    is six tets whose (a, b) chain closes, run from its tet of lowest centroid key. When
//    every tet lies on such a ring, the rings run in the Morton order of their axis
//    midpoints, each in its canonical ring order (the split-hex patches).
//  - Otherwise (and for Hex8) the elements run in the Morton order of their centroids,
//    which puts elements that share nodes next to each other whatever the numbering.
struct ElementOrder {
    std::vector<int32_t> order;
    bool rings = false;
};

inline ElementOrder element_order(const int32_t* conn, int64_t E, int nn, const std::vector<double>& X, bool try_rings) {
    ElementOrder eo;
    const MortonFrame mf(X);
    std::vector<uint64_t> key(E);
    for (int64_t e = 0; e < E; ++e) {
        double c[3] = {0.0, 0.0, 0.0};
        for (int a = 0; a < nn; ++a)
            for (int i = 0; i < 3; ++i) c[i] += X[3 * static_cast<size_t>(conn[nn * e + a]) + i];
        for (int i = 0; i < 3; ++i) c[i] /= nn;
        key[e] = mf.key(c);
    }
    auto by_key = [&](int32_t x, int32_t y) { return key[x] != key[y] ? key[x] < key[y] : x < y; };
    if (try_rings && nn == 4 && E % 6 == 0) {
        std::vector<int32_t> idx(E);
        for (int64_t e = 0; e < E; ++e) idx[e] = static_cast<int32_t>(e);
        auto axis = [&](int32_t e) {
            return (static_cast<uint64_t>(static_cast<uint32_t>(conn[4 * e])) << 32) | static_cast<uint32_t>(conn[4 * e + 3]);
        };
        std::sort(idx.begin(), idx.end(), [&](int32_t x, int32_t y) { return axis(x) != axis(y) ? axis(x) < axis(y) : x < y; });
        std::vector<std::pair<uint64_t, std::array<int32_t, 6>>> rings;
        rings.reserve(E / 6);
        bool ok = true;
        for (int64_t g = 0; g < E && ok; g += 6) {
            const uint64_t ax = axis(idx[g]);
            if (axis(idx[g + 5]) != ax || (g + 6 < E && axis(idx[g + 6]) == ax)) {
                ok = false;
                break;
            }
            int32_t start = idx[g];
            for (int k = 1; k < 6; ++k)
                if (by_key(idx[g + k], start)) start = idx[g + k];
            std::array<int32_t, 6> ring{};
            int32_t cur = start;
            for (int k = 0; k < 6 && ok; ++k) {
                ring[k] = cur;
                const int32_t b = conn[4 * cur + 2];
                int32_t next = -1;
                for (int j = 0; j < 6; ++j)
                    if (conn[4 * idx[g + j] + 1] == b) next = idx[g + j];
                if (next < 0 || (k < 5 && next == start)) ok = false;
                cur = next;
            }
            if (!ok || cur != start) {
                ok = false;
                break;
            }
            for (int k = 1; k < 6 && ok; ++k)
                for (int j = 0; j < k; ++j) ok = ok && ring[j] != ring[k];
            double mid[3];
            for (int i = 0; i < 3; ++i)
                mid[i] = 0.5 * (X[3 * static_cast<size_t>(conn[4 * start]) + i] + X[3 * static_cast<size_t>(conn[4 * start + 3]) + i]);
            rings.emplace_back(mf.key(mid), ring);
        }
        if (ok) {
            std::sort(rings.begin(), rings.end(), [&](const auto& x, const auto& y) {
                return x.first != y.first ? x.first < y.first : by_key(x.second[0], y.second[0]);
            });
            eo.order.reserve(E);
            for (const auto& r : rings) eo.order.insert(eo.order.end(), r.second.begin(), r.second.end());
            eo.rings = true;
            return eo;
        }
    }
    eo.order.resize(E);
    for (int64_t e = 0; e < E; ++e) eo.order[e] = static_cast<int32_t>(e);
    std::sort(eo.order.begin(), eo.order.end(), by_key);
    return eo;
}

}  // namespace am
