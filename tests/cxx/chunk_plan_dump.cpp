// Writes the warp-chunk plan the library builds (am_chunks.hpp) for a connectivity read
// from a file, so that a CPU test can check it against its restatement.
// Input (argv[1]): int64 E, int64 nn, then E x nn int32 node ids.
// Output (argv[2]): int64 ok, int64 C, int64 G, then ptr (C + 1 int32), nodes (G int32),
// code and rank (32 C nn / 4 uint32 each).
#include <cstdint>
#include <cstdio>
#include <vector>

#include "am_chunks.hpp"

int main(int argc, char** argv) {
    if (argc != 3) return 2;
    FILE* in = std::fopen(argv[1], "rb");
    if (!in) return 3;
    int64_t head[2];
    if (std::fread(head, sizeof(int64_t), 2, in) != 2) return 4;
    std::vector<int32_t> conn(static_cast<size_t>(head[0] * head[1]));
    if (std::fread(conn.data(), sizeof(int32_t), conn.size(), in) != conn.size()) return 5;
    std::fclose(in);
    am::WarpChunks wc;
    const int64_t ok = am::build_warp_chunks(conn.data(), head[0], static_cast<int>(head[1]), wc) ? 1 : 0;
    FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 6;
    const int64_t sizes[3] = {ok, static_cast<int64_t>(wc.ptr.size()) - 1, static_cast<int64_t>(wc.nodes.size())};
    std::fwrite(sizes, sizeof(int64_t), 3, out);
    std::fwrite(wc.ptr.data(), sizeof(int32_t), wc.ptr.size(), out);
    std::fwrite(wc.nodes.data(), sizeof(int32_t), wc.nodes.size(), out);
    std::fwrite(wc.code.data(), sizeof(uint32_t), wc.code.size(), out);
    std::fwrite(wc.rank.data(), sizeof(uint32_t), wc.rank.size(), out);
    std::fclose(out);
    return 0;
}
