// Round trip and rejection cases of the tree checkpoint format
// (checkpoint_file.h).  Built and run by tests/test_checkpoint_cpu.py with a
// scratch directory as argv[1]; exits non-zero on the first failure.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <random>
#include <string>
#include <vector>

#include "checkpoint_file.h"

#define CHECK(c)                                                         \
    do {                                                                 \
        if (!(c)) {                                                      \
            fprintf(stderr, "check failed line %d: %s\n", __LINE__, #c); \
            return 1;                                                    \
        }                                                                \
    } while (0)

static std::vector<unsigned char> slurp(const std::string &p) {
    std::vector<unsigned char> b;
    FILE *f = fopen(p.c_str(), "rb");
    if (!f) return b;
    int c;
    while ((c = fgetc(f)) != EOF) b.push_back((unsigned char)c);
    fclose(f);
    return b;
}
static void spit(const std::string &p, const std::vector<unsigned char> &b) {
    FILE *f = fopen(p.c_str(), "wb");
    fwrite(b.data(), 1, b.size(), f);
    fclose(f);
}

int main(int argc, char **argv) {
    if (argc < 2) return 2;
    const std::string dir = argv[1], path = dir + "/tree.ckpt";
    std::mt19937 rng(77);
    std::vector<uint32_t> q(1000), r(1234), q2, r2;
    for (auto &v : q) v = rng();
    for (auto &v : r) v = rng();
    CHECK(!gpupi::ckpt_read(path.c_str(), 8, q2, r2));             // no file
    CHECK(gpupi::ckpt_write(path.c_str(), 8, q, r));
    CHECK(slurp(path + ".tmp").empty());                            // renamed into place
    CHECK(gpupi::ckpt_read(path.c_str(), 8, q2, r2) && q2 == q && r2 == r);
    CHECK(!gpupi::ckpt_read(path.c_str(), 16, q2, r2));             // another tree size
    const std::vector<unsigned char> good = slurp(path);
    CHECK(good.size() == sizeof(gpupi::CkptHeader) + 4 * (q.size() + r.size()));
    for (size_t pos : {size_t(0), size_t(9), sizeof(gpupi::CkptHeader) + 17, good.size() - 1}) {
        std::vector<unsigned char> bad = good;
        bad[pos] ^= 0x10;                                           // a flipped bit anywhere
        spit(path, bad);
        CHECK(!gpupi::ckpt_read(path.c_str(), 8, q2, r2));
    }
    std::vector<unsigned char> cut(good.begin(), good.end() - 4);   // truncated
    spit(path, cut);
    CHECK(!gpupi::ckpt_read(path.c_str(), 8, q2, r2));
    std::vector<unsigned char> longer = good;                       // trailing bytes
    longer.push_back(0);
    spit(path, longer);
    CHECK(!gpupi::ckpt_read(path.c_str(), 8, q2, r2));
    // damaged length fields (header offsets 16: Q limbs, 20: R limbs): a
    // huge length is rejected by the file-size check before any allocation;
    // moving one word from R to Q keeps the size but not the checksum
    auto set_u32 = [](std::vector<unsigned char> &b, size_t off, uint32_t v) { memcpy(b.data() + off, &v, 4); };
    for (uint32_t lq : {0xFFFFFFF0u, 0x40000000u, 0u}) {
        std::vector<unsigned char> bad = good;
        set_u32(bad, 16, lq);
        spit(path, bad);
        CHECK(!gpupi::ckpt_read(path.c_str(), 8, q2, r2));
    }
    {
        std::vector<unsigned char> bad = good;
        set_u32(bad, 16, (uint32_t)q.size() + 1u);
        set_u32(bad, 20, (uint32_t)r.size() - 1u);
        spit(path, bad);
        CHECK(!gpupi::ckpt_read(path.c_str(), 8, q2, r2));
    }
    spit(path, good);
    CHECK(!gpupi::ckpt_read(path.c_str(), 8, q2, r2, 1233));        // R above the caller's bound
    CHECK(gpupi::ckpt_read(path.c_str(), 8, q2, r2, 1234) && q2 == q && r2 == r);
    // an unwritable location: the write fails cleanly and leaves nothing
    const std::string nodir = dir + "/missing/tree.ckpt";
    CHECK(!gpupi::ckpt_write(nodir.c_str(), 8, q, r));
    CHECK(slurp(nodir + ".tmp").empty());
    printf("checkpoint ok\n");
    return 0;
}
