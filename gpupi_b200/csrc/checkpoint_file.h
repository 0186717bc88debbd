// File format of the splitting tree's checkpoint (host side, no CUDA):
// a header {"GPUPICK1", version 1, tree size N, Q limbs, R limbs, 64-bit
// checksum of the limbs} followed by Q's and R's limbs, little-endian.
// Written to <path>.tmp and renamed, so a file that exists is complete; a
// read checks the header, N and the checksum, and that nothing follows.
#pragma once

#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

namespace gpupi {

struct CkptHeader {
    char magic[8];
    uint32_t version, N, lq, lr;
    uint64_t sum;
};

inline uint64_t ckpt_checksum(const uint32_t *a, size_t n, uint64_t h) {
    for (size_t i = 0; i < n; ++i) {
        h ^= a[i];
        h *= 0x100000001b3ull;   // FNV-1a prime, one 32-bit word per step
        h ^= h >> 29;
    }
    return h;
}

inline uint64_t ckpt_sum(const std::vector<uint32_t> &q, const std::vector<uint32_t> &r) {
    return ckpt_checksum(r.data(), r.size(), ckpt_checksum(q.data(), q.size(), 0xcbf29ce484222325ull));
}

// true and q, r filled when path holds a valid checkpoint for tree size N
inline bool ckpt_read(const char *path, uint32_t N, std::vector<uint32_t> &q, std::vector<uint32_t> &r) {
    FILE *f = fopen(path, "rb");
    if (!f) return false;
    CkptHeader h{};
    bool ok = fread(&h, sizeof h, 1, f) == 1 && memcmp(h.magic, "GPUPICK1", 8) == 0 && h.version == 1u &&
              h.N == N && h.lq > 0u && h.lr > 0u;
    if (ok) {
        q.resize(h.lq);
        r.resize(h.lr);
        ok = fread(q.data(), 4, h.lq, f) == h.lq && fread(r.data(), 4, h.lr, f) == h.lr && fgetc(f) == EOF;
    }
    fclose(f);
    return ok && ckpt_sum(q, r) == h.sum;
}

inline bool ckpt_write(const char *path, uint32_t N, const std::vector<uint32_t> &q,
                       const std::vector<uint32_t> &r) {
    CkptHeader h{};
    memcpy(h.magic, "GPUPICK1", 8);
    h.version = 1u;
    h.N = N;
    h.lq = (uint32_t)q.size();
    h.lr = (uint32_t)r.size();
    h.sum = ckpt_sum(q, r);
    const std::string tmp = std::string(path) + ".tmp";
    FILE *f = fopen(tmp.c_str(), "wb");
    if (!f) return false;
    bool ok = fwrite(&h, sizeof h, 1, f) == 1 && fwrite(q.data(), 4, q.size(), f) == q.size() &&
              fwrite(r.data(), 4, r.size(), f) == r.size();
    ok = (fclose(f) == 0) && ok && rename(tmp.c_str(), path) == 0;
    if (!ok) remove(tmp.c_str());
    return ok;
}

}  // namespace gpupi
