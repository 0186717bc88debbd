// File format of the splitting tree's checkpoint (host side, no CUDA):
// a header {"GPUPICK1", version 2, tree size N, Q limbs, R limbs, 64-bit
// checksum of both lengths and the limbs} followed by Q's and R's limbs,
// little-endian.
// Written to <path>.tmp, flushed to the disk (fsync), renamed and the
// directory synced, so a file that exists under <path> is complete even
// after a crash.  A read checks the header, N, that the file's size is
// exactly the header's lengths (before anything is allocated, so a damaged
// length field cannot make it allocate) and the checksum.  The checksum is
// unkeyed: it catches damage, not a deliberately forged file.
#pragma once

#include <fcntl.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <unistd.h>

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

// The lengths are hashed first: the limbs alone would give one checksum
// for every split of the same words into Q and R.
inline uint64_t ckpt_sum(const std::vector<uint32_t> &q, const std::vector<uint32_t> &r) {
    const uint32_t lens[2] = {(uint32_t)q.size(), (uint32_t)r.size()};
    const uint64_t h = ckpt_checksum(lens, 2, 0xcbf29ce484222325ull);
    return ckpt_checksum(r.data(), r.size(), ckpt_checksum(q.data(), q.size(), h));
}

// true and q, r filled when path holds a valid checkpoint for tree size N
// whose lengths lie in [1, max_limbs]
inline bool ckpt_read(const char *path, uint32_t N, std::vector<uint32_t> &q, std::vector<uint32_t> &r,
                      uint64_t max_limbs = UINT32_MAX) {
    FILE *f = fopen(path, "rb");
    if (!f) return false;
    CkptHeader h{};
    bool ok = fread(&h, sizeof h, 1, f) == 1 && memcmp(h.magic, "GPUPICK1", 8) == 0 && h.version == 2u &&
              h.N == N && h.lq > 0u && h.lr > 0u && h.lq <= max_limbs && h.lr <= max_limbs;
    if (ok) {
        // the lengths must describe exactly this file before any allocation
        const long at = ftell(f);
        ok = at >= 0 && fseek(f, 0, SEEK_END) == 0 &&
             (uint64_t)ftell(f) == (uint64_t)sizeof h + 4ull * ((uint64_t)h.lq + h.lr) && fseek(f, at, SEEK_SET) == 0;
    }
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
    h.version = 2u;
    h.N = N;
    h.lq = (uint32_t)q.size();
    h.lr = (uint32_t)r.size();
    h.sum = ckpt_sum(q, r);
    const std::string tmp = std::string(path) + ".tmp";
    FILE *f = fopen(tmp.c_str(), "wb");
    if (!f) return false;
    bool ok = fwrite(&h, sizeof h, 1, f) == 1 && fwrite(q.data(), 4, q.size(), f) == q.size() &&
              fwrite(r.data(), 4, r.size(), f) == r.size();
    // the data reaches the disk before the name does
    ok = ok && fflush(f) == 0 && fsync(fileno(f)) == 0;
    ok = (fclose(f) == 0) && ok && rename(tmp.c_str(), path) == 0;
    if (!ok) {
        remove(tmp.c_str());
        return false;
    }
    // make the rename itself durable: sync the directory that holds path
    std::string dir(path);
    const size_t slash = dir.find_last_of('/');
    dir = (slash == std::string::npos) ? std::string(".") : (slash == 0 ? std::string("/") : dir.substr(0, slash));
    const int fd = open(dir.c_str(), O_RDONLY | O_DIRECTORY);
    if (fd >= 0) {
        fsync(fd);
        close(fd);
    }
    return true;
}

}  // namespace gpupi
