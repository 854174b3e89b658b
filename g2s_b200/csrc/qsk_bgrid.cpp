// G2S .bgrid grids (the serialised DataImage of the G2S data directory):
//   size_t   total size in bytes (this header included)
//   unsigned number of dimensions, then each dimension (x first)
//   unsigned number of variables, then one type per variable (0 continuous, 1 categorical)
//   unsigned encoding (0 float, 1 int, 2 uint)
//   prod(dims) * nvar 32-bit values, variables interleaved
// optionally gzip-compressed (.bgrid.gz).  Same layout and limits as
// G2S include/DataImage.hpp:143-223 (serialize / validateSerializedData) and
// src/DataImage.cpp:35-165 (file access), so files move between both.
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include <zlib.h>

#include "../../include/g2s_b200.h"
#include "qsk_internal.h"

namespace {

constexpr size_t kMaxBytes = size_t(1) << 30;   // DataImage::MaxSerializedBytes
constexpr unsigned kMaxDims = 16;
constexpr unsigned kMaxVars = 4096;

bool ends_with(const std::string &s, const char *suf) {
    size_t n = std::strlen(suf);
    return s.size() >= n && s.compare(s.size() - n, n, suf) == 0;
}

bool read_all(const std::string &path, std::vector<unsigned char> &out) {
    out.clear();
    if (ends_with(path, ".gz")) {
        gzFile f = gzopen(path.c_str(), "rb");
        if (!f) return false;
        unsigned char buf[1 << 16];
        for (;;) {
            int r = gzread(f, buf, sizeof(buf));
            if (r < 0 || out.size() + size_t(r) > kMaxBytes) {
                gzclose(f);
                return false;
            }
            if (r == 0) break;
            out.insert(out.end(), buf, buf + r);
        }
        gzclose(f);
        return true;
    }
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    if (std::fseek(f, 0L, SEEK_END) != 0) {
        std::fclose(f);
        return false;
    }
    long sz = std::ftell(f);
    if (sz < 0 || size_t(sz) > kMaxBytes) {
        std::fclose(f);
        return false;
    }
    std::rewind(f);
    out.resize(size_t(sz));
    bool ok = out.empty() || std::fread(out.data(), 1, out.size(), f) == out.size();
    std::fclose(f);
    return ok;
}

struct Header {
    std::vector<unsigned> dims;
    std::vector<int> types;
    int encoding = 0;
    size_t data_offset = 0;
    size_t values = 0;
};

// the checks of DataImage::validateSerializedData
bool parse(const std::vector<unsigned char> &raw, Header &h) {
    const size_t n = raw.size();
    if (n < sizeof(size_t) + 3 * sizeof(unsigned)) return false;
    size_t full = 0;
    std::memcpy(&full, raw.data(), sizeof(full));
    if (full != n || full > kMaxBytes) return false;
    size_t off = sizeof(size_t);
    auto get = [&](unsigned &v) {
        if (off + sizeof(unsigned) > n) return false;
        std::memcpy(&v, raw.data() + off, sizeof(unsigned));
        off += sizeof(unsigned);
        return true;
    };
    unsigned nd = 0;
    if (!get(nd) || nd == 0 || nd > kMaxDims) return false;
    size_t cells = 1;
    h.dims.resize(nd);
    for (unsigned d = 0; d < nd; ++d) {
        if (!get(h.dims[d]) || h.dims[d] == 0 || cells > std::numeric_limits<size_t>::max() / h.dims[d]) return false;
        cells *= h.dims[d];
    }
    unsigned nv = 0;
    if (!get(nv) || nv == 0 || nv > kMaxVars) return false;
    h.types.resize(nv);
    for (unsigned v = 0; v < nv; ++v) {
        unsigned t = 0;
        if (!get(t) || t > 1) return false;
        h.types[v] = int(t);
    }
    unsigned enc = 0;
    if (!get(enc) || enc > 2) return false;
    h.encoding = int(enc);
    if (cells > kMaxBytes / 4 / nv) return false;
    h.values = cells * nv;
    h.data_offset = off;
    return h.values * 4 == n - off;
}

}  // namespace

extern "C" {

int qsk_bgrid_read(const char *path, int *ndim, unsigned *dims, int *nvar, int *types, int types_capacity,
                   int *encoding, void *data, long long capacity, long long *count) {
    if (!path || !ndim || !dims || !nvar || !encoding || !count) return qsk::set_error(QSK_ERR_ARG, "null argument");
    std::vector<unsigned char> raw;
    if (!read_all(path, raw)) return qsk::set_error(QSK_ERR_ARG, "cannot read %s", path);
    Header h;
    if (!parse(raw, h)) return qsk::set_error(QSK_ERR_ARG, "%s is not a valid .bgrid", path);
    *ndim = int(h.dims.size());
    for (size_t d = 0; d < h.dims.size(); ++d) dims[d] = h.dims[d];
    *nvar = int(h.types.size());
    if (types)
        for (int v = 0; v < int(h.types.size()) && v < types_capacity; ++v) types[v] = h.types[v];
    *encoding = h.encoding;
    *count = (long long)h.values;
    if (data) {
        if (capacity < (long long)h.values)
            return qsk::set_error(QSK_ERR_ARG, "%s holds %zu values, capacity %lld", path, h.values, capacity);
        std::memcpy(data, raw.data() + h.data_offset, h.values * 4);
    }
    return QSK_OK;
}

int qsk_bgrid_write(const char *path, int ndim, const unsigned *dims, int nvar, const int *types, int encoding,
                    const void *data, int compress) {
    if (!path || !dims || !types || !data || ndim < 1 || ndim > int(kMaxDims) || nvar < 1 || nvar > int(kMaxVars) ||
        encoding < 0 || encoding > 2)
        return qsk::set_error(QSK_ERR_ARG, "invalid grid description");
    size_t cells = 1;
    for (int d = 0; d < ndim; ++d) {
        if (dims[d] == 0) return qsk::set_error(QSK_ERR_ARG, "zero dimension");
        cells *= dims[d];
    }
    const size_t full = sizeof(size_t) + sizeof(unsigned) * (1 + size_t(ndim) + 1 + size_t(nvar) + 1) + cells * nvar * 4;
    if (full > kMaxBytes) return qsk::set_error(QSK_ERR_UNSUPPORTED, "grid above the 1 GiB .bgrid limit");
    std::vector<unsigned char> raw(full);
    size_t off = 0;
    auto put = [&](const void *p, size_t b) {
        std::memcpy(raw.data() + off, p, b);
        off += b;
    };
    put(&full, sizeof(full));
    unsigned u = unsigned(ndim);
    put(&u, sizeof(u));
    put(dims, sizeof(unsigned) * ndim);
    u = unsigned(nvar);
    put(&u, sizeof(u));
    for (int v = 0; v < nvar; ++v) {
        u = types[v] ? 1u : 0u;
        put(&u, sizeof(u));
    }
    u = unsigned(encoding);
    put(&u, sizeof(u));
    put(data, cells * nvar * 4);
    if (compress) {
        gzFile f = gzopen(path, "wb");
        if (!f) return qsk::set_error(QSK_ERR_ARG, "cannot write %s", path);
        bool ok = gzwrite(f, raw.data(), unsigned(raw.size())) == int(raw.size());
        ok &= gzclose(f) == Z_OK;
        return ok ? QSK_OK : qsk::set_error(QSK_ERR_ARG, "write to %s failed", path);
    }
    FILE *f = std::fopen(path, "wb");
    if (!f) return qsk::set_error(QSK_ERR_ARG, "cannot write %s", path);
    bool ok = std::fwrite(raw.data(), 1, raw.size(), f) == raw.size();
    ok &= std::fclose(f) == 0;
    return ok ? QSK_OK : qsk::set_error(QSK_ERR_ARG, "write to %s failed", path);
}

}  // extern "C"
