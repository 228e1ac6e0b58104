// formats.cu -- graph files on the host: the reference's 772-byte records to the
// BANG / DiskANN disk layout that scripts/bang-preprocess.py:37-72 writes.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/vann.h"
#include "kernels.h"

namespace vann {

// records: n x (4 * dim + 4 + 4 * degree) bytes, modified in place (ids sorted)
vann_status write_bang(std::vector<unsigned char>& records, uint64_t n, uint32_t dim, uint32_t degree,
                       uint32_t medoid, const char* out_prefix) {
    const size_t rec = 4ull * dim + 4 + 4ull * degree;
    for (uint64_t i = 0; i < n; ++i) {
        unsigned char* r = records.data() + i * rec;
        uint32_t       d = 0;
        memcpy(&d, r + 4ull * dim, 4);
        if (d == 0 || d > degree) {
            set_last_error(("node " + std::to_string(i) + " has " + std::to_string(d) +
                            " neighbours; the disk layout needs 1..degree")
                               .c_str());
            return VANN_ERR_STATE;
        }
        std::vector<uint32_t> ids(d);
        memcpy(ids.data(), r + 4ull * dim + 4, 4ull * d);
        std::sort(ids.begin(), ids.end());
        memcpy(r + 4ull * dim + 4, ids.data(), 4ull * d);
    }
    const std::string index_path = std::string(out_prefix) + "_disk.bin";
    const std::string meta_path  = std::string(out_prefix) + "_disk_metadata.bin";
    FILE*             f          = fopen(index_path.c_str(), "wb");
    if (!f) {
        set_last_error(("cannot open " + index_path).c_str());
        return VANN_ERR_IO;
    }
    const size_t put = n ? fwrite(records.data(), rec, n, f) : 0;
    fclose(f);
    if (put != n) {
        set_last_error("short write");
        return VANN_ERR_IO;
    }
    // u64 medoid, u64 record bytes, u32 data type (2: float), u32 dim, u32 degree, u32 n
    unsigned char  meta[32];
    const uint64_t m64 = medoid, rec64 = rec;
    const uint32_t dtype = 2, n32 = (uint32_t)n;
    memcpy(meta, &m64, 8);
    memcpy(meta + 8, &rec64, 8);
    memcpy(meta + 16, &dtype, 4);
    memcpy(meta + 20, &dim, 4);
    memcpy(meta + 24, &degree, 4);
    memcpy(meta + 28, &n32, 4);
    f = fopen(meta_path.c_str(), "wb");
    if (!f) {
        set_last_error(("cannot open " + meta_path).c_str());
        return VANN_ERR_IO;
    }
    const size_t mput = fwrite(meta, 1, sizeof(meta), f);
    fclose(f);
    if (mput != sizeof(meta)) {
        set_last_error("short write");
        return VANN_ERR_IO;
    }
    return VANN_OK;
}

}  // namespace vann

extern "C" vann_status vann_convert_graph_file(const char* in_path, uint64_t n, uint32_t dim, uint32_t degree,
                                               uint32_t medoid, const char* out_prefix) {
    if (!in_path || !out_prefix || dim == 0 || degree == 0 || n >= 0xFFFFFFFFull) {
        vann::set_last_error("bad argument");
        return VANN_ERR_INVALID;
    }
    const size_t rec = 4ull * dim + 4 + 4ull * degree;
    FILE*        f   = fopen(in_path, "rb");
    if (!f) {
        vann::set_last_error((std::string("cannot open ") + in_path).c_str());
        return VANN_ERR_IO;
    }
    std::vector<unsigned char> buf(rec * n);
    const size_t               got = n ? fread(buf.data(), rec, n, f) : 0;
    fclose(f);
    if (got != n) {
        vann::set_last_error("short read");
        return VANN_ERR_IO;
    }
    return vann::write_bang(buf, n, dim, degree, medoid, out_prefix);
}
