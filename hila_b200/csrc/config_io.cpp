// Gauge configuration files in HILA's binary format (GaugeField::config_write /
// config_read, gaugefield.h:196-271; Field::write / read, field_io.h:128-330):
//
//   int64 header: 394824242 (gaugefield.h:28), NDIM = 4, sizeof(SU<3,double>) = 144,
//                 Lx, Ly, Lz, Lt
//   then for dir = 0..3: the V links of that direction in lexicographic site order
//   (x fastest), each 3x3 complex double row-major.
//
// The payload is exactly the library's host link layout double[4][V][3][3][2].
// A file whose dimensions divide the lattice's is replicated periodically to fill
// it (field_io.h:261-323).  Host-only; no device work.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "hw_internal.h"

namespace {

constexpr int64_t kConfigFlag = 394824242;
constexpr int64_t kLinkBytes = 18 * sizeof(double);

struct File {
    std::FILE *f = nullptr;
    explicit File(std::FILE *p) : f(p) {}
    ~File() {
        if (f) std::fclose(f);
    }
};

// header -> dims; HW_OK or HW_ERR_INVALID with the reference's messages (gaugefield.h:224-259)
int read_header(std::FILE *f, const char *path, int64_t dims[4]) {
    int64_t h[7];
    if (std::fread(h, sizeof(int64_t), 7, f) != 7) {
        hw::set_error("CONFIG ERROR in file %s: header too short", path);
        return HW_ERR_INVALID;
    }
    if (h[0] != kConfigFlag) {
        hw::set_error("CONFIG ERROR in file %s: wrong id, should be %lld is %lld", path, (long long)kConfigFlag,
                      (long long)h[0]);
        return HW_ERR_INVALID;
    }
    if (h[1] != 4) {
        hw::set_error("CONFIG ERROR in file %s: wrong dimensionality, should be 4 is %lld", path, (long long)h[1]);
        return HW_ERR_INVALID;
    }
    if (h[2] != kLinkBytes) {
        hw::set_error("CONFIG ERROR in file %s: wrong size of field element, should be %lld is %lld", path,
                      (long long)kLinkBytes, (long long)h[2]);
        return HW_ERR_INVALID;
    }
    for (int d = 0; d < 4; d++) {
        if (h[3 + d] < 1 || h[3 + d] > (1 << 20)) {
            hw::set_error("CONFIG ERROR in file %s: bad lattice dimension %d: %lld", path, d, (long long)h[3 + d]);
            return HW_ERR_INVALID;
        }
        dims[d] = h[3 + d];
    }
    return HW_OK;
}

}  // namespace

extern "C" {

int hw_gauge_config_dims(const char *path, int dims[4]) {
    HW_CHECK_ARG(path && dims, "null argument");
    File f(std::fopen(path, "rb"));
    HW_CHECK_ARG(f.f, "cannot open %s", path);
    int64_t d64[4];
    int rc = read_header(f.f, path, d64);
    if (rc != HW_OK) return rc;
    for (int d = 0; d < 4; d++) dims[d] = (int)d64[d];
    return HW_OK;
}

int hw_gauge_config_write(const char *path, const int dims[4], const double *links) {
    HW_CHECK_ARG(path && dims && links, "null argument");
    int64_t V = 1;
    for (int d = 0; d < 4; d++) {
        HW_CHECK_ARG(dims[d] >= 1, "bad lattice dimension %d", dims[d]);
        V *= dims[d];
    }
    File f(std::fopen(path, "wb"));
    HW_CHECK_ARG(f.f, "cannot open %s for writing", path);
    const int64_t h[7] = {kConfigFlag, 4, kLinkBytes, dims[0], dims[1], dims[2], dims[3]};
    bool ok = std::fwrite(h, sizeof(int64_t), 7, f.f) == 7;
    ok = ok && std::fwrite(links, (size_t)kLinkBytes, (size_t)(4 * V), f.f) == (size_t)(4 * V);
    ok = (std::fflush(f.f) == 0) && ok;
    if (!ok) {
        hw::set_error("write to %s failed", path);
        return HW_ERR_INVALID;
    }
    return HW_OK;
}

int hw_gauge_config_read(const char *path, const int dims[4], double *links) {
    HW_CHECK_ARG(path && dims && links, "null argument");
    File f(std::fopen(path, "rb"));
    HW_CHECK_ARG(f.f, "cannot open %s", path);
    int64_t in[4];
    int rc = read_header(f.f, path, in);
    if (rc != HW_OK) return rc;
    int64_t V = 1, Vin = 1;
    for (int d = 0; d < 4; d++) {
        if (dims[d] < 1 || dims[d] % in[d] != 0) {
            hw::set_error("CONFIG ERROR in file %s: incorrect lattice dimension %d is %lld should be (or divide) %d",
                          path, d, (long long)in[d], dims[d]);
            return HW_ERR_INVALID;
        }
        V *= dims[d];
        Vin *= in[d];
    }
    std::vector<double> buf((size_t)Vin * 18);
    for (int dir = 0; dir < 4; dir++) {
        if (std::fread(buf.data(), (size_t)kLinkBytes, (size_t)Vin, f.f) != (size_t)Vin) {
            hw::set_error("CONFIG ERROR in file %s: file ends inside direction %d", path, dir);
            return HW_ERR_INVALID;
        }
        double *dst = links + (size_t)dir * V * 18;
        // every site of the lattice takes the file's site at its coordinates modulo the file's size
        for (int64_t t = 0; t < dims[3]; t++)
            for (int64_t z = 0; z < dims[2]; z++)
                for (int64_t y = 0; y < dims[1]; y++)
                    for (int64_t x = 0; x < dims[0]; x++) {
                        const int64_t s = x + dims[0] * (y + dims[1] * (z + dims[2] * t));
                        const int64_t r = x % in[0] + in[0] * (y % in[1] + in[1] * (z % in[2] + in[2] * (t % in[3])));
                        std::memcpy(dst + s * 18, buf.data() + r * 18, (size_t)kLinkBytes);
                    }
    }
    return HW_OK;
}

}  // extern "C"
