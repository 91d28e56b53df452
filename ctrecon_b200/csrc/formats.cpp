// formats.cpp -- the reference's projection and image files (ProjectionData.m:113-176,
// ReconImage.m:60-117): little-endian doubles, header scalars in the order the MATLAB classes
// write them, the data array, then the 3-entry storage order. Host code only.
#include "internal.h"

#include <cmath>
#include <cstdio>
#include <string>

namespace ctr {
void set_noctx_error(const std::string& m);
}
using namespace ctr;

namespace {

ctrecon_status fail(ctrecon_status c, const std::string& m) {
    set_noctx_error(m);
    return c;
}

// element count of an array whose dimensions are given as doubles (they must be whole,
// non-negative and small enough to address)
bool count_of(const double* dims, int nd, size_t* n) {
    double v = 1.0;
    for (int i = 0; i < nd; ++i) {
        if (!(dims[i] >= 0) || dims[i] != std::floor(dims[i]) || dims[i] > 4.0e15) return false;
        v *= dims[i];
    }
    if (v > 4.0e15) return false;
    *n = (size_t)v;
    return true;
}

bool valid_order(const double* o) {
    bool seen[4] = {false, false, false, false};
    for (int i = 0; i < 3; ++i) {
        if (o[i] != 1 && o[i] != 2 && o[i] != 3) return false;
        seen[(int)o[i]] = true;
    }
    return seen[1] && seen[2] && seen[3];
}

struct File {
    FILE* f = nullptr;
    explicit File(const char* path, const char* mode) { f = std::fopen(path, mode); }
    ~File() { if (f) std::fclose(f); }
};

// header of nh doubles, n data doubles, 3 order doubles; the header is read first, `count`
// gives n from it
template <class Count>
ctrecon_status read_file(const char* path, double* hdr, int nh, Count count, double* data,
                         size_t capacity, double* order, const char* what) {
    if (!path || !hdr) return fail(CTRECON_ERR_INVALID_ARGUMENT, "NULL argument");
    File F(path, "rb");
    if (!F.f) return fail(CTRECON_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
    if (std::fseek(F.f, 0, SEEK_END) != 0) return fail(CTRECON_ERR_INVALID_ARGUMENT, "cannot seek");
    const long size = std::ftell(F.f);
    std::rewind(F.f);
    if (size < (long)(nh * 8) || std::fread(hdr, 8, nh, F.f) != (size_t)nh)
        return fail(CTRECON_ERR_INVALID_ARGUMENT, std::string(what) + ": file shorter than its header");
    size_t n = 0;
    if (!count(hdr, &n))
        return fail(CTRECON_ERR_INVALID_ARGUMENT, std::string(what) + ": bad dimensions in the header");
    if ((size_t)size != (nh + n + 3) * 8)
        return fail(CTRECON_ERR_INVALID_ARGUMENT,
                    std::string(what) + ": file size " + std::to_string(size) +
                        " bytes does not match its header (" +
                        std::to_string((nh + n + 3) * 8) + " expected)");
    if (std::fseek(F.f, (long)((nh + n) * 8), SEEK_SET) != 0 || std::fread(order, 8, 3, F.f) != 3)
        return fail(CTRECON_ERR_INVALID_ARGUMENT, std::string(what) + ": cannot read the storage order");
    if (!valid_order(order))
        return fail(CTRECON_ERR_INVALID_ARGUMENT, std::string(what) + ": storage order is not a permutation of 1 2 3");
    if (data) {
        if (capacity < n)
            return fail(CTRECON_ERR_INVALID_ARGUMENT, std::string(what) + ": data buffer holds " +
                                                          std::to_string(capacity) + " of " +
                                                          std::to_string(n) + " values");
        if (std::fseek(F.f, (long)(nh * 8), SEEK_SET) != 0 || std::fread(data, 8, n, F.f) != n)
            return fail(CTRECON_ERR_INVALID_ARGUMENT, std::string(what) + ": short read");
    }
    return CTRECON_OK;
}

ctrecon_status write_file(const char* path, const double* hdr, int nh, const double* data,
                          size_t n, const double* order, const char* what) {
    if (!path || !hdr || (!data && n)) return fail(CTRECON_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!valid_order(order))
        return fail(CTRECON_ERR_INVALID_ARGUMENT, std::string(what) + ": storage order is not a permutation of 1 2 3");
    File F(path, "wb");
    if (!F.f) return fail(CTRECON_ERR_INVALID_ARGUMENT, std::string("cannot create ") + path);
    if (std::fwrite(hdr, 8, nh, F.f) != (size_t)nh || std::fwrite(data, 8, n, F.f) != n ||
        std::fwrite(order, 8, 3, F.f) != 3)
        return fail(CTRECON_ERR_INVALID_ARGUMENT, std::string(what) + ": short write");
    return CTRECON_OK;
}

constexpr int kProjHeader = 14;  // ProjectionData.m:115-130
constexpr int kImgHeader = 12;   // ReconImage.m:62-76

}  // namespace

extern "C" {

ctrecon_status ctrecon_projfile_read(const char* path, ctrecon_projfile_header* h, double* data,
                                     size_t capacity) {
    if (!h) return fail(CTRECON_ERR_INVALID_ARGUMENT, "NULL argument");
    double hdr[kProjHeader];
    // data count: DetResoU * DetResoV * TotalProjectionNumber (ProjectionData.m:149)
    auto count = [](const double* x, size_t* n) {
        const double d[3] = {x[2], x[3], x[12]};
        return count_of(d, 3, n);
    };
    const ctrecon_status s =
        read_file(path, hdr, kProjHeader, count, data, capacity, h->storage_order, "projection file");
    if (s != CTRECON_OK) return s;
    double* dst[kProjHeader] = {&h->source_to_center, &h->source_to_detector, &h->det_reso_u,
                                &h->det_reso_v, &h->det_pixel_u, &h->det_pixel_v,
                                &h->det_center_u, &h->det_center_v, &h->is_arc,
                                &h->start_angle_deg, &h->start_z, &h->pitch, &h->total_views,
                                &h->views_per_turn};
    for (int i = 0; i < kProjHeader; ++i) *dst[i] = hdr[i];
    return CTRECON_OK;
}

ctrecon_status ctrecon_projfile_write(const char* path, const ctrecon_projfile_header* h,
                                      const double* data) {
    if (!h) return fail(CTRECON_ERR_INVALID_ARGUMENT, "NULL argument");
    const double hdr[kProjHeader] = {h->source_to_center, h->source_to_detector, h->det_reso_u,
                                     h->det_reso_v, h->det_pixel_u, h->det_pixel_v,
                                     h->det_center_u, h->det_center_v, h->is_arc,
                                     h->start_angle_deg, h->start_z, h->pitch, h->total_views,
                                     h->views_per_turn};
    const double d[3] = {h->det_reso_u, h->det_reso_v, h->total_views};
    size_t n = 0;
    if (!count_of(d, 3, &n))
        return fail(CTRECON_ERR_INVALID_ARGUMENT, "projection file: bad dimensions in the header");
    return write_file(path, hdr, kProjHeader, data, n, h->storage_order, "projection file");
}

ctrecon_status ctrecon_imgfile_read(const char* path, ctrecon_imgfile_header* h, double* data,
                                    size_t capacity) {
    if (!h) return fail(CTRECON_ERR_INVALID_ARGUMENT, "NULL argument");
    double hdr[kImgHeader];
    auto count = [](const double* x, size_t* n) { return count_of(x, 3, n); };  // resoX*resoY*resoZ
    const ctrecon_status s =
        read_file(path, hdr, kImgHeader, count, data, capacity, h->storage_order, "image file");
    if (s != CTRECON_OK) return s;
    for (int i = 0; i < 3; ++i) {
        h->reso[i] = hdr[i];
        h->pixel[i] = hdr[3 + i];
        h->ctr_idx[i] = hdr[6 + i];
        h->center[i] = hdr[9 + i];
    }
    return CTRECON_OK;
}

ctrecon_status ctrecon_imgfile_write(const char* path, const ctrecon_imgfile_header* h,
                                     const double* data) {
    if (!h) return fail(CTRECON_ERR_INVALID_ARGUMENT, "NULL argument");
    double hdr[kImgHeader];
    for (int i = 0; i < 3; ++i) {
        hdr[i] = h->reso[i];
        hdr[3 + i] = h->pixel[i];
        hdr[6 + i] = h->ctr_idx[i];
        hdr[9 + i] = h->center[i];
    }
    size_t n = 0;
    if (!count_of(h->reso, 3, &n))
        return fail(CTRECON_ERR_INVALID_ARGUMENT, "image file: bad dimensions in the header");
    return write_file(path, hdr, kImgHeader, data, n, h->storage_order, "image file");
}

}  // extern "C"
