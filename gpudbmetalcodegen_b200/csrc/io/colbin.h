#pragma once
// ===================================================================
// .colbin v2 reader: the reference's primary on-disk column store
// (src/infra.h:512-782). A file is a 48-byte header (magic "TPCHCB01",
// u32 version = 2, u32 column count, u64 row count, u64 source size, i64
// source mtime, u64 pad), a directory of 32-byte column descriptors (i32
// source field index, u8 type, u8 pad, u16 fixed width, u64 offset, u64
// bytes, u64 pad) and the payloads at 16 KiB-aligned offsets. Types: 0
// int32, 1 float32, 2 date (int32 YYYYMMDD), 3 one-byte char, 4 fixed-width
// chars. The file is memory-mapped read-only; payloads are read in place.
// ===================================================================

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace gpudb {

struct ColbinDesc {
    int32_t columnIndex = 0;
    uint8_t dtype = 0;
    uint16_t fixedWidth = 0;
    uint64_t offset = 0;
    uint64_t sizeBytes = 0;
};

class ColbinFile {
public:
    // Maps and validates `path`; throws std::runtime_error with the reason.
    explicit ColbinFile(const std::string& path);
    ~ColbinFile();
    ColbinFile(const ColbinFile&) = delete;
    ColbinFile& operator=(const ColbinFile&) = delete;

    uint64_t rows() const { return rows_; }
    const std::vector<ColbinDesc>& columns() const { return descs_; }
    // The descriptor of source field `columnIndex`; throws if absent.
    const ColbinDesc& find(int32_t columnIndex) const;
    const unsigned char* payload(const ColbinDesc& d) const { return base_ + d.offset; }
    // Bytes per row of a descriptor's type.
    static size_t width(const ColbinDesc& d);

private:
    const unsigned char* base_ = nullptr;
    size_t size_ = 0;
    uint64_t rows_ = 0;
    std::vector<ColbinDesc> descs_;
};

// Days since 1992-01-01 of a YYYYMMDD date (the configurations' day
// numbers; proleptic Gregorian calendar). Throws on an invalid date.
int32_t colbinDayNumber(int32_t yyyymmdd);

}  // namespace gpudb
