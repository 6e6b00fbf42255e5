#include "colbin.h"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstring>
#include <stdexcept>

namespace gpudb {

namespace {
constexpr char kMagic[8] = {'T', 'P', 'C', 'H', 'C', 'B', '0', '1'};
constexpr uint32_t kVersion = 2;
constexpr size_t kHeaderBytes = 48;
constexpr size_t kDescBytes = 32;

template <typename T>
T readAt(const unsigned char* p, size_t off) {
    T v;
    std::memcpy(&v, p + off, sizeof(T));
    return v;
}

// Days from 1970-01-01 of a proleptic Gregorian date (H. Hinnant's
// published days-from-civil method: 400-year eras of 146097 days, years
// starting in March so the leap day is last).
long long daysFromCivil(long long y, unsigned m, unsigned d) {
    y -= m <= 2;
    const long long era = (y >= 0 ? y : y - 399) / 400;
    const unsigned yoe = (unsigned)(y - era * 400);
    const unsigned doy = (153 * (m + (m > 2 ? -3 : 9)) + 2) / 5 + d - 1;
    const unsigned doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
    return era * 146097 + (long long)doe - 719468;
}
}  // namespace

ColbinFile::ColbinFile(const std::string& path) {
    const int fd = ::open(path.c_str(), O_RDONLY);
    if (fd < 0) throw std::runtime_error("colbin: cannot open " + path);
    struct stat st {};
    if (::fstat(fd, &st) != 0) {
        ::close(fd);
        throw std::runtime_error("colbin: cannot stat " + path);
    }
    size_ = (size_t)st.st_size;
    if (size_ < kHeaderBytes) {
        ::close(fd);
        throw std::runtime_error("colbin: " + path + " is shorter than its header");
    }
    void* m = ::mmap(nullptr, size_, PROT_READ, MAP_PRIVATE, fd, 0);
    ::close(fd);
    if (m == MAP_FAILED) throw std::runtime_error("colbin: cannot map " + path);
    base_ = (const unsigned char*)m;
    try {
        if (std::memcmp(base_, kMagic, 8) != 0) throw std::runtime_error("colbin: bad magic in " + path);
        const uint32_t version = readAt<uint32_t>(base_, 8);
        if (version != kVersion)
            throw std::runtime_error("colbin: version " + std::to_string(version) + " in " + path + ", expected 2");
        const uint32_t ncols = readAt<uint32_t>(base_, 12);
        rows_ = readAt<uint64_t>(base_, 16);
        if (kHeaderBytes + (size_t)ncols * kDescBytes > size_)
            throw std::runtime_error("colbin: column directory beyond the end of " + path);
        for (uint32_t i = 0; i < ncols; i++) {
            const size_t o = kHeaderBytes + (size_t)i * kDescBytes;
            ColbinDesc d;
            d.columnIndex = readAt<int32_t>(base_, o);
            d.dtype = readAt<uint8_t>(base_, o + 4);
            d.fixedWidth = readAt<uint16_t>(base_, o + 6);
            d.offset = readAt<uint64_t>(base_, o + 8);
            d.sizeBytes = readAt<uint64_t>(base_, o + 16);
            if (d.dtype > 4) throw std::runtime_error("colbin: unknown column type " + std::to_string(d.dtype));
            if (d.offset > size_ || d.sizeBytes > size_ - d.offset)
                throw std::runtime_error("colbin: payload of column " + std::to_string(d.columnIndex) +
                                         " beyond the end of " + path);
            // rows x width must not wrap: a huge row count with a tiny
            // payload would otherwise pass the size check below
            const uint64_t w = width(d);
            if ((w == 0 && rows_ != 0) || (w != 0 && rows_ > (uint64_t)size_ / w))
                throw std::runtime_error("colbin: " + std::to_string(rows_) + " rows of column " +
                                         std::to_string(d.columnIndex) + " cannot fit in " + path);
            if (d.sizeBytes != rows_ * w)
                throw std::runtime_error("colbin: column " + std::to_string(d.columnIndex) + " holds " +
                                         std::to_string(d.sizeBytes) + " bytes, not rows x width");
            descs_.push_back(d);
        }
    } catch (...) {
        ::munmap((void*)base_, size_);
        base_ = nullptr;
        throw;
    }
}

ColbinFile::~ColbinFile() {
    if (base_) ::munmap((void*)base_, size_);
}

const ColbinDesc& ColbinFile::find(int32_t columnIndex) const {
    for (const auto& d : descs_)
        if (d.columnIndex == columnIndex) return d;
    throw std::runtime_error("colbin: no column with source index " + std::to_string(columnIndex));
}

size_t ColbinFile::width(const ColbinDesc& d) {
    switch (d.dtype) {
        case 0:
        case 1:
        case 2: return 4;
        case 3: return 1;
        default: return d.fixedWidth;
    }
}

int32_t colbinDayNumber(int32_t v) {
    const int y = v / 10000, m = (v / 100) % 100, d = v % 100;
    static const int mdays[13] = {0, 31, 29, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31};
    if (v <= 0 || m < 1 || m > 12 || d < 1 || d > mdays[m])
        throw std::runtime_error("colbin: invalid YYYYMMDD date " + std::to_string(v));
    const bool leap = (y % 4 == 0 && y % 100 != 0) || y % 400 == 0;
    if (m == 2 && d == 29 && !leap) throw std::runtime_error("colbin: invalid YYYYMMDD date " + std::to_string(v));
    return (int32_t)(daysFromCivil(y, (unsigned)m, (unsigned)d) - daysFromCivil(1992, 1, 1));
}

}  // namespace gpudb
