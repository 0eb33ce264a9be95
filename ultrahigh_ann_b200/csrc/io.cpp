// Host-side data files of the path: the versioned importance-probability file
// bound to its representative matrix by SHA-256
// (src/io/importance_probability_io.cpp, include/ultrahigh_ann/io/sha256.hpp)
// and the NPY matrices / label vectors of the transformed datasets
// (src/datasets/representative_query_dataset.cpp:23-309).
//
// SHA-256 follows FIPS 180-4. Its constants are derived here from their
// definition (the first 32 fractional bits of the square roots of the first 8
// primes and of the cube roots of the first 64 primes), computed exactly with
// integer roots.
//
// Probability file layout (little-endian): "UHANNPR2", kind byte (1 = L1,
// 2 = L2), 7 zero bytes, u64 representative count, u64 coordinate count,
// 32-byte SHA-256 of the representative-matrix file, coordinate count x
// binary64 probabilities in [0, 1]; nothing after them.
#include "common.h"

#include <sys/stat.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <limits>
#include <string>
#include <string_view>
#include <vector>

using uha::fail;
using uha::guarded;

namespace {

// ------------------------------------------------------------------ SHA-256

uint64_t integer_root(unsigned __int128 value, int degree)
{
    // largest k with k^degree <= value (k < 2^40 here)
    uint64_t lo = 0;
    uint64_t hi = uint64_t{1} << 40;
    while (lo < hi) {
        const uint64_t mid = lo + (hi - lo + 1) / 2;
        unsigned __int128 pow = 1;
        for (int i = 0; i < degree; ++i) {
            pow *= mid;
        }
        if (pow <= value) {
            lo = mid;
        } else {
            hi = mid - 1;
        }
    }
    return lo;
}

struct Sha256Constants {
    std::array<uint32_t, 64> k{};
    std::array<uint32_t, 8> h{};
    Sha256Constants()
    {
        std::array<uint32_t, 64> primes{};
        uint32_t n = 0;
        for (uint32_t c = 2; n < 64; ++c) {
            bool prime = true;
            for (uint32_t d = 2; d * d <= c; ++d) {
                prime = prime && (c % d != 0);
            }
            if (prime) {
                primes[n++] = c;
            }
        }
        for (int i = 0; i < 64; ++i) {
            // floor(cbrt(p) * 2^32) = floor(cbrt(p * 2^96))
            const unsigned __int128 v = static_cast<unsigned __int128>(primes[i]) << 96;
            k[i] = static_cast<uint32_t>(integer_root(v, 3));
        }
        for (int i = 0; i < 8; ++i) {
            // floor(sqrt(p) * 2^32) = floor(sqrt(p * 2^64))
            const unsigned __int128 v = static_cast<unsigned __int128>(primes[i]) << 64;
            h[i] = static_cast<uint32_t>(integer_root(v, 2));
        }
    }
};

const Sha256Constants& sha_constants()
{
    static const Sha256Constants c;
    return c;
}

inline uint32_t rotr(uint32_t x, int n)
{
    return (x >> n) | (x << (32 - n));
}

class Sha256 {
public:
    Sha256() : state_(sha_constants().h) {}

    void update(const unsigned char* data, size_t size)
    {
        length_ += static_cast<uint64_t>(size);
        while (size > 0) {
            const size_t take = std::min(size, block_.size() - used_);
            std::memcpy(block_.data() + used_, data, take);
            used_ += take;
            data += take;
            size -= take;
            if (used_ == block_.size()) {
                compress(block_.data());
                used_ = 0;
            }
        }
    }

    std::array<uint8_t, 32> finish()
    {
        const uint64_t bits = length_ * 8;
        const unsigned char one = 0x80;
        update(&one, 1);
        const unsigned char zero = 0;
        while (used_ != 56) {
            update(&zero, 1);
        }
        std::array<unsigned char, 8> len{};
        for (int i = 0; i < 8; ++i) {
            len[i] = static_cast<unsigned char>(bits >> (56 - 8 * i));
        }
        update(len.data(), len.size());
        std::array<uint8_t, 32> out{};
        for (int i = 0; i < 8; ++i) {
            for (int b = 0; b < 4; ++b) {
                out[4 * i + b] = static_cast<uint8_t>(state_[i] >> (24 - 8 * b));
            }
        }
        return out;
    }

private:
    void compress(const unsigned char* p)
    {
        const auto& k = sha_constants().k;
        std::array<uint32_t, 64> w{};
        for (int i = 0; i < 16; ++i) {
            w[i] = (uint32_t{p[4 * i]} << 24) | (uint32_t{p[4 * i + 1]} << 16) |
                   (uint32_t{p[4 * i + 2]} << 8) | uint32_t{p[4 * i + 3]};
        }
        for (int i = 16; i < 64; ++i) {
            const uint32_t s0 = rotr(w[i - 15], 7) ^ rotr(w[i - 15], 18) ^ (w[i - 15] >> 3);
            const uint32_t s1 = rotr(w[i - 2], 17) ^ rotr(w[i - 2], 19) ^ (w[i - 2] >> 10);
            w[i] = w[i - 16] + s0 + w[i - 7] + s1;
        }
        uint32_t a = state_[0], b = state_[1], c = state_[2], d = state_[3];
        uint32_t e = state_[4], f = state_[5], g = state_[6], h = state_[7];
        for (int i = 0; i < 64; ++i) {
            const uint32_t S1 = rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25);
            const uint32_t ch = (e & f) ^ (~e & g);
            const uint32_t t1 = h + S1 + ch + k[i] + w[i];
            const uint32_t S0 = rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22);
            const uint32_t maj = (a & b) ^ (a & c) ^ (b & c);
            const uint32_t t2 = S0 + maj;
            h = g;
            g = f;
            f = e;
            e = d + t1;
            d = c;
            c = b;
            b = a;
            a = t1 + t2;
        }
        state_[0] += a;
        state_[1] += b;
        state_[2] += c;
        state_[3] += d;
        state_[4] += e;
        state_[5] += f;
        state_[6] += g;
        state_[7] += h;
    }

    std::array<uint32_t, 8> state_;
    std::array<unsigned char, 64> block_{};
    size_t used_ = 0;
    uint64_t length_ = 0;
};

// ------------------------------------------------------ probability file

constexpr char kMagic[8] = {'U', 'H', 'A', 'N', 'N', 'P', 'R', '2'};

[[noreturn]] void probability_error(const std::string& path, const std::string& message)
{
    fail(UHA_RUNTIME_ERROR, "invalid importance-probability file " + path + ": " + message);
}

void put_u64(std::string& out, uint64_t v)
{
    for (int i = 0; i < 8; ++i) {
        out.push_back(static_cast<char>((v >> (8 * i)) & 0xffu));
    }
}

uint64_t get_u64(const unsigned char* p)
{
    uint64_t v = 0;
    for (int i = 0; i < 8; ++i) {
        v |= uint64_t{p[i]} << (8 * i);
    }
    return v;
}

void check_probabilities(const double* p, uint64_t n, const std::string& path)
{
    for (uint64_t i = 0; i < n; ++i) {
        if (!std::isfinite(p[i]) || p[i] < 0.0 || p[i] > 1.0) {
            probability_error(path, "probabilities must be finite and in [0, 1]");
        }
    }
}

std::vector<unsigned char> read_file(const std::string& path, bool* opened)
{
    std::ifstream in(path, std::ios::binary);
    *opened = static_cast<bool>(in);
    if (!*opened) {
        return {};
    }
    return std::vector<unsigned char>(std::istreambuf_iterator<char>(in),
                                      std::istreambuf_iterator<char>());
}

// --------------------------------------------------------------------- NPY

[[noreturn]] void npy_error(const std::string& path, const std::string& message)
{
    fail(UHA_RUNTIME_ERROR, "cannot load " + path + ": " + message);
}

struct NpyArray {
    std::string descr;
    bool fortran = false;
    std::vector<uint64_t> shape;
    size_t data_offset = 0;
};

size_t field_colon(std::string_view header, std::string_view field, const std::string& path)
{
    const size_t at = header.find(field);
    if (at == std::string_view::npos) {
        npy_error(path, "NPY header has no " + std::string(field));
    }
    const size_t colon = header.find(':', at + field.size());
    if (colon == std::string_view::npos) {
        npy_error(path, "malformed NPY field " + std::string(field));
    }
    return colon;
}

std::string_view trim(std::string_view v)
{
    const size_t first = v.find_first_not_of(" \t");
    if (first == std::string_view::npos) {
        return {};
    }
    return v.substr(first, v.find_last_not_of(" \t") - first + 1);
}

NpyArray parse_npy(const std::vector<unsigned char>& bytes, const std::string& path)
{
    static const unsigned char magic[6] = {0x93, 'N', 'U', 'M', 'P', 'Y'};
    if (bytes.size() < 6) {
        npy_error(path, "truncated while reading NPY magic");
    }
    if (std::memcmp(bytes.data(), magic, 6) != 0) {
        npy_error(path, "invalid NPY magic");
    }
    if (bytes.size() < 8) {
        npy_error(path, "truncated while reading NPY version");
    }
    const unsigned major = bytes[6];
    size_t pos = 8;
    uint64_t header_length = 0;
    if (major == 1) {
        if (bytes.size() < pos + 2) {
            npy_error(path, "truncated while reading NPY header length");
        }
        header_length = uint64_t{bytes[pos]} | (uint64_t{bytes[pos + 1]} << 8);
        pos += 2;
    } else if (major == 2 || major == 3) {
        if (bytes.size() < pos + 4) {
            npy_error(path, "truncated while reading NPY header length");
        }
        header_length = uint64_t{bytes[pos]} | (uint64_t{bytes[pos + 1]} << 8) |
                        (uint64_t{bytes[pos + 2]} << 16) | (uint64_t{bytes[pos + 3]} << 24);
        pos += 4;
    } else {
        npy_error(path, "unsupported NPY format version");
    }
    if (header_length == 0 || header_length > 1024u * 1024u) {
        npy_error(path, "unreasonable NPY header length");
    }
    if (bytes.size() < pos + header_length) {
        npy_error(path, "truncated while reading NPY header");
    }
    const std::string header(reinterpret_cast<const char*>(bytes.data()) + pos,
                             static_cast<size_t>(header_length));
    NpyArray a;
    a.data_offset = pos + static_cast<size_t>(header_length);
    {
        const size_t colon = field_colon(header, "descr", path);
        const size_t quote = header.find_first_of("'\"", colon + 1);
        if (quote == std::string::npos) {
            npy_error(path, "malformed NPY dtype descriptor");
        }
        const size_t end = header.find(header[quote], quote + 1);
        if (end == std::string::npos) {
            npy_error(path, "unterminated NPY dtype descriptor");
        }
        a.descr = header.substr(quote + 1, end - quote - 1);
    }
    {
        const size_t colon = field_colon(header, "fortran_order", path);
        const size_t v = header.find_first_not_of(" \t", colon + 1);
        if (v == std::string::npos) {
            npy_error(path, "malformed NPY fortran_order field");
        }
        if (header.compare(v, 4, "True") == 0) {
            a.fortran = true;
        } else if (header.compare(v, 5, "False") == 0) {
            a.fortran = false;
        } else {
            npy_error(path, "invalid NPY fortran_order value");
        }
    }
    {
        const size_t colon = field_colon(header, "shape", path);
        const size_t open = header.find('(', colon + 1);
        const size_t close = open == std::string::npos ? std::string::npos
                                                        : header.find(')', open + 1);
        if (open == std::string::npos || close == std::string::npos) {
            npy_error(path, "malformed NPY shape field");
        }
        std::string_view contents(header.data() + open + 1, close - open - 1);
        size_t start = 0;
        while (start <= contents.size()) {
            const size_t comma = contents.find(',', start);
            const size_t end = comma == std::string_view::npos ? contents.size() : comma;
            const std::string_view token = trim(contents.substr(start, end - start));
            if (!token.empty()) {
                uint64_t dim = 0;
                for (char ch : token) {
                    if (ch < '0' || ch > '9' ||
                        dim > (std::numeric_limits<uint64_t>::max() - 9) / 10) {
                        npy_error(path, "invalid dimension in NPY shape");
                    }
                    dim = dim * 10 + static_cast<uint64_t>(ch - '0');
                }
                a.shape.push_back(dim);
            }
            if (comma == std::string_view::npos) {
                break;
            }
            start = comma + 1;
        }
        if (a.shape.empty()) {
            npy_error(path, "scalar NPY arrays are not supported");
        }
    }
    return a;
}

uint64_t npy_count(const NpyArray& a, const std::string& path)
{
    uint64_t n = 1;
    for (uint64_t d : a.shape) {
        if (d != 0 && n > std::numeric_limits<uint64_t>::max() / d) {
            npy_error(path, "NPY shape overflows addressable memory");
        }
        n *= d;
    }
    return n;
}

// Payload of an array with dtype `descr` (little-endian) and `elem` bytes
// per element, in C order.
const unsigned char* npy_payload(const std::vector<unsigned char>& bytes, const NpyArray& a,
                                 const char* descr, uint64_t elem, const std::string& path,
                                 uint64_t* count)
{
    if (a.descr != descr) {
        npy_error(path, std::string("expected dtype ") + descr + ", found " + a.descr);
    }
    if (a.fortran) {
        npy_error(path, "Fortran-order arrays are not supported");
    }
    const uint64_t n = npy_count(a, path);
    if (n > std::numeric_limits<uint64_t>::max() / elem) {
        npy_error(path, "NPY payload is too large");
    }
    if (bytes.size() - a.data_offset < n * elem) {
        npy_error(path, "truncated while reading NPY array data");
    }
    if (bytes.size() - a.data_offset != n * elem) {
        npy_error(path, "unexpected trailing data");
    }
    *count = n;
    return bytes.data() + a.data_offset;
}

}  // namespace

extern "C" uha_status uha_sha256(const void* data, uint64_t size, uint8_t* out)
{
    return guarded([&] {
        if (out == nullptr || (data == nullptr && size != 0)) {
            fail(UHA_INVALID_ARGUMENT, "data and output must not be null");
        }
        Sha256 h;
        h.update(static_cast<const unsigned char*>(data), static_cast<size_t>(size));
        const auto d = h.finish();
        std::memcpy(out, d.data(), d.size());
    });
}

extern "C" uha_status uha_sha256_file(const char* path, uint8_t* out)
{
    return guarded([&] {
        if (path == nullptr || out == nullptr) {
            fail(UHA_INVALID_ARGUMENT, "path and output must not be null");
        }
        std::ifstream in(path, std::ios::binary);
        if (!in) {
            fail(UHA_RUNTIME_ERROR, std::string("cannot open file for hashing: ") + path);
        }
        Sha256 h;
        std::vector<char> buf(1 << 20);
        while (in) {
            in.read(buf.data(), static_cast<std::streamsize>(buf.size()));
            const std::streamsize got = in.gcount();
            if (got > 0) {
                h.update(reinterpret_cast<const unsigned char*>(buf.data()),
                         static_cast<size_t>(got));
            }
        }
        if (in.bad()) {
            fail(UHA_RUNTIME_ERROR, std::string("failed while hashing file: ") + path);
        }
        const auto d = h.finish();
        std::memcpy(out, d.data(), d.size());
    });
}

extern "C" uha_status uha_probabilities_save(const char* path, uha_metric kind,
                                             uint64_t representative_count,
                                             const uint8_t* representatives_sha256,
                                             const double* probabilities, uint64_t count)
{
    return guarded([&] {
        if (path == nullptr || representatives_sha256 == nullptr ||
            (probabilities == nullptr && count != 0)) {
            fail(UHA_INVALID_ARGUMENT, "path, digest and probabilities must not be null");
        }
        if (kind != UHA_L1 && kind != UHA_L2) {
            fail(UHA_INVALID_ARGUMENT, "unknown importance-probability kind");
        }
        const std::string p(path);
        check_probabilities(probabilities, count, p);
        std::string out;
        out.reserve(64 + count * 8);
        out.append(kMagic, sizeof(kMagic));
        out.push_back(static_cast<char>(kind == UHA_L1 ? 1 : 2));
        out.append(7, '\0');
        put_u64(out, representative_count);
        put_u64(out, count);
        out.append(reinterpret_cast<const char*>(representatives_sha256), 32);
        for (uint64_t i = 0; i < count; ++i) {
            uint64_t bits = 0;
            std::memcpy(&bits, probabilities + i, sizeof(bits));
            put_u64(out, bits);
        }
        // parent directories, as the reference creates them
        for (size_t slash = p.find('/', 1); slash != std::string::npos;
             slash = p.find('/', slash + 1)) {
            (void)::mkdir(p.substr(0, slash).c_str(), 0777);
        }
        std::ofstream f(p, std::ios::binary | std::ios::trunc);
        if (!f) {
            probability_error(p, "cannot open for writing");
        }
        f.write(out.data(), static_cast<std::streamsize>(out.size()));
        if (!f) {
            probability_error(p, "failed while writing");
        }
    });
}

extern "C" uha_status uha_probabilities_load(const char* path, uha_metric* kind,
                                             uint64_t* representative_count,
                                             uint8_t* representatives_sha256,
                                             double* probabilities, uint64_t capacity,
                                             uint64_t* count)
{
    return guarded([&] {
        if (path == nullptr || count == nullptr) {
            fail(UHA_INVALID_ARGUMENT, "path and count must not be null");
        }
        const std::string p(path);
        bool opened = false;
        const std::vector<unsigned char> b = read_file(p, &opened);
        if (!opened) {
            probability_error(p, "does not exist or cannot be opened");
        }
        size_t pos = 0;
        auto need = [&](size_t n, const char* what) {
            if (b.size() - pos < n) {
                probability_error(p, std::string("truncated while reading ") + what);
            }
        };
        need(8, "magic");
        if (std::memcmp(b.data(), kMagic, 8) != 0) {
            probability_error(p, "wrong magic or unsupported version");
        }
        pos = 8;
        need(1, "probability kind");
        const unsigned raw = b[pos++];
        if (raw != 1 && raw != 2) {
            probability_error(p, "unknown probability kind");
        }
        need(7, "reserved header bytes");
        for (int i = 0; i < 7; ++i) {
            if (b[pos + i] != 0) {
                probability_error(p, "reserved header bytes are not zero");
            }
        }
        pos += 7;
        need(8, "representative count");
        const uint64_t reps = get_u64(b.data() + pos);
        pos += 8;
        need(8, "coordinate count");
        const uint64_t n = get_u64(b.data() + pos);
        pos += 8;
        need(32, "representative-matrix SHA-256");
        const size_t digest_at = pos;
        pos += 32;
        if (n > (b.size() - pos) / 8) {
            probability_error(p, "truncated while reading probability");
        }
        std::vector<double> values(static_cast<size_t>(n));
        for (uint64_t i = 0; i < n; ++i) {
            const uint64_t bits = get_u64(b.data() + pos);
            std::memcpy(&values[i], &bits, sizeof(bits));
            pos += 8;
        }
        if (pos != b.size()) {
            probability_error(p, "unexpected trailing data");
        }
        check_probabilities(values.data(), n, p);
        *count = n;
        if (kind != nullptr) {
            *kind = raw == 1 ? UHA_L1 : UHA_L2;
        }
        if (representative_count != nullptr) {
            *representative_count = reps;
        }
        if (representatives_sha256 != nullptr) {
            std::memcpy(representatives_sha256, b.data() + digest_at, 32);
        }
        if (probabilities != nullptr) {
            if (capacity < n) {
                fail(UHA_LENGTH_ERROR, "probability output is too small");
            }
            std::memcpy(probabilities, values.data(), n * sizeof(double));
        }
    });
}

extern "C" uha_status uha_npy_load_f32(const char* path, float* out, uint64_t capacity,
                                       uint64_t* rows, uint64_t* cols)
{
    return guarded([&] {
        if (path == nullptr || rows == nullptr || cols == nullptr) {
            fail(UHA_INVALID_ARGUMENT, "path and shape outputs must not be null");
        }
        const std::string p(path);
        bool opened = false;
        const std::vector<unsigned char> b = read_file(p, &opened);
        if (!opened) {
            npy_error(p, "file does not exist or cannot be opened");
        }
        const NpyArray a = parse_npy(b, p);
        uint64_t n = 0;
        const unsigned char* data = npy_payload(b, a, "<f4", 4, p, &n);
        if (a.shape.size() != 2) {
            npy_error(p, "expected a two-dimensional matrix");
        }
        for (uint64_t i = 0; i < n; ++i) {
            float v;
            std::memcpy(&v, data + 4 * i, 4);
            if (!std::isfinite(v)) {
                npy_error(p, "matrix contains a non-finite value");
            }
        }
        *rows = a.shape[0];
        *cols = a.shape[1];
        if (out != nullptr) {
            if (capacity < n) {
                fail(UHA_LENGTH_ERROR, "matrix output is too small");
            }
            std::memcpy(out, data, n * 4);
        }
    });
}

extern "C" uha_status uha_npy_load_u16(const char* path, uint64_t* out, uint64_t capacity,
                                       uint64_t* count)
{
    return guarded([&] {
        if (path == nullptr || count == nullptr) {
            fail(UHA_INVALID_ARGUMENT, "path and count must not be null");
        }
        const std::string p(path);
        bool opened = false;
        const std::vector<unsigned char> b = read_file(p, &opened);
        if (!opened) {
            npy_error(p, "file does not exist or cannot be opened");
        }
        const NpyArray a = parse_npy(b, p);
        uint64_t n = 0;
        const unsigned char* data = npy_payload(b, a, "<u2", 2, p, &n);
        if (a.shape.size() != 1) {
            npy_error(p, "expected a one-dimensional label array");
        }
        *count = n;
        if (out != nullptr) {
            if (capacity < n) {
                fail(UHA_LENGTH_ERROR, "label output is too small");
            }
            for (uint64_t i = 0; i < n; ++i) {
                out[i] = uint64_t{data[2 * i]} | (uint64_t{data[2 * i + 1]} << 8);
            }
        }
    });
}
