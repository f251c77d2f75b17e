// NRRD files of projections straight from and into device memory.
//
// Reference (modules/src/io/nrrd/nrrdfileio.tpp): the header is the magic line
// "NRRD000<v>", then lines that are comments ("#..."), key-value pairs
// ("key:=value") or fields ("field: description"), ended by an empty line
// (metaInfo, :20-105; parseField, :352-450).  NrrdFileIO::writeHeader
// (:252-337) with the meta information of BaseTypeIO::write(ProjectionData)
// (io/basetypeio.tpp:342-362) writes projections as
//   NRRD0004 / type: float / dimension: 4 / sizes: C R M V /
//   labels: "num channel" "num row" "num det module" "num proj" /
//   encoding: raw / endian: little / type hint:=projection data / (empty line)
// followed by the raw data, channel fastest.  The data moves through the same
// pinned double-buffered staging as DEN files.
#include "ctlcu.h"
#include "internal.cuh"

#include <cctype>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <vector>

namespace ctlcu {

namespace {

std::string trim(const std::string& s)
{
    size_t a = 0, b = s.size();
    while (a < b && std::isspace((unsigned char)s[a]))
        ++a;
    while (b > a && std::isspace((unsigned char)s[b - 1]))
        --b;
    return s.substr(a, b - a);
}

// Bytes per element of an NRRD type name, 0 if unknown; is_float for float/double
uint32_t type_bytes(const std::string& t, bool& is_float)
{
    static const struct {
        const char* name;
        uint32_t bytes;
        bool fp;
    } table[] = {
        { "int8", 1, false },   { "signed char", 1, false },  { "int8_t", 1, false },
        { "uint8", 1, false },  { "uchar", 1, false },        { "unsigned char", 1, false },
        { "uint8_t", 1, false }, { "int16", 2, false },       { "short", 2, false },
        { "int16_t", 2, false }, { "uint16", 2, false },      { "ushort", 2, false },
        { "unsigned short", 2, false }, { "uint16_t", 2, false }, { "int32", 4, false },
        { "int", 4, false },    { "int32_t", 4, false },      { "uint32", 4, false },
        { "uint", 4, false },   { "unsigned int", 4, false }, { "uint32_t", 4, false },
        { "int64", 8, false },  { "longlong", 8, false },     { "int64_t", 8, false },
        { "uint64", 8, false }, { "ulonglong", 8, false },    { "uint64_t", 8, false },
        { "float", 4, true },   { "double", 8, true },
    };
    for (const auto& e : table)
        if (t == e.name) {
            is_float = e.fp;
            return e.bytes;
        }
    return 0;
}

}  // namespace

int nrrd_header(const char* path, NrrdHeader& h, std::string& msg)
{
    FILE* f = std::fopen(path, "rb");
    if (!f) {
        msg = std::string("cannot open ") + path;
        return CTLCU_ERR_INVALID_ARGUMENT;
    }
    auto read_line = [&](std::string& line) {
        line.clear();
        int c;
        while ((c = std::fgetc(f)) != EOF) {
            line.push_back((char)c);
            if (c == '\n')
                return true;
        }
        return !line.empty();
    };
    auto bad = [&](const std::string& why) {
        std::fclose(f);
        msg = why;
        return CTLCU_ERR_INVALID_ARGUMENT;
    };
    std::string line;
    if (!read_line(line) || line.compare(0, 7, "NRRD000") != 0 || line.size() < 8 ||
        !std::isdigit((unsigned char)line[7]))
        return bad("no valid nrrd file: the magic first line is missing");
    h = NrrdHeader{};
    h.version = (uint32_t)(line[7] - '0');
    bool have_type = false, raw = true, little = true, have_sizes = false;
    while (true) {
        if (!read_line(line))
            return bad("the header has no terminating empty line");
        if (line == "\n")
            break;  // end of header
        if (line[0] == '#')
            continue;  // comment
        const size_t kv = line.find(":=");
        const size_t fd = line.find(": ");
        if (kv != std::string::npos && (fd == std::string::npos || kv < fd))
            continue;  // key-value pair
        if (fd == std::string::npos || fd == 0)
            return bad("invalid header entry: " + trim(line));
        std::string field = trim(line.substr(0, fd)), desc = trim(line.substr(fd + 2));
        for (auto& c : field)
            c = (char)std::tolower((unsigned char)c);
        if (field == "dimension") {
            if (h.n_dims)
                return bad("dimension given twice");
            const long d = std::strtol(desc.c_str(), nullptr, 10);
            if (d < 1 || d > 4)
                return bad("dimension must lie in 1..4");
            h.n_dims = (uint32_t)d;
        } else if (field == "sizes") {
            if (!h.n_dims || have_sizes)
                return bad("sizes before dimension, or given twice");
            std::istringstream is(desc);
            uint32_t k = 0;
            unsigned long long v;
            while (is >> v) {
                if (k >= 4 || v == 0 || v > 0xFFFFFFFFull)
                    return bad("invalid sizes");
                h.sizes[k++] = (uint32_t)v;
            }
            if (k != h.n_dims)
                return bad("the number of sizes differs from the dimension");
            have_sizes = true;
        } else if (field == "type") {
            if (have_type)
                return bad("type given twice");
            h.elem = type_bytes(desc, h.is_float);
            if (!h.elem)
                return bad("unknown type " + desc);
            have_type = true;
        } else if (field == "encoding") {
            raw = desc == "raw";
        } else if (field == "endian") {
            little = desc == "little";
        }
        // other fields (labels, spacings, space origin, ...) do not change the data layout
    }
    h.offset = (uint64_t)std::ftell(f);
    std::fclose(f);
    if (!have_type || !have_sizes) {
        msg = "type or sizes missing";
        return CTLCU_ERR_INVALID_ARGUMENT;
    }
    if (!raw || !little) {
        msg = "only raw little-endian data is supported";
        return CTLCU_ERR_INVALID_ARGUMENT;
    }
    return CTLCU_OK;
}

int nrrd_write_projections(const char* path, const float* data, uint32_t views, uint32_t modules, uint32_t rows,
                           uint32_t channels, cudaStream_t st, DenStaging* stage, std::string& msg)
{
    if (!views || !modules || !rows || !channels) {
        msg = "empty data";
        return CTLCU_ERR_INVALID_ARGUMENT;
    }
    FILE* f = std::fopen(path, "wb");
    if (!f) {
        msg = std::string("cannot open ") + path + " for writing";
        return CTLCU_ERR_INVALID_ARGUMENT;
    }
    std::ostringstream hd;
    hd << "NRRD0004\n"
       << "type: float\n"
       << "dimension: 4\n"
       << "sizes: " << channels << ' ' << rows << ' ' << modules << ' ' << views << '\n'
       << "labels: \"num channel\" \"num row\" \"num det module\" \"num proj\"\n"
       << "encoding: raw\n"
       << "endian: little\n"
       << "type hint:=projection data\n"
       << '\n';
    const std::string head = hd.str();
    const size_t total = (size_t)views * modules * rows * channels * sizeof(float);
    int r = std::fwrite(head.data(), 1, head.size(), f) == head.size()
                ? file_write_data(f, data, total, st, stage, msg)
                : CTLCU_ERR_INVALID_ARGUMENT;
    const bool closed = std::fclose(f) == 0;
    if (r == CTLCU_OK && !closed)
        r = CTLCU_ERR_INVALID_ARGUMENT;
    if (r == CTLCU_ERR_INVALID_ARGUMENT && msg.empty())
        msg = std::string("writing ") + path + " failed";
    return r;
}

int nrrd_read(const char* path, void* data, uint64_t capacity, cudaStream_t st, DenStaging* stage, std::string& msg)
{
    NrrdHeader h;
    int r = nrrd_header(path, h, msg);
    if (r)
        return r;
    uint64_t total = h.elem;
    for (uint32_t k = 0; k < h.n_dims; ++k)
        total *= h.sizes[k];
    if (total > capacity) {
        msg = "destination smaller than the data";
        return CTLCU_ERR_INVALID_ARGUMENT;
    }
    FILE* f = std::fopen(path, "rb");
    if (!f) {
        msg = std::string("cannot open ") + path;
        return CTLCU_ERR_INVALID_ARGUMENT;
    }
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    if (size < 0 || (uint64_t)size < h.offset + total || std::fseek(f, (long)h.offset, SEEK_SET) != 0) {
        std::fclose(f);
        msg = "raw data size of the file does not fit the sizes in the header";
        return CTLCU_ERR_INVALID_ARGUMENT;
    }
    r = file_read_data(f, data, total, st, stage, msg);
    std::fclose(f);
    if (r == CTLCU_ERR_INVALID_ARGUMENT && msg.empty())
        msg = std::string("reading ") + path + " failed";
    return r;
}

}  // namespace ctlcu
