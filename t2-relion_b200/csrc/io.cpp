// On-disk formats of real data: MRC image stacks and STAR metadata (host code).
//
// MRC (the reference's reader and writer: src/rwMRC.h): the 1024-byte header
// (+ nsymbt bytes of extended header) of MRC2014; nx, ny, nz (a stack of nz
// images), mode 0 (signed 8-bit, as the reference since 3.1), 1 (int16), 2
// (float32), 6 (uint16), 12 (IEEE half); a header whose mode or nx reads as
// larger than 2^16 is byte-swapped, data included (src/rwMRC.h:159-172); the
// pixel size is cella.x / mx (:252-253).  Written files are mode 2, little
// endian, machine stamp 0x44 0x41.
//
// STAR (the reference's parser: MetaDataTable::readStar, readStarLoop,
// readStarList, src/metadata_table.cpp:959-1262, and nextTokenInSTAR,
// src/strings.cpp:588-660): data_<name> blocks holding either label-value
// pairs ("_rlnLabel value") or a loop_ (label lines "_rlnLabel #n", then one
// row per line up to an empty line); '#' starts a comment outside a token;
// tokens may be quoted with ' or ".  Unknown labels are kept.  A loop also
// ends at the next data_ or loop_ line (the reference requires the empty line).
#include "../../include/t2b.h"

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace t2b {
void set_error(const std::string& msg);
}

namespace {

struct IoError {
    int code;
    std::string msg;
};

template <typename F>
int io_guarded(F&& f)
{
    try {
        f();
        return T2B_OK;
    } catch (const IoError& e) {
        t2b::set_error(e.msg);
        return e.code;
    } catch (const std::bad_alloc&) {
        t2b::set_error("host allocation failed");
        return T2B_ERR_NOMEM;
    } catch (const std::exception& e) {
        t2b::set_error(e.what());
        return T2B_ERR_ARG;
    }
}

// ---------------------------------------------------------------- MRC
struct MrcHeader {
    int32_t nx, ny, nz, mode;
    int32_t nxstart, nystart, nzstart;
    int32_t mx, my, mz;
    float cella[3], cellb[3];
    int32_t mapc, mapr, maps;
    float dmin, dmax, dmean;
    int32_t ispg, nsymbt;
    int32_t extra[25];
    float origin[3];
    char map[4];
    unsigned char machst[4];
    float rms;
    int32_t nlabl;
    char labels[10][80];
};
static_assert(sizeof(MrcHeader) == 1024, "MRC header size");

void swap4(void* p, size_t n)
{
    unsigned char* b = static_cast<unsigned char*>(p);
    for (size_t i = 0; i + 3 < n; i += 4) {
        std::swap(b[i], b[i + 3]);
        std::swap(b[i + 1], b[i + 2]);
    }
}

struct MrcFile {
    MrcHeader h{};
    bool swap = false;
    size_t elem = 4;
    FILE* f = nullptr;
    ~MrcFile()
    {
        if (f) std::fclose(f);
    }
};

void mrc_open(const char* path, MrcFile& m)
{
    if (!path) throw IoError{T2B_ERR_ARG, "null path"};
    m.f = std::fopen(path, "rb");
    if (!m.f) throw IoError{T2B_ERR_ARG, std::string("cannot open ") + path + ": " + std::strerror(errno)};
    if (std::fread(&m.h, sizeof(MrcHeader), 1, m.f) != 1) throw IoError{T2B_ERR_ARG, std::string("short MRC header: ") + path};
    const int trig = 1 << 16;
    if (std::abs(m.h.mode) > trig || std::abs(m.h.nx) > trig) {
        m.swap = true;
        swap4(&m.h, 1024 - 800);   // the labels are text
    }
    switch (m.h.mode) {
    case 0: m.elem = 1; break;
    case 1: case 6: case 12: m.elem = 2; break;
    case 2: m.elem = 4; break;
    default:
        throw IoError{T2B_ERR_UNSUPPORTED, "unsupported MRC mode " + std::to_string(m.h.mode) + " in " + path};
    }
    if (m.h.nx <= 0 || m.h.ny <= 0 || m.h.nz <= 0 || m.h.nsymbt < 0)
        throw IoError{T2B_ERR_ARG, std::string("bad MRC dimensions in ") + path};
}

// IEEE 754 binary16 -> binary32 (sign, 5-bit exponent with bias 15, 10-bit fraction)
float half_to_float(uint16_t v)
{
    const uint32_t sign = (uint32_t)(v >> 15) << 31;
    const int e = (v >> 10) & 0x1f;
    const uint32_t frac = v & 0x3ff;
    uint32_t bits;
    if (e == 0) {
        if (frac == 0) {
            bits = sign;
        } else {                      // subnormal: frac * 2^-24
            const float x = std::ldexp((float)frac, -24);
            std::memcpy(&bits, &x, 4);
            bits |= sign;
        }
    } else if (e == 31) {
        bits = sign | 0x7f800000u | (frac << 13);
    } else {
        bits = sign | ((uint32_t)(e - 15 + 127) << 23) | (frac << 13);
    }
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

// ---------------------------------------------------------------- STAR
bool next_token(const std::string& s, size_t& i, std::string& out)
{
    const size_t n = s.size();
    while (i < n && (s[i] == ' ' || s[i] == '\t' || s[i] == '\r' || s[i] == '\n')) ++i;
    if (i >= n || s[i] == '#') return false;
    if (s[i] == '\'' || s[i] == '"') {
        const char q = s[i];
        size_t j = i + 1;
        while (j < n) {
            if (s[j] == q && (j + 1 == n || s[j + 1] == ' ' || s[j + 1] == '\t')) break;
            ++j;
        }
        if (j < n) {
            out = s.substr(i + 1, j - i - 1);
            i = j + 1;
            return true;
        }
        // no closing quote: the token runs to the next blank, quote included
    }
    size_t j = i;
    while (j < n && s[j] != ' ' && s[j] != '\t' && s[j] != '\r' && s[j] != '\n') ++j;
    out = s.substr(i, j - i);
    i = j;
    return true;
}

bool blank(const std::string& s)
{
    for (char ch : s)
        if (ch != ' ' && ch != '\t' && ch != '\r' && ch != '\n') return false;
    return true;
}

}  // namespace

struct t2b_star {
    std::string name;
    std::vector<std::string> labels;
    std::vector<std::vector<std::string>> rows;
    int column(const char* label) const
    {
        if (!label) return -1;
        std::string l = label;
        if (!l.empty() && l[0] == '_') l = l.substr(1);
        for (size_t c = 0; c < labels.size(); ++c)
            if (labels[c] == l) return (int)c;
        return -1;
    }
};

namespace {

void star_parse(std::istream& in, const std::string& want, t2b_star& t)
{
    std::string line;
    bool found = false;
    while (std::getline(in, line)) {
        std::string tok;
        size_t i = 0;
        if (!next_token(line, i, tok)) continue;
        if (tok.compare(0, 5, "data_") == 0) {
            if (want.empty() || tok.substr(5) == want) {
                t.name = tok.substr(5);
                found = true;
                break;
            }
        }
    }
    if (!found) throw IoError{T2B_ERR_ARG, want.empty() ? "no data block" : "no data block data_" + want};
    // the block: a list of label-value pairs, or a loop
    std::streampos after_header = in.tellg();
    bool loop = false;
    while (std::getline(in, line)) {
        std::string tok;
        size_t i = 0;
        if (!next_token(line, i, tok)) continue;
        if (tok == "loop_") loop = true;
        break;
    }
    if (!loop) {
        in.clear();
        in.seekg(after_header);
        std::vector<std::string> row;
        while (std::getline(in, line)) {
            std::string tok, val;
            size_t i = 0;
            if (!next_token(line, i, tok)) continue;
            if (tok.compare(0, 5, "data_") == 0 || tok == "loop_") break;
            if (tok[0] != '_') continue;
            if (!next_token(line, i, val)) throw IoError{T2B_ERR_ARG, "STAR: no value after " + tok};
            t.labels.push_back(tok.substr(1));
            row.push_back(val);
        }
        if (!t.labels.empty()) t.rows.push_back(row);
        return;
    }
    // loop_: label lines, then rows up to an empty line (or the next block)
    std::string pending;
    bool have_pending = false;
    while (std::getline(in, line)) {
        std::string tok;
        size_t i = 0;
        if (!next_token(line, i, tok)) {
            if (blank(line) && !t.labels.empty()) return;   // a loop without rows
            continue;
        }
        if (tok[0] == '_') {
            t.labels.push_back(tok.substr(1));
            continue;
        }
        pending = line;
        have_pending = true;
        break;
    }
    const size_t nc = t.labels.size();
    while (have_pending || std::getline(in, line)) {
        if (have_pending) {
            line = pending;
            have_pending = false;
        }
        if (blank(line)) break;
        std::vector<std::string> row;
        std::string tok;
        size_t i = 0;
        while (next_token(line, i, tok)) row.push_back(tok);
        if (row.empty()) continue;                          // a comment line
        if (row[0].compare(0, 5, "data_") == 0 || row[0] == "loop_") break;
        if (row.size() != nc)
            throw IoError{T2B_ERR_ARG, "STAR: a row has " + std::to_string(row.size()) + " values for " +
                                           std::to_string(nc) + " labels"};
        t.rows.push_back(std::move(row));
    }
}

}  // namespace

extern "C" {

int t2b_mrc_info(const char* path, int* nx, int* ny, int* nz, int* mode, double* pixel_size)
{
    return io_guarded([&] {
        MrcFile m;
        mrc_open(path, m);
        if (nx) *nx = m.h.nx;
        if (ny) *ny = m.h.ny;
        if (nz) *nz = m.h.nz;
        if (mode) *mode = m.h.mode;
        if (pixel_size) *pixel_size = (m.h.mx && m.h.cella[0] != 0.f) ? (double)m.h.cella[0] / m.h.mx : 0.;
    });
}

int t2b_mrc_read(const char* path, long long first, long long count, float* out)
{
    return io_guarded([&] {
        if (!out) throw IoError{T2B_ERR_ARG, "null output"};
        MrcFile m;
        mrc_open(path, m);
        if (first < 0 || count < 0 || first + count > m.h.nz)
            throw IoError{T2B_ERR_ARG, "sections out of range of " + std::string(path)};
        const size_t sec = (size_t)m.h.nx * m.h.ny;
        const long long off = 1024LL + m.h.nsymbt + (long long)first * (long long)(sec * m.elem);
        if (fseeko(m.f, off, SEEK_SET) != 0) throw IoError{T2B_ERR_ARG, "seek failed in " + std::string(path)};
        std::vector<unsigned char> buf(sec * m.elem);
        for (long long s = 0; s < count; ++s) {
            if (std::fread(buf.data(), 1, buf.size(), m.f) != buf.size())
                throw IoError{T2B_ERR_ARG, "short read in " + std::string(path)};
            if (m.swap && m.elem > 1)
                for (size_t i = 0; i < sec; ++i) std::reverse(&buf[i * m.elem], &buf[i * m.elem] + m.elem);
            float* o = out + (size_t)s * sec;
            for (size_t i = 0; i < sec; ++i) {
                const unsigned char* p = &buf[i * m.elem];
                switch (m.h.mode) {
                case 0: o[i] = (float)(int8_t)p[0]; break;
                case 1: { int16_t v; std::memcpy(&v, p, 2); o[i] = v; break; }
                case 6: { uint16_t v; std::memcpy(&v, p, 2); o[i] = v; break; }
                case 12: { uint16_t v; std::memcpy(&v, p, 2); o[i] = half_to_float(v); break; }
                default: std::memcpy(&o[i], p, 4); break;
                }
            }
        }
    });
}

int t2b_mrc_write(const char* path, const float* data, int nx, int ny, int nz, double pixel_size)
{
    return io_guarded([&] {
        if (!path || !data || nx <= 0 || ny <= 0 || nz <= 0) throw IoError{T2B_ERR_ARG, "bad MRC write arguments"};
        MrcHeader h{};
        h.nx = nx;
        h.ny = ny;
        h.nz = nz;
        h.mode = 2;
        h.mx = nx;
        h.my = ny;
        h.mz = nz;
        h.cella[0] = (float)(pixel_size * nx);
        h.cella[1] = (float)(pixel_size * ny);
        h.cella[2] = (float)(pixel_size * nz);
        h.cellb[0] = h.cellb[1] = h.cellb[2] = 90.f;
        h.mapc = 1;
        h.mapr = 2;
        h.maps = 3;
        const size_t n = (size_t)nx * ny * nz;
        double mn = data[0], mx = data[0], sum = 0., sum2 = 0.;
        for (size_t i = 0; i < n; ++i) {
            mn = std::min(mn, (double)data[i]);
            mx = std::max(mx, (double)data[i]);
            sum += data[i];
            sum2 += (double)data[i] * data[i];
        }
        const double mean = sum / n;
        h.dmin = (float)mn;
        h.dmax = (float)mx;
        h.dmean = (float)mean;
        h.rms = (float)std::sqrt(std::max(0., sum2 / n - mean * mean));
        std::memcpy(h.map, "MAP ", 4);
        h.machst[0] = 0x44;
        h.machst[1] = 0x41;
        FILE* f = std::fopen(path, "wb");
        if (!f) throw IoError{T2B_ERR_ARG, std::string("cannot write ") + path};
        const bool ok = std::fwrite(&h, sizeof h, 1, f) == 1 && std::fwrite(data, sizeof(float), n, f) == n;
        std::fclose(f);
        if (!ok) throw IoError{T2B_ERR_ARG, std::string("write failed: ") + path};
    });
}

int t2b_star_open(const char* path, const char* block, t2b_star** out)
{
    return io_guarded([&] {
        if (!path || !out) throw IoError{T2B_ERR_ARG, "null argument"};
        std::ifstream in(path);
        if (!in) throw IoError{T2B_ERR_ARG, std::string("cannot open ") + path};
        std::unique_ptr<t2b_star> t(new t2b_star());
        star_parse(in, block ? block : "", *t);
        *out = t.release();
    });
}

int t2b_star_shape(const t2b_star* t, long long* rows, int* cols)
{
    return io_guarded([&] {
        if (!t) throw IoError{T2B_ERR_ARG, "null table"};
        if (rows) *rows = (long long)t->rows.size();
        if (cols) *cols = (int)t->labels.size();
    });
}

int t2b_star_label(const t2b_star* t, int col, char* buf, int cap)
{
    return io_guarded([&] {
        if (!t || !buf || cap < 1 || col < 0 || col >= (int)t->labels.size()) throw IoError{T2B_ERR_ARG, "bad column"};
        std::snprintf(buf, cap, "%s", t->labels[col].c_str());
    });
}

int t2b_star_column(const t2b_star* t, const char* label, double* out)
{
    return io_guarded([&] {
        if (!t || !out) throw IoError{T2B_ERR_ARG, "null argument"};
        const int c = t->column(label);
        if (c < 0) throw IoError{T2B_ERR_ARG, std::string("no column ") + (label ? label : "")};
        for (size_t r = 0; r < t->rows.size(); ++r) {
            const std::string& s = t->rows[r][c];
            char* end = nullptr;
            const double v = std::strtod(s.c_str(), &end);
            if (end == s.c_str() || *end != '\0')
                throw IoError{T2B_ERR_ARG, "STAR: not a number in column " + std::string(label) + ": " + s};
            out[r] = v;
        }
    });
}

int t2b_star_value(const t2b_star* t, const char* label, long long row, char* buf, int cap)
{
    return io_guarded([&] {
        if (!t || !buf || cap < 1) throw IoError{T2B_ERR_ARG, "null argument"};
        const int c = t->column(label);
        if (c < 0 || row < 0 || row >= (long long)t->rows.size()) throw IoError{T2B_ERR_ARG, "no such value"};
        std::snprintf(buf, cap, "%s", t->rows[row][c].c_str());
    });
}

void t2b_star_close(t2b_star* t) { delete t; }

int t2b_star_write(const char* path, const char* block, int ncols, const char* const* labels, long long nrows,
                   const double* values, int append)
{
    return io_guarded([&] {
        if (!path || !block || ncols < 1 || !labels || nrows < 0 || (nrows > 0 && !values))
            throw IoError{T2B_ERR_ARG, "bad STAR write arguments"};
        std::ofstream o(path, append ? std::ios::app : std::ios::trunc);
        if (!o) throw IoError{T2B_ERR_ARG, std::string("cannot write ") + path};
        o << "\n# version 30001\n\ndata_" << block << "\n\nloop_\n";
        for (int c = 0; c < ncols; ++c) {
            const char* l = labels[c];
            o << (l[0] == '_' ? "" : "_") << l << " #" << (c + 1) << "\n";
        }
        char buf[64];
        for (long long r = 0; r < nrows; ++r) {
            for (int c = 0; c < ncols; ++c) {
                std::snprintf(buf, sizeof buf, "%.17g", values[(size_t)r * ncols + c]);
                o << (c ? " " : "") << buf;
            }
            o << "\n";
        }
        o << "\n";
        if (!o) throw IoError{T2B_ERR_ARG, std::string("write failed: ") + path};
    });
}

}  // extern "C"
