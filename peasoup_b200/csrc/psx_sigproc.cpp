// psx_sigproc.cpp -- SIGPROC filterbank headers and sample rows, and the DM
// list file: the host input side of the reference's main program
// (include/data_types/header.hpp:171-212, 222-300, 339-403;
// include/data_types/filterbank.hpp:261-328; src/pipeline_multi.cu:313-337).
//
// A SIGPROC header is a sequence of keywords, each an int length and that
// many characters, between HEADER_START and HEADER_END; a keyword is
// followed by its value in the file's binary layout (int, double or one
// byte), except source_name and rawdatafile whose value is the next
// string.  The sample rows follow the header, time slowest.
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>

#include "psx_common.cuh"

using psx::clear_error;
using psx::set_error;

namespace {

enum Kind { kInt, kDouble, kByte };

struct Key {
    const char* name;
    Kind kind;
    size_t offset;
};

#define PSX_KEY(n, k) {#n, k, offsetof(psx_sigproc_header, n)}
const Key kKeys[] = {
    PSX_KEY(az_start, kDouble),    PSX_KEY(za_start, kDouble),   PSX_KEY(src_raj, kDouble),
    PSX_KEY(src_dej, kDouble),     PSX_KEY(tstart, kDouble),     PSX_KEY(tsamp, kDouble),
    PSX_KEY(period, kDouble),      PSX_KEY(fch1, kDouble),       PSX_KEY(foff, kDouble),
    PSX_KEY(nchans, kInt),         PSX_KEY(telescope_id, kInt),  PSX_KEY(machine_id, kInt),
    PSX_KEY(data_type, kInt),      PSX_KEY(ibeam, kInt),         PSX_KEY(nbeams, kInt),
    PSX_KEY(nbits, kInt),          PSX_KEY(barycentric, kInt),   PSX_KEY(pulsarcentric, kInt),
    PSX_KEY(nbins, kInt),          PSX_KEY(nsamples, kInt),      PSX_KEY(nifs, kInt),
    PSX_KEY(npuls, kInt),          PSX_KEY(refdm, kDouble),
    {"signed", kByte, offsetof(psx_sigproc_header, signed_data)},
};
#undef PSX_KEY

size_t value_size(Kind k) { return k == kInt ? sizeof(int) : k == kDouble ? sizeof(double) : 1; }

// Header bytes in memory, read front to back.
struct Cursor {
    const char* p;
    size_t n, pos;
    bool read(void* dst, size_t k)
    {
        if (pos + k > n) return false;
        std::memcpy(dst, p + pos, k);
        pos += k;
        return true;
    }
};

// One header string; false at the end of the bytes or for a length outside
// 1..79 (the reference's limit).
bool read_string(Cursor& c, std::string* s)
{
    int len = 0;
    if (!c.read(&len, sizeof(int))) return false;
    if (len <= 0 || len >= 80) return false;
    char buf[80];
    if (!c.read(buf, (size_t)len)) return false;
    s->assign(buf, (size_t)len);
    return true;
}

// PSX_OK, PSX_ERR_IO (no HEADER_START, bad string) or PSX_ERR_OVERFLOW
// (the bytes end before HEADER_END).
int parse(const char* bytes, size_t n, psx_sigproc_header* h)
{
    std::memset(h, 0, sizeof(*h));
    Cursor c{bytes, n, 0};
    std::string s;
    if (!read_string(c, &s) || s != "HEADER_START") {
        set_error("SIGPROC header: no HEADER_START");
        return PSX_ERR_IO;
    }
    bool want_source = false, want_raw = false;
    for (;;) {
        size_t at = c.pos;
        if (!read_string(c, &s)) {
            if (at + 80 + sizeof(int) > n) {
                set_error("SIGPROC header: the bytes end before HEADER_END");
                return PSX_ERR_OVERFLOW;
            }
            set_error("SIGPROC header: malformed keyword at byte %zu", at);
            return PSX_ERR_IO;
        }
        if (s == "HEADER_END") break;
        if (s == "source_name") { want_source = true; continue; }
        if (s == "rawdatafile") { want_raw = true; continue; }
        const Key* key = nullptr;
        for (const Key& k : kKeys)
            if (s == k.name) key = &k;
        if (key) {
            char* dst = reinterpret_cast<char*>(h) + key->offset;
            if (!c.read(dst, value_size(key->kind))) {
                set_error("SIGPROC header: the bytes end inside the value of %s", key->name);
                return PSX_ERR_OVERFLOW;
            }
        } else if (want_source) {
            std::snprintf(h->source_name, sizeof(h->source_name), "%s", s.c_str());
            want_source = false;
        } else if (want_raw) {
            std::snprintf(h->rawdatafile, sizeof(h->rawdatafile), "%s", s.c_str());
            want_raw = false;
        } else {
            std::fprintf(stderr, "Warning: read_header: unknown parameter %s\n", s.c_str());
        }
    }
    h->header_size = c.pos;
    return PSX_OK;
}

void write_string(std::ofstream& f, const char* s)
{
    int len = (int)std::strlen(s);
    f.write(reinterpret_cast<const char*>(&len), sizeof(int));
    f.write(s, len);
}

}  // namespace

extern "C" {

int psx_sigproc_parse_header(const void* bytes, size_t n, psx_sigproc_header* h)
{
    clear_error();
    if (!bytes || !h) return PSX_ERR_INVALID;
    return parse(static_cast<const char*>(bytes), n, h);
}

int psx_sigproc_read_header(const char* path, psx_sigproc_header* h)
{
    clear_error();
    if (!path || !h) return PSX_ERR_INVALID;
    std::ifstream f(path, std::ios::in | std::ios::binary);
    if (!f) {
        set_error("psx_sigproc_read_header: cannot open %s", path);
        return PSX_ERR_IO;
    }
    f.seekg(0, std::ios::end);
    const size_t total = (size_t)f.tellg();
    // headers are a few hundred bytes; read more only if one is longer
    std::string buf;
    int rc = PSX_ERR_OVERFLOW;
    for (size_t want = 4096; rc == PSX_ERR_OVERFLOW; want *= 4) {
        size_t k = std::min(want, total);
        buf.resize(k ? k : 1);
        f.clear();
        f.seekg(0, std::ios::beg);
        f.read(&buf[0], (std::streamsize)k);
        rc = parse(buf.data(), (size_t)f.gcount(), h);
        if (rc == PSX_ERR_OVERFLOW && k == total) {
            set_error("psx_sigproc_read_header: %s ends before HEADER_END", path);
            return PSX_ERR_IO;
        }
    }
    if (rc != PSX_OK) return rc;
    if (h->nsamples == 0 && h->nchans > 0 && h->nbits > 0) {
        size_t data = total >= h->header_size ? total - h->header_size : 0;
        // the reference's order of operations: bytes / nchans * 8 / nbits
        h->nsamples = (int)(data / (size_t)h->nchans * 8 / (size_t)h->nbits);
    }
    return PSX_OK;
}

int psx_sigproc_read(const char* path, const psx_sigproc_header* h, size_t start_sample,
                     size_t nsamples, void* h_dst, size_t* h_nread)
{
    clear_error();
    if (!path || !h || (!h_dst && nsamples) || h->nchans <= 0 || h->nbits <= 0) {
        set_error("psx_sigproc_read: bad arguments");
        return PSX_ERR_INVALID;
    }
    size_t bits = (size_t)h->nchans * (size_t)h->nbits;
    if (bits % 8 != 0) {
        set_error("psx_sigproc_read: a row of %d %d-bit channels is not whole bytes", h->nchans,
                  h->nbits);
        return PSX_ERR_INVALID;
    }
    size_t row = bits / 8;
    std::ifstream f(path, std::ios::in | std::ios::binary);
    if (!f) {
        set_error("psx_sigproc_read: cannot open %s", path);
        return PSX_ERR_IO;
    }
    f.seekg((std::streamoff)(h->header_size + start_sample * row), std::ios::beg);
    size_t got = 0;
    if (f) {
        f.read(static_cast<char*>(h_dst), (std::streamsize)(nsamples * row));
        got = (size_t)f.gcount();
    }
    if (h_nread) *h_nread = got / row;
    return PSX_OK;
}

int psx_sigproc_write_header(const char* path, const psx_sigproc_header* h, size_t* h_size)
{
    clear_error();
    if (!path || !h) return PSX_ERR_INVALID;
    std::ofstream f(path, std::ios::out | std::ios::binary | std::ios::trunc);
    if (!f) {
        set_error("psx_sigproc_write_header: cannot create %s", path);
        return PSX_ERR_IO;
    }
    write_string(f, "HEADER_START");
    char name[81];
    if (h->source_name[0]) {
        write_string(f, "source_name");
        std::snprintf(name, sizeof(name), "%.79s", h->source_name);
        write_string(f, name);
    }
    if (h->rawdatafile[0]) {
        write_string(f, "rawdatafile");
        std::snprintf(name, sizeof(name), "%.79s", h->rawdatafile);
        write_string(f, name);
    }
    for (const Key& k : kKeys) {
        const char* src = reinterpret_cast<const char*>(h) + k.offset;
        bool set = false;
        for (size_t i = 0; i < value_size(k.kind); ++i) set = set || src[i] != 0;
        // the observing keywords a reader needs are written even when zero
        bool always = !std::strcmp(k.name, "nchans") || !std::strcmp(k.name, "nbits") ||
                      !std::strcmp(k.name, "tsamp") || !std::strcmp(k.name, "fch1") ||
                      !std::strcmp(k.name, "foff") || !std::strcmp(k.name, "tstart") ||
                      !std::strcmp(k.name, "nifs") || !std::strcmp(k.name, "data_type");
        if (!set && !always) continue;
        write_string(f, k.name);
        f.write(src, (std::streamsize)value_size(k.kind));
    }
    write_string(f, "HEADER_END");
    if (!f) {
        set_error("psx_sigproc_write_header: write to %s failed", path);
        return PSX_ERR_IO;
    }
    if (h_size) *h_size = (size_t)f.tellp();
    return PSX_OK;
}

int psx_read_dm_file(const char* path, float* h_out, size_t cap, size_t* n_out)
{
    clear_error();
    if (!path || !n_out) return PSX_ERR_INVALID;
    std::ifstream f(path);
    if (!f) {
        set_error("psx_read_dm_file: cannot open %s", path);
        return PSX_ERR_IO;
    }
    std::string line;
    float value = 0.0f;
    size_t n = 0;
    while (std::getline(f, line)) {
        if (!line.empty()) value = (float)std::atof(line.c_str());
        if (h_out && n < cap) h_out[n] = value;
        ++n;
    }
    *n_out = n;
    if (n > cap || (!h_out && n)) {
        set_error("psx_read_dm_file: %zu DMs do not fit in %zu", n, cap);
        return PSX_ERR_OVERFLOW;
    }
    return PSX_OK;
}

}  // extern "C"
