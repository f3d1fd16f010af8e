// DADA file ingest and output for the beamforming path (C ABI objects behind
// sw_dada_*).
//
// Reference: cpp/skyweaver/src/ObservationHeader.cpp:6-33 (header keys),
// cpp/skyweaver/src/Header.cpp (ASCII key lookup: a key at the start of a
// line, its value the next whitespace-separated token, "unset" rejected),
// cpp/skyweaver/src/MultiFileReader.cu:34-303 (several DADA files read as one
// contiguous payload, optional OBS_OFFSET contiguity check, seek),
// cpp/skyweaver/src/FileOutputStream.cpp:80-150 (payload split over files of
// a fixed size, each file led by a DADA header whose FILE_NUMBER,
// OBS_OFFSET and FILE_SIZE are updated, files named
// <base>_<payload offset, 16 digits><extension>).  The reader tracks its
// position in payload bytes across all files.
#include <sys/stat.h>

#include <cerrno>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "../sw_common.cuh"

namespace {

// value of `key` in a DADA header (nullptr-terminated within `size`)
bool header_lookup(const char* hdr, size_t size, const char* key, std::string& value)
{
    const size_t klen = std::strlen(key);
    size_t i = 0;
    while(i < size && hdr[i]) {
        // at the start of a line
        const size_t line_end = [&] {
            size_t j = i;
            while(j < size && hdr[j] && hdr[j] != '\n') ++j;
            return j;
        }();
        if(line_end - i > klen && std::strncmp(hdr + i, key, klen) == 0 &&
           (hdr[i + klen] == ' ' || hdr[i + klen] == '\t')) {
            size_t v = i + klen;
            while(v < line_end && (hdr[v] == ' ' || hdr[v] == '\t')) ++v;
            size_t e = v;
            while(e < line_end && hdr[e] != ' ' && hdr[e] != '\t' && hdr[e] != '\r') ++e;
            value.assign(hdr + v, e - v);
            return true;
        }
        i = line_end + 1;
    }
    return false;
}

int header_get(const char* hdr, size_t size, const char* key, std::string& value)
{
    if(!header_lookup(hdr, size, key, value)) {
        swb::set_error("Could not find %s key in DADA header.", key);
        return SW_ERR_INVALID;
    }
    if(value == "unset") {
        swb::set_error("The header key %s was unset", key);
        return SW_ERR_INVALID;
    }
    return SW_OK;
}

// replace the value of `key` or append "key value" as a new line
int header_set(std::vector<char>& hdr, const char* key, const char* value)
{
    std::string text(hdr.data(), strnlen(hdr.data(), hdr.size()));
    std::string out;
    bool done = false;
    std::istringstream in(text);
    std::string line;
    const size_t klen = std::strlen(key);
    while(std::getline(in, line)) {
        if(!done && line.size() > klen && line.compare(0, klen, key) == 0 &&
           (line[klen] == ' ' || line[klen] == '\t')) {
            std::string pad = line.substr(klen);
            size_t ws = pad.find_first_not_of(" \t");
            out += std::string(key) + pad.substr(0, ws == std::string::npos ? 1 : ws) + value +
                   "\n";
            done = true;
        } else {
            out += line + "\n";
        }
    }
    if(!done) out += std::string(key) + " " + value + "\n";
    if(out.size() + 1 > hdr.size()) {
        swb::set_error("DADA header of %zu bytes cannot hold key %s", hdr.size(), key);
        return SW_ERR_INVALID;
    }
    std::fill(hdr.begin(), hdr.end(), 0);
    std::memcpy(hdr.data(), out.data(), out.size());
    return SW_OK;
}

void copy_str(char* dst, size_t cap, const std::string& s)
{
    std::snprintf(dst, cap, "%s", s.c_str());
}

}  // namespace

struct sw_dada_reader {
    std::vector<std::string> files;
    std::vector<size_t> sizes;  // payload bytes per file
    std::vector<sw_observation_header> headers;
    size_t header_size = 4096, total = 0, pos = 0;
    int cur = -1;
    std::ifstream in;

    int open_file(int i, size_t offset)
    {
        in.close();
        in.clear();
        in.open(files[i], std::ios::in | std::ios::binary);
        if(!in.is_open()) {
            swb::set_error("Could not open file %s", files[i].c_str());
            return SW_ERR_INVALID;
        }
        in.seekg((std::streamoff)(header_size + offset), std::ios::beg);
        cur = i;
        return SW_OK;
    }
};

struct sw_dada_writer {
    std::string dir, base, ext;
    size_t bytes_per_file = 0, total = 0, in_file = 0;
    int file_count = 0;
    std::vector<char> header;
    std::ofstream out;
    bool open = false;

    int new_file()
    {
        if(out.is_open()) out.close();
        char name[64];
        std::snprintf(name, sizeof(name), "_%016zu", total);
        const std::string path = dir + "/" + base + name + ext;
        std::vector<char> h = header;
        char num[32];
        std::snprintf(num, sizeof(num), "%zu", bytes_per_file);
        SW_TRY(header_set(h, "FILE_SIZE", num));
        std::snprintf(num, sizeof(num), "%d", file_count);
        SW_TRY(header_set(h, "FILE_NUMBER", num));
        std::snprintf(num, sizeof(num), "%zu", total);
        SW_TRY(header_set(h, "OBS_OFFSET", num));
        out.open(path, std::ios::out | std::ios::binary | std::ios::trunc);
        if(!out.is_open()) {
            swb::set_error("Could not open file %s", path.c_str());
            return SW_ERR_INVALID;
        }
        out.write(h.data(), (std::streamsize)h.size());
        if(!out) {
            swb::set_error("Unable to write header to %s", path.c_str());
            return SW_ERR_INVALID;
        }
        in_file = 0;
        ++file_count;
        return SW_OK;
    }
};

extern "C" {

int sw_dada_header_get(const char* header, size_t header_size, const char* key, char* value,
                       size_t value_capacity)
{
    SW_REQUIRE(header && key && value && value_capacity > 0, "sw_dada_header_get: null argument");
    std::string v;
    SW_TRY(header_get(header, header_size, key, v));
    SW_REQUIRE(v.size() < value_capacity, "sw_dada_header_get: value of %s too long", key);
    copy_str(value, value_capacity, v);
    return SW_OK;
}

int sw_dada_parse_header(const char* header, size_t header_size, sw_observation_header* out)
{
    SW_REQUIRE(header && out, "sw_dada_parse_header: null argument");
    std::memset(out, 0, sizeof(*out));
    std::string v;
    auto u = [&](const char* k, size_t& dst) {
        if(header_get(header, header_size, k, v) != SW_OK) return SW_ERR_INVALID;
        dst = std::strtoull(v.c_str(), nullptr, 0);
        return SW_OK;
    };
    auto d = [&](const char* k, double& dst) {
        if(header_get(header, header_size, k, v) != SW_OK) return SW_ERR_INVALID;
        dst = std::strtod(v.c_str(), nullptr);
        return SW_OK;
    };
    auto s = [&](const char* k, char* dst, size_t cap) {
        if(header_get(header, header_size, k, v) != SW_OK) return SW_ERR_INVALID;
        copy_str(dst, cap, v);
        return SW_OK;
    };
    // the keys and order of read_dada_header (ObservationHeader.cpp:6-33)
    SW_TRY(u("NCHAN", out->nchans));
    SW_TRY(u("OBS_NCHAN", out->obs_nchans));
    SW_TRY(u("NPOL", out->npol));
    SW_TRY(u("NBIT", out->nbits));
    SW_TRY(u("NANT", out->nantennas));
    SW_TRY(u("SAMPLE_CLOCK_START", out->sample_clock_start));
    SW_TRY(d("BW", out->bandwidth));
    SW_TRY(d("OBS_BW", out->obs_bandwidth));
    SW_TRY(d("FREQ", out->frequency));
    SW_TRY(d("OBS_FREQ", out->obs_frequency));
    SW_TRY(d("TSAMP", out->tsamp));
    SW_TRY(d("SAMPLE_CLOCK", out->sample_clock));
    SW_TRY(d("SYNC_TIME", out->sync_time));
    SW_TRY(d("UTC_START", out->utc_start));
    SW_TRY(d("MJD_START", out->mjd_start));
    SW_TRY(s("SOURCE", out->source_name, sizeof(out->source_name)));
    SW_TRY(s("RA", out->ra, sizeof(out->ra)));
    SW_TRY(s("DEC", out->dec, sizeof(out->dec)));
    SW_TRY(s("TELESCOPE", out->telescope, sizeof(out->telescope)));
    SW_TRY(s("INSTRUMENT", out->instrument, sizeof(out->instrument)));
    SW_TRY(u("CHAN0_IDX", out->chan0_idx));
    SW_TRY(u("OBS_OFFSET", out->obs_offset));
    return SW_OK;
}

int sw_dada_validate_header(const sw_observation_header* h, int nantennas, int nchans, int npol)
{
    SW_REQUIRE(h, "sw_dada_validate_header: null header");
    // ObservationHeader.cpp:35-62
    SW_REQUIRE((int)h->nantennas <= nantennas,
               "Input data contains too many antennas for the configured antenna count");
    SW_REQUIRE((int)h->nchans == nchans,
               "Input data contains incorrect number of channels for the configuration");
    SW_REQUIRE((int)h->npol == npol,
               "Input data contains incorrect number of polarisations for the configuration");
    SW_REQUIRE(h->nbits == 8,
               "Input data contains incorrect number of bits per sample, currently only 8-bit "
               "input supported");
    return SW_OK;
}

int sw_dada_reader_open(const char* const* files, int nfiles, size_t header_size,
                        int check_contiguity, sw_dada_reader** out)
{
    SW_REQUIRE(out && files && nfiles > 0 && header_size > 0, "sw_dada_reader_open: bad argument");
    *out = nullptr;
    std::unique_ptr<sw_dada_reader> r(new sw_dada_reader());
    r->header_size = header_size;
    std::vector<char> hdr(header_size + 1, 0);
    for(int i = 0; i < nfiles; ++i) {
        SW_REQUIRE(files[i], "sw_dada_reader_open: null file name");
        std::ifstream f(files[i], std::ios::in | std::ios::binary);
        SW_REQUIRE(f.is_open(), "Could not open file %s", files[i]);
        f.seekg(0, std::ios::end);
        const size_t size = (size_t)f.tellg();
        SW_REQUIRE(size >= header_size, "File %s is shorter than its DADA header", files[i]);
        f.seekg(0, std::ios::beg);
        f.read(hdr.data(), (std::streamsize)header_size);
        SW_REQUIRE((size_t)f.gcount() == header_size, "Could not read the header of %s", files[i]);
        sw_observation_header h{};
        SW_TRY(sw_dada_parse_header(hdr.data(), header_size, &h));
        r->files.push_back(files[i]);
        r->headers.push_back(h);
        r->sizes.push_back(size - header_size);
        r->total += size - header_size;
    }
    if(check_contiguity) {  // MultiFileReader.cu:66-81
        size_t so_far = r->sizes[0];
        for(int i = 1; i < nfiles; ++i) {
            SW_REQUIRE(r->headers[i].obs_offset == so_far, "These are not contiguous:%s and %s",
                       files[i - 1], files[i]);
            so_far += r->sizes[i];
        }
    }
    SW_TRY(r->open_file(0, 0));
    *out = r.release();
    return SW_OK;
}

void sw_dada_reader_close(sw_dada_reader* r) { delete r; }

int sw_dada_reader_header(const sw_dada_reader* r, int file_idx, sw_observation_header* out)
{
    SW_REQUIRE(r && out && file_idx >= 0 && file_idx < (int)r->headers.size(),
               "sw_dada_reader_header: bad argument");
    *out = r->headers[file_idx];
    return SW_OK;
}

size_t sw_dada_reader_total_bytes(const sw_dada_reader* r) { return r ? r->total : 0; }
size_t sw_dada_reader_tell(const sw_dada_reader* r) { return r ? r->pos : 0; }

int sw_dada_reader_seek(sw_dada_reader* r, size_t payload_offset)
{
    SW_REQUIRE(r, "sw_dada_reader_seek: null reader");
    SW_REQUIRE(payload_offset <= r->total, "Invalid seek position: %zu", payload_offset);
    size_t cum = 0;
    for(size_t i = 0; i < r->files.size(); ++i) {
        if(payload_offset < cum + r->sizes[i] || i + 1 == r->files.size()) {
            SW_TRY(r->open_file((int)i, payload_offset - cum));
            r->pos = payload_offset;
            return SW_OK;
        }
        cum += r->sizes[i];
    }
    return SW_OK;
}

int sw_dada_reader_read(sw_dada_reader* r, void* dst, size_t bytes, size_t* nread)
{
    SW_REQUIRE(r && (dst || bytes == 0), "sw_dada_reader_read: null argument");
    size_t done = 0;
    char* p = static_cast<char*>(dst);
    while(done < bytes && r->pos < r->total) {
        size_t cum = 0;
        for(int i = 0; i < r->cur; ++i) cum += r->sizes[i];
        const size_t left_in_file = cum + r->sizes[r->cur] - r->pos;
        if(left_in_file == 0) {
            SW_TRY(r->open_file(r->cur + 1, 0));
            continue;
        }
        const size_t n = std::min(bytes - done, left_in_file);
        r->in.read(p + done, (std::streamsize)n);
        const size_t got = (size_t)r->in.gcount();
        SW_REQUIRE(got == n, "Error: Unable to read from %s: %s", r->files[r->cur].c_str(),
                   std::strerror(errno));
        done += got;
        r->pos += got;
    }
    if(nread) *nread = done;
    return SW_OK;
}

int sw_dada_writer_open(const char* directory, const char* base_filename, const char* extension,
                        size_t bytes_per_file, const char* header_template, size_t header_size,
                        sw_dada_writer** out)
{
    SW_REQUIRE(out && directory && base_filename && extension, "sw_dada_writer_open: null argument");
    *out = nullptr;
    SW_REQUIRE(bytes_per_file > 0, "The number of bytes per file must be greater than zero");
    SW_REQUIRE(header_size >= 64, "sw_dada_writer_open: header size too small");
    std::unique_ptr<sw_dada_writer> w(new sw_dada_writer());
    w->dir = directory;
    w->base = base_filename;
    w->ext = extension;
    w->bytes_per_file = bytes_per_file;
    w->header.assign(header_size, 0);
    const std::string tmpl = header_template ? header_template : "HEADER DADA\nHDR_VERSION 1.0\n";
    SW_REQUIRE(tmpl.size() < header_size, "sw_dada_writer_open: header template too long");
    std::memcpy(w->header.data(), tmpl.data(), tmpl.size());
    char num[32];
    std::snprintf(num, sizeof(num), "%zu", header_size);
    SW_TRY(header_set(w->header, "HDR_SIZE", num));
    std::error_code ec;
    umask(0022);
    std::filesystem::create_directories(w->dir, ec);
    SW_REQUIRE(std::filesystem::is_directory(w->dir), "Failed to create directory: %s",
               w->dir.c_str());
    *out = w.release();
    return SW_OK;
}

int sw_dada_writer_set(sw_dada_writer* w, const char* key, const char* value)
{
    SW_REQUIRE(w && key && value, "sw_dada_writer_set: null argument");
    return header_set(w->header, key, value);
}

int sw_dada_writer_write(sw_dada_writer* w, const void* data, size_t bytes)
{
    SW_REQUIRE(w && (data || bytes == 0), "sw_dada_writer_write: null argument");
    const char* p = static_cast<const char*>(data);
    while(bytes > 0) {
        if(!w->out.is_open() || w->in_file == w->bytes_per_file) SW_TRY(w->new_file());
        const size_t n = std::min(bytes, w->bytes_per_file - w->in_file);
        w->out.write(p, (std::streamsize)n);
        SW_REQUIRE((bool)w->out, "Error writing DADA output: %s", std::strerror(errno));
        w->in_file += n;
        w->total += n;
        p += n;
        bytes -= n;
    }
    return SW_OK;
}

int sw_dada_writer_close(sw_dada_writer* w)
{
    if(!w) return SW_OK;
    if(w->out.is_open()) w->out.close();
    delete w;
    return SW_OK;
}

}  // extern "C"
