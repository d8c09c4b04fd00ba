// formats.cpp -- see formats.h.
#include "formats.h"

#include <dirent.h>
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>

namespace pgio {

static bool read_i32(std::ifstream& f, int32_t& x) { return (bool)f.read((char*)&x, 4); }

bool read_csr(const std::string& path, Csr& g, std::string& err)
{
    std::ifstream f(path, std::ios::binary);
    if (!f.good()) { err = "cannot open " + path; return false; }
    int32_t rl = 0, cl = 0, vl = 0;
    if (!read_i32(f, rl) || rl < 1) { err = path + ": bad row header"; return false; }
    g.R.resize(rl);
    if (!f.read((char*)g.R.data(), 4LL * rl)) { err = path + ": truncated row array"; return false; }
    if (!read_i32(f, cl) || cl < 0) { err = path + ": bad column header"; return false; }
    g.C.resize(cl);
    if (cl && !f.read((char*)g.C.data(), 4LL * cl)) { err = path + ": truncated column array"; return false; }
    g.V.clear();
    if (read_i32(f, vl)) {
        if (vl != cl) { err = path + ": value length differs from column length"; return false; }
        g.V.resize(vl);
        if (vl && !f.read((char*)g.V.data(), 4LL * vl)) { err = path + ": truncated value array"; return false; }
    }
    if (g.R[0] != 0 || g.R.back() != cl) { err = path + ": R[N] does not match the column count"; return false; }
    for (size_t i = 0; i + 1 < g.R.size(); i++)
        if (g.R[i + 1] < g.R[i]) { err = path + ": row offsets decrease"; return false; }
    const int32_t n = g.n();
    for (int32_t c : g.C)
        if (c < 0 || c >= n) { err = path + ": column index out of range"; return false; }
    return true;
}

bool write_csr(const std::string& path, const Csr& g)
{
    std::string tmp = path + ".tmp";
    {
        std::ofstream f(tmp, std::ios::binary);
        if (!f.good()) return false;
        int32_t rl = (int32_t)g.R.size(), cl = (int32_t)g.C.size();
        f.write((char*)&rl, 4);
        f.write((char*)g.R.data(), 4LL * rl);
        f.write((char*)&cl, 4);
        f.write((char*)g.C.data(), 4LL * cl);
        if (!g.V.empty()) {
            f.write((char*)&cl, 4);
            f.write((char*)g.V.data(), 4LL * cl);
        }
        if (!f.good()) return false;
    }
    return std::rename(tmp.c_str(), path.c_str()) == 0;
}

bool write_nm(const std::string& path, const std::vector<float>& x)
{
    std::ofstream f(path, std::ios::binary);
    int32_t n = (int32_t)x.size();
    f.write((char*)&n, 4);
    f.write((char*)x.data(), 4LL * n);
    return f.good();
}

bool write_modu(const std::string& path, const std::vector<int32_t>& labels)
{
    std::ofstream f(path, std::ios::binary);
    int32_t n = (int32_t)labels.size();
    f.write((char*)&n, 4);
    f.write((char*)labels.data(), 4LL * n);
    return f.good();
}

bool write_cormat(const std::string& path, const float* r, long long M1)
{
    std::ofstream f(path, std::ios::binary);
    int32_t m = (int32_t)(uint32_t)(unsigned long long)M1;
    f.write((char*)&m, 4);
    f.write((const char*)r, 4LL * M1);
    return f.good();
}

bool read_nm(const std::string& path, std::vector<float>& x)
{
    std::ifstream f(path, std::ios::binary);
    int32_t n = 0;
    if (!f.read((char*)&n, 4) || n < 0) return false;
    x.resize((size_t)n);
    return (bool)f.read((char*)x.data(), (std::streamsize)(4 * (size_t)n));
}

bool write_values(const std::string& path, const std::vector<double>& v)
{
    std::ofstream f(path);
    for (double x : v) f << std::setprecision(6) << x << "\n";
    return f.good();
}

bool read_first_value(const std::string& path, double& v)
{
    std::ifstream f(path);
    return (bool)(f >> v);
}

namespace {
template <class T>
T swapped(T v)
{
    unsigned char* b = (unsigned char*)&v;
    for (size_t i = 0; i < sizeof(T) / 2; i++) std::swap(b[i], b[sizeof(T) - 1 - i]);
    return v;
}
template <class T>
T field(const unsigned char* hdr, int at, bool swap)
{
    T v;
    memcpy(&v, hdr + at, sizeof(T));
    return swap ? swapped(v) : v;
}
template <class T>
bool read_values(std::ifstream& f, long long total, bool swap, std::vector<float>& out)
{
    std::vector<T> b((size_t)total);
    if (!f.read((char*)b.data(), (std::streamsize)(sizeof(T) * total))) return false;
    for (long long q = 0; q < total; q++) out[q] = (float)(swap ? swapped(b[q]) : b[q]);
    return true;
}
}  // namespace

bool read_nifti(const std::string& path, Nifti& img, std::string& err)
{
    std::ifstream f(path, std::ios::binary);
    if (!f.good()) { err = "cannot open " + path; return false; }
    unsigned char hdr[352];
    if (!f.read((char*)hdr, 352)) { err = path + ": truncated NIfTI header"; return false; }
    memcpy(img.header, hdr, 352);
    // sizeof_hdr is 348; read in the other byte order it marks a big-endian file
    const bool swap = field<int32_t>(hdr, 0, false) != 348 && field<int32_t>(hdr, 0, true) == 348;
    img.swapped = swap;
    img.dims[0] = field<int16_t>(hdr, 42, swap);
    img.dims[1] = field<int16_t>(hdr, 44, swap);
    img.dims[2] = field<int16_t>(hdr, 46, swap);
    const int16_t t = field<int16_t>(hdr, 48, swap);
    img.T = t > 0 ? t : 1;
    img.datatype = field<int16_t>(hdr, 70, swap);
    img.bitpix = field<int16_t>(hdr, 72, swap);
    // the data starts at vox_offset (352 when there are no extensions)
    const float vox_offset = field<float>(hdr, 108, swap);
    const long long at = vox_offset >= 352.0f ? (long long)vox_offset : 352;
    img.vox_offset = at;
    const float slope = field<float>(hdr, 112, swap), inter = field<float>(hdr, 116, swap);
    const long long V = (long long)img.dims[0] * img.dims[1] * img.dims[2];
    if (V <= 0) { err = path + ": empty volume"; return false; }
    const long long total = V * img.T;
    img.data.resize((size_t)total);
    f.seekg(at);
    bool ok;
    if (img.datatype == 2 || (img.datatype == 0 && img.bitpix == 8)) ok = read_values<uint8_t>(f, total, false, img.data);
    else if (img.datatype == 4) ok = read_values<int16_t>(f, total, swap, img.data);
    else if (img.datatype == 8) ok = read_values<int32_t>(f, total, swap, img.data);
    else if (img.datatype == 16 || (img.datatype == 0 && img.bitpix == 32)) ok = read_values<float>(f, total, swap, img.data);
    else if (img.datatype == 64 || (img.datatype == 0 && img.bitpix == 64)) ok = read_values<double>(f, total, swap, img.data);
    else {
        err = path + ": data type is not uint8, int16, int32, float32 or float64";
        return false;
    }
    if (!ok) { err = path + ": truncated data"; return false; }
    // NIfTI value scaling, when the header asks for one
    if (slope != 0.0f && (slope != 1.0f || inter != 0.0f))
        for (float& v : img.data) v = v * slope + inter;
    return true;
}

bool write_nifti_like(const std::string& path, const Nifti& like, const std::vector<float>& vol)
{
    unsigned char hdr[352];
    memcpy(hdr, like.header, 352);
    auto put16 = [&](int at, int16_t v) {
        if (like.swapped) v = swapped(v);
        memcpy(hdr + at, &v, 2);
    };
    auto putf = [&](int at, float v) {
        if (like.swapped) v = swapped(v);
        memcpy(hdr + at, &v, 4);
    };
    put16(70, 16);   // float32
    put16(72, 32);
    if (like.vox_offset != 352) {
        // the output carries no extensions: the data follows the header
        putf(108, 352.0f);
        memset(hdr + 348, 0, 4);
    }
    {
        const float slope = field<float>(like.header, 112, like.swapped);
        const float inter = field<float>(like.header, 116, like.swapped);
        if (slope != 0.0f && (slope != 1.0f || inter != 0.0f)) {   // the values are written unscaled
            putf(112, 0.0f);
            putf(116, 0.0f);
        }
    }
    std::ofstream f(path, std::ios::binary);
    f.write((const char*)hdr, 352);
    if (like.swapped) {
        std::vector<float> b(vol.size());
        for (size_t q = 0; q < vol.size(); q++) b[q] = swapped(vol[q]);
        f.write((const char*)b.data(), (std::streamsize)(4 * b.size()));
    } else {
        f.write((const char*)vol.data(), (std::streamsize)(4 * vol.size()));
    }
    return f.good();
}

std::vector<std::string> list_dir(const std::string& dir, const std::string& ext, const std::string& skip)
{
    std::vector<std::string> out;
    DIR* dp = opendir(dir.c_str());
    if (!dp) return out;
    while (dirent* e = readdir(dp)) {
        std::string nm = e->d_name;
        size_t dot = nm.find_last_of('.');
        if (dot == std::string::npos || nm.size() <= ext.size()) continue;
        if (nm.substr(dot) != ext) continue;
        if (nm == skip) continue;
        out.push_back(nm);
    }
    closedir(dp);
    std::sort(out.begin(), out.end());
    return out;
}

std::string join(const std::string& dir, const std::string& name)
{
    if (dir.empty()) return name;
    char last = dir.back();
    return (last == '/' || last == '\\') ? dir + name : dir + "/" + name;
}

std::string stem(const std::string& path)
{
    size_t dot = path.find_last_of('.');
    size_t slash = path.find_last_of("/\\");
    if (dot == std::string::npos || (slash != std::string::npos && dot < slash)) return path;
    return path.substr(0, dot);
}

uint64_t surrogate_seed(uint64_t salt)
{
    const char* e = getenv("PAGANI_SEED");
    uint64_t s = e ? strtoull(e, nullptr, 10) : 20261203ULL;
    return s * 0x9E3779B97F4A7C15ULL + salt;
}

pg_ctx* open_ctx()
{
    pg_ctx* ctx = nullptr;
    const char* d = getenv("PAGANI_DEVICE");
    pg_status s = pg_create(&ctx, d ? atoi(d) : 0);
    if (s != PG_OK) {
        fprintf(stderr, "cannot open the GPU: %s\n", pg_status_string(s));
        exit(2);
    }
    return ctx;
}

void check(pg_ctx* ctx, pg_status s, const char* what)
{
    if (s != PG_OK) {
        fprintf(stderr, "%s failed: %s (%s)\n", what, pg_status_string(s), pg_last_error(ctx));
        exit(3);
    }
}

pg_graph* upload(pg_ctx* ctx, const Csr& g)
{
    pg_graph* h = nullptr;
    check(ctx, pg_graph_from_csr(ctx, g.R.data(), g.C.data(), g.V.empty() ? nullptr : g.V.data(), g.n(),
                                 (int64_t)g.C.size(), 0, &h),
          "upload");
    return h;
}

Csr download(pg_ctx* ctx, const pg_graph* g)
{
    int32_t n = 0, w = 0;
    int64_t nnz = 0;
    pg_graph_info(g, &n, &nnz, &w);
    Csr c;
    c.R.resize((size_t)n + 1);
    c.C.resize((size_t)nnz);
    if (w) c.V.resize((size_t)nnz);
    check(ctx, pg_graph_to_csr(ctx, g, c.R.data(), c.C.data(), w ? c.V.data() : nullptr, 0), "download");
    return c;
}

}  // namespace pgio
