// formats.h -- the reference's on-disk formats and directory conventions
// (user manual pp. 10-11; writers cited per function), shared by the CLI
// tools in this directory.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/pagani.h"

namespace pgio {

struct Csr {
    std::vector<int32_t> R, C;
    std::vector<float> V;  // empty for a binary graph
    int32_t n() const { return (int32_t)R.size() - 1; }
};

// .csr: int32 Rlength=N+1, R[N+1], int32 Clength=nnz, C[nnz]
// [, int32 Vlength=nnz, float V[nnz]] (CorMat.cpp:337-342; W CorMat.cpp:340-347).
bool read_csr(const std::string& path, Csr& g, std::string& err);
bool write_csr(const std::string& path, const Csr& g);
// .nm: int32 N, float[N] (e.g. U/Degree/Degree/Degree.cpp:99-101).
bool write_nm(const std::string& path, const std::vector<float>& x);
bool read_nm(const std::string& path, std::vector<float>& x);
// .modu: int32 N, int32 label[N] (U/cuda_EC/cuda_EC/modularity_GPU.cu:653-655).
bool write_modu(const std::string& path, const std::vector<int32_t>& labels);
// .cormat: int32 M1 (low 32 bits of the long long, CorMat.cpp:291), float[M1].
bool write_cormat(const std::string& path, const float* r, long long M1);
// Text file of values, one per line, printed with 6 significant digits as
// ofstream << setprecision(6) (Cp_main.cpp:178-180).
bool write_values(const std::string& path, const std::vector<double>& v);
bool read_first_value(const std::string& path, double& v);

// NIfTI-1 as the reference reads it (CorMat.cpp:138-235): 352-byte header
// viewed as short[176]: dims hdr[21..23], time points hdr[24], datatype
// hdr[35], bitpix hdr[36]; data at byte 352.  Beyond the reference, the data
// is read at vox_offset (files with extensions), scl_slope/scl_inter are
// applied when they are not the identity, big-endian files are byte-swapped,
// and int16/int32 volumes are accepted; the files the reference reads give
// the same values.
struct Nifti {
    int dims[3] = {0, 0, 0};
    int T = 1;
    int datatype = 0, bitpix = 0;
    long long vox_offset = 352;
    bool swapped = false;             // big-endian file
    unsigned char header[352] = {};   // as read
    std::vector<float> data;  // voxel-major per volume: data[t * V + k]
};
bool read_nifti(const std::string& path, Nifti& img, std::string& err);
// A float32 volume with the header of `like` (datatype 16, bitpix 32), as
// ConvertNII writes it (ConvertNII.cpp:139-157): header bytes kept, except
// that a header with extensions or value scaling is written without them.
bool write_nifti_like(const std::string& path, const Nifti& like, const std::vector<float>& vol);

// Files in `dir` with extension `ext` (".csr", ".nii", ...), sorted by name;
// `skip` is left out (the mask).
std::vector<std::string> list_dir(const std::string& dir, const std::string& ext, const std::string& skip = "");
std::string join(const std::string& dir, const std::string& name);
std::string stem(const std::string& path);   // path without its last extension

// Seed for the random surrogates: PAGANI_SEED if set, else a fixed default
// (the reference used time(0), which makes runs unrepeatable).
uint64_t surrogate_seed(uint64_t salt);

// Creates a context or exits with a message (CLI helper).
pg_ctx* open_ctx();
void check(pg_ctx* ctx, pg_status s, const char* what);
pg_graph* upload(pg_ctx* ctx, const Csr& g);
Csr download(pg_ctx* ctx, const pg_graph* g);

}  // namespace pgio
