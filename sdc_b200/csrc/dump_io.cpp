// dump_io.cpp -- state files in the reference's binary dump format (host side).
//
// Format of matrix_folder_writer::write_binary_file / read_binary_file
// (gpu_flow/code/output/matrix_folder_writer.cu:3-101): int number_of_matrices, then per
// matrix int ndim, int dims[ndim] and the complex entries (x fastest). The reference
// writes CUDA_FLOAT, i.e. 8-byte complex (FP32) in its default build and 16-byte complex
// with PRECISION_DOUBLE (gpu_flow/code/cuda_defines.h:9-27); both are read here, the
// element size being told apart by the file size. State files hold one 3-d matrix:
// theta, f, g with dims (Nx/2+1, Ny, L), F and G with (1, 1, L), named like main.cu:697-713
// (theta_%08d.bin, ...). The AB2 history file is this library's extension: one file with
// five matrices (B^-1 N of the previous step for theta, f, g, F, G), always FP64.
#include "rbc.h"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace rbchost {

struct Matrix {
    std::vector<int> dims;
    std::vector<double> data; // interleaved complex, FP64
};

static bool read_all(const char* path, std::vector<unsigned char>& buf)
{
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return false;
    std::fseek(fp, 0, SEEK_END);
    const long n = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    if (n < 0) { std::fclose(fp); return false; }
    buf.resize((size_t)n);
    const size_t got = n ? std::fread(buf.data(), 1, (size_t)n, fp) : 0;
    std::fclose(fp);
    return got == (size_t)n;
}

// Parses a container of matrices. The complex element size (8 or 16 bytes) is chosen
// so that the matrices exactly fill the file.
static bool parse(const std::vector<unsigned char>& buf, std::vector<Matrix>& out, std::string& err)
{
    for (int esize : {16, 8}) {
        out.clear();
        size_t o = 0;
        auto rd_int = [&](int& v) {
            if (o + 4 > buf.size()) return false;
            std::memcpy(&v, buf.data() + o, 4);
            o += 4;
            return true;
        };
        int nmat = 0;
        if (!rd_int(nmat) || nmat < 1 || nmat > 64) { err = "bad matrix count"; return false; }
        bool ok = true;
        for (int m = 0; m < nmat && ok; ++m) {
            int nd = 0;
            if (!rd_int(nd) || nd < 1 || nd > 8) { ok = false; break; }
            Matrix M;
            size_t n = 1;
            for (int d = 0; d < nd; ++d) {
                int v = 0;
                if (!rd_int(v) || v < 1) { ok = false; break; }
                M.dims.push_back(v);
                n *= (size_t)v;
            }
            if (!ok || o + n * esize > buf.size()) { ok = false; break; }
            M.data.resize(2 * n);
            if (esize == 16) {
                std::memcpy(M.data.data(), buf.data() + o, n * 16);
            } else {
                std::vector<float> tmp(2 * n);
                std::memcpy(tmp.data(), buf.data() + o, n * 8);
                for (size_t i = 0; i < 2 * n; ++i) M.data[i] = tmp[i];
            }
            o += n * esize;
            out.push_back(std::move(M));
        }
        if (ok && o == buf.size()) return true;
    }
    err = "file size does not match an FP32 or FP64 dump";
    return false;
}

static bool write_container(const char* path, const std::vector<const Matrix*>& mats, int real_bytes)
{
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return false;
    bool ok = true;
    const int nmat = (int)mats.size();
    ok &= std::fwrite(&nmat, 4, 1, fp) == 1;
    for (const Matrix* M : mats) {
        const int nd = (int)M->dims.size();
        ok &= std::fwrite(&nd, 4, 1, fp) == 1;
        ok &= std::fwrite(M->dims.data(), 4, (size_t)nd, fp) == (size_t)nd;
        if (real_bytes == 8) {
            ok &= std::fwrite(M->data.data(), 8, M->data.size(), fp) == M->data.size();
        } else {
            std::vector<float> tmp(M->data.begin(), M->data.end());
            ok &= std::fwrite(tmp.data(), 4, tmp.size(), fp) == tmp.size();
        }
    }
    ok &= std::fclose(fp) == 0;
    return ok;
}

} // namespace rbchost

using namespace rbchost;

extern "C" {

rbc_status rbc_dump_read(const char* path, int index, int* dims, int maxdims, int* ndims, double* out, long long maxvals)
{
    if (!path || !dims || !ndims || maxdims < 1) return RBC_ERR_INVALID_ARG;
    std::vector<unsigned char> buf;
    if (!read_all(path, buf)) return RBC_ERR_IO;
    std::vector<Matrix> mats;
    std::string err;
    if (!parse(buf, mats, err)) return RBC_ERR_IO;
    if (index < 0 || index >= (int)mats.size()) return RBC_ERR_INVALID_ARG;
    const Matrix& M = mats[index];
    if ((int)M.dims.size() > maxdims) return RBC_ERR_INVALID_ARG;
    *ndims = (int)M.dims.size();
    for (size_t d = 0; d < M.dims.size(); ++d) dims[d] = M.dims[d];
    if (out) {
        if ((long long)M.data.size() > 2 * maxvals) return RBC_ERR_INVALID_ARG;
        std::memcpy(out, M.data.data(), M.data.size() * sizeof(double));
    }
    return RBC_OK;
}

rbc_status rbc_dump_write(const char* path, const int* dims, int ndims, const double* data, int real_bytes)
{
    if (!path || !dims || ndims < 1 || !data || (real_bytes != 4 && real_bytes != 8)) return RBC_ERR_INVALID_ARG;
    Matrix M;
    size_t n = 1;
    for (int d = 0; d < ndims; ++d) {
        if (dims[d] < 1) return RBC_ERR_INVALID_ARG;
        M.dims.push_back(dims[d]);
        n *= (size_t)dims[d];
    }
    M.data.assign(data, data + 2 * n);
    return write_container(path, {&M}, real_bytes) ? RBC_OK : RBC_ERR_IO;
}

// TRKSS track file, version 'a' (gpu_flow/code/output/track_movie.cpp:256-325): header
// "TRKSS", 'a', uint32 tracks, uint32 frame rate (1, track_writer.cu:15), uint32 length
// and the description, uint32 first and last frame time, uint32 frame count; then per
// frame uint32 time and x, y, z float32 per track.
rbc_status rbc_track_write(const char* path, const char* description, const float* xyz, const unsigned int* times,
                           int nframes, int n)
{
    if (!path || nframes < 0 || n < 0 || (nframes > 0 && (!xyz || !times))) return RBC_ERR_INVALID_ARG;
    const std::string desc = description ? description : "";
    std::vector<unsigned char> out;
    auto put = [&out](const void* p, size_t k) {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        out.insert(out.end(), b, b + k);
    };
    auto put32 = [&put](uint32_t v) { put(&v, 4); };
    put("TRKSS", 5);
    put("a", 1);
    put32((uint32_t)n);
    put32(1u);
    put32((uint32_t)desc.size());
    put(desc.data(), desc.size());
    put32(nframes > 0 ? times[0] : 0u);
    put32(nframes > 0 ? times[nframes - 1] : 0u);
    put32((uint32_t)nframes);
    for (int f = 0; f < nframes; ++f) {
        put32(times[f]);
        const float* fx = xyz + (size_t)f * 3 * n;
        for (int j = 0; j < n; ++j) {
            put(fx + j, 4);
            put(fx + n + j, 4);
            put(fx + 2 * (size_t)n + j, 4);
        }
    }
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return RBC_ERR_IO;
    const bool ok = std::fwrite(out.data(), 1, out.size(), fp) == out.size();
    return (std::fclose(fp) == 0 && ok) ? RBC_OK : RBC_ERR_IO;
}

} // extern "C"
