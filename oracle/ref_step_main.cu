// Test infrastructure: a command-line driver over the reference's OWN FP64 step, built
// from the reference's sources where they lie by oracle/build_ref_step.sh into
// oracle/_ref/ref_step (never shipped, never linked by the library). It produces the
// golden step outputs the oracle and the library are checked against
// (tests/golden/make_ref_step_golden.py turns its output files into fixtures).
//
// It drives the classes exactly as the reference's iteration loop does
// (gpu_flow/code/main.cu:431-454 construction, :612-616 step_time + make_real_signal):
//   Coeff<double>(L); linear_implicit_operator / inverse_B_matrix /
//   nonlinear_operator_rayleigh_noslip ::init_operator; implicit_explicit_step;
//   then per iteration stepper->step_time(state, dt); make_real_signal(state).
// The operator mode calls nonlinear_operator_rayleigh_noslip::calculate_operator once
// (operator/nonlinear_operator_rayleigh_noslip.cu:83-1394) on the given state.
//
// usage: ref_step nx ny L lx ly ra pr dt in.bin out_prefix steps N1,N2,...
//        ref_step nx ny L lx ly ra pr dt in.bin out_prefix operator
// in.bin / out files: theta, f, g as [L][ny][nx/2+1] complex128, then F, G as [L]
// complex128, little-endian, no header. Step mode writes out_prefix_<N>.bin after the
// N-th iteration for each listed N (increasing).
#include "timestepping/implicit_explicit_stepping.h"
#include "util/coeff.h"
#include "util/util.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

static matrix_folder* upload(const CUDA_FLOAT* src, std::vector<int> dims)
{
    matrix_host host(dims);
    std::memcpy(host.get_data(), src, sizeof(CUDA_FLOAT) * host.get_number_of_matrix_entries());
    matrix_device* dev = new matrix_device(&host, matrix_device::Copy);
    matrix_folder* f = new matrix_folder(1);
    f->add_matrix(0, dev);
    return f;
}

static void download(matrix_folder* f, CUDA_FLOAT* dst)
{
    matrix_host host(f->get_matrix(0), matrix_host::Copy);
    std::memcpy(dst, host.get_data(), sizeof(CUDA_FLOAT) * host.get_number_of_matrix_entries());
}

static bool write_state(const std::string& path, matrix_folder** st, size_t nplane, size_t L)
{
    std::vector<CUDA_FLOAT> buf(3 * nplane + 2 * L);
    for (int i = 0; i < 3; ++i) download(st[i], buf.data() + i * nplane);
    download(st[3], buf.data() + 3 * nplane);
    download(st[4], buf.data() + 3 * nplane + L);
    FILE* fp = std::fopen(path.c_str(), "wb");
    if (!fp) return false;
    const size_t n = std::fwrite(buf.data(), sizeof(CUDA_FLOAT), buf.size(), fp);
    std::fclose(fp);
    return n == buf.size();
}

int main(int argc, char** argv)
{
    static_assert(sizeof(CUDA_FLOAT) == 16, "build with -DPRECISION_DOUBLE");
    if (argc < 12) {
        std::fprintf(stderr, "usage: %s nx ny L lx ly ra pr dt in.bin out_prefix steps N1,N2,... | operator\n", argv[0]);
        return 2;
    }
    const int nx = std::atoi(argv[1]), ny = std::atoi(argv[2]), L = std::atoi(argv[3]);
    const double lx = std::atof(argv[4]), ly = std::atof(argv[5]), ra = std::atof(argv[6]), pr = std::atof(argv[7]),
                 dt = std::atof(argv[8]);
    const std::string in = argv[9], prefix = argv[10], mode = argv[11];
    if (nx < 4 || ny < 4 || L < 2 || L > 16 || (nx & 1)) {
        std::fprintf(stderr, "bad sizes\n");
        return 2;
    }
    const size_t mox = nx / 2 + 1, nplane = (size_t)L * ny * mox;
    std::vector<CUDA_FLOAT> buf(3 * nplane + 2 * L);
    {
        FILE* fp = std::fopen(in.c_str(), "rb");
        if (!fp) {
            std::fprintf(stderr, "cannot open %s\n", in.c_str());
            return 2;
        }
        const size_t n = std::fread(buf.data(), sizeof(CUDA_FLOAT), buf.size(), fp);
        std::fclose(fp);
        if (n != buf.size()) {
            std::fprintf(stderr, "%s: expected %zu complex values, read %zu\n", in.c_str(), buf.size(), n);
            return 2;
        }
    }
    std::vector<int> dims(3);
    dims[0] = (int)mox;
    dims[1] = ny;
    dims[2] = L;
    std::vector<int> one(3);
    one[0] = 1;
    one[1] = 1;
    one[2] = L;
    matrix_folder* st[5];
    for (int i = 0; i < 3; ++i) st[i] = upload(buf.data() + i * nplane, dims);
    st[3] = upload(buf.data() + 3 * nplane, one);
    st[4] = upload(buf.data() + 3 * nplane + L, one);
    make_real_signal(st);

    std::vector<CUDA_FLOAT_REAL> clen(3);
    clen[0] = lx;
    clen[1] = ly;
    clen[2] = 1.0;
    Coeff<double> coeff(L);
    nonlinear_operator_rayleigh_noslip* nonlin =
        nonlinear_operator_rayleigh_noslip::init_operator(dims, clen, pr, coeff, 0.0f);

    if (mode == "operator") {
        matrix_folder** out = nonlin->calculate_operator(st[0], st[1], st[2], st[3], st[4]);
        cudaDeviceSynchronize();
        if (cudaGetLastError() != cudaSuccess || !write_state(prefix + "_op.bin", out, nplane, L)) {
            std::fprintf(stderr, "operator failed\n");
            return 1;
        }
        std::printf("wrote %s_op.bin\n", prefix.c_str());
        return 0;
    }
    if (mode != "steps" || argc < 13) {
        std::fprintf(stderr, "mode must be 'steps N1,N2,...' or 'operator'\n");
        return 2;
    }
    std::vector<int> marks;
    for (const char* p = argv[12]; *p;) {
        marks.push_back(std::atoi(p));
        const char* c = std::strchr(p, ',');
        if (!c) break;
        p = c + 1;
    }
    linear_implicit_operator* lin = linear_implicit_operator::init_operator(dims, clen, ra, pr, coeff, dt);
    inverse_B_matrix* invB = inverse_B_matrix::init_operator(dims, clen, pr, coeff);
    implicit_explicit_step* stepper = implicit_explicit_step::init_timestepping(lin, invB, nonlin, dt);
    int done = 0;
    for (int m : marks) {
        if (m < done) {
            std::fprintf(stderr, "step marks must increase\n");
            return 2;
        }
        for (; done < m; ++done) {
            stepper->step_time(st, dt);
            make_real_signal(st);
        }
        cudaDeviceSynchronize();
        if (cudaGetLastError() != cudaSuccess) {
            std::fprintf(stderr, "CUDA error at step %d\n", done);
            return 1;
        }
        const std::string path = prefix + "_" + std::to_string(m) + ".bin";
        if (!write_state(path, st, nplane, L)) {
            std::fprintf(stderr, "cannot write %s\n", path.c_str());
            return 1;
        }
        std::printf("wrote %s\n", path.c_str());
    }
    return 0;
}
