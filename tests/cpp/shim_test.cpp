// The reference's operator surface over liblamino_b200 (include/lamino_tomocam.hpp),
// compiled against the reference's own polar_grid.h / array.h: the host side a
// maintainer of the reference would run.  Reads the inputs the test wrote into
// <dir> as raw files, runs forward / adjoint / sysmat / gradient / residual,
// the summed normal operator and MBIR1 / MBIR3 through tomocam::gpu, and writes
// each result as <dir>/out_<name>.f32 for tests/test_gpu_cpp_shim.py.
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <tuple>
#include <vector>

#include "polar_grid.h"
#include "lamino_tomocam.hpp"

using tomocam::Array;
using tomocam::dims_t;
using tomocam::PolarGrid;

template <class T>
static std::vector<T> read_raw(const std::string &path) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) throw std::runtime_error("cannot open " + path);
    const std::streamsize n = f.tellg();
    f.seekg(0);
    std::vector<T> v((size_t)n / sizeof(T));
    f.read(reinterpret_cast<char *>(v.data()), n);
    return v;
}

static void write_raw(const std::string &path, const float *p, size_t n) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char *>(p), (std::streamsize)(n * sizeof(float)));
    if (!f) throw std::runtime_error("cannot write " + path);
}

static void write3(const std::string &path, const std::array<Array<float>, 3> &a) {
    std::vector<float> v;
    for (const auto &c : a) v.insert(v.end(), c.begin(), c.begin() + c.size());
    write_raw(path, v.data(), v.size());
}

static std::array<Array<float>, 3> volume(const std::vector<float> &v, const dims_t &d) {
    std::array<Array<float>, 3> a;
    for (int i = 0; i < 3; ++i) {
        a[i] = Array<float>(d);
        std::copy(v.begin() + i * d.size(), v.begin() + (i + 1) * d.size(), a[i].begin());
    }
    return a;
}

static Array<float> projections(const std::vector<float> &v, const dims_t &d) {
    Array<float> a(d);
    std::copy(v.begin(), v.begin() + d.size(), a.begin());
    return a;
}

// the fields of tomocam::ReconParams (include/config.h:146-158) that MBIR reads
struct ReconParams {
    size_t maxIters = 50, innerIters = 3;
    float sigma = 1000.0f, p = 1.2f, lambda = 0.1f, mu = 10.0f, tol = 1e-5f, xtol = 1e-5f, PAD_FACTOR = 1.4142f;
};

int main(int argc, char **argv) {
    if (argc != 2) {
        std::cerr << "usage: shim_test <dir>\n";
        return 2;
    }
    const std::string dir = argv[1];
    try {
        // meta: n1 n2 n3, (nproj nrows ncols) x 2 operator grids, (nproj nrows ncols) x 2 MBIR
        // datasets, MBIR recon n1 n2 n3, MBIR1 iterations, MBIR3 iterations
        const std::vector<int64_t> m = read_raw<int64_t>(dir + "/meta.i64");
        const std::vector<float> gam = read_raw<float>(dir + "/gammas.f32");  // op g0, g1, mbir g0, g1
        const dims_t vd(m[0], m[1], m[2]);
        std::vector<PolarGrid<float>> grids;
        for (int g = 0; g < 2; ++g)
            grids.emplace_back(read_raw<float>(dir + "/angles" + std::to_string(g) + ".f32"), m[4 + 3 * g],
                               m[5 + 3 * g], gam[g]);
        const auto x = volume(read_raw<float>(dir + "/x.f32"), vd);
        const auto yT = volume(read_raw<float>(dir + "/yT.f32"), vd);
        const float yTy = read_raw<float>(dir + "/yTy.f32")[0];
        const Array<float> proj = projections(read_raw<float>(dir + "/proj.f32"), grids[0].dims());

        for (int g = 0; g < 2; ++g) {
            const Array<float> p = tomocam::gpu::forward(x, grids[g], gam[g]);
            write_raw(dir + "/out_forward" + std::to_string(g) + ".f32", p.begin(), p.size());
            write3(dir + "/out_sysmat" + std::to_string(g) + ".f32", tomocam::gpu::sysmat(x, grids[g], gam[g]));
            write3(dir + "/out_gradient" + std::to_string(g) + ".f32",
                   tomocam::gpu::gradient(x, yT, grids[g], gam[g]));
        }
        write3(dir + "/out_adjoint0.f32", tomocam::gpu::adjoint(proj, grids[0], vd, gam[0]));
        const float r = tomocam::gpu::residual(x, yT, grids[0], yTy, gam[0]);
        write_raw(dir + "/out_residual0.f32", &r, 1);
        const tomocam::gpu::Normal A({{&grids[0], gam[0]}, {&grids[1], gam[1]}}, vd);
        write3(dir + "/out_normal.f32", A(x));

        // MBIR1 and MBIR3 on the datasets of the MBIR fixture
        std::vector<std::tuple<Array<float>, std::vector<float>, float>> data;
        for (int g = 0; g < 2; ++g) {
            const dims_t pd(m[9 + 3 * g], m[10 + 3 * g], m[11 + 3 * g]);
            data.emplace_back(projections(read_raw<float>(dir + "/mproj" + std::to_string(g) + ".f32"), pd),
                              read_raw<float>(dir + "/mangles" + std::to_string(g) + ".f32"), gam[2 + g]);
        }
        const dims_t rd(m[15], m[16], m[17]);
        ReconParams p1;
        p1.maxIters = (size_t)m[18];
        p1.innerIters = 2;
        write3(dir + "/out_mbir1.f32", tomocam::gpu::MBIR1(data, rd, p1));
        ReconParams p3;
        p3.maxIters = (size_t)m[19];
        p3.innerIters = 2;
        write3(dir + "/out_mbir3.f32", tomocam::gpu::MBIR3(data, rd, p3));

        // the reference's exception types come back from the status codes
        bool threw = false;
        try {
            const PolarGrid<float> empty(std::vector<float>{}, m[5], m[6], gam[0]);
            tomocam::gpu::forward(x, empty, gam[0]);
        } catch (const std::invalid_argument &) {
            threw = true;
        } catch (const std::exception &e) {
            std::cerr << "unexpected exception type: " << e.what() << "\n";
        }
        std::cout << "invalid_argument on a grid without projections: " << (threw ? "yes" : "no") << "\n";
    } catch (const std::exception &e) {
        std::cerr << "shim_test: " << e.what() << "\n";
        return 1;
    }
    return 0;
}
