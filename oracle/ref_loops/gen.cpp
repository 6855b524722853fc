// The reference's test problem generators, compiled unchanged with the
// release flags: the channel with a cube
// (examples/common/generator/channel_with_cube.inl + lame.inl; the matrix
// rows in its own entry order and the right-hand sides of its constant and
// divergence forms) and the cube configurations 0-4 (cube.inl).
#include <cstring>

#include "include_ref.h"
#include "ref_loops.h"
#include "generator/channel_with_cube.inl"
#include "generator/cube.inl"

using namespace refloops;

namespace {

struct Channel {
    int scale, const_rhs, nv;
    XAMG::matrix::csr_matrix<double, int, int, int, int> m;
    vector x, b;
    template <int NV> void run() {
        generate_channel_with_cube<double, int, int, int, int, NV>(m, x, b, (uint8_t)scale, const_rhs != 0);
    }
};

struct Cube {
    int64_t nx, ny, nz; int config;
    XAMG::matrix::csr_matrix<double, int, int, int, int> m;
    vector x, b;
    template <int NV> void run() {
        generate_cube<double, int, int, int, int, NV>(m, x, b, (uint64_t)nx, (uint64_t)ny, (uint64_t)nz,
                                                      (size_t)config);
    }
};

}  // namespace

// The last generated problem, kept between the size query and the copy-out
// call so that the (slow: spline metric terms per entry) generator runs once.
static Channel *g_last = nullptr;

extern "C" {
int64_t ref_channel_cube_d(int scale, int const_rhs, int nv, int64_t *nnz, int *rp, int *ci, double *v,
                           double *b) {
    if (scale < 1 || scale > 3) return -1;
    if (!g_last || g_last->scale != scale || g_last->const_rhs != const_rhs || g_last->nv != nv) {
        delete g_last;
        g_last = new Channel{scale, const_rhs, nv, {}, {}, {}};
        if (dispatch_nv(nv, *g_last)) {
            delete g_last;
            g_last = nullptr;
            return -1;
        }
    }
    Channel &f = *g_last;
    const int64_t n = (int64_t)f.m.nrows, z = (int64_t)f.m.nonzeros;
    if (nnz) *nnz = z;
    if (rp) std::memcpy(rp, f.m.row.get_aligned_ptr<int>(), sizeof(int) * (size_t)(n + 1));
    if (ci) std::memcpy(ci, f.m.col.get_aligned_ptr<int>(), sizeof(int) * (size_t)z);
    if (v) std::memcpy(v, f.m.val.get_aligned_ptr<double>(), sizeof(double) * (size_t)z);
    if (b) std::memcpy(b, f.b.get_aligned_ptr<double>(), sizeof(double) * (size_t)(n * nv));
    if (rp || ci || v || b) {
        delete g_last;
        g_last = nullptr;
    }
    return n;
}
int64_t ref_cube_d(int64_t nx, int64_t ny, int64_t nz, int config, int64_t *nnz, int *rp, int *ci,
                   double *v) {
    if (config < 0 || config > 4 || nx < 1 || ny < 1 || nz < 1) return -1;
    Cube f{nx, ny, nz, config, {}, {}, {}};
    f.run<1>();
    const int64_t n = (int64_t)f.m.nrows, z = (int64_t)f.m.nonzeros;
    if (nnz) *nnz = z;
    if (rp) std::memcpy(rp, f.m.row.get_aligned_ptr<int>(), sizeof(int) * (size_t)(n + 1));
    if (ci) std::memcpy(ci, f.m.col.get_aligned_ptr<int>(), sizeof(int) * (size_t)z);
    if (v) std::memcpy(v, f.m.val.get_aligned_ptr<double>(), sizeof(double) * (size_t)z);
    return n;
}
}
