// The reference's binary system reader (src/io/detail/reader.inl), compiled
// unchanged with the release flags, one process.
#include <cstring>
#include <string>

#include "include_ref.h"
#include "ref_loops.h"
#include "io/detail/reader.inl"

using namespace refloops;

namespace {

struct Reader {
    std::string path;
    int nv;
    XAMG::matrix::csr_matrix<double, int, int, int, int> m;
    vector x, b;
    template <int NV> void run() {
        XAMG::io::read_system<XAMG::matrix::csr_matrix<double, int, int, int, int>, NV>(m, x, b, path);
    }
};

}  // namespace

extern "C" {
int64_t ref_read_system_d(const char *path, int nv, int64_t *nnz, int *rp, int *ci, double *v, double *b,
                          double *x) {
    Reader f{path, nv, {}, {}, {}};
    if (dispatch_nv(nv, f)) return -1;
    const int64_t n = (int64_t)f.m.nrows, z = (int64_t)f.m.nonzeros;
    if (nnz) *nnz = z;
    if (rp) std::memcpy(rp, f.m.row.get_aligned_ptr<int>(), sizeof(int) * (size_t)(n + 1));
    if (ci) std::memcpy(ci, f.m.col.get_aligned_ptr<int>(), sizeof(int) * (size_t)z);
    if (v) std::memcpy(v, f.m.val.get_aligned_ptr<double>(), sizeof(double) * (size_t)z);
    if (b) std::memcpy(b, f.b.get_aligned_ptr<double>(), sizeof(double) * (size_t)(n * nv));
    if (x) std::memcpy(x, f.x.get_aligned_ptr<double>(), sizeof(double) * (size_t)(n * nv));
    return n;
}
}
